"""Elastic force as a torch.autograd.Function with the hand-written adjoint kernels.

forward(u, lambda, mu, X) -> f = dPsi/du (NLAssembler::assemble_gradient,
assembler/Assembler.cpp:574-643), computed by libpfgpu's gradient kernel.

backward(p) returns the vector-Jacobian products of f:
  d(p.f)/dlambda, d(p.f)/dmu : minus the two halves of
      ElasticForceDerivative::force_material_derivative
      (optimization/force_derivatives/ElasticForceDerivative.cpp:91-132), whose
      term carries a leading minus sign (term = -p . df/d(lambda, mu));
  d(p.f)/dX                  : ElasticForceDerivative::force_shape_derivative
      (ElasticForceDerivative.cpp:207-260), which equals +p . df/dX_rest;
  d(p.f)/du                  : H p, the assembled Hessian (structurally and
      numerically symmetric) times p, by the library's own SpMV
      (pfg_hessian_apply): bitwise deterministic.
Each backward term recomputes F and the basis gradients per quadrature point
from (u, lambda, mu, X); nothing from the forward pass is stored on the device
beyond the four inputs.
"""
from __future__ import annotations

import torch

from .assembler import NeoHookeanAssembler


class ElasticForce(torch.autograd.Function):
    """f = grad_u Psi(u; lambda, mu, X) on the GPU, with adjoint backward."""

    @staticmethod
    def forward(ctx, u, lam, mu, X, asm: NeoHookeanAssembler, precision: str = "fp64"):
        for name, t in (("u", u), ("lambda", lam), ("mu", mu), ("X", X)):
            if not (t.is_cuda and t.dtype == torch.float64):
                raise ValueError(f"{name} must be a float64 CUDA tensor")
        u, lam, mu, X = (t.detach().contiguous() for t in (u, lam, mu, X))
        asm.set_lame(lam, mu)
        asm.set_rest_positions(X.reshape(-1))
        f = asm.assemble_gradient(u, precision)
        ctx.save_for_backward(u, lam, mu, X)
        ctx.asm = asm
        ctx.precision = precision
        return f

    @staticmethod
    def backward(ctx, p):
        u, lam, mu, X = ctx.saved_tensors
        asm: NeoHookeanAssembler = ctx.asm
        p = p.detach().contiguous().to(torch.float64)
        # the context may have been re-parameterised by a later forward
        asm.set_lame(lam, mu)
        asm.set_rest_positions(X.reshape(-1))
        g_u = g_lam = g_mu = g_X = None
        if ctx.needs_input_grad[1] or ctx.needs_input_grad[2]:
            term = asm.force_material_derivative(u, p)
            E = asm.n_elements
            g_lam = -term[:E] if ctx.needs_input_grad[1] else None
            g_mu = -term[E:] if ctx.needs_input_grad[2] else None
        if ctx.needs_input_grad[3]:
            g_X = asm.force_shape_derivative(u, p, ctx.precision).reshape(X.shape)
        if ctx.needs_input_grad[0]:
            asm.assemble_hessian_into_context(u, ctx.precision)
            g_u = asm.hessian_apply(p)
        return g_u, g_lam, g_mu, g_X, None, None


def elastic_force(u, lam, mu, X, asm: NeoHookeanAssembler, precision: str = "fp64"):
    """Functional form of ElasticForce.apply."""
    return ElasticForce.apply(u, lam, mu, X, asm, precision)
