"""B200-native NeoHookean assembly (energy, gradient, Hessian, adjoint VJPs) for PolyFEM.

The compute path is the CUDA library ``libpfgpu.so`` (C ABI in include/pfgpu.h);
this package is its host-side mirror of PolyFEM's NLAssembler / ElasticForm API.
``polyfem_b200.autograd`` (imported on demand, it needs torch) wraps the gradient
and the adjoint kernels as a torch.autograd.Function; ``ConjugateGradient`` and
``DirectSolver`` (sparse Cholesky) solve with the assembled Hessian on the device.
"""
from . import mesh
from ._lib import PfgError, build, lib
from .assembler import ElasticForceDerivative, ElasticForm, NeoHookeanAssembler
from .linear_solver import ConjugateGradient, DirectSolver, direct_symbolic

__all__ = ["mesh", "build", "lib", "PfgError", "NeoHookeanAssembler", "ElasticForm", "ElasticForceDerivative",
           "ConjugateGradient", "DirectSolver", "direct_symbolic"]
