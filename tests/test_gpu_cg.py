"""Device conjugate gradient (pfg_cg_solve, polyfem_b200.ConjugateGradient): the
linear solve NewtonMethod makes after every assembly, run on the Hessian the
assembler left on the GPU.  Checked against the oracle's restatement of Eigen's
ConjugateGradient with the diagonal preconditioner on the same matrix, and
against a direct solve."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle.binding import conjugate_gradient
from polyfem_b200 import ConjugateGradient, NeoHookeanAssembler, PfgError
from polyfem_b200 import mesh as M
from polyfem_b200._lib import PFG_MEM_HOST, lib

from _cases import make_case, rel_err

pytestmark = pytest.mark.gpu

CASES = [(M.P1_TET, 3), (M.P2_TET, 2), (M.Q1_HEX, 3)]


def reduced_system(et, g, seed=3, compress=True):
    """Dirichlet-reduced (x = 0 face fixed), PSD-projected Hessian: symmetric positive definite."""
    mesh, lam, mu, u, _ = make_case(et, g, seed=seed, jitter=0.1 if et != M.P1_TET else 0.0)
    if compress:
        rng = np.random.default_rng(seed + 1)
        u = (-0.2 * mesh.node_pos + 0.02 * mesh.h * rng.standard_normal(mesh.node_pos.shape)).ravel()
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    face = np.flatnonzero(mesh.node_pos[:, 0] <= 1e-12)
    asm.set_dirichlet((3 * face[:, None] + np.arange(3)).ravel())
    H = asm.assemble_hessian_reduced(u, "fp64", project_to_psd=True)  # host mode: values stay in the context
    g_red = asm.assemble_gradient_reduced(u, "fp64")
    return mesh, asm, u, H, g_red


@pytest.mark.parametrize("et,g", CASES, ids=["P1", "P2", "Q1"])
def test_reduced_solve_matches_oracle_and_direct(require_gpu, et, g):
    mesh, asm, u, H, grad = reduced_system(et, g)
    b = -grad
    cg = ConjugateGradient(asm, "reduced")
    cg.set_parameters({"tolerance": 1e-11, "max_iter": 5000})
    cg.analyze_pattern(H, H.shape[0])
    cg.factorize()
    x = cg.solve(b)
    info = cg.get_info()
    xo, it_o, res_o = conjugate_gradient(H.indptr, H.indices, H.data, b, 1e-11, 5000)
    # same iteration up to the rounding of the dot products (tree vs sequential order)
    assert abs(info["solver_iter"] - it_o) <= max(2, it_o // 50), (info, it_o)
    assert info["solver_error"] < 1e-11 and res_o < 1e-11
    res = np.linalg.norm(b - H @ x) / np.linalg.norm(b)
    assert res <= 2e-11 and abs(res - info["solver_error"]) <= 1e-11
    xd = spla.spsolve(H.tocsc(), b)
    assert rel_err(x, xd) <= 1e-8
    assert rel_err(x, xo) <= 1e-8
    asm.close()


def test_device_mode_deterministic_and_equal_to_host_mode(require_gpu):
    import torch
    mesh, asm, u, H, grad = reduced_system(M.P2_TET, 2)
    cg = ConjugateGradient(asm, "reduced")
    cg.set_parameters({"tolerance": 1e-10, "max_iter": 2000})
    xh = cg.solve(-grad)
    bd = torch.tensor(-grad, dtype=torch.float64, device="cuda")
    x1 = cg.solve(bd).cpu().numpy()
    x2 = cg.solve(bd).cpu().numpy()
    assert np.array_equal(x1, x2)
    assert np.array_equal(x1, xh)
    asm.close()


def test_caller_values_on_the_full_system(require_gpu):
    """The full Hessian is singular (rigid motions); a caller-supplied values array
    H + s I (device memory) takes the context's place."""
    import torch
    mesh, lam, mu, u, _ = make_case(M.P1_TET, 3, seed=5)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    vals = asm.assemble_hessian_values(u, "fp64", project_to_psd=True)
    outer, inner = asm.hessian_pattern()
    n = asm.n_dofs
    cols = np.repeat(np.arange(n), np.diff(outer))
    shift = 1e-3 * np.abs(vals).max()
    vals_s = vals.copy()
    vals_s[inner == cols] += shift
    A = sp.csc_matrix((vals_s, inner, outer), shape=(n, n))
    b = np.random.default_rng(2).standard_normal(n)
    cg = ConjugateGradient(asm, "full")
    cg.set_parameters({"tolerance": 1e-12, "max_iter": 5000})
    cg.factorize(torch.tensor(vals_s, device="cuda"))
    x = cg.solve(b)
    assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) <= 2e-12
    xo, it_o, _ = conjugate_gradient(outer, inner, vals_s, b, 1e-12, 5000)
    assert abs(cg.get_info()["solver_iter"] - it_o) <= max(2, it_o // 50)
    assert rel_err(x, xo) <= 1e-9
    asm.close()


def test_guess_zero_rhs_and_iteration_cap(require_gpu):
    mesh, asm, u, H, grad = reduced_system(M.P1_TET, 3)
    b = -grad
    cg = ConjugateGradient(asm, "reduced")
    cg.set_parameters({"tolerance": 1e-10, "max_iter": 3000})
    x = cg.solve(b)
    # starting from the solution: converged before the first iteration
    x2 = x.copy()
    cg.solve(b, x2, guess=True)
    assert cg.get_info()["solver_iter"] == 0 and np.array_equal(x2, x)
    # b = 0: x = 0 without iterating, whatever the guess
    xz = np.ones_like(b)
    cg.solve(np.zeros_like(b), xz, guess=True)
    assert cg.get_info() == {"solver_iter": 0, "solver_error": 0.0} and not xz.any()
    # the iteration cap is reached and reported through the residual, not as an error
    cg.set_parameters({"max_iter": 3})
    cg.solve(b)
    info = cg.get_info()
    assert info["solver_iter"] == 3 and info["solver_error"] > 1e-10
    _, it_o, res_o = conjugate_gradient(H.indptr, H.indices, H.data, b, 1e-10, 3)
    assert it_o == 3 and abs(info["solver_error"] - res_o) <= 1e-9 * res_o
    asm.close()


def test_newton_step_is_a_descent_direction(require_gpu):
    """dx = -H^-1 g with the projected reduced Hessian: g.dx < 0 and the energy drops
    along dx (the step NewtonMethod takes)."""
    mesh, asm, u, H, grad = reduced_system(M.P2_TET, 2)
    cg = ConjugateGradient(asm, "reduced")
    cg.set_parameters({"tolerance": 1e-10, "max_iter": 3000})
    dx = cg.solve(-grad)
    assert grad @ dx < 0
    du = asm.reduced_to_full(dx, np.zeros(asm.n_dofs))
    e0 = asm.assemble_energy(u)
    e1 = asm.assemble_energy(u + 1e-3 * du)
    assert e1 < e0
    asm.close()


def test_argument_and_state_errors(require_gpu):
    mesh, lam, mu, u, _ = make_case(M.P1_TET, 2, seed=1)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    L = lib()
    b = np.zeros(asm.n_dofs)
    x = np.zeros(asm.n_dofs)
    bp, xp = ctypes.c_void_p(b.ctypes.data), ctypes.c_void_p(x.ctypes.data)
    it, res = ctypes.c_int(), ctypes.c_double()
    args = (bp, PFG_MEM_HOST, 1e-10, 100, 0, xp, ctypes.byref(it), ctypes.byref(res))
    assert L.pfg_cg_solve(asm.handle, 7, None, *args) == 1               # PFG_ERR_INVALID: no such system
    assert L.pfg_cg_solve(asm.handle, 1, None, *args) == 5               # PFG_ERR_STATE: no Dirichlet set
    assert L.pfg_cg_solve(asm.handle, 0, None, bp, PFG_MEM_HOST, -1.0, 100, 0, xp, None, None) == 1
    with pytest.raises(PfgError):
        ConjugateGradient(asm, "reduced").solve(np.zeros(0))
    asm.close()
