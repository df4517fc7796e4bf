"""Sparse direct solve on the device (pfg_direct_*, polyfem_b200.DirectSolver): the
factorisation polysolve's direct choices compute for the Newton system, run on the
Hessian the assembler left on the GPU.  Checked against scipy's SuperLU solve of
the same matrix and by the residual; the factor and solution are bitwise
deterministic."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from polyfem_b200 import DirectSolver, NeoHookeanAssembler, PfgError
from polyfem_b200 import mesh as M
from polyfem_b200._lib import PFG_ERR_NUMERIC, PFG_ERR_STATE

from _cases import make_case, rel_err

pytestmark = pytest.mark.gpu

CASES = [(M.P1_TET, 3), (M.P2_TET, 2), (M.Q1_HEX, 3), (M.P1_TET, 8), (M.P2_TET, 5), (M.Q1_HEX, 7)]


def reduced_system(et, g, seed=3):
    """Dirichlet-reduced (x = 0 face fixed), PSD-projected Hessian of a compressed
    state: symmetric positive definite."""
    mesh, lam, mu, u, _ = make_case(et, g, seed=seed, jitter=0.1 if et != M.P1_TET else 0.0)
    rng = np.random.default_rng(seed + 1)
    u = (-0.2 * mesh.node_pos + 0.02 * mesh.h * rng.standard_normal(mesh.node_pos.shape)).ravel()
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    face = np.flatnonzero(mesh.node_pos[:, 0] <= 1e-12)
    asm.set_dirichlet((3 * face[:, None] + np.arange(3)).ravel())
    H = asm.assemble_hessian_reduced(u, "fp64", project_to_psd=True)  # values stay in the context
    g_red = asm.assemble_gradient_reduced(u, "fp64")
    return mesh, asm, u, H, g_red


@pytest.mark.parametrize("et,g", CASES, ids=["P1-3", "P2-2", "Q1-3", "P1-8", "P2-5", "Q1-7"])
def test_reduced_solve_matches_superlu(require_gpu, et, g):
    mesh, asm, u, H, grad = reduced_system(et, g)
    b = -grad
    ds = DirectSolver(asm, "reduced")
    ds.analyze_pattern(H, H.shape[0])
    info = ds.get_info()
    assert info["n"] == H.shape[0] and info["fronts"] >= 1
    assert info["nnz_L"] >= (H.nnz + H.shape[0]) // 2  # L holds A's lower triangle
    ds.factorize()
    x = ds.solve(b)
    res = np.linalg.norm(b - H @ x) / np.linalg.norm(b)
    assert res <= 1e-12, res
    xd = spla.spsolve(H.tocsc(), b)
    assert rel_err(x, xd) <= 1e-10
    asm.close()


def test_medium_system_residual(require_gpu):
    """P2 12^3 (about 45k free dofs, fronts up to ~3,900): the residual of the
    device solve, checked with a host sparse product."""
    mesh, asm, u, H, grad = reduced_system(M.P2_TET, 12)
    ds = DirectSolver(asm, "reduced")
    ds.analyze_pattern()
    ds.factorize()
    b = -grad
    x = ds.solve(b)
    assert np.linalg.norm(b - H @ x) / np.linalg.norm(b) <= 1e-11
    asm.close()


def test_deterministic_device_and_host_mode(require_gpu):
    import torch
    mesh, asm, u, H, grad = reduced_system(M.P2_TET, 3)
    ds = DirectSolver(asm, "reduced")
    ds.analyze_pattern()
    ds.factorize()
    xh = ds.solve(-grad)
    bd = torch.tensor(-grad, dtype=torch.float64, device="cuda")
    x1 = ds.solve(bd).cpu().numpy()
    ds.factorize()  # a second factorisation of the same values
    x2 = ds.solve(bd).cpu().numpy()
    assert np.array_equal(x1, x2)
    assert np.array_equal(x1, xh)
    # in place: x aliases b
    bd2 = bd.clone()
    ds.solve(bd2, bd2)
    assert np.array_equal(bd2.cpu().numpy(), x1)
    asm.close()


def test_caller_values_and_not_positive_definite(require_gpu):
    """Caller values (device memory) replace the context's: H + s I on the full
    (singular) system solves; -H on the reduced system is refused with
    PFG_ERR_NUMERIC, after which the solver needs a successful factorisation."""
    import torch
    mesh, lam, mu, u, _ = make_case(M.P1_TET, 3, seed=5)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    H = asm.assemble_hessian(u, "fp64", project_to_psd=True).tocsc()
    H.sort_indices()
    s = 1e-3 * abs(H.diagonal()).max()
    A = (H + s * sp.identity(H.shape[0], format="csc")).tocsc()
    A.sort_indices()
    assert np.array_equal(A.indptr, H.indptr) and np.array_equal(A.indices, H.indices)
    ds = DirectSolver(asm, "full")
    ds.analyze_pattern()
    vals = torch.tensor(A.data, dtype=torch.float64, device="cuda")
    ds.factorize(vals)
    b = np.random.default_rng(1).standard_normal(H.shape[0])
    x = ds.solve(b)
    assert rel_err(x, spla.spsolve(A, b)) <= 1e-10
    with pytest.raises(PfgError) as ei:
        ds.factorize(-vals)
    assert ei.value.status == PFG_ERR_NUMERIC
    with pytest.raises(PfgError) as ei:
        ds.solve(b)
    assert ei.value.status == PFG_ERR_STATE
    ds.factorize(vals)
    assert np.array_equal(ds.solve(b), x)
    asm.close()


def test_state_errors(require_gpu):
    mesh, asm, u, H, grad = reduced_system(M.P1_TET, 3)
    ds = DirectSolver(asm, "reduced")
    with pytest.raises(PfgError) as ei:
        ds.factorize()
    assert ei.value.status == PFG_ERR_STATE
    ds.analyze_pattern()
    ds.factorize()
    x = ds.solve(-grad)
    # a new Dirichlet set changes the reduced pattern: the analysis is discarded
    face = np.flatnonzero(mesh.node_pos[:, 0] <= 1e-12)
    asm.set_dirichlet((3 * face[:, None] + np.arange(3)).ravel())
    with pytest.raises(PfgError) as ei:
        ds.solve(-grad)
    assert ei.value.status == PFG_ERR_STATE
    H2 = asm.assemble_hessian_reduced(u, "fp64", project_to_psd=True)
    ds.analyze_pattern()
    ds.factorize()
    assert np.array_equal(ds.solve(-grad), x)
    with pytest.raises(ValueError):
        ds.solve(np.zeros(H2.shape[0] + 1))
    # released: the factor is gone until the next analysis
    ds.free()
    with pytest.raises(PfgError) as ei:
        ds.solve(-grad)
    assert ei.value.status == PFG_ERR_STATE
    ds.analyze_pattern()
    ds.factorize()
    assert np.array_equal(ds.solve(-grad), x)
    asm.close()


def test_newton_step_direct_equals_cg(require_gpu):
    """One Newton step of NLProblem with the direct solve: the step agrees with the
    tight CG solve of the same system (to the CG residual times the condition)."""
    from polyfem_b200 import ConjugateGradient
    mesh, asm, u, H, grad = reduced_system(M.Q1_HEX, 4)
    ds = DirectSolver(asm, "reduced")
    ds.analyze_pattern()
    ds.factorize()
    xd = ds.solve(-grad)
    cg = ConjugateGradient(asm, "reduced")
    cg.set_parameters({"tolerance": 1e-13, "max_iter": 20000})
    xc = cg.solve(-grad)
    assert rel_err(xd, xc) <= 1e-7
    asm.close()
