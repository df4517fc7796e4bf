"""Dirichlet reduction on the device (NLProblem with the projecting BCLagrangianForm):
reduced Hessian assembled straight into its reduced CSC, reduced gradient and
reduced_to_full, against the oracle's restatement of BCLagrangianForm."""
import numpy as np
import pytest

from oracle.binding import Oracle, project_gradient, project_hessian, reduced_to_full
from polyfem_b200 import NeoHookeanAssembler
from polyfem_b200 import mesh as M

from _cases import make_case, rel_err

pytestmark = pytest.mark.gpu


def constrained_dofs(mesh, seed=0):
    """All dofs of the nodes on the x = 0 face, plus single components of a few
    other nodes (partially constrained nodes)."""
    face = np.flatnonzero(mesh.node_pos[:, 0] <= 1e-12)
    dofs = list((3 * face[:, None] + np.arange(3)).ravel())
    rng = np.random.default_rng(seed)
    others = np.setdiff1d(np.arange(mesh.n_nodes), face)
    for node in rng.choice(others, 5, replace=False):
        dofs.append(3 * node + int(rng.integers(3)))
    return np.array(dofs)


@pytest.mark.parametrize("et,g", [(M.P1_TET, 4), (M.P2_TET, 3), (M.Q1_HEX, 4)], ids=["P1", "P2", "Q1"])
def test_reduced_hessian_gradient_against_oracle(require_gpu, et, g):
    mesh, lam, mu, u, _ = make_case(et, g, seed=12, jitter=0.1 if et != M.P1_TET else 0.0)
    dofs = constrained_dofs(mesh)
    orc = Oracle(mesh, lam, mu)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.set_dirichlet(np.concatenate([dofs, dofs[:3]]))  # duplicates are ignored
    o, i, v = orc.hessian(u)
    ro, ri, rv = project_hessian(o, i, v, dofs)
    assert asm.n_free == mesh.n_dofs - len(np.unique(dofs))
    outer, inner = asm.reduced_pattern()
    assert np.array_equal(outer, ro) and np.array_equal(inner, ri)
    h = asm.assemble_hessian_reduced_values(u, "fp64")
    assert rel_err(h, rv) <= 1e-12
    assert rel_err(asm.assemble_hessian_reduced_values(u, "split32"), rv) <= 1e-6
    _, _, vp = orc.hessian(u, project_psd=True)
    _, _, rvp = project_hessian(o, i, vp, dofs)
    assert rel_err(asm.assemble_hessian_reduced_values(u, "fp64", project_to_psd=True), rvp) <= 1e-11
    gr = asm.assemble_gradient_reduced(u)
    assert rel_err(gr, project_gradient(orc.gradient(u), dofs)) <= 1e-12
    y = np.random.default_rng(1).standard_normal(asm.n_free)
    x_bc = np.random.default_rng(2).standard_normal(mesh.n_dofs)
    assert np.array_equal(asm.reduced_to_full(y, x_bc), reduced_to_full(y, x_bc, dofs))
    # the full Hessian is still available and unchanged
    assert rel_err(asm.assemble_hessian_values(u, "fp64"), v) <= 1e-12
    asm.close()


def test_reduced_device_mode_and_empty_set(require_gpu):
    import torch
    mesh, lam, mu, u, _ = make_case(M.P2_TET, 2, seed=13)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.set_dirichlet([])
    assert asm.n_free == mesh.n_dofs
    o, i = asm.hessian_pattern()
    ro, ri = asm.reduced_pattern()
    assert np.array_equal(o, ro) and np.array_equal(i, ri)
    ud = torch.tensor(u, dtype=torch.float64, device="cuda")
    hd = asm.assemble_hessian_reduced_values(ud, "fp64")
    assert hd.is_cuda
    assert np.array_equal(hd.cpu().numpy(), asm.assemble_hessian_values(u, "fp64"))
    dofs = constrained_dofs(mesh, seed=3)
    asm.set_dirichlet(dofs)
    hd = asm.assemble_hessian_reduced_values(ud, "fp64")
    assert np.array_equal(hd.cpu().numpy(), asm.assemble_hessian_reduced_values(u, "fp64"))
    gd = asm.assemble_gradient_reduced(ud)
    assert np.array_equal(gd.cpu().numpy(), asm.assemble_gradient_reduced(u))
    asm.close()


def test_reduction_argument_checks(require_gpu):
    import ctypes

    from polyfem_b200 import _lib
    L = _lib.lib()
    mesh, lam, mu, u, _ = make_case(M.P1_TET, 2, seed=14)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    h = asm.handle
    n = ctypes.c_int()
    nnz = ctypes.c_longlong()
    # before any Dirichlet set: state errors
    assert L.pfg_reduced_pattern(h, ctypes.byref(n), ctypes.byref(nnz)) == 5
    ub = np.ascontiguousarray(u)
    out = np.empty(mesh.n_dofs)
    assert L.pfg_hessian_reduced(h, ctypes.c_void_p(ub.ctypes.data), 0, 0, 0, None) == 5
    assert L.pfg_gradient_reduced(h, ctypes.c_void_p(ub.ctypes.data), 0, 0, ctypes.c_void_p(out.ctypes.data)) == 5
    # out-of-range and negative dofs are rejected
    bad = np.array([0, mesh.n_dofs], dtype=np.int32)
    assert L.pfg_set_dirichlet(h, ctypes.c_void_p(bad.ctypes.data), 2) == 1
    bad = np.array([-1], dtype=np.int32)
    assert L.pfg_set_dirichlet(h, ctypes.c_void_p(bad.ctypes.data), 1) == 1
    assert L.pfg_set_dirichlet(h, None, 3) == 1
    assert L.pfg_set_dirichlet(None, None, 0) == 1
    # all dofs constrained: empty reduced system
    asm.set_dirichlet(np.arange(mesh.n_dofs))
    assert asm.n_free == 0
    outer, inner = asm.reduced_pattern()
    assert list(outer) == [0] and inner.size == 0
    assert asm.assemble_hessian_reduced_values(u).size == 0
    asm.close()
