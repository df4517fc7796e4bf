"""Hessian with project_to_psd (Assembler.cpp:693-694 -> ipc::project_to_psd, CLAMP):
the GPU projection against the oracle's restatement, on compressed meshes where
every element matrix is indefinite."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle.binding import Oracle
from polyfem_b200 import ElasticForm, NeoHookeanAssembler
from polyfem_b200 import mesh as M

from _cases import make_case, rel_err

pytestmark = pytest.mark.gpu

CASES = [(M.P1_TET, 3), (M.P2_TET, 2), (M.Q1_HEX, 3)]


def compressed(et, g, seed=5):
    """30% uniform compression plus noise: NeoHookean element Hessians are indefinite."""
    mesh, lam, mu, _, _ = make_case(et, g, seed=seed, jitter=0.1 if et != M.P1_TET else 0.0)
    rng = np.random.default_rng(seed + 1)
    u = (-0.3 * mesh.node_pos + 0.02 * mesh.h * rng.standard_normal(mesh.node_pos.shape)).ravel()
    return mesh, lam, mu, u


@pytest.mark.parametrize("et,g", CASES, ids=["P1", "P2", "Q1"])
def test_projected_hessian_matches_oracle(require_gpu, et, g):
    mesh, lam, mu, u = compressed(et, g)
    orc = Oracle(mesh, lam, mu)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    o, i, v_psd = orc.hessian(u, project_psd=True)
    _, _, v_raw = orc.hessian(u, project_psd=False)
    assert rel_err(v_psd, v_raw) > 1e-3  # the projection changes this matrix
    outer, inner = asm.hessian_pattern()
    assert np.array_equal(outer, o) and np.array_equal(inner, i)
    g64 = asm.assemble_hessian_values(u, "fp64", project_to_psd=True)
    assert rel_err(g64, v_psd) <= 1e-11
    assert np.array_equal(g64, asm.assemble_hessian_values(u, "fp64", project_to_psd=True))
    gs = asm.assemble_hessian_values(u, "split32", project_to_psd=True)
    assert rel_err(gs, v_psd) <= 1e-6
    # without the flag the plain Hessian comes back
    assert rel_err(asm.assemble_hessian_values(u, "fp64"), v_raw) <= 1e-12
    # a sum of PSD element matrices is PSD
    n = mesh.n_dofs
    H = sp.csc_matrix((g64, inner, outer), shape=(n, n)).toarray()
    w = np.linalg.eigvalsh(0.5 * (H + H.T))
    assert w.min() >= -1e-10 * np.abs(w).max()
    asm.close()


@pytest.mark.parametrize("et,g", CASES, ids=["P1", "P2", "Q1"])
def test_psd_elements_are_left_unchanged(require_gpu, et, g):
    """At the rest state every element matrix is the PSD linear-elastic stiffness
    (its rigid motions are exact null vectors), so the projection changes values
    at rounding level only."""
    mesh, lam, mu, _, _ = make_case(et, g, seed=9, jitter=0.1 if et != M.P1_TET else 0.0)
    u = np.zeros(mesh.n_dofs)
    orc = Oracle(mesh, lam, mu)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    _, _, v_raw = orc.hessian(u)
    g = asm.assemble_hessian_values(u, "fp64", project_to_psd=True)
    assert rel_err(g, v_raw) <= 1e-12
    asm.close()


def test_elastic_form_project_to_psd_flag(require_gpu):
    mesh, lam, mu, u = compressed(M.P1_TET, 3, seed=7)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    form = ElasticForm(asm)
    form.set_project_to_psd(True)
    H = form.second_derivative(u)
    _, _, v_psd = Oracle(mesh, lam, mu).hessian(u, project_psd=True)
    assert rel_err(H.data, v_psd) <= 1e-11
    asm.close()


def test_projection_keeps_nan_of_inverted_elements(require_gpu):
    """An inverted element (J <= 0) has NaN entries (log J); the projection leaves
    them alone, so the NaN still reaches the assembled matrix as in the reference."""
    mesh, lam, mu, u, _ = make_case(M.P1_TET, 2, seed=15)
    u = u.copy()
    # collapse element 0 through its first node
    n0 = mesh.conn[0, 0]
    c = mesh.node_pos[mesh.conn[0]].mean(axis=0)
    u[3 * n0:3 * n0 + 3] = 2.5 * (c - mesh.node_pos[n0])
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    plain = asm.assemble_hessian_values(u, "fp64")
    proj = asm.assemble_hessian_values(u, "fp64", project_to_psd=True)
    assert np.isnan(plain).any()
    assert np.array_equal(np.isnan(plain), np.isnan(proj))
    asm.close()
