"""Mass matrix (pfg_mass_matrix; MassMatrixAssembler = LinearAssembler + Mass term)
against the oracle's restatement, which integrates with its own quadrature."""
import numpy as np
import pytest

from oracle.binding import Oracle
from polyfem_b200 import NeoHookeanAssembler
from polyfem_b200 import mesh as M

from _cases import make_case, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("et,g", [(M.P1_TET, 3), (M.P2_TET, 2), (M.Q1_HEX, 3)], ids=["P1", "P2", "Q1"])
def test_mass_matrix_matches_oracle(require_gpu, et, g):
    import torch
    mesh, lam, mu, u, _ = make_case(et, g, seed=11, jitter=0.1 if et != M.P1_TET else 0.0)
    rho = np.exp(np.random.default_rng(12).normal(np.log(1000.0), 0.3, mesh.n_elements))
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    orc = Oracle(mesh, lam, mu)
    outer, inner, vals = orc.mass_matrix(rho)
    go, gi = asm.hessian_pattern()
    assert np.array_equal(go, outer) and np.array_equal(gi, inner)
    v = asm.assemble_mass_matrix_values(rho)
    assert rel_err(v, vals) <= 1e-13
    vd = asm.assemble_mass_matrix_values(torch.tensor(rho, device="cuda")).cpu().numpy()
    assert np.array_equal(v, vd)
    assert np.array_equal(v, asm.assemble_mass_matrix_values(rho))  # deterministic
    _, _, v1 = orc.mass_matrix()
    assert rel_err(asm.assemble_mass_matrix_values(), v1) <= 1e-13
    # the mass matrix does not disturb the Hessian kept in the context
    h1 = asm.assemble_hessian_values(u)
    asm.assemble_mass_matrix_values(rho)
    assert np.array_equal(asm.assemble_hessian_values(u), h1)
    # total mass of a unit-density cube (x components)
    Mm = asm.assemble_mass_matrix()
    ex = np.zeros(mesh.n_dofs)
    ex[0::3] = 1.0
    assert abs(ex @ (Mm @ ex) - 1.0) <= 1e-12
    asm.close()


@pytest.mark.parametrize("et,g", [(M.P1_TET, 3), (M.P2_TET, 2), (M.Q1_HEX, 3)], ids=["P1", "P2", "Q1"])
def test_lump_matrix_matches_oracle(require_gpu, et, g):
    """pfg_lump_matrix (utils::lump_matrix) bit-exact against the oracle's restatement
    on the same values, including values whose row sums depend on the summation
    order; the lumped mass within the mass matrix's bound, and its total mass."""
    import torch
    from oracle.binding import lump_matrix
    mesh, lam, mu, u, _ = make_case(et, g, seed=13, jitter=0.1 if et != M.P1_TET else 0.0)
    rho = np.exp(np.random.default_rng(14).normal(np.log(1000.0), 0.3, mesh.n_elements))
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    orc = Oracle(mesh, lam, mu)
    outer, inner, mvals = orc.mass_matrix(rho)
    # wide dynamic range and both signs: any other summation order changes bits
    rng = np.random.default_rng(15)
    wild = rng.normal(size=asm.hessian_nnz()) * 10.0 ** rng.uniform(-8, 8, asm.hessian_nnz())
    for vals in (mvals, wild):
        ref = lump_matrix(outer, inner, vals)
        got = asm.lump_matrix(vals)
        assert np.array_equal(got, ref)
        got_d = asm.lump_matrix(torch.tensor(vals, device="cuda")).cpu().numpy()
        assert np.array_equal(got_d, ref)
    lm = asm.assemble_lumped_mass(rho)
    ref = lump_matrix(outer, inner, mvals)
    assert rel_err(lm, ref) <= 1e-13
    vol_rho = float(np.asarray(asm.assemble_mass_matrix(rho).sum()))  # 3 * sum_e rho_e |e|
    assert abs(lm.sum() - vol_rho) <= 1e-12 * abs(vol_rho)
    assert np.all(lm[0::3] == lm[1::3]) and np.all(lm[0::3] == lm[2::3])  # rho I blocks
    asm.close()


def test_lump_matrix_edges(require_gpu):
    """Wrong-length values raise; nodes of no element have no row entry: 0."""
    mesh, lam, mu, u, _ = make_case(M.P1_TET, 2, seed=16)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    with pytest.raises(ValueError):
        asm.lump_matrix(np.zeros(asm.hessian_nnz() + 1))
    asm.close()
    empty = NeoHookeanAssembler(M.P1_TET, np.zeros((0, 4), dtype=np.int32), np.zeros((5, 3)), np.zeros(0),
                                np.zeros(0), n_nodes=5)
    d = empty.lump_matrix(np.zeros(empty.hessian_nnz()))
    assert d.shape == (15,) and np.all(d == 0.0)
    empty.close()
