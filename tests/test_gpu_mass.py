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
