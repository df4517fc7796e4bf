"""Meshes whose elements and nodes are numbered at random (no locality, no
first-touch order): every operation against the oracle on the renumbered mesh,
and invariance of the results under the renumbering."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle.binding import Oracle
from polyfem_b200 import NeoHookeanAssembler
from polyfem_b200 import mesh as M

from _cases import make_case, permuted, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("et,g", [(M.P1_TET, 4), (M.P2_TET, 3), (M.Q1_HEX, 4)], ids=["P1", "P2", "Q1"])
def test_random_numbering(require_gpu, et, g):
    mesh, lam, mu, u, p = make_case(et, g, seed=19, jitter=0.1 if et != M.P1_TET else 0.0)
    m2, u2, pn, pe = permuted(mesh, u, seed=5)
    lam2, mu2 = lam[pe], mu[pe]
    orc = Oracle(m2, lam2, mu2)
    asm = NeoHookeanAssembler.from_mesh(m2, lam2, mu2)
    # parity on the renumbered mesh
    assert abs(asm.assemble_energy(u2) - orc.energy(u2)) <= 1e-12 * abs(orc.energy(u2))
    g2 = asm.assemble_gradient(u2)
    assert rel_err(g2, orc.gradient(u2)) <= 1e-12
    o, i, v = orc.hessian(u2)
    outer, inner = asm.hessian_pattern()
    assert np.array_equal(outer, o) and np.array_equal(inner, i)
    h2 = asm.assemble_hessian_values(u2, "fp64")
    assert rel_err(h2, v) <= 1e-12
    assert rel_err(asm.assemble_hessian_values(u2, "split32"), v) <= 1e-6
    p2 = np.empty_like(p)
    p2.reshape(-1, 3)[pn] = p.reshape(-1, 3)
    assert rel_err(asm.force_material_derivative(u2, p2), orc.material_vjp(u2, p2)) <= 1e-12
    assert rel_err(asm.force_shape_derivative(u2, p2), orc.shape_vjp(u2, p2)) <= 1e-12
    # invariance: the same physics as the original numbering
    asm0 = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    e0 = asm0.assemble_energy(u)
    assert abs(asm.assemble_energy(u2) - e0) <= 1e-12 * abs(e0)
    assert rel_err(g2.reshape(-1, 3)[pn], asm0.assemble_gradient(u).reshape(-1, 3)) <= 1e-12
    H0 = asm0.assemble_hessian(u)
    H2 = sp.csc_matrix((h2, inner, outer), shape=H0.shape)
    dof = (3 * pn[:, None] + np.arange(3)).ravel()  # old dof k -> new dof dof[k]
    assert abs(H2[dof][:, dof] - H0).max() <= 1e-12 * abs(H0).max()
    asm0.close()
    asm.close()
