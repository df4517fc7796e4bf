"""Other materials of the GenericElastic family on the GPU (pfg_set_material):
IsochoricNeoHookean and isotropic SaintVenant, FP64 energy, gradient and Hessian
(with project_to_psd and the Dirichlet reduction) against the oracle's
restatement (autodiff of psi(F), as the reference's GenericElastic does)."""
import ctypes

import numpy as np
import pytest

from oracle.binding import Oracle, project_hessian
from polyfem_b200 import NeoHookeanAssembler, PfgError
from polyfem_b200 import mesh as M
from polyfem_b200._lib import lib

from _cases import make_case, rel_err

pytestmark = pytest.mark.gpu

MATS = ["IsochoricNeoHookean", "SaintVenant"]
ELEMS = [(M.P1_TET, 3), (M.P2_TET, 2), (M.Q1_HEX, 3)]


def setup(et, g, mat, seed=3, disp=0.05):
    mesh, lam, mu, u, p = make_case(et, g, seed=seed, jitter=0.1 if et != M.P1_TET else 0.0, disp_scale=disp)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.set_material(mat)
    return mesh, asm, Oracle(mesh, lam, mu, material=mat), u, p


@pytest.mark.parametrize("mat", MATS)
@pytest.mark.parametrize("et,g", ELEMS, ids=["P1", "P2", "Q1"])
def test_energy_gradient_hessian_match_oracle(require_gpu, mat, et, g):
    mesh, asm, orc, u, _ = setup(et, g, mat)
    assert abs(asm.assemble_energy(u) - orc.energy(u)) <= 1e-12 * abs(orc.energy(u))
    assert rel_err(asm.assemble_energy_per_element(u), orc.energy_per_element(u)) <= 1e-12
    assert rel_err(asm.assemble_gradient(u), orc.gradient(u)) <= 1e-12
    outer, inner, vals = orc.hessian(u)
    o2, i2 = asm.hessian_pattern()
    assert np.array_equal(o2, outer) and np.array_equal(i2, inner)
    v = asm.assemble_hessian_values(u, "fp64")
    assert rel_err(v, vals) <= 1e-12
    assert np.array_equal(v, asm.assemble_hessian_values(u, "fp64"))  # deterministic
    asm.close()


@pytest.mark.parametrize("mat", MATS)
def test_projected_and_reduced_hessian(require_gpu, mat):
    mesh, asm, orc, _, _ = setup(M.P2_TET, 2, mat, seed=5)
    rng = np.random.default_rng(6)
    u = (-0.25 * mesh.node_pos + 0.02 * mesh.h * rng.standard_normal(mesh.node_pos.shape)).ravel()
    outer, inner, v_psd = orc.hessian(u, project_psd=True)
    _, _, v_raw = orc.hessian(u)
    assert rel_err(v_psd, v_raw) > 1e-6  # the projection changes this matrix
    assert rel_err(asm.assemble_hessian_values(u, "fp64", project_to_psd=True), v_psd) <= 1e-11
    face = np.flatnonzero(mesh.node_pos[:, 0] <= 1e-12)
    dofs = (3 * face[:, None] + np.arange(3)).ravel()
    asm.set_dirichlet(dofs)
    ro, ri, rv = project_hessian(outer, inner, v_raw, dofs)
    go, gi = asm.reduced_pattern()
    assert np.array_equal(go, ro) and np.array_equal(gi, ri)
    assert rel_err(asm.assemble_hessian_reduced_values(u, "fp64"), rv) <= 1e-12
    assert rel_err(asm.assemble_gradient_reduced(u, "fp64"), np.delete(orc.gradient(u), np.unique(dofs))) <= 1e-12
    asm.close()


def test_material_switch_and_unsupported_calls(require_gpu):
    mesh, lam, mu, u, p = make_case(M.P1_TET, 2, seed=7)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    e_nh = asm.assemble_energy(u)
    asm.set_material("SaintVenant")
    assert abs(asm.assemble_energy(u) - Oracle(mesh, lam, mu, material="SaintVenant").energy(u)) <= 1e-12 * abs(e_nh)
    for call in (lambda: asm.assemble_energy(u, "fp32"), lambda: asm.assemble_hessian_values(u, "split32"),
                 lambda: asm.force_material_derivative(u, p), lambda: asm.force_shape_derivative(u, p)):
        with pytest.raises(PfgError) as ei:
            call()
        assert ei.value.status == 4  # PFG_ERR_UNSUPPORTED
    assert lib().pfg_set_material(asm.handle, 12) == 1  # PFG_ERR_INVALID
    asm.set_material("NeoHookean")
    assert asm.assemble_energy(u) == e_nh  # back on the NeoHookean path, bit for bit
    with pytest.raises(ValueError):
        asm.set_material("Ogden")
    asm.close()
