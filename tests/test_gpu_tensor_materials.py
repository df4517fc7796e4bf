"""The elasticity-tensor formulations on the GPU (pfg_materials.cu):
HookeLinearElasticity and SaintVenant with one anisotropic elasticity tensor
(pfg_set_elasticity_tensor), FP64 energy, gradient and Hessian against the oracle's
restatement (HookeLinearElasticity.cpp:372-421, SaintVenantElasticity.cpp:209-267,
ElasticityTensor::compute_stress), and their isotropic limits against
LinearElasticity and the lambda/mu SaintVenant."""
import numpy as np
import pytest

from oracle.binding import Oracle
from polyfem_b200 import NeoHookeanAssembler, PfgError
from polyfem_b200 import mesh as M
from polyfem_b200._lib import lib

from _cases import hooke_tensor, make_case, rel_err

pytestmark = pytest.mark.gpu

ELEMS = [(M.P1_TET, 3), (M.P2_TET, 2), (M.Q1_HEX, 3)]


@pytest.mark.parametrize("et,g", ELEMS, ids=["P1", "P2", "Q1"])
def test_hooke_matches_oracle(require_gpu, et, g):
    mesh, lam, mu, u, _ = make_case(et, g, seed=3, jitter=0.1 if et != M.P1_TET else 0.0, disp_scale=0.05)
    c21 = hooke_tensor(3)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.set_material("HookeLinearElasticity", elasticity_tensor=c21)
    orc = Oracle(mesh, lam, mu, material="HookeLinearElasticity", params={"elasticity_tensor": c21})
    e_o = orc.energy(u)
    assert abs(asm.assemble_energy(u) - e_o) <= 1e-12 * abs(e_o)
    assert rel_err(asm.assemble_energy_per_element(u), orc.energy_per_element(u)) <= 1e-12
    assert rel_err(asm.assemble_gradient(u), orc.gradient(u)) <= 1e-12
    outer, inner, vals = orc.hessian(u)
    o2, i2 = asm.hessian_pattern()
    assert np.array_equal(o2, outer) and np.array_equal(i2, inner)
    v = asm.assemble_hessian_values(u, "fp64")
    assert rel_err(v, vals) <= 1e-12
    assert np.array_equal(v, asm.assemble_hessian_values(u, "fp64"))  # deterministic
    asm.close()


def test_hooke_linear_elasticity(require_gpu):
    """HookeLinearElasticity: with the isotropic tensor it gives LinearElasticity's
    results; with an anisotropic tensor its Hessian is constant; the tensor must be
    set before use; it has no adjoint terms (the reference's assembler throws)."""
    mesh, lam, mu, u, p = make_case(M.Q1_HEX, 3, seed=24, jitter=0.1, disp_scale=0.05)
    E = mesh.n_elements
    lam0, mu0 = 7.5e4, 3.2e4
    asm = NeoHookeanAssembler.from_mesh(mesh, np.full(E, lam0), np.full(E, mu0))
    assert lib().pfg_set_material(asm.handle, 7) == 0
    with pytest.raises(PfgError) as ei:
        asm.assemble_energy(u)
    assert ei.value.status == 5  # no tensor yet
    asm.set_material("LinearElasticity")
    e_l, g_l, h_l = asm.assemble_energy(u), asm.assemble_gradient(u), asm.assemble_hessian_values(u, "fp64")
    asm.set_material("HookeLinearElasticity",
                     elasticity_tensor=NeoHookeanAssembler.isotropic_elasticity_tensor(lam0, mu0))
    assert abs(asm.assemble_energy(u) - e_l) <= 1e-12 * abs(e_l)
    assert rel_err(asm.assemble_gradient(u), g_l) <= 1e-12
    assert rel_err(asm.assemble_hessian_values(u, "fp64"), h_l) <= 1e-12
    asm.set_material("HookeLinearElasticity", elasticity_tensor=hooke_tensor(25))
    v0 = asm.assemble_hessian_values(np.zeros(mesh.n_dofs), "fp64")
    assert rel_err(asm.assemble_hessian_values(u, "fp64"), v0) <= 1e-12
    with pytest.raises(PfgError) as ei:
        asm.force_shape_derivative(u, p)
    assert ei.value.status == 4
    with pytest.raises(PfgError) as ei:
        asm.force_material_derivative(u, p)
    assert ei.value.status == 4
    with pytest.raises(ValueError):
        asm.set_material("HookeLinearElasticity", elasticity_tensor=np.ones(20))
    asm.close()


@pytest.mark.parametrize("et,g", ELEMS, ids=["P1", "P2", "Q1"])
def test_saint_venant_tensor(require_gpu, et, g):
    """SaintVenant with an anisotropic elasticity tensor (PFG_MAT_SAINT_VENANT_TENSOR)
    against the oracle; with the isotropic tensor it gives the lambda/mu SaintVenant;
    like the reference it has no shape derivative."""
    mesh, lam, mu, u, p = make_case(et, g, seed=29, jitter=0.1 if et != M.P1_TET else 0.0, disp_scale=0.05)
    c21 = hooke_tensor(30)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.set_material("SaintVenant", elasticity_tensor=c21)
    orc = Oracle(mesh, lam, mu, material="SaintVenantTensor", params={"elasticity_tensor": c21})
    e_o = orc.energy(u)
    assert abs(asm.assemble_energy(u) - e_o) <= 1e-12 * abs(e_o)
    assert rel_err(asm.assemble_energy_per_element(u), orc.energy_per_element(u)) <= 1e-12
    assert rel_err(asm.assemble_gradient(u), orc.gradient(u)) <= 1e-12
    outer, inner, vals = orc.hessian(u)
    assert rel_err(asm.assemble_hessian_values(u, "fp64"), vals) <= 1e-12
    _, _, v_psd = orc.hessian(u, project_psd=True)
    assert rel_err(asm.assemble_hessian_values(u, "fp64", project_to_psd=True), v_psd) <= 1e-11
    with pytest.raises(PfgError) as ei:
        asm.force_shape_derivative(u, p)
    assert ei.value.status == 4
    E = mesh.n_elements
    lam0, mu0 = 7.5e4, 3.2e4
    asm.set_lame(np.full(E, lam0), np.full(E, mu0))
    asm.set_material("SaintVenant")
    e_s, g_s, h_s = asm.assemble_energy(u), asm.assemble_gradient(u), asm.assemble_hessian_values(u, "fp64")
    asm.set_material("SaintVenant", elasticity_tensor=NeoHookeanAssembler.isotropic_elasticity_tensor(lam0, mu0))
    assert abs(asm.assemble_energy(u) - e_s) <= 1e-12 * abs(e_s)
    assert rel_err(asm.assemble_gradient(u), g_s) <= 1e-12
    assert rel_err(asm.assemble_hessian_values(u, "fp64"), h_s) <= 1e-12
    asm.close()


def test_hooke_inverted_element_and_reduced_saint_venant(require_gpu):
    """An element turned inside out: HookeLinearElasticity has no ln J and stays finite,
    the per-element energies follow the oracle and the inverted count sees it.  The
    anisotropic SaintVenant through the Dirichlet reduction: reduced pattern and values
    against the oracle's restatement of BCLagrangianForm::project_hessian."""
    from oracle.binding import project_hessian
    mesh, lam, mu, _, _ = make_case(M.P1_TET, 2, seed=17)
    bad = np.zeros(mesh.n_dofs)
    c = mesh.conn[0]
    X = mesh.node_pos
    bad.reshape(-1, 3)[c[3]] = 2.0 * (X[c[:3]].mean(axis=0) - X[c[3]])  # vertex 3 through the opposite face
    c21 = hooke_tensor(31)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.set_material("HookeLinearElasticity", elasticity_tensor=c21)
    orc = Oracle(mesh, lam, mu, material="HookeLinearElasticity", params={"elasticity_tensor": c21})
    pe = asm.assemble_energy_per_element(bad)
    assert np.all(np.isfinite(pe))
    assert rel_err(pe, orc.energy_per_element(bad)) <= 1e-12
    assert rel_err(asm.assemble_gradient(bad), orc.gradient(bad)) <= 1e-12
    assert asm.inverted_count() >= 1
    asm.close()

    mesh, lam, mu, u, _ = make_case(M.P2_TET, 2, seed=32, jitter=0.1, disp_scale=0.05)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.set_material("SaintVenant", elasticity_tensor=c21)
    orc = Oracle(mesh, lam, mu, material="SaintVenantTensor", params={"elasticity_tensor": c21})
    outer, inner, vals = orc.hessian(u)
    face = np.flatnonzero(mesh.node_pos[:, 0] <= 1e-12)
    dofs = (3 * face[:, None] + np.arange(3)).ravel()
    asm.set_dirichlet(dofs)
    ro, ri, rv = project_hessian(outer, inner, vals, dofs)
    go, gi = asm.reduced_pattern()
    assert np.array_equal(go, ro) and np.array_equal(gi, ri)
    assert rel_err(asm.assemble_hessian_reduced_values(u, "fp64"), rv) <= 1e-12
    assert rel_err(asm.assemble_gradient_reduced(u, "fp64"), np.delete(orc.gradient(u), np.unique(dofs))) <= 1e-12
    asm.close()
