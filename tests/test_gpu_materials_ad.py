"""Energy-defined formulations on the GPU (pfg_materials.cu): LinearElasticity,
MooneyRivlin, MooneyRivlin3Param, VolumePenalty and the two Ogden formulations
(principal stretches from the invariants' characteristic cubic), differentiated on the device by
dual and hyper-dual numbers.  FP64 energy, gradient and Hessian (with
project_to_psd and the Dirichlet reduction) against the oracle, which
differentiates the same energies with second-order dual numbers over F as the
reference's GenericElastic does (AutodiffType::STRESS)."""
import numpy as np
import pytest

from oracle.binding import Oracle, project_hessian
from polyfem_b200 import NeoHookeanAssembler, PfgError
from polyfem_b200 import mesh as M
from polyfem_b200._lib import lib

from _cases import make_case, material_params, rel_err

pytestmark = pytest.mark.gpu

MATS = ["LinearElasticity", "MooneyRivlin", "MooneyRivlin3Param", "VolumePenalty", "UnconstrainedOgden",
        "IncompressibleOgden", "MooneyRivlin3ParamSymbolic"]
ELEMS = [(M.P1_TET, 3), (M.P2_TET, 2), (M.Q1_HEX, 3)]


def setup(et, g, mat, seed=3, disp=0.05):
    mesh, lam, mu, u, p = make_case(et, g, seed=seed, jitter=0.1 if et != M.P1_TET else 0.0, disp_scale=disp)
    prm = material_params(mat, mesh.n_elements, seed=seed)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.set_material(mat, **prm)
    return mesh, asm, Oracle(mesh, lam, mu, material=mat, params=prm), u, p


@pytest.mark.parametrize("mat", MATS)
@pytest.mark.parametrize("et,g", ELEMS, ids=["P1", "P2", "Q1"])
def test_energy_gradient_hessian_match_oracle(require_gpu, mat, et, g):
    mesh, asm, orc, u, _ = setup(et, g, mat)
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


@pytest.mark.parametrize("mat", ["MooneyRivlin", "MooneyRivlin3Param", "UnconstrainedOgden", "IncompressibleOgden",
        "MooneyRivlin3ParamSymbolic"])
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


def test_linear_elasticity_hessian_constant_on_device(require_gpu):
    mesh, asm, orc, u, _ = setup(M.Q1_HEX, 2, "LinearElasticity", seed=8)
    v0 = asm.assemble_hessian_values(np.zeros(mesh.n_dofs), "fp64")
    v1 = asm.assemble_hessian_values(u, "fp64")
    assert rel_err(v1, v0) <= 1e-12
    asm.close()


def test_device_parameters_and_state_errors(require_gpu):
    import torch
    mesh, lam, mu, u, _ = make_case(M.P2_TET, 2, seed=9)
    E = mesh.n_elements
    prm = material_params("MooneyRivlin3Param", E, seed=9)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    # the material before its parameters: PFG_ERR_STATE
    assert lib().pfg_set_material(asm.handle, 5) == 0
    with pytest.raises(PfgError) as ei:
        asm.assemble_energy(u)
    assert ei.value.status == 5
    # parameters as CUDA tensors give the host-array results bit for bit
    asm.set_material("MooneyRivlin3Param", **{k: torch.tensor(v, device="cuda") for k, v in prm.items()})
    e_dev, g_dev = asm.assemble_energy(u), asm.assemble_gradient(u)
    asm.set_material("MooneyRivlin3Param", **prm)
    assert asm.assemble_energy(u) == e_dev and np.array_equal(asm.assemble_gradient(u), g_dev)
    # scalars broadcast to every element
    asm.set_material("VolumePenalty", k=2.5e5)
    orc = Oracle(mesh, lam, mu, material="VolumePenalty", params={"k": 2.5e5})
    assert abs(asm.assemble_energy(u) - orc.energy(u)) <= 1e-12 * abs(orc.energy(u))
    # a parameter count that does not match the material: PFG_ERR_STATE
    assert lib().pfg_set_material(asm.handle, 4) == 0
    with pytest.raises(PfgError) as ei:
        asm.assemble_hessian_values(u, "fp64")
    assert ei.value.status == 5
    # FP32 paths stay NeoHookean-only; bad counts and names are rejected
    asm.set_material("MooneyRivlin", **material_params("MooneyRivlin", E))
    with pytest.raises(PfgError) as ei:
        asm.assemble_gradient(u, "fp32")
    assert ei.value.status == 4
    assert lib().pfg_set_material_params(asm.handle, None, 5, 0) == 1
    with pytest.raises(ValueError):
        asm.set_material("MooneyRivlin", c1=1.0)
    asm.close()


@pytest.mark.parametrize("mat", MATS)
def test_inverted_element(require_gpu, mat):
    """An element turned inside out: ln J and J^(-2/3) of a negative J give NaN, which
    propagates as in the reference (no clamp); the linear formulations stay finite.  The
    per-element energies, the gradient's NaN pattern and the inverted count follow the
    oracle."""
    mesh, lam, mu, _, _ = make_case(M.P1_TET, 2, seed=17)
    bad = np.zeros(mesh.n_dofs)
    c = mesh.conn[0]
    X = mesh.node_pos
    bad.reshape(-1, 3)[c[3]] = 2.0 * (X[c[:3]].mean(axis=0) - X[c[3]])  # vertex 3 through the opposite face
    prm = material_params(mat, mesh.n_elements, seed=17)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.set_material(mat, **prm)
    orc = Oracle(mesh, lam, mu, material=mat, params=prm)
    pe, pe_o = asm.assemble_energy_per_element(bad), orc.energy_per_element(bad)
    assert np.array_equal(np.isnan(pe), np.isnan(pe_o))
    assert np.isnan(pe[0]) == (mat not in ("LinearElasticity", "HookeLinearElasticity"))
    ok = ~np.isnan(pe_o)
    assert rel_err(pe[ok], pe_o[ok]) <= 1e-12
    g, g_o = asm.assemble_gradient(bad), orc.gradient(bad)
    assert np.array_equal(np.isnan(g), np.isnan(g_o))
    assert rel_err(g[~np.isnan(g_o)], g_o[~np.isnan(g_o)]) <= 1e-12
    assert asm.inverted_count() >= 1
    asm.close()


SHAPE_MATS = ["IsochoricNeoHookean", "LinearElasticity", "MooneyRivlin", "MooneyRivlin3Param", "VolumePenalty",
              "UnconstrainedOgden", "IncompressibleOgden", "MooneyRivlin3ParamSymbolic"]


@pytest.mark.parametrize("mat", SHAPE_MATS)
@pytest.mark.parametrize("et,g", ELEMS, ids=["P1", "P2", "Q1"])
def test_shape_vjp_matches_oracle(require_gpu, mat, et, g):
    """force_shape_derivative for the formulations whose reference assembler has
    compute_stress_grad_multiply_mat: the stress and its directional derivative along
    grad p from hyper-dual numbers over the invariants (closed form for LinearElasticity)."""
    mesh, lam, mu, u, p = make_case(et, g, seed=11, jitter=0.1 if et != M.P1_TET else 0.0, disp_scale=0.05)
    prm = material_params(mat, mesh.n_elements, seed=11)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.set_material(mat, **prm)
    orc = Oracle(mesh, lam, mu, material=mat, params=prm)
    t = asm.force_shape_derivative(u, p)
    assert rel_err(t, orc.shape_vjp(u, p)) <= 1e-11
    assert np.array_equal(t, asm.force_shape_derivative(u, p))  # deterministic
    asm.close()


@pytest.mark.parametrize("et,g", ELEMS, ids=["P1", "P2", "Q1"])
def test_linear_elasticity_material_vjp_matches_oracle(require_gpu, et, g):
    mesh, lam, mu, u, p = make_case(et, g, seed=12, jitter=0.1 if et != M.P1_TET else 0.0)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.set_material("LinearElasticity")
    orc = Oracle(mesh, lam, mu, material="LinearElasticity")
    assert rel_err(asm.force_material_derivative(u, p), orc.material_vjp(u, p)) <= 1e-12
    asm.close()


def test_adjoint_terms_the_reference_lacks(require_gpu):
    """The reference throws for the material derivative of the GenericElastic materials
    and for SaintVenant's shape derivative: PFG_ERR_UNSUPPORTED here; FP32 shape terms
    stay NeoHookean-only."""
    mesh, lam, mu, u, p = make_case(M.P1_TET, 2, seed=13)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    for mat in ("IsochoricNeoHookean", "SaintVenant", "MooneyRivlin", "MooneyRivlin3Param", "VolumePenalty"):
        asm.set_material(mat, **material_params(mat, mesh.n_elements))
        with pytest.raises(PfgError) as ei:
            asm.force_material_derivative(u, p)
        assert ei.value.status == 4
    asm.set_material("SaintVenant")
    with pytest.raises(PfgError) as ei:
        asm.force_shape_derivative(u, p)
    assert ei.value.status == 4
    asm.set_material("LinearElasticity")
    with pytest.raises(PfgError) as ei:
        asm.force_shape_derivative(u, p, "fp32")
    assert ei.value.status == 4
    asm.close()
