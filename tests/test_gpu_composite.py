"""Compositions of formulations on the GPU (pfg_set_component / pfg_set_composite):
MaterialSum (SumModel) and MultiModels (MultiModel) against the oracle's
restatement, which composes the oracle's element energies, gradients and Hessians
per element (projecting the composed element matrix)."""
import numpy as np
import pytest

from oracle.binding import composite_reference, project_hessian
from polyfem_b200 import NeoHookeanAssembler, PfgError
from polyfem_b200 import mesh as M

from _cases import make_case, material_params, rel_err

pytestmark = pytest.mark.gpu

ELEMS = [(M.P1_TET, 3), (M.P2_TET, 2), (M.Q1_HEX, 3)]


def _components(mesh, lam, mu, seed):
    """NeoHookean with its own Lame parameters, MooneyRivlin, UnconstrainedOgden: the
    assembler's component dicts and the oracle's (material, lam, mu, params)."""
    E = mesh.n_elements
    rng = np.random.default_rng(seed)
    lam2, mu2 = lam * rng.uniform(0.5, 1.5, E), mu * rng.uniform(0.5, 1.5, E)
    mr = material_params("MooneyRivlin", E, seed=seed)
    og = material_params("UnconstrainedOgden", E, seed=seed)
    dev = [dict(formulation="NeoHookean", lam=lam2, mu=mu2), dict(formulation="MooneyRivlin", **mr),
           dict(formulation="UnconstrainedOgden", **og)]
    orc = [("NeoHookean", lam2, mu2, None), ("MooneyRivlin", lam, mu, mr), ("UnconstrainedOgden", lam, mu, og)]
    return dev, orc


def _dense(asm, vals, n):
    outer, inner = asm.hessian_pattern()
    D = np.zeros((n, n))
    D[inner, np.repeat(np.arange(n), np.diff(outer))] = vals
    return D


@pytest.mark.parametrize("multi", [False, True], ids=["MaterialSum", "MultiModels"])
@pytest.mark.parametrize("et,g", ELEMS, ids=["P1", "P2", "Q1"])
def test_composite_matches_oracle(require_gpu, et, g, multi):
    import torch
    mesh, lam, mu, u, _ = make_case(et, g, seed=31, jitter=0.1 if et != M.P1_TET else 0.0, disp_scale=0.05)
    dev, orc = _components(mesh, lam, mu, 32)
    sel = None
    if multi:  # bodies: by element, the three components cycling
        sel = np.arange(mesh.n_elements) % 3
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.set_composite(dev, sel)
    per, grad, H = composite_reference(mesh, orc, sel, u)
    assert rel_err(asm.assemble_energy_per_element(u), per) <= 1e-12
    assert abs(asm.assemble_energy(u) - per.sum()) <= 1e-12 * abs(per.sum())
    assert rel_err(asm.assemble_gradient(u), grad) <= 1e-12
    v = asm.assemble_hessian_values(u)
    assert rel_err(_dense(asm, v, mesh.n_dofs), H) <= 1e-12
    assert np.array_equal(v, asm.assemble_hessian_values(torch.tensor(u, device="cuda")).cpu().numpy())
    # projected after the composition
    _, _, Hp = composite_reference(mesh, orc, sel, u, project=True)
    vp = asm.assemble_hessian_values(u, project_to_psd=True)
    assert rel_err(_dense(asm, vp, mesh.n_dofs), Hp) <= 1e-11
    # Dirichlet reduction of the composition
    face = np.flatnonzero(mesh.node_pos[:, 0] <= 1e-12)
    dofs = (3 * face[:, None] + np.arange(3)).ravel()
    asm.set_dirichlet(dofs)
    outer, inner = asm.hessian_pattern()
    ro, ri, rv = project_hessian(outer, inner, v, dofs)
    assert rel_err(asm.assemble_hessian_reduced_values(u, "fp64"), rv) <= 1e-12
    assert rel_err(asm.assemble_gradient_reduced(u, "fp64"), np.delete(grad, np.unique(dofs))) <= 1e-12
    asm.close()


def test_composite_of_one_component_and_state(require_gpu):
    """A composition of one component assembles the same Hessian, bit for bit, as the
    formulation alone; FP64 only; no adjoint terms; set_material leaves it."""
    mesh, lam, mu, u, p = make_case(M.P2_TET, 2, seed=33, disp_scale=0.05)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    h_nh = asm.assemble_hessian_values(u, "fp64")
    prm = material_params("MooneyRivlin", mesh.n_elements, seed=34)
    asm.set_material("MooneyRivlin", **prm)
    h_mr = asm.assemble_hessian_values(u, "fp64")
    asm.set_composite([dict(formulation="NeoHookean")])
    assert np.array_equal(asm.assemble_hessian_values(u, "fp64"), h_nh)
    asm.set_composite([dict(formulation="MooneyRivlin", **prm)])
    assert np.array_equal(asm.assemble_hessian_values(u, "fp64"), h_mr)
    for call in (lambda: asm.assemble_hessian_values(u, "split32"), lambda: asm.force_shape_derivative(u, p),
                 lambda: asm.force_material_derivative(u, p)):
        with pytest.raises(PfgError) as ei:
            call()
        assert ei.value.status == 4  # PFG_ERR_UNSUPPORTED
    with pytest.raises(PfgError):
        asm.set_composite([dict(formulation="NeoHookean")], np.full(mesh.n_elements, 1))  # component 1 unset
    asm.set_material("NeoHookean")
    assert np.array_equal(asm.assemble_hessian_values(u, "fp64"), h_nh)
    asm.close()
