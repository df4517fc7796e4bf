"""GPU parity: libpfgpu (through its C ABI) against the CPU oracle on the same seeded inputs.

Tolerances:
  FP64 paths      : normwise relative error <= 1e-12, CSC indices bit-exact
  FP32 paths      : energy 1e-6, gradient / Hessian / shape VJP 1e-5 (normwise, vs the FP64 oracle)
  SPLIT32 Hessian : <= 1e-6 relative Frobenius error vs the FP64 oracle
"""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle.binding import Oracle
from polyfem_b200 import ElasticForm, NeoHookeanAssembler
from polyfem_b200 import mesh as M

from _cases import ELEM_NAMES, make_case, rel_err

pytestmark = pytest.mark.gpu

SMALL = [(M.P1_TET, 4, 0.0), (M.P2_TET, 3, 0.1), (M.Q1_HEX, 4, 0.1)]
TOL64 = 1e-12


@pytest.fixture(scope="module", params=SMALL, ids=lambda c: ELEM_NAMES[c[0]])
def case(request, require_gpu):
    et, g, jit = request.param
    mesh, lam, mu, u, p = make_case(et, g, seed=21, jitter=jit)
    orc = Oracle(mesh, lam, mu, n_threads=4, fast_pattern=True)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    yield dict(mesh=mesh, lam=lam, mu=mu, u=u, p=p, orc=orc, asm=asm)
    asm.close()


def test_energy_fp64(case):
    e_ref = case["orc"].energy(case["u"])
    e = case["asm"].assemble_energy(case["u"])
    assert abs(e - e_ref) <= TOL64 * abs(e_ref)


def test_energy_per_element_fp64(case):
    ref = case["orc"].energy_per_element(case["u"])
    got = case["asm"].assemble_energy_per_element(case["u"])
    assert rel_err(got, ref) <= TOL64
    assert np.abs(got - ref).max() <= TOL64 * np.abs(ref).max()
    assert abs(got.sum() - case["asm"].assemble_energy(case["u"])) <= 1e-10 * abs(got.sum())


def test_gradient_fp64(case):
    ref = case["orc"].gradient(case["u"])
    got = case["asm"].assemble_gradient(case["u"])
    assert rel_err(got, ref) <= TOL64


def test_hessian_fp64_pattern_and_values(case):
    o_ref, i_ref, v_ref = case["orc"].hessian(case["u"])
    outer, inner = case["asm"].hessian_pattern()
    assert np.array_equal(outer, o_ref), "CSC outer indices differ"
    assert np.array_equal(inner, i_ref), "CSC inner indices differ"
    vals = case["asm"].assemble_hessian_values(case["u"])
    assert rel_err(vals, v_ref) <= TOL64
    # second call (slot-map path) reproduces the first
    vals2 = case["asm"].assemble_hessian_values(case["u"])
    assert rel_err(vals2, v_ref) <= TOL64


def test_material_vjp_fp64(case):
    ref = case["orc"].material_vjp(case["u"], case["p"])
    got = case["asm"].force_material_derivative(case["u"], case["p"])
    assert rel_err(got, ref) <= TOL64


def test_shape_vjp_fp64(case):
    ref = case["orc"].shape_vjp(case["u"], case["p"])
    got = case["asm"].force_shape_derivative(case["u"], case["p"], "fp64")
    assert rel_err(got, ref) <= TOL64


def test_fp32_paths_within_stated_bounds(case):
    u, orc, asm = case["u"], case["orc"], case["asm"]
    e_ref = orc.energy(u)
    assert abs(asm.assemble_energy(u, "fp32") - e_ref) <= 1e-6 * abs(e_ref)
    assert rel_err(asm.assemble_gradient(u, "fp32"), orc.gradient(u)) <= 1e-5
    _, _, v_ref = orc.hessian(u)
    assert rel_err(asm.assemble_hessian_values(u, "fp32"), v_ref) <= 1e-5
    assert rel_err(asm.force_shape_derivative(u, case["p"], "fp32"), orc.shape_vjp(u, case["p"])) <= 1e-4


@pytest.mark.parametrize("prec", ["split32", "split32_simt"])
def test_split32_hessian_within_bound(case, prec):
    """split32 (tensor cores for P2 and Q1) and split32_simt (CUDA cores) both
    within the 1e-6 relative Frobenius bound of the split mode."""
    u, orc, asm = case["u"], case["orc"], case["asm"]
    _, _, v_ref = orc.hessian(u)
    assert rel_err(asm.assemble_hessian_values(u, prec), v_ref) <= 1e-6


def test_device_mode_matches_host_mode(case):
    import torch
    u, asm = case["u"], case["asm"]
    ud = torch.tensor(u, device="cuda", dtype=torch.float64)
    pd = torch.tensor(case["p"], device="cuda", dtype=torch.float64)
    assert float(asm.assemble_energy(ud).cpu()) == asm.assemble_energy(u)
    assert rel_err(asm.assemble_gradient(ud).cpu().numpy(), asm.assemble_gradient(u)) <= 1e-15
    assert rel_err(asm.assemble_hessian_values(ud).cpu().numpy(), asm.assemble_hessian_values(u)) <= 1e-15
    assert np.array_equal(asm.force_material_derivative(ud, pd).cpu().numpy(),
                          asm.force_material_derivative(u, case["p"]))
    H = asm.assemble_hessian(ud)
    Hh = asm.assemble_hessian(u)
    y = (H @ pd.unsqueeze(1)).squeeze(1).cpu().numpy()
    assert rel_err(y, Hh @ case["p"]) <= 1e-13


def test_energy_is_deterministic(case):
    u, asm = case["u"], case["asm"]
    vals = {asm.assemble_energy(u) for _ in range(5)}
    assert len(vals) == 1


def test_elastic_form_weighting(case):
    form = ElasticForm(case["asm"])
    u = case["u"]
    e0 = form.value(u)
    form.set_weight(2.5)
    form.set_scale(0.5)
    assert abs(form.value(u) - 5.0 * e0) <= 1e-13 * abs(e0)
    assert rel_err(form.first_derivative(u), 5.0 * case["asm"].assemble_gradient(u)) <= 1e-15
    assert form.is_step_valid(u, u)


def test_inverted_element_propagates_nan(require_gpu):
    mesh, lam, mu, u, _ = make_case(M.P1_TET, 2, seed=3)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    bad = np.zeros(mesh.n_dofs)
    # collapse element 0 through itself: move its vertex 3 onto the opposite face and beyond
    c = mesh.conn[0]
    X = mesh.node_pos
    centroid = X[c[:3]].mean(axis=0)
    bad.reshape(-1, 3)[c[3]] = 2.0 * (centroid - X[c[3]])
    assert np.isnan(asm.assemble_energy(bad))
    assert np.isnan(asm.assemble_gradient(bad)).any()
    assert asm.inverted_count() >= 1
    assert not ElasticForm(asm).is_step_valid(bad, bad)
    orc = Oracle(mesh, lam, mu)
    assert np.isnan(orc.energy(bad))
    assert np.array_equal(np.isnan(asm.assemble_gradient(bad)), np.isnan(orc.gradient(bad)))
    asm.close()


def test_empty_mesh(require_gpu):
    conn = np.zeros((0, 4), dtype=np.int32)
    X = np.zeros((5, 3))
    asm = NeoHookeanAssembler(M.P1_TET, conn, X, np.zeros(0), np.zeros(0), n_nodes=5)
    u = np.zeros(15)
    assert asm.assemble_energy(u) == 0.0
    assert np.all(asm.assemble_gradient(u) == 0.0)
    assert asm.hessian_nnz() == 0
    assert asm.assemble_hessian_values(u).size == 0
    assert asm.force_material_derivative(u, u).size == 0
    assert np.all(asm.force_shape_derivative(u, u) == 0.0)
    asm.close()


def test_single_element_each_type(require_gpu):
    for et in (M.P1_TET, M.P2_TET, M.Q1_HEX):
        mesh, lam, mu, u, p = make_case(et, 1, seed=31, jitter=0.0)
        keep = 1
        conn = mesh.conn[:keep]
        gconn = mesh.gconn[:keep]
        used = np.unique(conn)
        remap = -np.ones(mesh.n_nodes, dtype=np.int64)
        remap[used] = np.arange(used.size)
        gused = np.unique(gconn)
        gremap = -np.ones(mesh.n_geom_nodes, dtype=np.int64)
        gremap[gused] = np.arange(gused.size)
        sub = M.Mesh(et, remap[conn].astype(np.int32), gremap[gconn].astype(np.int32), mesh.X[gused],
                     used.size, mesh.node_pos[used], mesh.h, 1)
        if et != M.P2_TET:
            sub.gconn = sub.conn
        us = u.reshape(-1, 3)[used].ravel()
        orc = Oracle(sub, lam[:keep], mu[:keep])
        asm = NeoHookeanAssembler.from_mesh(sub, lam[:keep], mu[:keep])
        assert abs(asm.assemble_energy(us) - orc.energy(us)) <= TOL64 * abs(orc.energy(us))
        o, i, v = orc.hessian(us)
        assert np.array_equal(asm.hessian_pattern()[1], i)
        assert rel_err(asm.assemble_hessian_values(us), v) <= TOL64
        asm.close()


def test_config1_full_size_against_oracle(require_gpu):
    """20^3 P1 tets (48,000 elements, 27,783 dofs, 1,157,229 nnz), homogeneous E=1e5, nu=0.35."""
    mesh = M.structured_tet_mesh(20, 1)
    lam, mu = M.homogeneous_lame(mesh.n_elements)
    u = M.random_displacement(mesh, 0.02, 1)
    orc = Oracle(mesh, lam, mu, n_threads=8, fast_pattern=True)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    assert abs(asm.assemble_energy(u) - orc.energy(u)) <= TOL64 * abs(orc.energy(u))
    assert rel_err(asm.assemble_gradient(u), orc.gradient(u)) <= TOL64
    o, i, v = orc.hessian(u)
    assert asm.hessian_nnz() == 1157229 == len(i)
    outer, inner = asm.hessian_pattern()
    assert np.array_equal(outer, o) and np.array_equal(inner, i)
    assert rel_err(asm.assemble_hessian_values(u), v) <= TOL64
    asm.close()


@pytest.mark.parametrize("which", ["P2-40", "Q1-96"])
def test_full_size_hessian_properties(require_gpu, which):
    """BASELINE sizes, checked through size-independent properties on the device:
    nnz, symmetry (CSC == CSC of the transpose), rigid translations in the null space,
    split32 vs fp64 agreement, and a gradient that sums to zero per direction."""
    import torch
    if which == "P2-40":
        mesh = M.structured_tet_mesh(40, 2)
        lam, mu = M.lognormal_lame(mesh.n_elements, 5)
        u = M.random_displacement(mesh, 0.02, 2)
        nnz_expected = 134475849
    else:
        mesh = M.structured_hex_mesh(96, jitter=0.1, seed=3)
        lam, mu = M.lognormal_lame(mesh.n_elements, 6)
        u = M.smooth_displacement(mesh, 0.05, 0.005, 4)
        nnz_expected = 217238121
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    assert asm.hessian_nnz() == nnz_expected
    ud = torch.tensor(u, device="cuda", dtype=torch.float64)
    H64 = asm.assemble_hessian(ud, "fp64")
    n = mesh.n_dofs
    for d in range(3):
        t = torch.zeros(n, dtype=torch.float64, device="cuda")
        t[d::3] = 1.0
        r = (H64 @ t.unsqueeze(1)).squeeze(1)
        scale = torch.linalg.vector_norm(H64.values()) / np.sqrt(n)
        assert float(torch.linalg.vector_norm(r)) <= 1e-10 * float(scale) * np.sqrt(n)
    # symmetry: H x . y == x . H y for random x, y
    gen = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
    y = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
    a = torch.dot((H64 @ x.unsqueeze(1)).squeeze(1), y)
    b = torch.dot(x, (H64 @ y.unsqueeze(1)).squeeze(1))
    assert abs(float(a - b)) <= 1e-12 * abs(float(a))
    v64 = H64.values().clone()
    del H64
    vs = asm.assemble_hessian_values(ud, "split32")
    err = float(torch.linalg.vector_norm(vs - v64) / torch.linalg.vector_norm(v64))
    assert err <= 1e-6
    g = asm.assemble_gradient(ud)
    assert float(torch.abs(g.view(-1, 3).sum(0)).max()) <= 1e-9 * float(torch.abs(g).max())
    asm.close()


@pytest.mark.parametrize("et,g", [(M.P1_TET, 26), (M.P2_TET, 16), (M.Q1_HEX, 32)], ids=["P1-26", "P2-16", "Q1-32"])
def test_medium_mesh_hessian_against_oracle(require_gpu, et, g):
    """Medium meshes (20k-105k elements, many CTAs and warps of both Hessian
    passes): pattern bit-exact, FP64 and split32 values within their bounds, and
    every call bitwise identical."""
    mesh, lam, mu, u, _ = make_case(et, g, seed=31, jitter=0.1 if et != M.P1_TET else 0.0)
    orc = Oracle(mesh, lam, mu, n_threads=8, fast_pattern=True)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    o, i, v = orc.hessian(u)
    outer, inner = asm.hessian_pattern()
    assert np.array_equal(outer, o) and np.array_equal(inner, i)
    h64 = asm.assemble_hessian_values(u, "fp64")
    assert rel_err(h64, v) <= TOL64
    assert np.array_equal(h64, asm.assemble_hessian_values(u, "fp64"))
    for prec in ("split32", "split32_simt"):
        hs = asm.assemble_hessian_values(u, prec)
        assert rel_err(hs, v) <= 1e-6, prec
        assert np.array_equal(hs, asm.assemble_hessian_values(u, prec)), prec
    asm.close()
