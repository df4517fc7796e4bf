"""Pins the CPU oracle (CPU only, no GPU).

* the reference's own SparseMatrixCache known-answer test (tests/test_matrix.cpp:202-249);
* an independent restatement of the reference-element tables
  (autogen/auto_p_bases.cpp, autogen/auto_q_bases_3d_grad_1.cpp, quadrature/*.cpp);
* the reference's autodiff-equality method (tests/test_assembler.cpp:127-286)
  with torch float64 autograd in place of NeoHookeanAutodiff;
* the reference's finite-difference method (tests/test_form_derivatives.cpp:166-226);
* closed-form known answers of the NeoHookean law.
"""
import itertools

import numpy as np
import pytest
import scipy.sparse as sp

from oracle.binding import Oracle, SparseMatrixCache, tables
from polyfem_b200 import mesh as M

from _cases import ELEM_NAMES, make_case, rel_err

ELEMS = [M.P1_TET, M.P2_TET, M.Q1_HEX]


# --------------------------------------------------------------------------- KAT
def test_sparse_matrix_cache_known_answer():
    """Restates TEST_CASE("cache", "[matrix]") of tests/test_matrix.cpp:202-249."""
    cache = SparseMatrixCache(10)
    for args in [(0, 0, 0, 1), (0, 0, 1, 2), (0, 9, 4, 3), (0, 9, 4, 3), (0, 9, 9, 4)]:
        cache.add_value(*args)
    cache.get_matrix()
    assert [cache.coeff(0, 0), cache.coeff(0, 1), cache.coeff(9, 4), cache.coeff(9, 9)] == [1, 2, 6, 4]

    cache1 = SparseMatrixCache(10)
    cache1.add_value(0, 0, 0, 1)
    cache1.add_value(0, 0, 1, 2)
    cache1.prune()
    cache1.add_value(0, 9, 4, 3)
    cache1.add_value(0, 9, 4, 3)
    cache1.add_value(0, 9, 9, 4)
    cache1.get_matrix()
    assert [cache1.coeff(0, 0), cache1.coeff(0, 1), cache1.coeff(9, 4), cache1.coeff(9, 9)] == [1, 2, 6, 4]

    cache2 = SparseMatrixCache(other=cache1)
    cache2.add_value(0, 0, 0, 1)
    cache2.add_value(0, 0, 1, 2)
    cache2.prune()
    cache2.add_value(0, 9, 4, 3)
    cache2.add_value(0, 9, 4, 3)
    cache2.add_value(0, 9, 9, 4)
    cache2.get_matrix()
    assert [cache2.coeff(0, 0), cache2.coeff(0, 1), cache2.coeff(9, 4), cache2.coeff(9, 9)] == [1, 2, 6, 4]


def test_lump_matrix_known_answer():
    """utils::lump_matrix (utils/MatrixUtils.cpp:84-101) restated: row sums in
    ascending column order, starting from the first value (setFromTriplets)."""
    from oracle.binding import lump_matrix
    # row 0 holds 1e16, 1, -1e16 in columns 0, 1, 2: (1e16 + 1) - 1e16 == 0 in FP64,
    # while the column-2-first order would give 1
    A = sp.csc_matrix(np.array([[1e16, 1.0, -1e16, 0.0],
                                [2.0, 3.0, 0.0, 0.0],
                                [0.0, 0.0, 0.0, 0.0],
                                [-0.0, 0.0, 0.0, 5.0]]))
    A.eliminate_zeros()
    d = lump_matrix(A.indptr, A.indices, A.data)
    assert d.tolist() == [0.0, 5.0, 0.0, 5.0]
    # structurally present zeros are summed like any value
    d = lump_matrix(np.array([0, 1, 2]), np.array([0, 0]), np.array([-0.0, 2.5]))
    assert d.tolist() == [2.5, 0.0]
    B = sp.random(40, 40, density=0.2, random_state=4, format="csc")
    assert np.allclose(lump_matrix(B.indptr, B.indices, B.data), np.asarray(B.sum(axis=1)).ravel(), rtol=1e-14)


# ------------------------------------------------------------------ tables
def _indep_tables(et):
    """Second, independent reading of the reference tables."""
    if et == M.P1_TET:
        pts = np.array([[0.25, 0.25, 0.25]])
        w = np.array([1.0]) / 6
    elif et == M.P2_TET:
        a = 0.13819660112501053195188660538406111299991607666015625
        b = 0.58541019662496840414434018384781666100025177001953125
        pts = np.array([[a, a, b], [a, b, a], [b, a, a], [a, a, a]])
        w = np.full(4, 0.25) / 6
    else:
        x = np.array([-0.5773502691896257645, 0.5773502691896257645]) / 2 + 0.5
        pts = np.array([[x[k], x[j], x[i]] for i in range(2) for j in range(2) for k in range(2)])
        w = np.full(8, 0.125)

    def p1(x, y, z):
        return np.array([[-1, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)

    def p2(x, y, z):
        L0 = 1 - x - y - z
        lam = [L0, x, y, z]
        dl = np.array([[-1, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)
        g = [(4 * lam[i] - 1) * dl[i] for i in range(4)]
        for (i, j) in [(0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3)]:
            g.append(4 * (lam[i] * dl[j] + lam[j] * dl[i]))
        return np.array(g)

    def q1(x, y, z):
        out = []
        for (cx, cy, cz) in M.HEX_CORNERS:
            fx = (x if cx else 1 - x, 1.0 if cx else -1.0)
            fy = (y if cy else 1 - y, 1.0 if cy else -1.0)
            fz = (z if cz else 1 - z, 1.0 if cz else -1.0)
            out.append([fx[1] * fy[0] * fz[0], fx[0] * fy[1] * fz[0], fx[0] * fy[0] * fz[1]])
        return np.array(out)

    f = {M.P1_TET: p1, M.P2_TET: p2, M.Q1_HEX: q1}[et]
    gf = {M.P1_TET: p1, M.P2_TET: p1, M.Q1_HEX: q1}[et]
    return pts, w, np.array([f(*p) for p in pts]), np.array([gf(*p) for p in pts])


@pytest.mark.parametrize("et", ELEMS, ids=lambda e: ELEM_NAMES[e])
def test_reference_tables(et):
    qp, qw, gr, gg = tables(et)
    qp2, qw2, gr2, gg2 = _indep_tables(et)
    np.testing.assert_allclose(qp, qp2, rtol=0, atol=1e-15)
    np.testing.assert_allclose(qw, qw2, rtol=0, atol=1e-16)
    np.testing.assert_allclose(gr, gr2, rtol=0, atol=1e-14)
    np.testing.assert_allclose(gg, gg2, rtol=0, atol=1e-14)
    # partition of unity: gradients sum to zero at every point
    assert np.abs(gr.sum(axis=1)).max() < 1e-14
    # weights sum to the reference volume (quadrature tests of tests/test_quadrature.cpp)
    assert abs(qw.sum() - (1.0 if et == M.Q1_HEX else 1.0 / 6.0)) < 1e-15


@pytest.mark.parametrize("et", ELEMS, ids=lambda e: ELEM_NAMES[e])
def test_quadrature_exactness(et):
    qp, qw, _, _ = tables(et)
    if et == M.Q1_HEX:
        # 2-point Gauss per axis is exact for degree <= 3 in each variable
        for px, py, pz in itertools.product(range(4), repeat=3):
            exact = 1 / ((px + 1) * (py + 1) * (pz + 1))
            got = (qw * qp[:, 0] ** px * qp[:, 1] ** py * qp[:, 2] ** pz).sum()
            assert abs(got - exact) < 1e-14
    else:
        from math import factorial
        deg = 1 if et == M.P1_TET else 2
        for px, py, pz in itertools.product(range(deg + 1), repeat=3):
            if px + py + pz > deg:
                continue
            exact = factorial(px) * factorial(py) * factorial(pz) / factorial(px + py + pz + 3)
            got = (qw * qp[:, 0] ** px * qp[:, 1] ** py * qp[:, 2] ** pz).sum()
            assert abs(got - exact) < 1e-15


# ----------------------------------------------------------- autodiff equality
def _torch_element(et, Xe, Ue, lam, mu):
    """NeoHookeanAutodiff restated with torch float64 autograd."""
    import torch
    qp, qw, gr, gg = _indep_tables(et)
    Xe = torch.tensor(Xe, dtype=torch.float64)
    grt = torch.tensor(gr)
    ggt = torch.tensor(gg)

    def energy(uflat):
        U = uflat.reshape(-1, 3)
        e = torch.zeros((), dtype=torch.float64)
        for q in range(len(qw)):
            Jac = ggt[q].T @ Xe                 # rows d/dxi_r
            Jit = torch.linalg.inv(Jac).T
            gphi = grt[q] @ Jit                 # n x 3
            F = torch.eye(3, dtype=torch.float64) + U.T @ gphi
            J = torch.linalg.det(F)
            lj = torch.log(J)
            psi = mu / 2 * ((F * F).sum() - 3 - 2 * lj) + lam / 2 * lj * lj
            e = e + psi * torch.linalg.det(Jac) * qw[q]
        return e

    u0 = torch.tensor(Ue.ravel(), dtype=torch.float64, requires_grad=True)
    E0 = energy(u0)
    (g0,) = torch.autograd.grad(E0, u0)
    H0 = torch.autograd.functional.hessian(energy, u0.detach())
    return float(E0.detach()), g0.numpy(), H0.numpy()


@pytest.mark.parametrize("et", ELEMS, ids=lambda e: ELEM_NAMES[e])
def test_element_autodiff_equality(et):
    mesh, lam, mu, u, _ = make_case(et, 2, seed=3, jitter=0.1)
    orc = Oracle(mesh, lam, mu)
    rng = np.random.default_rng(5)
    for e in rng.choice(mesh.n_elements, 4, replace=False):
        for scale in (0.02, 0.2):
            uu = u * (scale / 0.02)
            en, g, H = orc.element(int(e), uu)
            Xe = mesh.X[mesh.gconn[e]]
            Ue = uu.reshape(-1, 3)[mesh.conn[e]]
            ea, ga, Ha = _torch_element(et, Xe, Ue, lam[e], mu[e])
            if np.isnan(ea) or np.isnan(en):
                # inverted element: both sides must report NaN (test_assembler.cpp:178-181)
                assert np.isnan(ea) and np.isnan(en)
                continue
            assert abs(en - ea) <= 1e-11 * max(abs(ea), 1.0)
            assert rel_err(g, ga) < 1e-11
            assert rel_err(H, Ha) < 1e-11


# ----------------------------------------------------------- finite differences
@pytest.mark.parametrize("et", ELEMS, ids=lambda e: ELEM_NAMES[e])
def test_form_finite_differences(et):
    """tests/test_form_derivatives.cpp:166-226 method: SECOND-order FD, step 1e-7."""
    mesh, lam, mu, _, _ = make_case(et, 2, seed=1, lognormal=False)
    orc = Oracle(mesh, lam, mu)
    rng = np.random.default_rng(0)
    x = np.zeros(mesh.n_dofs)
    step = 1e-7
    for it in range(3):
        g = orc.gradient(x)
        d = rng.standard_normal(x.size)
        fd = (orc.energy(x + step * d) - orc.energy(x - step * d)) / (2 * step)
        assert abs(fd - g @ d) <= 1e-4 * max(1.0, abs(fd))
        o, i, v = orc.hessian(x)
        H = sp.csc_matrix((v, i, o), shape=(x.size, x.size))
        fdh = (orc.gradient(x + step * d) - orc.gradient(x - step * d)) / (2 * step)
        assert rel_err(H @ d, fdh) < 1e-5
        x = rng.uniform(-1, 1, x.size) / 100


# ----------------------------------------------------------- closed-form KATs
def _psi(F, lam, mu):
    J = np.linalg.det(F)
    return mu / 2 * ((F * F).sum() - 3 - 2 * np.log(J)) + lam / 2 * np.log(J) ** 2


@pytest.mark.parametrize("et", ELEMS, ids=lambda e: ELEM_NAMES[e])
def test_homogeneous_deformation_known_answer(et):
    """u = (F0 - I) x gives F = F0 everywhere: energy = |Omega| psi(F0), sum of forces = 0."""
    mesh, _, _, _, _ = make_case(et, 2, seed=2, jitter=0.15)
    lam, mu = M.homogeneous_lame(mesh.n_elements)
    F0 = np.array([[1.05, 0.02, -0.01], [0.01, 0.97, 0.03], [-0.02, 0.015, 1.02]])
    u = ((F0 - np.eye(3)) @ mesh.node_pos.T).T.ravel()
    orc = Oracle(mesh, lam, mu)
    vol = 1.0  # jitter keeps the unit cube's boundary
    assert abs(orc.energy(u) - vol * _psi(F0, lam[0], mu[0])) < 1e-10 * vol * _psi(F0, lam[0], mu[0])
    g = orc.gradient(u).reshape(-1, 3)
    assert np.abs(g.sum(axis=0)).max() < 1e-9 * np.abs(g).max()
    # pure rotation: zero energy, zero gradient
    th = 0.3
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    ur = ((R - np.eye(3)) @ mesh.node_pos.T).T.ravel()
    assert abs(orc.energy(ur)) < 1e-9 * mu[0]
    assert np.abs(orc.gradient(ur)).max() < 1e-9 * mu[0]


# ----------------------------------------------------------- pattern + threads
@pytest.mark.parametrize("et", ELEMS, ids=lambda e: ELEM_NAMES[e])
def test_fast_pattern_equals_triplet_pattern(et):
    mesh, lam, mu, u, _ = make_case(et, 2, seed=4)
    a = Oracle(mesh, lam, mu, n_threads=2)
    b = Oracle(mesh, lam, mu, n_threads=3, fast_pattern=True)
    oa, ia, va = a.hessian(u)
    ob, ib, vb = b.hessian(u)
    assert np.array_equal(oa, ob) and np.array_equal(ia, ib)
    assert rel_err(vb, va) < 1e-14
    n = mesh.conn.shape[1]
    for e in (0, mesh.n_elements - 1):
        for k in range(0, 9 * n * n, 7):
            assert a.slot(e, k) == b.slot(e, k)
    # second call goes through the slot map and must reproduce the first
    oa2, ia2, va2 = a.hessian(u)
    assert np.array_equal(ia2, ia) and rel_err(va2, va) < 1e-14
    H = sp.csc_matrix((va, ia, oa), shape=(mesh.n_dofs,) * 2)
    assert abs(H - H.T).max() <= 1e-13 * np.abs(va).max()


def test_thread_count_does_not_change_results():
    mesh, lam, mu, u, p = make_case(M.P2_TET, 2, seed=9)
    r1 = Oracle(mesh, lam, mu, n_threads=1)
    r4 = Oracle(mesh, lam, mu, n_threads=4)
    assert abs(r1.energy(u) - r4.energy(u)) <= 1e-13 * abs(r1.energy(u))
    assert rel_err(r4.gradient(u), r1.gradient(u)) < 1e-14
    assert rel_err(r4.material_vjp(u, p), r1.material_vjp(u, p)) < 1e-14
    assert rel_err(r4.shape_vjp(u, p), r1.shape_vjp(u, p)) < 1e-14


def test_geometry_cache_threshold_changes_nothing():
    mesh, lam, mu, u, _ = make_case(M.Q1_HEX, 2, seed=6, jitter=0.1)
    cached = Oracle(mesh, lam, mu, cache_size=10**9)
    uncached = Oracle(mesh, lam, mu, cache_size=0)
    assert cached.energy(u) == uncached.energy(u)
    assert np.array_equal(cached.gradient(u), uncached.gradient(u))


# ----------------------------------------------------------- adjoint terms
@pytest.mark.parametrize("et", ELEMS, ids=lambda e: ELEM_NAMES[e])
def test_material_vjp_finite_differences(et):
    """term[e] = -p . df/dlambda_e, term[E+e] = -p . df/dmu_e (ElasticForceDerivative.cpp:124-125)."""
    mesh, lam, mu, u, p = make_case(et, 2, seed=8)
    orc = Oracle(mesh, lam, mu)
    term = orc.material_vjp(u, p)
    E = mesh.n_elements
    for e in (0, E // 2, E - 1):
        for which, arr in ((0, lam), (1, mu)):
            h = 1e-6 * arr[e]
            ap, am = arr.copy(), arr.copy()
            ap[e] += h
            am[e] -= h
            lp, mp = (ap, mu) if which == 0 else (lam, ap)
            lm, mm = (am, mu) if which == 0 else (lam, am)
            fp = Oracle(mesh, lp, mp).gradient(u) @ p
            fm = Oracle(mesh, lm, mm).gradient(u) @ p
            fd = (fp - fm) / (2 * h)
            got = -term[e + which * E]
            assert abs(got - fd) <= 1e-6 * max(abs(fd), 1e-12) + 1e-9


@pytest.mark.parametrize("et", ELEMS, ids=lambda e: ELEM_NAMES[e])
def test_shape_vjp_finite_differences(et):
    """term[3v+d] = p . df/dX_{v,d} (ElasticForceDerivative.cpp:207-260)."""
    mesh, lam, mu, u, p = make_case(et, 2, seed=10, jitter=0.1)
    orc = Oracle(mesh, lam, mu)
    term = orc.shape_vjp(u, p)
    rng = np.random.default_rng(1)
    for v in rng.choice(mesh.n_geom_nodes, 5, replace=False):
        for d in range(3):
            h = 1e-6 * mesh.h
            mp_, mm_ = _moved(mesh, v, d, h), _moved(mesh, v, d, -h)
            fd = (Oracle(mp_, lam, mu).gradient(u) @ p - Oracle(mm_, lam, mu).gradient(u) @ p) / (2 * h)
            assert abs(term[3 * v + d] - fd) <= 1e-6 * max(abs(fd), 1.0)


def _moved(mesh, v, d, h):
    import copy
    m2 = copy.copy(mesh)
    m2.X = mesh.X.copy()
    m2.X[v, d] += h
    return m2


# ------------------------------------------------------ project_to_psd (CLAMP)
def test_project_psd_restatement_against_numpy_eigh():
    """ipc::project_to_psd (CLAMP) restated in the oracle == V max(l, 0) V^T from
    numpy's eigh; PSD matrices come back unchanged (bitwise)."""
    from oracle.binding import project_psd
    rng = np.random.default_rng(0)
    for m in (12, 24, 30):
        B = rng.standard_normal((m, m))
        A = B + B.T
        w, V = np.linalg.eigh(A)
        ref = (V * np.maximum(w, 0.0)) @ V.T
        P = project_psd(A)
        assert np.linalg.norm(P - ref) <= 1e-13 * np.linalg.norm(ref)
        assert np.allclose(P, P.T, rtol=0, atol=1e-13 * np.abs(P).max())
        C = B @ B.T + np.eye(m)
        assert np.array_equal(project_psd(C), C)


def test_projected_oracle_hessian_is_psd():
    from oracle.binding import Oracle
    mesh, lam, mu, _, _ = make_case(M.P1_TET, 2, seed=3)
    rng = np.random.default_rng(4)
    u = (-0.3 * mesh.node_pos + 0.02 * mesh.h * rng.standard_normal(mesh.node_pos.shape)).ravel()
    o, i, v = Oracle(mesh, lam, mu).hessian(u, project_psd=True)
    import scipy.sparse as sp
    H = sp.csc_matrix((v, i, o), shape=(mesh.n_dofs, mesh.n_dofs)).toarray()
    w = np.linalg.eigvalsh(0.5 * (H + H.T))
    assert w.min() >= -1e-10 * np.abs(w).max()


# ------------------------------------------------------ Dirichlet reduction
def test_project_hessian_known_answer():
    """BCLagrangianForm::project_hessian on a 4x4 matrix with dof 1 constrained."""
    from oracle.binding import project_gradient, project_hessian, reduced_to_full
    A = np.array([[4.0, 1.0, 0.0, 2.0],
                  [1.0, 5.0, 3.0, 0.0],
                  [0.0, 3.0, 6.0, 7.0],
                  [2.0, 0.0, 7.0, 8.0]])
    C = sp.csc_matrix(A)
    o, i, v = project_hessian(C.indptr, C.indices, C.data, [1])
    R = sp.csc_matrix((v, i, o), shape=(3, 3)).toarray()
    assert np.array_equal(R, A[np.ix_([0, 2, 3], [0, 2, 3])])
    assert list(o) == [0, 2, 4, 7] and list(i) == [0, 2, 1, 2, 0, 1, 2]
    assert np.array_equal(project_gradient(np.arange(4.0), [1]), [0.0, 2.0, 3.0])
    assert np.array_equal(reduced_to_full([10.0, 20.0, 30.0], [-1.0, -2.0, -3.0, -4.0], [1]), [10.0, -2.0, 20.0, 30.0])


def test_dense_matrix_cache_restatement():
    """DenseMatrixCache (MatrixCache.cpp:326-403): add_value sums duplicates, and
    get_matrix is the sparseView that drops exact zeros."""
    from oracle.binding import DenseMatrixCache
    c = DenseMatrixCache(3)
    c.add_value(0, 0, 0, 1.5)
    c.add_value(1, 0, 0, 2.0)
    c.add_value(0, 1, 2, 4.0)
    c.add_value(1, 1, 2, -4.0)  # cancels to an exact zero: not stored
    c.add_value(0, 2, 1, 7.0)
    assert c.mat[0, 0] == 3.5 and c.mat[1, 2] == 0.0
    m = c.get_matrix()
    assert m.nnz == 2 and m[0, 0] == 3.5 and m[2, 1] == 7.0
