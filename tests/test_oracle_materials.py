"""The oracle's restatement of the other elastic formulations (IsochoricNeoHookean,
SaintVenant, LinearElasticity, MooneyRivlin, MooneyRivlin3Param, VolumePenalty,
HookeLinearElasticity, UnconstrainedOgden, IncompressibleOgden):
derivatives by central finite differences, as the reference checks its forms
(tests/test_form_derivatives.cpp:166-226), and closed-form known answers."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle.binding import Oracle
from polyfem_b200 import mesh as M

from _cases import make_case, material_params

MATS = ["IsochoricNeoHookean", "SaintVenant", "LinearElasticity", "MooneyRivlin", "MooneyRivlin3Param",
        "VolumePenalty", "HookeLinearElasticity", "SaintVenantTensor", "UnconstrainedOgden", "IncompressibleOgden",
        "MooneyRivlin3ParamSymbolic"]
ELEMS = [(M.P1_TET, "P1"), (M.P2_TET, "P2"), (M.Q1_HEX, "Q1")]


@pytest.mark.parametrize("mat", MATS)
@pytest.mark.parametrize("et,name", ELEMS, ids=[n for _, n in ELEMS])
def test_material_derivatives_finite_differences(mat, et, name):
    mesh, lam, mu, u, p = make_case(et, 2, seed=3, jitter=0.1 if et != M.P1_TET else 0.0, disp_scale=0.05)
    o = Oracle(mesh, lam, mu, material=mat, params=material_params(mat, mesh.n_elements))
    g = o.gradient(u)
    h = 1e-6 * np.abs(u).max() / np.abs(p).max()
    fd = (o.energy(u + h * p) - o.energy(u - h * p)) / (2 * h)
    assert abs(g @ p - fd) <= 1e-7 * abs(fd)
    outer, inner, vals = o.hessian(u)
    H = sp.csc_matrix((vals, inner, outer), shape=(mesh.n_dofs, mesh.n_dofs))
    fdg = (o.gradient(u + h * p) - o.gradient(u - h * p)) / (2 * h)
    assert np.linalg.norm(H @ p - fdg) <= 1e-7 * np.linalg.norm(fdg)
    assert abs(H - H.T).max() <= 1e-14 * abs(H).max()
    assert np.isclose(o.energy_per_element(u).sum(), o.energy(u), rtol=1e-13)


@pytest.mark.parametrize("mat", MATS[:2])
def test_material_known_answers(mat):
    mesh, lam, mu, _, _ = make_case(M.P2_TET, 2, seed=4)
    o = Oracle(mesh, lam, mu, material=mat)
    scale = float(np.median(mu)) * 1.0  # energy density scale of a unit strain
    # rest state: zero energy and zero gradient
    assert abs(o.energy(np.zeros(mesh.n_dofs))) <= 1e-12 * scale
    assert np.abs(o.gradient(np.zeros(mesh.n_dofs))).max() <= 1e-10 * scale
    # a rigid rotation stores no energy
    th = 0.7
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    ur = (mesh.node_pos @ R.T - mesh.node_pos).ravel()
    assert abs(o.energy(ur)) <= 1e-11 * scale
    # a uniform dilation F = s I
    s_ = 1.3
    us = ((s_ - 1) * mesh.node_pos).ravel()
    if mat == "IsochoricNeoHookean":
        assert abs(o.energy(us)) <= 1e-11 * scale  # isochoric: no energy in volume change
    else:
        e = 0.5 * (s_ * s_ - 1)  # E = e I: psi = lambda/2 (3e)^2 + mu 3 e^2, volume 1
        lam_v, mu_v = np.asarray(lam), np.asarray(mu)
        vol = o.energy_per_element(us) / (lam_v / 2 * 9 * e * e + mu_v * 3 * e * e)
        assert np.isclose(vol.sum(), 1.0, rtol=1e-12)



def _uniform(mesh, F):
    """Displacement of the homogeneous deformation x -> F x."""
    return (mesh.node_pos @ (np.asarray(F) - np.eye(3)).T).ravel()


def test_energy_defined_materials_known_answers():
    """Homogeneous deformations of the unit cube, where psi is known in closed form:
    the energy is psi times the volume (1) for every element type."""
    for et in (M.P1_TET, M.P2_TET, M.Q1_HEX):
        mesh, lam, mu, _, _ = make_case(et, 2, seed=4)
        E = mesh.n_elements
        lam1, mu1 = 2.0e5, 0.7e5
        lam = np.full(E, lam1)
        mu = np.full(E, mu1)
        c1, c2, c3, d1, k = 1.1e5, 0.4e5, 0.3e5, 2.0e5, 3.0e5
        s_, th, g_, a_ = 1.2, 0.6, 0.3, 1.25
        dil = np.eye(3) * s_
        rot = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
        shear = np.eye(3) + g_ * np.outer([1, 0, 0], [0, 1, 0])
        iso = np.diag([a_, a_ ** -0.5, a_ ** -0.5])  # J = 1
        I1, I2 = a_ ** 2 + 2 / a_, 2 * a_ + 1 / a_ ** 2  # invariants of F F^T for iso
        cases = {
            "LinearElasticity": ({}, [(dil, mu1 * 3 * (s_ - 1) ** 2 + lam1 / 2 * 9 * (s_ - 1) ** 2),
                                      (rot, mu1 * 2 * (np.cos(th) - 1) ** 2 + lam1 / 2 * 4 * (np.cos(th) - 1) ** 2),
                                      (shear, mu1 * g_ ** 2 / 2)]),
            "MooneyRivlin": ({"c1": c1, "c2": c2, "k": k}, [(dil, k / 2 * (3 * np.log(s_)) ** 2), (rot, 0.0),
                                                            (iso, c1 * (I1 - 3) + c2 * (I2 - 3))]),
            "MooneyRivlin3Param": ({"c1": c1, "c2": c2, "c3": c3, "d1": d1},
                                   [(dil, d1 * (s_ ** 3 - 1) ** 2), (rot, 0.0),
                                    (iso, c1 * (I1 - 3) + (c2 + c3 * (I1 - 3)) * (I2 - 3))]),
            "VolumePenalty": ({"k": k}, [(dil, k / 2 * ((s_ ** 6 - 1) / 2 - 3 * np.log(s_))), (rot, 0.0), (iso, 0.0)]),
            "MooneyRivlin3ParamSymbolic": ({"c1": c1, "c2": c2, "c3": c3, "d1": d1},
                                           [(dil, d1 * (3 * np.log(s_)) ** 2), (rot, 0.0),
                                            (iso, c1 * (I1 - 3) + c2 * (I2 - 3) + c3 * (I1 - 3) * (I2 - 3))]),
        }
        for mat, (prm, checks) in cases.items():
            o = Oracle(mesh, lam, mu, material=mat, params=prm)
            assert abs(o.energy(np.zeros(mesh.n_dofs))) <= 1e-12 * c1
            assert np.abs(o.gradient(np.zeros(mesh.n_dofs))).max() <= 1e-9 * c1
            for F, psi in checks:
                assert abs(o.energy(_uniform(mesh, F)) - psi) <= 1e-11 * max(abs(psi), c1), (mat, et, psi)


def test_linear_elasticity_hessian_is_constant():
    """LinearElasticity is quadratic in u: the Hessian does not depend on u and the
    energy is 1/2 u^T H u."""
    mesh, lam, mu, u, _ = make_case(M.P2_TET, 2, seed=6, jitter=0.1)
    o = Oracle(mesh, lam, mu, material="LinearElasticity")
    outer, inner, v0 = o.hessian(np.zeros(mesh.n_dofs))
    _, _, v1 = o.hessian(u)
    assert np.abs(v1 - v0).max() <= 1e-9 * np.abs(v0).max()
    H = sp.csc_matrix((v0, inner, outer), shape=(mesh.n_dofs, mesh.n_dofs))
    assert np.isclose(0.5 * u @ (H @ u), o.energy(u), rtol=1e-12)


def test_saint_venant_tensor_known_answers():
    """SaintVenant with the isotropic tensor of (lambda, mu) given as 21 entries is the
    lambda/mu SaintVenant; with an anisotropic tensor and a homogeneous deformation
    F the energy is |domain| 1/2 e.C e, e the Voigt Green strain with doubled shears."""
    from polyfem_b200 import NeoHookeanAssembler
    from _cases import hooke_tensor
    mesh, lam, mu, u, _ = make_case(M.Q1_HEX, 2, seed=26, jitter=0.1, disp_scale=0.05)
    lam0, mu0 = 7.5e4, 3.2e4
    E = mesh.n_elements
    iso = NeoHookeanAssembler.isotropic_elasticity_tensor(lam0, mu0)
    o_t = Oracle(mesh, np.full(E, lam0), np.full(E, mu0), material="SaintVenantTensor",
                 params={"elasticity_tensor": iso})
    o_s = Oracle(mesh, np.full(E, lam0), np.full(E, mu0), material="SaintVenant")
    assert np.isclose(o_t.energy(u), o_s.energy(u), rtol=1e-13)
    gs = o_s.gradient(u)
    assert np.abs(o_t.gradient(u) - gs).max() <= 1e-13 * np.abs(gs).max()
    c21 = hooke_tensor(27)
    C = np.zeros((6, 6))
    C[np.triu_indices(6)] = c21
    C = C + np.triu(C, 1).T
    G = np.random.default_rng(28).normal(scale=5e-2, size=(3, 3))
    uh = (mesh.node_pos @ G.T).ravel()
    F = np.eye(3) + G
    Eg = 0.5 * (F.T @ F - np.eye(3))
    e = np.array([Eg[0, 0], Eg[1, 1], Eg[2, 2], 2 * Eg[1, 2], 2 * Eg[0, 2], 2 * Eg[0, 1]])
    o = Oracle(mesh, lam, mu, material="SaintVenantTensor", params={"elasticity_tensor": c21})
    assert np.isclose(o.energy(uh), 0.5 * e @ C @ e, rtol=1e-12)  # unit cube


def test_hooke_known_answers():
    """HookeLinearElasticity: with the isotropic tensor of (lambda, mu)
    (ElasticityTensor::set_from_lambda_mu) it is LinearElasticity; with an
    anisotropic tensor and a homogeneous strain u = G x the energy is
    |domain| 1/2 v.C v (v the Voigt strain with doubled shears), the Hessian is
    constant and the energy is 1/2 u^T H u."""
    from polyfem_b200 import NeoHookeanAssembler
    from _cases import hooke_tensor
    mesh, lam, mu, u, _ = make_case(M.P2_TET, 2, seed=21, jitter=0.1, disp_scale=0.05)
    lam0, mu0 = 7.5e4, 3.2e4
    iso = NeoHookeanAssembler.isotropic_elasticity_tensor(lam0, mu0)
    E = mesh.n_elements
    o_h = Oracle(mesh, np.full(E, lam0), np.full(E, mu0), material="HookeLinearElasticity",
                 params={"elasticity_tensor": iso})
    o_l = Oracle(mesh, np.full(E, lam0), np.full(E, mu0), material="LinearElasticity")
    assert np.isclose(o_h.energy(u), o_l.energy(u), rtol=1e-13)
    assert np.allclose(o_h.gradient(u), o_l.gradient(u), rtol=0, atol=1e-13 * np.abs(o_l.gradient(u)).max())
    c21 = hooke_tensor(22)
    C = np.zeros((6, 6))
    C[np.triu_indices(6)] = c21
    C = C + np.triu(C, 1).T
    G = np.random.default_rng(23).normal(scale=1e-2, size=(3, 3))
    uh = (mesh.node_pos @ G.T).ravel()
    v = np.array([G[0, 0], G[1, 1], G[2, 2], G[1, 2] + G[2, 1], G[0, 2] + G[2, 0], G[0, 1] + G[1, 0]])
    o = Oracle(mesh, lam, mu, material="HookeLinearElasticity", params={"elasticity_tensor": c21})
    assert np.isclose(o.energy(uh), 0.5 * v @ C @ v, rtol=1e-12)  # unit cube
    outer, inner, h0 = o.hessian(np.zeros(mesh.n_dofs))
    _, _, h1 = o.hessian(u)
    assert np.abs(h1 - h0).max() <= 1e-9 * np.abs(h0).max()
    H = sp.csc_matrix((h0, inner, outer), shape=(mesh.n_dofs, mesh.n_dofs))
    assert np.isclose(0.5 * u @ (H @ u), o.energy(u), rtol=1e-12)


@pytest.mark.parametrize("et", [M.P1_TET, M.P2_TET, M.Q1_HEX], ids=["P1", "P2", "Q1"])
def test_oracle_mass_matrix_known_answers(et):
    """The oracle's mass matrix: symmetric, in the Hessian's pattern, total mass
    rho * volume; its basis values are the antiderivatives of the gradient tables the
    stiffness uses (same node order)."""
    mesh, lam, mu, u, _ = make_case(et, 2, seed=13, jitter=0.1 if et != M.P1_TET else 0.0)
    o = Oracle(mesh, lam, mu)
    outer, inner, vals = o.mass_matrix(np.full(mesh.n_elements, 2.5))
    Mm = sp.csc_matrix((vals, inner, outer), shape=(mesh.n_dofs, mesh.n_dofs))
    assert abs(Mm - Mm.T).max() == 0.0
    ho, hi, _ = o.hessian(u)
    assert np.array_equal(ho, outer) and np.array_equal(hi, inner)
    ex = np.zeros(mesh.n_dofs)
    ex[1::3] = 1.0
    assert abs(ex @ (Mm @ ex) - 2.5) <= 1e-12
    from oracle.binding import lib as olib, tables
    L = olib()
    qp, qw, gr, _ = tables(et)
    nq, n = gr.shape[0], gr.shape[1]
    h = 1e-6
    for q in range(nq):
        for i in range(n):
            for d in range(3):
                xp, xm = qp[q].copy(), qp[q].copy()
                xp[d] += h
                xm[d] -= h
                fd = (L.orc_basis_value(et, i, *xp) - L.orc_basis_value(et, i, *xm)) / (2 * h)
                assert abs(fd - gr[q, i, d]) <= 1e-8
    vals_q = [sum(L.orc_basis_value(et, i, *qp[q]) for i in range(n)) for q in range(nq)]
    assert np.allclose(vals_q, 1.0, atol=1e-14)  # partition of unity


def test_oracle_p1_mass_closed_form():
    """On an affine P1 tet, int lambda_a lambda_b dV = |T| (1 + delta_ab) / 20: the
    oracle's quadrature (its own conical-product Gauss rule) must reproduce it."""
    mesh, lam, mu, _, _ = make_case(M.P1_TET, 1, seed=3)
    o = Oracle(mesh, lam, mu)
    rho = np.arange(1, mesh.n_elements + 1, dtype=float)
    outer, inner, vals = o.mass_matrix(rho)
    Mx = sp.csc_matrix((vals, inner, outer), shape=(mesh.n_dofs, mesh.n_dofs)).toarray()[0::3, 0::3]
    ref = np.zeros((mesh.n_nodes, mesh.n_nodes))
    for e in range(mesh.n_elements):
        Xe = mesh.X[mesh.gconn[e]]
        vol = np.linalg.det(np.stack([Xe[1] - Xe[0], Xe[2] - Xe[0], Xe[3] - Xe[0]], 1)) / 6
        ref[np.ix_(mesh.conn[e], mesh.conn[e])] += rho[e] * vol * (np.ones((4, 4)) + np.eye(4)) / 20
    assert np.abs(Mx - ref).max() <= 1e-14 * np.abs(ref).max()


# ----------------------------------------------------------- adjoint terms
SHAPE_MATS = ["IsochoricNeoHookean", "LinearElasticity", "MooneyRivlin", "MooneyRivlin3Param", "VolumePenalty",
              "UnconstrainedOgden", "IncompressibleOgden", "MooneyRivlin3ParamSymbolic"]


def _moved(mesh, v, d, h):
    import copy
    m2 = copy.copy(mesh)
    m2.X = mesh.X.copy()
    m2.X[v, d] += h
    return m2


@pytest.mark.parametrize("mat", SHAPE_MATS)
@pytest.mark.parametrize("et,name", [(M.P2_TET, "P2"), (M.Q1_HEX, "Q1")], ids=["P2", "Q1"])
def test_shape_vjp_finite_differences_other_materials(mat, et, name):
    """term[3v+d] = p . df/dX_{v,d}, with P and C:(grad u V) from the material's dual
    numbers (GenericElastic / LinearElasticity compute_stress_grad_multiply_mat)."""
    mesh, lam, mu, u, p = make_case(et, 2, seed=10, jitter=0.1, disp_scale=0.05)
    prm = material_params(mat, mesh.n_elements, seed=10)
    orc = Oracle(mesh, lam, mu, material=mat, params=prm)
    term = orc.shape_vjp(u, p)
    rng = np.random.default_rng(1)
    for v in rng.choice(mesh.n_geom_nodes, 4, replace=False):
        for d in range(3):
            h = 1e-5 * mesh.h  # between the O(h^2) truncation (8e-6 at 1e-4 h) and rounding (3e-6 at 1e-6 h)
            fp = Oracle(_moved(mesh, v, d, h), lam, mu, material=mat, params=prm).gradient(u) @ p
            fm = Oracle(_moved(mesh, v, d, -h), lam, mu, material=mat, params=prm).gradient(u) @ p
            fd = (fp - fm) / (2 * h)
            assert abs(term[3 * v + d] - fd) <= 1e-6 * max(abs(fd), 1.0), (mat, v, d, term[3 * v + d], fd)


def test_linear_elasticity_material_vjp_finite_differences():
    """LinearElasticity's term[e] = -p . df/dlambda_e, term[E+e] = -p . df/dmu_e."""
    mesh, lam, mu, u, p = make_case(M.P2_TET, 2, seed=8)
    orc = Oracle(mesh, lam, mu, material="LinearElasticity")
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
            fp = Oracle(mesh, lp, mp, material="LinearElasticity").gradient(u) @ p
            fm = Oracle(mesh, lm, mm, material="LinearElasticity").gradient(u) @ p
            fd = (fp - fm) / (2 * h)
            assert abs(-term[e + which * E] - fd) <= 1e-6 * max(abs(fd), 1e-12) + 1e-9


def test_ogden_known_answers():
    """Homogeneous deformations F = R diag(a, b, c) of the unit cube: the principal
    stretches are (a, b, c), so both Ogden energies are known in closed form; zero
    energy and gradient at rest, and under a rotation."""
    a, b, c = 1.15, 0.93, 1.04
    J = a * b * c
    th = 0.5
    R = np.array([[np.cos(th), 0, np.sin(th)], [0, 1, 0], [-np.sin(th), 0, np.cos(th)]])
    F = R @ np.diag([a, b, c])
    st = np.array([a, b, c]) * J ** (-1 / 3)
    al, mu_, D = [1.3, 5.0], [1.2e5, 2.0e3], [2e-6, 5e-5]
    cs, ms, k = [1.5e5, 4.0e3, -3.0e3], [1.3, 5.0, -2.0], 8e5
    psi_u = sum(2 * m_ / x ** 2 * ((st ** x).sum() - 3) for x, m_ in zip(al, mu_)) + \
        sum((J - 1) ** (2 * (t + 1)) / D[t] for t in range(2))
    psi_i = sum(c_ / m_ ** 2 * ((st ** m_).sum() - 3) for c_, m_ in zip(cs, ms)) + 0.5 * k * np.log(J) ** 2
    for et in (M.P1_TET, M.P2_TET, M.Q1_HEX):
        mesh, lam, mu, _, _ = make_case(et, 2, seed=4)
        for mat, prm, psi in (("UnconstrainedOgden", {"alphas": al, "mus": mu_, "Ds": D}, psi_u),
                              ("IncompressibleOgden", {"c": cs, "m": ms, "k": k}, psi_i)):
            o = Oracle(mesh, lam, mu, material=mat, params=prm)
            assert abs(o.energy(np.zeros(mesh.n_dofs))) <= 1e-12 * 1e5
            assert np.abs(o.gradient(np.zeros(mesh.n_dofs))).max() <= 1e-9 * 1e5
            assert abs(o.energy(_uniform(mesh, R))) <= 1e-9 * 1e5
            assert abs(o.energy(_uniform(mesh, F)) - psi) <= 1e-10 * abs(psi), (mat, et)
