"""The oracle's restatement of the GenericElastic materials (IsochoricNeoHookean,
SaintVenant): derivatives by central finite differences, as the reference checks its
forms (tests/test_form_derivatives.cpp:166-226), and closed-form known answers."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle.binding import Oracle
from polyfem_b200 import mesh as M

from _cases import make_case

MATS = ["IsochoricNeoHookean", "SaintVenant"]
ELEMS = [(M.P1_TET, "P1"), (M.P2_TET, "P2"), (M.Q1_HEX, "Q1")]


@pytest.mark.parametrize("mat", MATS)
@pytest.mark.parametrize("et,name", ELEMS, ids=[n for _, n in ELEMS])
def test_material_derivatives_finite_differences(mat, et, name):
    mesh, lam, mu, u, p = make_case(et, 2, seed=3, jitter=0.1 if et != M.P1_TET else 0.0, disp_scale=0.05)
    o = Oracle(mesh, lam, mu, material=mat)
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


@pytest.mark.parametrize("mat", MATS)
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
