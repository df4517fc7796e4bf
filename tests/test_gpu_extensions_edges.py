"""Edge cases of the added entry points (pfg_set_material, pfg_mass_matrix,
pfg_cg_solve): an empty mesh, a single element of every type, and NaN from an
inverted element under IsochoricNeoHookean (J^(-2/3) of a negative J)."""
import numpy as np
import pytest

from oracle.binding import Oracle
from polyfem_b200 import ConjugateGradient, NeoHookeanAssembler
from polyfem_b200 import mesh as M

from _cases import make_case, rel_err

pytestmark = pytest.mark.gpu


def test_empty_mesh_extensions(require_gpu):
    conn = np.zeros((0, 4), dtype=np.int32)
    asm = NeoHookeanAssembler(M.P1_TET, conn, np.zeros((5, 3)), np.zeros(0), np.zeros(0), n_nodes=5)
    u = np.zeros(15)
    assert asm.assemble_mass_matrix_values().size == 0
    for mat in ("IsochoricNeoHookean", "SaintVenant"):
        asm.set_material(mat)
        assert asm.assemble_energy(u) == 0.0
        assert np.all(asm.assemble_gradient(u) == 0.0)
        assert asm.assemble_hessian_values(u).size == 0
    asm.set_material("NeoHookean")
    asm.assemble_hessian_values(u)
    cg = ConjugateGradient(asm, "full")
    cg.set_parameters({"max_iter": 5})
    x = cg.solve(np.ones(15))  # no element, H = 0: p.Hp = 0, the iteration runs to the cap as Eigen's does
    assert x.shape == (15,) and cg.get_info()["solver_iter"] == 5
    asm.close()


def single(et, seed=31):
    mesh, lam, mu, u, _ = make_case(et, 1, seed=seed, jitter=0.0)
    conn, gconn = mesh.conn[:1], mesh.gconn[:1]
    used, gused = np.unique(conn), np.unique(gconn)
    remap = -np.ones(mesh.n_nodes, dtype=np.int64)
    remap[used] = np.arange(used.size)
    gremap = -np.ones(mesh.n_geom_nodes, dtype=np.int64)
    gremap[gused] = np.arange(gused.size)
    sub = M.Mesh(et, remap[conn].astype(np.int32), gremap[gconn].astype(np.int32), mesh.X[gused],
                 used.size, mesh.node_pos[used], mesh.h, 1)
    if et != M.P2_TET:
        sub.gconn = sub.conn
    return sub, lam[:1], mu[:1], u.reshape(-1, 3)[used].ravel()


@pytest.mark.parametrize("et", [M.P1_TET, M.P2_TET, M.Q1_HEX], ids=["P1", "P2", "Q1"])
def test_single_element_extensions(require_gpu, et):
    sub, lam, mu, us = single(et)
    asm = NeoHookeanAssembler.from_mesh(sub, lam, mu)
    _, _, mv = Oracle(sub, lam, mu).mass_matrix()
    assert rel_err(asm.assemble_mass_matrix_values(), mv) <= 1e-13
    for mat in ("IsochoricNeoHookean", "SaintVenant"):
        orc = Oracle(sub, lam, mu, material=mat)
        asm.set_material(mat)
        assert abs(asm.assemble_energy(us) - orc.energy(us)) <= 1e-12 * abs(orc.energy(us))
        assert rel_err(asm.assemble_gradient(us), orc.gradient(us)) <= 1e-12
        assert rel_err(asm.assemble_hessian_values(us), orc.hessian(us)[2]) <= 1e-12
    asm.close()


def test_inverted_element_nan_isochoric(require_gpu):
    mesh, lam, mu, u, _ = make_case(M.P1_TET, 2, seed=17)
    bad = np.zeros(mesh.n_dofs)
    # move vertex 3 of element 0 through the opposite face: the element turns inside out
    c = mesh.conn[0]
    X = mesh.node_pos
    bad.reshape(-1, 3)[c[3]] = 2.0 * (X[c[:3]].mean(axis=0) - X[c[3]])
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.set_material("IsochoricNeoHookean")
    orc = Oracle(mesh, lam, mu, material="IsochoricNeoHookean")
    assert np.isnan(orc.energy(bad)) and np.isnan(asm.assemble_energy(bad))
    assert np.array_equal(np.isnan(asm.assemble_gradient(bad)), np.isnan(orc.gradient(bad)))
    assert asm.inverted_count() >= 1
    asm.close()
