"""Seeded small workloads shared by the tests (same generators as the benchmarks)."""
import numpy as np

from polyfem_b200 import mesh as M

ELEM_NAMES = {M.P1_TET: "P1", M.P2_TET: "P2", M.Q1_HEX: "Q1"}


def make_case(elem_type: int, g: int, seed: int = 0, jitter: float = 0.0, lognormal: bool = True,
              disp_scale: float = 0.02):
    if elem_type == M.P1_TET:
        mesh = M.structured_tet_mesh(g, 1, jitter=jitter, seed=seed + 7)
    elif elem_type == M.P2_TET:
        mesh = M.structured_tet_mesh(g, 2, jitter=jitter, seed=seed + 7)
    else:
        mesh = M.structured_hex_mesh(g, jitter=jitter, seed=seed + 7)
    if lognormal:
        lam, mu = M.lognormal_lame(mesh.n_elements, seed + 11)
    else:
        lam, mu = M.homogeneous_lame(mesh.n_elements)
    u = M.random_displacement(mesh, disp_scale, seed + 13)
    p = np.random.default_rng(seed + 17).standard_normal(mesh.n_dofs)
    return mesh, lam, mu, u, p


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
