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


def permuted(mesh, u, seed=0):
    """The same mesh with elements, FE nodes and geometric nodes renumbered at
    random (no locality left).  Returns (mesh', u', node_perm, elem_perm): FE node
    i becomes node_perm[i], element elem_perm[k] becomes element k, and
    u'[3*node_perm[i] + d] = u[3*i + d]."""
    import copy
    rng = np.random.default_rng(seed)
    m2 = copy.copy(mesh)
    pe = rng.permutation(mesh.n_elements)
    pn = rng.permutation(mesh.n_nodes)
    m2.conn = np.ascontiguousarray(pn[mesh.conn[pe]].astype(np.int32))
    node_pos = np.empty_like(mesh.node_pos)
    node_pos[pn] = mesh.node_pos
    m2.node_pos = node_pos
    X = np.empty_like(mesh.X)
    if mesh.gconn is mesh.conn:
        m2.gconn = m2.conn
        X[pn] = mesh.X
    else:
        pg = rng.permutation(mesh.n_geom_nodes)
        m2.gconn = np.ascontiguousarray(pg[mesh.gconn[pe]].astype(np.int32))
        X[pg] = mesh.X
    m2.X = X
    u2 = np.empty_like(u)
    u2.reshape(-1, 3)[pn] = u.reshape(-1, 3)
    return m2, u2, pn, pe


# GenericMatParam names of the parameterised formulations (MooneyRivlinElasticity.hpp,
# MooneyRivlin3ParamElasticity.hpp, VolumePenalty.hpp)
MATERIAL_PARAM_NAMES = {"MooneyRivlin": ("c1", "c2", "k"), "MooneyRivlin3Param": ("c1", "c2", "c3", "d1"),
                        "VolumePenalty": ("k",), "MooneyRivlin3ParamSymbolic": ("c1", "c2", "c3", "d1")}


def hooke_tensor(seed=0, lam=86419.75, mu=37037.04):
    """21 entries (i <= j, row by row) of a seeded anisotropic elasticity tensor: the
    isotropic (lam, mu) tensor plus a random symmetric positive semi-definite part
    that couples every pair of Voigt components."""
    rng = np.random.default_rng(seed)
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    C[[0, 1, 2], [0, 1, 2]] = 2 * mu + lam
    C[[3, 4, 5], [3, 4, 5]] = mu
    R = rng.standard_normal((6, 6))
    C += 1e4 * (R @ R.T) / 6
    return C[np.triu_indices(6)]


def material_params(mat, n_elements, seed=0):
    """Per-element parameter values of a parameterised material (stress scale ~1e5);
    the one elasticity tensor of HookeLinearElasticity and of the anisotropic
    SaintVenant (the oracle's "SaintVenantTensor")."""
    if mat in ("HookeLinearElasticity", "SaintVenantTensor"):
        return {"elasticity_tensor": hooke_tensor(seed)}
    rng = np.random.default_rng(seed)
    if mat == "UnconstrainedOgden":  # two terms (alpha, mu, D), a rubber-like fit
        f = lambda v: v * rng.uniform(0.8, 1.2, n_elements)
        return {"alphas": [f(1.3), f(5.0)], "mus": [f(1.2e5), f(2.0e3)], "Ds": [f(2e-6), f(5e-5)]}
    if mat == "IncompressibleOgden":  # three terms (c, m) with a negative exponent, and k
        f = lambda v: v * rng.uniform(0.8, 1.2, n_elements)
        return {"c": [f(1.5e5), f(4.0e3), f(-3.0e3)], "m": [f(1.3), f(5.0), f(-2.0)], "k": f(8e5)}
    return {n: 1e5 * rng.uniform(0.5, 1.5, n_elements) for n in MATERIAL_PARAM_NAMES.get(mat, ())}
