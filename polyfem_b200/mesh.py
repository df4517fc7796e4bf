"""Structured synthetic meshes with PolyFEM's node-numbering rules.

The assembly path only consumes three arrays per mesh, exactly what PolyFEM's
``Basis::global()`` tables and geometric bases hand to ``NLAssembler``:

* ``conn``  (E x n, int32): FE node index of each local basis function;
* ``gconn`` (E x n_g, int32): geometric node index of each local geometric basis;
* ``X``     (N_g x 3, float64): rest position of each geometric node.

Numbering follows ``MeshNodes::node_id_from_primitive`` (mesh/MeshNodes.cpp:159-175):
a node gets the next free id the first time an element touches its primitive,
visiting elements in order and, inside an element, the local order of
``tet_local_to_global`` (basis/LagrangeBasis3d.cpp:238-300): the 4 vertices, then
the edges (v0v1, v1v2, v2v0, v0v3, v1v3, v2v3).  For P2 on a linear mesh the
geometry is P1 with its own vertex numbering (State.cpp:466-491), so ``gconn`` and
``conn`` differ; for P1 and Q1 the bases are isoparametric and ``gconn is conn``.

Tetrahedra come from a Kuhn split of each grid cell along the v000->v111 diagonal
(6 tets per cell, one per axis permutation, all positively oriented); hexahedra
use the Q1 local vertex order of autogen/auto_q_bases_3d_nodes.cpp:12-22.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from itertools import permutations

import numpy as np

P1_TET = 1
P2_TET = 2
Q1_HEX = 3

NODES_PER_ELEMENT = {P1_TET: 4, P2_TET: 10, Q1_HEX: 8}
GEOM_NODES_PER_ELEMENT = {P1_TET: 4, P2_TET: 4, Q1_HEX: 8}
QUAD_POINTS_PER_ELEMENT = {P1_TET: 1, P2_TET: 4, Q1_HEX: 8}

# Local edge order of a P2 tetrahedron (LagrangeBasis3d.cpp:275-281).
TET_EDGES = ((0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3))
# Q1 reference-cube corner order (auto_q_bases_3d_nodes.cpp:12-22).
HEX_CORNERS = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
               (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))


@dataclass
class Mesh:
    """A mesh in the form the assembly boundary consumes."""
    elem_type: int
    conn: np.ndarray            # (E, n) int32, FE node ids
    gconn: np.ndarray           # (E, n_g) int32, geometric node ids
    X: np.ndarray               # (N_g, 3) float64 rest positions of geometric nodes
    n_nodes: int                # N (FE nodes)
    node_pos: np.ndarray        # (N, 3) float64 rest positions of FE nodes
    h: float                    # grid spacing
    grid: int                   # cells per axis
    meta: dict = field(default_factory=dict)

    @property
    def n_elements(self) -> int:
        return int(self.conn.shape[0])

    @property
    def n_geom_nodes(self) -> int:
        return int(self.X.shape[0])

    @property
    def n_dofs(self) -> int:
        return 3 * self.n_nodes


def _first_touch(prims: np.ndarray):
    """Renumber primitive ids in order of first appearance in the flattened list.

    Returns (new_ids of the flattened list reshaped like ``prims``, order) where
    ``order[k]`` is the primitive that received node id k.
    """
    flat = prims.reshape(-1)
    uniq, first_idx, inverse = np.unique(flat, return_index=True, return_inverse=True)
    order_of_uniq = np.argsort(first_idx, kind="stable")
    rank = np.empty_like(order_of_uniq)
    rank[order_of_uniq] = np.arange(order_of_uniq.size)
    new_ids = rank[inverse].reshape(prims.shape).astype(np.int32)
    return new_ids, uniq[order_of_uniq]


def _grid_vertices(g: int, jitter: float, seed: int):
    h = 1.0 / g
    idx = np.arange(g + 1)
    k, j, i = np.meshgrid(idx, idx, idx, indexing="ij")
    pos = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64) * h
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        d = rng.uniform(-1.0, 1.0, size=pos.shape) * (jitter * h)
        interior = np.all((np.stack([i.ravel(), j.ravel(), k.ravel()], 1) > 0)
                          & (np.stack([i.ravel(), j.ravel(), k.ravel()], 1) < g), axis=1)
        pos[interior] += d[interior]
    return pos, h


def _vid(i, j, k, g):
    return i + (g + 1) * (j + (g + 1) * k)


def _kuhn_tets(g: int, pos: np.ndarray) -> np.ndarray:
    """(6*g^3, 4) vertex ids of the Kuhn split, cells in lexicographic order."""
    c = np.arange(g)
    ck, cj, ci = np.meshgrid(c, c, c, indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    unit = np.eye(3, dtype=np.int64)
    tets = []
    for perm in permutations(range(3)):
        a = np.zeros(3, dtype=np.int64)
        b = a + unit[perm[0]]
        cc = b + unit[perm[1]]
        d = np.ones(3, dtype=np.int64)
        loc = [a, b, cc, d]
        # orientation of the un-jittered reference tet decides the vertex order
        m = np.stack([loc[1] - loc[0], loc[2] - loc[0], loc[3] - loc[0]])
        if np.linalg.det(m.astype(np.float64)) < 0:
            loc = [loc[0], loc[1], loc[3], loc[2]]
        tets.append(np.stack([_vid(ci + p[0], cj + p[1], ck + p[2], g) for p in loc], axis=1))
    out = np.stack(tets, axis=1).reshape(-1, 4)  # cell-major, 6 tets per cell
    return out.astype(np.int64)


def structured_tet_mesh(g: int, order: int = 1, jitter: float = 0.0, seed: int = 0) -> Mesh:
    """Unit cube, g^3 cells, 6 tets per cell; P1 (order=1) or P2 (order=2) nodes."""
    pos, h = _grid_vertices(g, jitter, seed)
    tv = _kuhn_tets(g, pos)
    if order == 1:
        conn, vorder = _first_touch(tv)
        X = pos[vorder]
        return Mesh(P1_TET, conn, conn, X, X.shape[0], X, h, g,
                    {"jitter": jitter, "seed": seed})
    if order != 2:
        raise ValueError("order must be 1 or 2")
    nv = pos.shape[0]
    a = np.stack([tv[:, e0] for e0, _ in TET_EDGES], axis=1)
    b = np.stack([tv[:, e1] for _, e1 in TET_EDGES], axis=1)
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = lo * nv + hi
    ukey, einv = np.unique(key.ravel(), return_inverse=True)
    edge_prim = nv + einv.reshape(key.shape)
    prims = np.concatenate([tv, edge_prim], axis=1)
    conn, porder = _first_touch(prims)
    # FE node positions: vertices or edge midpoints
    node_pos = np.empty((porder.size, 3))
    isv = porder < nv
    node_pos[isv] = pos[porder[isv]]
    ek = ukey[porder[~isv] - nv]
    node_pos[~isv] = 0.5 * (pos[ek // nv] + pos[ek % nv])
    gconn, vorder = _first_touch(tv)
    X = pos[vorder]
    return Mesh(P2_TET, conn, gconn, X, porder.size, node_pos, h, g,
                {"jitter": jitter, "seed": seed})


def structured_hex_mesh(g: int, jitter: float = 0.0, seed: int = 0) -> Mesh:
    """Unit cube, g^3 Q1 hexahedra, cells in lexicographic order."""
    pos, h = _grid_vertices(g, jitter, seed)
    c = np.arange(g)
    ck, cj, ci = np.meshgrid(c, c, c, indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    hv = np.stack([_vid(ci + p[0], cj + p[1], ck + p[2], g) for p in HEX_CORNERS], axis=1)
    conn, vorder = _first_touch(hv)
    X = pos[vorder]
    return Mesh(Q1_HEX, conn, conn, X, X.shape[0], X, h, g, {"jitter": jitter, "seed": seed})


# ---------------------------------------------------------------------------
# Material parameters and fields used by the workloads
# ---------------------------------------------------------------------------

def lame_from_E_nu(E: float, nu: float):
    """3D conversion of MatParams.cpp:11-22 (convert_to_lambda / convert_to_mu)."""
    lam = (E * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    return lam, mu


def homogeneous_lame(n_elements: int, E: float = 1e5, nu: float = 0.35):
    lam, mu = lame_from_E_nu(E, nu)
    return np.full(n_elements, lam), np.full(n_elements, mu)


def lognormal_lame(n_elements: int, seed: int, mu_median: float = 3.7e4,
                   sigma: float = 0.3, nu: float = 0.35):
    """Per-element mu ~ exp(N(ln mu_median, sigma)), lambda = 2 nu mu / (1 - 2 nu)."""
    rng = np.random.default_rng(seed)
    mu = np.exp(rng.normal(np.log(mu_median), sigma, size=n_elements))
    lam = mu * (2.0 * nu) / (1.0 - 2.0 * nu)
    return lam, mu


def random_displacement(mesh: Mesh, scale: float, seed: int) -> np.ndarray:
    """u = scale * h * N(0,1) per dof, node-major (u[node*3+d])."""
    rng = np.random.default_rng(seed)
    return scale * mesh.h * rng.standard_normal(mesh.n_dofs)


def smooth_displacement(mesh: Mesh, amp: float, noise: float, seed: int) -> np.ndarray:
    """u = amp*sin(2 pi x)[1,1,1] + noise*h*N(0,1), x = rest position of the node."""
    rng = np.random.default_rng(seed)
    s = amp * np.sin(2.0 * np.pi * mesh.node_pos[:, 0])
    u = np.repeat(s[:, None], 3, axis=1).reshape(-1)
    return u + noise * mesh.h * rng.standard_normal(mesh.n_dofs)


# ---------------------------------------------------------------------------
# The five benchmark workloads (seeded; the same inputs for the tests, the
# benchmark and the CPU baseline)
# ---------------------------------------------------------------------------
WORKLOADS = {
    1: "P1 tets 20^3 x 6 (48,000), homogeneous E=1e5 nu=0.35, u = 0.02 h N(0,1)",
    2: "P2 tets 40^3 x 6 (384,000), lognormal Lame, u = 0.02 h N(0,1)",
    3: "Q1 hexes 96^3 (884,736), jittered 0.1 h, lognormal Lame, u = 0.05 sin(2 pi x)[1,1,1] + 0.005 h N(0,1)",
    4: "P1 tets 48^3 x 6 (663,552), lognormal Lame, u = 0.02 h N(0,1), adjoint p = N(0,1)",
    5: "P2 tets 32^3 x 6 (196,608), jittered 0.1 h, homogeneous E=1e5 nu=0.35, u = 0.02 h N(0,1), adjoint p = N(0,1)",
}
SEED_JITTER, SEED_LAME, SEED_U, SEED_P = 3, 5, 2, 7


def workload(k: int, grid: int | None = None):
    """(mesh, lam, mu, u, p) of benchmark workload k (1..5); `grid` overrides the
    cells per axis (same generators, for smaller cases of the same kind)."""
    if k == 1:
        mesh = structured_tet_mesh(grid or 20, 1)
        lam, mu = homogeneous_lame(mesh.n_elements)
    elif k == 2:
        mesh = structured_tet_mesh(grid or 40, 2)
        lam, mu = lognormal_lame(mesh.n_elements, SEED_LAME)
    elif k == 3:
        mesh = structured_hex_mesh(grid or 96, jitter=0.1, seed=SEED_JITTER)
        lam, mu = lognormal_lame(mesh.n_elements, SEED_LAME)
    elif k == 4:
        mesh = structured_tet_mesh(grid or 48, 1)
        lam, mu = lognormal_lame(mesh.n_elements, SEED_LAME)
    elif k == 5:
        mesh = structured_tet_mesh(grid or 32, 2, jitter=0.1, seed=SEED_JITTER)
        lam, mu = homogeneous_lame(mesh.n_elements)
    else:
        raise ValueError("workload must be 1..5")
    if k == 3:
        u = smooth_displacement(mesh, 0.05, 0.005, SEED_U)
    else:
        u = random_displacement(mesh, 0.02, SEED_U)
    p = np.random.default_rng(SEED_P).standard_normal(mesh.n_dofs)
    return mesh, lam, mu, u, p
