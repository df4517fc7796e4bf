"""Host analysis of the sparse direct solve (pfg_direct_symbolic, no GPU): nested
dissection ordering and front structure of Hessian patterns and of edge-case
patterns.  The analysis checks every index map it builds against the front it
addresses and fails with PFG_ERR_STATE otherwise, so these runs also exercise
those checks."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import binding as B
from polyfem_b200 import PfgError, direct_symbolic
from polyfem_b200 import mesh as M
from polyfem_b200._lib import PFG_ERR_INVALID


def _check(st, n, nnz):
    assert st["n"] == n
    if n == 0:
        assert st["fronts"] == 0 and st["nnz_L"] == 0
        return
    assert 1 <= st["fronts"] <= n and st["levels"] >= 1
    assert (nnz + n) // 2 <= st["nnz_L"] <= n * (n + 1) // 2
    assert st["max_front"] <= n and st["front_doubles"] >= st["nnz_L"]


@pytest.mark.parametrize("name", ["P1", "P2", "Q1"])
def test_hessian_patterns(name):
    mesh = {"P1": lambda: M.structured_tet_mesh(5, 1), "P2": lambda: M.structured_tet_mesh(3, 2),
            "Q1": lambda: M.structured_hex_mesh(6, jitter=0.1, seed=3)}[name]()
    lam, mu = M.lognormal_lame(mesh.n_elements, 7)
    orc = B.Oracle(mesh, lam, mu)
    u = M.random_displacement(mesh, 0.02, 11)
    outer, inner, vals = orc.hessian(u)
    n = outer.size - 1
    st = direct_symbolic(outer, inner)
    _check(st, n, inner.size)
    # the Dirichlet-reduced pattern (x = 0 face fixed)
    face = np.flatnonzero(mesh.node_pos[:, 0] <= 1e-12)
    cons = (3 * face[:, None] + np.arange(3)).ravel()
    ro, ri, rv = B.project_hessian(outer, inner, vals, cons)
    _check(direct_symbolic(ro, ri), ro.size - 1, ri.size)


def test_edge_patterns():
    # empty, one dof, a diagonal matrix (no edges: every column its own front)
    _check(direct_symbolic(np.zeros(1, np.int32), np.zeros(0, np.int32)), 0, 0)
    _check(direct_symbolic(np.array([0, 1], np.int32), np.array([0], np.int32)), 1, 1)
    d = direct_symbolic(np.arange(501, dtype=np.int32), np.arange(500, dtype=np.int32))
    _check(d, 500, 500)
    assert d["nnz_L"] == 500 and d["levels"] == 1
    # two disconnected random blocks and a dense block
    rng = np.random.default_rng(2)
    blocks = []
    for m_, dens in ((300, 0.02), (200, 0.05), (40, 1.0)):
        R = sp.random(m_, m_, density=dens, random_state=rng.integers(1 << 30))
        blocks.append((R + R.T + sp.identity(m_)).tocsc())
    A = sp.block_diag(blocks, format="csc")
    A.sort_indices()
    _check(direct_symbolic(A.indptr, A.indices), A.shape[0], A.nnz)
    # a long path (deep dissection): single-vertex separators; the leaf parts (at
    # most 96 dofs) are dense fronts, so L holds up to ~48 entries per column
    n = 5000
    P = sp.diags([np.ones(n - 1), np.ones(n), np.ones(n - 1)], [-1, 0, 1], format="csc")
    P.sort_indices()
    st = direct_symbolic(P.indptr, P.indices)
    _check(st, n, P.nnz)
    assert st["nnz_L"] <= 50 * n and st["levels"] >= 6


def test_invalid_patterns():
    with pytest.raises(PfgError) as ei:
        direct_symbolic(np.array([0, 2, 3], np.int32), np.array([1, 0, 1], np.int32))  # unsorted rows
    assert ei.value.status == PFG_ERR_INVALID
    with pytest.raises(PfgError):
        direct_symbolic(np.array([0, 1, 2], np.int32), np.array([0, 5], np.int32))  # row out of range
    with pytest.raises(PfgError):
        direct_symbolic(np.array([1, 1, 2], np.int32), np.array([0, 1], np.int32))  # outer[0] != 0
