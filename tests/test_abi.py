"""C-ABI boundary checks that need no GPU: the library loads, exports exactly what
include/pfgpu.h declares, and rejects bad input before touching a device."""
import ctypes
import os
import re

import numpy as np
import pytest

from polyfem_b200 import _lib
from polyfem_b200 import mesh as M

from conftest import gpu_available

HEADER = os.path.join(_lib.REPO, "include", "pfgpu.h")


def _declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pfg_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    declared = _declared_symbols()
    assert len(declared) >= 19
    for name in declared:
        assert hasattr(L, name), f"{name} declared in pfgpu.h but not exported"
    assert set(declared) == set(_lib.SIGNATURES), "ctypes signature table out of sync with pfgpu.h"


def test_version_and_status_strings():
    L = _lib.lib()
    assert L.pfg_version() >= 100
    assert L.pfg_status_string(0) == b"ok"
    assert L.pfg_status_string(1) == b"invalid argument"
    assert L.pfg_status_string(99) == b"unknown status"


def _create(desc):
    h = ctypes.c_void_p()
    st = _lib.lib().pfg_create(ctypes.byref(desc), ctypes.byref(h))
    return st, h


def _desc(mesh, lam, mu, conn=None, gconn=None, et=None):
    conn = np.ascontiguousarray(mesh.conn if conn is None else conn, dtype=np.int32)
    g = None if gconn is None else np.ascontiguousarray(gconn, dtype=np.int32)
    X = np.ascontiguousarray(mesh.X)
    keep = (conn, g, X, lam, mu)
    d = _lib.MeshDesc(mesh.elem_type if et is None else et, mesh.n_elements, mesh.n_nodes, mesh.n_geom_nodes,
                      conn.ctypes.data, None if g is None else g.ctypes.data, X.ctypes.data,
                      lam.ctypes.data, mu.ctypes.data, 0)
    return d, keep


def test_create_rejects_out_of_range_connectivity():
    mesh = M.structured_tet_mesh(1, 1)
    lam, mu = M.homogeneous_lame(mesh.n_elements)
    bad = mesh.conn.copy()
    bad[3, 2] = mesh.n_nodes  # one past the end
    d, keep = _desc(mesh, lam, mu, conn=bad)
    st, h = _create(d)
    assert st == 1 and not h.value
    assert b"conn[14]" in _lib.lib().pfg_last_error(None)
    bad[3, 2] = -1
    d, keep = _desc(mesh, lam, mu, conn=bad)
    assert _create(d)[0] == 1


def test_create_rejects_bad_type_and_missing_geometry():
    mesh = M.structured_tet_mesh(1, 2)
    lam, mu = M.homogeneous_lame(mesh.n_elements)
    d, keep = _desc(mesh, lam, mu, et=7)
    assert _create(d)[0] == 1
    d, keep = _desc(mesh, lam, mu)  # P2 without gconn
    assert _create(d)[0] == 1
    assert b"gconn" in _lib.lib().pfg_last_error(None)
    st, h = _lib.lib().pfg_create(None, ctypes.byref(ctypes.c_void_p())), None
    assert st == 1


def test_null_context_calls_are_rejected():
    L = _lib.lib()
    assert L.pfg_destroy(None) == 1
    assert L.pfg_synchronize(None) == 1
    assert L.pfg_energy(None, None, 0, 0, None) == 1
    assert L.pfg_hessian(None, None, 0, 0, 0, None) == 1


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_create_without_device_reports_cuda_error():
    mesh = M.structured_tet_mesh(1, 1)
    lam, mu = M.homogeneous_lame(mesh.n_elements)
    d, keep = _desc(mesh, lam, mu)
    st, h = _create(d)
    assert st == 2 and not h.value
    assert b"CUDA" in _lib.lib().pfg_last_error(None) or b"device" in _lib.lib().pfg_last_error(None)


def test_python_wrapper_raises_on_failure():
    mesh = M.structured_tet_mesh(1, 1)
    lam, mu = M.homogeneous_lame(mesh.n_elements)
    bad = mesh.conn.copy()
    bad[0, 0] = 10**6
    from polyfem_b200 import NeoHookeanAssembler, PfgError
    with pytest.raises(PfgError):
        NeoHookeanAssembler(M.P1_TET, bad, mesh.X, lam, mu, n_nodes=mesh.n_nodes)


def test_noalloc_refuses_misaligned_caller_pointers_before_any_launch():
    """pfg_energy_noalloc takes caller-owned device pointers; (lambda, mu) is read as
    one 16-byte pair, so a pointer 8 bytes off (a slice of a larger pool) is refused
    on the host with PFG_ERR_INVALID.  The pointers are never dereferenced: the
    check runs before any CUDA call, so this needs no GPU."""
    L = _lib.lib()
    base = 1 << 20  # a 256-byte aligned fake device address, never touched
    p = lambda off: ctypes.c_void_p(base + off)
    st = L.pfg_energy_noalloc(M.P1_TET, 6, 8, 8, p(0), None, p(0), p(8), p(0), 0, p(0), None)
    assert st == 1
    assert b"16-byte aligned" in L.pfg_last_error(None)
    st = L.pfg_energy_noalloc(M.P1_TET, 6, 8, 8, p(0), None, p(4), p(0), p(0), 0, p(0), None)
    assert st == 1 and b"8-byte aligned" in L.pfg_last_error(None)
    st = L.pfg_energy_noalloc(M.P1_TET, 6, 8, 8, p(2), None, p(0), p(0), p(0), 0, p(0), None)
    assert st == 1 and b"4-byte aligned" in L.pfg_last_error(None)
    # the size limits pfg_create applies
    st = L.pfg_energy_noalloc(M.P1_TET, 6, 1 << 30, 8, p(0), None, p(0), p(0), p(0), 0, p(0), None)
    assert st == 4 and b"too many nodes" in L.pfg_last_error(None)
