"""pfg_energy_noalloc: the energy entry point for callers that must not allocate.

Callers that pre-plan every byte of device memory, or that run inside a memory
pool they do not own, cannot use pfg_create (it allocates).  They hand every
array to pfg_energy_noalloc, whose reduction scratch is a fixed array inside the
library.  This test calls it through the C ABI on device buffers the test owns
and checks it against pfg_energy on the same inputs, on two calls in a row (the
shared scratch keeps the previous call's contents, which must not leak into the
next result).  It runs last so a failure here cannot hide other failures.
"""
import ctypes

import numpy as np
import pytest

from polyfem_b200 import NeoHookeanAssembler
from polyfem_b200 import _lib
from polyfem_b200 import mesh as M

from _cases import make_case

pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


# FP64 agrees with pfg_energy to 1e-12; the FP32 and split modes (FP32 kinematics,
# FP64 det / log J and reduction) are held to the 1e-6 energy bound of those modes.
PRECS = [(_lib.PFG_FP64, "fp64", 1e-12), (_lib.PFG_FP32, "fp32", 1e-6), (_lib.PFG_SPLIT32, "split32", 1e-6)]


@pytest.mark.parametrize("prec,prec_name,tol", PRECS, ids=[p[1] for p in PRECS])
@pytest.mark.parametrize("et,g", [(M.P1_TET, 6), (M.P2_TET, 4), (M.Q1_HEX, 5)])
def test_noalloc_energy_matches_pfg_energy(require_gpu, et, g, prec, prec_name, tol):
    import torch
    L = _lib.lib()
    mesh, lam, mu, u, _ = make_case(et, g, seed=41, jitter=0.1 if et != M.P1_TET else 0.0)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    dev = "cuda"
    conn = torch.tensor(np.ascontiguousarray(mesh.conn.T), dtype=torch.int32, device=dev)
    gconn = torch.tensor(np.ascontiguousarray(mesh.gconn.T), dtype=torch.int32, device=dev)
    X = torch.tensor(mesh.X, dtype=torch.float64, device=dev)
    lame = torch.tensor(np.stack([lam, mu], axis=1), dtype=torch.float64, device=dev)
    for call in range(2):
        ud = torch.tensor(u * (1.0 + 0.5 * call), dtype=torch.float64, device=dev)
        out = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
        st = L.pfg_energy_noalloc(et, mesh.n_elements, mesh.n_nodes, mesh.n_geom_nodes, _vp(conn), _vp(gconn), _vp(X),
                                  _vp(lame), _vp(ud), prec, _vp(out), None)
        assert st == 0, L.pfg_last_error(None)
        torch.cuda.synchronize()
        ref = asm.assemble_energy(u * (1.0 + 0.5 * call), prec_name)
        got = float(out.cpu())
        assert abs(got - ref) <= tol * abs(ref), (call, got, ref)
    asm.close()


def test_noalloc_rejects_oversized_mesh(require_gpu):
    L = _lib.lib()
    too_many = 256 * 65536 + 1
    st = L.pfg_energy_noalloc(M.P1_TET, too_many, 10, 10, ctypes.c_void_p(16), None, ctypes.c_void_p(16),
                              ctypes.c_void_p(16), ctypes.c_void_p(16), 0, ctypes.c_void_p(16), None)
    assert st == 4
    assert b"exceeds the limit" in L.pfg_last_error(None)


@pytest.mark.parametrize("et,per_block", [(M.P2_TET, 256), (M.Q1_HEX, 256)])
def test_noalloc_limit_follows_the_energy_kernel_blocks(require_gpu, et, per_block):
    L = _lib.lib()
    too_many = per_block * 65536 + 1
    st = L.pfg_energy_noalloc(et, too_many, 10, 10, ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16),
                              ctypes.c_void_p(16), ctypes.c_void_p(16), 0, ctypes.c_void_p(16), None)
    assert st == 4
    assert b"exceeds the limit" in L.pfg_last_error(None)
