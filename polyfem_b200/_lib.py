"""Loader and build recipe of the in-tree CUDA library ``libpfgpu.so``.

The library exposes exactly the C ABI of ``include/pfgpu.h``.  There is no
fallback: if the library is missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_PATH = os.path.join(HERE, "libpfgpu.so")
SOURCES = ["pfg_api.cu", "pfg_kernels.cu", "pfg_materials.cu", "pfg_solve.cu", "pfg_noalloc.cu", "pfg_tc.cu", "pfg_direct.cu"]
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]

PFG_OK = 0
PFG_ERR_INVALID = 1
PFG_ERR_OOM = 3
PFG_ERR_STATE = 5
PFG_ERR_NUMERIC = 6
PFG_MEM_HOST = 0
PFG_MEM_DEVICE = 1
PFG_FP64 = 0
PFG_FP32 = 1
PFG_SPLIT32 = 2
PFG_SPLIT32_SIMT = 3

_lib = None


def _sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def needs_build() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = _sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(REPO, "include", "pfgpu.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile libpfgpu.so for sm_100a with nvcc (works without a GPU)."""
    if not force and not needs_build():
        return LIB_PATH
    nvcc = os.environ.get("NVCC", "nvcc")
    build_dir = os.path.join(HERE, "_build")
    os.makedirs(build_dir, exist_ok=True)
    cmds, objs = [], []
    for src in _sources():
        obj = os.path.join(build_dir, os.path.basename(src) + ".o")
        cmd = [nvcc, *ARCH_FLAGS, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
               "-I", os.path.join(REPO, "include"), "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        cmds.append(cmd)
        objs.append(obj)
    # the translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(subprocess.check_call, c) for c in cmds]:
            f.result()
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc, *ARCH_FLAGS, "-shared", "-o", tmp, *objs, "-lpthread"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


class MeshDesc(ctypes.Structure):
    _fields_ = [
        ("elem_type", ctypes.c_int),
        ("n_elements", ctypes.c_int),
        ("n_nodes", ctypes.c_int),
        ("n_geom_nodes", ctypes.c_int),
        ("conn", _vp),
        ("gconn", _vp),
        ("X", _vp),
        ("lam", _vp),
        ("mu", _vp),
        ("device", ctypes.c_int),
    ]


# name -> (restype, argtypes); every symbol include/pfgpu.h declares
SIGNATURES = {
    "pfg_create": (ctypes.c_int, [ctypes.POINTER(MeshDesc), ctypes.POINTER(_vp)]),
    "pfg_destroy": (ctypes.c_int, [_vp]),
    "pfg_set_stream": (ctypes.c_int, [_vp, _vp]),
    "pfg_set_lame": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "pfg_set_rest_positions": (ctypes.c_int, [_vp, _vp, ctypes.c_int]),
    "pfg_energy": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "pfg_energy_per_element": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "pfg_gradient": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "pfg_hessian_pattern": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "pfg_hessian_pattern_copy": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "pfg_hessian": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    "pfg_hessian_apply": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    "pfg_hessian_device_csc": (ctypes.c_int, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "pfg_material_vjp": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    "pfg_shape_vjp": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "pfg_inverted_count": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "pfg_synchronize": (ctypes.c_int, [_vp]),
    "pfg_last_error": (ctypes.c_char_p, [_vp]),
    "pfg_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "pfg_version": (ctypes.c_int, []),
    "pfg_energy_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp,
                                          _vp, ctypes.c_int, _vp, _vp]),
    "pfg_set_dirichlet": (ctypes.c_int, [_vp, _vp, ctypes.c_int]),
    "pfg_reduced_pattern": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)]),
    "pfg_reduced_pattern_copy": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "pfg_hessian_reduced": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    "pfg_gradient_reduced": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "pfg_reduced_to_full": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    "pfg_set_material": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pfg_set_material_params": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int]),
    "pfg_set_elasticity_tensor": (ctypes.c_int, [_vp, _vp]),
    "pfg_mass_matrix": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp]),
    "pfg_lump_matrix": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp]),
    "pfg_dense_matrix": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp]),
    "pfg_set_component": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _vp, ctypes.c_int]),
    "pfg_set_composite": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "pfg_cg_solve": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_int, _vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]),
    "pfg_direct_analyze": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pfg_direct_factorize": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "pfg_direct_solve": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int, _vp]),
    "pfg_direct_stats": (ctypes.c_int, [_vp, _vp]),
    "pfg_direct_free": (ctypes.c_int, [_vp]),
    "pfg_direct_symbolic": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp]),
}


class PfgError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str):
        super().__init__(f"{where}: {detail} (status {status})")
        self.status = status


def lib():
    """Load libpfgpu.so (building it first only when it does not exist)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libpfgpu.so not found at {LIB_PATH}; run polyfem_b200._lib.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, ctx, where: str):
    if status != PFG_OK:
        detail = lib().pfg_last_error(ctx)
        raise PfgError(status, where, (detail or b"").decode() or lib().pfg_status_string(status).decode())
