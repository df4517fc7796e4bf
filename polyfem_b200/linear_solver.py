"""Linear solve on the device for the assembled Hessian (pfg_cg_solve).

PolyFEM's Newton solver hands every assembled Hessian to a polysolve
linear::Solver -- ``analyze_pattern(A, precond_num)``, ``factorize(A)``,
``solve(b, x)``, ``get_info(info)``: the Hessian NLProblem::hessian returns
(solver/NLProblem.cpp:615-621) is solved inside the Newton step of polysolve@47dc48d
(cmake/recipes/polysolve.cmake:11; external, not in the reference tree), which owns
that call sequence.  ``ConjugateGradient`` mirrors that
interface for the solver polysolve names "Eigen::ConjugateGradient" (Eigen's
conjugate gradient with the diagonal preconditioner), run by libpfgpu on the
matrix the assembler left on the device, so the Hessian never leaves the GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import PFG_MEM_DEVICE, PFG_MEM_HOST, check, lib
from .assembler import NeoHookeanAssembler, _is_device

PFG_SYS_FULL = 0
PFG_SYS_REDUCED = 1


class ConjugateGradient:
    """Jacobi-preconditioned CG on the assembler's full or Dirichlet-reduced Hessian.

    Parameters (``set_parameters``): ``max_iter`` (default 1000) and
    ``tolerance`` (default 1e-10), the relative residual |b - H x| / |b| at which
    the iteration stops.  ``get_info()`` returns ``solver_iter`` and
    ``solver_error`` of the last solve.
    """

    def __init__(self, assembler: NeoHookeanAssembler, system: str = "reduced"):
        if system not in ("full", "reduced"):
            raise ValueError("system must be 'full' or 'reduced'")
        self.asm = assembler
        self.system = PFG_SYS_REDUCED if system == "reduced" else PFG_SYS_FULL
        self.max_iter = 1000
        self.tolerance = 1e-10
        self._values = None
        self._info = {"solver_iter": 0, "solver_error": 0.0}

    @staticmethod
    def name() -> str:
        return "Eigen::ConjugateGradient"

    def size(self) -> int:
        return getattr(self.asm, "n_free", 0) if self.system == PFG_SYS_REDUCED else self.asm.n_dofs

    def set_parameters(self, params: dict):
        if "max_iter" in params:
            self.max_iter = int(params["max_iter"])
        if "tolerance" in params:
            self.tolerance = float(params["tolerance"])

    def get_info(self) -> dict:
        return dict(self._info)

    def analyze_pattern(self, A=None, precond_num: int = 0):
        """The pattern is the assembler's (built with the first assembly): nothing to do."""

    def factorize(self, values=None):
        """Binds the matrix values: a float64 CUDA tensor of the system's nnz, or
        None for the values the last host-mode (or values-less) assembly left in
        the assembler's context.  The diagonal preconditioner is formed in solve."""
        if values is not None and not _is_device(values):
            raise ValueError("values must be a float64 CUDA tensor (device memory)")
        self._values = values

    def solve(self, b, x=None, guess: bool = False):
        """x with H x = b; ``x`` (same memory space as b) receives the solution and is
        the starting guess when ``guess`` is true.  Returns x."""
        n = self.size()
        if int(b.numel() if hasattr(b, "numel") else np.size(b)) != n:
            raise ValueError(f"b must have {n} entries")
        if guess and x is None:
            raise ValueError("guess needs x")
        h = self.asm.handle
        if _is_device(b):
            import torch
            if x is None:
                x = torch.empty(n, dtype=torch.float64, device=b.device)
            mem = PFG_MEM_DEVICE
            check(lib().pfg_set_stream(h, ctypes.c_void_p(torch.cuda.current_stream(b.device).cuda_stream)), h,
                  "pfg_set_stream")
            bp, xp = ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x.data_ptr())
        else:
            b = np.ascontiguousarray(b, dtype=np.float64)
            if x is None:
                x = np.zeros(n, dtype=np.float64)
            elif not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous):
                raise ValueError("x must be a contiguous float64 numpy array")
            mem = PFG_MEM_HOST
            check(lib().pfg_set_stream(h, None), h, "pfg_set_stream")
            bp, xp = ctypes.c_void_p(b.ctypes.data), ctypes.c_void_p(x.ctypes.data)
        vp = None if self._values is None else ctypes.c_void_p(self._values.data_ptr())
        it = ctypes.c_int()
        err = ctypes.c_double()
        check(lib().pfg_cg_solve(h, self.system, vp, bp, mem, self.tolerance, self.max_iter, int(bool(guess)), xp,
                                 ctypes.byref(it), ctypes.byref(err)), h, "pfg_cg_solve")
        self._info = {"solver_iter": int(it.value), "solver_error": float(err.value)}
        return x


class DirectSolver:
    """Sparse Cholesky on the device (pfg_direct_*): the factorisation polysolve's
    direct choices (Eigen::SimplicialLDLT, Cholmod, Pardiso) compute for the SPD
    Newton system, here multifrontal with a nested dissection ordering.

    ``analyze_pattern`` orders the pattern of the assembler's full or
    Dirichlet-reduced Hessian, ``factorize`` factorises its values (the last
    assembly's, or a float64 CUDA tensor in the same pattern), ``solve`` returns
    x = A^-1 b for numpy arrays or CUDA tensors.  A matrix that is not positive
    definite raises PfgError with status PFG_ERR_NUMERIC from ``factorize``.
    ``get_info()`` reports the analysis: fronts, tree levels, entries of L, the
    largest front and the factorisation's flops.
    """

    STATS = ("n", "fronts", "levels", "front_doubles", "nnz_L", "max_front", "flops")

    def __init__(self, assembler: NeoHookeanAssembler, system: str = "reduced"):
        if system not in ("full", "reduced"):
            raise ValueError("system must be 'full' or 'reduced'")
        self.asm = assembler
        self.system = PFG_SYS_REDUCED if system == "reduced" else PFG_SYS_FULL
        self._info = {}

    @staticmethod
    def name() -> str:
        return "Cholesky (multifrontal LLT, nested dissection)"

    def size(self) -> int:
        return getattr(self.asm, "n_free", 0) if self.system == PFG_SYS_REDUCED else self.asm.n_dofs

    def set_parameters(self, params: dict):
        """A direct solve has no parameters."""

    def get_info(self) -> dict:
        return dict(self._info)

    def analyze_pattern(self, A=None, precond_num: int = 0):
        """Orders and analyses the system's pattern (the assembler's; `A` is not read)."""
        h = self.asm.handle
        check(lib().pfg_direct_analyze(h, self.system), h, "pfg_direct_analyze")
        st = (ctypes.c_longlong * 7)()
        check(lib().pfg_direct_stats(h, st), h, "pfg_direct_stats")
        self._info = dict(zip(self.STATS, (int(v) for v in st)))

    def factorize(self, values=None):
        """Factorises `values` (a float64 CUDA tensor of the system's nnz) or, with
        None, the values the last assembly left in the assembler's context."""
        if values is not None and not _is_device(values):
            raise ValueError("values must be a float64 CUDA tensor (device memory)")
        h = self.asm.handle
        vp = None if values is None else ctypes.c_void_p(values.data_ptr())
        if values is not None:
            import torch
            check(lib().pfg_set_stream(h, ctypes.c_void_p(torch.cuda.current_stream(values.device).cuda_stream)), h,
                  "pfg_set_stream")
        check(lib().pfg_direct_factorize(h, self.system, vp), h, "pfg_direct_factorize")

    def free(self):
        """Releases the analysis and the factor's device memory (the dense fronts)."""
        h = self.asm.handle
        check(lib().pfg_direct_free(h), h, "pfg_direct_free")
        self._info = {}

    def solve(self, b, x=None):
        """x with A x = b (``x``, in b's memory space, receives it).  Returns x."""
        n = self.size()
        if int(b.numel() if hasattr(b, "numel") else np.size(b)) != n:
            raise ValueError(f"b must have {n} entries")
        h = self.asm.handle
        if _is_device(b):
            import torch
            if x is None:
                x = torch.empty(n, dtype=torch.float64, device=b.device)
            check(lib().pfg_set_stream(h, ctypes.c_void_p(torch.cuda.current_stream(b.device).cuda_stream)), h,
                  "pfg_set_stream")
            check(lib().pfg_direct_solve(h, self.system, ctypes.c_void_p(b.data_ptr()), PFG_MEM_DEVICE,
                                         ctypes.c_void_p(x.data_ptr())), h, "pfg_direct_solve")
            return x
        b = np.ascontiguousarray(b, dtype=np.float64)
        if x is None:
            x = np.zeros(n, dtype=np.float64)
        elif not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous):
            raise ValueError("x must be a contiguous float64 numpy array")
        check(lib().pfg_set_stream(h, None), h, "pfg_set_stream")
        check(lib().pfg_direct_solve(h, self.system, ctypes.c_void_p(b.ctypes.data), PFG_MEM_HOST,
                                     ctypes.c_void_p(x.ctypes.data)), h, "pfg_direct_solve")
        return x


def direct_symbolic(outer, inner) -> dict:
    """Host-only analysis of a symmetric CSC pattern (full storage, sorted rows):
    the fronts, tree levels, entries of L, largest front and flops the device
    factorisation of that pattern would have.  Needs no GPU."""
    outer = np.ascontiguousarray(outer, dtype=np.int32)
    inner = np.ascontiguousarray(inner, dtype=np.int32)
    n = outer.size - 1
    st = (ctypes.c_longlong * 7)()
    check(lib().pfg_direct_symbolic(n, ctypes.c_void_p(outer.ctypes.data), ctypes.c_void_p(inner.ctypes.data), st),
          None, "pfg_direct_symbolic")
    return dict(zip(DirectSolver.STATS, (int(v) for v in st)))
