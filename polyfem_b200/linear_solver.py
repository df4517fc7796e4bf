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
