#!/usr/bin/env python
"""Benchmark: NeoHookean element Hessians/s on B200 (split-FP32 vs FP64, rel err vs FP64).

Workload (the configuration the metric is quoted on): P2 tetrahedra on a 40^3 cube
split 6 tets/hex (384,000 elements, 531,441 nodes, 1,594,323 dofs, 134,475,849
CSC nonzeros), 4-point quadrature, per-element lognormal Lame parameters, seeded
synthetic displacement u = 0.02 h N(0,1).  One step = one assembly of the global
Hessian CSC values through the path's C ABI (pfg_hessian), which launches two
kernels: the element blocks (split32: k_hessian_blocks_tc on the tensor cores; FP64:
k_hessian_blocks on CUDA cores) -> one packed block triangle per element, and the
reduction kernel (blocks -> CSC columns, summed per entry in a fixed order).

  value     : split-precision Hessian assembly, inputs resident in HBM (elements/s)
  e2e       : the same call with host buffers (pinned u in, CSC values out) (elements/s)
  fp64      : the plain FP64 drop-in kernel, same workload (elements/s)
  split32_simt : the same split with the element contraction on CUDA cores
  configs   : the other four workloads' operations (energy, gradient, Hessian, adjoint terms)
  cpu_baseline / --impl reference : the CPU oracle port of the reference's TBB
              assembly (NLAssembler::assemble_hessian) on the host cores.

Run:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
      python bench.py --grid G          (same line on a G^3 P2 cube: small profiling case)
      python bench.py --suite           (per-operation timings on all five workloads)
"""
from __future__ import annotations

import argparse
import faulthandler
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "NeoHookean elem Hessians/s on 1 B200: split-FP32 vs FP64, rel err vs FP64"
UNIT = "elements/s"
SEED_LAME, SEED_U = 5, 2
PRECISION_NOTE = ("split32 = FP64 kinematics (J^-T, M = dx/dxi, det/log J, M^-T) + element contraction on the "
                  "tensor cores (tcgen05 kind::tf32, each FP32 operand split into two TF32 halves, 3 products, FP32 "
                  "accumulation in TMEM) + FP32 staged element blocks + FP64 per-entry sums and CSC values")


def workload_name(grid: int) -> str:
    E = 6 * grid ** 3
    return (f"P2 tet NeoHookean Hessian assembly, {grid}^3 cube x 6 tets ({E:,} elements, "
            f"{3 * (2 * grid + 1) ** 3:,} dofs), 4-pt quadrature, lognormal Lame")


def _rank_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def _workload(grid: int):
    from polyfem_b200 import mesh as M
    mesh = M.structured_tet_mesh(grid, 2)
    lam, mu = M.lognormal_lame(mesh.n_elements, SEED_LAME)
    u = M.random_displacement(mesh, 0.02, SEED_U)
    return mesh, lam, mu, u


def algorithmic_bytes(mesh, nnz: int) -> int:
    """Bytes a Hessian assembly must move at least once: conn + gconn + Lame + X + u
    + node-block slot map (one int32 per element node pair) + column offsets read,
    CSC values written."""
    E, n, ng = mesh.n_elements, mesh.conn.shape[1], mesh.gconn.shape[1]
    return (E * n * 4 + E * ng * 4 + E * 16 + mesh.n_geom_nodes * 24 + mesh.n_nodes * 24
            + E * n * n * 4 + mesh.n_nodes * 4 + nnz * 8)


def staged_bytes(mesh, nnz: int, tri_bytes: int) -> int:
    """HBM bytes the two-pass design moves when the staged blocks do not stay in L2:
    algorithmic bytes + the block triangles written by pass 1 and read once by
    pass 2 (one padded triangle of 9 n(n+1)/2 values per element; the second read
    of an off-diagonal block comes from L2).  The 32-bit reduction plan is the
    algorithmic slot map's 4 bytes per node pair."""
    E, n = mesh.n_elements, mesh.conn.shape[1]
    return algorithmic_bytes(mesh, nnz) + 2 * E * tri_bytes


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML every few ms while the
    timed region runs (falls back to nvidia-smi at 100 ms when NVML is missing)."""

    # NVML clocks-event-reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, cuda_index: int, period_s: float = 0.001):
        self.cuda_index = cuda_index
        self.period = period_s
        self.samples = []   # (sm_mhz, max_mhz, reasons bitmask)
        self._stop = threading.Event()
        self._thread = None
        self._proc = None
        self._lines = []
        self.source = None

    def _nvml_handle(self):
        """NVML handle of the CUDA device, matched by PCI domain/bus/device numbers
        (CUDA and NVML may enumerate devices differently)."""
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.cuda_index)
        want = tuple(int(getattr(props, k, -1)) for k in ("pci_domain_id", "pci_bus_id", "pci_device_id"))
        for i in range(pynvml.nvmlDeviceGetCount()):
            h = pynvml.nvmlDeviceGetHandleByIndex(i)
            pi = pynvml.nvmlDeviceGetPciInfo(h)
            if (int(pi.domain), int(pi.bus), int(pi.device)) == want:
                return pynvml, h
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def start(self):
        try:
            nv, hdl = self._nvml_handle()
            reasons_fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            smax = nv.nvmlDeviceGetMaxClockInfo(hdl, nv.NVML_CLOCK_SM)

            def loop():
                while not self._stop.is_set():
                    try:
                        self.samples.append((nv.nvmlDeviceGetClockInfo(hdl, nv.NVML_CLOCK_SM), smax,
                                             int(reasons_fn(hdl))))
                    except Exception:
                        pass
                    time.sleep(self.period)

            self.source = "nvml"
            self._thread = threading.Thread(target=loop, daemon=True)
            self._thread.start()
            return
        except Exception:
            pass
        try:
            fields = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
                      "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                      "clocks_event_reasons.sw_power_cap")
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.cuda_index}", f"--query-gpu={fields}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._thread = threading.Thread(target=lambda: [self._lines.append(x.strip()) for x in self._proc.stdout],
                                            daemon=True)
            self._thread.start()
            self.source = "nvidia-smi"
        except Exception:
            self.source = None

    def stop(self):
        if self.source is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"], "samples": 0}
        self._stop.set()
        if self._proc is not None:
            time.sleep(0.2)
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
            bits = [0x8, 0x40, 0x20, 0x4]
            for ln in self._lines:
                p = [x.strip() for x in ln.split(",")]
                if len(p) < 6:
                    continue
                try:
                    mask = sum(b for b, v in zip(bits, p[2:6]) if v.lower() == "active")
                    self.samples.append((float(p[0]), float(p[1]), mask))
                except ValueError:
                    continue
        elif self._thread is not None:
            self._thread.join(timeout=2)
        sm = [s[0] for s in self.samples]
        mask = 0
        for s in self.samples:
            mask |= s[2]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(s[1] for s in self.samples) if self.samples else None,
                "reasons": sorted(name for bit, name in self.REASONS.items() if mask & bit),
                "samples": len(sm), "source": self.source}


# ----------------------------------------------------------------- CPU side
def cpu_threads_for(nnz: int) -> int:
    """All host cores, capped so the reference algorithm's per-thread nnz-sized
    value buffers (Assembler.cpp:669) fit in 40% of the available memory."""
    ncpu = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 32 << 30
    per_thread = nnz * 8 + (64 << 20)
    return int(max(1, min(ncpu, 64, (0.4 * avail) // per_thread)))


def time_cpu_reference(mesh, lam, mu, u, n_threads: int, reps: int):
    """Steady-state Hessian assembly of the CPU oracle (port of the reference's
    NLAssembler::assemble_hessian with SparseMatrixCache) on the host cores."""
    from oracle.binding import Oracle
    orc = Oracle(mesh, lam, mu, n_threads=n_threads, fast_pattern=True)
    t0 = time.perf_counter()
    orc.hessian(u)  # first call: pattern + slot map
    t_first = time.perf_counter() - t0
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        orc.hessian(u)
        times.append(time.perf_counter() - t0)
    return times, t_first


# ----------------------------------------------------------------- reference arm
def run_reference(args):
    rank, world, _ = _rank_info()
    if rank != 0:
        return 0
    mesh, lam, mu, u = _workload(args.grid)
    nnz = _nnz_p2(args.grid)
    nt = cpu_threads_for(nnz)
    times, t_first = time_cpu_reference(mesh, lam, mu, u, nt, args.warmup + args.steps)
    timed = times[args.warmup:]
    t = sum(timed) / len(timed)
    value = mesh.n_elements / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded mesh, lognormal Lame, u = 0.02 h N(0,1))",
        "config": {"workload": workload_name(args.grid), "precision": "fp64",
                   "implementation": "C++ restatement of NLAssembler::assemble_hessian + SparseMatrixCache "
                                     "(oracle/pf_oracle.cpp), std::thread element-parallel"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nt, "kind": "port",
                         "sample": f"full {args.grid}^3 P2 Hessian per step ({mesh.n_elements:,} elements), "
                                   f"steady-state calls; first call (pattern build) {t_first:.2f} s"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _nnz_p2(grid: int) -> int:
    """CSC nonzeros of the P2 Kuhn-split g^3 cube: exact at 40, scaled by volume
    otherwise (only used to size the CPU port's per-thread buffers)."""
    return int(134475849 * max(1.0, (grid / 40.0) ** 3)) if grid >= 40 else int(134475849 * (grid / 40.0) ** 3) + 1


# ----------------------------------------------------------------- GPU arm
def max_over_ranks_of(x: float, device="cpu") -> float:
    """Slowest rank's time: every rank contributes x and receives the maximum
    (identity outside an initialised process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return x
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t)


def _events_ms(stream, fn, steps):
    import torch
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        fn()
    end.record(stream)
    torch.cuda.synchronize()
    return start.elapsed_time(end) / steps


def _events_ms_flushed(stream, fn, steps, flush):
    """Mean device time of fn over `steps` launches, each timed alone with CUDA
    events after an L2 flush on the same stream: a 256 MB write (evicts the
    operation's lines) followed by a 256 MB read (evicts the flush's own dirty
    lines, so their write-back does not land inside the timed launch)."""
    import torch
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    half = flush.numel() // 2
    with torch.cuda.stream(stream):
        for i in range(steps):
            flush[:half].zero_()
            flush[half:].sum()
            starts[i].record(stream)
            fn()
            ends[i].record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in zip(starts, ends)) / steps


def run_gpu(args):
    import torch

    rank, world, local = _rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from polyfem_b200 import NeoHookeanAssembler
    from polyfem_b200._lib import PFG_FP64, PFG_MEM_DEVICE, PFG_MEM_HOST, PFG_SPLIT32, PFG_SPLIT32_SIMT, check, lib

    mesh, lam, mu, u = _workload(args.grid)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu, device=local)
    nnz = asm.hessian_nnz()
    E = mesh.n_elements
    L = lib()
    h = asm.handle
    stream = torch.cuda.Stream(device=local)
    check(L.pfg_set_stream(h, ctypes_ptr(stream.cuda_stream)), h, "pfg_set_stream")
    ud = torch.tensor(u, device=f"cuda:{local}", dtype=torch.float64)
    vals_dev = torch.empty(nnz, device=f"cuda:{local}", dtype=torch.float64)
    uptr = ctypes_ptr(ud.data_ptr())

    def call(prec, mem, up, vptr):
        check(L.pfg_hessian(h, up, mem, prec, 0, vptr), h, "pfg_hessian")

    def max_over_ranks(x):
        return max_over_ranks_of(x, f"cuda:{local}")

    def timed_device(prec, sampler=None):
        for _ in range(args.warmup):
            call(prec, PFG_MEM_DEVICE, uptr, None)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        if sampler is not None:
            sampler.start()
        ms = _events_ms(stream, lambda: call(prec, PFG_MEM_DEVICE, uptr, None), args.steps)
        clocks = sampler.stop() if sampler is not None else None
        if dist is not None:
            dist.barrier()
        return max_over_ranks(ms), clocks

    # accuracy of the headline precision against the FP64 drop-in
    call(PFG_FP64, PFG_MEM_DEVICE, uptr, ctypes_ptr(vals_dev.data_ptr()))
    torch.cuda.synchronize()
    v64 = vals_dev.clone()
    call(PFG_SPLIT32, PFG_MEM_DEVICE, uptr, ctypes_ptr(vals_dev.data_ptr()))
    torch.cuda.synchronize()
    rel_err = float(torch.linalg.vector_norm(vals_dev - v64) / torch.linalg.vector_norm(v64))
    del v64

    ms64, _ = timed_device(PFG_FP64)
    ms_simt, _ = timed_device(PFG_SPLIT32_SIMT)
    ms_split, clocks = timed_device(PFG_SPLIT32, ClockSampler(local))

    # end to end through the C ABI with host buffers: pinned u in, CSC values out
    # (the call copies u to the device, assembles, copies the values back and syncs)
    u_host = torch.tensor(u, dtype=torch.float64).pin_memory()
    v_host = torch.empty(nnz, dtype=torch.float64).pin_memory()
    hptr_u, hptr_v = ctypes_ptr(u_host.data_ptr()), ctypes_ptr(v_host.data_ptr())
    for _ in range(args.warmup):
        call(PFG_SPLIT32, PFG_MEM_HOST, hptr_u, hptr_v)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e2e_ms = _events_ms(stream, lambda: call(PFG_SPLIT32, PFG_MEM_HOST, hptr_u, hptr_v), args.steps)
    e2e_ms = max_over_ranks(e2e_ms)

    # one Newton step that keeps the matrix on the device: pinned u in; the reduced
    # (x = 0 face clamped) gradient and PSD-projected FP64 Hessian, the device CG on it
    # (relative residual 1e-6), the full step; pinned step out.  Times the whole step
    # and each part with CUDA events on the context's stream.
    newton = newton_direct = None
    if rank == 0 and world == 1 and not args.no_newton:
        newton = time_newton_step(asm, h, mesh, u_host, stream, min(args.steps, 5))
        newton_direct = time_newton_step_direct(asm, h, mesh, u_host, stream, 2)

    tri_bytes = 4 * 8 * ((9 * 55 + 7) // 8)  # P2 block triangle in FP32
    bytes_alg = algorithmic_bytes(mesh, nnz)
    peak, peak_src = _peaks()
    achieved = bytes_alg / (ms_split * 1e-3) / 1e9
    traffic = _profiled_traffic(args.grid)

    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        configs = measure_configs(stream, peak)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        nt = cpu_threads_for(nnz)
        times, t_first = time_cpu_reference(mesh, lam, mu, u, nt, 5)
        t = statistics.median(times)
        # one host thread on a bounded sample of the same kind (P2 12^3, seeded alike)
        ms_, ls_, mus_, us_ = _workload(12)
        t1, _ = time_cpu_reference(ms_, ls_, mus_, us_, 1, 5)
        t1 = statistics.median(t1)
        cpu = {"value": E / t, "unit": UNIT, "cores": nt, "kind": "port", "host_cores": os.cpu_count(),
               "sample": f"full {args.grid}^3 P2 Hessian ({E:,} elements), median of 5 steady-state calls "
                         f"of the oracle's std::thread port on {nt} threads (host has {os.cpu_count()} cores); "
                         f"pattern build {t_first:.1f} s",
               "one_thread": {"value": ms_.n_elements / t1, "unit": UNIT, "cores": 1,
                              "sample": f"P2 12^3 ({ms_.n_elements:,} elements), median of 5 steady-state calls"}}

    if rank == 0:
        line = {
            "metric": METRIC, "value": world * E / (ms_split * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_split, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 kinematics + f32 contraction, f64 CSC",
            "data": f"synthetic (seeded {args.grid}^3 P2 mesh, lognormal Lame, u = 0.02 h N(0,1))",
            "config": {"workload": workload_name(args.grid), "global_batch": world * E,
                       "parallelism": f"replicas x{world}", "precision": "split32",
                       "precision_detail": PRECISION_NOTE, "nnz": nnz,
                       "l2": "no flush; every step writes the 1.08 GB CSC values and 0.76 GB of element "
                             "block triangles, both larger than the 126 MB L2"},
            "fp64": {"value": world * E / (ms64 * 1e-3), "unit": UNIT, "ms_per_step": ms64},
            "split32_simt": {"value": world * E / (ms_simt * 1e-3), "unit": UNIT, "ms_per_step": ms_simt,
                             "note": "the same split with the element contraction on CUDA cores"},
            "split_over_fp64": ms64 / ms_split,
            "rel_err_vs_fp64": rel_err,
            "e2e": {"value": world * E / (e2e_ms * 1e-3), "unit": UNIT, "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": u_host.numel() * 8, "d2h_bytes_per_step": nnz * 8},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                         "bytes_alg_per_launch": bytes_alg,
                         "staged_bytes_per_launch": staged_bytes(mesh, nnz, tri_bytes),
                         "note": "one pfg_hessian call = k_hessian_blocks_tc + the reduction kernel, CUDA events "
                                 "on the context's stream; frac of measured HBM copy bandwidth; traffic = ncu "
                                 "DRAM bytes per element of the 24^3 capture x elements"},
            "cpu_baseline": cpu,
            "e2e_newton_step": newton,
            "e2e_newton_step_direct": newton_direct,
            "configs": configs,
            "clocks": clocks,
            "gpu_launches": 2 * args.steps,
        }
        print(json.dumps(line), flush=True)
    asm.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def time_newton_step(asm, h, mesh, u_host, stream, steps):
    """One Newton step of the device-resident path (NLProblem with the projecting
    Dirichlet form: NLProblem::gradient / hessian reduced, the linear solve, the step
    reduced_to_full): H2D of u and D2H of the step inside the timed region."""
    import ctypes

    import torch
    from polyfem_b200._lib import check, lib
    L = lib()
    face = np.flatnonzero(mesh.node_pos[:, 0] <= 1e-12)
    asm.set_dirichlet((3 * face[:, None] + np.arange(3)).ravel())
    L.pfg_set_stream(h, ctypes_ptr(stream.cuda_stream))
    nf, ndof = asm.n_free, mesh.n_dofs
    ud = torch.empty(ndof, dtype=torch.float64, device="cuda")
    g = torch.empty(nf, dtype=torch.float64, device="cuda")
    x = torch.empty(nf, dtype=torch.float64, device="cuda")
    dx = torch.empty(ndof, dtype=torch.float64, device="cuda")
    dx_host = torch.empty(ndof, dtype=torch.float64).pin_memory()
    it, rr = ctypes.c_int(), ctypes.c_double()
    P = ctypes_ptr
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]

    def step():
        with torch.cuda.stream(stream):
            ev[0].record(stream)
            ud.copy_(u_host, non_blocking=True)
            check(L.pfg_gradient_reduced(h, P(ud.data_ptr()), 1, 0, P(g.data_ptr())), h, "pfg_gradient_reduced")
            ev[1].record(stream)
            check(L.pfg_hessian_reduced(h, P(ud.data_ptr()), 1, 0, 1, None), h, "pfg_hessian_reduced")
            ev[2].record(stream)
            check(L.pfg_cg_solve(h, 1, None, P(g.data_ptr()), 1, 1e-6, 5000, 0, P(x.data_ptr()), ctypes.byref(it),
                                 ctypes.byref(rr)), h, "pfg_cg_solve")
            ev[3].record(stream)
            check(L.pfg_reduced_to_full(h, P(x.data_ptr()), None, 1, P(dx.data_ptr())), h, "pfg_reduced_to_full")
            dx_host.copy_(dx, non_blocking=True)
            ev[4].record(stream)
        torch.cuda.synchronize()
        return [ev[i].elapsed_time(ev[i + 1]) for i in range(4)]

    step()
    parts = [step() for _ in range(steps)]
    med = [statistics.median(p[i] for p in parts) for i in range(4)]
    total = sum(med)
    E = mesh.n_elements
    return {"value": E / (total * 1e-3), "unit": UNIT, "ms_per_step": total,
            "h2d_bytes_per_step": ndof * 8, "d2h_bytes_per_step": ndof * 8,
            "ms_gradient": med[0], "ms_hessian_psd": med[1], "ms_cg": med[2], "ms_step_out": med[3],
            "cg_iterations": it.value, "cg_rel_residual": rr.value, "n_free": nf,
            "note": "NLProblem's Newton step with the matrix kept on the device: reduced gradient, reduced "
                    "PSD-projected FP64 Hessian, Jacobi-preconditioned CG to 1e-6, reduced_to_full; "
                    "median of the timed steps"}


def time_newton_step_direct(asm, h, mesh, u_host, stream, steps):
    """The same Newton step with the sparse direct solve (pfg_direct_*) in place of
    CG, on the same context and Dirichlet set (the analysis is made once, as
    polysolve's analyzePattern, and timed apart): pinned u in, reduced gradient,
    reduced PSD-projected FP64 Hessian, factorisation, solve, reduced_to_full,
    pinned step out.  The CG solve of the same system (to 1e-6) is timed beside it.
    The factor is released afterwards."""
    import ctypes
    import time

    import torch

    from polyfem_b200 import PfgError
    from polyfem_b200._lib import PFG_ERR_OOM, check, lib
    L = lib()
    P = ctypes_ptr
    L.pfg_set_stream(h, P(stream.cuda_stream))
    nf, ndof = asm.n_free, mesh.n_dofs
    ud = torch.empty(ndof, dtype=torch.float64, device="cuda")
    g = torch.empty(nf, dtype=torch.float64, device="cuda")
    x = torch.empty(nf, dtype=torch.float64, device="cuda")
    xc = torch.empty(nf, dtype=torch.float64, device="cuda")
    dx = torch.empty(ndof, dtype=torch.float64, device="cuda")
    dx_host = torch.empty(ndof, dtype=torch.float64).pin_memory()
    with torch.cuda.stream(stream):
        ud.copy_(u_host, non_blocking=True)
        check(L.pfg_hessian_reduced(h, P(ud.data_ptr()), 1, 0, 1, None), h, "pfg_hessian_reduced")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    try:
        check(L.pfg_direct_analyze(h, 1), h, "pfg_direct_analyze")
    except PfgError as e:
        if e.status != PFG_ERR_OOM:
            raise
        return {"unavailable": str(e)}
    t_an = time.perf_counter() - t0
    st = (ctypes.c_longlong * 7)()
    check(L.pfg_direct_stats(h, st), h, "pfg_direct_stats")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(7)]

    def step():
        with torch.cuda.stream(stream):
            ev[0].record(stream)
            ud.copy_(u_host, non_blocking=True)
            check(L.pfg_gradient_reduced(h, P(ud.data_ptr()), 1, 0, P(g.data_ptr())), h, "pfg_gradient_reduced")
            ev[1].record(stream)
            check(L.pfg_hessian_reduced(h, P(ud.data_ptr()), 1, 0, 1, None), h, "pfg_hessian_reduced")
            ev[2].record(stream)
            check(L.pfg_direct_factorize(h, 1, None), h, "pfg_direct_factorize")
            ev[3].record(stream)
            check(L.pfg_direct_solve(h, 1, P(g.data_ptr()), 1, P(x.data_ptr())), h, "pfg_direct_solve")
            ev[4].record(stream)
            check(L.pfg_reduced_to_full(h, P(x.data_ptr()), None, 1, P(dx.data_ptr())), h, "pfg_reduced_to_full")
            dx_host.copy_(dx, non_blocking=True)
            ev[5].record(stream)
        torch.cuda.synchronize()
        return [ev[i].elapsed_time(ev[i + 1]) for i in range(5)]

    step()
    parts = [step() for _ in range(steps)]
    med = [statistics.median(p[i] for p in parts) for i in range(5)]
    check(L.pfg_direct_free(h), h, "pfg_direct_free")
    it, rr = ctypes.c_int(), ctypes.c_double()
    with torch.cuda.stream(stream):
        ev[5].record(stream)
        check(L.pfg_cg_solve(h, 1, None, P(g.data_ptr()), 1, 1e-6, 20000, 0, P(xc.data_ptr()), ctypes.byref(it),
                             ctypes.byref(rr)), h, "pfg_cg_solve")
        ev[6].record(stream)
    torch.cuda.synchronize()
    cg_ms = ev[5].elapsed_time(ev[6])
    diff = float((x - xc).norm() / x.norm())
    total = sum(med)
    E = mesh.n_elements
    return {"value": E / (total * 1e-3), "unit": UNIT, "ms_per_step": total, "n_free": nf,
            "h2d_bytes_per_step": ndof * 8, "d2h_bytes_per_step": ndof * 8,
            "ms_gradient": med[0], "ms_hessian_psd": med[1], "ms_factorize": med[2], "ms_solve": med[3],
            "ms_step_out": med[4], "s_analyze": t_an, "fronts": st[1], "nnz_L": st[4], "max_front": st[5],
            "front_GB": st[3] * 8e-9, "factorize_flops": st[6],
            "factorize_tflops": st[6] / (med[2] * 1e-3) / 1e12,
            "cg_ms_same_system": cg_ms, "cg_iterations": it.value, "rel_diff_vs_cg_1e-6": diff,
            "note": "NLProblem's Newton step with the sparse direct solve on the device (multifrontal "
                    "Cholesky, nested dissection) on the workload's own reduced system; the analysis is made "
                    "once per pattern; median of the timed steps"}


# ----------------------------------------------------------------- the other four workloads
def measure_configs(stream, peak):
    """Device times of the operations the other workloads name, inputs resident in
    HBM, L2 flushed before every timed launch (CUDA events on the context's stream):
      1  P1 20^3: FP64 energy, gradient, Hessian (L2-resident sizes: the flush makes
         every launch read from DRAM)
      1L P1 48^3: FP64 and FP32 energy and gradient (the HBM roofline of P1)
      3  Q1 96^3 jittered: FP32 energy and gradient (FP64 det and reduction), split32
         Hessian on the tensor cores, FP64 Hessian, split error vs FP64
      4  P1 48^3: material VJP
      5  P2 32^3 jittered: shape VJP, FP64 and FP32
    Algorithmic bytes: conn + gconn (when distinct) + Lame + X + u (+ p) read once,
    outputs written once (+ the Hessian's one int32 per element node pair)."""
    import ctypes

    import torch

    from polyfem_b200 import NeoHookeanAssembler
    from polyfem_b200 import mesh as M
    from polyfem_b200._lib import lib

    L = lib()
    vp = ctypes.c_void_p
    flush = torch.zeros(128 << 20, dtype=torch.float32, device="cuda")
    out = {}

    def timed(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        return _events_ms_flushed(stream, fn, reps, flush)

    def entry(ms, E, nbytes):
        gbs = nbytes / (ms * 1e-3) / 1e9
        return {"ms": round(ms, 4), "elements_per_s": E / (ms * 1e-3), "alg_bytes": int(nbytes),
                "alg_GBps": round(gbs, 1), "frac_hbm": round(gbs / peak, 4)}

    plan = [("1_p1_20", 1, None), ("1L_p1_48", 4, None), ("3_q1_96", 3, None), ("4_p1_48", 4, None),
            ("5_p2_32", 5, None)]
    for key, k, grid in plan:
        mesh, lam, mu, u, p = M.workload(k, grid)
        E, n, ng = mesh.n_elements, mesh.conn.shape[1], mesh.gconn.shape[1]
        asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
        h = asm.handle
        L.pfg_set_stream(h, vp(stream.cuda_stream))
        ud = torch.tensor(u, dtype=torch.float64, device="cuda")
        pd = torch.tensor(p, dtype=torch.float64, device="cuda")
        o = torch.empty(max(mesh.n_dofs, 2 * E, 3 * mesh.n_geom_nodes), dtype=torch.float64, device="cuda")
        U, P, O = vp(ud.data_ptr()), vp(pd.data_ptr()), vp(o.data_ptr())
        ins = (E * n * 4 + (E * ng * 4 if mesh.gconn is not mesh.conn else 0) + E * 16
               + mesh.n_geom_nodes * 24 + mesh.n_nodes * 24)
        res = {"workload": M.WORKLOADS[k] if grid is None else f"workload {k} at {grid}^3", "E": E}
        if key == "1_p1_20":
            nnz = asm.hessian_nnz()
            res["energy_fp64"] = entry(timed(lambda: L.pfg_energy(h, U, 1, 0, O), 50), E, ins + 8)
            res["gradient_fp64"] = entry(timed(lambda: L.pfg_gradient(h, U, 1, 0, O), 50), E, ins + mesh.n_dofs * 8)
            res["hessian_fp64"] = entry(timed(lambda: L.pfg_hessian(h, U, 1, 0, 0, None), 20), E,
                                        algorithmic_bytes(mesh, nnz))
        elif key == "1L_p1_48":
            for prec, name in ((0, "fp64"), (1, "fp32")):
                res[f"energy_{name}"] = entry(timed(lambda: L.pfg_energy(h, U, 1, prec, O), 50), E, ins + 8)
                res[f"gradient_{name}"] = entry(timed(lambda: L.pfg_gradient(h, U, 1, prec, O), 50), E,
                                                ins + mesh.n_dofs * 8)
        elif key == "3_q1_96":
            nnz = asm.hessian_nnz()
            res["energy_fp32"] = entry(timed(lambda: L.pfg_energy(h, U, 1, 1, O), 30), E, ins + 8)
            res["gradient_fp32"] = entry(timed(lambda: L.pfg_gradient(h, U, 1, 1, O), 30), E, ins + mesh.n_dofs * 8)
            v64 = torch.empty(nnz, dtype=torch.float64, device="cuda")
            vs = torch.empty(nnz, dtype=torch.float64, device="cuda")
            V64, VS = vp(v64.data_ptr()), vp(vs.data_ptr())
            res["hessian_split32"] = entry(timed(lambda: L.pfg_hessian(h, U, 1, 2, 0, VS), 10), E,
                                           algorithmic_bytes(mesh, nnz))
            res["hessian_fp64"] = entry(timed(lambda: L.pfg_hessian(h, U, 1, 0, 0, V64), 10), E,
                                        algorithmic_bytes(mesh, nnz))
            torch.cuda.synchronize()
            res["hessian_split32"]["rel_err_vs_fp64"] = float(torch.linalg.vector_norm(vs - v64)
                                                              / torch.linalg.vector_norm(v64))
            res["split_over_fp64"] = res["hessian_fp64"]["ms"] / res["hessian_split32"]["ms"]
            del v64, vs
        elif key == "4_p1_48":
            res["material_vjp"] = entry(timed(lambda: L.pfg_material_vjp(h, U, P, 1, O), 50), E,
                                        ins + mesh.n_nodes * 24 + 2 * E * 8)
        elif key == "5_p2_32":
            for prec, name in ((0, "fp64"), (1, "fp32")):
                res[f"shape_vjp_{name}"] = entry(timed(lambda: L.pfg_shape_vjp(h, U, P, 1, prec, O), 30), E,
                                                 ins + mesh.n_nodes * 24 + 3 * mesh.n_geom_nodes * 8)
            torch.cuda.synchronize()
        out[key] = res
        asm.close()
        torch.cuda.empty_cache()
    return out


# ----------------------------------------------------------------- per-operation suite
SUITE = {
    # key: (element order or 'hex', grid, jitter, lognormal Lame, displacement kind, description)
    "P1-20": ("p1", 20, 0.0, False, "rand", "P1 tets 20^3 x 6 (48,000), homogeneous E=1e5 nu=0.35"),
    "P1-48": ("p1", 48, 0.0, True, "rand", "P1 tets 48^3 x 6 (663,552), lognormal Lame"),
    "P2-40": ("p2", 40, 0.0, True, "rand", "P2 tets 40^3 x 6 (384,000), lognormal Lame"),
    "P2-32j": ("p2", 32, 0.1, False, "rand", "P2 tets 32^3 x 6 (196,608), jittered rest positions, homogeneous"),
    "P2-24": ("p2", 24, 0.0, True, "rand", "P2 tets 24^3 x 6 (82,944), lognormal Lame: the small case of the ncu captures"),
    "Q1-96j": ("hex", 96, 0.1, True, "smooth", "Q1 hexes 96^3 (884,736), jittered, lognormal Lame, smooth u"),
}


def run_suite(args):
    """Per-operation device timings on every workload: inputs resident in HBM, L2
    flushed before every timed launch, CUDA events around each launch."""
    import ctypes

    import torch

    from polyfem_b200 import NeoHookeanAssembler
    from polyfem_b200 import mesh as M
    from polyfem_b200._lib import check, lib

    L = lib()
    vp = ctypes.c_void_p
    stream = torch.cuda.Stream()
    peak, _ = _peaks()
    names = args.only.split(",") if args.only else list(SUITE)
    flush = torch.zeros(128 << 20, dtype=torch.float32, device="cuda")  # 2 x 256 MB, each > 126 MB L2
    for name in names:
        kind, g, jit, logn, disp, desc = SUITE[name]
        if kind == "hex":
            mesh = M.structured_hex_mesh(g, jitter=jit, seed=3)
        else:
            mesh = M.structured_tet_mesh(g, 1 if kind == "p1" else 2, jitter=jit, seed=3)
        E = mesh.n_elements
        lam, mu = M.lognormal_lame(E, SEED_LAME) if logn else M.homogeneous_lame(E)
        u = M.random_displacement(mesh, 0.02, SEED_U) if disp == "rand" else M.smooth_displacement(mesh, 0.05, 0.005, 4)
        asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
        nnz = asm.hessian_nnz()
        h = asm.handle
        L.pfg_set_stream(h, vp(stream.cuda_stream))
        ud = torch.tensor(u, dtype=torch.float64, device="cuda")
        pd = torch.randn(mesh.n_dofs, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(7))
        out = torch.empty(max(mesh.n_dofs, 2 * E, 3 * mesh.n_geom_nodes), dtype=torch.float64, device="cuda")
        U, P, O = vp(ud.data_ptr()), vp(pd.data_ptr()), vp(out.data_ptr())
        mvals = torch.empty(nnz, dtype=torch.float64, device="cuda")
        MV = vp(mvals.data_ptr())
        ops = {
            "energy_fp64": lambda: L.pfg_energy(h, U, 1, 0, O),
            "energy_fp32": lambda: L.pfg_energy(h, U, 1, 1, O),
            "gradient_fp64": lambda: L.pfg_gradient(h, U, 1, 0, O),
            "gradient_fp32": lambda: L.pfg_gradient(h, U, 1, 1, O),
            "hessian_fp64": lambda: L.pfg_hessian(h, U, 1, 0, 0, None),
            "hessian_fp32": lambda: L.pfg_hessian(h, U, 1, 1, 0, None),
            "hessian_split32": lambda: L.pfg_hessian(h, U, 1, 2, 0, None),
            "hessian_psd_fp64": lambda: L.pfg_hessian(h, U, 1, 0, 1, None),
            "hessian_psd_split32": lambda: L.pfg_hessian(h, U, 1, 2, 1, None),
            "material_vjp": lambda: L.pfg_material_vjp(h, U, P, 1, O),
            "shape_vjp_fp64": lambda: L.pfg_shape_vjp(h, U, P, 1, 0, O),
            "shape_vjp_fp32": lambda: L.pfg_shape_vjp(h, U, P, 1, 1, O),
            "mass_matrix": lambda: L.pfg_mass_matrix(h, None, 1, MV),
            # row-sum lumping of the mass values just assembled (utils::lump_matrix)
            "lump_matrix": lambda: L.pfg_lump_matrix(h, MV, 1, O),
        }
        # algorithmic bytes of the HBM-bound operations
        n, ng = mesh.conn.shape[1], mesh.gconn.shape[1]
        ins = E * n * 4 + (E * ng * 4 if mesh.gconn is not mesh.conn else 0) + E * 16 + mesh.n_geom_nodes * 24 + mesh.n_nodes * 24
        alg = {"energy_fp64": ins + 8, "energy_fp32": ins + 8,
               "gradient_fp64": ins + mesh.n_dofs * 8, "gradient_fp32": ins + mesh.n_dofs * 8,
               "material_vjp": ins + mesh.n_nodes * 24 + 2 * E * 8,
               "hessian_fp64": algorithmic_bytes(mesh, nnz), "hessian_fp32": algorithmic_bytes(mesh, nnz),
               "hessian_split32": algorithmic_bytes(mesh, nnz),
               # every value read once, the diagonal written, the column starts read
               "lump_matrix": nnz * 8 + mesh.n_dofs * 8 + (mesh.n_dofs + 1) * 4}
        # Dirichlet reduction: the dofs of the x = 0 face constrained
        face = np.flatnonzero(mesh.node_pos[:, 0] <= 1e-12)
        asm.set_dirichlet((3 * face[:, None] + np.arange(3)).ravel())
        L.pfg_set_stream(h, vp(stream.cuda_stream))
        ops["hessian_dirichlet_split32"] = lambda: L.pfg_hessian_reduced(h, U, 1, 2, 0, None)
        ops["hessian_dirichlet_fp64"] = lambda: L.pfg_hessian_reduced(h, U, 1, 0, 0, None)
        res = {}
        for op, fn in ops.items():
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            reps = 10 if op.startswith("hessian") else 50
            ms = _events_ms_flushed(stream, fn, reps, flush)
            r = {"us": round(ms * 1e3, 2), "elements_per_s": E / (ms * 1e-3)}
            if op in alg:
                gbs = alg[op] / (ms * 1e-3) / 1e9
                r["alg_GBps"] = round(gbs, 1)
                r["frac_hbm"] = round(gbs / peak, 4)
            res[op] = r
        # device conjugate gradient on the reduced, PSD-projected FP64 Hessian: 50
        # iterations (tolerance 0), one |r|^2 read-back per iteration included
        check(L.pfg_hessian_reduced(h, U, 1, 0, 1, None), h, "pfg_hessian_reduced")
        nf, rnnz = asm.n_free, asm._red_nnz
        bd = torch.randn(nf, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(9))
        xd = torch.empty(nf, dtype=torch.float64, device="cuda")
        it, rr = ctypes.c_int(), ctypes.c_double()
        cg = lambda: L.pfg_cg_solve(h, 1, None, vp(bd.data_ptr()), 1, 0.0, 50, 0, vp(xd.data_ptr()),
                                    ctypes.byref(it), ctypes.byref(rr))
        cg()
        ms = _events_ms_flushed(stream, cg, 3, flush)
        # per iteration: values + rows of the SpMV (12 B per nonzero), its column
        # offsets, gathered p and q (4 + 8 + 8 B per dof), then x, r, z, p, q, D^-1
        # read and x, r, z, p written by the update kernels (88 B per dof)
        it_bytes = 12 * rnnz + 108 * nf
        per_it = ms / max(it.value, 1)
        gbs = it_bytes / (per_it * 1e-3) / 1e9
        res["cg_reduced_psd"] = {"us": round(ms * 1e3, 2), "iterations": it.value,
                                 "us_per_iteration": round(per_it * 1e3, 2), "alg_GBps": round(gbs, 1),
                                 "frac_hbm": round(gbs / peak, 4), "n": nf, "nnz": rnnz}
        # the other materials (FP64): energy, gradient and the Hessian; the
        # parameterised ones with (c1, c2, k), (c1, c2, c3, d1), (k) of stress scale mu
        mu_s = float(np.median(mu))
        mpar = {4: [mu_s, 0.5 * mu_s, 10 * mu_s], 5: [mu_s, 0.5 * mu_s, 0.2 * mu_s, 10 * mu_s], 6: [10 * mu_s],
                # Ogden: two terms (alpha, mu, D) / three terms (c, m) and k
                9: [1.3, 5.0, mu_s, 0.02 * mu_s, 0.1 / mu_s, 1.0 / mu_s],
                10: [mu_s, 0.03 * mu_s, -0.02 * mu_s, 1.3, 5.0, -2.0, 10 * mu_s]}
        # HookeLinearElasticity and the anisotropic SaintVenant: the isotropic tensor of
        # (2.333 mu, mu) (nu = 0.35) plus a seeded symmetric positive semi-definite part
        Ct = np.zeros((6, 6))
        Ct[:3, :3] = 2.333 * mu_s
        Ct[[0, 1, 2], [0, 1, 2]] += 2 * mu_s
        Ct[[3, 4, 5], [3, 4, 5]] = mu_s
        Rt = np.random.default_rng(7).standard_normal((6, 6))
        Ct += 0.25 * mu_s * (Rt @ Rt.T) / 6
        c21 = np.ascontiguousarray(Ct[np.triu_indices(6)])
        check(L.pfg_set_elasticity_tensor(h, vp(c21.ctypes.data)), h, "pfg_set_elasticity_tensor")
        for mname, mid in (("iso_neohookean", 1), ("saint_venant", 2), ("linear_elasticity", 3),
                           ("mooney_rivlin", 4), ("mooney_rivlin_3param", 5), ("volume_penalty", 6),
                           ("hooke", 7), ("saint_venant_tensor", 8), ("unconstrained_ogden", 9),
                           ("incompressible_ogden", 10)):
            if mid in mpar:
                pv = np.ascontiguousarray(np.repeat(np.asarray(mpar[mid], dtype=np.float64)[:, None], E, axis=1))
                check(L.pfg_set_material_params(h, vp(pv.ctypes.data), len(mpar[mid]), 0), h,
                      "pfg_set_material_params")
                L.pfg_set_stream(h, vp(stream.cuda_stream))
            check(L.pfg_set_material(h, mid), h, "pfg_set_material")
            mops = {f"energy_{mname}": lambda: L.pfg_energy(h, U, 1, 0, O),
                    f"gradient_{mname}": lambda: L.pfg_gradient(h, U, 1, 0, O),
                    f"hessian_{mname}": lambda: L.pfg_hessian(h, U, 1, 0, 0, None)}
            for op, fn in mops.items():
                for _ in range(3):
                    fn()
                torch.cuda.synchronize()
                ms = _events_ms_flushed(stream, fn, 10 if op.startswith("hessian") else 50, flush)
                res[op] = {"us": round(ms * 1e3, 2), "elements_per_s": E / (ms * 1e-3)}
        check(L.pfg_set_material(h, 0), h, "pfg_set_material")
        print(json.dumps({"suite": name, "workload": desc, "E": E, "N": mesh.n_nodes, "nnz": nnz, "ops": res}), flush=True)
        asm.close()
    return 0


def run_profile_case(args):
    """The Hessian assembly of one precision alone on a G^3 P2 cube (the command the
    ncu captures run): warm-up calls, then `steps` timed calls; prints one line."""
    import torch

    from polyfem_b200 import NeoHookeanAssembler
    from polyfem_b200._lib import check, lib
    from polyfem_b200.assembler import PRECISIONS

    prec = PRECISIONS[args.profile]
    mesh, lam, mu, u = _workload(args.grid)
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu)
    asm.hessian_nnz()
    L = lib()
    h = asm.handle
    stream = torch.cuda.Stream()
    check(L.pfg_set_stream(h, ctypes_ptr(stream.cuda_stream)), h, "pfg_set_stream")
    ud = torch.tensor(u, device="cuda", dtype=torch.float64)
    fn = lambda: check(L.pfg_hessian(h, ctypes_ptr(ud.data_ptr()), 1, prec, 0, None), h, "pfg_hessian")
    for _ in range(args.warmup):
        fn()
    torch.cuda.synchronize()
    ms = _events_ms(stream, fn, args.steps)
    check(L.pfg_synchronize(h), h, "pfg_synchronize")
    print(json.dumps({"profile_case": workload_name(args.grid), "precision": args.profile, "ms": ms,
                      "elements_per_s": mesh.n_elements / (ms * 1e-3)}), flush=True)
    asm.close()
    return 0


def ctypes_ptr(p):
    import ctypes
    return ctypes.c_void_p(int(p))


def _peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s"


def _profiled_traffic(grid: int):
    """DRAM bytes per pfg_hessian call (both kernels) from the committed ncu summary,
    scaled from the profiled case to this workload by elements (traffic grows in
    proportion to the elements processed)."""
    path = os.path.join(REPO, "profiles", "hessian_p2_split32.txt")
    try:
        per_elem = None
        for ln in open(path):
            if ln.startswith("traffic_bytes_per_element"):
                per_elem = float(ln.split("=")[1].split()[0])
        if per_elem is not None:
            return per_elem * 6 * grid ** 3
    except Exception:
        pass
    return None


def main():
    faulthandler.enable()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=40, help="P2 cube cells per axis (40 = the benchmark workload)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-configs", action="store_true", help="skip the per-workload timings of configs 1, 3, 4, 5")
    ap.add_argument("--suite", action="store_true", help="per-operation timings on all workloads")
    ap.add_argument("--no-newton", action="store_true", help="skip the device-resident Newton step")
    ap.add_argument("--profile", default="", choices=["", "fp64", "fp32", "split32", "split32_simt"],
                    help="time only this precision's Hessian on the --grid cube (the ncu capture command)")
    ap.add_argument("--only", default="", help="comma-separated suite workload keys (" + ",".join(SUITE) + ")")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile:
        return run_profile_case(args)
    if args.suite:
        return run_suite(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
