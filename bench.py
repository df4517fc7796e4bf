#!/usr/bin/env python
"""Benchmark: NeoHookean element Hessians/s on B200 (split-FP32 vs FP64, rel err vs FP64).

Workload (the configuration the metric is quoted on): P2 tetrahedra on a 40^3 cube
split 6 tets/hex (384,000 elements, 531,441 nodes, 1,594,323 dofs, 134,475,849
CSC nonzeros), 4-point quadrature, per-element lognormal Lame parameters, seeded
synthetic displacement u = 0.02 h N(0,1).  One step = one assembly of the global
Hessian CSC values through the path's C ABI (pfg_hessian).

  value     : split-precision Hessian assembly, inputs resident in HBM (elements/s)
  e2e       : the same call with host buffers (pinned u in, CSC values out) (elements/s)
  fp64      : the plain FP64 drop-in kernel, same workload (elements/s)
  cpu_baseline / --impl reference : the CPU oracle port of the reference's TBB
              assembly (NLAssembler::assemble_hessian) on the host cores.

Run:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
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

WORKLOAD = "P2 tet NeoHookean Hessian assembly, 40^3 cube x 6 tets (384,000 elements, 1,594,323 dofs)"
METRIC = "NeoHookean elem Hessians/s on 1 B200: split-FP32 vs FP64, rel err vs FP64"
UNIT = "elements/s"
GRID = 40
SEED_LAME, SEED_U = 5, 2


def _rank_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def _workload():
    from polyfem_b200 import mesh as M
    mesh = M.structured_tet_mesh(GRID, 2)
    lam, mu = M.lognormal_lame(mesh.n_elements, SEED_LAME)
    u = M.random_displacement(mesh, 0.02, SEED_U)
    return mesh, lam, mu, u


def algorithmic_bytes(mesh, nnz: int) -> int:
    """Bytes a Hessian assembly must move at least once (documented in DESIGN.md):
    conn + gconn + Lame + X + u + slot map + column strides read, CSC values written."""
    E, n, ng = mesh.n_elements, mesh.conn.shape[1], mesh.gconn.shape[1]
    return (E * n * 4 + E * ng * 4 + E * 16 + mesh.n_geom_nodes * 24 + mesh.n_nodes * 24
            + E * n * n * 4 + mesh.n_nodes * 4 + nnz * 8)


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """Samples nvidia-smi during the timed region (clocks and throttle reasons)."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


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
    mesh, lam, mu, u = _workload()
    import psutil  # noqa: F401  (memory probe inside cpu_threads_for)
    nnz = 134475849
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
        "config": {"workload": WORKLOAD, "precision": "fp64",
                   "implementation": "C++ restatement of NLAssembler::assemble_hessian + SparseMatrixCache (oracle/pf_oracle.cpp), std::thread"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nt, "kind": "port",
                         "sample": f"full 40^3 P2 Hessian per step (384,000 elements), steady-state calls; first call (pattern build) {t_first:.2f} s"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------- GPU arm
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
    from polyfem_b200._lib import PFG_FP64, PFG_MEM_DEVICE, PFG_MEM_HOST, PFG_SPLIT32, check, lib

    mesh, lam, mu, u = _workload()
    asm = NeoHookeanAssembler.from_mesh(mesh, lam, mu, device=local)
    nnz = asm.hessian_nnz()
    E = mesh.n_elements
    L = lib()
    h = asm.handle
    stream = torch.cuda.Stream(device=local)
    check(L.pfg_set_stream(h, ctypes_ptr(stream.cuda_stream)), h, "pfg_set_stream")
    ud = torch.tensor(u, device=f"cuda:{local}", dtype=torch.float64)
    vals_dev = torch.empty(nnz, device=f"cuda:{local}", dtype=torch.float64)

    def call(prec, mem, uptr, vptr):
        check(L.pfg_hessian(h, uptr, mem, prec, 0, vptr), h, "pfg_hessian")

    def timed_device(prec, steps, warmup):
        for _ in range(warmup):
            call(prec, PFG_MEM_DEVICE, ctypes_ptr(ud.data_ptr()), None)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(steps):
            call(prec, PFG_MEM_DEVICE, ctypes_ptr(ud.data_ptr()), None)
        end.record(stream)
        torch.cuda.synchronize()
        ms = start.elapsed_time(end) / steps
        if dist is not None:
            t = torch.tensor([ms], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t)
        return ms

    # accuracy of the headline precision against the FP64 drop-in
    call(PFG_FP64, PFG_MEM_DEVICE, ctypes_ptr(ud.data_ptr()), ctypes_ptr(vals_dev.data_ptr()))
    torch.cuda.synchronize()
    v64 = vals_dev.clone()
    call(PFG_SPLIT32, PFG_MEM_DEVICE, ctypes_ptr(ud.data_ptr()), ctypes_ptr(vals_dev.data_ptr()))
    torch.cuda.synchronize()
    rel_err = float(torch.linalg.vector_norm(vals_dev - v64) / torch.linalg.vector_norm(v64))
    del v64

    ms64 = timed_device(PFG_FP64, args.steps, args.warmup)
    sampler = ClockSampler(local)
    sampler.start()
    ms_split = timed_device(PFG_SPLIT32, args.steps, args.warmup)
    clocks = sampler.stop()

    # end to end through the C ABI with host buffers (pinned u in, pinned CSC values out)
    u_host = torch.tensor(u, dtype=torch.float64).pin_memory()
    v_host = torch.empty(nnz, dtype=torch.float64).pin_memory()
    for _ in range(max(1, args.warmup)):
        call(PFG_SPLIT32, PFG_MEM_HOST, ctypes_ptr(u_host.data_ptr()), ctypes_ptr(v_host.data_ptr()))
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        call(PFG_SPLIT32, PFG_MEM_HOST, ctypes_ptr(u_host.data_ptr()), ctypes_ptr(v_host.data_ptr()))
    e2e_s = (time.perf_counter() - t0) / args.steps
    if dist is not None:
        t = torch.tensor([e2e_s], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t)

    bytes_alg = algorithmic_bytes(mesh, nnz)
    peaks = _peaks()
    achieved = bytes_alg / (ms_split * 1e-3) / 1e9
    traffic = _profiled_traffic()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        nt = cpu_threads_for(nnz)
        times, t_first = time_cpu_reference(mesh, lam, mu, u, nt, 2)
        t = min(times)
        cpu = {"value": E / t, "unit": UNIT, "cores": nt, "kind": "port",
               "sample": f"full 40^3 P2 Hessian (384,000 elements), best of 2 steady-state calls; pattern build {t_first:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": world * E / (ms_split * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_split, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (3xTF32 split) + f64 det/CSC",
            "data": "synthetic (seeded 40^3 P2 mesh, lognormal Lame, u = 0.02 h N(0,1))",
            "config": {"workload": WORKLOAD, "global_batch": world * E, "parallelism": f"replicas x{world}",
                       "precision": "split32", "nnz": nnz, "l2": "inputs larger than L2 (1.08 GB CSC values)"},
            "fp64": {"value": world * E / (ms64 * 1e-3), "unit": UNIT, "ms_per_step": ms64},
            "split_over_fp64": ms64 / ms_split,
            "rel_err_vs_fp64": rel_err,
            "e2e": {"value": world * E / e2e_s, "unit": UNIT, "h2d_bytes_per_step": u_host.numel() * 8,
                    "d2h_bytes_per_step": nnz * 8},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks[0], "unit": "GB/s",
                         "frac": achieved / peaks[0], "traffic": traffic, "peak_source": peaks[1],
                         "bytes_alg_per_launch": bytes_alg,
                         "note": "pfg_hessian call (value zeroing + assembly kernel), CUDA events on its stream"},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": args.steps * 1,
        }
        print(json.dumps(line), flush=True)
    asm.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
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


def _profiled_traffic():
    """DRAM bytes per launch of the Hessian assembly from the committed ncu summary."""
    path = os.path.join(REPO, "profiles", "hessian_p2_40.txt")
    try:
        for ln in open(path):
            if ln.startswith("traffic_bytes_per_launch"):
                return float(ln.split("=")[1].split()[0])
    except Exception:
        pass
    return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
