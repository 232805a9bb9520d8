#!/usr/bin/env python
"""Benchmark: Global SPAI MR + PCG to 1e-8 on the 64^3 7-point log-normal
diffusion operator, mixed precision vs FP64, on one B200 per rank.

Workload (synthetic, seeded; no public data set is involved):
  A      7-point variable-coefficient diffusion on a 64^3 grid, face
         coefficients exp(N(0,1)) (numpy default_rng(0)), Dirichlet boundary:
         n = 262,144, nnz = 1,810,432.
  SPAI   Global MR (reference src/global_spai/minimal_residual.cpp), 30
         iterations, M0 = diag(A)^-1, Pr = diag(A)^-1 (the reference default),
         dropping on with at most 16 entries per column by magnitude.
  PCG    b = A x*, x* ~ N(0,1) (default_rng(0)), x0 = 0, relative tolerance
         1e-8, true-residual refresh every 50 iterations, preconditioned with
         the symmetric part (M + M^T)/2 of the SPAI result (PCG needs a
         symmetric preconditioner; MR iterates are not symmetric).
  step   one SPAI build followed by one PCG solve.

`value` is SPAI iterations per second of the mixed-precision step (FP32
storage of M, R, Z, A; FP64 reductions; PCG in FP64 with FP32 M-apply), timed
with CUDA events on the library's stream, inputs resident in HBM, L2 flushed
before every step.  The same line carries the PCG time to 1e-8, the FP64 step
for comparison, the end-to-end figure through the C ABI with host buffers,
the roofline of the dominant kernel and the CPU baseline, plus a batched leg
(256 independent systems in one call, against one call per system).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "SPAI iters/s + PCG time to 1e-8, mixed vs FP64 on one B200, 64³ 7-pt"
UNIT = "SPAI iters/s"


def parse_args():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--grid", type=int, default=64, help="grid edge of the 7-point operator (64 -> 64^3)")
    p.add_argument("--spai-iterations", type=int, default=30)
    p.add_argument("--topk", type=int, default=16)
    p.add_argument("--pcg-tolerance", type=float, default=1e-8)
    p.add_argument("--pcg-refresh", type=int, default=50)
    p.add_argument("--pcg-max-iterations", type=int, default=5000)
    p.add_argument("--skip-cpu-baseline", action="store_true")
    p.add_argument("--skip-e2e", action="store_true")
    p.add_argument("--skip-batched", action="store_true")
    p.add_argument("--batch-count", type=int, default=256, help="systems in the batched leg")
    p.add_argument("--batch-iterations", type=int, default=15)
    p.add_argument("--batch-topk", type=int, default=10)
    return p.parse_args()


def workload(args):
    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import problems
    A = problems.diffusion_3d(args.grid, 1.0, 0)
    M0 = problems.diagonal_inverse(A)
    b, _ = problems.solution_rhs(A, seed=0)
    return A, M0, b


def config_dict(args, A):
    n = A.shape[0]
    return {
        "workload": f"Global SPAI MR ({args.spai_iterations} it, top-{args.topk}/column) + PCG to "
                    f"{args.pcg_tolerance:g} on 7-pt log-normal diffusion {args.grid}^3",
        "grid": args.grid, "n": n, "nnz": int(A.nnz),
        "spai_method": "global_spai.mr", "spai_iterations": args.spai_iterations,
        "dropping": f"top-{args.topk} per column by magnitude (diagonal kept)",
        "m0": "diag(A)^-1", "pr": "diag(A)^-1",
        "pcg_tolerance": args.pcg_tolerance, "pcg_refresh_period": args.pcg_refresh,
        "pcg_preconditioner": "(M + M^T)/2 of the SPAI result",
        "precision": "mixed: FP32 storage of A, M, R, Z; FP64 reductions; PCG FP64 with FP32 M-apply",
        "l2": "flushed (256 MiB write) before every timed step",
    }


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device_index)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, sm_max, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                sm_max = max(sm_max, float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": sm_max or None,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peak_hbm():
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    path = ROOT / "profiles" / "roofline_traffic.json"
    try:
        data = json.loads(path.read_text())
        return data.get(kernel, {}).get("dram_bytes_per_launch")
    except (OSError, ValueError):
        return None


# ---------------------------------------------------------------------------
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    group = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        group = dist
    return world, rank, local, group


def barrier(group, device):
    """All ranks meet here (an all-reduce of one element), device drained."""
    if group is not None:
        import torch
        t = torch.zeros(1, device=device)
        group.all_reduce(t)
        if torch.device(device).type == "cuda":
            torch.cuda.synchronize(device)


def max_over_ranks(group, value, device):
    if group is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    group.all_reduce(t, op=group.ReduceOp.MAX)
    return float(t.item())


def run_ours(args):
    import torch
    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import Session, _lib, backward_error, global_spai

    world, rank, local, group = dist_setup(args)
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    lib = _lib.load()
    A, M0, b = workload(args)
    n = A.shape[0]
    sessions = {}
    for prec in ("mixed", "fp64"):
        s = Session("global_spai", "mr", A, M0=M0, max_iterations=args.spai_iterations, tolerance=1e-12,
                    max_density=float(args.topk) / n, precision=prec, topk_per_column=args.topk, device=local)
        s.set_rhs(b)
        sessions[prec] = s
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)  # 256 MiB > 126 MB L2

    def one_step(prec, record):
        s = sessions[prec]
        stream = torch.cuda.ExternalStream(s.stream, device=device)
        flush.zero_()
        torch.cuda.synchronize(device)
        torch.cuda.nvtx.range_push(f"{prec}_step" if record is not None else f"{prec}_warmup")
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e2 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        iterations, nnz_m = s.run()
        e1.record(stream)
        hist, status = s.pcg(args.pcg_max_iterations, args.pcg_tolerance, refresh_period=args.pcg_refresh,
                             m_precision=prec, symmetric_part=True)
        e2.record(stream)
        e2.synchronize()
        torch.cuda.nvtx.range_pop()
        spai_ms = e0.elapsed_time(e1)
        pcg_ms = e1.elapsed_time(e2)
        if record is not None:
            record.append({"spai_ms": spai_ms, "pcg_ms": pcg_ms, "iterations": iterations, "nnz_m": nnz_m,
                           "pcg_iterations": len(hist) - 1, "pcg_status": status, "pcg_final": float(hist[-1])})

    for _ in range(args.warmup):
        one_step("mixed", None)
        one_step("fp64", None)

    results = {"mixed": [], "fp64": []}
    barrier(group, device)
    torch.cuda.synchronize(device)
    launches0 = lib.spai_kernel_launches()
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            one_step("mixed", results["mixed"])
        launches = lib.spai_kernel_launches() - launches0
        for _ in range(args.steps):
            one_step("fp64", results["fp64"])
    torch.cuda.synchronize(device)
    barrier(group, device)

    # kernel classes: the same mixed steps again with the library's per-launch CUDA events
    # (kept out of the timed steps above, whose numbers they would perturb)
    lib.spai_profile_reset()
    lib.spai_profile_enable(1)
    for _ in range(args.steps):
        one_step("mixed", [])
    lib.spai_profile_enable(0)

    def agg(rows):
        spai = sum(r["spai_ms"] for r in rows)
        pcg = sum(r["pcg_ms"] for r in rows)
        its = sum(r["iterations"] for r in rows)
        return spai, pcg, its

    spai_ms, pcg_ms, its = agg(results["mixed"])
    spai_ms_max = max_over_ranks(group, spai_ms, device)
    step_ms_max = max_over_ranks(group, spai_ms + pcg_ms, device)
    f_spai, f_pcg, f_its = agg(results["fp64"])
    f_spai = max_over_ranks(group, f_spai, device)
    f_step = max_over_ranks(group, f_spai + f_pcg, device)

    # kernel classes from the library's CUDA-event accounting; the dominant one gives the roofline
    import ctypes
    peak, peak_kind = measured_peak_hbm()
    kernel_table = {}
    for name in ("fused_residual", "fused_drop", "fused_decide", "spgemm_numeric", "spgemm_symbolic",
                 "spgemm_compact", "drop_update", "union", "transpose", "filter", "pcg_solve", "pcg_spmv"):
        m2, c2, b2 = ctypes.c_double(0.0), ctypes.c_int64(0), ctypes.c_double(0.0)
        lib.spai_profile_read(name.encode(), ctypes.byref(m2), ctypes.byref(c2), ctypes.byref(b2))
        if c2.value == 0:
            continue
        kernel_table[name] = {"ms": round(m2.value, 3), "launches": c2.value,
                              "ms_per_launch": round(m2.value / c2.value, 4),
                              "bytes_per_launch": round(b2.value / c2.value) if b2.value > 0 else None,
                              "gbs": round(b2.value / (m2.value * 1e6), 1) if m2.value > 0 and b2.value > 0 else None,
                              "frac_of_hbm_peak": round(b2.value / (m2.value * 1e6) / peak, 4)
                              if m2.value > 0 and b2.value > 0 else None}
    dominant = max((k for k in kernel_table if kernel_table[k]["gbs"] is not None and k != "pcg_solve"),
                   key=lambda k: kernel_table[k]["ms"], default=None)
    dom = kernel_table.get(dominant, {})
    achieved = dom.get("gbs") or 0.0
    traffic = ncu_traffic(dominant) if dominant else None

    mixed_error = mixed_vs_fp64(sessions, results) if rank == 0 else None
    line = None
    if rank == 0:
        rows = results["mixed"]
        line = {
            "metric": METRIC,
            "value": round(world * its / (spai_ms_max * 1e-3), 3),
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(step_ms_max / args.steps, 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32-storage/f64-reductions",
            "data": "synthetic (seeded 64^3 log-normal diffusion operator; no public data set)",
            "config": config_dict(args, A),
            "spai_ms_per_build": round(spai_ms_max / args.steps, 3),
            "pcg_ms_to_tolerance": round((step_ms_max - spai_ms_max) / args.steps, 3),
            "pcg_iterations": rows[-1]["pcg_iterations"],
            "pcg_status": rows[-1]["pcg_status"],
            "pcg_final_relative_residual": rows[-1]["pcg_final"],
            "nnz_m": rows[-1]["nnz_m"],
            "fp64": {
                "spai_iters_per_s": round(world * f_its / (f_spai * 1e-3), 3),
                "spai_ms_per_build": round(f_spai / args.steps, 3),
                "pcg_ms_to_tolerance": round((f_step - f_spai) / args.steps, 3),
                "pcg_iterations": results["fp64"][-1]["pcg_iterations"],
                "ms_per_step": round(f_step / args.steps, 3),
            },
            "speedup_mixed_vs_fp64": round(f_step / step_ms_max, 3),
            "roofline": {
                "kernel": KERNEL_NOTES.get(dominant, dominant),
                "class": dominant,
                "measured": "library CUDA events on the session stream around each launch, in a second pass of "
                            "the same mixed steps with the fused iteration launched kernel by kernel",
                "bound": "hbm",
                "achieved": achieved,
                "peak": peak,
                "unit": "GB/s",
                "frac": round(achieved / peak, 4) if peak else None,
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "traffic": traffic,
                "launches": dom.get("launches"),
                "ms_per_launch": dom.get("ms_per_launch"),
                "algorithmic_bytes_per_launch": dom.get("bytes_per_launch"),
            },
            "graph": {"spai_iterations": "one CUDA graph launch per build: WHILE node over the fused drop, "
                                         "residual/projection and decide kernels (mr_fused.cu)",
                      "pcg": "one CUDA graph launch per solve: WHILE node over the PCG iteration (pcg.cu)"},
            "mixed_error": mixed_error,
            "kernel_classes_mixed": kernel_table,
            "clocks": clocks.summary(),
            "gpu_launches": launches,
        }
    for s in sessions.values():
        s.close()

    if rank == 0 and world == 1:
        if not args.skip_batched:
            line["batched"] = batched_leg(args, local)
        if not args.skip_e2e:
            line["e2e"] = e2e(args, A, M0, b)
        if not args.skip_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args, A, M0, b)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if group is not None:
        group.destroy_process_group()


KERNEL_NOTES = {
    "fused_residual": "fused_residual (FusedResidualKernel, one warp per column: R = I - A M, Z = Pr R written "
                      "with its transpose, ||R(:,j)||^2, then the MR projection of A Z from the Z column in "
                      "shared memory)",
    "fused_drop": "fused_drop (FusedDropKernel, one warp per column: 0.5 (U + U^T) with U = M + alpha Z formed "
                  "from M, Z and their transposes, threshold and top-k)",
    "spgemm_numeric": "spgemm_numeric (ColumnProductKernel: R = I - A M with Z and the column sums fused, and the "
                      "MR projection of A Z)",
}


def mixed_vs_fp64(sessions, results):
    """The error of the mixed-precision result against the FP64 one on the
    benched problem: M, the residual history, and PCG iterations to tolerance."""
    from scipy import sparse
    m_mixed = sparse.csc_matrix(sessions["mixed"].result().M)
    m_fp64 = sparse.csc_matrix(sessions["fp64"].result().M)
    h_mixed = sessions["mixed"].history()["residual_norm"]
    h_fp64 = sessions["fp64"].history()["residual_norm"]
    rows = min(len(h_mixed), len(h_fp64))
    diff = sparse.linalg.norm(m_mixed - m_fp64) / sparse.linalg.norm(m_fp64)
    return {
        "m_rel_frobenius": float(diff),
        "history_max_rel": float(np.max(np.abs(h_mixed[:rows] - h_fp64[:rows]) / h_fp64[:rows])),
        "final_residual_mixed": float(h_mixed[-1]), "final_residual_fp64": float(h_fp64[-1]),
        "nnz_mixed": int(m_mixed.nnz), "nnz_fp64": int(m_fp64.nnz),
        "pcg_iterations_mixed_m_fp32_apply": results["mixed"][-1]["pcg_iterations"],
        "pcg_iterations_fp64_m": results["fp64"][-1]["pcg_iterations"],
        "against": "the FP64 device run of the same build (itself bit-identical to the FP64 oracle)",
    }


def batched_leg(args, device):
    """Many small systems: `global_spai.mr_batched` (one block-diagonal batch,
    every launch over all systems) against one `global_spai.mr` call per
    system, both through the public API with host buffers (wall clock; host
    assembly, uploads and downloads included)."""
    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import global_spai, problems
    systems = problems.diffusion_batch(args.batch_count, seed=0)
    kw = dict(max_iterations=args.batch_iterations, tolerance=1e-12, max_density=1.0,
              topk_per_column=args.batch_topk, precision="mixed", device=device)
    global_spai.mr_batched(systems, **kw)  # warm-up
    times = []
    for _ in range(2):
        t0 = time.perf_counter()
        out = global_spai.mr_batched(systems, **kw)
        times.append(time.perf_counter() - t0)
    seconds = statistics.mean(times)
    iterations = sum(r.iterations for r in out)
    t0 = time.perf_counter()
    for A in systems:
        global_spai.mr(A, **kw)
    one_by_one = time.perf_counter() - t0
    return {
        "workload": f"{len(systems)} systems, n log-uniform in [1000, 64000], 2-D 5-pt / 3-D 7-pt, sigma 0.5, "
                    f"diagonal shift U(0, 0.1); Global MR {args.batch_iterations} it, top-{args.batch_topk}, mixed",
        "rows": int(sum(A.shape[0] for A in systems)),
        "nnz": int(sum(A.nnz for A in systems)),
        "seconds_per_batch": round(seconds, 4),
        "systems_per_s": round(len(systems) / seconds, 2),
        "spai_iters_per_s": round(iterations / seconds, 1),
        "one_call_per_system_seconds": round(one_by_one, 3),
        "speedup_vs_one_call_per_system": round(one_by_one / seconds, 2),
        "timing": "wall clock around the public API call, mean of 2 after 1 warm-up",
    }


def e2e(args, A, M0, b):
    """The same step through the public API with host buffers (pinned), copies included."""
    import torch
    from scipy import sparse
    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import backward_error, global_spai
    from parallellocallyoptimalapproximatesparsematrixinverses_b200.methods import as_csc

    def pinned(arr):
        t = torch.empty(arr.shape, dtype=getattr(torch, str(arr.dtype)), pin_memory=True)
        out = t.numpy()
        out[...] = arr
        return out, t

    keep = []
    A_csc = as_csc(A)
    M0_csc = as_csc(M0)
    for m in (A_csc, M0_csc):
        for attr in ("indptr", "indices", "data"):
            arr, t = pinned(getattr(m, attr))
            keep.append(t)
            setattr(m, attr, arr)
    A_csr = sparse.csr_matrix(A)
    A_csr.sort_indices()
    a_arrays = []
    for arr in (A_csr.data.astype(np.float64), A_csr.indices.astype(np.int64), A_csr.indptr.astype(np.int64)):
        p, t = pinned(arr)
        keep.append(t)
        a_arrays.append(p)
    b_pinned, t = pinned(np.ascontiguousarray(b))
    keep.append(t)
    n = A.shape[0]
    times_spai, times_pcg = [], []
    h2d = d2h = 0
    for rep in range(max(1, min(args.steps, 3)) + 1):
        t0 = time.perf_counter()
        r = global_spai.mr(A_csc, M0=M0_csc, max_iterations=args.spai_iterations, tolerance=1e-12,
                           max_density=float(args.topk) / n, precision="mixed", topk_per_column=args.topk)
        t1 = time.perf_counter()
        # M's CSC arrays read as CSR are M^T, whose symmetric part (M^T + M)/2 is the
        # preconditioner asked for: the same entries, the same bits, no host transpose
        M_csc = r.M
        hist, status = backward_error.pcg(a_arrays[0], a_arrays[1], a_arrays[2], M_csc.data, M_csc.indices,
                                          M_csc.indptr, b_pinned, args.pcg_max_iterations, 1, args.pcg_tolerance,
                                          refresh_period=args.pcg_refresh, m_precision="mixed", symmetric_part=True)
        t2 = time.perf_counter()
        if rep == 0:
            continue  # first call pays context creation
        times_spai.append(t1 - t0)
        times_pcg.append(t2 - t1)
        h2d = (A_csc.indptr.nbytes + A_csc.indices.nbytes + A_csc.data.nbytes + M0_csc.indptr.nbytes
               + M0_csc.indices.nbytes + M0_csc.data.nbytes + sum(x.nbytes for x in a_arrays)
               + M_csc.data.nbytes + 8 * M_csc.indices.size + 8 * M_csc.indptr.size + b_pinned.nbytes)
        d2h = (r.M.indptr.nbytes + r.M.indices.nbytes + r.M.data.nbytes + r.history.nbytes
               + 8 * args.pcg_max_iterations)
    spai_s = statistics.median(times_spai)
    pcg_s = statistics.median(times_pcg)
    return {"value": round(args.spai_iterations / spai_s, 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "spai_ms_per_build": round(spai_s * 1e3, 3),
            "pcg_ms_to_tolerance": round(pcg_s * 1e3, 3), "ms_per_step": round((spai_s + pcg_s) * 1e3, 3),
            "timing": "time.perf_counter around global_spai.mr and backward_error.pcg (host buffers, synchronous)",
            "api": "global_spai.mr(..., precision='mixed', topk_per_column=K) -> spai_run_ex; "
                   "backward_error.pcg(..., symmetric_part=True) -> spai_pcg"}


def cpu_build(args, A, M0, threads):
    """One full CPU SPAI build of the workload: the oracle port (FP64, the
    reference's summation order over `threads` column batches, OpenMP on
    `threads` host threads), all args.spai_iterations iterations, timed whole
    as the reference times a method call (scripts/methods_thread_speedup.py:34-45)."""
    from oracle import pyoracle
    n = A.shape[0]
    t0 = time.perf_counter()
    r = pyoracle.run("global_spai", "mr", A, M0=M0, max_iterations=args.spai_iterations, tolerance=1e-12,
                     max_density=float(args.topk) / n, num_threads=threads, omp_threads=threads,
                     topk_per_column=args.topk, order=pyoracle.ORDER_REFERENCE)
    return time.perf_counter() - t0, r


def cpu_pcg(args, A, M, b, threads):
    """PCG to args.pcg_tolerance with (M + M^T)/2 of the CPU-built M: the
    reference's own compiled backward_error.pcg when present, else the oracle port."""
    from scipy import sparse
    from oracle import pyoracle
    msym = sparse.csr_matrix((M + M.T) * 0.5)
    msym.sort_indices()
    A_csr = sparse.csr_matrix(A)
    A_csr.sort_indices()
    ref = pyoracle.reference_pcg_module()
    t0 = time.perf_counter()
    if ref is not None:
        hist, status = ref.pcg(A_csr.data, A_csr.indices.astype(np.int64), A_csr.indptr.astype(np.int64),
                               msym.data, msym.indices.astype(np.int64), msym.indptr.astype(np.int64), b,
                               args.pcg_max_iterations, threads, args.pcg_tolerance)
        kind = "reference (methods_cython/backward_error.pyx compiled from the reference source)"
    else:
        hist, status = pyoracle.pcg(A_csr, msym, b, args.pcg_max_iterations, args.pcg_tolerance)
        kind = "port"
    return time.perf_counter() - t0, hist, int(status), kind


def cpu_baseline(args, A, M0, b, threads=None):
    """The CPU path on the host cores: one whole SPAI build (no extrapolation)
    and PCG on its M, at all host threads, plus the same PCG on one thread."""
    threads = threads or os.cpu_count() or 1
    build_s, r = cpu_build(args, A, M0, threads)
    pcg_s, hist, status, kind = cpu_pcg(args, A, r.M, b, threads)
    pcg_1_s, _, _, _ = cpu_pcg(args, A, r.M, b, 1)
    return {"value": round(r.iterations / build_s, 4), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"one whole {r.iterations}-iteration Global MR build of the same operator (top-"
                      f"{args.topk}), FP64 CPU oracle port, {threads} OpenMP threads over {threads} column batches, "
                      f"timed whole; then PCG on its M",
            "spai_seconds_per_build": round(build_s, 3),
            "pcg_ms_to_tolerance": round(pcg_s * 1e3, 3), "pcg_ms_to_tolerance_1_thread": round(pcg_1_s * 1e3, 3),
            "pcg_iterations": len(hist) - 1, "pcg_status": status, "pcg_kind": kind,
            "pcg_note": "preconditioner = (M+M^T)/2 of the CPU-built M"}


REFERENCE_MAX_STEPS = 3
REFERENCE_MAX_WARMUP = 1


def run_reference(args):
    """--impl reference: the reference's CPU implementation of the path on the
    host cores -- the oracle port for SPAI (the reference's own SPAI needs
    Eigen, absent here), the reference's compiled PCG -- each step one whole
    build plus PCG, at all host threads.  A step takes about 15 s at 64^3, so at
    most REFERENCE_MAX_STEPS timed steps after REFERENCE_MAX_WARMUP warm-up
    steps run; the line's `steps` and `warmup` are the counts that ran."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    A, M0, b = workload(args)
    threads = os.cpu_count() or 1
    steps = max(1, min(args.steps, REFERENCE_MAX_STEPS))
    warmup = min(args.warmup, REFERENCE_MAX_WARMUP)
    for _ in range(warmup):
        cpu_build(args, A, M0, threads)
    builds, pcgs, its = [], [], 0
    pcg_info = None
    for _ in range(steps):
        build_s, r = cpu_build(args, A, M0, threads)
        pcg_s, hist, status, kind = cpu_pcg(args, A, r.M, b, threads)
        builds.append(build_s)
        pcgs.append(pcg_s)
        its += r.iterations
        pcg_info = (len(hist) - 1, status, kind)
    value = its / sum(builds)
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": warmup, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": round(1e3 * (sum(builds) + sum(pcgs)) / steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded 64^3 log-normal diffusion operator; no public data set)",
        "config": config_dict(args, A), "impl": "reference",
        "spai_seconds_per_build": round(sum(builds) / steps, 3),
        "pcg_ms_to_tolerance": round(1e3 * sum(pcgs) / steps, 3),
        "pcg_iterations": pcg_info[0], "pcg_status": pcg_info[1],
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{steps} whole {args.spai_iterations}-iteration Global MR builds (FP64 oracle "
                                   f"port, the reference's summation order, {threads} OpenMP threads), each followed "
                                   f"by PCG on its M",
                         "pcg_kind": pcg_info[2]},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
