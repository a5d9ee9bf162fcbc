#!/usr/bin/env python
"""Benchmark of the dense LU solve path (dgesv) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--n 16384] [--nrhs 1]
    python bench.py --impl reference ...      # the reference's CPU path

Workload (one step = one dgesv of the whole system): n x n A with entries
iid Uniform(-1,1) drawn from the reference's DLARNV stream (seed
[1988,1989,1990,1991], no diagonal shift, cond ~ n), x_true continuing the
stream, b = A x_true; column-major float64 in HBM. The inputs (8 n^2 bytes)
are larger than L2, so no flush is needed between steps.

Forms timed (each reports GFLOP/s on the FP64-equivalent count
2/3 n^3 + 2 n^2 nrhs, the normwise backward error
||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) and the forward error
against x_true):
  fp64_exact   trailing updates with the reference's rounding (bit-identical LU)
  fp64_fma     trailing updates with fused multiply-adds
  mixed_*      low-precision LU + FP64 iterative refinement (when built)
The headline `value` is the fastest form whose backward error is within
10 n 2^-53 (the FP64 level).

Multi-GPU (torchrun): replicas — every rank solves its own system (seed
word 4 = 1991 + 2 rank); value = all ranks' flops / max-over-ranks time.
"""

from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "dgesv GFLOP/s, FP64 vs mixed-precision+IR at equal backward error; p99 latency"
SEEDY = [1988, 1989, 1990, 1991]
# DRAM bytes per algorithmic flop of the CUDA-core trailing-update kernel, per
# form, from ncu captures of its largest launch at n = 4096 (profiles/); a
# form without a capture reports traffic null.
GEMM_TRAFFIC_PER_FLOP = {}


def flops_dgesv(n: int, nrhs: int) -> float:
    return 2.0 / 3.0 * n**3 - 0.5 * n**2 - n / 6.0 + 2.0 * n * n * nrhs


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--n", type=int, default=16384)
    ap.add_argument("--nrhs", type=int, default=1)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--forms", default="")
    ap.add_argument("--cpu-n", type=int, default=1024, help="order of the CPU-baseline sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


# --------------------------------------------------------------------------- dist
def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while a region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_id()}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def gpu_id(self):
        try:
            import torch

            u = str(torch.cuda.get_device_properties(self.index).uuid)
            return u if u.startswith("GPU-") else "GPU-" + u
        except Exception:  # noqa: BLE001
            return str(self.index)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------- forms
def form_registry():
    """name -> (needs_restore, solve(ctx, A, b, n, nrhs) -> None)."""
    from algebra_linear_b200 import _lib

    forms = {
        "fp64_exact": (True, lambda ctx, A, b, n, nrhs: ctx.dgesv(A, b, n, nrhs, update=_lib.UPDATE_EXACT)),
        "fp64_fma": (True, lambda ctx, A, b, n, nrhs: ctx.dgesv(A, b, n, nrhs, update=_lib.UPDATE_FMA)),
    }
    try:
        from algebra_linear_b200 import mixed  # noqa: F401

        for prec in ("tf32", "bf16"):
            forms[f"mixed_{prec}"] = (False, (lambda p: lambda ctx, A, b, n, nrhs: mixed.dgesv_mixed_dev(
                ctx, A, b, n, nrhs, precision=p))(prec))
    except ImportError:
        pass
    return forms


def backward_error(A0, x, b0, n, nrhs):
    import torch

    Am = A0.view(n, n).t()  # column-major storage seen as A
    X = x.view(nrhs, n).t()
    B = b0.view(nrhs, n).t()
    r = B - Am @ X
    anorm = Am.abs().sum(dim=1).max()
    num = r.abs().amax(dim=0)
    den = anorm * X.abs().amax(dim=0) + B.abs().amax(dim=0)
    return float((num / den).max())


def run_form(name, spec, ctx, A0, b0, xt, n, nrhs, steps, warmup, pg, sample_clocks, dev_index):
    import torch

    from algebra_linear_b200 import _lib

    lib = _lib.load()
    needs_restore, solve = spec
    A = A0.clone() if needs_restore else A0
    b = b0.clone()
    for _ in range(warmup):
        if needs_restore:
            A.copy_(A0)
        b.copy_(b0)
        solve(ctx, A, b, n, nrhs)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    ctx.set_profiling(True)
    ctx.profile_reset()
    launches0 = lib.alg_kernel_launch_count()
    sampler = ClockSampler(dev_index) if sample_clocks else None
    if sampler:
        sampler.__enter__()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        if needs_restore:
            A.copy_(A0)
        b.copy_(b0)
        solve(ctx, A, b, n, nrhs)
    e1.record()
    torch.cuda.synchronize()
    if sampler:
        sampler.__exit__()
    ms = e0.elapsed_time(e1)
    launches = lib.alg_kernel_launch_count() - launches0
    prof = ctx.profile()
    ctx.set_profiling(False)
    if pg:
        t = torch.tensor([ms], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
        pg.barrier()
    eta = backward_error(A0, b, b0, n, nrhs)
    fwd = float((b - xt).abs().max() / xt.abs().max())
    return {
        "ms_per_step": ms / steps,
        "gflops": flops_dgesv(n, nrhs) / (ms / steps) / 1e6,
        "backward_error": eta,
        "forward_error": fwd,
        "gpu_launches": int(launches),
        "profile": prof,
        "clocks": sampler.summary() if sampler else None,
    }


def gemm_peaks_tflops():
    """cuBLAS GEMM throughput at 8192^3 (torch.matmul), best of 4, measured in
    this run: the ceilings of the update kernels — "f64" (DGEMM) for the FP64
    forms, "f32" (SGEMM on CUDA cores, TF32 off) for the FP32 LU of the mixed
    form, "tf32" for its tensor-core TF32 LU."""
    import torch

    out = {}
    saved = torch.backends.cuda.matmul.allow_tf32
    for key, dt, tf32 in (("f64", torch.float64, False), ("f32", torch.float32, False),
                          ("tf32", torch.float32, True)):
        torch.backends.cuda.matmul.allow_tf32 = tf32
        a = torch.rand(8192, 8192, dtype=dt, device="cuda")
        b = torch.rand(8192, 8192, dtype=dt, device="cuda")
        best = 1e9
        for _ in range(4):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        out[key] = 2 * 8192**3 / best / 1e9
    torch.backends.cuda.matmul.allow_tf32 = saved
    return out


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except ValueError:
            pass
    return {}


def roofline(res, form, peaks, gemm_peaks):
    prof = res["profile"]
    if not prof:
        return None
    cls, rec = max(prof.items(), key=lambda kv: kv[1]["ms"])
    per_launch_ms = rec["ms"] / max(rec["launches"], 1)
    if cls in ("gemm", "gemm_tc", "panel", "trsm"):
        achieved = rec["flops"] / rec["ms"] / 1e9  # TFLOP/s
        if cls == "gemm_tc" and form == "mixed_bf16":
            peak = peaks.get("bf16_tflops")
            src = "MEASURED_PEAKS.json bf16_tflops (measured)" if peak else "fallback 1590"
            peak = peak or 1590.0
        elif cls == "gemm_tc":
            peak, src = gemm_peaks["tf32"], "cuBLAS TF32 GEMM measured in this run"
        elif form.startswith("fp64"):
            peak, src = gemm_peaks["f64"], "cuBLAS DGEMM measured in this run"
        else:
            peak, src = gemm_peaks["f32"], "cuBLAS SGEMM (CUDA cores, TF32 off) measured in this run"
        traffic = None
        if cls == "gemm" and GEMM_TRAFFIC_PER_FLOP.get(form) is not None:
            traffic = GEMM_TRAFFIC_PER_FLOP[form] * rec["flops"] / max(rec["launches"], 1)
        return {"kernel": cls, "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": src,
                "launches": rec["launches"], "avg_launch_ms": per_launch_ms, "share_of_step":
                rec["ms"] / sum(v["ms"] for v in prof.values())}
    achieved = rec["bytes"] / rec["ms"] / 1e6  # GB/s
    peak = peaks.get("hbm_gbs", 6650.0)
    return {"kernel": cls, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": None, "launches": rec["launches"],
            "avg_launch_ms": per_launch_ms}


def e2e_run(form, A0, b0, n, nrhs, steps):
    import numpy as np
    import torch

    from algebra_linear_b200 import _lib

    lib = _lib.load()
    hA0 = A0.cpu().pin_memory()
    hb0 = b0.cpu().pin_memory()
    hA = torch.empty_like(hA0).pin_memory()
    hb = torch.empty_like(hb0).pin_memory()
    times = []
    for it in range(steps + 1):
        hA.copy_(hA0)
        hb.copy_(hb0)
        t0 = time.perf_counter()
        if form.startswith("mixed"):
            from algebra_linear_b200 import mixed

            rc = mixed.dgesv_mixed_host(hA.data_ptr(), hb.data_ptr(), n, nrhs, precision=form.split("_")[1])
        else:
            upd = _lib.UPDATE_EXACT if form == "fp64_exact" else _lib.UPDATE_FMA
            rc = lib.alg_dgesv_ex(upd, hA.data_ptr(), hb.data_ptr(), n, nrhs, None)
        dt = time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError(f"e2e solve failed: {_lib.status_string(rc)}")
        if it > 0:
            times.append(dt)
    t = statistics.median(times)
    h2d = 8 * n * n + 8 * n * nrhs
    d2h = 8 * n * nrhs + (0 if form.startswith("mixed") else 8 * n * n)
    return {"value": flops_dgesv(n, nrhs) / t / 1e9, "unit": "GFLOP/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": 1e3 * t, "form": form, "steps": steps,
            "api": "alg_dgesv_ex" if not form.startswith("mixed") else "alg_dgesv_mixed"}


def cpu_baseline(n_cpu: int, reps: int = 3):
    """The oracle (C++ restatement of lapack::dgesv, mod.rs:309-354) on one
    host core, dgesv at order n_cpu, median of reps."""
    from oracle import dense as oracle

    a, _, b = oracle.c1_system(n_cpu)
    ts = []
    for _ in range(reps):
        aw, bw = a.copy(), b.copy()
        t0 = time.perf_counter()
        rc, _ = oracle.dgesv(aw, bw, n_cpu)
        ts.append(time.perf_counter() - t0)
        assert rc == 0
    t = statistics.median(ts)
    return {"value": flops_dgesv(n_cpu, 1) / t / 1e9, "unit": "GFLOP/s", "cores": 1, "kind": "port",
            "sample": f"dgesv n={n_cpu}, 1 RHS, same larnv workload, median of {reps} "
                      f"({t:.2f} s each); the reference path is single-threaded"}


# --------------------------------------------------------------------------- arms
def run_reference(args, world, rank, pg):
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from oracle import dense as oracle

    n_cpu = args.cpu_n
    a, _, b = oracle.c1_system(n_cpu)
    for _ in range(args.warmup):
        oracle.dgesv(a.copy(), b.copy(), n_cpu)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.dgesv(a.copy(), b.copy(), n_cpu)
    dt = (time.perf_counter() - t0) / args.steps
    v = flops_dgesv(n_cpu, 1) / dt / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (larnv Symmetric, seed "
        f"{SEEDY})",
        "config": {"workload": f"dense dgesv, A iid U(-1,1), 1 RHS; reference CPU path sampled at n={n_cpu}",
                   "n": n_cpu, "nrhs": 1, "parallelism": "1 host core"},
        "cpu_baseline": {"value": v, "unit": "GFLOP/s", "cores": 1, "kind": "port",
                         "sample": f"one dgesv of order {n_cpu} per step (the reference is single-threaded; "
                                   "its Rust crate cannot be built here, so the oracle's C++ restatement runs)"},
        "e2e": {"value": v, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local, pg):
    import torch

    from algebra_linear_b200 import device

    torch.cuda.set_device(local)
    n, nrhs = args.n, args.nrhs
    seed = [SEEDY[0], SEEDY[1], SEEDY[2], SEEDY[3] + 2 * rank]
    peaks = measured_peaks()
    gemm_peaks = gemm_peaks_tflops()
    ctx = device.Context()
    A0, s1 = ctx.larnv(2, seed, n * n)
    xt, _ = ctx.larnv(2, s1, n * nrhs)
    b0 = (A0.view(n, n).t() @ xt.view(nrhs, n).t()).t().contiguous().view(-1)
    torch.cuda.synchronize()

    reg = form_registry()
    # default forms: the FP64 pair and the mixed forms whose LU is a strong
    # enough preconditioner at this order (BF16 falls back to FP64 past n ~ 4096)
    default = [f for f in reg if f != "mixed_bf16" or n <= 4096]
    names = [f for f in (args.forms.split(",") if args.forms else default) if f in reg]
    results = {}
    for name in names:
        results[name] = run_form(name, reg[name], ctx, A0, b0, xt, n, nrhs, args.steps, args.warmup, pg,
                                 sample_clocks=True, dev_index=local)
    tol = 10 * n * 2.0**-53
    ok = {k: v for k, v in results.items() if v["backward_error"] <= tol}
    head = max(ok or results, key=lambda k: (ok or results)[k]["gflops"])
    hr = results[head]
    value = hr["gflops"] * world
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "GFLOP/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": hr["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if head.startswith("fp64") else "f32/" + head.split("_")[1] + "+f64",
        "data": f"synthetic: larnv Symmetric U(-1,1) stream, seed {seed} (rank r: word 4 = 1991+2r)",
        "config": {"workload": f"dense dgesv n={n}, {nrhs} RHS, A iid U(-1,1) no shift, b = A x_true",
                   "n": n, "nrhs": nrhs, "form": head, "parallelism": f"replicas x{world}",
                   "l2": "inputs (8 n^2 B) larger than L2; no flush"},
        "forms": {k: {**{kk: vv for kk, vv in v.items() if kk != "profile"},
                      "kernel_ms_per_step": {c: r["ms"] / args.steps for c, r in (v["profile"] or {}).items()}}
                  for k, v in results.items()},
        "backward_error_bound": tol,
        "gpu_launches": hr["gpu_launches"],
        "clocks": hr["clocks"],
        "roofline": roofline(hr, head, peaks, gemm_peaks),
        "cublas_gemm_peaks_tflops": gemm_peaks,
    }
    if not args.no_e2e:
        line["e2e"] = e2e_run(head, A0, b0, n, nrhs, steps=max(2, min(args.steps, 3)))
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(args.cpu_n)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()


def main():
    args = parse_args()
    world, rank, local, pg = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank, pg)
        else:
            run_ours(args, world, rank, local, pg)
    finally:
        if pg:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
