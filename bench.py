"""Benchmark: field values/s of the spectral-sum generator on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one full generation request):
  Shinozuka-Deodatis method 2 on a 128^3 structured grid, spacing 0.05,
  corrL = (2, 1, 0.5), gaussian marginal, Nmc = 64, 24^3 wavenumbers x 4 sign
  quadrants (K = 55,296), seed_start = rank; BF16 trig tiles with hi/lo BF16
  amplitude side on tcgen05, FP32 accumulation, FP64 phase reduction.
  n * Nmc = 134,217,728 field values per step.  Synthetic inputs (the
  reference publishes no dataset).

value   device-resident points and result (rf_generate_device), CUDA events on
        the launching stream, L2 flushed (256 MiB write) between timed steps;
e2e     the flat C-ABI call rf_create_standard_gaussian_field_unstruct with
        pinned host buffers: host->device copy of the points and device->host
        copy of the whole FP64 result inside the timed region.
N > 1   one process per GPU, independent replicas (weak scaling, no
        collective on the data path); time = max over ranks.
--impl reference   times the reference CPU algorithm (the FP64 restatement of
        gen_Std_Gauss_Shinozuka's slab / Netlib DGEMM / cos / GEMV loop) on the
        host cores, on a bounded row sample of the same workload per step.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GRID_N, SPACING, NMC, KN = 128, 0.05, 64, 24
GRID = (GRID_N, GRID_N, GRID_N)
CORRL = (2.0, 1.0, 0.5)
WORKLOAD = "shinozuka-3d-grid128^3-h0.05-corrL(2,1,0.5)-Nmc64-K24^3x4"
FLUSH_BYTES = 256 << 20


def grid_points():
    ax = [np.arange(g, dtype=np.float64) * SPACING for g in GRID]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")  # axis 1 fastest (setGrid)
    return np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)  # n x 3 == Fortran 3 x n


def extent():
    return tuple((g - 1) * SPACING for g in GRID)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return j, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_bench_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": ["no samples"]}
        load = [s for s in sm if s > 0.5 * (mx or max(sm))] or sm
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_rate(x, rows, nr, nthreads=0):
    """Reference CPU algorithm on `rows` points x `nr` realizations, full K."""
    from oracle import oracle as O

    rq = O.OracleRequest(x, Nmc=NMC, kNStep=(KN, KN, KN), corrL=CORRL, xRange=extent())
    row0 = (x.shape[0] // 2) - rows // 2
    _, t = rq.baseline(row0, rows, 0, nr, nthreads=nthreads)
    return rows * nr / t, t


def cpu_sample(x, target_s, nthreads):
    """Grow the row sample until one run takes about target_s seconds."""
    rows = 16
    rate, t = cpu_rate(x, rows, 1, nthreads)
    rows = max(16, min(x.shape[0], int(rows * target_s / max(t, 1e-3))))
    rate, t = cpu_rate(x, rows, 1, nthreads)
    return rate, rows, t


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import oracle as O

    O.lib()
    x = grid_points()
    cores = os.cpu_count() or 1
    rate, rows, t = cpu_sample(x, 2.0, cores)
    for _ in range(args.warmup):
        cpu_rate(x, rows, 1, cores)
    times = []
    for _ in range(args.steps):
        r, t = cpu_rate(x, rows, 1, cores)
        times.append(t)
    total = sum(times)
    value = rows * args.steps / total
    line = {
        "impl": "reference", "metric": "field values/s", "value": value, "unit": "field values/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": f"{rows} points x 1 realization per step, full K = 55296"},
        "cpu_baseline": {"value": value, "unit": "field values/s", "cores": cores, "kind": "port",
                         "sample": f"{rows} points x 1 realization, full K, per step"},
        "e2e": {"value": value, "unit": "field values/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def end_to_end(args, rf, torch, dist, xh, n, opts, world, local):
    """The flat C-ABI call with pinned host buffers: H2D of the points and
    D2H of the whole FP64 field inside the timed region."""
    values = n * NMC
    xpin = torch.from_numpy(np.ascontiguousarray(xh)).pin_memory()
    opin = torch.empty((NMC, n), dtype=torch.float64).pin_memory()
    xa = xpin.numpy().T  # 3 x n view, Fortran order
    oa = opin.numpy().T  # n x Nmc view, Fortran order
    e2e_steps = max(3, args.steps // 2)
    for _ in range(2):
        rf.create_standard_gaussian_field_unstruct(xa, 1, 1, CORRL, 0.0, 1.0, NMC, 2, randField=oa, **opts)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        rf.create_standard_gaussian_field_unstruct(xa, 1, 1, CORRL, 0.0, 1.0, NMC, 2, randField=oa, **opts)
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": world * values * e2e_steps / e2e_s, "unit": "field values/s",
           "h2d_bytes_per_step": int(xh.nbytes), "d2h_bytes_per_step": int(n * NMC * 8),
           "api": "rf_create_standard_gaussian_field_unstruct (host buffers, pinned)"}
    return e2e


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="bf16", choices=["bf16", "fp16", "bf16_fast", "fp32"])
    ap.add_argument("--no-forms", action="store_true", help="skip the other precision forms")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end timing")
    ap.add_argument("--grid", default="128,128,128",
                    help="grid points per axis; a smaller grid (e.g. 32,32,18 = one wave of 144 tiles) "
                         "keeps profiler captures short; the headline workload is 128,128,128")
    args = ap.parse_args()
    global GRID
    GRID = tuple(int(v) for v in args.grid.split(","))

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist

    import randomfield_b200 as rf

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    xh = grid_points()
    n = xh.shape[0]
    opts = dict(precision=args.precision, k_nstep=(KN, KN, KN), seed_start=rank, x_range=extent(), device=local)
    ctx = rf.Context(local)
    ctx.set_timing(True)
    stream = torch.cuda.Stream(device=local)
    dx = torch.from_numpy(np.ascontiguousarray(xh)).cuda(local)
    dout = torch.empty((NMC, n), dtype=torch.float64, device=f"cuda:{local}")
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")

    def step(prec=None):
        o = dict(opts)
        if prec:
            o["precision"] = prec
        ctx.generate(dx, 3, n, 1, 1, CORRL, 0.0, 1.0, NMC, 2, dout, stream=stream.cuda_stream, **o)

    def timed(nsteps, nwarm, prec=None):
        with torch.cuda.stream(stream):
            for _ in range(nwarm):
                step(prec)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nsteps)]
        kern_ms, launches = [], 0
        with torch.cuda.stream(stream):
            for a, b in ev:
                flush.zero_()  # L2 flush outside the timed events
                a.record(stream)
                step(prec)
                b.record(stream)
                t_tab, t_con, t_post, nl = ctx.last_times()
                kern_ms.append(t_con)
                launches += nl
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        total = sum(a.elapsed_time(b) for a, b in ev)
        return total, float(np.mean(kern_ms)), launches

    clk = Clocks(local)
    with clk:
        total_ms, kern_ms, launches = timed(args.steps, args.warmup)
    if world > 1:
        t = torch.tensor([total_ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    values = n * NMC
    value = world * values * args.steps / (total_ms / 1e3)

    # accuracy of the timed form on a row sample (oracle, FP64)
    from oracle import oracle as O

    acc = None
    if rank == 0:
        rows = np.random.RandomState(7).choice(n, 48, replace=False)
        rq = O.OracleRequest(xh, Nmc=NMC, kNStep=(KN, KN, KN), corrL=CORRL, seedStart=rank, xRange=extent())
        ref = rq.generate(rows=rows)
        got = dout.cpu().numpy()[:, rows]
        d = got - ref
        acc = {"rel_l2": float(np.linalg.norm(d) / np.linalg.norm(ref)),
               "max_abs_over_std": float(np.abs(d).max() / ref.std()),
               "worst_realization_rel_l2": float(max(np.linalg.norm(d[r]) / np.linalg.norm(ref[r])
                                                     for r in range(NMC))),
               "sample": "48 random points x 64 realizations vs the FP64 oracle"}

    # other precision forms, same workload (fewer steps)
    forms = {}
    if not args.no_forms:
        for prec in ("fp16", "bf16_fast", "fp32"):
            if prec == args.precision:
                continue
            ns = 2 if prec == "fp32" else max(3, args.steps // 2)
            tot, km, _ = timed(ns, 1, prec)
            forms[prec] = {"value": world * values * ns / (tot / 1e3), "unit": "field values/s",
                           "ms_per_step": tot / ns, "contract_ms": km}
        if "fp32" in forms:
            forms["bf16_over_fp32_plain"] = value / forms["fp32"]["value"]

    # end to end through the flat C-ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        e2e = end_to_end(args, rf, torch, dist, xh, n, opts, world, local)

    pk, src = peaks()
    pk, src = peaks()
    K = 4 * KN ** 3
    flops = 2.0 * n * (2 * K) * NMC  # algorithmic: the hi/lo split's second MMA is not credited
    tflops = flops / (kern_ms / 1e3) / 1e12
    peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp) and GRID == (128, 128, 128):
        with open(tp) as f:
            traffic = json.load(f).get(args.precision)
    roof = {"bound": "tensor", "achieved": tflops, "peak": peak, "unit": "TFLOP/s", "frac": tflops / peak,
            "traffic": traffic, "kernel": "rf_tc_kernel (tcgen05 contraction + fused epilogue)",
            "kernel_ms": kern_ms, "peak_source": f"bf16_tflops_sustained, {src}",
            "algorithmic_flops_per_launch": flops}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = os.cpu_count() or 1
        rate, rows_s, t = cpu_sample(xh, 3.0, cores)
        cpu = {"value": rate, "unit": "field values/s", "cores": cores, "kind": "port",
               "sample": f"{rows_s} points x 1 realization, full K = {K}, reference slab/DGEMM/cos/GEMV loop"}

    if world > 1:
        dist.barrier()
    ctx.close()
    if rank == 0:
        line = {
            "metric": "field values/s", "value": value, "unit": "field values/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"bf16": "bf16", "fp16": "f16", "bf16_fast": "bf16", "fp32": "f32"}[args.precision],
            "data": "synthetic",
            "config": {"workload": WORKLOAD if GRID == (128, 128, 128) else f"{WORKLOAD} on a {GRID} grid", "n_points": n, "Nmc": NMC, "K": K, "precision": args.precision,
                       "l2": "flushed between timed steps (256 MiB write); output 1 GiB per step",
                       "parallelism": f"replicas x{world}"},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "accuracy": acc,
            "forms": forms,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
