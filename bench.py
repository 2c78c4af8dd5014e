"""Benchmark: field values/s of the spectral-sum generator on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one full generation request):
  Shinozuka-Deodatis method 2 on a 128^3 structured grid, spacing 0.05,
  corrL = (2, 1, 0.5), gaussian marginal, Nmc = 64, 24^3 wavenumbers x 4 sign
  quadrants (K = 55,296), seed_start = rank; the outer-group contraction on
  CTA pairs: BF16 operands, TF32 on the K-steps that carry 75 % of the field
  variance, tcgen05 with FP32 accumulation, FP64 phase reduction.
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
import tempfile
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
        fd, self.path = tempfile.mkstemp(prefix="rf_bench_clocks_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        try:
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
        try:
            return self._summary()
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass

    def _summary(self):
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


def field_accuracy(O, dout, seed):
    """Relative-L2 and max-abs errors of the whole device field against the
    oracle's FP64 whole-grid reference (O.separable_field), overall and per
    realization."""
    ref = O.separable_field((0.0, 0.0, 0.0), (SPACING,) * 3, GRID, CORRL, NMC, kNStep=(KN, KN, KN), seedStart=seed)
    got = dout.cpu().numpy()
    per = np.empty(NMC)
    dmax, dsq, rsq = 0.0, 0.0, 0.0
    for r in range(NMC):
        d = got[r] - ref[r]
        e, q = float(np.dot(d, d)), float(np.dot(ref[r], ref[r]))
        per[r] = np.sqrt(e / q)
        dsq += e
        rsq += q
        dmax = max(dmax, float(np.abs(d).max()))
    return {"rel_l2": float(np.sqrt(dsq / rsq)), "max_abs_over_std": dmax / float(np.sqrt(rsq / ref.size)),
            "worst_realization_rel_l2": float(per.max()), "median_realization_rel_l2": float(np.median(per)),
            "sample": f"the whole field: {ref.shape[1]} points x {NMC} realizations vs the FP64 oracle "
                      "(whole-grid reference from the oracle's wavevectors and phases)"}


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


# ----------------------------------------------------------------- batched / serving
BATCH_REQUESTS = 512
SERVE_RATE = 200.0


def draw_request(rs, large_frac=0.0):
    """One request of the batched mix: n log-uniform in [1e3, 1e6] points
    uniform in a box of side U[1, 20], Nmc U{1..128}, method 1 or 2 (p = .5),
    corrL per axis U[0.5, 4], gaussian or lognormal marginal (p = .5).  The
    wavevector count is fixed per method: Shinozuka 24^3 x 4, isotropic
    64 radii x 64 directions (the reference rule would give up to ~6e5
    wavevectors at side 20 and corrL 0.5).  With probability large_frac the
    request is a 256^3 structured grid (spacing 0.05) with Nmc = 16, generated
    as the localization blend of 8 subdomains."""
    method = 1 if rs.uniform() < 0.5 else 2
    marg = "lognormal" if rs.uniform() < 0.5 else "gaussian"
    corrL = tuple(float(v) for v in rs.uniform(0.5, 4.0, 3))
    if large_frac and rs.uniform() < large_frac:
        # 256^3 grid, spacing 0.05, blended from 2 x 2 x 2 subdomains of 134^3
        # sharing 12 points (overlap 0.65 corrL, about 10% of a subdomain)
        pts, Nmc, kind, corrL = None, 16, "grid256", (1.0, 1.0, 1.0)
    else:
        n = int(np.exp(rs.uniform(np.log(1e3), np.log(1e6))))
        side = rs.uniform(1.0, 20.0)
        pts = rs.uniform(0.0, side, size=(n, 3)).astype(np.float32).astype(np.float64)
        Nmc, kind = int(rs.randint(1, 129)), "box"
    opts = dict(k_nstep=(KN, KN, KN)) if method == 2 else dict(iso_n_radial=64, iso_n_dir=64)
    avg, var = (1.0, 0.25) if marg == "lognormal" else (0.0, 1.0)
    return dict(points=pts, Nmc=Nmc, method=method, marg=marg, corrL=corrL, avg=avg, var=var, opts=opts, kind=kind)


def bench_configs(args, rf, torch, local, sfu_rate, peak_tflops):
    """The other single-request configs, device-resident, each timed with
    CUDA events over a few calls: config 1 (Shinozuka 32^3, spacing 0.1,
    Nmc 4, 16^3 x 4 wavevectors) and config 2 (isotropic, 200k points uniform
    in [0, 10]^3, lognormal avg 1 var 0.25, Nmc 64, 64 x 64 wavevectors),
    in the BF16 form and the plain FP32 form.  Config 2 runs GEN_TABLE, whose
    bound is the SFU: one (sin, cos) pair per point and wavevector."""
    out = {}
    rs = np.random.RandomState(12)
    ax = np.arange(32, dtype=np.float64) * 0.1
    z, y, x = np.meshgrid(ax, ax, ax, indexing="ij")
    c1 = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    c2 = rs.uniform(0.0, 10.0, size=(200000, 3)).astype(np.float32).astype(np.float64)
    cases = {
        "cfg1_shinozuka_32cubed": (c1, 4, 2, "gaussian", 0.0, 1.0, dict(k_nstep=(16, 16, 16))),
        "cfg2_isotropic_200k": (c2, 64, 1, "lognormal", 1.0, 0.25, dict(iso_n_radial=64, iso_n_dir=64)),
    }
    ctx = rf.Context(local)
    ctx.set_timing(True)
    for name, (pts, Nmc, method, marg, avg, var, o) in cases.items():
        n = pts.shape[0]
        dx = torch.from_numpy(np.ascontiguousarray(pts)).cuda(local)
        dout = torch.empty((Nmc, n), dtype=torch.float64, device=f"cuda:{local}")
        res = {"n_points": n, "Nmc": Nmc}
        for prec in ("bf16", "fp32"):
            def call():
                ctx.generate(dx, 3, n, 1, marg, (1.0, 1.0, 1.0), avg, var, Nmc, method, dout, precision=prec, **o)
            for _ in range(2):
                call()
            ctx.synchronize()
            reps = 5 if prec == "bf16" else 2
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            kms = []
            a.record()
            for _ in range(reps):
                call()
                kms.append(ctx.last_times()[1])
            b.record()
            torch.cuda.synchronize()
            ms = a.elapsed_time(b) / reps
            res[prec] = {"value": n * Nmc / (ms / 1e3), "unit": "field values/s", "ms_per_call": ms,
                         "contract_ms": float(np.mean(kms))}
        K = 4 * 16 ** 3 if method == 2 else 64 * 64
        flops = 2.0 * n * 2 * K * Nmc
        res["bounds_ms"] = {"tensor": flops / (peak_tflops * 1e12) * 1e3,
                            "sfu": (n * K if method == 1 else n * 48) / sfu_rate * 1e3}
        res["bf16_over_fp32_plain"] = res["bf16"]["value"] / res["fp32"]["value"]
        out[name] = res
        del dx, dout
    ctx.close()
    return out


def bench_grid(args, rf, torch, local):
    """The headline workload through rf_generate_grid: the same Shinozuka
    field on the same 128^3 grid (same wavevectors, phases and marginal),
    evaluated axis by axis in FP64 because both the points and the
    wavevectors are tensor grids.  Device time with CUDA events (L2 flushed
    between calls), the FP64 multiply-adds of the three axis stages against
    the nominal FP64 rate (64 FMA per clock per SM at the maximum SM clock),
    accuracy on the oracle's 48-point sample, and an end-to-end time that
    includes the copy of the whole field into pinned host memory."""
    n = int(np.prod(GRID))
    ctx = rf.Context(local)
    ctx.set_timing(True)
    stream = torch.cuda.Stream(device=local)
    dout = torch.empty((NMC, n), dtype=torch.float64, device=f"cuda:{local}")
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")
    o = dict(k_nstep=(KN, KN, KN), seed_start=0, device=local)

    def call():
        ctx.generate_grid(dout, (0.0, 0.0, 0.0), (SPACING,) * 3, GRID, 1, 1, CORRL, 0.0, 1.0, NMC,
                          stream=stream.cuda_stream, **o)

    with torch.cuda.stream(stream):
        for _ in range(3):
            call()
    torch.cuda.synchronize()
    steps = max(5, args.steps)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    kms, launches = [], 0
    with torch.cuda.stream(stream):
        for a, b in ev:
            flush.zero_()
            a.record(stream)
            call()
            b.record(stream)
            t_tab, t_axes, _, nl = ctx.last_times()
            kms.append((t_tab, t_axes))
            launches += nl
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev) / steps
    n1 = n2 = n3 = KN
    N1, N2, N3 = GRID
    fma = NMC * (8.0 * n1 * n2 * n3 * N3 + 4.0 * n1 * n2 * N2 * N3 + 2.0 * n1 * N1 * N2 * N3)
    props = torch.cuda.get_device_properties(local)
    peak = 2.0 * 64 * props.multi_processor_count * 1.965e9 / 1e12
    axes_ms = float(np.mean([k[1] for k in kms]))
    from oracle import oracle as O

    rows = np.random.RandomState(7).choice(n, 48, replace=False)
    rq = O.OracleRequest(grid_points(), Nmc=NMC, kNStep=(KN, KN, KN), corrL=CORRL, seedStart=0)
    ref = rq.generate(rows=rows)
    got = dout.cpu().numpy()[:, rows]
    rel = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    # end to end through the host-buffer C-ABI call (rf_create_standard_gaussian_field_grid): the
    # field is computed on the device and copied whole into the caller's page-locked array
    host = torch.empty((NMC, n), dtype=torch.float64).pin_memory()
    oa = host.numpy().T  # n x Nmc view, Fortran order
    gargs = ((0.0, 0.0, 0.0), (SPACING,) * 3, GRID, 1, 1, CORRL, 0.0, 1.0, NMC)
    rf.create_standard_gaussian_field_grid(*gargs, randField=oa, **o)
    e_steps = 3
    t0 = time.perf_counter()
    for _ in range(e_steps):
        rf.create_standard_gaussian_field_grid(*gargs, randField=oa, **o)
    e2e_s = (time.perf_counter() - t0) / e_steps
    ctx.close()
    del dout, flush, host
    torch.cuda.empty_cache()
    return {"api": "rf_generate_grid (device field)", "workload": WORKLOAD, "value": n * NMC / (ms / 1e3),
            "unit": "field values/s", "ms_per_call": ms, "phasor_coeff_ms": float(np.mean([k[0] for k in kms])),
            "axes_ms": axes_ms, "gpu_launches_per_call": launches / steps, "dtype": "f64",
            "rel_l2_vs_oracle": rel, "accuracy_sample": "48 random points x 64 realizations vs the FP64 oracle",
            "roofline": {"bound": "fp64", "achieved": 2.0 * fma / (axes_ms / 1e3) / 1e12, "peak": peak,
                         "unit": "TFLOP/s", "frac": 2.0 * fma / (axes_ms / 1e3) / 1e12 / peak,
                         "peak_source": "nominal: 64 FP64 FMA/clk/SM x SMs x 1965 MHz",
                         "algorithmic_fma_per_call": fma,
                         "hbm_ms": 8.0 * n * NMC / (peaks()[0].get("hbm_gbs", 6650.0) * 1e9) * 1e3},
            "e2e": {"value": n * NMC / e2e_s, "unit": "field values/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(8 * n * NMC),
                    "api": "rf_create_standard_gaussian_field_grid (host randField, pinned)"}}


def bench_batched(args, rf, torch, local):
    """512 requests in one grouped launch (rf_generate_batch_device, CUDA
    graph replay after the first batch), device-resident buffers; e2e through
    rf_generate_batch with host buffers when host memory allows."""
    rs = np.random.RandomState(2024)
    mix = [draw_request(rs) for _ in range(BATCH_REQUESTS)]
    values = float(sum(m["points"].shape[0] * m["Nmc"] for m in mix))
    ctx = rf.Context(local)
    keep, reqs = [], []
    for i, m in enumerate(mix):
        dx = torch.from_numpy(m["points"]).cuda(local)
        dout = torch.empty((m["Nmc"], m["points"].shape[0]), dtype=torch.float64, device=f"cuda:{local}")
        keep.append((dx, dout))
        reqs.append(rf.make_request(dx, "gaussian", m["marg"], m["corrL"], m["avg"], m["var"], m["Nmc"], m["method"],
                                    dout, precision="bf16", seed_start=i, nDim=3, n=m["points"].shape[0],
                                    **m["opts"]))
    stream = torch.cuda.Stream(device=local)
    for _ in range(max(2, args.warmup)):  # the first batch runs the tuner
        ctx.generate_batch_device(reqs, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    steps = max(2, min(args.steps, 3))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with torch.cuda.stream(stream):
        for a, b in ev:
            a.record(stream)
            ctx.generate_batch_device(reqs, stream=stream.cuda_stream)
            b.record(stream)
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in ev]
    st = ctx.batch_stats()
    out = {"workload": f"{BATCH_REQUESTS} requests: n log-uniform 1e3-1e6 in a box of side U[1,20], Nmc U{{1..128}}, "
                       "method 1|2, corrL U[0.5,4]^3, gaussian|lognormal; Shinozuka 24^3x4, isotropic 64x64",
           "field_values_per_batch": values, "value": values * steps / (sum(ms) / 1e3), "unit": "field values/s",
           "ms_per_batch": float(np.mean(ms)), "p50_ms": float(np.percentile(ms, 50)),
           "p99_ms": float(np.percentile(ms, 99)),
           "latency_note": "one grouped launch: every request of a batch completes with it",
           "grouped_launch": st, "precision": "bf16"}
    # end to end with host buffers (needs about 2x the fields in host memory)
    need = 8.0 * values + sum(m["points"].nbytes for m in mix)
    try:
        import psutil
        avail = float(psutil.virtual_memory().available)
    except Exception:
        avail = 0.0
    del keep
    torch.cuda.empty_cache()
    if avail > 2.0 * need and not args.no_e2e:
        hx = [np.asfortranarray(m["points"].T) for m in mix]
        ho = [np.empty((m["points"].shape[0], m["Nmc"]), order="F") for m in mix]
        hreqs = [rf.make_request(hx[i], "gaussian", m["marg"], m["corrL"], m["avg"], m["var"], m["Nmc"], m["method"],
                                 ho[i], precision="bf16", seed_start=i, **m["opts"]) for i, m in enumerate(mix)]
        rf.generate_batch(ctx, hreqs)
        t0 = time.perf_counter()
        rf.generate_batch(ctx, hreqs)
        dt = time.perf_counter() - t0
        out["e2e"] = {"value": values / dt, "unit": "field values/s", "ms_per_batch": dt * 1e3,
                      "h2d_bytes_per_step": int(sum(m["points"].nbytes for m in mix)),
                      "d2h_bytes_per_step": int(8 * values), "api": "rf_generate_batch (pageable host buffers)"}
        del hx, ho
    else:
        out["e2e"] = {"value": None, "reason": f"host memory available {avail / 1e9:.0f} GB < 2x {need / 1e9:.0f} GB"}
    ctx.close()
    return out


class PinnedRing:
    """Page-locked output buffers for the serving run: one arena handed out
    in arrival order and returned in the same order (requests are reaped in
    submission order), so a ring suffices; alloc returns None when the
    outstanding requests hold the whole arena."""

    def __init__(self, torch, doubles):
        import collections
        import threading

        self.t = torch.empty(int(doubles), dtype=torch.float64).pin_memory()
        self.a = self.t.numpy()
        self.cap = int(doubles)
        self.head = 0
        self.live = collections.deque()
        self.lock = threading.Lock()

    def alloc(self, n):
        n = (int(n) + 31) // 32 * 32
        with self.lock:
            if not self.live:
                start = 0
            else:
                tail = self.live[0][0]
                if self.head >= tail:
                    start = self.head if self.head + n <= self.cap else (0 if n <= tail else None)
                else:
                    start = self.head if self.head + n <= tail else None
            if start is None:
                return None
            self.live.append((start, start + n))
            self.head = start + n
            return start

    def free_oldest(self):
        with self.lock:
            self.live.popleft()
            if not self.live:
                self.head = 0


def bench_serving(args, rf, torch, local, rate=SERVE_RATE, seconds=None, arena_gb=None):
    """Open-loop Poisson arrivals at `rate` requests/s for `seconds` into the
    serving loop (rf_server_submit / rf_server_submit_blended).

    Every arrival is a fresh request with its own seed (seed_start = arrival
    index): sizes as the batched mix (n log-uniform 1e3-1e6 in a box of side
    U[1, 20], Nmc U{1..128}, method 1|2, corrL U[0.5, 4]^3, gaussian|lognormal)
    plus, with probability 5%, a 256^3 structured grid (spacing 0.05,
    Nmc 16) blended from 8 subdomains with about 10% overlap.  Points come from
    a pool of unit-box point sets: a request of box side s and correlation
    lengths L is issued as the same request on the unit box with correlation
    lengths L / s (the generator divides the points by corrL first, and the
    wavevector counts are explicit, so the field is the same).  Outputs come
    from a page-locked ring; an arrival that finds the ring full is shed and
    counted.  Latency runs from the arrival's scheduled time to the field in
    the caller's buffer: the delay before the submit call plus the server's
    time from entering rf_server_submit.  No client pool: arrivals never wait
    for a client."""
    import threading

    T = float(seconds if seconds is not None else args.serve_seconds)
    try:
        import psutil
        avail = float(psutil.virtual_memory().available)
    except Exception:
        avail = 64e9
    gb = arena_gb if arena_gb is not None else min(48.0, 0.4 * avail / 1e9)
    ring = PinnedRing(torch, gb * 1e9 / 8)
    rs = np.random.RandomState(77)
    pool = [np.ascontiguousarray(rs.uniform(0.0, 1.0, size=(1000000, 3)).astype(np.float32).astype(np.float64))
            for _ in range(4)]
    pool = [torch.from_numpy(p).pin_memory().numpy() for p in pool]
    srv = rf.Server(device=local, precision="bf16")
    big = rf.BlendGrid.make((256, 256, 256), (0.05, 0.05, 0.05), (2, 2, 2), 0.65)
    G = 256 ** 3

    def draw(k):
        q = np.random.RandomState(1000003 + k)
        method = 1 if q.uniform() < 0.5 else 2
        marg = "lognormal" if q.uniform() < 0.5 else "gaussian"
        corrL = q.uniform(0.5, 4.0, 3)
        avg, var = (1.0, 0.25) if marg == "lognormal" else (0.0, 1.0)
        opts = dict(k_nstep=(KN, KN, KN)) if method == 2 else dict(iso_n_radial=64, iso_n_dir=64)
        if q.uniform() < 0.05:
            return dict(kind="grid256", n=G, Nmc=16, method=2, marg=marg, corrL=(1.0, 1.0, 1.0), avg=avg, var=var,
                        opts=dict(k_nstep=(KN, KN, KN)))
        n = int(np.exp(q.uniform(np.log(1e3), np.log(1e6))))
        side = q.uniform(1.0, 20.0)
        return dict(kind="box", n=n, Nmc=int(q.randint(1, 129)), method=method, marg=marg,
                    corrL=tuple(float(c) / side for c in corrL), avg=avg, var=var, opts=opts)

    # warm the slots (tuner, graphs, grid path) outside the measured window
    for k in range(6):
        m = draw(10 ** 7 + k)
        if m["kind"] != "box":
            continue
        o = np.empty((m["n"], m["Nmc"]), order="F")
        xa = pool[0][:m["n"]].T
        srv.wait(srv.submit(rf.make_request(xa, "gaussian", m["marg"], m["corrL"], m["avg"], m["var"], m["Nmc"],
                                            m["method"], o, seed_start=10 ** 7 + k, **m["opts"])))
    ob = np.empty((G, 16), order="F")
    srv.wait(srv.submit_blended(big, "gaussian", "gaussian", (1.0, 1.0, 1.0), 0.0, 1.0, 16, 2, ob, seed_start=1,
                                k_nstep=(KN, KN, KN)))
    del ob

    base = srv.stats()
    gaps = np.random.RandomState(78).exponential(1.0 / rate, size=int(rate * T * 1.5) + 16)
    arrivals = np.cumsum(gaps)
    arrivals = arrivals[arrivals < T]
    pending, lat, done_vals, errors = [], [], [0.0], []
    lock = threading.Lock()
    fin = threading.Event()
    t_last = [0.0]

    def reaper():
        while True:
            with lock:
                item = pending.pop(0) if pending else None
            if item is None:
                if fin.is_set():
                    return
                time.sleep(0.0005)
                continue
            ticket, t_sched, t_call, vals = item
            try:
                ms = srv.wait(ticket, timeout_s=300.0)
                lat.append((t_call - t_sched) * 1e3 + ms)
                done_vals[0] += vals
            except rf.RandomFieldError as e:  # reported in the line
                errors.append(str(e))
            ring.free_oldest()
            t_last[0] = time.perf_counter()

    th = threading.Thread(target=reaper)
    th.start()
    submitted = shed = 0
    offered = 0.0
    t0 = time.perf_counter()
    for k, ta in enumerate(arrivals):
        m = draw(k)
        vals = float(m["n"] * m["Nmc"])
        offered += vals
        while time.perf_counter() - t0 < ta:
            time.sleep(0.0001)
        start = ring.alloc(m["n"] * m["Nmc"])
        if start is None:
            shed += 1
            continue
        out = ring.a[start:start + m["n"] * m["Nmc"]].reshape(m["Nmc"], m["n"]).T  # n x Nmc, Fortran order
        t_call = time.perf_counter()
        if m["kind"] == "grid256":
            ticket = srv.submit_blended(big, "gaussian", m["marg"], m["corrL"], m["avg"], m["var"], m["Nmc"],
                                        m["method"], out, seed_start=k, **m["opts"])
        else:
            xa = pool[k % len(pool)][:m["n"]].T  # 3 x n, Fortran order
            req = rf.make_request(xa, "gaussian", m["marg"], m["corrL"], m["avg"], m["var"], m["Nmc"], m["method"],
                                  out, seed_start=k, **m["opts"])
            ticket = srv.submit(req, keep=xa)
        submitted += 1
        with lock:
            pending.append((ticket, t0 + ta, t_call, vals))
    t_arr = time.perf_counter() - t0
    fin.set()
    th.join(timeout=600.0)
    wall = max(t_last[0] - t0, t_arr)
    st = srv.stats()
    srv.close()
    del ring
    lat = np.asarray(lat) if lat else np.zeros(1)
    return {"workload": f"open-loop Poisson {rate:.0f} req/s for {T:.0f} s; fresh requests (own seed) as the batched "
                        "mix plus 5% 256^3 grids with Nmc 16, each blended from 8 subdomains (134^3, 12 shared "
                        "points) through the structured-grid path",
            "arrivals": int(len(arrivals)), "offered_rate_req_s": len(arrivals) / T,
            "submitted": submitted, "achieved_rate_req_s": submitted / T, "shed": shed,
            "shed_reason": f"page-locked output ring of {gb:.0f} GB full", "completed": int(st["completed"] - base["completed"]),
            "failed": int(st["failed"] - base["failed"]), "errors": errors[:3], "n_errors": len(errors),
            "value": done_vals[0] / wall, "unit": "field values/s", "offered_field_values_per_s": offered / T,
            "duration_s": wall,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "max_ms": float(lat.max()),
            "server_p50_ms": st["p50_ms"], "server_p99_ms": st["p99_ms"], "batches": st["batches"] - base["batches"],
            "latency": "scheduled arrival -> field in the caller's page-locked buffer (the delay before the submit "
                       "call plus the server's time from entering rf_server_submit)"}


def run_grid_case(args):
    """The structured-grid path alone: Shinozuka on the --grid grid (spacing
    0.05, corrL (2, 1, 0.5), 24^3 x 4 wavevectors, Nmc 64) through
    rf_generate_grid; W untimed and K timed calls, device field."""
    import torch

    import randomfield_b200 as rf

    torch.cuda.set_device(0)
    n = int(np.prod(GRID))
    ctx = rf.Context(0)
    ctx.set_timing(True)
    dout = torch.empty((NMC, n), dtype=torch.float64, device="cuda")

    def call():
        ctx.generate_grid(dout, (0.0, 0.0, 0.0), (SPACING,) * 3, GRID, 1, 1, CORRL, 0.0, 1.0, NMC,
                          k_nstep=(KN, KN, KN))

    for _ in range(args.warmup):
        call()
    ctx.synchronize()
    kms = []
    for _ in range(args.steps):
        call()
        t_tab, t_axes, _, _ = ctx.last_times()
        kms.append(t_tab + t_axes)
    ctx.synchronize()
    if not torch.isfinite(dout).all().item():
        raise RuntimeError("non-finite field values")
    ms = float(np.mean(kms))
    print(json.dumps({"case": "grid", "workload": f"shinozuka {GRID} grid, h {SPACING}, K {KN}^3 x 4, Nmc {NMC}",
                      "ms_per_call": ms, "value": n * NMC / (ms / 1e3), "unit": "field values/s",
                      "steps": args.steps, "warmup": args.warmup}))
    ctx.close()


def run_iso_case(args):
    """The isotropic request of config 2 alone (GEN_TABLE, BF16 unless
    --precision): n points U[0,10]^3, 64 x 64 wavevectors, lognormal avg 1
    var 0.25, Nmc 64; W untimed and K timed calls, device-resident."""
    import torch

    import randomfield_b200 as rf

    torch.cuda.set_device(0)
    rs = np.random.RandomState(12)
    n = args.points
    pts = rs.uniform(0.0, 10.0, size=(n, 3)).astype(np.float32).astype(np.float64)
    ctx = rf.Context(0)
    ctx.set_timing(True)
    dx = torch.from_numpy(pts).cuda()
    dout = torch.empty((64, n), dtype=torch.float64, device="cuda")

    def call():
        ctx.generate(dx, 3, n, 1, 2, (1.0, 1.0, 1.0), 1.0, 0.25, 64, 1, dout, precision=args.precision,
                     iso_n_radial=64, iso_n_dir=64)

    for _ in range(args.warmup):
        call()
    ctx.synchronize()
    kms = []
    for _ in range(args.steps):
        call()
        kms.append(ctx.last_times()[1])
    ctx.synchronize()
    if not torch.isfinite(dout).all().item():
        raise RuntimeError("non-finite field values")
    ms = float(np.mean(kms))
    print(json.dumps({"case": "isotropic", "workload": f"{n} points U[0,10]^3, isotropic 64 x 64, Nmc 64, lognormal",
                      "precision": args.precision, "contract_ms": ms, "value": n * 64 / (ms / 1e3),
                      "unit": "field values/s", "steps": args.steps, "warmup": args.warmup}))
    ctx.close()


def run_batch_case(args):
    """--case batch: a batch of --batch-requests requests of the batched mix
    with point counts capped at --batch-max-points (the operand tables are as
    large as in the full mix, the device footprint small), run through the
    grouped launch --warmup + --steps times; one JSON line with the grouped
    launch's phase times.  For profiler captures of the grouped kernels."""
    import torch
    import randomfield_b200 as rf

    rs = np.random.RandomState(2024)
    ctx = rf.Context(0)
    keep, reqs = [], []
    for i in range(args.batch_requests):
        m = draw_request(rs)
        pts = m["points"][: args.batch_max_points]
        dx = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
        dout = torch.empty((m["Nmc"], pts.shape[0]), dtype=torch.float64, device="cuda")
        keep.append((dx, dout))
        reqs.append(rf.make_request(dx, "gaussian", m["marg"], m["corrL"], m["avg"], m["var"], m["Nmc"], m["method"],
                                    dout, precision=args.precision, seed_start=i, nDim=3, n=pts.shape[0],
                                    **m["opts"]))
    tab, con = [], []
    for it in range(args.warmup + args.steps):
        ctx.generate_batch_device(reqs)
        torch.cuda.synchronize()
        st = ctx.batch_stats()
        if it >= args.warmup:
            tab.append(st["tables_ms"])
            con.append(st["contract_ms"])
    print(json.dumps({"case": "batch", "workload": f"{args.batch_requests} requests of the batched mix, points capped "
                      f"at {args.batch_max_points}", "precision": args.precision, "units": st["units"],
                      "tables_ms": float(np.mean(tab)), "contract_ms": float(np.mean(con)), "steps": args.steps,
                      "warmup": args.warmup}))
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="bf16", choices=["bf16", "fp16", "bf16_fast", "fp8", "fp32"])
    ap.add_argument("--no-forms", action="store_true", help="skip the other precision forms")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end timing")
    ap.add_argument("--no-batched", action="store_true", help="skip the 512-request batched form")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop form")
    ap.add_argument("--no-grid", action="store_true", help="skip the structured-grid path (rf_generate_grid)")
    ap.add_argument("--serve-low-rate", type=float, default=30.0,
                    help="second serving run at this arrival rate (requests/s), below the device's capacity")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="duration of the Poisson arrival stream (the serving config: 60 s)")
    ap.add_argument("--serve-sat-rate", type=float, default=600.0,
                    help="arrival rate (requests/s) of the saturated serving run")
    ap.add_argument("--case", default="headline", choices=["headline", "iso", "grid", "batch"],
                    help="iso: only the isotropic request of config 2 (GEN_TABLE), on --points points; grid: only "
                         "the structured-grid path (rf_generate_grid) on --grid; batch: a small batch of the "
                         "batched mix (--batch-requests, --batch-max-points); all for profiler captures of those "
                         "kernels, each printing one JSON line of its own")
    ap.add_argument("--batch-requests", type=int, default=24, help="requests of the --case batch batch")
    ap.add_argument("--batch-max-points", type=int, default=5000, help="point cap of the --case batch requests")
    ap.add_argument("--points", type=int, default=200000, help="points of the --case iso request")
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
    if args.case == "iso":
        run_iso_case(args)
        return
    if args.case == "grid":
        run_grid_case(args)
        return
    if args.case == "batch":
        run_batch_case(args)
        return

    import torch
    import torch.distributed as dist

    import randomfield_b200 as rf
    from randomfield_b200 import replicas

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    xh = grid_points()
    n = xh.shape[0]
    opts = dict(precision=args.precision, k_nstep=(KN, KN, KN), seed_start=replicas.replica_seed(0, rank),
                x_range=extent(), device=local)
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
    values = n * NMC
    # whole job: the work of all replicas over the slowest rank's time
    units, secs = replicas.aggregate(values * args.steps, total_ms / 1e3, dist if world > 1 else None,
                                     device=f"cuda:{local}")
    total_ms = secs * 1e3
    value = units / secs

    # accuracy of the timed form over the whole field, outside the timed
    # region: the FP64 reference of every value, summed axis by axis from the
    # oracle's own wavevectors and phases (the checker; the gaussian marginal
    # with avg 0 and var 1 is the identity)
    from oracle import oracle as O

    acc = None
    if rank == 0:
        acc = field_accuracy(O, dout, seed=rank)

    # other precision forms, same workload (fewer steps)
    forms = {}
    if not args.no_forms:
        for prec in ("fp16", "bf16_fast", "fp8", "fp32"):
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
    K = 4 * KN ** 3
    flops = 2.0 * n * (2 * K) * NMC  # algorithmic: the TF32 K-steps' second MMA is not credited
    tflops = flops / (kern_ms / 1e3) / 1e12
    peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp) and GRID == (128, 128, 128):
        with open(tp) as f:
            traffic = json.load(f).get(args.precision)
    # the three bounds of the step: tensor MMA, SFU sincos, HBM bytes (the SFU
    # rate is measured live by a MUFU microbenchmark kernel of the library)
    sfu = rf.measure_sfu_rate(local)
    pairs = float(n) * 3 * KN  # GEN_GRID3: per-axis phasors only
    hbm_bytes = 8.0 * n * NMC + 24.0 * n + 2.0 * (2 * K) * (2 * NMC)
    bounds = {"tensor_ms": flops / (peak * 1e12) * 1e3, "sfu_ms": pairs / sfu * 1e3,
              "hbm_ms": hbm_bytes / (pk.get("hbm_gbs", 6650.0) * 1e9) * 1e3}
    # the 16-bit forms of this 3-D grid workload run the outer-group contraction on CTA pairs, FP8 the
    # trig-tile one
    kname = ("rf_outer_pair_kernel (outer-group tcgen05.mma.cta_group::2 contraction + fused i3 epilogue)"
             if args.precision in ("bf16", "fp16", "bf16_fast") else
             "rf_tc_kernel (tcgen05 contraction + fused epilogue)")
    roof = {"bound": "tensor", "achieved": tflops, "peak": peak, "unit": "TFLOP/s", "frac": tflops / peak,
            "traffic": traffic, "kernel": kname,
            "kernel_ms": kern_ms, "peak_source": f"bf16_tflops_sustained, {src}",
            "algorithmic_flops_per_launch": flops, "bounds": bounds,
            "sfu_pairs_per_s": sfu, "sfu_pairs_per_launch": pairs,
            "note": "the slowest of the three bounds is the tensor MMA (algorithmic FLOPs 2 n 2K Nmc; the extra "
                    "MMA cycles of the TF32 K-steps and of zero realization columns are not credited); the "
                    "outer-group generators need sincos only for the per-axis phasors (n1 + n2 + n3 per point), "
                    "GEN_TABLE one pair per (point, wavevector)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = os.cpu_count() or 1
        rate, rows_s, t = cpu_sample(xh, 3.0, cores)
        cpu = {"value": rate, "unit": "field values/s", "cores": cores, "kind": "port",
               "sample": f"{rows_s} points x 1 realization, full K = {K}, reference slab/DGEMM/cos/GEMV loop"}

    if world > 1:
        dist.barrier()
    ctx.close()
    del dx, dout, flush
    torch.cuda.empty_cache()
    batched = serving = configs = sgrid = None
    def section(fn, *a, **kw):
        """One optional part of the line; an error is reported in its place."""
        try:
            return fn(*a, **kw)
        except Exception as e:  # noqa: BLE001 - the headline line must still be printed
            return {"error": f"{type(e).__name__}: {e}"}

    if rank == 0 and world == 1 and not args.no_forms:
        configs = section(bench_configs, args, rf, torch, local, sfu, peak)
    if rank == 0 and world == 1 and not args.no_grid and GRID == (128, 128, 128):
        sgrid = section(bench_grid, args, rf, torch, local)
    if rank == 0 and world == 1 and not args.no_batched and args.precision != "fp32":
        batched = section(bench_batched, args, rf, torch, local)
    if rank == 0 and world == 1 and not args.no_serve and args.precision != "fp32":
        serving = section(bench_serving, args, rf, torch, local)
        if "error" not in serving:
            # the same loop far above its capacity (the ring sheds the excess): the throughput it sustains
            serving["saturated"] = section(bench_serving, args, rf, torch, local, rate=args.serve_sat_rate,
                                           seconds=15.0)
            # and well below it: the latency of an unsaturated loop
            serving["at_low_rate"] = section(bench_serving, args, rf, torch, local, rate=args.serve_low_rate,
                                             seconds=15.0)
    if rank == 0:
        line = {
            "metric": "field values/s", "value": value, "unit": "field values/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"bf16": "bf16", "fp16": "f16", "bf16_fast": "bf16", "fp8": "e4m3", "fp32": "f32"}[args.precision],
            "data": "synthetic",
            "config": {"workload": WORKLOAD if GRID == (128, 128, 128) else f"{WORKLOAD} on a {GRID} grid", "n_points": n, "Nmc": NMC, "K": K, "precision": args.precision,
                       "operands": {"bf16": "bf16; tf32 on the K-steps carrying 75 % of the variance",
                                    "fp16": "f16", "bf16_fast": "bf16", "fp8": "e4m3 hi/lo",
                                    "fp32": "f32"}[args.precision],
                       "l2": "flushed between timed steps (256 MiB write); output 1 GiB per step",
                       "parallelism": f"replicas x{world}"},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "accuracy": acc,
            "forms": forms,
            "configs": configs,
            "structured_grid": sgrid,
            "batched": batched,
            "serving": serving,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
