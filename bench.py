"""Benchmark of the filtering hot path on B200.

Default workload (the large bootstrap-PF configuration): LGSSM with Dx=16,
Dy=8, A random orthogonal * 0.95, Q = 0.1 I, H_ij ~ N(0, 1/Dx), R = 0.2 I,
N = 2^20 particles in FP32 SoA, T = 1000, systematic resampling when
ESS < 0.5 N, FP64 normaliser and cumulative weights, in-kernel Philox noise.
One step = one full filter run (N * T particle-steps).  The line also carries
`parity` (the estimate against the exact Kalman log-likelihood in Monte-Carlo
standard deviations; a full-N teacher-forced check of the first steps against
the FP64 oracle with ancestor boundary counts), the 16-thread and
single-thread CPU baselines, and `secondary`: the batched Kalman bank (65,536
uneven filters) and the serving loop at 200 and 1000 req/s from the same process.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload pf|pf1d|kf|smooth|rbpf|serve|csmc|kfgrad]

Under torchrun each rank runs an independent replica (the filters shard by
filter; no data-path collective).  Rank 0 prints one JSON line.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ssmproblems.jl_b200"))

import numpy as np  # noqa: E402

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0  # GB/s, used only when MEASURED_PEAKS.json is absent


def _peaks():
    try:
        with open(PEAKS_FILE) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # let nvidia-smi finish starting up before the timed region begins
            t0 = time.perf_counter()
            while not self.rows and time.perf_counter() - t0 < 3.0:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=2)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def _dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _max_over_ranks(x, world, dev):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------------------------- #
def cpu_baseline_pf(model, ys, N, seconds=12.0, threads=None):
    """The FP64 oracle port timed on this host: same model, N particles, a
    bounded number of time steps (sample), all host threads."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    threads = threads or os.cpu_count() or 1
    om = O.LGModel(model.prior.mu0, model.prior.Sigma0, model.dyn.A, model.dyn.b, model.dyn.Q,
                   model.obs.H, model.obs.c, model.obs.R)
    # calibrate with 1 step, then run as many steps as fit the time budget
    t0 = time.perf_counter()
    O.pf_run(om, N, ys[:1], threshold=0.5, seed=1, threads=threads)
    one = time.perf_counter() - t0
    steps = int(max(1, min(len(ys), seconds / max(one, 1e-3))))
    t0 = time.perf_counter()
    O.pf_run(om, N, ys[:steps], threshold=0.5, seed=1, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": N * steps / dt, "unit": "particle-steps/s", "cores": threads,
            "kind": "port",
            "sample": f"FP64 C oracle, same Dx=16/Dy=8 model, N={N}, first {steps} of T steps, "
                      f"{threads} OpenMP threads (serial cumsum/LSE as in the reference)"}


def pf_parity(ctx, model, ys, N, ll_timed, seeds=8, tf_steps=4):
    """Accuracy of the headline configuration against FP64 (outside the timed
    region): (1) the log-likelihood estimate against the exact Kalman value, in
    Monte-Carlo standard deviations of the estimate over `seeds` independent
    runs; (2) teacher forcing at full N: one run of the first `tf_steps` steps
    records every state, then each step is re-done by the FP64 oracle from the
    GPU's own previous state with the same injected noise and uniforms."""
    import torch
    import gfb200 as G
    from gfb200.plans import PfPlan
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    om = O.LGModel(model.prior.mu0, model.prior.Sigma0, model.dyn.A, model.dyn.b, model.dyn.Q,
                   model.obs.H, model.obs.c, model.obs.R)
    T = len(ys)
    ll_kf = O.kf_filter(om, ys)[0]
    algo = G.BF(N, threshold=0.5)
    ys_dev = torch.tensor(ys, dtype=torch.float64, device=f"cuda:{ctx.device}")
    lls = []
    for s in range(seeds):
        p = PfPlan(model, algo, T, seed=5000 + s, ctx=ctx, graph=True)
        p.run(ys_dev)
        ctx.synchronize()
        lls.append(float(p.ll.item()))
        p.close()
    lls = np.array(lls)
    sd = float(lls.std(ddof=1))
    # teacher forcing at full N
    rng = np.random.default_rng(77)
    Tt = tf_steps
    dx = model.dyn.A.shape[0]
    noise = rng.standard_normal((Tt + 1, dx, N)).astype(np.float32)
    unif = rng.random(Tt)
    cb = G.DenseAncestorCallback()
    st, _ = G.filter(model, algo, ys[:Tt], noise=noise, uniforms=unif, callback=cb, ctx=ctx)
    hist, lwh, anc = cb.container._hist, cb.container.weights, cb.container.ancestors
    err_x = err_ll = 0.0
    bad = boundary = slots = n_res = 0
    for t in range(1, Tt + 1):
        ref = O.pf_step(om, hist[t - 1].T.astype(np.float64), np.zeros(N) if t == 1 else lwh[t - 2],
                        ys[t - 1], noise[t].astype(np.float64), unif[t - 1], uniform=t == 1,
                        threshold=0.5)
        n_res += int(ref["resampled"])
        diff = anc[t - 1] != ref["ancestors"]
        inside = ref["margins"] <= 1e-8
        bad += int(np.sum(diff & ~inside))
        boundary += int(np.sum(diff & inside))
        slots += N if ref["resampled"] else 0
        if not diff.any():
            err_x = max(err_x, float(np.max(np.abs(hist[t].T - ref["x"]) / (np.abs(ref["x"]) + 1.0))))
        err_ll = max(err_ll, abs(float(st.ll_steps[t - 1]) - ref["ll_inc"]))
    return {
        "ll_kf_exact": ll_kf, "ll_timed_run": ll_timed,
        "ll_pf_mean": float(lls.mean()), "ll_pf_sd": sd, "ll_runs": seeds,
        "ll_dev_in_sd": (ll_timed - ll_kf) / sd if sd > 0 else None,
        "ll_mean_dev_in_se": (float(lls.mean()) - ll_kf) / (sd / np.sqrt(seeds)) if sd > 0 else None,
        # log Z-hat is biased low by about Var(log Z-hat) / 2 (Z-hat unbiased and
        # near log-normal): the mean's deviation after that correction
        "ll_mean_dev_bias_corrected_in_se":
            (float(lls.mean()) + sd * sd / 2 - ll_kf) / (sd / np.sqrt(seeds)) if sd > 0 else None,
        "teacher_forced": {"N": N, "steps": Tt, "resampling_steps": n_res,
                           "state_max_err_rel_plus_1": err_x, "ll_inc_max_abs_err": err_ll,
                           "ancestor_mismatches_outside_1e-8_band": bad,
                           "ancestor_boundary_cases": boundary, "ancestor_slots_checked": slots,
                           "oracle": "FP64 C restatement of the reference PF step"},
    }


def _pf_wide(args, world, rank, local):
    """The Dx=64, Dy=32 half of the large-PF configuration: N = 2^18, T = 200,
    FP32 state on the tensor-core propagation; graph replays timed with events,
    the propagate per launch from eager events for its roofline."""
    import torch
    import gfb200 as G
    from gfb200 import workloads as W
    from gfb200.plans import PfPlan
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    ctx = G.Context(local)
    N, T, dx, dy, K = 2**18, 200, 64, 32, 3
    model, ys = W.lgssm_rot(seed=64, dx=dx, dy=dy, T=T)
    algo = G.BF(N, threshold=0.5)
    ys_dev = torch.tensor(ys, dtype=torch.float64, device=dev)
    plan = PfPlan(model, algo, T, seed=3 + rank, ctx=ctx, graph=True)
    for _ in range(3):
        plan.run(ys_dev)
    ctx.synchronize()
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(ext)
        for _ in range(K):
            plan.run(ys_dev)
        e1.record(ext)
        e1.synchronize()
    ms = _max_over_ranks(e0.elapsed_time(e1), world, dev)
    ll, n_res = float(plan.ll.item()), int(plan.resampled.sum().item())
    plan.close()
    eplan = PfPlan(model, algo, T, seed=3 + rank, ctx=ctx, graph=False)
    prof = _profiled(ctx, lambda: eplan.run(ys_dev), 1, [(0, "propagate"), (1, "resample"),
                                                         (5, "ancestor_fill")])
    eplan.close()
    ctx.close()
    pms, pn = prof["propagate"]
    avg = pms / max(pn, 1)
    bytes_launch = N * (8 * dx + 8)
    peak, peak_kind = _peaks()
    return {"metric": "particle-steps/s", "value": N * T * K * world / (ms / 1e3),
            "unit": "particle-steps/s", "ms_per_step": ms / K,
            "config": {"workload": f"bootstrap PF, LGSSM Dx={dx} Dy={dy} (A orthogonal*0.95, Q=0.1I, "
                                   f"H~N(0,1/{dx}), R=0.2I), N=2^18, T={T}, systematic at ESS<0.5N",
                       "resampled_steps": n_res, "ll": ll, "precision": "FP32 state, FP64 normaliser"},
            "roofline": {"bound": "hbm", "achieved": bytes_launch / (avg / 1e3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": bytes_launch / (avg / 1e3) / 1e9 / peak,
                         "kernel": "pf_lg_propagate_tc<64,32> (tcgen05 3xTF32)", "peak_source": peak_kind,
                         "avg_launch_ms": avg, "bytes_per_launch": bytes_launch},
            "kernels_ms": {k: v[0] for k, v in prof.items()}, "clocks": clk.summary()}


def _secondary(args, world, rank, local):
    """The other halves of the metric, from the same process: the Dx=64 half of
    the large PF, the RBPF (config 4), the batched Kalman bank (config 3) and
    the serving loop at stated request rates."""
    import copy
    out = {"pf_dx64": _pf_wide(args, world, rank, local)}
    a = copy.copy(args)
    a.steps, a.warmup, a.no_cpu_baseline = 3, 3, True
    rb = bench_rbpf(a, world, rank, local)
    out["rbpf"] = {k: rb[k] for k in ("metric", "value", "unit", "ms_per_step", "config", "e2e",
                                      "roofline", "clocks")}
    a = copy.copy(args)
    a.steps, a.warmup = 2, 3
    kf = bench_kf(a, world, rank, local, accuracy_sample=32)
    out["kf_bank"] = {k: kf[k] for k in ("metric", "value", "unit", "ms_per_step", "config",
                                          "roofline", "plain_form_kf_steps_per_s",
                                          "batched_over_plain", "accuracy", "clocks")}
    out["serving"] = []
    for rate, reqs in ((200.0, 1000), (1000.0, 2000)):
        a = copy.copy(args)
        a.steps, a.warmup, a.serve_rate, a.serve_requests = 1, 1, rate, reqs
        sv = bench_serve(a, world, rank, local)
        out["serving"].append({"offered_req_s": sv["config"]["offered_req_s"],
                               "served_req_s": sv["value"], "latency_ms": sv["latency_ms"],
                               "completed": sv["completed"], "failed": sv["failed"],
                               "kf_steps_per_s": sv["kf_steps_per_s"],
                               "particle_steps_per_s": sv["particle_steps_per_s"],
                               "workload": sv["config"]["workload"]})
    return out


def bench_pf(args, world, rank, local):
    import torch
    import gfb200 as G
    from gfb200 import _lib as L
    from gfb200 import workloads as W
    from gfb200.plans import PfPlan

    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    ctx = G.Context(local)
    N, T, dx, dy = 2**20, args.pf_T, 16, 8
    model, ys = W.lgssm_rot(seed=1234, dx=dx, dy=dy, T=T)
    algo = G.BF(N, threshold=0.5)
    ys_dev = torch.tensor(ys, dtype=torch.float64, device=dev)
    # ---- timed region: graph replay of the plan (its normal form), inputs resident in HBM
    gplan = PfPlan(model, algo, T, seed=1000 + rank, ctx=ctx, graph=True)
    for _ in range(args.warmup):
        gplan.run(ys_dev)
    ctx.synchronize()
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    _barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0.record(ext)
        for _ in range(args.steps):
            gplan.run(ys_dev)
        ev1.record(ext)
        ev1.synchronize()
    torch.cuda.synchronize()
    _barrier(world)
    ms = ev0.elapsed_time(ev1)
    ms_max = _max_over_ranks(ms, world, dev)
    n_res = int(gplan.resampled.sum().item())
    ll = float(gplan.ll.item())
    gplan.close()
    # ---- per-kernel durations: the same K runs launched eagerly on the same
    # stream with CUDA events around every launch (graph nodes cannot be timed)
    plan = PfPlan(model, algo, T, seed=1000 + rank, ctx=ctx, graph=False)
    plan.run(ys_dev)
    ctx.synchronize()
    ctx.profile(True)
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(ext)
    for _ in range(args.steps):
        plan.run(ys_dev)
    p1.record(ext)
    p1.synchronize()
    eager_ms = p0.elapsed_time(p1) / args.steps
    prop_ms, prop_n = ctx.profile_read(0)
    scan_ms, scan_n = ctx.profile_read(1)
    prep_ms, prep_n = ctx.profile_read(4)
    fill_ms, fill_n = ctx.profile_read(5)
    ctx.profile(False)
    # ---- e2e through the C ABI with pinned host buffers
    import ctypes as C
    ys_pin = torch.tensor(ys, dtype=torch.float64).pin_memory()
    ll_pin = torch.zeros(1, dtype=torch.float64).pin_memory()
    steps_pin = torch.zeros(T, dtype=torch.float64).pin_memory()
    mc = model._c_struct()
    cfg, _, _ = __import__("gfb200.filtering", fromlist=["_pf_config"])._pf_config(algo, T, 7 + rank)
    out = L.PFOutC(ll_pin.data_ptr(), steps_pin.data_ptr(), None, None, None, None, None, None,
                   None)
    lib = L.load()
    e2e_times = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.check(ctx.h, lib.gf_pf_run(ctx.h, C.byref(mc), C.byref(cfg), T, ys_pin.data_ptr(), None,
                                     None, L.GF_MEM_HOST, C.byref(out)))
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_times.append(dt)
    e2e_s = _max_over_ranks(sum(e2e_times), world, dev)
    units = N * T * args.steps * world
    value = units / (ms_max / 1e3)
    peak, peak_kind = _peaks()
    # algorithmic bytes of one propagate launch (FP32 state): state read + write
    # 8*Dx, log-weight write 4, and either the log-weight read (no resample) or
    # the ancestor-index read (resample) 4
    launches = T * args.steps
    bytes_total = N * launches * (8 * dx + 8)
    prop_avg_ms = prop_ms / max(prop_n, 1)
    achieved = bytes_total / launches / (prop_avg_ms / 1e3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "pf_propagate_traffic.json")
    if os.path.exists(tf):
        try:
            traffic = json.load(open(tf)).get("dram_bytes_per_launch")
        except Exception:
            traffic = None
    line = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "bootstrap PF, LGSSM Dx=16 Dy=8 (A orthogonal*0.95, Q=0.1I, "
                               "H~N(0,1/16), R=0.2I), N=2^20, " f"T={T}, systematic at ESS<0.5N",
                   "N": N, "T": T, "dx": dx, "dy": dy, "precision": "FP32 state, FP64 normaliser",
                   "noise": "in-kernel Philox4x32-10", "parallelism": f"replicas x{world}",
                   "l2": "working set per time step ~140 MB > 126 MB L2 (no flush)",
                   "resampled_steps": n_res, "ll": ll},
        "e2e": {"value": units / e2e_s, "unit": "particle-steps/s",
                "h2d_bytes_per_step": int(ys.nbytes), "d2h_bytes_per_step": int(8 + 8 * T),
                "call": "gf_pf_run(GF_MEM_HOST) from pinned host buffers"},
        "gpu_launches": int(prop_n + scan_n + fill_n + prep_n + 2 * args.steps),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": "pf_lg_propagate_tc<16,8> (tcgen05 3xTF32)", "peak_source": peak_kind,
                     "avg_launch_ms": prop_avg_ms, "launches": prop_n,
                     "bytes_per_launch": bytes_total / launches},
        "kernels_ms": {"propagate": prop_ms, "resample": scan_ms, "ancestor_fill": fill_ms,
                       "prep_init": prep_ms},
        "timing": "value: CUDA events around K graph replays; kernels_ms / roofline: "
                  "events around every launch in K eager runs on the same stream",
        "eager_profiled_ms_per_step": eager_ms,
        "clocks": clk.summary(),
    }
    plan.close()
    if rank == 0 and not args.no_parity:
        line["parity"] = pf_parity(ctx, model, ys, N, ll)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_pf(model, ys, N, seconds=args.cpu_seconds)
        line["cpu_baseline_single_thread"] = cpu_baseline_pf(model, ys, N, seconds=args.cpu_seconds,
                                                             threads=1)
    ctx.close()
    if not args.no_secondary:
        line["secondary"] = _secondary(args, world, rank, local)
    return line


def bench_kf(args, world, rank, local, accuracy_sample=0):
    """Batched Kalman filters: 65536 uneven LGSSMs (Dx 2..32, Dy 1..Dx, T 64..2048),
    per-step ll / mean / covariance outputs, one graph-captured persistent plan
    with autotuned block sizes; the plain one-launch-per-filter form is timed on a
    sample for comparison."""
    import torch
    import gfb200 as G
    from gfb200 import _lib as L
    from gfb200 import workloads as W
    from gfb200.plans import KfPlan
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    ctx = G.Context(local)
    B = args.kf_filters
    algo = G.SRKF() if args.kf_algo == "srkf" else G.KalmanFilter()
    models, Ts, _ = W.kf_bank(B, seed=7 + rank, make_ys=False)
    plan = KfPlan(models, algo, Ts, ctx=ctx, flags=L.GF_PLAN_AUTOTUNE)
    ys = torch.randn(plan.n_y, dtype=torch.float64, device=dev)
    steps = torch.empty(plan.n_steps, dtype=torch.float64, device=dev)
    means = torch.empty(plan.n_means, dtype=torch.float32, device=dev)
    covs = torch.empty(plan.n_covs, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        plan.run(ys, steps, means, covs)
    ctx.synchronize()
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    _barrier(world)
    with ClockSampler(local) as clk:
        e0.record(ext)
        for _ in range(args.steps):
            plan.run(ys, steps, means, covs)
        e1.record(ext)
        e1.synchronize()
    ms = _max_over_ranks(e0.elapsed_time(e1), world, dev)
    assert int(plan.status.abs().sum().item()) == 0
    n_steps = plan.n_steps
    value = n_steps * args.steps * world / (ms / 1e3)
    dxs = np.array([m.dx for m in models], dtype=np.float64)
    dys = np.array([m.dy for m in models], dtype=np.float64)
    Tarr = np.array(Ts, dtype=np.float64)
    bytes_run = float(np.sum(Tarr * (8 * dys + 8 + 4 * dxs + 4 * dxs * dxs)))
    flops_run = float(np.sum(Tarr * 2 * (4 * dxs**3 + 4 * dys * dxs**2 + 4 * dys**2 * dxs + dys**3 / 3)))
    run_s = ms / 1e3 / args.steps
    peak, peak_kind = _peaks()
    # plain form: one launch per filter on a sample, extrapolated per KF step
    sample = min(256, B)
    idx = np.random.default_rng(0).choice(B, sample, replace=False)
    pm = [models[i] for i in idx]
    pT = [Ts[i] for i in idx]
    pplan = KfPlan(pm, algo, pT, ctx=ctx, flags=L.GF_PLAN_PLAIN | L.GF_PLAN_NO_GRAPH)
    pys = torch.randn(pplan.n_y, dtype=torch.float64, device=dev)
    pplan.run(pys)
    ctx.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(ext)
    pplan.run(pys)
    p1.record(ext)
    p1.synchronize()
    plain_value = pplan.n_steps / (p0.elapsed_time(p1) / 1e3)
    pplan.close()
    accuracy = None
    if accuracy_sample and rank == 0:
        # the timed run's own outputs for a sample of filters against the FP64
        # oracle fed the same observations
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        ys_h = ys.cpu().numpy()
        ll_h = plan.ll.cpu().numpy()
        offs = np.concatenate([[0], np.cumsum([t * m.dy for t, m in zip(Ts, models)])])
        worst = 0.0
        pick = np.random.default_rng(1).choice(B, min(accuracy_sample, B), replace=False)
        for f in pick:
            m = models[f]
            om = O.LGModel(m.prior.mu0, m.prior.Sigma0, m.dyn.A, m.dyn.b, m.dyn.Q, m.obs.H,
                           m.obs.c, m.obs.R)
            yf = ys_h[offs[f]:offs[f + 1]].reshape(Ts[f], m.dy)
            rll = O.kf_filter(om, yf, algo=args.kf_algo)[0]
            worst = max(worst, abs(ll_h[f] - rll) / max(1.0, abs(rll)))
        accuracy = {"filters_checked": int(len(pick)), "max_rel_ll_err_vs_fp64": worst,
                    "bar": "|d ll| / max(1, |ll|) <= 1e-4"}
    line = {
        "metric": "KF-steps/s", "value": value, "unit": "KF-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"{B} uneven LGSSMs, Dx~U{{2..32}}, Dy~U{{1..Dx}}, T~U{{64..2048}}, "
                               f"{'SRKF' if args.kf_algo == 'srkf' else 'KF'} with per-step ll/mean/cov",
                   "filters": B, "kf_steps": n_steps, "form": "one graph of persistent per-bucket launches, autotuned",
                   "l2": "outputs ~100 GB per run > L2 (no flush)"},
        "roofline": {"bound": "hbm", "achieved": bytes_run / run_s / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": bytes_run / run_s / 1e9 / peak, "traffic": None,
                     "fp32_tflops": flops_run / run_s / 1e12, "fp32_nominal_tflops": 74.4,
                     "fp32_frac_of_nominal": flops_run / run_s / 1e12 / 74.4,
                     "peak_source": peak_kind},
        "plain_form_kf_steps_per_s": plain_value,
        "batched_over_plain": value / world / plain_value,
        "accuracy": accuracy,
        "clocks": clk.summary(),
    }
    plan.close()
    ctx.close()
    return line


def _serve_stream(rng, mix, ypool, m1, y1, hm, yr):
    """Models, algorithms and observations of a request stream (serving_mix)."""
    import gfb200 as G
    from gfb200 import workloads as W
    out = []
    for t, kind, p in mix:
        if kind == "kf":
            dx, dy, T = p["dx"], p["dy"], p["T"]
            A = W.random_orthogonal(rng, dx) * rng.uniform(0.8, 0.99)
            H = rng.standard_normal((dy, dx)) / np.sqrt(dx)
            q = float(np.exp(rng.uniform(np.log(1e-3), 0.0)))
            r = float(np.exp(rng.uniform(np.log(1e-2), 0.0)))
            m = G.create_homogeneous_linear_gaussian_model(
                np.zeros(dx), np.eye(dx), A, np.zeros(dx), q * np.eye(dx), H, np.zeros(dy),
                r * np.eye(dy))
            out.append((t, m, G.KF(), ypool[:T * dy].reshape(T, dy), 0, T, 0))
        elif kind == "bf":
            out.append((t, m1, G.BF(p["N"], threshold=0.5), y1[:p["T"]], p["seed"], p["T"], p["N"]))
        else:
            algo = G.RBPF(G.BF(p["N"], threshold=0.5), G.KalmanFilter())
            out.append((t, hm, algo, yr[:p["T"]], p["seed"], p["T"], p["N"]))
    return out


def bench_serve(args, world, rank, local):
    """Served filtering (Poisson arrivals of a 70% KF / 25% BF / 5% RBPF mix):
    requests are submitted from host memory at their arrival times through the
    serving C ABI and each result returns to host memory; the line reports
    completed requests per second and the submit-to-result latency quantiles."""
    import gfb200 as G
    from gfb200 import workloads as W
    rate, M = args.serve_rate, args.serve_requests
    rng = np.random.default_rng(5 + rank)
    ypool = rng.standard_normal(5000 * 32)
    m1, y1 = W.lgssm_1d(seed=3, T=2000)
    hm, yr = W.rb_trend(seed=4, T=500)
    warm = _serve_stream(rng, W.serving_mix(60, rate, seed=99 + rank), ypool, m1, y1, hm, yr)
    streams = [_serve_stream(rng, W.serving_mix(M, rate, seed=11 + 100 * k + rank), ypool, m1, y1,
                             hm, yr) for k in range(args.steps)]
    srv = G.Server(device=local, hbm_budget_bytes=args.serve_hbm_gb << 30,
                   host_budget_bytes=4 << 30)

    def play(stream):
        t0 = time.perf_counter()
        h2d = 0
        for t, m, algo, ys, seed, T, N in stream:
            d = t0 + t - time.perf_counter()
            if d > 0:
                time.sleep(d)
            while True:
                try:
                    srv.submit(m, algo, ys, seed=seed, want_mean=True)
                    break
                except G.GFError as e:
                    if e.code != 8:  # GF_ERR_BUSY: back off and retry
                        raise
                    time.sleep(1e-4)
            h2d += ys.nbytes
        srv.drain()
        srv.poll(max_results=1 << 16)
        return h2d

    for _ in range(args.warmup):
        play(warm)
    srv.reset_stats()
    s0 = srv.stats()
    with ClockSampler(local) as clk:
        h2d = sum(play(st) for st in streams)
    st = srv.stats()
    srv.close()
    el = st["elapsed_ms"] / 1e3
    served = st["completed"] / el
    offered = M * args.steps / sum(s[-1][0] for s in streams)
    line = {
        "metric": "served requests/s", "value": served, "unit": "req/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": st["elapsed_ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"Poisson request stream at {rate:g} req/s: 70% KF (Dx 2..32, "
                               f"T 100..5000), 25% BF on the 1-D LGSSM (N 4096..262144, T 100..2000), "
                               f"5% RBPF (N 4096..32768, T 500)", "requests_per_step": M,
                   "offered_req_s": offered, "hbm_budget_gb": args.serve_hbm_gb},
        "latency_ms": {"p50": st["p50_ms"], "p99": st["p99_ms"], "mean": st["mean_ms"],
                       "max": st["max_ms"]},
        "completed": st["completed"], "failed": st["failed"], "rejected": st["rejected"],
        "kf_steps_per_s": st["kf_steps"] / el, "particle_steps_per_s": st["particle_steps"] / el,
        "gpu_launches": st["launches"] - s0["launches"],
        "e2e": {"value": served, "unit": "req/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": None},
        "hbm_peak_gb": st["hbm_peak"] / 2**30,
        "clocks": clk.summary(),
    }
    return line


def _profiled(ctx, fn, reps, classes):
    """Per-kernel-class (ms per launch, launches) over `reps` calls of fn with
    CUDA events around every launch on the context stream."""
    ctx.profile(True)
    for _ in range(reps):
        fn()
    ctx.synchronize()
    res = {}
    for cls, name in classes:
        ms, n = ctx.profile_read(cls)
        res[name] = (ms, n)
    ctx.profile(False)
    return res


def bench_rbpf(args, world, rank, local):
    """Rao-Blackwellised PF: outer 2-D AR(1) state, inner 8-D Kalman bank per
    particle with stochastic-volatility Q, 4-D observations; N = 65536, T = 500,
    systematic resampling at ESS < 0.5 N.  One step = one gf_rbpf_run call on
    device-resident observations (N * T particle-steps)."""
    import ctypes as C

    import torch
    import gfb200 as G
    from gfb200 import _lib as L
    from gfb200 import workloads as W
    from gfb200.filtering import _pf_config
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    ctx = G.Context(local)
    N, T = 65536, 500
    hm, ys = W.rb_trend(seed=1234, T=T)
    algo = G.RBPF(G.BF(N, threshold=0.5), G.KalmanFilter())
    mc = hm._c_struct()
    cfg, _, _ = _pf_config(algo.pf, T, 7 + rank)
    lib = L.load()
    ys_dev = torch.tensor(ys, dtype=torch.float64, device=dev)
    ll_dev = torch.zeros(1, dtype=torch.float64, device=dev)
    res_dev = torch.zeros(T, dtype=torch.int8, device=dev)
    out = L.PFOutC(ll_dev.data_ptr(), None, None, res_dev.data_ptr(), None, None, None, None, None)

    def run():
        L.check(ctx.h, lib.gf_rbpf_run(ctx.h, C.byref(mc), C.byref(cfg), T, ys_dev.data_ptr(), None,
                                       None, L.GF_MEM_DEVICE, C.byref(out), None))

    for _ in range(args.warmup):
        run()
    ctx.synchronize()
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    _barrier(world)
    with ClockSampler(local) as clk:
        e0.record(ext)
        for _ in range(args.steps):
            run()
        e1.record(ext)
        e1.synchronize()
    ms = _max_over_ranks(e0.elapsed_time(e1), world, dev)
    n_res = int(res_dev.sum().item())
    ll = float(ll_dev.item())
    prof = _profiled(ctx, run, args.steps, [(3, "rbpf_propagate"), (1, "resample"), (5, "ancestor_fill"),
                                             (4, "init")])
    # e2e: host observations in pinned memory, ll back to host
    ys_pin = torch.tensor(ys, dtype=torch.float64).pin_memory()
    ll_pin = torch.zeros(1, dtype=torch.float64).pin_memory()
    hout = L.PFOutC(ll_pin.data_ptr(), None, None, None, None, None, None, None, None)
    t_e2e = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.check(ctx.h, lib.gf_rbpf_run(ctx.h, C.byref(mc), C.byref(cfg), T, ys_pin.data_ptr(), None,
                                       None, L.GF_MEM_HOST, C.byref(hout), None))
        if i >= args.warmup:
            t_e2e.append(time.perf_counter() - t0)
    e2e_s = _max_over_ranks(sum(t_e2e), world, dev)
    units = N * T * args.steps * world
    value = units / (ms / 1e3)
    dxo, dz = 2, 8
    width = dxo + dz + dz * (dz + 1) // 2
    pms, pn = prof["rbpf_propagate"]
    avg = pms / max(pn, 1)
    bytes_launch = N * (8 * width + 8)  # state read + write, log-weight, ancestor / log-weight read
    peak, peak_kind = _peaks()
    line = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "RBPF on a hierarchical LGSSM: outer 2-D z_t = 0.9 z_{t-1} + N(0,0.3^2 I), "
                               "inner Dx=8 (A orthogonal*0.95, Q = 0.05 exp(z_t[1]) I), H 4x8, R = 0.1 I; "
                               "N=65536, T=500, systematic at ESS<0.5N",
                   "N": N, "T": T, "resampled_steps": n_res, "ll": ll,
                   "precision": "FP32 bank, FP64 innovation Cholesky and normaliser",
                   "l2": "state 2 x 12 MB per step fits in L2; inputs resident (no flush)"},
        "e2e": {"value": units / e2e_s, "unit": "particle-steps/s",
                "h2d_bytes_per_step": int(ys.nbytes), "d2h_bytes_per_step": 8,
                "call": "gf_rbpf_run(GF_MEM_HOST) from pinned host buffers"},
        # profiled classes + the unprofiled init, initial scalars and finish launches of each run
        "gpu_launches": int(sum(v[1] for v in prof.values()) + 3 * args.steps),
        "roofline": {"bound": "hbm", "achieved": bytes_launch / (avg / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": bytes_launch / (avg / 1e3) / 1e9 / peak, "traffic": None,
                     "kernel": "rbpf_propagate<2,8,4>", "peak_source": peak_kind,
                     "avg_launch_ms": avg, "bytes_per_launch": bytes_launch},
        "kernels_ms": {k: v[0] for k, v in prof.items()},
        "timing": "value: CUDA events around K gf_rbpf_run calls (allocation included); kernels: "
                  "events around every launch in K more calls",
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_rbpf(hm, ys, N, seconds=args.cpu_seconds)
    ctx.close()
    return line


def cpu_baseline_rbpf(hm, ys, N, seconds=12.0, threads=None):
    """The FP64 oracle's RBPF on this host: same model and N, a bounded number of
    time steps, all host threads."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    threads = threads or os.cpu_count() or 1
    op, od = hm.outer_prior, hm.outer_dyn
    ip, idn, ob = hm.inner_model.prior, hm.inner_model.dyn, hm.inner_model.obs
    om = O.RBModel(op.mu0, op.Sigma0, od.A, od.b, od.Q, ip.mu0, ip.Sigma0, idn.A, idn.b, idn.C,
                   idn.Q, ob.H, ob.c, ob.R, q_gamma=idn.q_gamma, q_index=idn.q_index)
    t0 = time.perf_counter()
    O.rbpf_run(om, N, ys[:1], threshold=0.5, seed=1, threads=threads)
    one = time.perf_counter() - t0
    steps = int(max(1, min(len(ys), seconds / max(one, 1e-3))))
    t0 = time.perf_counter()
    O.rbpf_run(om, N, ys[:steps], threshold=0.5, seed=1, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": N * steps / dt, "unit": "particle-steps/s", "cores": threads, "kind": "port",
            "sample": f"FP64 C oracle RBPF, same model, N={N}, first {steps} of T steps, "
                      f"{threads} OpenMP threads"}


def bench_pf1d(args, world, rank, local):
    """The README model (x_t = x_{t-1} + N(0, 0.1^2), y_t = x_t + N(0, 0.2^2)),
    bootstrap PF with N = 1024, T = 100, FP64, systematic at ESS < 0.5 N: a
    latency case (the whole filter runs in one block); one step = one filter
    run, the metric its device latency."""
    import ctypes as C

    import torch
    import gfb200 as G
    from gfb200 import _lib as L
    from gfb200 import workloads as W
    from gfb200.filtering import _pf_config
    from gfb200.plans import PfPlan
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    ctx = G.Context(local)
    N, T = 1024, 100
    model, ys = W.lgssm_1d(seed=1234, T=T)
    algo = G.BF(N, threshold=0.5, precision="f64")
    ys_dev = torch.tensor(ys, dtype=torch.float64, device=dev)
    plan = PfPlan(model, algo, T, seed=1000 + rank, ctx=ctx, graph=True)
    for _ in range(args.warmup):
        plan.run(ys_dev)
    ctx.synchronize()
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 50  # filter runs per step: one run is ~1 ms
    _barrier(world)
    with ClockSampler(local) as clk:
        e0.record(ext)
        for _ in range(args.steps * reps):
            plan.run(ys_dev)
        e1.record(ext)
        e1.synchronize()
    ms = _max_over_ranks(e0.elapsed_time(e1), world, dev) / (args.steps * reps)
    ll = float(plan.ll.item())
    plan.close()
    eplan = PfPlan(model, algo, T, seed=1000 + rank, ctx=ctx, graph=False)
    eplan.run(ys_dev)
    prof = _profiled(ctx, lambda: eplan.run(ys_dev), args.steps,
                     [(0, "propagate"), (1, "resample"), (5, "ancestor_fill"), (4, "prep_init")])
    eplan.close()
    # e2e through the C ABI from pinned host memory
    mc = model._c_struct()
    cfg, _, _ = _pf_config(algo, T, 7 + rank)
    ys_pin = torch.tensor(ys, dtype=torch.float64).pin_memory()
    ll_pin = torch.zeros(1, dtype=torch.float64).pin_memory()
    out = L.PFOutC(ll_pin.data_ptr(), None, None, None, None, None, None, None, None)
    lib = L.load()
    t_e2e = []
    for i in range(args.warmup + args.steps * 10):
        t0 = time.perf_counter()
        L.check(ctx.h, lib.gf_pf_run(ctx.h, C.byref(mc), C.byref(cfg), T, ys_pin.data_ptr(), None,
                                     None, L.GF_MEM_HOST, C.byref(out)))
        if i >= args.warmup:
            t_e2e.append(time.perf_counter() - t0)
    e2e_ms = statistics.median(t_e2e) * 1e3
    pms, pn = prof["propagate"]
    avg = pms / max(pn, 1)
    # one launch runs the whole filter in one block: per particle-step FP64 state
    # read + write, log-weight write + read / ancestor
    bytes_launch = T * N * (8 * 1 * 2 + 16)
    peak, peak_kind = _peaks()
    line = {
        "metric": "filter latency", "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "README LGSSM (x_t = x_{t-1} + N(0,0.1^2), y_t = x_t + N(0,0.2^2)), "
                               "bootstrap PF N=1024, T=100, FP64, systematic at ESS<0.5N",
                   "N": N, "T": T, "ll": ll, "runs_per_step": reps,
                   "l2": "latency case: the whole filter lives in L2"},
        "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": int(ys.nbytes),
                "d2h_bytes_per_step": 8, "call": "gf_pf_run(GF_MEM_HOST), median"},
        "gpu_launches": int(sum(v[1] for v in prof.values()) + 2 * args.steps),
        "roofline": {"bound": "hbm", "achieved": bytes_launch / (avg / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": bytes_launch / (avg / 1e3) / 1e9 / peak, "traffic": None,
                     "kernel": "pf_lg_small_filter<double,1,1> (all T steps in one block)",
                     "peak_source": peak_kind, "avg_launch_ms": avg, "bytes_per_launch": bytes_launch,
                     "note": "latency-bound: one block walks the filter's steps, each a chain of "
                             "block-wide phases"},
        "kernels_ms": {k: v[0] for k, v in prof.items()},
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        O.build()
        om = O.LGModel(model.prior.mu0, model.prior.Sigma0, model.dyn.A, model.dyn.b, model.dyn.Q,
                       model.obs.H, model.obs.c, model.obs.R)
        tt = []
        for _ in range(20):
            t0 = time.perf_counter()
            O.pf_run(om, N, ys, threshold=0.5, seed=1, threads=1)
            tt.append(time.perf_counter() - t0)
        line["cpu_baseline"] = {"value": statistics.median(tt) * 1e3, "unit": "ms", "cores": 1,
                                "kind": "port",
                                "sample": "FP64 C oracle, the whole filter (N=1024, T=100), one thread "
                                          "as the reference, median of 20"}
    ctx.close()
    return line


def bench_smooth(args, world, rank, local):
    """RTS smoother (smooth(model, KalmanSmoother(), ys)) over a bank of uneven
    LGSSMs (Dx 2..32, Dy 1..Dx, T 64..2048): forward Kalman bank plus the
    backward pass, smoothed means and covariances of every step, on a resident
    plan.  One step = one smoothing run of the whole bank."""
    import torch
    import gfb200 as G
    from gfb200 import workloads as W
    from gfb200.plans import KfPlan
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    ctx = G.Context(local)
    B = args.smooth_filters
    models, Ts, _ = W.kf_bank(B, seed=7 + rank, make_ys=False)
    plan = KfPlan(models, G.KalmanFilter(), Ts, ctx=ctx)
    ys = torch.randn(plan.n_y, dtype=torch.float64, device=dev)
    means = torch.empty(plan.n_means, dtype=torch.float32, device=dev)
    covs = torch.empty(plan.n_covs, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        plan.smooth(ys, means, covs)
    ctx.synchronize()
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    _barrier(world)
    with ClockSampler(local) as clk:
        e0.record(ext)
        for _ in range(args.steps):
            plan.smooth(ys, means, covs)
        e1.record(ext)
        e1.synchronize()
    ms = _max_over_ranks(e0.elapsed_time(e1), world, dev)
    assert int(plan.status.abs().sum().item()) == 0
    ctx.profile(True)
    plan.smooth(ys, means, covs)
    kms, kn = ctx.profile_read(2)
    ctx.profile(False)
    n_steps = plan.n_steps
    value = n_steps * args.steps * world / (ms / 1e3)
    dxs = np.array([m.dx for m in models], dtype=np.float64)
    dys = np.array([m.dy for m in models], dtype=np.float64)
    Tarr = np.array(Ts, dtype=np.float64)
    # forward outputs, then the backward pass reads them and rewrites them
    bytes_run = float(np.sum(Tarr * (8 * dys + 8 + 3 * (4 * dxs + 4 * dxs * dxs))))
    run_s = ms / 1e3 / args.steps
    peak, peak_kind = _peaks()
    line = {
        "metric": "smoothed KF-steps/s", "value": value, "unit": "KF-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"RTS smoother over {B} uneven LGSSMs, Dx~U{{2..32}}, Dy~U{{1..Dx}}, "
                               "T~U{64..2048}: forward Kalman bank + backward pass, smoothed means and "
                               "covariances of every step", "filters": B, "kf_steps": n_steps,
                   "l2": "outputs far larger than L2 (no flush)"},
        "roofline": {"bound": "hbm", "achieved": bytes_run / run_s / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": bytes_run / run_s / 1e9 / peak, "traffic": None, "peak_source": peak_kind},
        "gpu_launches": int(kn),
        "kernel_ms_per_run": kms,
        "clocks": clk.summary(),
    }
    plan.close()
    ctx.close()
    return line


def bench_kfgrad(args, world, rank, local):
    """Gradients of kf_loglikelihood (the ChainRules pullback) for a bank of
    uneven LGSSMs (Dx 2..16, Dy 1..Dx, T 64..512), FP64: one step = forward
    filter with checkpoints plus the backward gradient recursion of every
    model (gf_kf_loglikelihood_grad on device buffers)."""
    import ctypes as C

    import torch
    import gfb200 as G
    from gfb200 import _lib as L
    from gfb200 import workloads as W
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    ctx = G.Context(local)
    lib = L.load()
    B = args.kfgrad_models
    models, Ts, yss = W.kf_bank(B, seed=11 + rank, dx_range=(2, 16), T_range=(64, 512))
    mcs = (L.LGModelC * B)(*[m._c_struct() for m in models])
    Ta = np.array(Ts, np.int32)
    ys_h = np.concatenate([np.asarray(y, np.float64).ravel() for y in yss])
    yd = torch.tensor(ys_h, device=dev)
    dxs = np.array([m.dx for m in models])
    dys = np.array([m.dy for m in models])
    sizes = [B, dxs.sum(), (dxs * dxs).sum(), (dxs * dxs).sum(), dxs.sum(), (dxs * dxs).sum(),
             (dys * dxs).sum(), dys.sum(), (dys * dys).sum()]
    outs = [torch.empty(int(n), dtype=torch.float64, device=dev) for n in sizes]
    status = torch.zeros(B, dtype=torch.int32, device=dev)
    o = L.KFGradOutC(*[L.ptr(t) for t in outs], L.ptr(status))

    def run():
        L.check(ctx.h, lib.gf_kf_loglikelihood_grad(ctx.h, mcs, B, Ta.ctypes.data_as(C.POINTER(C.c_int32)),
                                                    L.ptr(yd), 0.0, 0, L.GF_MEM_DEVICE, C.byref(o)))

    for _ in range(args.warmup):
        run()
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    _barrier(world)
    with ClockSampler(local) as clk:
        e0.record(ext)
        for _ in range(args.steps):
            run()
        e1.record(ext)
        e1.synchronize()
    ms = _max_over_ranks(e0.elapsed_time(e1), world, dev)
    assert int(status.abs().sum().item()) == 0
    n_steps = int(np.sum(Ts))
    value = n_steps * args.steps * world / (ms / 1e3)
    # end to end through the public API with host buffers
    t0 = time.perf_counter()
    for _ in range(args.steps):
        G.kf_loglikelihood_grad_batch(models, yss, ctx=ctx)
    e2e_s = time.perf_counter() - t0
    Tarr = np.array(Ts, dtype=np.float64)
    # checkpoint write + read (8 (dx + dx^2) each) and y read (8 dy) per step
    bytes_run = float(np.sum(Tarr * (16 * (dxs + dxs * dxs) + 8 * dys)))
    run_s = ms / 1e3 / args.steps
    peak, peak_kind = _peaks()
    line = {
        "metric": "KF gradient steps/s", "value": value, "unit": "KF-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"kf_loglikelihood pullback over {B} uneven LGSSMs, Dx~U{{2..16}}, "
                               "Dy~U{1..Dx}, T~U{64..512}: FP64 forward with checkpoints + backward "
                               "gradient recursion, gradients of mu0, Sigma0, A, b, Q, H, c, R",
                   "models": B, "kf_steps": n_steps, "l2": "no flush (latency-bound)"},
        "roofline": {"bound": "hbm", "achieved": bytes_run / run_s / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": bytes_run / run_s / 1e9 / peak, "traffic": None, "peak_source": peak_kind,
                     "limiter": "serial FP64 per-step chain of each model (one CTA per model)"},
        "e2e": {"value": n_steps * args.steps / e2e_s, "unit": "KF-steps/s",
                "h2d_bytes_per_step": int(ys_h.nbytes), "d2h_bytes_per_step": int(sum(n * 8 for n in sizes))},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_kfgrad(models, yss, seconds=args.cpu_seconds)
    ctx.close()
    return line


def cpu_baseline_kfgrad(models, yss, seconds=12.0):
    """The FP64 oracle's pullback (numpy, one core) over the bank's models in
    order until `seconds` have passed."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    steps, done = 0, 0
    t0 = time.perf_counter()
    for m, ys in zip(models, yss):
        p, d, o = m.prior, m.dyn, m.obs
        O.kf_loglikelihood_grad(O.LGModel(p.mu0, p.Sigma0, d.A, d.b, d.Q, o.H, o.c, o.R), ys)
        steps += len(ys)
        done += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": steps / dt, "unit": "KF-steps/s", "cores": 1, "kind": "port",
            "sample": f"FP64 numpy oracle pullback, the first {done} models of the bank ({steps} KF steps)"}


def cpu_baseline_csmc(model, ys, N, seconds=12.0, threads=None):
    """The FP64 oracle's CSMC-AS on this host: same model and N, chains spread
    over all host threads, a bounded number of sweeps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    threads = threads or os.cpu_count() or 1
    p, d, o = model.prior, model.dyn, model.obs
    om = O.LGModel(p.mu0, p.Sigma0, d.A, d.b, d.Q, o.H, o.c, o.R)
    T = len(ys)
    t0 = time.perf_counter()
    O.csmc_run(om, N, ys, threshold=0.6, refresh=O.CSMC_ANCESTOR, chains=threads, iters=1, seed=1,
               threads=threads)
    one = time.perf_counter() - t0
    iters = int(max(1, seconds / max(one, 1e-4)))
    t0 = time.perf_counter()
    O.csmc_run(om, N, ys, threshold=0.6, refresh=O.CSMC_ANCESTOR, chains=threads, iters=iters,
               seed=1, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": threads * iters * T * N / dt, "unit": "particle-steps/s", "cores": threads,
            "kind": "port",
            "sample": f"FP64 C oracle CSMC-AS, same model and N={N}, T={T}, {threads} chains x "
                      f"{iters} sweeps, {threads} OpenMP threads (one chain per thread)"}


def bench_csmc(args, world, rank, local):
    """Particle Gibbs: ConditionalSMC(BF(256; threshold=0.6), AncestorSampling())
    on an LGSSM Dx=4, Dy=2, K=100.  One step = `--csmc-sweeps` conditional SMC
    sweeps of each of `--csmc-chains` chains (one CTA per chain, a whole chain
    per launch), each chain continuing from its previous step's reference."""
    import ctypes as C

    import torch
    import gfb200 as G
    from gfb200 import _lib as L
    from gfb200 import csmc as CS
    from gfb200 import workloads as W
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    ctx = G.Context(local)
    lib = L.load()
    K, N, dx = 100, 256, 4
    chains, sweeps = args.csmc_chains, args.csmc_sweeps
    model, ys = W.lgssm_rot(seed=1234 + rank, dx=dx, dy=2, T=K)
    yd = torch.tensor(ys, dtype=torch.float64, device=dev)
    traj = torch.empty((chains, sweeps, K + 1, dx), dtype=torch.float64, device=dev)
    lls = torch.empty((chains, sweeps), dtype=torch.float64, device=dev)
    ref = torch.zeros((chains, K + 1, dx), dtype=torch.float64, device=dev)
    status = torch.zeros(chains, dtype=torch.int32, device=dev)
    cfg = L.CsmcConfigC(N, 0.6, L.GF_RS_SYSTEMATIC, L.GF_CSMC_ANCESTOR, 0)
    out = L.CsmcOutC(L.ptr(traj), L.ptr(lls), L.ptr(ref), L.ptr(status))
    mc = model._c_struct()

    def run(i):
        cfg.seed = 1000 + i
        L.check(ctx.h, lib.gf_csmc_run(ctx.h, C.byref(mc), C.byref(cfg), K, L.ptr(yd), chains, sweeps, 0,
                                       int(i > 0), None, None, L.GF_MEM_DEVICE, C.byref(out)))

    for i in range(args.warmup):
        run(i)
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    _barrier(world)
    with ClockSampler(local) as clk:
        e0.record(ext)
        for i in range(args.steps):
            run(args.warmup + i)
        e1.record(ext)
        e1.synchronize()
    ms = _max_over_ranks(e0.elapsed_time(e1), world, dev)
    assert int(status.abs().sum().item()) == 0
    psteps = chains * sweeps * K * N
    value = psteps * args.steps * world / (ms / 1e3)
    # end to end: the public API with host buffers (ys in, every kept trajectory
    # and log-likelihood out), continuing the chains from the device references
    last = ref.cpu().numpy()
    cm = G.CSMCModel(model, ys)
    csmc = G.ConditionalSMC(G.BF(N, threshold=0.6), G.AncestorSampling())
    CS.sample(cm, csmc, sweeps, chains=chains, seed=7, initial=last, ctx=ctx)
    t0 = time.perf_counter()
    for i in range(args.steps):
        _, _, last = CS.sample(cm, csmc, sweeps, chains=chains, seed=8 + i, initial=last, ctx=ctx)
    e2e_s = time.perf_counter() - t0
    h2d = ys.nbytes + last.nbytes
    d2h = chains * sweeps * (K + 1) * dx * 8 + chains * sweeps * 8 + last.nbytes
    # algorithmic bytes per particle-step: state write + gathered read (16 dx),
    # log-weight write + read (16), ancestor write (4)
    b_ps = 16 * dx + 20
    run_s = ms / 1e3 / args.steps
    peak, peak_kind = _peaks()
    line = {
        "metric": "CSMC particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"particle Gibbs: ConditionalSMC(BF({N}; threshold=0.6), AncestorSampling()) "
                               f"on LGSSM Dx={dx} Dy=2 K={K}; {chains} chains x {sweeps} sweeps per step, "
                               "one CTA per chain", "chains": chains, "sweeps_per_step": sweeps,
                   "sweeps_per_s": chains * sweeps * args.steps * world / (ms / 1e3),
                   "l2": "per-chain histories (1 MB each) stay in L2 between steps; no flush"},
        "roofline": {"bound": "hbm", "achieved": psteps * b_ps / run_s / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": psteps * b_ps / run_s / 1e9 / peak, "traffic": None, "peak_source": peak_kind,
                     "limiter": "per-step CTA barriers of each chain (latency); 4 chains per SM"},
        "e2e": {"value": psteps * args.steps / e2e_s, "unit": "particle-steps/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_csmc(model, ys, N, seconds=args.cpu_seconds)
    ctx.close()
    return line


def bench_reference(args, world, rank, local):
    """The reference arm: the FP64 oracle port of the reference algorithm on the
    host cores (the reference is Julia and cannot run on this image)."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from gfb200 import workloads as W
    N, T = 2**20, 1000
    model, ys = W.lgssm_rot(seed=1234, dx=16, dy=8, T=T)
    vals = []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline_pf(model, ys, N, seconds=args.cpu_seconds)
        if i >= args.warmup:
            vals.append(cb["value"])
    v = statistics.median(vals)
    cb["value"] = v
    return {"impl": "reference", "metric": "particle-steps/s", "value": v,
            "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "bootstrap PF, LGSSM Dx=16 Dy=8, N=2^20, T=1000 (bounded "
                                   "sample of time steps per step), systematic at ESS<0.5N"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pf", choices=["pf", "pf1d", "kf", "smooth", "rbpf", "serve", "csmc", "kfgrad"])
    ap.add_argument("--kfgrad-models", type=int, default=8192)
    ap.add_argument("--csmc-chains", type=int, default=592)
    ap.add_argument("--csmc-sweeps", type=int, default=20)
    ap.add_argument("--smooth-filters", type=int, default=16384)
    ap.add_argument("--serve-rate", type=float, default=1000.0)
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-hbm-gb", type=int, default=64)
    ap.add_argument("--kf-filters", type=int, default=65536)
    ap.add_argument("--kf-algo", default="kf", choices=["kf", "srkf"])
    ap.add_argument("--pf-T", type=int, default=1000,
                    help="time steps of the PF workload (smaller only for profiler captures)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the accuracy block of the PF line (profiler captures)")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the KF-bank and serving entries of the PF line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = _dist_setup(args)
    if world > 1 and args.impl == "ours":
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        line = bench_reference(args, world, rank, local)
    elif args.workload == "kf":
        line = bench_kf(args, world, rank, local)
    elif args.workload == "serve":
        line = bench_serve(args, world, rank, local)
    elif args.workload == "smooth":
        line = bench_smooth(args, world, rank, local)
    elif args.workload == "rbpf":
        line = bench_rbpf(args, world, rank, local)
    elif args.workload == "pf1d":
        line = bench_pf1d(args, world, rank, local)
    elif args.workload == "csmc":
        line = bench_csmc(args, world, rank, local)
    elif args.workload == "kfgrad":
        line = bench_kfgrad(args, world, rank, local)
    else:
        line = bench_pf(args, world, rank, local)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if world > 1 and args.impl == "ours":
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
