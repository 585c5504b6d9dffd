#!/usr/bin/env python
"""Benchmark: MRA log-likelihood evaluations per second on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c3] [--precision fp64|mixed]
    python bench.py --impl reference ...      # the reference's own CPU code on this host

A step is one exact log-likelihood evaluation (prior + posterior pass over the
whole partition tree) of a seeded synthetic configuration, with the partition,
observations and all working buffers resident in HBM.  ``value`` is timed on the
device with CUDA events recorded on the library's own stream; ``e2e`` times the
same evaluation through the C ABI with the step's inputs (observation values y
and theta) copied from pinned host memory and the result read back, every step.
The multi-GPU form runs independent replicas (the path is not sharded: one
likelihood evaluation fits one GPU), one process per GPU.

Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MRA loglik evals/sec at n=1M (mixed vs plain FP64, same GPU, ≤1e-6 rel err); fit wall-time"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
# per-launch DRAM traffic of the dominant kernels, from ncu captures (see the file)
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "dram_traffic.md")


def traffic_lookup(key: str):
    """Bytes per launch for `config:precision:kernel:level` from the table rows
    "| key | bytes | ... |" of profiles/dram_traffic.md, else None."""
    if not os.path.exists(TRAFFIC_FILE):
        return None
    for line in open(TRAFFIC_FILE):
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if len(cells) >= 2 and cells[0] == key:
            try:
                return float(cells[1])
            except ValueError:
                return None
    return None
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "mra_ref_ext")


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--config", default="c3", choices=["c1", "c2", "c2s", "c3"])
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-graph", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-autotune", action="store_true")
    p.add_argument("--fit", action="store_true",
                   help="instead of the log-likelihood line: fit wall-time of the plain optimizer vs the "
                        "surrogate-assisted one (19 nonstationary parameters, c2 layout)")
    p.add_argument("--fit-evals", type=int, default=2000)
    p.add_argument("--fit-curve", action="store_true",
                   help="with --fit: the best log-likelihood against exact evaluations and wall time of the plain "
                        "optimizer and of the surrogate-assisted one for several training-set sizes")
    p.add_argument("--fit-ntrain", default="100,200,400", help="training-set sizes of --fit-curve")
    p.add_argument("--sweep", action="store_true",
                   help="instead of the log-likelihood line: the scaling sweep n in {1M, 2M, 4M} x M in "
                        "{10, 11, 12} x r in {32, 64, 128} (one JSON line per case)")
    p.add_argument("--predict", action="store_true",
                   help="instead of the log-likelihood line: prediction throughput on the workload with its "
                        "prediction points (log-likelihood with the predictive factors kept, then prediction)")
    p.add_argument("--mixed-report", action="store_true",
                   help="instead of the log-likelihood line: the mixed path against the FP64 path on the same "
                        "inputs, per stage (device time of each launch, error of each part of d), with the "
                        "observed values and with y = 0 (log-determinants alone)")
    p.add_argument("--shard", action="store_true",
                   help="with N ranks: one log-likelihood per step split over the ranks by sub-trees "
                        "(strong scaling; shard.py) instead of N independent replicas")
    p.add_argument("--surrogate-forward", action="store_true",
                   help="instead of the log-likelihood line: the surrogate network's prediction on 65,536 "
                        "parameter vectors, values only (tcgen05 kernel) and with input gradients (FP32 cores)")
    p.add_argument("--no-compare", action="store_true",
                   help="skip timing the other precision on the same inputs")
    return p.parse_args()


def workload_name(cfg) -> str:
    layout = {"uniform": "uniform", "mix70": "70% in 16 clusters + 30% uniform",
              "mix10": "90% uniform + 10% in 16 clusters"}[cfg.layout]
    return (f"{cfg.name}: n={cfg.n} locations on [0,1]^2 ({layout}), M={cfg.M}, J={cfg.J}, r={cfg.r}, "
            f"nonstationary Matern nu={cfg.nu_x2}/2 with 9-RBF log-sigma/log-range fields")


# ---------------------------------------------------------------------------
# data
# ---------------------------------------------------------------------------
def make_problem(cfg, with_pred=False):
    from nonstationary_mra_b200 import partition, synth
    rng = np.random.Generator(np.random.PCG64(cfg.seed))
    xy, pred = synth.locations(cfg, rng)
    theta = synth.true_theta(cfg, rng)
    md = synth.model_from_theta(theta, cfg.nu_x2)
    st = partition.build_by_program(xy[0], xy[1], np.zeros(cfg.n), cfg.J, cfg.M, cfg.r, math.exp(1) / 100,
                                    pred[0] if with_pred else None, pred[1] if with_pred else None,
                                    distance=2, all_lon=xy[0], all_lat=xy[1])
    return xy, pred, theta, md, st


def draw_values(ctx, st, seed):
    """y from the MRA prior at the true parameters (standard normals from PCG64)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    z_int = rng.standard_normal(st.n_interior * st.r)
    z_obs = rng.standard_normal(st.n_obs)
    ctx.set_theta()
    return ctx.sample_prior(z_int, z_obs)


# ---------------------------------------------------------------------------
# measurement helpers
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit()) if rows else None}


def fp64_peak_tflops():
    """cuBLAS DGEMM throughput (torch.matmul in float64), best of 5 at 8192^3."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    best = 0.0
    for _ in range(6):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def measured_peaks():
    try:
        return json.load(open(PEAKS_FILE))
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own code (oracle/_ref, built from its sources)
# ---------------------------------------------------------------------------
# Workloads whose reference layout fits in host memory are timed whole (c2: about
# 15 GB of finest-level A~).  At c3 the reference would hold about 386 GB of A~,
# so it cannot run; it is reported as unavailable, with a labelled estimate from
# two smaller samples of the same generator scaled by algorithmic FLOPs.
REF_RUNS_WHOLE = ("c1", "c2s", "c2")


def cpu_sample_config(cfg, shrink_levels):
    """Same generator and model with 4^k times fewer points and the tree k levels
    shallower (same mean number of observations per finest region)."""
    from nonstationary_mra_b200 import synth
    return synth.Config(f"{cfg.name}-sample{shrink_levels}", cfg.n >> (2 * shrink_levels), cfg.M - shrink_levels,
                        cfg.J, cfg.r, cfg.nu_x2, 0, cfg.layout, cfg.range_sd, cfg.seed + 1000 + shrink_levels)


def canonical_flops(st):
    """Algorithmic FLOPs of one log-likelihood (same count as the library's plan)."""
    J, M, R = st.J, st.M, float(st.r)
    total = 0.0
    for m in range(M - 1):
        cnt = float(J ** m)
        total += 2 * cnt * R ** 3 * (m * (m - 1) / 2 + m + 1.0 / 6)
        total += 2 * cnt * (R ** 3 * (1.0 / 3 + m + m * (m - 1) / 2) + R * R * (0.5 + m))
    Lv = M - 1
    n = np.diff(st.obs_offset).astype(np.float64)
    n = n[n > 0]
    total += 2 * np.sum(R * R * n * Lv * (Lv - 1) / 2 + Lv * R * R * n / 2 + Lv * R * n * n / 2 + n ** 3 / 6 +
                        n * n / 2 + Lv * n * n * R / 2 + Lv * R * n + Lv * R * R * n / 2 +
                        Lv * (Lv - 1) / 2 * R * R * n)
    return float(total)


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def time_reference(cfg, reps):
    """Approximation::likelihood() of the reference on the whole workload ``cfg``
    (the partition is built once, outside the timed calls; each call on a fresh
    Approximation as the reference's optimizer does), all host threads with
    OpenBLAS single-threaded inside OpenMP.  Observation values come from
    synth.smooth_values (the reference's work does not depend on them).  Falls
    back to the numpy restatement of the oracle, single-threaded, when the
    reference binary is absent.  Returns (seconds per call, kind, cores, n_obs, FLOPs)."""
    from nonstationary_mra_b200 import refio, synth
    xy, _, theta, md, st = make_problem(cfg)
    flops = canonical_flops(st)
    y = synth.smooth_values(xy, theta, cfg.seed + 500)
    cores = os.cpu_count() or 1
    tmp = tempfile.mkdtemp(prefix="mra_cpu_")
    try:
        synth.write_case(tmp, cfg, xy, y, np.zeros((2, 0)), theta)
        if os.path.exists(REF_BIN):
            X = refio.parse_parameters(os.path.join(tmp, "ext_parameters"))
            env = dict(os.environ, OMP_NUM_THREADS=str(cores), OPENBLAS_NUM_THREADS="1",
                       **{k: str(v) for k, v in X.items()})
            res = subprocess.run([REF_BIN, "--reps", str(reps)], cwd=tmp, env=env, capture_output=True,
                                 text=True, timeout=3600)
            if res.returncode != 0:
                raise RuntimeError(res.stdout[-1000:] + res.stderr[-1000:])
            secs = [float(tok.split("=")[1]) for line in res.stdout.splitlines() if line.startswith("ORACLE rep=")
                    for tok in line.split() if tok.startswith("likelihood_seconds=")]
            kind, used = "reference", cores
        else:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import mra_oracle as oracle
            ost, omd, _ = oracle.load_case(tmp, mode="likelihood")
            secs = []
            for _ in range(reps):
                t0 = time.perf_counter()
                oracle.loglik(ost, omd)
                secs.append(time.perf_counter() - t0)
            kind, used = "port", 1
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return secs, kind, used, st.n_obs, flops


def reference_estimate(cfg, reps=3):
    """For a workload the reference cannot hold: the FLOP-scaled projection from a
    sample 64x smaller (three levels shallower), and the same projection from a
    sample 256x smaller as a check of the scaling (the two should agree)."""
    _, _, _, _, st_full = make_problem(cfg)
    f_full = canonical_flops(st_full)
    out = {}
    for k in (4, 3):
        sc = cpu_sample_config(cfg, k)
        secs, kind, cores, n_obs, f = time_reference(sc, reps + 1)
        t = statistics.median(secs[1:])
        out[k] = {"points": sc.n, "M": sc.M, "seconds": t, "flops": f, "evals_per_s_scaled": f / (f_full * t)}
    a, b = out[4], out[3]
    return {"value": b["evals_per_s_scaled"], "unit": "evals/s", "kind": kind, "cores": cores,
            "method": (f"likelihood() of a {b['points']}-point M={b['M']} sample of the same generator "
                       f"(median {b['seconds']:.3f} s) scaled by algorithmic FLOPs ({f_full:.3e} / {b['flops']:.3e})"),
            "scaling_check": {"sample_points": [a["points"], b["points"]], "sample_M": [a["M"], b["M"]],
                              "seconds": [a["seconds"], b["seconds"]], "flops": [a["flops"], b["flops"]],
                              "time_ratio": b["seconds"] / a["seconds"], "flop_ratio": b["flops"] / a["flops"]},
            "cpu": cpu_model()}


def cpu_baseline_for(cfg, reps):
    """cpu_baseline object of the line: the whole workload where the reference
    fits in host memory, else the labelled FLOP-scaled estimate."""
    if cfg.name in REF_RUNS_WHOLE:
        secs, kind, cores, n_obs, _ = time_reference(cfg, reps + 1)
        t = statistics.median(secs[1:]) if len(secs) > 1 else secs[0]
        return {"value": 1.0 / t, "unit": "evals/s", "cores": cores, "kind": kind, "same_config": True,
                "cpu": cpu_model(),
                "sample": (f"the whole {cfg.name} workload ({n_obs} observations): median of {len(secs) - 1} "
                           f"likelihood() calls after one untimed call = {t:.3f} s")}
    est = reference_estimate(cfg)
    return {"value": est["value"], "unit": "evals/s", "cores": est["cores"], "kind": est["kind"],
            "same_config": False, "cpu": est["cpu"], "estimate": True,
            "sample": ("ESTIMATE: the reference cannot hold this workload (about 386 GB of finest-level A~ "
                       "in its layout); " + est["method"]), "scaling_check": est["scaling_check"]}


def reference_arm(args):
    from nonstationary_mra_b200 import synth
    cfg = synth.CONFIGS[args.config]
    base = {"metric": METRIC, "unit": "evals/s", "n_gpus": args.gpus, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": workload_name(cfg), "parallelism": "cpu"}}
    if cfg.name not in REF_RUNS_WHOLE:
        est = reference_estimate(cfg)
        line = dict(base, value=None, steps=0, warmup=0, ms_per_step=None,
                    unavailable=(f"the reference's layout needs about 386 GB of host memory for the finest-level "
                                 f"A~ at {cfg.name} and one likelihood() would take minutes; "
                                 f"see 'estimate' and 'bench.py --config c2 --impl reference' for a measured "
                                 f"same-config comparison"),
                    estimate=est,
                    cpu_baseline={"value": None, "unit": "evals/s", "cores": est["cores"], "kind": est["kind"],
                                  "sample": "not run: " + est["method"]},
                    e2e={"value": None, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        print(json.dumps(line))
        return
    steps, warmup = max(args.steps, 1), max(args.warmup, 0)
    secs, kind, cores, n_obs, _ = time_reference(cfg, steps + warmup)
    secs = secs[warmup:]
    t = statistics.median(secs)
    value = 1.0 / t
    line = dict(base, value=value, steps=len(secs), warmup=warmup, ms_per_step=1000.0 * t,
                cpu_baseline={"value": value, "unit": "evals/s", "cores": cores, "kind": kind, "same_config": True,
                              "cpu": cpu_model(),
                              "sample": (f"the whole {cfg.name} workload ({n_obs} observations), one likelihood() "
                                         f"per step; median of {len(secs)}")},
                e2e={"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    line["config"]["seconds_per_step"] = secs
    print(json.dumps(line))


def fit_curve_arm(args):
    """The surrogate's effect, measured: the best exact log-likelihood reached
    after k exact evaluations (and the wall time), for the plain optimizer and
    for the surrogate-assisted optimizer trained on its first n_train
    evaluations, n_train from --fit-ntrain; the same seeded start and bounds as
    --fit."""
    from nonstationary_mra_b200 import api, synth
    from nonstationary_mra_b200.fit import FitConfig, NonstationaryObjective, fit_plain, fit_surrogate
    cfg = synth.CONFIGS["c2" if args.config == "c3" else args.config]
    xy, pred, theta, md, st = make_problem(cfg)
    ctx = api.Context(st, md)
    y = draw_values(ctx, st, cfg.seed + 7)
    ctx.set_obs_values(y)
    ctx.set_theta()
    ctx.capture_graph()
    rng = np.random.Generator(np.random.PCG64(cfg.seed + 11))
    th0 = np.concatenate([0.3 * rng.standard_normal(9), cfg.range_sd * rng.standard_normal(9), [np.log(0.1)]])
    lo = np.concatenate([-2.5 * np.ones(18), [np.log(1e-3)]])
    hi = np.concatenate([2.5 * np.ones(18), [0.0]])
    icpt = (0.0, float(np.log(0.1)))
    marks = [k for k in (50, 100, 200, 300, 400, 500, 750, 1000, 1250, 1500, 1750, 2000, 2500, 3000)
             if k <= args.fit_evals]

    def curve(trace):
        best = np.maximum.accumulate(np.asarray(trace.loglik))
        return {str(k): {"loglik": float(best[k - 1]), "seconds": float(trace.seconds[k - 1])}
                for k in marks if k <= len(best)}

    plain = NonstationaryObjective(ctx, *icpt)
    fit_plain(plain, th0, lo, hi, FitConfig(max_evals=args.fit_evals))
    L = plain.trace.best_loglik()
    target = L - 1e-6 * abs(L)
    out = {"metric": "surrogate-assisted fitting: best exact loglik vs exact evaluations",
           "workload": workload_name(cfg) + ", theta = 9 log-sigma + 9 log-range + log tau^2",
           "seconds_per_eval": float(np.median(np.diff(plain.trace.seconds))),
           "plain": {"final_loglik": L, "evals": len(plain.trace.loglik), "curve": curve(plain.trace),
                     "evals_to_final": plain.trace.evals_to_reach(target)}}
    for nt in [int(v) for v in args.fit_ntrain.split(",") if v]:
        sur = NonstationaryObjective(ctx, *icpt)
        _, Ls, info = fit_surrogate(sur, th0, lo, hi, FitConfig(max_evals=args.fit_evals, n_train=nt))
        out[f"surrogate_ntrain{nt}"] = {"final_loglik": Ls, "evals": info["evals"], "proposals": info["proposals"],
                                        "accepted": info["accepted"], "curve": curve(sur.trace),
                                        "evals_to_plain_final": sur.trace.evals_to_reach(target),
                                        "seconds_to_plain_final": sur.trace.time_to_reach(target)}
    ctx.close()
    print(json.dumps(out))


def fit_arm(args):
    """Surrogate-assisted fitting vs the plain optimizer from the same seeded
    theta0 on the exact GPU log-likelihood: wall time of each to reach the
    plain optimizer's final log-likelihood (within 1e-6 relative)."""
    from nonstationary_mra_b200 import api, synth
    from nonstationary_mra_b200.fit import FitConfig, NonstationaryObjective, fit_plain, fit_surrogate
    cfg = synth.CONFIGS["c2" if args.config == "c3" else args.config]
    xy, pred, theta, md, st = make_problem(cfg)
    ctx = api.Context(st, md)
    y = draw_values(ctx, st, cfg.seed + 7)
    ctx.set_obs_values(y)
    ctx.set_theta()
    ctx.capture_graph()
    rng = np.random.Generator(np.random.PCG64(cfg.seed + 11))
    th0 = np.concatenate([0.3 * rng.standard_normal(9), cfg.range_sd * rng.standard_normal(9), [np.log(0.1)]])
    lo = np.concatenate([-2.5 * np.ones(18), [np.log(1e-3)]])
    hi = np.concatenate([2.5 * np.ones(18), [0.0]])
    icpt = (0.0, float(np.log(0.1)))
    fc = FitConfig(max_evals=args.fit_evals)
    plain = NonstationaryObjective(ctx, *icpt)
    t = time.perf_counter()
    fit_plain(plain, th0, lo, hi, fc)
    t_plain = time.perf_counter() - t
    L = plain.trace.best_loglik()
    target = L - 1e-6 * abs(L)
    sur = NonstationaryObjective(ctx, *icpt)
    t = time.perf_counter()
    _, L_sur, info = fit_surrogate(sur, th0, lo, hi, fc)
    t_sur = time.perf_counter() - t
    ctx.close()
    reach = sur.trace.time_to_reach(target)
    line = {"metric": "fit wall-time to the plain optimizer's final loglik (within 1e-6 relative)",
            "value": reach, "unit": "s", "higher_is_better": False,
            "config": {"workload": workload_name(cfg) + ", theta = 9 log-sigma + 9 log-range + log tau^2",
                       "max_evals": args.fit_evals, "n_train": fc.n_train},
            "plain": {"seconds": t_plain, "evals": len(plain.trace.loglik), "loglik": L},
            "surrogate": {"seconds": t_sur, "evals": info["evals"], "loglik": L_sur,
                          "proposals": info["proposals"], "accepted": info["accepted"],
                          "seconds_to_plain_final": reach,
                          "evals_to_plain_final": sur.trace.evals_to_reach(target)},
            "ratio_to_plain": (reach / t_plain) if reach else None}
    print(json.dumps(line))


def sweep_arm(args):
    """Scaling sweep (uniform locations, nu = 1/2, J = 4, 4 observations per finest
    region): per case the FP64 log-likelihood and log-likelihood + prediction
    (16,384 points) times, the device memory high-water and the dominant
    launch's FP64 tensor throughput; cases that do not fit in device memory are
    reported as such (the library's allocation fails cleanly)."""
    import torch
    from nonstationary_mra_b200 import api, capi, synth
    cases = [(1 << 20, 10), (1 << 21, 11), (1 << 22, 12)]
    peak = fp64_peak_tflops()
    for n, M in cases:
        for r in (32, 64, 128):
            cfg = synth.Config(f"sweep-{n}-{M}-{r}", n, M, 4, r, 1, 16384, "uniform", 0.3, 5)
            line = {"metric": "MRA loglik evals/sec (scaling sweep)", "unit": "evals/s", "n": n, "M": M, "r": r,
                    "workload": workload_name(cfg)}
            with_pred = True
            try:
                xy, pred, theta, md, st = make_problem(cfg, with_pred=True)
                ctx = api.Context(st, md)
            except capi.MRAError:
                # the prediction buffers (G is as large as U) may not fit where the
                # log-likelihood alone does
                torch.cuda.empty_cache()
                with_pred = False
                try:
                    xy, pred, theta, md, st = make_problem(cfg, with_pred=False)
                    ctx = api.Context(st, md)
                    line.update(note="prediction buffers do not fit: log-likelihood only")
                except capi.MRAError as exc:
                    line.update(value=None, infeasible=str(exc)[:200])
                    print(json.dumps(line), flush=True)
                    continue
            try:
                y = draw_values(ctx, st, cfg.seed + 7)
                ctx.set_obs_values(y)
                ctx.set_theta()
                for _ in range(max(args.warmup, 1)):
                    ctx.loglik()
                ctx.capture_graph()
                ctx.loglik()
                steps = max(args.steps, 1)
                ctx.timer_start()
                for _ in range(steps):
                    _, ll = ctx.loglik()
                ms = ctx.timer_stop() / steps
                stats = ctx.stats()
                dom = max(stats["launches"], key=lambda l: l["ms"])
                ms_pred = None
                if with_pred:
                    ctx.predict()
                    ctx.timer_start()
                    ctx.predict()
                    ms_pred = ctx.timer_stop()
                line.update(value=1000.0 / ms, ms_per_eval=ms, loglik=ll, flop_per_eval=stats["flop_last"],
                            predict_ms=ms_pred, predictions=int(st.n_pred) if with_pred else 0,
                            device_gb=stats["bytes_device"] / 1e9,
                            dominant=f"{dom['kernel']}(level {dom['level']})",
                            dominant_tflops=dom["flop"] / (dom["ms"] * 1e-3) / 1e12, fp64_peak_tflops=peak)
            except capi.MRAError as exc:
                line.update(value=None, failed=str(exc)[:200])
            finally:
                ctx.close()
                torch.cuda.empty_cache()
            print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def predict_arm(args):
    """Prediction throughput: the workload's prediction points resident with the
    tree; one step = log-likelihood with the predictive factors kept + the
    prediction of every point (the reference's likelihood() + predict()),
    replayed from one captured CUDA graph.  Reports predictions/s of the whole
    step and of the prediction launch alone (CUDA events on the library's
    stream), and the other precision on the same inputs with its error per
    output against the FP64 path."""
    from nonstationary_mra_b200 import api, capi, synth
    cfg = synth.CONFIGS[args.config]
    line = {"metric": "MRA predictions/sec (likelihood + predict)", "unit": "predictions/s",
            "workload": workload_name(cfg), "n_pred": cfg.n_pred, "precision": args.precision,
            "cuda_graph": not args.no_graph}
    try:
        xy, pred, theta, md, st = make_problem(cfg, with_pred=True)
    except capi.MRAError as exc:
        line.update(value=None, infeasible=str(exc)[:200])
        print(json.dumps(line), flush=True)
        return
    y = None

    def run(precision):
        nonlocal y
        ctx = api.Context(st, md, precision=precision)
        try:
            if y is None:
                y = draw_values(ctx, st, cfg.seed + 7)
            ctx.set_obs_values(y)
            ctx.set_theta()
            for _ in range(max(args.warmup, 1)):
                ctx.predict()
            if not args.no_graph:
                ctx.capture_graph()
                ctx.predict()
            steps = max(args.steps, 1)
            ctx.timer_start()
            for _ in range(steps):
                mean, var = ctx.predict()
            ms = ctx.timer_stop() / steps
            stats = ctx.stats()
            ms_kernel = sum(l["ms"] for l in stats["launches"] if l["kernel"] == "predict")
            return {"ms": ms, "ms_kernel": ms_kernel, "mean": mean, "var": var, "gb": stats["bytes_device"] / 1e9,
                    "steps": steps}
        finally:
            ctx.close()

    try:
        a = run(args.precision)
        line.update(value=st.n_pred / (a["ms"] * 1e-3), ms_per_step=a["ms"], predict_launch_ms=a["ms_kernel"],
                    predict_launch_per_s=st.n_pred / (a["ms_kernel"] * 1e-3) if a["ms_kernel"] > 0 else None,
                    device_gb=a["gb"], mean_abs=float(np.mean(np.abs(a["mean"]))), steps=a["steps"],
                    warmup=args.warmup)
        if not args.no_compare:
            oprec = "mixed" if args.precision == "fp64" else "fp64"
            b = run(oprec)
            f64, mix = (a, b) if args.precision == "fp64" else (b, a)
            err = lambda u, v: float(np.max(np.abs(u - v) / np.maximum(1.0, np.abs(v))))
            line["other_precision"] = {
                "precision": oprec, "ms_per_step": b["ms"], "predict_launch_ms": b["ms_kernel"],
                "mixed_err_vs_fp64": {"mean": err(mix["mean"], f64["mean"]), "var": err(mix["var"], f64["var"])},
                "mixed_speedup_vs_fp64": f64["ms"] / mix["ms"]}
    except capi.MRAError as exc:
        line.update(value=None, failed=str(exc)[:200])
    print(json.dumps(line), flush=True)


def mixed_report_arm(args):
    """Attribution of the mixed path's error and time, stage by stage, on the
    device.  Every variant evaluates the same tree and values: FP64, the mixed
    path (prior levels and finest level in FP32, posterior FP64), and the mixed
    path with only the prior levels or only the finest level in FP32
    (MRA_MIXED_FP32).  For each: the device time of every launch and the error of
    d and of the log-likelihood against FP64, with the observed values and with
    y = 0, where d is the log-determinants alone (separating them from the
    quadratic forms); and the error of every part of d (mra_get_terms)."""
    from nonstationary_mra_b200 import api, synth
    cfg = synth.CONFIGS[args.config]
    xy, pred, theta, md, st = make_problem(cfg)
    out = {"metric": "mixed-path attribution", "workload": workload_name(cfg), "M": cfg.M}
    variants = [("fp64", "fp64", None), ("mixed", "mixed", "prior,finest"), ("mixed-prior-only", "mixed", "prior"),
                ("mixed-finest-only", "mixed", "finest")]
    runs = {}
    y = None
    for name, prec, stages in variants:
        if stages is None:
            os.environ.pop("MRA_MIXED_FP32", None)
        else:
            os.environ["MRA_MIXED_FP32"] = stages
        ctx = api.Context(st, md, precision=prec)
        if y is None:
            y = draw_values(ctx, st, cfg.seed + 7)
        res = {}
        for label, vals in (("y", y), ("y0", np.zeros_like(y))):
            ctx.set_obs_values(vals)
            ctx.set_theta()
            for _ in range(max(args.warmup, 1)):
                ctx.loglik()
            d, ll = ctx.loglik()
            stats = ctx.stats()
            res[label] = {"d": d, "loglik": ll, "terms": ctx.terms().tolist(),
                          "launches": [(l["kernel"], l["level"], round(l["ms"], 3)) for l in stats["launches"]],
                          "ms_total": stats["ms_total"],
                          "stage_ms": {k: stats[k] for k in ("ms_prior", "ms_finest", "ms_posterior")}}
        ctx.close()
        runs[name] = res
    os.environ.pop("MRA_MIXED_FP32", None)
    ref = runs["fp64"]
    for name, _, _ in variants[1:]:
        v = {}
        for label in ("y", "y0"):
            a, b = ref[label], runs[name][label]
            v[label] = {"d_minus_fp64": b["d"] - a["d"], "d_rel_err": abs(b["d"] - a["d"]) / abs(a["d"]),
                        "loglik_rel_err": abs(b["loglik"] - a["loglik"]) / abs(a["loglik"]),
                        "parts_minus_fp64": [bt - at for at, bt in zip(a["terms"], b["terms"])]}
        v["ms_total"] = runs[name]["y"]["ms_total"]
        v["stage_ms"] = runs[name]["y"]["stage_ms"]
        v["launches"] = runs[name]["y"]["launches"]
        out[name] = v
    out["fp64"] = {"d": ref["y"]["d"], "loglik": ref["y"]["loglik"], "d_y0": ref["y0"]["d"],
                   "ms_total": ref["y"]["ms_total"], "stage_ms": ref["y"]["stage_ms"], "launches": ref["y"]["launches"],
                   "parts": ref["y"]["terms"]}
    print(json.dumps(out))


def shard_arm(args, world, rank, local):
    """One log-likelihood per step over all ranks (sub-tree sharding, shard.py):
    every rank evaluates its sub-trees, rank 0 gathers the split level's records,
    finishes the top levels and broadcasts the result.  Strong scaling: the job
    evaluates the same tree whatever N.  Timed with CUDA events on each rank's
    current stream around the whole step (the library's work and the exchange),
    synchronised on both sides, max over ranks."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from nonstationary_mra_b200 import api, replicas, shard, synth
    torch.cuda.set_device(local)
    api.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    cfg = synth.CONFIGS[args.config]
    xy, pred, theta, md, st = make_problem(cfg)
    sp = shard.plan(st, world)
    ctx = api.Context(st, md)
    # the values: rank 0 draws them (whole-tree evaluation) and broadcasts
    y = draw_values(ctx, st, cfg.seed + 7) if rank == 0 else None
    if world > 1:
        box = [y]
        dist.broadcast_object_list(box, src=0)
        y = box[0]
    ctx.set_obs_values(y)
    ctx.set_theta()
    for _ in range(max(args.warmup, 0)):
        d, ll = shard.loglik(ctx, sp, rank, world)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    barrier()
    with ClockSampler(local) as clk:
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(args.steps):
            d, ll = shard.loglik(ctx, sp, rank, world)
        t1.record()
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1)
    barrier()
    launches = ctx.shard_launches
    ctx.close()
    ms = replicas.max_over_ranks([ms], device="cuda")[0]
    line = {"metric": METRIC, "value": args.steps / (ms * 1e-3), "unit": "evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, y drawn from the MRA prior)",
            "config": {"workload": workload_name(cfg), "parallelism": f"subtrees{world}", "split_level": sp.split,
                       "subtrees_per_rank": [int((sp.owner == k).sum()) for k in range(world)],
                       "estimated_load_imbalance": float(sp.load.max() / max(sp.load.mean(), 1e-300)),
                       "loglik": ll, "d": d, "l2": "inputs larger than L2"},
            "gpu_launches": launches * args.steps, "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def surrogate_forward_arm(args):
    """The surrogate's batched prediction (19 -> 128 -> 128 -> 1, 65,536 parameter vectors per call): values
    only, whose 128 x 128 layer runs on the tensor cores (tcgen05), and values with input gradients on the FP32
    cores.  Per call, with the host copies of the inputs and results, CUDA-stream wall clock after warm-up."""
    from nonstationary_mra_b200.fit import Surrogate
    net = Surrogate(19, seed=1)
    x = np.random.default_rng(0).standard_normal((65536, 19)).astype(np.float32)
    for _ in range(max(args.warmup, 1)):
        y = net.predict(x)
    steps = max(args.steps, 1) * 4
    t0 = time.perf_counter()
    for _ in range(steps):
        y = net.predict(x)
    t1 = time.perf_counter()
    for _ in range(steps):
        y2, _ = net.predict(x, with_grad=True)
    t2 = time.perf_counter()
    net.close()
    print(json.dumps({"metric": "surrogate predictions/s (65,536 per call, host copies included)",
                      "values_tcgen05": {"ms_per_call": 1e3 * (t1 - t0) / steps,
                                         "predictions_per_s": 65536 * steps / (t1 - t0)},
                      "values_and_input_gradients_fp32": {"ms_per_call": 1e3 * (t2 - t1) / steps,
                                                          "predictions_per_s": 65536 * steps / (t2 - t1)},
                      "max_abs_difference": float(np.max(np.abs(y - y2))), "steps": steps}))


def main():
    args = parse_args()
    if args.mixed_report:
        mixed_report_arm(args)
        return
    if args.fit:
        if args.fit_curve:
            fit_curve_arm(args)
        else:
            fit_arm(args)
        return
    if args.predict:
        predict_arm(args)
        return
    if args.sweep:
        sweep_arm(args)
        return
    if args.surrogate_forward:
        surrogate_forward_arm(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            reference_arm(args)
        return
    if args.shard:
        shard_arm(args, world, rank, local)
        return
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from nonstationary_mra_b200 import api, synth

    torch.cuda.set_device(local)
    api.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    cfg = synth.CONFIGS[args.config]
    t_setup = time.perf_counter()
    xy, pred, theta, md, st = make_problem(cfg)
    ctx = api.Context(st, md, precision=args.precision)
    y = draw_values(ctx, st, cfg.seed + 7)
    ctx.set_obs_values(y)
    ctx.set_theta()
    setup_s = time.perf_counter() - t_setup

    for _ in range(max(args.warmup, 0)):
        ctx.loglik()
    if not args.no_graph:
        ctx.capture_graph()
        ctx.loglik()
    tiles, tune_ms = ctx.autotune(1) if not args.no_autotune else (None, None)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    # device-resident timing
    barrier()
    with ClockSampler(local) as clk:
        ctx.timer_start()
        for _ in range(args.steps):
            d, ll = ctx.loglik()
        ms = ctx.timer_stop()
    barrier()
    stats = ctx.stats()

    # end to end through the C ABI: pinned y -> device, theta -> device, evaluate, result -> host
    y_pinned = torch.from_numpy(y.copy()).pin_memory()
    ctx.timer_start()
    for _ in range(args.steps):
        ctx.set_obs_values_ptr(y_pinned.data_ptr())
        ctx.set_theta()
        d2, ll2 = ctx.loglik()
    ms_e2e = ctx.timer_stop()
    barrier()

    from nonstationary_mra_b200 import replicas
    ms, ms_e2e = replicas.max_over_ranks([ms, ms_e2e], device="cuda")
    value = replicas.job_throughput(args.steps, world, ms)
    e2e = replicas.job_throughput(args.steps, world, ms_e2e)

    # roofline of the dominant stage of one evaluation.  A prior level is two
    # kernels: its covariance-block launches (k_cov_level: covariance entries,
    # reported as bytes written) and its region launches (k_prior_level: the
    # stage's products and factorizations, all of its algorithmic FLOPs); the
    # roofline is the region launches' own, the stage figure is kept beside it.
    launches = stats["launches"]
    dom = max(launches, key=lambda l: l["ms"])
    split = dom["kernel"] == "prior_level" and dom["ms_cov"] > 0
    kernel_ms = dom["ms"] - dom["ms_cov"] if split else dom["ms"]
    achieved = dom["flop"] / (kernel_ms * 1e-3) / 1e12
    achieved_stage = dom["flop"] / (dom["ms"] * 1e-3) / 1e12
    peak = fp64_peak_tflops() if rank == 0 else None
    key = f"{args.config}:{args.precision}"
    traffic_stage = traffic_lookup(f"{key}:{dom['kernel']}:{dom['level']}")
    traffic = traffic_lookup(f"{key}:prior_level_regions:{dom['level']}") if split else traffic_stage
    cov = None
    if split:
        m = dom["level"]
        entries = float(st.J) ** m * (m + 1) * st.r * st.r
        elem = 8 if args.precision == "fp64" else 4
        cov = {"kernel": f"k_cov_level (level {m})", "ms": dom["ms_cov"], "entries": entries,
               "entries_per_s": entries / (dom["ms_cov"] * 1e-3),
               "written_gb_per_s": entries * elem / (dom["ms_cov"] * 1e-3) / 1e9,
               "traffic": traffic_lookup(f"{key}:cov_level:{m}")}
    ctx.close()

    # the other precision on the same inputs, same GPU (after the first context is freed)
    other = None
    if not args.no_compare and world == 1:
        oprec = "mixed" if args.precision == "fp64" else "fp64"
        octx = api.Context(st, md, precision=oprec)
        octx.set_obs_values(y)
        octx.set_theta()
        for _ in range(max(args.warmup, 0)):
            octx.loglik()
        if not args.no_graph:
            octx.capture_graph()
            octx.loglik()
        torch.cuda.synchronize()
        octx.timer_start()
        for _ in range(args.steps):
            od, oll = octx.loglik()
        oms = octx.timer_stop()
        octx.close()
        fp64_ll = ll if args.precision == "fp64" else oll
        mixed_ll = oll if args.precision == "fp64" else ll
        other = {"precision": oprec, "evals_per_s": args.steps / (oms * 1e-3), "ms_per_step": oms / args.steps,
                 "loglik": oll, "mixed_rel_err_vs_fp64": abs(mixed_ll - fp64_ll) / abs(fp64_ll),
                 "mixed_speedup_vs_fp64": (ms / oms) if args.precision == "fp64" else (oms / ms)}

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        try:
            cpu = cpu_baseline_for(cfg, 2)
        except Exception as exc:  # reported, never silently replaced
            cpu = {"value": None, "unit": "evals/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {exc}"[:300]}
    line = {
        "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "mixed-f32tc-f64",
        "data": "synthetic (seeded, y drawn from the MRA prior)",
        "config": {"workload": workload_name(cfg), "precision": args.precision, "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (whole tree resident in HBM, no flush needed)",
                   "cuda_graph": not args.no_graph, "loglik": ll, "d": d, "n_obs": st.n_obs,
                   "autotuned_tile_widths": tiles,
                   "setup_seconds": setup_s, "device_gb": stats["bytes_device"] / 1e9,
                   "flop_per_eval": stats["flop_last"],
                   "stage_ms": {k: stats[k] for k in ("ms_fields", "ms_prior", "ms_finest", "ms_posterior")},
                   "other_precision": other},
        "roofline": {"bound": "tensor",
                     "kernel": (f"k_prior_level (level {dom['level']}: the level's region launches, "
                                f"{kernel_ms:.2f} ms)") if split else f"{dom['kernel']}(level {dom['level']})",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None, "traffic": traffic,
                     "peak_source": "FP64: cuBLAS DGEMM 8192^3 measured in this run (no FP64 figure in "
                                    "MEASURED_PEAKS.json)",
                     "stage": {"what": f"{dom['kernel']}(level {dom['level']}) with its covariance launches",
                               "ms": dom["ms"], "achieved": achieved_stage,
                               "frac": achieved_stage / peak if peak else None, "traffic": traffic_stage},
                     "covariance": cov},
        "e2e": {"value": e2e, "unit": "evals/s", "h2d_bytes_per_step": 8 * st.n_obs + 16 * 8 + 8 * 18,
                "d2h_bytes_per_step": 8 + 16},
        "gpu_launches": stats["kernel_launches"] * args.steps,
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
