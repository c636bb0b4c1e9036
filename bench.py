"""Benchmark: stage-2 PS x ifg per second per gamma iteration on B200.

Workload: the full-scale stage-2 patch (2,000,000 PS candidates, 150
interferograms, 256x256 grid at 50 m, 161 trial multipliers), seeded synthetic
data from pystamps_b200.synth. One step = one gamma iteration (bin -> CLAP ->
resample -> topofit -> convergence / P-square update) over the whole patch.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs its own replica of the patch (the
single-patch path has no cross-GPU exchange; weak scaling), the timed region is
bracketed by barriers and the max over ranks is reported by rank 0.

value  : device-resident inputs, K iterations timed with CUDA events on the
         library's stream, N_ps * N_ifg * K / t (whole job: summed over ranks).
e2e    : one public-API stage-2 run per step from pinned host buffers (upload,
         layout, iterate to convergence, download of K/C/coh/N_opt), metric =
         N_ps * N_ifg * iterations / t.
--impl reference : the oracle (C++ restatement of the reference's native
         stage 2) on all host cores: each step one whole gamma iteration on the
         PS of the patch's 96 x 96-cell corner (see cpu_baseline.sample); the
         product library is not loaded on this path.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Stage-2 PS×ifg/s per gamma iter, FP32 vs plain FP64 GPU at max|Δγ|≤1e-4"
UNIT = "PS*ifg/s"
FP32_LANES_PER_SM = 128
# DRAM bytes (read + write) per PS x ifg of one k_topofit_f32 launch, from an ncu
# capture (dram__bytes_read.sum + dram__bytes_write.sum) of the full-scale shape
# with 250,000 PS x 150 ifg (256x256 grid): 537.4 MB per launch; the reported
# traffic scales it by N x M.
TOPOFIT_TRAFFIC_BYTES_PER_PS_IFG = 537.9e6 / (250_000 * 150)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="E",
                    help="A, B, D or E (default E, the full-scale patch), or C: 64 uneven patches")
    ap.add_argument("--n-ps", type=int, default=0, help="override the PS count (profiling a smaller case)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-stage3", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="one patch split over the ranks by cell ranges (strong scaling) instead of replicas")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks ----
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------- workload -----
def make_workload(name: str, rank: int, n_ps: int = 0):
    from pystamps_b200 import synth

    w = synth.ALIASES.get(name) or synth.WORKLOADS[name]
    if n_ps:
        import dataclasses

        w = dataclasses.replace(w, name=f"{w.name}-at-{n_ps}-ps", n_ps=n_ps)
    patch = synth.make_workload(w, patch_id=rank)
    return w, patch


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0, "fallback": True}


# ------------------------------------------------------------ CPU leg -------
# The CPU figures time the oracle (the C++ restatement of the reference's
# native stage 2, crates/pystamps-core/src/native_stage2.rs) doing WHOLE gamma
# iterations (fill + bin, CLAP of every interferogram, extract, topofit,
# weighting update, convergence test: the loop body :261-406) on a spatial
# sample of the workload: the PS of the workload's corner of
# SAMPLE_CELLS x SAMPLE_CELLS grid cells (every interferogram, the same trial
# count and PS density). Work per PS x ifg is then that of the whole patch
# (CLAP cost follows the cell count, topofit the PS count); nothing is scaled.
SAMPLE_CELLS = 96


def workload_config(w, n_ps: int, n_ifg: int, n_i: int, n_j: int, trials: int) -> dict:
    """The config dict both arms print (identical by construction)."""
    return {"workload": w.name, "n_ps": int(n_ps), "n_ifg": int(n_ifg), "grid": [int(n_i), int(n_j)],
            "trials": int(trials),
            "l2": (f"inputs larger than L2 (ph_nm {n_ps * n_ifg * 8 / 1e9:.2f} GB per step)"
                   if n_ps * n_ifg * 8 > 126e6 else "inputs smaller than L2 (no flush; small config)")}


def corner_subpatch(patch: dict, cells: int) -> dict:
    """The PS of the patch's first `cells` x `cells` grid cells (the
    reference's grid rule, via the oracle) as a patch of their own, rows in
    their original order."""
    from oracle import oracle as O

    gij = O.grid_indices(patch["xy"], float(patch["parms"].get("filter_grid_size", 50.0)))
    keep = np.where((gij[:, 0] <= cells) & (gij[:, 1] <= cells))[0]
    sub = dict(patch)
    for k in ("ph", "bperp_mat", "D_A", "xy"):
        sub[k] = np.ascontiguousarray(np.asarray(patch[k])[keep])
    sub.pop("truth", None)
    return sub


def oracle_iterations(patch: dict, n_iter: int, threads: int, n_rand: int = 20_000) -> dict:
    """n_iter whole iterations of the oracle's stage-2 loop on `patch` (the
    stop rule disabled so exactly n_iter run), with the random-phase
    histogram from n_rand rows (setup, outside the timed loop). Returns the
    wall time of each iteration."""
    from oracle import oracle as O

    p = dict(patch, parms=dict(patch["parms"], gamma_change_convergence=0.0, gamma_max_iterations=int(n_iter)))
    bp = np.asarray(patch["bperp"], dtype=np.float64).reshape(-1)
    bp_nm = np.delete(bp, int(patch.get("master_ix", 1)) - 1)
    lam = float(p["parms"].get("lambda", 0.0555))
    max_k = float(p["parms"].get("max_topo_err", 15.0)) / (lam * 830_000.0 * math.sin(float(p["mean_incidence"])) /
                                                          (4.0 * math.pi))
    ntw = float((bp_nm.max() - bp_nm.min()) * max_k / (2.0 * math.pi))
    nr, mx = O.random_hist(bp_nm, ntw, n_rand=n_rand, threads=threads)
    p["nr_override"] = np.concatenate([nr, [mx]])
    res = O.stage2_run(p, threads=threads)
    return {"iter_seconds": [float(t) for t in res["iter_seconds"]], "n_ps": int(np.asarray(p["ph"]).shape[0]),
            "n_ifg": int(res["n_ifg"]), "grid": [int(res["n_i"]), int(res["n_j"])], "trials": int(res["n_trials"])}


def cpu_baseline_sample(sub: dict, n_iter: int, threads: int) -> dict:
    """Whole oracle iterations on a corner sub-patch (corner_subpatch)."""
    r = oracle_iterations(sub, n_iter, threads)
    t = statistics.median(r["iter_seconds"])
    return {"value": r["n_ps"] * r["n_ifg"] / t, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"whole oracle gamma iterations (median of {n_iter}, {t:.2f} s each) on the PS of the "
                       f"{SAMPLE_CELLS}x{SAMPLE_CELLS}-cell corner of the patch: {r['n_ps']} PS x {r['n_ifg']} ifg, "
                       f"{r['grid'][0]}x{r['grid'][1]} grid, {r['trials']} trials, all {threads} host threads"),
            "what": "C++ restatement of crates/pystamps-core/src/native_stage2.rs (Rust toolchain absent)"}


def ncores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args, rank: int, world: int):
    """The reference arm: the oracle (CPU restatement of the reference's
    native stage 2) on all host threads, rank 0 only. Each step is one whole
    oracle gamma iteration on the PS of the workload's corner of
    SAMPLE_CELLS x SAMPLE_CELLS cells; the metric is PS x ifg of the sample
    per second of iteration. No product library is loaded on this path."""
    if rank != 0:
        return
    from oracle import oracle as O
    from pystamps_b200 import synth

    w = synth.ALIASES.get(args.workload) or synth.WORKLOADS[args.workload]
    if args.n_ps:
        import dataclasses

        w = dataclasses.replace(w, name=f"{w.name}-at-{args.n_ps}-ps", n_ps=args.n_ps)
    patch = synth.make_workload(w, patch_id=0)
    gij = O.grid_indices(patch["xy"], 50.0)
    n_i, n_j = int(gij[:, 0].max()), int(gij[:, 1].max())
    config = workload_config(w, patch["ph"].shape[0], patch["ph"].shape[1] - 1, n_i, n_j, w.n_trials)
    sub = corner_subpatch(patch, SAMPLE_CELLS)
    del patch
    threads = ncores()
    r = oracle_iterations(sub, args.warmup + args.steps, threads)
    ts = r["iter_seconds"][args.warmup:]
    t_total = float(sum(ts))
    v = r["n_ps"] * r["n_ifg"] * len(ts) / t_total
    sample = (f"per step: one whole oracle gamma iteration on the PS of the {SAMPLE_CELLS}x{SAMPLE_CELLS}-cell "
              f"corner of the patch ({r['n_ps']} PS x {r['n_ifg']} ifg, {r['grid'][0]}x{r['grid'][1]} grid, "
              f"{r['trials']} trials), all {threads} host threads; {args.warmup} warm-up iterations untimed")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_total / len(ts) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, pystamps_b200.synth)", "config": config,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                         "what": "C++ restatement of crates/pystamps-core/src/native_stage2.rs (Rust toolchain absent)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "iter_seconds": ts,
    }
    print(json.dumps(line), flush=True)


def adjoint_leg(prep, dev: int) -> dict:
    """ps2_coherence_forward / _backward (the torch.autograd.Function's two
    calls) on the workload, FP32, timed with CUDA events on the current
    stream: ms per call and PS x ifg per second."""
    import torch

    from pystamps_b200 import autograd as AG

    cmap = AG.CoherenceMap(prep, dev)
    try:
        d = torch.device("cuda", dev)
        ph = torch.from_numpy(np.ascontiguousarray(prep.ph_nm, dtype=np.complex64)).to(d)
        K = torch.zeros(prep.n_ps, dtype=torch.float32, device=d)
        w = torch.from_numpy(np.asarray(prep.weight0, dtype=np.float32)).to(d)
        g = torch.ones(prep.n_ps, dtype=torch.float32, device=d)
        for _ in range(2):
            cmap.forward(ph, K, w, prep.clap_alpha, prep.clap_beta)
            cmap.backward(ph, K, w, prep.clap_alpha, prep.clap_beta, g)
        out = {}
        for name, fn in (("forward", lambda: cmap.forward(ph, K, w, prep.clap_alpha, prep.clap_beta)),
                         ("backward", lambda: cmap.backward(ph, K, w, prep.clap_alpha, prep.clap_beta, g))):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(3):
                fn()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / 3
            out[name + "_ms"] = ms
            out[name + "_ps_ifg_per_s"] = prep.n_ps * prep.n_ifg / (ms / 1e3)
        out["what"] = "FP32 coherence map with K given: bin, CLAP, resample, coherence; backward recomputes the forward"
        return out
    finally:
        cmap.close()


def stage3_leg(ctx, prep, rank: int, cpu: bool = True) -> dict:
    """Stage-3 re-estimate of the PS whose converged stage-2 coherence
    exceeds 0.3: through ps2_stage3_reestimate on the context that ran stage 2
    (selection in, results out to host memory, or kept on the device), and
    through ps3_reestimate (every input from host memory, the reference's
    stage-3 interface); the oracle re-estimates a bounded sample of the same
    rows on the host cores for the CPU figure."""
    import torch

    from pystamps_b200 import stage3

    pm = ctx.download(["coh_ps", "ph_grid"])
    sel = np.where(pm["coh_ps"] > 0.3)[0]
    gij = np.rint(prep.grid_ij).astype(np.int64)
    bp = np.asarray(prep.bperp, dtype=np.float32)
    bp = np.broadcast_to(bp, (prep.n_ps, prep.n_ifg)) if bp.ndim == 1 else bp
    fit = np.arange(prep.n_ifg)
    ntw = float(prep.n_trial_wraps)
    kw = dict(clap_alpha=prep.clap_alpha, clap_beta=prep.clap_beta, low_pass=prep.low_pass, n_trial_wraps=ntw)

    def best(fn, reps=2):
        fn()  # warm-up
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return min(ts)

    t_res = best(lambda: stage3.reestimate_resident(ctx, sel, fit))
    t_dev = best(lambda: stage3.reestimate_resident(ctx, sel, fit, on_device=True))
    t_host = best(lambda: stage3.reestimate(pm["ph_grid"], gij, sel, prep.ph_nm, bp, fit, **kw))
    out = {"selected_ps": int(sel.size), "n_ifg": prep.n_ifg, "seconds": t_res, "ps_per_s": sel.size / t_res,
           "cells": int(np.unique(gij[sel, 0] * 100000 + gij[sel, 1]).size),
           "what": "stage3.reestimate_resident: selection H2D, patch CLAP per PS cell + stage-3 topofit on the "
                   "stage-2 context's resident grid/phases/bperp, results D2H",
           "outputs_on_device_seconds": t_dev,
           "host_entry_seconds": t_host,
           "host_entry_what": "stage3.reestimate: gather rows + ps3_reestimate (grid, phases, bperp H2D; results D2H)"}
    if cpu and rank == 0:
        from oracle import oracle as O

        k = min(2000, sel.size)
        t0 = time.perf_counter()
        O.s3_reestimate(pm["ph_grid"], gij, sel[:k], prep.ph_nm, bp, fit, alpha=prep.clap_alpha,
                        beta=prep.clap_beta, low_pass=prep.low_pass, n_trial_wraps=ntw)
        tc = time.perf_counter() - t0
        out["cpu_baseline"] = {"ps_per_s": k / tc, "cores": ncores(), "kind": "port",
                               "sample": f"oracle re-estimate of {k} of the {sel.size} selected PS"}
    return out


# ------------------------------------------------------------- GPU leg ------
def run_ours(args, rank: int, world: int, dist):
    import torch

    from pystamps_b200 import stage2 as S
    from pystamps_b200 import _lib

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    w, patch = make_workload(args.workload, rank, args.n_ps)
    t0 = time.perf_counter()
    prep = S.prepare_patch(patch)
    t_prep = time.perf_counter() - t0
    inc = float(patch["mean_incidence"])
    lam = float(patch["parms"].get("lambda", 0.0555))
    cpu_patch = corner_subpatch(patch, SAMPLE_CELLS) if rank == 0 and not args.no_cpu else None
    del patch
    n, m = prep.n_ps, prep.n_ifg
    T = 2 * math.ceil(8 * prep.n_trial_wraps) + 1

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    # ---------------- value: device-resident inputs -------------------------
    ctx = S.Stage2Context(dev)
    ctx.load(prep, "fp32")
    ctx.iterate(max(args.warmup, 1))
    barrier()
    clk = ClockSampler(dev)
    clk.start()
    ctx.iterate(args.steps)
    total_ms, per = ctx.timing()
    launches = ctx.launch_count()
    clocks = clk.stop()
    barrier()
    t_max = total_ms
    if dist is not None:
        tt = torch.tensor([total_ms], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    value = world * n * m * args.steps / (t_max / 1e3)
    ms_per_step = t_max / args.steps
    topo_ms = per[2] / args.steps
    bin_ms = per[0] / args.steps
    clap_ms = per[1] / args.steps
    # roofline of the dominant kernel (topofit): algorithmic flops per launch
    flops = (8 * T + 32) * n * m
    sm_max = float(load_peaks().get("sm_max_mhz", 1965.0))
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    fp32_peak_tflops = 2 * FP32_LANES_PER_SM * sms * sm_max * 1e6 / 1e12
    achieved = flops / (topo_ms / 1e3) / 1e12
    peaks = load_peaks()
    bin_bytes = n * m * (8 + (0 if prep.row_invariant else 4)) + prep.n_i * prep.n_j * m * 8
    roofline = {
        "kernel": "k_topofit_f32", "bound": "fp32", "achieved": achieved, "peak": fp32_peak_tflops,
        "unit": "TFLOP/s", "frac": achieved / fp32_peak_tflops,
        "traffic": TOPOFIT_TRAFFIC_BYTES_PER_PS_IFG * n * m,
        "traffic_source": "ncu dram__bytes_read+write at 250k PS x 150 ifg (256x256 grid) scaled by PS x ifg",
        "algorithmic": f"(8*T+32) flop per PS x ifg, T={T}: {flops:.3e} flop per launch",
        "peak_source": f"nominal FP32 FMA rate {sms} SM x {FP32_LANES_PER_SM} lanes x 2 x {sm_max:.0f} MHz "
                       "(MEASURED_PEAKS.json has no FP32 figure)",
        "share_of_step": topo_ms / ms_per_step,
    }
    bin_roof = {"kernel": "k_bin", "bound": "hbm", "achieved": bin_bytes / (bin_ms / 1e3) / 1e9,
                "peak": float(peaks.get("hbm_gbs", 6650.0)), "unit": "GB/s",
                "frac": bin_bytes / (bin_ms / 1e3) / 1e9 / float(peaks.get("hbm_gbs", 6650.0)),
                "algorithmic": "12 B per PS x ifg (ph_nm c64 + bperp f32) + 8 B per cell x ifg",
                "peak_source": ("fallback 6.65 TB/s (MEASURED_PEAKS.json absent)" if peaks.get("fallback")
                                else "measured copy bandwidth, MEASURED_PEAKS.json hbm_gbs")}
    ctx.close()

    # ---------------- plain FP64 GPU path ------------------------------------
    fp64 = None
    if not args.no_fp64:
        c64 = S.Stage2Context(dev)
        c64.load(prep, "fp64")
        c64.iterate(1)
        k64 = 2
        c64.iterate(k64)
        t64, per64 = c64.timing()
        fp64 = {"value": world * n * m * k64 / (t64 / 1e3), "ms_per_step": t64 / k64,
                "topofit_ms": per64[2] / k64}
        c64.close()

    # ---------------- e2e: public API from pinned host buffers ---------------
    pin = {}
    for name, arr in (("ph_nm", prep.ph_nm), ("bperp", prep.bperp), ("grid_lin", prep.grid_lin),
                      ("weight0", prep.weight0)):
        t = torch.from_numpy(np.ascontiguousarray(arr)).pin_memory()
        pin[name] = t.numpy()
    import dataclasses

    prep_pinned = dataclasses.replace(prep, **pin)
    h2d = (prep.ph_nm.nbytes + prep.bperp.nbytes + prep.grid_lin.nbytes + prep.weight0.nbytes +
           prep.low_pass.nbytes + prep.nr.nbytes)
    d2h = 4 * n * 8
    e2e_vals, iters = [], []
    ectx = S.Stage2Context(dev)
    # the results land in pinned host buffers allocated once, as the inputs come from them
    e2e_out = {k: torch.empty(n, dtype=torch.float64).pin_memory().numpy()
               for k in ("K_ps", "C_ps", "coh_ps", "N_opt")}
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        barrier()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        tw = time.perf_counter()
        ev0.record()
        ectx.load(prep_pinned, "fp32")
        st = ectx.run()
        out = ectx.download(["K_ps", "C_ps", "coh_ps", "N_opt"], out=e2e_out)
        ev1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - tw
        if i == 0:
            continue  # warm-up
        t = max(ev0.elapsed_time(ev1) / 1e3, wall)
        if dist is not None:
            tt = torch.tensor([t], dtype=torch.float64, device=f"cuda:{dev}")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        e2e_vals.append(world * n * m * st["i_loop"] / t)
        iters.append(st["i_loop"])
    # ---------------- adjoint of the coherence (forward + backward) ------------
    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_leg(prep, dev)
    # ---------------- stage-3 re-estimate on the converged patch ---------------
    stage3 = None
    if not args.no_stage3 and e2e_vals:
        stage3 = stage3_leg(ectx, prep, rank, cpu=not args.no_cpu)
    ectx.close()
    e2e = None if not e2e_vals else {"value": statistics.median(e2e_vals), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "iterations_per_step": iters,
           "what": "per step: ps2_load_patch (H2D + cell layout) + ps2_run_to_convergence + ps2_download(K,C,coh,N_opt) "
                   "into pinned host buffers"}

    # ---------------- precision vs the plain FP64 path -----------------------
    prec = None
    if fp64 is not None:
        kconv = lam * 830_000.0 * math.sin(inc) / (4 * math.pi)  # rad/m -> m of DEM error
        # first iteration: both paths from the same state, the arithmetic alone
        with S.Stage2Context(dev) as c32, S.Stage2Context(dev) as c64:
            c32.load(prep, "fp32")
            c64.load(prep, "fp64")
            c32.iterate(1)
            c64.iterate(1)
            a1 = c32.download(["coh_ps", "K_ps"])
            b1 = c64.download(["coh_ps", "K_ps", "ph_patch"])
        d1 = np.abs(a1["coh_ps"] - b1["coh_ps"])
        dk1 = np.abs(a1["K_ps"] - b1["K_ps"]) * kconv
        # PS beyond the bounds, classified by the FP64 trial search of their rows
        from pystamps_b200.precision import classify_ties

        out_rows = np.flatnonzero((d1 > 1e-4) | (dk1 > 1e-3))
        bp_rows = prep.bperp if prep.row_invariant else prep.bperp[out_rows]
        cls = classify_ties(prep.ph_nm[out_rows], b1["ph_patch"][out_rows], bp_rows, prep.n_trial_wraps)
        del b1
        nontie = ~cls["tie"]
        tie_rows = out_rows[cls["tie"]]
        # to convergence, each path on its own trajectory
        a = S.run_stage2(prep, precision="fp32", keys=["coh_ps", "K_ps"])
        b = S.run_stage2(prep, precision="fp64", keys=["coh_ps", "K_ps"])
        d = np.abs(a["coh_ps"] - b["coh_ps"])
        dk = np.abs(a["K_ps"] - b["K_ps"]) * kconv
        prec = {"first_iteration": {
                    "dgamma_max": float(d1.max()), "dgamma_p9999": float(np.quantile(d1, 0.9999)),
                    "n_dgamma_above_1e-4": int((d1 > 1e-4).sum()), "dK_m_p9999": float(np.nanquantile(dk1, 0.9999)),
                    "n_dK_above_1e-3_m": int((dk1 > 1e-3).sum()),
                    "n_argmax_ties": int(cls["argmax_tie"].sum()), "n_fp32_near_ties": int(cls["near_tie"].sum()),
                    "n_wrap_ties": int(cls["wrap_tie"].sum()),
                    "n_nontie_above_1e-4": int((d1[out_rows] > 1e-4)[nontie].sum()),
                    "n_nontie_above_1e-3_m": int((dk1[out_rows] > 1e-3)[nontie].sum()),
                    "nontie_dgamma_max": float(np.delete(d1, tie_rows).max()),
                    "nontie_dK_m_max": float(np.nanmax(np.delete(dk1, tie_rows))),
                    "note": "PS above the bounds classified by an FP64 trial search of their rows "
                            "(pystamps_b200.precision.classify_ties): argmax ties (best and runner-up trial "
                            "within 1e-6 relative), FP32 near ties (within 1e-6 of max(best, 0.5), not argmax "
                            "ties) and refinement wrap ties (a residual angle within 1e-4 rad of +-pi)"},
                "converged": {"iterations_fp32": a["i_loop"], "iterations_fp64": b["i_loop"],
                              "dgamma_median": float(np.median(d)), "dgamma_p99": float(np.quantile(d, 0.99)),
                              "dgamma_max": float(d.max()), "dK_m_median": float(np.nanmedian(dk)),
                              "dK_m_p99": float(np.nanquantile(dk, 0.99))}}

    cpu = None
    if rank == 0 and not args.no_cpu and cpu_patch is not None:
        cpu = cpu_baseline_sample(cpu_patch, 3, ncores())
    del cpu_patch

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator pystamps_b200.synth)",
            "config": workload_config(w, n, m, prep.n_i, prep.n_j, T),
            "parallelism": f"replicas x{world}",
            "per_kernel_ms": {"bin": bin_ms, "clap": clap_ms, "topofit": topo_ms, "finalize": per[3] / args.steps},
            "prepare_s": t_prep,
            "roofline": roofline, "roofline_bin": bin_roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(launches), "clocks": clocks, "fp64_gpu": fp64,
            "fp32_over_fp64": (value / fp64["value"]) if fp64 else None, "precision_vs_fp64": prec,
            "stage3_reestimate": stage3, "adjoint": adjoint,
        }
        print(json.dumps(line), flush=True)


def run_shard(args, rank: int, world: int, dist):
    """One patch over all ranks (pystamps_b200.shard): rank r owns the PS of a
    contiguous cell range; per iteration bin -> halo exchange of the cells each
    rank's CLAP reads -> CLAP/overlap of its cells -> topofit of its rows ->
    all-reduce of 102 statistics -> finalize. value = N*M*K / t, t the K timed
    iterations (barriers and a device synchronise around them, host clock, max
    over ranks): strong scaling, the total work fixed."""
    import torch

    from pystamps_b200 import shard
    from pystamps_b200 import stage2 as S

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    w, patch = make_workload(args.workload, 0, args.n_ps)  # the same patch on every rank
    prep = S.prepare_patch(patch)
    del patch
    n, m = prep.n_ps, prep.n_ifg
    T = 2 * math.ceil(8 * prep.n_trial_wraps) + 1
    ranges = shard.split_cells(prep.grid_lin, prep.n_i * prep.n_j, world)
    lo, hi = ranges[rank]
    plan = shard.halo_plan(ranges, prep.n_i, prep.n_j, prep.clap_window)
    r = shard.ShardRank(prep, lo, hi, device=dev)
    halo_bytes = sum((c1 - c0) for q, dst, c0, c1 in plan if q == rank) * (r.grid.numel() // (prep.n_i * prep.n_j)) \
        * r.grid.element_size()

    def one_iteration():
        g = r.bin()
        if dist is not None:
            shard.halo_exchange(g, plan, rank, prep.n_i * prep.n_j)
        r.filter(g)
        st = r.fit()
        if dist is not None:
            t = torch.from_numpy(st).to(g.device)
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
            st = t.cpu().numpy()
        return r.finalize(st, n)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    barrier()
    for _ in range(max(args.warmup, 1)):
        one_iteration()
    barrier()
    clk = ClockSampler(dev)
    clk.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        one_iteration()
    barrier()
    t = time.perf_counter() - t0
    clocks = clk.stop()
    if dist is not None:
        tt = torch.tensor([t], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    r.close()
    if rank == 0:
        line = {"metric": METRIC, "value": n * m * args.steps / t, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded generator pystamps_b200.synth)",
                "config": workload_config(w, n, m, prep.n_i, prep.n_j, T),
                "parallelism": f"shard x{world} (cell ranges, halo exchange)", "clocks": clocks,
                "halo_bytes_rank0_per_iteration": int(halo_bytes), "cells_rank0": [lo, hi],
                "timing": "host clock around K synchronous shard iterations, barriers on both sides"}
        print(json.dumps(line), flush=True)


def run_batched(args, rank: int, world: int, dist):
    """The uneven multi-patch workload: 64 patches, PS log-uniform in 5k-400k,
    30-120 interferograms, LPT-assigned to ranks. Every patch of the rank is
    loaded into its own context and all run together with ps2_batch_run (one
    launch per step per iteration over every still-iterating patch).
    value = sum over patches of N*M*iterations / t, t = one batched run to
    convergence (library CUDA events, max over ranks); e2e = load + batched
    run + download of K/C/coh/N_opt per step, from pinned host buffers."""
    import dataclasses

    import torch

    from pystamps_b200 import batch, stage2 as S, synth

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    shapes = synth.batched_workload_shapes(64)
    costs = [batch.patch_cost(n, m, t, c, c) for n, m, c, t in shapes]
    share = batch.lpt_assign(costs, world)[rank]
    preps = []
    for i in share:
        n, m, cells, t = shapes[i]
        p = synth.make_patch(n, m, cells, t, seed=2005 + 2000 + i)
        pr = S.prepare_patch(p)
        pin = {k: torch.from_numpy(np.ascontiguousarray(getattr(pr, k))).pin_memory().numpy()
               for k in ("ph_nm", "bperp", "grid_lin", "weight0")}
        preps.append(dataclasses.replace(pr, **pin))

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        tt = torch.tensor([x], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    def sum_over_ranks(x: float) -> float:
        if dist is None:
            return x
        tt = torch.tensor([x], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(tt, op=dist.ReduceOp.SUM)
        return float(tt.item())

    b = batch.Batch(preps, dev)
    for _ in range(max(args.warmup, 1)):
        b.reset()
        b.run()
    times, units, launches = [], [], 0
    clk = ClockSampler(dev)
    for step in range(args.steps):
        b.reset()
        barrier()
        if step == 0:
            clk.start()
        stats = b.run()
        times.append(b.timing_ms() / 1e3)
        units.append(sum(st["i_loop"] * p.n_ps * p.n_ifg for st, p in zip(stats, preps)))
        launches = b.launch_count()
    clocks = clk.stop()
    iters = [st["i_loop"] for st in stats]
    t_step = max_over_ranks(statistics.median(times))
    u_step = sum_over_ranks(float(statistics.median(units)))

    # e2e: the same contexts (device buffers kept) reload every patch from
    # pinned host buffers, run together, and download K/C/coh/N_opt
    e2e_vals = []
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        barrier()
        tw = time.perf_counter()
        b.load(preps)
        st_e = b.run()
        res = b.download()
        torch.cuda.synchronize()
        wall = max_over_ranks(time.perf_counter() - tw)
        if i == 0:
            continue
        done = sum_over_ranks(float(sum(s_["i_loop"] * p.n_ps * p.n_ifg for s_, p in zip(st_e, preps))))
        e2e_vals.append(done / wall)
    b.close()

    if rank == 0:
        line = {"metric": METRIC, "value": u_step / t_step, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator pystamps_b200.synth)",
                "config": {"workload": "batched-64-uneven-patches", "patches": 64,
                           "ps_x_ifg_total": int(sum(n * m for n, m, _, _ in shapes)),
                           "iterations_rank0": iters,
                           "l2": "inputs larger than L2 (patch data several GB)",
                           "parallelism": f"LPT by patch over {world} GPU(s); ps2_batch_run per GPU"},
                "gpu_launches": int(launches), "clocks": clocks,
                "e2e": None if not e2e_vals else {
                    "value": statistics.median(e2e_vals), "unit": UNIT,
                    "h2d_bytes_per_step": int(sum(p.ph_nm.nbytes + p.bperp.nbytes + p.grid_lin.nbytes +
                                                  p.weight0.nbytes for p in preps)),
                    "d2h_bytes_per_step": int(sum(32 * p.n_ps for p in preps)),
                    "what": "per step: ps2_load_patch of every patch (8 host threads, device buffers reused) + "
                            "ps2_batch_run + ps2_download of K/C/coh/N_opt"}}
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    # the shard mode takes the process group even for one rank when launched by
    # torchrun (MASTER_ADDR set): the same NCCL all-reduce and exchange calls
    if world > 1 or (args.shard and "MASTER_ADDR" in os.environ):
        import datetime

        import torch
        import torch.distributed as tdist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        dist = tdist
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.workload == "C":
            run_batched(args, rank, world, dist)
        elif args.shard:
            run_shard(args, rank, world, dist)
        else:
            run_ours(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
