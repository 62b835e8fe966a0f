#!/usr/bin/env python
"""Benchmark of the LaughlinEdge B200 engine.

Default line: the learned-proposal form (the workload the metric "effective
samples/s and S/H updates/s, learned vs plain MC" is quoted on).  Laughlin
nu = 1/3 (m = 3), N = 200 electrons, V = omega r^2 + kappa r^4 with
omega = 1e-3, kappa = 5e-6, edge sectors dL = 1..20 (2713 power-sum states),
65536 walkers, Philox seed 42.  The DeepSets proposal is trained first (5000
ES+Adam steps on 2^20 configurations of the plain chain).  Synthetic by
construction: walkers start uniformly in the disk of radius sqrt(2 m N) and are
burnt in before anything is timed.

A step is one pass of the hot path over all walkers: one Metropolis sweep
(N single-particle moves per walker), one measurement record, the basis build
and the TF32x3 contraction of S, H2, H4 for every sector.  The same step is
timed with three samplers: the learned proposal, the plain Gaussian step at
the same sigma = 0.3, and the plain step tuned to 50 % acceptance (the
reference's own criterion).

Metric: effective samples/s = walkers x steps / tau_int / time.  tau_int (in
sweeps, max over Re/Im p_1..p_4) comes from a separate, untimed chain of the
same sampler, thousands of sweeps long (>= 50 tau), by Sokal's windowing with
a binning plateau beside it; it is never estimated from the timed steps.

``--impl reference`` times the oracle's C restatement of the reference
estimator (one Metropolis chain per basis row guided by |P_a Psi|^2, per-row
ratio sums) on all host cores on a bounded sample of the same workload, with
tau_int from a long chain of that estimator.
``--mixed`` gives the mixed-precision line (N = 50, dL = 0..12, 272 states),
``--batched`` the batched line (N = 100, dL = 1..20, 16 kappas) and
``--evolution`` the time-evolution pipeline, ``--occupation`` the two-state
walker's occupations, each as its own JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = {
    "workload": "learned_proposal_m3_N200_dL1-20_W65536",
    "particles": 200, "inverse_filling": 3, "omega": 1e-3, "kappa": 5e-6,
    "sectors": list(range(1, 21)), "walkers": 65536, "sigma": 0.3, "seed": 42,
    "gram_mode": "tf32x3", "train_configs": 1 << 20, "train_steps": 5000, "train_batch": 1024,
    "train_pairs": 32, "tau_walkers": 8192, "tau_sweeps_plain": 12000, "tau_sweeps_learned": 8000,
    "burn": 1000,
}
MIXED = {
    "workload": "mixed_precision_m3_N50_dL0-12_W65536",
    "particles": 50, "inverse_filling": 3, "omega": 5e-3, "kappa": 2e-5,
    "sectors": list(range(13)), "walkers": 65536, "sigma": 0.3, "seed": 42,
    "gram_mode": "tf32x3", "tau_walkers": 8192, "tau_sweeps": 4000, "burn": 1000,
}
METRIC = "effective_samples_per_s"
UNIT = "samples/s"


def sum_d2(sectors, N):
    import laughlinedge_b200 as L
    rows, _, _ = L.partitions(N, sectors)
    from collections import Counter
    cnt = Counter(r[0] for r in rows)
    return sum(v * v for v in cnt.values()), sum(cnt.values())


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
            "sm_max_mhz": 1965.0}, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [l.split(",") for l in Path(self.f.name).read_text().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = max(smax, float(r[2]))
                for k, n in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def allreduce_max(x, ws):
    if ws == 1:
        return x
    from laughlinedge_b200.replicas import max_over_ranks
    return max_over_ranks(x)


def rank_seed(seed, rank):
    from laughlinedge_b200.replicas import rank_seed as rs
    return rs(seed, rank)


def gram_mode_id(name):
    import laughlinedge_b200 as L
    return {"fp64": L._lib.GRAM_FP64, "bf16x3": L._lib.GRAM_BF16X3, "bf16x4": L._lib.GRAM_BF16X4,
            "tf32x3": L._lib.GRAM_TF32X3}[name]


def traffic_from_profiles():
    """Per-launch DRAM bytes of each kernel from the committed ncu summary, if any."""
    f = ROOT / "profiles" / "ncu_traffic.txt"
    out = {}
    if f.exists():
        for line in f.read_text().splitlines():
            parts = line.split()
            if len(parts) == 2 and not line.startswith("#"):
                try:
                    out[parts[0]] = float(parts[1])
                except ValueError:
                    pass
    return out


def cpu_port(w, threads=0, budget_s=15.0, tau_sweeps=6000, tau_sectors=(1, 2, 3, 4)):
    """The oracle's C restatement of the reference estimator (one Metropolis
    chain per basis row guided by |P_a Psi|^2, per-row ratio sums over every
    row of the workload's sectors) on the host cores.

    Throughput: a bounded sample (about budget_s of CPU work) of the full
    workload.  tau_int: a separate chain of the same estimator and step,
    tau_sweeps measured sweeps long with four walkers per thread (the guide rows
    of tau_sectors; the p_1..p_4 series does not depend on the basis size),
    Sokal windowing with the binning plateau beside it."""
    import numpy as np

    import laughlinedge_b200 as L
    from oracle import oracle as O
    O.load()
    nth = threads or O.load().orc_max_threads()
    N, m = w["particles"], w["inverse_filling"]
    t0 = time.perf_counter()
    tres = O.run_rows(N, m, 4 * nth, w["sigma"], w["seed"] + 5, 200, tau_sweeps, list(tau_sectors),
                      nthreads=nth)
    t_tau = time.perf_counter() - t0
    tau = L.sampler.series_tau(np.asarray(tres["series"]))
    # calibrate on a tiny run, then size the sample to the budget
    wc = nth
    t0 = time.perf_counter()
    O.run_rows(N, m, wc, w["sigma"], w["seed"], 2, 3, w["sectors"], nthreads=nth)
    per = (time.perf_counter() - t0) / (wc * 5)  # seconds per walker-sweep (all cores)
    n_meas = 20
    W = max(nth, min(4096, int(budget_s / max(per, 1e-9) / (n_meas + 5))))
    W -= W % nth
    t0 = time.perf_counter()
    O.run_rows(N, m, W, w["sigma"], w["seed"], 5, n_meas, w["sectors"], nthreads=nth)
    dt = time.perf_counter() - t0
    D = sum_d2(w["sectors"], N)[1]
    ws_per_s = W * (n_meas + 5) / dt
    tv = tau_value(tau)
    return {"value": ws_per_s / tv if tv else None, "unit": UNIT, "cores": nth, "kind": "port",
            "sample": f"{W} walkers x ({n_meas} measured + 5 burn-in) sweeps of the per-row reference "
                      f"estimator over all {D} rows, {dt:.1f} s wall; tau_int from a separate "
                      f"{tau_sweeps}-sweep chain of {4 * nth} walkers ({t_tau:.1f} s)",
            "walker_sweeps_per_s": ws_per_s, "tau_int": tv, "tau_int_detail": tau}


def tau_value(t):
    """The tau_int a line uses: Sokal's window estimate; the binning plateau when
    the window estimate is undefined (series too short for it) but the plateau
    was reached; otherwise None (no effective-sample rate is claimed)."""
    if t["sokal"] == t["sokal"]:
        t["estimator"] = "sokal"
        return t["sokal"]
    if t.get("binning_plateau") and t["binning"] == t["binning"]:
        t["estimator"] = "binning"
        return t["binning"]
    t["estimator"] = None
    return None


def reference_cuda_sampler(N):
    """The reference's own CUDA sampler (edgeMC::spectrum_compute, compiled from
    its sources for sm_100a by oracle/Makefile into oracle/_ref) timed on this
    GPU by its own cudaEvents around the row launch (em_spectrum.cu:273-287):
    one basis row (dL = 1) of its default grid, 32 x 128 walkers, 100 burn-in
    + 200 measured sweeps.  None when the build or a GPU is absent."""
    exe = ROOT / "oracle" / "_ref" / ("ref_edge200_e2" if N == 200 else "ref_edge_e2")
    if not exe.exists():
        return None
    with tempfile.TemporaryDirectory() as tmp:
        out = Path(tmp) / "ref.json"
        try:
            subprocess.run([str(exe), "spectrum", "1", "100", "200", "1", "0.3", "4242", "32",
                            str(out), str(Path(tmp) / "run")], check=True, timeout=600,
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            d = json.loads(out.read_text())
        except Exception as exc:  # reported, never required
            return {"error": str(exc)}
    ms = d["runs"][0]["kernel_ms"]
    return {"walker_sweeps_per_s_per_row": d["walkers"] * 300 / (sum(ms) * 1e-3),
            "kernel_ms_per_row": sum(ms) / len(ms), "particles": d["particles"],
            "walkers": d["walkers"], "sweeps_per_launch": 300,
            "note": "the reference's mcmc_hamiltonian, one basis row per launch; our "
                    "walker-sweep covers every row of every sector"}


def run_reference(args, ws, rank):
    if rank != 0:
        return
    w = MIXED if args.mixed else WORKLOAD
    cb = cpu_port(w)
    rc = reference_cuda_sampler(w["particles"])
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {k: w[k] for k in ("workload", "particles", "inverse_filling", "walkers")},
            "cpu_baseline": cb, "reference_cuda_sampler": rc,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def long_chain_tau(L, cfg, sectors, n_burn, n_meas, proposal=None, init_xy=None, tune=None):
    """tau_int of a sampler from a separate untimed chain: n_burn unmeasured and
    n_meas measured sweeps; the walker-mean p_1..p_4 series gives Sokal and
    binning estimates.  tune = (target, tol) tunes the step first."""
    smp = L.Sampler(cfg, sectors)
    if proposal is not None:
        smp.set_proposal(proposal)
    smp.init_walkers(init_xy)
    tuned = None
    if tune is not None:
        tuned = smp.tune_step(*tune)
    smp.run(n_burn, measure=False)
    smp.reset()
    smp.run(n_meas, measure=True)
    out = L.sampler.series_tau(smp.series())
    out["acceptance"] = smp.stats().acceptance
    if tuned is not None:
        out["sigma"] = tuned[0]
    smp.close()
    return out


def timed_steps(L, torch, cfg, sectors, steps, warmup, proposal=None, init_xy=None, clocks_index=None):
    """K full steps (sweep + record + basis + contraction of every sector) on the
    context stream, CUDA events around them; returns (ms, stats, clocks)."""
    smp = L.Sampler(cfg, sectors)
    if proposal is not None:
        smp.set_proposal(proposal)
    smp.init_walkers(init_xy)
    smp.run(warmup, measure=True)
    smp.reset()
    st_ = torch.cuda.ExternalStream(smp.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    smp.synchronize()
    torch.cuda.synchronize()
    clk = Clocks(clocks_index) if clocks_index is not None else None
    a.record(st_)
    smp.run(steps, measure=True)
    b.record(st_)
    b.synchronize()
    clocks = clk.stop() if clk else None
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    stats = smp.stats()
    smp.close()
    return ms, stats, clocks


def kernel_profile(L, cfg, sectors, steps, proposal=None, init_xy=None, burn=0):
    """Per-kernel device times (ms per launch) from a profiled pass: CUDA events
    between the sweep, basis and contraction launches of each step."""
    pc = dict(cfg.__dict__)
    pc.update(profile=True, graph_batch=0)
    smp = L.Sampler(L.SamplerConfig(**pc), sectors)
    if proposal is not None:
        smp.set_proposal(proposal)
    smp.init_walkers(init_xy)
    if burn:
        smp.run(burn, measure=False)
    smp.run(steps, measure=True)
    st = smp.stats()
    smp.close()
    return st.ms_sweep / steps, st.ms_basis / steps, st.ms_gram / steps


def learned_move_flop(N, reverse=1.0, k_nn=16, hidden=64):
    """Algorithmic FP32 FLOP of one learned move: the network evaluation at z
    (phi: k_nn x 2 -> hidden, rho: hidden+1 -> hidden, head: hidden -> 4; 2
    FLOP per multiply-add) with its kNN distance scan (3 FLOP per other
    particle), the Jastrow ratio (12 FLOP per pair term), and, for the share
    `reverse` of moves whose reverse density can change the decision, the
    second evaluation and scan at z'."""
    net = 2 * (k_nn * 2 * hidden + (hidden + 1) * hidden + hidden * 4)
    return (1.0 + reverse) * (net + 3 * (N - 1)) + 12 * (N - 1)


def rooflines(L, w, mode, t_sweep, t_basis, t_gram, learned, clocks, reverse=1.0):
    peaks, peak_kind = measured_peaks()
    N, W = w["particles"], w["walkers"]
    sd2, D = sum_d2(w["sectors"], N)
    K = max(4, max(w["sectors"]))
    fp32_peak = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) / 1e6  # TFLOP/s, nominal at max clock
    if learned:
        flop_sweep = W * N * learned_move_flop(N, reverse)
    else:
        flop_sweep = W * (12.0 * N * (N - 1) + N * (16.0 * K + 40.0))
    bytes_basis = W * (8.0 * D + 8.0 * K)
    flop_gram = W * 8.0 * 3 * sd2
    traffic = traffic_from_profiles()
    tag = w["workload"]
    tf32_peak = peaks["bf16_tflops"] / 2.0 if mode == L._lib.GRAM_TF32X3 else peaks["bf16_tflops"]
    roofs = {
        "sweep": {"bound": "fp32", "achieved": flop_sweep / (t_sweep * 1e-3) / 1e12,
                  "peak": fp32_peak, "unit": "TFLOP/s",
                  "peak_source": "nominal FP32 (148 SMs x 128 lanes x 2 x max SM clock)",
                  "kernel": "learned_sweep_kernel" if learned else "sweep_kernel",
                  "traffic": traffic.get(("learned_sweep" if learned else "sweep") + "@" + tag),
                  "ms_per_launch": t_sweep},
        "basis": {"bound": "hbm", "achieved": bytes_basis / (t_basis * 1e-3) / 1e9,
                  "peak": peaks["hbm_gbs"], "unit": "GB/s", "peak_source": f"{peak_kind} hbm_gbs",
                  "kernel": "basis_kernel", "traffic": traffic.get("basis@" + tag),
                  "ms_per_launch": t_basis},
        "gram": {"bound": "tensor", "achieved": flop_gram / (t_gram * 1e-3) / 1e12,
                 "peak": tf32_peak, "unit": "TFLOP/s",
                 "peak_source": (f"{peak_kind} bf16_tflops / 2 (dense TF32 rate)" if mode == L._lib.GRAM_TF32X3
                                 else f"{peak_kind} bf16_tflops"),
                 "kernel": "gram_tc_kernel", "traffic": traffic.get("gram@" + tag),
                 "ms_per_launch": t_gram},
    }
    for r in roofs.values():
        r["frac"] = r["achieved"] / r["peak"]
    return roofs


def ratio(a, b):
    x, y = a["effective_samples_per_s"], b["effective_samples_per_s"]
    return x / y if x and y else None


def run_ours(args, ws, rank, local):
    import numpy as np
    import torch

    import laughlinedge_b200 as L
    w = WORKLOAD
    torch.cuda.set_device(local)
    N, m, W = w["particles"], w["inverse_filling"], w["walkers"]
    mode = gram_mode_id(args.gram or w["gram_mode"])
    seed = rank_seed(w["seed"], rank)
    sectors = w["sectors"]
    gb = args.graph_batch

    # 1) burnt-in plain chain: the common start of every sampler, and the
    #    training configurations of the proposal
    plain0 = L.Sampler(L.SamplerConfig(N, m, W, step_sigma=w["sigma"], seed=seed,
                                       lanes_per_walker=-1), [1, 2, 3, 4])
    plain0.init_walkers()
    plain0.run(args.burn, measure=False)
    G = plain0.lanes_per_walker()
    n_snap = w["train_configs"] // W
    cfg_buf = torch.empty((n_snap * W, N, 2), dtype=torch.float32, device="cuda")
    for k in range(n_snap):
        plain0.run(10, measure=False)
        plain0.copy_positions_device(cfg_buf[k * W:(k + 1) * W].data_ptr())
    start_xy = plain0.positions()
    plain0.close()
    # the plain step tuned to 50 % acceptance (the reference's criterion,
    # em_bisection.cu:49-153) on a copy of the burnt-in walkers; the proposal
    # starts from that isotropic step, so training can only improve on it
    tctx = L.Sampler(L.SamplerConfig(N, m, w["tau_walkers"], step_sigma=w["sigma"], seed=seed + 3,
                                     lanes_per_walker=G), [1, 2, 3, 4])
    tctx.init_walkers(start_xy[:w["tau_walkers"]])
    sigma_tuned, _ = tctx.tune_step(0.5, 0.01, 100)
    tctx.close()
    prop = L.LearnedProposal(N, m, init_sigma=sigma_tuned, seed=w["seed"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    trace = prop.train(cfg_buf.data_ptr(), cfg_buf.shape[0], steps=w["train_steps"],
                       batch=w["train_batch"], pairs=w["train_pairs"], lr=3e-3, es_sigma=0.02,
                       seed=w["seed"])
    t_train = time.perf_counter() - t0
    del cfg_buf

    # 2) tau_int of each sampler from separate untimed long chains
    Wt = w["tau_walkers"]
    tau_xy = start_xy[:Wt]
    mk = lambda WW, sg, lanes=G, **kw: L.SamplerConfig(N, m, WW, step_sigma=sg, seed=seed + 7,
                                                        lanes_per_walker=lanes, **kw)
    tau_plain = long_chain_tau(L, mk(Wt, w["sigma"]), [1, 2, 3, 4], 200, w["tau_sweeps_plain"],
                               init_xy=tau_xy)
    tau_tuned = long_chain_tau(L, mk(Wt, sigma_tuned), [1, 2, 3, 4], 200, w["tau_sweeps_plain"],
                               init_xy=tau_xy)
    tau_tuned["sigma"] = sigma_tuned
    tau_learned = long_chain_tau(L, mk(Wt, w["sigma"], lanes=0), [1, 2, 3, 4], 200,
                                 w["tau_sweeps_learned"], proposal=prop, init_xy=tau_xy)

    # 3) timed full steps of each sampler at W = 65536, all 20 sectors
    full = lambda sg: L.SamplerConfig(N, m, W, step_sigma=sg, seed=seed + 11, lanes_per_walker=G,
                                      gram_mode=mode, graph_batch=gb)
    if ws > 1:
        torch.distributed.barrier()
    ms_l, st_l, clocks = timed_steps(L, torch, full(w["sigma"]), sectors, args.steps, args.warmup,
                                     proposal=prop, init_xy=start_xy, clocks_index=local)
    ms_p, st_p, _ = timed_steps(L, torch, full(w["sigma"]), sectors, args.steps, args.warmup,
                                init_xy=start_xy)
    ms_t, st_t, _ = timed_steps(L, torch, full(sigma_tuned), sectors, args.steps, args.warmup,
                                init_xy=start_xy)
    if ws > 1:
        torch.distributed.barrier()
    ms_max = allreduce_max(ms_l, ws)
    sd2, D = sum_d2(sectors, N)
    total = W * args.steps * ws
    tv_l, tv_p, tv_t = tau_value(tau_learned), tau_value(tau_plain), tau_value(tau_tuned)
    value = total / tv_l / (ms_max * 1e-3) if tv_l else None
    arms = {}
    for name, ms, tau, tv, st, sg in (
            ("learned", ms_max, tau_learned, tv_l, st_l, w["sigma"]),
            ("plain_equal_sigma", allreduce_max(ms_p, ws), tau_plain, tv_p, st_p, w["sigma"]),
            ("plain_tuned_sigma", allreduce_max(ms_t, ws), tau_tuned, tv_t, st_t, sigma_tuned)):
        arms[name] = {"effective_samples_per_s": total / tv / (ms * 1e-3) if tv else None,
                      "ms_per_step": ms / args.steps, "sigma": sg, "tau_int": tv,
                      "tau_int_chain": tau, "acceptance_timed": st.acceptance,
                      "walker_sweeps_per_s": total / (ms * 1e-3)}
    sh_updates = total * sd2 * 3 / (ms_max * 1e-3)

    # 4) per-kernel device times (profiled pass) and rooflines, learned and plain
    npro = 5
    ks_l = kernel_profile(L, full(w["sigma"]), sectors, npro, proposal=prop, init_xy=start_xy)
    ks_p = kernel_profile(L, full(w["sigma"]), sectors, npro, init_xy=start_xy)
    roofs = rooflines(L, w, mode, *ks_l, True, clocks, reverse=st_l.reverse_fraction)
    roofs["sweep"]["reverse_fraction"] = st_l.reverse_fraction
    roofs_plain = rooflines(L, w, mode, *ks_p, False, clocks)
    dominant = max(roofs, key=lambda k: roofs[k]["ms_per_launch"])
    # the mixed-precision workload's rooflines (N = 50, dL = 0..12), plain sampler
    wm = MIXED
    cm = L.SamplerConfig(wm["particles"], m, wm["walkers"], step_sigma=wm["sigma"], seed=seed,
                         lanes_per_walker=4, gram_mode=mode)
    ks_m = kernel_profile(L, cm, wm["sectors"], 20, burn=400)
    roofs_mixed = rooflines(L, wm, mode, *ks_m, False, None)

    # 5) end to end through the public API with host buffers (learned sampler)
    e_steps = max(10, min(args.steps, 40))
    host = torch.from_numpy(start_xy).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    esmp = L.Sampler(L.SamplerConfig(N, m, W, step_sigma=w["sigma"], seed=seed + 13,
                                     lanes_per_walker=G, gram_mode=mode), sectors)
    esmp.set_proposal(prop)
    esmp.init_walkers(host.numpy())
    for _ in range(e_steps):
        esmp.run(1, measure=True)  # per step: device work + d2h of the step's series entry
    grams = [esmp.gram(s) for s in range(len(sectors))]
    for S, H2, H4, _ in grams:
        L.normalise(S, H2, H4, w["omega"], w["kappa"])
    t_e2e = time.perf_counter() - t0
    esmp.close()
    h2d = W * N * 8
    d2h = 64 * e_steps + sum(3 * 16 * g_[0].size for g_ in grams)
    e2e = {"value": W * e_steps * ws / tv_l / t_e2e if tv_l else None, "unit": UNIT,
           "h2d_bytes_per_step": h2d / e_steps, "d2h_bytes_per_step": d2h / e_steps,
           "steps": e_steps, "tau_int_used": tv_l,
           "note": "lemc_create + init from pinned host positions + per-step lemc_run(1) with "
                   "series read-back + Gram read-back and normalisation of 20 sectors, wall clock"}
    prop.close()
    if rank != 0:
        return
    cb = None
    if not args.no_cpu_baseline:
        try:
            cb = cpu_port(w)
            cb["tau_int_gpu_plain_same_sigma"] = tau_plain["sokal"]
        except Exception as exc:  # the baseline is reported, never required
            cb = {"error": str(exc)}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+bf16-net+tf32x3" if mode == L._lib.GRAM_TF32X3 else "f32+bf16-net",
        "data": "synthetic",
        "config": {"workload": w["workload"], "particles": N, "inverse_filling": m,
                   "omega": w["omega"], "kappa": w["kappa"], "sectors": "1..20",
                   "basis_states": D, "sum_d2": sd2, "walkers_per_gpu": W, "sigma": w["sigma"],
                   "sampler": "learned DeepSets proposal (exact MH)",
                   "gram_mode": args.gram or w["gram_mode"], "lanes_per_walker_plain": G,
                   "graph_batch": gb, "l2": "inputs larger than L2 (V planes 1.4 GB per step)",
                   "parallelism": f"replicas x{ws} (walkers sharded, no collective)"},
        "tau_int": tv_l,
        "tau_source": f"Sokal window on a separate untimed chain: {Wt} walkers, "
                      f"{w['tau_sweeps_learned']} measured sweeps after 200 burn-in, from the "
                      f"burnt-in plain configurations (binning plateau beside it)",
        "samplers": arms,
        "learned_over_plain_equal_sigma": ratio(arms["learned"], arms["plain_equal_sigma"]),
        "learned_over_plain_tuned_sigma": ratio(arms["learned"], arms["plain_tuned_sigma"]),
        "sh_updates_per_s": sh_updates, "walker_sweeps_per_s": total / (ms_max * 1e-3),
        "kernel_ms": {"sweep": ks_l[0], "basis": ks_l[1], "gram": ks_l[2]},
        "roofline": dict(roofs[dominant], which=dominant),
        "rooflines": roofs, "rooflines_plain_sampler": roofs_plain,
        "rooflines_mixed_precision_N50": dict(roofs_mixed, workload=wm["workload"]),
        "train_seconds": t_train,
        "train_objective_first_last": [float(np.mean(trace[:50])), float(np.mean(trace[-50:]))],
        "clocks": clocks,
        # per step: sweep, basis, contraction (+ the counter kernel inside a graph)
        "gpu_launches": (4 * (args.steps // gb) * gb + 3 * (args.steps % gb)) if gb else 3 * args.steps,
        "e2e": e2e,
        "cpu_baseline": cb,
    }
    print(json.dumps(line), flush=True)


def run_mixed(args, ws, rank, local):
    """Mixed-precision line: N = 50, dL = 0..12 (272 states), plain step
    sigma = 0.3, TF32x3 contraction, W = 65536; tau_int from a separate
    4000-sweep chain."""
    import numpy as np
    import torch

    import laughlinedge_b200 as L
    w = MIXED
    torch.cuda.set_device(local)
    N, m, W = w["particles"], w["inverse_filling"], w["walkers"]
    mode = gram_mode_id(args.gram or w["gram_mode"])
    seed = rank_seed(w["seed"], rank)
    p0 = L.Sampler(L.SamplerConfig(N, m, W, step_sigma=w["sigma"], seed=seed, lanes_per_walker=-1),
                   [1, 2, 3, 4])
    p0.init_walkers()
    p0.run(args.burn, measure=False)
    G = p0.lanes_per_walker()
    start_xy = p0.positions()
    p0.close()
    tau = long_chain_tau(L, L.SamplerConfig(N, m, w["tau_walkers"], step_sigma=w["sigma"],
                                            seed=seed + 7, lanes_per_walker=G),
                         [1, 2, 3, 4], 200, w["tau_sweeps"], init_xy=start_xy[:w["tau_walkers"]])
    cfg = L.SamplerConfig(N, m, W, step_sigma=w["sigma"], seed=seed + 11, lanes_per_walker=G,
                          gram_mode=mode, graph_batch=args.graph_batch)
    ms, st, clocks = timed_steps(L, torch, cfg, w["sectors"], args.steps, args.warmup,
                                 init_xy=start_xy, clocks_index=local)
    ms_max = allreduce_max(ms, ws)
    sd2, D = sum_d2(w["sectors"], N)
    total = W * args.steps * ws
    ks = kernel_profile(L, cfg, w["sectors"], 40, init_xy=start_xy)
    roofs = rooflines(L, w, mode, *ks, False, clocks)
    dominant = max(roofs, key=lambda k: roofs[k]["ms_per_launch"])
    if rank != 0:
        return
    tv = tau_value(tau)
    line = {"metric": METRIC, "value": total / tv / (ms_max * 1e-3) if tv else None, "unit": UNIT,
            "workload": w["workload"], "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "data": "synthetic",
            "dtype": "f32+tf32x3", "config": {k: w[k] for k in w if k != "sectors"},
            "tau_int": tv, "tau_int_chain": tau, "acceptance": st.acceptance,
            "sh_updates_per_s": total * sd2 * 3 / (ms_max * 1e-3),
            "walker_sweeps_per_s": total / (ms_max * 1e-3),
            "kernel_ms": {"sweep": ks[0], "basis": ks[1], "gram": ks[2]},
            "roofline": dict(roofs[dominant], which=dominant), "rooflines": roofs, "clocks": clocks}
    print(json.dumps(line), flush=True)


BATCHED = {
    "workload": "batched_m3_N100_dL1-20_W131072",
    "particles": 100, "inverse_filling": 3, "omega": 2e-3, "sectors": list(range(1, 21)),
    "kappas": "16 log-spaced in [1e-6, 1e-4]", "walkers": 131072, "sigma": 0.3, "seed": 42,
    "gram_mode": "tf32x3", "graph_batch": 8,
}


def run_batched(args, rank, local):
    """Batched form: all 20 sectors (2713 states) and 16 quartic strengths.

    Timed region: `steps` measured sweeps (sweep, basis, TF32x3 contraction
    of S, H2, H4 for every sector) as CUDA-graph replays, CUDA events.  Then
    the FP64 GPU tail solves every sector for the 16 strengths
    (lemc_geneig_sweep), timed on the host clock."""
    if rank != 0:
        return
    import numpy as np
    import torch

    import laughlinedge_b200 as L
    w = BATCHED
    torch.cuda.set_device(local)
    N, m, W = w["particles"], w["inverse_filling"], w["walkers"]
    steps = max(8, min(args.steps, 64))
    steps -= steps % w["graph_batch"]
    smp = L.Sampler(L.SamplerConfig(N, m, W, step_sigma=w["sigma"], seed=w["seed"],
                                    lanes_per_walker=-1, gram_mode=L._lib.GRAM_TF32X3,
                                    graph_batch=w["graph_batch"]), w["sectors"])
    smp.init_walkers()
    smp.run(args.burn, measure=False)
    smp.run(max(args.warmup, w["graph_batch"]), measure=True)
    smp.reset()
    st_ = torch.cuda.ExternalStream(smp.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    smp.synchronize()
    clk = Clocks(local)
    a.record(st_)
    smp.run(steps, measure=True)
    b.record(st_)
    b.synchronize()
    clocks = clk.stop()
    ms = a.elapsed_time(b) / steps
    sd2, D = sum_d2(w["sectors"], N)
    grams = [smp.gram(s)[:3] for s in range(len(w["sectors"]))]
    acc = smp.stats().acceptance
    G = smp.lanes_per_walker()
    smp.close()
    kap = np.logspace(-6, -4, 16)
    t0 = time.perf_counter()
    lowest = []
    for S, H2, H4 in grams:
        ev, _ = L.geneig_sweep(S, H2, H4, np.full(16, w["omega"]), kap, eps=1e-10)
        lowest.append(float(ev[0, 0]))
    t_tail = time.perf_counter() - t0
    sh = W * sd2 * 3 / (ms * 1e-3)
    line = {"metric": "sh_updates_per_s", "value": sh, "unit": "updates/s", "workload": w["workload"],
            "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "dtype": "f32+tf32x3", "data": "synthetic",
            "config": dict({k: w[k] for k in w if k not in ("workload", "sectors")},
                           basis_states=D, sum_d2=sd2, lanes_per_walker=G),
            "walker_sweeps_per_s": W / (ms * 1e-3), "acceptance": acc,
            "contraction_tflops_algorithmic": W * 8.0 * 3 * sd2 / (ms * 1e-3) / 1e12,
            "kappa_sweep_tail_s": t_tail, "kappa_sweep_problems": 16 * len(grams),
            "lowest_level_per_sector_kappa0": lowest, "clocks": clocks}
    print(json.dumps(line), flush=True)


EVOLUTION = {
    "workload": "time_evolution_m3_N100_dL0-16even_W65536",
    "particles": 100, "inverse_filling": 3, "omega": 2e-3, "kappa": 2e-5,
    "sectors": list(range(0, 17, 2)), "k": 2, "eps": 1e-3, "t0": 50.0, "tau": 10.0,
    "walkers": 65536, "sigma": 0.3, "seed": 42, "dt": 0.05, "steps": 4000, "n_theta": 256,
    "burn": 1000, "sweeps": 200, "train_configs": 1 << 20, "train_steps": 5000,
}


def run_evolution(args, rank, local):
    """Time-evolution pipeline: the DeepSets proposal trained on the plain
    chain; matrix elements of sectors {0, 2, ..., 16} (526 states) under the
    drive r^2 cos(2 theta) with the learned proposal and the TF32x3
    contraction; FP64 RK4 evolution of 4000 steps of dt = 0.05 in the
    S-orthonormal basis on the GPU; delta rho(theta, t) on 256 angles.  Each
    stage timed on the host clock after a device synchronisation."""
    if rank != 0:
        return
    import numpy as np
    import torch

    import laughlinedge_b200 as L
    w = EVOLUTION
    torch.cuda.set_device(local)
    N, m, W = w["particles"], w["inverse_filling"], w["walkers"]
    t_all = time.perf_counter()
    p0 = L.Sampler(L.SamplerConfig(N, m, W, step_sigma=w["sigma"], seed=w["seed"], lanes_per_walker=-1),
                   [1, 2, 3, 4])
    p0.init_walkers()
    p0.run(w["burn"], measure=False)
    n_snap = w["train_configs"] // W
    buf = torch.empty((n_snap * W, N, 2), dtype=torch.float32, device="cuda")
    for k in range(n_snap):
        p0.run(10, measure=False)
        p0.copy_positions_device(buf[k * W:(k + 1) * W].data_ptr())
    start_xy = p0.positions()
    p0.close()
    tctx = L.Sampler(L.SamplerConfig(N, m, 8192, step_sigma=w["sigma"], seed=w["seed"] + 3), [1, 2])
    tctx.init_walkers(start_xy[:8192])
    sigma_tuned, _ = tctx.tune_step(0.5, 0.01, 100)
    tctx.close()
    prop = L.LearnedProposal(N, m, init_sigma=sigma_tuned, seed=w["seed"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    prop.train(buf.data_ptr(), buf.shape[0], steps=w["train_steps"], batch=1024, pairs=32, lr=3e-3,
               es_sigma=0.02, seed=w["seed"])
    t_train = time.perf_counter() - t0
    del buf
    prof = lambda t: w["eps"] * math.exp(-((t - w["t0"]) ** 2) / (2 * w["tau"] ** 2))
    out = L.edge_response(N, m, w["sectors"], w["k"], w["omega"], w["kappa"], prof,
                          end_time=w["steps"] * w["dt"], save_step=w["dt"], n_walkers=W, burn_in=100,
                          sweeps=w["sweeps"], step_sigma=sigma_tuned, seed=w["seed"] + 1,
                          gram_mode=L._lib.GRAM_TF32X3, proposal=prop, substeps=1,
                          n_theta=w["n_theta"], init_xy=start_xy, graph_batch=args.graph_batch)
    prop.close()
    dens = out["density"]
    rho_t = out["rho_t"]
    D = out["M"].shape[0]
    line = {"metric": "edge_density_response_pipeline_s", "value": sum(out["timings"].values()),
            "unit": "s", "workload": w["workload"], "n_gpus": 1, "higher_is_better": False,
            "data": "synthetic", "dtype": "f32+bf16-net+tf32x3 sampling, f64 evolution",
            "config": {k: w[k] for k in w if k != "sectors"}, "basis_states": D,
            "timings_s": dict(out["timings"], train_proposal_s=t_train),
            "sampling_walker_sweeps_per_s": W * (w["sweeps"] + 100) / out["timings"]["sampling_s"],
            "evolution_steps_per_s": w["steps"] / out["timings"]["evolution_s"],
            "acceptance": out["acceptance"], "rank": out["rank"],
            "norm_drift": float(np.max(np.abs(out["norms"] - 1.0))),
            "max_abs_delta_rho": float(np.max(np.abs(dens))),
            "max_abs_delta_rho_l": [float(np.max(np.abs(rho_t[:, q] - rho_t[0, q])))
                                   for q in range(rho_t.shape[1])],
            "n_times": int(dens.shape[0]), "n_theta": int(dens.shape[1]),
            "total_wall_s": time.perf_counter() - t_all}
    print(json.dumps(line), flush=True)


def run_occupation(args, rank, local):
    """Orbital occupations of the two-state walker (lemc_occupation) for every
    (L, R) row pair of one sector in one launch: N = 50, m = 3, dL = 4 (25
    pairs), l_cutoff = m (N - 1) + 15, W = 65536 walkers split over the pairs,
    50 burn-in + 100 measured sweeps.  Timed on the host clock around the
    public call (allocation, launch and read-back included) after a warm-up
    call; beside it the oracle's C restatement of the reference's walker on
    the host cores, one pair, a bounded sample."""
    if rank != 0:
        return
    import os

    import laughlinedge_b200 as L
    import torch
    torch.cuda.set_device(local)
    N, m, dL, W, burn, meas = 50, 3, 4, 65536, 50, 100
    Lc = m * (N - 1) + 15
    L.sampler.occupation(N, m, dL, Lc, W, 10, burn_in=5)
    t0 = time.perf_counter()
    _, acc = L.sampler.occupation(N, m, dL, Lc, W, meas, burn_in=burn)
    t = time.perf_counter() - t0
    rate = W * (burn + meas) / t
    line = {"metric": "occupation_walker_sweeps_per_s", "value": rate, "unit": "walker-sweeps/s",
            "n_gpus": 1, "higher_is_better": True, "data": "synthetic", "dtype": "f32+f64",
            "config": {"workload": "occupation_m3_N50_dL4_W65536", "particles": N,
                       "inverse_filling": m, "dL": dL, "l_cutoff": Lc, "walkers": W,
                       "burn_in": burn, "sweeps": meas, "row_pairs": 25},
            "seconds": t, "acceptance": acc}
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        th = os.cpu_count() or 1
        Wc, bc, mc = 64 * th, 100, 2000
        t0 = time.perf_counter()
        O.occupation(N, m, Wc, 0.3, 42, bc, mc, dL, 0, 0, Lc, nthreads=th)
        tc = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": Wc * (bc + mc) / tc, "unit": "walker-sweeps/s",
                                "cores": th, "kind": "port",
                                "sample": f"{Wc} walkers x ({bc} + {mc}) sweeps of one row pair, {tc:.1f} s"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--burn", type=int, default=1000, help="untimed burn-in sweeps")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--gram", default=None, choices=["fp64", "bf16x3", "bf16x4", "tf32x3"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mixed", action="store_true",
                    help="mixed-precision form N=50, dL 0..12 (its own JSON line)")
    ap.add_argument("--batched", action="store_true",
                    help="batched form N=100, dL 1..20, 16 kappas (its own JSON line)")
    ap.add_argument("--evolution", action="store_true",
                    help="time-evolution pipeline N=100, dL 0,2..16 (its own JSON line)")
    ap.add_argument("--occupation", action="store_true",
                    help="two-state walker occupations N=50, dL 4 (its own JSON line)")
    ap.add_argument("--graph-batch", type=int, default=4,
                    help="measured steps per CUDA-graph replay in the timed run (0: direct launches)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_init()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        elif args.batched:
            run_batched(args, rank, local)
        elif args.evolution:
            run_evolution(args, rank, local)
        elif args.occupation:
            run_occupation(args, rank, local)
        elif args.mixed:
            run_mixed(args, ws, rank, local)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
