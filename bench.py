#!/usr/bin/env python
"""Benchmark of the LaughlinEdge B200 engine on the mixed-precision workload.

Workload (one GPU): Laughlin nu = 1/3 (m = 3), N = 50 electrons, confinement
V = omega r^2 + kappa r^4 with omega = 5e-3, kappa = 2e-5, edge sectors
dL = 0..12 (272 power-sum states), 65536 walkers, Gaussian step sigma = 0.3,
Philox seed 42, basis in FP32 with (z/R)^k scaling, S/H contraction in
TF32 hi/lo split precision on tcgen05 with FP32 accumulation flushed to FP64.
Synthetic by construction: walkers start uniformly in the disk of radius
sqrt(2 m N) and are burnt in before timing.

A step is one pass of the hot path over all walkers: one Metropolis sweep
(N single-particle moves per walker), one measurement record, the basis build
and the S, H2, H4 contraction.  Metric: effective samples/s
= walkers x steps / tau_int / time, tau_int the integrated autocorrelation time
(in sweeps) of p_1..p_4, max over the four, measured on the timed steps.

``--impl reference`` times the oracle's C restatement of the reference
estimator (one Metropolis chain per basis row guided by |P_a Psi|^2, per-row
ratio sums) on all host cores, on a bounded sample of the same workload.
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
    "workload": "mixed_precision_m3_N50_dL0-12_W65536",
    "particles": 50,
    "inverse_filling": 3,
    "omega": 5e-3,
    "kappa": 2e-5,
    "sectors": list(range(13)),
    "walkers": 65536,
    "sigma": 0.3,
    "seed": 42,
    "gram_mode": "tf32x3",
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
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


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


def cpu_baseline(w, steps_hint=None, threads=0, budget_s=15.0):
    """The oracle's restatement of the reference estimator on the host cores."""
    from oracle import oracle as O
    O.load()
    nth = threads or O.load().orc_max_threads()
    N, m = w["particles"], w["inverse_filling"]
    # calibrate on a tiny run, then size the sample to the budget
    wc = 8 * nth
    t0 = time.perf_counter()
    O.run_rows(N, m, wc, w["sigma"], w["seed"], 10, 30, w["sectors"], nthreads=nth)
    per = (time.perf_counter() - t0) / (wc * 40)  # seconds per walker-sweep (all cores)
    n_meas = int(steps_hint or 1000)
    W = max(nth, int(budget_s / max(per, 1e-9) / (n_meas + 50)))
    W = min(W, 4096)
    t0 = time.perf_counter()
    res = O.run_rows(N, m, W, w["sigma"], w["seed"], 50, n_meas, w["sectors"], nthreads=nth)
    dt = time.perf_counter() - t0
    taus = O.tau_int(res["series"])
    tau = float(max(0.5 * (taus[2 * k] + taus[2 * k + 1]) for k in range(4)))
    value = W * n_meas / tau / dt
    return {"value": value, "unit": UNIT, "cores": nth, "kind": "port",
            "sample": f"{W} walkers x ({n_meas} measured + 50 burn-in) sweeps of the per-row "
                      f"reference estimator, all 272 rows, tau_int={tau:.2f} sweeps, "
                      f"{dt:.1f} s wall", "walker_sweeps_per_s": W * (n_meas + 50) / dt,
            "tau_int": tau}


def run_reference(args, ws, rank):
    if rank != 0:
        return
    w = WORKLOAD
    cb = cpu_baseline(w, steps_hint=min(max(args.steps, 200), 2000))
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {k: w[k] for k in ("workload", "particles", "inverse_filling", "walkers")},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, ws, rank, local):
    import numpy as np
    import torch

    import laughlinedge_b200 as L
    w = WORKLOAD
    torch.cuda.set_device(local)
    N, m, W = w["particles"], w["inverse_filling"], w["walkers"]
    mode = gram_mode_id(args.gram or w["gram_mode"])
    seed = w["seed"] + 1000003 * rank
    cfg = L.SamplerConfig(N, m, W, step_sigma=w["sigma"], seed=seed, lanes_per_walker=-1,
                          gram_mode=mode, graph_batch=args.graph_batch)
    smp = L.Sampler(cfg, w["sectors"])
    smp.init_walkers()
    smp.run(args.burn, measure=False)
    smp.run(args.warmup, measure=True)
    smp.reset()
    stream = torch.cuda.ExternalStream(smp.stream())
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    start.record(stream)
    smp.run(args.steps, measure=True)
    end.record(stream)
    end.synchronize()
    clocks = clk.stop()
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    if ws > 1:
        torch.distributed.barrier()
    st = smp.stats()
    tau = st.tau_int
    ms_max = allreduce_max(ms, ws)
    sd2, D = sum_d2(w["sectors"], N)
    total_samples = W * args.steps * ws
    value = total_samples / tau / (ms_max * 1e-3)
    sh_updates = total_samples * sd2 * 3 / (ms_max * 1e-3)

    # per-kernel device times (separate profiled pass, events between kernels)
    G = smp.lanes_per_walker()
    psmp = L.Sampler(L.SamplerConfig(N, m, W, step_sigma=w["sigma"], seed=seed + 7,
                                     lanes_per_walker=G, gram_mode=mode,
                                     profile=True), w["sectors"])
    psmp.init_walkers()
    psmp.run(args.burn // 4, measure=False)
    npro = min(200, max(20, args.steps // 5))
    psmp.run(npro, measure=True)
    pst = psmp.stats()
    t_sweep, t_basis, t_gram = pst.ms_sweep / npro, pst.ms_basis / npro, pst.ms_gram / npro
    psmp.close()

    peaks, peak_kind = measured_peaks()
    K = max(4, max(w["sectors"]))
    clk_ghz = (clocks or {}).get("sm_mhz", peaks.get("sm_max_mhz", 1965.0)) / 1e3
    fp32_peak = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) / 1e6  # TFLOP/s, nominal at max clock
    flop_sweep = W * (12.0 * N * (N - 1) + N * (16.0 * K + 40.0))
    bytes_basis = W * (8.0 * D + 8.0 * K)
    flop_gram = W * 8.0 * 3 * sd2
    traffic = traffic_from_profiles()
    tf32_peak = peaks["bf16_tflops"] / 2.0 if mode == L._lib.GRAM_TF32X3 else peaks["bf16_tflops"]
    roofs = {
        "sweep": {"bound": "fp32", "achieved": flop_sweep / (t_sweep * 1e-3) / 1e12,
                  "peak": fp32_peak, "unit": "TFLOP/s",
                  "peak_source": "nominal FP32 (148 SMs x 128 lanes x 2 x max SM clock)",
                  "traffic": traffic.get("sweep"), "ms_per_launch": t_sweep},
        "basis": {"bound": "hbm", "achieved": bytes_basis / (t_basis * 1e-3) / 1e9,
                  "peak": peaks["hbm_gbs"], "unit": "GB/s", "peak_source": f"{peak_kind} hbm_gbs",
                  "traffic": traffic.get("basis"), "ms_per_launch": t_basis},
        "gram": {"bound": "tensor", "achieved": flop_gram / (t_gram * 1e-3) / 1e12,
                 "peak": tf32_peak, "unit": "TFLOP/s",
                 "peak_source": (f"{peak_kind} bf16_tflops / 2 (dense TF32 rate)" if mode == L._lib.GRAM_TF32X3
                                 else f"{peak_kind} bf16_tflops"),
                 "traffic": traffic.get("gram"), "ms_per_launch": t_gram},
    }
    for r in roofs.values():
        r["frac"] = r["achieved"] / r["peak"]
    dominant = max(roofs, key=lambda k: roofs[k]["ms_per_launch"])
    G = smp.lanes_per_walker()
    smp.close()

    # end-to-end through the public API with host buffers
    e2e = None
    if rank == 0 or ws > 1:
        g = np.random.default_rng(seed)
        r0 = math.sqrt(2 * m * N)
        rr = r0 * np.sqrt(g.random((W, N)))
        th = 2 * math.pi * g.random((W, N))
        host = torch.from_numpy(np.stack([rr * np.cos(th), rr * np.sin(th)], -1).astype(np.float32)).pin_memory()
        e_steps = max(50, args.steps // 4)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        esmp = L.Sampler(L.SamplerConfig(N, m, W, step_sigma=w["sigma"], seed=seed + 11,
                                         lanes_per_walker=G, gram_mode=mode),
                         w["sectors"])
        esmp.init_walkers(host.numpy())
        for _ in range(e_steps):
            esmp.run(1, measure=True)  # per step: device work + d2h of the step's series entry
        grams = [esmp.gram(s) for s in range(len(w["sectors"]))]
        for s, (S, H2, H4, _) in enumerate(grams):
            Mn, Hn = L.normalise(S, H2, H4, w["omega"], w["kappa"])
        t_e2e = time.perf_counter() - t0
        etau = esmp.stats().tau_int
        esmp.close()
        h2d = W * N * 8
        d2h = 64 * e_steps + sum(3 * 16 * g_[0].size for g_ in grams)
        # tau_int is a property of the chain, not of the call path: the same
        # estimate (from the longer device-timed run) converts both arms, the
        # shorter run's own estimate is reported beside it.
        e2e = {"value": W * e_steps * ws / tau / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": h2d / e_steps, "d2h_bytes_per_step": d2h / e_steps,
               "steps": e_steps, "tau_int_used": tau, "tau_int_this_run": etau,
               "note": "lemc_create + init from pinned host positions + per-step lemc_run(1) with "
                       "series read-back + Gram read-back + normalisation, wall clock"}

    if rank != 0:
        return
    cb = None
    if not args.no_cpu_baseline:
        try:
            cb = cpu_baseline(w, steps_hint=min(args.steps, 1000))
        except Exception as exc:  # the baseline is reported, never required
            cb = {"error": str(exc)}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+tf32x3" if mode == L._lib.GRAM_TF32X3 else "f32",
        "data": "synthetic",
        "config": {"workload": w["workload"], "particles": N, "inverse_filling": m,
                   "sectors": "0..12", "basis_states": D, "walkers_per_gpu": W,
                   "sigma": w["sigma"], "gram_mode": args.gram or w["gram_mode"],
                   "lanes_per_walker": G, "graph_batch": args.graph_batch,
                   "l2": "inputs larger than L2 (V planes 143 MB per step)",
                   "parallelism": f"replicas x{ws} (walkers sharded, no collective)"},
        "tau_int": tau, "tau_int_each": list(st.tau_int_each), "acceptance": st.acceptance,
        "sh_updates_per_s": sh_updates, "walker_sweeps_per_s": total_samples / (ms_max * 1e-3),
        "kernel_ms": {"sweep": t_sweep, "basis": t_basis, "gram": t_gram},
        "roofline": dict(roofs[dominant], kernel=dominant),
        "rooflines": roofs,
        "clocks": clocks,
        "gpu_launches": 3 * args.steps,
        "e2e": e2e,
        "cpu_baseline": cb,
    }
    print(json.dumps(line), flush=True)


LEARNED = {
    "workload": "learned_proposal_m3_N200",
    "particles": 200, "inverse_filling": 3, "omega": 1e-3, "kappa": 5e-6,
    "sigma": 0.3, "walkers": 65536, "tau_walkers": 8192, "seed": 42,
    "train_configs": 1 << 20, "train_steps": 5000, "train_batch": 1024, "train_pairs": 32,
}


def run_learned(args, rank, local):
    """Learned vs plain single-particle proposal at equal sigma (N=200, m=3).

    One line: walker-sweeps/s of each sampler (sweep kernel only, W=65536,
    CUDA events), tau_int of p_1..p_4 of each (W=8192 chains, 1500 measured
    sweeps after burn-in), effective samples/s = walker-sweeps/s / tau_int,
    acceptance, and the training cost (5000 ES+Adam steps on 2^20
    configurations drawn from the plain sampler)."""
    if rank != 0:
        return
    import numpy as np
    import torch

    import laughlinedge_b200 as L
    w = LEARNED
    torch.cuda.set_device(local)
    N, m, W = w["particles"], w["inverse_filling"], w["walkers"]
    sectors = [1, 2, 3, 4]

    def timed_sweeps(smp, n):
        st = torch.cuda.ExternalStream(smp.stream())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        smp.synchronize()
        a.record(st)
        smp.run(n, measure=False)
        b.record(st)
        b.synchronize()
        return a.elapsed_time(b) / 1e3

    # training data: snapshots of the plain chain
    plain = L.Sampler(L.SamplerConfig(N, m, W, step_sigma=w["sigma"], seed=w["seed"],
                                      lanes_per_walker=-1), sectors)
    plain.init_walkers()
    plain.run(args.burn + 100, measure=False)
    n_snap = w["train_configs"] // W
    cfg = torch.empty((n_snap * W, N, 2), dtype=torch.float32, device="cuda")
    for k in range(n_snap):
        plain.run(10, measure=False)
        plain.copy_positions_device(cfg[k * W:(k + 1) * W].data_ptr())
    plain.synchronize()
    t_plain = timed_sweeps(plain, 20) / 20
    plain.close()

    prop = L.LearnedProposal(N, m, init_sigma=w["sigma"], seed=w["seed"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    trace = prop.train(cfg.data_ptr(), cfg.shape[0], steps=w["train_steps"], batch=w["train_batch"],
                       pairs=w["train_pairs"], lr=3e-3, es_sigma=0.02, seed=w["seed"])
    t_train = time.perf_counter() - t0
    del cfg

    lsmp = L.Sampler(L.SamplerConfig(N, m, W, step_sigma=w["sigma"], seed=w["seed"] + 1), sectors)
    lsmp.set_proposal(prop)
    lsmp.init_walkers()
    lsmp.run(50, measure=False)
    t_learned = timed_sweeps(lsmp, 5) / 5
    lsmp.close()

    def tau_run(use_prop):
        smp = L.Sampler(L.SamplerConfig(N, m, w["tau_walkers"], step_sigma=w["sigma"],
                                        seed=w["seed"] + 7, lanes_per_walker=0), sectors)
        if use_prop:
            smp.set_proposal(prop)
        smp.init_walkers()
        smp.run(args.burn + 400, measure=False)
        smp.run(1500, measure=True)
        st = smp.stats()
        out = {"tau_int": st.tau_int, "tau_int_each": list(st.tau_int_each),
               "acceptance": st.acceptance}
        smp.close()
        return out

    tp, tl = tau_run(False), tau_run(True)
    res = {}
    for name, t, tau in (("plain", t_plain, tp), ("learned", t_learned, tl)):
        ws_s = W / t
        res[name] = dict(tau, walker_sweeps_per_s=ws_s, ms_per_sweep=1e3 * t,
                         effective_samples_per_s=ws_s / tau["tau_int"])
    line = {"metric": "effective_samples_per_s", "workload": w["workload"], "n_gpus": 1,
            "unit": "samples/s", "higher_is_better": True, "data": "synthetic",
            "config": {k: w[k] for k in w if k != "workload"},
            "plain": res["plain"], "learned": res["learned"],
            "learned_over_plain": res["learned"]["effective_samples_per_s"] /
            res["plain"]["effective_samples_per_s"],
            "tau_ratio_plain_over_learned": tp["tau_int"] / tl["tau_int"],
            "train_seconds": t_train,
            "train_objective_first_last": [float(np.mean(trace[:50])), float(np.mean(trace[-50:]))]}
    prop.close()
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--burn", type=int, default=400, help="untimed burn-in sweeps")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--gram", default=None, choices=["fp64", "bf16x3", "bf16x4", "tf32x3"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batched", action="store_true",
                    help="batched form N=100, dL 1..20, 16 kappas (its own JSON line)")
    ap.add_argument("--learned", action="store_true",
                    help="learned vs plain proposal at N=200 (its own JSON line)")
    ap.add_argument("--graph-batch", type=int, default=32,
                    help="measured sweeps per CUDA-graph replay in the timed run (0: direct launches)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_init()
    try:
        if args.learned:
            run_learned(args, rank, local)
        elif args.batched:
            run_batched(args, rank, local)
        elif args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
