"""Generates the fixtures that pin the oracle and the CUDA path to the
reference itself: the reference's own sampler (edgeMC::spectrum_compute,
edgeMC::dsf_compute, greenFunctionMC::occupation_numbers_compute), compiled
from its sources for sm_100a by oracle/Makefile (target refmc, with the Eigen
stand-in of oracle/eigen_shim), run on a B200 through oracle/ref_edge_main.cu.

Physics: the plain-method configuration, m = 3, N = 8, sigma = 0.3 (kept by
setAcceptanceBisectionParams(100, 0.5, 1.0)).  The reference has one
compile-time confinement sum_i (r_i/R_cl)^e, so it is built twice (e = 2, 4)
and, H being linear in V, the physical confinement omega r^2 + kappa r^4 with
omega = 1e-2, kappa = 1e-4 is H = omega R_cl^2 H_2 + kappa R_cl^4 H_4, with M
the mean of the two runs' metrics.  Each repetition reseeds the reference
(the harness supplies the clock its seed is drawn from).

Outputs (run on the GPU machine; argument = output directory):
  config1_reference_run.json        spectrum: mean / std over repetitions of the
                                    normalised M, H (real parts) and of the
                                    generalized eigenvalues, dL = 1..6
  dsf_reference_run.json            DSF energies and weights for sum (r/R_cl)^4,
                                    dL = 1..4
  occupation_reference_run.json     occupations (normalised to N, Hermitised)
                                    of every row pair, dL = 2
  reference_timing.json             the reference's own cudaEvent kernel times
"""
import json
import subprocess
import sys
import time
from pathlib import Path

import numpy as np
import scipy.linalg as sl

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF = ROOT / "oracle" / "_ref"
OMEGA, KAPPA = 1e-2, 1e-4


def run(binary, mode, sectors, burn, samples, reps, clock0, blocks, out, work):
    cmd = [str(REF / binary), mode, ",".join(map(str, sectors)), str(burn), str(samples), str(reps),
           "0.3", str(clock0), str(blocks), str(out), str(work)]
    t0 = time.time()
    with open(str(out) + ".log", "w") as log:
        subprocess.run(cmd, check=True, stdout=log, stderr=subprocess.STDOUT)
    return json.loads(Path(out).read_text()), time.time() - t0


def cplx(a):
    a = np.asarray(a, float)
    return a[..., 0] + 1j * a[..., 1]


def main(outdir):
    outdir = Path(outdir).resolve()
    outdir.mkdir(parents=True, exist_ok=True)
    work = Path("/tmp/ref_edge_work/run")
    reps, burn, samples, blocks = int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4]), int(sys.argv[5])
    sectors = [1, 2, 3, 4, 5, 6]
    timing = {"walkers": blocks * 128, "burn_in": burn, "samples": samples}
    # spectrum, exponent 2 and 4 (independent chains, same clocks)
    r2, t2 = run("ref_edge_e2", "spectrum", sectors, burn, samples, reps, 5000, blocks,
                 outdir / "raw_spec_e2.json", work)
    r4, t4 = run("ref_edge_e4", "spectrum", sectors, burn, samples, reps, 9000, blocks,
                 outdir / "raw_spec_e4.json", work)
    rcl = r2["RCl"]
    fix = {"source": "reference sampler (edgeMC::spectrum_compute) compiled from its sources, run on B200",
           "physics": {"N": 8, "m": 3, "omega": OMEGA, "kappa": KAPPA, "sigma": 0.3, "RCl": rcl},
           "sampling": {"walkers": blocks * 128, "burn_in": burn, "measurements": samples,
                        "replicas": reps}, "sectors": {}}
    ms = []
    for dL in sectors:
        e2 = [x for x in r2["runs"] if x["dL"] == dL]
        e4 = [x for x in r4["runs"] if x["dL"] == dL]
        Ms, Hs, evs = [], [], []
        for a, b in zip(e2, e4):
            M = 0.5 * (cplx(a["M"]) + cplx(b["M"]))
            H = OMEGA * rcl ** 2 * cplx(a["H"]) + KAPPA * rcl ** 4 * cplx(b["H"])
            Ms.append(M)
            Hs.append(H)
            evs.append(sl.eigh(H, M, eigvals_only=True))
            ms += a["kernel_ms"] + b["kernel_ms"]
        Ms, Hs, evs = np.array(Ms), np.array(Hs), np.array(evs)
        fix["sectors"][str(dL)] = {
            "eig_mean": evs.mean(0).tolist(), "eig_std": evs.std(0, ddof=1).tolist(),
            "M_re_mean": Ms.real.mean(0).tolist(), "M_re_std": Ms.real.std(0, ddof=1).tolist(),
            "H_re_mean": Hs.real.mean(0).tolist(), "H_re_std": Hs.real.std(0, ddof=1).tolist()}
    (outdir / "config1_reference_run.json").write_text(json.dumps(fix))
    timing["spectrum_row_kernel_ms"] = ms
    timing["spectrum_walker_sweeps_per_s"] = (len(ms) * blocks * 128 * (burn + samples)
                                              / (sum(ms) * 1e-3))
    timing["spectrum_wall_s"] = t2 + t4
    # DSF with the quartic confinement (non-degenerate modes), dL = 1..4
    dsec = [1, 2, 3, 4]
    rd, td = run("ref_edge_e4", "dsf", dsec, burn, samples, reps, 13000, blocks,
                 outdir / "raw_dsf_e4.json", work)
    dfix = {"source": "reference sampler (edgeMC::dsf_compute) compiled from its sources, run on B200",
            "physics": {"N": 8, "m": 3, "confinement": "sum (r/RCl)^4", "RCl": rcl, "sigma": 0.3},
            "sampling": fix["sampling"], "sectors": {}}
    for dL in dsec:
        es = np.array([x["energy_dsf"] for x in rd["runs"] if x["dL"] == dL], float)
        dfix["sectors"][str(dL)] = {"E_mean": es[..., 0].mean(0).tolist(),
                                    "E_std": es[..., 0].std(0, ddof=1).tolist(),
                                    "S_mean": es[..., 1].mean(0).tolist(),
                                    "S_std": es[..., 1].std(0, ddof=1).tolist()}
    (outdir / "dsf_reference_run.json").write_text(json.dumps(dfix))
    timing["dsf_wall_s"] = td
    # occupation numbers, dL = 2 (two rows, four pairs)
    ro, to = run("ref_edge_e2", "occupation", [2], burn, samples, reps, 17000, blocks,
                 outdir / "raw_occ.json", work)
    lc = ro["angular_momentum_cutoff"]
    occ = []
    for x in ro["runs"]:
        arr = np.zeros((2, 2, lc), complex)
        for a, b, l, re, im in x["occupation"]:
            arr[a, b, l] = re + 1j * im
        occ.append(arr)
    occ = np.array(occ)
    ofix = {"source": "reference sampler (greenFunctionMC::occupation_numbers_compute) compiled "
                      "from its sources, run on B200",
            "physics": {"N": 8, "m": 3, "dL": 2, "l_cutoff": lc, "sigma": 0.3},
            "sampling": fix["sampling"],
            "re_mean": occ.real.mean(0).tolist(), "re_std": occ.real.std(0, ddof=1).tolist(),
            "im_mean": occ.imag.mean(0).tolist(), "im_std": occ.imag.std(0, ddof=1).tolist()}
    (outdir / "occupation_reference_run.json").write_text(json.dumps(ofix))
    timing["occupation_wall_s"] = to
    timing["occupation_pair_kernel_ms"] = [v for x in ro["runs"] for v in x["kernel_ms"]]
    (outdir / "reference_timing.json").write_text(json.dumps(timing))


if __name__ == "__main__":
    main(sys.argv[1])
