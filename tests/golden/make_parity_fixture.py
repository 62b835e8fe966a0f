"""Generates config1_reference_estimator.json: the reference estimator (one
Metropolis chain per basis row guided by |P_a Psi_m|^2, per-row ratio sums,
reference normalisation and Hermitisation) run by the oracle's C restatement
at the plain-method physics: m = 3, N = 8, V = omega r^2 + kappa r^4 with
omega = 1e-2, kappa = 1e-4, sectors dL = 1..6, sigma = 0.3.  Thirty-two
independent replicas (seeds 1000..1031) give mean and standard deviation of
every generalized eigenvalue and of the normalised matrices M and H.
"""
import json
import sys
import time
from pathlib import Path

import numpy as np
import scipy.linalg as sl

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
from oracle import oracle as O  # noqa: E402

N, M_FILL, OMEGA, KAPPA, SIGMA = 8, 3, 1e-2, 1e-4, 0.3
SECTORS = [1, 2, 3, 4, 5, 6]
W, BURN, MEAS, REPS = 512, 500, 2000, 32


def main():
    t0 = time.time()
    out = {"physics": {"N": N, "m": M_FILL, "omega": OMEGA, "kappa": KAPPA, "sigma": SIGMA},
           "sampling": {"walkers": W, "burn_in": BURN, "measurements": MEAS, "replicas": REPS},
           "sectors": {}}
    for dL in SECTORS:
        evs, Ms, Hs = [], [], []
        for r in range(REPS):
            res = O.run_rows(N, M_FILL, W, SIGMA, 1000 + r, BURN, MEAS, [dL])
            fh = OMEGA * res["fh2"] + KAPPA * res["fh4"]
            Mx, Hx = O.reference_matrices(res["fg"], res["gg"], fh, res["n_row"])
            evs.append(sl.eigh(Hx, Mx, eigvals_only=True))
            Ms.append(Mx)
            Hs.append(Hx)
        evs, Ms, Hs = np.array(evs), np.array(Ms), np.array(Hs)
        out["sectors"][str(dL)] = {
            "eig_mean": evs.mean(0).tolist(), "eig_std": evs.std(0, ddof=1).tolist(),
            "M_re_mean": Ms.real.mean(0).tolist(), "M_re_std": Ms.real.std(0, ddof=1).tolist(),
            "H_re_mean": Hs.real.mean(0).tolist(), "H_re_std": Hs.real.std(0, ddof=1).tolist()}
        print(dL, evs.mean(0), evs.std(0, ddof=1), flush=True)
    out["seconds"] = time.time() - t0
    (HERE / "config1_reference_estimator.json").write_text(json.dumps(out))


if __name__ == "__main__":
    main()
