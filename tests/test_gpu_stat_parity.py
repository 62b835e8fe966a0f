"""Statistical parity of the CUDA estimators with the reference estimator.

The fixture (tests/golden/config1_reference_estimator.json, made by
make_parity_fixture.py) holds the oracle's restatement of the reference
estimator -- one chain per basis row guided by |P_a Psi_m|^2 -- at m = 3,
N = 8, omega = 1e-2, kappa = 1e-4, dL = 1..6: eight replicas, mean and
standard deviation of the normalised M and H and of the spectrum.

The GPU runs the same physics with (i) the shared Laughlin guide and the
tcgen05 S/H contraction and (ii) its own port of the per-row reference
estimator.  Normalised matrix entries agree within 4 combined standard
errors; spectra of replica-averaged matrices agree within 3 combined
standard errors of the eigenvalues.
"""
import json
from pathlib import Path

import numpy as np
import pytest
import scipy.linalg as sl

pytestmark = pytest.mark.gpu
GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "config1_reference_estimator.json").read_text())
PHY = GOLD["physics"]
SECTORS = [1, 2, 3, 4, 5, 6]


def _gpu_replicas(lemc, guide, mode, reps=4, W=4096, burn=500, meas=2000):
    out = {dL: {"M": [], "H": [], "ev": []} for dL in SECTORS}
    for r in range(reps):
        cfg = lemc.SamplerConfig(PHY["N"], PHY["m"], W, step_sigma=PHY["sigma"], seed=77 + r,
                                 guide=guide, gram_mode=mode)
        if guide == lemc._lib.GUIDE_LAUGHLIN:
            smp = lemc.Sampler(cfg, SECTORS)
            smp.init_walkers()
            smp.run(burn, measure=False)
            smp.run(meas, measure=True)
            for s, dL in enumerate(SECTORS):
                S, H2, H4, _ = smp.gram(s)
                M, H = lemc.normalise(S, H2, H4, PHY["omega"], PHY["kappa"])
                out[dL]["M"].append(M.real)
                out[dL]["H"].append(H.real)
                out[dL]["ev"].append(lemc.geneig(H, M))
            smp.close()
        else:
            for dL in SECTORS:  # the reference samples one sector per call
                smp = lemc.Sampler(cfg, [dL])
                smp.init_walkers()
                smp.run(burn, measure=False)
                smp.run(meas, measure=True)
                fg, gg, fh, n = smp.rows(PHY["omega"], PHY["kappa"])
                M = fg / np.sqrt(gg)
                H = fh / np.sqrt(gg)
                M, H = 0.5 * (M + M.conj().T), 0.5 * (H + H.conj().T)
                out[dL]["M"].append(M.real)
                out[dL]["H"].append(H.real)
                out[dL]["ev"].append(lemc.geneig(H, M))
                smp.close()
    return out


def _check(lemc, out, label):
    R_ref = GOLD["sampling"]["replicas"]
    report = []
    for dL in SECTORS:
        ref = GOLD["sectors"][str(dL)]
        reps = len(out[dL]["M"])
        for key in ("M", "H"):
            g = np.array(out[dL][key])
            gm, gs = g.mean(0), g.std(0, ddof=1) / np.sqrt(reps)
            rm = np.array(ref[f"{key}_re_mean"])
            rs = np.array(ref[f"{key}_re_std"]) / np.sqrt(R_ref)
            sig = np.sqrt(gs ** 2 + rs ** 2) + 1e-9 * (1 + np.abs(rm))
            z = np.abs(gm - rm) / sig
            report.append((label, dL, key, float(z.max())))
            print(label, dL, key, "max z %.2f" % z.max(), flush=True)
            assert np.all(z < 4.0), (label, dL, key, z.max())
        # spectra of the replica-averaged matrices
        Mg, Hg = np.mean(out[dL]["M"], 0), np.mean(out[dL]["H"], 0)
        Mr, Hr = np.array(ref["M_re_mean"]), np.array(ref["H_re_mean"])
        eg = sl.eigh(Hg, Mg, eigvals_only=True)
        er = sl.eigh(Hr, Mr, eigvals_only=True)
        se = np.sqrt(np.array(out[dL]["ev"]).std(0, ddof=1) ** 2 / reps +
                     np.array(ref["eig_std"]) ** 2 / R_ref) + 1e-12
        zev = np.abs(eg - er) / se
        report.append((label, dL, "eig", float(zev.max())))
        print(label, dL, "eig", eg, er, "max z %.2f" % zev.max(), flush=True)
        assert np.all(zev < 3.0), (label, dL, eg, er, se)
    print(report)


def test_laughlin_guide_tc_gram_matches_reference_estimator(lemc, cuda_ctx):
    out = _gpu_replicas(lemc, lemc._lib.GUIDE_LAUGHLIN, lemc._lib.GRAM_TF32X3)
    _check(lemc, out, "laughlin+tf32x3")


def test_gpu_reference_estimator_matches_oracle(lemc, cuda_ctx):
    out = _gpu_replicas(lemc, lemc._lib.GUIDE_ROW, lemc._lib.GRAM_FP64, W=4096)
    _check(lemc, out, "rows")
