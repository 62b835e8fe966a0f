"""Statistical parity of the CUDA estimators with the reference estimator.

Two fixtures hold the reference estimator at m = 3, N = 8, omega = 1e-2,
kappa = 1e-4, dL = 1..6 (mean and standard deviation over independent
replicas of the normalised M and H and of the spectrum):
  config1_reference_run.json        the reference's own sampler
      (edgeMC::spectrum_compute compiled from its sources, run on a B200 by
      make_reference_fixture.py; exponent-2 and exponent-4 builds combined);
  config1_reference_estimator.json  the oracle's C restatement of it
      (make_parity_fixture.py).

The GPU runs the same physics with (i) the shared Laughlin guide and the
tcgen05 S/H contraction and (ii) its own port of the per-row reference
estimator, 8 replicas each.  Every normalised matrix entry and every
eigenvalue of the replica-averaged matrices is compared by Welch's t
statistic (standard errors of both means, Welch-Satterthwaite degrees of
freedom) against the two-sided Student-t critical value at a family-wise
false-alarm rate of 1e-3, Bonferroni-corrected over all comparisons of one
estimator.
"""
import json
from pathlib import Path

import numpy as np
import pytest
import scipy.linalg as sl
from scipy import stats

pytestmark = pytest.mark.gpu
FIXTURES = ["config1_reference_run.json", "config1_reference_estimator.json"]
_DIR = Path(__file__).resolve().parent / "golden"
PHY = json.loads((_DIR / FIXTURES[1]).read_text())["physics"]
SECTORS = [1, 2, 3, 4, 5, 6]
_OUT = {}


FAMILY_ALPHA = 1e-3


def _gpu_replicas(lemc, guide, mode, reps=8, W=4096, burn=500, meas=1500):
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


def _welch(g_mean, g_var, n_g, r_mean, r_var, n_r):
    """Welch t statistic and Welch-Satterthwaite degrees of freedom; the
    variances are those of the replica means."""
    se2 = g_var + r_var
    t = np.abs(g_mean - r_mean) / np.sqrt(se2)
    dof = se2 ** 2 / (g_var ** 2 / (n_g - 1) + r_var ** 2 / (n_r - 1))
    return t, dof


def _check(lemc, out, label, gold):
    R_ref = gold["sampling"]["replicas"]
    tests = []  # (what, t, dof)
    for dL in SECTORS:
        ref = gold["sectors"][str(dL)]
        reps = len(out[dL]["M"])
        for key in ("M", "H"):
            g = np.array(out[dL][key])
            gv = g.var(0, ddof=1) / reps
            rv = np.array(ref[f"{key}_re_std"]) ** 2 / R_ref
            live = (gv + rv) > 1e-24  # the unit diagonal of M has no spread
            t, dof = _welch(g.mean(0)[live], gv[live], reps,
                            np.array(ref[f"{key}_re_mean"])[live], rv[live], R_ref)
            tests += [((dL, key), ti, di) for ti, di in zip(t, dof)]
        # spectra of the replica-averaged matrices
        Mg, Hg = np.mean(out[dL]["M"], 0), np.mean(out[dL]["H"], 0)
        Mr, Hr = np.array(ref["M_re_mean"]), np.array(ref["H_re_mean"])
        eg = sl.eigh(Hg, Mg, eigvals_only=True)
        er = sl.eigh(Hr, Mr, eigvals_only=True)
        gv = np.array(out[dL]["ev"]).var(0, ddof=1) / reps
        rv = np.array(ref["eig_std"]) ** 2 / R_ref
        t, dof = _welch(eg, gv, reps, er, rv, R_ref)
        tests += [((dL, "eig"), ti, di) for ti, di in zip(t, dof)]
        print(label, dL, "eig", eg, er, "max t %.2f" % t.max(), flush=True)
    per_test = FAMILY_ALPHA / len(tests)
    worst = max(tests, key=lambda x: x[1] / stats.t.isf(per_test / 2, x[2]))
    print(label, len(tests), "comparisons; worst", worst, flush=True)
    for what, t, dof in tests:
        crit = stats.t.isf(per_test / 2, dof)
        assert t < crit, (label, what, t, dof, crit)


def _replicas(lemc, guide):
    if guide not in _OUT:  # the GPU replicas are shared by both fixtures
        if guide == lemc._lib.GUIDE_LAUGHLIN:
            _OUT[guide] = _gpu_replicas(lemc, guide, lemc._lib.GRAM_TF32X3)
        else:
            _OUT[guide] = _gpu_replicas(lemc, guide, lemc._lib.GRAM_FP64, W=4096)
    return _OUT[guide]


@pytest.mark.parametrize("fixture", FIXTURES)
def test_laughlin_guide_tc_gram_matches_reference_estimator(lemc, cuda_ctx, fixture):
    gold = json.loads((_DIR / fixture).read_text())
    _check(lemc, _replicas(lemc, lemc._lib.GUIDE_LAUGHLIN), "laughlin+tf32x3 vs " + fixture, gold)


@pytest.mark.parametrize("fixture", FIXTURES)
def test_gpu_reference_estimator_matches_reference(lemc, cuda_ctx, fixture):
    gold = json.loads((_DIR / fixture).read_text())
    _check(lemc, _replicas(lemc, lemc._lib.GUIDE_ROW), "rows vs " + fixture, gold)
