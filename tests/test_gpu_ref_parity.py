"""Statistical parity of the CUDA path with the reference's own sampler: DSF
and occupation numbers.

The fixtures (tests/golden/dsf_reference_run.json and
occupation_reference_run.json, made by make_reference_fixture.py) hold outputs
of the reference's edgeMC::dsf_compute and
greenFunctionMC::occupation_numbers_compute, compiled from its sources for
sm_100a and run on a B200 (m = 3, N = 8, sigma = 0.3): mean and standard
deviation over independently seeded repetitions.  The CUDA path runs the same
physics in 8 replicas; every DSF energy and weight and every occupation entry
is compared by Welch's t statistic against the two-sided Student-t critical
value at a family-wise false-alarm rate of 1e-3, Bonferroni-corrected.
"""
import json
from pathlib import Path

import numpy as np
import pytest
from scipy import stats

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
FAMILY_ALPHA = 1e-3


def _welch(gm, gv, ng, rm, rv, nr):
    se2 = gv + rv
    t = np.abs(gm - rm) / np.sqrt(se2)
    dof = se2 ** 2 / (gv ** 2 / (ng - 1) + rv ** 2 / (nr - 1))
    return t, dof


def _assert_all(tests, label):
    per = FAMILY_ALPHA / len(tests)
    worst = max(tests, key=lambda x: x[1] / stats.t.isf(per / 2, x[2]))
    print(label, len(tests), "comparisons; worst", worst, flush=True)
    for what, t, dof in tests:
        assert t < stats.t.isf(per / 2, dof), (label, what, t, dof)


def _compare(tests, key, g, rm, rs, R, floor=1e-30, quantum=0.0):
    """quantum: the rounding step of the reference's printed values (its .tsv
    files keep 6 decimals), whose uniform error adds quantum^2 / 12 per value."""
    rm, rs = np.ravel(rm), np.ravel(rs)
    g = g.reshape(len(g), -1)
    gv, rv = g.var(0, ddof=1) / len(g), (rs ** 2 + quantum ** 2 / 12) / R
    live = (gv + rv) > floor
    t, dof = _welch(g.mean(0)[live], gv[live], len(g), rm[live], rv[live], R)
    tests += [(key, ti, di) for ti, di in zip(t, dof)]


def test_dsf_matches_reference_run(lemc, cuda_ctx):
    fx = json.loads((GOLD / "dsf_reference_run.json").read_text())
    R = fx["sampling"]["replicas"]
    rcl = fx["physics"]["RCl"]
    tests = []
    for dL, ref in fx["sectors"].items():
        E, S = [], []
        for r in range(8):
            # the reference's confinement sum (r / R_cl)^4: omega = 0, kappa = R_cl^-4
            e, w, *_ = lemc.dsf_compute(8, 3, int(dL), 8192, 500, 1500, 0.0, rcl ** -4, seed=300 + r)
            E.append(e)
            S.append(w)
        E, S = np.array(E), np.array(S)
        _compare(tests, (dL, "E"), E, ref["E_mean"], ref["E_std"], R)
        _compare(tests, (dL, "S"), S, ref["S_mean"], ref["S_std"], R)
        print("dsf", dL, E.mean(0), ref["E_mean"], S.mean(0), ref["S_mean"], flush=True)
    _assert_all(tests, "dsf")


def test_occupations_match_reference_run(lemc, cuda_ctx):
    fx = json.loads((GOLD / "occupation_reference_run.json").read_text())
    R = fx["sampling"]["replicas"]
    N, m, dL, Lc = 8, 3, fx["physics"]["dL"], fx["physics"]["l_cutoff"]
    reps = []
    for r in range(8):
        raw, _ = lemc.sampler.occupation(N, m, dL, Lc, 8192, 1500, burn_in=500, seed=500 + r)
        n = raw / raw.sum(-1, keepdims=True) * N  # the reference's normalisation per (L, R)
        reps.append(0.5 * (n + np.conj(np.transpose(n, (1, 0, 2)))))  # Hermitised per l
    reps = np.array(reps)
    tests = []
    _compare(tests, "re", reps.real, fx["re_mean"], fx["re_std"], R, 1e-14, quantum=1e-6)
    _compare(tests, "im", reps.imag, fx["im_mean"], fx["im_std"], R, 1e-14, quantum=1e-6)
    print("occupation diag", reps.real.mean(0)[0, 0, :12], np.array(fx["re_mean"])[0][0][:12])
    _assert_all(tests, "occupation")
