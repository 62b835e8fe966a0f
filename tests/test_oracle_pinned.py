"""The oracle pinned to the reference itself: the oracle's C restatement of the
reference estimator (config1_reference_estimator.json, make_parity_fixture.py)
against the reference's own sampler compiled from its sources and run on a
B200 (config1_reference_run.json, make_reference_fixture.py), same physics
(m = 3, N = 8, omega = 1e-2, kappa = 1e-4, sigma = 0.3, dL = 1..6).  Every
normalised M and H entry and every eigenvalue of the replica-averaged
matrices: Welch's t against the
two-sided Student-t critical value at a family-wise false-alarm rate of 1e-3
(Bonferroni).  Fixture files only: no GPU, no reference checkout."""
import json
from pathlib import Path

import numpy as np
import scipy.linalg as sl
from scipy import stats

GOLD = Path(__file__).resolve().parent / "golden"


def test_oracle_restatement_matches_reference_run():
    orc = json.loads((GOLD / "config1_reference_estimator.json").read_text())
    ref = json.loads((GOLD / "config1_reference_run.json").read_text())
    assert orc["physics"]["omega"] == ref["physics"]["omega"]
    assert orc["physics"]["kappa"] == ref["physics"]["kappa"]
    ro, rr = orc["sampling"]["replicas"], ref["sampling"]["replicas"]
    tests = []
    for dL in map(str, range(1, 7)):
        o, r = orc["sectors"][dL], ref["sectors"][dL]
        # eigenvalues of the replica-averaged matrices: the mean of per-replica
        # eigenvalues carries a bias that grows with the per-replica noise, and
        # the two fixtures have different replica sizes
        o["eig_of_mean"] = sl.eigh(np.array(o["H_re_mean"]), np.array(o["M_re_mean"]), eigvals_only=True)
        r["eig_of_mean"] = sl.eigh(np.array(r["H_re_mean"]), np.array(r["M_re_mean"]), eigvals_only=True)
        for mean, std in (("M_re_mean", "M_re_std"), ("H_re_mean", "H_re_std"), ("eig_of_mean", "eig_std")):
            om, osd = np.ravel(o[mean]), np.ravel(o[std])
            rm, rsd = np.ravel(r[mean]), np.ravel(r[std])
            ov, rv = osd ** 2 / ro, rsd ** 2 / rr
            live = (ov + rv) > 1e-24
            se2 = ov[live] + rv[live]
            t = np.abs(om[live] - rm[live]) / np.sqrt(se2)
            dof = se2 ** 2 / (ov[live] ** 2 / (ro - 1) + rv[live] ** 2 / (rr - 1))
            tests += [((dL, mean), ti, di) for ti, di in zip(t, dof)]
    per = 1e-3 / len(tests)
    worst = max(tests, key=lambda x: x[1] / stats.t.isf(per / 2, x[2]))
    print(len(tests), "comparisons; worst", worst)
    for what, t, dof in tests:
        assert t < stats.t.isf(per / 2, dof), (what, t, dof)
