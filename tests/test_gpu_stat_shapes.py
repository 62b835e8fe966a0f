"""Statistical checks at the larger workloads' particle numbers.

N = 50 (the mixed-precision workload): the harmonic known answer (every
eigenvalue of a sector equals 2 omega (m N (N-1)/2 + dL + N) for V = omega r^2)
with the shared guide and the TF32x3 contraction; and the two estimators (shared
Laughlin guide + TF32x3, per-row reference guide + FP64) agreeing entry by
entry.  N = 200 (the learned-proposal workload): the learned proposal's
normalised M and H and spectrum agree with the plain sampler's.  Welch's t
per entry against the two-sided Student-t critical value at a family-wise
false-alarm rate of 1e-3, Bonferroni-corrected."""
import numpy as np
import pytest
import scipy.linalg as sl
from scipy import stats

pytestmark = pytest.mark.gpu


def _welch_all(A, B, label):
    """A, B: [replicas, ...] arrays of independent estimates."""
    A = np.array(A).reshape(len(A), -1)
    B = np.array(B).reshape(len(B), -1)
    va, vb = A.var(0, ddof=1) / len(A), B.var(0, ddof=1) / len(B)
    live = (va + vb) > 1e-24
    se2 = va[live] + vb[live]
    t = np.abs(A.mean(0)[live] - B.mean(0)[live]) / np.sqrt(se2)
    dof = se2 ** 2 / (va[live] ** 2 / (len(A) - 1) + vb[live] ** 2 / (len(B) - 1))
    crit = stats.t.isf(1e-3 / len(t) / 2, dof)
    print(label, len(t), "comparisons; worst t/crit %.2f" % np.max(t / crit), flush=True)
    assert np.all(t < crit), (label, t.max())


def test_harmonic_known_answer_n50(lemc, cuda_ctx):
    N, m, om = 50, 3, 5e-3
    smp = lemc.Sampler(lemc.SamplerConfig(N, m, 16384, seed=8, gram_mode=lemc._lib.GRAM_TF32X3),
                       [2, 3, 4])
    smp.init_walkers()
    smp.run(600, measure=False)
    smp.run(200, measure=True)
    for s, dL in enumerate([2, 3, 4]):
        S, H2, H4, _ = smp.gram(s)
        M, H = lemc.normalise(S, H2, H4, om, 0.0)
        ev = lemc.geneig(H, M)
        level = 2 * om * (m * N * (N - 1) / 2 + dL + N)
        assert abs(np.mean(ev) - level) < 2e-3 * level, (dL, ev, level)
        assert np.max(np.abs(ev - level)) < 1e-2 * level, (dL, ev, level)
    smp.close()


def test_estimators_agree_n50(lemc, cuda_ctx):
    N, m, om, ka = 50, 3, 5e-3, 2e-5
    sectors = [2, 3]
    out = {"lg": [], "row": []}
    for r in range(4):
        smp = lemc.Sampler(lemc.SamplerConfig(N, m, 16384, seed=20 + r,
                                              gram_mode=lemc._lib.GRAM_TF32X3), sectors)
        smp.init_walkers()
        smp.run(600, measure=False)
        smp.run(300, measure=True)
        blocks = []
        for s in range(len(sectors)):
            S, H2, H4, _ = smp.gram(s)
            M, H = lemc.normalise(S, H2, H4, om, ka)
            blocks += [M.real.ravel(), H.real.ravel()]
        out["lg"].append(np.concatenate(blocks))
        smp.close()
        smp = lemc.Sampler(lemc.SamplerConfig(N, m, 16384, seed=40 + r, guide=lemc._lib.GUIDE_ROW),
                           sectors)
        smp.init_walkers()
        smp.run(600, measure=False)
        smp.run(300, measure=True)
        fg, gg, fh, _ = smp.rows(om, ka)
        M = fg / np.sqrt(gg)
        H = fh / np.sqrt(gg)
        M, H = 0.5 * (M + M.conj().T), 0.5 * (H + H.conj().T)
        blocks, f = [], 0
        for d in smp.dims:
            blocks += [M[f:f + d, f:f + d].real.ravel(), H[f:f + d, f:f + d].real.ravel()]
            f += d
        out["row"].append(np.concatenate(blocks))
        smp.close()
    _welch_all(out["lg"], out["row"], "N=50 shared guide vs row guide")


def test_learned_matches_plain_n200(lemc, cuda_ctx):
    N, m, om, ka = 200, 3, 1e-3, 5e-6
    sectors = [1, 2, 3]
    W = 4096
    base = lemc.Sampler(lemc.SamplerConfig(N, m, W, seed=3), [1, 2, 3, 4])
    base.init_walkers()
    base.run(800, measure=False)
    xy = base.positions()
    base.close()
    prop = lemc.LearnedProposal(N, m, init_sigma=1.0, seed=5)
    res = {"learned": [], "plain": []}
    for r in range(4):
        for name in ("learned", "plain"):
            smp = lemc.Sampler(lemc.SamplerConfig(N, m, W, step_sigma=1.2, seed=60 + 2 * r + (name == "plain")),
                               sectors)
            if name == "learned":
                smp.set_proposal(prop)
            smp.init_walkers(xy)
            smp.run(100, measure=False)
            smp.run(400, measure=True)
            vals = []
            for s in range(len(sectors)):
                S, H2, H4, _ = smp.gram(s)
                M, H = lemc.normalise(S, H2, H4, om, ka)
                vals += [M.real.ravel(), H.real.ravel(), sl.eigh(H.real, M.real, eigvals_only=True)]
            res[name].append(np.concatenate(vals))
            smp.close()
    prop.close()
    _welch_all(res["learned"], res["plain"], "N=200 learned vs plain")
