"""Occupation numbers (two-state walker) on the GPU: the nu = 1 known answer
and statistical parity with the oracle's restatement of the reference estimator."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _normalised(occ, N):
    return (occ / occ.sum(axis=-1, keepdims=True) * N)


def test_occupation_nu1_ground_state(lemc, cuda_ctx):
    N = 5
    occ, acc = lemc.sampler.occupation(N, 1, 0, 3 * N, 8192, 800, burn_in=300, step_sigma=0.5, seed=5)
    n = _normalised(occ, N)[0, 0].real
    assert 0.2 < acc < 0.95
    assert np.all(np.abs(n[:N] - 1.0) < 0.03), n
    assert np.all(np.abs(n[N:]) < 0.03), n


def test_occupation_matches_oracle(lemc, oracle, cuda_ctx):
    N, m, dL = 6, 3, 2
    Lc = m * (N - 1) + 6
    reps_g, reps_o = [], []
    for r in range(4):
        occ, _ = lemc.sampler.occupation(N, m, dL, Lc, 4 * 2048, 600, burn_in=300, seed=100 + r)
        reps_g.append(_normalised(occ, N).real)
    for r in range(4):
        per = np.zeros((2, 2, Lc))
        for a in range(2):
            for b in range(2):
                o = oracle.occupation(N, m, 512, 0.3, 500 + r, 300, 600, dL, a, b, Lc)
                per[a, b] = (o / o.sum() * N).real
        reps_o.append(per)
    g, o = np.array(reps_g), np.array(reps_o)
    sig = np.sqrt(g.std(0, ddof=1) ** 2 / 4 + o.std(0, ddof=1) ** 2 / 4) + 2e-3
    z = np.abs(g.mean(0) - o.mean(0)) / sig
    assert z.max() < 4.5, z.max()
    assert np.allclose(g.sum(-1), N)
