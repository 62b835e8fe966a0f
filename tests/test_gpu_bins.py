"""Bins and jackknife error bars of a sampling run on the GPU: the bins add up
to the run's Gram sums, and the jackknife error of one run predicts the
spread of independent runs (the error-bar analysis the reference leaves to
repeated runs, main.cu:18-20)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, M_FILL, OMEGA, KAPPA = 8, 3, 1e-2, 1e-4


def _run(lemc, seed, bins=10, per_bin=200, W=2048):
    smp = lemc.Sampler(lemc.SamplerConfig(N, M_FILL, W, seed=seed, gram_mode=lemc._lib.GRAM_TF32X3),
                       [3, 4])
    smp.init_walkers()
    smp.run(300, measure=False)
    for _ in range(bins):
        smp.run(per_bin, measure=True)
        smp.close_bin()
    return smp


def test_bins_sum_to_run(lemc, cuda_ctx):
    smp = _run(lemc, 5)
    assert smp.n_bins() == 10
    for s in range(2):
        S, H2, H4, n = smp.gram(s)
        parts = [smp.gram_bin(b, s) for b in range(10)]
        for i, X in enumerate((S, H2, H4)):
            tot = sum(p[i] for p in parts)
            assert np.allclose(tot, X, rtol=1e-12, atol=1e-12 * np.abs(X).max())
        assert sum(p[3] for p in parts) == n
    smp.reset()
    assert smp.n_bins() == 0
    smp.close()


def test_jackknife_error_predicts_replica_spread(lemc, cuda_ctx):
    evs, errs = [], []
    for r in range(8):
        smp = _run(lemc, 100 + r)
        ev, er, _, _ = smp.jackknife(1, OMEGA, KAPPA)
        evs.append(ev)
        errs.append(er)
        smp.close()
    spread = np.array(evs).std(0, ddof=1)
    ratio = np.mean(errs, 0) / spread
    print("jackknife / replica spread", ratio)
    # 8 replicas: the sample spread itself is uncertain by about 25 %
    assert np.all((ratio > 0.4) & (ratio < 2.5)), ratio
