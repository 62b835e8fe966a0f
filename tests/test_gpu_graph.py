"""CUDA-graph replay of measured sweeps (lemc_config.graph_batch) against direct
launches of the same context, through the C-ABI: same walkers, same Gram planes,
same walker-mean series, including graph reuse across calls and re-capture after a
setter changes the launch arguments."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(lemc, graph_batch, mode):
    N, m, W = 8, 3, 4096
    sectors = list(range(7))
    smp = lemc.Sampler(lemc.SamplerConfig(N, m, W, seed=31, lanes_per_walker=4, gram_mode=mode,
                                          graph_batch=graph_batch), sectors)
    smp.init_walkers()
    smp.run(20, measure=False)
    smp.run(37, measure=True)          # 4 replays of 8 + 5 direct sweeps
    smp.run(16, measure=True)          # the cached graph again
    smp.lib.lemc_set_step(smp._h, 0.25)
    smp.run(19, measure=True)          # re-captured after the step change
    smp.synchronize()
    out = {"pos": smp.positions(), "series": smp.series(),
           "gram": [smp.gram(s)[:3] for s in range(len(sectors))], "stats": smp.stats()}
    smp.close()
    return out


@pytest.mark.parametrize("mode", [3, 0])
def test_graph_replay_matches_direct_launches(lemc, cuda_ctx, mode):
    ref = _run(lemc, 0, mode)
    got = _run(lemc, 8, mode)
    assert np.array_equal(ref["pos"], got["pos"])
    assert ref["stats"].sweeps == got["stats"].sweeps
    assert ref["stats"].measurements == got["stats"].measurements
    np.testing.assert_allclose(got["series"], ref["series"], rtol=1e-12, atol=1e-14)
    for (S, H2, H4), (S2, H22, H42) in zip(ref["gram"], got["gram"]):
        for X, Y in ((S, S2), (H2, H22), (H4, H42)):
            np.testing.assert_allclose(Y, X, rtol=1e-12, atol=1e-12 * np.abs(X).max())
