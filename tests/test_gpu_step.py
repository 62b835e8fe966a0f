"""Step tuning (lemc_tune_step, the reference's optimal_step of
em_bisection.cu:49-153) on the GPU: from a step far from the target, the
search ends with an acceptance within the tolerance, and an independent
measurement at the returned step agrees."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("start", [0.05, 3.0])
def test_tune_step_reaches_target(lemc, cuda_ctx, start):
    N, m, W = 8, 3, 4096
    smp = lemc.Sampler(lemc.SamplerConfig(N, m, W, step_sigma=start, seed=3), [1, 2])
    smp.init_walkers()
    smp.run(200, measure=False)
    sigma, acc = smp.tune_step(0.5, 0.01, 100)
    assert abs(acc - 0.5) < 0.01, (sigma, acc)
    # an independent measurement at the tuned step: 4096 walkers x 8 moves x 200
    # sweeps give a statistical error far below the tolerance
    smp.reset()
    smp.run(200, measure=False)
    again = smp.stats().acceptance
    assert abs(again - 0.5) < 0.015, (sigma, again)
    smp.close()


def test_tune_step_drop_in(lemc, cuda_ctx):
    """The C++ drop-in's optimal_step path goes through the same search: with
    the reference's default tolerance (0.01) the sampler's final step gives 50 %."""
    smp = lemc.Sampler(lemc.SamplerConfig(50, 3, 8192, step_sigma=0.8, seed=4), [1])
    smp.init_walkers()
    smp.run(300, measure=False)
    sigma, acc = smp.tune_step(0.5, 0.01, 100)
    assert 0.2 < sigma < 2.0 and abs(acc - 0.5) < 0.01
    smp.close()
