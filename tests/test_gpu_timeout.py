"""The contraction's bounded waits on the GPU: with a short bound and the
loader held back (nothing ever fills an operand stage), every mbarrier wait of
gram_tc_kernel expires; the kernel must report LEMC_ERR_TIMEOUT through the
context, leave the CUDA context usable, and a reset context must compute
again.  Nothing faults or hangs: the waits are bounded and no copy or MMA is
ever issued."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TIMEOUT = -4


def _sampler(lemc, seed):
    smp = lemc.Sampler(lemc.SamplerConfig(8, 3, 2048, seed=seed, gram_mode=lemc._lib.GRAM_TF32X3),
                       [2, 3])
    smp.init_walkers()
    smp.run(50, measure=False)
    return smp


def test_bounded_wait_expires_and_reports(lemc, cuda_ctx):
    lib = lemc.load()
    smp = _sampler(lemc, 3)
    try:
        assert lib.lemc_debug_gram_wait(2_000_000, 1) == 0  # about 1 ms, loads held
        assert lib.lemc_run(smp._h, 1, 1) == TIMEOUT
        assert lib.lemc_synchronize(smp._h) == TIMEOUT
    finally:
        assert lib.lemc_debug_gram_wait(0, 0) == 0
    # the CUDA context is intact: the same context computes after a reset
    smp.reset()
    smp.run(20, measure=True)
    S, H2, H4, n = smp.gram(0)
    assert n == 20 * 2048 and np.all(np.isfinite(S)) and np.real(S[0, 0]) > 0
    smp.close()
    # and a fresh context runs clean
    smp = _sampler(lemc, 4)
    smp.run(10, measure=True)
    assert lib.lemc_synchronize(smp._h) == 0
    smp.close()
