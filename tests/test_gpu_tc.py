"""tcgen05 split-precision S/H contraction against the FP64 accumulation of the
same samples (same V planes, same weights), through the C-ABI."""
import ctypes as C
import math

import numpy as np
import pytest

from test_gpu_parity import dev_sweep

pytestmark = pytest.mark.gpu

# Error measure: for each Gram matrix X (S, H2, H4) of each sector, the largest
# |X_tc - X_fp64| / sqrt(S_aa S_bb), divided by the largest |X_fp64| / sqrt(S_aa S_bb)
# of that matrix (1 for S, whose normalised diagonal is 1): a max-norm relative
# error of the normalised matrix.  Per mode: the BF16 hi/lo split carries 16
# significant bits (~1e-5 on heavy-tailed sums, with or without the lo*lo product);
# TF32 hi/lo (22 bits) is held to the 1e-6 target.
TOL = {1: 3e-5, 2: 2e-5, 3: 1e-6}


def _records(lemc, oracle, torch, N, m, W, sectors, seed, sweeps):
    R = math.sqrt(2 * m * N)
    K = max(4, max(sectors))
    pos0 = oracle.init_walkers(W, N, R, seed)
    # thermalise a little on the device, then take one measured sweep
    gpos, _, _, _ = dev_sweep(lemc, torch, pos0, m, 0.3, seed, 0, sweeps, K, R, 0)
    gpos, rp, rw, _ = dev_sweep(lemc, torch, gpos, m, 0.3, seed, sweeps, 1, K, R, 0, measure=1)
    return rp, rw


def _gram_both(lemc, torch, N, m, W, sectors, rp, rw, mode, flush=0):
    lib = lemc.load()
    out = {}
    Wpad = (W + 63) // 64 * 64
    for md in (lemc._lib.GRAM_FP64, mode):
        smp = lemc.Sampler(lemc.SamplerConfig(N, m, W, flush_every=flush), sectors)
        rec_p = torch.from_numpy(np.ascontiguousarray(rp)).cuda()
        rec_w = torch.zeros((lemc._lib.N_WEIGHTS, Wpad), dtype=torch.float32, device="cuda")
        rec_w[:rw.shape[0], :W] = torch.from_numpy(np.ascontiguousarray(rw)).cuda()
        V = torch.zeros((2 * smp.total_dim, Wpad), dtype=torch.float32, device="cuda")
        assert lib.lemc_basis_device(smp._h, C.c_void_p(rec_p.data_ptr()), W,
                                     C.c_void_p(V.data_ptr()), Wpad, None) == 0
        assert lib.lemc_gram_device(smp._h, C.c_void_p(V.data_ptr()), C.c_void_p(rec_w.data_ptr()),
                                    W, Wpad, md, None) == 0
        torch.cuda.synchronize()
        smp.synchronize()
        out[md] = [smp.gram(s)[:3] for s in range(len(sectors))]
        smp.close()
    return out[lemc._lib.GRAM_FP64], out[mode]


def _rel_err(ref, got):
    worst = 0.0
    for (S, H2, H4), (S2, H22, H42) in zip(ref, got):
        d = np.sqrt(np.real(np.diag(S)))
        nrm = np.outer(d, d)
        for X, Y, sc in ((S, S2, 1.0), (H2, H22, np.max(np.abs(H2 / nrm))), (H4, H42, np.max(np.abs(H4 / nrm)))):
            worst = max(worst, float(np.max(np.abs(X - Y) / nrm) / sc))
    return worst


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_tc_gram_small(lemc, oracle, cuda_ctx, mode):
    N, m, W = 8, 3, 4096
    sectors = [0, 1, 2, 3, 4, 5, 6]
    rp, rw = _records(lemc, oracle, cuda_ctx, N, m, W, sectors, 21, 20)
    ref, got = _gram_both(lemc, cuda_ctx, N, m, W, sectors, rp, rw, mode)
    err = _rel_err(ref, got)
    print(f"mode {mode}: max normalised error {err:.3e}")
    assert err < TOL[mode]


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_tc_gram_config2_shapes(lemc, oracle, cuda_ctx, mode):
    N, m, W = 50, 3, 8192
    sectors = list(range(13))
    rp, rw = _records(lemc, oracle, cuda_ctx, N, m, W, sectors, 5, 10)
    ref, got = _gram_both(lemc, cuda_ctx, N, m, W, sectors, rp, rw, mode)
    err = _rel_err(ref, got)
    print(f"mode {mode}: max normalised error {err:.3e}")
    assert err < TOL[mode]


def test_tf32x3_bench_shape(lemc, oracle, cuda_ctx):
    """TF32x3 at the mixed-precision workload's own shape: N = 50, dL = 0..12,
    W = 65536 (the walker split of the timed runs), burnt-in walkers."""
    N, m, W = 50, 3, 65536
    sectors = list(range(13))
    rp, rw = _records(lemc, oracle, cuda_ctx, N, m, W, sectors, 9, 40)
    ref, got = _gram_both(lemc, cuda_ctx, N, m, W, sectors, rp, rw, 3)
    err = _rel_err(ref, got)
    print(f"tf32x3 N=50 W=65536: max normalised error {err:.3e}")
    assert err < TOL[3]


@pytest.mark.parametrize("N, sectors, W, splits", [
    (200, list(range(1, 21)), 65536, 4),   # 604 tiles: 4.08 waves at split 1, 16.3 of 17 at 4
    (200, list(range(1, 21)), 8192, 1),    # a wave-adding split keeps >= 8192 walkers per job
    (50, list(range(13)), 65536, 7),       # 20 tiles: 140 jobs in one wave
])
def test_contraction_split_fills_waves(lemc, cuda_ctx, N, sectors, W, splits):
    """The default walker split of the tcgen05 contraction (one CTA per SM on
    the B200's 148 SMs): fill whole waves of jobs."""
    import torch
    if torch.cuda.get_device_properties(0).multi_processor_count != 148:
        pytest.skip("split counts stated for 148 SMs")
    smp = lemc.Sampler(lemc.SamplerConfig(N, 3, W, lanes_per_walker=4,
                                          gram_mode=lemc._lib.GRAM_TF32X3), sectors)
    smp.init_walkers()
    smp.run(1, measure=True)
    smp.synchronize()
    assert smp.gram_splits() == splits
    smp.close()
