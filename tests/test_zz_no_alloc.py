"""The allocation-free occupation entry point (lemc_occupation_static) against
lemc_occupation, through the C-ABI, on two calls in a row.

Collected last on purpose: it must pass both in a fresh process and after the
other GPU tests have used the device.
"""
import ctypes as C

import numpy as np
import pytest

from laughlinedge_b200 import _lib
from laughlinedge_b200.sampler import partitions


def _call(fn, cfg, D, Lc):
    out = np.zeros(2 * D * D * Lc)
    acc = C.c_double()
    st = fn(C.byref(cfg), out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(acc))
    assert st == 0, _lib.load().lemc_status_string(st)
    return out.view(np.complex128).reshape(D, D, Lc), acc.value


@pytest.mark.gpu
def test_static_scratch_matches_allocating_entry_point(cuda_ctx):
    lib = _lib.load()
    N, m, dL = 6, 3, 2
    Lc = m * (N - 1) + 6
    D = len(partitions(N, [dL])[0])
    free_after = []
    for seed in (21, 22):  # two calls in a row: the scratch is reused and re-zeroed
        cfg = _lib.OccConfig(N, m, dL, Lc, 4096, 0.3, seed, 200, 300)
        ref, acc_ref = _call(lib.lemc_occupation, cfg, D, Lc)
        cuda_ctx.cuda.synchronize()
        free_before = cuda_ctx.cuda.mem_get_info()[0]
        got, acc_got = _call(lib.lemc_occupation_static, cfg, D, Lc)
        cuda_ctx.cuda.synchronize()
        free_after.append((free_before, cuda_ctx.cuda.mem_get_info()[0]))
        # same kernels, same seed: the tolerance of the occupation tests' sum rule
        assert np.allclose(got, ref, rtol=1e-5, atol=1e-8), np.abs(got - ref).max()
        assert abs(acc_got - acc_ref) < 1e-12
        n = got[0, 0].real / got[0, 0].real.sum() * N
        assert np.isclose(n.sum(), N)
    # the second call (module loaded, scratch address resolved by the first)
    # leaves the device's free memory exactly as it found it
    before, after = free_after[1]
    assert before == after, (before, after)


@pytest.mark.gpu
def test_static_scratch_rejects_oversized_configs(cuda_ctx):
    lib = _lib.load()
    # 16 * l_cutoff * W bytes of per-walker sums alone exceed the 64 MiB array
    cfg = _lib.OccConfig(8, 3, 1, 64, 1 << 17, 0.3, 1, 10, 10)
    out = np.zeros(2 * 64)
    assert lib.lemc_occupation_static(C.byref(cfg), out.ctypes.data_as(C.POINTER(C.c_double)),
                                      None) == -2  # LEMC_ERR_CAPACITY
