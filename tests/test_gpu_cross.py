"""Excitation and edge-density matrices on the same records (row a11 of the
reference's excitationResponse_sampler, em_edgeResponse.tpp:26-194): the
cross-sector sums Cuser, Ccos, Csin that the CUDA path accumulates from V and
the weight planes, against an FP64 numpy contraction of the same V planes and
weights.  U is a caller potential written into the USER plane (as a hook
does), the cos/sin planes are the sweep kernel's own probe records."""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_cross_sums_match_numpy_on_same_records(lemc, oracle, cuda_ctx):
    torch = cuda_ctx
    lib = lemc.load()
    N, m, W, seed = 8, 3, 4096, 31
    sectors, probes = [0, 2, 4], [2, 4]
    R = math.sqrt(2 * m * N)
    K = 4
    Wpad = (W + 63) // 64 * 64
    pos = torch.from_numpy(oracle.init_walkers(W, N, R, seed)).cuda()
    rec_p = torch.zeros((K, W, 2), dtype=torch.float32, device="cuda")
    rec_w = torch.zeros((lemc._lib.N_WEIGHTS, Wpad), dtype=torch.float32, device="cuda")
    prb = np.array(probes, np.int32)
    for sweep0, n, meas in ((0, 300, 0), (300, 1, 1)):
        st = lib.lemc_sweep_device(C.c_void_p(pos.data_ptr()), W, N, m, 0.3, seed, sweep0, n, K, R,
                                   0, meas, lemc._lib.i32ptr(prb), len(probes),
                                   C.c_void_p(rec_p.data_ptr()), C.c_void_p(rec_w.data_ptr()),
                                   None, None)
        assert st == 0, st
    torch.cuda.synchronize()
    xy = pos.cpu().numpy().astype(np.float64)
    U = np.sum((xy[..., 0] / R) ** 2, axis=1)  # the reference main.cu's example potential
    rec_w[lemc._lib.W_USER, :W] = torch.from_numpy(U.astype(np.float32)).cuda()
    smp = lemc.Sampler(lemc.SamplerConfig(N, m, W), sectors, probes=probes)
    V = torch.zeros((2 * smp.total_dim, Wpad), dtype=torch.float32, device="cuda")
    assert lib.lemc_basis_device(smp._h, C.c_void_p(rec_p.data_ptr()), W, C.c_void_p(V.data_ptr()),
                                 Wpad, None) == 0
    # the cross planes are accumulated when probes are set
    assert lib.lemc_gram_device(smp._h, C.c_void_p(V.data_ptr()), C.c_void_p(rec_w.data_ptr()), W,
                                Wpad, lemc._lib.GRAM_FP64, None) == 0
    torch.cuda.synchronize()
    smp.synchronize()
    Vh = V.cpu().numpy().astype(np.float64)[:, :W]
    wts = rec_w.cpu().numpy().astype(np.float64)[:, :W]
    # complex basis values per sector: rows [2 f, 2 f + d) Re, [2 f + d, 2 f + 2 d) Im
    vals, first = [], 0
    for d in smp.dims:
        vals.append(Vh[2 * first:2 * first + d] + 1j * Vh[2 * first + d:2 * first + 2 * d])
        first += d
    checked = 0
    for a, la in enumerate(sectors):
        for b, lb in enumerate(sectors):
            if a == b:
                continue
            cu, cc, cs = smp.cross(a, b)
            va, vb = vals[a], vals[b]
            ref_u = np.einsum("w,aw,bw->ab", wts[0] * wts[lemc._lib.W_USER], va.conj(), vb)
            scale = np.sqrt(np.einsum("aw,aw->a", va.conj(), va).real)
            scale = np.outer(scale, np.sqrt(np.einsum("bw,bw->b", vb.conj(), vb).real))
            assert np.max(np.abs(cu - ref_u) / scale) < 1e-9
            l = abs(lb - la)
            if l in probes:
                q = probes.index(l)
                for got, plane in ((cc, 4 + 2 * q), (cs, 5 + 2 * q)):
                    ref = np.einsum("w,aw,bw->ab", wts[0] * wts[plane], va.conj(), vb)
                    assert np.max(np.abs(got - ref) / scale) < 1e-9
                    checked += 1
            else:
                assert np.all(cc == 0) and np.all(cs == 0)
    assert checked == 12  # every ordered pair of distinct sectors x {cos, sin}
    smp.close()
