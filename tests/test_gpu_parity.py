"""Parity of the CUDA path (through the C-ABI) with the oracle.

Deterministic parity on the same Philox stream: sweep trajectories, records,
basis values and FP64 Gram sums.  Statistical parity: known answers (harmonic
degeneracy, nu = 1 closed forms) and the reference estimator run by the oracle.
"""
import ctypes as C
import json
import math
from pathlib import Path

import numpy as np
import pytest
import scipy.linalg as sl

from kat import gram_m1, harmonic_level, spectrum_m1

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def dev_sweep(lemc, torch, pos_np, m, sigma, seed, sweep0, n_sweeps, K, R, G, measure=0, lprobe=0):
    lib = lemc.load()
    W, N = pos_np.shape[:2]
    pos = torch.from_numpy(np.ascontiguousarray(pos_np, np.float32)).cuda()
    rec_p = torch.zeros((K, W, 2), dtype=torch.float32, device="cuda")
    nprb = 1 if lprobe else 0
    rec_w = torch.zeros((4 + 2 * nprb, W), dtype=torch.float32, device="cuda")
    acc = torch.zeros(W, dtype=torch.int32, device="cuda")
    prb = np.array([lprobe], np.int32)
    st = lib.lemc_sweep_device(C.c_void_p(pos.data_ptr()), W, N, m, sigma, seed, sweep0, n_sweeps,
                               K, R, G, measure, lemc._lib.i32ptr(prb), nprb,
                               C.c_void_p(rec_p.data_ptr()), C.c_void_p(rec_w.data_ptr()),
                               C.c_void_p(acc.data_ptr()), None)
    assert st == 0, st
    torch.cuda.synchronize()
    return (pos.cpu().numpy(), rec_p.cpu().numpy(), rec_w.cpu().numpy(),
            acc.cpu().numpy().astype(np.int64))


# A walker may leave the oracle's trajectory only at a near tie: a move whose
# ln A (FP32 product chains on the GPU, FP64 in the oracle) lies within this
# distance of ln u, where the two roundings can decide differently.
TIE = 1e-3


def _compare_trajectories(gpu_pos, gpu_acc, orc_pos, orc_acc, max_bad, margins):
    same = (gpu_acc == orc_acc.astype(np.int64))
    close = np.max(np.abs(gpu_pos - orc_pos), axis=(1, 2)) < 1e-3
    good = same & close
    assert np.sum(~good) <= max_bad, (np.sum(~same), np.sum(~close))
    assert np.max(np.abs(gpu_pos[good] - orc_pos[good])) < 1e-3
    # every walker that diverged had a near-tie decision on the oracle's path
    assert np.all(margins[~good] < TIE), margins[~good]


@pytest.mark.parametrize("G", [1, 2, 4, 8, 16, 32])
def test_sweep_matches_oracle_move_by_move(lemc, oracle, cuda_ctx, G):
    N, m, W, sigma, seed = 8, 3, 64, 0.3, 42
    R = math.sqrt(2 * m * N)
    pos0 = oracle.init_walkers(W, N, R, seed)
    gpos, _, _, gacc = dev_sweep(lemc, cuda_ctx, pos0, m, sigma, seed, 5, 3, 6, R, G)
    opos = pos0.copy()
    mg = np.zeros(W)
    oacc = oracle.sweep(opos, m, sigma, seed, 5, 3, R, margins=mg)
    _compare_trajectories(gpos, gacc, opos, oacc, max_bad=2, margins=mg)


@pytest.mark.parametrize("G", [8, 32])
def test_sweep_matches_oracle_n50(lemc, oracle, cuda_ctx, G):
    N, m, W, sigma, seed = 50, 3, 32, 0.3, 7
    R = math.sqrt(2 * m * N)
    pos0 = oracle.init_walkers(W, N, R, seed)
    gpos, _, _, gacc = dev_sweep(lemc, cuda_ctx, pos0, m, sigma, seed, 0, 2, 12, R, G)
    opos = pos0.copy()
    mg = np.zeros(W)
    oacc = oracle.sweep(opos, m, sigma, seed, 0, 2, R, margins=mg)
    _compare_trajectories(gpos, gacc, opos, oacc, max_bad=2, margins=mg)


def test_records_match_oracle(lemc, oracle, cuda_ctx):
    N, m, W, K, seed = 8, 3, 128, 6, 3
    R = math.sqrt(2 * m * N)
    pos0 = oracle.init_walkers(W, N, R, seed)
    gpos, rp, rw, _ = dev_sweep(lemc, cuda_ctx, pos0, m, 0.3, seed, 0, 1, K, R, 8, measure=1,
                                lprobe=3)
    p_o, w_o = oracle.measure(gpos, K, R, lprobe=3)
    p_g = rp[..., 0].T + 1j * rp[..., 1].T
    scale = np.abs(p_o) + np.sqrt(N)
    assert np.max(np.abs(p_g - p_o) / scale) < 2e-6
    assert np.allclose(rw[1], w_o[:, 1], rtol=2e-6)
    assert np.allclose(rw[2], w_o[:, 2], rtol=2e-6)
    assert np.allclose(rw[4], w_o[:, 3], atol=2e-5)  # cos(3 theta) plane
    assert np.allclose(rw[5], w_o[:, 4], atol=2e-5)  # sin(3 theta) plane
    assert np.all(rw[0] == 1.0) and np.all(rw[3] == 0.0)


def _sampler(lemc, **kw):
    cfg = lemc.SamplerConfig(**{k: v for k, v in kw.items() if k != "sectors"})
    return lemc.Sampler(cfg, kw["sectors"])


@pytest.mark.parametrize("W", [256, 201])  # paired-walker and single-walker basis kernels
def test_basis_and_fp64_gram_match_oracle(lemc, oracle, cuda_ctx, W):
    torch = cuda_ctx
    N, m, seed = 8, 3, 11
    sectors = [0, 1, 2, 3, 4, 5, 6]
    R = math.sqrt(2 * m * N)
    smp = _sampler(lemc, particles=N, inverse_filling=m, n_walkers=W, sectors=sectors)
    lib = lemc.load()
    K = 6
    pos0 = oracle.init_walkers(W, N, R, seed)
    gpos, rp, rw, _ = dev_sweep(lemc, torch, pos0, m, 0.3, seed, 0, 2, K, R, 8, measure=1)
    Wpad = (W + 63) // 64 * 64
    rec_p = torch.from_numpy(np.ascontiguousarray(rp)).cuda()
    rec_w = torch.zeros((lemc._lib.N_WEIGHTS, Wpad), dtype=torch.float32, device="cuda")
    rec_w[:rw.shape[0], :W] = torch.from_numpy(rw).cuda()
    D = smp.total_dim
    V = torch.zeros((2 * D, Wpad), dtype=torch.float32, device="cuda")
    assert lib.lemc_basis_device(smp._h, C.c_void_p(rec_p.data_ptr()), W, C.c_void_p(V.data_ptr()),
                                 Wpad, None) == 0
    torch.cuda.synchronize()
    Vh = V.cpu().numpy().astype(np.float64)
    # oracle basis from the same records
    rows = oracle.partitions(N, sectors)
    p = rp[..., 0].T.astype(np.float64) + 1j * rp[..., 1].T.astype(np.float64)
    vo = oracle.basis_values(p, N, rows)
    first = 0
    for s, dim in enumerate(smp.dims):
        vg = Vh[2 * first:2 * first + dim, :W] + 1j * Vh[2 * first + dim:2 * first + 2 * dim, :W]
        ref = vo[:, first:first + dim].T
        assert np.max(np.abs(vg - ref) / (np.abs(ref) + 1e-30)) < 5e-6
        first += dim
    # FP64 Gram from the same V
    assert lib.lemc_gram_device(smp._h, C.c_void_p(V.data_ptr()), C.c_void_p(rec_w.data_ptr()), W,
                                Wpad, lemc._lib.GRAM_FP64, None) == 0
    torch.cuda.synchronize()
    first = 0
    for s, dim in enumerate(smp.dims):
        S, H2, H4, _ = smp.gram(s)
        vg = Vh[2 * first:2 * first + dim, :W] + 1j * Vh[2 * first + dim:2 * first + 2 * dim, :W]
        Sr = vg.conj() @ vg.T
        H2r = (vg.conj() * rw[1].astype(np.float64)) @ vg.T
        H4r = (vg.conj() * rw[2].astype(np.float64)) @ vg.T
        for X, Y in ((S, Sr), (H2, H2r), (H4, H4r)):
            assert np.max(np.abs(X - Y)) <= 1e-12 * np.max(np.abs(Y))
        first += dim
    smp.close()


def _spectra(lemc, N, m, W, sectors, seed, burn, meas, omega, kappa, guide=0, mode=0):
    smp = _sampler(lemc, particles=N, inverse_filling=m, n_walkers=W, sectors=sectors, seed=seed,
                   guide=guide, gram_mode=mode)
    smp.init_walkers()
    smp.run(burn, measure=False)
    smp.run(meas, measure=True)
    out = []
    for s in range(len(sectors)):
        if guide == 0:
            S, H2, H4, _ = smp.gram(s)
            M, H = lemc.normalise(S, H2, H4, omega, kappa)
        out.append(lemc.geneig(H, M))
    st = smp.stats()
    smp.close()
    return out, st


def test_gpu_harmonic_degeneracy(lemc, cuda_ctx):
    N, m = 8, 3
    sectors = [1, 2, 3, 4, 5, 6]
    evs, st = _spectra(lemc, N, m, 4096, sectors, 5, 300, 600, 1.0, 0.0)
    assert 0.3 < st.acceptance < 0.95
    for dL, ev in zip(sectors, evs):
        lvl = harmonic_level(N, m, dL)
        assert abs(np.mean(ev) - lvl) < 0.005 * lvl, (dL, ev, lvl)
        assert np.max(np.abs(ev - lvl)) < 0.03 * lvl


def test_gpu_m1_closed_forms(lemc, cuda_ctx):
    N, m = 5, 1
    sectors = [2, 3, 4]
    R = math.sqrt(2 * m * N)
    reps = []
    for r in range(4):
        smp = _sampler(lemc, particles=N, inverse_filling=m, n_walkers=4096, sectors=sectors,
                       seed=200 + r, step_sigma=0.5)
        smp.init_walkers()
        smp.run(300, measure=False)
        smp.run(800, measure=True)
        reps.append([smp.gram(s) for s in range(len(sectors))])
        smp.close()
    rows_all = lemc.partitions(N, sectors)[0]
    first = 0
    for s, dL in enumerate(sectors):
        rows = rows_all[first:first + reps[0][s][0].shape[0]]
        first += len(rows)
        ex = gram_m1(N, rows, R)
        de = np.sqrt(np.diag(ex))
        Me = ex / np.outer(de, de)
        Ms, evs, norms = [], [], []
        for rep in reps:
            S, H2, H4, n = rep[s]
            M, H = lemc.normalise(S, H2, H4, 0.01, 1e-3)
            Ms.append(M.real)
            evs.append(lemc.geneig(H, M))
            norms.append(S[0, 0].real / n)
        mean, err = np.mean(Ms, 0), np.std(Ms, 0, ddof=1) / 2 + 2e-4
        assert np.all(np.abs(mean - Me) < 5 * err), (dL, mean, Me)
        emean, eerr = np.mean(evs, 0), np.std(evs, 0, ddof=1) / 2 + 1e-5
        assert np.all(np.abs(emean - spectrum_m1(N, dL, 0.01, 1e-3)) < 5 * eerr)
        assert abs(np.mean(norms) / ex[0, 0] - 1) < 5 * np.std(norms, ddof=1) / 2 / ex[0, 0] + 1e-3


def test_gpu_row_guide_matches_oracle_move_by_move(lemc, oracle, cuda_ctx):
    N, m, W, seed, dL = 8, 3, 64, 9, 4
    R = math.sqrt(2 * m * N)
    smp = lemc.Sampler(lemc.SamplerConfig(N, m, W, seed=seed, guide=lemc._lib.GUIDE_ROW,
                                          lanes_per_walker=8), [dL])
    pos0 = oracle.init_walkers(W, N, R, seed)
    smp.init_walkers(pos0)
    smp.run(3, measure=False)
    gpos = smp.positions()
    st = smp.stats()
    rows = oracle.partitions(N, [dL])
    D = len(rows)
    wr = (np.arange(W) * D) // W
    opos = pos0.copy()
    mg = np.zeros(W)
    oacc = oracle.sweep(opos, m, 0.3, seed, 0, 3, R, rows=rows, walker_row=wr, margins=mg)
    close = np.max(np.abs(gpos - opos), axis=(1, 2)) < 1e-3
    assert np.sum(~close) <= 2
    assert np.all(mg[~close] < TIE), mg[~close]
    assert abs(st.acceptance - oacc.sum() / (3 * W * N)) < 0.01
    smp.close()


def test_cross_sector_sums_match_numpy(lemc, oracle, cuda_ctx):
    """USER / cos / sin planes between sector pairs, FP64 path, same records."""
    torch = cuda_ctx
    lib = lemc.load()
    N, m, W, seed = 8, 3, 256, 19
    sectors = [0, 2, 4]
    probes = [0, 2, 4]
    R = math.sqrt(2 * m * N)
    smp = lemc.Sampler(lemc.SamplerConfig(N, m, W), sectors, probes=probes)
    K = 4
    pos0 = oracle.init_walkers(W, N, R, seed)
    prb = np.array(probes, np.int32)
    pos = torch.from_numpy(pos0).cuda()
    rec_p = torch.zeros((K, W, 2), dtype=torch.float32, device="cuda")
    Wpad = W
    rec_w = torch.zeros((lemc._lib.N_WEIGHTS, Wpad), dtype=torch.float32, device="cuda")
    assert lib.lemc_sweep_device(C.c_void_p(pos.data_ptr()), W, N, m, 0.3, seed, 0, 2, K, R, 8, 1,
                                 lemc._lib.i32ptr(prb), len(probes), C.c_void_p(rec_p.data_ptr()),
                                 C.c_void_p(rec_w.data_ptr()), None, None) == 0
    user = torch.rand(W, device="cuda")
    rec_w[lemc._lib.W_USER] = user
    V = torch.zeros((2 * smp.total_dim, Wpad), dtype=torch.float32, device="cuda")
    assert lib.lemc_basis_device(smp._h, C.c_void_p(rec_p.data_ptr()), W, C.c_void_p(V.data_ptr()),
                                 Wpad, None) == 0
    assert lib.lemc_gram_device(smp._h, C.c_void_p(V.data_ptr()), C.c_void_p(rec_w.data_ptr()), W,
                                Wpad, lemc._lib.GRAM_FP64, None) == 0
    torch.cuda.synchronize()
    Vh = V.cpu().numpy().astype(np.float64)
    rw = rec_w.cpu().numpy().astype(np.float64)
    firsts = np.cumsum([0] + smp.dims)
    blocks = []
    for s, d in enumerate(smp.dims):
        f = firsts[s]
        blocks.append(Vh[2 * f:2 * f + d] + 1j * Vh[2 * f + d:2 * f + 2 * d])
    for i in range(3):
        for j in range(3):
            Cu, Cc, Cs = smp.cross(i, j)
            l = abs(sectors[j] - sectors[i])
            q = probes.index(l)
            va, vb = blocks[i], blocks[j]
            ref_u = (va.conj() * rw[lemc._lib.W_USER]) @ vb.T
            ref_c = (va.conj() * rw[lemc._lib.W_PROBE0 + 2 * q]) @ vb.T
            ref_s = (va.conj() * rw[lemc._lib.W_PROBE0 + 2 * q + 1]) @ vb.T
            for X, Y in ((Cu, ref_u), (Cc, ref_c), (Cs, ref_s)):
                assert np.max(np.abs(X - Y)) <= 1e-11 * max(1.0, np.max(np.abs(Y)))
    smp.close()
