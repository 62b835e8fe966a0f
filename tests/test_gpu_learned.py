"""Learned Metropolis-Hastings proposal, through the C-ABI: the network and
the exact acceptance ratio against a numpy restatement, exactness of the
sampled distribution (closed-form <sum r^2> of the Laughlin state), and
training (the objective rises)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H, NB = 64, 16


def _bf16(x):
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _split(p):
    p = _bf16(p)
    o = 0
    W1 = p[o:o + 2 * H].reshape(H, 2); o += 2 * H
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * (H + 1)].reshape(H, H + 1); o += H * (H + 1)
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + 4 * H].reshape(4, H); o += 4 * H
    b3 = p[o:o + 4]
    return W1, b1, W2, b2, W3, b3


def _net(P, zs, i, zc, R):
    W1, b1, W2, b2, W3, b3 = P
    r = math.hypot(zc[0], zc[1])
    c, s = (zc[0] / r, zc[1] / r) if r > 1e-10 else (1.0, 0.0)
    others = [j for j in range(len(zs)) if j != i]
    d = zs[others].astype(np.float32) - np.float32(zc).astype(np.float32)
    d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]).astype(np.float32)
    keys = (d2.view(np.uint32) & np.uint32(0xFFFFFF00)) | np.array(others, dtype=np.uint32)
    sel = [others[k] for k in np.argsort(keys, kind="stable")[:NB]]
    g = np.zeros(H)
    for j in sel:
        dx, dy = zs[j, 0] - zc[0], zs[j, 1] - zc[1]
        x = np.array([(dx * c + dy * s) * 0.5, (dy * c - dx * s) * 0.5])
        g += np.maximum(W1 @ x + b1, 0.0)
    g /= len(sel)
    k = np.maximum(W2[:, :H] @ g + W2[:, H] * (r / R - 1.0) + b2, 0.0)
    o = W3 @ k + b3
    return o[0], o[1], np.clip(o[2], 0.0, math.log(4.0)), np.clip(o[3], 0.0, math.log(4.0))


def _propose(P, zs, i, eps, m, R):
    zo = zs[i].astype(np.float64)
    mr, mt, lr, lt = _net(P, zs, i, zo, R)
    dr, dt = mr + math.exp(lr) * eps[0], mt + math.exp(lt) * eps[1]
    r = math.hypot(*zo)
    c, s = zo / r
    zn = zo + np.array([c * dr - s * dt, s * dr + c * dt])
    lqf = -0.5 * (eps[0] ** 2 + eps[1] ** 2) - lr - lt
    zs2 = zs.astype(np.float64).copy()
    bmr, bmt, blr, blt = _net(P, zs2, i, zn, R)
    rn = math.hypot(*zn)
    cb, sb = zn / rn
    bx, by = zo - zn
    br, bt = bx * cb + by * sb, by * cb - bx * sb
    lqb = -0.5 * (((br - bmr) / math.exp(blr)) ** 2 + ((bt - bmt) / math.exp(blt)) ** 2) - blr - blt
    others = np.array([j for j in range(len(zs)) if j != i])
    lj = np.sum(np.log(np.sum((zn - zs[others]) ** 2, 1)) - np.log(np.sum((zo - zs[others]) ** 2, 1)))
    la = m * lj - 0.5 * (rn * rn - r * r) + lqb - lqf
    return (mr, mt, lr, lt, zn[0], zn[1], la, np.sum((zn - zo) ** 2))


def _random_params(lemc, rng, sigma=0.4, N=20):
    prop = lemc.LearnedProposal(N, 3, init_sigma=sigma, seed=5)
    p = prop.params.copy()
    # make mu and s depend on the neighbourhood
    n_w3 = 4 * H + 4
    p[-n_w3:-4] += 0.005 * rng.standard_normal(4 * H).astype(np.float32)
    prop.params = p
    return prop


def test_network_and_ratio_match_numpy(lemc, cuda_ctx):
    rng = np.random.default_rng(11)
    N, m = 20, 3
    R = math.sqrt(2 * m * N)
    prop = _random_params(lemc, rng)
    n = 24
    rad = R * np.sqrt(rng.random((n, N)))
    th = 2 * math.pi * rng.random((n, N))
    xy = np.stack([rad * np.cos(th), rad * np.sin(th)], -1).astype(np.float32)
    part = rng.integers(0, N, n).astype(np.int32)
    eps = rng.standard_normal((n, 2)).astype(np.float32)
    _check_against_numpy(prop, xy, part, eps, m, R)
    prop.close()


def _check_against_numpy(prop, xy, part, eps, m, R):
    out = prop.evaluate(xy, part, eps)
    P = _split(prop.params)
    for s in range(xy.shape[0]):
        ref = _propose(P, xy[s].astype(np.float64), int(part[s]), eps[s].astype(np.float64), m, R)
        np.testing.assert_allclose(out[s, :4], ref[:4], atol=2e-4, rtol=1e-3)
        np.testing.assert_allclose(out[s, 4:6], ref[4:6], atol=2e-4, rtol=1e-4)
        assert abs(out[s, 6] - ref[6]) < 2e-3 * max(1.0, abs(ref[6])), (s, out[s, 6], ref[6])
        np.testing.assert_allclose(out[s, 7], ref[7], rtol=1e-3, atol=1e-5)


def test_neighbour_selection_paths_match_numpy(lemc, cuda_ctx):
    """N=200 (eight particles per lane, sixteen selection rounds): the
    network and the ratio against numpy for sampled Laughlin configurations,
    uniform-disk ones, a tight cluster and a sparse spread."""
    rng = np.random.default_rng(21)
    N, m = 200, 3
    R = math.sqrt(2 * m * N)
    prop = _random_params(lemc, rng, sigma=1.0, N=N)
    smp = lemc.Sampler(lemc.SamplerConfig(N, m, 64, step_sigma=1.2, seed=4), [0])
    smp.init_walkers()
    smp.run(300, measure=False)
    laughlin = smp.positions().reshape(64, N, 2)[:12].astype(np.float32)
    smp.close()
    n = 12
    fams = [laughlin]
    for scale in (1.0, 0.05, 3.0):  # uniform disk, cluster, spread
        rad = scale * R * np.sqrt(rng.random((n, N)))
        th = 2 * math.pi * rng.random((n, N))
        fams.append(np.stack([rad * np.cos(th), rad * np.sin(th)], -1).astype(np.float32))
    for xy in fams:
        part = rng.integers(0, N, xy.shape[0]).astype(np.int32)
        eps = rng.standard_normal((xy.shape[0], 2)).astype(np.float32)
        _check_against_numpy(prop, np.ascontiguousarray(xy), part, eps, m, R)
    prop.close()


def _r2_mean(lemc, N, m, W, seed, proposal=None):
    smp = lemc.Sampler(lemc.SamplerConfig(N, m, W, step_sigma=0.4, seed=seed), [0])
    if proposal is not None:
        smp.set_proposal(proposal)
    smp.init_walkers()
    smp.run(600, measure=False)
    smp.run(200, measure=True)
    S, H2, _, _ = smp.gram(0)
    st = smp.stats()
    smp.close()
    # every accepted move had its reverse density evaluated; the Gaussian step has none
    if proposal is None:
        assert st.reverse_fraction == 0.0
    else:
        assert st.acceptance <= st.reverse_fraction <= 1.0, (st.acceptance, st.reverse_fraction)
    return float(np.real(H2[0, 0] / S[0, 0])), st.acceptance


def test_learned_sampler_is_exact(lemc, cuda_ctx):
    """<sum_i |z_i|^2> of the Laughlin state is 2 (m N (N-1)/2 + N) exactly."""
    rng = np.random.default_rng(12)
    N, m, W = 20, 3, 2048
    prop = _random_params(lemc, rng)
    exact = 2.0 * (m * N * (N - 1) / 2 + N)
    learned = [_r2_mean(lemc, N, m, W, 100 + r, prop) for r in range(4)]
    plain = [_r2_mean(lemc, N, m, W, 200 + r) for r in range(4)]
    for vals in (learned, plain):
        v = np.array([x[0] for x in vals])
        err = v.std(ddof=1) / math.sqrt(len(v)) + 1e-4 * exact
        assert abs(v.mean() - exact) < 5 * err, (v, exact)
    assert 0.3 < np.mean([x[1] for x in learned]) < 0.99
    prop.close()


def test_training_raises_the_objective(lemc, cuda_ctx):
    import torch
    N, m, W = 20, 3, 2048
    smp = lemc.Sampler(lemc.SamplerConfig(N, m, W, step_sigma=0.3, seed=3), [1])
    smp.init_walkers()
    smp.run(400, measure=False)
    cfg = torch.empty((W, N, 2), dtype=torch.float32, device="cuda")
    smp.copy_positions_device(cfg.data_ptr())
    smp.synchronize()
    # start at the smallest step the family allows (s = 1); the objective's
    # per-step noise is about 0.2 %, so a 5 % rise is the training's doing
    prop = lemc.LearnedProposal(N, m, init_sigma=1.0, seed=9)
    trace = prop.train(cfg.data_ptr(), W, steps=300, batch=512, pairs=16, lr=5e-3)
    assert np.all(np.isfinite(trace))
    assert trace[-30:].mean() > 1.05 * trace[:30].mean(), (trace[:30].mean(), trace[-30:].mean())
    smp.close()
    prop.close()


def _u01(x):
    # lemc_rng.h u01: ((x >> 9) + 1/2) * 2^-23, exact in FP32
    return (float(x >> 9) + 0.5) * 2.0 ** -23


def test_learned_chain_matches_numpy_move_by_move(lemc, oracle, cuda_ctx):
    """Two sweeps of the learned sampler (N=20, 24 walkers) against a numpy
    restatement that always evaluates the full Metropolis-Hastings ratio with
    the same Philox draws {move, sweep, walker, 4}: the sweep's early
    rejection (the reverse network skipped when ln u >= ln A without it)
    must take the same decisions.  A walker may leave the numpy trajectory
    only at a near tie |ln A - ln u| < 1e-3 (FP32 network against FP64)."""
    rng = np.random.default_rng(31)
    N, m, W, seed, n_sweeps = 20, 3, 24, 977, 2
    R = math.sqrt(2 * m * N)
    prop = _random_params(lemc, rng, sigma=1.5, N=N)
    smp = lemc.Sampler(lemc.SamplerConfig(N, m, W, step_sigma=0.3, seed=seed), [0])
    smp.set_proposal(prop)
    rad = R * np.sqrt(rng.random((W, N)))
    th = 2 * math.pi * rng.random((W, N))
    xy0 = np.stack([rad * np.cos(th), rad * np.sin(th)], -1).astype(np.float32)
    smp.init_walkers(xy0)
    smp.run(n_sweeps, measure=False)
    got = smp.positions().reshape(W, N, 2)
    st = smp.stats()
    smp.close()
    P = _split(prop.params)
    key = (seed & 0xFFFFFFFF, seed >> 32)
    good, ties, skipped = 0, 0, 0
    for w in range(W):
        zs = xy0[w].astype(np.float64).copy()
        margin = np.inf
        for sw in range(n_sweeps):
            for i in range(N):
                r = oracle.philox([i, sw, w, 4], key)
                rad_ = math.sqrt(-2.0 * math.log(_u01(r[0])))
                ang = 2.0 * math.pi * _u01(r[1])
                eps = np.array([rad_ * math.cos(ang), rad_ * math.sin(ang)])
                lu = math.log(_u01(r[2]))
                out = _propose(P, zs.astype(np.float32).astype(np.float64), i, eps, m, R)
                la = out[6]
                margin = min(margin, abs(la - lu))
                if lu < la:
                    zs[i] = [out[4], out[5]]
        if np.allclose(got[w], zs, atol=2e-3, rtol=0):
            good += 1
        else:
            assert margin < 1e-3, (w, margin)
            ties += 1
    assert good >= W - 2, (good, ties)
    # the early rejection ran: fewer reverse evaluations than moves, and
    # never fewer than accepted moves
    assert st.acceptance <= st.reverse_fraction < 1.0, (st.acceptance, st.reverse_fraction)
    prop.close()
