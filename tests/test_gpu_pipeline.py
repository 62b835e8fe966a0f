"""The edge-response pipeline on the GPU (the reference's
excitationResponse_compute + edgeDensityResponse_compute): the built-in
multipole drive and the edge-density probes on the run path against a host
FP64 contraction of the same measurement, then sampling -> FP64 evolution ->
density on an angular grid, with the evolution checked against the host
Cash-Karp integrator, norm conservation and first-order response."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _host_values(L, xy, N, m, sectors):
    R = math.sqrt(2 * m * N)
    z = (xy[..., 0] + 1j * xy[..., 1]).astype(np.complex128) / R
    K = max(4, max(sectors))
    p = np.stack([np.sum(z ** k, axis=1) for k in range(1, K + 1)], 1)
    rows, _, _ = L.partitions(N, sectors)
    v = np.ones((xy.shape[0], len(rows)), complex)
    for b, (_, pr) in enumerate(rows):
        for k, mult in pr:
            v[:, b] *= (float(N) if k == 0 else p[:, k - 1]) ** mult
    return v, [d for d, _ in rows]


def test_multipole_drive_and_probes_on_run_path(lemc, cuda_ctx):
    N, m, W = 8, 3, 4096
    sectors, probes = [0, 2, 4], [2, 4]
    smp = lemc.Sampler(lemc.SamplerConfig(N, m, W, seed=12), sectors, probes=probes)
    assert smp.lib.lemc_set_multipole_potential(smp._h, 2, 1.0) == 0
    smp.init_walkers()
    smp.run(200, measure=False)
    smp.run(1, measure=True)  # one measurement at the positions read below
    xy = smp.positions().astype(np.float64)
    v, dls = _host_values(lemc, xy, N, m, sectors)
    U = np.sum(xy[..., 0] ** 2 - xy[..., 1] ** 2, axis=1)
    th = np.arctan2(xy[..., 1], xy[..., 0])
    dls = np.array(dls)
    for a, la in enumerate(sectors):
        for b, lb in enumerate(sectors):
            cu, cc, cs = smp.cross(a, b)
            va, vb = v[:, dls == la], v[:, dls == lb]
            den = np.outer(np.sqrt(np.sum(np.abs(va) ** 2, 0)), np.sqrt(np.sum(np.abs(vb) ** 2, 0)))
            ref = np.einsum("w,wa,wb->ab", U, va.conj(), vb)
            assert np.max(np.abs(cu - ref) / den) < 2e-5 * max(1.0, np.abs(ref / den).max())
            l = abs(lb - la)
            if l in probes:
                for got, w in ((cc, np.sum(np.cos(l * th), 1)), (cs, np.sum(np.sin(l * th), 1))):
                    ref = np.einsum("w,wa,wb->ab", w, va.conj(), vb)
                    assert np.max(np.abs(got - ref) / den) < 2e-5 * max(1.0, np.abs(ref / den).max())
    smp.close()


def test_edge_response_pipeline_small(lemc, cuda_ctx):
    N, m = 8, 3
    sectors = [0, 2, 4]
    eps, t0, tau = 1e-3, 5.0, 1.5
    prof = lambda t: eps * math.exp(-((t - t0) ** 2) / (2 * tau ** 2))
    out = lemc.edge_response(N, m, sectors, 2, 1e-2, 1e-4, prof, end_time=20.0, save_step=0.05,
                             n_walkers=8192, burn_in=300, sweeps=400,
                             gram_mode=lemc._lib.GRAM_FP64, substeps=2)
    rho_t, norms = out["rho_t"], out["norms"]
    assert rho_t.shape == (400, 3) and out["density"].shape == (400, 256)
    assert np.max(np.abs(norms - 1.0)) < 1e-8
    assert np.max(np.abs(rho_t[:, 0] - N * norms)) < 1e-6 * N
    # density grid against the formula on the host
    th = 2 * np.pi * np.arange(256) / 256
    d = rho_t - rho_t[0]
    ref = (d[:, 0].real[:, None] + 2 * (np.real(d[:, 1:, None] * np.exp(-1j * np.array([2, 4])[None, :, None] * th[None, None, :]))).sum(1)) / (2 * np.pi)
    assert np.allclose(out["density"], ref, atol=1e-12)
    # the GPU RK4 against the host adaptive Cash-Karp on the same matrices
    _, rho_h, norms_h = lemc.evolve(out["M"], out["H"], out["U"], out["rho"], prof, 20.0, 0.05)
    scale = np.abs(rho_h[:, 1]).max()
    assert np.max(np.abs(rho_t[:, 1:] - rho_h[:, 1:])) < 1e-5 * max(scale, 1.0)
    # first order in the drive: the k = 2 drive moves <rho_2>; <rho_4> only at second order
    d2, d4 = np.abs(d[:, 1]).max(), np.abs(d[:, 2]).max()
    assert d2 > 0 and d4 < 0.05 * d2, (d2, d4)
