"""Edge density response: sampling of the matrix elements under a multipole
drive, FP64 evolution in the S-orthonormal edge basis, and the density
response on an angular grid -- the reference's excitationResponse_compute
followed by timeEvolution::edgeDensityResponse_compute
(em_edgeResponse.tpp:26-194; dynamics.cpp:149-308), all through liblemc.

The drive is delta V(r, theta, t) = amp r^k cos(k theta) f(t).  The matrix
elements (M, H of every sector, U = <f|sum_i r_i^k cos(k theta_i)|g>, and the
edge-density Fourier matrices rho_l = <f|sum_i e^{i l theta_i}|g> between
sectors l apart) come from one sampling context; rho_0 = N M.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import _lib
from ._lib import check, dptr, i32ptr
from .sampler import Sampler, SamplerConfig, evolve_device, normalise


def density_grid(ls, rho_t, n_theta=256, rho_ref=None):
    """delta rho(theta_g, t) = (1/2pi)[d_0 + 2 Re sum_{l>0} e^{-i l theta_g} d_l(t)],
    d_l = <rho_l>(t) - rho_ref (default: the first time), theta_g = 2 pi g / n_theta;
    computed on the GPU (lemc_edge_density_grid).  Returns [n_times, n_theta]."""
    lib = _lib.load()
    l = np.ascontiguousarray(ls, dtype=np.int32)
    r = np.ascontiguousarray(rho_t, dtype=np.complex128)
    nt, L = r.shape
    ref = None if rho_ref is None else np.ascontiguousarray(rho_ref, dtype=np.complex128).view(np.float64)
    out = np.zeros(nt * n_theta)
    check(lib.lemc_edge_density_grid(L, i32ptr(l), nt, dptr(r.view(np.float64).ravel()),
                                     None if ref is None else dptr(ref), n_theta, dptr(out)),
          "lemc_edge_density_grid")
    return out.reshape(nt, n_theta)


def response_matrices(smp: Sampler, sectors, omega, kappa):
    """M, H (block diagonal, normalised), U and rho_l (l = every sector's dL)
    from a context sampled with a multipole potential and the probes l > 0,
    normalised by sqrt(S_aa S_bb) and Hermitised (reference layout)."""
    D = smp.total_dim
    M = np.zeros((D, D), complex)
    H = np.zeros((D, D), complex)
    U = np.zeros((D, D), complex)
    first, nrm = [], []
    f = 0
    for si, d in enumerate(smp.dims):
        S, H2, H4, _ = smp.gram(si)
        Mn, Hn = normalise(S, H2, H4, omega, kappa)
        M[f:f + d, f:f + d] = Mn
        H[f:f + d, f:f + d] = Hn
        nrm.extend(np.sqrt(np.real(np.diag(S))))
        first.append(f)
        f += d
    nrm = np.array(nrm)
    ls = list(sectors)
    rho = {l: np.zeros((D, D), complex) for l in ls}
    for si in range(len(sectors)):
        for sj in range(len(sectors)):
            cu, cc, cs = smp.cross(si, sj)
            a0, b0, da, db = first[si], first[sj], smp.dims[si], smp.dims[sj]
            den = np.outer(nrm[a0:a0 + da], nrm[b0:b0 + db])
            U[a0:a0 + da, b0:b0 + db] = cu / den
            l = abs(sectors[sj] - sectors[si])
            if l > 0 and l in rho:
                rho[l][a0:a0 + da, b0:b0 + db] = (cc + 1j * cs) / den
    if 0 in rho:
        rho[0] = smp.cfg.particles * M
    herm = lambda X: 0.5 * (X + X.conj().T)
    return herm(M), herm(H), herm(U), [rho[l] for l in ls]


def edge_response(particles, inverse_filling, sectors, k, omega, kappa, profile, end_time, save_step,
                  n_walkers=65536, burn_in=1000, sweeps=200, step_sigma=0.3, seed=42,
                  gram_mode=_lib.GRAM_TF32X3, proposal=None, substeps=1, n_theta=256,
                  init_xy=None, graph_batch=0, eps=1e-10):
    """The whole pipeline; returns a dict with the matrices, times, <rho_l>(t),
    norms, the density grid [n_save, n_theta] and the time of each stage."""
    sectors = list(sectors)
    if sectors[0] != 0:
        raise ValueError("the Laughlin state (dL = 0) must be the first sector (initial state)")
    probes = sorted({abs(a - b) for a in sectors for b in sectors} - {0})
    probes = [l for l in probes if l in sectors]
    t = {}
    t0 = time.perf_counter()
    smp = Sampler(SamplerConfig(particles, inverse_filling, n_walkers, step_sigma=step_sigma, seed=seed,
                                gram_mode=gram_mode, graph_batch=graph_batch), sectors, probes=probes)
    try:
        if proposal is not None:
            smp.set_proposal(proposal)
        check(smp.lib.lemc_set_multipole_potential(smp._h, int(k), 1.0), "lemc_set_multipole_potential")
        smp.init_walkers(init_xy)
        smp.run(burn_in, measure=False)
        smp.run(sweeps, measure=True)
        smp.synchronize()
        t["sampling_s"] = time.perf_counter() - t0
        M, H, U, rho = response_matrices(smp, sectors, omega, kappa)
        acc = smp.stats().acceptance
    finally:
        smp.close()
    t1 = time.perf_counter()
    times, rho_t, norms, rank = evolve_device(M, H, U, rho, profile, end_time, save_step,
                                              substeps=substeps, eps=eps)
    t["evolution_s"] = time.perf_counter() - t1
    t2 = time.perf_counter()
    grid = density_grid(sectors, rho_t, n_theta)
    t["density_grid_s"] = time.perf_counter() - t2
    return {"M": M, "H": H, "U": U, "rho": rho, "times": times, "rho_t": rho_t, "norms": norms,
            "rank": rank, "density": grid, "acceptance": acc, "timings": t, "sectors": sectors}
