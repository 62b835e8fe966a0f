"""Python face of the C-ABI: the sampling context and the FP64 dense tail.

Names mirror the reference's host API (modules/edge_montecarlo.h:199-236):
:func:`spectrum_compute`, :func:`metric_compute` and :func:`dsf_compute` run the
same estimators the C++ drop-in layer runs, through ``liblemc.so``.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, dptr, fptr, i32ptr


def partitions(particles: int, sectors):
    """Basis rows in reference order: list of (dL, [(part, mult), ...])."""
    lib = _lib.load()
    sec = np.ascontiguousarray(sectors, dtype=np.int32)
    n_rows, n_ints, maxdeg, longest = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    check(lib.lemc_partitions(particles, i32ptr(sec), len(sec), None, 0, None, 0,
                              C.byref(n_rows), C.byref(n_ints), C.byref(maxdeg), C.byref(longest)),
          "lemc_partitions")
    rows = (_lib.PartitionRow * max(1, n_rows.value))()
    pairs = np.zeros(max(1, n_ints.value), dtype=np.int32)
    check(lib.lemc_partitions(particles, i32ptr(sec), len(sec), rows, n_rows.value, i32ptr(pairs),
                              len(pairs), C.byref(n_rows), C.byref(n_ints), None, None),
          "lemc_partitions")
    out = []
    for r in rows[: n_rows.value]:
        pr = [(int(pairs[r.pairs_off + 2 * q]), int(pairs[r.pairs_off + 2 * q + 1]))
              for q in range(r.n_pairs)]
        out.append((int(r.dL), pr))
    return out, maxdeg.value, longest.value


def _cplx(buf: np.ndarray, D: int) -> np.ndarray:
    return buf.view(np.complex128).reshape(D, D)


def geneig(H: np.ndarray, M: np.ndarray, eps: float = 1e-12, vectors: bool = False):
    """Generalized Hermitian eigenproblem H c = E M c (FP64, liblemc)."""
    lib = _lib.load()
    D = H.shape[0]
    Hb = np.ascontiguousarray(H, dtype=np.complex128).view(np.float64)
    Mb = np.ascontiguousarray(M, dtype=np.complex128).view(np.float64)
    ev = np.zeros(D)
    vec = np.zeros(2 * D * D) if vectors else None
    rank = C.c_int()
    check(lib.lemc_geneig(D, dptr(Hb.ravel()), dptr(Mb.ravel()), eps, dptr(ev),
                          dptr(vec) if vectors else None, C.byref(rank)), "lemc_geneig")
    if vectors:
        return ev, _cplx(vec, D), rank.value
    return ev


def geneig_sweep(S, H2, H4, omegas, kappas, eps: float = 1e-12):
    """Generalized spectra of one sector for many (omega, kappa), FP64 on the GPU.

    Returns (evals [n, D] ascending, NaN beyond the kept rank; rank)."""
    lib = _lib.load()
    D = S.shape[0]
    om = np.ascontiguousarray(omegas, dtype=np.float64)
    ka = np.ascontiguousarray(kappas, dtype=np.float64)
    assert om.shape == ka.shape and om.ndim == 1
    buf = [np.ascontiguousarray(X, dtype=np.complex128).view(np.float64).ravel() for X in (S, H2, H4)]
    ev = np.zeros(len(om) * D)
    rank = C.c_int()
    check(lib.lemc_geneig_sweep(D, dptr(buf[0]), dptr(buf[1]), dptr(buf[2]), dptr(om), dptr(ka),
                                len(om), eps, dptr(ev), C.byref(rank)), "lemc_geneig_sweep")
    return ev.reshape(len(om), D), rank.value


def jackknife_spectrum(S_bins, H2_bins, H4_bins, omega, kappa, eps: float = 1e-12):
    """Leave-one-bin-out jackknife of one sector's spectrum from per-bin raw Gram
    sums ([B, D, D] complex each): (evals, evals_err, M_err, H_err)."""
    lib = _lib.load()
    B, D = S_bins.shape[0], S_bins.shape[1]
    a = [np.ascontiguousarray(X, dtype=np.complex128).view(np.float64).ravel()
         for X in (S_bins, H2_bins, H4_bins)]
    ev, er = np.zeros(D), np.zeros(D)
    me, he = np.zeros(D * D), np.zeros(D * D)
    check(lib.lemc_jackknife_spectrum(D, B, dptr(a[0]), dptr(a[1]), dptr(a[2]), omega, kappa, eps,
                                      dptr(ev), dptr(er), dptr(me), dptr(he)),
          "lemc_jackknife_spectrum")
    return ev, er, me.reshape(D, D), he.reshape(D, D)


def dsf_weights(H, M, Vc, Vs, eps: float = 1e-12):
    """Edge dynamic structure factor (energies, weights) of the normalised
    {0, dL} matrices (row 0 = Laughlin state), liblemc's lemc_dsf_weights."""
    lib = _lib.load()
    D = H.shape[0]
    a = [np.ascontiguousarray(X, dtype=np.complex128).view(np.float64).ravel() for X in (H, M, Vc, Vs)]
    e, w = np.zeros(D - 1), np.zeros(D - 1)
    n = C.c_int()
    check(lib.lemc_dsf_weights(D, dptr(a[0]), dptr(a[1]), dptr(a[2]), dptr(a[3]), eps, dptr(e),
                               dptr(w), C.byref(n)), "lemc_dsf_weights")
    return e[: n.value], w[: n.value]


def _herm(X):
    return 0.5 * (X + X.conj().T)


def dsf_compute(particles, inverse_filling, dL, n_walkers, burn_in, sweeps, omega, kappa,
                step_sigma=0.3, seed=42, guide=_lib.GUIDE_LAUGHLIN, gram_mode=_lib.GRAM_FP64):
    """Edge DSF of sector dL, as edgeMC::dsf_compute (em_dsf.cu:233-260): one
    context over the sectors {0, dL} with the angular probe dL; normalised H, M
    and the cos / sin(dL theta) excitation matrices, Hermitised, then
    dsf_weights.  Returns (energies, weights, H, M, Vc, Vs)."""
    smp = Sampler(SamplerConfig(particles, inverse_filling, n_walkers, step_sigma=step_sigma, seed=seed,
                                guide=guide, gram_mode=gram_mode), [0, dL], probes=[dL])
    try:
        smp.init_walkers()
        smp.run(burn_in, measure=False)
        smp.run(sweeps, measure=True)
        D = smp.total_dim
        d0 = smp.dims[0]
        M = np.zeros((D, D), complex)
        H = np.zeros((D, D), complex)
        Vc = np.zeros((D, D), complex)
        Vs = np.zeros((D, D), complex)
        if guide == _lib.GUIDE_ROW:
            fg, gg, fh, n, fc, fs, _ = smp.rows(omega, kappa, extra=True)
            sq = np.sqrt(gg)
            sec = np.array([0] * d0 + [1] * (D - d0))
            same = sec[:, None] == sec[None, :]
            M[same], H[same] = (fg / sq)[same], (fh / sq)[same]
            Vc[~same], Vs[~same] = (fc / sq)[~same], (fs / sq)[~same]
        else:
            nrm = []
            first = 0
            for si, d in enumerate(smp.dims):
                S, H2, H4, _ = smp.gram(si)
                Mn, Hn = normalise(S, H2, H4, omega, kappa)
                M[first:first + d, first:first + d] = Mn
                H[first:first + d, first:first + d] = Hn
                nrm.extend(np.sqrt(np.real(np.diag(S))))
                first += d
            nrm = np.array(nrm)
            for sa, sb in ((0, 1), (1, 0)):
                _, cc, cs = smp.cross(sa, sb)
                fa, fb = (0, d0) if sa == 0 else (d0, 0)
                da, db = smp.dims[sa], smp.dims[sb]
                den = np.outer(nrm[fa:fa + da], nrm[fb:fb + db])
                Vc[fa:fa + da, fb:fb + db] = cc / den
                Vs[fa:fa + da, fb:fb + db] = cs / den
        H, M, Vc, Vs = _herm(H), _herm(M), _herm(Vc), _herm(Vs)
        e, w = dsf_weights(H, M, Vc, Vs)
        return e, w, H, M, Vc, Vs
    finally:
        smp.close()


def normalise(S, H2=None, H4=None, omega=0.0, kappa=0.0):
    """Reference normalisation M = S/sqrt(S_aa S_bb), H = (w H2 + k H4)/sqrt(..), Hermitised."""
    lib = _lib.load()
    D = S.shape[0]
    f = lambda X: None if X is None else dptr(np.ascontiguousarray(X, dtype=np.complex128).view(np.float64).ravel())
    keep = [np.ascontiguousarray(X, dtype=np.complex128) for X in (S, H2, H4) if X is not None]
    Mo = np.zeros(2 * D * D)
    Ho = np.zeros(2 * D * D)
    check(lib.lemc_normalise(D, f(S), f(H2), f(H4), omega, kappa, dptr(Mo), dptr(Ho)), "lemc_normalise")
    del keep
    return _cplx(Mo, D), _cplx(Ho, D)


def evolve(M, H, U, rho, profile, end_time, save_step):
    """FP64 edge-basis time evolution; returns (times, <rho_l>(t) [n_save, L], norms)."""
    lib = _lib.load()
    D = M.shape[0]
    rho = [np.ascontiguousarray(r, dtype=np.complex128) for r in rho]
    L = len(rho)
    rb = np.ascontiguousarray(np.stack(rho) if L else np.zeros((1, D, D), complex)).view(np.float64).ravel()
    ns = int(math.ceil(end_time / save_step))
    out = np.zeros(2 * ns * max(L, 1))
    norms = np.zeros(ns)
    n_save = C.c_int()
    cb = _lib.PROFILE_FN(lambda t, u: float(profile(t)))
    a = [np.ascontiguousarray(X, dtype=np.complex128).view(np.float64).ravel() for X in (M, H, U)]
    check(lib.lemc_evolve(D, dptr(a[0]), dptr(a[1]), dptr(a[2]), L, dptr(rb), cb, None,
                          end_time, save_step, dptr(out), dptr(norms), C.byref(n_save)), "lemc_evolve")
    times = np.arange(ns) * save_step
    return times, out.view(np.complex128).reshape(ns, max(L, 1))[:, :L], norms


def evolve_device(M, H, U, rho, profile, end_time, save_step, substeps=4, eps=1e-12):
    """Fixed-step FP64 GPU evolution in the S-orthonormal basis; returns
    (times, <rho_l>(t) [n_save, L], norms, rank)."""
    lib = _lib.load()
    D = M.shape[0]
    rho = [np.ascontiguousarray(r, dtype=np.complex128) for r in rho]
    L = len(rho)
    rb = np.ascontiguousarray(np.stack(rho) if L else np.zeros((1, D, D), complex)).view(np.float64).ravel()
    ns = int(math.ceil(end_time / save_step))
    out = np.zeros(2 * ns * max(L, 1))
    norms = np.zeros(ns)
    n_save, rank = C.c_int(), C.c_int()
    cb = _lib.PROFILE_FN(lambda t, u: float(profile(t)))
    a = [np.ascontiguousarray(X, dtype=np.complex128).view(np.float64).ravel() for X in (M, H, U)]
    check(lib.lemc_evolve_device(D, dptr(a[0]), dptr(a[1]), dptr(a[2]), L, dptr(rb), cb, None,
                                 end_time, save_step, substeps, eps, dptr(out), dptr(norms),
                                 C.byref(n_save), C.byref(rank)), "lemc_evolve_device")
    times = np.arange(ns) * save_step
    return times, out.view(np.complex128).reshape(ns, max(L, 1))[:, :L], norms, rank.value


def occupation(particles, inverse_filling, dL, l_cutoff, n_walkers, sweeps, burn_in=200,
               step_sigma=0.3, seed=42):
    """Occupation averages for every (L, R) row pair of sector dL: complex [D, D, l_cutoff]."""
    lib = _lib.load()
    rows, _, _ = partitions(particles, [dL])
    D = len(rows)
    cfg = _lib.OccConfig(particles, inverse_filling, dL, l_cutoff, n_walkers, step_sigma, seed,
                         burn_in, sweeps)
    out = np.zeros(2 * D * D * l_cutoff)
    acc = C.c_double()
    check(lib.lemc_occupation(C.byref(cfg), dptr(out), C.byref(acc)), "lemc_occupation")
    return out.view(np.complex128).reshape(D, D, l_cutoff), acc.value


def tau_sokal(x, c: float = 5.0) -> float:
    """Sokal windowed integrated autocorrelation time of a series (NaN when the
    series is too short for a self-consistent window)."""
    a = np.ascontiguousarray(x, dtype=np.float64)
    t = C.c_double()
    check(_lib.load().lemc_tau_sokal(dptr(a), len(a), c, C.byref(t)), "lemc_tau_sokal")
    return t.value


def tau_binning(x, min_bins: int = 16):
    """Binning analysis of a series: (tau, tau_err, error of the mean, converged)."""
    a = np.ascontiguousarray(x, dtype=np.float64)
    t, te, em, cv = C.c_double(), C.c_double(), C.c_double(), C.c_int()
    check(_lib.load().lemc_tau_binning(dptr(a), len(a), min_bins, C.byref(t), C.byref(te),
                                       C.byref(em), C.byref(cv)), "lemc_tau_binning")
    return t.value, te.value, em.value, bool(cv.value)


def series_tau(series: np.ndarray):
    """tau_int of p_1..p_4 from a walker-mean series [T, 8] (Re/Im per k): per k
    the mean of the Re and Im estimates, Sokal and binning; the max over k."""
    sok, binn, conv = [], [], True
    for k in range(4):
        s = [tau_sokal(series[:, 2 * k + c]) for c in range(2)]
        b = [tau_binning(series[:, 2 * k + c]) for c in range(2)]
        sok.append(0.5 * (s[0] + s[1]))
        binn.append(0.5 * (b[0][0] + b[1][0]))
        conv = conv and b[0][3] and b[1][3]
    return {"sokal": float(max(sok)), "sokal_each": [float(v) for v in sok],
            "binning": float(max(binn)), "binning_each": [float(v) for v in binn],
            "binning_plateau": bool(conv), "series_length": int(series.shape[0])}


def spectral_weights(occ, H, M, particles, eps: float = 1e-12):
    """Energy-resolved occupations of one sector (lemc_spectral_weights):
    (energies [D], weights [D, Lc]) with sum_l weights[j, l] = particles."""
    lib = _lib.load()
    D, Lc = occ.shape[0], occ.shape[2]
    o = np.ascontiguousarray(occ, dtype=np.complex128).view(np.float64).ravel()
    h = np.ascontiguousarray(H, dtype=np.complex128).view(np.float64).ravel()
    m = np.ascontiguousarray(M, dtype=np.complex128).view(np.float64).ravel()
    e, w = np.zeros(D), np.zeros(D * Lc)
    n = C.c_int()
    check(lib.lemc_spectral_weights(D, Lc, dptr(o), dptr(h), dptr(m), particles, eps, dptr(e),
                                    dptr(w), C.byref(n)), "lemc_spectral_weights")
    return e, w.reshape(D, Lc)


def spectral_function(particles, inverse_filling, dL, omega, kappa, n_walkers=8192, burn_in=500,
                      sweeps=2000, l_cutoff=None, step_sigma=0.3, seed=42):
    """Edge spectral function of sector dL: the normalised M, H of the sector
    (shared-guide sampler) and its occupation matrices (two-state walker),
    combined by spectral_weights.  Returns (energies, weights [D, l_cutoff])."""
    Lc = l_cutoff or inverse_filling * (particles - 1) + 15
    smp = Sampler(SamplerConfig(particles, inverse_filling, n_walkers, step_sigma=step_sigma, seed=seed),
                  [dL])
    try:
        smp.init_walkers()
        smp.run(burn_in, measure=False)
        smp.run(sweeps, measure=True)
        S, H2, H4, _ = smp.gram(0)
    finally:
        smp.close()
    M, H = normalise(S, H2, H4, omega, kappa)
    occ, _ = occupation(particles, inverse_filling, dL, Lc, n_walkers, sweeps, burn_in=burn_in,
                        step_sigma=step_sigma, seed=seed + 1)
    return spectral_weights(occ, H, M, particles)


@dataclass
class SamplerConfig:
    particles: int
    inverse_filling: int
    n_walkers: int
    step_sigma: float = 0.3
    seed: int = 42
    lanes_per_walker: int = 0
    guide: int = _lib.GUIDE_LAUGHLIN
    radius_scale: float = 0.0
    init_radius: float = 0.0
    gram_mode: int = _lib.GRAM_FP64
    flush_every: int = 0
    graph_batch: int = 0
    profile: bool = False

    def to_c(self) -> _lib.Config:
        return _lib.Config(self.particles, self.inverse_filling, self.n_walkers,
                           self.lanes_per_walker, self.step_sigma, self.guide, self.seed,
                           self.radius_scale, self.init_radius, self.gram_mode,
                           self.graph_batch, self.flush_every, 1 if self.profile else 0)


class Sampler:
    """One sampling context on the current CUDA device (wraps lemc_ctx)."""

    def __init__(self, cfg: SamplerConfig, sectors, guide_rows=None, probes=None):
        self.lib = _lib.load()
        self.cfg = cfg
        self._h = C.c_void_p()
        c = cfg.to_c()
        check(self.lib.lemc_create(C.byref(c), C.byref(self._h)), "lemc_create")
        if probes:
            pr = np.ascontiguousarray(probes, dtype=np.int32)
            check(self.lib.lemc_set_probes(self._h, i32ptr(pr), len(pr)), "lemc_set_probes")
        self.sectors = list(sectors)
        sec = np.ascontiguousarray(self.sectors, dtype=np.int32)
        check(self.lib.lemc_set_sectors(self._h, i32ptr(sec), len(sec)), "lemc_set_sectors")
        if guide_rows is not None:
            gr = np.ascontiguousarray(guide_rows, dtype=np.int32)
            check(self.lib.lemc_set_guide_rows(self._h, i32ptr(gr), len(gr)), "lemc_set_guide_rows")
        self.dims = []
        for s in range(len(self.sectors)):
            d = C.c_int()
            check(self.lib.lemc_sector_dim(self._h, s, C.byref(d)), "lemc_sector_dim")
            self.dims.append(d.value)
        d = C.c_int()
        check(self.lib.lemc_total_dim(self._h, C.byref(d)), "lemc_total_dim")
        self.total_dim = d.value

    def close(self):
        if self._h:
            self.lib.lemc_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_walkers(self, xy: np.ndarray | None = None):
        if xy is None:
            check(self.lib.lemc_init_walkers(self._h, None), "lemc_init_walkers")
        else:
            a = np.ascontiguousarray(xy, dtype=np.float32)
            check(self.lib.lemc_init_walkers(self._h, fptr(a.ravel())), "lemc_init_walkers")

    def run(self, n_sweeps: int, measure: bool = True):
        check(self.lib.lemc_run(self._h, int(n_sweeps), 1 if measure else 0), "lemc_run")

    def run_hooked(self, n_sweeps: int, hook):
        """Measured sweeps; hook(dev_xy, dev_user_plane, W, N, stream) fills U per walker."""
        def _cb(user, xy, up, W, N, stream):
            try:
                return int(hook(xy, up, W, N, stream) or 0)
            except Exception:  # surface Python errors as an argument error
                return -1
        self._hook = _lib.STEP_HOOK(_cb)
        check(self.lib.lemc_run_hooked(self._h, int(n_sweeps), self._hook, None), "lemc_run_hooked")

    def close_bin(self):
        """End the current bin of measurements (jackknife error bars)."""
        check(self.lib.lemc_close_bin(self._h), "lemc_close_bin")

    def n_bins(self) -> int:
        n = C.c_int()
        check(self.lib.lemc_n_bins(self._h, C.byref(n)), "lemc_n_bins")
        return n.value

    def gram_bin(self, bin_index: int, sector_index: int):
        D = self.dims[sector_index]
        bufs = [np.zeros(2 * D * D) for _ in range(3)]
        n = C.c_double()
        check(self.lib.lemc_read_gram_bin(self._h, bin_index, sector_index,
                                          *[dptr(b) for b in bufs], C.byref(n)), "lemc_read_gram_bin")
        return tuple(_cplx(b, D) for b in bufs) + (n.value,)

    def jackknife(self, sector_index: int, omega: float, kappa: float, eps: float = 1e-12):
        """Spectrum of one sector with jackknife errors over the closed bins:
        (evals, evals_err, M_err, H_err)."""
        bins = [self.gram_bin(b, sector_index) for b in range(self.n_bins())]
        S, H2, H4 = (np.array([b[i] for b in bins]) for i in range(3))
        return jackknife_spectrum(S, H2, H4, omega, kappa, eps)

    def set_step(self, sigma: float):
        check(self.lib.lemc_set_step(self._h, float(sigma)), "lemc_set_step")

    def tune_step(self, target: float = 0.5, tol: float = 0.01, moves: int = 100):
        """Tune the Gaussian step on the live chain; returns (sigma, acceptance)."""
        sg, acc = C.c_float(), C.c_double()
        check(self.lib.lemc_tune_step(self._h, target, tol, moves, C.byref(sg), C.byref(acc)),
              "lemc_tune_step")
        return sg.value, acc.value

    def reset(self):
        check(self.lib.lemc_reset_accumulators(self._h), "lemc_reset_accumulators")

    def lanes_per_walker(self) -> int:
        g = C.c_int()
        check(self.lib.lemc_lanes_per_walker(self._h, C.byref(g)), "lemc_lanes_per_walker")
        return g.value

    def gram_splits(self) -> int:
        g = C.c_int()
        check(self.lib.lemc_gram_splits(self._h, C.byref(g)), "lemc_gram_splits")
        return g.value

    def stream(self) -> int:
        h = C.c_void_p()
        check(self.lib.lemc_stream(self._h, C.byref(h)), "lemc_stream")
        return h.value or 0

    def synchronize(self):
        check(self.lib.lemc_synchronize(self._h), "lemc_synchronize")

    def gram(self, sector_index: int):
        D = self.dims[sector_index]
        bufs = [np.zeros(2 * D * D) for _ in range(3)]
        n = C.c_double()
        check(self.lib.lemc_read_gram(self._h, sector_index, *[dptr(b) for b in bufs], C.byref(n)),
              "lemc_read_gram")
        return tuple(_cplx(b, D) for b in bufs) + (n.value,)

    def cross(self, sa: int, sb: int):
        """(Cuser, Ccos, Csin) raw cross sums between selected sectors sa != sb."""
        Da, Db = self.dims[sa], self.dims[sb]
        bufs = [np.zeros(2 * Da * Db) for _ in range(3)]
        check(self.lib.lemc_read_cross(self._h, sa, sb, *[dptr(b) for b in bufs]), "lemc_read_cross")
        return tuple(b.view(np.complex128).reshape(Da, Db) for b in bufs)

    def rows(self, omega: float, kappa: float, extra: bool = False):
        """Reference-estimator row averages (fg, gg, fh, n[, fcos, fsin, fuser])."""
        D = self.total_dim
        fg, gg, fh = np.zeros(2 * D * D), np.zeros(D * D), np.zeros(2 * D * D)
        fc, fs, fu = np.zeros(2 * D * D), np.zeros(2 * D * D), np.zeros(2 * D * D)
        n = np.zeros(D)
        check(self.lib.lemc_read_rows(self._h, omega, kappa, dptr(fg), dptr(gg), dptr(fh), dptr(fc),
                                      dptr(fs), dptr(fu), dptr(n)), "lemc_read_rows")
        if extra:
            return _cplx(fg, D), gg.reshape(D, D), _cplx(fh, D), n, _cplx(fc, D), _cplx(fs, D), _cplx(fu, D)
        return _cplx(fg, D), gg.reshape(D, D), _cplx(fh, D), n

    def stats(self) -> _lib.Stats:
        st = _lib.Stats()
        check(self.lib.lemc_read_stats(self._h, C.byref(st)), "lemc_read_stats")
        return st

    def set_proposal(self, proposal):
        """Use a LearnedProposal for the sweeps (None: the plain Gaussian step)."""
        check(self.lib.lemc_set_proposal(self._h, proposal._h if proposal is not None else None),
              "lemc_set_proposal")
        self._proposal = proposal  # keep the weights alive while in use

    def copy_positions_device(self, dst_ptr: int):
        """Device-to-device copy of the walker positions ([W][N] float2)."""
        check(self.lib.lemc_copy_positions_device(self._h, C.c_void_p(dst_ptr)),
              "lemc_copy_positions_device")

    def positions(self) -> np.ndarray:
        W, N = self.cfg.n_walkers, self.cfg.particles
        out = np.zeros(W * N * 2, dtype=np.float32)
        check(self.lib.lemc_read_positions(self._h, fptr(out)), "lemc_read_positions")
        return out.reshape(W, N, 2)

    def series(self) -> np.ndarray:
        n = C.c_int()
        check(self.lib.lemc_read_series(self._h, None, 0, C.byref(n)), "lemc_read_series")
        out = np.zeros(8 * max(1, n.value))
        check(self.lib.lemc_read_series(self._h, dptr(out), n.value, C.byref(n)), "lemc_read_series")
        return out[: 8 * n.value].reshape(n.value, 8)
