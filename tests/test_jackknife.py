"""Jackknife error bars over bins (lemc_jackknife_spectrum, host FP64) against
a numpy/scipy restatement, on synthetic per-bin Gram sums: bins of samples of
a correlated complex basis vector v with weights r2 > 0, r4 > 0."""
import numpy as np
import scipy.linalg as sl


def _bins(rng, B, D, per_bin):
    A = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
    S, H2, H4 = [], [], []
    for _ in range(B):
        z = rng.normal(size=(per_bin, D)) + 1j * rng.normal(size=(per_bin, D))
        v = z @ A.T
        r2 = 1.0 + rng.random(per_bin)
        S.append(np.einsum("wa,wb->ab", v.conj(), v))
        H2.append(np.einsum("w,wa,wb->ab", r2, v.conj(), v))
        H4.append(np.einsum("w,wa,wb->ab", r2 ** 2, v.conj(), v))
    return np.array(S), np.array(H2), np.array(H4)


def _norm(S, H2, H4, om, ka):
    d = np.sqrt(np.real(np.diag(S)))
    n = np.outer(d, d)
    M, H = S / n, (om * H2 + ka * H4) / n
    return 0.5 * (M + M.conj().T), 0.5 * (H + H.conj().T)


def test_jackknife_matches_numpy(lemc):
    rng = np.random.default_rng(3)
    B, D, om, ka = 12, 5, 0.7, 0.2
    S, H2, H4 = _bins(rng, B, D, 400)
    ev, er, me, he = lemc.jackknife_spectrum(S, H2, H4, om, ka)
    M, H = _norm(S.sum(0), H2.sum(0), H4.sum(0), om, ka)
    assert np.allclose(ev, sl.eigh(H, M, eigvals_only=True), rtol=1e-9)
    evb, Mb, Hb = [], [], []
    for b in range(B):
        Mx, Hx = _norm(S.sum(0) - S[b], H2.sum(0) - H2[b], H4.sum(0) - H4[b], om, ka)
        evb.append(sl.eigh(Hx, Mx, eigvals_only=True))
        Mb.append(Mx)
        Hb.append(Hx)
    f = (B - 1) / B
    evb, Mb, Hb = np.array(evb), np.array(Mb), np.array(Hb)
    assert np.allclose(er, np.sqrt(f * ((evb - evb.mean(0)) ** 2).sum(0)), rtol=1e-7)
    assert np.allclose(me, np.sqrt(f * (np.abs(Mb - Mb.mean(0)) ** 2).sum(0)), rtol=1e-7, atol=1e-15)
    assert np.allclose(he, np.sqrt(f * (np.abs(Hb - Hb.mean(0)) ** 2).sum(0)), rtol=1e-7, atol=1e-15)


def test_jackknife_error_tracks_spread(lemc):
    """The jackknife error of one run predicts the spread of independent runs."""
    rng = np.random.default_rng(4)
    B, D, om, ka = 16, 4, 1.0, 0.1
    runs, errs = [], []
    for _ in range(24):
        S, H2, H4 = _bins(rng, B, D, 200)
        ev, er, _, _ = lemc.jackknife_spectrum(S, H2, H4, om, ka)
        runs.append(ev)
        errs.append(er)
    spread = np.array(runs).std(0, ddof=1)
    ratio = np.mean(errs, 0) / spread
    assert np.all((ratio > 0.6) & (ratio < 1.6)), ratio
