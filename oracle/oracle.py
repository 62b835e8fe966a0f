"""ctypes wrapper of the C oracle (oracle/lemc_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker of the CUDA path and
never as the product.  Builds _build/liblemc_oracle.so with make on first use.
"""
from __future__ import annotations

import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liblemc_oracle.so"
MAXK = 24
MAXGP = 8

_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB.exists() or LIB.stat().st_mtime < (HERE / "lemc_oracle.c").stat().st_mtime:
            subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
        _lib = C.CDLL(str(LIB))
        _lib.orc_max_threads.restype = C.c_int
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def philox(ctr, key):
    lib = load()
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib.orc_philox(c, k, o)
    return list(o)


def partitions(N, sectors, max_rows=20000):
    """Basis rows: list of (dL, [(part, mult), ...]) in reference order."""
    lib = load()
    sec = np.ascontiguousarray(sectors, dtype=np.int32)
    dL = np.zeros(max_rows, np.int32)
    npairs = np.zeros(max_rows, np.int32)
    pairs = np.zeros(max_rows * 2 * MAXK, np.int32)
    n = lib.orc_partitions(C.c_int(N), _p(sec), C.c_int(len(sec)), _p(dL), _p(npairs), _p(pairs),
                           C.c_int(max_rows))
    if n < 0:
        raise ValueError("too many rows")
    rows = []
    for r in range(n):
        pr = [(int(pairs[r * 2 * MAXK + 2 * q]), int(pairs[r * 2 * MAXK + 2 * q + 1]))
              for q in range(npairs[r])]
        rows.append((int(dL[r]), pr))
    return rows


def _guide_arrays(rows):
    D = len(rows)
    gp = np.zeros(D * 2 * MAXGP, np.int32)
    gn = np.zeros(D, np.int32)
    for r, (_, pr) in enumerate(rows):
        gn[r] = len(pr)
        for q, (k, m) in enumerate(pr):
            gp[r * 2 * MAXGP + 2 * q] = k
            gp[r * 2 * MAXGP + 2 * q + 1] = m
    return gp, gn


def init_walkers(W, N, radius, seed):
    lib = load()
    pos = np.zeros((W, N, 2), np.float32)
    lib.orc_init(_p(pos), C.c_int(W), C.c_int(N), C.c_double(radius), C.c_uint64(seed))
    return pos


def sweep(pos, m, sigma, seed, sweep0, n_sweeps, R, rows=None, walker_row=None, accepted=None,
          nthreads=0, margins=None):
    """Advance positions in place (float32 [W, N, 2]); returns accepted counts.
    margins (float64 [W], optional) receives each walker's smallest
    |ln A - ln u| over its moves."""
    lib = load()
    W, N = pos.shape[0], pos.shape[1]
    acc = np.zeros(W, np.uint32) if accepted is None else accepted
    mg = None if margins is None else _p(margins)
    if rows is not None:
        gp, gn = _guide_arrays(rows)
        wr = np.ascontiguousarray(walker_row, dtype=np.int32)
        lib.orc_sweep_margin(_p(pos), C.c_int(W), C.c_int(N), C.c_int(m), C.c_double(sigma),
                             C.c_uint64(seed), C.c_uint32(sweep0), C.c_int(n_sweeps),
                             C.c_double(1.0 / R), _p(wr), _p(gp), _p(gn), _p(acc), mg,
                             C.c_int(nthreads))
    else:
        lib.orc_sweep_margin(_p(pos), C.c_int(W), C.c_int(N), C.c_int(m), C.c_double(sigma),
                             C.c_uint64(seed), C.c_uint32(sweep0), C.c_int(n_sweeps),
                             C.c_double(1.0 / R), None, None, None, _p(acc), mg, C.c_int(nthreads))
    return acc


def measure(pos, K, R, lprobe=0):
    """Records: (p [W, K] complex128, weights [W, 6])."""
    lib = load()
    W, N = pos.shape[0], pos.shape[1]
    rp = np.zeros((W, K, 2))
    rw = np.zeros((W, 6))
    lib.orc_measure(_p(np.ascontiguousarray(pos)), C.c_int(W), C.c_int(N), C.c_int(K),
                    C.c_double(1.0 / R), C.c_int(lprobe), _p(rp), _p(rw))
    return rp[..., 0] + 1j * rp[..., 1], rw


def basis_values(p, N, rows):
    """v[W, D] = prod p_k^mult (p_0 = N) for the rows."""
    W = p.shape[0]
    v = np.ones((W, len(rows)), complex)
    for b, (_, pr) in enumerate(rows):
        for k, m in pr:
            base = np.full(W, float(N), complex) if k == 0 else p[:, k - 1]
            v[:, b] *= base ** m
    return v


def _rows_arrays(rows):
    D = len(rows)
    np_ = np.array([len(pr) for _, pr in rows], np.int32)
    pairs = np.zeros(D * 2 * MAXK, np.int32)
    dl = np.array([d for d, _ in rows], np.int32)
    for r, (_, pr) in enumerate(rows):
        for q, (k, m) in enumerate(pr):
            pairs[r * 2 * MAXK + 2 * q] = k
            pairs[r * 2 * MAXK + 2 * q + 1] = m
    return np_, pairs, dl


def run_rows(N, m, W, sigma, seed, n_burn, n_meas, sectors, R=None, init_radius=None,
             nthreads=0):
    """Reference estimator (row guides).  Returns dict of raw sums and the
    walker-mean series of Re/Im p_1..p_4 per measurement."""
    lib = load()
    rows = partitions(N, sectors)
    D = len(rows)
    K = max(4, max(k for _, pr in rows for k, _ in pr))
    R = R or math.sqrt(2 * m * N)
    init_radius = init_radius or math.sqrt(2 * m * N)
    np_, pairs, dl = _rows_arrays(rows)
    fg = np.zeros(2 * D * D)
    gg = np.zeros(D * D)
    fh2 = np.zeros(2 * D * D)
    fh4 = np.zeros(2 * D * D)
    nrow = np.zeros(D)
    series = np.zeros(max(1, n_meas) * 8)
    lib.orc_run_rows(C.c_int(N), C.c_int(m), C.c_int(W), C.c_double(sigma), C.c_uint64(seed),
                     C.c_int(n_burn), C.c_int(n_meas), C.c_double(1.0 / R), C.c_double(init_radius),
                     C.c_int(D), _p(np_), _p(pairs), _p(dl), C.c_int(K), _p(fg), _p(gg), _p(fh2),
                     _p(fh4), _p(nrow), _p(series), C.c_int(nthreads))
    cz = lambda b: b.view(np.complex128).reshape(D, D)
    return {"rows": rows, "fg": cz(fg), "gg": gg.reshape(D, D), "fh2": cz(fh2), "fh4": cz(fh4),
            "n_row": nrow, "series": series[: 8 * n_meas].reshape(n_meas, 8)}


def run_gram(N, m, W, sigma, seed, n_burn, n_meas, sectors, R=None, init_radius=None, nthreads=0):
    """Shared Laughlin guide.  Returns (rows, S, H2, H4) raw sums (D x D, same-sector blocks)."""
    lib = load()
    rows = partitions(N, sectors)
    D = len(rows)
    K = max(4, max(k for _, pr in rows for k, _ in pr))
    R = R or math.sqrt(2 * m * N)
    init_radius = init_radius or math.sqrt(2 * m * N)
    np_, pairs, dl = _rows_arrays(rows)
    S = np.zeros(2 * D * D)
    H2 = np.zeros(2 * D * D)
    H4 = np.zeros(2 * D * D)
    series = np.zeros(max(1, n_meas) * 8)
    lib.orc_run_gram(C.c_int(N), C.c_int(m), C.c_int(W), C.c_double(sigma), C.c_uint64(seed),
                     C.c_int(n_burn), C.c_int(n_meas), C.c_double(1.0 / R), C.c_double(init_radius),
                     C.c_int(D), _p(np_), _p(pairs), _p(dl), C.c_int(K), _p(S), _p(H2), _p(H4),
                     _p(series), C.c_int(nthreads))
    cz = lambda b: b.view(np.complex128).reshape(D, D)
    return rows, cz(S), cz(H2), cz(H4)


def tau_int(series, c=5.0):
    """Sokal automatic-window integrated autocorrelation time of each column."""
    x = np.asarray(series, float)
    out = []
    for col in x.T:
        T = len(col)
        y = col - col.mean()
        c0 = np.dot(y, y) / T
        if T < 8 or c0 <= 0:
            out.append(float("nan"))
            continue
        tau = 0.5
        for t in range(1, T // 2):
            tau += np.dot(y[:-t], y[t:]) / T / c0
            if t >= c * tau:
                break
        out.append(tau)
    return np.array(out)


def reference_matrices(fg, gg, fh, n_row):
    """Reference normalisation of per-row averages: X(a,b) = <x>[a][b] / sqrt(<gg>[a][b])
    then (X + X^H)/2 (modules/edge_mc/em_spectrum.cu:318-335, :383-390)."""
    n = np.asarray(n_row, float)[:, None]
    fg, gg, fh = fg / n, gg / n, fh / n
    M = fg / np.sqrt(gg)
    H = fh / np.sqrt(gg)
    return 0.5 * (M + M.conj().T), 0.5 * (H + H.conj().T)


def occupation(N, m, W, sigma, seed, n_burn, n_meas, dL, rowL, rowR, Lc, nthreads=0):
    """Occupation averages of the pair (rowL, rowR) of sector dL: complex [Lc]."""
    lib = load()
    rows = partitions(N, [dL])

    def parts(r):
        pr = rows[r][1]
        k = np.zeros(MAXGP, np.int32)
        m_ = np.zeros(MAXGP, np.int32)
        for q, (kk, mm) in enumerate(pr):
            k[q] = kk
            m_[q] = mm if kk > 0 else 0
        return k, m_, len(pr)

    kL, rL, nL = parts(rowL)
    kR, rR, nR = parts(rowR)
    out = np.zeros(2 * Lc)
    lib.orc_occupation(C.c_int(N), C.c_int(m), C.c_int(W), C.c_double(sigma), C.c_uint64(seed),
                       C.c_int(n_burn), C.c_int(n_meas), _p(kL), _p(rL), C.c_int(nL), _p(kR),
                       _p(rR), C.c_int(nR), C.c_int(Lc), _p(out), C.c_int(nthreads))
    return out.view(np.complex128)
