"""Closed-form known answers for the nu = 1 (m = 1) Laughlin state.

For m = 1, Psi_1 is the Slater determinant of the orbitals z^0..z^{N-1}.
Frobenius: p_lambda = sum_mu chi^mu(lambda) s_mu, and s_mu Psi_1 is the Slater
determinant with orbitals n_j = mu_j + N - j, orthogonal with norms
prod_j 2 pi 2^{n_j} n_j!  (||z^n e^{-|z|^2/4}||^2 = 2 pi 2^n n!).  Hence
  <p_l Psi|p_n Psi>/<Psi|Psi> = R^{-2|l|} sum_mu chi^mu(l) chi^mu(n) prod_j 2^{mu_j}(mu_j+N-j)!/(N-j)!
and, for V = w r^2 + k r^4 (diagonal in the orbitals: <r^2>_l = 2(l+1),
<r^4>_l = 4(l+1)(l+2)), the generalized eigenvalues are
  E_mu = sum_j [2 w (n_j+1) + 4 k (n_j+1)(n_j+2)].
Characters by the Murnaghan-Nakayama rule on beta-sets (rim hooks).
"""
from functools import lru_cache
from math import factorial

import numpy as np


def partitions_desc(n, maxpart=None):
    if maxpart is None:
        maxpart = n
    if n == 0:
        yield ()
        return
    for k in range(min(n, maxpart), 0, -1):
        for rest in partitions_desc(n - k, k):
            yield (k,) + rest


@lru_cache(maxsize=None)
def character(mu, lam):
    """chi^mu(lam), mu and lam descending tuples of the same size."""
    if sum(mu) == 0:
        return 1
    r = lam[0]
    rest = lam[1:]
    L = len(mu)
    beta = [mu[j] + (L - 1 - j) for j in range(L)]
    bset = set(beta)
    total = 0
    for b in beta:
        nb = b - r
        if nb < 0 or nb in bset:
            continue
        sign = (-1) ** sum(1 for c in beta if nb < c < b)
        newb = sorted([c for c in beta if c != b] + [nb], reverse=True)
        Ln = len(newb)
        newmu = tuple(x for x in (newb[j] - (Ln - 1 - j) for j in range(Ln)) if x > 0)
        total += sign * character(newmu, rest)
    return total


def row_to_desc(pairs):
    parts = []
    for k, m in pairs:
        parts += [k] * m
    return tuple(sorted(parts, reverse=True))


def gram_m1(N, rows, R=1.0):
    """Exact normalised-by-<Psi|Psi> Gram matrix of the rows (all same dL)."""
    lams = [row_to_desc(pr) for _, pr in rows]
    n = sum(lams[0])
    mus = [mu for mu in partitions_desc(n) if len(mu) <= N]
    w = []
    for mu in mus:
        v = 1.0
        for j, mj in enumerate(mu, start=1):
            v *= 2.0 ** mj * factorial(mj + N - j) / factorial(N - j)
        w.append(v)
    X = np.array([[character(mu, lam) for mu in mus] for lam in lams], dtype=float)
    return (X * np.array(w)) @ X.T / R ** (2 * n)


def gram_m1_weighted(N, rows, R=1.0):
    """Exact (sum r^2)- and (sum r^4)-weighted Gram matrices of the rows at nu = 1.

    The Schur states s_mu Psi_1 are Slater determinants of the orbitals
    n_j = mu_j + N - j (j = 1..N), and sum_i |z_i|^2, sum_i |z_i|^4 are diagonal
    in them with values sum_j 2(n_j+1) and sum_j 4(n_j+1)(n_j+2); the weighted
    Gram matrices are gram_m1 with those factors inside the character sum."""
    lams = [row_to_desc(pr) for _, pr in rows]
    n = sum(lams[0])
    mus = [mu for mu in partitions_desc(n) if len(mu) <= N]
    w, w2, w4 = [], [], []
    for mu in mus:
        v = 1.0
        for j, mj in enumerate(mu, start=1):
            v *= 2.0 ** mj * factorial(mj + N - j) / factorial(N - j)
        ns = [(mu[j] if j < len(mu) else 0) + N - 1 - j for j in range(N)]
        w.append(v)
        w2.append(v * sum(2.0 * (x + 1) for x in ns))
        w4.append(v * sum(4.0 * (x + 1) * (x + 2) for x in ns))
    X = np.array([[character(mu, lam) for mu in mus] for lam in lams], dtype=float)
    sc = R ** (2 * n)
    return (X * np.array(w2)) @ X.T / sc, (X * np.array(w4)) @ X.T / sc


def spectrum_m1(N, dL, omega, kappa):
    out = []
    for mu in partitions_desc(dL):
        if len(mu) > N:
            continue
        ns = [(mu[j] if j < len(mu) else 0) + N - 1 - j for j in range(N)]
        out.append(sum(2 * omega * (x + 1) + 4 * kappa * (x + 1) * (x + 2) for x in ns))
    return np.sort(np.array(out))


def harmonic_level(N, m, dL):
    """Every state of sector dL has <sum r^2> = 2(L_tot + N), L_tot = m N(N-1)/2 + dL."""
    return 2.0 * (m * N * (N - 1) / 2 + dL + N)
