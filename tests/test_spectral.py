"""Energy-resolved edge occupations (lemc_spectral_weights, host FP64) against a
numpy/scipy restatement, and the sum rule sum_l w_j(l) = N."""
import numpy as np
import scipy.linalg as sl


def test_spectral_weights_match_numpy(lemc):
    g = np.random.default_rng(11)
    D, Lc, N = 4, 7, 5
    X = g.normal(size=(D, D)) + 1j * g.normal(size=(D, D))
    M = X @ X.conj().T + D * np.eye(D)
    d = np.sqrt(np.real(np.diag(M)))
    M = M / np.outer(d, d)
    Y = g.normal(size=(D, D)) + 1j * g.normal(size=(D, D))
    H = 0.5 * (Y + Y.conj().T) + 5 * np.eye(D)
    occ = g.random((D, D, Lc)) + 0.2 * 1j * g.normal(size=(D, D, Lc))
    e, w = lemc.spectral_weights(occ, H, M, N)
    n = occ / occ.sum(-1, keepdims=True) * N * M[:, :, None]
    n = 0.5 * (n + np.conj(np.transpose(n, (1, 0, 2))))
    er, c = sl.eigh(H, M)
    wr = np.einsum("aj,abl,bj->jl", c.conj(), n, c).real
    assert np.allclose(e, er, rtol=1e-10)
    assert np.allclose(w, wr, rtol=1e-8, atol=1e-10)
    assert np.allclose(w.sum(1), N)
