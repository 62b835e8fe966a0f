"""lemc_dsf_weights (host FP64) against a numpy/scipy restatement of the
reference's extract_dsf_coefficients (generalized_eigenproblem.cpp:54-95)."""
import numpy as np
import scipy.linalg as sl


def _herm(X):
    return 0.5 * (X + X.conj().T)


def test_dsf_weights_match_scipy(lemc):
    g = np.random.default_rng(7)
    D = 8
    X = g.normal(size=(D, D)) + 1j * g.normal(size=(D, D))
    M = X @ X.conj().T + D * np.eye(D)
    d = np.sqrt(np.real(np.diag(M)))
    M = M / np.outer(d, d)
    H = _herm(g.normal(size=(D, D)) + 1j * g.normal(size=(D, D)))
    Vc = _herm(g.normal(size=(D, D)) + 1j * g.normal(size=(D, D)))
    Vs = _herm(g.normal(size=(D, D)) + 1j * g.normal(size=(D, D)))
    e, w = lemc.dsf_weights(H, M, Vc, Vs)
    er, vr = sl.eigh(H[1:, 1:], M[1:, 1:])
    v = (Vc - 1j * Vs)[0, 1:]
    wr = np.abs(v @ vr) ** 2
    assert np.allclose(e, er, rtol=1e-10, atol=1e-12)
    assert np.allclose(w, wr, rtol=1e-8, atol=1e-12)


def test_dsf_weights_closed_form(lemc):
    """With M = 1 on the dL block, the weights are |<v, e_j>|^2 of H's eigenvectors:
    their sum is |v|^2 (completeness)."""
    g = np.random.default_rng(8)
    D = 6
    H = np.diag(np.arange(D, dtype=float)).astype(complex)
    M = np.eye(D, dtype=complex)
    Vc = _herm(g.normal(size=(D, D)) + 0j)
    Vs = np.zeros((D, D), complex)
    e, w = lemc.dsf_weights(H, M, Vc, Vs)
    assert np.allclose(e, np.arange(1, D))
    assert np.isclose(w.sum(), np.sum(np.abs(Vc[0, 1:]) ** 2))
