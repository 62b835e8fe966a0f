"""FP64 dense tail of liblemc (host code): eigensolver, normalisation, evolution."""
import numpy as np
import pytest
import scipy.integrate as si
import scipy.linalg as sl


def _herm(rng, D):
    A = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
    return A + A.conj().T


@pytest.mark.parametrize("D", [1, 2, 7, 30, 90])
def test_geneig_matches_scipy(lemc, D):
    rng = np.random.default_rng(D)
    H = _herm(rng, D)
    B = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
    M = B @ B.conj().T + 0.5 * D * np.eye(D)
    ev = lemc.geneig(H, M)
    ref = sl.eigh(H, M, eigvals_only=True)
    assert np.max(np.abs(ev - ref)) < 1e-9 * max(1, np.max(np.abs(ref)))
    ev2, V, rank = lemc.geneig(H, M, vectors=True)
    assert rank == D
    assert np.max(np.abs(H @ V - M @ V * ev2)) < 1e-8 * max(1, np.max(np.abs(ref)))
    assert np.max(np.abs(V.conj().T @ M @ V - np.eye(D))) < 1e-9


def test_geneig_degenerate_vectors(lemc):
    # harmonic-like case: H = c M, fully degenerate spectrum
    rng = np.random.default_rng(3)
    D = 12
    B = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
    M = B @ B.conj().T + D * np.eye(D)
    ev, V, rank = lemc.geneig(3.5 * M, M, vectors=True)
    assert np.allclose(ev, 3.5, atol=1e-10)
    assert np.max(np.abs(V.conj().T @ M @ V - np.eye(D))) < 1e-9


def test_geneig_singular_metric_floor(lemc):
    rng = np.random.default_rng(5)
    D, r = 10, 6
    B = rng.normal(size=(D, r)) + 1j * rng.normal(size=(D, r))
    M = B @ B.conj().T  # rank 6
    H = _herm(rng, D)
    ev, V, rank = lemc.geneig(H, M, eps=1e-10, vectors=True)
    assert rank == r
    assert np.all(np.isnan(ev[r:]))
    # compare with the projected problem
    w, U = np.linalg.eigh(M)
    X = U[:, w > 1e-10 * w.max()] / np.sqrt(w[w > 1e-10 * w.max()])
    ref = np.linalg.eigvalsh(X.conj().T @ H @ X)
    assert np.max(np.abs(np.sort(ev[:r]) - ref)) < 1e-8


def test_normalise_reference_convention(lemc):
    rng = np.random.default_rng(9)
    D = 6
    B = rng.normal(size=(D, 40)) + 1j * rng.normal(size=(D, 40))
    S = B.conj() @ B.T
    H2 = (B.conj() * rng.uniform(1, 2, 40)) @ B.T
    H4 = (B.conj() * rng.uniform(1, 4, 40)) @ B.T
    M, H = lemc.normalise(S, H2, H4, 0.3, 0.05)
    d = np.sqrt(np.diag(S).real)
    Mr = S / np.outer(d, d)
    Hr = (0.3 * H2 + 0.05 * H4) / np.outer(d, d)
    assert np.allclose(M, 0.5 * (Mr + Mr.conj().T), atol=1e-13)
    assert np.allclose(H, 0.5 * (Hr + Hr.conj().T), atol=1e-13)


def test_evolve_matches_scipy(lemc):
    rng = np.random.default_rng(11)
    D = 5
    B = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
    M = B @ B.conj().T + D * np.eye(D)
    H = _herm(rng, D) * 0.2 + M * 0.5
    U = _herm(rng, D) * 0.1
    rho = [_herm(rng, D), _herm(rng, D) + 1j * 0.0]
    prof = lambda t: 0.3 * np.exp(-((t - 2.0) ** 2) / 2.0)
    T, dt = 6.0, 0.5
    times, out, norms = lemc.evolve(M, H, U, rho, prof, T, dt)
    A = np.linalg.solve(M, H)
    Bm = np.linalg.solve(M, U)
    f = lambda t, c: -1j * (A + prof(t) * Bm) @ c
    c0 = np.zeros(D, complex)
    c0[0] = 1
    sol = si.solve_ivp(f, (0, times[-1]), c0, t_eval=times, rtol=1e-11, atol=1e-13, method="DOP853")
    for s, t in enumerate(times):
        c = sol.y[:, s]
        for l, r in enumerate(rho):
            assert abs(out[s, l] - c.conj() @ r @ c) < 1e-6 * (1 + abs(c.conj() @ r @ c))
        assert abs(norms[s] - (c.conj() @ M @ c).real) < 1e-6 * norms[0]


def test_geneig_m1_closed_form_spectrum(lemc):
    """Host solver on the exact nu = 1 Gram matrices: E_mu in closed form."""
    import kat
    N, dL = 6, 5
    rows = lemc.partitions(N, [dL])[0]
    S = kat.gram_m1(N, rows).astype(complex)
    H2, H4 = kat.gram_m1_weighted(N, rows)
    M, H = lemc.normalise(S, H2.astype(complex), H4.astype(complex), 1e-2, 1e-4)
    np.testing.assert_allclose(lemc.geneig(H, M), kat.spectrum_m1(N, dL, 1e-2, 1e-4), rtol=1e-9)
