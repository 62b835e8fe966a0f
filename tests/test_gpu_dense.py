"""FP64 GPU tail: lemc_geneig_sweep (kappa sweep of one sector, canonical
orthogonalisation on the device) against the host solver and a numpy
restatement of the same algorithm, through the C-ABI."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _hermitian(rng, D, scale=1.0):
    A = rng.standard_normal((D, D)) + 1j * rng.standard_normal((D, D))
    return scale * (A + A.conj().T) / 2


def _canonical(S, H2, H4, om, ka, eps):
    d = np.sqrt(np.real(np.diag(S)))
    nrm = np.outer(d, d)
    M = (S + S.conj().T) / 2 / nrm
    m, U = np.linalg.eigh(M)
    keep = m > eps * m.max()
    X = U[:, keep] / np.sqrt(m[keep])
    out = []
    for o, k in zip(om, ka):
        H = (o * (H2 + H2.conj().T) / 2 + k * (H4 + H4.conj().T) / 2) / nrm
        out.append(np.linalg.eigvalsh(X.conj().T @ H @ X))
    return np.array(out), int(keep.sum())


def test_sweep_matches_host_solver(lemc, cuda_ctx):
    rng = np.random.default_rng(3)
    D = 48
    B = rng.standard_normal((D, D)) + 1j * rng.standard_normal((D, D))
    S = B @ B.conj().T + D * np.eye(D)
    H2, H4 = _hermitian(rng, D), _hermitian(rng, D, 0.1)
    om = np.full(16, 2e-3)
    ka = np.logspace(-6, -4, 16)
    ev, rank = lemc.geneig_sweep(S, H2, H4, om, ka)
    assert rank == D
    for j in range(16):
        M, H = lemc.normalise(S, H2, H4, om[j], ka[j])
        ref = lemc.geneig(H, M)
        np.testing.assert_allclose(ev[j], ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())


def test_sweep_drops_null_directions_like_canonical_orthogonalisation(lemc, cuda_ctx):
    rng = np.random.default_rng(4)
    D, r = 40, 31
    B = rng.standard_normal((D, r)) + 1j * rng.standard_normal((D, r))
    S = B @ B.conj().T + 1e-14 * np.eye(D)      # numerically rank r
    H2, H4 = _hermitian(rng, D), _hermitian(rng, D, 0.1)
    om, ka = np.array([1e-2, 5e-3]), np.array([1e-4, 2e-5])
    ev, rank = lemc.geneig_sweep(S, H2, H4, om, ka, eps=1e-10)
    ref, rref = _canonical(S, H2, H4, om, ka, 1e-10)
    assert rank == rref == r
    assert np.all(np.isnan(ev[:, r:]))
    np.testing.assert_allclose(ev[:, :r], ref, rtol=1e-7, atol=1e-9 * np.abs(ref).max())


def test_sweep_m1_closed_form(lemc, cuda_ctx):
    """nu = 1: the Gram matrices of power-sum states are known exactly, and the
    generalized spectrum is E_mu = sum_j [2 omega (n_j+1) + 4 kappa (n_j+1)(n_j+2)]
    (known-answer test), here for 16 quartic strengths at once."""
    import kat
    N, dL = 6, 5
    rows = lemc.partitions(N, [dL])[0]
    S = kat.gram_m1(N, rows)
    H2, H4 = kat.gram_m1_weighted(N, rows)
    ka = np.logspace(-6, -4, 16)
    ev, rank = lemc.geneig_sweep(S, H2, H4, np.full(16, 1e-2), ka)
    assert rank == len(rows)
    for j, k in enumerate(ka):
        np.testing.assert_allclose(ev[j], kat.spectrum_m1(N, dL, 1e-2, k), rtol=1e-9)


def test_evolve_device_matches_host_integrator(lemc, cuda_ctx):
    """GPU fixed-step RK4 in the S-orthonormal basis against the host adaptive
    Cash-Karp integrator of M dC/dt = -i (H + f(t) U) C, C(0) = e_0."""
    rng = np.random.default_rng(6)
    D = 14
    B = rng.standard_normal((D, D)) + 1j * rng.standard_normal((D, D))
    M = B @ B.conj().T / D + np.eye(D)
    H = _hermitian(rng, D) + 40.0 * M          # large common energy: a global phase
    U = _hermitian(rng, D, 0.3)
    rho = [_hermitian(rng, D), rng.standard_normal((D, D)) + 1j * rng.standard_normal((D, D))]
    prof = lambda t: 0.05 * math.exp(-((t - 3.0) ** 2) / 2.0)
    t1, o1, n1 = lemc.evolve(M, H, U, rho, prof, 8.0, 0.1)
    t2, o2, n2, rank = lemc.evolve_device(M, H, U, rho, prof, 8.0, 0.1, substeps=20)
    assert rank == D
    # the reference is the host adaptive integrator (rel 1e-8 per step): its
    # norm drifts by ~2e-6 over the run, while the unitary RK4 in the
    # orthonormal basis keeps y^H y to RK4 accuracy
    assert np.ptp(n2) < 1e-9 * n2[0]
    np.testing.assert_allclose(n2, n1, rtol=1e-5)
    np.testing.assert_allclose(o2, o1, rtol=1e-5, atol=1e-5 * np.abs(o1).max())
