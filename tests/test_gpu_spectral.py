"""Edge spectral function (energy-resolved orbital occupations) on the GPU
against the nu = 1 closed form: at m = 1 the edge eigenstates of
V = omega r^2 + kappa r^4 are the Schur states s_mu Psi_1, Slater
determinants of the orbitals n_j = mu_j + N - j, so every eigenstate's
occupation is exactly 1 on those orbitals and 0 elsewhere, and its energy is
E_mu = sum_j [2 omega (n_j + 1) + 4 kappa (n_j + 1)(n_j + 2)]."""
import numpy as np
import pytest

from kat import partitions_desc

pytestmark = pytest.mark.gpu


def test_spectral_function_nu1_closed_form(lemc, cuda_ctx):
    N, m, dL, om, ka = 6, 1, 3, 1e-2, 1e-3
    e, w = lemc.spectral_function(N, m, dL, om, ka, n_walkers=16384, burn_in=400, sweeps=1500,
                                  step_sigma=0.5, seed=21)
    Lc = w.shape[1]
    expect = []
    for mu in partitions_desc(dL):
        mu = list(mu) + [0] * (N - len(mu))
        orb = [mu[j] + N - 1 - j for j in range(N)]
        E = sum(2 * om * (n + 1) + 4 * ka * (n + 1) * (n + 2) for n in orb)
        occ = np.zeros(Lc)
        occ[orb] = 1.0
        expect.append((E, occ))
    expect.sort(key=lambda x: x[0])
    assert np.allclose(w.sum(1), N, atol=1e-9)
    for j, (E, occ) in enumerate(expect):
        assert abs(e[j] - E) < 0.02 * E, (j, e[j], E)
        assert np.max(np.abs(w[j] - occ)) < 0.06, (j, np.round(w[j], 3), occ)
