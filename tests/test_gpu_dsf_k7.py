"""Self-consistency of the sampled excitation matrix elements with the
contraction (the DSF known answer for the multipole drive sum_i z_i^k): p_k Psi
is itself the basis state (k) of sector k, so <Psi| sum_i r_i^k cos(k theta_i)
|v_a Psi> = (N R^k / 2) <p_k Psi|v_a Psi> for every state a of sector k (the
other half, <Psi|p_k v_a Psi>, vanishes by rotation symmetry).  The cross sums
of the built-in drive (lemc_set_multipole_potential) and the Gram row of the
state (k) estimate the two sides from the same samples; they must agree
within the replicas' statistical error, and so must the DSF weights they give
for the confinement eigenstates of sector k."""
import math

import numpy as np
import pytest
import scipy.linalg as sl
from scipy import stats

pytestmark = pytest.mark.gpu


def test_drive_cross_sums_match_gram_row(lemc, cuda_ctx):
    N, m, k, om, ka = 8, 3, 2, 1e-2, 1e-4
    R = math.sqrt(2 * m * N)
    rows, _, _ = lemc.partitions(N, [k])
    rk = [i for i, (_, pr) in enumerate(rows) if pr == [(k, 1)]][0]
    lhs, rhs, wl, wr = [], [], [], []
    for r in range(6):
        smp = lemc.Sampler(lemc.SamplerConfig(N, m, 8192, seed=70 + r), [0, k])
        assert smp.lib.lemc_set_multipole_potential(smp._h, k, 1.0) == 0
        smp.init_walkers()
        smp.run(300, measure=False)
        smp.run(600, measure=True)
        cu, _, _ = smp.cross(0, 1)
        S, H2, H4, _ = smp.gram(1)
        smp.close()
        a = cu[0] * 2.0 / (N * R ** k)   # <Psi|U|v_a Psi> scaled to <p_k Psi|v_a Psi>
        b = S[rk]
        lhs.append(np.concatenate([a.real, a.imag]))
        rhs.append(np.concatenate([b.real, b.imag]))
        # DSF weights of the sector's eigenstates (H c = E S c, c^H S c = 1)
        M, H = lemc.normalise(S, H2, H4, om, ka)
        e, c = sl.eigh(H, M)
        d = np.sqrt(np.real(np.diag(S)))
        cn = c / d[:, None]                 # eigenvectors in the raw (unnormalised) basis
        wl.append(np.abs(a @ cn) ** 2)       # |<p_k Psi|c_j>|^2 from either side
        wr.append(np.abs(b @ cn) ** 2)
    for A, B, label in ((lhs, rhs, "cross vs Gram row"), (wl, wr, "DSF weights")):
        A, B = np.array(A), np.array(B)
        va, vb = A.var(0, ddof=1) / len(A), B.var(0, ddof=1) / len(B)
        live = (va + vb) > 1e-30 * (np.abs(B).max() ** 2)
        se2 = va[live] + vb[live]
        t = np.abs(A.mean(0)[live] - B.mean(0)[live]) / np.sqrt(se2)
        dof = se2 ** 2 / (va[live] ** 2 / (len(A) - 1) + vb[live] ** 2 / (len(B) - 1))
        crit = stats.t.isf(1e-3 / len(t) / 2, dof)
        print(label, A.mean(0), B.mean(0), "max t", t.max(), flush=True)
        assert np.all(t < crit), (label, t, crit)
