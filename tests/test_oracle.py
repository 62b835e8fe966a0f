"""The oracle pinned against golden vectors and closed forms (CPU only)."""
import json
import math
from pathlib import Path

import numpy as np
import pytest
import scipy.linalg as sl

from kat import gram_m1, harmonic_level, spectrum_m1

GOLD = Path(__file__).resolve().parent / "golden"


def test_philox_known_answers(oracle):
    kat = json.loads((GOLD / "philox_kat.json").read_text())
    for v in kat["vectors"]:
        assert oracle.philox(v["ctr"], v["key"]) == v["out"]


def test_partitions_match_reference_generator(oracle):
    gold = json.loads((GOLD / "partitions_ref.json").read_text())
    for case in gold["cases"]:
        rows = oracle.partitions(case["N"], case["sectors"])
        assert len(rows) == case["dim"]
        for got, want in zip(rows, case["rows"]):
            assert got[0] == want["dL"]
            assert [list(p) for p in got[1]] == want["pairs"]


def test_partition_counts(oracle):
    # p(n) for n = 0..20
    pn = [1, 1, 2, 3, 5, 7, 11, 15, 22, 30, 42, 56, 77, 101, 135, 176, 231, 297, 385, 490, 627]
    for n, want in enumerate(pn):
        assert len(oracle.partitions(64, [n])) == want


def _replicas(oracle, fn, nrep, **kw):
    return [fn(seed=1000 + r, **kw) for r in range(nrep)]


def test_oracle_m1_closed_form_gram_and_spectrum(oracle):
    N, m, dL = 4, 1, 3
    R = math.sqrt(2 * m * N)
    ests, evs = [], []
    for r in range(4):
        rows, S, H2, H4 = oracle.run_gram(N, m, 512, 0.5, 100 + r, 200, 600, [dL])
        d = np.sqrt(np.real(np.diag(S)))
        ests.append((S / np.outer(d, d)).real)
        H = (0.01 * H2 + 1e-3 * H4) / np.outer(d, d)
        evs.append(sl.eigh(H, S / np.outer(d, d), eigvals_only=True))
    ex = gram_m1(N, rows, R)
    de = np.sqrt(np.diag(ex))
    Me = ex / np.outer(de, de)
    mean, err = np.mean(ests, 0), np.std(ests, 0, ddof=1) / 2 + 1e-4
    assert np.all(np.abs(mean - Me) < 5 * err)
    emean, eerr = np.mean(evs, 0), np.std(evs, 0, ddof=1) / 2 + 1e-5
    assert np.all(np.abs(emean - spectrum_m1(N, dL, 0.01, 1e-3)) < 5 * eerr)


@pytest.mark.parametrize("mode", ["rows", "gram"])
def test_oracle_harmonic_degeneracy(oracle, mode):
    N, m, dL = 6, 3, 3
    evs = []
    for r in range(4):
        if mode == "rows":
            res = oracle.run_rows(N, m, 256, 0.3, 7 + r, 200, 400, [dL])
            M, H = oracle.reference_matrices(res["fg"], res["gg"], res["fh2"], res["n_row"])
        else:
            rows, S, H2, _ = oracle.run_gram(N, m, 256, 0.3, 7 + r, 200, 400, [dL])
            d = np.sqrt(np.real(np.diag(S)))
            M, H = S / np.outer(d, d), H2 / np.outer(d, d)
        evs.append(sl.eigh(H, M, eigvals_only=True))
    # noise splits the degenerate level symmetrically (eigenvalue repulsion):
    # the centre is unbiased, the spread shrinks with the sample count
    lvl = harmonic_level(N, m, dL)
    centres = [np.mean(e) for e in evs]
    assert abs(np.mean(centres) - lvl) < 5 * np.std(centres, ddof=1) / 2 + 1e-3 * lvl
    assert np.max(np.abs(np.array(evs) - lvl)) < 0.02 * lvl
