"""The Eigen stand-in under oracle/eigen_shim (test infrastructure that lets the
reference's own sampler compile) against scipy.linalg.eigh on random Hermitian
problems: eigenvalues, and eigenvectors up to phase with x^H B x = 1."""
import subprocess
from pathlib import Path

import numpy as np
import pytest
import scipy.linalg as sl

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def shim_exe(tmp_path_factory):
    exe = tmp_path_factory.mktemp("shim") / "eigen_shim_check"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{ROOT / 'oracle' / 'eigen_shim'}",
                    str(ROOT / "tests" / "cpp" / "eigen_shim_check.cpp"), "-o", str(exe)], check=True)
    return exe


def _run(exe, A, B):
    n = A.shape[0]
    txt = [str(n)]
    for M in (A, B):
        txt += [f"{float(z.real)!r} {float(z.imag)!r}" for z in M.ravel()]
    out = subprocess.run([str(exe)], input="\n".join(txt), capture_output=True, text=True,
                         check=True).stdout.split("\n")
    ev = np.array([float(x) for x in out[:n]])
    vec = np.array([complex(*map(float, l.split())) for l in out[n:n + n * n]]).reshape(n, n)
    return ev, vec, int(out[n + n * n])


@pytest.mark.parametrize("n,seed", [(1, 0), (2, 1), (5, 2), (11, 3), (30, 4)])
def test_shim_matches_scipy(shim_exe, n, seed):
    g = np.random.default_rng(seed)
    X = g.normal(size=(n, n)) + 1j * g.normal(size=(n, n))
    A = X + X.conj().T
    Y = g.normal(size=(n, n)) + 1j * g.normal(size=(n, n))
    B = Y @ Y.conj().T + n * np.eye(n)
    ev, vec, ncap = _run(shim_exe, A, B)
    ref = sl.eigh(A, B, eigvals_only=True)
    assert np.allclose(ev, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())
    # A x = lambda B x and x^H B x = 1 for every returned vector
    assert np.allclose(A @ vec, (B @ vec) * ev[None, :], atol=1e-9 * np.abs(ref).max())
    assert np.allclose(vec.conj().T @ B @ vec, np.eye(n), atol=1e-9)
    assert ncap == 2  # both solver calls were captured


def test_shim_degenerate_and_indefinite(shim_exe):
    n = 4
    A = np.diag([2.0, 2.0, 1.0, 3.0]).astype(complex)
    ev, _, _ = _run(shim_exe, A, np.eye(n, dtype=complex))
    assert np.allclose(ev, [1, 2, 2, 3])
    B = np.diag([1.0, -1.0, 1.0, 1.0]).astype(complex)
    ev, _, _ = _run(shim_exe, A, B)
    assert np.all(np.isnan(ev))
