"""The C++ drop-in layer: the reference's main.cu usage compiles against
include/modules and links to liblemc.so (CPU); on a GPU it runs and writes the
reference's output files (gpu)."""
import math
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "drop_in_main.cu"
OUT_BIN = ROOT / "laughlinedge_b200" / "_build" / "drop_in_main"


def _build(lemc):
    OUT_BIN.parent.mkdir(exist_ok=True)
    cmd = ["/usr/local/cuda/bin/nvcc", "-std=c++17", "--extended-lambda", "-O2",
           "-gencode", "arch=compute_100a,code=sm_100a", "-I", str(ROOT / "include" / "modules"),
           str(SRC), "-L", str(ROOT / "laughlinedge_b200"), "-llemc",
           f"-Xlinker=-rpath={ROOT / 'laughlinedge_b200'}", "-o", str(OUT_BIN)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_drop_in_program_compiles_and_links(lemc):
    _build(lemc)
    assert OUT_BIN.exists()


def test_sys_params_generator(tmp_path):
    exe = tmp_path / "gen"
    subprocess.run(["g++", "-O1", "-o", str(exe), str(ROOT / "include" / "system_parameters.cpp")],
                   check=True)
    (tmp_path / "modules").mkdir()
    subprocess.run([str(exe)], cwd=tmp_path, check=True)
    txt = (tmp_path / "modules" / "sys_params.h").read_text()
    for name in ("particlesNumber", "inverseFilling", "confinementExponent", "confinementStrength",
                 "RCl", "DCl", "RCl_reciprocal", "R0_reciprocal", "ansatzExtendedMaxDegree",
                 "ansatzMaxPartitionSize", "ansatzSubspaceDimension", "ansatzMultipletSize",
                 "ansatzMaxAngularMomentum", "angularMomentumCutoff", "confinementOmega",
                 "confinementKappa"):
        assert f" {name} = " in txt, name


@pytest.mark.gpu
def test_drop_in_program_runs(lemc, cuda_ctx, tmp_path):
    _build(lemc)
    work = tmp_path / "run"
    work.mkdir()
    r = subprocess.run([str(OUT_BIN)], cwd=work, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    lines = {l.split()[0]: l.split()[1:] for l in r.stdout.splitlines() if l[:4] in ("SPEC", "DSF ", "DYNA", "OCCU")}
    # spectrum of dL = 3 with V = 1e-2 r^2 + 1e-4 r^4 at N = 8, m = 3: three levels near
    # the harmonic value 1e-2 * 2 (L_tot + N) = 1.90 plus the quartic shift
    ev = np.array(lines["SPECTRUM"], float)
    assert len(ev) == 3 and np.all(np.diff(ev) >= 0) and np.all((ev > 2.3) & (ev < 2.7))
    dsf = np.array(lines["DSF"], float).reshape(-1, 2)
    assert len(dsf) == 2 and np.all(dsf[:, 1] >= 0)
    out = tmp_path / "output" / "N=8_m=3"
    for f in ("dL=3/Statistics/Hamiltonian/0.tsv", "dL=3/Statistics/Metric/0.tsv",
              "dL=2/Statistics/cosine_excitation/0.tsv", "dL=2/Statistics/sine_excitation/0.tsv",
              "ExternalExcitation/Statistics/Hamiltonian/0.tsv",
              "ExternalExcitation/Statistics/ExcitationPotential/0.tsv",
              "ExternalExcitation/Statistics/EdgeDenstiy_FourierTransform/dL=2/0.tsv",
              "ExternalExcitation/Statistics/edgeDynamics/dL=2/0.tsv",
              "dL=0/Statistics/OccupationNumbers_not_normalized/0.tsv"):
        assert (out / f).exists(), f
    M = np.loadtxt(out / "dL=3/Statistics/Metric/0.tsv")
    assert np.allclose(M[M[:, 0] == M[:, 1]][:, 2], 1.0, atol=1e-6)  # normalised diagonal
    occ = np.loadtxt(out / "dL=0/Statistics/OccupationNumbers_not_normalized/0.tsv")
    assert abs(occ[:, 3].sum() - 8.0) < 1e-4  # sum rule, N = 8 (6-decimal files)
    dyn = np.loadtxt(out / "ExternalExcitation/Statistics/edgeDynamics/dL=0/0.tsv")
    assert dyn.shape[0] == 80 and np.all(np.isfinite(dyn))
