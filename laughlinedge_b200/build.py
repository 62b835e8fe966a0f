"""In-tree build of the native library ``liblemc.so`` (CUDA sm_100a + host C++).

The library is compiled with nvcc for ``-gencode arch=compute_100a,code=sm_100a``
only; nvcc cross-compiles without a GPU.  Objects go to ``_build/`` next to the
sources and are relinked only when a source or header is newer.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "liblemc.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
                     "-DLEMC_BUILD"]
HOST_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-DLEMC_BUILD"]


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _headers():
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.hpp")) + sorted((ROOT / "include").glob("*.h"))


def _newest(paths):
    return max((p.stat().st_mtime for p in paths), default=0.0)


def _compile(src: Path, hdr_time: float, verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_time):
        return obj
    if src.suffix == ".cu":
        cmd = [NVCC] + CUDA_FLAGS + ["-c", str(src), "-o", str(obj)]
    else:
        cmd = [NVCC, "-x", "c++", "-Xcompiler", ",".join(HOST_FLAGS), "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compilation failed: {src.name}\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile every CUDA/C++ source under csrc/ and link liblemc.so."""
    BUILD.mkdir(exist_ok=True)
    srcs = _sources()
    hdr_time = _newest(_headers())
    if force:
        for o in BUILD.glob("*.o"):
            o.unlink()
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, hdr_time, verbose), srcs))
    if LIB.exists() and LIB.stat().st_mtime >= _newest(objs) and not force:
        return LIB
    cmd = [NVCC] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + ["-lcudart", "-lcusolver", "-lcublas"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
