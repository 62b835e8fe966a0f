"""ctypes binding of the C-ABI in include/lemc.h.

The product path is the native library only: if ``liblemc.so`` cannot be
loaded the import raises, and every compute entry point returns the library's
status, which is turned into :class:`LemcError`.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "liblemc.so"

LEMC_OK = 0
STATUS = {0: "ok", -1: "invalid argument", -2: "capacity exceeded", -3: "CUDA error",
          -4: "device wait timed out", -5: "numerical failure", -6: "call out of order",
          -7: "no CUDA device", -8: "file i/o error"}

GUIDE_LAUGHLIN, GUIDE_ROW = 0, 1
MAX_PROBES = 8
GRAM_FP64, GRAM_BF16X3, GRAM_BF16X4, GRAM_TF32X3 = 0, 1, 2, 3
MAX_DEGREE = 24
W_ONE, W_R2, W_R4, W_USER, W_PROBE0 = range(5)
N_WEIGHTS = W_PROBE0 + 2 * MAX_PROBES


class LemcError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS.get(status, status)} {detail}".strip())


class Config(C.Structure):
    _fields_ = [("particles", C.c_int32), ("inverse_filling", C.c_int32),
                ("n_walkers", C.c_int32), ("lanes_per_walker", C.c_int32),
                ("step_sigma", C.c_float), ("guide", C.c_int32), ("seed", C.c_uint64),
                ("radius_scale", C.c_double), ("init_radius", C.c_double),
                ("gram_mode", C.c_int32), ("graph_batch", C.c_int32),
                ("flush_every", C.c_int32), ("profile", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("sweeps", C.c_uint64), ("measurements", C.c_uint64),
                ("acceptance", C.c_double), ("tau_int", C.c_double),
                ("tau_int_each", C.c_double * 4), ("ms_sweep", C.c_double),
                ("ms_basis", C.c_double), ("ms_gram", C.c_double),
                ("reverse_fraction", C.c_double)]


class OccConfig(C.Structure):
    _fields_ = [("particles", C.c_int32), ("inverse_filling", C.c_int32), ("dL", C.c_int32),
                ("l_cutoff", C.c_int32), ("n_walkers", C.c_int32), ("step_sigma", C.c_float),
                ("seed", C.c_uint64), ("burn_in", C.c_int32), ("sweeps", C.c_int32)]


class TrainConfig(C.Structure):
    _fields_ = [("steps", C.c_int32), ("batch", C.c_int32), ("pairs", C.c_int32),
                ("lr", C.c_float), ("es_sigma", C.c_float), ("seed", C.c_uint64)]


class PartitionRow(C.Structure):
    _fields_ = [("dL", C.c_int32), ("sector_size", C.c_int32), ("n_pairs", C.c_int32),
                ("pairs_off", C.c_int32)]


PROFILE_FN = C.CFUNCTYPE(C.c_double, C.c_double, C.c_void_p)
STEP_HOOK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p)

_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)
_I32P = C.POINTER(C.c_int32)
_FP = C.POINTER(C.c_float)

_SIGNATURES = {
    "lemc_version": ([], _I),
    "lemc_status_string": ([_I], C.c_char_p),
    "lemc_device_count": ([_IP], _I),
    "lemc_partitions": ([_I, _I32P, _I, C.POINTER(PartitionRow), _I, _I32P, _I, _IP, _IP, _IP, _IP], _I),
    "lemc_create": ([C.POINTER(Config), C.POINTER(_P)], _I),
    "lemc_destroy": ([_P], _I),
    "lemc_set_sectors": ([_P, _I32P, _I], _I),
    "lemc_lanes_per_walker": ([_P, _IP], _I),
    "lemc_gram_splits": ([_P, _IP], _I),
    "lemc_set_guide_rows": ([_P, _I32P, _I], _I),
    "lemc_init_walkers": ([_P, _FP], _I),
    "lemc_run": ([_P, _I, _I], _I),
    "lemc_reset_accumulators": ([_P], _I),
    "lemc_synchronize": ([_P], _I),
    "lemc_stream": ([_P, C.POINTER(_P)], _I),
    "lemc_sector_dim": ([_P, _I, _IP], _I),
    "lemc_total_dim": ([_P, _IP], _I),
    "lemc_read_gram": ([_P, _I, _DP, _DP, _DP, _DP], _I),
    "lemc_read_cross": ([_P, _I, _I, _DP, _DP, _DP], _I),
    "lemc_read_rows": ([_P, _D, _D, _DP, _DP, _DP, _DP, _DP, _DP, _DP], _I),
    "lemc_set_step": ([_P, C.c_float], _I),
    "lemc_tune_step": ([_P, _D, _D, _I, _FP, _DP], _I),
    "lemc_occupation": ([C.POINTER(OccConfig), _DP, _DP], _I),
    "lemc_occupation_static": ([C.POINTER(OccConfig), _DP, _DP], _I),
    "lemc_read_stats": ([_P, C.POINTER(Stats)], _I),
    "lemc_read_positions": ([_P, _FP], _I),
    "lemc_read_series": ([_P, _DP, _I, _IP], _I),
    "lemc_tau_sokal": ([_DP, _I, _D, _DP], _I),
    "lemc_debug_gram_wait": ([C.c_longlong, _I], _I),
    "lemc_close_bin": ([_P], _I),
    "lemc_n_bins": ([_P, _IP], _I),
    "lemc_read_gram_bin": ([_P, _I, _I, _DP, _DP, _DP, _DP], _I),
    "lemc_jackknife_spectrum": ([_I, _I, _DP, _DP, _DP, _D, _D, _D, _DP, _DP, _DP, _DP], _I),
    "lemc_tau_binning": ([_DP, _I, _I, _DP, _DP, _DP, _IP], _I),
    "lemc_sweep_device": ([_P, _I, _I, _I, C.c_float, C.c_uint64, C.c_uint32, _I, _I, _D, _I, _I,
                           _I32P, _I, _P, _P, _P, _P], _I),
    "lemc_set_probes": ([_P, _I32P, _I], _I),
    "lemc_run_hooked": ([_P, _I, STEP_HOOK, _P], _I),
    "lemc_basis_device": ([_P, _P, _I, _P, _I, _P], _I),
    "lemc_gram_device": ([_P, _P, _P, _I, _I, _I, _P], _I),
    "lemc_geneig": ([_I, _DP, _DP, _D, _DP, _DP, _IP], _I),
    "lemc_spectral_weights": ([_I, _I, _DP, _DP, _DP, _I, _D, _DP, _DP, _IP], _I),
    "lemc_dsf_weights": ([_I, _DP, _DP, _DP, _DP, _D, _DP, _DP, _IP], _I),
    "lemc_proposal_n_params": ([_IP], _I),
    "lemc_proposal_create": ([_I, _I, C.c_float, C.c_uint64, C.POINTER(_P)], _I),
    "lemc_proposal_destroy": ([_P], _I),
    "lemc_proposal_get_params": ([_P, _FP, _I], _I),
    "lemc_proposal_set_params": ([_P, _FP, _I], _I),
    "lemc_proposal_eval": ([_P, _FP, _I, _I32P, _FP, _FP], _I),
    "lemc_proposal_train": ([_P, _P, _I, C.POINTER(TrainConfig), _DP], _I),
    "lemc_set_proposal": ([_P, _P], _I),
    "lemc_copy_positions_device": ([_P, _P], _I),
    "lemc_geneig_sweep": ([_I, _DP, _DP, _DP, _DP, _DP, _I, _D, _DP, _IP], _I),
    "lemc_normalise": ([_I, _DP, _DP, _DP, _D, _D, _DP, _DP], _I),
    "lemc_edge_density_grid": ([_I, _I32P, _I, _DP, _DP, _I, _DP], _I),
    "lemc_set_multipole_potential": ([_P, _I, _D], _I),
    "lemc_evolve": ([_I, _DP, _DP, _DP, _I, _DP, PROFILE_FN, _P, _D, _D, _DP, _DP, _IP], _I),
    "lemc_evolve_device": ([_I, _DP, _DP, _DP, _I, _DP, PROFILE_FN, _P, _D, _D, _I, _D, _DP, _DP,
                            _IP, _IP], _I),
}

_lib = None


def load(path: os.PathLike | None = None) -> C.CDLL:
    """Load liblemc.so and declare every exported signature (raises if missing)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"native library {p} not built; run python -m laughlinedge_b200.build")
    lib = C.CDLL(str(p))
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if path is None:
        _lib = lib
    return lib


def check(status: int, where: str) -> None:
    if status != LEMC_OK:
        detail = ""
        try:
            detail = "(" + load().lemc_status_string(status).decode() + ")"
        except Exception:  # pragma: no cover
            pass
        raise LemcError(status, where, detail)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_FP)


def i32ptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I32P)
