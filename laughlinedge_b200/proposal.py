"""Learned Metropolis-Hastings proposal (DeepSets network) through the C-ABI.

The network and its exact acceptance rule live in ``liblemc.so`` (CUDA for
sm_100a); this module owns a ``lemc_proposal`` handle: its FP32 weights, the
evolution-strategies + Adam training on device-resident configurations, and a
per-sample evaluation used by the tests.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, fptr, i32ptr


def n_params() -> int:
    n = C.c_int()
    check(_lib.load().lemc_proposal_n_params(C.byref(n)), "lemc_proposal_n_params")
    return n.value


class LearnedProposal:
    """Weights of the learned single-particle proposal for N particles at nu = 1/m."""

    def __init__(self, particles: int, inverse_filling: int, init_sigma: float = 0.3,
                 seed: int = 1):
        self.lib = _lib.load()
        self.particles, self.inverse_filling = particles, inverse_filling
        self._h = C.c_void_p()
        check(self.lib.lemc_proposal_create(particles, inverse_filling, init_sigma, seed,
                                            C.byref(self._h)), "lemc_proposal_create")

    def close(self):
        if self._h:
            self.lib.lemc_proposal_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass

    @property
    def params(self) -> np.ndarray:
        out = np.zeros(n_params(), dtype=np.float32)
        check(self.lib.lemc_proposal_get_params(self._h, fptr(out), out.size),
              "lemc_proposal_get_params")
        return out

    @params.setter
    def params(self, value):
        v = np.ascontiguousarray(value, dtype=np.float32)
        check(self.lib.lemc_proposal_set_params(self._h, fptr(v), v.size),
              "lemc_proposal_set_params")

    def evaluate(self, xy: np.ndarray, particle, eps) -> np.ndarray:
        """[n, 8]: mu_r, mu_t, log s_r, log s_t, z'.x, z'.y, ln A, |z'-z|^2."""
        xy = np.ascontiguousarray(xy, dtype=np.float32)
        n = xy.shape[0]
        pi = np.ascontiguousarray(particle, dtype=np.int32)
        e = np.ascontiguousarray(eps, dtype=np.float32)
        out = np.zeros((n, 8), dtype=np.float32)
        check(self.lib.lemc_proposal_eval(self._h, fptr(xy.ravel()), n, i32ptr(pi),
                                          fptr(e.ravel()), fptr(out.ravel())),
              "lemc_proposal_eval")
        return out

    def train(self, configs_device_ptr: int, n_configs: int, steps: int, batch: int = 1024,
              pairs: int = 32, lr: float = 3e-3, es_sigma: float = 0.02, seed: int = 7):
        """Evolution-strategies + Adam on device configurations ([n][N] float2)."""
        tc = _lib.TrainConfig(steps, batch, pairs, lr, es_sigma, seed)
        trace = np.zeros(steps)
        check(self.lib.lemc_proposal_train(self._h, C.c_void_p(configs_device_ptr), n_configs,
                                           C.byref(tc), trace.ctypes.data_as(_lib._DP)),
              "lemc_proposal_train")
        return trace
