"""LaughlinEdge B200: variational Monte Carlo of Laughlin edge states on sm_100a.

The compute path is the native library ``liblemc.so`` (hand-written CUDA for
sm_100a behind the C-ABI of include/lemc.h); this package only binds it.
"""
from . import _lib, dynamics
from ._lib import LemcError, load
from .dynamics import density_grid, edge_response
from .proposal import LearnedProposal
from .sampler import (Sampler, SamplerConfig, dsf_compute, dsf_weights, evolve, evolve_device, geneig,
                      geneig_sweep, jackknife_spectrum, normalise, occupation, partitions, series_tau,
                      spectral_function, spectral_weights, tau_binning, tau_sokal)

__all__ = ["LearnedProposal", "LemcError", "Sampler", "SamplerConfig", "density_grid", "dsf_compute",
           "dsf_weights", "edge_response", "evolve",
           "evolve_device", "geneig", "geneig_sweep", "jackknife_spectrum", "load", "occupation",
           "spectral_function", "spectral_weights", "normalise", "partitions", "series_tau",
           "tau_binning", "tau_sokal", "_lib"]
