"""LaughlinEdge B200: variational Monte Carlo of Laughlin edge states on sm_100a.

The compute path is the native library ``liblemc.so`` (hand-written CUDA for
sm_100a behind the C-ABI of include/lemc.h); this package only binds it.
"""
from . import _lib
from ._lib import LemcError, load
from .proposal import LearnedProposal
from .sampler import (Sampler, SamplerConfig, evolve, evolve_device, geneig, geneig_sweep, normalise,
                      partitions)

__all__ = ["LearnedProposal", "LemcError", "Sampler", "SamplerConfig", "evolve", "evolve_device", "geneig", "geneig_sweep", "load",
           "normalise", "partitions", "_lib"]
