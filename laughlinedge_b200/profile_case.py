"""A short, fixed sampling run for profilers.

``python -m laughlinedge_b200.profile_case [walkers] [gram_mode] [lanes]`` builds
the N=50, m=3, dL=0..12 context (272 basis states), runs 10 burn-in sweeps and
6 measured sweeps (sweep -> basis -> contraction per sweep) and reads one Gram
block back.  Launch order on the context stream: the walker initialisation,
10 unmeasured sweeps, then per measured sweep one sweep, one basis build and
one contraction (plus the per-sector reduce at the end), so ``-s``/``-c`` of a
profiler select e.g. the third contraction with ``-k regex:gram_tc -s 2 -c 1``.
"""
from __future__ import annotations

import sys

from . import SamplerConfig, Sampler


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    W = int(argv[0]) if len(argv) > 0 else 16384
    mode = int(argv[1]) if len(argv) > 1 else 3
    lanes = int(argv[2]) if len(argv) > 2 else 4
    smp = Sampler(SamplerConfig(50, 3, W, lanes_per_walker=lanes, gram_mode=mode), list(range(13)))
    smp.init_walkers()
    smp.run(10, measure=False)
    smp.run(6, measure=True)
    smp.synchronize()
    S, H2, H4, n = smp.gram(12)
    print("ok", n, float(S[0, 0].real))
    smp.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
