"""A short, fixed sampling run for profilers.

``python -m laughlinedge_b200.profile_case [walkers] [gram_mode] [lanes] [N]
[dL_min] [dL_max]`` builds the m=3 context (default N=50, dL=0..12, 272 basis
states; N=100, dL 1..20 gives the 2713-state batched shape), runs 10 burn-in
sweeps and 6 measured sweeps (sweep -> basis -> contraction per sweep) and
reads one Gram block back.  Launch order on the context stream: the walker
initialisation, 10 unmeasured sweeps, then per measured sweep one sweep, one
basis build and one contraction (plus the per-sector reduce at the end), so
``-s``/``-c`` of a profiler select e.g. the third contraction with
``-k regex:gram_tc -s 2 -c 1``.
"""
from __future__ import annotations

import sys

from . import SamplerConfig, Sampler


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    W = int(argv[0]) if len(argv) > 0 else 16384
    mode = int(argv[1]) if len(argv) > 1 else 3
    lanes = int(argv[2]) if len(argv) > 2 else 4
    N = int(argv[3]) if len(argv) > 3 else 50
    dl_min = int(argv[4]) if len(argv) > 4 else 0
    dl_max = int(argv[5]) if len(argv) > 5 else 12
    sectors = list(range(dl_min, dl_max + 1))
    smp = Sampler(SamplerConfig(N, 3, W, lanes_per_walker=lanes, gram_mode=mode), sectors)
    smp.init_walkers()
    smp.run(10, measure=False)
    smp.run(6, measure=True)
    smp.synchronize()
    S, H2, H4, n = smp.gram(len(sectors) - 1)
    print("ok", n, float(S[0, 0].real))
    smp.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
