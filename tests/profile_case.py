"""Short, fixed sampling runs for profilers (test support; not collected by pytest).

``python tests/profile_case.py [walkers] [gram_mode] [lanes] [N] [dL_min] [dL_max]``
builds the m=3 context (default N=50, dL=0..12, 272 basis states; N=100,
dL 1..20 gives the 2713-state batched shape), runs 10 burn-in sweeps and 6
measured sweeps (sweep -> basis -> contraction per sweep) and reads one Gram
block back.  Launch order on the context stream: the walker initialisation,
10 unmeasured sweeps, then per measured sweep one sweep, one basis build and
one contraction (plus the per-sector reduce at the end), so ``-s``/``-c`` of a
profiler select e.g. the third contraction with ``-k regex:gram_tc -s 2 -c 1``.

``python tests/profile_case.py learned [walkers]`` burns in a W-walker plain
context (N=200, m=3, default W=4096, 300 sweeps), trains the DeepSets
proposal on its configurations (init sigma 1.24, 1000 ES steps), then runs
three single unmeasured learned sweeps from the burnt-in walkers; the learned
sweeps are the last three launches of `learned_sweep_kernel`.

``python tests/profile_case.py learned_step [walkers] [steps]`` runs the
learned workload's full step: N=200, m=3, dL 1..20, TF32x3, default W=65536;
300 plain burn-in sweeps, a proposal trained for 1000 ES steps on those
walkers, then 2 unmeasured learned sweeps and `steps` (default 4) measured
steps (learned sweep -> basis -> contraction).

``python tests/profile_case.py occupation [walkers] [sweeps]`` runs one
occupation estimate (N=50, m=3, dL=4, l_cutoff = m(N-1)+15, sweeps/2 burn-in
+ sweeps measured in one launch; defaults 65536 walkers, 100 sweeps).
"""
from __future__ import annotations

import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

from laughlinedge_b200 import LearnedProposal, Sampler, SamplerConfig  # noqa: E402
from laughlinedge_b200.sampler import occupation  # noqa: E402


def learned(argv) -> int:
    import torch
    W = int(argv[0]) if argv else 4096
    N, m = 200, 3
    burn = Sampler(SamplerConfig(N, m, W, step_sigma=1.24, seed=1), [1])
    burn.init_walkers()
    burn.run(300, measure=False)
    cfg = torch.empty((W, N, 2), dtype=torch.float32, device="cuda")
    burn.copy_positions_device(cfg.data_ptr())
    burn.synchronize()
    xy = burn.positions()
    burn.close()
    prop = LearnedProposal(N, m, init_sigma=1.24, seed=5)
    prop.train(cfg.data_ptr(), W, steps=1000, batch=1024, pairs=32, lr=3e-3)
    smp = Sampler(SamplerConfig(N, m, W, step_sigma=0.3, seed=1, lanes_per_walker=0), [1])
    smp.set_proposal(prop)
    smp.init_walkers(xy)
    for _ in range(3):
        smp.run(1, measure=False)
    smp.synchronize()
    st = smp.stats()
    print("ok", st.acceptance, st.reverse_fraction)
    smp.close()
    prop.close()
    return 0


def learned_step(argv) -> int:
    import torch
    W = int(argv[0]) if argv else 65536
    steps = int(argv[1]) if len(argv) > 1 else 4
    N, m = 200, 3
    sectors = list(range(1, 21))
    burn = Sampler(SamplerConfig(N, m, W, step_sigma=1.24, seed=1, lanes_per_walker=8), [1])
    burn.init_walkers()
    burn.run(300, measure=False)
    cfg = torch.empty((W, N, 2), dtype=torch.float32, device="cuda")
    burn.copy_positions_device(cfg.data_ptr())
    burn.synchronize()
    xy = burn.positions()
    burn.close()
    prop = LearnedProposal(N, m, init_sigma=1.24, seed=5)
    prop.train(cfg.data_ptr(), W, steps=1000, batch=1024, pairs=32, lr=3e-3)
    del cfg
    smp = Sampler(SamplerConfig(N, m, W, step_sigma=0.3, seed=1, lanes_per_walker=0,
                                gram_mode=3), sectors)
    smp.set_proposal(prop)
    smp.init_walkers(xy)
    smp.run(2, measure=False)
    smp.run(steps, measure=True)
    smp.synchronize()
    st = smp.stats()
    print("ok", st.acceptance, st.reverse_fraction)
    smp.close()
    prop.close()
    return 0


def occ(argv) -> int:
    W = int(argv[0]) if argv else 65536
    sweeps = int(argv[1]) if len(argv) > 1 else 100
    N, m = 50, 3
    out, acc = occupation(N, m, 4, m * (N - 1) + 15, W, sweeps, burn_in=sweeps // 2)
    print("ok", acc, out.shape)
    return 0


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if argv and argv[0] == "learned":
        return learned(argv[1:])
    if argv and argv[0] == "learned_step":
        return learned_step(argv[1:])
    if argv and argv[0] == "occupation":
        return occ(argv[1:])
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
