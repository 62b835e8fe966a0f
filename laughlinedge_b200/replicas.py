"""Walker replicas over several GPUs: one process per GPU, each with its own
walkers and Philox key, no collective inside a sampling step.  The only
cross-rank steps are the timing reduction of a benchmark (max over ranks) and
the final sum of the FP64 Gram planes, after which the combined raw sums are
normalised as one run's (lemc_normalise).  The reference has no multi-GPU
path; its walkers are one grid on one GPU."""
from __future__ import annotations

import numpy as np


def rank_seed(seed: int, rank: int) -> int:
    """Philox key of a rank's walkers: disjoint streams for every rank."""
    return int(seed) + 1000003 * int(rank)


def _device():
    import torch
    import torch.distributed as dist
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" \
        else torch.device("cpu")


def max_over_ranks(x: float) -> float:
    """Max of a scalar over the ranks of the default process group (the
    device time of a step is the slowest rank's)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(arrays):
    """Elementwise FP64 sum over ranks of a list of numpy arrays (complex arrays
    are summed as their real and imaginary parts): the raw Gram sums S, H2, H4
    and sample counts of every rank's walkers, combined into one estimate."""
    import torch
    import torch.distributed as dist
    out = []
    for a in arrays:
        a = np.ascontiguousarray(a)
        if not dist.is_initialized() or dist.get_world_size() == 1:
            out.append(a.copy())
            continue
        real = a.view(np.float64) if np.iscomplexobj(a) else a.astype(np.float64)
        t = torch.from_numpy(np.ascontiguousarray(real).ravel().copy()).to(_device())
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        r = t.cpu().numpy()
        out.append(r.view(np.complex128).reshape(a.shape) if np.iscomplexobj(a) else r.reshape(a.shape))
    return out
