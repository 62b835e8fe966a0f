"""The replica path (one process per GPU, no collective inside a step) with two
gloo ranks on CPU: distinct Philox keys per rank, the max-over-ranks timing
reduction, and the final FP64 sum of the raw Gram planes, whose normalised
result equals that of one run over both ranks' samples."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _grams(rank):
    g = np.random.default_rng(100 + rank)
    v = g.normal(size=(500, 4)) + 1j * g.normal(size=(500, 4))
    r2 = 1 + g.random(500)
    S = np.einsum("wa,wb->ab", v.conj(), v)
    H2 = np.einsum("w,wa,wb->ab", r2, v.conj(), v)
    return S, H2, np.array([500.0])


def _worker(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    from laughlinedge_b200 import replicas
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        seed = replicas.rank_seed(42, rank)
        tmax = replicas.max_over_ranks(1.5 + rank)
        S, H2, n = replicas.sum_over_ranks(list(_grams(rank)))
        np.save(out / f"r{rank}.npy", np.array([seed, tmax, n[0]]))
        np.save(out / f"S{rank}.npy", S)
        np.save(out / f"H{rank}.npy", H2)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    mp.spawn(_worker, args=(2, _free_port(), tmp_path), nprocs=2, join=True)
    r0, r1 = np.load(tmp_path / "r0.npy"), np.load(tmp_path / "r1.npy")
    assert r0[0] != r1[0]                       # disjoint Philox keys
    assert r0[1] == r1[1] == 2.5                # the slowest rank's time, on every rank
    assert r0[2] == r1[2] == 1000               # samples of both ranks
    S0, S1 = np.load(tmp_path / "S0.npy"), np.load(tmp_path / "S1.npy")
    assert np.array_equal(S0, S1)
    a, b = _grams(0), _grams(1)
    assert np.allclose(S0, a[0] + b[0], rtol=1e-14)
    assert np.allclose(np.load(tmp_path / "H0.npy"), a[1] + b[1], rtol=1e-14)
