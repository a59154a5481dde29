"""The data-parallel step on two CPU ranks (backend gloo, 127.0.0.1): each rank
computes its NEE_DS sigma gradient with its own Philox key -- on the CPU the
oracle stands in for the path kernels -- and allreduce_grads leaves every rank
with the sum of both ranks' gradients; timings reduce to the slowest rank."""
import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from rendervous_b200 import distributed as vdist
from rendervous_b200 import synthetic
from tests.helpers import oracle_desc

H = W = 8
SPP = 4


def _grad(rank: int, step: int) -> np.ndarray:
    import oracle
    sig = synthetic.gaussian_blobs(9, 3, 4.0, seed=8)
    sc = oracle.OracleScene(oracle_desc(sig, albedo=0.7, env=1.0, sun_dir=(0.2, 1.0, 0.1), g=0.3, max_bounces=8),
                            with_grads=True)
    wimg = np.random.default_rng(3).random((1, H, W, 3)).astype(np.float32)
    oracle.capture_bw(sc, "ds", synthetic.ring_poses(1), W, H, math.pi / 4, True, SPP, vdist.rank_seed(step, rank), wimg)
    return sc.sigma_grad.copy()


def _rank(rank: int, world: int, port: int, out: str) -> None:
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = torch.nn.Parameter(torch.zeros(9, 9, 9, 1))
        p.grad = torch.from_numpy(_grad(rank, step=5))
        vdist.allreduce_grads([p])
        slowest = vdist.max_over_ranks(10.0 * (rank + 1))
        total = vdist.sum_over_ranks(1.0 + rank)
        np.save(f"{out}_{rank}.npy", p.grad.numpy())
        np.save(f"{out}_{rank}_red.npy", np.array([slowest, total]))
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_rank_seeds_are_distinct():
    # past 1000 steps too (an earlier key, 1000 * (rank + 1) + step, repeated there)
    seeds = {vdist.rank_seed(k, r) for k in range(5000) for r in range(8)}
    assert len(seeds) == 5000 * 8
    assert vdist.rank_seed(1000, 0) != vdist.rank_seed(0, 1)
    assert all(0 < s < (1 << 62) for s in seeds)


def test_two_rank_gradient_allreduce(tmp_path):
    import oracle
    oracle.build()
    out = str(tmp_path / "g")
    mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    expect = _grad(0, 5) + _grad(1, 5)
    assert np.abs(_grad(0, 5) - _grad(1, 5)).sum() > 0          # the ranks' paths differ
    for r in range(2):
        g = np.load(f"{out}_{r}.npy")
        # the oracle's threads add into the gradient in any order: float rounding only
        assert np.allclose(g, expect, rtol=1e-5, atol=1e-6 * np.abs(expect).max())
        slowest, total = np.load(f"{out}_{r}_red.npy")
        assert slowest == 20.0 and total == 3.0
