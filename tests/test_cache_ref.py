"""The radiance-cache FP64 reference on the CPU: its hand-written backward
against torch autograd, the encoding's partition of unity, level sizes."""
import math

import pytest
import torch

from oracle import cache_ref
from rendervous_b200 import cache


def _problem(n=64, seed=0):
    g = torch.Generator().manual_seed(seed)
    res = cache.level_resolutions(2, 9)
    ng = cache.grid_size(res)
    grid = (torch.rand(ng, generator=g, dtype=torch.float64) - 0.5) * 0.5
    w = (torch.rand(cache.N_WEIGHTS, generator=g, dtype=torch.float64) - 0.5) * 0.6
    pos = torch.rand(n, 3, generator=g, dtype=torch.float64) * 2 - 1
    d = torch.randn(n, 3, generator=g, dtype=torch.float64)
    d = d / d.norm(dim=1, keepdim=True)
    tgt = torch.rand(n, 3, generator=g, dtype=torch.float64)
    return res, grid, w, pos, d, tgt


def test_level_resolutions_geometric():
    res = cache.level_resolutions(16, 128)
    assert len(res) == 16 and res[0] == 16 and res[-1] == 128
    assert all(b >= a for a, b in zip(res, res[1:]))
    assert cache.grid_size(res) == sum((r + 1) ** 3 * 2 for r in res)


def test_grid_size_matches_library():
    from rendervous_b200 import _lib
    ffi, lib = _lib.ffi_lib()
    res = cache.level_resolutions(16, 128)
    assert lib.vrt_cache_grid_size(ffi.new("int32_t[16]", res)) == cache.grid_size(res)


def test_sh_orthonormal():
    # Monte Carlo over the sphere: E[Y_i Y_j] * 4 pi == delta_ij
    g = torch.Generator().manual_seed(1)
    d = torch.randn(400000, 3, generator=g, dtype=torch.float64)
    d = d / d.norm(dim=1, keepdim=True)
    Y = cache_ref.sh4(d)
    gram = Y.T @ Y / d.shape[0] * 4 * math.pi
    assert torch.allclose(gram, torch.eye(16, dtype=torch.float64), atol=2e-2)


def test_encoding_partition_of_unity():
    res, grid, w, pos, d, tgt = _problem()
    x, _ = cache_ref.encode(torch.ones_like(grid), res, [-1, -1, -1], [1, 1, 1], pos, d)
    assert torch.allclose(x[:, :32], torch.ones(pos.shape[0], 32, dtype=torch.float64))
    assert torch.all(x[:, 48] == 1) and torch.all(x[:, 49:] == 0)


@pytest.mark.parametrize("seed", [0, 1])
def test_backward_matches_autograd(seed, monkeypatch):
    monkeypatch.setattr(cache_ref, "ROUND", False)
    res, grid, w, pos, d, tgt = _problem(seed=seed)
    bmin, bmax = [-1, -1, -1], [1, 1, 1]
    loss, dw, dgrid = cache_ref.train_grads(grid, w, res, bmin, bmax, pos, d, tgt)
    gg, ww = grid.clone().requires_grad_(), w.clone().requires_grad_()
    x, _ = cache_ref.encode(gg, res, bmin, bmax, pos, d)
    y, _ = cache_ref.mlp_forward(ww, x)
    yy = y[:, :3]
    l = ((yy - tgt) ** 2 / (yy.detach() ** 2 + 0.01)).sum() / pos.shape[0]
    l.backward()
    assert float(loss) == pytest.approx(l.item(), rel=1e-12)
    assert torch.allclose(dw, ww.grad, rtol=1e-9, atol=1e-12)
    assert torch.allclose(dgrid, gg.grad, rtol=1e-9, atol=1e-12)
