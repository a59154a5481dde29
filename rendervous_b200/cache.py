"""Radiance cache: grid encoding + MLP trained online from the path tracer.

The network (``vrt_cache`` in include/vrt.h) runs on the tcgen05 tensor
cores with BF16 operands and FP32 accumulation; parameters, gradients and the
Adam state are FP32 tensors owned here.  There is no reference counterpart.
"""
from __future__ import annotations

import math

import torch

from . import _lib

LEVELS = 16
N_WEIGHTS = 4 * 64 * 64 + 16 * 64


def level_resolutions(n_min: int = 16, n_max: int = 128, levels: int = LEVELS) -> list:
    """Cells per axis of each level, growing geometrically from n_min to n_max."""
    b = (n_max / n_min) ** (1.0 / (levels - 1))
    return [int(math.floor(n_min * b ** l + 1e-6)) for l in range(levels)]


def grid_size(res) -> int:
    return sum((r + 1) ** 3 * 2 for r in res)


class RadianceCache:
    def __init__(self, bmin, bmax, device, n_min: int = 16, n_max: int = 128, seed: int = 0,
                 grid_init: float = 1e-4):
        self.device = torch.device(device)
        self.res = level_resolutions(n_min, n_max)
        self.bmin = [float(v) for v in torch.as_tensor(bmin).reshape(3).tolist()]
        self.bmax = [float(v) for v in torch.as_tensor(bmax).reshape(3).tolist()]
        g = torch.Generator().manual_seed(seed)
        n_grid = grid_size(self.res)
        grid = (torch.rand(n_grid, generator=g) * 2 - 1) * grid_init
        w = []
        for l in range(5):
            fan_out, fan_in = (64, 64) if l < 4 else (16, 64)
            bound = math.sqrt(6.0 / (fan_in + fan_out))
            w.append(((torch.rand(fan_out, fan_in, generator=g) * 2 - 1) * bound).reshape(-1))
        weights = torch.cat(w)
        # one flat parameter vector so one Adam launch updates everything
        self.params = torch.cat([grid, weights]).to(self.device)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.n_grid = n_grid
        self.step = 0
        self._loss = torch.zeros(1, device=self.device)

    @property
    def grid(self) -> torch.Tensor:
        return self.params[: self.n_grid]

    @property
    def weights(self) -> torch.Tensor:
        return self.params[self.n_grid:]

    def struct(self):
        ffi, lib = _lib.ffi_lib()
        c = ffi.new("vrt_cache *")
        c.grid = _lib.fptr(self.params)
        c.grid_grad = _lib.fptr(self.grads)
        c.weights = ffi.cast("float *", self.params.data_ptr() + 4 * self.n_grid)
        c.weights_grad = ffi.cast("float *", self.grads.data_ptr() + 4 * self.n_grid)
        c.levels = LEVELS
        for i, r in enumerate(self.res):
            c.res[i] = r
        for i in range(3):
            c.bmin[i] = self.bmin[i]
            c.bmax[i] = self.bmax[i]
        return c

    def infer(self, pos: torch.Tensor, dir: torch.Tensor) -> torch.Tensor:
        ffi, lib = _lib.ffi_lib()
        pos = pos.reshape(-1, 3).contiguous().float()
        dir = dir.reshape(-1, 3).contiguous().float()
        out = torch.empty(pos.shape[0], 3, device=self.device)
        _lib.check(lib.vrt_cache_infer(self.struct(), _lib.fptr(pos), _lib.fptr(dir), pos.shape[0], _lib.fptr(out),
                                       _lib.stream_handle(self.device)), "vrt_cache_infer")
        return out

    def accumulate_grad(self, pos, dir, target) -> torch.Tensor:
        """Adds the gradient of mean relative-L2 loss; returns the loss (device)."""
        ffi, lib = _lib.ffi_lib()
        pos = pos.reshape(-1, 3).contiguous().float()
        dir = dir.reshape(-1, 3).contiguous().float()
        target = target.reshape(-1, 3).contiguous().float()
        self._loss.zero_()
        _lib.check(lib.vrt_cache_train(self.struct(), _lib.fptr(pos), _lib.fptr(dir), _lib.fptr(target), pos.shape[0],
                                       _lib.fptr(self._loss), _lib.stream_handle(self.device)), "vrt_cache_train")
        return self._loss.clone()

    def train_step(self, pos, dir, target, lr: float = 1e-2, beta1: float = 0.9, beta2: float = 0.99,
                   eps: float = 1e-15) -> torch.Tensor:
        loss = self.accumulate_grad(pos, dir, target)
        self.step += 1
        ffi, lib = _lib.ffi_lib()
        _lib.check(lib.vrt_cache_adam(_lib.fptr(self.params), _lib.fptr(self.grads), _lib.fptr(self.m),
                                      _lib.fptr(self.v), self.params.numel(), lr, beta1, beta2, eps, self.step,
                                      _lib.stream_handle(self.device)), "vrt_cache_adam")
        return loss


def mlp_forward(weights: torch.Tensor, inputs: torch.Tensor) -> torch.Tensor:
    """The MLP alone on [n, 64] inputs -> [n, 16] (tensor cores)."""
    ffi, lib = _lib.ffi_lib()
    x = inputs.contiguous().float()
    out = torch.empty(x.shape[0], 16, device=x.device)
    _lib.check(lib.vrt_cache_mlp_fw(_lib.fptr(weights.contiguous()), _lib.fptr(x), x.shape[0], _lib.fptr(out),
                                    _lib.stream_handle(x.device)), "vrt_cache_mlp_fw")
    return out
