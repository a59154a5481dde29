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


class CachedRenderer:
    """Renders an NEE path-integrator field through a camera with the radiance
    cache: every path is traced without bias for its first `cut` collisions
    (next-event estimation at each) and at its (cut+1)-th collision adds
    W * cache(x, w) instead of continuing.  Each frame first trains the cache on
    `train_paths` full paths from random pixels (their first `rec` collisions
    give 2^16 samples at the defaults), then renders `spp` paths per pixel with
    it.  Training paths stop into the cache themselves at their
    (train_cut+1)-th collision (self-training; train_cut < 0 traces them to
    the end).  `render()` returns the mean of its frames.
    """

    def __init__(self, field, camera, cache: RadianceCache = None, *, cut: int = 2, train_paths: int = 1 << 14,
                 rec: int = 4, train_cut: int = 16, lr: float = 1e-2, seed: int = 0):
        field = field.cast(input_dim=6)
        if getattr(field, "FW", None) != 0:
            raise NotImplementedError("the radiance cache terminates NEE path-integrator paths")
        self.desc = field.lower()
        self.dev = self.desc.sigma.device
        self.m = self.desc.to_struct()
        self.cam, self._poses = camera.to_struct(self.dev)
        self.shape = (camera.views, camera.height, camera.width, 3)
        self.npix = camera.views * camera.height * camera.width
        bmin = self.desc.box_min.detach().float().cpu()
        bmax = self.desc.box_max.detach().float().cpu()
        self.cache = cache if cache is not None else RadianceCache(bmin, bmax, self.dev, seed=seed)
        self.cut, self.train_paths, self.rec, self.lr = int(cut), int(train_paths), int(rec), float(lr)
        self.train_cut = int(train_cut)
        self.samples = torch.empty(4, self.train_paths * self.rec, 3, device=self.dev)
        self.work = torch.empty(12 * self.train_paths, device=self.dev)
        self._queries = None
        self._seed = (int(seed) * 0x9E3779B1 + 0x1234567) & 0xFFFFFFFF
        self.frames = 0
        self.last_loss = None

    def _next_seed(self) -> int:
        self._seed = (self._seed * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        return self._seed >> 16

    def train_frame(self) -> torch.Tensor:
        ffi, lib = _lib.ffi_lib()
        vctx = _lib.context(self.dev)
        c = self.cache.struct() if self.train_cut >= 0 else ffi.NULL
        _lib.check(lib.vrt_capture_train_samples(vctx.ptr, self.m, self.cam, c, self.train_cut, self.train_paths,
                                                 self._next_seed(), self.rec, _lib.fptr(self.samples),
                                                 _lib.fptr(self.work), _lib.stream_handle(self.dev)),
                   "vrt_capture_train_samples")
        self.last_loss = self.cache.train_step(self.samples[0], self.samples[1], self.samples[2], lr=self.lr)
        return self.last_loss

    def render_frame(self, rgb: torch.Tensor, spp: int = 1) -> None:
        """Adds one spp-sample estimate into rgb [views, H, W, 3]."""
        ffi, lib = _lib.ffi_lib()
        n = self.npix * spp
        if self._queries is None or self._queries.shape[1] != n:
            self._queries = torch.empty(3, n, 3, device=self.dev)
        vctx = _lib.context(self.dev)
        stream = _lib.stream_handle(self.dev)
        _lib.check(lib.vrt_capture_prefix_fw(vctx.ptr, self.m, self.cam, spp, self._next_seed(), self.cut,
                                             _lib.fptr(rgb), _lib.fptr(self._queries), stream), "vrt_capture_prefix_fw")
        _lib.check(lib.vrt_cache_resolve(self.cache.struct(), _lib.fptr(self._queries), n, self.npix, 1.0 / spp,
                                         _lib.fptr(rgb), stream), "vrt_cache_resolve")
        self.frames += 1

    def render(self, frames: int, spp: int = 1, train: bool = True) -> torch.Tensor:
        rgb = torch.zeros(self.shape, device=self.dev)
        for _ in range(frames):
            if train:
                self.train_frame()
            self.render_frame(rgb, spp)
        return rgb / frames

    def check(self) -> None:
        """Raises if a kernel of the renderer or the cache reported a device error."""
        ffi, lib = _lib.ffi_lib()
        _lib.context(self.dev).sync()
        _lib.check(lib.vrt_cache_status(_lib.stream_handle(self.dev)), "radiance cache")
