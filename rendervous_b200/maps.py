"""The reference's map API for the volume hot path, backed by libvrt.so.

Class names, constructor signatures and sub-map IO layouts follow rendervous
``_maps.py`` (citations per class).  A map here is a ``torch.nn.Module``; the
maps on the hot path are callable on CUDA tensors and differentiable, the
others (phase, samplers, constants used as sub-maps) are descriptors that a
path integrator lowers into its ``vrt_medium`` (see ``lowering.py``).

Every call runs a CUDA kernel; there is no CPU path.  Gradients accumulate
into ``param.grad`` exactly once per backward (through autograd).
"""
from __future__ import annotations

import math
import typing

import numpy as np
import torch

from . import _lib
from .lowering import TR_MODES, lower_collision_integrator, lower_integrator, lower_transmittance_map

# ----------------------------------------------------------------- seeds --
_MANUAL_SEED: dict = {"value": None}
_SYNC_CHECKS = {"on": True}


def seed(manual_seed: typing.Optional[int] = None) -> None:
    """rendervous.seed (_internal.py:21-23): reseed torch before the next draw."""
    _MANUAL_SEED["value"] = manual_seed


def next_seed() -> int:
    """A fresh 62-bit Philox key from torch's CPU generator (the reference draws
    four int32 seeds per dispatch the same way, _internal.py:26-34)."""
    if _MANUAL_SEED["value"] is not None:
        torch.manual_seed(_MANUAL_SEED["value"])
        _MANUAL_SEED["value"] = None
    return int(torch.randint(0, 1 << 62, (1,), dtype=torch.int64).item())


def set_sync_checks(on: bool) -> None:
    """When on (default), every operator waits for its kernels and raises if a
    kernel recorded an error, matching the reference's synchronous dispatch and
    post-dispatch checks (_maps.py:1188-1208).  Turn off to pipeline calls and
    check explicitly with ``check()``."""
    _SYNC_CHECKS["on"] = bool(on)


def check(device=None) -> dict:
    """Waits for the device, raises VrtError on a recorded kernel error and
    returns (and clears) the path/vertex/step counters."""
    return _lib.context(device).sync()


def _after_call(device) -> None:
    if _SYNC_CHECKS["on"]:
        _lib.context(device).sync()


def device() -> torch.device:
    return torch.device("cuda", torch.cuda.current_device())


def vec3(x: float, y: float, z: float) -> torch.Tensor:
    return torch.tensor([x, y, z], dtype=torch.float32)


def _as_vec3(v) -> torch.Tensor:
    return torch.as_tensor(v, dtype=torch.float32).reshape(3).clone()


def parameter(p):
    """_maps.py:1032-1038: tensors become frozen Parameters; trainable ones must
    already be Parameters."""
    if p is None:
        return None
    if isinstance(p, torch.nn.Parameter):
        return p
    assert not p.requires_grad, "Tensors used as parameters can not require grads. Use Parameter instead."
    return torch.nn.Parameter(p, requires_grad=False)


# ------------------------------------------------------------------- maps --
class MapBase(torch.nn.Module):
    """MapBase (_maps.py:1211): a map R^INPUT_DIM -> R^OUTPUT_DIM."""

    def __init__(self, input_dim: typing.Optional[int] = None, output_dim: typing.Optional[int] = None):
        super().__init__()
        self.input_dim = input_dim
        self.output_dim = output_dim

    def cast(self, input_dim: typing.Optional[int] = None, output_dim: typing.Optional[int] = None):
        """Dimension check of sub-map slots (_maps.py:2957-2966)."""
        if input_dim is not None and self.input_dim is not None and self.input_dim != input_dim:
            raise AssertionError(f"{type(self).__name__} takes {self.input_dim} inputs, {input_dim} required")
        if output_dim is not None and self.output_dim is not None and self.output_dim != output_dim:
            if not (self.output_dim == 1 and output_dim > 1):  # scalar promotion
                raise AssertionError(f"{type(self).__name__} gives {self.output_dim} outputs, {output_dim} required")
        return self

    def forward(self, *args):
        raise NotImplementedError(f"{type(self).__name__} is evaluated only inside a path integrator here")

    # map algebra (_maps.py:1347-1415): the forms the lowering recognises
    def after(self, prev_map: "MapBase") -> "MapBase":
        """CompositionMap(prev_map, self): self applied to prev_map's output."""
        return CompositionMap(prev_map, self)

    def __mul__(self, other):
        return MultiplicationMap(self, other if isinstance(other, MapBase) else const[other])

    def __rmul__(self, other):
        return MultiplicationMap(self, other if isinstance(other, MapBase) else const[other])


class CompositionMap(MapBase):
    """CompositionMap (_maps.py:1804): map_b(map_a(x))."""

    def __init__(self, map_a: MapBase, map_b: MapBase):
        super().__init__(map_a.input_dim, map_b.output_dim)
        self.map_a = map_a
        self.map_b = map_b


class MultiplicationMap(MapBase):
    """MultiplicationMap (_maps.py:1918): map_a(x) * map_b(x) (a scalar side promoted)."""

    def __init__(self, map_a: MapBase, map_b: MapBase):
        dims = [d for d in (map_a.output_dim, map_b.output_dim) if d is not None]
        super().__init__(map_a.input_dim or map_b.input_dim, max(dims) if dims else None)
        self.map_a = map_a
        self.map_b = map_b


class RayDirection(MapBase):
    """RayDirection (_maps.py:3164-3185): (x, w) -> w."""

    def __init__(self):
        super().__init__(6, 3)


ray_direction = RayDirection()


class ConstantMap(MapBase):
    """ConstantMap / const[...] (_maps.py:4799, include/maps/constant.h)."""

    def __init__(self, value: torch.Tensor, input_dim: typing.Optional[int] = None):
        value = torch.as_tensor(value, dtype=torch.float32).reshape(-1)
        super().__init__(input_dim, value.numel())
        self.value = value

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        return self.value.to(x.device).expand(*x.shape[:-1], self.output_dim).clone()


class ParametricMap:
    """map[args] factory (_maps.py:4755-4778)."""

    def __init__(self, factory):
        self.factory = factory

    def __getitem__(self, item):
        if not isinstance(item, tuple):
            item = (item,)
        kwargs = {}
        if item and isinstance(item[-1], dict):
            kwargs = item[-1]
            item = item[:-1]
        return self.factory(*item, **kwargs)


def _const_factory(*args, input_dim: typing.Optional[int] = None):
    if len(args) == 1 and isinstance(args[0], torch.Tensor):
        return ConstantMap(args[0], input_dim=input_dim)
    if len(args) == 1 and isinstance(args[0], (list, tuple)):
        args = tuple(args[0])
    return ConstantMap(torch.tensor([float(a) for a in args], dtype=torch.float32), input_dim=input_dim)


const = ParametricMap(_const_factory)
ZERO = None  # set below
ONE = None


class _Grid3DFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, grid, bmin, bmax):
        ffi, lib = _lib.ffi_lib()
        xs = x.detach().reshape(-1, 3).contiguous()
        out = torch.empty(xs.shape[0], grid.shape[-1], device=x.device, dtype=torch.float32)
        g = ffi.new("vrt_grid *")
        from .lowering import _fill_grid
        _fill_grid(g, grid.detach(), None)
        b0 = ffi.new("float[3]", bmin.tolist())
        ib = ffi.new("float[3]", (1.0 / (bmax - bmin)).tolist())
        _lib.check(lib.vrt_grid3d_fw(g, b0, ib, _lib.fptr(xs), xs.shape[0], _lib.fptr(out),
                                     _lib.stream_handle(x.device)), "vrt_grid3d_fw")
        _after_call(x.device)
        ctx.save_for_backward(xs, grid)
        ctx.box = (bmin, bmax)
        ctx.xshape = x.shape
        return out.reshape(*x.shape[:-1], grid.shape[-1])

    @staticmethod
    def backward(ctx, dout):
        xs, grid = ctx.saved_tensors
        gg = None
        if ctx.needs_input_grad[1]:
            ffi, lib = _lib.ffi_lib()
            gg = torch.zeros_like(grid)
            g = ffi.new("vrt_grid *")
            from .lowering import _fill_grid
            _fill_grid(g, grid.detach(), gg)
            bmin, bmax = ctx.box
            b0 = ffi.new("float[3]", bmin.tolist())
            ib = ffi.new("float[3]", (1.0 / (bmax - bmin)).tolist())
            d = dout.reshape(-1, grid.shape[-1]).contiguous().float()
            _lib.check(lib.vrt_grid3d_bw(g, b0, ib, _lib.fptr(xs), _lib.fptr(d), xs.shape[0],
                                         _lib.stream_handle(xs.device)), "vrt_grid3d_bw")
            _after_call(xs.device)
        dx = torch.zeros(ctx.xshape, device=xs.device) if ctx.needs_input_grad[0] else None
        return dx, gg, None, None


class Grid3D(MapBase):
    """Grid3D (_maps.py:2319-2365, include/maps/grid3d.h): node-centred trilinear
    lookup of a [D,H,W,C] grid over the box [bmin, bmax], zero outside."""

    def __init__(self, grid: torch.Tensor, bmin=vec3(-1.0, -1.0, -1.0), bmax=vec3(1.0, 1.0, 1.0)):
        assert len(grid.shape) == 4
        super().__init__(3, grid.shape[-1])
        self.grid = parameter(grid)
        self.bmin = _as_vec3(bmin)
        self.bmax = _as_vec3(bmax)
        self.inv_bsize = 1.0 / (self.bmax - self.bmin)
        self.width = grid.shape[2]
        self.height = grid.shape[1]
        self.depth = grid.shape[0]

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        return _Grid3DFn.apply(x, self.grid, self.bmin, self.bmax)

    def get_maximum(self) -> float:
        return self.grid.max().item()

    def support_maximum_query(self) -> bool:
        return True


class _RayBoxFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rays, bmin, bmax):
        ffi, lib = _lib.ffi_lib()
        r = rays.detach().reshape(-1, 6).contiguous()
        out = torch.empty(r.shape[0], 2, device=rays.device, dtype=torch.float32)
        b0 = ffi.new("float[3]", bmin.tolist())
        b1 = ffi.new("float[3]", bmax.tolist())
        _lib.check(lib.vrt_ray_box(_lib.fptr(r), r.shape[0], b0, b1, _lib.fptr(out), _lib.stream_handle(rays.device)),
                   "vrt_ray_box")
        _after_call(rays.device)
        return out.reshape(*rays.shape[:-1], 2)

    @staticmethod
    def backward(ctx, d):
        return None, None, None


class RayBoxIntersection(MapBase):
    """RayBoxIntersection (_maps.py:4128-4154): (x,w) -> (tMin, tMax)."""

    def __init__(self, box_min, box_max, **kwargs):
        super().__init__(6, 2)
        self.box_min = _as_vec3(box_min)
        self.box_max = _as_vec3(box_max)

    def forward(self, rays: torch.Tensor) -> torch.Tensor:
        return _RayBoxFn.apply(rays, self.box_min, self.box_max)


ray_box_intersection = ParametricMap(RayBoxIntersection)


def normalized_box(s) -> typing.Tuple[torch.Tensor, torch.Tensor]:
    """_maps.py:4780-4788: box of half-extent (shape-1)*0.5/max_dim."""
    shape = s.shape if isinstance(s, torch.Tensor) else s
    max_dim = max(shape[0], shape[1], shape[2]) - 1
    b_max = vec3(shape[2] - 1, shape[1] - 1, shape[0] - 1) * 0.5 / max_dim
    return -b_max, b_max


class MajorantGrid(MapBase):
    """Majorant map (x,w) -> (majorant, distance) backed by a grid of brick^3-cell
    bricks over a Grid3D sigma (no reference counterpart; the reference's
    majorant is the constant of _objects.py:96-101).  With ``auto_update`` the
    bounds are rebuilt from the current sigma on every lowering, so they stay
    valid while sigma is optimised."""

    def __init__(self, sigma: Grid3D, brick: int = 8, auto_update: bool = True):
        super().__init__(6, 2)
        if not isinstance(sigma, Grid3D):
            raise TypeError("MajorantGrid needs a Grid3D sigma")
        self.sigma = sigma
        self.brick = int(brick)
        self.auto_update = auto_update
        self._tensor = None

    def update(self) -> torch.Tensor:
        ffi, lib = _lib.ffi_lib()
        grid = self.sigma.grid.detach()
        g = ffi.new("vrt_grid *")
        from .lowering import _fill_grid
        _fill_grid(g, grid, None)
        dims = ffi.new("int32_t[3]")
        _lib.check(lib.vrt_majorant_build(g, self.brick, ffi.NULL, dims, _lib.stream_handle(grid.device)))
        if self._tensor is None or tuple(self._tensor.shape) != (dims[2], dims[1], dims[0]):
            self._tensor = torch.empty(dims[2], dims[1], dims[0], device=grid.device, dtype=torch.float32)
        _lib.check(lib.vrt_majorant_build(g, self.brick, _lib.fptr(self._tensor), dims, _lib.stream_handle(grid.device)),
                   "vrt_majorant_build")
        _after_call(grid.device)
        return self._tensor

    def tensor(self) -> torch.Tensor:
        if self._tensor is None or self.auto_update:
            return self.update()
        return self._tensor


class GridMaximumMajorant(ConstantMap):
    """The reference's medium_majorant_grid builder (_objects.py:96-101): a constant
    [max sigma, 1e6] that is recomputed from the grid whenever it is lowered."""

    def __init__(self, sigma: Grid3D):
        super().__init__(torch.tensor([0.0, 1e6]), input_dim=6)
        self.sigma = sigma

    @property
    def value(self):
        return torch.tensor([self.sigma.get_maximum(), 1000000.0], dtype=torch.float32)

    @value.setter
    def value(self, v):
        pass


# ---------------------------------------------------- image environments --
class Image2D(MapBase):
    """Image2D (_maps.py:2288-2316, include/maps/image2d.h): bilinear lookup of an
    [H, W, C] image over the box [bmin, bmax] (clamped to the border)."""

    def __init__(self, grid: torch.Tensor, bmin=None, bmax=None):
        assert len(grid.shape) == 3
        super().__init__(2, grid.shape[-1])
        self.grid = parameter(grid)
        self.bmin = torch.tensor([-1.0, -1.0]) if bmin is None else torch.as_tensor(bmin, dtype=torch.float32)
        bmax = torch.tensor([1.0, 1.0]) if bmax is None else torch.as_tensor(bmax, dtype=torch.float32)
        self.inv_bsize = 1.0 / (bmax - self.bmin)


class XRProjection(MapBase):
    """XRProjection (_maps.py:2405-2425, include/maps/xr_projection.h): a direction
    (or the direction of a ray) to equirectangular coordinates in [-1, 1]^2."""

    def __init__(self, ray_input: bool = False):
        super().__init__(6 if ray_input else 3, 2)
        self.ray_input = ray_input


xr_projection = XRProjection(False)


class XRQuadtreeRandomDirection(MapBase):
    """XRQuadtreeRandomDirection (_maps.py:2494-2549): [w, weight] with w drawn
    from a probability quadtree over an equirectangular image (see
    create_density_quadtree) and weight = pixel solid angle / probability."""

    def __init__(self, input_dim: int, densities: torch.Tensor, levels: int):
        super().__init__(input_dim, 4)
        self.densities = densities
        self.levels = int(levels)


def create_density_quadtree(densities: torch.Tensor) -> torch.Tensor:
    """_functions.py:509-530: the node probabilities of a square power-of-two
    [R, R, 1] density image, coarsest level first (2x2, 4x4, ..., RxR), each
    level in Morton order (x in the low bit), each node the sum of its four
    children -- so node k's children sit at 4k+1 .. 4k+4 counted from the
    start (the layout XRQuadtreeRandomDirection walks)."""
    R = densities.shape[0]
    assert densities.dim() == 3 and densities.shape[1] == R and densities.shape[2] == 1
    assert R >= 2 and (R & (R - 1)) == 0, "resolution must be a power of two"
    d = densities[..., 0].to(torch.float32)
    levels = []
    while d.shape[0] > 1:
        levels.append(_morton_flatten(d))
        d = d.reshape(d.shape[0] // 2, 2, d.shape[1] // 2, 2).sum(dim=(1, 3))
    levels.reverse()
    return torch.cat(levels).reshape(-1, 1)


def _morton_flatten(img: torch.Tensor) -> torch.Tensor:
    """img[y, x] in Morton order of (x, y) with x in the low bit."""
    n = img.shape[0]
    bits = n.bit_length() - 1
    ys, xs = torch.meshgrid(torch.arange(n), torch.arange(n), indexing="ij")
    code = torch.zeros_like(xs)
    for b in range(bits):
        code |= ((xs >> b) & 1) << (2 * b)
        code |= ((ys >> b) & 1) << (2 * b + 1)
    out = torch.empty(n * n, dtype=img.dtype, device=img.device)
    out[code.reshape(-1).to(img.device)] = img.reshape(-1)
    return out


def environment_quadtree(env_image: torch.Tensor, levels: int = 10) -> torch.Tensor:
    """The sampling quadtree of an equirectangular environment image
    (_objects.py:180-193): luminance resampled to 2^levels square, each row
    weighted by its solid angle, normalised, then create_density_quadtree."""
    res = 1 << int(levels)
    lum = env_image.detach().to(torch.float32).sum(-1)[None, None]
    img = torch.nn.functional.interpolate(lum, size=(res, res), mode="bilinear", align_corners=False)[0, 0]
    py = torch.arange(res, dtype=torch.float64, device=img.device)
    wrow = (torch.cos(py * math.pi / res) - torch.cos((py + 1) * math.pi / res)).to(torch.float32)
    img = img.clamp_min(0.0) * wrow[:, None]
    img = img / img.sum().clamp_min(1e-8)
    return create_density_quadtree(img[..., None])


# ----------------------------------------------------- phase and sampling --
class HGPhase(MapBase):
    """HGPhase (_maps.py:4436-4460): evaluates 0.8*HG(g) + 0.2*HG(g/5)."""

    def __init__(self, phase_g: MapBase):
        super().__init__(9, 1)
        self.phase_g = phase_g.cast(3, 1)


class VHGPhaseSampler(MapBase):
    """VHGPhaseSampler (_maps.py:4463-4484): draws HG(g/5) with p=0.8, else HG(g); weight 1."""

    def __init__(self, phase_g: MapBase):
        super().__init__(6, 4)
        self.phase_g = phase_g.cast(3, 1)


class HGDirectionSampler(MapBase):
    """HGDirectionSampler (_maps.py:4487-4507).  Its output layout [w, 1/p] does not
    match the [rho, w] phase-sampler slot, so integrators reject it (as the
    reference's casts would mis-read it)."""

    def __init__(self, phase_g: MapBase):
        super().__init__(6, 4)
        self.phase_g = phase_g


class HenyeyGreensteinPhase(MapBase):
    """Pure Henyey-Greenstein phase (no reference counterpart: the reference's
    HGPhase evaluates a mixture that its sampler does not draw)."""

    def __init__(self, phase_g: MapBase):
        super().__init__(9, 1)
        self.phase_g = phase_g.cast(3, 1)


class HenyeyGreensteinPhaseSampler(MapBase):
    """Draws exactly HG(g) with weight 1; pairs with HenyeyGreensteinPhase."""

    def __init__(self, phase_g: MapBase):
        super().__init__(6, 4)
        self.phase_g = phase_g.cast(3, 1)


class UniformDirectionSampler(MapBase):
    """UniformDirectionSampler (_maps.py:2482-2491): uniform sphere direction, weight 4pi."""

    def __init__(self, input_dim: int):
        super().__init__(input_dim, 4)


class _functionsampler(MapBase):
    """_functionsampler (_maps.py:2552-2585): [f(w) * weight, w]."""

    def __init__(self, point_sampler: MapBase, function_map: MapBase):
        assert point_sampler.output_dim - 1 == function_map.input_dim or function_map.input_dim is None
        super().__init__(point_sampler.input_dim, point_sampler.output_dim - 1 + function_map.output_dim)
        self.point_sampler = point_sampler
        self.function_map = function_map


class DirectionalLight(torch.nn.Module):
    """A directional emitter sampled by next-event estimation at every real
    collision (no reference counterpart).  ``direction`` points towards the light."""

    def __init__(self, direction, radiance):
        super().__init__()
        d = _as_vec3(direction)
        self.direction = d / d.norm()
        r = torch.as_tensor(radiance, dtype=torch.float32).reshape(-1)
        self.radiance = (r.expand(3) if r.numel() == 1 else r.reshape(3)).clone()


# ---------------------------------------------------------- transmittance --
class _TransmittanceFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rays, sigma_grid, desc, mode, seed):
        ffi, lib = _lib.ffi_lib()
        r = rays.detach().reshape(-1, 6).contiguous()
        T = torch.empty(r.shape[0], device=rays.device, dtype=torch.float32)
        m = desc.to_struct()
        vctx = _lib.context(rays.device)
        _lib.check(lib.vrt_transmittance_fw(vctx.ptr, m, mode, _lib.fptr(r), r.shape[0], seed, _lib.fptr(T),
                                            _lib.stream_handle(rays.device)), "vrt_transmittance_fw")
        _after_call(rays.device)
        ctx.save_for_backward(r)
        ctx.desc, ctx.mode, ctx.seed, ctx.rshape = desc, mode, seed, rays.shape
        return T.reshape(*rays.shape[:-1], 1)

    @staticmethod
    def backward(ctx, dT):
        r, = ctx.saved_tensors
        gs = None
        if ctx.needs_input_grad[1]:
            ffi, lib = _lib.ffi_lib()
            gs = torch.zeros_like(ctx.desc.sigma)
            m = ctx.desc.to_struct(sigma_grad=gs)
            d = dT.reshape(-1).contiguous().float()
            vctx = _lib.context(r.device)
            _lib.check(lib.vrt_transmittance_bw(vctx.ptr, m, ctx.mode, _lib.fptr(r), r.shape[0], ctx.seed, _lib.fptr(d),
                                                _lib.stream_handle(r.device)), "vrt_transmittance_bw")
            _after_call(r.device)
        dr = torch.zeros(ctx.rshape, device=r.device) if ctx.needs_input_grad[0] else None
        return dr, gs, None, None, None


class _TransmittanceMap(MapBase):
    def __init__(self):
        super().__init__(6, 1)

    def _mode(self) -> int:
        raise NotImplementedError

    def forward(self, rays: torch.Tensor, seed: typing.Optional[int] = None) -> torch.Tensor:
        desc = lower_transmittance_map(self)
        return _TransmittanceFn.apply(rays, desc.sigma, desc, self._mode(), next_seed() if seed is None else seed)


class GridDDATransmittance(_TransmittanceMap):
    """GridDDATransmittance (_maps.py:2640-2667, include/vr_transmittance_DDA.h).
    ``exact=False`` keeps the reference's per-cell midpoint rule; ``exact=True``
    integrates the trilinear field exactly per cell."""

    def __init__(self, grid: Grid3D, boundary: MapBase, exact: bool = False):
        super().__init__()
        self.boundary = boundary
        self.exact = bool(exact)
        self.grid_model = None
        self.update_grid(grid)

    def update_grid(self, grid: typing.Optional[Grid3D] = None):
        if grid is None:
            assert self.grid_model is not None
            grid = self.grid_model
        else:
            self.grid_model = grid
        self.grid = grid.grid
        self.box_min = grid.bmin.clone()
        self.box_max = grid.bmax.clone()

    def _mode(self) -> int:
        return TR_MODES["dda_exact" if self.exact else "dda"]


class _GridTrackingTransmittance(_TransmittanceMap):
    """Shared constructor of GridRatiotrackingTransmittance and
    GridDeltatrackingTransmittance (_maps.py:2588-2637): tracking over the
    grid's own cells with per-cell majorant and minorant, no majorant map.
    Forward only, as in the reference (its maps define no backward): the
    gradient through them is zero."""

    def __init__(self, grid: Grid3D, boundary: MapBase):
        super().__init__()
        self.grid_model = grid
        self.grid = grid.grid
        self.box_min = grid.bmin.clone()
        self.box_max = grid.bmax.clone()
        self.boundary = boundary.cast(6, 2)

    def update_grid(self, grid: typing.Optional[Grid3D] = None):
        if grid is None:
            assert self.grid_model is not None
            grid = self.grid_model
        else:
            self.grid_model = grid
        self.grid = grid.grid
        self.box_min = grid.bmin.clone()
        self.box_max = grid.bmax.clone()


class GridRatiotrackingTransmittance(_GridTrackingTransmittance):
    """GridRatiotrackingTransmittance (_maps.py:2588-2614, include/vr_transmittance_GRT.h)."""

    def _mode(self) -> int:
        return TR_MODES["grt"]


class GridDeltatrackingTransmittance(_GridTrackingTransmittance):
    """GridDeltatrackingTransmittance (_maps.py:2617-2637, include/vr_transmittance_GDT.h)."""

    def _mode(self) -> int:
        return TR_MODES["gdt"]


class RatiotrackingTransmittance(_TransmittanceMap):
    """RatiotrackingTransmittance (_maps.py:2670-2682, include/vr_transmittance_RT.h)."""

    def __init__(self, sigma: MapBase, boundary: MapBase, majorant: MapBase):
        super().__init__()
        self.sigma = sigma.cast(3, 1)
        self.boundary = boundary.cast(6, 2)
        self.majorant = majorant.cast(6, 2)

    def _mode(self) -> int:
        return TR_MODES["rt"]


class DeltatrackingTransmittance(_TransmittanceMap):
    """DeltatrackingTransmittance (_maps.py:2685-2697, include/vr_transmittance_DT.h)."""

    def __init__(self, sigma: MapBase, boundary: MapBase, majorant: MapBase):
        super().__init__()
        self.sigma = sigma
        self.boundary = boundary
        self.majorant = majorant

    def _mode(self) -> int:
        return TR_MODES["dt"]


# -------------------------------------------------------- path integrators --
class _RadianceFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rays, sigma_grid, albedo_grid, emission_grid, integrator, desc, fw_mode, bw_mode, seed):
        ffi, lib = _lib.ffi_lib()
        r = rays.detach().reshape(-1, 6).contiguous()
        R = torch.empty(r.shape[0], 3, device=rays.device, dtype=torch.float32)
        m = desc.to_struct()
        vctx = _lib.context(rays.device)
        _lib.check(lib.vrt_radiance_fw(vctx.ptr, m, fw_mode, _lib.fptr(r), r.shape[0], seed, _lib.fptr(R),
                                       _lib.stream_handle(rays.device)), "vrt_radiance_fw")
        _after_call(rays.device)
        ctx.save_for_backward(r)
        ctx.desc, ctx.bw_mode, ctx.seed, ctx.rshape = desc, bw_mode, seed, rays.shape
        return R.reshape(*rays.shape[:-1], 3)

    @staticmethod
    def backward(ctx, dR):
        r, = ctx.saved_tensors
        desc = ctx.desc
        if ctx.bw_mode is None:
            raise NotImplementedError("this integrator's adjoint is not available")
        gs = torch.zeros_like(desc.sigma) if ctx.needs_input_grad[1] else None
        ga = torch.zeros_like(desc.albedo_grid) if (ctx.needs_input_grad[2] and desc.albedo_grid is not None) else None
        ge = (torch.zeros_like(desc.emission_grid)
              if (ctx.needs_input_grad[3] and desc.emission_grid is not None) else None)
        if gs is not None or ga is not None or ge is not None:
            ffi, lib = _lib.ffi_lib()
            m = desc.to_struct(sigma_grad=gs, albedo_grad=ga, emission_grad=ge)
            d = dR.reshape(-1, 3).contiguous().float()
            vctx = _lib.context(r.device)
            _lib.check(lib.vrt_radiance_bw(vctx.ptr, m, ctx.bw_mode, _lib.fptr(r), r.shape[0], ctx.seed, _lib.fptr(d),
                                           _lib.stream_handle(r.device)), "vrt_radiance_bw")
            _after_call(r.device)
        dr = torch.zeros(ctx.rshape, device=r.device) if ctx.needs_input_grad[0] else None
        return dr, gs, ga, ge, None, None, None, None, None


class _PathIntegrator(MapBase):
    FW = 0       # VRT_PI_*
    BW = None    # VRT_BW_* or None

    def __init__(self, **subs):
        super().__init__(6, 3)
        self.max_bounces = int(subs.pop("max_bounces", 0) or 0)
        self.directional_light = subs.pop("directional_light", None)
        self.ds_compat = bool(subs.pop("ds_compat", False))
        for k, v in subs.items():
            setattr(self, k, v)

    def lower(self):
        return lower_integrator(self)

    def grid_tensors(self):
        """(sigma, albedo, emission) grid parameters the adjoint may write (None where constant)."""
        sg = self.sigma.grid
        ag = self.scattering_albedo.grid if isinstance(self.scattering_albedo, Grid3D) else None
        return sg, ag, None

    def forward(self, rays: torch.Tensor, seed: typing.Optional[int] = None) -> torch.Tensor:
        desc = self.lower()
        sg, ag, eg = self.grid_tensors()
        return _RadianceFn.apply(rays, sg, ag, eg, self, desc, self.FW, self.BW, next_seed() if seed is None else seed)


def _nee_subs(sigma, scattering_albedo, emission, environment, environment_sampler, phase, phase_sampler, boundary,
              majorant, transmittance):
    return dict(
        sigma=sigma.cast(3, 1), scattering_albedo=scattering_albedo.cast(3, 3), emission=emission.cast(6, 3),
        environment=environment.cast(3, 3), environment_sampler=environment_sampler.cast(6, 6),
        phase=phase.cast(9, 1), phase_sampler=phase_sampler.cast(6, 4), boundary=boundary.cast(6, 2),
        majorant=majorant.cast(6, 2), transmittance=transmittance.cast(6, 1))


class DeltatrackingPathIntegrator(_PathIntegrator):
    """DeltatrackingPathIntegrator (_maps.py:2886-2921): include/vr_path_integrator_DT.h fw and bw."""
    FW, BW = 1, 1

    def __init__(self, sigma, scattering_albedo, emission, environment, phase_sampler, boundary, majorant,
                 ds_epsilon: float, **ext):
        super().__init__(sigma=sigma, scattering_albedo=scattering_albedo, emission=emission,
                         environment=environment, phase_sampler=phase_sampler, boundary=boundary,
                         majorant=majorant, ds_epsilon=ds_epsilon, **ext)


class DeltatrackingNEEPathIntegrator(_PathIntegrator):
    """DeltatrackingNEEPathIntegrator (_maps.py:2924-2978): NEE forward
    (vr_path_integrator_NEE.h), defensive-sampling replay adjoint (vr_path_integrator_NEE_DS.h)."""
    FW, BW = 0, 0

    def __init__(self, sigma, scattering_albedo, emission, environment, environment_sampler, phase, phase_sampler,
                 boundary, majorant, transmittance, ds_epsilon: float, **ext):
        super().__init__(**_nee_subs(sigma, scattering_albedo, emission, environment, environment_sampler, phase,
                                     phase_sampler, boundary, majorant, transmittance), ds_epsilon=ds_epsilon, **ext)


class DRTPathIntegrator(_PathIntegrator):
    """DRTPathIntegrator (_maps.py:2981-3022): NEE forward, differential ratio
    tracking adjoint (vr_path_integrator_NEE_DRT.h)."""
    FW, BW = 0, 2

    def __init__(self, sigma, scattering_albedo, emission, environment, environment_sampler, phase, phase_sampler,
                 boundary, majorant, transmittance, **ext):
        super().__init__(**_nee_subs(sigma, scattering_albedo, emission, environment, environment_sampler, phase,
                                     phase_sampler, boundary, majorant, transmittance), ds_epsilon=0.0, **ext)


class DRTQPathIntegrator(DRTPathIntegrator):
    """DRTQPathIntegrator (_maps.py:3025-3066): NEE forward; differential ratio
    tracking adjoint with a scatter-gradient term on every path segment
    (vr_path_integrator_NEE_DRTQ.h)."""
    BW = 3


class DRTDSPathIntegrator(_PathIntegrator):
    """DRTDSPathIntegrator (_maps.py:3070-3114): NEE forward; differential ratio
    tracking adjoint whose reservoir term samples a defensive collision position
    (vr_path_integrator_NEE_DRTDS.h)."""
    FW, BW = 0, 4

    def __init__(self, sigma, scattering_albedo, emission, environment, environment_sampler, phase, phase_sampler,
                 boundary, majorant, transmittance, ds_epsilon: float, **ext):
        super().__init__(**_nee_subs(sigma, scattering_albedo, emission, environment, environment_sampler, phase,
                                     phase_sampler, boundary, majorant, transmittance), ds_epsilon=ds_epsilon, **ext)


class SPSPathIntegrator(DRTPathIntegrator):
    """SPSPathIntegrator (_maps.py:3118-3159): NEE forward; singular-path sampling
    adjoint with MIS between collision and uniform segment vertices
    (vr_path_integrator_NEE_SPS.h)."""
    BW = 5


# ---------------------------------------------------- collision integrators --
class _CollisionSampleFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rays, sigma_grid, desc, seed):
        ffi, lib = _lib.ffi_lib()
        r = rays.detach().reshape(-1, 6).contiguous()
        out = torch.empty(r.shape[0], 3, device=rays.device, dtype=torch.float32)
        _lib.check(lib.vrt_collision_sample_fw(_lib.context(rays.device).ptr, desc.to_struct(), _lib.fptr(r),
                                               r.shape[0], seed, _lib.fptr(out), _lib.stream_handle(rays.device)),
                   "vrt_collision_sample_fw")
        _after_call(rays.device)
        ctx.save_for_backward(r)
        ctx.desc, ctx.seed, ctx.rshape = desc, seed, rays.shape
        return out.reshape(*rays.shape[:-1], 3)

    @staticmethod
    def backward(ctx, dout):
        r, = ctx.saved_tensors
        gs = None
        if ctx.needs_input_grad[1]:
            ffi, lib = _lib.ffi_lib()
            gs = torch.zeros_like(ctx.desc.sigma)
            d = dout.reshape(-1, 3).contiguous().float()
            _lib.check(lib.vrt_collision_sample_bw(_lib.context(r.device).ptr, ctx.desc.to_struct(sigma_grad=gs),
                                                   _lib.fptr(r), r.shape[0], ctx.seed, _lib.fptr(d),
                                                   _lib.stream_handle(r.device)), "vrt_collision_sample_bw")
            _after_call(r.device)
        dr = torch.zeros(ctx.rshape, device=r.device) if ctx.needs_input_grad[0] else None
        return dr, gs, None, None


class DeltatrackingCollisionSampler(MapBase):
    """DeltatrackingCollisionSampler (_maps.py:2714-2727, include/vr_collision_sampler_DT.h):
    (x, w) -> (C, t, T): a delta-tracking collision (C = 1, T = 0) at distance t,
    or none (C = 0, T = 1, t at the exit).  Backward: the defensively sampled
    adjoint of dL/dC and dL/dT (ds_epsilon); dL/dt is not propagated."""

    def __init__(self, sigma: MapBase, boundary: MapBase, majorant: MapBase, ds_epsilon: float):
        super().__init__(6, 3)
        self.sigma = sigma
        self.boundary = boundary
        self.majorant = majorant
        self.ds_epsilon = float(ds_epsilon)

    def lower(self):
        from .lowering import MediumDesc, lower_boundary, lower_majorant, lower_sigma
        kw: dict = {}
        lower_sigma(self.sigma, kw)
        lower_boundary(self.boundary, kw)
        lower_majorant(self.majorant, self.sigma, kw)
        kw["ds_epsilon"] = self.ds_epsilon
        return MediumDesc(**kw)

    def forward(self, rays: torch.Tensor, seed: typing.Optional[int] = None) -> torch.Tensor:
        desc = self.lower()
        return _CollisionSampleFn.apply(rays, desc.sigma, desc, next_seed() if seed is None else seed)


class MCScatteredRadiance(MapBase):
    """MCScatteredRadiance (_maps.py:2730-2743, include/maps/scattered_radiance_mc.h):
    exitance sa(x) * rho * radiance(x, wo), (rho, wo) from the phase sampler;
    an exitance radiance of the collision integrators (radiance =
    transmittance * environment.after(ray_direction))."""

    def __init__(self, scattering_albedo: MapBase, phase_sampler: MapBase, radiance: MapBase):
        super().__init__(6, 3)
        self.scattering_albedo = scattering_albedo
        self.phase_sampler = phase_sampler
        self.radiance = radiance


class MCScatteredEmittedRadiance(MapBase):
    """MCScatteredEmittedRadiance (_maps.py:2746-2760, include/maps/scattered_emitted_radiance_mc.h):
    MCScatteredRadiance plus (1 - sa) * emission(x)."""

    def __init__(self, scattering_albedo: MapBase, emission: MapBase, phase_sampler: MapBase, radiance: MapBase):
        super().__init__(6, 3)
        self.scattering_albedo = scattering_albedo
        self.emission = emission
        self.phase_sampler = phase_sampler
        self.radiance = radiance


class _CollisionIntegrator(_PathIntegrator):
    def lower(self):
        return lower_collision_integrator(self)

    def _sigma_grid3d(self) -> Grid3D:
        raise NotImplementedError

    def grid_tensors(self):
        ex = self.exitance_radiance
        ag = eg = None
        if isinstance(ex, (MCScatteredRadiance, MCScatteredEmittedRadiance)) and \
                isinstance(ex.scattering_albedo, Grid3D):
            ag = ex.scattering_albedo.grid
        em = ex.emission if isinstance(ex, MCScatteredEmittedRadiance) else ex
        if isinstance(em, Grid3D):
            eg = em.grid
        return self._sigma_grid3d().grid, ag, eg


class MCCollisionIntegrator(_CollisionIntegrator):
    """MCCollisionIntegrator (_maps.py:2792-2808, include/maps/collision_integrator_mc.h):
    C * exitance_radiance(x_t, -w) + T * environment(w) from one collision sample."""
    FW, BW = 2, 6

    def __init__(self, collision_sampler: MapBase, exitance_radiance: MapBase, environment: MapBase):
        super().__init__(collision_sampler=collision_sampler, exitance_radiance=exitance_radiance,
                         environment=environment)

    def _sigma_grid3d(self) -> Grid3D:
        return self.collision_sampler.sigma


class GridDDACollisionIntegrator(_CollisionIntegrator):
    """GridDDACollisionIntegrator (_maps.py:2811-2852, include/vr_collision_integrator_DDA.h):
    emission-absorption along the grid's DDA walk, one random point per cell."""
    FW, BW = 3, 7

    def __init__(self, sigma_grid: Grid3D, exitance_radiance: MapBase, environment: MapBase, boundary: MapBase):
        super().__init__(sigma_grid=sigma_grid, exitance_radiance=exitance_radiance, environment=environment,
                         boundary=boundary)
        self.grid = sigma_grid.grid
        self.box_min = sigma_grid.bmin.clone()
        self.box_max = sigma_grid.bmax.clone()

    def _sigma_grid3d(self) -> Grid3D:
        return self.sigma_grid

    def update_grid(self, grid: typing.Optional[Grid3D] = None):
        if grid is not None:
            self.sigma_grid = grid
        self.grid = self.sigma_grid.grid
        self.box_min = self.sigma_grid.bmin.clone()
        self.box_max = self.sigma_grid.bmax.clone()


# ------------------------------------------------------------------ sensors --
class _CaptureFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sigma_grid, albedo_grid, emission_grid, camera, field, desc, fw_samples, bw_samples, seed,
                sensors):
        ffi, lib = _lib.ffi_lib()
        dev = sigma_grid.device
        if sensors is None:
            out = torch.empty(camera.views, camera.height, camera.width, 3, device=dev, dtype=torch.float32)
        else:
            out = torch.empty(*sensors.shape[:-1], 3, device=dev, dtype=torch.float32)
        m = desc.to_struct()
        cam, keep = camera.to_struct(dev, sensors)
        vctx = _lib.context(dev)
        _lib.check(lib.vrt_capture_fw(vctx.ptr, m, field.FW, cam, fw_samples, seed, _lib.fptr(out),
                                      _lib.stream_handle(dev)), "vrt_capture_fw")
        _after_call(dev)
        ctx.desc, ctx.camera, ctx.field, ctx.bw_samples, ctx.seed = desc, camera, field, bw_samples, seed
        ctx.sensors = sensors
        return out

    @staticmethod
    def backward(ctx, dI):
        desc = ctx.desc
        if ctx.field.BW is None:
            raise NotImplementedError(f"{type(ctx.field).__name__} has no adjoint here yet")
        gs = torch.zeros_like(desc.sigma) if ctx.needs_input_grad[0] else None
        ga = torch.zeros_like(desc.albedo_grid) if (ctx.needs_input_grad[1] and desc.albedo_grid is not None) else None
        ge = (torch.zeros_like(desc.emission_grid)
              if (ctx.needs_input_grad[2] and desc.emission_grid is not None) else None)
        if gs is not None or ga is not None or ge is not None:
            ffi, lib = _lib.ffi_lib()
            dev = desc.sigma.device
            m = desc.to_struct(sigma_grad=gs, albedo_grad=ga, emission_grad=ge)
            cam, keep = ctx.camera.to_struct(dev, ctx.sensors)
            d = dI.contiguous().float()
            vctx = _lib.context(dev)
            _lib.check(lib.vrt_capture_bw(vctx.ptr, m, ctx.field.BW, cam, ctx.bw_samples, ctx.seed, _lib.fptr(d),
                                          _lib.stream_handle(dev)), "vrt_capture_bw")
            _after_call(dev)
        return gs, ga, ge, None, None, None, None, None, None, None


class PerspectiveCameraSensor(MapBase):
    """PerspectiveCameraSensor (_maps.py:1765-1802, include/maps/sensor_perspective_camera.h)."""

    def __init__(self, width: int, height: int, poses: torch.Tensor, *, fov: float = np.pi / 4, jittered: bool = False):
        super().__init__(3, 6)
        self.poses = poses
        self.fov = float(fov)
        self.znear = 0.001
        self.width = int(width)
        self.height = int(height)
        self.views = int(poses.shape[0])
        self.generation_mode = 0 if not jittered else 1

    def to_struct(self, dev, sensors: typing.Optional[torch.Tensor] = None):
        """The vrt_camera of this sensor, over every pixel or over a sensors
        batch (an int64 [n, 3] tensor of (view, row, col) on `dev`)."""
        ffi, _ = _lib.ffi_lib()
        poses = self.poses.detach().to(device=dev, dtype=torch.float32).reshape(-1, 9).contiguous()
        c = ffi.new("vrt_camera *")
        c.poses = _lib.fptr(poses)
        c.views, c.height, c.width = poses.shape[0], self.height, self.width
        c.fov, c.znear = self.fov, self.znear
        c.jittered = self.generation_mode
        if sensors is not None:
            c.sensors = ffi.cast("int64_t *", sensors.data_ptr())
            c.n_sensors = sensors.numel() // 3
        return c, (poses, sensors)

    @property
    def index_shape(self) -> typing.Tuple[int, int, int]:
        """Sensor index ranges (views, height, width) (SensorsBase.index_shape, _maps.py:1695)."""
        return (self.views, self.height, self.width)

    def random_sensors(self, batch_size: int, out: typing.Optional[torch.Tensor] = None) -> torch.Tensor:
        """SensorsBase.random_sensors (_maps.py:1756-1765): batch_size uniform
        (view, row, col) triples, int64 [batch_size, 3] on the current device."""
        dev = device() if out is None else out.device
        idx = torch.stack([torch.randint(0, d, (int(batch_size),), device=dev, dtype=torch.int64)
                           for d in self.index_shape], dim=-1)
        if out is None:
            return idx
        out.copy_(idx)
        return out

    def _checked_sensors(self, sensors_batch: torch.Tensor, dev) -> torch.Tensor:
        if sensors_batch.shape[-1] != 3:
            raise ValueError("sensors_batch must end in 3 indices (view, row, col)")
        s = sensors_batch.to(device=dev, dtype=torch.int64).reshape(-1, 3).contiguous()
        if s.shape[0] == 0:
            raise ValueError("sensors_batch is empty")
        lo = s.min(dim=0).values
        hi = s.max(dim=0).values
        lim = torch.tensor(self.index_shape, device=dev, dtype=torch.int64)
        if bool((lo < 0).any()) or bool((hi >= lim).any()):
            raise IndexError(f"sensors_batch indices outside the camera's {self.index_shape}")
        return s.reshape(*sensors_batch.shape)

    def capture(self, field: MapBase, sensors_batch: typing.Optional[torch.Tensor] = None,
                batch_size: typing.Optional[int] = None, fw_samples: int = 1, bw_samples: int = 1,
                debug_out: typing.Optional[torch.Tensor] = None, seed: typing.Optional[int] = None) -> torch.Tensor:
        """SensorsBase.capture (_maps.py:1741-1749): [views, H, W, 3] mean of
        fw_samples paths per pixel (or sensors_batch.shape[:-1] + [3] for a
        batch of (view, row, col) sensors, e.g. from random_sensors); backward
        replays bw_samples paths per pixel with the same per-path Philox
        streams.  batch_size only splits the reference's dispatches; one
        launch covers every sensor here, so it does not change the result."""
        if debug_out is not None:
            raise NotImplementedError("debug_out counters are reported by rendervous_b200.check() instead")
        if not isinstance(field, _PathIntegrator):
            raise NotImplementedError("capture supports path-integrator and collision-integrator fields")
        field = field.cast(input_dim=6)
        desc = field.lower()
        sg, ag, eg = field.grid_tensors()
        sensors = None if sensors_batch is None else self._checked_sensors(sensors_batch, sg.device)
        return _CaptureFn.apply(sg, ag, eg, self, field, desc, int(fw_samples), int(bw_samples),
                                next_seed() if seed is None else int(seed), sensors)


ZERO = const[0.0]
ONE = const[1.0]
