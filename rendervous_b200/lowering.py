"""Lowering of a map graph to the plain medium description the C ABI consumes.

The reference code-generates one GLSL super-kernel per map graph
(rendervous _maps.py:211-291, 509-633).  Here the graph is recognised and
reduced to the fixed forms the CUDA kernels implement (a vrt_medium struct):

  sigma                Grid3D (C == 1)
  scattering_albedo    const[...] or Grid3D (C 1 or 3, same box as sigma)
  emission             const[...]
  environment          const[...]
  environment_sampler  _functionsampler(UniformDirectionSampler, const)
  phase / sampler      HGPhase + VHGPhaseSampler (reference mixture),
                       HenyeyGreensteinPhase + HenyeyGreensteinPhaseSampler,
                       or const[1/4pi] with an isotropic sampler
  boundary             RayBoxIntersection
  majorant             const[[m, 1e6]] (reference) or MajorantGrid
  transmittance        Ratiotracking / Deltatracking / GridDDA transmittance

Anything else raises NotImplementedError -- there is no generic fallback.
"""
from __future__ import annotations

import dataclasses
import math
import typing

import numpy as np
import torch

from . import _lib

TR_MODES = {"rt": 0, "dt": 1, "dda": 2, "dda_exact": 3, "grt": 4, "gdt": 5}


@dataclasses.dataclass
class MediumDesc:
    sigma: torch.Tensor                      # [D,H,W,1]
    bmin: torch.Tensor
    bmax: torch.Tensor
    box_min: torch.Tensor
    box_max: torch.Tensor
    albedo_grid: typing.Optional[torch.Tensor] = None
    albedo_const: tuple = (0.0, 0.0, 0.0)
    emission: tuple = (0.0, 0.0, 0.0)
    env: tuple = (0.0, 0.0, 0.0)
    sun_dir: typing.Optional[tuple] = None
    sun_radiance: tuple = (0.0, 0.0, 0.0)
    phase_mode: int = 0
    phase_g: float = 0.0
    majorant_mode: int = 0
    global_majorant: float = 0.0
    maj_grid: typing.Optional[torch.Tensor] = None
    maj_brick: int = 8
    transmittance_mode: int = 0
    max_bounces: int = 0
    ds_epsilon: float = 0.1
    ds_compat: int = 0
    exitance_mode: int = 0                   # collision integrators: 0 emission, 1 scattered, 2 scattered+emitted
    emission_grid: typing.Optional[torch.Tensor] = None  # [D,H,W,C], C 1 or 3, sigma's box
    env_image: typing.Optional[torch.Tensor] = None      # [H,W,3] equirectangular environment (else env is constant)
    env_quadtree: typing.Optional[torch.Tensor] = None   # NEE directions from the image's quadtree (else uniform)
    env_levels: int = 0

    # -- derived quantities, computed in float32 exactly as the kernels read them
    def inv_bsize(self) -> np.ndarray:
        bmin = self.bmin.detach().cpu().to(torch.float32)
        bmax = self.bmax.detach().cpu().to(torch.float32)
        return (1.0 / (bmax - bmin)).numpy().astype(np.float32)

    def maj_dims(self) -> tuple:
        if self.maj_grid is None:
            return (0, 0, 0)
        d, h, w = self.maj_grid.shape
        return (int(w), int(h), int(d))

    def maj_scale(self) -> np.ndarray:
        D, H, W = self.sigma.shape[:3]
        ib = torch.from_numpy(self.inv_bsize())
        dim = torch.tensor([W - 1, H - 1, D - 1], dtype=torch.float32)
        return (ib * dim / float(self.maj_brick)).numpy().astype(np.float32)

    def to_numpy(self) -> dict:
        """Host copy for the CPU oracle (identical bytes)."""
        f = lambda t: None if t is None else np.ascontiguousarray(t.detach().cpu().numpy().astype(np.float32))
        v3 = lambda v: np.asarray(v, np.float32).reshape(3)
        return dict(
            sigma=f(self.sigma), bmin=v3(f(self.bmin)), bmax=v3(f(self.bmax)), inv_bsize=self.inv_bsize(),
            box_min=v3(f(self.box_min)), box_max=v3(f(self.box_max)), albedo=f(self.albedo_grid),
            albedo_const=v3(self.albedo_const), emission=v3(self.emission), env=v3(self.env),
            has_sun=self.sun_dir is not None, sun_dir=v3(self.sun_dir if self.sun_dir is not None else (0, 0, 0)),
            sun_radiance=v3(self.sun_radiance), phase_mode=self.phase_mode, phase_g=self.phase_g,
            majorant_mode=self.majorant_mode, global_majorant=self.global_majorant,
            maj_grid=f(self.maj_grid), maj_dims=self.maj_dims(), maj_scale=self.maj_scale(),
            transmittance_mode=self.transmittance_mode, max_bounces=self.max_bounces,
            ds_epsilon=self.ds_epsilon, ds_compat=self.ds_compat, exitance_mode=self.exitance_mode,
            emission_grid=f(self.emission_grid), env_image=f(self.env_image), env_quadtree=f(self.env_quadtree),
            env_levels=self.env_levels)

    # -- the C struct (device pointers); keep the returned object alive during the call
    def to_struct(self, sigma_grad: torch.Tensor | None = None, albedo_grad: torch.Tensor | None = None,
                  emission_grad: torch.Tensor | None = None):
        ffi, _ = _lib.ffi_lib()
        m = ffi.new("vrt_medium *")
        _fill_grid(m.sigma, self.sigma, sigma_grad)
        for name, val in (("bmin", self.bmin), ("bmax", self.bmax), ("box_min", self.box_min),
                          ("box_max", self.box_max)):
            v = val.detach().cpu().to(torch.float32).reshape(3).tolist()
            for i in range(3):
                getattr(m, name)[i] = v[i]
        ib = self.inv_bsize()
        for i in range(3):
            m.inv_bsize[i] = float(ib[i])
            m.albedo_const[i] = float(self.albedo_const[i])
            m.emission[i] = float(self.emission[i])
            m.env[i] = float(self.env[i])
            m.sun_radiance[i] = float(self.sun_radiance[i])
            m.sun_dir[i] = float(self.sun_dir[i]) if self.sun_dir is not None else 0.0
        m.has_sun = 1 if self.sun_dir is not None else 0
        if self.albedo_grid is not None:
            m.albedo_is_grid = 1
            _fill_grid(m.albedo, self.albedo_grid, albedo_grad)
        m.phase_mode = self.phase_mode
        m.phase_g = float(self.phase_g)
        m.majorant_mode = self.majorant_mode
        m.global_majorant = float(self.global_majorant)
        if self.maj_grid is not None:
            m.maj_grid = _lib.fptr(self.maj_grid)
            dims = self.maj_dims()
            sc = self.maj_scale()
            for i in range(3):
                m.maj_dims[i] = dims[i]
                m.maj_scale[i] = float(sc[i])
        m.transmittance_mode = self.transmittance_mode
        m.max_bounces = int(self.max_bounces)
        m.ds_epsilon = float(self.ds_epsilon)
        m.ds_compat = int(self.ds_compat)
        m.exitance_mode = int(self.exitance_mode)
        if self.env_image is not None:
            img = self.env_image
            if img.dim() != 3 or img.shape[-1] != 3 or not img.is_contiguous() or not img.is_cuda:
                raise ValueError("the environment image must be a contiguous CUDA [H, W, 3] float32 tensor")
            m.env_mode = 1
            m.env_image = _lib.fptr(img)
            m.env_hw[0], m.env_hw[1] = int(img.shape[0]), int(img.shape[1])
        if self.env_quadtree is not None:
            m.env_sampler = 1
            m.env_quadtree = _lib.fptr(self.env_quadtree)
            m.env_levels = int(self.env_levels)
        if self.emission_grid is not None:
            m.emission_is_grid = 1
            _fill_grid(m.emission_grid, self.emission_grid, emission_grad)
        return m


def _fill_grid(g, t: torch.Tensor, grad: torch.Tensor | None):
    if t.dim() != 4:
        raise ValueError("grids are [D, H, W, C] tensors")
    if t.dtype != torch.float32:
        raise TypeError("grids are float32")
    if not t.is_cuda:
        raise ValueError("grid tensors must be CUDA tensors (there is no CPU path)")
    if t.shape[3] > 1 and t.stride(3) != 1:
        raise ValueError("grid channel stride must be 1")
    g.data = _lib.fptr(t)
    if grad is not None:
        if grad.shape != t.shape or grad.stride()[:3] != t.stride()[:3]:
            raise ValueError("grad must match the grid's shape and strides")
        g.grad = _lib.fptr(grad)
    for i in range(4):
        g.shape[i] = int(t.shape[i])
        g.strides[i] = int(t.stride(i)) if i < 3 else 1


def _const_values(m, n: int) -> tuple:
    from . import maps
    if not isinstance(m, maps.ConstantMap):
        raise NotImplementedError(f"expected a constant map, got {type(m).__name__}")
    v = m.value.detach().reshape(-1).cpu().tolist()
    if len(v) == 1:
        v = v * n
    if len(v) != n:
        raise NotImplementedError(f"constant of {len(v)} values where {n} are needed")
    return tuple(float(a) for a in v)


def _check_same_grid(a, b, what: str):
    if a is not b and not (a.grid is b.grid):
        raise NotImplementedError(f"{what} must use the integrator's sigma Grid3D")


def lower_sigma(sigma, desc_kwargs: dict):
    from . import maps
    if not isinstance(sigma, maps.Grid3D):
        raise NotImplementedError("sigma must be a Grid3D")
    if sigma.grid.shape[-1] != 1:
        raise NotImplementedError("sigma Grid3D must have one channel")
    desc_kwargs.update(sigma=sigma.grid, bmin=sigma.bmin, bmax=sigma.bmax)


def lower_boundary(boundary, desc_kwargs: dict):
    from . import maps
    if not isinstance(boundary, maps.RayBoxIntersection):
        raise NotImplementedError("boundary must be a RayBoxIntersection")
    desc_kwargs.update(box_min=boundary.box_min, box_max=boundary.box_max)


def lower_majorant(majorant, sigma, desc_kwargs: dict):
    from . import maps
    if isinstance(majorant, maps.MajorantGrid):
        _check_same_grid(majorant.sigma, sigma, "MajorantGrid")
        desc_kwargs.update(majorant_mode=1, maj_grid=majorant.tensor(), maj_brick=majorant.brick,
                           global_majorant=0.0)
        return
    v = _const_values(majorant, 2)
    if v[1] < 1e5:
        raise NotImplementedError("a constant majorant must have distance >= 1e5 (the reference uses 1e6)")
    desc_kwargs.update(majorant_mode=0, global_majorant=v[0])


def lower_transmittance(tr, sigma, desc_kwargs: dict):
    from . import maps
    if isinstance(tr, maps.GridDDATransmittance):
        _check_same_grid(tr.grid_model, sigma, "GridDDATransmittance")
        desc_kwargs["transmittance_mode"] = 3 if tr.exact else 2
    elif isinstance(tr, maps.RatiotrackingTransmittance):
        _check_same_grid(tr.sigma, sigma, "RatiotrackingTransmittance")
        desc_kwargs["transmittance_mode"] = 0
    elif isinstance(tr, maps.DeltatrackingTransmittance):
        _check_same_grid(tr.sigma, sigma, "DeltatrackingTransmittance")
        desc_kwargs["transmittance_mode"] = 1
    elif isinstance(tr, (maps.GridRatiotrackingTransmittance, maps.GridDeltatrackingTransmittance)):
        _check_same_grid(tr.grid_model, sigma, type(tr).__name__)
        desc_kwargs["transmittance_mode"] = tr._mode()
    else:
        raise NotImplementedError(f"transmittance map {type(tr).__name__} is not supported")


def lower_phase(phase, sampler, desc_kwargs: dict):
    """Returns (phase_mode, g)."""
    from . import maps
    if isinstance(sampler, maps.VHGPhaseSampler):
        g = _const_values(sampler.phase_g, 1)[0]
        if isinstance(phase, maps.HGPhase):
            gp = _const_values(phase.phase_g, 1)[0]
            if gp != g:
                raise NotImplementedError("phase and phase sampler disagree on g")
            mode = 1
        elif phase is None or isinstance(phase, maps.ConstantMap):
            if phase is not None:
                pv = _const_values(phase, 1)[0]
                if abs(pv - 1.0 / (4 * math.pi)) > 1e-6:
                    raise NotImplementedError("a constant phase must be isotropic (1/4pi)")
            if abs(g) >= 0.001:
                raise NotImplementedError("an isotropic phase needs g == 0 in its sampler")
            mode = 0
        else:
            raise NotImplementedError(f"phase {type(phase).__name__} with VHGPhaseSampler")
    elif isinstance(sampler, maps.HenyeyGreensteinPhaseSampler):
        g = _const_values(sampler.phase_g, 1)[0]
        if phase is not None and not isinstance(phase, maps.HenyeyGreensteinPhase):
            raise NotImplementedError("HenyeyGreensteinPhaseSampler pairs with HenyeyGreensteinPhase")
        if phase is not None and _const_values(phase.phase_g, 1)[0] != g:
            raise NotImplementedError("phase and phase sampler disagree on g")
        mode = 0
    else:
        raise NotImplementedError(f"phase sampler {type(sampler).__name__} is not supported")
    desc_kwargs.update(phase_mode=mode, phase_g=g)


def lower_environment(env, kw: dict):
    """A constant environment, or Image2D(image).after(xr_projection) with the
    image's default box (_objects.py:165-172)."""
    from . import maps
    if isinstance(env, maps.CompositionMap) and isinstance(env.map_a, maps.XRProjection) and \
            isinstance(env.map_b, maps.Image2D):
        img = env.map_b
        if img.grid.shape[-1] != 3:
            raise NotImplementedError("an environment image has 3 channels")
        if not (torch.allclose(img.bmin.cpu(), torch.tensor([-1.0, -1.0])) and
                torch.allclose(img.inv_bsize.cpu(), torch.tensor([0.5, 0.5]))):
            raise NotImplementedError("an environment image keeps Image2D's default box [-1, 1]^2")
        kw["env_image"] = img.grid.detach().contiguous()
        kw["env"] = (0.0, 0.0, 0.0)
        return
    kw["env"] = _const_values(env, 3)


def _same_environment(a, b) -> bool:
    from . import maps
    if a is b:
        return True
    if isinstance(a, maps.ConstantMap) and isinstance(b, maps.ConstantMap):
        return _const_values(a, 3) == _const_values(b, 3)
    if isinstance(a, maps.CompositionMap) and isinstance(b, maps.CompositionMap):
        return a.map_b is b.map_b
    return False


def lower_environment_sampler(es, env, kw: dict):
    """_functionsampler(UniformDirectionSampler | XRQuadtreeRandomDirection,
    environment) (_objects.py:180-203) over the integrator's environment."""
    from . import maps
    if not isinstance(es, maps._functionsampler):
        raise NotImplementedError("the environment sampler must be a _functionsampler")
    if not _same_environment(es.function_map, env):
        raise NotImplementedError("the environment sampler must sample the integrator's environment")
    ps = es.point_sampler
    if isinstance(ps, maps.UniformDirectionSampler):
        return
    if isinstance(ps, maps.XRQuadtreeRandomDirection):
        if ps.levels < 1 or ps.levels > 14:
            raise NotImplementedError("quadtree levels must be in 1..14")
        qt = ps.densities() if callable(ps.densities) else ps.densities
        if qt.numel() != sum(4 ** l for l in range(1, ps.levels + 1)):
            raise NotImplementedError("quadtree size does not match its levels")
        kw["env_quadtree"] = qt.detach().reshape(-1).contiguous().to(torch.float32)
        kw["env_levels"] = ps.levels
        return
    raise NotImplementedError(f"environment direction sampler {type(ps).__name__} is not supported")


def lower_integrator(pi) -> MediumDesc:
    """MediumDesc of a path-integrator map (DeltatrackingPathIntegrator, ...)."""
    from . import maps
    kw: dict = {}
    lower_sigma(pi.sigma, kw)
    alb = pi.scattering_albedo
    if isinstance(alb, maps.Grid3D):
        if alb.grid.shape[-1] not in (1, 3):
            raise NotImplementedError("albedo Grid3D must have 1 or 3 channels")
        if not (torch.equal(alb.bmin.cpu(), pi.sigma.bmin.cpu()) and torch.equal(alb.bmax.cpu(), pi.sigma.bmax.cpu())):
            raise NotImplementedError("albedo Grid3D must share sigma's box")
        kw["albedo_grid"] = alb.grid
    else:
        kw["albedo_const"] = _const_values(alb, 3)
    kw["emission"] = _const_values(pi.emission, 3)
    lower_environment(pi.environment, kw)
    es = getattr(pi, "environment_sampler", None)
    if es is not None:
        lower_environment_sampler(es, pi.environment, kw)
    lower_phase(getattr(pi, "phase", None), pi.phase_sampler, kw)
    lower_boundary(pi.boundary, kw)
    lower_majorant(pi.majorant, pi.sigma, kw)
    tr = getattr(pi, "transmittance", None)
    if tr is not None:
        lower_transmittance(tr, pi.sigma, kw)
    light = getattr(pi, "directional_light", None)
    if light is not None:
        kw["sun_dir"] = tuple(float(v) for v in light.direction.reshape(3).tolist())
        kw["sun_radiance"] = tuple(float(v) for v in light.radiance.reshape(3).tolist())
    kw["max_bounces"] = int(getattr(pi, "max_bounces", 0))
    kw["ds_epsilon"] = float(getattr(pi, "ds_epsilon", 0.1) or 0.0)
    kw["ds_compat"] = 1 if getattr(pi, "ds_compat", False) else 0
    return MediumDesc(**kw)


def _lower_albedo(alb, sigma, kw: dict):
    from . import maps
    if isinstance(alb, maps.Grid3D):
        if alb.grid.shape[-1] not in (1, 3):
            raise NotImplementedError("albedo Grid3D must have 1 or 3 channels")
        if not (torch.equal(alb.bmin.cpu(), sigma.bmin.cpu()) and torch.equal(alb.bmax.cpu(), sigma.bmax.cpu())):
            raise NotImplementedError("albedo Grid3D must share sigma's box")
        kw["albedo_grid"] = alb.grid
    else:
        kw["albedo_const"] = _const_values(alb, 3)


def _lower_emission(em, sigma, kw: dict):
    """The emission map of an exitance radiance: a constant, or a Grid3D of 1 or
    3 channels over sigma's box (read at the position; it ignores the direction)."""
    from . import maps
    if isinstance(em, maps.Grid3D):
        if em.grid.shape[-1] not in (1, 3):
            raise NotImplementedError("an emission Grid3D must have 1 or 3 channels")
        if not (torch.equal(em.bmin.cpu(), sigma.bmin.cpu()) and torch.equal(em.bmax.cpu(), sigma.bmax.cpu())):
            raise NotImplementedError("an emission Grid3D must share sigma's box")
        kw["emission_grid"] = em.grid
    else:
        kw["emission"] = _const_values(em, 3)


def _lower_phase_sampler(sampler, kw: dict):
    """A phase sampler used alone (no phase map is evaluated): VHGPhaseSampler
    draws the reference's mixture (phase_mode 1), HenyeyGreensteinPhaseSampler
    pure HG (phase_mode 0); both report weight 1."""
    from . import maps
    if isinstance(sampler, maps.VHGPhaseSampler):
        kw["phase_mode"] = 1
    elif isinstance(sampler, maps.HenyeyGreensteinPhaseSampler):
        kw["phase_mode"] = 0
    else:
        raise NotImplementedError(f"phase sampler {type(sampler).__name__} is not supported")
    kw["phase_g"] = _const_values(sampler.phase_g, 1)[0]


def _transmitted_environment(radiance):
    """(transmittance map, environment constant) of a radiance map of the form
    transmittance * environment.after(ray_direction) (_objects.py:262-265)."""
    from . import maps
    if not isinstance(radiance, maps.MultiplicationMap):
        raise NotImplementedError("the radiance of a scattered exitance must be transmittance * environment")
    a, b = radiance.map_a, radiance.map_b
    if isinstance(a, maps.CompositionMap):
        a, b = b, a
    if not (isinstance(b, maps.CompositionMap) and isinstance(b.map_a, maps.RayDirection)):
        raise NotImplementedError("the radiance of a scattered exitance must be transmittance * environment")
    return a, b.map_b


def lower_collision_integrator(ci) -> MediumDesc:
    """MediumDesc of MCCollisionIntegrator (_maps.py:2792-2808) or
    GridDDACollisionIntegrator (_maps.py:2811-2852): sigma, boundary (and the
    collision sampler's majorant and epsilon), the environment constant, and
    the exitance radiance -- an emission map, MCScatteredRadiance or
    MCScatteredEmittedRadiance over transmittance * environment."""
    from . import maps
    kw: dict = {}
    if isinstance(ci, maps.MCCollisionIntegrator):
        cs = ci.collision_sampler
        if not isinstance(cs, maps.DeltatrackingCollisionSampler):
            raise NotImplementedError("the collision sampler must be a DeltatrackingCollisionSampler")
        sigma = cs.sigma
        lower_sigma(sigma, kw)
        lower_boundary(cs.boundary, kw)
        lower_majorant(cs.majorant, sigma, kw)
        kw["ds_epsilon"] = float(cs.ds_epsilon)
    else:
        sigma = ci.sigma_grid
        lower_sigma(sigma, kw)
        lower_boundary(ci.boundary, kw)
    lower_environment(ci.environment, kw)
    ex = ci.exitance_radiance
    if isinstance(ex, (maps.MCScatteredRadiance, maps.MCScatteredEmittedRadiance)):
        kw["exitance_mode"] = 1 if isinstance(ex, maps.MCScatteredRadiance) else 2
        _lower_albedo(ex.scattering_albedo, sigma, kw)
        _lower_phase_sampler(ex.phase_sampler, kw)
        tr, env = _transmitted_environment(ex.radiance)
        if not _same_environment(env, ci.environment):
            raise NotImplementedError("the scattered radiance's environment must be the integrator's environment")
        lower_transmittance(tr, sigma, kw)
        tmaj = getattr(tr, "majorant", None)
        if tmaj is not None:
            if isinstance(ci, maps.MCCollisionIntegrator) and tmaj is not ci.collision_sampler.majorant:
                raise NotImplementedError("the transmittance and the collision sampler must share the majorant")
            lower_majorant(tmaj, sigma, kw)
        if isinstance(ex, maps.MCScatteredEmittedRadiance):
            _lower_emission(ex.emission, sigma, kw)
    else:
        kw["exitance_mode"] = 0
        _lower_emission(ex, sigma, kw)
    return MediumDesc(**kw)


def lower_transmittance_map(tr) -> MediumDesc:
    """MediumDesc of a transmittance map evaluated on rays."""
    from . import maps
    kw: dict = {}
    if isinstance(tr, maps.GridDDATransmittance):
        lower_sigma(tr.grid_model, kw)
        kw["transmittance_mode"] = 3 if tr.exact else 2
    elif isinstance(tr, (maps.GridRatiotrackingTransmittance, maps.GridDeltatrackingTransmittance)):
        lower_sigma(tr.grid_model, kw)
        kw["transmittance_mode"] = tr._mode()
    else:
        lower_sigma(tr.sigma, kw)
        lower_majorant(tr.majorant, tr.sigma, kw)
        kw["transmittance_mode"] = 0 if isinstance(tr, maps.RatiotrackingTransmittance) else 1
    lower_boundary(tr.boundary, kw)
    return MediumDesc(**kw)
