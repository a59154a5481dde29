"""Scene-assembly builders for the volume hot path.

Mirrors the reference's DependencySet (_internal.py:256-334) and the
``medium_*`` builders of ``_objects.py`` that assemble a path integrator, so
that reference scene scripts port line for line.  Builders outside the volume
path (surfaces, image environments, quadtree samplers) are not provided.
Where the reference builder is broken (``medium_environment_sampler_uniform``
calls a missing ``ds.includes``, ``medium_phase_sampler_uniform`` a missing
``_maps.identity``; _objects.py:201-203, 229-233) the working form is given.
"""
from __future__ import annotations

import math
import typing

import torch

from . import maps


class DependencySet:
    """Named fields built on demand by builder functions (_internal.py:256-334).
    Callables given to add_parameters are re-evaluated by forward_dependency()."""

    def __init__(self, parent: "DependencySet" = None):
        object.__setattr__(self, "_fields", {})
        object.__setattr__(self, "_lambdas", {})
        object.__setattr__(self, "_parent", parent)

    def ensures(self, field_name, field_type) -> bool:
        return (field_name in self._fields and isinstance(self._fields[field_name], field_type)) or (
            self._parent is not None and self._parent.ensures(field_name, field_type))

    def assert_ensures(self, field_name, field_type):
        assert self.ensures(field_name, field_type), f"Required field {field_name} of type {field_type} not found."

    def branch(self) -> "DependencySet":
        return DependencySet(parent=self)

    def add_parameters(self, **kwargs):
        for k, v in kwargs.items():
            if not isinstance(v, torch.nn.Module) and callable(v):
                self._lambdas[k] = v
                v = v()
            self._fields[k] = v

    def requires(self, builder: typing.Callable, **kwargs):
        builder(self, **kwargs)

    def forward_dependency(self):
        if self._parent is not None:
            self._parent.forward_dependency()
        for k, f in self._lambdas.items():
            t = self._fields[k]
            with torch.no_grad():
                t.copy_(f())

    def __getattr__(self, item):
        if item in self._fields:
            return self._fields[item]
        if self._parent is not None:
            return getattr(self._parent, item)
        raise AttributeError(item)


# ------------------------------------------------------------------ builders --
def medium_box_AABB(ds, *, bmin=maps.vec3(-1.0, -1.0, -1.0), bmax=maps.vec3(1.0, 1.0, 1.0)):
    ds.add_parameters(box=(bmin, bmax))


def medium_box_normalized(ds, *, t):
    ds.add_parameters(box=maps.normalized_box(t))


def medium_box(ds):
    if ds.ensures("box", tuple):
        return
    if ds.ensures("sigma_tensor", torch.Tensor):
        medium_box_normalized(ds, t=ds.sigma_tensor)
    elif ds.ensures("sigma", maps.Grid3D):
        medium_box_normalized(ds, t=ds.sigma.grid)
    else:
        medium_box_AABB(ds)


def medium_boundary(ds):
    if ds.ensures("boundary", maps.MapBase):
        return
    ds.requires(medium_box)
    bmin, bmax = ds.box
    ds.add_parameters(boundary=maps.RayBoxIntersection(bmin, bmax))


def build_map_from_tensor(ds, *, field_name: str):
    ds.requires(medium_box)
    bmin, bmax = ds.box
    ds.assert_ensures(field_name + "_tensor", torch.Tensor)
    tensor = getattr(ds, field_name + "_tensor")
    if len(tensor.shape) == 1:
        return maps.const[tensor]
    return maps.Grid3D(tensor, bmin, bmax)


def medium_sigma(ds):
    if not ds.ensures("sigma", maps.MapBase):
        ds.add_parameters(sigma=build_map_from_tensor(ds, field_name="sigma"))


def medium_scattering_albedo(ds):
    if not ds.ensures("scattering_albedo", maps.MapBase):
        ds.add_parameters(scattering_albedo=build_map_from_tensor(ds, field_name="scattering_albedo"))


def medium_emission(ds):
    if not ds.ensures("emission", maps.MapBase):
        if ds.ensures("emission_tensor", torch.Tensor):
            ds.add_parameters(emission=maps.const[ds.emission_tensor])
        else:
            ds.add_parameters(emission=maps.ZERO)


def medium_environment(ds):
    """_objects.py:160-177: a constant, or an equirectangular image
    Image2D(tensor).after(xr_projection)."""
    if not ds.ensures("environment", maps.MapBase):
        ds.assert_ensures("environment_tensor", torch.Tensor)
        t = ds.environment_tensor
        if len(t.shape) == 1:
            ds.add_parameters(environment=maps.const[t])
        else:
            ds.add_parameters(environment=maps.Image2D(t).after(maps.xr_projection))


def medium_environment_sampler_uniform(ds):
    ds.requires(medium_environment)
    ds.add_parameters(environment_sampler=maps._functionsampler(maps.UniformDirectionSampler(6), ds.environment))


def medium_environment_sampler_quadtree(ds, *, levels: int = 10):
    """_objects.py:180-199: NEE directions from the probability quadtree of an
    image environment."""
    ds.requires(medium_environment)
    ds.assert_ensures("environment_tensor", torch.Tensor)
    if len(ds.environment_tensor.shape) != 3:
        raise NotImplementedError("a quadtree sampler needs an image environment")
    qt = maps.environment_quadtree(ds.environment_tensor, levels=levels)
    ds.add_parameters(environment_sampler_quadtree=qt)
    sampler = maps.XRQuadtreeRandomDirection(6, qt, levels)
    ds.add_parameters(environment_sampler=maps._functionsampler(sampler, ds.environment))


def medium_environment_sampler(ds):
    """_objects.py:205-212: the quadtree sampler for image environments, else uniform."""
    if ds.ensures("environment_sampler", maps.MapBase):
        return
    ds.requires(medium_environment)
    if len(ds.environment_tensor.shape) == 3:
        medium_environment_sampler_quadtree(ds)
    else:
        medium_environment_sampler_uniform(ds)


def medium_phase_g(ds):
    if not ds.ensures("phase_g", maps.MapBase):
        ds.add_parameters(phase_g=build_map_from_tensor(ds, field_name="phase_g"))


def medium_phase(ds):
    if ds.ensures("phase", maps.MapBase):
        return
    if ds.ensures("phase_g", maps.MapBase) or ds.ensures("phase_g_tensor", torch.Tensor):
        ds.requires(medium_phase_g)
        ds.add_parameters(phase=maps.HGPhase(ds.phase_g))
    else:
        ds.add_parameters(phase=maps.const[1.0 / (4 * math.pi)])


def medium_phase_sampler(ds):
    if ds.ensures("phase_sampler", maps.MapBase):
        return
    if ds.ensures("phase_g", maps.MapBase) or ds.ensures("phase_g_tensor", torch.Tensor):
        ds.requires(medium_phase_g)
        ds.add_parameters(phase_sampler=maps.VHGPhaseSampler(ds.phase_g))
    else:
        ds.add_parameters(phase_sampler=maps.VHGPhaseSampler(maps.const[0.0]))


def medium_majorant(ds):
    """_objects.py:103-114: majorant tensor if given, else [max sigma, 1e6]."""
    if ds.ensures("majorant", maps.MapBase):
        return
    if ds.ensures("majorant_tensor", torch.Tensor):
        ds.add_parameters(majorant=maps.const[ds.majorant_tensor])
        return
    ds.requires(medium_sigma)
    ds.assert_ensures("sigma", maps.Grid3D)
    ds.add_parameters(majorant=maps.GridMaximumMajorant(ds.sigma))


def medium_majorant_bricks(ds, *, brick: int = 8):
    """Majorant grid over the sigma Grid3D (no reference counterpart)."""
    ds.requires(medium_sigma)
    ds.assert_ensures("sigma", maps.Grid3D)
    ds.add_parameters(majorant=maps.MajorantGrid(ds.sigma, brick=brick))


def medium_transmittance_DDA(ds, *, exact: bool = False):
    ds.requires(medium_sigma)
    ds.requires(medium_boundary)
    ds.add_parameters(transmittance=maps.GridDDATransmittance(ds.sigma, ds.boundary, exact=exact))


def medium_transmittance_DT(ds):
    ds.requires(medium_sigma)
    ds.requires(medium_boundary)
    ds.requires(medium_majorant)
    ds.add_parameters(transmittance=maps.DeltatrackingTransmittance(ds.sigma, ds.boundary, ds.majorant))


def medium_transmittance_RT(ds):
    ds.requires(medium_sigma)
    ds.requires(medium_boundary)
    ds.requires(medium_majorant)
    ds.add_parameters(transmittance=maps.RatiotrackingTransmittance(ds.sigma, ds.boundary, ds.majorant))


def medium_transmittance(ds):
    if not ds.ensures("transmittance", maps.MapBase):
        medium_transmittance_RT(ds)


def _common(ds):
    ds.requires(medium_sigma)
    if not ds.ensures("scattering_albedo", maps.MapBase):
        if ds.ensures("scattering_albedo_tensor", torch.Tensor):
            medium_scattering_albedo(ds)
        else:
            ds.add_parameters(scattering_albedo=maps.ZERO)
    ds.requires(medium_emission)
    ds.requires(medium_boundary)
    ds.requires(medium_majorant)
    ds.requires(medium_environment)


def medium_radiance_path_integrator_DT(ds, *, ds_epsilon: float = 0.1, **ext):
    _common(ds)
    ds.requires(medium_phase_sampler)
    ds.add_parameters(radiance=maps.DeltatrackingPathIntegrator(
        ds.sigma, ds.scattering_albedo, ds.emission, ds.environment, ds.phase_sampler, ds.boundary, ds.majorant,
        ds_epsilon, **ext))


def _nee_args(ds):
    _common(ds)
    ds.requires(medium_environment_sampler)
    ds.requires(medium_phase)
    ds.requires(medium_phase_sampler)
    ds.requires(medium_transmittance)
    return (ds.sigma, ds.scattering_albedo, ds.emission, ds.environment, ds.environment_sampler, ds.phase,
            ds.phase_sampler, ds.boundary, ds.majorant, ds.transmittance)


def medium_radiance_path_integrator_NEE_DT(ds, *, ds_epsilon: float = 0.1, **ext):
    ds.add_parameters(radiance=maps.DeltatrackingNEEPathIntegrator(*_nee_args(ds), ds_epsilon, **ext))


def medium_radiance_path_integrator_NEE_DRT(ds, **ext):
    ds.add_parameters(radiance=maps.DRTPathIntegrator(*_nee_args(ds), **ext))


def medium_radiance_path_integrator_NEE_DRTQ(ds, **ext):
    ds.add_parameters(radiance=maps.DRTQPathIntegrator(*_nee_args(ds), **ext))


def medium_radiance_path_integrator_NEE_DRTDS(ds, *, ds_epsilon: float = 0.1, **ext):
    ds.add_parameters(radiance=maps.DRTDSPathIntegrator(*_nee_args(ds), ds_epsilon, **ext))


def medium_radiance_path_integrator_NEE_SPS(ds, **ext):
    ds.add_parameters(radiance=maps.SPSPathIntegrator(*_nee_args(ds), **ext))


def medium_radiance(ds):
    if not ds.ensures("radiance", maps.MapBase):
        ds.requires(medium_radiance_path_integrator_DT)


def camera_sensors(ds, *, width: int, height: int, jittered: bool = False, fov: float = math.pi / 4):
    ds.assert_ensures("camera_poses", torch.Tensor)
    ds.add_parameters(camera=maps.PerspectiveCameraSensor(width, height, ds.camera_poses, fov=fov, jittered=jittered))
