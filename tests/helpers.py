"""Scene construction shared by the CPU oracle tests and the GPU parity tests."""
from __future__ import annotations

import math

import numpy as np
import torch

from rendervous_b200 import maps, synthetic
from rendervous_b200.lowering import MediumDesc


def oracle_desc(sigma: np.ndarray, *, albedo=0.9, albedo_grid: np.ndarray | None = None, emission=0.0, env=1.0,
                sun_dir=None, sun_radiance=3.0, phase_mode=0, g=0.0, majorant="global", brick=8, tr="rt",
                max_bounces=0, ds_epsilon=0.1, ds_compat=0, box=None, exitance_mode=0,
                emission_grid: np.ndarray | None = None) -> dict:
    """A medium description for the oracle built directly from numpy arrays."""
    import oracle
    sigma = np.ascontiguousarray(sigma, np.float32)
    if box is None:
        bmin, bmax = maps.normalized_box(list(sigma.shape))
    else:
        bmin, bmax = torch.tensor(box[0], dtype=torch.float32), torch.tensor(box[1], dtype=torch.float32)
    desc = MediumDesc(sigma=torch.from_numpy(sigma), bmin=bmin, bmax=bmax, box_min=bmin.clone(), box_max=bmax.clone())
    if albedo_grid is not None:
        desc.albedo_grid = torch.from_numpy(np.ascontiguousarray(albedo_grid, np.float32))
    a = np.broadcast_to(np.asarray(albedo, np.float32), (3,))
    desc.albedo_const = tuple(float(v) for v in a)
    desc.emission = tuple(float(v) for v in np.broadcast_to(np.asarray(emission, np.float32), (3,)))
    desc.env = tuple(float(v) for v in np.broadcast_to(np.asarray(env, np.float32), (3,)))
    if sun_dir is not None:
        d = np.asarray(sun_dir, np.float64)
        desc.sun_dir = tuple(float(v) for v in (d / np.linalg.norm(d)).astype(np.float32))
        desc.sun_radiance = tuple(float(v) for v in np.broadcast_to(np.asarray(sun_radiance, np.float32), (3,)))
    desc.phase_mode = phase_mode
    desc.phase_g = float(g)
    if majorant == "global":
        desc.majorant_mode = 0
        desc.global_majorant = float(sigma.max())
    else:
        desc.majorant_mode = 1
        desc.maj_brick = brick
        desc.maj_grid = torch.from_numpy(oracle.majorant_build(sigma, brick))
    desc.transmittance_mode = {"rt": 0, "dt": 1, "dda": 2, "dda_exact": 3, "grt": 4, "gdt": 5}[tr]
    desc.max_bounces = max_bounces
    desc.ds_epsilon = ds_epsilon
    desc.ds_compat = ds_compat
    desc.exitance_mode = exitance_mode
    if emission_grid is not None:
        desc.emission_grid = torch.from_numpy(np.ascontiguousarray(emission_grid, np.float32))
    return desc.to_numpy()


def homogeneous(res: int, value: float) -> np.ndarray:
    return np.full((res, res, res, 1), value, np.float32)


def build_field(sigma: torch.Tensor, *, albedo=0.9, albedo_grid: torch.Tensor | None = None, env=1.0, sun_dir=None,
                sun_radiance=3.0, g=0.0, phase="hg", majorant="global", brick=8, tr="rt", max_bounces=0,
                integrator="nee_ds", ds_epsilon=0.1, ds_compat=False, sigma_requires_grad=False):
    """A path-integrator map assembled through the public map API (as a
    reference user would), on the device of ``sigma``."""
    bmin, bmax = maps.normalized_box(sigma)
    sig_p = torch.nn.Parameter(sigma, requires_grad=sigma_requires_grad)
    sg = maps.Grid3D(sig_p, bmin, bmax)
    if albedo_grid is not None:
        alb = maps.Grid3D(albedo_grid if isinstance(albedo_grid, torch.nn.Parameter) else
                          torch.nn.Parameter(albedo_grid, requires_grad=False), bmin, bmax)
    else:
        a = np.broadcast_to(np.asarray(albedo, np.float32), (3,))
        alb = maps.const[tuple(float(v) for v in a)]
    e = np.broadcast_to(np.asarray(env, np.float32), (3,))
    envm = maps.const[tuple(float(v) for v in e)]
    boundary = maps.ray_box_intersection[bmin, bmax]
    if majorant == "global":
        maj = maps.const[[float(sigma.max().item()), 1000000.0]]
    else:
        maj = maps.MajorantGrid(sg, brick=brick)
    if phase == "hg":
        ph, ps = maps.HenyeyGreensteinPhase(maps.const[g]), maps.HenyeyGreensteinPhaseSampler(maps.const[g])
    else:
        ph, ps = maps.HGPhase(maps.const[g]), maps.VHGPhaseSampler(maps.const[g])
    if tr == "rt":
        trm = maps.RatiotrackingTransmittance(sg, boundary, maj)
    elif tr == "dt":
        trm = maps.DeltatrackingTransmittance(sg, boundary, maj)
    elif tr == "grt":
        trm = maps.GridRatiotrackingTransmittance(sg, boundary)
    elif tr == "gdt":
        trm = maps.GridDeltatrackingTransmittance(sg, boundary)
    else:
        trm = maps.GridDDATransmittance(sg, boundary, exact=(tr == "dda_exact"))
    light = None if sun_dir is None else maps.DirectionalLight(torch.tensor(sun_dir, dtype=torch.float32), sun_radiance)
    env_sampler = maps._functionsampler(maps.UniformDirectionSampler(6), envm)
    ext = dict(max_bounces=max_bounces, directional_light=light)
    if integrator == "dt":
        return maps.DeltatrackingPathIntegrator(sg, alb, maps.ZERO, envm, ps, boundary, maj, ds_epsilon, **ext)
    if integrator == "nee_ds":
        return maps.DeltatrackingNEEPathIntegrator(sg, alb, maps.ZERO, envm, env_sampler, ph, ps, boundary, maj, trm,
                                                   ds_epsilon, ds_compat=ds_compat, **ext)
    if integrator == "drtq":
        return maps.DRTQPathIntegrator(sg, alb, maps.ZERO, envm, env_sampler, ph, ps, boundary, maj, trm, **ext)
    if integrator == "drtds":
        return maps.DRTDSPathIntegrator(sg, alb, maps.ZERO, envm, env_sampler, ph, ps, boundary, maj, trm, ds_epsilon,
                                        **ext)
    if integrator == "sps":
        return maps.SPSPathIntegrator(sg, alb, maps.ZERO, envm, env_sampler, ph, ps, boundary, maj, trm, **ext)
    return maps.DRTPathIntegrator(sg, alb, maps.ZERO, envm, env_sampler, ph, ps, boundary, maj, trm, **ext)


def front_camera(views: int = 1) -> torch.Tensor:
    return torch.from_numpy(synthetic.ring_poses(views, radius=2.0, elevation_deg=20.0))
