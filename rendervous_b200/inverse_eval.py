"""Inverse-rendering loop (workload inverse_rendering_128).

Target: a seeded 256^3 blob volume (64 blobs, max sigma 40, like the
differentiable tracer's) rendered from 8 cameras on a ring of radius
2 (elevation 20 degrees) at 256x256, 128 spp.  Optimised: a 128^3 FP32 sigma
grid initialised to 1.0, albedo fixed at 0.9, HG g = 0.3, unit environment
plus a directional light.  Each iteration captures all 8 views in one call (16
spp, at most 32 bounces, NEE with ratio-tracking shadows over an 8^3-brick
majorant grid), runs the NEE_DS path-replay adjoint, and takes an Adam step
(lr 0.01); sigma is clamped at 0 after each step.  Reports iterations/s (CUDA
events around the whole loop), the loss after the last iteration, and the loss
on held-out views (the cameras half-way between the training ones) before and
after the optimisation.

Run: python -m rendervous_b200.inverse_eval [--iterations 500 ...]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import maps, synthetic


def build_field(sigma: torch.Tensor, *, albedo: float, g: float, max_bounces: int, sun_dir, sun_radiance: float,
                env: float = 1.0, brick: int = 8):
    bmin, bmax = maps.normalized_box(sigma)
    sg = maps.Grid3D(sigma, bmin, bmax)
    alb = maps.const[(albedo, albedo, albedo)]
    envm = maps.const[(env, env, env)]
    boundary = maps.ray_box_intersection[bmin, bmax]
    maj = maps.MajorantGrid(sg, brick=brick)
    ph, ps = maps.HenyeyGreensteinPhase(maps.const[g]), maps.HenyeyGreensteinPhaseSampler(maps.const[g])
    trm = maps.RatiotrackingTransmittance(sg, boundary, maj)
    light = maps.DirectionalLight(torch.tensor(sun_dir, dtype=torch.float32), sun_radiance)
    env_sampler = maps._functionsampler(maps.UniformDirectionSampler(6), envm)
    return maps.DeltatrackingNEEPathIntegrator(sg, alb, maps.ZERO, envm, env_sampler, ph, ps, boundary, maj, trm, 0.1,
                                               max_bounces=max_bounces, directional_light=light)


def downsample(sigma: torch.Tensor, res: int) -> torch.Tensor:
    """Node values of a [D,H,W,1] grid resampled trilinearly at a res^3 node lattice
    over the same box (for comparing the optimised grid with the target)."""
    g = torch.nn.functional.interpolate(sigma[None, ..., 0][:, None], size=(res, res, res), mode="trilinear",
                                        align_corners=True)
    return g[0, 0, ..., None]


def run(iterations: int = 500, width: int = 256, spp: int = 16, target_spp: int = 128, views: int = 8,
        res: int = 128, target_res: int = 256, seed: int = 0, device=None, log=None, lr: float = None) -> dict:
    wl = synthetic.WORKLOADS["inverse_rendering_128"]
    dev = torch.device(device or "cuda")
    maps.set_sync_checks(False)
    kind, args = wl["target_sigma"]
    args = dict(args, res=target_res)
    target_sigma = torch.from_numpy(synthetic.make_sigma((kind, args))).to(dev)
    sun = tuple(float(v) for v in synthetic.gaussian_direction(6))
    common = dict(albedo=wl["albedo"], g=wl["phase_g"], max_bounces=wl["max_bounces"], sun_dir=sun, sun_radiance=3.0)
    # training views: the ring of `views` cameras; held-out views: the cameras half-way between them
    ring = torch.from_numpy(synthetic.ring_poses(2 * views, radius=2.0, elevation_deg=20.0)).to(dev)
    cam = maps.PerspectiveCameraSensor(width, width, ring[0::2].contiguous(), jittered=True)
    held = maps.PerspectiveCameraSensor(width, width, ring[1::2].contiguous(), jittered=True)
    with torch.no_grad():
        tfield = build_field(torch.nn.Parameter(target_sigma, requires_grad=False), **common)
        target = cam.capture(tfield, fw_samples=target_spp, seed=10_000 + seed)
        target_held = held.capture(tfield, fw_samples=target_spp, seed=20_000 + seed)
    sigma = torch.nn.Parameter(torch.full((res, res, res, 1), float(wl["init_sigma"]), device=dev))
    field = build_field(sigma, **common)
    lr = float(wl["lr"] if lr is None else lr)
    opt = torch.optim.Adam([sigma], lr=lr)
    ref = downsample(target_sigma, res)

    def held_loss():
        with torch.no_grad():
            img = held.capture(field, fw_samples=target_spp, seed=30_000 + seed)
            return float(((img - target_held) ** 2).mean())

    held0 = held_loss()
    losses = []
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.time()
    e0.record()
    for it in range(iterations):
        opt.zero_grad(set_to_none=True)
        img = cam.capture(field, fw_samples=spp, bw_samples=spp, seed=1000 * (seed + 1) + it)
        loss = ((img - target) ** 2).mean()
        loss.backward()
        opt.step()
        with torch.no_grad():
            sigma.clamp_(min=0.0)
        losses.append(loss.detach())
        if log is not None and (it % 50 == 0 or it == iterations - 1):
            log(dict(iteration=it, loss=float(loss)))
    e1.record()
    e1.synchronize()
    seconds = e0.elapsed_time(e1) / 1000.0
    maps.check()
    held1 = held_loss()
    losses = torch.stack(losses).cpu().numpy()
    err = float(((sigma.detach() - ref) ** 2).sum().sqrt() / (ref ** 2).sum().sqrt())
    err0 = float(((torch.full_like(ref, float(wl["init_sigma"])) - ref) ** 2).sum().sqrt() / (ref ** 2).sum().sqrt())
    return dict(workload="inverse_rendering_128" if (iterations, width, res) == (500, 256, 128) else
                f"inverse_{res}_{width}px_{iterations}it",
                iterations=iterations, views=views, width=width, spp=spp, target_spp=target_spp, res=res, lr=lr,
                target_res=target_res, iterations_per_s=iterations / seconds, seconds=seconds,
                wall_s=time.time() - t0, loss_first=float(losses[0]), loss_final=float(losses[-1]),
                loss_final_mean10=float(losses[-10:].mean()), heldout_loss_initial=held0, heldout_loss_final=held1,
                sigma_rel_err_initial=err0, sigma_rel_err_final=err)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--iterations", type=int, default=500)
    ap.add_argument("--width", type=int, default=256)
    ap.add_argument("--spp", type=int, default=16)
    ap.add_argument("--target-spp", type=int, default=128)
    ap.add_argument("--views", type=int, default=8)
    ap.add_argument("--res", type=int, default=128)
    ap.add_argument("--target-res", type=int, default=256)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--lr", type=float, default=None, help="Adam learning rate (default: the workload's 0.01)")
    ap.add_argument("--out", type=str, default=None)
    a = ap.parse_args(argv)
    out = run(a.iterations, a.width, a.spp, a.target_spp, a.views, a.res, a.target_res, a.seed,
              log=lambda d: print(json.dumps(d), flush=True), lr=a.lr)
    print(json.dumps(out))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(out, f, indent=1)
    return out


if __name__ == "__main__":
    main()
