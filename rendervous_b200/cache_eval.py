"""Equal-time evaluation of the radiance cache against the plain tracer.

Workload (radiance_cache_512): 512^3 six-octave value noise scaled to max
sigma 200, albedo 0.99, Henyey-Greenstein g = 0.8, unit environment plus a
directional light, one 1024x1024 view, NEE integrator with delta-tracking
shadow rays over an 8^3-brick majorant grid.  The plain tracer runs up to 512
bounces; the cached renderer traces 2 bounces and stops into the cache.

Error is measured on a fixed set of square crops against a high-spp estimate of
the same pixels from the FP64 plain tracer (vrt_capture_fw_fp64: every quantity
in double, path for path with the CPU restatement's double instantiation in
the parity tests), rendered as a sensors batch of the crop pixels.

Run: python -m rendervous_b200.cache_eval [--res 512 --size 1024 ...]
Prints one JSON line per method checkpoint and a summary line.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from . import _lib, cache, maps, synthetic


def build_field(sigma: torch.Tensor, *, albedo=0.99, g=0.8, env=1.0, sun_dir=(0.3, 0.8, 0.5), sun_radiance=3.0,
                max_bounces=512, brick=8):
    bmin, bmax = maps.normalized_box(sigma)
    sg = maps.Grid3D(torch.nn.Parameter(sigma, requires_grad=False), bmin, bmax)
    alb = maps.const[(albedo, albedo, albedo)]
    envm = maps.const[(env, env, env)]
    boundary = maps.ray_box_intersection[bmin, bmax]
    maj = maps.MajorantGrid(sg, brick=brick)
    ph, ps = maps.HenyeyGreensteinPhase(maps.const[g]), maps.HenyeyGreensteinPhaseSampler(maps.const[g])
    trm = maps.DeltatrackingTransmittance(sg, boundary, maj)
    d = torch.tensor(sun_dir, dtype=torch.float32)
    light = maps.DirectionalLight(d / d.norm(), sun_radiance)
    env_sampler = maps._functionsampler(maps.UniformDirectionSampler(6), envm)
    return maps.DeltatrackingNEEPathIntegrator(sg, alb, maps.ZERO, envm, env_sampler, ph, ps, boundary, maj, trm, 0.1,
                                               max_bounces=max_bounces, directional_light=light)


def camera_rays(pose: torch.Tensor, width: int, height: int, fov: float, znear: float, pixels: torch.Tensor,
                gen: torch.Generator) -> torch.Tensor:
    """Jittered rays [n, 6] through the given pixel indices (row * width + col),
    with the model of the perspective sensor (sensor_perspective_camera.h)."""
    dev = pixels.device
    o, dd, up = pose[0:3].double(), pose[3:6].double(), pose[6:9].double()
    z = dd / dd.norm()
    x = torch.linalg.cross(up, z)
    x = x / x.norm()
    y = torch.linalg.cross(z, x)
    row = (pixels // width).double()
    col = (pixels % width).double()
    j = torch.rand(pixels.shape[0], 2, generator=gen, dtype=torch.float64, device=dev)
    sx = ((col + j[:, 0]) * 2 - width) * znear / height
    sy = ((row + j[:, 1]) * 2 - height) * znear / height
    sz = znear / math.tan(fov * 0.5)
    w = x[None] * sx[:, None] + y[None] * sy[:, None] + z[None] * sz
    org = o[None] + w
    w = w / w.norm(dim=1, keepdim=True)
    return torch.cat([org, w], dim=1).float().contiguous()


def crop_pixels(width: int, height: int, crops: int, crop: int, seed: int = 0) -> torch.Tensor:
    """Pixel indices of `crops` square crops placed on a grid over the image."""
    g = np.random.default_rng(seed)
    k = int(math.ceil(math.sqrt(crops)))
    idx = []
    for c in range(crops):
        cy, cx = divmod(c, k)
        y0 = int((cy + 0.5) * height / k - crop / 2 + g.integers(-crop // 4, crop // 4 + 1))
        x0 = int((cx + 0.5) * width / k - crop / 2 + g.integers(-crop // 4, crop // 4 + 1))
        y0 = min(max(y0, 0), height - crop)
        x0 = min(max(x0, 0), width - crop)
        yy, xx = np.meshgrid(np.arange(y0, y0 + crop), np.arange(x0, x0 + crop), indexing="ij")
        idx.append((yy * width + xx).reshape(-1))
    return torch.from_numpy(np.concatenate(idx))


def reference_pixels(field, pose, width, height, fov, znear, pixels, spp, seed, chunk=1 << 22):
    """Mean radiance of `pixels` over spp jittered paths each (ray mode, NEE)."""
    dev = pixels.device
    ffi, lib = _lib.ffi_lib()
    desc = field.cast(input_dim=6).lower()
    m = desc.to_struct()
    gen = torch.Generator(device=dev).manual_seed(seed)
    acc = torch.zeros(pixels.shape[0], 3, dtype=torch.float64, device=dev)
    per = max(1, chunk // pixels.shape[0])
    done = 0
    out = torch.empty(per * pixels.shape[0], 3, device=dev)
    vctx = _lib.context(dev)
    while done < spp:
        k = min(per, spp - done)
        px = pixels.repeat(k)
        rays = camera_rays(pose, width, height, fov, znear, px, gen)
        o = out[: rays.shape[0]]
        _lib.check(lib.vrt_radiance_fw(vctx.ptr, m, 0, _lib.fptr(rays), rays.shape[0], seed * 1000003 + done,
                                       _lib.fptr(o), _lib.stream_handle(dev)), "vrt_radiance_fw")
        acc += o.double().reshape(k, pixels.shape[0], 3).sum(0)
        done += k
    return (acc / spp).float()


def reference_pixels_fp64(field, cam, pixels, spp, seed, chunk_paths=1 << 24):
    """FP64 mean radiance of `pixels` (row * width + col of view 0) over spp
    paths each, as float64 [n, 3]."""
    dev = pixels.device
    ffi, lib = _lib.ffi_lib()
    desc = field.cast(input_dim=6).lower()
    m = desc.to_struct()
    sens = torch.stack([torch.zeros_like(pixels), pixels // cam.width, pixels % cam.width], dim=-1).to(torch.int64)
    sens = sens.contiguous()
    c, keep = cam.to_struct(dev, sens)
    acc = torch.zeros(pixels.shape[0], 3, dtype=torch.float64, device=dev)
    out = torch.empty_like(acc)
    per = max(1, min(spp, chunk_paths // max(1, pixels.shape[0])))
    done, k = 0, 0
    vctx = _lib.context(dev)
    while done < spp:
        n = min(per, spp - done)
        _lib.check(lib.vrt_capture_fw_fp64(vctx.ptr, m, c, n, seed * 1000003 + k, ffi.cast("double *", out.data_ptr()),
                                           _lib.stream_handle(dev)), "vrt_capture_fw_fp64")
        acc += out * n
        done += n
        k += 1
    return acc / spp


class Timer:
    def __init__(self):
        self.total = 0.0

    def run(self, fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        self.total += a.elapsed_time(b) / 1000.0


def plain_curve(field, cam, pixels, ref, budget_s, spp_chunk, seed):
    """(seconds, mse) after every chunk of spp_chunk samples per pixel."""
    dev = pixels.device
    acc = torch.zeros(cam.views, cam.height, cam.width, 3, device=dev)
    t = Timer()
    curve = []
    n = 0
    while n == 0 or t.total < budget_s:
        img = {}
        t.run(lambda: img.setdefault("x", cam.capture(field, fw_samples=spp_chunk, seed=seed + n)))
        acc += img["x"]
        n += 1
        est = (acc / n).reshape(-1, 3)[pixels]
        curve.append((t.total, ((est - ref) ** 2).mean().item(), n * spp_chunk))
    return curve


def cached_curve(field, cam, pixels, ref, budget_s, spp, warmup, seed, **kw):
    dev = pixels.device
    r = cache.CachedRenderer(field, cam, seed=seed, **kw)
    t = Timer()

    def warm():
        for _ in range(warmup):
            r.train_frame()

    t.run(warm)
    acc = torch.zeros(cam.views, cam.height, cam.width, 3, device=dev)
    curve = []
    n = 0
    while n == 0 or t.total < budget_s:  # at least one frame, even when the warm-up used the budget
        def frame():
            r.train_frame()
            r.render_frame(acc, spp)
        t.run(frame)
        n += 1
        est = (acc / n).reshape(-1, 3)[pixels]
        curve.append((t.total, ((est - ref) ** 2).mean().item(), n * spp))
    r.check()
    return curve, float(r.last_loss)


def time_to_reach(curve, mse):
    for t, e, _ in curve:
        if e <= mse:
            return t
    return None


def equal_time(res=512, size=1024, max_sigma=200.0, crops=4, crop=32, ref_spp=4096, budget=20.0, plain_chunk=1,
               cache_budget=None, cache_spp=1, warmup=64, train_paths=1 << 14, train_cut=16, rec=4, cut=2, lr=1e-2,
               seed=11, curves=None):
    """Equal-time comparison of the cached renderer against the plain tracer on
    the cache workload; returns the summary dict (curves, when a list is
    given, receives the per-frame checkpoints)."""
    dev = torch.device("cuda", torch.cuda.current_device())
    maps.set_sync_checks(False)
    t0 = time.time()
    sigma = synthetic.value_noise(res, 6, max_sigma, seed, device=dev)
    field = build_field(sigma)
    poses = torch.from_numpy(synthetic.ring_poses(1, radius=2.0, elevation_deg=20.0)).to(dev)
    cam = maps.PerspectiveCameraSensor(size, size, poses, jittered=True)
    pixels = crop_pixels(size, size, crops, crop).to(dev)
    tr = Timer()
    ref = {}
    tr.run(lambda: ref.setdefault("x", reference_pixels_fp64(field, cam, pixels, ref_spp, seed=7)))
    ref = ref["x"].float()
    plain = plain_curve(field, cam, pixels, ref, budget, plain_chunk, seed=1000)
    cached, loss = cached_curve(field, cam, pixels, ref, cache_budget or budget, cache_spp, warmup, seed=5, cut=cut,
                                train_paths=train_paths, rec=rec, train_cut=train_cut, lr=lr)
    if curves is not None:
        for name, curve in (("plain", plain), ("cached", cached)):
            for t, e, s in curve:
                curves.append(dict(method=name, seconds=round(t, 4), mse=e, spp=s))
    target = plain[-1][1]
    t_cache = time_to_reach(cached, target)
    maps.check()
    return dict(
        workload="radiance_cache_512" if (res, size) == (512, 1024) else f"noise_{res}_{size}",
        res=res, size=size, max_sigma=max_sigma, eval_pixels=int(pixels.shape[0]), oracle="fp64",
        ref_spp=ref_spp, ref_seconds=round(tr.total, 3), ref_pixel_mean=float(ref.mean()),
        plain_seconds=round(plain[-1][0], 3), plain_spp=plain[-1][2], plain_mse=target,
        cached_seconds_to_plain_mse=None if t_cache is None else round(t_cache, 3),
        speedup=None if t_cache is None else round(plain[-1][0] / t_cache, 2),
        cached_final_mse=cached[-1][1], cached_final_seconds=round(cached[-1][0], 3), cached_spp=cached[-1][2],
        cache_loss=loss, cut=cut, train_cut=train_cut, train_paths=train_paths, rec=rec, warmup_frames=warmup,
        wall_s=round(time.time() - t0, 1))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--res", type=int, default=512)
    ap.add_argument("--size", type=int, default=1024)
    ap.add_argument("--max-sigma", type=float, default=200.0)
    ap.add_argument("--crops", type=int, default=4)
    ap.add_argument("--crop", type=int, default=32)
    ap.add_argument("--ref-spp", type=int, default=4096)
    ap.add_argument("--budget", type=float, default=20.0, help="seconds of plain-tracer rendering")
    ap.add_argument("--plain-chunk", type=int, default=1)
    ap.add_argument("--cache-budget", type=float, default=None)
    ap.add_argument("--cache-spp", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=64)
    ap.add_argument("--train-paths", type=int, default=1 << 14)
    ap.add_argument("--train-cut", type=int, default=16)
    ap.add_argument("--rec", type=int, default=4)
    ap.add_argument("--cut", type=int, default=2)
    ap.add_argument("--lr", type=float, default=1e-2)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--out", type=str, default=None)
    args = ap.parse_args(argv)
    torch.cuda.set_device(0)
    lines = []
    summary = equal_time(res=args.res, size=args.size, max_sigma=args.max_sigma, crops=args.crops, crop=args.crop,
                         ref_spp=args.ref_spp, budget=args.budget, plain_chunk=args.plain_chunk,
                         cache_budget=args.cache_budget, cache_spp=args.cache_spp, warmup=args.warmup,
                         train_paths=args.train_paths, train_cut=args.train_cut, rec=args.rec, cut=args.cut,
                         lr=args.lr, seed=args.seed, curves=lines)
    for l in lines:
        print(json.dumps(l))
    print(json.dumps(summary))
    if args.out:
        with open(args.out, "w") as f:
            json.dump(dict(summary=summary, curve=lines), f, indent=1)
    return summary


if __name__ == "__main__":
    main()
