"""Seeded synthetic volumes, rays and cameras for the benchmark workloads.

All generators run on the CPU in float64 and return contiguous float32 numpy
arrays, so the CUDA path and the CPU oracle see identical bytes.  No dataset
is involved: the workloads are defined by their shapes, sizes and value
distributions only.

Grids are node-centred ``[D, H, W, 1]`` tensors over the box that
``normalized_box`` gives (``[-0.5, 0.5]^3`` for a cube, reference
``_maps.py:4780-4788``); node ``i`` of an axis sits at unit coordinate
``i / (n - 1)``.
"""
from __future__ import annotations

import math

import numpy as np


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(int(seed)))


def gaussian_blobs(res: int, n_blobs: int, max_sigma: float, seed: int,
                   centre_range=(0.2, 0.8), std_range=(0.05, 0.15)) -> np.ndarray:
    """Sum of isotropic Gaussians (centres U[centre_range]^3, std U[std_range]),
    rescaled so that the maximum node value is ``max_sigma``.

    Separable evaluation: sigma[z,y,x] = sum_b gz[b,z] gy[b,y] gx[b,x], done as
    one (res*res, n_blobs) x (n_blobs, res) matrix product.
    """
    g = _rng(seed)
    centres = g.uniform(centre_range[0], centre_range[1], size=(n_blobs, 3))
    stds = g.uniform(std_range[0], std_range[1], size=(n_blobs,))
    u = np.arange(res, dtype=np.float64) / (res - 1)
    gx = np.exp(-0.5 * ((u[None, :] - centres[:, 0:1]) / stds[:, None]) ** 2)
    gy = np.exp(-0.5 * ((u[None, :] - centres[:, 1:2]) / stds[:, None]) ** 2)
    gz = np.exp(-0.5 * ((u[None, :] - centres[:, 2:3]) / stds[:, None]) ** 2)
    a = (gz[:, :, None] * gy[:, None, :]).reshape(n_blobs, res * res)  # (b, z*y)
    vol = (a.T @ gx).reshape(res, res, res)
    vol *= max_sigma / vol.max()
    return np.ascontiguousarray(vol.astype(np.float32)[..., None])


def _interp_matrix(res: int, freq: int) -> np.ndarray:
    """(res, freq+1) linear-interpolation weights of node positions on a lattice."""
    u = np.arange(res, dtype=np.float64) / (res - 1) * freq
    i0 = np.minimum(np.floor(u).astype(np.int64), freq - 1)
    a = u - i0
    m = np.zeros((res, freq + 1))
    m[np.arange(res), i0] = 1.0 - a
    m[np.arange(res), i0 + 1] += a
    return m


def value_noise(res: int, octaves: int, max_sigma: float, seed: int, base_freq: int = 4, device=None):
    """Multi-octave value noise: octave o is the trilinear interpolation of a
    (f+1)^3 lattice of U[0,1) values with f = base_freq * 2^o, weighted 0.5^o.
    The sum is centred on its expected value, clamped at 0 and scaled to
    ``max_sigma``, which leaves roughly half of the box empty.  With a torch
    ``device`` the same lattices are interpolated there (float64) and a
    [res,res,res,1] float32 tensor is returned.
    """
    if device is not None:
        return _value_noise_torch(res, octaves, max_sigma, seed, base_freq, device)
    g = _rng(seed)
    vol = np.zeros((res, res, res), np.float64)
    amp_total = 0.0
    for o in range(octaves):
        f = base_freq * (2 ** o)
        amp = 0.5 ** o
        lat = g.uniform(0.0, 1.0, size=(f + 1, f + 1, f + 1))
        m = _interp_matrix(res, f)
        # mode products: x, then y, then z
        t = np.einsum("abc,xc->abx", lat, m)
        t = np.einsum("abx,yb->ayx", t, m)
        t = np.einsum("ayx,za->zyx", t, m)
        vol += amp * t
        amp_total += amp
    vol -= 0.5 * amp_total
    np.maximum(vol, 0.0, out=vol)
    vol *= max_sigma / vol.max()
    return np.ascontiguousarray(vol.astype(np.float32)[..., None])


def _value_noise_torch(res, octaves, max_sigma, seed, base_freq, device):
    import torch
    g = _rng(seed)
    vol = torch.zeros(res, res, res, dtype=torch.float64, device=device)
    amp_total = 0.0
    for o in range(octaves):
        f = base_freq * (2 ** o)
        amp = 0.5 ** o
        lat = torch.from_numpy(g.uniform(0.0, 1.0, size=(f + 1, f + 1, f + 1))).to(device)
        m = torch.from_numpy(_interp_matrix(res, f)).to(device)
        t = torch.einsum("abc,xc->abx", lat, m)
        t = torch.einsum("abx,yb->ayx", t, m)
        vol += amp * torch.einsum("ayx,za->zyx", t, m)
        amp_total += amp
        del t
    vol -= 0.5 * amp_total
    vol.clamp_(min=0.0)
    vol *= max_sigma / vol.max()
    return vol.to(torch.float32).unsqueeze(-1).contiguous()


def uniform_grid(res: int, lo: float, hi: float, seed: int, channels: int = 1) -> np.ndarray:
    g = _rng(seed)
    return np.ascontiguousarray(g.uniform(lo, hi, size=(res, res, res, channels)).astype(np.float32))


def sphere_rays(n: int, seed: int, radius: float = 1.5, box=(-0.5, 0.5)) -> np.ndarray:
    """Origins uniform on the sphere of ``radius``, each aimed at a uniform
    point of the box; returns (n, 6) rays with unit directions."""
    g = _rng(seed)
    o = g.normal(size=(n, 3))
    o *= radius / np.linalg.norm(o, axis=1, keepdims=True)
    tgt = g.uniform(box[0], box[1], size=(n, 3))
    w = tgt - o
    w /= np.linalg.norm(w, axis=1, keepdims=True)
    return np.ascontiguousarray(np.concatenate([o, w], axis=1).astype(np.float32))


def uniform_weights(n: int, seed: int) -> np.ndarray:
    return np.ascontiguousarray(_rng(seed).uniform(0.0, 1.0, size=(n,)).astype(np.float32))


def gaussian_direction(seed: int) -> np.ndarray:
    v = _rng(seed).normal(size=3)
    return (v / np.linalg.norm(v)).astype(np.float32)


def ring_poses(views: int, radius: float = 2.0, elevation_deg: float = 20.0, target=(0.0, 0.0, 0.0)) -> np.ndarray:
    """(views, 9) camera poses (origin, direction, up) evenly spaced on a ring
    around ``target`` -- the layout PerspectiveCameraSensor expects."""
    el = math.radians(elevation_deg)
    poses = []
    for i in range(views):
        az = 2 * math.pi * i / views
        o = np.array([radius * math.cos(el) * math.sin(az), radius * math.sin(el), radius * math.cos(el) * math.cos(az)])
        d = np.asarray(target) - o
        d /= np.linalg.norm(d)
        poses.append(np.concatenate([o, d, [0.0, 1.0, 0.0]]))
    return np.ascontiguousarray(np.array(poses, np.float32))


# ---------------------------------------------------------------------------
# The benchmark workloads, by name.
# ---------------------------------------------------------------------------
WORKLOADS = {
    "plain_forward_64": dict(
        sigma=("blobs", dict(res=64, n_blobs=12, max_sigma=20.0, seed=1)),
        albedo=0.9, phase_g=0.0, env=1.0, sun_intensity=3.0, sun_seed=1,
        width=128, height=128, spp=16, max_bounces=16, views=1, render_seed=2),
    # the one-path-per-thread adjoints (DT, DRT, DRTQ, DRTDS, SPS) beside the NEE_DS wavefront, on the
    # first configuration's medium with a trainable sigma
    "path_adjoints_64": dict(
        sigma=("blobs", dict(res=64, n_blobs=12, max_sigma=20.0, seed=1)),
        albedo=0.9, phase_g=0.4, env=1.0, sun_intensity=3.0, sun_seed=1, ds_epsilon=0.1,
        width=128, height=128, spp=4, max_bounces=16, views=1),
    "dda_transmittance_256": dict(
        sigma=("noise", dict(res=256, octaves=4, max_sigma=50.0, seed=3)),
        n_rays=1 << 20, ray_seed=4, weight_seed=5, brick=8),
    "differentiable_pt_256": dict(
        sigma=("blobs", dict(res=256, n_blobs=64, max_sigma=40.0, seed=6)),
        albedo=("uniform", dict(res=256, lo=0.6, hi=0.95, seed=8)), phase_g=0.6, env=1.0, sun_intensity=3.0,
        sun_seed=6, width=512, height=512, spp=64, max_bounces=64, views=1, render_seed=9, target_seed=7),
    # the target: a 256^3 seeded blob volume like the differentiable tracer's (64 blobs, max sigma 40),
    # with its own seed
    "inverse_rendering_128": dict(
        target_sigma=("blobs", dict(res=256, n_blobs=64, max_sigma=40.0, seed=10)), res=128, init_sigma=1.0,
        albedo=0.9, phase_g=0.3, views=8, width=256, height=256, target_spp=128, spp=16, max_bounces=32,
        lr=0.01, iterations=500),
    "radiance_cache_512": dict(
        sigma=("noise", dict(res=512, octaves=6, max_sigma=200.0, seed=11)),
        albedo=0.99, phase_g=0.8, width=1024, height=1024),
}


def make_sigma(kind_args) -> np.ndarray:
    kind, args = kind_args
    if kind == "blobs":
        return gaussian_blobs(**args)
    if kind == "noise":
        return value_noise(**args)
    raise ValueError(kind)
