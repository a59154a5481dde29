"""The benchmark workloads at their stated sizes: CUDA path vs the oracle,
through the C ABI (needs a B200).

* the timed workload of bench.py itself (256^3 blob sigma, 256^3 albedo grid,
  HG g = 0.6, at most 64 bounces, ratio-tracking shadows over 8^3 bricks,
  environment + sun, NEE_DS adjoint) on a 32 x 32 crop of its 512 x 512
  camera (a sensors batch) at 4 spp: image and both gradients path for path;
* the plain forward workload (64^3 blobs, 128 x 128, 16 spp, 16 bounces)
  at its full size, path for path;
* the DDA transmittance workload (256^3 four-octave noise, 2^20 rays):
  the adjoint against FP64 central differences on 64 seeded voxels.

Tolerances are written in each test.
"""
import math

import numpy as np
import pytest
import torch

import bench
import oracle
from rendervous_b200 import maps, synthetic
from rendervous_b200.lowering import lower_transmittance_map

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _setup(cuda):
    maps.set_sync_checks(True)
    yield


def test_bench_workload_on_a_crop_matches_oracle(cuda):
    wl, sigma, albedo, target_sigma, sun, poses = bench.workload_arrays()
    sig_p = torch.nn.Parameter(torch.from_numpy(sigma).to(cuda))
    alb_p = torch.nn.Parameter(torch.from_numpy(albedo).to(cuda))
    field = bench.build_field(sig_p, alb_p, wl, sun)
    cam = maps.PerspectiveCameraSensor(wl["width"], wl["height"], torch.from_numpy(poses).to(cuda), jittered=True)
    # the 32 x 32 pixels at the centre of the 512 x 512 view, as a sensors batch
    r0 = wl["height"] // 2 - 16
    c0 = wl["width"] // 2 - 16
    rr, cc = np.meshgrid(np.arange(r0, r0 + 32), np.arange(c0, c0 + 32), indexing="ij")
    sensors_np = np.stack([np.zeros_like(rr), rr, cc], axis=-1).astype(np.int64)
    sensors = torch.from_numpy(sensors_np).to(cuda)
    spp, seed = 4, 4242
    img = cam.capture(field, sensors_batch=sensors, fw_samples=spp, bw_samples=spp, seed=seed)
    assert tuple(img.shape) == (32, 32, 3)
    dimg = torch.from_numpy(np.random.default_rng(1).random(img.shape).astype(np.float32)).to(cuda)
    (img * dimg).sum().backward()

    sc = oracle.OracleScene(field.lower().to_numpy(), with_grads=True)
    ref, cnt = oracle.capture_fw(sc, "nee", poses, wl["width"], wl["height"], math.pi / 4, True, spp, seed,
                                 sensors=sensors_np)
    oracle.capture_bw(sc, "ds", poses, wl["width"], wl["height"], math.pi / 4, True, spp, seed,
                      dimg.cpu().numpy(), sensors=sensors_np)
    a = img.detach().cpu().numpy()
    assert cnt["vertices"] > 10 * 32 * 32                 # the crop scatters (several vertices per path)
    close = np.isclose(a, ref, rtol=1e-3, atol=1e-5).all(axis=-1)
    assert close.mean() >= 0.99, close.mean()             # >= 99% of pixels agree path for path
    for grad, refg in ((sig_p.grad, sc.sigma_grad), (alb_p.grad, sc.albedo_grad)):
        g = grad.cpu().numpy()
        rel = np.abs(g - refg).sum() / max(np.abs(refg).sum(), 1e-30)
        assert np.abs(refg).sum() > 0 and rel < 1e-2, rel  # relative L1 of the whole gradient grid


def test_sensors_batch_of_every_pixel_equals_the_full_capture(cuda):
    """A sensors batch that lists every pixel in raster order runs the same
    Philox paths as the full capture (sample s of pixel p is path s*npix + p)."""
    wl = synthetic.WORKLOADS["plain_forward_64"]
    sig = torch.from_numpy(synthetic.make_sigma(wl["sigma"])).to(cuda)
    from tests.helpers import build_field, front_camera
    field = build_field(sig, albedo=0.9, env=1.0, sun_dir=(0.3, 0.8, 0.5), g=0.3, max_bounces=16,
                        majorant="grid", brick=8)
    H, W = 24, 40
    cam = maps.PerspectiveCameraSensor(W, H, front_camera(2).to(cuda), jittered=True)
    full = cam.capture(field, fw_samples=4, seed=77)
    idx = torch.stack(torch.meshgrid(torch.arange(2), torch.arange(H), torch.arange(W), indexing="ij"), -1)
    part = cam.capture(field, sensors_batch=idx.reshape(-1, 3).to(cuda), fw_samples=4, seed=77)
    close = torch.isclose(part.reshape(full.shape), full, rtol=1e-5, atol=1e-6).all(-1).float().mean()
    assert float(close) >= 0.999
    rnd = cam.random_sensors(100)
    assert rnd.shape == (100, 3) and rnd.dtype == torch.int64
    assert int(rnd[:, 1].max()) < H and int(rnd[:, 2].max()) < W and int(rnd.min()) >= 0
    with pytest.raises(IndexError):
        cam.capture(field, sensors_batch=torch.tensor([[0, H, 0]], device=cuda), fw_samples=1, seed=1)


def test_plain_forward_workload_full_size_matches_oracle(cuda):
    wl = synthetic.WORKLOADS["plain_forward_64"]
    from tests.helpers import build_field
    sig = torch.from_numpy(synthetic.make_sigma(wl["sigma"])).to(cuda)
    sun = tuple(float(v) for v in synthetic.gaussian_direction(wl["sun_seed"]))
    field = build_field(sig, albedo=wl["albedo"], env=wl["env"], sun_dir=sun, sun_radiance=wl["sun_intensity"],
                        g=wl["phase_g"], max_bounces=wl["max_bounces"])
    H, W, spp = wl["height"], wl["width"], wl["spp"]            # 128 x 128 x 16 spp
    poses = synthetic.ring_poses(wl["views"])
    cam = maps.PerspectiveCameraSensor(W, H, torch.from_numpy(poses).to(cuda), jittered=True)
    img = cam.capture(field, fw_samples=spp, seed=wl["render_seed"]).cpu().numpy()
    sc = oracle.OracleScene(field.lower().to_numpy())
    ref, cnt = oracle.capture_fw(sc, "nee", poses, W, H, math.pi / 4, True, spp, wl["render_seed"])
    close = np.isclose(img, ref, rtol=1e-3, atol=1e-5).all(axis=-1)
    assert close.mean() >= 0.99, close.mean()
    assert abs(img.mean() - ref.mean()) <= 1e-3 * abs(ref.mean())
    assert cnt["paths"] == H * W * spp


def test_dda_workload_adjoint_matches_fp64_central_differences(cuda):
    """dL/dsigma of L = sum_i w_i T_i on the 256^3 noise grid and 2^20 rays, at
    64 seeded voxels, against FP64 central differences of the same midpoint
    DDA (tau is linear in sigma, so the difference is exact up to the
    exponential's curvature).  Only rays that cross the 2x2x2 cells around a
    voxel can change with it; the differences are taken over those."""
    wl = synthetic.WORKLOADS["dda_transmittance_256"]
    sig_np = synthetic.make_sigma(wl["sigma"])
    t = torch.nn.Parameter(torch.from_numpy(sig_np).to(cuda))
    bmin, bmax = maps.normalized_box(t)
    g = maps.Grid3D(t, bmin, bmax)
    tr = maps.GridDDATransmittance(g, maps.ray_box_intersection[bmin, bmax])
    rays_np = synthetic.sphere_rays(wl["n_rays"], seed=wl["ray_seed"])
    w_np = synthetic.uniform_weights(wl["n_rays"], wl["weight_seed"])
    T = tr(torch.from_numpy(rays_np).to(cuda))[:, 0]
    (T * torch.from_numpy(w_np).to(cuda)).sum().backward()
    grad = t.grad.cpu().numpy()[..., 0]

    desc = lower_transmittance_map(tr).to_numpy()
    res = sig_np.shape[0]
    vox = np.random.default_rng(wl["weight_seed"] + 100).integers(1, res - 1, size=(64, 3))  # (z, y, x)
    bmin_np = bmin.numpy().astype(np.float64)
    cell = (bmax.numpy().astype(np.float64) - bmin_np) / (res - 1)
    o = rays_np[:, :3].astype(np.float64)
    d = rays_np[:, 3:].astype(np.float64)
    inv = 1.0 / np.where(np.abs(d) < 1e-12, 1e-12, d)
    errs = []
    for z, y, x in vox:
        # rays through the box of the 8 cells that share node (x, y, z), widened by a cell
        lo = bmin_np + (np.array([x, y, z]) - 2) * cell
        hi = bmin_np + (np.array([x, y, z]) + 2) * cell
        t0 = (lo - o) * inv
        t1 = (hi - o) * inv
        tn = np.minimum(t0, t1).max(axis=1)
        tf = np.maximum(t0, t1).min(axis=1)
        sel = np.nonzero(tf >= np.maximum(tn, 0.0))[0]
        h = 1e-3 * max(1.0, float(sig_np[z, y, x, 0]))
        taus = []
        for sgn in (1.0, -1.0):
            sp = sig_np.copy()
            sp[z, y, x, 0] = np.float32(sig_np[z, y, x, 0] + sgn * h)
            dd = dict(desc)
            dd["sigma"] = sp
            taus.append(oracle.dda_tau_fp64(oracle.OracleScene(dd), rays_np[sel]))
        hp = float(np.float32(sig_np[z, y, x, 0] + h)) - float(np.float32(sig_np[z, y, x, 0] - h))
        fd = float((w_np[sel].astype(np.float64) * (np.exp(-taus[0]) - np.exp(-taus[1]))).sum() / hp)
        errs.append(abs(grad[z, y, x] - fd) / max(abs(fd), 1e-3 * np.abs(grad).max()))
    errs = np.array(errs)
    assert np.median(errs) < 1e-4 and errs.max() < 1e-3, (np.median(errs), errs.max())


def test_uncapped_paths_run_on_the_wavefront(cuda):
    """The reference's default (no bounce cap) runs on the wavefront kernels.  In
    a dense, high-albedo medium many paths outlive the 64-vertex pass: with the
    automatic buffers they go on in place; with a round capped at 4096 items
    the forward saves and resumes them in later rounds and the NEE_DS adjoint
    hands them to the state machine.  Image and gradients match the oracle's
    uncapped paths either way."""
    from rendervous_b200 import _lib
    from tests.helpers import build_field, front_camera
    ffi, lib = _lib.ffi_lib()
    ctx = _lib.context(cuda)
    stream = _lib.stream_handle(cuda)
    sig = torch.from_numpy(synthetic.gaussian_blobs(33, 6, 80.0, seed=4)).to(cuda)
    H = W = 24
    cam = maps.PerspectiveCameraSensor(W, H, front_camera(1).to(cuda), jittered=True)
    dimg = torch.from_numpy(np.random.default_rng(6).random((1, H, W, 3)).astype(np.float32)).to(cuda)
    ks = ffi.new("vrt_kernel_stat[]", lib.VRT_K_COUNT)
    runs = []
    for limit in (0, 4096):
        alb = torch.nn.Parameter(torch.full((33, 33, 33, 3), 0.985, device=cuda))
        field = build_field(sig, albedo_grid=alb, env=1.0, sun_dir=(0.3, 0.8, 0.5), sun_radiance=2.0, g=0.3,
                            max_bounces=0, majorant="grid", brick=4, sigma_requires_grad=True)
        _lib.check(lib.vrt_set_wave_batch_limit(ctx.ptr, limit))
        try:
            maps.check()
            _lib.check(lib.vrt_kernel_stats(ctx.ptr, stream, ks))
            img = cam.capture(field, fw_samples=4, bw_samples=4, seed=21)
            (img * dimg).sum().backward()
            maps.check()
            _lib.check(lib.vrt_kernel_stats(ctx.ptr, stream, ks))
        finally:
            _lib.check(lib.vrt_set_wave_batch_limit(ctx.ptr, 0))
        runs.append((img.detach().cpu().numpy(), field.sigma.grid.grad.cpu().numpy(), alb.grad.cpu().numpy(),
                     ks[lib.VRT_K_WALK_FW].launches, ks[lib.VRT_K_DS_PRIMAL].launches))
    assert runs[0][3] >= 1 and runs[0][4] >= 1                 # the wavefront ran
    assert runs[1][3] >= 2                                     # small rounds: paths were saved and resumed
    field = build_field(sig, albedo=0.985, env=1.0, sun_dir=(0.3, 0.8, 0.5), sun_radiance=2.0, g=0.3,
                        max_bounces=0, majorant="grid", brick=4)
    d = field.lower()
    d.albedo_grid = torch.full((33, 33, 33, 3), 0.985)
    sc = oracle.OracleScene(d.to_numpy(), with_grads=True)
    ref, cnt = oracle.capture_fw(sc, "nee", front_camera(1).numpy(), W, H, math.pi / 4, True, 4, 21)
    oracle.capture_bw(sc, "ds", front_camera(1).numpy(), W, H, math.pi / 4, True, 4, 21, dimg.cpu().numpy())
    assert cnt["vertices"] > 64 * 50                            # long paths exist
    for img, gs, ga, _, _ in runs:
        close = np.isclose(img, ref, rtol=1e-3, atol=1e-5).all(axis=-1)
        assert close.mean() >= 0.98, close.mean()
        for g, rg in ((gs, sc.sigma_grad), (ga, sc.albedo_grad)):
            rel = np.abs(g - rg).sum() / max(np.abs(rg).sum(), 1e-30)
            assert rel < 2e-2, rel
