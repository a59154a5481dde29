"""Radiance-cache rendering path on the GPU: the unbiased prefix with its cache
queries, the training samples, the resolve step, and what the trained cache
gains over the plain tracer.  Needs a B200.

Prefix and training samples share the Philox keys of the CPU oracle
(oracle.capture_prefix / oracle.train_samples), so rows are compared path for
path; >= 99% of rows must agree within rtol 1e-3 (float rounding lets a few
stochastic paths branch differently, as in the plain capture tests).
"""
import math
import time

import numpy as np
import pytest
import torch

import oracle
from rendervous_b200 import _lib, cache, maps, synthetic
from tests.helpers import build_field, front_camera

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _setup(cuda):
    maps.set_sync_checks(True)
    yield


def _field(cuda, res=32, max_sigma=60.0, albedo=0.95, g=0.6, tr="dt", majorant="grid", max_bounces=0):
    sig = torch.from_numpy(synthetic.value_noise(res, 3, max_sigma, seed=21)).to(cuda)
    return build_field(sig, albedo=albedo, env=1.0, sun_dir=(0.3, 0.8, 0.5), sun_radiance=3.0, g=g,
                       majorant=majorant, tr=tr, max_bounces=max_bounces)


def _camera(cuda, H, W):
    return maps.PerspectiveCameraSensor(W, H, front_camera(1).to(cuda), jittered=True)


def _prefix_gpu(field, cam, spp, seed, cut, cuda):
    ffi, lib = _lib.ffi_lib()
    desc = field.cast(input_dim=6).lower()
    m = desc.to_struct()
    c, keep = cam.to_struct(cuda)
    rgb = torch.zeros(1, cam.height, cam.width, 3, device=cuda)
    n = cam.height * cam.width * spp
    q = torch.empty(3, n, 3, device=cuda)
    _lib.check(lib.vrt_capture_prefix_fw(_lib.context(cuda).ptr, m, c, spp, seed, cut, _lib.fptr(rgb), _lib.fptr(q),
                                         _lib.stream_handle(cuda)))
    assert maps.check()["status"] == 0
    return rgb, q, desc


def _oracle_scene(desc):
    return oracle.OracleScene(desc.to_numpy())


def _rows_close(a, b, rtol=1e-3, atol=1e-5):
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    both_nan = np.isnan(a) & np.isnan(b)
    ok = np.isclose(a, b, rtol=rtol, atol=atol) | both_nan
    return ok.all(axis=1)


@pytest.mark.parametrize("cut", [0, 2, 5])
def test_prefix_matches_oracle(cuda, cut):
    field = _field(cuda)
    H = W = 32
    spp = 4
    cam = _camera(cuda, H, W)
    rgb, q, desc = _prefix_gpu(field, cam, spp, 77, cut, cuda)
    ref_rgb, ref_q = oracle.capture_prefix(_oracle_scene(desc), front_camera(1).numpy(), W, H, math.pi / 4, True,
                                           spp, 77, cut)
    close = np.isclose(rgb.cpu().numpy(), ref_rgb, rtol=1e-3, atol=1e-5).all(axis=-1)
    assert close.mean() >= 0.99, close.mean()
    qg = q.cpu().numpy().transpose(1, 0, 2)      # rows: (position, direction, W)
    qr = ref_q.transpose(1, 0, 2)
    rows = _rows_close(qg, qr)
    assert rows.mean() >= 0.99, rows.mean()
    assert (qr[:, 2].max(axis=1) > 0).mean() > 0.05  # a share of paths reach the cut


def test_prefix_without_cut_is_the_plain_capture(cuda):
    field = _field(cuda, max_bounces=24)
    H = W = 32
    spp = 4
    cam = _camera(cuda, H, W)
    rgb, q, _ = _prefix_gpu(field, cam, spp, 5, 1000, cuda)
    plain = cam.capture(field, fw_samples=spp, seed=5)
    # the same paths; only the order of the per-pixel atomic sums differs
    assert torch.allclose(rgb, plain, rtol=1e-5, atol=1e-7)
    assert torch.all(q[2] == 0)


@pytest.mark.parametrize("self_train", [False, True])
def test_train_samples_match_oracle(cuda, self_train):
    """Full training paths, and self-training paths stopped into a cache whose
    weights are all zero (it returns exactly 0, so the oracle's truncated
    paths are the reference)."""
    field = _field(cuda)
    H = W = 32
    cam = _camera(cuda, H, W)
    desc = field.cast(input_dim=6).lower()
    ffi, lib = _lib.ffi_lib()
    n_paths, rec, cut = 3000, 4, 6
    smp = torch.empty(4, n_paths * rec, 3, device=cuda)
    work = torch.empty(12 * n_paths, device=cuda)
    c, keep = cam.to_struct(cuda)
    rc = cache.RadianceCache([-1, -1, -1], [1, 1, 1], cuda, n_min=4, n_max=24)
    rc.params.zero_()
    cs = rc.struct() if self_train else ffi.NULL
    _lib.check(lib.vrt_capture_train_samples(_lib.context(cuda).ptr, desc.to_struct(), c, cs, cut, n_paths, 99, rec,
                                             _lib.fptr(smp), _lib.fptr(work), _lib.stream_handle(cuda)))
    assert maps.check()["status"] == 0
    ref = oracle.train_samples(_oracle_scene(desc), front_camera(1).numpy(), W, H, math.pi / 4, True, n_paths, 99,
                               rec, cut if self_train else -1)
    g = smp.cpu().numpy().transpose(1, 0, 2)
    r = ref.transpose(1, 0, 2)
    rows = _rows_close(g, r, rtol=2e-3, atol=1e-5)
    assert rows.mean() >= 0.99, rows.mean()
    valid = np.isfinite(r[:, 2]).all(axis=1)
    assert valid.mean() > 0.3
    assert np.all(r[valid, 2] >= -1e-6)           # in-scattered radiance is non-negative
    assert np.all(r[valid, 3] > 0)


def test_resolve_accumulates_weighted_cache(cuda):
    rc = cache.RadianceCache([-1, -1, -1], [1, 1, 1], cuda, n_min=4, n_max=24, seed=5, grid_init=0.3)
    n, npix = 5000, 777
    g = torch.Generator().manual_seed(3)
    pos = (torch.rand(n, 3, generator=g) * 2 - 1).to(cuda)
    d = torch.nn.functional.normalize(torch.randn(n, 3, generator=g), dim=1).to(cuda)
    W = torch.rand(n, 3, generator=g).to(cuda)
    W[::3] = 0.0                                     # rows without a query
    q = torch.stack([pos, d, W]).contiguous()
    rgb = torch.zeros(npix, 3, device=cuda)
    ffi, lib = _lib.ffi_lib()
    _lib.check(lib.vrt_cache_resolve(rc.struct(), _lib.fptr(q), n, npix, 0.25, _lib.fptr(rgb),
                                     _lib.stream_handle(cuda)))
    y = rc.infer(pos, d)
    ref = torch.zeros(npix, 3, device=cuda).index_add_(0, torch.arange(n, device=cuda) % npix, 0.25 * W * y)
    assert torch.allclose(rgb, ref, rtol=1e-4, atol=1e-6)


def test_trained_cache_beats_plain_tracer_at_equal_time(cuda):
    """Dense, high-albedo medium (long paths): the cached renderer, warm-up
    training included in its time, reaches a lower error against a high-spp
    FP64 plain estimate of a set of crops than the plain tracer given the same
    measured GPU time."""
    from rendervous_b200 import cache_eval
    maps.set_sync_checks(False)
    try:
        sigma = synthetic.value_noise(96, 6, 200.0, seed=11, device=cuda)
        field = cache_eval.build_field(sigma)
        size = 128
        poses = torch.from_numpy(synthetic.ring_poses(1, radius=2.0, elevation_deg=20.0)).to(cuda)
        cam = maps.PerspectiveCameraSensor(size, size, poses, jittered=True)
        pixels = cache_eval.crop_pixels(size, size, 4, 16).to(cuda)
        ref = cache_eval.reference_pixels_fp64(field, cam, pixels, 2048, seed=7).float()
        cached, loss = cache_eval.cached_curve(field, cam, pixels, ref, 0.4, 1, 32, seed=5, train_paths=1 << 12)
        t_cache, mse_cache = cached[-1][0], cached[-1][1]
        plain = cache_eval.plain_curve(field, cam, pixels, ref, t_cache, 1, seed=1000)
        t_plain, mse_plain = plain[-1][0], plain[-1][1]
        print(f"cached {t_cache:.3f}s mse {mse_cache:.3e} ({cached[-1][2]} spp) | "
              f"plain {t_plain:.3f}s mse {mse_plain:.3e} ({plain[-1][2]} spp) | loss {loss:.3e}")
        assert t_plain >= t_cache
        assert mse_cache < mse_plain, (mse_cache, mse_plain)
    finally:
        maps.set_sync_checks(True)


def test_fp64_capture_matches_the_fp64_oracle(cuda):
    """The FP64 reference tracer (the estimate the cache's error is measured
    against) follows the oracle's double-precision NEE path for path on a
    32 x 32 crop of a dense, high-albedo medium like the cache benchmark's
    (six-octave noise, albedo 0.99, g 0.8, delta-tracking shadows, 8^3
    bricks): >= 98 % of pixels within 1e-9 relative; the FP32 tracer takes the
    same paths for >= 90 % of the pixels (within 1e-3)."""
    import math
    from rendervous_b200 import _lib
    from rendervous_b200.cache_eval import build_field
    ffi, lib = _lib.ffi_lib()
    sigma = synthetic.value_noise(65, 6, 200.0, 11, device=cuda)
    field = build_field(sigma, max_bounces=512)
    poses = torch.from_numpy(synthetic.ring_poses(1, radius=2.0, elevation_deg=20.0)).to(cuda)
    cam = maps.PerspectiveCameraSensor(128, 128, poses, jittered=True)
    rr, cc = np.meshgrid(np.arange(48, 80), np.arange(48, 80), indexing="ij")
    sens_np = np.stack([np.zeros_like(rr), rr, cc], -1).reshape(-1, 3).astype(np.int64)
    sens = torch.from_numpy(sens_np).to(cuda)
    desc = field.lower()
    c, keep = cam.to_struct(cuda, sens)
    out = torch.empty(sens.shape[0], 3, dtype=torch.float64, device=cuda)
    _lib.check(lib.vrt_capture_fw_fp64(_lib.context(cuda).ptr, desc.to_struct(), c, 2, 5,
                                       ffi.cast("double *", out.data_ptr()), _lib.stream_handle(cuda)))
    maps.check()
    got = out.cpu().numpy()
    sc = oracle.OracleScene(desc.to_numpy())
    ref = oracle.capture_fw_fp64(sc, poses.cpu().numpy(), 128, 128, math.pi / 4, True, 2, 5, sensors=sens_np)
    close = np.isclose(got, ref, rtol=1e-9, atol=1e-12).all(axis=-1)
    assert close.mean() >= 0.98, close.mean()
    f32 = cam.capture(field, sensors_batch=sens, fw_samples=2, seed=5).cpu().numpy().astype(np.float64)
    assert np.isclose(f32, got, rtol=1e-3, atol=1e-5).all(axis=-1).mean() >= 0.9   # mostly the same paths
