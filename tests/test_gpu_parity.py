"""CUDA path vs the CPU oracle, through the C ABI (needs a B200).

Same inputs and the same Philox keys on both sides, so most paths agree draw
for draw; float rounding (FMA contraction, libm vs CUDA transcendentals) lets a
tiny fraction of stochastic paths take a different branch, which the tests
bound explicitly.  Deterministic quantities (DDA, grids, majorants) are
compared element-wise.  Tolerances are written in each test.
"""
import math

import numpy as np
import pytest
import torch

import oracle
from rendervous_b200 import _lib, maps, synthetic
from tests.helpers import build_field, front_camera, homogeneous

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _setup(cuda):
    maps.set_sync_checks(True)
    yield


def _scene(field):
    d = field.lower()
    return d, oracle.OracleScene(d.to_numpy())


def _grad_scene(field):
    d = field.lower()
    return d, oracle.OracleScene(d.to_numpy(), with_grads=True)


# ------------------------------------------------------------------- grids --
def test_grid3d_fw_bw(cuda):
    g = torch.rand(9, 10, 11, 3, device=cuda)
    bmin, bmax = maps.vec3(-0.7, -0.5, -0.4), maps.vec3(0.6, 0.5, 0.45)
    grid = maps.Grid3D(torch.nn.Parameter(g), bmin, bmax)
    x = (torch.rand(20000, 3, device=cuda) * 1.6 - 0.8)
    y = grid(x)
    ib = (1.0 / (bmax - bmin)).numpy()
    ref = oracle.grid3d_fw(g.cpu().numpy(), bmin.numpy(), ib, x.cpu().numpy())
    assert torch.allclose(y.cpu(), torch.from_numpy(ref), rtol=1e-6, atol=1e-6)
    dout = torch.rand_like(y)
    (y * dout).sum().backward()
    gref = oracle.grid3d_bw(g.cpu().numpy(), bmin.numpy(), ib, x.cpu().numpy(), dout.cpu().numpy())
    assert torch.allclose(grid.grid.grad.cpu(), torch.from_numpy(gref), rtol=1e-5, atol=1e-5)


def test_ray_box(cuda):
    rays = torch.from_numpy(synthetic.sphere_rays(5000, 1)).to(cuda)
    rb = maps.ray_box_intersection[maps.vec3(-0.5, -0.4, -0.3), maps.vec3(0.5, 0.4, 0.3)]
    out = rb(rays).cpu().numpy()
    ref = oracle.ray_box(rays.cpu().numpy(), [-0.5, -0.4, -0.3], [0.5, 0.4, 0.3])
    assert np.allclose(out, ref, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("brick", [4, 8])
def test_majorant_grid_build(cuda, brick):
    sig = synthetic.gaussian_blobs(37, 6, 9.0, seed=2)
    grid = maps.Grid3D(torch.from_numpy(sig).to(cuda), *maps.normalized_box(list(sig.shape)))
    mg = maps.MajorantGrid(grid, brick=brick)
    assert np.array_equal(mg.tensor().cpu().numpy(), oracle.majorant_build(sig, brick))


# --------------------------------------------------------------------- DDA --
def _dda_map(sig_np, cuda, exact, requires_grad=False):
    t = torch.from_numpy(sig_np).to(cuda)
    bmin, bmax = maps.normalized_box(t)
    g = maps.Grid3D(torch.nn.Parameter(t, requires_grad=requires_grad), bmin, bmax)
    return maps.GridDDATransmittance(g, maps.ray_box_intersection[bmin, bmax], exact=exact)


@pytest.mark.parametrize("exact", [False, True])
def test_dda_transmittance_matches_oracle(cuda, exact):
    sig = synthetic.value_noise(65, 4, 50.0, seed=3)
    tr = _dda_map(sig, cuda, exact, requires_grad=True)
    rays_np = synthetic.sphere_rays(1 << 15, seed=4)
    rays = torch.from_numpy(rays_np).to(cuda)
    T = tr(rays)
    d, sc = _grad_scene_from_dda(tr)
    # the same algorithm in FP64 on the CPU: optical depth within 1e-5 relative.
    # The midpoint mode keeps the reference's stop 1e-4 short of the exit, so a
    # last sliver of < 1e-4 length may be taken on one side and not the other
    # (bounded by sigma_max * 1e-4 in tau) on at most 0.1% of the rays.
    Tref = oracle.transmittance_fw(sc, "dda_exact" if exact else "dda", rays_np, 0, fp64=True)
    if exact:
        _assert_tau_close(T.detach().cpu().numpy()[:, 0], Tref, 1e-5)
    else:
        Tg = T.detach().cpu().numpy()[:, 0].astype(np.float64)
        ok = Tref > 1e-30
        dtau = np.abs(np.log(np.maximum(Tg[ok], 1e-300)) - np.log(Tref[ok]))
        rel = dtau / np.maximum(-np.log(Tref[ok]), 1.0)
        assert (rel <= 1e-5).mean() >= 0.999, (rel > 1e-5).mean()
        assert dtau.max() <= float(sig.max()) * 1e-4 * 1.01
    w = torch.from_numpy(synthetic.uniform_weights(rays.shape[0], 5)).to(cuda)
    (T[:, 0] * w).sum().backward()
    oracle.transmittance_bw(sc, "dda_exact" if exact else "dda", rays_np, 0, w.cpu().numpy())
    g = tr.grid.grad.cpu().numpy()
    scale = np.abs(sc.sigma_grad).max()
    assert np.abs(g - sc.sigma_grad).max() <= 1e-4 * scale


def _assert_tau_close(T, Tref, rtol):
    """|tau - tau_ref| <= rtol * max(tau_ref, 1) with tau = -log T (T relative error for tau < 1)."""
    T = np.asarray(T, np.float64)
    Tref = np.asarray(Tref, np.float64)
    ok = Tref > 1e-30
    tau, tref = -np.log(np.maximum(T[ok], 1e-300)), -np.log(Tref[ok])
    err = np.abs(tau - tref) / np.maximum(tref, 1.0)
    assert err.max() <= rtol, (err.max(), int(err.argmax()))


def _grad_scene_from_dda(tr):
    from rendervous_b200.lowering import lower_transmittance_map
    d = lower_transmittance_map(tr)
    return d, oracle.OracleScene(d.to_numpy(), with_grads=True)


def test_dda_exact_vs_fp64_raymarch(cuda):
    sig = synthetic.value_noise(65, 4, 50.0, seed=3)
    tr = _dda_map(sig, cuda, True)
    rays_np = synthetic.sphere_rays(2048, seed=8)
    T = tr(torch.from_numpy(rays_np).to(cuda)).detach().cpu().numpy()[:, 0].astype(np.float64)
    d, sc = _grad_scene_from_dda(tr)
    tau = oracle.tau_raymarch_fp64(sc, rays_np, 64)
    _assert_tau_close(T, np.exp(-tau), 1e-5)


def test_dda_full_size_properties(cuda):
    """256^3, 2^20 rays: T in [0,1]; exact against the FP64 march on a sample;
    Euler identity of the adjoint (tau is linear in sigma):
    sum_k sigma_k dL/dsigma_k = -sum_i w_i T_i tau_i."""
    sig = synthetic.value_noise(256, 4, 50.0, seed=3)
    tr = _dda_map(sig, cuda, True, requires_grad=True)
    rays_np = synthetic.sphere_rays(1 << 20, seed=4)
    rays = torch.from_numpy(rays_np).to(cuda)
    w = torch.from_numpy(synthetic.uniform_weights(1 << 20, 5)).to(cuda)
    T = tr(rays)[:, 0]
    Td = T.detach()
    assert float(Td.min()) >= 0.0 and float(Td.max()) <= 1.0
    d, sc = _grad_scene_from_dda(tr)
    idx = np.arange(0, 1 << 20, 512)
    tau = oracle.tau_raymarch_fp64(sc, rays_np[idx], 16)
    _assert_tau_close(Td.cpu().numpy()[idx], np.exp(-tau), 1e-5)
    (T * w).sum().backward()
    lhs = float((tr.grid.grad.double() * tr.grid.detach().double()).sum())
    Td = Td.double().clamp_min(1e-30)
    rhs = float(-(w.double() * Td * (-torch.log(Td))).sum())
    assert abs(lhs - rhs) <= 1e-3 * abs(rhs)


# ---------------------------------------------------- ratio / delta tracking --
def _tracking_map(sig_np, cuda, mode, majorant, brick=8, requires_grad=False):
    t = torch.from_numpy(sig_np).to(cuda)
    bmin, bmax = maps.normalized_box(t)
    g = maps.Grid3D(torch.nn.Parameter(t, requires_grad=requires_grad), bmin, bmax)
    maj = maps.const[[float(sig_np.max()), 1e6]] if majorant == "global" else maps.MajorantGrid(g, brick=brick)
    cls = maps.RatiotrackingTransmittance if mode == "rt" else maps.DeltatrackingTransmittance
    return cls(g, maps.ray_box_intersection[bmin, bmax], maj)


@pytest.mark.parametrize("majorant", ["global", "grid"])
@pytest.mark.parametrize("mode", ["rt", "dt"])
def test_tracking_transmittance_matches_oracle(cuda, mode, majorant):
    sig = synthetic.gaussian_blobs(33, 6, 20.0, seed=1)
    tr = _tracking_map(sig, cuda, mode, majorant, brick=4, requires_grad=True)
    rays_np = synthetic.sphere_rays(1 << 14, seed=2)
    T = tr(torch.from_numpy(rays_np).to(cuda), seed=77)
    from rendervous_b200.lowering import lower_transmittance_map
    d = lower_transmittance_map(tr)
    sc = oracle.OracleScene(d.to_numpy(), with_grads=True)
    Tref = oracle.transmittance_fw(sc, mode, rays_np, 77)
    Tg = T.detach().cpu().numpy()[:, 0]
    same = np.isclose(Tg, Tref, rtol=1e-4, atol=1e-6)
    assert same.mean() >= 0.999, same.mean()      # <= 0.1% of rays may branch differently
    w = np.ones(rays_np.shape[0], np.float32)
    T.sum().backward()
    oracle.transmittance_bw(sc, mode, rays_np, 77, w)
    g = tr.sigma.grid.grad.cpu().numpy()
    rel = np.abs(g - sc.sigma_grad).sum() / np.abs(sc.sigma_grad).sum()
    assert rel < 5e-3, rel


# ------------------------------------------------------------ path tracing --
def _c1_field(cuda, **kw):
    wl = synthetic.WORKLOADS["plain_forward_64"]
    sig = torch.from_numpy(synthetic.make_sigma(wl["sigma"])).to(cuda)
    sun = tuple(float(v) for v in synthetic.gaussian_direction(wl["sun_seed"]))
    args = dict(albedo=wl["albedo"], env=wl["env"], sun_dir=sun, sun_radiance=wl["sun_intensity"], g=0.0,
                max_bounces=wl["max_bounces"])
    args.update(kw)
    return build_field(sig, **args)


def _capture(field, cuda, H, W, spp, seed, jittered=True, views=1):
    cam = maps.PerspectiveCameraSensor(W, H, front_camera(views).to(cuda), jittered=jittered)
    return cam, cam.capture(field, fw_samples=spp, bw_samples=spp, seed=seed)


def _oracle_capture(sc, integ, H, W, spp, seed, views=1, jittered=True):
    return oracle.capture_fw(sc, integ, front_camera(views).numpy(), W, H, math.pi / 4, jittered, spp, seed)


@pytest.mark.parametrize("variant", [
    dict(),                                           # C1: RT shadows, global majorant
    dict(majorant="grid", brick=8),
    dict(tr="dt"),
    dict(tr="dda_exact"),
    dict(phase="reference", g=0.6),
    dict(g=0.6, max_bounces=0),
])
def test_capture_forward_matches_oracle(cuda, variant):
    field = _c1_field(cuda, **variant)
    H = W = 64
    spp = 8
    _, img = _capture(field, cuda, H, W, spp, seed=123)
    d, sc = _scene(field)
    ref, cnt = _oracle_capture(sc, "nee", H, W, spp, 123)
    a, b = img.cpu().numpy(), ref
    close = np.isclose(a, b, rtol=1e-3, atol=1e-5).all(axis=-1)
    assert close.mean() >= 0.99, close.mean()         # >= 99% of pixels agree path for path
    assert abs(a.mean() - b.mean()) <= 1e-3 * abs(b.mean()) + 1e-5
    counters = maps.check()
    assert counters["status"] == 0


def test_capture_forward_statistics_independent_seeds(cuda):
    """8x8 blocks of GPU and oracle images from independent seeds agree within
    3 standard errors (4 allowed on a few blocks)."""
    field = _c1_field(cuda)
    H = W = 64
    spp = 16
    gpu = np.stack([_capture(field, cuda, H, W, spp, seed=1000 + s)[1].cpu().numpy() for s in range(4)])
    d, sc = _scene(field)
    cpu = np.stack([_oracle_capture(sc, "nee", H, W, spp, 5000 + s)[0] for s in range(4)])
    def blocks(x):  # (k, 1, H, W, 3) -> (k, nblocks)
        return x.reshape(x.shape[0], H // 8, 8, W // 8, 8, 3).mean(axis=(2, 4, 5)).reshape(x.shape[0], -1)
    bg, bc = blocks(gpu), blocks(cpu)
    se = np.sqrt(bg.var(0, ddof=1) / 4 + bc.var(0, ddof=1) / 4) + 1e-6
    z = np.abs(bg.mean(0) - bc.mean(0)) / se
    assert (z < 3).mean() >= 0.9 and z.max() < 6, z


def test_dt_integrator_matches_oracle(cuda):
    field = _c1_field(cuda, integrator="dt", sun_dir=None)
    H = W = 48
    _, img = _capture(field, cuda, H, W, 8, seed=9)
    d, sc = _scene(field)
    ref, _ = _oracle_capture(sc, "dt", H, W, 8, 9)
    close = np.isclose(img.cpu().numpy(), ref, rtol=1e-3, atol=1e-5).all(axis=-1)
    assert close.mean() >= 0.99


@pytest.mark.parametrize("bw, kw", [
    ("ds", dict()),
    ("ds", dict(majorant="grid", brick=8)),
    ("ds", dict(ds_compat=True)),
    ("dt", dict(integrator="dt", sun_dir=None)),
    ("drt", dict(integrator="drt")),
    ("drt", dict(integrator="drt", majorant="grid", brick=8)),
    ("drt", dict(integrator="drt", max_bounces=0)),
    ("drtq", dict(integrator="drtq")),
    ("drtq", dict(integrator="drtq", majorant="grid", brick=8)),
    ("drtq", dict(integrator="drtq", max_bounces=0)),
    ("drtds", dict(integrator="drtds")),
    ("drtds", dict(integrator="drtds", majorant="grid", brick=8)),
    ("sps", dict(integrator="sps")),
    ("sps", dict(integrator="sps", majorant="grid", brick=8)),
    ("sps", dict(integrator="sps", max_bounces=0)),
])
def test_capture_backward_matches_oracle(cuda, bw, kw):
    wl = synthetic.WORKLOADS["plain_forward_64"]
    sig = torch.from_numpy(synthetic.make_sigma(wl["sigma"])).to(cuda)
    alb = torch.from_numpy(synthetic.uniform_grid(64, 0.6, 0.95, seed=8)).to(cuda)
    args = dict(albedo_grid=torch.nn.Parameter(alb), env=1.0, sun_dir=(0.3, 0.8, 0.5), sun_radiance=3.0, g=0.4,
                max_bounces=16, sigma_requires_grad=True, integrator="nee_ds")
    args.update(kw)
    field = build_field(sig, **args)
    H = W = 32
    spp = 4
    cam, img = _capture(field, cuda, H, W, spp, seed=31)
    dimg = torch.from_numpy(np.random.default_rng(0).random(img.shape).astype(np.float32)).to(cuda)
    (img * dimg).sum().backward()
    d, sc = _grad_scene(field)
    oracle.capture_bw(sc, bw, front_camera(1).numpy(), W, H, math.pi / 4, True, spp, 31, dimg.cpu().numpy())
    gs = field.sigma.grid.grad.cpu().numpy()
    rel = np.abs(gs - sc.sigma_grad).sum() / max(np.abs(sc.sigma_grad).sum(), 1e-30)
    assert rel < 1e-2, rel
    if bw == "ds":
        ga = field.scattering_albedo.grid.grad.cpu().numpy()
        rela = np.abs(ga - sc.albedo_grad).sum() / max(np.abs(sc.albedo_grad).sum(), 1e-30)
        assert rela < 1e-2, rela


@pytest.mark.parametrize("limit", [1, 3000])
def test_ds_collision_log_overflow_rewalks(cuda, limit):
    """Paths whose collisions do not fit the NEE_DS collision log (capped here
    at `limit` records: none or part of the paths fit) are replayed by walking
    them again; the gradients equal those of the fully logged replay up to the
    order of the float atomics."""
    ffi, lib = _lib.ffi_lib()
    stream = _lib.stream_handle(cuda)
    ctx = _lib.context(cuda)
    wl = synthetic.WORKLOADS["plain_forward_64"]
    sig = torch.from_numpy(synthetic.make_sigma(wl["sigma"])).to(cuda)
    alb = torch.from_numpy(synthetic.uniform_grid(64, 0.6, 0.95, seed=8)).to(cuda)
    dimg = None
    grads, stats = [], []
    ks = ffi.new("vrt_kernel_stat[]", lib.VRT_K_COUNT)
    for lim in (0, limit):
        field = build_field(sig, albedo_grid=torch.nn.Parameter(alb.clone()), env=1.0, sun_dir=(0.3, 0.8, 0.5),
                            sun_radiance=3.0, g=0.4, max_bounces=16, sigma_requires_grad=True, integrator="nee_ds",
                            majorant="grid", brick=8)
        _lib.check(lib.vrt_set_collision_log_limit(ctx.ptr, lim))
        try:
            maps.check()
            _lib.check(lib.vrt_kernel_stats(ctx.ptr, stream, ks))
            cam, img = _capture(field, cuda, 32, 32, 4, seed=31)
            if dimg is None:
                dimg = torch.from_numpy(np.random.default_rng(0).random(img.shape).astype(np.float32)).to(cuda)
            (img * dimg).sum().backward()
            maps.check()
            _lib.check(lib.vrt_kernel_stats(ctx.ptr, stream, ks))
        finally:
            _lib.check(lib.vrt_set_collision_log_limit(ctx.ptr, 0))
        grads.append((field.sigma.grid.grad.cpu().numpy(), field.scattering_albedo.grid.grad.cpu().numpy()))
        stats.append({k: getattr(ks[lib.VRT_K_DS_REWALK], k) for k in ("steps", "lookups", "reds")})
    assert stats[0]["reds"] == 0 and stats[1]["reds"] > 0 and stats[1]["lookups"] > 0, stats
    for a, b in zip(grads[0], grads[1]):
        rel = np.abs(a - b).sum() / max(np.abs(a).sum(), 1e-30)
        assert np.abs(a).sum() > 0 and rel < 1e-4, rel


@pytest.mark.parametrize("integrator", ["drt", "drtds", "drtq", "sps"])
def test_drt_wavefront_in_rounds_matches_one_round(cuda, integrator):
    """With the wavefront's round size capped (vrt_set_wave_batch_limit), the
    DRT / DRTDS / DRTQ / SPS adjoints take their paths in several rounds
    (primal, light rays, replay, branches per round); the gradients equal the
    one-round run's up to the order of the float sums."""
    ffi, lib = _lib.ffi_lib()
    stream = _lib.stream_handle(cuda)
    ctx = _lib.context(cuda)
    wl = synthetic.WORKLOADS["plain_forward_64"]
    sig = torch.from_numpy(synthetic.make_sigma(wl["sigma"])).to(cuda)
    ks = ffi.new("vrt_kernel_stat[]", lib.VRT_K_COUNT)
    primal = lib.VRT_K_SPS_PRIMAL if integrator == "sps" else lib.VRT_K_DRT_PRIMAL
    dimg, grads, launches = None, [], []
    for limit in (0, 4096):
        field = build_field(sig, albedo=0.9, env=1.0, sun_dir=(0.3, 0.8, 0.5), sun_radiance=3.0, g=0.4,
                            max_bounces=16, sigma_requires_grad=True, integrator=integrator, majorant="grid", brick=8)
        _lib.check(lib.vrt_set_wave_batch_limit(ctx.ptr, limit))
        try:
            maps.check()
            _lib.check(lib.vrt_kernel_stats(ctx.ptr, stream, ks))
            cam, img = _capture(field, cuda, 128, 128, 8, seed=29)  # more paths than lanes: rounds can split
            if dimg is None:
                dimg = torch.from_numpy(np.random.default_rng(3).random(img.shape).astype(np.float32)).to(cuda)
            (img * dimg).sum().backward()
            maps.check()
            _lib.check(lib.vrt_kernel_stats(ctx.ptr, stream, ks))
        finally:
            _lib.check(lib.vrt_set_wave_batch_limit(ctx.ptr, 0))
        grads.append(field.sigma.grid.grad.cpu().numpy())
        launches.append(ks[primal].launches)
    assert launches[0] == 1 and launches[1] > 1, launches
    rel = np.abs(grads[0] - grads[1]).sum() / max(np.abs(grads[0]).sum(), 1e-30)
    assert np.abs(grads[0]).sum() > 0 and rel < 1e-4, rel


@pytest.mark.parametrize("integrator", ["drt", "drtq", "sps"])
def test_drt_wavefront_on_rays_matches_sequential_form(cuda, integrator):
    """The same on rays (the map evaluated on a ray batch, backward through
    vrt_radiance_bw): the wavefront against the sequential form (collision log
    capped at one record), delta-tracking light rays, an uncapped path budget."""
    ffi, lib = _lib.ffi_lib()
    ctx = _lib.context(cuda)
    wl = synthetic.WORKLOADS["plain_forward_64"]
    sig = torch.from_numpy(synthetic.make_sigma(wl["sigma"])).to(cuda)
    rays = torch.from_numpy(synthetic.sphere_rays(4096, seed=12)).to(cuda)
    wts = torch.from_numpy(np.random.default_rng(2).random((4096, 3)).astype(np.float32)).to(cuda)
    grads = []
    for lim in (0, 1):
        field = build_field(sig, albedo=0.9, env=1.0, sun_dir=(0.3, 0.8, 0.5), sun_radiance=3.0, g=0.4,
                            max_bounces=0, sigma_requires_grad=True, integrator=integrator, tr="dt")
        _lib.check(lib.vrt_set_collision_log_limit(ctx.ptr, lim))
        try:
            maps.check()
            R = field(rays, seed=23)
            (R * wts).sum().backward()
            maps.check()
        finally:
            _lib.check(lib.vrt_set_collision_log_limit(ctx.ptr, 0))
        grads.append(field.sigma.grid.grad.cpu().numpy())
    rel = np.abs(grads[0] - grads[1]).sum() / max(np.abs(grads[0]).sum(), 1e-30)
    assert np.abs(grads[0]).sum() > 0 and rel < 1e-4, rel


@pytest.mark.parametrize("integrator", ["drt", "drtds", "drtq", "sps"])
@pytest.mark.parametrize("limit", [1, 3000])
def test_drt_wavefront_matches_sequential_form(cuda, limit, integrator):
    """The DRT (DRTDS, DRTQ, SPS) adjoint's wavefront (primal with collision log, light-ray T
    and adjoint jobs, log replay, reservoir branch or per-segment scatter terms) against its
    sequential form:
    with the collision log capped at `limit` records, the paths that do not fit
    run whole on the sequential form (all of them at 1), so the gradients of
    both runs agree up to the order of the float sums."""
    ffi, lib = _lib.ffi_lib()
    stream = _lib.stream_handle(cuda)
    ctx = _lib.context(cuda)
    wl = synthetic.WORKLOADS["plain_forward_64"]
    sig = torch.from_numpy(synthetic.make_sigma(wl["sigma"])).to(cuda)
    ks = ffi.new("vrt_kernel_stat[]", lib.VRT_K_COUNT)
    dimg, grads, stats = None, [], []
    for lim in (0, limit):
        field = build_field(sig, albedo=0.9, env=1.0, sun_dir=(0.3, 0.8, 0.5), sun_radiance=3.0, g=0.4,
                            max_bounces=16, sigma_requires_grad=True, integrator=integrator, majorant="grid", brick=8)
        _lib.check(lib.vrt_set_collision_log_limit(ctx.ptr, lim))
        try:
            maps.check()
            _lib.check(lib.vrt_kernel_stats(ctx.ptr, stream, ks))
            cam, img = _capture(field, cuda, 32, 32, 4, seed=17)
            if dimg is None:
                dimg = torch.from_numpy(np.random.default_rng(1).random(img.shape).astype(np.float32)).to(cuda)
            (img * dimg).sum().backward()
            maps.check()
            _lib.check(lib.vrt_kernel_stats(ctx.ptr, stream, ks))
        finally:
            _lib.check(lib.vrt_set_collision_log_limit(ctx.ptr, 0))
        grads.append(field.sigma.grid.grad.cpu().numpy())
        replay = lib.VRT_K_SPS_REPLAY if integrator == "sps" else lib.VRT_K_DRT_REPLAY
        stats.append({k: getattr(ks[replay], k) for k in ("steps", "reds")})
    assert stats[0]["steps"] > 0 and stats[0]["reds"] > 0, stats  # the automatic log holds the paths
    if limit == 1:
        assert stats[1]["steps"] == 0, stats  # nothing fit: every path ran on the sequential form
    rel = np.abs(grads[0] - grads[1]).sum() / max(np.abs(grads[0]).sum(), 1e-30)
    assert np.abs(grads[0]).sum() > 0 and rel < 1e-4, rel


def test_ds_adjoint_matches_finite_difference(cuda):
    """E[dL/ds] along sigma -> s*sigma from the replay adjoint vs a central
    difference of the GPU forward with common random numbers."""
    wl = synthetic.WORKLOADS["plain_forward_64"]
    sig0 = torch.from_numpy(synthetic.make_sigma(wl["sigma"])).to(cuda)
    H = W = 32
    spp = 256
    wimg = torch.from_numpy(np.random.default_rng(1).random((1, H, W, 3)).astype(np.float32)).to(cuda)
    grads, fds = [], []
    for rep in range(6):
        f = build_field(sig0.clone(), albedo=0.8, env=1.0, sun_dir=(0.2, 1, 0.3), g=0.3, sigma_requires_grad=True)
        f.majorant = maps.const[[25.0, 1e6]]
        f.transmittance.majorant = f.majorant
        cam, img = _capture(f, cuda, H, W, spp, seed=100 + rep)
        (img * wimg).sum().backward()
        grads.append(float((f.sigma.grid.grad.double() * sig0.double()).sum()))
        vals = []
        for s in (1.05, 0.95):
            f2 = build_field(sig0 * s, albedo=0.8, env=1.0, sun_dir=(0.2, 1, 0.3), g=0.3)
            f2.majorant = maps.const[[25.0, 1e6]]
            f2.transmittance.majorant = f2.majorant
            _, im2 = _capture(f2, cuda, H, W, spp, seed=200 + rep)
            vals.append(float((im2 * wimg).sum()))
        fds.append((vals[0] - vals[1]) / 0.1)
    g, f = np.array(grads), np.array(fds)
    err = math.sqrt(g.var(ddof=1) / len(g) + f.var(ddof=1) / len(f))
    assert abs(g.mean() - f.mean()) < 4 * err + 0.03 * abs(f.mean()), (g, f)


# ------------------------------------------------------------ error paths --
def test_iteration_cap_reports_and_recovers(cuda):
    """A majorant of 1e12 makes ratio tracking take ~1e12 steps; the kernel stops
    at its iteration bound, records VRT_E_ITER_CAP, and the context stays usable."""
    sig = homogeneous(5, 1.0)
    t = torch.from_numpy(sig).to(cuda)
    bmin, bmax = maps.normalized_box(t)
    g = maps.Grid3D(t, bmin, bmax)
    tr = maps.RatiotrackingTransmittance(g, maps.ray_box_intersection[bmin, bmax], maps.const[[1e12, 1e6]])
    rays = torch.tensor([[-2.0, 0.0, 0.0, 1.0, 0.0, 0.0]], device=cuda)
    maps.set_sync_checks(False)
    try:
        tr(rays)
        with pytest.raises(_lib.VrtError) as e:
            maps.check()
        assert e.value.status == 4
        ok = maps.RatiotrackingTransmittance(g, maps.ray_box_intersection[bmin, bmax], maps.const[[1.5, 1e6]])(rays)
        maps.check()  # no error left over: the context is usable again
        assert 0.0 <= float(ok) <= 1.0
    finally:
        maps.set_sync_checks(True)


def test_nonfinite_rays_are_misses(cuda):
    field = _c1_field(cuda)
    rays = torch.tensor([[float("nan"), 0, -2, 0, 0, 1], [0, 0, -2, 0, 0, 1]], device=cuda)
    R = field(rays, seed=3)
    assert torch.isfinite(R).all()


def test_invalid_arguments_raise(cuda):
    field = _c1_field(cuda)
    d = field.lower()
    d.phase_mode = 7
    ffi, lib = _lib.ffi_lib()
    m = d.to_struct()
    rays = torch.zeros(4, 6, device=cuda)
    R = torch.empty(4, 3, device=cuda)
    st = lib.vrt_radiance_fw(_lib.context().ptr, m, 0, _lib.fptr(rays), 4, 0, _lib.fptr(R), _lib.stream_handle(cuda))
    assert st == 1


def test_ds_gradient_statistics_independent_seeds(cuda):
    """NEE_DS sigma gradients of the GPU and the oracle from independent seeds:
    sums over 8^3-voxel blocks agree within 3 standard errors (6 estimates a
    side; 90 % of the blocks under 3, none above 8 -- the per-block estimates
    are heavy-tailed and the variances come from 6 samples)."""
    wl = synthetic.WORKLOADS["plain_forward_64"]
    sig = torch.from_numpy(synthetic.make_sigma(wl["sigma"])).to(cuda)
    H = W = 32
    spp = 8
    dimg = torch.from_numpy(np.random.default_rng(5).random((1, H, W, 3)).astype(np.float32)).to(cuda)

    def blocks(g):
        g = np.asarray(g, np.float64).reshape(64, 64, 64)[:64, :64, :64]
        return g.reshape(8, 8, 8, 8, 8, 8).sum(axis=(1, 3, 5)).ravel()

    gpu, cpu = [], []
    for k in range(6):
        field = build_field(sig.clone(), albedo=0.8, env=1.0, sun_dir=(0.3, 0.8, 0.5), g=0.4, max_bounces=16,
                            sigma_requires_grad=True)
        cam, img = _capture(field, cuda, H, W, spp, seed=400 + k)
        (img * dimg).sum().backward()
        gpu.append(blocks(field.sigma.grid.grad.cpu().numpy()))
        d, sc = _grad_scene(field)
        oracle.capture_bw(sc, "ds", front_camera(1).numpy(), W, H, math.pi / 4, True, spp, 900 + k,
                          dimg.cpu().numpy())
        cpu.append(blocks(sc.sigma_grad))
    bg, bc = np.stack(gpu), np.stack(cpu)
    live = (np.abs(bg).mean(0) + np.abs(bc).mean(0)) > 1e-6 * np.abs(bc).mean(0).max()
    se = np.sqrt(bg.var(0, ddof=1) / 6 + bc.var(0, ddof=1) / 6) + 1e-12
    z = np.abs(bg.mean(0) - bc.mean(0))[live] / se[live]
    assert live.sum() > 50
    assert (z < 3).mean() >= 0.9 and z.max() < 8, (np.sort(z)[-5:], live.sum())


def test_kernel_stats_add_up(cuda):
    """vrt_kernel_stats: with timing on, the wavefront kernels of a capture and
    its adjoint report launches, event time and tallies; the per-kernel lookups
    add up to the context's total."""
    ffi, lib = _lib.ffi_lib()
    stream = _lib.stream_handle(cuda)
    ctx = _lib.context(cuda)
    nk = lib.VRT_K_COUNT
    ks = ffi.new("vrt_kernel_stat[]", nk)
    maps.check()
    _lib.check(lib.vrt_kernel_stats(ctx.ptr, stream, ks))
    lib.vrt_set_kernel_timing(1)
    maps.set_sync_checks(False)  # keep the context totals of both calls
    try:
        field = _c1_field(cuda, majorant="grid", brick=8, sigma_requires_grad=True)
        cam, img = _capture(field, cuda, 32, 32, 4, seed=3)
        img.sum().backward()
        _lib.check(lib.vrt_kernel_stats(ctx.ptr, stream, ks))
        totals = maps.check()
    finally:
        lib.vrt_set_kernel_timing(0)
        maps.set_sync_checks(True)
    nee = range(lib.VRT_K_DS_REWALK + 1)  # the NEE forward and NEE_DS adjoint kernels (not the DRT ones)
    assert all(ks[i].launches > 0 and ks[i].ms > 0 for i in nee)
    assert all(ks[i].launches == 0 for i in range(lib.VRT_K_DS_REWALK + 1, nk))
    assert sum(ks[i].lookups for i in range(nk)) == totals["lookups"]
    assert ks[1].steps > 0 and ks[4].reds > 0
    # the replay reads the primal's collision log (no lookups of its own); with
    # the automatic log size no path is left to the re-walk
    assert ks[lib.VRT_K_DS_PRIMAL].log_bytes > 0
    assert 0 < ks[lib.VRT_K_DS_REPLAY].log_bytes <= ks[lib.VRT_K_DS_PRIMAL].log_bytes
    assert ks[lib.VRT_K_DS_REPLAY].lookups == 0 and ks[lib.VRT_K_DS_REPLAY].steps > 0
    assert ks[lib.VRT_K_DS_REWALK].steps == 0 and ks[lib.VRT_K_DS_REWALK].reds == 0
