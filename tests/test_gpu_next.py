"""The rows next to the hot path: grid decomposition tracking (GRT / GDT),
collision samplers and integrators, and the image environment with its
quadtree sampler -- CUDA path vs the oracle through the C ABI (needs a B200).
Same inputs and Philox keys on both sides; tolerances are written in each test.
"""
import math

import numpy as np
import pytest
import torch

import oracle
from rendervous_b200 import maps, synthetic
from rendervous_b200.lowering import lower_transmittance_map
from tests.helpers import build_field, front_camera

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _setup(cuda):
    maps.set_sync_checks(True)
    yield


def _grid(sig_np, cuda, requires_grad=False):
    t = torch.nn.Parameter(torch.from_numpy(sig_np).to(cuda), requires_grad=requires_grad)
    bmin, bmax = maps.normalized_box(t)
    return maps.Grid3D(t, bmin, bmax), maps.ray_box_intersection[bmin, bmax]


# ------------------------------------------------------------------ GRT / GDT --
@pytest.mark.parametrize("mode", ["grt", "gdt"])
def test_grid_tracking_transmittance_matches_oracle(cuda, mode):
    sig = synthetic.value_noise(65, 4, 30.0, seed=3)
    g, boundary = _grid(sig, cuda)
    cls = maps.GridRatiotrackingTransmittance if mode == "grt" else maps.GridDeltatrackingTransmittance
    tr = cls(g, boundary)
    rays_np = synthetic.sphere_rays(1 << 15, seed=4)
    T = tr(torch.from_numpy(rays_np).to(cuda), seed=99)[:, 0].cpu().numpy()
    sc = oracle.OracleScene(lower_transmittance_map(tr).to_numpy())
    ref = oracle.transmittance_fw(sc, mode, rays_np, 99)
    close = np.isclose(T, ref, rtol=1e-4, atol=1e-6)
    assert close.mean() >= 0.995, close.mean()             # ray for ray, same draws
    assert abs(T.mean() - ref.mean()) <= 2e-3 * ref.mean()
    assert maps.check()["status"] == 0


@pytest.mark.parametrize("mode", ["grt", "gdt"])
def test_capture_with_grid_tracking_shadows_matches_oracle(cuda, mode):
    wl = synthetic.WORKLOADS["plain_forward_64"]
    sig = torch.from_numpy(synthetic.make_sigma(wl["sigma"])).to(cuda)
    field = build_field(sig, albedo=0.9, env=1.0, sun_dir=(0.3, 0.8, 0.5), g=0.3, max_bounces=16, tr=mode,
                        majorant="grid", brick=8)
    H = W = 48
    cam = maps.PerspectiveCameraSensor(W, H, front_camera(1).to(cuda), jittered=True)
    img = cam.capture(field, fw_samples=4, seed=5).cpu().numpy()
    sc = oracle.OracleScene(field.lower().to_numpy())
    ref, _ = oracle.capture_fw(sc, "nee", front_camera(1).numpy(), W, H, math.pi / 4, True, 4, 5)
    close = np.isclose(img, ref, rtol=1e-3, atol=1e-5).all(axis=-1)
    assert close.mean() >= 0.99, close.mean()


# ------------------------------------------------- collision integrators --
def _collision_field(cuda, kind, exitance, majorant="grid"):
    sig = synthetic.value_noise(33, 3, 20.0, seed=21)
    g, boundary = _grid(sig, cuda, requires_grad=True)
    bmin, bmax = g.bmin, g.bmax
    alb = maps.Grid3D(torch.nn.Parameter(torch.from_numpy(synthetic.uniform_grid(33, 0.5, 0.95, seed=22,
                                                                                 channels=3)).to(cuda)), bmin, bmax)
    em = maps.Grid3D(torch.nn.Parameter(torch.from_numpy(synthetic.uniform_grid(33, 0.1, 2.0, seed=23,
                                                                                channels=3)).to(cuda)), bmin, bmax)
    maj = maps.MajorantGrid(g, brick=4) if majorant == "grid" else maps.const[[float(sig.max()), 1e6]]
    env = maps.const[0.8, 0.9, 1.0]
    radiance = maps.RatiotrackingTransmittance(g, boundary, maj) * env.after(maps.ray_direction)
    ps = maps.HenyeyGreensteinPhaseSampler(maps.const[0.4])
    ex = {"emission": em, "scattered": maps.MCScatteredRadiance(alb, ps, radiance),
          "both": maps.MCScatteredEmittedRadiance(alb, em, ps, radiance)}[exitance]
    if kind == "mc_collision":
        cs = maps.DeltatrackingCollisionSampler(g, boundary, maj, 0.1)
        return maps.MCCollisionIntegrator(cs, ex, env), g, alb, em
    return maps.GridDDACollisionIntegrator(g, ex, env, boundary), g, alb, em


def _rel_l1(a, b):
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-30)


@pytest.mark.parametrize("majorant", ["grid", "const"])
def test_collision_sampler_matches_oracle(cuda, majorant):
    sig = synthetic.value_noise(33, 3, 20.0, seed=21)
    g, boundary = _grid(sig, cuda, requires_grad=True)
    maj = maps.MajorantGrid(g, brick=4) if majorant == "grid" else maps.const[[float(sig.max()), 1e6]]
    cs = maps.DeltatrackingCollisionSampler(g, boundary, maj, 0.1)
    rays_np = synthetic.sphere_rays(1 << 14, seed=7)
    out = cs(torch.from_numpy(rays_np).to(cuda), seed=5)
    sc = oracle.OracleScene(cs.lower().to_numpy(), with_grads=True)
    ref = oracle.collision_sample_fw(sc, rays_np, 5)
    o = out.detach().cpu().numpy()
    same = (o[:, 0] == ref[:, 0]) & np.isclose(o[:, 1], ref[:, 1], rtol=1e-4, atol=1e-5)
    assert same.mean() >= 0.995, same.mean()
    assert o[:, 0].mean() > 0.1                                   # the rays do collide
    dout = torch.from_numpy(np.random.default_rng(2).random(o.shape).astype(np.float32)).to(cuda)
    (out * dout).sum().backward()
    oracle.collision_sample_bw(sc, rays_np, 5, dout.cpu().numpy())
    assert _rel_l1(g.grid.grad.cpu().numpy(), sc.sigma_grad) < 1e-2


@pytest.mark.parametrize("kind", ["mc_collision", "dda_collision"])
@pytest.mark.parametrize("exitance", ["emission", "scattered", "both"])
def test_collision_integrator_matches_oracle(cuda, kind, exitance):
    field, g, alb, em = _collision_field(cuda, kind, exitance)
    rays_np = synthetic.sphere_rays(1 << 13, seed=8)
    R = field(torch.from_numpy(rays_np).to(cuda), seed=9)
    sc = oracle.OracleScene(field.lower().to_numpy(), with_grads=True)
    ref, cnt = oracle.radiance_fw(sc, kind, rays_np, 9)
    r = R.detach().cpu().numpy()
    close = np.isclose(r, ref, rtol=1e-3, atol=1e-5).all(axis=-1)
    assert close.mean() >= 0.99, close.mean()                    # ray for ray, same draws
    dR = torch.from_numpy(np.random.default_rng(3).random(r.shape).astype(np.float32)).to(cuda)
    (R * dR).sum().backward()
    oracle.radiance_bw(sc, kind, rays_np, 9, dR.cpu().numpy())
    assert _rel_l1(g.grid.grad.cpu().numpy(), sc.sigma_grad) < 1e-2
    if exitance != "emission":
        assert _rel_l1(alb.grid.grad.cpu().numpy(), sc.albedo_grad) < 1e-2
    if exitance != "scattered":
        assert _rel_l1(em.grid.grad.cpu().numpy(), sc.emission_grad) < 1e-2
    assert maps.check()["status"] == 0


@pytest.mark.parametrize("kind", ["mc_collision", "dda_collision"])
def test_collision_integrator_capture_matches_oracle(cuda, kind):
    field, g, alb, em = _collision_field(cuda, kind, "both")
    H = W = 32
    cam = maps.PerspectiveCameraSensor(W, H, front_camera(1).to(cuda), jittered=True)
    img = cam.capture(field, fw_samples=4, bw_samples=4, seed=12)
    dimg = torch.from_numpy(np.random.default_rng(4).random(img.shape).astype(np.float32)).to(cuda)
    (img * dimg).sum().backward()
    sc = oracle.OracleScene(field.lower().to_numpy(), with_grads=True)
    ref, _ = oracle.capture_fw(sc, kind, front_camera(1).numpy(), W, H, math.pi / 4, True, 4, 12)
    oracle.capture_bw(sc, kind, front_camera(1).numpy(), W, H, math.pi / 4, True, 4, 12, dimg.cpu().numpy())
    close = np.isclose(img.detach().cpu().numpy(), ref, rtol=1e-3, atol=1e-5).all(axis=-1)
    assert close.mean() >= 0.99, close.mean()
    assert _rel_l1(g.grid.grad.cpu().numpy(), sc.sigma_grad) < 1e-2
    assert _rel_l1(em.grid.grad.cpu().numpy(), sc.emission_grad) < 1e-2


# ------------------------------------------------------ image environment --
def _sky_env(cuda, sampler):
    rng = np.random.default_rng(3)
    img = 0.2 + rng.random((32, 64, 3)).astype(np.float32)
    img[4:7, 40:44] += 30.0
    t = torch.from_numpy(img).to(cuda)
    env = maps.Image2D(t).after(maps.xr_projection)
    if sampler == "uniform":
        ps = maps.UniformDirectionSampler(6)
    else:
        ps = maps.XRQuadtreeRandomDirection(6, maps.environment_quadtree(t, levels=6), 6)
    return env, maps._functionsampler(ps, env)


@pytest.mark.parametrize("sampler", ["uniform", "quadtree"])
def test_image_environment_capture_matches_oracle(cuda, sampler):
    wl = synthetic.WORKLOADS["plain_forward_64"]
    sig = torch.nn.Parameter(torch.from_numpy(synthetic.make_sigma(wl["sigma"])).to(cuda))
    bmin, bmax = maps.normalized_box(sig)
    sg = maps.Grid3D(sig, bmin, bmax)
    boundary = maps.ray_box_intersection[bmin, bmax]
    maj = maps.MajorantGrid(sg, brick=8)
    env, es = _sky_env(cuda, sampler)
    g = maps.const[0.3]
    field = maps.DeltatrackingNEEPathIntegrator(
        sg, maps.const[0.9, 0.9, 0.9], maps.ZERO, env, es, maps.HenyeyGreensteinPhase(g),
        maps.HenyeyGreensteinPhaseSampler(g), boundary, maj, maps.RatiotrackingTransmittance(sg, boundary, maj), 0.1,
        max_bounces=16, directional_light=maps.DirectionalLight((0.3, 0.8, 0.5), 2.0))
    H = W = 48
    cam = maps.PerspectiveCameraSensor(W, H, front_camera(1).to(cuda), jittered=True)
    img = cam.capture(field, fw_samples=4, bw_samples=4, seed=17)
    dimg = torch.from_numpy(np.random.default_rng(5).random(img.shape).astype(np.float32)).to(cuda)
    (img * dimg).sum().backward()
    sc = oracle.OracleScene(field.lower().to_numpy(), with_grads=True)
    ref, _ = oracle.capture_fw(sc, "nee", front_camera(1).numpy(), W, H, math.pi / 4, True, 4, 17)
    oracle.capture_bw(sc, "ds", front_camera(1).numpy(), W, H, math.pi / 4, True, 4, 17, dimg.cpu().numpy())
    close = np.isclose(img.detach().cpu().numpy(), ref, rtol=1e-3, atol=1e-5).all(axis=-1)
    assert close.mean() >= 0.99, close.mean()
    assert _rel_l1(sig.grad.cpu().numpy(), sc.sigma_grad) < 1e-2


@pytest.mark.parametrize("kind", ["dt", "dda_collision"])
def test_image_environment_other_integrators_match_oracle(cuda, kind):
    sig = synthetic.value_noise(33, 3, 20.0, seed=21)
    g, boundary = _grid(sig, cuda)
    env, es = _sky_env(cuda, "quadtree")
    if kind == "dt":
        maj = maps.MajorantGrid(g, brick=4)
        field = maps.DeltatrackingPathIntegrator(g, maps.const[0.8, 0.8, 0.8], maps.ZERO, env,
                                                 maps.HenyeyGreensteinPhaseSampler(maps.const[0.2]), boundary, maj,
                                                 0.1, max_bounces=16)
        integ = "dt"
    else:
        em = maps.const[0.5, 0.25, 0.1]
        field = maps.GridDDACollisionIntegrator(g, em, env, boundary)
        integ = "dda_collision"
    rays_np = synthetic.sphere_rays(1 << 12, seed=31)
    R = field(torch.from_numpy(rays_np).to(cuda), seed=4).cpu().numpy()
    sc = oracle.OracleScene(field.lower().to_numpy())
    ref, _ = oracle.radiance_fw(sc, integ, rays_np, 4)
    close = np.isclose(R, ref, rtol=1e-3, atol=1e-5).all(axis=-1)
    assert close.mean() >= 0.99, close.mean()
    assert R.max() > 1.0                                   # the image's bright patch shows
