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
