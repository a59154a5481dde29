"""Host-side checks of the C ABI and the map lowering (CPU only: no kernel runs).

The library must load and export every function include/vrt.h declares;
argument validation must reject bad inputs with status codes before touching
the GPU (the host-side fault injection the reference's asserts correspond to).
"""
import math
import subprocess

import numpy as np
import pytest
import torch

from rendervous_b200 import _lib, build, maps
from rendervous_b200.lowering import lower_integrator
from tests.helpers import build_field


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.ffi_lib()


def test_library_exports_every_declared_symbol(lib):
    ffi, L = lib
    declared = _lib.exported_symbols()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(declared) <= exported


def test_status_strings(lib):
    ffi, L = lib
    assert L.vrt_version() >= 1
    assert ffi.string(L.vrt_status_string(0)) == b"ok"
    assert ffi.string(L.vrt_status_string(4)).startswith(b"device loop")


def _grid(ffi, shape, strides, data=1):
    g = ffi.new("vrt_grid *")
    g.data = ffi.cast("float *", data)
    for i in range(4):
        g.shape[i] = shape[i]
        g.strides[i] = strides[i]
    return g


def test_argument_validation_before_launch(lib):
    """Every one of these returns an error code without any CUDA call."""
    ffi, L = lib
    b = ffi.new("float[3]", [0, 0, 0])
    out = ffi.new("float[4]")
    x = ffi.new("float[3]")
    ok_grid = _grid(ffi, [4, 4, 4, 1], [16, 4, 1, 1], 0x1000)
    assert L.vrt_grid3d_fw(ffi.NULL, b, b, x, 1, out, ffi.NULL) == 2                      # null grid
    assert L.vrt_grid3d_fw(_grid(ffi, [1, 4, 4, 1], [16, 4, 1, 1], 0x1000), b, b, x, 1, out, ffi.NULL) == 3  # D < 2
    assert L.vrt_grid3d_fw(_grid(ffi, [4, 4, 4, 2], [32, 8, 2, 2], 0x1000), b, b, x, 1, out, ffi.NULL) == 3  # C stride
    assert L.vrt_grid3d_fw(_grid(ffi, [4, 4, 4, 1], [16, 4, 1, 1], 0), b, b, x, 1, out, ffi.NULL) == 2      # null data
    assert L.vrt_grid3d_fw(_grid(ffi, [2048, 2048, 2048, 1], [2048 * 2048, 2048, 1, 1], 0x1000), b, b, x, 1, out,
                           ffi.NULL) == 3  # beyond 32-bit offsets
    assert L.vrt_grid3d_fw(ok_grid, b, b, x, -1, out, ffi.NULL) == 3
    assert L.vrt_grid3d_fw(ok_grid, b, b, x, 0, out, ffi.NULL) == 0                        # empty input: no-op
    assert L.vrt_ray_box(ffi.NULL, 0, b, b, ffi.NULL, ffi.NULL) == 0
    assert L.vrt_ray_box(ffi.NULL, 3, b, b, out, ffi.NULL) == 2
    dims = ffi.new("int32_t[3]")
    assert L.vrt_majorant_build(ok_grid, 0, ffi.NULL, dims, ffi.NULL) == 1                 # brick < 1
    assert L.vrt_majorant_build(ok_grid, 2, ffi.NULL, dims, ffi.NULL) == 0                 # dims only
    assert list(dims) == [2, 2, 2]
    m = ffi.new("vrt_medium *")
    assert L.vrt_transmittance_fw(ffi.NULL, m, 0, ffi.NULL, 0, 0, ffi.NULL, ffi.NULL) == 2  # null context
    assert L.vrt_capture_fw(ffi.NULL, m, 0, ffi.NULL, 1, 0, ffi.NULL, ffi.NULL) == 2
    assert L.vrt_context_destroy(ffi.NULL) == 2
    assert L.vrt_context_sync(ffi.NULL, ffi.NULL, ffi.NULL) == 2
    # the no-allocation transmittance checks everything before its first CUDA call
    NA = L.vrt_transmittance_fw_noalloc
    rays = ffi.cast("float *", 0x1000)
    assert NA(ffi.NULL, 0, 0, rays, 1, 0, out, ffi.NULL, ffi.NULL) == 2          # null medium
    assert NA(m, 9, 0, rays, 1, 0, out, ffi.NULL, ffi.NULL) == 1                 # bad mode
    assert NA(m, 0, -1, rays, 1, 0, out, ffi.NULL, ffi.NULL) == 1                # bad brick
    assert NA(m, 0, 0, rays, -1, 0, out, ffi.NULL, ffi.NULL) == 3                # n < 0
    assert NA(m, 0, 0, ffi.NULL, 0, 0, ffi.NULL, ffi.NULL, ffi.NULL) == 0        # empty input: no-op
    assert NA(m, 0, 0, ffi.NULL, 1, 0, out, ffi.NULL, ffi.NULL) == 2             # null rays
    assert NA(m, 0, 0, ffi.cast("float *", 0x1004), 1, 0, out, ffi.NULL, ffi.NULL) == 1  # rays not 8-byte aligned
    big = ffi.new("vrt_medium *")
    big.sigma = _grid(ffi, [130, 130, 130, 1], [130 * 130, 130, 1, 1], 0x1000)[0]
    assert NA(big, 0, 2, rays, 1, 0, out, ffi.NULL, ffi.NULL) == 3               # 65^3 bricks > 64^3


def test_lowering_of_reference_style_scene():
    sig = torch.rand(9, 9, 9, 1)
    f = build_field(sig, albedo=0.8, env=(1.0, 0.5, 0.25), g=0.4, phase="reference", sun_dir=(0, 1, 0), tr="rt",
                    max_bounces=7, integrator="nee_ds", ds_epsilon=0.2)
    d = lower_integrator(f)
    assert d.phase_mode == 1 and abs(d.phase_g - 0.4) < 1e-7
    assert d.env == (1.0, 0.5, 0.25)
    assert d.albedo_const == pytest.approx((0.8, 0.8, 0.8))
    assert d.majorant_mode == 0 and d.global_majorant == pytest.approx(float(sig.max()))
    assert d.transmittance_mode == 0 and d.max_bounces == 7 and d.ds_epsilon == pytest.approx(0.2)
    assert d.sun_dir == (0.0, 1.0, 0.0)
    n = d.to_numpy()
    assert np.allclose(n["bmin"], [-0.5] * 3) and np.allclose(n["inv_bsize"], [1.0] * 3)


def test_lowering_rejects_unsupported_graphs():
    sig = torch.rand(5, 5, 5, 1)
    f = build_field(sig)
    f.phase_sampler = maps.HGDirectionSampler(maps.const[0.3])   # wrong output layout for the slot
    with pytest.raises(NotImplementedError):
        lower_integrator(f)
    f = build_field(sig)
    f.sigma = maps.const[1.0]
    with pytest.raises(NotImplementedError):
        lower_integrator(f)
    f = build_field(sig, g=0.3, phase="reference")
    f.phase = maps.HGPhase(maps.const[0.5])                      # phase and sampler disagree
    with pytest.raises(NotImplementedError):
        lower_integrator(f)


def test_builders_assemble_the_reference_integrators():
    from rendervous_b200 import objects
    ds = objects.DependencySet()
    ds.add_parameters(sigma_tensor=torch.rand(9, 9, 9, 1), scattering_albedo_tensor=torch.tensor([0.9, 0.9, 0.9]),
                      environment_tensor=torch.tensor([1.0, 1.0, 1.0]), phase_g_tensor=torch.tensor([0.0]))
    ds.requires(objects.medium_radiance_path_integrator_NEE_DRT)
    d = lower_integrator(ds.radiance)
    assert isinstance(ds.radiance, maps.DRTPathIntegrator)
    assert d.phase_mode == 1 and d.transmittance_mode == 0
    assert np.allclose(d.to_numpy()["box_max"], [0.5] * 3)


def test_normalized_box_matches_reference_formula():
    bmin, bmax = maps.normalized_box([64, 32, 16])   # [D, H, W]
    assert torch.allclose(bmax, torch.tensor([15, 31, 63]) * 0.5 / 63)
    assert torch.allclose(bmin, -bmax)


def test_cpu_tensors_never_reach_the_kernels():
    sig = torch.rand(5, 5, 5, 1)
    d = lower_integrator(build_field(sig))
    with pytest.raises(ValueError):
        d.to_struct()


def test_lowering_of_collision_integrators():
    """MCCollisionIntegrator / GridDDACollisionIntegrator graphs as the
    reference's builders assemble them (_objects.py:243-307) lower to the
    exitance forms the kernels run; other radiance maps are refused."""
    from rendervous_b200.lowering import lower_collision_integrator
    sig = torch.rand(9, 9, 9, 1)
    bmin, bmax = maps.normalized_box(sig)
    g = maps.Grid3D(sig, bmin, bmax)
    boundary = maps.ray_box_intersection[bmin, bmax]
    maj = maps.const[[1.0, 1e6]]
    env = maps.const[0.5, 0.6, 0.7]
    alb = maps.Grid3D(torch.rand(9, 9, 9, 3), bmin, bmax)
    tr = maps.RatiotrackingTransmittance(g, boundary, maj)
    ps = maps.VHGPhaseSampler(maps.const[0.3])
    scat = maps.MCScatteredEmittedRadiance(alb, maps.const[1.0, 2.0, 3.0], ps, tr * env.after(maps.ray_direction))
    mc = maps.MCCollisionIntegrator(maps.DeltatrackingCollisionSampler(g, boundary, maj, 0.2), scat, env)
    d = lower_collision_integrator(mc)
    assert d.exitance_mode == 2 and d.albedo_grid is alb.grid and d.emission == (1.0, 2.0, 3.0)
    assert d.phase_mode == 1 and abs(d.phase_g - 0.3) < 1e-7 and abs(d.ds_epsilon - 0.2) < 1e-7
    assert d.transmittance_mode == 0 and np.allclose(d.env, (0.5, 0.6, 0.7))
    em = maps.Grid3D(torch.rand(9, 9, 9, 3), bmin, bmax)
    dda = maps.GridDDACollisionIntegrator(g, em, env, boundary)
    d2 = lower_collision_integrator(dda)
    assert d2.exitance_mode == 0 and d2.emission_grid is em.grid
    with pytest.raises(NotImplementedError):   # a radiance map that is not transmittance * environment
        lower_collision_integrator(maps.GridDDACollisionIntegrator(
            g, maps.MCScatteredRadiance(alb, ps, env.after(maps.ray_direction)), env, boundary))
    with pytest.raises(NotImplementedError):   # environments must agree
        lower_collision_integrator(maps.GridDDACollisionIntegrator(
            g, maps.MCScatteredRadiance(alb, ps, tr * maps.const[1.0, 1.0, 1.0].after(maps.ray_direction)), env,
            boundary))
