"""CPU oracle for the volumetric path-integration hot path -- TEST INFRASTRUCTURE.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this package; it is the checker, never the product.  ``liboracle.so`` is
built by ``oracle/Makefile`` (``build()`` in ``__graft_entry__`` runs it).

The restated reference functions and their citations are in ``vrt_oracle.cpp``.
Parity with the reference is UNPINNED (no reference tests or golden vectors
exist and its shaders need Vulkan); the analytic pins live in
``tests/test_oracle_*.py``.
"""
from __future__ import annotations

import os
import subprocess
import threading

import numpy as np
import cffi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_LOCK = threading.Lock()
_STATE = {}


def _cdef_text() -> str:
    text = open(os.path.join(_HERE, "oracle.h")).read()
    return text.split("/* CDEF-BEGIN */")[1].split("/* CDEF-END */")[0]


def build(quiet: bool = True) -> str:
    """Compile liboracle.so with make (no-op when up to date)."""
    out = subprocess.run(["make", "-C", _HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    return _LIB_PATH


def lib():
    """(ffi, lib) for liboracle.so, building it first if it is missing."""
    with _LOCK:
        if "lib" not in _STATE:
            if not os.path.exists(_LIB_PATH):
                build()
            ffi = cffi.FFI()
            ffi.cdef(_cdef_text())
            _STATE["ffi"] = ffi
            _STATE["lib"] = ffi.dlopen(_LIB_PATH)
        return _STATE["ffi"], _STATE["lib"]


def ptr(ffi, arr: np.ndarray | None, ctype: str = "float *"):
    if arr is None:
        return ffi.NULL
    assert arr.flags["C_CONTIGUOUS"]
    return ffi.cast(ctype, arr.ctypes.data)


TRANSMITTANCE_MODES = {"rt": 0, "dt": 1, "dda": 2, "dda_midpoint": 2, "dda_exact": 3, "grt": 4, "gdt": 5}
BW_MODES = {"ds": 0, "dt": 1, "drt": 2, "drtq": 3, "drtds": 4, "sps": 5, "mc_collision": 6, "dda_collision": 7}
INTEGRATORS = {"nee": 0, "dt": 1, "mc_collision": 2, "dda_collision": 3}


class OracleScene:
    """Owns the numpy buffers behind one ``orc_scene`` struct.

    ``desc`` is the host-side medium description produced by
    ``rendervous_b200.lowering.MediumDesc.to_numpy()`` (plain numpy arrays and
    scalars), so the oracle and the CUDA path read identical bytes.
    """

    def __init__(self, desc: dict, with_grads: bool = False):
        ffi, _ = lib()
        self.ffi = ffi
        self.keep = []
        s = ffi.new("orc_scene *")
        self.sigma = np.ascontiguousarray(desc["sigma"], dtype=np.float32)
        assert self.sigma.ndim == 4 and self.sigma.shape[3] == 1
        self.sigma_grad = np.zeros_like(self.sigma) if with_grads else None
        self._grid(s.sigma, self.sigma, self.sigma_grad)
        for k in ("bmin", "bmax", "inv_bsize", "box_min", "box_max", "albedo_const", "emission", "env",
                  "sun_dir", "sun_radiance", "maj_scale"):
            v = np.asarray(desc[k], dtype=np.float32)
            for i in range(3):
                getattr(s, k)[i] = float(v[i])
        alb = desc.get("albedo")
        self.albedo_grad = None
        if alb is not None:
            self.albedo = np.ascontiguousarray(alb, dtype=np.float32)
            self.albedo_grad = np.zeros_like(self.albedo) if with_grads else None
            self._grid(s.albedo, self.albedo, self.albedo_grad)
            s.albedo_is_grid = 1
        else:
            s.albedo_is_grid = 0
        s.has_sun = int(desc["has_sun"])
        s.phase_mode = int(desc["phase_mode"])
        s.phase_g = float(desc["phase_g"])
        s.majorant_mode = int(desc["majorant_mode"])
        s.global_majorant = float(desc["global_majorant"])
        if desc.get("maj_grid") is not None:
            self.maj = np.ascontiguousarray(desc["maj_grid"], dtype=np.float32)
            s.maj_grid = ptr(ffi, self.maj)
            for i in range(3):
                s.maj_dims[i] = int(desc["maj_dims"][i])
        s.transmittance_mode = int(desc["transmittance_mode"])
        s.max_bounces = int(desc["max_bounces"])
        s.ds_epsilon = float(desc["ds_epsilon"])
        s.ds_compat = int(desc["ds_compat"])
        s.exitance_mode = int(desc.get("exitance_mode", 0))
        img = desc.get("env_image")
        if img is not None:
            self.env_image = np.ascontiguousarray(img, dtype=np.float32)
            s.env_mode = 1
            s.env_image = ptr(ffi, self.env_image)
            s.env_hw[0], s.env_hw[1] = int(self.env_image.shape[0]), int(self.env_image.shape[1])
        qt = desc.get("env_quadtree")
        if qt is not None:
            self.env_quadtree = np.ascontiguousarray(qt, dtype=np.float32).reshape(-1)
            s.env_sampler = 1
            s.env_quadtree = ptr(ffi, self.env_quadtree)
            s.env_levels = int(desc["env_levels"])
        em = desc.get("emission_grid")
        self.emission_grad = None
        if em is not None:
            self.emission_grid = np.ascontiguousarray(em, dtype=np.float32)
            self.emission_grad = np.zeros_like(self.emission_grid) if with_grads else None
            self._grid(s.emission_grid, self.emission_grid, self.emission_grad)
            s.emission_is_grid = 1
        self.s = s

    def _grid(self, g, arr, grad):
        g.data = ptr(self.ffi, arr)
        g.grad = ptr(self.ffi, grad)
        g.D, g.H, g.W, g.C = [int(v) for v in arr.shape]


class _CameraKeep:
    """The numpy buffers an orc_camera points into, and the capture's image shape."""

    def __init__(self, poses, sensors, height, width, batch_shape=None):
        self.poses = poses
        self.sensors = sensors
        self.shape = (poses.shape[0], height, width) if sensors is None else tuple(batch_shape)

    @property
    def npix(self) -> int:
        return int(np.prod(self.shape))


def make_camera(poses: np.ndarray, width: int, height: int, fov: float, jittered: bool, znear: float = 0.001,
                sensors: np.ndarray | None = None):
    """orc_camera over every pixel of every view, or over a sensors batch
    [n, 3] of (view, row, col) (SensorsBase.capture's sensors_batch)."""
    ffi, _ = lib()
    poses = np.ascontiguousarray(poses, dtype=np.float32).reshape(-1, 9)
    cam = ffi.new("orc_camera *")
    cam.poses = ptr(ffi, poses)
    cam.views = poses.shape[0]
    cam.height = height
    cam.width = width
    cam.fov = float(fov)
    cam.znear = float(znear)
    cam.jittered = 1 if jittered else 0
    batch_shape = None
    if sensors is not None:
        batch_shape = np.shape(sensors)[:-1]
        sensors = np.ascontiguousarray(sensors, dtype=np.int64).reshape(-1, 3)
        cam.sensors = ffi.cast("int64_t *", sensors.ctypes.data)
        cam.n_sensors = sensors.shape[0]
    return cam, _CameraKeep(poses, sensors, height, width, batch_shape)


# ---------------------------------------------------------------- wrappers --

def philox(key0: int, key1: int, ctr) -> np.ndarray:
    ffi, L = lib()
    c = ffi.new("uint32_t[4]", [int(v) & 0xFFFFFFFF for v in ctr])
    o = ffi.new("uint32_t[4]")
    L.orc_philox4x32_10(key0 & 0xFFFFFFFF, key1 & 0xFFFFFFFF, c, o)
    return np.array([o[i] for i in range(4)], dtype=np.uint32)


def random_sequence(seed: int, path: int, stream: int, start: int, n: int) -> np.ndarray:
    ffi, L = lib()
    out = np.empty(n, np.float32)
    L.orc_random_sequence(seed, path, stream, start, n, ptr(ffi, out))
    return out


def ray_box(rays: np.ndarray, bmin, bmax) -> np.ndarray:
    ffi, L = lib()
    rays = np.ascontiguousarray(rays, np.float32)
    out = np.empty((rays.shape[0], 2), np.float32)
    b0 = np.asarray(bmin, np.float32)
    b1 = np.asarray(bmax, np.float32)
    L.orc_ray_box(ptr(ffi, rays), rays.shape[0], ptr(ffi, b0), ptr(ffi, b1), ptr(ffi, out))
    return out


def grid3d_fw(grid: np.ndarray, bmin, inv_bsize, x: np.ndarray) -> np.ndarray:
    ffi, L = lib()
    grid = np.ascontiguousarray(grid, np.float32)
    g = ffi.new("orc_grid *")
    g.data = ptr(ffi, grid)
    g.D, g.H, g.W, g.C = grid.shape
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty((x.shape[0], grid.shape[3]), np.float32)
    b0 = np.asarray(bmin, np.float32)
    ib = np.asarray(inv_bsize, np.float32)
    L.orc_grid3d_fw(g, ptr(ffi, b0), ptr(ffi, ib), ptr(ffi, x), x.shape[0], ptr(ffi, out))
    return out


def grid3d_bw(grid: np.ndarray, bmin, inv_bsize, x: np.ndarray, dout: np.ndarray) -> np.ndarray:
    ffi, L = lib()
    grid = np.ascontiguousarray(grid, np.float32)
    grad = np.zeros_like(grid)
    g = ffi.new("orc_grid *")
    g.data = ptr(ffi, grid)
    g.grad = ptr(ffi, grad)
    g.D, g.H, g.W, g.C = grid.shape
    x = np.ascontiguousarray(x, np.float32)
    dout = np.ascontiguousarray(dout, np.float32)
    b0 = np.asarray(bmin, np.float32)
    ib = np.asarray(inv_bsize, np.float32)
    L.orc_grid3d_bw(g, ptr(ffi, b0), ptr(ffi, ib), ptr(ffi, x), ptr(ffi, dout), x.shape[0])
    return grad


def majorant_build(sigma: np.ndarray, brick: int):
    ffi, L = lib()
    sigma = np.ascontiguousarray(sigma, np.float32)
    g = ffi.new("orc_grid *")
    g.data = ptr(ffi, sigma)
    g.D, g.H, g.W, g.C = sigma.shape
    dims = ffi.new("int32_t[3]")
    L.orc_majorant_build(g, brick, ffi.NULL, dims)
    out = np.empty((dims[2], dims[1], dims[0]), np.float32)
    L.orc_majorant_build(g, brick, ptr(ffi, out), dims)
    return out


def majorant_query(scene: OracleScene, rays: np.ndarray) -> np.ndarray:
    ffi, L = lib()
    rays = np.ascontiguousarray(rays, np.float32)
    out = np.empty((rays.shape[0], 2), np.float32)
    L.orc_majorant_query(scene.s, ptr(ffi, rays), rays.shape[0], ptr(ffi, out))
    return out


def transmittance_fw(scene: OracleScene, mode: str, rays: np.ndarray, seed: int, fp64: bool = False) -> np.ndarray:
    ffi, L = lib()
    rays = np.ascontiguousarray(rays, np.float32)
    out = np.empty(rays.shape[0], np.float32)
    L.orc_transmittance_fw(scene.s, TRANSMITTANCE_MODES[mode], ptr(ffi, rays), rays.shape[0], seed, int(fp64),
                           ptr(ffi, out))
    return out


def transmittance_bw(scene: OracleScene, mode: str, rays: np.ndarray, seed: int, dL_dT: np.ndarray) -> None:
    """Accumulates into scene.sigma_grad."""
    ffi, L = lib()
    rays = np.ascontiguousarray(rays, np.float32)
    g = np.ascontiguousarray(dL_dT, np.float32).reshape(-1)
    L.orc_transmittance_bw(scene.s, TRANSMITTANCE_MODES[mode], ptr(ffi, rays), rays.shape[0], seed, ptr(ffi, g))


def dda_tau_fp64(scene: OracleScene, rays: np.ndarray, exact: bool = False) -> np.ndarray:
    """The DDA's optical depth along each ray, in FP64 (no exp)."""
    ffi, L = lib()
    rays = np.ascontiguousarray(rays, np.float32)
    out = np.empty(rays.shape[0], np.float64)
    L.orc_dda_tau_fp64(scene.s, int(exact), ptr(ffi, rays), rays.shape[0], ptr(ffi, out, "double *"))
    return out


def collision_sample_fw(scene: OracleScene, rays: np.ndarray, seed: int) -> np.ndarray:
    """DeltatrackingCollisionSampler on rays: [n, 3] = (C, t, T)."""
    ffi, L = lib()
    rays = np.ascontiguousarray(rays, np.float32)
    out = np.empty((rays.shape[0], 3), np.float32)
    L.orc_collision_sample_fw(scene.s, ptr(ffi, rays), rays.shape[0], seed, ptr(ffi, out))
    return out


def collision_sample_bw(scene: OracleScene, rays: np.ndarray, seed: int, dL_dout: np.ndarray) -> None:
    """Accumulates into scene.sigma_grad."""
    ffi, L = lib()
    rays = np.ascontiguousarray(rays, np.float32)
    g = np.ascontiguousarray(dL_dout, np.float32).reshape(-1, 3)
    L.orc_collision_sample_bw(scene.s, ptr(ffi, rays), rays.shape[0], seed, ptr(ffi, g))


def tau_raymarch_fp64(scene: OracleScene, rays: np.ndarray, substeps: int = 32) -> np.ndarray:
    ffi, L = lib()
    rays = np.ascontiguousarray(rays, np.float32)
    out = np.empty(rays.shape[0], np.float64)
    L.orc_tau_raymarch_fp64(scene.s, ptr(ffi, rays), rays.shape[0], substeps, ptr(ffi, out, "double *"))
    return out


def phase_sample(scene: OracleScene, w_in: np.ndarray, seed: int) -> np.ndarray:
    ffi, L = lib()
    w_in = np.ascontiguousarray(w_in, np.float32)
    out = np.empty((w_in.shape[0], 4), np.float32)
    L.orc_phase_sample(scene.s, ptr(ffi, w_in), w_in.shape[0], seed, ptr(ffi, out))
    return out


def env_sample(scene: OracleScene, n: int, seed: int) -> np.ndarray:
    ffi, L = lib()
    out = np.empty((n, 6), np.float32)
    L.orc_env_sample(scene.s, n, seed, ptr(ffi, out))
    return out


def camera_rays(poses, width, height, fov, jittered, spp, seed) -> np.ndarray:
    ffi, L = lib()
    cam, keep = make_camera(poses, width, height, fov, jittered)
    out = np.empty((spp, keep.shape[0] * height * width, 6), np.float32)
    L.orc_camera_rays(cam, spp, seed, ptr(ffi, out))
    return out


def radiance_fw(scene: OracleScene, integrator: str, rays: np.ndarray, seed: int):
    ffi, L = lib()
    rays = np.ascontiguousarray(rays, np.float32)
    out = np.empty((rays.shape[0], 3), np.float32)
    c = ffi.new("orc_counters *")
    L.orc_radiance_fw(scene.s, INTEGRATORS[integrator], ptr(ffi, rays), rays.shape[0], seed, ptr(ffi, out), c)
    return out, dict(paths=c.paths, vertices=c.vertices, steps=c.steps)


def radiance_bw(scene: OracleScene, bw_mode: str, rays: np.ndarray, seed: int, dL_dR: np.ndarray) -> None:
    ffi, L = lib()
    rays = np.ascontiguousarray(rays, np.float32)
    g = np.ascontiguousarray(dL_dR, np.float32)
    L.orc_radiance_bw(scene.s, BW_MODES[bw_mode], ptr(ffi, rays), rays.shape[0], seed, ptr(ffi, g))


def capture_fw(scene: OracleScene, integrator: str, poses, width, height, fov, jittered, spp, seed, sensors=None):
    """[views, H, W, 3], or sensors.shape[:-1] + [3] for a sensors batch of (view, row, col)."""
    ffi, L = lib()
    cam, keep = make_camera(poses, width, height, fov, jittered, sensors=sensors)
    out = np.empty(keep.shape + (3,), np.float32)
    c = ffi.new("orc_counters *")
    L.orc_capture_fw(scene.s, INTEGRATORS[integrator], cam, spp, seed, ptr(ffi, out), c)
    return out, dict(paths=c.paths, vertices=c.vertices, steps=c.steps)


def capture_fw_fp64(scene: OracleScene, poses, width, height, fov, jittered, spp, seed, sensors=None) -> np.ndarray:
    """The NEE capture in double precision: float64 [..., 3]."""
    ffi, L = lib()
    cam, keep = make_camera(poses, width, height, fov, jittered, sensors=sensors)
    out = np.empty(keep.shape + (3,), np.float64)
    L.orc_capture_fw_fp64(scene.s, cam, spp, seed, ptr(ffi, out, "double *"))
    return out


def capture_bw(scene: OracleScene, bw_mode: str, poses, width, height, fov, jittered, spp, seed, dL_drgb,
               sensors=None) -> None:
    ffi, L = lib()
    cam, keep = make_camera(poses, width, height, fov, jittered, sensors=sensors)
    g = np.ascontiguousarray(dL_drgb, np.float32)
    assert g.size == 3 * keep.npix
    L.orc_capture_bw(scene.s, BW_MODES[bw_mode], cam, spp, seed, ptr(ffi, g))


def capture_prefix(scene: OracleScene, poses, width, height, fov, jittered, spp, seed, cut):
    """Radiance-cache prefix: (rgb of the prefixes, queries [3, n, 3])."""
    ffi, L = lib()
    cam, keep = make_camera(poses, width, height, fov, jittered)
    rgb = np.zeros((keep.shape[0], height, width, 3), np.float32)
    n = keep.shape[0] * height * width * spp
    q = np.empty((3, n, 3), np.float32)
    L.orc_capture_prefix(scene.s, cam, spp, seed, cut, ptr(ffi, rgb), ptr(ffi, q))
    return rgb, q


def train_samples(scene: OracleScene, poses, width, height, fov, jittered, n_paths, seed, rec, cut=-1):
    """Radiance-cache training samples [4, n_paths*rec, 3]: position, direction, target, W.
    cut >= 0: paths stop at their (cut+1)-th collision (a cache returning 0)."""
    ffi, L = lib()
    cam, keep = make_camera(poses, width, height, fov, jittered)
    out = np.empty((4, n_paths * rec, 3), np.float32)
    L.orc_train_samples(scene.s, cam, n_paths, seed, rec, cut, ptr(ffi, out))
    return out


def set_threads(n: int) -> None:
    _, L = lib()
    L.orc_set_threads(n)


def get_threads() -> int:
    _, L = lib()
    return int(L.orc_get_threads())
