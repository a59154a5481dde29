"""The transmittance entry point that allocates nothing (needs a B200).

vrt_transmittance_fw_noalloc serves callers that cannot call cudaMalloc (code
running inside another framework's pre-sized memory pool, plugins that must
not grow the device footprint): its majorant grid and kernel counters live in
a fixed array inside libvrt.so instead of a context or caller buffers.  It must
give the same transmittance as vrt_transmittance_fw with a caller-built
majorant grid of the same brick size, call after call; leave the device's free
memory unchanged; refuse grids whose bricks do not fit its fixed array; and,
when asked, report the device error word of its call.  The file is collected
last so that a run stopping at the first failure has already run every other
test.
"""
import pytest
import torch

from rendervous_b200 import _lib, maps, synthetic
from rendervous_b200.lowering import lower_transmittance_map

pytestmark = pytest.mark.gpu


def _map(sig_np, dev, mode, brick):
    t = torch.from_numpy(sig_np).to(dev)
    bmin, bmax = maps.normalized_box(t)
    g = maps.Grid3D(t, bmin, bmax)
    cls = maps.RatiotrackingTransmittance if mode == "rt" else maps.DeltatrackingTransmittance
    return cls(g, maps.ray_box_intersection[bmin, bmax], maps.MajorantGrid(g, brick=brick))


def _plain(desc):
    """The medium without a majorant grid: the entry point installs its own."""
    ffi, _ = _lib.ffi_lib()
    m = desc.to_struct()
    m.majorant_mode = 0
    m.maj_grid = ffi.NULL
    return m


@pytest.mark.parametrize("mode", ["rt", "dt"])
def test_noalloc_matches_allocating_entry_point(cuda, mode):
    ffi, lib = _lib.ffi_lib()
    maps.set_sync_checks(True)
    sig = synthetic.gaussian_blobs(65, 8, 30.0, seed=5)
    brick = 8
    tr = _map(sig, cuda, mode, brick)
    rays = torch.from_numpy(synthetic.sphere_rays(1 << 16, seed=6)).to(cuda)
    desc = lower_transmittance_map(tr)          # majorant grid built into a torch buffer
    code = 0 if mode == "rt" else 1
    stream = _lib.stream_handle(cuda)
    status = ffi.new("int64_t *")
    for call, seed in enumerate((21, 22)):      # two calls in a row share the fixed array
        ref = torch.empty(rays.shape[0], device=cuda)
        st = lib.vrt_transmittance_fw(_lib.context(cuda).ptr, desc.to_struct(), code, _lib.fptr(rays),
                                      rays.shape[0], seed, _lib.fptr(ref), stream)
        assert st == 0
        out = torch.full((rays.shape[0],), -1.0, device=cuda)
        # the second call also asks for its error word (and so waits for its kernels)
        st = lib.vrt_transmittance_fw_noalloc(_plain(desc), code, brick, _lib.fptr(rays), rays.shape[0], seed,
                                              _lib.fptr(out), status if call else ffi.NULL, stream)
        assert st == 0
        if call:
            assert status[0] == 0
        torch.cuda.synchronize(cuda)
        # same kernel, same bounds, same draws: identical up to 1e-6 relative
        assert torch.allclose(out, ref, rtol=1e-6, atol=1e-7), (call, (out - ref).abs().max())
        assert float(out.min()) >= 0.0


def test_noalloc_leaves_free_device_memory_unchanged(cuda):
    """After a first call (which loads the kernels), a call on a grid of another
    size allocates nothing: the device's free memory is the same before and after."""
    ffi, lib = _lib.ffi_lib()
    stream = _lib.stream_handle(cuda)
    status = ffi.new("int64_t *")
    rays = torch.from_numpy(synthetic.sphere_rays(1 << 14, seed=9)).to(cuda)
    T = torch.empty(rays.shape[0], device=cuda)
    descs = [lower_transmittance_map(_map(synthetic.gaussian_blobs(n, 6, 10.0, seed=n), cuda, "rt", 4))
             for n in (33, 57)]
    assert lib.vrt_transmittance_fw_noalloc(_plain(descs[0]), 0, 4, _lib.fptr(rays), rays.shape[0], 1, _lib.fptr(T),
                                            status, stream) == 0
    torch.cuda.synchronize(cuda)
    free0, _ = torch.cuda.mem_get_info(cuda)
    assert lib.vrt_transmittance_fw_noalloc(_plain(descs[1]), 0, 4, _lib.fptr(rays), rays.shape[0], 2, _lib.fptr(T),
                                            status, stream) == 0
    torch.cuda.synchronize(cuda)
    free1, _ = torch.cuda.mem_get_info(cuda)
    assert free1 == free0
    assert float(T.min()) >= 0.0 and float(T.max()) <= 1.0


def test_noalloc_reports_its_error_word(cuda):
    """A majorant of 1e12 makes ratio tracking run into its iteration bound; with
    status_out the call waits, returns VRT_E_ITER_CAP and stores its bit, and the
    next call (which clears the array's counters) is clean again."""
    ffi, lib = _lib.ffi_lib()
    sig = torch.ones(5, 5, 5, 1, device=cuda)
    bmin, bmax = maps.normalized_box(sig)
    g = maps.Grid3D(sig, bmin, bmax)
    stream = _lib.stream_handle(cuda)
    status = ffi.new("int64_t *")
    rays = torch.tensor([[-2.0, 0.0, 0.0, 1.0, 0.0, 0.0]], device=cuda)
    T = torch.empty(1, device=cuda)
    huge = lower_transmittance_map(maps.RatiotrackingTransmittance(g, maps.ray_box_intersection[bmin, bmax],
                                                                   maps.const[[1e12, 1e6]]))
    st = lib.vrt_transmittance_fw_noalloc(huge.to_struct(), 0, 0, _lib.fptr(rays), 1, 3, _lib.fptr(T), status, stream)
    assert st == 4 and status[0] == 1 << 4
    fine = lower_transmittance_map(maps.RatiotrackingTransmittance(g, maps.ray_box_intersection[bmin, bmax],
                                                                   maps.const[[1.5, 1e6]]))
    st = lib.vrt_transmittance_fw_noalloc(fine.to_struct(), 0, 0, _lib.fptr(rays), 1, 3, _lib.fptr(T), status, stream)
    assert st == 0 and status[0] == 0
    assert 0.0 <= float(T) <= 1.0


def test_noalloc_rejects_grids_beyond_its_array(cuda):
    ffi, lib = _lib.ffi_lib()
    small = torch.zeros(8, 8, 8, 1, device=cuda)
    m = ffi.new("vrt_medium *")
    # a 130^3 grid with brick 2 needs 65^3 bricks (> 64^3): refused before any launch
    m.sigma.data = _lib.fptr(small)
    for i, v in enumerate((130, 130, 130, 1)):
        m.sigma.shape[i] = v
    for i, v in enumerate((130 * 130, 130, 1, 1)):
        m.sigma.strides[i] = v
    for i in range(3):
        m.inv_bsize[i] = 1.0
        m.bmin[i], m.bmax[i] = -0.5, 0.5
        m.box_min[i], m.box_max[i] = -0.5, 0.5
    rays = torch.zeros(4, 6, device=cuda)
    T = torch.empty(4, device=cuda)
    st = lib.vrt_transmittance_fw_noalloc(m, 0, 2, _lib.fptr(rays), 4, 0, _lib.fptr(T), ffi.NULL,
                                          _lib.stream_handle(cuda))
    assert st == 3  # VRT_E_BAD_SHAPE
