"""Radiance-cache kernels (tcgen05, BF16 operands) vs the FP64 reference that
rounds at the same points (oracle/cache_ref.py).  Needs a B200.

Tolerances: the kernels sum in FP32 in a different order, so a hidden
activation can round to the neighbouring BF16 value (2^-8 relative); outputs
and gradients are compared by relative norm error <= 1e-2 and elementwise
within 3e-2 of the largest magnitude.
"""
import pytest
import torch

from oracle import cache_ref
from rendervous_b200 import cache

pytestmark = pytest.mark.gpu


def _close(a, b, rel_norm=1e-2, rel_max=3e-2):
    a = a.double().cpu()
    b = b.double().cpu()
    scale = b.abs().max().item() + 1e-30
    err = (a - b).norm().item() / (b.norm().item() + 1e-30)
    assert err <= rel_norm, f"relative norm error {err:.3e}"
    assert (a - b).abs().max().item() <= rel_max * scale, f"max error {(a - b).abs().max().item():.3e} vs {scale:.3e}"
    return err


def _rc(dev, seed=0, grid_scale=0.3):
    rc = cache.RadianceCache([-1, -1, -1], [1, 1, 1], dev, n_min=4, n_max=24, seed=seed, grid_init=grid_scale)
    return rc


def _samples(n, dev, seed=0):
    g = torch.Generator().manual_seed(seed)
    pos = torch.rand(n, 3, generator=g) * 2.2 - 1.1  # a few outside the box (clamped)
    d = torch.randn(n, 3, generator=g)
    d = d / d.norm(dim=1, keepdim=True)
    tgt = torch.rand(n, 3, generator=g) * 2
    return pos.to(dev), d.to(dev), tgt.to(dev)


@pytest.mark.parametrize("n", [1, 127, 128, 300, 4096 + 5])
def test_mlp_forward_tensor_cores(cuda, n):
    rc = _rc(cuda)
    g = torch.Generator().manual_seed(n)
    x = (torch.rand(n, 64, generator=g) * 2 - 1).to(cuda)
    out = cache.mlp_forward(rc.weights, x)
    ref, _ = cache_ref.mlp_forward(rc.weights.cpu(), x.cpu())
    _close(out, ref)


def test_mlp_forward_many_tiles_per_cta(cuda):
    # more tiles than resident CTAs: every CTA loops over several tiles
    rc = _rc(cuda, seed=3)
    n = 148 * 4 * 128 * 3 + 77
    x = (torch.rand(n, 64, device=cuda) * 2 - 1)
    out = cache.mlp_forward(rc.weights, x)
    sel = torch.arange(0, n, 997)
    ref, _ = cache_ref.mlp_forward(rc.weights.cpu(), x[sel].cpu())
    _close(out[sel], ref)
    assert cache_status_ok()


def cache_status_ok():
    from rendervous_b200 import _lib
    ffi, lib = _lib.ffi_lib()
    return lib.vrt_cache_status(_lib.stream_handle(torch.device("cuda", 0))) == 0


@pytest.mark.parametrize("n", [5, 1000])
def test_infer_encoding_and_mlp(cuda, n):
    rc = _rc(cuda, seed=1)
    pos, d, _ = _samples(n, cuda, seed=n)
    rgb = rc.infer(pos, d)
    x, _ = cache_ref.encode(rc.grid.cpu(), rc.res, rc.bmin, rc.bmax, pos.cpu(), d.cpu())
    ref, _ = cache_ref.mlp_forward(rc.weights.cpu(), x)
    _close(rgb, ref[:, :3])
    assert cache_status_ok()


@pytest.mark.parametrize("n", [100, 2048 + 17])
def test_train_gradients(cuda, n):
    rc = _rc(cuda, seed=2)
    pos, d, tgt = _samples(n, cuda, seed=7 + n)
    loss = rc.accumulate_grad(pos, d, tgt)
    l_ref, dw_ref, dg_ref = cache_ref.train_grads(rc.grid.cpu(), rc.weights.cpu(), rc.res, rc.bmin, rc.bmax,
                                                  pos.cpu(), d.cpu(), tgt.cpu())
    assert float(loss) == pytest.approx(float(l_ref), rel=1e-2)
    dw = rc.grads[rc.n_grid:]
    dg = rc.grads[: rc.n_grid]
    for l in range(5):
        o = l * 4096
        size = 4096 if l < 4 else 1024
        _close(dw[o:o + size], dw_ref[o:o + size], rel_norm=2e-2, rel_max=5e-2)
    _close(dg, dg_ref, rel_norm=2e-2, rel_max=5e-2)
    assert cache_status_ok()


def test_adam_step(cuda):
    n = 10000
    p = torch.randn(n, device=cuda)
    g = torch.randn(n, device=cuda)
    m = torch.zeros(n, device=cuda)
    v = torch.zeros(n, device=cuda)
    p0, g0 = p.clone(), g.clone()
    from rendervous_b200 import _lib
    ffi, lib = _lib.ffi_lib()
    for step in (1, 2):
        g.copy_(g0)
        _lib.check(lib.vrt_cache_adam(_lib.fptr(p), _lib.fptr(g), _lib.fptr(m), _lib.fptr(v), n, 1e-2, 0.9, 0.99,
                                      1e-8, step, _lib.stream_handle(cuda)))
        assert torch.all(g == 0)
    # reference Adam
    pr, mr, vr = p0.double(), torch.zeros(n, dtype=torch.float64, device=cuda), torch.zeros(n, dtype=torch.float64, device=cuda)
    for step in (1, 2):
        gr = g0.double()
        mr = 0.9 * mr + 0.1 * gr
        vr = 0.99 * vr + 0.01 * gr * gr
        pr = pr - 1e-2 * (mr / (1 - 0.9 ** step)) / ((vr / (1 - 0.99 ** step)).sqrt() + 1e-8)
    assert torch.allclose(p.double(), pr, atol=1e-5)


def test_training_fits_a_field(cuda):
    # radiance that varies smoothly with position and direction: the loss must fall by 10x
    rc = cache.RadianceCache([-1, -1, -1], [1, 1, 1], cuda, seed=4)
    torch.manual_seed(0)

    def field(p, d):
        return torch.stack([1 + 0.5 * torch.sin(3 * p[:, 0]) * d[:, 2], 0.5 + 0.4 * p[:, 1] * p[:, 2],
                            0.8 + 0.3 * torch.cos(2 * p[:, 2] + d[:, 0])], dim=1)

    first = None
    for it in range(300):
        pos = torch.rand(16384, 3, device=cuda) * 2 - 1
        d = torch.nn.functional.normalize(torch.randn(16384, 3, device=cuda), dim=1)
        loss = rc.train_step(pos, d, field(pos, d), lr=1e-2)
        if it == 0:
            first = float(loss)
    pos = torch.rand(8192, 3, device=cuda) * 2 - 1
    d = torch.nn.functional.normalize(torch.randn(8192, 3, device=cuda), dim=1)
    err = ((rc.infer(pos, d) - field(pos, d)).abs() / field(pos, d).abs()).mean().item()
    assert float(loss) < first / 10, (first, float(loss))
    assert err < 0.05, err
    assert cache_status_ok()
