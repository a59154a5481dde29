"""FP64 CPU reference of the radiance-cache network -- TEST INFRASTRUCTURE.

Restates the encoding and the MLP of rendervous_b200/csrc/vrt_cache.cu in
float64 torch, rounding to BF16 at the same points as the tensor-core kernels
(network inputs, weights, hidden activations, backward tiles), so the GPU
results are compared with their exact BF16-operand / high-precision-sum
counterpart.  Used only by tests/.
"""
from __future__ import annotations

import torch

SH = (0.28209479177387814, 0.4886025119029199, 1.0925484305920792, 0.31539156525252005, 0.5462742152960396,
      0.5900435899266435, 2.890611442640554, 0.4570457994644658, 0.3731763325901154, 1.445305721320277)


ROUND = True  # emulate the kernels' BF16 operand rounding; False = plain float64


def bf16(x: torch.Tensor) -> torch.Tensor:
    if not ROUND:
        return x.double()
    return x.to(torch.bfloat16).to(torch.float64)


def sh4(d: torch.Tensor) -> torch.Tensor:
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    xx, yy, zz = x * x, y * y, z * z
    c = SH
    return torch.stack([
        torch.full_like(x, c[0]), -c[1] * y, c[1] * z, -c[1] * x,
        c[2] * x * y, -c[2] * y * z, c[3] * (2 * zz - xx - yy), -c[2] * x * z, c[4] * (xx - yy),
        -c[5] * y * (3 * xx - yy), c[6] * x * y * z, -c[7] * y * (4 * zz - xx - yy),
        c[8] * z * (2 * zz - 3 * xx - 3 * yy), -c[7] * x * (4 * zz - xx - yy), c[9] * z * (xx - yy),
        -c[5] * x * (xx - 3 * yy)], dim=1)


def level_offsets(res):
    off, out = 0, []
    for r in res:
        out.append(off)
        off += (r + 1) ** 3 * 2
    return out


def corners(u: torch.Tensor, r: int):
    g = u * r
    i = torch.clamp(g.floor().long(), max=r - 1)
    a = g - i
    out = []
    for k in range(8):
        dx, dy, dz = k & 1, (k >> 1) & 1, k >> 2
        idx = ((i[:, 2] + dz) * (r + 1) + (i[:, 1] + dy)) * (r + 1) + (i[:, 0] + dx)
        w = (a[:, 0] if dx else 1 - a[:, 0]) * (a[:, 1] if dy else 1 - a[:, 1]) * (a[:, 2] if dz else 1 - a[:, 2])
        out.append((idx, w))
    return out


def encode(grid, res, bmin, bmax, pos, dir):
    grid = grid.double()
    pos, dir = pos.double(), dir.double()
    u = ((pos - torch.tensor(bmin, dtype=torch.float64)) / (torch.tensor(bmax, dtype=torch.float64) -
                                                           torch.tensor(bmin, dtype=torch.float64))).clamp(0, 1)
    feats = []
    for l, (r, off) in enumerate(zip(res, level_offsets(res))):
        f = torch.zeros(pos.shape[0], 2, dtype=torch.float64)
        for idx, w in corners(u, r):
            f += w[:, None] * grid[off + 2 * idx[:, None] + torch.arange(2)]
        feats.append(f)
    x = torch.cat(feats + [sh4(dir), torch.ones(pos.shape[0], 1, dtype=torch.float64),
                           torch.zeros(pos.shape[0], 15, dtype=torch.float64)], dim=1)
    return x, u


def split_weights(w: torch.Tensor):
    w = w.double()
    Ws, o = [], 0
    for l in range(5):
        n = 64 if l < 4 else 16
        Ws.append(w[o:o + n * 64].reshape(n, 64))
        o += n * 64
    return Ws


def mlp_forward(weights, x):
    """Returns the output [n,16] and the BF16 layer inputs a0..a4."""
    Ws = [bf16(W) for W in split_weights(weights)]
    a = bf16(x.double())
    acts = [a]
    for l in range(5):
        y = a @ Ws[l].T
        if l < 4:
            a = bf16(torch.relu(y))
            acts.append(a)
    return y, acts


def train_grads(grid, weights, res, bmin, bmax, pos, dir, target):
    """(loss, d weights, d grid) of the relative L2 loss with the kernels' rounding."""
    n = pos.shape[0]
    x, u = encode(grid, res, bmin, bmax, pos, dir)
    y, acts = mlp_forward(weights, x)
    Ws = [bf16(W) for W in split_weights(weights)]
    t = target.double()
    yy = y[:, :3]
    den = yy * yy + 0.01
    loss = ((yy - t) ** 2 / den).sum() / n
    g = torch.zeros(n, 16, dtype=torch.float64)
    g[:, :3] = 2 * (yy - t) / den / n
    g = bf16(g)
    dW = [None] * 5
    for l in range(4, -1, -1):
        dW[l] = g.T @ acts[l]
        dx = g @ Ws[l]
        if l > 0:
            g = bf16(dx * (acts[l] > 0))
    dgrid = torch.zeros(grid.numel(), dtype=torch.float64)
    for l, (r, off) in enumerate(zip(res, level_offsets(res))):
        for idx, w in corners(u, r):
            for f in range(2):
                dgrid.index_add_(0, off + 2 * idx + f, w * dx[:, 2 * l + f])
    return loss, torch.cat([d.reshape(-1) for d in dW]), dgrid
