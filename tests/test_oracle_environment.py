"""Image environment and its quadtree direction sampler (CPU only):
Image2D(image).after(xr_projection) and XRQuadtreeRandomDirection
(_maps.py:2494-2549, _objects.py:165-199, _functions.py:509-530)."""
import math

import numpy as np
import torch

import oracle
from rendervous_b200 import maps, synthetic
from tests.helpers import oracle_desc


def _sky(h=32, w=64, seed=3):
    rng = np.random.default_rng(seed)
    img = 0.2 + rng.random((h, w, 3)).astype(np.float32)
    img[4:7, 40:44] += 30.0                      # a small bright "sun" patch
    return img


def test_quadtree_layout_sums_children():
    """Each node holds its region's probability: levels sum to 1 and every
    node is the sum of its four children (children of node k at 4k+1..4k+4)."""
    qt = maps.environment_quadtree(torch.from_numpy(_sky()), levels=4).reshape(-1).numpy().astype(np.float64)
    assert qt.size == 4 + 16 + 64 + 256
    off = 0
    for l in range(1, 5):
        assert abs(qt[off:off + 4 ** l].sum() - 1.0) < 1e-5
        off += 4 ** l
    for k in range(0, 4 + 16 + 64):           # nodes with children
        node = k + 1                           # entry k holds node k+1 (root is node 0)
        ch = qt[4 * node:4 * node + 4]
        assert abs(qt[k] - ch.sum()) <= 1e-6 + 1e-5 * qt[k]


def test_quadtree_sampler_is_unbiased_and_importance_samples():
    """E[E(w) * weight] under the quadtree sampler equals the uniform-sphere
    estimate of the same integral of the image over directions, with far less
    spread, and most draws land on the bright patch."""
    img = _sky()
    desc = oracle_desc(synthetic.gaussian_blobs(5, 1, 1.0, seed=1))
    desc["env_image"] = img
    uni = oracle.OracleScene(desc)
    n = 200000
    eu = oracle.env_sample(uni, n, 5)[:, :3].astype(np.float64)
    desc_q = dict(desc)
    desc_q["env_quadtree"] = maps.environment_quadtree(torch.from_numpy(img), levels=6).numpy()
    desc_q["env_levels"] = 6
    q = oracle.OracleScene(desc_q)
    sq = oracle.env_sample(q, n, 7).astype(np.float64)
    eq = sq[:, :3]
    se = np.sqrt(eu.var(0) / n + eq.var(0) / n)
    assert (np.abs(eu.mean(0) - eq.mean(0)) < 4 * se).all(), (eu.mean(0), eq.mean(0), se)
    assert (eq.std(0) < 0.5 * eu.std(0)).all()
    # directions towards the patch (rows 4..6 of 32, columns 40..43 of 64)
    def on_patch(w):
        theta = np.arccos(np.clip(w[:, 1], -1, 1)) / math.pi * 32
        phi = (np.arctan2(w[:, 0], w[:, 2]) / math.pi + 1) / 2 * 64
        return ((theta > 4) & (theta < 7) & (phi > 40) & (phi < 44)).mean()
    assert on_patch(sq[:, 3:]) > 10 * on_patch(oracle.env_sample(uni, n, 5)[:, 3:].astype(np.float64))
