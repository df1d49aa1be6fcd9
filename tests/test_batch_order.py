"""Host-side check of the Morton group order used by batched windows (no GPU)."""

import numpy as np
import torch

from pyftle_b200.batch import morton_order
from pyftle_b200.interpolate import GridSpec


def _seeds(cents, d=1e-3):
    dim = cents.shape[1]
    offs = []
    for a in range(dim):
        e = np.zeros(dim)
        e[a] = d
        offs += [-e, e] if a == 0 else [e, -e]
    return torch.as_tensor(np.concatenate([cents + o for o in offs]))


def _key(c, grid, bits):
    k = 0
    for a in range(grid.dim):
        ext = grid.spacing[a] * (grid.shape[a] if grid.periodic else grid.shape[a] - 1)
        f = (c[a] - grid.origin[a]) / ext
        f = f - np.floor(f) if grid.periodic else f
        cell = min(max(int(f * (1 << bits)), 0), (1 << bits) - 1)
        for b in range(bits):
            k |= ((cell >> b) & 1) << (grid.dim * b + a)
    return k


def test_morton_order_sorts_groups_by_centroid_cell():
    rng = np.random.default_rng(0)
    for dim, periodic in ((2, False), (3, True)):
        shape = (40, 30) if dim == 2 else (20, 16, 12)
        grid = GridSpec(shape=shape, origin=(0.5,) * dim, spacing=(0.25,) * dim, periodic=periodic)
        hi = [grid.origin[a] + grid.spacing[a] * (shape[a] - 1) for a in range(dim)]
        cents = rng.uniform(grid.origin[0], min(hi), (500, dim))
        pos = _seeds(cents)
        perm = morton_order(pos, grid).numpy()
        assert sorted(perm.tolist()) == list(range(500))
        bits = 10 if dim == 2 else 7
        keys = [_key(cents[g], grid, bits) for g in perm]
        assert all(a <= b for a, b in zip(keys, keys[1:]))


def test_morton_order_puts_non_finite_groups_last():
    grid = GridSpec(shape=(16, 16), origin=(0.0, 0.0), spacing=(1.0, 1.0))
    cents = np.random.default_rng(1).uniform(0.0, 14.0, (64, 2))
    cents[7] = np.nan
    perm = morton_order(_seeds(cents), grid).numpy()
    assert sorted(perm.tolist()) == list(range(64))
    assert perm[-1] == 7
