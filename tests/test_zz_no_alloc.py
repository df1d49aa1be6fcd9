"""The allocation-free window entry point (collected last on purpose).

``ftle_window_run_mixed_chunked_static`` serves callers that cannot give the
engine device memory -- a host program whose own pool owns all device memory,
or a plugin that may not call cudaMalloc -- by using a 32 MiB workspace built
into the library.  It must give exactly the results of
``ftle_window_run_mixed_chunked`` with a caller workspace (same kernels, same
arithmetic: the tolerance is bit-exact), call after call, although every call
reuses the same built-in array.  Covered: 2D and 3D, RK4 and AB2 (whose history
buffers make the workspace larger), and windows whose workspace is just under
the 32 MiB limit.
"""

import math

import numpy as np
import pytest
import torch

from pyftle_b200 import SnapshotSeries, _lib, flows
from pyftle_b200._device import stream_ptr
from pyftle_b200.interpolate import GridSpec
from pyftle_b200.window import window_descriptor

pytestmark = pytest.mark.gpu

LIMIT = 32 << 20
STEPS = 60


def _series(dim):
    n = 32
    ax = flows.periodic_axis(n)
    S = 8
    dt = 2 * math.pi / S
    if dim == 3:
        snaps = flows.abc_snapshots(ax, ax, ax, np.arange(S) * dt)
        pts = flows.grid_points_3d(ax, ax, ax)
        grid = GridSpec.from_points(pts, (n, n, n), periodic=True)
    else:
        turb = flows.FourierTurbulence2D(seed=4, num_modes=32, kmin=2, kmax=8, urms=0.3)
        snaps = turb.snapshots(n, np.arange(S) * dt)
        X, Y = np.meshgrid(ax, ax)
        grid = GridSpec.from_points(np.stack((X.ravel(), Y.ravel())), (n, n), periodic=True)
    return SnapshotSeries(grid, snaps, precision="fx15", periodic_time=True), dt


def _seeds(dim, num_groups, seed):
    cents = np.random.default_rng(seed).uniform(0, 2 * math.pi, (num_groups, dim))
    return flows.seeds_3d(cents, 1e-3) if dim == 3 else flows.seeds_2d(cents, 1e-3)


def _desc(series, pos, ftle, dt, integrator):
    return window_descriptor(series, pos, ftle, integrator=integrator, time_mode="blend",
                             h=0.02, num_steps=STEPS, map_period=STEPS * 0.02, snapshot_dt=dt)


def _buffers(series, pos0):
    K = 2 * series.grid.dim
    pos = torch.as_tensor(pos0, device="cuda")
    return pos, torch.empty(pos.shape[0] // K, dtype=torch.float64, device="cuda")


def _run_with_workspace(series, pos0, dt, integrator):
    pos, ftle = _buffers(series, pos0)
    w = _desc(series, pos, ftle, dt, integrator)
    need = _lib.load().ftle_window_workspace_bytes(w)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    _lib.call("ftle_window_run_mixed_chunked", w, ws.data_ptr(), need, 7, 1, stream_ptr())
    torch.cuda.synchronize()
    return pos.cpu().numpy(), ftle.cpu().numpy()


def _run_static(series, pos0, dt, integrator):
    pos, ftle = _buffers(series, pos0)
    _lib.call("ftle_window_run_mixed_chunked_static", _desc(series, pos, ftle, dt, integrator),
              7, 1, stream_ptr())
    torch.cuda.synchronize()
    return pos.cpu().numpy(), ftle.cpu().numpy()


def _workspace_bytes(series, num_groups, integrator):
    """Workspace of a window of `num_groups` groups (the size rule reads only the
    descriptor's shape fields; the buffers here are never touched)."""
    dim = series.grid.dim
    pos = torch.empty((2 * dim, dim), dtype=torch.float64, device="cuda")
    w = _desc(series, pos, None, 1.0, integrator)
    w.num_groups = num_groups
    return _lib.load().ftle_window_workspace_bytes(w)


def _largest_groups_that_fit(series, integrator):
    lo, hi = 1, 1 << 22
    while lo < hi:
        mid = (lo + hi + 1) // 2
        if _workspace_bytes(series, mid, integrator) <= LIMIT:
            lo = mid
        else:
            hi = mid - 1
    return lo


@pytest.mark.parametrize("dim,integrator", [(3, "rk4"), (2, "rk4"), (3, "ab2"), (2, "ab2")])
def test_static_workspace_matches_caller_workspace_twice(dim, integrator):
    series, dt = _series(dim)
    pos0 = _seeds(dim, 3000, 5)
    ref_pos, ref_ftle = _run_with_workspace(series, pos0, dt, integrator)
    for _ in range(2):  # the second call finds the first call's data in the array
        pos, ftle = _run_static(series, pos0, dt, integrator)
        np.testing.assert_array_equal(pos, ref_pos)
        np.testing.assert_array_equal(ftle, ref_ftle)
    # a different, smaller window right after: nothing of the previous call leaks in
    pos2 = _seeds(dim, 1001, 9)
    ref_pos2, ref_ftle2 = _run_with_workspace(series, pos2, dt, integrator)
    pos, ftle = _run_static(series, pos2, dt, integrator)
    np.testing.assert_array_equal(pos, ref_pos2)
    np.testing.assert_array_equal(ftle, ref_ftle2)


@pytest.mark.parametrize("dim,integrator", [(3, "rk4"), (2, "ab2")])
def test_static_workspace_at_its_limit(dim, integrator):
    """The largest window whose workspace fits the 32 MiB is accepted and gives the
    caller-workspace bits; one group more is rejected."""
    series, dt = _series(dim)
    n = _largest_groups_that_fit(series, integrator)
    assert LIMIT - 4096 < _workspace_bytes(series, n, integrator) <= LIMIT
    assert _workspace_bytes(series, n + 1, integrator) > LIMIT
    pos0 = _seeds(dim, n, 11)
    ref_pos, ref_ftle = _run_with_workspace(series, pos0, dt, integrator)
    for _ in range(2):
        pos, ftle = _run_static(series, pos0, dt, integrator)
        np.testing.assert_array_equal(pos, ref_pos)
        np.testing.assert_array_equal(ftle, ref_ftle)
    pos, ftle = _buffers(series, _seeds(dim, n + 1, 12))
    with pytest.raises(_lib.FTLEError, match="built-in workspace holds"):
        _lib.call("ftle_window_run_mixed_chunked_static", _desc(series, pos, ftle, dt, integrator),
                  7, 1, stream_ptr())


def test_static_workspace_rejects_windows_beyond_its_size():
    series, dt = _series(3)
    big = 400_000  # groups: needs more than the 32 MiB built-in workspace
    pos = torch.zeros((6 * big, 3), dtype=torch.float64, device="cuda")
    w = _desc(series, pos, None, dt, "rk4")
    assert _lib.load().ftle_window_workspace_bytes(w) > LIMIT
    with pytest.raises(_lib.FTLEError, match="built-in workspace holds"):
        _lib.call("ftle_window_run_mixed_chunked_static", w, 7, 1, stream_ptr())
