"""The allocation-free window entry point (collected last on purpose).

``ftle_window_run_mixed_chunked_static`` serves callers that cannot give the
engine device memory -- a host program whose own pool owns all device memory,
or a plugin that may not call cudaMalloc -- by using a 32 MiB workspace built
into the library.  It must give exactly the results of
``ftle_window_run_mixed_chunked`` with a caller workspace (same kernels, same
arithmetic: the tolerance is bit-exact), call after call, although every call
reuses the same built-in array.
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


def _case(num_groups, seed):
    n = 32
    ax = flows.periodic_axis(n)
    S = 8
    snaps = flows.abc_snapshots(ax, ax, ax, np.arange(S) * (2 * math.pi / S))
    pts = flows.grid_points_3d(ax, ax, ax)
    grid = GridSpec.from_points(pts, (n, n, n), periodic=True)
    series = SnapshotSeries(grid, snaps, precision="fx15", periodic_time=True)
    cents = np.random.default_rng(seed).uniform(0, 2 * math.pi, (num_groups, 3))
    return series, flows.seeds_3d(cents, 1e-3), 2 * math.pi / S


def _desc(series, pos, ftle, dt):
    return window_descriptor(series, pos, ftle, integrator="rk4", time_mode="blend", h=0.02,
                             num_steps=60, map_period=60 * 0.02, snapshot_dt=dt)


def _run_with_workspace(series, pos0, dt):
    pos = torch.as_tensor(pos0, device="cuda")
    ftle = torch.empty(pos.shape[0] // 6, dtype=torch.float64, device="cuda")
    w = _desc(series, pos, ftle, dt)
    need = _lib.load().ftle_window_workspace_bytes(w)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    _lib.call("ftle_window_run_mixed_chunked", w, ws.data_ptr(), need, 7, 1, stream_ptr())
    torch.cuda.synchronize()
    return pos.cpu().numpy(), ftle.cpu().numpy()


def _run_static(series, pos0, dt):
    pos = torch.as_tensor(pos0, device="cuda")
    ftle = torch.empty(pos.shape[0] // 6, dtype=torch.float64, device="cuda")
    _lib.call("ftle_window_run_mixed_chunked_static", _desc(series, pos, ftle, dt), 7, 1,
              stream_ptr())
    torch.cuda.synchronize()
    return pos.cpu().numpy(), ftle.cpu().numpy()


def test_static_workspace_matches_caller_workspace_twice():
    series, pos0, dt = _case(3000, 5)
    ref_pos, ref_ftle = _run_with_workspace(series, pos0, dt)
    for _ in range(2):  # the second call finds the first call's data in the array
        pos, ftle = _run_static(series, pos0, dt)
        np.testing.assert_array_equal(pos, ref_pos)
        np.testing.assert_array_equal(ftle, ref_ftle)
    # a different, smaller window right after: nothing of the previous call leaks in
    series2, pos2, dt2 = _case(1001, 9)
    ref_pos2, ref_ftle2 = _run_with_workspace(series2, pos2, dt2)
    pos, ftle = _run_static(series2, pos2, dt2)
    np.testing.assert_array_equal(pos, ref_pos2)
    np.testing.assert_array_equal(ftle, ref_ftle2)


def test_static_workspace_rejects_windows_beyond_its_size():
    series, pos0, dt = _case(2, 1)
    big = 400_000  # groups: needs more than the 32 MiB built-in workspace
    pos = torch.zeros((6 * big, 3), dtype=torch.float64, device="cuda")
    w = _desc(series, pos, None, dt)
    assert _lib.load().ftle_window_workspace_bytes(w) > 32 << 20
    with pytest.raises(_lib.FTLEError, match="built-in workspace holds"):
        _lib.call("ftle_window_run_mixed_chunked_static", w, 7, 1, stream_ptr())
