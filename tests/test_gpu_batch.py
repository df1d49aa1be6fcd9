"""Many windows in one persistent launch (config-3 style batches).

Every window of a batch must come out bit-identical to the same window run on
its own (same per-group arithmetic, only the scheduling differs), also through a
captured CUDA graph and after autotuning.
"""

import math

import numpy as np
import pytest
import torch

from pyftle_b200 import SnapshotSeries, flows, run_window
from pyftle_b200.batch import Schedule, WindowBatch, WindowSpecRun
from pyftle_b200.interpolate import GridSpec

pytestmark = pytest.mark.gpu

N_GRID = 128
S = 40
DT = 0.05


@pytest.fixture(scope="module")
def series():
    turb = flows.FourierTurbulence2D(seed=3, num_modes=96, kmin=4, kmax=30)
    snaps = turb.snapshots(N_GRID, np.arange(S) * DT)
    ax = flows.periodic_axis(N_GRID)
    X, Y = np.meshgrid(ax, ax)
    pts = np.stack((X.ravel(), Y.ravel()))
    grid = GridSpec.from_points(pts, (N_GRID, N_GRID), periodic=True)
    return SnapshotSeries(grid, snaps, precision="fx15")


def _windows(rng, count=7):
    L = 2 * math.pi
    out = []
    for i in range(count):
        ng = int(rng.integers(20, 3000))
        cents = rng.uniform(0, L, (ng, 2))
        h = 0.01 if i % 3 else -0.01
        steps = int(rng.integers(5, 90))
        span = steps * abs(h)
        t_end = (S - 1) * DT
        t0 = rng.uniform(span, t_end) if h < 0 else rng.uniform(0.0, t_end - span)
        out.append((flows.seeds_2d(cents, 5e-4), t0, h, steps))
    return out


def _batch(series, wins):
    runs = [WindowSpecRun(torch.as_tensor(p, device="cuda"), t0, h, st) for p, t0, h, st in wins]
    return WindowBatch(series, runs, snapshot_dt=DT), runs


def _alone(series, wins):
    res = []
    for p, t0, h, st in wins:
        pt = torch.as_tensor(p, device="cuda")
        f = run_window(series, pt, integrator="rk4", time_mode="blend", h=h, num_steps=st, t0=t0,
                       snapshot_dt=DT)
        torch.cuda.synchronize()
        res.append((pt.cpu().numpy(), f.cpu().numpy()))
    return res


@pytest.mark.parametrize("schedule", [Schedule(3, 1), Schedule(1, 0), Schedule(2, 1)])
def test_batch_equals_windows_alone(series, schedule):
    wins = _windows(np.random.default_rng(1))
    ref = _alone(series, wins)
    batch, runs = _batch(series, wins)
    ftles = batch.run(schedule)
    torch.cuda.synchronize()
    for (rp, rf), run, f in zip(ref, runs, ftles):
        np.testing.assert_array_equal(run.positions.cpu().numpy(), rp)
        np.testing.assert_array_equal(f.cpu().numpy(), rf)


def test_batch_graph_replay_and_autotune(series):
    wins = _windows(np.random.default_rng(2), count=5)
    ref = _alone(series, wins)
    batch, runs = _batch(series, wins)
    pristine = [r.positions.clone() for r in runs]

    def reset():
        for r, p in zip(runs, pristine):
            r.positions.copy_(p)

    best = batch.autotune(prologue=reset, use_cache=False)
    assert isinstance(best, Schedule) and len(batch.tuning) == 8  # 1..4 CTAs/SM x 2 orders
    batch.capture(prologue=reset)
    for _ in range(2):
        ftles = batch.replay()
        torch.cuda.synchronize()
        for (rp, rf), run, f in zip(ref, runs, ftles):
            np.testing.assert_array_equal(run.positions.cpu().numpy(), rp)
            np.testing.assert_array_equal(f.cpu().numpy(), rf)


def test_batch_rejects_mixed_series(series):
    wins = _windows(np.random.default_rng(4), count=2)
    other = SnapshotSeries(series.grid, torch.zeros((S, 2, N_GRID * N_GRID), device="cuda"),
                           precision="fx15")
    runs = [WindowSpecRun(torch.as_tensor(p, device="cuda"), t0, h, st) for p, t0, h, st in wins]
    batch = WindowBatch(series, runs, snapshot_dt=DT)
    from pyftle_b200 import _lib
    from pyftle_b200.window import window_descriptor

    batch.desc[1] = window_descriptor(other, runs[1].positions, runs[1].ftle, integrator="rk4",
                                      time_mode="blend", h=runs[1].h,
                                      num_steps=runs[1].num_steps, map_period=1.0,
                                      snapshot_dt=DT)
    with pytest.raises(_lib.FTLEError, match="share"):
        batch.run()


def test_device_turbulence_snapshots_match_host():
    turb = flows.FourierTurbulence2D(seed=5, num_modes=64, kmin=4, kmax=20)
    times = np.array([0.0, 0.37])
    host = turb.snapshots(64, times)
    dev = turb.snapshots_device(64, times).cpu().numpy()
    np.testing.assert_allclose(dev, host, rtol=0, atol=1e-12)
