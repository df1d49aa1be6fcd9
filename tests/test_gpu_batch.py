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


@pytest.mark.parametrize("schedule", [Schedule(3, 1), Schedule(1, 0), Schedule(2, 1), Schedule(4, 2)])
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
    assert isinstance(best, Schedule) and len(batch.tuning) == 12  # 1..4 CTAs/SM x 3 orders
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


@pytest.mark.parametrize("integrator,time_mode", [("euler", "blend"), ("ab2", "blend"),
                                                  ("rk4", "hold"), ("ab2", "hold")])
def test_batch_integrators_and_hold_equal_windows_alone(series, integrator, time_mode):
    """The persistent kernel's Euler / AB2 paths and HOLD windows (step i holds snapshot
    first_snapshot + i) give the bits of the same windows run one by one."""
    rng = np.random.default_rng(7)
    runs, alone = [], []
    for i in range(5):
        cents = rng.uniform(0, 2 * math.pi, (int(rng.integers(40, 2500)), 2))
        pos = flows.seeds_2d(cents, 5e-4)
        steps = int(rng.integers(4, 18))  # HOLD: first + steps stays inside the 40 snapshots
        if time_mode == "hold":
            h = DT if i % 2 else -DT
            first = int(rng.integers(steps, S - steps))
            t0 = 0.0
        else:
            h = 0.01 if i % 2 else -0.01
            first = 0
            span = steps * abs(h)
            t0 = rng.uniform(span, (S - 1) * DT) if h < 0 else rng.uniform(0, (S - 1) * DT - span)
        mp = 0.37 + 0.01 * i  # explicit: both routes then normalise by the same T
        pt = torch.as_tensor(pos, device="cuda")
        f = run_window(series, pt, integrator=integrator, time_mode=time_mode, h=h,
                       num_steps=steps, t0=t0, first_snapshot=first, map_period=mp,
                       snapshot_dt=DT)
        torch.cuda.synchronize()
        alone.append((pt.cpu().numpy(), f.cpu().numpy()))
        runs.append(WindowSpecRun(torch.as_tensor(pos, device="cuda"), t0, h, steps,
                                  map_period=mp, first_snapshot=first))
    batch = WindowBatch(series, runs, integrator=integrator, time_mode=time_mode,
                        snapshot_dt=DT)
    ftles = batch.run(Schedule(4, 1))
    torch.cuda.synchronize()
    for (rp, rf), run, f in zip(alone, runs, ftles):
        np.testing.assert_array_equal(run.positions.cpu().numpy(), rp)
        np.testing.assert_array_equal(f.cpu().numpy(), rf)


@pytest.mark.parametrize("integrator", ["rk4", "ab2"])
def test_batch_3d_periodic_equals_windows_alone(integrator):
    n, S3 = 24, 8
    dt = 2 * math.pi / S3
    ax = flows.periodic_axis(n)
    snaps = flows.abc_snapshots(ax, ax, ax, np.arange(S3) * dt)
    grid = GridSpec.from_points(flows.grid_points_3d(ax, ax, ax), (n, n, n), periodic=True)
    s3 = SnapshotSeries(grid, snaps, precision="fx15", periodic_time=True)
    rng = np.random.default_rng(9)
    runs, alone = [], []
    for i in range(4):
        pos = flows.seeds_3d(rng.uniform(0, 2 * math.pi, (int(rng.integers(30, 900)), 3)), 1e-3)
        h = 0.02 if i % 2 else -0.02
        steps = int(rng.integers(10, 70))
        t0 = rng.uniform(0, 10.0)  # the series is periodic in time
        pt = torch.as_tensor(pos, device="cuda")
        f = run_window(s3, pt, integrator=integrator, time_mode="blend", h=h, num_steps=steps,
                       t0=t0, snapshot_dt=dt)
        torch.cuda.synchronize()
        alone.append((pt.cpu().numpy(), f.cpu().numpy()))
        runs.append(WindowSpecRun(torch.as_tensor(pos, device="cuda"), t0, h, steps))
    ftles = WindowBatch(s3, runs, integrator=integrator, snapshot_dt=dt).run(Schedule(2, 0))
    torch.cuda.synchronize()
    for (rp, rf), run, f in zip(alone, runs, ftles):
        np.testing.assert_array_equal(run.positions.cpu().numpy(), rp)
        np.testing.assert_array_equal(f.cpu().numpy(), rf)


def test_batch_spatial_order_is_bit_identical(series):
    """Morton-ordered groups (the default) and the caller's order give the same bits,
    for windows that update their positions and windows sharing read-only seeds."""
    rng = np.random.default_rng(12)
    shared = torch.as_tensor(flows.seeds_2d(rng.uniform(0, 2 * math.pi, (1500, 2)), 5e-4),
                             device="cuda")
    own = [flows.seeds_2d(rng.uniform(0, 2 * math.pi, (int(rng.integers(50, 900)), 2)), 5e-4)
           for _ in range(3)]
    out = []
    for order in (False, True):
        runs = [WindowSpecRun(shared, 0.3 + 0.2 * i, 0.01, 20 + 7 * i, keep_positions=True)
                for i in range(3)]
        runs += [WindowSpecRun(torch.as_tensor(p, device="cuda"), 0.5, -0.01, 25) for p in own]
        f = WindowBatch(series, runs, snapshot_dt=DT, spatial_order=order).run(Schedule(4, 1))
        torch.cuda.synchronize()
        out.append(([x.cpu().numpy() for x in f], [r.positions.cpu().numpy() for r in runs[3:]]))
    for a, b in zip(out[0][0], out[1][0]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(out[0][1], out[1][1]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(shared.cpu().numpy()[:4],
                                  flows.seeds_2d(np.random.default_rng(12).uniform(
                                      0, 2 * math.pi, (1500, 2)), 5e-4)[:4])


def test_batch_hold_default_map_period_equals_window_alone(series):
    """HOLD windows without an explicit map period are normalised like the reference
    (T = (steps - 1)|h|, ftle_solver.py:156), in a batch as when run alone."""
    rng = np.random.default_rng(21)
    runs, alone = [], []
    for i in range(3):
        pos = flows.seeds_2d(rng.uniform(0, 2 * math.pi, (int(rng.integers(40, 700)), 2)), 5e-4)
        steps = int(rng.integers(4, 15))
        h = DT if i % 2 else -DT
        first = int(rng.integers(steps, S - steps))
        pt = torch.as_tensor(pos, device="cuda")
        f = run_window(series, pt, integrator="rk4", time_mode="hold", h=h, num_steps=steps,
                       first_snapshot=first, snapshot_dt=DT)
        torch.cuda.synchronize()
        alone.append(f.cpu().numpy())
        runs.append(WindowSpecRun(torch.as_tensor(pos, device="cuda"), 0.0, h, steps,
                                  first_snapshot=first))
    ftles = WindowBatch(series, runs, time_mode="hold", snapshot_dt=DT).run(Schedule(4, 1))
    torch.cuda.synchronize()
    for rf, f in zip(alone, ftles):
        np.testing.assert_array_equal(f.cpu().numpy(), rf)


def test_batch_and_window_reject_bad_ftle_buffers(series):
    pos = torch.as_tensor(flows.seeds_2d(np.full((10, 2), 1.0), 5e-4), device="cuda")
    bad = [torch.empty(9, dtype=torch.float64, device="cuda"),
           torch.empty(10, dtype=torch.float32, device="cuda"),
           torch.empty(20, dtype=torch.float64, device="cuda")[::2],
           torch.empty(10, dtype=torch.float64)]
    for f in bad:
        with pytest.raises(ValueError, match="ftle must be"):
            run_window(series, pos.clone(), time_mode="blend", h=0.01, num_steps=3,
                       snapshot_dt=DT, ftle_out=f)
        with pytest.raises(ValueError, match="ftle must be"):
            WindowBatch(series, [WindowSpecRun(pos.clone(), 0.0, 0.01, 3, ftle=f)],
                        snapshot_dt=DT)


def test_batch_prefix_view_of_shared_seeds_is_not_shared(series):
    """A window over a prefix view of another window's read-only seeds starts at the same
    address; it must get its own ordered copy (and its own N), not the larger one."""
    rng = np.random.default_rng(31)
    big_h = flows.seeds_2d(rng.uniform(0, 2 * math.pi, (900, 2)), 5e-4)
    big = torch.as_tensor(big_h, device="cuda")
    n_small = 300
    prefix = big[:4 * n_small]  # same data_ptr, fewer rows (role blocks of its own)
    runs = [WindowSpecRun(big, 0.3, 0.01, 12, keep_positions=True),
            WindowSpecRun(prefix, 0.3, 0.01, 12, keep_positions=True)]
    ftles = WindowBatch(series, runs, snapshot_dt=DT).run(Schedule(4, 1))
    torch.cuda.synchronize()
    ref_big = run_window(series, big.clone(), integrator="rk4", time_mode="blend", h=0.01,
                         num_steps=12, t0=0.3, snapshot_dt=DT)
    ref_prefix = run_window(series, prefix.clone(), integrator="rk4", time_mode="blend",
                            h=0.01, num_steps=12, t0=0.3, snapshot_dt=DT)
    torch.cuda.synchronize()
    assert ftles[1].numel() == n_small
    np.testing.assert_array_equal(ftles[0].cpu().numpy(), ref_big.cpu().numpy())
    np.testing.assert_array_equal(ftles[1].cpu().numpy(), ref_prefix.cpu().numpy())


# ---------------------------------------------------------------------------
# FP64 judge on a 1% sample of every window, FP64 re-advection of failing windows
# ---------------------------------------------------------------------------

@pytest.fixture(scope="module")
def bf16_and_fp64():
    turb = flows.FourierTurbulence2D(seed=3, num_modes=96, kmin=4, kmax=30)
    snaps = turb.snapshots(N_GRID, np.arange(S) * DT)
    ax = flows.periodic_axis(N_GRID)
    X, Y = np.meshgrid(ax, ax)
    grid = GridSpec.from_points(np.stack((X.ravel(), Y.ravel())), (N_GRID, N_GRID), periodic=True)
    # BF16 storage: errors of 1e-3..1e-2, so a tolerance in between splits the windows
    return (SnapshotSeries(grid, snaps, precision="bf16"),
            SnapshotSeries(grid, snaps, precision="fp64"))


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_judge_readvects_exactly_the_windows_above_tolerance(bf16_and_fp64):
    sbf, s64 = bf16_and_fp64
    wins = _windows(np.random.default_rng(11), count=8)
    mixed = _alone(sbf, wins)
    fp64 = _alone(s64, wins)
    stride = 10
    # the judge's error of window i: groups i % stride, i % stride + stride, ...
    expect = []
    for i, ((_, fm), (_, f64)) in enumerate(zip(mixed, fp64)):
        sel = np.arange(i % stride if fm.size > i % stride else 0, fm.size, stride)
        expect.append(_rel_l2(fm[sel], f64[sel]))
    tol = float(np.median(expect))
    batch, runs = _batch(sbf, wins)
    rep = batch.run_judged(s64, tol=tol, sample_stride=stride)
    torch.cuda.synchronize()
    np.testing.assert_allclose(rep.errors, expect, rtol=1e-12)
    assert rep.readvected == [e > tol for e in rep.errors]
    assert 0 < sum(rep.readvected) < len(wins)
    for run, redo, (pm, fm), (p64, f64) in zip(runs, rep.readvected, mixed, fp64):
        want_p, want_f = (p64, f64) if redo else (pm, fm)
        np.testing.assert_array_equal(run.ftle.cpu().numpy(), want_f)
        np.testing.assert_array_equal(run.positions.cpu().numpy(), want_p)


def test_judge_without_fallback_only_reports(bf16_and_fp64):
    sbf, s64 = bf16_and_fp64
    wins = _windows(np.random.default_rng(12), count=4)
    mixed = _alone(sbf, wins)
    batch, runs = _batch(sbf, wins)
    rep = batch.run_judged(s64, tol=0.0, fallback=False)
    torch.cuda.synchronize()
    assert rep.readvected == [False] * len(wins) and all(e > 0 for e in rep.errors)
    for run, (pm, fm) in zip(runs, mixed):
        np.testing.assert_array_equal(run.ftle.cpu().numpy(), fm)
        np.testing.assert_array_equal(run.positions.cpu().numpy(), pm)


def test_judge_readvects_windows_over_shared_read_only_seeds(bf16_and_fp64):
    sbf, s64 = bf16_and_fp64
    rng = np.random.default_rng(13)
    seeds = torch.as_tensor(flows.seeds_2d(rng.uniform(0, 2 * math.pi, (1500, 2)), 5e-4),
                            device="cuda")
    seeds0 = seeds.clone()
    specs = [(0.1, 60), (0.4, 25), (0.9, 80)]
    runs = [WindowSpecRun(seeds, t0, 0.01, st, keep_positions=True) for t0, st in specs]
    batch = WindowBatch(sbf, runs, snapshot_dt=DT)
    rep = batch.run_judged(s64, tol=0.0)
    torch.cuda.synchronize()
    assert rep.readvected == [True] * len(specs)
    torch.testing.assert_close(seeds, seeds0, rtol=0, atol=0)
    for run, (t0, st) in zip(runs, specs):
        f = run_window(s64, seeds0.clone(), integrator="rk4", time_mode="blend", h=0.01,
                       num_steps=st, t0=t0, snapshot_dt=DT)
        torch.testing.assert_close(run.ftle, f, rtol=0, atol=0)


def test_judge_rejects_a_mixed_series_as_judge(bf16_and_fp64):
    sbf, _ = bf16_and_fp64
    batch, _ = _batch(sbf, _windows(np.random.default_rng(14), count=2))
    with pytest.raises(ValueError, match="fp64"):
        batch.run_judged(sbf)


def test_judge_hold_ab2_windows_readvect_to_the_fp64_bits(bf16_and_fp64):
    """HOLD windows (step i holds snapshot first_snapshot + i, the reference's T = (p-1)|h|)
    with AB2: the judge hands the FP64 kernel the windows' own integrator, time mode,
    first snapshot and FTLE period, so re-advected windows equal the plain FP64 path
    run alone, bit for bit."""
    sbf, s64 = bf16_and_fp64
    rng = np.random.default_rng(15)
    specs, runs = [], []
    for i in range(3):
        pos = flows.seeds_2d(rng.uniform(0, 2 * math.pi, (int(rng.integers(200, 1500)), 2)),
                             5e-4)
        steps = int(rng.integers(6, 15))
        h = DT if i % 2 else -DT
        first = int(rng.integers(steps, S - steps))
        specs.append((pos, h, steps, first))
        runs.append(WindowSpecRun(torch.as_tensor(pos, device="cuda"), 0.0, h, steps,
                                  first_snapshot=first))
    batch = WindowBatch(sbf, runs, integrator="ab2", time_mode="hold", snapshot_dt=DT)
    rep = batch.run_judged(s64, tol=0.0, sample_stride=7)
    torch.cuda.synchronize()
    assert rep.readvected == [True] * 3
    for run, (pos, h, steps, first) in zip(runs, specs):
        pt = torch.as_tensor(pos, device="cuda")
        f = run_window(s64, pt, integrator="ab2", time_mode="hold", h=h, num_steps=steps,
                       first_snapshot=first, snapshot_dt=DT)
        torch.testing.assert_close(run.ftle, f, rtol=0, atol=0)
        torch.testing.assert_close(run.positions, pt, rtol=0, atol=0)


def test_judge_rejects_a_judge_series_of_other_snapshots(bf16_and_fp64):
    sbf, s64 = bf16_and_fp64
    batch, _ = _batch(sbf, _windows(np.random.default_rng(16), count=2))
    periodic = SnapshotSeries(s64.grid, torch.zeros((S, 2, s64.grid.nodes), dtype=torch.float64,
                                                    device="cuda"),
                              precision="fp64", periodic_time=True)
    with pytest.raises(ValueError, match="time periodicity"):
        batch.run_judged(periodic)
