"""Parity on the full-size benchmark configurations (not toy grids).

The GPU runs each configuration at its full size; the CPU oracle (pinned to
pyFTLE's own outputs by tests/test_oracle.py) advects a strided subset of the
same seed groups, which is exact because groups are independent.

Tolerances (written per test):
  * plain FP64 path: positions bit-exact, FTLE rtol 1e-10 against the oracle;
  * chosen mixed path (FX15 snapshots, FP32 split advection, FP64 Cauchy-Green):
    FTLE relative error <= 1e-3, where the FTLE relative error of a field is
    ||F - F_ref||_2 / ||F_ref||_2 over the field (relative L2).  The pointwise
    99th percentile of |F - F_ref| / rms(F_ref) is checked too (<= 5e-3).

Configurations:
  1-ref  2D double gyre (A = 0.1, eps = 0.25, omega = 2 pi/10) on a 512 x 256 grid
         over [0,2] x [0,1], 201 snapshots at dt = 0.05, 400 x 200 centroids x 4
         neighbours at delta = 1e-3, the reference's HOLD RK4 with h = dt: through the
         reference-facing FTLESolver on all 80,000 groups, 2,500 random groups checked.
  1      the same field time-blended, RK4 h = 0.01 over T = 10 (1000 steps).
  2      3D time-periodic ABC flow on a periodic 128^3 grid, 64 snapshots over one
         period, 256^3 centroids x 6 neighbours at delta = 1e-3, RK4 h = 0.02 over
         T = 8 (400 steps), time-blended: the chosen path chunked (50 steps) with cell
         sorts on all 16.8M groups, 4,096 groups checked.
"""

import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from pyftle_b200 import (FTLESolver, MemoryBatchSource, SnapshotSeries, create_integrator,
                         create_interpolator, flows, run_window)
from pyftle_b200.interpolate import GridSpec

pytestmark = pytest.mark.gpu

FTLE_RTOL_F64 = 1e-10
FTLE_REL_L2 = 1e-3
FTLE_P99 = 5e-3


def _subset(pos, K, N, idx):
    return np.ascontiguousarray(np.concatenate([pos[r * N + idx] for r in range(K)]))


def _errors(got, ref):
    d = got - ref
    rel_l2 = float(np.linalg.norm(d) / np.linalg.norm(ref))
    p99 = float(np.quantile(np.abs(d), 0.99) / np.sqrt(np.mean(ref ** 2)))
    return rel_l2, p99


@pytest.fixture(scope="module")
def gyre():
    shape = (512, 256)
    pts = flows.grid_points_2d(*shape, (0.0, 2.0), (0.0, 1.0))
    dt = 0.05
    snaps = flows.double_gyre_snapshots(pts, np.arange(201) * dt)
    pos0 = flows.seeds_2d(flows.centroid_grid_2d(400, 200, (0.005, 1.995), (0.005, 0.995)), 1e-3)
    N = pos0.shape[0] // 4
    # 2,500 groups drawn uniformly (seeded): a sample of the whole field, edges included
    # in proportion (a regular stride aliases with the 400-wide seed rows)
    idx = np.sort(np.random.default_rng(400).choice(N, 2500, replace=False))
    return dict(shape=shape, pts=pts, dt=dt, snaps=snaps, pos0=pos0, N=N, idx=idx)


def test_config1_ref_hold_solver_bitexact(gyre):
    g = gyre
    src = MemoryBatchSource(list(g["snaps"]), g["pts"], g["pos0"].copy(), g["dt"],
                            grid_shape=g["shape"])
    integ = create_integrator("rk4", create_interpolator("grid", g["shape"]))
    solver = FTLESolver(src, integ)
    ftle = solver.run()
    pos = solver.particles.positions_host()
    gmin, gdel = O.grid_axes(g["pts"], g["shape"])
    sub = _subset(g["pos0"], 4, g["N"], g["idx"])
    p_ref, f_ref = O.run_window(g["snaps"], g["shape"], gmin, gdel, sub, integrator="rk4",
                                snap_dt=g["dt"])
    assert len(g["idx"]) >= 2000
    np.testing.assert_array_equal(_subset(pos, 4, g["N"], g["idx"]), p_ref)
    np.testing.assert_allclose(ftle[g["idx"]], f_ref, rtol=FTLE_RTOL_F64, atol=0)


def test_config1_blend_fp64_and_fx15(gyre):
    g = gyre
    grid = GridSpec.from_points(g["pts"], g["shape"])
    d_snaps = torch.from_numpy(g["snaps"]).cuda()
    kw = dict(integrator="rk4", time_mode="blend", h=0.01, num_steps=1000,
              snapshot_dt=g["dt"], map_period=10.0)
    gmin, gdel = O.grid_axes(g["pts"], g["shape"])
    sub = _subset(g["pos0"], 4, g["N"], g["idx"])
    p_ref, f_ref = O.run_window(g["snaps"], g["shape"], gmin, gdel, sub, integrator="rk4",
                                time_mode=O.BLEND, h=0.01, num_steps=1000, snap_dt=g["dt"],
                                map_period=10.0)
    # plain FP64 on the checked groups: the oracle's bits
    s64 = SnapshotSeries(grid, d_snaps, precision="fp64")
    p = torch.from_numpy(sub).cuda()
    f = run_window(s64, p, **kw)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(p.cpu().numpy(), p_ref)
    np.testing.assert_allclose(f.cpu().numpy(), f_ref, rtol=FTLE_RTOL_F64, atol=0)
    # chosen FX15 path on every group (chunked, cell-sorted)
    sfx = SnapshotSeries(grid, d_snaps, precision="fx15")
    p = torch.from_numpy(g["pos0"]).cuda()
    f = run_window(sfx, p, chunk_steps=100, sort_every=1, **kw)
    torch.cuda.synchronize()
    rel_l2, p99 = _errors(f.cpu().numpy()[g["idx"]], f_ref)
    assert rel_l2 <= FTLE_REL_L2, rel_l2
    assert p99 <= FTLE_P99, p99


@pytest.fixture(scope="module")
def abc128():
    n, S = 128, 64
    L = 2 * math.pi
    ax = flows.periodic_axis(n, L)
    dt = L / S
    snaps_d = flows.abc_snapshots_device(ax, ax, ax, np.arange(S) * dt)
    grid = GridSpec(shape=(n, n, n), origin=(0.0,) * 3, spacing=(ax[1],) * 3, periodic=True)
    m = 256
    c = (np.arange(m) + 0.5) * (L / m)
    X, Y, Z = np.meshgrid(c, c, c)
    cents = np.column_stack((X.ravel(), Y.ravel(), Z.ravel()))
    del X, Y, Z
    pos0 = flows.seeds_3d(cents, 1e-3)
    del cents
    N = pos0.shape[0] // 6
    idx = np.arange(0, N, N // 4096)
    return dict(n=n, ax=ax, dt=dt, snaps_d=snaps_d, grid=grid, pos0=pos0, N=N, idx=idx)


def test_config2_abc128_chosen_path_vs_oracle(abc128):
    a = abc128
    kw = dict(integrator="rk4", time_mode="blend", h=0.02, num_steps=400, snapshot_dt=a["dt"],
              map_period=8.0)
    sub = _subset(a["pos0"], 6, a["N"], a["idx"])
    n = a["n"]
    gmin = np.zeros(3)
    gdel = np.full(3, a["ax"][1])
    p_ref, f_ref = O.run_window(a["snaps_d"].cpu().numpy(), (n, n, n), gmin, gdel, sub,
                                integrator="rk4", time_mode=O.BLEND, h=0.02, num_steps=400,
                                snap_dt=a["dt"], periodic_space=True, periodic_time=True,
                                map_period=8.0)
    # plain FP64 path on the checked groups: the oracle's bits
    s64 = SnapshotSeries(a["grid"], a["snaps_d"], precision="fp64", periodic_time=True)
    p = torch.from_numpy(sub).cuda()
    f = run_window(s64, p, **kw)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(p.cpu().numpy(), p_ref)
    np.testing.assert_allclose(f.cpu().numpy(), f_ref, rtol=FTLE_RTOL_F64, atol=0)
    del s64
    # the chosen path as benchmarked: all 16.8M groups, 50-step chunks, cell sort each
    # time, in both 16-bit fixed-point storages
    for storage in ("fx15", "fx16"):
        sfx = SnapshotSeries(a["grid"], a["snaps_d"], precision=storage, periodic_time=True)
        p = torch.from_numpy(a["pos0"]).cuda()
        f = run_window(sfx, p, chunk_steps=50, sort_every=1, **kw)
        torch.cuda.synchronize()
        got = f.cpu().numpy()[a["idx"]]
        del p, f, sfx
        torch.cuda.empty_cache()
        rel_l2, p99 = _errors(got, f_ref)
        assert rel_l2 <= FTLE_REL_L2, (storage, rel_l2)
        assert p99 <= FTLE_P99, (storage, p99)


def test_config3_turbulence_batch_vs_oracle():
    """Config 3's field (2D random-Fourier turbulence, 256 modes, k in [4, 128], rms
    speed 0.02, 1024^2 periodic grid, FX15 snapshots at dt = 0.05) and six uneven windows
    in one persistent launch (RK4 h = 0.025, delta = 5e-4).  Two of them are checked
    against the oracle on 1,000 random groups each: the plain FP64 path bit-exact, the
    batched FX15 windows within 1e-3 (relative L2).  The oracle gets only the snapshots
    of each window's time range (snapshot index offset by the window's first one)."""
    from pyftle_b200.batch import WindowBatch, WindowSpecRun

    n, dt, h = 1024, 0.05, 0.025
    L = 2 * math.pi
    turb = flows.FourierTurbulence2D(seed=7, num_modes=256, kmin=4, kmax=128, urms=0.02)
    S = 280
    snaps_d = turb.snapshots_device(n, np.arange(S) * dt)
    ax = flows.periodic_axis(n)
    grid = GridSpec(shape=(n, n), origin=(0.0, 0.0), spacing=(ax[1], ax[1]), periodic=True)
    sfx = SnapshotSeries(grid, snaps_d, precision="fx15")
    rng = np.random.default_rng(33)
    specs = [(512, 3.0, 80), (96, 1.1, 40), (256, 10.0, 120), (200, 5.0, 300), (64, 0.2, 20),
             (1024, 8.0, 60)]  # (seeds per row, t0, steps)
    runs, seeds = [], []
    for nx, t0, steps in specs:
        ny = max(1, nx // 2)
        cx = (np.arange(nx) + 0.5) * (L / nx)
        cy = (np.arange(ny) + 0.5) * (L / ny)
        X, Y = np.meshgrid(cx, cy)
        pos = flows.seeds_2d(np.column_stack((X.ravel(), Y.ravel())), 5e-4)
        seeds.append(pos)
        runs.append(WindowSpecRun(torch.as_tensor(pos, device="cuda"), t0, h, steps))
    ftles = WindowBatch(sfx, runs, snapshot_dt=dt).run()
    torch.cuda.synchronize()
    gmin, gdel = np.zeros(2), np.full(2, ax[1])
    for w in (0, 2):
        nx, t0, steps = specs[w]
        pos = seeds[w]
        N = pos.shape[0] // 4
        idx = np.sort(rng.choice(N, 1000, replace=False))
        sub = _subset(pos, 4, N, idx)
        s0 = int(np.floor(t0 / dt))
        s1 = int(np.ceil((t0 + steps * h) / dt)) + 1
        host = turb.snapshots(n, np.arange(s0, s1) * dt)
        kw = dict(integrator="rk4", time_mode=O.BLEND, h=h, num_steps=steps, t0=t0,
                  snap_t0=s0 * dt, snap_dt=dt, periodic_space=True, map_period=steps * h)
        p_ref, f_ref = O.run_window(host, (n, n), gmin, gdel, sub, **kw)
        # the oracle's own snapshots (the device-built ones agree to ~1e-12, not bitwise)
        s64 = SnapshotSeries(grid, torch.from_numpy(host).cuda(), precision="fp64")
        p = torch.from_numpy(sub).cuda()
        f = run_window(s64, p, integrator="rk4", time_mode="blend", h=h, num_steps=steps, t0=t0,
                       snapshot_t0=s0 * dt, snapshot_dt=dt, map_period=steps * h)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(p.cpu().numpy(), p_ref)
        np.testing.assert_allclose(f.cpu().numpy(), f_ref, rtol=FTLE_RTOL_F64, atol=0)
        rel_l2, p99 = _errors(ftles[w].cpu().numpy()[idx], f_ref)
        assert rel_l2 <= FTLE_REL_L2, (w, rel_l2)
