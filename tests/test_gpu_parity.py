"""GPU parity: the CUDA engine against the reference's golden vectors and the oracle.

Tolerances (written per test):
  * gathers, HOLD positions, BLEND/periodic positions: bit-exact;
  * FTLE vs the reference: rtol 1e-10 (2D is in practice exact);
  * FTLE vs the oracle: rtol 1e-12 (same formulas; log may differ by an ulp).
"""

import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from pyftle_b200 import (
    BlendedSnapshotSource,
    EngineOptions,
    FTLESolver,
    MemoryBatchSource,
    NeighboringParticles,
    SnapshotSeries,
    create_integrator,
    create_interpolator,
    flows,
    run_window,
)
from pyftle_b200 import _lib
from pyftle_b200._device import ptr, stream_ptr
from pyftle_b200.ftle import (
    compute_cauchy_green_2x2,
    compute_cauchy_green_3x3,
    compute_ftle_2x2,
    compute_ftle_3x3,
    max_eigenvalue_2x2,
    max_eigenvalue_3x3,
)
from pyftle_b200.interpolate import GridSpec

pytestmark = pytest.mark.gpu

FTLE_RTOL_REF = 1e-10
FTLE_RTOL_ORACLE = 1e-12


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


# ---------------------------------------------------------------------------
# gathers (GridInterp.cpp replacement)
# ---------------------------------------------------------------------------

def test_interp2d_bitexact(golden):
    g = golden("ginterp.npz")
    v, p = dev(g["v2"]), dev(g["p2"])
    out = torch.empty(len(g["p2"]), dtype=torch.float64, device="cuda")
    _lib.call("ftle_interp2d_vec_inplace", ptr(v), v.shape[0], v.shape[1], ptr(p), p.shape[0],
              ptr(out), stream_ptr())
    np.testing.assert_array_equal(host(out), g["o2"])


def test_interp3d_bitexact(golden):
    g = golden("ginterp.npz")
    v, p = dev(g["v3"]), dev(g["p3"])
    out = torch.empty(len(g["p3"]), dtype=torch.float64, device="cuda")
    _lib.call("ftle_interp3d_vec_inplace", ptr(v), *v.shape, ptr(p), p.shape[0], ptr(out),
              stream_ptr())
    np.testing.assert_array_equal(host(out), g["o3"])


@pytest.mark.parametrize("d", [2, 3])
def test_grid_interpolator_bitexact(golden, d):
    g = golden("interpolator.npz")
    it = create_interpolator("grid", tuple(g[f"shape{d}"]))
    it.update(g[f"vel{d}"], g[f"pts{d}"])
    out = it.interpolate(g[f"q{d}"])
    np.testing.assert_array_equal(host(out), g[f"out{d}"])


def test_interpolator_update_without_points_reuses_grid(golden):
    g = golden("interpolator.npz")
    it = create_interpolator("grid", tuple(g["shape2"]))
    it.update(g["vel2"], g["pts2"])
    it.update(g["vel2"])  # the reference crashes on the next call here
    np.testing.assert_array_equal(host(it.interpolate(g["q2"])), g["out2"])


# ---------------------------------------------------------------------------
# per-step path (Integrator / Interpolator API, one launch per step)
# ---------------------------------------------------------------------------

def _stepsource(d, direction, positions=None):
    snaps = d["snaps"] if direction == "fwd" else d["snaps"][::-1]
    dt = float(d["dt"]) * (1 if direction == "fwd" else -1)
    pos = d["positions"] if positions is None else positions
    return snaps, dt, pos


@pytest.mark.parametrize("direction", ["fwd", "bwd"])
@pytest.mark.parametrize("integrator", ["euler", "ab2", "rk4"])
def test_per_step_solver_2d_matches_reference(golden, direction, integrator):
    d = golden("windows_2d.npz")
    shape = tuple(d["shape"])
    snaps, dt, pos = _stepsource(d, direction)
    src = MemoryBatchSource(list(snaps), d["points"], pos, dt, grid_shape=shape)
    integ = create_integrator(integrator, create_interpolator("grid", shape))
    solver = FTLESolver(src, integ)
    solver._fused_ok = lambda: False  # force the per-step path
    ftle = solver.run()
    np.testing.assert_array_equal(solver.particles.positions_host(),
                                  d[f"{direction}_{integrator}_pos"])
    np.testing.assert_allclose(ftle, d[f"{direction}_{integrator}_ftle"], rtol=FTLE_RTOL_REF,
                               atol=0)


@pytest.mark.parametrize("integrator", ["euler", "ab2", "rk4"])
def test_per_step_solver_3d_matches_reference(golden, integrator):
    d = golden("windows_3d.npz")
    shape = tuple(d["shape"])
    src = MemoryBatchSource(list(d["snaps"]), d["points"], d["positions"], float(d["dt"]),
                            grid_shape=shape)
    integ = create_integrator(integrator, create_interpolator("grid", shape))
    solver = FTLESolver(src, integ)
    solver._fused_ok = lambda: False
    ftle = solver.run()
    np.testing.assert_array_equal(solver.particles.positions_host(), d[f"fwd_{integrator}_pos"])
    np.testing.assert_allclose(ftle, d[f"fwd_{integrator}_ftle"], rtol=FTLE_RTOL_REF, atol=0)


class Mock:
    """pyFTLE's test double: v = 0.1 x (tests/conftest.py of the reference)."""

    def interpolate(self, x):
        return x * 0.1


@pytest.mark.parametrize("integrator", ["euler", "ab2", "rk4"])
@pytest.mark.parametrize("h", [0.1, -0.3])
def test_generic_interpolator_integrators_bitexact(golden, integrator, h):
    g = golden("integrate.npz")
    p = NeighboringParticles(positions=g["pos0"])
    integ = create_integrator(integrator, Mock())
    integ.integrate(h, p)
    np.testing.assert_array_equal(p.positions_host(), g[f"{integrator}_{h}_1"])
    integ.integrate(h, p)
    np.testing.assert_array_equal(p.positions_host(), g[f"{integrator}_{h}_2"])


# ---------------------------------------------------------------------------
# fused FP64 window
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("direction", ["fwd", "bwd"])
@pytest.mark.parametrize("integrator", ["euler", "ab2", "rk4"])
def test_fused_hold_2d_matches_reference(golden, direction, integrator):
    d = golden("windows_2d.npz")
    shape = tuple(d["shape"])
    snaps, dt, pos = _stepsource(d, direction)
    src = MemoryBatchSource(snaps, d["points"], pos, dt, grid_shape=shape)
    solver = FTLESolver(src, create_integrator(integrator, create_interpolator("grid", shape)))
    assert solver._fused_ok()
    ftle = solver.run()
    np.testing.assert_array_equal(solver.particles.positions_host(),
                                  d[f"{direction}_{integrator}_pos"])
    np.testing.assert_allclose(ftle, d[f"{direction}_{integrator}_ftle"], rtol=FTLE_RTOL_REF,
                               atol=0)


@pytest.mark.parametrize("integrator", ["euler", "ab2", "rk4"])
def test_fused_hold_3d_matches_reference(golden, integrator):
    d = golden("windows_3d.npz")
    shape = tuple(d["shape"])
    src = MemoryBatchSource(d["snaps"], d["points"], d["positions"], float(d["dt"]),
                            grid_shape=shape)
    solver = FTLESolver(src, create_integrator(integrator, create_interpolator("grid", shape)))
    ftle = solver.run()
    np.testing.assert_array_equal(solver.particles.positions_host(), d[f"fwd_{integrator}_pos"])
    np.testing.assert_allclose(ftle, d[f"fwd_{integrator}_ftle"], rtol=FTLE_RTOL_REF, atol=0)


def test_fused_hold_3d_backward_and_edges(golden):
    d = golden("windows_3d.npz")
    shape = tuple(d["shape"])
    src = MemoryBatchSource(d["snaps"][::-1], d["points"], d["positions"], -float(d["dt"]),
                            grid_shape=shape)
    solver = FTLESolver(src, create_integrator("rk4", create_interpolator("grid", shape)))
    ftle = solver.run()
    np.testing.assert_array_equal(solver.particles.positions_host(), d["bwd_rk4_pos"])
    np.testing.assert_allclose(ftle, d["bwd_rk4_ftle"], rtol=FTLE_RTOL_REF, atol=0)
    e = golden("windows_2d.npz")
    src = MemoryBatchSource(e["snaps"], e["points"], e["edge_positions"], float(e["dt"]),
                            grid_shape=tuple(e["shape"]))
    solver = FTLESolver(src, create_integrator("rk4", create_interpolator("grid",
                                                                          tuple(e["shape"]))))
    ftle = solver.run()
    np.testing.assert_array_equal(solver.particles.positions_host(), e["edge_rk4_pos"])
    np.testing.assert_allclose(ftle, e["edge_rk4_ftle"], rtol=FTLE_RTOL_REF, atol=0)


def _blend_case_2d(n_groups_x=37, n_groups_y=19):
    shape = (96, 48)
    pts = flows.grid_points_2d(*shape)
    times = np.arange(12) * 0.05
    snaps = flows.double_gyre_snapshots(pts, times)
    pos = flows.seeds_2d(flows.centroid_grid_2d(n_groups_x, n_groups_y, (0.05, 1.95),
                                                (0.05, 0.95)), 1e-3)
    return shape, pts, snaps, pos


@pytest.mark.parametrize("integrator", ["euler", "ab2", "rk4"])
@pytest.mark.parametrize("h", [0.013, -0.013])
def test_fused_blend_2d_matches_oracle(integrator, h):
    shape, pts, snaps, pos = _blend_case_2d()
    t0 = 0.02 if h > 0 else 0.53
    src = BlendedSnapshotSource(snaps, pts, pos, shape, h=h, num_steps=40, snapshot_dt=0.05,
                                t0=t0)
    solver = FTLESolver(src, create_integrator(integrator, create_interpolator("grid", shape)))
    ftle = solver.run()
    gmin, gdel = O.grid_axes(pts, shape)
    p_ref, f_ref = O.run_window(snaps, shape, gmin, gdel, pos, integrator=integrator,
                                time_mode=O.BLEND, snap_dt=0.05, h=h, num_steps=40, t0=t0)
    np.testing.assert_array_equal(solver.particles.positions_host(), p_ref)
    np.testing.assert_allclose(ftle, f_ref, rtol=FTLE_RTOL_ORACLE, atol=0)


@pytest.mark.parametrize("integrator", ["euler", "ab2", "rk4"])
def test_fused_blend_3d_periodic_matches_oracle(integrator):
    n = 24
    ax = flows.periodic_axis(n)
    S = 8
    times = np.arange(S) * (2 * math.pi / S)
    snaps = flows.abc_snapshots(ax, ax, ax, times)
    pts = flows.grid_points_3d(ax, ax, ax)
    cents = np.random.default_rng(3).uniform(0, 2 * math.pi, (300, 3))
    pos = flows.seeds_3d(cents, 1e-3)
    src = BlendedSnapshotSource(snaps, pts, pos, (n, n, n), h=0.05, num_steps=60,
                                snapshot_dt=2 * math.pi / S, t0=5.9, periodic_space=True,
                                periodic_time=True)
    solver = FTLESolver(src, create_integrator(integrator,
                                               create_interpolator("grid", (n, n, n))))
    ftle = solver.run()
    gmin, gdel = O.grid_axes(pts, (n, n, n))
    p_ref, f_ref = O.run_window(snaps, (n, n, n), gmin, gdel, pos, integrator=integrator,
                                time_mode=O.BLEND, snap_dt=2 * math.pi / S, h=0.05,
                                num_steps=60, t0=5.9, periodic_space=True, periodic_time=True)
    np.testing.assert_array_equal(solver.particles.positions_host(), p_ref)
    np.testing.assert_allclose(ftle, f_ref, rtol=FTLE_RTOL_ORACLE, atol=0)


def test_fused_empty_and_ragged():
    """Zero groups is a no-op; group counts that do not fill a block are handled."""
    shape, pts, snaps, _ = _blend_case_2d()
    grid = GridSpec.from_points(pts, shape)
    series = SnapshotSeries(grid, snaps)
    empty = torch.empty((0, 2), dtype=torch.float64, device="cuda")
    f = run_window(series, empty, h=0.05, num_steps=3, time_mode="hold")
    assert f.numel() == 0
    for ng in (1, 63, 65, 129):
        cents = np.random.default_rng(ng).uniform([0.1, 0.1], [1.9, 0.9], (ng, 2))
        pos = flows.seeds_2d(cents, 1e-3)
        pt = torch.as_tensor(pos, device="cuda")
        f = run_window(series, pt, h=0.05, num_steps=5, time_mode="hold")
        gmin, gdel = O.grid_axes(pts, shape)
        p_ref, f_ref = O.run_window(snaps, shape, gmin, gdel, pos, integrator="rk4",
                                    snap_dt=0.05, num_steps=5)
        np.testing.assert_array_equal(host(pt), p_ref)
        np.testing.assert_allclose(host(f), f_ref, rtol=FTLE_RTOL_ORACLE, atol=0)


def test_window_rejects_bad_arguments():
    shape, pts, snaps, pos = _blend_case_2d(4, 4)
    series = SnapshotSeries(GridSpec.from_points(pts, shape), snaps)
    pt = torch.as_tensor(pos, device="cuda")
    with pytest.raises(_lib.FTLEError, match="first_snapshot \\+ num_steps"):
        run_window(series, pt, h=0.05, num_steps=len(snaps) + 1, time_mode="hold")
    with pytest.raises(ValueError):
        run_window(series, pt[:5], h=0.05, num_steps=2)


# ---------------------------------------------------------------------------
# FTLE building blocks (ftle.py / cauchy_green.py)
# ---------------------------------------------------------------------------

def test_ftle_building_blocks(golden):
    f = golden("ftle.npz")
    np.testing.assert_allclose(host(compute_cauchy_green_2x2(f["j2"])), f["cg2"], rtol=1e-12)
    np.testing.assert_allclose(host(compute_cauchy_green_3x3(f["j3"])), f["cg3"], rtol=1e-12)
    np.testing.assert_allclose(host(max_eigenvalue_2x2(f["cg2"])), f["lam2"], rtol=1e-12)
    np.testing.assert_allclose(host(max_eigenvalue_3x3(f["cg3"])), f["lam3"], rtol=1e-10)
    np.testing.assert_allclose(host(compute_ftle_2x2(f["j2"], 1.0)), f["f2"], rtol=1e-12,
                               atol=1e-15)
    np.testing.assert_allclose(host(compute_ftle_2x2(f["j2"], 2.5)), f["f2b"], rtol=1e-12,
                               atol=1e-15)
    np.testing.assert_allclose(host(compute_ftle_3x3(f["j3"], 2.0)), f["f3"], rtol=1e-10,
                               atol=1e-15)
    ident = np.repeat(np.eye(2)[None], 3, 0)
    np.testing.assert_allclose(host(compute_ftle_2x2(ident, 1.0)), np.zeros(3), atol=1e-12)
    assert host(compute_ftle_2x2(2 * np.eye(2)[None], 1.0))[0] > 0.0


@pytest.mark.parametrize("dim", [2, 3])
def test_neighboring_particles_on_device(dim):
    if dim == 2:
        pos = np.array([[0.0, 0.0], [1.0, 0.0], [0.5, 1.0], [0.5, 0.0]])
    else:
        pos = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.5, 1.0, 0.0], [0.5, -1.0, 0.0],
                        [0.5, 0.0, 1.0], [0.5, 0.0, -1.0]])
    p = NeighboringParticles(positions=pos)
    assert len(p) == 1
    np.testing.assert_array_equal(host(p.initial_delta_right_left), (pos[1] - pos[0])[None])
    np.testing.assert_array_equal(host(p.initial_delta_top_bottom), (pos[2] - pos[3])[None])
    if dim == 3:
        np.testing.assert_array_equal(host(p.initial_delta_front_back), (pos[4] - pos[5])[None])
    np.testing.assert_array_equal(host(p.initial_centroid), np.mean(pos, axis=0)[None])
    p.positions += 0.2
    np.testing.assert_array_equal(host(p.initial_delta_right_left), (pos[1] - pos[0])[None])


# ---------------------------------------------------------------------------
# mixed precision: FTLE error against the FP64 oracle
# ---------------------------------------------------------------------------

def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("precision,tol", [("fx15", 1e-3), ("fx16", 6e-4), ("fp16", 2e-3),
                                           ("bf16", 1.5e-2)])
def test_mixed_2d_double_gyre_error(precision, tol):
    shape = (256, 128)
    pts = flows.grid_points_2d(*shape)
    times = np.arange(41) * 0.05
    snaps = flows.double_gyre_snapshots(pts, times)
    pos = flows.seeds_2d(flows.centroid_grid_2d(100, 50, (0.02, 1.98), (0.02, 0.98)), 1e-3)
    src = BlendedSnapshotSource(snaps, pts, pos, shape, h=0.01, num_steps=200, snapshot_dt=0.05)
    solver = FTLESolver(src, create_integrator("rk4", create_interpolator("grid", shape)),
                        options=EngineOptions(precision=precision))
    ftle = solver.run()
    gmin, gdel = O.grid_axes(pts, shape)
    _, f_ref = O.run_window(snaps, shape, gmin, gdel, pos, integrator="rk4", time_mode=O.BLEND,
                            snap_dt=0.05, h=0.01, num_steps=200)
    err = rel_l2(ftle, f_ref)
    print(f"{precision} 2D FTLE rel L2 error vs FP64 oracle: {err:.3e}")
    assert err < tol


@pytest.mark.parametrize("integrator", ["euler", "ab2", "rk4"])
@pytest.mark.parametrize("precision,tol", [("fx15", 1e-3), ("fx16", 6e-4), ("fp16", 2e-3)])
def test_mixed_3d_abc_error(integrator, precision, tol):
    n = 48
    ax = flows.periodic_axis(n)
    S = 16
    times = np.arange(S) * (2 * math.pi / S)
    snaps = flows.abc_snapshots(ax, ax, ax, times)
    pts = flows.grid_points_3d(ax, ax, ax)
    cents = flows.centroid_grid_3d(12, 12, 12, (0.1, 0.1, 0.1), (6.1, 6.1, 6.1))
    pos = flows.seeds_3d(cents, 1e-3)
    kw = dict(h=0.02, num_steps=200, snapshot_dt=2 * math.pi / S, periodic_space=True,
              periodic_time=True)
    src = BlendedSnapshotSource(snaps, pts, pos, (n, n, n), **kw)
    solver = FTLESolver(src, create_integrator(integrator,
                                               create_interpolator("grid", (n, n, n))),
                        options=EngineOptions(precision=precision))
    ftle = solver.run()
    gmin, gdel = O.grid_axes(pts, (n, n, n))
    _, f_ref = O.run_window(snaps, (n, n, n), gmin, gdel, pos, integrator=integrator,
                            time_mode=O.BLEND, snap_dt=kw["snapshot_dt"], h=0.02, num_steps=200,
                            periodic_space=True, periodic_time=True)
    err = rel_l2(ftle, f_ref)
    print(f"{precision} 3D {integrator} FTLE rel L2 error vs FP64 oracle: {err:.3e}")
    assert err < tol


@pytest.mark.parametrize("integrator", ["euler", "ab2", "rk4"])
@pytest.mark.parametrize("chunk,sort_every", [(7, 1), (25, 2), (1000, 1)])
def test_mixed_chunked_sorted_equals_single_launch(integrator, chunk, sort_every):
    """Chunking and cell-sorting the groups leave every group's arithmetic unchanged."""
    n = 32
    ax = flows.periodic_axis(n)
    S = 8
    snaps = flows.abc_snapshots(ax, ax, ax, np.arange(S) * (2 * math.pi / S))
    pts = flows.grid_points_3d(ax, ax, ax)
    grid = GridSpec.from_points(pts, (n, n, n), periodic=True)
    series = SnapshotSeries(grid, snaps, precision="fx15", periodic_time=True)
    cents = np.random.default_rng(11).uniform(0, 2 * math.pi, (1000, 3))
    pos = flows.seeds_3d(cents, 1e-3)
    kw = dict(integrator=integrator, time_mode="blend", h=0.02, num_steps=60,
              snapshot_dt=2 * math.pi / S)
    p1 = torch.as_tensor(pos, device="cuda")
    f1 = run_window(series, p1, **kw)
    p2 = torch.as_tensor(pos, device="cuda")
    f2 = run_window(series, p2, chunk_steps=chunk, sort_every=sort_every, **kw)
    np.testing.assert_array_equal(host(p2), host(p1))
    np.testing.assert_array_equal(host(f2), host(f1))


def test_mixed_chunked_2d_nonperiodic_equals_single_launch():
    shape, pts, snaps, pos = _blend_case_2d(50, 25)
    series = SnapshotSeries(GridSpec.from_points(pts, shape), snaps, precision="fx15")
    kw = dict(integrator="rk4", time_mode="blend", h=0.013, num_steps=40, snapshot_dt=0.05)
    p1 = torch.as_tensor(pos, device="cuda")
    f1 = run_window(series, p1, **kw)
    p2 = torch.as_tensor(pos, device="cuda")
    f2 = run_window(series, p2, chunk_steps=9, sort_every=1, **kw)
    np.testing.assert_array_equal(host(p2), host(p1))
    np.testing.assert_array_equal(host(f2), host(f1))


@pytest.mark.parametrize("precision", ["fp64", "fx15"])
def test_keep_positions_leaves_seeds_and_same_ftle(precision):
    shape, pts, snaps, pos = _blend_case_2d(30, 15)
    series = SnapshotSeries(GridSpec.from_points(pts, shape), snaps, precision=precision)
    kw = dict(integrator="rk4", time_mode="blend", h=0.013, num_steps=40, snapshot_dt=0.05)
    p1 = torch.as_tensor(pos, device="cuda")
    f1 = run_window(series, p1, **kw)
    p2 = torch.as_tensor(pos, device="cuda")
    f2 = run_window(series, p2, keep_positions=True, **kw)
    np.testing.assert_array_equal(host(p2), pos)
    np.testing.assert_array_equal(host(f2), host(f1))


@pytest.mark.parametrize("chunk", [None, 10])
@pytest.mark.parametrize("dim", [2, 3])
def test_mixed_non_finite_group_leaves_other_groups_unchanged(dim, chunk):
    """A group whose seeds are NaN shares its warp's off-cell gather queue with valid
    groups; every other group must come out exactly as without it."""
    if dim == 2:
        shape, pts, snaps, pos = _blend_case_2d(16, 8)
        series = SnapshotSeries(GridSpec.from_points(pts, shape), snaps, precision="fx15")
        kw = dict(integrator="rk4", time_mode="blend", h=0.013, num_steps=40, snapshot_dt=0.05)
    else:
        n, S = 24, 8
        ax = flows.periodic_axis(n)
        snaps = flows.abc_snapshots(ax, ax, ax, np.arange(S) * (2 * math.pi / S))
        grid = GridSpec.from_points(flows.grid_points_3d(ax, ax, ax), (n, n, n), periodic=True)
        series = SnapshotSeries(grid, snaps, precision="fx15", periodic_time=True)
        pos = flows.seeds_3d(np.random.default_rng(4).uniform(0, 2 * math.pi, (128, 3)), 1e-3)
        kw = dict(integrator="rk4", time_mode="blend", h=0.02, num_steps=60,
                  snapshot_dt=2 * math.pi / S)
    if chunk:
        kw.update(chunk_steps=chunk, sort_every=1)
    K = 2 * dim
    N = pos.shape[0] // K
    bad = 5
    rows = np.arange(K) * N + bad
    p1 = torch.as_tensor(pos, device="cuda")
    f1 = host(run_window(series, p1, **kw))
    pos2 = pos.copy()
    pos2[rows] = np.nan
    p2 = torch.as_tensor(pos2, device="cuda")
    f2 = host(run_window(series, p2, **kw))
    keep = np.setdiff1d(np.arange(K * N), rows)
    np.testing.assert_array_equal(host(p2)[keep], host(p1)[keep])
    np.testing.assert_array_equal(np.delete(f2, bad), np.delete(f1, bad))


def test_fx15_range_is_exact_and_repeatable_with_negative_zeros():
    """The FX15 value range (per-component min / max over the series) must not depend
    on the order of the device's atomic updates; exact -0.0 values (a velocity field
    vanishing on a boundary) once let a min of -0.0 override a negative minimum."""
    rng = np.random.default_rng(3)
    nx, ny, S = 250, 200, 6
    snaps = rng.uniform(-1.0, 1.0, (S, 2, nx * ny))
    snaps[:, :, ::7] = -0.0
    grid = GridSpec(shape=(nx, ny), origin=(0.0, 0.0), spacing=(1.0, 1.0))
    headers = []
    for _ in range(5):
        series = SnapshotSeries(grid, snaps, precision="fx15")
        headers.append(np.frombuffer(series.packed[:64].cpu().numpy().tobytes(), np.float32))
    for h in headers[1:]:
        np.testing.assert_array_equal(h, headers[0])
    vmin, vmax = headers[0][8:10], headers[0][12:14]
    for c in range(2):
        lo, hi = snaps[:, c].min(), snaps[:, c].max()
        assert vmin[c] <= lo and np.nextafter(vmin[c], np.float32(np.inf)) > lo
        assert vmax[c] >= hi and np.nextafter(vmax[c], np.float32(-np.inf)) < hi


@pytest.mark.parametrize("dim", [2, 3])
def test_fx16_codes_decode_to_the_nearest_level(dim):
    """FX16 packs each value as the 16-bit code whose decoded level (the kernels' FX15
    byte-permute decode: 0.5 + q/65536 up to q = 32768, 1 + (q - 32768)/32768 above, then
    scale * f + offset) is nearest, over the whole series' range."""
    rng = np.random.default_rng(11)
    shape = (40, 30) if dim == 2 else (12, 10, 8)
    nodes = int(np.prod(shape))
    S = 4
    snaps = rng.uniform(-2.5, 3.5, (S, dim, nodes))
    snaps[0, :, 0] = -2.5
    snaps[1, :, 1] = 3.5
    grid = GridSpec(shape=shape, origin=(0.0,) * dim, spacing=(1.0,) * dim)
    series = SnapshotSeries(grid, snaps, precision="fx16")
    raw = series.packed.cpu().numpy()
    hdr = np.frombuffer(raw[:64].tobytes(), np.float32)
    scale, offset = hdr[0:4].astype(np.float64), hdr[4:8].astype(np.float64)
    rec = 8 if dim == 2 else 16
    recs = np.frombuffer(raw[256:256 + rec * nodes * S].tobytes(), np.uint16)
    recs = recs.reshape(S, nodes, rec // 2)
    cols = [0, 1] if dim == 2 else [0, 1, 2]  # first half of each pair record: snapshot s
    q = recs[:, :, cols].astype(np.float64)
    f = np.where(q <= 32768, 0.5 + q / 65536.0, 1.0 + (q - 32768) / 32768.0)
    for c in range(dim):
        u = scale[c] * f[:, :, c] + offset[c]
        v = snaps[:, c, :]
        step = scale[c] * np.where(q[:, :, c] < 32768, 1.0 / 65536.0, 1.0 / 32768.0)
        assert np.all(np.abs(u - v) <= 0.5 * step * (1 + 1e-6) + 1e-6 * np.abs(v)), c
        assert (scale[c] * (2.0 - 2.0 ** -15) + offset[c]) >= v.max() - 1e-6


# ---------------------------------------------------------------------------
# FP64 judge of a mixed-precision window (FTLESolver, EngineOptions.judge_tol)
# ---------------------------------------------------------------------------

def _abc_judge_case():
    n = 32
    ax = flows.periodic_axis(n)
    S = 16
    dt = 2 * math.pi / S
    snaps = flows.abc_snapshots(ax, ax, ax, np.arange(S) * dt)
    pts = flows.grid_points_3d(ax, ax, ax)
    cents = np.random.default_rng(21).uniform(0, 2 * math.pi, (1500, 3))
    pos = flows.seeds_3d(cents, 1e-3)
    kw = dict(h=0.02, num_steps=150, snapshot_dt=dt, periodic_space=True, periodic_time=True)
    return snaps, pts, pos, (n, n, n), kw


def _solve(snaps, pts, pos, shape, kw, **opts):
    src = BlendedSnapshotSource(snaps, pts, pos, shape, **kw)
    solver = FTLESolver(src, create_integrator("rk4", create_interpolator("grid", shape)),
                        options=EngineOptions(**opts))
    f = solver.run()
    return f, solver.particles.positions.cpu().numpy(), solver


def test_judge_readvects_a_window_above_tolerance():
    """BF16 storage misses a tight tolerance: the window comes back as the plain FP64
    path's bits (FTLE and final positions), and the judge reports the sampled error."""
    snaps, pts, pos, shape, kw = _abc_judge_case()
    f64, p64, _ = _solve(snaps, pts, pos, shape, kw)
    fbf, _, _ = _solve(snaps, pts, pos, shape, kw, precision="bf16")
    f, p, solver = _solve(snaps, pts, pos, shape, kw, precision="bf16", judge_tol=1e-6,
                          judge_stride=10)
    sel = np.arange(0, f64.size, 10)
    assert solver.judge["readvected"] and solver.judge["sample_groups"] == sel.size
    assert solver.judge["error"] == pytest.approx(rel_l2(fbf[sel], f64[sel]), rel=1e-12)
    np.testing.assert_array_equal(f, f64)
    np.testing.assert_array_equal(p, p64)


def test_judge_keeps_a_window_within_tolerance():
    snaps, pts, pos, shape, kw = _abc_judge_case()
    fx, px, _ = _solve(snaps, pts, pos, shape, kw, precision="fx16", chunk_steps=40)
    f, p, solver = _solve(snaps, pts, pos, shape, kw, precision="fx16", chunk_steps=40,
                          judge_tol=1e-3)
    assert not solver.judge["readvected"] and 0 < solver.judge["error"] <= 1e-3
    np.testing.assert_array_equal(f, fx)
    np.testing.assert_array_equal(p, px)
