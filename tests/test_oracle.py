"""Pins the CPU oracle to the reference (CPU only).

Golden vectors come from running pyFTLE itself (tests/golden/make_golden.py).
Tolerances: the interpolator and HOLD-window positions are bit-exact; the 2D
FTLE is bit-exact; the 3D FTLE (Jacobi vs LAPACK dgeev for lambda_max) agrees
to rtol 1e-12.
"""

import math

import numpy as np
import pytest

from oracle import oracle as O
from pyftle_b200 import flows


def test_ginterp_2d_bitexact(golden):
    g = golden("ginterp.npz")
    out = np.empty(len(g["p2"]))
    O.interp2d_vec_inplace(g["v2"], g["p2"], out)
    np.testing.assert_array_equal(out, g["o2"])


def test_ginterp_3d_bitexact(golden):
    g = golden("ginterp.npz")
    out = np.empty(len(g["p3"]))
    O.interp3d_vec_inplace(g["v3"], g["p3"], out)
    np.testing.assert_array_equal(out, g["o3"])


@pytest.mark.parametrize("direction", ["fwd", "bwd"])
@pytest.mark.parametrize("integrator", ["euler", "ab2", "rk4"])
def test_hold_window_2d_matches_reference(golden, direction, integrator):
    d = golden("windows_2d.npz")
    shape = tuple(d["shape"])
    gmin, gdel = O.grid_axes(d["points"], shape)
    dt = float(d["dt"])
    snaps = d["snaps"] if direction == "fwd" else d["snaps"][::-1]
    h = dt if direction == "fwd" else -dt
    pos, ftle = O.run_window(snaps, shape, gmin, gdel, d["positions"], integrator=integrator,
                             snap_dt=h)
    np.testing.assert_array_equal(pos, d[f"{direction}_{integrator}_pos"])
    np.testing.assert_array_equal(ftle, d[f"{direction}_{integrator}_ftle"])


@pytest.mark.parametrize("integrator", ["euler", "ab2", "rk4"])
def test_hold_window_3d_matches_reference(golden, integrator):
    d = golden("windows_3d.npz")
    shape = tuple(d["shape"])
    gmin, gdel = O.grid_axes(d["points"], shape)
    pos, ftle = O.run_window(d["snaps"], shape, gmin, gdel, d["positions"],
                             integrator=integrator, snap_dt=float(d["dt"]))
    np.testing.assert_array_equal(pos, d[f"fwd_{integrator}_pos"])
    np.testing.assert_allclose(ftle, d[f"fwd_{integrator}_ftle"], rtol=1e-12, atol=0)


def test_hold_window_3d_backward(golden):
    d = golden("windows_3d.npz")
    shape = tuple(d["shape"])
    gmin, gdel = O.grid_axes(d["points"], shape)
    pos, ftle = O.run_window(d["snaps"][::-1], shape, gmin, gdel, d["positions"],
                             integrator="rk4", snap_dt=-float(d["dt"]))
    np.testing.assert_array_equal(pos, d["bwd_rk4_pos"])
    np.testing.assert_allclose(ftle, d["bwd_rk4_ftle"], rtol=1e-12, atol=0)


def test_particles_leaving_grid(golden):
    d = golden("windows_2d.npz")
    shape = tuple(d["shape"])
    gmin, gdel = O.grid_axes(d["points"], shape)
    pos, ftle = O.run_window(d["snaps"], shape, gmin, gdel, d["edge_positions"],
                             integrator="rk4", snap_dt=float(d["dt"]))
    np.testing.assert_array_equal(pos, d["edge_rk4_pos"])
    np.testing.assert_array_equal(ftle, d["edge_rk4_ftle"])


def test_ftle_from_jacobians(golden):
    f = golden("ftle.npz")
    np.testing.assert_array_equal(O.ftle_from_jacobians(f["j2"], 1.0), f["f2"])
    np.testing.assert_array_equal(O.ftle_from_jacobians(f["j2"], 2.5), f["f2b"])
    np.testing.assert_allclose(O.ftle_from_jacobians(f["j3"], 2.0), f["f3"], rtol=1e-12,
                               atol=1e-15)
    # reference test_ftle.py: identity gives 0, stronger stretch gives larger FTLE
    assert np.all(O.ftle_from_jacobians(np.repeat(np.eye(2)[None], 3, 0), 1.0) == 0.0)
    assert O.ftle_from_jacobians(2 * np.eye(2)[None], 1.0)[0] > 0.0


def test_blend_constant_in_time_matches_hold():
    """With every snapshot equal, BLEND reduces to HOLD up to the blend's rounding."""
    shape = (40, 20)
    pts = flows.grid_points_2d(*shape)
    snap = flows.double_gyre_snapshots(pts, [0.3])[0]
    snaps = np.stack([snap] * 4)
    gmin, gdel = O.grid_axes(pts, shape)
    pos0 = flows.seeds_2d(flows.centroid_grid_2d(15, 8, (0.2, 1.8), (0.2, 0.8)), 1e-3)
    ph, fh = O.run_window(snaps, shape, gmin, gdel, pos0, integrator="rk4", time_mode=O.HOLD,
                          snap_dt=0.05, h=0.05, num_steps=4)
    pb, fb = O.run_window(snaps, shape, gmin, gdel, pos0, integrator="rk4", time_mode=O.BLEND,
                          snap_dt=0.1, h=0.05, num_steps=4, map_period=3 * 0.05)
    np.testing.assert_allclose(pb, ph, rtol=0, atol=1e-13)
    np.testing.assert_allclose(fb, fh, rtol=1e-8)


def test_periodic_matches_extended_grid():
    """A periodic grid equals the same field on a grid with node n = node 0 appended."""
    n = 16
    L = 2 * math.pi
    ax = flows.periodic_axis(n, L)
    ext = np.append(ax, L)
    times = [0.0, 0.5]
    sp = flows.abc_snapshots(ax, ax, ax, times)
    se = flows.abc_snapshots(ext, ext, ext, times)
    # abc is periodic, so node n of the extended grid equals node 0 up to sin(2pi) rounding;
    # copy node 0 exactly so the comparison is exact
    se = se.reshape(2, 3, n + 1, n + 1, n + 1)
    se[:, :, n, :, :] = se[:, :, 0, :, :]
    se[:, :, :, n, :] = se[:, :, :, 0, :]
    se[:, :, :, :, n] = se[:, :, :, :, 0]
    se = se.reshape(2, 3, -1)
    pos0 = flows.seeds_3d(flows.centroid_grid_3d(4, 4, 4, (1, 1, 1), (5, 5, 5)), 1e-3)
    sp_shape, se_shape = (n, n, n), (n + 1, n + 1, n + 1)
    gdel = np.full(3, L / n)
    gmin = np.zeros(3)
    pp, fp = O.run_window(sp, sp_shape, gmin, gdel, pos0, integrator="rk4", time_mode=O.BLEND,
                          snap_dt=0.5, h=0.01, num_steps=20, periodic_space=True)
    pe, fe = O.run_window(se, se_shape, gmin, gdel, pos0, integrator="rk4", time_mode=O.BLEND,
                          snap_dt=0.5, h=0.01, num_steps=20, periodic_space=False)
    np.testing.assert_array_equal(pp, pe)
    np.testing.assert_array_equal(fp, fe)


def test_blend_rk4_converges_to_analytic_flow():
    """BLEND RK4 on a fine double-gyre grid tracks the closed-form flow."""
    shape = (257, 129)
    pts = flows.grid_points_2d(*shape)
    times = np.arange(0, 21) * 0.05
    snaps = flows.double_gyre_snapshots(pts, times)
    gmin, gdel = O.grid_axes(pts, shape)
    pos0 = flows.seeds_2d(flows.centroid_grid_2d(6, 3, (0.3, 1.7), (0.3, 0.7)), 1e-3)
    pg, _ = O.run_window(snaps, shape, gmin, gdel, pos0, integrator="rk4", time_mode=O.BLEND,
                         snap_dt=0.05, h=0.01, num_steps=100)
    # closed-form reference trajectory with small RK4 steps
    x = pos0.copy()
    h = 0.002
    for i in range(500):
        t = i * h
        k1 = flows.double_gyre_velocity(t, x)
        k2 = flows.double_gyre_velocity(t + h / 2, x + h / 2 * k1)
        k3 = flows.double_gyre_velocity(t + h / 2, x + h / 2 * k2)
        k4 = flows.double_gyre_velocity(t + h, x + h * k3)
        x = x + h / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
    assert np.max(np.abs(pg - x)) < 2e-4
