"""Closed-form velocity fields on the GPU and AnalyticalSolver.

* freeze_time=True reproduces pyFTLE's analytical path (its interpolator keeps
  t = 0): positions and FTLE against the reference's golden vectors (the device
  kernel's sin/cos differ from numpy's by an ulp: rtol 1e-12 on positions, 1e-10
  on FTLE; the callable path evaluates the same numpy function: bit-exact);
* with advancing time the device kernel and the callable path agree;
* the closed-form field is the interpolation-free reference for the grid path:
  BLEND on a fine grid converges to it.
"""

import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from pyftle_b200 import NeighboringParticles, flows
from pyftle_b200.api import ABCFlow, AnalyticalSolver, DoubleGyre

pytestmark = pytest.mark.gpu

NOTEBOOK_GYRE = DoubleGyre(A=0.1, eps=0.25, omega=2.0)


@pytest.mark.parametrize("integrator", ["euler", "rk4"])
@pytest.mark.parametrize("dt", [0.01, -0.01])
def test_frozen_time_matches_reference(golden, integrator, dt):
    g = golden("analytical.npz")
    ref_f = g[f"{integrator}_{dt}_ftle"]
    ref_p = g[f"{integrator}_{dt}_pos"]
    # device kernel
    part = NeighboringParticles(positions=g["positions"])
    solver = AnalyticalSolver(NOTEBOOK_GYRE, part, dt, 0.1, 1, integrator, freeze_time=True)
    f = solver.run()
    np.testing.assert_allclose(f, ref_f, rtol=1e-10, atol=0)
    # callable path with the notebook's numpy velocity function: bit-exact positions
    # (the FTLE's log may differ from libm's by an ulp)
    from pyftle_b200.api import advect_callable

    fn = lambda t, x: flows.double_gyre_velocity(t, x, A=0.1, eps=0.25, omega=2.0)  # noqa
    p = NeighboringParticles(positions=g["positions"])
    advect_callable(fn, p, t0=0.0, h=dt, num_steps=11, integrator=integrator, freeze_time=True)
    np.testing.assert_array_equal(p.positions_host(), ref_p)
    solver = AnalyticalSolver(fn, part, dt, 0.1, 1, integrator, freeze_time=True)
    np.testing.assert_allclose(solver.run(), ref_f, rtol=1e-12, atol=0)


@pytest.mark.parametrize("flow,cents", [
    (DoubleGyre(), flows.centroid_grid_2d(20, 10, (0.1, 1.9), (0.1, 0.9))),
    (ABCFlow(), flows.centroid_grid_3d(6, 6, 6, (0.5, 0.5, 0.5), (5.5, 5.5, 5.5))),
])
@pytest.mark.parametrize("integrator", ["euler", "ab2", "rk4"])
def test_device_field_matches_callable_with_time(flow, cents, integrator):
    seeds = flows.seeds_2d(cents, 1e-3) if flow.dim == 2 else flows.seeds_3d(cents, 1e-3)
    part = NeighboringParticles(positions=seeds)
    a = AnalyticalSolver(flow, part, 0.02, 1.0, 3, integrator).run()
    b = AnalyticalSolver(lambda t, x: flow(t, x), part, 0.02, 1.0, 3, integrator).run()
    assert a.shape == (3, len(cents))
    np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-12)
    assert not np.allclose(a[0], a[2])  # time advances between the windows


def test_grid_blend_converges_to_closed_form():
    flow = DoubleGyre()
    cents = flows.centroid_grid_2d(30, 15, (0.2, 1.8), (0.2, 0.8))
    seeds = flows.seeds_2d(cents, 1e-3)
    T, h = 2.0, 0.01
    exact = AnalyticalSolver(flow, NeighboringParticles(positions=seeds), h, T, 1, "rk4").run()
    errs = []
    for nx in (129, 257, 513):
        shape = (nx, (nx + 1) // 2)
        pts = flows.grid_points_2d(*shape)
        snaps = flows.double_gyre_snapshots(pts, np.arange(0, 42) * 0.05)
        gmin, gdel = O.grid_axes(pts, shape)
        _, f = O.run_window(snaps, shape, gmin, gdel, seeds, integrator="rk4", time_mode=O.BLEND,
                            snap_dt=0.05, h=h, num_steps=int(round(T / h)) + 1,
                            map_period=T)
        errs.append(np.linalg.norm(f - exact) / np.linalg.norm(exact))
    assert errs[2] < errs[1] < errs[0]
    assert errs[2] < 2e-2
