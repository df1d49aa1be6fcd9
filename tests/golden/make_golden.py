"""Generate the golden vectors in tests/golden/ by running pyFTLE itself.

Run where the pyFTLE source tree is available (``$PYFTLE_REFERENCE_ROOT``, else a
checkout named ``reference`` beside this repository):

    python tests/golden/make_golden.py

Recipe: the reference's ``src/pyftle`` package is staged into a temporary
directory (never into this repository), its native ``ginterp`` module is the
one ``oracle/build.py`` compiled from the reference's own GridInterp.cpp, and
tiny import stubs stand in for packages that are absent here but are not on
the hot path (nptyping type aliases, matplotlib's exception class, pyvista,
colorama, configargparse).  Every vector below is produced by the reference's
public functions; inputs are seeded.

Outputs (all float64, small):
  ginterp.npz      ginterp.interp2d_vec_inplace / interp3d_vec_inplace values
                   on random, edge, integer, out-of-grid and non-finite points
  interpolator.npz HighPerfInterpolator("grid").update(...).interpolate(...)
  ftle.npz         compute_cauchy_green_*, max_eigenvalue_*, compute_ftle_*
                   on the reference's own Jacobian fixtures and random ones
  integrate.npz    one/two steps of Euler/AB2/RK4 with the v = 0.1 x mock
  windows_2d.npz   FTLESolver.run over double-gyre windows (Euler/AB2/RK4,
                   forward and backward time): final positions and FTLE
  windows_3d.npz   FTLESolver.run over ABC windows on a cubic grid
  analytical.npz   FTLESolver.run with AnalyticalBatchSource / AnalyticalInterpolator
                   (pyFTLE's notebook double gyre; the reference evaluates it at t = 0)
"""

from __future__ import annotations

import math
import os
import shutil
import sys
import tempfile
import textwrap

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
# the pyFTLE source tree: $PYFTLE_REFERENCE_ROOT, else a checkout named `reference`
# beside this repository
REF_ROOT = os.environ.get("PYFTLE_REFERENCE_ROOT") or os.path.join(os.path.dirname(REPO),
                                                                   "reference")

STUBS = {
    "nptyping/__init__.py": """
        import numpy as _np
        class _Sub:
            def __class_getitem__(cls, item):
                return _np.ndarray
        class NDArray(_Sub): pass
        class Shape(_Sub): pass
        Float64 = _np.float64
    """,
    "matplotlib/__init__.py": """
        class ExecutableNotFoundError(FileNotFoundError):
            pass
    """,
    "pyvista/__init__.py": """
        class StructuredGrid:
            def __init__(self, *a, **k): pass
        class PolyData:
            def __init__(self, *a, **k): pass
    """,
    "colorama/__init__.py": """
        class _C:
            def __getattr__(self, name): return ""
        Fore = _C(); Style = _C()
        def init(*a, **k): pass
    """,
    "configargparse/__init__.py": """
        from argparse import *  # noqa
    """,
}


def stage_reference() -> str:
    sys.path.insert(0, REPO)
    from oracle.build import REF_MOD, build_reference

    build_reference()
    tmp = tempfile.mkdtemp(prefix="pyftle_ref_stage_")
    shutil.copytree(os.path.join(REF_ROOT, "src", "pyftle"), os.path.join(tmp, "pyftle"))
    shutil.copy(REF_MOD, os.path.join(tmp, "pyftle", os.path.basename(REF_MOD)))
    for rel, body in STUBS.items():
        path = os.path.join(tmp, "stubs", rel)
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            f.write(textwrap.dedent(body))
    sys.path.insert(0, os.path.join(tmp, "stubs"))
    sys.path.insert(0, tmp)
    return tmp


class MemSource:
    """In-memory BatchSource (data_source.py:29-83); passes the grid points on
    every update so HighPerfInterpolator re-initialises (interpolate.py:467-473
    mishandles ``points=None``)."""

    def __init__(self, snapshots, points, positions, timestep, ident="mem"):
        self.snapshots = snapshots
        self.points = points
        self.positions = positions
        self._dt = timestep
        self._id = ident

    @property
    def timestep(self):
        return self._dt

    @property
    def num_steps(self):
        return len(self.snapshots)

    @property
    def id(self):
        return self._id

    def get_particles(self):
        from pyftle.particles import NeighboringParticles

        return NeighboringParticles(positions=self.positions.copy())

    def update_interpolator(self, interpolator, step_index):
        interpolator.update(self.snapshots[step_index], self.points)


def gen_ginterp(rng):
    from pyftle import ginterp

    v2 = rng.standard_normal((13, 9))
    p2 = np.concatenate([
        rng.uniform(-1.5, 14.0, (400, 2)),
        rng.uniform(0.0, 12.0, (200, 2)) * np.array([1.0, 8.0 / 12.0]),
        np.floor(rng.uniform(0.0, 13.0, (50, 2))),
        np.array([[12.0, 3.5], [np.nextafter(12.0, 0.0), 3.5], [0.0, 0.0], [-0.0, 2.0],
                  [-1e-300, 2.0], [3.0, 8.0], [3.0, np.nextafter(8.0, 0.0)], [np.nan, 1.0],
                  [np.inf, 1.0], [-np.inf, 1.0], [1e300, 1.0], [5.5, -1e300]]),
    ])
    o2 = np.empty(len(p2))
    ginterp.interp2d_vec_inplace(v2, p2, o2)
    v3 = rng.standard_normal((7, 6, 9))
    p3 = np.concatenate([
        rng.uniform(-1.0, 9.5, (500, 3)),
        rng.uniform(0.0, 1.0, (200, 3)) * np.array([6.0, 5.0, 8.0]),
        np.array([[6.0, 1.0, 1.0], [np.nextafter(6.0, 0), 1.0, 1.0], [1.0, 5.0, 1.0],
                  [1.0, 1.0, 8.0], [1.0, 1.0, np.nextafter(8.0, 0)], [np.nan, 1, 1],
                  [0.0, 0.0, 0.0], [-0.0, -0.0, -0.0]]),
    ])
    o3 = np.empty(len(p3))
    ginterp.interp3d_vec_inplace(v3, p3, o3)
    np.savez(os.path.join(HERE, "ginterp.npz"), v2=v2, p2=p2, o2=o2, v3=v3, p3=p3, o3=o3)


def gen_interpolator(rng):
    from pyftle.interpolate import create_interpolator
    from pyftle_b200 import flows

    shape2 = (17, 11)
    pts2 = flows.grid_points_2d(*shape2, (0.0, 2.0), (0.0, 1.0))
    vel2 = rng.standard_normal((2, pts2.shape[1]))
    q2 = np.concatenate([rng.uniform(-0.2, 2.2, (300, 1)), rng.uniform(-0.1, 1.1, (300, 1))], 1)
    it = create_interpolator("grid", shape2)
    it.update(vel2, pts2)
    out2 = it.interpolate(q2).copy()
    shape3 = (9, 9, 7)
    x = np.linspace(0.0, 1.0, 9)
    z = np.linspace(-0.5, 0.5, 7)
    pts3 = flows.grid_points_3d(x, x, z)
    vel3 = rng.standard_normal((3, pts3.shape[1]))
    q3 = np.column_stack([rng.uniform(-0.1, 1.1, 300), rng.uniform(-0.1, 1.1, 300),
                          rng.uniform(-0.6, 0.6, 300)])
    it3 = create_interpolator("grid", shape3)
    it3.update(vel3, pts3)
    out3 = it3.interpolate(q3).copy()
    np.savez(os.path.join(HERE, "interpolator.npz"), shape2=np.array(shape2), pts2=pts2,
             vel2=vel2, q2=q2, out2=out2, shape3=np.array(shape3), pts3=pts3, vel3=vel3, q3=q3,
             out3=out3)


def gen_ftle(rng):
    from pyftle import ftle as F

    j2_fix = np.array([[[2.0, 0.0], [0.0, 1.0]], [[1.5, 0.5], [0.5, 1.5]]])
    j3_fix = np.array([np.eye(3), [[1.0, 0.2, 0.0], [0.0, 1.5, 0.1], [0.0, 0.0, 1.2]]])
    j2 = np.concatenate([j2_fix, np.repeat(np.eye(2)[None], 3, 0),
                         np.exp(rng.uniform(-3, 3, (64, 1, 1))) * rng.standard_normal((64, 2, 2))])
    j3 = np.concatenate([j3_fix, np.exp(rng.uniform(-3, 3, (64, 1, 1)))
                         * rng.standard_normal((64, 3, 3))])
    cg2 = F.compute_cauchy_green_2x2(j2)
    cg3 = F.compute_cauchy_green_3x3(j3)
    lam2 = F.max_eigenvalue_2x2(cg2)
    lam3 = F.max_eigenvalue_3x3(cg3)
    assert np.isrealobj(lam3)
    f2 = F.compute_ftle_2x2(j2, 1.0)
    f2b = F.compute_ftle_2x2(j2, 2.5)
    f3 = F.compute_ftle_3x3(j3, 2.0)
    np.savez(os.path.join(HERE, "ftle.npz"), j2=j2, j3=j3, cg2=cg2, cg3=cg3, lam2=lam2,
             lam3=lam3, f2=f2, f2b=f2b, f3=f3)


def gen_integrate():
    from pyftle.integrate import create_integrator
    from pyftle.particles import NeighboringParticles

    class Mock:
        def interpolate(self, x):
            return x * 0.1

    pos0 = np.arange(1.0, 17.0).reshape(8, 2)
    res = {"pos0": pos0}
    for name in ("euler", "ab2", "rk4"):
        for h in (0.1, -0.3):
            p = NeighboringParticles(positions=pos0.copy())
            integ = create_integrator(name, Mock())
            integ.integrate(h, p)
            res[f"{name}_{h}_1"] = p.positions.copy()
            integ.integrate(h, p)
            res[f"{name}_{h}_2"] = p.positions.copy()
    np.savez(os.path.join(HERE, "integrate.npz"), **res)


def run_solver(snaps, points, positions, dt, integrator, shape):
    from pyftle.ftle_solver import FTLESolver
    from pyftle.integrate import create_integrator
    from pyftle.interpolate import create_interpolator

    src = MemSource(snaps, points, positions, dt)
    integ = create_integrator(integrator, create_interpolator("grid", shape))
    solver = FTLESolver(src, integ)
    ftle = solver.run()
    return solver.particles.positions.copy(), np.asarray(ftle).copy()


def gen_windows_2d():
    from pyftle_b200 import flows

    shape = (48, 24)
    pts = flows.grid_points_2d(*shape, (0.0, 2.0), (0.0, 1.0))
    dt = 0.05
    times = np.arange(11) * dt
    snaps = flows.double_gyre_snapshots(pts, times, omega=2.0 * math.pi / 10.0)
    cents = flows.centroid_grid_2d(20, 10, (0.1, 1.9), (0.1, 0.9))
    pos = flows.seeds_2d(cents, 1e-2)
    res = {"shape": np.array(shape), "points": pts, "snaps": snaps, "positions": pos,
           "dt": np.array(dt)}
    for name in ("euler", "ab2", "rk4"):
        p, f = run_solver(list(snaps), pts, pos, dt, name, shape)
        res[f"fwd_{name}_pos"], res[f"fwd_{name}_ftle"] = p, f
        p, f = run_solver(list(snaps[::-1]), pts, pos, -dt, name, shape)
        res[f"bwd_{name}_pos"], res[f"bwd_{name}_ftle"] = p, f
    # particles leaving the grid (velocity 0 outside, GridInterp.cpp:126)
    edge = flows.seeds_2d(np.array([[0.004, 0.5], [1.996, 0.5], [1.0, 0.004], [1.0, 0.999]]),
                          1e-2)
    p, f = run_solver(list(snaps), pts, edge, dt, "rk4", shape)
    res.update(edge_positions=edge, edge_rk4_pos=p, edge_rk4_ftle=f)
    np.savez_compressed(os.path.join(HERE, "windows_2d.npz"), **res)


def gen_windows_3d():
    from pyftle_b200 import flows

    n = 12
    ax = np.linspace(0.0, 2.0 * math.pi, n)
    pts = flows.grid_points_3d(ax, ax, ax)
    dt = 0.1
    times = np.arange(6) * dt
    snaps = flows.abc_snapshots(ax, ax, ax, times)
    cents = flows.centroid_grid_3d(5, 5, 5, (1.0, 1.0, 1.0), (5.0, 5.0, 5.0))
    pos = flows.seeds_3d(cents, 1e-2)
    res = {"shape": np.array((n, n, n)), "points": pts, "snaps": snaps, "positions": pos,
           "dt": np.array(dt)}
    for name in ("euler", "ab2", "rk4"):
        p, f = run_solver(list(snaps), pts, pos, dt, name, (n, n, n))
        res[f"fwd_{name}_pos"], res[f"fwd_{name}_ftle"] = p, f
    p, f = run_solver(list(snaps[::-1]), pts, pos, -dt, "rk4", (n, n, n))
    res["bwd_rk4_pos"], res["bwd_rk4_ftle"] = p, f
    np.savez_compressed(os.path.join(HERE, "windows_3d.npz"), **res)


def gen_analytical():
    from pyftle.data_source import AnalyticalBatchSource
    from pyftle.ftle_solver import FTLESolver
    from pyftle.integrate import create_integrator
    from pyftle.interpolate import create_interpolator
    from pyftle.particles import NeighboringParticles
    from pyftle_b200 import flows

    A, EPS, OMEGA = 0.1, 0.25, 2.0  # the notebook's constants

    def velocity_fn(t, coordinates):
        return flows.double_gyre_velocity(t, coordinates, A=A, eps=EPS, omega=OMEGA)

    pos = flows.seeds_2d(flows.centroid_grid_2d(15, 8, (0.2, 1.8), (0.2, 0.8)), 1e-3)
    res = {"positions": pos}
    for name in ("euler", "rk4"):
        for dt in (0.01, -0.01):
            T = 0.1
            p = int(T / abs(dt)) + 1
            times = np.arange(p) * dt
            src = AnalyticalBatchSource(velocity_fn, NeighboringParticles(pos.copy()), dt, times)
            integ = create_integrator(name, create_interpolator("analytical",
                                                              velocity_fn=velocity_fn))
            solver = FTLESolver(src, integ)
            f = solver.run()
            res[f"{name}_{dt}_ftle"] = np.asarray(f)
            res[f"{name}_{dt}_pos"] = solver.particles.positions.copy()
    np.savez(os.path.join(HERE, "analytical.npz"), **res)


def main():
    tmp = stage_reference()
    try:
        rng = np.random.default_rng(20261203)
        gen_ginterp(rng)
        gen_interpolator(rng)
        gen_ftle(rng)
        gen_integrate()
        gen_windows_2d()
        gen_windows_3d()
        gen_analytical()
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
