"""The reference's CPU hot path, driven around its own compiled ``ginterp``.

TEST / BASELINE INFRASTRUCTURE ONLY: bench.py's reference arm and cpu_baseline
leg time this; the product never imports it.

``oracle/_ref/ginterp*.so`` is pyFTLE's ``GridInterp.cpp`` built from the
reference sources by ``oracle/build.py``.  The Python around it restates, call
for call, what pyFTLE does per step (the Python package itself cannot travel
to the GPU host):

* ``HighPerfInterpolator.update(vel, points)`` -> reshape / transpose,
  ``linspace`` axes, one ``Interp3D``/``Interp2D`` per component with
  ``np.ascontiguousarray(v)`` (interpolate.py:342-425, grid_interp.py:30-38);
* ``interpolate(points)`` -> per component, the ``(x - min)/delta`` index
  transform into a reused buffer, then ``ginterp.interp*d_vec_inplace``
  (interpolate.py:475-543, grid_interp.py:40-85, 123-172);
* ``RungeKutta4Integrator.integrate`` -> k1..k4 with numpy stage
  temporaries and the final update (integrate.py:291-342, :81-109).

When ``oracle/_ref`` is absent the C restatement (``oracle/liboracle.so``)
stands in; the result's ``kind`` says which ran.
"""

from __future__ import annotations

import glob
import importlib.util
import multiprocessing as mp
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_ginterp():
    mods = glob.glob(os.path.join(HERE, "_ref", "ginterp*.so"))
    if not mods:
        return None
    spec = importlib.util.spec_from_file_location("ginterp", mods[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _Interp:
    """Interp2D / Interp3D restated (grid_interp.py)."""

    def __init__(self, fn, v, axes):
        self.fn = fn
        self.v = np.ascontiguousarray(v)
        self.mins = [ax[0] for ax in axes]
        self.deltas = [(ax[-1] - ax[0]) / (ax.shape[0] - 1) for ax in axes]
        self._buf = None

    def __call__(self, t, out):
        arr = np.atleast_2d(t)
        if self._buf is None or self._buf.shape[0] != arr.shape[0]:
            self._buf = np.empty_like(arr)
        for a in range(arr.shape[1]):
            self._buf[:, a] = (arr[:, a] - self.mins[a]) / self.deltas[a]
        self.fn(self.v, self._buf, out)
        return out


class RefGridInterpolator:
    """HighPerfInterpolator("grid") restated around the reference's ginterp."""

    def __init__(self, ginterp, grid_shape):
        self.g = ginterp
        self.grid_shape = tuple(grid_shape)
        self.comps = None
        self._bufs = None

    def update(self, velocities, points):
        shape = self.grid_shape
        dim = len(shape)
        coords = points.reshape((dim, *shape))
        axes = [np.linspace(np.min(coords[a]), np.max(coords[a]), shape[a]) for a in range(dim)]
        if dim == 2:
            v = velocities.reshape((dim, *shape), order="F")
            fn = self.g.interp2d_vec_inplace
        else:
            v = np.transpose(velocities.reshape((dim, *shape)), axes=(0, 2, 1, 3))
            fn = self.g.interp3d_vec_inplace
        self.comps = [_Interp(fn, v[c], axes) for c in range(dim)]

    def interpolate(self, pts):
        n, dim = pts.shape
        if self._bufs is None or self._bufs[0].shape[0] != n:
            self._bufs = [np.empty(n) for _ in range(dim)]
        out = np.empty_like(pts)
        for c in range(dim):
            self.comps[c](pts, self._bufs[c])
            out[:, c] = self._bufs[c]
        return out


def rk4_step(interp, positions, h):
    """RungeKutta4Integrator.integrate restated (integrate.py:291-342)."""
    k1 = interp.interpolate(positions).copy()
    tmp = positions.copy()
    tmp += 0.5 * h * k1
    k2 = interp.interpolate(tmp).copy()
    tmp = positions.copy()
    tmp += 0.5 * h * k2
    k3 = interp.interpolate(tmp).copy()
    tmp = positions.copy()
    tmp += h * k3
    k4 = interp.interpolate(tmp).copy()
    positions += (h / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)


def _worker(args):
    kind, snaps, points, shape, positions, h, nthreads = args
    t0 = time.perf_counter()
    if kind == "reference":
        g = load_ginterp()
        interp = RefGridInterpolator(g, shape)
        pos = positions.copy()
        for s in range(len(snaps)):
            interp.update(snaps[s], points)
            rk4_step(interp, pos, h)
    else:
        from oracle import oracle as O

        gmin, gdel = O.grid_axes(points, shape)
        O.run_window(snaps, shape, gmin, gdel, positions, integrator="rk4", snap_dt=h,
                     with_ftle=False, nthreads=nthreads)
    return time.perf_counter() - t0


def time_reference(snaps, points, shape, positions_per_worker, h, workers: int | None = None):
    """Particle-steps/s of the reference CPU path over ``workers`` processes.

    Each worker advects its own particle block through ``len(snaps)`` HOLD
    RK4 steps (a window slice, as the reference's ParallelExecutor gives each
    process whole windows).  Returns a dict with value, cores and kind.
    """
    kind = "reference" if load_ginterp() is not None else "port"
    if workers is None:
        workers = max(1, min(os.cpu_count() or 1, 32))
    particles = positions_per_worker.shape[0]
    steps = len(snaps)
    if kind == "port":
        # one process, OpenMP over all host threads
        wall = _worker((kind, snaps, points, shape, positions_per_worker, h, workers))
        ps = particles * steps
        return {"value": ps / wall, "cores": workers, "kind": kind, "seconds": wall,
                "particle_steps": ps}
    ctx = mp.get_context("spawn")
    args = [(kind, snaps, points, shape, positions_per_worker, h, 1)] * workers
    t0 = time.perf_counter()
    with ctx.Pool(workers) as pool:
        per = pool.map(_worker, args)
    wall = time.perf_counter() - t0
    ps = particles * steps * workers
    # throughput over the slowest worker's compute time (process start-up excluded)
    return {"value": ps / max(per), "cores": workers, "kind": kind, "seconds": max(per),
            "wall_with_startup": wall, "particle_steps": ps}
