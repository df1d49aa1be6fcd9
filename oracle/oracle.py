"""ctypes front end of the CPU oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s cpu_baseline /
reference legs import this module, and only as the checker or the timed CPU
baseline -- never as a product path.

The oracle is pinned against the reference itself: ``tests/test_oracle.py``
compares it with golden vectors that ``tests/golden/make_golden.py`` produced by
running pyFTLE (interpolator bit-exact, HOLD windows bit-exact, FTLE rtol 1e-12).
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from oracle.build import LIB, build_oracle

_lib = None

EULER, AB2, RK4 = 0, 1, 2
HOLD, BLEND = 0, 1
INTEGRATORS = {"euler": EULER, "ab2": AB2, "rk4": RK4}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build_oracle()
        L = ctypes.CDLL(LIB)
        L.oracle_interp2d.argtypes = [_dp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int64, _dp]
        L.oracle_interp3d.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                                      ctypes.c_int64, _dp]
        L.oracle_window_f64.restype = ctypes.c_int
        L.oracle_window_f64.argtypes = [
            ctypes.c_int, _ip, _dp, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
            ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double,
            ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int64, ctypes.c_double,
            _dp, ctypes.c_int]
        L.oracle_ftle_from_jacobians.argtypes = [ctypes.c_int, _dp, ctypes.c_int64,
                                                 ctypes.c_double, _dp]
        L.oracle_ftle_from_positions.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_int64,
                                                 ctypes.c_double, _dp]
        L.oracle_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def interp2d_vec_inplace(v, points, out) -> None:
    """Same contract as the reference's ``ginterp.interp2d_vec_inplace``."""
    v = np.ascontiguousarray(v, dtype=np.float64)
    points = np.ascontiguousarray(points, dtype=np.float64)
    assert v.ndim == 2 and points.ndim == 2 and points.shape[1] == 2
    lib().oracle_interp2d(_p(v), v.shape[0], v.shape[1], _p(points), points.shape[0], _p(out))


def interp3d_vec_inplace(v, points, out) -> None:
    """Same contract as the reference's ``ginterp.interp3d_vec_inplace``."""
    v = np.ascontiguousarray(v, dtype=np.float64)
    points = np.ascontiguousarray(points, dtype=np.float64)
    assert v.ndim == 3 and points.ndim == 2 and points.shape[1] == 3
    lib().oracle_interp3d(_p(v), *v.shape, _p(points), points.shape[0], _p(out))


def grid_axes(points: np.ndarray, grid_shape) -> tuple[np.ndarray, np.ndarray]:
    """Grid origin and spacing as the reference derives them.

    interpolate.py:365-401 builds ``linspace(min(coord), max(coord), n)`` and
    grid_interp.py:32-35 takes ``(x[-1] - x[0]) / (n - 1)``.
    """
    dim = len(grid_shape)
    gmin = np.zeros(3)
    gdelta = np.ones(3)
    for a in range(dim):
        ax = np.linspace(np.min(points[a]), np.max(points[a]), grid_shape[a])
        gmin[a] = ax[0]
        gdelta[a] = (ax[-1] - ax[0]) / (ax.shape[0] - 1)
    return gmin, gdelta


def run_window(snapshots: np.ndarray, grid_shape, gmin, gdelta, positions: np.ndarray, *,
               integrator="rk4", time_mode=HOLD, h=None, num_steps=None, t0=0.0,
               snap_t0=0.0, snap_dt=1.0, first_snapshot=0, periodic_space=False,
               periodic_time=False, map_period=None, with_ftle=True, nthreads=0):
    """Advect ``positions`` (copied) through one window; returns (positions, ftle).

    ``snapshots`` is (S, dim, nodes) in the reference layout.  HOLD defaults
    follow FTLESolver: num_steps = S - first_snapshot, h = snap_dt,
    map_period = (num_steps - 1)*|h|.
    """
    snaps = np.ascontiguousarray(snapshots, dtype=np.float64)
    S, dim, nodes = snaps.shape
    assert nodes == int(np.prod(grid_shape)) and dim == len(grid_shape)
    pos = np.array(positions, dtype=np.float64, order="C", copy=True)
    K = 2 * dim
    assert pos.shape[1] == dim and pos.shape[0] % K == 0
    N = pos.shape[0] // K
    if h is None:
        h = snap_dt
    if num_steps is None:
        num_steps = S - first_snapshot
    if map_period is None:
        map_period = (num_steps - 1) * abs(h) if time_mode == HOLD else num_steps * abs(h)
    n = np.zeros(3, dtype=np.int32)
    n[:dim] = grid_shape
    gmin = np.ascontiguousarray(gmin, dtype=np.float64).reshape(-1)
    gdelta = np.ascontiguousarray(gdelta, dtype=np.float64).reshape(-1)
    gm = np.zeros(3); gm[:dim] = gmin[:dim]
    gd = np.ones(3); gd[:dim] = gdelta[:dim]
    ftle = np.zeros(N) if with_ftle else None
    rc = lib().oracle_window_f64(
        dim, n.ctypes.data_as(_ip), _p(gm), _p(gd), int(periodic_space), _p(snaps), S,
        int(time_mode), float(snap_t0), float(snap_dt), int(periodic_time), int(first_snapshot),
        float(t0), float(h), int(num_steps), INTEGRATORS[integrator] if isinstance(integrator, str)
        else int(integrator), _p(pos), N, float(map_period),
        _p(ftle) if ftle is not None else ctypes.cast(None, _dp), int(nthreads))
    if rc != 0:
        raise ValueError("oracle_window_f64 rejected its arguments")
    return pos, ftle


def ftle_from_jacobians(J: np.ndarray, map_period: float) -> np.ndarray:
    J = np.ascontiguousarray(J, dtype=np.float64)
    dim = J.shape[1]
    out = np.empty(J.shape[0])
    lib().oracle_ftle_from_jacobians(dim, _p(J), J.shape[0], float(map_period), _p(out))
    return out


def ftle_from_positions(positions, initial, map_period: float) -> np.ndarray:
    positions = np.ascontiguousarray(positions, dtype=np.float64)
    initial = np.ascontiguousarray(initial, dtype=np.float64)
    dim = positions.shape[1]
    N = positions.shape[0] // (2 * dim)
    out = np.empty(N)
    lib().oracle_ftle_from_positions(dim, _p(positions), _p(initial), N, float(map_period),
                                     _p(out))
    return out
