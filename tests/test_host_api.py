"""Host-side checks that need no GPU: the C ABI library, struct layouts and the
Python plugin surface (factories, keys, errors) mirroring pyFTLE."""

import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from pyftle_b200 import _lib, flows
from pyftle_b200.integrate import (
    AdamsBashforth2Integrator,
    EulerIntegrator,
    RungeKutta4Integrator,
    create_integrator,
)
from pyftle_b200.interpolate import GridSpec, create_interpolator

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "pyftle_b200.h")


def header_functions():
    src = open(HEADER).read()
    return re.findall(r"^(?:int|int64_t|const char \*)\s*(ftle_\w+)\s*\(", src, re.M)


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 19
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.SIGNATURES), "ctypes signatures and header disagree"
    assert lib.ftle_version() >= 10000


def test_packed_sizes():
    lib = _lib.load()
    assert lib.ftle_packed_snapshot_bytes(2, 100, 3, _lib.F64) == 100 * 3 * 32
    assert lib.ftle_packed_snapshot_bytes(3, 100, 3, _lib.F64) == 100 * 3 * 48
    assert lib.ftle_packed_snapshot_bytes(2, 100, 3, _lib.F16) == 256 + 100 * 3 * 8
    assert lib.ftle_packed_snapshot_bytes(3, 100, 3, _lib.BF16) == 256 + 100 * 3 * 16
    assert lib.ftle_packed_snapshot_bytes(3, 100, 3, _lib.FX15) == 256 + 100 * 3 * 16
    assert lib.ftle_packed_snapshot_bytes(4, 100, 3, _lib.F16) == -1


def test_invalid_arguments_return_status_without_gpu():
    """Argument validation happens on the host: no kernel runs, status + message come back."""
    lib = _lib.load()
    w = _lib.FtleWindow()
    w.grid.dim = 5
    assert lib.ftle_window_run_f64(ctypes.byref(w), None) == _lib.FTLE_ERR_INVALID
    assert b"dim" in lib.ftle_last_error()
    g = _lib.FtleGrid()
    g.dim = 2
    g.n[0] = 1
    assert lib.ftle_grid_interpolate(ctypes.byref(g), None, None, 0, None, None) == \
        _lib.FTLE_ERR_INVALID
    assert lib.ftle_axpy(None, None, 1.0, None, -1, None) == _lib.FTLE_ERR_INVALID
    assert lib.ftle_axpy(None, None, 1.0, None, 0, None) == _lib.FTLE_OK  # empty is a no-op
    with pytest.raises(_lib.FTLEError, match="dim must be 2 or 3"):
        _lib.call("ftle_from_positions", 4, None, None, 1, 1.0, None, None)


def test_struct_layout_matches_c_header():
    """ctypes mirrors of ftle_grid / ftle_window have the C compiler's layout."""
    prog = r"""
    #include <stdio.h>
    #include <stddef.h>
    #include "pyftle_b200.h"
    int main(void) {
      printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(ftle_grid), sizeof(ftle_window),
             offsetof(ftle_window, snapshots), offsetof(ftle_window, h),
             offsetof(ftle_window, positions), offsetof(ftle_window, map_period),
             offsetof(ftle_window, ftle));
      return 0;
    }
    """
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "p.c")
        exe = os.path.join(d, "p")
        open(c, "w").write(prog)
        subprocess.check_call(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe])
        got = [int(x) for x in subprocess.check_output([exe]).split()]
    W = _lib.FtleWindow
    want = [ctypes.sizeof(_lib.FtleGrid), ctypes.sizeof(W), W.snapshots.offset, W.h.offset,
            W.positions.offset, W.map_period.offset, W.ftle.offset]
    assert got == want


def test_create_integrator_keys_and_errors():
    interp = object()
    assert isinstance(create_integrator("ab2", interp), AdamsBashforth2Integrator)
    assert isinstance(create_integrator("euler", interp), EulerIntegrator)
    assert isinstance(create_integrator("rk4", interp), RungeKutta4Integrator)
    assert isinstance(create_integrator("AB2", interp), AdamsBashforth2Integrator)
    assert isinstance(create_integrator("EULER", interp), EulerIntegrator)
    assert isinstance(create_integrator("rK4", interp), RungeKutta4Integrator)
    with pytest.raises(ValueError, match="Invalid integrator name 'invalid'.*"):
        create_integrator("invalid", interp)
    with pytest.raises(ValueError, match="Invalid integrator name ''.*"):
        create_integrator("", interp)


def test_create_interpolator_errors():
    with pytest.raises(ValueError, match="Invalid interpolation type"):
        create_interpolator("nonsense")
    with pytest.raises(NotImplementedError):
        create_interpolator("cubic")
    with pytest.raises(ValueError):
        create_interpolator("analytical")


def test_gridspec_matches_reference_axes(golden):
    """Origin/spacing follow linspace(min, max, n) and (x[-1]-x[0])/(n-1)."""
    d = golden("interpolator.npz")
    for key, sh in (("pts2", "shape2"), ("pts3", "shape3")):
        shape = tuple(d[sh])
        g = GridSpec.from_points(d[key], shape)
        for a in range(len(shape)):
            ax = np.linspace(np.min(d[key][a]), np.max(d[key][a]), shape[a])
            assert g.origin[a] == ax[0]
            assert g.spacing[a] == (ax[-1] - ax[0]) / (shape[a] - 1)


def test_seed_layout_is_role_blocked():
    c = np.array([[0.5, 0.5], [1.0, 0.25]])
    s = flows.seeds_2d(c, 0.1)
    np.testing.assert_allclose(s[0:2], c - [0.1, 0])   # left
    np.testing.assert_allclose(s[2:4], c + [0.1, 0])   # right
    np.testing.assert_allclose(s[4:6], c + [0, 0.1])   # top
    np.testing.assert_allclose(s[6:8], c - [0, 0.1])   # bottom
    c3 = np.array([[1.0, 2.0, 3.0]])
    s3 = flows.seeds_3d(c3, 0.5)
    np.testing.assert_allclose(s3[4], c3[0] + [0, 0, 0.5])  # front
    np.testing.assert_allclose(s3[5], c3[0] - [0, 0, 0.5])  # back


def test_grid_layout_is_meshgrid_xy():
    """Node (i, j) of a 2D snapshot sits at j*nx + i; (i, j, k) of 3D at (j*nx + i)*nz + k."""
    p = flows.grid_points_2d(5, 3, (0, 4), (0, 2))
    assert p[0, 1 * 5 + 2] == 2.0 and p[1, 1 * 5 + 2] == 1.0
    x = np.arange(4.0)
    y = np.arange(3.0) * 10
    z = np.arange(2.0) * 100
    p3 = flows.grid_points_3d(x, y, z)
    i, j, k = 3, 2, 1
    n = (j * 4 + i) * 2 + k
    assert (p3[0, n], p3[1, n], p3[2, n]) == (3.0, 20.0, 100.0)
    s = flows.abc_snapshots(x, y, z, [0.0])
    ref = flows.abc_velocity(0.0, p3.T)
    np.testing.assert_allclose(s[0].T, ref, rtol=1e-14, atol=1e-14)
