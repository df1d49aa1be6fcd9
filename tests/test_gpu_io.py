"""File-fed windows on the GPU: pyFTLE's golden double-gyre window written to
.mat files and read back through FileBatchSource must reproduce the reference
bit for bit; the sliding-window runner must reproduce the oracle on every window."""

import numpy as np
import pytest
import torch
from scipy.io import loadmat, savemat

from oracle import oracle as O
from pyftle_b200 import FTLESolver, create_integrator, create_interpolator, flows, io
from pyftle_b200.scheduler import SlidingWindowRunner

pytestmark = pytest.mark.gpu


def _write_case(tmp_path, d, direction="fwd"):
    shape = tuple(d["shape"])
    nx, ny = shape
    snaps = d["snaps"] if direction == "fwd" else d["snaps"][::-1]
    files = []
    for i, s in enumerate(snaps):
        f = tmp_path / f"vel_{i:03d}.mat"
        savemat(f, {"velocity_x": s[0].reshape(ny, nx), "velocity_y": s[1].reshape(ny, nx)})
        files.append(str(f))
    cf = tmp_path / "coords.mat"
    savemat(cf, {"coordinate_x": d["points"][0].reshape(ny, nx),
                 "coordinate_y": d["points"][1].reshape(ny, nx)})
    pos = d["positions"]
    N = pos.shape[0] // 4
    pf = tmp_path / "seeds.mat"
    savemat(pf, {"left": pos[:N], "right": pos[N:2 * N], "top": pos[2 * N:3 * N],
                 "bottom": pos[3 * N:]})
    return files, str(cf), str(pf)


@pytest.mark.parametrize("direction", ["fwd", "bwd"])
@pytest.mark.parametrize("fused", [True, False])
def test_file_batch_source_matches_reference(golden, tmp_path, direction, fused):
    d = golden("windows_2d.npz")
    shape = tuple(d["shape"])
    files, cf, pf = _write_case(tmp_path, d, direction)
    dt = float(d["dt"]) * (1 if direction == "fwd" else -1)
    src = io.FileBatchSource(files, [cf] * len(files), pf, dt, len(files), grid_shape=shape)
    solver = FTLESolver(src, create_integrator("rk4", create_interpolator("grid", shape)))
    if not fused:
        solver._fused_ok = lambda: False
    ftle = solver.run()
    np.testing.assert_array_equal(solver.particles.positions_host(), d[f"{direction}_rk4_pos"])
    np.testing.assert_allclose(ftle, d[f"{direction}_rk4_ftle"], rtol=1e-10, atol=0)


@pytest.mark.parametrize("precision", ["fp64", "fx15"])
def test_sliding_windows_match_oracle(golden, tmp_path, precision):
    d = golden("windows_2d.npz")
    shape = tuple(d["shape"])
    files, cf, pf = _write_case(tmp_path, d)
    dt = float(d["dt"])
    runner = SlidingWindowRunner(files, [cf], [pf], dt, flow_map_period=4 * dt, grid_shape=shape,
                                 precision=precision)
    assert runner.window_length == 5
    fields = runner.run()
    assert len(fields) == len(files) - 5 + 1
    gmin, gdel = O.grid_axes(d["points"], shape)
    for i, f in enumerate(fields):
        _, ref = O.run_window(d["snaps"], shape, gmin, gdel, d["positions"], integrator="rk4",
                              snap_dt=dt, first_snapshot=i, num_steps=5)
        if precision == "fp64":
            np.testing.assert_allclose(f, ref, rtol=1e-12, atol=0)
        else:
            assert np.linalg.norm(f - ref) / np.linalg.norm(ref) < 1e-3


def test_sliding_windows_backward_with_writer(golden, tmp_path):
    d = golden("windows_2d.npz")
    shape = tuple(d["shape"])
    files, cf, pf = _write_case(tmp_path, d)
    dt = float(d["dt"])
    writer = io.create_writer("mat", str(tmp_path / "out"), grid_shape=None)
    runner = SlidingWindowRunner(files, [cf], [pf], -dt, flow_map_period=3 * dt,
                                 grid_shape=shape, writer=writer)
    assert runner.run() is None
    gmin, gdel = O.grid_axes(d["points"], shape)
    rev = d["snaps"][::-1]
    for i, (first, _, _, ident) in enumerate(runner.windows()):
        m = loadmat(tmp_path / "out" / f"ftle_{ident}.mat")
        _, ref = O.run_window(rev, shape, gmin, gdel, d["positions"], integrator="rk4",
                              snap_dt=-dt, first_snapshot=first, num_steps=4)
        np.testing.assert_allclose(m["ftle"].ravel(), ref, rtol=1e-12, atol=0)
    assert runner.windows()[0][3] == "vel_010"  # backward windows start from the last file


@pytest.mark.parametrize("direction", [1, -1])
def test_streaming_windows_equal_resident_series(golden, tmp_path, direction):
    """The streamed feed (pinned host ring, device ring of p + depth packed snapshots
    wrapping many times) gives the bits of the all-resident series, window by window,
    forward and backward."""
    d = golden("windows_2d.npz")
    shape = tuple(d["shape"])
    files, cf, pf = _write_case(tmp_path, d)
    dt = float(d["dt"]) * direction
    kw = dict(flow_map_period=2 * abs(dt), grid_shape=shape, workers=2)
    resident = SlidingWindowRunner(files, [cf], [pf], dt, streaming=False, **kw)
    b = resident.run()
    for by_steps in (True, False):  # the head windows by per-step launches, or all fused
        streamed = SlidingWindowRunner(files, [cf], [pf], dt, streaming=True, device_depth=1,
                                       head_per_step=by_steps, **kw)
        a = streamed.run()
        assert streamed.stats["device_ring_snapshots"] == streamed.window_length + 1
        assert len(a) == len(b) == len(files) - streamed.window_length + 1
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("integrator", ["euler", "ab2"])
def test_streaming_head_windows_other_integrators(golden, tmp_path, integrator):
    d = golden("windows_2d.npz")
    shape = tuple(d["shape"])
    files, cf, pf = _write_case(tmp_path, d)
    dt = float(d["dt"])
    kw = dict(flow_map_period=3 * dt, grid_shape=shape, workers=2, integrator_name=integrator)
    b = SlidingWindowRunner(files, [cf], [pf], dt, streaming=False, **kw).run()
    for head in (None, 1, 4):  # the default (p + 1) // 2, one, all p = 4 head windows
        r = SlidingWindowRunner(files, [cf], [pf], dt, streaming=True, head_windows=head, **kw)
        a = r.run()
        H = (r.window_length + 1) // 2 if head is None else head
        assert r.stats["head_windows"] == H  # then fused windows follow
        assert r.stats["fused_windows"] == len(b) - H
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("integrator", ["rk4", "ab2"])
def test_streaming_head_windows_edge_cases(golden, tmp_path, integrator):
    """Every window a head window (no fused window at all), and windows that alternate
    between two particle files (the head stops at the first window with another file)."""
    d = golden("windows_2d.npz")
    shape = tuple(d["shape"])
    files, cf, pf = _write_case(tmp_path, d)
    dt = float(d["dt"])
    kw = dict(grid_shape=shape, workers=2, integrator_name=integrator)
    long = dict(kw, flow_map_period=6 * dt)  # p = 7: windows 0..4 all start before file 6
    b = SlidingWindowRunner(files, [cf], [pf], dt, streaming=False, **long).run()
    r = SlidingWindowRunner(files, [cf], [pf], dt, streaming=True, head_windows=7, **long)
    a = r.run()
    assert r.stats["head_windows"] == len(b) and r.stats["fused_windows"] == 0
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    # a second particle file: the first half of the first file's groups, in role blocks
    pos = d["positions"]
    N = pos.shape[0] // 4
    M = N // 2
    pf2 = tmp_path / "seeds2.mat"
    savemat(pf2, {"left": pos[:M], "right": pos[N:N + M], "top": pos[2 * N:2 * N + M],
                  "bottom": pos[3 * N:3 * N + M]})
    two = dict(kw, flow_map_period=2 * dt)
    b = SlidingWindowRunner(files, [cf], [pf, str(pf2)], dt, streaming=False, **two).run()
    r = SlidingWindowRunner(files, [cf], [pf, str(pf2)], dt, streaming=True, **two)
    a = r.run()
    assert r.stats["head_windows"] == 1
    assert [x.shape[0] for x in a] == [x.shape[0] for x in b]
    assert {x.shape[0] for x in a} == {N, M}
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_streaming_head_windows_capped_by_memory(golden, tmp_path, monkeypatch):
    """The head windows' position blocks stay within the runner's memory budget: with a
    budget of two windows' positions only two windows are head windows (same bits)."""
    from pyftle_b200 import scheduler

    d = golden("windows_2d.npz")
    shape = tuple(d["shape"])
    files, cf, pf = _write_case(tmp_path, d)
    dt = float(d["dt"])
    kw = dict(flow_map_period=5 * dt, grid_shape=shape, workers=2)
    b = SlidingWindowRunner(files, [cf], [pf], dt, streaming=False, **kw).run()
    monkeypatch.setattr(scheduler, "HEAD_BYTES", d["positions"].size * 8 * 2)
    r = SlidingWindowRunner(files, [cf], [pf], dt, streaming=True, head_windows=6, **kw)
    a = r.run()
    assert r.stats["head_windows"] == 2
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
