"""Sliding FTLE windows over one resident snapshot series.

Replaces the reference's window driver (``MultipleFTLEProcessManager``,
``__main__.py:18-207``): with n snapshot files and a flow-map period T, the window
length is p = int(T/|dt|) + 1 and there are n - p + 1 overlapping windows
(``__main__.py:111-166``); negative dt reverses the file lists
(``__main__.py:91-109``); window i uses particle file i (cycled) and is named
after its first snapshot file.  The reference runs each window in its own
process and re-reads its p snapshot files; here all n snapshots are read once
(in parallel, copied to the device while reading), packed once, and every
window runs from that resident series -- one launch per window on the FP64
path, or all windows in one persistent launch on the mixed path.
"""

from __future__ import annotations

import itertools
from pathlib import Path
from typing import List, Optional

import numpy as np
import torch

from pyftle_b200 import io
from pyftle_b200.batch import WindowBatch, WindowSpecRun
from pyftle_b200.interpolate import GridSpec
from pyftle_b200.particles import NeighboringParticles
from pyftle_b200.window import SnapshotSeries, run_window


class SlidingWindowRunner:
    def __init__(self, snapshot_files: List[str], coordinate_files: List[str],
                 particle_files: List[str], snapshot_timestep: float, flow_map_period: float,
                 grid_shape: tuple, integrator_name: str = "rk4", writer=None,
                 precision: str = "fp64", periodic_space: bool = False, workers: int = 8):
        self.snapshot_files = list(snapshot_files)
        self.coordinate_files = list(coordinate_files)
        self.particle_files = list(particle_files)
        self.timestep = float(snapshot_timestep)
        self.flow_map_period = float(flow_map_period)
        self.grid_shape = tuple(grid_shape)
        self.integrator = integrator_name.lower()
        self.writer = writer
        self.precision = precision
        self.periodic_space = periodic_space
        self.workers = workers
        if self.timestep < 0:  # backward time: reverse the file order
            self.snapshot_files.reverse()
            self.coordinate_files.reverse()
            self.particle_files.reverse()

    @property
    def window_length(self) -> int:
        return int(self.flow_map_period / abs(self.timestep)) + 1

    def windows(self):
        """(first snapshot, particle file, coordinate files, id) for every window."""
        n = len(self.snapshot_files)
        p = self.window_length
        coord_cycle = list(itertools.islice(itertools.cycle(self.coordinate_files), n + p - 1))
        part_cycle = list(itertools.islice(itertools.cycle(self.particle_files), n))
        return [(i, part_cycle[i], coord_cycle[i:i + p], Path(self.snapshot_files[i]).stem)
                for i in range(n - p + 1)]

    def run(self) -> Optional[List[np.ndarray]]:
        wins = self.windows()
        if not wins:
            return [] if self.writer is None else None
        if len(set(self.coordinate_files)) != 1:
            return self._run_moving_grid(wins)
        points = io.read_coordinate(self.coordinate_files[0])
        grid = GridSpec.from_points(points, self.grid_shape, self.periodic_space)
        snaps = io.load_snapshots(self.snapshot_files, grid.dim, grid.nodes, workers=self.workers)
        series = SnapshotSeries(grid, snaps, precision=self.precision)
        del snaps
        p = self.window_length
        dt = self.timestep
        seeds = {}
        particles = []
        for _, pf, _, _ in wins:
            if pf not in seeds:
                seeds[pf] = io.read_seed_particles_coordinates(pf)
            particles.append(NeighboringParticles(positions=seeds[pf].positions))
        kw = dict(integrator=self.integrator, time_mode="hold", h=dt, num_steps=p,
                  map_period=(p - 1) * abs(dt), snapshot_dt=dt)
        if self.precision == "fp64":
            fields = [run_window(series, part.positions, first_snapshot=first, **kw)
                      for (first, _, _, _), part in zip(wins, particles)]
        else:
            runs = [WindowSpecRun(part.positions, 0.0, dt, p, map_period=(p - 1) * abs(dt),
                                  first_snapshot=first)
                    for (first, _, _, _), part in zip(wins, particles)]
            fields = WindowBatch(series, runs, integrator=self.integrator, time_mode="hold",
                                 snapshot_dt=dt).run()
        torch.cuda.synchronize()
        return self._emit(wins, particles, fields)

    def _run_moving_grid(self, wins):
        """Coordinates change between snapshots: the reference loop, one window at a time."""
        from pyftle_b200.ftle_solver import FTLESolver
        from pyftle_b200.integrate import create_integrator
        from pyftle_b200.interpolate import create_interpolator

        fields, particles = [], []
        p = self.window_length
        for first, pf, coords, _ in wins:
            src = io.FileBatchSource(self.snapshot_files[first:first + p], coords, pf,
                                     self.timestep, p, grid_shape=self.grid_shape)
            integ = create_integrator(self.integrator,
                                      create_interpolator("grid", self.grid_shape))
            solver = FTLESolver(src, integ)
            fields.append(solver.run_device())
            particles.append(solver.particles)
        return self._emit(wins, particles, fields)

    def _emit(self, wins, particles, fields):
        out = []
        for (_, _, _, ident), part, f in zip(wins, particles, fields):
            arr = f.cpu().numpy()
            if self.writer is not None:
                self.writer.write(f"ftle_{ident}", arr, part.initial_centroid.cpu().numpy())
            else:
                out.append(arr)
        return None if self.writer is not None else out
