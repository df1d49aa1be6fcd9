"""Batch sources (mirror of pyFTLE's ``data_source.py`` protocol).

``BatchSource`` keeps the reference protocol (``data_source.py:29-83``):
``timestep``, ``num_steps``, ``id``, ``get_particles()`` and
``update_interpolator(interpolator, step_index)``.

Two in-memory sources add what the fused GPU path needs -- the whole snapshot
stack at once -- through ``window_spec()``:

* ``MemoryBatchSource`` -- reference semantics (HOLD): ``num_steps`` =
  number of snapshots, step i uses snapshot i with h = ``timestep`` (the
  snapshot spacing; negative for backward time with the snapshots already in
  backward order, as ``__main__.py:91-109`` arranges them).
* ``BlendedSnapshotSource`` -- time-interpolated (BLEND) windows: a step h
  independent of the snapshot spacing, velocities blended linearly between
  the snapshots around each RK4 stage time.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Protocol

import numpy as np

from pyftle_b200.interpolate import GridSpec, Interpolator
from pyftle_b200.particles import NeighboringParticles


class BatchSource(Protocol):
    @property
    def timestep(self) -> float: ...

    @property
    def num_steps(self) -> int: ...

    @property
    def id(self) -> str: ...

    def get_particles(self) -> NeighboringParticles: ...

    def update_interpolator(self, interpolator: Interpolator, step_index: int) -> None: ...


@dataclass
class WindowSpec:
    """Everything the fused path needs for one window."""

    grid: GridSpec
    snapshots: object            # (S, dim, nodes) host array or device tensor
    time_mode: str               # "hold" | "blend"
    h: float
    num_steps: int
    map_period: float
    t0: float = 0.0
    first_snapshot: int = 0
    snapshot_t0: float = 0.0
    snapshot_dt: float = 1.0
    periodic_time: bool = False


class MemoryBatchSource:
    """Snapshots held in memory, reference (HOLD) semantics."""

    def __init__(self, snapshots, points, positions, timestep: float, grid_shape=None,
                 ident: str = "mem", periodic_space: bool = False):
        self.snapshots = snapshots
        self.points = points
        self.positions = positions
        self._timestep = float(timestep)
        self._id = ident
        dim = np.shape(points)[0]
        if grid_shape is None:
            raise ValueError("grid_shape is required")
        if len(grid_shape) != dim:
            raise ValueError("grid_shape and points disagree on the dimension")
        self.grid_shape = tuple(grid_shape)
        self.periodic_space = periodic_space

    @property
    def timestep(self) -> float:
        return self._timestep

    @property
    def num_steps(self) -> int:
        return len(self.snapshots)

    @property
    def id(self) -> str:
        return self._id

    def get_particles(self) -> NeighboringParticles:
        return NeighboringParticles(positions=self.positions)

    def update_interpolator(self, interpolator: Interpolator, step_index: int) -> None:
        interpolator.update(self.snapshots[step_index], self.points if step_index == 0 else None)

    def window_spec(self) -> WindowSpec:
        grid = GridSpec.from_points(self.points, self.grid_shape, self.periodic_space)
        n = self.num_steps
        return WindowSpec(grid=grid, snapshots=self.snapshots, time_mode="hold",
                          h=self._timestep, num_steps=n, map_period=(n - 1) * abs(self._timestep),
                          snapshot_dt=self._timestep)


class BlendedSnapshotSource:
    """Time-blended windows over a snapshot series (no reference counterpart)."""

    def __init__(self, snapshots, points, positions, grid_shape, *, h: float, num_steps: int,
                 snapshot_dt: float, t0: float = 0.0, snapshot_t0: float = 0.0,
                 periodic_space: bool = False, periodic_time: bool = False,
                 ident: Optional[str] = None, map_period: Optional[float] = None):
        self.snapshots = snapshots
        self.points = points
        self.positions = positions
        self.grid_shape = tuple(grid_shape)
        self.h = float(h)
        self._num_steps = int(num_steps)
        self.snapshot_dt = float(snapshot_dt)
        self.t0 = float(t0)
        self.snapshot_t0 = float(snapshot_t0)
        self.periodic_space = periodic_space
        self.periodic_time = periodic_time
        self._id = ident if ident is not None else f"{self.t0:06f}"
        self.map_period = float(map_period) if map_period is not None else self._num_steps * abs(h)

    @property
    def timestep(self) -> float:
        return self.h

    @property
    def num_steps(self) -> int:
        return self._num_steps

    @property
    def id(self) -> str:
        return self._id

    def get_particles(self) -> NeighboringParticles:
        return NeighboringParticles(positions=self.positions)

    def update_interpolator(self, interpolator: Interpolator, step_index: int) -> None:
        raise NotImplementedError(
            "blended windows run only through the fused path (FTLESolver with the grid "
            "interpolator)")

    def window_spec(self) -> WindowSpec:
        grid = GridSpec.from_points(self.points, self.grid_shape, self.periodic_space)
        return WindowSpec(grid=grid, snapshots=self.snapshots, time_mode="blend", h=self.h,
                          num_steps=self._num_steps, map_period=self.map_period, t0=self.t0,
                          snapshot_t0=self.snapshot_t0, snapshot_dt=self.snapshot_dt,
                          periodic_time=self.periodic_time)
