"""Velocity interpolators (mirror of pyFTLE's ``interpolate.py`` for the "grid" key).

``create_interpolator("grid", grid_shape)`` returns a ``HighPerfInterpolator``
whose ``update(velocities, points)`` / ``interpolate(points)`` keep the
reference contract (``interpolate.py:297-543``):

* ``velocities`` and ``points`` are ``(dim, nodes)`` arrays in meshgrid-"xy"
  flattening (2D node (i, j) at ``j*nx + i``, 3D node (i, j, k) at
  ``(j*nx + i)*nz + k``);
* the grid axes are ``linspace(min(coord), max(coord), n)`` and the spacing
  is ``(x[-1] - x[0]) / (n - 1)`` (``interpolate.py:365-401``,
  ``grid_interp.py:32-35``);
* ``interpolate`` maps ``(M, dim)`` physical points to ``(M, dim)``
  velocities, bilinear/trilinear, 0 outside the grid.

Here the snapshot stays on the GPU and one CUDA launch
(``ftle_grid_interpolate``) does the index transform and all components.

Deliberate differences: ``update(velocities)`` without points reuses the
stored grid (the reference's ``HighPerfInterpolator.update`` then crashes on
the next ``interpolate``, ``interpolate.py:467-472``); 3D grids use the
meshgrid-"xy" layout for every shape (the reference is only right for
``nx == ny``, ``interpolate.py:383-385``); ``periodic=True`` wraps the grid
(no reference counterpart).
"""

from __future__ import annotations

from abc import ABC, abstractmethod
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np
import torch

from pyftle_b200 import _lib
from pyftle_b200._device import as_device_f64, ptr, require_cuda, stream_ptr, to_host


@dataclass(frozen=True)
class GridSpec:
    """Regular grid: nodes per axis, origin and spacing (C-ABI ``ftle_grid``)."""

    shape: tuple
    origin: tuple
    spacing: tuple
    periodic: bool = False

    @property
    def dim(self) -> int:
        return len(self.shape)

    @property
    def nodes(self) -> int:
        return int(np.prod(self.shape))

    @classmethod
    def from_points(cls, points, grid_shape, periodic: bool = False) -> "GridSpec":
        """Origin/spacing exactly as interpolate.py:365-401 + grid_interp.py:32-35 derive them."""
        pts = to_host(points)
        dim = len(grid_shape)
        if pts.shape[0] != dim:
            raise ValueError(f"points must have shape ({dim}, nodes)")
        origin, spacing = [], []
        for a in range(dim):
            ax = np.linspace(np.min(pts[a]), np.max(pts[a]), grid_shape[a])
            origin.append(float(ax[0]))
            spacing.append(float((ax[-1] - ax[0]) / (ax.shape[0] - 1)))
        return cls(tuple(int(n) for n in grid_shape), tuple(origin), tuple(spacing), periodic)

    def to_abi(self) -> _lib.FtleGrid:
        g = _lib.FtleGrid()
        g.dim = self.dim
        for a in range(3):
            g.n[a] = self.shape[a] if a < self.dim else 1
            g.origin[a] = self.origin[a] if a < self.dim else 0.0
            g.spacing[a] = self.spacing[a] if a < self.dim else 1.0
        g.periodic = 1 if self.periodic else 0
        return g


class Interpolator(ABC):
    """Interpolator interface (interpolate.py:19-111)."""

    def __init__(self):
        self.velocities = None
        self.points = None
        self.grid_shape: Optional[tuple] = None

    def update(self, velocities, points=None) -> None:
        self.velocities = velocities
        if points is not None:
            self.points = points

    @abstractmethod
    def interpolate(self, new_points):
        ...


class HighPerfInterpolator(Interpolator):
    """Regular-grid bi/trilinear interpolator on the GPU (the "grid" key)."""

    def __init__(self, grid_shape: tuple, periodic: bool = False):
        super().__init__()
        if len(grid_shape) not in (2, 3):
            raise ValueError(f"Unsupported grid dimensionality: {len(grid_shape)}")
        self.grid_shape = tuple(int(n) for n in grid_shape)
        self.periodic = periodic
        self.grid: Optional[GridSpec] = None
        self.snapshot: Optional[torch.Tensor] = None  # (dim, nodes) float64 on the device

    def update(self, velocities, points=None) -> None:
        dim = len(self.grid_shape)
        vel = as_device_f64(velocities)
        if vel.ndim != 2 or vel.shape[0] != dim or vel.shape[1] != int(np.prod(self.grid_shape)):
            raise ValueError(
                f"velocities must have shape ({dim}, {int(np.prod(self.grid_shape))})")
        self.velocities = vel
        self.snapshot = vel
        if points is not None:
            self.points = points
            self.grid = GridSpec.from_points(points, self.grid_shape, self.periodic)
        if self.grid is None:
            raise ValueError("Velocities and points must be set before initialization.")

    def interpolate(self, new_points, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        if self.grid is None or self.snapshot is None:
            raise AssertionError("interpolator was not initialised with update(velocities, points)")
        pts = as_device_f64(new_points)
        dim = self.grid.dim
        if pts.ndim != 2 or pts.shape[1] != dim:
            raise ValueError(f"Unsupported point dimension: {pts.shape[-1]}")
        if out is None:
            out = torch.empty_like(pts)
        g = self.grid.to_abi()
        _lib.call("ftle_grid_interpolate", g, ptr(self.snapshot), ptr(pts), pts.shape[0], ptr(out),
                  stream_ptr())
        return out


class AnalyticalInterpolator(Interpolator):
    """Closed-form velocity ``velocity_fn(t, points) -> velocities`` (interpolate.py:765-829).

    The callable receives and returns device tensors of shape (M, dim); the
    integrators add their stage arithmetic with the CUDA update kernels.
    """

    def __init__(self, velocity_fn: Callable):
        super().__init__()
        self.velocity_fn = velocity_fn
        self.time = 0.0

    def interpolate(self, new_points):
        if not callable(self.velocity_fn):
            raise ValueError("velocity_fn was not assigned properly")
        return self.velocity_fn(self.time, new_points)

    def update(self, velocities, points=None) -> None:
        pass


_OUT_OF_SCOPE = ("cubic", "linear", "nearest")


def create_interpolator(interpolation_type: str, grid_shape: Optional[tuple] = None,
                        velocity_fn: Optional[Callable] = None, *,
                        periodic: bool = False) -> Interpolator:
    """Factory with the reference's keys (interpolate.py:832-901)."""
    interpolation_type = interpolation_type.lower()
    known = ["cubic", "linear", "nearest", "analytical", "grid"]
    if interpolation_type not in known:
        raise ValueError(
            f"Invalid interpolation type '{interpolation_type}'. Choose from {known}.")
    if interpolation_type == "analytical":
        if not callable(velocity_fn):
            raise ValueError("velocity_fn was not assigned properly")
        return AnalyticalInterpolator(velocity_fn)
    if interpolation_type in _OUT_OF_SCOPE:
        raise NotImplementedError(
            f"'{interpolation_type}' (scattered-data / scipy) interpolation is not part of the "
            "GPU engine; use 'grid'")
    if grid_shape is None:
        raise ValueError("the 'grid' interpolator needs grid_shape")
    require_cuda()
    return HighPerfInterpolator(grid_shape, periodic=periodic)
