"""Fused FTLE windows: one CUDA launch advects every particle of a window and
computes its FTLE field (replaces the step loop of ``FTLESolver.run``,
``ftle_solver.py:68-161``).

``SnapshotSeries`` uploads a ``(S, dim, nodes)`` snapshot stack once and packs
it into the engine's pair-record layout (FP64 for the plain path, FP16/BF16
for the mixed path).  ``run_window`` then launches ``ftle_window_run_f64`` or
``ftle_window_run_mixed`` on the current torch stream.

Time modes:

* ``"hold"`` -- pyFTLE's semantics: step i uses snapshot ``first_snapshot+i``
  frozen for every RK4 stage; the FTLE uses T = (num_steps - 1)*|h|.
* ``"blend"`` -- the velocity at time t is the linear blend of the two
  snapshots around t (snapshot s at ``snapshot_t0 + s*snapshot_dt``); stage
  times t, t+h/2, t+h; T = num_steps*|h|.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import torch

from pyftle_b200 import _lib
from pyftle_b200._device import as_device_f64, ptr, require_cuda, stream_ptr
from pyftle_b200.interpolate import GridSpec


@dataclass
class EngineOptions:
    """Knobs of the fused path (no reference counterpart)."""

    # "fp64" (plain, the reference's arithmetic) | "fx16" | "fx15" | "fp16" | "bf16"
    precision: str = "fp64"
    time_mode: str = "hold"      # "hold" (reference) | "blend"
    periodic_time: bool = False  # snapshot index wraps modulo the series length
    chunk_steps: Optional[int] = None  # mixed path: steps per launch (None: one launch)
    sort_every: int = 1          # mixed chunked path: cell-sort the groups every n chunks
    # mixed path: the plain FP64 kernel judges the field on every judge_stride-th group
    # (1 % by default) and re-advects the window in FP64 when the sampled FTLE error is
    # above judge_tol (FTLESolver keeps a copy of the seeds for that)
    judge_tol: Optional[float] = None
    judge_stride: int = 100


class SnapshotSeries:
    """A device-resident, packed series of velocity snapshots."""

    def __init__(self, grid: GridSpec, snapshots, precision: str = "fp64",
                 periodic_time: bool = False, keep_source: bool = False):
        require_cuda()
        if precision not in _lib.STORAGE_CODES:
            raise ValueError(f"precision must be one of {list(_lib.STORAGE_CODES)}")
        src = as_device_f64(snapshots)
        if src.ndim != 3 or src.shape[1] != grid.dim or src.shape[2] != grid.nodes:
            raise ValueError(f"snapshots must have shape (S, {grid.dim}, {grid.nodes})")
        self.grid = grid
        self.precision = precision
        self.storage = _lib.STORAGE_CODES[precision]
        self.periodic_time = bool(periodic_time)
        self.num_snapshots = src.shape[0]
        nbytes = _lib.load().ftle_packed_snapshot_bytes(grid.dim, grid.nodes, self.num_snapshots,
                                                        self.storage)
        if nbytes < 0:
            raise ValueError("unsupported snapshot layout")
        # uint8 storage from the caching allocator is 512-byte aligned
        self.packed = torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device=src.device)
        _lib.call("ftle_pack_snapshots", grid.dim, grid.nodes, self.num_snapshots,
                  int(self.periodic_time), ptr(src), self.storage, ptr(self.packed), stream_ptr())
        self.source = src if keep_source else None

    @property
    def nbytes(self) -> int:
        return self.packed.numel()


def window_descriptor(series: SnapshotSeries, positions: torch.Tensor, ftle: Optional[torch.Tensor],
                      *, integrator: str, time_mode: str, h: float, num_steps: int,
                      map_period: float, t0: float = 0.0, first_snapshot: int = 0,
                      snapshot_t0: float = 0.0, snapshot_dt: float = 1.0,
                      keep_positions: bool = False) -> _lib.FtleWindow:
    dim = series.grid.dim
    K = 2 * dim
    if positions.dtype != torch.float64 or not positions.is_cuda or not positions.is_contiguous():
        raise ValueError("positions must be a contiguous float64 CUDA tensor")
    if positions.ndim != 2 or positions.shape[1] != dim or positions.shape[0] % K:
        raise ValueError(f"positions must have shape ({K}*N, {dim})")
    n = positions.shape[0] // K
    if ftle is not None:
        # the kernels write N float64 values through the raw pointer: anything else
        # would be written out of bounds or misread
        if (ftle.dtype != torch.float64 or ftle.device != positions.device
                or not ftle.is_contiguous() or ftle.numel() != n):
            raise ValueError(f"ftle must be a contiguous float64 tensor of {n} elements on "
                             f"{positions.device}")
    w = _lib.FtleWindow()
    w.grid = series.grid.to_abi()
    w.snapshots = series.packed.data_ptr()
    w.num_snapshots = series.num_snapshots
    w.storage = series.storage
    w.time_mode = _lib.TIME_MODES[time_mode]
    w.periodic_time = int(series.periodic_time)
    w.snapshot_t0 = float(snapshot_t0)
    w.snapshot_dt = float(snapshot_dt)
    w.first_snapshot = int(first_snapshot)
    w.integrator = _lib.INTEGRATOR_CODES[integrator.lower()]
    w.t0 = float(t0)
    w.h = float(h)
    w.num_steps = int(num_steps)
    w.flags = _lib.KEEP_POSITIONS if keep_positions else 0
    w.positions = positions.data_ptr()
    w.num_groups = n
    w.map_period = float(map_period)
    w.ftle = 0 if ftle is None else ftle.data_ptr()
    return w


def run_window(series: SnapshotSeries, positions: torch.Tensor, *, integrator: str = "rk4",
               time_mode: str = "hold", h: float, num_steps: int,
               map_period: Optional[float] = None, t0: float = 0.0, first_snapshot: int = 0,
               snapshot_t0: float = 0.0, snapshot_dt: Optional[float] = None,
               ftle_out: Optional[torch.Tensor] = None, with_ftle: bool = True,
               stream: Optional[torch.cuda.Stream] = None, chunk_steps: Optional[int] = None,
               sort_every: int = 1, workspace: Optional[torch.Tensor] = None,
               keep_positions: bool = False) -> Optional[torch.Tensor]:
    """Advect ``positions`` (in place) through one window; return the FTLE field.

    Mixed precision only: ``chunk_steps`` splits the window into launches of that
    many steps with the group state in a device workspace (allocated here unless
    ``workspace`` is given) and a cell sort of the groups every ``sort_every``
    chunks.
    """
    if time_mode not in _lib.TIME_MODES:
        raise ValueError(f"time_mode must be one of {list(_lib.TIME_MODES)}")
    if integrator.lower() not in _lib.INTEGRATOR_CODES:
        raise ValueError(f"Invalid integrator name '{integrator}'.")
    if map_period is None:
        map_period = (num_steps - 1) * abs(h) if time_mode == "hold" else num_steps * abs(h)
    if snapshot_dt is None:
        snapshot_dt = h if time_mode == "hold" else 1.0
    K = 2 * series.grid.dim
    n = positions.shape[0] // K
    ftle = None
    if with_ftle:
        ftle = ftle_out if ftle_out is not None else torch.empty(
            n, dtype=torch.float64, device=positions.device)
    w = window_descriptor(series, positions, ftle, integrator=integrator, time_mode=time_mode,
                          h=h, num_steps=num_steps, map_period=map_period, t0=t0,
                          first_snapshot=first_snapshot, snapshot_t0=snapshot_t0,
                          snapshot_dt=snapshot_dt, keep_positions=keep_positions)
    if series.storage == _lib.F64:
        _lib.call("ftle_window_run_f64", w, stream_ptr(stream))
    elif chunk_steps is None or n == 0:
        _lib.call("ftle_window_run_mixed", w, stream_ptr(stream))
    else:
        need = _lib.load().ftle_window_workspace_bytes(w)
        if workspace is None or workspace.numel() < need:
            workspace = torch.empty(max(need, 256), dtype=torch.uint8, device=positions.device)
        _lib.call("ftle_window_run_mixed_chunked", w, workspace.data_ptr(), workspace.numel(),
                  int(chunk_steps), int(sort_every), stream_ptr(stream))
    return ftle
