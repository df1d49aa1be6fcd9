"""Many FTLE windows in one persistent launch, CUDA-graph capture and an autotuner.

The reference computes each FTLE window in its own OS process
(``ParallelExecutor``, parallel.py:171-271; windows from ``__main__.py:111-166``
or ``api.py:125-155``).  Here every window of a batch -- each with its own seed
set, start time, step, length and FTLE period, all over one resident snapshot
series -- runs in one launch of ``windows_persistent_kernel``: persistent CTAs
take work items (128 groups of one window) from a counter, longest windows first.

``WindowBatch`` builds the plan once (``ftle_windows_plan``), keeps it on the
device, and runs it directly or as a captured CUDA graph (``capture()`` /
``replay()``).  A persistent work item keeps its 128 groups for the whole window (the
single-window path re-sorts between chunks instead), so by default the batch hands the
kernel each seed buffer in Morton order of the groups' initial centroids: a work item
then holds a compact patch of the domain and its gathers share cache lines.  Each run
gathers the seeds into that order, runs the kernel, and scatters FTLE (and the final
positions of windows that update them) back to the caller's order; per-group results
are the same bits in either order.  ``autotune()`` times the schedule candidates (CTAs per SM,
ordering) on the batch itself and keeps the fastest; results are cached per
batch shape in ``~/.cache/pyftle_b200/tuning.json``.
"""

from __future__ import annotations

import contextlib
import ctypes
import json
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import torch

from pyftle_b200 import _lib
from pyftle_b200._device import stream_ptr
from pyftle_b200.window import SnapshotSeries, run_window, window_descriptor

TUNING_PATH = os.path.join(os.path.expanduser("~"), ".cache", "pyftle_b200", "tuning.json")


@dataclass
class WindowSpecRun:
    """One window of a batch (positions are advected in place)."""

    positions: torch.Tensor          # (K*N, dim) float64 CUDA, role-blocked
    t0: float
    h: float
    num_steps: int
    map_period: Optional[float] = None
    ftle: Optional[torch.Tensor] = None
    first_snapshot: int = 0  # HOLD windows: snapshot used by step 0
    keep_positions: bool = False  # read-only seeds (windows may share one buffer)


@dataclass
class JudgeReport:
    """Per-window outcome of ``WindowBatch.run_judged``."""

    errors: List[float]       # sampled relative L2 error against FP64, before any fallback
    readvected: List[bool]    # window recomputed by the plain FP64 kernel
    tol: float
    sample_stride: int
    events: tuple = ()        # CUDA events: before the batch, after it, after the judge

    @property
    def batch_ms(self) -> float:
        """Device time of the batch launch (with its seed gather / result scatter)."""
        self.events[2].synchronize()
        return self.events[0].elapsed_time(self.events[1])

    @property
    def judge_ms(self) -> float:
        """Device time of the FP64 samples and the FP64 re-advections."""
        self.events[2].synchronize()
        return self.events[1].elapsed_time(self.events[2])


@dataclass(frozen=True)
class Schedule:
    ctas_per_sm: int = 4  # the kernel fits 4 blocks of 128 threads per SM
    order: int = 1  # 1: longest windows first, 2: by start of the time range, 0: as given


def _spread_bits(x: torch.Tensor, bits: int, dim: int) -> torch.Tensor:
    r = torch.zeros_like(x)
    for b in range(bits):
        r |= ((x >> b) & 1) << (dim * b)
    return r


def morton_order(positions: torch.Tensor, grid) -> torch.Tensor:
    """Permutation of a role-blocked (K*N, dim) seed buffer's N groups that sorts them by
    the Morton code of their centroid's cell on a 2^bits-per-axis coarse grid (2D 10
    bits, 3D 7).  Non-finite centroids sort to the grid's far corner."""
    dim = grid.dim
    K = 2 * dim
    n = positions.shape[0] // K
    cent = positions.view(K, n, dim).mean(dim=0)
    bits = 10 if dim == 2 else 7
    key = torch.zeros(n, dtype=torch.int64, device=positions.device)
    for a in range(dim):
        extent = grid.spacing[a] * (grid.shape[a] if grid.periodic else max(grid.shape[a] - 1, 1))
        f = (cent[:, a] - grid.origin[a]) / extent
        if grid.periodic:
            f = f - torch.floor(f)
        f = torch.nan_to_num(f, nan=1.0, posinf=1.0, neginf=0.0)
        cell = (f * (1 << bits)).clamp(0, (1 << bits) - 1).to(torch.int64)
        key |= _spread_bits(cell, bits, dim) << a
    return torch.argsort(key, stable=True)


class WindowBatch:
    def __init__(self, series: SnapshotSeries, windows: Sequence[WindowSpecRun], *,
                 integrator: str = "rk4", time_mode: str = "blend",
                 snapshot_t0: float = 0.0, snapshot_dt: float = 1.0,
                 schedule: Schedule = Schedule(), spatial_order: bool = True):
        if series.storage == _lib.F64:
            raise ValueError("batched windows run on the mixed-precision path (fx15/fp16/bf16)")
        self.series = series
        self.windows = list(windows)
        self.kw = dict(integrator=integrator, time_mode=time_mode, snapshot_t0=snapshot_t0,
                       snapshot_dt=snapshot_dt)
        dim = series.grid.dim
        K = 2 * dim
        # Spatial order: one permuted copy per distinct seed buffer (windows sharing
        # read-only seeds share it), one FTLE buffer per window in that order.
        self.spatial_order = bool(spatial_order)
        self._src: List[torch.Tensor] = []      # caller's seed buffers
        self._perm: List[torch.Tensor] = []     # group permutation per buffer
        self._sorted: List[torch.Tensor] = []   # seeds in Morton order
        self._shared: List[bool] = []          # buffer is read-only seeds (shareable)
        self._win_src: List[int] = []
        self._win_ftle: List[torch.Tensor] = []
        for w in self.windows:
            p = w.positions
            if (p.dtype != torch.float64 or not p.is_cuda or not p.is_contiguous()
                    or p.ndim != 2 or p.shape[1] != dim or p.shape[0] % K):
                raise ValueError(f"positions must be a contiguous float64 CUDA tensor of shape "
                                 f"({K}*N, {dim})")
            n = w.positions.shape[0] // K
            if w.ftle is None:
                w.ftle = torch.empty(n, dtype=torch.float64, device=w.positions.device)
            elif (w.ftle.dtype != torch.float64 or w.ftle.device != p.device
                  or not w.ftle.is_contiguous() or w.ftle.numel() != n):
                raise ValueError(f"ftle must be a contiguous float64 tensor of {n} elements "
                                 f"on {p.device}")
            if not self.spatial_order:
                continue
            # read-only seeds are shared only with a window over the very same buffer
            # (same start and shape; a prefix view of a larger buffer is not the same)
            k = next((i for i, t in enumerate(self._src)
                      if w.keep_positions and self._shared[i]
                      and t.data_ptr() == p.data_ptr() and t.shape == p.shape), None)
            if k is None:
                self._src.append(w.positions)
                self._shared.append(bool(w.keep_positions))
                perm = morton_order(w.positions, series.grid)
                self._perm.append(perm)
                self._sorted.append(torch.empty_like(w.positions))
                k = len(self._src) - 1
            self._win_src.append(k)
            self._win_ftle.append(torch.empty_like(w.ftle))
        self._gather()
        arr = (_lib.FtleWindow * len(self.windows))()
        self._map_period: List[float] = []
        for i, w in enumerate(self.windows):
            pos = self._sorted[self._win_src[i]] if self.spatial_order else w.positions
            ftle = self._win_ftle[i] if self.spatial_order else w.ftle
            if w.map_period is not None:
                mp = w.map_period
            elif time_mode == "hold":  # the reference's T = (p - 1)|dt| (ftle_solver.py:156)
                mp = (w.num_steps - 1) * abs(w.h)
            else:
                mp = w.num_steps * abs(w.h)
            self._map_period.append(mp)
            arr[i] = window_descriptor(series, pos, ftle, h=w.h, num_steps=w.num_steps,
                                       map_period=mp, t0=w.t0, first_snapshot=w.first_snapshot,
                                       keep_positions=w.keep_positions, **self.kw)
        self.desc = arr
        self.count = len(self.windows)
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        self._plans = {}
        self.schedule = schedule

    # ------------------------------------------------------------------
    def _plan(self, order: int) -> torch.Tensor:
        if order in self._plans:
            return self._plans[order]
        lib = _lib.load()
        nbytes = lib.ftle_windows_plan_bytes(self.desc, self.count)
        if nbytes < 0:
            raise ValueError("invalid batch")
        host = np.zeros(nbytes, dtype=np.uint8)
        _lib.call("ftle_windows_plan", self.desc, self.count, int(order),
                  host.ctypes.data_as(ctypes.c_void_p), nbytes)
        dev = torch.from_numpy(host).to(self.windows[0].positions.device)
        self._plans[order] = dev
        return dev

    def _view(self, t: torch.Tensor) -> torch.Tensor:
        K = 2 * self.series.grid.dim
        return t.view(K, t.shape[0] // K, self.series.grid.dim)

    def _gather(self) -> None:
        """Seeds (caller's order) -> Morton-ordered copies."""
        for src, perm, dst in zip(self._src, self._perm, self._sorted):
            torch.index_select(self._view(src), 1, perm, out=self._view(dst))

    def _scatter(self) -> None:
        """FTLE, and the final positions of windows that update them, back to the
        caller's order."""
        for i, w in enumerate(self.windows):
            k = self._win_src[i]
            w.ftle.index_copy_(0, self._perm[k], self._win_ftle[i])
            if not w.keep_positions:
                self._view(w.positions).index_copy_(1, self._perm[k], self._view(self._sorted[k]))

    def run(self, schedule: Optional[Schedule] = None, stream=None) -> List[torch.Tensor]:
        sch = schedule or self.schedule
        plan = self._plan(sch.order)
        with torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext():
            if self.spatial_order:
                self._gather()
            _lib.call("ftle_windows_run_mixed", self.desc, self.count, plan.data_ptr(),
                      plan.numel(), int(sch.ctas_per_sm), stream_ptr(stream))
            if self.spatial_order:
                self._scatter()
        return [w.ftle for w in self.windows]

    def run_judged(self, series64: SnapshotSeries, *, tol: float = 1e-3,
                   sample_stride: int = 100, fallback: bool = True,
                   schedule: Optional[Schedule] = None) -> "JudgeReport":
        """Run the batch, then judge every window against the plain FP64 path (the
        batch's integrator and time mode) on a sample of its groups and re-advect in
        FP64 every window whose sampled error exceeds ``tol``.

        The sample of window i is every ``sample_stride``-th group starting at group
        ``i mod sample_stride`` (1% at the default), advected by the plain FP64
        kernel over ``series64`` (the same snapshots stored as ``"fp64"``) with the
        window's own start, step, length and FTLE period.  The window's error is the
        relative L2 norm ||F - F64|| / ||F64|| over the sample (the absolute norm
        where F64 is zero there).  With ``fallback`` every window above ``tol`` is
        recomputed by the plain FP64 kernel over all its groups, so its FTLE (and
        its final positions, for a window that updates them) become the FP64 ones;
        windows that advect in place keep a copy of their seeds for this, taken
        before the run.
        """
        if series64.storage != _lib.F64:
            raise ValueError("series64 must hold the snapshots as \"fp64\"")
        if (series64.grid.shape != self.series.grid.shape
                or series64.num_snapshots != self.series.num_snapshots
                or series64.periodic_time != self.series.periodic_time):
            raise ValueError("series64 must hold the batch's snapshots: same grid, number "
                             "of snapshots and time periodicity")
        if sample_stride < 1:
            raise ValueError("sample_stride must be >= 1")
        K = 2 * self.series.grid.dim
        seeds0 = [w.positions if w.keep_positions or not fallback else w.positions.clone()
                  for w in self.windows]
        samples = []
        for i, w in enumerate(self.windows):
            n = w.positions.shape[0] // K
            sel = torch.arange(i % sample_stride if n > i % sample_stride else 0, n,
                               sample_stride, device=w.positions.device)
            sub = self._view(seeds0[i])[:, sel, :]  # advanced indexing: a copy
            samples.append((sel, sub.reshape(-1, self.series.grid.dim).contiguous()))
        ev = tuple(torch.cuda.Event(enable_timing=True) for _ in range(3))
        ev[0].record()
        self.run(schedule)
        ev[1].record()
        kw = dict(integrator=self.kw["integrator"], time_mode=self.kw["time_mode"],
                  snapshot_t0=self.kw["snapshot_t0"], snapshot_dt=self.kw["snapshot_dt"])
        errors, readvected = [], []
        for i, w in enumerate(self.windows):
            sel, sub = samples[i]
            win = dict(h=w.h, num_steps=w.num_steps, map_period=self._map_period[i], t0=w.t0,
                       first_snapshot=w.first_snapshot, **kw)
            f64 = run_window(series64, sub, **win)
            ref = torch.linalg.vector_norm(f64)
            diff = torch.linalg.vector_norm(w.ftle[sel] - f64)
            err = float(diff / ref) if float(ref) > 0 else float(diff)
            errors.append(err)
            redo = fallback and not err <= tol  # NaN errors are re-advected too
            if redo:
                pos = seeds0[i]
                run_window(series64, pos, ftle_out=w.ftle, keep_positions=w.keep_positions,
                           **win)
                if not w.keep_positions:
                    w.positions.copy_(pos)
            readvected.append(redo)
        ev[2].record()
        return JudgeReport(errors=errors, readvected=readvected, tol=tol,
                           sample_stride=sample_stride, events=ev)

    @property
    def particle_steps(self) -> int:
        return sum(w.positions.shape[0] * w.num_steps for w in self.windows)

    @property
    def shape_key(self) -> str:
        g = self.series.grid
        steps = sorted(w.num_steps for w in self.windows)
        groups = sum(w.positions.shape[0] for w in self.windows) // (2 * g.dim)
        return (f"d{g.dim}-{self.series.precision}-{self.kw['integrator']}-w{self.count}"
                f"-g{int(np.log2(max(groups, 1)))}-s{steps[len(steps) // 2]}")

    # ------------------------------------------------------------------
    def capture(self, prologue=None) -> torch.cuda.CUDAGraph:
        """Capture (optional prologue, e.g. resetting positions) + the batch run."""
        self._plan(self.schedule.order)  # plan built and uploaded outside the capture
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            if prologue is not None:  # warm any lazy allocation outside the graph
                prologue()
            self.run(stream=s)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=s):
            if prologue is not None:
                prologue()
            self.run(stream=s)
        self.graph = g
        return g

    def replay(self) -> List[torch.Tensor]:
        if self.graph is None:
            raise RuntimeError("capture() first")
        self.graph.replay()
        return [w.ftle for w in self.windows]

    # ------------------------------------------------------------------
    def autotune(self, prologue=None, candidates: Optional[Sequence[Schedule]] = None,
                 use_cache: bool = True) -> Schedule:
        """Time every candidate schedule on this batch and keep the fastest."""
        cache = _load_cache() if use_cache else {}
        if use_cache and self.shape_key in cache:
            self.schedule = Schedule(**cache[self.shape_key]["schedule"])
            return self.schedule
        # blocks per SM the kernel can keep resident: 4 in 3D, up to 8 in 2D
        ctas = (1, 2, 3, 4) if self.series.grid.dim == 3 else (2, 4, 6, 8)
        cands = list(candidates) if candidates else [Schedule(c, o) for c in ctas
                                                     for o in (1, 2, 0)]
        timings = []
        for sch in cands:
            if prologue:
                prologue()
            self.run(sch)  # warm-up (and builds the plan for this order)
            if prologue:
                prologue()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            self.run(sch)
            b.record()
            torch.cuda.synchronize()
            timings.append((a.elapsed_time(b), sch))
        best_ms, best = min(timings, key=lambda x: x[0])
        self.schedule = best
        self.tuning = [{"ms": ms, "ctas_per_sm": s.ctas_per_sm, "order": s.order}
                       for ms, s in timings]
        if use_cache:
            cache[self.shape_key] = {"schedule": {"ctas_per_sm": best.ctas_per_sm,
                                                  "order": best.order}, "ms": best_ms}
            _save_cache(cache)
        return best


def _load_cache() -> dict:
    try:
        with open(TUNING_PATH) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save_cache(cache: dict) -> None:
    try:
        os.makedirs(os.path.dirname(TUNING_PATH), exist_ok=True)
        with open(TUNING_PATH, "w") as f:
            json.dump(cache, f, indent=1)
    except OSError:
        pass
