"""Many FTLE windows in one persistent launch, CUDA-graph capture and an autotuner.

The reference computes each FTLE window in its own OS process
(``ParallelExecutor``, parallel.py:171-271; windows from ``__main__.py:111-166``
or ``api.py:125-155``).  Here every window of a batch -- each with its own seed
set, start time, step, length and FTLE period, all over one resident snapshot
series -- runs in one launch of ``windows_persistent_kernel``: persistent CTAs
take work items (128 groups of one window) from a counter, longest windows first.

``WindowBatch`` builds the plan once (``ftle_windows_plan``), keeps it on the
device, and runs it directly or as a captured CUDA graph (``capture()`` /
``replay()``).  ``autotune()`` times the schedule candidates (CTAs per SM,
ordering) on the batch itself and keeps the fastest; results are cached per
batch shape in ``~/.cache/pyftle_b200/tuning.json``.
"""

from __future__ import annotations

import ctypes
import json
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import torch

from pyftle_b200 import _lib
from pyftle_b200._device import stream_ptr
from pyftle_b200.window import SnapshotSeries, window_descriptor

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


@dataclass(frozen=True)
class Schedule:
    ctas_per_sm: int = 4  # the kernel fits 4 blocks of 128 threads per SM
    order: int = 1  # 1: longest windows first, 0: as given


class WindowBatch:
    def __init__(self, series: SnapshotSeries, windows: Sequence[WindowSpecRun], *,
                 integrator: str = "rk4", time_mode: str = "blend",
                 snapshot_t0: float = 0.0, snapshot_dt: float = 1.0,
                 schedule: Schedule = Schedule()):
        if series.storage == _lib.F64:
            raise ValueError("batched windows run on the mixed-precision path (fx15/fp16/bf16)")
        self.series = series
        self.windows = list(windows)
        self.kw = dict(integrator=integrator, time_mode=time_mode, snapshot_t0=snapshot_t0,
                       snapshot_dt=snapshot_dt)
        arr = (_lib.FtleWindow * len(self.windows))()
        for i, w in enumerate(self.windows):
            n = w.positions.shape[0] // (2 * series.grid.dim)
            if w.ftle is None:
                w.ftle = torch.empty(n, dtype=torch.float64, device=w.positions.device)
            mp = w.map_period if w.map_period is not None else w.num_steps * abs(w.h)
            arr[i] = window_descriptor(series, w.positions, w.ftle, h=w.h, num_steps=w.num_steps,
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

    def run(self, schedule: Optional[Schedule] = None, stream=None) -> List[torch.Tensor]:
        sch = schedule or self.schedule
        plan = self._plan(sch.order)
        _lib.call("ftle_windows_run_mixed", self.desc, self.count, plan.data_ptr(), plan.numel(),
                  int(sch.ctas_per_sm), stream_ptr(stream))
        return [w.ftle for w in self.windows]

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
                                                     for o in (1, 0)]
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
