"""FTLESolver (mirror of pyFTLE's ``ftle_solver.py``).

``FTLESolver(source, integrator, progress_queue=None, output_writer=None).run()``
integrates one window and returns the FTLE field (or writes it as
``ftle_<id>`` with the initial centroids when a writer is given), like
``ftle_solver.py:56-161``.

Two paths, same results:

* fused -- when the integrator's interpolator is the GPU "grid" one and the
  source can hand over its whole snapshot stack (``window_spec()``), the
  window is one CUDA launch (advection of every particle plus the FTLE
  epilogue, ``ftle_window_run_f64``).  ``options.precision`` "fx16" / "fx15" /
  "fp16" / "bf16" selects the mixed-precision kernel instead; with
  ``options.judge_tol`` the plain FP64 kernel judges that window on a sample of
  its groups and re-advects it when the sampled FTLE error exceeds the tolerance
  (``self.judge`` holds the outcome).
* per-step -- otherwise the reference loop runs as written:
  ``update_interpolator(i)`` then ``integrator.integrate(timestep)`` per step
  (each a CUDA launch), then the fused FTLE kernel with
  T = (num_steps - 1)*|timestep| (ftle_solver.py:151-161).

``run()`` returns a numpy array like the reference; ``run_device()`` returns
the torch CUDA tensor.
"""

from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from pyftle_b200.data_source import BatchSource
from pyftle_b200.ftle import compute_ftle_from_positions
from pyftle_b200.integrate import Integrator
from pyftle_b200.interpolate import HighPerfInterpolator
from pyftle_b200.window import EngineOptions, SnapshotSeries, run_window


class FTLESolver:
    def __init__(self, source: BatchSource, integrator: Integrator, progress_queue=None,
                 output_writer=None, options: Optional[EngineOptions] = None):
        self.source = source
        self.integrator = integrator
        self.progress_queue = progress_queue
        self.output_writer = output_writer
        self.options = options or EngineOptions()
        self.particles = None
        self.series: Optional[SnapshotSeries] = None
        self.judge: Optional[dict] = None

    # ------------------------------------------------------------------
    def _fused_ok(self) -> bool:
        return isinstance(self.integrator.interpolator, HighPerfInterpolator) and hasattr(
            self.source, "window_spec")

    def run_device(self) -> torch.Tensor:
        self.particles = self.source.get_particles()
        ident = self.source.id
        spec = self.source.window_spec() if self._fused_ok() else None
        if spec is not None:
            precision = self.options.precision
            judge = self.options.judge_tol is not None and precision != "fp64"
            self.series = SnapshotSeries(spec.grid, spec.snapshots, precision=precision,
                                         periodic_time=spec.periodic_time, keep_source=judge)
            win = dict(integrator=self.integrator.name, time_mode=spec.time_mode, h=spec.h,
                       num_steps=spec.num_steps, map_period=spec.map_period, t0=spec.t0,
                       first_snapshot=spec.first_snapshot, snapshot_t0=spec.snapshot_t0,
                       snapshot_dt=spec.snapshot_dt)
            seeds = self.particles.positions.clone() if judge else None
            ftle = run_window(self.series, self.particles.positions,
                              chunk_steps=self.options.chunk_steps,
                              sort_every=self.options.sort_every, **win)
            if judge:
                ftle = self._judge(ftle, seeds, spec, win)
            if self.progress_queue:
                for i in range(spec.num_steps):
                    self.progress_queue.put((ident, i))
        else:
            if self.options.precision != "fp64":
                raise ValueError("mixed precision needs the fused path (grid interpolator and a "
                                 "source with window_spec())")
            self.integrator.reset()
            timestep = self.source.timestep
            num_steps = self.source.num_steps
            for i in range(num_steps):
                self.source.update_interpolator(self.integrator.interpolator, i)
                self.integrator.integrate(timestep, self.particles)
                if self.progress_queue:
                    self.progress_queue.put((ident, i))
            ftle = compute_ftle_from_positions(self.particles, (num_steps - 1) * abs(timestep))
        if self.progress_queue:
            self.progress_queue.put((ident, "done"))
        return ftle

    def run(self):
        ftle = self.run_device()
        # back through pinned memory (torch's host allocator reuses the block; the
        # returned array keeps it alive): ~50 GB/s instead of a pageable copy's few GB/s
        host = torch.empty(ftle.shape, dtype=ftle.dtype, pin_memory=True)
        host.copy_(ftle, non_blocking=True)
        torch.cuda.current_stream(ftle.device).synchronize()
        field = host.numpy()
        if self.output_writer is not None:
            self.output_writer.write(f"ftle_{self.source.id}", field,
                                     self.particles.initial_centroid.cpu().numpy())
            return None
        return field

    def _judge(self, ftle: torch.Tensor, seeds: torch.Tensor, spec, win) -> torch.Tensor:
        """FP64 judge of a mixed-precision window: the plain FP64 kernel advects every
        ``judge_stride``-th group of the window's seeds; if the sampled FTLE's relative
        L2 error exceeds ``judge_tol`` (or is not finite), the whole window is re-advected
        by the plain FP64 kernel (FTLE and final positions become the FP64 ones).  The
        outcome is left in ``self.judge``."""
        opts = self.options
        stride = max(1, int(opts.judge_stride))
        K = 2 * spec.grid.dim
        n = seeds.shape[0] // K
        sel = torch.arange(0, n, stride, device=seeds.device)
        sub = seeds.view(K, n, spec.grid.dim)[:, sel, :].reshape(-1, spec.grid.dim).contiguous()
        series64 = SnapshotSeries(spec.grid, self.series.source, precision="fp64",
                                  periodic_time=spec.periodic_time)
        self.series.source = None
        f64 = run_window(series64, sub, **win)
        ref = torch.linalg.vector_norm(f64)
        diff = torch.linalg.vector_norm(ftle[sel] - f64)
        err = float(diff / ref) if float(ref) > 0 else float(diff)
        redo = not err <= opts.judge_tol
        if redo:
            ftle = run_window(series64, seeds, **win)
            self.particles.positions.copy_(seeds)
        self.judge = {"error": err, "tol": float(opts.judge_tol), "readvected": redo,
                      "sample_groups": int(sel.numel())}
        return ftle

    def _compute_ftle(self) -> np.ndarray:
        """FTLE of the current positions with the reference's T = (num_steps - 1)*|dt|."""
        T = (self.source.num_steps - 1) * abs(self.source.timestep)
        return compute_ftle_from_positions(self.particles, T).cpu().numpy()
