"""FTLESolver (mirror of pyFTLE's ``ftle_solver.py``).

``FTLESolver(source, integrator, progress_queue=None, output_writer=None).run()``
integrates one window and returns the FTLE field (or writes it as
``ftle_<id>`` with the initial centroids when a writer is given), like
``ftle_solver.py:56-161``.

Two paths, same results:

* fused -- when the integrator's interpolator is the GPU "grid" one and the
  source can hand over its whole snapshot stack (``window_spec()``), the
  window is one CUDA launch (advection of every particle plus the FTLE
  epilogue, ``ftle_window_run_f64``).  ``options.precision`` "fp16"/"bf16"
  selects the mixed-precision kernel instead.
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
            self.series = SnapshotSeries(spec.grid, spec.snapshots, precision=precision,
                                         periodic_time=spec.periodic_time)
            ftle = run_window(self.series, self.particles.positions,
                              integrator=self.integrator.name, time_mode=spec.time_mode,
                              h=spec.h, num_steps=spec.num_steps, map_period=spec.map_period,
                              t0=spec.t0, first_snapshot=spec.first_snapshot,
                              snapshot_t0=spec.snapshot_t0, snapshot_dt=spec.snapshot_dt,
                              chunk_steps=self.options.chunk_steps,
                              sort_every=self.options.sort_every)
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

    def _compute_ftle(self) -> np.ndarray:
        """FTLE of the current positions with the reference's T = (num_steps - 1)*|dt|."""
        T = (self.source.num_steps - 1) * abs(self.source.timestep)
        return compute_ftle_from_positions(self.particles, T).cpu().numpy()
