"""Sliding FTLE windows over one resident snapshot series.

Replaces the reference's window driver (``MultipleFTLEProcessManager``,
``__main__.py:18-207``): with n snapshot files and a flow-map period T, the window
length is p = int(T/|dt|) + 1 and there are n - p + 1 overlapping windows
(``__main__.py:111-166``); negative dt reverses the file lists
(``__main__.py:91-109``); window i uses particle file i (cycled) and is named
after its first snapshot file.  The reference runs each window in its own
process and re-reads its p snapshot files; here each snapshot is read once.
On the FP64 path (the default, streaming) the files are read by a thread pool
into a fixed ring of pinned buffers and copied and packed into a device ring of
p + 2 snapshots while the previous window's kernel runs, one launch per window
as soon as its snapshots are in place.  On the mixed path all n snapshots are
read (in parallel, copied to the device while reading), packed once (FX15 needs
the whole series' value range), and every window runs in one persistent launch.
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


# device memory the head windows' position blocks may take (see _run_streaming)
HEAD_BYTES = 1 << 30


class SlidingWindowRunner:
    def __init__(self, snapshot_files: List[str], coordinate_files: List[str],
                 particle_files: List[str], snapshot_timestep: float, flow_map_period: float,
                 grid_shape: tuple, integrator_name: str = "rk4", writer=None,
                 precision: str = "fp64", periodic_space: bool = False, workers: int = 4,
                 streaming: bool = True, device_depth: int = 2,
                 head_per_step: bool = True, head_windows: Optional[int] = None):
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
        self.streaming = bool(streaming)
        self.device_depth = max(1, int(device_depth))
        self.head_per_step = bool(head_per_step)
        self.head_windows = head_windows
        self.stats: dict = {}
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
        if self.precision == "fp64" and self.streaming:
            return self._run_streaming(wins, grid)
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

    def _run_streaming(self, wins, grid):
        """FP64 windows fed while they run (fixed grid, the reference's HOLD windows).

        Snapshot files are read by a thread pool into a fixed ring of pinned host
        buffers (``io.PinnedRing``), copied to the device on a side stream and packed
        into a device ring of ``p + device_depth`` snapshot blocks, which the kernel
        addresses modulo the ring length (``periodic_time`` with ``first_snapshot`` =
        window index mod ring length; HOLD reads one snapshot per step).  Window i is
        launched as soon as its p snapshots are packed, reading its particle file's
        seeds without writing them; the read, copy and packing of snapshot i + p
        (needed by window i + 1) then run while window i's kernel runs, and a ring block
        is overwritten only after the last window reading it finished.  Up to DEPTH
        windows are in flight: each window's FTLE goes back to host memory on a stream
        of its own (one pinned array for all windows when no writer is given) and is
        emitted while the next windows run.

        With ``head_per_step`` the first windows -- ``head_windows`` of them (default
        (p + 1) // 2), at most the p that start before window 0's last file arrives,
        only while they share window 0's particle file, and no more than fit their
        positions in ``HEAD_BYTES`` (at least one) -- do not wait for their p files:
        when snapshot j arrives, every such window w with w <= j < w + p takes its step
        j - w, all of them on snapshot j (HOLD), in one ``ftle_grid_step`` launch over
        their adjacent position blocks, and a window's FTLE is taken from its final
        positions (``ftle_from_positions``): the fused kernel's bits (same step
        arithmetic, same FTLE device function), with the GPU busy while the first files
        are still being read.  Device memory holds p + device_depth snapshots instead of
        all n.
        """
        import time
        from concurrent.futures import ThreadPoolExecutor

        from pyftle_b200 import _lib
        from pyftle_b200._device import stream_ptr
        from pyftle_b200.window import window_descriptor

        t_start = time.perf_counter()
        dim, nodes = grid.dim, grid.nodes
        n = len(self.snapshot_files)
        p = self.window_length
        W = len(wins)
        dt = self.timestep
        dev = torch.device("cuda", torch.cuda.current_device())
        block = int(_lib.load().ftle_packed_snapshot_bytes(dim, nodes, 1, _lib.F64))
        R = min(n, p + self.device_depth)
        ring_dev = torch.empty(R * block, dtype=torch.uint8, device=dev)
        raw = [torch.empty((dim, nodes), dtype=torch.float64, device=dev) for _ in range(2)]
        # node-ordered snapshots: packed from, and read by the first window's steps
        node_bufs = [torch.empty((dim, nodes), dtype=torch.float64, device=dev)
                     for _ in range(2)]
        node_used: List[Optional[torch.cuda.Event]] = [None, None]
        ev_node = [torch.cuda.Event(), torch.cuda.Event()]
        series = _RingSeries(grid, ring_dev, R)
        comp = torch.cuda.current_stream(dev)
        copy = torch.cuda.Stream(device=dev)
        copy.wait_stream(comp)
        host = io.PinnedRing(min(n, self.workers + 2),
                             (io.snapshot_slot_bytes(self.snapshot_files, dim, nodes),),
                             dtype=torch.uint8)
        packed: List[Optional[torch.cuda.Event]] = [None] * n
        done: List[Optional[torch.cuda.Event]] = [None] * W
        seeds = {}
        for _, pf, _, _ in wins:
            if pf not in seeds:
                seeds[pf] = io.read_seed_particles_coordinates(pf)
        N = {pf: len(part) for pf, part in seeds.items()}
        # windows in flight: window i's FTLE is emitted while windows up to i + DEPTH - 1
        # are queued, so host work never leaves the GPU idle between windows
        DEPTH = 4
        nmax = max(N.values())
        # fields returned in memory land straight in one pinned result array (no per-window
        # host copy); with a writer, or a result too large to pin, a ring of DEPTH buffers
        results = None
        if self.writer is None and W * nmax * 8 <= (2 << 30):
            results = torch.empty((W, nmax), dtype=torch.float64, pin_memory=True)
        out_pin = [torch.empty(nmax, dtype=torch.float64, pin_memory=True)
                   for _ in range(DEPTH)] if results is None else None
        out_ev: List[Optional[torch.cuda.Event]] = [None] * DEPTH
        ftle_dev = [torch.empty(nmax, dtype=torch.float64, device=dev) for _ in range(DEPTH)]
        # events made once and reused by window i % DEPTH: a slot is recorded again only
        # after its previous window was emitted (its kernel time read there)
        kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(DEPTH)]
        oev = [torch.cuda.Event() for _ in range(DEPTH)]
        ev_ftle = [torch.cuda.Event() for _ in range(DEPTH)]
        fused = [0, 0.0]  # windows timed, their kernel milliseconds
        descs = {}  # one window descriptor per particle file, re-pointed per window
        plans = {}  # host slot -> device copy plans (io.slot_to_device)

        def host_out(i, n):
            return results[i, :n] if results is not None else out_pin[i % DEPTH][:n]

        # FTLE fields go back on a stream of their own, so the compute stream runs window
        # after window without the copies between them
        back = torch.cuda.Stream(device=dev)

        def fetch(i, f, after):
            """Window i's FTLE `f` to host memory once `after` (an event on the compute
            stream) has passed; out_ev[i % DEPTH] marks the copy's end."""
            back.wait_event(after)
            with torch.cuda.stream(back):
                host_out(i, f.shape[0]).copy_(f, non_blocking=True)
            oev[i % DEPTH].record(back)
            out_ev[i % DEPTH] = oev[i % DEPTH]
        fields = []

        pool = ThreadPoolExecutor(max_workers=max(1, self.workers))
        futures = [pool.submit(io.read_velocity_into, f, host, j, dim, nodes)
                   for j, f in enumerate(self.snapshot_files)]

        def stage(j):
            slot, layout = futures[j].result()
            with torch.cuda.stream(copy):
                prev = j - R  # the snapshot that last used ring block j % R
                last = min(prev, W - 1)  # the last window that read it from the ring
                if prev >= 0 and done[last] is not None:  # (head windows do not read it)
                    copy.wait_event(done[last])
                nb = node_bufs[j % 2]
                if node_used[j % 2] is not None:  # a step of the first window still reads it
                    copy.wait_event(node_used[j % 2])
                # the file's data ranges to the device, reordered there into node order
                buf = io.slot_to_device(host.bufs[slot], layout, dim, nodes, raw[j % 2], nb,
                                        cache=plans)
                _lib.call("ftle_pack_snapshots", dim, nodes, 1, 0, buf.data_ptr(), _lib.F64,
                          ring_dev.data_ptr() + (j % R) * block, stream_ptr(copy))
                e = torch.cuda.Event()
                e.record(copy)  # the slot's copy and the packing are done
                host.release_after(slot, e)
                packed[j] = e

        def emit(i):
            _, pf, _, ident = wins[i]
            out_ev[i % DEPTH].synchronize()
            if i >= start:  # a fused window: its kernel time, before the events are reused
                k0, k1 = kev[i % DEPTH]
                fused[0] += 1
                fused[1] += k0.elapsed_time(k1)
            arr = host_out(i, N[pf]).numpy()
            if results is None:
                arr = arr.copy()  # the ring slot is reused
            if self.writer is not None:
                self.writer.write(f"ftle_{ident}", arr,
                                  seeds[pf].initial_centroid.cpu().numpy())
            else:
                fields.append(arr)

        # head windows: a prefix of windows sharing window 0's particle file, at most
        # head_windows (default: half a window length, which balances the per-step
        # work against the reading of the first files), and no more than keep their
        # positions (and AB2 histories) within HEAD_BYTES of device memory
        H = 0
        if self.head_per_step and p <= n:
            cap = (p + 1) // 2 if self.head_windows is None else int(self.head_windows)
            per = seeds[wins[0][1]].positions.numel() * 8 * (2 if self.integrator == "ab2" else 1)
            cap = max(1, min(W, p, cap, HEAD_BYTES // max(per, 1)))
            while H < cap and wins[H][1] == wins[0][1]:
                H += 1

        def head_windows_by_steps():
            """Windows 0 .. H-1 advanced one launch per arriving snapshot (see above)."""
            _, pf, _, _ = wins[0]
            part = seeds[pf]
            m = part.positions.shape[0]  # particles per window
            big = torch.empty((H,) + tuple(part.positions.shape), dtype=torch.float64,
                              device=dev)
            code = _lib.INTEGRATOR_CODES[self.integrator]
            hist = torch.empty_like(big) if self.integrator == "ab2" else None
            idl = part.initial_deltas()
            T = float((p - 1) * abs(dt))
            gabi = grid.to_abi()
            sp = stream_ptr(comp)

            def step(lo, hi, j, valid):  # windows lo..hi take their step on snapshot j
                _lib.call("ftle_grid_step", gabi, node_bufs[j % 2].data_ptr(), code, float(dt),
                          big[lo].data_ptr(), (hi - lo + 1) * m,
                          hist[lo].data_ptr() if hist is not None else None, int(valid), sp)

            for j in range(H + p - 1):
                stage(j)
                comp.wait_event(packed[j])
                lo, hi = max(0, j - p + 1), min(j, H - 1)
                if j < H:  # window j starts: its seeds, then its first step
                    big[j].copy_(part.positions)
                    if hist is not None:
                        step(j, j, j, False)  # AB2's first step is Euler
                        hi = j - 1
                if lo <= hi:
                    step(lo, hi, j, True)
                node_used[j % 2] = ev_node[j % 2]
                ev_node[j % 2].record(comp)
                w = j - p + 1  # the window whose last snapshot is j
                if w >= 0:
                    f = ftle_dev[w % DEPTH][:N[pf]]
                    _lib.call("ftle_from_positions", dim, big[w].data_ptr(), idl.data_ptr(),
                              N[pf], T, f.data_ptr(), sp)
                    ev_ftle[w % DEPTH].record(comp)
                    fetch(w, f, ev_ftle[w % DEPTH])
                    if w >= DEPTH - 1:
                        emit(w - (DEPTH - 1))

        start = H
        try:
            if start:
                head_windows_by_steps()
                if H + p - 1 < n:
                    stage(H + p - 1)  # the last snapshot of window H
            else:
                for j in range(min(p, n)):
                    stage(j)
            t_first = time.perf_counter()
            sp = stream_ptr(comp)
            for i in range(start, W):
                _, pf, _, _ = wins[i]
                comp.wait_event(packed[i + p - 1])  # in order: every earlier block is packed too
                f = ftle_dev[i % DEPTH][:N[pf]]
                w = descs.get(pf)
                if w is None:  # the seeds are read, never written (no per-window copy)
                    w = descs[pf] = window_descriptor(
                        series, seeds[pf].positions, f, integrator=self.integrator,
                        time_mode="hold", h=dt, num_steps=p, map_period=(p - 1) * abs(dt),
                        first_snapshot=i % R, snapshot_dt=dt, keep_positions=True)
                w.first_snapshot = i % R
                w.ftle = f.data_ptr()
                k0, k1 = kev[i % DEPTH]
                k0.record(comp)
                _lib.call("ftle_window_run_f64", w, sp)
                k1.record(comp)
                done[i] = k1
                fetch(i, f, k1)
                if i + p < n:
                    stage(i + p)  # overlaps the windows in flight
                if i >= DEPTH - 1:
                    emit(i - (DEPTH - 1))
            for i in range(max(0, W - (DEPTH - 1)), W):
                emit(i)
        except BaseException:
            host.abort()
            for fut in futures:
                fut.cancel()
            raise
        finally:
            pool.shutdown(wait=True)
        torch.cuda.synchronize()
        nf, fused_ms = fused
        self.stats = {"seconds": time.perf_counter() - t_start,
                      "head_s": t_first - t_start, "head_windows": H,
                      "fused_windows": nf, "fused_kernel_ms": fused_ms,
                      # every window's kernel time, the first one counted at the fused rate
                      "kernel_ms": fused_ms * W / nf if nf else 0.0,
                      "windows": W, "device_ring_snapshots": R,
                      "host_ring_buffers": len(host.bufs)}
        return None if self.writer is not None else fields

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


class _RingSeries:
    """A device ring of FP64 snapshot blocks seen through the SnapshotSeries fields that
    ``window_descriptor`` reads (time-periodic, so snapshot indices wrap at its length)."""

    def __init__(self, grid: GridSpec, packed: torch.Tensor, length: int):
        from pyftle_b200 import _lib

        self.grid = grid
        self.packed = packed
        self.num_snapshots = int(length)
        self.storage = _lib.F64
        self.precision = "fp64"
        self.periodic_time = True
