"""File I/O around the engine: MATLAB readers, a file-fed BatchSource, writers.

Host-side code (not the hot path), mirroring pyFTLE's ``file_readers.py``,
``data_source.py`` (``FileBatchSource``) and ``file_writers.py``:

* ``read_velocity`` / ``read_coordinate`` -- ``.mat`` keys ``velocity_x/y(/z)`` and
  ``coordinate_x/y(/z)``, each raveled in C order and stacked to ``(dim, N)``
  (file_readers.py:35-118);
* ``read_seed_particles_coordinates`` -- keys ``left, right, top, bottom(, front,
  back)`` concatenated in that order into ``NeighboringParticles``
  (file_readers.py:121-182);
* ``FileBatchSource`` -- the reference's per-step protocol plus ``window_spec()``:
  all snapshot files of a window are read by a thread pool into a fixed ring of
  pinned host buffers (``PinnedRing``) and copied to the device on a side stream
  while later files are still being read, so the fused path receives a
  device-resident stack;
* ``MatWriter`` / ``VTKWriter`` / ``create_writer`` -- ``ftle_<id>.mat`` with keys
  ``ftle, x, y(, z)`` (reshaped to the grid when ``grid_shape`` is given) and VTK
  XML ``.vts`` (structured) / ``.vtp`` (point cloud), written directly
  (file_writers.py:68-302; no pyvista needed).
"""

from __future__ import annotations

import base64
import os
import struct
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path
from typing import List, Optional, Sequence

import numpy as np
import torch
from scipy.io import loadmat, savemat

from pyftle_b200.data_source import WindowSpec
from pyftle_b200.interpolate import GridSpec, Interpolator
from pyftle_b200.particles import NeighboringParticles

# ----------------------------------------------------------------------------
# readers
# ----------------------------------------------------------------------------


def _stack(data: dict, prefix: str, path) -> np.ndarray:
    if f"{prefix}_x" not in data or f"{prefix}_y" not in data:
        raise ValueError(f"The MATLAB file {path} does not contain the expected keys "
                         f"'{prefix}_x' and '{prefix}_y'.")
    comps = [np.asarray(data[f"{prefix}_x"]).ravel(), np.asarray(data[f"{prefix}_y"]).ravel()]
    if f"{prefix}_z" in data:
        comps.append(np.asarray(data[f"{prefix}_z"]).ravel())
    return np.stack(comps).astype(np.float64, copy=False)


# MAT-file level 5 element types and array class used by the direct reader
_MI_INT8, _MI_INT32, _MI_UINT32, _MI_DOUBLE, _MI_MATRIX = 1, 5, 6, 9, 14
_MX_DOUBLE_CLASS = 6


def _mat_parse(raw, names, optional=()) -> Optional[dict]:
    """Locate real double 2D arrays in the bytes of an uncompressed little-endian MAT v5
    file (``raw``: bytes or a memoryview): name -> (byte offset of the data, element
    count, (rows, cols)); the data are the matrix's doubles in MATLAB's column-major
    order, 8-byte aligned.  loadmat returns the same doubles as a (rows, cols) array.
    None when the file uses anything else (compression, big-endian, other classes or
    types, missing names): the caller then reads it with loadmat."""
    n = len(raw)
    if n < 136 or bytes(raw[126:128]) != b"IM":
        return None
    want = set(names)
    every = want | set(optional)
    out = {}

    def sub(p):  # (type, nbytes, data offset, next offset) of a subelement at p
        t, nb = struct.unpack_from("<II", raw, p)
        if t >> 16:  # small data element: 4 bytes of data inside the tag
            return t & 0xFFFF, t >> 16, p + 4, p + 8
        return t, nb, p + 8, p + 8 + ((nb + 7) // 8) * 8

    pos = 128
    try:
        while pos + 8 <= n and every - out.keys():
            t, nb = struct.unpack_from("<II", raw, pos)
            if t >> 16 or t != _MI_MATRIX:
                if t >> 16 or t == 15:  # compressed elements: leave them to loadmat
                    return None
                pos += 8 + ((nb + 7) // 8) * 8
                continue
            end = pos + 8 + nb
            st, snb, sd, p = sub(pos + 8)
            if st != _MI_UINT32 or snb < 8:
                return None
            flags = struct.unpack_from("<I", raw, sd)[0]
            st, snb, sd, p = sub(p)
            if st != _MI_INT32:
                return None
            dims = struct.unpack_from(f"<{snb // 4}i", raw, sd)
            st, snb, sd, p = sub(p)
            if st != _MI_INT8:
                return None
            name = bytes(raw[sd:sd + snb]).decode("ascii", "replace")
            if name in every:
                if (flags & 0xFF) != _MX_DOUBLE_CLASS or flags & 0x800 or len(dims) != 2:
                    return None
                st, snb, sd, p = sub(p)
                count = dims[0] * dims[1]
                if st != _MI_DOUBLE or snb != 8 * count or sd + snb > min(end, n) or sd % 8:
                    return None
                out[name] = (sd, count, (dims[0], dims[1]))
            pos = pos + 8 + ((nb + 7) // 8) * 8
    except (struct.error, ValueError):
        return None
    return out if not (want - out.keys()) else None


def _component_layout(parsed, prefix: str):
    """[(offset, count)] of prefix_x/y(/z) and their common (rows, cols), or None."""
    if parsed is None:
        return None
    comps = [parsed[f"{prefix}_x"], parsed[f"{prefix}_y"]]
    if f"{prefix}_z" in parsed:
        comps.append(parsed[f"{prefix}_z"])
    if any(c[2] != comps[0][2] for c in comps):
        return None
    return [(off, cnt) for off, cnt, _ in comps], comps[0][2]


def _raw_components(file_path, prefix: str):
    """The file's ``prefix_x/y(/z)`` as column-major flat arrays with their common
    (rows, cols), or None (a file the direct reader does not take)."""
    try:
        with open(file_path, "rb") as f:
            raw = f.read()
    except OSError:
        return None
    lay = _component_layout(_mat_parse(raw, [f"{prefix}_x", f"{prefix}_y"], [f"{prefix}_z"]),
                            prefix)
    if lay is None:
        return None
    spans, order = lay
    return [np.frombuffer(raw, dtype="<f8", count=cnt, offset=off) for off, cnt in spans], order


def _read_stack(file_path, prefix: str) -> np.ndarray:
    raw = _raw_components(file_path, prefix)
    if raw is not None:
        arrays, (rows, cols) = raw  # C-order ravel of each (rows, cols) matrix
        return np.stack([a.reshape(cols, rows).T.ravel() for a in arrays])
    return _stack(loadmat(file_path), prefix, file_path)


def read_velocity(file_path) -> np.ndarray:
    return _read_stack(file_path, "velocity")


def read_coordinate(file_path) -> np.ndarray:
    return _read_stack(file_path, "coordinate")


def read_seed_positions(file_path) -> np.ndarray:
    """Role-blocked (K*N, dim) seed positions: left, right, top, bottom(, front, back)."""
    data = loadmat(file_path)
    if any(k not in data for k in ("left", "right", "top", "bottom")):
        raise ValueError("The MATLAB file must contain at least 'left', 'right', 'top' and "
                         "'bottom' keys. ('front' and 'back' for 3D)")
    keys = ["left", "right", "top", "bottom"]
    if "front" in data and "back" in data:
        keys += ["front", "back"]
    return np.concatenate([np.asarray(data[k], dtype=np.float64) for k in keys], axis=0)


def read_seed_particles_coordinates(file_path) -> NeighboringParticles:
    return NeighboringParticles(positions=read_seed_positions(file_path))


# ----------------------------------------------------------------------------
# file-fed source
# ----------------------------------------------------------------------------


class FileBatchSource:
    """One window fed from ``.mat`` files (data_source.py:86-211), HOLD semantics."""

    def __init__(self, snapshot_files: List[str], coordinate_files: List[str],
                 particle_file: str, snapshot_timestep: float, flow_map_period,
                 grid_shape: Optional[tuple] = None, periodic_space: bool = False,
                 workers: int = 8):
        self.snapshot_files = list(snapshot_files)
        self.coordinate_files = list(coordinate_files)
        self.particle_file = particle_file
        self.snapshot_timestep = float(snapshot_timestep)
        self.flow_map_period = flow_map_period
        self._id = Path(self.snapshot_files[0]).stem
        self.reuse_coordinates = len(set(self.coordinate_files)) == 1
        self.grid_shape = tuple(grid_shape) if grid_shape is not None else None
        self.periodic_space = periodic_space
        self.workers = workers

    @property
    def id(self) -> str:
        return self._id

    @property
    def num_steps(self) -> int:
        return len(self.snapshot_files)

    @property
    def timestep(self) -> float:
        return self.snapshot_timestep

    def get_particles(self) -> NeighboringParticles:
        return read_seed_particles_coordinates(self.particle_file)

    def get_data_for_step(self, step_index: int):
        velocities = read_velocity(self.snapshot_files[step_index])
        coordinates = None
        if step_index == 0 or not self.reuse_coordinates:
            coordinates = read_coordinate(self.coordinate_files[step_index])
        return velocities, coordinates

    def update_interpolator(self, interpolator: Interpolator, step_index: int) -> None:
        velocities, coordinates = self.get_data_for_step(step_index)
        interpolator.update(velocities, coordinates)

    def window_spec(self) -> Optional[WindowSpec]:
        """Device-resident snapshot stack for the fused path (None for moving grids)."""
        if not self.reuse_coordinates or self.grid_shape is None:
            return None
        points = read_coordinate(self.coordinate_files[0])
        grid = GridSpec.from_points(points, self.grid_shape, self.periodic_space)
        snaps = load_snapshots(self.snapshot_files, grid.dim, grid.nodes, workers=self.workers)
        n = self.num_steps
        dt = self.snapshot_timestep
        return WindowSpec(grid=grid, snapshots=snaps, time_mode="hold", h=dt, num_steps=n,
                          map_period=(n - 1) * abs(dt), snapshot_dt=dt)


class PinnedRing:
    """A fixed set of pinned host buffers that every snapshot read reuses.

    File number ``ticket`` always lands in slot ``ticket % slots``: ``acquire(ticket)``
    waits until the slot's previous file (``ticket - slots``) has been released and
    its host-to-device copy has completed (the CUDA event given to
    ``release_after``).  Tickets are released in order by the consumer, so readers
    running ahead can never take each other's slots.  Pinning happens once, here,
    not per file.
    """

    def __init__(self, slots: int, shape, dtype=torch.float64):
        import threading

        self.bufs = [torch.empty(shape, dtype=dtype).pin_memory() for _ in range(slots)]
        self._events: List[Optional[torch.cuda.Event]] = [None] * slots
        self._gen = [0] * slots
        self._cv = threading.Condition()
        self._aborted = False

    def acquire(self, ticket: int) -> int:
        n = len(self.bufs)
        slot, want = ticket % n, ticket // n
        with self._cv:
            self._cv.wait_for(lambda: self._aborted or self._gen[slot] == want)
            if self._aborted:
                raise RuntimeError("snapshot reading was aborted")
        ev = self._events[slot]
        if ev is not None:
            ev.synchronize()
        return slot

    def release_after(self, slot: int, event: Optional[torch.cuda.Event]) -> None:
        with self._cv:
            self._events[slot] = event
            self._gen[slot] += 1
            self._cv.notify_all()

    def abort(self) -> None:
        """Wake every reader waiting for a slot with an error (the consumer stopped)."""
        with self._cv:
            self._aborted = True
            self._cv.notify_all()


def snapshot_slot_bytes(files: Sequence[str], dim: int, nodes: int) -> int:
    """Bytes of a ring slot that holds any of ``files`` whole (or their values)."""
    size = dim * nodes * 8
    for f in files:
        try:
            size = max(size, os.path.getsize(f))
        except OSError:
            pass
    return (size + 4095) // 4096 * 4096


def read_velocity_into(path, ring: PinnedRing, ticket: int, dim: int, nodes: int):
    """Read velocity file number ``ticket`` into its slot of ``ring`` (a ring of pinned
    byte buffers).

    Returns (slot, layout).  An uncompressed MAT v5 file is read whole, straight into
    the slot (one readinto, no host-side copy); layout is then ([(byte offset,
    count)] of each component, (rows, cols)) -- the components' column-major doubles
    inside the slot, which ``slot_to_device`` copies and reorders on the device.  Any
    other file goes through loadmat and the slot holds (dim, nodes) float64 values in
    node order at offset 0 (layout None)."""
    slot = ring.acquire(ticket)
    buf = ring.bufs[slot]
    try:
        with open(path, "rb") as f:
            got = f.readinto(memoryview(buf.numpy()))
            whole = f.read(1) == b""
    except OSError:
        got, whole = 0, False
    if whole:
        mv = memoryview(buf.numpy())[:got]
        lay = _component_layout(_mat_parse(mv, ["velocity_x", "velocity_y"], ["velocity_z"]),
                                "velocity")
        if lay is not None and len(lay[0]) == dim and all(c == nodes for _, c in lay[0]):
            return slot, lay
    v = read_velocity(path)
    if v.shape != (dim, nodes):
        raise ValueError(f"{path}: velocity has shape {v.shape}, expected {(dim, nodes)}")
    buf[:dim * nodes * 8].view(torch.float64).numpy()[...] = v.ravel()
    return slot, None


def slot_to_device(slot_buf: torch.Tensor, layout, dim: int, nodes: int, raw: torch.Tensor,
                   out: torch.Tensor, cache: Optional[dict] = None) -> torch.Tensor:
    """Copy a ring slot to the device (current stream) and return it in node order
    (``out``, (dim, nodes) float64; ``raw`` is device scratch of the same shape).

    ``cache`` (a dict the caller keeps) holds the copy plan -- the tensor views of each
    (slot, scratch, output, layout) combination -- so a stream of files with one layout
    builds its views once per ring slot instead of once per file."""
    key = None
    if cache is not None:
        lk = None if layout is None else (tuple(layout[0]), layout[1])
        key = (slot_buf.data_ptr(), raw.data_ptr(), out.data_ptr(), lk)
        plan = cache.get(key)
        if plan is not None:
            for dst, src in plan:
                dst.copy_(src, non_blocking=True)
            return out
    if layout is None:
        plan = [(out, slot_buf[:dim * nodes * 8].view(torch.float64).view(dim, nodes))]
    else:
        spans, order = layout
        plan = [(raw[c], slot_buf[off:off + 8 * cnt].view(torch.float64))
                for c, (off, cnt) in enumerate(spans)]
        if order is None:
            if out.data_ptr() != raw.data_ptr():
                plan.append((out, raw))
        else:
            rows, cols = order
            plan.append((out.view(dim, rows, cols), raw.view(dim, cols, rows).transpose(1, 2)))
    for dst, src in plan:
        dst.copy_(src, non_blocking=True)
    if key is not None:
        cache[key] = plan
    return out


def load_snapshots(files: Sequence[str], dim: int, nodes: int, workers: int = 8,
                   device=None) -> torch.Tensor:
    """Read velocity files in parallel into a (S, dim, nodes) float64 device tensor.

    Files are read by a thread pool into a fixed ring of pinned host buffers
    (``workers + 2`` of them, reused); each is copied to the device on a side stream
    as soon as it is read, overlapping the copies with the remaining reads.
    """
    device = device or torch.device("cuda", torch.cuda.current_device())
    out = torch.empty((len(files), dim, nodes), dtype=torch.float64, device=device)
    if not len(files):
        return out
    copy_stream = torch.cuda.Stream(device=device)
    # `out` comes from the current stream's pool: work still queued there may own
    # its memory until it finishes, so the copies wait for that work first
    copy_stream.wait_stream(torch.cuda.current_stream(device))
    ring = PinnedRing(min(len(files), max(1, workers) + 2),
                      (snapshot_slot_bytes(files, dim, nodes),), dtype=torch.uint8)
    staging = torch.empty((dim, nodes), dtype=torch.float64, device=device)
    with ThreadPoolExecutor(max_workers=max(1, workers)) as pool:
        futures = [pool.submit(read_velocity_into, f, ring, i, dim, nodes)
                   for i, f in enumerate(files)]
        try:
            with torch.cuda.stream(copy_stream):
                for i, fut in enumerate(futures):
                    slot, layout = fut.result()
                    slot_to_device(ring.bufs[slot], layout, dim, nodes, staging, out[i])
                    ev = torch.cuda.Event()
                    ev.record(copy_stream)
                    ring.release_after(slot, ev)
        except BaseException:
            ring.abort()
            for fut in futures:
                fut.cancel()
            raise
    torch.cuda.current_stream(device).wait_stream(copy_stream)
    copy_stream.synchronize()
    return out


# ----------------------------------------------------------------------------
# writers
# ----------------------------------------------------------------------------


class FTLEWriter:
    def __init__(self, directory_path, grid_shape: Optional[tuple] = None) -> None:
        self.path = directory_path
        os.makedirs(self.path, exist_ok=True)
        self.grid_shape = grid_shape
        self.dim: Optional[int] = None

    def write(self, filename: str, ftle_field, particles_centroid) -> None:
        raise NotImplementedError


def _host(a) -> np.ndarray:
    return a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)


class MatWriter(FTLEWriter):
    """``<filename>.mat`` with keys ftle, x, y(, z) (file_writers.py:68-164)."""

    def write(self, filename: str, ftle_field, particles_centroid) -> None:
        ftle_field = _host(ftle_field)
        particles_centroid = _host(particles_centroid)
        if self.dim is None:
            self.dim = particles_centroid.shape[1]
        out = os.path.join(self.path, filename + ".mat")
        if self.grid_shape:
            if len(self.grid_shape) == 2:
                nx, ny = self.grid_shape
                nz = 1
            elif len(self.grid_shape) == 3:
                nx, ny, nz = self.grid_shape
            else:
                raise ValueError(
                    f"Invalid grid_shape length {len(self.grid_shape)}. Must be 2 or 3.")
            f = ftle_field.reshape(nx, ny, nz)
            c = particles_centroid.reshape(nx, ny, nz, self.dim)
            data = {"ftle": f, "x": c[..., 0], "y": c[..., 1]}
            if self.dim == 3:
                data["z"] = c[..., 2]
        else:
            data = {"ftle": ftle_field.ravel(), "x": particles_centroid[:, 0],
                    "y": particles_centroid[:, 1]}
            if self.dim == 3:
                data["z"] = particles_centroid[:, 2]
        savemat(out, data)


def _b64(arr: np.ndarray) -> str:
    raw = np.ascontiguousarray(arr).tobytes()
    return base64.b64encode(struct.pack("<Q", len(raw)) + raw).decode("ascii")


def _vtk_header(kind: str) -> str:
    return (f'<?xml version="1.0"?>\n<VTKFile type="{kind}" version="1.0" '
            f'byte_order="LittleEndian" header_type="UInt64">\n')


class VTKWriter(FTLEWriter):
    """VTK XML ``.vts`` (structured grid) or ``.vtp`` (points) (file_writers.py:167-266).

    Point and cell-free layouts follow the reference: 2D structured points are
    arranged in Fortran order with z = 0; 3D FTLE values are transposed to the
    (y, x, z) cartesian order before the Fortran ravel.
    """

    def write(self, filename: str, ftle_field, particles_centroid) -> None:
        ftle_field = _host(ftle_field).astype(np.float64)
        pc = _host(particles_centroid).astype(np.float64)
        if self.dim is None:
            self.dim = pc.shape[1]
        base = os.path.join(self.path, filename)
        if self.grid_shape is not None:
            if len(self.grid_shape) == 2:
                nx, ny = self.grid_shape
                nz = 1
                c = pc.reshape(nx, ny, nz, self.dim, order="F")
                x, y = c[..., 0], c[..., 1]
                z = np.zeros_like(x)
                values = ftle_field.ravel(order="F")
            elif len(self.grid_shape) == 3:
                nx, ny, nz = self.grid_shape
                c = pc.reshape(nx, ny, nz, self.dim)
                x, y, z = c[..., 0], c[..., 1], c[..., 2]
                values = np.transpose(ftle_field.reshape((nx, ny, nz)), (1, 0, 2)).ravel(order="F")
            else:
                raise ValueError(
                    f"Invalid grid_shape length {len(self.grid_shape)}. Must be 2 or 3.")
            pts = np.stack([x.ravel(order="F"), y.ravel(order="F"), z.ravel(order="F")], axis=1)
            ext = f"0 {x.shape[0] - 1} 0 {x.shape[1] - 1} 0 {x.shape[2] - 1}"
            with open(base + ".vts", "w") as f:
                f.write(_vtk_header("StructuredGrid"))
                f.write(f'<StructuredGrid WholeExtent="{ext}">\n<Piece Extent="{ext}">\n')
                f.write('<PointData Scalars="ftle">\n<DataArray type="Float64" Name="ftle" '
                        f'format="binary">{_b64(values)}</DataArray>\n</PointData>\n')
                f.write('<Points>\n<DataArray type="Float64" NumberOfComponents="3" '
                        f'format="binary">{_b64(pts)}</DataArray>\n</Points>\n')
                f.write("</Piece>\n</StructuredGrid>\n</VTKFile>\n")
        else:
            pts = np.hstack([pc, np.zeros((pc.shape[0], 1))]) if self.dim == 2 else pc
            n = pts.shape[0]
            conn = np.arange(n, dtype=np.int64)
            with open(base + ".vtp", "w") as f:
                f.write(_vtk_header("PolyData"))
                f.write(f'<PolyData>\n<Piece NumberOfPoints="{n}" NumberOfVerts="{n}" '
                        'NumberOfLines="0" NumberOfStrips="0" NumberOfPolys="0">\n')
                f.write('<PointData Scalars="ftle">\n<DataArray type="Float64" Name="ftle" '
                        f'format="binary">{_b64(ftle_field.ravel())}</DataArray>\n</PointData>\n')
                f.write('<Points>\n<DataArray type="Float64" NumberOfComponents="3" '
                        f'format="binary">{_b64(pts)}</DataArray>\n</Points>\n')
                f.write('<Verts>\n<DataArray type="Int64" Name="connectivity" format="binary">'
                        f'{_b64(conn)}</DataArray>\n<DataArray type="Int64" Name="offsets" '
                        f'format="binary">{_b64(conn + 1)}</DataArray>\n</Verts>\n')
                f.write("</Piece>\n</PolyData>\n</VTKFile>\n")


def create_writer(output_format: str, directory_path: str,
                  grid_shape: Optional[tuple] = None) -> FTLEWriter:
    if output_format == "mat":
        return MatWriter(directory_path, grid_shape)
    if output_format == "vtk":
        return VTKWriter(directory_path, grid_shape)
    raise ValueError(f"Unsupported output format: {output_format}")


def read_vtk_xml(path: str) -> dict:
    """Decode the binary DataArrays of a file written by VTKWriter (for checks)."""
    import re

    text = open(path).read()
    out = {}
    for m in re.finditer(r'<DataArray type="(\w+)"([^>]*)format="binary">([^<]*)</DataArray>',
                         text):
        typ, attrs, payload = m.group(1), m.group(2), m.group(3)
        name = re.search(r'Name="(\w+)"', attrs)
        ncomp = re.search(r'NumberOfComponents="(\d+)"', attrs)
        raw = base64.b64decode(payload)
        n = struct.unpack("<Q", raw[:8])[0]
        arr = np.frombuffer(raw[8:8 + n], dtype={"Float64": np.float64, "Int64": np.int64}[typ])
        if ncomp:
            arr = arr.reshape(-1, int(ncomp.group(1)))
        out[name.group(1) if name else "points"] = arr
    return out
