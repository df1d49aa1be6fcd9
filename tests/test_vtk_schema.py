"""VTK XML output checked by an XML parser against the VTK file-format rules (no GPU).

The writer's own decoder (``io.read_vtk_xml``) is not used here.  The files are
parsed with ``xml.etree`` and checked against the rules of VTK's XML formats for
uncompressed binary data: the root element and its attributes, the structured
grid's extents and the number of points they imply, base64 payloads that decode
strictly and start with a UInt64 byte count equal to the payload length, array
lengths matching points x components, a PointData ``Scalars`` name that exists,
and for PolyData vertex cells whose connectivity indexes existing points and whose
offsets are increasing and end at the connectivity length.
"""

import base64
import struct
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from pyftle_b200 import io

TYPES = {"Float64": np.float64, "Float32": np.float32, "Int64": np.int64, "Int32": np.int32,
         "UInt64": np.uint64, "UInt8": np.uint8}


def _array(el, count_expected=None):
    """Decode one <DataArray format="binary"> by the VTK rules (header_type UInt64)."""
    assert el.tag == "DataArray"
    assert el.get("format") == "binary"
    dtype = np.dtype(TYPES[el.get("type")])
    raw = base64.b64decode((el.text or "").strip(), validate=True)
    assert len(raw) >= 8
    (nbytes,) = struct.unpack("<Q", raw[:8])
    assert nbytes == len(raw) - 8, "UInt64 header must give the payload length"
    assert nbytes % dtype.itemsize == 0
    arr = np.frombuffer(raw[8:], dtype=dtype.newbyteorder("<"))
    ncomp = int(el.get("NumberOfComponents", "1"))
    assert arr.size % ncomp == 0
    if count_expected is not None:
        assert arr.size == count_expected * ncomp, (el.get("Name"), arr.size, count_expected)
    return arr.reshape(-1, ncomp) if ncomp > 1 else arr


def _root(path, kind):
    tree = ET.parse(path)
    root = tree.getroot()
    assert root.tag == "VTKFile"
    assert root.get("type") == kind
    assert root.get("byte_order") == "LittleEndian"
    assert root.get("header_type") == "UInt64"
    assert root.get("version") in ("0.1", "1.0", "2.0", "2.2")
    assert root.get("compressor") is None  # uncompressed payloads
    children = list(root)
    assert len(children) == 1 and children[0].tag == kind
    return children[0]


def _point_data(piece, npts):
    pd = piece.find("PointData")
    assert pd is not None
    arrays = {a.get("Name"): _array(a, npts) for a in pd.findall("DataArray")}
    assert pd.get("Scalars") in arrays
    return arrays


def check_vts(path):
    grid = _root(path, "StructuredGrid")
    whole = [int(v) for v in grid.get("WholeExtent").split()]
    assert len(whole) == 6
    pieces = grid.findall("Piece")
    assert len(pieces) == 1
    piece = pieces[0]
    ext = [int(v) for v in piece.get("Extent").split()]
    assert ext == whole
    dims = [ext[2 * a + 1] - ext[2 * a] + 1 for a in range(3)]
    assert all(d >= 1 for d in dims)
    npts = int(np.prod(dims))
    data = _point_data(piece, npts)
    pts_el = piece.find("Points")
    assert pts_el is not None and len(pts_el.findall("DataArray")) == 1
    da = pts_el.find("DataArray")
    assert da.get("NumberOfComponents") == "3"
    pts = _array(da, npts)
    return dims, pts, data


def check_vtp(path):
    poly = _root(path, "PolyData")
    piece = poly.find("Piece")
    npts = int(piece.get("NumberOfPoints"))
    nverts = int(piece.get("NumberOfVerts"))
    for k in ("NumberOfLines", "NumberOfStrips", "NumberOfPolys"):
        assert int(piece.get(k, "0")) == 0
    data = _point_data(piece, npts)
    pts = _array(piece.find("Points").find("DataArray"), npts)
    verts = {a.get("Name"): a for a in piece.find("Verts").findall("DataArray")}
    conn = _array(verts["connectivity"])
    offs = _array(verts["offsets"], nverts)
    assert np.all(np.diff(offs) > 0) and offs[0] > 0 and offs[-1] == conn.size
    assert conn.min() >= 0 and conn.max() < npts
    return pts, data, conn, offs


def test_vts_2d_structured_follows_vtk_rules(tmp_path):
    nx, ny = 5, 3
    w = io.create_writer("vtk", str(tmp_path), grid_shape=(nx, ny))
    X, Y = np.meshgrid(np.linspace(0, 2, nx), np.linspace(0, 1, ny), indexing="ij")
    cents = np.stack([X.ravel(order="F"), Y.ravel(order="F")], axis=1)
    ftle = np.random.default_rng(1).random(nx * ny)
    w.write("f2", ftle, cents)
    dims, pts, data = check_vts(tmp_path / "f2.vts")
    assert dims == [nx, ny, 1]
    # point (i, j) sits at index i + nx*j; x grows with i, y with j, z = 0
    P = pts.reshape(ny, nx, 3)
    assert np.all(np.diff(P[:, :, 0], axis=1) > 0) and np.all(np.diff(P[:, :, 1], axis=0) > 0)
    assert np.all(P[:, :, 2] == 0)
    np.testing.assert_array_equal(data["ftle"], ftle)


def test_vts_3d_structured_follows_vtk_rules(tmp_path):
    nx, ny, nz = 4, 3, 2
    w = io.create_writer("vtk", str(tmp_path), grid_shape=(nx, ny, nz))
    X, Y, Z = np.meshgrid(np.arange(nx) * 1.0, np.arange(ny) * 10.0, np.arange(nz) * 100.0,
                          indexing="ij")
    cents = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    ftle = np.arange(nx * ny * nz, dtype=np.float64)
    w.write("f3", ftle, cents)
    dims, pts, data = check_vts(tmp_path / "f3.vts")
    assert dims == [nx, ny, nz]
    P = pts.reshape(nz, ny, nx, 3)  # VTK order: i fastest, then j, then k
    assert np.all(np.diff(P[..., 0], axis=2) > 0)
    assert np.all(np.diff(P[..., 1], axis=1) > 0)
    assert np.all(np.diff(P[..., 2], axis=0) > 0)
    assert data["ftle"].shape == (nx * ny * nz,)
    np.testing.assert_array_equal(np.sort(data["ftle"]), ftle)


@pytest.mark.parametrize("dim", [2, 3])
def test_vtp_points_follow_vtk_rules(tmp_path, dim):
    w = io.create_writer("vtk", str(tmp_path))
    n = 7
    cents = np.random.default_rng(dim).random((n, dim))
    ftle = np.linspace(-1, 1, n)
    w.write("p", ftle, cents)
    pts, data, conn, offs = check_vtp(tmp_path / "p.vtp")
    np.testing.assert_array_equal(pts[:, :dim], cents)
    if dim == 2:
        assert np.all(pts[:, 2] == 0)
    np.testing.assert_array_equal(data["ftle"], ftle)
    np.testing.assert_array_equal(conn, np.arange(n))
    np.testing.assert_array_equal(offs, np.arange(1, n + 1))
