"""File formats on the host (no GPU): readers and writers mirror pyFTLE's keys,
orders and shapes (file_readers.py, file_writers.py)."""

import numpy as np
import pytest
from scipy.io import loadmat, savemat

from pyftle_b200 import io


def test_read_velocity_and_coordinate(tmp_path):
    savemat(tmp_path / "v2.mat", {"velocity_x": np.array([1.0, 2.0, 3.0]),
                                  "velocity_y": np.array([4.0, 5.0, 6.0])})
    v = io.read_velocity(tmp_path / "v2.mat")
    np.testing.assert_array_equal(v, [[1, 2, 3], [4, 5, 6]])
    savemat(tmp_path / "c3.mat", {"coordinate_x": np.arange(6.0).reshape(2, 3),
                                  "coordinate_y": np.ones((2, 3)),
                                  "coordinate_z": np.zeros((2, 3))})
    c = io.read_coordinate(tmp_path / "c3.mat")
    assert c.shape == (3, 6)
    np.testing.assert_array_equal(c[0], np.arange(6.0))  # C-order ravel
    savemat(tmp_path / "bad.mat", {"velocity_x": np.zeros(3)})
    with pytest.raises(ValueError):
        io.read_velocity(tmp_path / "bad.mat")


def test_seed_positions_concatenation_order(tmp_path):
    d = {"top": [[1.0, 2.0], [3.0, 4.0]], "bottom": [[5.0, 6.0], [7.0, 8.0]],
         "left": [[9.0, 10.0], [11.0, 12.0]], "right": [[13.0, 14.0], [15.0, 16.0]]}
    savemat(tmp_path / "s2.mat", d)
    p = io.read_seed_positions(tmp_path / "s2.mat")
    np.testing.assert_array_equal(p, np.concatenate([d["left"], d["right"], d["top"],
                                                     d["bottom"]]))
    d3 = {k: np.arange(6.0).reshape(2, 3) + i for i, k in
          enumerate(["top", "bottom", "left", "right", "front", "back"])}
    savemat(tmp_path / "s3.mat", d3)
    p3 = io.read_seed_positions(tmp_path / "s3.mat")
    assert p3.shape == (12, 3)
    np.testing.assert_array_equal(p3[8:10], d3["front"])
    with pytest.raises(ValueError):
        savemat(tmp_path / "bad.mat", {"top": [[1.0, 2.0]]})
        io.read_seed_positions(tmp_path / "bad.mat")


def test_mat_writer_structured_and_unstructured(tmp_path):
    w = io.create_writer("mat", str(tmp_path / "out"), grid_shape=(3, 2))
    ftle = np.arange(6.0)
    cents = np.stack([np.arange(6.0), -np.arange(6.0)], axis=1)
    w.write("ftle_a", ftle, cents)
    m = loadmat(tmp_path / "out" / "ftle_a.mat")
    assert m["ftle"].shape == (3, 2, 1)
    np.testing.assert_array_equal(m["x"].ravel(), cents[:, 0])
    u = io.create_writer("mat", str(tmp_path / "out2"))
    u.write("ftle_b", ftle, np.hstack([cents, np.ones((6, 1))]))
    m = loadmat(tmp_path / "out2" / "ftle_b.mat")
    np.testing.assert_array_equal(m["ftle"].ravel(), ftle)
    assert "z" in m
    with pytest.raises(ValueError):
        io.create_writer("hdf5", str(tmp_path))


def test_vtk_writer_roundtrip(tmp_path):
    w = io.create_writer("vtk", str(tmp_path), grid_shape=(4, 3))
    X, Y = np.meshgrid(np.arange(4.0), np.arange(3.0), indexing="ij")
    cents = np.stack([X.ravel(order="F"), Y.ravel(order="F")], axis=1)
    ftle = np.arange(12.0)
    w.write("ftle_s", ftle, cents)
    d = io.read_vtk_xml(str(tmp_path / "ftle_s.vts"))
    np.testing.assert_array_equal(d["ftle"], ftle)
    assert d["points"].shape == (12, 3) and np.all(d["points"][:, 2] == 0)
    np.testing.assert_array_equal(d["points"][:, :2], cents)
    text = open(tmp_path / "ftle_s.vts").read()
    assert 'WholeExtent="0 3 0 2 0 0"' in text
    p = io.create_writer("vtk", str(tmp_path))
    p.write("ftle_p", ftle[:5], np.random.default_rng(0).random((5, 3)))
    d = io.read_vtk_xml(str(tmp_path / "ftle_p.vtp"))
    np.testing.assert_array_equal(d["ftle"], ftle[:5])
    np.testing.assert_array_equal(d["offsets"], np.arange(1, 6))


def test_direct_mat_reader_matches_loadmat(tmp_path):
    """The direct MAT v5 reader returns loadmat's doubles (C-order ravel of each stored
    matrix) for 2D matrices, row vectors and three components, and hands every other
    file (compressed, integer arrays, mismatched shapes) to loadmat."""
    rng = np.random.default_rng(3)
    cases = {
        "m2": {"velocity_x": rng.random((7, 5)), "velocity_y": rng.random((7, 5))},
        "vec": {"velocity_x": rng.random(11), "velocity_y": rng.random(11)},
        "m3": {"velocity_x": rng.random((4, 6)), "velocity_y": rng.random((4, 6)),
               "velocity_z": rng.random((4, 6)), "other": np.arange(3)},
    }
    for name, data in cases.items():
        f = tmp_path / f"{name}.mat"
        savemat(f, data)
        raw = io._raw_components(f, "velocity")
        assert raw is not None, name
        ref = io._stack(loadmat(f), "velocity", f)
        np.testing.assert_array_equal(io.read_velocity(f), ref)
        # what the streamed feed ships: column-major bytes, reordered on the device
        arrays, (rows, cols) = raw
        shipped = np.stack(arrays).reshape(len(arrays), cols, rows).transpose(0, 2, 1)
        np.testing.assert_array_equal(shipped.reshape(len(arrays), -1), ref)
    fz = tmp_path / "zipped.mat"
    savemat(fz, cases["m2"], do_compression=True)
    assert io._raw_components(fz, "velocity") is None
    np.testing.assert_array_equal(io.read_velocity(fz), io._stack(loadmat(fz), "velocity", fz))
    fi = tmp_path / "ints.mat"
    savemat(fi, {"velocity_x": np.arange(6).reshape(2, 3), "velocity_y": np.ones((2, 3))})
    assert io._raw_components(fi, "velocity") is None
    np.testing.assert_array_equal(io.read_velocity(fi), io._stack(loadmat(fi), "velocity", fi))
    fm = tmp_path / "mixed.mat"
    savemat(fm, {"velocity_x": rng.random((2, 3)), "velocity_y": rng.random((3, 2))})
    assert io._raw_components(fm, "velocity") is None


def test_slot_copy_plan_cache_gives_each_files_values(tmp_path):
    """The copy plan cached per (slot, scratch, output, layout) serves later files of the
    same layout in the same slot: each comes out in the reference's node order (what
    read_velocity returns), with or without the cache (CPU tensors stand in for the
    device here; the plan is the same tensor views either way)."""
    import torch

    ny, nx = 6, 9
    rng = np.random.default_rng(3)
    files = []
    for i in range(3):
        f = tmp_path / f"v{i}.mat"
        savemat(f, {"velocity_x": rng.random((ny, nx)), "velocity_y": rng.random((ny, nx))})
        files.append(str(f))
    size = max(len(open(f, "rb").read()) for f in files)
    slot = torch.zeros(size + 64, dtype=torch.uint8)
    raw = torch.empty((2, nx * ny), dtype=torch.float64)
    kept = torch.empty((2, nx * ny), dtype=torch.float64)  # the cached path's output
    cache = {}
    for f in files:
        data = open(f, "rb").read()
        slot.zero_()
        slot[:len(data)] = torch.frombuffer(bytearray(data), dtype=torch.uint8)
        lay = io._component_layout(
            io._mat_parse(memoryview(slot.numpy())[:len(data)], ["velocity_x", "velocity_y"],
                          ["velocity_z"]), "velocity")
        assert lay is not None
        want = io.read_velocity(f)
        got = io.slot_to_device(slot, lay, 2, nx * ny, raw,
                                torch.empty((2, nx * ny), dtype=torch.float64))
        np.testing.assert_array_equal(got.numpy(), want)
        got = io.slot_to_device(slot, lay, 2, nx * ny, raw, kept, cache=cache)
        assert got.data_ptr() == kept.data_ptr()
        np.testing.assert_array_equal(kept.numpy(), want)
    assert len(cache) == 1  # one slot, one scratch, one output, one layout: one plan
