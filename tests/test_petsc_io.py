"""PETSc binary AIJ files, read and written on the host (no device).

The reference reads PETSc's binary matrix format (readMatrix,
gallery/matrix_IO.cpp:24-110; readParMatrix, gallery/par_matrix_IO.cpp)
and ships its fixtures in it.  Written from the fixtures' arrays (in file
order, tests/golden/raptor_golden.npz), every file must equal the
reference's file byte for byte (SHA-256 and size recorded by
tests/golden/make_golden.py --digests), and read back it must give the same
arrays.  Malformed files (another class id, truncation, row lengths that do
not add up, a column out of range) must be refused.  The device writer
(rb_write_petsc) must give the same bytes from a device matrix.
"""
import hashlib
import json
import os
import struct

import numpy as np
import pytest

rb = pytest.importorskip("raptor_b200")

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "raptor_golden.npz"))
with open(os.path.join(HERE, "golden", "petsc_digests.json")) as _f:
    DIGESTS = json.load(_f)


def arrays(name):
    m, n = (int(v) for v in G[name + "__shape"])
    return m, n, G[name + "__rowptr"], G[name + "__cols"], G[name + "__vals"]


@pytest.mark.parametrize("name", sorted(DIGESTS))
def test_writer_reproduces_reference_files(tmp_path, name):
    m, n, rp, ci, cv = arrays(name)
    path = tmp_path / (name + ".pm")
    rb.petsc_write_host(path, m, n, rp, ci, cv)
    data = path.read_bytes()
    assert len(data) == DIGESTS[name]["bytes"]
    assert hashlib.sha256(data).hexdigest() == DIGESTS[name]["sha256"]
    m2, n2, rp2, ci2, cv2 = rb.petsc_read_host(path)
    assert (m2, n2) == (m, n)
    np.testing.assert_array_equal(rp2, rp)
    np.testing.assert_array_equal(ci2, ci)
    np.testing.assert_array_equal(cv2, cv)


def test_empty_and_rectangular(tmp_path):
    p = tmp_path / "e.pm"
    rb.petsc_write_host(p, 0, 0, np.zeros(1, np.int32), [], [])
    assert rb.petsc_read_host(p)[:2] == (0, 0)
    rp, ci, cv = np.array([0, 2, 2, 3]), np.array([0, 4, 1]), np.array([1.5, -2.0, 3.25])
    rb.petsc_write_host(p, 3, 5, rp, ci, cv)
    m, n, rp2, ci2, cv2 = rb.petsc_read_host(p)
    assert (m, n) == (3, 5)
    np.testing.assert_array_equal(rp2, rp)
    np.testing.assert_array_equal(ci2, ci)
    np.testing.assert_array_equal(cv2, cv)


def write_raw(path, hdr, lens, cols, vals):
    with open(path, "wb") as f:
        f.write(struct.pack(">4i", *hdr))
        f.write(np.asarray(lens, ">i4").tobytes())
        f.write(np.asarray(cols, ">i4").tobytes())
        f.write(np.asarray(vals, ">f8").tobytes())


@pytest.mark.parametrize("case", ["classid", "truncated", "lengths", "column"])
def test_malformed_files_are_refused(tmp_path, case):
    p = tmp_path / "bad.pm"
    hdr, lens, cols, vals = [1211216, 2, 2, 3], [2, 1], [0, 1, 1], [1.0, 2.0, 3.0]
    if case == "classid":
        hdr[0] = 1211214
    elif case == "lengths":
        lens = [2, 2]
    elif case == "column":
        cols = [0, 2, 1]
    write_raw(p, hdr, lens, cols, vals)
    if case == "truncated":
        p.write_bytes(p.read_bytes()[:-5])
    with pytest.raises(rb.RaptorError):
        rb.petsc_read_host(p)


def test_writer_checks_its_arrays(tmp_path):
    with pytest.raises(rb.RaptorError):
        rb.petsc_write_host(tmp_path / "x.pm", 2, 2, [0, 1, 2], [0, 2], [1.0, 1.0])
    with pytest.raises(rb.RaptorError):
        rb.petsc_write_host(tmp_path / "x.pm", 2, 2, [0, 2, 1], [0, 1], [1.0, 1.0])


@pytest.mark.gpu
def test_device_writer_matches(tmp_path):
    rb.init(0)
    m, n, rp, ci, cv = arrays("aniso")
    A = rb.ParCSRMatrix.from_arrays(m, n, rp, ci, cv)
    p = tmp_path / "aniso.pm"
    rb.write_petsc(A, p)
    assert hashlib.sha256(p.read_bytes()).hexdigest() == DIGESTS["aniso"]["sha256"]
