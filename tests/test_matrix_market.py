"""MatrixMarket reading and writing (gallery/matrix_market.cpp,
gallery/par_matrix_market.cpp).

The reference's fixtures sas_P0.mtx (general), aniso_S.mtx (symmetric) and
aniso.mtx (symmetric) are kept byte for byte in tests/golden/raptor_mm.npz;
sas_P0 and aniso_S have PETSc-binary twins in raptor_golden.npz, so the
parsed matrices are pinned against independently stored copies.  The host
parser runs without a device; the device readers are the same parser plus
one upload (marked gpu).
"""
import os

import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

from tests.conftest import ROOT

rb = pytest.importorskip("raptor_b200")

GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def mm_files(tmp_path_factory):
    z = np.load(os.path.join(GOLD, "raptor_mm.npz"))
    d = tmp_path_factory.mktemp("mm")
    out = {}
    for name in z.files:
        p = d / (name + ".mtx")
        p.write_bytes(z[name].tobytes())
        out[name] = p
    return out


@pytest.fixture(scope="module")
def petsc():
    return np.load(os.path.join(GOLD, "raptor_golden.npz"))


def sorted_rows(rp, ci, cv):
    ci, cv = np.array(ci), np.array(cv)
    for i in range(len(rp) - 1):
        s, e = rp[i], rp[i + 1]
        o = np.argsort(ci[s:e], kind="stable")
        ci[s:e], cv[s:e] = ci[s:e][o], cv[s:e][o]
    return ci, cv


def scipy_csr(path):
    """scipy's own reader (it mirrors symmetric files, each diagonal once)."""
    try:
        M = scipy.io.mmread(str(path), spmatrix=False)
    except TypeError:   # scipy without the spmatrix switch
        M = scipy.io.mmread(str(path))
    M = sp.csr_matrix(M)
    M.sort_indices()
    return M


def file_triplets(path):
    """(i, j, v) of the entries in file order, 0-based, from the text."""
    rows = []
    with open(path) as f:
        lines = [l for l in f if not l.startswith("%") and l.strip()]
    for l in lines[1:]:
        i, j, v = l.split()[:3]
        rows.append((int(i) - 1, int(j) - 1, float(v)))
    return rows


def test_read_par_mm_matches_petsc_twins(mm_files, petsc):
    # general (sas_P0) and symmetric (aniso_S, mirrored) files against the
    # reference's PETSc-binary copies of the same matrices
    for name in ("sas_P0", "aniso_S"):
        m, n, rp, ci, cv = rb.mm_read_host(mm_files[name], mirror=True, sort_rows=True)
        assert (m, n) == tuple(petsc[name + "__shape"])
        grp = petsc[name + "__rowptr"]
        gci, gcv = sorted_rows(grp, petsc[name + "__cols"], petsc[name + "__vals"])
        assert np.array_equal(rp, grp) and np.array_equal(ci, gci)
        np.testing.assert_allclose(cv, gcv, rtol=1e-15, atol=1e-15)


def test_symmetric_mirror_matches_scipy(mm_files):
    # aniso.mtx stores the lower triangle (2977 entries, 625 on the diagonal)
    m, n, rp, ci, cv = rb.mm_read_host(mm_files["aniso"], mirror=True, sort_rows=True)
    ref = scipy_csr(mm_files["aniso"])
    assert (m, n) == ref.shape and len(ci) == 2 * 2977 - 625 == ref.nnz
    assert np.array_equal(rp, ref.indptr) and np.array_equal(ci, ref.indices)
    assert np.array_equal(cv, ref.data)


def test_read_mm_keeps_file_order_and_ignores_symmetry(mm_files):
    # the sequential reader: the stored triangle only, file order per row
    m, n, rp, ci, cv = rb.mm_read_host(mm_files["aniso"], mirror=False, sort_rows=False)
    trip = file_triplets(mm_files["aniso"])
    assert len(ci) == len(trip) == 2977
    want_rp = np.zeros(m + 1, np.int64)
    for i, _, _ in trip:
        want_rp[i + 1] += 1
    assert np.array_equal(rp, np.cumsum(want_rp))
    nxt = rp[:-1].copy()
    for i, j, v in trip:
        assert ci[nxt[i]] == j and cv[nxt[i]] == v
        nxt[i] += 1


def test_write_round_trip_is_byte_identical(mm_files, tmp_path):
    # the reference's own test: read, write, diff (sas_P0 is written in the
    # same "%d %d %.15e" row order that write_mm produces)
    m, n, rp, ci, cv = rb.mm_read_host(mm_files["sas_P0"], mirror=False, sort_rows=False)
    out = tmp_path / "out.mtx"
    rb.mm_write_host(out, m, n, rp, ci, cv)
    assert out.read_bytes() == mm_files["sas_P0"].read_bytes()
    m2, n2, rp2, ci2, cv2 = rb.mm_read_host(out, mirror=False, sort_rows=False)
    assert (m2, n2) == (m, n)
    assert np.array_equal(rp2, rp) and np.array_equal(ci2, ci) and np.array_equal(cv2, cv)


def test_fields_comments_and_skew(tmp_path):
    p = tmp_path / "a.mtx"
    p.write_text("%%MatrixMarket matrix coordinate integer skew-symmetric\n"
                 "% comment\n\n% another\n3 3 2\n2 1 5\n3 2 -7\n")
    m, n, rp, ci, cv = rb.mm_read_host(p)
    dense = sp.csr_matrix((cv, ci, rp), shape=(m, n)).toarray()
    assert np.array_equal(dense, [[0, -5, 0], [5, 0, 7], [0, -7, 0]])
    p.write_text("%%MatrixMarket matrix coordinate pattern general\n2 3 2\n1 3\n2 1\n")
    m, n, rp, ci, cv = rb.mm_read_host(p)
    assert (m, n) == (2, 3) and list(ci) == [2, 0] and list(cv) == [1.0, 1.0]
    # an empty matrix
    p.write_text("%%MatrixMarket matrix coordinate real general\n4 2 0\n")
    m, n, rp, ci, cv = rb.mm_read_host(p)
    assert (m, n) == (4, 2) and list(rp) == [0] * 5 and len(ci) == 0


@pytest.mark.parametrize("text,what", [
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", "format"),
    ("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n", "field"),
    ("%%MatrixMarket matrix coordinate real hermitian\n1 1 1\n1 1 1\n", "symmetry"),
    ("MatrixMarket matrix coordinate real general\n1 1 1\n1 1 1\n", "banner"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n", "ends"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n", "outside"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 x 1\n", "column index"),
])
def test_malformed_files_are_status_codes(tmp_path, text, what):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    with pytest.raises(rb.RaptorError) as e:
        rb.mm_read_host(p)
    assert what in str(e.value)


def test_missing_file():
    with pytest.raises(rb.RaptorError) as e:
        rb.mm_read_host("/nonexistent/x.mtx")
    assert "cannot open" in str(e.value)


@pytest.mark.gpu
def test_device_readers_and_writer(mm_files, tmp_path):
    rb.init(0)
    A = rb.read_par_mm(mm_files["aniso"])
    ref = scipy_csr(mm_files["aniso"])
    rp, ci, cv = A.arrays()
    assert np.array_equal(rp, ref.indptr) and np.array_equal(ci, ref.indices)
    assert np.array_equal(cv, ref.data)
    B = rb.read_mm(mm_files["sas_P0"])
    out = tmp_path / "o.mtx"
    rb.write_mm(B, out)
    assert out.read_bytes() == mm_files["sas_P0"].read_bytes()
    # a product on the device from a file-read matrix
    x = np.linspace(-1.0, 1.0, ref.shape[1])
    y = rb.ParVector(ref.shape[0])
    A.mult(rb.ParVector(ref.shape[1], values=x), y)
    np.testing.assert_allclose(y.numpy(), ref @ x, rtol=1e-13, atol=1e-13)
