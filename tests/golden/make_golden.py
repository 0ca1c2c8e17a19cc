"""Generate tests/golden/raptor_golden.npz from the reference's test_data.

The reference (13manan/raptor) ships pyamg-generated fixtures in
``test_data/`` (see its ``test_data/README.md``): PETSc binary matrices
(``*.pm``) and text vectors.  This script reads the ones the AMG path's tests
use and stores them, unchanged, as numpy arrays in one compressed file so the
test suite never needs the reference checkout at run time.

Run once in the build container:  python tests/golden/make_golden.py
(``--digests``: only the SHA-256 digests of the PETSc files).
"""
import os
import sys

import numpy as np

REF = os.environ.get("RAPTOR_REFERENCE_ROOT", "/root/reference")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "raptor_golden.npz")
# MatrixMarket files, kept byte for byte (the reader and writer tests parse
# and rewrite them); sas_P0 and aniso_S have PETSc twins above
OUT_MM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "raptor_mm.npz")
# SHA-256 and size of each PETSc file above (the writer's output must equal
# the reference's files byte for byte); --digests writes only this file
OUT_DIGESTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "petsc_digests.json")
MM_FILES = ["sas_P0", "aniso_S", "aniso"]

MATRICES = [
    "aniso", "laplacian27", "random", "laplacian",
    "rss_A0", "rss_A1", "rss_A2", "rss_P0", "rss_P1", "rss_S0", "rss_S1",
    "aniso_S", "aniso_P_mod_class", "aniso_P_extend",
    "laplacian_S", "laplacian_P_mod_class", "laplacian_P_extend",
    "aniso_P_direct", "laplacian_P_direct",
    "sas_A0", "sas_S0", "sas_T0", "sas_P0", "sas_A1", "sas_S1", "sas_T1", "sas_P1",
]
INT_VECTORS = [
    "rss_cf0_pmis", "rss_cf1_pmis", "aniso_split", "laplacian_split",
    "rss_cf0", "rss_cf1", "rss_cf0_rs", "rss_cf1_rs",
    "sas_mis0", "sas_agg0", "sas_mis1", "sas_agg1",
]
REAL_VECTORS = [
    "weights", "cg_res", "bicgstab_res",
    "aniso_ones_b", "aniso_inc_b", "aniso_ones_b_T", "aniso_inc_b_T",
    "laplacian27_ones_b", "laplacian27_inc_b", "laplacian27_ones_b_T", "laplacian27_inc_b_T",
    "random_ones_b", "random_inc_b", "random_ones_b_T", "random_inc_b_T",
]


def read_petsc(path):
    """PETSc binary AIJ: big-endian int32 header (1211216, M, N, nnz), row
    lengths, column indices, float64 values (gallery/matrix_IO.cpp:24-110)."""
    with open(path, "rb") as f:
        hdr = np.frombuffer(f.read(16), dtype=">i4")
        assert int(hdr[0]) == 1211216, path
        m, n, nnz = int(hdr[1]), int(hdr[2]), int(hdr[3])
        lens = np.frombuffer(f.read(4 * m), dtype=">i4").astype(np.int32)
        cols = np.frombuffer(f.read(4 * nnz), dtype=">i4").astype(np.int32)
        vals = np.frombuffer(f.read(8 * nnz), dtype=">f8").astype(np.float64)
    rowptr = np.zeros(m + 1, dtype=np.int32)
    np.cumsum(lens, out=rowptr[1:])
    return m, n, rowptr, cols, vals


def write_digests(td):
    import hashlib
    import json

    out = {}
    for name in MATRICES:
        with open(os.path.join(td, name + ".pm"), "rb") as f:
            data = f.read()
        out[name] = {"sha256": hashlib.sha256(data).hexdigest(), "bytes": len(data)}
    with open(OUT_DIGESTS, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", OUT_DIGESTS)


def main():
    td = os.path.join(REF, "test_data")
    if not os.path.isdir(td):
        sys.exit("reference test_data not found at %s" % td)
    write_digests(td)
    if "--digests" in sys.argv[1:]:
        return
    out = {}
    for name in MATRICES:
        m, n, rp, ci, cv = read_petsc(os.path.join(td, name + ".pm"))
        out[name + "__shape"] = np.array([m, n], dtype=np.int64)
        out[name + "__rowptr"] = rp
        out[name + "__cols"] = ci
        out[name + "__vals"] = cv
    for name in INT_VECTORS:
        out[name] = np.loadtxt(os.path.join(td, name + ".txt"), dtype=np.int64).astype(np.int32)
    for name in REAL_VECTORS:
        out[name] = np.loadtxt(os.path.join(td, name + ".txt"), dtype=np.float64)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")
    mm = {}
    for name in MM_FILES:
        with open(os.path.join(td, name + ".mtx"), "rb") as f:
            mm[name] = np.frombuffer(f.read(), dtype=np.uint8)
    np.savez_compressed(OUT_MM, **mm)
    print("wrote", OUT_MM, os.path.getsize(OUT_MM), "bytes")


if __name__ == "__main__":
    main()
