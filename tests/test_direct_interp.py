"""Direct interpolation (ruge_stuben/par_interpolation.cpp:1453-1715).

The CPU restatement is pinned on the reference's fixtures
(aniso_P_direct, laplacian_P_direct in tests/test_oracle_golden.py) and on
the reference's own compiled routine (tests/test_oracle_vs_reference.py).
Here the per-row code the CUDA kernels run (direct_interp.cuh) is built for
the host and must reproduce the restatement exactly; the GPU test runs the
kernels through the C ABI and the hierarchy."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import ROOT

CSRC = os.path.join(ROOT, "raptor_b200", "csrc")


def problems():
    aniso = O.sort_diag_first(O.stencil_grid(O.diffusion_stencil_2d(0.001, np.pi / 8), [60, 60]))
    lap = O.sort_diag_first(O.stencil_grid(O.laplace_stencil_27pt(), [12, 12, 12]))
    return {"aniso60": aniso, "lap27_12": lap}


def split(A):
    S = O.sort_diag_first(O.classical_strength(A, 0.25))
    st = O.split_pmis(S, O.rand_weights(A.shape[0]))
    return S, st


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("direct") / "libdirect_rows.so"
    subprocess.check_call(["g++", "-O2", "-std=c++14", "-ffp-contract=off", "-fPIC", "-shared",
                           "-I", CSRC, os.path.join(ROOT, "tests", "cxx", "direct_rows.cpp"),
                           "-o", str(out)])
    L = C.CDLL(str(out))
    I = np.ctypeslib.ndpointer(np.int32, flags="C")
    D = np.ctypeslib.ndpointer(np.float64, flags="C")
    L.direct_rows_count.restype = C.c_int
    L.direct_rows_count.argtypes = [C.c_int, I, I, I, I]
    L.direct_rows_fill.argtypes = [C.c_int, I, I, D, I, I, I, I, I, D]
    return L


@pytest.mark.parametrize("name", ["aniso60", "lap27_12"])
def test_kernel_rows_on_the_host_match_the_restatement(host_lib, name):
    A = problems()[name]
    S, st = split(A)
    n = A.shape[0]
    arp, aci, acv = A.arrays()
    srp, sci, _ = S.arrays()
    st = np.ascontiguousarray(st, np.int32)
    rp = np.zeros(n + 1, np.int32)
    nnz = host_lib.direct_rows_count(n, srp, sci, st, rp)
    pc = np.zeros(max(nnz, 1), np.int32)
    pv = np.zeros(max(nnz, 1), np.float64)
    host_lib.direct_rows_fill(n, arp, aci, acv, srp, sci, st, rp, pc, pv)
    cmap = np.cumsum(st == 1) - 1
    ref = O.interpolation(A, S, st, kind="direct")
    rrp, rci, rcv = ref.arrays()
    assert np.array_equal(rp, rrp)
    assert np.array_equal(cmap[pc[:nnz]], rci)
    assert np.array_equal(pv[:nnz], rcv)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["aniso60", "lap27_12"])
def test_gpu_direct_interpolation_and_hierarchy(name):
    rb = pytest.importorskip("raptor_b200")
    from tests.test_gpu_parity import assert_csr_equal, oc_tuple, rb_tuple, to_rb
    rb.init(0)
    A = problems()[name]
    S, st = split(A)
    Ab, Sb = to_rb(A), to_rb(S)
    P = rb.direct_interpolation(Ab, Sb, st)
    assert_csr_equal(rb_tuple(P), oc_tuple(O.interpolation(A, S, st, kind="direct")))
    # a whole RS hierarchy with Direct interpolation against the restatement
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Direct, rb.Classical, rb.L1Jacobi)
    ml.setup(Ab)
    om = O.Hierarchy(A, interp="direct", relax="l1_jacobi")
    assert ml.num_levels == om.num_levels
    for l in range(ml.num_levels - 1):
        assert_csr_equal(rb_tuple(ml.level_matrix(l, "P")), oc_tuple(om.P(l)))
    n = A.shape[0]
    bh = np.random.default_rng(9).uniform(-1.0, 1.0, n)
    x = rb.ParVector(n)
    res = []
    rb.PCG(Ab, ml, x, rb.ParVector(n, values=bh), res, tol=1e-8, max_iter=300,
           mode=rb.PCG_TRUE_RESIDUAL)
    xo, ores, _ = O.pcg(A, om, np.zeros(n), bh, tol=1e-8, max_iter=300, mode=1)
    assert len(res) == len(ores)
    np.testing.assert_allclose(res, ores, rtol=1e-6, atol=0)
