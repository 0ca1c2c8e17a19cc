"""The one-launch cluster tail of the V-cycle against separate launches.

Levels from a start level down to the coarsest can run as one launch of one
thread-block cluster (tail_cycle.cuh), with the cluster barrier between
phases.  Each phase computes what the separate kernels compute, in the same
order, so a cycle and a whole PCG solve must give bit-identical results with
and without the tail, for every start level, in both precisions, with
L1-Jacobi, weighted Jacobi and the reference's no-op Jacobi.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

rb = pytest.importorskip("raptor_b200")


@pytest.fixture(scope="module", autouse=True)
def _device():
    rb.init(0)


@pytest.fixture(scope="module")
def problem():
    Ao = O.stencil_grid(O.laplace_stencil_27pt(), [36, 36, 36])
    n = Ao.shape[0]
    rp, ci, cv = Ao.arrays()
    A = rb.ParCSRMatrix.from_arrays(n, n, rp, ci, cv)
    bh = np.random.default_rng(20261203).uniform(-1, 1, n)
    return A, bh


def make(A, prec, relax, fuse, compat=0):
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, relax)
    ml.precision = prec
    ml.jacobi_compat = compat
    if relax == rb.Jacobi:
        ml.relax_weight = 2.0 / 3.0
    ml.fuse_coarse = fuse
    ml.setup(A)
    return ml


@pytest.mark.parametrize("prec", [rb.FP64, rb.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("relax,compat", [(rb.L1Jacobi, 0), (rb.Jacobi, 0), (rb.Jacobi, 1)],
                         ids=["l1_jacobi", "jacobi", "jacobi_noop"])
def test_tail_cycle_bit_identical(problem, prec, relax, compat):
    A, bh = problem
    n = A.global_num_rows
    ref = make(A, prec, relax, 0, compat)
    L = ref.num_levels
    assert L >= 4
    assert ref.tail_info()[0] == -1
    b = rb.ParVector(n, values=bh)
    x0 = rb.ParVector(n)
    ref.cycle(x0, b)
    want = x0.numpy()
    # with the no-op Jacobi the cycle is coarse-grid correction only, a
    # singular preconditioner, so only the cycle itself is compared there
    pcg = not compat
    res0 = []
    if pcg:
        x = rb.ParVector(n)
        rb.PCG(A, ref, x, b, res0, tol=1e-8, mode=rb.PCG_TRUE_RESIDUAL)
    for start in sorted({1, L - 2}):
        ml = make(A, prec, relax, start + 1, compat)
        f, ctas = ml.tail_info()
        assert f == start and ctas >= 8
        x1 = rb.ParVector(n)
        ml.cycle(x1, b)
        np.testing.assert_array_equal(x1.numpy(), want)
        if pcg:
            res1 = []
            x = rb.ParVector(n)
            rb.PCG(A, ml, x, b, res1, tol=1e-8, mode=rb.PCG_TRUE_RESIDUAL)
            np.testing.assert_array_equal(np.array(res1), np.array(res0))


def test_tail_choice_is_timed_and_valid(problem):
    A, _ = problem
    ml = make(A, rb.FP32, rb.L1Jacobi, 1)
    f, ctas = ml.tail_info()
    assert f == -1 or (1 <= f <= ml.num_levels - 2 and ctas >= 8)


@pytest.mark.parametrize("prec", [rb.FP64, rb.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("shape", [(36, 36, 36), (150, 150)], ids=["lap27_36", "aniso_150"])
def test_fused_first_sweep_bit_identical(prec, shape, monkeypatch):
    """The first sweep fused with the residual (one pass gathering b d) gives
    the cycle the separate sweep and residual give, bit for bit, on every
    storage the levels use (diagonals, 32- and 16-bit column indices)."""
    st = O.laplace_stencil_27pt() if len(shape) == 3 else O.diffusion_stencil_2d(0.001, np.pi / 8)
    Ao = O.stencil_grid(st, list(shape))
    n = Ao.shape[0]
    rp, ci, cv = Ao.arrays()
    A = rb.ParCSRMatrix.from_arrays(n, n, rp, ci, cv)
    b = rb.ParVector(n, values=np.random.default_rng(8).uniform(-1, 1, n))
    got = {}
    for force in ("0", "1"):
        monkeypatch.setenv("RAPTOR_B200_FUSE_FIRST", force)
        ml = make(A, prec, rb.L1Jacobi, 0)
        assert all(ml.level_fused_first(l) == (force == "1") for l in range(ml.num_levels - 1))
        x = rb.ParVector(n)
        ml.cycle(x, b)
        got[force] = x.numpy()
    np.testing.assert_array_equal(got["0"], got["1"])


@pytest.mark.parametrize("prec", [rb.FP64, rb.FP32], ids=["fp64", "fp32"])
def test_shared_memory_schedule_bit_identical(prec, monkeypatch):
    """The coarse operators' shared-memory schedule (x's window staged per
    chunk of rows, tiled.cuh) sums each row in the order of the strided row
    kernel, so a cycle and a PCG solve are bit-identical with and without it."""
    Ao = O.stencil_grid(O.laplace_stencil_27pt(), [48, 48, 48])
    n = Ao.shape[0]
    rp, ci, cv = Ao.arrays()
    A = rb.ParCSRMatrix.from_arrays(n, n, rp, ci, cv)
    b = rb.ParVector(n, values=np.random.default_rng(9).uniform(-1, 1, n))
    got, hist = {}, {}
    for force in ("0", "1"):
        monkeypatch.setenv("RAPTOR_B200_TILED", force)
        monkeypatch.setenv("RAPTOR_B200_FUSE_FIRST", "1")
        ml = make(A, prec, rb.L1Jacobi, 0)
        lanes = [ml.level_lanes(l) for l in range(ml.num_levels)]
        tiled = any(v & 128 for lv in lanes for v in lv)
        assert tiled == (force == "1"), lanes
        x = rb.ParVector(n)
        ml.cycle(x, b)
        got[force] = x.numpy()
        res = []
        x = rb.ParVector(n)
        rb.PCG(A, ml, x, b, res, tol=1e-8, mode=rb.PCG_TRUE_RESIDUAL)
        hist[force] = np.array(res)
    np.testing.assert_array_equal(got["0"], got["1"])
    np.testing.assert_array_equal(hist["0"], hist["1"])
