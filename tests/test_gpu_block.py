"""GPU tests of the k right-hand-side path (block V-cycle and block PCG).

The block kernels are checked against the single-vector path column by
column: one block V-cycle equals k single V-cycles to rounding (1e-11
relative in FP64, 1e-5 in FP32, where only the summation order differs), and
each column of a block PCG solve meets the tolerance on its own true
residual, takes the iterations of a single-vector solve of that column
(within one), and agrees with that solution.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.test_gpu_parity import aniso, aniso7, lap27, to_rb

pytestmark = pytest.mark.gpu

rb = pytest.importorskip("raptor_b200")


@pytest.fixture(scope="module", autouse=True)
def _device():
    rb.init(0)


def make_ml(A, solver, prec, relax=None):
    if solver == "sa":
        ml = rb.ParSmoothedAggregationSolver(0.0, relax_type=relax or rb.L1Jacobi)
    else:
        ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, relax or rb.L1Jacobi)
    ml.precision = prec
    ml.setup(A)
    return ml


def block(cols):
    """n x k columns -> interleaved ParVector (entry (i, c) at i * k + c)."""
    return rb.ParVector(cols.size, values=np.ascontiguousarray(cols).reshape(-1))


PROBS = {"lap27_14": lambda: lap27(14), "aniso7_16": lambda: aniso7(16),
         "aniso64": lambda: aniso(64)}


@pytest.mark.parametrize("prob", sorted(PROBS))
@pytest.mark.parametrize("solver", ["rs", "sa"])
@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("k", [2, 5, 8, 32])
def test_block_cycle_equals_single_cycles(prob, solver, prec, k):
    Ao = PROBS[prob]()
    A = to_rb(Ao)
    n = Ao.shape[0]
    ml = make_ml(A, solver, prec)
    Bh = np.random.default_rng(k).uniform(-1, 1, (n, k))
    Xb = rb.ParVector(n * k)
    ml.cycle_block(Xb, block(Bh), k)
    got = Xb.numpy().reshape(n, k)
    tol = 1e-11 if prec == rb.FP64 else 1e-5
    for c in range(k):
        x = rb.ParVector(n)
        ml.cycle(x, rb.ParVector(n, values=Bh[:, c]))
        ref = x.numpy()
        assert np.linalg.norm(got[:, c] - ref) <= tol * np.linalg.norm(ref), c


@pytest.mark.parametrize("prob,solver", [("lap27_14", "rs"), ("aniso7_16", "sa"),
                                         ("aniso64", "rs")])
@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("k", [2, 8, 32])
def test_block_pcg_columns_match_single_solves(prob, solver, prec, k):
    Ao = PROBS[prob]()
    A = to_rb(Ao)
    n = Ao.shape[0]
    ml = make_ml(A, solver, prec)
    Bh = np.random.default_rng(100 + k).uniform(-1, 1, (n, k))
    Xb = rb.ParVector(n * k)
    rc, iters, relres = rb.PCG_block(A, ml, Xb, block(Bh), k, tol=1e-8, max_iter=500)
    assert rc == 0
    X = Xb.numpy().reshape(n, k)
    for c in range(k):
        # the column's own true residual, computed independently
        bnorm = np.linalg.norm(Bh[:, c])
        r = Bh[:, c] - O.spmv(Ao, X[:, c])
        assert np.linalg.norm(r) <= 1e-8 * bnorm * (1 + 1e-6)
        assert abs(relres[c] - np.linalg.norm(r) / bnorm) <= 1e-3 * relres[c] + 1e-15
        x = rb.ParVector(n)
        res = []
        rb.PCG(A, ml, x, rb.ParVector(n, values=Bh[:, c]), res, tol=1e-8, max_iter=500,
               mode=rb.PCG_TRUE_RESIDUAL)
        assert abs(int(iters[c]) - (len(res) - 1)) <= 1, (c, iters[c], len(res) - 1)
        xs = x.numpy()
        assert np.linalg.norm(X[:, c] - xs) <= 1e-6 * np.linalg.norm(xs)


def test_block_pcg_zero_column_and_single_column():
    Ao = lap27(12)
    A = to_rb(Ao)
    n = Ao.shape[0]
    ml = make_ml(A, "rs", rb.FP64)
    Bh = np.random.default_rng(1).uniform(-1, 1, (n, 3))
    Bh[:, 1] = 0.0
    Xb = rb.ParVector(n * 3)
    rc, iters, relres = rb.PCG_block(A, ml, Xb, block(Bh), 3, tol=1e-8)
    assert rc == 0
    assert iters[1] == 0 and relres[1] == 0.0
    assert np.all(Xb.numpy().reshape(n, 3)[:, 1] == 0.0)
    assert iters[0] > 0 and iters[2] > 0
    # k = 1 runs the single-vector solver
    x1 = rb.ParVector(n)
    rc, it1, rr1 = rb.PCG_block(A, ml, x1, rb.ParVector(n, values=Bh[:, 0]), 1, tol=1e-8)
    assert rc == 0 and rr1[0] <= 1e-8 and it1[0] > 0


def test_block_path_rejects_sor_smoothing():
    Ao = lap27(10)
    A = to_rb(Ao)
    n = Ao.shape[0]
    ml = make_ml(A, "rs", rb.FP64, relax=rb.SOR)
    with pytest.raises(rb.RaptorError):
        rb.PCG_block(A, ml, rb.ParVector(n * 4), rb.ParVector(n * 4, values=np.ones(n * 4)), 4)


@pytest.mark.parametrize("prec", [0, 1])
def test_block_pcg_columns_match_oracle_pcg(prec):
    """Each column of a block solve against the CPU restatement's own PCG
    (true-residual mode) on the same hierarchy, which the restatement builds
    itself: the iterations of the restatement's solve (within one) and its
    solution (within 1e-6)."""
    Ao = lap27(14)
    A = to_rb(Ao)
    n = Ao.shape[0]
    ml = make_ml(A, "rs", prec)
    om = O.Hierarchy(Ao, interp="extended", interp_filter=0.3, relax="l1_jacobi")
    k = 4
    Bh = np.random.default_rng(41).uniform(-1, 1, (n, k))
    Xb = rb.ParVector(n * k)
    rc, iters, relres = rb.PCG_block(A, ml, Xb, block(Bh), k, tol=1e-8, max_iter=300)
    assert rc == 0
    X = Xb.numpy().reshape(n, k)
    for c in range(k):
        xo, ho, _ = O.pcg(Ao, om, np.zeros(n), Bh[:, c], tol=1e-8, max_iter=300, mode=1)
        assert abs(int(iters[c]) - (len(ho) - 1)) <= 1, (c, iters[c], len(ho) - 1)
        assert np.linalg.norm(X[:, c] - xo) <= 1e-6 * np.linalg.norm(xo), c
