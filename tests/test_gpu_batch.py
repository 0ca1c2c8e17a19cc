"""GPU tests of the uneven batch of independent systems (rb_batch_*).

Every system of a batch must behave as if solved alone: its hierarchy has
the levels a standalone setup builds, one batch V-cycle equals the
standalone V-cycle of each system (to rounding: 1e-11 relative in FP64,
1e-5 in FP32), and the batch PCG gives each system the iterations (within
one) and the solution of its standalone true-residual PCG, with its
iterations run on the device (a few host waits per solve, not one per
iteration).
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

rb = pytest.importorskip("raptor_b200")


@pytest.fixture(scope="module", autouse=True)
def _device():
    rb.init(0)


def systems(seed, count, lo=12, hi=70, tiny=True):
    """Rotated anisotropic diffusion systems of uneven sizes and parameters."""
    rng = np.random.default_rng(seed)
    mats = []
    for s in range(count):
        side = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        eps = math.exp(rng.uniform(math.log(1e-3), 0.0))
        theta = rng.uniform(0.0, math.pi)
        mats.append(rb.par_stencil_grid(rb.diffusion_stencil_2d(eps, theta), [side, side]))
    if tiny:
        # a system no larger than max_coarse: its hierarchy is the dense solve
        mats.append(rb.par_stencil_grid(rb.diffusion_stencil_2d(0.5, 0.3), [6, 6]))
    return mats


def make_ml(kind, prec, relax=None):
    if kind == "sa":
        ml = rb.ParSmoothedAggregationSolver(0.25, relax_type=relax or rb.L1Jacobi)
    else:
        ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.ModClassical, rb.Classical,
                                    relax or rb.L1Jacobi)
    ml.precision = prec
    return ml


@pytest.mark.parametrize("kind", ["rs", "sa"])
@pytest.mark.parametrize("prec", [0, 1])
def test_batch_cycle_equals_standalone_cycles(kind, prec):
    mats = systems(3, 6)
    B = rb.Batch(mats, make_ml(kind, prec))
    rng = np.random.default_rng(5)
    bh = rng.uniform(-1, 1, B.total_rows)
    x = rb.ParVector(B.total_rows)
    B.cycle(x, rb.ParVector(B.total_rows, values=bh))
    got = x.numpy()
    tol = 1e-11 if prec == rb.FP64 else 1e-5
    for s, A in enumerate(mats):
        lo, hi = B.offsets[s], B.offsets[s + 1]
        ml = make_ml(kind, prec)
        ml.setup(A)
        assert ml.num_levels == B.levels[s]
        xs = rb.ParVector(hi - lo)
        ml.cycle(xs, rb.ParVector(hi - lo, values=bh[lo:hi]))
        ref = xs.numpy()
        assert np.linalg.norm(got[lo:hi] - ref) <= tol * np.linalg.norm(ref), s


@pytest.mark.parametrize("kind", ["rs", "sa"])
@pytest.mark.parametrize("prec", [0, 1])
def test_batch_pcg_matches_standalone_solves(kind, prec):
    mats = systems(11, 8)
    B = rb.Batch(mats, make_ml(kind, prec))
    bh = np.random.default_rng(9).uniform(-1, 1, B.total_rows)
    x = rb.ParVector(B.total_rows)
    rc, iters, relres = B.pcg(x, rb.ParVector(B.total_rows, values=bh), tol=1e-8, max_iter=400)
    assert rc == 0
    # the iterations run on the device: the host waits once per launch of
    # the device loop (one, plus one per failed true-residual confirmation),
    # not once per iteration
    assert 1 <= B.host_waits <= 3 < int(max(iters)), (B.host_waits, int(max(iters)))
    got = x.numpy()
    for s, A in enumerate(mats):
        lo, hi = B.offsets[s], B.offsets[s + 1]
        n = hi - lo
        rp, ci, cv = A.arrays()
        Ao = O.CSR.from_arrays(n, n, rp, ci, cv)
        r = bh[lo:hi] - O.spmv(Ao, got[lo:hi])
        bn = np.linalg.norm(bh[lo:hi])
        assert np.linalg.norm(r) <= 1e-8 * bn * (1 + 1e-6), s
        assert relres[s] <= 1e-8
        ml = make_ml(kind, prec)
        ml.setup(A)
        xs = rb.ParVector(n)
        res = []
        rb.PCG(A, ml, xs, rb.ParVector(n, values=bh[lo:hi]), res, tol=1e-8, max_iter=400,
               mode=rb.PCG_TRUE_RESIDUAL)
        assert abs(int(iters[s]) - (len(res) - 1)) <= 1, (s, iters[s], len(res) - 1)
        ref = xs.numpy()
        assert np.linalg.norm(got[lo:hi] - ref) <= 1e-6 * np.linalg.norm(ref), s


def test_batch_with_multicolour_ssor_and_zero_system():
    # symmetric multicolour SSOR keeps the preconditioner symmetric for CG
    mats = systems(21, 4, tiny=False)
    B = rb.Batch(mats, make_ml("rs", rb.FP64, relax=rb.SSOR))
    bh = np.random.default_rng(2).uniform(-1, 1, B.total_rows)
    bh[B.offsets[1]:B.offsets[2]] = 0.0
    x = rb.ParVector(B.total_rows)
    rc, iters, relres = B.pcg(x, rb.ParVector(B.total_rows, values=bh), tol=1e-8, max_iter=400)
    assert rc == 0
    assert iters[1] == 0 and np.all(x.numpy()[B.offsets[1]:B.offsets[2]] == 0.0)
    assert all(iters[s] > 0 for s in (0, 2, 3))


@pytest.mark.parametrize("prec", [0, 1])
def test_batch_stopped_systems_left_alone(prec):
    """Systems that stop early leave the batch's cycle and outer iteration
    (their rows are passed over from then on): a zero right-hand side stops
    before the first iteration and its solution stays exactly zero, and every
    other system, whichever iteration it stopped at, ends with the solution
    and iteration count of its standalone solve."""
    mats = systems(31, 5)
    B = rb.Batch(mats, make_ml("rs", prec))
    bh = np.random.default_rng(4).uniform(-1, 1, B.total_rows)
    bh[B.offsets[2]:B.offsets[3]] = 0.0
    x = rb.ParVector(B.total_rows)
    rc, iters, relres = B.pcg(x, rb.ParVector(B.total_rows, values=bh), tol=1e-8, max_iter=400)
    assert rc == 0
    got = x.numpy()
    assert iters[2] == 0 and np.all(got[B.offsets[2]:B.offsets[3]] == 0.0)
    assert int(max(iters)) > int(min(i for i in iters if i > 0))
    for s, A in enumerate(mats):
        if s == 2:
            continue
        lo, hi = B.offsets[s], B.offsets[s + 1]
        n = hi - lo
        ml = make_ml("rs", prec)
        ml.setup(A)
        xs = rb.ParVector(n)
        res = []
        rb.PCG(A, ml, xs, rb.ParVector(n, values=bh[lo:hi]), res, tol=1e-8, max_iter=400,
               mode=rb.PCG_TRUE_RESIDUAL)
        assert abs(int(iters[s]) - (len(res) - 1)) <= 1, (s, iters[s], len(res) - 1)
        ref = xs.numpy()
        assert np.linalg.norm(got[lo:hi] - ref) <= 1e-6 * np.linalg.norm(ref), s


def test_batch_pcg_matches_oracle_pcg():
    """Every system of a batch solve against the CPU restatement's own PCG
    (true-residual mode) on the hierarchy the restatement builds for it: the
    iterations (within one) and the solution (within 1e-6)."""
    mats = systems(13, 5)
    B = rb.Batch(mats, make_ml("rs", rb.FP64))
    bh = np.random.default_rng(17).uniform(-1, 1, B.total_rows)
    x = rb.ParVector(B.total_rows)
    rc, iters, relres = B.pcg(x, rb.ParVector(B.total_rows, values=bh), tol=1e-8, max_iter=400)
    assert rc == 0
    got = x.numpy()
    for s, A in enumerate(mats):
        lo, hi = B.offsets[s], B.offsets[s + 1]
        n = hi - lo
        rp, ci, cv = A.arrays()
        Ao = O.CSR.from_arrays(n, n, rp, ci, cv)
        om = O.Hierarchy(Ao, interp="mod_classical", relax="l1_jacobi")
        xo, ho, _ = O.pcg(Ao, om, np.zeros(n), bh[lo:hi], tol=1e-8, max_iter=400, mode=1)
        assert abs(int(iters[s]) - (len(ho) - 1)) <= 1, (s, iters[s], len(ho) - 1)
        assert np.linalg.norm(got[lo:hi] - xo) <= 1e-6 * np.linalg.norm(xo), s
