"""GPU parity of the smoothed-aggregation setup (mis2, aggregate,
fit_candidates, jacobi_prolongation) and of SA hierarchies and solves.

The components are checked against the reference's own fixtures
(aggregation/tests/test_par_smoothed_aggregation.cpp reads the sas_* files)
and bit-exactly against the oracle on larger seeded problems; hierarchies
level by level (patterns, values and entry order), and solve histories
within 1e-10 relative.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import golden_csr
from tests.test_gpu_parity import (aniso, aniso7, assert_csr_equal, lap27, oc_tuple,
                                   rb_tuple, to_rb)

pytestmark = pytest.mark.gpu

rb = pytest.importorskip("raptor_b200")


@pytest.fixture(scope="module", autouse=True)
def _device():
    rb.init(0)


def golden_rb(g, name):
    return rb.ParCSRMatrix.from_arrays(*golden_csr(g, name))


def golden_oc(g, name):
    return O.CSR.from_arrays(*golden_csr(g, name))


# ------------------------------------------------------- golden fixtures --
@pytest.mark.parametrize("lvl", [0, 1])
def test_mis2_golden(golden, lvl):
    S = golden_rb(golden, "sas_S%d" % lvl)
    S.sort_diag_first()
    n = S.global_num_rows
    states = rb.mis2(S, golden["weights"][:n])
    np.testing.assert_array_equal(states, golden["sas_mis%d" % lvl])


@pytest.mark.parametrize("lvl", [0, 1])
def test_aggregate_golden(golden, lvl):
    A = golden_rb(golden, "sas_A%d" % lvl)
    A.sort_diag_first()
    S = golden_rb(golden, "sas_S%d" % lvl)
    S.sort_diag_first()
    n = S.global_num_rows
    states = golden["sas_mis%d" % lvl]
    n_aggs, agg = rb.aggregate(A, S, states, golden["weights"][:n])
    roots = np.nonzero(states > 0)[0]
    assert n_aggs == len(roots)
    np.testing.assert_array_equal(roots[golden["sas_agg%d" % lvl]], agg)


def test_tentative_and_smoothed_prolongator_golden(golden):
    # level 0 of test_par_smoothed_aggregation.cpp: T0 from all-ones B, P0
    A = golden_rb(golden, "sas_A0")
    A.sort_diag_first()
    n = A.global_num_rows
    states = golden["sas_mis0"]
    roots = np.nonzero(states > 0)[0]
    agg = roots[golden["sas_agg0"]].astype(np.int32)
    T, R = rb.fit_candidates(n, len(roots), agg, np.ones(n))
    ref_t = golden_csr(golden, "sas_T0")
    got_t = rb_tuple(T)
    assert_csr_equal(got_t, ref_t, rtol=1e-6)
    P = rb.jacobi_prolongation(A, T)
    assert_csr_equal(rb_tuple(P), golden_csr(golden, "sas_P0"), rtol=1e-6)
    # A_1 = P^T A P without moving the diagonal (the SA solver's order)
    Ac = rb.rap(A, P, diag_first=False)
    assert_csr_equal(rb_tuple(Ac), golden_csr(golden, "sas_A1"), rtol=1e-6)


# -------------------------------------------------- bit-exact vs oracle --
PROBS = {
    "aniso100": lambda: aniso(100),
    "aniso7_16": lambda: aniso7(16),
    "lap27_14": lambda: lap27(14),
}


@pytest.mark.parametrize("prob", sorted(PROBS))
@pytest.mark.parametrize("theta", [0.0, 0.25])
def test_sa_components_bit_exact(prob, theta):
    Ao = O.sort_diag_first(PROBS[prob]())
    n = Ao.shape[0]
    w = O.rand_weights(n)
    So = O.symmetric_strength(Ao, theta)
    A = to_rb(Ao)
    S = A.strength(rb.Symmetric, theta)
    assert_csr_equal(rb_tuple(S), oc_tuple(So), exact_order=True)
    st_o = O.mis2(So, w)
    st = rb.mis2(S, w)
    np.testing.assert_array_equal(st, st_o)
    na_o, agg_o = O.aggregate(Ao, So, st_o)
    na, agg = rb.aggregate(A, S, st)
    assert na == na_o
    np.testing.assert_array_equal(agg, agg_o)
    B = np.random.default_rng(5).uniform(0.5, 1.5, n)
    To, Ro = O.fit_candidates(n, na_o, agg_o, B)
    T, R = rb.fit_candidates(n, na, agg, B)
    assert_csr_equal(rb_tuple(T), oc_tuple(To), exact_order=True)
    np.testing.assert_array_equal(R, Ro)
    for steps in (1, 2):
        Po = O.jacobi_prolongation(Ao, To, 4.0 / 3, steps)
        P = rb.jacobi_prolongation(A, T, 4.0 / 3, steps)
        assert_csr_equal(rb_tuple(P), oc_tuple(Po), exact_order=True)


def sa_pair(Ao, theta, relax, **kw):
    A = to_rb(Ao)
    ml = rb.ParSmoothedAggregationSolver(theta, relax_type={"jacobi": rb.Jacobi,
                                                            "l1_jacobi": rb.L1Jacobi,
                                                            "sor": rb.SOR}[relax])
    for k, v in kw.items():
        setattr(ml, k, v)
    ml.setup(A)
    om = O.Hierarchy(Ao, solver="sa", strong_threshold=theta,
                     relax={"sor": "mc_sor"}.get(relax, relax), **kw)
    return A, ml, om


@pytest.mark.parametrize("prob", sorted(PROBS))
def test_sa_hierarchy_bit_exact(prob):
    Ao = PROBS[prob]()
    A, ml, om = sa_pair(Ao, 0.0, "jacobi")
    assert ml.num_levels == om.num_levels
    for l in range(ml.num_levels):
        assert_csr_equal(rb_tuple(ml.level_matrix(l, "A")), oc_tuple(om.A(l)), exact_order=True)
        if l < ml.num_levels - 1:
            assert_csr_equal(rb_tuple(ml.level_matrix(l, "P")), oc_tuple(om.P(l)),
                             exact_order=True)


@pytest.mark.parametrize("prob", ["lap27_14", "aniso7_16"])
def test_sa_solve_history_jacobi(prob):
    Ao = PROBS[prob]()
    A, ml, om = sa_pair(Ao, 0.0, "jacobi", relax_weight=2.0 / 3.0, solve_tol=1e-8)
    n = Ao.shape[0]
    bh = O.spmv(Ao, np.ones(n))
    x = rb.ParVector(n)
    it = ml.solve(x, rb.ParVector(n, values=bh))
    xo, ito, ho = om.solve(np.zeros(n), bh)
    assert it == ito
    # 1e-10 relative, above an absolute floor of 1e-15: once ||r|| / ||b||
    # nears 1e-8, b - A x cancels all but the last few digits of A x, and the
    # GPU's different (equally rounded) summation order moves the history by
    # about 5e-17 absolute, more than 1e-10 of such small entries
    np.testing.assert_allclose(ml.get_residuals(), ho, rtol=1e-10, atol=1e-15)
    np.testing.assert_allclose(x.numpy(), xo, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("prob", ["aniso100", "lap27_14"])
def test_sa_pcg_reference_history(prob):
    Ao = PROBS[prob]()
    A, ml, om = sa_pair(Ao, 0.0, "l1_jacobi")
    n = Ao.shape[0]
    bh = np.random.default_rng(3).uniform(-1, 1, n)
    x = rb.ParVector(n)
    res = []
    rb.PCG(A, ml, x, rb.ParVector(n, values=bh), res, tol=1e-8)
    xo, ho, _ = O.pcg(Ao, om, np.zeros(n), bh, tol=1e-8)
    assert len(res) == len(ho)
    np.testing.assert_allclose(res, ho, rtol=1e-10)
    np.testing.assert_allclose(x.numpy(), xo, rtol=1e-9, atol=1e-12)


def test_sa_fp32_cycle_reaches_fp64_accuracy():
    Ao = aniso7(24)
    A = to_rb(Ao)
    n = Ao.shape[0]
    bh = np.random.default_rng(7).uniform(-1, 1, n)
    b = rb.ParVector(n, values=bh)
    xs = {}
    for prec in (rb.FP64, rb.FP32):
        ml = rb.ParSmoothedAggregationSolver(0.0, relax_type=rb.L1Jacobi)
        ml.precision = prec
        ml.setup(A)
        x = rb.ParVector(n)
        res = []
        rb.PCG(A, ml, x, b, res, tol=1e-8, max_iter=300, mode=rb.PCG_TRUE_RESIDUAL)
        r = rb.ParVector(n)
        A.residual(x, b, r)
        assert r.norm(2) / np.linalg.norm(bh) <= 1e-8
        xs[prec] = x.numpy()
    assert np.linalg.norm(xs[rb.FP32] - xs[rb.FP64]) <= 1e-6 * np.linalg.norm(xs[rb.FP64])
