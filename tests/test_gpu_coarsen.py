"""GPU parity of the Ruge-Stuben C/F splittings against the reference's own
parallel setup at one rank.

RS (the sequential first and second passes of ruge_stuben/cf_splitting.cpp,
run by the library on the host; Falgout from level 3, as
par_ruge_stuben_solver.hpp:77-87 does), CLJP (GPU rounds of
par_cf_splitting.cpp:1383-1607), Falgout (RS then CLJP on what is left) and
HMIS (the RS first pass then the PMIS loop): every level's C/F states, P_l
and A_l of the library's hierarchy must equal, bit for bit, those of the
reference's ParRugeStubenSolver with the same coarsening, compiled unmodified
into oracle/_ref.  The component entry point rb_split must give the
reference's states on the finest strength matrix, and a PCG solve on each
hierarchy must converge.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

rb = pytest.importorskip("raptor_b200")
REF = O.par_ref()
need_ref = pytest.mark.skipif(REF is None, reason="reference parallel path not built")

KINDS = {"rs": 0, "cljp": 1, "falgout": 2, "hmis": 4}


def aniso7(n):
    st = [0.0] * 27
    st[13] = 4.02
    st[12] = st[14] = st[10] = st[16] = -1.0
    st[4] = st[22] = -0.01
    return st


PROBLEMS = {
    "aniso2d_64": lambda L: O.RefMatrix.diffusion(L, 0.001, math.pi / 8, 64, 64),
    "lap27_14": lambda L: O.RefMatrix.laplace27(L, 14, 14, 14),
    "aniso7_18": lambda L: O.RefMatrix.stencil(L, aniso7(18), [18, 18, 18]),
}


@pytest.fixture(scope="module", autouse=True)
def _device():
    rb.init(0)


def rb_from_ref(Ar):
    n, m, _ = Ar.shape
    rp, ci, cv = Ar.arrays()
    return rb.ParCSRMatrix.from_arrays(n, m, rp, ci, cv)


def sorted_rows(rp, ci, cv):
    ci, cv = np.array(ci), np.array(cv)
    for i in range(len(rp) - 1):
        o = np.argsort(ci[rp[i]:rp[i + 1]], kind="stable")
        ci[rp[i]:rp[i + 1]], cv[rp[i]:rp[i + 1]] = ci[rp[i]:rp[i + 1]][o], cv[rp[i]:rp[i + 1]][o]
    return rp, ci, cv


@need_ref
@pytest.mark.parametrize("prob", sorted(PROBLEMS))
@pytest.mark.parametrize("kind", sorted(KINDS))
def test_hierarchy_matches_reference(kind, prob):
    Ar = PROBLEMS[prob](REF)
    A = rb_from_ref(Ar)
    ml = rb.ParRugeStubenSolver(0.25, KINDS[kind], rb.ModClassical, rb.Classical, rb.L1Jacobi)
    ml.setup(A)
    rml = O.RefHierarchy(Ar, theta=0.25, coarsen=kind, interp="mod_classical", relax="jacobi")
    assert ml.num_levels == rml.num_levels
    for l in range(ml.num_levels):
        got = ml.level_matrix(l, "A").arrays()
        ref = rml.A(l).arrays()
        for a, b, what in zip(got, ref, ("rowptr", "cols", "vals")):
            np.testing.assert_array_equal(a, b, err_msg="A_%d %s" % (l, what))
        if l < ml.num_levels - 1:
            np.testing.assert_array_equal(ml.level_states(l), rml.states(l), err_msg="states %d" % l)
            for a, b, what in zip(sorted_rows(*ml.level_matrix(l, "P").arrays()),
                                  sorted_rows(*rml.P(l).arrays()), ("rowptr", "cols", "vals")):
                np.testing.assert_array_equal(a, b, err_msg="P_%d %s" % (l, what))
    n = A.global_num_rows
    b = rb.ParVector(n, values=np.random.default_rng(3).uniform(-1, 1, n))
    x = rb.ParVector(n)
    res = []
    assert rb.PCG(A, ml, x, b, res, tol=1e-8, max_iter=300, mode=rb.PCG_TRUE_RESIDUAL) == 0
    assert res[-1] <= 1e-8


@need_ref
@pytest.mark.parametrize("kind", sorted(KINDS))
def test_split_component_matches_reference(kind):
    Ar = PROBLEMS["aniso2d_64"](REF)
    A = rb_from_ref(Ar)
    S = A.strength(rb.Classical, 0.25)
    st = rb.split(S, KINDS[kind])
    rml = O.RefHierarchy(Ar, theta=0.25, coarsen=kind, interp="mod_classical", relax="jacobi")
    np.testing.assert_array_equal(st, rml.states(0))
