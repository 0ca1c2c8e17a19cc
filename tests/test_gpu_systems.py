"""GPU parity of the unknown-based systems form of the Ruge-Stuben solver
(ParMultilevel::num_variables > 1) against the reference's own setup.

With k variables, row i is variable i % k (form_variable_list,
par_ruge_stuben_solver.hpp:44-53), classical strength only couples rows of
one variable (par_strength.cpp:8-339), and ModClassical / Extended
interpolation only count a weak connection to a row of the same variable
(par_interpolation.cpp:811, 918, 1308, 1390).  Every level's states, P_l and
A_l must equal those of the reference's ParRugeStubenSolver with the same
num_variables, compiled unmodified into oracle/_ref; a PCG solve on the
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

COARSEN = {"pmis": rb.PMIS, "rs": rb.RS}
INTERP = {"mod_classical": rb.ModClassical, "extended": rb.Extended}
PROBLEMS = {
    # (matrix, variables): the variable count divides the grid's line
    # length, so that grid neighbours a line apart share a variable
    "aniso2d_64_k2": (lambda L: O.RefMatrix.diffusion(L, 0.001, math.pi / 8, 64, 64), 2),
    "lap27_14_k2": (lambda L: O.RefMatrix.laplace27(L, 14, 14, 14), 2),
    "lap27_15_k3": (lambda L: O.RefMatrix.laplace27(L, 15, 15, 15), 3),
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
@pytest.mark.parametrize("coarsen", sorted(COARSEN))
@pytest.mark.parametrize("interp", sorted(INTERP))
def test_systems_hierarchy_matches_reference(prob, coarsen, interp):
    make, nv = PROBLEMS[prob]
    Ar = make(REF)
    A = rb_from_ref(Ar)
    ml = rb.ParRugeStubenSolver(0.25, COARSEN[coarsen], INTERP[interp], rb.Classical, rb.L1Jacobi)
    ml.num_variables = nv
    ml.setup(A)
    rml = O.RefHierarchy(Ar, theta=0.25, coarsen=coarsen, interp=interp, relax="jacobi",
                         num_variables=nv)
    for l in range(min(ml.num_levels, rml.num_levels)):
        for a, b, what in zip(ml.level_matrix(l, "A").arrays(), rml.A(l).arrays(),
                              ("rowptr", "cols", "vals")):
            np.testing.assert_array_equal(a, b, err_msg="A_%d %s" % (l, what))
        if l < min(ml.num_levels, rml.num_levels) - 1:
            np.testing.assert_array_equal(ml.level_states(l), rml.states(l), err_msg="states %d" % l)
            for a, b, what in zip(sorted_rows(*ml.level_matrix(l, "P").arrays()),
                                  sorted_rows(*rml.P(l).arrays()), ("rowptr", "cols", "vals")):
                np.testing.assert_array_equal(a, b, err_msg="P_%d %s" % (l, what))
    assert ml.num_levels == rml.num_levels, [ml.level_info(l) for l in range(ml.num_levels)]
    n = A.global_num_rows
    b = rb.ParVector(n, values=np.random.default_rng(5).uniform(-1, 1, n))
    x = rb.ParVector(n)
    res = []
    rc = rb.PCG(A, ml, x, b, res, tol=1e-8, max_iter=500, mode=rb.PCG_TRUE_RESIDUAL)
    assert rc == 0 and res[-1] <= 1e-8


def test_num_variables_is_validated():
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended)
    ml.num_variables = 0
    with pytest.raises(rb.RaptorError):
        ml.setup(rb.par_stencil_grid(rb.laplace_stencil_27pt(), [6, 6, 6]))
