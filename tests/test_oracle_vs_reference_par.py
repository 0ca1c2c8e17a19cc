"""The oracle against the reference's own parallel solve path at one rank.

oracle/build.py compiles the reference's parallel sources unmodified
(ParCSRMatrix, ParRugeStubenSolver, ParSmoothedAggregationSolver,
ParMultilevel, PCG, CG, BiCGStab) against a single-rank MPI stand-in and
OpenBLAS's dgetrf_/dgetrs_, once as they are and once with the Jacobi sweep
fixed (the reference's jacobi_helper never reads the diagonal, so its sweep
leaves x unchanged: raptor/util/linalg/par_relax.cpp:127-146).  These tests
run the reference and the C restatement on the same seeded inputs and require
every level's A_l and P_l (pattern, values and entry order) and C/F states to
be identical, and the residual histories to agree within 1e-10 relative.
Skipped where the reference build is absent.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

REF = O.par_ref()
REF_FIX = O.par_ref(jacobi_fix=True)
pytestmark = pytest.mark.skipif(REF is None or REF_FIX is None,
                                reason="reference parallel path not built here")

AMG_SEED = 20261203


def sort_rows(rp, ci, cv):
    ci, cv = np.array(ci), np.array(cv)
    for i in range(len(rp) - 1):
        o = np.argsort(ci[rp[i]:rp[i + 1]], kind="stable")
        ci[rp[i]:rp[i + 1]], cv[rp[i]:rp[i + 1]] = ci[rp[i]:rp[i + 1]][o], cv[rp[i]:rp[i + 1]][o]
    return rp, ci, cv


def assert_same_matrix(ref_mat, o_arrays, what, any_row_order=False):
    r = ref_mat.arrays()
    if any_row_order:
        r, o_arrays = sort_rows(*r), sort_rows(*o_arrays)
    for a, b, name in zip(r, o_arrays, ("rowptr", "cols", "vals")):
        np.testing.assert_array_equal(a, b, err_msg="%s %s" % (what, name))


def oracle_states(A, theta, weights, coarsen="pmis"):
    """The splitting ParRugeStubenSolver::extend_hierarchy computes for a level
    (raptor/ruge_stuben/par_ruge_stuben_solver.hpp:72-106), restated."""
    S = O.classical_strength(A, theta)
    n = A.shape[0]
    if coarsen == "pmis":
        return O.split_pmis(S, weights[:n])
    raise ValueError(coarsen)


def assert_same_hierarchy(rml, oml, theta, coarsen="pmis", states=True,
                          coarsest_any_order=False):
    """coarsest_any_order: the smoothed-aggregation solver leaves its coarsest
    A_c in the column order of the Galerkin product (no setup routine runs on
    it: raptor/aggregation/par_smoothed_aggregation_solver.hpp:95-103), where
    the oracle stores every level diagonal first; the coarse solve densifies
    A_c, so only the entries matter there."""
    assert rml.num_levels == oml.num_levels
    w = O.rand_weights(rml.A(0).shape[0])
    for l in range(rml.num_levels):
        last = l == rml.num_levels - 1
        assert_same_matrix(rml.A(l), oml.A(l).arrays(), "A_%d" % l,
                           any_row_order=coarsest_any_order and last)
        if l < rml.num_levels - 1:
            assert_same_matrix(rml.P(l), oml.P(l).arrays(), "P_%d" % l)
            if states:
                np.testing.assert_array_equal(rml.states(l), oracle_states(oml.A(l), theta, w,
                                                                           coarsen))


def rel_close(a, b, rtol):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    np.testing.assert_allclose(a, b, rtol=rtol, atol=0)


# --- configuration 1: 100^2 rotated anisotropic, PMIS, ModClassical, Jacobi ----

@pytest.fixture(scope="module")
def c1():
    eps, theta_rot = 0.001, math.pi / 8
    Ar = O.RefMatrix.diffusion(REF, eps, theta_rot, 100, 100)
    Af = O.RefMatrix.diffusion(REF_FIX, eps, theta_rot, 100, 100)
    Ao = O.stencil_grid(O.diffusion_stencil_2d(eps, theta_rot), [100, 100])
    return Ar, Af, Ao


def test_c1_stencil_matrix_identical(c1):
    Ar, _, Ao = c1
    assert_same_matrix(Ar, Ao.arrays(), "A")


@pytest.mark.parametrize("fixed", [False, True], ids=["as_is", "jacobi_fixed"])
def test_c1_hierarchy_and_solve_history(c1, fixed):
    Ar, Af, Ao = c1
    A = Af if fixed else Ar
    kw = dict(theta=0.25, coarsen="pmis", interp="mod_classical", relax="jacobi",
              relax_weight=2.0 / 3.0)
    rml = O.RefHierarchy(A, **kw)
    oml = O.Hierarchy(Ao, relax="jacobi", interp="mod_classical", relax_weight=2.0 / 3.0,
                      jacobi_compat=0 if fixed else 1)
    assert_same_hierarchy(rml, oml, 0.25)
    n = A.shape[0]
    b = A.spmv(np.ones(n))
    xr, itr, hr = rml.solve(np.zeros(n), b, tol=1e-8, max_iter=100)
    xo, ito, ho = oml.solve(np.zeros(n), b)
    assert itr == ito
    rel_close(hr, ho, 1e-10)
    np.testing.assert_allclose(xr, xo, rtol=1e-9, atol=1e-12)
    if fixed:
        assert hr[-1] < hr[0] * 1e-3  # a real smoother reduces the residual
    else:
        assert itr == 100  # the reference's no-op Jacobi stalls (coarse correction only)
    assert REF.rp_pending_messages() == 0


# --- 27-point Laplacian, PMIS, extended interpolation with filter 0.3 -------

@pytest.fixture(scope="module")
def lap27_24():
    return (O.RefMatrix.laplace27(REF, 24, 24, 24), O.RefMatrix.laplace27(REF_FIX, 24, 24, 24),
            O.stencil_grid(O.laplace_stencil_27pt(), [24, 24, 24]))


def test_lap27_extended_filter_hierarchy(lap27_24):
    Ar, _, Ao = lap27_24
    assert_same_matrix(Ar, Ao.arrays(), "A")
    rml = O.RefHierarchy(Ar, theta=0.25, coarsen="pmis", interp="extended", interp_filter=0.3,
                         relax="sor")
    oml = O.Hierarchy(Ao, relax="sor", interp="extended", interp_filter=0.3)
    assert rml.num_levels >= 3
    assert_same_hierarchy(rml, oml, 0.25)


@pytest.mark.parametrize("relax", ["jacobi", "sor", "ssor"])
def test_lap27_pcg_history(lap27_24, relax):
    """PCG (reference mode: its stopping rule, restart every 8 iterations)."""
    _, Af, Ao = lap27_24
    rml = O.RefHierarchy(Af, theta=0.25, coarsen="pmis", interp="extended", interp_filter=0.3,
                         relax=relax, relax_weight=(2.0 / 3.0 if relax == "jacobi" else 1.0))
    oml = O.Hierarchy(Ao, relax=relax, interp="extended", interp_filter=0.3,
                      relax_weight=(2.0 / 3.0 if relax == "jacobi" else 1.0))
    n = Af.shape[0]
    b = np.random.default_rng(AMG_SEED).uniform(-1, 1, n)
    xr, hr = O.ref_pcg(Af, rml, np.zeros(n), b, tol=1e-10, max_iter=200)
    xo, ho, _ = O.pcg(Ao, oml, np.zeros(n), b, tol=1e-10, max_iter=200)
    rel_close(hr, ho, 1e-10)
    np.testing.assert_allclose(xr, xo, rtol=1e-9, atol=1e-12)


def test_coarse_lu_solve_matches_dense_solve(lap27_24):
    """The reference's coarsest-level step (dgetrf_ at setup, dgetrs_ per
    cycle, of A_c^T) against numpy's dense solve, and the oracle's LU."""
    Ar, _, Ao = lap27_24
    rml = O.RefHierarchy(Ar, theta=0.25, coarsen="pmis", interp="extended", interp_filter=0.3)
    L = rml.num_levels - 1
    Ac = rml.A(L)
    nc = Ac.shape[0]
    rp, ci, cv = Ac.arrays()
    dense = np.zeros((nc, nc))
    for i in range(nc):
        dense[i, ci[rp[i]:rp[i + 1]]] = cv[rp[i]:rp[i + 1]]
    b = np.random.default_rng(5).uniform(-1, 1, nc)
    xr = rml.cycle(np.zeros(nc), b, level=L)
    # the reference hands its row-major A_c to column-major dgetrf_, so it
    # factors and solves with A_c^T
    xd = np.linalg.solve(dense.T, b)
    np.testing.assert_allclose(xr, xd, rtol=1e-12, atol=1e-14)
    lu = np.ascontiguousarray(dense.reshape(-1))  # column-major view of A_c^T
    piv = np.zeros(nc, np.int32)
    O.lib().oc_dense_lu(nc, lu, piv)
    xo = b.copy()
    O.lib().oc_dense_lu_solve(nc, lu, piv, xo)
    np.testing.assert_allclose(xo, xr, rtol=1e-12, atol=1e-14)


# --- smoothed aggregation ----------------------------------------------------

def test_sa_hierarchy_and_pcg():
    st = np.zeros(27)
    # 7-point anisotropic diffusion with coefficients (1, 1, 0.01) as a 3^3 array
    c = {(1, 1, 0): 0.01, (1, 1, 2): 0.01, (1, 0, 1): 1.0, (1, 2, 1): 1.0, (0, 1, 1): 1.0,
         (2, 1, 1): 1.0}
    for (i, j, k), v in c.items():
        st[i * 9 + j * 3 + k] = -v
    st[13] = 2 * (1 + 1 + 0.01)
    Ar = O.RefMatrix.stencil(REF, st, [16, 16, 16])
    Ao = O.stencil_grid(st, [16, 16, 16])
    assert_same_matrix(Ar, Ao.arrays(), "A")
    rml = O.RefHierarchy(Ar, solver="sa", theta=0.25, strength="symmetric", relax="sor")
    oml = O.Hierarchy(Ao, solver="sa", strong_threshold=0.25, relax="sor")
    assert rml.num_levels >= 3
    assert_same_hierarchy(rml, oml, 0.25, states=False, coarsest_any_order=True)
    n = Ar.shape[0]
    b = np.random.default_rng(AMG_SEED).uniform(-1, 1, n)
    xr, hr = O.ref_pcg(Ar, rml, np.zeros(n), b, tol=1e-10, max_iter=200)
    xo, ho, _ = O.pcg(Ao, oml, np.zeros(n), b, tol=1e-10, max_iter=200)
    rel_close(hr, ho, 1e-10)


# --- Krylov without a preconditioner, and the SpMV family --------------------

def test_cg_and_bicgstab_histories():
    Ar = O.RefMatrix.diffusion(REF, 0.001, math.pi / 8, 50, 50)
    Ao = O.stencil_grid(O.diffusion_stencil_2d(0.001, math.pi / 8), [50, 50])
    n = Ar.shape[0]
    b = np.random.default_rng(3).uniform(-1, 1, n)
    _, hr = O.ref_cg(Ar, np.zeros(n), b, tol=1e-8)
    _, ho = O.cg(Ao, np.zeros(n), b, tol=1e-8)
    rel_close(hr, ho, 1e-10)
    _, hr = O.ref_bicgstab(Ar, np.zeros(n), b, tol=1e-8)
    _, ho = O.bicgstab(Ao, np.zeros(n), b, tol=1e-8)
    rel_close(hr, ho, 1e-9)


def test_spmv_family(lap27_24):
    Ar, _, Ao = lap27_24
    n = Ar.shape[0]
    x = np.random.default_rng(1).uniform(-1, 1, n)
    b = np.random.default_rng(2).uniform(-1, 1, n)
    np.testing.assert_array_equal(Ar.spmv(x), O.spmv(Ao, x))
    np.testing.assert_array_equal(Ar.residual(x, b), O.residual(Ao, x, b))
    np.testing.assert_allclose(Ar.spmv_T(x), O.spmv_T(Ao, x), rtol=1e-14, atol=1e-14)


def test_hierarchy_from_levels_solves_like_setup(lap27_24):
    """The reference's ParMultilevel over levels handed to it (no setup;
    duplicate_coarse factors A_c) runs the same PCG as after its own setup:
    the form bench.py uses to time the reference's solve phase on a
    hierarchy the GPU built (bit-identical to the reference's, as the
    hierarchy tests show)."""
    Ar, _, _ = lap27_24
    kw = dict(theta=0.25, coarsen="pmis", interp="extended", interp_filter=0.3, relax="sor")
    rml = O.RefHierarchy(Ar, **kw)
    As = [rml.A(l).arrays() for l in range(rml.num_levels)]
    Ps = [(rml.A(l + 1).shape[0],) + tuple(rml.P(l).arrays()) for l in range(rml.num_levels - 1)]
    hml = O.RefHierarchy.from_levels(REF, As, Ps, **kw)
    assert hml.num_levels == rml.num_levels
    n = Ar.shape[0]
    b = np.random.default_rng(AMG_SEED).uniform(-1, 1, n)
    x1, h1 = O.ref_pcg(Ar, rml, np.zeros(n), b, tol=1e-10, max_iter=100)
    x2, h2 = O.ref_pcg(Ar, hml, np.zeros(n), b, tol=1e-10, max_iter=100)
    np.testing.assert_array_equal(h1, h2)
    np.testing.assert_array_equal(x1, x2)
