"""ctypes front end of the C oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs import this module.  It loads ``oracle/_build/libraptor_oracle.so``
(building it first when it is missing and gcc is available) and, where they
were built (oracle/build.py), the reference's own code:
``oracle/_ref/libraptor_seq_ref.so`` (sequential routines) and
``oracle/_ref/libraptor_par_ref{,_jfix}.so`` (the parallel solve path at one
rank; ``_jfix`` with the Jacobi sweep fixed).
"""
import contextlib
import ctypes as C
import os
import sys

import numpy as np

from . import build as _build

_I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_P = C.c_void_p

RELAX = {"jacobi": 0, "sor": 1, "ssor": 2, "l1_jacobi": 3, "mc_sor": 4, "mc_ssor": 5}
INTERP = {"direct": 0, "mod_classical": 1, "extended": 2}


class Opts(C.Structure):
    _fields_ = [
        ("solver", C.c_int), ("interp", C.c_int), ("relax", C.c_int),
        ("jacobi_compat", C.c_int), ("num_smooth_sweeps", C.c_int),
        ("max_coarse", C.c_int), ("max_levels", C.c_int), ("max_iterations", C.c_int),
        ("strong_threshold", C.c_double), ("relax_weight", C.c_double),
        ("solve_tol", C.c_double), ("interp_filter", C.c_double),
        ("prolong_weight", C.c_double), ("prolong_smooth_steps", C.c_int),
        ("seed_offset", C.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        so = _build.ORACLE_SO
        src = os.path.join(os.path.dirname(so), "..", "raptor_oracle.c")
        if not os.path.exists(so) or (os.path.exists(src) and
                                      os.path.getmtime(src) > os.path.getmtime(so)):
            _build.build_oracle()
        L = C.CDLL(so)
        L.oc_set_threads.argtypes = [C.c_int]
        L.oc_get_threads.restype = C.c_int
        L.oc_csr_new.restype = _P
        L.oc_csr_new.argtypes = [C.c_int, C.c_int, C.c_int, _I, _I, _D]
        L.oc_csr_free.argtypes = [_P]
        L.oc_csr_info.argtypes = [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.oc_csr_export.argtypes = [_P, _I, _I, _D]
        L.oc_csr_sort.argtypes = [_P]
        L.oc_csr_move_diag.argtypes = [_P]
        L.oc_diffusion_stencil_2d.argtypes = [C.c_double, C.c_double, _D]
        L.oc_laplace_stencil_27pt.argtypes = [_D]
        L.oc_stencil_grid.restype = _P
        L.oc_stencil_grid.argtypes = [_D, _I, C.c_int]
        for f in ("oc_spmv", "oc_spmv_T", "oc_spmv_append"):
            getattr(L, f).argtypes = [_P, _D, _D]
        L.oc_residual.argtypes = [_P, _D, _D, _D]
        L.oc_bsr_spmv.argtypes = [C.c_int, C.c_int, C.c_int, _I, _I, _D, _D, _D]
        L.oc_bsr_append.argtypes = [C.c_int, C.c_int, C.c_int, _I, _I, _D, _D, _D]
        L.oc_bsr_residual.argtypes = [C.c_int, C.c_int, C.c_int, _I, _I, _D, _D, _D, _D]
        L.oc_bsr_spmv_T.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _I, _I, _D, _D, _D]
        L.oc_bsr_to_csr.restype = _P
        L.oc_bsr_to_csr.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _I, _I, _D]
        L.oc_classical_strength.restype = _P
        L.oc_classical_strength.argtypes = [_P, C.c_double]
        L.oc_symmetric_strength.restype = _P
        L.oc_symmetric_strength.argtypes = [_P, C.c_double]
        L.oc_split_pmis.argtypes = [_P, _D, _I]
        L.oc_split_cljp.argtypes = [_P, _D, _I]
        L.oc_split_rs.argtypes = [_P, _I, C.c_int, C.c_int]
        L.oc_mis2.argtypes = [_P, _D, _I]
        L.oc_aggregate.restype = C.c_int
        L.oc_aggregate.argtypes = [_P, _P, _I, _I, C.c_void_p]
        L.oc_fit_candidates.restype = _P
        L.oc_fit_candidates.argtypes = [C.c_int, C.c_int, _I, _D, _D, C.c_double]
        L.oc_jacobi_prolongation.restype = _P
        L.oc_jacobi_prolongation.argtypes = [_P, _P, C.c_double, C.c_int]
        L.oc_mod_classical_interp.restype = _P
        L.oc_mod_classical_interp.argtypes = [_P, _P, _I]
        L.oc_direct_interp.restype = _P
        L.oc_direct_interp.argtypes = [_P, _P, _I]
        L.oc_extended_interp.restype = _P
        L.oc_extended_interp.argtypes = [_P, _P, _I, C.c_double]
        for f in ("oc_spgemm", "oc_spgemm_T"):
            getattr(L, f).restype = _P
            getattr(L, f).argtypes = [_P, _P]
        L.oc_rap.restype = _P
        L.oc_rap.argtypes = [_P, _P, C.c_int]
        L.oc_colour_rows.restype = C.c_int
        L.oc_colour_rows.argtypes = [_P, _I]
        L.oc_default_opts.argtypes = [C.POINTER(Opts)]
        L.oc_ml_setup.restype = _P
        L.oc_ml_setup.argtypes = [_P, C.POINTER(Opts), C.c_void_p, C.c_int]
        L.oc_ml_free.argtypes = [_P]
        L.oc_ml_num_levels.restype = C.c_int
        L.oc_ml_num_levels.argtypes = [_P]
        L.oc_ml_level_A.restype = _P
        L.oc_ml_level_A.argtypes = [_P, C.c_int]
        L.oc_ml_level_P.restype = _P
        L.oc_ml_level_P.argtypes = [_P, C.c_int]
        L.oc_ml_cycle.argtypes = [_P, _D, _D]
        L.oc_ml_solve.restype = C.c_int
        L.oc_ml_solve.argtypes = [_P, _D, _D, _D, C.c_int]
        L.oc_pcg.restype = C.c_int
        L.oc_pcg.argtypes = [_P, _P, _D, _D, C.c_double, C.c_int, _D, C.c_int]
        L.oc_pcg_mode.restype = C.c_int
        L.oc_pcg_mode.argtypes = [_P, _P, _D, _D, C.c_double, C.c_int, C.c_int, _D, C.c_int]
        L.oc_cg.restype = C.c_int
        L.oc_cg.argtypes = [_P, _D, _D, C.c_double, C.c_int, _D, C.c_int]
        L.oc_bicgstab.restype = C.c_int
        L.oc_bicgstab.argtypes = [_P, _D, _D, C.c_double, C.c_int, _D, C.c_int]
        L.oc_pre_bicgstab.restype = C.c_int
        L.oc_pre_bicgstab.argtypes = [_P, _P, _D, _D, C.c_double, C.c_int, _D, C.c_int]
        L.oc_form_rand_weights.argtypes = [C.c_int, C.c_int, _D]
        L.oc_dense_lu.argtypes = [C.c_int, _D, _I]
        L.oc_dense_lu_solve.argtypes = [C.c_int, _D, _I, _D]
        _lib = L
    return _lib


class CSR:
    """Owning handle on an oracle CSR matrix."""

    def __init__(self, ptr):
        self.ptr = ptr

    @classmethod
    def from_arrays(cls, n_rows, n_cols, rowptr, cols, vals):
        rp = np.ascontiguousarray(rowptr, dtype=np.int32)
        ci = np.ascontiguousarray(cols, dtype=np.int32)
        cv = np.ascontiguousarray(vals, dtype=np.float64)
        if len(ci) == 0:
            ci = np.zeros(1, np.int32)
            cv = np.zeros(1, np.float64)
        return cls(lib().oc_csr_new(int(n_rows), int(n_cols), int(rp[-1]), rp, ci, cv))

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.oc_csr_free(self.ptr)
            self.ptr = None

    @property
    def shape(self):
        r, c, z = C.c_int(), C.c_int(), C.c_int()
        lib().oc_csr_info(self.ptr, C.byref(r), C.byref(c), C.byref(z))
        return r.value, c.value, z.value

    def arrays(self):
        n, m, z = self.shape
        rp = np.zeros(n + 1, np.int32)
        ci = np.zeros(max(z, 1), np.int32)
        cv = np.zeros(max(z, 1), np.float64)
        lib().oc_csr_export(self.ptr, rp, ci, cv)
        return rp, ci[:z], cv[:z]

    def to_scipy(self):
        import scipy.sparse as sp
        n, m, _ = self.shape
        rp, ci, cv = self.arrays()
        return sp.csr_matrix((cv, ci, rp), shape=(n, m))


class Borrowed(CSR):
    """CSR owned by an oracle hierarchy (not freed here)."""

    def __del__(self):
        pass


def set_threads(n):
    """Threads for the oracle's row-parallel loops (results are the same
    for any count; see oc_set_threads)."""
    lib().oc_set_threads(int(n))


def get_threads():
    return int(lib().oc_get_threads())


def stencil_grid(stencil, grid):
    st = np.ascontiguousarray(stencil, np.float64)
    g = np.ascontiguousarray(grid, np.int32)
    return CSR(lib().oc_stencil_grid(st, g, len(g)))


def diffusion_stencil_2d(eps=1.0, theta=0.0):
    out = np.zeros(9)
    lib().oc_diffusion_stencil_2d(eps, theta, out)
    return out


def laplace_stencil_27pt():
    out = np.zeros(27)
    lib().oc_laplace_stencil_27pt(out)
    return out


def spmv(A, x):
    b = np.zeros(A.shape[0])
    lib().oc_spmv(A.ptr, np.ascontiguousarray(x, np.float64), b)
    return b


def spmv_T(A, x):
    b = np.zeros(A.shape[1])
    lib().oc_spmv_T(A.ptr, np.ascontiguousarray(x, np.float64), b)
    return b


def residual(A, x, b):
    r = np.zeros(A.shape[0])
    lib().oc_residual(A.ptr, np.ascontiguousarray(x, np.float64),
                      np.ascontiguousarray(b, np.float64), r)
    return r


class BSR:
    """Host block CSR: n_rows x n_cols blocks of b_rows x b_cols values,
    blocks as an (nnz, b_rows, b_cols) array (core/matrix.hpp:962-1060)."""

    def __init__(self, n_rows, n_cols, b_rows, b_cols, rowptr, cols, blocks):
        self.n_rows, self.n_cols = int(n_rows), int(n_cols)
        self.b_rows, self.b_cols = int(b_rows), int(b_cols)
        self.rowptr = np.ascontiguousarray(rowptr, np.int32)
        self.cols = np.ascontiguousarray(cols, np.int32)
        self.blocks = np.ascontiguousarray(blocks, np.float64).reshape(
            len(self.cols), self.b_rows, self.b_cols)

    @property
    def shape(self):
        return self.n_rows * self.b_rows, self.n_cols * self.b_cols

    def _args(self):
        v = self.blocks.reshape(-1) if self.blocks.size else np.zeros(1)
        c = self.cols if self.cols.size else np.zeros(1, np.int32)
        return self.rowptr, c, np.ascontiguousarray(v)


def bsr_spmv(A, x):
    b = np.zeros(A.shape[0])
    lib().oc_bsr_spmv(A.n_rows, A.b_rows, A.b_cols, *A._args(),
                      np.ascontiguousarray(x, np.float64), b)
    return b


def bsr_append(A, x, b):
    out = np.array(b, dtype=np.float64)
    lib().oc_bsr_append(A.n_rows, A.b_rows, A.b_cols, *A._args(),
                        np.ascontiguousarray(x, np.float64), out)
    return out


def bsr_residual(A, x, b):
    r = np.zeros(A.shape[0])
    lib().oc_bsr_residual(A.n_rows, A.b_rows, A.b_cols, *A._args(),
                          np.ascontiguousarray(x, np.float64),
                          np.ascontiguousarray(b, np.float64), r)
    return r


def bsr_spmv_T(A, x):
    b = np.zeros(A.shape[1])
    lib().oc_bsr_spmv_T(A.n_rows, A.n_cols, A.b_rows, A.b_cols, *A._args(),
                        np.ascontiguousarray(x, np.float64), b)
    return b


def bsr_to_csr(A):
    return CSR(lib().oc_bsr_to_csr(A.n_rows, A.n_cols, A.b_rows, A.b_cols, *A._args()))


def sort_diag_first(A):
    lib().oc_csr_sort(A.ptr)
    lib().oc_csr_move_diag(A.ptr)
    return A


def classical_strength(A, theta):
    return CSR(lib().oc_classical_strength(A.ptr, theta))


def symmetric_strength(A, theta):
    return CSR(lib().oc_symmetric_strength(A.ptr, theta))


def split_pmis(S, weights):
    st = np.zeros(S.shape[0], np.int32)
    lib().oc_split_pmis(S.ptr, np.ascontiguousarray(weights[: S.shape[0]], np.float64), st)
    return st


def split_cljp(S, weights):
    st = np.zeros(max(S.shape[0], 1), np.int32)
    lib().oc_split_cljp(S.ptr, np.ascontiguousarray(weights[: S.shape[0]], np.float64), st)
    return st[: S.shape[0]]


def split_rs(S, second_pass=True, states=None):
    """RS splitting; with states given they are kept where assigned (the
    parallel driver's NoNeighbors), else every point starts unassigned."""
    n = S.shape[0]
    st = np.zeros(max(n, 1), np.int32)
    if states is not None:
        st[:n] = states
    lib().oc_split_rs(S.ptr, st, int(states is not None), int(second_pass))
    return st[:n]


def mis2(S, weights):
    st = np.zeros(S.shape[0], np.int32)
    lib().oc_mis2(S.ptr, np.ascontiguousarray(weights[: S.shape[0]], np.float64), st)
    return st


def aggregate(A, S, states, r=None):
    agg = np.zeros(S.shape[0], np.int32)
    st = np.ascontiguousarray(states, np.int32).copy()
    rr = None
    if r is not None:
        rr = np.ascontiguousarray(r, np.float64)
    n_aggs = lib().oc_aggregate(A.ptr, S.ptr, st, agg,
                                rr.ctypes.data_as(C.c_void_p) if rr is not None else None)
    return n_aggs, agg


def fit_candidates(n, n_aggs, agg, B):
    R = np.zeros(max(n_aggs, 1))
    T = CSR(lib().oc_fit_candidates(n, n_aggs, np.ascontiguousarray(agg, np.int32),
                                    np.ascontiguousarray(B, np.float64), R, 1e-10))
    return T, R[:n_aggs]


def jacobi_prolongation(A, T, omega=4.0 / 3, steps=1):
    return CSR(lib().oc_jacobi_prolongation(A.ptr, T.ptr, omega, steps))


def interpolation(A, S, states, kind="mod_classical", filt=0.0):
    st = np.ascontiguousarray(states, np.int32)
    if kind == "extended":
        return CSR(lib().oc_extended_interp(A.ptr, S.ptr, st, filt))
    if kind == "direct":
        return CSR(lib().oc_direct_interp(A.ptr, S.ptr, st))
    return CSR(lib().oc_mod_classical_interp(A.ptr, S.ptr, st))


def spgemm(A, B):
    return CSR(lib().oc_spgemm(A.ptr, B.ptr))


def spgemm_T(P, B):
    """P^T B with P's columns walked in increasing row order (matmult.cpp:139-204)."""
    return CSR(lib().oc_spgemm_T(P.ptr, B.ptr))


def rap(A, P, diag_first=True):
    return CSR(lib().oc_rap(A.ptr, P.ptr, 1 if diag_first else 0))


def colour_rows(A):
    c = np.zeros(A.shape[0], np.int32)
    nc = lib().oc_colour_rows(A.ptr, c)
    return nc, c


def rand_weights(n, first_row=0):
    w = np.zeros(max(n, 1))
    lib().oc_form_rand_weights(n, first_row, w)
    return w[:n]


def default_opts(**kw):
    o = Opts()
    lib().oc_default_opts(C.byref(o))
    for k, v in kw.items():
        if k == "relax" and isinstance(v, str):
            v = RELAX[v]
        if k == "interp" and isinstance(v, str):
            v = INTERP[v]
        if k == "solver" and isinstance(v, str):
            v = {"rs": 0, "sa": 1}[v]
        setattr(o, k, v)
    return o


class Hierarchy:
    """An oracle AMG hierarchy (ParMultilevel restated)."""

    def __init__(self, A, weights=None, **kw):
        self.opts = default_opts(**kw)
        w = None
        nw = 0
        if weights is not None:
            self._w = np.ascontiguousarray(weights, np.float64)
            w = self._w.ctypes.data_as(C.c_void_p)
            nw = len(self._w)
        self.ptr = lib().oc_ml_setup(A.ptr, C.byref(self.opts), w, nw)
        self.n = A.shape[0]

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.oc_ml_free(self.ptr)
            self.ptr = None

    @property
    def num_levels(self):
        return lib().oc_ml_num_levels(self.ptr)

    def A(self, l):
        return Borrowed(lib().oc_ml_level_A(self.ptr, l))

    def P(self, l):
        return Borrowed(lib().oc_ml_level_P(self.ptr, l))

    def cycle(self, x, b):
        x = np.ascontiguousarray(x, np.float64).copy()
        lib().oc_ml_cycle(self.ptr, x, np.ascontiguousarray(b, np.float64))
        return x

    def solve(self, x, b, cap=1000):
        x = np.ascontiguousarray(x, np.float64).copy()
        hist = np.zeros(cap)
        it = lib().oc_ml_solve(self.ptr, x, np.ascontiguousarray(b, np.float64), hist, cap)
        return x, it, hist[: min(it + 1, cap)]


def pcg(A, ml, x, b, tol=1e-5, max_iter=-1, cap=10000, mode=0):
    """mode 0: the reference's PCG; mode 1: stop on the true relative residual."""
    x = np.ascontiguousarray(x, np.float64).copy()
    hist = np.zeros(cap)
    if max_iter <= 0:
        max_iter = int(1.3 * A.shape[0]) + 2
    nh = lib().oc_pcg_mode(A.ptr, ml.ptr, x, np.ascontiguousarray(b, np.float64), tol, max_iter,
                           mode, hist, cap)
    return x, hist[: min(abs(nh), cap)], nh


def cg(A, x, b, tol=1e-5, max_iter=-1, cap=10000):
    x = np.ascontiguousarray(x, np.float64).copy()
    hist = np.zeros(cap)
    nh = lib().oc_cg(A.ptr, x, np.ascontiguousarray(b, np.float64), tol, max_iter, hist, cap)
    return x, hist[: min(abs(nh), cap)]


def bicgstab(A, x, b, tol=1e-5, max_iter=-1, cap=10000, ml=None):
    x = np.ascontiguousarray(x, np.float64).copy()
    hist = np.zeros(cap)
    if ml is None:
        nh = lib().oc_bicgstab(A.ptr, x, np.ascontiguousarray(b, np.float64), tol, max_iter,
                               hist, cap)
    else:
        nh = lib().oc_pre_bicgstab(A.ptr, ml.ptr, x, np.ascontiguousarray(b, np.float64), tol,
                                   max_iter, hist, cap)
    return x, hist[: min(abs(nh), cap)]


# --- the reference's own sequential routines (build container only) --------

_ref = None


def ref_lib():
    """The reference's sequential sources compiled under oracle/_ref, or None."""
    global _ref
    if _ref is None:
        so = _build.REF_SO
        if not os.path.exists(so):
            try:
                so = _build.build_reference()
            except Exception:  # noqa: BLE001 - no compiler or no checkout
                so = None
        if not so or not os.path.exists(so):
            return None
        L = C.CDLL(so)
        L.rs_free.argtypes = [_P]
        L.rs_info.argtypes = [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.rs_export.argtypes = [_P, _I, _I, _D]
        L.rs_spmv.argtypes = [C.c_int, C.c_int, _I, _I, _D, _D, _D]
        L.rs_residual.argtypes = [C.c_int, C.c_int, _I, _I, _D, _D, _D, _D]
        for f in ("rs_spgemm", "rs_spgemm_T"):
            getattr(L, f).restype = _P
            getattr(L, f).argtypes = [C.c_int, C.c_int, _I, _I, _D, C.c_int, C.c_int, _I, _I, _D]
        L.rs_strength.restype = _P
        L.rs_strength.argtypes = [C.c_int, _I, _I, _D, C.c_double, C.c_int]
        L.rs_split_pmis.argtypes = [C.c_int, _I, _I, _D, _D, _I]
        L.rs_split_cljp.argtypes = [C.c_int, _I, _I, _D, _D, _I]
        L.rs_split_rs.argtypes = [C.c_int, _I, _I, _D, C.c_int, _I]
        L.rs_mis2.argtypes = [C.c_int, _I, _I, _D, _D, _I]
        L.rs_bsr_apply.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _I, _I, _D, C.c_int, _D,
                                   _D, _D]
        L.rs_bsr_to_csr.restype = _P
        L.rs_bsr_to_csr.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _I, _I, _D]
        L.rs_bsr_sort_diag_first.restype = C.c_int
        L.rs_bsr_sort_diag_first.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _I, _I, _D, _I,
                                             _I, _D]
        L.rs_bcoo_to_bsr.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _I, _I, _D, _I,
                                     _I, _D]
        L.rs_interp.restype = _P
        L.rs_interp.argtypes = [C.c_int, _I, _I, _D, _I, _I, _D, _I, C.c_int]
        _ref = L
    return _ref


def ref_take(ptr):
    """Copy a shim result into numpy arrays and free it."""
    L = ref_lib()
    r, c, z = C.c_int(), C.c_int(), C.c_int()
    L.rs_info(ptr, C.byref(r), C.byref(c), C.byref(z))
    rp = np.zeros(r.value + 1, np.int32)
    ci = np.zeros(max(z.value, 1), np.int32)
    cv = np.zeros(max(z.value, 1), np.float64)
    L.rs_export(ptr, rp, ci, cv)
    L.rs_free(ptr)
    return (r.value, c.value), rp, ci[: z.value], cv[: z.value]


# --- the reference's own parallel solve path (oracle/_ref/libraptor_par_ref*.so)

# the reference's enums (raptor/core/types.hpp:156-162)
REF_COARSEN = {"rs": 0, "cljp": 1, "falgout": 2, "pmis": 3, "hmis": 4}
REF_INTERP = {"direct": 0, "mod_classical": 1, "extended": 2}
REF_RELAX = {"jacobi": 0, "sor": 1, "ssor": 2}
REF_STRENGTH = {"classical": 0, "symmetric": 1}


class RefOpts(C.Structure):
    _fields_ = [
        ("solver", C.c_int), ("theta", C.c_double), ("coarsen", C.c_int),
        ("interp", C.c_int), ("strength", C.c_int), ("relax", C.c_int),
        ("relax_weight", C.c_double), ("num_smooth_sweeps", C.c_int),
        ("interp_filter", C.c_double), ("max_coarse", C.c_int), ("max_levels", C.c_int),
        ("num_variables", C.c_int),
    ]


_par = {}


def par_ref(jacobi_fix=False):
    """The reference's parallel path compiled at one rank, or None if not built."""
    key = bool(jacobi_fix)
    if key in _par:
        return _par[key]
    so = _build.PAR_JFIX_SO if key else _build.PAR_SO
    if not os.path.exists(so):
        try:
            _build.build_reference_parallel()
        except Exception:  # noqa: BLE001 - no compiler, checkout or OpenBLAS
            pass
    if not os.path.exists(so):
        _par[key] = None
        return None
    L = C.CDLL(so)
    L.rp_matrix_from_csr.restype = _P
    L.rp_matrix_from_csr.argtypes = [C.c_int, C.c_int, _I, _I, _D, C.c_int, C.c_int, C.c_int]
    L.rp_matrix_flags.argtypes = [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.rp_hierarchy_from_levels.restype = _P
    L.rp_hierarchy_from_levels.argtypes = [C.c_int, C.POINTER(_P), C.POINTER(_P),
                                           C.POINTER(RefOpts)]
    L.rp_diffusion_grid.restype = _P
    L.rp_diffusion_grid.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int]
    L.rp_laplace27_grid.restype = _P
    L.rp_laplace27_grid.argtypes = [C.c_int, C.c_int, C.c_int]
    L.rp_stencil_grid.restype = _P
    L.rp_stencil_grid.argtypes = [_D, _I, C.c_int]
    L.rp_matrix_free.argtypes = [_P]
    L.rp_matrix_info.argtypes = [_P, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.POINTER(C.c_longlong)]
    L.rp_matrix_export.restype = C.c_int
    L.rp_matrix_export.argtypes = [_P, _I, _I, _D]
    L.rp_spmv.argtypes = [_P, _D, _D]
    L.rp_spmv_T.argtypes = [_P, _D, _D]
    L.rp_residual.argtypes = [_P, _D, _D, _D]
    L.rp_default_opts.argtypes = [C.POINTER(RefOpts)]
    L.rp_last_error.restype = C.c_char_p
    L.rp_setup.restype = _P
    L.rp_setup.argtypes = [_P, C.POINTER(RefOpts)]
    L.rp_free.argtypes = [_P]
    L.rp_num_levels.restype = C.c_int
    L.rp_num_levels.argtypes = [_P]
    L.rp_level.restype = _P
    L.rp_level.argtypes = [_P, C.c_int, C.c_int]
    L.rp_level_states.restype = C.c_int
    L.rp_level_states.argtypes = [_P, C.c_int, _I]
    L.rp_solve.restype = C.c_int
    L.rp_solve.argtypes = [_P, _D, _D, C.c_double, C.c_int, _D, C.c_int]
    L.rp_cycle.argtypes = [_P, _D, _D, C.c_int]
    L.rp_pcg.restype = C.c_int
    L.rp_pcg.argtypes = [_P, _P, _D, _D, C.c_double, C.c_int, _D, C.c_int]
    L.rp_cg.restype = C.c_int
    L.rp_cg.argtypes = [_P, _D, _D, C.c_double, C.c_int, _D, C.c_int]
    L.rp_bicgstab.restype = C.c_int
    L.rp_bicgstab.argtypes = [_P, _D, _D, C.c_double, C.c_int, _D, C.c_int]
    L.rp_pending_messages.restype = C.c_int
    _par[key] = L
    return L


@contextlib.contextmanager
def quiet_stdout():
    """Send the C library's stdout to stderr (the reference's PCG and
    BiCGStab print their iteration counts with printf)."""
    libc = C.CDLL(None)
    sys.stdout.flush()
    libc.fflush(None)
    saved = os.dup(1)
    try:
        os.dup2(2, 1)
        yield
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)


def _ref_arrays(L, ptr):
    r, c, z = C.c_int(), C.c_int(), C.c_longlong()
    L.rp_matrix_info(ptr, C.byref(r), C.byref(c), C.byref(z))
    rp = np.zeros(r.value + 1, np.int32)
    ci = np.zeros(max(z.value, 1), np.int32)
    cv = np.zeros(max(z.value, 1), np.float64)
    if L.rp_matrix_export(ptr, rp, ci, cv) != 0:
        raise RuntimeError("reference matrix has off-process entries at one rank")
    return (r.value, c.value), rp, ci[: z.value], cv[: z.value]


class RefMatrix:
    """A reference ParCSRMatrix (owned unless borrowed from a hierarchy)."""

    def __init__(self, L, ptr, owner=None):
        self.L, self.ptr, self._owner = L, ptr, owner

    @classmethod
    def from_csr(cls, L, rowptr, cols, vals, n_cols=None):
        rp = np.ascontiguousarray(rowptr, np.int32)
        n = len(rp) - 1
        return cls(L, L.rp_matrix_from_csr(n, n if n_cols is None else n_cols, rp,
                                           np.ascontiguousarray(cols, np.int32),
                                           np.ascontiguousarray(vals, np.float64), 0, 0, 0))

    def flags(self):
        """(sorted, diag_first) of the on-process block."""
        a, b = C.c_int(), C.c_int()
        self.L.rp_matrix_flags(self.ptr, C.byref(a), C.byref(b))
        return a.value, b.value

    @classmethod
    def diffusion(cls, L, eps, theta, nx, ny):
        return cls(L, L.rp_diffusion_grid(eps, theta, nx, ny))

    @classmethod
    def laplace27(cls, L, nx, ny, nz):
        return cls(L, L.rp_laplace27_grid(nx, ny, nz))

    @classmethod
    def stencil(cls, L, stencil, grid):
        return cls(L, L.rp_stencil_grid(np.ascontiguousarray(stencil, np.float64),
                                        np.ascontiguousarray(grid, np.int32), len(grid)))

    def __del__(self):
        if self._owner is None and getattr(self, "ptr", None):
            self.L.rp_matrix_free(self.ptr)
            self.ptr = None

    @property
    def shape(self):
        r, c, z = C.c_int(), C.c_int(), C.c_longlong()
        self.L.rp_matrix_info(self.ptr, C.byref(r), C.byref(c), C.byref(z))
        return r.value, c.value, z.value

    def arrays(self):
        return _ref_arrays(self.L, self.ptr)[1:]

    def spmv(self, x):
        y = np.zeros(self.shape[0])
        self.L.rp_spmv(self.ptr, np.ascontiguousarray(x, np.float64), y)
        return y

    def spmv_T(self, x):
        y = np.zeros(self.shape[1])
        self.L.rp_spmv_T(self.ptr, np.ascontiguousarray(x, np.float64), y)
        return y

    def residual(self, x, b):
        r = np.zeros(self.shape[0])
        self.L.rp_residual(self.ptr, np.ascontiguousarray(x, np.float64),
                           np.ascontiguousarray(b, np.float64), r)
        return r


def ref_opts(L, **kw):
    """Options of the reference's solver classes; strings name its enums."""
    o = RefOpts()
    L.rp_default_opts(C.byref(o))
    maps = {"coarsen": REF_COARSEN, "interp": REF_INTERP, "relax": REF_RELAX,
            "strength": REF_STRENGTH, "solver": {"rs": 0, "sa": 1}}
    for k, v in kw.items():
        if isinstance(v, str):
            v = maps[k][v]
        setattr(o, k, v)
    return o


class RefHierarchy:
    """ml = new ParRugeStubenSolver / ParSmoothedAggregationSolver; ml->setup(A)."""

    def __init__(self, A, **kw):
        self.L = A.L
        self.opts = ref_opts(self.L, **kw)
        self.A0 = A
        self.ptr = self.L.rp_setup(A.ptr, C.byref(self.opts))
        if not self.ptr:
            raise RuntimeError("reference setup failed: %s" % self.L.rp_last_error().decode())

    @classmethod
    def from_levels(cls, L, As, Ps, A_flags=(1, 1), **kw):
        """The reference's hierarchy object over given levels: As[l] =
        (rowptr, cols, vals) of A_l in its entry order (diagonal first, as
        setup leaves every level; A_flags are its sorted / diag_first flags),
        Ps[l] = (n_cols, rowptr, cols, vals) of P_l in its entry order; no
        setup runs (duplicate_coarse factors A_c as setup would)."""
        self = cls.__new__(cls)
        self.L = L
        self.opts = ref_opts(L, **kw)
        nl = len(As)
        a_ptrs = (_P * nl)()
        p_ptrs = (_P * max(nl - 1, 1))()
        for l, (rp, ci, cv) in enumerate(As):
            n = len(rp) - 1
            a_ptrs[l] = L.rp_matrix_from_csr(n, n, np.ascontiguousarray(rp, np.int32),
                                             np.ascontiguousarray(ci, np.int32),
                                             np.ascontiguousarray(cv, np.float64), 1,
                                             A_flags[0], A_flags[1])
        for l, (m, rp, ci, cv) in enumerate(Ps):
            p_ptrs[l] = L.rp_matrix_from_csr(len(rp) - 1, m, np.ascontiguousarray(rp, np.int32),
                                             np.ascontiguousarray(ci, np.int32),
                                             np.ascontiguousarray(cv, np.float64), 1, 0, 0)
        self.ptr = L.rp_hierarchy_from_levels(nl, a_ptrs, p_ptrs, C.byref(self.opts))
        self.A0 = self.A(0)
        return self

    def __del__(self):
        if getattr(self, "ptr", None):
            self.L.rp_free(self.ptr)
            self.ptr = None

    @property
    def num_levels(self):
        return self.L.rp_num_levels(self.ptr)

    def A(self, l):
        return RefMatrix(self.L, self.L.rp_level(self.ptr, l, 0), owner=self)

    def P(self, l):
        return RefMatrix(self.L, self.L.rp_level(self.ptr, l, 1), owner=self)

    def states(self, l):
        n = self.A(l).shape[0]
        st = np.zeros(max(n, 1), np.int32)
        if self.L.rp_level_states(self.ptr, l, st) < 0:
            raise ValueError("states exist for Ruge-Stuben levels above the coarsest")
        return st[:n]

    def solve(self, x, b, tol=1e-8, max_iter=100):
        x = np.ascontiguousarray(x, np.float64).copy()
        hist = np.zeros(max_iter + 1)
        it = self.L.rp_solve(self.ptr, x, np.ascontiguousarray(b, np.float64), tol, max_iter,
                             hist, len(hist))
        return x, it, hist[: it + 1]

    def cycle(self, x, b, level=0):
        x = np.ascontiguousarray(x, np.float64).copy()
        self.L.rp_cycle(self.ptr, x, np.ascontiguousarray(b, np.float64), level)
        return x


def ref_pcg(A, ml, x, b, tol=1e-5, max_iter=-1, cap=10000):
    """The reference's PCG(A, ml, x, b, res, tol, max_iter)."""
    x = np.ascontiguousarray(x, np.float64).copy()
    hist = np.zeros(cap)
    with quiet_stdout():
        nh = A.L.rp_pcg(A.ptr, ml.ptr, x, np.ascontiguousarray(b, np.float64), tol, max_iter,
                        hist, cap)
    return x, hist[: min(nh, cap)]


def ref_cg(A, x, b, tol=1e-5, max_iter=-1, cap=10000):
    x = np.ascontiguousarray(x, np.float64).copy()
    hist = np.zeros(cap)
    with quiet_stdout():
        nh = A.L.rp_cg(A.ptr, x, np.ascontiguousarray(b, np.float64), tol, max_iter, hist, cap)
    return x, hist[: min(nh, cap)]


def ref_bicgstab(A, x, b, tol=1e-5, max_iter=-1, cap=10000):
    x = np.ascontiguousarray(x, np.float64).copy()
    hist = np.zeros(cap)
    with quiet_stdout():
        nh = A.L.rp_bicgstab(A.ptr, x, np.ascontiguousarray(b, np.float64), tol, max_iter, hist,
                             cap)
    return x, hist[: min(nh, cap)]
