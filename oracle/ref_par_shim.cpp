// ref_par_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C-callable shim over the reference's own *parallel* solve path
// (13manan/raptor: ParCSRMatrix, ParRugeStubenSolver / ParSmoothedAggregation
// Solver, ParMultilevel::setup / cycle / solve, PCG, CG, BiCGStab), compiled
// unmodified from its sources by oracle/build.py into oracle/_ref/ and linked
// against the single-rank MPI stand-in in oracle/mpi_stub/ and the LAPACK
// dgetrf_/dgetrs_ of an OpenBLAS shipped with the Python environment.  At one
// rank every ParCSRMatrix has an empty off_proc block, so its on_proc block,
// with local column indices, is the whole matrix.
//
// The tests use it to pin the C restatement (raptor_oracle.c) and the GPU
// library on the reference's own run: per-level A_l, P_l and C/F states of the
// hierarchy the reference builds, and the residual histories of its solve,
// PCG and BiCGStab on the same inputs.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "core/types.hpp"
#include "core/par_matrix.hpp"
#include "core/par_vector.hpp"
#include "gallery/diffusion.hpp"
#include "gallery/laplacian27pt.hpp"
#include "gallery/par_stencil.hpp"
#include "krylov/par_bicgstab.hpp"
#include "krylov/par_cg.hpp"
#include "multilevel/par_multilevel.hpp"
#include "ruge_stuben/par_cf_splitting.hpp"
#include "ruge_stuben/par_ruge_stuben_solver.hpp"
#include "aggregation/par_smoothed_aggregation_solver.hpp"

extern "C" int mpi_stub_pending_messages(void);

using namespace raptor;

extern "C" {

struct rp_opts {
    int solver;           // 0 Ruge-Stuben, 1 smoothed aggregation
    double theta;         // strong threshold
    int coarsen;          // coarsen_t: RS, CLJP, Falgout, PMIS, HMIS
    int interp;           // interp_t: Direct, ModClassical, Extended
    int strength;         // strength_t: Classical, Symmetric
    int relax;            // relax_t: Jacobi, SOR, SSOR
    double relax_weight;
    int num_smooth_sweeps;
    double interp_filter;
    int max_coarse;
    int max_levels;
    int num_variables;    // ParMultilevel::num_variables (RS solver: the systems form)
};

}  // extern "C"

namespace {

struct Solver {
    ParMultilevel* ml;
    rp_opts o;
    int n0;
};

std::string g_error;

void set_vec(ParVector& v, const double* a) {
    for (int i = 0; i < v.local_n; i++) v.local[i] = a[i];
}

void get_vec(ParVector& v, double* a) {
    for (int i = 0; i < v.local_n; i++) a[i] = v.local[i];
}

int copy_hist(const aligned_vector<double>& h, int n, double* hist, int cap) {
    for (int i = 0; i < n && i < cap; i++) hist[i] = h[i];
    return n;
}

}  // namespace

extern "C" {

// A ParCSRMatrix with n rows and m columns holding the given rows
// (finalize sorts each row by column, as every reference constructor does).
// keep_order puts the caller's entry order back afterwards, with the
// matrix's sorted / diag_first flags set as given: a level exported from a
// hierarchy then sums its rows in the order the hierarchy did.
void* rp_matrix_from_csr(int n, int m, const int* rowptr, const int* cols, const double* vals,
                         int keep_order, int sorted, int diag_first) {
    ParCSRMatrix* A = new ParCSRMatrix(n, m);
    int nnz = rowptr[n];
    A->on_proc->n_rows = n;
    A->on_proc->n_cols = m;
    A->on_proc->idx1.assign(rowptr, rowptr + n + 1);
    A->on_proc->idx2.assign(cols, cols + nnz);
    A->on_proc->vals.assign(vals, vals + nnz);
    A->on_proc->nnz = nnz;
    A->off_proc->n_rows = n;
    A->off_proc->n_cols = m;
    A->off_proc->idx1.assign(n + 1, 0);
    A->off_proc->nnz = 0;
    A->finalize();
    if (keep_order) {
        A->on_proc->idx2.assign(cols, cols + nnz);
        A->on_proc->vals.assign(vals, vals + nnz);
        A->on_proc->sorted = sorted != 0;
        A->on_proc->diag_first = diag_first != 0;
    }
    return A;
}

void rp_matrix_flags(void* p, int* sorted, int* diag_first) {
    ParCSRMatrix* A = (ParCSRMatrix*)p;
    *sorted = A->on_proc->sorted ? 1 : 0;
    *diag_first = A->on_proc->diag_first ? 1 : 0;
}

// par_stencil_grid(diffusion_stencil_2d(eps, theta), {nx, ny}, 2)
void* rp_diffusion_grid(double eps, double theta, int nx, int ny) {
    int grid[2] = {nx, ny};
    data_t* st = diffusion_stencil_2d(eps, theta);
    ParCSRMatrix* A = par_stencil_grid(st, grid, 2);
    delete[] st;
    return A;
}

// par_stencil_grid(laplace_stencil_27pt(), {nx, ny, nz}, 3)
void* rp_laplace27_grid(int nx, int ny, int nz) {
    int grid[3] = {nx, ny, nz};
    data_t* st = laplace_stencil_27pt();
    ParCSRMatrix* A = par_stencil_grid(st, grid, 3);
    delete[] st;
    return A;
}

// par_stencil_grid with a caller's 3^dim stencil.
void* rp_stencil_grid(const double* stencil, const int* grid, int dim) {
    int len = 1;
    for (int d = 0; d < dim; d++) len *= 3;
    data_t* st = new data_t[len];
    for (int i = 0; i < len; i++) st[i] = stencil[i];
    int g[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) g[d] = grid[d];
    ParCSRMatrix* A = par_stencil_grid(st, g, dim);
    delete[] st;
    return A;
}

void rp_matrix_free(void* A) { delete (ParCSRMatrix*)A; }

void rp_matrix_info(void* p, int* n_rows, int* n_cols, long long* nnz) {
    ParCSRMatrix* A = (ParCSRMatrix*)p;
    *n_rows = A->global_num_rows;
    *n_cols = A->on_proc_num_cols;
    *nnz = (long long)A->on_proc->idx1[A->local_num_rows];
}

// Rows in the matrix's own entry order, with on_proc's local column indices
// (the positions in the ParVector that a product with this matrix reads; at
// one rank they number every column).  Returns -1, writing nothing, if the
// off_proc block holds entries (it cannot at one rank).
int rp_matrix_export(void* p, int* rowptr, int* cols, double* vals) {
    ParCSRMatrix* A = (ParCSRMatrix*)p;
    if (A->off_proc->nnz) return -1;
    int n = A->local_num_rows;
    long long k = 0;
    rowptr[0] = 0;
    for (int i = 0; i < n; i++) {
        for (int j = A->on_proc->idx1[i]; j < A->on_proc->idx1[i + 1]; j++) {
            cols[k] = A->on_proc->idx2[j];
            vals[k++] = A->on_proc->vals[j];
        }
        rowptr[i + 1] = (int)k;
    }
    return 0;
}

void rp_spmv(void* p, const double* x, double* b) {
    ParCSRMatrix* A = (ParCSRMatrix*)p;
    ParVector vx(A->global_num_cols, A->on_proc_num_cols), vb(A->global_num_rows, A->local_num_rows);
    set_vec(vx, x);
    A->mult(vx, vb);
    get_vec(vb, b);
}

void rp_residual(void* p, const double* x, const double* b, double* r) {
    ParCSRMatrix* A = (ParCSRMatrix*)p;
    ParVector vx(A->global_num_cols, A->on_proc_num_cols), vb(A->global_num_rows, A->local_num_rows),
        vr(A->global_num_rows, A->local_num_rows);
    set_vec(vx, x);
    set_vec(vb, b);
    A->residual(vx, vb, vr);
    get_vec(vr, r);
}

void rp_spmv_T(void* p, const double* x, double* b) {
    ParCSRMatrix* A = (ParCSRMatrix*)p;
    ParVector vx(A->global_num_rows, A->local_num_rows), vb(A->global_num_cols, A->on_proc_num_cols);
    set_vec(vx, x);
    A->mult_T(vx, vb);
    get_vec(vb, b);
}

void rp_default_opts(rp_opts* o) {
    o->solver = 0;
    o->theta = 0.25;
    o->coarsen = PMIS;
    o->interp = Extended;
    o->strength = Classical;
    o->relax = SOR;
    o->relax_weight = 1.0;
    o->num_smooth_sweeps = 1;
    o->interp_filter = 0.3;
    o->max_coarse = 50;
    o->max_levels = 25;
    o->num_variables = 1;
}

const char* rp_last_error(void) { return g_error.c_str(); }

// new ParRugeStubenSolver(...) or ParSmoothedAggregationSolver(...), the
// caller's field settings, then ml->setup(A) (which copies A).  NULL, with
// the exception's text in rp_last_error(), if the setup throws.
void* rp_setup(void* pA, const rp_opts* o) {
    ParCSRMatrix* A = (ParCSRMatrix*)pA;
    Solver* s = new Solver;
    s->ml = NULL;
    s->o = *o;
    s->n0 = A->local_num_rows;
    if (o->solver == 0) {
        ParRugeStubenSolver* rs = new ParRugeStubenSolver(
            o->theta, (coarsen_t)o->coarsen, (interp_t)o->interp, (strength_t)o->strength,
            (relax_t)o->relax);
        rs->interp_filter = o->interp_filter;
        s->ml = rs;
    } else {
        s->ml = new ParSmoothedAggregationSolver(o->theta, MIS, JacobiProlongation,
                                                 (strength_t)o->strength, (relax_t)o->relax);
    }
    s->ml->relax_weight = o->relax_weight;
    s->ml->num_smooth_sweeps = o->num_smooth_sweeps;
    s->ml->max_coarse = o->max_coarse;
    s->ml->max_levels = o->max_levels;
    if (o->solver == 0) s->ml->num_variables = o->num_variables;
    try {
        s->ml->setup(A);
    } catch (const std::exception& e) {
        g_error = std::string("setup threw ") + e.what();
        // the partly built hierarchy is left as it is (its state is unknown)
        delete s;
        return NULL;
    }
    g_error.clear();
    return s;
}

// A ParRugeStubenSolver whose levels are given (A_l with the diagonal first,
// P_l), finished the way ParMultilevel::setup_helper finishes its own
// (level vectors sized, duplicate_coarse gathering A_c and factoring it with
// dgetrf_), without running the setup: the reference's solve phase on a
// hierarchy built elsewhere.  The hierarchy owns the matrices afterwards.
void* rp_hierarchy_from_levels(int L, void** As, void** Ps, const rp_opts* o) {
    Solver* s = new Solver;
    s->o = *o;
    s->n0 = ((ParCSRMatrix*)As[0])->local_num_rows;
    ParRugeStubenSolver* rs = new ParRugeStubenSolver(
        o->theta, (coarsen_t)o->coarsen, (interp_t)o->interp, (strength_t)o->strength,
        (relax_t)o->relax);
    rs->interp_filter = o->interp_filter;
    rs->relax_weight = o->relax_weight;
    rs->num_smooth_sweeps = o->num_smooth_sweeps;
    rs->max_coarse = o->max_coarse;
    rs->max_levels = o->max_levels;
    for (int l = 0; l < L; l++) {
        ParLevel* lv = new ParLevel();
        lv->A = (ParCSRMatrix*)As[l];
        lv->P = (l + 1 < L) ? (ParCSRMatrix*)Ps[l] : NULL;
        lv->x.resize(lv->A->global_num_rows, lv->A->local_num_rows);
        lv->b.resize(lv->A->global_num_rows, lv->A->local_num_rows);
        lv->tmp.resize(lv->A->global_num_rows, lv->A->local_num_rows);
        rs->levels.push_back(lv);
    }
    rs->num_levels = L;
    rs->duplicate_coarse();
    s->ml = rs;
    return s;
}

void rp_free(void* p) {
    Solver* s = (Solver*)p;
    delete s->ml;
    delete s;
}

int rp_num_levels(void* p) { return ((Solver*)p)->ml->num_levels; }

// Level l's A (which = 0) or P (which = 1), owned by the hierarchy.
void* rp_level(void* p, int l, int which) {
    Solver* s = (Solver*)p;
    if (l < 0 || l >= s->ml->num_levels) return NULL;
    return which == 0 ? (void*)s->ml->levels[l]->A : (void*)s->ml->levels[l]->P;
}

// The C/F states of level l of a Ruge-Stuben hierarchy: the reference's
// strength and splitting routines applied to its stored A_l with the
// weights its setup drew (srand(2448422 + first row), one array for level 0
// whose prefix every coarser level reads), exactly as
// ParRugeStubenSolver::extend_hierarchy calls them.
int rp_level_states(void* p, int l, int* states_out) {
    Solver* s = (Solver*)p;
    if (s->o.solver != 0 || l < 0 || l >= s->ml->num_levels - 1) return -1;
    double* w = new double[s->n0 > 0 ? s->n0 : 1];
    srand(2448422 + 0);
    for (int i = 0; i < s->n0; i++) w[i] = double(rand()) / RAND_MAX;
    // the solver's variable list (form_variable_list: row i of level 0 is
    // variable i % num_variables), compacted to the C points after every
    // level as extend_hierarchy does (par_ruge_stuben_solver.hpp:124-133):
    // the levels below l are split again to follow it
    const int nv = s->o.num_variables > 1 ? s->o.num_variables : 1;
    std::vector<int> vars;
    if (nv > 1) {
        vars.resize(s->n0 > 0 ? s->n0 : 1);
        for (int i = 0; i < s->n0; i++) vars[i] = i % nv;
    }
    aligned_vector<int> states;
    for (int lv = (nv > 1 ? 0 : l); lv <= l; lv++) {
        ParCSRMatrix* A = s->ml->levels[lv]->A;
        ParCSRMatrix* S = A->strength((strength_t)s->o.strength, s->o.theta, false, nv,
                                      nv > 1 ? vars.data() : NULL);
        aligned_vector<int> off_proc_states;
        states.clear();
        switch (s->o.coarsen) {
        case RS:
            if (lv < 3) split_rs(S, states, off_proc_states, false);
            else split_falgout(S, states, off_proc_states, false, w);
            break;
        case CLJP: split_cljp(S, states, off_proc_states, false, w); break;
        case Falgout: split_falgout(S, states, off_proc_states, false, w); break;
        case PMIS: split_pmis(S, states, off_proc_states, false, w); break;
        case HMIS: split_hmis(S, states, off_proc_states, false, w); break;
        }
        delete S;
        if (nv > 1 && lv < l) {
            int ctr = 0;
            for (int i = 0; i < A->local_num_rows; i++)
                if (states[i] == 1) vars[ctr++] = vars[i];
        }
    }
    ParCSRMatrix* A = s->ml->levels[l]->A;
    for (int i = 0; i < A->local_num_rows; i++) states_out[i] = states[i];
    delete[] w;
    return A->local_num_rows;
}

// ml->solve(x, b) with solve_tol and max_iterations set; the history is
// ml->get_residuals()[0..iterations].
int rp_solve(void* p, double* x, const double* b, double tol, int max_iter, double* hist,
             int cap) {
    Solver* s = (Solver*)p;
    ParCSRMatrix* A = s->ml->levels[0]->A;
    ParVector vx(A->global_num_rows, A->local_num_rows), vb(A->global_num_rows, A->local_num_rows);
    set_vec(vx, x);
    set_vec(vb, b);
    s->ml->solve_tol = tol;
    s->ml->max_iterations = max_iter;
    int it = s->ml->solve(vx, vb);
    get_vec(vx, x);
    copy_hist(s->ml->get_residuals(), it + 1, hist, cap);
    return it;
}

// One V-cycle from level `level` (ml->cycle(x, b, level)); at the coarsest
// level this is the LU solve with A_c that setup factored (dgetrs_).
void rp_cycle(void* p, double* x, const double* b, int level) {
    Solver* s = (Solver*)p;
    ParCSRMatrix* A = s->ml->levels[level]->A;
    ParVector vx(A->global_num_rows, A->local_num_rows), vb(A->global_num_rows, A->local_num_rows);
    set_vec(vx, x);
    set_vec(vb, b);
    s->ml->cycle(vx, vb, level);
    get_vec(vx, x);
}

// PCG(A, ml, x, b, res, tol, max_iter); returns the number of history entries.
int rp_pcg(void* pA, void* p, double* x, const double* b, double tol, int max_iter,
           double* hist, int cap) {
    ParCSRMatrix* A = (ParCSRMatrix*)pA;
    Solver* s = (Solver*)p;
    ParVector vx(A->global_num_rows, A->local_num_rows), vb(A->global_num_rows, A->local_num_rows);
    set_vec(vx, x);
    set_vec(vb, b);
    aligned_vector<double> res;
    PCG(A, s->ml, vx, vb, res, tol, max_iter);
    get_vec(vx, x);
    return copy_hist(res, (int)res.size(), hist, cap);
}

int rp_cg(void* pA, double* x, const double* b, double tol, int max_iter, double* hist, int cap) {
    ParCSRMatrix* A = (ParCSRMatrix*)pA;
    ParVector vx(A->global_num_rows, A->local_num_rows), vb(A->global_num_rows, A->local_num_rows);
    set_vec(vx, x);
    set_vec(vb, b);
    aligned_vector<double> res;
    CG(A, vx, vb, res, tol, max_iter);
    get_vec(vx, x);
    return copy_hist(res, (int)res.size(), hist, cap);
}

int rp_bicgstab(void* pA, double* x, const double* b, double tol, int max_iter, double* hist,
                int cap) {
    ParCSRMatrix* A = (ParCSRMatrix*)pA;
    ParVector vx(A->global_num_rows, A->local_num_rows), vb(A->global_num_rows, A->local_num_rows);
    set_vec(vx, x);
    set_vec(vb, b);
    aligned_vector<double> res;
    BiCGStab(A, vx, vb, res, tol, max_iter);
    get_vec(vx, x);
    return copy_hist(res, (int)res.size(), hist, cap);
}

int rp_pending_messages(void) { return mpi_stub_pending_messages(); }

}  // extern "C"
