// A reference-style caller compiled against include/raptor_b200.hpp: the
// body is written as a user of the reference writes it (gallery matrix,
// ParVector, ParRugeStubenSolver with field tweaks, setup, PCG and a
// stationary solve), with only the namespace changed.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "raptor_b200.hpp"

using namespace raptor_b200;

int main(int argc, char** argv) {
    const int m = argc > 1 ? std::atoi(argv[1]) : 20;
    try {
        double* stencil = laplace_stencil_27pt();
        int grid[3] = {m, m, m};
        ParCSRMatrix* A = par_stencil_grid(stencil, grid, 3);
        delete[] stencil;
        const int n = A->global_num_rows;
        ParVector x(n, n), b(n, n), ones(n, n);
        ones.set_const_value(1.0);
        A->mult(ones, b);   // b = A * ones
        x.set_const_value(0.0);

        ParMultilevel* ml = new ParRugeStubenSolver(0.25, PMIS, Extended, Classical, L1Jacobi);
        ml->max_iterations = 200;
        ml->solve_tol = 1e-8;
        ml->setup(A);
        aligned_vector<double> res;
        PCG(A, ml, x, b, res, 1e-8);
        ParVector r(n, n);
        A->residual(x, b, r);
        std::printf("levels %d pcg_hist %zu relres %.17e\n", ml->num_levels, res.size(),
                    r.norm(2) / b.norm(2));
        std::printf("pcg");
        for (double v : res) std::printf(" %.17e", v);
        std::printf("\n");
        x.set_const_value(0.0);
        const int it = ml->solve(x, b);
        std::printf("solve_iters %d last %.17e\n", it, ml->get_residuals().back());
        std::printf("solve");
        for (double v : ml->get_residuals()) std::printf(" %.17e", v);
        std::printf("\n");
        delete ml;
        delete A;
    } catch (const error& e) {
        std::printf("error %d %s\n", e.code, e.what());
        return e.code == RB_ERR_NO_DEVICE ? 3 : 1;
    }
    return 0;
}
