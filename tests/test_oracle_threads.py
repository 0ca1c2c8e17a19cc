"""The oracle's row-parallel loops give the same results for any thread
count (each row is computed alone, in the same order), so the CPU baseline
may time it on every host core without changing what it computes."""
import numpy as np

from oracle import oracle as O


def test_threaded_oracle_pcg_is_identical():
    A = O.stencil_grid(O.laplace_stencil_27pt(), [20, 20, 20])
    n = A.shape[0]
    b = np.random.default_rng(5).uniform(-1.0, 1.0, n)
    ml = O.Hierarchy(A, interp="extended", relax="l1_jacobi")
    old = O.get_threads()
    try:
        out = []
        for t in (1, 4):
            O.set_threads(t)
            assert O.get_threads() == t
            x, hist, _ = O.pcg(A, ml, np.zeros(n), b, tol=1e-8, max_iter=200, mode=1)
            out.append((np.asarray(x), np.asarray(hist)))
            y = O.spmv(A, b)
            out.append((y, O.residual(A, b, y)))
        assert np.array_equal(out[0][0], out[2][0]) and np.array_equal(out[0][1], out[2][1])
        assert np.array_equal(out[1][0], out[3][0]) and np.array_equal(out[1][1], out[3][1])
    finally:
        O.set_threads(old)
