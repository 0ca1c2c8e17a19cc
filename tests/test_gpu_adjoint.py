"""GPU tests of the differentiation form: finite-volume assembly, SDDMM,
assembly backward, adjoint solves, and the torch.autograd harness.

References are written here independently in dense FP64 numpy: the
operator face by face, the adjoint gradient dL/dt_f = -(l_i - l_j)(x_i - x_j)
per interior face (-l_i x_i per wall face) chained through the harmonic
mean, and central finite differences (h = 1e-6) of the dense model's loss.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

rb = pytest.importorskip("raptor_b200")
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _device():
    rb.init(0)


def faces(nx, ny):
    """Interior faces (i, j) and wall faces (i) of the grid, i = y nx + x."""
    idx = np.arange(nx * ny).reshape(ny, nx)
    inner = [np.stack([idx[:, :-1].ravel(), idx[:, 1:].ravel()], 1),
             np.stack([idx[:-1, :].ravel(), idx[1:, :].ravel()], 1)]
    inner = np.concatenate(inner)
    walls = np.concatenate([idx[0, :], idx[-1, :], idx[:, 0], idx[:, -1]])
    return inner, walls


def dense_fv(k, nx, ny):
    inner, walls = faces(nx, ny)
    n = nx * ny
    A = np.zeros((n, n))
    i, j = inner[:, 0], inner[:, 1]
    t = 2.0 * k[i] * k[j] / (k[i] + k[j])
    np.add.at(A, (i, i), t)
    np.add.at(A, (j, j), t)
    np.add.at(A, (i, j), -t)
    np.add.at(A, (j, i), -t)
    np.add.at(A, (walls, walls), 2.0 * k[walls])
    return A


def dense_grad_k(k, x, lam, nx, ny):
    inner, walls = faces(nx, ny)
    g = np.zeros_like(k)
    i, j = inner[:, 0], inner[:, 1]
    dLdt = -(lam[i] - lam[j]) * (x[i] - x[j])
    s = k[i] + k[j]
    np.add.at(g, i, dLdt * 2.0 * k[j] ** 2 / s ** 2)
    np.add.at(g, j, dLdt * 2.0 * k[i] ** 2 / s ** 2)
    np.add.at(g, walls, -lam[walls] * x[walls] * 2.0)
    return g


def csr_to_dense(A):
    n, m, _ = A.info()
    rp, ci, cv = A.arrays()
    D = np.zeros((n, m))
    for r in range(n):
        D[r, ci[rp[r]:rp[r + 1]]] += cv[rp[r]:rp[r + 1]]
    return D


def dev(a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("nx,ny", [(37, 23), (1, 9), (16, 16)])
def test_fv_assembly_matches_dense(nx, ny):
    k = np.exp(np.random.default_rng(nx * ny).standard_normal(nx * ny))
    kt = dev(k)
    h = rb.C.c_void_p()
    rb.check(rb.lib().rb_fv_assemble(nx, ny, rb.C.c_void_p(kt.data_ptr()), rb.C.byref(h)))
    A = rb.ParCSRMatrix(h)
    _, _, nnz = A.info()
    assert nnz == nx * ny + 2 * ((nx - 1) * ny + nx * (ny - 1))
    rp, ci, _ = A.arrays()
    for r in range(nx * ny):   # columns increase along every row
        assert np.all(np.diff(ci[rp[r]:rp[r + 1]]) > 0)
    np.testing.assert_allclose(csr_to_dense(A), dense_fv(k, nx, ny), rtol=1e-14, atol=1e-14)


def test_sddmm_and_backward_match_dense_adjoint_formula():
    nx, ny = 20, 13
    n = nx * ny
    rng = np.random.default_rng(4)
    k = np.exp(rng.standard_normal(n))
    x = rng.standard_normal(n)
    lam = rng.standard_normal(n)
    kt, xt, lt = dev(k), dev(x), dev(lam)
    h = rb.C.c_void_p()
    rb.check(rb.lib().rb_fv_assemble(nx, ny, rb.C.c_void_p(kt.data_ptr()), rb.C.byref(h)))
    A = rb.ParCSRMatrix(h)
    _, _, nnz = A.info()
    gA = torch.empty(nnz, dtype=torch.float64, device="cuda")
    rb.check(rb.lib().rb_sddmm(A.h, rb.C.c_void_p(lt.data_ptr()), rb.C.c_void_p(xt.data_ptr()),
                               -1.0, rb.C.c_void_p(gA.data_ptr())))
    rb.check(rb.lib().rb_synchronize())
    rp, ci, _ = A.arrays()
    rows = np.repeat(np.arange(n), np.diff(rp))
    np.testing.assert_array_equal(gA.cpu().numpy(), -lam[rows] * x[ci])
    gk = torch.empty(n, dtype=torch.float64, device="cuda")
    rb.check(rb.lib().rb_fv_backward(nx, ny, rb.C.c_void_p(kt.data_ptr()), A.h,
                                     rb.C.c_void_p(gA.data_ptr()), rb.C.c_void_p(gk.data_ptr())))
    rb.check(rb.lib().rb_synchronize())
    np.testing.assert_allclose(gk.cpu().numpy(), dense_grad_k(k, x, lam, nx, ny), rtol=1e-12,
                               atol=1e-12)


@pytest.mark.parametrize("prec", [0, 1])
def test_adjoint_solve_symmetric(prec):
    nx = ny = 48
    n = nx * ny
    k = np.exp(rb.autograd.grf(nx, ny, 8.0, seed=3))
    kt = dev(k)
    h = rb.C.c_void_p()
    rb.check(rb.lib().rb_fv_assemble(nx, ny, rb.C.c_void_p(kt.data_ptr()), rb.C.byref(h)))
    A = rb.ParCSRMatrix(h)
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
    ml.precision = prec
    ml.setup(A)
    g = np.random.default_rng(8).uniform(-1, 1, n)
    lv = rb.ParVector(n)
    gv = rb.ParVector(n, values=g)
    it, rr = rb.C.c_int(), rb.C.c_double()
    rc = rb.lib().rb_adjoint_solve(A.h, ml.h, lv.h, gv.h, 1e-10, 300, rb.C.byref(it),
                                   rb.C.byref(rr))
    assert rc == 0 and rr.value <= 1e-10 and it.value > 0
    ref = np.linalg.solve(dense_fv(k, nx, ny).T, g)
    np.testing.assert_allclose(lv.numpy(), ref, rtol=0, atol=1e-7 * np.abs(ref).max())


@pytest.mark.parametrize("prec", [0, 1])
def test_adjoint_solve_nonsymmetric_uses_transposed_cycle(prec):
    # 2D diffusion with upwinded convection: west/east and south/north
    # couplings differ, so A^T != A
    st = np.zeros(9)
    st[4] = 4.6
    st[3], st[5] = -1.5, -0.7
    st[1], st[7] = -1.25, -0.95
    nx = 40
    A = rb.par_stencil_grid(st, [nx, nx])
    n = nx * nx
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.ModClassical, rb.Classical, rb.Jacobi)
    ml.relax_weight = 2.0 / 3.0
    ml.precision = prec
    ml.setup(A)
    g = np.random.default_rng(12).uniform(-1, 1, n)
    lv = rb.ParVector(n)
    gv = rb.ParVector(n, values=g)
    it, rr = rb.C.c_int(), rb.C.c_double()
    rc = rb.lib().rb_adjoint_solve(A.h, ml.h, lv.h, gv.h, 1e-10, 300, rb.C.byref(it),
                                   rb.C.byref(rr))
    assert rc == 0 and rr.value <= 1e-9
    D = csr_to_dense(A)
    assert np.abs(D - D.T).max() > 0.1
    ref = np.linalg.solve(D.T, g)
    np.testing.assert_allclose(lv.numpy(), ref, rtol=0, atol=1e-7 * np.abs(ref).max())


def loss_and_grad(nx, ny, g, bh, xt, tol, prec):
    gt = dev(g).requires_grad_(True)
    bt = dev(bh).requires_grad_(True)
    x = rb.autograd.DiffusionSolve.apply(torch.exp(gt), bt, nx, ny, tol, 500, prec)
    loss = 0.5 * ((x - dev(xt)) ** 2).sum()
    loss.backward()
    return float(loss.detach()), gt.grad.cpu().numpy(), bt.grad.cpu().numpy(), x.detach().cpu().numpy()


@pytest.mark.parametrize("prec", [0, 1])
def test_gradients_match_dense_reference_and_finite_differences(prec):
    from scipy.linalg import lu_factor, lu_solve

    nx = ny = 64
    n = nx * ny
    g = rb.autograd.grf(nx, ny, 32.0, seed=20261203)
    rng = np.random.default_rng(20261204)
    bh = rng.uniform(-1, 1, n)
    xt = rng.uniform(0, 1, n)
    L, dg, db, x = loss_and_grad(nx, ny, g, bh, xt, 1e-11, prec)
    # dense FP64 reference: forward, adjoint, per-face gradient
    k = np.exp(g)
    A = dense_fv(k, nx, ny)
    xr = np.linalg.solve(A, bh)
    assert np.linalg.norm(x - xr) <= 1e-8 * np.linalg.norm(xr)
    lam = np.linalg.solve(A.T, xr - xt)
    dg_ref = dense_grad_k(k, xr, lam, nx, ny) * k
    np.testing.assert_allclose(db, lam, rtol=0, atol=1e-7 * np.abs(lam).max())
    np.testing.assert_allclose(dg, dg_ref, rtol=0, atol=1e-7 * np.abs(dg_ref).max())

    if prec != rb.FP32:
        return
    # central differences (h = 1e-6) of the dense model's loss
    lu0 = lu_factor(A)

    def dense_loss(gg, bb, lu=None):
        xx = lu_solve(lu, bb) if lu is not None else np.linalg.solve(dense_fv(np.exp(gg), nx, ny), bb)
        return 0.5 * np.sum((xx - xt) ** 2)

    h = 1e-6
    pick = np.random.default_rng(5).choice(n, 5, replace=False)
    scale_g, scale_b = np.abs(dg_ref).max(), np.abs(lam).max()
    for c in pick:
        e = np.zeros(n)
        e[c] = h
        fd_g = (dense_loss(g + e, bh) - dense_loss(g - e, bh)) / (2 * h)
        fd_b = (dense_loss(g, bh + e, lu0) - dense_loss(g, bh - e, lu0)) / (2 * h)
        assert abs(fd_g - dg[c]) <= 1e-5 * scale_g, (c, fd_g, dg[c])
        assert abs(fd_b - db[c]) <= 1e-5 * scale_b, (c, fd_b, db[c])


def test_grf_statistics():
    g = rb.autograd.grf(512, 512, 32.0, seed=1)
    assert abs(g.mean()) < 0.5 and 0.6 < g.var() < 1.4
    f = g.reshape(512, 512)
    # neighbouring cells are strongly correlated, cells 4 correlation lengths apart are not
    c1 = np.corrcoef(f[:, :-1].ravel(), f[:, 1:].ravel())[0, 1]
    c128 = np.corrcoef(f[:, :-128].ravel(), f[:, 128:].ravel())[0, 1]
    assert c1 > 0.99 and abs(c128) < 0.2
