"""GPU tests of the row-partitioned ParCSR products (raptor_b200.distributed).

The send-buffer packing kernel (rb_vec_gather) must gather exactly and turn
an index outside the vector into NaN.  Partitions held by one process (here
three partitions of one matrix on one GPU, exchanging their halos through
device copies with the plan every rank would build) must give the rows of
A x and b - A x of the whole matrix: on_proc x_local + off_proc x_ghost sums
a row in another grouping than the single product, so the check is to
1e-14 of sum_j |a_ij x_j| against an FP64 numpy product and the library's
own product of the whole matrix (and likewise A^T x, whose off_proc part
goes back to the owners of the columns).  CG over three partitions must follow the
library's CG on the whole matrix (histories to 1e-8); PCG over one partition
with its block-Jacobi AMG (then the whole matrix's AMG) must give the
library's reference-mode PCG history to 1e-10 (to within one iteration),
and over four uneven
partitions must converge.  A one-rank NCCL group runs the communicating path
itself (plan built by all_gather, dots by all_reduce, CG through it equal to
CG in process).
The NCCL point-to-point halo between several GPUs is not run here (one GPU
per run); its plan and exchange are checked on gloo CPU ranks in
tests/test_distributed.py.
"""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

rb = pytest.importorskip("raptor_b200")
torch = pytest.importorskip("torch")
from raptor_b200 import distributed as D  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _device():
    rb.init(0)
    yield
    # later tests run on the library's own stream again
    rb.synchronize()
    rb.set_stream(0)
    D._STREAM = None


def csr_of(A):
    rp, ci, cv = A.arrays()
    return np.asarray(rp), np.asarray(ci), np.asarray(cv)


def scale_of(rp, ci, cv, x):
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    s = np.zeros(len(rp) - 1)
    np.add.at(s, rows, np.abs(cv * x[ci]))
    return s


def product(rp, ci, cv, x):
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    y = np.zeros(len(rp) - 1)
    np.add.at(y, rows, cv * x[ci])
    return y


def random_csr(n, per_row, seed):
    rng = np.random.default_rng(seed)
    rp, ci, cv = [0], [], []
    for i in range(n):
        cols = np.unique(np.concatenate([[i], rng.integers(0, n, size=per_row)]))
        ci.extend(cols.tolist())
        cv.extend(rng.uniform(-1, 1, size=cols.size).tolist())
        rp.append(len(ci))
    return np.array(rp), np.array(ci), np.array(cv)


def test_vec_gather():
    x = rb.ParVector(10, values=np.arange(10, dtype=float) + 0.5)
    idx = torch.tensor([3, 0, 9, 12, -1], dtype=torch.int32, device="cuda")
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    x.gather(idx.data_ptr(), 5, out.data_ptr())
    rb.synchronize()
    got = out.cpu().numpy()
    np.testing.assert_array_equal(got[:3], [3.5, 0.5, 9.5])
    assert np.isnan(got[3]) and np.isnan(got[4])


MATRICES = {
    "lap27_14": lambda: csr_of(rb.par_stencil_grid(rb.laplace_stencil_27pt(), [14, 14, 14])),
    "aniso2d_60": lambda: csr_of(rb.par_stencil_grid(rb.diffusion_stencil_2d(0.001, np.pi / 8), [60, 60])),
    "random_3000": lambda: random_csr(3000, 12, 5),
}


@pytest.mark.parametrize("name", sorted(MATRICES))
@pytest.mark.parametrize("parts", ["even3", "uneven4"])
def test_partitions_in_one_process_match_whole_matrix(name, parts):
    rp, ci, cv = MATRICES[name]()
    n = len(rp) - 1
    part = (D.RowPartition.even(n, 3) if parts == "even3"
            else D.RowPartition([0, n // 7, n // 7 + 1, (2 * n) // 3, n]))
    maps = []
    for r in range(part.world):
        f, l = part.local_range(r)
        maps.append(D.split_rows(rp[f:l + 1] - rp[f], ci[rp[f]:rp[l]], cv[rp[f]:rp[l]], f, l)[2])
    plans = D.ParComm.plan_all(part, maps)
    mats = [D.DistParCSRMatrix.from_global(rp, ci, cv, part, r, comm=plans[r])
            for r in range(part.world)]
    rng = np.random.default_rng(9)
    x = rng.uniform(-1, 1, n)
    bvec = rng.uniform(-1, 1, n)
    xs = [rb.ParVector(n, local_n=m.local_num_rows, values=x[slice(*part.local_range(r))])
          for r, m in enumerate(mats)]
    bs = [rb.ParVector(n, local_n=m.local_num_rows, values=bvec[slice(*part.local_range(r))])
          for r, m in enumerate(mats)]
    ys = [rb.ParVector(n, local_n=m.local_num_rows) for m in mats]
    D.DistParCSRMatrix.mult_in_process(mats, xs, ys)
    y = np.concatenate([v.numpy() for v in ys])
    want = product(rp, ci, cv, x)
    tol = 1e-14 * scale_of(rp, ci, cv, x) + 1e-300
    assert np.all(np.abs(y - want) <= tol)
    A = rb.ParCSRMatrix.from_arrays(n, n, rp, ci, cv)
    yw = rb.ParVector(n)
    A.mult(rb.ParVector(n, values=x), yw)
    assert np.all(np.abs(y - yw.numpy()) <= tol)
    rs = [rb.ParVector(n, local_n=m.local_num_rows) for m in mats]
    D.DistParCSRMatrix.residual_in_process(mats, xs, bs, rs)
    r = np.concatenate([v.numpy() for v in rs])
    assert np.all(np.abs(r - (bvec - want)) <= tol + 1e-15 * np.abs(bvec))
    # transpose product: off_proc^T x back to the column owners
    D.DistParCSRMatrix.mult_T_in_process(mats, xs, ys)
    yt = np.concatenate([v.numpy() for v in ys])
    rows = np.repeat(np.arange(n), np.diff(rp))
    want_t = np.zeros(n)
    np.add.at(want_t, ci, cv * x[rows])
    scale_t = np.zeros(n)
    np.add.at(scale_t, ci, np.abs(cv * x[rows]))
    assert np.all(np.abs(yt - want_t) <= 1e-14 * scale_t + 1e-300)
    A.mult_T(rb.ParVector(n, values=x), yw)
    assert np.all(np.abs(yt - yw.numpy()) <= 1e-14 * scale_t + 1e-300)


def partitions_of(rp, ci, cv, part):
    maps = []
    for r in range(part.world):
        f, l = part.local_range(r)
        maps.append(D.split_rows(rp[f:l + 1] - rp[f], ci[rp[f]:rp[l]], cv[rp[f]:rp[l]], f, l)[2])
    plans = D.ParComm.plan_all(part, maps)
    return D.Partitions([D.DistParCSRMatrix.from_global(rp, ci, cv, part, r, comm=plans[r])
                         for r in range(part.world)])


def test_cg_over_partitions_matches_whole_matrix_cg():
    rp, ci, cv = csr_of(rb.par_stencil_grid(rb.laplace_stencil_27pt(), [12, 12, 12]))
    n = len(rp) - 1
    P = partitions_of(rp, ci, cv, D.RowPartition.even(n, 3))
    b = np.random.default_rng(4).uniform(-1, 1, n)
    xs, bs = P.vectors(), P.vectors(b)
    res = []
    assert D.CG(P, xs, bs, res, tol=1e-8, max_iter=400) == 0
    A = rb.ParCSRMatrix.from_arrays(n, n, rp, ci, cv)
    x2, res2 = rb.ParVector(n), []
    assert rb.CG(A, x2, rb.ParVector(n, values=b), res2, tol=1e-8, max_iter=400) == 0
    assert abs(len(res) - len(res2)) <= 1
    k = min(len(res), len(res2))
    np.testing.assert_allclose(res[:k], res2[:k], rtol=1e-8, atol=1e-15)
    x = np.concatenate([v.numpy() for v in xs])
    assert np.linalg.norm(x - x2.numpy()) <= 1e-7 * np.linalg.norm(x2.numpy())


def make_amg():
    return rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)


def test_pcg_one_partition_is_the_libraries_pcg():
    rp, ci, cv = csr_of(rb.par_stencil_grid(rb.laplace_stencil_27pt(), [20, 20, 20]))
    n = len(rp) - 1
    P = partitions_of(rp, ci, cv, D.RowPartition.even(n, 1))
    M = D.BlockJacobiAMG(P, make_amg)
    b = np.random.default_rng(6).uniform(-1, 1, n)
    xs, bs = P.vectors(), P.vectors(b)
    res = []
    assert D.PCG(P, M, xs, bs, res, tol=1e-8, max_iter=100) == 0
    A = rb.ParCSRMatrix.from_arrays(n, n, rp, ci, cv)
    ml = make_amg()
    ml.setup(A)
    x2, res2 = rb.ParVector(n), []
    assert rb.PCG(A, ml, x2, rb.ParVector(n, values=b), res2, tol=1e-8, max_iter=100,
                  mode=rb.PCG_REFERENCE) == 0
    assert abs(len(res) - len(res2)) <= 1
    k = min(len(res), len(res2))
    np.testing.assert_allclose(res[:k], res2[:k], rtol=1e-10, atol=1e-18)


def test_pcg_block_jacobi_amg_over_partitions_converges():
    rp, ci, cv = csr_of(rb.par_stencil_grid(rb.laplace_stencil_27pt(), [20, 20, 20]))
    n = len(rp) - 1
    P = partitions_of(rp, ci, cv, D.RowPartition([0, 2000, 5000, 6500, n]))
    M = D.BlockJacobiAMG(P, make_amg)
    b = np.random.default_rng(8).uniform(-1, 1, n)
    xs, bs = P.vectors(), P.vectors(b)
    res = []
    assert D.PCG(P, M, xs, bs, res, tol=1e-10, max_iter=300) == 0
    x = np.concatenate([v.numpy() for v in xs])
    r = b - product(rp, ci, cv, x)
    assert np.linalg.norm(r) <= 1e-4 * np.linalg.norm(b)
    assert len(res) < 120


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_one_rank_nccl_group():
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1,
                            timeout=__import__("datetime").timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        rp, ci, cv = MATRICES["lap27_14"]()
        n = len(rp) - 1
        part = D.RowPartition.even(n, 1)
        M = D.DistParCSRMatrix.from_global(rp, ci, cv, part, 0)
        assert M.comm.num_send == 0 and M.comm.num_recv == 0 and M.off_proc is None
        x = np.random.default_rng(2).uniform(-1, 1, n)
        xv, yv = rb.ParVector(n, values=x), rb.ParVector(n)
        M.mult(xv, yv)
        want = product(rp, ci, cv, x)
        assert np.all(np.abs(yv.numpy() - want) <= 1e-14 * scale_of(rp, ci, cv, x))
        assert abs(M.inner_product(xv, xv) - xv.inner_product(xv)) == 0.0
        assert abs(M.norm(xv) - np.linalg.norm(x)) <= 1e-12 * np.linalg.norm(x)
        # CG through the process group (halo and dots over NCCL) against the
        # same CG with the partition in process
        P = D.Partitions([M])
        assert not P.in_process
        bvec = np.random.default_rng(3).uniform(-1, 1, n)
        xs, res = P.vectors(), []
        assert D.CG(P, xs, P.vectors(bvec), res, tol=1e-8, max_iter=400) == 0
        Q = D.Partitions([M], in_process=True)
        xq, resq = Q.vectors(), []
        assert D.CG(Q, xq, Q.vectors(bvec), resq, tol=1e-8, max_iter=400) == 0
        assert res == resq
    finally:
        rb.synchronize()
        dist.destroy_process_group()
