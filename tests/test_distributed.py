"""Host logic of the row-partitioned ParCSR (raptor_b200.distributed), on CPU
ranks: the reference's default row partition (core/partition.hpp:52-64), the
split of a rank's rows into on_proc and off_proc blocks with the sorted
off_proc column map (core/par_matrix.cpp:76-157), and the ParComm plan and
halo exchange (core/comm_pkg.hpp:400-466) over torch.distributed with gloo,
world sizes 2 and 3.  On every rank the plan built by exchanging index lists
must equal the plan computed for all ranks in one process, the exchange must
deliver x at the column map, and on_proc x_local + off_proc x_ghost (taken
here with numpy, as a check) must be that rank's rows of A x; the transpose
exchange (off_proc^T x_local sent back to the owners and added into their
rows) must give that rank's rows of A^T x.  The
matrix-row exchange that the distributed Galerkin product needs
(CommPkg::communicate, core/comm_mat.cpp:39-192) must deliver, in column-map
order, the owners' rows with global columns, on_proc entries first.  The
device products are covered by tests/test_gpu_distributed.py.
"""
import os
import socket

import numpy as np
import pytest

from raptor_b200.distributed import ParComm, RowPartition, global_rows, split_rows


def random_csr(n, density, seed):
    rng = np.random.default_rng(seed)
    rp, ci, cv = [0], [], []
    for i in range(n):
        k = rng.binomial(n, density)
        cols = np.unique(np.concatenate([[i], rng.integers(0, n, size=k)]))
        ci.extend(cols.tolist())
        cv.extend(rng.uniform(-1, 1, size=cols.size).tolist())
        rp.append(len(ci))
    return np.array(rp), np.array(ci), np.array(cv)


def stencil_csr(m):
    """5-point Laplacian on an m x m grid (rows couple to rows m apart)."""
    rp, ci, cv = [0], [], []
    for i in range(m * m):
        y, x = divmod(i, m)
        for dy, dx, v in ((-1, 0, -1.0), (0, -1, -1.0), (0, 0, 4.0), (0, 1, -1.0), (1, 0, -1.0)):
            if 0 <= y + dy < m and 0 <= x + dx < m:
                ci.append((y + dy) * m + x + dx)
                cv.append(v)
        rp.append(len(ci))
    return np.array(rp), np.array(ci), np.array(cv)


def dense(rp, ci, cv, n_cols):
    A = np.zeros((len(rp) - 1, n_cols))
    for i in range(len(rp) - 1):
        for j in range(rp[i], rp[i + 1]):
            A[i, ci[j]] += cv[j]
    return A


def test_even_partition_is_the_references():
    assert RowPartition.even(10, 3).first.tolist() == [0, 4, 7, 10]
    assert RowPartition.even(9, 3).first.tolist() == [0, 3, 6, 9]
    assert RowPartition.even(2, 3).first.tolist() == [0, 1, 2, 2]
    p = RowPartition([0, 5, 5, 12])
    assert p.owner([0, 4, 5, 11]).tolist() == [0, 0, 2, 2]


@pytest.mark.parametrize("first,last", [(0, 40), (40, 77), (77, 120), (30, 31)])
def test_split_rows_rebuilds_the_rows(first, last):
    rp, ci, cv = random_csr(120, 0.05, 3)
    a, b = rp[first], rp[last]
    (orp, oci, ocv), (frp, fci, fcv), colmap = split_rows(rp[first:last + 1] - a, ci[a:b], cv[a:b],
                                                          first, last)
    assert np.all(np.diff(colmap) > 0)
    assert not np.any((colmap >= first) & (colmap < last))
    want = dense(rp, ci, cv, 120)[first:last]
    got = np.zeros_like(want)
    got[:, first:last] = dense(orp, oci, ocv, last - first)
    got[:, colmap] += dense(frp, fci, fcv, len(colmap))
    np.testing.assert_array_equal(got, want)
    for rpb, cib in ((orp, oci), (frp, fci)):   # rows sorted by column
        for i in range(len(rpb) - 1):
            assert np.all(np.diff(cib[rpb[i]:rpb[i + 1]]) > 0)


def test_rank_without_rows_is_refused():
    from raptor_b200 import RaptorError
    from raptor_b200.distributed import DistParCSRMatrix

    part = RowPartition.even(2, 3)   # the last rank owns no rows
    with pytest.raises(RaptorError):
        DistParCSRMatrix(part, 2, np.zeros(1, np.int32), [], [])
    with pytest.raises(RaptorError):   # rows of another size than the partition's
        DistParCSRMatrix(RowPartition([0, 3]), 0, np.zeros(3, np.int32), [], [])


def test_plan_all_sends_what_each_rank_needs():
    rp, ci, cv = stencil_csr(12)
    part = RowPartition.even(144, 3)
    maps = []
    for r in range(3):
        f, l = part.local_range(r)
        maps.append(split_rows(rp[f:l + 1] - rp[f], ci[rp[f]:rp[l]], cv[rp[f]:rp[l]], f, l)[2])
    plans = ParComm.plan_all(part, maps)
    x = np.arange(144, dtype=float) * 1.5
    for q in range(3):
        ghost = np.empty(len(maps[q]))
        for k, r in enumerate(plans[q].recv_procs):
            j = plans[r].send_procs.index(q)
            sl = plans[r].send_idx[plans[r].send_ptr[j]:plans[r].send_ptr[j + 1]]
            ghost[plans[q].recv_ptr[k]:plans[q].recv_ptr[k + 1]] = x[part.local_range(r)[0] + sl]
        np.testing.assert_array_equal(ghost, x[maps[q]])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, kind, out):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        n = 144 if kind == "stencil" else 90
        rp, ci, cv = stencil_csr(12) if kind == "stencil" else random_csr(n, 0.06, 7)
        part = RowPartition.even(n, world) if kind == "stencil" else RowPartition([0, 50, 51, 90][:world] + [n])
        maps, blocks = [], []
        for r in range(world):
            f, l = part.local_range(r)
            blk = split_rows(rp[f:l + 1] - rp[f], ci[rp[f]:rp[l]], cv[rp[f]:rp[l]], f, l)
            blocks.append(blk)
            maps.append(blk[2])
        plan = ParComm.build(part, maps[rank], rank)
        ref = ParComm.plan_all(part, maps)[rank]
        same = (plan.recv_procs == ref.recv_procs and plan.send_procs == ref.send_procs
                and np.array_equal(plan.recv_ptr, ref.recv_ptr)
                and np.array_equal(plan.send_ptr, ref.send_ptr)
                and np.array_equal(plan.send_idx, ref.send_idx))
        x = np.random.default_rng(11).uniform(-1, 1, n)
        f, l = part.local_range(rank)
        send = torch.as_tensor(x[f:l][plan.send_idx] if plan.num_send else np.zeros(1))
        recv = torch.zeros(max(plan.num_recv, 1), dtype=torch.float64)
        for w in plan.exchange_packed(send, recv):
            w.wait()
        ghost = recv.numpy()[:plan.num_recv]
        (orp, oci, ocv), (frp, fci, fcv), colmap = blocks[rank]
        y = dense(orp, oci, ocv, l - f) @ x[f:l]
        if len(colmap):
            y = y + dense(frp, fci, fcv, len(colmap)) @ ghost
        want = dense(rp, ci, cv, n)[f:l] @ x
        # transpose: off_proc^T x_local back to the owners, added into their rows
        t = (dense(frp, fci, fcv, len(colmap)).T @ x[f:l]) if len(colmap) else np.zeros(1)
        recv_t = torch.zeros(max(plan.num_send, 1), dtype=torch.float64)
        for w in plan.exchange_packed_T(torch.as_tensor(t), recv_t):
            w.wait()
        yt = dense(orp, oci, ocv, l - f).T @ x[f:l]
        rt = recv_t.numpy()
        for k in range(len(plan.send_procs)):
            a, e = plan.send_ptr[k], plan.send_ptr[k + 1]
            yt[plan.send_idx[a:e]] += rt[a:e]
        want_t = dense(rp, ci, cv, n).T[f:l] @ x
        np.save(out % rank, np.array([float(same), float(np.array_equal(ghost, x[colmap])),
                                      float(np.max(np.abs(y - want), initial=0.0)),
                                      float(np.max(np.abs(yt - want_t), initial=0.0))]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,kind", [(2, "stencil"), (3, "stencil"), (3, "random")])
def test_gloo_plan_and_exchange(tmp_path, world, kind):
    import torch.multiprocessing as mp

    out = str(tmp_path / "r%d.npy")
    mp.start_processes(_rank_main, args=(world, _free_port(), kind, out), nprocs=world,
                       start_method="spawn", join=True)
    for r in range(world):
        same, ghost_ok, err, err_t = np.load(out % r)
        assert same == 1.0, "plan differs on rank %d" % r
        assert ghost_ok == 1.0, "halo values wrong on rank %d" % r
        assert err < 1e-13 and err_t < 1e-13


def owner_rows(rp, ci, cv, part, r):
    f, l = part.local_range(r)
    on, off, colmap = split_rows(rp[f:l + 1] - rp[f], ci[rp[f]:rp[l]], cv[rp[f]:rp[l]], f, l)
    return global_rows(on, off, f, colmap), colmap


def test_global_rows_keep_each_row():
    """On_proc entries (global columns) then off_proc entries, per row; the
    row's entries are the matrix row's."""
    rp, ci, cv = random_csr(60, 0.08, 4)
    part = RowPartition([0, 17, 41, 60])
    for r in range(3):
        f, l = part.local_range(r)
        (grp, gci, gcv), _ = owner_rows(rp, ci, cv, part, r)
        for i in range(l - f):
            row_c, row_v = gci[grp[i]:grp[i + 1]], gcv[grp[i]:grp[i + 1]]
            inside = (row_c >= f) & (row_c < l)
            k = int(inside.sum())
            assert inside[:k].all() and not inside[k:].any()
            assert sorted(zip(row_c, row_v)) == sorted(zip(ci[rp[f + i]:rp[f + i + 1]],
                                                            cv[rp[f + i]:rp[f + i + 1]]))


def _rows_rank_main(rank, world, port, kind, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        n = 144 if kind == "stencil" else 90
        rp, ci, cv = stencil_csr(12) if kind == "stencil" else random_csr(n, 0.06, 9)
        part = (RowPartition.even(n, world) if kind == "stencil"
                else RowPartition([0, 50, 51, 90][:world] + [n]))
        (grp, gci, gcv), colmap = owner_rows(rp, ci, cv, part, rank)
        plan = ParComm.build(part, colmap, rank)
        rrp, rci, rcv = plan.communicate_rows(grp, gci, gcv)
        ok = len(rrp) == len(colmap) + 1
        for k, g in enumerate(colmap):
            q = int(part.owner(np.array([g]))[0])
            (orp, oci, ocv), _ = owner_rows(rp, ci, cv, part, q)
            i = g - part.local_range(q)[0]
            ok = ok and np.array_equal(rci[rrp[k]:rrp[k + 1]], oci[orp[i]:orp[i + 1]])
            ok = ok and np.array_equal(rcv[rrp[k]:rrp[k + 1]], ocv[orp[i]:orp[i + 1]])
        np.save(out % rank, np.array([float(ok), float(len(colmap)), float(rrp[-1])]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,kind", [(2, "stencil"), (3, "stencil"), (3, "random")])
def test_gloo_matrix_rows_exchange(tmp_path, world, kind):
    import torch.multiprocessing as mp

    out = str(tmp_path / "r%d.npy")
    mp.start_processes(_rows_rank_main, args=(world, _free_port(), kind, out), nprocs=world,
                       start_method="spawn", join=True)
    for r in range(world):
        ok, n_ghost, n_entries = np.load(out % r)
        assert ok == 1.0, "received rows differ on rank %d" % r
        assert n_ghost == 0 or n_entries > 0
