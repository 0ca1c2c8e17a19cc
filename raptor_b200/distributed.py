"""Row-partitioned ParCSR across processes: RAPtor's halo exchange (ParComm)
and its distributed products, one process per GPU.

The reference distributes a matrix by contiguous row blocks
(core/partition.hpp:52-64).  Each rank stores its rows as an ``on_proc``
block (columns it owns, local numbering) and an ``off_proc`` block whose
columns are condensed to the sorted ``off_proc_column_map``
(core/par_matrix.cpp:76-157).  ``ParComm`` (core/comm_pkg.hpp:400-466) turns
that map into receive messages, one per owning rank and contiguous in the map,
and send lists.  Each rank tells the owners which of their rows it needs.
``ParMatrix::mult`` (util/linalg/par_spmv.cpp:25-59) starts the exchange of
x's halo values, multiplies ``on_proc`` meanwhile, waits, then appends
``off_proc`` times the received values; dots add the local dots over all
ranks (core/par_vector.cpp:88-121).

Here the transport is torch.distributed point-to-point (NCCL over NVLink on
GPUs; the same calls run on gloo CPU ranks, which is how the plan and the
exchange are tested without several GPUs).  The local products, the send
buffer packing (``rb_vec_gather``) and the vectors live in the CUDA library.
The library and the module's torch calls share one CUDA stream (``stream()``;
the library is switched to it), so that the pack, the NCCL transfer, the
``on_proc`` product and the ``off_proc`` product follow one another on the
device with no host wait.  The ``on_proc`` product runs while the transfer
is in flight, as in the reference.

Scope: the distributed products (mult, residual, mult_append, mult_T), the distributed
dot and norm, and the reference's CG and PCG over them (krylov/par_cg.cpp),
the PCG preconditioned by one AMG cycle of each partition's own block (block
Jacobi).  The distributed AMG setup of the reference (C/F splitting across
ranks, the P-row exchange of RAP, coarse agglomeration) is not built.
Partitions that share one process, such as several partitions on one GPU,
exchange through device copies (``mult_in_process``, ``Partitions``).
"""
import numpy as np

from . import ParCSRMatrix, ParVector, RaptorError, set_stream

_STREAM = None


def stream():
    """The CUDA stream of the distributed products (created on first use;
    the library's calls are ordered on it from then on)."""
    global _STREAM
    if _STREAM is None:
        import torch

        _STREAM = torch.cuda.Stream()
        set_stream(_STREAM.cuda_stream)
    return _STREAM


def _on_stream():
    import torch

    return torch.cuda.stream(stream())


class RowPartition:
    """Contiguous row blocks: rank q owns global rows [first[q], first[q+1])."""

    def __init__(self, first):
        self.first = np.asarray(first, dtype=np.int64)
        if self.first.ndim != 1 or self.first.size < 2 or np.any(np.diff(self.first) < 0):
            raise RaptorError(-1, "row partition must be nondecreasing with world + 1 entries")
        self.world = self.first.size - 1
        self.global_num_rows = int(self.first[-1])

    @classmethod
    def even(cls, n, world):
        """The reference's default partition (core/partition.hpp:52-64): n //
        world rows a rank, one more on each of the first n % world ranks."""
        avg, extra = divmod(int(n), int(world))
        first = [avg * q + min(q, extra) for q in range(world + 1)]
        return cls(first)

    def local_range(self, rank):
        return int(self.first[rank]), int(self.first[rank + 1])

    def owner(self, cols):
        """Rank owning each global column (row) index."""
        return np.searchsorted(self.first, np.asarray(cols, dtype=np.int64), side="right") - 1


def split_rows(rowptr, cols, vals, first, last):
    """Split rows of a CSR matrix with global column indices into the
    on_proc block (columns in [first, last), numbered from first) and the
    off_proc block (columns condensed to the sorted unique off_proc column
    map), each row sorted by column (par_matrix.cpp:76-157).  Returns
    ((rowptr, cols, vals) on_proc, (rowptr, cols, vals) off_proc, colmap)."""
    rowptr = np.asarray(rowptr, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.float64)
    n = rowptr.size - 1
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    on = (cols >= first) & (cols < last)
    colmap = np.unique(cols[~on])

    def block(mask, newcols):
        r, c, v = rows[mask], newcols, vals[mask]
        o = np.lexsort((c, r))
        rp = np.zeros(n + 1, dtype=np.int64)
        np.add.at(rp, r + 1, 1)
        return (np.cumsum(rp).astype(np.int32), c[o].astype(np.int32), v[o])

    on_blk = block(on, cols[on] - first)
    off_blk = block(~on, np.searchsorted(colmap, cols[~on]))
    return on_blk, off_blk, colmap.astype(np.int64)


def global_rows(on, off, first, colmap):
    """A rank's rows with global column indices, each row's on_proc entries
    then its off_proc entries: the rows CommPkg::init_par_mat_comm packs
    (core/comm_mat.cpp:53-96).  on and off are host (rowptr, cols, vals);
    on_proc columns are local (global - first), off_proc columns index
    colmap.  Returns (rowptr int64, cols int64, vals float64)."""
    orp, oci, ocv = (np.asarray(a) for a in on)
    frp, fci, fcv = (np.asarray(a) for a in off)
    n = len(orp) - 1
    on_len, off_len = np.diff(orp), np.diff(frp)
    rowptr = np.zeros(n + 1, np.int64)
    rowptr[1:] = np.cumsum(on_len + off_len)
    cols = np.empty(int(rowptr[-1]), np.int64)
    vals = np.empty(int(rowptr[-1]), np.float64)
    r_on = np.repeat(np.arange(n), on_len)
    dest = rowptr[r_on] + (np.arange(len(oci)) - orp[r_on])
    cols[dest] = np.asarray(oci, np.int64) + first
    vals[dest] = ocv
    r_off = np.repeat(np.arange(n), off_len)
    dest = rowptr[r_off] + on_len[r_off] + (np.arange(len(fci)) - frp[r_off])
    cols[dest] = np.asarray(colmap, np.int64)[np.asarray(fci, np.int64)]
    vals[dest] = fcv
    return rowptr, cols, vals


class ParComm:
    """Halo-exchange plan of one rank (core/comm_pkg.hpp:400-466).

    recv_procs[k] sends this rank ghost values recv_ptr[k]:recv_ptr[k+1] of
    the off_proc column map (the map is sorted and owners hold contiguous
    rows, so each owner's columns are one run); send_procs[k] receives this
    rank's local rows send_idx[send_ptr[k]:send_ptr[k+1]], in the order the
    receiver's map lists them."""

    def __init__(self, recv_procs, recv_ptr, send_procs, send_ptr, send_idx):
        self.recv_procs = [int(q) for q in recv_procs]
        self.recv_ptr = np.asarray(recv_ptr, dtype=np.int64)
        self.send_procs = [int(q) for q in send_procs]
        self.send_ptr = np.asarray(send_ptr, dtype=np.int64)
        self.send_idx = np.asarray(send_idx, dtype=np.int32)

    @property
    def num_recv(self):
        return int(self.recv_ptr[-1])

    @property
    def num_send(self):
        return int(self.send_ptr[-1])

    @staticmethod
    def _recv_runs(partition, colmap):
        owners = partition.owner(colmap)
        procs, ptr = [], [0]
        for k in range(len(colmap)):
            if not procs or owners[k] != procs[-1]:
                if procs:
                    ptr.append(k)
                procs.append(int(owners[k]))
        if procs:
            ptr.append(len(colmap))
        return procs, ptr

    @classmethod
    def plan_all(cls, partition, colmaps):
        """Every rank's plan from every rank's column map, in one process (no
        communication): what build() computes on each rank."""
        runs = [cls._recv_runs(partition, np.asarray(m, dtype=np.int64)) for m in colmaps]
        plans = []
        for r in range(partition.world):
            send_procs, send_ptr, send_idx = [], [0], []
            first = partition.local_range(r)[0]
            for q in range(partition.world):
                procs, ptr = runs[q]
                if r in procs:
                    k = procs.index(r)
                    seg = np.asarray(colmaps[q], dtype=np.int64)[ptr[k]:ptr[k + 1]]
                    send_procs.append(q)
                    send_idx.extend((seg - first).tolist())
                    send_ptr.append(len(send_idx))
            procs, ptr = runs[r]
            plans.append(cls(procs, ptr, send_procs, send_ptr, send_idx))
        return plans

    @classmethod
    def build(cls, partition, colmap, rank, group=None, device="cpu"):
        """This rank's plan, exchanging index lists with the other ranks over
        torch.distributed (``device``: where the messages live; CUDA for
        NCCL).  Every rank of the group must call it."""
        import torch
        import torch.distributed as dist

        colmap = np.asarray(colmap, dtype=np.int64)
        world = partition.world
        procs, ptr = cls._recv_runs(partition, colmap)
        need = torch.zeros(world, dtype=torch.int64, device=device)
        for k, q in enumerate(procs):
            need[q] = ptr[k + 1] - ptr[k]
        # recv sizes of every rank (the reference all-reduces them; gathering
        # the whole table also tells each rank whom it sends to)
        table = [torch.zeros(world, dtype=torch.int64, device=device) for _ in range(world)]
        dist.all_gather(table, need, group=group)
        counts = [int(table[q][rank]) for q in range(world)]
        send_procs = [q for q in range(world) if counts[q] > 0 and q != rank]
        ops, bufs = [], []
        cm = torch.as_tensor(colmap, device=device)
        for k, q in enumerate(procs):
            ops.append(dist.P2POp(dist.isend, cm[ptr[k]:ptr[k + 1]].contiguous(), q, group=group))
        for q in send_procs:
            b = torch.empty(counts[q], dtype=torch.int64, device=device)
            bufs.append(b)
            ops.append(dist.P2POp(dist.irecv, b, q, group=group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        first = partition.local_range(rank)[0]
        send_ptr = [0]
        send_idx = []
        for b in bufs:
            send_idx.extend((b.cpu().numpy() - first).tolist())
            send_ptr.append(len(send_idx))
        return cls(procs, ptr, send_procs, send_ptr, send_idx)

    def exchange_packed(self, send_buf, recv_buf, group=None):
        """Start the exchange: send_buf holds this rank's send_idx values
        (packed), recv_buf receives the ghost values in column-map order.
        Returns the requests to wait on (empty when nothing moves)."""
        import torch.distributed as dist

        ops = []
        for k, q in enumerate(self.recv_procs):
            a, b = int(self.recv_ptr[k]), int(self.recv_ptr[k + 1])
            ops.append(dist.P2POp(dist.irecv, recv_buf[a:b], q, group=group))
        for k, q in enumerate(self.send_procs):
            a, b = int(self.send_ptr[k]), int(self.send_ptr[k + 1])
            ops.append(dist.P2POp(dist.isend, send_buf[a:b], q, group=group))
        return dist.batch_isend_irecv(ops) if ops else []

    def communicate_rows(self, rowptr, cols, vals, group=None, device="cpu"):
        """Matrix rows along the halo plan (CommPkg::communicate(ParCSRMatrix*),
        core/comm_mat.cpp:39-96, 145-192): each receiver gets the rows of this
        rank that its column map names, whole, in the order it lists them; this
        rank gets, in its column-map order, the rows the other ranks own.
        rowptr / cols / vals are this rank's rows on the host (global column
        indices, global_rows); ``device`` is where the messages live (CUDA for
        NCCL).  Row lengths go first, then the column indices, then the values;
        a message without entries is not sent.  Every rank of the group must
        call it.  Returns the received rows (rowptr int64, cols int64, vals
        float64) on the host."""
        import torch
        import torch.distributed as dist

        rowptr = np.asarray(rowptr, np.int64)
        cols = np.asarray(cols, np.int64)
        vals = np.asarray(vals, np.float64)
        lens = np.diff(rowptr)
        sent_len = lens[self.send_idx] if self.num_send else np.zeros(0, np.int64)
        send_len = torch.as_tensor(sent_len if len(sent_len) else np.zeros(1, np.int64),
                                   device=device)
        recv_len = torch.zeros(max(self.num_recv, 1), dtype=torch.int64, device=device)
        for w in self.exchange_packed(send_len, recv_len, group=group):
            w.wait()
        got_len = recv_len.cpu().numpy()[:self.num_recv]
        # the entries of the sent rows, row after row, message after message
        starts = rowptr[self.send_idx] if self.num_send else np.zeros(0, np.int64)
        total = int(sent_len.sum())
        pos = np.repeat(starts, sent_len) + (np.arange(total) - np.repeat(
            np.cumsum(sent_len) - sent_len, sent_len))
        send_eptr = np.concatenate([[0], np.cumsum(sent_len)])[self.send_ptr]
        recv_eptr = np.concatenate([[0], np.cumsum(got_len)])[self.recv_ptr]
        out = {}
        for name, data, dtype in (("cols", cols, torch.int64), ("vals", vals, torch.float64)):
            sbuf = torch.as_tensor(np.ascontiguousarray(data[pos]) if total else
                                   np.zeros(1, data.dtype), device=device)
            rbuf = torch.zeros(max(int(recv_eptr[-1]), 1), dtype=dtype, device=device)
            ops = []
            for k, q in enumerate(self.recv_procs):
                a, b = int(recv_eptr[k]), int(recv_eptr[k + 1])
                if b > a:
                    ops.append(dist.P2POp(dist.irecv, rbuf[a:b], q, group=group))
            for k, q in enumerate(self.send_procs):
                a, b = int(send_eptr[k]), int(send_eptr[k + 1])
                if b > a:
                    ops.append(dist.P2POp(dist.isend, sbuf[a:b], q, group=group))
            if ops:
                for w in dist.batch_isend_irecv(ops):
                    w.wait()
            out[name] = rbuf.cpu().numpy()[:int(recv_eptr[-1])]
        out_rowptr = np.zeros(self.num_recv + 1, np.int64)
        out_rowptr[1:] = np.cumsum(got_len)
        return out_rowptr, out["cols"], out["vals"]

    def exchange_packed_T(self, ghost_buf, recv_buf, group=None):
        """The transpose exchange (init_comm_T, core/comm_pkg.hpp:187-196):
        ghost_buf holds values in column-map order, each owner's run sent
        back to it; recv_buf receives, in send-list order, what the other
        ranks send for this rank's rows.  Returns the requests."""
        import torch.distributed as dist

        ops = []
        for k, q in enumerate(self.send_procs):
            a, b = int(self.send_ptr[k]), int(self.send_ptr[k + 1])
            ops.append(dist.P2POp(dist.irecv, recv_buf[a:b], q, group=group))
        for k, q in enumerate(self.recv_procs):
            a, b = int(self.recv_ptr[k]), int(self.recv_ptr[k + 1])
            ops.append(dist.P2POp(dist.isend, ghost_buf[a:b], q, group=group))
        return dist.batch_isend_irecv(ops) if ops else []


class DistParCSRMatrix:
    """This rank's rows of a row-partitioned matrix on its GPU
    (core/par_matrix.hpp:78-343): the on_proc and off_proc blocks as device
    CSR matrices, the halo plan, the packed send buffer and the ghost vector.
    Vectors are ParVector of the local size (local_num_rows)."""

    def __init__(self, partition, rank, rowptr, cols, vals, comm=None, group=None):
        import torch

        self.partition, self.rank, self.group = partition, int(rank), group
        first, last = partition.local_range(rank)
        self.local_num_rows = last - first
        if self.local_num_rows <= 0:
            # (the reference allows ranks without rows when n < p; here every
            # rank's blocks and vectors are device arrays of its rows)
            raise RaptorError(-1, "rank %d owns no rows: use fewer ranks than rows" % rank)
        if len(rowptr) != self.local_num_rows + 1:
            raise RaptorError(-1, "rowptr must have local_num_rows + 1 entries")
        (orp, oci, ocv), (frp, fci, fcv), self.colmap = split_rows(rowptr, cols, vals, first, last)
        self.on_proc = ParCSRMatrix.from_arrays(self.local_num_rows, self.local_num_rows, orp, oci, ocv)
        self.off_proc_num_cols = len(self.colmap)
        self.off_proc = (ParCSRMatrix.from_arrays(self.local_num_rows, self.off_proc_num_cols,
                                                  frp, fci, fcv)
                         if self.off_proc_num_cols else None)
        if comm is None:
            comm = ParComm.build(partition, self.colmap, rank, group=group, device="cuda")
        self.comm = comm
        with _on_stream():
            self.send_idx = torch.as_tensor(comm.send_idx, device="cuda")
            self.send_buf = torch.empty(max(comm.num_send, 1), dtype=torch.float64, device="cuda")
            self.recv_T = torch.empty(max(comm.num_send, 1), dtype=torch.float64, device="cuda")
        stream().synchronize()
        self.ghost = ParVector(max(self.off_proc_num_cols, 1))
        self.ghost_buf = self.ghost.torch_view()
        self.tmp = ParVector(max(self.local_num_rows, 1))
        stream()

    @classmethod
    def from_global(cls, rowptr, cols, vals, partition, rank, group=None, comm=None):
        """This rank's rows of a global host CSR matrix."""
        first, last = partition.local_range(rank)
        rowptr = np.asarray(rowptr, dtype=np.int64)
        a, b = int(rowptr[first]), int(rowptr[last])
        return cls(partition, rank, rowptr[first:last + 1] - a, np.asarray(cols)[a:b],
                   np.asarray(vals)[a:b], comm=comm, group=group)

    # ---------------------------------------------------------------- halo
    def pack(self, x):
        if self.comm.num_send:
            x.gather(self.send_idx.data_ptr(), self.comm.num_send, self.send_buf.data_ptr())

    def start_halo(self, x):
        self.pack(x)
        with _on_stream():
            return self.comm.exchange_packed(self.send_buf, self.ghost_buf, group=self.group)

    @staticmethod
    def _wait(reqs):
        with _on_stream():
            for w in reqs:
                w.wait()

    # ---------------------------------------------------------- row exchange
    def communicate_rows(self, device="cuda"):
        """The P-row exchange of the distributed Galerkin product
        (CommPkg::communicate(ParCSRMatrix*), core/comm_mat.cpp:39-96): this
        rank's rows that the other ranks' column maps name go to them, and the
        rows this rank's column map names arrive, whole, with global column
        indices (on_proc entries first), in column-map order, on the host."""
        on = self.on_proc.arrays()
        if self.off_proc is not None:
            off = self.off_proc.arrays()
        else:
            off = (np.zeros(self.local_num_rows + 1, np.int32), np.zeros(0, np.int32),
                   np.zeros(0, np.float64))
        first = self.partition.local_range(self.rank)[0]
        rows = global_rows(on, off, first, self.colmap)
        return self.comm.communicate_rows(*rows, group=self.group, device=device)

    # ------------------------------------------------------------ products
    def mult(self, x, b):
        """b = A x (par_spmv.cpp:25-59): halo exchange in flight while the
        on_proc product runs, then b += off_proc * ghost."""
        reqs = self.start_halo(x)
        self.on_proc.mult(x, b)
        self._wait(reqs)
        if self.off_proc is not None:
            self.off_proc.mult_append(self.ghost, b)

    def mult_append(self, x, b):
        """b += A x (par_spmv.cpp:91-125)."""
        reqs = self.start_halo(x)
        self.on_proc.mult_append(x, b)
        self._wait(reqs)
        if self.off_proc is not None:
            self.off_proc.mult_append(self.ghost, b)

    def _add_received_T(self, b):
        """b[send_idx] += received values, one message after another (a row
        can arrive from several ranks; within a message rows are distinct)."""
        c = self.comm
        for k in range(len(c.send_procs)):
            a, e = int(c.send_ptr[k]), int(c.send_ptr[k + 1])
            b.scatter_add(self.send_idx.data_ptr() + 4 * a, self.recv_T.data_ptr() + 8 * a, e - a)

    def mult_T(self, x, b):
        """b = A^T x (par_spmv.cpp:157-187; A square, x and b partitioned like
        the rows): off_proc^T x goes back to the owners of those columns
        while on_proc^T x is formed, then the received values are added."""
        if self.off_proc is not None:
            self.off_proc.mult_T(x, self.ghost)
        with _on_stream():
            reqs = self.comm.exchange_packed_T(self.ghost_buf, self.recv_T, group=self.group)
        self.on_proc.mult_T(x, b)
        self._wait(reqs)
        self._add_received_T(b)

    def residual(self, x, b, r):
        """r = b - A x (par_spmv.cpp:215-252)."""
        reqs = self.start_halo(x)
        self.on_proc.residual(x, b, r)
        self._wait(reqs)
        if self.off_proc is not None:
            self.off_proc.mult(self.ghost, self.tmp)
            r.axpy(self.tmp, -1.0)

    # ---------------------------------------------------------------- dots
    def inner_product(self, x, y):
        """Global x.y: local dots summed over the ranks (par_vector.cpp:101-121)."""
        import torch
        import torch.distributed as dist

        with _on_stream():
            t = torch.tensor([x.inner_product(y)], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, group=self.group)
            return float(t.item())

    def norm(self, x):
        return float(np.sqrt(self.inner_product(x, x)))

    # ------------------------------------------- partitions in one process
    @staticmethod
    def exchange_in_process(mats, xs):
        """The halo exchange between partitions held by one process (several
        partitions on one GPU): each partition's packed values copied into
        the ghost vectors of the partitions that need them."""
        for m, x in zip(mats, xs):
            m.pack(x)
        with _on_stream():
            for q, mq in enumerate(mats):
                for k, r in enumerate(mq.comm.recv_procs):
                    mr = mats[r]
                    j = mr.comm.send_procs.index(q)
                    a, b = int(mr.comm.send_ptr[j]), int(mr.comm.send_ptr[j + 1])
                    c, d = int(mq.comm.recv_ptr[k]), int(mq.comm.recv_ptr[k + 1])
                    mq.ghost_buf[c:d].copy_(mr.send_buf[a:b])

    @staticmethod
    def mult_in_process(mats, xs, bs):
        """b_r = (A x)_r for every partition r held by this process."""
        DistParCSRMatrix.exchange_in_process(mats, xs)
        for m, x, b in zip(mats, xs, bs):
            m.on_proc.mult(x, b)
            if m.off_proc is not None:
                m.off_proc.mult_append(m.ghost, b)

    @staticmethod
    def mult_T_in_process(mats, xs, bs):
        """b_r = (A^T x)_r for every partition r held by this process."""
        for m, x in zip(mats, xs):
            if m.off_proc is not None:
                m.off_proc.mult_T(x, m.ghost)
        with _on_stream():
            for q, mq in enumerate(mats):
                for k, r in enumerate(mq.comm.send_procs):
                    mr = mats[r]
                    j = mr.comm.recv_procs.index(q)
                    a, b = int(mr.comm.recv_ptr[j]), int(mr.comm.recv_ptr[j + 1])
                    c, d = int(mq.comm.send_ptr[k]), int(mq.comm.send_ptr[k + 1])
                    mq.recv_T[c:d].copy_(mr.ghost_buf[a:b])
        for m, x, b in zip(mats, xs, bs):
            m.on_proc.mult_T(x, b)
            m._add_received_T(b)

    @staticmethod
    def residual_in_process(mats, xs, bs, rs):
        DistParCSRMatrix.exchange_in_process(mats, xs)
        for m, x, b, r in zip(mats, xs, bs, rs):
            m.on_proc.residual(x, b, r)
            if m.off_proc is not None:
                m.off_proc.mult(m.ghost, m.tmp)
                r.axpy(m.tmp, -1.0)


# ------------------------------------------------------------------ Krylov --
class Partitions:
    """The partitions of one row-partitioned matrix that this process holds:
    one (a process per GPU; products exchange over the process group, dots
    all_reduce) or all of them (several partitions in one process; products
    exchange by device copies, dots add up locally).  Vectors are lists of
    ParVector, one per held partition."""

    def __init__(self, mats, in_process=None):
        import torch.distributed as dist

        self.mats = list(mats)
        world = self.mats[0].partition.world
        if in_process is None:
            in_process = len(self.mats) == world and (world > 1 or not dist.is_initialized())
        if in_process and len(self.mats) != world:
            raise RaptorError(-1, "in-process partitions must be all %d partitions" % world)
        if not in_process and len(self.mats) != 1:
            raise RaptorError(-1, "a process of a process group holds one partition")
        self.in_process = in_process
        self.global_n = self.mats[0].partition.global_num_rows

    def vectors(self, values=None):
        """New vectors, from a global array of values (or zero)."""
        out = []
        for m in self.mats:
            f, l = m.partition.local_range(m.rank)
            v = ParVector(self.global_n, local_n=l - f, first_local=f)
            if values is not None:
                v.set_values(np.asarray(values, dtype=np.float64)[f:l])
            else:
                v.set_const_value(0.0)
            out.append(v)
        return out

    def mult(self, xs, ys):
        if self.in_process:
            DistParCSRMatrix.mult_in_process(self.mats, xs, ys)
        else:
            self.mats[0].mult(xs[0], ys[0])

    def residual(self, xs, bs, rs):
        if self.in_process:
            DistParCSRMatrix.residual_in_process(self.mats, xs, bs, rs)
        else:
            self.mats[0].residual(xs[0], bs[0], rs[0])

    def dot(self, xs, ys):
        if self.in_process:
            return float(sum(x.inner_product(y) for x, y in zip(xs, ys)))
        return self.mats[0].inner_product(xs[0], ys[0])

    def norm(self, xs):
        return float(np.sqrt(self.dot(xs, xs)))

    @staticmethod
    def axpy(ys, xs, a):
        for y, x in zip(ys, xs):
            y.axpy(x, a)

    @staticmethod
    def scale(ys, a):
        for y in ys:
            y.scale(a)

    @staticmethod
    def copy(ys, xs):
        for y, x in zip(ys, xs):
            y.copy(x)

    @staticmethod
    def set_const(ys, v):
        for y in ys:
            y.set_const_value(v)


class BlockJacobiAMG:
    """Preconditioner of the distributed PCG: one AMG V-cycle per partition
    on its own on_proc block (block Jacobi over the partitions, an AMG solve
    of each block).  The reference's PCG at several ranks cycles one
    distributed hierarchy instead, whose setup is not built here; at one
    partition the two are the same.  ``make_solver()`` returns an unset-up
    ParMultilevel (for example ParRugeStubenSolver(...))."""

    def __init__(self, parts, make_solver):
        self.parts = parts
        self.levels = []
        for m in parts.mats:
            ml = make_solver()
            ml.setup(m.on_proc)
            self.levels.append(ml)

    def cycle(self, zs, rs):
        """z = M^-1 r from z = 0, on every held partition."""
        for ml, z, r in zip(self.levels, zs, rs):
            z.set_const_value(0.0)
            ml.cycle(z, r)


def _breakdown():
    from ._capi import Breakdown

    return Breakdown(-4, "Indefinite matrix detected in CG")


def CG(parts, xs, bs, res, tol=1e-5, max_iter=-1):
    """Conjugate gradients over the partitions (krylov/par_cg.cpp:8-118): the
    true residual every 8 iterations (and first), stopping when ||r|| <= tol
    ||r_0||; res gets ||r|| / ||b|| per iteration.  Returns 0 when it
    converged, -5 at the iteration limit; p.Ap < 0 raises Breakdown (the
    reference exits)."""
    P = parts
    r, p, Ap = P.vectors(), P.vectors(), P.vectors()
    b_norm = P.norm(bs)
    if b_norm < 1e-16:
        b_norm = 1.0
    if max_iter <= 0:
        max_iter = int(1.3 * P.global_n) + 2
    P.residual(xs, bs, r)
    P.copy(p, r)
    rr = P.dot(r, r)
    norm_r = float(np.sqrt(rr))
    res.append(norm_r / b_norm)
    if norm_r != 0.0:
        tol = tol * norm_r
    recompute_r, it = 8, 0
    while norm_r > tol and it < max_iter:
        P.mult(p, Ap)
        app = P.dot(Ap, p)
        if app < 0.0 or not np.isfinite(app):
            raise _breakdown()
        alpha = rr / app
        P.axpy(xs, p, alpha)
        if (it % recompute_r) and it > 0:
            P.axpy(r, Ap, -alpha)
        else:
            P.residual(xs, bs, r)
        nxt = P.dot(r, r)
        beta = nxt / rr
        P.scale(p, beta)
        P.axpy(p, r, 1.0)
        rr = nxt
        norm_r = float(np.sqrt(rr))
        res.append(norm_r / b_norm)
        it += 1
    return -5 if it == max_iter and norm_r > tol else 0


def PCG(parts, precond, xs, bs, res, tol=1e-5, max_iter=-1):
    """Preconditioned CG over the partitions (krylov/par_cg.cpp:121-263),
    with the reference's stopping rule and history: the first entry is
    sqrt(r.z), then (r.z) / (b.Mb) per iteration, stopping when r.z < tol
    sqrt(b.Mb); the true residual every 8 iterations.  ``precond.cycle(z, r)``
    applies M^-1 from z = 0 (BlockJacobiAMG).  Returns 0 or -5 as CG."""
    P = parts
    r, z, p, Ap = P.vectors(), P.vectors(), P.vectors(), P.vectors()
    if max_iter <= 0:
        max_iter = int(1.3 * P.global_n) + 2
    precond.cycle(z, bs)
    b_inner = P.dot(bs, z)
    norm_b = float(np.sqrt(b_inner))
    if norm_b > 1e-16:
        tol = tol * norm_b
    P.residual(xs, bs, r)
    precond.cycle(z, r)
    P.copy(p, z)
    rz = P.dot(r, z)
    res.append(float(np.sqrt(rz)))
    recompute_r, it, converged = 8, 0, False
    while it < max_iter:
        it += 1
        P.mult(p, Ap)
        app = P.dot(Ap, p)
        if app < 0.0 or not np.isfinite(app):
            raise _breakdown()
        alpha = rz / app
        P.axpy(xs, p, alpha)
        full_r = recompute_r and it % recompute_r == 0
        if full_r:
            P.residual(xs, bs, r)
        else:
            P.axpy(r, Ap, -alpha)
        precond.cycle(z, r)
        nxt = P.dot(r, z)
        beta = nxt / rz
        res.append(nxt / b_inner)
        if nxt < tol:
            converged = True
            break
        if full_r:
            P.copy(p, z)
        else:
            P.scale(p, beta)
            P.axpy(p, z, 1.0)
        rz = nxt
    return 0 if converged else -5
