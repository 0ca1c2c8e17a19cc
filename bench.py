"""Benchmark: AMG-preconditioned CG to 1e-8 relative residual on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--size 192] [--impl b200|reference]

A step is one complete AMG-PCG solve (x0 = 0, stop at ||b - A x|| / ||b|| <
1e-8) of the 3D 27-point Laplacian (laplace_stencil_27pt through
par_stencil_grid) on a size^3 grid with b uniform in [-1, 1] from a fixed
seed; Ruge-Stuben AMG with classical strength 0.25, PMIS, extended+i
interpolation (filter 0.3) and L1-Jacobi.  The hierarchy and V-cycle run in
FP32, the outer CG (residual, dots, A p) and the coarse LU in FP64.  The same
solve with an all-FP64 hierarchy is timed too (`fp64_form`), giving the
FP32/FP64 speed-up at the same verified accuracy.

Inputs stay resident in HBM during the device-timed steps (the FP64 matrix
alone is larger than L2, so no flush is needed); `e2e` times the public API
with host buffers: pinned b uploaded and x downloaded every step.

Under torchrun each rank solves its own copy (replicas; the solve does not
shard), timings are the max over ranks.

`--impl reference` times the reference's own solve path on the host, rank 0
only: its ParRugeStubenSolver setup (untimed) and PCG, compiled unmodified
into oracle/_ref against a single-rank MPI stand-in (one core: the
reference has no threads), on the same 192^3 problem, with the reference's
default SOR smoother (it has no L1-Jacobi) and its PCG tolerance calibrated
so that the solution meets the same ||b - A x|| / ||b|| <= 1e-8.  Where that
build is absent, the CPU restatement (oracle/) runs the same solve instead,
on every host core.  The GPU line's `cpu_baseline` is one such reference
solve on the hierarchy the GPU built (bit-identical to the reference's own
setup, as the parity tests show), so the sample needs no CPU setup.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 20261203
METRIC = "AMG-PCG time to 1e-8 rel-res"
TOL = 1e-8
WORKLOAD = ("laplacian27 %d^3, b ~ U[-1,1]: AMG-PCG to ||b - A x|| / ||b|| <= 1e-8 "
            "(RS: classical strength 0.25, PMIS, extended+i interpolation, filter 0.3)")
# the reference's solver options for the same problem (its default SOR
# smoother: its Jacobi sweep is a no-op and it has no L1-Jacobi)
REF_KW = dict(theta=0.25, coarsen="pmis", interp="extended", interp_filter=0.3, relax="sor")


def bench_config(S, n, nnz, levels, world):
    """The workload both arms report (the smoother and precisions each arm
    uses are reported beside it, under "method")."""
    return {"workload": WORKLOAD % S, "rows": n, "nnz": nnz, "levels": levels,
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (A0 FP64 = %.2f GB)" % (nnz * 12 / 1e9)}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--size", type=int, default=192)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--cpu-sample", type=int, default=96)
    p.add_argument("--batch-size", type=int, default=160,
                   help="grid side of the k right-hand-side workload (0 skips it)")
    p.add_argument("--batch-ks", default="1,8,32",
                   help="comma-separated right-hand-side counts of that workload")
    p.add_argument("--systems", type=int, default=64,
                   help="independent systems of the uneven batch (0 skips it)")
    p.add_argument("--diff-size", type=int, default=512,
                   help="grid side of the differentiation workload (0 skips it)")
    p.add_argument("--aniso-size", type=int, default=4096,
                   help="grid side of the 2D anisotropic precision-form workload "
                        "(0 skips it)")
    p.add_argument("--plain-size", type=int, default=128,
                   help="grid side of the all-FP64 plain-method workload with its "
                        "SpMV and V-cycle bandwidth figures (0 skips it)")
    p.add_argument("--bsr-cases", default="96x3,112x2,64x4",
                   help="block CSR product workloads as grid-side x block-size, "
                        "comma-separated (empty skips them)")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Dist:
    """Replica bookkeeping across ranks: a barrier and the max of a scalar.
    NCCL on GPUs (one rank per GPU), gloo on CPU; rendezvous from the
    torchrun environment (MASTER_ADDR / MASTER_PORT)."""

    def __init__(self, world, local, backend=None):
        self.world = world
        self.pg = None
        if world > 1:
            import datetime

            import torch
            import torch.distributed as td
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            self.device = "cuda" if backend == "nccl" else "cpu"
            if backend == "nccl":
                torch.cuda.set_device(local)
            td.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.td = td
            self.torch = torch

    def barrier(self):
        if self.world > 1:
            self.td.barrier()

    def max(self, v):
        if self.world == 1:
            return v
        t = self.torch.tensor([float(v)], device=self.device)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.td.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:  # noqa: BLE001
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout=3.0):
        """Block until nvidia-smi has printed a sample (it takes a moment to
        start), so that the timed region that follows is sampled."""
        t0 = time.perf_counter()
        while self.proc and not self.lines and time.perf_counter() - t0 < timeout:
            time.sleep(0.02)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:  # noqa: BLE001
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ b200 ----
def a_bytes(ml, l, vbytes):
    """Bytes of one pass over A_l in its stored format: CSR z(v+4) + (n+1)4,
    the sliced diagonals nd * 32 ceil(n/32) v (no indices), or, for
    diagonals with constant coefficients, one 4-byte mask a row (none in the
    box-grid form, whose kernels read only the vectors)."""
    n, z, _ = ml.level_info(l)
    nd = ml.level_storage(l)
    cc = ml.level_const_coef(l) if nd else 0
    if cc == 2:
        return 0
    if cc:
        return 4 * n
    if nd:
        return nd * 32 * ((n + 31) // 32) * vbytes
    return z * (vbytes + 4) + (n + 1) * 4


def cycle_bytes(ml, vbytes):
    """Algorithmic bytes of one V-cycle (1 pre- and 1 post-sweep, zero guess).

    Per level l with n rows, p = nnz(P_l), v = value bytes, i = 4: B_A = one
    pass over A_l in its stored format (a_bytes), B_P = B_R = p(v+i) +
    (rows+1)i.  Pre-smooth from a zero guess reads b and the inverse diagonal
    and writes x (3nv), then the residual B_A + 3nv; where the level runs the
    two as one pass (level_fused_first) that pass is B_A + 4nv (b, D^-1 in,
    x, r out); restriction B_R + n v + n_c v; prolongation B_P + (2n + n_c) v;
    post-smooth B_A + 4nv (x, b, D^-1 in, x out).  Coarsest level: the dense
    inverse product (n_c^2 8 bytes)."""
    L = ml.num_levels
    tot = 0.0
    per = []
    for l in range(L):
        n, z, p = ml.level_info(l)
        if l == L - 1:
            b = 1.0 * n * n * 8
        else:
            nc = ml.level_info(l + 1)[0]
            BA = a_bytes(ml, l, vbytes)
            BP = p * (vbytes + 4) + (n + 1) * 4
            BR = p * (vbytes + 4) + (nc + 1) * 4
            if ml.level_fused_first(l):
                first = BA + 4 * n * vbytes
            else:
                first = (3 * n * vbytes) + (BA + 3 * n * vbytes)
            b = first + (BR + n * vbytes + nc * vbytes) + \
                (BP + (2 * n + nc) * vbytes) + (BA + 4 * n * vbytes)
        per.append(b)
        tot += b
    return tot, per


def aniso7_stencil(cz=0.01):
    """3D 7-point anisotropic diffusion (1, 1, cz) as a 27-entry stencil."""
    st = [0.0] * 27
    st[13] = 4.0 + 2.0 * cz
    st[12] = st[14] = -1.0
    st[10] = st[16] = -1.0
    st[4] = st[22] = -cz
    return st


def run_batching(rb, ev, sync, S, ks=(1, 8, 32), steps=2):
    """k right-hand sides over one smoothed-aggregation hierarchy: the
    7-point anisotropic diffusion (1, 1, 0.01) on S^3, FP32 V-cycle, FP64
    outer CG, each column to 1e-8 true relative residual."""
    A = rb.par_stencil_grid(aniso7_stencil(), [S, S, S])
    n = A.global_num_rows
    ml = rb.ParSmoothedAggregationSolver(0.25, relax_type=rb.L1Jacobi)
    ml.precision = rb.FP32
    ml.setup(A)
    out = {"workload": "SA (symmetric strength 0.25, mis2 aggregates, Jacobi-smoothed "
                       "prolongator, L1-Jacobi) on 7-point aniso (1, 1, 0.01) %d^3, FP32 "
                       "V-cycle, FP64 outer CG to 1e-8 per column" % S,
           "rows": n, "nnz": A.local_nnz, "levels": ml.num_levels,
           "setup_s": ml.setup_seconds, "k": {}}
    rng = np.random.default_rng(SEED + 7)
    for k in ks:
        Bv = rb.ParVector(n * k, values=rng.uniform(-1.0, 1.0, n * k))
        Xv = rb.ParVector(n * k)
        times = []
        iters = relres = None
        for s in range(1 + steps):
            Xv.set_const_value(0.0)
            sync()
            e0 = ev()
            rc, iters, relres = rb.PCG_block(A, ml, Xv, Bv, k, tol=TOL, max_iter=500)
            e1 = ev()
            sync()
            if s >= 1:
                times.append(e0.elapsed_time(e1))
        ms = sum(times) / len(times)
        out["k"][str(k)] = {"ms": ms, "ms_per_rhs": ms / k, "iters_max": int(max(iters)),
                            "iters_min": int(min(iters)),
                            "max_true_rel_res": float(max(relres)), "status": rc}
        del Bv, Xv
    k1 = out["k"].get("1")
    for k in ks:
        if k1 and k != 1:
            out["k"][str(k)]["per_rhs_speedup_vs_k1"] = k1["ms"] / out["k"][str(k)]["ms_per_rhs"]
    return out


def run_aniso_precision(rb, ev, sync, S, steps=2):
    """The precision form's second workload: 2D rotated anisotropic
    diffusion (eps 0.001, theta pi/8) on S^2, RS (PMIS, extended+i,
    L1-Jacobi), PCG in true-residual mode to 1e-8, FP32 and FP64 cycles."""
    A = rb.par_stencil_grid(rb.diffusion_stencil_2d(0.001, math.pi / 8.0), [S, S])
    n = A.global_num_rows
    b = rb.ParVector(n, values=np.random.default_rng(SEED).uniform(-1.0, 1.0, n))
    out = {"workload": "aniso (eps 0.001, theta pi/8) %d^2 AMG-PCG to 1e-8 (RS PMIS, "
                       "extended+i, L1-Jacobi)" % S, "rows": n, "nnz": A.local_nnz}
    for name, prec in (("fp32", rb.FP32), ("fp64", rb.FP64)):
        ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
        ml.precision = prec
        ml.setup(A)
        x = rb.ParVector(n)
        times, res = [], []
        for s in range(1 + steps):
            x.set_const_value(0.0)
            res = []
            sync()
            e0 = ev()
            rb.PCG(A, ml, x, b, res, tol=TOL, max_iter=500, mode=rb.PCG_TRUE_RESIDUAL)
            e1 = ev()
            sync()
            if s >= 1:
                times.append(e0.elapsed_time(e1))
        out[name] = {"ms": sum(times) / len(times), "iters": len(res) - 1,
                     "final_rel_res": float(res[-1]), "setup_s": ml.setup_seconds,
                     "levels": ml.num_levels}
        del ml
    out["speedup_fp32_over_fp64"] = out["fp64"]["ms"] / out["fp32"]["ms"]
    return out


def run_plain_fp64(rb, ev, sync, S, steps=3):
    """The plain method at scale in FP64: laplacian27 on S^3, RS (PMIS,
    extended+i, L1-Jacobi), hierarchy and V-cycle in FP64, PCG to 1e-8 true
    relative residual (b = A 1); plus the standalone bandwidth figures on the
    finest matrix the reference's examples/benchmark_spmv.cpp times: one
    SpMV b = A x through the public entry point on the caller's FP64 CSR
    matrix, and one FP64 V-cycle."""
    A = rb.par_stencil_grid(rb.laplace_stencil_27pt(), [S, S, S])
    n = A.global_num_rows
    nnz = A.local_nnz
    ones = rb.ParVector(n)
    ones.set_const_value(1.0)
    b = rb.ParVector(n)
    A.mult(ones, b)
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
    ml.precision = rb.FP64
    ml.setup(A)
    x = rb.ParVector(n)
    times, res = [], []
    for s in range(1 + steps):
        x.set_const_value(0.0)
        res = []
        sync()
        e0 = ev()
        rb.PCG(A, ml, x, b, res, tol=TOL, max_iter=500, mode=rb.PCG_TRUE_RESIDUAL)
        e1 = ev()
        sync()
        if s >= 1:
            times.append(e0.elapsed_time(e1))
    # SpMV through rb_spmv on the FP64 CSR matrix: 12 B a nonzero, the row
    # pointers, x gathered once and b written (algorithmic bytes)
    y = rb.ParVector(n)
    A.mult(ones, y)
    sync()
    reps = 20
    e0 = ev()
    for _ in range(reps):
        A.mult(ones, y)
    e1 = ev()
    sync()
    spmv_ms = e0.elapsed_time(e1) / reps
    spmv_bytes = nnz * 12 + (n + 1) * 4 + 2 * n * 8
    cyc_ms = ml.time_operator(0, 5, reps=20)
    cb, _ = cycle_bytes(ml, 8)
    peak, kind = peaks()
    return {"workload": "laplacian27 %d^3, b = A 1: AMG-PCG to 1e-8 (RS: PMIS, extended+i, "
                        "L1-Jacobi), hierarchy, V-cycle and PCG all FP64" % S,
            "rows": n, "nnz": nnz, "levels": ml.num_levels, "setup_s": ml.setup_seconds,
            "pcg_ms": sum(times) / len(times), "iters": len(res) - 1,
            "final_rel_res": float(res[-1]),
            "spmv": {"ms": spmv_ms, "alg_bytes": spmv_bytes,
                     "gbs": spmv_bytes / (spmv_ms * 1e-3) / 1e9,
                     "frac_of_%s_peak" % kind: spmv_bytes / (spmv_ms * 1e-3) / 1e9 / peak,
                     "storage": "the caller's CSR, FP64 values, int32 indices"},
            "vcycle": {"ms": cyc_ms, "alg_bytes": cb,
                       "gbs": cb / (cyc_ms * 1e-3) / 1e9,
                       "frac_of_%s_peak" % kind: cb / (cyc_ms * 1e-3) / 1e9 / peak}}


def block_stencil_pattern(m):
    """Block pattern of a periodic 7-point stencil on an m^3 grid of blocks:
    every block row holds 7 blocks (itself first, then its six neighbours)."""
    idx = np.arange(m ** 3).reshape(m, m, m)
    cols = [np.roll(idx, (-dz, -dy, -dx), axis=(0, 1, 2)).reshape(-1)
            for dz, dy, dx in [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0),
                               (0, 0, -1), (0, 0, 1)]]
    cols = np.stack(cols, axis=1).astype(np.int32).reshape(-1)
    rowptr = (np.arange(m ** 3 + 1) * 7).astype(np.int32)
    return rowptr, cols


def run_block_csr(rb, ev, sync, cases, reps=40):
    """Block CSR (BSRMatrix) products: b = A x and b = A^T x on a 7-point
    block pattern with b x b blocks of uniform values, and b = A x on the
    same matrix expanded to CSR (to_CSR).  Algorithmic bytes of the block
    product: the blocks (b^2 8 + 4 B each), the row pointers, x and b."""
    peak, kind = peaks()
    out = []
    for m, bsz in cases:
        rowptr, cols = block_stencil_pattern(m)
        nb = m ** 3
        vals = np.random.default_rng(SEED).uniform(-1.0, 1.0, len(cols) * bsz * bsz)
        A = rb.BSRMatrix.from_arrays(nb, nb, bsz, bsz, rowptr, cols, vals)
        n = nb * bsz
        x = rb.ParVector(n, values=np.random.default_rng(SEED + 1).uniform(-1.0, 1.0, n))
        y = rb.ParVector(n)

        def timed(f):
            for _ in range(5):
                f()
            sync()
            e0 = ev()
            for _ in range(reps):
                f()
            e1 = ev()
            sync()
            return e0.elapsed_time(e1) / reps

        alg = len(cols) * (bsz * bsz * 8 + 4) + (nb + 1) * 4 + 2 * n * 8
        mult_ms = timed(lambda: A.mult(x, y))
        mult_t_ms = timed(lambda: A.mult_T(x, y))
        Acsr = A.to_CSR()
        z = Acsr.local_nnz
        csr_alg = z * 12 + (n + 1) * 4 + 2 * n * 8
        csr_ms = timed(lambda: Acsr.mult(x, y))
        out.append({"grid": "%d^3 blocks" % m, "block": "%dx%d" % (bsz, bsz),
                    "block_rows": nb, "blocks": len(cols), "alg_bytes": alg,
                    "mult_ms": mult_ms, "mult_gbs": alg / (mult_ms * 1e-3) / 1e9,
                    "mult_frac_of_%s_peak" % kind: alg / (mult_ms * 1e-3) / 1e9 / peak,
                    "mult_T_ms": mult_t_ms,
                    "mult_T_gbs": alg / (mult_t_ms * 1e-3) / 1e9,
                    "csr_nnz": z, "csr_alg_bytes": csr_alg, "csr_mult_ms": csr_ms,
                    "csr_mult_gbs": csr_alg / (csr_ms * 1e-3) / 1e9,
                    "bsr_speedup_over_csr": csr_ms / mult_ms})
        del A, Acsr, x, y
    return {"workload": "BSRMatrix products on a periodic 7-point block pattern, FP64 "
                        "blocks ~ U[-1, 1]; CSR product of the same matrix after to_CSR",
            "cases": out}


def run_uneven_batch(rb, ev, sync, count=64, steps=2):
    """An uneven batch of independent 2D rotated-diffusion systems: grid side
    log-uniform in [64, 1024], eps log-uniform in [1e-3, 1], theta uniform in
    [0, pi] (seeded); RS AMG (PMIS, extended+i, L1-Jacobi), FP32 V-cycle, FP64
    outer CG per system to 1e-8.  The batch solves all systems together; the
    baseline solves them one after another with standalone hierarchies."""
    rng = np.random.default_rng(SEED + 64)
    mats, params = [], []
    for _ in range(count):
        side = int(round(math.exp(rng.uniform(math.log(64), math.log(1024)))))
        eps = math.exp(rng.uniform(math.log(1e-3), 0.0))
        theta = rng.uniform(0.0, math.pi)
        params.append((side, eps, theta))
        mats.append(rb.par_stencil_grid(rb.diffusion_stencil_2d(eps, theta), [side, side]))

    def opts():
        ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
        ml.precision = rb.FP32
        return ml

    t0 = time.perf_counter()
    B = rb.Batch(mats, opts())
    setup_s = time.perf_counter() - t0
    N = B.total_rows
    bh = rng.uniform(-1.0, 1.0, N)
    b = rb.ParVector(N, values=bh)
    x = rb.ParVector(N)
    times = []
    iters = relres = None
    for s in range(1 + steps):
        x.set_const_value(0.0)
        sync()
        e0 = ev()
        rc, iters, relres = B.pcg(x, b, tol=TOL, max_iter=500)
        e1 = ev()
        sync()
        if s >= 1:
            times.append(e0.elapsed_time(e1))
    batch_ms = sum(times) / len(times)
    # baseline: the same systems solved one after another
    singles = []
    for s, A in enumerate(mats):
        ml = opts()
        ml.setup(A)
        lo, hi = int(B.offsets[s]), int(B.offsets[s + 1])
        singles.append((A, ml, rb.ParVector(hi - lo, values=bh[lo:hi]), rb.ParVector(hi - lo)))
    seq = []
    for s in range(1 + steps):
        sync()
        e0 = ev()
        for A, ml, bs, xs in singles:
            xs.set_const_value(0.0)
            rb.PCG(A, ml, xs, bs, [], tol=TOL, max_iter=500, mode=rb.PCG_TRUE_RESIDUAL)
        e1 = ev()
        sync()
        if s >= 1:
            seq.append(e0.elapsed_time(e1))
    seq_ms = sum(seq) / len(seq)
    sides = [p[0] for p in params]
    rows = [int(B.offsets[s + 1]) - int(B.offsets[s]) for s in range(count)]
    # the row work the systems need (each its own iterations) against running
    # every system for the slowest one's iterations
    need = sum(int(i) * r for i, r in zip(iters, rows)) / (max(int(i) for i in iters) * N)
    return {"workload": "%d rotated-diffusion systems, side log-uniform [64, 1024], eps "
                        "log-uniform [1e-3, 1], theta uniform [0, pi]; RS PMIS extended+i "
                        "L1-Jacobi, FP32 V-cycle, FP64 outer CG per system to 1e-8" % count,
            "total_rows": N, "side_min": min(sides), "side_max": max(sides),
            "packed_levels": int(max(B.levels)), "setup_s": setup_s, "status": rc,
            "batch_ms": batch_ms, "sequential_ms": seq_ms, "speedup_vs_sequential": seq_ms / batch_ms,
            "iters_max": int(max(iters)), "iters_min": int(min(iters)),
            "row_iterations_needed_vs_all_to_max": need,
            "stopped_systems": "skipped by the row gates (each system's rows leave the cycle "
                               "and the outer iteration once it has converged)",
            "max_true_rel_res": float(max(relres))}


def run_differentiation(rb, ev, sync, side=512, steps=3):
    """Forward and backward of x = A(k)^-1 b through the torch.autograd
    harness: 5-point finite-volume diffusion with harmonic-mean faces on a
    side^2 grid, k = exp(g) with g a Gaussian random field (correlation
    length 32 cells, unit variance), L = 0.5 ||x - x_t||^2; FP32 V-cycle,
    FP64 outer PCG and adjoint PCG to 1e-8."""
    import torch
    from raptor_b200 import autograd as AG

    n = side * side
    g = torch.tensor(AG.grf(side, side, 32.0, seed=SEED), dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(SEED + 5)
    b = torch.tensor(rng.uniform(-1.0, 1.0, n), dtype=torch.float64, device="cuda")
    xt = torch.tensor(rng.uniform(0.0, 1.0, n), dtype=torch.float64, device="cuda")
    fwd, bwd = [], []
    for s in range(1 + steps):
        gg = g.clone().requires_grad_(True)
        bb = b.clone().requires_grad_(True)
        torch.cuda.synchronize()
        sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e2 = torch.cuda.Event(enable_timing=True)
        e0.record()
        x = AG.DiffusionSolve.apply(torch.exp(gg), bb, side, side, TOL, 500, rb.FP32)
        loss = 0.5 * ((x - xt) ** 2).sum()
        e1.record()
        loss.backward()
        e2.record()
        torch.cuda.synchronize()
        sync()
        if s >= 1:
            fwd.append(e0.elapsed_time(e1))
            bwd.append(e1.elapsed_time(e2))
    return {"workload": "FV diffusion %d^2, harmonic-mean faces, k = exp(GRF, corr 32, var 1); "
                        "L = 0.5||x - x_t||^2; forward AMG-PCG + adjoint AMG-PCG, SDDMM, assembly "
                        "backward (RS PMIS extended+i, L1-Jacobi, FP32 V-cycle, FP64 outer, 1e-8)"
                        % side,
            "rows": n, "forward_ms": sum(fwd) / len(fwd), "backward_ms": sum(bwd) / len(bwd),
            "forward_includes": "assembly, AMG setup, PCG",
            "backward_includes": "adjoint PCG, SDDMM, assembly backward",
            "grad_g_norm": float(gg.grad.norm()), "grad_b_norm": float(bb.grad.norm())}


def run_b200(args, rank, world, local):
    import raptor_b200 as rb

    import ctypes as C
    import torch

    dist = Dist(world, local)
    rb.init(local)
    # every library call is ordered on this stream; the CUDA events that time
    # the steps are recorded on it
    ts = torch.cuda.Stream(device=local)
    rb.check(rb.lib().rb_set_stream(C.c_void_p(ts.cuda_stream)))

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(ts)
        return e
    S = args.size
    A = rb.par_stencil_grid(rb.laplace_stencil_27pt(), [S, S, S])
    n = A.global_num_rows
    nnz = A.local_nnz
    bh = np.random.default_rng(SEED).uniform(-1.0, 1.0, n)
    b = rb.ParVector(n, values=bh)
    x = rb.ParVector(n)
    bnorm = float(np.linalg.norm(bh))

    def make(prec, const_coef=1):
        ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
        ml.precision = prec
        ml.const_coef = const_coef
        ml.setup(A)
        return ml

    def solve(ml):
        x.set_const_value(0.0)
        res = []
        rc = rb.PCG(A, ml, x, b, res, tol=TOL, max_iter=500, mode=rb.PCG_TRUE_RESIDUAL)
        return rc, len(res) - 1

    def timed(ml, steps, warmup):
        for _ in range(warmup):
            solve(ml)
        rb.lib().rb_synchronize()
        dist.barrier()
        c0 = rb.launch_count()
        e0 = ev()
        iters = []
        for _ in range(steps):
            rc, it = solve(ml)
            iters.append(it)
        e1 = ev()
        rb.lib().rb_synchronize()
        el = e0.elapsed_time(e1) * 1e-3
        launches = rb.launch_count() - c0
        dist.barrier()
        return dist.max(el) / steps, iters, launches

    def true_relres():
        r = rb.ParVector(n)
        A.residual(x, b, r)
        return r.norm(2) / bnorm

    ml32 = make(rb.FP32)
    setup32 = ml32.setup_seconds
    clocks = ClockSampler(local)
    clocks.start()
    clocks.wait_first()
    t32, iters32, launches = timed(ml32, args.steps, args.warmup)
    clk = clocks.stop()
    rel32 = true_relres()
    xs32 = x.numpy()

    # per-level cycle profile and the dominant kernel
    prof = ml32.cycle_profile()
    cyc_prof_ms = float(prof.sum())
    cbytes, per_level = cycle_bytes(ml32, 4)
    # the preconditioner as PCG runs it: one graph replay of FP64 r -> FP32
    # b, the V-cycle, FP32 x -> FP64 z (conversion bytes 12 + 12 per row)
    cyc_ms = ml32.time_operator(0, 5, reps=20)
    cbytes_pc = cbytes + 24.0 * n
    # dominant kernel: the finest-level row kernel of the cycle (the
    # post-smoothing sweep; the residual is the same kernel with one vector less)
    op_ms = {}
    for op, name in ((0, "residual_A0_fp32"), (3, "jacobi_A0_fp32"), (4, "spmv_dot_A0_fp64"),
                     (1, "restrict_R0_fp32"), (2, "prolong_P0_fp32"),
                     (6, "first_sweep_residual_A0_fp32"), (7, "first_sweep_A0_fp32")):
        op_ms[name] = ml32.time_operator(0, op, reps=20)
    n0, z0, p0 = ml32.level_info(0)
    n1 = ml32.level_info(1)[0]
    BA0 = a_bytes(ml32, 0, 4)
    alg = {
        "residual_A0_fp32": BA0 + 3 * n0 * 4,
        "jacobi_A0_fp32": BA0 + 4 * n0 * 4,
        "spmv_dot_A0_fp64": BA0 + 2 * n0 * 8,
        "restrict_R0_fp32": p0 * 8 + (n1 + 1) * 4 + n0 * 4 + n1 * 4,
        "prolong_P0_fp32": p0 * 8 + (n0 + 1) * 4 + (2 * n0 + n1) * 4,
        "first_sweep_residual_A0_fp32": BA0 + 4 * n0 * 4,
        "first_sweep_A0_fp32": 3 * n0 * 4,
    }
    peak, peak_kind = peaks()
    # the dominant kernel: the longest of the level-0 operations an iteration
    # runs once each
    dom = max(("residual_A0_fp32", "jacobi_A0_fp32", "spmv_dot_A0_fp64", "restrict_R0_fp32",
               "prolong_P0_fp32"), key=lambda k: op_ms[k])
    achieved = alg[dom] / (op_ms[dom] * 1e-3) / 1e9
    a0_const = ml32.level_const_coef(0)

    # FP64 form
    fp64 = None
    xs64 = None
    if not args.no_fp64:
        ml64 = make(rb.FP64)
        t64, iters64, _ = timed(ml64, max(2, args.steps // 2), 2)
        rel64 = true_relres()
        xs64 = x.numpy()
        fp64 = {"seconds": t64, "iters": iters64[-1], "final_rel_res": rel64,
                "setup_s": ml64.setup_seconds,
                "speedup_fp32_over_fp64": t64 / t32,
                "x_rel_diff_fp32_vs_fp64": float(np.linalg.norm(xs32 - xs64) / np.linalg.norm(xs64))}
        ml = ml64
    else:
        ml = ml32

    # both forms again with level 0's stored values read (no constant-
    # coefficient mask): what a stencil with varying coefficients would cost
    stored = None
    if not args.no_fp64 and ml32.level_const_coef(0):
        stored = {}
        for name, prec in (("fp32_form", rb.FP32), ("fp64_form", rb.FP64)):
            mls = make(prec, const_coef=0)
            ts_, its_, _ = timed(mls, max(2, args.steps // 2), 2)
            stored[name] = {"seconds": ts_, "iters": its_[-1],
                            "cycle_ms": mls.time_operator(0, 5, reps=20)}
            del mls
        stored["speedup_fp32_over_fp64"] = (stored["fp64_form"]["seconds"] /
                                            stored["fp32_form"]["seconds"])

    # end to end through the public API with host buffers
    import ctypes as C
    try:
        import torch
        hb = torch.empty(n, dtype=torch.float64, pin_memory=True)
        hx = torch.empty(n, dtype=torch.float64, pin_memory=True)
        hb.numpy()[:] = bh
        hbp, hxp = hb.data_ptr(), hx.data_ptr()
        pinned = True
    except Exception:  # noqa: BLE001
        hbn = np.ascontiguousarray(bh)
        hxn = np.empty(n)
        hbp, hxp = hbn.ctypes.data, hxn.ctypes.data
        pinned = False
    L = rb.lib()
    Dp = C.POINTER(C.c_double)
    ml_e2e = ml32
    e2e_t = []
    for s in range(args.warmup + args.steps):
        L.rb_vec_upload.argtypes = [C.c_void_p, C.c_void_p]
        L.rb_vec_download.argtypes = [C.c_void_p, C.c_void_p]
        rb.lib().rb_synchronize()
        dist.barrier()
        e0 = ev()
        assert L.rb_vec_upload(b.h, C.c_void_p(hbp)) == 0
        x.set_const_value(0.0)
        res = []
        rb.PCG(A, ml_e2e, x, b, res, tol=TOL, max_iter=500, mode=rb.PCG_TRUE_RESIDUAL)
        assert L.rb_vec_download(x.h, C.c_void_p(hxp)) == 0
        e1 = ev()
        rb.lib().rb_synchronize()
        el = e0.elapsed_time(e1) * 1e-3
        if s >= args.warmup:
            e2e_t.append(dist.max(el))
    # restore numpy-typed signatures
    from raptor_b200 import _capi
    L.rb_vec_upload.argtypes = _capi.SIGNATURES["rb_vec_upload"][1]
    L.rb_vec_download.argtypes = _capi.SIGNATURES["rb_vec_download"][1]
    e2e = sum(e2e_t) / len(e2e_t)

    out = {
        "metric": METRIC, "value": t32, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t32 * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32-vcycle/fp64-outer",
        "data": "synthetic (27-point Laplacian stencil, b ~ U[-1,1] seed %d)" % SEED,
        "config": bench_config(S, n, nnz, None, world),
        "method": {"smoother": "L1-Jacobi, 1 pre- and 1 post-sweep",
                   "cycle": "V-cycle in FP32 (hierarchy values FP32, int32 indices)",
                   "outer": "PCG in FP64, stopping on the true relative residual",
                   "coarse": "FP64 LU of A_c^T (explicit inverse product)"},
        "iters": iters32[-1], "final_rel_res": rel32, "setup_s": setup32,
        "vcycle": {"ms": cyc_ms, "alg_bytes": cbytes_pc,
                   "gbs": cbytes_pc / (cyc_ms * 1e-3) / 1e9,
                   "frac_of_%s_peak" % peak_kind: cbytes_pc / (cyc_ms * 1e-3) / 1e9 / peak,
                   "timed": "graph replay of z = M r (FP32 cycle with its FP64 conversions)",
                   "profile_ms_per_level": [round(float(v), 5) for v in prof.sum(axis=1)],
                   "alg_bytes_per_level": per_level,
                   "first_sweep_fused": [ml32.level_fused_first(l)
                                         for l in range(ml32.num_levels - 1)],
                   "tail": dict(zip(("start_level", "ctas"), ml32.tail_info()),
                                cycle_ms_by_start=ml32.tail_timings()),
                   "levels": [ml32.level_info(l) for l in range(ml32.num_levels)],
                   "lanes": [ml32.level_lanes(l) for l in range(ml32.num_levels)]},
        "fp64_form": fp64,
        "stored_values_level0": stored,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic_for(dom + ({0: "", 1: "_const", 2: "_grid"}[a0_const]
                                                  if "_A0_" in dom else "")),
                     "peak_source": peak_kind, "ops_ms": op_ms, "alg_bytes": alg,
                     "a0_storage": ({0: "sliced-diagonals nd=%d",
                                     1: "constant-coefficient diagonals nd=%d (a 4-byte mask a "
                                        "row)",
                                     2: "constant-coefficient stencil nd=%d on a box (x staged "
                                        "in shared memory by planes, no mask)"}[a0_const]
                                    % ml32.level_storage(0))
                     if ml32.level_storage(0) else "csr"},
        "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": n * 8,
                "d2h_bytes_per_step": n * 8, "pinned": pinned},
        "gpu_launches": launches,
        "clocks": clk,
    }
    out["config"]["levels"] = ml.num_levels
    if args.batch_size > 0:
        out["batching"] = run_batching(rb, ev, lambda: rb.lib().rb_synchronize(),
                                       args.batch_size,
                                       ks=tuple(int(v) for v in args.batch_ks.split(",")))
    if args.systems > 0:
        out["uneven_batch"] = run_uneven_batch(rb, ev, lambda: rb.lib().rb_synchronize(),
                                               args.systems)
    if args.diff_size > 0:
        out["differentiation"] = run_differentiation(rb, ev, lambda: rb.lib().rb_synchronize(),
                                                     args.diff_size)
    if args.aniso_size > 0:
        out["aniso_precision"] = run_aniso_precision(rb, ev, lambda: rb.lib().rb_synchronize(),
                                                     args.aniso_size)
    if args.plain_size > 0:
        out["plain_fp64"] = run_plain_fp64(rb, ev, lambda: rb.lib().rb_synchronize(),
                                           args.plain_size)
    if args.bsr_cases:
        cases = [tuple(int(v) for v in c.split("x")) for c in args.bsr_cases.split(",")]
        try:
            out["block_csr"] = run_block_csr(rb, ev, lambda: rb.lib().rb_synchronize(), cases)
        except Exception as e:  # noqa: BLE001 - a side workload must not void the line
            out["block_csr"] = {"error": str(e)}
    if rank == 0 and args.cpu_sample > 0:
        out["cpu_baseline"], x_ref = cpu_baseline(ml32, bh, args.cpu_sample, S)
        if x_ref is not None:
            nref = float(np.linalg.norm(x_ref))
            fe = {"fp32_form": float(np.linalg.norm(xs32 - x_ref) / nref),
                  "reference": out["cpu_baseline"]["reference_solution"]["timed_solve_rel_error"],
                  "x_ref": "the reference's PCG on the same hierarchy and b, true relative "
                           "residual %.1e" % out["cpu_baseline"]["reference_solution"]["true_rel_res"]}
            if xs64 is not None:
                fe["fp64_form"] = float(np.linalg.norm(xs64 - x_ref) / nref)
            out["final_error_vs_fp64_reference"] = fe
    dist.close()
    if rank == 0:
        print(json.dumps(out))


def traffic_for(kernel):
    """DRAM bytes per launch from the committed ncu summary, when present."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get(kernel)
    except Exception:  # noqa: BLE001
        return None


# ------------------------------------------------------------- CPU legs ----
def host_cores():
    """Host cores this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class CpuSample:
    """The oracle's AMG-PCG with the same options on an m^3 grid, stopped on
    the same true relative residual (FP64); setup is not timed.  Its
    row-parallel loops (SpMV, residual, sweeps, axpy) run on every host
    core; dots and the restriction's transposed scatter stay sequential, as
    in the restatement, and the results are the same for any core count."""

    def __init__(self, m):
        from oracle import oracle as O
        self.O = O
        self.cores = host_cores()
        O.set_threads(self.cores)
        self.A = O.stencil_grid(O.laplace_stencil_27pt(), [m, m, m])
        self.n = self.A.shape[0]
        self.b = np.random.default_rng(SEED).uniform(-1.0, 1.0, self.n)
        self.ml = O.Hierarchy(self.A, interp="extended", relax="l1_jacobi")

    def solve(self):
        t0 = time.perf_counter()
        _, hist, _ = self.O.pcg(self.A, self.ml, np.zeros(self.n), self.b, tol=TOL, max_iter=500,
                                mode=1)
        return time.perf_counter() - t0, len(hist) - 1


class RefSolve:
    """The reference's PCG (raptor/krylov/par_cg.cpp:121-263) on a reference
    hierarchy, run to the same true relative residual as the GPU arm.  The
    reference stops when r.z < tol sqrt(b.Mb) (its history records r.z /
    b.Mb), not on ||b - A x|| / ||b||, so its tolerance is calibrated: a
    first solve to r.z / b.Mb <= 1e-18 gives the ratio c of the squared true
    relative residual to r.z / b.Mb at its end; the tolerance is then set for
    r.z / b.Mb <= 0.25 (1e-8)^2 / c, and divided by 10 until a solve's true
    relative residual (the reference's own residual routine) is <= 1e-8.
    These calibration solves are the warm-up; every timed solve then stops
    at the first iteration the calibrated test allows."""

    def __init__(self, O, A, ml, b):
        self.O, self.A, self.ml, self.b = O, A, ml, b
        self.bnorm = float(np.linalg.norm(b))
        z = ml.cycle(np.zeros(len(b)), b)
        self.sqrt_bMb = math.sqrt(max(float(np.dot(b, z)), 1e-300))
        self.tol = 1e-18 * self.sqrt_bMb
        self.iters = None
        self.relres = None
        self.last_rz = None

    def solve(self, tol=None, max_iter=500):
        t0 = time.perf_counter()
        x, hist = self.O.ref_pcg(self.A, self.ml, np.zeros(len(self.b)), self.b,
                                 tol=self.tol if tol is None else tol, max_iter=max_iter)
        el = time.perf_counter() - t0
        self.x = x
        self.iters = len(hist) - 1
        self.last_rz = float(hist[-1])
        self.relres = float(np.linalg.norm(self.A.residual(x, self.b)) / self.bnorm)
        return el

    def calibrate(self, max_tries=5):
        """Solves that set the tolerance; returns their count."""
        self.solve()
        if self.relres <= TOL and self.last_rz > 0:
            c = self.relres ** 2 / self.last_rz
            self.tol = 0.25 * TOL * TOL / c * self.sqrt_bMb
        for k in range(2, max_tries + 2):
            self.solve()
            if self.relres <= TOL:
                return k
            self.tol /= 10.0
        raise RuntimeError("reference PCG did not reach 1e-8 (relres %.3e)" % self.relres)


def cpu_baseline(ml, bh, m, S):
    """One reference PCG solve at the full size on the hierarchy the GPU
    built (exported level by level into the reference's ParMultilevel, whose
    duplicate_coarse factors A_c as its setup would), on one core; the CPU
    restatement on an m^3 sample, scaled by rows, where the reference build
    is absent.  Returns (entry, x_ref): x_ref is the reference's FP64
    solution of the same system taken much further (2.5 times the timed
    solve's iterations, true relative residual near 1e-15), against which
    the GPU solutions' final errors are stated (None without the build)."""
    from oracle import oracle as O
    L = O.par_ref()
    if L is None:
        el, it, n, cores = cpu_sample_solve(m)
        return {"value": el * (S ** 3) / n, "unit": "s", "cores": cores, "kind": "port",
                "sample": "CPU restatement's AMG-PCG solve on %d^3 (%d rows, %d iterations, "
                          "%.2f s on %d threads), scaled by rows to %d^3 (the reference "
                          "build is absent)" % (m, n, it, el, cores, S)}, None
    nl = ml.num_levels
    As = [ml.level_matrix(l, "A").arrays() for l in range(nl)]
    Ps = [(ml.level_info(l + 1)[0],) + tuple(ml.level_matrix(l, "P").arrays())
          for l in range(nl - 1)]
    hml = O.RefHierarchy.from_levels(L, As, Ps, **REF_KW)
    del As, Ps
    rs = RefSolve(O, hml.A(0), hml, bh)
    warm = rs.calibrate()
    el = rs.solve()
    entry = {"value": el, "unit": "s", "cores": 1, "kind": "reference",
             "sample": "one %d^3 solve: the reference's own PCG and V-cycle (compiled "
                       "unmodified, single-rank MPI stand-in, one core; SOR smoother) on the "
                       "GPU-built hierarchy of %d levels, %d iterations to true relative "
                       "residual %.2e (PCG tol %.1e after %d calibration solves)"
                       % (S, nl, rs.iters, rs.relres, rs.tol, warm)}
    x_timed, its, rel_timed = rs.x, rs.iters, rs.relres
    rs.solve(tol=1e-300, max_iter=int(2.5 * its) + 1)
    x_ref = rs.x
    entry["reference_solution"] = {
        "iters": rs.iters, "true_rel_res": rs.relres,
        "timed_solve_rel_error": float(np.linalg.norm(x_timed - x_ref) / np.linalg.norm(x_ref)),
        "timed_solve_rel_res": rel_timed}
    return entry, x_ref


def cpu_sample_solve(m):
    cs = CpuSample(m)
    el, it = cs.solve()
    return el, it, cs.n, cs.cores


def ref_line(args, world, value, steps, warmup, cfg, cpu, extra):
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": value * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp64", "data": "synthetic (27-point Laplacian, b ~ U[-1,1] seed %d)" % SEED,
        "config": cfg, "cpu_baseline": dict(cpu, value=value),
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    line.update(extra)
    return line


def run_reference(args, rank, world):
    """The reference's own setup (untimed) and PCG solve on the full problem,
    rank 0 only; the timed steps are capped so the run stays within a few
    minutes (the count timed is the line's "steps")."""
    if rank != 0:
        return
    from oracle import oracle as O
    S = args.size
    L = O.par_ref()
    bh = np.random.default_rng(SEED).uniform(-1.0, 1.0, S ** 3)
    budget_s = float(os.environ.get("RAPTOR_B200_REF_BUDGET_S", "120"))
    if L is None:
        # the CPU restatement of the same solve, on every host core
        cs = CpuSample(S)
        for _ in range(max(1, min(args.warmup, 1))):
            cs.solve()
        times = []
        while len(times) < args.steps and (not times or sum(times) + times[-1] <= budget_s):
            el, it = cs.solve()
            times.append(el)
        v = sum(times) / len(times)
        cfg = bench_config(S, cs.n, int(cs.A.shape[2]), cs.ml.num_levels, world)
        print(json.dumps(ref_line(args, world, v, len(times), 1, cfg, {
            "unit": "s", "cores": cs.cores, "kind": "port",
            "sample": "CPU restatement of the reference's AMG-PCG (its compiled build is "
                      "absent), %d^3, L1-Jacobi, %d iterations, %d of %d requested steps timed "
                      "on %d threads" % (S, it, len(times), args.steps, cs.cores)},
            {"method": {"smoother": "L1-Jacobi", "outer": "PCG in FP64 (true residual)"}})))
        return
    t0 = time.perf_counter()
    A = O.RefMatrix.laplace27(L, S, S, S)
    n, _, nnz = A.shape
    try:
        ml = O.RefHierarchy(A, **REF_KW)
        setup_note = "the reference's own ParRugeStubenSolver setup"
    except RuntimeError as e:
        # At one rank the reference's extended interpolation counts an upper
        # bound of P's nonzeros in an int (par_interpolation.cpp:531-569),
        # which overflows past about 2^31 / 570 rows of this stencil (so at
        # 192^3, not at 128^3) and makes the vector resize throw.  The
        # hierarchy then comes from the CPU restatement's setup, which is
        # identical to the reference's (A_l, P_l, states, entry order)
        # wherever the reference runs, and the reference's solve phase is
        # timed on it.
        Ao = O.stencil_grid(O.laplace_stencil_27pt(), [S, S, S])
        om = O.Hierarchy(Ao, relax="sor", interp="extended", interp_filter=0.3)
        As = [om.A(l).arrays() for l in range(om.num_levels)]
        Ps = [(om.A(l + 1).shape[0],) + tuple(om.P(l).arrays())
              for l in range(om.num_levels - 1)]
        del om, Ao
        ml = O.RefHierarchy.from_levels(L, As, Ps, **REF_KW)
        del As, Ps
        why = str(e).split("setup threw ")[-1]
        setup_note = ("the CPU restatement's setup (the reference's own ParRugeStubenSolver::"
                      "setup throws std::length_error (%s) at this size at one rank: its int "
                      "bound on P's nonzeros in extended interpolation overflows, "
                      "par_interpolation.cpp:531-569), handed level by level to the "
                      "reference's ParMultilevel" % why)
    setup_s = time.perf_counter() - t0
    rs = RefSolve(O, A, ml, bh)
    warm = rs.calibrate()
    times = []
    while len(times) < args.steps and (not times or sum(times) + times[-1] <= budget_s):
        times.append(rs.solve())
        if rs.relres > TOL:
            raise RuntimeError("reference solve missed 1e-8: %.3e" % rs.relres)
    v = sum(times) / len(times)
    cfg = bench_config(S, n, nnz, ml.num_levels, world)
    print(json.dumps(ref_line(args, world, v, len(times), warm, cfg, {
        "unit": "s", "cores": 1, "kind": "reference",
        "sample": "the reference's own PCG and V-cycle (compiled unmodified with a "
                  "single-rank MPI stand-in and OpenBLAS LU; one core, the reference has no "
                  "threads) on the full %d^3 problem, hierarchy from %s (%.1f s, untimed); SOR "
                  "smoother; %d iterations to true relative residual %.2e (PCG tol %.1e after "
                  "%d calibration solves); %d of the %d requested steps timed within %.0f s"
                  % (S, setup_note, setup_s, rs.iters, rs.relres, rs.tol, warm, len(times),
                     args.steps, budget_s)},
        {"setup_s": setup_s, "iters": rs.iters, "final_rel_res": rs.relres,
         "method": {"smoother": "SOR (the reference's default; its Jacobi is a no-op, it has "
                                "no L1-Jacobi), 1 pre- and 1 post-sweep",
                    "cycle": "V-cycle in FP64", "outer": "the reference's PCG in FP64",
                    "coarse": "dgetrf_/dgetrs_ (OpenBLAS) of A_c^T"}})))


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_b200(args, rank, world, local)


if __name__ == "__main__":
    main()
