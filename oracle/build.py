"""Build recipe for the test oracle (TEST INFRASTRUCTURE ONLY).

Compiles ``oracle/raptor_oracle.c`` into ``oracle/_build/libraptor_oracle.so``
with ``-ffp-contract=off`` so that every multiply and add rounds separately,
as in the reference's ``-O3`` x86-64 build (no FMA).

When the reference checkout is present (only in the build container, never on
the GPU box; ``RAPTOR_REFERENCE_ROOT`` names it, default the container's
read-only checkout) it also compiles, from the reference's unmodified sources:

* its *sequential* routines, which build with no MPI and no LAPACK, with the
  shim ``oracle/ref_shim.cpp`` into ``oracle/_ref/libraptor_seq_ref.so``;
* its *parallel* solve path (ParCSRMatrix, ParRugeStubenSolver,
  ParSmoothedAggregationSolver, ParMultilevel, PCG, CG, BiCGStab and every
  source they call) with the shim ``oracle/ref_par_shim.cpp`` into
  ``oracle/_ref/libraptor_par_ref.so``.  MPI is absent on both machines, so
  ``oracle/mpi_stub/`` (a single-rank stand-in written for this project)
  provides ``<mpi.h>``; LAPACK's ``dgetrf_``/``dgetrs_`` come from the
  OpenBLAS 0.3.15 shipped inside the Python environment (opencv's wheel);
* the same parallel path with the one-statement Jacobi fix into
  ``oracle/_ref/libraptor_par_ref_jfix.so``: the reference's
  ``jacobi_helper`` sets ``diag = 0`` and never reads the diagonal, so its
  Jacobi sweep leaves x unchanged (``raptor/util/linalg/par_relax.cpp:127``);
  the fixed copy reads the row's leading (diagonal) entry there instead.  The
  patched file is written under ``oracle/_ref/`` at build time; nothing of
  the reference is kept in the repository.

Flags follow the reference's build (``-O3 -std=c++11``, no ``-march``, hence
no FMA contraction on x86-64).  All outputs are git-ignored build artefacts
that travel with the working tree.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(BUILD, "libraptor_oracle.so")
REF_SO = os.path.join(REF_OUT, "libraptor_seq_ref.so")
PAR_OUT = os.path.join(REF_OUT, "par")
PAR_SO = os.path.join(REF_OUT, "libraptor_par_ref.so")
PAR_JFIX_SO = os.path.join(REF_OUT, "libraptor_par_ref_jfix.so")
MPI_STUB = os.path.join(HERE, "mpi_stub")
REFERENCE_ROOT = os.environ.get("RAPTOR_REFERENCE_ROOT", "/root/reference")
# dgetrf_/dgetrs_ for the reference's coarse solve
OPENBLAS_DIR = os.environ.get(
    "RAPTOR_OPENBLAS_DIR",
    os.path.join(sys.prefix, "lib", "python%d.%d" % sys.version_info[:2], "site-packages",
                 "opencv_python_headless.libs"))

# The reference's sequential sources for the AMG path (paths inside the
# reference project).  They compile as-is with g++ -O3 -std=c++11.
REF_SOURCES = [
    "raptor/core/matrix.cpp",
    "raptor/core/vector.cpp",
    "raptor/util/linalg/spmv.cpp",
    "raptor/util/linalg/matmult.cpp",
    "raptor/util/linalg/add.cpp",
    "raptor/strength.cpp",
    "raptor/ruge_stuben/cf_splitting.cpp",
    "raptor/ruge_stuben/interpolation.cpp",
    "raptor/aggregation/mis.cpp",
    "raptor/aggregation/aggregate.cpp",
    "raptor/aggregation/candidates.cpp",
    "raptor/aggregation/prolongation.cpp",
]


# The reference's sources on its parallel solve path, and the sequential
# kernels they call (paths inside the reference project).
PAR_SOURCES = [
    "raptor/core/vector.cpp", "raptor/core/matrix.cpp", "raptor/core/mpi_types.cpp",
    "raptor/core/comm_data.cpp", "raptor/core/tap_comm.cpp", "raptor/core/comm_pkg.cpp",
    "raptor/core/comm_mat.cpp", "raptor/core/par_vector.cpp", "raptor/core/par_matrix.cpp",
    "raptor/util/linalg/spmv.cpp", "raptor/util/linalg/matmult.cpp", "raptor/util/linalg/add.cpp",
    "raptor/util/linalg/relax.cpp", "raptor/util/linalg/par_spmv.cpp",
    "raptor/util/linalg/par_matmult.cpp", "raptor/util/linalg/par_add.cpp",
    "raptor/util/linalg/par_relax.cpp", "raptor/util/linalg/repartition.cpp",
    "raptor/strength.cpp", "raptor/par_strength.cpp",
    "raptor/ruge_stuben/cf_splitting.cpp", "raptor/ruge_stuben/interpolation.cpp",
    "raptor/ruge_stuben/par_cf_splitting.cpp", "raptor/ruge_stuben/par_interpolation.cpp",
    "raptor/aggregation/mis.cpp", "raptor/aggregation/aggregate.cpp",
    "raptor/aggregation/candidates.cpp", "raptor/aggregation/prolongation.cpp",
    "raptor/aggregation/par_mis.cpp", "raptor/aggregation/par_aggregate.cpp",
    "raptor/aggregation/par_candidates.cpp", "raptor/aggregation/par_prolongation.cpp",
    "raptor/krylov/cg.cpp", "raptor/krylov/bicgstab.cpp", "raptor/krylov/par_cg.cpp",
    "raptor/krylov/par_bicgstab.cpp", "raptor/krylov/partial_inner.cpp",
    "raptor/profiling/profile_comm.cpp",
]
JACOBI_FILE = "raptor/util/linalg/par_relax.cpp"
# The one statement the Jacobi fix replaces (jacobi_helper's diagonal).
JACOBI_BROKEN = "            diag = 0;\n"
JACOBI_FIXED = "            diag = A->on_proc->vals[A->on_proc->idx1[i]];\n"


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_oracle(force=False):
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "raptor_oracle.c")
    hdr = os.path.join(HERE, "raptor_oracle.h")
    if force or _stale(ORACLE_SO, [src, hdr, __file__]):
        _run(["gcc", "-O2", "-std=c99", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
              "-fopenmp", "-shared", "-o", ORACLE_SO, src, "-lm"])
    return ORACLE_SO


def build_reference(force=False):
    """Compile the reference's sequential sources (only where they exist)."""
    if not os.path.isdir(os.path.join(REFERENCE_ROOT, "raptor")):
        return REF_SO if os.path.exists(REF_SO) else None
    os.makedirs(REF_OUT, exist_ok=True)
    srcs = [os.path.join(REFERENCE_ROOT, s) for s in REF_SOURCES]
    shim = os.path.join(HERE, "ref_shim.cpp")
    if force or _stale(REF_SO, srcs + [shim, __file__]):
        objs = []
        for s in srcs:
            o = os.path.join(REF_OUT, os.path.basename(s).replace(".cpp", ".o"))
            _run(["g++", "-O3", "-std=c++11", "-fPIC", "-w", "-I",
                  os.path.join(REFERENCE_ROOT, "raptor"), "-c", s, "-o", o])
            objs.append(o)
        so = os.path.join(REF_OUT, "ref_shim.o")
        _run(["g++", "-O3", "-std=c++11", "-fPIC", "-w", "-I",
              os.path.join(REFERENCE_ROOT, "raptor"), "-c", shim, "-o", so])
        _run(["g++", "-shared", "-o", REF_SO] + objs + [so])
    return REF_SO


def _openblas():
    libs = sorted(glob.glob(os.path.join(OPENBLAS_DIR, "libopenblas*.so*")))
    if not libs:
        raise RuntimeError("no OpenBLAS (dgetrf_/dgetrs_) under %s" % OPENBLAS_DIR)
    return libs[0]


def build_reference_parallel(force=False, jobs=None):
    """Compile the reference's parallel solve path (only where its sources exist).

    Returns (plain library, Jacobi-fixed library), or the already built pair
    (or None) where the checkout is absent.
    """
    if not os.path.isdir(os.path.join(REFERENCE_ROOT, "raptor")):
        if os.path.exists(PAR_SO) and os.path.exists(PAR_JFIX_SO):
            return PAR_SO, PAR_JFIX_SO
        return None
    os.makedirs(PAR_OUT, exist_ok=True)
    inc = ["-I", os.path.join(REFERENCE_ROOT, "raptor"), "-I", MPI_STUB]
    flags = ["g++", "-O3", "-std=c++11", "-fPIC", "-w"] + inc
    stub_src = os.path.join(MPI_STUB, "mpi_stub.cpp")
    shim_src = os.path.join(HERE, "ref_par_shim.cpp")
    deps = [os.path.join(MPI_STUB, "mpi.h"), __file__]

    # the Jacobi-fixed copy of par_relax.cpp, written under oracle/_ref only
    with open(os.path.join(REFERENCE_ROOT, JACOBI_FILE)) as f:
        text = f.read()
    if text.count(JACOBI_BROKEN) != 1:
        raise RuntimeError("the Jacobi statement to fix is not unique in %s" % JACOBI_FILE)
    fixed_src = os.path.join(PAR_OUT, "par_relax_jacobi_fixed.cpp")
    fixed_text = text.replace(JACOBI_BROKEN, JACOBI_FIXED)
    if not os.path.exists(fixed_src) or open(fixed_src).read() != fixed_text:
        with open(fixed_src, "w") as f:
            f.write(fixed_text)

    units = []  # (source, object)
    for rel in PAR_SOURCES:
        units.append((os.path.join(REFERENCE_ROOT, rel),
                      os.path.join(PAR_OUT, rel.replace("raptor/", "").replace("/", "_")[:-4] + ".o")))
    units.append((stub_src, os.path.join(PAR_OUT, "mpi_stub.o")))
    units.append((shim_src, os.path.join(PAR_OUT, "ref_par_shim.o")))
    units.append((fixed_src, os.path.join(PAR_OUT, "par_relax_jacobi_fixed.o")))
    todo = [(s, o) for s, o in units if force or _stale(o, [s] + deps)]

    def compile_one(so):
        s, o = so
        cmd = flags + ["-c", s, "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("compile failed: %s\n%s" % (" ".join(cmd), r.stderr[-4000:]))
        return o

    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        list(ex.map(compile_one, todo))

    blas = _openblas()
    blas_dir = os.path.dirname(blas)
    # DT_RPATH (not RUNPATH) so that OpenBLAS's own libgfortran resolves too
    link_tail = ["-L", blas_dir, "-l:" + os.path.basename(blas),
                 "-Wl,--disable-new-dtags,-rpath," + blas_dir, "-Wl,--no-undefined"]
    relax_src = os.path.join(REFERENCE_ROOT, JACOBI_FILE)
    fixed_obj = dict(units)[fixed_src]
    plain = [o for s, o in units if s != fixed_src]
    fixed = [fixed_obj if s == relax_src else o for s, o in units if s != fixed_src]
    for target, objs in ((PAR_SO, plain), (PAR_JFIX_SO, fixed)):
        if todo or force or _stale(target, objs):
            _run(["g++", "-shared", "-o", target] + objs + link_tail)
    return PAR_SO, PAR_JFIX_SO


if __name__ == "__main__":
    build_oracle(force="--force" in sys.argv)
    build_reference(force="--force" in sys.argv)
    build_reference_parallel(force="--force" in sys.argv)
