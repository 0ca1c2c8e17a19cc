"""Build recipe for the test oracle (TEST INFRASTRUCTURE ONLY).

Compiles ``oracle/raptor_oracle.c`` into ``oracle/_build/libraptor_oracle.so``
with ``-ffp-contract=off`` so that every multiply and add rounds separately,
as in the reference's ``-O3`` x86-64 build (no FMA).

When the reference checkout is present (only in the build container, never on
the GPU box) it also compiles the reference's own *sequential* sources, which
build from their own files with no MPI and no LAPACK, together with the shim
``oracle/ref_shim.cpp`` into ``oracle/_ref/libraptor_seq_ref.so``.  The
reference's parallel path (``ParMultilevel``, ``PCG``) needs MPI, an external
library absent here, so it is not built.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(BUILD, "libraptor_oracle.so")
REF_SO = os.path.join(REF_OUT, "libraptor_seq_ref.so")
REFERENCE_ROOT = os.environ.get("RAPTOR_REFERENCE_ROOT", "/root/reference")

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


if __name__ == "__main__":
    build_oracle(force="--force" in sys.argv)
    build_reference(force="--force" in sys.argv)
