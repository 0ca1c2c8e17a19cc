"""Build libraptor_b200.so in-tree for sm_100a (nvcc cross-compiles; no GPU needed).

    python -m raptor_b200.build [--force]

Every ``csrc/*.cu`` file is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; the setup kernels
(``setup.cu``, ``aggregation.cu``) and the block CSR products (``bsr.cu``) add
``-fmad=false`` so FP64 products and sums round separately
as in the reference's x86-64 build.  Objects go to ``raptor_b200/_build`` and
the library to ``raptor_b200/libraptor_b200.so`` (git-ignored, shipped with the
working tree).
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libraptor_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
                 "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
                 "-I", CSRC, "-I", INCLUDE]
PER_FILE = {"setup.cu": ["-fmad=false"], "aggregation.cu": ["-fmad=false"],
            "bsr.cu": ["-fmad=false"]}


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, jobs=None):
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    cc = nvcc()
    todo = []
    objs = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s, __file__] + headers):
            cmd = [cc] + COMMON + PER_FILE.get(os.path.basename(s), []) + ["-c", s, "-o", o]
            todo.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("compile failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
        return r.stderr

    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for err in ex.map(run, todo):
            if err and verbose:
                print(err)
    if todo or force or not os.path.exists(LIB):
        cmd = [cc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-ldl", "-lrt", "-lpthread"]
        run(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
