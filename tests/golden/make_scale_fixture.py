"""Generate tests/golden/lap27_192_hierarchy.json: the 192^3 bench problem's
AMG hierarchy and FP64 PCG history from the CPU restatement (oracle/), which
is pinned bit for bit on the reference's own parallel setup and solve
wherever the reference runs (tests/test_oracle_vs_reference_par.py; at
192^3 at one rank the reference's setup stops, its int bound on P's
nonzeros overflowing).

The fixture is small: per level the rows and nonzeros of A_l and P_l, CRC32
checksums of their CSR arrays (A_l in its diagonal-first entry order, P_l
with each row sorted by column) and of the C/F states, and the 13-entry
residual history of the L1-Jacobi PCG in true-residual mode (b uniform in
[-1, 1] from seed 20261203).  The GPU test compares the library's 192^3
hierarchy and FP64 solve with it.

Run once in the build container (about 2 minutes on 8 cores):
    python tests/golden/make_scale_fixture.py
"""
import json
import os
import sys
import time
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

SIDE = 192
SEED = 20261203
OUT = os.path.join(HERE, "lap27_%d_hierarchy.json" % SIDE)


def crc(*arrays):
    c = 0
    for a in arrays:
        c = zlib.crc32(np.ascontiguousarray(a).tobytes(), c)
    return c


def sorted_rows(rp, ci, cv):
    """Each row's entries sorted by column (a stable lexicographic sort)."""
    n = len(rp) - 1
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp))
    o = np.lexsort((ci, rows))
    return rp, ci[o], cv[o]


def main():
    O.set_threads(os.cpu_count() or 1)
    t0 = time.time()
    A = O.stencil_grid(O.laplace_stencil_27pt(), [SIDE, SIDE, SIDE])
    ml = O.Hierarchy(A, interp="extended", interp_filter=0.3, relax="l1_jacobi")
    print("setup %.1f s, %d levels" % (time.time() - t0, ml.num_levels), flush=True)
    w = O.rand_weights(A.shape[0])
    levels = []
    for l in range(ml.num_levels):
        Al = ml.A(l)
        rp, ci, cv = Al.arrays()
        lev = {"rows": int(Al.shape[0]), "nnz_A": int(Al.shape[2]), "crc_A": crc(rp, ci, cv)}
        if l < ml.num_levels - 1:
            P = ml.P(l)
            prp, pci, pcv = sorted_rows(*P.arrays())
            lev.update({"nnz_P": int(P.shape[2]), "cols_P": int(P.shape[1]),
                        "crc_P_sorted": crc(prp, pci, pcv)})
            st = O.split_pmis(O.classical_strength(Al, 0.25), w[: Al.shape[0]])
            lev["crc_states"] = crc(st.astype(np.int32))
        levels.append(lev)
        print("level", l, lev, flush=True)
    n = A.shape[0]
    b = np.random.default_rng(SEED).uniform(-1.0, 1.0, n)
    t0 = time.time()
    x, hist, _ = O.pcg(A, ml, np.zeros(n), b, tol=1e-8, max_iter=500, mode=1)
    print("pcg %.1f s, %d iterations" % (time.time() - t0, len(hist) - 1), flush=True)
    out = {
        "problem": "laplace_stencil_27pt on %d^3 (par_stencil_grid); RS: classical strength "
                   "0.25, PMIS (glibc weights, seed 2448422), extended+i interpolation, "
                   "filter 0.3" % SIDE,
        "made_by": "tests/golden/make_scale_fixture.py from the CPU restatement (oracle/)",
        "levels": levels,
        "pcg": {"solver": "PCG in true-residual mode, L1-Jacobi (w = 1), FP64, tol 1e-8",
                "b": "uniform [-1, 1], numpy default_rng(%d)" % SEED,
                "history": [float(v) for v in hist]},
    }
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
