"""GPU tests of the constant-coefficient forms of diagonal storage.

A stencil_grid operator has one value per diagonal; the cycle's diagonal
kernels then read a 4-byte mask a row (which stencil entries the row has)
instead of the row's values, or, on a box whose rows hold exactly their
in-box neighbours, no mask at all: x is staged in shared memory plane by
plane with a zero halo (the box-grid form).  Every row's products, and their
order, are those of the stored values, so one V-cycle must give the same
result bit for bit in all three forms (RAPTOR_B200_CONST_DIA=0: stored
values; RAPTOR_B200_GRID_DIA=0: the mask; RAPTOR_B200_GRID_DIA=1 or 2: the
box grid with one or two rows in x a thread).  The outer A p of PCG sums its p.Ap over rows in another grouping in
each form, so a whole solve agrees to rounding: iterations within one,
residual histories within 1e-9 relative (1e-13 absolute: the histories are
relative to the first residual, and the dots' rounding reaches about 1e-14
of it) on the well-conditioned 27- and 7-point problems and within 1e-6 on
the rotated anisotropic one, where CG's round-off grows over its 54
iterations.  The runs are child processes sharing one autotuner cache, so
that they also make the same schedule choices.  Box sizes that are not
multiples of the kernel's tiles (32 x 8 in 3D, 256 in 2D) or of its planes
per block are included.  On a box that is not a cube the reference's
stencil_grid (which the gallery reproduces) leaves some rows without in-box
neighbours along the fastest axis, so those operators are not box stencils:
the row-by-row check at setup must keep them in the mask form, with the same
results.  An operator whose diagonals hold different values must keep the
stored values.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

rb = pytest.importorskip("raptor_b200")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys
import numpy as np
import raptor_b200 as rb
m, prec, stencil, out = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3], sys.argv[4]
rb.init(0)
if stencil == "lap27":
    A = rb.par_stencil_grid(rb.laplace_stencil_27pt(), [m, m, m])
elif stencil.startswith("aniso7"):
    st = [0.0] * 27
    st[13] = 4.02
    st[12] = st[14] = st[10] = st[16] = -1.0
    st[4] = st[22] = -0.01
    A = rb.par_stencil_grid(st, [m, m + 3, m + 5] if stencil == "aniso7_uneven" else [m, m, m])
else:
    A = rb.par_stencil_grid(rb.diffusion_stencil_2d(0.001, np.pi / 8), [m, m])
n = A.global_num_rows
b = rb.ParVector(n, values=np.random.default_rng(7).uniform(-1.0, 1.0, n))
ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
ml.precision = prec
ml.setup(A)
z = rb.ParVector(n)
ml.cycle(z, b)
x = rb.ParVector(n)
res = []
rc = rb.PCG(A, ml, x, b, res, tol=1e-8, max_iter=300, mode=rb.PCG_TRUE_RESIDUAL)
np.savez(out, rc=rc, res=np.array(res), x=x.numpy(), z=z.numpy(), const=ml.level_const_coef(0),
         nd=ml.level_storage(0))
"""


FORMS = {"stored": ("0", "0"), "masked": ("1", "0"), "grid": ("1", "1"), "grid2": ("1", "2")}


def run_child(tmp_path, tag, m, prec, stencil):
    env = dict(os.environ)
    env["RAPTOR_B200_CONST_DIA"], env["RAPTOR_B200_GRID_DIA"] = FORMS[tag]
    env["RAPTOR_B200_TUNE_CACHE"] = str(tmp_path / "tune.json")
    out = str(tmp_path / (tag + ".npz"))
    subprocess.run([sys.executable, "-c", CHILD, str(m), str(prec), stencil, out], cwd=ROOT,
                   env=env, check=True, timeout=600)
    return np.load(out)


@pytest.mark.parametrize("stencil,m,prec", [
    ("lap27", 48, 0), ("lap27", 48, 1), ("lap27", 45, 1), ("aniso7", 37, 1),
    ("aniso7_uneven", 37, 1), ("aniso2d", 512, 0), ("aniso2d", 512, 1), ("aniso2d", 500, 1)])
def test_constant_coefficients_bit_identical(tmp_path, stencil, m, prec):
    off = run_child(tmp_path, "stored", m, prec, stencil)
    assert int(off["nd"]) > 0 and int(off["const"]) == 0 and int(off["rc"]) == 0
    rtol = 1e-6 if stencil == "aniso2d" else 1e-9
    grid_code = 1 if stencil == "aniso7_uneven" else 2
    for form, code in (("masked", 1), ("grid", grid_code), ("grid2", grid_code)):
        on = run_child(tmp_path, form, m, prec, stencil)
        assert int(on["nd"]) == int(off["nd"])
        assert int(on["const"]) == code, form
        assert int(on["rc"]) == 0
        assert np.array_equal(off["z"], on["z"]), form
        k = min(len(off["res"]), len(on["res"]))
        assert abs(len(off["res"]) - len(on["res"])) <= 1
        np.testing.assert_allclose(on["res"][:k], off["res"][:k], rtol=rtol, atol=1e-13,
                                   err_msg=form)
        assert np.linalg.norm(on["x"] - off["x"]) <= rtol * np.linalg.norm(off["x"])


def test_variable_coefficients_keep_values():
    rb.init(0)
    m = 40
    A = rb.par_stencil_grid(rb.laplace_stencil_27pt(), [m, m, m])
    rp, ci, cv = A.arrays()
    n = m ** 3
    # scale each row's off-diagonal entries: still symmetric positive
    # definite after a symmetric scaling D A D, but no diagonal is constant
    d = np.random.default_rng(3).uniform(0.5, 1.5, n)
    rows = np.repeat(np.arange(n), np.diff(rp))
    cv2 = cv * d[rows] * d[ci]
    B = rb.ParCSRMatrix.from_arrays(n, n, rp, ci, cv2)
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
    ml.precision = rb.FP32
    ml.setup(B)
    assert not ml.level_const_coef(0)
    x = rb.ParVector(n)
    res = []
    bv = rb.ParVector(n, values=np.random.default_rng(8).uniform(-1, 1, n))
    assert rb.PCG(B, ml, x, bv, res, tol=1e-8, max_iter=300, mode=rb.PCG_TRUE_RESIDUAL) == 0
