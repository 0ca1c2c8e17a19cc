"""The header-only C++ shim (include/raptor_b200.hpp) compiles against the
library with the reference's call sequence, and fails loudly without a GPU
(no CPU fallback); with a GPU the same program solves."""
import os
import shutil
import subprocess

import pytest

from tests.conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cxx", "shim_pcg.cpp")
LIBDIR = os.path.join(ROOT, "raptor_b200")


def build(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    exe = str(tmp_path / "shim_pcg")
    cmd = [gxx, "-std=c++17", "-O1", "-Wall", "-Werror", SRC, "-I", os.path.join(ROOT, "include"),
           "-L", LIBDIR, "-lraptor_b200", "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_shim_compiles_and_reports_missing_device(tmp_path):
    exe = build(tmp_path)
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    r = subprocess.run([exe, "8"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 3, r.stdout + r.stderr   # RB_ERR_NO_DEVICE, thrown as raptor_b200::error
    assert "error -6" in r.stdout


@pytest.mark.gpu
def test_shim_solves_on_the_gpu(tmp_path):
    """The compiled caller's PCG and stationary-solve histories equal those
    of the same calls through the Python mirror (one library, two front
    ends).  The two processes may pick different lane counts for a row
    kernel (the autotuner times them), which reorders a row's sums, so the
    histories agree to 1e-10 relative above a floor of 1e-15 of the first
    entry rather than bit for bit."""
    exe = build(tmp_path)
    r = subprocess.run([exe, "20"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = {ln.split()[0]: ln.split()[1:] for ln in r.stdout.splitlines() if ln.strip()}
    pcg_cxx = [float(v) for v in lines["pcg"]]
    solve_cxx = [float(v) for v in lines["solve"]]

    import numpy as np
    import raptor_b200 as rb
    rb.init(0)
    A = rb.par_stencil_grid(rb.laplace_stencil_27pt(), [20, 20, 20])
    n = A.global_num_rows
    ones = rb.ParVector(n)
    ones.set_const_value(1.0)
    b = rb.ParVector(n)
    A.mult(ones, b)
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
    ml.max_iterations = 200
    ml.solve_tol = 1e-8
    ml.setup(A)
    x = rb.ParVector(n)
    res = []
    rb.PCG(A, ml, x, b, res, 1e-8)
    np.testing.assert_allclose(pcg_cxx, res, rtol=1e-10, atol=1e-15 * res[0])
    x.set_const_value(0.0)
    ml.solve(x, b)
    np.testing.assert_allclose(solve_cxx, ml.get_residuals(), rtol=1e-10,
                               atol=1e-15 * ml.get_residuals()[0])
    assert solve_cxx[-1] <= 1e-8
