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
    exe = build(tmp_path)
    r = subprocess.run([exe, "20"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    fields = r.stdout.split()
    relres = float(fields[fields.index("relres") + 1])
    # the reference's PCG stops on r.z < tol sqrt(b.Mb), not on ||r|| / ||b||
    assert relres < 1e-4
    last = float(fields[fields.index("last") + 1])
    assert last <= 1e-8
