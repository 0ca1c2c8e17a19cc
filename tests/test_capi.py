"""C-ABI checks that need no GPU: the library loads, exports every symbol the
public header declares, and compute calls fail loudly (never fall back)."""
import ctypes
import os
import re

import numpy as np
import pytest

from tests.conftest import ROOT

HEADER = os.path.join(ROOT, "include", "raptor_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rb_[A-Za-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from raptor_b200 import _capi
    lib = _capi.lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    # and the Python binding covers the header
    assert set(declared_symbols()) <= set(_capi.exported_symbols())


def test_library_targets_sm100a_only():
    # the fat binary holds sm_100a code; cuobjdump-free check: the build flags
    from raptor_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def test_version_and_errors_without_device():
    import raptor_b200 as rb
    assert "sm_100a" in rb.version()
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(rb.RaptorError) as ei:
        rb.ParVector(10)
    assert ei.value.code == -6  # RB_ERR_NO_DEVICE: no CPU fallback


def test_default_opts_mirror_reference_defaults():
    import raptor_b200 as rb
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.SOR)
    # multilevel/par_multilevel.hpp:87-99 and par_ruge_stuben_solver.hpp:24
    assert ml.num_smooth_sweeps == 1
    assert ml.relax_weight == 1.0
    assert ml.max_coarse == 50
    assert ml.max_levels == 25
    assert ml.max_iterations == 100
    assert abs(ml.solve_tol - 1e-7) < 1e-20
    assert abs(ml.interp_filter - 0.3) < 1e-15
    assert ml.interp_type == rb.Extended


def test_unknown_coarsening_is_rejected():
    import raptor_b200 as rb
    with pytest.raises(rb.RaptorError):
        rb.ParRugeStubenSolver(0.25, 7, rb.ModClassical)
    ml = rb.ParRugeStubenSolver(0.25, rb.CLJP, rb.ModClassical)
    assert ml.coarsen_type == rb.CLJP
    # the reference's default coarsening is Ruge-Stuben
    assert rb.ParRugeStubenSolver().coarsen_type == rb.RS


@pytest.mark.parametrize("field,value,message", [
    ("interp_type", 3, "interpolation must be"),
    ("strength_type", 5, "strength"),
    ("relax_type", 9, "relaxation"),
    ("precision", 2, "precision"),
    ("coarsen_type", 9, "coarsening"),
    ("max_levels", 0, "max_levels"),
    ("solver", 7, "solver"),
])
def test_amg_options_are_checked_before_the_matrix(field, value, message):
    # every option is validated before the matrix handle is touched, so the
    # checks run without a device; an unknown option is an error, never a
    # silent substitute
    import raptor_b200 as rb
    L = rb.lib()
    opts = rb.AmgOpts()
    L.rb_amg_default_opts(ctypes.byref(opts))
    setattr(opts, field, value)
    h = ctypes.c_void_p()
    assert L.rb_amg_setup(None, ctypes.byref(opts), None, ctypes.byref(h)) == -1
    assert message in rb.last_error()
    # valid options: the missing matrix is what is reported
    L.rb_amg_default_opts(ctypes.byref(opts))
    assert L.rb_amg_setup(None, ctypes.byref(opts), None, ctypes.byref(h)) == -1
    assert "A is NULL" in rb.last_error()
