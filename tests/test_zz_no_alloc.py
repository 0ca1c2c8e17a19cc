"""The allocation-free residual norm against the allocating entry points.

rb_residual_norm_noalloc exists for callers that cannot allocate device
memory while they run (under a fixed memory budget, in real-time loops).  Its
scratch is a static device array shared by
every call and left holding the last call's contents, so this test calls it
twice in a row and checks both results against rb_residual followed by
rb_vec_norm2 (which allocate), within the 1e-12 relative tolerance used for
solve-phase values, and that the library's device-allocation count
(rb_device_alloc_count, bumped by every cudaMalloc the library makes) does
not move across the two calls.  It sits in a file of its own that pytest collects last,
and passes alone in a fresh process as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

rb = pytest.importorskip("raptor_b200")


@pytest.fixture()
def caller_stream():
    """A stream the caller owns: the library's other entry points are ordered
    on it (rb_set_stream) and the allocation-free call is given it too."""
    torch = pytest.importorskip("torch")
    rb.init(0)
    s = torch.cuda.Stream(device=0)
    rb.check(rb.lib().rb_set_stream(C.c_void_p(s.cuda_stream)))
    yield C.c_void_p(s.cuda_stream)
    rb.check(rb.lib().rb_synchronize())
    rb.check(rb.lib().rb_set_stream(None))


def _dev_ptrs(A):
    rp, ci, cv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    rb.check(rb.lib().rb_csr_device_arrays(A.h, C.byref(rp), C.byref(ci), C.byref(cv)))
    return rp, ci, cv


@pytest.mark.parametrize("shape", [(40, 40, 40), (300, 300)])
def test_residual_norm_noalloc_matches_allocating_path(shape, caller_stream):
    st = rb.laplace_stencil_27pt() if len(shape) == 3 else rb.diffusion_stencil_2d(0.001, 0.3927)
    A = rb.par_stencil_grid(st, list(shape))
    n = A.global_num_rows
    rng = np.random.default_rng(11)
    x = rb.ParVector(n, values=rng.uniform(-1, 1, n))
    b = rb.ParVector(n, values=rng.uniform(-1, 1, n))
    r = rb.ParVector(n)
    A.residual(x, b, r)
    ref = r.norm(2)
    out = rb.ParVector(1)
    rp, ci, cv = _dev_ptrs(A)
    allocs_before = C.c_int64()
    rb.check(rb.lib().rb_device_alloc_count(C.byref(allocs_before)))
    for _ in range(2):   # two calls in a row share the static scratch
        out.set_const_value(-1.0)
        rc = rb.lib().rb_residual_norm_noalloc(n, rp, ci, cv, C.c_void_p(x.device_ptr()),
                                               C.c_void_p(b.device_ptr()),
                                               C.c_void_p(out.device_ptr()), caller_stream)
        assert rc == 0, rb.last_error()
        rb.lib().rb_synchronize()
        got = out.numpy()[0]
        assert abs(got - ref) <= 1e-12 * ref, (got, ref)
    allocs_after = C.c_int64()
    rb.check(rb.lib().rb_device_alloc_count(C.byref(allocs_after)))
    assert allocs_after.value == allocs_before.value


def test_residual_norm_noalloc_rejects_bad_arguments():
    rb.init(0)
    # every case is rejected on the host before any pointer is touched
    one = C.c_void_p(1)
    rc = rb.lib().rb_residual_norm_noalloc((1 << 24) + 1, one, one, one, one, one, one, None)
    assert rc == -1 and "2^24" in rb.last_error()
    rc = rb.lib().rb_residual_norm_noalloc(-1, one, one, one, one, one, one, None)
    assert rc == -1 and "< 0" in rb.last_error()
    for null_at in range(6):
        args = [one] * 6
        args[null_at] = None
        rc = rb.lib().rb_residual_norm_noalloc(10, *args, None)
        assert rc == -1 and "NULL" in rb.last_error(), null_at
