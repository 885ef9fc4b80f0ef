"""The allocation-free inner product (dg_vec_dot_noalloc) through the C ABI.

Some callers of this library cannot allocate device memory -- for example a
per-iteration convergence check inside a solver whose device memory is
owned by another allocator, or a loop that must not take the device-wide
synchronisation of cudaMalloc/cudaFree.  dg_vec_dot_noalloc serves them from
a fixed array in the library's device memory.  This test compares it with
dg_vec_dot (which allocates its partial sums) on two calls in a row, the
second one shorter so that leftover partial sums of the first would show,
and checks the size limit.  The file sorts last so that a run stopping at
the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative to sum |x_i y_i|, as the other FP64 dot tests
MAX_N = 268_435_456


def _dot(fn, x, y, stream_ptr=None):
    import torch
    out = torch.full((1,), float("nan"), dtype=torch.float64, device=x.device)
    st = fn(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), x.numel(), C.c_void_p(out.data_ptr()), stream_ptr)
    torch.cuda.synchronize()
    return st, float(out.item())


def test_noalloc_dot_matches_allocating_dot(gpu):
    import torch
    from dendro_b200._lib import lib
    L = lib()
    rng = np.random.default_rng(2024)
    for n in (3_000_001, 10_007):  # two calls in a row, the second much shorter
        xh, yh = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
        x, y = torch.tensor(xh, device="cuda"), torch.tensor(yh, device="cuda")
        st_ref, ref = _dot(L.dg_vec_dot, x, y)
        st, got = _dot(L.dg_vec_dot_noalloc, x, y)
        assert st_ref == 0 and st == 0
        scale = float(np.abs(xh) @ np.abs(yh))
        assert abs(got - ref) <= TOL * scale, (n, got, ref)
        assert abs(got - float(xh @ yh)) <= TOL * scale


def test_noalloc_dot_on_a_stream_and_empty_input(gpu):
    import torch
    from dendro_b200._lib import lib
    L = lib()
    s = torch.cuda.Stream()
    x = torch.arange(5000, dtype=torch.float64, device="cuda")
    with torch.cuda.stream(s):
        st, got = _dot(L.dg_vec_dot_noalloc, x, x, C.c_void_p(s.cuda_stream))
    assert st == 0 and got == float((np.arange(5000.0) ** 2).sum())
    e = torch.empty(0, dtype=torch.float64, device="cuda")
    st, got = _dot(L.dg_vec_dot_noalloc, e, e)
    assert st == 0 and got == 0.0


def test_noalloc_dot_rejects_sizes_beyond_the_limit(gpu):
    import torch
    from dendro_b200._lib import lib
    L = lib()
    x = torch.zeros(1, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = L.dg_vec_dot_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), MAX_N + 1,
                              C.c_void_p(out.data_ptr()), None)
    assert st == 1  # DG_EINVAL, before any device work
    buf = C.create_string_buffer(512)
    L.dg_last_error(buf, 512)
    assert b"268435456" in buf.value
