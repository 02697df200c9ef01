"""nb_glsc3_noalloc: the inner product for callers that cannot allocate
device memory (its scratch is a static device array).  Checked through the
C ABI against cuda_glsc3 on two calls in a row.  Kept in a file that pytest
collects last, so a stop at the first failure has already run every other
test; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_glsc3_noalloc_matches_glsc3(nblib):
    import torch
    rng = np.random.default_rng(77)
    vp = ctypes.c_void_p
    stream = vp(torch.cuda.current_stream().cuda_stream)
    # two calls in a row, different sizes and data: the shared scratch keeps
    # the previous call's contents and must not leak into the next result
    for n in (3000017, 262144):
        a, b, c = (torch.as_tensor(rng.standard_normal(n), device="cuda") for _ in range(3))
        nn = ctypes.c_int(n)
        ref = nblib.cuda_glsc3(vp(a.data_ptr()), vp(b.data_ptr()), vp(c.data_ptr()),
                               ctypes.byref(nn), stream)
        out = ctypes.c_double(np.nan)
        st = nblib.nb_glsc3_noalloc(vp(a.data_ptr()), vp(b.data_ptr()), vp(c.data_ptr()), n,
                                    ctypes.byref(out), stream)
        assert st == 0, nblib.nb_last_error()
        scale = float((a * b * c).abs().sum())
        assert abs(out.value - ref) <= 1e-13 * scale, (n, out.value, ref)


def test_glsc3_noalloc_rejects_oversize(nblib):
    out = ctypes.c_double(0.0)
    vp = ctypes.c_void_p
    st = nblib.nb_glsc3_noalloc(vp(16), vp(16), vp(16), 33554433, ctypes.byref(out), vp(0))
    assert st == 1
    assert b"33554432" in nblib.nb_last_error()
