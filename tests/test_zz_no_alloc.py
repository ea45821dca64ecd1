"""aq_state_error_noalloc, the variant of aq_state_error that allocates no
device memory (for callers whose host owns the device heap or that must
not enter the allocator), against aq_state_error itself through the C ABI.

Kept in a file that pytest collects last.  Two calls in a row with
different inputs check that the shared scratch array is cleared between
calls; the results must equal those of the allocating entry point within
the 1e-12 relative tolerance that f64 atomic summation order allows (maxima
are exact)."""
import ctypes as C

import numpy as np
import pytest

from autoquantizer_b200 import _lib

pytestmark = pytest.mark.gpu


def _call(fn, a, b, ns):
    sq = (C.c_double * ns)()
    mx = (C.c_double * ns)()
    rc = fn(C.c_void_p(a.data_ptr()), int(a.dtype.itemsize == 8), C.c_void_p(b.data_ptr()),
            int(b.dtype.itemsize == 8), a.shape[0], ns, sq, mx, _lib.stream_ptr())
    _lib.check(rc, fn.__name__)
    return np.array(sq[:]), np.array(mx[:])


def test_noalloc_matches_allocating_entry_point_twice():
    import torch

    L = _lib.lib()
    rng = np.random.default_rng(0)
    for call, (n, ns, f64) in enumerate([(200_003, 24, False), (50_001, 9, True)]):
        a = torch.from_numpy(rng.normal(size=(n, ns))).cuda()
        b = torch.from_numpy(rng.normal(size=(n, ns)) * (call + 1)).cuda()
        if not f64:
            a, b = a.float(), b.float()
        sq_ref, mx_ref = _call(L.aq_state_error, a, b, ns)
        sq, mx = _call(L.aq_state_error_noalloc, a, b, ns)
        assert sq == pytest.approx(sq_ref, rel=1e-12)
        assert np.array_equal(mx, mx_ref)
        direct = ((a.double() - b.double()) ** 2).sum(0).cpu().numpy()
        assert sq == pytest.approx(direct, rel=1e-9)


def test_noalloc_rejects_sizes_above_its_limit():
    import torch

    a = torch.zeros((4, 257), device="cuda")
    sq = (C.c_double * 257)()
    mx = (C.c_double * 257)()
    rc = _lib.lib().aq_state_error_noalloc(C.c_void_p(a.data_ptr()), 0, C.c_void_p(a.data_ptr()), 0, 4, 257, sq, mx,
                                           _lib.stream_ptr())
    assert rc == -6  # AQ_E_LIMIT
