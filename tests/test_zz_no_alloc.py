"""The no-allocation scalar product (cvcb_spinor_scalar_product_co_noalloc).

It exists for callers that cannot allocate device memory -- their memory
belongs to a pool of their own, or a cudaMalloc would synchronise a device
they keep busy.  Its scratch is a fixed device array inside the library, so
this test checks, through the C ABI, that two calls in a row (sharing that
array) give the same result as the regular entry point, and that sizes
beyond the array's limit are refused.  Kept in its own file so that it runs
after every other test."""
import ctypes

import numpy as np
import pytest

from conftest import seeded

pytestmark = pytest.mark.gpu

MAX_SITES = 5592405


def test_noalloc_matches_regular_entry_point_twice(cb):
    torch = pytest.importorskip("torch")
    lib = cb.load()
    dims = (8, 8, 8, 16)
    V = 8 * 8 * 8 * 16
    lat = cb.Lattice(*dims, device=0)
    results = []
    for call in range(2):
        a = seeded(300 + call, 24 * V)
        b = seeded(400 + call, 24 * V)
        da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        w = torch.zeros(2, dtype=torch.float64, device="cuda")
        rc = lib.cvcb_spinor_scalar_product_co_noalloc(0, w.data_ptr(), da.data_ptr(),
                                                       db.data_ptr(), V, None)
        assert rc == 0, cb.last_error()
        torch.cuda.synchronize()
        got = complex(w[0].item(), w[1].item())
        ref = lat.spinor_scalar_product_co(a, b, V)
        assert abs(got - ref) <= 1e-13 * abs(ref)
        results.append(got)
    assert results[0] != results[1]
    lat.close()


def test_noalloc_partial_volume_and_limits(cb):
    torch = pytest.importorskip("torch")
    lib = cb.load()
    V = 1000
    a = seeded(7, 24 * V)
    b = seeded(8, 24 * V)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    w = torch.zeros(2, dtype=torch.float64, device="cuda")
    for nv in (V, 37):
        assert lib.cvcb_spinor_scalar_product_co_noalloc(0, w.data_ptr(), da.data_ptr(),
                                                         db.data_ptr(), nv, None) == 0
        torch.cuda.synchronize()
        x = (a[:24 * nv:2] + 1j * a[1:24 * nv:2])
        y = (b[:24 * nv:2] + 1j * b[1:24 * nv:2])
        ref = np.sum(np.conj(x) * y)
        assert abs(complex(w[0].item(), w[1].item()) - ref) <= 1e-13 * abs(ref)
    # beyond the fixed scratch array, and host memory: refused, nothing launched
    assert lib.cvcb_spinor_scalar_product_co_noalloc(0, w.data_ptr(), da.data_ptr(),
                                                     db.data_ptr(), MAX_SITES + 1, None) == -1
    assert "outside" in cb.last_error()
    h = np.zeros(2)
    assert lib.cvcb_spinor_scalar_product_co_noalloc(0, h.ctypes.data, da.data_ptr(),
                                                     db.data_ptr(), V, None) == -1


def test_noalloc_allocates_nothing_on_a_caller_stream(cb):
    """The property the entry point exists for: after a first call on the
    device (which looks up the fixed array's address), further calls change
    no device memory usage, also when enqueued on a stream of the caller's
    (stream-ordered: the result is ready when that stream reaches it)."""
    torch = pytest.importorskip("torch")
    lib = cb.load()
    V = 4096
    a = seeded(11, 24 * V)
    b = seeded(12, 24 * V)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    w = torch.zeros(2, dtype=torch.float64, device="cuda")
    assert lib.cvcb_spinor_scalar_product_co_noalloc(0, w.data_ptr(), da.data_ptr(),
                                                     db.data_ptr(), V, None) == 0
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    free0, _ = torch.cuda.mem_get_info()
    x = (a[0::2] + 1j * a[1::2])
    y = (b[0::2] + 1j * b[1::2])
    ref = np.sum(np.conj(x) * y)
    for _ in range(3):
        w.zero_()
        torch.cuda.synchronize()
        assert lib.cvcb_spinor_scalar_product_co_noalloc(0, w.data_ptr(), da.data_ptr(),
                                                         db.data_ptr(), V, s.cuda_stream) == 0
        s.synchronize()
        assert abs(complex(w[0].item(), w[1].item()) - ref) <= 1e-13 * abs(ref)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
