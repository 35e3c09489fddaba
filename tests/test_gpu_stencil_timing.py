"""cvcb_time_stencil, the timing entry point behind the profiles and the
benchmark's stencil figures: every kind runs on a small lattice and returns a
positive time; an unknown kind is an argument error, not a launch."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [1, 2], ids=["fp32", "fp16"])
def test_every_kind_times(cb, prec):
    dims = (16, 8, 8, 8)
    lat = cb.Lattice(*dims, kappa=0.155, mu=0.005 / 0.31)
    lat.upload_gauge(cb.gauge_random(*dims, 0.25, 11))
    ms = ctypes.c_double()
    for kind in (0, 1, 2, 3):
        rc = lat._lib.cvcb_time_stencil(lat._h, kind, prec, 12, 6, 3, ctypes.byref(ms))
        assert rc == 0, (kind, cb.last_error())
        assert ms.value > 0, kind
    for kind in (-1, 4):
        ms.value = 0.0
        rc = lat._lib.cvcb_time_stencil(lat._h, kind, prec, 12, 6, 3, ctypes.byref(ms))
        assert rc == cb._lib.CVCB_ERR_ARG and ms.value == 0.0, kind
    lat.close()
