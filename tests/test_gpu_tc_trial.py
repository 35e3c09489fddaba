"""The tensor-core trial of the stencil's link product (cvcb_time_link_product):
the mma.sync TF32 variants compute the same 8-link products of a half
lattice as the packed FP32x2 FMAs, to TF32 accuracy (one product: 2e-3
relative to the largest component) and to FP32 accuracy with three TF32
products (1e-5)."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def test_link_product_variants_agree(cb):
    dims = (16, 8, 8, 8)
    lat = cb.Lattice(*dims, kappa=0.155, mu=0.005 / 0.31)
    lat.upload_gauge(cb.gauge_random(*dims, 0.25, 11))
    for v, tol in ((0, 0.0), (1, 2e-3), (2, 1e-5)):
        ms, diff = ctypes.c_double(), ctypes.c_double()
        rc = lat._lib.cvcb_time_link_product(lat._h, v, 3, ctypes.byref(ms), ctypes.byref(diff))
        assert rc == 0, cb.last_error()
        assert ms.value > 0 and diff.value <= tol, (v, diff.value)
    lat.close()
