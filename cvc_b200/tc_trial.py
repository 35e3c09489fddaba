"""Tensor-core trial of the stencil's link product, through
cvcb_time_link_product: the product u = W h of the 8 links of every site of
a half lattice with one block of 2 spins x 12 right-hand sides, as packed
FP32x2 FMAs (what the stencil does), as mma.sync TF32 tiles holding two
sites' links block-diagonally, and as the same with three TF32 products
(FP32 accuracy).

    python -m cvc_b200.tc_trial --dims 48 24 24 24 --reps 50

prints, per variant, the time per launch, the equivalent rate of useful
flops (6 x 6 x 24 x 2 per site and link) and the deviation from the FFMA2
result relative to its largest component.
"""
import argparse
import ctypes

from . import lattice as _lat

NAMES = {0: "packed FP32x2 FMAs", 1: "mma.sync TF32", 2: "mma.sync 3xTF32"}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--dims", type=int, nargs=4, default=(48, 24, 24, 24),
                    metavar=("T", "LX", "LY", "LZ"))
    ap.add_argument("--reps", type=int, default=50)
    ap.add_argument("--eps", type=float, default=0.25)
    ap.add_argument("--seed", type=int, default=11)
    a = ap.parse_args(argv)
    dims = tuple(a.dims)
    lat = _lat.Lattice(*dims, kappa=0.155, mu=0.005 / 0.31)
    lat.upload_gauge(_lat.gauge_random(*dims, a.eps, a.seed))
    vh = dims[0] * dims[1] * dims[2] * dims[3] // 2
    useful = vh * 8 * 6 * 6 * 24 * 2
    for v in (0, 1, 2):
        ms, diff = ctypes.c_double(), ctypes.c_double()
        _lat._check("cvcb_time_link_product", lat._lib.cvcb_time_link_product(
            lat._h, v, a.reps, ctypes.byref(ms), ctypes.byref(diff)))
        print(f"variant {v} ({NAMES[v]}): {ms.value:.4f} ms per launch, "
              f"{useful / ms.value / 1e9:.1f} TFLOP/s useful, rel. deviation {diff.value:.2e}",
              flush=True)
    lat.close()


if __name__ == "__main__":
    main()
