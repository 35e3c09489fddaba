"""Times the CVC contraction (cvcb_cvc_contract) on device-resident fields.

    python -m cvc_b200.contract_timing --dims 48 24 24 24 --reps 5

120 random FP64 propagator columns on the GPU, random gauge field; prints
milliseconds per contraction and the rates against the per-site counts of
the reference's algorithm: 663,552 flop and 23,872 compulsory bytes per
site and source (120 columns x 192 B + 4 links x 144 B + Pi 16 x 16 B).
"""
import argparse
import time

import numpy as np

from .lattice import Lattice, gauge_random

FLOP_PER_SITE = 663552
BYTES_PER_SITE = 120 * 192 + 4 * 144 + 16 * 16


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--dims", type=int, nargs=4, default=(48, 24, 24, 24),
                    metavar=("T", "LX", "LY", "LZ"))
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--source", type=int, default=0)
    a = ap.parse_args(argv)
    import torch
    dims = tuple(a.dims)
    V = int(np.prod(dims))
    lat = Lattice(*dims, kappa=0.155, mu=0.005 / 0.31)
    lat.upload_gauge(gauge_random(*dims, 0.25, 11))
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1)
    fields = [torch.rand(24 * V, dtype=torch.float64, device="cuda", generator=gen) - 0.5
              for _ in range(120)]
    conn = torch.zeros(32 * V, dtype=torch.float64, device="cuda")
    lat.cvc_contract(fields, a.source, conn=conn)  # warm-up
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(a.reps):
        t = time.perf_counter()
        lat.cvc_contract(fields, a.source, conn=conn)
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t)
    print(f"contraction {list(dims)}: {best * 1e3:.2f} ms, "
          f"{FLOP_PER_SITE * V / best / 1e12:.2f} TFLOP/s (reference flop count), "
          f"{BYTES_PER_SITE * V / best / 1e9:.0f} GB/s compulsory bytes")
    lat.close()


if __name__ == "__main__":
    main()
