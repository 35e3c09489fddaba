"""Times the operator kernels alone, with CUDA events, through cvcb_time_stencil.

    python -m cvc_b200.stencil_timing --kind 2 --precision single --recon 12 --nrhs 12

kind 0: Q_phi_tbc on one FP64 field (all V sites); kind 1: one half-lattice
sweep of the batched solver's stencil; kind 2: one application of its normal
operator M^+ M (four sweeps); kind 3: the same with the fused partial sums of
|M p|^2 of a CG iteration (no extra field traffic).  The lattice and gauge field are those of the
solver benchmark (24^3x48, ranlxd seed 11, eps 0.25) unless overridden.
Prints one line: milliseconds per call, algorithmic GB/s (compulsory traffic:
each input spinor, output spinor and link once) and, labelled, the no-reuse
figure (every one of the 8 neighbour spinors and 8 links of a site counted at
each use, links once per rhs pair of the packed kernel), which counts what the
caches serve and can exceed the HBM peak; and the flop rate in the Wilson
convention (1320 flop per site for the hopping term, 48 for the diagonal
term, 24 for the factor -1/2: 1392 per output site and rhs).
"""
import argparse
import ctypes

from . import lattice as _lat

_PREC = {"double": 0, "single": 1, "half": 2}
_SPINOR = {0: 192, 1: 96, 2: 52}           # bytes per site and rhs
_LINK = {(0, 18): 144, (1, 12): 48, (1, 18): 72, (2, 12): 24, (2, 18): 72}


def algorithmic_bytes(kind, prec, recon, nrhs, dims):
    T, LX, LY, LZ = dims
    V = T * LX * LY * LZ
    Vh = V // 2
    if kind == 0:
        # spinor in and out, and the 4 links of the site (each link serves the
        # forward hop of its site and the backward hop of its neighbour)
        return V * (2 * 192 + 4 * 144)
    links = 4 * V * _LINK[(prec, 18 if prec == 0 else recon)]
    sweep = lambda nf: nrhs * Vh * nf * _SPINOR[prec] + links
    return sweep(2) if kind == 1 else 2 * sweep(2) + 2 * sweep(3)  # kinds 2 and 3


FLOP_PER_SITE = 1320 + 48 + 24


def flops(kind, nrhs, dims):
    """Wilson-convention flops of one call: 1392 per output site and rhs and sweep."""
    T, LX, LY, LZ = dims
    V = T * LX * LY * LZ
    if kind == 0:
        return V * FLOP_PER_SITE
    sweep = nrhs * (V // 2) * FLOP_PER_SITE
    return sweep if kind == 1 else 4 * sweep


def no_reuse_bytes(kind, prec, recon, nrhs, dims, rhs_per_link=2):
    """8 neighbour spinors + 8 links + output (+ the diagonal term's input)
    per output site and rhs, links shared by `rhs_per_link` rhs (FP64
    full-lattice operator: 8 x 192 + 8 x 144 + 192 + 192 = 3072 B per site)."""
    T, LX, LY, LZ = dims
    V = T * LX * LY * LZ
    if kind == 0:
        return V * (8 * 192 + 8 * 144 + 2 * 192)
    s = _SPINOR[prec]
    r = _LINK[(prec, 18 if prec == 0 else recon)]
    per = lambda aux: 8 * s + 8 * r / rhs_per_link + s * (1 + aux)
    sweep = lambda aux: nrhs * (V // 2) * per(aux)
    return sweep(0) if kind == 1 else 2 * sweep(0) + 2 * sweep(1)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--kind", type=int, default=1, choices=(0, 1, 2, 3))
    ap.add_argument("--precision", default="single", choices=tuple(_PREC))
    ap.add_argument("--recon", type=int, default=12, choices=(12, 18))
    ap.add_argument("--nrhs", type=int, default=12)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--dims", type=int, nargs=4, default=(48, 24, 24, 24), metavar=("T", "LX", "LY", "LZ"))
    ap.add_argument("--eps", type=float, default=0.25)
    ap.add_argument("--seed", type=int, default=11)
    a = ap.parse_args(argv)
    prec = _PREC[a.precision]
    lat = _lat.Lattice(*a.dims, kappa=0.155, mu=0.005 / 0.31)
    lat.upload_gauge(_lat.gauge_random(*a.dims, a.eps, a.seed))
    ms = ctypes.c_double()
    _lat._check("cvcb_time_stencil", lat._lib.cvcb_time_stencil(
        lat._h, a.kind, prec, a.recon, a.nrhs, a.reps, ctypes.byref(ms)))
    nbytes = algorithmic_bytes(a.kind, prec, a.recon, a.nrhs, a.dims)
    nr = no_reuse_bytes(a.kind, prec, a.recon, a.nrhs, a.dims)
    print(f"kind {a.kind} {a.precision} recon {a.recon} nrhs {a.nrhs} dims {list(a.dims)}: "
          f"{ms.value:.4f} ms per call, {nbytes / ms.value / 1e6:.1f} GB/s algorithmic "
          f"({nr / ms.value / 1e6:.1f} GB/s no-reuse), "
          f"{flops(a.kind, a.nrhs, a.dims) / ms.value / 1e9:.2f} TFLOP/s")
    lat.close()


if __name__ == "__main__":
    main()
