"""cvc_b200 -- B200 (sm_100a) implementation of CVC's propagator-and-
contraction path.

The work is done by libcvcb200.so (CUDA kernels + C ABI, include/cvcb.h).
This package is the host-side mirror of the reference's interface for the
path: `Lattice` holds the state that CVC keeps in globals (geometry, g_kappa,
g_mu, BCangle, g_gauge_field) and its methods carry the reference function
names (Q_phi_tbc, Hopping, Qf5, Q_phi, g5_phi, mul_one_pm_imu_inv,
spinor_scalar_product_co/_re, invert_Qtm, invert_Qtm_her, plaquette) with
the same argument meaning; the contraction of cvc_exact2_xspace.c and the
sequential source of p2gg_xspace.c are `cvc_contract` and `p2gg_seq_source`.
"""
from ._lib import (PREC_DOUBLE, PREC_HALF, PREC_SINGLE, SolverParams, SolverStats,  # noqa: F401
                   last_error, load)
from .lattice import (CvcbError, Lattice, boundary_phases, gamma_tables,  # noqa: F401
                      gauge_random, geometry_tables, ranlxd, solver_defaults)

__all__ = [
    "Lattice", "CvcbError", "geometry_tables", "gamma_tables", "boundary_phases",
    "ranlxd", "gauge_random", "solver_defaults", "SolverParams", "SolverStats",
    "PREC_DOUBLE", "PREC_SINGLE", "PREC_HALF", "load", "last_error",
]
