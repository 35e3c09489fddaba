/* cvcb_tmlqcd.h -- the tmLQCD library-wrapper ABI (tmLQCD.h:33-58 of the
 * reference, the header CVC includes under HAVE_TMLQCD_LIBWRAPPER), served by
 * libcvcb200_tmlqcd.so over the B200 solver.  A program built against
 * tmLQCD.h links this library instead of tmLQCD; the types and functions
 * keep tmLQCD's names, layouts and meaning:
 *
 *  - one process, one GPU: the MPI parameters describe a single rank;
 *  - operators: each "BeginOperator ... EndOperator" block of the input file
 *    (kappa, 2KappaMu, SolverPrecision, MaxSolverIterations,
 *    UseRelativePrecision) is one op_id; SolverPrecision is the squared
 *    residual |b - D x|^2, absolute unless UseRelativePrecision = yes, as in
 *    tmLQCD's input files;
 *  - tmLQCD_invert returns the solution of D psi = source with tmLQCD's
 *    normalisation D = 2 kappa Q = (1 + 2 i kappa mu g5) - kappa H, i.e.
 *    psi = Q^-1 source / (2 kappa), in CVC's field layout;
 *  - all functions return 0 on success.
 * Input keys and defaults are listed in the library source
 * (cvc_b200/compat/tmlqcd_compat.cpp). */
#ifndef CVCB_TMLQCD_H
#define CVCB_TMLQCD_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  unsigned int LX, LY, LZ, T, nstore, nsave, no_operators;
} tmLQCD_lat_params;

/* tmLQCD.h:38-44 (without the MPI communicator, which a build without MPI
 * does not have either) */
typedef struct {
  unsigned int nproc, nproc_t, nproc_x, nproc_y, nproc_z, cart_id, proc_id, time_rank,
      omp_num_threads;
  unsigned int proc_coords[4];
} tmLQCD_mpi_params;

/* tmLQCD.h:46: reads the input file (argv "-f <file>", default
 * "invert.input") and sets up the lattice on the GPU. */
int tmLQCD_invert_init(int argc, char *argv[], const int verbose);

/* tmLQCD.h:47: reads the ILDG gauge file "<GaugeConfigInputFile>.%04d". */
int tmLQCD_read_gauge(const int nconfig);

/* tmLQCD.h:48-49: propagator = D(op_id)^-1 source (CVC layout, 24*V doubles
 * each); write_prop != 0 also writes it as "<PropagatorFilePrefix>.%04d.%02d.inverted"
 * (nstore, running index). */
int tmLQCD_invert(double *const propagator, double *const source, const int op_id,
                  const int write_prop);

/* tmLQCD.h:50: releases the GPU context and the gauge field. */
int tmLQCD_finalise();

/* tmLQCD.h:52-54 */
int tmLQCD_get_gauge_field_pointer(double **gf);
int tmLQCD_get_mpi_params(tmLQCD_mpi_params *params);
int tmLQCD_get_lat_params(tmLQCD_lat_params *params);

#ifdef __cplusplus
}
#endif
#endif
