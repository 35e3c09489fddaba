/* extern "C" access to the unmodified reference functions, for the oracle.
 *
 * Test infrastructure only: compiled with the reference sources into
 * oracle/_ref/libcvcref.so and loaded by the tests (and by the CPU-baseline
 * leg of the benchmark) to pin the plain-C restatement and the CUDA path.
 *
 * The reference keeps all state in globals inside namespace cvc (global.h);
 * this file defines them (MAIN_PROGRAM) and exposes set-up and calls with
 * plain pointers and sizes.
 */
#define MAIN_PROGRAM
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include "global.h"
#include "cvc_complex.h"
#include "cvc_linalg.h"
#include "cvc_geometry.h"
#include "cvc_utils.h"
#include "mpi_init.h"
#include "Q_phi.h"
#include "invert_Qtm.h"
#include "ranlxd.h"
#include "dml.h"

using namespace cvc;

static int ref_nwork = 0;

extern "C" {

/* Geometry + globals as cvc_exact2_xspace.c:64-185 sets them in a non-MPI
 * build: mpi_init (mpi_init.c:792-846), init_geometry (cvc_geometry.c:343),
 * geometry (cvc_geometry.c:179). */
int ref_init(int t, int lx, int ly, int lz, double kappa, double mu, const double *bc_angle) {
  static int done = 0;
  if (done) {
    free_geometry();
    if (g_gauge_field) { free(g_gauge_field); g_gauge_field = NULL; }
    if (g_spinor_field) {
      for (int i = 0; i < ref_nwork; i++) free(g_spinor_field[i]);
      free(g_spinor_field); g_spinor_field = NULL;
    }
  }
  T_global = t; LX = lx; LY = ly; LZ = lz;
  g_kappa = kappa; g_mu = mu;
  for (int i = 0; i < 4; i++) BCangle[i] = bc_angle[i];
  mpi_init(0, NULL);
  if (init_geometry() != 0) return 1;
  geometry();
  alloc_gauge_field(&g_gauge_field, VOLUMEPLUSRAND);
  ref_nwork = 8;
  g_spinor_field = (double **)calloc(ref_nwork, sizeof(double *));
  for (int i = 0; i < ref_nwork; i++) alloc_spinor_field(&g_spinor_field[i], VOLUMEPLUSRAND);
  g_cart_id = 0;
  done = 1;
  return 0;
}

void ref_set_params(double kappa, double mu) { g_kappa = kappa; g_mu = mu; }
int ref_volume(void) { return VOLUME; }

/* Geometry tables, as laid out by init_geometry (cvc_geometry.c:391-430). */
void ref_get_tables(int *ipt, int *iup, int *idn, int *lexic2eo, int *eo2lexic, int *iseven,
                    int *isevent, int *lexic2eot, int *eot2lexic) {
  size_t nipt = (size_t)(T + 2) * LX * LY * LZ;
  memcpy(ipt, &g_ipt[0][0][0][0], nipt * sizeof(int));
  memcpy(iup, &g_iup[0][0], (size_t)4 * VOLUME * sizeof(int));
  memcpy(idn, &g_idn[0][0], (size_t)4 * VOLUME * sizeof(int));
  memcpy(lexic2eo, g_lexic2eo, (size_t)VOLUME * sizeof(int));
  memcpy(eo2lexic, g_eo2lexic, (size_t)VOLUME * sizeof(int));
  memcpy(iseven, g_iseven, (size_t)VOLUME * sizeof(int));
  memcpy(isevent, g_isevent, (size_t)VOLUME * sizeof(int));
  memcpy(lexic2eot, g_lexic2eot, (size_t)VOLUME * sizeof(int));
  memcpy(eot2lexic, g_eot2lexic, (size_t)VOLUME * sizeof(int));
}

void ref_get_gamma(int *perm, int *sign) {
  memcpy(perm, gamma_permutation, sizeof(gamma_permutation));
  memcpy(sign, gamma_sign, sizeof(gamma_sign));
}

void ref_get_phase(double *ph) {
  for (int i = 0; i < 4; i++) { ph[2 * i] = co_phase_up[i].re; ph[2 * i + 1] = co_phase_up[i].im; }
}

void ref_set_gauge(const double *g) { memcpy(g_gauge_field, g, (size_t)72 * VOLUME * sizeof(double)); }

void ref_Q_phi_tbc(double *xi, double *phi) { Q_phi_tbc(xi, phi); }
void ref_Hopping(double *xi, double *phi) { Hopping(xi, phi); }
void ref_Qf5(double *xi, double *phi, double mutm) { Qf5(xi, phi, mutm); }
void ref_Q_phi(double *xi, double *phi, double mutm) { Q_phi(xi, phi, mutm); }
void ref_g5_phi(double *phi) { g5_phi(phi); }
void ref_mul_one_pm_imu_inv(double *phi, double sign, int v) { mul_one_pm_imu_inv(phi, sign, v); }

void ref_scalar_product_co(double *w, double *xi, double *phi, int v) {
  complex c; spinor_scalar_product_co(&c, xi, phi, v); w[0] = c.re; w[1] = c.im;
}
void ref_scalar_product_re(double *r, double *xi, double *phi, int v) {
  spinor_scalar_product_re(r, xi, phi, v);
}

/* The solvers print per-iteration lines; `quiet` routes stdout to /dev/null. */
static int ref_call_solver(int her, double *xi, double *phi, double prec, int nmax, int quiet) {
  solver_precision = prec; niter_max = nmax;
  fflush(stdout);
  FILE *saved = NULL;
  int fd_saved = -1;
  if (quiet) { fd_saved = dup(fileno(stdout)); saved = freopen("/dev/null", "w", stdout); }
  int r = her ? invert_Qtm_her(xi, phi, 0) : invert_Qtm(xi, phi, 0);
  if (quiet && saved) { fflush(stdout); dup2(fd_saved, fileno(stdout)); close(fd_saved); }
  return r;
}
int ref_invert_Qtm(double *xi, double *phi, double prec, int nmax, int quiet) {
  return ref_call_solver(0, xi, phi, prec, nmax, quiet);
}
int ref_invert_Qtm_her(double *xi, double *phi, double prec, int nmax, int quiet) {
  return ref_call_solver(1, xi, phi, prec, nmax, quiet);
}

void ref_plaquette(double *pl) { plaquette(pl); }

void ref_rlxd_init(int level, int seed) { rlxd_init(level, seed); }
void ref_ranlxd(double *r, int n) { ranlxd(r, n); }
int ref_rangauss(double *y, int n) { return rangauss(y, n); }

void ref_get_filename(char *fn, int nu, int sc, int sign, const char *prefix, const char *prefix2,
                      int nconf, int fmt, int source_location) {
  strcpy(filename_prefix, prefix); strcpy(filename_prefix2, prefix2);
  Nconf = nconf; format = fmt; g_source_location = source_location;
  get_filename(fn, nu, sc, sign);
}

}  // extern "C"

extern "C" void ref_get_work(int i, double *out) {
  memcpy(out, g_spinor_field[i], (size_t)24 * VOLUME * sizeof(double));
}

/* SciDAC checksum step of the reference (dml.c) and its CRC-32 (DML_crc32.c). */
extern "C" void ref_dml_checksum_accum(unsigned int *sums, unsigned int rank, const void *buf,
                                       size_t size) {
  DML_Checksum c;
  c.suma = sums[0];
  c.sumb = sums[1];
  DML_checksum_accum(&c, (DML_SiteRank)rank, (char *)buf, size);
  sums[0] = c.suma;
  sums[1] = c.sumb;
}
extern "C" unsigned int ref_dml_crc32(unsigned int crc, const void *buf, size_t len) {
  return DML_crc32(crc, (const unsigned char *)buf, len);
}

/* Hopping-parameter-expansion helpers of the reference (Q_phi.c:536-781). */
extern "C" void ref_BHn(double *xi, double *phi, int n) { BHn(xi, phi, n); }
extern "C" void ref_BH(double *xi, double *phi) { BH(xi, phi); }
extern "C" void ref_BH2(double *xi, double *phi) { BH2(xi, phi); }
extern "C" void ref_BH3(double *xi, double *phi) { BH3(xi, phi); }
extern "C" void ref_BH5(double *xi, double *phi) { BH5(xi, phi); }
extern "C" void ref_BH7(double *xi, double *phi) { BH7(xi, phi); }
extern "C" void ref_gamma5_BdagH4_gamma5(double *xi, double *phi, double *work) {
  gamma5_BdagH4_gamma5(xi, phi, work);
}
