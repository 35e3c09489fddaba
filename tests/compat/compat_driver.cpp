// Test program: reference code linked against the drop-in library.
//
// Built by `make -C oracle compat` from this file, the unmodified reference
// objects for geometry and utilities, and libcvcb200_cvc.so in place of
// Q_phi.o and invert_Qtm.o.  It sets up the reference's globals as its
// programs do, reads a raw gauge field and spinor, and calls the reference
// interface: Q_phi_tbc, Qf5, the scalar products, invert_Qtm_her, and the
// reference's own check_source (cvc_utils.c), which itself calls Q_phi and
// spinor_scalar_product_re -- now bound to the GPU versions.  Then the
// point-source breakdown of invert_Qtm, and Q_phi_tbc after one link of
// g_gauge_field was edited in place.
//
// usage: compat_driver T LX LY LZ kappa mu gauge.bin phi.bin out_prefix
#define MAIN_PROGRAM
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "global.h"
#include "cvc_complex.h"
#include "cvc_geometry.h"
#include "cvc_utils.h"
#include "mpi_init.h"
#include "Q_phi.h"
#include "invert_Qtm.h"

using namespace cvc;

static void read_raw(const char *fn, double *p, size_t n) {
  FILE *f = fopen(fn, "rb");
  if (!f || fread(p, sizeof(double), n, f) != n) { fprintf(stderr, "cannot read %s\n", fn); exit(2); }
  fclose(f);
}
static void write_raw(const char *prefix, const char *tag, const double *p, size_t n) {
  char fn[512];
  snprintf(fn, sizeof fn, "%s.%s", prefix, tag);
  FILE *f = fopen(fn, "wb");
  fwrite(p, sizeof(double), n, f);
  fclose(f);
}

int main(int argc, char **argv) {
  if (argc != 10) { fprintf(stderr, "usage: %s T LX LY LZ kappa mu gauge phi out\n", argv[0]); return 2; }
  T_global = atoi(argv[1]); LX = atoi(argv[2]); LY = atoi(argv[3]); LZ = atoi(argv[4]);
  g_kappa = atof(argv[5]); g_mu = atof(argv[6]);
  BCangle[0] = 1.; BCangle[1] = BCangle[2] = BCangle[3] = 0.;
  g_gpu_device_number = 0;
  mpi_init(argc, argv);
  if (init_geometry() != 0) return 3;
  geometry();
  alloc_gauge_field(&g_gauge_field, VOLUMEPLUSRAND);
  read_raw(argv[7], g_gauge_field, (size_t)72 * VOLUME);
  double *phi, *xi, *work;
  alloc_spinor_field(&phi, VOLUMEPLUSRAND);
  alloc_spinor_field(&xi, VOLUMEPLUSRAND);
  alloc_spinor_field(&work, VOLUMEPLUSRAND);
  read_raw(argv[8], phi, (size_t)24 * VOLUME);

  Q_phi_tbc(xi, phi);
  write_raw(argv[9], "Q_phi_tbc", xi, (size_t)24 * VOLUME);
  Qf5(xi, phi, -g_mu);
  write_raw(argv[9], "Qf5_minus", xi, (size_t)24 * VOLUME);
  complex w;
  spinor_scalar_product_co(&w, phi, xi, VOLUME);
  printf("dot %.17e %.17e\n", w.re, w.im);

  // point source at the origin, spin-colour 4; solve with the reference's
  // stopping rule and check with the reference's own check_source
  memset(phi, 0, sizeof(double) * 24 * VOLUME);
  phi[2 * 4] = 1.0;
  memset(xi, 0, sizeof(double) * 24 * VOLUME);
  solver_precision = 1e-20;
  niter_max = 2000;
  int n = invert_Qtm_her(xi, phi, 0);
  printf("niter %d\n", n);
  write_raw(argv[9], "x", xi, (size_t)24 * VOLUME);
  check_source(xi, work, g_mu, 0, 4);

  // plain BiCGStab breaks down on a point source: the reference's -3
  memset(xi, 0, sizeof(double) * 24 * VOLUME);
  printf("breakdown %d\n", invert_Qtm(xi, phi, 0));

  // edit one link in place (site 37, mu 2, times e^{0.7 i}) and apply the
  // operator again: the library must notice and upload the field again
  read_raw(argv[8], phi, (size_t)24 * VOLUME);
  double *u = g_gauge_field + 18 * (4 * 37 + 2);
  const double c = cos(0.7), s = sin(0.7);
  for (int k = 0; k < 9; ++k) {
    const double re = u[2 * k], im = u[2 * k + 1];
    u[2 * k] = c * re - s * im;
    u[2 * k + 1] = s * re + c * im;
  }
  Q_phi_tbc(xi, phi);
  write_raw(argv[9], "Q_phi_tbc_edit", xi, (size_t)24 * VOLUME);
  return 0;
}
