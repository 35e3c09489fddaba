/* Follows the tmLQCD-library branch of cvc_exact2_xspace.c (:131-150 init and
 * parameters, :206-216 gauge field, :436-547 the two operators x 12
 * spin-colour point-source inversions at the unshifted source, :1032
 * finalise) against libcvcb200_tmlqcd.so, and dumps the gauge field it got
 * and the propagators as raw doubles for the test to compare; then one
 * inversion of a source of norm 1e-3 (absolute SolverPrecision).
 *   tmlqcd_driver -f <input> <t> <x> <y> <z> <outdir> */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cvcb_tmlqcd.h"

static int dump(const char *dir, const char *name, const double *v, size_t n) {
  char fn[2048];
  snprintf(fn, sizeof fn, "%s/%s", dir, name);
  FILE *f = fopen(fn, "wb");
  if (!f) return 1;
  size_t w = fwrite(v, sizeof(double), n, f);
  fclose(f);
  return w != n;
}

int main(int argc, char **argv) {
  if (argc < 8) return 100;
  const int src[4] = {atoi(argv[3]), atoi(argv[4]), atoi(argv[5]), atoi(argv[6])};
  const char *out = argv[7];
  tmLQCD_mpi_params mpi;
  tmLQCD_lat_params lat;
  if (tmLQCD_invert_init(argc, argv, 1) != 0) exit(557);
  if (tmLQCD_get_mpi_params(&mpi) != 0) exit(558);
  if (tmLQCD_get_lat_params(&lat) != 0) exit(559);
  if (mpi.nproc != 1 || mpi.cart_id != 0) return 101;
  if (tmLQCD_read_gauge(lat.nstore) != 0) exit(560);
  double *gauge = NULL;
  if (tmLQCD_get_gauge_field_pointer(&gauge) != 0 || !gauge) exit(561);
  const size_t V = (size_t)lat.T * lat.LX * lat.LY * lat.LZ;
  if (dump(out, "gauge.raw", gauge, 72 * V)) return 102;
  double *source = calloc(24 * V, sizeof(double)), *prop = calloc(24 * V, sizeof(double));
  const size_t ix = (((size_t)src[0] * lat.LX + src[1]) * lat.LY + src[2]) * lat.LZ + src[3];
  for (unsigned op = 0; op < lat.no_operators; ++op)
    for (int ia = 0; ia < 12; ++ia) {
      memset(source, 0, 24 * V * sizeof(double));
      source[24 * ix + 2 * ia] = 1.;
      if (tmLQCD_invert(prop, source, (int)op, op == 0 && ia == 0) != 0) exit(7);
      char name[64];
      snprintf(name, sizeof name, "prop.%u.%02d.raw", op, ia);
      if (dump(out, name, prop, 24 * V)) return 103;
    }
  /* a source of norm 1e-3: SolverPrecision is absolute, as in tmLQCD */
  memset(source, 0, 24 * V * sizeof(double));
  source[24 * ix] = 1e-3;
  if (tmLQCD_invert(prop, source, 0, 0) != 0) exit(8);
  if (dump(out, "prop.scaled.raw", prop, 24 * V)) return 104;
  free(source);
  free(prop);
  tmLQCD_finalise();
  return 0;
}
