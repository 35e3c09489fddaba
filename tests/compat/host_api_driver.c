/* A C99 program on the host-only part of the C ABI (include/cvcb.h): the
 * geometry, gamma and phase tables, RANLUX, the gauge generator, CRC-32 and
 * the LIME gauge/spinor files.  It prints one line of "key value" pairs that
 * the Python test compares with the same calls made through ctypes, so the
 * header and library are checked from C, as a non-Python host (cgo, JNI or
 * N-API stubs) would use them.  No GPU is needed.
 *
 *   host_api_driver <scratch directory>
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cvcb.h"

#define CHECK(call)                                                        \
  do {                                                                     \
    int rc_ = (call);                                                      \
    if (rc_ != CVCB_OK) {                                                  \
      fprintf(stderr, "%s: %d (%s)\n", #call, rc_, cvcb_last_error());     \
      return 1;                                                            \
    }                                                                      \
  } while (0)

static long long isum(const int *a, long n) {
  long long s = 0;
  for (long i = 0; i < n; ++i) s += (long long)(i % 7 + 1) * a[i];
  return s;
}

static double dsum(const double *a, long n) {
  double s = 0.0;
  for (long i = 0; i < n; ++i) s += (double)(i % 5 + 1) * a[i];
  return s;
}

int main(int argc, char **argv) {
  if (argc != 2) {
    fprintf(stderr, "usage: %s <scratch directory>\n", argv[0]);
    return 2;
  }
  const int T = 8, LX = 4, LY = 4, LZ = 2;
  const long V = (long)T * LX * LY * LZ;
  int *ipt = calloc((size_t)(T + 2) * LX * LY * LZ, sizeof(int));
  int *iup = calloc((size_t)4 * V, sizeof(int)), *idn = calloc((size_t)4 * V, sizeof(int));
  int *l2eo = calloc((size_t)V, sizeof(int));
  int perm[16 * 24], sign[16 * 24];
  double ph[8], bc[4] = {1.0, 0.5, 0.0, 0.25};
  double r[1000];
  double *g = malloc(sizeof(double) * 72 * (size_t)V), *g2 = malloc(sizeof(double) * 72 * (size_t)V);
  double *s = malloc(sizeof(double) * 24 * (size_t)V), *s2 = malloc(sizeof(double) * 24 * (size_t)V);
  if (!ipt || !iup || !idn || !l2eo || !g || !g2 || !s || !s2) return 3;

  CHECK(cvcb_geometry_tables(T, LX, LY, LZ, ipt, iup, idn, l2eo, NULL, NULL, NULL, NULL, NULL));
  CHECK(cvcb_gamma_tables(perm, sign));
  CHECK(cvcb_boundary_phases(T, LX, LY, LZ, bc, ph));
  CHECK(cvcb_ranlxd(1, 17, r, 1000));
  CHECK(cvcb_gauge_random(g, T, LX, LY, LZ, 0.3, 1234));
  for (long i = 0; i < 24 * V; ++i) s[i] = r[i % 1000] - 0.5;

  uint32_t crc = 0;
  CHECK(cvcb_crc32(0, "cvc-b200", 8, &crc));

  char fg[4096], fs[4096];
  snprintf(fg, sizeof fg, "%s/gauge.ildg", argv[1]);
  snprintf(fs, sizeof fs, "%s/spinor.lime", argv[1]);
  uint32_t cw[2], cr[2], sw[2], sr[2];
  CHECK(cvcb_write_lime_gauge_field(fg, g, T, LX, LY, LZ, 64, cw));
  CHECK(cvcb_read_lime_gauge_field_doubleprec(fg, g2, T, LX, LY, LZ, cr));
  CHECK(cvcb_write_lime_spinor(s, fs, 0, 64, T, LX, LY, LZ, sw));
  CHECK(cvcb_read_lime_spinor(s2, fs, 0, T, LX, LY, LZ, sr));
  const int gauge_same = memcmp(g, g2, sizeof(double) * 72 * (size_t)V) == 0;
  const int spinor_same = memcmp(s, s2, sizeof(double) * 24 * (size_t)V) == 0;

  printf("ipt %lld iup %lld idn %lld lexic2eo %lld perm %lld sign %lld "
         "ph %.17g ranlxd %.17g gauge %.17g crc %u "
         "gauge_sums %u %u %u %u spinor_sums %u %u %u %u gauge_same %d spinor_same %d\n",
         isum(ipt, (long)(T + 2) * LX * LY * LZ), isum(iup, 4 * V), isum(idn, 4 * V),
         isum(l2eo, V), isum(perm, 16 * 24), isum(sign, 16 * 24), dsum(ph, 8), dsum(r, 1000),
         dsum(g, 72 * V), (unsigned)crc, (unsigned)cw[0], (unsigned)cw[1], (unsigned)cr[0],
         (unsigned)cr[1], (unsigned)sw[0], (unsigned)sw[1], (unsigned)sr[0], (unsigned)sr[1],
         gauge_same, spinor_same);
  free(ipt);
  free(iup);
  free(idn);
  free(l2eo);
  free(g);
  free(g2);
  free(s);
  free(s2);
  return 0;
}
