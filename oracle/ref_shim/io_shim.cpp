/* Raw-binary stand-ins for the four LIME-dependent symbols that the
 * reference's operator / solver / contraction path links against.
 *
 * This file is test infrastructure for the oracle build: it is compiled
 * together with the unmodified reference sources into oracle/_ref/ and is
 * never part of the shipped library.
 *
 * File format (chosen here, not the reference's): native-endian IEEE doubles
 * in CVC's in-memory order, no header.
 *   gauge      : 72*VOLUME doubles, link (x,mu) at 18*(4x+mu)   (global.h:_GGI)
 *   propagator : one or more records of 24*VOLUME doubles; `position`
 *                selects the record, as the LIME record index does in
 *                read_lime_spinor (propagator_io.c:771-840)
 *   contraction: 2*N*VOLUME doubles, written as conn[] is held in memory
 *                (contractions_io.c:289 writes the same values as LIME).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "global.h"
#include "cvc_utils.h"

namespace cvc {

static int oracle_read_raw(const char *fn, double *dst, size_t n, size_t skip) {
  FILE *f = fopen(fn, "rb");
  if (!f) { fprintf(stderr, "[io_shim] cannot open %s\n", fn); return 1; }
  if (skip && fseek(f, (long)(skip * sizeof(double)), SEEK_SET) != 0) {
    fclose(f); fprintf(stderr, "[io_shim] seek failed in %s\n", fn); return 2;
  }
  size_t got = fread(dst, sizeof(double), n, f);
  fclose(f);
  if (got != n) { fprintf(stderr, "[io_shim] short read %zu/%zu in %s\n", got, n, fn); return 3; }
  return 0;
}

int read_lime_gauge_field_doubleprec(const char *filename) {
  return oracle_read_raw(filename, g_gauge_field, (size_t)72 * VOLUME, 0);
}

int read_lime_spinor(double *const s, char *filename, const int position) {
  return oracle_read_raw(filename, s, (size_t)24 * VOLUME, (size_t)position * 24 * VOLUME);
}

int write_lime_contraction(double *const s, char *filename, const int prec, const int N,
                           char *type, const int gid, const int sid) {
  (void)prec; (void)type; (void)gid; (void)sid;
  FILE *f = fopen(filename, "wb");
  if (!f) { fprintf(stderr, "[io_shim] cannot write %s\n", filename); return 1; }
  size_t n = (size_t)2 * N * VOLUME;
  size_t put = fwrite(s, sizeof(double), n, f);
  fclose(f);
  return put == n ? 0 : 2;
}

}  // namespace cvc

/* LAPACK is only reached through cm_proj (cvc_utils.c:2794-2920), which is
 * off the path; these stubs make the link succeed and abort if ever called. */
extern "C" int ilaenv(int *, char *, char *, int *, int *, int *, int *) {
  fprintf(stderr, "[io_shim] LAPACK ilaenv called; not available in the oracle build\n");
  abort();
}
extern "C" void zheev(char *, char *, int *, double *, int *, double *, double *, int *,
                       double *, int *) {
  fprintf(stderr, "[io_shim] LAPACK zheev called; not available in the oracle build\n");
  abort();
}
