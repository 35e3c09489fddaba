// Host-side lattice tables, gamma tables, boundary phases, RANLUX and the
// gauge-field generator.  No GPU is touched here.
#include <cmath>
#include <cstring>
#include <vector>

#include "cvcb_internal.h"

namespace cvcb {

// CVC lexicographic index with periodic wrap (cvc_geometry.c:17-26, non-MPI).
static inline int lex_wrap(int t, int x, int y, int z, int T, int LX, int LY, int LZ) {
  t = (t + T) % T;
  x = (x + LX) % LX;
  y = (y + LY) % LY;
  z = (z + LZ) % LZ;
  return ((t * LX + x) * LY + y) * LZ + z;
}

void boundary_phases(int T, int LX, int LY, int LZ, const double bc[4], double ph[8]) {
  // cvc_geometry.c:452-459 with one process per direction.
  const int ext[4] = {T, LX, LY, LZ};
  for (int mu = 0; mu < 4; ++mu) {
    ph[2 * mu] = std::cos(bc[mu] * M_PI / (double)ext[mu]);
    ph[2 * mu + 1] = std::sin(bc[mu] * M_PI / (double)ext[mu]);
  }
}

// The 16 gamma structures in init_gamma's order (cvc_utils.c:707-748):
// g0..g3, 1, g5 = g0 g1 g2 g3, g_mu g5 (mu = 0..3), then g0g1, g0g2, g0g3,
// g1g2, g1g3, g2g3.  Each is a signed permutation of spin components with
// entries +-1 or +-i, stored as a permutation of the 24 reals plus signs.
void gamma_tables(int perm[16][24], int sign[16][24]) {
  struct C { double re, im; };
  C g[16][4][4];
  std::memset(g, 0, sizeof g);
  auto mul = [](C r[4][4], C a[4][4], C b[4][4]) {
    C tmp[4][4];
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) {
        double re = 0, im = 0;
        for (int k = 0; k < 4; ++k) {
          re += a[i][k].re * b[k][j].re - a[i][k].im * b[k][j].im;
          im += a[i][k].re * b[k][j].im + a[i][k].im * b[k][j].re;
        }
        tmp[i][j] = {re, im};
      }
    std::memcpy(r, tmp, sizeof tmp);
  };
  // basis of cvc_linalg.h:10-40
  g[0][0][2].re = -1; g[0][1][3].re = -1; g[0][2][0].re = -1; g[0][3][1].re = -1;
  g[1][0][3].im = -1; g[1][1][2].im = -1; g[1][2][1].im = 1;  g[1][3][0].im = 1;
  g[2][0][3].re = -1; g[2][1][2].re = 1;  g[2][2][1].re = 1;  g[2][3][0].re = -1;
  g[3][0][2].im = -1; g[3][1][3].im = 1;  g[3][2][0].im = 1;  g[3][3][1].im = -1;
  for (int a = 0; a < 4; ++a) g[4][a][a].re = 1;
  mul(g[5], g[0], g[1]);
  mul(g[5], g[5], g[2]);
  mul(g[5], g[5], g[3]);
  for (int mu = 0; mu < 4; ++mu) mul(g[6 + mu], g[mu], g[5]);
  int n = 10;
  for (int a = 0; a < 4; ++a)
    for (int b = a + 1; b < 4; ++b) mul(g[n++], g[a], g[b]);
  for (int k = 0; k < 16; ++k)
    for (int a = 0; a < 4; ++a) {
      int b = 0;
      for (int j = 0; j < 4; ++j)
        if (std::fabs(g[k][a][j].re) + std::fabs(g[k][a][j].im) > 0.5) b = j;
      const C v = g[k][a][b];
      for (int c = 0; c < 3; ++c) {
        const int ra = 2 * (3 * a + c), rb = 2 * (3 * b + c);
        if (std::fabs(v.im) < 0.5) {
          const int s = v.re > 0 ? 1 : -1;
          perm[k][ra] = rb;         sign[k][ra] = s;
          perm[k][ra + 1] = rb + 1; sign[k][ra + 1] = s;
        } else {  // (s i)(re + i im) = -s im + i s re
          const int s = v.im > 0 ? 1 : -1;
          perm[k][ra] = rb + 1; sign[k][ra] = -s;
          perm[k][ra + 1] = rb; sign[k][ra + 1] = s;
        }
      }
    }
}

int geometry_tables(int T, int LX, int LY, int LZ, int *ipt, int *iup, int *idn, int *lexic2eo,
                    int *eo2lexic, int *iseven, int *isevent, int *lexic2eot, int *eot2lexic) {
  if (T <= 0 || LX <= 0 || LY <= 0 || LZ <= 0) return CVCB_ERR_ARG;
  const int V = T * LX * LY * LZ;
  std::vector<int> even(V), even_tzyx(V), lexpt((size_t)(T + 2) * LX * LY * LZ, 0);
  for (int t = 0; t < T; ++t)
    for (int x = 0; x < LX; ++x)
      for (int y = 0; y < LY; ++y)
        for (int z = 0; z < LZ; ++z) {
          const int ix = lex_wrap(t, x, y, z, T, LX, LY, LZ);
          lexpt[((size_t)(t * LX + x) * LY + y) * LZ + z] = ix;
          if (iup) {
            iup[4 * ix + 0] = lex_wrap(t + 1, x, y, z, T, LX, LY, LZ);
            iup[4 * ix + 1] = lex_wrap(t, x + 1, y, z, T, LX, LY, LZ);
            iup[4 * ix + 2] = lex_wrap(t, x, y + 1, z, T, LX, LY, LZ);
            iup[4 * ix + 3] = lex_wrap(t, x, y, z + 1, T, LX, LY, LZ);
          }
          if (idn) {
            idn[4 * ix + 0] = lex_wrap(t - 1, x, y, z, T, LX, LY, LZ);
            idn[4 * ix + 1] = lex_wrap(t, x - 1, y, z, T, LX, LY, LZ);
            idn[4 * ix + 2] = lex_wrap(t, x, y - 1, z, T, LX, LY, LZ);
            idn[4 * ix + 3] = lex_wrap(t, x, y, z - 1, T, LX, LY, LZ);
          }
          even[ix] = ((t + x + y + z) % 2) == 0;
          even_tzyx[((t * LZ + z) * LY + y) * LX + x] = even[ix];
        }
  if (ipt) std::memcpy(ipt, lexpt.data(), lexpt.size() * sizeof(int));
  if (iseven) std::memcpy(iseven, even.data(), (size_t)V * sizeof(int));
  if (isevent) std::memcpy(isevent, even_tzyx.data(), (size_t)V * sizeof(int));
  // Even sites first, each class in increasing lexicographic order
  // (cvc_geometry.c:268-279).
  int ne = 0, no = 0;
  for (int ix = 0; ix < V; ++ix) {
    const int k = even[ix] ? ne++ : V / 2 + no++;
    if (lexic2eo) lexic2eo[ix] = k;
    if (eo2lexic) eo2lexic[k] = ix;
  }
  // Same split, but visiting sites in (t, z, y, x) order (cvc_geometry.c:281-298).
  ne = 0; no = 0;
  int itzyx = 0;
  for (int t = 0; t < T; ++t)
    for (int z = 0; z < LZ; ++z)
      for (int y = 0; y < LY; ++y)
        for (int x = 0; x < LX; ++x, ++itzyx) {
          const int ix = lexpt[((size_t)(t * LX + x) * LY + y) * LZ + z];
          const int k = even_tzyx[itzyx] ? ne++ : V / 2 + no++;
          if (lexic2eot) lexic2eot[ix] = k;
          if (eot2lexic) eot2lexic[k] = ix;
        }
  return CVCB_OK;
}

// ---------------------------------------------------------------------------
// RANLUX, double-precision variant, as published by M. Luescher ("Algorithms
// used in ranlux v3.0", 2001) and implemented in the reference's ranlxd.c
// (plain-C branch, :350-600).  24-bit subtract-with-borrow x_n = x_{n-10} -
// x_{n-24} - c over four interleaved streams, with p = 202 (level 1) or 397
// (level 2) values generated per 12 delivered pairs; a double is built from
// two 24-bit words.  The seeding shift register and the delivery order must
// be the reference's to reproduce its numbers bit for bit.
// ---------------------------------------------------------------------------
class Ranlxd {
 public:
  Ranlxd(int level, int seed) {
    for (int k = 0; k < 96; ++k) nxt_[k] = (k % 4 == 3) ? (k + 5) % 96 : (k + 1) % 96;
    pr_ = level == 2 ? 397 : 202;
    int bits[31];
    int s = seed;
    for (int k = 0; k < 31; ++k) { bits[k] = s % 2; s /= 2; }
    int ib = 0, jb = 18;
    for (int lane = 0; lane < 4; ++lane)
      for (int k = 0; k < 24; ++k) {
        int v = 0;
        for (int l = 0; l < 24; ++l) {
          v = 2 * v + bits[ib];
          bits[ib] = (bits[ib] + bits[jb]) % 2;
          ib = (ib + 1) % 31;
          jb = (jb + 1) % 31;
        }
        if (k % 4 != lane) v = 0xffffff - v;
        w_[4 * k + lane] = v;
      }
    for (int j = 0; j < 4; ++j) carry_[j] = 0;
    ir_ = 0; jr_ = 7; is_ = 91; is_old_ = 0;
  }

  double next() {
    is_ = nxt_[is_];
    if (is_ == is_old_) refill();
    const double eps = std::ldexp(1.0, -24);
    return eps * ((double)w_[is_ + 4] + eps * (double)w_[is_]);
  }

 private:
  // One subtract-with-borrow step on the 8 words of block i (lag block j):
  // words 0..3 are the low halves of four streams, 4..7 the high halves.
  void step(int i, int j) {
    int *wi = w_ + 8 * i;
    const int *wj = w_ + 8 * j;
    for (int lane = 0; lane < 4; ++lane) {
      int d = wj[lane] - wi[lane] - carry_[lane];
      wi[4 + lane] += (d < 0);
      wi[lane] = (d + 0x1000000) & 0xffffff;
      d = wj[4 + lane] - wi[4 + lane];
      carry_[lane] = (d < 0);
      wi[4 + lane] = (d + 0x1000000) & 0xffffff;
    }
  }
  void refill() {
    int i = ir_, j = jr_;
    for (int k = 0; k < pr_; ++k) {
      step(i, j);
      if (++i == 12) i = 0;
      if (++j == 12) j = 0;
    }
    ir_ = (ir_ + pr_ % 12) % 12;
    jr_ = (jr_ + pr_ % 12) % 12;
    is_ = 8 * ir_;
    is_old_ = is_;
  }
  int w_[96];
  int carry_[4];
  int nxt_[96];
  int pr_, ir_, jr_, is_, is_old_;
};

int ranlxd_fill(int level, int seed, double *r, long n) {
  if ((level != 1 && level != 2) || seed <= 0 || !r || n < 0) return CVCB_ERR_ARG;
  Ranlxd g(level, seed);
  for (long k = 0; k < n; ++k) r[k] = g.next();
  return CVCB_OK;
}

// ---------------------------------------------------------------------------
// Gauge generator U = exp(i eps H), H = sum_a w_a lambda_a / 2.
// ---------------------------------------------------------------------------
namespace {
struct M3 { double re[9], im[9]; };

M3 mat_mul(const M3 &a, const M3 &b) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double re = 0, im = 0;
      for (int k = 0; k < 3; ++k) {
        re += a.re[3 * i + k] * b.re[3 * k + j] - a.im[3 * i + k] * b.im[3 * k + j];
        im += a.re[3 * i + k] * b.im[3 * k + j] + a.im[3 * i + k] * b.re[3 * k + j];
      }
      r.re[3 * i + j] = re;
      r.im[3 * i + j] = im;
    }
  return r;
}

// exp(A) by scaling and squaring with a truncated Taylor series (Moler and
// Van Loan, "Nineteen dubious ways to compute the exponential of a matrix",
// method 3): exp(A) = (sum_{k<=16} (A/2^s)^k / k!)^(2^s), s chosen so that
// |A/2^s| <= 1/2, which leaves the truncation far below double rounding.
M3 mat_exp(const M3 &A) {
  double nrm = 0;
  for (int k = 0; k < 9; ++k) nrm += std::fabs(A.re[k]) + std::fabs(A.im[k]);
  int s = 0;
  while (nrm > 0.5) { nrm *= 0.5; ++s; }
  const double scale = std::ldexp(1.0, -s);
  M3 a;
  for (int k = 0; k < 9; ++k) { a.re[k] = A.re[k] * scale; a.im[k] = A.im[k] * scale; }
  M3 sum{}, term{};
  for (int i = 0; i < 3; ++i) { sum.re[4 * i] = 1; term.re[4 * i] = 1; }
  for (int k = 1; k <= 16; ++k) {
    term = mat_mul(term, a);
    for (int q = 0; q < 9; ++q) { term.re[q] /= k; term.im[q] /= k; }
    for (int q = 0; q < 9; ++q) { sum.re[q] += term.re[q]; sum.im[q] += term.im[q]; }
  }
  for (int k = 0; k < s; ++k) sum = mat_mul(sum, sum);
  return sum;
}

// Rows 0, 1 orthonormalised by Gram-Schmidt, row 2 = conj(row0 x row1),
// which makes the matrix exactly special-unitary up to rounding.
void reunitarise(M3 &u) {
  double n0 = 0;
  for (int j = 0; j < 3; ++j) n0 += u.re[j] * u.re[j] + u.im[j] * u.im[j];
  n0 = 1.0 / std::sqrt(n0);
  for (int j = 0; j < 3; ++j) { u.re[j] *= n0; u.im[j] *= n0; }
  double pr = 0, pi = 0;  // <row0, row1>
  for (int j = 0; j < 3; ++j) {
    pr += u.re[j] * u.re[3 + j] + u.im[j] * u.im[3 + j];
    pi += u.re[j] * u.im[3 + j] - u.im[j] * u.re[3 + j];
  }
  for (int j = 0; j < 3; ++j) {
    u.re[3 + j] -= pr * u.re[j] - pi * u.im[j];
    u.im[3 + j] -= pr * u.im[j] + pi * u.re[j];
  }
  double n1 = 0;
  for (int j = 0; j < 3; ++j) n1 += u.re[3 + j] * u.re[3 + j] + u.im[3 + j] * u.im[3 + j];
  n1 = 1.0 / std::sqrt(n1);
  for (int j = 0; j < 3; ++j) { u.re[3 + j] *= n1; u.im[3 + j] *= n1; }
  for (int j = 0; j < 3; ++j) {
    const int a = (j + 1) % 3, b = (j + 2) % 3;
    // (row0 x row1)_j = r0_a r1_b - r0_b r1_a ; row2 = conj of it
    const double cr = (u.re[a] * u.re[3 + b] - u.im[a] * u.im[3 + b]) -
                      (u.re[b] * u.re[3 + a] - u.im[b] * u.im[3 + a]);
    const double ci = (u.re[a] * u.im[3 + b] + u.im[a] * u.re[3 + b]) -
                      (u.re[b] * u.im[3 + a] + u.im[b] * u.re[3 + a]);
    u.re[6 + j] = cr;
    u.im[6 + j] = -ci;
  }
}
}  // namespace

int gauge_random(double *gauge, int T, int LX, int LY, int LZ, double eps, int seed) {
  if (!gauge || T <= 0 || LX <= 0 || LY <= 0 || LZ <= 0 || seed <= 0) return CVCB_ERR_ARG;
  const long V = (long)T * LX * LY * LZ;
  Ranlxd rng(1, seed);
  const double s3 = 1.0 / std::sqrt(3.0);
  for (long ix = 0; ix < V; ++ix)
    for (int mu = 0; mu < 4; ++mu) {
      double w[8];
      for (int k = 0; k < 4; ++k) {  // Box-Muller pairs, as rangauss does
        const double x1 = rng.next();
        const double x2 = rng.next();
        const double r = std::sqrt(-2.0 * std::log(x1));
        w[2 * k] = r * std::cos(2 * M_PI * x2);
        w[2 * k + 1] = r * std::sin(2 * M_PI * x2);
      }
      // H = sum_a w_a lambda_a / 2 (Gell-Mann matrices), A = i eps H
      M3 H{};
      H.re[1] += w[0]; H.re[3] += w[0];                 // lambda_1
      H.im[1] += -w[1]; H.im[3] += w[1];                // lambda_2
      H.re[0] += w[2]; H.re[4] += -w[2];                // lambda_3
      H.re[2] += w[3]; H.re[6] += w[3];                 // lambda_4
      H.im[2] += -w[4]; H.im[6] += w[4];                // lambda_5
      H.re[5] += w[5]; H.re[7] += w[5];                 // lambda_6
      H.im[5] += -w[6]; H.im[7] += w[6];                // lambda_7
      H.re[0] += w[7] * s3; H.re[4] += w[7] * s3; H.re[8] += -2 * w[7] * s3;  // lambda_8
      M3 A;
      for (int q = 0; q < 9; ++q) {
        // i eps (re + i im) / 2 = -eps im / 2 + i eps re / 2
        A.re[q] = -0.5 * eps * H.im[q];
        A.im[q] = 0.5 * eps * H.re[q];
      }
      M3 U = mat_exp(A);
      reunitarise(U);
      double *g = gauge + 18 * (4 * ix + mu);
      for (int q = 0; q < 9; ++q) { g[2 * q] = U.re[q]; g[2 * q + 1] = U.im[q]; }
    }
  return CVCB_OK;
}

}  // namespace cvcb
