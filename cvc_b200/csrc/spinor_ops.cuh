// Register-level spinor algebra shared by the stencil kernels.
//
// Gamma basis (the reference's, cvc_linalg.h:10-40):
//   g0 = [[0,0,-1,0],[0,0,0,-1],[-1,0,0,0],[0,-1,0,0]]
//   g1 = [[0,0,0,-i],[0,0,-i,0],[0,i,0,0],[i,0,0,0]]
//   g2 = [[0,0,0,-1],[0,0,1,0],[0,1,0,0],[-1,0,0,0]]
//   g3 = [[0,0,-i,0],[0,0,0,i],[i,0,0,0],[0,-i,0,0]]
//   g5 = diag(1,1,-1,-1)
// (1 -+ g_mu) has rank 2: spins 0,1 of the projected spinor determine spins
// 2,3.  The stencil therefore multiplies only a half spinor h (2 spins x 3
// colours) by the link and rebuilds spins 2,3 afterwards:
//   mu  (1 + s g_mu), s = -1 (forward hop) or +1 (backward hop)
//   0   h0 = f0 - s f2     h1 = f1 - s f3     r2 = -s h0     r3 = -s h1
//   1   h0 = f0 - s i f3   h1 = f1 - s i f2   r2 =  s i h1   r3 =  s i h0
//   2   h0 = f0 - s f3     h1 = f1 + s f2     r2 =  s h1     r3 = -s h0
//   3   h0 = f0 - s i f2   h1 = f1 + s i f3   r2 =  s i h0   r3 = -s i h1
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace cvcb {

template <typename R>
struct Cx {
  R re, im;
};

template <typename R>
__device__ __forceinline__ Cx<R> cx(R a, R b) {
  Cx<R> c;
  c.re = a;
  c.im = b;
  return c;
}
template <typename R>
__device__ __forceinline__ Cx<R> operator+(Cx<R> a, Cx<R> b) { return cx(a.re + b.re, a.im + b.im); }
template <typename R>
__device__ __forceinline__ Cx<R> operator-(Cx<R> a, Cx<R> b) { return cx(a.re - b.re, a.im - b.im); }
template <typename R>
__device__ __forceinline__ Cx<R> operator*(R s, Cx<R> a) { return cx(s * a.re, s * a.im); }
// i * a
template <typename R>
__device__ __forceinline__ Cx<R> mul_i(Cx<R> a) { return cx(-a.im, a.re); }
// a * b
template <typename R>
__device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b) {
  return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
// conj(a) * b
template <typename R>
__device__ __forceinline__ Cx<R> cmulc(Cx<R> a, Cx<R> b) {
  return cx(a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re);
}
// acc += a * b
template <typename R>
__device__ __forceinline__ void cfma(Cx<R> &acc, Cx<R> a, Cx<R> b) {
  acc.re = fma(a.re, b.re, acc.re);
  acc.re = fma(-a.im, b.im, acc.re);
  acc.im = fma(a.re, b.im, acc.im);
  acc.im = fma(a.im, b.re, acc.im);
}
// acc += conj(a) * b
template <typename R>
__device__ __forceinline__ void cfmac(Cx<R> &acc, Cx<R> a, Cx<R> b) {
  acc.re = fma(a.re, b.re, acc.re);
  acc.re = fma(a.im, b.im, acc.re);
  acc.im = fma(a.re, b.im, acc.im);
  acc.im = fma(-a.im, b.re, acc.im);
}

template <typename R>
struct Spinor {
  Cx<R> c[4][3];
};
template <typename R>
struct HalfSpinor {
  Cx<R> c[2][3];
};
template <typename R>
struct Link {
  Cx<R> m[3][3];
};

// s * z for s = +-1 and z = a or i*a, chosen at compile time by the caller.
template <typename R>
__device__ __forceinline__ Cx<R> sgn(int s, Cx<R> a) {
  return s > 0 ? a : cx(-a.re, -a.im);
}

template <typename R>
__device__ __forceinline__ HalfSpinor<R> project(int mu, int s, const Spinor<R> &f) {
  HalfSpinor<R> h;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    switch (mu) {
      case 0:
        h.c[0][c] = f.c[0][c] + sgn(-s, f.c[2][c]);
        h.c[1][c] = f.c[1][c] + sgn(-s, f.c[3][c]);
        break;
      case 1:
        h.c[0][c] = f.c[0][c] + sgn(-s, mul_i(f.c[3][c]));
        h.c[1][c] = f.c[1][c] + sgn(-s, mul_i(f.c[2][c]));
        break;
      case 2:
        h.c[0][c] = f.c[0][c] + sgn(-s, f.c[3][c]);
        h.c[1][c] = f.c[1][c] + sgn(s, f.c[2][c]);
        break;
      default:
        h.c[0][c] = f.c[0][c] + sgn(-s, mul_i(f.c[2][c]));
        h.c[1][c] = f.c[1][c] + sgn(s, mul_i(f.c[3][c]));
        break;
    }
  }
  return h;
}

// acc += (1 + s g_mu)-reconstruction of the half spinor u.
template <typename R>
__device__ __forceinline__ void accum_recon(int mu, int s, Spinor<R> &acc, const HalfSpinor<R> &u) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    acc.c[0][c] = acc.c[0][c] + u.c[0][c];
    acc.c[1][c] = acc.c[1][c] + u.c[1][c];
    switch (mu) {
      case 0:
        acc.c[2][c] = acc.c[2][c] + sgn(-s, u.c[0][c]);
        acc.c[3][c] = acc.c[3][c] + sgn(-s, u.c[1][c]);
        break;
      case 1:
        acc.c[2][c] = acc.c[2][c] + sgn(s, mul_i(u.c[1][c]));
        acc.c[3][c] = acc.c[3][c] + sgn(s, mul_i(u.c[0][c]));
        break;
      case 2:
        acc.c[2][c] = acc.c[2][c] + sgn(s, u.c[1][c]);
        acc.c[3][c] = acc.c[3][c] + sgn(-s, u.c[0][c]);
        break;
      default:
        acc.c[2][c] = acc.c[2][c] + sgn(s, mul_i(u.c[0][c]));
        acc.c[3][c] = acc.c[3][c] + sgn(-s, mul_i(u.c[1][c]));
        break;
    }
  }
}

// u = U h (each of the two spin rows).
template <typename R>
__device__ __forceinline__ HalfSpinor<R> link_mul(const Link<R> &U, const HalfSpinor<R> &h) {
  HalfSpinor<R> u;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      Cx<R> acc = cmul(U.m[i][0], h.c[a][0]);
      cfma(acc, U.m[i][1], h.c[a][1]);
      cfma(acc, U.m[i][2], h.c[a][2]);
      u.c[a][i] = acc;
    }
  return u;
}

// u = U^dagger h.
template <typename R>
__device__ __forceinline__ HalfSpinor<R> link_dag_mul(const Link<R> &U, const HalfSpinor<R> &h) {
  HalfSpinor<R> u;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      Cx<R> acc = cmulc(U.m[0][i], h.c[a][0]);
      cfmac(acc, U.m[1][i], h.c[a][1]);
      cfmac(acc, U.m[2][i], h.c[a][2]);
      u.c[a][i] = acc;
    }
  return u;
}

// Third row of an SU(3) matrix from the first two: row2 = conj(row0 x row1).
template <typename R>
__device__ __forceinline__ void reconstruct_row2(Link<R> &U) {
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int a = (j + 1) % 3, b = (j + 2) % 3;
    Cx<R> v = cmul(U.m[0][a], U.m[1][b]) - cmul(U.m[0][b], U.m[1][a]);
    U.m[2][j] = cx(v.re, -v.im);
  }
}

// ---- loads / stores of the device layouts ---------------------------------
__device__ __forceinline__ Spinor<double> load_spinor(const double2 *__restrict__ f, size_t stride,
                                                      int j) {
  Spinor<double> s;
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    const double2 v = __ldg(f + k * stride + j);
    s.c[k / 3][k % 3] = cx(v.x, v.y);
  }
  return s;
}

__device__ __forceinline__ void store_spinor(double2 *__restrict__ f, size_t stride, int j,
                                             const Spinor<double> &s) {
#pragma unroll
  for (int k = 0; k < 12; ++k) f[k * stride + j] = make_double2(s.c[k / 3][k % 3].re, s.c[k / 3][k % 3].im);
}

__device__ __forceinline__ Link<double> load_link64(const double2 *__restrict__ U, size_t V, int mu,
                                                    int j) {
  Link<double> L;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double2 v = __ldg(U + (size_t)(mu * 9 + k) * V + j);
    L.m[k / 3][k % 3] = cx(v.x, v.y);
  }
  return L;
}

}  // namespace cvcb
