// Even/odd (Schur-complement) stencil and vector kernels for the batched
// solver, templated on the storage of spinors and links.
//
// With Q = A + (-1/2) H, A = 1/(2 kappa) + i mu g5 (site-diagonal) and H the
// hopping sum, the odd-site Schur complement is
//   M = A_oo - 1/4 H_oe A_ee^-1 H_eo,   M(mu)^+ = g5 M(-mu) g5,
// and one application of M^+ M is four half-lattice stencil sweeps of the
// single kernel k_eo_hop:
//   out_p = D2 aux_p + D1 ( c [g5] H_pq ([g5] in_q) )
// with D1, D2 site-diagonal operators alpha + i beta g5.
//
// Multi-RHS: the threads that handle the same sites for different
// right-hand sides share each link load (registers within a thread, L1/L2
// across threads), so link traffic per right-hand side falls as 1/N.
#pragma once

#include <cuda_fp16.h>

#include <type_traits>

#include "cvcb_internal.h"
#include "spinor_ops.cuh"

namespace cvcb {

// ---- spinor storage accessors ---------------------------------------------
// Element (rhs r, site j) of a field set; `stride` separates the complex
// components (SoA), `rstride` separates right-hand sides.
struct F64Acc {
  using R = double;
  double2 *p;
  size_t stride, rstride;
  __device__ __forceinline__ Spinor<double> load(int r, int j) const {
    return load_spinor(p + r * rstride, stride, j);
  }
  __device__ __forceinline__ void store(int r, int j, const Spinor<double> &s) const {
    store_spinor(p + r * rstride, stride, j, s);
  }
};

struct F32Acc {
  using R = float;
  float4 *p;
  size_t stride, rstride;
  __device__ __forceinline__ Spinor<float> load(int r, int j) const {
    const float4 *q = p + r * rstride + j;
    Spinor<float> s;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const float4 v = __ldg(q + k * stride);
      s.c[(2 * k) / 3][(2 * k) % 3] = cx(v.x, v.y);
      s.c[(2 * k + 1) / 3][(2 * k + 1) % 3] = cx(v.z, v.w);
    }
    return s;
  }
  // unscaled load (FP32 storage has no per-site scale: nm = 1)
  __device__ __forceinline__ Spinor<float> load_raw(int r, int j, float &nm) const {
    nm = 1.f;
    return load(r, j);
  }
  __device__ __forceinline__ void store(int r, int j, const Spinor<float> &s) const {
    float4 *q = p + r * rstride + j;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const Cx<float> a = s.c[(2 * k) / 3][(2 * k) % 3], b = s.c[(2 * k + 1) / 3][(2 * k + 1) % 3];
      q[k * stride] = make_float4(a.re, a.im, b.re, b.im);
    }
  }
};

// FP16 with one float scale per site: value = half * norm, |half| <= 1.
struct F16Acc {
  using R = float;
  uint4 *p;
  float *norm;
  size_t stride, rstride;
  __device__ __forceinline__ Spinor<float> load(int r, int j) const {
    float nm;
    Spinor<float> s = load_raw(r, j, nm);
#pragma unroll
    for (int c = 0; c < 12; ++c) s.c[c / 3][c % 3] = nm * s.c[c / 3][c % 3];
    return s;
  }
  // the stored halves as floats, and the site's scale (value = half * nm)
  __device__ __forceinline__ Spinor<float> load_raw(int r, int j, float &nm) const {
    const uint4 *q = p + r * rstride + j;
    nm = __ldg(norm + r * stride + j);
    Spinor<float> s;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const uint4 v = __ldg(q + k * stride);
      const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&w[m]));
        const int c = 4 * k + m;
        s.c[c / 3][c % 3] = cx(f.x, f.y);
      }
    }
    return s;
  }
  __device__ __forceinline__ void store(int r, int j, const Spinor<float> &s) const {
    float mx = 0.f;
#pragma unroll
    for (int c = 0; c < 12; ++c)
      mx = fmaxf(mx, fmaxf(fabsf(s.c[c / 3][c % 3].re), fabsf(s.c[c / 3][c % 3].im)));
    // A site whose largest component is below the smallest normal float
    // (far from a point source) is stored as zero: 1/mx would overflow.
    if (!(mx >= 1.17549435e-38f)) mx = 0.f;
    const float inv = mx > 0.f ? 1.f / mx : 0.f;
    uint4 *q = p + r * rstride + j;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      unsigned w[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int c = 4 * k + m;
        __half2 h = __floats2half2_rn(s.c[c / 3][c % 3].re * inv, s.c[c / 3][c % 3].im * inv);
        w[m] = *reinterpret_cast<unsigned *>(&h);
      }
      q[k * stride] = make_uint4(w[0], w[1], w[2], w[3]);
    }
    norm[r * stride + j] = mx;
  }
};

// ---- link accessors ---------------------------------------------------------
// Every accessor returns the phased link W = e^{i theta_mu} U.  The 12-real
// forms store rows 0, 1 of W; since W is SU(3) times a phase, row 2 is
// e^{3 i theta_mu} conj(W_0 x W_1) (ph holds e^{3 i theta_mu}; the product is
// skipped in directions without a phase).
struct L64 {
  using R = double;
  static constexpr bool kPhased = true;
  const double2 *U;
  size_t V;
  double2 ph[4];
  __device__ __forceinline__ Link<double> load(int mu, int j) const { return load_link64(U, V, mu, j); }
};

struct L32f {  // 18 reals, single, phased
  using R = float;
  static constexpr bool kPhased = true;
  const float2 *U;
  size_t V;
  float2 ph[4];
  __device__ __forceinline__ Link<float> load(int mu, int j) const {
    Link<float> L;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const float2 v = __ldg(U + (size_t)(mu * 9 + k) * V + j);
      L.m[k / 3][k % 3] = cx(v.x, v.y);
    }
    return L;
  }
};

__device__ __forceinline__ void apply_row2_phase(Link<float> &L, float2 ph) {
  if (ph.x != 1.f || ph.y != 0.f) {
#pragma unroll
    for (int j = 0; j < 3; ++j) L.m[2][j] = cmul(L.m[2][j], cx(ph.x, ph.y));
  }
}

struct L32c {  // 12 reals, single, phased rows 0 and 1
  using R = float;
  static constexpr bool kPhased = true;
  const float4 *U;
  size_t V;
  float2 ph[4];
  __device__ __forceinline__ Link<float> load(int mu, int j) const {
    Link<float> L;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const float4 v = __ldg(U + (size_t)(mu * 3 + q) * V + j);
      L.m[(2 * q) / 3][(2 * q) % 3] = cx(v.x, v.y);
      L.m[(2 * q + 1) / 3][(2 * q + 1) % 3] = cx(v.z, v.w);
    }
    reconstruct_row2(L);
    apply_row2_phase(L, ph[mu]);
    return L;
  }
};

struct L16c {  // 12 reals, half, phased rows 0 and 1
  using R = float;
  static constexpr bool kPhased = true;
  const uint2 *U;
  size_t V;
  float2 ph[4];
  __device__ __forceinline__ Link<float> load(int mu, int j) const {
    Link<float> L;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const uint2 v = __ldg(U + (size_t)(mu * 3 + q) * V + j);
      const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&v.x));
      const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&v.y));
      L.m[(2 * q) / 3][(2 * q) % 3] = cx(a.x, a.y);
      L.m[(2 * q + 1) / 3][(2 * q + 1) % 3] = cx(b.x, b.y);
    }
    reconstruct_row2(L);
    apply_row2_phase(L, ph[mu]);
    return L;
  }
};

template <typename R>
__device__ __forceinline__ Cx<R> to_cx(double2 v) {
  return cx((R)v.x, (R)v.y);
}
template <typename R>
__device__ __forceinline__ Cx<R> to_cx(float2 v) {
  return cx((R)v.x, (R)v.y);
}

template <typename R>
__device__ __forceinline__ HalfSpinor<R> cscale(const HalfSpinor<R> &h, Cx<R> z) {
  HalfSpinor<R> o;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) o.c[a][c] = cmul(h.c[a][c], z);
  return o;
}

// out = (alpha + i beta g5) v
template <typename R>
__device__ __forceinline__ Spinor<R> diag_op(R alpha, R beta, const Spinor<R> &v) {
  Spinor<R> o;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const R b = s < 2 ? beta : -beta;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const Cx<R> x = v.c[s][c];
      o.c[s][c] = cx(alpha * x.re - b * x.im, alpha * x.im + b * x.re);
    }
  }
  return o;
}

template <typename R>
__device__ __forceinline__ void g5_inplace(Spinor<R> &v) {
#pragma unroll
  for (int s = 2; s < 4; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) v.c[s][c] = cx(-v.c[s][c].re, -v.c[s][c].im);
}

struct EoGeom {
  Geom g;
  int p;  // output parity
};

// Per-call arguments of the stencil kernel.
template <class SF, class LF>
struct HopArgs {
  SF out, in, aux;
  LF links;
  EoGeom eg;
  int nrhs;
  const int *done;  // per right-hand side, may be null
  double d1a, d1b;  // D1 = d1a + i d1b g5
  double d2a, d2b;  // D2 = d2a + i d2b g5
  double c;         // hop coefficient
  // optional (k_eo_hop_x2 only): per-warp partial sums of |out|^2,
  // dot_part[rhs * dot_np + warp], warp = site block * (blockDim.x / 32) +
  // warp in the row; null = off
  double *dot_part;
  int dot_np;
  // optional (k_eo_hop_pt with the residual update): instead of storing
  // out, r -= alpha[rhs] * out on the field set `rup` (and dot_part gets
  // |r|^2)
  SF rup;
  const double *alpha;
  // k_eo_hop_ptb: set to 1 if a staged copy did not complete in time
  int *err;
};

// |a|^2 of one site, accumulated in FP64
__device__ __forceinline__ double norm2_site(const Spinor<float> &a) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      s += (double)a.c[k][c].re * a.c[k][c].re + (double)a.c[k][c].im * a.c[k][c].im;
  return s;
}

// Thread mapping: each thread handles one output site for NR right-hand
// sides; blockDim.y groups of NR share the block.  The link of every
// direction is loaded (and, for 12-real storage, rebuilt and multiplied by
// its phase) once per thread and applied to all NR spinors from registers.
// Grid: blockIdx.x = block of rhs groups (fastest), blockIdx.y (and a stride
// loop) = block of sites, so consecutive blocks share their sites' links in
// L2.
constexpr int kHopMaxThreads = 256;

template <typename R, class LF>
__device__ __forceinline__ Link<R> phased_link(const LF &lk, int mu, int j) {
  Link<R> W = lk.load(mu, j);
  if (!LF::kPhased) {
    const Cx<R> ph = cx((R)lk.ph[mu].x, (R)lk.ph[mu].y);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) W.m[a][b] = cmul(W.m[a][b], ph);
  }
  return W;
}

// Launch bounds: (256 threads, min resident blocks) caps registers at
// 65536 / (256 * blocks).  Measured at 24^3x48, 12 rhs: the FP32-arithmetic
// sweep with one rhs per thread runs best at 80 registers (3 blocks: 1.23 ms
// per M^+M, with a few spills to L1); a bound of 1 block lets the compiler
// take 176 registers and costs 46 %; 4 blocks (64 registers) spills too
// much.  More rhs per thread need more registers.  FP64 sweeps keep the
// plain thread bound (the compiler then uses about 150 registers).
template <int NR>
struct HopMinBlocks {
  static constexpr int value = NR == 1 ? 3 : NR <= 3 ? 2 : 1;
};

template <class SF, class LF, int NR, bool G5IN, bool G5HOP, bool AUX>
__device__ __forceinline__ void eo_hop_body(const HopArgs<SF, LF> &A) {
  using R = typename SF::R;
  const int r0 = (blockIdx.x * blockDim.y + threadIdx.y) * NR;
  const Geom &g = A.eg.g;
  if (r0 >= A.nrhs) return;
  bool act[NR];
  bool any = false;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    act[k] = r0 + k < A.nrhs && !(A.done && A.done[r0 + k]);
    any = any || act[k];
  }
  if (!any) return;
  const int p = A.eg.p;
  const int qoff = (1 - p) * g.Vh;
  for (int sb = blockIdx.y; sb * (int)blockDim.x < g.Vh; sb += gridDim.y) {
    const int i = sb * blockDim.x + threadIdx.x;
    if (i >= g.Vh) return;
    const SiteCoord cd = site_coord(g, p, i);
    const int self = p * g.Vh + i;

    Spinor<R> acc[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k)
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[k].c[s][c] = cx((R)0, (R)0);

#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
      {  // backward: (1 + g_mu) U_mu(x-mu)^+ in(x-mu)
        const int j = nb_lex(g, cd, mu, -1) >> 1;
        const Link<R> W = phased_link<R>(A.links, mu, qoff + j);
#pragma unroll
        for (int k = 0; k < NR; ++k) {
          if (!act[k]) continue;
          Spinor<R> f = A.in.load(r0 + k, j);
          if (G5IN) g5_inplace(f);
          accum_recon(mu, +1, acc[k], link_dag_mul(W, project(mu, +1, f)));
        }
      }
      {  // forward: (1 - g_mu) U_mu(x) in(x+mu)
        const int j = nb_lex(g, cd, mu, +1) >> 1;
        const Link<R> W = phased_link<R>(A.links, mu, self);
#pragma unroll
        for (int k = 0; k < NR; ++k) {
          if (!act[k]) continue;
          Spinor<R> f = A.in.load(r0 + k, j);
          if (G5IN) g5_inplace(f);
          accum_recon(mu, -1, acc[k], link_mul(W, project(mu, -1, f)));
        }
      }
    }
    const R c = (R)A.c;
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      if (!act[k]) continue;
      if (G5HOP) g5_inplace(acc[k]);
      Spinor<R> o;
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int q = 0; q < 3; ++q) o.c[s][q] = c * acc[k].c[s][q];
      o = diag_op((R)A.d1a, (R)A.d1b, o);
      if (AUX) {
        const Spinor<R> x = diag_op((R)A.d2a, (R)A.d2b, A.aux.load(r0 + k, i));
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
          for (int q = 0; q < 3; ++q) o.c[s][q] = o.c[s][q] + x.c[s][q];
      }
      A.out.store(r0 + k, i, o);
    }
  }
}

template <class SF, class LF, int NR, bool G5IN, bool G5HOP, bool AUX>
__global__ void __launch_bounds__(kHopMaxThreads, HopMinBlocks<NR>::value)
    k_eo_hop(HopArgs<SF, LF> A) {
  eo_hop_body<SF, LF, NR, G5IN, G5HOP, AUX>(A);
}

template <class LF, bool G5IN, bool G5HOP, bool AUX>
__global__ void __launch_bounds__(kHopMaxThreads) k_eo_hop64(HopArgs<F64Acc, LF> A) {
  eo_hop_body<F64Acc, LF, 1, G5IN, G5HOP, AUX>(A);
}

// ---- two right-hand sides per thread in packed FP32x2 arithmetic -----------
// Lane x of every float2 belongs to rhs a, lane y to rhs b.  The link is the
// same for both, so each complex multiply-add of the link product is two
// packed FMAs (one instruction per two rhs); the link rebuild, the neighbour
// indices and the addresses are shared by the pair as well.
struct CP {  // complex pair: re = (a.re, b.re), im = (a.im, b.im)
  float2 re, im;
};
__device__ __forceinline__ float2 bc(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 neg2(float2 v) { return make_float2(-v.x, -v.y); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, neg2(b)); }

struct HalfPair {
  CP c[2][3];
};
struct SpinorPair {
  CP c[4][3];
};

__device__ __forceinline__ HalfPair pair_half(const HalfSpinor<float> &a, const HalfSpinor<float> &b) {
  HalfPair h;
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      h.c[s][c].re = make_float2(a.c[s][c].re, b.c[s][c].re);
      h.c[s][c].im = make_float2(a.c[s][c].im, b.c[s][c].im);
    }
  return h;
}

// Per-site scales of FP16+norm storage, applied after the projection to the
// 12 values of the half-spinor pair (packed) instead of 2 x 24 components;
// FP32 storage has none.
template <class SF>
__device__ __forceinline__ HalfPair scale_pair(const HalfPair &h, float na, float nb) {
  if constexpr (std::is_same<SF, F32Acc>::value) {
    return h;
  } else {
    const float2 n = make_float2(na, nb);
    HalfPair o;
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        o.c[s][c].re = __fmul2_rn(n, h.c[s][c].re);
        o.c[s][c].im = __fmul2_rn(n, h.c[s][c].im);
      }
    return o;
  }
}

// u = W h (dag = false) or W^+ h (dag = true), both rhs at once
template <bool DAG>
__device__ __forceinline__ HalfPair link_mul_pair(const Link<float> &W, const HalfPair &h) {
  HalfPair u;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    // row i of W (or of W^+): w_j = W[i][j] or conj(W[j][i])
    float wr[3], wi[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      wr[j] = DAG ? W.m[j][i].re : W.m[i][j].re;
      wi[j] = DAG ? -W.m[j][i].im : W.m[i][j].im;
    }
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      float2 re = __fmul2_rn(bc(wr[0]), h.c[s][0].re);
      float2 im = __fmul2_rn(bc(wr[0]), h.c[s][0].im);
      re = __ffma2_rn(bc(-wi[0]), h.c[s][0].im, re);
      im = __ffma2_rn(bc(wi[0]), h.c[s][0].re, im);
#pragma unroll
      for (int j = 1; j < 3; ++j) {
        re = __ffma2_rn(bc(wr[j]), h.c[s][j].re, re);
        im = __ffma2_rn(bc(wr[j]), h.c[s][j].im, im);
        re = __ffma2_rn(bc(-wi[j]), h.c[s][j].im, re);
        im = __ffma2_rn(bc(wi[j]), h.c[s][j].re, im);
      }
      u.c[s][i].re = re;
      u.c[s][i].im = im;
    }
  }
  return u;
}

// acc += (1 + s g_mu)-reconstruction of u, both rhs (see accum_recon)
__device__ __forceinline__ void accum_recon_pair(int mu, int s, SpinorPair &acc, const HalfPair &u) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    acc.c[0][c].re = add2(acc.c[0][c].re, u.c[0][c].re);
    acc.c[0][c].im = add2(acc.c[0][c].im, u.c[0][c].im);
    acc.c[1][c].re = add2(acc.c[1][c].re, u.c[1][c].re);
    acc.c[1][c].im = add2(acc.c[1][c].im, u.c[1][c].im);
    // spins 2, 3: +-u or +-i u of spins 0, 1; i (x + i y) = -y + i x
    switch (mu) {
      case 0:  // r2 = -s u0, r3 = -s u1
        if (s > 0) {
          acc.c[2][c].re = sub2(acc.c[2][c].re, u.c[0][c].re);
          acc.c[2][c].im = sub2(acc.c[2][c].im, u.c[0][c].im);
          acc.c[3][c].re = sub2(acc.c[3][c].re, u.c[1][c].re);
          acc.c[3][c].im = sub2(acc.c[3][c].im, u.c[1][c].im);
        } else {
          acc.c[2][c].re = add2(acc.c[2][c].re, u.c[0][c].re);
          acc.c[2][c].im = add2(acc.c[2][c].im, u.c[0][c].im);
          acc.c[3][c].re = add2(acc.c[3][c].re, u.c[1][c].re);
          acc.c[3][c].im = add2(acc.c[3][c].im, u.c[1][c].im);
        }
        break;
      case 1:  // r2 = s i u1, r3 = s i u0
        if (s > 0) {
          acc.c[2][c].re = sub2(acc.c[2][c].re, u.c[1][c].im);
          acc.c[2][c].im = add2(acc.c[2][c].im, u.c[1][c].re);
          acc.c[3][c].re = sub2(acc.c[3][c].re, u.c[0][c].im);
          acc.c[3][c].im = add2(acc.c[3][c].im, u.c[0][c].re);
        } else {
          acc.c[2][c].re = add2(acc.c[2][c].re, u.c[1][c].im);
          acc.c[2][c].im = sub2(acc.c[2][c].im, u.c[1][c].re);
          acc.c[3][c].re = add2(acc.c[3][c].re, u.c[0][c].im);
          acc.c[3][c].im = sub2(acc.c[3][c].im, u.c[0][c].re);
        }
        break;
      case 2:  // r2 = s u1, r3 = -s u0
        if (s > 0) {
          acc.c[2][c].re = add2(acc.c[2][c].re, u.c[1][c].re);
          acc.c[2][c].im = add2(acc.c[2][c].im, u.c[1][c].im);
          acc.c[3][c].re = sub2(acc.c[3][c].re, u.c[0][c].re);
          acc.c[3][c].im = sub2(acc.c[3][c].im, u.c[0][c].im);
        } else {
          acc.c[2][c].re = sub2(acc.c[2][c].re, u.c[1][c].re);
          acc.c[2][c].im = sub2(acc.c[2][c].im, u.c[1][c].im);
          acc.c[3][c].re = add2(acc.c[3][c].re, u.c[0][c].re);
          acc.c[3][c].im = add2(acc.c[3][c].im, u.c[0][c].im);
        }
        break;
      default:  // r2 = s i u0, r3 = -s i u1
        if (s > 0) {
          acc.c[2][c].re = sub2(acc.c[2][c].re, u.c[0][c].im);
          acc.c[2][c].im = add2(acc.c[2][c].im, u.c[0][c].re);
          acc.c[3][c].re = add2(acc.c[3][c].re, u.c[1][c].im);
          acc.c[3][c].im = sub2(acc.c[3][c].im, u.c[1][c].re);
        } else {
          acc.c[2][c].re = add2(acc.c[2][c].re, u.c[0][c].im);
          acc.c[2][c].im = sub2(acc.c[2][c].im, u.c[0][c].re);
          acc.c[3][c].re = sub2(acc.c[3][c].re, u.c[1][c].im);
          acc.c[3][c].im = add2(acc.c[3][c].im, u.c[1][c].re);
        }
        break;
    }
  }
}

// Packed-pair stencil: thread = (site, rhs pair); same sweep as k_eo_hop.
// The aux term is loaded after the neighbours: starting the accumulator from
// it instead (one load fewer at the end) measured 2.5 % slower in FP32.
template <class SF, class LF, bool G5IN, bool G5HOP, bool AUX>
__global__ void __launch_bounds__(kHopMaxThreads, 2) k_eo_hop_x2(HopArgs<SF, LF> A) {
  static_assert(sizeof(typename SF::R) == 4, "packed pairs need FP32 arithmetic");
  const int ra = (blockIdx.x * blockDim.y + threadIdx.y) * 2;
  if (ra >= A.nrhs) return;
  const bool act_a = !(A.done && A.done[ra]);
  const bool has_b = ra + 1 < A.nrhs;
  const bool act_b = has_b && !(A.done && A.done[ra + 1]);
  if (!act_a && !act_b) return;
  const int rb = has_b ? ra + 1 : ra;  // a lone last rhs runs twice, stores once
  const Geom &g = A.eg.g;
  const int p = A.eg.p;
  const int qoff = (1 - p) * g.Vh;
  for (int sb = blockIdx.y; sb * (int)blockDim.x < g.Vh; sb += gridDim.y) {
    const int i = sb * blockDim.x + threadIdx.x;
    double da = 0.0, db = 0.0;  // |out|^2 of this site, rhs a and b
    if (i < g.Vh) {
    const SiteCoord cd = site_coord(g, p, i);
    SpinorPair acc;
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) acc.c[s][c].re = acc.c[s][c].im = make_float2(0.f, 0.f);
    // Directions in the order z, y, x, t: the z neighbours of a block's
    // sites are its own index range of the other parity, and the y neighbours
    // overlap it, so the loads of z+, y- and y+ find most of their lines in
    // L1 right after z-.  1.085 ms per M^+M at 24^3x48, 12 rhs, against
    // 1.129 ms in the order t, x, y, z, where the t and x loads evict the
    // block's lines between the y and z loads.  (The FP64 staged sweep is
    // slower in this order and keeps t, x, y, z.)
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int mu = 3 - m;
      {  // backward: (1 + g_mu) U_mu(x-mu)^+ in(x-mu)
        const int j = nb_lex(g, cd, mu, -1) >> 1;
        const Link<float> W = phased_link<float>(A.links, mu, qoff + j);
        float na, nb;
        Spinor<float> fa = A.in.load_raw(ra, j, na), fb = A.in.load_raw(rb, j, nb);
        if (G5IN) {
          g5_inplace(fa);
          g5_inplace(fb);
        }
        const HalfPair h = scale_pair<SF>(pair_half(project(mu, +1, fa), project(mu, +1, fb)), na, nb);
        accum_recon_pair(mu, +1, acc, link_mul_pair<true>(W, h));
      }
      {  // forward: (1 - g_mu) U_mu(x) in(x+mu)
        const int j = nb_lex(g, cd, mu, +1) >> 1;
        const Link<float> W = phased_link<float>(A.links, mu, p * g.Vh + i);
        float na, nb;
        Spinor<float> fa = A.in.load_raw(ra, j, na), fb = A.in.load_raw(rb, j, nb);
        if (G5IN) {
          g5_inplace(fa);
          g5_inplace(fb);
        }
        const HalfPair h = scale_pair<SF>(pair_half(project(mu, -1, fa), project(mu, -1, fb)), na, nb);
        accum_recon_pair(mu, -1, acc, link_mul_pair<false>(W, h));
      }
    }
    const float c = (float)A.c;
#pragma unroll
    for (int lane = 0; lane < 2; ++lane) {
      if (lane == 0 ? !act_a : !act_b) continue;
      const int r = lane == 0 ? ra : rb;
      Spinor<float> o;
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const CP v = acc.c[s][q];
          o.c[s][q] = lane == 0 ? cx(c * v.re.x, c * v.im.x) : cx(c * v.re.y, c * v.im.y);
        }
      if (G5HOP) g5_inplace(o);
      o = diag_op((float)A.d1a, (float)A.d1b, o);
      if (AUX) {
        const Spinor<float> x = diag_op((float)A.d2a, (float)A.d2b, A.aux.load(r, i));
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
          for (int q = 0; q < 3; ++q) o.c[s][q] = o.c[s][q] + x.c[s][q];
      }
      if (A.dot_part) (lane == 0 ? da : db) = norm2_site(o);
      A.out.store(r, i, o);
    }
    }  // i < Vh
    if (A.dot_part) {  // the whole warp is here: one row, warp-aligned block width
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        da += __shfl_down_sync(0xffffffffu, da, o);
        db += __shfl_down_sync(0xffffffffu, db, o);
      }
      if ((threadIdx.x & 31) == 0) {
        const int w = sb * (blockDim.x >> 5) + (threadIdx.x >> 5);
        A.dot_part[(size_t)ra * A.dot_np + w] = da;
        if (has_b) A.dot_part[(size_t)rb * A.dot_np + w] = db;
      }
    }
  }
}

// Shared-memory staged variant, one rhs per thread, blockDim.y rhs rows per
// block: the 8 links of each site (phased, 12-real forms rebuilt) and its 8
// neighbour indices are produced once per block -- thread row ty builds link
// slots ty, ty + blockDim.y, ... -- and read from shared memory by every rhs
// row.  Link traffic from L2 and the link arithmetic per rhs fall by the
// number of rows.  Shared memory: 8 * 9 * blockDim.x complex + 8 * blockDim.x
// ints (slot d = 2 mu + 1 forward, 2 mu backward).
template <typename R>
__host__ __device__ constexpr size_t staged_smem_bytes(int bx) {
  return (size_t)8 * 9 * bx * sizeof(Cx<R>) + (size_t)8 * bx * sizeof(int);
}

template <class SF, class LF, bool G5IN, bool G5HOP, bool AUX>
__device__ __forceinline__ void eo_hop_staged_body(const HopArgs<SF, LF> &A) {
  using R = typename SF::R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int bx = blockDim.x, tx = threadIdx.x, ty = threadIdx.y;
  Cx<R> *sl = reinterpret_cast<Cx<R> *>(smem_raw);  // [8][9][bx]
  int *snb = reinterpret_cast<int *>(smem_raw + (size_t)8 * 9 * bx * sizeof(Cx<R>));  // [8][bx]
  const int r = blockIdx.x * blockDim.y + ty;
  const bool act = r < A.nrhs && !(A.done && A.done[r]);
  if (!__syncthreads_or(act)) return;  // uniform: no row of this block is active
  const Geom &g = A.eg.g;
  const int p = A.eg.p;
  const int qoff = (1 - p) * g.Vh;
  for (int sb = blockIdx.y; sb * bx < g.Vh; sb += gridDim.y) {
    const int i = sb * bx + tx;
    const bool valid = i < g.Vh;
    if (valid) {
      const SiteCoord cd = site_coord(g, p, i);
      for (int d = ty; d < 8; d += blockDim.y) {
        const int mu = d >> 1;
        const bool fwd = d & 1;
        const int j = nb_lex(g, cd, mu, fwd ? +1 : -1) >> 1;
        const Link<R> W = phased_link<R>(A.links, mu, fwd ? p * g.Vh + i : qoff + j);
#pragma unroll
        for (int k = 0; k < 9; ++k) sl[(d * 9 + k) * bx + tx] = W.m[k / 3][k % 3];
        snb[d * bx + tx] = j;
      }
    }
    __syncthreads();
    if (valid && act) {
      Spinor<R> acc;
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc.c[s][c] = cx((R)0, (R)0);
#pragma unroll
      for (int mu = 0; mu < 4; ++mu) {
#pragma unroll
        for (int fwd = 0; fwd < 2; ++fwd) {
          const int d = 2 * mu + fwd;
          Link<R> W;
#pragma unroll
          for (int k = 0; k < 9; ++k) W.m[k / 3][k % 3] = sl[(d * 9 + k) * bx + tx];
          Spinor<R> f = A.in.load(r, snb[d * bx + tx]);
          if (G5IN) g5_inplace(f);
          if (fwd)  // (1 - g_mu) U_mu(x) in(x+mu)
            accum_recon(mu, -1, acc, link_mul(W, project(mu, -1, f)));
          else  // (1 + g_mu) U_mu(x-mu)^+ in(x-mu)
            accum_recon(mu, +1, acc, link_dag_mul(W, project(mu, +1, f)));
        }
      }
      if (G5HOP) g5_inplace(acc);
      const R c = (R)A.c;
      Spinor<R> o;
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int q = 0; q < 3; ++q) o.c[s][q] = c * acc.c[s][q];
      o = diag_op((R)A.d1a, (R)A.d1b, o);
      if (AUX) {
        const Spinor<R> x = diag_op((R)A.d2a, (R)A.d2b, A.aux.load(r, i));
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
          for (int q = 0; q < 3; ++q) o.c[s][q] = o.c[s][q] + x.c[s][q];
      }
      A.out.store(r, i, o);
    }
    __syncthreads();  // the next site block overwrites the staged links
  }
}

// FP32 arithmetic: capped at 128 registers (2 blocks of 256).  FP64: at most
// 128 threads per block and 128 registers (4 blocks): 0.58 ms per sweep of
// 12 rhs at 24^3x48, against 0.65 ms with the compiler's own choice (about
// 150 registers) and 0.61-0.71 ms at 3 or 2 blocks.
template <class SF, class LF, bool G5IN, bool G5HOP, bool AUX>
__global__ void __launch_bounds__(kHopMaxThreads, 2) k_eo_hop_staged(HopArgs<SF, LF> A) {
  eo_hop_staged_body<SF, LF, G5IN, G5HOP, AUX>(A);
}
template <class LF, bool G5IN, bool G5HOP, bool AUX>
__global__ void __launch_bounds__(128, 4) k_eo_hop_staged64(HopArgs<F64Acc, LF> A) {
  eo_hop_staged_body<F64Acc, LF, G5IN, G5HOP, AUX>(A);
}

}  // namespace cvcb
