// Pair-tiled storage and its kernels for the FP32 inner iterations of the
// batched solver.
//
// Right-hand sides 2q and 2q+1 ("pair q") are stored interleaved per complex
// spin-colour component, so that 16 bytes hold both right-hand sides of a
// component in the register order of the packed FP32x2 instructions
// (FFMA2/FADD2/FMUL2), and two components of a site are adjacent:
//   float4 P[pair][tile = j / 32][component pair k / 2][j % 32][k % 2]
//   float4 = (re of rhs 2q, re of rhs 2q+1, im of rhs 2q, im of rhs 2q+1)
// One 256-bit load per thread reads components 2m and 2m+1 of its site; a
// warp reads 1 KB contiguous; the 6 component pairs of a site lie at fixed
// offsets (m * 1 KB) from one address, so a neighbour costs one address
// computation and six loads.  Links are tiled by 32 even/odd link indices
// too, with 18 reals (phase multiplied in; nothing to rebuild) or 12 reals
// (rows 0, 1; row 2 rebuilt in registers).
//
// Compared with per-rhs structure-of-arrays storage packed into FP32x2 pairs
// after the loads (k_eo_hop_x2), the stencil needs no register moves to form
// the pairs, projects and reconstructs both right-hand sides with packed
// additions, and applies the site-diagonal epilogue in packed arithmetic.
#pragma once

#include "eo_kernels.cuh"

namespace cvcb {

constexpr int kTile = 32;

__device__ __forceinline__ CP cp_of(float4 v) {
  CP c;
  c.re = make_float2(v.x, v.y);
  c.im = make_float2(v.z, v.w);
  return c;
}
__device__ __forceinline__ float4 f4_of(const CP &c) {
  return make_float4(c.re.x, c.re.y, c.im.x, c.im.y);
}

// 256-bit global accesses (sm_100): two float4 from 32-byte-aligned
// addresses in one instruction.  The asm statements are volatile with a
// memory clobber so that the compiler keeps them in order with the other
// memory accesses of the thread (a field is often read and then written by
// the same thread).
__device__ __forceinline__ void ldg_v8(const float4 *q, float4 &a, float4 &b) {
  asm volatile("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z),
                 "=f"(b.w)
               : "l"(q)
               : "memory");
}
__device__ __forceinline__ void stg_v8(float4 *q, const float4 &a, const float4 &b) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(q), "f"(a.x),
               "f"(a.y), "f"(a.z), "f"(a.w), "f"(b.x), "f"(b.y), "f"(b.z), "f"(b.w)
               : "memory");
}

// FP32 pair-tiled field set: pair pr, half-lattice site j.  Within a tile of
// 32 sites, component k of the site in position l sits at float4
// comp(k) + 2 l = (k / 2) * 64 + k % 2 + 2 l: components 2m and 2m + 1 of a
// site are 32 contiguous bytes, read or written with one 256-bit access
// (a warp: 1 KB contiguous), six per site and rhs pair.
struct P32 {
  using R = float;
  float4 *p;
  size_t pstride;  // float4 per pair (tiles x 12 x 32)
  __device__ __forceinline__ static constexpr int comp(int k) { return (k >> 1) * (2 * kTile) + (k & 1); }
  // the site's slot: component k at at(pr, j) + comp(k)
  __device__ __forceinline__ float4 *at(int pr, int j) const {
    return p + (size_t)pr * pstride + (size_t)(j >> 5) * (12 * kTile) + 2 * (j & (kTile - 1));
  }
  __device__ __forceinline__ SpinorPair load_pair(int pr, int j) const {
    const float4 *q = at(pr, j);
    SpinorPair s;
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      float4 a, b;
      ldg_v8(q + m * 2 * kTile, a, b);
      s.c[(2 * m) / 3][(2 * m) % 3] = cp_of(a);
      s.c[(2 * m + 1) / 3][(2 * m + 1) % 3] = cp_of(b);
    }
    return s;
  }
  __device__ __forceinline__ void store_pair(int pr, int j, const SpinorPair &s) const {
    float4 *q = at(pr, j);
#pragma unroll
    for (int m = 0; m < 6; ++m)
      stg_v8(q + m * 2 * kTile, f4_of(s.c[(2 * m) / 3][(2 * m) % 3]),
             f4_of(s.c[(2 * m + 1) / 3][(2 * m + 1) % 3]));
  }
  // one lane of a pair (lane 0: rhs 2 pr, lane 1: rhs 2 pr + 1); the other
  // lane's values are left as they are
  __device__ __forceinline__ void store_lane(int pr, int lane, int j, const SpinorPair &s) const {
    float *q = reinterpret_cast<float *>(at(pr, j)) + lane;
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      const CP &c = s.c[k / 3][k % 3];
      q[4 * comp(k)] = lane ? c.re.y : c.re.x;
      q[4 * comp(k) + 2] = lane ? c.im.y : c.im.x;
    }
  }
  // per-rhs access (for the kernels that run once per reliable update)
  __device__ __forceinline__ Spinor<float> load(int r, int j) const {
    const float4 *q = at(r >> 1, j);
    const bool b = r & 1;
    Spinor<float> s;
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      float4 v[2];
      ldg_v8(q + m * 2 * kTile, v[0], v[1]);
#pragma unroll
      for (int h = 0; h < 2; ++h)
        s.c[(2 * m + h) / 3][(2 * m + h) % 3] = cx(b ? v[h].y : v[h].x, b ? v[h].w : v[h].z);
    }
    return s;
  }
  __device__ __forceinline__ Spinor<float> load_raw(int r, int j, float &nm) const {
    nm = 1.f;
    return load(r, j);
  }
  __device__ __forceinline__ void store(int r, int j, const Spinor<float> &s) const {
    float *q = reinterpret_cast<float *>(at(r >> 1, j)) + (r & 1);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      q[4 * comp(k)] = s.c[k / 3][k % 3].re;
      q[4 * comp(k) + 2] = s.c[k / 3][k % 3].im;
    }
  }
};

inline size_t p32_pair_float4(int Vh) { return (size_t)((Vh + kTile - 1) / kTile) * 12 * kTile; }

// 18-real phased links, tiled: float2 U[idx / 32][mu][9][idx % 32]
struct LT32f {
  using R = float;
  static constexpr bool kPhased = true;
  const float2 *U;
  float2 ph[4];  // unused: the phase is multiplied in
  __device__ __forceinline__ Link<float> load(int mu, int idx) const {
    const float2 *q = U + (size_t)(idx >> 5) * (36 * kTile) + mu * 9 * kTile + (idx & (kTile - 1));
    Link<float> L;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const float2 v = __ldg(q + k * kTile);
      L.m[k / 3][k % 3] = cx(v.x, v.y);
    }
    return L;
  }
  // the loaded words and the link built from them, separately (so that a
  // kernel can issue the loads early and build the link when it needs it)
  struct Raw {
    float2 v[9];
  };
  __device__ __forceinline__ Raw load_raw(int mu, int idx) const {
    const float2 *q = U + (size_t)(idx >> 5) * (36 * kTile) + mu * 9 * kTile + (idx & (kTile - 1));
    Raw r;
#pragma unroll
    for (int k = 0; k < 9; ++k) r.v[k] = __ldg(q + k * kTile);
    return r;
  }
  __device__ __forceinline__ Link<float> build(const Raw &r, int) const {
    Link<float> L;
#pragma unroll
    for (int k = 0; k < 9; ++k) L.m[k / 3][k % 3] = cx(r.v[k].x, r.v[k].y);
    return L;
  }
};

// 12-real phased links (rows 0, 1), tiled: float4 U[idx / 32][mu][3][idx % 32];
// row 2 = e^{3 i theta_mu} conj(row0 x row1) (ph = e^{3 i theta_mu})
struct LT32c {
  using R = float;
  static constexpr bool kPhased = true;
  const float4 *U;
  float2 ph[4];
  __device__ __forceinline__ Link<float> load(int mu, int idx) const {
    const float4 *q = U + (size_t)(idx >> 5) * (12 * kTile) + mu * 3 * kTile + (idx & (kTile - 1));
    Link<float> L;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float4 v = __ldg(q + k * kTile);
      L.m[(2 * k) / 3][(2 * k) % 3] = cx(v.x, v.y);
      L.m[(2 * k + 1) / 3][(2 * k + 1) % 3] = cx(v.z, v.w);
    }
    reconstruct_row2(L);
    apply_row2_phase(L, ph[mu]);
    return L;
  }
  struct Raw {
    float4 v[3];
  };
  __device__ __forceinline__ Raw load_raw(int mu, int idx) const {
    const float4 *q = U + (size_t)(idx >> 5) * (12 * kTile) + mu * 3 * kTile + (idx & (kTile - 1));
    Raw r;
#pragma unroll
    for (int k = 0; k < 3; ++k) r.v[k] = __ldg(q + k * kTile);
    return r;
  }
  __device__ __forceinline__ Link<float> build(const Raw &r, int mu) const {
    Link<float> L;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      L.m[(2 * k) / 3][(2 * k) % 3] = cx(r.v[k].x, r.v[k].y);
      L.m[(2 * k + 1) / 3][(2 * k + 1) % 3] = cx(r.v[k].z, r.v[k].w);
    }
    reconstruct_row2(L);
    apply_row2_phase(L, ph[mu]);
    return L;
  }
};

// h = (1 + s g_mu) f projected to spins 0, 1, both rhs (table in
// spinor_ops.cuh); with g5 on the input the sign of the lower spins flips
template <int MU, int S>
__device__ __forceinline__ HalfPair project_pair(const SpinorPair &f) {
  HalfPair h;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const CP &f0 = f.c[0][c], &f1 = f.c[1][c], &f2 = f.c[2][c], &f3 = f.c[3][c];
    if (MU == 0) {  // h0 = f0 - s f2, h1 = f1 - s f3
      h.c[0][c].re = S > 0 ? sub2(f0.re, f2.re) : add2(f0.re, f2.re);
      h.c[0][c].im = S > 0 ? sub2(f0.im, f2.im) : add2(f0.im, f2.im);
      h.c[1][c].re = S > 0 ? sub2(f1.re, f3.re) : add2(f1.re, f3.re);
      h.c[1][c].im = S > 0 ? sub2(f1.im, f3.im) : add2(f1.im, f3.im);
    } else if (MU == 1) {  // h0 = f0 - s i f3, h1 = f1 - s i f2; i z = (-z.im, z.re)
      h.c[0][c].re = S > 0 ? add2(f0.re, f3.im) : sub2(f0.re, f3.im);
      h.c[0][c].im = S > 0 ? sub2(f0.im, f3.re) : add2(f0.im, f3.re);
      h.c[1][c].re = S > 0 ? add2(f1.re, f2.im) : sub2(f1.re, f2.im);
      h.c[1][c].im = S > 0 ? sub2(f1.im, f2.re) : add2(f1.im, f2.re);
    } else if (MU == 2) {  // h0 = f0 - s f3, h1 = f1 + s f2
      h.c[0][c].re = S > 0 ? sub2(f0.re, f3.re) : add2(f0.re, f3.re);
      h.c[0][c].im = S > 0 ? sub2(f0.im, f3.im) : add2(f0.im, f3.im);
      h.c[1][c].re = S > 0 ? add2(f1.re, f2.re) : sub2(f1.re, f2.re);
      h.c[1][c].im = S > 0 ? add2(f1.im, f2.im) : sub2(f1.im, f2.im);
    } else {  // h0 = f0 - s i f2, h1 = f1 + s i f3
      h.c[0][c].re = S > 0 ? add2(f0.re, f2.im) : sub2(f0.re, f2.im);
      h.c[0][c].im = S > 0 ? sub2(f0.im, f2.re) : add2(f0.im, f2.re);
      h.c[1][c].re = S > 0 ? sub2(f1.re, f3.im) : add2(f1.re, f3.im);
      h.c[1][c].im = S > 0 ? add2(f1.im, f3.re) : sub2(f1.im, f3.re);
    }
  }
  return h;
}

// out = (a_s + i b_s) v per spin s (site-diagonal, per-spin coefficients)
__device__ __forceinline__ void diag_pair(SpinorPair &o, const SpinorPair &v, const float (&a)[4],
                                          const float (&b)[4], bool accumulate) {
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const CP &x = v.c[s][c];
      float2 re = accumulate ? __ffma2_rn(bc(a[s]), x.re, o.c[s][c].re) : __fmul2_rn(bc(a[s]), x.re);
      float2 im = accumulate ? __ffma2_rn(bc(a[s]), x.im, o.c[s][c].im) : __fmul2_rn(bc(a[s]), x.im);
      re = __ffma2_rn(bc(-b[s]), x.im, re);
      im = __ffma2_rn(bc(b[s]), x.re, im);
      o.c[s][c].re = re;
      o.c[s][c].im = im;
    }
}

// |v|^2 of one site for both right-hand sides, accumulated in FP64
__device__ __forceinline__ double2 norm2_pair(const SpinorPair &v) {
  double2 n = make_double2(0.0, 0.0);
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const CP &z = v.c[s][c];
      n.x = fma((double)z.re.x, (double)z.re.x, n.x);
      n.x = fma((double)z.im.x, (double)z.im.x, n.x);
      n.y = fma((double)z.re.y, (double)z.re.y, n.y);
      n.y = fma((double)z.im.y, (double)z.im.y, n.y);
    }
  return n;
}

__device__ __forceinline__ void store_active(const P32 &f, int pr, int j, const SpinorPair &v,
                                             bool act_a, bool act_b) {
  if (act_a && act_b)
    f.store_pair(pr, j, v);
  else
    f.store_lane(pr, act_a ? 0 : 1, j, v);
}

template <int MU, class LF>
__device__ __forceinline__ void hop_pair_dir(SpinorPair &acc, const HopArgs<P32, LF> &A,
                                             const SiteCoord &cd, int pr, int self, int qoff,
                                             bool g5in) {
  const Geom &g = A.eg.g;
  {  // backward: (1 + g_mu) U_mu(x-mu)^+ in(x-mu)
    const int j = nb_lex(g, cd, MU, -1) >> 1;
    const Link<float> W = A.links.load(MU, qoff + j);
    const SpinorPair f = A.in.load_pair(pr, j);
    const HalfPair h = g5in ? project_pair<MU, -1>(f) : project_pair<MU, +1>(f);
    accum_recon_pair(MU, +1, acc, link_mul_pair<true>(W, h));
  }
  {  // forward: (1 - g_mu) U_mu(x) in(x+mu)
    const int j = nb_lex(g, cd, MU, +1) >> 1;
    const Link<float> W = A.links.load(MU, self);
    const SpinorPair f = A.in.load_pair(pr, j);
    const HalfPair h = g5in ? project_pair<MU, +1>(f) : project_pair<MU, -1>(f);
    accum_recon_pair(MU, -1, acc, link_mul_pair<false>(W, h));
  }
}

// The even/odd stencil sweep (same operator as k_eo_hop) on pair-tiled
// fields: thread = (site, rhs pair).  Directions in the order z, y, x, t (the
// z and y neighbours of a block's sites are in L1 after z-).  A pair with one
// inactive right-hand side computes both and stores only the active one;
// with dot_part, per-warp partials of |out|^2 per rhs (as k_eo_hop_x2).
// RUPD: the sweep that produces A p of a CG iteration updates the residual
// instead, r -= alpha A p, and its partials are those of |r|^2; A p itself
// is not stored (CG needs it for nothing else).
template <class LF, bool G5IN, bool G5HOP, bool AUX, bool RUPD = false>
__global__ void __launch_bounds__(kHopMaxThreads, 2) k_eo_hop_pt(HopArgs<P32, LF> A) {
  const int pr = blockIdx.x * blockDim.y + threadIdx.y;
  const int ra = 2 * pr;
  if (ra >= A.nrhs) return;
  const bool act_a = !(A.done && A.done[ra]);
  const bool has_b = ra + 1 < A.nrhs;
  const bool act_b = has_b && !(A.done && A.done[ra + 1]);
  if (!act_a && !act_b) return;
  const Geom &g = A.eg.g;
  const int p = A.eg.p;
  const int qoff = (1 - p) * g.Vh;
  // epilogue coefficients per spin: out = D1 (c [g5] hop) + D2 aux with
  // D = alpha + i beta g5; c and the optional g5 folded into D1
  float a1[4], b1[4], a2[4], b2[4];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const float g5 = s < 2 ? 1.f : -1.f;
    const float gh = G5HOP ? g5 : 1.f;
    a1[s] = (float)(A.c * A.d1a) * gh;
    b1[s] = (float)(A.c * A.d1b) * g5 * gh;
    a2[s] = (float)A.d2a;
    b2[s] = (float)A.d2b * g5;
  }
  for (int sb = blockIdx.y; sb * (int)blockDim.x < g.Vh; sb += gridDim.y) {
    const int i = sb * blockDim.x + threadIdx.x;
    double2 n2 = make_double2(0.0, 0.0);  // |out|^2 (or |r|^2) of this site, rhs a and b
    if (i < g.Vh) {
      const SiteCoord cd = site_coord(g, p, i);
      const int self = p * g.Vh + i;
      SpinorPair acc;
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc.c[s][c].re = acc.c[s][c].im = make_float2(0.f, 0.f);
      hop_pair_dir<3>(acc, A, cd, pr, self, qoff, G5IN);
      hop_pair_dir<2>(acc, A, cd, pr, self, qoff, G5IN);
      hop_pair_dir<1>(acc, A, cd, pr, self, qoff, G5IN);
      hop_pair_dir<0>(acc, A, cd, pr, self, qoff, G5IN);
      SpinorPair o;
      diag_pair(o, acc, a1, b1, false);
      if (AUX) diag_pair(o, A.aux.load_pair(pr, i), a2, b2, true);
      if (RUPD) {
        const float2 na = make_float2(-(float)A.alpha[ra], has_b ? -(float)A.alpha[ra + 1] : 0.f);
        SpinorPair rv = A.rup.load_pair(pr, i);
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            rv.c[s][c].re = __ffma2_rn(na, o.c[s][c].re, rv.c[s][c].re);
            rv.c[s][c].im = __ffma2_rn(na, o.c[s][c].im, rv.c[s][c].im);
          }
        if (A.dot_part) n2 = norm2_pair(rv);
        store_active(A.rup, pr, i, rv, act_a, act_b);
      } else {
        if (A.dot_part) n2 = norm2_pair(o);
        store_active(A.out, pr, i, o, act_a, act_b);
      }
    }
    if (A.dot_part) {  // the whole warp is here: one row, warp-aligned block width
      double da = n2.x, db = n2.y;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        da += __shfl_down_sync(0xffffffffu, da, o);
        db += __shfl_down_sync(0xffffffffu, db, o);
      }
      if ((threadIdx.x & 31) == 0) {
        const int w = sb * (blockDim.x >> 5) + (threadIdx.x >> 5);
        A.dot_part[(size_t)ra * A.dot_np + w] = da;
        if (has_b) A.dot_part[(size_t)(ra + 1) * A.dot_np + w] = db;
      }
    }
  }
}

// ---- the same sweep with the accumulator in tensor memory --------------------
// The register budget of k_eo_hop_pt (a 48-register two-rhs accumulator, the
// 60 registers of one direction's loads) caps it at 16 warps per SM, and the
// sweep is bound by load latency at that occupancy.  Here the accumulator
// lives in tensor memory (TMEM, 512 columns x 128 lanes of 32 bits per SM):
// thread = lane of its warp's 32-lane quarter (warp w of a 128-thread block
// owns lanes 32 w .. 32 w + 31), component k = 3 spin + colour of the site's
// two-rhs spinor at columns 4 k .. 4 k + 3 = (re a, re b, im a, im b).  Each
// direction adds its reconstructed contribution with tcgen05.ld / add /
// tcgen05.st in three 16-column chunks, component by component in the same
// order as the register accumulator (the results are bitwise those of
// k_eo_hop_pt).  The freed registers buy either more warps (PIPE false: 80
// registers, 24 warps per SM) or the next direction's loads in flight while
// one direction is computed (PIPE true: 128 registers, 16 warps).
// Each block allocates 64 columns (48 used) once and frees them before it
// exits; at most 8 blocks of this kernel fit the 512 columns of an SM, and
// both register budgets keep residency at or below that (6 and 4 blocks).
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

constexpr int kTmemThreads = 128;
constexpr int kTmemCols = 64;

__device__ __forceinline__ void tmem_ld16(unsigned a, float (&v)[16]) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(a));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tmem_st16(unsigned a, const float (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16};" ::"r"(a),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15]))
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// component (s, c) of the (1 + S g_mu)-reconstruction of u added to a (the
// table of accum_recon_pair, one component)
template <int MU, int S>
__device__ __forceinline__ void recon_add(CP &a, int s, int c, const HalfPair &u) {
  if (s < 2) {
    a.re = add2(a.re, u.c[s][c].re);
    a.im = add2(a.im, u.c[s][c].im);
  } else if (MU == 0) {  // r2 = -S u0, r3 = -S u1
    const CP &v = u.c[s - 2][c];
    a.re = S > 0 ? sub2(a.re, v.re) : add2(a.re, v.re);
    a.im = S > 0 ? sub2(a.im, v.im) : add2(a.im, v.im);
  } else if (MU == 1) {  // r2 = S i u1, r3 = S i u0
    const CP &v = u.c[s == 2 ? 1 : 0][c];
    a.re = S > 0 ? sub2(a.re, v.im) : add2(a.re, v.im);
    a.im = S > 0 ? add2(a.im, v.re) : sub2(a.im, v.re);
  } else if (MU == 2) {  // r2 = S u1, r3 = -S u0
    const CP &v = u.c[s == 2 ? 1 : 0][c];
    const bool plus = (s == 2) == (S > 0);
    a.re = plus ? add2(a.re, v.re) : sub2(a.re, v.re);
    a.im = plus ? add2(a.im, v.im) : sub2(a.im, v.im);
  } else {  // r2 = S i u0, r3 = -S i u1
    const CP &v = u.c[s - 2][c];
    const bool plus = (s == 2) == (S > 0);  // a += i v
    a.re = plus ? sub2(a.re, v.im) : add2(a.re, v.im);
    a.im = plus ? add2(a.im, v.re) : sub2(a.im, v.re);
  }
}

// acc (tensor memory, this thread's lane from column tacc) += reconstruction
// of u; FIRST: the accumulator starts from zero (nothing loaded)
template <int MU, int S, bool FIRST>
__device__ __forceinline__ void tmem_accum(unsigned tacc, const HalfPair &u) {
  if (!FIRST) tmem_wait_st();  // the previous direction's stores are complete
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    float v[16];
    if (FIRST) {
#pragma unroll
      for (int k = 0; k < 16; ++k) v[k] = 0.f;
    } else {
      tmem_ld16(tacc + 16 * q, v);
    }
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const int k = 4 * q + kk;
      CP a;
      a.re = make_float2(v[4 * kk], v[4 * kk + 1]);
      a.im = make_float2(v[4 * kk + 2], v[4 * kk + 3]);
      recon_add<MU, S>(a, k / 3, k % 3, u);
      v[4 * kk] = a.re.x;
      v[4 * kk + 1] = a.re.y;
      v[4 * kk + 2] = a.im.x;
      v[4 * kk + 3] = a.im.y;
    }
    tmem_st16(tacc + 16 * q, v);
  }
}

// the loads of direction D (mu = 3, 3, 2, 2, 1, 1, 0, 0: z, y, x, t;
// backward for even D, forward for odd D: the order of hop_pair_dir)
template <class LF>
struct DirLoads {
  SpinorPair f;
  typename LF::Raw w;
};
template <int D, class LF>
__device__ __forceinline__ DirLoads<LF> load_dir(const HopArgs<P32, LF> &A, const SiteCoord &cd,
                                                 int pr, int self, int qoff) {
  constexpr int MU = 3 - (D >> 1);
  constexpr int DIR = (D & 1) ? 1 : -1;
  const int j = nb_lex(A.eg.g, cd, MU, DIR) >> 1;
  DirLoads<LF> d;
  d.w = A.links.load_raw(MU, DIR < 0 ? qoff + j : self);
  d.f = A.in.load_pair(pr, j);
  return d;
}
template <int D, class LF>
__device__ __forceinline__ void apply_dir(unsigned tacc, const HopArgs<P32, LF> &A,
                                          const DirLoads<LF> &d, bool g5in) {
  constexpr int MU = 3 - (D >> 1);
  const Link<float> W = A.links.build(d.w, MU);
  if constexpr (D & 1) {  // forward: (1 - g_mu) U_mu(x) in(x+mu)
    const HalfPair h = g5in ? project_pair<MU, +1>(d.f) : project_pair<MU, -1>(d.f);
    tmem_accum<MU, -1, false>(tacc, link_mul_pair<false>(W, h));
  } else {  // backward: (1 + g_mu) U_mu(x-mu)^+ in(x-mu)
    const HalfPair h = g5in ? project_pair<MU, -1>(d.f) : project_pair<MU, +1>(d.f);
    tmem_accum<MU, +1, D == 0>(tacc, link_mul_pair<true>(W, h));
  }
}

// out component = D1 acc (+ D2 aux) per spin s, as diag_pair for one component
__device__ __forceinline__ CP diag_comp(const CP &x, float a, float b) {
  CP o;
  o.re = __fmul2_rn(bc(a), x.re);
  o.im = __fmul2_rn(bc(a), x.im);
  o.re = __ffma2_rn(bc(-b), x.im, o.re);
  o.im = __ffma2_rn(bc(b), x.re, o.im);
  return o;
}
__device__ __forceinline__ void diag_comp_acc(CP &o, const CP &x, float a, float b) {
  CP r;
  r.re = __ffma2_rn(bc(a), x.re, o.re);
  r.im = __ffma2_rn(bc(a), x.im, o.im);
  r.re = __ffma2_rn(bc(-b), x.im, r.re);
  r.im = __ffma2_rn(bc(b), x.re, r.im);
  o = r;
}

template <class LF, bool G5IN, bool G5HOP, bool AUX, bool RUPD, bool PIPE>
__global__ void __launch_bounds__(kTmemThreads, PIPE ? 4 : 6) k_eo_hop_ptm(HopArgs<P32, LF> A) {
  const int pr = blockIdx.x;  // one rhs pair per block: every exit below is block-uniform
  const int ra = 2 * pr;
  if (ra >= A.nrhs) return;
  const bool act_a = !(A.done && A.done[ra]);
  const bool has_b = ra + 1 < A.nrhs;
  const bool act_b = has_b && !(A.done && A.done[ra + 1]);
  if (!act_a && !act_b) return;
  __shared__ unsigned tm_base;
  const int warp = threadIdx.x >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tm_base)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const unsigned tacc = tm_base + ((unsigned)(warp * 32) << 16);
  const Geom &g = A.eg.g;
  const int p = A.eg.p;
  const int qoff = (1 - p) * g.Vh;
  for (int sb = blockIdx.y; sb * kTmemThreads < g.Vh; sb += gridDim.y) {
    const int i_raw = sb * kTmemThreads + threadIdx.x;
    const bool valid = i_raw < g.Vh;  // the tensor-memory accesses need the whole warp
    const int i = valid ? i_raw : g.Vh - 1;
    const SiteCoord cd = site_coord(g, p, i);
    const int self = p * g.Vh + i;
    if constexpr (PIPE) {
      DirLoads<LF> cur = load_dir<0>(A, cd, pr, self, qoff), nxt;
      nxt = load_dir<1>(A, cd, pr, self, qoff);
      apply_dir<0>(tacc, A, cur, G5IN);
      cur = load_dir<2>(A, cd, pr, self, qoff);
      apply_dir<1>(tacc, A, nxt, G5IN);
      nxt = load_dir<3>(A, cd, pr, self, qoff);
      apply_dir<2>(tacc, A, cur, G5IN);
      cur = load_dir<4>(A, cd, pr, self, qoff);
      apply_dir<3>(tacc, A, nxt, G5IN);
      nxt = load_dir<5>(A, cd, pr, self, qoff);
      apply_dir<4>(tacc, A, cur, G5IN);
      cur = load_dir<6>(A, cd, pr, self, qoff);
      apply_dir<5>(tacc, A, nxt, G5IN);
      nxt = load_dir<7>(A, cd, pr, self, qoff);
      apply_dir<6>(tacc, A, cur, G5IN);
      apply_dir<7>(tacc, A, nxt, G5IN);
    } else {
      apply_dir<0>(tacc, A, load_dir<0>(A, cd, pr, self, qoff), G5IN);
      apply_dir<1>(tacc, A, load_dir<1>(A, cd, pr, self, qoff), G5IN);
      apply_dir<2>(tacc, A, load_dir<2>(A, cd, pr, self, qoff), G5IN);
      apply_dir<3>(tacc, A, load_dir<3>(A, cd, pr, self, qoff), G5IN);
      apply_dir<4>(tacc, A, load_dir<4>(A, cd, pr, self, qoff), G5IN);
      apply_dir<5>(tacc, A, load_dir<5>(A, cd, pr, self, qoff), G5IN);
      apply_dir<6>(tacc, A, load_dir<6>(A, cd, pr, self, qoff), G5IN);
      apply_dir<7>(tacc, A, load_dir<7>(A, cd, pr, self, qoff), G5IN);
    }
    // epilogue, four components at a time: out = D1 (c [g5] hop) + D2 aux
    // (or r -= alpha out), |out|^2 (or |r|^2) in FP64 in component order
    const float2 na = RUPD ? make_float2(-(float)A.alpha[ra], has_b ? -(float)A.alpha[ra + 1] : 0.f)
                           : make_float2(0.f, 0.f);
    double2 n2 = make_double2(0.0, 0.0);
    tmem_wait_st();
    const float4 *auxp = AUX ? A.aux.at(pr, i) : nullptr;
    float4 *dst = RUPD ? A.rup.at(pr, i) : A.out.at(pr, i);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      float v[16];
      tmem_ld16(tacc + 16 * q, v);
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const int k = 4 * q + kk, s = k / 3;
        const float g5 = s < 2 ? 1.f : -1.f;
        const float gh = G5HOP ? g5 : 1.f;
        CP x;
        x.re = make_float2(v[4 * kk], v[4 * kk + 1]);
        x.im = make_float2(v[4 * kk + 2], v[4 * kk + 3]);
        CP o = diag_comp(x, (float)(A.c * A.d1a) * gh, (float)(A.c * A.d1b) * g5 * gh);
        if (AUX) diag_comp_acc(o, cp_of(__ldg(auxp + P32::comp(k))), (float)A.d2a, (float)A.d2b * g5);
        if (RUPD) {
          CP rv = cp_of(__ldg(dst + P32::comp(k)));
          rv.re = __ffma2_rn(na, o.re, rv.re);
          rv.im = __ffma2_rn(na, o.im, rv.im);
          o = rv;
        }
        if (valid) {
          if (A.dot_part) {
            n2.x = fma((double)o.re.x, (double)o.re.x, n2.x);
            n2.x = fma((double)o.im.x, (double)o.im.x, n2.x);
            n2.y = fma((double)o.re.y, (double)o.re.y, n2.y);
            n2.y = fma((double)o.im.y, (double)o.im.y, n2.y);
          }
          if (act_a && act_b) {
            dst[P32::comp(k)] = f4_of(o);
          } else {
            float *qf = reinterpret_cast<float *>(dst + P32::comp(k)) + (act_a ? 0 : 1);
            qf[0] = act_a ? o.re.x : o.re.y;
            qf[2] = act_a ? o.im.x : o.im.y;
          }
        }
      }
    }
    if (A.dot_part) {  // whole warps: the block width is a multiple of 32
      double da = n2.x, db = n2.y;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        da += __shfl_down_sync(0xffffffffu, da, o);
        db += __shfl_down_sync(0xffffffffu, db, o);
      }
      if ((threadIdx.x & 31) == 0) {
        const int w = sb * (kTmemThreads >> 5) + warp;
        A.dot_part[(size_t)ra * A.dot_np + w] = da;
        if (has_b) A.dot_part[(size_t)(ra + 1) * A.dot_np + w] = db;
      }
    }
  }
  tmem_fence_before_sync();
  __syncthreads();  // every warp's tensor-memory accesses are complete
  tmem_fence_after_sync();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm_base),
                 "r"(kTmemCols));
}

// ---- the same sweep with the t and x neighbours staged by bulk copies -------
// On lattices with LY*LZ/2 a multiple of 32, the 32 sites of a tile share
// their t and x coordinates, so the t+-, x+- neighbours of a tile are again
// one whole tile (6 KB per rhs pair): one cp.async.bulk each, issued by lane 0
// of the warp that owns the tile into shared memory and completed on an
// mbarrier.  The two t copies start before the z and y hops (plain loads,
// mostly L1 hits) are computed, the x copies reuse the stage buffers as soon
// as the t data has been read, so the long-latency neighbours arrive while
// the warp computes and hold no registers while in flight.  Waits are
// bounded: a copy not complete after about a second sets *err and the
// kernel returns after a bounded wait for the copies it still has in flight.
constexpr int kBulkWarps = 4;  // warps per block: 4 consecutive tiles of one rhs pair
constexpr unsigned kTileBytes = 12 * kTile * sizeof(float4);  // 6144
constexpr size_t kBulkSmem = (size_t)kBulkWarps * 2 * kTileBytes;

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// one arrival that also announces `bytes` of transaction for this phase
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes,
                                         unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for the phase with the given parity to complete
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
  for (int n = 0; n < (1 << 20); ++n)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ SpinorPair stage_load(const float4 *S, int lane) {
  SpinorPair f;
#pragma unroll
  for (int k = 0; k < 12; ++k) f.c[k / 3][k % 3] = cp_of(S[P32::comp(k) + 2 * lane]);
  return f;
}

template <int MU, int S>
__device__ __forceinline__ void hop_from(SpinorPair &acc, const Link<float> &W,
                                         const SpinorPair &f, bool g5in) {
  if (S > 0) {  // backward: (1 + g_mu) U_mu(x-mu)^+ in(x-mu)
    const HalfPair h = g5in ? project_pair<MU, -1>(f) : project_pair<MU, +1>(f);
    accum_recon_pair(MU, +1, acc, link_mul_pair<true>(W, h));
  } else {  // forward: (1 - g_mu) U_mu(x) in(x+mu)
    const HalfPair h = g5in ? project_pair<MU, +1>(f) : project_pair<MU, -1>(f);
    accum_recon_pair(MU, -1, acc, link_mul_pair<false>(W, h));
  }
}

// Block = kBulkWarps warps on consecutive tiles of rhs pair blockIdx.x;
// dynamic shared memory kBulkSmem.  dot_part (if given) holds one partial
// per tile (dot_np = V/2 / 32).
template <class LF, bool G5IN, bool G5HOP, bool AUX, bool RUPD = false>
__global__ void __launch_bounds__(kBulkWarps * 32, 4) k_eo_hop_ptb(HopArgs<P32, LF> A) {
  extern __shared__ __align__(128) float4 stage[];
  __shared__ __align__(8) unsigned long long bars[kBulkWarps][2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pr = blockIdx.x;
  const int ra = 2 * pr;
  if (ra >= A.nrhs) return;  // uniform over the block
  const bool act_a = !(A.done && A.done[ra]);
  const bool has_b = ra + 1 < A.nrhs;
  const bool act_b = has_b && !(A.done && A.done[ra + 1]);
  if (!act_a && !act_b) return;  // uniform over the block
  const Geom &g = A.eg.g;
  const int p = A.eg.p;
  const int qoff = (1 - p) * g.Vh;
  float a1[4], b1[4], a2[4], b2[4];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const float g5 = s < 2 ? 1.f : -1.f;
    const float gh = G5HOP ? g5 : 1.f;
    a1[s] = (float)(A.c * A.d1a) * gh;
    b1[s] = (float)(A.c * A.d1b) * g5 * gh;
    a2[s] = (float)A.d2a;
    b2[s] = (float)A.d2b * g5;
  }
  float4 *S0 = stage + (size_t)warp * 2 * 12 * kTile, *S1 = S0 + 12 * kTile;
  unsigned long long *b0 = &bars[warp][0], *b1b = &bars[warp][1];
  if (lane == 0) {
    mbar_init(b0, 1);
    mbar_init(b1b, 1);
    fence_mbar_init();
  }
  __syncwarp();
  unsigned ph0 = 0, ph1 = 0;
  const int ntiles = g.Vh / kTile;
  const float4 *in_pair = A.in.p + (size_t)pr * A.in.pstride;
  for (int tile = blockIdx.y * kBulkWarps + warp; tile < ntiles;
       tile += gridDim.y * kBulkWarps) {
    const int i = tile * kTile + lane;
    const SiteCoord cd = site_coord(g, p, i);
    const int self = p * g.Vh + i;
    const int jtm = nb_lex(g, cd, 0, -1) >> 1, jtp = nb_lex(g, cd, 0, +1) >> 1;
    const int jxm = nb_lex(g, cd, 1, -1) >> 1, jxp = nb_lex(g, cd, 1, +1) >> 1;
    if (lane == 0) {  // whole neighbour tiles: lane 0's neighbour is the tile start
      fence_proxy_async();  // the previous tile's reads of S0, S1 come first
      mbar_expect_tx(b0, kTileBytes);
      bulk_g2s(S0, in_pair + (size_t)(jtm >> 5) * 12 * kTile, kTileBytes, b0);
      mbar_expect_tx(b1b, kTileBytes);
      bulk_g2s(S1, in_pair + (size_t)(jtp >> 5) * 12 * kTile, kTileBytes, b1b);
    }
    SpinorPair acc;
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) acc.c[s][c].re = acc.c[s][c].im = make_float2(0.f, 0.f);
    hop_pair_dir<3>(acc, A, cd, pr, self, qoff, G5IN);
    hop_pair_dir<2>(acc, A, cd, pr, self, qoff, G5IN);
    // every wait's outcome is made warp-uniform, so all lanes take the same
    // branches (and reach every __syncwarp)
    bool ok = __all_sync(0xffffffffu, mbar_wait(b0, ph0));
    if (ok) {
      ph0 ^= 1;
      hop_from<0, +1>(acc, A.links.load(0, qoff + jtm), stage_load(S0, lane), G5IN);
      __syncwarp();
      if (lane == 0) {
        fence_proxy_async();
        mbar_expect_tx(b0, kTileBytes);
        bulk_g2s(S0, in_pair + (size_t)(jxm >> 5) * 12 * kTile, kTileBytes, b0);
      }
      ok = __all_sync(0xffffffffu, mbar_wait(b1b, ph1));
    }
    if (ok) {
      ph1 ^= 1;
      hop_from<0, -1>(acc, A.links.load(0, self), stage_load(S1, lane), G5IN);
      __syncwarp();
      if (lane == 0) {
        fence_proxy_async();
        mbar_expect_tx(b1b, kTileBytes);
        bulk_g2s(S1, in_pair + (size_t)(jxp >> 5) * 12 * kTile, kTileBytes, b1b);
      }
      ok = __all_sync(0xffffffffu, mbar_wait(b0, ph0));
    }
    if (ok) {
      ph0 ^= 1;
      hop_from<1, +1>(acc, A.links.load(1, qoff + jxm), stage_load(S0, lane), G5IN);
      ok = __all_sync(0xffffffffu, mbar_wait(b1b, ph1));
    }
    if (!ok) {
      // a copy did not complete: report, let the copies in flight land
      // (bounded), leave
      if (lane == 0 && A.err) atomicExch(A.err, 1);
      mbar_wait(b0, ph0);
      mbar_wait(b1b, ph1);
      return;
    }
    ph1 ^= 1;
    hop_from<1, -1>(acc, A.links.load(1, self), stage_load(S1, lane), G5IN);
    __syncwarp();
    SpinorPair o;
    diag_pair(o, acc, a1, b1, false);
    if (AUX) diag_pair(o, A.aux.load_pair(pr, i), a2, b2, true);
    double2 n2 = make_double2(0.0, 0.0);
    if (RUPD) {
      const float2 na = make_float2(-(float)A.alpha[ra], has_b ? -(float)A.alpha[ra + 1] : 0.f);
      SpinorPair rv = A.rup.load_pair(pr, i);
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          rv.c[s][c].re = __ffma2_rn(na, o.c[s][c].re, rv.c[s][c].re);
          rv.c[s][c].im = __ffma2_rn(na, o.c[s][c].im, rv.c[s][c].im);
        }
      if (A.dot_part) n2 = norm2_pair(rv);
      store_active(A.rup, pr, i, rv, act_a, act_b);
    } else {
      if (A.dot_part) n2 = norm2_pair(o);
      store_active(A.out, pr, i, o, act_a, act_b);
    }
    if (A.dot_part) {
      double da = n2.x, db = n2.y;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        da += __shfl_down_sync(0xffffffffu, da, o);
        db += __shfl_down_sync(0xffffffffu, db, o);
      }
      if (lane == 0) {
        A.dot_part[(size_t)ra * A.dot_np + tile] = da;
        if (has_b) A.dot_part[(size_t)(ra + 1) * A.dot_np + tile] = db;
      }
    }
  }
}

// Whether a lattice admits k_eo_hop_ptb: the t and x neighbours of a tile
// are whole tiles when LY*LZ/2 is a multiple of 32.
inline bool bulk_stencil_ok(const Geom &g) { return (g.LY * g.LZ / 2) % kTile == 0; }

}  // namespace cvcb
