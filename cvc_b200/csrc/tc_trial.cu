// Tensor-core trial for the stencil's link product (the multi-rhs
// link x spinor-block product of Q_phi.c:66-80, _cm_eq_cm_ti_co /
// _fv_eq_cm_ti_fv, applied to N right-hand sides at once).
//
// Per site and link the product is u = W h with W a 3x3 complex link and h a
// 3 x (2 spins x N rhs) complex block, i.e. the real 6x6 matrix
// [[Re W, -Im W], [Im W, Re W]] times a 6 x 2N real block.  Each site has
// its own W, so a tensor-core tile can only hold links block-diagonally:
// mma.sync.m16n8k8 (TF32) takes two sites per 16x16 A tile (K = 16 in two
// steps, 28 % of the tile's multiply-adds useful), and tcgen05 tiles of
// M = 64 or 128 would hold 10 or 21 sites on the diagonal (under 5 %
// useful).  This file measures the most favourable of these against the
// packed FP32x2 FMAs the stencil uses, on the same data: for every site of a
// half lattice, 8 links (the stencil's 8 hops) times one block of N = 12 rhs,
// summed.  Variants: 0 packed FP32x2 FMAs (thread = site x rhs pair);
// 1 mma.sync TF32 (warp = 2 sites x 24 columns); 2 the same with three TF32
// products (hi*hi + hi*lo + lo*hi), which keeps FP32 accuracy.  The result is
// reported through cvcb_time_link_product; the stencil keeps variant 0.
#include <cstdint>

#include "cvcb_internal.h"
#include "eo_kernels.cuh"
#include "pair_kernels.cuh"

namespace cvcb {
namespace {

constexpr int kTcN = 12;  // right-hand sides

// h: float2 H[site][spin 2][colour 3][rhs 12] (complex), site-major (the
// mma variants' layout); out the same shape
__global__ void k_tc_init(float2 *h, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  unsigned x = 2654435761u * (unsigned)(k + 1);
  x ^= x >> 15;
  x *= 2246822519u;
  x ^= x >> 13;
  const float a = (float)(x & 0xffff) / 65536.f - 0.5f, b = (float)(x >> 16) / 65536.f - 0.5f;
  h[k] = make_float2(a, b);
}

// 8 links of site i: the forward link of each direction at (p, i) and the
// link of the other parity at the same half index (standing in for the
// backward links; the arithmetic is the same)
__device__ __forceinline__ int trial_link_index(const Geom &g, int i, int d) {
  return (d & 1) ? g.Vh + i : i;
}

// Pair-tiled copy of a site-major block (the layout the stencil's fields
// have): float4 P[pair q][tile][k = 3 s + c][32] = (re rhs 2q, re rhs 2q+1,
// im rhs 2q, im rhs 2q+1).  dir 0: site-major -> pair-tiled, 1: back.
__global__ void k_tc_convert(float4 *pt, float2 *sm, int vh, int dir) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int q = blockIdx.y;
  if (i >= vh) return;
  const int ntile = (vh + 31) / 32;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    float4 *d = pt + (((size_t)q * ntile + (i >> 5)) * 6 + k) * 32 + (i & 31);
    float2 *a = sm + ((size_t)i * 6 + k) * kTcN + 2 * q;
    if (dir == 0) {
      *d = make_float4(a[0].x, a[1].x, a[0].y, a[1].y);
    } else {
      const float4 v = *d;
      a[0] = make_float2(v.x, v.z);
      a[1] = make_float2(v.y, v.w);
    }
  }
}

// variant 0: thread = (site, rhs pair), packed FP32x2 FMAs (link_mul_pair),
// coalesced pair-tiled input and output
__global__ void __launch_bounds__(128) k_tc_ffma2(float4 *__restrict__ out,
                                                  const float4 *__restrict__ h, LT32f links,
                                                  Geom g) {
  const int q = blockIdx.y;  // rhs pair
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.Vh) return;
  const int ntile = (g.Vh + 31) / 32;
  const size_t base = (((size_t)q * ntile + (i >> 5)) * 6) * 32 + (i & 31);
  HalfPair hp;
#pragma unroll
  for (int k = 0; k < 6; ++k) hp.c[k / 3][k % 3] = cp_of(__ldg(h + base + k * 32));
  HalfPair acc;
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc.c[s][c].re = acc.c[s][c].im = make_float2(0.f, 0.f);
#pragma unroll
  for (int d = 0; d < 8; ++d) {
    const Link<float> W = links.load(d >> 1, trial_link_index(g, i, d));
    const HalfPair u = link_mul_pair<false>(W, hp);
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        acc.c[s][c].re = add2(acc.c[s][c].re, u.c[s][c].re);
        acc.c[s][c].im = add2(acc.c[s][c].im, u.c[s][c].im);
      }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) out[base + k * 32] = f4_of(acc.c[k / 3][k % 3]);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Element (row m, col k) of the block-diagonal A tile of two sites' real
// 6x6 link matrices [[Re W, -Im W], [Im W, Re W]] (rows/cols 12..15 zero),
// loaded directly: each lane reads only the link entries of its fragment.
__device__ __forceinline__ float a_load(const LT32f &lk, int mu, int idx0, int idx1, int m, int k) {
  const int sm = m / 6, sk = k / 6;
  if (sm != sk || sm > 1) return 0.f;
  const int idx = sm == 0 ? idx0 : idx1;
  const int mm = m % 6, kk = k % 6;
  const int r = mm % 3, c = kk % 3;
  const float2 w = __ldg(lk.U + (size_t)(idx >> 5) * (36 * kTile) + mu * 9 * kTile + (idx & (kTile - 1)) +
                         (r * 3 + c) * kTile);
  if (mm < 3) return kk < 3 ? w.x : -w.y;
  return kk < 3 ? w.y : w.x;
}

// variants 1, 2: warp = 2 sites (a site pair) x 24 columns (spin x rhs);
// A = block-diagonal links (16 x 16, two k-steps), B = the two sites' h
// (16 x 24, three n-tiles), C accumulated over the 8 links
template <bool SPLIT>
__global__ void __launch_bounds__(128) k_tc_mma(float2 *__restrict__ out, const float2 *__restrict__ h,
                                                LT32f links, Geom g) {
  const int lane = threadIdx.x & 31;
  const int gid = lane >> 2, tig = lane & 3;
  const int pairsite = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // warp index
  const int i0 = 2 * pairsite;
  if (i0 >= g.Vh) return;  // whole warp
  // B fragments (constant over the 8 links): b[kstep][ntile][0..1]
  uint32_t bh[2][3][2], bl[2][3][2];
#pragma unroll
  for (int ks = 0; ks < 2; ++ks)
#pragma unroll
    for (int nt = 0; nt < 3; ++nt)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int k = 8 * ks + tig + 4 * e, n = 8 * nt + gid;
        float v = 0.f;
        if (k < 12) {
          const int site = i0 + k / 6, kk = k % 6, s = n / kTcN, r = n % kTcN;
          const float2 z = h[(((size_t)site * 2 + s) * 3 + kk % 3) * kTcN + r];
          v = kk < 3 ? z.x : z.y;
        }
        bh[ks][nt][e] = to_tf32(v);
        bl[ks][nt][e] = to_tf32(v - __uint_as_float(bh[ks][nt][e]));
      }
  float c[3][4];
#pragma unroll
  for (int nt = 0; nt < 3; ++nt)
#pragma unroll
    for (int e = 0; e < 4; ++e) c[nt][e] = 0.f;
#pragma unroll 1
  for (int d = 0; d < 8; ++d) {
    const int idx0 = trial_link_index(g, i0, d), idx1 = trial_link_index(g, i0 + 1, d);
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      uint32_t ah[4], al[4];
      const int rows[4] = {gid, gid + 8, gid, gid + 8};
      const int cols[4] = {8 * ks + tig, 8 * ks + tig, 8 * ks + tig + 4, 8 * ks + tig + 4};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float v = a_load(links, d >> 1, idx0, idx1, rows[e], cols[e]);
        ah[e] = to_tf32(v);
        al[e] = to_tf32(v - __uint_as_float(ah[e]));
      }
#pragma unroll
      for (int nt = 0; nt < 3; ++nt) {
        mma_tf32(c[nt], ah, bh[ks][nt]);
        if (SPLIT) {
          mma_tf32(c[nt], ah, bl[ks][nt]);
          mma_tf32(c[nt], al, bh[ks][nt]);
        }
      }
    }
  }
  // C(m, n): rows 0..5 site i0, 6..11 site i0+1 (Re colours 0..2, Im 0..2)
#pragma unroll
  for (int nt = 0; nt < 3; ++nt)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int m = gid + 8 * (e >> 1), n = 8 * nt + 2 * tig + (e & 1);
      if (m >= 12) continue;
      const int site = i0 + m / 6, mm = m % 6, s = n / kTcN, r = n % kTcN;
      float *o = reinterpret_cast<float *>(out + (((size_t)site * 2 + s) * 3 + mm % 3) * kTcN + r);
      o[mm < 3 ? 0 : 1] = c[nt][e];
    }
}

__global__ void k_tc_maxdiff(const float2 *a, const float2 *b, size_t n, float *dmax, float *amax) {
  float d = 0.f, m = 0.f;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    d = fmaxf(d, fmaxf(fabsf(a[k].x - b[k].x), fabsf(a[k].y - b[k].y)));
    m = fmaxf(m, fmaxf(fabsf(b[k].x), fabsf(b[k].y)));
  }
  for (int o = 16; o > 0; o >>= 1) {
    d = fmaxf(d, __shfl_down_sync(0xffffffffu, d, o));
    m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(reinterpret_cast<int *>(dmax), __float_as_int(d));  // non-negative floats
    atomicMax(reinterpret_cast<int *>(amax), __float_as_int(m));
  }
}

}  // namespace

int time_link_product(cvcb_lattice *L, int variant, int reps, double *ms, double *rel_diff) {
  const Geom &g = L->g;
  if (g.Vh % 2) {
    set_error("the trial needs an even number of sites per parity");
    return CVCB_ERR_ARG;
  }
  if (g.Vh % 32) {
    set_error("the trial needs a multiple of 32 sites per parity");
    return CVCB_ERR_ARG;
  }
  const size_t n = (size_t)g.Vh * 2 * 3 * kTcN;  // complex numbers per block
  void *buf;
  CVCB_TRY(ensure_buffer(L, SLOT_F5, 5 * n * sizeof(float2) + 256, &buf));
  float2 *h = static_cast<float2 *>(buf), *o0 = h + n, *o1 = o0 + n;
  float4 *hpt = reinterpret_cast<float4 *>(o1 + n), *opt = hpt + n / 2;
  float *red = reinterpret_cast<float *>(opt + n / 2);
  k_tc_init<<<(unsigned)((n + 255) / 256), 256, 0, L->stream>>>(h, (int)n);
  CVCB_LAUNCHED(L);
  const dim3 cgrid((g.Vh + 127) / 128, kTcN / 2);
  k_tc_convert<<<cgrid, 128, 0, L->stream>>>(hpt, h, g.Vh, 0);
  CVCB_LAUNCHED(L);
  LT32f links{L->UT32f, {}};
  auto run = [&](int v, float2 *out) {
    if (v == 0) {
      k_tc_ffma2<<<cgrid, 128, 0, L->stream>>>(opt, hpt, links, g);
    } else {
      const int warps = g.Vh / 2;
      const unsigned blocks = (unsigned)((warps + 3) / 4);
      if (v == 1)
        k_tc_mma<false><<<blocks, 128, 0, L->stream>>>(out, h, links, g);
      else
        k_tc_mma<true><<<blocks, 128, 0, L->stream>>>(out, h, links, g);
    }
    CVCB_LAUNCHED(L);
    return CVCB_OK;
  };
  CVCB_TRY(run(0, o0));  // reference result, in site-major order
  k_tc_convert<<<cgrid, 128, 0, L->stream>>>(opt, o0, g.Vh, 1);
  CVCB_LAUNCHED(L);
  CVCB_TRY(run(variant, o1));
  if (variant == 0) {
    k_tc_convert<<<cgrid, 128, 0, L->stream>>>(opt, o1, g.Vh, 1);
    CVCB_LAUNCHED(L);
  }
  cudaEvent_t a, b;
  CVCB_CUDA(cudaEventCreate(&a));
  CVCB_CUDA(cudaEventCreate(&b));
  CVCB_CUDA(cudaEventRecord(a, L->stream));
  for (int k = 0; k < reps; ++k) CVCB_TRY(run(variant, o1));
  CVCB_CUDA(cudaEventRecord(b, L->stream));
  CVCB_CUDA(cudaMemsetAsync(red, 0, 2 * sizeof(float), L->stream));
  k_tc_maxdiff<<<296, 256, 0, L->stream>>>(o1, o0, n, red, red + 1);
  CVCB_LAUNCHED(L);
  float hr[2];
  CVCB_CUDA(cudaMemcpyAsync(hr, red, sizeof hr, cudaMemcpyDeviceToHost, L->stream));
  CVCB_CUDA(cudaEventSynchronize(b));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  float t;
  CVCB_CUDA(cudaEventElapsedTime(&t, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = t / reps;
  *rel_diff = hr[1] > 0 ? hr[0] / hr[1] : 0.0;
  return CVCB_OK;
}

}  // namespace cvcb

extern "C" int cvcb_time_link_product(cvcb_lattice *L, int variant, int reps, double *ms,
                                      double *rel_diff) {
  if (!L || !ms || !rel_diff) return CVCB_ERR_NULL;
  if (variant < 0 || variant > 2 || reps <= 0) return CVCB_ERR_ARG;
  if (!L->have_gauge) {
    cvcb::set_error("no gauge field uploaded");
    return CVCB_ERR_STATE;
  }
  CVCB_CUDA(cudaSetDevice(L->device));
  return cvcb::time_link_product(L, variant, reps, ms, rel_diff);
}
