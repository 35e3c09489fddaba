// Batched even/odd preconditioned CG on the normal equations of the Schur
// complement, with reduced-precision inner iterations and FP64 reliable
// updates.  Solves Q x_i = b_i for N right-hand sides per launch; Q is the
// operator of Q_phi_tbc (Q_phi.c:38-188).  No counterpart in the reference,
// which obtains propagators from files or from tmLQCD
// (cvc_exact2_xspace.c:401-547).
//
// Per right-hand side (all kept on the device, one slot per rhs):
//   b_hat = b_o + 1/2 H_oe A_ee^-1 b_e,  b_N = M^+ b_hat
//   CG on M^+ M x_o = b_N in sloppy precision (FP32 or FP16+norm spinors,
//   12-real or 18-real links); every time the sloppy residual has fallen by
//   `delta` (or the residual estimate reaches the target) the FP64 solution
//   absorbs the sloppy one, the true residual r_hat = b_hat - M x is
//   recomputed in FP64 with the exact 18-real operator, and the sloppy
//   recursion restarts from r_N = M^+ r_hat (formed in sloppy precision).
//   |r_hat| is the residual of the full system (the even rows vanish by
//   construction), so convergence is decided on |b - Q x| / |b| in FP64.
//   Finally x_e = A_ee^-1 (b_e + 1/2 H_eo x_o), Q x is recomputed in FP64 on
//   both parities and |b - Q x| / |b| is checked.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <numeric>
#include <tuple>
#include <type_traits>
#include <vector>

#include "cvcb_internal.h"
#include "eo_kernels.cuh"
#include "pair_kernels.cuh"
#include "reduce.cuh"

namespace cvcb {

namespace {

// Right-hand sides per batch: up to 96, so that the 8 x 12 columns of the
// benchmark can advance as one set (each link loaded once per site for all).
constexpr int kMaxBatch = 96;
// Tuner keys of the pair-tiled FP32 fields: precision + kPairKey.
constexpr int kPairKey = 10;
constexpr size_t kMaxStagedSmem = 200 * 1024;  // opt-in dynamic shared memory of the staged stencil

// ---- batched reductions: blockIdx.y = right-hand side ----------------------
struct BatchRed {
  double *partials;    // [rhs][block]
  unsigned *counters;  // [rhs]
};

template <class F, class E>
__global__ void __launch_bounds__(kRedThreads)
    k_reduce_rhs(F f, E e, int nsites, BatchRed br, const int *__restrict__ skip) {
  const int r = blockIdx.y;
  if (skip && skip[r]) return;
  __shared__ double sh[1][kRedThreads / 32];
  __shared__ bool last;
  double v[1] = {0.0};
  for (int s = blockIdx.x * kRedThreads + threadIdx.x; s < nsites; s += gridDim.x * kRedThreads)
    v[0] += f(r, s);
  block_sum<1>(v, sh);
  double *part = br.partials + (size_t)r * kMaxRedBlocks;
  if (threadIdx.x == 0) {
    part[blockIdx.x] = v[0];
    __threadfence();
    last = atomicAdd(br.counters + r, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  v[0] = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += kRedThreads) v[0] += __ldcg(part + b);
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) {
    br.counters[r] = 0;
    e(r, v[0]);
  }
}

template <typename R>
__device__ __forceinline__ double norm2(const Spinor<R> &a) {
  double s = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) s += (double)a.c[k][c].re * a.c[k][c].re + (double)a.c[k][c].im * a.c[k][c].im;
  return s;
}
template <typename R>
__device__ __forceinline__ double redot(const Spinor<R> &a, const Spinor<R> &b) {
  double s = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      s += (double)a.c[k][c].re * b.c[k][c].re + (double)a.c[k][c].im * b.c[k][c].im;
  return s;
}
template <typename R, typename S>
__device__ __forceinline__ Spinor<R> convert(const Spinor<S> &a) {
  Spinor<R> o;
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) o.c[k][c] = cx((R)a.c[k][c].re, (R)a.c[k][c].im);
  return o;
}

// The sloppy recursion works in units of the last true residual: sloppy
// fields = scale * (true fields), scale = 1 / |r_hat| from the latest
// reliable update, so its magnitudes stay O(1) whatever the size of b
// (a source of 1e-33 would otherwise reach FP32 denormals).
struct Scal {  // per right-hand side, device arrays
  double *rr, *pAp, *alpha, *beta, *rhat2, *rn2;
  double *scale, *scale_prev;
  int *done;
};

// pAp = Re <p, Ap>; alpha = rr / pAp (kernels other than the packed one;
// the packed one takes pAp = |M p|^2 from the sweep that writes M p)
template <class SF>
struct RedPAp {
  SF p, Ap;
  __device__ double operator()(int r, int s) const { return redot(p.load(r, s), Ap.load(r, s)); }
};
struct EpiAlphaB {
  Scal S;
  __device__ void operator()(int r, double t) const {
    S.pAp[r] = t;
    // M^+ M is positive definite; a non-positive <p, M^+ M p> only comes from
    // rounding at the end of convergence: take no step and let the host's
    // reliable update refresh the residual.
    S.alpha[r] = (t > 0 && isfinite(t)) ? S.rr[r] / t : 0.0;
  }
};

// Sum of the per-warp partials of <p, M^+M p> = |M p|^2 that the second
// sweep of M^+M wrote (fixed order: deterministic), then the epilogue (alpha).
template <class E>
__global__ void __launch_bounds__(kRedThreads)
    k_dot_finish(const double *__restrict__ part, int np, E e, const int *__restrict__ skip) {
  const int r = blockIdx.x;
  if (skip && skip[r]) return;
  __shared__ double sh[1][kRedThreads / 32];
  double v[1] = {0.0};
  for (int k = threadIdx.x; k < np; k += kRedThreads) v[0] += part[(size_t)r * np + k];
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) e(r, v[0]);
}

// r_s -= alpha Ap; rr_new = |r_s|^2; beta = rr_new / rr.  The x update
// waits for k_p_upd, which reads p anyway: 3 instead of 6 field passes here
// for 2 more there.
template <class SF>
struct RedUpdate {
  SF Ap, rs;
  Scal S;
  __device__ double operator()(int r, int s) const {
    using R = typename SF::R;
    const R a = (R)S.alpha[r];
    const Spinor<R> apv = Ap.load(r, s);
    Spinor<R> rv = rs.load(r, s);
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        rv.c[k][c].re -= a * apv.c[k][c].re;
        rv.c[k][c].im -= a * apv.c[k][c].im;
      }
    rs.store(r, s, rv);
    return norm2(rv);
  }
};
struct EpiBetaB {
  Scal S;
  __device__ void operator()(int r, double t) const {
    S.beta[r] = t / S.rr[r];
    S.rr[r] = t;
  }
};

// x_s += alpha p; p = r_s + beta p
template <class SF, class XF>
__global__ void k_p_upd(SF p, SF rs, XF xs, Scal S, int nsites, int nrhs) {
  using R = typename SF::R;
  using RX = typename XF::R;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (s >= nsites || r >= nrhs || S.done[r]) return;
  const R b = (R)S.beta[r];
  const RX a = (RX)S.alpha[r];
  const Spinor<R> rv = rs.load(r, s);
  Spinor<R> pv = p.load(r, s);
  Spinor<RX> xv = xs.load(r, s);
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      xv.c[k][c].re += a * (RX)pv.c[k][c].re;
      xv.c[k][c].im += a * (RX)pv.c[k][c].im;
      pv.c[k][c] = rv.c[k][c] + b * pv.c[k][c];
    }
  xs.store(r, s, xv);
  p.store(r, s, pv);
}

// Pair-tiled form of the CG vector update (thread = site x rhs pair, packed
// FP32x2 arithmetic; an inactive right-hand side keeps its values).  The
// residual update r -= alpha A p runs inside the last stencil sweep.
// x_s += alpha p; p = r_s + beta p
__global__ void k_p_upd_pt(P32 p, P32 rs, P32 xs, Scal S, int nsites, int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int ra = 2 * blockIdx.y;
  if (s >= nsites) return;
  const bool act_a = !S.done[ra];
  const bool act_b = ra + 1 < nrhs && !S.done[ra + 1];
  if (!act_a && !act_b) return;
  const float2 a = make_float2((float)S.alpha[ra], act_b ? (float)S.alpha[ra + 1] : 0.f);
  const float2 b = make_float2((float)S.beta[ra], act_b ? (float)S.beta[ra + 1] : 0.f);
  const SpinorPair rv = rs.load_pair(blockIdx.y, s);
  SpinorPair pv = p.load_pair(blockIdx.y, s);
  SpinorPair xv = xs.load_pair(blockIdx.y, s);
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      xv.c[k][c].re = __ffma2_rn(a, pv.c[k][c].re, xv.c[k][c].re);
      xv.c[k][c].im = __ffma2_rn(a, pv.c[k][c].im, xv.c[k][c].im);
      pv.c[k][c].re = __ffma2_rn(b, pv.c[k][c].re, rv.c[k][c].re);
      pv.c[k][c].im = __ffma2_rn(b, pv.c[k][c].im, rv.c[k][c].im);
    }
  store_active(xs, blockIdx.y, s, xv, act_a, act_b);
  store_active(p, blockIdx.y, s, pv, act_a, act_b);
}

// Pair-tiled forms of the reliable-update kernels below: thread = site x rhs
// pair, so each pair-tiled field is read once (the per-rhs forms read both
// lanes of every float4 for one rhs).  skip[r] != 0 leaves rhs r unchanged.
struct PairLanes {
  int ra;
  bool has_b, act_a, act_b;
};
__device__ __forceinline__ PairLanes pair_lanes(int pr, int nrhs, const int *skip) {
  PairLanes m;
  m.ra = 2 * pr;
  m.has_b = m.ra + 1 < nrhs;
  m.act_a = !(skip && skip[m.ra]);
  m.act_b = m.has_b && !(skip && skip[m.ra + 1]);
  return m;
}
__device__ __forceinline__ float lane_re(const CP &c, int l) { return l ? c.re.y : c.re.x; }
__device__ __forceinline__ float lane_im(const CP &c, int l) { return l ? c.im.y : c.im.x; }

// x64 += x_s / scale; x_s = 0
__global__ void k_absorb_pt(F64Acc x64, P32 xs, const double *scale, const int *skip, int nsites,
                            int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int pr = blockIdx.y;
  const PairLanes m = pair_lanes(pr, nrhs, skip);
  if (s >= nsites || (!m.act_a && !m.act_b)) return;
  const SpinorPair v = xs.load_pair(pr, s);
#pragma unroll
  for (int l = 0; l < 2; ++l) {
    if (!(l ? m.act_b : m.act_a)) continue;
    const int r = m.ra + l;
    const double w = 1.0 / scale[r];
    Spinor<double> xv = x64.load(r, s);
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        xv.c[k][c].re = fma(w, (double)lane_re(v.c[k][c], l), xv.c[k][c].re);
        xv.c[k][c].im = fma(w, (double)lane_im(v.c[k][c], l), xv.c[k][c].im);
      }
    x64.store(r, s, xv);
  }
  SpinorPair z;
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) z.c[k][c].re = z.c[k][c].im = make_float2(0.f, 0.f);
  store_active(xs, pr, s, z, m.act_a, m.act_b);
}

// sloppy <- scale * FP64
__global__ void k_to_sloppy_pt(P32 dst, F64Acc src, const double *scale, const int *skip,
                               int nsites, int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int pr = blockIdx.y;
  const PairLanes m = pair_lanes(pr, nrhs, skip);
  if (s >= nsites || (!m.act_a && !m.act_b)) return;
  SpinorPair o;
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) o.c[k][c].re = o.c[k][c].im = make_float2(0.f, 0.f);
#pragma unroll
  for (int l = 0; l < 2; ++l) {
    if (!(l ? m.act_b : m.act_a)) continue;
    const int r = m.ra + l;
    const double w = scale[r];
    const Spinor<double> v = src.load(r, s);
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float re = (float)(w * v.c[k][c].re), im = (float)(w * v.c[k][c].im);
        if (l) {
          o.c[k][c].re.y = re;
          o.c[k][c].im.y = im;
        } else {
          o.c[k][c].re.x = re;
          o.c[k][c].im.x = im;
        }
      }
  }
  store_active(dst, pr, s, o, m.act_a, m.act_b);
}

// p = p - r_s (the kept direction q, see k_dir_strip)
__global__ void k_dir_strip_pt(P32 p, P32 rs, const int *skip, int nsites, int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int pr = blockIdx.y;
  const PairLanes m = pair_lanes(pr, nrhs, skip);
  if (s >= nsites || (!m.act_a && !m.act_b)) return;
  SpinorPair pv = p.load_pair(pr, s);
  const SpinorPair rv = rs.load_pair(pr, s);
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      pv.c[k][c].re = sub2(pv.c[k][c].re, rv.c[k][c].re);
      pv.c[k][c].im = sub2(pv.c[k][c].im, rv.c[k][c].im);
    }
  store_active(p, pr, s, pv, m.act_a, m.act_b);
}

// p = (a - i b) r_s' + u q, per-lane coefficients as in k_dir_restore
__global__ void k_dir_restore_pt(P32 p, P32 rs, Scal S, const int *skip, int nsites, int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int pr = blockIdx.y;
  const PairLanes m = pair_lanes(pr, nrhs, skip);
  if (s >= nsites || (!m.act_a && !m.act_b)) return;
  float ca[2] = {1.f, 1.f}, cb[2] = {0.f, 0.f}, cu[2] = {0.f, 0.f};
#pragma unroll
  for (int l = 0; l < 2; ++l) {
    if (!(l ? m.act_b : m.act_a)) continue;
    const int r = m.ra + l;
    const double u = S.scale[r] / S.scale_prev[r];
    const double n2 = S.rr[r], cre = u * S.pAp[r], cim = u * S.alpha[r];
    const bool ok = n2 > 0 && isfinite(n2) && isfinite(cre) && isfinite(cim) && isfinite(u);
    ca[l] = (float)(ok ? 1.0 - cre / n2 : 1.0);
    cb[l] = (float)(ok ? cim / n2 : 0.0);
    cu[l] = (float)(ok ? u : 0.0);
  }
  const float2 a = make_float2(ca[0], ca[1]), b = make_float2(cb[0], cb[1]),
               uq = make_float2(cu[0], cu[1]);
  SpinorPair pv = p.load_pair(pr, s);
  const SpinorPair rv = rs.load_pair(pr, s);
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const CP x = rv.c[k][c];
      // re = uq q.re + a x.re + b x.im ; im = uq q.im + a x.im - b x.re
      float2 re = __fmul2_rn(uq, pv.c[k][c].re), im = __fmul2_rn(uq, pv.c[k][c].im);
      re = __ffma2_rn(a, x.re, re);
      re = __ffma2_rn(b, x.im, re);
      im = __ffma2_rn(a, x.im, im);
      im = __ffma2_rn(make_float2(-b.x, -b.y), x.re, im);
      pv.c[k][c].re = re;
      pv.c[k][c].im = im;
    }
  store_active(p, pr, s, pv, m.act_a, m.act_b);
}

__global__ void k_copy_pt(P32 dst, P32 src, const int *skip, int nsites, int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int pr = blockIdx.y;
  const PairLanes m = pair_lanes(pr, nrhs, skip);
  if (s >= nsites || (!m.act_a && !m.act_b)) return;
  store_active(dst, pr, s, src.load_pair(pr, s), m.act_a, m.act_b);
}

// <a, b> = sum conj(a) b per rhs, real and imaginary parts from one pass:
// blockIdx.y = pair; partials[(2 rhs + part) * kMaxRedBlocks + block]
// (part 0 real, 1 imaginary); the last block writes re[r], im[r].
__global__ void __launch_bounds__(kRedThreads)
    k_cdot_pt(P32 a, P32 b, int nsites, int nrhs, double *partials, unsigned *counters,
              const int *__restrict__ skip, double *re, double *im) {
  const int pr = blockIdx.y;
  const PairLanes m = pair_lanes(pr, nrhs, skip);
  if (!m.act_a && !m.act_b) return;
  __shared__ double sh[4][kRedThreads / 32];
  __shared__ bool last;
  double v[4] = {0.0, 0.0, 0.0, 0.0};  // re a, im a, re b, im b
  for (int s = blockIdx.x * kRedThreads + threadIdx.x; s < nsites; s += gridDim.x * kRedThreads) {
    const SpinorPair u = a.load_pair(pr, s), w = b.load_pair(pr, s);
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const CP &x = u.c[k][c], &y = w.c[k][c];
        v[0] += (double)x.re.x * y.re.x + (double)x.im.x * y.im.x;
        v[1] += (double)x.re.x * y.im.x - (double)x.im.x * y.re.x;
        v[2] += (double)x.re.y * y.re.y + (double)x.im.y * y.im.y;
        v[3] += (double)x.re.y * y.im.y - (double)x.im.y * y.re.y;
      }
  }
  block_sum<4>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q)
      partials[((size_t)2 * m.ra + q) * kMaxRedBlocks + blockIdx.x] = v[q];
    __threadfence();
    last = atomicAdd(counters + pr, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int q = 0; q < 4; ++q) v[q] = 0.0;
  for (int blk = threadIdx.x; blk < (int)gridDim.x; blk += kRedThreads)
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] += __ldcg(partials + ((size_t)2 * m.ra + q) * kMaxRedBlocks + blk);
  block_sum<4>(v, sh);
  if (threadIdx.x == 0) {
    counters[pr] = 0;
    if (m.act_a) re[m.ra] = v[0], im[m.ra] = v[1];
    if (m.act_b) re[m.ra + 1] = v[2], im[m.ra + 1] = v[3];
  }
}

// Reliable update, step 1: x64 += x_s / scale; x_s = 0 (rhs with skip[r] == 0)
template <class XF>
__global__ void k_absorb(F64Acc x64, XF xs, const double *scale, const int *skip, int nsites,
                         int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (s >= nsites || r >= nrhs || skip[r]) return;
  using RX = typename XF::R;
  const double w = 1.0 / scale[r];
  Spinor<double> xv = x64.load(r, s);
  const Spinor<RX> d = xs.load(r, s);
  Spinor<RX> z;
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      xv.c[k][c].re = fma(w, (double)d.c[k][c].re, xv.c[k][c].re);
      xv.c[k][c].im = fma(w, (double)d.c[k][c].im, xv.c[k][c].im);
      z.c[k][c] = cx((RX)0, (RX)0);
    }
  x64.store(r, s, xv);
  xs.store(r, s, z);
}

// r_hat = b_hat - y; returns |r_hat|^2
struct RedRhat {
  F64Acc bhat, y;
  __device__ double operator()(int r, int s) const {
    const Spinor<double> b = bhat.load(r, s);
    Spinor<double> v = y.load(r, s);
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) v.c[k][c] = b.c[k][c] - v.c[k][c];
    y.store(r, s, v);
    return norm2(v);
  }
};
struct EpiStore {
  double *dst;
  __device__ void operator()(int r, double t) const { dst[r] = t; }
};
// |r_hat|^2, and the new unit of the sloppy recursion
struct EpiRhat {
  Scal S;
  __device__ void operator()(int r, double t) const {
    S.rhat2[r] = t;
    S.scale_prev[r] = S.scale[r];
    S.scale[r] = (t > 0 && isfinite(t)) ? rsqrt(t) : 1.0;
  }
};

struct EpiRR {
  Scal S;
  __device__ void operator()(int r, double t) const {
    S.rr[r] = t;
    S.rn2[r] = t;
  }
};

// sloppy <- FP64 (rhs with skip[r] == 0)
template <class SF>
__global__ void k_to_sloppy(SF dst, F64Acc src, const double *scale, const int *skip, int nsites,
                            int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (s >= nsites || r >= nrhs || (skip && skip[r])) return;
  Spinor<double> v = src.load(r, s);
  const double w = scale[r];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) v.c[k][c] = w * v.c[k][c];
  dst.store(r, s, convert<typename SF::R>(v));
}

// FP64 <- sloppy (per rhs)
template <class SF>
__global__ void k_from_sloppy(F64Acc dst, SF src, int nsites, int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (s >= nsites || r >= nrhs) return;
  dst.store(r, s, convert<double>(src.load(r, s)));
}

template <class SF>
struct RedNormS {
  SF v;
  __device__ double operator()(int r, int s) const { return norm2(v.load(r, s)); }
};

// Reliable update, direction kept: before r_s is replaced, q = p - r_s
// (= beta p_prev of the last iteration) is kept in p ...
template <class SF>
__global__ void k_dir_strip(SF p, SF rs, const int *skip, int nsites, int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (s >= nsites || r >= nrhs || skip[r]) return;
  using R = typename SF::R;
  Spinor<R> pv = p.load(r, s);
  const Spinor<R> rv = rs.load(r, s);
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) pv.c[k][c] = pv.c[k][c] - rv.c[k][c];
  p.store(r, s, pv);
}

// ... and with the new residual r_s', p = r_s' + q - (<r_s', q> / |r_s'|^2) r_s':
// q is made orthogonal to r_s' again, so that <r_s', p> = |r_s'|^2 as in
// exact CG and the Krylov directions built so far are not thrown away.
template <class SF>
struct RedCdot {  // Re or Im of <a, b> = sum conj(a) b
  SF a, b;
  int imag;
  __device__ double operator()(int r, int s) const {
    const auto u = a.load(r, s), v = b.load(r, s);
    double t = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        t += imag ? (double)u.c[k][c].re * v.c[k][c].im - (double)u.c[k][c].im * v.c[k][c].re
                  : (double)u.c[k][c].re * v.c[k][c].re + (double)u.c[k][c].im * v.c[k][c].im;
    return t;
  }
};
template <class SF>
__global__ void k_dir_restore(SF p, SF rs, Scal S, const int *skip, int nsites, int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (s >= nsites || r >= nrhs || skip[r]) return;
  using R = typename SF::R;
  // q was stored in the previous unit: q' = u q with u = scale / scale_prev,
  // and <r_s', q'> = u <r_s', q> (the reductions ran on the unrescaled q)
  const double u = S.scale[r] / S.scale_prev[r];
  const double n2 = S.rr[r], cre = u * S.pAp[r], cim = u * S.alpha[r];
  const bool ok = n2 > 0 && isfinite(n2) && isfinite(cre) && isfinite(cim) && isfinite(u);
  const R a = (R)(ok ? 1.0 - cre / n2 : 1.0), b = (R)(ok ? cim / n2 : 0.0);
  const R uq = (R)(ok ? u : 0.0);
  Spinor<R> pv = p.load(r, s);
  const Spinor<R> rv = rs.load(r, s);
  // p = (a - i b) r_s' + u q
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const Cx<R> x = rv.c[k][c];
      pv.c[k][c] = uq * pv.c[k][c] + cx(a * x.re + b * x.im, a * x.im - b * x.re);
    }
  p.store(r, s, pv);
}

// copy r_s into p (restart of the direction)
template <class SF>
__global__ void k_copy(SF dst, SF src, const int *skip, int nsites, int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (s >= nsites || r >= nrhs || (skip && skip[r])) return;
  dst.store(r, s, src.load(r, s));
}

// t = D v (site-diagonal), FP64 fields
__global__ void k_diag64(F64Acc out, F64Acc in, double a, double b, int nsites, int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (s >= nsites || r >= nrhs) return;
  out.store(r, s, diag_op(a, b, in.load(r, s)));
}

// |v|^2 over the full lattice (both halves), FP64
struct RedNorm64 {
  F64Acc v;
  __device__ double operator()(int r, int s) const { return norm2(v.load(r, s)); }
};

// y = a - b on full fields
struct RedResid {
  F64Acc a, b;
  __device__ double operator()(int r, int s) const {
    const Spinor<double> u = a.load(r, s), v = b.load(r, s);
    double t = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double dr = u.c[k][c].re - v.c[k][c].re, di = u.c[k][c].im - v.c[k][c].im;
        t += dr * dr + di * di;
      }
    return t;
  }
};

}  // namespace

// ---------------------------------------------------------------------------
// Control values between host and device.  The per-rhs scalars the host
// reads every chunk and the flags it sets do not use cudaMemcpyAsync: a small
// copy shares the DMA engines with the field transfers of the solve pipeline
// and would wait behind them.  Values come back through a mapped pinned
// mailbox that a one-warp kernel writes; flags go down as kernel arguments.
// ---------------------------------------------------------------------------
namespace {

struct FlagArgs {
  int v[kMaxBatch];
};
__global__ void k_put_flags(int *__restrict__ dst, FlagArgs f, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = f.v[i];
}
__global__ void k_fetch(double *__restrict__ dst, const double *__restrict__ src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

constexpr int kMailSlots = 4;  // hb2, rr, rhat2, spare

int put_flags(cvcb_lattice *L, int *dev, const std::vector<int> &h, int n) {
  FlagArgs f{};
  for (int i = 0; i < n; ++i) f.v[i] = h[i];
  k_put_flags<<<1, 128, 0, L->stream>>>(dev, f, n);
  CVCB_LAUNCHED(L);
  return CVCB_OK;
}

// n doubles from the device into mailbox slot `slot`; the values are in
// mailbox(L, slot) once L->stream has been synchronised.
int fetch(cvcb_lattice *L, const double *dev, int n, int slot) {
  if (!L->mbox_host) {
    CVCB_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&L->mbox_host),
                            sizeof(double) * kMaxBatch * kMailSlots, cudaHostAllocMapped));
    CVCB_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void **>(&L->mbox_dev), L->mbox_host, 0));
  }
  k_fetch<<<1, 128, 0, L->stream>>>(L->mbox_dev + slot * kMaxBatch, dev, n);
  CVCB_LAUNCHED(L);
  return CVCB_OK;
}
void mailbox(cvcb_lattice *L, int slot, std::vector<double> &out, int n) {
  const volatile double *m = L->mbox_host + slot * kMaxBatch;
  for (int i = 0; i < n; ++i) out[i] = m[i];
}

}  // namespace

// ---------------------------------------------------------------------------
// The solver object for one batch
// ---------------------------------------------------------------------------
struct LaunchShape {
  int bx = 64, by = 1, nr = 1;  // sites per block, rhs groups per block, rhs per thread
  int pk = 0;                   // 1: nr == 2 in packed FP32x2 arithmetic (k_eo_hop_x2, k_eo_hop_pt);
                                // pair-tiled only: 2 k_eo_hop_ptb, 3 and 4 k_eo_hop_ptm
};

// Autotuner results, per process: (V, precision, recon, n) -> launch shape,
// (V, precision, recon, total rhs) -> right-hand sides per batch.
std::map<std::tuple<int, int, int, int>, LaunchShape> g_tuned_shape;
std::map<std::tuple<int, int, int, int>, int> g_tuned_batch;

namespace {

// Bytes of one stored spinor / link, for the algorithmic traffic model.
template <class LF>
constexpr double link_bytes();
template <> constexpr double link_bytes<L64>() { return 144; }
template <> constexpr double link_bytes<L32f>() { return 72; }
template <> constexpr double link_bytes<L32c>() { return 48; }
template <> constexpr double link_bytes<L16c>() { return 24; }
template <> constexpr double link_bytes<LT32f>() { return 72; }
template <> constexpr double link_bytes<LT32c>() { return 48; }
template <class SF>
constexpr double spinor_bytes();
template <> constexpr double spinor_bytes<F64Acc>() { return 192; }
template <> constexpr double spinor_bytes<F32Acc>() { return 96; }
template <> constexpr double spinor_bytes<F16Acc>() { return 52; }  // 48 + float norm
template <> constexpr double spinor_bytes<P32>() { return 96; }

int red_blocks_sites(int n) {
  int b = (n + kRedThreads * 2 - 1) / (kRedThreads * 2);
  return std::max(1, std::min(b, kMaxRedBlocks));
}

template <class SF, class XF, class LF>
struct Batch {
  cvcb_lattice *L;
  int n;  // rhs in this batch
  Geom g;
  LaunchShape shape;
  LaunchShape shape64;  // FP64 sweeps when the inner iterations are sloppy
  // FP64 fields: full lattice, stride V, rhs stride 12V
  double2 *b64, *x64, *t64, *y64, *bh64;
  // sloppy fields: half lattice, compact
  SF p, Ap, rs, te, yo, te2;
  XF xs;
  void *xs_mem;
  size_t xs_bytes;
  Scal S;
  // [rhs][dot_np] partials of <p, M^+M p> = |M p|^2, fused into the sweep
  // that produces M p
  double *dot_part = nullptr;
  int dot_np = 0;
  int *err = nullptr;  // set by a stencil whose staged copy did not complete
  int *ru_skip;   // per rhs: 1 = skip in the reliable update
  int *rst_skip;  // per rhs: 0 = restart the direction from the residual
  BatchRed br;
  LF links;
  L64 links64;
  double mu, kap;
  // stencil timing (instrumentation): events recorded around the sloppy
  // stencil launches of one iteration per chunk
  bool prof_rec = false;
  bool capturing = false;
  struct Rec {
    cudaEvent_t a, b;
    double bytes_per_rhs, link_bytes;
  };
  std::vector<Rec> recs;

  F64Acc f64(double2 *base, int parity) const {
    return F64Acc{base + (size_t)parity * g.Vh, (size_t)g.V, (size_t)12 * g.V};
  }
  F64Acc f64full(double2 *base) const { return F64Acc{base, (size_t)g.V, (size_t)12 * g.V}; }

  // With dot_part (packed kernel only, warp-aligned blocks), the sweep also
  // writes per-warp partials of |out|^2 (dot_np per rhs).
  template <class AF, class LL, bool G5IN, bool G5HOP, bool AUX>
  int hop(AF out, AF in, AF aux, LL lk, int parity, const int *done, double d1a, double d1b,
          double d2a, double d2b, double c, double *dot_part = nullptr) {
    HopArgs<AF, LL> a{out, in, aux, lk, EoGeom{g, parity}, n, done, d1a, d1b, d2a, d2b, c};
    if (dot_part) {
      if (!dot_fusable()) {
        set_error("fused norm needs the packed stencil with warp-aligned blocks");
        return CVCB_ERR_STATE;
      }
      a.dot_part = dot_part;
      a.dot_np = dot_parts();
      dot_np = a.dot_np;
    }
    a.err = err;
    // FP64 sweeps of a reduced-precision solve (reliable updates) have their
    // own tuned shape; FP64 kernels keep one rhs per thread (register budget).
    LaunchShape sh = sizeof(typename AF::R) == 8 && sizeof(typename SF::R) != 8 ? shape64 : shape;
    if (sizeof(typename AF::R) == 8) sh.nr = 1;
    const int groups = (n + sh.nr - 1) / sh.nr;
    const int by = std::min(sh.by, groups);
    const int site_blocks = (g.Vh + sh.bx - 1) / sh.bx;
    dim3 block(sh.bx, by), grid((groups + by - 1) / by, std::min(site_blocks, 65535));
    Rec rec{};
    const bool rec_this = prof_rec && std::is_same<AF, SF>::value;
    if (rec_this) {
      CVCB_CUDA(cudaEventCreate(&rec.a));
      CVCB_CUDA(cudaEventCreate(&rec.b));
      CVCB_CUDA(cudaEventRecordWithFlags(rec.a, L->stream, capturing ? cudaEventRecordExternal : 0));
    }
    bool packed = false;
    if constexpr (std::is_same<AF, P32>::value) {  // pair-tiled fields
      CVCB_TRY((launch_pt<LL, G5IN, G5HOP, AUX, false>(a, sh)));
      packed = true;
    } else if constexpr (sizeof(typename AF::R) == 4) {
      if (sh.pk) {  // two rhs per thread in packed FP32x2 arithmetic
        k_eo_hop_x2<AF, LL, G5IN, G5HOP, AUX><<<grid, block, 0, L->stream>>>(a);
        packed = true;
      }
    }
    if constexpr (std::is_same<AF, P32>::value) {
    } else if (packed) {
    } else if (by > 1 && sh.nr == 1) {
      // rows of the block share links staged in shared memory
      auto kern = [] {
        if constexpr (sizeof(typename AF::R) == 8)
          return k_eo_hop_staged64<LL, G5IN, G5HOP, AUX>;
        else
          return k_eo_hop_staged<AF, LL, G5IN, G5HOP, AUX>;
      }();
      const size_t smem = staged_smem_bytes<typename AF::R>(sh.bx);
      static std::atomic<unsigned long long> attr_set{0};  // per instantiation, bit per device
      const unsigned long long bit = 1ull << (L->device & 63);
      if (!(attr_set.load() & bit)) {
        CVCB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kMaxStagedSmem));
        attr_set.fetch_or(bit);
      }
      if (smem > kMaxStagedSmem) {
        set_error("staged stencil: %zu bytes of shared memory", smem);
        return CVCB_ERR_ARG;
      }
      kern<<<grid, block, smem, L->stream>>>(a);
    } else if constexpr (sizeof(typename AF::R) == 8) {
      k_eo_hop64<LL, G5IN, G5HOP, AUX><<<grid, block, 0, L->stream>>>(a);
    } else {
      switch (sh.nr) {
        case 2: k_eo_hop<AF, LL, 2, G5IN, G5HOP, AUX><<<grid, block, 0, L->stream>>>(a); break;
        case 3: k_eo_hop<AF, LL, 3, G5IN, G5HOP, AUX><<<grid, block, 0, L->stream>>>(a); break;
        case 4: k_eo_hop<AF, LL, 4, G5IN, G5HOP, AUX><<<grid, block, 0, L->stream>>>(a); break;
        default: k_eo_hop<AF, LL, 1, G5IN, G5HOP, AUX><<<grid, block, 0, L->stream>>>(a); break;
      }
    }
    if (!std::is_same<AF, P32>::value) CVCB_LAUNCHED(L);  // launch_pt counts its own
    if (rec_this) {
      CVCB_CUDA(cudaEventRecordWithFlags(rec.b, L->stream, capturing ? cudaEventRecordExternal : 0));
      rec.bytes_per_rhs = (double)g.Vh * spinor_bytes<AF>() * (AUX ? 3 : 2);
      rec.link_bytes = 4.0 * g.V * link_bytes<LL>();
      recs.push_back(rec);
    }
    return CVCB_OK;
  }

  // The last sweep of M^+M on pair-tiled fields, fused with the residual
  // update of CG: r_s -= alpha (A(-mu) yo + 1/2 g5 H_oe te2) and per-warp
  // partials of |r_s|^2 (A p itself is not stored)
  int hop_rupd(SF in, SF aux, double d2a, double d2b) {
    if constexpr (std::is_same<SF, P32>::value) {
      HopArgs<SF, LF> a{rs, in, aux, links, EoGeom{g, 1}, n, S.done, 1, 0, d2a, d2b, 0.5};
      if (!dot_fusable()) {
        set_error("fused residual update needs warp-aligned blocks");
        return CVCB_ERR_STATE;
      }
      a.dot_part = dot_part;
      a.dot_np = dot_parts();
      dot_np = a.dot_np;
      a.rup = rs;
      a.alpha = S.alpha;
      a.err = err;
      Rec rec{};
      if (prof_rec) {
        CVCB_CUDA(cudaEventCreate(&rec.a));
        CVCB_CUDA(cudaEventCreate(&rec.b));
        CVCB_CUDA(cudaEventRecordWithFlags(rec.a, L->stream, capturing ? cudaEventRecordExternal : 0));
      }
      CVCB_TRY((launch_pt<LF, false, true, true, true>(a, shape)));
      if (prof_rec) {
        CVCB_CUDA(cudaEventRecordWithFlags(rec.b, L->stream, capturing ? cudaEventRecordExternal : 0));
        // neighbours, aux, r read and r written
        rec.bytes_per_rhs = (double)g.Vh * spinor_bytes<SF>() * 4;
        rec.link_bytes = 4.0 * g.V * link_bytes<LF>();
        recs.push_back(rec);
      }
      return CVCB_OK;
    } else {
      (void)in, (void)aux, (void)d2a, (void)d2b;
      set_error("fused residual update needs pair-tiled fields");
      return CVCB_ERR_STATE;
    }
  }

  // diagonal coefficients
  double ka() const { return 0.5 / kap; }
  void ainv(double m, double &a, double &b) const {
    const double d = ka() * ka() + m * m;
    a = ka() / d;
    b = -m / d;
  }

  // <p, M^+M p> = |M p|^2 in the sweep that writes M p: the packed FP32x2
  // kernels with blocks a multiple of a warp wide
  bool dot_fusable() const {
    return sizeof(typename SF::R) == 4 && shape.pk >= 1 && shape.bx % 32 == 0;
  }
  // partial sums per rhs of the fused norms: one per warp of the site blocks
  // (one per 32-site tile for the bulk-staged stencil)
  int dot_parts() const {
    if (shape.pk == 2) return g.Vh / kTile;
    return ((g.Vh + shape.bx - 1) / shape.bx) * (shape.bx / 32);
  }

  // Pair-tiled stencil launch: pk 2 = bulk-staged t and x neighbours
  // (k_eo_hop_ptb, whole-tile lattices only), pk 3, 4 = accumulator in
  // tensor memory (k_eo_hop_ptm, 24 warps per SM / next direction's loads in
  // flight), else plain loads (k_eo_hop_pt)
  template <class LL, bool G5IN, bool G5HOP, bool AUX, bool RUPD>
  int launch_pt(const HopArgs<P32, LL> &a, const LaunchShape &sh) {
    const int groups = (n + 1) / 2;
    if (sh.pk == 2) {
      if (!bulk_stencil_ok(g) || !a.err) {
        set_error("bulk-staged stencil needs LY*LZ/2 a multiple of 32");
        return CVCB_ERR_ARG;
      }
      auto kern = k_eo_hop_ptb<LL, G5IN, G5HOP, AUX, RUPD>;
      static std::atomic<unsigned long long> attr_set{0};  // per instantiation, bit per device
      const unsigned long long bit = 1ull << (L->device & 63);
      if (!(attr_set.load() & bit)) {
        CVCB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kBulkSmem));
        attr_set.fetch_or(bit);
      }
      const int tiles = g.Vh / kTile;
      dim3 grid(groups, std::min((tiles + kBulkWarps - 1) / kBulkWarps, 65535));
      kern<<<grid, kBulkWarps * 32, kBulkSmem, L->stream>>>(a);
    } else {
      const int by = std::min(sh.by, groups);
      const int site_blocks = (g.Vh + sh.bx - 1) / sh.bx;
      dim3 block(sh.bx, by), grid((groups + by - 1) / by, std::min(site_blocks, 65535));
      if (sh.pk == 3 || sh.pk == 4) {  // accumulator in tensor memory: 128 sites, one pair per block
        if (sh.bx != kTmemThreads || sh.by != 1) {
          set_error("tensor-memory stencil needs 128 sites and one rhs pair per block");
          return CVCB_ERR_ARG;
        }
        if (sh.pk == 3)
          k_eo_hop_ptm<LL, G5IN, G5HOP, AUX, RUPD, false><<<grid, kTmemThreads, 0, L->stream>>>(a);
        else
          k_eo_hop_ptm<LL, G5IN, G5HOP, AUX, RUPD, true><<<grid, kTmemThreads, 0, L->stream>>>(a);
      } else {
        k_eo_hop_pt<LL, G5IN, G5HOP, AUX, RUPD><<<grid, block, 0, L->stream>>>(a);
      }
    }
    CVCB_LAUNCHED(L);
    return CVCB_OK;
  }

  // out_o = M^+ M in_o with sloppy fields (te, yo, te2 as intermediates);
  // with dot_part, per-warp partials of <in, M^+M in> = |M in|^2 as well,
  // taken in the sweep that writes M in (no extra field read)
  int normal_op_sloppy(SF out, SF in, const int *done, double *dot_part = nullptr) {
    double ia, ib, ja, jb;
    ainv(mu, ia, ib);
    ainv(-mu, ja, jb);
    // K1: te = A^-1(mu) (-1/2 H_eo in)
    CVCB_TRY((hop<SF, LF, false, false, false>(te, in, in, links, 0, done, ia, ib, 0, 0, -0.5)));
    // K2: yo = A(mu) in + 1/2 H_oe te  (= M in)
    CVCB_TRY((hop<SF, LF, false, false, true>(yo, te, in, links, 1, done, 1, 0, ka(), mu, 0.5,
                                              dot_part)));
    // K1': te2 = A^-1(-mu) (-1/2 H_eo g5 yo)
    CVCB_TRY((hop<SF, LF, true, false, false>(te2, yo, yo, links, 0, done, ja, jb, 0, 0, -0.5)));
    // K2': out = A(-mu) yo + 1/2 g5 H_oe te2
    return hop<SF, LF, false, true, true>(out, te2, yo, links, 1, done, 1, 0, ka(), -mu, 0.5);
  }

  // one CG iteration (sloppy)
  int iteration() {
    if constexpr (std::is_same<SF, P32>::value) {
      // pair-tiled fields: alpha = |r|^2 / |M p|^2 between the two
      // applications of M, and the last sweep updates r itself
      const int np = (n + 1) / 2;
      double ia, ib, ja, jb;
      ainv(mu, ia, ib);
      ainv(-mu, ja, jb);
      CVCB_TRY((hop<SF, LF, false, false, false>(te, p, p, links, 0, S.done, ia, ib, 0, 0, -0.5)));
      CVCB_TRY((hop<SF, LF, false, false, true>(yo, te, p, links, 1, S.done, 1, 0, ka(), mu, 0.5,
                                                dot_part)));
      k_dot_finish<<<n, kRedThreads, 0, L->stream>>>(dot_part, dot_np, EpiAlphaB{S}, S.done);
      CVCB_LAUNCHED(L);
      CVCB_TRY((hop<SF, LF, true, false, false>(te2, yo, yo, links, 0, S.done, ja, jb, 0, 0, -0.5)));
      CVCB_TRY(hop_rupd(te2, yo, ka(), -mu));
      k_dot_finish<<<n, kRedThreads, 0, L->stream>>>(dot_part, dot_np, EpiBetaB{S}, S.done);
      CVCB_LAUNCHED(L);
      k_p_upd_pt<<<dim3((g.Vh + 127) / 128, np), 128, 0, L->stream>>>(p, rs, xs, S, g.Vh, n);
      CVCB_LAUNCHED(L);
      return CVCB_OK;
    }
    dim3 rg(red_blocks_sites(g.Vh), n);
    if (dot_fusable()) {
      CVCB_TRY(normal_op_sloppy(Ap, p, S.done, dot_part));
      k_dot_finish<<<n, kRedThreads, 0, L->stream>>>(dot_part, dot_np, EpiAlphaB{S}, S.done);
    } else {
      CVCB_TRY(normal_op_sloppy(Ap, p, S.done));
      k_reduce_rhs<<<rg, kRedThreads, 0, L->stream>>>(RedPAp<SF>{p, Ap}, EpiAlphaB{S}, g.Vh, br,
                                                      S.done);
    }
    CVCB_LAUNCHED(L);
    k_reduce_rhs<<<rg, kRedThreads, 0, L->stream>>>(RedUpdate<SF>{Ap, rs, S},
                                                    EpiBetaB{S}, g.Vh, br, S.done);
    CVCB_LAUNCHED(L);
    dim3 eg((g.Vh + 127) / 128, n);
    k_p_upd<<<eg, 128, 0, L->stream>>>(p, rs, xs, S, g.Vh, n);
    CVCB_LAUNCHED(L);
    return CVCB_OK;
  }

  // FP64: out_o = M(m) in_o  (t64 even half as intermediate)
  int schur64(double2 *out, double2 *in, double m, const int *skip) {
    double ia, ib;
    ainv(m, ia, ib);
    CVCB_TRY((hop<F64Acc, L64, false, false, false>(f64(t64, 0), f64(in, 1), f64(in, 1), links64, 0,
                                                    skip, ia, ib, 0, 0, -0.5)));
    return hop<F64Acc, L64, false, false, true>(f64(out, 1), f64(t64, 0), f64(in, 1), links64, 1,
                                                skip, 1, 0, ka(), m, 0.5);
  }
  // sloppy: out_o = M(mu)^+ in_o = g5 M(-mu) g5 in_o (te2 as intermediate)
  int dag_sloppy(SF out, SF in, const int *skip) {
    double ja, jb;
    ainv(-mu, ja, jb);
    CVCB_TRY((hop<SF, LF, true, false, false>(te2, in, in, links, 0, skip, ja, jb, 0, 0, -0.5)));
    return hop<SF, LF, false, true, true>(out, te2, in, links, 1, skip, 1, 0, ka(), -mu, 0.5);
  }

  // Reliable update (rhs with ru_skip[r] == 0): x64 += x_s; r_hat = b_hat - M x64
  // and |r_hat|^2 in FP64 with the exact operator (the convergence criterion);
  // then the sloppy recursion restarts from r_s = M^+ r_hat, which only feeds
  // the sloppy iterations and is therefore formed in sloppy precision.
  // absorb = false is the start from x = 0, where M x = 0 needs no sweep.
  int reliable_update(bool absorb) {
    dim3 eg((g.Vh + 127) / 128, n);
    if (absorb) {
      if constexpr (std::is_same<XF, P32>::value)
        k_absorb_pt<<<dim3(eg.x, (n + 1) / 2), 128, 0, L->stream>>>(f64(x64, 1), xs, S.scale,
                                                                    ru_skip, g.Vh, n);
      else
        k_absorb<<<eg, 128, 0, L->stream>>>(f64(x64, 1), xs, S.scale, ru_skip, g.Vh, n);
      CVCB_LAUNCHED(L);
      CVCB_TRY(schur64(y64, x64, mu, ru_skip));
    } else {
      CVCB_CUDA(cudaMemsetAsync(y64, 0, (size_t)12 * g.V * sizeof(double2) * n, L->stream));
    }
    dim3 rg(red_blocks_sites(g.Vh), n);
    k_reduce_rhs<<<rg, kRedThreads, 0, L->stream>>>(RedRhat{f64(bh64, 1), f64(y64, 1)},
                                                    EpiRhat{S}, g.Vh, br, ru_skip);
    CVCB_LAUNCHED(L);
    if constexpr (std::is_same<SF, P32>::value)
      k_to_sloppy_pt<<<dim3(eg.x, (n + 1) / 2), 128, 0, L->stream>>>(yo, f64(y64, 1), S.scale,
                                                                      ru_skip, g.Vh, n);
    else
      k_to_sloppy<<<eg, 128, 0, L->stream>>>(yo, f64(y64, 1), S.scale, ru_skip, g.Vh, n);
    CVCB_LAUNCHED(L);
    CVCB_TRY(dag_sloppy(rs, yo, ru_skip));
    k_reduce_rhs<<<rg, kRedThreads, 0, L->stream>>>(RedNormS<SF>{rs}, EpiRR{S}, g.Vh, br, ru_skip);
    CVCB_LAUNCHED(L);
    return CVCB_OK;
  }
};

template <class SF>
SF make_sloppy(void *base, size_t Vh, int r_count, float *norm_base);

template <>
F32Acc make_sloppy<F32Acc>(void *base, size_t Vh, int, float *) {
  return F32Acc{static_cast<float4 *>(base), Vh, 6 * Vh};
}
template <>
F16Acc make_sloppy<F16Acc>(void *base, size_t Vh, int, float *norm) {
  return F16Acc{static_cast<uint4 *>(base), norm, Vh, 3 * Vh};
}
template <>
F64Acc make_sloppy<F64Acc>(void *base, size_t Vh, int, float *) {
  return F64Acc{static_cast<double2 *>(base), Vh, 12 * Vh};
}
template <>
P32 make_sloppy<P32>(void *base, size_t Vh, int, float *) {
  return P32{static_cast<float4 *>(base), p32_pair_float4((int)Vh)};
}

template <class SF>
size_t sloppy_site_bytes();
template <>
size_t sloppy_site_bytes<F32Acc>() { return 96; }
template <>
size_t sloppy_site_bytes<F16Acc>() { return 48; }
template <>
size_t sloppy_site_bytes<F64Acc>() { return 192; }
template <>
size_t sloppy_site_bytes<P32>() { return 96; }

// Bytes of one sloppy field set of n right-hand sides (pair-tiled sets hold
// whole pairs of whole tiles).
template <class SF>
size_t sloppy_field_bytes(size_t Vh, int n) {
  if (std::is_same<SF, P32>::value) return p32_pair_float4((int)Vh) * sizeof(float4) * ((n + 1) / 2);
  return sloppy_site_bytes<SF>() * Vh * n;
}

template <class LF>
LF make_links(cvcb_lattice *L);
template <>
L64 make_links<L64>(cvcb_lattice *L) {
  L64 l{L->U64, (size_t)L->g.V, {}};
  for (int m = 0; m < 4; ++m) l.ph[m] = make_double2(L->phase[2 * m], L->phase[2 * m + 1]);
  return l;
}
// e^{3 i theta_mu}: row 2 of a phased SU(3) link W = e^{i theta} U is
// e^{3 i theta} conj(W_0 x W_1)
static float2 phase_cubed(const cvcb_lattice *L, int m) {
  const double c = L->phase[2 * m], d = L->phase[2 * m + 1];
  const double c2 = c * c - d * d, d2 = 2 * c * d;
  return make_float2((float)(c2 * c - d2 * d), (float)(c2 * d + d2 * c));
}
template <>
L32c make_links<L32c>(cvcb_lattice *L) {
  L32c l{L->U32c, (size_t)L->g.V, {}};
  for (int m = 0; m < 4; ++m) l.ph[m] = phase_cubed(L, m);
  return l;
}
template <>
L32f make_links<L32f>(cvcb_lattice *L) {
  L32f l{L->U32f, (size_t)L->g.V, {}};
  for (int m = 0; m < 4; ++m) l.ph[m] = make_float2((float)L->phase[2 * m], (float)L->phase[2 * m + 1]);
  return l;
}
template <>
LT32f make_links<LT32f>(cvcb_lattice *L) {
  return LT32f{L->UT32f, {}};
}
template <>
LT32c make_links<LT32c>(cvcb_lattice *L) {
  LT32c l{L->UT32c, {}};
  for (int m = 0; m < 4; ++m) l.ph[m] = phase_cubed(L, m);
  return l;
}
template <>
L16c make_links<L16c>(cvcb_lattice *L) {
  L16c l{L->U16c, (size_t)L->g.V, {}};
  for (int m = 0; m < 4; ++m) l.ph[m] = phase_cubed(L, m);
  return l;
}

// Device memory of one batch of n right-hand sides.
struct BatchMem {
  size_t f64_bytes, sl_bytes, norm_bytes;
  char *base = nullptr;
};

template <class SF, class XF, class LF>
int setup_batch(cvcb_lattice *L, Batch<SF, XF, LF> &B, int n, bool with_fp64 = true) {
  const Geom &g = L->g;
  B.L = L;
  B.n = n;
  B.g = g;
  B.mu = L->mu;
  B.kap = L->kappa;
  B.links = make_links<LF>(L);
  B.links64 = make_links<L64>(L);
  // one FP64 full field set (none when only the sloppy stencil is timed)
  const size_t f64 = with_fp64 ? (size_t)12 * g.V * sizeof(double2) * n : 0;
  const size_t sl = sloppy_field_bytes<SF>(g.Vh, n);
  const size_t xsl = sloppy_field_bytes<XF>(g.Vh, n);
  const size_t nrm = sizeof(float) * (size_t)g.Vh * n;
  auto rnd = [](size_t b) { return (b + 255) & ~size_t(255); };  // every piece 256-aligned
  const size_t scal = 8 * rnd(sizeof(double) * kMaxBatch) + 3 * rnd(sizeof(int) * kMaxBatch);
  const size_t part = rnd(sizeof(double) * kMaxRedBlocks * kMaxBatch * 2) +
                      rnd(sizeof(unsigned) * kMaxBatch);
  const size_t dotb = sizeof(double) * (size_t)n * (g.Vh / 32 + 64);
  const size_t total = 5 * rnd(f64) + 6 * (rnd(sl) + rnd(nrm)) + rnd(xsl) + rnd(nrm) + scal + part +
                       rnd(dotb) + rnd(sizeof(int));
  void *mem;
  CVCB_TRY(ensure_buffer(L, SLOT_MIX0, total, &mem));
  char *p = static_cast<char *>(mem);
  auto take = [&](size_t bytes) {
    char *q = p;
    p += rnd(bytes);
    return q;
  };
  B.b64 = (double2 *)take(f64);
  B.x64 = (double2 *)take(f64);
  B.t64 = (double2 *)take(f64);
  B.y64 = (double2 *)take(f64);
  B.bh64 = (double2 *)take(f64);
  SF *sl_fields[6] = {&B.p, &B.Ap, &B.rs, &B.te, &B.yo, &B.te2};
  for (SF *f : sl_fields) {
    void *b = take(sl);
    float *nb = (float *)take(nrm);
    *f = make_sloppy<SF>(b, g.Vh, n, nb);
  }
  {
    void *b = take(xsl);
    float *nb = (float *)take(nrm);
    B.xs = make_sloppy<XF>(b, g.Vh, n, nb);
    B.xs_mem = b;
    B.xs_bytes = xsl;
  }
  B.S.rr = (double *)take(sizeof(double) * kMaxBatch);
  B.S.pAp = (double *)take(sizeof(double) * kMaxBatch);
  B.S.alpha = (double *)take(sizeof(double) * kMaxBatch);
  B.S.beta = (double *)take(sizeof(double) * kMaxBatch);
  B.S.rhat2 = (double *)take(sizeof(double) * kMaxBatch);
  B.S.rn2 = (double *)take(sizeof(double) * kMaxBatch);
  B.S.scale = (double *)take(sizeof(double) * kMaxBatch);
  B.S.scale_prev = (double *)take(sizeof(double) * kMaxBatch);
  B.S.done = (int *)take(sizeof(int) * kMaxBatch);
  B.ru_skip = (int *)take(sizeof(int) * kMaxBatch);
  B.rst_skip = (int *)take(sizeof(int) * kMaxBatch);
  B.br.partials = (double *)take(sizeof(double) * kMaxRedBlocks * kMaxBatch * 2);
  B.br.counters = (unsigned *)take(sizeof(unsigned) * kMaxBatch);
  B.dot_part = (double *)take(dotb);
  B.err = (int *)take(sizeof(int));
  CVCB_CUDA(cudaMemsetAsync(B.err, 0, sizeof(int), L->stream));
  CVCB_CUDA(cudaMemsetAsync(B.br.counters, 0, sizeof(unsigned) * kMaxBatch, L->stream));
  CVCB_CUDA(cudaMemsetAsync(B.S.done, 0, sizeof(int) * kMaxBatch, L->stream));
  CVCB_CUDA(cudaMemsetAsync(B.ru_skip, 0, sizeof(int) * kMaxBatch, L->stream));
  CVCB_CUDA(cudaMemsetAsync(B.S.scale, 0, 2 * rnd(sizeof(double) * kMaxBatch), L->stream));
  return CVCB_OK;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Times `fn` (which enqueues work on L->stream) with CUDA events, best of reps.
template <class Fn>
int time_ms(cvcb_lattice *L, Fn fn, int reps, float *best) {
  cudaEvent_t a, b;
  CVCB_CUDA(cudaEventCreate(&a));
  CVCB_CUDA(cudaEventCreate(&b));
  *best = 1e30f;
  for (int i = 0; i < reps; ++i) {
    CVCB_CUDA(cudaEventRecord(a, L->stream));
    CVCB_TRY(fn());
    CVCB_CUDA(cudaEventRecord(b, L->stream));
    CVCB_CUDA(cudaEventSynchronize(b));
    float ms;
    CVCB_CUDA(cudaEventElapsedTime(&ms, a, b));
    *best = std::min(*best, ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return CVCB_OK;
}

// Autotuner for the stencil launch shape: sites per block x right-hand sides
// per block, timed on the sloppy normal operator.
template <class SF, class XF, class LF>
int tune_shape(cvcb_lattice *L, Batch<SF, XF, LF> &B, int prec, int recon, int block_threads = 0) {
  if (block_threads > 0) {  // caller's choice: that many sites per block, one rhs (pair) per thread
    B.shape = std::is_same<SF, P32>::value ? LaunchShape{block_threads, 1, 2, 1}
                                           : LaunchShape{block_threads, 1, 1};
    return CVCB_OK;
  }
  constexpr bool pairs = std::is_same<SF, P32>::value;
  auto key = std::make_tuple(L->g.V, prec + (pairs ? kPairKey : 0), recon, B.n);
  auto it = g_tuned_shape.find(key);
  if (it != g_tuned_shape.end()) {
    B.shape = it->second;
    return CVCB_OK;
  }
  // CVCB_SHAPE="sites,rows,rhs_per_thread[,packed]" pins the shape
  // (reproducible runs, profiling); otherwise every admissible shape is timed.
  if (const char *env = getenv("CVCB_SHAPE")) {
    LaunchShape f;
    const int nf = sscanf(env, "%d,%d,%d,%d", &f.bx, &f.by, &f.nr, &f.pk);
    if (nf >= 3 && f.bx > 0 && f.by > 0 && f.nr >= 1 && f.nr <= 4 &&
        f.bx * f.by <= kHopMaxThreads) {
      if (nf < 4 || f.nr != 2) f.pk = 0;
      if (sizeof(typename SF::R) == 8) f.nr = 1, f.pk = 0;
      if (pairs) {  // pair-tiled fields: one rhs pair per thread; 4th field 2 = bulk-staged
        f.nr = 2;
        f.pk = (nf >= 4 && f.pk == 2 && bulk_stencil_ok(L->g)) ? 2
               : (nf >= 4 && (f.pk == 3 || f.pk == 4))           ? f.pk
                                                                 : 1;
        if (f.pk == 2) f.bx = kBulkWarps * 32, f.by = 1;
        if (f.pk >= 3) f.bx = kTmemThreads, f.by = 1;
      }
      B.shape = f;
      g_tuned_shape[key] = f;
      return CVCB_OK;
    }
  }
  // a pair-tiled batch always has a valid shape: one pair per thread, even
  // for a single right-hand side (the second lane of its pair idles)
  LaunchShape best = pairs ? LaunchShape{64, 1, 2, 1} : LaunchShape{};
  float best_ms = 1e30f;
  const int bxs[] = {32, 64, 128, 256};
  const int bys[] = {1, 2, 3, 4, 6};
  // (rhs per thread, packed): 2 rhs per thread either as two unpacked
  // spinors or as FP32x2 pairs
  const int nrs[][2] = {{1, 0}, {2, 0}, {3, 0}, {4, 0}, {2, 1}};
  const bool fp64 = sizeof(typename SF::R) == 8;
  for (const auto &np : nrs)
    for (int bx : bxs)
    for (int by : bys) {
      const int nr = np[0];
      if (fp64 && nr > 1) continue;
      if (pairs && !(nr == 2 && np[1] == 1)) continue;
      if (bx * by > kHopMaxThreads || bx * by < 32) continue;
      if (pairs ? by > (B.n + 1) / 2 : (nr > B.n || by * nr > B.n)) continue;
      B.shape.bx = bx;
      B.shape.by = by;
      B.shape.nr = nr;
      B.shape.pk = np[1];
      float ms;
      if (time_ms(L, [&] { return B.normal_op_sloppy(B.Ap, B.p, nullptr); }, 3, &ms) != CVCB_OK) {
        cudaGetLastError();
        continue;
      }
      if (ms < best_ms) {
        best_ms = ms;
        best = B.shape;
      }
    }
  if (pairs) {  // the tensor-memory accumulator: one fixed block shape, two register budgets
    for (int pk : {3, 4}) {
      B.shape = LaunchShape{kTmemThreads, 1, 2, pk};
      float ms;
      if (time_ms(L, [&] { return B.normal_op_sloppy(B.Ap, B.p, nullptr); }, 3, &ms) != CVCB_OK) {
        cudaGetLastError();
      } else if (ms < best_ms) {
        best_ms = ms;
        best = B.shape;
      }
    }
  }
  if (pairs && bulk_stencil_ok(L->g)) {  // the bulk-staged stencil: one fixed block shape
    B.shape = LaunchShape{kBulkWarps * 32, 1, 2, 2};
    float ms;
    if (time_ms(L, [&] { return B.normal_op_sloppy(B.Ap, B.p, nullptr); }, 3, &ms) != CVCB_OK) {
      cudaGetLastError();
    } else if (ms < best_ms) {
      best_ms = ms;
      best = B.shape;
    }
  }
  B.shape = best;
  g_tuned_shape[key] = best;
  return CVCB_OK;
}

// Shape of the FP64 sweeps of the reliable updates in a reduced-precision
// solve, timed on M(mu) in FP64 (two sweeps).
template <class SF, class XF, class LF>
int tune_shape64(cvcb_lattice *L, Batch<SF, XF, LF> &B) {
  auto key = std::make_tuple(L->g.V, -1, 18, B.n);
  auto it = g_tuned_shape.find(key);
  if (it != g_tuned_shape.end()) {
    B.shape64 = it->second;
    return CVCB_OK;
  }
  const LaunchShape cands[] = {{64, 1, 1}, {128, 1, 1}, {32, 2, 1}, {64, 2, 1}, {32, 3, 1},
                               {32, 4, 1}, {16, 4, 1}, {16, 8, 1}, {16, 6, 1}};
  LaunchShape best{64, 1, 1};
  float best_ms = 1e30f;
  for (const LaunchShape &c : cands) {
    B.shape64 = c;
    float ms;
    if (time_ms(L, [&] { return B.schur64(B.y64, B.x64, B.mu, nullptr); }, 3, &ms) != CVCB_OK) {
      cudaGetLastError();
      continue;
    }
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  B.shape64 = best;
  g_tuned_shape[key] = best;
  return CVCB_OK;
}

template <class SF, class XF, class LF>
int run_batch(cvcb_lattice *L, double *const *x, const double *const *b, int n,
              const cvcb_solver_params *P, cvcb_solver_stats *st, LaunchShape *shape_out,
              cudaEvent_t inputs_read = nullptr) {
  Batch<SF, XF, LF> B;
  CVCB_TRY(setup_batch(L, B, n));
  const Geom &g = L->g;
  const size_t fs = (size_t)12 * g.V;
  dim3 eg((g.Vh + 127) / 128, n);
  dim3 egf((g.V + 127) / 128, n);
  dim3 rg(red_blocks_sites(g.Vh), n), rgf(red_blocks_sites(g.V), n);

  for (int i = 0; i < n; ++i) CVCB_TRY(spinor_in(L, B.b64 + i * fs, b[i], g.V));
  if (inputs_read) CVCB_CUDA(cudaEventRecord(inputs_read, L->stream));
  CVCB_TRY(tune_shape(L, B, P->precision, P->link_recon, P->block_threads));
  if (sizeof(typename SF::R) != 8) CVCB_TRY(tune_shape64(L, B));
  if (shape_out) *shape_out = B.shape;

  // |b|^2 over the full lattice
  double *bnorm2 = B.S.rn2;  // temporary use
  k_reduce_rhs<<<rgf, kRedThreads, 0, L->stream>>>(RedNorm64{B.f64full(B.b64)},
                                                   EpiStore{bnorm2}, g.V, B.br, nullptr);
  CVCB_LAUNCHED(L);
  std::vector<double> hb2(n);
  CVCB_TRY(fetch(L, bnorm2, n, 0));
  // b_hat = b_o + 1/2 H_oe A_ee^-1 b_e
  double ia, ib;
  B.ainv(B.mu, ia, ib);
  k_diag64<<<eg, 128, 0, L->stream>>>(B.f64(B.t64, 0), B.f64(B.b64, 0), ia, ib, g.Vh, n);
  CVCB_LAUNCHED(L);
  CVCB_TRY((B.template hop<F64Acc, L64, false, false, true>(B.f64(B.bh64, 1), B.f64(B.t64, 0),
                                                            B.f64(B.b64, 1), B.links64, 1,
                                                            nullptr, 1, 0, 1, 0, 0.5)));
  // x = 0, x_s = 0; reliable update from x = 0 gives r_hat = b_hat, r_N = b_N
  CVCB_CUDA(cudaMemsetAsync(B.x64, 0, fs * n * sizeof(double2), L->stream));
  CVCB_TRY(B.reliable_update(false));
  // x_s = 0 (all-zero bits are 0.0), p = r_s
  CVCB_CUDA(cudaMemsetAsync(B.xs_mem, 0, B.xs_bytes, L->stream));
  if constexpr (std::is_same<SF, P32>::value)
    k_copy_pt<<<dim3(eg.x, (n + 1) / 2), 128, 0, L->stream>>>(B.p, B.rs, nullptr, g.Vh, n);
  else
    k_copy<<<eg, 128, 0, L->stream>>>(B.p, B.rs, nullptr, g.Vh, n);
  CVCB_LAUNCHED(L);
  std::vector<double> rr(n), rr_max(n), rhat2(n), ratio2(n), target2(n);
  std::vector<int> done(n, 0), iters(n, 0), since(n, 0), skip(n, 0), rst(n, 1);
  CVCB_TRY(fetch(L, B.S.rr, n, 1));
  CVCB_TRY(fetch(L, B.S.rhat2, n, 2));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  mailbox(L, 0, hb2, n);
  mailbox(L, 1, rr, n);
  mailbox(L, 2, rhat2, n);
  const double margin = 0.5;
  for (int i = 0; i < n; ++i) {
    target2[i] = std::pow(P->tol * margin, 2) * hb2[i];
    rr_max[i] = rr[i];
    ratio2[i] = rhat2[i] > 0 ? rr[i] / rhat2[i] : 1.0;
    if (!(hb2[i] > 0)) done[i] = 1;  // zero right-hand side: x = 0
    else if (rhat2[i] <= target2[i]) done[i] = 1;
  }
  CVCB_TRY(put_flags(L, B.S.done, done, n));

  // One CG iteration is captured in a CUDA graph; between two host checks the
  // graph is launched k times, k <= kmax, with k cut to the number of
  // iterations each rhs is predicted to need (from its measured convergence
  // rate) so that the last chunk does not overshoot convergence.
  const int kmax = 10;
  // The executable graph and the stencil timing events are released on every
  // exit path, early error returns included.
  struct Release {
    cudaGraphExec_t exec = nullptr;
    std::vector<typename Batch<SF, XF, LF>::Rec> *recs = nullptr;
    ~Release() {
      if (exec) cudaGraphExecDestroy(exec);
      if (recs) {
        for (auto &r : *recs) {
          cudaEventDestroy(r.a);
          cudaEventDestroy(r.b);
        }
        recs->clear();
      }
    }
  } release;
  release.recs = &B.recs;
  cudaGraphExec_t &gexec = release.exec;
  long long graph_nodes = 0;
  if (P->use_graph) {
    cudaGraph_t graph = nullptr;
    const long long before = L->nlaunch;
    CVCB_CUDA(cudaStreamBeginCapture(L->stream, cudaStreamCaptureModeThreadLocal));
    B.capturing = true;
    B.prof_rec = L->prof;
    int rc = B.iteration();
    B.prof_rec = false;
    B.capturing = false;
    cudaError_t ec = cudaStreamEndCapture(L->stream, &graph);
    if (rc != CVCB_OK || ec != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      if (rc != CVCB_OK) return rc;
      CVCB_CUDA(ec);
    }
    ec = cudaGraphInstantiate(&gexec, graph, 0);
    cudaGraphDestroy(graph);
    CVCB_CUDA(ec);
    graph_nodes = L->nlaunch - before;  // kernels per graph launch
    L->nlaunch = before;
  }
  auto harvest = [&](int active) -> int {
    // per-launch device time of the recorded stencil launches (instrumentation)
    for (auto &r : B.recs) {
      float ms;
      CVCB_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
      L->prof_ms += ms;
      L->prof_launches += 1;
      L->prof_bytes += r.bytes_per_rhs * active + r.link_bytes;
    }
    if (!gexec) {
      for (auto &r : B.recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
      }
      B.recs.clear();
    }
    return CVCB_OK;
  };

  // delta 0: by the storage of the inner iterations -- an FP16 recursion
  // drifts from the true residual after about three decades, FP32 after six
  const double delta = P->delta > 0 ? P->delta
                       : std::is_same<SF, F16Acc>::value ? 0.1
                       : sizeof(typename SF::R) == 4 ? 1e-4 : 1e-8;
  const double delta2 = delta * delta;
  int total_iter = 0, nru = 0, nrestart = 0;
  // rr at the previous check (same units) and the measured per-iteration
  // factor of rr (0 = not known yet)
  std::vector<double> rr_ref(rr), rate(n, 0.0);
  const double t0 = now_s();
  int rc = CVCB_OK;
  while (true) {
    bool all = true;
    for (int i = 0; i < n; ++i) all = all && done[i];
    if (all) break;
    if (total_iter >= P->max_iter) break;
    int active = 0;
    for (int i = 0; i < n; ++i) active += !done[i];
    int chunk = std::min(kmax, P->max_iter - total_iter);
    for (int i = 0; i < n; ++i) {
      if (done[i] || !(rate[i] > 0 && rate[i] < 1) || !(rr[i] > 0)) continue;
      const double need = std::log(target2[i] * ratio2[i] / rr[i]) / std::log(rate[i]);
      if (std::isfinite(need)) chunk = std::min(chunk, std::max(1, (int)std::ceil(need)));
    }
    if (gexec) {
      for (int k = 0; k < chunk && rc == CVCB_OK; ++k) {
        cudaError_t e = cudaGraphLaunch(gexec, L->stream);
        if (e != cudaSuccess) {
          set_error("graph launch: %s", cudaGetErrorString(e));
          rc = CVCB_ERR_CUDA;
        }
        L->nlaunch += graph_nodes;
      }
      if (rc != CVCB_OK) break;
    } else {
      for (int k = 0; k < chunk; ++k) {
        B.prof_rec = L->prof && k == 0;
        if ((rc = B.iteration()) != CVCB_OK) break;
      }
      B.prof_rec = false;
      if (rc != CVCB_OK) break;
    }
    total_iter += chunk;
    CVCB_TRY(fetch(L, B.S.rr, n, 1));
    CVCB_CUDA(cudaStreamSynchronize(L->stream));
    mailbox(L, 1, rr, n);
    if (L->prof) CVCB_TRY(harvest(active));
    bool any = false;
    for (int i = 0; i < n; ++i) {
      skip[i] = 1;
      if (done[i]) continue;
      iters[i] += chunk;
      since[i] += chunk;
      if (std::isfinite(rr[i]) && rr[i] > 0 && rr_ref[i] > 0 && rr[i] < rr_ref[i])
        rate[i] = std::pow(rr[i] / rr_ref[i], 1.0 / chunk);
      rr_ref[i] = rr[i];
      const bool bad = !std::isfinite(rr[i]);
      const bool dropped = rr[i] < delta2 * rr_max[i];
      const bool near = rr[i] / ratio2[i] < target2[i];
      if (bad || dropped || near || since[i] >= 1000) {
        skip[i] = 0;
        any = true;
      }
    }
    if (!any) continue;
    CVCB_TRY(put_flags(L, B.ru_skip, skip, n));
    // keep the search direction: q = p - r_s now, p = r_s' + q (q orthogonalised
    // against r_s') after the update
    const dim3 egp(eg.x, (n + 1) / 2);  // pair-tiled fields: one thread per site and pair
    if constexpr (std::is_same<SF, P32>::value)
      k_dir_strip_pt<<<egp, 128, 0, L->stream>>>(B.p, B.rs, B.ru_skip, g.Vh, n);
    else
      k_dir_strip<<<eg, 128, 0, L->stream>>>(B.p, B.rs, B.ru_skip, g.Vh, n);
    CVCB_LAUNCHED(L);
    CVCB_TRY(B.reliable_update(true));
    if constexpr (std::is_same<SF, P32>::value) {
      k_cdot_pt<<<dim3(rg.x, (n + 1) / 2), kRedThreads, 0, L->stream>>>(
          B.rs, B.p, g.Vh, n, B.br.partials, B.br.counters, B.ru_skip, B.S.pAp, B.S.alpha);
      CVCB_LAUNCHED(L);
      k_dir_restore_pt<<<egp, 128, 0, L->stream>>>(B.p, B.rs, B.S, B.ru_skip, g.Vh, n);
    } else {
      k_reduce_rhs<<<rg, kRedThreads, 0, L->stream>>>(RedCdot<SF>{B.rs, B.p, 0},
                                                      EpiStore{B.S.pAp}, g.Vh, B.br, B.ru_skip);
      CVCB_LAUNCHED(L);
      k_reduce_rhs<<<rg, kRedThreads, 0, L->stream>>>(RedCdot<SF>{B.rs, B.p, 1},
                                                      EpiStore{B.S.alpha}, g.Vh, B.br, B.ru_skip);
      CVCB_LAUNCHED(L);
      k_dir_restore<<<eg, 128, 0, L->stream>>>(B.p, B.rs, B.S, B.ru_skip, g.Vh, n);
    }
    CVCB_LAUNCHED(L);
    // a residual that stopped being finite restarts from the recomputed one
    bool restart = false;
    for (int i = 0; i < n; ++i) {
      rst[i] = (skip[i] || std::isfinite(rr[i])) ? 1 : 0;
      restart = restart || !rst[i];
    }
    if (restart) {
      CVCB_TRY(put_flags(L, B.rst_skip, rst, n));
      if constexpr (std::is_same<SF, P32>::value)
        k_copy_pt<<<egp, 128, 0, L->stream>>>(B.p, B.rs, B.rst_skip, g.Vh, n);
      else
        k_copy<<<eg, 128, 0, L->stream>>>(B.p, B.rs, B.rst_skip, g.Vh, n);
      CVCB_LAUNCHED(L);
      for (int i = 0; i < n; ++i) nrestart += !rst[i];
    }
    ++nru;
    CVCB_TRY(fetch(L, B.S.rr, n, 1));
    CVCB_TRY(fetch(L, B.S.rhat2, n, 2));
    CVCB_CUDA(cudaStreamSynchronize(L->stream));
    mailbox(L, 1, rr, n);
    mailbox(L, 2, rhat2, n);
    for (int i = 0; i < n; ++i) {
      if (skip[i]) continue;
      since[i] = 0;
      rr_max[i] = rr[i];
      rr_ref[i] = rr[i];
      if (rhat2[i] > 0) ratio2[i] = rr[i] / rhat2[i];
      if (rhat2[i] <= target2[i]) done[i] = 1;
    }
    CVCB_TRY(put_flags(L, B.S.done, done, n));
  }
  if (gexec) cudaGraphExecDestroy(gexec);
  gexec = nullptr;
  for (auto &r : B.recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  B.recs.clear();
  if (rc != CVCB_OK) return rc;

  // x_e = A^-1 (b_e + 1/2 H_eo x_o)
  CVCB_TRY((B.template hop<F64Acc, L64, false, false, true>(B.f64(B.x64, 0), B.f64(B.x64, 1),
                                                            B.f64(B.b64, 0), B.links64, 0,
                                                            nullptr, ia, ib, ia, ib, 0.5)));
  // final FP64 check |b - Q x| / |b| over the whole lattice: t_p = (Q x)_p =
  // A x_p - 1/2 H_pq x_q for both parities, batched over the rhs
  double worst = 0.0;
  int nconv = 0;
  for (int par = 0; par < 2; ++par)
    CVCB_TRY((B.template hop<F64Acc, L64, false, false, true>(
        B.f64(B.t64, par), B.f64(B.x64, 1 - par), B.f64(B.x64, par), B.links64, par, nullptr, 1.0,
        0.0, B.ka(), B.mu, -0.5)));
  k_reduce_rhs<<<rgf, kRedThreads, 0, L->stream>>>(
      RedResid{B.f64full(B.t64), B.f64full(B.b64)}, EpiStore{B.S.rhat2}, g.V, B.br, nullptr);
  CVCB_LAUNCHED(L);
  CVCB_TRY(fetch(L, B.S.rhat2, n, 2));
  for (int i = 0; i < n; ++i) CVCB_TRY(spinor_out(L, x[i], B.x64 + i * fs, g.V));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  mailbox(L, 2, rhat2, n);
  for (int i = 0; i < n; ++i) {
    const double rel = hb2[i] > 0 ? std::sqrt(rhat2[i] / hb2[i]) : 0.0;
    worst = std::max(worst, rel);
    if (rel <= P->tol) ++nconv;
  }
  int staged_err = 0;
  CVCB_CUDA(cudaMemcpyAsync(&staged_err, B.err, sizeof(int), cudaMemcpyDeviceToHost, L->stream));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  if (staged_err) {
    set_error("a staged neighbour copy of the stencil did not complete in time");
    return CVCB_ERR_CUDA;
  }
  st->iterations += std::accumulate(iters.begin(), iters.end(), 0);
  st->reliable_updates += nru;
  st->restarts += nrestart;
  st->converged += nconv;
  st->max_true_res = std::max(st->max_true_res, worst);
  st->seconds += now_s() - t0;
  return CVCB_OK;
}

template <class SF, class XF, class LF>
int time_stencil_t(cvcb_lattice *L, int kind, int prec, int recon, int nrhs, int reps, double *ms) {
  Batch<SF, XF, LF> B;
  CVCB_TRY(setup_batch(L, B, nrhs, /*with_fp64=*/false));
  // zero contents: timing of the stencil does not depend on the values
  CVCB_CUDA(cudaMemsetAsync(B.p.p, 0, sloppy_field_bytes<SF>(L->g.Vh, nrhs), L->stream));
  CVCB_CUDA(cudaMemsetAsync(B.S.done, 0, sizeof(int) * nrhs, L->stream));
  CVCB_TRY(tune_shape(L, B, prec, recon));
  double ia, ib;
  B.ainv(B.mu, ia, ib);
  auto one = [&] {
    if (kind == 2) return B.normal_op_sloppy(B.Ap, B.p, nullptr);
    if (kind == 3)
      return B.normal_op_sloppy(B.Ap, B.p, nullptr, B.dot_fusable() ? B.dot_part : nullptr);
    return B.template hop<SF, LF, false, false, false>(B.te, B.p, B.p, B.links, 0, nullptr, ia,
                                                       ib, 0, 0, -0.5);
  };
  CVCB_TRY(one());
  float best;
  cudaEvent_t a, b;
  CVCB_CUDA(cudaEventCreate(&a));
  CVCB_CUDA(cudaEventCreate(&b));
  CVCB_CUDA(cudaEventRecord(a, L->stream));
  for (int i = 0; i < reps; ++i) CVCB_TRY(one());
  CVCB_CUDA(cudaEventRecord(b, L->stream));
  CVCB_CUDA(cudaEventSynchronize(b));
  CVCB_CUDA(cudaEventElapsedTime(&best, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = best / reps;
  return CVCB_OK;
}

}  // namespace

namespace {
// M^+M of the batched solver's inner iterations on n fields (odd sites of
// CVC-layout FP64 fields in and out; even sites of out are zero).
template <class SF, class XF, class LF>
int sloppy_normal_op_t(cvcb_lattice *L, int prec, int recon, int n, const double *const *in,
                       double *const *out) {
  Batch<SF, XF, LF> B;
  CVCB_TRY(setup_batch(L, B, n));
  CVCB_TRY(tune_shape(L, B, prec, recon, 0));
  const Geom &g = L->g;
  const size_t fs = (size_t)12 * g.V;
  for (int i = 0; i < n; ++i) CVCB_TRY(spinor_in(L, B.b64 + i * fs, in[i], g.V));
  std::vector<double> ones(kMaxBatch, 1.0);
  CVCB_CUDA(cudaMemcpyAsync(B.S.scale, ones.data(), sizeof(double) * n, cudaMemcpyHostToDevice,
                            L->stream));
  dim3 eg((g.Vh + 127) / 128, n);
  k_to_sloppy<<<eg, 128, 0, L->stream>>>(B.p, B.f64(B.b64, 1), B.S.scale, nullptr, g.Vh, n);
  CVCB_LAUNCHED(L);
  CVCB_TRY(B.normal_op_sloppy(B.Ap, B.p, nullptr));
  CVCB_CUDA(cudaMemsetAsync(B.y64, 0, fs * n * sizeof(double2), L->stream));
  k_from_sloppy<<<eg, 128, 0, L->stream>>>(B.f64(B.y64, 1), B.Ap, g.Vh, n);
  CVCB_LAUNCHED(L);
  for (int i = 0; i < n; ++i) CVCB_TRY(spinor_out(L, out[i], B.y64 + i * fs, g.V));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  return CVCB_OK;
}
}  // namespace

int sloppy_normal_op(cvcb_lattice *L, int prec, int recon, int layout, int n,
                     const double *const *in, double *const *out) {
  if (!L->have_gauge) {
    set_error("no gauge field uploaded");
    return CVCB_ERR_STATE;
  }
  if (n <= 0 || n > kMaxBatch || prec < 0 || prec > 2 || (recon != 12 && recon != 18) ||
      layout < 0 || layout > 1 || (layout == 1 && prec != CVCB_PREC_SINGLE)) {
    set_error("invalid arguments");
    return CVCB_ERR_ARG;
  }
  if (prec == CVCB_PREC_DOUBLE) return sloppy_normal_op_t<F64Acc, F64Acc, L64>(L, prec, 18, n, in, out);
  if (layout == 1)
    return recon == 12 ? sloppy_normal_op_t<P32, P32, LT32c>(L, prec, recon, n, in, out)
                       : sloppy_normal_op_t<P32, P32, LT32f>(L, prec, recon, n, in, out);
  if (prec == CVCB_PREC_SINGLE)
    return recon == 12 ? sloppy_normal_op_t<F32Acc, F32Acc, L32c>(L, prec, recon, n, in, out)
                       : sloppy_normal_op_t<F32Acc, F32Acc, L32f>(L, prec, recon, n, in, out);
  return recon == 12 ? sloppy_normal_op_t<F16Acc, F32Acc, L16c>(L, prec, recon, n, in, out)
                     : sloppy_normal_op_t<F16Acc, F32Acc, L32f>(L, prec, recon, n, in, out);
}

// FP32 inner iterations on pair-tiled fields (k_eo_hop_pt and the pair CG
// kernels), the default; CVCB_PAIRS=0 selects the per-rhs fields with the
// packed-pair stencil k_eo_hop_x2 instead (read once per process).
bool use_pairs() {
  static const bool on = [] {
    const char *e = getenv("CVCB_PAIRS");
    return !e || atoi(e) != 0;
  }();
  return on;
}

int time_stencil(cvcb_lattice *L, int kind, int prec, int recon, int nrhs, int reps, double *ms) {
  if (!L->have_gauge) {
    set_error("no gauge field uploaded");
    return CVCB_ERR_STATE;
  }
  if (reps <= 0 || nrhs <= 0 || nrhs > kMaxBatch || kind < 0 || kind > 3) return CVCB_ERR_ARG;
  if (kind == 0) {
    const size_t fb = (size_t)L->g.V * 12 * sizeof(double2);
    void *f0, *f1;
    CVCB_TRY(ensure_buffer(L, SLOT_F0, fb, &f0));
    CVCB_TRY(ensure_buffer(L, SLOT_F1, fb, &f1));
    CVCB_CUDA(cudaMemsetAsync(f0, 0, fb, L->stream));
    auto one = [&] {
      return launch_tm_full(L, (double2 *)f1, (const double2 *)f0, 0.5 / L->kappa, L->mu, -0.5,
                            false, nullptr);
    };
    CVCB_TRY(one());
    cudaEvent_t a, b;
    CVCB_CUDA(cudaEventCreate(&a));
    CVCB_CUDA(cudaEventCreate(&b));
    CVCB_CUDA(cudaEventRecord(a, L->stream));
    for (int i = 0; i < reps; ++i) CVCB_TRY(one());
    CVCB_CUDA(cudaEventRecord(b, L->stream));
    CVCB_CUDA(cudaEventSynchronize(b));
    float t;
    CVCB_CUDA(cudaEventElapsedTime(&t, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms = t / reps;
    return CVCB_OK;
  }
  if (prec == CVCB_PREC_DOUBLE)
    return time_stencil_t<F64Acc, F64Acc, L64>(L, kind, prec, 18, nrhs, reps, ms);
  if (prec == CVCB_PREC_SINGLE && use_pairs())
    return recon == 12 ? time_stencil_t<P32, P32, LT32c>(L, kind, prec, recon, nrhs, reps, ms)
                       : time_stencil_t<P32, P32, LT32f>(L, kind, prec, recon, nrhs, reps, ms);
  if (prec == CVCB_PREC_SINGLE)
    return recon == 12 ? time_stencil_t<F32Acc, F32Acc, L32c>(L, kind, prec, recon, nrhs, reps, ms)
                       : time_stencil_t<F32Acc, F32Acc, L32f>(L, kind, prec, recon, nrhs, reps, ms);
  return recon == 12 ? time_stencil_t<F16Acc, F32Acc, L16c>(L, kind, prec, recon, nrhs, reps, ms)
                     : time_stencil_t<F16Acc, F32Acc, L32f>(L, kind, prec, recon, nrhs, reps, ms);
}

// Autotuner for the number of right-hand sides per batch: the sloppy normal
// operator is timed (with its own tuned launch shape) for each candidate
// batch size n, and the n with the least predicted time for all nrhs,
// ceil(nrhs / n) * t(n), wins.  Larger batches share each link load among
// more right-hand sides but hold more device memory.  Host-resident fields
// take batches of at most 24, so that the transfers of one batch overlap the
// solve of another; device-resident ones may advance as one set of up to 96.
// A batch whose memory would exceed 45 % of the free device memory is not
// tried.
template <class SF, class XF, class LF>
int tune_batch(cvcb_lattice *L, const cvcb_solver_params *P, int recon, int nrhs, bool host_fields,
               int *nb_out) {
  const int cands[] = {4, 6, 8, 12, 16, 24, 32, 48, 96};
  double best_t = 1e300;
  int best = std::min(nrhs, 12);
  size_t free_b = 0, total_b = 0;
  CVCB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  for (int n : cands) {
    if (n > kMaxBatch || (n > nrhs && n != cands[0])) continue;
    if (host_fields && n > 24) continue;
    const double need = 5.0 * 12 * L->g.V * sizeof(double2) * n +
                        8.0 * sloppy_field_bytes<SF>(L->g.Vh, n);
    if (n > cands[0] && need > 0.45 * (double)free_b) continue;
    Batch<SF, XF, LF> B;
    CVCB_TRY(setup_batch(L, B, n, /*with_fp64=*/false));
    CVCB_CUDA(cudaMemsetAsync(B.p.p, 0, sloppy_field_bytes<SF>(L->g.Vh, n), L->stream));
    CVCB_TRY(tune_shape(L, B, P->precision, recon, P->block_threads));
    float ms;
    if (time_ms(L, [&] { return B.normal_op_sloppy(B.Ap, B.p, nullptr); }, 3, &ms) != CVCB_OK) {
      cudaGetLastError();
      continue;
    }
    const double t = (double)((nrhs + n - 1) / n) * ms;
    if (t < best_t * 0.98) {  // prefer the smaller batch unless clearly slower
      best_t = t;
      best = std::min(n, nrhs);
    }
  }
  *nb_out = best;
  return CVCB_OK;
}

// Host-resident fields over several batches: one copy stream brings the
// sources of batch k+1 into device staging (raw CVC layout) and another takes
// the solutions of batch k-1 back to the host while batch k is solved, so the
// PCIe traffic of both directions overlaps the solve.  Staging is double-buffered; events hand
// each buffer between the streams (inputs consumed -> next prefetch,
// outputs copied -> next write).
template <class Run>
int solve_pipelined(cvcb_lattice *L, double *const *x, const double *const *b, int nrhs, int nb,
                    Run &run) {
  const size_t fbytes = (size_t)L->g.V * 24 * sizeof(double);
  if (!L->copy_stream) {
    CVCB_CUDA(cudaStreamCreateWithFlags(&L->copy_stream, cudaStreamNonBlocking));
    CVCB_CUDA(cudaStreamCreateWithFlags(&L->copy_stream_out, cudaStreamNonBlocking));
    for (cudaEvent_t &e : L->pipe_ev) CVCB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  cudaStream_t cs = L->copy_stream, co = L->copy_stream_out;
  // events per buffer k%2: [0,1] inputs landed, [2,3] inputs read, [4,5] outputs copied out
  cudaEvent_t *landed = L->pipe_ev, *read = L->pipe_ev + 2, *drained = L->pipe_ev + 4;
  double *in[2], *out[2];
  for (int k = 0; k < 2; ++k) {
    void *a, *c;
    CVCB_TRY(ensure_buffer(L, SLOT_PIPE_IN0 + k, fbytes * nb, &a));
    CVCB_TRY(ensure_buffer(L, SLOT_PIPE_OUT0 + k, fbytes * nb, &c));
    in[k] = static_cast<double *>(a);
    out[k] = static_cast<double *>(c);
  }
  // Batches: a short first one (nb/3 rhs), so that the solve starts after a
  // short upload, then full ones; the last takes the rest.  Only the first
  // upload and the last download do not overlap a solve.
  std::vector<int> boff, bn;
  for (int off = 0; off < nrhs;) {
    const int n = std::min(boff.empty() && nrhs > 2 * nb ? std::max(1, nb / 3) : nb, nrhs - off);
    boff.push_back(off);
    bn.push_back(n);
    off += n;
  }
  const int nbatch = (int)boff.size();
  auto prefetch = [&](int k) -> int {
    const int off = boff[k], n = bn[k], s = k % 2;
    if (k >= 2) CVCB_CUDA(cudaStreamWaitEvent(cs, read[s], 0));
    for (int i = 0; i < n; ++i)
      CVCB_CUDA(cudaMemcpyAsync(in[s] + (size_t)i * fbytes / sizeof(double), b[off + i], fbytes,
                                cudaMemcpyHostToDevice, cs));
    CVCB_CUDA(cudaEventRecord(landed[s], cs));
    return CVCB_OK;
  };
  int rc = prefetch(0);
  std::vector<double *> xs(nb);
  std::vector<const double *> bs(nb);
  for (int k = 0; k < nbatch && rc >= 0; ++k) {
    const int off = boff[k], n = bn[k], s = k % 2;
    if (k + 1 < nbatch && (rc = prefetch(k + 1)) < 0) break;
    for (int i = 0; i < n; ++i) {
      bs[i] = in[s] + (size_t)i * fbytes / sizeof(double);
      xs[i] = out[s] + (size_t)i * fbytes / sizeof(double);
    }
    CVCB_CUDA(cudaStreamWaitEvent(L->stream, landed[s], 0));
    if (k >= 2) CVCB_CUDA(cudaStreamWaitEvent(L->stream, drained[s], 0));
    rc = run(xs.data(), bs.data(), n, read[s]);
    if (rc < 0) break;
    // run() returned after its stream finished: the solutions are in out[s]
    for (int i = 0; i < n; ++i)
      CVCB_CUDA(cudaMemcpyAsync(x[off + i], xs[i], fbytes, cudaMemcpyDeviceToHost, co));
    CVCB_CUDA(cudaEventRecord(drained[s], co));
  }
  cudaError_t e = cudaStreamSynchronize(cs);
  const cudaError_t e2 = cudaStreamSynchronize(co);
  if (e == cudaSuccess) e = e2;
  if (rc < 0) return rc;
  if (e != cudaSuccess) {
    set_error("solve pipeline: %s", cudaGetErrorString(e));
    return CVCB_ERR_CUDA;
  }
  return CVCB_OK;
}

int solve_batched(cvcb_lattice *L, double *const *x, const double *const *b, int nrhs,
                  const cvcb_solver_params *P, cvcb_solver_stats *st) {
  if (!L->have_gauge) {
    set_error("no gauge field uploaded");
    return CVCB_ERR_STATE;
  }
  if (nrhs <= 0) return CVCB_OK;
  if (P->precision < 0 || P->precision > 2 || (P->link_recon != 12 && P->link_recon != 18) ||
      !(P->tol > 0) || !(P->delta >= 0 && P->delta < 1) || P->max_iter <= 0 ||
      P->block_rhs < 0 || P->block_rhs > kMaxBatch || P->block_threads < 0 ||
      P->block_threads > kHopMaxThreads || P->block_threads % 32 != 0) {
    set_error("invalid solver parameters");
    return CVCB_ERR_ARG;
  }
  int recon = P->link_recon;
  if (recon == 12 && !(L->unitarity >= 0 && L->unitarity < 1e-6)) recon = 18;  // not SU(3)
  std::memset(st, 0, sizeof *st);
  bool host_fields = true;  // every field in host memory: batches pipeline the transfers
  for (int i = 0; i < nrhs && host_fields; ++i)
    host_fields = !is_device_ptr(x[i]) && !is_device_ptr(b[i]);
  int nb = P->block_rhs;
  if (!nb) {
    const bool pairs = P->precision == CVCB_PREC_SINGLE && use_pairs();
    auto key = std::make_tuple(L->g.V,
                               P->precision + (pairs ? kPairKey : 0) + (host_fields ? 100 : 0),
                               recon, nrhs);
    auto it = g_tuned_batch.find(key);
    if (it != g_tuned_batch.end()) {
      nb = it->second;
    } else {
      int rc;
      const bool hf = host_fields;
      if (P->precision == CVCB_PREC_DOUBLE)
        rc = tune_batch<F64Acc, F64Acc, L64>(L, P, recon, nrhs, hf, &nb);
      else if (pairs)
        rc = recon == 12 ? tune_batch<P32, P32, LT32c>(L, P, recon, nrhs, hf, &nb)
                         : tune_batch<P32, P32, LT32f>(L, P, recon, nrhs, hf, &nb);
      else if (P->precision == CVCB_PREC_SINGLE)
        rc = recon == 12 ? tune_batch<F32Acc, F32Acc, L32c>(L, P, recon, nrhs, hf, &nb)
                         : tune_batch<F32Acc, F32Acc, L32f>(L, P, recon, nrhs, hf, &nb);
      else
        rc = recon == 12 ? tune_batch<F16Acc, F32Acc, L16c>(L, P, recon, nrhs, hf, &nb)
                         : tune_batch<F16Acc, F32Acc, L32f>(L, P, recon, nrhs, hf, &nb);
      if (rc < 0) return rc;
      g_tuned_batch[key] = nb;
    }
  }
  st->batch_rhs = nb;
  auto run = [&](double *const *xs, const double *const *bs, int n, cudaEvent_t read) {
    if (P->precision == CVCB_PREC_DOUBLE)
      return run_batch<F64Acc, F64Acc, L64>(L, xs, bs, n, P, st, nullptr, read);
    if (P->precision == CVCB_PREC_SINGLE && use_pairs())
      return recon == 12 ? run_batch<P32, P32, LT32c>(L, xs, bs, n, P, st, nullptr, read)
                         : run_batch<P32, P32, LT32f>(L, xs, bs, n, P, st, nullptr, read);
    if (P->precision == CVCB_PREC_SINGLE)
      return recon == 12 ? run_batch<F32Acc, F32Acc, L32c>(L, xs, bs, n, P, st, nullptr, read)
                         : run_batch<F32Acc, F32Acc, L32f>(L, xs, bs, n, P, st, nullptr, read);
    return recon == 12 ? run_batch<F16Acc, F32Acc, L16c>(L, xs, bs, n, P, st, nullptr, read)
                       : run_batch<F16Acc, F32Acc, L32f>(L, xs, bs, n, P, st, nullptr, read);
  };
  if (host_fields && nrhs > nb) {
    const int rc = solve_pipelined(L, x, b, nrhs, nb, run);
    if (rc < 0) return rc;
  } else {
    for (int off = 0; off < nrhs; off += nb) {
      const int rc = run(x + off, b + off, std::min(nb, nrhs - off), nullptr);
      if (rc < 0) return rc;
    }
  }
  return st->converged == nrhs ? CVCB_OK : CVCB_NO_CONVERGENCE;
}

}  // namespace cvcb

extern "C" {

void cvcb_solver_defaults(cvcb_solver_params *p) {
  if (!p) return;
  p->precision = CVCB_PREC_SINGLE;
  p->link_recon = 12;
  p->block_rhs = 0;
  p->block_threads = 0;
  p->max_iter = 20000;
  p->use_graph = 1;
  p->tol = 1e-10;
  p->delta = 0.0;
}

int cvcb_profile(cvcb_lattice *L, int enable) {
  if (!L) return CVCB_ERR_NULL;
  L->prof = enable != 0;
  if (enable) {
    L->prof_launches = 0;
    L->prof_ms = 0.0;
    L->prof_bytes = 0.0;
  }
  return CVCB_OK;
}

int cvcb_counters(cvcb_lattice *L, long long *kernel_launches, long long *stencil_launches_timed,
                  double *stencil_ms, double *stencil_bytes) {
  if (!L) return CVCB_ERR_NULL;
  if (kernel_launches) *kernel_launches = L->nlaunch;
  if (stencil_launches_timed) *stencil_launches_timed = L->prof_launches;
  if (stencil_ms) *stencil_ms = L->prof_ms;
  if (stencil_bytes) *stencil_bytes = L->prof_bytes;
  return CVCB_OK;
}

int cvcb_tuned_shape(cvcb_lattice *L, int precision, int link_recon, int nrhs, int *sites_per_block,
                     int *rows_per_block, int *rhs_per_thread, int *variant) {
  if (!L || !sites_per_block || !rows_per_block || !rhs_per_thread || !variant)
    return CVCB_ERR_NULL;
  const bool pairs = precision == CVCB_PREC_SINGLE && cvcb::use_pairs();
  auto it = cvcb::g_tuned_shape.find(std::make_tuple(
      L->g.V, precision + (pairs ? cvcb::kPairKey : 0), link_recon, nrhs));
  if (it == cvcb::g_tuned_shape.end()) {
    cvcb::set_error("no tuned shape for this configuration yet");
    return CVCB_ERR_STATE;
  }
  const cvcb::LaunchShape &s = it->second;
  *sites_per_block = s.bx;
  *rows_per_block = s.by;
  *rhs_per_thread = s.nr;
  *variant = pairs ? (s.pk >= 3 ? 1 + s.pk : s.pk == 2 ? 6 : 3) : s.pk ? 2 : (s.by > 1 && s.nr == 1) ? 1 : 0;
  return CVCB_OK;
}

int cvcb_sloppy_normal_op(cvcb_lattice *L, int precision, int link_recon, int layout, int nrhs,
                          const double *const *in, double *const *out) {
  if (!L || !in || !out) return CVCB_ERR_NULL;
  for (int i = 0; i < nrhs; ++i)
    if (!in[i] || !out[i]) return CVCB_ERR_NULL;
  CVCB_CUDA(cudaSetDevice(L->device));
  return cvcb::sloppy_normal_op(L, precision, link_recon, layout, nrhs, in, out);
}

int cvcb_time_stencil(cvcb_lattice *L, int kind, int precision, int link_recon, int nrhs,
                      int reps, double *ms_per_launch) {
  if (!L || !ms_per_launch) return CVCB_ERR_NULL;
  CVCB_CUDA(cudaSetDevice(L->device));
  return cvcb::time_stencil(L, kind, precision, link_recon, nrhs, reps, ms_per_launch);
}

int cvcb_solve(cvcb_lattice *L, double *const *x, const double *const *b, int nrhs,
               const cvcb_solver_params *params, cvcb_solver_stats *stats) {
  if (!L || !x || !b || !params || !stats) return CVCB_ERR_NULL;
  for (int i = 0; i < nrhs; ++i)
    if (!x[i] || !b[i]) return CVCB_ERR_NULL;
  CVCB_CUDA(cudaSetDevice(L->device));
  return cvcb::solve_batched(L, x, b, nrhs, params, stats);
}

}  // extern "C"
