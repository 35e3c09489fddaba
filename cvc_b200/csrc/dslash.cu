// Full-lattice FP64 twisted-mass Wilson operator with per-link boundary
// phases: the kernel behind Q_phi_tbc, Q_phi, Qf5 and Hopping.
//
//   out(x) = a in(x) + i b g5 in(x)
//          + c sum_mu [ (1 - g_mu) U_mu(x) in(x+mu) + (1 + g_mu) U_mu(x-mu)^+ in(x-mu) ]
//   (then out = g5 out when g5out)
//
// Q_phi_tbc (Q_phi.c:38-188): a = 1/(2 kappa), b = mu, c = -1/2.
// Q_phi(mutm) (Q_phi.c:1092-1242): b = mutm.  Qf5(mutm) (Q_phi.c:789-934):
// b = mutm, g5out.  Hopping (Q_phi.c:399-528): a = b = 0, c = -kappa.
//
// One thread per output site; both parities in one launch.  The stencil is
// HBM-bound: per site it must read 8 neighbour spinors (mostly L1/L2 hits:
// each spinor is used by 8 sites), 8 links (each used by 2 sites), its own
// spinor, and write one spinor.  Compulsory traffic 2*192 + 4*144 = 960 B.
#include "cvcb_internal.h"
#include "spinor_ops.cuh"

namespace cvcb {

template <bool G5OUT, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_tm_full_f64(double2 *__restrict__ out,
                                                     const double2 *__restrict__ in,
                                                     const double2 *__restrict__ U, Geom g,
                                                     double a, double b, double c,
                                                     const int *__restrict__ done) {
  if (done && *done) return;
  // Blocks alternate between the parities (block 2k: even sites of range k,
  // block 2k+1: odd sites of range k).  A link serves the forward hop of one
  // parity and the backward hop of the other; with the parities interleaved
  // its second use follows the first by a few MB of traffic and finds it in
  // L2, where parity after parity would read all links from DRAM twice.
  const int p = blockIdx.x & 1;
  const int i = (blockIdx.x >> 1) * blockDim.x + threadIdx.x;
  if (i >= g.Vh) return;
  const int s = p * g.Vh + i;
  const SiteCoord cd = site_coord(g, p, i);
  const size_t V = g.V;
  const int qoff = (1 - p) * g.Vh;

  Spinor<double> acc;
#pragma unroll
  for (int sp = 0; sp < 4; ++sp)
#pragma unroll
    for (int co = 0; co < 3; ++co) acc.c[sp][co] = cx(0.0, 0.0);

#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    {  // backward: (1 + g_mu) U_mu(x-mu)^+ in(x-mu)
      const int j = qoff + (nb_lex(g, cd, mu, -1) >> 1);
      const HalfSpinor<double> h = project(mu, +1, load_spinor(in, V, j));
      const Link<double> W = load_link64(U, V, mu, j);
      accum_recon(mu, +1, acc, link_dag_mul(W, h));
    }
    {  // forward: (1 - g_mu) U_mu(x) in(x+mu)
      const int j = qoff + (nb_lex(g, cd, mu, +1) >> 1);
      const HalfSpinor<double> h = project(mu, -1, load_spinor(in, V, j));
      const Link<double> W = load_link64(U, V, mu, s);
      accum_recon(mu, -1, acc, link_mul(W, h));
    }
  }

  const Spinor<double> f = load_spinor(in, V, s);
  Spinor<double> r;
#pragma unroll
  for (int sp = 0; sp < 4; ++sp) {
    const double bs = sp < 2 ? b : -b;  // i b g5
#pragma unroll
    for (int co = 0; co < 3; ++co) {
      const Cx<double> v = f.c[sp][co];
      Cx<double> o;
      o.re = fma(c, acc.c[sp][co].re, fma(a, v.re, -bs * v.im));
      o.im = fma(c, acc.c[sp][co].im, fma(a, v.im, bs * v.re));
      if (G5OUT && sp >= 2) o = cx(-o.re, -o.im);
      r.c[sp][co] = o;
    }
  }
  store_spinor(out, V, s, r);
}

// Launch variants (threads per block, minimum resident blocks per SM); the
// second number caps the registers per thread.  The variant is chosen once
// per process by timing (tm_full_variant).
template <int NT, int MINB>
static void launch_variant(cvcb_lattice *L, double2 *out, const double2 *in, double a, double b,
                           double c, bool g5out, const int *done) {
  const Geom &g = L->g;
  const int blocks = 2 * ((g.Vh + NT - 1) / NT);  // both parities, interleaved
  if (g5out)
    k_tm_full_f64<true, NT, MINB><<<blocks, NT, 0, L->stream>>>(out, in, L->U64, g, a, b, c, done);
  else
    k_tm_full_f64<false, NT, MINB><<<blocks, NT, 0, L->stream>>>(out, in, L->U64, g, a, b, c, done);
}

static int g_tm_variant = -1;
int tm_full_variant() { return g_tm_variant; }
void set_tm_full_variant(int v) { g_tm_variant = v; }

static void launch_by_variant(int v, cvcb_lattice *L, double2 *out, const double2 *in, double a,
                              double b, double c, bool g5out, const int *done) {
  switch (v) {
    case 1: launch_variant<128, 4>(L, out, in, a, b, c, g5out, done); break;
    case 2: launch_variant<256, 2>(L, out, in, a, b, c, g5out, done); break;
    case 3: launch_variant<64, 8>(L, out, in, a, b, c, g5out, done); break;
    case 4: launch_variant<128, 1>(L, out, in, a, b, c, g5out, done); break;
    default: launch_variant<128, 3>(L, out, in, a, b, c, g5out, done); break;
  }
}

int launch_tm_full(cvcb_lattice *L, double2 *out, const double2 *in, double a, double b, double c,
                   bool g5out, const int *done) {
  if (g_tm_variant < 0) {
    // one-time choice: time each variant on this lattice (output to `out`,
    // which the real launch below overwrites)
    cudaEvent_t e0, e1;
    CVCB_CUDA(cudaEventCreate(&e0));
    CVCB_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int bestv = 0;
    for (int v = 0; v < 5; ++v) {
      launch_by_variant(v, L, out, in, a, b, c, g5out, nullptr);
      CVCB_CUDA(cudaEventRecord(e0, L->stream));
      for (int k = 0; k < 5; ++k) launch_by_variant(v, L, out, in, a, b, c, g5out, nullptr);
      CVCB_CUDA(cudaEventRecord(e1, L->stream));
      CVCB_CUDA(cudaEventSynchronize(e1));
      float ms;
      CVCB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best) {
        best = ms;
        bestv = v;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    g_tm_variant = bestv;
  }
  launch_by_variant(g_tm_variant, L, out, in, a, b, c, g5out, done);
  CVCB_LAUNCHED(L);
  return CVCB_OK;
}

// f = g5 f on the first nsites sites (device layout: spins 2,3 are k = 6..11)
__global__ void k_g5(double2 *f, Geom g, int nsites_lex) {
  const int lex = blockIdx.x * blockDim.x + threadIdx.x;
  if (lex >= nsites_lex) return;
  const int j = lex_to_eo(g, lex);
#pragma unroll
  for (int k = 6; k < 12; ++k) {
    double2 v = f[(size_t)k * g.V + j];
    f[(size_t)k * g.V + j] = make_double2(-v.x, -v.y);
  }
}

int launch_g5(cvcb_lattice *L, double2 *f, int nsites) {
  k_g5<<<(nsites + 127) / 128, 128, 0, L->stream>>>(f, L->g, nsites);
  CVCB_LAUNCHED(L);
  return CVCB_OK;
}

// f = (1 - i sign m g5) f / (1 + m^2), m = 2 kappa mu  (Q_phi.c:576-589)
__global__ void k_one_pm_imu_inv(double2 *f, Geom g, int nsites_lex, double cm, double norminv) {
  const int lex = blockIdx.x * blockDim.x + threadIdx.x;
  if (lex >= nsites_lex) return;
  const int j = lex_to_eo(g, lex);
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    const double cc = k < 6 ? cm : -cm;  // cm * g5
    double2 v = f[(size_t)k * g.V + j];
    // v + i cc v
    const double re = v.x + (-cc * v.y);
    const double im = v.y + (cc * v.x);
    f[(size_t)k * g.V + j] = make_double2(re * norminv, im * norminv);
  }
}

int launch_one_pm_imu_inv(cvcb_lattice *L, double2 *f, double sign, int nsites) {
  const double m = 2.0 * L->kappa * L->mu;
  k_one_pm_imu_inv<<<(nsites + 127) / 128, 128, 0, L->stream>>>(f, L->g, nsites, -sign * m,
                                                                  1.0 / (1.0 + m * m));
  CVCB_LAUNCHED(L);
  return CVCB_OK;
}

}  // namespace cvcb
