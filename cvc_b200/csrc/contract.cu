// Conserved-vector-current contraction Pi_mu_nu(x) (cvc_exact2_xspace.c:
// 577-861), Ward-identity divergence (:928-1008), the P->gamma gamma
// sequential source (p2gg_xspace.c:525-539) and the plaquette
// (cvc_utils.c:384-436).
//
// Restructuring of the reference's 4608 volume sweeps.  For one source
// index nu and one of the two parts, the reference accumulates
//   sum_{g,ir,ia,ib} k(g,ir) us(ia,ib) [ chi_d(x)^+ g5 (g_mu - 1) U_mu(x) phi_c(x+mu)
//                                       + chi_d(x+mu)^+ g5 (g_mu + 1) U_mu(x)^+ phi_c(x) ]
// with c = (ir,ia), d = (gperm_g(ir), ib), k = +-1 or +-i and us an entry of
// the (phased) source link.  The brackets are linear in chi, so the
// coefficient sum can be moved onto the chi side once per site:
//   Z_c(x) = sum_{g,ib} conj(k us) chi_{d(g,ir,ib)}(x)
// after which Pi_mu_nu needs, per column c, one forward and one backward
// hop of phi_c and two 12-component inner products with Z_c.  Kernel
// k_cvc_z_sites (or k_cvc_z) builds the 24 Z columns of one nu (both parts);
// k_cvc_pi does the hops and dots, accumulating in FP64 registers.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cvcb_internal.h"
#include "contract_plan.h"
#include "reduce.cuh"
#include "spinor_ops.cuh"

namespace cvcb {


// Z columns of one nu: thread per site, reads 12 or 24 dn columns, writes 24.
__global__ void __launch_bounds__(128) k_cvc_z(double2 *__restrict__ Z,
                                               const double2 *__restrict__ dn, ZPlan plan,
                                               int V) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const size_t fs = (size_t)12 * V;  // field stride
  for (int col = 0; col < 24; ++col) {
    Cx<double> acc[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = cx(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const ZTerm tm = plan.t[col][q];
      const double2 *f = dn + tm.src * fs;
      const Cx<double> cf = cx(tm.coef.x, tm.coef.y);
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        const double2 v = __ldg(f + (size_t)k * V + s);
        cfma(acc[k], cf, cx(v.x, v.y));
      }
    }
    double2 *z = Z + col * fs;
#pragma unroll
    for (int k = 0; k < 12; ++k) z[(size_t)k * V + s] = make_double2(acc[k].re, acc[k].im);
  }
}

// The same Z columns with each dn column that one nu needs read once per
// site: thread = (site, spinor component k = blockIdx.y).  Its inputs (at
// most 24 columns) are staged in shared memory, because the plan picks them
// at run time, and every output is formed with the same terms in the same
// order as k_cvc_z (the same bits).  k_cvc_z reads 6 inputs per output
// column, 144 field reads per nu, most of them from L2 or DRAM again.
constexpr int kZThreads = 128;
struct ZPlanLocal {
  double2 coef[24][6];
  int field[24];             // dn column (0..59) of local input f
  unsigned char loc[24][6];  // local input of term q of output column col
  int nin;                   // local inputs in use
};

__global__ void __launch_bounds__(kZThreads) k_cvc_z_sites(double2 *__restrict__ Z,
                                                          const double2 *__restrict__ dn,
                                                          ZPlanLocal plan, int V) {
  __shared__ double2 in[24][kZThreads];
  const int s = blockIdx.x * kZThreads + threadIdx.x;
  if (s >= V) return;  // each thread reads only its own slots: no barrier below
  const size_t fs = (size_t)12 * V, off = (size_t)blockIdx.y * V + s;
  for (int f = 0; f < plan.nin; ++f) in[f][threadIdx.x] = __ldg(dn + plan.field[f] * fs + off);
  for (int col = 0; col < 24; ++col) {
    Cx<double> acc = cx(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const double2 v = in[plan.loc[col][q]][threadIdx.x];
      cfma(acc, cx(plan.coef[col][q].x, plan.coef[col][q].y), cx(v.x, v.y));
    }
    Z[col * fs + off] = make_double2(acc.re, acc.im);
  }
}

__device__ __forceinline__ Cx<double> dot_g5(const Spinor<double> &a, const Spinor<double> &b) {
  // <a, g5 b> = sum over spins 0,1 of conj(a) b - sum over spins 2,3
  Cx<double> p = cx(0.0, 0.0), m = cx(0.0, 0.0);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    cfmac(p, a.c[0][c], b.c[0][c]);
    cfmac(p, a.c[1][c], b.c[1][c]);
    cfmac(m, a.c[2][c], b.c[2][c]);
    cfmac(m, a.c[3][c], b.c[3][c]);
  }
  return p - m;
}

__device__ __forceinline__ Spinor<double> recon_full(int mu, int s, const HalfSpinor<double> &u) {
  Spinor<double> r;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) r.c[a][c] = cx(0.0, 0.0);
  accum_recon(mu, s, r, u);
  return r;
}

// Pi_mu_nu for one nu: P0 = up columns of part 0 (unshifted source),
// P1 = up columns of part 1 (source shifted by nu), Z = 24 columns from
// k_cvc_z.  conn is CVC layout (lexicographic, 32 doubles per site).
// MINB: minimum resident blocks of 128 threads per SM, which caps the
// registers (2: about 254, 8 warps per SM; 4: 128, 16 warps, a few spills);
// the variant is chosen once per process by timing (cvc_pi_variant).
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_cvc_pi(double *__restrict__ conn,
                                                const double2 *__restrict__ P0,
                                                const double2 *__restrict__ P1,
                                                const double2 *__restrict__ Z,
                                                const double2 *__restrict__ U, Geom g, int nu) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const int p = s >= g.Vh;
  const SiteCoord cd = site_coord(g, p, s - p * g.Vh);
  const size_t V = g.V, fs = (size_t)12 * V;
  const int qoff = (1 - p) * g.Vh;

  Cx<double> pi[4];
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) pi[mu] = cx(0.0, 0.0);

#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    const int j = qoff + (nb_lex(g, cd, mu, +1) >> 1);
    const Link<double> W = load_link64(U, V, mu, s);
    for (int part = 0; part < 2; ++part) {
      const double2 *P = part == 0 ? P0 : P1;
      for (int c = 0; c < 12; ++c) {
        const double2 *Pc = P + c * fs;
        const double2 *Zc = Z + (part * 12 + c) * fs;
        // forward: g5 (g_mu - 1) U_mu(x) P_c(x+mu) = -g5 (1 - g_mu) U P
        {
          const HalfSpinor<double> h = project(mu, -1, load_spinor(Pc, V, j));
          const Spinor<double> r = recon_full(mu, -1, link_mul(W, h));
          const Cx<double> w = dot_g5(load_spinor(Zc, V, s), r);
          pi[mu] = pi[mu] - w;
        }
        // backward: g5 (g_mu + 1) U_mu(x)^+ P_c(x), dotted with Z_c(x+mu)
        {
          const HalfSpinor<double> h = project(mu, +1, load_spinor(Pc, V, s));
          const Spinor<double> r = recon_full(mu, +1, link_dag_mul(W, h));
          const Cx<double> w = dot_g5(load_spinor(Zc, V, j), r);
          pi[mu] = pi[mu] + w;
        }
      }
    }
  }
  double *o = conn + (size_t)cd.lex * 32;
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    o[2 * (4 * mu + nu)] = -0.25 * pi[mu].re;  // normalisation, :861
    o[2 * (4 * mu + nu) + 1] = -0.25 * pi[mu].im;
  }
}

// The same Pi_mu_nu with one thread per (site, mu), mu = blockIdx.y: four
// times the threads, each with one link and a quarter of the loop (no
// unrolled mu loop holding its state), so that more warps fit under the
// same register cap.  Each thread accumulates pi_mu over (part, c) in the
// order of k_cvc_pi and writes only its own mu entry: the same bits.
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_cvc_pi_mu(double *__restrict__ conn,
                                                   const double2 *__restrict__ P0,
                                                   const double2 *__restrict__ P1,
                                                   const double2 *__restrict__ Z,
                                                   const double2 *__restrict__ U, Geom g, int nu) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const int mu = blockIdx.y;
  const int p = s >= g.Vh;
  const SiteCoord cd = site_coord(g, p, s - p * g.Vh);
  const size_t V = g.V, fs = (size_t)12 * V;
  const int j = (1 - p) * g.Vh + (nb_lex(g, cd, mu, +1) >> 1);
  const Link<double> W = load_link64(U, V, mu, s);
  Cx<double> pi = cx(0.0, 0.0);
  for (int part = 0; part < 2; ++part) {
    const double2 *P = part == 0 ? P0 : P1;
    for (int c = 0; c < 12; ++c) {
      const double2 *Pc = P + c * fs;
      const double2 *Zc = Z + (part * 12 + c) * fs;
      {  // forward: g5 (g_mu - 1) U_mu(x) P_c(x+mu), dotted with Z_c(x)
        const HalfSpinor<double> h = project(mu, -1, load_spinor(Pc, V, j));
        const Spinor<double> r = recon_full(mu, -1, link_mul(W, h));
        pi = pi - dot_g5(load_spinor(Zc, V, s), r);
      }
      {  // backward: g5 (g_mu + 1) U_mu(x)^+ P_c(x), dotted with Z_c(x+mu)
        const HalfSpinor<double> h = project(mu, +1, load_spinor(Pc, V, s));
        const Spinor<double> r = recon_full(mu, +1, link_dag_mul(W, h));
        pi = pi + dot_g5(load_spinor(Zc, V, j), r);
      }
    }
  }
  double *o = conn + (size_t)cd.lex * 32;
  o[2 * (4 * mu + nu)] = -0.25 * pi.re;  // normalisation, :861
  o[2 * (4 * mu + nu) + 1] = -0.25 * pi.im;
}

// Ward identity divergence on the CVC-layout conn (cvc_exact2_xspace.c:938-953)
__global__ void k_cvc_ward(double *__restrict__ wi, const double *__restrict__ conn, Geom g) {
  const int lex = blockIdx.x * blockDim.x + threadIdx.x;
  if (lex >= g.V) return;
  SiteCoord cd;
  cd.z = lex % g.LZ;
  int r = lex / g.LZ;
  cd.y = r % g.LY;
  r /= g.LY;
  cd.x = r % g.LX;
  cd.t = r / g.LX;
  cd.lex = lex;
  int dn[4];
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) dn[mu] = nb_lex(g, cd, mu, -1);
  for (int nu = 0; nu < 4; ++nu)
    for (int ri = 0; ri < 2; ++ri) {
      double w = 0;
#pragma unroll
      for (int mu = 0; mu < 4; ++mu) w += conn[(size_t)lex * 32 + 2 * (4 * mu + nu) + ri];
#pragma unroll
      for (int mu = 0; mu < 4; ++mu) w -= conn[(size_t)dn[mu] * 32 + 2 * (4 * mu + nu) + ri];
      wi[(size_t)lex * 8 + 2 * nu + ri] = w;
    }
}

// Sequential source (p2gg_xspace.c:525-539): on timeslice t,
// source(x) = exp(i phase(x)) Gamma prop(x); elsewhere zero.  Works on the
// CVC layout directly (one thread per site of the whole lattice).
struct GammaTab {
  int perm[24];
  int sign[24];
};
__global__ void k_seq_source(double *__restrict__ src, const double *__restrict__ prop, Geom g,
                             int t0, int m0, int m1, int m2, double sgn2pi, GammaTab gt) {
  const int lex = blockIdx.x * blockDim.x + threadIdx.x;
  if (lex >= g.V) return;
  double *o = src + (size_t)lex * 24;
  const int t = lex / g.s3;
  if (t != t0) {
#pragma unroll
    for (int k = 0; k < 24; ++k) o[k] = 0.0;
    return;
  }
  const int x1 = (lex / g.s2) % g.LX, x2 = (lex / g.s1) % g.LY, x3 = lex % g.LZ;
  // same operation order as the reference: int products, then / (double)L
  const double phase =
      sgn2pi * ((x1 * m0) / (double)g.LX + (x2 * m1) / (double)g.LY + (x3 * m2) / (double)g.LZ);
  double sn, cs;
  sincos(phase, &sn, &cs);
  const double *pp = prop + (size_t)lex * 24;
  double s1[24];
#pragma unroll
  for (int k = 0; k < 24; ++k) s1[k] = pp[gt.perm[k]] * gt.sign[k];
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    const double re = s1[2 * k], im = s1[2 * k + 1];
    o[2 * k] = re * cs - im * sn;
    o[2 * k + 1] = re * sn + im * cs;
  }
}

// Plaquette: sum over sites and mu < nu of Re tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+)
struct PlaqF {
  const double2 *U;  // raw (unphased) links, device layout, as cvc_utils.c:393-394 uses
  Geom g;
  __device__ void operator()(size_t s, double (&acc)[1]) const {
    const int p = (int)s >= g.Vh;
    const SiteCoord cd = site_coord(g, p, (int)s - p * g.Vh);
    const int qoff = (1 - p) * g.Vh;
    double sum = 0;
    for (int mu = 0; mu < 3; ++mu)
      for (int nu = mu + 1; nu < 4; ++nu) {
        const int jm = qoff + (nb_lex(g, cd, mu, +1) >> 1);
        const int jn = qoff + (nb_lex(g, cd, nu, +1) >> 1);
        const Link<double> A = load_link64(U, g.V, mu, (int)s);
        const Link<double> B = load_link64(U, g.V, nu, jm);
        const Link<double> C = load_link64(U, g.V, nu, (int)s);
        const Link<double> D = load_link64(U, g.V, mu, jn);
        // Re tr[(A B)(C D)^+] = sum_ij Re (AB)_ij conj((CD)_ij)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            Cx<double> ab = cx(0.0, 0.0), cdm = cx(0.0, 0.0);
            for (int k = 0; k < 3; ++k) {
              cfma(ab, A.m[i][k], B.m[k][j]);
              cfma(cdm, C.m[i][k], D.m[k][j]);
            }
            sum += ab.re * cdm.re + ab.im * cdm.im;
          }
      }
    acc[0] += sum;
  }
};

// raw links in device layout straight from the host copy (exact, no phase)
__global__ void k_gauge_raw_eo(double2 *__restrict__ out, const double2 *__restrict__ raw, Geom g) {
  const int lex = blockIdx.x * blockDim.x + threadIdx.x;
  if (lex >= g.V) return;
  const int eo = lex_to_eo(g, lex);
  for (int mu = 0; mu < 4; ++mu)
    for (int k = 0; k < 9; ++k)
      out[(size_t)(mu * 9 + k) * g.V + eo] = raw[((size_t)lex * 4 + mu) * 9 + k];
}

struct LinkSumF {
  const double2 *raw;
  __device__ void operator()(size_t k, double (&acc)[2]) const {
    const double2 v = __ldg(raw + k);
    acc[0] += v.x;
    acc[1] += v.y;
  }
};

// Coefficient plans of the Z columns for the four nu (see the file comment),
// and the phased source links Usource[nu] (cvc_exact2_xspace.c:293-304).
int make_zplans(cvcb_lattice *L, int src, ZPlan plans[4], double Us[4][18], ZMeta *meta) {
  // the reference's gamma bookkeeping (cvc_exact2_xspace.c:336-383)
  int perm[16][24], sign[16][24];
  gamma_tables(perm, sign);
  int gperm[5][4], isimag[4];
  double gsign[5][4];
  for (int ir = 0; ir < 4; ++ir) {
    gperm[4][ir] = perm[5][6 * ir] / 6;
    gsign[4][ir] = sign[5][6 * ir];
  }
  for (int nu = 0; nu < 4; ++nu) {
    for (int ir = 0; ir < 4; ++ir) {
      gperm[nu][ir] = perm[6 + nu][6 * ir] / 6;
      gsign[nu][ir] = sign[6 + nu][6 * ir];
    }
    isimag[nu] = perm[6 + nu][0] % 2;
  }
  // phased source links Usource[nu] (:293-304)
  const double *G = L->gauge_host.data();
  for (int nu = 0; nu < 4; ++nu)
    for (int k = 0; k < 9; ++k) {
      const double re = G[18 * (4 * (size_t)src + nu) + 2 * k],
                   im = G[18 * (4 * (size_t)src + nu) + 2 * k + 1];
      const double pr = L->phase[2 * nu], pi = L->phase[2 * nu + 1];
      Us[nu][2 * k] = re * pr - im * pi;
      Us[nu][2 * k + 1] = re * pi + im * pr;
    }

  for (int nu = 0; nu < 4; ++nu) {
    ZPlan &plan = plans[nu];
    for (int part = 0; part < 2; ++part)
      for (int ir = 0; ir < 4; ++ir)
        for (int ia = 0; ia < 3; ++ia) {
          const int col = part * 12 + 3 * ir + ia;
          int q = 0;
          for (int gg = 0; gg < 2; ++gg) {
            const int gi = gg == 0 ? nu : 4;
            // k: +-1 or +-i
            double kr, ki;
            if (gg == 0) {
              kr = isimag[nu] ? 0.0 : gsign[nu][ir];
              ki = isimag[nu] ? -gsign[nu][ir] : 0.0;
            } else {
              kr = part == 0 ? -gsign[4][ir] : gsign[4][ir];
              ki = 0.0;
            }
            for (int ib = 0; ib < 3; ++ib) {
              double ur, ui;  // us
              if (part == 0) {
                ur = Us[nu][2 * (3 * ia + ib)];
                ui = Us[nu][2 * (3 * ia + ib) + 1];
              } else {
                ur = Us[nu][2 * (3 * ib + ia)];
                ui = -Us[nu][2 * (3 * ib + ia) + 1];
              }
              const double cr = kr * ur - ki * ui, ci = kr * ui + ki * ur;
              const int d = 3 * gperm[gi][ir] + ib;
              // chi: part 0 -> dn shifted by nu (block nu), part 1 -> dn unshifted (block 4)
              plan.t[col][q].src = (part == 0 ? nu * 12 : 48) + d;
              plan.t[col][q].coef = make_double2(cr, -ci);
              if (meta) {
                ZMeta &m = meta[(nu * 24 + col) * 6 + q];
                m.k = make_double2(kr, ki);
                m.ia = ia;
                m.ib = ib;
                m.part = part;
              }
              ++q;
            }
          }
        }
  }
  return CVCB_OK;
}

// Z columns of one nu into Z (24 fields), from the 60 dn fields at dn:
// k_cvc_z_sites when the plan draws on at most 24 distinct dn columns (one
// nu: the 12 shifted by nu and the 12 unshifted ones), else k_cvc_z.
int launch_cvc_z(cvcb_lattice *L, double2 *Z, const double2 *dn, const ZPlan &plan) {
  ZPlanLocal lp{};
  bool fits = true;
  for (int col = 0; col < 24 && fits; ++col)
    for (int q = 0; q < 6 && fits; ++q) {
      const int src = plan.t[col][q].src;
      int f = 0;
      while (f < lp.nin && lp.field[f] != src) ++f;
      if (f == lp.nin) {
        if (lp.nin == 24) {
          fits = false;
          break;
        }
        lp.field[lp.nin++] = src;
      }
      lp.loc[col][q] = (unsigned char)f;
      lp.coef[col][q] = plan.t[col][q].coef;
    }
  if (fits) {
    dim3 grid((L->g.V + kZThreads - 1) / kZThreads, 12);
    k_cvc_z_sites<<<grid, kZThreads, 0, L->stream>>>(Z, dn, lp, L->g.V);
  } else {
    k_cvc_z<<<(L->g.V + 127) / 128, 128, 0, L->stream>>>(Z, dn, plan, L->g.V);
  }
  CVCB_LAUNCHED(L);
  return CVCB_OK;
}

static int need_gauge(cvcb_lattice *L) {
  if (!L->have_gauge) {
    set_error("no gauge field uploaded");
    return CVCB_ERR_STATE;
  }
  return CVCB_OK;
}

// Copy the Pi buffer (CVC layout on the device) to the caller.
static int conn_out(cvcb_lattice *L, double *dst, const double *src, size_t ndouble) {
  CVCB_CUDA(cudaMemcpyAsync(dst, src, ndouble * sizeof(double), cudaMemcpyDefault, L->stream));
  return CVCB_OK;
}

// Variant of the Pi kernel (0-2: k_cvc_pi at 2, 3, 4 blocks per SM; 3-5:
// k_cvc_pi_mu likewise), timed on first use; CVCB_CVC_PI=v pins it.
static int g_cvc_pi_variant = -1;

int cvc_contract(cvcb_lattice *L, const double *const *fields, int src, double *conn,
                 double *contact) {
  CVCB_TRY(need_gauge(L));
  const Geom &g = L->g;
  if (src < 0 || src >= g.V) {
    set_error("source site %d outside [0, %d)", src, g.V);
    return CVCB_ERR_ARG;
  }
  for (int f = 0; f < 120; ++f)
    if (!fields[f]) {
      set_error("field %d is NULL", f);
      return CVCB_ERR_NULL;
    }
  const size_t fs = (size_t)12 * g.V;  // double2 per field
  void *props, *zb, *cb;
  CVCB_TRY(ensure_buffer(L, SLOT_PROPS, 120 * fs * sizeof(double2), &props));
  CVCB_TRY(ensure_buffer(L, SLOT_F2, 24 * fs * sizeof(double2), &zb));
  CVCB_TRY(ensure_buffer(L, SLOT_CONN, (size_t)g.V * 32 * sizeof(double), &cb));
  double2 *P = static_cast<double2 *>(props);
  for (int f = 0; f < 120; ++f) CVCB_TRY(spinor_in(L, P + f * fs, fields[f], g.V));

  ZPlan plans[4];
  double Us[4][18];
  int perm[16][24], sign[16][24];
  gamma_tables(perm, sign);
  make_zplans(L, src, plans, Us, nullptr);
  const int blocks = (g.V + 127) / 128;
  auto pi = [&](int v, int nu) {
    double *c = static_cast<double *>(cb);
    const double2 *P1 = P + (size_t)nu * 12 * fs, *Z = static_cast<const double2 *>(zb);
    const dim3 gmu(blocks, 4);  // k_cvc_pi_mu: one thread per (site, mu)
    switch (v) {
      case 1: k_cvc_pi<3><<<blocks, 128, 0, L->stream>>>(c, P + 48 * fs, P1, Z, L->U64, g, nu); break;
      case 2: k_cvc_pi<4><<<blocks, 128, 0, L->stream>>>(c, P + 48 * fs, P1, Z, L->U64, g, nu); break;
      case 3: k_cvc_pi_mu<2><<<gmu, 128, 0, L->stream>>>(c, P + 48 * fs, P1, Z, L->U64, g, nu); break;
      case 4: k_cvc_pi_mu<3><<<gmu, 128, 0, L->stream>>>(c, P + 48 * fs, P1, Z, L->U64, g, nu); break;
      case 5: k_cvc_pi_mu<4><<<gmu, 128, 0, L->stream>>>(c, P + 48 * fs, P1, Z, L->U64, g, nu); break;
      default: k_cvc_pi<2><<<blocks, 128, 0, L->stream>>>(c, P + 48 * fs, P1, Z, L->U64, g, nu); break;
    }
  };
  for (int nu = 0; nu < 4; ++nu) {
    CVCB_TRY(launch_cvc_z(L, static_cast<double2 *>(zb), P + 60 * fs, plans[nu]));
    if (g_cvc_pi_variant < 0)
      if (const char *env = getenv("CVCB_CVC_PI")) {
        const int v = atoi(env);
        if (v >= 0 && v < 6) g_cvc_pi_variant = v;
      }
    if (g_cvc_pi_variant < 0) {  // first use in this process: time the variants (same results)
      cudaEvent_t e0, e1;
      CVCB_CUDA(cudaEventCreate(&e0));
      CVCB_CUDA(cudaEventCreate(&e1));
      float best = 1e30f;
      for (int v = 0; v < 6; ++v) {
        CVCB_CUDA(cudaEventRecord(e0, L->stream));
        pi(v, nu);
        CVCB_CUDA(cudaEventRecord(e1, L->stream));
        CVCB_CUDA(cudaEventSynchronize(e1));
        float ms;
        CVCB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) best = ms, g_cvc_pi_variant = v;
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
    }
    pi(g_cvc_pi_variant, nu);
    CVCB_LAUNCHED(L);
  }
  CVCB_TRY(conn_out(L, conn, static_cast<const double *>(cb), (size_t)g.V * 32));

  if (contact) {
    // contact term (:697-704, :837-844) from a handful of spinors
    std::vector<double> sp(24);
    double ct[8] = {0};
    int iup[4];
    {
      const int z = src % g.LZ, y = (src / g.LZ) % g.LY, x = (src / g.s2) % g.LX, t = src / g.s3;
      iup[0] = ((t + 1) % g.T) * g.s3 + x * g.s2 + y * g.s1 + z;
      iup[1] = t * g.s3 + ((x + 1) % g.LX) * g.s2 + y * g.s1 + z;
      iup[2] = t * g.s3 + x * g.s2 + ((y + 1) % g.LY) * g.s1 + z;
      iup[3] = t * g.s3 + x * g.s2 + y * g.s1 + (z + 1) % g.LZ;
    }
    auto fetch = [&](const double *f, int site, double *out24) -> int {
      CVCB_CUDA(cudaMemcpyAsync(out24, f + 24 * (size_t)site, 24 * sizeof(double),
                                cudaMemcpyDefault, L->stream));
      return CVCB_OK;
    };
    for (int part = 0; part < 2; ++part)
      for (int nu = 0; nu < 4; ++nu)
        for (int ir = 0; ir < 4; ++ir)
          for (int ia = 0; ia < 3; ++ia) {
            const double *phi = part == 0 ? fields[48 + 3 * ir + ia] : fields[nu * 12 + 3 * ir + ia];
            CVCB_TRY(fetch(phi, part == 0 ? iup[nu] : src, sp.data()));
            CVCB_CUDA(cudaStreamSynchronize(L->stream));
            double s1[24], s2[24];
            for (int a = 0; a < 4; ++a)
              for (int i = 0; i < 3; ++i) {
                double re = 0, im = 0;
                for (int j = 0; j < 3; ++j) {
                  // part 0: Usource phi; part 1: Usource^+ phi
                  double ur, ui;
                  if (part == 0) { ur = Us[nu][2 * (3 * i + j)]; ui = Us[nu][2 * (3 * i + j) + 1]; }
                  else { ur = Us[nu][2 * (3 * j + i)]; ui = -Us[nu][2 * (3 * j + i) + 1]; }
                  const double vr = sp[2 * (3 * a + j)], vi = sp[2 * (3 * a + j) + 1];
                  re += ur * vr - ui * vi;
                  im += ur * vi + ui * vr;
                }
                s1[2 * (3 * a + i)] = re;
                s1[2 * (3 * a + i) + 1] = im;
              }
            for (int k = 0; k < 24; ++k) s2[k] = s1[perm[nu][k]] * sign[nu][k];
            const int k0 = 2 * (3 * ir + ia);
            if (part == 0) {
              ct[2 * nu] += -0.5 * (s2[k0] - s1[k0]);
              ct[2 * nu + 1] += -0.5 * (s2[k0 + 1] - s1[k0 + 1]);
            } else {
              ct[2 * nu] += 0.5 * (s2[k0] + s1[k0]);
              ct[2 * nu + 1] += 0.5 * (s2[k0 + 1] + s1[k0 + 1]);
            }
          }
    std::memcpy(contact, ct, sizeof ct);
  }
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  return CVCB_OK;
}

int cvc_ward(cvcb_lattice *L, const double *conn, double *wi) {
  const Geom &g = L->g;
  void *cb, *wb;
  CVCB_TRY(ensure_buffer(L, SLOT_CONN, (size_t)g.V * 32 * sizeof(double), &cb));
  CVCB_TRY(ensure_buffer(L, SLOT_STAGE_B, (size_t)g.V * 24 * sizeof(double), &wb));
  CVCB_CUDA(cudaMemcpyAsync(cb, conn, (size_t)g.V * 32 * sizeof(double), cudaMemcpyDefault,
                            L->stream));
  k_cvc_ward<<<(g.V + 127) / 128, 128, 0, L->stream>>>(static_cast<double *>(wb),
                                                        static_cast<const double *>(cb), g);
  CVCB_LAUNCHED(L);
  CVCB_CUDA(cudaMemcpyAsync(wi, wb, (size_t)g.V * 8 * sizeof(double), cudaMemcpyDefault,
                            L->stream));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  return CVCB_OK;
}

int p2gg_seq_source(cvcb_lattice *L, double *source, const double *prop, int t, const int mom[3],
                    int gamma_id, int pos) {
  const Geom &g = L->g;
  if (t < 0 || t >= g.T || gamma_id < 0 || gamma_id > 15) {
    set_error("timeslice %d or gamma id %d out of range", t, gamma_id);
    return CVCB_ERR_ARG;
  }
  const double *dprop = prop;
  double *dsrc = source;
  void *a, *b;
  const size_t bytes = (size_t)g.V * 24 * sizeof(double);
  if (!is_device_ptr(prop)) {
    CVCB_TRY(ensure_buffer(L, SLOT_STAGE_A, bytes, &a));
    CVCB_CUDA(cudaMemcpyAsync(a, prop, bytes, cudaMemcpyHostToDevice, L->stream));
    dprop = static_cast<const double *>(a);
  }
  const bool host_out = !is_device_ptr(source);
  if (host_out) {
    CVCB_TRY(ensure_buffer(L, SLOT_STAGE_B, bytes, &b));
    dsrc = static_cast<double *>(b);
  }
  int perm[16][24], sign[16][24];
  gamma_tables(perm, sign);
  GammaTab gt;
  for (int k = 0; k < 24; ++k) {
    gt.perm[k] = perm[gamma_id][k];
    gt.sign[k] = sign[gamma_id][k];
  }
  const double sgn2pi = (1. - 2. * pos) * 2. * M_PI;
  k_seq_source<<<(g.V + 127) / 128, 128, 0, L->stream>>>(dsrc, dprop, g, t, mom[0], mom[1], mom[2],
                                                          sgn2pi, gt);
  CVCB_LAUNCHED(L);
  if (host_out)
    CVCB_CUDA(cudaMemcpyAsync(source, dsrc, bytes, cudaMemcpyDeviceToHost, L->stream));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  return CVCB_OK;
}

struct StorePlaq {
  double *out;
  __device__ void operator()(const double (&t)[1]) const { out[0] = t[0]; }
};
struct StoreLinksum {
  double *out;
  __device__ void operator()(const double (&t)[2]) const {
    out[1] = t[0];
    out[2] = t[1];
  }
};

int plaquette(cvcb_lattice *L, double *plaq, double *linksum) {
  CVCB_TRY(need_gauge(L));
  const Geom &g = L->g;
  void *raw, *eo;
  CVCB_TRY(ensure_buffer(L, SLOT_STAGE_A, (size_t)g.V * 72 * sizeof(double), &raw));
  CVCB_TRY(ensure_buffer(L, SLOT_F0, (size_t)g.V * 36 * sizeof(double2), &eo));
  CVCB_CUDA(cudaMemcpyAsync(raw, L->gauge_host.data(), (size_t)g.V * 72 * sizeof(double),
                            cudaMemcpyHostToDevice, L->stream));
  k_gauge_raw_eo<<<(g.V + 127) / 128, 128, 0, L->stream>>>(static_cast<double2 *>(eo),
                                                            static_cast<const double2 *>(raw), g);
  CVCB_LAUNCHED(L);
  CVCB_TRY(launch_reduce<1>(L, PlaqF{static_cast<const double2 *>(eo), g},
                            StorePlaq{L->red_result}, (size_t)g.V));
  CVCB_TRY(launch_reduce<2>(L, LinkSumF{static_cast<const double2 *>(raw)},
                            StoreLinksum{L->red_result}, (size_t)g.V * 36));
  double r[3];
  CVCB_CUDA(cudaMemcpyAsync(r, L->red_result, 3 * sizeof(double), cudaMemcpyDeviceToHost,
                            L->stream));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  if (plaq) *plaq = r[0] / ((double)g.V * 18.0);
  if (linksum) {
    linksum[0] = r[1];
    linksum[1] = r[2];
  }
  return CVCB_OK;
}

}  // namespace cvcb

using namespace cvcb;

extern "C" {

int cvcb_cvc_contract(cvcb_lattice *L, const double *const *fields, int source_site, double *conn,
                      double *contact) {
  if (!L || !fields || !conn) return CVCB_ERR_NULL;
  CVCB_CUDA(cudaSetDevice(L->device));
  return cvc_contract(L, fields, source_site, conn, contact);
}

int cvcb_cvc_ward(cvcb_lattice *L, const double *conn, double *wi) {
  if (!L || !conn || !wi) return CVCB_ERR_NULL;
  CVCB_CUDA(cudaSetDevice(L->device));
  return cvc_ward(L, conn, wi);
}

int cvcb_p2gg_seq_source(cvcb_lattice *L, double *source, const double *prop, int timeslice,
                         const int momentum[3], int gamma_id, int propagator_position) {
  if (!L || !source || !prop || !momentum) return CVCB_ERR_NULL;
  CVCB_CUDA(cudaSetDevice(L->device));
  return p2gg_seq_source(L, source, prop, timeslice, momentum, gamma_id, propagator_position);
}

int cvcb_plaquette(cvcb_lattice *L, double *plaq, double *linksum) {
  if (!L) return CVCB_ERR_NULL;
  CVCB_CUDA(cudaSetDevice(L->device));
  return plaquette(L, plaq, linksum);
}

}  // extern "C"
