// Derivatives of Pi_mu_nu: a forward / tangent / backward triple.
// No counterpart in the reference.
//
// Forward: the 120 propagator columns of one source point y (up = Q(mu)^-1,
// dn = Q(-mu)^-1, point sources at y + mu-hat, mu = 0..3, and at y; the
// column order of cvc_exact2_xspace.c:401-430) are solved with the batched
// solver and contracted (contract.cu).  They are kept on the device when
// they fit the caller's memory budget, otherwise recomputed when needed.
//
// Tangent (dPi/dmu, dPi/dkappa): Pi = C(up, dn) is linear in the up columns
// and antilinear in the dn columns, so dPi = C(up', dn) + C(up, dn') with
//   up' = -Q(mu)^-1 (dQ(mu)/dt) up,  dn' = -Q(-mu)^-1 (dQ(-mu)/dt) dn,
//   dQ(+-mu)/dmu = +-i g5,  dQ/dkappa = -1/(2 kappa^2):
// one extra solve per column.
//
// Backward (adjoint) for a real scalar L = Re sum_x conj(w_munu(x)) Pi_munu(x):
//   * the contraction's transpose gives adjoint sources A_up, A_dn with
//     dL = Re sum <A, d(column)>, and the explicit dependence on the sink
//     links (conserved-current vertices) and on the source links;
//   * lambda = Q^-dagger A, with Q(mu)^-dagger = g5 Q(-mu)^-1 g5 (one
//     adjoint solve per column, of the opposite flavour);
//   * dL = -Re sum <lambda, dQ column>: the gauge force (outer products of
//     lambda and the column at each link), dL/dmu and dL/dkappa.
// The link gradient is returned per raw link entry U_ab as
// dL/dRe U_ab + i dL/dIm U_ab, in the CVC gauge layout.
#include <cmath>
#include <cstring>
#include <vector>

#include "contract_plan.h"
#include "reduce.cuh"
#include "spinor_ops.cuh"

namespace cvcb {
namespace {

constexpr int kMaxCols = 24;

struct ColPtrs {
  const double2 *in[kMaxCols];
  double2 *out[kMaxCols];
};

__device__ __forceinline__ Spinor<double> g5s(Spinor<double> v) {
#pragma unroll
  for (int s = 2; s < 4; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) v.c[s][c] = cx(-v.c[s][c].re, -v.c[s][c].im);
  return v;
}
__device__ __forceinline__ Spinor<double> recon_only(int mu, int s, const HalfSpinor<double> &u) {
  Spinor<double> r;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) r.c[a][c] = cx(0.0, 0.0);
  accum_recon(mu, s, r, u);
  return r;
}
__device__ __forceinline__ void axpy_c(Spinor<double> &acc, Cx<double> w, const Spinor<double> &t) {
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) cfma(acc.c[a][c], w, t.c[a][c]);
}
__device__ __forceinline__ Cx<double> weight(const double *w, int lex, int mu, int nu) {
  const double *p = w + 32 * (size_t)lex + 2 * (4 * mu + nu);
  return cx(p[0], p[1]);
}

// MODE 0 (transpose of the contraction w.r.t. the dn columns, acting on up):
//   out(x) = sum_mu [ conj(w_mu(x))    g5 (g_mu - 1) W_mu(x)      in(x+mu)
//                   + conj(w_mu(x-mu)) g5 (1 + g_mu) W_mu(x-mu)^+ in(x-mu) ]
// MODE 1 (transpose w.r.t. the up columns, acting on Z):
//   out(y) = sum_mu [ w_mu(y-mu) W_mu(y-mu)^+ (g_mu - 1) g5 in(y-mu)
//                   + w_mu(y)    W_mu(y)    (1 + g_mu) g5 in(y+mu) ]
// w_mu(x) = w_{mu nu}(x); out = out*ACC + scale*result.  blockIdx.y = column.
template <int MODE>
__global__ void __launch_bounds__(128) k_weighted_hop(ColPtrs cp, const double *__restrict__ w,
                                                      int nu, const double2 *__restrict__ U,
                                                      Geom g, double scale, int acc_out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const double2 *in = cp.in[blockIdx.y];
  double2 *out = cp.out[blockIdx.y];
  const size_t V = g.V;
  const int p = s >= g.Vh;
  const SiteCoord cd = site_coord(g, p, s - p * g.Vh);
  const int qoff = (1 - p) * g.Vh;
  Spinor<double> acc;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc.c[a][c] = cx(0.0, 0.0);
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    const int lf = nb_lex(g, cd, mu, +1), lb = nb_lex(g, cd, mu, -1);
    const int jf = qoff + (lf >> 1), jb = qoff + (lb >> 1);
    const Link<double> Wx = load_link64(U, V, mu, s);
    const Link<double> Wb = load_link64(U, V, mu, jb);
    const Cx<double> w0 = weight(w, cd.lex, mu, nu), w1 = weight(w, lb, mu, nu);
    if (MODE == 0) {
      Spinor<double> t = g5s(recon_only(mu, -1, link_mul(Wx, project(mu, -1, load_spinor(in, V, jf)))));
      axpy_c(acc, cx(-w0.re, w0.im), t);  // -conj(w0): g5 (g_mu - 1) = -g5 (1 - g_mu)
      t = g5s(recon_only(mu, +1, link_dag_mul(Wb, project(mu, +1, load_spinor(in, V, jb)))));
      axpy_c(acc, cx(w1.re, -w1.im), t);
    } else {
      Spinor<double> t =
          recon_only(mu, -1, link_dag_mul(Wb, project(mu, -1, g5s(load_spinor(in, V, jb)))));
      axpy_c(acc, cx(-w1.re, -w1.im), t);  // (g_mu - 1) = -(1 - g_mu)
      t = recon_only(mu, +1, link_mul(Wx, project(mu, +1, g5s(load_spinor(in, V, jf)))));
      axpy_c(acc, w0, t);
    }
  }
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    const Cx<double> a = acc.c[k / 3][k % 3];
    double2 o = make_double2(scale * a.re, scale * a.im);
    if (acc_out) {
      const double2 q = out[k * V + s];
      o.x += q.x;
      o.y += q.y;
    }
    out[k * V + s] = o;
  }
}

// out_col += sum_q coef_q in_{src_q}   (all device-layout fields)
struct MixTerm {
  int src;
  double2 coef;
};
struct MixPlan {
  int nout;
  int out_index[24];   // destination field index (into `outs`)
  int nterm[24];
  MixTerm t[24][6];
};
__global__ void __launch_bounds__(128) k_mix(double2 *outs, const double2 *ins, MixPlan plan,
                                             int V) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const size_t fs = (size_t)12 * V;
  for (int o = 0; o < plan.nout; ++o) {
    double2 *dst = outs + plan.out_index[o] * fs;
    for (int k = 0; k < 12; ++k) {
      Cx<double> a = cx(dst[k * (size_t)V + s].x, dst[k * (size_t)V + s].y);
      for (int q = 0; q < plan.nterm[o]; ++q) {
        const double2 v = __ldg(ins + plan.t[o][q].src * fs + k * (size_t)V + s);
        cfma(a, cx(plan.t[o][q].coef.x, plan.t[o][q].coef.y), cx(v.x, v.y));
      }
      dst[k * (size_t)V + s] = make_double2(a.re, a.im);
    }
  }
}

// Link gradient from pairs (left_k, right_k), per link (x, mu):
//   c_ij = sum_k sum_s conj(S1(left_k(x))_si)  right_k(x+mu)_sj
//   e_ij = sum_k sum_s conj(S2(left_k(x+mu))_sj) right_k(x)_si
//   G_mu(x)_ij += e^{-i theta_mu} (alpha(x) conj(c_ij) + beta(x) e_ij)
// KIND 0 (dQ in the solver operator): S1 = 1 - g_mu, S2 = 1 + g_mu,
//   alpha = beta = 1/2.
// KIND 1 (the contraction's own sink links): S1 = (g_mu - 1) g5,
//   S2 = (1 + g_mu) g5, alpha = -w_munu(x)/4, beta = -conj(w_munu(x))/4.
struct PairPtrs {
  const double2 *left[kMaxCols];
  const double2 *right[kMaxCols];
  int n;
};
template <int KIND>
__global__ void __launch_bounds__(128) k_force(double2 *__restrict__ G, PairPtrs pp,
                                               const double *__restrict__ w, int nu, Geom g,
                                               double4 ph01, double4 ph23) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (s >= g.V) return;
  const size_t V = g.V;
  const int p = s >= g.Vh;
  const SiteCoord cd = site_coord(g, p, s - p * g.Vh);
  const int jf = (1 - p) * g.Vh + (nb_lex(g, cd, mu, +1) >> 1);
  Cx<double> c[3][3], e[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) c[i][j] = e[i][j] = cx(0.0, 0.0);
  for (int k = 0; k < pp.n; ++k) {
    Spinor<double> a = load_spinor(pp.left[k], V, s);
    Spinor<double> b = load_spinor(pp.right[k], V, jf);
    Spinor<double> a2 = load_spinor(pp.left[k], V, jf);
    Spinor<double> b2 = load_spinor(pp.right[k], V, s);
    if (KIND == 1) {
      a = g5s(a);
      a2 = g5s(a2);
    }
    a = recon_only(mu, -1, project(mu, -1, a));   // (1 - g_mu) a
    a2 = recon_only(mu, +1, project(mu, +1, a2));  // (1 + g_mu) a2
#pragma unroll
    for (int sp = 0; sp < 4; ++sp)
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          cfmac(c[i][j], a.c[sp][i], b.c[sp][j]);
          cfmac(e[i][j], a2.c[sp][j], b2.c[sp][i]);
        }
  }
  Cx<double> al, be;
  if (KIND == 0) {
    al = be = cx(0.5, 0.0);
  } else {
    const Cx<double> ww = weight(w, cd.lex, mu, nu);
    al = cx(0.25 * ww.re, 0.25 * ww.im);    // -(g_mu - 1) = (1 - g_mu): sign folded here
    be = cx(-0.25 * ww.re, 0.25 * ww.im);   // -conj(w)/4
  }
  const double2 phs[4] = {make_double2(ph01.x, ph01.y), make_double2(ph01.z, ph01.w),
                          make_double2(ph23.x, ph23.y), make_double2(ph23.z, ph23.w)};
  const Cx<double> emi = cx(phs[mu].x, -phs[mu].y);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      Cx<double> t = cmul(al, cx(c[i][j].re, -c[i][j].im));
      cfma(t, be, e[i][j]);
      t = cmul(emi, t);
      double2 *gp = G + (size_t)(mu * 9 + 3 * i + j) * V + s;
      *gp = make_double2(gp->x + t.re, gp->y + t.im);
    }
}

// Per-pair complex dots sum_x <a(x), b(x)> (optionally <a, g5 b>) into
// per-block partials [pair][block] (summed on the host in block order).
struct DotPairs {
  const double2 *a[kMaxCols * 6];
  const double2 *b[kMaxCols * 6];
};
__global__ void __launch_bounds__(256) k_pair_dots(DotPairs dp, int V, int g5, double2 *partials,
                                                   int nblocks) {
  __shared__ double sh[2][8];
  const int pr = blockIdx.y;
  const double2 *a = dp.a[pr], *b = dp.b[pr];
  double v[2] = {0, 0};
  for (int s = blockIdx.x * 256 + threadIdx.x; s < V; s += nblocks * 256) {
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      const double2 x = __ldg(a + (size_t)k * V + s), y = __ldg(b + (size_t)k * V + s);
      const double sg = (g5 && k >= 6) ? -1.0 : 1.0;
      v[0] += sg * (x.x * y.x + x.y * y.y);
      v[1] += sg * (x.x * y.y - x.y * y.x);
    }
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) partials[(size_t)pr * nblocks + blockIdx.x] = make_double2(v[0], v[1]);
}

// CVC-layout (24 doubles per site) helpers on the device
__global__ void k_cvc_scale_g5(double *out, const double *in, double fr, double fi, int g5,
                               size_t nsites) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= nsites * 12) return;
  const size_t site = i / 12;
  const int k = (int)(i % 12);
  const double sg = (g5 && k >= 6) ? -1.0 : 1.0;
  const double re = in[2 * i], im = in[2 * i + 1];
  out[2 * i] = sg * (fr * re - fi * im);
  out[2 * i + 1] = sg * (fr * im + fi * re);
  (void)site;
}

__global__ void k_point_sources(double *b, Geom g, int src, size_t fstride) {
  // 60 fields: column 12*m + sc, point at y + m-hat (m < 4) or y (m = 4)
  const int f = blockIdx.x;
  if (f >= 60 || threadIdx.x != 0) return;
  const int m = f / 12, sc = f % 12;
  SiteCoord cd;
  cd.lex = src;
  cd.z = src % g.LZ;
  cd.y = (src / g.LZ) % g.LY;
  cd.x = (src / g.s2) % g.LX;
  cd.t = src / g.s3;
  const int site = m < 4 ? nb_lex(g, cd, m, +1) : src;
  b[f * fstride + 24 * (size_t)site + 2 * sc] = 1.0;
}

// G (device EO, [4][9][V]) -> CVC gauge layout (72 doubles per site)
__global__ void k_grad_to_cvc(double *out, const double2 *G, Geom g) {
  const int lex = blockIdx.x * blockDim.x + threadIdx.x;
  if (lex >= g.V) return;
  const int eo = lex_to_eo(g, lex);
  for (int mu = 0; mu < 4; ++mu)
    for (int k = 0; k < 9; ++k) {
      const double2 v = G[(size_t)(mu * 9 + k) * g.V + eo];
      out[18 * (4 * (size_t)lex + mu) + 2 * k] = v.x;
      out[18 * (4 * (size_t)lex + mu) + 2 * k + 1] = v.y;
    }
}

double2 host_sum_partials(const std::vector<double2> &p, int pr, int nb) {
  double re = 0, im = 0;
  for (int b = 0; b < nb; ++b) {
    re += p[(size_t)pr * nb + b].x;
    im += p[(size_t)pr * nb + b].y;
  }
  return make_double2(re, im);
}

}  // namespace

// ---------------------------------------------------------------------------
struct AdjointState {
  bool valid = false;
  int src = 0;
  cvcb_solver_params params{};
  double keep_bytes = 0;
  bool have_props = false;
};
static AdjointState &state(cvcb_lattice *L) {
  static std::vector<std::pair<cvcb_lattice *, AdjointState>> states;
  for (auto &s : states)
    if (s.first == L) return s.second;
  states.push_back({L, AdjointState{}});
  return states.back().second;
}

// Device buffers used here
enum { SLOT_ADJ_CVC = SLOT_MIX0 + 1, SLOT_ADJ_B, SLOT_ADJ_PROPS, SLOT_ADJ_WORK, SLOT_ADJ_W,
       SLOT_ADJ_G, SLOT_ADJ_PART };

// Solve the 120 columns into CVC-layout device buffers `cols` (60 up, 60 dn).
static int solve_columns(cvcb_lattice *L, double *cols, const double *bsrc,
                         const cvcb_solver_params *P, double mu_up, double mu_dn, int nup,
                         int ndn, const size_t fstride) {
  std::vector<double *> x(nup + ndn);
  std::vector<const double *> b(nup + ndn);
  for (int i = 0; i < nup + ndn; ++i) {
    x[i] = cols + i * fstride;
    b[i] = bsrc + i * fstride;
  }
  const double mu0 = L->mu;
  cvcb_solver_stats st{};
  int rc = CVCB_OK;
  if (nup) {
    L->mu = mu_up;
    rc = solve_batched(L, x.data(), b.data(), nup, P, &st);
  }
  if (rc >= 0 && ndn) {
    L->mu = mu_dn;
    cvcb_solver_stats st2{};
    rc = solve_batched(L, x.data() + nup, b.data() + nup, ndn, P, &st2);
  }
  L->mu = mu0;
  return rc;
}

// The 120 columns in device layout at props (120 x 12V double2).
static int columns(cvcb_lattice *L, double2 **props_out) {
  AdjointState &S = state(L);
  const Geom &g = L->g;
  const size_t fs = (size_t)12 * g.V, fstride = (size_t)24 * g.V;
  void *props, *cvc, *bsrc;
  CVCB_TRY(ensure_buffer(L, SLOT_ADJ_PROPS, 120 * fs * sizeof(double2), &props));
  double2 *P = static_cast<double2 *>(props);
  if (!S.have_props) {
    CVCB_TRY(ensure_buffer(L, SLOT_ADJ_CVC, 120 * fstride * sizeof(double), &cvc));
    CVCB_TRY(ensure_buffer(L, SLOT_ADJ_B, 120 * fstride * sizeof(double), &bsrc));
    CVCB_CUDA(cudaMemsetAsync(bsrc, 0, 120 * fstride * sizeof(double), L->stream));
    k_point_sources<<<60, 32, 0, L->stream>>>(static_cast<double *>(bsrc), g, S.src, fstride);
    CVCB_LAUNCHED(L);
    // dn sources are the same points
    CVCB_CUDA(cudaMemcpyAsync(static_cast<double *>(bsrc) + 60 * fstride, bsrc,
                              60 * fstride * sizeof(double), cudaMemcpyDeviceToDevice, L->stream));
    const int rc = solve_columns(L, static_cast<double *>(cvc), static_cast<double *>(bsrc),
                                 &S.params, L->mu, -L->mu, 60, 60, fstride);
    if (rc < 0) return rc;
    for (int f = 0; f < 120; ++f)
      CVCB_TRY(spinor_in(L, P + f * fs, static_cast<double *>(cvc) + f * fstride, g.V));
    S.have_props = true;
  }
  *props_out = P;
  return CVCB_OK;
}

static int release_columns_if_over_budget(cvcb_lattice *L) {
  AdjointState &S = state(L);
  const double bytes = 120.0 * 12 * L->g.V * sizeof(double2);
  if (bytes > S.keep_bytes) {
    S.have_props = false;
    if ((int)L->bufs.size() > SLOT_ADJ_PROPS && L->bufs[SLOT_ADJ_PROPS].ptr) {
      CVCB_CUDA(cudaStreamSynchronize(L->stream));
      CVCB_CUDA(cudaFree(L->bufs[SLOT_ADJ_PROPS].ptr));
      L->bufs[SLOT_ADJ_PROPS] = Buffer{};
    }
  }
  return CVCB_OK;
}

int pi_forward(cvcb_lattice *L, int src, const cvcb_solver_params *P, double keep_bytes,
               double *conn, double *contact) {
  const Geom &g = L->g;
  if (src < 0 || src >= g.V) {
    set_error("source site %d outside [0, %d)", src, g.V);
    return CVCB_ERR_ARG;
  }
  AdjointState &S = state(L);
  S.valid = true;
  S.src = src;
  S.params = *P;
  S.keep_bytes = keep_bytes;
  S.have_props = false;
  double2 *props;
  CVCB_TRY(columns(L, &props));
  // contraction on the columns (CVC layout is its interface: use the solved
  // CVC-layout buffers, still valid here)
  const size_t fstride = (size_t)24 * g.V;
  double *cvc = static_cast<double *>(L->bufs[SLOT_ADJ_CVC].ptr);
  std::vector<const double *> f(120);
  for (int i = 0; i < 120; ++i) f[i] = cvc + i * fstride;
  CVCB_TRY(cvc_contract(L, f.data(), src, conn, contact));
  return release_columns_if_over_budget(L);
}

int pi_tangent(cvcb_lattice *L, int param, double *dconn) {
  AdjointState &S = state(L);
  if (!S.valid) {
    set_error("call cvcb_pi_forward first");
    return CVCB_ERR_STATE;
  }
  if (param != 0 && param != 1) {
    set_error("parameter must be 0 (mu) or 1 (kappa)");
    return CVCB_ERR_ARG;
  }
  const Geom &g = L->g;
  const size_t fs = (size_t)12 * g.V, fstride = (size_t)24 * g.V;
  double2 *props;
  CVCB_TRY(columns(L, &props));
  void *cvc, *bsrc, *work;
  CVCB_TRY(ensure_buffer(L, SLOT_ADJ_CVC, 120 * fstride * sizeof(double), &cvc));
  CVCB_TRY(ensure_buffer(L, SLOT_ADJ_B, 120 * fstride * sizeof(double), &bsrc));
  CVCB_TRY(ensure_buffer(L, SLOT_ADJ_WORK, 120 * fstride * sizeof(double), &work));
  double *C = static_cast<double *>(cvc), *B = static_cast<double *>(bsrc),
         *W = static_cast<double *>(work);
  // columns back in CVC layout (C), right-hand sides of the tangent solves (B)
  for (int f = 0; f < 120; ++f) CVCB_TRY(spinor_out(L, C + f * fstride, props + f * fs, g.V));
  const double k2 = 1.0 / (2.0 * L->kappa * L->kappa);
  const int nb = (int)((fstride / 2 + 255) / 256);
  for (int f = 0; f < 120; ++f) {
    // mu: rhs = i g5 column; kappa: rhs = column / (2 kappa^2)
    if (param == 0)
      k_cvc_scale_g5<<<nb, 256, 0, L->stream>>>(B + f * fstride, C + f * fstride, 0.0, 1.0, 1,
                                                (size_t)g.V);
    else
      k_cvc_scale_g5<<<nb, 256, 0, L->stream>>>(B + f * fstride, C + f * fstride, k2, 0.0, 0,
                                                (size_t)g.V);
    CVCB_LAUNCHED(L);
  }
  const int rc = solve_columns(L, W, B, &S.params, L->mu, -L->mu, 60, 60, fstride);
  if (rc < 0) return rc;
  if (param == 0) {  // up' = -Q(mu)^-1 (i g5 up); dn' = +Q(-mu)^-1 (i g5 dn)
    for (int f = 0; f < 60; ++f) {
      k_cvc_scale_g5<<<nb, 256, 0, L->stream>>>(W + f * fstride, W + f * fstride, -1.0, 0.0, 0,
                                                (size_t)g.V);
      CVCB_LAUNCHED(L);
    }
  }
  // dPi = C(up', dn) + C(up, dn')
  std::vector<const double *> f1(120), f2(120);
  for (int i = 0; i < 60; ++i) {
    f1[i] = W + i * fstride;
    f1[60 + i] = C + (60 + i) * fstride;
    f2[i] = C + i * fstride;
    f2[60 + i] = W + (60 + i) * fstride;
  }
  std::vector<double> a((size_t)32 * g.V), b2((size_t)32 * g.V);
  CVCB_TRY(cvc_contract(L, f1.data(), S.src, a.data(), nullptr));
  CVCB_TRY(cvc_contract(L, f2.data(), S.src, b2.data(), nullptr));
  for (size_t k = 0; k < a.size(); ++k) a[k] += b2[k];
  CVCB_CUDA(cudaMemcpyAsync(dconn, a.data(), a.size() * sizeof(double), cudaMemcpyDefault,
                            L->stream));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  return release_columns_if_over_budget(L);
}

int pi_backward(cvcb_lattice *L, const double *wts, double *dLdU, double *dLdmu,
                double *dLdkappa) {
  AdjointState &S = state(L);
  if (!S.valid) {
    set_error("call cvcb_pi_forward first");
    return CVCB_ERR_STATE;
  }
  const Geom &g = L->g;
  const size_t V = g.V, fs = (size_t)12 * V, fstride = (size_t)24 * V;
  double2 *P;
  CVCB_TRY(columns(L, &P));
  void *wbuf, *work, *gbuf, *cvc, *bsrc;
  CVCB_TRY(ensure_buffer(L, SLOT_ADJ_W, 32 * V * sizeof(double), &wbuf));
  // work: A (120 fields) + Z (24) + H (24), device layout
  CVCB_TRY(ensure_buffer(L, SLOT_ADJ_WORK, 168 * fs * sizeof(double2), &work));
  CVCB_TRY(ensure_buffer(L, SLOT_ADJ_G, 36 * V * sizeof(double2), &gbuf));
  CVCB_TRY(ensure_buffer(L, SLOT_ADJ_CVC, 120 * fstride * sizeof(double), &cvc));
  CVCB_TRY(ensure_buffer(L, SLOT_ADJ_B, 120 * fstride * sizeof(double), &bsrc));
  double *w = static_cast<double *>(wbuf);
  double2 *A = static_cast<double2 *>(work), *Z = A + 120 * fs, *H = Z + 24 * fs;
  double2 *G = static_cast<double2 *>(gbuf);
  CVCB_CUDA(cudaMemcpyAsync(w, wts, 32 * V * sizeof(double), cudaMemcpyDefault, L->stream));
  CVCB_CUDA(cudaMemsetAsync(A, 0, 120 * fs * sizeof(double2), L->stream));
  CVCB_CUDA(cudaMemsetAsync(G, 0, 36 * V * sizeof(double2), L->stream));

  ZPlan plans[4];
  double Us[4][18];
  std::vector<ZMeta> meta(4 * 24 * 6);
  CVCB_TRY(make_zplans(L, S.src, plans, Us, meta.data()));
  const int blocks = (g.V + 127) / 128;
  const double4 ph01 = make_double4(L->phase[0], L->phase[1], L->phase[2], L->phase[3]);
  const double4 ph23 = make_double4(L->phase[4], L->phase[5], L->phase[6], L->phase[7]);
  const int nbl = 64;  // blocks per pair in k_pair_dots
  void *pbuf;
  CVCB_TRY(ensure_buffer(L, SLOT_ADJ_PART, (size_t)144 * nbl * sizeof(double2), &pbuf));
  std::vector<double2> part((size_t)144 * nbl);
  double gsrc[4][18];
  std::memset(gsrc, 0, sizeof gsrc);

  for (int nu = 0; nu < 4; ++nu) {
    CVCB_TRY(launch_cvc_z(L, Z, P + 60 * fs, plans[nu]));
    const double2 *Pcol[24];
    for (int c = 0; c < 12; ++c) {
      Pcol[c] = P + (48 + c) * fs;            // part 0: up at y
      Pcol[12 + c] = P + (12 * nu + c) * fs;  // part 1: up at y + nu-hat
    }
    // adjoint sources of the up columns: A_up += -1/4 K(Z)
    ColPtrs cp;
    for (int col = 0; col < 24; ++col) {
      cp.in[col] = Z + col * fs;
      cp.out[col] = A + (col < 12 ? 48 + col : 12 * nu + (col - 12)) * fs;
    }
    // part-0 and part-1 targets can coincide only for nu = 4, never here
    k_weighted_hop<1><<<dim3(blocks, 24), 128, 0, L->stream>>>(cp, w, nu, L->U64, g, -0.25, 1);
    CVCB_LAUNCHED(L);
    // H columns (transpose w.r.t. the dn columns)
    for (int col = 0; col < 24; ++col) {
      cp.in[col] = Pcol[col];
      cp.out[col] = H + col * fs;
    }
    k_weighted_hop<0><<<dim3(blocks, 24), 128, 0, L->stream>>>(cp, w, nu, L->U64, g, 1.0, 0);
    CVCB_LAUNCHED(L);
    // A_dn[d] += -1/4 conj(coef) H[col] for every plan term (col, d)
    MixPlan mp{};
    std::vector<int> outs;
    for (int col = 0; col < 24; ++col)
      for (int q = 0; q < 6; ++q) {
        const int d = plans[nu].t[col][q].src;  // 0..59 within dn
        int o = -1;
        for (int k = 0; k < (int)outs.size(); ++k)
          if (outs[k] == d) o = k;
        if (o < 0) {
          o = (int)outs.size();
          outs.push_back(d);
          mp.out_index[o] = 60 + d;
          mp.nterm[o] = 0;
        }
        const double2 cf = plans[nu].t[col][q].coef;
        MixTerm &t = mp.t[o][mp.nterm[o]++];
        t.src = col;
        t.coef = make_double2(-0.25 * cf.x, 0.25 * cf.y);  // -1/4 conj(coef)
      }
    mp.nout = (int)outs.size();
    k_mix<<<blocks, 128, 0, L->stream>>>(A, H, mp, g.V);
    CVCB_LAUNCHED(L);
    // T[col][q] = -1/4 sum_x <X_d(x), H_col(x)>, for the source-link gradient
    DotPairs dp;
    for (int col = 0; col < 24; ++col)
      for (int q = 0; q < 6; ++q) {
        dp.a[col * 6 + q] = P + (60 + plans[nu].t[col][q].src) * fs;
        dp.b[col * 6 + q] = H + col * fs;
      }
    k_pair_dots<<<dim3(nbl, 144), 256, 0, L->stream>>>(dp, g.V, 0, static_cast<double2 *>(pbuf),
                                                      nbl);
    CVCB_LAUNCHED(L);
    CVCB_CUDA(cudaMemcpyAsync(part.data(), pbuf, part.size() * sizeof(double2),
                              cudaMemcpyDeviceToHost, L->stream));
    CVCB_CUDA(cudaStreamSynchronize(L->stream));
    const double pr = L->phase[2 * nu], pi = L->phase[2 * nu + 1];
    for (int col = 0; col < 24; ++col)
      for (int q = 0; q < 6; ++q) {
        const double2 T0 = host_sum_partials(part, col * 6 + q, nbl);
        const double Tr = -0.25 * T0.x, Ti = -0.25 * T0.y;
        const ZMeta &m = meta[(nu * 24 + col) * 6 + q];
        const double kTr = m.k.x * Tr - m.k.y * Ti, kTi = m.k.x * Ti + m.k.y * Tr;  // k T
        if (m.part == 0) {  // L += Re(k T e^{i th} U[ia][ib]) -> G += conj(k T e^{i th})
          const double ar = kTr * pr - kTi * pi, ai = kTr * pi + kTi * pr;
          gsrc[nu][2 * (3 * m.ia + m.ib)] += ar;
          gsrc[nu][2 * (3 * m.ia + m.ib) + 1] += -ai;
        } else {  // L += Re(k T conj(e^{i th} U[ib][ia])) -> G += k T e^{-i th}
          const double ar = kTr * pr + kTi * pi, ai = kTi * pr - kTr * pi;
          gsrc[nu][2 * (3 * m.ib + m.ia)] += ar;
          gsrc[nu][2 * (3 * m.ib + m.ia) + 1] += ai;
        }
      }
    // explicit sink-link gradient of the conserved-current vertices
    PairPtrs pp;
    pp.n = 24;
    for (int col = 0; col < 24; ++col) {
      pp.left[col] = Z + col * fs;
      pp.right[col] = Pcol[col];
    }
    k_force<1><<<dim3(blocks, 4), 128, 0, L->stream>>>(G, pp, w, nu, g, ph01, ph23);
    CVCB_LAUNCHED(L);
  }

  // adjoint solves: lambda_up = g5 Q(-mu)^-1 g5 A_up, lambda_dn = g5 Q(mu)^-1 g5 A_dn
  double *C = static_cast<double *>(cvc), *B = static_cast<double *>(bsrc);
  for (int f = 0; f < 120; ++f) {
    CVCB_TRY(launch_g5(L, A + f * fs, g.V));
    CVCB_TRY(spinor_out(L, B + f * fstride, A + f * fs, g.V));
  }
  int rc = solve_columns(L, C, B, &S.params, -L->mu, L->mu, 60, 60, fstride);
  if (rc < 0) return rc;
  double2 *Lam = A;  // reuse
  for (int f = 0; f < 120; ++f) {
    CVCB_TRY(spinor_in(L, Lam + f * fs, C + f * fstride, g.V));
    CVCB_TRY(launch_g5(L, Lam + f * fs, g.V));
  }
  // dL/dmu, dL/dkappa
  DotPairs dp;
  for (int f = 0; f < 120; ++f) {
    dp.a[f] = Lam + f * fs;
    dp.b[f] = P + f * fs;
  }
  std::vector<double2> p1((size_t)120 * nbl), p2((size_t)120 * nbl);
  void *pbuf2;
  CVCB_TRY(ensure_buffer(L, SLOT_ADJ_PART, (size_t)144 * nbl * sizeof(double2), &pbuf2));
  k_pair_dots<<<dim3(nbl, 120), 256, 0, L->stream>>>(dp, g.V, 1, static_cast<double2 *>(pbuf2),
                                                    nbl);
  CVCB_LAUNCHED(L);
  CVCB_CUDA(cudaMemcpyAsync(p1.data(), pbuf2, p1.size() * sizeof(double2), cudaMemcpyDeviceToHost,
                            L->stream));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  k_pair_dots<<<dim3(nbl, 120), 256, 0, L->stream>>>(dp, g.V, 0, static_cast<double2 *>(pbuf2),
                                                    nbl);
  CVCB_LAUNCHED(L);
  CVCB_CUDA(cudaMemcpyAsync(p2.data(), pbuf2, p2.size() * sizeof(double2), cudaMemcpyDeviceToHost,
                            L->stream));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  double dmu = 0, dka = 0;
  for (int f = 0; f < 120; ++f) {
    const double2 d5 = host_sum_partials(p1, f, nbl), d1 = host_sum_partials(p2, f, nbl);
    dmu += f < 60 ? d5.y : -d5.y;  // Im<lam_up, g5 up> - Im<lam_dn, g5 dn>
    dka += d1.x;
  }
  dka *= 1.0 / (2.0 * L->kappa * L->kappa);
  if (dLdmu) *dLdmu = dmu;
  if (dLdkappa) *dLdkappa = dka;

  if (dLdU) {
    // gauge force of the 120 (lambda, column) pairs
    for (int f0 = 0; f0 < 120; f0 += kMaxCols) {
      PairPtrs pp;
      pp.n = std::min(kMaxCols, 120 - f0);
      for (int k = 0; k < pp.n; ++k) {
        pp.left[k] = Lam + (f0 + k) * fs;
        pp.right[k] = P + (f0 + k) * fs;
      }
      k_force<0><<<dim3(blocks, 4), 128, 0, L->stream>>>(G, pp, w, 0, g, ph01, ph23);
      CVCB_LAUNCHED(L);
    }
    std::vector<double> out((size_t)72 * V);
    void *gcvc;
    CVCB_TRY(ensure_buffer(L, SLOT_ADJ_B, 72 * V * sizeof(double), &gcvc));
    k_grad_to_cvc<<<blocks, 128, 0, L->stream>>>(static_cast<double *>(gcvc), G, g);
    CVCB_LAUNCHED(L);
    CVCB_CUDA(cudaMemcpyAsync(out.data(), gcvc, out.size() * sizeof(double),
                              cudaMemcpyDeviceToHost, L->stream));
    CVCB_CUDA(cudaStreamSynchronize(L->stream));
    for (int nu = 0; nu < 4; ++nu)
      for (int k = 0; k < 18; ++k) out[18 * (4 * (size_t)S.src + nu) + k] += gsrc[nu][k];
    CVCB_CUDA(cudaMemcpyAsync(dLdU, out.data(), out.size() * sizeof(double), cudaMemcpyDefault,
                              L->stream));
    CVCB_CUDA(cudaStreamSynchronize(L->stream));
  }
  return release_columns_if_over_budget(L);
}

}  // namespace cvcb

extern "C" {

int cvcb_pi_forward(cvcb_lattice *L, int source_site, const cvcb_solver_params *params,
                    double keep_bytes, double *conn, double *contact) {
  if (!L || !params || !conn) return CVCB_ERR_NULL;
  if (!L->have_gauge) {
    cvcb::set_error("no gauge field uploaded");
    return CVCB_ERR_STATE;
  }
  CVCB_CUDA(cudaSetDevice(L->device));
  return cvcb::pi_forward(L, source_site, params, keep_bytes, conn, contact);
}

int cvcb_pi_tangent(cvcb_lattice *L, int parameter, double *dconn) {
  if (!L || !dconn) return CVCB_ERR_NULL;
  CVCB_CUDA(cudaSetDevice(L->device));
  return cvcb::pi_tangent(L, parameter, dconn);
}

int cvcb_pi_backward(cvcb_lattice *L, const double *weights, double *dL_dU, double *dL_dmu,
                     double *dL_dkappa) {
  if (!L || !weights) return CVCB_ERR_NULL;
  CVCB_CUDA(cudaSetDevice(L->device));
  return cvcb::pi_backward(L, weights, dL_dU, dL_dmu, dL_dkappa);
}

}  // extern "C"
