/* cvc_oracle.c -- plain-C restatement of the CVC hot path (test checker only).
 *
 * Test infrastructure: only tests, the smoke check and the benchmark's CPU
 * baseline load liboracle.so.  It restates, loop for loop where the result
 * depends on it, the reference functions cited at each definition, so that
 * the CUDA path can be compared with it on the same inputs.  Its own
 * agreement with the unmodified reference is checked separately (the
 * reference compiled from its sources into oracle/_ref/, and the committed
 * golden fixtures under tests/golden/).
 */
#include "cvc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------
 * geometry: cvc_geometry.c:17-177 (get_index), :179-341 (geometry),
 * :343-465 (init_geometry), non-MPI build (no halo; neighbours wrap).
 * ---------------------------------------------------------------------- */
static int lexic(const orc_lattice *L, int t, int x, int y, int z) {
  t = (t + L->T) % L->T;
  x = (x + L->LX) % L->LX;
  y = (y + L->LY) % L->LY;
  z = (z + L->LZ) % L->LZ;
  return ((t * L->LX + x) * L->LY + y) * L->LZ + z;
}

void orc_phases(int T, int LX, int LY, int LZ, const double bc[4], double ph[8]) {
  /* cvc_geometry.c:452-459; g_nproc_* = 1 without MPI. */
  const int ext[4] = {T, LX, LY, LZ};
  for (int mu = 0; mu < 4; mu++) {
    ph[2 * mu] = cos(bc[mu] * M_PI / (double)ext[mu]);
    ph[2 * mu + 1] = sin(bc[mu] * M_PI / (double)ext[mu]);
  }
}

/* The 16 gamma structures of init_gamma (cvc_utils.c:707-1520), in its order
 * 0..3 = g0..g3, 4 = 1, 5 = g5, 6..9 = g_mu g5, 10..15 = g0g1, g0g2, g0g3,
 * g1g2, g1g3, g2g3, in the basis of cvc_utils.c:708-748.  Each has one entry
 * per row equal to +-1 or +-i, so it acts on the 24 reals of a spinor as a
 * permutation with signs; that is the table form the reference stores. */
typedef struct { double re, im; } cplx;
static void mat_mul4(cplx c[4][4], cplx a[4][4], cplx b[4][4]) {
  cplx r[4][4];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double re = 0, im = 0;
      for (int k = 0; k < 4; k++) {
        re += a[i][k].re * b[k][j].re - a[i][k].im * b[k][j].im;
        im += a[i][k].re * b[k][j].im + a[i][k].im * b[k][j].re;
      }
      r[i][j].re = re; r[i][j].im = im;
    }
  memcpy(c, r, sizeof r);
}

void orc_gamma_tables(int perm[16][24], int sign[16][24]) {
  cplx g[16][4][4];
  memset(g, 0, sizeof g);
  /* gamma_0 */
  g[0][0][2].re = -1; g[0][1][3].re = -1; g[0][2][0].re = -1; g[0][3][1].re = -1;
  /* gamma_1 */
  g[1][0][3].im = -1; g[1][1][2].im = -1; g[1][2][1].im = 1; g[1][3][0].im = 1;
  /* gamma_2 */
  g[2][0][3].re = -1; g[2][1][2].re = 1; g[2][2][1].re = 1; g[2][3][0].re = -1;
  /* gamma_3 */
  g[3][0][2].im = -1; g[3][1][3].im = 1; g[3][2][0].im = 1; g[3][3][1].im = -1;
  for (int a = 0; a < 4; a++) g[4][a][a].re = 1;
  mat_mul4(g[5], g[0], g[1]);
  mat_mul4(g[5], g[5], g[2]);
  mat_mul4(g[5], g[5], g[3]);
  for (int mu = 0; mu < 4; mu++) mat_mul4(g[6 + mu], g[mu], g[5]);
  int k = 10;
  for (int a = 0; a < 4; a++)
    for (int b = a + 1; b < 4; b++) mat_mul4(g[k++], g[a], g[b]);

  for (int n = 0; n < 16; n++)
    for (int a = 0; a < 4; a++) {
      int b = 0;
      for (int j = 0; j < 4; j++)
        if (fabs(g[n][a][j].re) + fabs(g[n][a][j].im) > 0.5) b = j;
      cplx v = g[n][a][b];
      for (int c = 0; c < 3; c++) {
        int ra = 2 * (3 * a + c), rb = 2 * (3 * b + c);
        if (fabs(v.im) < 0.5) {
          int s = v.re > 0 ? 1 : -1;
          perm[n][ra] = rb;     sign[n][ra] = s;
          perm[n][ra + 1] = rb + 1; sign[n][ra + 1] = s;
        } else { /* (s i)(re + i im) = -s im + i s re */
          int s = v.im > 0 ? 1 : -1;
          perm[n][ra] = rb + 1; sign[n][ra] = -s;
          perm[n][ra + 1] = rb;     sign[n][ra + 1] = s;
        }
      }
    }
}

int orc_lattice_init(orc_lattice *L, int T, int LX, int LY, int LZ, double kappa, double mu,
                     const double bc[4]) {
  memset(L, 0, sizeof *L);
  L->T = T; L->LX = LX; L->LY = LY; L->LZ = LZ;
  L->V = T * LX * LY * LZ;
  L->kappa = kappa; L->mu = mu;
  double ph[8];
  orc_phases(T, LX, LY, LZ, bc, ph);
  for (int m = 0; m < 4; m++) { L->phase[m][0] = ph[2 * m]; L->phase[m][1] = ph[2 * m + 1]; }
  L->iup = (int *)malloc(sizeof(int) * 4 * (size_t)L->V);
  L->idn = (int *)malloc(sizeof(int) * 4 * (size_t)L->V);
  if (!L->iup || !L->idn) return 1;
  for (int t = 0; t < T; t++)
    for (int x = 0; x < LX; x++)
      for (int y = 0; y < LY; y++)
        for (int z = 0; z < LZ; z++) {
          int ix = lexic(L, t, x, y, z);
          L->iup[4 * ix + 0] = lexic(L, t + 1, x, y, z);
          L->iup[4 * ix + 1] = lexic(L, t, x + 1, y, z);
          L->iup[4 * ix + 2] = lexic(L, t, x, y + 1, z);
          L->iup[4 * ix + 3] = lexic(L, t, x, y, z + 1);
          L->idn[4 * ix + 0] = lexic(L, t - 1, x, y, z);
          L->idn[4 * ix + 1] = lexic(L, t, x - 1, y, z);
          L->idn[4 * ix + 2] = lexic(L, t, x, y - 1, z);
          L->idn[4 * ix + 3] = lexic(L, t, x, y, z - 1);
        }
  orc_gamma_tables(L->gperm, L->gsign);
  return 0;
}

void orc_lattice_free(orc_lattice *L) {
  free(L->iup); free(L->idn);
  L->iup = L->idn = NULL;
}

/* All tables of geometry() (cvc_geometry.c:179-298) for a non-MPI build:
 * g_ipt is the (T+2)*LX*LY*LZ block of init_geometry (rows T, T+1 stay 0),
 * g_isevent is indexed by ((t*LZ+z)*LY+y)*LX+x. */
void orc_geometry_tables(const orc_lattice *L, int *ipt, int *iup, int *idn, int *lexic2eo,
                         int *eo2lexic, int *iseven, int *isevent, int *lexic2eot,
                         int *eot2lexic) {
  const int T = L->T, LX = L->LX, LY = L->LY, LZ = L->LZ, V = L->V;
  memset(ipt, 0, sizeof(int) * (size_t)(T + 2) * LX * LY * LZ);
  for (int t = 0; t < T; t++)
    for (int x = 0; x < LX; x++)
      for (int y = 0; y < LY; y++)
        for (int z = 0; z < LZ; z++) {
          int ix = lexic(L, t, x, y, z);
          ipt[((t * LX + x) * LY + y) * LZ + z] = ix;
          iseven[ix] = ((t + x + y + z) % 2) == 0;
          isevent[((t * LZ + z) * LY + y) * LX + x] = iseven[ix];
        }
  memcpy(iup, L->iup, sizeof(int) * 4 * (size_t)V);
  memcpy(idn, L->idn, sizeof(int) * 4 * (size_t)V);
  int ie = 0, io = 0;
  for (int ix = 0; ix < V; ix++) {
    if (iseven[ix]) { lexic2eo[ix] = ie; eo2lexic[ie] = ix; ie++; }
    else { lexic2eo[ix] = io + V / 2; eo2lexic[io + V / 2] = ix; io++; }
  }
  ie = 0; io = 0;
  int itzyx = 0;
  for (int t = 0; t < T; t++)
    for (int z = 0; z < LZ; z++)
      for (int y = 0; y < LY; y++)
        for (int x = 0; x < LX; x++) {
          int ix = ipt[((t * LX + x) * LY + y) * LZ + z];
          if (isevent[itzyx]) { lexic2eot[ix] = ie; eot2lexic[ie] = ix; ie++; }
          else { lexic2eot[ix] = io + V / 2; eot2lexic[io + V / 2] = ix; io++; }
          itzyx++;
        }
}

/* ------------------------------------------------------------------------
 * small algebra, with the semantics of cvc_linalg.h / cvc_complex.h
 * ---------------------------------------------------------------------- */
static void fv_gamma(const orc_lattice *L, double *s, int g, const double *t) {
  /* _fv_eq_gamma_ti_fv, cvc_linalg.h:1344 */
  for (int i = 0; i < 24; i++) s[i] = t[L->gperm[g][i]] * L->gsign[g][i];
}
static void cm_ti_co(double *A, const double *B, const double c[2]) {
  /* _cm_eq_cm_ti_co, cvc_linalg.h:271 */
  for (int i = 0; i < 9; i++) {
    double re = B[2 * i], im = B[2 * i + 1];
    A[2 * i] = re * c[0] - im * c[1];
    A[2 * i + 1] = re * c[1] + im * c[0];
  }
}
static void fv_cm_ti_fv(double *s, const double *A, const double *t) {
  /* _fv_eq_cm_ti_fv, cvc_linalg.h:1111: s_a = A t_a per spin a, with the
   * macro's left-to-right evaluation order (so results are bit-identical) */
  for (int a = 0; a < 4; a++) {
    const double *u = t + 6 * a;
    double *o = s + 6 * a;
    for (int i = 0; i < 3; i++) {
      const double *r = A + 6 * i;
      o[2 * i] = r[0] * u[0] - r[1] * u[1] + r[2] * u[2] - r[3] * u[3] + r[4] * u[4] - r[5] * u[5];
      o[2 * i + 1] = r[0] * u[1] + r[1] * u[0] + r[2] * u[3] + r[3] * u[2] + r[4] * u[5] + r[5] * u[4];
    }
  }
}
static void fv_cm_dag_ti_fv(double *s, const double *A, const double *t) {
  /* _fv_eq_cm_dag_ti_fv, cvc_linalg.h:1227: s_a = A^dagger t_a */
  for (int a = 0; a < 4; a++) {
    const double *u = t + 6 * a;
    double *o = s + 6 * a;
    for (int i = 0; i < 3; i++) {
      const double *c0 = A + 2 * i, *c1 = A + 6 + 2 * i, *c2 = A + 12 + 2 * i;
      o[2 * i] = c0[0] * u[0] + c0[1] * u[1] + c1[0] * u[2] + c1[1] * u[3] + c2[0] * u[4] + c2[1] * u[5];
      o[2 * i + 1] = c0[0] * u[1] - c0[1] * u[0] + c1[0] * u[3] - c1[1] * u[2] + c2[0] * u[5] - c2[1] * u[4];
    }
  }
}
static void co_fv_dag_ti_fv(double c[2], const double *s, const double *t) {
  /* _co_eq_fv_dag_ti_fv, cvc_linalg.h:669: c = sum_k conj(s_k) t_k, summed
   * over the 24 reals left to right as the macro does */
  double re = s[0] * t[0], im = s[0] * t[1] - s[1] * t[0];
  re += s[1] * t[1];
  for (int k = 2; k < 24; k += 2) {
    re = re + s[k] * t[k];
    re = re + s[k + 1] * t[k + 1];
    im = im + s[k] * t[k + 1];
    im = im - s[k + 1] * t[k];
  }
  c[0] = re; c[1] = im;
}

/* ------------------------------------------------------------------------
 * operators
 * ---------------------------------------------------------------------- */
/* The hopping sum  sum_mu [ (1 - g_mu) U_mu(x) phi(x+mu)
 *                          + (1 + g_mu) U_mu(x-mu)^dagger phi(x-mu) ]
 * with the boundary phase on every link, in the order of Q_phi.c:54-146
 * (-t, +t, -x, +x, -y, +y, -z, +z). */
static void hop_sum(const orc_lattice *L, int ix, double *acc, const double *phi) {
  double U[18], s1[24], s2[24];
  for (int i = 0; i < 24; i++) acc[i] = 0;
  for (int mu = 0; mu < 4; mu++) {
    /* negative mu direction */
    int jx = L->idn[4 * ix + mu];
    const double *p = phi + 24 * (size_t)jx;
    fv_gamma(L, s1, mu, p);
    for (int i = 0; i < 24; i++) s1[i] += p[i];
    cm_ti_co(U, L->gauge + 18 * (4 * (size_t)jx + mu), L->phase[mu]);
    fv_cm_dag_ti_fv(s2, U, s1);
    for (int i = 0; i < 24; i++) acc[i] += s2[i];
    /* positive mu direction */
    jx = L->iup[4 * ix + mu];
    p = phi + 24 * (size_t)jx;
    fv_gamma(L, s1, mu, p);
    for (int i = 0; i < 24; i++) s1[i] = -s1[i] + p[i];
    cm_ti_co(U, L->gauge + 18 * (4 * (size_t)ix + mu), L->phase[mu]);
    fv_cm_ti_fv(s2, U, s1);
    for (int i = 0; i < 24; i++) acc[i] += s2[i];
  }
}

/* xi = [1/(2 kappa) + i mutm g5] phi - 1/2 hop_sum  (Q_phi.c:38-188 with
 * mutm = g_mu; Q_phi.c:1092-1242 for explicit mutm). */
static void q_site(const orc_lattice *L, int ix, double *out, const double *phi, double mutm) {
  double acc[24], s1[24];
  hop_sum(L, ix, acc, phi);
  const double *p = phi + 24 * (size_t)ix;
  const double k2 = 0.5 / L->kappa;
  fv_gamma(L, s1, 5, p);
  for (int k = 0; k < 12; k++) {
    /* i*mutm*(re + i im) = -mutm*im + i mutm*re */
    out[2 * k] = -0.5 * acc[2 * k] + k2 * p[2 * k] + (-mutm * s1[2 * k + 1]);
    out[2 * k + 1] = -0.5 * acc[2 * k + 1] + k2 * p[2 * k + 1] + (mutm * s1[2 * k]);
  }
}

void orc_Q_phi_tbc(const orc_lattice *L, double *xi, const double *phi) {
  for (int ix = 0; ix < L->V; ix++) q_site(L, ix, xi + 24 * (size_t)ix, phi, L->mu);
}

void orc_Q_phi(const orc_lattice *L, double *xi, const double *phi, double mutm) {
  for (int ix = 0; ix < L->V; ix++) q_site(L, ix, xi + 24 * (size_t)ix, phi, mutm);
}

/* Q_phi.c:789-934: xi = g5 Q(mutm) phi, written per site after the sum. */
void orc_Qf5(const orc_lattice *L, double *xi, const double *phi, double mutm) {
  double s3[24];
  for (int ix = 0; ix < L->V; ix++) {
    q_site(L, ix, s3, phi, mutm);
    fv_gamma(L, xi + 24 * (size_t)ix, 5, s3);
  }
}

/* Q_phi.c:399-528: xi = -kappa * hop_sum. */
void orc_Hopping(const orc_lattice *L, double *xi, const double *phi) {
  double acc[24];
  for (int ix = 0; ix < L->V; ix++) {
    hop_sum(L, ix, acc, phi);
    for (int i = 0; i < 24; i++) xi[24 * (size_t)ix + i] = -L->kappa * acc[i];
  }
}

/* Q_phi.c:350-362 */
void orc_g5_phi(const orc_lattice *L, double *phi) {
  double s[24];
  for (int ix = 0; ix < L->V; ix++) {
    fv_gamma(L, s, 5, phi + 24 * (size_t)ix);
    memcpy(phi + 24 * (size_t)ix, s, sizeof s);
  }
}

/* Q_phi.c:576-589: phi = (1 - i sign 2 kappa mu g5) phi / (1 + (2 kappa mu)^2) */
void orc_mul_one_pm_imu_inv(const orc_lattice *L, double *phi, double sign, int V) {
  const double m = 2. * L->kappa * L->mu;
  const double norminv = 1. / (1. + m * m);
  double s1[24];
  for (int ix = 0; ix < V; ix++) {
    double *p = phi + 24 * (size_t)ix;
    fv_gamma(L, s1, 5, p);
    const double c = -sign * m;
    for (int k = 0; k < 12; k++) {
      double re = p[2 * k] + (-c * s1[2 * k + 1]);
      double im = p[2 * k + 1] + (c * s1[2 * k]);
      p[2 * k] = re * norminv;
      p[2 * k + 1] = im * norminv;
    }
  }
}

/* ------------------------------------------------------------------------
 * reductions: invert_Qtm.c:28-84 (per-site dot, then left-to-right sum)
 * ---------------------------------------------------------------------- */
void orc_scalar_product_co(double w[2], const double *xi, const double *phi, int V) {
  double re = 0, im = 0, c[2];
  for (int ix = 0; ix < V; ix++) {
    co_fv_dag_ti_fv(c, xi + 24 * (size_t)ix, phi + 24 * (size_t)ix);
    re += c[0]; im += c[1];
  }
  w[0] = re; w[1] = im;
}

void orc_scalar_product_re(double *r, const double *xi, const double *phi, int V) {
  double re = 0, c[2];
  for (int ix = 0; ix < V; ix++) {
    co_fv_dag_ti_fv(c, xi + 24 * (size_t)ix, phi + 24 * (size_t)ix);
    re += c[0];
  }
  *r = re;
}

/* ------------------------------------------------------------------------
 * solvers
 * ---------------------------------------------------------------------- */
static void c_div(double r[2], const double a[2], const double b[2]) {
  /* _co_eq_co_ti_co_inv, cvc_complex.h:26: a * conj(b) / |b|^2 */
  double n = b[0] * b[0] + b[1] * b[1];
  double re = (a[0] * b[0] + a[1] * b[1]) / n;
  double im = (a[1] * b[0] - a[0] * b[1]) / n;
  r[0] = re; r[1] = im;
}
static void c_mul(double r[2], const double a[2], const double b[2]) {
  double re = a[0] * b[0] - a[1] * b[1];
  double im = a[0] * b[1] + a[1] * b[0];
  r[0] = re; r[1] = im;
}
/* y = a - c*b over n complex numbers */
static void v_amcb(double *y, const double *a, const double c[2], const double *b, size_t n) {
  for (size_t k = 0; k < n; k++) {
    double br = b[2 * k], bi = b[2 * k + 1];
    double re = a[2 * k] - (c[0] * br - c[1] * bi);
    double im = a[2 * k + 1] - (c[0] * bi + c[1] * br);
    y[2 * k] = re; y[2 * k + 1] = im;
  }
}

typedef void (*orc_op)(const orc_lattice *L, double *out, const double *in, double *aux);

static void op_Q(const orc_lattice *L, double *out, const double *in, double *aux) {
  (void)aux;
  orc_Q_phi_tbc(L, out, in);
}
/* invert_Qtm.c:325-327: Qf5(aux, in, -mu); Qf5(out, aux, +mu) */
static void op_her(const orc_lattice *L, double *out, const double *in, double *aux) {
  orc_Qf5(L, aux, in, -L->mu);
  orc_Qf5(L, out, aux, L->mu);
}

/* The BiCGStab loop shared by invert_Qtm (invert_Qtm.c:86-270) and
 * invert_Qtm_her (:276-478): identical updates, operator and right-hand side
 * differ. */
static int bicgstab(const orc_lattice *L, orc_op A, double *x, const double *rhs, double normb,
                    double prec, int nmax, double *work, double *norm_out) {
  const size_t n = 12 * (size_t)L->V, N = 24 * (size_t)L->V;
  double *r1 = work, *r2 = work + N, *s = work + 2 * N, *t = work + 3 * N, *p = work + 4 * N,
         *p2 = work + 5 * N, *aux = work + 6 * N;
  double alpha[2], beta[2], omega[2], w[2], w2[2], w3[2], r0rn[2], u, norm;
  A(L, p, x, aux);
  for (size_t k = 0; k < N; k++) p[k] = rhs[k] - p[k];
  orc_scalar_product_re(&norm, p, p, L->V);
  if (norm <= prec * normb) { *norm_out = norm; return -100; } /* start guess already solves */
  memcpy(r1, p, N * sizeof(double));
  memcpy(r2, p, N * sizeof(double));
  A(L, p2, p, aux);
  int niter;
  for (niter = 0; niter <= nmax; niter++) {
    orc_scalar_product_co(r0rn, r2, r1, L->V);
    orc_scalar_product_co(w, r2, p2, L->V);
    c_div(alpha, r0rn, w);
    v_amcb(s, r1, alpha, p2, n);
    A(L, t, s, aux);
    orc_scalar_product_co(w, t, s, L->V);
    orc_scalar_product_re(&u, t, t, L->V);
    /* _co_eq_co_ti_re(&omega, &w, 1./u) expands to w.re*1./u = w.re/u */
    omega[0] = w[0] * 1. / u; omega[1] = w[1] * 1. / u;
    v_amcb(r1, s, omega, t, n);
    orc_scalar_product_re(&norm, r1, r1, L->V);
    if (norm <= prec * normb) break;
    for (size_t k = 0; k < n; k++) {
      double sr = s[2 * k], si = s[2 * k + 1], pr = p[2 * k], pi = p[2 * k + 1];
      x[2 * k] += omega[0] * sr - omega[1] * si;
      x[2 * k + 1] += omega[0] * si + omega[1] * sr;
      x[2 * k] += alpha[0] * pr - alpha[1] * pi;
      x[2 * k + 1] += alpha[0] * pi + alpha[1] * pr;
    }
    orc_scalar_product_co(w, r2, r1, L->V);
    c_div(w2, w, r0rn);
    c_div(w3, alpha, omega);
    c_mul(beta, w2, w3);
    r0rn[0] = w[0]; r0rn[1] = w[1];
    for (size_t k = 0; k < n; k++) {
      /* p = r1 + beta (p - omega p2) */
      double qr = p[2 * k] - (omega[0] * p2[2 * k] - omega[1] * p2[2 * k + 1]);
      double qi = p[2 * k + 1] - (omega[0] * p2[2 * k + 1] + omega[1] * p2[2 * k]);
      p[2 * k] = r1[2 * k] + (beta[0] * qr - beta[1] * qi);
      p[2 * k + 1] = r1[2 * k + 1] + (beta[0] * qi + beta[1] * qr);
    }
    A(L, p2, p, aux);
  }
  *norm_out = norm;
  return niter;
}

static double true_res2(const orc_lattice *L, const double *x, const double *phi, double *tmp) {
  const size_t N = 24 * (size_t)L->V;
  double r;
  orc_Q_phi_tbc(L, tmp, x);
  for (size_t k = 0; k < N; k++) tmp[k] -= phi[k];
  orc_scalar_product_re(&r, tmp, tmp, L->V);
  return r;
}

int orc_invert_Qtm(const orc_lattice *L, double *xi, const double *phi, double prec, int nmax,
                   double *work, double *tr2) {
  if (!xi || !phi || !work) return -2;
  double normb, norm;
  orc_scalar_product_re(&normb, phi, phi, L->V);
  int niter = bicgstab(L, op_Q, xi, phi, normb, prec, nmax, work, &norm);
  if (niter == -100) return 0; /* invert_Qtm.c:144-147 */
  if (!(norm <= prec * normb && niter <= nmax)) return -3;
  if (tr2) *tr2 = true_res2(L, xi, phi, work + 4 * 24 * (size_t)L->V) / normb;
  return niter;
}

int orc_invert_Qtm_her(const orc_lattice *L, double *xi, const double *phi, double prec,
                       int nmax, double *work, double *tr2) {
  if (!xi || !phi || !work) return -2;
  const size_t N = 24 * (size_t)L->V;
  double normb, norm;
  orc_scalar_product_re(&normb, phi, phi, L->V);
  /* rhs = g5 phi (invert_Qtm.c:329-333); kept in the p-slot's successor */
  double *g5phi = (double *)malloc(N * sizeof(double));
  if (!g5phi) return -2;
  memcpy(g5phi, phi, N * sizeof(double));
  orc_g5_phi(L, g5phi);
  int niter = bicgstab(L, op_her, xi, g5phi, normb, prec, nmax, work, &norm);
  free(g5phi);
  /* invert_Qtm.c:344-347 returns before the final Qf5(-mu) when the start
   * guess already satisfies the (normal-equation) criterion */
  if (niter == -100) return 0;
  /* x = Qf5(x, -mu) (invert_Qtm.c:443-446) */
  double *aux = work + 6 * N;
  orc_Qf5(L, aux, xi, -L->mu);
  memcpy(xi, aux, N * sizeof(double));
  if (!(norm <= prec * normb && niter <= nmax)) return -3;
  if (tr2) *tr2 = true_res2(L, xi, phi, work + 4 * N) / normb;
  return niter;
}

/* ------------------------------------------------------------------------
 * contraction: cvc_exact2_xspace.c:577-861, restated loop for loop.
 * gperm/gperm_sign/isimag follow :336-383.
 * ---------------------------------------------------------------------- */
static void cvc_hops(const orc_lattice *L, int mu, int ix, const double *phi, const double *chi,
                     double wf[2], double wb[2]) {
  double U[18], s1[24], s2[24];
  cm_ti_co(U, L->gauge + 18 * (4 * (size_t)ix + mu), L->phase[mu]);
  /* forward: chi(x)^dagger g5 (g_mu - 1) U phi(x+mu)   (:601-606) */
  fv_cm_ti_fv(s1, U, phi + 24 * (size_t)L->iup[4 * ix + mu]);
  fv_gamma(L, s2, mu, s1);
  for (int i = 0; i < 24; i++) s2[i] -= s1[i];
  fv_gamma(L, s1, 5, s2);
  co_fv_dag_ti_fv(wf, chi + 24 * (size_t)ix, s1);
  /* backward: chi(x+mu)^dagger g5 (g_mu + 1) U^dagger phi(x)   (:624-629) */
  fv_cm_dag_ti_fv(s1, U, phi + 24 * (size_t)ix);
  fv_gamma(L, s2, mu, s1);
  for (int i = 0; i < 24; i++) s2[i] += s1[i];
  fv_gamma(L, s1, 5, s2);
  co_fv_dag_ti_fv(wb, chi + 24 * (size_t)L->iup[4 * ix + mu], s1);
}

void orc_cvc_contract(const orc_lattice *L, const double *const *F, int src, double *conn,
                      double *contact) {
  const int V = L->V;
  int gperm[5][4], isimag[4];
  double gsign[5][4], Usrc[4][18];
  for (int ir = 0; ir < 4; ir++) {
    gperm[4][ir] = L->gperm[5][6 * ir] / 6;
    gsign[4][ir] = L->gsign[5][6 * ir];
  }
  for (int nu = 0; nu < 4; nu++) {
    for (int ir = 0; ir < 4; ir++) {
      gperm[nu][ir] = L->gperm[6 + nu][6 * ir] / 6;
      gsign[nu][ir] = L->gsign[6 + nu][6 * ir];
    }
    isimag[nu] = L->gperm[6 + nu][0] % 2;
    cm_ti_co(Usrc[nu], L->gauge + 18 * (4 * (size_t)src + nu), L->phase[nu]); /* :293-304 */
  }
  memset(conn, 0, sizeof(double) * 32 * (size_t)V);
  memset(contact, 0, sizeof(double) * 8);

  for (int part = 0; part < 2; part++) {
    for (int nu = 0; nu < 4; nu++) {
      for (int ir = 0; ir < 4; ir++) {
        /* g = 0: the g_nu g5 term (:581-640 / :727-786), g = 1: the g5 term
         * (:643-705 / :789-846), each looping ia, ib, mu as the reference */
        for (int g = 0; g < 2; g++) {
          int gi = g == 0 ? nu : 4;
          for (int ia = 0; ia < 3; ia++) {
            const double *phi = part == 0 ? F[4 * 12 + 3 * ir + ia] : F[nu * 12 + 3 * ir + ia];
            for (int ib = 0; ib < 3; ib++) {
              const double *chi = part == 0 ? F[60 + nu * 12 + 3 * gperm[gi][ir] + ib]
                                            : F[60 + 4 * 12 + 3 * gperm[gi][ir] + ib];
              /* part 0 multiplies Usource[nu](ia,ib); part 1 conj(Usource[nu](ib,ia)) */
              double us[2];
              if (part == 0) { us[0] = Usrc[nu][2 * (3 * ia + ib)]; us[1] = Usrc[nu][2 * (3 * ia + ib) + 1]; }
              else { us[0] = Usrc[nu][2 * (3 * ib + ia)]; us[1] = -Usrc[nu][2 * (3 * ib + ia) + 1]; }
              for (int mu = 0; mu < 4; mu++) {
                int imunu = 4 * mu + nu;
                for (int ix = 0; ix < V; ix++) {
                  double wf[2], wb[2], w1[2];
                  cvc_hops(L, mu, ix, phi, chi, wf, wb);
                  double *c = conn + 2 * (16 * (size_t)ix + imunu);
                  for (int h = 0; h < 2; h++) {
                    c_mul(w1, h == 0 ? wf : wb, us);
                    if (g == 0) {
                      if (!isimag[nu]) { c[0] += gsign[nu][ir] * w1[0]; c[1] += gsign[nu][ir] * w1[1]; }
                      else { c[0] += gsign[nu][ir] * w1[1]; c[1] -= gsign[nu][ir] * w1[0]; }
                    } else if (part == 0) {
                      c[0] -= gsign[4][ir] * w1[0]; c[1] -= gsign[4][ir] * w1[1];
                    } else {
                      c[0] += gsign[4][ir] * w1[0]; c[1] += gsign[4][ir] * w1[1];
                    }
                  }
                }
              }
            }
            if (g == 0) continue;
            /* contact term (:697-704, :837-844) */
            double s1[24], s2[24];
            if (part == 0) {
              fv_cm_ti_fv(s1, Usrc[nu], phi + 24 * (size_t)L->iup[4 * src + nu]);
              fv_gamma(L, s2, nu, s1);
              for (int i = 0; i < 24; i++) s2[i] -= s1[i];
              contact[2 * nu] += -0.5 * s2[2 * (3 * ir + ia)];
              contact[2 * nu + 1] += -0.5 * s2[2 * (3 * ir + ia) + 1];
            } else {
              fv_cm_dag_ti_fv(s1, Usrc[nu], phi + 24 * (size_t)src);
              fv_gamma(L, s2, nu, s1);
              for (int i = 0; i < 24; i++) s2[i] += s1[i];
              contact[2 * nu] += 0.5 * s2[2 * (3 * ir + ia)];
              contact[2 * nu + 1] += 0.5 * s2[2 * (3 * ir + ia) + 1];
            }
          }
        }
      }
    }
  }
  for (size_t k = 0; k < 32 * (size_t)V; k++) conn[k] *= -0.25; /* :861 */
}

void orc_cvc_ward(const orc_lattice *L, const double *conn, double *wi) {
  for (int ix = 0; ix < L->V; ix++)
    for (int nu = 0; nu < 4; nu++)
      for (int ri = 0; ri < 2; ri++) {
        double w = 0;
        for (int mu = 0; mu < 4; mu++) w += conn[2 * (16 * (size_t)ix + 4 * mu + nu) + ri];
        for (int mu = 0; mu < 4; mu++)
          w -= conn[2 * (16 * (size_t)L->idn[4 * ix + mu] + 4 * mu + nu) + ri];
        wi[8 * (size_t)ix + 2 * nu + ri] = w;
      }
}

/* p2gg_xspace.c:525-539 (single process: g_proc_coords = 0). */
void orc_p2gg_seq_source(const orc_lattice *L, double *source, const double *prop, int x0,
                         const int mom[3], int gamma_id, int pos) {
  memset(source, 0, sizeof(double) * 24 * (size_t)L->V);
  double s1[24];
  for (int x1 = 0; x1 < L->LX; x1++)
    for (int x2 = 0; x2 < L->LY; x2++)
      for (int x3 = 0; x3 < L->LZ; x3++) {
        int ix = lexic(L, x0, x1, x2, x3);
        double phase = (1. - 2. * pos) * 2. * M_PI *
                       ((x1)*mom[0] / (double)L->LX + (x2)*mom[1] / (double)L->LY +
                        (x3)*mom[2] / (double)L->LZ);
        double w[2] = {cos(phase), sin(phase)};
        fv_gamma(L, s1, gamma_id, prop + 24 * (size_t)ix);
        for (int k = 0; k < 12; k++) {
          double re = s1[2 * k], im = s1[2 * k + 1];
          source[24 * (size_t)ix + 2 * k] = re * w[0] - im * w[1];
          source[24 * (size_t)ix + 2 * k + 1] = re * w[1] + im * w[0];
        }
      }
}

/* cvc_utils.c:384-436, with the evaluation order of _cm_eq_cm_ti_cm
 * (cvc_linalg.h:382), _cm_eq_cm_ti_cm_dag (:296) and _co_eq_tr_cm (:195). */
static void cm_ti_cm(double *A, const double *B, const double *C) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      const double *b = B + 6 * i;
      A[2 * (3 * i + j)] = b[0] * C[2 * j] - b[1] * C[2 * j + 1] + b[2] * C[6 + 2 * j] -
                           b[3] * C[6 + 2 * j + 1] + b[4] * C[12 + 2 * j] - b[5] * C[12 + 2 * j + 1];
      A[2 * (3 * i + j) + 1] = b[0] * C[2 * j + 1] + b[1] * C[2 * j] + b[2] * C[6 + 2 * j + 1] +
                               b[3] * C[6 + 2 * j] + b[4] * C[12 + 2 * j + 1] + b[5] * C[12 + 2 * j];
    }
}
void orc_plaquette(const orc_lattice *L, double *pl, double linksum[2]) {
  double acc = 0;
  for (int ix = 0; ix < L->V; ix++)
    for (int mu = 0; mu < 3; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        const double *A = L->gauge + 72 * (size_t)ix + 18 * mu;
        const double *B = L->gauge + 72 * (size_t)L->iup[4 * ix + mu] + 18 * nu;
        const double *C = L->gauge + 72 * (size_t)ix + 18 * nu;
        const double *D = L->gauge + 72 * (size_t)L->iup[4 * ix + nu] + 18 * mu;
        double s[18], t[18], d[3];
        cm_ti_cm(s, A, B);
        cm_ti_cm(t, C, D);
        /* diagonal of u = s t^dagger: u_ii = sum_k s_ik conj(t_ik) */
        for (int i = 0; i < 3; i++) {
          const double *x = s + 6 * i, *y = t + 6 * i;
          d[i] = x[0] * y[0] + x[1] * y[1] + x[2] * y[2] + x[3] * y[3] + x[4] * y[4] + x[5] * y[5];
        }
        acc += d[0] + d[1] + d[2];
      }
  *pl = acc / ((double)L->V * 18.);
  linksum[0] = linksum[1] = 0;
  for (size_t k = 0; k < 36 * (size_t)L->V; k++) {
    linksum[0] += L->gauge[2 * k];
    linksum[1] += L->gauge[2 * k + 1];
  }
}
