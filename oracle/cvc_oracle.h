/* cvc_oracle.h -- plain-C restatement of the CVC propagator-and-contraction
 * path, used ONLY as the checker for the CUDA implementation.
 *
 * This is test infrastructure.  Nothing in the shipped library links or calls
 * it; the tests, the smoke check and the CPU-baseline leg of the benchmark do.
 *
 * Every function states the reference file:line it restates.  Field layouts
 * are CVC's in-memory layouts (global.h:55-61):
 *   spinor  : 24 doubles per site at 24*ix, component 2*(3*spin+colour)+re/im
 *   gauge   : 18 doubles per link at 18*(4*ix+mu), 3x3 complex row-major
 *   Pi_mu_nu: conn[2*(16*ix + 4*mu + nu) + re/im]
 * Sites are CVC lexicographic: ix = ((t*LX + x)*LY + y)*LZ + z.
 */
#ifndef CVC_ORACLE_H
#define CVC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int T, LX, LY, LZ, V;
  double kappa, mu;          /* g_kappa, g_mu (bare mu, Q_phi.c:25-36) */
  double phase[4][2];        /* co_phase_up (cvc_geometry.c:451-459) */
  int *iup, *idn;            /* g_iup / g_idn, 4 per site */
  const double *gauge;       /* 72*V doubles */
  int gperm[16][24], gsign[16][24]; /* gamma_permutation / gamma_sign */
} orc_lattice;

/* --- geometry (cvc_geometry.c:17-465) -------------------------------- */
int orc_lattice_init(orc_lattice *L, int T, int LX, int LY, int LZ, double kappa, double mu,
                     const double bc_angle[4]);
void orc_lattice_free(orc_lattice *L);
void orc_geometry_tables(const orc_lattice *L, int *ipt, int *iup, int *idn, int *lexic2eo,
                         int *eo2lexic, int *iseven, int *isevent, int *lexic2eot, int *eot2lexic);
void orc_gamma_tables(int perm[16][24], int sign[16][24]);
void orc_phases(int T, int LX, int LY, int LZ, const double bc_angle[4], double ph[8]);

/* --- operators (Q_phi.c) ---------------------------------------------- */
void orc_Q_phi_tbc(const orc_lattice *L, double *xi, const double *phi);
void orc_Hopping(const orc_lattice *L, double *xi, const double *phi);
void orc_Qf5(const orc_lattice *L, double *xi, const double *phi, double mutm);
void orc_Q_phi(const orc_lattice *L, double *xi, const double *phi, double mutm);
void orc_g5_phi(const orc_lattice *L, double *phi);
void orc_mul_one_pm_imu_inv(const orc_lattice *L, double *phi, double sign, int V);

/* --- reductions and solvers (invert_Qtm.c) ---------------------------- */
void orc_scalar_product_co(double w[2], const double *xi, const double *phi, int V);
void orc_scalar_product_re(double *r, const double *xi, const double *phi, int V);
/* work: caller-provided 7*24*V doubles.  Returns niter, -2, or -3 as the
 * reference does; true_res2 (may be NULL) receives |Qx-phi|^2/|phi|^2. */
int orc_invert_Qtm(const orc_lattice *L, double *xi, const double *phi, double solver_precision,
                   int niter_max, double *work, double *true_res2);
int orc_invert_Qtm_her(const orc_lattice *L, double *xi, const double *phi,
                       double solver_precision, int niter_max, double *work, double *true_res2);

/* --- contraction (cvc_exact2_xspace.c:577-861) -------------------------
 * fields[0..59] = "up" (5 source shifts x 12 spin-colour), fields[60..119] =
 * "dn"; source = lexicographic source site.  conn (32*V doubles) is
 * overwritten; contact (8 doubles) receives the contact term. */
void orc_cvc_contract(const orc_lattice *L, const double *const *fields, int source_site,
                      double *conn, double *contact);
/* Ward identity divergence sum_mu [Pi_mu_nu(x) - Pi_mu_nu(x-mu)]
 * (cvc_exact2_xspace.c:928-1008); wi is 8*V doubles (4 nu, re/im). */
void orc_cvc_ward(const orc_lattice *L, const double *conn, double *wi);

/* --- P->gamma gamma sequential source (p2gg_xspace.c:525-539) ---------- */
void orc_p2gg_seq_source(const orc_lattice *L, double *source, const double *prop, int timeslice,
                         const int mom[3], int gamma_id, int propagator_position);

/* --- plaquette (cvc_utils.c:384-436) ----------------------------------- */
void orc_plaquette(const orc_lattice *L, double *pl, double linksum[2]);

#ifdef __cplusplus
}
#endif
#endif
