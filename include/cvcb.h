/* cvcb.h -- C ABI of the B200 implementation of CVC's propagator-and-
 * contraction path: the twisted-mass Wilson operator with boundary phases,
 * the BiCGStab/CG propagator solvers with their reductions, and the
 * conserved-vector-current contraction Pi_mu_nu(x).
 *
 * Conventions shared by every entry point
 * ---------------------------------------
 * - Field layouts are CVC's own (global.h:55-61 of the reference):
 *     spinor field : 24 doubles per site, site ix at 24*ix, component
 *                    2*(3*spin + colour) + re/im;
 *     gauge field  : 72 doubles per site, link U_mu(ix) at 18*(4*ix + mu),
 *                    3x3 complex row-major, WITHOUT the boundary phase;
 *     Pi_mu_nu     : conn[2*(16*ix + 4*mu + nu) + re/im].
 *   Sites are CVC lexicographic, ix = ((t*LX + x)*LY + y)*LZ + z, mu = 0..3
 *   is t, x, y, z.  All extents must be even.
 * - Pointers may be host memory or device memory of the lattice's GPU; the
 *   library detects which and copies host data through its own staging.
 * - Every call is asynchronous with respect to nothing: it returns after its
 *   results are in the caller's buffers.  Calls on one cvcb_lattice must come
 *   from one host thread at a time (the reference is single-threaded too).
 * - Return values: >= 0 success (solvers: iteration count), otherwise one of
 *   the CVCB_* codes below.  The library never calls exit().
 */
#ifndef CVCB_H
#define CVCB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  -2 and -3 are the reference's own solver returns
 * (invert_Qtm.c:112-113, 242-251); the others are new.  CVCB_BREAKDOWN:
 * a BiCGStab recursion scalar (alpha, omega, beta) became non-finite, which
 * the reference reports as -3 (invert_Qtm.c:213-216, 250); the namespace-cvc
 * drop-in and the Python mirror map it back to -3. */
#define CVCB_OK 0
#define CVCB_ERR_ARG (-1)
#define CVCB_ERR_NULL (-2)
#define CVCB_NO_CONVERGENCE (-3)
#define CVCB_BREAKDOWN (-4)
#define CVCB_ERR_STATE (-5)
#define CVCB_ERR_NOMEM (-6)
#define CVCB_ERR_CUDA (-7)

typedef struct cvcb_lattice cvcb_lattice;

/* Human-readable text of the last error on this host thread. */
const char *cvcb_last_error(void);
/* Library version string. */
const char *cvcb_version(void);

/* ---------------------------------------------------------------------
 * Geometry and tables (host only; no GPU needed)
 * ------------------------------------------------------------------- */

/* All index tables of the reference's init_geometry()/geometry() for a
 * single process (cvc_geometry.c:17-465): g_ipt as the (T+2)*LX*LY*LZ block
 * (rows t = T, T+1 zero), g_iup/g_idn as 4*V, g_lexic2eo, g_eo2lexic,
 * g_iseven, g_isevent, g_lexic2eot, g_eot2lexic as V each.  Bit-exact with
 * the reference.  Any pointer may be NULL to skip that table. */
int cvcb_geometry_tables(int T, int LX, int LY, int LZ, int *ipt, int *iup, int *idn,
                         int *lexic2eo, int *eo2lexic, int *iseven, int *isevent,
                         int *lexic2eot, int *eot2lexic);

/* gamma_permutation[16][24] / gamma_sign[16][24] of init_gamma
 * (cvc_utils.c:707-1520), bit-exact. */
int cvcb_gamma_tables(int *perm, int *sign);

/* co_phase_up[mu] = exp(i pi BCangle[mu] / L_mu) (cvc_geometry.c:452-459);
 * ph[2*mu] = re, ph[2*mu+1] = im. */
int cvcb_boundary_phases(int T, int LX, int LY, int LZ, const double bc_angle[4], double ph[8]);

/* ---------------------------------------------------------------------
 * Input generation (host only).  The reference has no generator for the
 * benchmark's gauge recipe, so this one is new; it uses the reference's RNG.
 * ------------------------------------------------------------------- */

/* RANLUX double-precision generator, restated from ranlxd.c:493-600
 * (rlxd_init(level, seed) followed by ranlxd(r, n)).  Bit-exact with the
 * reference for the same level and seed. */
int cvcb_ranlxd(int level, int seed, double *r, long n);

/* Gauge field U = exp(i eps H) per link, H = sum_a w_a lambda_a / 2 with
 * w_a standard normal from Box-Muller over ranlxd (as rangauss,
 * cvc_utils.c:2734-2760) after rlxd_init(1, seed); links filled in site
 * order, mu = 0..3, 8 normals per link.  U is then re-unitarised
 * (Gram-Schmidt on rows 0,1, row 2 = conj(row0 x row1)) so det U = 1 to
 * rounding.  Output in CVC layout, 72*V doubles. */
int cvcb_gauge_random(double *gauge, int T, int LX, int LY, int LZ, double eps, int seed);

/* ---------------------------------------------------------------------
 * Lattice context: one per GPU and host thread.  Holds the geometry, the
 * parameters (g_kappa, g_mu, BCangle), the gauge field in device layouts,
 * and device work space.
 * ------------------------------------------------------------------- */
int cvcb_lattice_create(cvcb_lattice **lat, int T, int LX, int LY, int LZ, int device);
int cvcb_lattice_destroy(cvcb_lattice *lat);

/* g_kappa, g_mu (the bare twisted mass, Q_phi.c:25-36) and BCangle[4]
 * (default_input_values.h:24-27: 1, 0, 0, 0). */
int cvcb_set_params(cvcb_lattice *lat, double kappa, double mu, const double bc_angle[4]);

/* Replaces g_gauge_field (72*V doubles, CVC layout, no phase).  The link
 * phases are applied inside the library, as Q_phi.c:66 does per use. */
int cvcb_upload_gauge(cvcb_lattice *lat, const double *gauge);

/* Largest deviation from SU(3) of the uploaded links: max over links of
 * max(|U U^dagger - 1|_max, |det U - 1|).  Compressed-link solvers are only
 * used when this is small (see cvcb_solver_params.link_recon). */
int cvcb_gauge_unitarity(cvcb_lattice *lat, double *dev);

/* ---------------------------------------------------------------------
 * Operators (reference: Q_phi.c).  xi and phi must not overlap.
 * ------------------------------------------------------------------- */

/* xi = Q phi, Q = 1/(2 kappa) + i mu g5 - 1/2 sum_mu [(1 - g_mu) U_mu(x)
 * phi(x+mu) + (1 + g_mu) U_mu(x-mu)^dagger phi(x-mu)], links times
 * co_phase_up.  Replaces void Q_phi_tbc(double *xi, double *phi),
 * Q_phi.c:38-188 (Q_phi.h:11). */
int cvcb_Q_phi_tbc(cvcb_lattice *lat, double *xi, const double *phi);

/* xi = -kappa sum_mu [...] (hopping term only, hopping-parameter
 * normalisation).  Replaces void Hopping(double *xi, double *phi),
 * Q_phi.c:399-528 (Q_phi.h:12). */
int cvcb_Hopping(cvcb_lattice *lat, double *xi, const double *phi);

/* xi = g5 Q(mutm) phi.  Replaces void Qf5(double *xi, double *phi,
 * double mutm), Q_phi.c:789-934 (Q_phi.h:27). */
int cvcb_Qf5(cvcb_lattice *lat, double *xi, const double *phi, double mutm);

/* xi = Q(mutm) phi.  Replaces void Q_phi(double *xi, double *phi,
 * const double mutm), Q_phi.c:1092-1242 (Q_phi.h:29). */
int cvcb_Q_phi(cvcb_lattice *lat, double *xi, const double *phi, double mutm);

/* phi = g5 phi in place.  Replaces void g5_phi(double *phi),
 * Q_phi.c:350-362 (Q_phi.h:51). */
int cvcb_g5_phi(cvcb_lattice *lat, double *phi);

/* phi = (1 - i sign 2 kappa mu g5) phi / (1 + (2 kappa mu)^2) on the first
 * V sites.  Replaces void mul_one_pm_imu_inv(double *phi, double sign,
 * int V), Q_phi.c:576-589 (Q_phi.h:14). */
int cvcb_mul_one_pm_imu_inv(cvcb_lattice *lat, double *phi, double sign, int V);

/* ---------------------------------------------------------------------
 * Reductions (reference: invert_Qtm.c:28-84).  Deterministic: the same
 * inputs give the same bits on every call.
 * ------------------------------------------------------------------- */

/* w = sum_x xi(x)^dagger phi(x) over the first V sites (w[0] = re,
 * w[1] = im).  Replaces void spinor_scalar_product_co(complex *w,
 * double *xi, double *phi, int V) (invert_Qtm.h:10). */
int cvcb_spinor_scalar_product_co(cvcb_lattice *lat, double *w, const double *xi,
                                  const double *phi, int V);
/* The same complex scalar product for callers that cannot allocate device
 * memory (their device memory belongs to a pool of their own, or a
 * cudaMalloc would synchronise a device they keep busy): no context is
 * needed and nothing is allocated.  No counterpart in the reference.
 * xi, phi (24*V doubles each) and w (2 doubles) are device memory of
 * `device`; stream is a cudaStream_t (NULL: the legacy default stream).
 * Stream-ordered: returns after enqueueing; w is ready when the stream
 * reaches the call.  Scratch is one fixed device array per GPU (about
 * 256 KB, held until the process exits), so V is limited to 5,592,405
 * sites; larger V returns CVCB_ERR_ARG.  All calls on a device share that
 * array: calls that overlap on the GPU race and must be serialised by the
 * caller.  The first call on a device looks up the array's address; make it
 * before any stream capture on that device. */
int cvcb_spinor_scalar_product_co_noalloc(int device, double *w, const double *xi,
                                          const double *phi, int V, void *stream);

/* r = Re sum_x xi(x)^dagger phi(x).  Replaces void
 * spinor_scalar_product_re(double *r, double *xi, double *phi, int V)
 * (invert_Qtm.h:9). */
int cvcb_spinor_scalar_product_re(cvcb_lattice *lat, double *r, const double *xi,
                                  const double *phi, int V);

/* ---------------------------------------------------------------------
 * FP64 solvers with the reference's algorithms and stopping rule:
 * |r|^2 <= solver_precision * |phi|^2 (squared norms, invert_Qtm.c:201).
 * xi holds the start guess on entry and the solution on exit.
 * Returns the iteration count, CVCB_ERR_NULL or CVCB_NO_CONVERGENCE as the
 * reference does, or CVCB_BREAKDOWN where the reference returns -3 after
 * its recursion produced a non-finite scalar.  true_res2 (may be NULL) receives |Q xi - phi|^2/|phi|^2.
 * ------------------------------------------------------------------- */

/* BiCGStab on Q.  Replaces int invert_Qtm(double *xi, double *phi,
 * int kwork), invert_Qtm.c:86-270 (invert_Qtm.h:11); the work fields
 * g_spinor_field[kwork..kwork+5] become device work space. */
int cvcb_invert_Qtm(cvcb_lattice *lat, double *xi, const double *phi, double solver_precision,
                    int niter_max, double *true_res2);

/* BiCGStab on g5 Q(mu) g5 Q(-mu) = Q(-mu)^dagger Q(-mu) with right-hand
 * side g5 phi, then xi = g5 Q(-mu) y.  Replaces int invert_Qtm_her(double
 * *xi, double *phi, int kwork), invert_Qtm.c:276-478 (invert_Qtm.h:12). */
int cvcb_invert_Qtm_her(cvcb_lattice *lat, double *xi, const double *phi,
                        double solver_precision, int niter_max, double *true_res2);

/* ---------------------------------------------------------------------
 * Batched solver: even/odd preconditioned CG on the normal equations of the
 * Schur complement, N right-hand sides per launch, optional reduced
 * precision with FP64 reliable updates.  No counterpart in the reference
 * (it reads propagators from files or calls tmLQCD, cvc_exact2_xspace.c:
 * 401-547); it solves the same system Q x = b.
 * ------------------------------------------------------------------- */
#define CVCB_PREC_DOUBLE 0
#define CVCB_PREC_SINGLE 1
#define CVCB_PREC_HALF 2

typedef struct {
  int precision;     /* CVCB_PREC_*: arithmetic/storage of the inner iterations */
  int link_recon;    /* 18 or 12 reals per link in the inner operator */
  int block_rhs;     /* right-hand sides per batch, at most 96 (0 = autotuned:
                        up to 96 for device fields, up to 24 for host fields,
                        whose transfers overlap the solve of another batch) */
  int block_threads; /* sites per stencil block, one rhs (FP32: one rhs pair) per
                        thread; a multiple
                        of 32 up to 256 (0 = autotuned shape) */
  int max_iter;      /* per right-hand side */
  int use_graph;     /* capture the inner iterations in a CUDA graph */
  double tol;        /* target |b - Q x|_2 / |b|_2, checked in FP64 */
  double delta;      /* reliable-update trigger: sloppy |r| fell by this factor
                        (0 = by inner precision: 0.1 FP16, 1e-4 FP32, 1e-8 FP64) */
} cvcb_solver_params;

typedef struct {
  int iterations;        /* inner iterations, summed over right-hand sides */
  int reliable_updates;  /* FP64 residual recomputations */
  int restarts;          /* directions restarted from the residual (after a
                            non-finite sloppy residual) */
  int converged;         /* right-hand sides that met tol */
  double max_true_res;   /* max over rhs of |b - Q x| / |b| in FP64 */
  double seconds;        /* wall time of the iterations */
  int batch_rhs;         /* right-hand sides per batch (given or autotuned) */
} cvcb_solver_stats;

/* Fills the defaults: single precision, 12-real links, autotuned blocks,
 * tol 1e-10, delta 0 (by precision), max_iter 20000, graphs on. */
void cvcb_solver_defaults(cvcb_solver_params *p);

/* x[i], b[i] for i < nrhs: CVC-layout spinor fields (host or device).  x is
 * output only (start guess zero). */
int cvcb_solve(cvcb_lattice *lat, double *const *x, const double *const *b, int nrhs,
               const cvcb_solver_params *params, cvcb_solver_stats *stats);

/* Average duration of one stencil launch on device-resident fields, timed
 * with CUDA events on the lattice's stream over `reps` back-to-back launches
 * after one warm-up launch.  kind 0: the full-lattice FP64 kernel behind
 * cvcb_Q_phi_tbc (one field, all V sites); kind 1: one half-lattice sweep of
 * the batched solver's stencil (V/2 output sites) for nrhs right-hand sides
 * in the given precision and link format, with the autotuned launch shape;
 * kind 2: one application of the solver's normal operator M^+ M (four such
 * sweeps), reported per application; kind 3: the same with the partial sums
 * of |M p|^2 that a CG iteration takes along (where the kernel fuses them).
 * Field contents are zero (timing does not depend on them). */
int cvcb_time_stencil(cvcb_lattice *lat, int kind, int precision, int link_recon, int nrhs,
                      int reps, double *ms_per_launch);

/* The normal operator M^+ M of the batched solver's inner iterations, as
 * the solver applies it: in[i] -> out[i] for i < nrhs (nrhs <= 96), CVC-layout
 * FP64 fields (host or device); the odd sites of in are the input (M is the
 * odd-site Schur complement A_oo - 1/4 H_oe A_ee^-1 H_eo of Q_phi_tbc's
 * operator, M(mu)^+ = g5 M(-mu) g5), even sites of out are set to zero.  The
 * fields go through the storage of `precision` (CVCB_PREC_*) with
 * link_recon reals per link; layout 1 selects the pair-tiled FP32 storage
 * (precision CVCB_PREC_SINGLE only), layout 0 the per-rhs one.  For checking
 * the reduced-precision operators against the FP64 one.  No counterpart in
 * the reference. */
int cvcb_sloppy_normal_op(cvcb_lattice *lat, int precision, int link_recon, int layout, int nrhs,
                          const double *const *in, double *const *out);

/* Tensor-core trial of the stencil's link product (u = W h for the 8 links
 * of every site of a half lattice and one block of 2 spins x 12 right-hand
 * sides, summed): variant 0 packed FP32x2 FMAs as the stencil does it,
 * 1 mma.sync TF32 with two sites per block-diagonal tile, 2 the same with
 * three TF32 products (FP32 accuracy).  Returns the average time of `reps`
 * launches and the largest deviation from variant 0 relative to the largest
 * component.  For the record of the trial; the stencil uses variant 0.  No
 * counterpart in the reference. */
int cvcb_time_link_product(cvcb_lattice *lat, int variant, int reps, double *ms,
                           double *rel_diff);

/* Launch shape the autotuner chose for the batched stencil for this lattice
 * volume, precision, link format and batch size: sites per thread block,
 * thread rows per block (each row a group of right-hand sides), right-hand
 * sides per thread, and the kernel variant (0: links per thread, 1: links
 * staged in shared memory for all rows, 2: two rhs per thread in packed
 * FP32x2 arithmetic, 3: pair-tiled fields, 4: pair-tiled fields with the
 * accumulator in tensor memory at 80 registers, 5: the same at 128 registers
 * with the next direction's loads in flight, 6: pair-tiled fields with the t
 * and x neighbours staged in shared memory by bulk copies); CVCB_ERR_STATE
 * before the first tuning. */
int cvcb_tuned_shape(cvcb_lattice *lat, int precision, int link_recon, int nrhs,
                     int *sites_per_block, int *rows_per_block, int *rhs_per_thread,
                     int *variant);

/* Instrumentation.  cvcb_profile(lat, 1) resets and starts timing the
 * batched solver's stencil: inside cvcb_solve, the stencil launches of one
 * iteration per chunk of iterations are bracketed by CUDA events on the
 * solver's stream (also inside its CUDA graph), and their device time and
 * algorithmic bytes (inputs, outputs and links read once; see
 * cvcb_time_stencil) are accumulated.  cvcb_counters reads the totals and
 * the number of kernels this context has launched (a graph launch counts
 * its kernel nodes). */
int cvcb_profile(cvcb_lattice *lat, int enable);
int cvcb_counters(cvcb_lattice *lat, long long *kernel_launches, long long *stencil_launches_timed,
                  double *stencil_ms, double *stencil_bytes);

/* ---------------------------------------------------------------------
 * Contractions
 * ------------------------------------------------------------------- */

/* Conserved-vector-current two-point function Pi_mu_nu(x) for one source
 * point, as cvc_exact2_xspace.c:577-861 computes it (including the -1/4
 * normalisation at :861).  fields[0..59]: "up" propagators, 12 spin-colour
 * columns (3*spin + colour) for each of the 5 source points y+mu (mu =
 * 0..3) and y (index 4), at fields[12*mu + sc]; fields[60..119]: "dn"
 * propagators in the same order.  source_site: lexicographic index of y.
 * conn: 32*V doubles (output); contact: 8 doubles (output, the contact term
 * printed at :697-716,837-855), may be NULL. */
int cvcb_cvc_contract(cvcb_lattice *lat, const double *const *fields, int source_site,
                      double *conn, double *contact);

/* Ward-identity divergence sum_mu [Pi_mu_nu(x) - Pi_mu_nu(x - mu)]
 * (cvc_exact2_xspace.c:928-1008); wi: 8*V doubles, wi[8*ix + 2*nu + re/im]. */
int cvcb_cvc_ward(cvcb_lattice *lat, const double *conn, double *wi);

/* Sequential source for the P -> gamma gamma three-point function
 * (p2gg_xspace.c:525-539): source = exp(i (1 - 2 pos) 2 pi p.x / L)
 * Gamma[gamma_id] prop(x) on timeslice t, zero elsewhere. */
int cvcb_p2gg_seq_source(cvcb_lattice *lat, double *source, const double *prop, int timeslice,
                         const int momentum[3], int gamma_id, int propagator_position);

/* ---------------------------------------------------------------------
 * Derivatives of Pi_mu_nu.  No counterpart in the reference.
 * ------------------------------------------------------------------- */

/* Forward pass: solves the 120 propagator columns of source point y
 * (up = Q(mu)^-1, dn = Q(-mu)^-1, point sources at y + mu-hat for mu =
 * 0..3 and at y, column order as cvcb_cvc_contract expects) with the
 * batched solver under `params`, and returns Pi_mu_nu (and the contact
 * term, may be NULL).  The columns are kept on the GPU for the calls below
 * when they need at most keep_bytes of device memory (120 * 192 * V bytes);
 * otherwise they are recomputed when needed. */
int cvcb_pi_forward(cvcb_lattice *lat, int source_site, const cvcb_solver_params *params,
                    double keep_bytes, double *conn, double *contact);

/* Tangent: dPi_mu_nu / d parameter for parameter 0 = mu (the bare twisted
 * mass g_mu) or 1 = kappa, at the state of the last forward pass (one extra
 * solve per column).  dconn: 32*V doubles, the layout of conn. */
int cvcb_pi_tangent(cvcb_lattice *lat, int parameter, double *dconn);

/* Backward (adjoint) pass for L = Re sum_{x,mu,nu} conj(w_munu(x))
 * Pi_munu(x), weights in the layout of conn (32*V doubles).  Returns
 * dL/dmu, dL/dkappa and, if dL_dU is not NULL, the gradient with respect to
 * the raw gauge links (72*V doubles, CVC gauge layout): for every link entry
 * U_ab the pair (dL/dRe U_ab, dL/dIm U_ab).  One adjoint solve per column
 * (Q(mu)^-dagger = g5 Q(-mu)^-1 g5). */
int cvcb_pi_backward(cvcb_lattice *lat, const double *weights, double *dL_dU, double *dL_dmu,
                     double *dL_dkappa);

/* Momentum-space Pi_mu_nu(q) (the step after the path in the reference's
 * momentum-space programs), with the conserved currents at their link
 * midpoints and the contact term subtracted:
 *   pimom_mu_nu(q) = e^{i q.y} e^{-i q_mu/2} e^{i q_nu/2} sum_x e^{-i q.x}
 *                    conn_mu_nu(x) - delta_mu_nu contact_nu,
 * q_mu = 2 pi k_mu / L_mu, output at pimom[2*(16*k + 4*mu + nu) + re/im] with
 * k = ((k_t*LX + k_x)*LY + k_y)*LZ + k_z; y = source_site (lexicographic);
 * contact (8 doubles, as from cvcb_cvc_contract) may be NULL (no
 * subtraction).  Then sum_mu 2 sin(q_mu/2) pimom_mu_nu(q) = 0, the Ward
 * identity of cvc_exact2_xspace.c:928-1008. */
int cvcb_pi_momentum(cvcb_lattice *lat, const double *conn, int source_site,
                     const double *contact, double *pimom);

/* Hopping-parameter expansion (Q_phi.c:536-781), B = (1 - i 2 kappa mu g5) /
 * (1 + (2 kappa mu)^2) as in mul_one_pm_imu_inv(+1), H = the hop sum of
 * Hopping.  The reference's side effects on phi are kept:
 *   cvcb_BHn: xi = (B H)^n phi; for n >= 2 phi becomes (B H)^(2 [n/2]) phi
 *   (Q_phi.c:753-781).  cvcb_BH, _BH3, _BH5, _BH7: n = 1, 3, 5, 7
 *   (Q_phi.c:598-751).  cvcb_BH2: phi = (B H)^2 phi, xi = B H phi
 *   (Q_phi.c:683-702).  cvcb_gamma5_BdagH4_gamma5: xi = g5 (B^+ H)^4 g5 phi,
 *   work = (B^+ H)^3 g5 phi, phi unchanged (Q_phi.c:536-570). */
int cvcb_BHn(cvcb_lattice *lat, double *xi, double *phi, int n);
int cvcb_BH(cvcb_lattice *lat, double *xi, double *phi);
int cvcb_BH2(cvcb_lattice *lat, double *xi, double *phi);
int cvcb_BH3(cvcb_lattice *lat, double *xi, double *phi);
int cvcb_BH5(cvcb_lattice *lat, double *xi, double *phi);
int cvcb_BH7(cvcb_lattice *lat, double *xi, double *phi);
int cvcb_gamma5_BdagH4_gamma5(cvcb_lattice *lat, double *xi, const double *phi, double *work);

/* Plaquette <Re tr U_munu>/(18 V) and link sum (cvc_utils.c:384-436). */
int cvcb_plaquette(cvcb_lattice *lat, double *plaq, double *linksum);

/* ---------------------------------------------------------------------
 * LIME / SciDAC / ILDG files (host memory, no GPU needed).  The reference
 * reads and writes these through c-lime / lemon; the lattice extents it
 * takes from globals are arguments here.  Fields are in CVC's layouts; every
 * call returns the SciDAC checksum (suma, sumb) of the binary record in
 * `checksum` (may be NULL).  Files are big-endian, 64- or 32-bit; readers
 * take the precision from the record length.
 * ------------------------------------------------------------------- */

/* CRC-32 (zlib polynomial) of len bytes continuing from crc, as DML_crc32
 * (DML_crc32.c). */
int cvcb_crc32(uint32_t crc, const void *buf, size_t len, uint32_t *out);

/* SciDAC checksum step (dml.c:22-50, DML_checksum_accum): sums[0] ^=
 * rotl(crc, rank % 29), sums[1] ^= rotl(crc, rank % 31), crc = CRC-32 of the
 * site's size bytes. */
int cvcb_dml_checksum_accum(uint32_t sums[2], uint64_t rank, const void *buf, size_t size);

/* Gauge field from the ildg-binary-data record of an ILDG file
 * (io.c:202-343 read_lime_gauge_field_doubleprec; 32-bit files as
 * read_lime_gauge_field_singleprec): gauge = 72*V doubles. */
int cvcb_read_lime_gauge_field_doubleprec(const char *filename, double *gauge, int T, int LX,
                                          int LY, int LZ, uint32_t checksum[2]);

/* ILDG gauge file: ildg-format, ildg-binary-data, scidac-checksum records
 * (gauge_io.c:198-340 write_lime_gauge_field); prec 64 or 32. */
int cvcb_write_lime_gauge_field(const char *filename, const double *gauge, int T, int LX, int LY,
                                int LZ, int prec, uint32_t checksum[2]);

/* Dirac field from the position-th scidac-binary-data record
 * (propagator_io.c:771-840 read_lime_spinor); s = 24*V doubles. */
int cvcb_read_lime_spinor(double *s, const char *filename, int position, int T, int LX, int LY,
                          int LZ, uint32_t checksum[2]);

/* Appends (append != 0) or writes a scidac-binary-data record and its
 * scidac-checksum (propagator_io.c:578-647 write_lime_spinor). */
int cvcb_write_lime_spinor(const double *s, const char *filename, int append, int prec, int T,
                           int LX, int LY, int LZ, uint32_t checksum[2]);

/* etmc-propagator-format record followed by write_lime_spinor
 * (propagator_io.c:125-132 write_propagator). */
int cvcb_write_propagator(const double *s, const char *filename, int prec, int T, int LX, int LY,
                          int LZ, uint32_t checksum[2]);

/* N-component contraction (N complex numbers per site, CVC site order; Pi
 * is N = 16): cvc_contraction-format, scidac-binary-data and scidac-checksum
 * records (contractions_io.c:56-137,338-420 write_lime_contraction, the
 * lemon variant; the reference's plain-LIME variant is a stub). */
int cvcb_write_lime_contraction(const double *s, const char *filename, int prec, int N,
                                const char *type, int gid, int sid, int T, int LX, int LY, int LZ,
                                uint32_t checksum[2]);

/* The position-th scidac-binary-data record as an N-component contraction
 * (contractions_io.c:140-235,420-480 read_lime_contraction). */
int cvcb_read_lime_contraction(double *s, const char *filename, int N, int position, int T, int LX,
                               int LY, int LZ, uint32_t checksum[2]);

#ifdef __cplusplus
}
#endif
#endif
