// Link-level drop-in for the reference's operator and solver objects.
//
// The reference is C compiled as C++ in namespace cvc, with its state in
// globals (global.h).  This file defines, with the reference's exact C++
// signatures (Q_phi.h, invert_Qtm.h), the functions of Q_phi.o and
// invert_Qtm.o that lie on the propagator path, and forwards them to the C
// ABI of libcvcb200.so.  A reference program linked against
// libcvcb200_cvc.so instead of those two objects runs them on the GPU; the
// reference's other objects (geometry, utilities) bind to these definitions
// unchanged.
//
// State: the globals below are the reference's own (declared here with the
// types global.h gives them; the program that links this library defines
// them).  One lattice context is created on first use on device
// g_gpu_device_number and recreated when the extents change.  Before every
// call the whole gauge field is hashed on the host (one pass over 72*VOLUME
// doubles, about 30 ms at 24^3x48), and it is uploaded again when
// g_gauge_field points elsewhere or its contents changed, so a program that
// edits the field in place never runs on stale links.
//
// Behaviour kept: argument meaning, field layouts, return values of the
// solvers (iterations, -2, -3; a broken-down BiCGStab, which the C ABI
// reports as CVCB_BREAKDOWN, returns -3 here as in the reference).  Fatal library errors print a message and
// exit(1), as the reference's EXIT() does.  The solvers print nothing.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/cvcb.h"

namespace cvc {
typedef struct {
  double re, im;
} complex;  // cvc_complex.h

extern int T, LX, LY, LZ, VOLUME;
extern double g_kappa, g_mu;
extern double BCangle[4];
extern double *g_gauge_field;
extern double solver_precision;
extern int niter_max;
extern int g_gpu_device_number;
}  // namespace cvc

namespace {

cvcb_lattice *g_ctx = nullptr;
int g_dims[4] = {0, 0, 0, 0};
const double *g_gauge_ptr = nullptr;
uint64_t g_gauge_hash = 0;
bool g_force_upload = false;

void fail(const char *where, int rc) {
  std::fprintf(stderr, "[cvc-b200] %s failed (%d): %s\n", where, rc, cvcb_last_error());
  std::exit(1);
}

// Hash of the field's bits: four independent multiply-xor lanes over the
// 64-bit words (word position enters through the lane and the order), so
// any change of any bit of any link changes it with probability 1 - 2^-64.
uint64_t hash_gauge() {
  const long n = 72L * cvc::VOLUME;
  const uint64_t *w = reinterpret_cast<const uint64_t *>(cvc::g_gauge_field);
  const uint64_t m = 0x9E3779B97F4A7C15ull;
  uint64_t h[4] = {1, 2, 3, 4};
  long i = 0;
  for (; i + 4 <= n; i += 4)
    for (int k = 0; k < 4; ++k) h[k] = (h[k] ^ w[i + k]) * m + (h[k] >> 29);
  for (; i < n; ++i) h[0] = (h[0] ^ w[i]) * m + (h[0] >> 29);
  return (h[0] * 3 + h[1]) * 5 + (h[2] * 7 + h[3]) * 11;
}

cvcb_lattice *ctx() {
  using namespace cvc;
  const int d[4] = {T, LX, LY, LZ};
  if (!g_ctx || std::memcmp(d, g_dims, sizeof d) != 0) {
    if (g_ctx) cvcb_lattice_destroy(g_ctx);
    g_ctx = nullptr;
    int rc = cvcb_lattice_create(&g_ctx, T, LX, LY, LZ, g_gpu_device_number);
    if (rc < 0) fail("cvcb_lattice_create", rc);
    std::memcpy(g_dims, d, sizeof d);
    g_gauge_ptr = nullptr;
  }
  int rc = cvcb_set_params(g_ctx, g_kappa, g_mu, BCangle);
  if (rc < 0) fail("cvcb_set_params", rc);
  if (!g_gauge_field) {
    std::fprintf(stderr, "[cvc-b200] g_gauge_field is not allocated\n");
    std::exit(1);
  }
  const uint64_t h = hash_gauge();
  if (g_force_upload || g_gauge_ptr != g_gauge_field || h != g_gauge_hash) {
    rc = cvcb_upload_gauge(g_ctx, g_gauge_field);
    if (rc < 0) fail("cvcb_upload_gauge", rc);
    g_gauge_ptr = g_gauge_field;
    g_gauge_hash = h;
    g_force_upload = false;
  }
  return g_ctx;
}

void check(const char *where, int rc) {
  if (rc < 0) fail(where, rc);
}

}  // namespace

// Forces the next call to upload the gauge field (the hash already detects
// every in-place change; kept for programs that call it).
extern "C" void cvcb_compat_gauge_changed(void) { g_force_upload = true; }

namespace cvc {

void Q_phi_tbc(double *xi, double *phi) { check("Q_phi_tbc", cvcb_Q_phi_tbc(ctx(), xi, phi)); }

void Hopping(double *xi, double *phi) { check("Hopping", cvcb_Hopping(ctx(), xi, phi)); }

void Qf5(double *xi, double *phi, double mutm) { check("Qf5", cvcb_Qf5(ctx(), xi, phi, mutm)); }

void Q_phi(double *xi, double *phi, const double mutm) {
  check("Q_phi", cvcb_Q_phi(ctx(), xi, phi, mutm));
}

void g5_phi(double *phi) { check("g5_phi", cvcb_g5_phi(ctx(), phi)); }

void mul_one_pm_imu_inv(double *phi, double sign, int V) {
  check("mul_one_pm_imu_inv", cvcb_mul_one_pm_imu_inv(ctx(), phi, sign, V));
}

void spinor_scalar_product_co(complex *w, double *xi, double *phi, int V) {
  double r[2];
  check("spinor_scalar_product_co", cvcb_spinor_scalar_product_co(ctx(), r, xi, phi, V));
  w->re = r[0];
  w->im = r[1];
}

void spinor_scalar_product_re(double *r, double *xi, double *phi, int V) {
  check("spinor_scalar_product_re", cvcb_spinor_scalar_product_re(ctx(), r, xi, phi, V));
}

// kwork: the reference's work fields g_spinor_field[kwork..] are not needed;
// the solver's work space lives on the GPU.
int invert_Qtm(double *xi, double *phi, int kwork) {
  (void)kwork;
  const int rc = cvcb_invert_Qtm(ctx(), xi, phi, solver_precision, niter_max, nullptr);
  if (rc == CVCB_BREAKDOWN) return CVCB_NO_CONVERGENCE;  // the reference's -3
  if (rc < 0 && rc != CVCB_ERR_NULL && rc != CVCB_NO_CONVERGENCE) fail("invert_Qtm", rc);
  return rc;
}

int invert_Qtm_her(double *xi, double *phi, int kwork) {
  (void)kwork;
  const int rc = cvcb_invert_Qtm_her(ctx(), xi, phi, solver_precision, niter_max, nullptr);
  if (rc == CVCB_BREAKDOWN) return CVCB_NO_CONVERGENCE;  // the reference's -3
  if (rc < 0 && rc != CVCB_ERR_NULL && rc != CVCB_NO_CONVERGENCE) fail("invert_Qtm_her", rc);
  return rc;
}

}  // namespace cvc
