// Reductions behind spinor_scalar_product_co/_re (invert_Qtm.c:28-84) and
// the C-ABI entry points of the operators.
#include <cmath>

#include "cvcb_internal.h"
#include "reduce.cuh"

namespace cvcb {

struct DotCo {
  const double2 *__restrict__ a;
  const double2 *__restrict__ b;
  __device__ void operator()(size_t k, double (&acc)[2]) const {
    const double2 x = __ldg(a + k), y = __ldg(b + k);
    acc[0] += x.x * y.x + x.y * y.y;  // Re conj(x) y
    acc[1] += x.x * y.y - x.y * y.x;  // Im conj(x) y
  }
};

int dot_co(cvcb_lattice *L, const double2 *a, const double2 *b, size_t n, double out[2]) {
  CVCB_TRY(launch_reduce<2>(L, DotCo{a, b}, StoreTotals<2>{L->red_result}, n));
  CVCB_CUDA(cudaMemcpyAsync(out, L->red_result, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                            L->stream));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  return CVCB_OK;
}

int dot_re(cvcb_lattice *L, const double2 *a, const double2 *b, size_t n, double *out) {
  double w[2];
  CVCB_TRY(dot_co(L, a, b, n, w));
  *out = w[0];
  return CVCB_OK;
}

}  // namespace cvcb

using namespace cvcb;

namespace {

int need_gauge(cvcb_lattice *L) {
  if (!L) return CVCB_ERR_NULL;
  if (!L->have_gauge) {
    set_error("no gauge field uploaded (cvcb_upload_gauge)");
    return CVCB_ERR_STATE;
  }
  return CVCB_OK;
}

// out = op(in) with the full-lattice kernel; in/out in CVC layout.
int apply_full(cvcb_lattice *L, double *xi, const double *phi, double a, double b, double c,
               bool g5out) {
  CVCB_TRY(need_gauge(L));
  if (!xi || !phi) return CVCB_ERR_NULL;
  CVCB_CUDA(cudaSetDevice(L->device));
  const size_t fb = (size_t)L->g.V * 12 * sizeof(double2);
  void *f0, *f1;
  CVCB_TRY(ensure_buffer(L, SLOT_F0, fb, &f0));
  CVCB_TRY(ensure_buffer(L, SLOT_F1, fb, &f1));
  CVCB_TRY(spinor_in(L, static_cast<double2 *>(f0), phi, L->g.V));
  CVCB_TRY(launch_tm_full(L, static_cast<double2 *>(f1), static_cast<const double2 *>(f0), a, b,
                          c, g5out, nullptr));
  CVCB_TRY(spinor_out(L, xi, static_cast<const double2 *>(f1), L->g.V));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  return CVCB_OK;
}

// Stage one CVC-layout field (host or device) to a device pointer usable by
// a reduction that ignores site order.
int stage_raw(cvcb_lattice *L, int slot, const double *src, int V, const double2 **out) {
  if (is_device_ptr(src)) {
    *out = reinterpret_cast<const double2 *>(src);
    return CVCB_OK;
  }
  void *st;
  CVCB_TRY(ensure_buffer(L, slot, (size_t)V * 24 * sizeof(double), &st));
  CVCB_CUDA(cudaMemcpyAsync(st, src, (size_t)V * 24 * sizeof(double), cudaMemcpyHostToDevice,
                            L->stream));
  *out = static_cast<const double2 *>(st);
  return CVCB_OK;
}

}  // namespace

extern "C" {

int cvcb_Q_phi_tbc(cvcb_lattice *L, double *xi, const double *phi) {
  if (!L) return CVCB_ERR_NULL;
  return apply_full(L, xi, phi, 0.5 / L->kappa, L->mu, -0.5, false);
}

int cvcb_Q_phi(cvcb_lattice *L, double *xi, const double *phi, double mutm) {
  if (!L) return CVCB_ERR_NULL;
  return apply_full(L, xi, phi, 0.5 / L->kappa, mutm, -0.5, false);
}

int cvcb_Qf5(cvcb_lattice *L, double *xi, const double *phi, double mutm) {
  if (!L) return CVCB_ERR_NULL;
  return apply_full(L, xi, phi, 0.5 / L->kappa, mutm, -0.5, true);
}

int cvcb_Hopping(cvcb_lattice *L, double *xi, const double *phi) {
  if (!L) return CVCB_ERR_NULL;
  return apply_full(L, xi, phi, 0.0, 0.0, -L->kappa, false);
}

int cvcb_g5_phi(cvcb_lattice *L, double *phi) {
  if (!L || !phi) return CVCB_ERR_NULL;
  CVCB_CUDA(cudaSetDevice(L->device));
  void *f0;
  CVCB_TRY(ensure_buffer(L, SLOT_F0, (size_t)L->g.V * 12 * sizeof(double2), &f0));
  CVCB_TRY(spinor_in(L, static_cast<double2 *>(f0), phi, L->g.V));
  CVCB_TRY(launch_g5(L, static_cast<double2 *>(f0), L->g.V));
  CVCB_TRY(spinor_out(L, phi, static_cast<const double2 *>(f0), L->g.V));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  return CVCB_OK;
}

int cvcb_mul_one_pm_imu_inv(cvcb_lattice *L, double *phi, double sign, int V) {
  if (!L || !phi) return CVCB_ERR_NULL;
  if (V < 0 || V > L->g.V) {
    set_error("V = %d outside [0, %d]", V, L->g.V);
    return CVCB_ERR_ARG;
  }
  if (V == 0) return CVCB_OK;
  CVCB_CUDA(cudaSetDevice(L->device));
  void *f0;
  CVCB_TRY(ensure_buffer(L, SLOT_F0, (size_t)L->g.V * 12 * sizeof(double2), &f0));
  CVCB_TRY(spinor_in(L, static_cast<double2 *>(f0), phi, V));
  CVCB_TRY(launch_one_pm_imu_inv(L, static_cast<double2 *>(f0), sign, V));
  CVCB_TRY(spinor_out(L, phi, static_cast<const double2 *>(f0), V));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  return CVCB_OK;
}

int cvcb_spinor_scalar_product_co(cvcb_lattice *L, double *w, const double *xi, const double *phi,
                                  int V) {
  if (!L || !w || !xi || !phi) return CVCB_ERR_NULL;
  if (V < 0 || V > L->g.V) {
    set_error("V = %d outside [0, %d]", V, L->g.V);
    return CVCB_ERR_ARG;
  }
  if (V == 0) {
    w[0] = w[1] = 0.0;
    return CVCB_OK;
  }
  CVCB_CUDA(cudaSetDevice(L->device));
  const double2 *a, *b;
  CVCB_TRY(stage_raw(L, SLOT_STAGE_A, xi, V, &a));
  CVCB_TRY(stage_raw(L, SLOT_STAGE_B, phi, V, &b));
  return dot_co(L, a, b, (size_t)V * 12, w);
}

int cvcb_spinor_scalar_product_re(cvcb_lattice *L, double *r, const double *xi, const double *phi,
                                  int V) {
  if (!r) return CVCB_ERR_NULL;
  double w[2];
  int rc = cvcb_spinor_scalar_product_co(L, w, xi, phi, V);
  if (rc < 0) return rc;
  *r = w[0];
  return CVCB_OK;
}

}  // extern "C"
