// Hopping-parameter-expansion helpers of Q_phi.c:536-781 on the GPU, built
// from the Hopping kernel (a = b = 0, c = -kappa) and the site-diagonal
// B(sign) = (1 - i sign 2 kappa mu g5) / (1 + (2 kappa mu)^2) of
// mul_one_pm_imu_inv.  B H is one "BH step".  The reference's argument
// semantics are kept, including the fields it overwrites on the way:
//   BHn(xi, phi, n)  xi = (B H)^n phi; for n >= 2 phi ends as (B H)^(2 [n/2]) phi
//                    and for even n xi is a copy of it (Q_phi.c:753-781)
//   BH, BH3, BH5, BH7 = BHn with n = 1, 3, 5, 7 (Q_phi.c:598-751)
//   BH2(xi, phi)     phi = (B H)^2 phi, xi = B H phi (Q_phi.c:683-702)
//   gamma5_BdagH4_gamma5(xi, phi, work)  xi = g5 (B^+ H)^4 g5 phi, B^+ = B(-1);
//                    work ends as (B^+ H)^3 g5 phi; phi unchanged (Q_phi.c:536-570)
#include "cvcb_internal.h"

using namespace cvcb;

namespace {

int prepare(cvcb_lattice *L, double2 **f0, double2 **f1) {
  if (!L) return CVCB_ERR_NULL;
  if (!L->have_gauge) {
    set_error("no gauge field uploaded (cvcb_upload_gauge)");
    return CVCB_ERR_STATE;
  }
  CVCB_CUDA(cudaSetDevice(L->device));
  const size_t fb = (size_t)L->g.V * 12 * sizeof(double2);
  void *a, *b;
  CVCB_TRY(ensure_buffer(L, SLOT_F0, fb, &a));
  CVCB_TRY(ensure_buffer(L, SLOT_F1, fb, &b));
  *f0 = static_cast<double2 *>(a);
  *f1 = static_cast<double2 *>(b);
  return CVCB_OK;
}

// dst = B(sign) H src
int bh_step(cvcb_lattice *L, double2 *dst, const double2 *src, double sign) {
  CVCB_TRY(launch_tm_full(L, dst, src, 0.0, 0.0, -L->kappa, false, nullptr));
  return launch_one_pm_imu_inv(L, dst, sign, L->g.V);
}

int finish(cvcb_lattice *L) {
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  return CVCB_OK;
}

}  // namespace

extern "C" {

int cvcb_BHn(cvcb_lattice *L, double *xi, double *phi, int n) {
  double2 *f0, *f1;
  CVCB_TRY(prepare(L, &f0, &f1));
  if (!xi || !phi) return CVCB_ERR_NULL;
  if (n < 0) {
    set_error("BHn: n = %d < 0", n);
    return CVCB_ERR_ARG;
  }
  const int V = L->g.V;
  CVCB_TRY(spinor_in(L, f0, phi, V));
  for (int i = 0; i < n / 2; ++i) {
    CVCB_TRY(bh_step(L, f1, f0, +1.0));
    CVCB_TRY(bh_step(L, f0, f1, +1.0));
  }
  if (n % 2) {
    CVCB_TRY(bh_step(L, f1, f0, +1.0));
    CVCB_TRY(spinor_out(L, xi, f1, V));
  } else {
    CVCB_TRY(spinor_out(L, xi, f0, V));
  }
  if (n >= 2) CVCB_TRY(spinor_out(L, phi, f0, V));
  return finish(L);
}

int cvcb_BH(cvcb_lattice *L, double *xi, double *phi) { return cvcb_BHn(L, xi, phi, 1); }
int cvcb_BH3(cvcb_lattice *L, double *xi, double *phi) { return cvcb_BHn(L, xi, phi, 3); }
int cvcb_BH5(cvcb_lattice *L, double *xi, double *phi) { return cvcb_BHn(L, xi, phi, 5); }
int cvcb_BH7(cvcb_lattice *L, double *xi, double *phi) { return cvcb_BHn(L, xi, phi, 7); }

int cvcb_BH2(cvcb_lattice *L, double *xi, double *phi) {
  double2 *f0, *f1;
  CVCB_TRY(prepare(L, &f0, &f1));
  if (!xi || !phi) return CVCB_ERR_NULL;
  const int V = L->g.V;
  CVCB_TRY(spinor_in(L, f0, phi, V));
  CVCB_TRY(bh_step(L, f1, f0, +1.0));
  CVCB_TRY(bh_step(L, f0, f1, +1.0));
  CVCB_TRY(spinor_out(L, xi, f1, V));
  CVCB_TRY(spinor_out(L, phi, f0, V));
  return finish(L);
}

int cvcb_gamma5_BdagH4_gamma5(cvcb_lattice *L, double *xi, const double *phi, double *work) {
  double2 *f0, *f1;
  CVCB_TRY(prepare(L, &f0, &f1));
  if (!xi || !phi || !work) return CVCB_ERR_NULL;
  const int V = L->g.V;
  CVCB_TRY(spinor_in(L, f0, phi, V));
  CVCB_TRY(launch_g5(L, f0, V));
  for (int i = 0; i < 2; ++i) {
    CVCB_TRY(bh_step(L, f1, f0, -1.0));
    CVCB_TRY(bh_step(L, f0, f1, -1.0));
  }
  CVCB_TRY(launch_g5(L, f0, V));
  CVCB_TRY(spinor_out(L, xi, f0, V));
  CVCB_TRY(spinor_out(L, work, f1, V));
  return finish(L);
}

}  // extern "C"
