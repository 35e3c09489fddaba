// Momentum-space Pi_mu_nu(q) from the position-space conn of
// cvc_exact2_xspace.c:577-861 -- the step the reference's momentum-space
// programs take after the path.  With the conserved currents at their link
// midpoints (x + mu/2 for J_mu(x), y + nu/2 at the source) and the contact
// term c_nu (cvc_exact2_xspace.c:697-716,837-855) subtracted,
//   Pi_mu_nu(q) = e^{i q.y} e^{-i q_mu/2} e^{+i q_nu/2} sum_x e^{-i q.x} Pi_mu_nu(x)
//                 - delta_mu_nu c_nu,          q_mu = 2 pi k_mu / L_mu,
// the lattice Ward identity (cvc_exact2_xspace.c:928-1008) becomes exact
// transversality: sum_mu 2 sin(q_mu/2) Pi_mu_nu(q) = 0 for every q.
//
// The Fourier sum is four separable DFT passes (one per direction, O(L) per
// output, L <= a few hundred), each a gather along one axis of the
// [T][LX][LY][LZ][16] complex array with a twiddle table in global memory
// (cached); FP64 throughout.
#include <cmath>
#include <vector>

#include "cvcb_internal.h"

namespace cvcb {
namespace {

// out[a][k][b] = sum_x tw[(k x) mod L] in[a][x][b]
__global__ void k_dft_axis(const double2 *__restrict__ in, double2 *__restrict__ out,
                           const double2 *__restrict__ tw, long long A, int L, long long B) {
  const long long n = A * L * B;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long b = i % B;
    const long long r = i / B;
    const int k = (int)(r % L);
    const long long a = r / L;
    const double2 *src = in + a * L * B + b;
    double re = 0.0, im = 0.0;
    int kx = 0;  // (k x) mod L
    for (int x = 0; x < L; ++x) {
      const double2 w = __ldg(tw + kx), v = __ldg(src + (long long)x * B);
      re = fma(w.x, v.x, re);
      re = fma(-w.y, v.y, re);
      im = fma(w.x, v.y, im);
      im = fma(w.y, v.x, im);
      kx += k;
      if (kx >= L) kx -= L;
    }
    out[i] = make_double2(re, im);
  }
}

struct PhaseArgs {
  int T, LX, LY, LZ;
  int y[4];
  double contact[8];
  int subtract;
};

// midpoint phases, source shift and contact subtraction; f[k][16]
__global__ void k_pi_phases(double2 *__restrict__ f, PhaseArgs P, long long V) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < V;
       k += (long long)gridDim.x * blockDim.x) {
    long long r = k;
    const int kz = (int)(r % P.LZ);
    r /= P.LZ;
    const int ky = (int)(r % P.LY);
    r /= P.LY;
    const int kx = (int)(r % P.LX);
    const int kt = (int)(r / P.LX);
    // q_mu / pi = 2 k_mu / L_mu, taken modulo 2 to keep the arguments small
    const double q[4] = {2.0 * kt / P.T, 2.0 * kx / P.LX, 2.0 * ky / P.LY, 2.0 * kz / P.LZ};
    const double qy = q[0] * P.y[0] + q[1] * P.y[1] + q[2] * P.y[2] + q[3] * P.y[3];
    for (int mu = 0; mu < 4; ++mu)
      for (int nu = 0; nu < 4; ++nu) {
        double s, c;
        sincospi(fmod(qy - 0.5 * q[mu] + 0.5 * q[nu], 2.0), &s, &c);
        double2 &v = f[k * 16 + 4 * mu + nu];
        const double2 z = make_double2(c * v.x - s * v.y, c * v.y + s * v.x);
        v = z;
        if (P.subtract && mu == nu) {
          v.x -= P.contact[2 * nu];
          v.y -= P.contact[2 * nu + 1];
        }
      }
  }
}

}  // namespace
}  // namespace cvcb

using namespace cvcb;

extern "C" int cvcb_pi_momentum(cvcb_lattice *L, const double *conn, int source_site,
                                const double *contact, double *pimom) {
  if (!L || !conn || !pimom) return CVCB_ERR_NULL;
  const Geom &g = L->g;
  if (source_site < 0 || source_site >= g.V) {
    set_error("source site %d outside the lattice", source_site);
    return CVCB_ERR_ARG;
  }
  CVCB_CUDA(cudaSetDevice(L->device));
  const size_t bytes = (size_t)g.V * 16 * sizeof(double2);
  void *a, *b, *t;
  CVCB_TRY(ensure_buffer(L, SLOT_F0, bytes, &a));
  CVCB_TRY(ensure_buffer(L, SLOT_F1, bytes, &b));
  const int ext[4] = {g.T, g.LX, g.LY, g.LZ};
  const int lmax = std::max(std::max(g.T, g.LX), std::max(g.LY, g.LZ));
  CVCB_TRY(ensure_buffer(L, SLOT_F2, (size_t)4 * lmax * sizeof(double2), &t));
  double2 *buf[2] = {static_cast<double2 *>(a), static_cast<double2 *>(b)};
  double2 *tw = static_cast<double2 *>(t);
  CVCB_CUDA(cudaMemcpyAsync(buf[0], conn, bytes,
                            is_device_ptr(conn) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            L->stream));
  // twiddles e^{-2 pi i j / L} per direction, computed on the host in FP64
  std::vector<double2> htw((size_t)4 * lmax);
  for (int d = 0; d < 4; ++d)
    for (int j = 0; j < ext[d]; ++j) {
      const double ph = -2.0 * M_PI * j / ext[d];
      htw[(size_t)d * lmax + j] = make_double2(std::cos(ph), std::sin(ph));
    }
  CVCB_CUDA(cudaMemcpyAsync(tw, htw.data(), htw.size() * sizeof(double2), cudaMemcpyHostToDevice,
                            L->stream));
  long long A = 1, B = (long long)g.V * 16;
  int cur = 0;
  for (int d = 0; d < 4; ++d) {
    B /= ext[d];
    const long long n = A * ext[d] * B;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 32);
    k_dft_axis<<<blocks, 256, 0, L->stream>>>(buf[cur], buf[1 - cur], tw + (size_t)d * lmax, A,
                                              ext[d], B);
    CVCB_LAUNCHED(L);
    cur = 1 - cur;
    A *= ext[d];
  }
  PhaseArgs P{};
  P.T = g.T;
  P.LX = g.LX;
  P.LY = g.LY;
  P.LZ = g.LZ;
  int r = source_site;
  P.y[3] = r % g.LZ;
  r /= g.LZ;
  P.y[2] = r % g.LY;
  r /= g.LY;
  P.y[1] = r % g.LX;
  P.y[0] = r / g.LX;
  P.subtract = contact != nullptr;
  if (contact)
    for (int i = 0; i < 8; ++i) P.contact[i] = contact[i];
  const int blocks = (int)std::min<long long>((g.V + 255) / 256, 148LL * 32);
  k_pi_phases<<<blocks, 256, 0, L->stream>>>(buf[cur], P, g.V);
  CVCB_LAUNCHED(L);
  CVCB_CUDA(cudaMemcpyAsync(pimom, buf[cur], bytes,
                            is_device_ptr(pimom) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                            L->stream));
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  return CVCB_OK;
}
