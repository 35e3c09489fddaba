// Internal declarations of the B200 library (not part of the public ABI).
//
// Device data layout (all fields live in HBM in these forms):
//   site order  : even/odd.  Site with lexicographic index lex = ((t*LX+x)*LY
//                 +y)*LZ+z and parity p = (t+x+y+z)&1 sits at p*Vh + lex/2.
//                 With LZ even, lex/2 is unique inside a parity.
//   FP64 spinor : double2 s[12][V]; complex component k = 3*spin + colour
//                 of site j at s[k*V + j] (structure of arrays, so a warp
//                 reads 32 consecutive sites with one 512-byte transaction).
//   FP32 spinor : float4  s[6][stride]   (components 2k, 2k+1 per float4)
//   FP16 spinor : uint4   s[3][stride] (8 halves each) + float norm[stride]
//   FP64 links  : double2 U[4][9][V], boundary phase already multiplied in
//                 (the reference multiplies it per use, Q_phi.c:66).
//   FP32 links  : float4  U[4][3][V], rows 0 and 1 of the phased link
//                 e^{i theta} U; row 2 = e^{3 i theta} conj(row0 x row1) is
//                 rebuilt in registers.
//   FP16 links  : uint2   U[4][3][V], same 12 reals in half precision.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/cvcb.h"

namespace cvcb {

// ---- host helpers (host_geometry.cpp) ------------------------------------
void boundary_phases(int T, int LX, int LY, int LZ, const double bc[4], double ph[8]);
void gamma_tables(int perm[16][24], int sign[16][24]);
int geometry_tables(int T, int LX, int LY, int LZ, int *ipt, int *iup, int *idn, int *lexic2eo,
                    int *eo2lexic, int *iseven, int *isevent, int *lexic2eot, int *eot2lexic);
int ranlxd_fill(int level, int seed, double *r, long n);
int gauge_random(double *gauge, int T, int LX, int LY, int LZ, double eps, int seed);

// ---- errors ----------------------------------------------------------------
void set_error(const char *fmt, ...);
const char *last_error();

#define CVCB_CUDA(expr)                                                              \
  do {                                                                               \
    cudaError_t e_ = (expr);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      ::cvcb::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(e_)); \
      return CVCB_ERR_CUDA;                                                          \
    }                                                                                \
  } while (0)

// After a kernel launch: count it and surface launch errors.
#define CVCB_LAUNCHED(Lp)                \
  do {                                   \
    ++(Lp)->nlaunch;                     \
    CVCB_CUDA(cudaGetLastError());       \
  } while (0)

#define CVCB_TRY(expr)             \
  do {                             \
    int r_ = (expr);               \
    if (r_ < 0) return r_;         \
  } while (0)

// ---- division by an invariant integer --------------------------------------
// q = n / d as (umulhi(n, m) + n) >> s with s = ceil(log2 d) and
// m = floor(2^32 (2^s - d) / d) + 1 (Granlund and Montgomery, "Division by
// invariant integers using multiplication", PLDI 1994); exact for
// 0 <= n < 2^31, which covers every site index here.
struct FastDiv {
  unsigned d, m, s;
};

inline FastDiv make_fastdiv(unsigned d) {
  FastDiv f;
  f.d = d;
  f.s = 0;
  while ((1u << f.s) < d) ++f.s;
  f.m = (unsigned)((((unsigned long long)1 << 32) * (((unsigned long long)1 << f.s) - d)) / d + 1);
  return f;
}

__host__ __device__ inline unsigned fdiv(unsigned n, const FastDiv &f) {
#ifdef __CUDA_ARCH__
  const unsigned t = __umulhi(n, f.m);
#else
  const unsigned t = (unsigned)(((unsigned long long)n * f.m) >> 32);
#endif
  return (t + n) >> f.s;
}

// ---- geometry passed to kernels by value ----------------------------------
struct Geom {
  int T, LX, LY, LZ;
  int V, Vh;
  int s1;  // LZ             : lex step of +y
  int s2;  // LY*LZ          : lex step of +x
  int s3;  // LX*LY*LZ       : lex step of +t
  FastDiv dLX, dLY, dLZ;
};

// Lexicographic coordinates of the even/odd site (p, i).
struct SiteCoord {
  int t, x, y, z, lex;
};

__host__ __device__ inline SiteCoord site_coord(const Geom &g, int p, int i) {
  SiteCoord c;
  const unsigned m = 2u * (unsigned)i;
  const unsigned r0 = fdiv(m, g.dLZ);
  const int z0 = (int)(m - r0 * (unsigned)g.LZ);
  const unsigned r1 = fdiv(r0, g.dLY);
  c.y = (int)(r0 - r1 * (unsigned)g.LY);
  const unsigned r2 = fdiv(r1, g.dLX);
  c.x = (int)(r1 - r2 * (unsigned)g.LX);
  c.t = (int)r2;
  c.z = z0 + ((p + c.t + c.x + c.y) & 1);
  c.lex = (int)m - z0 + c.z;
  return c;
}

// Neighbour lexicographic index in direction mu (0..3 = t,x,y,z), +1 or -1.
__host__ __device__ inline int nb_lex(const Geom &g, const SiteCoord &c, int mu, int dir) {
  switch (mu) {
    case 0:
      if (dir > 0) return c.t == g.T - 1 ? c.lex - (g.T - 1) * g.s3 : c.lex + g.s3;
      return c.t == 0 ? c.lex + (g.T - 1) * g.s3 : c.lex - g.s3;
    case 1:
      if (dir > 0) return c.x == g.LX - 1 ? c.lex - (g.LX - 1) * g.s2 : c.lex + g.s2;
      return c.x == 0 ? c.lex + (g.LX - 1) * g.s2 : c.lex - g.s2;
    case 2:
      if (dir > 0) return c.y == g.LY - 1 ? c.lex - (g.LY - 1) * g.s1 : c.lex + g.s1;
      return c.y == 0 ? c.lex + (g.LY - 1) * g.s1 : c.lex - g.s1;
    default:
      if (dir > 0) return c.z == g.LZ - 1 ? c.lex - (g.LZ - 1) : c.lex + 1;
      return c.z == 0 ? c.lex + (g.LZ - 1) : c.lex - 1;
  }
}

__host__ __device__ inline int lex_parity(const Geom &g, int lex) {
  const int z = lex % g.LZ;
  int r = lex / g.LZ;
  const int y = r % g.LY;
  r /= g.LY;
  const int x = r % g.LX;
  const int t = r / g.LX;
  return (t + x + y + z) & 1;
}

__host__ __device__ inline int lex_to_eo(const Geom &g, int lex) {
  return lex_parity(g, lex) * g.Vh + (lex >> 1);
}

// ---- device-side solver control block ------------------------------------
// Scalars of the Krylov recursions live on the device so that an iteration
// needs no host round trip; kernels read them and the last block of each
// reduction writes them.
struct SolverScalars {
  double2 rho, alpha, omega, beta, w;
  double normb, norm, u, prec;
  int done;       // 1: converged, 2: breakdown (non-finite scalar)
  int niter;      // iteration at which done was set
  int iter;       // iterations started
  int pad;
};

// ---- the context -----------------------------------------------------------
struct Buffer {
  void *ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace cvcb

struct cvcb_lattice {
  cvcb::Geom g;
  int device = 0;
  double kappa = 0.1, mu = 0.0;
  double bc[4] = {1, 0, 0, 0};
  double phase[8] = {0};
  cudaStream_t stream = nullptr;
  // second stream and events of the host<->device pipeline of cvcb_solve
  // (created on first use)
  cudaStream_t copy_stream = nullptr, copy_stream_out = nullptr;
  cudaEvent_t pipe_ev[6] = {};
  // mapped pinned mailbox for the solver's per-rhs control values (host and
  // device addresses of the same memory), created on first use
  double *mbox_host = nullptr, *mbox_dev = nullptr;
  bool have_gauge = false;
  double unitarity = -1.0;
  std::vector<double> gauge_host;  // raw CVC-layout copy (for re-phasing)

  // device gauge forms
  double2 *U64 = nullptr;   // [4][9][V], phased
  float4 *U32c = nullptr;   // [4][3][V], raw rows 0,1
  float2 *U32f = nullptr;   // [4][9][V], phased (18-real single)
  uint2 *U16c = nullptr;    // [4][3][V], raw rows 0,1 in half
  // the same single-precision forms tiled by 32 even/odd link indices (for
  // the pair-tiled stencil): [V/32][4][9][32] and [V/32][4][3][32]
  float2 *UT32f = nullptr;
  float4 *UT32c = nullptr;

  // reduction scratch: per-block partials, a completion counter, results
  double *partials = nullptr;  // [kMaxRedBlocks * 4]
  unsigned *red_counter = nullptr;
  double *red_result = nullptr;  // [8]
  cvcb::SolverScalars *scal = nullptr;

  // named device buffers, grown on demand
  std::vector<cvcb::Buffer> bufs;

  // instrumentation: kernels launched by this context (graph launches count
  // their kernel nodes), and CUDA-event timing of the solver's stencil
  long long nlaunch = 0;
  bool prof = false;
  long long prof_launches = 0;
  double prof_ms = 0.0, prof_bytes = 0.0;
};

namespace cvcb {

constexpr int kMaxRedBlocks = 1184;  // 8 x 148 SMs

// lattice.cu
int ensure_buffer(cvcb_lattice *L, int slot, size_t bytes, void **out);
bool is_device_ptr(const void *p);
// Copy a CVC-layout FP64 spinor (host or device) into device layout `dst`.
int spinor_in(cvcb_lattice *L, double2 *dst, const double *src, int nsites_aos);
// Copy device-layout `src` into a CVC-layout FP64 spinor (host or device).
int spinor_out(cvcb_lattice *L, double *dst, const double2 *src, int nsites_aos);
// Slots used by spinor_in/out staging
enum BufSlot {
  SLOT_STAGE_A = 0,
  SLOT_STAGE_B,
  SLOT_F0,
  SLOT_F1,
  SLOT_F2,
  SLOT_F3,
  SLOT_F4,
  SLOT_F5,
  SLOT_F6,
  SLOT_F7,
  SLOT_F8,
  SLOT_F9,
  SLOT_CONN,
  SLOT_PROPS,
  SLOT_MIX0,
  // double-buffered raw-layout staging of the solve pipeline (host fields)
  SLOT_PIPE_IN0 = 56,
  SLOT_PIPE_IN1,
  SLOT_PIPE_OUT0,
  SLOT_PIPE_OUT1,
  SLOT_NUM = 64
};

// dslash.cu: full-lattice FP64 twisted-mass operator, device layout.
//   out = a*in + i*b*g5*in + c*H in   (then g5 applied to out if g5out)
// H in = sum_mu [(1-g_mu) U_mu(x) in(x+mu) + (1+g_mu) U_mu(x-mu)^+ in(x-mu)]
int launch_tm_full(cvcb_lattice *L, double2 *out, const double2 *in, double a, double b, double c,
                   bool g5out, const int *done_flag);
int launch_g5(cvcb_lattice *L, double2 *f, int nsites);
int launch_one_pm_imu_inv(cvcb_lattice *L, double2 *f, double sign, int nsites);

// blas.cu
int dot_co(cvcb_lattice *L, const double2 *a, const double2 *b, size_t n, double out[2]);
int dot_re(cvcb_lattice *L, const double2 *a, const double2 *b, size_t n, double *out);

// solver_fp64.cu
int invert_bicgstab(cvcb_lattice *L, bool her, double *xi, const double *phi, double prec,
                    int niter_max, double *true_res2);

// contract.cu
int cvc_contract(cvcb_lattice *L, const double *const *fields, int source_site, double *conn,
                 double *contact);
int cvc_ward(cvcb_lattice *L, const double *conn, double *wi);
int p2gg_seq_source(cvcb_lattice *L, double *source, const double *prop, int t, const int mom[3],
                    int gamma_id, int pos);
int plaquette(cvcb_lattice *L, double *plaq, double *linksum);

// adjoint.cu
int pi_forward(cvcb_lattice *L, int src, const cvcb_solver_params *P, double keep_bytes,
               double *conn, double *contact);
int pi_tangent(cvcb_lattice *L, int param, double *dconn);
int pi_backward(cvcb_lattice *L, const double *wts, double *dLdU, double *dLdmu, double *dLdkappa);

// solver_mixed.cu
int time_stencil(cvcb_lattice *L, int kind, int prec, int recon, int nrhs, int reps, double *ms);
int sloppy_normal_op(cvcb_lattice *L, int prec, int recon, int layout, int n,
                     const double *const *in, double *const *out);
int solve_batched(cvcb_lattice *L, double *const *x, const double *const *b, int nrhs,
                  const cvcb_solver_params *p, cvcb_solver_stats *st);

}  // namespace cvcb
