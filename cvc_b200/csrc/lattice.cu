// Lattice context, parameters, gauge-field upload and the layout transforms
// between CVC's site-major fields and the device's even/odd structure-of-
// arrays layout.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "cvcb_internal.h"

namespace cvcb {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}
const char *last_error() { return g_err; }

bool is_device_ptr(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int ensure_buffer(cvcb_lattice *L, int slot, size_t bytes, void **out) {
  if ((int)L->bufs.size() <= slot) L->bufs.resize(slot + 1);
  Buffer &b = L->bufs[slot];
  if (b.bytes < bytes) {
    if (b.ptr) CVCB_CUDA(cudaFree(b.ptr));
    b.ptr = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMalloc(&b.ptr, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error("cudaMalloc of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
      return CVCB_ERR_NOMEM;
    }
    b.bytes = bytes;
  }
  *out = b.ptr;
  return CVCB_OK;
}

// ---------------------------------------------------------------------------
// layout transforms, tiled through shared memory: a block takes kTile
// consecutive lexicographic sites, whose CVC-layout data (12 complex numbers
// each) is one contiguous chunk -- read or written with consecutive threads on
// consecutive addresses -- and moves them to or from the 12 component arrays
// of the even/odd layout, where consecutive threads touch consecutive sites of
// one parity.
// ---------------------------------------------------------------------------
constexpr int kTile = 64;
constexpr int kTilePad = 13;  // row pitch of the tile (12 + 1 against bank conflicts)

// all V sites of dst are written: sites lex >= nsites become zero
__global__ void __launch_bounds__(128) k_spinor_aos_to_eo(double2 *__restrict__ dst,
                                                         const double2 *__restrict__ src, Geom g,
                                                         int nsites) {
  __shared__ double2 t[kTile * kTilePad];
  const int base = blockIdx.x * kTile;
  const int nloc = min(kTile, g.V - base);
  for (int q = threadIdx.x; q < nloc * 12; q += blockDim.x) {
    const int s = q / 12, k = q - 12 * s;
    t[s * kTilePad + k] = base + s < nsites ? src[(size_t)base * 12 + q] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nloc * 12; q += blockDim.x) {
    const int k = q / nloc, s = q - k * nloc;
    dst[(size_t)k * g.V + lex_to_eo(g, base + s)] = t[s * kTilePad + k];
  }
}

// sites lex < nsites of dst are written
__global__ void __launch_bounds__(128) k_spinor_eo_to_aos(double2 *__restrict__ dst,
                                                         const double2 *__restrict__ src, Geom g,
                                                         int nsites) {
  __shared__ double2 t[kTile * kTilePad];
  const int base = blockIdx.x * kTile;
  const int nloc = min(kTile, nsites - base);
  if (nloc <= 0) return;
  for (int q = threadIdx.x; q < nloc * 12; q += blockDim.x) {
    const int k = q / nloc, s = q - k * nloc;
    t[s * kTilePad + k] = src[(size_t)k * g.V + lex_to_eo(g, base + s)];
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nloc * 12; q += blockDim.x) {
    const int s = q / 12, k = q - 12 * s;
    dst[(size_t)base * 12 + q] = t[s * kTilePad + k];
  }
}

int spinor_in(cvcb_lattice *L, double2 *dst, const double *src, int nsites) {
  const Geom &g = L->g;
  const double2 *dsrc;
  if (is_device_ptr(src)) {
    dsrc = reinterpret_cast<const double2 *>(src);
  } else {
    void *st;
    CVCB_TRY(ensure_buffer(L, SLOT_STAGE_A, (size_t)g.V * 24 * sizeof(double), &st));
    CVCB_CUDA(cudaMemcpyAsync(st, src, (size_t)nsites * 24 * sizeof(double),
                              cudaMemcpyHostToDevice, L->stream));
    dsrc = static_cast<const double2 *>(st);
  }
  k_spinor_aos_to_eo<<<(g.V + kTile - 1) / kTile, 128, 0, L->stream>>>(dst, dsrc, g, nsites);
  CVCB_LAUNCHED(L);
  return CVCB_OK;
}

int spinor_out(cvcb_lattice *L, double *dst, const double2 *src, int nsites) {
  const Geom &g = L->g;
  if (is_device_ptr(dst)) {
    k_spinor_eo_to_aos<<<(g.V + kTile - 1) / kTile, 128, 0, L->stream>>>(
        reinterpret_cast<double2 *>(dst), src, g, nsites);
    CVCB_LAUNCHED(L);
    return CVCB_OK;
  }
  void *st;
  CVCB_TRY(ensure_buffer(L, SLOT_STAGE_B, (size_t)g.V * 24 * sizeof(double), &st));
  k_spinor_eo_to_aos<<<(g.V + kTile - 1) / kTile, 128, 0, L->stream>>>(static_cast<double2 *>(st), src,
                                                                  g, nsites);
  CVCB_LAUNCHED(L);
  CVCB_CUDA(cudaMemcpyAsync(dst, st, (size_t)nsites * 24 * sizeof(double),
                            cudaMemcpyDeviceToHost, L->stream));
  return CVCB_OK;
}

// ---------------------------------------------------------------------------
// gauge field: raw CVC layout -> the device forms
// ---------------------------------------------------------------------------
__device__ inline double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void k_gauge_forms(const double2 *__restrict__ raw, Geom g, double4 ph01, double4 ph23,
                              double2 *__restrict__ U64, float4 *__restrict__ U32c,
                              float2 *__restrict__ U32f, uint2 *__restrict__ U16c,
                              float2 *__restrict__ UT32f, float4 *__restrict__ UT32c) {
  const int lex = blockIdx.x * blockDim.x + threadIdx.x;
  if (lex >= g.V) return;
  const int eo = lex_to_eo(g, lex);
  const double2 ph[4] = {make_double2(ph01.x, ph01.y), make_double2(ph01.z, ph01.w),
                         make_double2(ph23.x, ph23.y), make_double2(ph23.z, ph23.w)};
  for (int mu = 0; mu < 4; ++mu) {
    double2 u[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) u[k] = raw[((size_t)lex * 4 + mu) * 9 + k];
    double2 w[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      // (re*pr - im*pi, re*pi + im*pr): the rounding of _cm_eq_cm_ti_co
      w[k] = cmul(u[k], ph[mu]);
      U64[((size_t)mu * 9 + k) * g.V + eo] = w[k];
      U32f[((size_t)mu * 9 + k) * g.V + eo] = make_float2((float)w[k].x, (float)w[k].y);
      // tiled by 32 even/odd indices: [eo / 32][mu][k][eo % 32]
      UT32f[(((size_t)(eo >> 5) * 4 + mu) * 9 + k) * 32 + (eo & 31)] =
          make_float2((float)w[k].x, (float)w[k].y);
    }
    // 12-real forms: rows 0 and 1 of the phased link
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double2 a = w[2 * q], b = w[2 * q + 1];
      U32c[((size_t)mu * 3 + q) * g.V + eo] =
          make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
      UT32c[(((size_t)(eo >> 5) * 4 + mu) * 3 + q) * 32 + (eo & 31)] =
          make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
      __half2 h0 = __floats2half2_rn((float)a.x, (float)a.y);
      __half2 h1 = __floats2half2_rn((float)b.x, (float)b.y);
      uint2 w;
      w.x = *reinterpret_cast<unsigned *>(&h0);
      w.y = *reinterpret_cast<unsigned *>(&h1);
      U16c[((size_t)mu * 3 + q) * g.V + eo] = w;
    }
  }
}

static int build_gauge_forms(cvcb_lattice *L) {
  const Geom &g = L->g;
  const size_t V = g.V;
  if (!L->U64) {
    CVCB_CUDA(cudaMalloc(&L->U64, V * 36 * sizeof(double2)));
    CVCB_CUDA(cudaMalloc(&L->U32c, V * 12 * sizeof(float4)));
    CVCB_CUDA(cudaMalloc(&L->U32f, V * 36 * sizeof(float2)));
    CVCB_CUDA(cudaMalloc(&L->U16c, V * 12 * sizeof(uint2)));
    const size_t tiles = (V + 31) / 32;
    CVCB_CUDA(cudaMalloc(&L->UT32f, tiles * 32 * 36 * sizeof(float2)));
    CVCB_CUDA(cudaMalloc(&L->UT32c, tiles * 32 * 12 * sizeof(float4)));
  }
  void *raw;
  CVCB_TRY(ensure_buffer(L, SLOT_STAGE_A, V * 72 * sizeof(double), &raw));
  CVCB_CUDA(cudaMemcpyAsync(raw, L->gauge_host.data(), V * 72 * sizeof(double),
                            cudaMemcpyHostToDevice, L->stream));
  const double *ph = L->phase;
  k_gauge_forms<<<(g.V + 127) / 128, 128, 0, L->stream>>>(
      static_cast<const double2 *>(raw), g, make_double4(ph[0], ph[1], ph[2], ph[3]),
      make_double4(ph[4], ph[5], ph[6], ph[7]), L->U64, L->U32c, L->U32f, L->U16c, L->UT32f,
      L->UT32c);
  CVCB_LAUNCHED(L);
  CVCB_CUDA(cudaStreamSynchronize(L->stream));
  return CVCB_OK;
}

// Largest deviation from SU(3) over all links (host, once per upload).
static double unitarity_deviation(const std::vector<double> &G, size_t nlinks) {
  double worst = 0.0;
  for (size_t l = 0; l < nlinks; ++l) {
    const double *u = G.data() + 18 * l;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double re = 0, im = 0;  // (U U^dagger)_ij
        for (int k = 0; k < 3; ++k) {
          const double ar = u[2 * (3 * i + k)], ai = u[2 * (3 * i + k) + 1];
          const double br = u[2 * (3 * j + k)], bi = -u[2 * (3 * j + k) + 1];
          re += ar * br - ai * bi;
          im += ar * bi + ai * br;
        }
        if (i == j) re -= 1.0;
        worst = std::fmax(worst, std::fmax(std::fabs(re), std::fabs(im)));
      }
    // det U by the rule of Sarrus
    auto c = [&](int i, int j, int part) { return u[2 * (3 * i + j) + part]; };
    double dr = 0, di = 0;
    const int P[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {0, 2, 1}, {1, 0, 2}, {2, 1, 0}};
    for (int s = 0; s < 6; ++s) {
      double pr = 1, pi = 0;
      for (int i = 0; i < 3; ++i) {
        const double xr = c(i, P[s][i], 0), xi = c(i, P[s][i], 1);
        const double nr = pr * xr - pi * xi, ni = pr * xi + pi * xr;
        pr = nr;
        pi = ni;
      }
      const double sg = s < 3 ? 1.0 : -1.0;
      dr += sg * pr;
      di += sg * pi;
    }
    worst = std::fmax(worst, std::hypot(dr - 1.0, di));
  }
  return worst;
}

}  // namespace cvcb

using namespace cvcb;

extern "C" {

const char *cvcb_last_error(void) { return cvcb::last_error(); }
const char *cvcb_version(void) { return "cvc-b200 0.1 (sm_100a)"; }

int cvcb_lattice_create(cvcb_lattice **out, int T, int LX, int LY, int LZ, int device) {
  if (!out) return CVCB_ERR_NULL;
  *out = nullptr;
  if (T <= 0 || LX <= 0 || LY <= 0 || LZ <= 0 || (T | LX | LY | LZ) & 1) {
    set_error("lattice extents must be positive and even (got %d %d %d %d)", T, LX, LY, LZ);
    return CVCB_ERR_ARG;
  }
  const long long V = (long long)T * LX * LY * LZ;
  if (V > (1LL << 28)) {
    set_error("lattice volume %lld too large", V);
    return CVCB_ERR_ARG;
  }
  int ndev = 0;
  CVCB_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) {
    set_error("device %d not available (%d devices)", device, ndev);
    return CVCB_ERR_ARG;
  }
  CVCB_CUDA(cudaSetDevice(device));
  cvcb_lattice *L = new cvcb_lattice();
  L->device = device;
  L->g.T = T; L->g.LX = LX; L->g.LY = LY; L->g.LZ = LZ;
  L->g.V = (int)V;
  L->g.Vh = (int)(V / 2);
  L->g.s1 = LZ;
  L->g.s2 = LY * LZ;
  L->g.s3 = LX * LY * LZ;
  L->g.dLX = make_fastdiv(LX);
  L->g.dLY = make_fastdiv(LY);
  L->g.dLZ = make_fastdiv(LZ);
  boundary_phases(T, LX, LY, LZ, L->bc, L->phase);
  cudaError_t e = cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&L->partials, kMaxRedBlocks * 4 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&L->red_counter, 16 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(L->red_counter, 0, 16 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc(&L->red_result, 8 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&L->scal, sizeof(SolverScalars));
  if (e != cudaSuccess) {
    set_error("context set-up failed: %s", cudaGetErrorString(e));
    cvcb_lattice_destroy(L);
    return CVCB_ERR_CUDA;
  }
  *out = L;
  return CVCB_OK;
}

int cvcb_lattice_destroy(cvcb_lattice *L) {
  if (!L) return CVCB_OK;
  cudaSetDevice(L->device);
  if (L->stream) cudaStreamSynchronize(L->stream);
  for (auto &b : L->bufs)
    if (b.ptr) cudaFree(b.ptr);
  cudaFree(L->U64);
  cudaFree(L->U32c);
  cudaFree(L->U32f);
  cudaFree(L->U16c);
  cudaFree(L->UT32f);
  cudaFree(L->UT32c);
  cudaFree(L->partials);
  cudaFree(L->red_counter);
  cudaFree(L->red_result);
  cudaFree(L->scal);
  for (cudaStream_t cs : {L->copy_stream, L->copy_stream_out})
    if (cs) {
      cudaStreamSynchronize(cs);
      cudaStreamDestroy(cs);
    }
  for (cudaEvent_t e : L->pipe_ev)
    if (e) cudaEventDestroy(e);
  if (L->mbox_host) cudaFreeHost(L->mbox_host);
  if (L->stream) cudaStreamDestroy(L->stream);
  delete L;
  return CVCB_OK;
}

int cvcb_set_params(cvcb_lattice *L, double kappa, double mu, const double bc_angle[4]) {
  if (!L) return CVCB_ERR_NULL;
  if (!(kappa > 0) || !std::isfinite(kappa) || !std::isfinite(mu)) {
    set_error("kappa must be positive and finite, mu finite");
    return CVCB_ERR_ARG;
  }
  CVCB_CUDA(cudaSetDevice(L->device));
  L->kappa = kappa;
  L->mu = mu;
  bool phase_changed = false;
  if (bc_angle) {
    for (int i = 0; i < 4; ++i) {
      if (L->bc[i] != bc_angle[i]) phase_changed = true;
      L->bc[i] = bc_angle[i];
    }
  }
  boundary_phases(L->g.T, L->g.LX, L->g.LY, L->g.LZ, L->bc, L->phase);
  if (phase_changed && L->have_gauge) return build_gauge_forms(L);
  return CVCB_OK;
}

int cvcb_upload_gauge(cvcb_lattice *L, const double *gauge) {
  if (!L || !gauge) return CVCB_ERR_NULL;
  CVCB_CUDA(cudaSetDevice(L->device));
  const size_t n = (size_t)L->g.V * 72;
  L->gauge_host.resize(n);
  if (is_device_ptr(gauge)) {
    CVCB_CUDA(cudaMemcpy(L->gauge_host.data(), gauge, n * sizeof(double), cudaMemcpyDeviceToHost));
  } else {
    std::memcpy(L->gauge_host.data(), gauge, n * sizeof(double));
  }
  L->unitarity = unitarity_deviation(L->gauge_host, (size_t)L->g.V * 4);
  CVCB_TRY(build_gauge_forms(L));
  L->have_gauge = true;
  return CVCB_OK;
}

int cvcb_gauge_unitarity(cvcb_lattice *L, double *dev) {
  if (!L || !dev) return CVCB_ERR_NULL;
  if (!L->have_gauge) {
    set_error("no gauge field uploaded");
    return CVCB_ERR_STATE;
  }
  *dev = L->unitarity;
  return CVCB_OK;
}

int cvcb_geometry_tables(int T, int LX, int LY, int LZ, int *ipt, int *iup, int *idn,
                         int *lexic2eo, int *eo2lexic, int *iseven, int *isevent, int *lexic2eot,
                         int *eot2lexic) {
  return geometry_tables(T, LX, LY, LZ, ipt, iup, idn, lexic2eo, eo2lexic, iseven, isevent,
                         lexic2eot, eot2lexic);
}

int cvcb_gamma_tables(int *perm, int *sign) {
  if (!perm || !sign) return CVCB_ERR_NULL;
  gamma_tables(reinterpret_cast<int(*)[24]>(perm), reinterpret_cast<int(*)[24]>(sign));
  return CVCB_OK;
}

int cvcb_boundary_phases(int T, int LX, int LY, int LZ, const double bc[4], double ph[8]) {
  if (!bc || !ph) return CVCB_ERR_NULL;
  if (T <= 0 || LX <= 0 || LY <= 0 || LZ <= 0) {
    set_error("boundary phases: extents %d x %d x %d x %d", T, LX, LY, LZ);
    return CVCB_ERR_ARG;
  }
  boundary_phases(T, LX, LY, LZ, bc, ph);
  return CVCB_OK;
}

int cvcb_ranlxd(int level, int seed, double *r, long n) { return ranlxd_fill(level, seed, r, n); }

int cvcb_gauge_random(double *gauge, int T, int LX, int LY, int LZ, double eps, int seed) {
  return gauge_random(gauge, T, LX, LY, LZ, eps, seed);
}

}  // extern "C"
