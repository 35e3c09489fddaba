// Complex spinor scalar product with no device allocation.
//
// Some callers cannot call cudaMalloc: host programs whose device memory is
// owned by a pool of their own (a solver framework that carves every buffer
// out of one up-front allocation and forbids others), and callers in the
// middle of an asynchronous pipeline, where cudaMalloc/cudaFree may
// synchronise the whole device and stall their other streams.  They also
// cannot create a cvcb_lattice, whose set-up allocates.  For them this file
// offers a variant of the reduction behind cvcb_spinor_scalar_product_co
// whose only scratch -- the per-block partial sums and the completion
// counter of the single-launch reduction -- lives in one file-scope
// __device__ array of fixed size, so the call allocates nothing.
//
// Limits and sharing:
//   * at most kNoAllocMaxSites lattice sites (one partial sum per block of
//     kElemsPerBlock / 12 sites must fit the array); larger V is rejected;
//   * the array exists once per GPU that loads the library and is held
//     until the process exits;
//   * every call on a device uses the same array and leaves its contents
//     behind; the completion counter is cleared at the start of each call
//     (stream-ordered), the partials are fully rewritten; calls that overlap
//     on the GPU (for example on two streams at once) race on the array and
//     must be serialised by the caller;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it; make
//     that first call before any stream capture on the device;
//   * the call is stream-ordered: it returns once the work is enqueued on
//     `stream`, and w holds the result when the stream reaches that point.
#include <mutex>

#include "cvcb_internal.h"
#include "reduce.cuh"

namespace cvcb {
namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocPerThread = 16;
constexpr int kElemsPerBlock = kNoAllocThreads * kNoAllocPerThread;  // complex numbers
constexpr int kNoAllocMaxBlocks = 16384;
// 12 complex numbers per site
constexpr long long kNoAllocMaxSites = (long long)kNoAllocMaxBlocks * kElemsPerBlock / 12;

// partials: 2 doubles per block; the last slot pair holds the counter.
constexpr int kScratchDoubles = 2 * kNoAllocMaxBlocks + 2;
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_mutex;
double *g_scratch_ptr[64] = {nullptr};

__global__ void __launch_bounds__(kNoAllocThreads)
    k_dot_co_noalloc(const double2 *__restrict__ a, const double2 *__restrict__ b, long long n,
                     double *__restrict__ scratch, double *__restrict__ out) {
  __shared__ double sh[2][kNoAllocThreads / 32];
  __shared__ bool last;
  double v[2] = {0.0, 0.0};
  const long long base = (long long)blockIdx.x * kElemsPerBlock;
#pragma unroll
  for (int j = 0; j < kNoAllocPerThread; ++j) {
    const long long k = base + threadIdx.x + (long long)j * kNoAllocThreads;
    if (k < n) {
      const double2 x = __ldg(a + k), y = __ldg(b + k);
      v[0] += x.x * y.x + x.y * y.y;
      v[1] += x.x * y.y - x.y * y.x;
    }
  }
  block_sum<2>(v, sh);
  unsigned *counter = reinterpret_cast<unsigned *>(scratch + 2 * kNoAllocMaxBlocks);
  if (threadIdx.x == 0) {
    scratch[2 * blockIdx.x] = v[0];
    scratch[2 * blockIdx.x + 1] = v[1];
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  v[0] = v[1] = 0.0;
  for (int blk = threadIdx.x; blk < (int)gridDim.x; blk += kNoAllocThreads) {
    v[0] += __ldcg(scratch + 2 * blk);
    v[1] += __ldcg(scratch + 2 * blk + 1);
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    out[0] = v[0];
    out[1] = v[1];
    *counter = 0;
  }
}

// Device address of the scratch array on `device` (looked up once).
int scratch_on(int device, double **ptr) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (device < 0 || device >= 64) {
    set_error("device ordinal %d out of range", device);
    return CVCB_ERR_ARG;
  }
  if (!g_scratch_ptr[device]) {
    int prev = 0;
    CVCB_CUDA(cudaGetDevice(&prev));
    CVCB_CUDA(cudaSetDevice(device));
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    cudaSetDevice(prev);
    if (e != cudaSuccess || !p) {
      set_error("cudaGetSymbolAddress of the scratch array failed on device %d: %s", device,
                cudaGetErrorString(e));
      return CVCB_ERR_CUDA;
    }
    g_scratch_ptr[device] = static_cast<double *>(p);
  }
  *ptr = g_scratch_ptr[device];
  return CVCB_OK;
}

bool on_device(const void *p, int device) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == device;
}

}  // namespace
}  // namespace cvcb

extern "C" int cvcb_spinor_scalar_product_co_noalloc(int device, double *w, const double *xi,
                                                     const double *phi, int V, void *stream) {
  using namespace cvcb;
  if (!w || !xi || !phi) return CVCB_ERR_NULL;
  if (V <= 0 || (long long)V > kNoAllocMaxSites) {
    set_error("V = %d outside [1, %lld]: the no-allocation scalar product keeps one partial sum "
              "per %d sites in a fixed device array",
              V, kNoAllocMaxSites, kElemsPerBlock / 12);
    return CVCB_ERR_ARG;
  }
  if (!on_device(w, device) || !on_device(xi, device) || !on_device(phi, device)) {
    set_error("w, xi and phi must be device memory of device %d", device);
    return CVCB_ERR_ARG;
  }
  double *scratch;
  CVCB_TRY(scratch_on(device, &scratch));
  int prev = 0;
  CVCB_CUDA(cudaGetDevice(&prev));
  CVCB_CUDA(cudaSetDevice(device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long n = 12LL * V;
  const int blocks = (int)((n + kElemsPerBlock - 1) / kElemsPerBlock);
  // the completion counter must start at zero
  cudaError_t e = cudaMemsetAsync(scratch + 2 * kNoAllocMaxBlocks, 0, sizeof(unsigned), s);
  if (e == cudaSuccess) {
    k_dot_co_noalloc<<<blocks, kNoAllocThreads, 0, s>>>(
        reinterpret_cast<const double2 *>(xi), reinterpret_cast<const double2 *>(phi), n, scratch,
        w);
    e = cudaGetLastError();
  }
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    set_error("no-allocation scalar product: %s", cudaGetErrorString(e));
    return CVCB_ERR_CUDA;
  }
  return CVCB_OK;
}
