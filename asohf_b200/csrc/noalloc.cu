// noalloc.cu -- the base-grid kernel deposit of DENSITY into a caller's grid,
// with no device allocation at all.
//
// Some callers cannot allocate device memory while they run: an application
// that hands the whole GPU memory to its own pool at start-up and forbids
// later cudaMalloc, or code that must not trigger the device-wide
// synchronisation that cudaMalloc/cudaFree can cause.  For them the float64
// accumulator this deposit needs lives in a fixed file-scope device array of
// ASOHF_NOALLOC_MAX_CELLS cells (16 MiB), and the entry point neither
// allocates nor frees anything.
//
// With CUDA's lazy module loading (the default since CUDA 12.2) the array and
// the two kernels are placed on a device when this module is first used
// there, not when the library is loaded.  The first call on each device
// therefore does that set-up (symbol lookup plus a load of both kernels); it
// is the one call that can need device memory, and must come before the
// application reserves its memory and before any stream capture.  A call with
// n = 0 is enough.  From then on the array is held on that device until the
// process exits.
#include <atomic>
#include <mutex>

#include "common.cuh"

static __device__ __align__(256) double g_noalloc_acc[ASOHF_NOALLOC_MAX_CELLS];

// Per-device set-up results.  Host code may not use the array's host-side
// stand-in as a device address, so the address comes from
// cudaGetSymbolAddress, looked up once per device with that device current.
// Readers take the published pointer with acquire ordering; the set-up runs
// under a mutex and publishes with release ordering, after the SM count.
namespace {
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
std::atomic<double*> g_acc_addr[kMaxDevices];
int g_sm_count[kMaxDevices];
}  // namespace

struct Level0Kernel {
  float w[3];  // W(-1), W(0), W(1) of COMPUTE_KERNELS level 0
};

// COMPUTE_KERNELS (grids.f:997-1067) for level 0 only (N = 1).
static Level0Kernel level0_kernel(int deg) {
  Level0Kernel k;
  float h32 = 1.0f + 0.5f;
  float h = 2.0f * h32 / 3.0f;
  for (int i = -1; i <= 1; i++) {
    float v;
    if (deg == 2) {
      float bas = (float)(i < 0 ? -i : i) / h;
      if (bas <= 0.5f) {
        v = 0.75f - bas * bas;
      } else {
        float t = 1.5f - bas;
        v = 0.5f * (t * t);
      }
    } else {
      v = 1.0f - (float)(i < 0 ? -i : i) / h32;
    }
    k.w[i + 1] = v;
  }
  float bas = 0.0f;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int q = 0; q < 3; q++) {
        volatile float t = k.w[i] * k.w[j];
        t = t * k.w[q];
        bas = bas + t;
      }
  bas = 1.0f / powf(bas, 1.0f / 3.0f);
  for (int i = 0; i < 3; i++) k.w[i] = bas * k.w[i];
  return k;
}

// The 27-cell periodic cloud of grids.f:787-820 accumulated in float64 into
// the file-scope array (same cloud terms as k_density_base_all).
__global__ void k_density_base_noalloc(const float* __restrict__ x, const float* __restrict__ y,
                                       const float* __restrict__ z, const float* __restrict__ m,
                                       int64_t n, int nx, float xl, float dx, Level0Kernel K,
                                       double* __restrict__ acc) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float bas = m[i];
    int ix = (int)((x[i] - xl) / dx) + 1;
    int jy = (int)((y[i] - xl) / dx) + 1;
    int kz = (int)((z[i] - xl) / dx) + 1;
    for (int kk = -1; kk <= 1; kk++)
      for (int jj = -1; jj <= 1; jj++)
        for (int ii = -1; ii <= 1; ii++) {
          int i1 = ix + ii, j1 = jy + jj, k1 = kz + kk;
          if (i1 > nx) i1 -= nx;
          if (i1 < 1) i1 += nx;
          if (j1 > nx) j1 -= nx;
          if (j1 < 1) j1 += nx;
          if (k1 > nx) k1 -= nx;
          if (k1 < 1) k1 += nx;
          if (i1 < 1 || i1 > nx || j1 < 1 || j1 > nx || k1 < 1 || k1 > nx) continue;  // outside the box
          float t = __fmul_rn(__fmul_rn(__fmul_rn(bas, K.w[ii + 1]), K.w[jj + 1]), K.w[kk + 1]);
          atomicAdd(&acc[((size_t)(k1 - 1) * nx + (j1 - 1)) * nx + (i1 - 1)], (double)t);
        }
  }
}

__global__ void k_finish_noalloc(const double* __restrict__ acc, int64_t g, float denbas,
                                 float* __restrict__ u1) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < g;
       c += (int64_t)gridDim.x * blockDim.x)
    u1[c] = (float)acc[c] / denbas;
}

// Loads the array and both kernels on device `dev` (current) and records the
// array's device address and the SM count.  Called under g_setup_mutex.
static int noalloc_setup(int dev) {
  double* addr = nullptr;
  ASOHF_CUDA(cudaGetSymbolAddress((void**)&addr, g_noalloc_acc));
  cudaFuncAttributes fa;
  ASOHF_CUDA(cudaFuncGetAttributes(&fa, k_density_base_noalloc));
  ASOHF_CUDA(cudaFuncGetAttributes(&fa, k_finish_noalloc));
  int sms = 0;
  ASOHF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  g_sm_count[dev] = sms > 0 ? sms : 1;
  g_acc_addr[dev].store(addr, std::memory_order_release);
  return ASOHF_OK;
}

extern "C" int asohf_density_base_noalloc(int nx, float lado0, float dx, float rote, float rete,
                                          int interp_degree, int64_t n, const float* x,
                                          const float* y, const float* z, const float* m,
                                          float* u1, void* cuda_stream) {
  if (nx <= 0 || !u1 || n < 0 || (n > 0 && (!x || !y || !z || !m)) ||
      (interp_degree != 1 && interp_degree != 2))
    return ASOHF_ERR_INVALID;
  int64_t g = (int64_t)nx * nx * nx;
  if (g > (int64_t)ASOHF_NOALLOC_MAX_CELLS) return ASOHF_ERR_CAPACITY;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) {
    cudaGetLastError();
    return ASOHF_ERR_NO_DEVICE;
  }
  ASOHF_CUDA(e);
  if (dev < 0 || dev >= kMaxDevices) return ASOHF_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)cuda_stream;
  if (s != nullptr && s != cudaStreamLegacy && s != cudaStreamPerThread) {
    // the array's address is per device: the stream must run on the current one
    int sdev = -1;
    ASOHF_CUDA(cudaStreamGetDevice(s, &sdev));
    if (sdev != dev) return ASOHF_ERR_INVALID;
  }
  double* acc = g_acc_addr[dev].load(std::memory_order_acquire);
  if (!acc) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    acc = g_acc_addr[dev].load(std::memory_order_acquire);
    if (!acc) {
      ASOHF_CHECK(noalloc_setup(dev));
      acc = g_acc_addr[dev].load(std::memory_order_acquire);
    }
  }
  const int max_blocks = g_sm_count[dev] * 16;
  // the array keeps the previous call's sums: clear the cells this grid uses
  ASOHF_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * (size_t)g, s));
  if (n > 0) {
    int64_t blocks = (n + 255) / 256;
    if (blocks > max_blocks) blocks = max_blocks;
    k_density_base_noalloc<<<(int)blocks, 256, 0, s>>>(x, y, z, m, n, nx, -lado0 / 2.0f, dx,
                                                       level0_kernel(interp_degree), acc);
    ASOHF_CUDA(cudaGetLastError());
  }
  float denbas = dx * dx * dx * rote * (rete * rete * rete);
  int64_t fb = (g + 255) / 256;
  if (fb > max_blocks) fb = max_blocks;
  k_finish_noalloc<<<(int)fb, 256, 0, s>>>(acc, g, denbas, u1);
  ASOHF_CUDA(cudaGetLastError());
  return ASOHF_OK;
}
