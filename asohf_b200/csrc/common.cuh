// common.cuh -- internals shared by the sm_100a kernels of libasohf_gpu.so:
// status handling, the per-caller context (stream, device particle store,
// scratch arena) and warp/block reduction helpers.
//
// Every kernel that restates a reference statement is compiled with
// -fmad=false, so a*b+c keeps two roundings like the Fortran it restates;
// sqrtf and '/' are IEEE (nvcc's -prec-sqrt / -prec-div defaults).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <thread>
#include <vector>

#include "../../include/asohf_gpu.h"

#define ASOHF_CUDA(call)                                                   \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) {                                               \
      asohf_set_last_cuda_error(e_, #call, __FILE__, __LINE__);            \
      return ASOHF_ERR_CUDA;                                               \
    }                                                                      \
  } while (0)

#define ASOHF_CHECK(rc_expr)      \
  do {                            \
    int rc_ = (rc_expr);          \
    if (rc_ != ASOHF_OK) return rc_; \
  } while (0)

void asohf_set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line);

// Device particle store owned by the context (SoA, MODULE PARTICLES order).
struct DevParticles {
  int64_t n = 0, cap = 0;
  float *x = nullptr, *y = nullptr, *z = nullptr;
  float *vx = nullptr, *vy = nullptr, *vz = nullptr;
  float *m = nullptr;
  int32_t* id = nullptr;
};

struct asohf_ctx {
  int device = 0;
  cudaStream_t stream = 0;
  // streams for per-halo launches that run beside the cluster launch,
  // forked from and joined back into `stream` with the events
  static const int NSIDE = 5;
  cudaStream_t side[NSIDE] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int side_prio = 0;  // the side streams take the context stream's priority
  cudaEvent_t ev_fork = nullptr, ev_join[NSIDE] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int num_sms = 148;
  // size tiers of the per-halo launches (members): >= cluster_min a CTA
  // cluster, >= tier2_k 256 threads, >= tier1_k 128 threads, else 32
  int64_t cluster_min = 32768;
  int64_t cluster_share = 32768;  // entries per CTA that set the halo kernel's cluster width
  int64_t tier2_k = 2048, tier1_k = 256;
  // seed of COMPUTE_EPOT's sampling estimator (asohf_set_epot_seed)
  uint32_t epot_seed = 1;
  DevParticles p;      // current store
  DevParticles alt;    // second buffer set for permutations
  // The store as rows (x, y, z, m | vx, vy, vz, id bits), 2 float4 per
  // particle, in two buffers: rows[rows_cur] holds the current order after
  // a permutation (-1: none since the upload), the other is the target of
  // the next one.  Gathers of one particle read one or two 16-byte rows
  // instead of one sector per field.
  float4* rows[2] = {nullptr, nullptr};
  int64_t rows_cap = 0;
  int rows_cur = -1;
  float norma = 0.f;   // MAXVAL(MASAP), refreshed on upload
  float mmin = 0.f;
  // x-slab index (SORT_DM_PARTICLES_X) and the column index built from it
  int nx_sorted = 0;
  int ndmpart_cap = 0;               // entries of d_ndmpart_x
  int32_t* d_ndmpart_x = nullptr;   // NX+1 entries
  int64_t ncols = 0;                // columns of the (y,z) index
  float col_xl = 0.f, col_dx = 0.f;
  int col_n = 0;                    // columns per axis
  int64_t* d_colstart = nullptr;    // ncols+1
  float4* d_colpart = nullptr;      // (x, y, z, position in x-sorted store as int bits)
  int64_t colpart_cap = 0;
  // bound-particle ID stream (PARTICLES_PER_HALO)
  int32_t* d_pph = nullptr;
  // sorted member segments of the subhaloes whose Jacobi radius is fixed,
  // in the order they were fixed (SUBSTRUCTURE_PARTICLES)
  // staging store of asohf_prefetch_particles: copied on copy_stream while
  // the context stream runs; taken by the matching asohf_upload_particles
  DevParticles stage;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t stage_ready = nullptr, stage_free = nullptr, chunk_done = nullptr;
  bool staged = false, stage_free_set = false;
  std::thread stager;       // issues the staged copy chunk by chunk
  int stage_status = 0;     // its status (read after join)
  // device -> host copies of asohf_copy_to_host_async, issued chunk by chunk
  // on out_stream by a helper thread
  struct OutJob {
    void* dst;
    const void* src;
    int64_t bytes;
  };
  cudaStream_t out_stream = nullptr;
  cudaEvent_t out_fork = nullptr, out_chunk = nullptr, out_done = nullptr;
  std::thread outer;
  std::mutex out_mu;
  std::vector<OutJob> out_jobs;
  bool out_running = false, out_any = false;
  int out_status = 0;
  const void* staged_src[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  int64_t staged_n = 0;
  unsigned long long* sfin_k = nullptr;
  int32_t* sfin_v = nullptr;
  int64_t sfin_cap = 0;
  int64_t pph_len = 0, pph_cap = 0;
  // scratch arena (bump allocator, reset at the start of every entry point)
  char* arena = nullptr;
  size_t arena_size = 0, arena_used = 0;
  // per-halo segment buffers (keys, distances, potentials...), grown between
  // kernel phases of one call, when the stream is idle
  char* seg = nullptr;
  size_t seg_size = 0, seg_used = 0;
  // Deferred patch deposit (asohf_set_density_overlap): with device outputs
  // the patch kernels of asohf_density (and RENORM_DENSITY's patch scaling)
  // run on dens_stream from the two density pools, which later calls do not
  // reuse, and finish after the call returns; dens_done marks their end.
  int density_overlap = 0;
  cudaStream_t dens_stream = nullptr;
  cudaEvent_t dens_fork = nullptr, dens_done = nullptr;
  bool dens_pending = false;
  struct Pool { char* base = nullptr; size_t size = 0, used = 0; };
  Pool dpool[2];
  // device copies kept between calls: MOMENTO's sin^2 table for s2_nx, and
  // the last RADX(0:NX+1) the layer was given (h_radx: its host copy)
  float* d_s2 = nullptr;
  int s2_nx = 0;
  // the FFT convolution's twiddle table W_N^j, j < tw_n
  float2* d_tw = nullptr;
  int tw_n = 0;
  float* d_radx = nullptr;
  float* h_radx = nullptr;
  int radx_n = 0;
  // counters of kernels launched by this context (reported by the bench)
  int64_t launches = 0;
  // work counters written by kernels (element-passes of the per-halo kernels)
  unsigned long long* d_work = nullptr;  // 8 counters
  // optional CUDA-event timing of named kernels (asohf_set_profiling)
  int profiling = 0;
  struct KRec { const char* name; cudaEvent_t a, b; cudaStream_t s; };  // events on the launch's stream
  KRec* krec = nullptr;
  int nkrec = 0, capkrec = 0;
  struct KSum { const char* name; double ms; int64_t n; };
  static constexpr int KSUM_CAP = 256;
  KSum ksum[KSUM_CAP];
  int nksum = 0;
};

// Brackets a kernel launch with events on the context stream when profiling.
int ktime_begin(asohf_ctx* c, const char* name, cudaStream_t s);
void ktime_end(asohf_ctx* c, int slot, cudaStream_t s);
inline int ktime_begin(asohf_ctx* c, const char* name) { return ktime_begin(c, name, c->stream); }
inline void ktime_end(asohf_ctx* c, int slot) { ktime_end(c, slot, c->stream); }
// Host wall time (ms) of a phase of an entry point, added to the same
// statistics as the kernels when profiling is on.
double htime_now();
void htime_end(asohf_ctx* c, const char* name, double t0);

// Scratch: reserve() may grow the arena only when nothing is allocated from it.
int arena_reserve(asohf_ctx* c, size_t bytes);
void* arena_alloc(asohf_ctx* c, size_t bytes);  // 256-byte aligned, nullptr if full
inline void arena_reset(asohf_ctx* c) { c->arena_used = 0; }

// Segment buffer: reserve() syncs the stream and regrows it (contents lost).
int seg_reserve(asohf_ctx* c, size_t bytes);
// Density pools 0 and 1 (bump allocators like the arena, reset by
// dpool_reserve; the caller has waited for any deferred patch work).
int dpool_reserve(asohf_ctx* c, int which, size_t bytes);
void* dpool_alloc(asohf_ctx* c, int which, size_t bytes);
// Waits (host) for a deferred patch deposit still in flight.
int density_settle(asohf_ctx* c);
void* seg_alloc(asohf_ctx* c, size_t bytes);

int ctx_ensure_particles(asohf_ctx* c, int64_t n);
void ctx_swap_particles(asohf_ctx* c);
int ctx_refresh_mass_range(asohf_ctx* c);

inline int grid_for(int64_t n, int block, int max_blocks = 148 * 32) {
  int64_t g = (n + block - 1) / block;
  if (g > max_blocks) g = max_blocks;
  if (g < 1) g = 1;
  return (int)g;
}

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int warp_sum_i(int v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of a double, result valid in every thread.  sbuf >= 32 doubles.
__device__ __forceinline__ double block_sum_d(double v, double* sbuf) {
  if (blockDim.x == 32) {  // one warp: butterfly, no shared memory
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
  }
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum_d(v);
  __syncthreads();
  if (lane == 0) sbuf[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (wid == 0) {
    t = lane < nw ? sbuf[lane] : 0.0;
    t = warp_sum_d(t);
    if (lane == 0) sbuf[0] = t;
  }
  __syncthreads();
  t = sbuf[0];
  __syncthreads();
  return t;
}

__device__ __forceinline__ long long block_sum_ll(long long v, long long* sbuf) {
  if (blockDim.x == 32) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
  }
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) sbuf[wid] = v;
  __syncthreads();
  long long t = 0;
  if (wid == 0) {
    t = lane < nw ? sbuf[lane] : 0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) sbuf[0] = t;
  }
  __syncthreads();
  t = sbuf[0];
  __syncthreads();
  return t;
}

__device__ __forceinline__ long long block_min_ll(long long v, long long* sbuf) {
  if (blockDim.x == 32) {
    for (int o = 16; o > 0; o >>= 1) {
      long long w = __shfl_xor_sync(0xffffffffu, v, o);
      v = w < v ? w : v;
    }
    return v;
  }
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    long long w = __shfl_down_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  __syncthreads();
  if (lane == 0) sbuf[wid] = v;
  __syncthreads();
  long long t = LLONG_MAX;
  if (wid == 0) {
    t = lane < nw ? sbuf[lane] : LLONG_MAX;
    for (int o = 16; o > 0; o >>= 1) {
      long long w = __shfl_down_sync(0xffffffffu, t, o);
      t = w < t ? w : t;
    }
    if (lane == 0) sbuf[0] = t;
  }
  __syncthreads();
  t = sbuf[0];
  __syncthreads();
  return t;
}

__device__ __forceinline__ float block_max_f(float v, float* sbuf) {
  if (blockDim.x == 32) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
  }
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) sbuf[wid] = v;
  __syncthreads();
  float t = -INFINITY;
  if (wid == 0) {
    t = lane < nw ? sbuf[lane] : -INFINITY;
    for (int o = 16; o > 0; o >>= 1) t = fmaxf(t, __shfl_down_sync(0xffffffffu, t, o));
    if (lane == 0) sbuf[0] = t;
  }
  __syncthreads();
  t = sbuf[0];
  __syncthreads();
  return t;
}

__device__ __forceinline__ float block_min_f(float v, float* sbuf) {
  return -block_max_f(-v, sbuf);
}

// Inclusive block scan of ints; returns the inclusive prefix; *total gets the
// block total.  sbuf >= 33 ints.
__device__ __forceinline__ int block_scan_i(int v, int* sbuf, int* total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  __syncthreads();
  if (lane == 31) sbuf[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int s = lane < nw ? sbuf[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) sbuf[lane] = s;
  }
  __syncthreads();
  int off = wid > 0 ? sbuf[wid - 1] : 0;
  int tot = sbuf[nw - 1];
  __syncthreads();
  if (total) *total = tot;
  return x + off;
}

// Inclusive block scan of doubles (left-to-right within the block).
__device__ __forceinline__ double block_scan_d(double v, double* sbuf, double* total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  double x = v;
  for (int o = 1; o < 32; o <<= 1) {
    double y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  __syncthreads();
  if (lane == 31) sbuf[wid] = x;
  __syncthreads();
  if (wid == 0) {
    double s = lane < nw ? sbuf[lane] : 0.0;
    for (int o = 1; o < 32; o <<= 1) {
      double y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) sbuf[lane] = s;
  }
  __syncthreads();
  double off = wid > 0 ? sbuf[wid - 1] : 0.0;
  double tot = sbuf[nw - 1];
  __syncthreads();
  if (total) *total = tot;
  return x + off;
}

// TSC weights of grids.f:1194-1213: BAS=|x-r|/d, 0.5(1.5-BAS)^2, 0.75-BAS^2.
__device__ __forceinline__ void tsc_weights(float xp, float rm, float r0, float rp, float d, float* v) {
  float b = fabsf(__fsub_rn(xp, rm)) / d;
  float t = __fsub_rn(1.5f, b);
  v[0] = __fmul_rn(0.5f, __fmul_rn(t, t));
  b = fabsf(__fsub_rn(xp, r0)) / d;
  v[1] = __fsub_rn(0.75f, __fmul_rn(b, b));
  b = fabsf(__fsub_rn(xp, rp)) / d;
  t = __fsub_rn(1.5f, b);
  v[2] = __fmul_rn(0.5f, __fmul_rn(t, t));
}

__device__ __forceinline__ int tsc_cell(float v, float xl, float dx, int nx) {
  int i = (int)((v - xl) / dx) + 1;
  return i < 1 ? 1 : (i > nx ? nx : i);
}

// Stable descending order of w[0..k) by key[] (an unsigned image of the
// value that preserves its order): LSD radix sort on the complemented key,
// 8 bits a pass, passes whose digit is the same for every entry skipped.
// Equal values keep their order, as in a stable comparison sort.
static inline void stable_desc(std::vector<uint32_t>& key, int32_t* w, int k) {
  std::vector<uint32_t> key2((size_t)k);
  std::vector<int32_t> tmp((size_t)k);
  for (int i = 0; i < k; i++) key[i] = ~key[i];
  for (int sh = 0; sh < 32; sh += 8) {
    int64_t cnt[257] = {0};
    for (int i = 0; i < k; i++) cnt[((key[i] >> sh) & 255u) + 1]++;
    bool one = false;
    for (int d = 0; d < 256; d++) one |= cnt[d + 1] == k;
    if (one) continue;
    for (int d = 0; d < 256; d++) cnt[d + 1] += cnt[d];
    for (int i = 0; i < k; i++) {
      const int64_t o = cnt[(key[i] >> sh) & 255u]++;
      tmp[o] = w[i];
      key2[o] = key[i];
    }
    memcpy(w, tmp.data(), 4 * (size_t)k);
    key.swap(key2);
  }
}

