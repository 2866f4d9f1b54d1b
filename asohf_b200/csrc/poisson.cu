// poisson.cu -- periodic FFT Poisson solve (MOMENTO + POFFT3D, poisson.f:98-249)
// and the differentiable deposit+Poisson layer with its adjoint.
//
// The reference packs the real density into a full complex array and runs a
// complex FFT (Numerical-Recipes FOURN) forward, multiplies by KKK, inverse,
// real part / N^3.  For real input that is exactly an R2C / C2R pair on the
// half spectrum.  For NX in {64, 128, 256, 512} it runs as cuFFT's 2-D R2C
// of the planes, one hand-written pass doing the z transforms and the
// Green's multiply (fftconv.cu), and cuFFT's 2-D C2R; for other sizes as a
// cuFFT 3-D pair with the Green's function KKK = -(DX/2)^2 / sum
// sin^2(pi k/N) (KKK(1,1,1) from the 1e30 denominator) and the 1/N^3
// normalisation applied in one pass over the half spectrum (k_green).
#include <cufft.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "common.cuh"

int fftconv_z_green_2d(asohf_ctx* c, int nx, int batch, void* spec, const float* s2, float del2, float inv_n3);
int tsc_base_batched_f32(asohf_ctx* c, int nx, float xl, float dx, const float* dradx, int batch,
                         int64_t n_per, const float* x, const float* y, const float* z,
                         const float* m, float denbas, float* acc);

#define ASOHF_CUFFT(call)                                                        \
  do {                                                                           \
    cufftResult r_ = (call);                                                     \
    if (r_ != CUFFT_SUCCESS) {                                                   \
      asohf_set_last_cuda_error(cudaErrorUnknown, #call, __FILE__, __LINE__);    \
      return ASOHF_ERR_CUDA;                                                     \
    }                                                                            \
  } while (0)

struct FftPlan {
  int nx = 0, batch = 0;
  cufftHandle r2c = 0, c2r = 0;      // 3-D, batch copies
  cufftHandle r2c2 = 0, c2r2 = 0;    // 2-D over the batch * nx planes
  cudaStream_t stream = 0;
};

static FftPlan g_plans[8];

// the sizes the fused z pass covers (fftconv.cu); the others take 3-D transforms
static bool fftconv_size(int nx) { return nx == 64 || nx == 128 || nx == 256 || nx == 512; }

static int get_plan(asohf_ctx* c, int nx, int batch, FftPlan** out) {
  for (auto& p : g_plans)
    if (p.nx == nx && p.batch == batch) {
      if (p.stream != c->stream) {
        for (cufftHandle h : {p.r2c, p.c2r, p.r2c2, p.c2r2})
          if (h) ASOHF_CUFFT(cufftSetStream(h, c->stream));
        p.stream = c->stream;
      }
      *out = &p;
      return ASOHF_OK;
    }
  FftPlan* slot = nullptr;
  for (auto& p : g_plans)
    if (p.nx == 0) { slot = &p; break; }
  if (!slot) {
    slot = &g_plans[0];
    for (cufftHandle h : {slot->r2c, slot->c2r, slot->r2c2, slot->c2r2})
      if (h) cufftDestroy(h);
    *slot = FftPlan();
  }
  if (fftconv_size(nx)) {  // 2-D transforms of the batch * nx planes
    int n2[2] = {nx, nx};
    int64_t g2 = (int64_t)nx * nx, gc2 = (int64_t)nx * (nx / 2 + 1);
    ASOHF_CUFFT(cufftPlanMany(&slot->r2c2, 2, n2, nullptr, 1, (int)g2, nullptr, 1, (int)gc2, CUFFT_R2C, batch * nx));
    ASOHF_CUFFT(cufftPlanMany(&slot->c2r2, 2, n2, nullptr, 1, (int)gc2, nullptr, 1, (int)g2, CUFFT_C2R, batch * nx));
    ASOHF_CUFFT(cufftSetStream(slot->r2c2, c->stream));
    ASOHF_CUFFT(cufftSetStream(slot->c2r2, c->stream));
  } else {
    int n[3] = {nx, nx, nx};
    int64_t g = (int64_t)nx * nx * nx, gc = (int64_t)nx * nx * (nx / 2 + 1);
    ASOHF_CUFFT(cufftPlanMany(&slot->r2c, 3, n, nullptr, 1, (int)g, nullptr, 1, (int)gc, CUFFT_R2C, batch));
    ASOHF_CUFFT(cufftPlanMany(&slot->c2r, 3, n, nullptr, 1, (int)gc, nullptr, 1, (int)g, CUFFT_C2R, batch));
    ASOHF_CUFFT(cufftSetStream(slot->r2c, c->stream));
    ASOHF_CUFFT(cufftSetStream(slot->c2r, c->stream));
  }
  slot->nx = nx;
  slot->batch = batch;
  slot->stream = c->stream;
  *out = slot;
  return ASOHF_OK;
}

// sin^2(pi k / N) per axis index, REAL*4 as MOMENTO computes it (host sinf).
static void momento_axis(int nx, float* s2) {
  float pi = acosf(-1.0f);
  float consta = pi / (float)nx;
  int n2 = nx / 2 + 2;
  for (int i = 1; i <= nx; i++) {
    int k = (i >= n2) ? i - nx - 1 : i - 1;
    float s = sinf(consta * (float)k);
    s2[i - 1] = s * s;
  }
}

// Half-spectrum multiply: spec[(k*N + j)*(N/2+1) + i] *= KKK(i,j,k) / N^3.
// A flat grid-stride loop over the complex values (consecutive threads take
// consecutive values, so every warp access is one contiguous 256-byte run);
// the (i, j, k) of a value come from its index, s2 from the L1-resident table.
__global__ void k_green(cufftComplex* __restrict__ spec, int nx, int batch, const float* __restrict__ s2,
                        float del2, float inv_n3) {
  const int64_t nh = nx / 2 + 1;
  const int64_t total = (int64_t)batch * nx * nx * nh;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = q / nh;
    const int i = (int)(q - row * nh), j = (int)(row % nx), k = (int)((row / nx) % nx);
    const float den = (i == 0 && j == 0 && k == 0) ? 1.0e30f : __fadd_rn(__fadd_rn(__ldg(s2 + i), __ldg(s2 + j)),
                                                                         __ldg(s2 + k));
    const float kkk = -del2 / den;
    const float f = __fmul_rn(kkk, inv_n3);
    cufftComplex v = spec[q];
    v.x = __fmul_rn(v.x, f);
    v.y = __fmul_rn(v.y, f);
    spec[q] = v;
  }
}

// MOMENTO's table on the device, computed once per NX.
static int green_table(asohf_ctx* c, int nx, const float** out) {
  if (c->s2_nx != nx) {
    ASOHF_CUDA(cudaStreamSynchronize(c->stream));
    cudaFree(c->d_s2);
    c->d_s2 = nullptr;
    c->s2_nx = 0;
    std::vector<float> hs2_v((size_t)nx);
    float* hs2 = hs2_v.data();
    momento_axis(nx, hs2);
    cudaError_t e = cudaMalloc(&c->d_s2, 4 * (size_t)nx);
    if (e == cudaSuccess) e = cudaMemcpy(c->d_s2, hs2, 4 * (size_t)nx, cudaMemcpyHostToDevice);
    ASOHF_CUDA(e);
    c->s2_nx = nx;
  }
  *out = c->d_s2;
  return ASOHF_OK;
}

// RADX(0:NX+1) on the device; re-uploaded only when its contents change.
int radx_device(asohf_ctx* c, int nx, const float* radx, const float** out) {
  const int n = nx + 2;
  if (c->radx_n != n || memcmp(c->h_radx, radx, 4 * (size_t)n) != 0) {
    ASOHF_CUDA(cudaStreamSynchronize(c->stream));
    if (c->radx_n != n) {
      cudaFree(c->d_radx);
      free(c->h_radx);
      c->d_radx = nullptr;
      c->h_radx = (float*)malloc(4 * (size_t)n);
      c->radx_n = 0;
      if (!c->h_radx) return ASOHF_ERR_CAPACITY;
      ASOHF_CUDA(cudaMalloc(&c->d_radx, 4 * (size_t)n));
      c->radx_n = n;
    }
    memcpy(c->h_radx, radx, 4 * (size_t)n);
    ASOHF_CUDA(cudaMemcpy(c->d_radx, radx, 4 * (size_t)n, cudaMemcpyHostToDevice));
  }
  *out = c->d_radx;
  return ASOHF_OK;
}

// FFT solve on the context stream; returns once enqueued.
static int poisson_dev(asohf_ctx* c, int nx, float dx, int batch, const float* rho, float* pot) {
  int64_t gc = (int64_t)nx * nx * (nx / 2 + 1) * batch;
  cufftComplex* spec = (cufftComplex*)arena_alloc(c, sizeof(cufftComplex) * gc);
  if (!spec) return ASOHF_ERR_CAPACITY;
  const float* ds2;
  ASOHF_CHECK(green_table(c, nx, &ds2));
  float del2 = (dx * 0.5f) * (dx * 0.5f);
  float inv_n3 = 1.0f / ((float)nx * (float)nx * (float)nx);
  FftPlan* P;
  ASOHF_CHECK(get_plan(c, nx, batch, &P));
  if (fftconv_size(nx)) {
    // 2-D R2C of the planes, the fused z pass (fftconv.cu), 2-D C2R
    int kt2 = ktime_begin(c, "fft_r2c_2d");
    ASOHF_CUFFT(cufftExecR2C(P->r2c2, (cufftReal*)rho, spec));
    ktime_end(c, kt2);
    ASOHF_CHECK(fftconv_z_green_2d(c, nx, batch, spec, ds2, del2, inv_n3));
    kt2 = ktime_begin(c, "fft_c2r_2d");
    ASOHF_CUFFT(cufftExecC2R(P->c2r2, spec, (cufftReal*)pot));
    ktime_end(c, kt2);
    ASOHF_CUDA(cudaGetLastError());
    return ASOHF_OK;
  }
  int kt_ = ktime_begin(c, "fft_r2c");
  ASOHF_CUFFT(cufftExecR2C(P->r2c, (cufftReal*)rho, spec));
  ktime_end(c, kt_);
  {
    int kt_ = ktime_begin(c, "green_multiply");
    const int64_t total = (int64_t)batch * nx * nx * (nx / 2 + 1);
    k_green<<<grid_for(total, 256, c->num_sms * 16), 256, 0, c->stream>>>(spec, nx, batch, ds2, del2, inv_n3);
    ktime_end(c, kt_);
  }
  c->launches++;
  kt_ = ktime_begin(c, "fft_c2r");
  ASOHF_CUFFT(cufftExecC2R(P->c2r, spec, (cufftReal*)pot));
  ktime_end(c, kt_);
  ASOHF_CUDA(cudaGetLastError());
  return ASOHF_OK;
}

static size_t poisson_bytes(int nx, int batch) {
  return sizeof(cufftComplex) * (size_t)nx * nx * (nx / 2 + 1) * batch + 4096;
}

extern "C" int asohf_poisson_fft(asohf_ctx* c, int nx, float dx, int batch, const float* rho,
                                 float* pot, int on_device) {
  if (!c || nx < 2 || batch < 1 || !rho || !pot) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  int64_t g = (int64_t)nx * nx * nx * batch;
  ASOHF_CHECK(arena_reserve(c, poisson_bytes(nx, batch) + (on_device ? 0 : 8 * g) + 1024));
  const float* drho = rho;
  float* dpot = pot;
  if (!on_device) {
    float* t = (float*)arena_alloc(c, 4 * g);
    dpot = (float*)arena_alloc(c, 4 * g);
    ASOHF_CUDA(cudaMemcpyAsync(t, rho, 4 * g, cudaMemcpyHostToDevice, c->stream));
    drho = t;
  }
  ASOHF_CHECK(poisson_dev(c, nx, dx, batch, drho, dpot));
  if (!on_device) {
    ASOHF_CUDA(cudaMemcpyAsync(pot, dpot, 4 * g, cudaMemcpyDeviceToHost, c->stream));
    ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  }
  return ASOHF_OK;
}

// ------------------------------------------------------------ layer
// The layer's particles are sorted once per call by a key of (copy, Morton
// code of the host cell), so a warp reads 32 particles of neighbouring cells
// and the grid cells it touches are close together.  Particles that share a
// host cell share all 27 target cells: a warp adds each run of equal keys
// as one segmented sum (shuffles) and issues one atomic per run and target.
// In a halo core, where hundreds of particles share a cell, this replaces
// 27 contended atomics per particle by 27 per run (warp-aggregated atomics).
// The sums are float32; a cell's terms are added in a different order than
// the sequential loop of grids.f:1163-1239, which changes the result within
// float32 rounding.

// bits 0..9 of v spread to every third bit (Morton interleave)
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

struct LayerSort {
  uint32_t* keys;  // sorted keys: copy << cbits | Morton(ix-1, jy-1, kz-1)
  int32_t* idx;    // sorted particle indices
  float4* pm;      // (x, y, z, m) in input order
  int cbits;
};

static int ceil_log2(int64_t v) {
  int b = 0;
  while ((1ll << b) < v) b++;
  return b;
}

// whether the sorted path applies: keys fit in 31 bits, indices in int32
static bool layer_sortable(int nx, int batch, int64_t ntot) {
  return nx <= 1024 && 3 * ceil_log2(nx) + ceil_log2(batch) <= 31 && ntot < (1ll << 31);
}

static size_t layer_sort_bytes(int nx, int batch, int64_t ntot) {
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint32_t*)nullptr, (uint32_t*)nullptr, (int32_t*)nullptr,
                                  (int32_t*)nullptr, (int)(ntot > 0 ? ntot : 1), 0,
                                  3 * ceil_log2(nx) + ceil_log2(batch));
  return 32 * (size_t)ntot + tb + 2048;
}

__global__ void k_layer_keys(const float* __restrict__ x, const float* __restrict__ y,
                             const float* __restrict__ z, const float* __restrict__ m, int64_t ntot,
                             int64_t n_per, int nx, float xl, float dx, int cbits, uint32_t* __restrict__ keys,
                             int32_t* __restrict__ idx, float4* __restrict__ pm) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < ntot;
       q += (int64_t)gridDim.x * blockDim.x) {
    const float xp = x[q], yp = y[q], zp = z[q];
    const int ix = tsc_cell(xp, xl, dx, nx), jy = tsc_cell(yp, xl, dx, nx), kz = tsc_cell(zp, xl, dx, nx);
    const uint32_t mort = spread3((uint32_t)(ix - 1)) | (spread3((uint32_t)(jy - 1)) << 1) |
                          (spread3((uint32_t)(kz - 1)) << 2);
    keys[q] = ((uint32_t)(q / n_per) << cbits) | mort;
    idx[q] = (int32_t)q;
    pm[q] = make_float4(xp, yp, zp, m[q]);
  }
}

static int layer_sort(asohf_ctx* c, int nx, float xl, float dx, int batch, int64_t n_per, const float* x,
                      const float* y, const float* z, const float* m, LayerSort* s) {
  const int64_t ntot = n_per * batch;
  const int bits = 3 * ceil_log2(nx) + ceil_log2(batch);
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint32_t*)nullptr, (uint32_t*)nullptr, (int32_t*)nullptr,
                                  (int32_t*)nullptr, (int)ntot, 0, bits);
  uint32_t* k0 = (uint32_t*)arena_alloc(c, 4 * (size_t)ntot);
  uint32_t* k1 = (uint32_t*)arena_alloc(c, 4 * (size_t)ntot);
  int32_t* v0 = (int32_t*)arena_alloc(c, 4 * (size_t)ntot);
  int32_t* v1 = (int32_t*)arena_alloc(c, 4 * (size_t)ntot);
  float4* pm = (float4*)arena_alloc(c, 16 * (size_t)ntot);
  void* t = arena_alloc(c, tb);
  if (!k0 || !k1 || !v0 || !v1 || !pm || !t) return ASOHF_ERR_CAPACITY;
  s->cbits = 3 * ceil_log2(nx);
  {
    int kt_ = ktime_begin(c, "layer_keys");
    k_layer_keys<<<grid_for(ntot, 256, c->num_sms * 16), 256, 0, c->stream>>>(x, y, z, m, ntot, n_per, nx, xl, dx,
                                                                             s->cbits, k0, v0, pm);
    ktime_end(c, kt_);
  }
  c->launches++;
  {
    int kt_ = ktime_begin(c, "layer_sort");
    ASOHF_CUDA(cub::DeviceRadixSort::SortPairs(t, tb, k0, k1, v0, v1, (int)ntot, 0, bits, c->stream));
    ktime_end(c, kt_);
  }
  s->keys = k1;
  s->idx = v1;
  s->pm = pm;
  ASOHF_CUDA(cudaGetLastError());
  return ASOHF_OK;
}

// TSC deposit (grids.f:1163-1239, periodic base grid) of the sorted
// particles, m / DENBAS per particle; one warp per 32 sorted particles.
__global__ void __launch_bounds__(256) k_layer_deposit(const uint32_t* __restrict__ keys,
                                                       const int32_t* __restrict__ idx,
                                                       const float4* __restrict__ pm, int64_t ntot, int nx,
                                                       int cbits, float xl, float dx,
                                                       const float* __restrict__ radx, float denbas,
                                                       float* __restrict__ rho) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const size_t G = (size_t)nx * nx * nx;
  for (int64_t base = warp * 32; base < ntot; base += nwarps * 32) {
    const int64_t i = base + lane;
    const bool valid = i < ntot;
    const uint32_t key = valid ? keys[i] : 0xffffffffu;  // past the end: one run of its own
    const float4 p = valid ? pm[idx[i]] : make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t prev = __shfl_up_sync(FULL, key, 1);
    const bool head = lane == 0 || prev != key;
    const unsigned heads = __ballot_sync(FULL, head);
    const bool runs = __ballot_sync(FULL, !head) != 0u;  // some run is longer than one particle
    const int rs = 31 - __clz(heads & (FULL >> (31 - lane)));  // first lane of my run
    const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
    const int ix = tsc_cell(p.x, xl, dx, nx), jy = tsc_cell(p.y, xl, dx, nx), kz = tsc_cell(p.z, xl, dx, nx);
    float wx[3], wy[3], wz[3];
    tsc_weights(p.x, radx[ix - 1], radx[ix], radx[ix + 1], dx, wx);
    tsc_weights(p.y, radx[jy - 1], radx[jy], radx[jy + 1], dx, wy);
    tsc_weights(p.z, radx[kz - 1], radx[kz], radx[kz + 1], dx, wz);
    const float mp = __fdiv_rn(p.w, denbas);
    float* a = rho + (size_t)(valid ? (key >> cbits) : 0u) * G;
#pragma unroll
    for (int kk = -1; kk <= 1; kk++) {
      int k1 = kz + kk;
      if (k1 == nx + 1) k1 = 1;
      if (k1 == 0) k1 = nx;
#pragma unroll
      for (int jj = -1; jj <= 1; jj++) {
        int j1 = jy + jj;
        if (j1 == nx + 1) j1 = 1;
        if (j1 == 0) j1 = nx;
#pragma unroll
        for (int ii = -1; ii <= 1; ii++) {
          int i1 = ix + ii;
          if (i1 == nx + 1) i1 = 1;
          if (i1 == 0) i1 = nx;
          float t = valid ? __fmul_rn(__fmul_rn(__fmul_rn(mp, wx[ii + 1]), wy[jj + 1]), wz[kk + 1]) : 0.f;
          const size_t cell = ((size_t)(k1 - 1) * nx + (j1 - 1)) * nx + (i1 - 1);
          if (runs) {
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
              const float v = __shfl_up_sync(FULL, t, d);
              if (lane - d >= rs) t = __fadd_rn(t, v);
            }
            if (valid && tail) atomicAdd(&a[cell], t);
          } else if (valid) {
            atomicAdd(&a[cell], t);
          }
        }
      }
    }
  }
}

// dL/dx_p = m_p/DENBAS * sum_c d(Wx Wy Wz)/dx_p * g_c,  g = G * w, over the
// sorted particles (neighbouring warps read neighbouring cells of g).
__global__ void k_layer_adjoint(const uint32_t* __restrict__ keys, const int32_t* __restrict__ idx,
                                const float4* __restrict__ pm, int64_t ntot, int nx, int cbits, float xl,
                                float dx, const float* __restrict__ radx, const float* __restrict__ gfield,
                                float inv_denbas, float* __restrict__ gx, float* __restrict__ gy,
                                float* __restrict__ gz, float* __restrict__ gm);

extern "C" int asohf_tsc_poisson_forward(asohf_ctx* c, int nx, float lado0, float dx,
                                         const float* radx, float rote, float rete, int batch,
                                         int64_t n_per, const float* x, const float* y,
                                         const float* z, const float* m, float* rho, float* pot) {
  if (!c || nx < 2 || batch < 1 || n_per < 0 || !radx || !rho || !pot) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  int64_t g = (int64_t)nx * nx * nx * batch;
  const int64_t ntot = n_per * batch;
  const bool sorted = ntot > 0 && layer_sortable(nx, batch, ntot);
  ASOHF_CHECK(arena_reserve(c, poisson_bytes(nx, batch) + (sorted ? layer_sort_bytes(nx, batch, ntot) : 0) + 1024));
  const float* dradx;
  ASOHF_CHECK(radx_device(c, nx, radx, &dradx));
  ASOHF_CUDA(cudaMemsetAsync(rho, 0, 4 * g, c->stream));
  // each particle deposits m / (DX^3 ROTE RETE^3): the division of the cell
  // sums (grids.f:1236-1238) moved onto the terms, so rho needs no extra pass
  float denbas = dx * dx * dx * rote * (rete * rete * rete);
  const float xl = -lado0 / 2.0f;
  if (sorted) {
    LayerSort s;
    ASOHF_CHECK(layer_sort(c, nx, xl, dx, batch, n_per, x, y, z, m, &s));
    int kt_ = ktime_begin(c, "layer_deposit");
    k_layer_deposit<<<grid_for(ntot, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        s.keys, s.idx, s.pm, ntot, nx, s.cbits, xl, dx, dradx, denbas, rho);
    ktime_end(c, kt_);
    c->launches++;
    ASOHF_CUDA(cudaGetLastError());
  } else {
    ASOHF_CHECK(tsc_base_batched_f32(c, nx, xl, dx, dradx, batch, n_per, x, y, z, m, denbas, rho));
  }
  return poisson_dev(c, nx, dx, batch, rho, pot);
}

// dW/dx of the three TSC weights (grids.f:1194-1213):
//   W- = 0.5 (1.5-b)^2, W0 = 0.75-b^2, W+ = 0.5 (1.5-b)^2, b = |x-r|/d.
__device__ __forceinline__ void tsc_w_dw(float xp, float rm, float r0, float rp, float d, float* w, float* dw) {
  float s, b, t;
  s = xp - rm; b = fabsf(s) / d; t = 1.5f - b;
  w[0] = 0.5f * t * t; dw[0] = -t * copysignf(1.0f, s) / d;
  s = xp - r0; b = fabsf(s) / d;
  w[1] = 0.75f - b * b; dw[1] = -2.0f * b * copysignf(1.0f, s) / d;
  s = xp - rp; b = fabsf(s) / d; t = 1.5f - b;
  w[2] = 0.5f * t * t; dw[2] = -t * copysignf(1.0f, s) / d;
}

// dL/dx_p = m_p/DENBAS * sum_c d(Wx Wy Wz)/dx_p * g_c,  g = G * w.
__global__ void k_tsc_adjoint(const float* __restrict__ x, const float* __restrict__ y,
                              const float* __restrict__ z, const float* __restrict__ m, int64_t n_per,
                              int batch, int nx, float xl, float dx, const float* __restrict__ radx,
                              const float* __restrict__ gfield, float inv_denbas, float* __restrict__ gx,
                              float* __restrict__ gy, float* __restrict__ gz, float* __restrict__ gm) {
  int64_t ntot = n_per * batch;
  size_t G = (size_t)nx * nx * nx;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < ntot;
       q += (int64_t)gridDim.x * blockDim.x) {
    int b = (int)(q / n_per);
    float xp = x[q], yp = y[q], zp = z[q];
    int ix = (int)((xp - xl) / dx) + 1, jy = (int)((yp - xl) / dx) + 1, kz = (int)((zp - xl) / dx) + 1;
    ix = ix < 1 ? 1 : (ix > nx ? nx : ix);
    jy = jy < 1 ? 1 : (jy > nx ? nx : jy);
    kz = kz < 1 ? 1 : (kz > nx ? nx : kz);
    float wx[3], wy[3], wz[3], dwx[3], dwy[3], dwz[3];
    tsc_w_dw(xp, radx[ix - 1], radx[ix], radx[ix + 1], dx, wx, dwx);
    tsc_w_dw(yp, radx[jy - 1], radx[jy], radx[jy + 1], dx, wy, dwy);
    tsc_w_dw(zp, radx[kz - 1], radx[kz], radx[kz + 1], dx, wz, dwz);
    const float* g = gfield + (size_t)b * G;
    float ax = 0.f, ay = 0.f, az = 0.f, am = 0.f;
#pragma unroll
    for (int kk = -1; kk <= 1; kk++) {
      int k1 = kz + kk;
      if (k1 == nx + 1) k1 = 1;
      if (k1 == 0) k1 = nx;
#pragma unroll
      for (int jj = -1; jj <= 1; jj++) {
        int j1 = jy + jj;
        if (j1 == nx + 1) j1 = 1;
        if (j1 == 0) j1 = nx;
#pragma unroll
        for (int ii = -1; ii <= 1; ii++) {
          int i1 = ix + ii;
          if (i1 == nx + 1) i1 = 1;
          if (i1 == 0) i1 = nx;
          float gv = g[((size_t)(k1 - 1) * nx + (j1 - 1)) * nx + (i1 - 1)];
          ax += dwx[ii + 1] * wy[jj + 1] * wz[kk + 1] * gv;
          ay += wx[ii + 1] * dwy[jj + 1] * wz[kk + 1] * gv;
          az += wx[ii + 1] * wy[jj + 1] * dwz[kk + 1] * gv;
          am += wx[ii + 1] * wy[jj + 1] * wz[kk + 1] * gv;
        }
      }
    }
    float mp = m[q] * inv_denbas;
    gx[q] = mp * ax;
    gy[q] = mp * ay;
    gz[q] = mp * az;
    if (gm) gm[q] = am * inv_denbas;
  }
}

__global__ void k_layer_adjoint(const uint32_t* __restrict__ keys, const int32_t* __restrict__ idx,
                                const float4* __restrict__ pm, int64_t ntot, int nx, int cbits, float xl,
                                float dx, const float* __restrict__ radx, const float* __restrict__ gfield,
                                float inv_denbas, float* __restrict__ gx, float* __restrict__ gy,
                                float* __restrict__ gz, float* __restrict__ gm) {
  const size_t G = (size_t)nx * nx * nx;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ntot;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t q = idx[i];
    const float4 p = pm[q];
    const int ix = tsc_cell(p.x, xl, dx, nx), jy = tsc_cell(p.y, xl, dx, nx), kz = tsc_cell(p.z, xl, dx, nx);
    float wx[3], wy[3], wz[3], dwx[3], dwy[3], dwz[3];
    tsc_w_dw(p.x, radx[ix - 1], radx[ix], radx[ix + 1], dx, wx, dwx);
    tsc_w_dw(p.y, radx[jy - 1], radx[jy], radx[jy + 1], dx, wy, dwy);
    tsc_w_dw(p.z, radx[kz - 1], radx[kz], radx[kz + 1], dx, wz, dwz);
    const float* g = gfield + (size_t)(keys[i] >> cbits) * G;
    float ax = 0.f, ay = 0.f, az = 0.f, am = 0.f;
#pragma unroll
    for (int kk = -1; kk <= 1; kk++) {
      int k1 = kz + kk;
      if (k1 == nx + 1) k1 = 1;
      if (k1 == 0) k1 = nx;
#pragma unroll
      for (int jj = -1; jj <= 1; jj++) {
        int j1 = jy + jj;
        if (j1 == nx + 1) j1 = 1;
        if (j1 == 0) j1 = nx;
#pragma unroll
        for (int ii = -1; ii <= 1; ii++) {
          int i1 = ix + ii;
          if (i1 == nx + 1) i1 = 1;
          if (i1 == 0) i1 = nx;
          float gv = g[((size_t)(k1 - 1) * nx + (j1 - 1)) * nx + (i1 - 1)];
          ax += dwx[ii + 1] * wy[jj + 1] * wz[kk + 1] * gv;
          ay += wx[ii + 1] * dwy[jj + 1] * wz[kk + 1] * gv;
          az += wx[ii + 1] * wy[jj + 1] * dwz[kk + 1] * gv;
          am += wx[ii + 1] * wy[jj + 1] * wz[kk + 1] * gv;
        }
      }
    }
    const float mp = p.w * inv_denbas;
    gx[q] = mp * ax;
    gy[q] = mp * ay;
    gz[q] = mp * az;
    if (gm) gm[q] = am * inv_denbas;
  }
}

extern "C" int asohf_tsc_poisson_adjoint(asohf_ctx* c, int nx, float lado0, float dx,
                                         const float* radx, float rote, float rete, int batch,
                                         int64_t n_per, const float* x, const float* y,
                                         const float* z, const float* m, const float* w,
                                         float* grad_x, float* grad_y, float* grad_z, float* grad_m) {
  if (!c || nx < 2 || batch < 1 || !radx || !w || !grad_x || !grad_y || !grad_z) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  int64_t g = (int64_t)nx * nx * nx * batch;
  int64_t ntot = n_per * batch;
  const bool sorted = ntot > 0 && layer_sortable(nx, batch, ntot);
  ASOHF_CHECK(arena_reserve(c, poisson_bytes(nx, batch) + 4 * g + (sorted ? layer_sort_bytes(nx, batch, ntot) : 0) +
                                   2048));
  const float* dradx;
  ASOHF_CHECK(radx_device(c, nx, radx, &dradx));
  float* gfield = (float*)arena_alloc(c, 4 * g);
  if (!gfield) return ASOHF_ERR_CAPACITY;
  float denbas = dx * dx * dx * rote * (rete * rete * rete);
  const float xl = -lado0 / 2.0f;
  LayerSort s;
  if (sorted) ASOHF_CHECK(layer_sort(c, nx, xl, dx, batch, n_per, x, y, z, m, &s));
  // the Green's operator is real and symmetric: its adjoint is itself
  ASOHF_CHECK(poisson_dev(c, nx, dx, batch, w, gfield));
  if (sorted) {
    int kt_ = ktime_begin(c, "layer_adjoint");
    k_layer_adjoint<<<grid_for(ntot, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        s.keys, s.idx, s.pm, ntot, nx, s.cbits, xl, dx, dradx, gfield, 1.0f / denbas, grad_x, grad_y, grad_z, grad_m);
    ktime_end(c, kt_);
    c->launches++;
  } else if (ntot > 0) {
    {
      int kt_ = ktime_begin(c, "tsc_adjoint_gather");
      k_tsc_adjoint<<<grid_for(ntot, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        x, y, z, m, n_per, batch, nx, -lado0 / 2.0f, dx, dradx, gfield, 1.0f / denbas, grad_x, grad_y,
        grad_z, grad_m);
      ktime_end(c, kt_);
    }
    c->launches++;
  }
  ASOHF_CUDA(cudaGetLastError());
  return ASOHF_OK;  // device outputs: enqueued on the context stream
}
