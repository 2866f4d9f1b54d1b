// sortx.cu -- SORT_DM_PARTICLES_X (grids.f:2726-2838) and the column index.
//
// ARGSORT (num.f:150-203) is a bottom-up merge sort that takes the element
// of the right run on equal keys.  Every pair of equal keys is compared at
// the merge where their runs first meet, with the higher index in the right
// run, so its output is the sort by (key ascending, index DESCENDING).  A
// stable radix sort fed the keys in reverse index order yields exactly that.
// Keys compare as REAL*4 .LT., under which -0.0 and +0.0 are equal: both map
// to the same radix key.
//
// The column index groups the x-sorted store by (y, z) columns of one base
// cell, keeping x order inside each column, so a sphere or cube query reads
// only the columns it overlaps and, inside each, a binary-searched x range.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"

int permute_store(asohf_ctx* c, const int64_t* perm);

__device__ __forceinline__ uint32_t float_key(float f) {
  uint32_t u = __float_as_uint(f);
  if (u == 0x80000000u) u = 0u;  // -0.0 == +0.0
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void k_xkeys_reversed(const float* __restrict__ x, int64_t n, uint32_t* __restrict__ key,
                                 int32_t* __restrict__ val) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    int64_t i = n - 1 - j;
    key[j] = float_key(x[i]);
    val[j] = (int32_t)i;
  }
}

__global__ void k_widen(const int32_t* __restrict__ a, int64_t n, int64_t* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = a[i];
}

// NDMPART_X(ix) = number of particles with x <= RADXR(ix), RADXR(ix) =
// XL + ix*DX with XL=-LADO0/2, DX=LADO0/NX (grids.f:2790-2813); NDMPART_X(0)=0.
__global__ void k_ndmpart_x(const float* __restrict__ xs, int64_t n, int nx, float xl, float dxl,
                            int32_t* __restrict__ nd) {
  int ix = blockIdx.x * blockDim.x + threadIdx.x;
  if (ix > nx) return;
  if (ix == 0) { nd[0] = 0; return; }
  float r = xl + (float)ix * dxl;
  int64_t lo = 0, hi = n;  // first index with x > r
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (xs[mid] > r) hi = mid; else lo = mid + 1;
  }
  nd[ix] = (int32_t)lo;
}

__device__ __forceinline__ int col_of(float v, float xl, float cdx, int ncol) {
  int b = (int)floorf((v - xl) / cdx);
  return b < 0 ? 0 : (b >= ncol ? ncol - 1 : b);
}

__global__ void k_colkeys(const float* __restrict__ y, const float* __restrict__ z, int64_t n,
                          float xl, float cdx, int ncol, uint32_t* __restrict__ key,
                          int32_t* __restrict__ val) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    key[i] = (uint32_t)(col_of(z[i], xl, cdx, ncol) * ncol + col_of(y[i], xl, cdx, ncol));
    val[i] = (int32_t)i;
  }
}

__global__ void k_colfill(const int32_t* __restrict__ order, const uint32_t* __restrict__ keys, int64_t n,
                          const float* __restrict__ x, const float* __restrict__ y,
                          const float* __restrict__ z, const float4* __restrict__ rows, float4* __restrict__ cp,
                          int64_t* __restrict__ colstart, int64_t ncols) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    int32_t p = order[q];
    if (rows) {
      const float4 r = rows[2 * (int64_t)p];
      cp[q] = make_float4(r.x, r.y, r.z, __int_as_float(p));
    } else {
      cp[q] = make_float4(x[p], y[p], z[p], __int_as_float(p));
    }
    uint32_t k = keys[q];
    uint32_t kp = q > 0 ? keys[q - 1] : 0xffffffffu;
    if (q == 0) {
      for (uint32_t c = 0; c <= k; c++) colstart[c] = 0;
    } else if (k != kp) {
      for (uint32_t c = kp + 1; c <= k; c++) colstart[c] = q;
    }
    if (q == n - 1)
      for (int64_t c = (int64_t)k + 1; c <= ncols; c++) colstart[c] = n;
  }
}

int build_column_index(asohf_ctx* c, int nx, float lado0) {
  int64_t n = c->p.n;
  int ncol = nx;
  int64_t ncols = (int64_t)ncol * ncol;
  if (c->colpart_cap < n) {
    cudaFree(c->d_colpart);
    c->d_colpart = nullptr;
    ASOHF_CUDA(cudaMalloc(&c->d_colpart, sizeof(float4) * (size_t)(n > 0 ? n : 1)));
    c->colpart_cap = n;
  }
  if (c->ncols != ncols || !c->d_colstart) {
    cudaFree(c->d_colstart);
    ASOHF_CUDA(cudaMalloc(&c->d_colstart, sizeof(int64_t) * (size_t)(ncols + 1)));
    c->ncols = ncols;
  }
  c->col_n = ncol;
  c->col_xl = -lado0 / 2.0f;
  c->col_dx = lado0 / (float)ncol;
  if (n == 0) {
    ASOHF_CUDA(cudaMemsetAsync(c->d_colstart, 0, sizeof(int64_t) * (size_t)(ncols + 1), c->stream));
    return ASOHF_OK;
  }
  int bits = 1;
  while ((1ll << bits) < ncols) bits++;
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint32_t*)nullptr, (uint32_t*)nullptr, (int32_t*)nullptr,
                                  (int32_t*)nullptr, (int)n, 0, bits);
  uint32_t* k0 = (uint32_t*)arena_alloc(c, 4 * n);
  uint32_t* k1 = (uint32_t*)arena_alloc(c, 4 * n);
  int32_t* v0 = (int32_t*)arena_alloc(c, 4 * n);
  int32_t* v1 = (int32_t*)arena_alloc(c, 4 * n);
  void* t = arena_alloc(c, tb);
  if (!k0 || !k1 || !v0 || !v1 || !t) return ASOHF_ERR_CAPACITY;
  {
    int kt_ = ktime_begin(c, "column_index_keys");
    k_colkeys<<<grid_for(n, 256), 256, 0, c->stream>>>(c->p.y, c->p.z, n, c->col_xl, c->col_dx, ncol, k0, v0);
    ktime_end(c, kt_);
  }
  int kt_ = ktime_begin(c, "column_index_radix");
  ASOHF_CUDA(cub::DeviceRadixSort::SortPairs(t, tb, k0, k1, v0, v1, (int)n, 0, bits, c->stream));
  ktime_end(c, kt_);
  {
    int kt_ = ktime_begin(c, "column_index_fill");
    k_colfill<<<grid_for(n, 256), 256, 0, c->stream>>>(
        v1, k1, n, c->p.x, c->p.y, c->p.z, c->rows_cur >= 0 ? c->rows[c->rows_cur] : nullptr, c->d_colpart,
        c->d_colstart, ncols);
    ktime_end(c, kt_);
  }
  c->launches += 2;
  ASOHF_CUDA(cudaGetLastError());
  return ASOHF_OK;
}

size_t column_index_bytes(int64_t n, int nx) {
  int64_t ncols = (int64_t)nx * nx;
  int bits = 1;
  while ((1ll << bits) < ncols) bits++;
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint32_t*)nullptr, (uint32_t*)nullptr, (int32_t*)nullptr,
                                  (int32_t*)nullptr, (int)n, 0, bits);
  return 16 * (size_t)n + tb + 4096;
}

extern "C" int asohf_sort_dm_particles_x(asohf_ctx* c, int nx, float lado0, int32_t* ndmpart_x) {
  if (!c || nx <= 0 || !ndmpart_x) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  int64_t n = c->p.n;
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint32_t*)nullptr, (uint32_t*)nullptr, (int32_t*)nullptr,
                                  (int32_t*)nullptr, (int)n);
  size_t need = 16 * (size_t)n + 8 * (size_t)n + tb + 4096;
  size_t need2 = column_index_bytes(n, nx);
  ASOHF_CHECK(arena_reserve(c, need > need2 ? need : need2));
  if (!c->d_ndmpart_x || c->ndmpart_cap < nx + 1) {  // grows only (cudaFree waits for the whole device)
    cudaFree(c->d_ndmpart_x);
    c->d_ndmpart_x = nullptr;
    c->ndmpart_cap = 0;
    ASOHF_CUDA(cudaMalloc(&c->d_ndmpart_x, sizeof(int32_t) * (size_t)(nx + 1)));
    c->ndmpart_cap = nx + 1;
  }
  if (n > 0) {
    uint32_t* k0 = (uint32_t*)arena_alloc(c, 4 * n);
    uint32_t* k1 = (uint32_t*)arena_alloc(c, 4 * n);
    int32_t* v0 = (int32_t*)arena_alloc(c, 4 * n);
    int32_t* v1 = (int32_t*)arena_alloc(c, 4 * n);
    int64_t* perm = (int64_t*)arena_alloc(c, 8 * n);
    void* t = arena_alloc(c, tb);
    if (!k0 || !k1 || !v0 || !v1 || !perm || !t) return ASOHF_ERR_CAPACITY;
    int kt_ = ktime_begin(c, "sort_x_keys");
    k_xkeys_reversed<<<grid_for(n, 256), 256, 0, c->stream>>>(c->p.x, n, k0, v0);
    ktime_end(c, kt_);
    kt_ = ktime_begin(c, "sort_x_radix");
    ASOHF_CUDA(cub::DeviceRadixSort::SortPairs(t, tb, k0, k1, v0, v1, (int)n, 0, 32, c->stream));
    ktime_end(c, kt_);
    kt_ = ktime_begin(c, "sort_x_widen");
    k_widen<<<grid_for(n, 256), 256, 0, c->stream>>>(v1, n, perm);
    ktime_end(c, kt_);
    c->launches += 2;
    ASOHF_CHECK(permute_store(c, perm));
  }
  float xl = -lado0 / 2.0f;
  float dxl = lado0 / (float)nx;
  {
    int kt_ = ktime_begin(c, "ndmpart_x");
    k_ndmpart_x<<<(nx + 1 + 255) / 256, 256, 0, c->stream>>>(c->p.x, n, nx, xl, dxl, c->d_ndmpart_x);
    ktime_end(c, kt_);
  }
  c->launches++;
  ASOHF_CUDA(cudaGetLastError());
  arena_reset(c);
  ASOHF_CHECK(build_column_index(c, nx, lado0));
  ASOHF_CUDA(cudaMemcpyAsync(ndmpart_x, c->d_ndmpart_x, sizeof(int32_t) * (size_t)(nx + 1),
                             cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  c->nx_sorted = nx;
  return ASOHF_OK;
}
