// deposit.cu -- species sort, kernel deposit (DENSITY), RENORM_DENSITY and
// the true-TSC deposit (INTERPOLATE_DENSITY_TSC) on sm_100a.
//
// Accumulation: every cloud term keeps the reference's REAL*4 expression
// (BAS*W(i)*W(j)*W(k), left to right).  Terms are summed in float64 and
// rounded once to float32, so the result depends on the particle order only
// through float64 rounding, unlike the reference's REDUCTION(+:U1)
// (grids.f:787-791) whose float32 sum does.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"

#define KW (2 * ASOHF_NMAX_KERNELS + 1)

// ------------------------------------------------------------ host tables
// COMPUTE_KERNELS (grids.f:997-1067), host side, same REAL*4 arithmetic.
static void compute_kernels_host(int nl, int deg, float* k /* (NLEVELS+1)*KW */) {
  memset(k, 0, sizeof(float) * KW * (ASOHF_NLEVELS + 1));
  for (int ir = 0; ir <= nl; ir++) {
    int n = 1 << ir;
    float h32 = (float)n + 0.5f;
    float h = 2.0f * h32 / 3.0f;
    float* kk = k + (size_t)ir * KW + ASOHF_NMAX_KERNELS;
    for (int i = -n; i <= n; i++) {
      if (deg == 2) {
        float bas = (float)abs(i) / h;
        if (bas <= 0.5f) {
          kk[i] = 0.75f - bas * bas;
        } else {
          float t = 1.5f - bas;
          kk[i] = 0.5f * (t * t);
        }
      } else {
        float bas = (float)abs(i) / h32;
        kk[i] = 1.0f - bas;
      }
    }
    float bas = 0.0f;
    for (int i = -n; i <= n; i++)
      for (int j = -n; j <= n; j++)
        for (int q = -n; q <= n; q++) {
          volatile float t = kk[i] * kk[j];  // keep two roundings on the host too
          t = t * kk[q];
          bas = bas + t;
        }
    bas = 1.0f / powf(bas, 1.0f / 3.0f);
    for (int i = -n; i <= n; i++) kk[i] = bas * kk[i];
  }
}

// ------------------------------------------------------------ species sort
__device__ __forceinline__ int ngp_index(float v, float xmin, float dx, int nx) {
  int i = (int)((v - xmin) / dx) + 1;
  if (i < 1) i = 1;
  if (i > nx) i = nx;
  return i - 1;
}

__global__ void k_ngp_count(const float* __restrict__ x, const float* __restrict__ y,
                            const float* __restrict__ z, int64_t n, int nx, float dx, float xmin,
                            int32_t* __restrict__ cell, int32_t* __restrict__ counts) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int ix = ngp_index(x[i], xmin, dx, nx), jy = ngp_index(y[i], xmin, dx, nx),
        kz = ngp_index(z[i], xmin, dx, nx);
    int c = (kz * nx + jy) * nx + ix;
    cell[i] = c;
    atomicAdd(&counts[c], 1);
  }
}

// dens(cell) for equal masses: the float32 running sum of `count` copies of
// m, as the sequential loop of reader.f:190-201 produces it, divided by bas.
__global__ void k_cell_density_eqmass(const int32_t* __restrict__ counts, int64_t g, float m,
                                      float bas, float* __restrict__ dens) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < g;
       c += (int64_t)gridDim.x * blockDim.x) {
    int k = counts[c];
    float s = 0.0f;
    for (int q = 0; q < k; q++) s = __fadd_rn(s, m);
    dens[c] = s / bas;
  }
}

// General masses: the particles of a cell in input order (stable sort).
__global__ void k_cell_density_general(const int32_t* __restrict__ offs, const int32_t* __restrict__ order,
                                       const float* __restrict__ m, int64_t g, float bas,
                                       float* __restrict__ dens) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < g;
       c += (int64_t)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int q = offs[c]; q < offs[c + 1]; q++) s = __fadd_rn(s, m[order[q]]);
    dens[c] = s / bas;
  }
}

__global__ void k_species(const int32_t* __restrict__ cell, const float* __restrict__ dens,
                          int64_t n, int n_esp, float log8, uint8_t* __restrict__ spec) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float b = dens[cell[i]];
    int l = 0;
    if (b > 0.0f) {
      // LOG of a REAL*4 rounded to float32 (correctly rounded), then the
      // REAL*4 quotient by LOG(8.0) and INT truncation.
      float lb = (float)log((double)b);
      l = (int)(lb / log8);
      if (l > n_esp - 1) l = n_esp - 1;
      if (l < 0) l = 0;
    }
    spec[i] = (uint8_t)l;
  }
}

#define SPEC_CHUNK 4096
#define SPEC_BLOCK 256

__global__ void k_species_block_counts(const uint8_t* __restrict__ spec, int64_t n, int nb,
                                       int32_t* __restrict__ bc) {
  __shared__ int cnt[ASOHF_N_ESP];
  if (threadIdx.x < ASOHF_N_ESP) cnt[threadIdx.x] = 0;
  __syncthreads();
  int64_t lo = (int64_t)blockIdx.x * SPEC_CHUNK, hi = min(lo + SPEC_CHUNK, n);
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) atomicAdd(&cnt[spec[i]], 1);
  __syncthreads();
  if (threadIdx.x < ASOHF_N_ESP) bc[(int64_t)threadIdx.x * nb + blockIdx.x] = cnt[threadIdx.x];
}

// Stable scatter: perm[dst] = i, dst = offset(species, block) + rank in block.
__global__ void k_species_scatter(const uint8_t* __restrict__ spec, int64_t n, int nb,
                                  const int32_t* __restrict__ boff, int64_t* __restrict__ perm) {
  __shared__ int wcnt[SPEC_BLOCK / 32][ASOHF_N_ESP];
  __shared__ int run[ASOHF_N_ESP];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x < ASOHF_N_ESP) run[threadIdx.x] = boff[(int64_t)threadIdx.x * nb + blockIdx.x];
  __syncthreads();
  int64_t lo = (int64_t)blockIdx.x * SPEC_CHUNK, hi = min(lo + SPEC_CHUNK, n);
  for (int64_t base = lo; base < hi; base += SPEC_BLOCK) {
    int64_t i = base + threadIdx.x;
    int s = i < hi ? spec[i] : -1;
    int myrank = 0;
    for (int q = 0; q < ASOHF_N_ESP; q++) {
      unsigned msk = __ballot_sync(0xffffffffu, s == q);
      if (s == q) myrank = __popc(msk & ((1u << lane) - 1));
      if (lane == 0) wcnt[wid][q] = __popc(msk);
    }
    __syncthreads();
    if (s >= 0) {
      int off = run[s];
      for (int w = 0; w < wid; w++) off += wcnt[w][s];
      perm[off + myrank] = i;
    }
    __syncthreads();
    if (threadIdx.x < ASOHF_N_ESP) {
      int t = 0;
      for (int w = 0; w < SPEC_BLOCK / 32; w++) t += wcnt[w][threadIdx.x];
      run[threadIdx.x] += t;
    }
    __syncthreads();
  }
}

// Store permutation in two passes: the store is packed row-wise (one
// 32-byte row per particle, read and written in order), then each output
// particle reads its whole source row with one random 32-byte access; a
// gather straight from the eight arrays would touch eight sectors per
// particle.
__global__ void k_pack_rows(int64_t n, DevParticles s, float4* __restrict__ rows) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    rows[2 * i] = make_float4(s.x[i], s.y[i], s.z[i], s.m[i]);
    rows[2 * i + 1] = make_float4(s.vx[i], s.vy[i], s.vz[i], __int_as_float(s.id[i]));
  }
}

// New store (fields and rows) in the order perm gives: d[i] = old[perm[i]].
// Four particles per thread and step: their rows are all requested before
// any is written.
__global__ void k_gather_rows(const int64_t* __restrict__ perm, int64_t n, const float4* __restrict__ rows,
                              DevParticles d, float4* __restrict__ out_rows) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i0 < n; i0 += 4 * stride) {
    int64_t j[4];
    float4 a[4], b[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int64_t i = i0 + u * stride;
      j[u] = i < n ? perm[i] : 0;
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (i0 + u * stride < n) {
        a[u] = rows[2 * j[u]];
        b[u] = rows[2 * j[u] + 1];
      }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int64_t i = i0 + u * stride;
      if (i < n) {
        d.x[i] = a[u].x; d.y[i] = a[u].y; d.z[i] = a[u].z; d.m[i] = a[u].w;
        d.vx[i] = b[u].x; d.vy[i] = b[u].y; d.vz[i] = b[u].z; d.id[i] = __float_as_int(b[u].w);
        out_rows[2 * i] = a[u];
        out_rows[2 * i + 1] = b[u];
      }
    }
  }
}

__global__ void k_iota(int32_t* __restrict__ a, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] = (int32_t)i;
}

int permute_store(asohf_ctx* c, const int64_t* perm) {
  int64_t n = c->p.n;
  if (c->rows_cap < n) {
    ASOHF_CUDA(cudaStreamSynchronize(c->stream));
    cudaFree(c->rows[0]);
    cudaFree(c->rows[1]);
    c->rows[0] = c->rows[1] = nullptr;
    c->rows_cap = 0;
    c->rows_cur = -1;
    ASOHF_CUDA(cudaMalloc(&c->rows[0], 32 * (size_t)(n > 0 ? n : 1)));
    ASOHF_CUDA(cudaMalloc(&c->rows[1], 32 * (size_t)(n > 0 ? n : 1)));
    c->rows_cap = n;
  }
  {
    int kt_ = ktime_begin(c, "store_permute");
    int src = c->rows_cur;
    if (src < 0) {  // no row copy of the current order yet
      src = 0;
      k_pack_rows<<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(n, c->p, c->rows[0]);
      c->launches++;
    }
    k_gather_rows<<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(perm, n, c->rows[src], c->alt,
                                                                          c->rows[1 - src]);
    c->rows_cur = 1 - src;
    ktime_end(c, kt_);
  }
  c->launches++;
  ASOHF_CUDA(cudaGetLastError());
  ctx_swap_particles(c);
  return ASOHF_OK;
}

extern "C" int asohf_sort_dm_particles_localdensity(asohf_ctx* c, int nx, float dx, float rodo,
                                                    float re0, int32_t* npart_esp) {
  if (!c || nx <= 0 || !npart_esp) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  int64_t n = c->p.n;
  int64_t g = (int64_t)nx * nx * nx;
  int nb = (int)((n + SPEC_CHUNK - 1) / SPEC_CHUNK);
  if (nb < 1) nb = 1;
  bool eq = (c->mmin == c->norma);
  size_t cub_bytes = 0;
  if (!eq) {
    cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (int32_t*)nullptr, (int32_t*)nullptr,
                                    (int32_t*)nullptr, (int32_t*)nullptr, (int)n);
  }
  size_t cub_scan = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cub_scan, (int32_t*)nullptr, (int32_t*)nullptr,
                                (int)(nb * ASOHF_N_ESP));
  size_t cub_scan2 = 0;
  if (!eq) cub::DeviceScan::ExclusiveSum(nullptr, cub_scan2, (int32_t*)nullptr, (int32_t*)nullptr, (int)(g + 1));
  size_t need = 4 * n + 4 * g + 4 * g + n + 4 * (size_t)nb * ASOHF_N_ESP * 2 + 8 * n +
                (eq ? 0 : (16 * n + 4 * (g + 1) * 2 + cub_bytes + cub_scan2)) + cub_scan + 8192;
  ASOHF_CHECK(arena_reserve(c, need));
  int32_t* cell = (int32_t*)arena_alloc(c, 4 * n);
  int32_t* counts = (int32_t*)arena_alloc(c, 4 * g);
  float* dens = (float*)arena_alloc(c, 4 * g);
  uint8_t* spec = (uint8_t*)arena_alloc(c, n + 16);
  int32_t* bc = (int32_t*)arena_alloc(c, 4 * (size_t)nb * ASOHF_N_ESP);
  int32_t* boff = (int32_t*)arena_alloc(c, 4 * (size_t)nb * ASOHF_N_ESP);
  int64_t* perm = (int64_t*)arena_alloc(c, 8 * n);
  void* tscan = arena_alloc(c, cub_scan);
  ASOHF_CUDA(cudaMemsetAsync(counts, 0, 4 * g, c->stream));
  float xmin = -((float)nx * dx) / 2.0f;
  {
    int kt_ = ktime_begin(c, "species_ngp_count");
    k_ngp_count<<<grid_for(n, 256), 256, 0, c->stream>>>(c->p.x, c->p.y, c->p.z, n, nx, dx, xmin,
                                                       cell, counts);
    ktime_end(c, kt_);
  }
  c->launches++;
  float bas = dx * dx * dx * rodo * (re0 * re0 * re0);
  if (eq) {
    {
      int kt_ = ktime_begin(c, "species_cell_density");
      k_cell_density_eqmass<<<grid_for(g, 256), 256, 0, c->stream>>>(counts, g, c->norma, bas, dens);
      ktime_end(c, kt_);
    }
    c->launches++;
  } else {
    // particles of each cell in input order: stable radix sort of (cell, i)
    int32_t* idx = (int32_t*)arena_alloc(c, 4 * n);
    int32_t* cell_s = (int32_t*)arena_alloc(c, 4 * n);
    int32_t* order = (int32_t*)arena_alloc(c, 4 * n);
    int32_t* offs = (int32_t*)arena_alloc(c, 4 * (g + 1));
    int32_t* cnt1 = (int32_t*)arena_alloc(c, 4 * (g + 1));
    void* tsort = arena_alloc(c, cub_bytes);
    void* tscan2 = arena_alloc(c, cub_scan2);
    if (!idx || !cell_s || !order || !offs || !cnt1 || !tsort || !tscan2) return ASOHF_ERR_CAPACITY;
    k_iota<<<grid_for(n, 256), 256, 0, c->stream>>>(idx, n);
    ASOHF_CUDA(cub::DeviceRadixSort::SortPairs(tsort, cub_bytes, cell, cell_s, idx, order, (int)n, 0,
                                               32, c->stream));
    ASOHF_CUDA(cudaMemsetAsync(cnt1 + g, 0, 4, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(cnt1, counts, 4 * g, cudaMemcpyDeviceToDevice, c->stream));
    ASOHF_CUDA(cub::DeviceScan::ExclusiveSum(tscan2, cub_scan2, cnt1, offs, (int)(g + 1), c->stream));
    k_cell_density_general<<<grid_for(g, 256), 256, 0, c->stream>>>(offs, order, c->p.m, g, bas, dens);
    c->launches += 2;
  }
  {
    int kt_ = ktime_begin(c, "species_classify");
    k_species<<<grid_for(n, 256), 256, 0, c->stream>>>(cell, dens, n, ASOHF_N_ESP, logf(8.0f), spec);
    k_species_block_counts<<<nb, SPEC_BLOCK, 0, c->stream>>>(spec, n, nb, bc);
    ASOHF_CUDA(cub::DeviceScan::ExclusiveSum(tscan, cub_scan, bc, boff, nb * ASOHF_N_ESP, c->stream));
    ktime_end(c, kt_);
  }
  {
    int kt_ = ktime_begin(c, "species_scatter");
    k_species_scatter<<<nb, SPEC_BLOCK, 0, c->stream>>>(spec, n, nb, boff, perm);
    ktime_end(c, kt_);
  }
  c->launches += 4;
  ASOHF_CUDA(cudaGetLastError());
  int32_t tot[ASOHF_N_ESP];
  int32_t last_off[ASOHF_N_ESP], last_cnt[ASOHF_N_ESP];
  for (int s = 0; s < ASOHF_N_ESP; s++) {
    ASOHF_CUDA(cudaMemcpyAsync(&last_off[s], boff + (int64_t)s * nb + nb - 1, 4, cudaMemcpyDeviceToHost, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(&last_cnt[s], bc + (int64_t)s * nb + nb - 1, 4, cudaMemcpyDeviceToHost, c->stream));
  }
  ASOHF_CHECK(permute_store(c, perm));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  int64_t prev = 0;
  for (int s = 0; s < ASOHF_N_ESP; s++) {
    int64_t end = (int64_t)last_off[s] + last_cnt[s];
    tot[s] = (int32_t)(end - prev);
    prev = end;
  }
  if (prev != n) return ASOHF_ERR_WRONG_SORTING;
  memcpy(npart_esp, tot, sizeof(tot));
  return ASOHF_OK;
}

// ------------------------------------------------------------ base deposit
// The 27-cell periodic cloud of grids.f:787-820 for particles whose host
// cell lies in the box; BASE_OUTLIER handles the rest (positions more than
// one cell outside the box), with the same wrap-once arithmetic.
__device__ __forceinline__ int wrap_once(int i, int nx) {
  if (i > nx) i -= nx;
  if (i < 1) i += nx;
  return i;
}

// Particles whose host cell lies outside the box, summed into the float64
// grid the tile kernel wrote.
__global__ void k_density_base_outliers(const float* __restrict__ x, const float* __restrict__ y,
                                        const float* __restrict__ z, const float* __restrict__ m, int64_t n,
                                        int nx, float xl, float dx, const float* __restrict__ k0,
                                        double* __restrict__ acc) {
  float w[3] = {k0[0], k0[1], k0[2]};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int ix = (int)((x[i] - xl) / dx) + 1;
    int jy = (int)((y[i] - xl) / dx) + 1;
    int kz = (int)((z[i] - xl) / dx) + 1;
    if (ix >= 1 && ix <= nx && jy >= 1 && jy <= nx && kz >= 1 && kz <= nx) continue;
    float bas = m[i];
    for (int kk = -1; kk <= 1; kk++)
      for (int jj = -1; jj <= 1; jj++)
        for (int ii = -1; ii <= 1; ii++) {
          int i1 = wrap_once(ix + ii, nx), j1 = wrap_once(jy + jj, nx), k1 = wrap_once(kz + kk, nx);
          if (i1 < 1 || i1 > nx || j1 < 1 || j1 > nx || k1 < 1 || k1 > nx) continue;  // outside the box
          float t = __fmul_rn(__fmul_rn(__fmul_rn(bas, w[ii + 1]), w[jj + 1]), w[kk + 1]);
          atomicAdd(&acc[((size_t)(k1 - 1) * nx + (j1 - 1)) * nx + (i1 - 1)], (double)t);
        }
  }
}

// Every particle with global float64 atomics (grids smaller than one tile).
__global__ void k_density_base_all(const float* __restrict__ x, const float* __restrict__ y,
                                   const float* __restrict__ z, const float* __restrict__ m, int64_t n, int nx,
                                   float xl, float dx, const float* __restrict__ k0, double* __restrict__ acc) {
  float w[3] = {k0[0], k0[1], k0[2]};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int ix = (int)((x[i] - xl) / dx) + 1;
    int jy = (int)((y[i] - xl) / dx) + 1;
    int kz = (int)((z[i] - xl) / dx) + 1;
    float bas = m[i];
    for (int kk = -1; kk <= 1; kk++)
      for (int jj = -1; jj <= 1; jj++)
        for (int ii = -1; ii <= 1; ii++) {
          int i1 = wrap_once(ix + ii, nx), j1 = wrap_once(jy + jj, nx), k1 = wrap_once(kz + kk, nx);
          if (i1 < 1 || i1 > nx || j1 < 1 || j1 > nx || k1 < 1 || k1 > nx) continue;  // outside the box
          float t = __fmul_rn(__fmul_rn(__fmul_rn(bas, w[ii + 1]), w[jj + 1]), w[kk + 1]);
          atomicAdd(&acc[((size_t)(k1 - 1) * nx + (j1 - 1)) * nx + (i1 - 1)], (double)t);
        }
  }
}

__global__ void k_finish_f64(const double* __restrict__ acc, int64_t g, float denbas,
                             float* __restrict__ u1) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < g;
       c += (int64_t)gridDim.x * blockDim.x)
    u1[c] = (float)acc[c] / denbas;
}

// ------------------------------------------------------------ spatial bins
// Coarse binning of the store (bins of `bw` base cells) so a patch finds the
// particles near it without scanning all N (the reference tests every
// particle against every patch, grids.f:879-893).
struct Bins {
  int nb;          // bins per axis
  float xl, bsz;   // origin and bin size
  int32_t* start;  // nb^3+1
  int32_t* idx;    // particle indices grouped by bin
};

__device__ __forceinline__ int bin_of(float v, float xl, float bsz, int nb) {
  int b = (int)floorf((v - xl) / bsz);
  return b < 0 ? 0 : (b >= nb ? nb - 1 : b);
}

// bin key and index of every particle, and the bin counts
__global__ void k_bin_keys(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
                           int64_t n, Bins B, uint32_t* __restrict__ keys, int32_t* __restrict__ vals,
                           int32_t* __restrict__ cnt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int b = (bin_of(z[i], B.xl, B.bsz, B.nb) * B.nb + bin_of(y[i], B.xl, B.bsz, B.nb)) * B.nb +
            bin_of(x[i], B.xl, B.bsz, B.nb);
    keys[i] = (uint32_t)b;
    vals[i] = (int32_t)i;
    atomicAdd(&cnt[b], 1);
  }
}

// Where a density buffer lives: the call's arena, or density pool 0 when
// the patch deposit is deferred (buffers the deferred kernels read).
struct DAlloc {
  asohf_ctx* c;
  bool pool;
  void* get(size_t bytes) const { return pool ? dpool_alloc(c, 0, bytes) : arena_alloc(c, bytes); }
};

// start[b] = first position of bin b (count and exclusive scan), idx = the
// particles grouped by bin (a stable radix sort of (bin, index): ascending
// index within a bin, the same grouping on every run).
static int bin_key_bits(int64_t nbin) {
  int bits = 1;
  while ((1ll << bits) < nbin) bits++;
  return bits;
}

static void bins_temp(int64_t n, int64_t nbin, size_t* scan_b, size_t* sort_b) {
  *scan_b = 0;
  *sort_b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, *scan_b, (int32_t*)nullptr, (int32_t*)nullptr, (int)(nbin + 1));
  cub::DeviceRadixSort::SortPairs(nullptr, *sort_b, (uint32_t*)nullptr, (uint32_t*)nullptr, (int32_t*)nullptr,
                                  (int32_t*)nullptr, (int)(n > 0 ? n : 1), 0, bin_key_bits(nbin));
}

static int build_bins(asohf_ctx* c, float lado0, float dx, int bw, Bins* B, DAlloc A = DAlloc{nullptr, false}) {
  int64_t n = c->p.n;
  int nx = (int)lrintf(lado0 / dx);
  int nb = (nx + bw - 1) / bw;
  if (nb < 1) nb = 1;
  int64_t nbin = (int64_t)nb * nb * nb;
  B->nb = nb;
  B->xl = -lado0 / 2.0f;
  B->bsz = lado0 / (float)nb;
  uint32_t* k0 = (uint32_t*)arena_alloc(c, 4 * n + 4);
  uint32_t* k1 = (uint32_t*)arena_alloc(c, 4 * n + 4);
  int32_t* v0 = (int32_t*)arena_alloc(c, 4 * n + 4);
  int32_t* cnt = (int32_t*)arena_alloc(c, 4 * (nbin + 1));
  B->start = (int32_t*)(A.pool ? A.get(4 * (nbin + 1)) : arena_alloc(c, 4 * (nbin + 1)));
  B->idx = (int32_t*)arena_alloc(c, 4 * n + 4);
  size_t ts, tr;
  bins_temp(n, nbin, &ts, &tr);
  void* t = arena_alloc(c, ts > tr ? ts : tr);
  if (!k0 || !k1 || !v0 || !cnt || !B->start || !B->idx || !t) return ASOHF_ERR_CAPACITY;
  int kt_ = ktime_begin(c, "particle_bins");
  ASOHF_CUDA(cudaMemsetAsync(cnt, 0, 4 * (nbin + 1), c->stream));
  k_bin_keys<<<grid_for(n, 256), 256, 0, c->stream>>>(c->p.x, c->p.y, c->p.z, n, *B, k0, v0, cnt);
  ASOHF_CUDA(cub::DeviceScan::ExclusiveSum(t, ts, cnt, B->start, (int)(nbin + 1), c->stream));
  if (n > 0)
    ASOHF_CUDA(cub::DeviceRadixSort::SortPairs(t, tr, k0, k1, v0, B->idx, (int)n, 0, bin_key_bits(nbin),
                                               c->stream));
  ktime_end(c, kt_);
  c->launches++;
  return ASOHF_OK;
}

static size_t bins_bytes(int64_t n, float lado0, float dx, int bw) {
  int nx = (int)lrintf(lado0 / dx);
  int nb = (nx + bw - 1) / bw;
  if (nb < 1) nb = 1;
  int64_t nbin = (int64_t)nb * nb * nb;
  size_t ts, tr;
  bins_temp(n, nbin, &ts, &tr);
  return 16 * (size_t)n + 8 * (size_t)(nbin + 1) + (ts > tr ? ts : tr) + 8192;
}

// Device copy of the patch table.
struct DevMesh {
  int np;
  int32_t *nx, *ny, *nz, *level;
  float *rx, *ry, *rz;
};

static int upload_mesh(asohf_ctx* c, const asohf_mesh* mh, DevMesh* d, DAlloc A = DAlloc{nullptr, false}) {
  int np = 0;
  for (int ir = 1; ir <= mh->nl; ir++) np += mh->npatch[ir];
  d->np = np;
  if (np == 0) return ASOHF_OK;
  int base = mh->npatch[0];
  for (int q = 0; q < np; q++) {
    int ip = base + q;
    if (mh->patchnx[ip] < 1 || mh->patchnx[ip] > ASOHF_NAMRX || mh->patchny[ip] < 1 || mh->patchny[ip] > ASOHF_NAMRX ||
        mh->patchnz[ip] < 1 || mh->patchnz[ip] > ASOHF_NAMRX)
      return ASOHF_ERR_INVALID;
  }
  std::vector<int32_t> hi_v(4 * (size_t)np);
  std::vector<float> hf_v(3 * (size_t)np);
  int32_t* hi = hi_v.data();
  float* hf = hf_v.data();
  int q = 0;
  for (int ir = 1; ir <= mh->nl; ir++)
    for (int p = 0; p < mh->npatch[ir]; p++, q++) {
      int ip = base + q;
      hi[q] = mh->patchnx[ip];
      hi[np + q] = mh->patchny[ip];
      hi[2 * np + q] = mh->patchnz[ip];
      hi[3 * np + q] = ir;
      hf[q] = mh->patchrx[ip];
      hf[np + q] = mh->patchry[ip];
      hf[2 * np + q] = mh->patchrz[ip];
    }
  int32_t* di = (int32_t*)(A.pool ? A.get(16 * (size_t)np) : arena_alloc(c, 16 * (size_t)np));
  float* df = (float*)(A.pool ? A.get(12 * (size_t)np) : arena_alloc(c, 12 * (size_t)np));
  if (!di || !df) return ASOHF_ERR_CAPACITY;
  cudaMemcpyAsync(di, hi, 16 * (size_t)np, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(df, hf, 12 * (size_t)np, cudaMemcpyHostToDevice, c->stream);
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  d->nx = di; d->ny = di + np; d->nz = di + 2 * np; d->level = di + 3 * np;
  d->rx = df; d->ry = df + np; d->rz = df + 2 * np;
  return ASOHF_OK;
}

// ------------------------------------------------------------ staging
// The store in bin order as float4 (x, y, z, m) plus the species index, so
// a patch reads its candidates as contiguous runs (one run per (y, z) row of
// bins).
#define NA ASOHF_NAMRX
#define ZH (NA / 2)
#define PD_BLOCK 512

__global__ void k_bin_stage(const int32_t* __restrict__ idx, int64_t n, int64_t ndep, const float* __restrict__ x,
                            const float* __restrict__ y, const float* __restrict__ z, const float* __restrict__ m,
                            const float4* __restrict__ rows, const int64_t* __restrict__ esp_end,
                            float4* __restrict__ P, uint8_t* __restrict__ S) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    int p = idx[t];
    P[t] = rows ? rows[2 * (int64_t)p] : make_float4(x[p], y[p], z[p], m[p]);
    int s = 0;
    while (s < ASOHF_N_ESP - 1 && (int64_t)p >= esp_end[s]) s++;
    S[t] = (int64_t)p < ndep ? (uint8_t)s : (uint8_t)255;  // 255: not deposited
  }
}

// ------------------------------------------------------------ base deposit, equal masses
// With one particle mass every particle of a host cell deposits the same
// 27 REAL*4 terms, so the grid is the 27-point stencil of the host-cell
// counts: U1(c) = sum_o count(c - o) * t_o, each product exact in float64.
__global__ void k_base_counts(const float* __restrict__ x, const float* __restrict__ y,
                              const float* __restrict__ z, int64_t n, int nx, float xl, float dx,
                              int32_t* __restrict__ cnt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int ix = (int)((x[i] - xl) / dx) + 1;
    int jy = (int)((y[i] - xl) / dx) + 1;
    int kz = (int)((z[i] - xl) / dx) + 1;
    if (ix >= 1 && ix <= nx && jy >= 1 && jy <= nx && kz >= 1 && kz <= nx)
      atomicAdd(&cnt[((int64_t)(kz - 1) * nx + (jy - 1)) * nx + (ix - 1)], 1);
  }
}

struct Terms27 {
  double t[27];  // t[(kk+1)*9 + (jj+1)*3 + (ii+1)] = ((m*W(ii))*W(jj))*W(kk) in REAL*4
};

// Symmetric level-0 kernel (W(-1) = W(1)): the 27 terms take 8 values
// t(|di|, |dj|, |dk|), so a cell needs the count sums of 8 neighbour
// patterns (integers) and 8 products.
__global__ void k_base_stencil_sym(const int32_t* __restrict__ cnt, int nx, Terms27 T, double* __restrict__ acc) {
  int64_t g = (int64_t)nx * nx * nx;
  double tp[8];
#pragma unroll
  for (int q = 0; q < 8; q++) tp[q] = T.t[((q >> 2) + 1) * 9 + (((q >> 1) & 1) + 1) * 3 + ((q & 1) + 1)];
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < g;
       c += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(c % nx) + 1, j = (int)((c / nx) % nx) + 1, k = (int)(c / ((int64_t)nx * nx)) + 1;
    const int im = wrap_once(i - 1, nx) - 1, ip = wrap_once(i + 1, nx) - 1;
    const int jm = wrap_once(j - 1, nx) - 1, jp = wrap_once(j + 1, nx) - 1;
    int a0[3], ax[3], ay[3], axy[3];
#pragma unroll
    for (int kk = -1; kk <= 1; kk++) {
      const int hk = wrap_once(k + kk, nx) - 1;
      const int32_t* pl = cnt + (int64_t)hk * nx * nx;
      const int32_t* r0 = pl + (int64_t)(j - 1) * nx;
      const int32_t* rm = pl + (int64_t)jm * nx;
      const int32_t* rp = pl + (int64_t)jp * nx;
      a0[kk + 1] = r0[i - 1];
      ax[kk + 1] = r0[im] + r0[ip];
      ay[kk + 1] = rm[i - 1] + rp[i - 1];
      axy[kk + 1] = (rm[im] + rm[ip]) + (rp[im] + rp[ip]);
    }
    const int c0 = a0[1], c1 = ax[1], c2 = ay[1], c3 = axy[1];
    const int c4 = a0[0] + a0[2], c5 = ax[0] + ax[2], c6 = ay[0] + ay[2], c7 = axy[0] + axy[2];
    double s = 0.0;
    if ((c0 | c1 | c2 | c3 | c4 | c5 | c6 | c7) != 0)
      s = (double)c0 * tp[0] + (double)c1 * tp[1] + (double)c2 * tp[2] + (double)c3 * tp[3] +
          (double)c4 * tp[4] + (double)c5 * tp[5] + (double)c6 * tp[6] + (double)c7 * tp[7];
    acc[c] = s;
  }
}

__global__ void k_base_stencil(const int32_t* __restrict__ cnt, int nx, Terms27 T, double* __restrict__ acc) {
  int64_t g = (int64_t)nx * nx * nx;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < g;
       c += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(c % nx) + 1, j = (int)((c / nx) % nx) + 1, k = (int)(c / ((int64_t)nx * nx)) + 1;
    double s = 0.0;
#pragma unroll
    for (int kk = -1; kk <= 1; kk++) {
      int hk = wrap_once(k - kk, nx);
#pragma unroll
      for (int jj = -1; jj <= 1; jj++) {
        int hj = wrap_once(j - jj, nx);
        const int32_t* row = cnt + ((int64_t)(hk - 1) * nx + (hj - 1)) * nx;
#pragma unroll
        for (int ii = -1; ii <= 1; ii++) {
          int hi = wrap_once(i - ii, nx);
          int q = row[hi - 1];
          if (q) s += (double)q * T.t[(kk + 1) * 9 + (jj + 1) * 3 + (ii + 1)];
        }
      }
    }
    acc[c] = s;
  }
}

// ------------------------------------------------------------ patch deposit
// Work unit: PZ z-planes of one patch, accumulated in float64 shared memory.
// A unit's candidates are the particles of the bins that overlap the patch
// box extended by MAXKERNELEXT = DX (grids.f:837-893), restricted in z to
// the unit's planes +- DX; they are split into slices of PSLICE so that a
// dense unit is shared by several CTAs, whose sums meet in a float64 scratch
// slab.  Inside a CTA all warps stride over the unit's candidates as one
// flat range.  A hit whose kernel level is 0 (27-cell cloud) is counted in
// a host-cell grid when all masses are equal and spread by the 27-point
// stencil at the end; every other hit deposits its clipped cloud with the
// 32 lanes of the warp, hits with the same host cell, level and mass once
// with the group size as factor.
#define PZ 4              // z planes per unit
#define PZ_BLOCK 256
#define NSLAB (NA / PZ)
#define PSLICE 8192       // candidates per work item
#define PROWS 128         // bin rows staged in shared memory at a time
#define CGX (NA + 2)      // host-cell count grid: x, y in [0, NA+1]
#define AROW (NA + 5)     // accumulator row stride (doubles): rows shifted by 5 banks pairs
#define APLANE (NA * AROW)
#define ACC_N (PZ * APLANE)
#define CGZ (PZ + 2)      //                       z in [zlo-1, zhi+1]

// Offset of the centre of level l in the compact kernel table that stores
// levels 0, 1, ... back to back (2*2^l+1 entries each).
__host__ __device__ __forceinline__ int ktab_center(int l) { return 3 * (1 << l) - 2 + l; }
__host__ __device__ __forceinline__ int ktab_size(int lmax) { return (1 << (lmax + 2)) - 1 + lmax; }

struct UnitGeo {
  int ip, slab, n1, n2, n3, ir, zlo, zhi;
  float dxpa, xlfix, ylfix, zlfix, pxl, pyl, pzl, pxr, pyr, pzr;
  int bx0, bx1, by0, by1, bz0, bz1, nby, rows;
};

__device__ __forceinline__ void unit_geo(const DevMesh& M, const Bins& B, const int32_t* order, int u, float dx,
                                         UnitGeo& g) {
  g.ip = order[u / NSLAB];
  g.slab = u % NSLAB;
  g.n1 = M.nx[g.ip]; g.n2 = M.ny[g.ip]; g.n3 = M.nz[g.ip]; g.ir = M.level[g.ip];
  g.zlo = g.slab * PZ + 1;
  g.zhi = min(g.slab * PZ + PZ, g.n3);
  g.dxpa = dx / exp2f((float)g.ir);
  g.xlfix = M.rx[g.ip] - g.dxpa; g.ylfix = M.ry[g.ip] - g.dxpa; g.zlfix = M.rz[g.ip] - g.dxpa;
  g.pxl = g.xlfix - dx; g.pyl = g.ylfix - dx; g.pzl = g.zlfix - dx;
  g.pxr = (g.xlfix + (float)g.n1 * g.dxpa) + dx;
  g.pyr = (g.ylfix + (float)g.n2 * g.dxpa) + dx;
  g.pzr = (g.zlfix + (float)g.n3 * g.dxpa) + dx;
  g.bx0 = bin_of(g.pxl, B.xl, B.bsz, B.nb); g.bx1 = bin_of(g.pxr, B.xl, B.bsz, B.nb);
  g.by0 = bin_of(g.pyl, B.xl, B.bsz, B.nb); g.by1 = bin_of(g.pyr, B.xl, B.bsz, B.nb);
  // a cloud reaches at most 2^ir cells = DX from its host cell: planes
  // zlo..zhi take hosts with z in [zlfix + (zlo-1) dxpa - DX, zlfix + zhi dxpa + DX]
  float za = fmaxf(g.pzl, (g.zlfix + (float)(g.zlo - 1) * g.dxpa) - dx);
  float zb = fminf(g.pzr, (g.zlfix + (float)g.zhi * g.dxpa) + dx);
  g.bz0 = bin_of(za, B.xl, B.bsz, B.nb); g.bz1 = bin_of(zb, B.xl, B.bsz, B.nb);
  g.nby = g.by1 - g.by0 + 1;
  g.rows = (g.zlo > g.zhi) ? 0 : g.nby * (g.bz1 - g.bz0 + 1);
}

__device__ __forceinline__ void row_range(const Bins& B, const UnitGeo& g, int row, int* lo, int* len) {
  int bz = g.bz0 + row / g.nby, by = g.by0 + row % g.nby;
  int64_t rb = ((int64_t)bz * B.nb + by) * B.nb;
  int a = B.start[rb + g.bx0], b = B.start[rb + g.bx1 + 1];
  *lo = a;
  *len = b - a;
}

// Candidates per unit (one warp per unit).
__global__ void k_patch_unit_counts(DevMesh M, Bins B, const int32_t* __restrict__ order, int nunits, float dx,
                                    int64_t* __restrict__ cnt) {
  int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (u >= nunits) return;
  UnitGeo g;
  unit_geo(M, B, order, u, dx, g);
  long long s = 0;
  for (int r = lane; r < g.rows; r += 32) {
    int lo, len;
    row_range(B, g, r, &lo, &len);
    s += len;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) cnt[u] = s;
}

struct PatchWork {
  const int2* items;         // (unit, slice)
  const int32_t* scratch_of; // per unit: scratch slab index, -1 for single-slice units
  double* scratch;           // NA*NA*PZ doubles per multi-slice unit
};

// One work item (a slice of one 4-plane unit of a patch) of the patch deposit.
__device__ __forceinline__ void density_patch_item(const int2 it, const DevMesh& M, const Bins& B,
                                                   const float4* __restrict__ P, const uint8_t* __restrict__ S,
                                                   const int32_t* __restrict__ order, const PatchWork& W, float dx,
                                                   const float* __restrict__ kernels, int eqmass,
                                                   float* __restrict__ u11, const float* __restrict__ denbas_lev) {
  extern __shared__ double acc[];  // ACC_N doubles (padded rows), count grid, kernel table
  int32_t* scnt = (int32_t*)(acc + ACC_N);
  float* ktab = (float*)(scnt + CGX * CGX * CGZ);
  __shared__ int s_lo[PROWS], s_pre[PROWS + 1], s_next;
  __shared__ double s_t27[27];
  __shared__ float s_rcp[NA + 1];  // 1/n for the clipped cloud widths n <= NA
  __shared__ int s_any;            // some level-0 host was counted
  UnitGeo g;
  unit_geo(M, B, order, it.x, dx, g);
  float* out = u11 + (size_t)g.ip * NA * NA * NA + (size_t)g.slab * PZ * NA * NA;
  if (g.zlo > g.zhi) {  // planes past the patch
    for (int q = threadIdx.x; q < NA * NA * PZ; q += blockDim.x) out[q] = 0.0f;
    return;
  }
  for (int q = threadIdx.x; q < ACC_N; q += blockDim.x) acc[q] = 0.0;
  for (int q = threadIdx.x; q < CGX * CGX * CGZ; q += blockDim.x) scnt[q] = 0;
  for (int l = 0; l <= g.ir; l++) {
    int nk = 1 << l, c0 = ktab_center(l);
    for (int i = threadIdx.x - nk; i <= nk; i += blockDim.x)
      ktab[c0 + i] = kernels[(size_t)l * KW + ASOHF_NMAX_KERNELS + i];
  }
  if (threadIdx.x >= 1 && threadIdx.x <= NA) s_rcp[threadIdx.x] = 1.0f / (float)threadIdx.x;
  if (threadIdx.x == 0) s_any = 0;
  __syncthreads();
  if (eqmass && threadIdx.x < 27) {  // level-0 terms of the common mass
    const float* kc = ktab + ktab_center(0);
    float m0 = P[0].w;  // any staged particle: all masses are equal
    int a = threadIdx.x % 3 - 1, b = (threadIdx.x / 3) % 3 - 1, cc = threadIdx.x / 9 - 1;
    s_t27[threadIdx.x] = (double)__fmul_rn(__fmul_rn(__fmul_rn(m0, kc[a]), kc[b]), kc[cc]);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t v0 = (int64_t)it.y * PSLICE, v1 = v0 + PSLICE;
  int64_t vbase = 0;
  for (int r0 = 0; r0 < g.rows; r0 += PROWS) {
    int nr = min(PROWS, g.rows - r0);
    __syncthreads();
    if (threadIdx.x < nr) {
      int lo, len;
      row_range(B, g, r0 + threadIdx.x, &lo, &len);
      s_lo[threadIdx.x] = lo;
      s_pre[threadIdx.x + 1] = len;
    }
    __syncthreads();
    if (warp == 0) {  // inclusive prefix of the row lengths in place, 32 rows at a time
      int run = 0;
      for (int r = 1 + lane; r - lane <= nr; r += 32) {
        int sc = r <= nr ? s_pre[r] : 0;
        for (int o = 1; o < 32; o <<= 1) {
          int y = __shfl_up_sync(0xffffffffu, sc, o);
          if (lane >= o) sc += y;
        }
        if (r <= nr) s_pre[r] = run + sc;
        run += __shfl_sync(0xffffffffu, sc, 31);
      }
      if (lane == 0) {
        s_pre[0] = 0;
        s_next = (int)(max(v0, vbase) - vbase);  // first candidate of this slice in these rows
      }
    }
    __syncthreads();
    const int tot = s_pre[nr];
    const int b = (int)(min(v1, vbase + tot) - vbase);
    // warps take 32 candidates at a time from a shared counter: a warp that
    // met wide clouds takes fewer
    for (;;) {
      int cbase = 0;
      if (lane == 0) cbase = atomicAdd(&s_next, 32);
      cbase = __shfl_sync(0xffffffffu, cbase, 0);
      if (cbase >= b) break;
      const int v = cbase + lane, vlast = min(cbase + 31, b - 1);
      // rows of the warp's first and last candidates (rows whose start is
      // not above them), then each lane's row between the two
      int c0 = 0, c1 = 0;
      for (int r = 1 + lane; r <= nr; r += 32) {
        int sp = s_pre[r];
        c0 += sp <= cbase;
        c1 += sp <= vlast;
      }
      int row = (int)__reduce_add_sync(0xffffffffu, (unsigned)c0);
      int rhi = (int)__reduce_add_sync(0xffffffffu, (unsigned)c1);
      while (row < rhi) {
        int mid = (row + rhi + 1) >> 1;
        if (s_pre[mid] <= v) row = mid; else rhi = mid - 1;
      }
      bool hit = false;
      float mp = 0.f;
      int ix = 0, jy = 0, kz = 0, lev = 0;
      if (v < b) {
        int e = s_lo[row] + (v - s_pre[row]);
        int s = S[e];
        float4 q = P[e];
        if (s != 255 && g.pxl < q.x && q.x < g.pxr && g.pyl < q.y && q.y < g.pyr && g.pzl < q.z && q.z < g.pzr) {
          lev = g.ir - s;
          if (lev < 0) lev = 0;
          int nk = 1 << lev;
          ix = (int)floorf((q.x - g.xlfix) / g.dxpa) + 1;
          jy = (int)floorf((q.y - g.ylfix) / g.dxpa) + 1;
          kz = (int)floorf((q.z - g.zlfix) / g.dxpa) + 1;
          if (!(ix - nk > g.n1 || ix + nk < 1 || jy - nk > g.n2 || jy + nk < 1 || kz - nk > g.n3 || kz + nk < 1) &&
              max(max(kz - nk, 1), g.zlo) <= min(min(kz + nk, g.n3), g.zhi)) {
            mp = q.w;
            if (eqmass && lev == 0) {  // host cell count (ix in [0, n1+1], kz in [zlo-1, zhi+1])
              atomicAdd(&scnt[((kz - g.zlo + 1) * CGX + jy) * CGX + ix], 1);
              s_any = 1;
            } else {
              hit = true;
            }
          }
        }
      }
      unsigned long long key =
          hit ? ((unsigned long long)(ix + 1024) << 52) | ((unsigned long long)(jy + 1024) << 41) |
                    ((unsigned long long)(kz + 1024) << 30) | ((unsigned long long)lev << 26) |
                    (unsigned long long)(__float_as_uint(mp) >> 6)
              : ~0ull - (unsigned long long)lane;
      // hits of one host cell, level and mass deposit once with the group size as factor
      unsigned grp = 1u << lane;
      if (__popc(__ballot_sync(0xffffffffu, hit)) > 1) grp = __match_any_sync(0xffffffffu, key);
      if (hit && (grp & (grp - 1))) {  // the key keeps 26 bits of the mass: confirm equal masses
        float m0 = __shfl_sync(grp, mp, __ffs(grp) - 1);
        unsigned same = __ballot_sync(grp, mp == m0);
        if (same != grp) grp = 1u << lane;
      }
      // host cell (11 bits per axis, offset 1024), level and group size of each hit
      const int pxy = (ix + 1024) | ((jy + 1024) << 16);
      const int pzl = (kz + 1024) | (lev << 16) | (__popc(grp) << 24);
      unsigned hm = __ballot_sync(0xffffffffu, hit && lane == __ffs(grp) - 1);
      while (hm) {
        int src = __ffs(hm) - 1;
        hm &= hm - 1;
        const float wm = __shfl_sync(0xffffffffu, mp, src);
        const int wxy = __shfl_sync(0xffffffffu, pxy, src), wzl = __shfl_sync(0xffffffffu, pzl, src);
        const int wix = (wxy & 0xffff) - 1024, wjy = (wxy >> 16) - 1024, wkz = (wzl & 0xffff) - 1024;
        const int wlev = (wzl >> 16) & 0xff, nk = 1 << wlev;
        const double wc = (double)(wzl >> 24);
        // the cloud clipped to the patch and to the unit's planes
        const int wi1 = max(wix - nk, 1), wj1 = max(wjy - nk, 1), wk1 = max(max(wkz - nk, 1), g.zlo);
        const int wdi = min(wix + nk, g.n1) - wi1 + 1, wdj = min(wjy + nk, g.n2) - wj1 + 1;
        const int wdk = min(min(wkz + nk, g.n3), g.zhi) - wk1 + 1;
        const float* kc = ktab + ktab_center(wlev);
        // lanes take the cloud's (ii, jj) pairs and walk its kk planes:
        // each lane forms (m*W(ii))*W(jj) once and the plane loop reads W(kk)
        // as a broadcast.  The pair quotient is exact in float (pairs < 2^11,
        // divisor <= 32).
        const int npair = wdi * wdj;
        const float rdi = s_rcp[wdi];
        const float* wzk = kc + (wk1 - wkz);  // W(kk) of the cloud's planes
        // pair p = (jj-j1)*di + (ii-i1): the lane's first pair by division,
        // the next ones (p += 32) by adding 32 = sj*di + si
        int ci, cj;
        {
          int q0 = (int)(((float)lane + 0.5f) * rdi);
          ci = lane - q0 * wdi;
          cj = q0;
        }
        const int sj = (int)((32.0f + 0.5f) * rdi), si = 32 - sj * wdi;
        for (int pq = lane; pq < npair; pq += 32) {
          const int ii = wi1 + ci, jj = wj1 + cj;
          float bw = __fmul_rn(__fmul_rn(wm, kc[ii - wix]), kc[jj - wjy]);
          double* col = acc + (wk1 - g.zlo) * APLANE + (jj - 1) * AROW + (ii - 1);
#pragma unroll
          for (int q = 0; q < PZ; q++)
            if (q < wdk) atomicAdd(col + q * APLANE, __dmul_rn((double)__fmul_rn(bw, wzk[q]), wc));
          ci += si;
          cj += sj;
          if (ci >= wdi) { ci -= wdi; cj++; }
        }
      }
    }
    vbase += tot;
  }
  __syncthreads();
  // level-0 hosts: 27-point stencil of the counts (cells inside the patch)
  if (eqmass && s_any && ktab[ktab_center(0) - 1] == ktab[ktab_center(0) + 1]) {
    // a symmetric level-0 kernel leaves 8 distinct terms, t(|di|, |dj|, |dk|):
    // a thread takes a column of cells, sums the counts of each neighbour
    // pattern plane by plane (integers) and forms 8 products per cell
    double tp[8];
#pragma unroll
    for (int q = 0; q < 8; q++) tp[q] = s_t27[((q >> 2) + 1) * 9 + (((q >> 1) & 1) + 1) * 3 + ((q & 1) + 1)];
    for (int col = threadIdx.x; col < NA * NA; col += blockDim.x) {
      const int i = col % NA + 1, j = col / NA + 1;
      if (i > g.n1 || j > g.n2) continue;
      int a0[CGZ], ax[CGZ], ay[CGZ], axy[CGZ];  // per count plane: centre, x pair, y pair, corners
#pragma unroll
      for (int pz = 0; pz < CGZ; pz++) {
        const int32_t* r0 = scnt + (pz * CGX + j) * CGX + i;
        const int32_t* rm = r0 - CGX;
        const int32_t* rp = r0 + CGX;
        a0[pz] = r0[0];
        ax[pz] = r0[-1] + r0[1];
        ay[pz] = rm[0] + rp[0];
        axy[pz] = (rm[-1] + rm[1]) + (rp[-1] + rp[1]);
      }
#pragma unroll
      for (int pz = 1; pz <= PZ; pz++) {  // output plane k = zlo + pz - 1
        if (g.zlo + pz - 1 > g.zhi) break;
        const int c0 = a0[pz], c1 = ax[pz], c2 = ay[pz], c3 = axy[pz];
        const int c4 = a0[pz - 1] + a0[pz + 1], c5 = ax[pz - 1] + ax[pz + 1];
        const int c6 = ay[pz - 1] + ay[pz + 1], c7 = axy[pz - 1] + axy[pz + 1];
        if ((c0 | c1 | c2 | c3 | c4 | c5 | c6 | c7) == 0) continue;
        double s = (double)c0 * tp[0] + (double)c1 * tp[1] + (double)c2 * tp[2] + (double)c3 * tp[3] +
                   (double)c4 * tp[4] + (double)c5 * tp[5] + (double)c6 * tp[6] + (double)c7 * tp[7];
        acc[(pz - 1) * APLANE + (j - 1) * AROW + (i - 1)] += s;
      }
    }
  } else if (eqmass && s_any) {
    for (int q = threadIdx.x; q < NA * NA * PZ; q += blockDim.x) {
      int i = q % NA + 1, j = (q / NA) % NA + 1, k = g.zlo + q / (NA * NA);
      if (i > g.n1 || j > g.n2 || k > g.zhi) continue;
      double s = 0.0;
      for (int kk = -1; kk <= 1; kk++)
        for (int jj = -1; jj <= 1; jj++)
          for (int ii = -1; ii <= 1; ii++) {
            int c = scnt[((k - kk - g.zlo + 1) * CGX + (j - jj)) * CGX + (i - ii)];
            if (c) s += (double)c * s_t27[(kk + 1) * 9 + (jj + 1) * 3 + (ii + 1)];
          }
      acc[(k - g.zlo) * APLANE + (j - 1) * AROW + (i - 1)] += s;
    }
  }
  const int sidx = W.scratch_of[it.x];
  if (sidx < 0) {
    __syncthreads();
    const float den = denbas_lev[g.ir];
    for (int q = threadIdx.x; q < NA * NA * PZ; q += blockDim.x) {
      int i = q % NA, j = (q / NA) % NA, k = g.slab * PZ + q / (NA * NA);
      float v = 0.0f;
      if (i < g.n1 && j < g.n2 && k < g.n3) v = (float)acc[(q / (NA * NA)) * APLANE + j * AROW + i] / den;
      out[q] = v;
    }
  } else {  // one slice of a shared unit
    __syncthreads();
    double* sc = W.scratch + (size_t)sidx * NA * NA * PZ;
    for (int q = threadIdx.x; q < NA * NA * PZ; q += blockDim.x) {
      double a = acc[(q / (NA * NA)) * APLANE + ((q / NA) % NA) * AROW + q % NA];
      if (a != 0.0) atomicAdd(&sc[q], a);
    }
  }
}

// The patch deposit over its work items: CTA b takes item b, and, with a
// work counter (a grid smaller than the item count), the next free item
// after each one.
__global__ void __launch_bounds__(PZ_BLOCK, 3)
k_density_patches(DevMesh M, Bins B, const float4* __restrict__ P, const uint8_t* __restrict__ S,
                  const int32_t* __restrict__ order, PatchWork W, float dx, const float* __restrict__ kernels,
                  int eqmass, float* __restrict__ u11, const float* __restrict__ denbas_lev, int nitems,
                  int* __restrict__ next_item) {
  __shared__ int s_item;
  int item = blockIdx.x;
  while (item < nitems) {
    density_patch_item(W.items[item], M, B, P, S, order, W, dx, kernels, eqmass, u11, denbas_lev);
    if (!next_item) break;
    __syncthreads();  // the item's last reads of shared memory are done
    if (threadIdx.x == 0) s_item = atomicAdd(next_item, 1) + (int)gridDim.x;
    __syncthreads();
    item = s_item;
  }
}

// Units shared by several slices: the summed scratch slab to U11.
__global__ void k_patch_finish(DevMesh M, const int32_t* __restrict__ order, const int32_t* __restrict__ multi,
                               const double* __restrict__ scratch, float* __restrict__ u11,
                               const float* __restrict__ denbas_lev) {
  int u = multi[blockIdx.x];
  int ip = order[u / NSLAB], slab = u % NSLAB;
  int n1 = M.nx[ip], n2 = M.ny[ip], n3 = M.nz[ip];
  float den = denbas_lev[M.level[ip]];
  const double* sc = scratch + (size_t)blockIdx.x * NA * NA * PZ;
  float* out = u11 + (size_t)ip * NA * NA * NA + (size_t)slab * PZ * NA * NA;
  for (int q = threadIdx.x; q < NA * NA * PZ; q += blockDim.x) {
    int i = q % NA, j = (q / NA) % NA, k = slab * PZ + q / (NA * NA);
    float v = 0.0f;
    if (i < n1 && j < n2 && k < n3) v = (float)sc[q] / den;
    out[q] = v;
  }
}

// Patch order of the deposit: finest level first, table order within a level.
static int patch_order(asohf_ctx* c, const asohf_mesh* mh, int32_t** d_order, DAlloc A = DAlloc{nullptr, false}) {
  int np = 0;
  for (int ir = 1; ir <= mh->nl; ir++) np += mh->npatch[ir];
  std::vector<int32_t> h((size_t)(np > 0 ? np : 1));
  int q = 0;
  for (int ir = mh->nl; ir >= 1; ir--) {
    int first = 0;
    for (int l = 1; l < ir; l++) first += mh->npatch[l];
    for (int p = 0; p < mh->npatch[ir]; p++) h[q++] = first + p;
  }
  const size_t bytes = 4 * (size_t)(np > 0 ? np : 1);
  *d_order = (int32_t*)(A.pool ? A.get(bytes) : arena_alloc(c, bytes));
  if (!*d_order) return ASOHF_ERR_CAPACITY;
  ASOHF_CUDA(cudaMemcpyAsync(*d_order, h.data(), 4 * (size_t)np, cudaMemcpyHostToDevice, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  return ASOHF_OK;
}

static float* upload_floats(asohf_ctx* c, const float* h, size_t n, DAlloc A = DAlloc{nullptr, false}) {
  float* d = (float*)(A.pool ? A.get(4 * n) : arena_alloc(c, 4 * n));
  if (d) cudaMemcpyAsync(d, h, 4 * n, cudaMemcpyHostToDevice, c->stream);
  return d;
}

// Output staging: returns a device pointer for `bytes` of output.
static int stage_out(asohf_ctx* c, float* user, size_t bytes, int on_device, float** dev) {
  if (on_device) { *dev = user; return ASOHF_OK; }
  *dev = (float*)arena_alloc(c, bytes);
  return *dev ? ASOHF_OK : ASOHF_ERR_CAPACITY;
}

extern "C" int asohf_density(asohf_ctx* c, int nx, float lado0, float dx, float rote, float rete,
                             const int32_t* npart_esp, const asohf_mesh* mesh, int interp_degree,
                             float* u1, float* u11, int on_device) {
  if (!c || nx <= 0 || !npart_esp || !u1 || (interp_degree != 1 && interp_degree != 2))
    return ASOHF_ERR_INVALID;
  int nl = mesh ? mesh->nl : 0;
  if (nl < 0 || nl > ASOHF_NLEVELS) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  int64_t n = 0;
  for (int s = 0; s < ASOHF_N_ESP; s++) n += npart_esp[s];
  if (n > c->p.n) return ASOHF_ERR_INVALID;
  int64_t g = (int64_t)nx * nx * nx;
  int np = 0;
  for (int ir = 1; ir <= nl; ir++) np += mesh->npatch[ir];
  if (np > 0 && !u11) return ASOHF_ERR_INVALID;
  const int64_t nall = c->p.n;
  const bool eqmass = c->mmin == c->norma;  // one particle mass in the store
  // the previous call's deferred patch work reads the pools and writes U11
  ASOHF_CHECK(density_settle(c));
  const bool defer = c->density_overlap && on_device && np > 0 && n > 0 && c->dens_stream;
  const DAlloc A{c, defer};
  size_t need = 12 * g + (on_device ? 0 : 4 * g + 4 * (size_t)np * NA * NA * NA) +
                4 * KW * (ASOHF_NLEVELS + 1) + 96 * (size_t)np + 16384 +
                (np ? bins_bytes(nall, lado0, dx, 2) + 17 * (size_t)nall : 0);
  ASOHF_CHECK(arena_reserve(c, need));
  if (defer) {  // what the deferred kernels read: kernels, mesh, order, bins, staged particles, renorm dims
    const int nbw = (int)lrintf(lado0 / dx);
    const int64_t nb = (nbw + 1) / 2, nbin = nb * nb * nb;
    ASOHF_CHECK(dpool_reserve(c, 0, 4 * KW * (ASOHF_NLEVELS + 1) + 4 * (ASOHF_NLEVELS + 1) + 48 * (size_t)np +
                                        4 * (size_t)(nbin + 1) + 17 * (size_t)nall + 4 * NSLAB * (size_t)np +
                                        16 * 256));
  }
  std::vector<float> hk_v((size_t)KW * (ASOHF_NLEVELS + 1));
  float* hk = hk_v.data();
  compute_kernels_host(nl, interp_degree, hk);
  float* dk = upload_floats(c, hk, (size_t)KW * (ASOHF_NLEVELS + 1), A);
  const float* h0 = hk + ASOHF_NMAX_KERNELS;  // level 0: W(-1), W(0), W(1) at h0[-1..1]
  Terms27 T27;
  for (int kk = -1; kk <= 1; kk++)
    for (int jj = -1; jj <= 1; jj++)
      for (int ii = -1; ii <= 1; ii++) {
        volatile float t = c->norma * h0[ii];
        t = t * h0[jj];
        t = t * h0[kk];
        T27.t[(kk + 1) * 9 + (jj + 1) * 3 + (ii + 1)] = (double)t;
      }
  bool sym27 = true;  // each term equals the one of its mirrored offsets
  for (int q = 0; q < 27; q++) {
    const int ii = q % 3 - 1, jj = (q / 3) % 3 - 1, kk = q / 9 - 1;
    const int m = (abs(kk) + 1) * 9 + (abs(jj) + 1) * 3 + (abs(ii) + 1);
    if (T27.t[q] != T27.t[m]) sym27 = false;
  }
  float* du1;
  ASOHF_CHECK(stage_out(c, u1, 4 * g, on_device, &du1));
  const float xl = -lado0 / 2.0f;
  const float denbas = dx * dx * dx * rote * (rete * rete * rete);
  double* acc = (double*)arena_alloc(c, 8 * g);
  int64_t hend[ASOHF_N_ESP];
  int64_t acc_n = 0;
  for (int s = 0; s < ASOHF_N_ESP; s++) { acc_n += npart_esp[s]; hend[s] = acc_n; }
  int64_t* dend = (int64_t*)arena_alloc(c, sizeof(hend));
  if (!acc || !dk || !dend) return ASOHF_ERR_CAPACITY;
  ASOHF_CUDA(cudaMemcpyAsync(dend, hend, sizeof(hend), cudaMemcpyHostToDevice, c->stream));
  const float* k0 = dk + ASOHF_NMAX_KERNELS - 1;  // level 0: W(-1), W(0), W(1)
  if (n > 0 && eqmass) {
    int32_t* cnt = (int32_t*)arena_alloc(c, 4 * g);
    if (!cnt) return ASOHF_ERR_CAPACITY;
    ASOHF_CUDA(cudaMemsetAsync(cnt, 0, 4 * g, c->stream));
    int kt_ = ktime_begin(c, "density_base");
    k_base_counts<<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(c->p.x, c->p.y, c->p.z, n, nx, xl,
                                                                          dx, cnt);
    if (sym27)  // 8 distinct terms
      k_base_stencil_sym<<<grid_for(g, 256, c->num_sms * 16), 256, 0, c->stream>>>(cnt, nx, T27, acc);
    else
      k_base_stencil<<<grid_for(g, 256, c->num_sms * 16), 256, 0, c->stream>>>(cnt, nx, T27, acc);
    k_density_base_outliers<<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(
      c->p.x, c->p.y, c->p.z, c->p.m, n, nx, xl, dx, k0, acc);
    ktime_end(c, kt_);
    c->launches += 3;
  } else {
    ASOHF_CUDA(cudaMemsetAsync(acc, 0, 8 * g, c->stream));
    if (n > 0) {
      int kt_ = ktime_begin(c, "density_base");
      k_density_base_all<<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        c->p.x, c->p.y, c->p.z, c->p.m, n, nx, xl, dx, k0, acc);
      ktime_end(c, kt_);
      c->launches++;
    }
  }
  {
    int kt_ = ktime_begin(c, "density_finish");
    k_finish_f64<<<grid_for(g, 256), 256, 0, c->stream>>>(acc, g, denbas, du1);
    ktime_end(c, kt_);
  }
  c->launches++;
  ASOHF_CUDA(cudaGetLastError());
  if (!on_device) ASOHF_CUDA(cudaMemcpyAsync(u1, du1, 4 * g, cudaMemcpyDeviceToHost, c->stream));
  if (np > 0) {
    DevMesh M;
    ASOHF_CHECK(upload_mesh(c, mesh, &M, A));
    float hden[ASOHF_NLEVELS + 1];
    for (int ir = 0; ir <= ASOHF_NLEVELS; ir++) {
      float dxpa = dx / powf(2.0f, (float)ir);
      hden[ir] = dxpa * dxpa * dxpa * rote * (rete * rete * rete);
    }
    float* dden = upload_floats(c, hden, ASOHF_NLEVELS + 1, A);
    float* du11;
    ASOHF_CHECK(stage_out(c, u11, 4 * (size_t)np * NA * NA * NA, on_device, &du11));
    int32_t* order = nullptr;
    if (!dden) return ASOHF_ERR_CAPACITY;
    ASOHF_CHECK(patch_order(c, mesh, &order, A));
    if (n > 0) {
      Bins B;
      ASOHF_CHECK(build_bins(c, lado0, dx, 2, &B, A));
      float4* bp = (float4*)A.get(16 * (size_t)nall);
      uint8_t* bs = (uint8_t*)A.get((size_t)nall);
      const int nunits = NSLAB * np;
      int64_t* ucnt = (int64_t*)arena_alloc(c, 8 * (size_t)nunits);
      int32_t* sof = (int32_t*)A.get(4 * (size_t)nunits);
      if (!bp || !bs || !ucnt || !sof) return ASOHF_ERR_CAPACITY;
      {
        int kt_ = ktime_begin(c, "density_bin_stage");
        k_bin_stage<<<grid_for(nall, 256, c->num_sms * 16), 256, 0, c->stream>>>(
            B.idx, nall, n, c->p.x, c->p.y, c->p.z, c->p.m, c->rows_cur >= 0 ? c->rows[c->rows_cur] : nullptr,
            dend, bp, bs);
        k_patch_unit_counts<<<(nunits + 7) / 8, 256, 0, c->stream>>>(M, B, order, nunits, dx, ucnt);
        ktime_end(c, kt_);
        c->launches += 2;
      }
      // work list: slices of PSLICE candidates, the densest units first
      std::vector<int64_t> hc_v((size_t)nunits);
      std::vector<int32_t> hs_v((size_t)nunits), ord_v((size_t)nunits);
      int64_t* hc = hc_v.data();
      int32_t* hs = hs_v.data();
      int32_t* ord = ord_v.data();
      ASOHF_CUDA(cudaMemcpyAsync(hc, ucnt, 8 * (size_t)nunits, cudaMemcpyDeviceToHost, c->stream));
      ASOHF_CUDA(cudaStreamSynchronize(c->stream));
      int64_t nitems = 0;
      int nmulti = 0;
      for (int u = 0; u < nunits; u++) {
        int64_t ns = hc[u] > 0 ? (hc[u] + PSLICE - 1) / PSLICE : 1;
        hs[u] = ns > 1 ? nmulti++ : -1;
        nitems += ns;
        ord[u] = u;
      }
      {  // counts descending, ties by unit index (stable radix sort of the counts)
        std::vector<uint32_t> key((size_t)nunits);
        for (int u = 0; u < nunits; u++) key[u] = (uint32_t)(hc[u] < 0xffffffffll ? hc[u] : 0xffffffffll);
        stable_desc(key, ord, nunits);
      }
      std::vector<int2> hitems_v((size_t)nitems);
      std::vector<int32_t> hmulti_v((size_t)(nmulti > 0 ? nmulti : 1));
      int2* hitems = hitems_v.data();
      int32_t* hmulti = hmulti_v.data();
      int64_t w = 0;
      for (int k = 0; k < nunits; k++) {
        int u = ord[k];
        int64_t ns = hc[u] > 0 ? (hc[u] + PSLICE - 1) / PSLICE : 1;
        for (int64_t q = 0; q < ns; q++) hitems[w++] = make_int2(u, (int)q);
        if (hs[u] >= 0) hmulti[hs[u]] = u;
      }
      size_t scratch_b = sizeof(double) * NA * NA * PZ * (size_t)nmulti;
      // work items, shared-unit list and scratch: the segment buffers, or
      // density pool 1 when deferred
      const size_t wbytes = sizeof(int2) * (size_t)nitems + 4 * (size_t)nmulti + scratch_b + 4096 + 256;
      int rcs = defer ? dpool_reserve(c, 1, wbytes) : seg_reserve(c, wbytes);
      auto walloc = [&](size_t b) { return defer ? dpool_alloc(c, 1, b) : seg_alloc(c, b); };
      int2* ditems = rcs == ASOHF_OK ? (int2*)walloc(sizeof(int2) * (size_t)nitems) : nullptr;
      int32_t* dmulti = rcs == ASOHF_OK ? (int32_t*)walloc(4 * (size_t)(nmulti > 0 ? nmulti : 1)) : nullptr;
      double* scratch = rcs == ASOHF_OK ? (double*)walloc(scratch_b > 0 ? scratch_b : 8) : nullptr;
      // one CTA per item; the kernel can also run as a smaller grid drawing
      // items from a counter (next_item), which measured slower beside the
      // halo finder (the patch deposit took 181 ms as one CTA per SM and
      // slowed the halo kernels by 38 ms), so the full grid is launched
      int* next_item = nullptr;
      if (!ditems || !dmulti || !scratch) return rcs != ASOHF_OK ? rcs : ASOHF_ERR_CAPACITY;
      ASOHF_CUDA(cudaMemcpyAsync(ditems, hitems, sizeof(int2) * (size_t)nitems, cudaMemcpyHostToDevice, c->stream));
      ASOHF_CUDA(cudaMemcpyAsync(sof, hs, 4 * (size_t)nunits, cudaMemcpyHostToDevice, c->stream));
      if (nmulti) {
        ASOHF_CUDA(cudaMemcpyAsync(dmulti, hmulti, 4 * (size_t)nmulti, cudaMemcpyHostToDevice, c->stream));
        ASOHF_CUDA(cudaMemsetAsync(scratch, 0, scratch_b, c->stream));
      }
      ASOHF_CUDA(cudaStreamSynchronize(c->stream));
      PatchWork W{ditems, sof, scratch};
      size_t smem = sizeof(double) * ACC_N + sizeof(int32_t) * CGX * CGX * CGZ + sizeof(float) * ktab_size(nl);
      ASOHF_CUDA(cudaFuncSetAttribute(k_density_patches, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      // deferred: the patch kernels run on the density stream after the
      // staging above, and the call returns without waiting for them
      cudaStream_t ps = c->stream;
      if (defer) {
        ASOHF_CUDA(cudaEventRecord(c->dens_fork, c->stream));
        ASOHF_CUDA(cudaStreamWaitEvent(c->dens_stream, c->dens_fork, 0));
        ps = c->dens_stream;
      }
      int kt_ = ktime_begin(c, "density_patches", ps);
      k_density_patches<<<(unsigned)nitems, PZ_BLOCK, smem, ps>>>(M, B, bp, bs, order, W, dx, dk, eqmass ? 1 : 0,
                                                               du11, dden, (int)nitems, next_item);
      if (nmulti) k_patch_finish<<<nmulti, 256, 0, ps>>>(M, order, dmulti, scratch, du11, dden);
      ktime_end(c, kt_, ps);
      c->launches += 1 + (nmulti > 0);
      if (defer) {
        ASOHF_CUDA(cudaEventRecord(c->dens_done, ps));
        c->dens_pending = true;
      }
    } else {  // no particles: empty patches
      ASOHF_CUDA(cudaMemsetAsync(du11, 0, 4 * (size_t)np * NA * NA * NA, c->stream));
    }
    ASOHF_CUDA(cudaGetLastError());
    if (!on_device)
      ASOHF_CUDA(cudaMemcpyAsync(u11, du11, 4 * (size_t)np * NA * NA * NA, cudaMemcpyDeviceToHost, c->stream));
  }
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  return ASOHF_OK;
}

// ------------------------------------------------------------ renorm
__global__ void k_scale(float* __restrict__ a, int64_t n, float f) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] = a[i] / f;
}

__global__ void k_scale_patches(float* __restrict__ u11, const int32_t* __restrict__ dims, int np,
                                float f) {
  int ip = blockIdx.x;
  int n1 = dims[ip], n2 = dims[np + ip], n3 = dims[2 * np + ip];
  float* u = u11 + (size_t)ip * NA * NA * NA;
  for (int q = threadIdx.x; q < NA * NA * NA; q += blockDim.x) {
    int i = q % NA, j = (q / NA) % NA, k = q / (NA * NA);
    if (i < n1 && j < n2 && k < n3) u[q] = u[q] / f;
  }
}

extern "C" int asohf_renorm_density(asohf_ctx* c, int nx, const asohf_mesh* mesh, float fdm,
                                    float* u1, float* u11, int on_device) {
  if (!c || nx <= 0 || !u1) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  int64_t g = (int64_t)nx * nx * nx;
  int np = 0, nl = mesh ? mesh->nl : 0;
  for (int ir = 1; ir <= nl; ir++) np += mesh->npatch[ir];
  ASOHF_CHECK(arena_reserve(c, (on_device ? 0 : 4 * g + 4 * (size_t)np * NA * NA * NA) + 16 * (size_t)np + 1024));
  float *d1 = u1, *d11 = u11;
  if (!on_device) {
    d1 = (float*)arena_alloc(c, 4 * g);
    ASOHF_CUDA(cudaMemcpyAsync(d1, u1, 4 * g, cudaMemcpyHostToDevice, c->stream));
    if (np) {
      d11 = (float*)arena_alloc(c, 4 * (size_t)np * NA * NA * NA);
      ASOHF_CUDA(cudaMemcpyAsync(d11, u11, 4 * (size_t)np * NA * NA * NA, cudaMemcpyHostToDevice, c->stream));
    }
  }
  k_scale<<<grid_for(g, 256), 256, 0, c->stream>>>(d1, g, fdm);
  c->launches++;
  if (np) {
    int base = mesh->npatch[0];
    std::vector<int32_t> hd(3 * (size_t)np);
    for (int q = 0; q < np; q++) {
      hd[q] = mesh->patchnx[base + q];
      hd[np + q] = mesh->patchny[base + q];
      hd[2 * np + q] = mesh->patchnz[base + q];
    }
    // after a deferred patch deposit the scaling follows it on its stream,
    // with the dimensions in its pool
    const bool deferred = on_device && c->dens_pending;
    int32_t* dd = (int32_t*)(deferred ? dpool_alloc(c, 0, 12 * (size_t)np) : arena_alloc(c, 12 * (size_t)np));
    if (!dd) return ASOHF_ERR_CAPACITY;
    // the dimensions go up on the context stream (a pageable copy on the
    // density stream would make the host wait for the patch kernels)
    ASOHF_CUDA(cudaMemcpyAsync(dd, hd.data(), 12 * (size_t)np, cudaMemcpyHostToDevice, c->stream));
    cudaStream_t ps = c->stream;
    if (deferred) {
      ASOHF_CUDA(cudaEventRecord(c->dens_fork, c->stream));
      ASOHF_CUDA(cudaStreamWaitEvent(c->dens_stream, c->dens_fork, 0));
      ps = c->dens_stream;
    }
    k_scale_patches<<<np, 256, 0, ps>>>(d11, dd, np, fdm);
    c->launches++;
    if (deferred) {
      ASOHF_CUDA(cudaGetLastError());
      ASOHF_CUDA(cudaEventRecord(c->dens_done, ps));
      ASOHF_CUDA(cudaStreamSynchronize(c->stream));  // the base grid; the patches follow on their stream
      return ASOHF_OK;
    }
    ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  }
  ASOHF_CUDA(cudaGetLastError());
  if (!on_device) {
    ASOHF_CUDA(cudaMemcpyAsync(u1, d1, 4 * g, cudaMemcpyDeviceToHost, c->stream));
    if (np)
      ASOHF_CUDA(cudaMemcpyAsync(u11, d11, 4 * (size_t)np * NA * NA * NA, cudaMemcpyDeviceToHost, c->stream));
  }
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  return ASOHF_OK;
}

// ------------------------------------------------------------ TSC deposit
// Base grid TSC for a batch of particle sets; acc has batch*nx^3 doubles or floats.
template <typename T>
__global__ void k_tsc_base(const float* __restrict__ x, const float* __restrict__ y,
                           const float* __restrict__ z, const float* __restrict__ m, int64_t n_per,
                           int batch, int nx, float xl, float dx, const float* __restrict__ radx,
                           float mdiv, T* __restrict__ acc) {
  int64_t ntot = n_per * batch;
  size_t g = (size_t)nx * nx * nx;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < ntot;
       q += (int64_t)gridDim.x * blockDim.x) {
    int b = (int)(q / n_per);
    float xp = x[q], yp = y[q], zp = z[q];
    int ix = tsc_cell(xp, xl, dx, nx), jy = tsc_cell(yp, xl, dx, nx), kz = tsc_cell(zp, xl, dx, nx);
    float wx[3], wy[3], wz[3];
    tsc_weights(xp, radx[ix - 1], radx[ix], radx[ix + 1], dx, wx);
    tsc_weights(yp, radx[jy - 1], radx[jy], radx[jy + 1], dx, wy);
    tsc_weights(zp, radx[kz - 1], radx[kz], radx[kz + 1], dx, wz);
    float mp = mdiv == 1.0f ? m[q] : __fdiv_rn(m[q], mdiv);  // mass, or mass / DENBAS
    T* a = acc + (size_t)b * g;
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
          float t = __fmul_rn(__fmul_rn(__fmul_rn(mp, wx[ii + 1]), wy[jj + 1]), wz[kk + 1]);
          atomicAdd(&a[((size_t)(k1 - 1) * nx + (j1 - 1)) * nx + (i1 - 1)], (T)t);
        }
      }
    }
  }
}

// PLEV (grids.f:1121-1152): the finest level with a patch that contains the
// particle inside a one-cell buffer.  One CTA per patch raises plev by
// atomicMax over the particles of the bins it overlaps.
__global__ void k_tsc_plev(DevMesh M, Bins B, const float* __restrict__ x, const float* __restrict__ y,
                           const float* __restrict__ z, float dx, int32_t* __restrict__ plev) {
  int ip = blockIdx.x;
  int ir = M.level[ip];
  float dxpa = dx / exp2f((float)ir);
  float xl = M.rx[ip] - 2.0f * dxpa, yl = M.ry[ip] - 2.0f * dxpa, zl = M.rz[ip] - 2.0f * dxpa;
  float xr = xl + (float)(M.nx[ip] + 2) * dxpa, yr = yl + (float)(M.ny[ip] + 2) * dxpa,
        zr = zl + (float)(M.nz[ip] + 2) * dxpa;
  int bx0 = bin_of(xl, B.xl, B.bsz, B.nb), bx1 = bin_of(xr, B.xl, B.bsz, B.nb);
  int by0 = bin_of(yl, B.xl, B.bsz, B.nb), by1 = bin_of(yr, B.xl, B.bsz, B.nb);
  int bz0 = bin_of(zl, B.xl, B.bsz, B.nb), bz1 = bin_of(zr, B.xl, B.bsz, B.nb);
  for (int bz = bz0; bz <= bz1; bz++)
    for (int by = by0; by <= by1; by++) {
      int lo = B.start[(bz * B.nb + by) * B.nb + bx0], hi = B.start[(bz * B.nb + by) * B.nb + bx1 + 1];
      for (int t = lo + threadIdx.x; t < hi; t += blockDim.x) {
        int p = B.idx[t];
        if (xl < x[p] && x[p] < xr && yl < y[p] && y[p] < yr && zl < z[p] && z[p] < zr)
          atomicMax(&plev[p], ir);
      }
    }
}

// Patch TSC (grids.f:1286-1372): one CTA per (patch, z-half).
__global__ void __launch_bounds__(PD_BLOCK)
k_tsc_patches(DevMesh M, Bins B, const float* __restrict__ x, const float* __restrict__ y,
              const float* __restrict__ z, const float* __restrict__ m, const int32_t* __restrict__ plev,
              float dx, float* __restrict__ u11, const float* __restrict__ denbas_lev) {
  extern __shared__ double acc[];
  int ip = blockIdx.x >> 1, half = blockIdx.x & 1;
  int n1 = M.nx[ip], n2 = M.ny[ip], n3 = M.nz[ip], ir = M.level[ip];
  int zlo = half * ZH + 1, zhi = min(half * ZH + ZH, n3);
  for (int q = threadIdx.x; q < NA * NA * ZH; q += blockDim.x) acc[q] = 0.0;
  __syncthreads();
  float dxpa = dx / exp2f((float)ir);
  float xl = M.rx[ip] - 2.0f * dxpa, yl = M.ry[ip] - 2.0f * dxpa, zl = M.rz[ip] - 2.0f * dxpa;
  float xr = xl + (float)(n1 + 2) * dxpa, yr = yl + (float)(n2 + 2) * dxpa, zr = zl + (float)(n3 + 2) * dxpa;
  if (zlo <= zhi) {
    int bx0 = bin_of(xl, B.xl, B.bsz, B.nb), bx1 = bin_of(xr, B.xl, B.bsz, B.nb);
    int by0 = bin_of(yl, B.xl, B.bsz, B.nb), by1 = bin_of(yr, B.xl, B.bsz, B.nb);
    int bz0 = bin_of(zl, B.xl, B.bsz, B.nb), bz1 = bin_of(zr, B.xl, B.bsz, B.nb);
    for (int bz = bz0; bz <= bz1; bz++)
      for (int by = by0; by <= by1; by++) {
        int lo = B.start[(bz * B.nb + by) * B.nb + bx0], hi = B.start[(bz * B.nb + by) * B.nb + bx1 + 1];
        for (int t = lo + threadIdx.x; t < hi; t += blockDim.x) {
          int p = B.idx[t];
          if (plev[p] < ir) continue;
          float xp = x[p], yp = y[p], zp = z[p];
          if (!(xl < xp && xp < xr && yl < yp && yp < yr && zl < zp && zp < zr)) continue;
          int ix = (int)((xp - xl) / dxpa) + 1 - 1;
          int jy = (int)((yp - yl) / dxpa) + 1 - 1;
          int kz = (int)((zp - zl) / dxpa) + 1 - 1;
          // MINIRADX(II) = PATCHRX + (II - 1.5) DXPA
          float wx[3], wy[3], wz[3];
          float rxm = M.rx[ip] + ((float)(ix - 1) - 1.5f) * dxpa, rx0 = M.rx[ip] + ((float)ix - 1.5f) * dxpa,
                rxp = M.rx[ip] + ((float)(ix + 1) - 1.5f) * dxpa;
          float rym = M.ry[ip] + ((float)(jy - 1) - 1.5f) * dxpa, ry0 = M.ry[ip] + ((float)jy - 1.5f) * dxpa,
                ryp = M.ry[ip] + ((float)(jy + 1) - 1.5f) * dxpa;
          float rzm = M.rz[ip] + ((float)(kz - 1) - 1.5f) * dxpa, rz0 = M.rz[ip] + ((float)kz - 1.5f) * dxpa,
                rzp = M.rz[ip] + ((float)(kz + 1) - 1.5f) * dxpa;
          tsc_weights(xp, rxm, rx0, rxp, dxpa, wx);
          tsc_weights(yp, rym, ry0, ryp, dxpa, wy);
          tsc_weights(zp, rzm, rz0, rzp, dxpa, wz);
          float mp = m[p];
          for (int kk = -1; kk <= 1; kk++)
            for (int jj = -1; jj <= 1; jj++)
              for (int ii = -1; ii <= 1; ii++) {
                int i1 = ix + ii, j1 = jy + jj, k1 = kz + kk;
                if (i1 > 0 && i1 <= n1 && j1 > 0 && j1 <= n2 && k1 >= zlo && k1 <= zhi) {
                  float tt = __fmul_rn(__fmul_rn(__fmul_rn(mp, wx[ii + 1]), wy[jj + 1]), wz[kk + 1]);
                  atomicAdd(&acc[((k1 - zlo) * NA + (j1 - 1)) * NA + (i1 - 1)], (double)tt);
                }
              }
        }
      }
  }
  __syncthreads();
  float den = denbas_lev[ir];
  float* out = u11 + (size_t)ip * NA * NA * NA;
  for (int q = threadIdx.x; q < NA * NA * ZH; q += blockDim.x) {
    int i = q % NA, j = (q / NA) % NA, kl = q / (NA * NA);
    int k = half * ZH + kl;
    float v = 0.0f;
    if (i < n1 && j < n2 && k < n3) v = (float)acc[q] / den;
    out[((size_t)k * NA + j) * NA + i] = v;
  }
}

extern "C" int asohf_interpolate_density_tsc(asohf_ctx* c, int nx, float lado0, float dx,
                                             const float* radx, float rote, float rete,
                                             const asohf_mesh* mesh, float* u1, float* u11,
                                             int on_device) {
  if (!c || nx <= 0 || !radx || !u1) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  int64_t n = c->p.n;
  int64_t g = (int64_t)nx * nx * nx;
  int nl = mesh ? mesh->nl : 0;
  int np = 0;
  for (int ir = 1; ir <= nl; ir++) np += mesh->npatch[ir];
  if (np > 0 && !u11) return ASOHF_ERR_INVALID;
  size_t need = 8 * g + 4 * g + 4 * (size_t)np * NA * NA * NA + 4 * (nx + 2) + 4 * n +
                64 * (size_t)np + 8192 + (np ? bins_bytes(n, lado0, dx, 2) : 0);
  ASOHF_CHECK(arena_reserve(c, need));
  float* dradx = upload_floats(c, radx, nx + 2);
  double* acc = (double*)arena_alloc(c, 8 * g);
  float* du1;
  ASOHF_CHECK(stage_out(c, u1, 4 * g, on_device, &du1));
  if (!dradx || !acc) return ASOHF_ERR_CAPACITY;
  ASOHF_CUDA(cudaMemsetAsync(acc, 0, 8 * g, c->stream));
  float xl = -lado0 / 2.0f;
  if (n > 0) {
    {
      int kt_ = ktime_begin(c, "tsc_base");
      k_tsc_base<double><<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(
        c->p.x, c->p.y, c->p.z, c->p.m, n, 1, nx, xl, dx, dradx, 1.0f, acc);
      ktime_end(c, kt_);
    }
    c->launches++;
  }
  float denbas = dx * dx * dx * rote * (rete * rete * rete);
  k_finish_f64<<<grid_for(g, 256), 256, 0, c->stream>>>(acc, g, denbas, du1);
  c->launches++;
  ASOHF_CUDA(cudaGetLastError());
  if (!on_device) ASOHF_CUDA(cudaMemcpyAsync(u1, du1, 4 * g, cudaMemcpyDeviceToHost, c->stream));
  if (np > 0) {
    DevMesh M;
    ASOHF_CHECK(upload_mesh(c, mesh, &M));
    Bins B;
    ASOHF_CHECK(build_bins(c, lado0, dx, 2, &B));
    int32_t* plev = (int32_t*)arena_alloc(c, 4 * n);
    float hden[ASOHF_NLEVELS + 1];
    for (int ir = 0; ir <= ASOHF_NLEVELS; ir++) {
      float dxpa = dx / powf(2.0f, (float)ir);
      hden[ir] = dxpa * dxpa * dxpa * rote * (rete * rete * rete);
    }
    float* dden = upload_floats(c, hden, ASOHF_NLEVELS + 1);
    float* du11;
    ASOHF_CHECK(stage_out(c, u11, 4 * (size_t)np * NA * NA * NA, on_device, &du11));
    if (!plev || !dden) return ASOHF_ERR_CAPACITY;
    ASOHF_CUDA(cudaMemsetAsync(plev, 0, 4 * n, c->stream));
    {
      int kt_ = ktime_begin(c, "tsc_plev");
      k_tsc_plev<<<np, 256, 0, c->stream>>>(M, B, c->p.x, c->p.y, c->p.z, dx, plev);
      ktime_end(c, kt_);
    }
    size_t smem = sizeof(double) * NA * NA * ZH;
    ASOHF_CUDA(cudaFuncSetAttribute(k_tsc_patches, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    {
      int kt_ = ktime_begin(c, "tsc_patches");
      k_tsc_patches<<<2 * np, PD_BLOCK, smem, c->stream>>>(M, B, c->p.x, c->p.y, c->p.z, c->p.m, plev, dx,
                                                         du11, dden);
      ktime_end(c, kt_);
    }
    c->launches += 2;
    ASOHF_CUDA(cudaGetLastError());
    if (!on_device)
      ASOHF_CUDA(cudaMemcpyAsync(u11, du11, 4 * (size_t)np * NA * NA * NA, cudaMemcpyDeviceToHost, c->stream));
  }
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  return ASOHF_OK;
}

// exported for poisson.cu (batched forward deposit of m / denbas)
int tsc_base_batched_f32(asohf_ctx* c, int nx, float xl, float dx, const float* dradx, int batch,
                         int64_t n_per, const float* x, const float* y, const float* z,
                         const float* m, float denbas, float* acc) {
  int64_t n = n_per * batch;
  if (n > 0) {
    {
      int kt_ = ktime_begin(c, "tsc_base_batched");
      k_tsc_base<float><<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(x, y, z, m, n_per, batch,
                                                                              nx, xl, dx, dradx, denbas, acc);
      ktime_end(c, kt_);
    }
    c->launches++;
  }
  ASOHF_CUDA(cudaGetLastError());
  return ASOHF_OK;
}

// ------------------------------------------------------------ CREATE_MESH particle counts
// The two counting loops of CREATE_MESH (grids.f:107-143 for the base grid,
// grids.f:357-380 for the patches of one level): NGP cell counts in which a
// particle weighs 1 when its species level PLEV is at most the level being
// refined (0 for the base grid) and REFINE_THR otherwise, then zero within
// BOR (BORAMR) cells of the faces.  PLEV(I) is the species whose index range
// (NPART_ESP, store order) holds I, and 0 past the last range (grids.f:83-91).
// The patch placement that consumes the counts is sequential and stays with
// the caller.

struct EspEnds {
  int64_t e[ASOHF_N_ESP];  // cumulative ends of the species ranges
};

__device__ __forceinline__ int plev_of(int64_t i, const EspEnds& E) {
  for (int s = 0; s < ASOHF_N_ESP; s++)
    if (i < E.e[s]) return s;
  return 0;
}

__global__ void k_mesh_base_counts(const float* __restrict__ x, const float* __restrict__ y,
                                   const float* __restrict__ z, int64_t n, int nx, float xl, float dx,
                                   int refine_thr, EspEnds E, int32_t* __restrict__ cnt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    // IX = INT((RXPA-XL)/DX)+1 clamped to 1..NX (a NaN offset counts as below)
    int c3[3];
    const float v3[3] = {x[i], y[i], z[i]};
    for (int a = 0; a < 3; a++) {
      const float v = __fdiv_rn(__fsub_rn(v3[a], xl), dx);
      c3[a] = v >= (float)nx ? nx : (v >= 1.0f ? (int)v + 1 : 1);
    }
    const int w = plev_of(i, E) == 0 ? 1 : refine_thr;
    atomicAdd(&cnt[((int64_t)(c3[2] - 1) * nx + (c3[1] - 1)) * nx + (c3[0] - 1)], w);
  }
}

__global__ void k_mesh_border(int32_t* __restrict__ cnt, int nx, int bor) {
  const int64_t g = (int64_t)nx * nx * nx;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < g; q += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(q % nx) + 1, jy = (int)((q / nx) % nx) + 1, kz = (int)(q / ((int64_t)nx * nx)) + 1;
    if (ix <= bor || ix >= nx - bor + 1 || jy <= bor || jy >= nx - bor + 1 || kz <= bor || kz >= nx - bor + 1)
      cnt[q] = 0;
  }
}

// One CTA per patch of the level: counts in shared memory (NAMRX^3 ints),
// candidates from the bins covering the patch widened by two fine cells
// (a superset of the particles the FLOOR test keeps, for cells wider than
// the float spacing of the coordinates).
__global__ void __launch_bounds__(PD_BLOCK)
k_mesh_patch_counts(const int32_t* __restrict__ pn, const float* __restrict__ pr, int np, Bins B,
                    const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
                    int irpa, float dxpa, int refine_thr, int boramr, EspEnds E, int32_t* __restrict__ out) {
  extern __shared__ int32_t s_cnt[];
  const int ip = blockIdx.x;
  const int n1 = pn[ip], n2 = pn[np + ip], n3 = pn[2 * np + ip];
  for (int q = threadIdx.x; q < NA * NA * NA; q += blockDim.x) s_cnt[q] = 0;
  __syncthreads();
  // XL = PATCHRX - DXPA (grids.f:358-360)
  const float xl = __fsub_rn(pr[ip], dxpa), yl = __fsub_rn(pr[np + ip], dxpa), zl = __fsub_rn(pr[2 * np + ip], dxpa);
  const float pad = 2.0f * dxpa;
  const int bx0 = bin_of(xl - pad, B.xl, B.bsz, B.nb), bx1 = bin_of(xl + (float)(n1 + 2) * dxpa, B.xl, B.bsz, B.nb);
  const int by0 = bin_of(yl - pad, B.xl, B.bsz, B.nb), by1 = bin_of(yl + (float)(n2 + 2) * dxpa, B.xl, B.bsz, B.nb);
  const int bz0 = bin_of(zl - pad, B.xl, B.bsz, B.nb), bz1 = bin_of(zl + (float)(n3 + 2) * dxpa, B.xl, B.bsz, B.nb);
  for (int bz = bz0; bz <= bz1; bz++)
    for (int by = by0; by <= by1; by++) {
      const int lo = B.start[(bz * B.nb + by) * B.nb + bx0], hi = B.start[(bz * B.nb + by) * B.nb + bx1 + 1];
      for (int t = lo + threadIdx.x; t < hi; t += blockDim.x) {
        const int p = B.idx[t];
        // IX = FLOOR((RXPA-XL)/DXPA)+1 kept when 1 <= IX <= N1
        const float vx = __fdiv_rn(__fsub_rn(x[p], xl), dxpa);
        if (!(vx >= 0.0f && vx < (float)n1)) continue;
        const float vy = __fdiv_rn(__fsub_rn(y[p], yl), dxpa);
        if (!(vy >= 0.0f && vy < (float)n2)) continue;
        const float vz = __fdiv_rn(__fsub_rn(z[p], zl), dxpa);
        if (!(vz >= 0.0f && vz < (float)n3)) continue;
        const int w = plev_of(p, E) <= irpa ? 1 : refine_thr;
        atomicAdd(&s_cnt[((int)vz * NA + (int)vy) * NA + (int)vx], w);
      }
    }
  __syncthreads();
  int32_t* o = out + (size_t)ip * NA * NA * NA;
  for (int q = threadIdx.x; q < NA * NA * NA; q += blockDim.x) {
    const int ix = q % NA + 1, jy = (q / NA) % NA + 1, kz = q / (NA * NA) + 1;
    int v = s_cnt[q];
    if (ix > n1 || jy > n2 || kz > n3 || ix <= boramr || ix >= n1 - boramr + 1 || jy <= boramr ||
        jy >= n2 - boramr + 1 || kz <= boramr || kz >= n3 - boramr + 1)
      v = 0;
    o[q] = v;
  }
}

static int esp_ends(const int32_t* npart_esp, EspEnds* E) {
  int64_t acc = 0;
  for (int s = 0; s < ASOHF_N_ESP; s++) {
    if (npart_esp[s] < 0) return ASOHF_ERR_INVALID;
    acc += npart_esp[s];
    E->e[s] = acc;
  }
  return ASOHF_OK;
}

extern "C" int asohf_mesh_base_counts(asohf_ctx* c, int nx, float dx, int refine_thr, int bor,
                                      const int32_t* npart_esp, int32_t* cr0, int on_device) {
  if (!c || nx <= 0 || !npart_esp || !cr0) return ASOHF_ERR_INVALID;
  EspEnds E;
  ASOHF_CHECK(esp_ends(npart_esp, &E));
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  const int64_t g = (int64_t)nx * nx * nx, n = c->p.n;
  ASOHF_CHECK(arena_reserve(c, 4 * (size_t)g + 4096));
  int32_t* d = on_device ? cr0 : (int32_t*)arena_alloc(c, 4 * (size_t)g);
  if (!d) return ASOHF_ERR_CAPACITY;
  ASOHF_CUDA(cudaMemsetAsync(d, 0, 4 * (size_t)g, c->stream));
  const float xl = -((float)nx * dx / 2.0f);  // XL = -NX*DX/2.
  int kt_ = ktime_begin(c, "mesh_base_counts");
  if (n > 0) {
    k_mesh_base_counts<<<grid_for(n, 256, c->num_sms * 16), 256, 0, c->stream>>>(c->p.x, c->p.y, c->p.z, n, nx, xl,
                                                                                  dx, refine_thr, E, d);
    c->launches++;
  }
  k_mesh_border<<<grid_for(g, 256), 256, 0, c->stream>>>(d, nx, bor);
  c->launches++;
  ktime_end(c, kt_);
  ASOHF_CUDA(cudaGetLastError());
  if (!on_device) ASOHF_CUDA(cudaMemcpyAsync(cr0, d, 4 * (size_t)g, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  return ASOHF_OK;
}

extern "C" int asohf_mesh_patch_counts(asohf_ctx* c, int nx, float lado0, float dx, int irpa, int refine_thr,
                                       int boramr, const int32_t* npart_esp, int npatch, const int32_t* patchnx,
                                       const int32_t* patchny, const int32_t* patchnz, const float* patchrx,
                                       const float* patchry, const float* patchrz, int32_t* cr01, int on_device) {
  if (!c || nx <= 0 || irpa < 1 || npatch < 0 || !npart_esp || (npatch > 0 && (!patchnx || !patchny || !patchnz ||
      !patchrx || !patchry || !patchrz || !cr01)))
    return ASOHF_ERR_INVALID;
  EspEnds E;
  ASOHF_CHECK(esp_ends(npart_esp, &E));
  for (int q = 0; q < npatch; q++)
    if (patchnx[q] < 1 || patchnx[q] > NA || patchny[q] < 1 || patchny[q] > NA || patchnz[q] < 1 || patchnz[q] > NA)
      return ASOHF_ERR_INVALID;
  if (npatch == 0) return ASOHF_OK;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  const int64_t n = c->p.n;
  const size_t outb = 4 * (size_t)npatch * NA * NA * NA;
  ASOHF_CHECK(arena_reserve(c, (on_device ? 0 : outb) + 24 * (size_t)npatch + bins_bytes(n, lado0, dx, 2) + 8192));
  int32_t* pn = (int32_t*)arena_alloc(c, 12 * (size_t)npatch);
  float* pr = (float*)arena_alloc(c, 12 * (size_t)npatch);
  int32_t* d = on_device ? cr01 : (int32_t*)arena_alloc(c, outb);
  if (!pn || !pr || !d) return ASOHF_ERR_CAPACITY;
  const int32_t* hn[3] = {patchnx, patchny, patchnz};
  const float* hr[3] = {patchrx, patchry, patchrz};
  for (int a = 0; a < 3; a++) {
    ASOHF_CUDA(cudaMemcpyAsync(pn + (size_t)a * npatch, hn[a], 4 * (size_t)npatch, cudaMemcpyHostToDevice, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(pr + (size_t)a * npatch, hr[a], 4 * (size_t)npatch, cudaMemcpyHostToDevice, c->stream));
  }
  Bins B;
  ASOHF_CHECK(build_bins(c, lado0, dx, 2, &B));
  const float dxpa = ldexpf(dx, -irpa);  // DX/(2.0**IRPA), exact
  const size_t smem = sizeof(int32_t) * NA * NA * NA;
  ASOHF_CUDA(cudaFuncSetAttribute(k_mesh_patch_counts, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int kt_ = ktime_begin(c, "mesh_patch_counts");
  k_mesh_patch_counts<<<npatch, PD_BLOCK, smem, c->stream>>>(pn, pr, npatch, B, c->p.x, c->p.y, c->p.z, irpa, dxpa,
                                                             refine_thr, boramr, E, d);
  c->launches++;
  ktime_end(c, kt_);
  ASOHF_CUDA(cudaGetLastError());
  if (!on_device) ASOHF_CUDA(cudaMemcpyAsync(cr01, d, outb, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  return ASOHF_OK;
}

// ------------------------------------------------------------ VEINSGRID_REDUCED
// grids.f:1771-2073.  Patch I (in order) marks the cells of each neighbour J
// that face an unmarked cell of I; a row reads only I's marks and writes
// only its neighbours', and the neighbour relation (intersecting cell boxes
// on the level's grid) is symmetric.  So rows whose patches do not
// intersect commute, and the rows are replayed in waves: a row's wave is
// one past the latest wave of its lower-index neighbours, and one launch
// takes a wave with one CTA per row.  The result equals the sequential one.

__device__ __forceinline__ int veins_int(float v) { return (int)__fadd_rn(v, 0.5f); }  // INT(v+0.5)

// Lower cell of each patch on the level's grid (IG1, JG1, KG1).
__global__ void k_veins_box(const int32_t* __restrict__ pn, const float* __restrict__ pr, int np, float dxpa,
                            float fix, int32_t* __restrict__ g1) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 3 * np) return;
  const float r1 = __fsub_rn(pr[q], __fmul_rn(0.5f, dxpa));
  g1[q] = veins_int(__fdiv_rn(__fsub_rn(r1, fix), dxpa)) + 1;
}

__device__ __forceinline__ bool veins_meet(const int32_t* g1, const int32_t* pn, int np, int i, int j) {
  bool ok = true;
  for (int a = 0; a < 3; a++) {
    const int gi = g1[a * np + i], gj = g1[a * np + j];
    ok = ok && gi <= gj + pn[a * np + j] - 1 && gj <= gi + pn[a * np + i] - 1;
  }
  return ok;
}

// Neighbours of each patch, in index order: counts (fill == nullptr) or the list.
__global__ void k_veins_neighbours(const int32_t* __restrict__ g1, const int32_t* __restrict__ pn, int np,
                                   int32_t* __restrict__ cnt, const int32_t* __restrict__ off,
                                   int32_t* __restrict__ fill) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  int k = 0;
  for (int j = 0; j < np; j++) {
    if (j == i || !veins_meet(g1, pn, np, i, j)) continue;
    if (fill) fill[off[i] + k] = j;
    k++;
  }
  if (!fill) cnt[i] = k;
}

// The overlap corners of one axis (the four cases of grids.f:1965-2026).
__device__ __forceinline__ void veins_axis_d(float r1, float r2, float rr1, float rr2, float dxpa, int n, int nn,
                                             int* c1, int* c2, int* cc1, int* cc2) {
  if (rr1 >= r1 && rr2 <= r2) {
    *c1 = veins_int(__fdiv_rn(__fsub_rn(rr1, r1), dxpa)) + 1;
    *c2 = veins_int(__fdiv_rn(__fsub_rn(rr2, r1), dxpa)) + 1;
    *cc1 = 1;
    *cc2 = nn;
  }
  if (rr1 >= r1 && rr2 > r2) {
    *c1 = veins_int(__fdiv_rn(__fsub_rn(rr1, r1), dxpa)) + 1;
    *c2 = n;
    *cc1 = 1;
    *cc2 = veins_int(__fdiv_rn(__fsub_rn(r2, rr1), dxpa)) + 1;
  }
  if (rr2 <= r2 && rr1 < r1) {
    *c1 = 1;
    *c2 = veins_int(__fdiv_rn(__fsub_rn(rr2, r1), dxpa)) + 1;
    *cc1 = veins_int(__fdiv_rn(__fsub_rn(r1, rr1), dxpa)) + 1;
    *cc2 = nn;
  }
  if (rr1 < r1 && rr2 > r2) {
    *c1 = 1;
    *c2 = n;
    *cc1 = veins_int(__fdiv_rn(__fsub_rn(r1, rr1), dxpa)) + 1;
    *cc2 = veins_int(__fdiv_rn(__fsub_rn(r2, rr1), dxpa)) + 1;
  }
}

// One CTA per row of the wave: patch I against each neighbour J.
__global__ void __launch_bounds__(256) k_veins_rows(const int32_t* __restrict__ rows, const int32_t* __restrict__ off,
                                                    const int32_t* __restrict__ nb, const int32_t* __restrict__ pn,
                                                    const float* __restrict__ pr, int np, float dxpa,
                                                    uint8_t* __restrict__ solap, int32_t* __restrict__ cr01,
                                                    int32_t* __restrict__ conta11) {
  const int i = rows[blockIdx.x];
  const size_t pc = (size_t)NA * NA * NA;
  float r1[3], r2[3];
  int n[3];
  for (int a = 0; a < 3; a++) {
    n[a] = pn[a * np + i];
    r1[a] = __fsub_rn(pr[a * np + i], __fmul_rn(0.5f, dxpa));
    r2[a] = __fadd_rn(r1[a], __fmul_rn((float)(n[a] - 1), dxpa));
  }
  for (int k = off[i]; k < off[i + 1]; k++) {
    const int j = nb[k];
    int c1[3], c2[3], cc1[3], cc2[3], e[3];
    for (int a = 0; a < 3; a++) {
      const int nn = pn[a * np + j];
      const float rr1 = __fsub_rn(pr[a * np + j], __fmul_rn(0.5f, dxpa));
      const float rr2 = __fadd_rn(rr1, __fmul_rn((float)(nn - 1), dxpa));
      c1[a] = c2[a] = cc1[a] = cc2[a] = 0;
      veins_axis_d(r1[a], r2[a], rr1, rr2, dxpa, n[a], nn, &c1[a], &c2[a], &cc1[a], &cc2[a]);
      e[a] = cc2[a] - cc1[a] + 1;
    }
    const int prod = e[2] * e[1] * e[0];
    const float ov = __fdiv_rn(__fdiv_rn(__fdiv_rn(fabsf((float)prod), (float)pn[j]), (float)pn[np + j]),
                               (float)pn[2 * np + j]);
    if (!(ov > 0.1f) || e[0] <= 0 || e[1] <= 0 || e[2] <= 0) continue;
    const int ncell = e[0] * e[1] * e[2];
    for (int q = threadIdx.x; q < ncell; q += blockDim.x) {
      const int ii = cc1[0] + q % e[0], jj = cc1[1] + (q / e[0]) % e[1], kk = cc1[2] + q / (e[0] * e[1]);
      const int ix = ii - cc1[0] + c1[0], jy = jj - cc1[1] + c1[1], kz = kk - cc1[2] + c1[2];
      if (ii < 1 || ii > NA || jj < 1 || jj > NA || kk < 1 || kk > NA || ix < 1 || ix > NA || jy < 1 || jy > NA ||
          kz < 1 || kz > NA)
        continue;  // outside the NAMRX^3 arrays
      const size_t qi = (size_t)i * pc + ((size_t)(kz - 1) * NA + (jy - 1)) * NA + (ix - 1);
      const size_t qj = (size_t)j * pc + ((size_t)(kk - 1) * NA + (jj - 1)) * NA + (ii - 1);
      if (solap[qi] == 0) {
        solap[qj] = 1;
        cr01[qj] = 0;
        if (conta11) conta11[qj] = 0;
      }
    }
  }
}

extern "C" int asohf_veinsgrid_reduced(asohf_ctx* c, int ir, float dx, float radx1, int npatch,
                                       const int32_t* patchnx, const int32_t* patchny, const int32_t* patchnz,
                                       const float* patchrx, const float* patchry, const float* patchrz,
                                       int max_neighbours, int32_t* cr01, int32_t* conta11, int on_device) {
  if (!c || ir < 1 || npatch < 0 || max_neighbours < 0 ||
      (npatch > 0 && (!patchnx || !patchny || !patchnz || !patchrx || !patchry || !patchrz || !cr01)))
    return ASOHF_ERR_INVALID;
  for (int q = 0; q < npatch; q++)
    if (patchnx[q] < 1 || patchnx[q] > NA || patchny[q] < 1 || patchny[q] > NA || patchnz[q] < 1 || patchnz[q] > NA)
      return ASOHF_ERR_INVALID;
  if (npatch == 0) return ASOHF_OK;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  const int np = npatch;
  const size_t pc = (size_t)NA * NA * NA;
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, (int32_t*)nullptr, (int32_t*)nullptr, np + 1);
  const size_t host_b = on_device ? 0 : 4 * pc * (size_t)np * (conta11 ? 2 : 1);
  ASOHF_CHECK(arena_reserve(c, host_b + pc * (size_t)np + 48 * (size_t)np + tb + 16 * 256 + 4096));
  int32_t* pn = (int32_t*)arena_alloc(c, 12 * (size_t)np);
  float* pr = (float*)arena_alloc(c, 12 * (size_t)np);
  int32_t* g1 = (int32_t*)arena_alloc(c, 12 * (size_t)np);
  int32_t* cnt = (int32_t*)arena_alloc(c, 4 * (size_t)np + 4);
  int32_t* off = (int32_t*)arena_alloc(c, 4 * (size_t)np + 4);
  int32_t* rows = (int32_t*)arena_alloc(c, 4 * (size_t)np);
  void* tmp = arena_alloc(c, tb);
  uint8_t* solap = (uint8_t*)arena_alloc(c, pc * (size_t)np);
  int32_t* dcr = on_device ? cr01 : (int32_t*)arena_alloc(c, 4 * pc * (size_t)np);
  int32_t* dct = (!conta11 || on_device) ? conta11 : (int32_t*)arena_alloc(c, 4 * pc * (size_t)np);
  if (!pn || !pr || !g1 || !cnt || !off || !rows || !tmp || !solap || !dcr || (conta11 && !dct))
    return ASOHF_ERR_CAPACITY;
  const int32_t* hn[3] = {patchnx, patchny, patchnz};
  const float* hr[3] = {patchrx, patchry, patchrz};
  for (int a = 0; a < 3; a++) {
    ASOHF_CUDA(cudaMemcpyAsync(pn + (size_t)a * np, hn[a], 4 * (size_t)np, cudaMemcpyHostToDevice, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(pr + (size_t)a * np, hr[a], 4 * (size_t)np, cudaMemcpyHostToDevice, c->stream));
  }
  if (!on_device) {
    ASOHF_CUDA(cudaMemcpyAsync(dcr, cr01, 4 * pc * (size_t)np, cudaMemcpyHostToDevice, c->stream));
    if (conta11) ASOHF_CUDA(cudaMemcpyAsync(dct, conta11, 4 * pc * (size_t)np, cudaMemcpyHostToDevice, c->stream));
  }
  ASOHF_CUDA(cudaMemsetAsync(solap, 0, pc * (size_t)np, c->stream));
  ASOHF_CUDA(cudaMemsetAsync(cnt, 0, 4 * (size_t)np + 4, c->stream));
  const float dxpa = ldexpf(dx, -ir);                       // DX/(2.**IR)
  const float fix = radx1 - dx * 0.5f + 0.5f * dxpa;        // RXFIX
  int kt_ = ktime_begin(c, "veinsgrid_reduced");
  k_veins_box<<<(3 * np + 255) / 256, 256, 0, c->stream>>>(pn, pr, np, dxpa, fix, g1);
  k_veins_neighbours<<<(np + 127) / 128, 128, 0, c->stream>>>(g1, pn, np, cnt, nullptr, nullptr);
  ASOHF_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, off, np + 1, c->stream));
  c->launches += 3;
  std::vector<int32_t> hoff(np + 1);
  ASOHF_CUDA(cudaMemcpyAsync(hoff.data(), off, 4 * (size_t)(np + 1), cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  const int ne = hoff[np];
  int maxnv = 0;
  for (int i = 0; i < np; i++) maxnv = std::max(maxnv, hoff[i + 1] - hoff[i]);
  if (maxnv > max_neighbours) {
    ktime_end(c, kt_);
    return ASOHF_ERR_CAPACITY;  // the reference stops: more neighbours than NPALEV2
  }
  int32_t* nb = nullptr;
  if (ne > 0) {
    // the list lives in the segment buffer (the arena is sized before the count is known)
    ASOHF_CHECK(seg_reserve(c, 4 * (size_t)ne + 256));
    nb = (int32_t*)seg_alloc(c, 4 * (size_t)ne);
    if (!nb) return ASOHF_ERR_CAPACITY;
    k_veins_neighbours<<<(np + 127) / 128, 128, 0, c->stream>>>(g1, pn, np, nullptr, off, nb);
    c->launches++;
  }
  std::vector<int32_t> hnb(ne > 0 ? ne : 1);
  if (ne > 0) ASOHF_CUDA(cudaMemcpyAsync(hnb.data(), nb, 4 * (size_t)ne, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  // waves: one past the latest wave of the lower-index neighbours
  std::vector<int32_t> wave(np, 0);
  int nwave = 0;
  for (int i = 0; i < np; i++) {
    int w = 0;
    for (int k = hoff[i]; k < hoff[i + 1]; k++)
      if (hnb[k] < i) w = std::max(w, wave[hnb[k]] + 1);
    wave[i] = w;
    nwave = std::max(nwave, w + 1);
  }
  std::vector<int32_t> wstart(nwave + 1, 0), horder(np);
  for (int i = 0; i < np; i++) wstart[wave[i] + 1]++;
  for (int w = 0; w < nwave; w++) wstart[w + 1] += wstart[w];
  {
    std::vector<int32_t> fillp(wstart.begin(), wstart.end() - 1);
    for (int i = 0; i < np; i++) horder[fillp[wave[i]]++] = i;
  }
  ASOHF_CUDA(cudaMemcpyAsync(rows, horder.data(), 4 * (size_t)np, cudaMemcpyHostToDevice, c->stream));
  for (int w = 0; w < nwave; w++) {
    const int nr = wstart[w + 1] - wstart[w];
    if (nr <= 0) continue;
    k_veins_rows<<<nr, 256, 0, c->stream>>>(rows + wstart[w], off, nb, pn, pr, np, dxpa, solap, dcr, dct);
    c->launches++;
  }
  ktime_end(c, kt_);
  ASOHF_CUDA(cudaGetLastError());
  if (!on_device) {
    ASOHF_CUDA(cudaMemcpyAsync(cr01, dcr, 4 * pc * (size_t)np, cudaMemcpyDeviceToHost, c->stream));
    if (conta11) ASOHF_CUDA(cudaMemcpyAsync(conta11, dct, 4 * pc * (size_t)np, cudaMemcpyDeviceToHost, c->stream));
  }
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  return ASOHF_OK;
}
