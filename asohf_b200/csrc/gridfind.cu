// gridfind.cu -- HALOFIND_GRID at the base level (haloes_grids.f:287-582) on
// the device, for a base grid without AMR recentering.
//
// The reference walks the candidate peaks of U1 (strict maxima over the six
// face neighbours above CONTRASTEC/6) from the densest down; a peak whose
// cell a kept halo has already covered (CONTA = 0) is skipped, any other one
// becomes a halo that grows in spherical shells (R_EXT = 0.8 DX, then
// MAX(R_EXT + 0.2 DX, 1.05 R_EXT)) until its mean density falls to
// CONTRASTEC, and marks the cells of its shells covered.
//
// A halo's growth reads U1 only; CONTA decides whether a peak starts a halo
// and nothing else.  So the candidates are taken in their sorted order in
// chunks: every candidate of a chunk whose peak is not yet covered grows at
// once (one warp each), then one warp replays the chunk in order -- a
// candidate is kept iff no kept candidate before it in the chunk covers its
// peak (the pairs come from a parallel test of the chunk's pairs) -- and the
// kept haloes are written to the catalogue and mark CONTA for the next
// chunk.  The result is the sequential one.
//
// Arithmetic follows the Fortran statement by statement: REAL*4 distances,
// box bounds INT((X-RADX(1))/DX+0.5)+1, and the shell sums added one cell
// at a time in (K, J, I) order (the warp tests 32 cells of a row at once and
// then adds the ones inside the shell in order).  The shell radii are the
// same sequence for every halo, so a halo is described by its shell count;
// the cells it covers are those whose distance falls in one of its shells
// and which lie in that shell's box.  Rows of a box are visited only where
// they can meet the shell (their distance bounds with a relative margin of
// 1e-4, far above the float rounding), which keeps the result exact.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <cub/device/device_radix_sort.cuh>

#include "common.cuh"

namespace {

constexpr int GF_CHUNK = 1024;  // candidates per ordered chunk
constexpr int GF_MAXSH = 1024;  // shell radii kept in the table
constexpr int GF_WORDS = GF_CHUNK / 32;

struct GridIn {
  const float* u;     // U1(NX,NX,NX), column-major
  const float* radx;  // RADX(0:NX+1)
  const float* R;     // R_EXT of shell t (t = 0, 1, ...)
  int nR;             // entries of R; R[nR-1] > BOUND (or the table is full)
  int nx;
  float dx, volcell, bound;
  float contrastec, rote, rodo, re03, rete3;  // RE0**3 and RETE**3 as (x*x)*x
};

struct GridChunk {
  const unsigned long long* keys;  // sorted candidate keys
  int64_t c0;                      // first candidate of the chunk
  int m;                           // candidates in the chunk
  int32_t* nsh;                    // shells grown: 0 covered before the chunk, -1 past BOUND
  float* masa;
  float* cm;                       // 3 per member
  uint32_t* pairs;                 // GF_CHUNK x GF_WORDS: bit d of row c = d covers c's peak
  int32_t* slot;                   // catalogue row of a kept member, -1 otherwise
  int32_t* state;                  // [0] haloes kept so far, [1] error status
};

struct GridCat {  // the catalogue columns the grid finder writes (device)
  int capacity;
  int32_t *realclus, *levhal, *patchclus;
  float *x, *y, *z, *radio, *masa, *xcm, *ycm, *zcm;
};

__device__ __forceinline__ int cell_of(unsigned long long key, int nx, int* i, int* j, int* k) {
  const uint32_t lin = 0xffffffffu - (uint32_t)(key & 0xffffffffull);
  *i = (int)(lin % (uint32_t)nx) + 1;
  *j = (int)((lin / (uint32_t)nx) % (uint32_t)nx) + 1;
  *k = (int)(lin / ((uint32_t)nx * (uint32_t)nx)) + 1;
  return (int)lin;
}

// NX1 = INT(((BASX-RADX(1))/DX)+0.5)+1, clamped (haloes_grids.f:491-497)
__device__ __forceinline__ int box_lo(float c, float r, float radx1, float dx) {
  const int v = (int)__fadd_rn(__fdiv_rn(__fsub_rn(__fsub_rn(c, r), radx1), dx), 0.5f) + 1;
  return v < 1 ? 1 : v;
}
__device__ __forceinline__ int box_hi(float c, float r, float radx1, float dx, int nx) {
  const int v = (int)__fadd_rn(__fdiv_rn(__fsub_rn(__fadd_rn(c, r), radx1), dx), 0.5f) + 1;
  return v > nx ? nx : v;
}

__device__ __forceinline__ float dist3f(float dx_, float dy_, float dz_) {
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx_, dx_), __fmul_rn(dy_, dy_)), __fmul_rn(dz_, dz_)));
}

// Whether a halo centred on (xc, yc, zc) with `nsh` shells covers cell
// (i, j, k): its distance lies in some shell t < nsh and the cell is inside
// that shell's box.
__device__ bool covers(const GridIn& G, float xc, float yc, float zc, int nsh, int i, int j, int k) {
  if (nsh <= 0) return false;
  const float aa = dist3f(__fsub_rn(G.radx[i], xc), __fsub_rn(G.radx[j], yc), __fsub_rn(G.radx[k], zc));
  if (!(aa < G.R[nsh - 1])) return false;
  int lo = 0, hi = nsh - 1;  // first t with aa < R[t]
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (aa < G.R[mid]) hi = mid; else lo = mid + 1;
  }
  const float r = G.R[lo], rx1 = G.radx[1];
  return i >= box_lo(xc, r, rx1, G.dx) && i <= box_hi(xc, r, rx1, G.dx, G.nx) && j >= box_lo(yc, r, rx1, G.dx) &&
         j <= box_hi(yc, r, rx1, G.dx, G.nx) && k >= box_lo(zc, r, rx1, G.dx) && k <= box_hi(zc, r, rx1, G.dx, G.nx);
}

// The i range of row (j, k) that can hold cells with r_in <= aa < r_out
// (up to two runs: left and right of the inner sphere's chord), as index
// bounds in the box [ilo, ihi]; margins keep every such cell inside.
__device__ __forceinline__ void row_runs(const GridIn& G, float xc, float s2, float r_in, float r_out, int ilo,
                                         int ihi, int* a0, int* a1, int* b0, int* b1) {
  const float o2 = __fmul_rn(__fmul_rn(r_out, r_out), 1.0001f);
  const float half_out = sqrtf(fmaxf(o2 - s2, 0.0f)) + G.dx;
  float half_in = -1.0f;
  const float i2 = __fmul_rn(__fmul_rn(r_in, r_in), 0.9999f);
  if (i2 > s2) half_in = sqrtf(i2 - s2) - G.dx;
  const float rx1 = G.radx[1];
  // cell i has centre RADX(1) + (i-1) DX
  int lo = (int)floorf((xc - half_out - rx1) / G.dx) + 1, hi = (int)ceilf((xc + half_out - rx1) / G.dx) + 1;
  lo = max(lo, ilo);
  hi = min(hi, ihi);
  if (half_in > 0.0f) {
    const int in0 = (int)ceilf((xc - half_in - rx1) / G.dx) + 1, in1 = (int)floorf((xc + half_in - rx1) / G.dx) + 1;
    if (in0 <= in1) {  // cells strictly inside the inner sphere are skipped
      *a0 = lo; *a1 = min(hi, in0 - 1);
      *b0 = max(lo, in1 + 1); *b1 = hi;
      return;
    }
  }
  *a0 = lo; *a1 = hi;
  *b0 = 1; *b1 = 0;
}

// CONTA(i,j,k) = 1 on the interior cells (BOR = 1), 0 on the border.
__global__ void k_grid_conta_init(uint8_t* __restrict__ conta, int nx) {
  const int64_t g = (int64_t)nx * nx * nx;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < g; c += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % nx) + 1, j = (int)((c / nx) % nx) + 1, k = (int)(c / ((int64_t)nx * nx)) + 1;
    conta[c] = (i >= 2 && i <= nx - 1 && j >= 2 && j <= nx - 1 && k >= 2 && k <= nx - 1) ? 1 : 0;
  }
}

// Candidate peaks (haloes_grids.f:308-330): interior cells with U >= thr
// that exceed their six face neighbours.  keys == nullptr: count only.
// Key: REAL*4 bits of 1/U (ascending) then the cell's (K, J, I) position,
// descending -- ARGSORT's order of 1/DDD (num.f:150-203, equal keys by
// descending position).
__global__ void k_grid_peaks(const float* __restrict__ u, int nx, float thr, unsigned long long* __restrict__ keys,
                             int64_t cap, unsigned long long* __restrict__ n_out) {
  const int64_t g = (int64_t)nx * nx * nx;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < g; c += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % nx) + 1, j = (int)((c / nx) % nx) + 1, k = (int)(c / ((int64_t)nx * nx)) + 1;
    if (i < 2 || i > nx - 1 || j < 2 || j > nx - 1 || k < 2 || k > nx - 1) continue;
    const float b = u[c];
    if (!(b >= thr)) continue;
    const int64_t sx = 1, sy = nx, sz = (int64_t)nx * nx;
    if (!(__fsub_rn(u[c + sx], b) < 0.0f)) continue;
    if (!(__fsub_rn(u[c + sy], b) < 0.0f)) continue;
    if (!(__fsub_rn(u[c + sz], b) < 0.0f)) continue;
    if (!(__fsub_rn(b, u[c - sx]) > 0.0f)) continue;
    if (!(__fsub_rn(b, u[c - sy]) > 0.0f)) continue;
    if (!(__fsub_rn(b, u[c - sz]) > 0.0f)) continue;
    const unsigned long long pos = atomicAdd(n_out, 1ull);
    if (keys && (int64_t)pos < cap)
      keys[pos] = ((unsigned long long)__float_as_uint(__fdiv_rn(1.0f, b)) << 32) |
                  (unsigned long long)(0xffffffffu - (uint32_t)c);
  }
}

// Growth of the chunk's uncovered candidates (haloes_grids.f:470-560), one
// warp each.
__global__ void __launch_bounds__(256) k_grid_grow(GridIn G, GridChunk C, const uint8_t* __restrict__ conta) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= C.m) return;
  int ic, jc, kc;
  const int lin = cell_of(C.keys[C.c0 + w], G.nx, &ic, &jc, &kc);
  if (conta[lin] != 1) {
    if (lane == 0) C.nsh[w] = 0;
    return;
  }
  const float xc = G.radx[ic], yc = G.radx[jc], zc = G.radx[kc], rx1 = G.radx[1];
  const int nx = G.nx;
  const float thr = __fmul_rn(G.contrastec, G.rote);
  float basx = 0.0f, basy = 0.0f, basz = 0.0f, basdelta = 0.0f, basmass = 0.0f, basvol = 0.0f;
  float delta = __fmul_rn(__fmul_rn(10.0f, G.contrastec), G.rote);
  int t = -1;
  bool bad = false;
  while (delta > thr) {
    if (t >= 0 && !(G.R[t] <= G.bound)) { bad = true; break; }  // STOP 1: growing not converged
    t++;
    if (t >= G.nR) { bad = true; break; }
    const float r_ext = G.R[t], r_int = t == 0 ? 0.0f : G.R[t - 1];
    const int lx = box_lo(xc, r_ext, rx1, G.dx), hx = box_hi(xc, r_ext, rx1, G.dx, nx);
    const int ly = box_lo(yc, r_ext, rx1, G.dx), hy = box_hi(yc, r_ext, rx1, G.dx, nx);
    const int lz = box_lo(zc, r_ext, rx1, G.dx), hz = box_hi(zc, r_ext, rx1, G.dx, nx);
    // BASX..BASZ restart from the box's upper bounds every shell (haloes_grids.f:513-518)
    basx = __fadd_rn(xc, r_ext);
    basy = __fadd_rn(yc, r_ext);
    basz = __fadd_rn(zc, r_ext);
    float shell = 0.0f;
    const float o2m = __fmul_rn(__fmul_rn(r_ext, r_ext), 1.0001f);
    for (int k = lz; k <= hz; k++) {
      const float rzk = G.radx[k], ddz = __fsub_rn(rzk, zc);
      for (int j = ly; j <= hy; j++) {
        const float ryj = G.radx[j], ddy = __fsub_rn(ryj, yc);
        const float s2 = __fadd_rn(__fmul_rn(ddy, ddy), __fmul_rn(ddz, ddz));
        if (s2 > o2m) continue;  // no cell of this row reaches the shell
        int a0, a1, b0, b1;
        row_runs(G, xc, s2, r_int, r_ext, lx, hx, &a0, &a1, &b0, &b1);
        for (int run = 0; run < 2; run++) {
          const int r0 = run ? b0 : a0, r1 = run ? b1 : a1;
          for (int i0 = r0; i0 <= r1; i0 += 32) {
            const int i = i0 + lane;
            bool in = false;
            float b = 0.0f, rxi = 0.0f;
            if (i <= r1) {
              rxi = G.radx[i];
              const float aa = dist3f(__fsub_rn(rxi, xc), ddy, ddz);
              in = aa >= r_int && aa < r_ext;
              if (in) b = __fmul_rn(G.u[((size_t)(k - 1) * nx + (j - 1)) * nx + (i - 1)], G.volcell);
            }
            unsigned msk = __ballot_sync(FULL, in);
            while (msk) {  // the cells inside the shell, in I order
              const int src = __ffs(msk) - 1;
              msk &= msk - 1;
              const float bb = __shfl_sync(FULL, b, src), xi = __shfl_sync(FULL, rxi, src);
              basvol = __fadd_rn(basvol, G.volcell);
              shell = __fadd_rn(shell, bb);
              basx = __fadd_rn(basx, __fmul_rn(xi, bb));
              basy = __fadd_rn(basy, __fmul_rn(ryj, bb));
              basz = __fadd_rn(basz, __fmul_rn(rzk, bb));
              basdelta = __fadd_rn(basdelta, bb);
            }
          }
        }
      }
    }
    basmass = __fadd_rn(basmass, __fmul_rn(__fmul_rn(shell, G.rodo), G.re03));
    if (basvol > 0.0f) delta = __fdiv_rn(basmass, __fmul_rn(basvol, G.rete3));
  }
  if (lane == 0) {
    C.nsh[w] = bad ? -1 : t + 1;
    C.masa[w] = basmass;
    C.cm[3 * w] = __fdiv_rn(basx, basdelta);
    C.cm[3 * w + 1] = __fdiv_rn(basy, basdelta);
    C.cm[3 * w + 2] = __fdiv_rn(basz, basdelta);
  }
}

// Pairs of the chunk: bit d of row c when member d (before c) covers the
// peak cell of member c.  One thread per (c, word of 32 d).
__global__ void k_grid_pairs(GridIn G, GridChunk C) {
  const int c = blockIdx.x, wd = threadIdx.x;
  if (c >= C.m || wd >= GF_WORDS) return;
  uint32_t bits = 0u;
  if (C.nsh[c] != 0) {
    int ic, jc, kc;
    cell_of(C.keys[C.c0 + c], G.nx, &ic, &jc, &kc);
    for (int q = 0; q < 32; q++) {
      const int d = wd * 32 + q;
      if (d >= c) break;
      const int n = C.nsh[d];
      if (n <= 0) continue;
      int id, jd, kd;
      cell_of(C.keys[C.c0 + d], G.nx, &id, &jd, &kd);
      if (covers(G, G.radx[id], G.radx[jd], G.radx[kd], n, ic, jc, kc)) bits |= 1u << q;
    }
  }
  C.pairs[(size_t)c * GF_WORDS + wd] = bits;
}

// The chunk in order (one warp): a member not covered before the chunk is
// kept iff no kept member before it covers its peak; kept members take the
// next catalogue rows.  A kept member that grew past BOUND stops the finder
// (the reference's STOP 1); so does a full catalogue.
__global__ void k_grid_replay(GridChunk C, int capacity) {
  const int lane = threadIdx.x;
  uint32_t kept = 0u;  // lane holds word `lane` of the kept set
  int nk = C.state[0];
  int err = C.state[1];
  for (int c = 0; c < C.m; c++) {
    int s = -1;
    if (err == 0 && C.nsh[c] != 0) {
      const bool hit = (C.pairs[(size_t)c * GF_WORDS + lane] & kept) != 0u;
      if (!__any_sync(0xffffffffu, hit)) {
        if (C.nsh[c] < 0) err = ASOHF_ERR_NOT_CONVERGED;
        else if (nk >= capacity) err = ASOHF_ERR_CAPACITY;
        else {
          s = nk++;
          if (lane == (c >> 5)) kept |= 1u << (c & 31);
        }
      }
    }
    if (lane == 0) C.slot[c] = s;
  }
  if (lane == 0) { C.state[0] = nk; C.state[1] = err; }
}

// Kept members: their catalogue rows, then CONTA = 0 over the cells they
// cover (one CTA each).
__global__ void __launch_bounds__(256) k_grid_commit(GridIn G, GridChunk C, GridCat K, uint8_t* __restrict__ conta) {
  const int c = blockIdx.x;
  if (c >= C.m) return;
  const int s = C.slot[c];
  if (s < 0) return;
  int ic, jc, kc;
  cell_of(C.keys[C.c0 + c], G.nx, &ic, &jc, &kc);
  const float xc = G.radx[ic], yc = G.radx[jc], zc = G.radx[kc], rx1 = G.radx[1];
  const int n = C.nsh[c];
  if (threadIdx.x == 0) {
    K.realclus[s] = -1;
    K.levhal[s] = 0;
    K.patchclus[s] = 0;
    K.x[s] = xc; K.y[s] = yc; K.z[s] = zc;
    K.radio[s] = G.R[n - 1];
    K.masa[s] = C.masa[c];
    K.xcm[s] = C.cm[3 * c]; K.ycm[s] = C.cm[3 * c + 1]; K.zcm[s] = C.cm[3 * c + 2];
  }
  const float r = G.R[n - 1];
  const int nx = G.nx;
  const int lx = box_lo(xc, r, rx1, G.dx), hx = box_hi(xc, r, rx1, G.dx, nx);
  const int ly = box_lo(yc, r, rx1, G.dx), hy = box_hi(yc, r, rx1, G.dx, nx);
  const int lz = box_lo(zc, r, rx1, G.dx), hz = box_hi(zc, r, rx1, G.dx, nx);
  const int ny_ = hy - ly + 1, nz_ = hz - lz + 1;
  const float o2m = __fmul_rn(__fmul_rn(r, r), 1.0001f);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  for (int row = warp; row < ny_ * nz_; row += nwarp) {  // a warp per (j, k) row
    const int j = ly + row % ny_, k = lz + row / ny_;
    const float ddy = __fsub_rn(G.radx[j], yc), ddz = __fsub_rn(G.radx[k], zc);
    const float s2 = __fadd_rn(__fmul_rn(ddy, ddy), __fmul_rn(ddz, ddz));
    if (s2 > o2m) continue;
    int a0, a1, b0, b1;
    row_runs(G, xc, s2, 0.0f, r, lx, hx, &a0, &a1, &b0, &b1);
    for (int i = a0 + lane; i <= a1; i += 32)
      if (covers(G, xc, yc, zc, n, i, j, k)) conta[((size_t)(k - 1) * nx + (j - 1)) * nx + (i - 1)] = 0;
  }
}

}  // namespace

extern "C" int asohf_halofind_grid_base(asohf_ctx* c, int nx, float dx, const float* u1, const float* radx,
                                        float contrastec, float rote, float rete, float rodo, float re0,
                                        float bound, float vol_solap_low, const asohf_mesh* mesh,
                                        asohf_catalogue* cat, int u1_on_device, int cat_on_device,
                                        int32_t* nhal) {
  if (!c || nx < 3 || nx > 1024 || !u1 || !radx || !cat || !nhal || cat->capacity < 0) return ASOHF_ERR_INVALID;
  if (mesh && mesh->nl > 0) {
    for (int ir = 1; ir <= mesh->nl; ir++)
      if (mesh->npatch[ir] > 0) return ASOHF_ERR_UNSUPPORTED;  // AMR recentering: not on the device
  }
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  const int64_t g = (int64_t)nx * nx * nx;
  // the shell radii (haloes_grids.f:484-486), the same for every halo
  float hR[GF_MAXSH];
  const float esp = 0.2f * dx, esp_log = 1.05f;
  int nR = 0;
  hR[nR++] = 0.8f * dx;
  while (hR[nR - 1] <= bound && nR < GF_MAXSH) {
    const float r = hR[nR - 1], a = r + esp, b = r * esp_log;
    hR[nR++] = a > b ? a : b;
  }
  // arena: the grid (when on the host), CONTA, RADX, the radii, counters and
  // the catalogue columns; segment arena: the candidates and chunk arrays
  const size_t cap = cat->capacity > 0 ? (size_t)cat->capacity : 1;
  ASOHF_CHECK(arena_reserve(c, (u1_on_device ? 0 : 4 * (size_t)g) + (size_t)g + 4 * (size_t)(nx + 2) +
                                   4 * GF_MAXSH + 64 + 64 + 44 * cap + 16 * 256));
  float* du = (float*)u1;
  if (!u1_on_device) {
    du = (float*)arena_alloc(c, 4 * (size_t)g);
    if (!du) return ASOHF_ERR_CAPACITY;
    ASOHF_CUDA(cudaMemcpyAsync(du, u1, 4 * (size_t)g, cudaMemcpyHostToDevice, c->stream));
  }
  uint8_t* conta = (uint8_t*)arena_alloc(c, (size_t)g);
  float* dradx = (float*)arena_alloc(c, 4 * (size_t)(nx + 2));
  float* dR = (float*)arena_alloc(c, 4 * GF_MAXSH);
  unsigned long long* dn = (unsigned long long*)arena_alloc(c, 64);
  int32_t* dstate = (int32_t*)arena_alloc(c, 64);
  GridCat K;
  K.capacity = (int)cap;
  K.realclus = (int32_t*)arena_alloc(c, 4 * cap);
  K.levhal = (int32_t*)arena_alloc(c, 4 * cap);
  K.patchclus = (int32_t*)arena_alloc(c, 4 * cap);
  K.x = (float*)arena_alloc(c, 4 * cap);
  K.y = (float*)arena_alloc(c, 4 * cap);
  K.z = (float*)arena_alloc(c, 4 * cap);
  K.radio = (float*)arena_alloc(c, 4 * cap);
  K.masa = (float*)arena_alloc(c, 4 * cap);
  K.xcm = (float*)arena_alloc(c, 4 * cap);
  K.ycm = (float*)arena_alloc(c, 4 * cap);
  K.zcm = (float*)arena_alloc(c, 4 * cap);
  if (!conta || !dradx || !dR || !dn || !dstate || !K.realclus || !K.levhal || !K.patchclus || !K.x || !K.y ||
      !K.z || !K.radio || !K.masa || !K.xcm || !K.ycm || !K.zcm)
    return ASOHF_ERR_CAPACITY;
  ASOHF_CUDA(cudaMemcpyAsync(dradx, radx, 4 * (size_t)(nx + 2), cudaMemcpyHostToDevice, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(dR, hR, 4 * (size_t)nR, cudaMemcpyHostToDevice, c->stream));
  ASOHF_CUDA(cudaMemsetAsync(dn, 0, 64, c->stream));
  ASOHF_CUDA(cudaMemsetAsync(dstate, 0, 64, c->stream));
  // candidates: count, then fill and sort
  const float thr_peak = contrastec / 6.0f;
  int kt_ = ktime_begin(c, "grid_peaks");
  k_grid_conta_init<<<grid_for(g, 256, c->num_sms * 16), 256, 0, c->stream>>>(conta, nx);
  k_grid_peaks<<<grid_for(g, 256, c->num_sms * 16), 256, 0, c->stream>>>(du, nx, thr_peak, nullptr, 0, dn);
  ktime_end(c, kt_);
  c->launches += 2;
  unsigned long long hn = 0;
  ASOHF_CUDA(cudaMemcpyAsync(&hn, dn, 8, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  const int64_t ncand = (int64_t)hn;
  if (ncand >= (1ll << 31)) return ASOHF_ERR_CAPACITY;
  const int nch = (int)((ncand + GF_CHUNK - 1) / GF_CHUNK);
  size_t tb = 0;
  cub::DeviceRadixSort::SortKeys(nullptr, tb, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                 (int)(ncand > 0 ? ncand : 1));
  ASOHF_CHECK(seg_reserve(c, 16 * (size_t)(ncand + 1) + tb + 4 * (size_t)GF_CHUNK * (6 + GF_WORDS) + 16 * 256));
  unsigned long long* k0 = (unsigned long long*)seg_alloc(c, 8 * (size_t)(ncand + 1));
  unsigned long long* k1 = (unsigned long long*)seg_alloc(c, 8 * (size_t)(ncand + 1));
  void* tmp = seg_alloc(c, tb);
  GridChunk C;
  C.nsh = (int32_t*)seg_alloc(c, 4 * GF_CHUNK);
  C.masa = (float*)seg_alloc(c, 4 * GF_CHUNK);
  C.cm = (float*)seg_alloc(c, 12 * GF_CHUNK);
  C.pairs = (uint32_t*)seg_alloc(c, 4 * (size_t)GF_CHUNK * GF_WORDS);
  C.slot = (int32_t*)seg_alloc(c, 4 * GF_CHUNK);
  C.state = dstate;
  if (!k0 || !k1 || !tmp || !C.nsh || !C.masa || !C.cm || !C.pairs || !C.slot) return ASOHF_ERR_CAPACITY;
  ASOHF_CUDA(cudaMemsetAsync(dn, 0, 64, c->stream));
  k_grid_peaks<<<grid_for(g, 256, c->num_sms * 16), 256, 0, c->stream>>>(du, nx, thr_peak, k0, ncand, dn);
  c->launches++;
  if (ncand > 0) ASOHF_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tb, k0, k1, (int)ncand, 0, 64, c->stream));
  GridIn G;
  G.u = du;
  G.radx = dradx;
  G.R = dR;
  G.nR = nR;
  G.nx = nx;
  G.dx = dx;
  G.volcell = dx * dx * dx;
  G.bound = bound;
  G.contrastec = contrastec;
  G.rote = rote;
  G.rodo = rodo;
  G.re03 = re0 * re0 * re0;
  G.rete3 = rete * rete * rete;
  C.keys = k1;
  kt_ = ktime_begin(c, "grid_chunks");
  for (int q = 0; q < nch; q++) {
    C.c0 = (int64_t)q * GF_CHUNK;
    C.m = (int)((ncand - C.c0) < GF_CHUNK ? (ncand - C.c0) : GF_CHUNK);
    k_grid_grow<<<(C.m + 7) / 8, 256, 0, c->stream>>>(G, C, conta);
    k_grid_pairs<<<C.m, 32, 0, c->stream>>>(G, C);
    k_grid_replay<<<1, 32, 0, c->stream>>>(C, (int)cap);
    k_grid_commit<<<C.m, 256, 0, c->stream>>>(G, C, K, conta);
    c->launches += 4;
  }
  ktime_end(c, kt_);
  ASOHF_CUDA(cudaGetLastError());
  int32_t st[2];
  ASOHF_CUDA(cudaMemcpyAsync(st, C.state, 8, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  if (st[1]) return st[1];
  const int nk = st[0];
  // the rows into the caller's catalogue (IF (IR.EQ.0) NCLUS=0)
  const cudaMemcpyKind kind = cat_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (nk > 0) {
    ASOHF_CUDA(cudaMemcpyAsync(cat->realclus, K.realclus, 4 * (size_t)nk, kind, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(cat->levhal, K.levhal, 4 * (size_t)nk, kind, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(cat->patchclus, K.patchclus, 4 * (size_t)nk, kind, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(cat->clusrx, K.x, 4 * (size_t)nk, kind, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(cat->clusry, K.y, 4 * (size_t)nk, kind, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(cat->clusrz, K.z, 4 * (size_t)nk, kind, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(cat->radio, K.radio, 4 * (size_t)nk, kind, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(cat->masa, K.masa, 4 * (size_t)nk, kind, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(cat->clusrxcm, K.xcm, 4 * (size_t)nk, kind, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(cat->clusrycm, K.ycm, 4 * (size_t)nk, kind, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(cat->clusrzcm, K.zcm, 4 * (size_t)nk, kind, c->stream));
  }
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  cat->nclus = nk;
  // OVERLAPPING at IR = 0 over the haloes just found (haloes_grids.f:577)
  int32_t nhallev[ASOHF_NLEVELS + 1] = {0};
  nhallev[0] = nk;
  int32_t nrem = 0;
  if (nk > 0) ASOHF_CHECK(asohf_overlapping(c, cat, 0, nhallev, vol_solap_low, cat_on_device, &nrem));
  *nhal = nk;
  return ASOHF_OK;
}
