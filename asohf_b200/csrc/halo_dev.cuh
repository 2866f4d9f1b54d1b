// halo_dev.cuh -- device building blocks of the per-halo particle stage:
// the x-slab range of FIND_PARTICLE_INDICES, column-index queries, the
// density-peak recentering, tile-wise block scans, and the halo state that
// the unbinding passes update.  One CTA works on one halo at a time; every
// per-halo decision is made from block-reduced values, so control flow stays
// uniform across the CTA.
#pragma once

#include "common.cuh"

#define HB 256          // threads per CTA of the per-halo kernels
#define IPT 4           // items per thread per tile
#define TILE (HB * IPT)
#define MAX_HIST 48     // recentering shrink steps kept in shared memory

struct Store {
  const float *x, *y, *z, *vx, *vy, *vz, *m;
  const int32_t* id;
  float norma;        // MAXVAL(MASAP)
  int eqmass_lt8;     // max/min mass < 8 over the whole store
};

struct ColIdx {
  const float4* cp;        // (x, y, z, x-sorted position as int bits)
  const int64_t* start;    // column starts
  int ncol;
  float xl, cdx;
  const int32_t* nd;       // NDMPART_X(0:NX)
  int nmax;                // NMAX (= NX)
  float dx;                // COMMON /ESPACIADO/ DX
  float xldom;             // -LADO0/2
};

struct HConst {
  float rote, rete, pi, cgr, um, uv, contrastec, omegaz, fdm, zeta;
  int min_num_part;
  int want_ids;            // FLAG_WDM.EQ.1 .OR. VAR.GT.1
  int nl;
  int lev_lo[ASOHF_NLEVELS + 2], lev_hi[ASOHF_NLEVELS + 2];  // 1-based patch ranges per level
};

// FIND_PARTICLE_INDICES (haloes_particles.f:117-143): 0-based half-open range
// [lo, hi) of the x-sorted store.
__device__ __forceinline__ void slab_range(const ColIdx& ci, float cx, float r, int64_t* lo,
                                           int64_t* hi) {
  int pos1 = (int)(__fdiv_rn(__fsub_rn(__fsub_rn(cx, r), ci.xldom), ci.dx)) + 1;
  int pos2 = (int)(__fdiv_rn(__fsub_rn(__fadd_rn(cx, r), ci.xldom), ci.dx)) + 1;
  if (pos1 < 1) pos1 = 1;
  if (pos2 > ci.nmax) pos2 = ci.nmax;
  if (pos1 > ci.nmax + 1) pos1 = ci.nmax + 1;
  if (pos2 < 0) pos2 = 0;
  *lo = ci.nd[pos1 - 1];
  *hi = ci.nd[pos2];
}

__device__ __forceinline__ int col_index(float v, float xl, float cdx, int n) {
  int b = (int)floorf((v - xl) / cdx);
  return b < 0 ? 0 : (b >= n ? n - 1 : b);
}

// Calls f(e) for every column-index entry whose x, y, z lie within r' >= r
// of (cx, cy, cz) (a superset of any open-cube or sphere test of radius r).
// Warps take columns round-robin; lanes stride the binary-searched x range.
template <class F>
__device__ __forceinline__ void query_box(const ColIdx& ci, float cx, float cy, float cz, float r, F&& f) {
  float rr = r * 1.0001f + 1e-6f;
  int iy0 = col_index(cy - rr, ci.xl, ci.cdx, ci.ncol), iy1 = col_index(cy + rr, ci.xl, ci.cdx, ci.ncol);
  int iz0 = col_index(cz - rr, ci.xl, ci.cdx, ci.ncol), iz1 = col_index(cz + rr, ci.xl, ci.cdx, ci.ncol);
  float xlo = cx - rr, xhi = cx + rr;
  int ny = iy1 - iy0 + 1;
  int ncols = ny * (iz1 - iz0 + 1);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c = wid; c < ncols; c += nw) {
    int64_t cid = (int64_t)(iz0 + c / ny) * ci.ncol + iy0 + c % ny;
    int64_t s = 0, e = 0;
    if (lane == 0) {
      int64_t a = ci.start[cid], b = ci.start[cid + 1];
      int64_t lo = a, hi = b;
      while (lo < hi) {  // first x >= xlo
        int64_t mid = (lo + hi) >> 1;
        if (ci.cp[mid].x < xlo) lo = mid + 1; else hi = mid;
      }
      s = lo;
      hi = b;
      while (lo < hi) {  // first x > xhi
        int64_t mid = (lo + hi) >> 1;
        if (ci.cp[mid].x <= xhi) lo = mid + 1; else hi = mid;
      }
      e = lo;
    }
    s = __shfl_sync(0xffffffffu, s, 0);
    e = __shfl_sync(0xffffffffu, e, 0);
    for (int64_t k = s + lane; k < e; k += 32) f(ci.cp[k]);
  }
}

__device__ __forceinline__ int ppos(const float4& e) { return __float_as_int(e.w); }

// Open cube of haloes_particles.f:405-407.
__device__ __forceinline__ bool in_cube(float x, float y, float z, float cx, float cy, float cz, float r) {
  return __fsub_rn(cx, r) < x && x < __fadd_rn(cx, r) && __fsub_rn(cy, r) < y && y < __fadd_rn(cy, r) &&
         __fsub_rn(cz, r) < z && z < __fadd_rn(cz, r);
}

// SQRT((XP-CX)**2+(YP-CY)**2+(ZP-CZ)**2) in REAL*4.
__device__ __forceinline__ float dist3(float x, float y, float z, float cx, float cy, float cz) {
  float ax = __fsub_rn(x, cx), ay = __fsub_rn(y, cy), az = __fsub_rn(z, cz);
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ax, ax), __fmul_rn(ay, ay)), __fmul_rn(az, az)));
}

struct RecShared {
  double dens[64];
  float hist[MAX_HIST][4];
  double dred[32];
  float fred[32];
  long long lred[32];
  int best;
};

// RECENTER_DENSITY_PEAK_PARTICLES (haloes_particles.f:367-574).  The member
// list of each shrink step is the first cube intersected with every later
// cube, so each step re-reads the first cube from the column index instead
// of storing the list.  Returns false if the shrink history overflows.
static __device__ bool recenter_block(const Store& S, const ColIdx& ci, float* pcx, float* pcy, float* pcz,
                               float R, float dxpamin, RecShared& sh) {
  float cx = *pcx, cy = *pcy, cz = *pcz;
  float radio = fmaxf(__fmul_rn(0.05f, R), dxpamin);
  int64_t lo, hi;
  long long cnt;
  float maxm, minm;
  for (int it = 0;; it++) {
    slab_range(ci, cx, radio, &lo, &hi);
    long long c = 0;
    float mx = -1.e30f, mn = 1.e30f;
    query_box(ci, cx, cy, cz, radio, [&](const float4& e) {
      int p = ppos(e);
      if (p >= lo && p < hi && in_cube(e.x, e.y, e.z, cx, cy, cz, radio)) {
        c++;
        float mp = S.m[p];
        mx = fmaxf(mx, mp);
        mn = fminf(mn, mp);
      }
    });
    cnt = block_sum_ll(c, sh.lred);
    maxm = block_max_f(mx, sh.fred);
    minm = block_min_f(mn, sh.fred);
    if (cnt > 32) break;
    radio = __fmul_rn(radio, 1.2f);
    if (it > 10000) return false;
  }
  const float c0x = cx, c0y = cy, c0z = cz, r0 = radio;
  const int64_t lo0 = lo, hi0 = hi;
  int nh = 0;
  float ddxx = __fdiv_rn(__fmul_rn(2.0f, radio), 4.0f);
  float xl = __fsub_rn(cx, radio), yl = __fsub_rn(cy, radio), zl = __fsub_rn(cz, radio);
  // membership: first cube and every recorded shrink cube
  auto member = [&](const float4& e, int upto) -> bool {
    int p = ppos(e);
    if (!(p >= lo0 && p < hi0 && in_cube(e.x, e.y, e.z, c0x, c0y, c0z, r0))) return false;
    for (int h = 0; h < upto; h++)
      if (!in_cube(e.x, e.y, e.z, sh.hist[h][0], sh.hist[h][1], sh.hist[h][2], sh.hist[h][3])) return false;
    return true;
  };
  for (;;) {
    for (int q = threadIdx.x; q < 64; q += blockDim.x) sh.dens[q] = 0.0;
    __syncthreads();
    bool ngp = __fdiv_rn(maxm, minm) < 8.0f;
    query_box(ci, c0x, c0y, c0z, r0, [&](const float4& e) {
      if (!member(e, nh)) return;
      int p = ppos(e);
      float mp = S.m[p];
      if (ngp) {
        int ix = (int)__fdiv_rn(__fsub_rn(e.x, xl), ddxx) + 1;
        int jy = (int)__fdiv_rn(__fsub_rn(e.y, yl), ddxx) + 1;
        int kz = (int)__fdiv_rn(__fsub_rn(e.z, zl), ddxx) + 1;
        ix = ix < 1 ? 1 : (ix > 4 ? 4 : ix);
        jy = jy < 1 ? 1 : (jy > 4 ? 4 : jy);
        kz = kz < 1 ? 1 : (kz > 4 ? 4 : kz);
        atomicAdd(&sh.dens[((kz - 1) * 4 + (jy - 1)) * 4 + (ix - 1)], (double)mp);
      } else {
        int ix = (int)floorf(__fdiv_rn(__fsub_rn(e.x, xl), ddxx)) + 1;
        int jy = (int)floorf(__fdiv_rn(__fsub_rn(e.y, yl), ddxx)) + 1;
        int kz = (int)floorf(__fdiv_rn(__fsub_rn(e.z, zl), ddxx)) + 1;
        int plev = (int)__fdiv_rn(logf(__fdiv_rn(mp, minm)), logf(8.0f));
        if (plev < 0) plev = 0;
        if (plev == 0) {
          ix = ix < 1 ? 1 : (ix > 4 ? 4 : ix);
          jy = jy < 1 ? 1 : (jy > 4 ? 4 : jy);
          kz = kz < 1 ? 1 : (kz > 4 ? 4 : kz);
          atomicAdd(&sh.dens[((kz - 1) * 4 + (jy - 1)) * 4 + (ix - 1)], (double)mp);
        } else {
          int ksize = (int)__fadd_rn(0.25f, __fmul_rn(0.5f, (float)(1 << plev)));
          int nden = ksize + 1;
          float bl = __fdiv_rn(1.0f, (float)nden);
          float norma = __fdiv_rn(1.0f, (float)(nden * nden * nden));
          int i1 = max(ix - ksize, 1), j1 = max(jy - ksize, 1), k1 = max(kz - ksize, 1);
          int i2 = min(ix + ksize, 4), j2 = min(jy + ksize, 4), k2 = min(kz + ksize, 4);
          for (int kk = k1; kk <= k2; kk++)
            for (int jj = j1; jj <= j2; jj++)
              for (int ii = i1; ii <= i2; ii++) {
                float kx = __fsub_rn(1.0f, __fmul_rn(bl, (float)abs(ii - ix)));
                float ky = __fsub_rn(1.0f, __fmul_rn(bl, (float)abs(jj - jy)));
                float kz2 = __fsub_rn(1.0f, __fmul_rn(bl, (float)abs(kk - kz)));
                float kern = __fmul_rn(__fmul_rn(__fmul_rn(kx, ky), kz2), norma);
                atomicAdd(&sh.dens[((kk - 1) * 4 + (jj - 1)) * 4 + (ii - 1)], (double)kern * (double)mp);
              }
        }
      }
    });
    __syncthreads();
    if (threadIdx.x == 0) {  // MAXLOC: first maximum, column-major
      int b = 0;
      for (int q = 1; q < 64; q++)
        if (sh.dens[q] > sh.dens[b]) b = q;
      sh.best = b;
    }
    __syncthreads();
    int b = sh.best;
    int ix = b % 4 + 1, jy = (b / 4) % 4 + 1, kz = b / 16 + 1;
    cx = __fadd_rn(xl, __fmul_rn(__fsub_rn((float)ix, 0.5f), ddxx));
    cy = __fadd_rn(yl, __fmul_rn(__fsub_rn((float)jy, 0.5f), ddxx));
    cz = __fadd_rn(zl, __fmul_rn(__fsub_rn((float)kz, 0.5f), ddxx));
    radio = __fdiv_rn(radio, 2.0f);
    xl = __fsub_rn(cx, radio);
    yl = __fsub_rn(cy, radio);
    zl = __fsub_rn(cz, radio);
    ddxx = __fdiv_rn(ddxx, 2.0f);
    if (nh >= MAX_HIST) return false;
    if (threadIdx.x == 0) {
      sh.hist[nh][0] = cx; sh.hist[nh][1] = cy; sh.hist[nh][2] = cz; sh.hist[nh][3] = radio;
    }
    __syncthreads();
    nh++;
    long long c = 0;
    float mx = -1.e30f, mn = 1.e30f;
    query_box(ci, c0x, c0y, c0z, r0, [&](const float4& e) {
      if (member(e, nh)) {
        c++;
        float mp = S.m[ppos(e)];
        mx = fmaxf(mx, mp);
        mn = fminf(mn, mp);
      }
    });
    cnt = block_sum_ll(c, sh.lred);
    maxm = block_max_f(mx, sh.fred);
    minm = block_min_f(mn, sh.fred);
    if (cnt < 32) break;
  }
  double bs = 0.0, bx = 0.0, by = 0.0, bz = 0.0;
  query_box(ci, c0x, c0y, c0z, r0, [&](const float4& e) {
    if (member(e, nh)) {
      float mp = S.m[ppos(e)];
      bs += (double)mp;
      bx += (double)__fmul_rn(e.x, mp);
      by += (double)__fmul_rn(e.y, mp);
      bz += (double)__fmul_rn(e.z, mp);
    }
  });
  bs = block_sum_d(bs, sh.dred);
  bx = block_sum_d(bx, sh.dred);
  by = block_sum_d(by, sh.dred);
  bz = block_sum_d(bz, sh.dred);
  *pcx = (float)(bx / bs);
  *pcy = (float)(by / bs);
  *pcz = (float)(bz / bs);
  return true;
}

// Tile-wise inclusive prefix over j in [a, b): val(j) gives the term,
// use(j, inclusive_prefix) consumes it in any order.  Each thread sums IPT
// consecutive items sequentially, then the block scans the thread totals.
// Returns carry + total.
template <class V, class U>
__device__ __forceinline__ double tile_prefix_d(int64_t a, int64_t b, double carry, V val, U use,
                                                double* sbuf) {
  for (int64_t t0 = a; t0 < b; t0 += TILE) {
    double loc[IPT];
    double run = 0.0;
    int64_t j0 = t0 + (int64_t)threadIdx.x * IPT;
#pragma unroll
    for (int q = 0; q < IPT; q++) {
      int64_t j = j0 + q;
      double v = j < b ? val(j) : 0.0;
      run += v;
      loc[q] = run;
    }
    double tot;
    double inc = block_scan_d(run, sbuf, &tot);
    double off = carry + (inc - run);
#pragma unroll
    for (int q = 0; q < IPT; q++) {
      int64_t j = j0 + q;
      if (j < b) use(j, off + loc[q]);
    }
    carry += tot;
  }
  return carry;
}
