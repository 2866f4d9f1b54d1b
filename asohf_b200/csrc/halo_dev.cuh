// halo_dev.cuh -- device building blocks of the per-halo particle stage:
// the x-slab range of FIND_PARTICLE_INDICES, column-index queries, the
// density-peak recentering, tile-wise block scans, and the halo state that
// the unbinding passes update.  One CTA works on one halo at a time; every
// per-halo decision is made from block-reduced values, so control flow stays
// uniform across the CTA.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"

namespace cg = cooperative_groups;

#define HB 256          // threads per CTA of the per-halo kernels (at most)
#define HW (HB / 32)    // warps per CTA (at most)
#define IPT 4           // items per thread per tile of the block scans
#define MAX_HIST 48     // recentering shrink steps kept in shared memory

// A halo is refined by a group of C CTAs: one CTA (C = 1; C = 0 marks a
// CTA of one warp, whose code keeps only the one-warp paths) or a
// thread-block cluster whose CTAs split every element loop into contiguous
// chunks and combine partial results through distributed shared memory.
template <int C>
struct Grp {
  __device__ __forceinline__ unsigned rank() const {
    if constexpr (C <= 1) return 0;
    else return cg::this_cluster().block_rank();
  }
  __device__ __forceinline__ void sync() const {
    if constexpr (C <= 1) __syncthreads();
    else cg::this_cluster().sync();
  }
  // this CTA's contiguous part of [a, b)
  __device__ __forceinline__ void chunk(int64_t a, int64_t b, int64_t* lo, int64_t* hi) const {
    if constexpr (C <= 1) {
      *lo = a;
      *hi = b;
    } else {
      int64_t n = b > a ? b - a : 0, per = (n + C - 1) / C, r = rank();
      *lo = a + (per * r < n ? per * r : n);
      *hi = a + (per * (r + 1) < n ? per * (r + 1) : n);
    }
  }
  // first global warp and warp stride for warp-strided loops
  __device__ __forceinline__ int warp0() const { return (int)rank() * (blockDim.x >> 5) + (threadIdx.x >> 5); }
  __device__ __forceinline__ int nwarps() const { return (C > 1 ? C : 1) * (blockDim.x >> 5); }
};

// Per-CTA exchange slots for group reductions.  A group reduction first
// reduces over the CTA, then (C > 1) thread 0 publishes the CTA's value and
// a few threads combine the C published values in rank order, so results are
// identical on every CTA and do not depend on scheduling.
struct GX {
  double vred[16][HW];  // per-warp partials of vector sums
  double bres[16];      // CTA totals
  double d[16];         // published CTA values
  double dres[16];      // group totals
  long long l[8];
  long long lres[8];
  long long lw[8][HW];  // per-warp minima (gmin_llv)
  float f[2];
  float fres[2];
};

// Warp reduce-scatter of K doubles (K <= 16, padded to a power of two KP):
// the pairings of the xor butterfly (distances 16, 8, 4, 2, 1), so every
// total is the butterfly's bit for bit, but while a lane holds several
// partial sums each level exchanges half of them (the lane keeps the upper
// half when its bit of that distance is set).  Returns the total of the value
// that lane holds; scatter_lane<K>(q) is a lane that holds value q.
template <int K>
struct Scatter {
  static constexpr int KP = K <= 1 ? 1 : K <= 2 ? 2 : K <= 4 ? 4 : K <= 8 ? 8 : 16;
  static constexpr int LOG = K <= 1 ? 0 : K <= 2 ? 1 : K <= 4 ? 2 : K <= 8 ? 3 : 4;
};

template <int K>
__device__ __forceinline__ double warp_sum_scatter(const double* v) {
  constexpr int KP = Scatter<K>::KP;
  double w[KP];
#pragma unroll
  for (int q = 0; q < KP; q++) w[q] = q < K ? v[q] : 0.0;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int lv = 0; lv < 5; lv++) {
    const int o = 16 >> lv;
    const int n = KP >> lv;  // partial sums a lane holds before this level
    if (n > 1) {
      const bool up = (lane & o) != 0;
#pragma unroll
      for (int i = 0; i < n / 2; i++) {
        const double send = up ? w[i] : w[i + n / 2];
        const double keep = up ? w[i + n / 2] : w[i];
        w[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    } else {
      w[0] += __shfl_xor_sync(0xffffffffu, w[0], o);
    }
  }
  return w[0];
}

// The same reduce-scatter for the minimum of K long longs (exact in any
// order).
template <int K>
__device__ __forceinline__ long long warp_min_scatter(const long long* v) {
  constexpr int KP = Scatter<K>::KP;
  long long w[KP];
#pragma unroll
  for (int q = 0; q < KP; q++) w[q] = q < K ? v[q] : LLONG_MAX;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int lv = 0; lv < 5; lv++) {
    const int o = 16 >> lv;
    const int n = KP >> lv;
    if (n > 1) {
      const bool up = (lane & o) != 0;
#pragma unroll
      for (int i = 0; i < n / 2; i++) {
        const long long send = up ? w[i] : w[i + n / 2];
        const long long keep = up ? w[i + n / 2] : w[i];
        const long long r = __shfl_xor_sync(0xffffffffu, send, o);
        w[i] = r < keep ? r : keep;
      }
    } else {
      const long long r = __shfl_xor_sync(0xffffffffu, w[0], o);
      w[0] = r < w[0] ? r : w[0];
    }
  }
  return w[0];
}

template <int K>
__device__ __forceinline__ int scatter_lane(int q) {
  constexpr int LOG = Scatter<K>::LOG;
  int l = 0;
#pragma unroll
  for (int lv = 0; lv < LOG; lv++) l |= ((q >> (LOG - 1 - lv)) & 1) << (4 - lv);
  return l;
}

// Sum of K doubles over the CTA; every thread receives the totals.
template <int K>
__device__ __forceinline__ void block_sum_dv(double* v, GX& x) {
  static_assert(K <= 16, "at most 16 sums");
  const int lane = threadIdx.x & 31;
  const double mine = warp_sum_scatter<K>(v);
  if (blockDim.x == 32) {  // one warp: no shared memory
#pragma unroll
    for (int q = 0; q < K; q++) v[q] = __shfl_sync(0xffffffffu, mine, scatter_lane<K>(q));
    return;
  }
  int wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
#pragma unroll
  for (int q = 0; q < K; q++)
    if (lane == scatter_lane<K>(q)) x.vred[q][wid] = mine;
  __syncthreads();
  for (int q = wid; q < K; q += nw) {
    double t = lane < nw ? x.vred[q][lane] : 0.0;
    t = warp_sum_d(t);
    if (lane == 0) x.bres[q] = t;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < K; q++) v[q] = x.bres[q];
  __syncthreads();
}

// Sum of K doubles over the group (v: per-thread values, in/out).
template <int K, int C>
__device__ __forceinline__ void gsum_dv(const Grp<C>& g, double* v, GX& x) {
  block_sum_dv<K>(v, x);
  if constexpr (C > 1) {
    if (threadIdx.x == 0) {
#pragma unroll
      for (int q = 0; q < K; q++) x.d[q] = v[q];
    }
    g.sync();
    if (threadIdx.x < K) {
      cg::cluster_group cl = cg::this_cluster();
      double t = 0.0;
#pragma unroll 1
      for (int r = 0; r < C; r++) t += *cl.map_shared_rank(&x.d[threadIdx.x], r);
      x.dres[threadIdx.x] = t;
    }
    g.sync();
#pragma unroll
    for (int q = 0; q < K; q++) v[q] = x.dres[q];
  }
}

template <int C>
__device__ __forceinline__ double gsum_d(const Grp<C>& g, double v, double* /*dred*/, GX& x) {
  gsum_dv<1>(g, &v, x);
  return v;
}

template <int C>
__device__ __forceinline__ long long gsum_ll(const Grp<C>& g, long long v, long long* lred, GX& x) {
  v = block_sum_ll(v, lred);
  if constexpr (C > 1) {
    if (threadIdx.x == 0) x.l[0] = v;
    g.sync();
    if (threadIdx.x == 0) {
      cg::cluster_group cl = cg::this_cluster();
      long long t = 0;
#pragma unroll 1
      for (int r = 0; r < C; r++) t += *cl.map_shared_rank(&x.l[0], r);
      x.lres[0] = t;
    }
    g.sync();
    v = x.lres[0];
  }
  return v;
}

// Minimum of K indices over the group (K <= 8).
template <int K, int C>
__device__ __forceinline__ void gmin_llv(const Grp<C>& g, long long* v, long long* /*lred*/, GX& x) {
  static_assert(K <= 8, "at most 8 minima");
  const int lane = threadIdx.x & 31;
  const long long mine = warp_min_scatter<K>(v);
  if (blockDim.x == 32) {
#pragma unroll
    for (int q = 0; q < K; q++) v[q] = __shfl_sync(0xffffffffu, mine, scatter_lane<K>(q));
  } else {
    const int wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; q++)
      if (lane == scatter_lane<K>(q)) x.lw[q][wid] = mine;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; q++) {
      long long t = LLONG_MAX;
      for (int w = 0; w < nw; w++) t = x.lw[q][w] < t ? x.lw[q][w] : t;
      v[q] = t;
    }
    __syncthreads();
  }
  if constexpr (C > 1) {
    if (threadIdx.x == 0) {
#pragma unroll
      for (int q = 0; q < K; q++) x.l[q] = v[q];
    }
    g.sync();
    if (threadIdx.x < K) {
      cg::cluster_group cl = cg::this_cluster();
      long long t = LLONG_MAX;
#pragma unroll 1
      for (int r = 0; r < C; r++) {
        long long w = *cl.map_shared_rank(&x.l[threadIdx.x], r);
        t = w < t ? w : t;
      }
      x.lres[threadIdx.x] = t;
    }
    g.sync();
#pragma unroll
    for (int q = 0; q < K; q++) v[q] = x.lres[q];
  }
}

template <int C>
__device__ __forceinline__ long long gmin_ll(const Grp<C>& g, long long v, long long* lred, GX& x) {
  gmin_llv<1>(g, &v, lred, x);
  return v;
}

template <int C>
__device__ __forceinline__ float gmax_f(const Grp<C>& g, float v, float* fred, GX& x) {
  v = block_max_f(v, fred);
  if constexpr (C > 1) {
    if (threadIdx.x == 0) x.f[0] = v;
    g.sync();
    if (threadIdx.x == 0) {
      cg::cluster_group cl = cg::this_cluster();
      float t = -INFINITY;
#pragma unroll 1
      for (int r = 0; r < C; r++) t = fmaxf(t, *cl.map_shared_rank(&x.f[0], r));
      x.fres[0] = t;
    }
    g.sync();
    v = x.fres[0];
  }
  return v;
}

template <int C>
__device__ __forceinline__ float gmin_f(const Grp<C>& g, float v, float* fred, GX& x) {
  return -gmax_f(g, -v, fred, x);
}

// Exclusive prefix (over ranks, in rank order) and total of one value per
// CTA (v: the CTA's value, the same in all its threads).
template <int C>
__device__ __forceinline__ void gexcl_d(const Grp<C>& g, double v, double* off, double* tot, GX& x) {
  if constexpr (C <= 1) {
    *off = 0.0;
    *tot = v;
  } else {
    if (threadIdx.x == 0) x.d[0] = v;
    g.sync();
    if (threadIdx.x == 0) {
      cg::cluster_group cl = cg::this_cluster();
      double o = 0.0, t = 0.0;
      unsigned me = g.rank();
#pragma unroll 1
      for (unsigned r = 0; r < (unsigned)C; r++) {
        double w = *cl.map_shared_rank(&x.d[0], r);
        if (r == me) o = t;
        t += w;
      }
      x.dres[0] = o;
      x.dres[1] = t;
    }
    g.sync();
    *off = x.dres[0];
    *tot = x.dres[1];
  }
}

template <int C>
__device__ __forceinline__ void gexcl_ll(const Grp<C>& g, long long v, long long* off, long long* tot, GX& x) {
  if constexpr (C <= 1) {
    *off = 0;
    *tot = v;
  } else {
    if (threadIdx.x == 0) x.l[0] = v;
    g.sync();
    if (threadIdx.x == 0) {
      cg::cluster_group cl = cg::this_cluster();
      long long o = 0, t = 0;
      unsigned me = g.rank();
#pragma unroll 1
      for (unsigned r = 0; r < (unsigned)C; r++) {
        long long w = *cl.map_shared_rank(&x.l[0], r);
        if (r == me) o = t;
        t += w;
      }
      x.lres[0] = o;
      x.lres[1] = t;
    }
    g.sync();
    *off = x.lres[0];
    *tot = x.lres[1];
  }
}

struct Store {
  const float *x, *y, *z, *vx, *vy, *vz, *m;
  const int32_t* id;
  const float4* rows;  // the same store as rows (x, y, z, m | vx, vy, vz, id), or null
  float meq;           // the common particle mass when all are equal, else 0
  __device__ __forceinline__ float mass(int p) const { return meq != 0.0f ? meq : m[p]; }
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
  int energies;            // DO_COMPUTE_ENERGIES.EQ.1
  int max_part_dsum;       // MAX_PART_DSUM: direct pair sums below it
  uint32_t epot_seed;      // seed of the sampling estimator at or above it
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
// When the query has fewer columns than twice the warps, each column's x
// range is cut into parts so every warp gets work.  Warp w of nw takes
// (column, part) items w, w+nw, ...; its lanes binary-search the x ranges of
// 32 items at once, then stride through each range.
template <class F>
__device__ __forceinline__ void query_box_w(const ColIdx& ci, float cx, float cy, float cz, float r, int w0, int nw,
                                           F&& f) {
  float rr = r * 1.0001f + 1e-6f;
  int iy0 = col_index(cy - rr, ci.xl, ci.cdx, ci.ncol), iy1 = col_index(cy + rr, ci.xl, ci.cdx, ci.ncol);
  int iz0 = col_index(cz - rr, ci.xl, ci.cdx, ci.ncol), iz1 = col_index(cz + rr, ci.xl, ci.cdx, ci.ncol);
  float xlo = cx - rr, xhi = cx + rr;
  int ny = iy1 - iy0 + 1;
  int ncols = ny * (iz1 - iz0 + 1);
  int parts = ncols >= 2 * nw ? 1 : (2 * nw + ncols - 1) / ncols;
  int nitems = ncols * parts;
  int lane = threadIdx.x & 31;
  for (int base = 0; w0 + base * nw < nitems; base += 32) {
    int it = w0 + (base + lane) * nw;
    int64_t s = 0, e = 0;
    if (it < nitems) {
      int c = it / parts, part = it - c * parts;
      int64_t cid = (int64_t)(iz0 + c / ny) * ci.ncol + iy0 + c % ny;
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
      if (parts > 1) {
        int64_t len = e - s, per = (len + parts - 1) / parts;
        int64_t ps = s + (per * part < len ? per * part : len);
        int64_t pe = s + (per * (part + 1) < len ? per * (part + 1) : len);
        s = ps;
        e = pe;
      }
    }
    for (int q = 0; q < 32 && w0 + (base + q) * nw < nitems; q++) {
      int64_t sq = __shfl_sync(0xffffffffu, s, q), eq = __shfl_sync(0xffffffffu, e, q);
#pragma unroll 4
      for (int64_t k = sq + lane; k < eq; k += 32) f(ci.cp[k]);
    }
  }
}

template <class F>
__device__ __forceinline__ void query_box(const ColIdx& ci, float cx, float cy, float cz, float r, F&& f) {
  query_box_w(ci, cx, cy, cz, r, threadIdx.x >> 5, blockDim.x >> 5, f);
}

// Group query balanced by entries: every CTA finds the x ranges of all the
// query's columns (up to QMAX) into shared memory, then the group's warps
// take equal contiguous shares of the concatenated ranges, so a few dense
// columns no longer keep one warp busy while the others wait.  More columns
// than QMAX: the per-column distribution of query_box_w.
#define QMAX 512
struct QBuf {
  long long s[QMAX];         // first entry of each column's x range
  long long pre[QMAX + 1];   // prefix of the range lengths
};

template <int C, class F>
__device__ __forceinline__ void gquery_box(const Grp<C>& g, const ColIdx& ci, float cx, float cy, float cz,
                                           float r, QBuf& qb, F&& f) {
  float rr = r * 1.0001f + 1e-6f;
  int iy0 = col_index(cy - rr, ci.xl, ci.cdx, ci.ncol), iy1 = col_index(cy + rr, ci.xl, ci.cdx, ci.ncol);
  int iz0 = col_index(cz - rr, ci.xl, ci.cdx, ci.ncol), iz1 = col_index(cz + rr, ci.xl, ci.cdx, ci.ncol);
  int ny = iy1 - iy0 + 1;
  int ncols = ny * (iz1 - iz0 + 1);
  if (ncols > QMAX) {
    query_box_w(ci, cx, cy, cz, r, g.warp0(), g.nwarps(), f);
    return;
  }
  float xlo = cx - rr, xhi = cx + rr;
  for (int c = threadIdx.x; c < ncols; c += blockDim.x) {
    int64_t cid = (int64_t)(iz0 + c / ny) * ci.ncol + iy0 + c % ny;
    int64_t a = ci.start[cid], b = ci.start[cid + 1];
    int64_t lo = a, hi = b;
    while (lo < hi) {  // first x >= xlo
      int64_t mid = (lo + hi) >> 1;
      if (ci.cp[mid].x < xlo) lo = mid + 1; else hi = mid;
    }
    int64_t s0 = lo;
    hi = b;
    while (lo < hi) {  // first x > xhi
      int64_t mid = (lo + hi) >> 1;
      if (ci.cp[mid].x <= xhi) lo = mid + 1; else hi = mid;
    }
    qb.s[c] = s0;
    qb.pre[c + 1] = lo - s0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 32) {  // prefix of the lengths, 32 columns per step
    long long carry = 0;
    for (int c0 = 0; c0 < ncols; c0 += 32) {
      int c = c0 + lane;
      long long v = c < ncols ? qb.pre[c + 1] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
      }
      if (c < ncols) qb.pre[c + 1] = carry + v;
      carry += __shfl_sync(0xffffffffu, v, 31);
    }
    if (lane == 0) qb.pre[0] = 0;
  }
  __syncthreads();
  const long long E = qb.pre[ncols];
  const int W = g.warp0(), NW = g.nwarps();
  const long long per = (E + NW - 1) / NW;
  long long lo = per * W < E ? per * W : E;
  const long long hi = lo + per < E ? lo + per : E;
  if (lo < hi) {
    int a = 0, b = ncols - 1;  // last column with pre[c] <= lo
    while (a < b) {
      int mid = (a + b + 1) >> 1;
      if (qb.pre[mid] <= lo) a = mid; else b = mid - 1;
    }
    for (int c = a; lo < hi && c < ncols; c++) {
      const long long cend = qb.pre[c + 1] < hi ? qb.pre[c + 1] : hi;
      const long long base = qb.s[c] - qb.pre[c];
#pragma unroll 4
      for (long long v = lo + lane; v < cend; v += 32) f(ci.cp[base + v]);
      if (cend > lo) lo = cend;
    }
  }
  __syncthreads();
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
  QBuf qb;
  double dens[64];
  float hist[MAX_HIST][4];
  double dred[32];
  float fred[32];
  long long lred[32];
  int best;
  GX x;
};

template <int C>
__device__ bool recenter_group_ngp(const Grp<C>& g, const Store& S, const ColIdx& ci, float* pcx, float* pcy,
                                   float* pcz, float R, float dxpamin, RecShared& sh);

// RECENTER_DENSITY_PEAK_PARTICLES (haloes_particles.f:367-574).  The member
// list of each shrink step is the first cube intersected with every later
// cube; instead of storing the list, each step re-reads the column index
// over the latest cube (which holds the intersection; the radius halves
// every step) and tests membership against all of them.  Returns false if
// the shrink history overflows.  When no two masses of the store are 8 or
// more apart every density step is the NGP one, and recenter_group_ngp
// takes the same steps with one pass per step.
template <int C>
__device__ bool recenter_group(const Grp<C>& g, const Store& S, const ColIdx& ci, float* pcx, float* pcy,
                               float* pcz, float R, float dxpamin, RecShared& sh) {
  if (S.eqmass_lt8) return recenter_group_ngp(g, S, ci, pcx, pcy, pcz, R, dxpamin, sh);
  float cx = *pcx, cy = *pcy, cz = *pcz;
  float radio = fmaxf(__fmul_rn(0.05f, R), dxpamin);
  int64_t lo, hi;
  long long cnt;
  float maxm, minm;
  for (int it = 0;; it++) {
    slab_range(ci, cx, radio, &lo, &hi);
    long long c = 0;
    float mx = -1.e30f, mn = 1.e30f;
    gquery_box(g, ci, cx, cy, cz, radio, sh.qb, [&](const float4& e) {
      int p = ppos(e);
      if (p >= lo && p < hi && in_cube(e.x, e.y, e.z, cx, cy, cz, radio)) {
        c++;
        float mp = S.mass(p);
        mx = fmaxf(mx, mp);
        mn = fminf(mn, mp);
      }
    });
    cnt = gsum_ll(g, c, sh.lred, sh.x);
    maxm = gmax_f(g, mx, sh.fred, sh.x);
    minm = gmin_f(g, mn, sh.fred, sh.x);
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
    for (int hh = 0; hh < upto; hh++)
      if (!in_cube(e.x, e.y, e.z, sh.hist[hh][0], sh.hist[hh][1], sh.hist[hh][2], sh.hist[hh][3])) return false;
    return true;
  };
  // the latest cube of the history (the first cube before any shrink)
  auto qcube = [&](int upto, float* qx, float* qy, float* qz, float* qr) {
    if (upto == 0) { *qx = c0x; *qy = c0y; *qz = c0z; *qr = r0; }
    else { *qx = sh.hist[upto - 1][0]; *qy = sh.hist[upto - 1][1]; *qz = sh.hist[upto - 1][2]; *qr = sh.hist[upto - 1][3]; }
  };
  float qx, qy, qz, qr;
  for (;;) {
    for (int q = threadIdx.x; q < 64; q += blockDim.x) sh.dens[q] = 0.0;
    __syncthreads();
    bool ngp = __fdiv_rn(maxm, minm) < 8.0f;
    qcube(nh, &qx, &qy, &qz, &qr);
    gquery_box(g, ci, qx, qy, qz, qr, sh.qb, [&](const float4& e) {
      if (!member(e, nh)) return;
      int p = ppos(e);
      float mp = S.mass(p);
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
    if constexpr (C > 1) {  // sum the 4^3 grids of the cluster
      g.sync();
      cg::cluster_group cl = cg::this_cluster();
      double t = 0.0;
      if (threadIdx.x < 64)
        for (int r = 0; r < C; r++) t += *cl.map_shared_rank(&sh.dens[threadIdx.x], r);
      g.sync();
      if (threadIdx.x < 64) sh.dens[threadIdx.x] = t;
      __syncthreads();
    }
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
    qcube(nh, &qx, &qy, &qz, &qr);
    gquery_box(g, ci, qx, qy, qz, qr, sh.qb, [&](const float4& e) {
      if (member(e, nh)) {
        c++;
        float mp = S.mass(ppos(e));
        mx = fmaxf(mx, mp);
        mn = fminf(mn, mp);
      }
    });
    cnt = gsum_ll(g, c, sh.lred, sh.x);
    maxm = gmax_f(g, mx, sh.fred, sh.x);
    minm = gmin_f(g, mn, sh.fred, sh.x);
    if (cnt < 32) break;
  }
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  qcube(nh, &qx, &qy, &qz, &qr);
  gquery_box(g, ci, qx, qy, qz, qr, sh.qb, [&](const float4& e) {
    if (member(e, nh)) {
      float mp = S.mass(ppos(e));
      v[0] += (double)mp;
      v[1] += (double)__fmul_rn(e.x, mp);
      v[2] += (double)__fmul_rn(e.y, mp);
      v[3] += (double)__fmul_rn(e.z, mp);
    }
  });
  gsum_dv<4>(g, v, sh.x);
  *pcx = (float)(v[1] / v[0]);
  *pcy = (float)(v[2] / v[0]);
  *pcz = (float)(v[3] / v[0]);
  return true;
}

// NGP cell (1..4 per axis, clamped) of the 4^3 grid from (xl, yl, zl), cell
// size ddxx: the density step's own arithmetic.
__device__ __forceinline__ int ngp_cell(const float4& e, float xl, float yl, float zl, float ddxx) {
  int ix = (int)__fdiv_rn(__fsub_rn(e.x, xl), ddxx) + 1;
  int jy = (int)__fdiv_rn(__fsub_rn(e.y, yl), ddxx) + 1;
  int kz = (int)__fdiv_rn(__fsub_rn(e.z, zl), ddxx) + 1;
  ix = ix < 1 ? 1 : (ix > 4 ? 4 : ix);
  jy = jy < 1 ? 1 : (jy > 4 ? 4 : jy);
  kz = kz < 1 ? 1 : (kz > 4 ? 4 : kz);
  return ((kz - 1) * 4 + (jy - 1)) * 4 + (ix - 1);
}

// recenter_group with every density step NGP (all mass ratios under 8).
// The steps and their arithmetic are recenter_group's; the passes are
// merged: the pass that counts a step's members (the opening cube, then
// each shrunk cube) also deposits them on the 4^3 grid of that cube, which
// is the grid the next density step reads, and adds their centre-of-mass
// sums, which the last step returns.  Each step's member set and the
// entries every thread visits are the same as in the separate passes.
template <int C>
__device__ bool recenter_group_ngp(const Grp<C>& g, const Store& S, const ColIdx& ci, float* pcx, float* pcy,
                                   float* pcz, float R, float dxpamin, RecShared& sh) {
  float cx = *pcx, cy = *pcy, cz = *pcz;
  float radio = fmaxf(__fmul_rn(0.05f, R), dxpamin);
  float ddxx, xl, yl, zl;
  int64_t lo, hi;
  long long cnt;
  // opening cube: grown x1.2 until it holds more than 32 members
  for (int it = 0;; it++) {
    slab_range(ci, cx, radio, &lo, &hi);
    ddxx = __fdiv_rn(__fmul_rn(2.0f, radio), 4.0f);
    xl = __fsub_rn(cx, radio); yl = __fsub_rn(cy, radio); zl = __fsub_rn(cz, radio);
    for (int q = threadIdx.x; q < 64; q += blockDim.x) sh.dens[q] = 0.0;
    __syncthreads();
    long long c = 0;
    gquery_box(g, ci, cx, cy, cz, radio, sh.qb, [&](const float4& e) {
      int p = ppos(e);
      if (p >= lo && p < hi && in_cube(e.x, e.y, e.z, cx, cy, cz, radio)) {
        c++;
        atomicAdd(&sh.dens[ngp_cell(e, xl, yl, zl, ddxx)], (double)S.mass(p));
      }
    });
    cnt = gsum_ll(g, c, sh.lred, sh.x);
    if (cnt > 32) break;
    radio = __fmul_rn(radio, 1.2f);
    if (it > 10000) return false;
  }
  const float c0x = cx, c0y = cy, c0z = cz, r0 = radio;
  const int64_t lo0 = lo, hi0 = hi;
  int nh = 0;
  auto member = [&](const float4& e, int upto) -> bool {
    int p = ppos(e);
    if (!(p >= lo0 && p < hi0 && in_cube(e.x, e.y, e.z, c0x, c0y, c0z, r0))) return false;
    for (int hh = 0; hh < upto; hh++)
      if (!in_cube(e.x, e.y, e.z, sh.hist[hh][0], sh.hist[hh][1], sh.hist[hh][2], sh.hist[hh][3])) return false;
    return true;
  };
  double v[4];
  for (;;) {
    // sh.dens holds the grid of the current members
    __syncthreads();
    if constexpr (C > 1) {  // sum the 4^3 grids of the cluster
      g.sync();
      cg::cluster_group cl = cg::this_cluster();
      double t = 0.0;
      if (threadIdx.x < 64)
        for (int r = 0; r < C; r++) t += *cl.map_shared_rank(&sh.dens[threadIdx.x], r);
      g.sync();
      if (threadIdx.x < 64) sh.dens[threadIdx.x] = t;
      __syncthreads();
    }
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
    for (int q = threadIdx.x; q < 64; q += blockDim.x) sh.dens[q] = 0.0;
    __syncthreads();
    nh++;
    // the shrunk cube's members: count, grid of the next step, centre of mass
    long long c = 0;
    v[0] = v[1] = v[2] = v[3] = 0.0;
    gquery_box(g, ci, sh.hist[nh - 1][0], sh.hist[nh - 1][1], sh.hist[nh - 1][2], sh.hist[nh - 1][3], sh.qb,
               [&](const float4& e) {
                 if (member(e, nh)) {
                   c++;
                   float mp = S.mass(ppos(e));
                   atomicAdd(&sh.dens[ngp_cell(e, xl, yl, zl, ddxx)], (double)mp);
                   v[0] += (double)mp;
                   v[1] += (double)__fmul_rn(e.x, mp);
                   v[2] += (double)__fmul_rn(e.y, mp);
                   v[3] += (double)__fmul_rn(e.z, mp);
                 }
               });
    cnt = gsum_ll(g, c, sh.lred, sh.x);
    if (cnt < 32) break;
  }
  gsum_dv<4>(g, v, sh.x);
  *pcx = (float)(v[1] / v[0]);
  *pcy = (float)(v[2] / v[0]);
  *pcz = (float)(v[3] / v[0]);
  return true;
}

// Tile-wise inclusive prefix over j in [a, b): val(j) gives the term,
// use(j, inclusive_prefix) consumes it in any order.  Each thread sums IPT
// consecutive items sequentially, then the block scans the thread totals.
// Returns carry + total.
template <class V, class U>
__device__ __forceinline__ double tile_prefix_d(int64_t a, int64_t b, double carry, V val, U use,
                                                double* sbuf) {
  const int64_t tile = (int64_t)blockDim.x * IPT;
  for (int64_t t0 = a; t0 < b; t0 += tile) {
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

__device__ __forceinline__ double warp_allsum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ long long warp_allsum_ll(long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Contiguous run of [lo, hi) taken by warp w of nw.
__device__ __forceinline__ void warp_run(int64_t lo, int64_t hi, int64_t* wlo, int64_t* whi) {
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int64_t n = hi - lo, per = (n + nw - 1) / nw;
  *wlo = lo + (per * w < n ? per * w : n);
  *whi = lo + (per * (w + 1) < n ? per * (w + 1) : n);
}

// Steps of 32 entries are walked in batches of SB: the terms of a batch are
// all read before its first consumer runs, so a warp has SB steps of loads
// in flight although the consumers store to memory (which the compiler
// cannot move loads across).
#define SB 2

// One warp's inclusive walk of [j0, j1) from *run: val(j) gives the term,
// use(j, prefix) consumes it; *run receives the total.
template <class V, class U>
__device__ __forceinline__ void warp_walk_d(int64_t j0, int64_t j1, double* run_io, V val, U use) {
  const int lane = threadIdx.x & 31;
  double run = *run_io;
#pragma unroll 1
  for (int64_t jb = j0; jb < j1; jb += 32 * SB) {
    double t[SB];
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const int64_t j = jb + 32 * u + lane;
      t[u] = j < j1 ? val(j) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const int64_t j = jb + 32 * u + lane;
      double s = t[u];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        double y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      if (j < j1) use(j, run + s);
      run += __shfl_sync(0xffffffffu, s, 31);
    }
  }
  *run_io = run;
}

// Inclusive prefix over [a, b) in index order: val(j) gives the term,
// use(j, prefix) consumes it.  The range is split into the group's CTA
// chunks and each chunk into one contiguous run per warp; a first pass sums
// the runs, a second walks each run 32 entries at a time with a warp scan,
// starting from the totals of everything before it, so a CTA synchronises a
// fixed number of times per call whatever the length.  val is evaluated
// twice per entry (once for a one-warp group, which walks directly) and
// must not read what use stores.  Returns carry + the group total; ends
// synchronised.
template <int C, class V, class U>
__device__ __forceinline__ double gscan_d(const Grp<C>& g, int64_t a, int64_t b, double carry, V val, U use,
                                          double* wbuf, GX& x) {
  if constexpr (C <= 1) {
    if (C == 0 || blockDim.x == 32) {  // one warp: the walk alone
      double run = carry;
      warp_walk_d(a, b, &run, val, use);
      __syncthreads();
      return run;
    }
  }
  int64_t lo, hi, wlo, whi;
  g.chunk(a, b, &lo, &hi);
  warp_run(lo, hi, &wlo, &whi);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double t = 0.0;
#pragma unroll 4
  for (int64_t j = wlo + lane; j < whi; j += 32) t += val(j);
  t = warp_allsum_d(t);
  if (lane == 0) wbuf[w] = t;
  __syncthreads();
  const double woff = warp_allsum_d(lane < w ? wbuf[lane] : 0.0);
  const double ctot = warp_allsum_d(lane < nw ? wbuf[lane] : 0.0);
  double off = 0.0, tot = ctot;
  if constexpr (C > 1) gexcl_d(g, ctot, &off, &tot, x);
  double run = carry + off + woff;
  warp_walk_d(wlo, whi, &run, val, use);
  g.sync();
  return carry + tot;
}

// Prefix of the recurrence M_j = M_{j-1} + m_j, Q_j = Q_{j-1} + M_j * w_j
// (a cumulative mass and a sum weighted by it) in one scan.  A run of
// entries is summarised by (sum m, sum w, its own Q from zero); runs combine
// left to right as (m1+m2, w1+w2, q1 + m1*w2 + q2).  Same run layout and
// passes as gscan_d; use(j, M_j, Q_j) consumes the prefixes.  Returns the
// totals (M, Q) through *mt, *qt.
struct Aff {
  double m, w, q;
};
__device__ __forceinline__ Aff aff_cat(const Aff& a, const Aff& b) {
  return Aff{a.m + b.m, a.w + b.w, a.q + a.m * b.w + b.q};
}
__device__ __forceinline__ Aff aff_shfl_up(const Aff& v, int o) {
  return Aff{__shfl_up_sync(0xffffffffu, v.m, o), __shfl_up_sync(0xffffffffu, v.w, o),
             __shfl_up_sync(0xffffffffu, v.q, o)};
}
__device__ __forceinline__ Aff aff_shfl(const Aff& v, int src) {
  return Aff{__shfl_sync(0xffffffffu, v.m, src), __shfl_sync(0xffffffffu, v.w, src),
             __shfl_sync(0xffffffffu, v.q, src)};
}
// inclusive warp scan of one entry per lane
__device__ __forceinline__ Aff aff_warp_scan(Aff v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    Aff y = aff_shfl_up(v, o);
    if (lane >= o) v = aff_cat(y, v);
  }
  return v;
}

// One warp's walk of [j0, j1) from *run (batches of SB steps, terms read
// first); *run receives the summary of everything walked.
template <class VM, class VW, class U>
__device__ __forceinline__ void warp_walk_aff(int64_t j0, int64_t j1, Aff* run_io, VM valm, VW valw, U use) {
  const int lane = threadIdx.x & 31;
  Aff run = *run_io;
#pragma unroll 1
  for (int64_t jb = j0; jb < j1; jb += 32 * SB) {
    double tm[SB], tw[SB];
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const int64_t j = jb + 32 * u + lane;
      tm[u] = j < j1 ? valm(j) : 0.0;
      tw[u] = j < j1 ? valw(j) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const int64_t j = jb + 32 * u + lane;
      Aff e{tm[u], tw[u], tm[u] * tw[u]};
      Aff s = aff_warp_scan(e);
      if (j < j1) {
        Aff p = aff_cat(run, s);
        use(j, p.m, p.q);
      }
      run = aff_cat(run, aff_shfl(s, 31));
    }
  }
  *run_io = run;
}

template <int C, class VM, class VW, class U>
__device__ __forceinline__ void gscan_aff(const Grp<C>& g, int64_t a, int64_t b, VM valm, VW valw, U use,
                                          double* wbuf /* 3 * HW */, GX& x, double* mt, double* qt) {
  if constexpr (C <= 1) {
    if (C == 0 || blockDim.x == 32) {  // one warp: the walk alone (its final run is the pass-1 summary)
      Aff run{0.0, 0.0, 0.0};
      warp_walk_aff(a, b, &run, valm, valw, use);
      __syncthreads();
      *mt = run.m;
      *qt = run.q;
      return;
    }
  }
  int64_t lo, hi, wlo, whi;
  g.chunk(a, b, &lo, &hi);
  warp_run(lo, hi, &wlo, &whi);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // pass 1: summary of this warp's run
  Aff run{0.0, 0.0, 0.0};
#pragma unroll 1
  for (int64_t jb = wlo; jb < whi; jb += 32 * SB) {
    double tm[SB], tw[SB];
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const int64_t j = jb + 32 * u + lane;
      tm[u] = j < whi ? valm(j) : 0.0;
      tw[u] = j < whi ? valw(j) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < SB; u++) {
      Aff e{tm[u], tw[u], tm[u] * tw[u]};
      run = aff_cat(run, aff_shfl(aff_warp_scan(e), 31));
    }
  }
  if (lane == 0) { wbuf[3 * w] = run.m; wbuf[3 * w + 1] = run.w; wbuf[3 * w + 2] = run.q; }
  __syncthreads();
  Aff pre{0.0, 0.0, 0.0}, tot{0.0, 0.0, 0.0};
  for (int q = 0; q < nw; q++) {  // warps in order (every lane computes the same)
    Aff s{wbuf[3 * q], wbuf[3 * q + 1], wbuf[3 * q + 2]};
    if (q < w) pre = aff_cat(pre, s);
    tot = aff_cat(tot, s);
  }
  if constexpr (C > 1) {  // CTAs of the cluster in rank order
    if (threadIdx.x == 0) { x.d[0] = tot.m; x.d[1] = tot.w; x.d[2] = tot.q; }
    g.sync();
    if (threadIdx.x == 0) {
      cg::cluster_group cl = cg::this_cluster();
      Aff o{0.0, 0.0, 0.0}, t{0.0, 0.0, 0.0};
      const unsigned me = g.rank();
#pragma unroll 1
      for (unsigned r = 0; r < (unsigned)C; r++) {
        Aff s{*cl.map_shared_rank(&x.d[0], r), *cl.map_shared_rank(&x.d[1], r), *cl.map_shared_rank(&x.d[2], r)};
        if (r == me) o = t;
        t = aff_cat(t, s);
      }
      x.dres[0] = o.m; x.dres[1] = o.w; x.dres[2] = o.q;
      x.dres[3] = t.m; x.dres[4] = t.w; x.dres[5] = t.q;
    }
    g.sync();
    Aff o{x.dres[0], x.dres[1], x.dres[2]};
    pre = aff_cat(o, pre);
    tot = Aff{x.dres[3], x.dres[4], x.dres[5]};
  }
  // pass 2: prefixes
  run = pre;
  warp_walk_aff(wlo, whi, &run, valm, valw, use);
  g.sync();
  *mt = tot.m;
  *qt = tot.q;
}
