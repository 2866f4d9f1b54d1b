// clean.cu -- catalogue cleaning: CHECK_RUBISH (haloes_particles.f:259-318)
// and ACCIDENTAL_SUBSTRUCTURE (haloes_particles.f:321-364), called after
// each level's particle refinement (asohf.f:672-675), and the grid finder's
// OVERLAPPING (haloes_grids.f:27-201, called at haloes_grids.f:577 and 1081).
//
// The first two remove (REALCLUS = 0) a halo because of a halo of a LOWER level, and
// the driver appends each level's haloes after the previous levels', so in
// a catalogue whose levels never decrease with the index the Fortran's
// sequential loops reduce to: a halo of level l is removed iff some halo of
// a level below l that is still alive once its own level is settled meets
// the test.  The device settles one level at a time, one thread per halo of
// that level against all lower haloes (tiles in shared memory).  A catalogue
// out of level order is refused (ASOHF_ERR_INVALID).
//
// CHECK_RUBISH's speed ratio A2 is assigned only when both speeds are
// nonzero; otherwise the Fortran reuses the value of the pair before, an
// order-dependent quantity.  Such a pair can only add a removal, so the
// result is known unless a halo no regular pair removes has a zero-speed
// pair passing the distance and mass tests: that case is reported as
// ASOHF_ERR_UNSUPPORTED instead of guessed.
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "common.cuh"

namespace {

struct CleanCat {
  const float *x, *y, *z, *vx, *vy, *vz, *m, *r;
  const int32_t* lev;
  int32_t* rc;
};

#define CT 256  // threads per CTA and lower haloes per shared-memory tile

__device__ __forceinline__ float dist_f(float x1, float y1, float z1, float x2, float y2, float z2) {
  const float dx = __fsub_rn(x1, x2), dy = __fsub_rn(y1, y2), dz = __fsub_rn(z1, z2);
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
}

__device__ __forceinline__ float speed_f(float vx, float vy, float vz) {
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz)));
}

// Every entry sorted by x (sidx: entries in x order, sx: their x).  A CTA
// takes 256 consecutive sorted entries; those of the level run [j0, j1)
// are its haloes, and only the lower haloes whose x lies within reach of
// theirs (a binary search of sx) are tested: a removal needs DIS below
// 1.01 R(J) (CHECK_RUBISH) or below R(I) (ACCIDENTAL_SUBSTRUCTURE), hence
// |dx| below the reach, padded for rounding.
// First sorted position whose x is not below v (UPPER: not at or below v);
// NaN x sort last and count as neither.
template <bool UPPER>
__device__ __forceinline__ int search_x(const float* sx, int n, float v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (UPPER ? sx[mid] <= v : sx[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// The sorted positions [*q0, *q1) whose x lies within w of the x of some
// active halo of the CTA.  DIS never falls below |dx| once the squares are
// normal numbers, so w is kept at least 1e-18; a NaN bound widens to the
// whole axis.  Called by every thread of the CTA.
__device__ __forceinline__ void cta_window(const float* sx, int n, bool act, float xj, float w, int* q0, int* q1) {
  __shared__ float s_red[2][CT / 32];
  __shared__ int s_q[2];
  float lo = INFINITY, hi = -INFINITY;
  if (act) {
    w = w == w ? fmaxf(w, 1e-18f) : INFINITY;
    lo = __fsub_rn(xj, w);
    hi = __fadd_rn(xj, w);
    if (lo != lo) lo = -INFINITY;
    if (hi != hi) hi = INFINITY;
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) { s_red[0][threadIdx.x >> 5] = lo; s_red[1][threadIdx.x >> 5] = hi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    float l = INFINITY, h = -INFINITY;
    for (int k = 0; k < CT / 32; k++) { l = fminf(l, s_red[0][k]); h = fmaxf(h, s_red[1][k]); }
    s_q[0] = l > h ? 0 : search_x<false>(sx, n, l);
    s_q[1] = l > h ? 0 : h == INFINITY ? n : search_x<true>(sx, n, h);
  }
  __syncthreads();
  *q0 = s_q[0];
  *q1 = s_q[1];
}

// Haloes j0..j1-1 (one level, the window's) against the lower haloes
// 0..i1-1: DIS < 1.01 MIN(R), MIN(M)/MAX(M) > 0.2, |V1-V2|/MAX(V) < 3.
__global__ void __launch_bounds__(CT) k_check_rubish(CleanCat c, const int32_t* __restrict__ sidx,
                                                     const float* __restrict__ sx, int n, int j0, int j1, int i1,
                                                     int* zero_speed, int* removed) {
  __shared__ float4 tp[CT];   // x, y, z, m
  __shared__ float2 tr[CT];   // radius, speed (< 0: not a candidate)
  __shared__ int tl[CT];
  const int ps = blockIdx.x * CT + threadIdx.x;
  const int j = ps < n ? sidx[ps] : -1;
  const bool act = j >= j0 && j < j1 && c.rc[j] != 0;
  float xj = 0.f, yj = 0.f, zj = 0.f, mj = 0.f, rj = 0.f, vj = 0.f;
  int lj = 0;
  if (act) {
    xj = c.x[j]; yj = c.y[j]; zj = c.z[j]; mj = c.m[j]; rj = c.r[j]; lj = c.lev[j];
    vj = speed_f(c.vx[j], c.vy[j], c.vz[j]);
  }
  int q0, q1;  // DIS < 1.01 MIN(R) <= 1.01 R(J)
  cta_window(sx, n, act, xj, __fmul_rn(1.02f, rj), &q0, &q1);
  bool kill = false, zero = false;
  for (int t0 = q0; t0 < q1; t0 += CT) {
    __syncthreads();
    const int q = t0 + threadIdx.x;
    if (q < q1) {
      const int i = sidx[q];
      const bool cand = i < i1 && c.rc[i] != 0;
      tp[threadIdx.x] = make_float4(c.x[i], c.y[i], c.z[i], c.m[i]);
      tr[threadIdx.x] = make_float2(c.r[i], cand ? speed_f(c.vx[i], c.vy[i], c.vz[i]) : -1.f);
      tl[threadIdx.x] = c.lev[i];
    }
    __syncthreads();
    if (!act || kill) continue;
    const int nt = q1 - t0 < CT ? q1 - t0 : CT;
    for (int t = 0; t < nt; t++) {
      const float2 rv = tr[t];
      if (rv.y < 0.f || !(lj > tl[t])) continue;
      const float4 p = tp[t];
      const float dis = dist_f(p.x, p.y, p.z, xj, yj, zj);
      const float a1 = __fdiv_rn(fminf(p.w, mj), fmaxf(p.w, mj));
      const float a3 = fminf(rv.x, rj);
      if (!(dis < __fmul_rn(1.01f, a3) && a1 > 0.2f)) continue;
      if (fminf(rv.y, vj) == 0.0f) { zero = true; continue; }  // A2 not assigned for this pair
      const float a2 = __fdiv_rn(fabsf(__fsub_rn(rv.y, vj)), fmaxf(rv.y, vj));
      if (a2 < 3.0f) { kill = true; break; }
    }
  }
  if (act && zero && !kill) atomicOr(zero_speed, 1);
  if (act && kill) {
    c.rc[j] = 0;
    atomicAdd(removed, 1);
  }
}

// Confirmed haloes j0..j1-1 (one level) inside a confirmed lower halo of
// 0..i1-1: DIS + R(J) <= 1.0 R(I); rmax bounds R(I).
__global__ void __launch_bounds__(CT) k_accidental(CleanCat c, const int32_t* __restrict__ sidx,
                                                   const float* __restrict__ sx, int n, int j0, int j1, int i1,
                                                   const float* __restrict__ rmax, int* removed) {
  __shared__ float4 tp[CT];  // x, y, z, radius (NaN: not a confirmed lower halo, fails every test)
  __shared__ int tl[CT];
  const int ps = blockIdx.x * CT + threadIdx.x;
  const int j = ps < n ? sidx[ps] : -1;
  const bool act = j >= j0 && j < j1 && c.rc[j] == -1;
  float xj = 0.f, yj = 0.f, zj = 0.f, rj = 0.f;
  int lj = 0;
  if (act) { xj = c.x[j]; yj = c.y[j]; zj = c.z[j]; rj = c.r[j]; lj = c.lev[j]; }
  int q0, q1;  // DIS <= R(I) - R(J) <= rmax + MAX(-R(J), 0)
  cta_window(sx, n, act, xj, __fmul_rn(1.02f, __fadd_rn(*rmax, fmaxf(-rj, 0.f))), &q0, &q1);
  bool kill = false;
  for (int t0 = q0; t0 < q1; t0 += CT) {
    __syncthreads();
    const int q = t0 + threadIdx.x;
    if (q < q1) {
      const int i = sidx[q];
      tp[threadIdx.x] = make_float4(c.x[i], c.y[i], c.z[i], i < i1 && c.rc[i] == -1 ? c.r[i] : __int_as_float(0x7fffffff));
      tl[threadIdx.x] = c.lev[i];
    }
    __syncthreads();
    if (!act || kill) continue;
    const int nt = q1 - t0 < CT ? q1 - t0 : CT;
    for (int t = 0; t < nt; t++) {
      const float4 p = tp[t];
      if (!(lj > tl[t])) continue;
      const float dis = dist_f(p.x, p.y, p.z, xj, yj, zj);
      if (__fadd_rn(dis, rj) <= __fmul_rn(1.0f, p.w)) { kill = true; break; }
    }
  }
  if (act && kill) {
    c.rc[j] = 0;
    atomicAdd(removed, 1);
  }
}

__global__ void k_x_keys(const float* __restrict__ x, int n, uint32_t* __restrict__ key, int32_t* __restrict__ val) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t u = __float_as_uint(x[i]);
  if (u == 0x80000000u) u = 0u;  // -0 beside +0
  key[i] = x[i] != x[i] ? 0xffffffffu : (u & 0x80000000u) ? ~u : (u | 0x80000000u);  // NaN last
  val[i] = i;
}

__global__ void k_sorted_x(const int32_t* __restrict__ sidx, const float* __restrict__ x, int n,
                           float* __restrict__ sx) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) sx[i] = x[sidx[i]];
}

// Largest radius of a confirmed halo among entries 0..n-1 (radii >= 0 compare as their bits).
__global__ void k_rmax(const float* __restrict__ r, const int32_t* __restrict__ rc, int n, int* out) {
  int m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (rc[i] == -1 && r[i] > 0.f) m = max(m, __float_as_int(r[i]));
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

size_t x_order_bytes(int n) {
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint32_t*)nullptr, (uint32_t*)nullptr, (int32_t*)nullptr,
                                  (int32_t*)nullptr, n > 0 ? n : 1);
  return tb + 20 * (size_t)n + 6 * 256;
}

// Entries in x order: sidx (entry per sorted position) and sx (its x).
int x_order(asohf_ctx* c, const float* dx, int n, int32_t** sidx, float** sx) {
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint32_t*)nullptr, (uint32_t*)nullptr, (int32_t*)nullptr,
                                  (int32_t*)nullptr, n > 0 ? n : 1);
  uint32_t* k0 = (uint32_t*)arena_alloc(c, 4 * (size_t)n + 4);
  uint32_t* k1 = (uint32_t*)arena_alloc(c, 4 * (size_t)n + 4);
  int32_t* v0 = (int32_t*)arena_alloc(c, 4 * (size_t)n + 4);
  int32_t* v1 = (int32_t*)arena_alloc(c, 4 * (size_t)n + 4);
  float* s = (float*)arena_alloc(c, 4 * (size_t)n + 4);
  void* t = arena_alloc(c, tb);
  if (!k0 || !k1 || !v0 || !v1 || !s || !t) return ASOHF_ERR_CAPACITY;
  if (n > 0) {
    int kt_ = ktime_begin(c, "clean_x_sort");
    k_x_keys<<<(n + 255) / 256, 256, 0, c->stream>>>(dx, n, k0, v0);
    ASOHF_CUDA(cub::DeviceRadixSort::SortPairs(t, tb, k0, k1, v0, v1, n, 0, 32, c->stream));
    k_sorted_x<<<(n + 255) / 256, 256, 0, c->stream>>>(v1, dx, n, s);
    ktime_end(c, kt_);
    c->launches += 2;
  }
  *sidx = v1;
  *sx = s;
  return ASOHF_OK;
}

// ---- OVERLAPPING (haloes_grids.f:27-201) ----
//
// The tests of both passes depend on positions, radii and levels only; the
// order enters through REALCLUS.  So every pair (I < J, J of the new level)
// that passes a test is found in parallel (x windows as above) and stored
// as a key (I, J, which of the two is removed), and one CTA replays the
// keys of each pass in the Fortran's (I, J) order over a bitmask of live
// haloes: a pair acts when I was live at the start of its row and J is live
// now.  The replay is exact for any catalogue order.

struct OverlapGeo {
  float pi12, pi43, thr;  // PI/12, 4*PI/3 in REAL*4; VOL_SOLAP_LOW
};

// Pass 1 (|R1-R2| >= DIST) and pass 2 (lens volume above the threshold):
// bit p-1 set when pass p's test holds; *jmin: the partner J is the one removed.
__device__ __forceinline__ int overlap_tests(float r1, float r2, int l1, int l2, float dist, const OverlapGeo& g,
                                             bool* jmin1, bool* jmin2) {
  int t = 0;
  if (fabsf(__fsub_rn(r1, r2)) >= dist) {
    t |= 1;
    *jmin1 = !(r2 > r1 && l2 <= l1);
  }
  const float sm = __fadd_rn(r1, r2), d = __fsub_rn(r1, r2);
  const float bas = __fdiv_rn(dist, sm);
  if (bas < 1.0f) {
    const float xi = bas, u = __fsub_rn(1.0f, xi), m = fminf(r1, r2);
    const float s3 = __fmul_rn(__fmul_rn(sm, sm), sm);
    const float t2 = __fdiv_rn(__fmul_rn(u, u), xi);
    const float t3 = __fsub_rn(__fadd_rn(__fmul_rn(xi, xi), __fmul_rn(2.0f, xi)),
                               __fdiv_rn(__fmul_rn(3.0f, __fmul_rn(d, d)), __fmul_rn(sm, sm)));
    float vint = __fmul_rn(__fmul_rn(__fmul_rn(g.pi12, s3), t2), t3);
    vint = __fdiv_rn(vint, __fmul_rn(g.pi43, __fmul_rn(__fmul_rn(m, m), m)));
    if (vint > g.thr) {
      t |= 2;
      *jmin2 = !(r2 > __fmul_rn(1.5f, r1) && l2 <= l1);
    }
  }
  return t;
}

// One thread per sorted entry; entries j0..j1-1 (the new level) look for
// partners I < J among the sorted x window.  Keys: ((I << b) | J) << 1 | (I removed).
__global__ void __launch_bounds__(CT) k_overlap_pairs(CleanCat c, const int32_t* __restrict__ sidx,
                                                      const float* __restrict__ sx, int n, int j0, int j1,
                                                      const float* __restrict__ rinfo, OverlapGeo g, int b,
                                                      unsigned long long* __restrict__ keys, int cap,
                                                      int* __restrict__ counts) {
  __shared__ float4 tp[CT];  // x, y, z, radius
  __shared__ int2 ti[CT];    // index, level
  const int ps = blockIdx.x * CT + threadIdx.x;
  const int j = ps < n ? sidx[ps] : -1;
  const bool act = j >= j0 && j < j1;
  float xj = 0.f, yj = 0.f, zj = 0.f, rj = 0.f;
  int lj = 0;
  if (act) { xj = c.x[j]; yj = c.y[j]; zj = c.z[j]; rj = c.r[j]; lj = c.lev[j]; }
  // DIST <= |R1-R2| or DIST < R1+R2, both at most R_absmax + |R(J)|; a
  // negative radius lets R1+R2 < 0 pass at any distance (rinfo[1] != 0)
  const float w = rinfo[1] != 0.f ? INFINITY : __fmul_rn(1.02f, __fadd_rn(rinfo[0], fabsf(rj)));
  int q0, q1;
  cta_window(sx, n, act, xj, w, &q0, &q1);
  for (int t0 = q0; t0 < q1; t0 += CT) {
    __syncthreads();
    const int q = t0 + threadIdx.x;
    if (q < q1) {
      const int i = sidx[q];
      tp[threadIdx.x] = make_float4(c.x[i], c.y[i], c.z[i], c.r[i]);
      ti[threadIdx.x] = make_int2(i, c.lev[i]);
    }
    __syncthreads();
    if (!act) continue;
    const int nt = q1 - t0 < CT ? q1 - t0 : CT;
    for (int t = 0; t < nt; t++) {
      const int2 il = ti[t];
      if (il.x >= j) continue;
      const float4 p = tp[t];
      // DIST as SQRT((X1-X2)**2+...) with I first
      const float dist = dist_f(p.x, p.y, p.z, xj, yj, zj);
      bool jm1 = true, jm2 = true;
      const int tt = overlap_tests(p.w, rj, il.y, lj, dist, g, &jm1, &jm2);
      if (!tt) continue;
      const unsigned long long base = (((unsigned long long)il.x << b) | (unsigned long long)j) << 1;
      if (tt & 1) {
        const int k = atomicAdd(&counts[0], 1);
        if (k < cap) keys[k] = base | (jm1 ? 0ull : 1ull);
      }
      if (tt & 2) {
        const int k = atomicAdd(&counts[1], 1);
        if (k < cap) keys[(size_t)cap + k] = base | (jm2 ? 0ull : 1ull);
      }
    }
  }
}

// R_absmax (as float bits, 0 = 0.0f) and whether any radius is negative or NaN.
__global__ void k_radius_info(const float* __restrict__ r, int n, int* out) {
  int m = 0, neg = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float v = r[i];
    if (!(v >= 0.f)) neg = 1;
    if (v == v) m = max(m, __float_as_int(fabsf(v)));
  }
  for (int o = 16; o > 0; o >>= 1) {
    m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    neg |= __shfl_xor_sync(0xffffffffu, neg, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, m);
    if (neg) atomicOr(out + 1, __float_as_int(1.0f));
  }
}

#define OV_CHUNK 4096  // keys staged in shared memory per replay step

// One CTA: live bitmask of entries 0..n-1 (in dynamic shared memory when
// it fits, else gbits), the two passes replayed in order, REALCLUS written
// and COUNT(REALCLUS(j0+1:j1) == 0) added to *zeros.
__global__ void __launch_bounds__(1024) k_overlap_replay(int32_t* __restrict__ rc, int n, int j0, int j1,
                                                         const unsigned long long* __restrict__ keys, int cap,
                                                         const int* __restrict__ counts, int b,
                                                         uint32_t* __restrict__ gbits, int use_smem, int* zeros) {
  extern __shared__ uint32_t s_bits[];
  __shared__ unsigned long long s_keys[OV_CHUNK];
  uint32_t* bits = use_smem ? s_bits : gbits;
  const int nw = (n + 31) >> 5;
  for (int w = threadIdx.x; w < nw; w += blockDim.x) {
    uint32_t v = 0;
    for (int k = 0; k < 32; k++) {
      const int i = (w << 5) + k;
      if (i < n && rc[i] != 0) v |= 1u << k;
    }
    bits[w] = v;
  }
  __syncthreads();
  const unsigned long long jmask = (1ull << b) - 1ull;
  for (int pass = 0; pass < 2; pass++) {
    const int ne = counts[pass];
    const unsigned long long* kp = keys + (size_t)pass * cap;
    long long row = -1;
    bool row_live = false;
    for (int e0 = 0; e0 < ne; e0 += OV_CHUNK) {
      const int m = ne - e0 < OV_CHUNK ? ne - e0 : OV_CHUNK;
      for (int e = threadIdx.x; e < m; e += blockDim.x) s_keys[e] = kp[e0 + e];
      __syncthreads();
      if (threadIdx.x == 0) {
        for (int e = 0; e < m; e++) {
          const unsigned long long k = s_keys[e];
          const int i = (int)(k >> (b + 1)), j = (int)((k >> 1) & jmask);
          if (i != row) {
            row = i;
            row_live = (bits[i >> 5] >> (i & 31)) & 1u;
          }
          if (!row_live || !((bits[j >> 5] >> (j & 31)) & 1u)) continue;
          const int v = (k & 1ull) ? i : j;
          bits[v >> 5] &= ~(1u << (v & 31));
        }
      }
      __syncthreads();
    }
  }
  int z = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (rc[i] != 0 && !((bits[i >> 5] >> (i & 31)) & 1u)) rc[i] = 0;
    if (i >= j0 && i < j1 && rc[i] == 0) z++;
  }
  for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(0xffffffffu, z, o);
  if ((threadIdx.x & 31) == 0 && z) atomicAdd(zeros, z);
}

// Device copies of the fields both routines read (entries 0..n-1), REALCLUS
// read back by the caller; with on_device the caller's arrays are used.
struct CleanIo {
  CleanCat d;
  int32_t* h_rc = nullptr;
  int n = 0;
  bool host = false;
};

// speeds: the velocities and masses are read too (not by OVERLAPPING, whose
// caller may leave them unset).
int clean_in(asohf_ctx* c, const asohf_catalogue* cat, int n, int on_device, CleanIo* io, bool speeds = true) {
  io->n = n;
  io->host = !on_device;
  io->h_rc = cat->realclus;
  ASOHF_CHECK(arena_reserve(c, (on_device ? 0 : (size_t)n * 40 + 10 * 256) + x_order_bytes(n) + 4096));
  if (on_device) {
    io->d = CleanCat{cat->clusrx, cat->clusry, cat->clusrz, speeds ? cat->vx : nullptr, speeds ? cat->vy : nullptr,
                     speeds ? cat->vz : nullptr, speeds ? cat->masa : nullptr, cat->radio, cat->levhal, cat->realclus};
    return ASOHF_OK;
  }
  const float* hf[8] = {cat->clusrx, cat->clusry, cat->clusrz, cat->vx, cat->vy, cat->vz, cat->masa, cat->radio};
  float* df[8];
  for (int q = 0; q < 8; q++) {
    df[q] = nullptr;
    if (!speeds && q >= 3 && q <= 6) continue;
    df[q] = (float*)arena_alloc(c, 4 * (size_t)n + 4);
    if (!df[q]) return ASOHF_ERR_CAPACITY;
    if (n) ASOHF_CUDA(cudaMemcpyAsync(df[q], hf[q], 4 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
  }
  int32_t* dl = (int32_t*)arena_alloc(c, 4 * (size_t)n + 4);
  int32_t* dr = (int32_t*)arena_alloc(c, 4 * (size_t)n + 4);
  if (!dl || !dr) return ASOHF_ERR_CAPACITY;
  if (n) {
    ASOHF_CUDA(cudaMemcpyAsync(dl, cat->levhal, 4 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(dr, cat->realclus, 4 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
  }
  io->d = CleanCat{df[0], df[1], df[2], df[3], df[4], df[5], df[6], df[7], dl, dr};
  return ASOHF_OK;
}

// Level of every entry 0..n-1 on the host (a copy when the catalogue is on
// the device); ASOHF_ERR_INVALID unless the levels never decrease.
int level_runs(asohf_ctx* c, const asohf_catalogue* cat, int n, int on_device, std::vector<int32_t>& lev_v) {
  lev_v.assign((size_t)(n > 0 ? n : 1), 0);
  int32_t* lev = lev_v.data();
  if (on_device) {
    if (n) ASOHF_CUDA(cudaMemcpyAsync(lev, cat->levhal, 4 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  } else if (n) {
    memcpy(lev, cat->levhal, 4 * (size_t)n);
  }
  for (int i = 1; i < n; i++)
    if (lev[i] < lev[i - 1]) return ASOHF_ERR_INVALID;
  return ASOHF_OK;
}

}  // namespace

extern "C" int asohf_check_rubish(asohf_ctx* c, asohf_catalogue* cat, int nclus, int low1, int low2,
                                  int on_device, int32_t* removed) {
  if (!c || !cat || nclus < 0 || nclus > cat->capacity || low1 < 1 || low2 > nclus) return ASOHF_ERR_INVALID;
  if (removed) *removed = 0;
  if (low2 < low1) return ASOHF_OK;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  std::vector<int32_t> lev_v;
  ASOHF_CHECK(level_runs(c, cat, nclus, on_device, lev_v));
  const int32_t* lev = lev_v.data();
  CleanIo io;
  int rc = clean_in(c, cat, nclus, on_device, &io);
  int* dflags = rc == ASOHF_OK ? (int*)arena_alloc(c, 8) : nullptr;
  if (rc != ASOHF_OK || !dflags) return rc != ASOHF_OK ? rc : ASOHF_ERR_CAPACITY;
  ASOHF_CUDA(cudaMemsetAsync(dflags, 0, 8, c->stream));
  int kt_ = ktime_begin(c, "check_rubish");
  int32_t* sidx = nullptr;
  float* sx = nullptr;
  rc = x_order(c, io.d.x, nclus, &sidx, &sx);
  if (rc != ASOHF_OK) return rc;
  // the window's levels in increasing order; each against everything before it
  for (int a = low1 - 1; a < low2;) {
    int b = a;
    while (b < low2 && lev[b] == lev[a]) b++;
    k_check_rubish<<<(nclus + CT - 1) / CT, CT, 0, c->stream>>>(io.d, sidx, sx, nclus, a, b, a, dflags,
                                                                 dflags + 1);
    c->launches++;
    a = b;
  }
  ktime_end(c, kt_);
  ASOHF_CUDA(cudaGetLastError());
  int hflags[2];
  ASOHF_CUDA(cudaMemcpyAsync(hflags, dflags, 8, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  if (hflags[0]) return ASOHF_ERR_UNSUPPORTED;  // a live pair with a zero speed (see the top of the file)
  if (io.host && low2 >= low1)
    ASOHF_CUDA(cudaMemcpyAsync(cat->realclus + low1 - 1, io.d.rc + low1 - 1, 4 * (size_t)(low2 - low1 + 1),
                               cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  if (removed) *removed = hflags[1];
  return ASOHF_OK;
}

extern "C" int asohf_accidental_substructure(asohf_ctx* c, asohf_catalogue* cat, int nclus, int on_device,
                                             int32_t* removed) {
  if (!c || !cat || nclus < 0 || nclus > cat->capacity) return ASOHF_ERR_INVALID;
  if (removed) *removed = 0;
  if (nclus == 0) return ASOHF_OK;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  std::vector<int32_t> lev_v;
  ASOHF_CHECK(level_runs(c, cat, nclus, on_device, lev_v));
  const int32_t* lev = lev_v.data();
  CleanIo io;
  int rc = clean_in(c, cat, nclus, on_device, &io);
  int* dcount = rc == ASOHF_OK ? (int*)arena_alloc(c, 8) : nullptr;
  if (rc != ASOHF_OK || !dcount) return rc != ASOHF_OK ? rc : ASOHF_ERR_CAPACITY;
  ASOHF_CUDA(cudaMemsetAsync(dcount, 0, 8, c->stream));  // removals, largest confirmed radius
  int kt_ = ktime_begin(c, "accidental_substructure");
  int32_t* sidx = nullptr;
  float* sx = nullptr;
  rc = x_order(c, io.d.x, nclus, &sidx, &sx);
  if (rc != ASOHF_OK) return rc;
  k_rmax<<<148, 256, 0, c->stream>>>(io.d.r, io.d.rc, nclus, dcount + 1);
  c->launches++;
  // level by level: the lowest level is never removed, each next one is
  // settled against the survivors of all levels before it
  int a = 0;
  while (a < nclus && lev[a] == lev[0]) a++;
  while (a < nclus) {
    int b = a;
    while (b < nclus && lev[b] == lev[a]) b++;
    k_accidental<<<(nclus + CT - 1) / CT, CT, 0, c->stream>>>(io.d, sidx, sx, nclus, a, b, a,
                                                              (const float*)(dcount + 1), dcount);
    c->launches++;
    a = b;
  }
  ktime_end(c, kt_);
  ASOHF_CUDA(cudaGetLastError());
  int hcount = 0;
  ASOHF_CUDA(cudaMemcpyAsync(&hcount, dcount, 4, cudaMemcpyDeviceToHost, c->stream));
  if (io.host)
    ASOHF_CUDA(cudaMemcpyAsync(cat->realclus, io.d.rc, 4 * (size_t)nclus, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  if (removed) *removed = hcount;
  return ASOHF_OK;
}

extern "C" int asohf_overlapping(asohf_ctx* c, asohf_catalogue* cat, int ir, const int32_t* nhallev,
                                 float vol_solap_low, int on_device, int32_t* removed) {
  if (!c || !cat || !nhallev || ir < 0) return ASOHF_ERR_INVALID;
  long long lowh3 = 1;
  for (int l = 0; l < ir; l++) {
    if (nhallev[l] < 0) return ASOHF_ERR_INVALID;
    lowh3 += nhallev[l];
  }
  if (nhallev[ir] < 0) return ASOHF_ERR_INVALID;
  const long long lowh2 = lowh3 - 1 + nhallev[ir];
  if (lowh2 > cat->capacity) return ASOHF_ERR_INVALID;
  if (removed) *removed = 0;
  if (lowh2 > (1 << 28)) return ASOHF_ERR_CAPACITY;  // 64-bit pair keys, int pair counts
  if (lowh2 < lowh3) return ASOHF_OK;  // no halo at this level: no pair, no count
  const int n = (int)lowh2, j0 = (int)lowh3 - 1, j1 = (int)lowh2;
  int b = 1;
  while (b < 31 && (1ll << b) < n) b++;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  CleanIo io;
  ASOHF_CHECK(clean_in(c, cat, n, on_device, &io, false));
  int* dw = (int*)arena_alloc(c, 32);  // pair counts [2], radius info [2], zeros
  if (!dw) return ASOHF_ERR_CAPACITY;
  ASOHF_CUDA(cudaMemsetAsync(dw, 0, 32, c->stream));
  int kt_ = ktime_begin(c, "overlapping");
  int32_t* sidx = nullptr;
  float* sx = nullptr;
  ASOHF_CHECK(x_order(c, io.d.x, n, &sidx, &sx));
  k_radius_info<<<148, 256, 0, c->stream>>>(io.d.r, n, dw + 2);
  c->launches++;
  const float pi = (float)acos(-1.0);
  const OverlapGeo g{pi / 12.0f, 4.0f * pi / 3.0f, vol_solap_low};
  const int nw = (n + 31) >> 5;
  const bool smem = (size_t)nw * 4 <= 192u * 1024u;
  int cap = 2 * n + 1024, cnt[2] = {0, 0};
  unsigned long long *keys = nullptr, *keys2 = nullptr;
  uint32_t* gbits = nullptr;
  void* tmp = nullptr;
  size_t tb = 0;
  for (int attempt = 0; attempt < 2; attempt++) {
    tb = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tb, (unsigned long long*)nullptr, (unsigned long long*)nullptr, cap);
    ASOHF_CHECK(seg_reserve(c, 32 * (size_t)cap + tb + (smem ? 0 : 4 * (size_t)nw) + 4096));
    keys = (unsigned long long*)seg_alloc(c, 16 * (size_t)cap);
    keys2 = (unsigned long long*)seg_alloc(c, 16 * (size_t)cap);
    tmp = seg_alloc(c, tb);
    gbits = smem ? nullptr : (uint32_t*)seg_alloc(c, 4 * (size_t)nw);
    if (!keys || !keys2 || !tmp || (!smem && !gbits)) return ASOHF_ERR_CAPACITY;
    ASOHF_CUDA(cudaMemsetAsync(dw, 0, 8, c->stream));
    k_overlap_pairs<<<(n + CT - 1) / CT, CT, 0, c->stream>>>(io.d, sidx, sx, n, j0, j1, (const float*)(dw + 2), g,
                                                             b, keys, cap, dw);
    c->launches++;
    ASOHF_CUDA(cudaGetLastError());
    ASOHF_CUDA(cudaMemcpyAsync(cnt, dw, 8, cudaMemcpyDeviceToHost, c->stream));
    ASOHF_CUDA(cudaStreamSynchronize(c->stream));
    if (cnt[0] <= cap && cnt[1] <= cap) break;
    if (attempt == 1) return ASOHF_ERR_CAPACITY;  // not reached: the pair set does not change between runs
    cap = (cnt[0] > cnt[1] ? cnt[0] : cnt[1]) + 1024;
  }
  for (int p = 0; p < 2; p++)
    if (cnt[p] > 0) {
      size_t t = tb;
      ASOHF_CUDA(cub::DeviceRadixSort::SortKeys(tmp, t, keys + (size_t)p * cap, keys2 + (size_t)p * cap, cnt[p], 0,
                                                2 * b + 1, c->stream));
      c->launches++;
    }
  const size_t dyn = smem ? 4 * (size_t)nw : 0;
  ASOHF_CUDA(cudaFuncSetAttribute(k_overlap_replay, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  k_overlap_replay<<<1, 1024, dyn, c->stream>>>(io.d.rc, n, j0, j1, keys2, cap, dw, b, gbits, smem ? 1 : 0,
                                                dw + 4);
  c->launches++;
  ktime_end(c, kt_);
  ASOHF_CUDA(cudaGetLastError());
  int z = 0;
  ASOHF_CUDA(cudaMemcpyAsync(&z, dw + 4, 4, cudaMemcpyDeviceToHost, c->stream));
  if (io.host) ASOHF_CUDA(cudaMemcpyAsync(cat->realclus, io.d.rc, 4 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  if (removed) *removed = z;
  return ASOHF_OK;
}

// RE_SORT_HALOES (haloes_particles.f:2-56) on the host arrays: one pass over
// the level's window moving the kept entries down; the renumbering uses the
// final old->new map of the window (the Fortran's RESORT(REALCLUS(I)) is
// undefined where REALCLUS points past I or at a dropped entry).
extern "C" int asohf_re_sort_haloes(asohf_ctx* c, asohf_catalogue* cat, int32_t* nhallev, int ir, uint8_t* keep) {
  if (!c || !cat || !nhallev || ir < 0) return ASOHF_ERR_INVALID;
  int64_t low1 = 1, low2 = 0;
  for (int l = 0; l < ir; l++) low1 += nhallev[l];
  low2 = low1 - 1 + nhallev[ir];
  if (nhallev[ir] < 0 || low2 > cat->capacity || low1 < 1) return ASOHF_ERR_INVALID;
  const int64_t w = low2 - low1 + 1;
  std::vector<int32_t> resort((size_t)(w > 0 ? w : 1), 0);
  int64_t j = low1 - 1;  // 0-based destination
  for (int64_t i = low1 - 1; i < low2; i++) {
    const bool k = cat->realclus[i] != 0;
    if (keep) keep[i - (low1 - 1)] = k ? 1 : 0;
    if (k) resort[(size_t)(i - (low1 - 1))] = (int32_t)(++j);  // 1-based new position
  }
  const int64_t kept = j - (low1 - 1);
  if (kept != w) {
    j = low1 - 1;
    for (int64_t i = low1 - 1; i < low2; i++) {
      const int32_t rc = cat->realclus[i];
      if (rc == 0) continue;
      cat->clusrx[j] = cat->clusrx[i];
      cat->clusry[j] = cat->clusry[i];
      cat->clusrz[j] = cat->clusrz[i];
      cat->radio[j] = cat->radio[i];
      cat->masa[j] = cat->masa[i];
      cat->levhal[j] = cat->levhal[i];
      cat->patchclus[j] = cat->patchclus[i];
      cat->dmpclus[j] = cat->dmpclus[i];
      cat->clusrxcm[j] = cat->clusrxcm[i];
      cat->clusrycm[j] = cat->clusrycm[i];
      cat->clusrzcm[j] = cat->clusrzcm[i];
      cat->realclus[j] = (rc > 0 && rc >= low1 && rc <= low2) ? resort[(size_t)(rc - low1)] : rc;
      j++;
    }
  }
  nhallev[ir] = (int32_t)kept;
  cat->nclus = (int32_t)(low1 - 1 + kept);
  return ASOHF_OK;
}
