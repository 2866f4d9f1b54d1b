// halo.cu -- PRUNE_POOR_HALOES and HALOFIND_PARTICLES on sm_100a.
//
// Pipeline of one call (haloes lowh1..lowh2, largest first):
//   k_halo_grow   density-peak recentering and the spherical-overdensity
//                 growth (counts and sums only);
//   (scan)        segment offsets from the final member counts;
//   k_halo_gather (halo, distance) keys and x-sorted positions of the
//                 members into each halo's segment;
//   radix sort    of all segments at once on (halo, distance), then
//   k_tiefix      orders equal distances by position, descending, which is
//                 ARGSORT's order (num.f:181) over the slab-ordered list;
//   k_halo_main   virial index, escape-velocity and sigma-clipping
//                 unbinding, SO walk, bound-particle properties;
//   k_write_ids   bound-particle IDs in halo order (PARTICLES_PER_HALO).
// Each per-halo kernel runs in two tiers: haloes of 32768 members or more
// (asohf_set_cluster_threshold)
// are refined by a thread-block cluster (16 CTAs, or 8 where 16 cannot be
// co-scheduled) that splits every pass over the members, the others by one
// CTA each on a second stream, so the clusters and the single CTAs share the
// SMs instead of the largest halo finishing alone.
// The reference scans a full-(y,z) x-slab per query (haloes_particles.f:
// 117-143); the column index returns the same member sets from the columns a
// sphere overlaps.
#include <vector>
#include <stdlib.h>
#include <string.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "halo_dev.cuh"

// ---------------------------------------------------------------- catalogue mirror
// A call reads and writes the entries of its own haloes, [w0, n), and (the
// subhalo calls) a few fields of earlier entries, their hosts.  With a host
// catalogue only those ranges cross PCIe; the device arrays keep the
// caller's indexing.
struct CatMirror {
  asohf_catalogue h;  // caller's
  asohf_catalogue d;  // device
  int n;              // entries 0..n-1 addressable
  int w0;             // first entry of the call's window
  bool host;
  bool prune;         // only the fields PRUNE_POOR_HALOES reads and writes move
};

#define CAT_F1(X) X(masa) X(radio) X(clusrx) X(clusry) X(clusrz) X(clusrxcm) X(clusrycm) X(clusrzcm) \
  X(msub) X(rsub) X(concentra) X(vmaxclus) X(vx) X(vy) X(vz) X(mean_vr) X(vcmax) X(mcmax) X(rcmax)     \
  X(m200c) X(r200c) X(m500c) X(r500c) X(m2500c) X(r2500c) X(m200m) X(r200m) X(m500m) X(r500m)          \
  X(m2500m) X(r2500m) X(velocity_dispersion) X(kinetic_e) X(potential_e)
#define CAT_I1(X) X(patchclus) X(realclus) X(levhal) X(dmpclus) X(iplip)
#define CAT_FM(X) X(angularm, 3) X(profiles, 2 * ASOHF_NBINS) X(eigenval, 3) X(inertia_tensor, 6)
// fields PRUNE_POOR_HALOES reads, and writes
#define CAT_PRUNE_IN(X) X(clusrx) X(clusry) X(clusrz) X(radio) X(realclus) X(dmpclus)
#define CAT_PRUNE_OUT(X) X(realclus) X(dmpclus)
// fields of host entries the subhalo kernels read
#define CAT_HOST(X) X(realclus, 1) X(masa, 1) X(msub, 1) X(clusrx, 1) X(clusry, 1) X(clusrz, 1) \
  X(profiles, 2 * ASOHF_NBINS)

static size_t cat_bytes(int n) {
  size_t b = 0;
#define F(f) b += 4 * (size_t)n + 256;
  CAT_F1(F) CAT_I1(F)
#undef F
#define M(f, w) b += 4 * (size_t)n * (w) + 256;
  CAT_FM(M)
#undef M
  b += 8 * (size_t)n + 256;  // indcs
  return b;
}

static int cat_mirror_in(asohf_ctx* c, asohf_catalogue* h, int n, int on_device, CatMirror* m, int w0,
                         bool hosts = false, bool prune = false) {
  m->h = *h;
  m->n = n;
  m->w0 = w0 < 0 ? 0 : (w0 > n ? n : w0);
  m->host = !on_device;
  m->prune = prune;
  if (on_device) { m->d = *h; return ASOHF_OK; }
  m->d = *h;
  const size_t a = (size_t)m->w0, cnt = (size_t)(n - m->w0);
  if (prune) {  // the prune kernels touch six fields of the window
#define P(f)                                                                                        \
  m->d.f = (decltype(m->d.f))arena_alloc(c, 4 * (size_t)n + 4);                                    \
  if (!m->d.f) return ASOHF_ERR_CAPACITY;                                                           \
  if (cnt) ASOHF_CUDA(cudaMemcpyAsync(m->d.f + a, h->f + a, 4 * cnt, cudaMemcpyHostToDevice, c->stream));
    CAT_PRUNE_IN(P)
#undef P
    return ASOHF_OK;
  }
#define F(f)                                                                                        \
  m->d.f = (decltype(m->d.f))arena_alloc(c, 4 * (size_t)n + 4);                                    \
  if (!m->d.f) return ASOHF_ERR_CAPACITY;                                                           \
  if (cnt) ASOHF_CUDA(cudaMemcpyAsync(m->d.f + a, h->f + a, 4 * cnt, cudaMemcpyHostToDevice, c->stream));
  CAT_F1(F) CAT_I1(F)
#undef F
#define M(f, w)                                                                                     \
  m->d.f = (float*)arena_alloc(c, 4 * (size_t)n * (w) + 4);                                        \
  if (!m->d.f) return ASOHF_ERR_CAPACITY;                                                           \
  if (cnt) ASOHF_CUDA(cudaMemcpyAsync(m->d.f + a * (w), h->f + a * (w), 4 * cnt * (w), cudaMemcpyHostToDevice, \
                                      c->stream));
  CAT_FM(M)
#undef M
  m->d.indcs = (int32_t*)arena_alloc(c, 8 * (size_t)n + 8);
  if (!m->d.indcs) return ASOHF_ERR_CAPACITY;
  if (cnt) ASOHF_CUDA(cudaMemcpyAsync(m->d.indcs + 2 * a, h->indcs + 2 * a, 8 * cnt, cudaMemcpyHostToDevice, c->stream));
  if (hosts && a) {
#define H(f, w) ASOHF_CUDA(cudaMemcpyAsync(m->d.f, h->f, 4 * a * (w), cudaMemcpyHostToDevice, c->stream));
    CAT_HOST(H)
#undef H
  }
  return ASOHF_OK;
}

static int cat_mirror_out(asohf_ctx* c, CatMirror* m) {
  if (!m->host || m->n == m->w0) return ASOHF_OK;
  const size_t a = (size_t)m->w0, cnt = (size_t)(m->n - m->w0);
  if (m->prune) {
#define P(f) ASOHF_CUDA(cudaMemcpyAsync(m->h.f + a, m->d.f + a, 4 * cnt, cudaMemcpyDeviceToHost, c->stream));
    CAT_PRUNE_OUT(P)
#undef P
    ASOHF_CUDA(cudaStreamSynchronize(c->stream));
    return ASOHF_OK;
  }
#define F(f) ASOHF_CUDA(cudaMemcpyAsync(m->h.f + a, m->d.f + a, 4 * cnt, cudaMemcpyDeviceToHost, c->stream));
  CAT_F1(F) CAT_I1(F)
#undef F
#define M(f, w) \
  ASOHF_CUDA(cudaMemcpyAsync(m->h.f + a * (w), m->d.f + a * (w), 4 * cnt * (w), cudaMemcpyDeviceToHost, c->stream));
  CAT_FM(M)
#undef M
  ASOHF_CUDA(cudaMemcpyAsync(m->h.indcs + 2 * a, m->d.indcs + 2 * a, 8 * cnt, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  return ASOHF_OK;
}

static ColIdx col_idx(asohf_ctx* c, const asohf_consts* k) {
  ColIdx ci;
  ci.cp = c->d_colpart;
  ci.start = c->d_colstart;
  ci.ncol = c->col_n;
  ci.xl = c->col_xl;
  ci.cdx = c->col_dx;
  ci.nd = c->d_ndmpart_x;
  ci.nmax = k->nx;
  ci.dx = k->dx;
  ci.xldom = -k->lado0 / 2.0f;
  return ci;
}

static Store store_of(asohf_ctx* c) {
  Store S;
  S.x = c->p.x; S.y = c->p.y; S.z = c->p.z;
  S.vx = c->p.vx; S.vy = c->p.vy; S.vz = c->p.vz;
  S.m = c->p.m; S.id = c->p.id;
  S.rows = c->rows_cur >= 0 ? c->rows[c->rows_cur] : nullptr;
  S.meq = (c->p.n > 0 && c->mmin == c->norma) ? c->norma : 0.0f;  // no gather of equal masses
  S.norma = c->norma;
  S.eqmass_lt8 = c->norma / c->mmin < 8.0f;
  return S;
}

static HConst hconst(const asohf_consts* k, const asohf_mesh* mesh) {
  HConst h;
  h.rote = k->rote; h.rete = k->rete; h.pi = k->pi; h.cgr = k->cgr; h.um = k->um; h.uv = k->uv;
  h.contrastec = k->contrastec; h.omegaz = k->omegaz; h.fdm = k->fdm; h.zeta = k->zeta;
  h.min_num_part = k->min_num_part;
  h.want_ids = (k->flag_wdm == 1 || k->var > 1);
  h.energies = k->do_compute_energies == 1;
  h.max_part_dsum = k->max_part_dsum;
  h.nl = mesh ? mesh->nl : 0;
  int acc = mesh ? mesh->npatch[0] : 0;
  for (int ir = 0; ir <= ASOHF_NLEVELS + 1; ir++) { h.lev_lo[ir] = 0; h.lev_hi[ir] = -1; }
  for (int ir = 1; ir <= h.nl; ir++) {
    h.lev_lo[ir] = acc + 1;
    h.lev_hi[ir] = acc + mesh->npatch[ir];
    acc += mesh->npatch[ir];
  }
  return h;
}

// ---------------------------------------------------------------- prune
// COUNT_PARTICLES_HALO (haloes_particles.f:147-182) for haloes low1..low2.
__global__ void __launch_bounds__(HB) k_prune(ColIdx ci, asohf_catalogue cat, int low1, float facrad,
                                             int min_num_part) {
  __shared__ long long lred[32];
  int i0 = low1 - 1 + blockIdx.x;
  float cx = cat.clusrx[i0], cy = cat.clusry[i0], cz = cat.clusrz[i0];
  float r = __fmul_rn(facrad, cat.radio[i0]);
  float r2 = __fmul_rn(r, r);
  int64_t lo, hi;
  slab_range(ci, cx, r, &lo, &hi);
  long long cnt = 0;
  query_box(ci, cx, cy, cz, r, [&](const float4& e) {
    int p = ppos(e);
    if (p < lo || p >= hi) return;
    float bx = __fsub_rn(e.x, cx);
    bx = __fmul_rn(bx, bx);
    if (bx > r2) return;
    float by = __fsub_rn(e.y, cy);
    by = __fmul_rn(by, by);
    if (by > r2) return;
    float bz = __fsub_rn(e.z, cz);
    bz = __fmul_rn(bz, bz);
    if (bz > r2) return;
    if (__fadd_rn(__fadd_rn(bx, by), bz) < r2) cnt++;
  });
  cnt = block_sum_ll(cnt, lred);
  if (threadIdx.x == 0) {
    if (cnt < min_num_part) cat.realclus[i0] = 0;
    cat.dmpclus[i0] = (int32_t)cnt;
  }
}

__global__ void k_prune_nocount(asohf_catalogue cat, int low1, int low2, int min_num_part) {
  int i0 = low1 - 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i0 < low2 && cat.dmpclus[i0] < min_num_part) cat.realclus[i0] = 0;
}

extern "C" int asohf_prune_poor_haloes(asohf_ctx* c, const asohf_consts* k, asohf_catalogue* cat,
                                       int low1, int low2, float facrad, int do_need_to_count,
                                       int on_device) {
  if (!c || !k || !cat || low1 < 1 || low2 > cat->nclus) return ASOHF_ERR_INVALID;
  if (low2 < low1) return ASOHF_OK;
  if (do_need_to_count == 1 && c->nx_sorted != k->nx) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  double ht = htime_now();
  arena_reset(c);
  ASOHF_CHECK(arena_reserve(c, cat_bytes(low2) + 4096));
  CatMirror m;
  ASOHF_CHECK(cat_mirror_in(c, cat, low2, on_device, &m, low1 - 1, false, true));
  int nh = low2 - low1 + 1;
  if (do_need_to_count == 1)
    {
      int kt_ = ktime_begin(c, "prune");
      k_prune<<<nh, HB, 0, c->stream>>>(col_idx(c, k), m.d, low1, facrad, k->min_num_part);
      ktime_end(c, kt_);
    }
  else
    k_prune_nocount<<<(nh + 255) / 256, 256, 0, c->stream>>>(m.d, low1, low2, k->min_num_part);
  c->launches++;
  ASOHF_CUDA(cudaGetLastError());
  ASOHF_CHECK(cat_mirror_out(c, &m));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  htime_end(c, "host:prune", ht);
  return ASOHF_OK;
}

// ---------------------------------------------------------------- launch helpers
// Size tiers of the per-halo launches, by member count: at least
// ctx->cluster_min -> a thread-block cluster; at least ctx->tier2_k -> one
// CTA of 256 threads; at least ctx->tier1_k -> 128 threads; the rest -> 32
// threads.  The small CTAs keep many small haloes resident per SM, whose
// passes are short and bound by latency.  The tiers run concurrently on four
// streams.
#define BIG_K 32768
#define TIER2_K 2048
#define TIER1_K 256
static const int kTierThreads[3] = {32, 128, 256};

template <typename... P, typename... A>
static cudaError_t launch_grp(void (*kern)(P...), int C, int ngroups, int threads, cudaStream_t s, A&&... args) {
  if (ngroups <= 0) return cudaSuccess;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(ngroups * C));
  cfg.blockDim = dim3((unsigned)threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = C > 1 ? 1 : 0;
  if (C > 8) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

// The side streams start after the work queued so far on the context stream;
// the context stream then waits for all of them.
static int fork_all(asohf_ctx* c) {
  ASOHF_CUDA(cudaEventRecord(c->ev_fork, c->stream));
  for (int i = 0; i < asohf_ctx::NSIDE; i++) ASOHF_CUDA(cudaStreamWaitEvent(c->side[i], c->ev_fork, 0));
  return ASOHF_OK;
}
static int join_all(asohf_ctx* c) {
  for (int i = 0; i < asohf_ctx::NSIDE; i++) {
    ASOHF_CUDA(cudaEventRecord(c->ev_join[i], c->side[i]));
    ASOHF_CUDA(cudaStreamWaitEvent(c->stream, c->ev_join[i], 0));
  }
  return ASOHF_OK;
}

struct Tiers {
  int n[4];           // slots per tier (0: 32 threads, 1: 128, 2: 256, 3: cluster)
  int32_t* slots[4];  // device slot lists
};

// Buckets entries 0..n-1 by hcount[] into the tiers; entry i stands for
// slot ids[i] (slot i when ids is null).  dbuf holds n entries.
static int split_tiers(asohf_ctx* c, const int32_t* hcount, int n, int32_t* dbuf, Tiers* T,
                       const int32_t* ids = nullptr) {
  std::vector<int32_t> h_v((size_t)(n > 0 ? n : 1));
  int32_t* h = h_v.data();
  int cnt[4] = {0, 0, 0, 0};
  auto tier = [&](int32_t k) {
    return k >= c->cluster_min ? 3 : (k >= c->tier2_k ? 2 : (k >= c->tier1_k ? 1 : 0));
  };
  for (int i = 0; i < n; i++) cnt[tier(hcount[i])]++;
  int off[4];
  off[3] = 0;
  off[2] = cnt[3];
  off[1] = off[2] + cnt[2];
  off[0] = off[1] + cnt[1];
  int fill[4] = {off[0], off[1], off[2], off[3]};
  for (int i = 0; i < n; i++) h[fill[tier(hcount[i])]++] = ids ? ids[i] : i;
  if (n) ASOHF_CUDA(cudaMemcpyAsync(dbuf, h, 4 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  for (int t = 0; t < 4; t++) {
    T->n[t] = cnt[t];
    T->slots[t] = dbuf + off[t];
  }
  return ASOHF_OK;
}

// Reorders the cluster tier's slot list (tier 3, at the front of its
// device buffer) into runs for clusters of cb (at most 16), 8 and 4 CTAs by
// member count: a CTA's share stays near ctx->cluster_share entries.
static int split_cluster_tier(asohf_ctx* c, const int32_t* hcount, int n, int cb, Tiers* T, int nsub[3],
                              int32_t* sub[3]) {
  const int64_t sh = c->cluster_share;
  auto pick = [&](int32_t k) {
    if (cb < 8) return 0;                      // no clusters: one CTA each
    if (cb < 16) return k > 4 * sh ? 0 : 2;  // 8 CTAs at most
    return k > 8 * sh ? 0 : (k > 4 * sh ? 1 : 2);
  };
  std::vector<int32_t> h_v((size_t)(T->n[3] > 0 ? T->n[3] : 1));
  int32_t* h = h_v.data();
  int cnt[3] = {0, 0, 0};
  for (int i = 0; i < n; i++)
    if (hcount[i] >= c->cluster_min) cnt[pick(hcount[i])]++;
  int fill[3] = {0, cnt[0], cnt[0] + cnt[1]};
  for (int i = 0; i < n; i++)
    if (hcount[i] >= c->cluster_min) h[fill[pick(hcount[i])]++] = i;
  if (T->n[3]) ASOHF_CUDA(cudaMemcpyAsync(T->slots[3], h, 4 * (size_t)T->n[3], cudaMemcpyHostToDevice, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  for (int q = 0; q < 3; q++) {
    nsub[q] = cnt[q];
    sub[q] = T->slots[3] + (q == 0 ? 0 : (q == 1 ? cnt[0] : cnt[0] + cnt[1]));
  }
  return ASOHF_OK;
}

template <int C>
__device__ __forceinline__ int group_slot(const int32_t* slots) {
  if constexpr (C <= 1) return slots[blockIdx.x];
  else return slots[blockIdx.x / C];
}

__device__ __forceinline__ bool leader(unsigned rank) { return rank == 0 && threadIdx.x == 0; }

// ---------------------------------------------------------------- grow
struct GrowOut {
  float *cx, *cy, *cz;     // recentred centre
  float *rgather;          // radius of the last gather (members)
  float *rclus;            // RCLUS after the last growth step
  int32_t* konta;          // members
  double* masadm;          // their mass
  int32_t* status;
};

__device__ __forceinline__ int level_of_patch(const HConst& H, int ipatch) {
  int irr;
  for (irr = 1; irr <= H.nl; irr++)
    if (H.lev_lo[irr] <= ipatch && ipatch <= H.lev_hi[irr]) break;
  return irr;
}

// Member-count caps of the growth by launch shape: a halo whose sphere
// outgrows the cap of its CTA size stops, leaves its centre and radius in
// GrowOut and is resumed by a larger group (the cost of the growth is known
// only as it runs: a small candidate inside a large halo grows to its size).
struct GrowCaps {
  int64_t c32, c128, c256;
};
#define GROW_ESCALATE 100  // status of a halo handed to a larger group

// Recentering + growth of HALOFIND_PARTICLES (haloes_particles.f:741-849);
// with resume set, the growth restarts from the saved centre and radius.
template <int C>
__global__ void __launch_bounds__(HB, 3)
k_halo_grow(const int32_t* __restrict__ slots, Store S, ColIdx ci, HConst H, asohf_catalogue cat,
            const int32_t* __restrict__ work, GrowOut o, GrowCaps caps, int resume) {
  __shared__ RecShared sh;
  Grp<C> G;
  int slot = group_slot<C>(slots);
  int i0 = work[slot];
  unsigned rk = G.rank();
  if (cat.realclus[i0] == 0) {
    if (leader(rk)) { o.konta[slot] = 0; o.status[slot] = 0; }
    return;
  }
  const int64_t kcap = C > 1 ? LLONG_MAX
                             : (blockDim.x <= 32 ? caps.c32 : (blockDim.x <= 128 ? caps.c128 : caps.c256));
  float cx, cy, cz, rclus;
  if (!resume) {
    int irr = level_of_patch(H, cat.patchclus[i0]);
    cx = cat.clusrx[i0]; cy = cat.clusry[i0]; cz = cat.clusrz[i0];
    float dxpamin = __fdiv_rn(ci.dx, exp2f((float)irr));
    if (!recenter_group(G, S, ci, &cx, &cy, &cz, cat.radio[i0], dxpamin, sh)) {
      if (leader(rk)) { o.konta[slot] = 0; o.status[slot] = ASOHF_ERR_CAPACITY; }
      return;
    }
    rclus = cat.radio[i0];
  } else {
    cx = o.cx[slot]; cy = o.cy[slot]; cz = o.cz[slot];
    rclus = o.rclus[slot];
  }
  float mino = __fmul_rn(fminf(200.0f, H.contrastec), H.fdm);
  float den0 = __fmul_rn(__fmul_rn(H.rote, __fmul_rn(__fmul_rn(H.rete, H.rete), H.rete)),
                         __fdiv_rn(__fmul_rn(4.0f, H.pi), 3.0f));
  float delta2 = __fmul_rn(100.0f, mino);
  float rg = rclus;
  long long konta = 0;
  double masadm = 0.0;
  int guard = 0;
  while (delta2 > __fmul_rn(0.99f, mino)) {
    int64_t lo, hi;
    slab_range(ci, cx, rclus, &lo, &hi);
    long long c = 0;
    double ms = 0.0;
    float bas = -1.0f;
    gquery_box(G, ci, cx, cy, cz, rclus, sh.qb, [&](const float4& e) {
      int p = ppos(e);
      if (p < lo || p >= hi) return;
      float a = dist3(e.x, e.y, e.z, cx, cy, cz);
      if (a < rclus) {
        c++;
        ms += (double)S.mass(p);
        bas = fmaxf(bas, a);
      }
    });
    konta = gsum_ll(G, c, sh.lred, sh.x);
    if (konta > kcap) {  // hand over to a larger group at this radius
      if (leader(rk)) {
        o.cx[slot] = cx; o.cy[slot] = cy; o.cz[slot] = cz;
        o.rclus[slot] = rclus;
        o.konta[slot] = (int32_t)(konta < INT32_MAX ? konta : INT32_MAX);
        o.status[slot] = GROW_ESCALATE;
      }
      return;
    }
    masadm = gsum_d(G, ms, sh.dred, sh.x);
    bas = gmax_f(G, bas, sh.fred, sh.x);
    float den = __fmul_rn(den0, __fmul_rn(__fmul_rn(bas, bas), bas));
    delta2 = (float)(masadm / (double)den);
    rg = rclus;
    if (delta2 > __fmul_rn(0.9f, mino)) rclus = __fmul_rn(1.25f, rclus);
    if (++guard > 100000) break;
  }
  if (leader(rk)) {
    cat.clusrx[i0] = cx; cat.clusry[i0] = cy; cat.clusrz[i0] = cz;
    o.cx[slot] = cx; o.cy[slot] = cy; o.cz[slot] = cz;
    o.rgather[slot] = rg;
    o.rclus[slot] = rclus;
    o.masadm[slot] = masadm;
    o.status[slot] = 0;
    if (masadm <= 0.0 || konta == 0) {
      cat.realclus[i0] = 0;
      o.konta[slot] = 0;
    } else {
      o.konta[slot] = (int32_t)konta;
    }
  }
}

// ---------------------------------------------------------------- gather
// Members of sphere (cx, r) of each slot into its segment as (slot, distance)
// keys and x-sorted positions; fill[] counts per slot (zeroed by the caller).
template <int C>
__global__ void __launch_bounds__(HB)
k_halo_gather(const int32_t* __restrict__ slots, Store S, ColIdx ci, const int32_t* __restrict__ konta,
              const int64_t* __restrict__ off, const float* __restrict__ hcx, const float* __restrict__ hcy,
              const float* __restrict__ hcz, const float* __restrict__ rg, int32_t* __restrict__ fill,
              unsigned long long* __restrict__ keys, int32_t* __restrict__ vals) {
  __shared__ QBuf qb;
  __shared__ int s_fill;  // the group's fill counter lives in rank 0's shared memory
  Grp<C> G;
  int slot = group_slot<C>(slots);
  int kmax = konta[slot];
  if (kmax == 0) return;
  if (threadIdx.x == 0) s_fill = 0;
  G.sync();
  int* cnt = &s_fill;
  if constexpr (C > 1) cnt = cg::this_cluster().map_shared_rank(&s_fill, 0);
  float cx = hcx[slot], cy = hcy[slot], cz = hcz[slot], r = rg[slot];
  int64_t lo, hi;
  slab_range(ci, cx, r, &lo, &hi);
  int64_t base = off[slot];
  unsigned long long hk = (unsigned long long)slot << 32;
  gquery_box(G, ci, cx, cy, cz, r, qb, [&](const float4& e) {
    int p = ppos(e);
    float a = dist3(e.x, e.y, e.z, cx, cy, cz);
    bool hit = p >= lo && p < hi && a < r;
    // one counter update per warp
    cg::coalesced_group act = cg::coalesced_threads();
    unsigned hm = act.ballot(hit);
    if (hm == 0u) return;
    int lead = __ffs(hm) - 1;
    int q0 = 0;
    if ((int)act.thread_rank() == lead) q0 = atomicAdd(cnt, __popc(hm));
    q0 = act.shfl(q0, lead);
    if (hit) {
      int q = q0 + __popc(hm & ((1u << act.thread_rank()) - 1u));
      if (q < kmax) {
        keys[base + q] = hk | __float_as_uint(a);
        vals[base + q] = p;
      }
    }
  });
  G.sync();  // every CTA is done with rank 0's counter
  if (G.rank() == 0 && threadIdx.x == 0) fill[slot] = s_fill;  // members written (diagnostic)
}

// Runs of equal (halo, distance) get their positions in descending (desc=1)
// or ascending order.
__global__ void k_tiefix(const unsigned long long* __restrict__ keys, int32_t* __restrict__ vals,
                         int64_t n, int desc) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (i > 0 && keys[i] == keys[i - 1]) continue;
    if (i + 1 >= n || keys[i + 1] != keys[i]) continue;
    int64_t e = i + 1;
    while (e < n && keys[e] == keys[i]) e++;
    for (int64_t a = i + 1; a < e; a++) {
      int32_t v = vals[a];
      int64_t b = a - 1;
      while (b >= i && (desc ? vals[b] < v : vals[b] > v)) {
        vals[b + 1] = vals[b];
        b--;
      }
      vals[b + 1] = v;
    }
  }
}

// ---------------------------------------------------------------- main
struct MainShared {
  double dred[32];
  float fred[32];
  long long lred[32];
  double v[16];
  long long iv[16];
  float inertia[9];
  float eig[3];
  double bestv[HB];
  long long bestj[HB];
  double bestb[HB];
};

// Block-wide minimum of an index (LLONG_MAX when none).
__device__ __forceinline__ long long bmin(long long v, MainShared& sh) { return block_min_ll(v, sh.lred); }

struct HaloState {
  float cm[3], v[3], masa, radio;
  int realclus;
};

__device__ __forceinline__ void unbind_result(HaloState& h, long long konta3, const float* cm,
                                              const float* vcm, float mmm, float um) {
  if (konta3 == 0) {
    for (int q = 0; q < 3; q++) { h.cm[q] = 0.0f; h.v[q] = 0.0f; }
    h.masa = 0.0f;
    h.radio = 0.0f;
    h.realclus = 0;
  } else {
    for (int q = 0; q < 3; q++) { h.cm[q] = cm[q]; h.v[q] = vcm[q]; }
    h.masa = __fmul_rn(mmm, um);
  }
}

// DIAGONALISE (num.f:2-116), REAL*8 Jacobi; `in` is column-major REAL*4.
__device__ void diagonalise_dev(const float* in, float* eig) {
  const int n = 3;
  double a[3][3], e[3], aux1[3], aux2[3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) a[i][j] = (double)in[j * 3 + i];
  for (int i = 0; i < n; i++) { aux1[i] = a[i][i]; e[i] = aux1[i]; aux2[i] = 0.0; }
  double sum_el = 0.0;
  for (int i = 0; i < n; i++)
    for (int j = i; j < n; j++) sum_el = __dadd_rn(sum_el, fabs(a[i][j]));
  for (int it = 1; it <= 100; it++) {
    double suma = 0.0;
    for (int i = 0; i < n - 1; i++)
      for (int j = i + 1; j < n; j++) suma = __dadd_rn(suma, fabs(a[i][j]));
    if (suma < __dmul_rn((double)1.e-4f, sum_el)) break;
    double upper = (it < 4) ? __dmul_rn(0.2, __dmul_rn(suma, suma)) : 0.0;
    for (int p = 0; p < n - 1; p++) {
      for (int q = p + 1; q < n; q++) {
        double var1 = __dmul_rn(100.0, fabs(a[p][q]));
        if (it > 4 && __dadd_rn(fabs(e[p]), var1) == fabs(e[p]) && __dadd_rn(fabs(e[q]), var1) == fabs(e[q])) {
          a[p][q] = 0.0;
        } else if (fabs(a[p][q]) > upper) {
          double var2 = __dsub_rn(e[q], e[p]), t;
          if (__dadd_rn(fabs(var2), var1) == fabs(var2)) {
            t = __ddiv_rn(a[p][q], var2);
          } else {
            double th = __ddiv_rn(__dmul_rn(0.5, var2), a[p][q]);
            t = __ddiv_rn(1.0, __dadd_rn(fabs(th), __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(th, th)))));
            if (th < 0.0) t = -t;
          }
          double cth = __ddiv_rn(1.0, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(t, t))));
          double s = __dmul_rn(t, cth);
          double tau = __ddiv_rn(s, __dadd_rn(1.0, cth));
          var2 = __dmul_rn(t, a[p][q]);
          aux2[p] = __dsub_rn(aux2[p], var2);
          aux2[q] = __dadd_rn(aux2[q], var2);
          e[p] = __dsub_rn(e[p], var2);
          e[q] = __dadd_rn(e[q], var2);
          a[p][q] = 0.0;
          for (int j = 0; j < p; j++) {
            double v1 = a[j][p], v2 = a[j][q];
            a[j][p] = __dsub_rn(v1, __dmul_rn(s, __dadd_rn(v2, __dmul_rn(v1, tau))));
            a[j][q] = __dadd_rn(v2, __dmul_rn(s, __dsub_rn(v1, __dmul_rn(v2, tau))));
          }
          for (int j = p + 1; j < q; j++) {
            double v1 = a[p][j], v2 = a[j][q];
            a[p][j] = __dsub_rn(v1, __dmul_rn(s, __dadd_rn(v2, __dmul_rn(v1, tau))));
            a[j][q] = __dadd_rn(v2, __dmul_rn(s, __dsub_rn(v1, __dmul_rn(v2, tau))));
          }
          for (int j = q + 1; j < n; j++) {
            double v1 = a[p][j], v2 = a[q][j];
            a[p][j] = __dsub_rn(v1, __dmul_rn(s, __dadd_rn(v2, __dmul_rn(v1, tau))));
            a[q][j] = __dadd_rn(v2, __dmul_rn(s, __dsub_rn(v1, __dmul_rn(v2, tau))));
          }
        }
      }
    }
    for (int i = 0; i < n; i++) { aux1[i] = __dadd_rn(aux1[i], aux2[i]); e[i] = aux1[i]; aux2[i] = 0.0; }
  }
  for (int i = 0; i < n; i++) eig[i] = (float)e[i];
}

__device__ void sort_eigen_dev(float* e) {
  for (int ii = 0; ii < 2; ii++) {
    int kk = ii;
    float valor = e[ii];
    for (int jj = ii + 1; jj < 3; jj++)
      if (e[jj] >= valor) { kk = jj; valor = e[jj]; }
    if (kk != ii) { e[kk] = e[ii]; e[ii] = valor; }
  }
}

__device__ __forceinline__ float so_den(float d, float rete, float pi) {
  float dr = __fmul_rn(d, rete);
  return __fmul_rn(__fmul_rn(pi, 1.3333334f), __fmul_rn(__fmul_rn(dr, dr), dr));
}

// ================================================================ main (group)
// The member list of one halo is staged contiguously (distance, x-sorted
// position, mass and velocity, position) so the unbinding passes, the SO
// walk and the property loop stream through it.  REORDENAR's in-place
// compaction becomes a copy into the second buffer set: entries past the new
// length are copied from the old list, so both sets hold what the in-place
// compaction would leave there (DISTA(K2+1) is read by the next UNBINDING8).
struct SegBuf {
  float2* dm;  // (distance, mass): what the cumulative-mass scans read
  float4* mv;  // (m, vx, vy, vz)
  float4* px;  // (x, y, z, x-sorted position as int bits)
};

struct SegView {
  float2* dm;
  float4* mv;
  float4* px;
};

__device__ __forceinline__ SegView view_at(const SegBuf& b, int64_t base) {
  return SegView{b.dm + base, b.mv + base, b.px + base};
}

struct SegG {
  const int32_t* konta;
  const int64_t* off;       // element offset of the segment (segments padded by 1)
  const unsigned long long* keys;
  const int32_t* vals;
  SegBuf a, b;
  double* pot;
  uint8_t* flag;
  uint8_t* final_b;         // 1: the final member list is in set b
  int32_t* nbound;          // IDs to write per slot (KONTA2 of the property loop)
  int32_t* nscan;           // entries the property loop scanned (NCAPAS)
  unsigned long long* work; // element-pass counter; with timing, [4..7] halo times
  int32_t* status;
  float* eig;               // 9 per slot: inertia tensor for k_eigen (NaN: none)
  int timing;               // record per-halo durations (profiling)
};

__device__ __forceinline__ unsigned long long gtimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

struct GShared {  // per-warp slots: HW warps at most
  double dred[HW];
  float fred[HW];
  long long lred[HW];
  double wv[HW];
  long long wj[HW];
  double wb[HW];
  double bc_d[2];
  long long bc_l[2];
  double wsum[HW];  // per-warp totals of the scans
  double wsum3[3 * HW];
  long long wcnt[HW];
  GX x;
};

// Values the leader (rank 0, thread 0) stored in sh.bc_* , seen by the group.
template <int C>
__device__ __forceinline__ void gbcast(const Grp<C>& g, double* d, long long* l, GShared& sh) {
  if constexpr (C <= 1) {
    __syncthreads();
    *d = sh.bc_d[0];
    *l = sh.bc_l[0];
    __syncthreads();
  } else {
    g.sync();
    cg::cluster_group cl = cg::this_cluster();
    *d = *cl.map_shared_rank(&sh.bc_d[0], 0);
    *l = *cl.map_shared_rank(&sh.bc_l[0], 0);
    g.sync();
  }
}

// (v, j, b) with the largest v, the smallest j among equal v; j = LLONG_MAX
// marks an empty entry.
__device__ __forceinline__ bool best_before(double v1, long long j1, double v2, long long j2) {
  if (j1 == LLONG_MAX) return false;
  if (j2 == LLONG_MAX) return true;
  return v1 > v2 || (v1 == v2 && j1 < j2);
}

template <int C>
__device__ void gbest(const Grp<C>& g, double* v, long long* j, double* b, GShared& sh) {
  double bv = *v, bb = *b;
  long long bj = *j;
  for (int o = 16; o > 0; o >>= 1) {
    double ov = __shfl_down_sync(0xffffffffu, bv, o);
    long long oj = __shfl_down_sync(0xffffffffu, bj, o);
    double ob = __shfl_down_sync(0xffffffffu, bb, o);
    if (best_before(ov, oj, bv, bj)) { bv = ov; bj = oj; bb = ob; }
  }
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { sh.wv[wid] = bv; sh.wj[wid] = bj; sh.wb[wid] = bb; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++)
      if (best_before(sh.wv[w], sh.wj[w], sh.wv[0], sh.wj[0])) {
        sh.wv[0] = sh.wv[w]; sh.wj[0] = sh.wj[w]; sh.wb[0] = sh.wb[w];
      }
  }
  __syncthreads();
  bv = sh.wv[0]; bj = sh.wj[0]; bb = sh.wb[0];
  __syncthreads();
  if constexpr (C > 1) {
    if (threadIdx.x == 0) { sh.x.d[0] = bv; sh.x.d[1] = bb; sh.x.l[0] = bj; }
    g.sync();
    if (threadIdx.x == 0) {
      cg::cluster_group cl = cg::this_cluster();
#pragma unroll 1
      for (int r = 0; r < C; r++) {
        double ov = *cl.map_shared_rank(&sh.x.d[0], r);
        double ob = *cl.map_shared_rank(&sh.x.d[1], r);
        long long oj = *cl.map_shared_rank(&sh.x.l[0], r);
        if (best_before(ov, oj, bv, bj)) { bv = ov; bj = oj; bb = ob; }
      }
      sh.x.dres[0] = bv; sh.x.dres[1] = bb; sh.x.lres[0] = bj;
    }
    g.sync();
    bv = sh.x.dres[0]; bb = sh.x.dres[1]; bj = sh.x.lres[0];
  }
  *v = bv; *j = bj; *b = bb;
}

// Stages the sorted members of one halo into set a.
template <int C>
__device__ void load_segment(const Grp<C>& g, const Store& S, const unsigned long long* keys,
                             const int32_t* vals, int64_t K, const SegView& a, const SegView& b, uint8_t* flag) {
  int64_t lo, hi;
  g.chunk(0, K, &lo, &hi);
  const int bd = blockDim.x;
  // four entries per thread: keys, then the store's fields, then the writes
#pragma unroll 1
  for (int64_t jb = lo + threadIdx.x; jb < hi; jb += 4 * bd) {
    unsigned long long kk[4];
    int p[4];
    float f[4][7];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int64_t j = jb + u * bd;
      kk[u] = j < hi ? keys[j] : 0ull;
      p[u] = j < hi ? vals[j] : 0;
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (jb + u * bd < hi) {
        const int q = p[u];
        if (S.rows) {
          const float4 r0 = S.rows[2 * (int64_t)q], r1 = S.rows[2 * (int64_t)q + 1];
          f[u][0] = r0.w; f[u][1] = r1.x; f[u][2] = r1.y; f[u][3] = r1.z;
          f[u][4] = r0.x; f[u][5] = r0.y; f[u][6] = r0.z;
        } else {
          f[u][0] = S.m[q]; f[u][1] = S.vx[q]; f[u][2] = S.vy[q]; f[u][3] = S.vz[q];
          f[u][4] = S.x[q]; f[u][5] = S.y[q]; f[u][6] = S.z[q];
        }
      }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int64_t j = jb + u * bd;
      if (j < hi) {
        a.dm[j] = make_float2(__uint_as_float((uint32_t)(kk[u] & 0xffffffffull)), f[u][0]);
        a.mv[j] = make_float4(f[u][0], f[u][1], f[u][2], f[u][3]);
        a.px[j] = make_float4(f[u][4], f[u][5], f[u][6], __int_as_float(p[u]));
        flag[j] = 1;
      }
    }
  }
  if (g.rank() == 0 && threadIdx.x == 0) {  // DISTA(K+1) of the sorted list
    a.dm[K] = make_float2(1.e10f, 0.f); b.dm[K] = a.dm[K];
    a.mv[K] = make_float4(0.f, 0.f, 0.f, 0.f); b.mv[K] = a.mv[K];
    a.px[K] = make_float4(0.f, 0.f, 0.f, 0.f); b.px[K] = a.px[K];
  }
  g.sync();
}

// CENTROMASAS_PART (haloes_particles.f:1731-1824) over the first n entries.
template <int C>
__device__ void centromasas_g(const Grp<C>& g, const SegView& v, int64_t n, float* cm, float* vcm, float* masa,
                              GShared& sh) {
  double a[7] = {0, 0, 0, 0, 0, 0, 0};
  int64_t lo, hi;
  g.chunk(0, n, &lo, &hi);
#pragma unroll 4
  for (int64_t j = lo + threadIdx.x; j < hi; j += blockDim.x) {
    float4 q = v.mv[j], p = v.px[j];
    double bas = (double)q.x;
    a[0] += (double)p.x * bas;
    a[1] += (double)p.y * bas;
    a[2] += (double)p.z * bas;
    a[3] += (double)q.y * bas;
    a[4] += (double)q.z * bas;
    a[5] += (double)q.w * bas;
    a[6] += bas;
  }
  gsum_dv<7>(g, a, sh.x);
  if (a[6] > 0.0) {
    for (int q = 0; q < 3; q++) { cm[q] = (float)(a[q] / a[6]); vcm[q] = (float)(a[3 + q] / a[6]); }
    *masa = (float)a[6];
  } else {
    for (int q = 0; q < 3; q++) { cm[q] = 0.0f; vcm[q] = 0.0f; }
    *masa = 0.0f;
  }
}

// One warp's stable compaction of [j0, j1) into dst from position d0: steps
// of 32 entries in pairs, both steps read before either is written.
// Returns the next free position; *reloc gets the lowest 1-based
// destination of a kept entry at or after 1-based position iv.
__device__ __forceinline__ int64_t compact_run(const SegView& src, const SegView& dst, const uint8_t* flag,
                                               int64_t j0, int64_t j1, int64_t iv, int64_t d0, long long* reloc) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
#pragma unroll 1
  for (int64_t jb = j0; jb < j1; jb += 64) {
    bool keep[2];
    float2 e0[2];
    float4 e1[2], e2[2];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int64_t j = jb + 32 * u + lane;
      keep[u] = j < j1 && flag[j];
      if (j < j1) {
        e0[u] = src.dm[j];
        e1[u] = src.mv[j];
        e2[u] = src.px[j];
      }
    }
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int64_t j = jb + 32 * u + lane;
      const unsigned m = __ballot_sync(0xffffffffu, keep[u]);
      if (keep[u]) {
        const int64_t d = d0 + __popc(m & below);
        dst.dm[d] = e0[u];
        dst.mv[d] = e1[u];
        dst.px[d] = e2[u];
        if (j + 1 >= iv && d + 1 < *reloc) *reloc = d + 1;
      }
      d0 += __popc(m);
    }
  }
  return d0;
}

// dst[j] = src[j] for j = j0, j0 + step, ... < j1, two entries read at a time.
__device__ __forceinline__ void copy_run(const SegView& src, const SegView& dst, int64_t j0, int64_t j1, int step) {
#pragma unroll 1
  for (int64_t jb = j0; jb < j1; jb += 2 * (int64_t)step) {
    float2 e0[2];
    float4 e1[2], e2[2];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int64_t j = jb + (int64_t)u * step;
      if (j < j1) {
        e0[u] = src.dm[j];
        e1[u] = src.mv[j];
        e2[u] = src.px[j];
      }
    }
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int64_t j = jb + (int64_t)u * step;
      if (j < j1) {
        dst.dm[j] = e0[u];
        dst.mv[j] = e1[u];
        dst.px[j] = e2[u];
      }
    }
  }
}

// REORDENAR(...,0,...) (haloes_particles.f:1696-1722): the kept entries of
// j < k2 in order into dst, IDX_VIR relocated to the first kept entry at or
// after it; dst[k2new, k2) = src[k2new, k2).
template <int C>
__device__ void compact_g(const Grp<C>& g, const SegView& src, const SegView& dst, const uint8_t* flag,
                          int64_t k2, int64_t* idx_vir, int64_t* k2new, GShared& sh) {
  if constexpr (C <= 1) {
    if (C == 0 || blockDim.x == 32) {  // one warp: offsets from the ballots as it goes
      const int lane = threadIdx.x;
      const int64_t iv = *idx_vir;  // 1-based
      long long reloc = LLONG_MAX;
      const int64_t d0 = compact_run(src, dst, flag, 0, k2, iv, 0, &reloc);
      copy_run(src, dst, d0 + lane, k2, 32);
      for (int o = 16; o > 0; o >>= 1) {
        long long y = __shfl_xor_sync(0xffffffffu, reloc, o);
        reloc = y < reloc ? y : reloc;
      }
      *k2new = d0;
      *idx_vir = reloc == LLONG_MAX ? d0 : reloc;
      __syncthreads();
      return;
    }
  }
  int64_t lo, hi, wlo, whi;
  g.chunk(0, k2, &lo, &hi);
  warp_run(lo, hi, &wlo, &whi);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  long long cnt = 0;
#pragma unroll 4
  for (int64_t j = wlo + lane; j < whi; j += 32) cnt += flag[j];
  cnt = warp_allsum_ll(cnt);
  if (lane == 0) sh.wcnt[w] = cnt;
  __syncthreads();
  const long long woff = warp_allsum_ll(lane < w ? sh.wcnt[lane] : 0);
  const long long ctot = warp_allsum_ll(lane < nw ? sh.wcnt[lane] : 0);
  long long off = 0, tot = ctot;
  if constexpr (C > 1) gexcl_ll(g, ctot, &off, &tot, sh.x);
  int64_t d0 = off + woff;
  long long reloc = LLONG_MAX;
  const int64_t iv = *idx_vir;  // 1-based
  compact_run(src, dst, flag, wlo, whi, iv, d0, &reloc);
  const int64_t nn = tot;
  g.chunk(nn, k2, &lo, &hi);
  copy_run(src, dst, lo + threadIdx.x, hi, blockDim.x);
  gmin_llv<1>(g, &reloc, sh.lred, sh.x);
  *k2new = nn;
  *idx_vir = reloc == LLONG_MAX ? nn : reloc;
  g.sync();
}

// What an UNBINDING8 call leaves for the next call on the same list.  The
// potential depends only on the list, its length and the outer radius, so a
// call on the list the previous call left unchanged (nothing removed) reads
// it back instead of scanning again.  When that previous call kept every
// entry, and the velocity centre it returned is the one it was given, a later
// call differs from it only in the factor BB: the previous call also counted
// the entries the smaller factors (16, 4) would remove, and a call whose
// factor removes none is known to return the same state, so it is skipped.
struct PotCache {
  bool valid = false;
  int64_t k2 = 0;
  float ref_max = 0.0f;
  double pot_jj = 0.0, pot1 = 0.0;  // pot[] holds the scan's Q
  bool flags_valid = false;         // the last flag pass kept every entry
  float hv[3] = {0.0f, 0.0f, 0.0f}; // the velocity centre that pass used
  double rm16 = 0.0, rm4 = 0.0;     // entries BB = 16 and BB = 4 would remove
};

// The same for UNBINDING_SIGMA: sigma depends on the list, IDX_VIR and the
// velocity centre; a call with all three unchanged reuses it, and, when the
// pass that computed it kept every entry, skips the flag pass too if its
// factor (25, 16 or 9) removes none.
struct SigCache {
  bool valid = false;
  int64_t k2 = 0, iv = 0;
  float v[3] = {0.0f, 0.0f, 0.0f};
  double sigma2 = 0.0;
  bool flags_valid = false;
  double rm[3] = {0.0, 0.0, 0.0};  // entries BB = 25, 16, 9 would remove
};

// UNBINDING8 (haloes_particles.f:1828-1983) on the staged list.
template <int C>
__device__ long long unbinding8_g(const Grp<C>& g, float normaf, const HConst& H, int fac, float ref_max,
                             const SegView& v, uint8_t* flag, double* pot, int64_t k2, int64_t idx_vir,
                             HaloState& h, GShared& sh, PotCache& pc) {
  float cm[3] = {0, 0, 0}, vcm[3] = {0, 0, 0}, mmm = 0.0f;
  long long konta3 = 0;
  if (k2 > 0) {
    double norma = (double)normaf;
    double pot_jj, pot1;
    if (pc.valid && pc.k2 == k2 && pc.ref_max == ref_max) {
      if (pc.flags_valid && fac >= 2 && h.v[0] == pc.hv[0] && h.v[1] == pc.hv[1] && h.v[2] == pc.hv[2] &&
          (fac == 2 ? pc.rm16 : pc.rm4) == 0.0)
        return k2;  // every entry kept again: the state stays as it is
      pot_jj = pc.pot_jj;
      pot1 = pc.pot1;
    } else {
      float lim = __fmul_rn(0.01f, ref_max);
      // first J with DISTA(J) > lim (the list is sorted by distance); K2+1 if none
      int64_t a = 0, b = k2;
      if (k2 > 4096) {  // narrow the range with one parallel probe per thread of the CTA
        const int64_t step = (k2 + blockDim.x - 1) / blockDim.x;
        const int64_t jp = (int64_t)threadIdx.x * step;
        bool above = jp < k2 && v.dm[jp].x > lim;
        __syncthreads();
        unsigned m = __ballot_sync(0xffffffffu, above);
        if ((threadIdx.x & 31) == 0) sh.wcnt[threadIdx.x >> 5] = m ? (long long)((threadIdx.x & ~31) + __ffs(m) - 1) : LLONG_MAX;
        __syncthreads();
        long long fp = LLONG_MAX;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) fp = sh.wcnt[w] < fp ? sh.wcnt[w] : fp;
        __syncthreads();
        // probes are sorted: the answer lies in (probe fp-1, probe fp]
        if (fp == LLONG_MAX) {  // after the last probe inside the list
          int64_t lastp = (k2 - 1) / step;
          if (lastp > (int64_t)blockDim.x - 1) lastp = (int64_t)blockDim.x - 1;
          a = lastp * step + 1;
        } else {
          b = fp * step;
          a = fp > 0 ? (fp - 1) * step + 1 : 0;
        }
      }
      while (a < b) {
        int64_t mid = (a + b) >> 1;
        if (v.dm[mid].x > lim) b = mid; else a = mid + 1;
      }
      int64_t jj = a + 1;
      // MASA8 and the POT recurrence of haloes_particles.f:1870-1893 in one
      // scan: POT(J) = POT(JJ) + Q(J), Q(J) = sum over JJ < I <= J of
      // MASA8(I) * BAS8(I) / DISTA(I)^2; pot[] receives Q
      double mk2, qk2, mjj_part = 0.0;
      gscan_aff(
          g, 0, k2, [&](int64_t j) { return (double)v.dm[j].y / norma; },
          [&](int64_t j) {
            if (j < jj) return 0.0;
            float dj = v.dm[j].x, dm1 = v.dm[j - 1].x;
            double bas8 = (dj != dm1) ? (double)__fsub_rn(dj, dm1) : 0.0;
            double djd = (double)dj;
            return bas8 / (djd * djd);
          },
          [&](int64_t j, double M, double Q) {
            pot[j] = Q;
            if (j == jj - 1) mjj_part = M;
          },
          sh.wsum3, sh.x, &mk2, &qk2);
      double mjj = mk2;
      if (jj <= k2) {
        gsum_dv<1>(g, &mjj_part, sh.x);
        mjj = mjj_part;
      }
      pot_jj = mjj / (double)v.dm[jj - 1].x;
      pot1 = (pot_jj + qk2) + mk2 / (double)ref_max;
      pc.valid = true;
      pc.k2 = k2;
      pc.ref_max = ref_max;
      pc.pot_jj = pot_jj;
      pc.pot1 = pot1;
    }
    int64_t lo, hi;
    double aa8 = norma * (double)__fdiv_rn(H.cgr, H.rete);
    float bb = 2.0f;
    if (fac == 1) bb = 8.0f;
    if (fac == 2) bb = 4.0f;
    bb = __fmul_rn(bb, bb);
    double s[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // 7 sums, the kept count, removals at BB = 16, 4
    g.chunk(0, k2, &lo, &hi);
    const int bd = blockDim.x;
    // pairs of entries per thread, both read before either flag is stored
#pragma unroll 1
    for (int64_t jb = lo + threadIdx.x; jb < hi; jb += 2 * bd) {
      double pt[2];
      float4 qv[2], pv[2];
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int64_t j = jb + u * bd;
        if (j < hi) {
          pt[u] = pot[j];
          qv[u] = v.mv[j];
          if (j < idx_vir) pv[u] = v.px[j];
        }
      }
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int64_t j = jb + u * bd;
        if (j >= hi) break;
        float potok = (float)(((pot_jj + pt[u]) - pot1) * aa8);
        float vesc2 = __fmul_rn(2.0f, fabsf(potok));
        const float4 q = qv[u];
        float ax = __fsub_rn(q.y, h.v[0]), ay = __fsub_rn(q.z, h.v[1]), az = __fsub_rn(q.w, h.v[2]);
        float vvv2 = __fadd_rn(__fadd_rn(__fmul_rn(ax, ax), __fmul_rn(ay, ay)), __fmul_rn(az, az));
        bool keep = !(vvv2 > __fmul_rn(bb, vesc2));
        flag[j] = keep;
        s[7] += keep ? 1.0 : 0.0;
        s[8] += vvv2 > __fmul_rn(16.0f, vesc2) ? 1.0 : 0.0;
        s[9] += vvv2 > __fmul_rn(4.0f, vesc2) ? 1.0 : 0.0;
        if (keep && j < idx_vir) {
          const float4 p = pv[u];
          double bas = (double)q.x;
          s[0] += (double)p.x * bas;
          s[1] += (double)p.y * bas;
          s[2] += (double)p.z * bas;
          s[3] += (double)q.y * bas;
          s[4] += (double)q.z * bas;
          s[5] += (double)q.w * bas;
          s[6] += bas;
        }
      }
    }
    gsum_dv<10>(g, s, sh.x);
    konta3 = (long long)s[7];
    pc.flags_valid = konta3 == k2;
    for (int q = 0; q < 3; q++) pc.hv[q] = h.v[q];
    pc.rm16 = s[8];
    pc.rm4 = s[9];
    if (s[6] > 0.0) {
      for (int q = 0; q < 3; q++) { cm[q] = (float)(s[q] / s[6]); vcm[q] = (float)(s[3 + q] / s[6]); }
      mmm = (float)s[6];
    }
  }
  unbind_result(h, konta3, cm, vcm, mmm, H.um);
  return konta3;
}

// UNBINDING_SIGMA (haloes_particles.f:1987-2095) on the staged list.
template <int C>
__device__ long long unbinding_sigma_g(const Grp<C>& g, const HConst& H, int fac, const SegView& v, uint8_t* flag,
                                  int64_t k2, int64_t idx_vir, HaloState& h, GShared& sh, SigCache& sc) {
  float bb = fmaxf(__fsub_rn(6.0f, __fmul_rn(1.0f, (float)(fac - 1))), 3.0f);
  bb = __fmul_rn(bb, bb);
  float cm[3] = {h.cm[0], h.cm[1], h.cm[2]}, vcm[3] = {h.v[0], h.v[1], h.v[2]}, mmm = 0.0f;
  long long konta3 = 0;
  if (k2 > 0) {
    int64_t lo, hi;
    double sigma2;
    if (sc.valid && sc.k2 == k2 && sc.iv == idx_vir && vcm[0] == sc.v[0] && vcm[1] == sc.v[1] &&
        vcm[2] == sc.v[2]) {
      if (sc.flags_valid && fac >= 2 && sc.rm[fac == 2 ? 0 : (fac == 3 ? 1 : 2)] == 0.0)
        return k2;  // every entry kept again: the state stays as it is
      sigma2 = sc.sigma2;
    } else {
      g.chunk(0, idx_vir < k2 ? idx_vir : k2, &lo, &hi);
      double s2 = 0.0;
#pragma unroll 4
      for (int64_t j = lo + threadIdx.x; j < hi; j += blockDim.x) {
        float4 q = v.mv[j];
        float ax = __fsub_rn(q.y, vcm[0]), ay = __fsub_rn(q.z, vcm[1]), az = __fsub_rn(q.w, vcm[2]);
        s2 += (double)__fadd_rn(__fadd_rn(__fmul_rn(ax, ax), __fmul_rn(ay, ay)), __fmul_rn(az, az));
      }
      sigma2 = gsum_d(g, s2, sh.dred, sh.x);
      if (idx_vir > 1) sigma2 = sigma2 / (double)(idx_vir - 1);
      sc.valid = true;
      sc.k2 = k2;
      sc.iv = idx_vir;
      for (int q = 0; q < 3; q++) sc.v[q] = vcm[q];
      sc.sigma2 = sigma2;
      sc.flags_valid = false;
    }
    double thr = (double)bb * sigma2;
    const double thr25 = (double)25.0f * sigma2, thr16 = (double)16.0f * sigma2, thr9 = (double)9.0f * sigma2;
    double s[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // 7 sums, the kept count, removals at BB = 25, 16, 9
    g.chunk(0, k2, &lo, &hi);
    const int bd = blockDim.x;
#pragma unroll 1
    for (int64_t jb = lo + threadIdx.x; jb < hi; jb += 2 * bd) {
      float4 qv[2], pv[2];
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int64_t j = jb + u * bd;
        if (j < hi) {
          qv[u] = v.mv[j];
          if (j < idx_vir) pv[u] = v.px[j];
        }
      }
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int64_t j = jb + u * bd;
        if (j >= hi) break;
        const float4 q = qv[u];
        float ax = __fsub_rn(q.y, vcm[0]), ay = __fsub_rn(q.z, vcm[1]), az = __fsub_rn(q.w, vcm[2]);
        float bas = __fadd_rn(__fadd_rn(__fmul_rn(ax, ax), __fmul_rn(ay, ay)), __fmul_rn(az, az));
        bool keep = !((double)bas > thr);
        flag[j] = keep;
        s[7] += keep ? 1.0 : 0.0;
        s[8] += (double)bas > thr25 ? 1.0 : 0.0;
        s[9] += (double)bas > thr16 ? 1.0 : 0.0;
        s[10] += (double)bas > thr9 ? 1.0 : 0.0;
        if (keep && j < idx_vir) {
          const float4 p = pv[u];
          double w = (double)q.x;
          s[0] += (double)p.x * w;
          s[1] += (double)p.y * w;
          s[2] += (double)p.z * w;
          s[3] += (double)q.y * w;
          s[4] += (double)q.z * w;
          s[5] += (double)q.w * w;
          s[6] += w;
        }
      }
    }
    gsum_dv<11>(g, s, sh.x);
    konta3 = (long long)s[7];
    sc.flags_valid = konta3 == k2;
    for (int q = 0; q < 3; q++) sc.rm[q] = s[8 + q];
    if (s[6] > 0.0) {
      for (int q = 0; q < 3; q++) { cm[q] = (float)(s[q] / s[6]); vcm[q] = (float)(s[3 + q] / s[6]); }
      mmm = (float)s[6];
    } else {
      for (int q = 0; q < 3; q++) { cm[q] = 0.0f; vcm[q] = 0.0f; }
      mmm = 0.0f;
    }
  }
  unbind_result(h, konta3, cm, vcm, mmm, H.um);
  return konta3;
}

// Bound-particle properties (haloes_particles.f:1187-1353) over j < konta of
// the staged list; flag[j] receives the ID mask.  Returns KONTA2.
// COMPUTE_EPOT (haloes_particles.f:1494-1628), direct summation over the
// konta entries whose flag is set: every pair's REAL*4 -m1*m2/r in float64.
// A thread sums the row of each of its entries against all entries (tiles
// of the list in shared memory; both members of a pair compute the same
// term, so the total is half the rows' sum), and the most bound entry is
// the first minimum of row / m (100000 for entries not in).  Returns the
// total through *epot8 and the entry through *jbest.
template <int C>
__device__ void epot_direct_g(const Grp<C>& g, const SegView& v, const uint8_t* flag, int64_t konta,
                              double* epot8, long long* jbest, GShared& sh) {
  __shared__ float4 tile[HB];
  int64_t lo, hi;
  g.chunk(0, konta, &lo, &hi);
  double rows = 0.0, best_v = -INFINITY, best_b = 0.0;  // best_v: -(row / m), the largest wins
  long long best_j = LLONG_MAX;
#pragma unroll 1
  for (int64_t j0 = lo; j0 < hi; j0 += blockDim.x) {  // the same trip count in every thread of the CTA
    const int64_t j = j0 + threadIdx.x;
    const bool act = j < hi && flag[j];
    float4 pj = make_float4(0.f, 0.f, 0.f, 0.f);
    if (act) {
      const float4 p = v.px[j];
      pj = make_float4(p.x, p.y, p.z, v.mv[j].x);
    }
    double e = 0.0;
#pragma unroll 1
    for (int64_t q0 = 0; q0 < konta; q0 += HB) {
      __syncthreads();
      for (int t = threadIdx.x; t < HB; t += blockDim.x) {
        const int64_t q = q0 + t;
        float4 w = make_float4(0.f, 0.f, 0.f, -1.f);  // m < 0: not in
        if (q < konta && flag[q]) {
          const float4 p = v.px[q];
          w = make_float4(p.x, p.y, p.z, v.mv[q].x);
        }
        tile[t] = w;
      }
      __syncthreads();
      if (act) {
        const int nt = konta - q0 < HB ? (int)(konta - q0) : HB;
        for (int t = 0; t < nt; t++) {
          const float4 w = tile[t];
          if (w.w < 0.f || q0 + t == j) continue;
          const float ax = __fsub_rn(pj.x, w.x), ay = __fsub_rn(pj.y, w.y), az = __fsub_rn(pj.z, w.z);
          const float r = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ax, ax), __fmul_rn(ay, ay)), __fmul_rn(az, az)));
          e += (double)__fdiv_rn(-__fmul_rn(pj.w, w.w), r);
        }
      }
    }
    if (j < hi) {
      const double ev = act ? e / (double)pj.w : 100000.0;
      if (act) rows += e;
      if (best_before(-ev, j, best_v, best_j)) { best_v = -ev; best_j = j; }
    }
  }
  double t = rows;
  gsum_dv<1>(g, &t, sh.x);
  gbest(g, &best_v, &best_j, &best_b, sh);
  *epot8 = 0.5 * t;
  *jbest = best_j;
}

// COMPUTE_EPOT's sampling branch (haloes_particles.f:1568-1626), for bound
// lists of MAX_PART_DSUM entries or more.  NSAMPLE = MAX(INT(MAX_PART_DSUM
// /1.4), INT(0.01*KONTA2)) draws of a bound entry J, each paired with
// NSAMPLE draws of a bound entry K != J, all uniform over the KONTA scanned
// entries with rejection of the unbound ones (J = 1 + FLOOR(U*KONTA)).
// Per draw J the REAL*8 sum BAS of the REAL*4 terms -m_J m_K / r_JK; EPOT8
// is the sum of the BAS in draw order scaled by FLOAT(KONTA(KONTA-1)/2) /
// FLOAT(NSAMPLE^2); the most bound entry is the J whose BAS/m_J first beats
// the running minimum, that minimum being kept in REAL*4 as the reference
// keeps LARGEST_ENERGY.
//
// The reference's U comes from RANDOM_NUMBER after an unseeded RANDOM_SEED
// (irreproducible).  Here U is counter-based: bits = mix(key_outer, inner +
// 0x9E3779B9 * attempt) with key_outer = mix(key_row, outer), key_row =
// mix(seed, row), mix(a, b) = fmix32(a ^ fmix32(b)) and fmix32 the
// MurmurHash3 32-bit finaliser, and U = (bits >> 8) * 2^-24 (24 bits, exact
// in REAL*4).  outer is the 1-based draw of J, inner 0 for J itself and
// 1..NSAMPLE for its partners, attempt counts the rejections.  Every draw J
// is summed by one thread in the reference's order and the final sum and
// minimum are taken by one thread in draw order, so the result equals the
// oracle's sequential loop bit for bit.  The BAS, BAS/m and J of each draw
// are kept in the halo's potential array and in its spare member-list set
// (free once the member list is final).  A draw that finds no bound entry
// after EPOT_MAX_ATTEMPTS tries makes the call return 1 (the caller reports
// ASOHF_ERR_TIMEOUT); the reference would loop on.
#define EPOT_MAX_ATTEMPTS 4096u

__device__ __forceinline__ uint32_t fmix32(uint32_t h) {
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

__device__ __forceinline__ uint32_t mix2(uint32_t a, uint32_t b) { return fmix32(a ^ fmix32(b)); }

// 0-based entry J-1 of one draw (clamped to the list: U*KONTA can round up
// to KONTA in REAL*4)
__device__ __forceinline__ int64_t epot_draw(uint32_t key_outer, uint32_t inner, uint32_t attempt, int64_t konta) {
  const uint32_t bits = mix2(key_outer, inner + 0x9E3779B9u * attempt);
  const float u = __fmul_rn((float)(bits >> 8), 5.9604644775390625e-8f);
  const int64_t j = (int64_t)floorf(__fmul_rn(u, (float)konta));
  return j < konta ? j : konta - 1;
}

template <int C>
__device__ int epot_sample_g(const Grp<C>& g, const SegView& v, const SegView& spare, double* pot,
                             const uint8_t* flag, int64_t konta, long long konta2, int max_part_dsum,
                             uint32_t key_row, double* epot8, long long* jbest, GShared& sh) {
  const int64_t ns_a = (int64_t)__fdiv_rn((float)max_part_dsum, 1.4f);
  const int64_t ns_b = (int64_t)__fmul_rn(0.01f, (float)konta2);
  const int64_t nsample = ns_a > ns_b ? ns_a : ns_b;
  double* bas_m = reinterpret_cast<double*>(spare.dm);   // 8 B per entry
  int32_t* jsel = reinterpret_cast<int32_t*>(spare.mv);   // 16 B per entry
  const int64_t tid = (int64_t)g.rank() * blockDim.x + threadIdx.x;
  const int64_t nth = (int64_t)(C > 1 ? C : 1) * blockDim.x;
  int bad = 0;
#pragma unroll 1
  for (int64_t o = tid; o < nsample && !bad; o += nth) {
    const uint32_t ko = mix2(key_row, (uint32_t)(o + 1));
    int64_t j = -1;
    for (uint32_t a = 0; a < EPOT_MAX_ATTEMPTS; a++) {
      const int64_t c = epot_draw(ko, 0u, a, konta);
      if (flag[c]) { j = c; break; }
    }
    if (j < 0) { bad = 1; break; }
    const float4 pj = v.px[j];
    const float m1 = v.mv[j].x;
    double bas = 0.0;
#pragma unroll 1
    for (int64_t q = 1; q <= nsample; q++) {
      int64_t kq = -1;
      for (uint32_t a = 0; a < EPOT_MAX_ATTEMPTS; a++) {
        const int64_t c = epot_draw(ko, (uint32_t)q, a, konta);
        if (flag[c] && c != j) { kq = c; break; }
      }
      if (kq < 0) { bad = 1; break; }
      const float4 pk = v.px[kq];
      const float m2 = v.mv[kq].x;
      const float ax = __fsub_rn(pj.x, pk.x), ay = __fsub_rn(pj.y, pk.y), az = __fsub_rn(pj.z, pk.z);
      const float r = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ax, ax), __fmul_rn(ay, ay)), __fmul_rn(az, az)));
      bas = bas - (double)__fdiv_rn(__fmul_rn(m1, m2), r);
    }
    pot[o] = bas;
    bas_m[o] = bas / (double)m1;
    jsel[o] = (int32_t)j;
  }
  double anybad = (double)bad;
  gsum_dv<1>(g, &anybad, sh.x);
  __threadfence();
  g.sync();
  if (anybad != 0.0) return 1;
  if (g.rank() == 0 && threadIdx.x == 0) {
    double e = 0.0;
    float lmin = 1000000.0f;
    long long best = 0;
    for (int64_t o = 0; o < nsample; o++) {
      e = e + pot[o];
      const double b = bas_m[o];
      if (b < (double)lmin) { lmin = (float)b; best = jsel[o]; }
    }
    const long long npt = (long long)konta * (long long)(konta - 1) / 2;
    const long long npr = (long long)nsample * (long long)nsample;
    *epot8 = e * (double)__fdiv_rn((float)npt, (float)npr);
    *jbest = best;
  }
  return 0;
}

template <int C, bool SYM = true>
__device__ long long properties_g(const Grp<C>& g, const Store& S, const HConst& H, asohf_catalogue& cat, int i0,
                                  const SegView& v, uint8_t* flag, int64_t konta, float rshell, float cx, float cy,
                                  float cz, const float* cmv, GShared& sh, int* unsupported, const SegView& spare,
                                  double* pot, float* eig_in) {
  float norma = S.norma;
  float vc[3] = {cat.vx[i0], cat.vy[i0], cat.vz[i0]};
  int64_t each_prof = konta / ASOHF_NBINS;
  if (each_prof == 0) each_prof = 1;
  double acc[18];
  for (int q = 0; q < 18; q++) acc[q] = 0.0;
  float vmax = -1.0f;
  gscan_d(g, 0, konta, 0.0,
            [&](int64_t j) {
              float4 p = v.px[j];
              bool in = dist3(p.x, p.y, p.z, cx, cy, cz) <= rshell;
              return in ? (double)__fdiv_rn(v.mv[j].x, norma) : 0.0;
            },
            [&](int64_t j, double basmas) {
              int64_t J = j + 1;
              float4 p = v.px[j], q = v.mv[j];
              const bool in = dist3(p.x, p.y, p.z, cx, cy, cz) <= rshell;
              flag[j] = in;
              if (!in) return;
              float bv[3] = {__fsub_rn(p.x, cx), __fsub_rn(p.y, cy), __fsub_rn(p.z, cz)};
              float aadm = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(bv[0], bv[0]), __fmul_rn(bv[1], bv[1])),
                                                __fmul_rn(bv[2], bv[2])));
              acc[16] += 1.0;
              if (J % each_prof == 0 && J / each_prof <= ASOHF_NBINS) {
                int64_t b = J / each_prof;
                cat.profiles[(size_t)i0 * 2 * ASOHF_NBINS + (b - 1)] = aadm;
                cat.profiles[(size_t)i0 * 2 * ASOHF_NBINS + ASOHF_NBINS + (b - 1)] =
                    (float)(basmas * (double)norma * (double)H.um);
              }
              float bc[3] = {__fsub_rn(p.x, cmv[0]), __fsub_rn(p.y, cmv[1]), __fsub_rn(p.z, cmv[2])};
              float bvc[3] = {__fsub_rn(q.y, vc[0]), __fsub_rn(q.z, vc[1]), __fsub_rn(q.w, vc[2])};
              float vvv2 = __fadd_rn(__fadd_rn(__fmul_rn(bvc[0], bvc[0]), __fmul_rn(bvc[1], bvc[1])),
                                     __fmul_rn(bvc[2], bvc[2]));
              float mp = q.x;
              acc[0] += (double)vvv2;
              acc[1] += (double)__fmul_rn(mp, vvv2);
              acc[2] += (double)__fmul_rn(mp, __fsub_rn(__fmul_rn(bc[1], bvc[2]), __fmul_rn(bc[2], bvc[1])));
              acc[3] += (double)__fmul_rn(mp, __fsub_rn(__fmul_rn(bc[2], bvc[0]), __fmul_rn(bc[0], bvc[2])));
              acc[4] += (double)__fmul_rn(mp, __fsub_rn(__fmul_rn(bc[0], bvc[1]), __fmul_rn(bc[1], bvc[0])));
              for (int jy = 0; jy < 3; jy++)
                for (int ix = 0; ix < 3; ix++)
                  acc[5 + jy * 3 + ix] += (double)__fmul_rn(__fmul_rn(mp, bc[ix]), bc[jy]);
              vmax = fmaxf(vmax, vvv2);
              if (aadm != 0.0f) {
                float aa = __fadd_rn(__fadd_rn(__fmul_rn(__fdiv_rn(bv[0], aadm), bvc[0]),
                                               __fmul_rn(__fdiv_rn(bv[1], aadm), bvc[1])),
                                     __fmul_rn(__fdiv_rn(bv[2], aadm), bvc[2]));
                acc[14] += (double)__fmul_rn(aa, mp);
              }
              acc[15] += (double)__fdiv_rn(mp, norma);
            },
            sh.wsum, sh.x);
  // SYM (haloes_particles.f:1322-1324): the lower triangle of the inertia
  // tensor is copied from the upper one, so only six sums are reduced; the
  // subhalo loop (substructure.f:1620-1626) keeps all nine
  double r[16] = {acc[0], acc[2], acc[3], acc[4], acc[5], acc[6], acc[7], acc[9], acc[10], acc[13],
                  acc[14], acc[15], acc[16], acc[8], acc[11], acc[12]};
  if constexpr (SYM) gsum_dv<13>(g, r, sh.x);
  else gsum_dv<16>(g, r, sh.x);
  const double* r2 = r + 10;
  vmax = gmax_f(g, vmax, sh.fred, sh.x);
  long long cnt = (long long)r2[2];
  // energies (haloes_particles.f:1297-1316): kinetic sum of the bound
  // entries, potential by direct summation below MAX_PART_DSUM entries and
  // by the seeded sampling estimator from there on
  double ekin = acc[1], epot8 = 0.0;
  long long jmb = 0;
  *unsupported = 0;
  if (H.energies && cnt >= H.min_num_part) {
    gsum_dv<1>(g, &ekin, sh.x);
    if (cnt >= H.max_part_dsum) {
      const uint32_t key_row = mix2(H.epot_seed, (uint32_t)i0);
      if (epot_sample_g(g, v, spare, pot, flag, konta, cnt, H.max_part_dsum, key_row, &epot8, &jmb, sh))
        *unsupported = 2;
    } else {
      epot_direct_g(g, v, flag, konta, &epot8, &jmb, sh);
    }
  }
  if (g.rank() == 0 && threadIdx.x == 0) {
    cat.dmpclus[i0] = (int32_t)cnt;
    if (cnt < H.min_num_part) {
      cat.realclus[i0] = 0;
      cat.vmaxclus[i0] = vmax;  // the running maximum of |v|^2 (-1 if none) stays
    } else if (H.energies) {
      const double gcons = (double)4.301e-9f;
      float epot = (float)epot8;
      epot = (float)((double)epot * (double)__fmul_rn(H.um, H.um) * gcons);
      cat.kinetic_e[i0] = (float)(0.5 * ekin * (double)H.um * (double)__fmul_rn(H.uv, H.uv));
      cat.potential_e[i0] = __fmul_rn(epot, __fadd_rn(1.0f, H.zeta));
      cat.iplip[i0] = S.id[__float_as_int(v.px[jmb].w)];
    } else {
      cat.potential_e[i0] = 0.0f;
      cat.iplip[i0] = S.id[__float_as_int(v.px[0].w)];
    }
    if (cnt >= H.min_num_part) {
      double basmas = r2[1];
      double den = basmas * (double)norma;
      cat.angularm[i0 * 3 + 0] = (float)(r[1] * (double)H.uv / den);
      cat.angularm[i0 * 3 + 1] = (float)(r[2] * (double)H.uv / den);
      cat.angularm[i0 * 3 + 2] = (float)(r[3] * (double)H.uv / den);
      cat.mean_vr[i0] = (float)(r2[0] / den * (double)H.uv);
      // in(ix, jy) column-major from the sums of bc(ix)*bc(jy) (jy <= ix kept)
      // in(jy*3+ix) = sum m*bc(ix)*bc(jy) / den; r[4..9] hold (0,0) (0,1) (0,2)
      // (1,1) (1,2) (2,2) as (jy,ix), r[13..15] the lower (1,0) (2,0) (2,1)
      float xx = (float)(r[4] / den), yx = (float)(r[5] / den), zx = (float)(r[6] / den);
      float yy = (float)(r[7] / den), zy = (float)(r[8] / den), zz = (float)(r[9] / den);
      float in[9] = {xx, yx, zx, yx, yy, zy, zx, zy, zz};
      if constexpr (!SYM) {
        in[3] = (float)(r[13] / den);
        in[6] = (float)(r[14] / den);
        in[7] = (float)(r[15] / den);
      }
      float* it = cat.inertia_tensor + (size_t)i0 * 6;
      it[0] = in[0]; it[1] = in[3]; it[2] = in[6]; it[3] = in[4]; it[4] = in[7]; it[5] = in[8];
      cat.velocity_dispersion[i0] = (float)(sqrt(r[0] / (double)(float)cnt) * (double)H.uv);
      cat.vmaxclus[i0] = __fmul_rn(__fsqrt_rn(vmax), H.uv);
      // the eigenvalues (DIAGONALISE, a serial FP64 Jacobi loop) come from
      // k_eigen, one thread per halo, instead of this group's lead thread
      for (int q = 0; q < 9; q++) eig_in[q] = in[q];
    }
  }
  g.sync();
  return cnt;
}

// Eigenvalues of the inertia tensors the per-halo kernels left in eig_in
// (9 entries per slot, NaN in the first: none): DIAGONALISE (num.f:2-116),
// the descending sort and SQRT(5*eig), one thread per slot.
__global__ void k_eigen(const float* __restrict__ eig_in, const int32_t* __restrict__ work, int ns,
                        float* __restrict__ eigenval) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  float in[9];
  for (int q = 0; q < 9; q++) in[q] = eig_in[(size_t)s * 9 + q];
  if (in[0] != in[0]) return;
  float be[3] = {0.0f, 0.0f, 0.0f};
  diagonalise_dev(in, be);
  sort_eigen_dev(be);
  const int i0 = work[s];
  for (int q = 0; q < 3; q++) eigenval[(size_t)i0 * 3 + q] = __fsqrt_rn(__fmul_rn(5.0f, be[q]));
}

template <int C>
__global__ void __launch_bounds__(C == 0 ? 32 : HB, C == 0 ? 24 : 3)
k_halo_main(const int32_t* __restrict__ slots, Store S, HConst H, asohf_catalogue cat,
            const int32_t* __restrict__ work, GrowOut go, SegG sg) {
  __shared__ GShared sh;
  Grp<C> g;
  const int slot = group_slot<C>(slots);
  const bool lead = leader(g.rank());
  const int i0 = work[slot];
  const int64_t K = go.konta[slot];
  const unsigned long long t_start = sg.timing ? gtimer_ns() : 0ull;
  if (lead) { sg.nbound[slot] = 0; sg.nscan[slot] = 0; sg.final_b[slot] = 0; }
  if (K == 0) return;
  const int64_t base = sg.off[slot] + slot;
  SegView va = view_at(sg.a, base), vb = view_at(sg.b, base);
  double* pot = sg.pot + base;
  uint8_t* flag = sg.flag + base;
  load_segment(g, S, sg.keys + sg.off[slot], sg.vals + sg.off[slot], K, va, vb, flag);
  SegView cur = va, nxt = vb;
  int which = 0;
  float cx = go.cx[slot], cy = go.cy[slot], cz = go.cz[slot];
  const int kk_entero = cat.realclus[i0];
  const float pi = H.pi, rote = H.rote, rete = H.rete, fdm = H.fdm, um = H.um;
  const float norma = S.norma;
  int64_t k2 = K, idx_vir = K;
  float ref_max = cur.dm[K - 1].x;
  HaloState h;
  h.radio = go.rclus[slot];
  h.masa = (float)(go.masadm[slot] * (double)um);
  h.realclus = kk_entero;
  // FIND_IDX_VIR (haloes_particles.f:1453-1491)
  {
    int64_t jjcore = min(idx_vir / 10, (int64_t)50);
    float den0 = __fmul_rn(__fmul_rn(rote, __fmul_rn(__fmul_rn(rete, rete), rete)),
                           __fdiv_rn(__fmul_rn(4.0f, pi), 3.0f));
    float cvir = __fmul_rn(H.contrastec, fdm);
    long long best = LLONG_MAX;
    gscan_d(g, 0, idx_vir, 0.0, [&](int64_t j) { return (double)cur.dm[j].y; },
              [&](int64_t j, double menc) {
                if (j + 1 <= jjcore) return;
                float d = cur.dm[j].x;
                float den = __fmul_rn(den0, __fmul_rn(__fmul_rn(d, d), d));
                float delta = (float)(menc / (double)den);
                if (delta < cvir && (long long)(j + 1) < best) best = j + 1;
              },
              sh.wsum, sh.x);
    gmin_llv<1>(g, &best, sh.lred, sh.x);
    if (best == LLONG_MAX) {
      if (lead) sg.status[slot] = ASOHF_ERR_NOT_PREFOUND_VIRIAL;
      return;
    }
    idx_vir = best;
  }
  float cm0[3], v0[3], m2;
  centromasas_g(g, cur, idx_vir, cm0, v0, &m2, sh);
  for (int q = 0; q < 3; q++) { h.cm[q] = cm0[q]; h.v[q] = v0[q]; }
  unsigned long long ep = (unsigned long long)K + (unsigned long long)idx_vir;  // element-passes
  // escape-velocity unbinding (haloes_particles.f:894-907)
  int64_t contaerr = K;
  int fac = 0;
  PotCache pc;
  while (contaerr > 0 || fac < 3) {
    fac++;
    int64_t prev = k2;
    ep += (unsigned long long)k2;
    long long kept = unbinding8_g(g, norma, H, fac, ref_max, cur, flag, pot, k2, idx_vir, h, sh, pc);
    if (kept != k2) {  // nothing removed: the list, IDX_VIR and the tail stay as they are
      int64_t nk2;
      compact_g(g, cur, nxt, flag, k2, &idx_vir, &nk2, sh);
      SegView t = cur; cur = nxt; nxt = t; which ^= 1;
      k2 = nk2;
      pc.valid = pc.flags_valid = false;
    }
    ref_max = k2 > 0 ? cur.dm[k2 - 1].x : 1.e10f;
    contaerr = prev - k2;
    if (fac > 100000) break;
  }
  const int fac8 = fac;
  // sigma clipping (haloes_particles.f:918-933)
  fac = 0;
  contaerr = k2;
  SigCache sc;
  while (contaerr > 0 || fac < 4) {
    fac++;
    int64_t prev = k2;
    ep += (unsigned long long)k2;
    long long kept = unbinding_sigma_g(g, H, fac, cur, flag, k2, idx_vir, h, sh, sc);
    if (kept != k2) {
      int64_t nk2;
      compact_g(g, cur, nxt, flag, k2, &idx_vir, &nk2, sh);
      SegView t = cur; cur = nxt; nxt = t; which ^= 1;
      k2 = nk2;
      sc.valid = sc.flags_valid = false;
    }
    ref_max = k2 > 0 ? cur.dm[k2 - 1].x : 1.e10f;
    contaerr = prev - k2;
    if (fac > 100000) break;
  }
  if (lead) sg.final_b[slot] = (uint8_t)which;
  if (k2 < H.min_num_part) {
    if (lead) {
      cat.realclus[i0] = 0;
      cat.radio[i0] = h.radio; cat.masa[i0] = h.masa;
      cat.clusrxcm[i0] = h.cm[0]; cat.clusrycm[i0] = h.cm[1]; cat.clusrzcm[i0] = h.cm[2];
      cat.vx[i0] = h.v[0]; cat.vy[i0] = h.v[1]; cat.vz[i0] = h.v[2];
      cat.dmpclus[i0] = (int32_t)K;
    }
    return;
  }
  // ---------------------------------------------------------- SO walk
  // haloes_particles.f:973-1182.  BAS8 is the cumulative mass; once the
  // virial crossing is found the loop subtracts that particle from BAS8 and
  // keeps walking until 200m is found too, so crossings past it see
  // BAS8 - m(J_vir).
  int64_t jjcore = (int64_t)fmaxf(10.0f, __fdiv_rn((float)k2, 100.0f));
  float thr[6] = {__fmul_rn(__fdiv_rn(2500.0f, H.omegaz), fdm), __fmul_rn(__fdiv_rn(500.0f, H.omegaz), fdm),
                  __fmul_rn(__fdiv_rn(200.0f, H.omegaz), fdm), __fmul_rn(2500.0f, fdm),
                  __fmul_rn(500.0f, fdm), __fmul_rn(200.0f, fdm)};
  float cvir = __fmul_rn(H.contrastec, fdm);
  int64_t jvir_min = (int64_t)__fmul_rn(0.1f, (float)k2);
  auto mn_of = [&](int64_t j) { return (double)__fdiv_rn(cur.dm[j].y, norma); };
  // pass A: virial crossing and the crossings at or before it; BAS8 of
  // every entry is kept in pot[] (free after the unbinding) for the later
  // passes, which read it instead of scanning again
  long long jt[7];
  for (int q = 0; q < 7; q++) jt[q] = LLONG_MAX;
  gscan_d(g, 0, k2, 0.0, mn_of,
            [&](int64_t j, double bas8) {
              pot[j] = bas8;
              int64_t J = j + 1;
              if (J <= jjcore) return;
              float vol = so_den(cur.dm[j].x, rete, pi);
              float delta2 = (float)((double)norma * bas8 / (double)vol / (double)rote);
              for (int q = 0; q < 6; q++)
                if (delta2 <= thr[q] && J < jt[q]) jt[q] = J;
              if (delta2 <= cvir && J > jvir_min && J < jt[6]) jt[6] = J;
            },
            sh.wsum, sh.x);
  gmin_llv<7>(g, jt, sh.lred, sh.x);
  long long jvir = jt[6];
  double mvir = 0.0;
  if (jvir != LLONG_MAX) {
    mvir = (double)__fdiv_rn(cur.mv[jvir - 1].x, norma);
    bool again = false;
    for (int q = 0; q < 6; q++)
      if (jt[q] > jvir) { jt[q] = LLONG_MAX; again = true; }
    if (again) {  // pass A2: crossings after the virial one, with BAS8 - m(J_vir)
      int64_t lo, hi;
      g.chunk(jvir, k2, &lo, &hi);
      for (int64_t j = lo + threadIdx.x; j < hi; j += blockDim.x) {
        const int64_t J = j + 1;
        double b8 = pot[j] - mvir;
        float vol = so_den(cur.dm[j].x, rete, pi);
        float delta2 = (float)((double)norma * b8 / (double)vol / (double)rote);
        for (int q = 0; q < 6; q++)
          if (delta2 <= thr[q] && J < jt[q]) jt[q] = J;
      }
      gmin_llv<6>(g, jt, sh.lred, sh.x);
    }
  }
  bool exit_found = jvir != LLONG_MAX && jt[5] != LLONG_MAX;
  int64_t jend = exit_found ? max(jvir, jt[5]) : k2;
  // pass B: BAS8 at the crossings (read from pot[]), V_c max over the walked
  // range, and the velocity sums up to the virial crossing (or the whole walk)
  double best_v = -1.0;
  long long best_j = LLONG_MAX;
  double best_b = 0.0;
  int64_t jv = jvir != LLONG_MAX ? jvir : jend;
  double sv[11];
  for (int q = 0; q < 11; q++) sv[q] = 0.0;
  if (lead) {  // one contribution per group
    for (int q = 0; q < 7; q++)
      if (jt[q] != LLONG_MAX && jt[q] <= jend) {
        const double bas8 = pot[jt[q] - 1];
        sv[q] = (q == 6 || jvir == LLONG_MAX || jt[q] <= jvir) ? bas8 : bas8 - mvir;
      }
    if (jv >= 1) sv[7] = pot[jv - 1];
  }
  {
    int64_t lo, hi;
    g.chunk(0, jend, &lo, &hi);
    for (int64_t j = lo + threadIdx.x; j < hi; j += blockDim.x) {
      const int64_t J = j + 1;
      if (j < jv) {
        float4 q = cur.mv[j];
        float mn = __fdiv_rn(q.x, norma);
        sv[8] += (double)__fmul_rn(mn, q.y);
        sv[9] += (double)__fmul_rn(mn, q.z);
        sv[10] += (double)__fmul_rn(mn, q.w);
      }
      if (J <= jjcore) continue;
      const double bas8 = pot[j];
      double b8 = (jvir != LLONG_MAX && J > jvir) ? bas8 - mvir : bas8;
      float bas2 = (float)(b8 / (double)cur.dm[j].x);
      if (best_before((double)bas2, J, best_v, best_j)) {
        best_v = bas2;
        best_j = J;
        best_b = b8;
      }
    }
  }
  gsum_dv<11>(g, sv, sh.x);
  gbest(g, &best_v, &best_j, &best_b, sh);
  float rshell = 0.0f;
  int64_t ncapas = 0;
  if (lead) {
    const double* s_at = sv;       // BAS8 at the crossings
    double s_vs[4] = {sv[7], sv[8], sv[9], sv[10]};
    if (best_j != LLONG_MAX) {
      cat.vcmax[i0] = (float)best_v;
      cat.mcmax[i0] = (float)best_b;
      cat.rcmax[i0] = cur.dm[best_j - 1].x;
    }
    float* mo[6] = {cat.m2500c, cat.m500c, cat.m200c, cat.m2500m, cat.m500m, cat.m200m};
    float* ro[6] = {cat.r2500c, cat.r500c, cat.r200c, cat.r2500m, cat.r500m, cat.r200m};
    bool f200m = false;
    for (int q = 0; q < 6; q++) {
      if (jt[q] != LLONG_MAX && jt[q] <= jend) {
        int64_t J = jt[q];
        float d = cur.dm[J - 1].x;
        float vol = so_den(d, rete, pi);
        float delta2 = (float)((double)norma * s_at[q] / (double)vol / (double)rote);
        mo[q][i0] = __fmul_rn(__fmul_rn(__fmul_rn(delta2, vol), rote), um);
        ro[q][i0] = d;
        if (J == jjcore + 1) { mo[q][i0] = -1.0f; ro[q][i0] = -1.0f; }
        if (q == 5) f200m = true;
      }
    }
    bool salida = false;
    if (jvir != LLONG_MAX) {
      float4 q = cur.mv[jvir - 1];
      float mn = __fdiv_rn(q.x, norma);
      double bas8 = s_vs[0] - (double)mn;
      double bvx = s_vs[1] - (double)__fmul_rn(mn, q.y);
      double bvy = s_vs[2] - (double)__fmul_rn(mn, q.z);
      double bvz = s_vs[3] - (double)__fmul_rn(mn, q.w);
      h.masa = (float)(bas8 * (double)norma * (double)um);
      float vol = (float)(((double)norma * bas8) / (double)__fmul_rn(__fmul_rn(H.contrastec, fdm), rote));
      h.radio = __fdiv_rn(powf(__fdiv_rn(__fmul_rn(3.0f, vol), __fmul_rn(4.0f, pi)), 1.0f / 3.0f), rete);
      h.v[0] = (float)(bvx / bas8);
      h.v[1] = (float)(bvy / bas8);
      h.v[2] = (float)(bvz / bas8);
      ncapas = jvir - 1;
      rshell = h.radio;
      salida = true;
    }
    {
      float bas = __fdiv_rn(__fmul_rn(__fmul_rn(cat.vcmax[i0], norma), H.cgr), rete);
      cat.vcmax[i0] = __fmul_rn(__fsqrt_rn(bas), H.uv);
      cat.mcmax[i0] = __fmul_rn(__fmul_rn(cat.mcmax[i0], norma), um);
    }
    if (kk_entero == -1 && !salida) {
      double bas8 = s_vs[0];
      h.masa = (float)(bas8 * (double)norma * (double)um);
      float vol = (float)(((double)norma * bas8) / (double)__fmul_rn(__fmul_rn(H.contrastec, fdm), rote));
      h.radio = __fdiv_rn(powf(__fdiv_rn(__fmul_rn(3.0f, vol), __fmul_rn(4.0f, pi)), 1.0f / 3.0f), rete);
      h.v[0] = (float)(s_vs[1] / bas8);
      h.v[1] = (float)(s_vs[2] / bas8);
      h.v[2] = (float)(s_vs[3] / bas8);
      ncapas = jend;  // J - 1 with J = KONTA2 + 1
      rshell = h.radio;
      if (!f200m) {
        cat.m200m[i0] = h.masa;
        cat.r200m[i0] = __fmul_rn(h.radio, powf(__fdiv_rn(H.contrastec, 200.0f), 1.0f / 3.0f));
      }
    }
    cat.radio[i0] = h.radio; cat.masa[i0] = h.masa;
    cat.clusrxcm[i0] = h.cm[0]; cat.clusrycm[i0] = h.cm[1]; cat.clusrzcm[i0] = h.cm[2];
    cat.vx[i0] = h.v[0]; cat.vy[i0] = h.v[1]; cat.vz[i0] = h.v[2];
    cat.realclus[i0] = h.realclus;
    cat.dmpclus[i0] = (int32_t)K;
    sh.bc_d[0] = rshell;
    sh.bc_l[0] = ncapas;
  }
  {
    double rs;
    long long nc;
    gbcast(g, &rs, &nc, sh);
    rshell = (float)rs;
    ncapas = nc;
  }
  if (ncapas < H.min_num_part) {
    if (lead) cat.realclus[i0] = 0;
    return;
  }
  int unsup = 0;
  long long nb = properties_g(g, S, H, cat, i0, cur, flag, ncapas, rshell, cx, cy, cz, cm0, sh, &unsup, nxt, pot,
                              sg.eig + (size_t)slot * 9);
  ep += (unsigned long long)(k2 + ncapas);  // SO walk and property loop
  if (lead) {
    atomicAdd(&sg.work[0], ep);
    if (sg.timing) {  // unbinding iterations in [2..3]; duration of this halo: max and sum,
                      // clusters in [4..5], single CTAs in [6..7]
      atomicAdd(&sg.work[2], (unsigned long long)fac8);
      atomicAdd(&sg.work[3], (unsigned long long)fac);
      unsigned long long dt = gtimer_ns() - t_start;
      atomicMax(&sg.work[C > 1 ? 4 : 6], dt);
      atomicAdd(&sg.work[C > 1 ? 5 : 7], dt);
    }
    bool ok = nb >= H.min_num_part && H.want_ids;
    sg.nbound[slot] = ok ? (int32_t)nb : 0;
    sg.nscan[slot] = ok ? (int32_t)ncapas : 0;
    sg.status[slot] = unsup == 1 ? ASOHF_ERR_UNSUPPORTED : unsup == 2 ? ASOHF_ERR_TIMEOUT : 0;
  }
}

// IDs of the bound particles, in radial order, at ids_off[slot].
template <int C>
__global__ void __launch_bounds__(HB)
k_write_ids(const int32_t* __restrict__ slots, const int32_t* __restrict__ nscan, const int64_t* __restrict__ off,
            const int64_t* __restrict__ ids_off, const uint8_t* __restrict__ final_b,
            const float4* __restrict__ px_a, const float4* __restrict__ px_b,
            const uint8_t* __restrict__ flag_all, const int32_t* __restrict__ id, int32_t* __restrict__ out) {
  __shared__ int sb[33];
  __shared__ long long lred[32];
  __shared__ GX x;
  Grp<C> g;
  int slot = group_slot<C>(slots);
  int64_t n = nscan[slot];
  if (n == 0) return;
  int64_t base = off[slot] + slot;
  const float4* px = (final_b[slot] ? px_b : px_a) + base;
  const uint8_t* flag = flag_all + base;
  int64_t lo, hi;
  g.chunk(0, n, &lo, &hi);
  long long mine = 0;
  if constexpr (C > 1) {
    for (int64_t j = lo + threadIdx.x; j < hi; j += blockDim.x) mine += flag[j];
    mine = block_sum_ll(mine, lred);
  }
  long long o = 0, tot = 0;
  gexcl_ll(g, mine, &o, &tot, x);
  int64_t carry = ids_off[slot] + o;
  for (int64_t t0 = lo; t0 < hi; t0 += blockDim.x) {
    int64_t j = t0 + threadIdx.x;
    bool k = j < hi && flag[j];
    int tt;
    int inc = block_scan_i(k ? 1 : 0, sb, &tt);
    if (k) out[carry + inc - 1] = id[__float_as_int(px[j].w)];
    carry += tt;
    __syncthreads();
  }
}

// ---------------------------------------------------------------- host driver
int ensure_pph(asohf_ctx* c, int64_t need) {
  if (need <= c->pph_cap) return ASOHF_OK;
  int64_t cap = need + need / 2 + 1024;
  int32_t* nb = nullptr;
  ASOHF_CUDA(cudaMalloc(&nb, 4 * (size_t)cap));
  if (c->d_pph && c->pph_len > 0)
    ASOHF_CUDA(cudaMemcpyAsync(nb, c->d_pph, 4 * (size_t)c->pph_len, cudaMemcpyDeviceToDevice, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(c->d_pph);
  c->d_pph = nb;
  c->pph_cap = cap;
  return ASOHF_OK;
}

// Host part of the ID concatenation (haloes_particles.f:1377-1408): INDCS of
// haloes low1..low2 from the counts, offsets for k_write_ids.
int assign_id_offsets(asohf_ctx* c, CatMirror& m, int low1, int low2, const int32_t* work, int nslots,
                      const int32_t* d_nbound, int64_t* d_ids_off, int64_t* total_out) {
  int n = low2;
  std::vector<int32_t> realclus_v((size_t)n);
  int32_t* realclus = realclus_v.data();
  std::vector<int32_t> indcs_v(2 * (size_t)n);
  int32_t* indcs = indcs_v.data();
  std::vector<int32_t> nbound_v((size_t)(nslots > 0 ? nslots : 1));
  int32_t* nbound = nbound_v.data();
  std::vector<int64_t> ids_off_v((size_t)(nslots > 0 ? nslots : 1));
  int64_t* ids_off = ids_off_v.data();
  std::vector<int32_t> slot_of_v((size_t)(low2 - low1 + 1));
  int32_t* slot_of = slot_of_v.data();
  // entries before the window: from the caller's arrays when they are on the host
  int h0 = m.host ? m.w0 : 0;
  if (h0) {
    memcpy(realclus, m.h.realclus, 4 * (size_t)h0);
    memcpy(indcs, m.h.indcs, 8 * (size_t)h0);
  }
  ASOHF_CUDA(cudaMemcpyAsync(realclus + h0, m.d.realclus + h0, 4 * (size_t)(n - h0), cudaMemcpyDeviceToHost,
                             c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(indcs + 2 * (size_t)h0, m.d.indcs + 2 * (size_t)h0, 8 * (size_t)(n - h0),
                             cudaMemcpyDeviceToHost, c->stream));
  if (nslots)
    ASOHF_CUDA(cudaMemcpyAsync(nbound, d_nbound, 4 * (size_t)nslots, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < low2 - low1 + 1; i++) slot_of[i] = -1;
  for (int s = 0; s < nslots; s++) slot_of[work[s] - (low1 - 1)] = s;
  int64_t j = 0;
  for (int i = 1; i < low1; i++)
    if (realclus[i - 1] != 0 && indcs[(i - 1) * 2 + 1] > j) j = indcs[(i - 1) * 2 + 1];
  for (int i = low1; i <= low2; i++) {
    if (realclus[i - 1] == 0) {
      indcs[(i - 1) * 2] = -1;
      indcs[(i - 1) * 2 + 1] = -1;
      continue;
    }
    int s = slot_of[i - low1];
    indcs[(i - 1) * 2] = (int32_t)(j + 1);
    if (s >= 0) {
      ids_off[s] = j;
      j += nbound[s];
    }
    indcs[(i - 1) * 2 + 1] = (int32_t)j;
  }
  for (int s = 0; s < nslots; s++)
    if (realclus[work[s]] == 0) ids_off[s] = 0;
  ASOHF_CUDA(cudaMemcpyAsync(m.d.indcs + 2 * (size_t)(low1 - 1), indcs + 2 * (size_t)(low1 - 1),
                             8 * (size_t)(low2 - low1 + 1), cudaMemcpyHostToDevice, c->stream));
  if (nslots)
    ASOHF_CUDA(cudaMemcpyAsync(d_ids_off, ids_off, 8 * (size_t)nslots, cudaMemcpyHostToDevice, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  *total_out = j;
  return ASOHF_OK;
}

// Work list: haloes of [low1, low2] with REALCLUS != 0, DMPCLUS descending
// (largest first keeps the longest CTAs from finishing last).
int make_work(asohf_ctx* c, CatMirror& m, int low1, int low2, std::vector<int32_t>& h_work, int* nslots,
              std::vector<int32_t>* h_dm = nullptr) {
  int nh = low2 - low1 + 1;
  std::vector<int32_t> rc_v((size_t)nh);
  int32_t* rc = rc_v.data();
  std::vector<int32_t> dm_v((size_t)nh);
  int32_t* dm = dm_v.data();
  ASOHF_CUDA(cudaMemcpyAsync(rc, m.d.realclus + low1 - 1, 4 * (size_t)nh, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(dm, m.d.dmpclus + low1 - 1, 4 * (size_t)nh, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  h_work.assign(nh > 0 ? nh : 1, 0);
  int32_t* w = h_work.data();
  int k = 0;
  for (int i = 0; i < nh; i++)
    if (rc[i] != 0) w[k++] = low1 - 1 + i;
  // sort by DMPCLUS descending (stable); the signed value biased to an
  // unsigned key of the same order
  std::vector<uint32_t> key((size_t)(k > 0 ? k : 1));
  for (int i = 0; i < k; i++) key[i] = (uint32_t)dm[w[i] - (low1 - 1)] ^ 0x80000000u;
  stable_desc(key, w, k);
  if (h_dm) {  // DMPCLUS of each slot
    h_dm->assign(k > 0 ? k : 1, 0);
    for (int i = 0; i < k; i++) (*h_dm)[i] = dm[w[i] - (low1 - 1)];
  }
  *nslots = k;
  return ASOHF_OK;
}

// Cluster size for the large haloes on this device: 16 CTAs where the
// device can co-schedule such clusters of k_halo_main, else 8, else 1.
static int g_big_cluster[64];

template <typename... P>
static int max_clusters(void (*kern)(P...), int C) {
  if (C > 8 && cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)C);
  cfg.blockDim = dim3(HB);
  cudaLaunchAttribute a[1];
  a[0].id = cudaLaunchAttributeClusterDimension;
  a[0].val.clusterDim.x = C;
  a[0].val.clusterDim.y = 1;
  a[0].val.clusterDim.z = 1;
  cfg.attrs = a;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

static int big_cluster(asohf_ctx* c) {
  int d = c->device;
  if (d < 0 || d >= 64) return 1;
  if (g_big_cluster[d] == 0) {
    int C = 1;
    if (max_clusters(k_halo_main<16>, 16) > 0 && max_clusters(k_halo_grow<16>, 16) > 0 &&
        max_clusters(k_halo_gather<16>, 16) > 0 && max_clusters(k_write_ids<16>, 16) > 0)
      C = 16;
    else if (max_clusters(k_halo_main<8>, 8) > 0 && max_clusters(k_halo_grow<8>, 8) > 0 &&
             max_clusters(k_halo_gather<8>, 8) > 0 && max_clusters(k_write_ids<8>, 8) > 0)
      C = 8;
    g_big_cluster[d] = C;
  }
  return g_big_cluster[d];
}

// Launches kern<C> for the `n` groups of slots[] on stream s (C in {1, 8, 16}).
#define LAUNCH_TIER(KERN, C, n, s, ...)                                              \
  ((C) == 16 ? launch_grp(KERN<16>, 16, (n), 256, (s), __VA_ARGS__)                  \
             : (C) == 8 ? launch_grp(KERN<8>, 8, (n), 256, (s), __VA_ARGS__)         \
                        : launch_grp(KERN<1>, 1, (n), 256, (s), __VA_ARGS__))

// The cluster tier on the context stream, the CTA tiers on the side streams,
// the context stream waiting for all.
#define LAUNCH_TIERS(KERN, CB, T, ...) LAUNCH_TIERS_W(KERN, CB, 1, T, __VA_ARGS__)
// W0: group template argument of the 32-thread tier (0: the one-warp build)
#define LAUNCH_TIERS_W(KERN, CB, W0, T, ...)                                                        \
  do {                                                                                              \
    ASOHF_CHECK(fork_all(c));                                                                       \
    if ((T).n[3] > 0) {                                                                             \
      int k3_ = ktime_begin(c, #KERN "/cluster", c->stream);                                        \
      ASOHF_CUDA(LAUNCH_TIER(KERN, CB, (T).n[3], c->stream, (T).slots[3], __VA_ARGS__));            \
      ktime_end(c, k3_, c->stream);                                                                 \
    }                                                                                               \
    for (int t_ = 2; t_ >= 0; t_--)                                                                 \
      if ((T).n[t_] > 0) {                                                                          \
        static const char* const nm_[3] = {#KERN "/cta32", #KERN "/cta128", #KERN "/cta256"};       \
        cudaStream_t s_ = c->side[2 - t_];                                                          \
        int k_ = ktime_begin(c, nm_[t_], s_);                                                       \
        if (t_ == 0)                                                                                \
          ASOHF_CUDA(launch_grp(KERN<W0>, 1, (T).n[0], 32, s_, (T).slots[0], __VA_ARGS__));         \
        else                                                                                        \
          ASOHF_CUDA(launch_grp(KERN<1>, 1, (T).n[t_], kTierThreads[t_], s_, (T).slots[t_], __VA_ARGS__)); \
        ktime_end(c, k_, s_);                                                                       \
      }                                                                                             \
    ASOHF_CHECK(join_all(c));                                                                       \
    for (int t_ = 0; t_ < 4; t_++) c->launches += (T).n[t_] > 0;                                    \
  } while (0)

// The same tiers for kernels that run on single CTAs only: the cluster tier
// becomes 256-thread CTAs on the context stream.
#define LAUNCH_TIERS_CTA(KERN, T, ...)                                                               \
  do {                                                                                              \
    ASOHF_CHECK(fork_all(c));                                                                       \
    if ((T).n[3] > 0) ASOHF_CUDA(launch_grp(KERN<1>, 1, (T).n[3], 256, c->stream, (T).slots[3], __VA_ARGS__)); \
    for (int t_ = 2; t_ >= 0; t_--)                                                                 \
      if ((T).n[t_] > 0)                                                                            \
        ASOHF_CUDA(launch_grp(KERN<1>, 1, (T).n[t_], kTierThreads[t_], c->side[2 - t_], (T).slots[t_], \
                              __VA_ARGS__));                                                        \
    ASOHF_CHECK(join_all(c));                                                                       \
    for (int t_ = 0; t_ < 4; t_++) c->launches += (T).n[t_] > 0;                                    \
  } while (0)

extern "C" int asohf_set_epot_seed(asohf_ctx* c, uint32_t seed) {
  if (!c) return ASOHF_ERR_INVALID;
  c->epot_seed = seed;
  return ASOHF_OK;
}

extern "C" int asohf_set_cluster_threshold(asohf_ctx* c, int64_t min_members) {
  if (!c || min_members < 0) return ASOHF_ERR_INVALID;
  c->cluster_min = min_members == 0 ? BIG_K : min_members;
  return ASOHF_OK;
}

extern "C" int asohf_set_cluster_share(asohf_ctx* c, int64_t members_per_cta) {
  if (!c || members_per_cta < 0) return ASOHF_ERR_INVALID;
  c->cluster_share = members_per_cta == 0 ? 32768 : members_per_cta;
  return ASOHF_OK;
}

extern "C" int asohf_set_group_tiers(asohf_ctx* c, int64_t tier1_members, int64_t tier2_members) {
  if (!c || tier1_members < 0 || tier2_members < 0) return ASOHF_ERR_INVALID;
  int64_t t1 = tier1_members == 0 ? TIER1_K : tier1_members;
  int64_t t2 = tier2_members == 0 ? TIER2_K : tier2_members;
  if (t2 < t1) return ASOHF_ERR_INVALID;
  c->tier1_k = t1;
  c->tier2_k = t2;
  return ASOHF_OK;
}

extern "C" int asohf_halofind_particles(asohf_ctx* c, const asohf_consts* k, const asohf_mesh* mesh,
                                        asohf_catalogue* cat, int lowh1, int lowh2, int on_device) {
  if (!c || !k || !cat || lowh1 < 1 || lowh2 > cat->nclus) return ASOHF_ERR_INVALID;
  if (lowh2 < lowh1) return ASOHF_OK;
  if (c->nx_sorted != k->nx) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  double ht = htime_now();
  arena_reset(c);
  int nh = lowh2 - lowh1 + 1;
  size_t need = cat_bytes(lowh2) + (size_t)nh * (96 + 40) + 65536;
  ASOHF_CHECK(arena_reserve(c, need));
  CatMirror m;
  ASOHF_CHECK(cat_mirror_in(c, cat, lowh2, on_device, &m, lowh1 - 1));
  std::vector<int32_t> hw_v, hdm_v;
  int ns;
  ASOHF_CHECK(make_work(c, m, lowh1, lowh2, hw_v, &ns, &hdm_v));
  int32_t* hw = hw_v.data();
  int32_t* hdm = hdm_v.data();
  htime_end(c, "host:halo_mirror_in+work", ht);
  ht = htime_now();
  Store S = store_of(c);
  ColIdx ci = col_idx(c, k);
  HConst H = hconst(k, mesh);
  H.epot_seed = c->epot_seed;
  const int CB = big_cluster(c);
  int rc = ASOHF_OK;
  if (ns > 0) {
    // per-slot buffers
    int32_t* d_work = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    int32_t* d_tg = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    int32_t* d_tm = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    int32_t* d_fill = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    uint8_t* d_final = (uint8_t*)arena_alloc(c, (size_t)ns);
    GrowOut g;
    g.cx = (float*)arena_alloc(c, 4 * (size_t)ns);
    g.cy = (float*)arena_alloc(c, 4 * (size_t)ns);
    g.cz = (float*)arena_alloc(c, 4 * (size_t)ns);
    g.rgather = (float*)arena_alloc(c, 4 * (size_t)ns);
    g.rclus = (float*)arena_alloc(c, 4 * (size_t)ns);
    g.konta = (int32_t*)arena_alloc(c, 4 * (size_t)ns + 4);
    g.masadm = (double*)arena_alloc(c, 8 * (size_t)ns);
    g.status = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    int64_t* d_off = (int64_t*)arena_alloc(c, 8 * (size_t)(ns + 1));
    int32_t* d_nbound = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    int32_t* d_nscan = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    int64_t* d_ids_off = (int64_t*)arena_alloc(c, 8 * (size_t)ns);
    if (!d_work || !d_tg || !d_tm || !d_fill || !d_final || !g.cx || !g.cy || !g.cz ||
        !g.rgather || !g.rclus || !g.konta || !g.masadm || !g.status || !d_off || !d_nbound || !d_nscan ||
        !d_ids_off) {
      return ASOHF_ERR_CAPACITY;
    }
    ASOHF_CUDA(cudaMemcpyAsync(d_work, hw, 4 * (size_t)ns, cudaMemcpyHostToDevice, c->stream));
    // growth, tiered first by DMPCLUS (the members counted when the candidate
    // was pruned); haloes that outgrow their group size resume in a larger one
    Tiers tg, tm;
    GrowCaps caps{c->tier2_k, 4 * c->tier2_k, CB > 1 ? c->cluster_min : (int64_t)LLONG_MAX};
    std::vector<int32_t> hk_v((size_t)ns);
    int32_t* hk = hk_v.data();
    std::vector<int32_t> hst_v((size_t)ns);
    int32_t* hst = hst_v.data();
    std::vector<int64_t> hoff_v((size_t)(ns + 1));
    int64_t* hoff = hoff_v.data();
    std::vector<int32_t> hesc_v((size_t)ns);
    int32_t* hesc = hesc_v.data();
    std::vector<int32_t> kesc_v((size_t)ns);
    int32_t* kesc = kesc_v.data();
    ASOHF_CHECK(split_tiers(c, hdm, ns, d_tg, &tg));
    for (int round = 0;; round++) {
      {
        int kt_ = ktime_begin(c, "halo_grow");
        LAUNCH_TIERS(k_halo_grow, CB, tg, S, ci, H, m.d, d_work, g, caps, round > 0 ? 1 : 0);
        ktime_end(c, kt_);
      }
      ASOHF_CUDA(cudaMemcpyAsync(hk, g.konta, 4 * (size_t)ns, cudaMemcpyDeviceToHost, c->stream));
      ASOHF_CUDA(cudaMemcpyAsync(hst, g.status, 4 * (size_t)ns, cudaMemcpyDeviceToHost, c->stream));
      ASOHF_CUDA(cudaStreamSynchronize(c->stream));
      int ne = 0;
      for (int s = 0; s < ns; s++)
        if (hst[s] == GROW_ESCALATE) { hesc[ne] = s; kesc[ne++] = hk[s]; }
      if (ne == 0) break;
      // escalated haloes: tiers by their member count at hand-over, slot ids
      // through the escalation list
      if (round >= 3) break;  // every tier was tried: reported below
      ASOHF_CHECK(split_tiers(c, kesc, ne, d_tg, &tg, hesc));
    }
    htime_end(c, "host:halo_grow", ht);
    ht = htime_now();
    hoff[0] = 0;
    bool left = false;  // haloes no group size could finish (not expected)
    for (int s = 0; s < ns; s++) {
      if (hst[s]) rc = hst[s] == GROW_ESCALATE ? ASOHF_ERR_CAPACITY : hst[s];
      if (hst[s] == GROW_ESCALATE) { hk[s] = 0; left = true; }
      hoff[s + 1] = hoff[s] + hk[s];
    }
    if (left) ASOHF_CUDA(cudaMemcpyAsync(g.konta, hk, 4 * (size_t)ns, cudaMemcpyHostToDevice, c->stream));
    int64_t T = hoff[ns];
    ASOHF_CUDA(cudaMemcpyAsync(d_off, hoff, 8 * (size_t)(ns + 1), cudaMemcpyHostToDevice, c->stream));
    ASOHF_CHECK(split_tiers(c, hk, ns, d_tm, &tm));
    // element buffers (allocated after the per-slot ones: the arena grows
    // only when empty, so reserve everything now)
    int bits = 1;
    while ((1ll << bits) < ns) bits++;
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                    (int32_t*)nullptr, (int32_t*)nullptr, (int)(T > 0 ? T : 1), 0, 32 + bits);
    size_t E = (size_t)T + ns;
    size_t elem = (size_t)T * (8 + 8 + 4 + 4) + tb + E * (2 * (8 + 16 + 16) + 8 + 1) + 32768;
    ASOHF_CHECK(seg_reserve(c, elem));
    unsigned long long* k0 = (unsigned long long*)seg_alloc(c, 8 * (size_t)T + 8);
    unsigned long long* k1 = (unsigned long long*)seg_alloc(c, 8 * (size_t)T + 8);
    int32_t* v0 = (int32_t*)seg_alloc(c, 4 * (size_t)T + 4);
    int32_t* v1 = (int32_t*)seg_alloc(c, 4 * (size_t)T + 4);
    void* t = seg_alloc(c, tb);
    SegG sg;
    sg.konta = g.konta;
    sg.off = d_off;
    sg.a.dm = (float2*)seg_alloc(c, 8 * E);
    sg.a.mv = (float4*)seg_alloc(c, 16 * E);
    sg.a.px = (float4*)seg_alloc(c, 16 * E);
    sg.b.dm = (float2*)seg_alloc(c, 8 * E);
    sg.b.mv = (float4*)seg_alloc(c, 16 * E);
    sg.b.px = (float4*)seg_alloc(c, 16 * E);
    sg.pot = (double*)seg_alloc(c, 8 * E);
    sg.flag = (uint8_t*)seg_alloc(c, E);
    sg.final_b = d_final;
    sg.nbound = d_nbound;
    sg.nscan = d_nscan;
    sg.work = c->d_work;
    sg.status = g.status;
    sg.timing = c->profiling;
    sg.eig = (float*)arena_alloc(c, 36 * (size_t)ns);
    if (!k0 || !k1 || !v0 || !v1 || !t || !sg.a.dm || !sg.a.mv || !sg.a.px || !sg.b.dm || !sg.b.mv || !sg.b.px ||
        !sg.pot || !sg.flag || !sg.eig) {
      return ASOHF_ERR_CAPACITY;
    }
    ASOHF_CUDA(cudaMemsetAsync(sg.eig, 0xff, 36 * (size_t)ns, c->stream));  // NaN: no tensor
    if (T > 0) {
      ASOHF_CUDA(cudaMemsetAsync(d_fill, 0, 4 * (size_t)ns, c->stream));
      {
        int kt_ = ktime_begin(c, "halo_gather");
        LAUNCH_TIERS(k_halo_gather, CB, tm, S, ci, g.konta, d_off, g.cx, g.cy, g.cz,
                     g.rgather, d_fill, k0, v0);
        ktime_end(c, kt_);
      }
      int kt_ = ktime_begin(c, "halo_radix_sort");
      ASOHF_CUDA(cub::DeviceRadixSort::SortPairs(t, tb, k0, k1, v0, v1, (int)T, 0, 32 + bits, c->stream));
      ktime_end(c, kt_);
      {
        int kt_ = ktime_begin(c, "halo_tiefix");
        k_tiefix<<<grid_for(T, 256), 256, 0, c->stream>>>(k1, v1, T, 1);
        ktime_end(c, kt_);
      }
      c->launches += 2;
    }
    sg.keys = k1;
    sg.vals = v1;
    ASOHF_CUDA(cudaStreamSynchronize(c->stream));
    htime_end(c, "host:halo_gather_sort", ht);
    ht = htime_now();
    {
      // the cluster tier by size: every cluster synchronisation costs the
      // same whatever the list length, so a halo gets the smallest cluster
      // that keeps its CTAs' shares near CLUSTER_SHARE entries
      int nsub[3] = {0, 0, 0};  // clusters of CB, 8, 4 CTAs
      int32_t* sub[3] = {tm.slots[3], tm.slots[3], tm.slots[3]};
      if (tm.n[3] > 0) ASOHF_CHECK(split_cluster_tier(c, hk, ns, CB, &tm, nsub, sub));
      int kt_ = ktime_begin(c, "halo_main");
      ASOHF_CHECK(fork_all(c));
      static const int subC[3] = {16, 8, 4};
      static const char* const subn[3] = {"k_halo_main/cluster", "k_halo_main/cluster8", "k_halo_main/cluster4"};
      for (int q = 0; q < 3; q++) {
        if (nsub[q] == 0) continue;
        cudaStream_t s_ = q == 0 ? c->stream : c->side[2 + q];
        int k_ = ktime_begin(c, subn[q], s_);
        const int cs = q == 0 ? CB : subC[q];
        if (cs == 16) ASOHF_CUDA(launch_grp(k_halo_main<16>, 16, nsub[q], HB, s_, sub[q], S, H, m.d, d_work, g, sg));
        else if (cs == 8) ASOHF_CUDA(launch_grp(k_halo_main<8>, 8, nsub[q], HB, s_, sub[q], S, H, m.d, d_work, g, sg));
        else if (cs == 4) ASOHF_CUDA(launch_grp(k_halo_main<4>, 4, nsub[q], HB, s_, sub[q], S, H, m.d, d_work, g, sg));
        else ASOHF_CUDA(launch_grp(k_halo_main<1>, 1, nsub[q], HB, s_, sub[q], S, H, m.d, d_work, g, sg));
        ktime_end(c, k_, s_);
        c->launches++;
      }
      for (int t_ = 2; t_ >= 0; t_--)
        if (tm.n[t_] > 0) {
          static const char* const nm_[3] = {"k_halo_main/cta32", "k_halo_main/cta128", "k_halo_main/cta256"};
          cudaStream_t s_ = c->side[2 - t_];
          int k_ = ktime_begin(c, nm_[t_], s_);
          if (t_ == 0) ASOHF_CUDA(launch_grp(k_halo_main<0>, 1, tm.n[0], 32, s_, tm.slots[0], S, H, m.d, d_work, g, sg));
          else ASOHF_CUDA(launch_grp(k_halo_main<1>, 1, tm.n[t_], kTierThreads[t_], s_, tm.slots[t_], S, H, m.d,
                                     d_work, g, sg));
          ktime_end(c, k_, s_);
          c->launches++;
        }
      ASOHF_CHECK(join_all(c));
      ktime_end(c, kt_);
    }
    {
      int kt_ = ktime_begin(c, "halo_eigen");
      k_eigen<<<(ns + 127) / 128, 128, 0, c->stream>>>(sg.eig, d_work, ns, m.d.eigenval);
      ktime_end(c, kt_);
    }
    c->launches++;
    ASOHF_CUDA(cudaGetLastError());
    ASOHF_CUDA(cudaMemcpyAsync(hst, g.status, 4 * (size_t)ns, cudaMemcpyDeviceToHost, c->stream));
    ASOHF_CUDA(cudaStreamSynchronize(c->stream));
    for (int s = 0; s < ns; s++)
      if (hst[s] && !rc) rc = hst[s];
    htime_end(c, "host:halo_main", ht);
    ht = htime_now();
    if (H.want_ids && rc == ASOHF_OK) {
      int64_t total;
      ASOHF_CHECK(assign_id_offsets(c, m, lowh1, lowh2, hw, ns, d_nbound, d_ids_off, &total));
      ASOHF_CHECK(ensure_pph(c, total));
      {
        int kt_ = ktime_begin(c, "halo_write_ids");
        LAUNCH_TIERS(k_write_ids, CB, tm, d_nscan, d_off, d_ids_off, d_final, sg.a.px,
                     sg.b.px, sg.flag, c->p.id, c->d_pph);
        ktime_end(c, kt_);
      }
      ASOHF_CUDA(cudaGetLastError());
      c->pph_len = total;
    }
  } else if (H.want_ids) {
    int64_t total;
    ASOHF_CHECK(assign_id_offsets(c, m, lowh1, lowh2, hw, 0, nullptr, nullptr, &total));
    c->pph_len = total;
  }
  htime_end(c, "host:halo_ids", ht);
  ht = htime_now();
  ASOHF_CHECK(cat_mirror_out(c, &m));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  htime_end(c, "host:halo_mirror_out", ht);
  return rc;
}

extern "C" int asohf_get_particles_per_halo(asohf_ctx* c, int32_t* out, int64_t cap, int64_t* n,
                                            int on_device) {
  if (!c || !n) return ASOHF_ERR_INVALID;
  *n = c->pph_len;
  if (!out) return ASOHF_OK;
  if (cap < c->pph_len) return ASOHF_ERR_CAPACITY;
  if (c->pph_len > 0)
    ASOHF_CUDA(cudaMemcpyAsync(out, c->d_pph, 4 * (size_t)c->pph_len,
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  return ASOHF_OK;
}

// ================================================================ substructure
// SUBSTRUCTURE_PARTICLES (substructure.f:756-1697).  Per call (subhaloes of
// one level): recentering and the host's enclosed mass (k_sub_prep); the
// Jacobi-radius search (gather, sort, k_sub_jacobi) repeated for the
// subhaloes whose radius must grow x1.5; a last gather at the final radius;
// then k_sub_main_g on the staged lists: unbinding, Jacobi trim, SO walk,
// properties.  The per-subhalo kernels run in the size tiers of the halo
// path, single CTAs only.

struct SubPrep {
  float *cx, *cy, *cz;
  float *mhost, *disthost;
  float *r;          // current Jacobi gather radius
  int32_t* status;
};

// Recentering (substructure.f:879-899) and host characterisation
// (substructure.f:933-983).
__global__ void __launch_bounds__(HB)
k_sub_prep(Store S, ColIdx ci, HConst H, asohf_catalogue cat, const int32_t* __restrict__ work, SubPrep o) {
  __shared__ RecShared sh;
  int slot = blockIdx.x;
  int i0 = work[slot];
  int irr = level_of_patch(H, cat.patchclus[i0]);
  float cx = cat.clusrx[i0], cy = cat.clusry[i0], cz = cat.clusrz[i0];
  float dxpamin = __fdiv_rn(ci.dx, exp2f((float)irr));
  if (!recenter_group(Grp<1>(), S, ci, &cx, &cy, &cz, cat.rsub[i0], dxpamin, sh)) {
    if (threadIdx.x == 0) o.status[slot] = ASOHF_ERR_CAPACITY;
    return;
  }
  if (threadIdx.x != 0) return;
  cat.clusrx[i0] = cx; cat.clusry[i0] = cy; cat.clusrz[i0] = cz;
  int ih = cat.realclus[i0] - 1;
  float mhost = (cat.realclus[ih] == -1) ? cat.masa[ih] : cat.msub[ih];
  float disthost = dist3(cat.clusrx[ih], cat.clusry[ih], cat.clusrz[ih], cx, cy, cz);
  const float* p1 = cat.profiles + (size_t)ih * 2 * ASOHF_NBINS;
  const float* p2 = p1 + ASOHF_NBINS;
  int nbp = ASOHF_NBINS, jj;
  for (jj = 1; jj <= ASOHF_NBINS; jj++)
    if (p1[jj - 1] == 0.0f) { nbp = jj - 1; break; }
  for (jj = 1; jj <= nbp; jj++)
    if (p1[jj - 1] > disthost) break;
  if (jj == 1) {
    float q = __fdiv_rn(disthost, p1[0]);
    mhost = __fmul_rn(p2[0], __fmul_rn(__fmul_rn(q, q), q));
  } else if (jj <= nbp) {
    float a1 = p1[jj - 2], a2 = p1[jj - 1];
    float d3 = __fmul_rn(__fmul_rn(disthost, disthost), disthost);
    float a13 = __fmul_rn(__fmul_rn(a1, a1), a1), a23 = __fmul_rn(__fmul_rn(a2, a2), a2);
    mhost = __fadd_rn(p2[jj - 2], __fdiv_rn(__fmul_rn(__fsub_rn(p2[jj - 1], p2[jj - 2]), __fsub_rn(d3, a13)),
                                            __fsub_rn(a23, a13)));
  } else {
    mhost = p2[nbp - 1 >= 0 ? nbp - 1 : 0];
  }
  o.cx[slot] = cx; o.cy[slot] = cy; o.cz[slot] = cz;
  o.mhost[slot] = mhost;
  o.disthost[slot] = disthost;
  o.r[slot] = __fmul_rn(2.0f, cat.rsub[i0]);
  o.status[slot] = 0;
}

// Members of the sphere r around the centre (count only).
__global__ void __launch_bounds__(HB)
k_sphere_count(ColIdx ci, const int32_t* __restrict__ act, const float* __restrict__ hcx,
               const float* __restrict__ hcy, const float* __restrict__ hcz, const float* __restrict__ r,
               int32_t* __restrict__ konta) {
  __shared__ long long lred[32];
  __shared__ QBuf qb;
  int s = act[blockIdx.x];
  float cx = hcx[s], cy = hcy[s], cz = hcz[s], rr = r[s];
  int64_t lo, hi;
  slab_range(ci, cx, rr, &lo, &hi);
  long long c = 0;
  gquery_box(Grp<1>(), ci, cx, cy, cz, rr, qb, [&](const float4& e) {
    int p = ppos(e);
    if (p >= lo && p < hi && dist3(e.x, e.y, e.z, cx, cy, cz) < rr) c++;
  });
  c = block_sum_ll(c, lred);
  if (threadIdx.x == 0) konta[blockIdx.x] = (int32_t)c;
}

__device__ __forceinline__ double eq_jacobi_dev(double basx, double basy) {
  double t = __dsub_rn(1.0, basx);
  return __dadd_rn(__dsub_rn(__dsub_rn(__ddiv_rn(1.0, __dmul_rn(t, t)), 1.0), __ddiv_rn(basy, __dmul_rn(basx, basx))),
                   __dmul_rn(__dadd_rn(1.0, basy), basx));
}

struct JacOut {
  int32_t* done;      // 1: radius fixed
  int32_t* jjac;      // J_JACOBI
  double* masadm;
  float* rclus;       // RCLUS = DISTA(J_JACOBI)
};

// Jacobi radius on the sorted members (substructure.f:1016-1112).  Slot s of
// the active list; segment [off[b], off[b]+konta[b]).
template <int C>
__global__ void __launch_bounds__(HB)
k_sub_jacobi(const int32_t* __restrict__ slots, Store S, HConst H, const int32_t* __restrict__ act,
             const int32_t* __restrict__ konta,
             const int64_t* __restrict__ off, const unsigned long long* __restrict__ keys,
             const int32_t* __restrict__ vals, const float* __restrict__ mhost_a,
             const float* __restrict__ disthost_a, float* __restrict__ r, JacOut o) {
  static_assert(C == 1, "one CTA per subhalo");
  __shared__ MainShared sh;
  __shared__ double s_m[4];
  int b = slots[blockIdx.x], s = act[b];
  int64_t K = konta[b];
  const unsigned long long* kk = keys + off[b];
  const int32_t* lip = vals + off[b];
  double um = (double)H.um;
  float mhost = mhost_a[s], disthost = disthost_a[s];
  auto dista = [&](int64_t J) -> float {  // DISTA(J), 1-based; 1e10 past the members
    return (J >= 1 && J <= K) ? __uint_as_float((uint32_t)(kk[J - 1] & 0xffffffffull)) : 1.e10f;
  };
  int64_t minj = max((int64_t)10, K / 50);
  double mh3 = (double)__fmul_rn(3.0f, mhost);
  double expo = (double)(1.0f / 3.0f);
  // estimation: first J > MINJ with r/D - (m/(m+3M))^(1/3) > 0
  long long jest = LLONG_MAX;
  tile_prefix_d(0, K, 0.0, [&](int64_t j) { return (double)S.mass(lip[j]); },
                [&](int64_t j, double mas) {
                  int64_t J = j + 1;
                  if (J <= minj) return;
                  double mu = mas * um;
                  double eq = (double)__fdiv_rn(dista(J), disthost) - pow(mu / (mu + mh3), expo);
                  if (eq > 0.0 && J < jest) jest = J;
                },
                sh.dred);
  jest = bmin(jest, sh);
  int64_t jj = jest == LLONG_MAX ? K : jest;
  // masses at jj and prefix lookups
  double mjj = 0.0;
  if (threadIdx.x == 0) s_m[0] = 0.0;
  __syncthreads();
  tile_prefix_d(0, K, 0.0, [&](int64_t j) { return (double)S.mass(lip[j]); },
                [&](int64_t j, double mas) { if (j + 1 == jj) s_m[0] = mas; }, sh.dred);
  __syncthreads();
  mjj = s_m[0];
  double basx = (double)__fdiv_rn(dista(jj), disthost);
  double basy = mjj * um / (double)mhost;
  double eq = eq_jacobi_dev(basx, basy);
  int flag = 0, dir = -1;
  long long jfound = LLONG_MAX;
  double masadm = mjj;
  // ABS(EQ_JACOBI_R).LT.0.D01 compares with 0.0D+01 = 0: never true
  if (eq < 0.0) {
    dir = 1;  // forward: first J > jj with EQ > 0
    long long f = LLONG_MAX;
    tile_prefix_d(0, K, 0.0, [&](int64_t j) { return (double)S.mass(lip[j]); },
                  [&](int64_t j, double mas) {
                    int64_t J = j + 1;
                    if (J <= jj) return;
                    double bx = (double)__fdiv_rn(dista(J), disthost);
                    double e2 = eq_jacobi_dev(bx, mas * um / (double)mhost);
                    if (e2 > 0.0 && J < f) f = J;
                  },
                  sh.dred);
    f = bmin(f, sh);
    if (f != LLONG_MAX) { flag = 1; jfound = f; }
  } else {
    // backward: largest J in [MINJ, jj-1] with EQ(prefix(J)) < 0
    long long f = -1;
    tile_prefix_d(0, K, 0.0, [&](int64_t j) { return (double)S.mass(lip[j]); },
                  [&](int64_t j, double mas) {
                    int64_t J = j + 1;
                    if (J < minj || J > jj - 1) return;
                    double bx = (double)__fdiv_rn(dista(J), disthost);
                    double e2 = eq_jacobi_dev(bx, mas * um / (double)mhost);
                    if (e2 < 0.0 && J > f) f = J;
                  },
                  sh.dred);
    f = -bmin(-f, sh);  // max (-1: none)
    if (f > 0) { flag = 1; jfound = f; }
  }
  int64_t jj2 = jj;
  if (flag) {
    jj2 = jfound;
  } else if (dir == -1) {
    jj2 = minj;
    flag = 1;
  }
  if (flag) {
    // MASADM at the final J: prefix(J) (forward and backward searches) or,
    // when the backward loop ran out, prefix(MINJ); a zero-trip backward
    // loop keeps prefix(jj)
    if (threadIdx.x == 0) s_m[1] = 0.0;
    __syncthreads();
    int64_t jm = jj2;
    if (dir == -1 && jfound == LLONG_MAX && jj - 1 < minj) jm = jj;
    tile_prefix_d(0, K, 0.0, [&](int64_t j) { return (double)S.mass(lip[j]); },
                  [&](int64_t j, double mas) { if (j + 1 == jm) s_m[1] = mas; }, sh.dred);
    __syncthreads();
    masadm = (jm >= 1 && jm <= K) ? s_m[1] : (jm > K ? mjj : 0.0);
  }
  if (threadIdx.x == 0) {
    o.done[b] = flag;
    if (flag) {
      o.jjac[b] = (int32_t)jj2;
      o.masadm[b] = masadm;
      o.rclus[b] = dista(jj2);
    } else {
      r[s] = __fmul_rn(1.5f, r[s]);
    }
  }
}

struct SubMainIn {
  const int32_t* konta;   // gathered members
  const int32_t* jjac;    // members kept (J_JACOBI)
  const double* masadm;
  const float* rclus;
  const float *cx, *cy, *cz, *mhost, *disthost;
};

// Work list of a substructure level: REALCLUS != 0, largest RSUB first.
// ---------------------------------------------------------------- subhalo main (staged)
// The members kept by the Jacobi search, staged like the halo lists; the
// subhalo list is the radially sorted list sorted a second time, which
// reverses each run of equal distances (substructure.f:1161-1162): the
// staging reads entry j from the mirror of j inside its run.
template <int C>
__device__ void load_segment_rev(const Grp<C>& g, const Store& S, const unsigned long long* keys,
                                 const int32_t* vals, int64_t K, const SegView& a, const SegView& b,
                                 uint8_t* flag) {
  int64_t lo, hi;
  g.chunk(0, K, &lo, &hi);
  for (int64_t j = lo + threadIdx.x; j < hi; j += blockDim.x) {
    const unsigned long long kj = keys[j];
    int64_t rs = j, re = j + 1;
    while (rs > 0 && keys[rs - 1] == kj) rs--;
    while (re < K && keys[re] == kj) re++;
    const int p = vals[rs + re - 1 - j];
    float4 r0, r1;
    if (S.rows) {
      r0 = S.rows[2 * (int64_t)p];
      r1 = S.rows[2 * (int64_t)p + 1];
    } else {
      r0 = make_float4(S.x[p], S.y[p], S.z[p], S.m[p]);
      r1 = make_float4(S.vx[p], S.vy[p], S.vz[p], 0.f);
    }
    a.dm[j] = make_float2(__uint_as_float((uint32_t)(kj & 0xffffffffull)), r0.w);
    a.mv[j] = make_float4(r0.w, r1.x, r1.y, r1.z);
    a.px[j] = make_float4(r0.x, r0.y, r0.z, __int_as_float(p));
    flag[j] = 1;
  }
  if (g.rank() == 0 && threadIdx.x == 0) {  // DISTA(KONTA+1) of the sorted list
    a.dm[K] = make_float2(1.e10f, 0.f); b.dm[K] = a.dm[K];
    a.mv[K] = make_float4(0.f, 0.f, 0.f, 0.f); b.mv[K] = a.mv[K];
    a.px[K] = make_float4(0.f, 0.f, 0.f, 0.f); b.px[K] = a.px[K];
  }
  g.sync();
}

// SUBSTRUCTURE_PARTICLES after the Jacobi radius (substructure.f:1115-1660):
// unbinding, Jacobi trim, SO walk without early exit, properties.
template <int C>
__global__ void __launch_bounds__(HB, 3)
k_sub_main_g(const int32_t* __restrict__ slots, Store S, HConst H, asohf_catalogue cat,
             const int32_t* __restrict__ work, SubMainIn in, SegG sg) {
  __shared__ GShared sh;
  Grp<C> g;
  const int slot = group_slot<C>(slots);
  const bool lead = leader(g.rank());
  const int i0 = work[slot];
  if (lead) { sg.nbound[slot] = 0; sg.nscan[slot] = 0; sg.final_b[slot] = 0; }
  const int64_t Kg = in.konta[slot];
  const int64_t konta = in.jjac[slot];
  const double masadm = in.masadm[slot];
  const float um = H.um;
  if (masadm <= 0.0 || konta < H.min_num_part || konta > Kg) {
    // RSUB/MSUB were set when the Jacobi radius was fixed (substructure.f:1115-1117)
    if (lead) {
      cat.rsub[i0] = in.rclus[slot];
      cat.msub[i0] = (float)(masadm * (double)um);
      cat.realclus[i0] = 0;
      sg.status[slot] = 0;
    }
    return;
  }
  const int64_t base = sg.off[slot] + slot;
  SegView va = view_at(sg.a, base), vb = view_at(sg.b, base);
  double* pot = sg.pot + base;
  uint8_t* flag = sg.flag + base;
  const float cx = in.cx[slot], cy = in.cy[slot], cz = in.cz[slot];
  const float mhost = in.mhost[slot], disthost = in.disthost[slot];
  load_segment_rev(g, S, sg.keys + sg.off[slot], sg.vals + sg.off[slot], konta, va, vb, flag);
  SegView cur = va, nxt = vb;
  int which = 0;
  float cm0[3], v0[3], m2;
  centromasas_g(g, cur, konta, cm0, v0, &m2, sh);
  HaloState h;
  for (int q = 0; q < 3; q++) { h.cm[q] = cm0[q]; h.v[q] = v0[q]; }
  h.radio = in.rclus[slot];                 // RSUB
  h.masa = (float)(masadm * (double)um);    // MSUB
  h.realclus = cat.realclus[i0];
  unsigned long long ep = 2ull * (unsigned long long)konta;
  int64_t k2 = konta;
  float ref_max = cur.dm[k2 - 1].x;
  const float norma = S.norma;
  auto write_back = [&]() {
    if (lead) {
      cat.clusrxcm[i0] = h.cm[0]; cat.clusrycm[i0] = h.cm[1]; cat.clusrzcm[i0] = h.cm[2];
      cat.vx[i0] = h.v[0]; cat.vy[i0] = h.v[1]; cat.vz[i0] = h.v[2];
      cat.rsub[i0] = h.radio; cat.msub[i0] = h.masa;
      cat.dmpclus[i0] = (int32_t)konta;
    }
  };
  auto finish_empty = [&]() {
    write_back();
    if (lead) {
      cat.realclus[i0] = 0;
      sg.final_b[slot] = (uint8_t)which;
      sg.status[slot] = 0;
    }
  };
  // escape-velocity unbinding with IDX_VIR = K2 (substructure.f:1172-1190)
  int64_t contaerr = konta;
  int fac = 0;
  PotCache pc;
  while (contaerr > 0 || fac < 3) {
    fac++;
    int64_t prev = k2, iv = k2;
    ep += (unsigned long long)k2;
    long long kept = unbinding8_g(g, norma, H, fac, ref_max, cur, flag, pot, k2, iv, h, sh, pc);
    if (kept != k2) {
      int64_t nk2;
      compact_g(g, cur, nxt, flag, k2, &iv, &nk2, sh);
      SegView t = cur; cur = nxt; nxt = t; which ^= 1;
      k2 = nk2;
      pc.valid = pc.flags_valid = false;
    }
    ref_max = k2 > 0 ? cur.dm[k2 - 1].x : 1.e10f;
    contaerr = prev - k2;
    if (fac > 100000) break;
  }
  if (k2 < H.min_num_part) { finish_empty(); return; }
  fac = 0;
  contaerr = k2;
  SigCache sc;
  while (contaerr > 0 || fac < 4) {
    fac++;
    int64_t prev = k2, iv = k2;
    ep += (unsigned long long)k2;
    long long kept = unbinding_sigma_g(g, H, fac, cur, flag, k2, iv, h, sh, sc);
    if (kept != k2) {
      int64_t nk2;
      compact_g(g, cur, nxt, flag, k2, &iv, &nk2, sh);
      SegView t = cur; cur = nxt; nxt = t; which ^= 1;
      k2 = nk2;
      sc.valid = sc.flags_valid = false;
    }
    ref_max = k2 > 0 ? cur.dm[k2 - 1].x : 1.e10f;
    contaerr = prev - k2;
    if (fac > 100000) break;
  }
  if (k2 < H.min_num_part) { finish_empty(); return; }
  // Jacobi trim after unbinding (substructure.f:1241-1264)
  int64_t ncapas = 0;
  float rshell = 0.0f;
  {
    const double m0 = (double)__fdiv_rn(h.masa, um);
    const double bx = (double)__fdiv_rn(cur.dm[k2 - 1].x, disthost);
    const double e0 = eq_jacobi_dev(bx, m0 * (double)um / (double)mhost);
    if (e0 > 0.0) {
      // M(J) = MASADM - sum_{i >= J} m_i ; largest J in [1, k2] with EQ < 0
      double tot = 0.0;
      {
        int64_t lo, hi;
        g.chunk(0, k2, &lo, &hi);
        for (int64_t j = lo + threadIdx.x; j < hi; j += blockDim.x) tot += (double)cur.dm[j].y;
        gsum_dv<1>(g, &tot, sh.x);
      }
      long long f = -1;
      double mf = 0.0;
      gscan_d(g, 0, k2, 0.0, [&](int64_t j) { return (double)cur.dm[j].y; },
              [&](int64_t j, double pre) {
                const int64_t J = j + 1;
                const double mj = m0 - (tot - pre + (double)cur.dm[j].y);  // after subtracting m(J..K2)
                const double bxj = (double)__fdiv_rn(cur.dm[j].x, disthost);
                const double e2 = eq_jacobi_dev(bxj, mj * (double)um / (double)mhost);
                if (e2 < 0.0 && J > f) { f = J; mf = mj; }
              },
              sh.wsum, sh.x);
      long long nf = f > 0 ? -f : LLONG_MAX;
      gmin_llv<1>(g, &nf, sh.lred, sh.x);
      const long long fmax = nf == LLONG_MAX ? -1 : -nf;
      double mfv = (f == fmax && f > 0) ? mf : 0.0;  // one entry holds it
      gsum_dv<1>(g, &mfv, sh.x);
      int64_t J;
      double mj;
      if (fmax <= 0) {
        J = 0;
        mj = m0 - tot;
      } else {
        J = fmax;
        mj = mfv;
      }
      h.radio = J + 1 <= k2 ? cur.dm[J].x : (J + 1 == k2 + 1 ? cur.dm[k2].x : 1.e10f);
      h.masa = (float)(mj * (double)um);
      k2 = J;
      ncapas = J;
      rshell = J >= 1 ? cur.dm[J - 1].x : 1.e10f;
    }
  }
  if (k2 < H.min_num_part) { finish_empty(); return; }
  // SO walk without early exit (substructure.f:1293-1463)
  const float pi = H.pi, rote = H.rote, rete = H.rete;
  const int64_t jjcore = (int64_t)fmaxf(10.0f, __fdiv_rn((float)k2, 100.0f));
  const float thr[6] = {__fdiv_rn(2500.0f, H.omegaz), __fdiv_rn(500.0f, H.omegaz), __fdiv_rn(200.0f, H.omegaz),
                        2500.0f, 500.0f, 200.0f};
  const int64_t jvir_min = (int64_t)__fmul_rn(0.1f, (float)k2);
  long long jt[7];
  for (int q = 0; q < 7; q++) jt[q] = LLONG_MAX;
  double best_v = -1.0;
  long long best_j = LLONG_MAX;
  double best_b = 0.0;
  auto mn_of = [&](int64_t j) { return (double)__fdiv_rn(cur.dm[j].y, norma); };
  const double btot = gscan_d(g, 0, k2, 0.0, mn_of,
                              [&](int64_t j, double bas8) {
                                const int64_t J = j + 1;
                                if (J <= jjcore) return;
                                const float d = cur.dm[j].x;
                                const float vol = so_den(d, rete, pi);
                                const float delta2 = (float)((double)norma * bas8 / (double)vol / (double)rote);
                                for (int q = 0; q < 6; q++)
                                  if (delta2 <= thr[q] && J < jt[q]) jt[q] = J;
                                if (delta2 <= H.contrastec && J > jvir_min && J < jt[6]) jt[6] = J;
                                const float bas2 = (float)(bas8 / (double)d);
                                if (best_before((double)bas2, J, best_v, best_j)) {
                                  best_v = bas2; best_j = J; best_b = bas8;
                                }
                              },
                              sh.wsum, sh.x);
  gmin_llv<7>(g, jt, sh.lred, sh.x);
  // BAS8 at the crossings and the momentum sums, in one more pass
  double sv[10];
  for (int q = 0; q < 10; q++) sv[q] = 0.0;
  gscan_d(g, 0, k2, 0.0, mn_of,
          [&](int64_t j, double bas8) {
            for (int q = 0; q < 7; q++)
              if (j + 1 == jt[q]) sv[q] = bas8;
            const float4 qv = cur.mv[j];
            const float mn = __fdiv_rn(qv.x, norma);
            sv[7] += (double)__fmul_rn(mn, qv.y);
            sv[8] += (double)__fmul_rn(mn, qv.z);
            sv[9] += (double)__fmul_rn(mn, qv.w);
          },
          sh.wsum, sh.x);
  gsum_dv<10>(g, sv, sh.x);
  gbest(g, &best_v, &best_j, &best_b, sh);
  if (lead) {
    if (best_j != LLONG_MAX) {
      cat.vcmax[i0] = (float)best_v;
      cat.mcmax[i0] = (float)best_b;
      cat.rcmax[i0] = cur.dm[best_j - 1].x;
    }
    float* mo[6] = {cat.m2500c, cat.m500c, cat.m200c, cat.m2500m, cat.m500m, cat.m200m};
    float* ro[6] = {cat.r2500c, cat.r500c, cat.r200c, cat.r2500m, cat.r500m, cat.r200m};
    for (int q = 0; q < 6; q++) {
      if (jt[q] != LLONG_MAX) {
        const int64_t J = jt[q];
        const float d = cur.dm[J - 1].x;
        const float vol = so_den(d, rete, pi);
        const float delta2 = (float)((double)norma * sv[q] / (double)vol / (double)rote);
        mo[q][i0] = __fmul_rn(__fmul_rn(__fmul_rn(delta2, vol), rote), um);
        ro[q][i0] = d;
        if (J == jjcore + 1) { mo[q][i0] = -1.0f; ro[q][i0] = -1.0f; }
      } else {
        mo[q][i0] = 0.0f;
        ro[q][i0] = 0.0f;
      }
    }
    if (jt[6] != LLONG_MAX) {
      const int64_t J = jt[6];
      const float d = cur.dm[J - 1].x;
      const float vol = so_den(d, rete, pi);
      const float delta2 = (float)((double)norma * sv[6] / (double)vol / (double)rote);
      cat.masa[i0] = __fmul_rn(__fmul_rn(__fmul_rn(delta2, vol), rote), um);
      cat.radio[i0] = d;
    } else {
      cat.masa[i0] = 0.0f;
      cat.radio[i0] = 0.0f;
    }
    h.v[0] = (float)(sv[7] / btot);
    h.v[1] = (float)(sv[8] / btot);
    h.v[2] = (float)(sv[9] / btot);
    const float bas = __fdiv_rn(__fmul_rn(__fmul_rn(cat.vcmax[i0], norma), H.cgr), rete);
    cat.vcmax[i0] = __fmul_rn(__fsqrt_rn(bas), H.uv);
    cat.mcmax[i0] = __fmul_rn(__fmul_rn(cat.mcmax[i0], norma), um);
    sg.final_b[slot] = (uint8_t)which;
  }
  // the velocity the leader computed reaches every CTA through the catalogue
  // (the properties read VX(I) from it, as the Fortran does)
  write_back();
  g.sync();
  int unsup = 0;
  long long nb = properties_g<C, false>(g, S, H, cat, i0, cur, flag, ncapas, rshell, cx, cy, cz, cm0, sh, &unsup,
                                        nxt, pot, sg.eig + (size_t)slot * 9);
  ep += (unsigned long long)(k2 + ncapas);
  if (lead) {
    atomicAdd(&sg.work[1], ep);
    const bool ok = nb >= H.min_num_part && H.want_ids;
    sg.nbound[slot] = ok ? (int32_t)nb : 0;
    sg.nscan[slot] = ok ? (int32_t)ncapas : 0;
    sg.status[slot] = unsup == 1 ? ASOHF_ERR_UNSUPPORTED : unsup == 2 ? ASOHF_ERR_TIMEOUT : 0;
  }
}

static int make_sub_work(asohf_ctx* c, CatMirror& m, int low1, int low2, std::vector<int32_t>& h_work,
                         int* nslots) {
  int nh = low2 - low1 + 1;
  std::vector<int32_t> rc_v((size_t)nh);
  int32_t* rc = rc_v.data();
  std::vector<float> rs_v((size_t)nh);
  float* rs = rs_v.data();
  ASOHF_CUDA(cudaMemcpyAsync(rc, m.d.realclus + low1 - 1, 4 * (size_t)nh, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(rs, m.d.rsub + low1 - 1, 4 * (size_t)nh, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  h_work.assign(nh > 0 ? nh : 1, 0);
  int32_t* w = h_work.data();
  int k = 0;
  for (int i = 0; i < nh; i++)
    if (rc[i] != 0) w[k++] = low1 - 1 + i;
  // sort by RSUB descending (stable): the float's bits mapped to an unsigned
  // key of the same order, -0 taken as +0 (they compare equal)
  std::vector<uint32_t> key((size_t)(k > 0 ? k : 1));
  for (int i = 0; i < k; i++) {
    const float v = rs[w[i] - (low1 - 1)];
    uint32_t b = 0u;
    if (v != 0.0f) memcpy(&b, &v, 4);
    key[i] = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  }
  stable_desc(key, w, k);
  *nslots = k;
  return ASOHF_OK;
}

// gather + segmented sort of the members of `na` spheres (active list act);
// keys/vals sorted in segments at offsets off (device).
// Counts, tiers (by count) of the spheres, gathers into segments and sorts
// them; d_tslots and d_fill hold na entries.
static int gather_sorted(asohf_ctx* c, const Store& S, const ColIdx& ci, int na, const int32_t* d_act,
                         const float* cx, const float* cy, const float* cz, const float* r,
                         int32_t* d_konta, int64_t* d_off, int64_t* h_off, unsigned long long** keys,
                         int32_t** vals, int64_t* total, bool with_work, Tiers* tiers, int32_t* d_tslots,
                         int32_t* d_fill) {
  {
    int kt_ = ktime_begin(c, "sub_sphere_count");
    k_sphere_count<<<na, HB, 0, c->stream>>>(ci, d_act, cx, cy, cz, r, d_konta);
    ktime_end(c, kt_);
  }
  c->launches++;
  std::vector<int32_t> hk_v((size_t)na);
  int32_t* hk = hk_v.data();
  ASOHF_CUDA(cudaMemcpyAsync(hk, d_konta, 4 * (size_t)na, cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  h_off[0] = 0;
  for (int s = 0; s < na; s++) h_off[s + 1] = h_off[s] + hk[s];
  // few subhaloes per call, each in a dense region: 256-thread CTAs (tier 2)
  // keep more of the GPU busy than the small tiers
  for (int s = 0; s < na; s++) hk[s] = 0;
  int64_t keep_t1 = c->tier1_k, keep_t2 = c->tier2_k;
  c->tier1_k = 0;
  c->tier2_k = 0;
  int rt = split_tiers(c, hk, na, d_tslots, tiers);
  c->tier1_k = keep_t1;
  c->tier2_k = keep_t2;
  ASOHF_CHECK(rt);
  int64_t T = h_off[na];
  ASOHF_CUDA(cudaMemcpyAsync(d_off, h_off, 8 * (size_t)(na + 1), cudaMemcpyHostToDevice, c->stream));
  int bits = 1;
  while ((1ll << bits) < na) bits++;
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                  (int32_t*)nullptr, (int32_t*)nullptr, (int)(T > 0 ? T : 1), 0, 32 + bits);
  size_t work = with_work ? ((size_t)T + na) * (2 * (8 + 16 + 16) + 8 + 1) + 16384 : 0;
  ASOHF_CHECK(seg_reserve(c, (size_t)T * 24 + tb + work + 16384));
  unsigned long long* k0 = (unsigned long long*)seg_alloc(c, 8 * (size_t)T + 8);
  unsigned long long* k1 = (unsigned long long*)seg_alloc(c, 8 * (size_t)T + 8);
  int32_t* v0 = (int32_t*)seg_alloc(c, 4 * (size_t)T + 4);
  int32_t* v1 = (int32_t*)seg_alloc(c, 4 * (size_t)T + 4);
  void* t = seg_alloc(c, tb);
  if (!k0 || !k1 || !v0 || !v1 || !t) return ASOHF_ERR_CAPACITY;
  if (T > 0) {
    // the per-sphere arrays are indexed by position in the active list
    ASOHF_CUDA(cudaMemsetAsync(d_fill, 0, 4 * (size_t)na, c->stream));
    {
      int kt_ = ktime_begin(c, "sub_gather");
      LAUNCH_TIERS_CTA(k_halo_gather, *tiers, S, ci, d_konta, d_off, cx, cy, cz, r, d_fill, k0, v0);
      ktime_end(c, kt_);
    }
    int kt_ = ktime_begin(c, "sub_radix_sort");
    ASOHF_CUDA(cub::DeviceRadixSort::SortPairs(t, tb, k0, k1, v0, v1, (int)T, 0, 32 + bits, c->stream));
    ktime_end(c, kt_);
    k_tiefix<<<grid_for(T, 256), 256, 0, c->stream>>>(k1, v1, T, 1);
    c->launches++;
  }
  *keys = k1;
  *vals = v1;
  *total = T;
  return ASOHF_OK;
}

__global__ void k_jacobi_scatter(const int32_t* __restrict__ act, int na, JacOut o, const float* __restrict__ rlast,
                                 int32_t* __restrict__ f_jjac, double* __restrict__ f_masadm,
                                 float* __restrict__ f_rclus, float* __restrict__ f_rlast) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= na || !o.done[b]) return;
  int s = act[b];
  f_jjac[s] = o.jjac[b];
  f_masadm[s] = o.masadm[b];
  f_rclus[s] = o.rclus[b];
  f_rlast[s] = rlast[b];
}

__global__ void k_iota32(int32_t* __restrict__ a, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

__global__ void k_gather_f(const int32_t* __restrict__ act, int na, const float* __restrict__ src, float* __restrict__ dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < na) dst[i] = src[act[i]];
}

// Copies segment b of (keys, vals) at off[b] (cnt[b] entries) to dst[b] of
// (dk, dv); dst[b] < 0: not copied.  One CTA per segment.
__global__ void k_copy_segments(const unsigned long long* __restrict__ keys, const int32_t* __restrict__ vals,
                                const int64_t* __restrict__ off, const int32_t* __restrict__ cnt,
                                const int64_t* __restrict__ dst, unsigned long long* __restrict__ dk,
                                int32_t* __restrict__ dv) {
  const int b = blockIdx.x;
  const int64_t d = dst[b];
  if (d < 0) return;
  const int64_t o = off[b], n = cnt[b];
  for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
    dk[d + j] = keys[o + j];
    dv[d + j] = vals[o + j];
  }
}

// Room for n entries in the store of fixed segments, keeping the first
// `keep` entries.
static int sfin_reserve(asohf_ctx* c, int64_t n, int64_t keep) {
  if (n <= c->sfin_cap) return ASOHF_OK;
  const int64_t cap = n + n / 2 + 4096;
  unsigned long long* nk = nullptr;
  int32_t* nv = nullptr;
  ASOHF_CUDA(cudaMalloc(&nk, 8 * (size_t)cap));
  if (cudaMalloc(&nv, 4 * (size_t)cap) != cudaSuccess) {
    cudaFree(nk);
    return ASOHF_ERR_CUDA;
  }
  if (keep > 0) {
    ASOHF_CUDA(cudaMemcpyAsync(nk, c->sfin_k, 8 * (size_t)keep, cudaMemcpyDeviceToDevice, c->stream));
    ASOHF_CUDA(cudaMemcpyAsync(nv, c->sfin_v, 4 * (size_t)keep, cudaMemcpyDeviceToDevice, c->stream));
  }
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(c->sfin_k);
  cudaFree(c->sfin_v);
  c->sfin_k = nk;
  c->sfin_v = nv;
  c->sfin_cap = cap;
  return ASOHF_OK;
}

extern "C" int asohf_substructure_particles(asohf_ctx* c, const asohf_consts* k, const asohf_mesh* mesh,
                                            asohf_catalogue* cat, int ir, const int32_t* subs_lev,
                                            int on_device) {
  if (!c || !k || !cat || !subs_lev || !mesh || ir < 1 || ir > mesh->nl) return ASOHF_ERR_INVALID;
  if (c->nx_sorted != k->nx) return ASOHF_ERR_INVALID;
  int lowh1 = 1, lowh2 = 0;
  for (int q = 0; q < ir; q++) lowh1 += subs_lev[q];
  for (int q = 0; q <= ir; q++) lowh2 += subs_lev[q];
  if (lowh2 > cat->nclus) return ASOHF_ERR_INVALID;
  if (lowh2 < lowh1) return ASOHF_OK;
  ASOHF_CUDA(cudaSetDevice(c->device));
  double ht = htime_now();
  arena_reset(c);
  int nh = lowh2 - lowh1 + 1;
  size_t need = cat_bytes(cat->nclus) + (size_t)nh * (192 + 40) + 65536;
  ASOHF_CHECK(arena_reserve(c, need));
  CatMirror m;
  ASOHF_CHECK(cat_mirror_in(c, cat, cat->nclus, on_device, &m, lowh1 - 1, true));
  std::vector<int32_t> hw_v;
  int ns;
  ASOHF_CHECK(make_sub_work(c, m, lowh1, lowh2, hw_v, &ns));
  int32_t* hw = hw_v.data();
  htime_end(c, "host:sub_mirror_in+work", ht);
  ht = htime_now();
  Store S = store_of(c);
  ColIdx ci = col_idx(c, k);
  HConst H = hconst(k, mesh);
  H.epot_seed = c->epot_seed;
  int rc = ASOHF_OK;
  if (ns > 0) {
    int32_t* d_work = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    SubPrep pr;
    pr.cx = (float*)arena_alloc(c, 4 * (size_t)ns); pr.cy = (float*)arena_alloc(c, 4 * (size_t)ns);
    pr.cz = (float*)arena_alloc(c, 4 * (size_t)ns); pr.mhost = (float*)arena_alloc(c, 4 * (size_t)ns);
    pr.disthost = (float*)arena_alloc(c, 4 * (size_t)ns); pr.r = (float*)arena_alloc(c, 4 * (size_t)ns);
    pr.status = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    int32_t* d_act = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    int32_t* d_konta = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    int64_t* d_off = (int64_t*)arena_alloc(c, 8 * (size_t)(ns + 1));
    float* t_cx = (float*)arena_alloc(c, 4 * (size_t)ns); float* t_cy = (float*)arena_alloc(c, 4 * (size_t)ns);
    float* t_cz = (float*)arena_alloc(c, 4 * (size_t)ns); float* t_r = (float*)arena_alloc(c, 4 * (size_t)ns);
    JacOut jo;
    jo.done = (int32_t*)arena_alloc(c, 4 * (size_t)ns); jo.jjac = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    jo.masadm = (double*)arena_alloc(c, 8 * (size_t)ns); jo.rclus = (float*)arena_alloc(c, 4 * (size_t)ns);
    int32_t* f_jjac = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    double* f_masadm = (double*)arena_alloc(c, 8 * (size_t)ns);
    float* f_rclus = (float*)arena_alloc(c, 4 * (size_t)ns);
    float* f_rlast = (float*)arena_alloc(c, 4 * (size_t)ns);
    int32_t* d_nbound = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    int32_t* d_nscan = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    int64_t* d_ids_off = (int64_t*)arena_alloc(c, 8 * (size_t)ns);
    std::vector<int64_t> h_off_v((size_t)(ns + 1));
    int64_t* h_off = h_off_v.data();
    std::vector<int32_t> h_act_v((size_t)ns);
    int32_t* h_act = h_act_v.data();
    std::vector<int32_t> h_done_v((size_t)ns);
    int32_t* h_done = h_done_v.data();
    std::vector<int32_t> h_st_v((size_t)ns);
    int32_t* h_st = h_st_v.data();
    if (!d_work || !pr.cx || !pr.status || !d_act || !d_konta || !d_off || !t_r || !jo.done || !jo.rclus ||
        !f_jjac || !f_masadm || !f_rclus || !f_rlast || !d_nbound || !d_nscan || !d_ids_off) {
      return ASOHF_ERR_CAPACITY;
    }
    ASOHF_CUDA(cudaMemcpyAsync(d_work, hw, 4 * (size_t)ns, cudaMemcpyHostToDevice, c->stream));
    {
      int kt_ = ktime_begin(c, "sub_prep");
      k_sub_prep<<<ns, HB, 0, c->stream>>>(S, ci, H, m.d, d_work, pr);
      ktime_end(c, kt_);
    }
    c->launches++;
    ASOHF_CUDA(cudaMemcpyAsync(h_st, pr.status, 4 * (size_t)ns, cudaMemcpyDeviceToHost, c->stream));
    ASOHF_CUDA(cudaStreamSynchronize(c->stream));
    int na = 0;
    for (int s = 0; s < ns; s++) {
      if (h_st[s]) rc = h_st[s];
      else h_act[na++] = s;
    }
    htime_end(c, "host:sub_prep", ht);
    ht = htime_now();
    // Jacobi radius, growing the unresolved ones
    int32_t* d_pos = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    int32_t* d_tsl = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    int32_t* d_fill = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
    if (!d_pos || !d_tsl || !d_fill) rc = ASOHF_ERR_CAPACITY;
    else k_iota32<<<(ns + 255) / 256, 256, 0, c->stream>>>(d_pos, ns);
    std::vector<int64_t> fin_off((size_t)ns, 0), fin_cnt((size_t)ns, 0), h_dst((size_t)ns, -1);
    int64_t fin_total = 0;
    for (int iter = 0; na > 0 && rc == ASOHF_OK; iter++) {
      if (iter > 200) { rc = ASOHF_ERR_TIMEOUT; break; }
      ASOHF_CUDA(cudaMemcpyAsync(d_act, h_act, 4 * (size_t)na, cudaMemcpyHostToDevice, c->stream));
      {
        int kt_ = ktime_begin(c, "sub_jacobi_prep");
        k_gather_f<<<(na + 255) / 256, 256, 0, c->stream>>>(d_act, na, pr.cx, t_cx);
        k_gather_f<<<(na + 255) / 256, 256, 0, c->stream>>>(d_act, na, pr.cy, t_cy);
        k_gather_f<<<(na + 255) / 256, 256, 0, c->stream>>>(d_act, na, pr.cz, t_cz);
        k_gather_f<<<(na + 255) / 256, 256, 0, c->stream>>>(d_act, na, pr.r, t_r);
        ktime_end(c, kt_);
      }
      c->launches += 4;
      unsigned long long* keys;
      int32_t* vals;
      int64_t T;
      Tiers tj;
      ASOHF_CHECK(gather_sorted(c, S, ci, na, d_pos, t_cx, t_cy, t_cz, t_r, d_konta, d_off, h_off, &keys, &vals,
                                &T, false, &tj, d_tsl, d_fill));
      {
        int kt_ = ktime_begin(c, "sub_jacobi");
        LAUNCH_TIERS_CTA(k_sub_jacobi, tj, S, H, d_act, d_konta, d_off, keys, vals, pr.mhost, pr.disthost, pr.r,
                         jo);
        ktime_end(c, kt_);
      }
      {
        int kt_ = ktime_begin(c, "sub_jacobi_scatter");
        k_jacobi_scatter<<<(na + 255) / 256, 256, 0, c->stream>>>(d_act, na, jo, t_r, f_jjac, f_masadm, f_rclus,
                                                                  f_rlast);
        ktime_end(c, kt_);
      }
      c->launches++;
      ASOHF_CUDA(cudaGetLastError());
      ASOHF_CUDA(cudaMemcpyAsync(h_done, jo.done, 4 * (size_t)na, cudaMemcpyDeviceToHost, c->stream));
      ASOHF_CUDA(cudaStreamSynchronize(c->stream));
      // the members of the subhaloes fixed in this round, gathered at their
      // final radius, are kept: the main pass reads them from there
      int64_t fin0 = fin_total;
      for (int q = 0; q < na; q++) {
        h_dst[q] = -1;
        if (h_done[q]) {
          const int s = h_act[q];
          fin_off[s] = fin_total;
          fin_cnt[s] = h_off[q + 1] - h_off[q];
          h_dst[q] = fin_total;
          fin_total += fin_cnt[s];
        }
      }
      if (fin_total > fin0) {
        ASOHF_CHECK(sfin_reserve(c, fin_total, fin0));
        ASOHF_CUDA(cudaMemcpyAsync(d_ids_off, h_dst.data(), 8 * (size_t)na, cudaMemcpyHostToDevice, c->stream));
        int kt_ = ktime_begin(c, "sub_keep_segments");
        k_copy_segments<<<na, 256, 0, c->stream>>>(keys, vals, d_off, d_konta, d_ids_off, c->sfin_k, c->sfin_v);
        ktime_end(c, kt_);
        c->launches++;
        ASOHF_CUDA(cudaGetLastError());
      }
      int nn = 0;
      for (int q = 0; q < na; q++)
        if (!h_done[q]) h_act[nn++] = h_act[q];
      na = nn;
    }
    htime_end(c, "host:sub_jacobi_loop", ht);
    ht = htime_now();
    if (rc == ASOHF_OK) {
      // every subhalo's members at its final radius, in slot order, from the
      // segments kept as the radii were fixed
      h_off[0] = 0;
      for (int s = 0; s < ns; s++) h_off[s + 1] = h_off[s] + fin_cnt[s];
      const int64_t T = h_off[ns];
      const size_t work = ((size_t)T + ns) * (2 * (8 + 16 + 16) + 8 + 1) + 16384;
      ASOHF_CHECK(seg_reserve(c, (size_t)T * 12 + work + 16384));
      unsigned long long* keys = (unsigned long long*)seg_alloc(c, 8 * (size_t)T + 8);
      int32_t* vals = (int32_t*)seg_alloc(c, 4 * (size_t)T + 4);
      int64_t* d_src = (int64_t*)seg_alloc(c, 8 * (size_t)ns);
      if (!keys || !vals || !d_src) return ASOHF_ERR_CAPACITY;
      for (int s = 0; s < ns; s++) { h_dst[s] = h_off[s]; h_st[s] = (int32_t)fin_cnt[s]; }
      ASOHF_CUDA(cudaMemcpyAsync(d_src, fin_off.data(), 8 * (size_t)ns, cudaMemcpyHostToDevice, c->stream));
      ASOHF_CUDA(cudaMemcpyAsync(d_ids_off, h_dst.data(), 8 * (size_t)ns, cudaMemcpyHostToDevice, c->stream));
      ASOHF_CUDA(cudaMemcpyAsync(d_konta, h_st, 4 * (size_t)ns, cudaMemcpyHostToDevice, c->stream));
      ASOHF_CUDA(cudaMemcpyAsync(d_off, h_off, 8 * (size_t)(ns + 1), cudaMemcpyHostToDevice, c->stream));
      if (T > 0) {
        int kt_ = ktime_begin(c, "sub_final_segments");
        k_copy_segments<<<ns, 256, 0, c->stream>>>(c->sfin_k, c->sfin_v, d_src, d_konta, d_ids_off, keys, vals);
        ktime_end(c, kt_);
        c->launches++;
      }
      ASOHF_CUDA(cudaGetLastError());
      ASOHF_CUDA(cudaStreamSynchronize(c->stream));
      htime_end(c, "host:sub_final_gather", ht);
      ht = htime_now();
      // staged lists of the kept members, tiers by that count
      const size_t E = (size_t)T + ns;
      SegG sg;
      sg.konta = d_konta;
      sg.off = d_off;
      sg.keys = keys;
      sg.vals = vals;
      sg.a.dm = (float2*)seg_alloc(c, 8 * E);
      sg.a.mv = (float4*)seg_alloc(c, 16 * E);
      sg.a.px = (float4*)seg_alloc(c, 16 * E);
      sg.b.dm = (float2*)seg_alloc(c, 8 * E);
      sg.b.mv = (float4*)seg_alloc(c, 16 * E);
      sg.b.px = (float4*)seg_alloc(c, 16 * E);
      sg.pot = (double*)seg_alloc(c, 8 * E);
      sg.flag = (uint8_t*)seg_alloc(c, E);
      sg.final_b = (uint8_t*)arena_alloc(c, (size_t)ns);
      sg.nbound = d_nbound;
      sg.nscan = d_nscan;
      sg.work = c->d_work;
      sg.status = pr.status;
      sg.timing = 0;
      sg.eig = (float*)arena_alloc(c, 36 * (size_t)ns);
      int32_t* d_ts = (int32_t*)arena_alloc(c, 4 * (size_t)ns);
      if (!sg.a.dm || !sg.a.mv || !sg.a.px || !sg.b.dm || !sg.b.mv || !sg.b.px || !sg.pot || !sg.flag ||
          !sg.final_b || !d_ts || !sg.eig) {
        return ASOHF_ERR_CAPACITY;
      }
      ASOHF_CUDA(cudaMemsetAsync(sg.eig, 0xff, 36 * (size_t)ns, c->stream));  // NaN: no tensor
      SubMainIn in;
      in.konta = d_konta; in.jjac = f_jjac; in.masadm = f_masadm; in.rclus = f_rclus;
      in.cx = pr.cx; in.cy = pr.cy; in.cz = pr.cz; in.mhost = pr.mhost; in.disthost = pr.disthost;
      Tiers ts;
      ASOHF_CUDA(cudaMemcpyAsync(h_st, f_jjac, 4 * (size_t)ns, cudaMemcpyDeviceToHost, c->stream));
      ASOHF_CUDA(cudaStreamSynchronize(c->stream));
      ASOHF_CHECK(split_tiers(c, h_st, ns, d_ts, &ts));
      {
        int kt_ = ktime_begin(c, "sub_main");
        LAUNCH_TIERS_CTA(k_sub_main_g, ts, S, H, m.d, d_work, in, sg);
        ktime_end(c, kt_);
      }
      {
        int kt_ = ktime_begin(c, "sub_eigen");
        k_eigen<<<(ns + 127) / 128, 128, 0, c->stream>>>(sg.eig, d_work, ns, m.d.eigenval);
        ktime_end(c, kt_);
      }
      c->launches++;
      ASOHF_CUDA(cudaGetLastError());
      ASOHF_CUDA(cudaMemcpyAsync(h_st, pr.status, 4 * (size_t)ns, cudaMemcpyDeviceToHost, c->stream));
      ASOHF_CUDA(cudaStreamSynchronize(c->stream));
      for (int s = 0; s < ns; s++)
        if (h_st[s] && !rc) rc = h_st[s];
      htime_end(c, "host:sub_main", ht);
      ht = htime_now();
      if (H.want_ids && rc == ASOHF_OK) {
        int64_t total;
        ASOHF_CHECK(assign_id_offsets(c, m, lowh1, lowh2, hw, ns, d_nbound, d_ids_off, &total));
        ASOHF_CHECK(ensure_pph(c, total));
        {
          int kt_ = ktime_begin(c, "sub_write_ids");
          LAUNCH_TIERS_CTA(k_write_ids, ts, d_nscan, d_off, d_ids_off, sg.final_b, sg.a.px, sg.b.px, sg.flag,
                           c->p.id, c->d_pph);
          ktime_end(c, kt_);
        }
        ASOHF_CUDA(cudaGetLastError());
        c->pph_len = total;
      }
    }
  } else if (H.want_ids) {
    int64_t total;
    ASOHF_CHECK(assign_id_offsets(c, m, lowh1, lowh2, hw, 0, nullptr, nullptr, &total));
    c->pph_len = total;
  }
  htime_end(c, "host:sub_ids", ht);
  ht = htime_now();
  ASOHF_CHECK(cat_mirror_out(c, &m));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  htime_end(c, "host:sub_mirror_out", ht);
  return rc;
}
