// ctx.cu -- context lifetime, scratch arena, device particle store.
#include <mutex>
#include <set>
#include <string>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "common.cuh"

static char g_last_detail[512] = "";

void asohf_set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  snprintf(g_last_detail, sizeof(g_last_detail), "%s: %s (%s:%d)", cudaGetErrorString(e), what,
           file, line);
}

extern "C" const char* asohf_last_error_detail(void) { return g_last_detail; }

extern "C" const char* asohf_strerror(int code) {
  switch (code) {
    case ASOHF_OK: return "ok";
    case ASOHF_ERR_INVALID: return "invalid argument";
    case ASOHF_ERR_CUDA: return "CUDA error";
    case ASOHF_ERR_CAPACITY: return "capacity exceeded";
    case ASOHF_ERR_TIMEOUT: return "device wait timed out";
    case ASOHF_ERR_NOT_PREFOUND_VIRIAL: return "NOT PRE-FOUND VIRIAL RADIUS!";
    case ASOHF_ERR_WRONG_SORTING: return "wrong sorting, cannot continue";
    case ASOHF_ERR_NO_DEVICE: return "no usable CUDA device";
    case ASOHF_ERR_UNSUPPORTED: return "unsupported option";
    case ASOHF_ERR_NOT_CONVERGED: return "growing not converged";
    default: return "unknown status";
  }
}

static int stage_join(asohf_ctx* c);
static int out_join(asohf_ctx* c);

static void free_particles(DevParticles& p) {
  cudaFree(p.x); cudaFree(p.y); cudaFree(p.z);
  cudaFree(p.vx); cudaFree(p.vy); cudaFree(p.vz);
  cudaFree(p.m); cudaFree(p.id);
  p = DevParticles();
}

static int alloc_particles(DevParticles& p, int64_t cap) {
  size_t fb = sizeof(float) * (size_t)cap;
  ASOHF_CUDA(cudaMalloc(&p.x, fb)); ASOHF_CUDA(cudaMalloc(&p.y, fb)); ASOHF_CUDA(cudaMalloc(&p.z, fb));
  ASOHF_CUDA(cudaMalloc(&p.vx, fb)); ASOHF_CUDA(cudaMalloc(&p.vy, fb)); ASOHF_CUDA(cudaMalloc(&p.vz, fb));
  ASOHF_CUDA(cudaMalloc(&p.m, fb));
  ASOHF_CUDA(cudaMalloc(&p.id, sizeof(int32_t) * (size_t)cap));
  p.cap = cap;
  return ASOHF_OK;
}

int ctx_ensure_particles(asohf_ctx* c, int64_t n) {
  // both sets: a prefetch can hand the store arrays of another capacity
  if (c->p.cap < n || c->alt.cap < n) {
    ASOHF_CUDA(cudaStreamSynchronize(c->stream));
    free_particles(c->p);
    free_particles(c->alt);
    ASOHF_CHECK(alloc_particles(c->p, n));
    ASOHF_CHECK(alloc_particles(c->alt, n));
  }
  c->p.n = n;
  c->alt.n = n;
  return ASOHF_OK;
}

void ctx_swap_particles(asohf_ctx* c) {
  DevParticles t = c->p;
  c->p = c->alt;
  c->alt = t;
}

int arena_reserve(asohf_ctx* c, size_t bytes) {
  bytes = (bytes + 255) & ~(size_t)255;
  if (c->arena_size >= bytes) return ASOHF_OK;
  if (c->arena_used != 0) return ASOHF_ERR_CAPACITY;
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(c->arena);
  c->arena = nullptr;
  c->arena_size = 0;
  size_t want = bytes + bytes / 4;
  ASOHF_CUDA(cudaMalloc(&c->arena, want));
  c->arena_size = want;
  return ASOHF_OK;
}

void* arena_alloc(asohf_ctx* c, size_t bytes) {
  size_t b = (bytes + 255) & ~(size_t)255;
  if (c->arena_used + b > c->arena_size) return nullptr;
  void* p = c->arena + c->arena_used;
  c->arena_used += b;
  return p;
}

int dpool_reserve(asohf_ctx* c, int which, size_t bytes) {
  asohf_ctx::Pool& p = c->dpool[which];
  p.used = 0;
  bytes = (bytes + 255) & ~(size_t)255;
  if (p.size >= bytes) return ASOHF_OK;
  cudaFree(p.base);
  p.base = nullptr;
  p.size = 0;
  size_t want = bytes + bytes / 4;
  ASOHF_CUDA(cudaMalloc(&p.base, want));
  p.size = want;
  return ASOHF_OK;
}

void* dpool_alloc(asohf_ctx* c, int which, size_t bytes) {
  asohf_ctx::Pool& p = c->dpool[which];
  size_t b = (bytes + 255) & ~(size_t)255;
  if (p.used + b > p.size) return nullptr;
  void* r = p.base + p.used;
  p.used += b;
  return r;
}

int density_settle(asohf_ctx* c) {
  if (!c->dens_pending) return ASOHF_OK;
  c->dens_pending = false;
  ASOHF_CUDA(cudaEventSynchronize(c->dens_done));
  return ASOHF_OK;
}

extern "C" int asohf_set_density_overlap(asohf_ctx* c, int on) {
  if (!c) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  if (on && !c->dens_stream) {
    // the least priority: its CTAs are scheduled when the hot path's streams
    // have none waiting, so the deferred deposit fills the gaps of the halo
    // finder instead of holding the SMs ahead of it
    int least = 0, greatest = 0;
    ASOHF_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    ASOHF_CUDA(cudaStreamCreateWithPriority(&c->dens_stream, cudaStreamNonBlocking, least));
    ASOHF_CUDA(cudaEventCreateWithFlags(&c->dens_fork, cudaEventDisableTiming));
    ASOHF_CUDA(cudaEventCreateWithFlags(&c->dens_done, cudaEventDisableTiming));
  }
  c->density_overlap = on ? 1 : 0;
  return ASOHF_OK;
}

extern "C" int asohf_density_wait(asohf_ctx* c, void* cuda_stream) {
  if (!c) return ASOHF_ERR_INVALID;
  if (c->dens_pending) ASOHF_CUDA(cudaStreamWaitEvent((cudaStream_t)cuda_stream, c->dens_done, 0));
  return ASOHF_OK;
}

int seg_reserve(asohf_ctx* c, size_t bytes) {
  c->seg_used = 0;
  bytes = (bytes + 255) & ~(size_t)255;
  if (c->seg_size >= bytes) return ASOHF_OK;
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(c->seg);
  c->seg = nullptr;
  c->seg_size = 0;
  size_t want = bytes + bytes / 4;
  ASOHF_CUDA(cudaMalloc(&c->seg, want));
  c->seg_size = want;
  return ASOHF_OK;
}

void* seg_alloc(asohf_ctx* c, size_t bytes) {
  size_t b = (bytes + 255) & ~(size_t)255;
  if (c->seg_used + b > c->seg_size) return nullptr;
  void* p = c->seg + c->seg_used;
  c->seg_used += b;
  return p;
}

__global__ void k_minmax(const float* __restrict__ m, int64_t n, float* out) {
  __shared__ float sb[32];
  float lo = INFINITY, hi = -INFINITY;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float v = m[i];
    lo = fminf(lo, v);
    hi = fmaxf(hi, v);
  }
  hi = block_max_f(hi, sb);
  lo = block_min_f(lo, sb);
  if (threadIdx.x == 0) {
    // float max/min through ordered int bit patterns (masses are >= 0)
    atomicMax((int*)&out[1], __float_as_int(hi));
    atomicMin((int*)&out[0], __float_as_int(lo));
  }
}

int ctx_refresh_mass_range(asohf_ctx* c) {
  float* d = (float*)arena_alloc(c, 2 * sizeof(float));
  if (!d) return ASOHF_ERR_CAPACITY;
  float init[2] = {INFINITY, 0.0f};
  ASOHF_CUDA(cudaMemcpyAsync(d, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
  k_minmax<<<grid_for(c->p.n, 256, 1024), 256, 0, c->stream>>>(c->p.m, c->p.n, d);
  c->launches++;
  float h[2];
  ASOHF_CUDA(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  c->mmin = h[0];
  c->norma = h[1];
  return ASOHF_OK;
}

extern "C" int asohf_create(int device, asohf_ctx** out) {
  if (!out) return ASOHF_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0)
    return ASOHF_ERR_NO_DEVICE;
  ASOHF_CUDA(cudaSetDevice(device));
  asohf_ctx* c = new asohf_ctx();
  c->device = device;
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  bool ok = arena_reserve(c, 64u << 20) == ASOHF_OK && cudaMalloc(&c->d_work, 64) == cudaSuccess &&
            cudaMemset(c->d_work, 0, 64) == cudaSuccess &&
            cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; ok && i < asohf_ctx::NSIDE; i++)
    ok = cudaStreamCreateWithFlags(&c->side[i], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&c->ev_join[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    for (int i = 0; i < asohf_ctx::NSIDE; i++) {
      if (c->ev_join[i]) cudaEventDestroy(c->ev_join[i]);
      if (c->side[i]) cudaStreamDestroy(c->side[i]);
    }
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    cudaFree(c->d_work);
    cudaFree(c->arena);
    delete c;
    return ASOHF_ERR_CUDA;
  }
  *out = c;
  return ASOHF_OK;
}

extern "C" int asohf_destroy(asohf_ctx* c) {
  if (!c) return ASOHF_ERR_INVALID;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  if (c->dens_stream) {
    cudaStreamSynchronize(c->dens_stream);
    cudaStreamDestroy(c->dens_stream);
    cudaEventDestroy(c->dens_fork);
    cudaEventDestroy(c->dens_done);
  }
  cudaFree(c->dpool[0].base);
  cudaFree(c->dpool[1].base);
  stage_join(c);
  out_join(c);
  if (c->out_stream) {
    cudaStreamSynchronize(c->out_stream);
    cudaStreamDestroy(c->out_stream);
    cudaEventDestroy(c->out_fork);
    cudaEventDestroy(c->out_chunk);
    cudaEventDestroy(c->out_done);
  }
  if (c->copy_stream) {
    cudaStreamSynchronize(c->copy_stream);
    cudaStreamDestroy(c->copy_stream);
    cudaEventDestroy(c->stage_ready);
    cudaEventDestroy(c->stage_free);
    cudaEventDestroy(c->chunk_done);
  }
  free_particles(c->p);
  free_particles(c->alt);
  free_particles(c->stage);
  cudaFree(c->rows[0]);
  cudaFree(c->rows[1]);
  cudaFree(c->d_s2);
  cudaFree(c->d_tw);
  cudaFree(c->d_radx);
  free(c->h_radx);
  cudaFree(c->d_ndmpart_x);
  cudaFree(c->d_colstart);
  cudaFree(c->d_colpart);
  cudaFree(c->d_pph);
  cudaFree(c->sfin_k);
  cudaFree(c->sfin_v);
  cudaFree(c->arena);
  cudaFree(c->seg);
  cudaFree(c->d_work);
  for (int i = 0; i < asohf_ctx::NSIDE; i++) {
    cudaStreamSynchronize(c->side[i]);
    cudaEventDestroy(c->ev_join[i]);
    cudaStreamDestroy(c->side[i]);
  }
  cudaEventDestroy(c->ev_fork);
  for (int i = 0; i < c->nkrec; i++) { cudaEventDestroy(c->krec[i].a); cudaEventDestroy(c->krec[i].b); }
  free(c->krec);
  delete c;
  return ASOHF_OK;
}

// The side streams (size tiers) run at the context stream's priority, so a
// caller that raises its stream's priority raises the whole hot path above
// the deferred deposit (created at the least priority).
extern "C" int asohf_set_stream(asohf_ctx* c, void* s) {
  if (!c) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  int prio = 0;
  ASOHF_CUDA(cudaStreamGetPriority((cudaStream_t)s, &prio));
  if (prio != c->side_prio) {
    for (int i = 0; i < asohf_ctx::NSIDE; i++) {
      cudaStream_t n = nullptr;
      ASOHF_CUDA(cudaStreamCreateWithPriority(&n, cudaStreamNonBlocking, prio));
      ASOHF_CUDA(cudaStreamSynchronize(c->side[i]));
      cudaStreamDestroy(c->side[i]);
      c->side[i] = n;
    }
    c->side_prio = prio;
  }
  c->stream = (cudaStream_t)s;
  return ASOHF_OK;
}

extern "C" int asohf_synchronize(asohf_ctx* c) {
  if (!c) return ASOHF_ERR_INVALID;
  ASOHF_CHECK(density_settle(c));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  return ASOHF_OK;
}

extern "C" int64_t asohf_launch_count(asohf_ctx* c) { return c ? c->launches : -1; }

int ktime_begin(asohf_ctx* c, const char* name, cudaStream_t s) {
  if (!c->profiling) return -1;
  if (c->nkrec == c->capkrec) {
    int cap = c->capkrec ? 2 * c->capkrec : 256;
    asohf_ctx::KRec* n = (asohf_ctx::KRec*)realloc(c->krec, sizeof(asohf_ctx::KRec) * cap);
    if (!n) return -1;
    c->krec = n;
    c->capkrec = cap;
  }
  asohf_ctx::KRec& r = c->krec[c->nkrec];
  r.name = name;
  r.s = s;
  if (cudaEventCreate(&r.a) != cudaSuccess) return -1;
  if (cudaEventCreate(&r.b) != cudaSuccess) { cudaEventDestroy(r.a); return -1; }
  cudaEventRecord(r.a, s);
  return c->nkrec++;
}

void ktime_end(asohf_ctx* c, int slot, cudaStream_t s) {
  if (slot < 0) return;
  cudaEventRecord(c->krec[slot].b, s);
}

static void ksum_add(asohf_ctx* c, const char* name, double ms) {
  int k;
  for (k = 0; k < c->nksum; k++)
    if (strcmp(c->ksum[k].name, name) == 0) break;
  if (k == c->nksum) {
    if (c->nksum >= asohf_ctx::KSUM_CAP) return;
    c->ksum[k].name = name;
    c->ksum[k].ms = 0.0;
    c->ksum[k].n = 0;
    c->nksum++;
  }
  c->ksum[k].ms += ms;
  c->ksum[k].n++;
}

double htime_now() {
  timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec * 1e3 + (double)t.tv_nsec * 1e-6;
}

void htime_end(asohf_ctx* c, const char* name, double t0) {
  if (c->profiling) ksum_add(c, name, htime_now() - t0);
}

// "idle:<name>" names, interned for the statistics table (a bounded set:
// one per timed region name)
static const char* idle_name(const char* name) {
  static std::mutex mu;
  static std::set<std::string> names;
  std::lock_guard<std::mutex> lock(mu);
  return names.insert(std::string("idle:") + name).first->c_str();
}

// Folds the recorded events into the statistics.  Besides each region's
// time, the gaps of the context stream between consecutive top-level regions
// on it (host work, synchronisations and untimed launches in between) are
// added as "idle:<next region>"; the per-tier sub-regions ("name/tier") sit
// inside their family's region and are left out of the gaps.
static void ktime_flush(asohf_ctx* c) {
  cudaStreamSynchronize(c->stream);
  int prev = -1;
  for (int i = 0; i < c->nkrec; i++) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->krec[i].a, c->krec[i].b);
    ksum_add(c, c->krec[i].name, ms);
    if (c->krec[i].s == c->stream && !strchr(c->krec[i].name, '/')) {  // top-level regions only
      if (prev >= 0) {
        float gap = 0.f;
        if (cudaEventElapsedTime(&gap, c->krec[prev].b, c->krec[i].a) == cudaSuccess && gap > 0.f)
          ksum_add(c, idle_name(c->krec[i].name), gap);
      }
      prev = i;
    }
  }
  for (int i = 0; i < c->nkrec; i++) {
    cudaEventDestroy(c->krec[i].a);
    cudaEventDestroy(c->krec[i].b);
  }
  cudaGetLastError();
  c->nkrec = 0;
}

extern "C" int asohf_set_profiling(asohf_ctx* c, int on) {
  if (!c) return ASOHF_ERR_INVALID;
  ktime_flush(c);
  c->profiling = on;
  c->nksum = 0;
  return ASOHF_OK;
}

extern "C" int asohf_kernel_stats(asohf_ctx* c, int i, const char** name, double* total_ms,
                                  int64_t* launches) {
  if (!c || !name || !total_ms || !launches) return ASOHF_ERR_INVALID;
  ktime_flush(c);
  if (i < 0 || i >= c->nksum) return ASOHF_ERR_INVALID;
  *name = c->ksum[i].name;
  *total_ms = c->ksum[i].ms;
  *launches = c->ksum[i].n;
  return ASOHF_OK;
}

static void host_fields(const asohf_particles* s, const void* f[8]) {
  f[0] = s->x; f[1] = s->y; f[2] = s->z; f[3] = s->vx; f[4] = s->vy; f[5] = s->vz; f[6] = s->m; f[7] = s->id;
}

// Copy of a prefetch, on the context's copy stream, in chunks of
// STAGE_CHUNK bytes issued one at a time: the copy engine serves copies in
// the order they were queued, so a 4 GB copy queued at once would hold every
// short copy the context stream issues meanwhile (mesh, catalogue windows)
// until it ends; chunk by chunk, such a copy waits for one chunk at most.
#define STAGE_CHUNK (32ll << 20)

static int stage_copy(asohf_ctx* c, const void* const src[8], int64_t n) {
  ASOHF_CUDA(cudaSetDevice(c->device));
  void* dst[8] = {c->stage.x, c->stage.y, c->stage.z, c->stage.vx, c->stage.vy, c->stage.vz, c->stage.m,
                  c->stage.id};
  const int64_t bytes = 4 * n;  // every field is 4 bytes an entry
  for (int64_t o = 0; o < bytes; o += STAGE_CHUNK) {
    const int64_t b = bytes - o < STAGE_CHUNK ? bytes - o : STAGE_CHUNK;
    for (int q = 0; q < 8; q++)
      ASOHF_CUDA(cudaMemcpyAsync((char*)dst[q] + o, (const char*)src[q] + o, (size_t)b, cudaMemcpyHostToDevice,
                                 c->copy_stream));
    ASOHF_CUDA(cudaEventRecord(c->chunk_done, c->copy_stream));
    ASOHF_CUDA(cudaEventSynchronize(c->chunk_done));
  }
  ASOHF_CUDA(cudaEventRecord(c->stage_ready, c->copy_stream));
  return ASOHF_OK;
}

// Waits until the stager has issued every chunk of the staged copy.
static int stage_join(asohf_ctx* c) {
  if (c->stager.joinable()) c->stager.join();
  int st = c->stage_status;
  c->stage_status = ASOHF_OK;
  return st;
}

extern "C" int asohf_prefetch_particles(asohf_ctx* c, const asohf_particles* s) {
  if (!c || !s || s->n < 0) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  ASOHF_CHECK(stage_join(c));  // an earlier prefetch not taken: its chunks are all issued
  c->staged = false;
  if (!c->copy_stream) {
    ASOHF_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    ASOHF_CUDA(cudaEventCreateWithFlags(&c->stage_ready, cudaEventDisableTiming));
    ASOHF_CUDA(cudaEventCreateWithFlags(&c->stage_free, cudaEventDisableTiming));
    ASOHF_CUDA(cudaEventCreateWithFlags(&c->chunk_done, cudaEventDisableTiming | cudaEventBlockingSync));
  }
  if (c->stage.cap < s->n) {  // a larger staging store: nothing may still copy into the old one
    ASOHF_CUDA(cudaStreamSynchronize(c->copy_stream));
    if (c->stage_free_set) ASOHF_CUDA(cudaEventSynchronize(c->stage_free));
    free_particles(c->stage);
    ASOHF_CHECK(alloc_particles(c->stage, s->n));
    c->stage_free_set = false;
  }
  c->stage.n = s->n;
  // the staging arrays were the store of an earlier call: copy into them once
  // the work issued before they were handed over is done
  if (c->stage_free_set) ASOHF_CUDA(cudaStreamWaitEvent(c->copy_stream, c->stage_free, 0));
  host_fields(s, c->staged_src);
  c->staged_n = s->n;
  c->staged = true;
  const void* src[8];
  for (int q = 0; q < 8; q++) src[q] = c->staged_src[q];
  const int64_t n = s->n;
  try {
    c->stager = std::thread([c, src, n]() { c->stage_status = stage_copy(c, src, n); });
  } catch (...) {  // no thread: the copy is issued from here, at once
    c->stage_status = stage_copy(c, src, n);
  }
  return ASOHF_OK;
}

// A prefetch of exactly these host arrays: the context stream waits for its
// copy and the staging store becomes the particle store; the store it
// replaces becomes the staging store of the next prefetch.
static bool take_staged(asohf_ctx* c, const asohf_particles* s) {
  if (!c->staged || c->staged_n != s->n) return false;
  const void* f[8];
  host_fields(s, f);
  for (int q = 0; q < 8; q++)
    if (f[q] != c->staged_src[q]) return false;
  return true;
}

extern "C" int asohf_upload_particles(asohf_ctx* c, const asohf_particles* s, int on_device) {
  if (!c || !s || s->n < 0) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  arena_reset(c);
  if (!on_device && take_staged(c, s)) {
    c->staged = false;
    ASOHF_CHECK(stage_join(c));
    ASOHF_CHECK(ctx_ensure_particles(c, s->n));
    ASOHF_CUDA(cudaStreamWaitEvent(c->stream, c->stage_ready, 0));
    DevParticles t = c->p;
    c->p = c->stage;
    c->stage = t;
    c->p.n = s->n;
    ASOHF_CUDA(cudaEventRecord(c->stage_free, c->stream));
    c->stage_free_set = true;
    c->nx_sorted = 0;
    c->rows_cur = -1;
    if (s->n > 0) ASOHF_CHECK(ctx_refresh_mass_range(c));
    return ASOHF_OK;
  }
  ASOHF_CHECK(ctx_ensure_particles(c, s->n));
  cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  size_t fb = sizeof(float) * (size_t)s->n;
  ASOHF_CUDA(cudaMemcpyAsync(c->p.x, s->x, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(c->p.y, s->y, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(c->p.z, s->z, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(c->p.vx, s->vx, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(c->p.vy, s->vy, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(c->p.vz, s->vz, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(c->p.m, s->m, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(c->p.id, s->id, sizeof(int32_t) * (size_t)s->n, k, c->stream));
  c->nx_sorted = 0;  // slab table and column index are stale
  c->rows_cur = -1;  // and so is the row copy
  if (s->n > 0) ASOHF_CHECK(ctx_refresh_mass_range(c));
  return ASOHF_OK;
}

extern "C" int asohf_download_particles(asohf_ctx* c, asohf_particles* d, int on_device) {
  if (!c || !d || d->n < c->p.n) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  size_t fb = sizeof(float) * (size_t)c->p.n;
  ASOHF_CUDA(cudaMemcpyAsync(d->x, c->p.x, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(d->y, c->p.y, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(d->z, c->p.z, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(d->vx, c->p.vx, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(d->vy, c->p.vy, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(d->vz, c->p.vz, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(d->m, c->p.m, fb, k, c->stream));
  ASOHF_CUDA(cudaMemcpyAsync(d->id, c->p.id, sizeof(int32_t) * (size_t)c->p.n, k, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  return ASOHF_OK;
}

extern "C" int asohf_work_counters(asohf_ctx* c, int64_t* out, int reset) {
  if (!c || !out) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaMemcpyAsync(out, c->d_work, 64, cudaMemcpyDeviceToHost, c->stream));
  if (reset) ASOHF_CUDA(cudaMemsetAsync(c->d_work, 0, 64, c->stream));
  ASOHF_CUDA(cudaStreamSynchronize(c->stream));
  return ASOHF_OK;
}

// ------------------------------------------------------------ host copies
// Device -> page-locked host copies on a copy engine, issued in chunks of
// STAGE_CHUNK bytes one at a time by a helper thread (the copy engine serves
// copies in the order they were queued: chunk by chunk, a short copy of the
// context stream waits for one chunk at most).
static void out_worker(asohf_ctx* c) {
  int st = ASOHF_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) st = ASOHF_ERR_CUDA;
  for (;;) {
    asohf_ctx::OutJob j;
    {
      std::lock_guard<std::mutex> lock(c->out_mu);
      if (c->out_jobs.empty()) {
        c->out_running = false;
        if (st != ASOHF_OK) c->out_status = st;
        return;
      }
      j = c->out_jobs.front();
      c->out_jobs.erase(c->out_jobs.begin());
    }
    for (int64_t o = 0; st == ASOHF_OK && o < j.bytes; o += STAGE_CHUNK) {
      const int64_t b = j.bytes - o < STAGE_CHUNK ? j.bytes - o : STAGE_CHUNK;
      if (cudaMemcpyAsync((char*)j.dst + o, (const char*)j.src + o, (size_t)b, cudaMemcpyDeviceToHost,
                          c->out_stream) != cudaSuccess ||
          cudaEventRecord(c->out_chunk, c->out_stream) != cudaSuccess ||
          cudaEventSynchronize(c->out_chunk) != cudaSuccess)
        st = ASOHF_ERR_CUDA;
    }
    if (st == ASOHF_OK && cudaEventRecord(c->out_done, c->out_stream) != cudaSuccess) st = ASOHF_ERR_CUDA;
  }
}

static int out_join(asohf_ctx* c) {
  if (c->outer.joinable()) c->outer.join();
  int st = c->out_status;
  c->out_status = ASOHF_OK;
  return st;
}

extern "C" int asohf_copy_to_host_async(asohf_ctx* c, void* host_dst, const void* dev_src, int64_t bytes) {
  if (!c || bytes < 0 || (bytes && (!host_dst || !dev_src))) return ASOHF_ERR_INVALID;
  if (bytes == 0) return ASOHF_OK;
  ASOHF_CUDA(cudaSetDevice(c->device));
  cudaPointerAttributes ha, da;
  ASOHF_CUDA(cudaPointerGetAttributes(&ha, host_dst));
  ASOHF_CUDA(cudaPointerGetAttributes(&da, dev_src));
  if (ha.type != cudaMemoryTypeHost || da.type != cudaMemoryTypeDevice || da.device != c->device)
    return ASOHF_ERR_INVALID;  // page-locked host memory and this context's device memory only
  if (!c->out_stream) {
    ASOHF_CUDA(cudaStreamCreateWithFlags(&c->out_stream, cudaStreamNonBlocking));
    ASOHF_CUDA(cudaEventCreateWithFlags(&c->out_fork, cudaEventDisableTiming));
    ASOHF_CUDA(cudaEventCreateWithFlags(&c->out_chunk, cudaEventDisableTiming | cudaEventBlockingSync));
    ASOHF_CUDA(cudaEventCreateWithFlags(&c->out_done, cudaEventDisableTiming));
  }
  // after the work issued so far: the context stream's and a deferred patch
  // deposit's
  ASOHF_CUDA(cudaEventRecord(c->out_fork, c->stream));
  ASOHF_CUDA(cudaStreamWaitEvent(c->out_stream, c->out_fork, 0));
  if (c->dens_pending) ASOHF_CUDA(cudaStreamWaitEvent(c->out_stream, c->dens_done, 0));
  std::lock_guard<std::mutex> lock(c->out_mu);
  c->out_jobs.push_back({host_dst, dev_src, bytes});
  c->out_any = true;
  if (!c->out_running) {
    if (c->outer.joinable()) c->outer.join();
    c->out_running = true;
    try {
      c->outer = std::thread(out_worker, c);
    } catch (...) {
      c->out_running = false;
      c->out_jobs.pop_back();
      return ASOHF_ERR_CAPACITY;
    }
  }
  return ASOHF_OK;
}

extern "C" int asohf_copy_wait(asohf_ctx* c, void* cuda_stream) {
  if (!c) return ASOHF_ERR_INVALID;
  ASOHF_CUDA(cudaSetDevice(c->device));
  ASOHF_CHECK(out_join(c));
  if (!c->out_any) return ASOHF_OK;
  if (cuda_stream) ASOHF_CUDA(cudaStreamWaitEvent((cudaStream_t)cuda_stream, c->out_done, 0));
  else ASOHF_CUDA(cudaEventSynchronize(c->out_done));
  return ASOHF_OK;
}

// Device -> page-locked host copy made by SM stores through the host
// buffer's device mapping instead of a copy engine: a large copy issued this
// way on a stream of its own does not queue ahead of the short copies the
// context's host phases make meanwhile.
__global__ void k_store_to_host(const uint4* __restrict__ src, uint4* __restrict__ dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

extern "C" int asohf_copy_to_host_sm(asohf_ctx* c, void* host_dst, const void* dev_src, int64_t bytes,
                                     void* stream) {
  if (!c || bytes < 0 || (bytes && (!host_dst || !dev_src))) return ASOHF_ERR_INVALID;
  if (bytes % 16 || (uintptr_t)host_dst % 16 || (uintptr_t)dev_src % 16) return ASOHF_ERR_INVALID;
  if (bytes == 0) return ASOHF_OK;
  ASOHF_CUDA(cudaSetDevice(c->device));
  cudaPointerAttributes ha, da;
  ASOHF_CUDA(cudaPointerGetAttributes(&ha, host_dst));
  ASOHF_CUDA(cudaPointerGetAttributes(&da, dev_src));
  if (ha.type != cudaMemoryTypeHost || !ha.devicePointer || da.type != cudaMemoryTypeDevice ||
      da.device != c->device)
    return ASOHF_ERR_INVALID;  // page-locked host memory and this context's device memory only
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  int64_t n = bytes / 16;
  int grid = c->num_sms / 4 > 0 ? c->num_sms / 4 : 1;
  k_store_to_host<<<grid, 256, 0, s>>>((const uint4*)dev_src, (uint4*)ha.devicePointer, n);
  ASOHF_CUDA(cudaGetLastError());
  c->launches++;
  return ASOHF_OK;
}
