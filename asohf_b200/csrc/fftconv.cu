// fftconv.cu -- the z pass of the periodic Poisson solve of POFFT3D
// (poisson.f:98-249) for NX in {64, 128, 256, 512}.
//
// The solve runs as three passes over the half spectrum: the library's
// batched 2-D R2C of every (copy, z) plane, then k_fft_z_green (FFT along z,
// the Green's multiply KKK/NX^3 of MOMENTO's table, inverse FFT along z, in
// place, one pass), then the library's 2-D C2R.  Against a library 3-D
// R2C, a separate multiply and a 3-D C2R, the z transforms and the multiply
// share one read and one write of the spectrum.
//
// Line transforms are done by one warp: an M = 32 R point line is held as
// R values per lane (lane l, register n1 = element l + 32 n1), transformed
// by an R-point decimation-in-frequency FFT in registers, a twiddle W_M^(l k1)
// and a 32-point decimation-in-frequency FFT across lanes (shuffles); lane l
// register p then holds frequency brev_R(p) + R brev_5(l).  The Green's
// factor is applied in that order and the inverse transform (the same
// stages undone in reverse, decimation in time) returns natural order, so
// the line goes through shared memory only on its way in and out.
// Twiddles W_N^j are a table computed on the host in double precision.  The
// result equals an FFT-based solve within float32 rounding (not bit for bit
// a library's).
#include <cuda_runtime.h>
#include <math.h>

#include <vector>

#include "common.cuh"

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// complex product with fused multiply-adds (two roundings per part)
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(__fmaf_rn(a.x, b.x, -__fmul_rn(a.y, b.y)), __fmaf_rn(a.x, b.y, __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

// index of a line element in shared memory, one pad element per 32: with an
// odd line stride, the tile's loads (one element of each of 16 lines) and a
// warp's reads along its line are free of bank conflicts
__host__ __device__ constexpr int pad(int f) { return f + (f >> 5); }

__host__ __device__ constexpr int ilog2(int v) { return v <= 1 ? 0 : 1 + ilog2(v >> 1); }
__host__ __device__ constexpr int brev_c(int p, int bits) {
  int r = 0;
  for (int b = 0; b < bits; b++)
    if ((p >> b) & 1) r |= 1 << (bits - 1 - b);
  return r;
}

template <bool INV>
__device__ __forceinline__ float2 twid(const float2* __restrict__ tw, int t) {
  const float2 w = __ldg(tw + t);
  return INV ? conjf2(w) : w;
}

// Per-lane twiddles of the 32-point stage across lanes, h = 16, 8, 4, 2:
// W_(2h)^(lane mod h) on the lanes that take the difference (lane bit h
// set), 1 on the others (forward sign).
template <int N>
__device__ __forceinline__ void lane_twiddles(const float2* __restrict__ tw, int lane, float2 (&wl)[4]) {
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int h = 16 >> q;
    const int t = (lane & (h - 1)) * (N / (2 * h));
    wl[q] = (t == 0 || (lane & h) == 0) ? make_float2(1.f, 0.f) : __ldg(tw + t);
  }
}

// frequency held by lane l, register p after warp_fft<R>
template <int R>
__device__ __forceinline__ int freq_of(int lane, int p) {
  return brev_c(p, ilog2(R)) + R * (int)(__brev((unsigned)lane) >> 27);
}

// Unnormalised DFT of an M = 32 R point line, sign -1 (INV: +1).
// In: v[n1] = x[lane + 32 n1].  Out: v[p] = X[freq_of<R>(lane, p)].
template <int N, int R, bool INV>
__device__ __forceinline__ void warp_fft(float2 (&v)[R], int lane, const float2* __restrict__ tw,
                                         const float2 (&wl)[4]) {
  constexpr int M = 32 * R;
  constexpr int S = N / M;
  // R-point DIF over the registers
#pragma unroll
  for (int h = R / 2; h >= 1; h >>= 1) {
#pragma unroll
    for (int b = 0; b < R; b += 2 * h) {
#pragma unroll
      for (int j = 0; j < h; j++) {
        const float2 a = v[b + j], c = v[b + j + h];
        v[b + j] = cadd(a, c);
        const float2 d = csub(a, c);
        const int t = j * (N / (2 * h));
        if (t == 0) v[b + j + h] = d;
        else if (t == N / 4) v[b + j + h] = INV ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
        else v[b + j + h] = cmul(d, twid<INV>(tw, t));
      }
    }
  }
  // W_M^(lane k1), k1 = brev_R(p)
#pragma unroll
  for (int p = 1; p < R; p++) {
    const int k1 = brev_c(p, ilog2(R));
    v[p] = cmul(v[p], twid<INV>(tw, lane * k1 * S));
  }
  // 32-point DIF across the lanes: the lane of a pair with bit h clear keeps
  // v + o, the other (o - v) W; one fused s v + o (s = +-1, exact) and one
  // product with the lane's twiddle (1 on the first lane) serve both
#pragma unroll
  for (int q = 0; q < 5; q++) {
    const int h = 16 >> q;
    const float sg = (lane & h) ? -1.f : 1.f;
#pragma unroll
    for (int p = 0; p < R; p++) {
      float2 o;
      o.x = __shfl_xor_sync(FULL, v[p].x, h);
      o.y = __shfl_xor_sync(FULL, v[p].y, h);
      const float2 d = make_float2(__fmaf_rn(sg, v[p].x, o.x), __fmaf_rn(sg, v[p].y, o.y));
      if (q < 4) v[p] = cmul(d, INV ? conjf2(wl[q]) : wl[q]);
      else v[p] = d;
    }
  }
}

// z-pass tile: TY lines of NX values (padded), ZT threads
template <int N>
struct Geo {
  static constexpr int NCOL = N / 2 + 1;         // kx = 0..N/2
  static constexpr int LSTR = N + N / 32 + 1;    // line stride (float2): padded, odd
  static constexpr int TY = 16;                  // lines per tile
  static constexpr int ZT = 256;                 // threads
  static constexpr size_t ZSMEM = sizeof(float2) * (size_t)TY * LSTR;
};

}  // namespace

// The exact inverse of warp_fft<N, R, false> up to the factor M: the
// unnormalised inverse DFT (sign +1) of a line held in warp_fft's output
// order.  In: v[p] = X[freq_of<R>(lane, p)].  Out: v[n1] = x[lane + 32 n1].
// Each stage undoes one of warp_fft's (decimation in time): across the lanes
// the value of the lane with bit h set is first multiplied by its conjugate
// twiddle, then the pair takes sum and difference.
template <int N, int R>
__device__ __forceinline__ void warp_ifft(float2 (&v)[R], int lane, const float2* __restrict__ tw,
                                          const float2 (&wl)[4]) {
  constexpr int M = 32 * R;
  constexpr int S = N / M;
#pragma unroll
  for (int q = 4; q >= 0; q--) {
    const int h = 16 >> q;
    const float sg = (lane & h) ? -1.f : 1.f;
#pragma unroll
    for (int p = 0; p < R; p++) {
      const float2 mm = q < 4 ? cmul(v[p], conjf2(wl[q])) : v[p];
      float2 o;
      o.x = __shfl_xor_sync(FULL, mm.x, h);
      o.y = __shfl_xor_sync(FULL, mm.y, h);
      v[p] = make_float2(__fmaf_rn(sg, mm.x, o.x), __fmaf_rn(sg, mm.y, o.y));
    }
  }
#pragma unroll
  for (int p = 1; p < R; p++) {
    const int k1 = brev_c(p, ilog2(R));
    v[p] = cmul(v[p], twid<true>(tw, lane * k1 * S));
  }
#pragma unroll
  for (int h = 1; h <= R / 2; h <<= 1) {
#pragma unroll
    for (int b = 0; b < R; b += 2 * h) {
#pragma unroll
      for (int j = 0; j < h; j++) {
        const float2 a = v[b + j], c = v[b + j + h];
        const int t = j * (N / (2 * h));
        float2 u;
        if (t == 0) u = c;
        else if (t == N / 4) u = make_float2(-c.y, c.x);  // c W^-1 = c i
        else u = cmul(c, twid<true>(tw, t));
        v[b + j] = cadd(a, u);
        v[b + j + h] = csub(a, u);
      }
    }
  }
}

// The z pass: a tile is TY consecutive values of one copy's (ky, kx) plane
// ([copy][z][ky][kx], NX/2+1 values per row, as the library's 2-D R2C leaves
// it), all NX z, in place: FFT along z, the Green's factor, inverse FFT
// along z.  KKK / N^3 = (-DEL2 / N^3) x 1 / (s2[kx] + s2[ky] + s2[kz])
// (denominator 1e30 at the origin; the reciprocal correctly rounded), on
// both parts.  One warp per line; the tile moves through shared memory so
// that every global access is a run of TY consecutive values.
template <int N>
__global__ void __launch_bounds__(Geo<N>::ZT)
k_fft_z_green(float2* __restrict__ spec, const float2* __restrict__ tw, const float* __restrict__ s2,
              float del2, float inv_n3) {
  using G = Geo<N>;
  constexpr int NW = G::ZT / 32, RZ = N / 32, QT = N * G::NCOL / G::TY;
  constexpr int PER = G::TY * N / G::ZT;  // tile values per thread
  extern __shared__ float2 sm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t t = blockIdx.x;
  const int q0 = (int)(t % QT) * G::TY;
  const int64_t copy = t / QT;
  const int64_t zstride = (int64_t)G::NCOL * N;
  float2* base = spec + copy * N * zstride + q0;
  {
    float2 r[PER];
#pragma unroll
    for (int i = 0; i < PER; i++) {
      const int e = threadIdx.x + G::ZT * i, z = e / G::TY, j = e % G::TY;
      r[i] = base[z * zstride + j];
    }
#pragma unroll
    for (int i = 0; i < PER; i++) {
      const int e = threadIdx.x + G::ZT * i, z = e / G::TY, j = e % G::TY;
      sm[j * G::LSTR + pad(z)] = r[i];
    }
  }
  __syncthreads();
  float2 wl[4];
  lane_twiddles<N>(tw, lane, wl);
  const float scale = __fmul_rn(-del2, inv_n3);
  for (int q = warp; q < G::TY; q += NW) {
    const int qq = q0 + q;
    const int kx = qq % G::NCOL, ky = qq / G::NCOL;
    float2* ln = sm + q * G::LSTR;
    float2 v[RZ];
#pragma unroll
    for (int n1 = 0; n1 < RZ; n1++) v[n1] = ln[pad(lane + 32 * n1)];
    warp_fft<N, RZ, false>(v, lane, tw, wl);
    const float sxy = __fadd_rn(__ldg(s2 + kx), __ldg(s2 + ky));
#pragma unroll
    for (int p = 0; p < RZ; p++) {
      const int kz = freq_of<RZ>(lane, p);
      const float den = (kx == 0 && ky == 0 && kz == 0) ? 1.0e30f : __fadd_rn(sxy, __ldg(s2 + kz));
      const float f = __fmul_rn(scale, __frcp_rn(den));
      v[p] = make_float2(__fmul_rn(v[p].x, f), __fmul_rn(v[p].y, f));
    }
    warp_ifft<N, RZ>(v, lane, tw, wl);
#pragma unroll
    for (int n1 = 0; n1 < RZ; n1++) ln[pad(lane + 32 * n1)] = v[n1];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < PER; i++) {
    const int e = threadIdx.x + G::ZT * i, z = e / G::TY, j = e % G::TY;
    base[z * zstride + j] = sm[j * G::LSTR + pad(z)];
  }
}

// W_N^j = exp(-2 pi i j / N), j < N, in double then rounded; exact at the
// quarter turns.  Kept on the context per N.
static int twiddles(asohf_ctx* c, int n, const float2** out) {
  if (c->tw_n != n) {
    ASOHF_CUDA(cudaStreamSynchronize(c->stream));
    cudaFree(c->d_tw);
    c->d_tw = nullptr;
    c->tw_n = 0;
    std::vector<float2> h((size_t)n);
    const double two_pi = 2.0 * acos(-1.0);
    for (int j = 0; j < n; j++) {
      const double a = two_pi * (double)j / (double)n;
      h[j] = make_float2((float)cos(a), (float)-sin(a));
    }
    h[0] = make_float2(1.f, 0.f);
    h[n / 4] = make_float2(0.f, -1.f);
    h[n / 2] = make_float2(-1.f, 0.f);
    h[3 * n / 4] = make_float2(0.f, 1.f);
    cudaError_t e = cudaMalloc(&c->d_tw, sizeof(float2) * (size_t)n);
    if (e == cudaSuccess) e = cudaMemcpy(c->d_tw, h.data(), sizeof(float2) * (size_t)n, cudaMemcpyHostToDevice);
    ASOHF_CUDA(e);
    c->tw_n = n;
  }
  *out = c->d_tw;
  return ASOHF_OK;
}

// The z pass on the context stream, on a half spectrum in the library 2-D
// transform's layout ([copy][z][ky][kx], NX/2+1 values per row, batch * NX
// planes): ASOHF_ERR_UNSUPPORTED unless NX is one of the sizes above and
// spec is 8-byte aligned.
int fftconv_z_green_2d(asohf_ctx* c, int nx, int batch, void* spec, const float* s2, float del2, float inv_n3) {
  if (nx != 64 && nx != 128 && nx != 256 && nx != 512) return ASOHF_ERR_UNSUPPORTED;
  if ((uintptr_t)spec & 7u) return ASOHF_ERR_UNSUPPORTED;
  const float2* tw;
  ASOHF_CHECK(twiddles(c, nx, &tw));
  float2* sp = (float2*)spec;
  int kt_ = ktime_begin(c, "fft_z_green");
  switch (nx) {
#define ZCASE(NN)                                                                                       \
  case NN:                                                                                              \
    ASOHF_CUDA(cudaFuncSetAttribute(k_fft_z_green<NN>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                    (int)Geo<NN>::ZSMEM));                                              \
    k_fft_z_green<NN><<<(unsigned)(batch * Geo<NN>::NCOL * (NN / Geo<NN>::TY)), Geo<NN>::ZT, Geo<NN>::ZSMEM, \
                        c->stream>>>(sp, tw, s2, del2, inv_n3);                                      \
    break;
    ZCASE(64)
    ZCASE(128)
    ZCASE(256)
    ZCASE(512)
#undef ZCASE
  }
  ktime_end(c, kt_);
  c->launches++;
  ASOHF_CUDA(cudaGetLastError());
  return ASOHF_OK;
}
