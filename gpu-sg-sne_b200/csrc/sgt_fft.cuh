// sgt_fft.cuh -- grid-to-grid (G2G) step: aperiodic convolution of the
// charge grids with K(r) = (1 + h^2 |r|^2)^-2.
//
// The reference computes it as 2^d half-shifted size-N cyclic convolutions
// with cuFFT (CU/non_periodic_convF.cu:14-517, HYB/non_periodic_conv.cpp);
// the sum of those terms is exactly the aperiodic convolution.  Here the
// same convolution is one cyclic convolution of length M >= 2N-1 per axis
// (the smallest M = 2^k or 3 * 2^k): output nodes x < N only meet kernel
// offsets |x - x'| <= N-1 <= M/2, so K_c[r] = K(min(r, M-r)) reproduces it.  Two real charge channels ride in
// one complex plane (K_c is real and even, so its transform is real and the
// channels separate after the inverse).
//
// FFTs are register-resident: one warp owns one line of M <= 1024 points, a
// lane holds the E = M/32 points lane + 32 e; butterflies whose span holds
// whole lanes (and the radix-3 stage of M = 3 * 2^k) stay inside a lane,
// shorter spans use warp shuffles.  Forward transforms are decimation in
// frequency (natural order in, digit-reversed out) and inverse transforms
// decimation in time (digit-reversed in, natural out), so spectra stay in
// that order in memory and no permutation pass exists.  Rows
// are read and written directly (coalesced); columns go through a shared
// memory transpose of 8 adjacent columns so every global access is a 64-byte
// segment.  Planes of zero charge (index >= N) are never stored or read.
// Kernels are persistent and size their work from the device-side grid
// decision, so the chain replays inside a CUDA graph as N changes.
#pragma once
#include "sgt_common.cuh"

#define SGT_FFT_COLS 8  // columns per CTA in column passes (one per warp)
#define SGT_FFT_PAD 1   // float2 padding per staged column
#define SGT_FFT_MAXM 1024  // longest FFT: twiddle tables hold M entries
// d = 2 grids with M <= SGT_FFT_SMALL_M: the whole convolution runs in one CTA
// in shared memory (conv2d_small_body), and the row passes return at once
#define SGT_FFT_SMALL_M 64

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 shfl_x2(float2 v, int m) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// tw[j] = exp(-2 pi i j / M), j < M (accurate sincospi)
__device__ __forceinline__ void fft_twiddles(float2 *tw, int M) {
  for (int j = threadIdx.x; j < M; j += blockDim.x) {
    float s, c;
    sincospif(2.0f * (float)j / (float)M, &s, &c);
    tw[j] = make_float2(c, -s);
  }
}

// FFT lengths: 2^k or 3 * 2^k, 32 <= M <= 1024.  A lane holds E = M/32
// points, lane + 32 e.  Forward (DIF): radix-2 stages whose span holds whole
// lanes (span >= 32, or >= 96 when M has the factor 3) run inside the lane;
// for M = 3 * 2^k a radix-3 stage at span 32 follows, also inside the lane
// (elements e, e+1, e+2 of a 96-point block, then twiddles W_96^(lane k));
// the last five radix-2 stages (spans 16 .. 1) exchange between lanes by
// shuffles.  The output order is the digit reversal these stages imply; the
// inverse (DIT, conjugate twiddles, unscaled) applies the same stages in
// reverse order and takes that order back to natural order, so spectra are
// only ever multiplied pointwise in the permuted order.
template <int M>
struct FftLen {
  static constexpr bool R3 = (M % 3) == 0;
  static constexpr int E = M / 32;
  static constexpr int LANE_MIN = R3 ? 96 : 32;  // smallest in-lane radix-2 span
};

template <int M>
__device__ __forceinline__ void wfft_dif(float2 *v, const float2 *__restrict__ tw) {
  constexpr int E = FftLen<M>::E;
  const int lane = threadIdx.x & 31;
  // in-lane radix-2 stages
#pragma unroll
  for (int hs = M / 2; hs >= FftLen<M>::LANE_MIN; hs /= 2) {
    if ((hs & 31) != 0) continue;
    const int he = hs / 32, stride = M / (2 * hs);
#pragma unroll
    for (int e = 0; e < E; e++) {
      if ((e / he) % 2 == 0) {
        const float2 w = tw[((lane + 32 * e) % hs) * stride];
        const float2 u = v[e], t = v[e + he];
        v[e] = cadd(u, t);
        v[e + he] = cmul(csub(u, t), w);
      }
    }
  }
  if constexpr (FftLen<M>::R3) {
    // radix 3 over elements e, e+1, e+2 (positions i, i+32, i+64 of a
    // 96-point block), then twiddles W_96^(lane k)
    const float s3 = 0.8660254037844386f;  // sqrt(3)/2
    const float2 w1 = tw[lane * (M / 96)], w2 = tw[2 * lane * (M / 96)];
#pragma unroll
    for (int e = 0; e < E; e += 3) {
      const float2 a = v[e], b = v[e + 1], c = v[e + 2];
      const float2 sm = cadd(b, c), df = csub(b, c);
      const float2 t = make_float2(a.x - 0.5f * sm.x, a.y - 0.5f * sm.y);
      const float2 u = make_float2(s3 * df.y, -s3 * df.x);  // -i sqrt(3)/2 (b - c)
      v[e] = cadd(a, sm);
      v[e + 1] = cmul(cadd(t, u), w1);
      v[e + 2] = cmul(csub(t, u), w2);
    }
  }
  // shuffle radix-2 stages, spans 16 .. 1
#pragma unroll
  for (int hs = 16; hs >= 1; hs /= 2) {
    const bool upper = (lane & hs) != 0;
    const float2 w = tw[(lane & (hs - 1)) * (M / (2 * hs))];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const float2 x = v[e], y = shfl_x2(x, hs);
      v[e] = upper ? cmul(csub(y, x), w) : cadd(x, y);
    }
  }
}

template <int M>
__device__ __forceinline__ void wfft_dit_inv(float2 *v, const float2 *__restrict__ tw) {
  constexpr int E = FftLen<M>::E;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int hs = 1; hs <= 16; hs *= 2) {
    const bool upper = (lane & hs) != 0;
    float2 w = tw[(lane & (hs - 1)) * (M / (2 * hs))];
    w.y = -w.y;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const float2 x = v[e], y = shfl_x2(x, hs);
      v[e] = upper ? csub(y, cmul(x, w)) : cadd(x, cmul(y, w));
    }
  }
  if constexpr (FftLen<M>::R3) {
    const float s3 = 0.8660254037844386f;
    float2 w1 = tw[lane * (M / 96)], w2 = tw[2 * lane * (M / 96)];
    w1.y = -w1.y;
    w2.y = -w2.y;
#pragma unroll
    for (int e = 0; e < E; e += 3) {
      const float2 a = v[e], b = cmul(v[e + 1], w1), c = cmul(v[e + 2], w2);
      const float2 sm = cadd(b, c), df = csub(b, c);
      const float2 t = make_float2(a.x - 0.5f * sm.x, a.y - 0.5f * sm.y);
      const float2 u = make_float2(-s3 * df.y, s3 * df.x);  // +i sqrt(3)/2 (b - c)
      v[e] = cadd(a, sm);
      v[e + 1] = cadd(t, u);
      v[e + 2] = csub(t, u);
    }
  }
#pragma unroll
  for (int hs = FftLen<M>::LANE_MIN; hs <= M / 2; hs *= 2) {
    if ((hs & 31) != 0) continue;
    const int he = hs / 32, stride = M / (2 * hs);
#pragma unroll
    for (int e = 0; e < E; e++) {
      if ((e / he) % 2 == 0) {
        float2 w = tw[((lane + 32 * e) % hs) * stride];
        w.y = -w.y;
        const float2 u = v[e], t = cmul(v[e + he], w);
        v[e] = cadd(u, t);
        v[e + he] = csub(u, t);
      }
    }
  }
}

__device__ __forceinline__ float kern_val(float hsq, int M, int x, int y, int z) {
  const int dx = min(x, M - x), dy = min(y, M - y), dz = min(z, M - z);
  const float r2 = (float)(dx * dx + dy * dy + dz * dz);
  const float b = 1.0f + hsq * r2;
  return 1.0f / (b * b);
}

template <int D>
__device__ __forceinline__ float2 node_plane(const typename Node<D>::T &v, int p) {
  if constexpr (D == 1) return v;
  else return p == 0 ? make_float2(v.x, v.y) : make_float2(v.z, D == 3 ? v.w : 0.f);
}

// the FFT lengths the grid decision picks (sgt_fft_length)
#define SGT_FFT_DISPATCH(M_EXPR, CALL)            \
  switch (M_EXPR) {                               \
    case 32: CALL(32); break;                     \
    case 64: CALL(64); break;                     \
    case 96: CALL(96); break;                     \
    case 128: CALL(128); break;                   \
    case 192: CALL(192); break;                   \
    case 256: CALL(256); break;                   \
    case 384: CALL(384); break;                   \
    case 512: CALL(512); break;                   \
    case 768: CALL(768); break;                   \
    default: CALL(1024); break;                   \
  }

// ---------------------------------------------------------------------------
// d = 1: the whole convolution in one warp
// ---------------------------------------------------------------------------
template <int M>
__device__ void conv1d_body(const SgtState *st, const float2 *__restrict__ V, float2 *__restrict__ Phi,
                            const float2 *tw) {
  constexpr int E = M / 32;
  const int N = st->N, lane = threadIdx.x & 31;
  const float hsq = st->h_eff * st->h_eff;
  float2 k[E], v[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int x = lane + 32 * e;
    k[e] = make_float2(kern_val(hsq, M, x, 0, 0), 0.f);
    v[e] = x < N ? V[x] : make_float2(0.f, 0.f);
  }
  wfft_dif<M>(k, tw);
  wfft_dif<M>(v, tw);
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = make_float2(v[e].x * k[e].x, v[e].y * k[e].x);
  wfft_dit_inv<M>(v, tw);
  const float inv = 1.0f / (float)M;
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int x = lane + 32 * e;
    if (x < N) Phi[x] = make_float2(v[e].x * inv, v[e].y * inv);
  }
}

__device__ __forceinline__ void k_conv1d_body(int vb_, int vg_, const SgtState *st, const float2 *__restrict__ V, float2 *__restrict__ Phi) {
  sgt_pdl_wait();
  __shared__ float2 tw[SGT_FFT_MAXM];
  fft_twiddles(tw, st->M);
  __syncthreads();
  if (threadIdx.x >= 32) return;
#define C1(L) conv1d_body<L>(st, V, Phi, tw)
  SGT_FFT_DISPATCH(st->M, C1)
#undef C1
}
__global__ void __launch_bounds__(SGT_THREADS)
k_conv1d(const SgtState *st, const float2 *__restrict__ V, float2 *__restrict__ Phi) {
  k_conv1d_body(blockIdx.x, gridDim.x, st, V, Phi);
}

// ---------------------------------------------------------------------------
// d >= 2, pass 1: build rows (x lines) of the data planes (rows y, z < N) and
// of the kernel plane (all rows), forward FFT along x.
// W plane p at W + p * M^d; the kernel plane is p = 2.
// ---------------------------------------------------------------------------
template <int D, int M>
__device__ void build_rows_body(int vb_, int vg_, const SgtState *st, const typename Node<D>::T *__restrict__ V,
                                float2 *__restrict__ W, const float2 *tw) {
  constexpr int E = M / 32;
  const int N = st->N, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float hsq = st->h_eff * st->h_eff;
  const long plane = D == 2 ? (long)M * M : (long)M * M * M;
  const int nz_d = D == 3 ? N : 1, nz_k = D == 3 ? M : 1;
  const long lines_d = 2L * N * nz_d, lines = lines_d + (long)M * nz_k;
  const int wpb = blockDim.x >> 5;
  for (long ln = (long)vb_ * wpb + warp; ln < lines; ln += (long)vg_ * wpb) {
    float2 v[E];
    int p, y, z;
    if (ln < lines_d) {
      p = (int)(ln / ((long)N * nz_d));
      const long r = ln % ((long)N * nz_d);
      z = (int)(r / N);
      y = (int)(r % N);
#pragma unroll
      for (int e = 0; e < E; e++) {
        const int x = lane + 32 * e;
        v[e] = x < N ? node_plane<D>(V[x + (long)N * y + (D == 3 ? (long)N * N * z : 0)], p)
                     : make_float2(0.f, 0.f);
      }
    } else {
      p = 2;
      const long r = ln - lines_d;
      z = (int)(r / M);
      y = (int)(r % M);
#pragma unroll
      for (int e = 0; e < E; e++) v[e] = make_float2(kern_val(hsq, M, lane + 32 * e, y, z), 0.f);
    }
    wfft_dif<M>(v, tw);
    float2 *row = W + p * plane + (long)M * y + (D == 3 ? (long)M * M * z : 0);
#pragma unroll
    for (int e = 0; e < E; e++) row[lane + 32 * e] = v[e];
  }
}

template <int D>
__device__ __forceinline__ void k_fft_build_x_body(int vb_, int vg_, const SgtState *st, const typename Node<D>::T *__restrict__ V, float2 *__restrict__ W) {
  sgt_pdl_wait();
  __shared__ float2 tw[SGT_FFT_MAXM];
  if (D == 2 && st->M <= SGT_FFT_SMALL_M) return;  // the column pass does it all
  fft_twiddles(tw, st->M);
  __syncthreads();
#define CB(L) build_rows_body<D, L>(vb_, vg_, st, V, W, tw)
  SGT_FFT_DISPATCH(st->M, CB)
#undef CB
}
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_fft_build_x(const SgtState *st, const typename Node<D>::T *__restrict__ V, float2 *__restrict__ W) {
  k_fft_build_x_body<D>(blockIdx.x, gridDim.x, st, V, W);
}

// ---------------------------------------------------------------------------
// d = 2, M <= SGT_FFT_SMALL_M: the three passes below in one CTA, with the
// planes in shared memory (rows padded to M + 1 points so that the column
// reads of the lanes fall in distinct banks).  The same transforms, products
// and scaling in the same order as the multi-CTA passes, so the potentials
// are the same; small grids (the h-driven grids of most runs) save two
// passes through global memory and the launch latency between them.
// Shared memory: twiddles (M), the kernel plane (M rows), the data planes
// (2 x N rows, N <= M / 2).
// ---------------------------------------------------------------------------
template <int M>
__device__ void conv2d_small_body(const SgtState *st, const float4 *__restrict__ V,
                                  float2 *__restrict__ Phi2, float2 *sm) {
  constexpr int E = M / 32, LS = M + 1;
  const int N = st->N, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const float hsq = st->h_eff * st->h_eff;
  float2 *tw = sm;
  float2 *kp = sm + M;
  float2 *dp = kp + M * LS;  // plane p, row y at dp + (p N + y) LS
  fft_twiddles(tw, M);
  __syncthreads();
  // rows along x: the kernel plane (all M rows), the data planes (y < N)
  for (int ln = warp; ln < M + 2 * N; ln += nw) {
    float2 v[E];
    float2 *row;
    if (ln < M) {
#pragma unroll
      for (int e = 0; e < E; e++) v[e] = make_float2(kern_val(hsq, M, lane + 32 * e, ln, 0), 0.f);
      row = kp + ln * LS;
    } else {
      const int r = ln - M, p = r / N, y = r % N;
#pragma unroll
      for (int e = 0; e < E; e++) {
        const int x = lane + 32 * e;
        v[e] = x < N ? node_plane<2>(V[x + (long)N * y], p) : make_float2(0.f, 0.f);
      }
      row = dp + (p * N + y) * LS;
    }
    wfft_dif<M>(v, tw);
#pragma unroll
    for (int e = 0; e < E; e++) row[lane + 32 * e] = v[e];
  }
  __syncthreads();
  // columns along y: the kernel spectrum (real part), then per data plane
  // forward, product, inverse; rows y >= N of the data are zero and dropped
  for (int c = warp; c < M; c += nw) {
    float2 v[E];
    float kr[E];
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = kp[(lane + 32 * e) * LS + c];
    wfft_dif<M>(v, tw);
#pragma unroll
    for (int e = 0; e < E; e++) kr[e] = v[e].x;
    for (int p = 0; p < 2; p++) {
#pragma unroll
      for (int e = 0; e < E; e++) {
        const int y = lane + 32 * e;
        v[e] = y < N ? dp[(p * N + y) * LS + c] : make_float2(0.f, 0.f);
      }
      wfft_dif<M>(v, tw);
#pragma unroll
      for (int e = 0; e < E; e++) v[e] = make_float2(v[e].x * kr[e], v[e].y * kr[e]);
      wfft_dit_inv<M>(v, tw);
#pragma unroll
      for (int e = 0; e < E; e++) {
        const int y = lane + 32 * e;
        if (y < N) dp[(p * N + y) * LS + c] = v[e];
      }
    }
  }
  __syncthreads();
  // rows inverse along x, scaled by 1/M^2, into the potential grid
  float inv = 1.0f / (float)M;
  inv = inv / (float)M;
  for (int ln = warp; ln < 2 * N; ln += nw) {
    const int p = ln % 2, y = ln / 2;
    float2 v[E];
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = dp[(p * N + y) * LS + lane + 32 * e];
    wfft_dit_inv<M>(v, tw);
    const long g0 = (long)N * y;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int x = lane + 32 * e;
      if (x < N) Phi2[2 * (g0 + x) + p] = make_float2(v[e].x * inv, v[e].y * inv);
    }
  }
}

// ---------------------------------------------------------------------------
// column passes: 8 adjacent columns per CTA staged through shared memory.
// MODE_LAST: last axis (y for d = 2, z for d = 3): kernel spectrum, data
//            forward, product with Re(K^), inverse, keep positions < N.
// MODE_MID_FWD / MODE_MID_INV: d = 3, axis y of the data planes z < N (and of
//            the kernel plane on the forward pass).
// ---------------------------------------------------------------------------
#define MODE_LAST 0
#define MODE_MID_FWD 1
#define MODE_MID_INV 2

template <int M>
__device__ __forceinline__ void stage_load(float2 *stg, const float2 *__restrict__ src, long stride,
                                           int lim) {
  constexpr int LS = M + SGT_FFT_PAD;
  for (int idx = threadIdx.x; idx < SGT_FFT_COLS * M; idx += blockDim.x) {
    const int t = idx / SGT_FFT_COLS, c = idx % SGT_FFT_COLS;
    stg[c * LS + t] = t < lim ? src[(long)t * stride + c] : make_float2(0.f, 0.f);
  }
}
template <int M>
__device__ __forceinline__ void stage_store(const float2 *stg, float2 *__restrict__ dst, long stride,
                                            int lim) {
  constexpr int LS = M + SGT_FFT_PAD;
  for (int idx = threadIdx.x; idx < SGT_FFT_COLS * lim; idx += blockDim.x) {
    const int t = idx / SGT_FFT_COLS, c = idx % SGT_FFT_COLS;
    dst[(long)t * stride + c] = stg[c * LS + t];
  }
}

template <int D, int MODE, int M>
__device__ void cols_body(int vb_, int vg_, const SgtState *st, float2 *__restrict__ W, const float2 *tw,
                          float2 *stg, float *kre) {
  constexpr int E = M / 32, LS = M + SGT_FFT_PAD;
  const int N = st->N, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long plane = D == 2 ? (long)M * M : (long)M * M * M;
  const int ncb = M / SGT_FFT_COLS;
  // last pass: lines along y (d = 2, stride M) or z (d = 3, stride M^2)
  const long stride = (MODE == MODE_LAST && D == 3) ? (long)M * M : (long)M;
  long items;
  if (MODE == MODE_LAST) items = D == 2 ? ncb : (long)ncb * M;  // d = 3: every y
  else if (MODE == MODE_MID_FWD) items = (long)ncb * (2L * N + M);  // data z < N, kernel all z
  else items = (long)ncb * 2L * N;
  float2 v[E];
  for (long it = vb_; it < items; it += vg_) {
    const int cb = (int)(it % ncb);
    const long rest = it / ncb;
    __syncthreads();
    if (MODE == MODE_LAST) {
      const long off = (long)cb * SGT_FFT_COLS + (D == 3 ? (long)M * rest : 0);
      // kernel spectrum of the 8 columns, real part kept
      stage_load<M>(stg, W + 2 * plane + off, stride, M);
      __syncthreads();
#pragma unroll
      for (int e = 0; e < E; e++) v[e] = stg[warp * LS + lane + 32 * e];
      wfft_dif<M>(v, tw);
#pragma unroll
      for (int e = 0; e < E; e++) kre[warp * M + lane + 32 * e] = v[e].x;
      for (int p = 0; p < 2; p++) {
        float2 *base = W + p * plane + off;
        __syncthreads();
        stage_load<M>(stg, base, stride, N);
        __syncthreads();
#pragma unroll
        for (int e = 0; e < E; e++) v[e] = stg[warp * LS + lane + 32 * e];
        wfft_dif<M>(v, tw);
#pragma unroll
        for (int e = 0; e < E; e++) {
          const float kr = kre[warp * M + lane + 32 * e];
          v[e] = make_float2(v[e].x * kr, v[e].y * kr);
        }
        wfft_dit_inv<M>(v, tw);
#pragma unroll
        for (int e = 0; e < E; e++) stg[warp * LS + lane + 32 * e] = v[e];
        __syncthreads();
        stage_store<M>(stg, base, stride, N);
      }
    } else {
      int p, z;
      if (rest < 2L * N) {
        p = (int)(rest / N);
        z = (int)(rest % N);
      } else {
        p = 2;
        z = (int)(rest - 2L * N);
      }
      float2 *base = W + p * plane + (long)M * M * z + (long)cb * SGT_FFT_COLS;
      if (MODE == MODE_MID_FWD) {
        stage_load<M>(stg, base, M, p == 2 ? M : N);
        __syncthreads();
#pragma unroll
        for (int e = 0; e < E; e++) v[e] = stg[warp * LS + lane + 32 * e];
        wfft_dif<M>(v, tw);
#pragma unroll
        for (int e = 0; e < E; e++) stg[warp * LS + lane + 32 * e] = v[e];
        __syncthreads();
        stage_store<M>(stg, base, M, M);
      } else {
        stage_load<M>(stg, base, M, M);
        __syncthreads();
#pragma unroll
        for (int e = 0; e < E; e++) v[e] = stg[warp * LS + lane + 32 * e];
        wfft_dit_inv<M>(v, tw);
#pragma unroll
        for (int e = 0; e < E; e++) stg[warp * LS + lane + 32 * e] = v[e];
        __syncthreads();
        stage_store<M>(stg, base, M, N);
      }
    }
  }
}

template <int D, int MODE>
__device__ __forceinline__ void k_fft_cols_body(int vb_, int vg_, const SgtState *st, float2 *__restrict__ W,
                                                const typename Node<D>::T *__restrict__ V,
                                                typename Node<D>::T *__restrict__ Phi) {
  sgt_pdl_wait();
  extern __shared__ float2 sm[];
  if constexpr (D == 2 && MODE == MODE_LAST) {
    if (st->M <= SGT_FFT_SMALL_M) {  // block-uniform
      if (vb_ == 0) {
        if (st->M == 32) conv2d_small_body<32>(st, V, reinterpret_cast<float2 *>(Phi), sm);
        else conv2d_small_body<64>(st, V, reinterpret_cast<float2 *>(Phi), sm);
      }
      return;
    }
  }
  float2 *tw = sm;
  float2 *stg = sm + SGT_FFT_MAXM;
  float *kre = reinterpret_cast<float *>(stg + SGT_FFT_COLS * (st->M + SGT_FFT_PAD));
  fft_twiddles(tw, st->M);
  __syncthreads();
#define CC(L) cols_body<D, MODE, L>(vb_, vg_, st, W, tw, stg, kre)
  SGT_FFT_DISPATCH(st->M, CC)
#undef CC
}
template <int D, int MODE>
__global__ void __launch_bounds__(SGT_THREADS)
k_fft_cols(const SgtState *st, float2 *__restrict__ W, const typename Node<D>::T *__restrict__ V,
           typename Node<D>::T *__restrict__ Phi) {
  k_fft_cols_body<D, MODE>(blockIdx.x, gridDim.x, st, W, V, Phi);
}

// ---------------------------------------------------------------------------
// final pass: inverse FFT along x of rows y (, z) < N, scale by 1/M^d, write
// the potential grid (channels packed per node: plane 0 -> .xy, 1 -> .zw).
// ---------------------------------------------------------------------------
template <int D, int M>
__device__ void final_rows_body(int vb_, int vg_, const SgtState *st, const float2 *__restrict__ W,
                                float2 *__restrict__ Phi2, const float2 *tw) {
  constexpr int E = M / 32;
  const int N = st->N, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long plane = D == 2 ? (long)M * M : (long)M * M * M;
  const long lines = 2L * N * (D == 3 ? N : 1);
  const int wpb = blockDim.x >> 5;
  float inv = 1.0f / (float)M;
  inv = inv / (float)M;
  if (D == 3) inv = inv / (float)M;
  for (long ln = (long)vb_ * wpb + warp; ln < lines; ln += (long)vg_ * wpb) {
    const int p = (int)(ln % 2);
    const long r = ln / 2;
    const int y = (int)(r % N), z = D == 3 ? (int)(r / N) : 0;
    const float2 *row = W + p * plane + (long)M * y + (D == 3 ? (long)M * M * z : 0);
    float2 v[E];
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = row[lane + 32 * e];
    wfft_dit_inv<M>(v, tw);
    const long g0 = (long)N * y + (D == 3 ? (long)N * N * z : 0);
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int x = lane + 32 * e;
      if (x < N) Phi2[2 * (g0 + x) + p] = make_float2(v[e].x * inv, v[e].y * inv);
    }
  }
}

template <int D>
__device__ __forceinline__ void k_fft_final_x_body(int vb_, int vg_, const SgtState *st, const float2 *__restrict__ W, typename Node<D>::T *__restrict__ Phi) {
  sgt_pdl_wait();
  __shared__ float2 tw[SGT_FFT_MAXM];
  if (D == 2 && st->M <= SGT_FFT_SMALL_M) return;  // the column pass did it all
  fft_twiddles(tw, st->M);
  __syncthreads();
#define CF(L) final_rows_body<D, L>(vb_, vg_, st, W, reinterpret_cast<float2 *>(Phi), tw)
  SGT_FFT_DISPATCH(st->M, CF)
#undef CF
}
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_fft_final_x(const SgtState *st, const float2 *__restrict__ W, typename Node<D>::T *__restrict__ Phi) {
  k_fft_final_x_body<D>(blockIdx.x, gridDim.x, st, W, Phi);
}

// shared memory of a column pass for FFT length Mmax; in d = 2 also enough
// for the one-CTA convolution of the small lengths that Mmax admits
__host__ __device__ inline size_t fft_cols_smem(int Mmax, int d = 3) {
  size_t b = sizeof(float2) * (SGT_FFT_MAXM + (size_t)SGT_FFT_COLS * (Mmax + SGT_FFT_PAD)) +
             sizeof(float) * (size_t)SGT_FFT_COLS * Mmax;
  if (d == 2) {
    const size_t m = Mmax < SGT_FFT_SMALL_M ? (size_t)Mmax : (size_t)SGT_FFT_SMALL_M;
    const size_t small = sizeof(float2) * (m + m * (m + 1) + m * (m + 1));  // twiddles, kernel, 2 x m/2 data rows
    if (small > b) b = small;
  }
  return b;
}
