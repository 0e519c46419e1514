// sgt_fft.cuh -- grid-to-grid (G2G) step: aperiodic convolution of the
// charge grids with K(r) = (1 + h^2 |r|^2)^-2.
//
// The reference computes it as 2^d half-shifted size-N cyclic convolutions
// with cuFFT (CU/non_periodic_convF.cu:14-517, HYB/non_periodic_conv.cpp);
// the sum of those terms is exactly the aperiodic convolution.  Here the
// same convolution is one cyclic convolution of length M = 2^k >= 2N-1 per
// axis: for output nodes x < N only kernel offsets |x - x'| <= N-1 <= M/2
// are touched, so K_c[r] = K(min(r, M-r)) reproduces it.  Two real charge
// channels ride in one complex plane (K_c is real and even, so its FFT is
// real and the channels separate after the inverse transform).
//
// Each pass transforms blocks of SGT_FFT_LINES lines in shared memory with a
// radix-2 FFT written here (decimation in time for forward transforms with a
// bit-reversed load, decimation in frequency for inverse transforms with a
// bit-reversed read-out).  Lines along y/z are taken 8 adjacent x positions
// at a time so every global access is a 64-byte segment.  Planes of zero
// charge (index >= N) are never stored or read.  Passes are persistent
// (fixed grid, loop over work items sized from the device-side grid
// decision), so the chain replays inside a CUDA graph as N changes.
#pragma once
#include "sgt_common.cuh"

#define SGT_LS(M) ((M) + 1)  // padded line stride in float2

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// tw[j] = exp(-2 pi i j / M), j < M/2
__device__ __forceinline__ void fft_twiddles(float2 *tw, int M) {
  for (int j = threadIdx.x; j < (M >> 1); j += blockDim.x) {
    float s, c;
    sincospif(2.0f * (float)j / (float)M, &s, &c);
    tw[j] = make_float2(c, -s);
  }
}

__device__ __forceinline__ int brev(int x, int logM) {
  return (int)(__brev((unsigned)x) >> (32 - logM));
}

// forward DIT, bit-reversed input -> natural output
__device__ void fft_dit(float2 *buf, int lines, int M, int logM,
                        const float2 *tw) {
  const int half = M >> 1, ls = SGT_LS(M);
  for (int s = 0; s < logM; s++) {
    const int hs = 1 << s, tsh = logM - 1 - s;
    for (int b = threadIdx.x; b < lines * half; b += blockDim.x) {
      const int l = b >> (logM - 1), k = b & (half - 1);
      const int pos = k & (hs - 1);
      const int i0 = ((k >> s) << (s + 1)) + pos, i1 = i0 + hs;
      float2 *L = buf + l * ls;
      const float2 w = tw[pos << tsh];
      const float2 u = L[i0], v = cmul(L[i1], w);
      L[i0] = make_float2(u.x + v.x, u.y + v.y);
      L[i1] = make_float2(u.x - v.x, u.y - v.y);
    }
    __syncthreads();
  }
}

// inverse DIF (conjugate twiddles, no scaling), natural input ->
// bit-reversed output
__device__ void fft_dif_inv(float2 *buf, int lines, int M, int logM,
                            const float2 *tw) {
  const int half = M >> 1, ls = SGT_LS(M);
  for (int s = logM - 1; s >= 0; s--) {
    const int hs = 1 << s, tsh = logM - 1 - s;
    for (int b = threadIdx.x; b < lines * half; b += blockDim.x) {
      const int l = b >> (logM - 1), k = b & (half - 1);
      const int pos = k & (hs - 1);
      const int i0 = ((k >> s) << (s + 1)) + pos, i1 = i0 + hs;
      float2 *L = buf + l * ls;
      float2 w = tw[pos << tsh];
      w.y = -w.y;
      const float2 u = L[i0], v = L[i1];
      L[i0] = make_float2(u.x + v.x, u.y + v.y);
      L[i1] = cmul(make_float2(u.x - v.x, u.y - v.y), w);
    }
    __syncthreads();
  }
}

__device__ __forceinline__ float kern_val(float hsq, int M, int x, int y, int z) {
  const int dx = min(x, M - x), dy = min(y, M - y), dz = min(z, M - z);
  const float r2 = (float)(dx * dx + dy * dy + dz * dz);
  const float b = 1.0f + hsq * r2;
  return 1.0f / (b * b);
}

// number of data planes (complex) for d: pairs of the d+1 real channels
template <int D> struct Planes { static constexpr int n = D == 1 ? 1 : 2; };

template <int D>
__device__ __forceinline__ float2 node_plane(const typename Node<D>::T &v, int p) {
  if constexpr (D == 1) return v;
  else return p == 0 ? make_float2(v.x, v.y) : make_float2(v.z, D == 3 ? v.w : 0.f);
}

// ---------------------------------------------------------------------------
// d = 1: whole convolution in one CTA
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(SGT_THREADS)
k_conv1d(const SgtState *st, const float2 *__restrict__ V, float2 *__restrict__ Phi) {
  extern __shared__ float2 sm[];
  const int N = st->N, M = st->M, logM = st->logM;
  const float hsq = st->h_eff * st->h_eff;
  float2 *tw = sm, *bk = sm + 512, *bd = bk + SGT_LS(M);
  fft_twiddles(tw, M);
  for (int x = threadIdx.x; x < M; x += blockDim.x) {
    const int r = brev(x, logM);
    bk[r] = make_float2(kern_val(hsq, M, x, 0, 0), 0.f);
    bd[r] = x < N ? V[x] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_dit(bk, 1, M, logM, tw);
  fft_dit(bd, 1, M, logM, tw);
  for (int x = threadIdx.x; x < M; x += blockDim.x) {
    const float kr = bk[x].x;
    bd[x] = make_float2(bd[x].x * kr, bd[x].y * kr);
  }
  __syncthreads();
  fft_dif_inv(bd, 1, M, logM, tw);
  const float inv = 1.0f / (float)M;
  for (int x = threadIdx.x; x < N; x += blockDim.x) {
    const float2 v = bd[brev(x, logM)];
    Phi[x] = make_float2(v.x * inv, v.y * inv);
  }
}

// ---------------------------------------------------------------------------
// d >= 2, pass 1: build rows (x lines) of the data planes and of the kernel
// plane, forward FFT along x.
// W plane p at W + p*M^d; kernel plane index Planes<D>::n.
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_fft_build_x(const SgtState *st, const typename Node<D>::T *__restrict__ V,
              float2 *__restrict__ W) {
  extern __shared__ float2 sm[];
  const int N = st->N, M = st->M, logM = st->logM;
  const float hsq = st->h_eff * st->h_eff;
  constexpr int P = Planes<D>::n;
  const long plane = D == 2 ? (long)M * M : (long)M * M * M;
  float2 *tw = sm, *buf = sm + 512;
  fft_twiddles(tw, M);
  const int nyb_d = (N + SGT_FFT_LINES - 1) / SGT_FFT_LINES;
  const int nz_d = D == 3 ? N : 1;
  const int nyb_k = M / SGT_FFT_LINES;
  const int nz_k = D == 3 ? M : 1;
  const int items_d = P * nyb_d * nz_d, items = items_d + nyb_k * nz_k;
  const int ls = SGT_LS(M);
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    int p, z, y0;
    const bool isk = it >= items_d;
    if (!isk) {
      p = it / (nyb_d * nz_d);
      const int r = it % (nyb_d * nz_d);
      z = r / nyb_d;
      y0 = (r % nyb_d) * SGT_FFT_LINES;
    } else {
      p = P;
      const int r = it - items_d;
      z = r / nyb_k;
      y0 = (r % nyb_k) * SGT_FFT_LINES;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < SGT_FFT_LINES * M; e += blockDim.x) {
      const int l = e / M, x = e % M, y = y0 + l;
      float2 v = make_float2(0.f, 0.f);
      if (isk) {
        v.x = kern_val(hsq, M, x, y, z);
      } else if (y < N && x < N) {
        long g = x + (long)N * y;
        if (D == 3) g += (long)N * N * z;
        v = node_plane<D>(V[g], p);
      }
      buf[l * ls + brev(x, logM)] = v;
    }
    __syncthreads();
    fft_dit(buf, SGT_FFT_LINES, M, logM, tw);
    float2 *Wp = W + p * plane;
    const int ymax = isk ? M : N;
    for (int e = threadIdx.x; e < SGT_FFT_LINES * M; e += blockDim.x) {
      const int l = e / M, x = e % M, y = y0 + l;
      if (y < ymax) {
        long g = x + (long)M * y;
        if (D == 3) g += (long)M * M * z;
        Wp[g] = buf[l * ls + x];
      }
    }
  }
}

// Load 8 adjacent-x lines along an axis with stride `stride` (in float2),
// rows < lim valid (others zero), into buf in bit-reversed or natural order.
__device__ __forceinline__ void load_lines(float2 *buf, const float2 *src,
                                           long stride, int M, int logM,
                                           int lim, bool bitrev) {
  const int ls = SGT_LS(M);
  for (int e = threadIdx.x; e < SGT_FFT_LINES * M; e += blockDim.x) {
    const int l = e % SGT_FFT_LINES, t = e / SGT_FFT_LINES;
    const float2 v = t < lim ? src[(long)t * stride + l] : make_float2(0.f, 0.f);
    buf[l * ls + (bitrev ? brev(t, logM) : t)] = v;
  }
}
__device__ __forceinline__ void store_lines(const float2 *buf, float2 *dst,
                                            long stride, int M, int logM,
                                            int lim, bool bitrev) {
  const int ls = SGT_LS(M);
  for (int e = threadIdx.x; e < SGT_FFT_LINES * lim; e += blockDim.x) {
    const int l = e % SGT_FFT_LINES, t = e / SGT_FFT_LINES;
    dst[(long)t * stride + l] = buf[l * ls + (bitrev ? brev(t, logM) : t)];
  }
}

// ---------------------------------------------------------------------------
// d = 3, pass along y (forward: data planes z < N and kernel plane; inverse:
// data planes z < N, keeping y < N).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(SGT_THREADS)
k_fft_mid_y(const SgtState *st, float2 *__restrict__ W, int inverse) {
  extern __shared__ float2 sm[];
  const int N = st->N, M = st->M, logM = st->logM;
  const long plane = (long)M * M * M;
  float2 *tw = sm, *buf = sm + 512;
  fft_twiddles(tw, M);
  const int nxb = M / SGT_FFT_LINES;
  const int items_d = 2 * N * nxb;
  const int items = inverse ? items_d : items_d + M * nxb;
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    int p, z, xb;
    const bool isk = it >= items_d;
    if (!isk) {
      p = it / (N * nxb);
      const int r = it % (N * nxb);
      z = r / nxb;
      xb = r % nxb;
    } else {
      p = 2;
      const int r = it - items_d;
      z = r / nxb;
      xb = r % nxb;
    }
    float2 *base = W + p * plane + (long)M * M * z + xb * SGT_FFT_LINES;
    __syncthreads();
    if (!inverse) {
      load_lines(buf, base, M, M, logM, isk ? M : N, true);
      __syncthreads();
      fft_dit(buf, SGT_FFT_LINES, M, logM, tw);
      store_lines(buf, base, M, M, logM, M, false);
    } else {
      load_lines(buf, base, M, M, logM, M, false);
      __syncthreads();
      fft_dif_inv(buf, SGT_FFT_LINES, M, logM, tw);
      store_lines(buf, base, M, M, logM, N, true);
    }
  }
}

// ---------------------------------------------------------------------------
// last axis (y for d = 2, z for d = 3): kernel spectrum, data forward,
// pointwise product with Re(K^), inverse, keep positions < N.
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_fft_last(const SgtState *st, float2 *__restrict__ W) {
  extern __shared__ float2 sm[];
  const int N = st->N, M = st->M, logM = st->logM;
  const long plane = D == 2 ? (long)M * M : (long)M * M * M;
  const long stride = D == 2 ? (long)M : (long)M * M;
  float2 *tw = sm, *bk = sm + 512, *bd = bk + SGT_FFT_LINES * SGT_LS(M);
  fft_twiddles(tw, M);
  const int nxb = M / SGT_FFT_LINES;
  const int items = D == 2 ? nxb : nxb * M;
  const int ls = SGT_LS(M);
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    const int xb = it % nxb, y = it / nxb;  // y used for d = 3
    const long off = xb * SGT_FFT_LINES + (D == 3 ? (long)M * y : 0);
    __syncthreads();
    load_lines(bk, W + 2 * plane + off, stride, M, logM, M, true);  // kernel plane
    __syncthreads();
    fft_dit(bk, SGT_FFT_LINES, M, logM, tw);
    for (int p = 0; p < 2; p++) {
      float2 *base = W + p * plane + off;
      load_lines(bd, base, stride, M, logM, N, true);
      __syncthreads();
      fft_dit(bd, SGT_FFT_LINES, M, logM, tw);
      for (int e = threadIdx.x; e < SGT_FFT_LINES * M; e += blockDim.x) {
        const int l = e / M, t = e % M;
        const float kr = bk[l * ls + t].x;
        const float2 v = bd[l * ls + t];
        bd[l * ls + t] = make_float2(v.x * kr, v.y * kr);
      }
      __syncthreads();
      fft_dif_inv(bd, SGT_FFT_LINES, M, logM, tw);
      store_lines(bd, base, stride, M, logM, N, true);
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// final pass: inverse FFT along x of rows y (, z) < N, scale by 1/M^d and
// write the potential grid (channels packed per node).
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_fft_final_x(const SgtState *st, const float2 *__restrict__ W,
              typename Node<D>::T *__restrict__ Phi) {
  extern __shared__ float2 sm[];
  const int N = st->N, M = st->M, logM = st->logM;
  const long plane = D == 2 ? (long)M * M : (long)M * M * M;
  float2 *tw = sm, *b0 = sm + 512, *b1 = b0 + SGT_FFT_LINES * SGT_LS(M);
  fft_twiddles(tw, M);
  const int nyb = (N + SGT_FFT_LINES - 1) / SGT_FFT_LINES;
  const int items = nyb * (D == 3 ? N : 1);
  const int ls = SGT_LS(M);
  float inv = 1.0f / (float)M;
  inv = inv / (float)M;
  if (D == 3) inv = inv / (float)M;
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    const int y0 = (it % nyb) * SGT_FFT_LINES, z = it / nyb;
    __syncthreads();
    for (int e = threadIdx.x; e < SGT_FFT_LINES * M; e += blockDim.x) {
      const int l = e / M, x = e % M, y = y0 + l;
      float2 v0 = make_float2(0.f, 0.f), v1 = v0;
      if (y < N) {
        long g = x + (long)M * y + (D == 3 ? (long)M * M * z : 0);
        v0 = W[g];
        v1 = W[plane + g];
      }
      b0[l * ls + x] = v0;
      b1[l * ls + x] = v1;
    }
    __syncthreads();
    fft_dif_inv(b0, SGT_FFT_LINES, M, logM, tw);
    fft_dif_inv(b1, SGT_FFT_LINES, M, logM, tw);
    for (int e = threadIdx.x; e < SGT_FFT_LINES * N; e += blockDim.x) {
      const int l = e / N, x = e % N, y = y0 + l;
      if (y >= N) continue;
      const float2 a = b0[l * ls + brev(x, logM)];
      const float2 b = b1[l * ls + brev(x, logM)];
      long g = x + (long)N * y + (D == 3 ? (long)N * N * z : 0);
      Phi[g] = make_float4(a.x * inv, a.y * inv, b.x * inv, b.y * inv);
    }
  }
}
