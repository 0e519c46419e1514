// sgt_common.cuh -- shared device types and helpers of the SG-t-SNE engine.
//
// Data layout in HBM (per embedding):
//   Y, Ynext, uY, gains, Frep  : point-major, padded stride S = 1,2,4 for
//                                d = 1,2,3 (one 4/8/16-byte load per point)
//   P (CSR)                    : rowptr int32[n+1], pairs int2[nnz]
//                                (.x = column, .y = float bits of p_ij)
//   grids V / PhiGrid          : node-major, channels packed in one float2
//                                (d=1) or float4 (d=2,3) per node, x fastest
//   FFT workspace              : NCH complex planes of M^d float2, x fastest
// All scalars that change per iteration (grid size, h, Z, means, alpha,
// momentum) live in one device-resident SgtState so a captured CUDA graph
// replays the whole iteration without host round trips.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define SGT_MAX_GRID 512        // largest grid (points per axis) of the size table
#define SGT_FFT_LINES 8         // lines per CTA in the FFT axis passes
#define SGT_THREADS 256

// Lagrange cubic weights on 4 nodes (CU/gridding.cuh:13-22,
// HYB/gridding.cpp:29-39).  Node f+a gets w[a]; the point lies between
// nodes f+1 and f+2.
__device__ __forceinline__ float sgt_l1(float x) {
  return 0.5f * x * x * x - 1.0f * x * x - 0.5f * x + 1.0f;
}
__device__ __forceinline__ float sgt_l2(float x) {
  const float cc = 1.0f / 6.0f;
  return -cc * x * x * x + 1.0f * x * x - 11.0f * cc * x + 1.0f;
}
__device__ __forceinline__ void sgt_weights(float s, int &f, float w[4]) {
  const float fl = floorf(s);
  f = (int)fl;
  const float dd = s - fl;
  w[0] = sgt_l2(1.0f + dd);
  w[1] = sgt_l1(dd);
  w[2] = sgt_l1(1.0f - dd);
  w[3] = sgt_l2(2.0f - dd);
}

// Per-embedding device state.  Written by the last CTA of the kernel that
// produces a value, read by the kernels that follow.
struct SgtState {
  // grid of the current iteration
  float miny[4];     // per-dim min of the centred coordinates (init 100.0)
  float mean[4];     // mean subtracted from Ynext when forming Y
  float maxy;        // max shifted coordinate over all dims
  float scale;       // float(N - 3): scaled coords lie in [0, N-3)
  float h_eff;       // grid spacing in embedding units
  int N;             // grid points per axis (n1 + 2)
  int M;             // FFT length per axis (2^k or 3 * 2^k, >= 2N-1)
  int T;             // tile edge in cells
  int tiles_dim;     // tiles per axis
  int ntiles;
  int nchunks;
  int chunk;         // points per chunk
  int grid_clamped;  // 1 if N was clamped to the allocated FFT size
  // reductions
  double Z;
  double sum[4];
  float minv[4], maxv[4];
  // schedule
  int iter;
  float alpha;
  float momentum;
  // counters for last-block reductions (reset by the block that finishes)
  unsigned int done_g2s;
  unsigned int done_row;
  unsigned int done_kl;
  unsigned int done_init;
  unsigned int done_bin;
  double kl;
  int error;
};

// Parameters fixed for a job (passed by value to kernels).
struct SgtJobParams {
  int n;
  int d;
  int grid_mode;      // 0: h-driven + per-iteration centring, 1: fixed grid
  int n1_fixed;       // inner grid size in fixed mode
  float h;            // target grid spacing (h mode)
  float alpha0;       // early exaggeration
  int early_iter;     // last iteration (inclusive) using alpha0
  int mom_switch;     // last iteration (inclusive) using momentum 0.5
  float eta;
  int mmax;           // largest FFT length per axis allocated
  int tile_cap;       // max tiles held by the tile arrays
  int chunk_cap;      // max chunks held by the chunk array
  int chunk_min;      // fewest points per S2G chunk (0: 1024, 256 in 3-D)
  int direct_max;     // largest N of a direct-mode grid (0: no direct mode)
};

// Direct mode (d <= 2): S2G and G2S work on the points in their own order
// with the whole grid in shared memory, without the tile sort, on grids that
// are not dense enough for cell mode.  2-D grids up to this many points per
// axis (64^2 float4 nodes = 64 KB); 1-D grids always.
#define SGT_DIRECT_N2 64

template <int D> struct Vec;
template <> struct Vec<1> { typedef float T; };
template <> struct Vec<2> { typedef float2 T; };
template <> struct Vec<3> { typedef float4 T; };

template <int D>
__device__ __forceinline__ float comp(const typename Vec<D>::T &v, int k);
template <> __device__ __forceinline__ float comp<1>(const float &v, int) { return v; }
template <> __device__ __forceinline__ float comp<2>(const float2 &v, int k) {
  return k == 0 ? v.x : v.y;
}
template <> __device__ __forceinline__ float comp<3>(const float4 &v, int k) {
  return k == 0 ? v.x : (k == 1 ? v.y : v.z);
}
template <int D>
__device__ __forceinline__ void setcomp(typename Vec<D>::T &v, int k, float x);
template <> __device__ __forceinline__ void setcomp<1>(float &v, int, float x) { v = x; }
template <> __device__ __forceinline__ void setcomp<2>(float2 &v, int k, float x) {
  if (k == 0) v.x = x; else v.y = x;
}
template <> __device__ __forceinline__ void setcomp<3>(float4 &v, int k, float x) {
  if (k == 0) v.x = x; else if (k == 1) v.y = x; else v.z = x;
}

// Grid node type: D+1 channels packed.
template <int D> struct Node { typedef float4 T; };
template <> struct Node<1> { typedef float2 T; };

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Programmatic dependent launch.  The kernels of the repulsion chain after
// the first are launched with programmatic stream serialisation, so the
// hardware stages a kernel's launch while its predecessor on the stream
// drains; every such kernel begins here, which waits until the predecessor
// has completed and its writes are visible.  Launched without the attribute
// (batches, the operator entry points, stage timing) the wait returns at once.
__device__ __forceinline__ void sgt_pdl_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_min_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// The 137-entry size table shared with the reference (CU/utils.cu:197-207).
__device__ __constant__ int c_grid_sizes[137] = {
    8,   9,   10,  11,  12,  13,  14,  15,  16,  20,  25,  26,  28,  32,  33,
    35,  36,  39,  40,  42,  44,  45,  48,  49,  50,  52,  54,  55,  56,  60,
    63,  64,  65,  66,  70,  72,  75,  77,  78,  80,  84,  88,  90,  91,  96,
    98,  99,  100, 104, 105, 108, 110, 112, 117, 120, 125, 126, 130, 132, 135,
    140, 144, 147, 150, 154, 156, 160, 165, 168, 175, 176, 180, 182, 189, 192,
    195, 196, 198, 200, 208, 210, 216, 220, 224, 225, 231, 234, 240, 245, 250,
    252, 260, 264, 270, 273, 275, 280, 288, 294, 297, 300, 308, 312, 315, 320,
    325, 330, 336, 343, 350, 351, 352, 360, 364, 375, 378, 385, 390, 392, 396,
    400, 416, 420, 432, 440, 441, 448, 450, 455, 462, 468, 480, 490, 495, 500,
    504, 512};

__device__ __forceinline__ int sgt_best_grid_size_dev(int ng) {
  for (int i = 0; i < 137; i++)
    if (ng + 2 <= c_grid_sizes[i]) return c_grid_sizes[i] - 2;
  return c_grid_sizes[136] - 2;
}

// Error bits in SgtState::error
#define SGT_EFLAG_NONFINITE 1
#define SGT_EFLAG_GRID_CLAMP 2
#define SGT_EFLAG_CHUNK_OVERFLOW 4
