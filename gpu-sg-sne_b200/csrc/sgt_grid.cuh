// sgt_grid.cuh -- repulsive-term kernels: grid decision, point binning,
// scatter-to-grid (S2G), gather-from-grid (G2S) with the Z reduction.
//
// Reference semantics (CU = code/cuda/SG-tSNE-CUDA/src):
//   min shift (thrust init 100.0)          CU/Frep.cu:96-102
//   max, h-driven grid size, table lookup  CU/gradient_descend_varGrid.cu:88-92
//   scale into [0, N-3), clamp 1-FLT_EPS   CU/nuconv.cu:9-36
//   cubic Lagrange S2G / G2S               CU/gridding.cu:90-338
//   Z = sum((1+2|y|^2)Phi0 - 2 y.Phi) - n,
//   F = (y Phi0 - Phi)/Z                   CU/Frep.cu:42-80, HYB/qq.cpp:75-106
//
// B200 structure: points are counting-sorted into T^d-cell tiles every
// iteration; S2G accumulates one tile per chunk of sorted points in shared
// memory and flushes with vector atomics, so global atomics scale with the
// grid, not with n*4^d.  Every kernel reads the grid decision from SgtState,
// so the chain is graph-capturable with fixed launch shapes.
#pragma once
#include "sgt_common.cuh"

#define SGT_HIST_MAX 4096  // tiles held in shared memory by the binning kernels
// Points a thread loads before it uses the first of them in the point loops
// of the binning, S2G (cell mode) and G2S kernels: these kernels are bound by
// load latency, not bandwidth, at a few warps per SM.
#define SGT_PTS_U 4

// Sums K per-lane values over the 32 lanes of a warp in K/2 + K/4 + ...
// shuffles instead of 5K: at each step with offset O a lane keeps one half of
// its values, sends the other half to lane ^ O and adds what it receives; once
// the count no longer halves, the remaining offsets add whole vectors.  On
// return acc[q], q < wsum_count(K, 16), of lane L holds the warp total of the
// entry values acc[base + q], with base (zero on entry) advanced by the call;
// lanes that share a base hold the same totals, and the lanes with
// (L & wsum_full_mask(K, 16)) == 0 are one of each.
__host__ __device__ constexpr int wsum_count(int k, int o) {
  return o == 0 ? k : ((k % 2 == 0) ? wsum_count(k / 2, o / 2) : wsum_count(k, o / 2));
}
__host__ __device__ constexpr int wsum_full_mask(int k, int o) {
  return o == 0 ? 0 : ((k % 2 == 0) ? wsum_full_mask(k / 2, o / 2) : (o | wsum_full_mask(k, o / 2)));
}
template <int K, int O>
__device__ __forceinline__ void warp_multi_sum(float *acc, int lane, int &base) {
  if constexpr (O > 0) {
    if constexpr (K % 2 == 0) {
      constexpr int H = K / 2;
      const bool up = (lane & O) != 0;
#pragma unroll
      for (int q = 0; q < H; q++) {
        const float send = up ? acc[q] : acc[q + H];
        const float keep = up ? acc[q + H] : acc[q];
        acc[q] = keep + __shfl_xor_sync(0xffffffffu, send, O);
      }
      if (up) base += H;
      warp_multi_sum<H, O / 2>(acc, lane, base);
    } else {
#pragma unroll
      for (int q = 0; q < K; q++) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], O);
      warp_multi_sum<K, O / 2>(acc, lane, base);
    }
  }
}

// Smallest FFT length >= need among 32, 64, 96, 128, 192, ..., 768, 1024
// (2^k and 3 * 2^k): the 3 * 2^k lengths cut the padding of grids just above
// a power of two (N = 33..48 takes 96 points per axis instead of 128).
__device__ __forceinline__ int sgt_fft_length(int need) {
  int m = 32;
  while (m < 1024) {
    if (m >= need) return m;
    if (m >= 64 && (m / 2) * 3 >= need) return (m / 2) * 3;
    m <<= 1;
  }
  return 1024;
}

// ---------------------------------------------------------------------------
// Grid decision from the stats of the coordinates that the next kernels bin.
// minv/maxv are per-dim min/max of Ynext, sums its per-dim sums; the
// coordinates actually binned are Y = Ynext - mean (mean = 0 if !centre).
// Rounding is monotone, so min/max of the rounded differences equal the
// rounded differences of min/max: the decision is the one the reference
// takes on the centred array.
// ---------------------------------------------------------------------------
template <int D>
__device__ void sgt_finalize_grid(SgtState *st, const SgtJobParams &jp,
                                  const float *minv, const float *maxv,
                                  const double *sums, bool centre) {
  float maxy = 0.0f;
  for (int k = 0; k < D; k++) {
    const float mean = centre ? (float)(sums[k] / (double)jp.n) : 0.0f;
    const float lo = __fsub_rn(minv[k], mean);
    const float hi = __fsub_rn(maxv[k], mean);
    const float mn = fminf(100.0f, lo);
    st->mean[k] = mean;
    st->miny[k] = mn;
    maxy = fmaxf(maxy, __fsub_rn(hi, mn));
  }
  if (!(maxy > 0.0f) || !isfinite(maxy)) {
    if (!isfinite(maxy)) st->error |= SGT_EFLAG_NONFINITE;
    maxy = 1.0f;  // all points coincide: any positive extent gives zero force
  }
  int n1;
  if (jp.grid_mode == 1) {
    n1 = jp.n1_fixed;
  } else {
    int ng = (int)ceilf(__fdiv_rn(maxy, jp.h));
    ng = ng < 14 ? 14 : ng;
    n1 = sgt_best_grid_size_dev(ng);
  }
  int N = n1 + 2;
  int M = sgt_fft_length(2 * N - 1);
  if (M > jp.mmax) {  // keep the grid inside the allocated FFT workspace
    st->error |= SGT_EFLAG_GRID_CLAMP;
    st->grid_clamped = 1;
    int i = 136;
    while (i > 0 && 2 * c_grid_sizes[i] - 1 > jp.mmax) i--;
    N = c_grid_sizes[i];
    n1 = N - 2;
    M = sgt_fft_length(2 * N - 1);
  }
  st->maxy = maxy;
  st->N = N;
  st->M = M;
  st->scale = (float)(unsigned)(N - 3);
  st->h_eff = __fdiv_rn(maxy, (float)(n1 - 1) - 1.1920928955078125e-7f);
  const int cells = n1 - 1;  // floor bins lie in [0, n1-2]
  long ncell = cells;
  if (D >= 2) ncell *= cells;
  if (D >= 3) ncell *= cells;
  // cell mode (tile = one cell): the cells fit the tile arrays and hold
  // enough points each that one block reduction per chunk of a cell is
  // cheaper than shared-memory atomics that all land on a few nodes
  const bool cell_mode = ncell <= SGT_HIST_MAX && (long)jp.n >= 64L * ncell;
  // direct mode (no sort, the grid in shared memory) for the other grids that
  // fit: few points per node, so its shared-memory atomics rarely collide
  if (!cell_mode && N <= jp.direct_max) {
    st->T = 0;
    st->tiles_dim = 0;
    st->ntiles = 0;
    return;
  }
  // 3-D tiles of 8 cells while the tile count fits the tile arrays: a
  // (8+3)^3 x 4-channel shared accumulator is 21 KB (a 16-cell tile: 110 KB),
  // so each chunk zeroes and flushes 5x fewer nodes and more CTAs fit an SM
  const int T = cell_mode ? 1 : (D == 1 ? 512 : (D == 2 ? 32 : (cells <= 128 ? 8 : 16)));
  const int td = (cells + T - 1) / T;
  int nt = td;
  if (D >= 2) nt *= td;
  if (D >= 3) nt *= td;
  st->T = T;
  st->tiles_dim = td;
  st->ntiles = nt;
}

// Scaled coordinate exactly as CU/nuconv.cu:9-36: (y - miny)/maxy, clamp to
// 1-FLT_EPSILON, times (N-3).  Returns the shifted coordinate too.
__device__ __forceinline__ float sgt_scale(float y, float miny, float maxy,
                                           float scale, float &shifted) {
  shifted = __fsub_rn(y, miny);
  float v = __fdiv_rn(shifted, maxy);
  if (v >= 1.0f) v = 1.0f - 1.1920928955078125e-7f;
  return __fmul_rn(v, scale);
}

template <int D>
__device__ __forceinline__ int sgt_tile_of(const int *f, int T, int td) {
  int t = f[0] / T;
  if (D >= 2) t += td * (f[1] / T);
  if (D >= 3) t += td * td * (f[2] / T);
  return t;
}

// ---------------------------------------------------------------------------
// init: stats of a given coordinate array (first iteration / operator mode)
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_init_stats(const typename Vec<D>::T *__restrict__ Y, int n, SgtState *st,
             SgtJobParams jp, float4 *part_min, float4 *part_max,
             double *part_sum, int centre) {
  __shared__ float smin[SGT_THREADS / 32][4], smax[SGT_THREADS / 32][4];
  __shared__ double ssum[SGT_THREADS / 32][4];
  __shared__ bool last;
  float mn[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
  float mx[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
  double sm[4] = {0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const typename Vec<D>::T y = Y[i];
#pragma unroll
    for (int k = 0; k < D; k++) {
      const float v = comp<D>(y, k);
      mn[k] = fminf(mn[k], v);
      mx[k] = fmaxf(mx[k], v);
      sm[k] += (double)v;
    }
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < D; k++) {
    mn[k] = warp_min_f(mn[k]);
    mx[k] = warp_max_f(mx[k]);
    sm[k] = warp_sum_d(sm[k]);
    if (l == 0) { smin[w][k] = mn[k]; smax[w][k] = mx[k]; ssum[w][k] = sm[k]; }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float4 a = make_float4(INFINITY, INFINITY, INFINITY, INFINITY);
    float4 b = make_float4(-INFINITY, -INFINITY, -INFINITY, -INFINITY);
    double s[4] = {0, 0, 0, 0};
    for (int j = 0; j < SGT_THREADS / 32; j++) {
      a.x = fminf(a.x, smin[j][0]); b.x = fmaxf(b.x, smax[j][0]); s[0] += ssum[j][0];
      if (D > 1) { a.y = fminf(a.y, smin[j][1]); b.y = fmaxf(b.y, smax[j][1]); s[1] += ssum[j][1]; }
      if (D > 2) { a.z = fminf(a.z, smin[j][2]); b.z = fmaxf(b.z, smax[j][2]); s[2] += ssum[j][2]; }
    }
    part_min[blockIdx.x] = a;
    part_max[blockIdx.x] = b;
    for (int k = 0; k < 4; k++) part_sum[blockIdx.x * 4 + k] = s[k];
    __threadfence();
    const unsigned prev = atomicAdd(&st->done_init, 1u);
    last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    float lo[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
    float hi[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
    double s[4] = {0, 0, 0, 0};
    for (int b = 0; b < (int)gridDim.x; b++) {
      lo[0] = fminf(lo[0], __ldcg(&part_min[b].x));
      hi[0] = fmaxf(hi[0], __ldcg(&part_max[b].x));
      if (D > 1) { lo[1] = fminf(lo[1], __ldcg(&part_min[b].y)); hi[1] = fmaxf(hi[1], __ldcg(&part_max[b].y)); }
      if (D > 2) { lo[2] = fminf(lo[2], __ldcg(&part_min[b].z)); hi[2] = fmaxf(hi[2], __ldcg(&part_max[b].z)); }
      for (int k = 0; k < D; k++) s[k] += __ldcg(&part_sum[b * 4 + k]);
    }
    for (int k = 0; k < D; k++) { st->minv[k] = lo[k]; st->maxv[k] = hi[k]; st->sum[k] = s[k]; }
    sgt_finalize_grid<D>(st, jp, lo, hi, s, centre != 0);
    st->done_init = 0;
  }
}


// ---------------------------------------------------------------------------
// bin scan (run by the last block of bin_count): tile offsets and the chunk
// work list
// ---------------------------------------------------------------------------
// exclusive scan over the threads of a block (blockDim a multiple of 32)
__device__ __forceinline__ int block_exclusive_scan(int v, int *total) {
  __shared__ int wsum[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < nw ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    wsum[lane] = s;
  }
  __syncthreads();
  const int excl = x - v + (w > 0 ? wsum[w - 1] : 0);
  *total = wsum[nw - 1];
  __syncthreads();
  return excl;
}

// Thread t owns the tiles [t per, t per + per); the counts (written by other
// blocks' atomics) are read from L2.
__device__ __forceinline__ void bin_scan_block(SgtState *st, const SgtJobParams &jp,
                                               int *__restrict__ tile_count,
                                               int *__restrict__ cursor,
                                               int4 *__restrict__ chunks, int nblk) {
  const int ntiles = st->ntiles;
  // chunk length: about two chunks per persistent S2G CTA, at least 1024
  // points (256 in 3-D, where a point costs 64 nodes and small jobs need more
  // chunks than they have 1024-point runs)
  int chunk = (jp.n + 2 * nblk - 1) / (2 * nblk);
  chunk = ((chunk + 255) / 256) * 256;
  const int cmin = jp.chunk_min > 0 ? jp.chunk_min : (jp.d == 3 ? 256 : 1024);
  if (chunk < cmin) chunk = cmin;
  const int per = (ntiles + blockDim.x - 1) / blockDim.x;
  const int t0 = threadIdx.x * per, t1 = min(t0 + per, ntiles);
  int mysum = 0, mych = 0;
  for (int t = t0; t < t1; t++) {
    const int c = __ldcg(&tile_count[t]);
    mysum += c;
    mych += (c + chunk - 1) / chunk;
  }
  int tot_pts, tot_ch;
  int base = block_exclusive_scan(mysum, &tot_pts);
  int cbase = block_exclusive_scan(mych, &tot_ch);
  for (int t = t0; t < t1; t++) {
    const int cnt = __ldcg(&tile_count[t]);
    const int cpt = (cnt + chunk - 1) / chunk;
    cursor[t] = base;
    for (int c = 0; c < cpt; c++) {
      const int idx = cbase + c;
      if (idx < jp.chunk_cap) {
        const int len = min(chunk, cnt - c * chunk);
        chunks[idx] = make_int4(t, base + c * chunk, len, 0);
      }
    }
    base += cnt;
    cbase += cpt;
    tile_count[t] = 0;  // ready for the next iteration
  }
  if (threadIdx.x == 0) {
    st->chunk = chunk;
    if (tot_ch > jp.chunk_cap) {
      st->error |= SGT_EFLAG_CHUNK_OVERFLOW;
      tot_ch = jp.chunk_cap;
    }
    st->nchunks = tot_ch;
  }
}

// ---------------------------------------------------------------------------
// bin_count: centre (Y = Ynext - mean), zero the grid V, count points per tile
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void k_bin_count_body(int vb_, int vg_, const typename Vec<D>::T *__restrict__ Ynext,
            typename Vec<D>::T *__restrict__ Y, int n, SgtState *st,
            int *__restrict__ tile_count, typename Node<D>::T *__restrict__ V,
            int write_centred, const SgtJobParams &jp, int *__restrict__ cursor,
            int4 *__restrict__ chunks, int nblk) {
  __shared__ int hist[SGT_HIST_MAX];
  const int ntiles = st->ntiles, T = st->T, td = st->tiles_dim, N = st->N;
  const float maxy = st->maxy, scale = st->scale;
  float mean[3], miny[3];
#pragma unroll
  for (int k = 0; k < D; k++) { mean[k] = st->mean[k]; miny[k] = st->miny[k]; }
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x) hist[t] = 0;
  // zero the grid for this iteration's S2G
  long nodes = N;
  if (D >= 2) nodes *= N;
  if (D >= 3) nodes *= N;
  typename Node<D>::T z;
  if constexpr (D == 1) z = make_float2(0.f, 0.f); else z = make_float4(0.f, 0.f, 0.f, 0.f);
  for (long g = vb_ * (long)blockDim.x + threadIdx.x; g < nodes;
       g += (long)vg_ * blockDim.x)
    V[g] = z;
  if (T == 0) {  // direct mode: centre only; k_bin_scatter does the S2G
    if (write_centred) {
      constexpr int U = SGT_PTS_U;
      const long stride = (long)vg_ * blockDim.x * U;
      for (long i0 = ((long)vb_ * blockDim.x + (threadIdx.x & ~31)) * U; i0 < n; i0 += stride) {
        typename Vec<D>::T yv[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const long i = i0 + 32 * u + (threadIdx.x & 31);
          if (i < n) yv[u] = Ynext[i];
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
          const long i = i0 + 32 * u + (threadIdx.x & 31);
          if (i < n) {
#pragma unroll
            for (int k = 0; k < D; k++) setcomp<D>(yv[u], k, __fsub_rn(comp<D>(yv[u], k), mean[k]));
            Y[i] = yv[u];
          }
        }
      }
    }
    return;
  }
  __syncthreads();
  // warp-uniform trip count: lanes with the same tile are merged with
  // match_any and add their count in one shared-memory atomic (points of an
  // embedding cluster on few tiles).  A warp takes SGT_PTS_U runs of 32
  // points per round and issues all their loads before the first use.
  const int lane = threadIdx.x & 31;
  constexpr int U = SGT_PTS_U;
  const long stride = (long)vg_ * blockDim.x * U;
  for (long i0 = ((long)vb_ * blockDim.x + (threadIdx.x & ~31)) * U; i0 < n; i0 += stride) {
    typename Vec<D>::T yv[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const long i = i0 + 32 * u + lane;
      if (i < n) yv[u] = Ynext[i];
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const long i = i0 + 32 * u + lane;
      int key = -1;
      if (i < n) {
        typename Vec<D>::T y = yv[u];
        int f[3] = {0, 0, 0};
#pragma unroll
        for (int k = 0; k < D; k++) {
          const float yc = __fsub_rn(comp<D>(y, k), mean[k]);
          setcomp<D>(y, k, yc);
          float sh;
          const float s = sgt_scale(yc, miny[k], maxy, scale, sh);
          f[k] = (int)floorf(s);
        }
        if (write_centred) Y[i] = y;
        key = sgt_tile_of<D>(f, T, td);
      }
      const unsigned grp = __match_any_sync(0xffffffffu, key);
      if (key >= 0 && lane == __ffs(grp) - 1) atomicAdd(&hist[key], __popc(grp));
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x)
    if (hist[t]) atomicAdd(&tile_count[t], hist[t]);
  // the last block to finish turns the tile counts into tile offsets and
  // the chunk list (no separate launch between the count and the sort)
  // (the barrier orders the block's count atomics before thread 0's
  // device-scope fence, which is cumulative over them)
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&st->done_bin, 1u) == (unsigned)vg_ - 1u;
    __threadfence();
  }
  __syncthreads();
  if (last) {
    bin_scan_block(st, jp, tile_count, cursor, chunks, nblk);
    if (threadIdx.x == 0) st->done_bin = 0;
  }
}
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_bin_count(const typename Vec<D>::T *__restrict__ Ynext,
            typename Vec<D>::T *__restrict__ Y, int n, SgtState *st,
            int *__restrict__ tile_count, typename Node<D>::T *__restrict__ V,
            int write_centred, SgtJobParams jp, int *__restrict__ cursor,
            int4 *__restrict__ chunks, int nblk) {
  k_bin_count_body<D>(blockIdx.x, gridDim.x, Ynext, Y, n, st, tile_count, V, write_centred,
                      jp, cursor, chunks, nblk);
}

// ---------------------------------------------------------------------------
// Direct-mode S2G (T = 0; d <= 2, grids of at most SGT_DIRECT_N2 points per
// axis in 2-D that hold fewer than 64 points per cell): no sort.  A block takes a contiguous range of the points in
// their own order, accumulates their weighted charges [1, y - c] in a copy of
// the whole grid in shared memory (m planes of N^d floats), and adds the
// touched nodes to V (zeroed by k_bin_count) with one vector atomic each.
// The lanes of a warp hold 32 consecutive points.  When they fall in at most
// four cells (points in a spatial order, the common case after the Morton
// relabelling), the warp sums each cell's 4^d m values by halving shuffles
// and distinct lanes publish the totals; otherwise (points scattered over
// the grid, as early in a run) each lane adds its own values with
// shared-memory atomics, which then rarely meet on one node.
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void s2g_direct_warp(float *Vs, int N, int nodes, int key,
                                                const int *f, const float (*w)[4],
                                                const float *qc, int lane) {
  constexpr int NN = D == 1 ? 4 : 16, C = D + 1, K = NN * C;
  const unsigned full = 0xffffffffu;
  const unsigned valid = __ballot_sync(full, key >= 0);
  if (valid == 0u) return;
  const unsigned grp = __match_any_sync(full, key);
  const bool leader = key >= 0 && lane == __ffs(grp) - 1;
  const int ngroups = __popc(__ballot_sync(full, leader));
  if (ngroups <= 4) {
    unsigned rem = valid;
    while (rem) {  // warp-uniform
      const int l0 = __ffs(rem) - 1;
      const int gk = __shfl_sync(full, key, l0);
      const int g0 = __shfl_sync(full, f[0], l0);
      const int g1 = D == 2 ? __shfl_sync(full, f[1], l0) : 0;
      const bool in = key == gk;
      const unsigned gm = __ballot_sync(full, in);
      float a[K];
#pragma unroll
      for (int a1 = 0; a1 < (D == 2 ? 4 : 1); a1++)
#pragma unroll
        for (int a0 = 0; a0 < 4; a0++) {
          const float wt = in ? (D == 2 ? w[1][a1] : 1.f) * w[0][a0] : 0.f;
          const int nd = a1 * 4 + a0;
          a[nd * C] = wt;
#pragma unroll
          for (int k = 0; k < D; k++) a[nd * C + 1 + k] = wt * qc[k];
        }
      int base = 0;
      warp_multi_sum<K, 16>(a, lane, base);
      if ((lane & wsum_full_mask(K, 16)) == 0) {
#pragma unroll
        for (int q = 0; q < wsum_count(K, 16); q++) {
          const int idx = base + q, nd = idx / C, ch = idx % C;
          const int node = g0 + (nd & 3) + (D == 2 ? N * (g1 + (nd >> 2)) : 0);
          atomicAdd(&Vs[ch * nodes + node], a[q]);
        }
      }
      rem &= ~gm;
    }
  } else if (key >= 0) {
#pragma unroll
    for (int a1 = 0; a1 < (D == 2 ? 4 : 1); a1++)
#pragma unroll
      for (int a0 = 0; a0 < 4; a0++) {
        const float wt = (D == 2 ? w[1][a1] : 1.f) * w[0][a0];
        const int node = f[0] + a0 + (D == 2 ? N * (f[1] + a1) : 0);
        atomicAdd(&Vs[node], wt);
#pragma unroll
        for (int k = 0; k < D; k++) atomicAdd(&Vs[(k + 1) * nodes + node], wt * qc[k]);
      }
  }
}

template <int D>
__device__ __forceinline__ void k_s2g_direct_body(int vb_, int vg_, const typename Vec<D>::T *__restrict__ Y,
                                                  int n, SgtState *st,
                                                  typename Node<D>::T *__restrict__ V) {
  static_assert(D <= 2, "direct mode is for d <= 2");
  sgt_pdl_wait();
  if (st->T != 0) return;  // cell and tile modes: the sort and k_s2g* do it
  extern __shared__ float sgt_direct_grid[];
  float *Vs = sgt_direct_grid;
  constexpr int C = D + 1;
  const int N = st->N, cells = N - 3;
  const int nodes = D == 1 ? N : N * N;
  const float maxy = st->maxy, scale = st->scale, hc = 0.5f * maxy;
  float miny[2];
#pragma unroll
  for (int k = 0; k < D; k++) miny[k] = st->miny[k];
  for (int e = threadIdx.x; e < C * nodes; e += blockDim.x) Vs[e] = 0.f;
  __syncthreads();
  const int per = (n + vg_ - 1) / vg_;
  const int lo = vb_ * per, hi = min(n, lo + per);
  const int lane = threadIdx.x & 31;
  constexpr int U = SGT_PTS_U;
  for (int i0 = lo + (threadIdx.x & ~31) * U; i0 < hi; i0 += blockDim.x * U) {
    typename Vec<D>::T yv[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = i0 + 32 * u + lane;
      if (i < hi) yv[u] = Y[i];
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = i0 + 32 * u + lane;
      int key = -1;
      int f[2] = {0, 0};
      float w[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}}, qc[2] = {0.f, 0.f};
      if (i < hi) {
#pragma unroll
        for (int k = 0; k < D; k++) {
          float sh;
          const float sv = sgt_scale(comp<D>(yv[u], k), miny[k], maxy, scale, sh);
          sgt_weights(sv, f[k], w[k]);
          qc[k] = sh - hc;
        }
        key = D == 1 ? f[0] : f[0] + cells * f[1];
        if ((unsigned)f[0] >= (unsigned)cells || (D == 2 && (unsigned)f[1] >= (unsigned)cells)) {
          atomicOr(&st->error, SGT_EFLAG_CHUNK_OVERFLOW);  // outside the grid: skip the point
          key = -1;
        }
      }
      s2g_direct_warp<D>(Vs, N, nodes, key, f, w, qc, lane);
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nodes; e += blockDim.x) {
    const float a0 = Vs[e], a1 = Vs[nodes + e], a2 = D == 2 ? Vs[2 * nodes + e] : 0.f;
    if (a0 == 0.f && a1 == 0.f && a2 == 0.f) continue;
    if constexpr (D == 1) atomicAdd(&V[e], make_float2(a0, a1));
    else atomicAdd(&V[e], make_float4(a0, a1, a2, 0.f));
  }
}
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_s2g_direct(const typename Vec<D>::T *__restrict__ Y, int n, SgtState *st,
             typename Node<D>::T *__restrict__ V) {
  k_s2g_direct_body<D>(blockIdx.x, gridDim.x, Y, n, st, V);
}

// ---------------------------------------------------------------------------
// bin_scatter: counting-sort points into tile order.  Each CTA owns a
// contiguous range; it counts per tile, reserves its slots with one global
// atomic per touched tile, then places its points.
// sorted[p] = (y_0, y_1, y_2 | idx) with idx in the .w bits (.z for d <= 2
// keeps the same slot: idx is always stored in .w).
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void k_bin_scatter_body(int vb_, int vg_, const typename Vec<D>::T *__restrict__ Y, int n, SgtState *st,
              int *__restrict__ cursor, float4 *__restrict__ sorted) {
  sgt_pdl_wait();
  __shared__ int lc[SGT_HIST_MAX];
  if (st->T == 0) return;  // direct mode: k_s2g_direct does the S2G
  const int ntiles = st->ntiles, T = st->T, td = st->tiles_dim;
  const float maxy = st->maxy, scale = st->scale;
  float miny[3];
#pragma unroll
  for (int k = 0; k < D; k++) miny[k] = st->miny[k];
  const int per = (n + vg_ - 1) / vg_;
  const int lo = vb_ * per, hi = min(n, lo + per);
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x) lc[t] = 0;
  __syncthreads();
  // warp-uniform trip counts; lanes of one tile are merged with match_any,
  // the group leader does the shared-memory atomic and the lanes take
  // consecutive slots in lane order.  A warp takes SGT_PTS_U runs of 32
  // points per round and issues all their loads before the first use.
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  constexpr int U = SGT_PTS_U;
  const int wstart = lo + (threadIdx.x & ~31) * U, wstep = blockDim.x * U;
  for (int i0 = wstart; i0 < hi; i0 += wstep) {
    typename Vec<D>::T yv[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = i0 + 32 * u + lane;
      if (i < hi) yv[u] = Y[i];
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = i0 + 32 * u + lane;
      int key = -1;
      if (i < hi) {
        int f[3] = {0, 0, 0};
#pragma unroll
        for (int k = 0; k < D; k++) {
          float sh;
          f[k] = (int)floorf(sgt_scale(comp<D>(yv[u], k), miny[k], maxy, scale, sh));
        }
        key = sgt_tile_of<D>(f, T, td);
      }
      const unsigned grp = __match_any_sync(0xffffffffu, key);
      if (key >= 0 && lane == __ffs(grp) - 1) atomicAdd(&lc[key], __popc(grp));
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x)
    if (lc[t]) lc[t] = atomicAdd(&cursor[t], lc[t]);
  __syncthreads();
  for (int i0 = wstart; i0 < hi; i0 += wstep) {
    typename Vec<D>::T yv[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = i0 + 32 * u + lane;
      if (i < hi) yv[u] = Y[i];
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = i0 + 32 * u + lane;
      int key = -1;
      float4 rec = make_float4(0.f, 0.f, 0.f, __int_as_float(i));
      if (i < hi) {
        int f[3] = {0, 0, 0};
#pragma unroll
        for (int k = 0; k < D; k++) {
          float sh;
          const float v = comp<D>(yv[u], k);
          f[k] = (int)floorf(sgt_scale(v, miny[k], maxy, scale, sh));
          if (k == 0) rec.x = v; else if (k == 1) rec.y = v; else rec.z = v;
        }
        key = sgt_tile_of<D>(f, T, td);
      }
      const unsigned grp = __match_any_sync(0xffffffffu, key);
      const int leader = __ffs(grp) - 1;
      int base = 0;
      if (key >= 0 && lane == leader) base = atomicAdd(&lc[key], __popc(grp));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (key >= 0) sorted[base + __popc(grp & below)] = rec;
    }
  }
}
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_bin_scatter(const typename Vec<D>::T *__restrict__ Y, int n, SgtState *st,
              int *__restrict__ cursor, float4 *__restrict__ sorted) {
  k_bin_scatter_body<D>(blockIdx.x, gridDim.x, Y, n, st, cursor, sorted);
}

// ---------------------------------------------------------------------------
// S2G over chunks of sorted points; one shared-memory tile per chunk.
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void sgt_point_stencil(const float4 &rec,
                                                  const float *miny, float maxy,
                                                  float scale, int *f,
                                                  float (*w)[4], float *ys) {
#pragma unroll
  for (int k = 0; k < D; k++) {
    const float v = k == 0 ? rec.x : (k == 1 ? rec.y : rec.z);
    const float s = sgt_scale(v, miny[k], maxy, scale, ys[k]);
    sgt_weights(s, f[k], w[k]);
  }
}

// TT: the tile edge this instance handles; the instances of the other tile
// edges (and k_s2g_cell in cell mode) return at once.
template <int D, int TT>
__device__ __forceinline__ void k_s2g_body(int vb_, int vg_, const float4 *__restrict__ sorted, SgtState *st,
      const int4 *__restrict__ chunks, typename Node<D>::T *__restrict__ V) {
  sgt_pdl_wait();
  extern __shared__ float acc[];  // [D+1][R^D]
  const int T = st->T, td = st->tiles_dim, N = st->N, nch = st->nchunks;
  if (T != TT) return;
  const float maxy = st->maxy, scale = st->scale;
  // charges are taken about the middle of the grid: F and Z are invariant to
  // the origin of y, and |y - c| <= maxy/2 halves the cancellation in
  // (1 + 2|y|^2) Phi0 - 2 y.Phi
  const float hc = 0.5f * maxy;
  float miny[3];
#pragma unroll
  for (int k = 0; k < D; k++) miny[k] = st->miny[k];
  const int R = T + 3;
  int RD = R;
  if (D >= 2) RD *= R;
  if (D >= 3) RD *= R;
  constexpr int m = D + 1;
  for (int c = vb_; c < nch; c += vg_) {
    const int4 ch = chunks[c];
    int o[3] = {0, 0, 0};
    o[0] = (ch.x % td) * T;
    if (D >= 2) o[1] = ((ch.x / td) % td) * T;
    if (D >= 3) o[2] = (ch.x / (td * td)) * T;
    for (int e = threadIdx.x; e < m * RD; e += blockDim.x) acc[e] = 0.f;
    __syncthreads();
    if constexpr (D == 3) {
      // The lanes of a warp share one point at a time, each owning 2 of its
      // 64 stencil nodes, so the 32 atomics of an instruction go to 32
      // distinct nodes.  (With a point per thread, the points of a cluster
      // sit in few cells and all lanes of a warp collide on the same nodes.)
      // Points come 32 per warp in one coalesced load; each lane computes
      // the stencil of its own point and the warp hands the stencils round
      // by shuffles.
      const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
      const int a0 = lane & 3, a1 = (lane >> 2) & 3, a2b = lane >> 4;
      for (int j0 = ch.y + 32 * wid; j0 < ch.y + ch.z; j0 += 32 * nw) {
        const int jm = min(32, ch.y + ch.z - j0);
        int f[3] = {0, 0, 0};
        float w[3][4], ys[3];
        int node0 = -1;  // this lane's point: base node in the tile, -1 if none
        if (lane < jm) {
          const float4 rec = sorted[j0 + lane];
          sgt_point_stencil<D>(rec, miny, maxy, scale, f, w, ys);
          const int l0 = f[0] - o[0], l1 = f[1] - o[1], l2 = f[2] - o[2];
          if ((unsigned)l0 < (unsigned)T && (unsigned)l1 < (unsigned)T &&
              (unsigned)l2 < (unsigned)T) {
            node0 = l0 + R * (l1 + R * l2);
          } else {  // the sort and the binning disagree: skip the point
            atomicOr(&st->error, SGT_EFLAG_CHUNK_OVERFLOW);
          }
        } else {
#pragma unroll
          for (int k = 0; k < 3; k++) {
            ys[k] = 0.f;
#pragma unroll
            for (int a = 0; a < 4; a++) w[k][a] = 0.f;
          }
        }
        for (int t = 0; t < jm; t++) {
          const int nb = __shfl_sync(0xffffffffu, node0, t);
          float wx[4], wy4[4], wz4[4], qc[3];
#pragma unroll
          for (int a = 0; a < 4; a++) {
            wx[a] = __shfl_sync(0xffffffffu, w[0][a], t);
            wy4[a] = __shfl_sync(0xffffffffu, w[1][a], t);
            wz4[a] = __shfl_sync(0xffffffffu, w[2][a], t);
          }
#pragma unroll
          for (int k = 0; k < 3; k++) qc[k] = __shfl_sync(0xffffffffu, ys[k], t) - hc;
          if (nb < 0) continue;  // uniform over the warp
          const float w0 = a0 == 0 ? wx[0] : (a0 == 1 ? wx[1] : (a0 == 2 ? wx[2] : wx[3]));
          const float w1 = a1 == 0 ? wy4[0] : (a1 == 1 ? wy4[1] : (a1 == 2 ? wy4[2] : wy4[3]));
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int a2 = a2b + 2 * h;
            const float w2 = a2 == 0 ? wz4[0] : (a2 == 1 ? wz4[1] : (a2 == 2 ? wz4[2] : wz4[3]));
            const float wt = (w1 * w2) * w0;  // the product order of the loop below
            const int node = nb + a0 + R * (a1 + R * a2);
            atomicAdd(&acc[node], wt);
#pragma unroll
            for (int k = 0; k < 3; k++) atomicAdd(&acc[(k + 1) * RD + node], wt * qc[k]);
          }
        }
      }
    } else {
    // each thread walks its own contiguous stretch of the chunk, so the lanes
    // of a warp sit far apart in the (spatially ordered) chunk and their
    // shared-memory atomics rarely meet on one node
    const int per = (ch.z + blockDim.x - 1) / blockDim.x;
    const int jb = ch.y + threadIdx.x * per, je = min(jb + per, ch.y + ch.z);
    for (int j = jb; j < je; j++) {
      const float4 rec = sorted[j];
      int f[3];
      float w[3][4], ys[3];
      sgt_point_stencil<D>(rec, miny, maxy, scale, f, w, ys);
      const int l0 = f[0] - o[0];
      const int l1 = D >= 2 ? f[1] - o[1] : 0;
      const int l2 = D >= 3 ? f[2] - o[2] : 0;
      // a point outside its tile would mean the sort and the binning
      // disagree; skip it rather than touch memory outside the tile
      if ((unsigned)l0 >= (unsigned)T || (unsigned)l1 >= (unsigned)T ||
          (unsigned)l2 >= (unsigned)T) {
        atomicOr(&st->error, SGT_EFLAG_CHUNK_OVERFLOW);
        continue;
      }
#pragma unroll
      for (int a2 = 0; a2 < (D >= 3 ? 4 : 1); a2++)
#pragma unroll
        for (int a1 = 0; a1 < (D >= 2 ? 4 : 1); a1++) {
          float wy = 1.f;
          if (D >= 2) wy *= w[1][a1];
          if (D >= 3) wy *= w[2][a2];
          const int rowbase = (l0) + R * ((l1 + a1) + R * (l2 + a2));
#pragma unroll
          for (int a0 = 0; a0 < 4; a0++) {
            const float wt = wy * w[0][a0];
            const int node = rowbase + a0;
            atomicAdd(&acc[node], wt);
#pragma unroll
            for (int k = 0; k < D; k++) atomicAdd(&acc[(k + 1) * RD + node], wt * (ys[k] - hc));
          }
        }
    }
    }
    __syncthreads();
    // flush the touched region of this tile into V
    for (int e = threadIdx.x; e < RD; e += blockDim.x) {
      const int lx = e % R;
      const int ly = D >= 2 ? (e / R) % R : 0;
      const int lz = D >= 3 ? e / (R * R) : 0;
      const int gx = o[0] + lx, gy = o[1] + ly, gz = o[2] + lz;
      if (gx >= N || (D >= 2 && gy >= N) || (D >= 3 && gz >= N)) continue;
      const float a0 = acc[e];
      const float a1 = acc[RD + e];
      const float a2 = D >= 2 ? acc[2 * RD + e] : 0.f;
      const float a3 = D >= 3 ? acc[3 * RD + e] : 0.f;
      if (a0 == 0.f && a1 == 0.f && a2 == 0.f && a3 == 0.f) continue;
      long g = gx;
      if (D >= 2) g += (long)N * gy;
      if (D >= 3) g += (long)N * N * gz;
      if constexpr (D == 1) {
        atomicAdd(&V[g], make_float2(a0, a1));
      } else {
        atomicAdd(&V[g], make_float4(a0, a1, a2, a3));
      }
    }
    __syncthreads();
  }
}
template <int D, int TT>
__global__ void __launch_bounds__(SGT_THREADS)
k_s2g(const float4 *__restrict__ sorted, SgtState *st,
      const int4 *__restrict__ chunks, typename Node<D>::T *__restrict__ V) {
  k_s2g_body<D, TT>(blockIdx.x, gridDim.x, sorted, st, chunks, V);
}

// ---------------------------------------------------------------------------
// S2G in cell mode (T = 1): every point of a chunk lies in the chunk's cell,
// so all of them touch the same 4^d nodes.  Each thread sums its points'
// weighted charges in registers (no shared-memory atomics), the block reduces
// once per chunk, and one global atomic per node and channel goes to V.
// d = 3 runs in four passes over the z offset of the stencil (64 sums each).
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void k_s2g_cell_body(int vb_, int vg_, const float4 *__restrict__ sorted, SgtState *st,
           const int4 *__restrict__ chunks, typename Node<D>::T *__restrict__ V) {
  sgt_pdl_wait();
  if (st->T != 1) return;  // tile mode: k_s2g does the work
  constexpr int NN = D == 1 ? 4 : 16;  // stencil nodes per pass
  constexpr int C = D + 1;             // charge channels
  constexpr int K = NN * C;
  constexpr int CS = D == 1 ? 2 : 4;   // floats per node of V
  constexpr int PASSES = D == 3 ? 4 : 1;
  __shared__ float red[SGT_THREADS / 32][K];
  const int td = st->tiles_dim, N = st->N, nch = st->nchunks;
  const float maxy = st->maxy, scale = st->scale;
  const float hc = 0.5f * maxy;  // charge origin, as in k_s2g
  float miny[3];
#pragma unroll
  for (int k = 0; k < D; k++) miny[k] = st->miny[k];
  float *Vf = reinterpret_cast<float *>(V);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int c = vb_; c < nch; c += vg_) {
    const int4 ch = chunks[c];
    int cf[3] = {0, 0, 0};
    cf[0] = ch.x % td;
    if (D >= 2) cf[1] = (ch.x / td) % td;
    if (D >= 3) cf[2] = ch.x / (td * td);
#pragma unroll
    for (int pass = 0; pass < PASSES; pass++) {
      float acc[K];
#pragma unroll
      for (int q = 0; q < K; q++) acc[q] = 0.f;
      constexpr int U = SGT_PTS_U;
      const int end = ch.y + ch.z;
      for (int j0 = ch.y + threadIdx.x; j0 < end; j0 += U * blockDim.x) {
        float4 rv[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const int j = j0 + u * blockDim.x;
          if (j < end) rv[u] = sorted[j];
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
          if (j0 + u * blockDim.x >= end) break;
          int f[3];
          float w[3][4], ys[3];
          sgt_point_stencil<D>(rv[u], miny, maxy, scale, f, w, ys);
          bool ok = f[0] == cf[0];
          if (D >= 2) ok = ok && f[1] == cf[1];
          if (D >= 3) ok = ok && f[2] == cf[2];
          if (!ok) {  // the sort and the binning disagree: skip the point
            atomicOr(&st->error, SGT_EFLAG_CHUNK_OVERFLOW);
            continue;
          }
          float qc[3];
#pragma unroll
          for (int k = 0; k < D; k++) qc[k] = ys[k] - hc;
          const float wz = D == 3 ? w[2][pass] : 1.f;
#pragma unroll
          for (int a1 = 0; a1 < (D >= 2 ? 4 : 1); a1++) {
            const float wy = (D >= 2 ? w[1][a1] : 1.f) * wz;
#pragma unroll
            for (int a0 = 0; a0 < 4; a0++) {
              const float wt = wy * w[0][a0];
              const int nd = a1 * 4 + a0;
              acc[nd * C] += wt;
#pragma unroll
              for (int k = 0; k < D; k++) acc[nd * C + 1 + k] += wt * qc[k];
            }
          }
        }
      }
      {
        int base = 0;
        warp_multi_sum<K, 16>(acc, lane, base);
        constexpr int KF = wsum_count(K, 16);
        if ((lane & wsum_full_mask(K, 16)) == 0) {
#pragma unroll
          for (int q = 0; q < KF; q++) red[wid][base + q] = acc[q];
        }
      }
      __syncthreads();
      for (int q = threadIdx.x; q < K; q += blockDim.x) {
        float sum = 0.f;
#pragma unroll
        for (int j = 0; j < SGT_THREADS / 32; j++) sum += red[j][q];
        const int nd = q / C, chn = q % C;
        long g = cf[0] + (nd & 3);
        if (D >= 2) g += (long)N * (cf[1] + (nd >> 2));
        if (D >= 3) g += (long)N * N * (cf[2] + pass);
        if (sum != 0.f) atomicAdd(&Vf[g * CS + chn], sum);
      }
      __syncthreads();
    }
  }
}
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_s2g_cell(const float4 *__restrict__ sorted, SgtState *st,
           const int4 *__restrict__ chunks, typename Node<D>::T *__restrict__ V) {
  k_s2g_cell_body<D>(blockIdx.x, gridDim.x, sorted, st, chunks, V);
}

// Interpolated potentials p[0..d] at a point with stencil weights w and base
// cell f: from a grid Phi (in global or shared memory), or (SM) from the
// block's copy cn of the 4^d nodes of the point's cell, node a0 + 4 a1 +
// 16 a2.  Same products in the same order either way.
template <int D, bool SM>
__device__ __forceinline__ void g2s_potentials(const float (*w)[4], const int *f, int N,
                                               const typename Node<D>::T *Phi,
                                               const typename Node<D>::T *cn, float *p) {
#pragma unroll
  for (int a2 = 0; a2 < (D >= 3 ? 4 : 1); a2++)
#pragma unroll
    for (int a1 = 0; a1 < (D >= 2 ? 4 : 1); a1++) {
      float wy = 1.f;
      if (D >= 2) wy *= w[1][a1];
      if (D >= 3) wy *= w[2][a2];
      long base = f[0];
      if (D >= 2) base += (long)N * (f[1] + a1);
      if (D >= 3) base += (long)N * N * (f[2] + a2);
#pragma unroll
      for (int a0 = 0; a0 < 4; a0++) {
        const float wt = wy * w[0][a0];
        typename Node<D>::T v;
        if constexpr (SM) v = cn[a0 + 4 * (a1 + 4 * a2)];
        else v = Phi[base + a0];
        p[0] += wt * v.x;
        p[1] += wt * v.y;
        if constexpr (D >= 2) {
          p[2] += wt * v.z;
          if constexpr (D >= 3) p[3] += wt * v.w;
        }
      }
    }
}

// Z of a G2S launch: the block's FP64 partial, then the last block to finish
// sums the partials in block order and writes Z = sum - n.
__device__ __forceinline__ void g2s_finish(int vb_, int vg_, SgtState *st, double *part_z, int n,
                                           double zacc, double *wz, bool &last) {
  zacc = warp_sum_d(zacc);
  if ((threadIdx.x & 31) == 0) wz[threadIdx.x >> 5] = zacc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int k = 0; k < SGT_THREADS / 32; k++) s += wz[k];
    part_z[vb_] = s;
    __threadfence();
    last = (atomicAdd(&st->done_g2s, 1u) == vg_ - 1);
  }
  __syncthreads();
  if (last) {
    __threadfence();
    double s = 0;
    for (int b = threadIdx.x; b < (int)vg_; b += blockDim.x) s += __ldcg(&part_z[b]);
    s = warp_sum_d(s);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) wz[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0;
      for (int k = 0; k < SGT_THREADS / 32; k++) t += wz[k];
      st->Z = t - (double)n;
      st->done_g2s = 0;
    }
  }
}

// ---------------------------------------------------------------------------
// G2S over chunks + repulsive force numerator + Z (FP64, fixed-order finish).
// Frep_un[i] = y_i*Phi0 - Phi_{1..d}; Z = sum_i z_i - n.
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void k_g2s_body(int vb_, int vg_, const float4 *__restrict__ sorted, SgtState *st,
      const int4 *__restrict__ chunks,
      const typename Node<D>::T *__restrict__ Phi,
      typename Vec<D>::T *__restrict__ Frep_un, double *part_z, int n) {
  sgt_pdl_wait();
  __shared__ double wz[SGT_THREADS / 32];
  __shared__ bool last;
  const int N = st->N, nch = st->nchunks;
  const float maxy = st->maxy, scale = st->scale;
  const float hc = 0.5f * maxy;  // charge origin used by S2G
  float miny[3];
#pragma unroll
  for (int k = 0; k < D; k++) miny[k] = st->miny[k];
  if (st->T == 0) return;  // direct mode: k_g2s_direct does the G2S
  double zacc = 0.0;
  // cell mode (T = 1): every point of a chunk reads the same 4^d nodes,
  // which the block stages once per chunk in shared memory
  constexpr int NNODES = D == 1 ? 4 : (D == 2 ? 16 : 64);
  __shared__ typename Node<D>::T cn[NNODES];
  const bool cell = st->T == 1;
  const int td = st->tiles_dim;
  for (int c = vb_; c < nch; c += vg_) {
    const int4 ch = chunks[c];
    int cf[3] = {-1, -1, -1};
    if (cell) {  // block-uniform
      cf[0] = ch.x % td;
      if (D >= 2) cf[1] = (ch.x / td) % td;
      if (D >= 3) cf[2] = ch.x / (td * td);
      __syncthreads();  // the previous chunk's points are done with cn
      for (int e = threadIdx.x; e < NNODES; e += blockDim.x) {
        long g = cf[0] + (e & 3);
        if (D >= 2) g += (long)N * (cf[1] + ((e >> 2) & 3));
        if (D >= 3) g += (long)N * N * (cf[2] + (e >> 4));
        cn[e] = Phi[g];
      }
      __syncthreads();
    }
    constexpr int U = SGT_PTS_U;
    const int end = ch.y + ch.z;
    for (int j0 = ch.y + threadIdx.x; j0 < end; j0 += U * blockDim.x) {
      float4 rv[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int j = j0 + u * blockDim.x;
        if (j < end) rv[u] = sorted[j];
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        if (j0 + u * blockDim.x >= end) break;
        const float4 rec = rv[u];
        int f[3];
        float w[3][4], ys[3];
        sgt_point_stencil<D>(rec, miny, maxy, scale, f, w, ys);
        bool here = cell && f[0] == cf[0];
        if (D >= 2) here = here && f[1] == cf[1];
        if (D >= 3) here = here && f[2] == cf[2];
        float p[4] = {0.f, 0.f, 0.f, 0.f};
        if (here) g2s_potentials<D, true>(w, f, N, Phi, cn, p);
        else g2s_potentials<D, false>(w, f, N, Phi, cn, p);
        double ysq = 0.0, dot = 0.0;
        typename Vec<D>::T fr;
#pragma unroll
        for (int k = 0; k < D; k++) {
          const float yk = ys[k] - hc;
          ysq += (double)yk * yk;
          dot += (double)yk * p[k + 1];
          setcomp<D>(fr, k, yk * p[0] - p[k + 1]);
        }
        zacc += (1.0 + 2.0 * ysq) * (double)p[0] - 2.0 * dot;
        Frep_un[__float_as_int(rec.w)] = fr;
      }
    }
  }
  g2s_finish(vb_, vg_, st, part_z, n, zacc, wz, last);
}
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_g2s(const float4 *__restrict__ sorted, SgtState *st,
      const int4 *__restrict__ chunks,
      const typename Node<D>::T *__restrict__ Phi,
      typename Vec<D>::T *__restrict__ Frep_un, double *part_z, int n) {
  k_g2s_body<D>(blockIdx.x, gridDim.x, sorted, st, chunks, Phi, Frep_un, part_z, n);
}

// ---------------------------------------------------------------------------
// Direct-mode G2S (T = 0): the points in their own order, the whole potential
// grid staged in shared memory, F written in place (coalesced), Z as in
// k_g2s.
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void k_g2s_direct_body(int vb_, int vg_, SgtState *st,
      const typename Node<D>::T *__restrict__ Phi,
      typename Vec<D>::T *__restrict__ Frep_un, double *part_z, int n,
      const typename Vec<D>::T *__restrict__ Y) {
  static_assert(D <= 2, "direct mode is for d <= 2");
  sgt_pdl_wait();
  __shared__ double wz[SGT_THREADS / 32];
  __shared__ bool last;
  if (st->T != 0) return;  // cell and tile modes: k_g2s does it
  const int N = st->N;
  const float maxy = st->maxy, scale = st->scale;
  const float hc = 0.5f * maxy;
  float miny[3];
#pragma unroll
  for (int k = 0; k < D; k++) miny[k] = st->miny[k];
  double zacc = 0.0;
  extern __shared__ float4 sgt_g2s_smem[];
  typename Node<D>::T *Ps = reinterpret_cast<typename Node<D>::T *>(sgt_g2s_smem);
  const int nodes = D == 1 ? N : N * N;
  for (int e = threadIdx.x; e < nodes; e += blockDim.x) Ps[e] = Phi[e];
  __syncthreads();
  constexpr int U = SGT_PTS_U;
  const int lane = threadIdx.x & 31;
  const long stride = (long)vg_ * blockDim.x * U;
  for (long i0 = ((long)vb_ * blockDim.x + (threadIdx.x & ~31)) * U; i0 < n; i0 += stride) {
    typename Vec<D>::T yv[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const long i = i0 + 32 * u + lane;
      if (i < n) yv[u] = Y[i];
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const long i = i0 + 32 * u + lane;
      if (i >= n) break;
      int f[3];
      float w[3][4], ys[3];
#pragma unroll
      for (int k = 0; k < D; k++) {
        const float sv = sgt_scale(comp<D>(yv[u], k), miny[k], maxy, scale, ys[k]);
        sgt_weights(sv, f[k], w[k]);
      }
      float p[4] = {0.f, 0.f, 0.f, 0.f};
      if ((unsigned)f[0] < (unsigned)(N - 3) && (D == 1 || (unsigned)f[1] < (unsigned)(N - 3)))
        g2s_potentials<D, false>(w, f, N, Ps, Ps, p);
      else  // outside the grid (S2G skipped it too): no force, no Z
        atomicOr(&st->error, SGT_EFLAG_CHUNK_OVERFLOW);
      double ysq = 0.0, dot = 0.0;
      typename Vec<D>::T fr;
#pragma unroll
      for (int k = 0; k < D; k++) {
        const float yk = ys[k] - hc;
        ysq += (double)yk * yk;
        dot += (double)yk * p[k + 1];
        setcomp<D>(fr, k, yk * p[0] - p[k + 1]);
      }
      zacc += (1.0 + 2.0 * ysq) * (double)p[0] - 2.0 * dot;
      Frep_un[i] = fr;
    }
  }
  g2s_finish(vb_, vg_, st, part_z, n, zacc, wz, last);
}
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_g2s_direct(SgtState *st, const typename Node<D>::T *__restrict__ Phi,
             typename Vec<D>::T *__restrict__ Frep_un, double *part_z, int n,
             const typename Vec<D>::T *__restrict__ Y) {
  k_g2s_direct_body<D>(blockIdx.x, gridDim.x, st, Phi, Frep_un, part_z, n, Y);
}

// ---------------------------------------------------------------------------
// Exact O(n^2) repulsion, for the -f error probe (CU/compute_error.cu:8-57):
// num_i = sum_{j != i} (y_i - y_j)/(1 + |y_i - y_j|^2)^2 and
// z_i = sum_{j != i} 1/(1 + |y_i - y_j|^2).  One point per thread; the other
// points stream through shared memory in tiles of SGT_THREADS, summed in
// FP32 within a tile and in FP64 across tiles.
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_frep_exact(const typename Vec<D>::T *__restrict__ Y, int n, double *__restrict__ num,
             double *__restrict__ z) {
  __shared__ float ts[SGT_THREADS][D];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float yi[3] = {0.f, 0.f, 0.f};
  if (i < n) {
    const typename Vec<D>::T v = Y[i];
#pragma unroll
    for (int k = 0; k < D; k++) yi[k] = comp<D>(v, k);
  }
  double an[3] = {0, 0, 0}, az = 0;
  for (int j0 = 0; j0 < n; j0 += SGT_THREADS) {
    const int j = j0 + threadIdx.x;
    if (j < n) {
      const typename Vec<D>::T v = Y[j];
#pragma unroll
      for (int k = 0; k < D; k++) ts[threadIdx.x][k] = comp<D>(v, k);
    }
    __syncthreads();
    const int m = min(SGT_THREADS, n - j0);
    float fn[3] = {0.f, 0.f, 0.f}, fz = 0.f;
    for (int t = 0; t < m; t++) {
      if (j0 + t == i) continue;
      float df[3], d2 = 0.f;
#pragma unroll
      for (int k = 0; k < D; k++) {
        df[k] = yi[k] - ts[t][k];
        d2 += df[k] * df[k];
      }
      const float q = 1.0f / (1.0f + d2);
      fz += q;
#pragma unroll
      for (int k = 0; k < D; k++) fn[k] += q * q * df[k];
    }
    az += fz;
#pragma unroll
    for (int k = 0; k < D; k++) an[k] += fn[k];
    __syncthreads();
  }
  if (i < n) {
    z[i] = az;
#pragma unroll
    for (int k = 0; k < D; k++) num[(long)i * D + k] = an[k];
  }
}
