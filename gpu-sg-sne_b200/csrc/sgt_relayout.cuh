// sgt_relayout.cuh -- locality relabelling of an embedding.
//
// t-SNE places graph neighbours close together, so once the embedding has
// structure, ordering the points along a space-filling curve of fine cells
// makes the neighbours of consecutive rows consecutive in memory: the
// coordinate gathers of the row kernel then hit L1 instead of L2.  Every R
// iterations the engine counting-sorts the points by the Morton code of their
// cell and rewrites P symmetrically in that order (columns remapped, each
// row's entries kept in their order, so every row sum is bit-identical) and
// permutes the per-point state.  A composite permutation maps engine slots to
// the caller's point order at the ABI.
#pragma once
#include "sgt_common.cuh"
#include "sgt_grid.cuh"

__device__ __forceinline__ unsigned spread2(unsigned x) {  // 16 bits -> even bits
  x &= 0xffffu;
  x = (x | (x << 8)) & 0x00ff00ffu;
  x = (x | (x << 4)) & 0x0f0f0f0fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  return x;
}
__device__ __forceinline__ unsigned spread3(unsigned x) {  // 10 bits -> every third bit
  x &= 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

// key of every point of Ynext: the Morton code of its cell in a fine
// lattice over the bounding box of the next binning (2-D: 512 x 512 cells;
// 3-D: 64^3 cells; 1-D: 2^18 cells; 18 bits in each case).  The lattice is
// far finer than the interpolation grid (16-25 points per axis in a typical
// run), so a cell holds a handful of points and graph neighbours that lie
// close in the embedding also lie close in memory.
template <int D>
__global__ void k_cell_keys(const typename Vec<D>::T *__restrict__ Ynext, int n,
                            const SgtState *st, unsigned *__restrict__ keys,
                            int *__restrict__ hist) {
  const float maxy = st->maxy;
  const float res = D == 1 ? 262144.f : D == 2 ? 512.f : 64.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const typename Vec<D>::T y = Ynext[i];
    unsigned f[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < D; k++) {
      float sh;
      const float yc = __fsub_rn(comp<D>(y, k), st->mean[k]);
      const float v = fmaxf(floorf(sgt_scale(yc, st->miny[k], maxy, res, sh)), 0.f);
      f[k] = min((unsigned)v, (unsigned)res - 1u);
    }
    unsigned key;
    if (D == 1) key = f[0];
    else if (D == 2) key = spread2(f[0]) | (spread2(f[1]) << 1);
    else key = spread3(f[0]) | (spread3(f[1]) << 1) | (spread3(f[2]) << 2);
    keys[i] = key;
    atomicAdd(&hist[key], 1);
  }
}

// ---- exclusive scan of int arrays (three passes, up to 4096 * 4096 items)
#define SGT_SCAN_PER_BLOCK 4096
__global__ void __launch_bounds__(1024) k_scan_blocks(const int *__restrict__ in, int len,
                                                       int *__restrict__ out,
                                                       int *__restrict__ block_sums) {
  __shared__ int ws[32];
  const int base = blockIdx.x * SGT_SCAN_PER_BLOCK + threadIdx.x * 4;
  int v[4], s = 0;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    v[q] = base + q < len ? in[base + q] : 0;
    s += v[q];
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[w] = x;
  __syncthreads();
  if (w == 0) {
    int t = ws[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    ws[lane] = t;
  }
  __syncthreads();
  int run = x - s + (w > 0 ? ws[w - 1] : 0);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    if (base + q < len) out[base + q] = run;
    run += v[q];
  }
  if (threadIdx.x == 1023) block_sums[blockIdx.x] = run;
}
__global__ void __launch_bounds__(1024) k_scan_sums(int *__restrict__ block_sums, int nb,
                                                     int *__restrict__ total) {
  // nb <= 4096: four per thread, exclusive in place
  __shared__ int ws[32];
  const int base = threadIdx.x * 4;
  int v[4], s = 0;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    v[q] = base + q < nb ? block_sums[base + q] : 0;
    s += v[q];
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[w] = x;
  __syncthreads();
  if (w == 0) {
    int t = ws[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    ws[lane] = t;
  }
  __syncthreads();
  int run = x - s + (w > 0 ? ws[w - 1] : 0);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    if (base + q < nb) block_sums[base + q] = run;
    run += v[q];
  }
  if (threadIdx.x == 1023 && total) *total = run;
}
__global__ void k_scan_add(int *__restrict__ out, int len, const int *__restrict__ block_sums) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x)
    out[i] += block_sums[i / SGT_SCAN_PER_BLOCK];
}

// counting-sort scatter: p[pos] = old slot, in key order
__global__ void k_key_scatter(const unsigned *__restrict__ keys, int n, int *__restrict__ cursor,
                              int *__restrict__ p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[atomicAdd(&cursor[keys[i]], 1)] = i;
}

// iperm, new row lengths, composite permutation to the caller's order
__global__ void k_perm_prep(const int *__restrict__ p, int n, const int *__restrict__ rowptr,
                            int *__restrict__ iperm, int *__restrict__ len_new,
                            const int *__restrict__ perm_old, int *__restrict__ perm_new) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int o = p[r];
    iperm[o] = r;
    len_new[r] = rowptr[o + 1] - rowptr[o];
    perm_new[r] = perm_old ? perm_old[o] : o;
  }
}

// warp per new row: copy the old row's pairs with remapped columns
__global__ void k_relabel_rows(const int *__restrict__ p, const int *__restrict__ iperm, int n,
                               const int *__restrict__ rowptr, const int2 *__restrict__ pairs,
                               const int *__restrict__ rowptr_new, int2 *__restrict__ pairs_new) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += warps) {
    const int o = p[r];
    const int s = rowptr[o], e = rowptr[o + 1], d0 = rowptr_new[r];
    for (int t = s + lane; t < e; t += 32) {
      const int2 pr = pairs[t];
      pairs_new[d0 + (t - s)] = make_int2(iperm[pr.x], pr.y);
    }
  }
}

template <int D>
__global__ void k_gather_vec(const typename Vec<D>::T *__restrict__ src, const int *__restrict__ p,
                             int n, typename Vec<D>::T *__restrict__ dst) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    dst[r] = src[p[r]];
}

// ---- the locality order a job starts from ---------------------------------
// Points are ordered once, at job creation, by the Morton code of coordinates
// from a few diffusion steps over P's graph: start from random coordinates
// and replace every point's coordinates by the P-weighted mean of its
// neighbours' a few times.  Neighbours in P end up with nearby coordinates
// (as in a diffusion map; the few steps keep the structure inside clusters,
// which more steps would flatten onto the cluster means), so the Morton
// order of these coordinates puts the neighbours of a row near it in memory
// before the embedding itself has any structure.

// uniform [-1, 1) from the point index (splitmix64)
__device__ __forceinline__ float sgt_hash_unit(unsigned long long x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  x ^= x >> 31;
  return (float)(x >> 40) * (1.0f / 8388608.0f) - 1.0f;
}

template <int D>
__global__ void k_diffuse_init(typename Vec<D>::T *__restrict__ z, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    typename Vec<D>::T v;
    if constexpr (D == 3) v.w = 0.f;
#pragma unroll
    for (int k = 0; k < D; k++) setcomp<D>(v, k, sgt_hash_unit((unsigned long long)i * 3 + k));
    z[i] = v;
  }
}

// one diffusion step, a warp per row: zout_i = sum_j p_ij zin_j / sum_j p_ij
template <int D>
__global__ void k_diffuse(const int *__restrict__ rowptr, const int2 *__restrict__ pairs,
                          const typename Vec<D>::T *__restrict__ zin,
                          typename Vec<D>::T *__restrict__ zout, int n) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * blockDim.x / 32;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / 32; i < n; i += warps) {
    float acc[3] = {0.f, 0.f, 0.f}, w = 0.f;
    for (int t = rowptr[i] + lane; t < rowptr[i + 1]; t += 32) {
      const int2 pr = pairs[t];
      const float p = __int_as_float(pr.y);
      const typename Vec<D>::T zj = zin[pr.x];
#pragma unroll
      for (int k = 0; k < D; k++) acc[k] += p * comp<D>(zj, k);
      w += p;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      w += __shfl_xor_sync(0xffffffffu, w, o);
#pragma unroll
      for (int k = 0; k < D; k++) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    }
    if (lane == 0) {
      typename Vec<D>::T v = zin[i];
      if (w > 0.f) {
#pragma unroll
        for (int k = 0; k < D; k++) setcomp<D>(v, k, acc[k] / w);
      }
      zout[i] = v;
    }
  }
}
