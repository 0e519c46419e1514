// sgt_rows.cuh -- attractive term, fused combine/update, KL cost.
//
// Reference semantics (CU = code/cuda/SG-tSNE-CUDA/src):
//   F_attr,i = sum_j p_ij (y_i - y_j) / (1 + |y_i - y_j|^2)
//        CU/pq.cuh:77-118 (COO), CU/hybridpq.cu:4-159 (ELL + COO),
//        HYB/pq.cpp:15-58 (CPU)
//   dY = alpha F_attr - F_rep                       CU/gradient_descend.cu:12-21
//   gains +0.2 / x0.8 (floor 0.01), uY = mu uY - eta g dY, Y += uY
//                                                   CU/gradient_descend.cu:29-44
//   per-iteration mean centring             CU/gradient_descend_varGrid.cu:41-65
//   alpha -> 1 after iteration early_iter, mu 0.5 -> 0.8 after iteration 250
//                                                   CU/gradient_descend.cu:226-233
//   KL = sum alpha p log((alpha p + FLT_MIN)/(q + FLT_MIN)), q = 1/(Z(1+d^2))
//                                                   CU/pq.cu:61-125
//
// B200 structure: the attractive SpMV streams P once per iteration (8 bytes
// per nonzero: column and value packed in an int2), a group of G lanes per
// row, neighbours' coordinates gathered as one 8/16-byte load.  It depends
// only on Y, so it runs concurrently with the latency-bound repulsion chain;
// one combine kernel (k_row_update) then applies the force combine, the
// gains/momentum update and the reductions that decide the next iteration's
// grid.  Y is double-buffered (the combine reads Y while writing Ynext).
#pragma once
#include "sgt_common.cuh"
#include "sgt_grid.cuh"

template <int D>
__device__ __forceinline__ void attr_term(const typename Vec<D>::T &yi,
                                          const typename Vec<D>::T &yj, float p,
                                          float *acc) {
  float df[3], dist = 0.f;
#pragma unroll
  for (int k = 0; k < D; k++) {
    df[k] = comp<D>(yi, k) - comp<D>(yj, k);
    dist += df[k] * df[k];
  }
  const float pq = __fdividef(p, 1.0f + dist);  // <= 2 ulp; p/(1+d^2) of the reference
#pragma unroll
  for (int k = 0; k < D; k++) acc[k] += pq * df[k];
}

template <int D, int G>
__device__ __forceinline__ void csr_row_sum(const int *__restrict__ rowptr,
                                            const int2 *__restrict__ pairs,
                                            const typename Vec<D>::T *__restrict__ Y,
                                            int i, int lane,
                                            const typename Vec<D>::T &yi,
                                            float *acc) {
  // P is streamed once per iteration: evict-first loads keep the gathered
  // coordinates resident in L2.  Four independent (column, value) loads and
  // four independent gathers per lane are in flight per step; a lane past
  // the row end gathers its own point with weight 0.
  const int s = __ldcs(&rowptr[i]), e = __ldcs(&rowptr[i + 1]);
  constexpr int U = 4;
  for (int t0 = s + lane; t0 < e; t0 += U * G) {
    int2 pr[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * G;
      pr[u] = t < e ? __ldcs(&pairs[t]) : make_int2(i, 0);
    }
    typename Vec<D>::T yj[U];
#pragma unroll
    for (int u = 0; u < U; u++) yj[u] = __ldg(&Y[pr[u].x]);
#pragma unroll
    for (int u = 0; u < U; u++) attr_term<D>(yi, yj[u], __int_as_float(pr[u].y), acc);
  }
}

// sum the partial row sums of a G-lane group (all 32 lanes must call it)
template <int D, int G>
__device__ __forceinline__ void group_reduce(float *acc) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1)
#pragma unroll
    for (int k = 0; k < D; k++) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o, G);
}

__device__ __forceinline__ float sgn_f(float x) {
  return x == 0.f ? 0.f : (x < 0.f ? -1.f : 1.f);
}

// Per-block min/max/sum of Ynext -> partials; the last block reduces all
// partials with every thread and turns them into the next grid decision.
template <int D>
__device__ __forceinline__ void block_finish_stats(int vb_, int vg_, SgtState *st, const SgtJobParams &jp,
                                                   float *mn, float *mx, double *sm,
                                                   float4 *part_min, float4 *part_max,
                                                   double *part_sum, int iter, float alpha,
                                                   float mom) {
  __shared__ float smin[SGT_THREADS / 32][3], smax[SGT_THREADS / 32][3];
  __shared__ double ssum[SGT_THREADS / 32][3];
  __shared__ bool last;
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < D; k++) {
    const float a = warp_min_f(mn[k]), b = warp_max_f(mx[k]);
    const double s = warp_sum_d(sm[k]);
    if (l == 0) { smin[w][k] = a; smax[w][k] = b; ssum[w][k] = s; }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float4 a = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
    float4 b = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
    double s[3] = {0, 0, 0};
    for (int j = 0; j < SGT_THREADS / 32; j++) {
      a.x = fminf(a.x, smin[j][0]); b.x = fmaxf(b.x, smax[j][0]); s[0] += ssum[j][0];
      if (D > 1) { a.y = fminf(a.y, smin[j][1]); b.y = fmaxf(b.y, smax[j][1]); s[1] += ssum[j][1]; }
      if (D > 2) { a.z = fminf(a.z, smin[j][2]); b.z = fmaxf(b.z, smax[j][2]); s[2] += ssum[j][2]; }
    }
    part_min[vb_] = a;
    part_max[vb_] = b;
    for (int k = 0; k < 3; k++) part_sum[vb_ * 4 + k] = s[k];
    __threadfence();
    last = (atomicAdd(&st->done_row, 1u) == vg_ - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  double s[3] = {0, 0, 0};
  for (int b = threadIdx.x; b < (int)vg_; b += blockDim.x) {
    const float4 a = __ldcg(&part_min[b]), c = __ldcg(&part_max[b]);
    lo[0] = fminf(lo[0], a.x); hi[0] = fmaxf(hi[0], c.x);
    lo[1] = fminf(lo[1], a.y); hi[1] = fmaxf(hi[1], c.y);
    lo[2] = fminf(lo[2], a.z); hi[2] = fmaxf(hi[2], c.z);
    for (int k = 0; k < D; k++) s[k] += __ldcg(&part_sum[b * 4 + k]);
  }
  // fixed-order tree: warp shuffles then warp 0 over the warp results
#pragma unroll
  for (int k = 0; k < D; k++) {
    lo[k] = warp_min_f(lo[k]);
    hi[k] = warp_max_f(hi[k]);
    s[k] = warp_sum_d(s[k]);
  }
  __syncthreads();
  if (l == 0)
    for (int k = 0; k < D; k++) { smin[w][k] = lo[k]; smax[w][k] = hi[k]; ssum[w][k] = s[k]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < D; k++) {
      lo[k] = INFINITY; hi[k] = -INFINITY; s[k] = 0;
      for (int j = 0; j < SGT_THREADS / 32; j++) {
        lo[k] = fminf(lo[k], smin[j][k]);
        hi[k] = fmaxf(hi[k], smax[j][k]);
        s[k] += ssum[j][k];
      }
      st->minv[k] = lo[k];
      st->maxv[k] = hi[k];
      st->sum[k] = s[k];
      if (!isfinite(lo[k]) || !isfinite(hi[k])) st->error |= SGT_EFLAG_NONFINITE;
    }
    sgt_finalize_grid<D>(st, jp, lo, hi, s, true);
    st->alpha = alpha;
    st->momentum = mom;
    st->iter = iter + 1;
    st->done_row = 0;
  }
}


// ---------------------------------------------------------------------------
// Fused iteration row kernel.  FUSED: compute F_attr from CSR; otherwise read
// it from Fattr (COO / ELL formats).  Writes Ynext, uY, gains; the last CTA
// turns the per-block min/max/sum of Ynext into the next grid decision.
// ---------------------------------------------------------------------------
template <int D, int G, bool FUSED>
__device__ __forceinline__ void k_row_update_body(int vb_, int vg_, const int *__restrict__ rowptr, const int2 *__restrict__ pairs,
             const typename Vec<D>::T *__restrict__ Fattr,
             const typename Vec<D>::T *__restrict__ Y,
             const typename Vec<D>::T *__restrict__ Frep_un,
             typename Vec<D>::T *__restrict__ uY,
             typename Vec<D>::T *__restrict__ gains,
             typename Vec<D>::T *__restrict__ Ynext, SgtState *st,
             SgtJobParams jp, float4 *part_min, float4 *part_max,
             double *part_sum) {
  const int n = jp.n;
  const int iter = st->iter;
  const float alpha = iter <= jp.early_iter ? jp.alpha0 : 1.0f;
  const float mom = iter <= jp.mom_switch ? 0.5f : 0.8f;
  const float eta = jp.eta;
  const float Zf = (float)st->Z;
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  double sm[3] = {0, 0, 0};
  const int lane = threadIdx.x % G;
  const int grp = (vb_ * blockDim.x + threadIdx.x) / G;
  const int ngrp = vg_ * blockDim.x / G;
  // uniform trip count per warp so the group shuffles stay converged
  const int rounds = (n + ngrp - 1) / ngrp;
  // the next row's extents are loaded one round ahead
  int nb_s = 0, nb_e = 0;
  if (FUSED && grp < n) {
    nb_s = __ldcs(&rowptr[grp]);
    nb_e = __ldcs(&rowptr[grp + 1]);
  }
  for (int r = 0; r < rounds; r++) {
    const int i = grp + r * ngrp;
    const bool valid = i < n;
    const int rs = nb_s, re = nb_e;
    if (FUSED && i + ngrp < n) {
      nb_s = __ldcs(&rowptr[i + ngrp]);
      nb_e = __ldcs(&rowptr[i + ngrp + 1]);
    }
    typename Vec<D>::T yi, fr, u, g;
    if (valid) {
      yi = Y[i];
      if (lane == 0) {  // update operands, independent of the row sum
        fr = __ldcs(&Frep_un[i]);
        u = __ldcs(&uY[i]);
        g = __ldcs(&gains[i]);
      }
    }
    float acc[3] = {0.f, 0.f, 0.f};
    if (FUSED) {
      if (valid) {
        constexpr int U = 4;
        for (int t0 = rs + lane; t0 < re; t0 += U * G) {
          int2 pr[U];
#pragma unroll
          for (int q = 0; q < U; q++) {
            const int t = t0 + q * G;
            pr[q] = t < re ? __ldcs(&pairs[t]) : make_int2(i, 0);
          }
          typename Vec<D>::T yj[U];
#pragma unroll
          for (int q = 0; q < U; q++) yj[q] = __ldg(&Y[pr[q].x]);
#pragma unroll
          for (int q = 0; q < U; q++) attr_term<D>(yi, yj[q], __int_as_float(pr[q].y), acc);
        }
      }
      group_reduce<D, G>(acc);
    } else if (valid) {
      const typename Vec<D>::T fa = Fattr[i];
#pragma unroll
      for (int k = 0; k < D; k++) acc[k] = comp<D>(fa, k);
    }
    if (valid && lane == 0) {
      typename Vec<D>::T yn = yi;
#pragma unroll
      for (int k = 0; k < D; k++) {
        const float frep = comp<D>(fr, k) / Zf;
        const float dy = alpha * acc[k] - frep;
        float gk = comp<D>(g, k), uk = comp<D>(u, k);
        gk = (sgn_f(dy) != sgn_f(uk)) ? (float)((double)gk + 0.2) : (float)((double)gk * 0.8);
        if ((double)gk < 0.01) gk = (float)0.01;
        uk = mom * uk - eta * gk * dy;
        const float y = comp<D>(yi, k) + uk;
        setcomp<D>(g, k, gk);
        setcomp<D>(u, k, uk);
        setcomp<D>(yn, k, y);
        mn[k] = fminf(mn[k], y);
        mx[k] = fmaxf(mx[k], y);
        sm[k] += (double)y;
      }
      if constexpr (D == 3) { u.w = 0.f; g.w = 0.f; yn.w = 0.f; }
      __stcs(&uY[i], u);
      __stcs(&gains[i], g);
      Ynext[i] = yn;
    }
  }
  block_finish_stats<D>(vb_, vg_, st, jp, mn, mx, sm, part_min, part_max, part_sum, iter, alpha, mom);
}
template <int D, int G, bool FUSED>
__global__ void __launch_bounds__(SGT_THREADS)
k_row_update(const int *__restrict__ rowptr, const int2 *__restrict__ pairs,
             const typename Vec<D>::T *__restrict__ Fattr,
             const typename Vec<D>::T *__restrict__ Y,
             const typename Vec<D>::T *__restrict__ Frep_un,
             typename Vec<D>::T *__restrict__ uY,
             typename Vec<D>::T *__restrict__ gains,
             typename Vec<D>::T *__restrict__ Ynext, SgtState *st,
             SgtJobParams jp, float4 *part_min, float4 *part_max,
             double *part_sum) {
  k_row_update_body<D, G, FUSED>(blockIdx.x, gridDim.x, rowptr, pairs, Fattr, Y, Frep_un, uY, gains, Ynext, st, jp, part_min, part_max, part_sum);
}


// ---------------------------------------------------------------------------
// Attractive term of the CSR path: one row per G-lane group, launched over
// all rows (ceil(n G / 256) blocks; the hardware refills SMs as blocks
// retire, so a long row delays one group, not a persistent warp).  Kept lean
// (no loop state across rows) so 48+ warps stay resident per SM.  It reads
// only Y and P, so the iteration runs it as a graph branch beside the
// repulsion chain; k_row_update combines the two forces.  Row i is point
// row0 + i of Y (a shard of a row-split embedding holds rows row0.. of P
// with global column indices and gathers from the whole Y).
// ---------------------------------------------------------------------------
template <int D, int G>
__device__ __forceinline__ void k_attr_rows_body(int vb_, int vg_, const int *__restrict__ rowptr, const int2 *__restrict__ pairs,
            const typename Vec<D>::T *__restrict__ Y, typename Vec<D>::T *__restrict__ Fattr,
            int n, int row0) {
  const int lane = threadIdx.x % G;
  const int i = (vb_ * blockDim.x + threadIdx.x) / G;
  const bool valid = i < n;
  float acc[3] = {0.f, 0.f, 0.f};
  if (valid) {
    const typename Vec<D>::T yi = Y[row0 + i];
    csr_row_sum<D, G>(rowptr, pairs, Y, i, lane, yi, acc);
  }
  group_reduce<D, G>(acc);
  if (valid && lane == 0) {
    typename Vec<D>::T f;
    if constexpr (D == 3) f.w = 0.f;
#pragma unroll
    for (int k = 0; k < D; k++) setcomp<D>(f, k, acc[k]);
    Fattr[i] = f;
  }
}
template <int D, int G>
__global__ void __launch_bounds__(SGT_THREADS, (D == 3 ? 6 : 8))
k_attr_rows(const int *__restrict__ rowptr, const int2 *__restrict__ pairs,
            const typename Vec<D>::T *__restrict__ Y, typename Vec<D>::T *__restrict__ Fattr,
            int n, int row0) {
  k_attr_rows_body<D, G>(blockIdx.x, gridDim.x, rowptr, pairs, Y, Fattr, n, row0);
}

// ---------------------------------------------------------------------------
// Attractive term only (operator entry points and the COO/ELL formats).
// ---------------------------------------------------------------------------
template <int D, int G>
__global__ void __launch_bounds__(SGT_THREADS)
k_attr_csr(const int *__restrict__ rowptr, const int2 *__restrict__ pairs,
           const typename Vec<D>::T *__restrict__ Y, typename Vec<D>::T *__restrict__ F,
           int n) {
  const int lane = threadIdx.x % G;
  const int ngrp = gridDim.x * blockDim.x / G;
  const int grp0 = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  // uniform trip count per warp so the group shuffles stay converged
  const int rounds = (n + ngrp - 1) / ngrp;
  for (int r = 0; r < rounds; r++) {
    const int i = grp0 + r * ngrp;
    float acc[3] = {0.f, 0.f, 0.f};
    if (i < n) {
      const typename Vec<D>::T yi = Y[i];
      csr_row_sum<D, G>(rowptr, pairs, Y, i, lane, yi, acc);
    }
    group_reduce<D, G>(acc);
    if (i < n && lane == 0) {
      typename Vec<D>::T f;
      if constexpr (D == 3) f.w = 0.f;
#pragma unroll
      for (int k = 0; k < D; k++) setcomp<D>(f, k, acc[k]);
      F[i] = f;
    }
  }
}

// ELL part, column-major slots (CU/hybridpq.cu:4-70): one thread per row,
// overwrites F.
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_attr_ell(int n, int W, const unsigned *__restrict__ cols,
           const float *__restrict__ vals, const typename Vec<D>::T *__restrict__ Y,
           typename Vec<D>::T *__restrict__ F) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const typename Vec<D>::T yi = Y[i];
    float acc[3] = {0.f, 0.f, 0.f};
    for (int k = 0; k < W; k++) {
      const long s = (long)k * n + i;
      const unsigned c = __ldg(&cols[s]);
      attr_term<D>(yi, __ldg(&Y[c]), __ldg(&vals[s]), acc);
    }
    typename Vec<D>::T f;
    if constexpr (D == 3) f.w = 0.f;
#pragma unroll
    for (int k = 0; k < D; k++) setcomp<D>(f, k, acc[k]);
    F[i] = f;
  }
}

// COO (rows sorted, CU/pq.cuh:77-118 and the hybrid tail CU/hybridpq.cu:71-113):
// one element per lane, warp segmented sum by row, one atomic per segment.
// F must hold the ELL result or zero.
template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
k_attr_coo(long nnz, const unsigned *__restrict__ rows, const unsigned *__restrict__ cols,
           const float *__restrict__ vals, const typename Vec<D>::T *__restrict__ Y,
           float *__restrict__ F /* Vec<D> viewed as floats */) {
  constexpr int S = D == 3 ? 4 : D;
  const int lane = threadIdx.x & 31;
  const long warps = (long)gridDim.x * blockDim.x / 32;
  for (long base = ((long)blockIdx.x * blockDim.x + threadIdx.x) / 32 * 32; base < nnz;
       base += warps * 32) {
    const long e = base + lane;
    const bool ok = e < nnz;
    unsigned r = ok ? __ldg(&rows[e]) : 0xffffffffu;
    float acc[3] = {0.f, 0.f, 0.f};
    if (ok) attr_term<D>(__ldg(&Y[r]), __ldg(&Y[__ldg(&cols[e])]), __ldg(&vals[e]), acc);
    // segmented inclusive scan (rows are non-decreasing along the warp)
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned ro = __shfl_up_sync(0xffffffffu, r, o);
#pragma unroll
      for (int k = 0; k < D; k++) {
        const float v = __shfl_up_sync(0xffffffffu, acc[k], o);
        if (lane >= o && ro == r) acc[k] += v;
      }
    }
    const unsigned rn = __shfl_down_sync(0xffffffffu, r, 1);
    const bool tail = ok && (lane == 31 || rn != r);
    if (tail) {
#pragma unroll
      for (int k = 0; k < D; k++) atomicAdd(&F[(long)r * S + k], acc[k]);
    }
  }
}

// ---------------------------------------------------------------------------
// KL divergence (FP64 terms and sum; fixed-order finish in the last CTA)
// ---------------------------------------------------------------------------
template <int D, int G>
__global__ void __launch_bounds__(SGT_THREADS)
k_kl(const int *__restrict__ rowptr, const int2 *__restrict__ pairs,
     const typename Vec<D>::T *__restrict__ Y, SgtState *st, double alpha,
     double *part, int n) {
  __shared__ double ws[SGT_THREADS / 32];
  __shared__ bool last;
  const double Z = st->Z;
  const int lane = threadIdx.x % G;
  const int ngrp = gridDim.x * blockDim.x / G;
  double acc = 0.0;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / G; i < n; i += ngrp) {
    const typename Vec<D>::T yi = Y[i];
    for (int t = rowptr[i] + lane; t < rowptr[i + 1]; t += G) {
      const int2 pr = pairs[t];
      const typename Vec<D>::T yj = Y[pr.x];
      double dist = 0;
#pragma unroll
      for (int k = 0; k < D; k++) {
        const double df = (double)comp<D>(yi, k) - (double)comp<D>(yj, k);
        dist += df * df;
      }
      const double p = alpha * (double)__int_as_float(pr.y);
      const double q = (1.0 / (1.0 + dist)) / Z;
      const double fmin = 1.17549435082228750797e-38;
      acc += p * log((p + fmin) / (q + fmin));
    }
  }
  acc = warp_sum_d(acc);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int k = 0; k < SGT_THREADS / 32; k++) s += ws[k];
    part[blockIdx.x] = s;
    __threadfence();
    last = (atomicAdd(&st->done_kl, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double s = 0;
    for (int b = 0; b < (int)gridDim.x; b++) s += __ldcg(&part[b]);
    st->kl = s;
    st->done_kl = 0;
  }
}

// ---------------------------------------------------------------------------
// layout conversion between the caller's arrays and the padded point-major
// layout.  dim_major: src[i + k*n]; otherwise src[i*d + k].
// ---------------------------------------------------------------------------
template <int D>
__global__ void k_pack(const float *__restrict__ src, int n, int dim_major,
                       typename Vec<D>::T *__restrict__ dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    typename Vec<D>::T v;
    if constexpr (D == 3) v.w = 0.f;
#pragma unroll
    for (int k = 0; k < D; k++)
      setcomp<D>(v, k, dim_major ? src[i + (long)k * n] : src[(long)i * D + k]);
    dst[i] = v;
  }
}
template <int D>
__global__ void k_unpack(const typename Vec<D>::T *__restrict__ src, int n,
                         int dim_major, float scale, const float *__restrict__ shift,
                         float *__restrict__ dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const typename Vec<D>::T v = src[i];
#pragma unroll
    for (int k = 0; k < D; k++) {
      float x = comp<D>(v, k);
      if (shift) x = x - shift[k];
      x = x * scale;
      if (dim_major) dst[i + (long)k * n] = x; else dst[(long)i * D + k] = x;
    }
  }
}

// dst[r] = src[perm[r]] (user order -> engine order), Vec<D> arrays
template <int D>
__global__ void k_permute_vec(const typename Vec<D>::T *__restrict__ src,
                              const int *__restrict__ perm, int n,
                              typename Vec<D>::T *__restrict__ dst) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    dst[r] = src[perm[r]];
}

