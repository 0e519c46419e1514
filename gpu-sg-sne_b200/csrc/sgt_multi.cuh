// sgt_multi.cuh -- one launch per stage of the iteration over many jobs.
//
// A batch of independent embeddings (sgt_batch_*) runs every stage of an
// iteration as one launch over all its jobs of one dimension, instead of one
// launch per job.  Every iteration kernel is written as a body that takes its
// block index and block count as arguments (k_*_body); here each block of a
// fused launch looks up the job it belongs to in a prefix table of the jobs'
// block counts, and runs that job's body with the job's own block index and
// count and the job's buffers from a table of job views.  A job thus sees
// exactly the blocks, reductions and last-block finishes of its own launch,
// and thousands of small launches become a dozen per iteration.
#pragma once
#include "sgt_common.cuh"
#include "sgt_fft.cuh"
#include "sgt_grid.cuh"
#include "sgt_rows.cuh"

struct SgtJobView {
  const void *Ynext_c;
  void *Ynext, *Y, *uY, *gains, *Frep, *Fattr;
  float4 *sorted;
  void *V, *Phi;
  float2 *W;
  int *tile_count, *cursor;
  int4 *chunks;
  float4 *part_min, *part_max;
  double *part_sum, *part_z;
  SgtState *st;
  const int *rowptr;
  const int2 *pairs;
  SgtJobParams jp;
  int n, nb_s2g, row0, pad;
};

// the job of block b: the last j with prefix[j] <= b (prefix has njobs + 1
// entries, prefix[0] = 0, prefix[njobs] = the launch's block count)
__device__ __forceinline__ int sgt_job_of(const int *__restrict__ prefix, int njobs, int b) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&prefix[mid]) <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

#define SGT_MULTI_JOB                                                  \
  const int j_ = sgt_job_of(prefix, njobs, blockIdx.x);                \
  const SgtJobView &v = views[j_];                                     \
  const int vb = blockIdx.x - __ldg(&prefix[j_]);                      \
  const int vg = __ldg(&prefix[j_ + 1]) - __ldg(&prefix[j_]);

template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
km_bin_count(const SgtJobView *__restrict__ views, const int *__restrict__ prefix, int njobs) {
  SGT_MULTI_JOB
  typedef typename Vec<D>::T VT;
  k_bin_count_body<D>(vb, vg, (const VT *)v.Ynext_c, (VT *)v.Y, v.n, v.st, v.tile_count,
                      (typename Node<D>::T *)v.V, 1, v.jp, v.cursor, v.chunks, v.nb_s2g);
}

template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
km_bin_scatter(const SgtJobView *__restrict__ views, const int *__restrict__ prefix, int njobs) {
  SGT_MULTI_JOB
  k_bin_scatter_body<D>(vb, vg, (const typename Vec<D>::T *)v.Y, v.n, v.st, v.cursor, v.sorted);
}

template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
km_s2g_direct(const SgtJobView *__restrict__ views, const int *__restrict__ prefix, int njobs) {
  SGT_MULTI_JOB
  k_s2g_direct_body<D>(vb, vg, (const typename Vec<D>::T *)v.Y, v.n, v.st,
                       (typename Node<D>::T *)v.V);
}

template <int D, int TT>
__global__ void __launch_bounds__(SGT_THREADS)
km_s2g(const SgtJobView *__restrict__ views, const int *__restrict__ prefix, int njobs) {
  SGT_MULTI_JOB
  k_s2g_body<D, TT>(vb, vg, v.sorted, v.st, v.chunks, (typename Node<D>::T *)v.V);
}

template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
km_s2g_cell(const SgtJobView *__restrict__ views, const int *__restrict__ prefix, int njobs) {
  SGT_MULTI_JOB
  k_s2g_cell_body<D>(vb, vg, v.sorted, v.st, v.chunks, (typename Node<D>::T *)v.V);
}

__global__ void __launch_bounds__(SGT_THREADS)
km_conv1d(const SgtJobView *__restrict__ views, const int *__restrict__ prefix, int njobs) {
  SGT_MULTI_JOB
  k_conv1d_body(vb, vg, v.st, (const float2 *)v.V, (float2 *)v.Phi);
}

template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
km_fft_build_x(const SgtJobView *__restrict__ views, const int *__restrict__ prefix, int njobs) {
  SGT_MULTI_JOB
  k_fft_build_x_body<D>(vb, vg, v.st, (const typename Node<D>::T *)v.V, v.W);
}

template <int D, int MODE>
__global__ void __launch_bounds__(SGT_THREADS)
km_fft_cols(const SgtJobView *__restrict__ views, const int *__restrict__ prefix, int njobs) {
  SGT_MULTI_JOB
  k_fft_cols_body<D, MODE>(vb, vg, v.st, v.W, (const typename Node<D>::T *)v.V,
                           (typename Node<D>::T *)v.Phi);
}

template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
km_fft_final_x(const SgtJobView *__restrict__ views, const int *__restrict__ prefix, int njobs) {
  SGT_MULTI_JOB
  k_fft_final_x_body<D>(vb, vg, v.st, v.W, (typename Node<D>::T *)v.Phi);
}

template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
km_g2s(const SgtJobView *__restrict__ views, const int *__restrict__ prefix, int njobs) {
  SGT_MULTI_JOB
  typedef typename Vec<D>::T VT;
  k_g2s_body<D>(vb, vg, v.sorted, v.st, v.chunks, (const typename Node<D>::T *)v.Phi,
                (VT *)v.Frep, v.part_z, v.n);
}

template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
km_g2s_direct(const SgtJobView *__restrict__ views, const int *__restrict__ prefix, int njobs) {
  SGT_MULTI_JOB
  typedef typename Vec<D>::T VT;
  k_g2s_direct_body<D>(vb, vg, v.st, (const typename Node<D>::T *)v.Phi, (VT *)v.Frep, v.part_z,
                       v.n, (const VT *)v.Y);
}

template <int D, int G>
__global__ void __launch_bounds__(SGT_THREADS, (D == 3 ? 6 : 8))
km_attr_rows(const SgtJobView *__restrict__ views, const int *__restrict__ prefix, int njobs) {
  SGT_MULTI_JOB
  typedef typename Vec<D>::T VT;
  k_attr_rows_body<D, G>(vb, vg, v.rowptr, v.pairs, (const VT *)v.Ynext_c, (VT *)v.Fattr, v.n,
                         v.row0);
}

template <int D>
__global__ void __launch_bounds__(SGT_THREADS)
km_row_update(const SgtJobView *__restrict__ views, const int *__restrict__ prefix, int njobs) {
  SGT_MULTI_JOB
  typedef typename Vec<D>::T VT;
  k_row_update_body<D, 1, false>(vb, vg, nullptr, nullptr, (const VT *)v.Fattr, (const VT *)v.Y,
                                 (const VT *)v.Frep, (VT *)v.uY, (VT *)v.gains, (VT *)v.Ynext,
                                 v.st, v.jp, v.part_min, v.part_max, v.part_sum);
}
