// sgt_knn.cu -- exact k nearest neighbours on the device: the kNN stage in
// front of the perplexity equalisation (the reference's command line tool
// calls FLANN, an approximate search, at
// CU/testing_modules/demo_perplexity.cu:131; this search is exact).
//
// One query per thread, 128 queries per CTA.  Candidates stream through
// shared memory in tiles of 64 points x 64 dimensions, queries in tiles of
// 128 x 64; rows are padded to 68 floats so each thread's float4 loads of
// its query and the (broadcast) float4 loads of a candidate are free of bank
// conflicts.  Each thread accumulates the 64 squared distances of a tile in
// registers as sums of squared differences (not |x|^2 + |y|^2 - 2 x.y, whose
// cancellation would reorder near neighbours), then offers them to its
// sorted top-k list (local memory) behind a threshold test: after the list
// fills, only candidates closer than its current k-th neighbour are
// inserted, so insertions are rare.  The self match is skipped.  Output rows
// are sorted by distance, ties by index.
#include "../../include/sgtsne_b200.h"
#include "sgt_internal.h"

#include <string>

namespace {

constexpr int KNN_Q = 128;   // queries per CTA
constexpr int KNN_C = 64;    // candidates per tile
constexpr int KNN_DC = 64;   // dimensions per chunk
constexpr int KNN_LD = KNN_DC + 4;
constexpr int KNN_MAXK = 128;

__device__ __forceinline__ bool knn_less(float da, int ia, float db, int ib) {
  return da < db || (da == db && ia < ib);
}

__global__ void __launch_bounds__(KNN_Q)
k_knn(const float *__restrict__ X, int n, int dim, int k, int *__restrict__ idx,
      float *__restrict__ d2) {
  extern __shared__ float sm[];
  float *sQ = sm;                   // [KNN_Q][KNN_LD]
  float *sC = sm + KNN_Q * KNN_LD;  // [KNN_C][KNN_LD]
  const int t = threadIdx.x;
  const int q0 = blockIdx.x * KNN_Q, q = q0 + t;
  float bd[KNN_MAXK];
  int bi[KNN_MAXK];
  int cnt = 0;
  float thr = INFINITY;
  int thi = 0x7fffffff;
  for (int c0 = 0; c0 < n; c0 += KNN_C) {
    float acc[KNN_C];
#pragma unroll
    for (int c = 0; c < KNN_C; c++) acc[c] = 0.f;
    for (int k0 = 0; k0 < dim; k0 += KNN_DC) {
      __syncthreads();
      for (int e = t; e < KNN_Q * KNN_DC; e += KNN_Q) {
        const int r = e / KNN_DC, cc = e % KNN_DC;
        const int gq = q0 + r, gk = k0 + cc;
        sQ[r * KNN_LD + cc] = (gq < n && gk < dim) ? X[(long)gq * dim + gk] : 0.f;
      }
      for (int e = t; e < KNN_C * KNN_DC; e += KNN_Q) {
        const int r = e / KNN_DC, cc = e % KNN_DC;
        const int gc = c0 + r, gk = k0 + cc;
        sC[r * KNN_LD + cc] = (gc < n && gk < dim) ? X[(long)gc * dim + gk] : 0.f;
      }
      __syncthreads();
      const int kmax = min(KNN_DC, dim - k0);  // zero padding adds nothing
      for (int kk = 0; kk < kmax; kk += 4) {
        const float4 qv = *reinterpret_cast<const float4 *>(&sQ[t * KNN_LD + kk]);
#pragma unroll
        for (int c = 0; c < KNN_C; c++) {
          const float4 cv = *reinterpret_cast<const float4 *>(&sC[c * KNN_LD + kk]);
          float df = qv.x - cv.x;
          acc[c] = fmaf(df, df, acc[c]);
          df = qv.y - cv.y;
          acc[c] = fmaf(df, df, acc[c]);
          df = qv.z - cv.z;
          acc[c] = fmaf(df, df, acc[c]);
          df = qv.w - cv.w;
          acc[c] = fmaf(df, df, acc[c]);
        }
      }
    }
    if (q < n) {
#pragma unroll
      for (int c = 0; c < KNN_C; c++) {
        const int j = c0 + c;
        const float dd = acc[c];
        if (j >= n || j == q) continue;
        if (cnt == k && !knn_less(dd, j, thr, thi)) continue;
        // insert into the sorted list (drop the last when full)
        int p = cnt < k ? cnt : k - 1;
        while (p > 0 && knn_less(dd, j, bd[p - 1], bi[p - 1])) {
          bd[p] = bd[p - 1];
          bi[p] = bi[p - 1];
          p--;
        }
        bd[p] = dd;
        bi[p] = j;
        if (cnt < k) cnt++;
        if (cnt == k) {
          thr = bd[k - 1];
          thi = bi[k - 1];
        }
      }
    }
  }
  if (q < n) {
    for (int s = 0; s < k; s++) {
      idx[(long)q * k + s] = s < cnt ? bi[s] : -1;
      d2[(long)q * k + s] = s < cnt ? bd[s] : INFINITY;
    }
  }
}

}  // namespace

extern "C" sgt_status sgt_knn(sgt_ctx *ctx, int n, int dim, const float *X, int k, int *idx,
                              float *d2) {
  if (!ctx || !X || !idx || !d2) return SGT_ERR_INVALID_ARG;
  if (n < 2 || dim < 1 || k < 1) return sgti_fail(ctx, SGT_ERR_INVALID_ARG, "sgt_knn: sizes");
  if (k > KNN_MAXK || k >= n)
    return sgti_fail(ctx, SGT_ERR_UNSUPPORTED,
                     "sgt_knn: k must be below n and at most " + std::to_string(KNN_MAXK));
  if (cudaSetDevice(sgti_device(ctx)) != cudaSuccess)
    return sgti_fail(ctx, SGT_ERR_CUDA, "sgt_knn: set device");
  const size_t smem = sizeof(float) * (size_t)(KNN_Q + KNN_C) * KNN_LD;
  cudaError_t e = cudaFuncSetAttribute(k_knn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e == cudaSuccess) {
    const int nb = (n + KNN_Q - 1) / KNN_Q;
    k_knn<<<nb, KNN_Q, smem, sgti_stream(ctx)>>>(X, n, dim, k, idx, d2);
    e = cudaGetLastError();
    // like the other preparation operators, return with the result ready
    if (e == cudaSuccess) e = cudaStreamSynchronize(sgti_stream(ctx));
  }
  if (e != cudaSuccess)
    return sgti_fail(ctx, SGT_ERR_CUDA, std::string("sgt_knn: ") + cudaGetErrorString(e));
  return SGT_OK;
}
