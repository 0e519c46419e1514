// Test-only harness around the reference's lambda bisection
// (code/cuda/SG-tSNE-CUDA/src/graph_rescaling.cu:11-107: bisectionSearchKernel,
// one warp per row, on the raw values; lambdaRescalingGPU launches it on
// 64 x 512 threads).  Compiled in place from the reference tree by
// oracle/build_ref.sh with cusparse_legacy_shim.h force-included.  Test use
// only: golden vectors for the engine's sgt_lambda_bisect.
#include <cuda_runtime.h>
#include <cstring>
#include "graph_rescaling.cuh"

// rowptr (n+1) and val (nnz, rescaled in place) on the host.  Returns a CUDA
// error code (0 on success).
extern "C" int ref_cu_lambda_rescale(int n, const int *rowptr, float *val, float lambda,
                                     int drop_leaf) {
  const int nnz = rowptr[n];
  int *dr = nullptr;
  float *dv = nullptr;
  cudaMalloc(&dr, sizeof(int) * (size_t)(n + 1));
  cudaMalloc(&dv, sizeof(float) * (size_t)(nnz > 0 ? nnz : 1));
  cudaMemcpy(dr, rowptr, sizeof(int) * (size_t)(n + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(dv, val, sizeof(float) * (size_t)nnz, cudaMemcpyHostToDevice);
  sparse_matrix<matval> P;
  memset(&P, 0, sizeof(P));
  P.m = n;
  P.n = n;
  P.nnz = nnz;
  P.row = dr;
  P.val = dv;
  lambdaRescalingGPU(P, lambda, true, drop_leaf != 0);
  cudaError_t e = cudaDeviceSynchronize();
  cudaMemcpy(val, dv, sizeof(float) * (size_t)nnz, cudaMemcpyDeviceToHost);
  cudaFree(dr);
  cudaFree(dv);
  return (int)e;
}
