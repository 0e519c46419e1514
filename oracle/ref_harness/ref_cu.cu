// Test-only harness around the reference's FP32 CUDA kernels
// (code/cuda/SG-tSNE-CUDA/src): AttractiveEstimation in COO format
// (pq.cu:24-57) and computeFrepulsive_interp on the fixed grid
// (Frep.cu:81-125, buffers and cuFFT plans set up as gradient_descend.cu:
// 137-188 does).  Compiled in place from the reference tree by
// oracle/build_ref.sh; used only to produce golden vectors.
#include <cmath>
#include <vector>
#include "Frep.cuh"
#include "pq.cuh"
#include "types.hpp"

int Blocks = 592;
int Threads = 256;
cudaStream_t streamAttr = 0;
cudaStream_t streamRep = 0;

extern "C" int ref_cu_attractive_coo(int n, int d, int nnz, const int *rows, const int *cols,
                                     const float *vals, const float *y_dim_major, float *F) {
  int *dr, *dc;
  float *dv, *dy, *dF;
  cudaMalloc(&dr, sizeof(int) * nnz);
  cudaMalloc(&dc, sizeof(int) * nnz);
  cudaMalloc(&dv, sizeof(float) * nnz);
  cudaMalloc(&dy, sizeof(float) * n * d);
  cudaMalloc(&dF, sizeof(float) * n * d);
  cudaMemcpy(dr, rows, sizeof(int) * nnz, cudaMemcpyHostToDevice);
  cudaMemcpy(dc, cols, sizeof(int) * nnz, cudaMemcpyHostToDevice);
  cudaMemcpy(dv, vals, sizeof(float) * nnz, cudaMemcpyHostToDevice);
  cudaMemcpy(dy, y_dim_major, sizeof(float) * n * d, cudaMemcpyHostToDevice);
  cudaMemset(dF, 0, sizeof(float) * n * d);
  sparse_matrix<float> P;
  memset(&P, 0, sizeof(P));
  P.n = n;
  P.m = n;
  P.nnz = nnz;
  P.format = 2;
  P.row = dr;
  P.col = dc;
  P.val = dv;
  AttractiveEstimation(P, d, dy, dF);
  cudaError_t e = cudaDeviceSynchronize();
  cudaMemcpy(F, dF, sizeof(float) * n * d, cudaMemcpyDeviceToHost);
  cudaFree(dr); cudaFree(dc); cudaFree(dv); cudaFree(dy); cudaFree(dF);
  return (int)e;
}

// Returns Z; F and y are dim-major (the CU layout); *grid = points per axis.
extern "C" float ref_cu_repulsive_fixed(int n, int d, int ng, const float *y_dim_major, float *F,
                                        int *grid) {
  const int n1 = getBestGridSize(ng), n2 = n1 + 2, m = d + 1, nVec = d + 1;
  cufftHandle plan, plan_rhs;
  if (d == 1) {
    int sz[1] = {n2};
    cufftPlan1d(&plan, n2, CUFFT_C2C, 1);
    cufftPlanMany(&plan_rhs, 1, sz, NULL, 1, n2, NULL, 1, n2, CUFFT_C2C, d + 1);
  } else if (d == 2) {
    int sz[2] = {n2, n2};
    cufftPlan2d(&plan, n2, n2, CUFFT_C2C);
    cufftPlanMany(&plan_rhs, 2, sz, NULL, 1, n2 * n2, NULL, 1, n2 * n2, CUFFT_C2C, d + 1);
  } else {
    int sz[3] = {n2, n2, n2};
    cufftPlanMany(&plan, 3, sz, NULL, 1, 0, NULL, 1, 0, CUFFT_C2C, 1);
    cufftPlanMany(&plan_rhs, 3, sz, NULL, 1, n2 * n2 * n2, NULL, 1, n2 * n2 * n2, CUFFT_C2C, d + 1);
  }
  const int szV = (int)std::pow((double)n2, d) * m;
  float *y, *yt, *VScat, *PhiScat, *VGrid, *PhiGrid, *Frep;
  ComplexF *Kc, *Xc;
  cudaMallocManaged(&y, sizeof(float) * n * d);
  cudaMallocManaged(&yt, sizeof(float) * n * d);
  cudaMallocManaged(&VScat, sizeof(float) * n * m);
  cudaMallocManaged(&PhiScat, sizeof(float) * n * m);
  cudaMallocManaged(&VGrid, sizeof(float) * szV);
  cudaMallocManaged(&PhiGrid, sizeof(float) * szV);
  cudaMallocManaged(&Kc, sizeof(ComplexF) * szV);
  cudaMallocManaged(&Xc, sizeof(ComplexF) * nVec * szV);
  cudaMallocManaged(&Frep, sizeof(float) * n * d);
  cudaMemcpy(y, y_dim_major, sizeof(float) * n * d, cudaMemcpyHostToDevice);
  cudaMemset(VGrid, 0, sizeof(float) * szV);
  cudaMemset(PhiGrid, 0, sizeof(float) * szV);
  cudaDeviceSynchronize();
  thrust::device_vector<float> zetaVec(n);
  double time_info[8] = {0};
  const float z = computeFrepulsive_interp<float, ComplexF>(Frep, y, n, d, 0.0f, time_info, n1, plan,
                                                            plan_rhs, yt, VScat, PhiScat, VGrid,
                                                            PhiGrid, Kc, Xc, zetaVec);
  cudaDeviceSynchronize();
  cudaMemcpy(F, Frep, sizeof(float) * n * d, cudaMemcpyDeviceToHost);
  *grid = n2;
  cufftDestroy(plan);
  cufftDestroy(plan_rhs);
  cudaFree(y); cudaFree(yt); cudaFree(VScat); cudaFree(PhiScat); cudaFree(VGrid);
  cudaFree(PhiGrid); cudaFree(Kc); cudaFree(Xc); cudaFree(Frep);
  return z;
}
