// Test-only harness around the reference's FP32 CUDA kernels
// (code/cuda/SG-tSNE-CUDA/src): AttractiveEstimation in COO format
// (pq.cu:24-57) and computeFrepulsive_interp on the fixed grid
// (Frep.cu:81-125, buffers and cuFFT plans set up as gradient_descend.cu:
// 137-188 does), the whole loop kl_minimization (gradient_descend.cu:
// 102-282; golden trajectories and timing of the reference's GPU path), the
// cost tsneCost (pq.cu:104-125) and perplexityEqualization
// (perplexity_search.cu:113-208).  Compiled in place from the reference tree
// by oracle/build_ref.sh; test and measurement use only.
#include <cmath>
#include <cstring>
#include <vector>
#include "Frep.cuh"
#include "gradient_descend.cuh"
#include "perplexity_search.cuh"
#include "pq.cuh"
#include "types.hpp"

// launch shape of the reference's kernels (declared extern by its sources;
// streamAttr/streamRep are defined by gradient_descend.cu)
int Blocks = 592;
int Threads = 256;

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

// The reference's whole gradient-descent loop on the fixed grid
// (kl_minimization, gradient_descend.cu:102-282) for `iters` iterations, on
// P in format 0 (CSR: rowptr, cols, vals), 2 (COO: rows, cols, vals) or 3
// (ELL of width ell_w, column-major, plus a COO tail).  The launch shape is
// the one the reference's demo picks (demo_perplexity.cu:17-30: occupancy of
// ell_spmv_kernel<float, 2>); the harness's golden-vector shape is restored
// afterwards.  y (host, dim-major n*d) is updated in place.  Returns the
// loop's own wall time in ms (timeInfo[7000], taken after its allocations
// and cuFFT plans), or a negative CUDA error code.
extern "C" double ref_cu_kl_minimization(int format, int n, int d, int nnz, int iters, int ng,
                                         const int *rowptr_or_rows, const int *cols,
                                         const float *vals, int ell_w,
                                         const unsigned *ell_cols, const float *ell_vals,
                                         int coo_n, const unsigned *coo_rows,
                                         const unsigned *coo_cols, const float *coo_vals,
                                         float *y_dim_major) {
  const int saved_blocks = Blocks, saved_threads = Threads;
  cudaOccupancyMaxPotentialBlockSize(&Blocks, &Threads, ell_spmv_kernel<float, 2>, 0, 0);
  sparse_matrix<float> P;
  memset(&P, 0, sizeof(P));
  P.m = n;
  P.n = n;
  P.nnz = nnz;
  P.format = format;
  std::vector<void *> bufs;
  auto dev = [&](const void *src, size_t bytes) {
    void *p = nullptr;
    cudaMallocManaged(&p, bytes);
    cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice);
    bufs.push_back(p);
    return p;
  };
  if (format == 0 || format == 2) {
    P.row = (int *)dev(rowptr_or_rows, sizeof(int) * (format == 0 ? (size_t)n + 1 : (size_t)nnz));
    P.col = (int *)dev(cols, sizeof(int) * (size_t)nnz);
    P.val = (float *)dev(vals, sizeof(float) * (size_t)nnz);
  } else {
    P.elements_in_rows = ell_w;
    P.coo_size = coo_n;
    P.ell_cols = (unsigned *)dev(ell_cols, sizeof(unsigned) * (size_t)n * ell_w);
    P.ell_data = (float *)dev(ell_vals, sizeof(float) * (size_t)n * ell_w);
    P.coo_row_ids = (unsigned *)dev(coo_rows, sizeof(unsigned) * (size_t)(coo_n > 0 ? coo_n : 1));
    P.coo_col_ids = (unsigned *)dev(coo_cols, sizeof(unsigned) * (size_t)(coo_n > 0 ? coo_n : 1));
    P.coo_data = (float *)dev(coo_vals, sizeof(float) * (size_t)(coo_n > 0 ? coo_n : 1));
  }
  float *y = (float *)dev(y_dim_major, sizeof(float) * (size_t)n * d);
  tsneparams params;
  params.d = d;
  params.n = n;
  params.maxIter = iters;
  params.earlyIter = 250;
  params.alpha = 12;
  params.ng = ng;
  params.format = format;
  params.ComputeError = -1;
  std::vector<double> time_info(7 * (size_t)(iters > 1000 ? iters : 1000) + 16, 0.0);
  kl_minimization(y, params, P, time_info.data());
  cudaError_t e = cudaDeviceSynchronize();
  const double ms = time_info[7 * 1000];
  cudaMemcpy(y_dim_major, y, sizeof(float) * (size_t)n * d, cudaMemcpyDeviceToHost);
  for (void *p : bufs) cudaFree(p);
  Blocks = saved_blocks;
  Threads = saved_threads;
  return e == cudaSuccess ? ms : -(double)e;
}

// tsneCost on P in COO form (rows, cols, vals per nonzero) and dim-major y,
// in FP32 (the reference's float instantiation) and FP64 (its double one).
template <typename T>
static T ref_cost(int n, int d, int nnz, const int *rows, const int *cols, const T *vals,
                  const T *y_dim_major, T alpha, T zeta) {
  int *dr, *dc;
  T *dv, *dy;
  cudaMallocManaged(&dr, sizeof(int) * (size_t)nnz);
  cudaMallocManaged(&dc, sizeof(int) * (size_t)nnz);
  cudaMallocManaged(&dv, sizeof(T) * (size_t)nnz);
  cudaMallocManaged(&dy, sizeof(T) * (size_t)n * d);
  cudaMemcpy(dr, rows, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice);
  cudaMemcpy(dc, cols, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice);
  cudaMemcpy(dv, vals, sizeof(T) * (size_t)nnz, cudaMemcpyHostToDevice);
  cudaMemcpy(dy, y_dim_major, sizeof(T) * (size_t)n * d, cudaMemcpyHostToDevice);
  cudaDeviceSynchronize();
  sparse_matrix<T> P;
  memset(&P, 0, sizeof(P));
  P.n = n;
  P.m = n;
  P.nnz = nnz;
  P.format = 2;
  P.row = dr;
  P.col = dc;
  P.val = dv;
  const T c = tsneCost(P, dy, n, d, alpha, zeta);
  cudaDeviceSynchronize();
  cudaFree(dr); cudaFree(dc); cudaFree(dv); cudaFree(dy);
  return c;
}

extern "C" float ref_cu_tsne_cost_f32(int n, int d, int nnz, const int *rows, const int *cols,
                                      const float *vals, const float *y_dim_major, float alpha,
                                      float zeta) {
  return ref_cost<float>(n, d, nnz, rows, cols, vals, y_dim_major, alpha, zeta);
}

extern "C" double ref_cu_tsne_cost_f64(int n, int d, int nnz, const int *rows, const int *cols,
                                       const double *vals, const double *y_dim_major,
                                       double alpha, double zeta) {
  return ref_cost<double>(n, d, nnz, rows, cols, vals, y_dim_major, alpha, zeta);
}

// perplexityEqualization: I and D are n x (nn + 1) (the point itself first,
// at distance 0, as the reference's kNN search returns them); out_row
// (n + 1), out_col and out_val (n * nn) receive the CSR it builds.  Returns
// a CUDA error code.
extern "C" int ref_cu_perplexity(int n, int nn, const int *I, const float *D, float u,
                                 int *out_row, int *out_col, float *out_val) {
  const size_t cnt = (size_t)n * (nn + 1);
  int *dI;
  float *dD;
  cudaMallocManaged(&dI, sizeof(int) * cnt);
  cudaMallocManaged(&dD, sizeof(float) * cnt);
  cudaMemcpy(dI, I, sizeof(int) * cnt, cudaMemcpyHostToDevice);
  cudaMemcpy(dD, D, sizeof(float) * cnt, cudaMemcpyHostToDevice);
  cudaDeviceSynchronize();
  sparse_matrix<float> P = perplexityEqualization(dI, dD, n, nn, u);
  cudaError_t e = cudaDeviceSynchronize();
  cudaMemcpy(out_row, P.row, sizeof(int) * (size_t)(n + 1), cudaMemcpyDeviceToHost);
  cudaMemcpy(out_col, P.col, sizeof(int) * (size_t)n * nn, cudaMemcpyDeviceToHost);
  cudaMemcpy(out_val, P.val, sizeof(float) * (size_t)n * nn, cudaMemcpyDeviceToHost);
  cudaFree(P.row); cudaFree(P.col); cudaFree(P.val);
  cudaFree(dI); cudaFree(dD);
  return (int)e;
}
