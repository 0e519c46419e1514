// sgt_prep.cuh -- building P: lambda rescaling, perplexity equalisation and
// the CSR -> COO row expansion.  One warp per row, FP64 row sums.
//
// Reference semantics:
//   lambda bisection  HYB/graph_rescaling.cpp:19-104 (FP64; dist flag)
//                     CU/graph_rescaling.cu:11-107 (warp per row, FP32)
//   perplexity        HYB/sgtsne.cpp:201-254 (FP64), CU/perplexity_search.cu
//   CSR -> COO        CU/prepareMatrix.cu:2-27 (binary search per nonzero)
#pragma once
#include "sgt_common.cuh"

// values hold distances (dist != 0) or probabilities (dist == 0, turned into
// -log p first).  On exit values hold the row-normalised exp(-sigma v).
__global__ void __launch_bounds__(SGT_THREADS)
k_lambda_bisect(int n, const int *__restrict__ rowptr, float *__restrict__ val,
                double lambda, double tol, int max_iter, int dist,
                float *__restrict__ sigma_out, int *__restrict__ iters_out) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * blockDim.x / 32;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / 32; i < n; i += warps) {
    const int s = rowptr[i], e = rowptr[i + 1];
    double fval = 1.0 - lambda, sig = 1.0, a = -1e3, c = INFINITY;
    if (!dist) {
      for (int t = s + lane; t < e; t += 32) val[t] = (float)(-log((double)val[t]));
      __syncwarp();
    } else {
      double sum = 0.0;
      for (int t = s + lane; t < e; t += 32) sum += exp(-(double)val[t]);
      fval = warp_sum_d(sum) - lambda;
    }
    int iter = 0;
    while (fabs(fval) > tol && iter < max_iter) {
      iter++;
      if (fval > 0) {
        a = sig;
        sig = isinf(c) ? 2.0 * a : 0.5 * (a + c);
      } else {
        c = sig;
        sig = 0.5 * (a + c);
      }
      double sum = 0.0;
      for (int t = s + lane; t < e; t += 32) sum += exp(-(double)val[t] * sig);
      fval = warp_sum_d(sum) - lambda;
    }
    double sum = 0.0;
    for (int t = s + lane; t < e; t += 32) sum += exp(-(double)val[t] * sig);
    sum = warp_sum_d(sum);
    for (int t = s + lane; t < e; t += 32)
      val[t] = (float)(exp(-(double)val[t] * sig) / sum);
    if (lane == 0) {
      if (sigma_out) sigma_out[i] = (float)sig;
      if (iters_out) iters_out[i] = iter;
    }
  }
}

// The steps of the reference's GPU kernel (CU/graph_rescaling.cu:11-94), for
// bit-level parity with it: FP32 sums of expf over the row's entries, lane
// by lane with a stride of 32 and then a shuffle-down tree; the bracket
// starts at [-1e3, 1e7] and its upper end never doubles; and the bisection
// step of the evaluation that meets the tolerance is still applied, so the
// row is normalised with the sigma one step past the one that met it (the
// reference updates sigma before its loop test sees the flag).  Values are
// used as given (the reference's GPU kernel has no -log transform).
__device__ __forceinline__ float warp_sum_down_f(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return __shfl_sync(0xffffffffu, v, 0);
}

__global__ void __launch_bounds__(SGT_THREADS)
k_lambda_bisect_cu(int n, const int *__restrict__ rowptr, float *__restrict__ val,
                   float lambda, float *__restrict__ sigma_out) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * blockDim.x / 32;
  const float tol = 1e-5f;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / 32; i < n; i += warps) {
    const int s = rowptr[i], e = rowptr[i + 1];
    float a = -1e3f, c = 1e7f, sigma = 1.0f;
    bool found = false;
    int iter = 0;
    while (!found && iter < 100) {
      float sum = 0.0f;
      for (int t = s + lane; t < e; t += 32) sum += expf(-val[t] * sigma);
      sum = warp_sum_down_f(sum);
      const float diff = sum - lambda;
      if (diff < tol && diff > -tol) found = true;
      if (diff > 0) {
        a = sigma;
        sigma = c > 1e7f ? 2 * a : (float)(0.5 * (double)(a + c));
      } else {
        c = sigma;
        sigma = (float)(0.5 * (double)(a + c));
      }
      iter++;
    }
    float sum = 0.0f;
    for (int t = s + lane; t < e; t += 32) {
      const float p = expf(-val[t] * sigma);
      val[t] = p;
      sum += p;
    }
    sum = warp_sum_down_f(sum);
    for (int t = s + lane; t < e; t += 32) val[t] = val[t] / sum;
    if (lane == 0 && sigma_out) sigma_out[i] = sigma;
  }
}

// D: n*k squared distances to the k nearest neighbours (self excluded).
// P: n*k output, each row sums to one.
#define SGT_PERP_MAXK 256
__global__ void __launch_bounds__(SGT_THREADS)
k_perplexity(int n, int k, const float *__restrict__ D, double perplexity,
             double tol, int max_iter, float *__restrict__ P,
             float *__restrict__ beta_out) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * blockDim.x / 32;
  constexpr int R = SGT_PERP_MAXK / 32;
  const double logu = log(perplexity);
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / 32; i < n; i += warps) {
    double dv[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int m = lane + 32 * r;
      dv[r] = m < k ? (double)D[(long)i * k + m] : 0.0;
    }
    double beta = 1.0, min_beta = -1.79769313486231570815e+308,
           max_beta = 1.79769313486231570815e+308, sum_P = 0.0, beta_eval = 1.0;
    bool found = false;
    int iter = 0;
    while (!found && iter < max_iter) {
      double s = 0.0, h = 0.0;
      beta_eval = beta;
#pragma unroll
      for (int r = 0; r < R; r++) {
        const int m = lane + 32 * r;
        if (m < k) {
          const double p = exp(-beta * dv[r]);
          s += p;
          h += beta * (dv[r] * p);
        }
      }
      sum_P = warp_sum_d(s) + 2.2250738585072014e-308;
      const double H = warp_sum_d(h) / sum_P + log(sum_P);
      const double Hdiff = H - logu;
      if (Hdiff < tol && -Hdiff < tol) {
        found = true;
      } else if (Hdiff > 0) {
        min_beta = beta;
        beta = (max_beta == 1.79769313486231570815e+308 || max_beta == -1.79769313486231570815e+308)
                   ? beta * 2.0 : (beta + max_beta) / 2.0;
      } else {
        max_beta = beta;
        beta = (min_beta == -1.79769313486231570815e+308 || min_beta == 1.79769313486231570815e+308)
                   ? beta / 2.0 : (beta + min_beta) / 2.0;
      }
      iter++;
    }
    // the reference normalises the row of the last evaluated beta
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int m = lane + 32 * r;
      if (m < k) P[(long)i * k + m] = (float)(exp(-beta_eval * dv[r]) / sum_P);
    }
    if (lane == 0 && beta_out) beta_out[i] = (float)beta_eval;
  }
}

// row index of every nonzero by binary search over rowptr (bit-exact with
// the reference's Csr2CooKernel: the last row r with rowptr[r] <= e)
__global__ void k_csr_to_coo(int n, long nnz, const int *__restrict__ rowptr,
                             unsigned *__restrict__ rows) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < nnz;
       e += (long)gridDim.x * blockDim.x) {
    int start = 0, end = n + 1, i = (n + 1) >> 1;
    while (end - start > 1) {
      const int j = rowptr[i];
      end = (j > e) ? i : end;
      start = (j <= e) ? i : start;
      i = (start + end) >> 1;
    }
    rows[e] = (unsigned)i;
  }
}

// pack CSR (col, val) into the int2 stream the row kernels read
__global__ void k_pack_pairs(long nnz, const int *__restrict__ col,
                             const float *__restrict__ val, int2 *__restrict__ pairs) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < nnz;
       e += (long)gridDim.x * blockDim.x)
    pairs[e] = make_int2(col[e], __float_as_int(val[e]));
}

// flags a CSR whose rowptr decreases or whose columns leave [0, ncols)
__global__ void k_validate_csr(int n, int ncols, const int *__restrict__ rowptr,
                               const int *__restrict__ col, int *__restrict__ bad) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int s = rowptr[i], e = rowptr[i + 1];
    if (e < s || s < 0 || (i == 0 && s != 0)) {
      atomicOr(bad, 1);
      continue;
    }
    for (int t = s; t < e; t++)
      if (col[t] < 0 || col[t] >= ncols) {
        atomicOr(bad, 1);
        break;
      }
  }
}

// rows with a single entry lose it (dropLeafEdge of the lambda rescaling,
// CU/graph_rescaling.cu:91, called with params.dropLeaf at CU/sgtsne.cu:54):
// the value becomes 0
__global__ void k_drop_leaf(int n, const int *__restrict__ rowptr, float *__restrict__ val) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    if (rowptr[r + 1] - rowptr[r] == 1) val[rowptr[r]] = 0.f;
}

