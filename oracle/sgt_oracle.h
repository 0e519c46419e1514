/*
 * sgt_oracle.h -- CPU restatement of the SG-t-SNE gradient-iteration path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA engine
 * under gpu-sg-sne_b200/.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  The product
 * never links it and has no CPU fallback.
 *
 * Every function restates the reference algorithm it cites (paths are relative
 * to the iakoviid/GPU-SG-SNE tree; CU = code/cuda/SG-tSNE-CUDA/src,
 * HYB = code/cuda/SG-tSNE-HYB/sgtsnepi/src).  FP64 functions follow the CPU
 * SG-t-SNE-Pi path (HYB *.cpp); *_f32 functions follow the FP32 CUDA path (CU)
 * operation by operation so that integer results (grid sizes, bin indices)
 * can be compared bit-exactly with the engine.
 *
 * Coordinates are point-major (Y[i*d + k]) unless a function says otherwise.
 */
#ifndef SGT_ORACLE_H
#define SGT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- grid size (CU/utils.cu:194-215, HYB/qq.cpp:108-129) ---------------- */
int orc_best_grid_size(int ng);
/* grid points per axis for h-driven grids:
   max(ceil(maxy/h),14) -> best size, +2 (HYB/qq.cpp:161-166) */
int orc_grid_points_h(double maxy, double h);

/* ---- sparse formats (integer, bit-exact) ------------------------------- */
/* CSR -> COO row ids by binary search (CU/prepareMatrix.cu:2-27) */
void orc_csr_to_coo(int n, int nnz, const int *rowptr, int *rows);
/* ELL width heuristic of CUSP compute_optimal_entries_per_row
   (called from CU/matrix_converter.cpp:236-239) */
int orc_ell_width_cusp(int n, const int *rowptr);
/* CSR -> ELL (column-major n*W, zero padded) + COO tail in row order
   (CU/matrix_converter.cpp:106-132,170-207).  Returns the COO size. */
int orc_csr_to_hybrid(int n, const int *rowptr, const int *col,
                      const float *val, int W, unsigned *ell_cols,
                      float *ell_vals, unsigned *coo_rows, unsigned *coo_cols,
                      float *coo_vals);
/* (P + P^T) * scale with columns sorted inside each row
   (CU/graph_rescaling.cu:266-398 with scale 1/(2n); HYB/sparsematrix.cpp:69-163).
   Pass out arrays NULL to get the nnz only. */
int orc_symmetrize(int n, const int *rowptr, const int *col, const double *val,
                   double scale, int *out_rowptr, int *out_col,
                   double *out_val);

/* ---- attractive term (HYB/pq.cpp:15-58; CU/pq.cuh:77-118) -------------- */
void orc_attractive(int n, int d, const int *rowptr, const int *col,
                    const double *val, const double *Y, double *F,
                    int nthreads);

/* ---- repulsive term ---------------------------------------------------- */
/* exact O(n^2) (HYB/qq.cpp:25-70); returns Z */
double orc_repulsive_exact(int n, int d, const double *Y, double *F,
                           int nthreads);
/* FFT-interpolated (HYB/qq.cpp:132-244, HYB/nuconv.cpp:22-153,
   HYB/gridding.cpp, HYB/non_periodic_conv.cpp).
   n1_force > 0 forces the inner grid size (grid points = n1_force+2, as the
   fixed-grid path CU/gradient_descend.cu:139-140 does); otherwise the grid
   follows h.  conv_mode 0 = even/odd FFT terms (reference structure),
   1 = direct aperiodic sum (cross-check).  Outputs: F (n*d), returns Z;
   grid_points / h_eff may be NULL. */
double orc_repulsive_interp(int n, int d, double h, int n1_force,
                            const double *Y, double *F, int *grid_points,
                            double *h_eff, int conv_mode, int nthreads);

/* The same pipeline stage by stage (for stage tests):
   scale points, S2G (channel-major grid V[c][..][x]), G2G, G2S. */
void orc_s2g(int n, int d, int N, const double *ys /*scaled, n*d*/,
             const double *q /*n*(d+1) charges*/, double *V);
void orc_g2g(int d, int N, int m, double h_eff, const double *V, double *Phi,
             int conv_mode, int nthreads);
void orc_g2s(int n, int d, int N, const double *ys, const double *PhiGrid,
             double *PhiScat /*n*(d+1)*/);

/* FP32 CUDA-path binning: per-dim min (thrust init 100.0, CU/Frep.cu:96-102),
   max, grid size, scaled coords (CU/nuconv.cu:9-36) and floor bins
   (CU/gridding.cu:159-167).  Y is point-major float.  n1_force as above,
   h in float.  Outputs: bins (n*d uint32), scaled (n*d float, may be NULL),
   shifted (n*d float, may be NULL); returns grid points per axis. */
int orc_bins_f32(int n, int d, float h, int n1_force, const float *Y,
                 uint32_t *bins, float *scaled, float *shifted,
                 float *maxy_out);

/* ---- plain FFT used by the oracle (exposed for its own test) ----------- */
void orc_fft(int L, double *re, double *im, int sign);

/* ---- update (HYB/gradient_descendHYB.cpp:29-78; CU/gradient_descend.cu:12-51) */
void orc_update(int n, int d, const double *dY, double *uY, double *Y,
                double *gains, double momentum, double eta, int center);

/* ---- full gradient descent (HYB/gradient_descendHYB.cpp:160-283;
        CU/gradient_descend_varGrid.cu:305-396; CU/gradient_descend.cu:102-282)
   grid_mode 0 = h-driven with per-iteration mean centring (varGrid/HYB),
   grid_mode 1 = fixed inner grid getBestGridSize(ng), centring at the end.
   Y (point-major) is updated in place.  zeta_out (max_iter) may be NULL. */
void orc_kl_minimization(int n, int d, const int *rowptr, const int *col,
                         const double *val, double *Y, int max_iter,
                         int early_iter, double alpha, double h, int grid_mode,
                         int ng, double *zeta_out, int nthreads);

/* ---- KL cost (CU/pq.cu:61-125; HYB csb bicsb.cpp:1821-1870) ------------ */
double orc_kl(int n, int d, const int *rowptr, const int *col,
              const double *val, const double *Y, double alpha, double zeta);

/* ---- P construction ---------------------------------------------------- */
/* lambda bisection, CUDA variant: values are used as distances as given,
   FP32 expf, 100 iterations, tol 1e-5 (CU/graph_rescaling.cu:11-107). */
void orc_lambda_rescale_f32(int n, const int *rowptr, float *val, float lambda,
                            float *sigma_out);
/* lambda bisection, CPU variant (HYB/graph_rescaling.cpp:19-104), FP64;
   dist != 0: values are distances; dist == 0: values are -log(p). */
void orc_lambda_rescale(int n, const int *rowptr, double *val, double lambda,
                        int dist, double *sigma_out);
/* perplexity bisection per row (HYB/sgtsne.cpp:201-254), FP64.  D is
   n*(k+1) squared distances with self first, P is n*k output. */
void orc_perplexity(int n, int k, const double *D, double perplexity,
                    double *P, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
