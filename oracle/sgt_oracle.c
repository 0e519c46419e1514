/*
 * sgt_oracle.c -- CPU restatement of the SG-t-SNE gradient-iteration path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine and the timed CPU
 * baseline.  Never linked by the product.  See sgt_oracle.h for the reference
 * function each routine follows.  FFTW (used by the reference CPU path,
 * HYB/non_periodic_conv.cpp) is absent in this image; orc_fft below is a
 * plain mixed-radix Cooley-Tukey FFT written for this oracle and checked
 * against numpy/scipy in tests/test_oracle.py.
 */
#include "sgt_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846

static void set_threads(int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
}

/* ========================================================================
 * Grid size table: the 137 "FFT friendly" sizes of CU/utils.cu:197-207 and
 * HYB/qq.cpp:111-120 (the same list in both).  A table of sizes has to be
 * identical to reproduce the reference's grid decisions bit-exactly.
 * ====================================================================== */
static const int kGridSizes[137] = {
    8,   9,   10,  11,  12,  13,  14,  15,  16,  20,  25,  26,  28,  32,  33,
    35,  36,  39,  40,  42,  44,  45,  48,  49,  50,  52,  54,  55,  56,  60,
    63,  64,  65,  66,  70,  72,  75,  77,  78,  80,  84,  88,  90,  91,  96,
    98,  99,  100, 104, 105, 108, 110, 112, 117, 120, 125, 126, 130, 132, 135,
    140, 144, 147, 150, 154, 156, 160, 165, 168, 175, 176, 180, 182, 189, 192,
    195, 196, 198, 200, 208, 210, 216, 220, 224, 225, 231, 234, 240, 245, 250,
    252, 260, 264, 270, 273, 275, 280, 288, 294, 297, 300, 308, 312, 315, 320,
    325, 330, 336, 343, 350, 351, 352, 360, 364, 375, 378, 385, 390, 392, 396,
    400, 416, 420, 432, 440, 441, 448, 450, 455, 462, 468, 480, 490, 495, 500,
    504, 512};

int orc_best_grid_size(int ng) {
  for (int i = 0; i < 137; i++)
    if (ng + 2 <= kGridSizes[i]) return kGridSizes[i] - 2;
  return kGridSizes[136] - 2;
}

int orc_grid_points_h(double maxy, double h) {
  int ng = (int)ceil(maxy / h);
  if (ng < 14) ng = 14;
  return orc_best_grid_size(ng) + 2;
}

/* ========================================================================
 * Sparse formats
 * ====================================================================== */
void orc_csr_to_coo(int n, int nnz, const int *rowptr, int *rows) {
  /* binary search over rowptr exactly as Csr2CooKernel: the last row r with
     rowptr[r] <= e (empty rows are skipped because their start equals the
     next row's start). */
  for (int e = 0; e < nnz; e++) {
    int start = 0, end = n + 1, i = (n + 1) >> 1;
    while (end - start > 1) {
      int j = rowptr[i];
      end = (j > e) ? i : end;
      start = (j <= e) ? i : start;
      i = (start + end) >> 1;
    }
    rows[e] = i;
  }
}

int orc_ell_width_cusp(int n, const int *rowptr) {
  /* CUSP (github.com/cusplib/cusplibrary, cusp/detail/format_utils.inl)
     compute_optimal_entries_per_row with its defaults relative_speed = 3.0,
     breakeven_threshold = 4096: the smallest width w such that the rows
     longer than w are fewer than n/3 or fewer than 4096.  CUSP is not
     vendored in the reference tree, so this restatement is unpinned. */
  int maxlen = 0;
  for (int r = 0; r < n; r++) {
    int len = rowptr[r + 1] - rowptr[r];
    if (len > maxlen) maxlen = len;
  }
  long *hist = (long *)calloc((size_t)maxlen + 1, sizeof(long));
  for (int r = 0; r < n; r++) hist[rowptr[r + 1] - rowptr[r]]++;
  int width = maxlen;
  long longer = n;
  for (int i = 0; i < maxlen; i++) {
    longer -= hist[i];
    if (3.0 * (double)longer < (double)n || longer < 4096) {
      width = i;
      break;
    }
  }
  free(hist);
  return width;
}

int orc_csr_to_hybrid(int n, const int *rowptr, const int *col,
                      const float *val, int W, unsigned *ell_cols,
                      float *ell_vals, unsigned *coo_rows, unsigned *coo_cols,
                      float *coo_vals) {
  for (long t = 0; t < (long)n * W; t++) {
    ell_cols[t] = 0;
    ell_vals[t] = 0.0f;
  }
  int id = 0;
  for (int r = 0; r < n; r++) {
    int s = rowptr[r], e = rowptr[r + 1];
    for (int t = s; t < e; t++) {
      int k = t - s;
      if (k < W) {
        ell_cols[(long)k * n + r] = (unsigned)col[t];
        ell_vals[(long)k * n + r] = val[t];
      } else {
        coo_rows[id] = (unsigned)r;
        coo_cols[id] = (unsigned)col[t];
        coo_vals[id] = val[t];
        id++;
      }
    }
  }
  return id;
}

int orc_symmetrize(int n, const int *rowptr, const int *col, const double *val,
                   double scale, int *out_rowptr, int *out_col,
                   double *out_val) {
  /* Build the pattern of P + P^T: row r holds col[] of row r and every row c
     that lists r.  Values add where both (r,c) and (c,r) exist.  Columns are
     sorted per row (the cuSPARSE csrgeam convention of CU/graph_rescaling.cu).
     Duplicate (r,c) entries inside one input row are summed. */
  long nnz = rowptr[n];
  int *cnt = (int *)calloc((size_t)n + 1, sizeof(int));
  for (int r = 0; r < n; r++)
    for (int t = rowptr[r]; t < rowptr[r + 1]; t++) {
      cnt[r]++;
      cnt[col[t]]++;
    }
  int *start = (int *)malloc(((size_t)n + 1) * sizeof(int));
  start[0] = 0;
  for (int r = 0; r < n; r++) start[r + 1] = start[r] + cnt[r];
  int *tc = (int *)malloc((size_t)(2 * nnz + 1) * sizeof(int));
  double *tv = (double *)malloc((size_t)(2 * nnz + 1) * sizeof(double));
  int *fill = (int *)calloc((size_t)n, sizeof(int));
  for (int r = 0; r < n; r++)
    for (int t = rowptr[r]; t < rowptr[r + 1]; t++) {
      int c = col[t];
      tc[start[r] + fill[r]] = c;
      tv[start[r] + fill[r]] = val[t];
      fill[r]++;
      tc[start[c] + fill[c]] = r;
      tv[start[c] + fill[c]] = val[t];
      fill[c]++;
    }
  /* sort each row by column (stable pairs via index sort) and merge dups */
  int total = 0;
  if (out_rowptr) out_rowptr[0] = 0;
  long maxrow = 0;
  for (int r = 0; r < n; r++)
    if (cnt[r] > maxrow) maxrow = cnt[r];
  long *key = (long *)malloc(((size_t)maxrow + 1) * sizeof(long));
  for (int r = 0; r < n; r++) {
    int s = start[r], len = cnt[r];
    for (int k = 0; k < len; k++) key[k] = ((long)tc[s + k] << 32) | k;
    {
      /* insertion sort by (column, position): kNN rows are short */
      for (int a = 1; a < len; a++) {
        long v = key[a];
        int b = a - 1;
        while (b >= 0 && key[b] > v) {
          key[b + 1] = key[b];
          b--;
        }
        key[b + 1] = v;
      }
    }
    int k = 0;
    while (k < len) {
      int c = (int)(key[k] >> 32);
      double acc = 0.0;
      while (k < len && (int)(key[k] >> 32) == c) {
        acc += tv[s + (int)(key[k] & 0xffffffffL)];
        k++;
      }
      if (out_col) out_col[total] = c;
      if (out_val) out_val[total] = acc * scale;
      total++;
    }
    if (out_rowptr) out_rowptr[r + 1] = total;
  }
  free(key);
  free(cnt);
  free(start);
  free(tc);
  free(tv);
  free(fill);
  return total;
}

/* ========================================================================
 * Attractive term: F_i = sum_j p_ij (y_i - y_j) / (1 + |y_i - y_j|^2)
 * (HYB/pq.cpp:37-52 accumulates p/(1+dist) * (Y_row - Y_col) into row).
 * ====================================================================== */
void orc_attractive(int n, int d, const int *rowptr, const int *col,
                    const double *val, const double *Y, double *F,
                    int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int i = 0; i < n; i++) {
    double acc[3] = {0, 0, 0};
    const double *yi = Y + (long)i * d;
    for (int t = rowptr[i]; t < rowptr[i + 1]; t++) {
      const double *yj = Y + (long)col[t] * d;
      double dist = 0;
      for (int k = 0; k < d; k++) dist += (yi[k] - yj[k]) * (yi[k] - yj[k]);
      double pq = val[t] / (1 + dist);
      for (int k = 0; k < d; k++) acc[k] += pq * (yi[k] - yj[k]);
    }
    for (int k = 0; k < d; k++) F[(long)i * d + k] = acc[k];
  }
}

/* ========================================================================
 * Exact repulsion (HYB/qq.cpp:25-70)
 * ====================================================================== */
double orc_repulsive_exact(int n, int d, const double *Y, double *F,
                           int nthreads) {
  set_threads(nthreads);
  double *zeta = (double *)calloc((size_t)n, sizeof(double));
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; i++) {
    double f[3] = {0, 0, 0}, z = 0;
    const double *yi = Y + (long)i * d;
    for (int j = 0; j < n; j++) {
      if (i == j) continue;
      const double *yj = Y + (long)j * d;
      double dist = 0;
      for (int k = 0; k < d; k++) dist += (yj[k] - yi[k]) * (yj[k] - yi[k]);
      for (int k = 0; k < d; k++)
        f[k] += (yi[k] - yj[k]) / ((1 + dist) * (1 + dist));
      z += 1.0 / (1.0 + dist);
    }
    for (int k = 0; k < d; k++) F[(long)i * d + k] = f[k];
    zeta[i] = z;
  }
  double Z = 0;
  for (int i = 0; i < n; i++) Z += zeta[i];
  for (long t = 0; t < (long)n * d; t++) F[t] /= Z;
  free(zeta);
  return Z;
}

/* ========================================================================
 * Lagrange cubic weights (HYB/gridding.cpp:29-39, CU/gridding.cuh:13-22).
 * Node f+a carries weight w[a]; the point lies between nodes f+1 and f+2.
 * ====================================================================== */
static inline double lag1(double x) {
  return 0.5 * x * x * x - 1.0 * x * x - 0.5 * x + 1;
}
static inline double lag2(double x) {
  double cc = 1.0 / 6.0;
  return -cc * x * x * x + 1.0 * x * x - 11 * cc * x + 1;
}
static inline void weights(double s, uint32_t *f, double w[4]) {
  uint32_t fi = (uint32_t)floor(s);
  double dd = s - (double)fi;
  w[0] = lag2(1 + dd);
  w[1] = lag1(dd);
  w[2] = lag1(1 - dd);
  w[3] = lag2(2 - dd);
  *f = fi;
}

/* S2G: V[c][z][y][x] += q_c * wx*wy*wz (HYB/gridding.cpp:57-101,164-221,298-368
   with np = 1, i.e. one private grid). */
static void s2g_range(int i0, int i1, int d, int N, const double *ys,
                      const double *q, double *V);

void orc_s2g(int n, int d, int N, const double *ys, const double *q,
             double *V) {
  /* np private grids reduced at the end, as HYB/nuconv.cpp:52-86 */
  int m = d + 1;
  long G = 1;
  for (int k = 0; k < d; k++) G *= N;
  memset(V, 0, sizeof(double) * (size_t)(G * m));
  int np = 1;
#ifdef _OPENMP
  np = omp_get_max_threads();
  if ((long)n < 20000L * np) np = 1;
#endif
  if (np == 1) {
    s2g_range(0, n, d, N, ys, q, V);
    return;
  }
  double *priv = (double *)calloc((size_t)np * G * m, sizeof(double));
#pragma omp parallel num_threads(np)
  {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    int i0 = (int)((long)n * t / np), i1 = (int)((long)n * (t + 1) / np);
    s2g_range(i0, i1, d, N, ys, q, priv + (size_t)t * G * m);
  }
#pragma omp parallel for schedule(static)
  for (long g = 0; g < G * m; g++) {
    double acc = 0;
    for (int t = 0; t < np; t++) acc += priv[(size_t)t * G * m + g];
    V[g] = acc;
  }
  free(priv);
}

static void s2g_range(int i0, int i1, int d, int N, const double *ys,
                      const double *q, double *V) {
  int m = d + 1;
  long G = 1;
  for (int k = 0; k < d; k++) G *= N;
  for (int i = i0; i < i1; i++) {
    uint32_t f[3] = {0, 0, 0};
    double w[3][4] = {{1, 0, 0, 0}, {1, 0, 0, 0}, {1, 0, 0, 0}};
    for (int k = 0; k < d; k++) weights(ys[(long)i * d + k], &f[k], w[k]);
    int a3 = d > 2 ? 4 : 1, a2 = d > 1 ? 4 : 1;
    for (int c = 0; c < m; c++) {
      double qv = q[(long)i * m + c];
      for (int i3 = 0; i3 < a3; i3++)
        for (int i2 = 0; i2 < a2; i2++)
          for (int i1 = 0; i1 < 4; i1++) {
            double wt = w[0][i1] * (d > 1 ? w[1][i2] : 1.0) *
                        (d > 2 ? w[2][i3] : 1.0);
            long node = (long)(f[0] + i1);
            if (d > 1) node += (long)(f[1] + i2) * N;
            if (d > 2) node += (long)(f[2] + i3) * N * N;
            V[c * G + node] += qv * wt;
          }
    }
  }
}

/* G2S: Phi_c(i) = sum_nodes w * PhiGrid[c][node] (HYB/gridding.cpp:455-624) */
void orc_g2s(int n, int d, int N, const double *ys, const double *PhiGrid,
             double *PhiScat) {
  int m = d + 1;
  long G = 1;
  for (int k = 0; k < d; k++) G *= N;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    uint32_t f[3] = {0, 0, 0};
    double w[3][4] = {{1, 0, 0, 0}, {1, 0, 0, 0}, {1, 0, 0, 0}};
    for (int k = 0; k < d; k++) weights(ys[(long)i * d + k], &f[k], w[k]);
    int a3 = d > 2 ? 4 : 1, a2 = d > 1 ? 4 : 1;
    for (int c = 0; c < m; c++) {
      double acc = 0;
      for (int i3 = 0; i3 < a3; i3++)
        for (int i2 = 0; i2 < a2; i2++)
          for (int i1 = 0; i1 < 4; i1++) {
            double wt = w[0][i1] * (d > 1 ? w[1][i2] : 1.0) *
                        (d > 2 ? w[2][i3] : 1.0);
            long node = (long)(f[0] + i1);
            if (d > 1) node += (long)(f[1] + i2) * N;
            if (d > 2) node += (long)(f[2] + i3) * N * N;
            acc += PhiGrid[c * G + node] * wt;
          }
      PhiScat[(long)i * m + c] = acc;
    }
  }
}

/* ========================================================================
 * FFT: recursive mixed-radix decimation in time.  For L = p*m,
 * X[u + m r] = sum_q (W_L^{qu} Y_q[u]) W_p^{qr}, Y_q = FFT_m(x[q + p j]).
 * ====================================================================== */
typedef struct {
  int L;
  double *twr, *twi; /* W_L^j = exp(sign*2*pi*i*j/L), j < L */
  int sign;
} fft_tab;

static int smallest_factor(int L) {
  if (L % 4 == 0) return 4;
  if (L % 2 == 0) return 2;
  for (int p = 3; p * p <= L; p += 2)
    if (L % p == 0) return p;
  return L;
}

static void fft_rec(const fft_tab *T, int L, const double *xr, const double *xi,
                    long stride, double *outr, double *outi) {
  if (L == 1) {
    outr[0] = xr[0];
    outi[0] = xi[0];
    return;
  }
  int p = smallest_factor(L);
  int m = L / p;
  for (int q = 0; q < p; q++)
    fft_rec(T, m, xr + q * stride, xi + q * stride, stride * p, outr + q * m,
            outi + q * m);
  int step = T->L / L;    /* W_L^k = W_T^{k*step} */
  int pstep = T->L / p;   /* W_p^k = W_T^{k*pstep} */
  double tr[64], ti[64];
  for (int u = 0; u < m; u++) {
    for (int q = 0; q < p; q++) {
      long e = ((long)q * u * step) % T->L;
      double ar = outr[q * m + u], ai = outi[q * m + u];
      tr[q] = ar * T->twr[e] - ai * T->twi[e];
      ti[q] = ar * T->twi[e] + ai * T->twr[e];
    }
    for (int r = 0; r < p; r++) {
      double sr = 0, si = 0;
      for (int q = 0; q < p; q++) {
        long e = ((long)q * r * pstep) % T->L;
        sr += tr[q] * T->twr[e] - ti[q] * T->twi[e];
        si += tr[q] * T->twi[e] + ti[q] * T->twr[e];
      }
      outr[u + m * r] = sr;
      outi[u + m * r] = si;
    }
  }
}

static void fft_tab_init(fft_tab *T, int L, int sign) {
  T->L = L;
  T->sign = sign;
  T->twr = (double *)malloc(sizeof(double) * (size_t)L);
  T->twi = (double *)malloc(sizeof(double) * (size_t)L);
  for (int j = 0; j < L; j++) {
    double a = sign * 2.0 * ORC_PI * (double)j / (double)L;
    T->twr[j] = cos(a);
    T->twi[j] = sin(a);
  }
}
static void fft_tab_free(fft_tab *T) {
  free(T->twr);
  free(T->twi);
}

/* in-place 1D FFT of a line (sign -1 forward, +1 inverse, no scaling) */
static void fft_line(const fft_tab *T, double *re, double *im, double *wr,
                     double *wi) {
  fft_rec(T, T->L, re, im, 1, wr, wi);
  memcpy(re, wr, sizeof(double) * (size_t)T->L);
  memcpy(im, wi, sizeof(double) * (size_t)T->L);
}

void orc_fft(int L, double *re, double *im, int sign) {
  fft_tab T;
  fft_tab_init(&T, L, sign);
  double *wr = (double *)malloc(sizeof(double) * (size_t)L);
  double *wi = (double *)malloc(sizeof(double) * (size_t)L);
  fft_line(&T, re, im, wr, wi);
  free(wr);
  free(wi);
  fft_tab_free(&T);
}

/* d-dimensional in-place FFT of an N^d complex array (x fastest). */
static void fftnd(int d, int N, double *re, double *im, int sign) {
  fft_tab T;
  fft_tab_init(&T, N, sign);
  long G = 1;
  for (int k = 0; k < d; k++) G *= N;
  for (int ax = 0; ax < d; ax++) {
    long st = 1;
    for (int k = 0; k < ax; k++) st *= N;
    long nlines = G / N;
#pragma omp parallel
    {
      double *lr = (double *)malloc(sizeof(double) * 4 * (size_t)N);
      double *li = lr + N, *wr = lr + 2 * N, *wi = lr + 3 * N;
#pragma omp for schedule(static)
      for (long ln = 0; ln < nlines; ln++) {
        long lo = ln % st, hi = ln / st;
        long base = hi * st * N + lo;
        for (int t = 0; t < N; t++) {
          lr[t] = re[base + t * st];
          li[t] = im[base + t * st];
        }
        fft_line(&T, lr, li, wr, wi);
        for (int t = 0; t < N; t++) {
          re[base + t * st] = lr[t];
          im[base + t * st] = li[t];
        }
      }
      free(lr);
    }
  }
  fft_tab_free(&T);
}

/* ========================================================================
 * G2G: aperiodic convolution with K(r) = (1 + h^2 |r|^2)^-2 over the grid.
 * conv_mode 0 restates HYB/non_periodic_conv.cpp + convolution_nopadding_helper
 * (and CU/non_periodic_convF.cu): for each of the 2^d even/odd combinations
 * s, the kernel is folded K_s[i] = sum over axes of K(i) or s*K(N-i), both the
 * kernel and the data carry the half-shift twiddle exp(-i pi i/N) on odd
 * axes, a size-N cyclic convolution is taken by FFT, the twiddle is undone
 * and 2^-d/N^d * Re(.) is accumulated.  conv_mode 1 is the direct sum.
 * ====================================================================== */
static inline double kern(double hsq, double r2) {
  return pow(1.0 + hsq * r2, -2);
}

void orc_g2g(int d, int N, int m, double h_eff, const double *V, double *Phi,
             int conv_mode, int nthreads) {
  set_threads(nthreads);
  long G = 1;
  for (int k = 0; k < d; k++) G *= N;
  double hsq = h_eff * h_eff;
  memset(Phi, 0, sizeof(double) * (size_t)(G * m));
  if (conv_mode == 1) {
#pragma omp parallel for schedule(dynamic, 16)
    for (long a = 0; a < G; a++) {
      long ax = a % N, ay = d > 1 ? (a / N) % N : 0, az = d > 2 ? a / (N * N) : 0;
      for (long b = 0; b < G; b++) {
        long bx = b % N, by = d > 1 ? (b / N) % N : 0, bz = d > 2 ? b / (N * N) : 0;
        double r2 = (double)((ax - bx) * (ax - bx) + (ay - by) * (ay - by) +
                             (az - bz) * (az - bz));
        double k = kern(hsq, r2);
        for (int c = 0; c < m; c++) Phi[c * G + a] += k * V[c * G + b];
      }
    }
    return;
  }
  double *Kr = (double *)malloc(sizeof(double) * (size_t)G);
  double *Ki = (double *)malloc(sizeof(double) * (size_t)G);
  double *Xr = (double *)malloc(sizeof(double) * (size_t)(G * m));
  double *Xi = (double *)malloc(sizeof(double) * (size_t)(G * m));
  double scale = pow(0.5, d) / (double)G;
  int nterms = 1 << d;
  for (int term = 0; term < nterms; term++) {
    int sg[3] = {1, 1, 1};
    for (int k = 0; k < d; k++) sg[k] = (term >> k) & 1 ? -1 : 1;
    /* folded kernel and twiddled data */
#pragma omp parallel for schedule(static)
    for (long a = 0; a < G; a++) {
      long idx[3] = {a % N, d > 1 ? (a / N) % N : 0, d > 2 ? a / ((long)N * N) : 0};
      double kv = 0;
      /* sum over the 2^d corner images: each axis picks i or N-i (i>0) */
      for (int img = 0; img < nterms; img++) {
        double sgn = 1.0, r2 = 0.0;
        int ok = 1;
        for (int k = 0; k < d; k++) {
          long i = idx[k];
          if ((img >> k) & 1) {
            if (i == 0) { ok = 0; break; }
            i = N - i;
            sgn *= sg[k];
          }
          r2 += (double)(i * i);
        }
        if (ok) kv += sgn * kern(hsq, r2);
      }
      double ph = 0;
      for (int k = 0; k < d; k++)
        if (sg[k] < 0) ph += -2.0 * ORC_PI * (double)idx[k] / (2.0 * N);
      double cr = cos(ph), ci = sin(ph);
      Kr[a] = kv * cr;
      Ki[a] = kv * ci;
      for (int c = 0; c < m; c++) {
        Xr[c * G + a] = V[c * G + a] * cr;
        Xi[c * G + a] = V[c * G + a] * ci;
      }
    }
    fftnd(d, N, Kr, Ki, -1);
    for (int c = 0; c < m; c++) {
      fftnd(d, N, Xr + c * G, Xi + c * G, -1);
      for (long a = 0; a < G; a++) {
        double ar = Xr[c * G + a], ai = Xi[c * G + a];
        Xr[c * G + a] = ar * Kr[a] - ai * Ki[a];
        Xi[c * G + a] = ar * Ki[a] + ai * Kr[a];
      }
      fftnd(d, N, Xr + c * G, Xi + c * G, +1);
    }
#pragma omp parallel for schedule(static)
    for (long a = 0; a < G; a++) {
      long idx[3] = {a % N, d > 1 ? (a / N) % N : 0, d > 2 ? a / ((long)N * N) : 0};
      double ph = 0;
      for (int k = 0; k < d; k++)
        if (sg[k] < 0) ph += 2.0 * ORC_PI * (double)idx[k] / (2.0 * N);
      double cr = cos(ph), ci = sin(ph);
      for (int c = 0; c < m; c++) {
        double re = Xr[c * G + a] * cr - Xi[c * G + a] * ci;
        Phi[c * G + a] += scale * re;
      }
    }
  }
  free(Kr);
  free(Ki);
  free(Xr);
  free(Xi);
}

/* ========================================================================
 * Interpolated repulsion (HYB/qq.cpp:132-244 + HYB/nuconv.cpp:22-153)
 * ====================================================================== */
double orc_repulsive_interp(int n, int d, double h, int n1_force,
                            const double *Y, double *F, int *grid_points,
                            double *h_eff, int conv_mode, int nthreads) {
  set_threads(nthreads);
  int m = d + 1;
  double *y = (double *)malloc(sizeof(double) * (size_t)n * d);
  double miny[3] = {INFINITY, INFINITY, INFINITY};
  for (int i = 0; i < n; i++)
    for (int k = 0; k < d; k++)
      if (miny[k] > Y[(long)i * d + k]) miny[k] = Y[(long)i * d + k];
  for (long t = 0; t < (long)n * d; t++) y[t] = Y[t] - miny[t % d];
  double maxy = 0;
  for (long t = 0; t < (long)n * d; t++)
    if (maxy < y[t]) maxy = y[t];
  int n1;
  if (n1_force > 0)
    n1 = n1_force;
  else {
    int ng = (int)ceil(maxy / h);
    if (ng < 14) ng = 14;
    n1 = orc_best_grid_size(ng);
  }
  int N = n1 + 2;
  /* charges [1, y] use the shifted coordinates (qq.cpp:196-202) */
  double *q = (double *)malloc(sizeof(double) * (size_t)n * m);
  for (int i = 0; i < n; i++) {
    q[(long)i * m] = 1.0;
    for (int k = 0; k < d; k++) q[(long)i * m + k + 1] = y[(long)i * d + k];
  }
  /* scale into [0, n1-1) (nuconv.cpp:30-41) */
  double *ys = (double *)malloc(sizeof(double) * (size_t)n * d);
  for (long t = 0; t < (long)n * d; t++) {
    double v = y[t] / maxy;
    if (v == 1) v = v - DBL_EPSILON;
    ys[t] = v * (double)(n1 - 1);
  }
  double he = maxy / ((double)(n1 - 1) - DBL_EPSILON);
  long G = 1;
  for (int k = 0; k < d; k++) G *= N;
  double *V = (double *)malloc(sizeof(double) * (size_t)(G * m));
  double *Pg = (double *)malloc(sizeof(double) * (size_t)(G * m));
  double *Phi = (double *)malloc(sizeof(double) * (size_t)n * m);
  orc_s2g(n, d, N, ys, q, V);
  orc_g2g(d, N, m, he, V, Pg, conv_mode, nthreads);
  orc_g2s(n, d, N, ys, Pg, Phi);
  /* zetaAndForce (qq.cpp:75-106) */
  double Z = 0;
  for (int i = 0; i < n; i++) {
    double ysq = 0;
    for (int k = 0; k < d; k++) {
      double yk = y[(long)i * d + k];
      ysq += yk * yk;
      Z -= 2 * (yk * Phi[(long)i * m + k + 1]);
    }
    Z += (1 + 2 * ysq) * Phi[(long)i * m];
  }
  Z = Z - n;
  for (int i = 0; i < n; i++)
    for (int k = 0; k < d; k++)
      F[(long)i * d + k] =
          (y[(long)i * d + k] * Phi[(long)i * m] - Phi[(long)i * m + k + 1]) / Z;
  if (grid_points) *grid_points = N;
  if (h_eff) *h_eff = he;
  free(y);
  free(q);
  free(ys);
  free(V);
  free(Pg);
  free(Phi);
  return Z;
}

/* ========================================================================
 * FP32 binning of the CUDA path.  Every step is one IEEE float operation in
 * the order the reference performs it; compile without FP contraction.
 * ====================================================================== */
int orc_bins_f32(int n, int d, float h, int n1_force, const float *Y,
                 uint32_t *bins, float *scaled, float *shifted,
                 float *maxy_out) {
  float miny[3] = {100.0f, 100.0f, 100.0f}; /* thrust::reduce init 100.0 */
  for (int i = 0; i < n; i++)
    for (int k = 0; k < d; k++) {
      float v = Y[(long)i * d + k];
      miny[k] = v < miny[k] ? v : miny[k];
    }
  float maxy = 0.0f; /* thrust::reduce init 0.0 */
  for (int i = 0; i < n; i++)
    for (int k = 0; k < d; k++) {
      volatile float s = Y[(long)i * d + k] - miny[k];
      maxy = maxy < s ? s : maxy;
    }
  int n1;
  if (n1_force > 0)
    n1 = n1_force;
  else {
    volatile float ratio = maxy / h;
    int ng = (int)ceilf(ratio);
    if (ng < 14) ng = 14;
    n1 = orc_best_grid_size(ng);
  }
  int N = n1 + 2;
  float fac = (float)(uint32_t)(N - 3);
  for (int i = 0; i < n; i++)
    for (int k = 0; k < d; k++) {
      volatile float s = Y[(long)i * d + k] - miny[k];
      if (shifted) shifted[(long)i * d + k] = s;
      volatile float v = s / maxy;
      if (v >= 1.0f) v = 1.0f - FLT_EPSILON;
      volatile float t = v * fac;
      if (scaled) scaled[(long)i * d + k] = t;
      bins[(long)i * d + k] = (uint32_t)floorf(t);
    }
  if (maxy_out) *maxy_out = maxy;
  return N;
}

/* ========================================================================
 * Update (HYB/gradient_descendHYB.cpp:46-78)
 * ====================================================================== */
static inline double sgn(double x) { return x == .0 ? .0 : (x < .0 ? -1.0 : 1.0); }

void orc_update(int n, int d, const double *dY, double *uY, double *Y,
                double *gains, double momentum, double eta, int center) {
  long nd = (long)n * d;
  for (long i = 0; i < nd; i++) {
    gains[i] = (sgn(dY[i]) != sgn(uY[i])) ? (gains[i] + .2) : (gains[i] * .8);
    if (gains[i] < .01) gains[i] = .01;
    uY[i] = momentum * uY[i] - eta * gains[i] * dY[i];
    Y[i] = Y[i] + uY[i];
  }
  if (!center) return;
  for (int k = 0; k < d; k++) {
    double s = 0;
    for (int i = 0; i < n; i++) s += Y[(long)i * d + k];
    s /= n;
    for (int i = 0; i < n; i++) Y[(long)i * d + k] -= s;
  }
}

void orc_kl_minimization(int n, int d, const int *rowptr, const int *col,
                         const double *val, double *Y, int max_iter,
                         int early_iter, double alpha, double h, int grid_mode,
                         int ng, double *zeta_out, int nthreads) {
  long nd = (long)n * d;
  double *dy = (double *)malloc(sizeof(double) * (size_t)nd);
  double *uy = (double *)calloc((size_t)nd, sizeof(double));
  double *gains = (double *)malloc(sizeof(double) * (size_t)nd);
  double *Fa = (double *)malloc(sizeof(double) * (size_t)nd);
  double *Fr = (double *)malloc(sizeof(double) * (size_t)nd);
  for (long i = 0; i < nd; i++) gains[i] = 1.0;
  double momentum = .5, final_momentum = .8, eta = 200.0;
  int mom_switch_iter = 250;
  int n1_fixed = grid_mode == 1 ? orc_best_grid_size(ng) : 0;
  for (int iter = 0; iter < max_iter; iter++) {
    double Z = orc_repulsive_interp(n, d, h, n1_fixed, Y, Fr, NULL, NULL, 0,
                                    nthreads);
    if (zeta_out) zeta_out[iter] = Z;
    orc_attractive(n, d, rowptr, col, val, Y, Fa, nthreads);
    for (long i = 0; i < nd; i++) dy[i] = alpha * Fa[i] - Fr[i];
    orc_update(n, d, dy, uy, Y, gains, momentum, eta, grid_mode == 0);
    if (iter == early_iter) alpha = 1;
    if (iter == mom_switch_iter) momentum = final_momentum;
  }
  if (grid_mode == 1) {
    for (int k = 0; k < d; k++) {
      double s = 0;
      for (int i = 0; i < n; i++) s += Y[(long)i * d + k];
      s /= n;
      for (int i = 0; i < n; i++) Y[(long)i * d + k] -= s;
    }
  }
  free(dy);
  free(uy);
  free(gains);
  free(Fa);
  free(Fr);
}

/* ========================================================================
 * KL cost
 * ====================================================================== */
double orc_kl(int n, int d, const int *rowptr, const int *col,
              const double *val, const double *Y, double alpha, double zeta) {
  double total = 0;
  for (int i = 0; i < n; i++) {
    for (int t = rowptr[i]; t < rowptr[i + 1]; t++) {
      int j = col[t];
      double dist = 0;
      for (int k = 0; k < d; k++) {
        double df = Y[(long)i * d + k] - Y[(long)j * d + k];
        dist += df * df;
      }
      double p = alpha * val[t];
      double q = (1.0 / (1.0 + dist)) / zeta;
      total += p * log((p + FLT_MIN) / (q + FLT_MIN));
    }
  }
  return total;
}

/* ========================================================================
 * lambda rescaling
 * ====================================================================== */
void orc_lambda_rescale_f32(int n, const int *rowptr, float *val, float lambda,
                            float *sigma_out) {
  const float tol = 1e-5f;
  for (int r = 0; r < n; r++) {
    float a = -1e3f, c = 1e7f, sigma = 1.0f;
    int found = 0, iter = 0;
    int s = rowptr[r], e = rowptr[r + 1];
    while (!found && iter < 100) {
      float sum = 0.0f;
      for (int t = s; t < e; t++) sum += expf(-val[t] * sigma);
      float diff = sum - lambda;
      if (diff < tol && diff > -tol) found = 1;
      if (diff > 0) {
        a = sigma;
        if (c > 1e7f)
          sigma = 2 * a;
        else
          sigma = 0.5f * (a + c);
      } else {
        c = sigma;
        sigma = 0.5f * (a + c);
      }
      iter++;
    }
    if (sigma_out) sigma_out[r] = sigma;
    float sum = 0.0f;
    for (int t = s; t < e; t++) {
      val[t] = expf(-val[t] * sigma);
      sum += val[t];
    }
    for (int t = s; t < e; t++) val[t] /= sum;
  }
}

void orc_lambda_rescale(int n, const int *rowptr, double *val, double lambda,
                        int dist, double *sigma_out) {
  const double tol = 1e-5;
  const int max_iter = 100;
#pragma omp parallel for schedule(dynamic, 1024)
  for (int i = 0; i < n; i++) {
    double fval = 1 - lambda, sig = 1, a = -1e3, c = INFINITY, sum = 0;
    int iter = 0;
    if (!dist) {
      for (int t = rowptr[i]; t < rowptr[i + 1]; t++) val[t] = -log(val[t]);
    } else {
      for (int t = rowptr[i]; t < rowptr[i + 1]; t++) sum += exp(-val[t]);
      fval = sum - lambda;
    }
    while (fabs(fval) > tol && iter < max_iter) {
      iter++;
      sum = 0;
      if (fval > 0) {
        a = sig;
        sig = isinf(c) ? 2 * a : 0.5 * (a + c);
      } else {
        c = sig;
        sig = 0.5 * (a + c);
      }
      for (int t = rowptr[i]; t < rowptr[i + 1]; t++) sum += exp(-val[t] * sig);
      fval = sum - lambda;
    }
    sum = 0;
    for (int t = rowptr[i]; t < rowptr[i + 1]; t++) {
      val[t] = exp(-val[t] * sig);
      sum += val[t];
    }
    for (int t = rowptr[i]; t < rowptr[i + 1]; t++) val[t] /= sum;
    if (sigma_out) sigma_out[i] = sig;
  }
}

void orc_perplexity(int n, int k, const double *D, double perplexity,
                    double *P, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; i++) {
    const double *dist = D + (long)i * (k + 1);
    double *p = P + (long)i * k;
    int found = 0, iter = 0;
    double beta = 1.0, min_beta = -DBL_MAX, max_beta = DBL_MAX, tol = 1e-5,
           sum_P = 0;
    while (!found && iter < 200) {
      for (int m = 0; m < k; m++) p[m] = exp(-beta * dist[m + 1]);
      sum_P = DBL_MIN;
      for (int m = 0; m < k; m++) sum_P += p[m];
      double H = 0;
      for (int m = 0; m < k; m++) H += beta * (dist[m + 1] * p[m]);
      H = (H / sum_P) + log(sum_P);
      double Hdiff = H - log(perplexity);
      if (Hdiff < tol && -Hdiff < tol) {
        found = 1;
      } else if (Hdiff > 0) {
        min_beta = beta;
        if (max_beta == DBL_MAX || max_beta == -DBL_MAX)
          beta *= 2.0;
        else
          beta = (beta + max_beta) / 2.0;
      } else {
        max_beta = beta;
        if (min_beta == -DBL_MAX || min_beta == DBL_MAX)
          beta /= 2.0;
        else
          beta = (beta + min_beta) / 2.0;
      }
      iter++;
    }
    for (int m = 0; m < k; m++) p[m] /= sum_P;
  }
}
