// sgt_host.cpp -- host-side sparse-format work of the engine (one-off
// preparation, integer results bit-exact with the reference):
//   sgt_ell_width      CUSP compute_optimal_entries_per_row as called by
//                      CU/matrix_converter.cpp:236-239
//   sgt_csr_to_hybrid  CU/prepareMatrix.cu:55-97, CU/matrix_converter.cpp:106-207
//   sgt_symmetrize     (P + P^T) * scale, columns sorted per row
//                      (CU/graph_rescaling.cu:266-398, scale 1/(2n))
#include "../../include/sgtsne_b200.h"

#include <algorithm>
#include <cstring>
#include <numeric>
#include <utility>
#include <vector>

extern "C" {

int sgt_ell_width(int n, const int *rowptr) {
  // The smallest width w with fewer than n/3 rows longer than w, or fewer
  // than 4096 of them (CUSP defaults relative_speed = 3, breakeven = 4096).
  if (n <= 0 || !rowptr) return 0;
  int maxlen = 0;
  for (int r = 0; r < n; r++) maxlen = std::max(maxlen, rowptr[r + 1] - rowptr[r]);
  std::vector<long> hist((size_t)maxlen + 1, 0);
  for (int r = 0; r < n; r++) hist[rowptr[r + 1] - rowptr[r]]++;
  long longer = n;
  for (int i = 0; i < maxlen; i++) {
    longer -= hist[i];
    if (3.0 * (double)longer < (double)n || longer < 4096) return i;
  }
  return maxlen;
}

sgt_status sgt_csr_to_hybrid(int n, const int *rowptr, const int *col, const float *val,
                             int width, unsigned *ell_cols, float *ell_vals,
                             unsigned *coo_rows, unsigned *coo_cols, float *coo_vals,
                             long *coo_size) {
  if (n < 0 || width < 0 || !rowptr || !col || !val || !coo_size) return SGT_ERR_INVALID_ARG;
  if (width > 0 && (!ell_cols || !ell_vals)) return SGT_ERR_INVALID_ARG;
  const size_t cells = (size_t)n * width;
  if (cells) {
    memset(ell_cols, 0, sizeof(unsigned) * cells);
    memset(ell_vals, 0, sizeof(float) * cells);
  }
  long id = 0;
  for (int r = 0; r < n; r++) {
    const int s = rowptr[r], e = rowptr[r + 1];
    for (int t = s; t < e; t++) {
      const int k = t - s;
      if (k < width) {
        ell_cols[(size_t)k * n + r] = (unsigned)col[t];
        ell_vals[(size_t)k * n + r] = val[t];
      } else {
        coo_rows[id] = (unsigned)r;
        coo_cols[id] = (unsigned)col[t];
        coo_vals[id] = val[t];
        id++;
      }
    }
  }
  *coo_size = id;
  return SGT_OK;
}

sgt_status sgt_symmetrize(int n, const int *rowptr, const int *col, const float *val, float scale,
                          int *out_rowptr, int *out_col, float *out_val, long *out_nnz) {
  if (n < 1 || !rowptr || !col || !val || !out_nnz) return SGT_ERR_INVALID_ARG;
  const long nnz = rowptr[n];
  for (long t = 0; t < nnz; t++)
    if (col[t] < 0 || col[t] >= n) return SGT_ERR_INVALID_ARG;
  // rows of P sorted by column (stable: equal columns keep input order)
  std::vector<int> pc(col, col + nnz);
  std::vector<float> pv(val, val + nnz);
  {
    std::vector<std::pair<int, float>> buf;
    for (int r = 0; r < n; r++) {
      const int s = rowptr[r], e = rowptr[r + 1];
      bool sorted = true;
      for (int t = s + 1; t < e; t++)
        if (pc[t] < pc[t - 1]) { sorted = false; break; }
      if (sorted) continue;
      buf.clear();
      for (int t = s; t < e; t++) buf.emplace_back(pc[t], pv[t]);
      std::stable_sort(buf.begin(), buf.end(),
                       [](const std::pair<int, float> &a, const std::pair<int, float> &b) {
                         return a.first < b.first;
                       });
      for (int t = s; t < e; t++) {
        pc[t] = buf[t - s].first;
        pv[t] = buf[t - s].second;
      }
    }
  }
  // P^T by counting sort (rows visited in order -> columns sorted)
  std::vector<int> trp((size_t)n + 1, 0);
  for (long t = 0; t < nnz; t++) trp[pc[t] + 1]++;
  for (int r = 0; r < n; r++) trp[r + 1] += trp[r];
  std::vector<int> tc(nnz);
  std::vector<float> tv(nnz);
  {
    std::vector<int> fill(trp.begin(), trp.end() - 1);
    for (int r = 0; r < n; r++)
      for (int t = rowptr[r]; t < rowptr[r + 1]; t++) {
        const int c = pc[t];
        tc[fill[c]] = r;
        tv[fill[c]] = pv[t];
        fill[c]++;
      }
  }
  // merge row r of P and of P^T, adding equal columns
  long total = 0;
  const bool write = out_col != nullptr;
  if (write && (!out_rowptr || !out_val)) return SGT_ERR_INVALID_ARG;
  if (write) out_rowptr[0] = 0;
  for (int r = 0; r < n; r++) {
    int a = rowptr[r], ae = rowptr[r + 1], b = trp[r], be = trp[r + 1];
    int last = -1;
    float acc = 0.f;
    auto emit = [&](int c, float v) {
      if (c == last) {
        acc += v;
        return;
      }
      if (last >= 0) {
        if (write) {
          out_col[total] = last;
          out_val[total] = acc * scale;
        }
        total++;
      }
      last = c;
      acc = v;
    };
    while (a < ae || b < be) {
      if (b >= be || (a < ae && pc[a] <= tc[b])) {
        emit(pc[a], pv[a]);
        a++;
      } else {
        emit(tc[b], tv[b]);
        b++;
      }
    }
    if (last >= 0) {
      if (write) {
        out_col[total] = last;
        out_val[total] = acc * scale;
      }
      total++;
    }
    if (write) out_rowptr[r + 1] = (int)total;
  }
  *out_nnz = total;
  return SGT_OK;
}

}  // extern "C"
