// sgt_sym.cu -- (P + P^T) * scale on the device, bit-identical to the host
// sgt_symmetrize (CU/graph_rescaling.cu:266-398 builds the same pattern with
// legacy cuSPARSE csrgeam; scale 1/(2n) at CU/graph_rescaling.cu:378-379).
//
// The host version sorts each row of P stably by column, builds P^T by a
// counting sort that visits rows in order, and merges row r of P with row r
// of P^T, taking P's entries first on equal columns and summing equal
// columns in that order.  Here every nonzero t of P (rows in order) emits two
// entries: (r, c, from P) into the first half of a buffer and (c, r, from
// P^T) into the second half, both halves in t order.  A stable LSD radix
// sort on the key (row, column, source) then yields, per output row, the
// host's merge sequence exactly: columns ascending, P before P^T, input
// order within each.  Runs of equal (row, column) are summed one after
// another in FP32 and scaled, as the host does.  The sort is CUB's device
// radix sort (this is preprocessing, not the iteration).
#include "../../include/sgtsne_b200.h"
#include "sgt_internal.h"

#include <algorithm>
#include <string>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

namespace {

constexpr int SYM_THREADS = 256;
constexpr int SYM_ROW_BITS = 24;  // n <= 2^24 rows

__device__ __forceinline__ unsigned long long sym_key(unsigned row, unsigned col, unsigned src) {
  return ((unsigned long long)row << (SYM_ROW_BITS + 1)) | ((unsigned long long)col << 1) | src;
}

// one thread per nonzero: its row by binary search over rowptr
__global__ void k_sym_emit(int n, long nnz, const int *__restrict__ rowptr,
                           const int *__restrict__ col, const float *__restrict__ val,
                           unsigned long long *__restrict__ keys, float *__restrict__ vals,
                           int *__restrict__ bad) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nnz;
       t += (long)gridDim.x * blockDim.x) {
    int lo = 0, hi = n;  // largest r with rowptr[r] <= t
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (rowptr[mid] <= t) lo = mid; else hi = mid;
    }
    const int c = col[t];
    if (c < 0 || c >= n) {
      atomicOr(bad, 1);
      keys[t] = keys[nnz + t] = 0ull;
      vals[t] = vals[nnz + t] = 0.f;
      continue;
    }
    const float v = val[t];
    keys[t] = sym_key((unsigned)lo, (unsigned)c, 0u);
    vals[t] = v;
    keys[nnz + t] = sym_key((unsigned)c, (unsigned)lo, 1u);
    vals[nnz + t] = v;
  }
}

// head[i] = 1 where (row, column) changes
__global__ void k_sym_heads(long m, const unsigned long long *__restrict__ keys,
                            int *__restrict__ head, int *__restrict__ row_count) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < m;
       i += (long)gridDim.x * blockDim.x) {
    const unsigned long long k = keys[i] >> 1;
    const int h = (i == 0 || (keys[i - 1] >> 1) != k) ? 1 : 0;
    head[i] = h;
    if (h) atomicAdd(&row_count[(int)(k >> SYM_ROW_BITS)], 1);
  }
}

// run heads sum their run in sorted order and write the output entry
__global__ void k_sym_reduce(long m, const unsigned long long *__restrict__ keys,
                             const float *__restrict__ vals, const int *__restrict__ head,
                             const int *__restrict__ pos, float scale, int *__restrict__ out_col,
                             float *__restrict__ out_val) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < m;
       i += (long)gridDim.x * blockDim.x) {
    if (!head[i]) continue;
    const unsigned long long k = keys[i] >> 1;
    float acc = vals[i];
    for (long j = i + 1; j < m && (keys[j] >> 1) == k; j++) acc += vals[j];
    const int p = pos[i];
    out_col[p] = (int)(k & ((1ull << SYM_ROW_BITS) - 1));
    out_val[p] = acc * scale;
  }
}

}  // namespace

extern "C" sgt_status sgt_symmetrize_device(sgt_ctx *ctx, int n, long nnz, const int *rowptr,
                                            const int *col, const float *val, float scale,
                                            int *out_rowptr, int *out_col, float *out_val,
                                            long *out_nnz) {
  if (!ctx || !rowptr || !col || !val || !out_rowptr || !out_col || !out_val || !out_nnz)
    return SGT_ERR_INVALID_ARG;
  if (n < 1 || nnz < 0) return SGT_ERR_INVALID_ARG;
  if (n > (1 << SYM_ROW_BITS))
    return sgti_fail(ctx, SGT_ERR_UNSUPPORTED, "sgt_symmetrize_device: n above 2^24");
  if (2 * nnz > 0x7fffffffL)
    return sgti_fail(ctx, SGT_ERR_UNSUPPORTED, "sgt_symmetrize_device: 2 nnz above 2^31");
  cudaStream_t s = sgti_stream(ctx);
  const long m = 2 * nnz;
  if (cudaSetDevice(sgti_device(ctx)) != cudaSuccess)
    return sgti_fail(ctx, SGT_ERR_CUDA, "sgt_symmetrize_device: set device");
  if (m == 0) {
    if (cudaMemsetAsync(out_rowptr, 0, sizeof(int) * ((size_t)n + 1), s) != cudaSuccess)
      return sgti_fail(ctx, SGT_ERR_CUDA, "sgt_symmetrize_device: memset");
    *out_nnz = 0;
    return SGT_OK;
  }
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  float *v0 = nullptr, *v1 = nullptr;
  int *head = nullptr, *pos = nullptr, *cnt = nullptr, *bad = nullptr;
  void *tmp = nullptr;
  size_t tmp_sort = 0, tmp_scan = 0, tmp_rows = 0;
  cudaError_t e = cudaSuccess;
  auto ok = [&](cudaError_t x) { if (e == cudaSuccess) e = x; return e == cudaSuccess; };
  const int end_bit = 2 * SYM_ROW_BITS + 1;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp_sort, k0, k1, v0, v1, (int)m, 0, end_bit, s);
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_scan, head, pos, (int)m, s);
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_rows, cnt, out_rowptr, n + 1, s);
  const size_t tmp_bytes = std::max(tmp_sort, std::max(tmp_scan, tmp_rows));
  ok(sgti_alloc(ctx, (void **)&k0, sizeof(unsigned long long) * m, s));
  ok(sgti_alloc(ctx, (void **)&k1, sizeof(unsigned long long) * m, s));
  ok(sgti_alloc(ctx, (void **)&v0, sizeof(float) * m, s));
  ok(sgti_alloc(ctx, (void **)&v1, sizeof(float) * m, s));
  ok(sgti_alloc(ctx, (void **)&head, sizeof(int) * m, s));
  ok(sgti_alloc(ctx, (void **)&pos, sizeof(int) * m, s));
  ok(sgti_alloc(ctx, (void **)&cnt, sizeof(int) * ((size_t)n + 1), s));
  ok(sgti_alloc(ctx, (void **)&bad, sizeof(int), s));
  ok(sgti_alloc(ctx, (void **)&tmp, tmp_bytes, s));
  int hbad = 0, total = 0;
  if (e == cudaSuccess) {
    const int nb = (int)std::min<long>((nnz + SYM_THREADS - 1) / SYM_THREADS, 148L * 16);
    const int mb = (int)std::min<long>((m + SYM_THREADS - 1) / SYM_THREADS, 148L * 16);
    ok(cudaMemsetAsync(bad, 0, sizeof(int), s));
    ok(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)n + 1), s));
    if (e == cudaSuccess) {
      k_sym_emit<<<nb, SYM_THREADS, 0, s>>>(n, nnz, rowptr, col, val, k0, v0, bad);
      ok(cudaGetLastError());
    }
    size_t tb = tmp_bytes;
    ok(cub::DeviceRadixSort::SortPairs(tmp, tb, k0, k1, v0, v1, (int)m, 0, end_bit, s));
    if (e == cudaSuccess) {
      k_sym_heads<<<mb, SYM_THREADS, 0, s>>>(m, k1, head, cnt);
      ok(cudaGetLastError());
    }
    tb = tmp_bytes;
    ok(cub::DeviceScan::ExclusiveSum(tmp, tb, head, pos, (int)m, s));
    if (e == cudaSuccess) {
      k_sym_reduce<<<mb, SYM_THREADS, 0, s>>>(m, k1, v1, head, pos, scale, out_col, out_val);
      ok(cudaGetLastError());
    }
    // row counts -> rowptr (cnt[n] = 0, so the last entry is the total)
    tb = tmp_bytes;
    ok(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, out_rowptr, n + 1, s));
    ok(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    ok(cudaMemcpyAsync(&total, out_rowptr + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    ok(cudaStreamSynchronize(s));
  }
  for (void *p : {(void *)k0, (void *)k1, (void *)v0, (void *)v1, (void *)head, (void *)pos,
                  (void *)cnt, (void *)bad, tmp})
    if (p) cudaFreeAsync(p, s);
  if (e != cudaSuccess)
    return sgti_fail(ctx, e == cudaErrorMemoryAllocation ? SGT_ERR_NO_MEMORY : SGT_ERR_CUDA,
                     std::string("sgt_symmetrize_device: ") + cudaGetErrorString(e));
  if (hbad) return sgti_fail(ctx, SGT_ERR_INVALID_ARG, "sgt_symmetrize_device: column out of range");
  *out_nnz = total;
  return SGT_OK;
}
