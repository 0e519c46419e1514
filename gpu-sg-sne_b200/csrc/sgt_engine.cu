// sgt_engine.cu -- host side of the engine: the C ABI of include/sgtsne_b200.h.
//
// One sgt_job holds an embedding's P, coordinates, momentum, gains, grids and
// scratch in HBM.  An iteration is captured once as a CUDA graph (fixed
// launch shapes; every size that changes per iteration is read by the
// kernels from the device-side SgtState) and replayed max_iter times with no
// host synchronisation.  Operators (sgt_attractive, sgt_repulsive, ...) run
// the same kernels on caller buffers for parity tests and for callers that
// drive the loop themselves.
#include "../../include/sgtsne_b200.h"
#include "sgt_internal.h"
#include "sgt_common.cuh"
#include "sgt_fft.cuh"
#include "sgt_grid.cuh"
#include "sgt_prep.cuh"
#include "sgt_rows.cuh"
#include "sgt_relayout.cuh"
#include "sgt_multi.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

struct sgt_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // branch stream of an iteration: the attractive SpMV runs on it beside the
  // repulsion chain on `stream` (forked and joined with events, so captured
  // graphs get two parallel branches)
  cudaStream_t side = nullptr;
  int nsm = 148;
  std::string err;
  sgt_job *scratch = nullptr;  // buffers of the operator entry points
  int scratch_n = 0, scratch_d = 0;
  int last_N = 0, last_d = 0;
  // sgt_batch_step: device tables of the fused launches (grown as needed)
  // and the fork/join events of up to three dimension groups
  void *step_tables = nullptr;
  size_t step_bytes = 0;
  cudaEvent_t step_ev[9] = {};
  // the context's memory pool (release threshold: never), trimmed by
  // sgt_destroy
  cudaMemPool_t pool = nullptr;
};

cudaError_t sgti_alloc(sgt_ctx *ctx, void **p, size_t bytes, cudaStream_t s) {
  return cudaMallocFromPoolAsync(p, bytes, ctx->pool, s);
}

struct sgt_job {
  sgt_ctx *ctx = nullptr;
  sgt_params p{};
  SgtJobParams jp{};
  int n = 0, d = 0, S = 1, G = 8, format = SGT_FORMAT_CSR;
  long nnz = 0;
  int *rowptr = nullptr;
  int2 *pairs = nullptr;
  unsigned *coo_rows = nullptr, *coo_cols = nullptr;
  float *coo_vals = nullptr;
  long coo_n = 0;
  unsigned *ell_cols = nullptr;
  float *ell_vals = nullptr;
  int ell_w = 0;
  int *perm = nullptr;  // engine slot -> caller's point index (nullptr: identity)
  // a shard of a row-split embedding (sgt_shard_*): its rows are points
  // row0.. of the whole coordinate array Ygather, from which the SpMV
  // gathers; nullptr / 0 for a whole embedding
  float *Ygather = nullptr;
  int row0 = 0;
  int n_gather = 0;  // points the columns of P index (n for a whole embedding)
  // locality relabelling (CSR format): scratch allocated on first use
  int *rowptr_alt = nullptr, *perm_alt = nullptr, *rl_p = nullptr, *rl_iperm = nullptr,
      *rl_hist = nullptr, *rl_len = nullptr, *rl_bsum = nullptr;
  unsigned *rl_keys = nullptr;
  int2 *pairs_alt = nullptr;
  float *gains_alt = nullptr;
  long host_iter = 0;  // iterations since the last set_y
  int relayouts = 0;
  float *Y = nullptr, *Ynext = nullptr, *uY = nullptr, *gains = nullptr,
        *Frep = nullptr, *Fattr = nullptr;
  float4 *sorted = nullptr;
  float *V = nullptr, *Phi = nullptr;
  float2 *W = nullptr;
  int mmax = 0, nmax = 0;
  int *tile_count = nullptr, *cursor = nullptr;
  int4 *chunks = nullptr;
  float4 *part_min = nullptr, *part_max = nullptr;
  double *part_sum = nullptr, *part_z = nullptr, *part_kl = nullptr;
  SgtState *st = nullptr;
  SgtState *st_host = nullptr;
  int nb_pts = 0, nb_bin = 0, nb_s2g = 0, nb_s2gc = 0, nb_g2s = 0, nb_fft = 0, nb_fft_rows = 0, nb_row = 0,
      nb_upd = 0, nb_part = 0;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;  // the two branches of an iteration
  size_t smem_s2g = 0, smem_s2g8 = 0, smem_fft1 = 0, smem_fft2 = 0;
  size_t smem_s2gd = 0, smem_g2sd = 0;  // direct-mode S2G and G2S (0: the job never takes it)
  int nb_s2g8 = 0;  // 3-D tiles of 8 cells
  cudaGraphExec_t gexec = nullptr;        // one iteration
  cudaGraphExec_t gexec_multi = nullptr;  // SGT_GRAPH_ITERS chained iterations
  std::vector<void *> allocs;
  double last_kl = 0.0;
  float tune_ms[4] = {0, 0, 0, 0};  // row kernel ms for G = 4, 8, 16, 32
};

// ---------------------------------------------------------------------------
// error plumbing
// ---------------------------------------------------------------------------
static sgt_status fail(sgt_ctx *ctx, sgt_status s, const std::string &msg) {
  if (ctx) ctx->err = msg;
  return s;
}
// The status of the error bits a step leaves in SgtState::error: non-finite
// coordinates first, then the capacity bits (outputs written, but not what
// the reference computes).
static sgt_status flag_status(sgt_ctx *ctx, int flags, int grid_points, const char *where) {
  if (flags & SGT_EFLAG_NONFINITE)
    return fail(ctx, SGT_ERR_NUMERIC, std::string(where) + ": non-finite coordinates");
  if (flags & SGT_EFLAG_CHUNK_OVERFLOW)
    return fail(ctx, SGT_ERR_CAPACITY,
                std::string(where) + ": the S2G guard skipped points (charge grid incomplete)");
  if (flags & SGT_EFLAG_GRID_CLAMP)
    return fail(ctx, SGT_ERR_CAPACITY,
                std::string(where) + ": the embedding needs a larger grid than provisioned; "
                "the step ran on " + std::to_string(grid_points) +
                " points per axis (raise max_grid)");
  return SGT_OK;
}
cudaStream_t sgti_stream(sgt_ctx *ctx) { return ctx->stream; }
int sgti_device(sgt_ctx *ctx) { return ctx->device; }
sgt_status sgti_fail(sgt_ctx *ctx, sgt_status s, const std::string &msg) { return fail(ctx, s, msg); }
#define CK(call)                                                              \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess)                                                    \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? SGT_ERR_NO_MEMORY    \
                                                       : SGT_ERR_CUDA,        \
                  std::string(#call) + ": " + cudaGetErrorString(e_));         \
  } while (0)
#define CKS(expr)                                                             \
  do {                                                                        \
    sgt_status s_ = (expr);                                                   \
    if (s_ != SGT_OK) return s_;                                              \
  } while (0)

// Device memory is stream-ordered (cudaMallocFromPoolAsync / cudaFreeAsync on
// the context's stream from the context's pool): creating or retiring a job
// never waits for work on other streams, which cudaFree would (it
// synchronises the device).  Jobs of one context share its stream, so
// every use of a buffer is ordered between its allocation and its free.
template <typename T>
static sgt_status jalloc(sgt_job *J, T **ptr, size_t count) {
  sgt_ctx *ctx = J->ctx;
  void *p = nullptr;
  if (count == 0) count = 1;
  CK(sgti_alloc(ctx, (void **)&p, count * sizeof(T), ctx->stream));
  J->allocs.push_back(p);
  *ptr = (T *)p;
  return SGT_OK;
}

static int grid_blocks(int nsm, int per_sm) { return std::max(1, nsm * std::max(1, per_sm)); }

// iterations per launch of a job's chained graph (sgt_job_run)
#define SGT_GRAPH_ITERS 16
// nonzeros of P from which a job's repulsion chain runs one block per SM
#define SGT_CHAIN_NARROW_NNZ 16000000L

static void drop_graphs(sgt_job *J) {
  if (J->gexec) cudaGraphExecDestroy(J->gexec);
  if (J->gexec_multi) cudaGraphExecDestroy(J->gexec_multi);
  J->gexec = nullptr;
  J->gexec_multi = nullptr;
}

extern "C" {

void sgt_params_default(sgt_params *p) {
  memset(p, 0, sizeof(*p));
  p->d = 2;
  p->lambda = 1.0f;
  p->alpha = 12.0f;
  p->max_iter = 1000;
  p->early_iter = 250;
  p->n = 0;
  p->h = -1.0f;
  p->format = SGT_FORMAT_COO;
  p->compute_error = -1;
  p->ng = 50;
  p->grid_mode = SGT_GRID_H;
  p->lambda_dist = 1;
  p->seed = 0;
  p->relayout_every = 0;
  p->locality_order = 1;
}

int sgt_abi_version(void) { return SGT_ABI_VERSION; }

const char *sgt_status_string(sgt_status s) {
  switch (s) {
    case SGT_OK: return "ok";
    case SGT_ERR_INVALID_ARG: return "invalid argument";
    case SGT_ERR_CUDA: return "CUDA error";
    case SGT_ERR_NO_MEMORY: return "out of memory";
    case SGT_ERR_UNSUPPORTED: return "unsupported";
    case SGT_ERR_NUMERIC: return "non-finite values";
    case SGT_ERR_NO_DEVICE: return "no CUDA device";
    case SGT_ERR_CAPACITY: return "device capacity reached";
  }
  return "unknown";
}

int sgt_best_grid_size(int ng) {
  static const int sizes[137] = {
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
  for (int i = 0; i < 137; i++)
    if (ng + 2 <= sizes[i]) return sizes[i] - 2;
  return sizes[136] - 2;
}

sgt_status sgt_create(int device, sgt_ctx **out) {
  if (!out) return SGT_ERR_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return SGT_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) return SGT_ERR_INVALID_ARG;
  sgt_ctx *ctx = new sgt_ctx();
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    e = cudaMemPoolCreate(&ctx->pool, &props);
    if (e == cudaSuccess) {
      unsigned long long keep = ~0ull;
      e = cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  if (e != cudaSuccess) {
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SGT_ERR_CUDA;
  }
  ctx->own_stream = true;
  *out = ctx;
  return SGT_OK;
}

void sgt_job_destroy(sgt_job *job);

void sgt_destroy(sgt_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->scratch) sgt_job_destroy(ctx->scratch);
  if (ctx->step_tables) {
    cudaFreeAsync(ctx->step_tables, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
  }
  for (cudaEvent_t e : ctx->step_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->pool) {
    // buffers still allocated (a job the caller did not destroy) keep the
    // pool alive until they are freed
    cudaStreamSynchronize(ctx->stream);
    cudaMemPoolTrimTo(ctx->pool, 0);
    cudaMemPoolDestroy(ctx->pool);
  }
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->side) cudaStreamDestroy(ctx->side);
  delete ctx;
}

sgt_status sgt_set_stream(sgt_ctx *ctx, void *stream) {
  if (!ctx) return SGT_ERR_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  // work queued so far (and the stream-ordered frees of jobs destroyed
  // later on the new stream) must not overlap: drain the old stream
  if (ctx->stream) CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->scratch) {
    sgt_job_destroy(ctx->scratch);
    ctx->scratch = nullptr;
  }
  if (ctx->own_stream && ctx->stream) CK(cudaStreamDestroy(ctx->stream));
  if (stream) {
    ctx->stream = (cudaStream_t)stream;
    ctx->own_stream = false;
  } else {
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->own_stream = true;
  }
  return SGT_OK;
}

const char *sgt_last_error(const sgt_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

}  // extern "C"

// ---------------------------------------------------------------------------
// validation of a CSR structure (host copy)
// ---------------------------------------------------------------------------
static sgt_status check_csr(sgt_ctx *ctx, int n, const int *rowptr, const int *col,
                           int ncols = -1) {
  if (ncols < 0) ncols = n;
  if (rowptr[0] != 0) return fail(ctx, SGT_ERR_INVALID_ARG, "rowptr[0] != 0");
  for (int i = 0; i < n; i++)
    if (rowptr[i + 1] < rowptr[i])
      return fail(ctx, SGT_ERR_INVALID_ARG, "rowptr not monotone at row " + std::to_string(i));
  const long nnz = rowptr[n];
  for (long t = 0; t < nnz; t++)
    if (col[t] < 0 || col[t] >= ncols)
      return fail(ctx, SGT_ERR_INVALID_ARG, "column out of range at nonzero " + std::to_string(t));
  return SGT_OK;
}

// CSR -> ELL (column-major, zero padded) + COO tail in row order on the
// device, given the row pointers on the host too (for the tail offsets).
// The same layout as sgt_csr_to_hybrid (CU/prepareMatrix.cu:55-97).
__global__ void k_csr_to_hybrid(int n, int w, const int *__restrict__ rowptr,
                                const int *__restrict__ col, const float *__restrict__ val,
                                const long *__restrict__ tail, unsigned *__restrict__ ell_cols,
                                float *__restrict__ ell_vals, unsigned *__restrict__ coo_rows,
                                unsigned *__restrict__ coo_cols, float *__restrict__ coo_vals) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int s0 = rowptr[r], len = rowptr[r + 1] - s0;
    for (int k = 0; k < w; k++) {  // consecutive rows write consecutive slots
      const bool in = k < len;
      ell_cols[(size_t)k * n + r] = in ? (unsigned)col[s0 + k] : 0u;
      ell_vals[(size_t)k * n + r] = in ? val[s0 + k] : 0.f;
    }
    const long t0 = tail[r];
    for (int k = w; k < len; k++) {
      coo_rows[t0 + k - w] = (unsigned)r;
      coo_cols[t0 + k - w] = (unsigned)col[s0 + k];
      coo_vals[t0 + k - w] = val[s0 + k];
    }
  }
}

static sgt_status hybrid_split_device(sgt_ctx *ctx, int n, const std::vector<int> &hrp,
                                      const int *rowptr, const int *col, const float *val, int w,
                                      unsigned *ell_cols, float *ell_vals, unsigned *coo_rows,
                                      unsigned *coo_cols, float *coo_vals, long *coo_size) {
  cudaStream_t s = ctx->stream;
  std::vector<long> tail((size_t)n + 1, 0);
  for (int r = 0; r < n; r++) tail[r + 1] = tail[r] + std::max(0, hrp[r + 1] - hrp[r] - w);
  long *dt = nullptr;
  CK(sgti_alloc(ctx, (void **)&dt, sizeof(long) * ((size_t)n + 1), s));
  cudaError_t e = cudaMemcpyAsync(dt, tail.data(), sizeof(long) * ((size_t)n + 1),
                                  cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    k_csr_to_hybrid<<<grid_blocks(ctx->nsm, 4), SGT_THREADS, 0, s>>>(
        n, w, rowptr, col, val, dt, ell_cols, ell_vals, coo_rows, coo_cols, coo_vals);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host tail array is freed next
  cudaFreeAsync(dt, s);
  CK(e);
  *coo_size = tail[n];
  return SGT_OK;
}

static int choose_group(long nnz, int n) {
  const double avg = n > 0 ? (double)nnz / n : 0.0;
  if (avg <= 6) return 4;
  if (avg <= 20) return 8;
  if (avg <= 72) return 16;
  return 32;
}

// ---------------------------------------------------------------------------
// job creation
// ---------------------------------------------------------------------------
template <int D>
static sgt_status job_shapes(sgt_job *J) {
  sgt_ctx *ctx = J->ctx;
  const int nsm = ctx->nsm;
  int occ = 0;
  J->nb_pts = grid_blocks(nsm, 4);
  constexpr int T = D == 1 ? 512 : (D == 2 ? 32 : 16);
  const int R = T + 3;
  J->smem_s2g = sizeof(float) * (D + 1) * (size_t)(D == 1 ? R : (D == 2 ? R * R : R * R * R));
  CK(cudaFuncSetAttribute(k_s2g<D, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)J->smem_s2g));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_s2g<D, T>, SGT_THREADS, J->smem_s2g));
  J->nb_s2g = grid_blocks(nsm, occ);
  if constexpr (D == 3) {
    J->smem_s2g8 = sizeof(float) * 4 * 11 * 11 * 11;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_s2g<3, 8>, SGT_THREADS, J->smem_s2g8));
    J->nb_s2g8 = grid_blocks(nsm, occ);
  }
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_s2g_cell<D>, SGT_THREADS, 0));
  J->nb_s2gc = grid_blocks(nsm, occ);
  // direct mode (d <= 2, jobs that can take it): the S2G's grid copy (m
  // planes of N^d floats) and the G2S's potential grid (N^d nodes)
  if constexpr (D <= 2) {
    const size_t dn = (size_t)J->jp.direct_max;
    const size_t dnodes = D == 1 ? dn : dn * dn;
    J->smem_s2gd = sizeof(float) * (D + 1) * dnodes;
    J->smem_g2sd = sizeof(typename Node<D>::T) * dnodes;
    // the attributes allow the largest job of this dimension (jobs of other
    // sizes set them too, and every job's launches must stay allowed)
    const size_t dmax = D == 1 ? 512 : (size_t)SGT_DIRECT_N2 * SGT_DIRECT_N2;
    CK(cudaFuncSetAttribute(k_s2g_direct<D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)(sizeof(float) * (D + 1) * dmax)));
    CK(cudaFuncSetAttribute(k_g2s_direct<D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)(sizeof(typename Node<D>::T) * dmax)));
  }
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_g2s<D>, SGT_THREADS, 0));
  J->nb_g2s = grid_blocks(nsm, occ);
  const int M = J->mmax;
  J->smem_fft1 = 0;
  J->smem_fft2 = fft_cols_smem(M, D);
  if constexpr (D == 1) {
    J->nb_fft = 1;
  } else {
    const int fmax = (int)fft_cols_smem(SGT_FFT_MAXM, D);  // the largest job's
    CK(cudaFuncSetAttribute(k_fft_cols<D, MODE_LAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, fmax));
    if constexpr (D == 3) {
      CK(cudaFuncSetAttribute(k_fft_cols<D, MODE_MID_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, fmax));
      CK(cudaFuncSetAttribute(k_fft_cols<D, MODE_MID_INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, fmax));
    }
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fft_cols<D, MODE_LAST>, SGT_THREADS, J->smem_fft2));
    J->nb_fft = grid_blocks(nsm, occ);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fft_build_x<D>, SGT_THREADS, 0));
    J->nb_fft_rows = grid_blocks(nsm, occ);
  }
  occ = 0;
  switch (J->G) {
    case 4: CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_row_update<D, 4, true>, SGT_THREADS, 0)); break;
    case 8: CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_row_update<D, 8, true>, SGT_THREADS, 0)); break;
    case 16: CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_row_update<D, 16, true>, SGT_THREADS, 0)); break;
    default: CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_row_update<D, 32, true>, SGT_THREADS, 0)); break;
  }
  J->nb_row = grid_blocks(nsm, occ);
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_row_update<D, 1, false>, SGT_THREADS, 0));
  J->nb_upd = grid_blocks(nsm, occ);
  // A job whose SpMV is large runs its repulsion chain beside an SpMV that
  // holds every SM: a chain kernel's blocks start only as SpMV blocks retire,
  // so one block per SM (each with more points) finishes sooner than four.
  // 1.3M points (67M nonzeros): 337 against 351 us per iteration; 400k
  // (20M): 114 against 119.
  J->nb_bin = J->nb_pts;
  if (J->nnz >= SGT_CHAIN_NARROW_NNZ) {
    J->nb_bin = std::min(J->nb_bin, nsm);
    J->nb_s2g = std::min(J->nb_s2g, nsm);
    J->nb_s2g8 = std::min(J->nb_s2g8, nsm);
    J->nb_s2gc = std::min(J->nb_s2gc, nsm);
    J->nb_g2s = std::min(J->nb_g2s, nsm);
  }
  // small embeddings launch no more blocks than there is work for: idle
  // blocks only take scheduling slots from the jobs that share the GPU
  const int cap = (int)std::max(1L, ((long)J->n + 255) / 256);
  J->nb_pts = std::min(J->nb_pts, cap);
  J->nb_bin = std::min(J->nb_bin, cap);
  J->nb_s2g = std::min(J->nb_s2g, cap);
  J->nb_s2g8 = std::min(J->nb_s2g8, cap);
  J->nb_s2gc = std::min(J->nb_s2gc, cap);
  J->nb_g2s = std::min(J->nb_g2s, cap);
  J->nb_row = std::min(J->nb_row, cap);
  J->nb_upd = std::min(J->nb_upd, cap);
  if constexpr (D == 2) {  // lines of the largest grid this job can take
    const int lines_rows = 2 * J->nmax + J->mmax, lines_cols = J->mmax / SGT_FFT_COLS;
    J->nb_fft_rows = std::min(J->nb_fft_rows, (lines_rows + 7) / 8);
    J->nb_fft = std::min(J->nb_fft, std::max(1, lines_cols));
  }
  J->nb_part = std::max(std::max(J->nb_pts, J->nb_row), std::max(J->nb_g2s, J->nb_s2g));
  J->nb_part = std::max(J->nb_part, J->nb_upd);
  return SGT_OK;
}

static sgt_status job_alloc(sgt_job *J) {
  sgt_ctx *ctx = J->ctx;
  const int D = J->d;
  J->S = D == 3 ? 4 : D;
  const size_t np = (size_t)J->n * J->S;
  CKS(jalloc(J, &J->Y, np));
  CKS(jalloc(J, &J->Ynext, np));
  CKS(jalloc(J, &J->uY, np));
  CKS(jalloc(J, &J->gains, np));
  CKS(jalloc(J, &J->Frep, np));
  CKS(jalloc(J, &J->sorted, (size_t)J->n));
  int max_grid = J->p.max_grid > 0 ? J->p.max_grid : (D <= 2 ? 512 : 128);
  // 3-D: at most 256 points per axis (tile histogram of 16^3 entries,
  // FFT planes of 512^3)
  max_grid = std::min(D == 3 ? 256 : 512, std::max(16, max_grid));
  int M = 1;
  while (M < 2 * max_grid - 1) M <<= 1;
  if (D == 1) M = std::max(M, 32);
  J->mmax = M;
  J->nmax = std::min(512, (M + 1) / 2);
  size_t nodes = J->nmax;
  if (D >= 2) nodes *= J->nmax;
  if (D >= 3) nodes *= J->nmax;
  const int ncomp = D == 1 ? 2 : 4;
  CKS(jalloc(J, &J->V, nodes * ncomp));
  CKS(jalloc(J, &J->Phi, nodes * ncomp));
  size_t plane = M;
  if (D >= 2) plane *= M;
  if (D >= 3) plane *= M;
  if (D >= 2) CKS(jalloc(J, &J->W, 3 * plane));
  CKS(jalloc(J, &J->tile_count, SGT_HIST_MAX));
  CKS(jalloc(J, &J->cursor, SGT_HIST_MAX));
  J->jp.chunk_cap = J->n / 256 + SGT_HIST_MAX + 16;  // 3-D chunks may hold 256 points
  CKS(jalloc(J, &J->chunks, (size_t)J->jp.chunk_cap));
  J->jp.mmax = M;
  J->jp.tile_cap = SGT_HIST_MAX;
  // direct mode for the grids up to direct_max that are too sparse for cell
  // mode; a job with enough points that all of them are dense never takes it
  // (and its kernels keep the small shared-memory footprint the concurrent
  // SpMV wants: the direct mode's grid copies shrink the SMs' L1)
  J->jp.direct_max = D == 1 ? J->nmax : (D == 2 ? std::min(SGT_DIRECT_N2, J->nmax) : 0);
  if (J->jp.direct_max > 0) {
    const long c = J->jp.direct_max - 3, dense = 64L * (D == 1 ? c : c * c);
    if ((long)J->n >= dense && (D == 1 ? c : c * c) <= SGT_HIST_MAX) J->jp.direct_max = 0;
  }
  CKS(jalloc(J, &J->st, 1));
  J->st_host = new SgtState();
  CK(cudaEventCreateWithFlags(&J->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&J->ev_join, cudaEventDisableTiming));
  CK(cudaMemsetAsync(J->tile_count, 0, sizeof(int) * SGT_HIST_MAX, ctx->stream));
  CK(cudaMemsetAsync(J->st, 0, sizeof(SgtState), ctx->stream));
  return SGT_OK;
}

static sgt_status job_alloc_parts(sgt_job *J) {
  CKS(jalloc(J, &J->part_min, (size_t)J->nb_part));
  CKS(jalloc(J, &J->part_max, (size_t)J->nb_part));
  CKS(jalloc(J, &J->part_sum, (size_t)J->nb_part * 4));
  CKS(jalloc(J, &J->part_z, (size_t)J->nb_part));
  CKS(jalloc(J, &J->part_kl, (size_t)J->nb_part));
  return SGT_OK;
}

static void fill_jp(sgt_job *J) {
  const sgt_params &p = J->p;
  J->jp.n = J->n;
  J->jp.d = J->d;
  J->jp.grid_mode = p.grid_mode;
  J->jp.n1_fixed = sgt_best_grid_size(p.ng > 0 ? p.ng : 50);
  float h = p.h;
  if (h <= 0) h = J->d == 1 ? 0.5f : (J->d == 2 ? 0.7f : 1.2f);
  J->jp.h = h;
  J->jp.alpha0 = p.alpha;
  J->jp.early_iter = p.early_iter;
  J->jp.mom_switch = 250;
  J->jp.eta = 200.0f;
}

// empty scratch job for operator calls (no P)
static sgt_status job_new(sgt_ctx *ctx, const sgt_params *p, int n, sgt_job **out) {
  sgt_job *J = new sgt_job();
  J->ctx = ctx;
  J->p = *p;
  J->n = n;
  J->d = p->d;
  J->format = p->format;
  fill_jp(J);
  sgt_status s = job_alloc(J);
  if (s == SGT_OK) {
    switch (J->d) {
      case 1: s = job_shapes<1>(J); break;
      case 2: s = job_shapes<2>(J); break;
      default: s = job_shapes<3>(J); break;
    }
  }
  if (s == SGT_OK) s = job_alloc_parts(J);
  if (s != SGT_OK) {
    sgt_job_destroy(J);
    return s;
  }
  *out = J;
  return SGT_OK;
}

// ---------------------------------------------------------------------------
// iteration enqueue
// ---------------------------------------------------------------------------
// A kernel of the repulsion chain after its first: with pdl set, launched
// with programmatic stream serialisation, so its launch is staged while its
// predecessor on the stream drains (the kernel waits in sgt_pdl_wait before
// it reads anything).  Stage timing passes pdl = false, so that the events
// between the stages see whole kernels.
template <typename... KArgs, typename... Args>
static cudaError_t launch_chain(bool pdl, void (*k)(KArgs...), int grid, int block, size_t smem,
                                cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, args...);
}

template <int D>
static sgt_status enqueue_g2g(sgt_job *J, cudaStream_t s, bool pdl) {
  sgt_ctx *ctx = J->ctx;
  typedef typename Node<D>::T NT;
  if constexpr (D == 1) {
    CK(launch_chain(pdl, k_conv1d, 1, 32, 0, s, (const SgtState *)J->st, (const float2 *)J->V,
                    (float2 *)J->Phi));
  } else {
    CK(launch_chain(pdl, k_fft_build_x<D>, J->nb_fft_rows, SGT_THREADS, 0, s,
                    (const SgtState *)J->st, (const NT *)J->V, J->W));
    if constexpr (D == 3)
      CK(launch_chain(pdl, k_fft_cols<D, MODE_MID_FWD>, J->nb_fft, SGT_THREADS, J->smem_fft2, s,
                      (const SgtState *)J->st, J->W, (const NT *)J->V, (NT *)J->Phi));
    CK(launch_chain(pdl, k_fft_cols<D, MODE_LAST>, J->nb_fft, SGT_THREADS, J->smem_fft2, s,
                    (const SgtState *)J->st, J->W, (const NT *)J->V, (NT *)J->Phi));
    if constexpr (D == 3)
      CK(launch_chain(pdl, k_fft_cols<D, MODE_MID_INV>, J->nb_fft, SGT_THREADS, J->smem_fft2, s,
                      (const SgtState *)J->st, J->W, (const NT *)J->V, (NT *)J->Phi));
    CK(launch_chain(pdl, k_fft_final_x<D>, J->nb_fft_rows, SGT_THREADS, 0, s,
                    (const SgtState *)J->st, (const float2 *)J->W, (NT *)J->Phi));
  }
  return SGT_OK;
}

// Centre Ynext into Y, count points per tile, zero the charge grid.
template <int D>
static sgt_status enqueue_bin_count(sgt_job *J, cudaStream_t s) {
  sgt_ctx *ctx = J->ctx;
  typedef typename Vec<D>::T VT;
  typedef typename Node<D>::T NT;
  k_bin_count<D><<<J->nb_bin, SGT_THREADS, 0, s>>>((const VT *)J->Ynext, (VT *)J->Y, J->n,
                                                   J->st, J->tile_count, (NT *)J->V, 1, J->jp,
                                                   J->cursor, J->chunks, J->nb_s2g);
  CK(cudaGetLastError());
  return SGT_OK;
}

// Sort and S2G (or the direct S2G): the charge grid of this job's points.
// ev (optional): events recorded after the binning and S2G stages.
template <int D>
static sgt_status enqueue_scatter_part(sgt_job *J, cudaStream_t s, cudaEvent_t *ev = nullptr) {
  sgt_ctx *ctx = J->ctx;
  typedef typename Vec<D>::T VT;
  typedef typename Node<D>::T NT;
  const int n = J->n;
  const bool pdl = ev == nullptr;
  // the S2G stage starts with the sort (tile modes) or is the whole direct
  // S2G (direct mode), both in k_bin_scatter
  if (ev) CK(cudaEventRecord(ev[1], s));
  CK(launch_chain(pdl, k_bin_scatter<D>, J->nb_bin, SGT_THREADS, 0, s, (const VT *)J->Y, n, J->st,
                  J->cursor, J->sorted));
  if constexpr (D <= 2)
    if (J->jp.direct_max > 0)
      CK(launch_chain(pdl, k_s2g_direct<D>, J->nb_bin, SGT_THREADS, J->smem_s2gd, s,
                      (const VT *)J->Y, n, J->st, (NT *)J->V));
  // tile mode and cell mode: the kernel of the other mode returns at once
  constexpr int TT = D == 1 ? 512 : (D == 2 ? 32 : 16);
  CK(launch_chain(pdl, k_s2g<D, TT>, J->nb_s2g, SGT_THREADS, J->smem_s2g, s,
                  (const float4 *)J->sorted, J->st, (const int4 *)J->chunks, (NT *)J->V));
  if constexpr (D == 3)
    CK(launch_chain(pdl, k_s2g<3, 8>, J->nb_s2g8, SGT_THREADS, J->smem_s2g8, s,
                    (const float4 *)J->sorted, J->st, (const int4 *)J->chunks, (NT *)J->V));
  CK(launch_chain(pdl, k_s2g_cell<D>, J->nb_s2gc, SGT_THREADS, 0, s, (const float4 *)J->sorted,
                  J->st, (const int4 *)J->chunks, (NT *)J->V));
  if (ev) CK(cudaEventRecord(ev[2], s));
  CK(cudaGetLastError());
  return SGT_OK;
}

// G2G and G2S: potentials at this job's points and Z (the sum over them,
// minus their count).  ev (optional): event recorded after G2G.
template <int D>
static sgt_status enqueue_gather_part(sgt_job *J, cudaStream_t s, cudaEvent_t *ev = nullptr) {
  sgt_ctx *ctx = J->ctx;
  typedef typename Vec<D>::T VT;
  typedef typename Node<D>::T NT;
  const bool pdl = ev == nullptr;
  CKS(enqueue_g2g<D>(J, s, pdl));
  if (ev) CK(cudaEventRecord(ev[3], s));
  CK(launch_chain(pdl, k_g2s<D>, J->nb_g2s, SGT_THREADS, 0, s, (const float4 *)J->sorted, J->st,
                  (const int4 *)J->chunks, (const NT *)J->Phi, (VT *)J->Frep, J->part_z, J->n));
  if constexpr (D <= 2)
    if (J->jp.direct_max > 0)
      CK(launch_chain(pdl, k_g2s_direct<D>, J->nb_g2s, SGT_THREADS, J->smem_g2sd, s, J->st,
                      (const NT *)J->Phi, (VT *)J->Frep, J->part_z, J->n, (const VT *)J->Y));
  CK(cudaGetLastError());
  return SGT_OK;
}

// The rest of the repulsion: tile offsets, sort, S2G, G2G, G2S and Z.
// ev (optional): events recorded after the binning, S2G and G2G stages.
template <int D>
static sgt_status enqueue_repulsion_rest(sgt_job *J, cudaStream_t s, cudaEvent_t *ev = nullptr) {
  CKS(enqueue_scatter_part<D>(J, s, ev));
  return enqueue_gather_part<D>(J, s, ev);
}

template <int D>
static sgt_status enqueue_repulsion(sgt_job *J, cudaStream_t s, cudaEvent_t *ev = nullptr) {
  CKS(enqueue_bin_count<D>(J, s));
  return enqueue_repulsion_rest<D>(J, s, ev);
}

// F_attr in the job's format.  It depends on coordinate differences only,
// so it reads Ynext (the coordinates before the binning pass subtracts
// their mean) and need not wait for that pass.
template <int D, int G>
static sgt_status enqueue_attractive(sgt_job *J, cudaStream_t s) {
  sgt_ctx *ctx = J->ctx;
  typedef typename Vec<D>::T VT;
  const int n = J->n;
  const VT *Yc = (const VT *)(J->Ygather ? J->Ygather : J->Ynext);
  if (J->format == SGT_FORMAT_CSR) {
    const int nb = (int)(((long)n * G + SGT_THREADS - 1) / SGT_THREADS);
    k_attr_rows<D, G><<<nb, SGT_THREADS, 0, s>>>(J->rowptr, J->pairs, Yc, (VT *)J->Fattr, n,
                                                 J->row0);
  } else {
    if (J->format == SGT_FORMAT_HYBRID) {
      k_attr_ell<D><<<J->nb_pts, SGT_THREADS, 0, s>>>(n, J->ell_w, J->ell_cols, J->ell_vals, Yc,
                                                      (VT *)J->Fattr);
    } else {
      CK(cudaMemsetAsync(J->Fattr, 0, sizeof(float) * (size_t)n * J->S, s));
    }
    if (J->coo_n > 0)
      k_attr_coo<D><<<J->nb_pts, SGT_THREADS, 0, s>>>(J->coo_n, J->coo_rows, J->coo_cols,
                                                      J->coo_vals, Yc, J->Fattr);
  }
  CK(cudaGetLastError());
  return SGT_OK;
}

template <int D>
static sgt_status dispatch_attractive(sgt_job *J, cudaStream_t s) {
  switch (J->G) {
    case 4: return enqueue_attractive<D, 4>(J, s);
    case 8: return enqueue_attractive<D, 8>(J, s);
    case 16: return enqueue_attractive<D, 16>(J, s);
    default: return enqueue_attractive<D, 32>(J, s);
  }
}

// dY, gains, momentum, Ynext, and the min/max/sum of Ynext that decide the
// next iteration's grid (one point per thread)
template <int D>
static sgt_status enqueue_combine(sgt_job *J, cudaStream_t s) {
  sgt_ctx *ctx = J->ctx;
  typedef typename Vec<D>::T VT;
  k_row_update<D, 1, false><<<J->nb_upd, SGT_THREADS, 0, s>>>(
      nullptr, nullptr, (const VT *)J->Fattr, (const VT *)J->Y, (const VT *)J->Frep,
      (VT *)J->uY, (VT *)J->gains, (VT *)J->Ynext, J->st, J->jp, J->part_min, J->part_max,
      J->part_sum);
  CK(cudaGetLastError());
  return SGT_OK;
}

// One iteration.  The attractive SpMV (bound by L1 gather throughput) reads
// only Ynext and P; the repulsion chain (a series of latency-bound kernels,
// starting with the binning pass that writes the centred Y) reads only
// Ynext and its own buffers.  The SpMV is forked onto the context's side
// stream and joined before the combine, so in the captured graph the two
// run concurrently.
template <int D>
static sgt_status enqueue_iteration(sgt_job *J, cudaStream_t s) {
  sgt_ctx *ctx = J->ctx;
  CK(cudaEventRecord(J->ev_fork, s));
  CK(cudaStreamWaitEvent(ctx->side, J->ev_fork, 0));
  CKS(dispatch_attractive<D>(J, ctx->side));
  CK(cudaEventRecord(J->ev_join, ctx->side));
  CKS(enqueue_bin_count<D>(J, s));
  CKS(enqueue_repulsion_rest<D>(J, s));
  CK(cudaStreamWaitEvent(s, J->ev_join, 0));
  return enqueue_combine<D>(J, s);
}

static sgt_status dispatch_iteration(sgt_job *J, cudaStream_t s) {
  switch (J->d) {
    case 1: return enqueue_iteration<1>(J, s);
    case 2: return enqueue_iteration<2>(J, s);
    default: return enqueue_iteration<3>(J, s);
  }
}

template <int D>
static sgt_status enqueue_init_stats(sgt_job *J, cudaStream_t s, int centre) {
  sgt_ctx *ctx = J->ctx;
  k_init_stats<D><<<J->nb_pts, SGT_THREADS, 0, s>>>((const typename Vec<D>::T *)J->Ynext, J->n,
                                                    J->st, J->jp, J->part_min, J->part_max,
                                                    J->part_sum, centre);
  CK(cudaGetLastError());
  return SGT_OK;
}
static sgt_status init_stats(sgt_job *J, cudaStream_t s, int centre) {
  switch (J->d) {
    case 1: return enqueue_init_stats<1>(J, s, centre);
    case 2: return enqueue_init_stats<2>(J, s, centre);
    default: return enqueue_init_stats<3>(J, s, centre);
  }
}

static sgt_status pack_y(sgt_job *J, const float *src, int layout, float *dst, cudaStream_t s) {
  sgt_ctx *ctx = J->ctx;
  const int nb = grid_blocks(ctx->nsm, 4);
  const int dm = layout == SGT_LAYOUT_DIM_MAJOR;
  switch (J->d) {
    case 1: k_pack<1><<<nb, SGT_THREADS, 0, s>>>(src, J->n, dm, (float *)dst); break;
    case 2: k_pack<2><<<nb, SGT_THREADS, 0, s>>>(src, J->n, dm, (float2 *)dst); break;
    default: k_pack<3><<<nb, SGT_THREADS, 0, s>>>(src, J->n, dm, (float4 *)dst); break;
  }
  CK(cudaGetLastError());
  return SGT_OK;
}

__global__ void k_fill(float *__restrict__ p, long count, float v) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x)
    p[i] = v;
}

template <int D>
__global__ void k_unpack_divz(const typename Vec<D>::T *__restrict__ src, int n, int dim_major,
                              const SgtState *st, float *__restrict__ dst) {
  const float z = (float)st->Z;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const typename Vec<D>::T v = src[i];
#pragma unroll
    for (int k = 0; k < D; k++) {
      const float x = comp<D>(v, k) / z;
      if (dim_major) dst[i + (long)k * n] = x; else dst[(long)i * D + k] = x;
    }
  }
}

template <int D>
__global__ void k_write_bins(const typename Vec<D>::T *__restrict__ Y, int n,
                             const SgtState *st, uint32_t *__restrict__ bins) {
  const float maxy = st->maxy, scale = st->scale;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const typename Vec<D>::T y = Y[i];
#pragma unroll
    for (int k = 0; k < D; k++) {
      float sh;
      bins[(long)i * D + k] = (uint32_t)floorf(sgt_scale(comp<D>(y, k), st->miny[k], maxy, scale, sh));
    }
  }
}

// mean of the current coordinates subtracted on the way out
template <int D>
__global__ void k_unpack_centred(const typename Vec<D>::T *__restrict__ src, int n, int dim_major,
                                 const SgtState *st, int use_next_mean, const int *perm,
                                 float *__restrict__ dst) {
  float mean[3];
  for (int k = 0; k < D; k++) mean[k] = use_next_mean ? (float)(st->sum[k] / (double)n) : 0.f;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const typename Vec<D>::T v = src[r];
    const int i = perm ? perm[r] : r;
#pragma unroll
    for (int k = 0; k < D; k++) {
      const float x = comp<D>(v, k) - mean[k];
      if (dim_major) dst[i + (long)k * n] = x; else dst[(long)i * D + k] = x;
    }
  }
}

static sgt_status ensure_scratch(sgt_ctx *ctx, int n, int d, int grid_mode, int ng, float h) {
  if (!ctx->scratch || ctx->scratch_n < n || ctx->scratch_d != d) {
    if (ctx->scratch) sgt_job_destroy(ctx->scratch);
    ctx->scratch = nullptr;
    sgt_params p;
    sgt_params_default(&p);
    p.d = d;
    p.format = SGT_FORMAT_CSR;
    CKS(job_new(ctx, &p, n, &ctx->scratch));
    ctx->scratch_n = n;
    ctx->scratch_d = d;
  }
  sgt_job *J = ctx->scratch;
  J->n = n;
  J->jp.n = n;
  J->p.grid_mode = grid_mode;
  J->jp.grid_mode = grid_mode;
  J->jp.n1_fixed = sgt_best_grid_size(ng > 0 ? ng : 50);
  J->jp.h = h > 0 ? h : (d == 1 ? 0.5f : (d == 2 ? 0.7f : 1.2f));
  return SGT_OK;
}


// ---------------------------------------------------------------------------
// autotuner: lanes per row of the attractive SpMV, timed on this job's P
// (scratch input and output arrays; the job's state is not touched).  The
// fastest of G = 4, 8, 16, 32 is kept.
// ---------------------------------------------------------------------------
template <int D, int G>
static float time_spmv(sgt_job *J, const float *tY, float *tF, cudaEvent_t e0, cudaEvent_t e1) {
  typedef typename Vec<D>::T VT;
  cudaStream_t s = J->ctx->stream;
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {  // the first launch warms caches
    cudaEventRecord(e0, s);
    const int nb = (int)(((long)J->n * G + SGT_THREADS - 1) / SGT_THREADS);
    k_attr_rows<D, G><<<nb, SGT_THREADS, 0, s>>>(J->rowptr, J->pairs, (const VT *)tY, (VT *)tF,
                                                 J->n, J->row0);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0) best = std::min(best, ms);
  }
  return best;
}

template <int D>
static sgt_status tune_group_d(sgt_job *J) {
  sgt_ctx *ctx = J->ctx;
  cudaStream_t s = ctx->stream;
  // coordinates for every point P's columns index, forces for its rows
  const size_t np = (size_t)std::max(J->n, J->n_gather) * J->S;
  float *buf = nullptr;
  CK(sgti_alloc(ctx, (void **)&buf, sizeof(float) * np * 2, s));
  CK(cudaMemsetAsync(buf, 0, sizeof(float) * np * 2, s));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const float *tY = buf;  // zero coordinates: the gather pattern of P, finite values
  float *tF = buf + np;
  const int cand[4] = {4, 8, 16, 32};
  float t[4];
  t[0] = time_spmv<D, 4>(J, tY, tF, e0, e1);
  t[1] = time_spmv<D, 8>(J, tY, tF, e0, e1);
  t[2] = time_spmv<D, 16>(J, tY, tF, e0, e1);
  t[3] = time_spmv<D, 32>(J, tY, tF, e0, e1);
  cudaError_t e = cudaStreamSynchronize(s);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(buf, s);
  CK(e);
  CK(cudaGetLastError());
  int best = 0;
  for (int k = 1; k < 4; k++)
    if (t[k] < t[best]) best = k;
  J->G = cand[best];
  for (int k = 0; k < 4; k++) J->tune_ms[k] = t[k];
  return SGT_OK;
}

static sgt_status tune_group(sgt_job *J) {
  switch (J->d) {
    case 1: return tune_group_d<1>(J);
    case 2: return tune_group_d<2>(J);
    default: return tune_group_d<3>(J);
  }
}


// ---------------------------------------------------------------------------
// locality relabelling (see sgt_relayout.cuh); runs between iterations
// ---------------------------------------------------------------------------
static sgt_status scan_exclusive(sgt_job *J, const int *in, int len, int *out, int *total,
                                 cudaStream_t s) {
  sgt_ctx *ctx = J->ctx;
  const int nb = (len + SGT_SCAN_PER_BLOCK - 1) / SGT_SCAN_PER_BLOCK;
  if (nb > 4096) return fail(ctx, SGT_ERR_UNSUPPORTED, "scan longer than 16M items");
  k_scan_blocks<<<nb, 1024, 0, s>>>(in, len, out, J->rl_bsum);
  k_scan_sums<<<1, 1024, 0, s>>>(J->rl_bsum, nb, total);
  k_scan_add<<<grid_blocks(ctx->nsm, 4), SGT_THREADS, 0, s>>>(out, len, J->rl_bsum);
  CK(cudaGetLastError());
  return SGT_OK;
}

template <int D>
static sgt_status relayout_d(sgt_job *J) {
  sgt_ctx *ctx = J->ctx;
  cudaStream_t s = ctx->stream;
  typedef typename Vec<D>::T VT;
  const int n = J->n;
  const int KEYS = 1 << 18;
  if (!J->rl_p) {
    CKS(jalloc(J, &J->rowptr_alt, (size_t)n + 1));
    CKS(jalloc(J, &J->pairs_alt, (size_t)J->nnz + 8));
    CKS(jalloc(J, &J->perm_alt, (size_t)n));
    CKS(jalloc(J, &J->rl_p, (size_t)n));
    CKS(jalloc(J, &J->rl_iperm, (size_t)n));
    CKS(jalloc(J, &J->rl_len, (size_t)n + 1));
    CKS(jalloc(J, &J->rl_hist, (size_t)KEYS + 1));
    CKS(jalloc(J, &J->rl_bsum, 4096));
    CKS(jalloc(J, &J->rl_keys, (size_t)n));
    CKS(jalloc(J, &J->gains_alt, (size_t)n * J->S));
    CK(cudaMemsetAsync(J->pairs_alt + J->nnz, 0, 8 * sizeof(int2), s));
  }
  const int nb = grid_blocks(ctx->nsm, 4);
  CK(cudaMemsetAsync(J->rl_hist, 0, sizeof(int) * KEYS, s));
  k_cell_keys<D><<<nb, SGT_THREADS, 0, s>>>((const VT *)J->Ynext, n, J->st, J->rl_keys, J->rl_hist);
  CKS(scan_exclusive(J, J->rl_hist, KEYS, J->rl_hist, nullptr, s));
  k_key_scatter<<<nb, SGT_THREADS, 0, s>>>(J->rl_keys, n, J->rl_hist, J->rl_p);
  k_perm_prep<<<nb, SGT_THREADS, 0, s>>>(J->rl_p, n, J->rowptr, J->rl_iperm, J->rl_len, J->perm,
                                         J->perm_alt);
  CKS(scan_exclusive(J, J->rl_len, n, J->rowptr_alt, J->rowptr_alt + n, s));
  k_relabel_rows<<<grid_blocks(ctx->nsm, 8), SGT_THREADS, 0, s>>>(
      J->rl_p, J->rl_iperm, n, J->rowptr, J->pairs, J->rowptr_alt, J->pairs_alt);
  // per-point state (all n*S floats): Ynext through the free Y buffer (the
  // next binning rewrites Y), uY through the free F_rep buffer (the next G2S
  // rewrites it), gains through its own spare buffer.  Everything is copied
  // back into the job's own buffers, so the captured iteration graphs (which
  // hold those pointers) stay valid.
  const size_t vb = sizeof(float) * (size_t)n * J->S;
  k_gather_vec<D><<<nb, SGT_THREADS, 0, s>>>((const VT *)J->Ynext, J->rl_p, n, (VT *)J->Y);
  k_gather_vec<D><<<nb, SGT_THREADS, 0, s>>>((const VT *)J->uY, J->rl_p, n, (VT *)J->Frep);
  k_gather_vec<D><<<nb, SGT_THREADS, 0, s>>>((const VT *)J->gains, J->rl_p, n, (VT *)J->gains_alt);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(J->Ynext, J->Y, vb, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(J->uY, J->Frep, vb, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(J->gains, J->gains_alt, vb, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(J->rowptr, J->rowptr_alt, sizeof(int) * ((size_t)n + 1),
                     cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(J->pairs, J->pairs_alt, sizeof(int2) * (size_t)J->nnz,
                     cudaMemcpyDeviceToDevice, s));
  if (!J->perm) CKS(jalloc(J, &J->perm, (size_t)n));
  CK(cudaMemcpyAsync(J->perm, J->perm_alt, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, s));
  J->relayouts++;
  return SGT_OK;
}

// diffusion steps of the initial locality order (more steps flatten the
// structure inside clusters onto the cluster means)
#define SGT_DIFFUSE_STEPS 10
#define SGT_ORDER_MIN_N 65536

// The job's first order: P, the per-point state and the caller <-> engine
// permutation relabelled along the Morton order of diffusion coordinates
// (see sgt_relayout.cuh).  Runs at creation, before the first sgt_job_set_y,
// so Ynext and Y are free to hold the coordinates.
template <int D>
static sgt_status locality_order_d(sgt_job *J) {
  sgt_ctx *ctx = J->ctx;
  cudaStream_t s = ctx->stream;
  typedef typename Vec<D>::T VT;
  const int n = J->n;
  VT *za = (VT *)J->Ynext, *zb = (VT *)J->Y;
  k_diffuse_init<D><<<grid_blocks(ctx->nsm, 4), SGT_THREADS, 0, s>>>(za, n);
  for (int t = 0; t < SGT_DIFFUSE_STEPS; t++) {
    k_diffuse<D><<<grid_blocks(ctx->nsm, 8), SGT_THREADS, 0, s>>>(J->rowptr, J->pairs, za, zb, n);
    std::swap(za, zb);
  }
  CK(cudaGetLastError());
  if (za != (VT *)J->Ynext)
    CK(cudaMemcpyAsync(J->Ynext, za, sizeof(VT) * (size_t)n, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemsetAsync(J->st, 0, sizeof(SgtState), s));
  CKS(init_stats(J, s, 1));  // the lattice of the Morton keys spans these coordinates
  CKS(relayout_d<D>(J));
  J->relayouts = 0;  // counts the relabellings during the run
  if (J->p.relayout_every <= 0) {
    // no relabelling during the run: give back the scratch of the relabelling
    void *scratch[] = {J->rowptr_alt, J->pairs_alt, J->perm_alt, J->rl_p, J->rl_iperm,
                       J->rl_len, J->rl_hist, J->rl_bsum, J->rl_keys, J->gains_alt};
    for (void *q : scratch) {
      auto it = std::find(J->allocs.begin(), J->allocs.end(), q);
      if (it != J->allocs.end()) {
        CK(cudaFreeAsync(q, s));
        J->allocs.erase(it);
      }
    }
    J->rowptr_alt = J->perm_alt = J->rl_p = J->rl_iperm = J->rl_len = J->rl_hist = J->rl_bsum =
        nullptr;
    J->pairs_alt = nullptr;
    J->rl_keys = nullptr;
    J->gains_alt = nullptr;
  }
  return SGT_OK;
}

static sgt_status locality_order(sgt_job *J) {
  switch (J->d) {
    case 1: return locality_order_d<1>(J);
    case 2: return locality_order_d<2>(J);
    default: return locality_order_d<3>(J);
  }
}

static sgt_status relayout(sgt_job *J) {
  if (J->format != SGT_FORMAT_CSR || J->n > (16 << 20)) return SGT_OK;
  switch (J->d) {
    case 1: return relayout_d<1>(J);
    case 2: return relayout_d<2>(J);
    default: return relayout_d<3>(J);
  }
}

static sgt_status job_create_impl(sgt_ctx *ctx, const sgt_params *params, int n, int ncols,
                                  const int *rowptr, const int *col, const float *val,
                                  int mem_is_device, sgt_job **out);

extern "C" {

// ---------------------------------------------------------------------------
// jobs
// ---------------------------------------------------------------------------
sgt_status sgt_job_create(sgt_ctx *ctx, const sgt_params *params, int n, const int *rowptr,
                          const int *col, const float *val, int mem_is_device, sgt_job **out) {
  return job_create_impl(ctx, params, n, n, rowptr, col, val, mem_is_device, out);
}

}  // extern "C"

// ncols: points the columns of P index (n for a whole embedding; all points
// for a shard, whose n rows are a stretch of them)
static sgt_status job_create_impl(sgt_ctx *ctx, const sgt_params *params, int n, int ncols,
                                  const int *rowptr, const int *col, const float *val,
                                  int mem_is_device, sgt_job **out) {
  if (!ctx || !params || !rowptr || !col || !val || !out) return SGT_ERR_INVALID_ARG;
  if (n < 2) return fail(ctx, SGT_ERR_INVALID_ARG, "need at least 2 points");
  if (params->d < 1 || params->d > 3) return fail(ctx, SGT_ERR_UNSUPPORTED, "d must be 1, 2 or 3");
  if (params->format != SGT_FORMAT_CSR && params->format != SGT_FORMAT_COO &&
      params->format != SGT_FORMAT_HYBRID)
    return fail(ctx, SGT_ERR_UNSUPPORTED, "format must be 0 (csr), 2 (coo) or 3 (hybrid)");
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  // host copy of the structure (validation, formats)
  std::vector<int> hrp(n + 1);
  if (mem_is_device) {
    CK(cudaMemcpyAsync(hrp.data(), rowptr, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  } else {
    memcpy(hrp.data(), rowptr, sizeof(int) * (n + 1));
  }
  const long nnz = hrp[n];
  if (nnz <= 0) return fail(ctx, SGT_ERR_INVALID_ARG, "P has no nonzeros");
  if (!mem_is_device) CKS(check_csr(ctx, n, hrp.data(), col, ncols));
  if (mem_is_device) {
    int *bad = nullptr;
    CK(sgti_alloc(ctx, (void **)&bad, sizeof(int), s));
    CK(cudaMemsetAsync(bad, 0, sizeof(int), s));
    k_validate_csr<<<grid_blocks(ctx->nsm, 4), SGT_THREADS, 0, s>>>(n, ncols, rowptr, col, bad);
    int hb = 0;
    CK(cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    cudaFreeAsync(bad, s);
    if (hb) return fail(ctx, SGT_ERR_INVALID_ARG, "malformed CSR (rowptr order or column range)");
  }
  sgt_job *J = new sgt_job();
  J->ctx = ctx;
  J->p = *params;
  J->p.n = n;
  J->n = n;
  J->d = params->d;
  J->nnz = nnz;
  J->n_gather = ncols;
  J->format = params->format;
  J->G = choose_group(nnz, n);
  fill_jp(J);
  sgt_status st = job_alloc(J);
  if (st == SGT_OK) {
    switch (J->d) {
      case 1: st = job_shapes<1>(J); break;
      case 2: st = job_shapes<2>(J); break;
      default: st = job_shapes<3>(J); break;
    }
  }
  if (st == SGT_OK) st = job_alloc_parts(J);
  if (st != SGT_OK) {
    sgt_job_destroy(J);
    return st;
  }
  auto bail = [&](sgt_status e) {
    sgt_job_destroy(J);
    return e;
  };
  // P on the device in the chosen format
  int *dcol = nullptr;
  float *dval = nullptr;
  st = jalloc(J, &J->rowptr, (size_t)n + 1);
  if (st != SGT_OK) return bail(st);
  if (J->format == SGT_FORMAT_CSR) {
    // 8 pairs of zero padding: the stream kernel reads whole 4-pair groups
    if ((st = jalloc(J, &J->pairs, (size_t)nnz + 8)) != SGT_OK) return bail(st);
    cudaMemsetAsync(J->pairs + nnz, 0, 8 * sizeof(int2), s);
  }
  const cudaMemcpyKind kind = mem_is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (cudaMemcpyAsync(J->rowptr, rowptr, sizeof(int) * (n + 1), kind, s) != cudaSuccess)
    return bail(fail(ctx, SGT_ERR_CUDA, "copy rowptr"));
  if (J->format == SGT_FORMAT_CSR || J->format == SGT_FORMAT_COO) {
    if (mem_is_device) {
      dcol = (int *)col;
      dval = (float *)val;
    } else {
      if (sgti_alloc(ctx, (void **)&dcol, sizeof(int) * nnz, s) != cudaSuccess ||
          sgti_alloc(ctx, (void **)&dval, sizeof(float) * nnz, s) != cudaSuccess)
        return bail(fail(ctx, SGT_ERR_NO_MEMORY, "staging P"));
      cudaMemcpyAsync(dcol, col, sizeof(int) * nnz, cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(dval, val, sizeof(float) * nnz, cudaMemcpyHostToDevice, s);
    }
    if (J->format == SGT_FORMAT_CSR) {
      k_pack_pairs<<<grid_blocks(ctx->nsm, 8), SGT_THREADS, 0, s>>>(nnz, dcol, dval, J->pairs);
    } else {
      J->coo_n = nnz;
      if ((st = jalloc(J, &J->coo_rows, (size_t)nnz)) != SGT_OK ||
          (st = jalloc(J, &J->coo_cols, (size_t)nnz)) != SGT_OK ||
          (st = jalloc(J, &J->coo_vals, (size_t)nnz)) != SGT_OK)
        return bail(st);
      k_csr_to_coo<<<grid_blocks(ctx->nsm, 8), SGT_THREADS, 0, s>>>(n, nnz, J->rowptr, J->coo_rows);
      cudaMemcpyAsync(J->coo_cols, dcol, sizeof(int) * nnz, cudaMemcpyDeviceToDevice, s);
      cudaMemcpyAsync(J->coo_vals, dval, sizeof(float) * nnz, cudaMemcpyDeviceToDevice, s);
    }
    if (cudaGetLastError() != cudaSuccess) return bail(fail(ctx, SGT_ERR_CUDA, "packing P"));
    if (!mem_is_device) {
      cudaFreeAsync(dcol, s);
      cudaFreeAsync(dval, s);
    }
  } else if (mem_is_device) {  // hybrid from device arrays: split on the device
    const int w = sgt_ell_width(n, hrp.data());
    long csz = 0;
    for (int r = 0; r < n; r++) csz += std::max(0, hrp[r + 1] - hrp[r] - w);
    J->ell_w = w;
    J->coo_n = csz;
    if ((st = jalloc(J, &J->ell_cols, (size_t)n * std::max(w, 1))) != SGT_OK ||
        (st = jalloc(J, &J->ell_vals, (size_t)n * std::max(w, 1))) != SGT_OK ||
        (st = jalloc(J, &J->coo_rows, (size_t)std::max(csz, 1L))) != SGT_OK ||
        (st = jalloc(J, &J->coo_cols, (size_t)std::max(csz, 1L))) != SGT_OK ||
        (st = jalloc(J, &J->coo_vals, (size_t)std::max(csz, 1L))) != SGT_OK)
      return bail(st);
    long got = 0;
    if ((st = hybrid_split_device(ctx, n, hrp, rowptr, col, val, w, J->ell_cols, J->ell_vals,
                                  J->coo_rows, J->coo_cols, J->coo_vals, &got)) != SGT_OK)
      return bail(st);
  } else {  // hybrid from host arrays: host split like CU/prepareMatrix.cu:55-97
    const int *hc = col;
    const float *hv = val;
    const int w = sgt_ell_width(n, hrp.data());
    std::vector<unsigned> ec((size_t)n * std::max(w, 1)), cr(nnz), cc(nnz);
    std::vector<float> ev((size_t)n * std::max(w, 1)), cv(nnz);
    long csz = 0;
    sgt_csr_to_hybrid(n, hrp.data(), hc, hv, w, ec.data(), ev.data(), cr.data(), cc.data(),
                      cv.data(), &csz);
    J->ell_w = w;
    J->coo_n = csz;
    if ((st = jalloc(J, &J->ell_cols, (size_t)n * std::max(w, 1))) != SGT_OK ||
        (st = jalloc(J, &J->ell_vals, (size_t)n * std::max(w, 1))) != SGT_OK ||
        (st = jalloc(J, &J->coo_rows, (size_t)std::max(csz, 1L))) != SGT_OK ||
        (st = jalloc(J, &J->coo_cols, (size_t)std::max(csz, 1L))) != SGT_OK ||
        (st = jalloc(J, &J->coo_vals, (size_t)std::max(csz, 1L))) != SGT_OK)
      return bail(st);
    cudaMemcpyAsync(J->ell_cols, ec.data(), sizeof(unsigned) * (size_t)n * w, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(J->ell_vals, ev.data(), sizeof(float) * (size_t)n * w, cudaMemcpyHostToDevice, s);
    if (csz > 0) {
      cudaMemcpyAsync(J->coo_rows, cr.data(), sizeof(unsigned) * csz, cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(J->coo_cols, cc.data(), sizeof(unsigned) * csz, cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(J->coo_vals, cv.data(), sizeof(float) * csz, cudaMemcpyHostToDevice, s);
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) return bail(fail(ctx, SGT_ERR_CUDA, "hybrid upload"));
  }
  if ((st = jalloc(J, &J->Fattr, (size_t)n * J->S)) != SGT_OK) return bail(st);
  if (J->format == SGT_FORMAT_CSR && params->locality_order > 0 && n >= SGT_ORDER_MIN_N &&
      ncols == n) {
    st = locality_order(J);
    if (st != SGT_OK) return bail(st);
  }
  if (J->format == SGT_FORMAT_CSR) {
    st = tune_group(J);
    if (st != SGT_OK) return bail(st);
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return bail(fail(ctx, SGT_ERR_CUDA, "job setup"));
  *out = J;
  return SGT_OK;
}

extern "C" {

void sgt_job_destroy(sgt_job *J) {
  if (!J) return;
  if (J->ctx) cudaSetDevice(J->ctx->device);
  drop_graphs(J);
  if (J->ctx) {
    cudaStream_t s = J->ctx->stream;
    for (void *p : J->allocs) cudaFreeAsync(p, s);
  }
  delete J->st_host;
  if (J->ev_fork) cudaEventDestroy(J->ev_fork);
  if (J->ev_join) cudaEventDestroy(J->ev_join);
  delete J;
}

sgt_status sgt_job_set_y(sgt_job *J, const float *y, int layout, int mem_is_device) {
  if (!J || !y) return SGT_ERR_INVALID_ARG;
  sgt_ctx *ctx = J->ctx;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const size_t bytes = sizeof(float) * (size_t)J->n * J->d;
  const float *src = y;
  float *staging = nullptr;
  if (!mem_is_device) {
    CK(sgti_alloc(ctx, (void **)&staging, bytes, s));
    CK(cudaMemcpyAsync(staging, y, bytes, cudaMemcpyHostToDevice, s));
    src = staging;
  }
  if (J->perm) {
    // caller order -> engine order through a scratch array (Frep is free here)
    CKS(pack_y(J, src, layout, J->Frep, s));
    const int nb = grid_blocks(ctx->nsm, 4);
    switch (J->d) {
      case 1: k_permute_vec<1><<<nb, SGT_THREADS, 0, s>>>((const float *)J->Frep, J->perm, J->n, (float *)J->Ynext); break;
      case 2: k_permute_vec<2><<<nb, SGT_THREADS, 0, s>>>((const float2 *)J->Frep, J->perm, J->n, (float2 *)J->Ynext); break;
      default: k_permute_vec<3><<<nb, SGT_THREADS, 0, s>>>((const float4 *)J->Frep, J->perm, J->n, (float4 *)J->Ynext); break;
    }
    CK(cudaGetLastError());
  } else {
    CKS(pack_y(J, src, layout, J->Ynext, s));
  }
  CK(cudaMemsetAsync(J->uY, 0, sizeof(float) * (size_t)J->n * J->S, s));
  k_fill<<<grid_blocks(ctx->nsm, 4), SGT_THREADS, 0, s>>>(J->gains, (long)J->n * J->S, 1.0f);
  CK(cudaMemsetAsync(J->st, 0, sizeof(SgtState), s));
  CK(cudaMemsetAsync(J->tile_count, 0, sizeof(int) * SGT_HIST_MAX, s));
  CKS(init_stats(J, s, 1));
  J->host_iter = 0;
  if (staging) {
    CK(cudaStreamSynchronize(s));
    CK(cudaFreeAsync(staging, s));
  }
  return SGT_OK;
}

// Capture `iters` chained iterations of a job into a graph (the kernels read
// every per-iteration size from the device-side state, so one capture
// serves every iteration).
static sgt_status capture_graph(sgt_job *J, int iters, cudaGraph_t *out) {
  sgt_ctx *ctx = J->ctx;
  cudaStream_t s = ctx->stream;
  *out = nullptr;
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  sgt_status es = SGT_OK;
  for (int r = 0; r < iters && es == SGT_OK; r++) es = dispatch_iteration(J, s);
  cudaError_t ce = cudaStreamEndCapture(s, &g);
  if (es != SGT_OK) {
    if (g) cudaGraphDestroy(g);
    return es;
  }
  CK(ce);
  *out = g;
  return SGT_OK;
}

// Node priorities of a captured iteration.  When both branches have blocks
// waiting, the block scheduler should pick the short, latency-bound kernels
// of the repulsion chain first (greatest priority) and fill the rest of the
// GPU with the long, throughput-bound attractive SpMV (least priority), so
// the chain's length hides under the SpMV.  Graphs are instantiated with
// cudaGraphInstantiateFlagUseNodePriority so these priorities apply whatever
// the priority of the stream they are launched into.
static bool is_attractive_kernel(const void *f) {
  static const void *const fs[] = {
      (const void *)k_attr_rows<1, 4>, (const void *)k_attr_rows<1, 8>,
      (const void *)k_attr_rows<1, 16>, (const void *)k_attr_rows<1, 32>,
      (const void *)k_attr_rows<2, 4>, (const void *)k_attr_rows<2, 8>,
      (const void *)k_attr_rows<2, 16>, (const void *)k_attr_rows<2, 32>,
      (const void *)k_attr_rows<3, 4>, (const void *)k_attr_rows<3, 8>,
      (const void *)k_attr_rows<3, 16>, (const void *)k_attr_rows<3, 32>,
      (const void *)k_attr_ell<1>, (const void *)k_attr_ell<2>, (const void *)k_attr_ell<3>,
      (const void *)k_attr_coo<1>, (const void *)k_attr_coo<2>, (const void *)k_attr_coo<3>};
  for (const void *g : fs)
    if (g == f) return true;
  return false;
}

static sgt_status prioritise(sgt_ctx *ctx, cudaGraph_t g) {
  size_t count = 0;
  CK(cudaGraphGetNodes(g, nullptr, &count));
  std::vector<cudaGraphNode_t> nodes(count);
  CK(cudaGraphGetNodes(g, nodes.data(), &count));
  int least = 0, greatest = 0;
  CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  for (cudaGraphNode_t nd : nodes) {
    cudaGraphNodeType t;
    CK(cudaGraphNodeGetType(nd, &t));
    if (t != cudaGraphNodeTypeKernel) continue;
    cudaKernelNodeParams kp;
    CK(cudaGraphKernelNodeGetParams(nd, &kp));
    cudaLaunchAttributeValue v;
    memset(&v, 0, sizeof(v));
    v.priority = is_attractive_kernel(kp.func) ? least : greatest;
    CK(cudaGraphKernelNodeSetAttribute(nd, cudaLaunchAttributePriority, &v));
  }
  return SGT_OK;
}

static sgt_status instantiate(sgt_job *J, int iters, cudaGraphExec_t *exec) {
  sgt_ctx *ctx = J->ctx;
  cudaGraph_t g = nullptr;
  CKS(capture_graph(J, iters, &g));
  sgt_status ps = prioritise(ctx, g);
  if (ps != SGT_OK) {
    cudaGraphDestroy(g);
    return ps;
  }
  cudaError_t ie = cudaGraphInstantiateWithFlags(exec, g, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(g);
  CK(ie);
  return SGT_OK;
}

static sgt_status run_one(sgt_job *J) {
  sgt_ctx *ctx = J->ctx;
  if (!J->gexec) CKS(instantiate(J, 1, &J->gexec));
  CK(cudaGraphLaunch(J->gexec, ctx->stream));
  return SGT_OK;
}

// `iters` iterations with nothing in between: chained graphs of 16, then
// single-iteration graphs
static sgt_status run_chunk(sgt_job *J, int iters) {
  sgt_ctx *ctx = J->ctx;
  int left = iters;
  if (left >= SGT_GRAPH_ITERS && !J->gexec_multi)
    CKS(instantiate(J, SGT_GRAPH_ITERS, &J->gexec_multi));
  for (; left >= SGT_GRAPH_ITERS; left -= SGT_GRAPH_ITERS)
    CK(cudaGraphLaunch(J->gexec_multi, ctx->stream));
  for (; left > 0; left--) CKS(run_one(J));
  return SGT_OK;
}

sgt_status sgt_job_prepare(sgt_job *J) {
  if (!J) return SGT_ERR_INVALID_ARG;
  sgt_ctx *ctx = J->ctx;
  CK(cudaSetDevice(ctx->device));
  if (!J->gexec) CKS(instantiate(J, 1, &J->gexec));
  if (!J->gexec_multi) CKS(instantiate(J, SGT_GRAPH_ITERS, &J->gexec_multi));
  return SGT_OK;
}

sgt_status sgt_job_run(sgt_job *J, int iters) {
  if (!J || iters < 0) return SGT_ERR_INVALID_ARG;
  sgt_ctx *ctx = J->ctx;
  CK(cudaSetDevice(ctx->device));
  const int every = J->p.relayout_every, kl_every = J->p.kl_every;
  // runs of iterations between the points where host work happens (a
  // relayout before every `every`-th iteration, a KL after every
  // `kl_every`-th), each run through the chained graphs
  int left = iters;
  while (left > 0) {
    if (every > 0 && J->host_iter > 0 && J->host_iter % every == 0) CKS(relayout(J));
    int run = left;
    if (every > 0) run = std::min(run, every - (int)(J->host_iter % every));
    if (kl_every > 0) run = std::min(run, kl_every - (int)(J->host_iter % kl_every));
    CKS(run_chunk(J, run));
    J->host_iter += run;
    left -= run;
    if (kl_every > 0 && (J->host_iter % kl_every) == 0) {
      double kl = 0;
      // KL of the coordinates the step just used (Y) with that step's Z
      CKS(sgt_job_kl(J, -1.0, &kl));
    }
  }
  return SGT_OK;
}

// ---------------------------------------------------------------------------
// batches: one graph, one branch of R chained iterations per job
// ---------------------------------------------------------------------------
// Fused form: the jobs of one dimension run every stage as one launch
// (sgt_multi.cuh).  A group holds the view table of its jobs, one prefix
// table of block counts per stage, and one view/prefix table per row-group
// lane count for the SpMV.
enum {
  FS_BIN_COUNT, FS_BIN_SCATTER, FS_S2G, FS_S2G8, FS_S2G_CELL, FS_FFT_X,
  FS_FFT_MID_FWD, FS_FFT_LAST, FS_FFT_MID_INV, FS_FFT_FINAL, FS_G2S, FS_UPDATE, FS_STAGES
};
struct BatchGroup {
  int D = 2, njobs = 0;
  const SgtJobView *views = nullptr;
  const int *prefix[FS_STAGES] = {};
  int blocks[FS_STAGES] = {};
  size_t smem_s2g = 0, smem_s2g8 = 0, smem_fft = 0, smem_s2gd = 0, smem_g2sd = 0;
  // SpMV: one launch per lane count G present
  struct Spmv {
    int G = 16, njobs = 0, blocks = 0;
    const SgtJobView *views = nullptr;
    const int *prefix = nullptr;
  };
  std::vector<Spmv> spmv;
  cudaStream_t chain = nullptr, side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_spmv = nullptr, ev_done = nullptr;
};

struct sgt_batch {
  sgt_ctx *ctx = nullptr;
  std::vector<sgt_job *> jobs;
  int R = 1;
  cudaGraphExec_t exec_r = nullptr, exec_1 = nullptr;
  bool fused = false;
  std::vector<BatchGroup> groups;
  void *dmem = nullptr;  // the groups' view and prefix tables
};

static sgt_status batch_build(sgt_batch *b, const std::vector<cudaGraph_t> &iter_graphs, int R,
                              cudaGraphExec_t *exec) {
  sgt_ctx *ctx = b->ctx;
  cudaGraph_t parent = nullptr;
  CK(cudaGraphCreate(&parent, 0));
  for (cudaGraph_t g : iter_graphs) {
    cudaGraphNode_t prev = nullptr;
    for (int r = 0; r < R; r++) {
      cudaGraphNode_t node = nullptr;
      const cudaError_t e = cudaGraphAddChildGraphNode(&node, parent, prev ? &prev : nullptr,
                                                       prev ? 1 : 0, g);
      if (e != cudaSuccess) {
        cudaGraphDestroy(parent);
        return fail(ctx, SGT_ERR_CUDA, std::string("batch graph: ") + cudaGetErrorString(e));
      }
      prev = node;
    }
  }
  const cudaError_t ie =
      cudaGraphInstantiateWithFlags(exec, parent, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(parent);
  CK(ie);
  return SGT_OK;
}

}  // extern "C"

static void stage_blocks(const sgt_job *J, int *b, int *nb_s2g2 = nullptr);

static SgtJobView job_view(const sgt_job *J) {
  SgtJobView v;
  memset(&v, 0, sizeof(v));
  v.Ynext_c = J->Ynext;
  v.Ynext = J->Ynext;
  v.Y = J->Y;
  v.uY = J->uY;
  v.gains = J->gains;
  v.Frep = J->Frep;
  v.Fattr = J->Fattr;
  v.sorted = J->sorted;
  v.V = J->V;
  v.Phi = J->Phi;
  v.W = J->W;
  v.tile_count = J->tile_count;
  v.cursor = J->cursor;
  v.chunks = J->chunks;
  v.part_min = J->part_min;
  v.part_max = J->part_max;
  v.part_sum = J->part_sum;
  v.part_z = J->part_z;
  v.st = J->st;
  v.rowptr = J->rowptr;
  v.pairs = J->pairs;
  v.jp = J->jp;
  v.n = J->n;
  int bl[FS_STAGES];
  stage_blocks(J, bl, &v.nb_s2g);  // the binning sizes chunks for the fused S2G grid
  // short chunks: a chunk is one block's serial work in S2G, and in a fused
  // launch the slowest block of the smallest jobs sets the stage's length
  v.jp.chunk_min = 256;
  v.row0 = J->row0;
  return v;
}

// Blocks a job gets in each stage of a fused launch (0: the stage does not
// exist for it).  A job launched alone sizes its grids to fill the GPU; in
// a fused launch its blocks share the GPU with every other job's, so each
// job gets blocks in proportion to its work instead (the kernels loop over
// whatever they are given): a block per 2048 points in the point passes and
// per 2048 points of chunks in S2G and G2S, up to the job's own grid, and the
// FFT passes a block per 8 lines of a 64-point grid (they loop over larger
// ones).  nb_s2g2 is the S2G block count the binning sizes its chunks for.
static void stage_blocks(const sgt_job *J, int *b, int *nb_s2g2) {
  for (int k = 0; k < FS_STAGES; k++) b[k] = 0;
  const int work = std::max(1, (J->n + 2047) / 2048);
  const int s2g = std::min(J->nb_s2g, work);
  b[FS_BIN_COUNT] = std::min(J->nb_bin, work);
  b[FS_BIN_SCATTER] = std::min(J->nb_bin, work);
  b[FS_S2G] = s2g;
  if (J->d == 3) b[FS_S2G8] = std::min(J->nb_s2g8, 2 * work);
  b[FS_S2G_CELL] = std::min(J->nb_s2gc, 2 * work);
  const int rows64 = J->d == 3 ? (2 * 64 * 64 + 128 * 128) / 8 : (2 * 64 + 128) / 8;
  b[FS_FFT_X] = J->d == 1 ? 1 : std::min(J->nb_fft_rows, rows64);
  if (J->d == 3) b[FS_FFT_MID_FWD] = b[FS_FFT_MID_INV] = std::min(J->nb_fft, 128);
  if (J->d >= 2) {
    b[FS_FFT_LAST] = std::min(J->nb_fft, J->d == 3 ? 128 : 16);
    b[FS_FFT_FINAL] = std::min(J->nb_fft_rows, rows64);
  }
  b[FS_G2S] = std::min(J->nb_g2s, 2 * work);
  b[FS_UPDATE] = std::min(J->nb_upd, work);
  if (nb_s2g2) *nb_s2g2 = s2g;
}

// Host images of the tables of fused launches over `jobs` (all CSR): the
// groups by dimension with their block counts, the views and the prefix
// tables; offsets into the two arrays stand in for device pointers until
// bind_fused_tables.
struct FusedImage {
  std::vector<SgtJobView> views;
  std::vector<int> ints;
  std::vector<BatchGroup> groups;
  struct Off {
    size_t views = 0, prefix[FS_STAGES] = {};
    std::vector<std::pair<size_t, size_t>> spmv;  // (views, prefix) per G
  };
  std::vector<Off> offs;
  size_t bytes() const { return sizeof(SgtJobView) * views.size() + sizeof(int) * ints.size(); }
};

static void build_fused_image(const std::vector<sgt_job *> &jobs, FusedImage &im) {
  for (int D = 1; D <= 3; D++) {
    std::vector<sgt_job *> js;
    for (sgt_job *J : jobs)
      if (J->d == D) js.push_back(J);
    if (js.empty()) continue;
    BatchGroup g;
    g.D = D;
    g.njobs = (int)js.size();
    FusedImage::Off o;
    o.views = im.views.size();
    for (sgt_job *J : js) {
      im.views.push_back(job_view(J));
      g.smem_s2g = std::max(g.smem_s2g, J->smem_s2g);
      g.smem_s2g8 = std::max(g.smem_s2g8, J->smem_s2g8);
      g.smem_fft = std::max(g.smem_fft, J->smem_fft2);
      g.smem_s2gd = std::max(g.smem_s2gd, J->smem_s2gd);
      g.smem_g2sd = std::max(g.smem_g2sd, J->smem_g2sd);
    }
    for (int k = 0; k < FS_STAGES; k++) {
      o.prefix[k] = im.ints.size();
      int acc = 0;
      im.ints.push_back(0);
      for (sgt_job *J : js) {
        int bl[FS_STAGES];
        stage_blocks(J, bl);
        acc += bl[k];
        im.ints.push_back(acc);
      }
      g.blocks[k] = acc;
    }
    for (int G : {4, 8, 16, 32}) {
      std::vector<sgt_job *> gj;
      for (sgt_job *J : js)
        if (J->G == G) gj.push_back(J);
      if (gj.empty()) continue;
      BatchGroup::Spmv sp;
      sp.G = G;
      sp.njobs = (int)gj.size();
      const size_t vo = im.views.size(), po = im.ints.size();
      int acc = 0;
      im.ints.push_back(0);
      for (sgt_job *J : gj) {
        im.views.push_back(job_view(J));
        acc += (int)(((long)J->n * G + SGT_THREADS - 1) / SGT_THREADS);
        im.ints.push_back(acc);
      }
      sp.blocks = acc;
      g.spmv.push_back(sp);
      o.spmv.push_back({vo, po});
    }
    im.groups.push_back(g);
    im.offs.push_back(o);
  }
}

// upload the image to `dmem` (image.bytes() bytes) on `s` and point the
// groups at it
static sgt_status bind_fused_image(sgt_ctx *ctx, FusedImage &im, void *dmem, cudaStream_t s) {
  const size_t vbytes = sizeof(SgtJobView) * im.views.size();
  CK(cudaMemcpyAsync(dmem, im.views.data(), vbytes, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync((char *)dmem + vbytes, im.ints.data(), sizeof(int) * im.ints.size(),
                     cudaMemcpyHostToDevice, s));
  const SgtJobView *dv = (const SgtJobView *)dmem;
  const int *di = (const int *)((char *)dmem + vbytes);
  for (size_t q = 0; q < im.groups.size(); q++) {
    BatchGroup &g = im.groups[q];
    g.views = dv + im.offs[q].views;
    for (int k = 0; k < FS_STAGES; k++) g.prefix[k] = di + im.offs[q].prefix[k];
    for (size_t t = 0; t < g.spmv.size(); t++) {
      g.spmv[t].views = dv + im.offs[q].spmv[t].first;
      g.spmv[t].prefix = di + im.offs[q].spmv[t].second;
    }
  }
  return SGT_OK;
}

static sgt_status batch_fused_tables(sgt_batch *b) {
  sgt_ctx *ctx = b->ctx;
  FusedImage im;
  build_fused_image(b->jobs, im);
  CK(sgti_alloc(ctx, (void **)&b->dmem, im.bytes(), ctx->stream));
  CKS(bind_fused_image(ctx, im, b->dmem, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));  // the host image goes out of scope
  b->groups = im.groups;
  for (BatchGroup &g : b->groups) {
    CK(cudaStreamCreateWithFlags(&g.chain, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&g.side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&g.ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&g.ev_spmv, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&g.ev_done, cudaEventDisableTiming));
  }
  return SGT_OK;
}

#define FL(k) g.blocks[k], SGT_THREADS
template <int D>
static sgt_status enqueue_fused_group(sgt_ctx *ctx, BatchGroup &g) {
  cudaStream_t c = g.chain, sd = g.side;
  const SgtJobView *v = g.views;
  const int nj = g.njobs;
  // attractive SpMV of every job, beside the repulsion chain
  for (const BatchGroup::Spmv &sp : g.spmv) {
    switch (sp.G) {
      case 4: km_attr_rows<D, 4><<<sp.blocks, SGT_THREADS, 0, sd>>>(sp.views, sp.prefix, sp.njobs); break;
      case 8: km_attr_rows<D, 8><<<sp.blocks, SGT_THREADS, 0, sd>>>(sp.views, sp.prefix, sp.njobs); break;
      case 16: km_attr_rows<D, 16><<<sp.blocks, SGT_THREADS, 0, sd>>>(sp.views, sp.prefix, sp.njobs); break;
      default: km_attr_rows<D, 32><<<sp.blocks, SGT_THREADS, 0, sd>>>(sp.views, sp.prefix, sp.njobs); break;
    }
  }
  CK(cudaEventRecord(g.ev_spmv, sd));
  km_bin_count<D><<<FL(FS_BIN_COUNT), 0, c>>>(v, g.prefix[FS_BIN_COUNT], nj);
  km_bin_scatter<D><<<FL(FS_BIN_SCATTER), 0, c>>>(v, g.prefix[FS_BIN_SCATTER], nj);
  if constexpr (D <= 2)
    if (g.smem_s2gd > 0)  // some job of the group can take the direct mode
      km_s2g_direct<D><<<FL(FS_BIN_SCATTER), g.smem_s2gd, c>>>(v, g.prefix[FS_BIN_SCATTER], nj);
  constexpr int TT = D == 1 ? 512 : (D == 2 ? 32 : 16);
  km_s2g<D, TT><<<FL(FS_S2G), g.smem_s2g, c>>>(v, g.prefix[FS_S2G], nj);
  if constexpr (D == 3) km_s2g<3, 8><<<FL(FS_S2G8), g.smem_s2g8, c>>>(v, g.prefix[FS_S2G8], nj);
  km_s2g_cell<D><<<FL(FS_S2G_CELL), 0, c>>>(v, g.prefix[FS_S2G_CELL], nj);
  if constexpr (D == 1) {
    km_conv1d<<<g.blocks[FS_FFT_X], 32, 0, c>>>(v, g.prefix[FS_FFT_X], nj);
  } else {
    km_fft_build_x<D><<<FL(FS_FFT_X), 0, c>>>(v, g.prefix[FS_FFT_X], nj);
    if constexpr (D == 3)
      km_fft_cols<D, MODE_MID_FWD><<<FL(FS_FFT_MID_FWD), g.smem_fft, c>>>(v, g.prefix[FS_FFT_MID_FWD], nj);
    km_fft_cols<D, MODE_LAST><<<FL(FS_FFT_LAST), g.smem_fft, c>>>(v, g.prefix[FS_FFT_LAST], nj);
    if constexpr (D == 3)
      km_fft_cols<D, MODE_MID_INV><<<FL(FS_FFT_MID_INV), g.smem_fft, c>>>(v, g.prefix[FS_FFT_MID_INV], nj);
    km_fft_final_x<D><<<FL(FS_FFT_FINAL), 0, c>>>(v, g.prefix[FS_FFT_FINAL], nj);
  }
  km_g2s<D><<<FL(FS_G2S), 0, c>>>(v, g.prefix[FS_G2S], nj);
  if constexpr (D <= 2)
    if (g.smem_g2sd > 0)
      km_g2s_direct<D><<<FL(FS_G2S), g.smem_g2sd, c>>>(v, g.prefix[FS_G2S], nj);
  CK(cudaStreamWaitEvent(c, g.ev_spmv, 0));
  km_row_update<D><<<FL(FS_UPDATE), 0, c>>>(v, g.prefix[FS_UPDATE], nj);
  CK(cudaGetLastError());
  return SGT_OK;
}
#undef FL

// R iterations of every job, captured: per iteration the groups run side by
// side, each group's SpMV beside its repulsion chain
static sgt_status batch_fused_graph(sgt_batch *b, int R, cudaGraphExec_t *exec) {
  sgt_ctx *ctx = b->ctx;
  cudaStream_t s = ctx->stream;
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  sgt_status es = SGT_OK;
  for (int r = 0; r < R && es == SGT_OK; r++) {
    for (BatchGroup &g : b->groups) {
      if (cudaEventRecord(g.ev_fork, s) != cudaSuccess ||
          cudaStreamWaitEvent(g.chain, g.ev_fork, 0) != cudaSuccess ||
          cudaStreamWaitEvent(g.side, g.ev_fork, 0) != cudaSuccess) {
        es = fail(ctx, SGT_ERR_CUDA, "batch capture: fork");
        break;
      }
      switch (g.D) {
        case 1: es = enqueue_fused_group<1>(ctx, g); break;
        case 2: es = enqueue_fused_group<2>(ctx, g); break;
        default: es = enqueue_fused_group<3>(ctx, g); break;
      }
      if (es != SGT_OK) break;
      if (cudaEventRecord(g.ev_done, g.chain) != cudaSuccess) es = fail(ctx, SGT_ERR_CUDA, "batch capture: join");
    }
    for (BatchGroup &g : b->groups)
      if (es == SGT_OK && cudaStreamWaitEvent(s, g.ev_done, 0) != cudaSuccess)
        es = fail(ctx, SGT_ERR_CUDA, "batch capture: join");
  }
  const cudaError_t ce = cudaStreamEndCapture(s, &graph);
  if (es != SGT_OK) {
    if (graph) cudaGraphDestroy(graph);
    return es;
  }
  CK(ce);
  const cudaError_t ie = cudaGraphInstantiate(exec, graph, 0);
  cudaGraphDestroy(graph);
  CK(ie);
  return SGT_OK;
}

template <int D>
static sgt_status fused_attributes(sgt_ctx *ctx, const BatchGroup &g) {
  constexpr int TT = D == 1 ? 512 : (D == 2 ? 32 : 16);
  if constexpr (D <= 2) {  // the largest any group of this dimension asks for
    const size_t dmax = D == 1 ? 512 : (size_t)SGT_DIRECT_N2 * SGT_DIRECT_N2;
    CK(cudaFuncSetAttribute(km_s2g_direct<D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)(sizeof(float) * (D + 1) * dmax)));
    CK(cudaFuncSetAttribute(km_g2s_direct<D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)(sizeof(typename Node<D>::T) * dmax)));
  }
  CK(cudaFuncSetAttribute(km_s2g<D, TT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem_s2g));
  if constexpr (D == 3)
    CK(cudaFuncSetAttribute(km_s2g<3, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem_s2g8));
  if constexpr (D >= 2) {
    CK(cudaFuncSetAttribute(km_fft_cols<D, MODE_LAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem_fft));
    if constexpr (D == 3) {
      CK(cudaFuncSetAttribute(km_fft_cols<D, MODE_MID_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem_fft));
      CK(cudaFuncSetAttribute(km_fft_cols<D, MODE_MID_INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem_fft));
    }
  }
  return SGT_OK;
}

extern "C" {

sgt_status sgt_batch_step(sgt_ctx *ctx, int njobs, sgt_job *const *jobs, int iters) {
  if (!ctx || njobs < 1 || !jobs || iters < 0) return SGT_ERR_INVALID_ARG;
  std::vector<sgt_job *> js(jobs, jobs + njobs);
  for (sgt_job *J : js) {
    if (!J || J->ctx->device != ctx->device)
      return fail(ctx, SGT_ERR_INVALID_ARG, "sgt_batch_step: jobs must live on the context's device");
    if (J->format != SGT_FORMAT_CSR || J->p.relayout_every > 0 || J->p.kl_every > 0 || J->Ygather)
      return fail(ctx, SGT_ERR_UNSUPPORTED,
                  "sgt_batch_step: CSR jobs without relayout, in-loop KL or sharding only");
  }
  if (iters == 0) return SGT_OK;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  FusedImage im;
  build_fused_image(js, im);
  if (im.groups.size() > 3) return fail(ctx, SGT_ERR_UNSUPPORTED, "sgt_batch_step: groups");
  if (im.bytes() > ctx->step_bytes) {
    // stream-ordered: the old tables are freed after the launches that read them
    if (ctx->step_tables) CK(cudaFreeAsync(ctx->step_tables, s));
    ctx->step_tables = nullptr;
    ctx->step_bytes = 0;
    const size_t want = std::max(im.bytes() * 2, (size_t)1 << 16);
    CK(sgti_alloc(ctx, (void **)&ctx->step_tables, want, s));
    ctx->step_bytes = want;
  }
  CKS(bind_fused_image(ctx, im, ctx->step_tables, s));
  for (size_t q = 0; q < im.groups.size(); q++) {
    BatchGroup &g = im.groups[q];
    for (int e = 0; e < 3; e++)
      if (!ctx->step_ev[3 * q + e])
        CK(cudaEventCreateWithFlags(&ctx->step_ev[3 * q + e], cudaEventDisableTiming));
    g.chain = s;
    g.side = ctx->side;
    g.ev_fork = ctx->step_ev[3 * q];
    g.ev_spmv = ctx->step_ev[3 * q + 1];
    g.ev_done = ctx->step_ev[3 * q + 2];
    switch (g.D) {
      case 1: CKS(fused_attributes<1>(ctx, g)); break;
      case 2: CKS(fused_attributes<2>(ctx, g)); break;
      default: CKS(fused_attributes<3>(ctx, g)); break;
    }
  }
  sgt_status st = SGT_OK;
  for (int it = 0; it < iters && st == SGT_OK; it++) {
    for (BatchGroup &g : im.groups) {
      CK(cudaEventRecord(g.ev_fork, s));
      CK(cudaStreamWaitEvent(g.side, g.ev_fork, 0));
      switch (g.D) {
        case 1: st = enqueue_fused_group<1>(ctx, g); break;
        case 2: st = enqueue_fused_group<2>(ctx, g); break;
        default: st = enqueue_fused_group<3>(ctx, g); break;
      }
      if (st != SGT_OK) break;
    }
  }
  // the groups' views live in ctx->step_tables; their host image goes out
  // of scope here (the uploads were staged at the call)
  if (st == SGT_OK)
    for (sgt_job *J : js) J->host_iter += iters;
  return st;
}

sgt_status sgt_batch_create(sgt_ctx *ctx, int njobs, sgt_job *const *jobs, int iters_per_launch,
                            sgt_batch **out) {
  if (!ctx || !out || njobs < 1 || !jobs || iters_per_launch < 1 || iters_per_launch > 256)
    return SGT_ERR_INVALID_ARG;
  *out = nullptr;
  for (int k = 0; k < njobs; k++) {
    if (!jobs[k] || jobs[k]->ctx != ctx)
      return fail(ctx, SGT_ERR_INVALID_ARG, "batch jobs must belong to the batch's context");
    if (jobs[k]->p.relayout_every > 0 || jobs[k]->p.kl_every > 0)
      return fail(ctx, SGT_ERR_UNSUPPORTED, "batch jobs cannot relayout or record KL in the loop");
  }
  CK(cudaSetDevice(ctx->device));
  sgt_batch *b = new sgt_batch();
  b->ctx = ctx;
  b->jobs.assign(jobs, jobs + njobs);
  b->R = iters_per_launch;
  // every job in CSR: one launch per stage over all jobs of a dimension
  bool all_csr = true;
  for (int k = 0; k < njobs; k++) all_csr = all_csr && jobs[k]->format == SGT_FORMAT_CSR;
  if (all_csr) {
    b->fused = true;
    sgt_status st = batch_fused_tables(b);
    for (size_t q = 0; q < b->groups.size() && st == SGT_OK; q++) {
      switch (b->groups[q].D) {
        case 1: st = fused_attributes<1>(ctx, b->groups[q]); break;
        case 2: st = fused_attributes<2>(ctx, b->groups[q]); break;
        default: st = fused_attributes<3>(ctx, b->groups[q]); break;
      }
    }
    if (st == SGT_OK) st = batch_fused_graph(b, b->R, &b->exec_r);
    if (st == SGT_OK && b->R > 1) st = batch_fused_graph(b, 1, &b->exec_1);
    if (st != SGT_OK) {
      sgt_batch_destroy(b);
      return st;
    }
    *out = b;
    return SGT_OK;
  }
  std::vector<cudaGraph_t> gs;
  sgt_status st = SGT_OK;
  for (int k = 0; k < njobs && st == SGT_OK; k++) {
    cudaGraph_t g = nullptr;
    st = capture_graph(jobs[k], 1, &g);
    if (st == SGT_OK) gs.push_back(g);
    if (st == SGT_OK) st = prioritise(ctx, g);
  }
  if (st == SGT_OK) st = batch_build(b, gs, b->R, &b->exec_r);
  if (st == SGT_OK && b->R > 1) st = batch_build(b, gs, 1, &b->exec_1);
  for (cudaGraph_t g : gs) cudaGraphDestroy(g);
  if (st != SGT_OK) {
    sgt_batch_destroy(b);
    return st;
  }
  *out = b;
  return SGT_OK;
}

sgt_status sgt_batch_run(sgt_batch *b, int iters) {
  if (!b || iters < 0) return SGT_ERR_INVALID_ARG;
  sgt_ctx *ctx = b->ctx;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  int left = iters;
  for (; left >= b->R; left -= b->R) CK(cudaGraphLaunch(b->exec_r, s));
  for (; left > 0; left--) CK(cudaGraphLaunch(b->R > 1 ? b->exec_1 : b->exec_r, s));
  for (sgt_job *J : b->jobs) J->host_iter += iters;
  return SGT_OK;
}

void sgt_batch_destroy(sgt_batch *b) {
  if (!b) return;
  cudaSetDevice(b->ctx->device);
  if (b->exec_r) cudaGraphExecDestroy(b->exec_r);
  if (b->exec_1) cudaGraphExecDestroy(b->exec_1);
  for (BatchGroup &g : b->groups) {
    if (g.chain) cudaStreamDestroy(g.chain);
    if (g.side) cudaStreamDestroy(g.side);
    if (g.ev_fork) cudaEventDestroy(g.ev_fork);
    if (g.ev_spmv) cudaEventDestroy(g.ev_spmv);
    if (g.ev_done) cudaEventDestroy(g.ev_done);
  }
  if (b->dmem) cudaFreeAsync(b->dmem, b->ctx->stream);
  delete b;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// One embedding split by rows over ranks (sgt_shard_*).  A shard is a job
// whose n rows are points row0 .. row0 + n - 1 of the whole embedding: P's
// rows of those points (global column indices), their momentum, gains and
// forces.  Three buffers belong to the caller and are exchanged between
// ranks by the caller's collectives between the phases of an iteration:
//   y_all  the coordinates of every point (stride S floats per point), the
//          shard's own rows updated in place by the update phase;
//   grid   the charge grid: S2G of the shard's own points, then the sum
//          over ranks (grid_floats floats, all of which the caller reduces);
//   zsum   one double: Z summed over the shard's own points, then over ranks.
// ---------------------------------------------------------------------------
struct sgt_shard {
  sgt_job *J = nullptr;
  int n_all = 0;       // points of the whole embedding
  float *y_all = nullptr;
  float *grid = nullptr;
  size_t grid_floats = 0;
  double *zsum = nullptr;
  SgtJobParams jp_all{};  // the job's parameters with n = n_all (grid decision)
};

template <int D>
static sgt_status shard_stats(sgt_shard *sh, cudaStream_t s) {
  sgt_job *J = sh->J;
  sgt_ctx *ctx = J->ctx;
  // min, max and mean over every point: the grid decision all ranks share
  k_init_stats<D><<<J->nb_pts, SGT_THREADS, 0, s>>>((const typename Vec<D>::T *)sh->y_all,
                                                    sh->n_all, J->st, sh->jp_all, J->part_min,
                                                    J->part_max, J->part_sum, 1);
  CK(cudaGetLastError());
  return SGT_OK;
}

template <int D>
static sgt_status shard_scatter_d(sgt_shard *sh) {
  sgt_job *J = sh->J;
  sgt_ctx *ctx = J->ctx;
  cudaStream_t s = ctx->stream;
  CKS(shard_stats<D>(sh, s));
  // the attractive SpMV of the own rows on the side stream: it overlaps the
  // grid reduction and the convolution, and the update phase joins it
  CK(cudaEventRecord(J->ev_fork, s));
  CK(cudaStreamWaitEvent(ctx->side, J->ev_fork, 0));
  CKS(dispatch_attractive<D>(J, ctx->side));
  CK(cudaEventRecord(J->ev_join, ctx->side));
  // every float of the buffer is reduced: clear what this grid does not use
  CK(cudaMemsetAsync(sh->grid, 0, sizeof(float) * sh->grid_floats, s));
  CKS(enqueue_bin_count<D>(J, s));
  return enqueue_scatter_part<D>(J, s);
}

template <int D>
static sgt_status shard_update_d(sgt_shard *sh) {
  sgt_job *J = sh->J;
  sgt_ctx *ctx = J->ctx;
  cudaStream_t s = ctx->stream;
  CK(cudaMemcpyAsync(&J->st->Z, sh->zsum, sizeof(double), cudaMemcpyDeviceToDevice, s));
  CK(cudaStreamWaitEvent(s, J->ev_join, 0));
  return enqueue_combine<D>(J, s);
}

extern "C" {

size_t sgt_shard_grid_floats(const sgt_params *params) {
  if (!params || params->d < 1 || params->d > 3) return 0;
  const int D = params->d;
  int max_grid = params->max_grid > 0 ? params->max_grid : (D <= 2 ? 512 : 128);
  max_grid = std::min(D == 3 ? 256 : 512, std::max(16, max_grid));
  int M = 1;
  while (M < 2 * max_grid - 1) M <<= 1;
  if (D == 1) M = std::max(M, 32);
  const size_t nmax = std::min(512, (M + 1) / 2);
  size_t nodes = nmax;
  if (D >= 2) nodes *= nmax;
  if (D >= 3) nodes *= nmax;
  return nodes * (D == 1 ? 2 : 4);
}

sgt_status sgt_shard_create(sgt_ctx *ctx, const sgt_params *params, int n_all, int row0,
                            int nrows, const int *rowptr, const int *col, const float *val,
                            int mem_is_device, float *y_all, float *grid, size_t grid_floats,
                            double *zsum, sgt_shard **out) {
  if (!ctx || !params || !rowptr || !col || !val || !y_all || !grid || !zsum || !out)
    return SGT_ERR_INVALID_ARG;
  if (n_all < 2 || row0 < 0 || nrows < 1 || (long)row0 + nrows > n_all)
    return fail(ctx, SGT_ERR_INVALID_ARG, "sgt_shard_create: rows outside [0, n_all)");
  if (params->format != SGT_FORMAT_CSR)
    return fail(ctx, SGT_ERR_UNSUPPORTED, "sgt_shard_create: shards take P in CSR format");
  if (params->relayout_every > 0 || params->kl_every > 0)
    return fail(ctx, SGT_ERR_UNSUPPORTED, "sgt_shard_create: no relayout or in-loop KL");
  sgt_job *J = nullptr;
  CKS(job_create_impl(ctx, params, nrows, n_all, rowptr, col, val, mem_is_device, &J));
  const size_t need = (size_t)J->nmax * (J->d >= 2 ? J->nmax : 1) * (J->d >= 3 ? J->nmax : 1) *
                      (J->d == 1 ? 2 : 4);
  if (grid_floats < need) {
    sgt_job_destroy(J);
    return fail(ctx, SGT_ERR_INVALID_ARG,
                "sgt_shard_create: grid holds " + std::to_string(grid_floats) +
                    " floats, the job's largest grid needs " + std::to_string(need));
  }
  sgt_shard *sh = new sgt_shard();
  sh->J = J;
  sh->n_all = n_all;
  sh->y_all = y_all;
  sh->grid = grid;
  sh->grid_floats = grid_floats;
  sh->zsum = zsum;
  J->row0 = row0;
  J->Ygather = y_all;
  J->Ynext = y_all + (size_t)row0 * J->S;  // the own rows of the shared array
  J->V = grid;
  sh->jp_all = J->jp;
  sh->jp_all.n = n_all;
  *out = sh;
  return SGT_OK;
}

void sgt_shard_destroy(sgt_shard *sh) {
  if (!sh) return;
  sgt_job_destroy(sh->J);
  delete sh;
}

sgt_status sgt_shard_set_y(sgt_shard *sh, const float *y, int layout, int mem_is_device) {
  if (!sh || !y) return SGT_ERR_INVALID_ARG;
  sgt_job *J = sh->J;
  sgt_ctx *ctx = J->ctx;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const size_t bytes = sizeof(float) * (size_t)sh->n_all * J->d;
  const float *src = y;
  float *staging = nullptr;
  if (!mem_is_device) {
    CK(sgti_alloc(ctx, (void **)&staging, bytes, s));
    CK(cudaMemcpyAsync(staging, y, bytes, cudaMemcpyHostToDevice, s));
    src = staging;
  }
  const int nb = grid_blocks(ctx->nsm, 4);
  const int dm = layout == SGT_LAYOUT_DIM_MAJOR;
  switch (J->d) {
    case 1: k_pack<1><<<nb, SGT_THREADS, 0, s>>>(src, sh->n_all, dm, sh->y_all); break;
    case 2: k_pack<2><<<nb, SGT_THREADS, 0, s>>>(src, sh->n_all, dm, (float2 *)sh->y_all); break;
    default: k_pack<3><<<nb, SGT_THREADS, 0, s>>>(src, sh->n_all, dm, (float4 *)sh->y_all); break;
  }
  CK(cudaGetLastError());
  CK(cudaMemsetAsync(J->uY, 0, sizeof(float) * (size_t)J->n * J->S, s));
  k_fill<<<grid_blocks(ctx->nsm, 4), SGT_THREADS, 0, s>>>(J->gains, (long)J->n * J->S, 1.0f);
  CK(cudaMemsetAsync(J->st, 0, sizeof(SgtState), s));
  CK(cudaMemsetAsync(J->tile_count, 0, sizeof(int) * SGT_HIST_MAX, s));
  if (staging) CK(cudaFreeAsync(staging, s));
  return SGT_OK;
}

sgt_status sgt_shard_scatter(sgt_shard *sh) {
  if (!sh) return SGT_ERR_INVALID_ARG;
  sgt_ctx *ctx = sh->J->ctx;
  CK(cudaSetDevice(ctx->device));
  switch (sh->J->d) {
    case 1: return shard_scatter_d<1>(sh);
    case 2: return shard_scatter_d<2>(sh);
    default: return shard_scatter_d<3>(sh);
  }
}

sgt_status sgt_shard_gather(sgt_shard *sh) {
  if (!sh) return SGT_ERR_INVALID_ARG;
  sgt_job *J = sh->J;
  sgt_ctx *ctx = J->ctx;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  switch (J->d) {
    case 1: CKS(enqueue_gather_part<1>(J, s)); break;
    case 2: CKS(enqueue_gather_part<2>(J, s)); break;
    default: CKS(enqueue_gather_part<3>(J, s)); break;
  }
  CK(cudaMemcpyAsync(sh->zsum, &J->st->Z, sizeof(double), cudaMemcpyDeviceToDevice, s));
  return SGT_OK;
}

sgt_status sgt_shard_update(sgt_shard *sh) {
  if (!sh) return SGT_ERR_INVALID_ARG;
  sgt_ctx *ctx = sh->J->ctx;
  CK(cudaSetDevice(ctx->device));
  switch (sh->J->d) {
    case 1: return shard_update_d<1>(sh);
    case 2: return shard_update_d<2>(sh);
    default: return shard_update_d<3>(sh);
  }
}

sgt_status sgt_shard_get_y(sgt_shard *sh, float *y, int layout, int mem_is_device, int centre) {
  if (!sh || !y) return SGT_ERR_INVALID_ARG;
  sgt_job *J = sh->J;
  sgt_ctx *ctx = J->ctx;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const size_t bytes = sizeof(float) * (size_t)sh->n_all * J->d;
  float *dst = y, *staging = nullptr;
  if (!mem_is_device) {
    CK(sgti_alloc(ctx, (void **)&staging, bytes, s));
    dst = staging;
  }
  // the mean over every point (the update phase leaves the own rows' one)
  switch (J->d) {
    case 1: CKS(shard_stats<1>(sh, s)); break;
    case 2: CKS(shard_stats<2>(sh, s)); break;
    default: CKS(shard_stats<3>(sh, s)); break;
  }
  const int nb = grid_blocks(ctx->nsm, 4);
  const int dm = layout == SGT_LAYOUT_DIM_MAJOR;
  switch (J->d) {
    case 1: k_unpack_centred<1><<<nb, SGT_THREADS, 0, s>>>((const float *)sh->y_all, sh->n_all, dm, J->st, centre, nullptr, dst); break;
    case 2: k_unpack_centred<2><<<nb, SGT_THREADS, 0, s>>>((const float2 *)sh->y_all, sh->n_all, dm, J->st, centre, nullptr, dst); break;
    default: k_unpack_centred<3><<<nb, SGT_THREADS, 0, s>>>((const float4 *)sh->y_all, sh->n_all, dm, J->st, centre, nullptr, dst); break;
  }
  CK(cudaGetLastError());
  if (staging) {
    CK(cudaMemcpyAsync(y, staging, bytes, cudaMemcpyDeviceToHost, s));
    CK(cudaFreeAsync(staging, s));
  }
  CK(cudaMemcpyAsync(J->st_host, J->st, sizeof(SgtState), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return flag_status(ctx, J->st_host->error, J->st_host->N, "sgt_shard_get_y");
}

sgt_status sgt_shard_get_info(sgt_shard *sh, sgt_job_info *info) {
  if (!sh) return SGT_ERR_INVALID_ARG;
  return sgt_job_get_info(sh->J, info);
}

// Device bytes of a job: the buffers of job_alloc, job_alloc_parts and P,
// plus the largest transient of job creation (host P staged on the device,
// or the autotuner's scratch copies).
size_t sgt_job_footprint(const sgt_params *p, int n, long nnz) {
  if (!p || n < 1 || nnz < 0 || p->d < 1 || p->d > 3) return 0;
  const int D = p->d, S = D == 3 ? 4 : D;
  const size_t np = (size_t)n * S;
  size_t b = 5 * np * 4 + (size_t)n * 16;  // Y, Ynext, uY, gains, Frep; sorted
  int max_grid = p->max_grid > 0 ? p->max_grid : (D <= 2 ? 512 : 128);
  max_grid = std::min(D == 3 ? 256 : 512, std::max(16, max_grid));
  size_t M = 1;
  while (M < (size_t)(2 * max_grid - 1)) M <<= 1;
  if (D == 1) M = std::max<size_t>(M, 32);
  size_t nmax = std::min<size_t>(512, (M + 1) / 2), nodes = nmax, plane = M;
  if (D >= 2) { nodes *= nmax; plane *= M; }
  if (D >= 3) { nodes *= nmax; plane *= M; }
  b += 2 * nodes * (D == 1 ? 2 : 4) * 4;                       // V, Phi
  if (D >= 2) b += 3 * plane * 8;                               // FFT planes
  b += 2 * 4096 * 4 + ((size_t)n / 256 + 4096 + 16) * 16;        // tiles, chunks
  const size_t parts = std::max<size_t>(148 * 16, ((size_t)n * 32 + 255) / 256);
  b += parts * (16 + 16 + 32 + 8 + 8) + 1024;                   // partials, state
  b += ((size_t)n + 1) * 4;                                     // rowptr
  size_t transient = 8 * (size_t)nnz;                           // staged col/val
  if (p->format == SGT_FORMAT_CSR) {
    b += ((size_t)nnz + 8) * 8 + np * 4;  // pairs, Fattr
    transient = std::max(transient, 2 * np * 4);
    if (p->locality_order > 0 && n >= SGT_ORDER_MIN_N) {
      b += (size_t)n * 4;  // caller <-> engine permutation
      // relabelling scratch: the relabelled P, its rowptr, permutations,
      // keys and the key histogram (held through the run when the job also
      // relabels during it)
      const size_t rl = ((size_t)nnz + 8) * 8 + (size_t)n * (24 + 4 * S) + ((size_t)1 << 20) * 4;
      if (p->relayout_every > 0) b += rl;
      else transient = std::max(transient, rl);
    }
  } else if (p->format == SGT_FORMAT_COO) {
    b += 12 * (size_t)nnz + np * 4;  // rows, cols, vals; Fattr
  } else {
    // ELL of width W (the CUSP rule keeps n*W below 3 nnz) and the COO tail
    b += 36 * (size_t)nnz + np * 4;
  }
  return b + transient;
}

sgt_status sgt_job_get_y(sgt_job *J, float *y, int layout, int mem_is_device, int centre) {
  if (!J || !y) return SGT_ERR_INVALID_ARG;
  sgt_ctx *ctx = J->ctx;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const size_t bytes = sizeof(float) * (size_t)J->n * J->d;
  float *dst = y, *staging = nullptr;
  if (!mem_is_device) {
    CK(sgti_alloc(ctx, (void **)&staging, bytes, s));
    dst = staging;
  }
  const int nb = grid_blocks(ctx->nsm, 4);
  const int dm = layout == SGT_LAYOUT_DIM_MAJOR;
  switch (J->d) {
    case 1: k_unpack_centred<1><<<nb, SGT_THREADS, 0, s>>>((const float *)J->Ynext, J->n, dm, J->st, centre, J->perm, dst); break;
    case 2: k_unpack_centred<2><<<nb, SGT_THREADS, 0, s>>>((const float2 *)J->Ynext, J->n, dm, J->st, centre, J->perm, dst); break;
    default: k_unpack_centred<3><<<nb, SGT_THREADS, 0, s>>>((const float4 *)J->Ynext, J->n, dm, J->st, centre, J->perm, dst); break;
  }
  CK(cudaGetLastError());
  if (staging) {
    CK(cudaMemcpyAsync(y, staging, bytes, cudaMemcpyDeviceToHost, s));
    CK(cudaFreeAsync(staging, s));
  }
  CK(cudaMemcpyAsync(J->st_host, J->st, sizeof(SgtState), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return flag_status(ctx, J->st_host->error, J->st_host->N, "sgt_job_get_y");
}

sgt_status sgt_job_get_info(sgt_job *J, sgt_job_info *info) {
  if (!J || !info) return SGT_ERR_INVALID_ARG;
  sgt_ctx *ctx = J->ctx;
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(J->st_host, J->st, sizeof(SgtState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  info->iter = J->st_host->iter;
  info->grid_points = J->st_host->N;
  info->h_eff = J->st_host->h_eff;
  info->zeta = J->st_host->Z;
  info->kl = J->last_kl;
  info->error_flags = J->st_host->error;
  info->nnz = J->nnz;
  info->row_group = J->G;
  for (int k = 0; k < 4; k++) info->tune_ms[k] = J->tune_ms[k];
  return SGT_OK;
}

}  // extern "C"

extern "C" {

// alpha < 0: the alpha of the last completed iteration
sgt_status sgt_job_kl(sgt_job *J, double alpha, double *kl) {
  if (!J || !kl) return SGT_ERR_INVALID_ARG;
  sgt_ctx *ctx = J->ctx;
  if (J->format != SGT_FORMAT_CSR)
    return fail(ctx, SGT_ERR_UNSUPPORTED, "KL on a job needs the CSR format");
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  if (alpha < 0) {
    CK(cudaMemcpyAsync(J->st_host, J->st, sizeof(SgtState), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    alpha = J->st_host->alpha > 0 ? J->st_host->alpha : J->p.alpha;
  }
  switch (J->d * 100 + J->G) {
#define KLC(DD, GG) case DD * 100 + GG: k_kl<DD, GG><<<J->nb_row, SGT_THREADS, 0, s>>>(J->rowptr, J->pairs, (const typename Vec<DD>::T *)J->Y, J->st, alpha, J->part_kl, J->n); break;
    KLC(1, 4) KLC(1, 8) KLC(1, 16) KLC(1, 32)
    KLC(2, 4) KLC(2, 8) KLC(2, 16) KLC(2, 32)
    KLC(3, 4) KLC(3, 8) KLC(3, 16) KLC(3, 32)
#undef KLC
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(J->st_host, J->st, sizeof(SgtState), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *kl = J->st_host->kl;
  J->last_kl = *kl;
  return SGT_OK;
}

}  // extern "C"

template <int D>
static sgt_status profile_iteration(sgt_job *J, cudaStream_t s, cudaEvent_t *ev) {
  sgt_ctx *ctx = J->ctx;
  CK(cudaEventRecord(ev[0], s));
  CKS(enqueue_repulsion<D>(J, s, ev));
  CK(cudaEventRecord(ev[4], s));
  CKS(dispatch_attractive<D>(J, s));
  CK(cudaEventRecord(ev[5], s));
  CKS(enqueue_combine<D>(J, s));
  CK(cudaEventRecord(ev[6], s));
  return SGT_OK;
}

// Iterations stage by stage with per-iteration stage times in the layout of
// the reference's timeInfo: slot 7 i + j of iteration i (counted from the
// last sgt_job_set_y; only i < 1000, the reference's array holds 1000
// iterations and puts its totals at 7000..7002).  j = 0 attractive term
// (CU/gradient_descend.cu:72-75), 1 S2G, 2 G2G, 3 G2S (CU/nuconv.cu:71-104),
// 4 forces and update (zetaAndForce, CU/Frep.cu:118-121; here the combine
// kernel, which also applies dY, gains and momentum), 5 S2G..G2S (the nuconv
// total, CU/Frep.cu:111-116), 6 preprocessing (min shift, charges, scaling;
// here the centring, grid decision and binning sort, CU/Frep.cu:92-110).
// Relayouts and KL records happen where sgt_job_run does them.
extern "C" sgt_status sgt_job_run_timed(sgt_job *J, int iters, double *time_info) {
  if (!J || iters < 0) return SGT_ERR_INVALID_ARG;
  sgt_ctx *ctx = J->ctx;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  cudaEvent_t ev[7] = {};
  sgt_status st = SGT_OK;
  for (int i = 0; i < 7 && st == SGT_OK; i++)
    if (cudaEventCreate(&ev[i]) != cudaSuccess) st = fail(ctx, SGT_ERR_CUDA, "event create");
  const int every = J->p.relayout_every, kl_every = J->p.kl_every;
  for (int it = 0; it < iters && st == SGT_OK; it++) {
    if (every > 0 && J->host_iter > 0 && J->host_iter % every == 0) {
      st = relayout(J);
      if (st != SGT_OK) break;
    }
    switch (J->d) {
      case 1: st = profile_iteration<1>(J, s, ev); break;
      case 2: st = profile_iteration<2>(J, s, ev); break;
      default: st = profile_iteration<3>(J, s, ev); break;
    }
    if (st != SGT_OK) break;
    cudaError_t e = cudaEventSynchronize(ev[6]);
    if (e != cudaSuccess) {
      st = fail(ctx, SGT_ERR_CUDA, std::string("sgt_job_run_timed: ") + cudaGetErrorString(e));
      break;
    }
    const long gi = J->host_iter;
    if (time_info && gi < 1000) {
      // (from event, to event) per slot
      static const int span[7][2] = {{4, 5}, {1, 2}, {2, 3}, {3, 4}, {5, 6}, {1, 4}, {0, 1}};
      for (int j = 0; j < 7; j++) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[span[j][0]], ev[span[j][1]]);
        time_info[7 * gi + j] = ms;
      }
    }
    J->host_iter++;
    if (kl_every > 0 && (J->host_iter % kl_every) == 0) {
      double kl = 0;
      st = sgt_job_kl(J, -1.0, &kl);
    }
  }
  for (int i = 0; i < 7; i++)
    if (ev[i]) cudaEventDestroy(ev[i]);
  return st;
}

extern "C" sgt_status sgt_job_profile(sgt_job *J, int iters, double *stage_ms) {
  if (!J || !stage_ms || iters < 0) return SGT_ERR_INVALID_ARG;
  sgt_ctx *ctx = J->ctx;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  cudaEvent_t ev[7];
  for (int i = 0; i < 7; i++) CK(cudaEventCreate(&ev[i]));
  for (int it = 0; it < iters; it++) {
    // the kernels of an iteration, one stage after another on one stream
    // (the captured iteration runs the SpMV beside the repulsion instead)
    switch (J->d) {
      case 1: CKS(profile_iteration<1>(J, s, ev)); break;
      case 2: CKS(profile_iteration<2>(J, s, ev)); break;
      default: CKS(profile_iteration<3>(J, s, ev)); break;
    }
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(ev[6]));
    float ms;
    for (int k = 0; k < 4; k++) {
      CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      stage_ms[k] += ms;
    }
    CK(cudaEventElapsedTime(&ms, ev[4], ev[6]));
    stage_ms[4] += ms;
    CK(cudaEventElapsedTime(&ms, ev[0], ev[6]));
    stage_ms[5] += ms;
    CK(cudaEventElapsedTime(&ms, ev[4], ev[5]));
    stage_ms[6] += ms;
    CK(cudaEventElapsedTime(&ms, ev[5], ev[6]));
    stage_ms[7] += ms;
  }
  for (int i = 0; i < 7; i++) cudaEventDestroy(ev[i]);
  return SGT_OK;
}

extern "C" {

// ---------------------------------------------------------------------------
// operators
// ---------------------------------------------------------------------------
sgt_status sgt_repulsive(sgt_ctx *ctx, int n, int d, float h, int ng_fixed, const float *y,
                         int layout, float *f, double *zeta, int *grid_points, float *h_eff) {
  if (!ctx || !y || !f) return SGT_ERR_INVALID_ARG;
  if (n < 2 || d < 1 || d > 3) return fail(ctx, SGT_ERR_INVALID_ARG, "need n >= 2 and 1 <= d <= 3");
  CK(cudaSetDevice(ctx->device));
  CKS(ensure_scratch(ctx, n, d, ng_fixed > 0 ? SGT_GRID_FIXED : SGT_GRID_H, ng_fixed, h));
  sgt_job *J = ctx->scratch;
  cudaStream_t s = ctx->stream;
  CK(cudaMemsetAsync(J->st, 0, sizeof(SgtState), s));
  CKS(pack_y(J, y, layout, J->Ynext, s));
  CKS(init_stats(J, s, 0));
  switch (d) {
    case 1: CKS(enqueue_repulsion<1>(J, s)); break;
    case 2: CKS(enqueue_repulsion<2>(J, s)); break;
    default: CKS(enqueue_repulsion<3>(J, s)); break;
  }
  const int nb = grid_blocks(ctx->nsm, 4);
  const int dm = layout == SGT_LAYOUT_DIM_MAJOR;
  switch (d) {
    case 1: k_unpack_divz<1><<<nb, SGT_THREADS, 0, s>>>((const float *)J->Frep, n, dm, J->st, f); break;
    case 2: k_unpack_divz<2><<<nb, SGT_THREADS, 0, s>>>((const float2 *)J->Frep, n, dm, J->st, f); break;
    default: k_unpack_divz<3><<<nb, SGT_THREADS, 0, s>>>((const float4 *)J->Frep, n, dm, J->st, f); break;
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(J->st_host, J->st, sizeof(SgtState), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (zeta) *zeta = J->st_host->Z;
  if (grid_points) *grid_points = J->st_host->N;
  if (h_eff) *h_eff = J->st_host->h_eff;
  ctx->last_N = J->st_host->N;
  ctx->last_d = d;
  return flag_status(ctx, J->st_host->error, J->st_host->N, "sgt_repulsive");
}

sgt_status sgt_bins(sgt_ctx *ctx, int n, int d, float h, int ng_fixed, const float *y, int layout,
                    uint32_t *bins, int *grid_points) {
  if (!ctx || !y || !bins) return SGT_ERR_INVALID_ARG;
  if (n < 2 || d < 1 || d > 3) return fail(ctx, SGT_ERR_INVALID_ARG, "need n >= 2 and 1 <= d <= 3");
  CK(cudaSetDevice(ctx->device));
  CKS(ensure_scratch(ctx, n, d, ng_fixed > 0 ? SGT_GRID_FIXED : SGT_GRID_H, ng_fixed, h));
  sgt_job *J = ctx->scratch;
  cudaStream_t s = ctx->stream;
  CK(cudaMemsetAsync(J->st, 0, sizeof(SgtState), s));
  CKS(pack_y(J, y, layout, J->Ynext, s));
  CKS(init_stats(J, s, 0));
  const int nb = grid_blocks(ctx->nsm, 4);
  switch (d) {
    case 1: k_write_bins<1><<<nb, SGT_THREADS, 0, s>>>((const float *)J->Ynext, n, J->st, bins); break;
    case 2: k_write_bins<2><<<nb, SGT_THREADS, 0, s>>>((const float2 *)J->Ynext, n, J->st, bins); break;
    default: k_write_bins<3><<<nb, SGT_THREADS, 0, s>>>((const float4 *)J->Ynext, n, J->st, bins); break;
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(J->st_host, J->st, sizeof(SgtState), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (grid_points) *grid_points = J->st_host->N;
  return SGT_OK;
}

sgt_status sgt_last_grids(sgt_ctx *ctx, float *v_grid, float *phi_grid) {
  if (!ctx || !ctx->scratch || ctx->last_N <= 0) return fail(ctx, SGT_ERR_INVALID_ARG, "no grids yet");
  CK(cudaSetDevice(ctx->device));
  sgt_job *J = ctx->scratch;
  const int d = ctx->last_d, N = ctx->last_N, m = d + 1, nc = d == 1 ? 2 : 4;
  size_t nodes = N;
  if (d >= 2) nodes *= N;
  if (d >= 3) nodes *= N;
  std::vector<float> tmp(nodes * nc);
  float *outs[2] = {v_grid, phi_grid};
  const float *srcs[2] = {J->V, J->Phi};
  for (int q = 0; q < 2; q++) {
    if (!outs[q]) continue;
    CK(cudaMemcpyAsync(tmp.data(), srcs[q], sizeof(float) * tmp.size(), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (size_t g = 0; g < nodes; g++)
      for (int c = 0; c < m; c++) outs[q][c * nodes + g] = tmp[g * nc + c];
  }
  return SGT_OK;
}

sgt_status sgt_attractive(sgt_ctx *ctx, int format, int n, int d, long nnz, const int *rowptr,
                          const unsigned *coo_rows, const int *col, const float *val,
                          const float *y, int layout, float *f) {
  if (!ctx || !col || !val || !y || !f || n < 1 || nnz < 0 || d < 1 || d > 3)
    return SGT_ERR_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  sgt_params p;
  sgt_params_default(&p);
  p.d = d;
  p.format = format;
  sgt_job tmp;  // holds temporary device buffers only
  tmp.ctx = ctx;
  tmp.d = d;
  tmp.n = n;
  tmp.S = d == 3 ? 4 : d;
  const int S = tmp.S;
  sgt_status st = SGT_OK;
  auto cleanup = [&]() { for (void *q : tmp.allocs) cudaFreeAsync(q, s); tmp.allocs.clear(); };
  float *Yp = nullptr, *Fp = nullptr;
  if ((st = jalloc(&tmp, &Yp, (size_t)n * S)) != SGT_OK || (st = jalloc(&tmp, &Fp, (size_t)n * S)) != SGT_OK) {
    cleanup();
    return st;
  }
  tmp.Y = Yp;
  st = pack_y(&tmp, y, layout, Yp, s);
  const int nb = grid_blocks(ctx->nsm, 8);
  const int G = choose_group(nnz, n);
  if (st == SGT_OK && format == SGT_FORMAT_CSR) {
    if (!rowptr) { cleanup(); return SGT_ERR_INVALID_ARG; }
    int2 *pairs = nullptr;
    if ((st = jalloc(&tmp, &pairs, (size_t)nnz)) == SGT_OK) {
      k_pack_pairs<<<nb, SGT_THREADS, 0, s>>>(nnz, col, val, pairs);
      switch (d * 100 + G) {
#define ATC(DD, GG) case DD * 100 + GG: k_attr_csr<DD, GG><<<nb, SGT_THREADS, 0, s>>>(rowptr, pairs, (const typename Vec<DD>::T *)Yp, (typename Vec<DD>::T *)Fp, n); break;
        ATC(1, 4) ATC(1, 8) ATC(1, 16) ATC(1, 32)
        ATC(2, 4) ATC(2, 8) ATC(2, 16) ATC(2, 32)
        ATC(3, 4) ATC(3, 8) ATC(3, 16) ATC(3, 32)
#undef ATC
      }
    }
  } else if (st == SGT_OK && format == SGT_FORMAT_COO) {
    if (!coo_rows) { cleanup(); return SGT_ERR_INVALID_ARG; }
    cudaMemsetAsync(Fp, 0, sizeof(float) * (size_t)n * S, s);
    switch (d) {
      case 1: k_attr_coo<1><<<nb, SGT_THREADS, 0, s>>>(nnz, coo_rows, (const unsigned *)col, val, (const float *)Yp, Fp); break;
      case 2: k_attr_coo<2><<<nb, SGT_THREADS, 0, s>>>(nnz, coo_rows, (const unsigned *)col, val, (const float2 *)Yp, Fp); break;
      default: k_attr_coo<3><<<nb, SGT_THREADS, 0, s>>>(nnz, coo_rows, (const unsigned *)col, val, (const float4 *)Yp, Fp); break;
    }
  } else if (st == SGT_OK && format == SGT_FORMAT_HYBRID) {
    if (!rowptr) { cleanup(); return SGT_ERR_INVALID_ARG; }
    std::vector<int> hrp(n + 1), hc(nnz);
    std::vector<float> hv(nnz);
    cudaMemcpyAsync(hrp.data(), rowptr, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hc.data(), col, sizeof(int) * nnz, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hv.data(), val, sizeof(float) * nnz, cudaMemcpyDeviceToHost, s);
    CK(cudaStreamSynchronize(s));
    const int w = sgt_ell_width(n, hrp.data());
    std::vector<unsigned> ec((size_t)n * std::max(w, 1)), cr(std::max(nnz, 1L)), cc(std::max(nnz, 1L));
    std::vector<float> ev((size_t)n * std::max(w, 1)), cv(std::max(nnz, 1L));
    long csz = 0;
    sgt_csr_to_hybrid(n, hrp.data(), hc.data(), hv.data(), w, ec.data(), ev.data(), cr.data(), cc.data(), cv.data(), &csz);
    unsigned *dec, *dcr, *dcc;
    float *dev_, *dcv;
    if ((st = jalloc(&tmp, &dec, ec.size())) == SGT_OK && (st = jalloc(&tmp, &dev_, ev.size())) == SGT_OK &&
        (st = jalloc(&tmp, &dcr, cr.size())) == SGT_OK && (st = jalloc(&tmp, &dcc, cc.size())) == SGT_OK &&
        (st = jalloc(&tmp, &dcv, cv.size())) == SGT_OK) {
      cudaMemcpyAsync(dec, ec.data(), sizeof(unsigned) * ec.size(), cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(dev_, ev.data(), sizeof(float) * ev.size(), cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(dcr, cr.data(), sizeof(unsigned) * cr.size(), cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(dcc, cc.data(), sizeof(unsigned) * cc.size(), cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(dcv, cv.data(), sizeof(float) * cv.size(), cudaMemcpyHostToDevice, s);
      switch (d) {
        case 1: k_attr_ell<1><<<nb, SGT_THREADS, 0, s>>>(n, w, dec, dev_, (const float *)Yp, (float *)Fp);
                if (csz) k_attr_coo<1><<<nb, SGT_THREADS, 0, s>>>(csz, dcr, dcc, dcv, (const float *)Yp, Fp); break;
        case 2: k_attr_ell<2><<<nb, SGT_THREADS, 0, s>>>(n, w, dec, dev_, (const float2 *)Yp, (float2 *)Fp);
                if (csz) k_attr_coo<2><<<nb, SGT_THREADS, 0, s>>>(csz, dcr, dcc, dcv, (const float2 *)Yp, Fp); break;
        default: k_attr_ell<3><<<nb, SGT_THREADS, 0, s>>>(n, w, dec, dev_, (const float4 *)Yp, (float4 *)Fp);
                 if (csz) k_attr_coo<3><<<nb, SGT_THREADS, 0, s>>>(csz, dcr, dcc, dcv, (const float4 *)Yp, Fp); break;
      }
      CK(cudaStreamSynchronize(s));
    }
  } else if (st == SGT_OK) {
    cleanup();
    return fail(ctx, SGT_ERR_UNSUPPORTED, "unknown format");
  }
  if (st == SGT_OK) {
    const int dm = layout == SGT_LAYOUT_DIM_MAJOR;
    switch (d) {
      case 1: k_unpack<1><<<nb, SGT_THREADS, 0, s>>>((const float *)Fp, n, dm, 1.0f, nullptr, f); break;
      case 2: k_unpack<2><<<nb, SGT_THREADS, 0, s>>>((const float2 *)Fp, n, dm, 1.0f, nullptr, f); break;
      default: k_unpack<3><<<nb, SGT_THREADS, 0, s>>>((const float4 *)Fp, n, dm, 1.0f, nullptr, f); break;
    }
    if (cudaGetLastError() != cudaSuccess) st = fail(ctx, SGT_ERR_CUDA, "attractive kernels");
    else if (cudaStreamSynchronize(s) != cudaSuccess) st = fail(ctx, SGT_ERR_CUDA, "attractive sync");
  }
  cleanup();
  return st;
}

sgt_status sgt_kl(sgt_ctx *ctx, int n, int d, long nnz, const int *rowptr, const int *col,
                  const float *val, const float *y, int layout, double alpha, double zeta,
                  double *kl) {
  if (!ctx || !rowptr || !col || !val || !y || !kl || n < 1 || d < 1 || d > 3)
    return SGT_ERR_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  sgt_job tmp;
  tmp.ctx = ctx;
  tmp.d = d;
  tmp.n = n;
  tmp.S = d == 3 ? 4 : d;
  sgt_status st;
  auto cleanup = [&]() { for (void *q : tmp.allocs) cudaFreeAsync(q, s); tmp.allocs.clear(); };
  float *Yp;
  int2 *pairs;
  SgtState *sd;
  double *part;
  const int nb = grid_blocks(ctx->nsm, 8);
  if ((st = jalloc(&tmp, &Yp, (size_t)n * tmp.S)) != SGT_OK || (st = jalloc(&tmp, &pairs, (size_t)nnz)) != SGT_OK ||
      (st = jalloc(&tmp, &sd, 1)) != SGT_OK || (st = jalloc(&tmp, &part, (size_t)nb)) != SGT_OK) {
    cleanup();
    return st;
  }
  SgtState h;
  memset(&h, 0, sizeof(h));
  h.Z = zeta;
  cudaMemcpyAsync(sd, &h, sizeof(h), cudaMemcpyHostToDevice, s);
  st = pack_y(&tmp, y, layout, Yp, s);
  k_pack_pairs<<<nb, SGT_THREADS, 0, s>>>(nnz, col, val, pairs);
  const int G = choose_group(nnz, n);
  switch (d * 100 + G) {
#define KLO(DD, GG) case DD * 100 + GG: k_kl<DD, GG><<<nb, SGT_THREADS, 0, s>>>(rowptr, pairs, (const typename Vec<DD>::T *)Yp, sd, alpha, part, n); break;
    KLO(1, 4) KLO(1, 8) KLO(1, 16) KLO(1, 32)
    KLO(2, 4) KLO(2, 8) KLO(2, 16) KLO(2, 32)
    KLO(3, 4) KLO(3, 8) KLO(3, 16) KLO(3, 32)
#undef KLO
  }
  if (cudaGetLastError() != cudaSuccess) {
    cleanup();
    return fail(ctx, SGT_ERR_CUDA, "kl kernel");
  }
  cudaMemcpyAsync(&h, sd, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    cleanup();
    return fail(ctx, SGT_ERR_CUDA, "kl sync");
  }
  *kl = h.kl;
  cleanup();
  return st;
}

sgt_status sgt_lambda_bisect(sgt_ctx *ctx, int n, const int *rowptr, float *val, float lambda,
                             int dist, float *sigma) {
  if (!ctx || !rowptr || !val || n < 1) return SGT_ERR_INVALID_ARG;
  if (dist < 0 || dist > 2)
    return fail(ctx, SGT_ERR_INVALID_ARG, "sgt_lambda_bisect: dist must be 0, 1 or 2");
  CK(cudaSetDevice(ctx->device));
  if (dist == 2)
    k_lambda_bisect_cu<<<grid_blocks(ctx->nsm, 8), SGT_THREADS, 0, ctx->stream>>>(
        n, rowptr, val, lambda, sigma);
  else
    k_lambda_bisect<<<grid_blocks(ctx->nsm, 8), SGT_THREADS, 0, ctx->stream>>>(
        n, rowptr, val, (double)lambda, 1e-5, 100, dist, sigma, nullptr);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return SGT_OK;
}

sgt_status sgt_perplexity(sgt_ctx *ctx, int n, int k, const float *dist, float perplexity,
                          float *p, float *beta) {
  if (!ctx || !dist || !p || n < 1 || k < 1) return SGT_ERR_INVALID_ARG;
  if (k > SGT_PERP_MAXK) return fail(ctx, SGT_ERR_UNSUPPORTED, "k > 256");
  CK(cudaSetDevice(ctx->device));
  k_perplexity<<<grid_blocks(ctx->nsm, 8), SGT_THREADS, 0, ctx->stream>>>(
      n, k, dist, (double)perplexity, 1e-5, 200, p, beta);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return SGT_OK;
}

sgt_status sgt_csr_to_coo(sgt_ctx *ctx, int n, long nnz, const int *rowptr, unsigned *rows) {
  if (!ctx || !rowptr || !rows || n < 1 || nnz < 0) return SGT_ERR_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  k_csr_to_coo<<<grid_blocks(ctx->nsm, 8), SGT_THREADS, 0, ctx->stream>>>(n, nnz, rowptr, rows);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return SGT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// library entry: the flow of sgtsneCUDA (CU/sgtsne.cu:25-129)
// ---------------------------------------------------------------------------
// Relative L2 error of the repulsive force of the job's last iteration (the
// numerator left in Frep over that iteration's Z) against the exact O(n^2)
// sum at the same coordinates (Y), as the -f probe (CU/compute_error.cu:
// 80-99) measures it.  Both forces are normalised by their own Z.
template <int D>
static sgt_status job_rep_error(sgt_job *J, double *out) {
  sgt_ctx *ctx = J->ctx;
  cudaStream_t s = ctx->stream;
  typedef typename Vec<D>::T VT;
  const int n = J->n;
  double *num = nullptr, *z = nullptr;
  CK(sgti_alloc(ctx, (void **)&num, sizeof(double) * (size_t)n * D, s));
  CK(sgti_alloc(ctx, (void **)&z, sizeof(double) * (size_t)n, s));
  k_frep_exact<D><<<(n + SGT_THREADS - 1) / SGT_THREADS, SGT_THREADS, 0, s>>>((const VT *)J->Y, n,
                                                                              num, z);
  std::vector<double> hn((size_t)n * D), hz((size_t)n);
  std::vector<float> hf((size_t)n * J->S);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(hn.data(), num, sizeof(double) * hn.size(), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hz.data(), z, sizeof(double) * hz.size(), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hf.data(), J->Frep, sizeof(float) * hf.size(), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(J->st_host, J->st, sizeof(SgtState), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFreeAsync(num, s);
  cudaFreeAsync(z, s);
  CK(e);
  double zx = 0;
  for (int i = 0; i < n; i++) zx += hz[i];
  const double ze = J->st_host->Z;
  double err2 = 0, nrm2 = 0;
  for (int i = 0; i < n; i++)
    for (int k = 0; k < D; k++) {
      const double fx = hn[(size_t)i * D + k] / zx, fe = (double)hf[(size_t)i * J->S + k] / ze;
      err2 += (fx - fe) * (fx - fe);
      nrm2 += fx * fx;
    }
  *out = nrm2 > 0 ? std::sqrt(err2 / nrm2) : 0.0;
  return SGT_OK;
}

extern "C" sgt_status sgt_job_repulsive_error(sgt_job *J, double *rel_err) {
  if (!J || !rel_err) return SGT_ERR_INVALID_ARG;
  sgt_ctx *ctx = J->ctx;
  if (J->host_iter < 1)
    return fail(ctx, SGT_ERR_INVALID_ARG, "the job has not run an iteration since set_y");
  CK(cudaSetDevice(ctx->device));
  switch (J->d) {
    case 1: return job_rep_error<1>(J, rel_err);
    case 2: return job_rep_error<2>(J, rel_err);
    default: return job_rep_error<3>(J, rel_err);
  }
}

extern "C" sgt_status sgt_embed(sgt_ctx *ctx, int n, const int *rowptr, const int *col,
                                const float *val, const sgt_params *params, const float *y_in,
                                float *y_out, double *time_info) {
  if (!ctx || !rowptr || !col || !val || !params || !y_out) return SGT_ERR_INVALID_ARG;
  if (n < 2) return fail(ctx, SGT_ERR_INVALID_ARG, "need at least 2 points");
  sgt_params p = *params;
  p.n = n;
  if (p.d < 1 || p.d > 3) return fail(ctx, SGT_ERR_UNSUPPORTED, "d must be 1, 2 or 3");
  // default h per dimension (CU/sgtsne.cu:29-40)
  if (p.h <= 0) p.h = p.d == 1 ? 0.5f : (p.d == 2 ? 0.7f : 1.2f);
  CK(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const auto t0 = std::chrono::steady_clock::now();
  // rowptr on the host (the lambda bisection reads rows by it); the column
  // indices are checked on the device by the symmetrisation, which rejects
  // any outside [0, n) before anything reads through them
  if (rowptr[0] != 0) return fail(ctx, SGT_ERR_INVALID_ARG, "rowptr[0] != 0");
  for (int i = 0; i < n; i++)
    if (rowptr[i + 1] < rowptr[i])
      return fail(ctx, SGT_ERR_INVALID_ARG, "rowptr not monotone at row " + std::to_string(i));
  const long nnz = rowptr[n];
  // P prepared on the device: lambda rescaling unless lambda == 1
  // (CU/sgtsne.cu:51-54), leaves dropped, (P + P^T)/(2n) (CU/sgtsne.cu:64-65)
  int *drp = nullptr, *dc = nullptr, *srp = nullptr, *sc = nullptr;
  float *dv = nullptr, *sv = nullptr;
  auto release = [&]() {
    for (void *q : {(void *)drp, (void *)dc, (void *)dv, (void *)srp, (void *)sc, (void *)sv})
      if (q) cudaFreeAsync(q, s);
  };
  cudaError_t ae = sgti_alloc(ctx, (void **)&drp, sizeof(int) * ((size_t)n + 1), s);
  if (ae == cudaSuccess) ae = sgti_alloc(ctx, (void **)&dc, sizeof(int) * (size_t)std::max(nnz, 1L), s);
  if (ae == cudaSuccess) ae = sgti_alloc(ctx, (void **)&dv, sizeof(float) * (size_t)std::max(nnz, 1L), s);
  if (ae == cudaSuccess) ae = sgti_alloc(ctx, (void **)&srp, sizeof(int) * ((size_t)n + 1), s);
  if (ae == cudaSuccess) ae = sgti_alloc(ctx, (void **)&sc, sizeof(int) * (size_t)std::max(2 * nnz, 1L), s);
  if (ae == cudaSuccess) ae = sgti_alloc(ctx, (void **)&sv, sizeof(float) * (size_t)std::max(2 * nnz, 1L), s);
  if (ae == cudaSuccess) ae = cudaMemcpyAsync(drp, rowptr, sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice, s);
  if (ae == cudaSuccess) ae = cudaMemcpyAsync(dc, col, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice, s);
  if (ae == cudaSuccess) ae = cudaMemcpyAsync(dv, val, sizeof(float) * (size_t)nnz, cudaMemcpyHostToDevice, s);
  if (ae != cudaSuccess) {
    release();
    return fail(ctx, ae == cudaErrorMemoryAllocation ? SGT_ERR_NO_MEMORY : SGT_ERR_CUDA,
                std::string("sgt_embed: staging P: ") + cudaGetErrorString(ae));
  }
  sgt_status ps = SGT_OK;
  if (p.lambda != 1.0f) {
    ps = sgt_lambda_bisect(ctx, n, drp, dv, p.lambda, p.lambda_dist, nullptr);
    if (ps == SGT_OK && p.drop_leaf) {
      k_drop_leaf<<<grid_blocks(ctx->nsm, 4), SGT_THREADS, 0, s>>>(n, drp, dv);
      if (cudaGetLastError() != cudaSuccess) ps = fail(ctx, SGT_ERR_CUDA, "sgt_embed: drop leaves");
    }
  }
  long snnz = 0;
  if (ps == SGT_OK)
    ps = sgt_symmetrize_device(ctx, n, nnz, drp, dc, dv, 1.0f / (2.0f * n), srp, sc, sv, &snnz);
  sgt_job *J = nullptr;
  if (ps == SGT_OK) ps = sgt_job_create(ctx, &p, n, srp, sc, sv, 1, &J);
  release();
  if (ps != SGT_OK) return ps;
  // initial coordinates: given, or 1e-4 N(0,1) as generateRandomGaussianCoord
  // (CU/utils.cu:185-193), dim-major
  std::vector<float> y0;
  const float *ysrc = y_in;
  if (!ysrc) {
    y0.resize((size_t)n * p.d);
    std::default_random_engine gen;
    if (p.seed) gen.seed((unsigned long)p.seed);
    std::normal_distribution<float> dist(0.0, 1.0);
    for (size_t i = 0; i < y0.size(); i++) y0[i] = 0.0001 * dist(gen);
    ysrc = y0.data();
  }
  sgt_status st = sgt_job_set_y(J, ysrc, SGT_LAYOUT_DIM_MAJOR, 0);
  const auto t1 = std::chrono::steady_clock::now();
  std::vector<double> errs;
  if (st == SGT_OK && p.compute_error > 0) {
    // every 10th iteration (0, 10, 20, ...) the error of its repulsive force
    // against the exact sum (CU/gradient_descend.cu:203-213)
    for (int it = 0; it < p.max_iter && st == SGT_OK;) {
      if (it % 10 == 0) {
        st = time_info ? sgt_job_run_timed(J, 1, time_info) : sgt_job_run(J, 1);
        double e = 0;
        if (st == SGT_OK) st = sgt_job_repulsive_error(J, &e);
        errs.push_back(e);
        it++;
      } else {
        const int k = std::min(10 - it % 10, p.max_iter - it);
        st = time_info ? sgt_job_run_timed(J, k, time_info) : sgt_job_run(J, k);
        it += k;
      }
    }
  } else if (st == SGT_OK) {
    // with time_info, every iteration's stage times as the reference
    // records them (stage by stage; the SpMV no longer overlaps the
    // repulsion), else the captured graphs
    st = time_info ? sgt_job_run_timed(J, p.max_iter, time_info) : sgt_job_run(J, p.max_iter);
  }
  if (st == SGT_OK) st = sgt_job_get_y(J, y_out, SGT_LAYOUT_DIM_MAJOR, 0, 1);
  const auto t2 = std::chrono::steady_clock::now();
  if (st == SGT_OK && time_info) {
    // as the reference: [7000] the gradient descent (CU/gradient_descend.cu:
    // 247), [7001] the preparation of P (CU/sgtsne.cu:98), [7002] the whole
    // call (the demo's total, demo_perplexity.cu:201); the per-iteration
    // stage times [7 i + j] were written by sgt_job_run_timed
    time_info[7000] = std::chrono::duration<double, std::milli>(t2 - t1).count();
    time_info[7001] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    time_info[7002] = std::chrono::duration<double, std::milli>(t2 - t0).count();
  }
  if (st == SGT_OK) {
    sgt_job_info info;
    st = sgt_job_get_info(J, &info);
    if (st == SGT_OK) st = flag_status(ctx, info.error_flags, info.grid_points, "sgt_embed");
  }
  if (st == SGT_OK && p.compute_error > 0) {
    // appended to errorInfo.txt in the working directory, one line per run,
    // as the reference does (CU/gradient_descend.cu:254-266; the reference
    // writes the values only when the file already exists, this engine
    // always writes them)
    FILE *f = fopen("errorInfo.txt", "a");
    if (!f) {
      st = fail(ctx, SGT_ERR_INVALID_ARG, "cannot append to errorInfo.txt");
    } else {
      for (double e : errs) fprintf(f, "%g ", e);
      fprintf(f, "\n");
      fclose(f);
    }
  }
  sgt_job_destroy(J);
  return st;
}

// ---------------------------------------------------------------------------
// Interpolated repulsion without device allocation.
//
// For callers that may not allocate device memory at all: applications whose
// own pool allocator has reserved the whole device (a cudaMalloc would fail
// or fragment their pool), and latency-sensitive loops where a cudaMalloc /
// cudaFree pair would stall on device synchronisation.  All scratch lives in
// one file-scope __device__ array, held by every GPU that loads this library
// until the process exits.  Limits: n <= SGT_NA_MAX_N points, d = 1 or 2,
// grids up to 128 points per axis in 2-D (512 in 1-D).
// ---------------------------------------------------------------------------
#include <cuda.h>  // CUcontext / CUresult of the two driver entry points below
#include <mutex>

namespace {
constexpr int SGT_NA_MAX_N = 32768;
constexpr int SGT_NA_MAX_GRID_2D = 128;   // points per axis -> FFT length 256
constexpr int SGT_NA_MMAX_2D = 256;
constexpr int SGT_NA_MMAX_1D = 1024;
constexpr int SGT_NA_PARTS = 4096;        // per-block partials of the reductions
constexpr int SGT_NA_CHUNKS = SGT_NA_MAX_N / 1024 + SGT_HIST_MAX + 16;
constexpr size_t na_al(size_t b) { return (b + 255) & ~(size_t)255; }
// byte offsets of every buffer inside the array
constexpr size_t NA_Y = 0;
constexpr size_t NA_YNEXT = NA_Y + na_al((size_t)SGT_NA_MAX_N * 2 * 4);
constexpr size_t NA_FREP = NA_YNEXT + na_al((size_t)SGT_NA_MAX_N * 2 * 4);
constexpr size_t NA_SORTED = NA_FREP + na_al((size_t)SGT_NA_MAX_N * 2 * 4);
constexpr size_t NA_NODES = (size_t)SGT_NA_MAX_GRID_2D * SGT_NA_MAX_GRID_2D;  // >= 512 (1-D)
constexpr size_t NA_V = NA_SORTED + na_al((size_t)SGT_NA_MAX_N * 16);
constexpr size_t NA_PHI = NA_V + na_al(NA_NODES * 16);
constexpr size_t NA_W = NA_PHI + na_al(NA_NODES * 16);
constexpr size_t NA_TILES = NA_W + na_al((size_t)3 * SGT_NA_MMAX_2D * SGT_NA_MMAX_2D * 8);
constexpr size_t NA_CURSOR = NA_TILES + na_al((size_t)SGT_HIST_MAX * 4);
constexpr size_t NA_CHUNKS = NA_CURSOR + na_al((size_t)SGT_HIST_MAX * 4);
constexpr size_t NA_PMIN = NA_CHUNKS + na_al((size_t)SGT_NA_CHUNKS * 16);
constexpr size_t NA_PMAX = NA_PMIN + na_al((size_t)SGT_NA_PARTS * 16);
constexpr size_t NA_PSUM = NA_PMAX + na_al((size_t)SGT_NA_PARTS * 16);
constexpr size_t NA_PZ = NA_PSUM + na_al((size_t)SGT_NA_PARTS * 4 * 8);
constexpr size_t NA_STATE = NA_PZ + na_al((size_t)SGT_NA_PARTS * 8);
constexpr size_t NA_BYTES = NA_STATE + na_al(sizeof(SgtState));
static_assert(NA_BYTES < 8u << 20, "no-alloc scratch stays a few MB");
}  // namespace

// The scratch itself.  In host code this name is only a host-side stand-in;
// kernels receive the device address obtained with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_sgt_noalloc_scratch[NA_BYTES];

// The array's device address is looked up once per device and cached with
// the identity of the CUDA context it was looked up in: after a
// cudaDeviceReset the primary context is a new one, the old address is
// stale, and the next call looks it up again.  The identity comes from the
// driver's cuCtxGetCurrent / cuCtxGetId, reached through the runtime's
// driver entry points (no link against libcuda); without them the address
// is looked up on every call.
typedef CUresult (*PfnCtxGetCurrent)(CUcontext *);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long *);

static unsigned long long current_context_id() {
  static PfnCtxGetCurrent get_current = nullptr;
  static PfnCtxGetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void *f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (PfnCtxGetCurrent)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (PfnCtxGetId)f;
    cudaGetLastError();
  });
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&c) != CUDA_SUCCESS || !c) return 0;
  if (get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

static std::mutex g_na_mutex;
static void *g_na_addr[64];                  // device address of the scratch, per device
static unsigned long long g_na_ctx_id[64];   // context the address belongs to (0: none)

static sgt_status noalloc_scratch(sgt_ctx *ctx, unsigned char **out) {
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (ctx->device < 0 || ctx->device >= 64) return fail(ctx, SGT_ERR_UNSUPPORTED, "device index >= 64");
  // the device is current here (the caller set it), so its primary context
  // is the current one
  const unsigned long long id = current_context_id();
  if (!g_na_addr[ctx->device] || id == 0 || g_na_ctx_id[ctx->device] != id) {
    void *p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_sgt_noalloc_scratch));
    g_na_addr[ctx->device] = p;
    g_na_ctx_id[ctx->device] = id;
  }
  *out = (unsigned char *)g_na_addr[ctx->device];
  return SGT_OK;
}

extern "C" sgt_status sgt_repulsive_noalloc(sgt_ctx *ctx, int n, int d, float h, int ng_fixed,
                                            const float *y, int layout, float *f, double *zeta,
                                            int *grid_points, float *h_eff) {
  if (!ctx || !y || !f) return SGT_ERR_INVALID_ARG;
  if (n < 2 || n > SGT_NA_MAX_N)
    return fail(ctx, SGT_ERR_INVALID_ARG,
                "sgt_repulsive_noalloc: n must be in [2, " + std::to_string(SGT_NA_MAX_N) + "]");
  if (d < 1 || d > 2)
    return fail(ctx, SGT_ERR_INVALID_ARG, "sgt_repulsive_noalloc: d must be 1 or 2");
  if (ng_fixed > 0 && d == 2 && sgt_best_grid_size(ng_fixed) + 2 > SGT_NA_MAX_GRID_2D)
    return fail(ctx, SGT_ERR_INVALID_ARG,
                "sgt_repulsive_noalloc: fixed grid larger than 128 points per axis");
  CK(cudaSetDevice(ctx->device));
  unsigned char *base = nullptr;
  CKS(noalloc_scratch(ctx, &base));
  cudaStream_t s = ctx->stream;
  // a job view over the static scratch (host stack only)
  sgt_job J;
  J.ctx = ctx;
  sgt_params_default(&J.p);
  J.p.d = d;
  J.p.format = SGT_FORMAT_CSR;
  J.n = n;
  J.d = d;
  J.S = d;
  J.G = 8;
  J.p.grid_mode = ng_fixed > 0 ? SGT_GRID_FIXED : SGT_GRID_H;
  fill_jp(&J);
  J.jp.grid_mode = J.p.grid_mode;
  J.jp.n1_fixed = sgt_best_grid_size(ng_fixed > 0 ? ng_fixed : 50);
  J.jp.h = h > 0 ? h : (d == 1 ? 0.5f : 0.7f);
  J.mmax = d == 1 ? SGT_NA_MMAX_1D : SGT_NA_MMAX_2D;
  J.nmax = d == 1 ? 512 : SGT_NA_MAX_GRID_2D;
  J.jp.mmax = J.mmax;
  J.jp.tile_cap = SGT_HIST_MAX;
  J.jp.direct_max = d == 1 ? J.nmax : std::min(SGT_DIRECT_N2, J.nmax);
  J.jp.chunk_cap = SGT_NA_CHUNKS;
  J.Y = (float *)(base + NA_Y);
  J.Ynext = (float *)(base + NA_YNEXT);
  J.Frep = (float *)(base + NA_FREP);
  J.sorted = (float4 *)(base + NA_SORTED);
  J.V = (float *)(base + NA_V);
  J.Phi = (float *)(base + NA_PHI);
  J.W = (float2 *)(base + NA_W);
  J.tile_count = (int *)(base + NA_TILES);
  J.cursor = (int *)(base + NA_CURSOR);
  J.chunks = (int4 *)(base + NA_CHUNKS);
  J.part_min = (float4 *)(base + NA_PMIN);
  J.part_max = (float4 *)(base + NA_PMAX);
  J.part_sum = (double *)(base + NA_PSUM);
  J.part_z = (double *)(base + NA_PZ);
  J.st = (SgtState *)(base + NA_STATE);
  sgt_status stt = d == 1 ? job_shapes<1>(&J) : job_shapes<2>(&J);
  if (stt != SGT_OK) return stt;
  if (std::max(std::max(J.nb_pts, J.nb_s2g), J.nb_g2s) > SGT_NA_PARTS)
    return fail(ctx, SGT_ERR_UNSUPPORTED, "sgt_repulsive_noalloc: too many blocks for the partials");
  // the array keeps the previous call's contents: clear what starts at zero
  CK(cudaMemsetAsync(J.st, 0, sizeof(SgtState), s));
  CK(cudaMemsetAsync(J.tile_count, 0, sizeof(int) * SGT_HIST_MAX, s));
  CKS(pack_y(&J, y, layout, J.Ynext, s));
  CKS(init_stats(&J, s, 0));
  if (d == 1) CKS(enqueue_repulsion<1>(&J, s));
  else CKS(enqueue_repulsion<2>(&J, s));
  const int nb = grid_blocks(ctx->nsm, 4);
  const int dm = layout == SGT_LAYOUT_DIM_MAJOR;
  if (d == 1) k_unpack_divz<1><<<nb, SGT_THREADS, 0, s>>>((const float *)J.Frep, n, dm, J.st, f);
  else k_unpack_divz<2><<<nb, SGT_THREADS, 0, s>>>((const float2 *)J.Frep, n, dm, J.st, f);
  CK(cudaGetLastError());
  SgtState hs;
  CK(cudaMemcpyAsync(&hs, J.st, sizeof(SgtState), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (hs.grid_clamped)
    return fail(ctx, SGT_ERR_INVALID_ARG,
                "sgt_repulsive_noalloc: the embedding needs a grid above 128 points per axis; "
                "use sgt_repulsive");
  if (zeta) *zeta = hs.Z;
  if (grid_points) *grid_points = hs.N;
  if (h_eff) *h_eff = hs.h_eff;
  return flag_status(ctx, hs.error, hs.N, "sgt_repulsive_noalloc");
}

// CSR -> ELL + COO on the device (the device twin of sgt_csr_to_hybrid)
extern "C" sgt_status sgt_csr_to_hybrid_device(sgt_ctx *ctx, int n, const int *rowptr,
                                               const int *col, const float *val, int width,
                                               unsigned *ell_cols, float *ell_vals,
                                               unsigned *coo_rows, unsigned *coo_cols,
                                               float *coo_vals, long *coo_size) {
  if (!ctx || n < 1 || width < 0 || !rowptr || !col || !val || !coo_size ||
      !coo_rows || !coo_cols || !coo_vals || (width > 0 && (!ell_cols || !ell_vals)))
    return SGT_ERR_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  std::vector<int> hrp((size_t)n + 1);
  CK(cudaMemcpyAsync(hrp.data(), rowptr, sizeof(int) * ((size_t)n + 1), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (hrp[0] != 0) return fail(ctx, SGT_ERR_INVALID_ARG, "rowptr[0] must be 0");
  for (int r = 0; r < n; r++)
    if (hrp[r + 1] < hrp[r]) return fail(ctx, SGT_ERR_INVALID_ARG, "rowptr must not decrease");
  return hybrid_split_device(ctx, n, hrp, rowptr, col, val, width, ell_cols, ell_vals, coo_rows,
                             coo_cols, coo_vals, coo_size);
}
