// sgt_knn.cu -- exact k nearest neighbours on the device: the kNN stage in
// front of the perplexity equalisation (the reference's command line tool
// calls FLANN, an approximate search, at
// CU/testing_modules/demo_perplexity.cu:131; this search is exact).
// Two methods return the same bits: the SIMT search (k_knn) and, for up to
// 64 dimensions and 32 neighbours, a tensor-core filter (k_knn_tc, further
// down) whose candidates are re-ranked with the SIMT search's arithmetic.
//
// SIMT search: one query per thread, 128 queries per CTA.  Candidates stream through
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
#include "sgt_async.cuh"

#include <algorithm>
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

// query of slot s: the s-th point, or the s-th entry of a query list
__device__ __forceinline__ int knn_query(const int *qlist, int nq, int s) {
  return s < nq ? (qlist ? qlist[s] : s) : -1;
}

// qlist == nullptr: every point is a query (nq == n); otherwise the nq
// points listed are.
__global__ void __launch_bounds__(KNN_Q)
k_knn(const float *__restrict__ X, int n, int dim, int k, const int *__restrict__ qlist, int nq,
      int *__restrict__ idx, float *__restrict__ d2) {
  extern __shared__ float sm[];
  float *sQ = sm;                   // [KNN_Q][KNN_LD]
  float *sC = sm + KNN_Q * KNN_LD;  // [KNN_C][KNN_LD]
  const int t = threadIdx.x;
  const int q0 = blockIdx.x * KNN_Q, q = knn_query(qlist, nq, q0 + t);
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
        const int gq = knn_query(qlist, nq, q0 + r), gk = k0 + cc;
        sQ[r * KNN_LD + cc] = (gq >= 0 && gk < dim) ? X[(long)gq * dim + gk] : 0.f;
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
    if (q >= 0) {
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
  if (q >= 0) {
    for (int s = 0; s < k; s++) {
      idx[(long)q * k + s] = s < cnt ? bi[s] : -1;
      d2[(long)q * k + s] = s < cnt ? bd[s] : INFINITY;
    }
  }
}


// ---------------------------------------------------------------------------
// Tensor-core filter (points of up to 64 dimensions, k up to 32).
//
// Every squared distance is evaluated on the tensor cores as one dot product
// of augmented rows: a query (q, 1, -|q|^2/2) and a candidate
// (c, -|c|^2/2, 1) give q.c - (|q|^2 + |c|^2)/2 = -d^2/2.  The MMAs are of
// kind::tf32 in three terms (hi.hi + hi.lo + lo.hi, where x = hi + lo with
// hi = tf32(x), lo = tf32(x - hi): about 22 bits of each product), FP32
// accumulation in tensor memory.  Each query keeps the KNN_TC_CAP nearest
// candidates under that approximation; the list is then re-ranked with the
// exact arithmetic of k_knn (sums of squared differences in dimension
// order), so returned distances are bit-identical to it.  A query whose list
// could miss a true neighbour -- the list's largest approximate distance
// minus the error bound EPS * (|q|^2 + max |c|^2) not above the k-th exact
// distance -- is redone by k_knn.
//
// Operands: each block of 128 points is stored once, before the search, as
// the image of its shared-memory tile in each role: K-major, no swizzle,
// core matrices of 8 rows x 16 bytes; unit u (4 dimensions) of all 128 rows
// is 2 KB, so the leading-dimension offset (next 4 dimensions) is 2048 B and
// the stride offset (next 8 rows) 128 B.  hi and lo images follow each
// other.  A CTA holds the images of one or two blocks of 128 queries and
// streams candidate images through two or three stages by bulk copies; one
// thread issues the MMAs of each 128 x 128 tile into one of two
// tensor-memory accumulators per query block while that block's four warps
// scan the other (tcgen05.ld, one query row per thread).
//
// Descriptor fields follow the PTX ISA's tcgen05 shared-memory and
// instruction descriptors (the same bit layout as CUTLASS's
// cute::UMMA::SmemDescriptor and UMMA::InstrDescriptor): start address,
// leading and stride byte offsets in 16-byte units, version 1 at bit 46,
// no swizzle; D format F32 at bit 4, A and B formats TF32 (2) at bits 7 and
// 10, both K-major, N/8 at bit 17 and M/16 at bit 24.
constexpr int KNN_TC_M = 128;
constexpr int KNN_TC_MAXK = 32;
constexpr float KNN_TC_EPS = 1e-4f;

__device__ __forceinline__ float tf32_rna(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}
// shared-memory matrix descriptor: K-major, no swizzle
__device__ __forceinline__ unsigned long long umma_desc(unsigned addr, unsigned lbo,
                                                        unsigned sbo) {
  return (unsigned long long)((addr >> 4) & 0x3FFFu) |
         ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void umma_tf32(unsigned dtmem, unsigned long long a,
                                          unsigned long long b, unsigned idesc, unsigned acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(dtmem), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(unsigned bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_ld32(unsigned taddr, float *v) {
  unsigned r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; j++) v[j] = __uint_as_float(r[j]);
}

// hi/lo images of every 128-point block in its two roles ([block][part]
// [unit][row] float4; unused dimensions are zero), and the squared norms
// (FP32, dimension order) with their maximum.  A query row is
// (x, 1, -|x|^2/2) and a candidate row (x, -|x|^2/2, 1) in dimensions
// dim and dim + 1, so one product is q.c - (|q|^2 + |c|^2)/2 = -d^2/2.
// Query rows past n are zero; candidate rows past n are (0, -1e30, 0), at
// distance 2e30 from every query, so they are admitted only while a list is
// not yet full and sort after every real candidate.
__global__ void k_knn_norms(const float *__restrict__ X, int n, int dim, float *__restrict__ nrm,
                            unsigned *__restrict__ nmax) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int kk = 0; kk < dim; kk++) s = fmaf(X[(long)i * dim + kk], X[(long)i * dim + kk], s);
    nrm[i] = s;
    atomicMax(nmax, __float_as_uint(s));  // non-negative floats order as integers
  }
}

__global__ void k_knn_split(const float *__restrict__ X, const float *__restrict__ nrm, int n,
                            int dim, int U, int nblk, float4 *__restrict__ imgA,
                            float4 *__restrict__ imgB) {
  const long total = (long)nblk * U * KNN_TC_M;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const int row = (int)(e % KNN_TC_M);
    const int u = (int)((e / KNN_TC_M) % U);
    const int b = (int)(e / ((long)KNN_TC_M * U));
    const int i = b * KNN_TC_M + row;
    float xa[4], xb[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int kk = 4 * u + c;
      float x = 0.f, ya = 0.f, yb = (i >= n && kk == dim) ? -1e30f : 0.f;
      if (i < n) {
        if (kk < dim) {
          x = X[(long)i * dim + kk];
          ya = yb = x;
        } else if (kk == dim) {
          ya = 1.f;
          yb = -0.5f * nrm[i];
        } else if (kk == dim + 1) {
          ya = -0.5f * nrm[i];
          yb = 1.f;
        }
      }
      xa[c] = ya;
      xb[c] = yb;
    }
    float ha[4], la[4], hb[4], lb[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
      ha[c] = tf32_rna(xa[c]);
      la[c] = tf32_rna(xa[c] - ha[c]);
      hb[c] = tf32_rna(xb[c]);
      lb[c] = tf32_rna(xb[c] - hb[c]);
    }
    const long base = (long)b * 2 * U * KNN_TC_M;
    const long oh = base + (long)u * KNN_TC_M + row, ol = base + (long)(U + u) * KNN_TC_M + row;
    imgA[oh] = make_float4(ha[0], ha[1], ha[2], ha[3]);
    imgA[ol] = make_float4(la[0], la[1], la[2], la[3]);
    imgB[oh] = make_float4(hb[0], hb[1], hb[2], hb[3]);
    imgB[ol] = make_float4(lb[0], lb[1], lb[2], lb[3]);
  }
}

// Candidate list of the filter, in registers (every index below is a
// compile-time constant after unrolling): KNN_TC_CAP entries, unordered,
// with the position and value of its largest entry (the admission
// threshold).  Candidates that beat the threshold wait in a per-thread queue;
// when one thread's queue could overflow, the whole warp merges its queues
// at once, so the lists of a warp's 32 queries are updated together rather
// than one query at a time.
constexpr int KNN_TC_CAP = 64;
constexpr int KNN_TC_QMAX = 64;

struct TcList {
  float d[KNN_TC_CAP];
  int j[KNN_TC_CAP];
  float thr;  // largest entry (distance, index) and its slot
  int thi, mp;
  float mthr;  // -thr/2: a tile value v (= -d^2/2) admits its candidate when v > mthr
  __device__ __forceinline__ void init() {
#pragma unroll
    for (int e = 0; e < KNN_TC_CAP; e++) {
      d[e] = INFINITY;
      j[e] = 0x7fffffff;
    }
    thr = INFINITY;
    thi = 0x7fffffff;
    mp = 0;
    mthr = -INFINITY;
  }
  __device__ __forceinline__ void offer(float dd, int jj) {
    if (!knn_less(dd, jj, thr, thi)) return;
#pragma unroll
    for (int e = 0; e < KNN_TC_CAP; e++)
      if (e == mp) {
        d[e] = dd;
        j[e] = jj;
      }
    thr = d[0];
    thi = j[0];
    mp = 0;
#pragma unroll
    for (int e = 1; e < KNN_TC_CAP; e++)
      if (knn_less(thr, thi, d[e], j[e])) {
        thr = d[e];
        thi = j[e];
        mp = e;
      }
    mthr = -0.5f * thr;
  }
};

// One CTA holds QB (1 or 2) blocks of 128 queries: warps 4a..4a+3 own query
// block a, whose two accumulators sit at tensor-memory columns 256a and
// 256a + 128; every candidate tile streamed in serves all of them.
__global__ void __launch_bounds__(2 * KNN_TC_M, 1)
k_knn_tc(const float4 *__restrict__ imgA, const float4 *__restrict__ imgB,
         const float *__restrict__ nrm, const unsigned *__restrict__ nmax,
         const float *__restrict__ X, int n, int dim, int U, int QB, int nstage, int k,
         int *__restrict__ idx, float *__restrict__ d2,
         int *__restrict__ redo, int *__restrict__ nredo, int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) unsigned long long bars[7];  // A full, B full x3, MMA done x2
  __shared__ unsigned tslot;
  __shared__ volatile int abort_flag;
  const int t = threadIdx.x, warp = t >> 5;
  const int nt = (n + KNN_TC_M - 1) / KNN_TC_M;
  const int qb0 = blockIdx.x * QB;           // first query block of the CTA
  const int na = min(QB, nt - qb0);          // query blocks that exist
  const int qa = warp >> 2;                  // this warp's query block
  const int q = (qb0 + qa) * KNN_TC_M + (t & (KNN_TC_M - 1));
  const unsigned tcols = 256u * (unsigned)QB;
  const unsigned ubytes = (unsigned)U * 2048u, pbytes = 2u * ubytes;
  const unsigned sA = smem_u32(smem);
  const unsigned barA = smem_u32(&bars[0]);
  const unsigned barM[2] = {smem_u32(&bars[4]), smem_u32(&bars[5])};
  const char *gA = reinterpret_cast<const char *>(imgA);
  const char *gB = reinterpret_cast<const char *>(imgB);
  if (t == 0) {
    abort_flag = 0;
    for (int b = 0; b < 6; b++) mbar_init(smem_u32(&bars[b]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(&tslot)), "r"(tcols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = tslot;
  // thread 0: copies and MMAs issued and not yet waited for, with the parity
  // of the phase each completes.  Tile ti sits in stage ti % nstage.
  bool cpend[3] = {false, false, false}, mpend[2] = {false, false};
  unsigned cpar[3] = {0, 0, 0}, mpar[2] = {0, 0};
  auto stage_addr = [&](int st) { return sA + (unsigned)(QB + st) * pbytes; };
  auto bar_full = [&](int st) { return smem_u32(&bars[1 + st]); };
  auto load_tile = [&](int ti) {
    const int st = ti % nstage;
    mbar_expect_tx(bar_full(st), pbytes);
    bulk_g2s(stage_addr(st), gB + (size_t)ti * pbytes, pbytes, bar_full(st));
    cpend[st] = true;
    cpar[st] = (unsigned)((ti / nstage) & 1);
  };
  if (t == 0) {
    mbar_expect_tx(barA, (unsigned)na * pbytes);
    for (int a = 0; a < na; a++)
      bulk_g2s(sA + (unsigned)a * pbytes, gA + (size_t)(qb0 + a) * pbytes, pbytes, barA);
    for (int ti = 0; ti < nstage && ti < nt; ti++) load_tile(ti);
  }
  // D = A B^T: M = 128, N = 128, FP32 accumulate, TF32 A and B, both K-major
  const unsigned idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) |
                         ((128u >> 4) << 24);
  const float qn = q < n ? nrm[q] : 0.f;
  TcList L;
  L.init();
  if (q >= n) {  // admits nothing
    L.thr = -INFINITY;
    L.mthr = INFINITY;
  }
  // queue of candidates that beat the threshold (local memory, written
  // rarely): drained, by the whole warp at once, once a thread could
  // overflow it during the next 32 columns
  float qd[KNN_TC_QMAX];
  int qi[KNN_TC_QMAX];
  int qc = 0;
  bool ok = true;
  for (int it = 0; it <= nt; it++) {
    if (it < nt && t == 0 && ok) {  // MMAs of tile it into accumulator it & 1
      const int st = it % nstage, s = it & 1;
      if (it == 0) ok = mbar_wait(barA, 0);
      if (ok) ok = mbar_wait(bar_full(st), (unsigned)((it / nstage) & 1));
      if (ok) {
        cpend[st] = false;
        tc_fence_after();
        const unsigned sb = stage_addr(st);
        // the start address is the descriptor's low field: a K step of
        // 4096 B adds 256
        const unsigned long long bh = umma_desc(sb, 2048, 128);
        const unsigned long long bl = umma_desc(sb + ubytes, 2048, 128);
        for (int a = 0; a < na; a++) {
          const unsigned dt = tmem + 256u * (unsigned)a + (unsigned)s * 128u;
          const unsigned long long ah = umma_desc(sA + (unsigned)a * pbytes, 2048, 128);
          const unsigned long long al = umma_desc(sA + (unsigned)a * pbytes + ubytes, 2048, 128);
          for (int ks = 0; ks < U / 2; ks++) {
            const unsigned long long o = (unsigned long long)ks * 256u;
            umma_tf32(dt, ah + o, bh + o, idesc, ks > 0 ? 1u : 0u);
            umma_tf32(dt, ah + o, bl + o, idesc, 1u);
            umma_tf32(dt, al + o, bh + o, idesc, 1u);
          }
        }
        umma_commit(barM[s]);
        mpend[s] = true;
        mpar[s] = (unsigned)((it >> 1) & 1);
      }
      if (!ok) abort_flag = 1;
    }
    if (it >= 1) {  // scan tile it - 1
      const int pt = it - 1, s = pt & 1;
      // warp-uniform decisions: tcgen05.ld is executed by whole warps
      bool go = __all_sync(0xffffffffu, ok && !abort_flag);
      if (go) {
        go = __all_sync(0xffffffffu, mbar_wait(barM[s], (unsigned)((pt >> 1) & 1)));
        if (!go) {
          ok = false;
          abort_flag = 1;
        }
      }
      __syncwarp();
      if (go) {
        tc_fence_after();
        if (t == 0) {
          mpend[s] = false;
          // the MMAs of tile pt are done with their stage: refill it
          if (pt + nstage < nt) load_tile(pt + nstage);
        }
      }
      if (go && qa < na) {
#pragma unroll 1
        for (int c0 = 0; c0 < 128; c0 += 32) {
          float v[32];
          __syncwarp();  // converged for the warp-wide tcgen05.ld
          tmem_ld32(tmem + ((unsigned)((warp & 3) * 32) << 16) + 256u * (unsigned)qa +
                        (unsigned)s * 128u + (unsigned)c0,
                    v);
          const int j0 = pt * KNN_TC_M + c0;
          // admission: -2 v < thr, i.e. v > -thr/2 (exact in FP32); the
          // query itself is admitted too and dropped at the re-rank
          const float m = L.mthr;
          bool any = false;
#pragma unroll
          for (int h = 0; h < 32; h++) any |= v[h] > m;
          if (any) {
#pragma unroll
            for (int h = 0; h < 32; h++)
              if (v[h] > m) {
                qd[qc] = -2.f * v[h];
                qi[qc] = j0 + h;
                qc++;
              }
          }
          if (__any_sync(0xffffffffu, qc > KNN_TC_QMAX - 32)) {
#pragma unroll 1
            for (int e = 0; e < qc; e++) L.offer(qd[e], qi[e]);
            qc = 0;
          }
        }
      }
      tc_fence_before();
      if (__syncthreads_or(!ok || abort_flag)) {  // block-uniform
        ok = false;
        break;
      }
    }
  }
#pragma unroll 1
  for (int e = 0; e < qc; e++) L.offer(qd[e], qi[e]);
  if (!ok) {
    if (t == 0) {
      atomicExch(err, 1);
      // let the copies and MMAs in flight finish before the memory is released
      for (int st = 0; st < 3; st++)
        if (cpend[st]) mbar_wait(bar_full(st), cpar[st]);
      for (int s = 0; s < 2; s++)
        if (mpend[s]) mbar_wait(barM[s], mpar[s]);
    }
  } else if (q < n) {
    // exact re-rank with the arithmetic of k_knn, then a sort by (distance,
    // index); unused slots keep (inf, INT_MAX) and sort last
    // a list that never filled holds every candidate
    const float tail = L.thr;
    const bool full = L.thr != INFINITY;
    const float *xq = X + (long)q * dim;
#pragma unroll
    for (int e = 0; e < KNN_TC_CAP; e++) {
      if (L.j[e] >= n || L.j[e] == q) {  // empty slot, padding row or the query itself
        L.d[e] = INFINITY;
        L.j[e] = 0x7fffffff;
        continue;
      }
      const float *xc = X + (long)L.j[e] * dim;
      float a = 0.f;
      for (int kk = 0; kk < dim; kk++) {
        const float df = __ldg(&xq[kk]) - __ldg(&xc[kk]);
        a = fmaf(df, df, a);
      }
      L.d[e] = a;
    }
#pragma unroll
    for (int size = 2; size <= KNN_TC_CAP; size <<= 1)
#pragma unroll
      for (int stride = size >> 1; stride > 0; stride >>= 1)
#pragma unroll
        for (int e = 0; e < KNN_TC_CAP; e++) {
          const int l = e ^ stride;
          if (l > e) {
            const bool up = (e & size) == 0;
            if (up == knn_less(L.d[l], L.j[l], L.d[e], L.j[e])) {
              const float td = L.d[e];
              const int tj = L.j[e];
              L.d[e] = L.d[l];
              L.j[e] = L.j[l];
              L.d[l] = td;
              L.j[l] = tj;
            }
          }
        }
    float dk = L.d[0];
#pragma unroll
    for (int e = 0; e < KNN_TC_CAP; e++)
      if (e == k - 1) dk = L.d[e];
    const float bound = KNN_TC_EPS * (qn + __uint_as_float(*nmax));
    if (!full || tail - bound > dk) {
#pragma unroll
      for (int e = 0; e < KNN_TC_CAP; e++)
        if (e < k) {
          idx[(long)q * k + e] = L.j[e];
          d2[(long)q * k + e] = L.d[e];
        }
    } else {
      redo[atomicAdd(nredo, 1)] = q;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols));
}

}  // namespace

static sgt_status knn_simt(sgt_ctx *ctx, int n, int dim, const float *X, int k,
                           const int *qlist, int nq, int *idx, float *d2) {
  const size_t smem = sizeof(float) * (size_t)(KNN_Q + KNN_C) * KNN_LD;
  cudaError_t e = cudaFuncSetAttribute(k_knn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e == cudaSuccess && nq > 0) {
    const int nb = (nq + KNN_Q - 1) / KNN_Q;
    k_knn<<<nb, KNN_Q, smem, sgti_stream(ctx)>>>(X, n, dim, k, qlist, nq, idx, d2);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess)
    return sgti_fail(ctx, SGT_ERR_CUDA, std::string("sgt_knn: ") + cudaGetErrorString(e));
  return SGT_OK;
}

static sgt_status knn_tc(sgt_ctx *ctx, int n, int dim, const float *X, int k, int *idx,
                         float *d2, int *n_redo) {
  cudaStream_t s = sgti_stream(ctx);
  const int U = ((dim + 2 + 7) / 8) * 2;  // the dimensions and two norm columns
  const int nblk = (n + KNN_TC_M - 1) / KNN_TC_M;
  const size_t img_bytes = (size_t)nblk * 2 * U * 2048;
  const size_t pbytes = (size_t)2 * U * 2048;
  // QB query tiles (two when they fit beside two candidate stages, so each
  // candidate tile streamed in serves 256 queries) and two or three candidate
  // stages; at least 120 KB so that one CTA runs per SM (its tensor-memory
  // columns are then never contended)
  const size_t smem_max = 227 * 1024 - 1024;
  const int QB = 4 * pbytes <= smem_max ? 2 : 1;
  const int nstage = (QB + 3) * pbytes <= smem_max ? 3 : 2;
  const size_t smem = std::max<size_t>((QB + nstage) * pbytes, 120 * 1024);
  char *buf = nullptr;
  const size_t o_nrm = 2 * img_bytes, o_max = o_nrm + sizeof(float) * (size_t)nblk * KNN_TC_M;
  const size_t o_cnt = o_max + 16, o_redo = o_cnt + 16;
  const size_t total = o_redo + sizeof(int) * (size_t)n;
  cudaError_t e = sgti_alloc(ctx, (void **)&buf, total, s);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();  // not sticky: clear it for the caller's next check
    return sgti_fail(ctx, SGT_ERR_NO_MEMORY, "sgt_knn: tensor-core operand images");
  }
  float4 *imgA = reinterpret_cast<float4 *>(buf);
  float4 *imgB = reinterpret_cast<float4 *>(buf + img_bytes);
  float *nrm = reinterpret_cast<float *>(buf + o_nrm);
  unsigned *nmax = reinterpret_cast<unsigned *>(buf + o_max);
  int *cnt = reinterpret_cast<int *>(buf + o_cnt);  // [0] queries to redo, [1] error
  int *redo = reinterpret_cast<int *>(buf + o_redo);
  int hc[2] = {0, 0};
  e = cudaMemsetAsync(buf + o_max, 0, 32, s);
  if (e == cudaSuccess) {
    const long items = (long)nblk * U * KNN_TC_M;
    const int nb = (int)std::min<long>((items + 255) / 256, 148L * 16);
    k_knn_norms<<<(n + 255) / 256, 256, 0, s>>>(X, n, dim, nrm, nmax);
    k_knn_split<<<nb, 256, 0, s>>>(X, nrm, n, dim, U, nblk, imgA, imgB);
    e = cudaFuncSetAttribute(k_knn_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  if (e == cudaSuccess) {
    k_knn_tc<<<(nblk + QB - 1) / QB, KNN_TC_M * QB, smem, s>>>(
        imgA, imgB, nrm, nmax, X, n, dim, U, QB, nstage, k, idx, d2, redo, cnt, cnt + 1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  sgt_status st = SGT_OK;
  if (e != cudaSuccess)
    st = sgti_fail(ctx, SGT_ERR_CUDA, std::string("sgt_knn: ") + cudaGetErrorString(e));
  else if (hc[1])
    st = sgti_fail(ctx, SGT_ERR_CUDA, "sgt_knn: a tensor-core pipeline wait timed out");
  else
    st = knn_simt(ctx, n, dim, X, k, redo, hc[0], idx, d2);  // queries the filter could not settle
  if (st == SGT_OK && n_redo) *n_redo = hc[0];
  cudaFreeAsync(buf, s);
  return st;
}

extern "C" sgt_status sgt_knn_ex(sgt_ctx *ctx, int n, int dim, const float *X, int k, int *idx,
                                 float *d2, int method, int *n_redo) {
  if (!ctx || !X || !idx || !d2) return SGT_ERR_INVALID_ARG;
  if (n < 2 || dim < 1 || k < 1) return sgti_fail(ctx, SGT_ERR_INVALID_ARG, "sgt_knn: sizes");
  if (method < SGT_KNN_AUTO || method > SGT_KNN_TENSOR)
    return sgti_fail(ctx, SGT_ERR_INVALID_ARG, "sgt_knn: method");
  if (k > KNN_MAXK || k >= n)
    return sgti_fail(ctx, SGT_ERR_UNSUPPORTED,
                     "sgt_knn: k must be below n and at most " + std::to_string(KNN_MAXK));
  const bool tc_ok = dim <= 64 && k <= KNN_TC_MAXK && n <= (1 << 28);
  if (method == SGT_KNN_TENSOR && !tc_ok)
    return sgti_fail(ctx, SGT_ERR_UNSUPPORTED,
                     "sgt_knn: the tensor-core filter takes dim <= 64 and k <= 32");
  if (cudaSetDevice(sgti_device(ctx)) != cudaSuccess)
    return sgti_fail(ctx, SGT_ERR_CUDA, "sgt_knn: set device");
  if (n_redo) *n_redo = 0;
  sgt_status st;
  if (method == SGT_KNN_TENSOR || (method == SGT_KNN_AUTO && tc_ok && n >= 4096)) {
    st = knn_tc(ctx, n, dim, X, k, idx, d2, n_redo);
    // the filter's operand images (about 16 bytes per point and dimension)
    // did not fit: the automatic choice falls back to the SIMT search
    if (st == SGT_ERR_NO_MEMORY && method == SGT_KNN_AUTO)
      st = knn_simt(ctx, n, dim, X, k, nullptr, n, idx, d2);
  } else {
    st = knn_simt(ctx, n, dim, X, k, nullptr, n, idx, d2);
  }
  if (st != SGT_OK) return st;
  // like the other preparation operators, return with the result ready
  const cudaError_t e = cudaStreamSynchronize(sgti_stream(ctx));
  if (e != cudaSuccess)
    return sgti_fail(ctx, SGT_ERR_CUDA, std::string("sgt_knn: ") + cudaGetErrorString(e));
  return SGT_OK;
}

extern "C" sgt_status sgt_knn(sgt_ctx *ctx, int n, int dim, const float *X, int k, int *idx,
                              float *d2) {
  return sgt_knn_ex(ctx, n, dim, X, k, idx, d2, SGT_KNN_AUTO, nullptr);
}
