/*
 * sgtsne_b200.h -- C ABI of the B200-native SG-t-SNE gradient engine.
 *
 * Plain pointers and sizes only.  Every entry point returns an sgt_status
 * (never exits the process); sgt_last_error() explains the last failure of a
 * context.  Device pointers must point to memory of the context's device;
 * work is queued on the context's stream and functions that return results
 * to the host synchronise that stream.
 *
 * Each declaration names the reference interface it replaces, by file:line
 * in iakoviid/GPU-SG-SNE (CU = code/cuda/SG-tSNE-CUDA/src).
 */
#ifndef SGTSNE_B200_H
#define SGTSNE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SGT_ABI_VERSION 1

typedef enum {
  SGT_OK = 0,
  SGT_ERR_INVALID_ARG = 1, /* bad size, null pointer, malformed CSR */
  SGT_ERR_CUDA = 2,        /* a CUDA call failed */
  SGT_ERR_NO_MEMORY = 3,   /* device or pinned allocation failed */
  SGT_ERR_UNSUPPORTED = 4, /* option outside what the engine implements */
  SGT_ERR_NUMERIC = 5,     /* non-finite coordinates detected */
  SGT_ERR_NO_DEVICE = 6,   /* no CUDA device */
  SGT_ERR_CAPACITY = 7     /* a device-side capacity was reached: the grid the
                              embedding needs is larger than the one provisioned
                              (max_grid; the step ran on the largest provisioned
                              grid instead) or the S2G guard skipped points.
                              The outputs are written but are not the ones the
                              reference computes; sgt_last_error says which. */
} sgt_status;

/* Storage format of P for the attractive term: the values of the reference
   CLI option -t (CU/testing_modules/demo_perplexity.cu:90-92) plus CSR,
   which is the reference's format 0 (CU/pq.cu:28-30) and this engine's
   fastest path. */
typedef enum {
  SGT_FORMAT_CSR = 0,
  SGT_FORMAT_COO = 2,
  SGT_FORMAT_HYBRID = 3 /* ELL + COO tail */
} sgt_format;

typedef enum {
  SGT_LAYOUT_DIM_MAJOR = 0,  /* y[i + k*n]: the reference CUDA layout */
  SGT_LAYOUT_POINT_MAJOR = 1 /* y[i*d + k]: the reference CPU layout */
} sgt_layout;

typedef enum {
  SGT_GRID_H = 0,    /* grid follows h every iteration, mean-centred
                        (CU/gradient_descend_varGrid.cu:68-186) */
  SGT_GRID_FIXED = 1 /* inner grid getBestGridSize(ng)
                        (CU/gradient_descend.cu:139-140) */
} sgt_grid_mode;

/* Parameters.  The first fourteen fields mirror tsneparams
   (CU/types.hpp:55-72) with its meaning and defaults; the rest are
   additions of this engine. */
typedef struct {
  int d;            /* embedding dimension, 1..3                       */
  float lambda;     /* lambda rescaling target (1 = skip, as the ref.)  */
  float alpha;      /* early exaggeration                               */
  int max_iter;     /* iterations                                       */
  int early_iter;   /* last iteration (inclusive) with alpha            */
  int n;            /* number of points                                 */
  float h;          /* grid spacing; <= 0 picks 0.5/0.7/1.2 for d=1/2/3 */
  int drop_leaf;    /* zero the edge of single-edge rows after lambda   */
  int np;           /* reference worker count; accepted and ignored     */
  int format;       /* sgt_format                                       */
  int bs;           /* reference block size; accepted and ignored       */
  int compute_error;/* > 0: relative L2 error of F_rep every 10 iters   */
  int ng;           /* inner grid size for SGT_GRID_FIXED (default 50)  */
  int sim;          /* reference synthetic-data switch; ignored         */
  /* additions */
  int grid_mode;    /* sgt_grid_mode (default SGT_GRID_H)               */
  int lambda_dist;  /* 1: P values are distances, 0: probabilities,
                       2: distances with the reference GPU kernel's steps
                       (see sgt_lambda_bisect)                          */
  int max_grid;     /* largest grid points per axis to provision
                       (0 = 512 for d <= 2, 128 for d = 3)              */
  int kl_every;     /* > 0: record the KL cost every kl_every iters     */
  uint64_t seed;    /* seed of the random Y0 when y_in is NULL          */
  int relayout_every; /* > 0: relabel points along the Morton order of
                         their grid cells every this many iterations
                         (memory locality of the attractive term; results
                         are returned in the caller's order).  0 = off    */
  int locality_order; /* 1 (default): a CSR job of at least 65,536 points
                         starts from a locality order of its points: the
                         Morton order of a few diffusion steps over P's
                         graph, so the attractive term's gathers stay near
                         each row from the first iteration (results are
                         returned in the caller's order).  0 = off        */
} sgt_params;

/* Fill *p with the reference defaults (d=2, lambda=1, alpha=12,
   max_iter=1000, early_iter=250, h=-1, format=SGT_FORMAT_COO, ng=50);
   relayout_every = 0, locality_order = 1. */
void sgt_params_default(sgt_params *p);

typedef struct sgt_ctx sgt_ctx;
typedef struct sgt_job sgt_job;

int sgt_abi_version(void);
const char *sgt_status_string(sgt_status s);

/* A context owns a stream and a stream-ordered device memory pool: jobs and
   operator calls allocate from it, and memory a retired job frees stays in
   the pool for the next job (no new pages are mapped).  sgt_destroy returns
   the pool's memory to the driver (buffers of jobs still alive are released
   when those jobs are destroyed). */
sgt_status sgt_create(int device, sgt_ctx **out);
void sgt_destroy(sgt_ctx *ctx);
/* Queue all work of ctx on a caller-owned cudaStream_t (NULL = own stream). */
sgt_status sgt_set_stream(sgt_ctx *ctx, void *cuda_stream);
const char *sgt_last_error(const sgt_ctx *ctx);

/* ---- library entry ------------------------------------------------------
 * Replaces sgtsneCUDA<float>(P, params, y_in, timeInfo)
 * (CU/sgtsne.cuh:21-27, CU/sgtsne.cu:25-129).
 * P: host CSR of the kNN graph (n rows, rowptr[n+1], col/val[rowptr[n]]).
 * As the reference: lambda rescaling unless lambda == 1, symmetrisation
 * (P + P^T)/(2n), format preparation, max_iter iterations, final centring.
 * y_in: host, dim-major n*d, or NULL for 1e-4 * N(0,1) from
 * std::default_random_engine (CU/utils.cu:185-193).  y_out: host, dim-major
 * n*d, caller-owned (the reference returned a malloc'd array).
 * time_info: NULL or >= 7003 doubles; as the reference, [7000] = gradient
 * descent ms, [7001] = preparation of P ms, [7002] = whole call ms, and the
 * stage times of iteration i < 1000 in [7 i + j] (the slots of
 * sgt_job_run_timed).  Measuring them runs every iteration stage by stage
 * on one stream, as the reference does, without the overlap of the
 * attractive SpMV and the repulsion that the captured graphs have, so the
 * iterations take longer.  NULL runs the captured graphs. */
sgt_status sgt_embed(sgt_ctx *ctx, int n, const int *rowptr, const int *col,
                     const float *val, const sgt_params *params,
                     const float *y_in, float *y_out, double *time_info);

/* ---- device-resident job (the iteration loop of kl_minimization,
 * CU/gradient_descend.cu:102-282, split so P and Y stay in HBM) ----------
 * P is the already symmetric, normalised CSR (what kl_minimization gets).
 * mem_is_device: 1 if the pointers are device pointers of ctx's device. */
sgt_status sgt_job_create(sgt_ctx *ctx, const sgt_params *params, int n,
                          const int *rowptr, const int *col, const float *val,
                          int mem_is_device, sgt_job **out);
void sgt_job_destroy(sgt_job *job);
/* Set coordinates and reset the schedule (iteration 0, uY = 0, gains = 1). */
sgt_status sgt_job_set_y(sgt_job *job, const float *y, int layout,
                         int mem_is_device);
/* Queue `iters` iterations (captured CUDA graph); asynchronous. */
sgt_status sgt_job_run(sgt_job *job, int iters);
/* sgt_job_run stage by stage on one stream with CUDA events, writing the
   stage times of iteration i (counted from the last sgt_job_set_y; i < 1000)
   into time_info[7 i + j] in the layout of the reference's timeInfo
   (kl_minimization, CU/gradient_descend.cu:53-101, 208-247; CU/Frep.cu:
   81-125; CU/nuconv.cu:37-112): j = 0 attractive term, 1 S2G, 2 G2G, 3 G2S,
   4 forces and update, 5 S2G to G2S, 6 centring, grid decision and binning.
   Synchronises once per iteration; time_info may be NULL. */
sgt_status sgt_job_run_timed(sgt_job *job, int iters, double *time_info);
/* Capture and instantiate the iteration graphs sgt_job_run launches (one
   iteration, and 16 chained iterations) now instead of on first use, so
   that later sgt_job_run calls only launch them.  Runs nothing on the GPU. */
sgt_status sgt_job_prepare(sgt_job *job);
/* Copy the current coordinates out (synchronises).  centre = 1 subtracts the
   mean like the reference does after the last iteration.  Returns
   SGT_ERR_CAPACITY (coordinates still written) when an iteration since the
   last sgt_job_set_y ran on a clamped grid or skipped points in S2G, and
   SGT_ERR_NUMERIC when coordinates became non-finite. */
sgt_status sgt_job_get_y(sgt_job *job, float *y, int layout, int mem_is_device,
                         int centre);
typedef struct {
  int iter;          /* iterations done                          */
  int grid_points;   /* grid points per axis of the last step     */
  float h_eff;       /* grid spacing of the last step             */
  double zeta;       /* Z of the last step                        */
  double kl;         /* last KL value recorded (kl_every > 0)     */
  int error_flags;   /* 1 non-finite, 2 grid clamped, 4 overflow  */
  long nnz;          /* nonzeros of P                             */
  int row_group;     /* lanes per row picked by the autotuner      */
  float tune_ms[4];  /* row kernel ms measured for 4, 8, 16, 32 lanes */
} sgt_job_info;
sgt_status sgt_job_get_info(sgt_job *job, sgt_job_info *info);
/* KL divergence of the current coordinates with the last Z (CU/pq.cu:104-125). */
sgt_status sgt_job_kl(sgt_job *job, double alpha, double *kl);
/* Run `iters` iterations stage by stage on one stream (the captured
   iteration overlaps the attractive SpMV with the repulsion instead), adding
   per-stage milliseconds into stage_ms[8] = {bin, s2g, g2g, g2s,
   attractive+combine, total, attractive SpMV, combine}. */
sgt_status sgt_job_profile(sgt_job *job, int iters, double *stage_ms);
/* Relative L2 error ||F_exact - F|| / ||F_exact|| of the repulsive force of
   the job's last iteration against the exact O(n^2) sum at the same
   coordinates, both normalised by their own Z.  Replaces computeError
   (CU/compute_error.cu:80-99), the probe behind the -f option; costs O(n^2)
   work.  sgt_embed with compute_error > 0 calls it every 10th iteration
   (0, 10, 20, ...) and appends the values to errorInfo.txt in the working
   directory, one line per run (CU/gradient_descend.cu:203-213, 254-266). */
sgt_status sgt_job_repulsive_error(sgt_job *job, double *rel_err);

/* ---- batches: many independent embeddings advanced together -----------
 * No counterpart in the reference, which runs one embedding per process
 * (CU/sgtsne.cu:25-129).  A batch holds jobs of one context.  sgt_batch_run
 * advances every job by the same number of iterations through one CUDA graph
 * whose independent branches are the jobs' iterations (iters_per_launch
 * chained iterations per branch), so the kernels of small embeddings run
 * side by side instead of one job after another.  Jobs keep their own state
 * (sgt_job_get_y, sgt_job_get_info work as usual) and must outlive the batch.
 * Jobs with relayout_every or kl_every set return SGT_ERR_UNSUPPORTED. */
typedef struct sgt_batch sgt_batch;
sgt_status sgt_batch_create(sgt_ctx *ctx, int njobs, sgt_job *const *jobs,
                            int iters_per_launch, sgt_batch **out);
/* Queue `iters` iterations of every job; asynchronous like sgt_job_run.
   When every job holds P in CSR, each stage of an iteration is one launch
   over all jobs of a dimension (blocks mapped to jobs through a table of
   their block counts), so a batch takes about a dozen launches per
   iteration whatever its job count; otherwise the graph has one branch of
   chained iterations per job. */
sgt_status sgt_batch_run(sgt_batch *batch, int iters);
void sgt_batch_destroy(sgt_batch *batch);
/* The same fused launches without a batch object or graph: queue `iters`
   iterations of the given jobs (CSR, no relayout or in-loop KL) on ctx's
   stream, for a set of jobs that changes from call to call.  Jobs may
   belong to other contexts of the same device; their streams must have
   finished the jobs' earlier work (the caller orders them, e.g. with
   events). */
sgt_status sgt_batch_step(sgt_ctx *ctx, int njobs, sgt_job *const *jobs, int iters);

/* ---- one embedding split by rows over ranks (one GPU per rank) ---------
 * No counterpart in the reference, which runs one embedding on one GPU.
 * Rank r holds rows row0 .. row0 + nrows - 1 of P (CSR of those rows,
 * rowptr[0] = 0, column indices over all n_all points), the momentum, gains
 * and forces of those points, and three caller-owned device buffers that
 * the caller's collectives (e.g. NCCL) exchange between the phases of an
 * iteration:
 *   y_all  n_all points x S floats (S = 1, 2, 4 for d = 1, 2, 3): every
 *          point's coordinates; the update phase writes the own rows;
 *   grid   sgt_shard_grid_floats(params) floats: the charge grid;
 *   zsum   one double: Z.
 * One iteration, every rank in the same order:
 *   sgt_shard_scatter   grid decision from all of y_all, S2G of the own
 *                       points into grid, the own rows' attractive SpMV
 *   (all-reduce grid, sum)
 *   sgt_shard_gather    G2G of grid, G2S of the own points, their Z into zsum
 *   (all-reduce zsum, sum)
 *   sgt_shard_update    forces, gains, momentum and coordinates of the own
 *                       rows, written into y_all
 *   (all-gather the own rows of y_all)
 * The phases only queue work on the context's stream (no host
 * synchronisation).  Every rank's sequence of iterations equals the one
 * embedding's: the grid, Z and schedule are global.  CSR only; no relayout
 * or in-loop KL.  Replaces, across GPUs, the loop of kl_minimization
 * (CU/gradient_descend.cu:102-282). */
typedef struct sgt_shard sgt_shard;
size_t sgt_shard_grid_floats(const sgt_params *params);
sgt_status sgt_shard_create(sgt_ctx *ctx, const sgt_params *params, int n_all, int row0,
                            int nrows, const int *rowptr, const int *col, const float *val,
                            int mem_is_device, float *y_all, float *grid, size_t grid_floats,
                            double *zsum, sgt_shard **out);
void sgt_shard_destroy(sgt_shard *shard);
/* All n_all points' coordinates (n_all x d, layout), resets the schedule. */
sgt_status sgt_shard_set_y(sgt_shard *shard, const float *y, int layout, int mem_is_device);
sgt_status sgt_shard_scatter(sgt_shard *shard);
sgt_status sgt_shard_gather(sgt_shard *shard);
sgt_status sgt_shard_update(sgt_shard *shard);
/* All n_all points' coordinates out of y_all (after the all-gather);
   synchronises; statuses as sgt_job_get_y. */
sgt_status sgt_shard_get_y(sgt_shard *shard, float *y, int layout, int mem_is_device,
                           int centre);
sgt_status sgt_shard_get_info(sgt_shard *shard, sgt_job_info *info);

/* Device bytes a job of these dimensions holds at its peak (creation
   included); what the server admits against its budget. */
size_t sgt_job_footprint(const sgt_params *params, int n, long nnz);

/* ---- serving: continuous batching of embedding requests ---------------
 * No counterpart in the reference.  A server on one device holds an HBM
 * budget and up to max_active running jobs, each on its own stream (stream
 * priority rises as n falls, so short requests are not stuck behind long
 * ones).  An admission thread turns waiting requests into jobs, in FIFO
 * order, as soon as their footprint fits the budget and a slot is free; a
 * scheduler thread keeps every running job `rounds_ahead` rounds of
 * `iters_per_round` iterations ahead of the GPU (one graph launch per
 * round), copies a finished job's coordinates to the caller's buffer and
 * returns its memory to the budget.  Requests that arrive while others run
 * are admitted while those are still on the GPU; their kernels overlap. */
typedef struct sgt_server sgt_server;
typedef struct {
  size_t hbm_budget;   /* device bytes the running jobs may hold          */
  int max_active;      /* running jobs (streams), 1..1024                 */
  int iters_per_round; /* iterations per graph launch, 1..256             */
  int rounds_ahead;    /* rounds queued ahead of the GPU per job, >= 1    */
} sgt_server_config;
typedef enum {
  SGT_REQ_WAITING = 0,
  SGT_REQ_RUNNING = 1,
  SGT_REQ_DONE = 2,
  SGT_REQ_FAILED = 3
} sgt_request_state;
typedef struct {
  int state;           /* sgt_request_state                               */
  sgt_status status;   /* why a request failed                            */
  int n, d, iters;     /* request dimensions                              */
  size_t footprint;    /* bytes admitted against the budget               */
  double t_submit;     /* seconds since the server was created (steady    */
  double t_admit;      /*   clock): submission, admission and the moment  */
  double t_done;       /*   its coordinates were in the caller's buffer   */
} sgt_request_info;
void sgt_server_config_default(sgt_server_config *cfg);
sgt_status sgt_server_create(int device, const sgt_server_config *cfg,
                             sgt_server **out);
/* Waits for running jobs to finish, then frees everything. */
void sgt_server_destroy(sgt_server *srv);
/* Queue a request.  rowptr/col/val: host CSR of the symmetric, normalised P
   (as sgt_job_create); y0 and y_out: host, point-major n*d.  All caller-owned
   and kept alive until the request is done or failed.  params->max_iter is
   the number of iterations; the result is centred as after the reference's
   last iteration.  Requests of fewer than 1,000,000 points run without the
   locality order of job creation (params->locality_order is ignored for
   them): its cost lands in the admission of every later request.  *id
   receives the request id (0, 1, 2, ...). */
sgt_status sgt_server_submit(sgt_server *srv, const sgt_params *params, int n,
                             const int *rowptr, const int *col,
                             const float *val, const float *y0, float *y_out,
                             long long *id);
/* Ids of requests finished (done or failed) since the last call, up to cap;
   waits up to wait_ms for at least one when none is ready. */
sgt_status sgt_server_poll(sgt_server *srv, double wait_ms, long long *ids,
                           int cap, int *count);
sgt_status sgt_server_request_info(sgt_server *srv, long long id,
                                   sgt_request_info *info);
/* Seconds on the server's clock (the time base of sgt_request_info). */
double sgt_server_now(const sgt_server *srv);

/* ---- stage operators (device pointers, queued on the context stream) --- */

/* F_attr = sum_j p_ij (y_i - y_j)/(1+|y_i-y_j|^2).  Replaces
   AttractiveEstimation (CU/pq.cu:24-57, CU/pq.cuh:8-10).
   format CSR: rowptr/col/val; COO: rowptr = NULL, rows in `coo_rows`;
   HYBRID: CSR input, split internally with the CUSP width rule. */
sgt_status sgt_attractive(sgt_ctx *ctx, int format, int n, int d, long nnz,
                          const int *rowptr, const unsigned *coo_rows,
                          const int *col, const float *val, const float *y,
                          int layout, float *f);

/* Interpolated repulsion.  Replaces computeFrepulsive_interp
   (CU/Frep.cu:81-125; h-driven grid as CU/Frep_varGrid.cu:79-107 and
   CU/gradient_descend_varGrid.cu:83-92).  ng_fixed > 0 forces the inner grid
   getBestGridSize(ng_fixed).  Outputs: f (normalised by Z, layout as y),
   *zeta, *grid_points, *h_eff (host pointers, any may be NULL).  An
   embedding whose h-driven grid exceeds the largest this operator provisions
   is computed on that largest grid and returns SGT_ERR_CAPACITY with the
   outputs written; for d <= 2 that is 512 points per axis, the end of the
   reference's grid-size table (CU/utils.cu:197-207), so only d = 3 (128
   points per axis) can reach it. */
sgt_status sgt_repulsive(sgt_ctx *ctx, int n, int d, float h, int ng_fixed,
                         const float *y, int layout, float *f, double *zeta,
                         int *grid_points, float *h_eff);

/* sgt_repulsive without any device allocation.  No counterpart in the
   reference: it exists for callers that must not allocate device memory,
   e.g. an application whose own pool allocator has reserved the whole GPU
   (a cudaMalloc would fail or fragment that pool) or a latency-sensitive
   loop where a cudaMalloc/cudaFree pair would stall on synchronisation.
   Same arguments and results as sgt_repulsive; all scratch lives in one
   fixed array of about 4 MB inside this library, which every GPU that loads
   the library holds until the process exits.
   Limits: 2 <= n <= 32768, d = 1 or 2, a grid of at most 128 points per axis
   in 2-D (512 in 1-D); anything larger is rejected with SGT_ERR_INVALID_ARG
   and a message (an embedding wider than the limit is detected after the
   work ran, its forces are not written to be used).  Points skipped by the
   S2G guard return SGT_ERR_CAPACITY, as in sgt_repulsive.
   The first call on a device (and the first after that device's context
   was reset) looks up the array's device address (cudaGetSymbolAddress) and
   should come before any stream capture.  Every call waits for its work on
   the context's stream to finish before it returns (it reads Z and the
   grid back to the host).  Calls share the array: calls that overlap on the
   GPU (other streams, other host threads on the same device) race and must
   be serialised by the caller. */
sgt_status sgt_repulsive_noalloc(sgt_ctx *ctx, int n, int d, float h,
                                 int ng_fixed, const float *y, int layout,
                                 float *f, double *zeta, int *grid_points,
                                 float *h_eff);

/* The integer part of the repulsion: per point and dim the floor bin of the
   scaled coordinate (CU/nuconv.cu:9-36 + CU/gridding.cu:159-167), and the
   grid size.  bins: device uint32 n*d point-major. */
sgt_status sgt_bins(sgt_ctx *ctx, int n, int d, float h, int ng_fixed,
                    const float *y, int layout, uint32_t *bins,
                    int *grid_points);

/* The charge grid after S2G and the potential grid after G2G of the last
   sgt_repulsive call: host float arrays of (d+1) * grid_points^d,
   channel-major [c][z][y][x].  Either may be NULL. */
sgt_status sgt_last_grids(sgt_ctx *ctx, float *v_grid, float *phi_grid);

/* getBestGridSize (CU/utils.cu:194-215): smallest table size >= ng+2, minus 2. */
int sgt_best_grid_size(int ng);

/* KL cost (CU/pq.cu:61-125, tsneCost) with FP64 terms and sum. */
sgt_status sgt_kl(sgt_ctx *ctx, int n, int d, long nnz, const int *rowptr,
                  const int *col, const float *val, const float *y, int layout,
                  double alpha, double zeta, double *kl);

/* lambda rescaling, one warp per row.  Replaces lambdaRescalingGPU
   (CU/graph_rescaling.cu:96-107).  dist = 1: values are distances, dist = 0:
   probabilities (-log p first); both with the semantics of the reference's
   CPU path HYB/graph_rescaling.cpp:19-104 and FP64 row sums: sigma solves
   sum_j exp(-sigma v_ij) = lambda to 1e-5.  dist = 2: distances with the
   steps of the reference's GPU kernel (CU/graph_rescaling.cu:11-94), bit for
   bit: FP32, and the row normalised with sigma one bisection step past the
   one that met the tolerance (rows that meet it early in a wide bracket
   then miss lambda).  val is rescaled in place; sigma (device, n) may be
   NULL. */
sgt_status sgt_lambda_bisect(sgt_ctx *ctx, int n, const int *rowptr,
                             float *val, float lambda, int dist, float *sigma);

/* Perplexity equalisation of kNN distances.  Replaces
   perplexityEqualization / SearchPerplexity (CU/perplexity_search.cu:113-208;
   FP64 as HYB/sgtsne.cpp:201-254).  dist: device n*k squared distances
   (self excluded), p: device n*k output rows summing to one, beta: device n
   or NULL.  k <= 256. */
sgt_status sgt_perplexity(sgt_ctx *ctx, int n, int k, const float *dist,
                          float perplexity, float *p, float *beta);

/* CSR -> COO row expansion (CU/prepareMatrix.cu:2-27); device pointers. */
sgt_status sgt_csr_to_coo(sgt_ctx *ctx, int n, long nnz, const int *rowptr,
                          unsigned *rows);

/* ELL width by the CUSP rule used in CU/matrix_converter.cpp:236-239
   (host rowptr). */
int sgt_ell_width(int n, const int *rowptr);

/* CSR -> ELL (column-major n*W, padding col 0 / val 0) + COO tail in row
   order (CU/prepareMatrix.cu:55-97, CU/matrix_converter.cpp:106-207).
   Host arrays; coo_* sized nnz.  *coo_size receives the tail length. */
sgt_status sgt_csr_to_hybrid(int n, const int *rowptr, const int *col,
                             const float *val, int width, unsigned *ell_cols,
                             float *ell_vals, unsigned *coo_rows,
                             unsigned *coo_cols, float *coo_vals,
                             long *coo_size);

/* Exact k nearest neighbours of n points in dim dimensions: squared
   Euclidean distances, the point itself excluded, each row sorted by
   distance (ties by index).  X: device, row-major n*dim; idx, d2: device,
   n*k.  1 <= k <= 128, k < n.  Replaces the kNN search of the reference's
   command line tool (allKNNsearchflann, FLANN, approximate;
   CU/testing_modules/demo_perplexity.cu:131) with an exact one; the result
   feeds sgt_perplexity directly.  Synchronises the context's stream. */
sgt_status sgt_knn(sgt_ctx *ctx, int n, int dim, const float *X, int k, int *idx,
                   float *d2);

/* Search methods of sgt_knn_ex; all return the same bits.
   SGT_KNN_SIMT: sums of squared differences, one query per thread.
   SGT_KNN_TENSOR: dim <= 64 and k <= 32 only.  Distances
     |q|^2 + |c|^2 - 2 q.c of all pairs on the tensor cores (TF32 in three
     terms, FP32 accumulation) keep a list of 64 candidates per query,
     re-ranked with the SIMT arithmetic; queries whose list could miss a
     neighbour under the filter's error bound are redone by the SIMT search.
   SGT_KNN_AUTO: the tensor-core filter where it applies and n >= 4096,
     the SIMT search otherwise or when the filter's operand images (about
     16 bytes per point and dimension) do not fit in device memory. */
enum { SGT_KNN_AUTO = 0, SGT_KNN_SIMT = 1, SGT_KNN_TENSOR = 2 };

/* sgt_knn with a method; *n_redo (may be NULL) receives the number of
   queries the tensor-core filter handed to the SIMT search. */
sgt_status sgt_knn_ex(sgt_ctx *ctx, int n, int dim, const float *X, int k, int *idx,
                      float *d2, int method, int *n_redo);

/* The same on the device: device arrays, out_col/out_val sized 2*nnz (an
   upper bound), out_rowptr n+1; *out_nnz receives the count (synchronises
   the context's stream).  Bit-identical to sgt_symmetrize.  n <= 2^24,
   nnz <= 2^30.  Replaces the cuSPARSE csrgeam path of SymmetrizeMatrix
   (CU/graph_rescaling.cu:266-398). */
sgt_status sgt_symmetrize_device(sgt_ctx *ctx, int n, long nnz, const int *rowptr,
                                 const int *col, const float *val, float scale,
                                 int *out_rowptr, int *out_col, float *out_val,
                                 long *out_nnz);

/* The same split on the device: device arrays (ell_* sized n*width, coo_*
   sized nnz); *coo_size receives the tail length (synchronises).
   Bit-identical to sgt_csr_to_hybrid. */
sgt_status sgt_csr_to_hybrid_device(sgt_ctx *ctx, int n, const int *rowptr,
                                    const int *col, const float *val, int width,
                                    unsigned *ell_cols, float *ell_vals,
                                    unsigned *coo_rows, unsigned *coo_cols,
                                    float *coo_vals, long *coo_size);

/* (P + P^T) * scale with sorted columns per row (CU/graph_rescaling.cu:266-398
   uses scale 1/(2n)).  Host arrays.  Call with out_col == NULL to get
   *out_nnz, then again with out arrays of that size. */
sgt_status sgt_symmetrize(int n, const int *rowptr, const int *col,
                          const float *val, float scale, int *out_rowptr,
                          int *out_col, float *out_val, long *out_nnz);

#ifdef __cplusplus
}
#endif
#endif /* SGTSNE_B200_H */
