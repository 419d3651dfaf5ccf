/*
 * als_b200.h -- C ABI of the B200 ALS engine (libGPUALS.so).
 *
 * Three layers, all plain C types (no C++ or framework types cross it):
 *
 *  1. Drop-in entry points with the exact declarations of the reference
 *     (IBMSparkGPU/CUDA-MLlib), so an existing caller links unchanged:
 *       doALSWithCSR   replaces als/src/cuda/als.h:96-103 (body als.cu:1001-1115)
 *       get_gpu        replaces utilities.h:39 (body utilities.cu:97-136)
 *       mallocBest     replaces utilities.h:40 (body utilities.cu:73-82), C++ linkage
 *       freeBest       replaces utilities.h:41 (body utilities.cu:85-95), C++ linkage
 *     The Spark JNI symbols of als/src/org_apache_spark_ml_recommendation_CuMFJNIInterface.h:31-40
 *     are exported from the same library (see cumf_jni.h).
 *
 *  2. Status-returning engine API on device buffers (new; cuMF has none):
 *     a resident model with both sides of the rating matrix, the full
 *     X-then-theta iteration, RMSE and predict.
 *
 *  3. als_train: the cuMF-standalone style full-iteration entry on host
 *     buffers (CSR/CSC arrays, m, n, f, lambda, iterations -> X, theta).
 *
 * Conventions: factors are row-major (row u of X is x_u, f floats); CSR row
 * pointers are int64 in the engine API (int32 in the drop-in one, as in the
 * reference); column indices int32; ratings float32. Every engine call is
 * stream-ordered on the stream passed in and does not synchronise unless it
 * returns a host value. Return codes: ALS_OK or an ALS_ERR_* value;
 * als_last_error() gives the message of the last failure on this thread.
 */
#ifndef ALS_B200_H_
#define ALS_B200_H_

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- 1. drop-in entry points ---------------- */

/* One ALS half-step, same contract as the reference (als/src/cuda/als.h:98-101):
 * solves X (m x f, row-major, written to the HOST buffer XTHost) from theta
 * (n x f, row-major, HOST buffer thetaTHost) and a 0-based CSR of R (m x n)
 * whose three arrays are DEVICE pointers (or mapped host memory from
 * mallocBest) that this call FREES, exactly as the reference does
 * (als.cu:1058, als.cu:1101-1102). lambda is scaled by each row's rating
 * count (als.cu:905-909). X_BATCH is accepted and ignored: the engine never
 * materialises the f x f systems in HBM, so it needs no batching.
 * CUDA failures throw thrust::system_error, as the reference's cudacall does
 * (als.h:43-53), so the JNI catch block (CuMFJNIInterface.cpp:129-131) still
 * sees them. Rows without ratings get x_u = 0 (the reference returns NaN). */
void doALSWithCSR(cudaStream_t cuda_stream, int *csrRowIndex, int *csrColIndex, float *csrVal,
                  float *thetaTHost, float *XTHost, const int m, const int n, const int f,
                  const long nnz, const float lambda, const int X_BATCH);

/* Round-robin device choice (utilities.cu:97-136). Unlike the reference it
 * does not reset every device on first use, which would destroy contexts that
 * other libraries in the same process hold. Returns -1 without devices. */
int get_gpu(void);

/* cudaMalloc, falling back to mapped pinned host memory (utilities.cu:73-82),
 * and the free of either kind of such allocation (utilities.cu:85-95).
 * The reference's utilities.h:36-41 gives C linkage to get_gpu only, so its
 * C++ callers (CuMFJNIInterface.cpp:93-95) bind the C++ names
 * mallocBest(void**, size_t) and freeBest(void*): those are declared below,
 * outside the extern "C" block, with the same linkage. C and FFI callers
 * (ctypes, cgo) use the C-linkage aliases als_malloc_best / als_free_best,
 * which are the same functions. */
cudaError_t als_malloc_best(void **devPtr, size_t size);
cudaError_t als_free_best(void *devPtr);

#ifdef __cplusplus
} /* extern "C" */
cudaError_t mallocBest(void **devPtr, size_t size);
cudaError_t freeBest(void *devPtr);
extern "C" {
#endif

/* ---------------- 2. engine API ---------------- */

enum {
  ALS_OK = 0,
  ALS_ERR_INVALID = 1,     /* bad argument                               */
  ALS_ERR_CUDA = 2,        /* CUDA runtime error (message has details)   */
  ALS_ERR_UNSUPPORTED = 3, /* e.g. rank outside the kernels' range       */
  ALS_ERR_NOT_CONVERGED = 4
};

enum { ALS_PREC_FP32 = 0, ALS_PREC_BF16 = 1, ALS_PREC_FP16 = 2 };
enum { ALS_SOLVER_CHOLESKY = 0, ALS_SOLVER_CG = 1 };
enum { ALS_WARM_ZERO = 0, ALS_WARM_PREVIOUS = 1, ALS_WARM_MLP = 2 };
enum { ALS_SIDE_USERS = 0, ALS_SIDE_ITEMS = 1 };

typedef struct als_options {
  int32_t precision;    /* ALS_PREC_*: FP32 factors + CUDA-core hermitian (rank f in
                           1..128), or a BF16/FP16 factor copy feeding the tensor-core
                           hermitian (f in 16..128: the warp-specialised persistent
                           kernel up to 112, a CTA per row above); other ranks give
                           ALS_ERR_UNSUPPORTED                                    */
  int32_t solver;       /* ALS_SOLVER_*                                          */
  int32_t warm_start;   /* ALS_WARM_* (CG starting point)                        */
  int32_t cg_max_steps; /* default 16                                            */
  float cg_tol;         /* CG relative residual target, default 1e-5             */
  float refine_tol;     /* FP32 relative residual above which an FP64-residual
                           refinement step runs, default 1e-5                    */
  int32_t use_graph;    /* capture one iteration as a CUDA graph and replay it  */
  /* learned warm start (ALS_WARM_MLP, tensor-core form with CG) */
  int32_t mlp_train_iters; /* iterations whose solves train the MLP (default 3)   */
  int32_t mlp_steps;       /* Adam steps per half-step while training (default 128) */
  int32_t mlp_batch;       /* rows per Adam step (default 8192)                   */
  float mlp_lr;            /* Adam learning rate (default 2e-3)                   */
  int32_t cg_jacobi;       /* 1: diagonal (Jacobi) preconditioner for CG (default 0:
                              it slowed convergence on the benchmark matrices) */
  int32_t solver_groups;   /* solver warpgroups per SM in the tensor-core kernel:
                              0 = chosen by the engine, 1, 2 or 3               */
  int32_t reserved[3];
} als_options;

typedef struct als_stats {
  uint64_t rows_solved;     /* rows processed since creation / last reset     */
  uint64_t rows_refined;    /* rows that took the FP64-residual refinement     */
  uint64_t rows_not_spd;    /* rows whose system had a non-positive pivot      */
  uint64_t cg_steps;        /* total CG iterations                             */
  uint64_t cg_fallbacks;    /* CG rows that fell back to Cholesky              */
  uint64_t kernel_errors;   /* 1 if a kernel gave up a bounded wait (results of
                               that half-step are incomplete)                  */
  uint64_t cg_r0_micro;     /* sum over CG rows of the starting relative residual
                               |b - A x0| / |b| (x0 after optimal scaling), x 1e6:
                               a measure of the warm start's quality          */
  uint32_t solver_groups[2]; /* warpgroup count the autotuner chose for the users /
                                items side (0: not tuned, or fixed by the options) */
} als_stats;

void als_default_options(als_options *opt);
/* Options the drop-in doALSWithCSR uses (process-wide; default: the FP32
 * form with Cholesky, which meets the reference's 1e-3 parity). A Spark
 * deployment can select the tensor-core form (BF16/FP16 + CG) here without
 * changing the call. No counterpart in the reference. */
int als_set_dropin_options(const als_options *opt);
int als_get_dropin_options(als_options *opt);

/* The drop-in half-step on HOST CSR arrays: what the Spark JNI call does as a
 * whole (CuMFJNIInterface.cpp:93-118 copies the three arrays into mallocBest
 * memory, then calls doALSWithCSR, als.cu:1001-1115), with the same inputs,
 * options (als_set_dropin_options) and result X, but pipelined: the ratings
 * are uploaded in `chunks` row ranges by rating count (0: chosen from nnz,
 * at most 8, or 12 for sides of more than one row per 1,000 ratings, whose
 * solve dominates; the first and last range half the size of the others,
 * since they do not overlap) on a copy stream, each range is solved on
 * `stream` as soon as it has landed, and its rows of X are downloaded while
 * the next range is solved. The arrays are the caller's and are not freed.
 * Host memory may be pageable (copied through pinned staging) or pinned
 * (copied directly; a pinned XTHost is also downloaded range by range).
 * Rows split across CTAs (longer than max(8192, range ratings / (4 * SMs)))
 * may differ from doALSWithCSR in the last bits, since the split depends on
 * the range; all other rows are bit-identical. Returns ALS_OK,
 * ALS_ERR_INVALID (bad sizes, row pointers that decrease or do not span nnz)
 * or ALS_ERR_CUDA (also when a kernel gave up a bounded wait); no exception.
 * Synchronises before it returns. The JNI entry of this library uses it. */
int als_half_step_host(cudaStream_t stream, const int *h_row_ptr, const int *h_col,
                       const float *h_val, const float *thetaTHost, float *XTHost, int m, int n,
                       int f, long nnz, float lambda, int chunks);
const char *als_last_error(void);
const char *als_version(void);

typedef struct als_model als_model;

/* Create a resident model. All device arrays are borrowed (the caller keeps
 * them alive and unchanged for the model's lifetime):
 *   users side  CSR  (m x n): csr_ptr[m+1], csr_col[nnz], csr_val[nnz]
 *   items side  CSC  (= CSR of R^T, n x m): csc_ptr[n+1], csc_row[nnz], csc_val[nnz]
 * The model allocates its factors (X: m x f, theta: n x f, FP32) and scratch. */
int als_model_create(als_model **out, int64_t m, int64_t n, int32_t f, int64_t nnz,
                     const int64_t *csr_ptr, const int32_t *csr_col, const float *csr_val,
                     const int64_t *csc_ptr, const int32_t *csc_row, const float *csc_val,
                     const als_options *opt, cudaStream_t stream);
void als_model_destroy(als_model *model);

/* Copy initial item factors (n x f, row stride ld) from device memory. */
int als_model_set_theta(als_model *model, const float *d_theta, int32_t ld, cudaStream_t stream);
/* Copy user factors (m x f) from device memory (warm start for CG). */
int als_model_set_x(als_model *model, const float *d_x, int32_t ld, cudaStream_t stream);

/* One half-step: ALS_SIDE_USERS solves X from theta, ALS_SIDE_ITEMS solves
 * theta from X. */
int als_model_half_step(als_model *model, int32_t side, float lambda, cudaStream_t stream);
/* Restrict a side's half-steps to rows [begin, end) (default: all rows).
 * Used to shard rows across GPUs: each rank solves its range, then the ranks
 * exchange the updated rows (see als_model_sync_lp). */
int als_model_set_row_range(als_model *model, int32_t side, int64_t begin, int64_t end,
                            cudaStream_t stream);
/* Rebuild the BF16/FP16 copy of a side's FP32 factors after they were
 * changed outside the engine (e.g. rows received from other GPUs). No-op in
 * the FP32 form. */
int als_model_sync_lp(als_model *model, int32_t side, cudaStream_t stream);
/* `iters` full iterations (users then items). */
int als_model_iterate(als_model *model, float lambda, int32_t iters, cudaStream_t stream);

/* Borrowed device pointers to the FP32 factors (row stride f). */
int als_model_factors(als_model *model, float **d_x, float **d_theta);
/* Per-row status words of the last half-step of each side (see ALS_ROW_*). */
int als_model_row_flags(als_model *model, int32_t side, const uint32_t **d_flags);
int als_model_stats(als_model *model, als_stats *out, int32_t reset);

/* Test RMSE over COO triplets (device arrays), FP64 reduction; blocks until
 * the value is on the host. */
int als_model_rmse(als_model *model, int64_t nt, const int32_t *d_u, const int32_t *d_i,
                   const float *d_r, double *rmse_out, cudaStream_t stream);

enum { ALS_ROW_EMPTY = 1, ALS_ROW_NOT_SPD = 2, ALS_ROW_REFINED_F64 = 4, ALS_ROW_CG_FALLBACK = 8 };

/* Row sharding across GPUs, one process per GPU (no counterpart in the
 * reference, which runs one problem on one GPU per call). Every rank holds the whole CSR/CSC and both factor
 * matrices in its model, solves an nnz-balanced contiguous range of each
 * side's rows, and after each half-step the ranges are exchanged by one NCCL
 * all-gather (equal blocks of the largest range's row count; the other ranks'
 * ranges are then copied into place) and the low-precision copy is rebuilt.
 * Test RMSE: each rank's share of the entries, summed by an NCCL all-reduce.
 * NCCL (libnccl.so.2) is loaded at the first call that needs it; without it
 * these calls return ALS_ERR_UNSUPPORTED. Every rank makes the same calls in
 * the same order (they are collective from als_shard_create on). */
typedef struct als_shard als_shard;
/* A 128-byte NCCL unique id: rank 0 makes it and sends a copy to every rank
 * (through whatever channel the job has) before als_shard_create. */
int als_shard_unique_id(void *id128);
/* Host only: the nnz-balanced contiguous row ranges [b[r], b[r+1]) of a side
 * with host row pointers h_ptr[rows + 1]; a row costs nnz * f^2 + f^3 / 3.
 * h_bounds holds world + 1 values. */
int als_shard_partition(const int64_t *h_ptr, int64_t rows, int32_t world, int32_t f,
                        int64_t *h_bounds);
/* Host only: the all-gather's block size in rows (the largest range) and, per
 * rank, the first row of the block it sends: start[r] = min(b[r], rows - span). */
int als_shard_blocks(const int64_t *h_bounds, int32_t world, int64_t *h_span, int64_t *h_start);
/* Collective: partitions both sides from host copies of the model's row
 * pointers (CSR m + 1 and CSC n + 1 values), restricts the model's half-steps
 * to this rank's ranges, and creates the communicator. The model stays owned
 * by the caller and must outlive the shard. */
int als_shard_create(als_shard **out, als_model *model, const int64_t *h_csr_ptr,
                     const int64_t *h_csc_ptr, int64_t m, int64_t n, int32_t f, int32_t world,
                     int32_t rank, const void *id128, cudaStream_t stream);
/* This rank's copy of a side's ranges (world + 1 values). */
int als_shard_bounds(const als_shard *shard, int32_t side, int64_t *h_bounds);
/* Collective: the all-gather of a side's ranges and the low-precision rebuild. */
int als_shard_exchange(als_shard *shard, int32_t side, cudaStream_t stream);
/* Collective: this rank's half-step of a side, then its exchange. */
int als_shard_half_step(als_shard *shard, int32_t side, float lambda, cudaStream_t stream);
/* Collective: `iters` full iterations (users, then items). */
int als_shard_iterate(als_shard *shard, float lambda, int32_t iters, cudaStream_t stream);
/* Collective: test RMSE over COO triplets (device arrays, the same on every
 * rank); blocks until the value is on the host. */
int als_shard_rmse(als_shard *shard, int64_t nt, const int32_t *d_u, const int32_t *d_i,
                   const float *d_r, double *rmse_out, cudaStream_t stream);
/* Collective: destroys the communicator and gives the model back its full row
 * ranges (so the model must still exist). */
void als_shard_destroy(als_shard *shard);

/* Stand-alone half-step on caller buffers (no model): src n x f (ld_src),
 * dst m x f (ld_dst). work must hold als_half_step_work_bytes(m) bytes. */
size_t als_half_step_work_bytes(int64_t m);
int als_half_step(int64_t m, int64_t n, int32_t f, const int64_t *d_row_ptr,
                  const int32_t *d_col, const float *d_val, const float *d_src, int32_t ld_src,
                  float *d_dst, int32_t ld_dst, float lambda, const als_options *opt,
                  void *d_work, size_t work_bytes, cudaStream_t stream);

/* The same FP32 half-step without a workspace argument, for callers that
 * cannot call cudaMalloc: a process whose device memory is already handed to
 * another allocator's pool (a Spark executor or PyTorch process whose pooling
 * allocator reserves the GPU, so a raw cudaMalloc fails or fragments it), or
 * a caller that must not pay the device-wide synchronisation that
 * cudaMalloc/cudaFree can cause. Its scratch (visiting order, row queue,
 * counters) is a file-scope __device__ array sized for at most
 * ALS_STATIC_MAX_ROWS rows (about 4 MiB, held on every GPU that loads the
 * library until the process exits), so a call allocates nothing.
 * Larger m is rejected with ALS_ERR_INVALID. The first call on each device
 * looks the array up with cudaGetSymbolAddress; make that first call before
 * any stream capture. After a device reset (which reloads the library's
 * device code at a new address) the next call looks it up again, so that
 * call too belongs before any capture. Calls that overlap in time (two
 * streams, two host threads) share the one array and race: serialise them.
 * No counterpart in the reference. */
#define ALS_STATIC_MAX_ROWS 1048576
int als_half_step_static(int64_t m, int64_t n, int32_t f, const int64_t *d_row_ptr,
                         const int32_t *d_col, const float *d_val, const float *d_src,
                         int32_t ld_src, float *d_dst, int32_t ld_dst, float lambda,
                         const als_options *opt, cudaStream_t stream);

/* RMSE / predict over COO triplets with caller factors. */
size_t als_rmse_work_bytes(void);
int als_rmse(int64_t nt, const int32_t *d_u, const int32_t *d_i, const float *d_r,
             const float *d_x, int32_t ldx, const float *d_theta, int32_t ldt, int32_t f,
             double *rmse_out, void *d_work, size_t work_bytes, cudaStream_t stream);
int als_predict(int64_t nt, const int32_t *d_u, const int32_t *d_i, const float *d_x,
                int32_t ldx, const float *d_theta, int32_t ldt, int32_t f, float *d_out,
                cudaStream_t stream);

/* Top-k recommendation (serving; no counterpart in the reference). For each of
 * the nq users in d_users, the k items (k <= 256) of largest x_u . theta_i over
 * all n items, best first (ties: lower item index), leaving out the items in
 * the user's row of a CSR of already-rated items (d_seen_ptr / d_seen_col,
 * columns ascending per row; both null to keep every item). Outputs are
 * nq x k, row-major; an item of -1 (score -inf) pads users with fewer than k
 * candidate items. f <= 128. */
int als_topk(int64_t nq, const int32_t *d_users, const float *d_x, int32_t ldx,
             const float *d_theta, int32_t ldt, int64_t n, int32_t f, int32_t k,
             const int64_t *d_seen_ptr, const int32_t *d_seen_col, int32_t *d_items,
             float *d_scores, cudaStream_t stream);

/* CSR (m x n, nnz ratings; int64 row pointers) -> CSC, i.e. the CSR of the
 * transpose (n x m), on the device: rows stay ascending within each column, so
 * the result equals als_csr_transpose's. A caller that keeps only one
 * orientation of the rating matrix can build the other for als_model_create.
 * Allocates its sort scratch and synchronises the stream. No counterpart in
 * the reference, whose loadCSRSparseMatrixBin (als.cu:914-933) gives a CSR
 * only. */
int als_csr_to_csc(int64_t m, int64_t n, int64_t nnz, const int64_t *d_row_ptr,
                   const int32_t *d_col, const float *d_val, int64_t *d_col_ptr,
                   int32_t *d_row, float *d_val_t, cudaStream_t stream);

/* Learned warm start: the MLP that maps a row's features
 * [b_u / n_u, diag(A_u) / n_u, log1p(n_u) / 8] (2f+1 values, BF16, row stride
 * als_mlp_feature_stride) to x0 (f floats). Layers 2f+1 -> 256 -> 256 -> f with
 * GELU, BF16 weights and activations, FP32 accumulation; tensor-core kernels
 * for forward, backward and Adam. No counterpart in the reference. */
typedef struct als_mlp als_mlp;
int als_mlp_create(als_mlp **out, int32_t f, int64_t batch_capacity, uint64_t seed,
                   cudaStream_t stream);
void als_mlp_destroy(als_mlp *mlp);
int als_mlp_feature_stride(const als_mlp *mlp);
int64_t als_mlp_param_count(int32_t f);
/* host <-> parameters, unpadded, in the order W1 [256 x (2f+1)], b1 [256],
 * W2 [256 x 256], b2 [256], W3 [f x 256], b3 [f] (W[out][in]) */
int als_mlp_get_params(als_mlp *mlp, float *host, cudaStream_t stream);
int als_mlp_set_params(als_mlp *mlp, const float *host, cudaStream_t stream);
/* loss = mean_b |y_b - t_b|^2 / f and its gradients (same layout as the
 * parameters) for `batch` rows, without updating; batch a multiple of 64 */
int als_mlp_gradients(als_mlp *mlp, int64_t batch, const void *d_features, const float *d_targets,
                      int32_t ldt, float *host_grads, double *loss, cudaStream_t stream);
int als_mlp_train_step(als_mlp *mlp, int64_t batch, const void *d_features,
                       const float *d_targets, int32_t ldt, float lr, cudaStream_t stream);
int als_mlp_forward(als_mlp *mlp, int64_t rows, const void *d_features, float *d_out, int32_t ldo,
                    cudaStream_t stream);
/* features of rows [0, m) of a CSR against source factors d_src (kind:
 * ALS_PREC_FP32 / BF16 / FP16, row stride ld_src) into d_features (BF16). */
int als_features(int64_t m, int32_t f, const int64_t *d_row_ptr, const int32_t *d_col,
                 const float *d_val, const void *d_src, int32_t ld_src, int32_t src_precision,
                 void *d_features, int32_t ldf, cudaStream_t stream);

/* Test support for the kernels' bounded waits: arms a one-shot fault for the
 * next tensor-core half-step (ranks 16..128 with a work plan): the MMA issuer
 * of its first CTA stops after its first row, without marking that row's
 * accumulator complete, as a stalled issuer would. The waits of that CTA's
 * solvers and producers give up (2 s), every role of the kernel leaves its
 * loop, the kernel returns with its error word set
 * (als_stats.kernel_errors == 1) and the half-step's results are incomplete;
 * doALSWithCSR throws. Nothing faults or hangs, and the next half-step runs
 * normally. 0 disarms. No counterpart in the reference. */
int als_debug_withhold_first_row(int32_t enable);

/* ---------------- 3. full training on host buffers ---------------- */

/* cuMF-standalone style entry (not present in the reference; new):
 * host CSR (m x n) and CSC of the same ratings, initial theta (n x f, row
 * major, host, overwritten with the result), X_out (m x f, host). Runs
 * `iterations` full iterations on the current device and stream 0.
 * stats may be NULL. */
int als_train(const int64_t *csr_ptr, const int32_t *csr_col, const float *csr_val,
              const int64_t *csc_ptr, const int32_t *csc_row, const float *csc_val, int64_t m,
              int64_t n, int32_t f, int64_t nnz, float lambda, int32_t iterations,
              const als_options *opt, float *X_out, float *theta_inout, als_stats *stats);

#ifdef __cplusplus
}
#endif
#endif /* ALS_B200_H_ */
