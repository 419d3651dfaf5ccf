// Internal launchers shared by the engine's translation units.
#pragma once
#include <string>
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "als_common.cuh"

namespace als {

// Low-precision storage kinds for factor copies read by the tensor-core path.
enum LpKind : int { kLpNone = 0, kLpBf16 = 1, kLpFp16 = 2 };

int fp32_padded_rank(int f);
cudaError_t launch_rows_fp32(const RowsArgs &a, int lp_kind, int num_sms, cudaStream_t st);

// Tensor-core form (tcgen05 SYRK). Returns cudaErrorNotSupported when f is
// outside its range; the caller reports that instead of silently falling back.
bool tc_supported(int f);
int tc_padded_ld(int f);  // row stride (elements) of the low-precision factor copy
// Rows longer than max(8192, nnz / (kPlanSplitDiv * CTAs)) ratings are split
// into chunks of that size, so no item exceeds 1 / kPlanSplitDiv of a CTA's
// share; fewer than kPlanSplitDiv * CTAs rows are split, into fewer than
// 2 * kPlanSplitDiv * CTAs chunks.
constexpr int kPlanSplitDiv = 4;
struct WsPlan;
// x0: CG starting points (rows of stride a.ld_dst), or null; scale_x0: scale
// each start optimally along itself before CG (for a learned start).
cudaError_t launch_rows_tc(const RowsArgs &a, int lp_kind, int solver, int cg_max_steps,
                           float cg_tol, int cg_jacobi, int groups, const float *x0,
                           int scale_x0, const WsPlan *plan, int num_sms, cudaStream_t st);

// Solver parameters of one launch.
struct TcSolve {
  int solver;          // 0: Cholesky, 1: CG with Cholesky fallback
  int cg_max_steps;
  float cg_tol2;       // squared relative residual target
  const float *x0;     // CG starting point (m x ld_x0), or null for zero
  int ld_x0;
  int scale_x0;        // 1: scale x0 optimally along itself first (a learned start)
  int jacobi;          // 1: diagonal preconditioner
  int groups;          // solver warpgroups per CTA of the warp-specialised kernel (1, 2 or 3)
  int prepare;         // 1: only load the kernel instance and set its attributes
  uint32_t flags_or;   // status bits added to every row's word (one-CTA-per-row kernel)
  int withhold_first;  // test support: CTA 0 withholds its first item's accumulator completion
};

// Test support (als_debug_withhold_first_row): one-shot; the next launch of
// the warp-specialised kernel takes it.
bool debug_take_withhold();

// Work list of the warp-specialised kernel, planned on the host per side:
// one item per row, or one per chunk of a row split across CTAs.
struct alignas(16) WorkItem {
  long long s, e;  // rating range [s, e) of this item
  int u;           // row
  int deg;         // the row's total number of ratings (lambda * n_u)
  int part;        // partial-sum slot of this chunk; -1 when the item is the whole row
  int heavy;       // index of the split row; -1 otherwise
};

// Floats of one fallback Cholesky tile in global scratch (f <= 112: 112 x 113).
constexpr int kCholFloats = 112 * 113;

struct WsPlan {
  const WorkItem *items = nullptr;
  int nitems = 0;                      // items, or (with nitems_dev) an upper bound
  const int *nitems_dev = nullptr;     // the exact item count, in device memory
  const int *heavy_nchunks = nullptr;  // per split row: number of chunks
  const int *heavy_base = nullptr;     // per split row: first partial slot
  unsigned *heavy_count = nullptr;     // per split row: chunks finished (reset by the last)
  float *partial = nullptr;            // [slots][128][part_ld]
  int part_ld = 0;
  int src_rows = 0;                    // rows of the source factor matrix (gather bounds)
  float *chol = nullptr;               // [ctas][3][kCholFloats] fallback Cholesky tiles
  int ctas = 0;                        // CTAs the scratch covers: a launch uses at most this many
  // rows of ranks f > 112 that CG did not finish, for the post-pass of the
  // one-CTA-per-row kernel: the rows, their count and the post-pass queue head
  int *fb_rows = nullptr;
  int *fb_count = nullptr;             // fb_count[0] rows, fb_count[1] queue head
  int64_t rows = 0;                    // rows the plan covers
};

// Planning of a side's rows [begin, begin + count) on the device (no host
// copy, no synchronisation): items sorted by size bin, largest first, rows
// above `split` ratings cut into chunks, dealt to min(grid, count) CTAs. The
// plan lives in caller memory of plan_ws_bytes() bytes (256-byte aligned),
// which must stay untouched while the plan is used. `error` (may be null) is
// set when the row pointers are malformed beyond the plan's bounds; the plan
// is then empty.
size_t plan_ws_bytes(int64_t count, int grid, int np);
cudaError_t plan_ws(const int64_t *d_row_ptr, int64_t begin, int64_t count, int grid, int np,
                    int src_rows, void *mem, size_t mem_bytes, WsPlan *plan, int *error,
                    cudaStream_t st);

// Warp-specialised tensor-core kernel (f in [16, 128]); launch_rows_tc
// dispatches to it when a plan is given and tc_ws_takes holds: every rank up
// to 112, and above that CG without the Jacobi preconditioner (its rows that
// CG does not finish go to a post-pass of the one-CTA-per-row kernel).
bool tc_ws_supported(int f);
bool tc_ws_takes(int f, int solver, int jacobi);
cudaError_t launch_rows_tc_ws(const RowsArgs &a, int lp_kind, const TcSolve &sv,
                              const WsPlan &plan, int num_sms, cudaStream_t st);
int tc_ws_np(int f);
cudaError_t prepare_rows_tc_ws(int f, int lp_kind, int groups);

// Degree-binned visiting order: rows sorted by descending floor(log2(degree)).
// work: 3 * kOrderBins unsigned ints of device scratch.
constexpr int kOrderBins = 64;
cudaError_t launch_degree_order(const int64_t *row_ptr, int64_t m, int32_t *order,
                                unsigned *work, cudaStream_t st, int64_t row_begin = 0);

// int32 row pointers (drop-in API) -> int64
cudaError_t launch_widen_ptr(const int32_t *in, int64_t count, int64_t *out, cudaStream_t st);

// FP32 rows (ld_src) -> bf16/fp16 rows (ld_dst), columns [f, ld_dst) zeroed.
cudaError_t launch_convert_lp(const float *src, int64_t rows, int f, int ld_src, void *dst,
                              int ld_dst, int kind, cudaStream_t st);

// RMSE over COO test entries: per-block FP64 partials, then one reduction.
// work: at least rmse_work_bytes() bytes.
size_t rmse_work_bytes();
cudaError_t launch_rmse(int64_t nt, const int32_t *u, const int32_t *i, const float *r,
                        const float *X, int ldx, const float *T, int ldt, int f, double *out_dev,
                        void *work, cudaStream_t st);
// The sum of squared errors over the entries (no root, no division): a
// shard's share of the test RMSE.
cudaError_t launch_rmse_sum(int64_t nt, const int32_t *u, const int32_t *i, const float *r,
                            const float *X, int ldx, const float *T, int ldt, int f,
                            double *sum_dev, void *work, cudaStream_t st);
// Sets the message als_last_error() returns and gives back the code (for the
// C ABI entry points outside als_api.cu).
int api_fail(int code, const std::string &msg);
}  // namespace als
struct als_model;
namespace als {
// A model's rows of each side and its rank (for the shard driver's checks).
void model_dims(const als_model *model, int64_t *m, int64_t *n, int32_t *f);
cudaError_t launch_predict(int64_t nt, const int32_t *u, const int32_t *i, const float *X, int ldx,
                           const float *T, int ldt, int f, float *out, cudaStream_t st);

int device_sm_count();

// Top-k items per query user by x_u . theta_i, items of the user's training
// row (seen_ptr/seen_col, may be null) left out; k <= 256, f <= 128.
cudaError_t launch_topk(int64_t nq, const int32_t *users, const float *X, int ldx, const float *T,
                        int ldt, int64_t n, int f, int k, const int64_t *seen_ptr,
                        const int32_t *seen_col, int32_t *out_items, float *out_scores,
                        cudaStream_t st);

// CSR (m x n, nnz ratings) -> CSC on the device, rows ascending per column
// (stable radix sort by column). Synchronises the stream; allocates its sort
// scratch.
cudaError_t csr_to_csc(int64_t m, int64_t n, int64_t nnz, const int64_t *ptr, const int32_t *col,
                       const float *val, int64_t *cptr, int32_t *crow, float *cval,
                       cudaStream_t st);

// Learned CG warm start (als_mlp.cu). The net is opaque to callers.
cudaError_t mlp_create(void **out, int f, int64_t cap, uint64_t seed, cudaStream_t st);
void mlp_destroy(void *net);
int mlp_ldf(const void *net);
int64_t mlp_nparam(const void *net);
int *mlp_error(const void *net);
int64_t mlp_param_count(int f);
cudaError_t mlp_features(int64_t m, int f, const int64_t *row_ptr, const int32_t *col,
                         const float *val, const void *src, int ld_src, int lp_kind, void *F,
                         int ldf, cudaStream_t st);
// The same features over a side's work plan (16-bit factors only): long rows
// are split across blocks like the half-step kernel splits them.
cudaError_t mlp_features_plan(const WsPlan &plan, int f, const int32_t *col, const float *val,
                              const void *src, int ld_src, int lp_kind, void *F, int ldf,
                              cudaStream_t st);
cudaError_t mlp_infer(void *net, int64_t m, const void *F, float *X0, int ldx, cudaStream_t st);
cudaError_t mlp_train(void *net, int64_t m, int64_t batch, int steps, const void *F,
                      const float *T, int ldt, float lr, uint64_t seed, cudaStream_t st);
cudaError_t mlp_gradients(void *net, int64_t B, const void *F, const float *T, int ldt,
                          cudaStream_t st);
cudaError_t mlp_step(void *net, int64_t B, const void *F, const float *T, int ldt, float lr,
                     cudaStream_t st);
cudaError_t mlp_io(void *net, float *host, int what, double *loss, cudaStream_t st);

}  // namespace als
