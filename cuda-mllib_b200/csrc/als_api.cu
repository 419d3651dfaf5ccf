// C ABI of the engine: resident model, half-step dispatch, the drop-in
// doALSWithCSR / utilities entry points, and host-buffer training.
#include <cuda.h>
#include <thrust/system/cuda/error.h>
#include <thrust/system_error.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <exception>
#include <iterator>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/als_b200.h"
#include "als_internal.h"

using namespace als;

namespace {

thread_local std::string g_last_error;

std::atomic<bool> &debug_withhold() {
  static std::atomic<bool> flag{false};
  return flag;
}
std::mutex g_dropin_mu;
als_options g_dropin;       // set on first use from als_default_options
bool g_dropin_set = false;

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *where) {
  return fail(ALS_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define ALS_TRY(call, where)                          \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return cuda_fail(e_, where); \
  } while (0)

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

int lp_kind_of(int precision) {
  return precision == ALS_PREC_BF16 ? kLpBf16 : precision == ALS_PREC_FP16 ? kLpFp16 : kLpNone;
}

int check_options(const als_options &o, int f) {
  if (o.precision < ALS_PREC_FP32 || o.precision > ALS_PREC_FP16)
    return fail(ALS_ERR_INVALID, "unknown precision");
  if (o.solver != ALS_SOLVER_CHOLESKY && o.solver != ALS_SOLVER_CG)
    return fail(ALS_ERR_INVALID, "unknown solver");
  if (o.precision == ALS_PREC_FP32) {
    if (o.solver != ALS_SOLVER_CHOLESKY)
      return fail(ALS_ERR_UNSUPPORTED, "the FP32 form solves with Cholesky only");
    if (fp32_padded_rank(f) < 0) return fail(ALS_ERR_UNSUPPORTED, "rank f must be 1..128");
  } else if (!tc_supported(f)) {
    return fail(ALS_ERR_UNSUPPORTED, "tensor-core form supports rank f in 16..128");
  }
  if (o.cg_max_steps < 0 || o.cg_max_steps > 256) return fail(ALS_ERR_INVALID, "cg_max_steps");
  if (o.solver_groups < 0 || o.solver_groups > 3) return fail(ALS_ERR_INVALID, "solver_groups must be 0 .. 3");
  if (o.warm_start < ALS_WARM_ZERO || o.warm_start > ALS_WARM_MLP)
    return fail(ALS_ERR_INVALID, "unknown warm start");
  if (o.warm_start == ALS_WARM_MLP &&
      (o.precision == ALS_PREC_FP32 || o.solver != ALS_SOLVER_CG || f > 128))
    return fail(ALS_ERR_UNSUPPORTED, "the learned warm start needs the tensor-core form with CG");
  if (o.warm_start == ALS_WARM_MLP && (o.mlp_batch < 64 || o.mlp_steps < 0 || !(o.mlp_lr > 0.f)))
    return fail(ALS_ERR_INVALID, "bad MLP training options");
  return ALS_OK;
}

// Scratch for one solve side.
struct Side {
  int64_t rows = 0, cols = 0;
  int64_t begin = 0, active = 0;  // rows [begin, begin + active) are solved
  const int64_t *ptr = nullptr;
  const int32_t *idx = nullptr;
  const float *val = nullptr;
  int32_t *order = nullptr;
  unsigned *queue = nullptr;  // [0]: head, [1..]: order scratch
  uint32_t *flags = nullptr;
  WsPlan plan;                // work list of the warp-specialised kernel
  void *plan_mem = nullptr;   // device memory of the plan (plan_ws_bytes for all rows)
  size_t plan_bytes = 0;
  bool has_plan = false;
};

// Dispatch one half-step: rows of `s` solved against factor `src`.
cudaError_t run_rows(const Side &s, int f, float lambda, const als_options &o, const float *src32,
                     int ld_src32, const void *src_lp, int ld_lp, float *dst32, void *dst_lp,
                     Counters *ctr, const float *x0, bool learned_x0, int num_sms,
                     cudaStream_t st) {
  if (s.active <= 0) return cudaSuccess;
  RowsArgs a{};
  a.m = s.active;
  a.f = f;
  a.lambda = lambda;
  a.row_ptr = s.ptr;
  a.col = s.idx;
  a.val = s.val;
  a.dst = dst32;
  a.ld_dst = f;
  a.dst_lp = dst_lp;
  a.ld_dst_lp = ld_lp;
  a.order = s.order;
  a.queue = s.queue;
  a.row_flags = s.flags;
  a.counters = ctr;
  a.refine_tol = o.refine_tol;
  a.error = ctr ? &ctr->error : nullptr;
  cudaError_t e = cudaMemsetAsync(s.queue, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  const int kind = lp_kind_of(o.precision);
  if (kind == kLpNone) {
    a.src = src32;
    a.ld_src = ld_src32;
    return launch_rows_fp32(a, kind, num_sms, st);
  }
  a.src = src_lp;
  a.ld_src = ld_lp;
  return launch_rows_tc(a, kind, o.solver, o.cg_max_steps, o.cg_tol, o.cg_jacobi,
                        o.solver_groups, x0, learned_x0 ? 1 : 0, s.has_plan ? &s.plan : nullptr,
                        num_sms, st);
}

}  // namespace

namespace als {
int api_fail(int code, const std::string &msg) { return fail(code, msg); }
}  // namespace als

struct als_model {
  int64_t m = 0, n = 0, nnz = 0;
  int32_t f = 0;
  als_options opt{};
  Side side[2];
  float *X = nullptr, *T = nullptr;      // FP32 factors, row stride f
  void *X_lp = nullptr, *T_lp = nullptr;  // low-precision copies (tensor-core form)
  int lp_ld = 0;
  Counters *ctr = nullptr;
  void *rmse_work = nullptr;
  double *rmse_dev = nullptr;
  int num_sms = 0;
  cudaGraphExec_t graph = nullptr;
  float graph_lambda = 0.f;
  void *block = nullptr;  // single allocation holding everything above
  // learned warm start: one net per side, features and x0 per side
  void *net[2] = {nullptr, nullptr};
  void *feat[2] = {nullptr, nullptr};
  float *x0[2] = {nullptr, nullptr};
  int ldf = 0;
  int halfsteps[2] = {0, 0};
  void *mlp_block = nullptr;
  // solver-warpgroup autotuning per side (options.solver_groups == 0)
  int tuned[2] = {0, 0};     // chosen warpgroup count, 0 while tuning
  int tune_idx[2] = {0, 0};  // half-steps timed so far
  float tune_ms[2][3] = {};
  cudaEvent_t tev[2] = {nullptr, nullptr};
};

namespace {
// Warpgroup counts tried for a side, in this order: the first and last runs
// bracket the middle one, so the steady drop of CG steps from one iteration
// to the next cancels out of the comparison. Up to f = 112 the candidates
// are two (rows in registers) and three (rows in TMEM) warpgroups; above it,
// two (rows in TMEM) and one (rows in registers: 255 registers a thread).
int tune_groups(int f, int k) {
  static constexpr int narrow[3] = {2, 3, 2}, wide[3] = {2, 1, 2};
  return f <= 112 ? narrow[k] : wide[k];
}
}  // namespace

namespace als {
void model_dims(const als_model *M, int64_t *m, int64_t *n, int32_t *f) {
  *m = M->m;
  *n = M->n;
  *f = M->f;
}
}  // namespace als

extern "C" {

void als_default_options(als_options *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = ALS_PREC_FP32;
  o->solver = ALS_SOLVER_CHOLESKY;
  o->warm_start = ALS_WARM_PREVIOUS;
  o->cg_max_steps = 16;
  o->cg_tol = 1e-5f;
  o->refine_tol = 1e-5f;
  o->use_graph = 0;
  o->mlp_train_iters = 3;
  o->mlp_steps = 128;
  o->mlp_batch = 8192;
  o->mlp_lr = 2e-3f;
  o->cg_jacobi = 0;
  o->solver_groups = 0;
}

const char *als_last_error(void) { return g_last_error.c_str(); }

int als_get_dropin_options(als_options *o) {
  if (!o) return fail(ALS_ERR_INVALID, "null options");
  std::lock_guard<std::mutex> lk(g_dropin_mu);
  if (!g_dropin_set) { als_default_options(&g_dropin); g_dropin_set = true; }
  *o = g_dropin;
  return ALS_OK;
}

int als_set_dropin_options(const als_options *o) {
  if (!o) return fail(ALS_ERR_INVALID, "null options");
  if (o->warm_start == ALS_WARM_MLP) return fail(ALS_ERR_UNSUPPORTED, "no learned warm start in the drop-in call");
  std::lock_guard<std::mutex> lk(g_dropin_mu);
  g_dropin = *o;
  g_dropin_set = true;
  return ALS_OK;
}
const char *als_version(void) { return "als_b200 1.0 (sm_100a)"; }

int als_debug_withhold_first_row(int32_t enable) {
  debug_withhold().store(enable != 0);
  return ALS_OK;
}

int als_model_create(als_model **out, int64_t m, int64_t n, int32_t f, int64_t nnz,
                     const int64_t *csr_ptr, const int32_t *csr_col, const float *csr_val,
                     const int64_t *csc_ptr, const int32_t *csc_row, const float *csc_val,
                     const als_options *opt, cudaStream_t st) {
  if (!out) return fail(ALS_ERR_INVALID, "out is null");
  *out = nullptr;
  if (m <= 0 || n <= 0 || f <= 0 || nnz < 0 || m > INT32_MAX || n > INT32_MAX)
    return fail(ALS_ERR_INVALID, "bad problem size");
  if (!csr_ptr || !csc_ptr || (nnz > 0 && (!csr_col || !csr_val || !csc_row || !csc_val)))
    return fail(ALS_ERR_INVALID, "null CSR/CSC array");
  als_options o;
  als_default_options(&o);
  if (opt) o = *opt;
  int rc = check_options(o, f);
  if (rc != ALS_OK) return rc;

  als_model *M = new als_model();
  M->m = m; M->n = n; M->f = f; M->nnz = nnz; M->opt = o;
  M->num_sms = device_sm_count();
  for (int i = 0; i < 2; ++i)
    if (cudaEventCreate(&M->tev[i]) != cudaSuccess) M->tev[i] = nullptr;  // no events: no tuning
  const int kind = lp_kind_of(o.precision);
  M->lp_ld = kind == kLpNone ? 0 : tc_padded_ld(f);
  // one allocation: factors, low-precision copies, orders, queues, flags, counters
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t p = off; off = align_up(off + bytes, 256); return p; };
  const size_t oX = take(sizeof(float) * m * f), oT = take(sizeof(float) * n * f);
  const size_t oXl = kind ? take(2ull * m * M->lp_ld) : 0, oTl = kind ? take(2ull * n * M->lp_ld) : 0;
  const size_t oOu = take(sizeof(int32_t) * m), oOi = take(sizeof(int32_t) * n);
  const size_t oQu = take(sizeof(unsigned) * (1 + 3 * kOrderBins)),
               oQi = take(sizeof(unsigned) * (1 + 3 * kOrderBins));
  const size_t oFu = take(sizeof(uint32_t) * m), oFi = take(sizeof(uint32_t) * n);
  const size_t oC = take(sizeof(Counters)), oR = take(rmse_work_bytes()), oRd = take(sizeof(double));
  cudaError_t e = cudaMalloc(&M->block, off);
  if (e != cudaSuccess) {
    delete M;
    return cuda_fail(e, "als_model_create: cudaMalloc");
  }
  char *b = static_cast<char *>(M->block);
  M->X = (float *)(b + oX);
  M->T = (float *)(b + oT);
  if (kind) { M->X_lp = b + oXl; M->T_lp = b + oTl; }
  M->ctr = (Counters *)(b + oC);
  M->rmse_work = b + oR;
  M->rmse_dev = (double *)(b + oRd);
  Side &U = M->side[ALS_SIDE_USERS], &I = M->side[ALS_SIDE_ITEMS];
  U.rows = m; U.cols = n; U.active = m; U.ptr = csr_ptr; U.idx = csr_col; U.val = csr_val;
  U.order = (int32_t *)(b + oOu); U.queue = (unsigned *)(b + oQu); U.flags = (uint32_t *)(b + oFu);
  I.rows = n; I.cols = m; I.active = n; I.ptr = csc_ptr; I.idx = csc_row; I.val = csc_val;
  I.order = (int32_t *)(b + oOi); I.queue = (unsigned *)(b + oQi); I.flags = (uint32_t *)(b + oFi);
  e = cudaMemsetAsync(M->block, 0, off, st);
  if (e == cudaSuccess) e = launch_degree_order(U.ptr, m, U.order, U.queue + 1, st);
  if (e == cudaSuccess) e = launch_degree_order(I.ptr, n, I.order, I.queue + 1, st);
  if (e != cudaSuccess) {
    cudaFree(M->block);
    delete M;
    return cuda_fail(e, "als_model_create");
  }
  if (kind != kLpNone && tc_ws_takes(f, o.solver, o.cg_jacobi)) {
    // plan memory for the whole side, so a row range (fewer rows) fits it too
    for (int sd = 0; sd < 2 && e == cudaSuccess; ++sd) {
      Side &S = M->side[sd];
      S.plan_bytes = plan_ws_bytes(S.rows, M->num_sms, tc_ws_np(f));
      e = cudaMalloc(&S.plan_mem, S.plan_bytes);
      if (e == cudaSuccess)
        e = plan_ws(S.ptr, 0, S.rows, M->num_sms, tc_ws_np(f), (int)S.cols, S.plan_mem,
                    S.plan_bytes, &S.plan, &M->ctr->error, st);
      S.has_plan = e == cudaSuccess;
    }
    // the autotuner's candidates are loaded now, so no timed launch pays for it
    for (int k = 0; k < 2 && e == cudaSuccess && o.solver_groups == 0; ++k)
      e = prepare_rows_tc_ws(f, kind, tune_groups(f, k));
    if (e != cudaSuccess) {
      als_model_destroy(M);
      return cuda_fail(e, "als_model_create: work plan");
    }
  }
  if (o.warm_start == ALS_WARM_MLP) {
    const int64_t cap = std::max<int64_t>(o.mlp_batch, 32768);
    for (int s = 0; s < 2 && e == cudaSuccess; ++s)
      e = mlp_create(&M->net[s], f, cap, 0x5eedULL + (uint64_t)s, st);
    if (e == cudaSuccess) {
      M->ldf = mlp_ldf(M->net[0]);
      size_t moff = 0;
      auto mtake = [&](size_t bytes) { size_t p = moff; moff = align_up(moff + bytes, 256); return p; };
      const size_t oF0 = mtake(2ull * m * M->ldf), oF1 = mtake(2ull * n * M->ldf),
                   oX0 = mtake(4ull * m * f), oX1 = mtake(4ull * n * f);
      e = cudaMalloc(&M->mlp_block, moff);
      if (e == cudaSuccess) {
        char *mb = (char *)M->mlp_block;
        M->feat[0] = mb + oF0; M->feat[1] = mb + oF1;
        M->x0[0] = (float *)(mb + oX0); M->x0[1] = (float *)(mb + oX1);
        e = cudaMemsetAsync(M->mlp_block, 0, moff, st);
      }
    }
    if (e != cudaSuccess) {
      als_model_destroy(M);
      return cuda_fail(e, "als_model_create: learned warm start");
    }
  }
  *out = M;
  return ALS_OK;
}

void als_model_destroy(als_model *M) {
  if (!M) return;
  if (M->graph) cudaGraphExecDestroy(M->graph);
  for (int i = 0; i < 2; ++i)
    if (M->tev[i]) cudaEventDestroy(M->tev[i]);
  for (int s = 0; s < 2; ++s) {
    mlp_destroy(M->net[s]);
    cudaFree(M->side[s].plan_mem);
  }
  cudaFree(M->mlp_block);
  cudaFree(M->block);
  delete M;
}

static int set_factor(als_model *M, const float *src, int32_t ld, int64_t rows, float *dst32,
                      void *dst_lp, cudaStream_t st) {
  if (!src || ld < M->f) return fail(ALS_ERR_INVALID, "bad factor pointer or stride");
  ALS_TRY(cudaMemcpy2DAsync(dst32, sizeof(float) * M->f, src, sizeof(float) * ld,
                            sizeof(float) * M->f, rows, cudaMemcpyDeviceToDevice, st),
          "set factor");
  if (dst_lp)
    ALS_TRY(launch_convert_lp(dst32, rows, M->f, M->f, dst_lp, M->lp_ld,
                              lp_kind_of(M->opt.precision), st),
            "convert factor");
  return ALS_OK;
}

int als_model_set_theta(als_model *M, const float *d, int32_t ld, cudaStream_t st) {
  if (!M) return fail(ALS_ERR_INVALID, "null model");
  return set_factor(M, d, ld, M->n, M->T, M->T_lp, st);
}

int als_model_set_x(als_model *M, const float *d, int32_t ld, cudaStream_t st) {
  if (!M) return fail(ALS_ERR_INVALID, "null model");
  return set_factor(M, d, ld, M->m, M->X, M->X_lp, st);
}

static cudaError_t model_half(als_model *M, int side, float lambda, cudaStream_t st) {
  const bool users = side == ALS_SIDE_USERS;
  const float *src32 = users ? M->T : M->X;
  const void *src_lp = users ? M->T_lp : M->X_lp;
  float *dst32 = users ? M->X : M->T;
  void *dst_lp = users ? M->X_lp : M->T_lp;
  const Side &S = M->side[side];
  const float *x0 = (M->opt.warm_start == ALS_WARM_PREVIOUS) ? dst32 : nullptr;
  bool train = false;
  if (M->opt.warm_start == ALS_WARM_MLP) {
    // features of this side's rows against the fixed factor (BF16/FP16 copy),
    // over the side's work plan when it has one
    cudaError_t e = cudaErrorNotSupported;
    if (S.has_plan)
      e = mlp_features_plan(S.plan, M->f, S.idx, S.val, src_lp, M->lp_ld,
                            lp_kind_of(M->opt.precision), M->feat[side], M->ldf, st);
    if (e == cudaErrorNotSupported)
      e = mlp_features(S.rows, M->f, S.ptr, S.idx, S.val, src_lp, M->lp_ld,
                       lp_kind_of(M->opt.precision), M->feat[side], M->ldf, st);
    if (e != cudaSuccess) return e;
    train = M->halfsteps[side] < M->opt.mlp_train_iters;
    if (train) {
      x0 = dst32;  // while the net learns, start CG from the previous iterate
    } else {
      if ((e = mlp_infer(M->net[side], S.rows, M->feat[side], M->x0[side], M->f, st)) != cudaSuccess)
        return e;
      x0 = M->x0[side];
    }
  }
  // Autotuner: with solver_groups = 0 each side's first half-steps time the
  // candidate warpgroup counts of the tensor-core kernel (not while a graph is
  // being captured); the faster one is kept for the side.
  als_options o = M->opt;
  bool timing = false;
  if (o.solver_groups == 0 && S.has_plan && lp_kind_of(o.precision) != kLpNone) {
    if (M->tuned[side]) {
      o.solver_groups = M->tuned[side];
    } else {
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      cudaStreamIsCapturing(st, &cs);
      if (cs == cudaStreamCaptureStatusNone && M->tev[0] && M->tev[1]) {
        o.solver_groups = tune_groups(M->f, M->tune_idx[side]);
        timing = true;
      }
    }
  }
  cudaError_t e;
  if (timing && (e = cudaEventRecord(M->tev[0], st)) != cudaSuccess) return e;
  // a learned start is scaled optimally along itself before CG; the previous
  // iterate is used as it is
  const bool learned = M->opt.warm_start == ALS_WARM_MLP && !train;
  e = run_rows(S, M->f, lambda, o, src32, M->f, src_lp, M->lp_ld, dst32, dst_lp, M->ctr, x0,
               learned, M->num_sms, st);
  if (e != cudaSuccess) return e;
  if (timing) {
    float ms = 0.f;
    if ((e = cudaEventRecord(M->tev[1], st)) != cudaSuccess) return e;
    if ((e = cudaEventSynchronize(M->tev[1])) != cudaSuccess) return e;
    if ((e = cudaEventElapsedTime(&ms, M->tev[0], M->tev[1])) != cudaSuccess) return e;
    M->tune_ms[side][M->tune_idx[side]++] = ms;
    if (M->tune_idx[side] == 3) {
      const float t2 = 0.5f * (M->tune_ms[side][0] + M->tune_ms[side][2]), t3 = M->tune_ms[side][1];
      M->tuned[side] = t3 < t2 ? tune_groups(M->f, 1) : tune_groups(M->f, 0);
    }
  }
  if (M->opt.warm_start == ALS_WARM_MLP) {
    if (train)
      e = mlp_train(M->net[side], S.rows, M->opt.mlp_batch, M->opt.mlp_steps, M->feat[side],
                    dst32, M->f, M->opt.mlp_lr, 77ULL + 1000ULL * M->halfsteps[side] + side, st);
    ++M->halfsteps[side];
  }
  return e;
}

int als_model_set_row_range(als_model *M, int32_t side, int64_t begin, int64_t end,
                            cudaStream_t st) {
  if (!M || (side != ALS_SIDE_USERS && side != ALS_SIDE_ITEMS)) return fail(ALS_ERR_INVALID, "bad args");
  Side &S = M->side[side];
  if (begin < 0 || end < begin || end > S.rows) return fail(ALS_ERR_INVALID, "row range outside the side");
  if (M->graph) { cudaGraphExecDestroy(M->graph); M->graph = nullptr; }
  S.begin = begin;
  S.active = end - begin;
  ALS_TRY(launch_degree_order(S.ptr, S.active, S.order, S.queue + 1, st, begin), "row range order");
  if (S.has_plan) {
    // the plan memory is sized for all rows of the side; a launch still
    // reading the old plan is ordered before this one on the stream
    cudaError_t e = plan_ws(S.ptr, begin, S.active, M->num_sms, tc_ws_np(M->f), (int)S.cols,
                            S.plan_mem, S.plan_bytes, &S.plan, &M->ctr->error, st);
    if (e != cudaSuccess) {
      S.has_plan = false;
      return cuda_fail(e, "row range plan");
    }
  }
  return ALS_OK;
}

int als_model_sync_lp(als_model *M, int32_t side, cudaStream_t st) {
  if (!M || (side != ALS_SIDE_USERS && side != ALS_SIDE_ITEMS)) return fail(ALS_ERR_INVALID, "bad args");
  if (!M->X_lp) return ALS_OK;
  const bool users = side == ALS_SIDE_USERS;
  ALS_TRY(launch_convert_lp(users ? M->X : M->T, users ? M->m : M->n, M->f, M->f,
                            users ? M->X_lp : M->T_lp, M->lp_ld, lp_kind_of(M->opt.precision), st),
          "sync low-precision factors");
  return ALS_OK;
}

int als_model_half_step(als_model *M, int32_t side, float lambda, cudaStream_t st) {
  if (!M) return fail(ALS_ERR_INVALID, "null model");
  if (side != ALS_SIDE_USERS && side != ALS_SIDE_ITEMS) return fail(ALS_ERR_INVALID, "bad side");
  if (!(lambda >= 0.f)) return fail(ALS_ERR_INVALID, "lambda must be >= 0");
  ALS_TRY(model_half(M, side, lambda, st), "als_model_half_step");
  return ALS_OK;
}

int als_model_iterate(als_model *M, float lambda, int32_t iters, cudaStream_t st) {
  if (!M) return fail(ALS_ERR_INVALID, "null model");
  if (iters < 0 || !(lambda >= 0.f)) return fail(ALS_ERR_INVALID, "bad iterations or lambda");
  if (!M->opt.use_graph || st == 0 || M->opt.warm_start == ALS_WARM_MLP) {
    for (int it = 0; it < iters; ++it) {
      ALS_TRY(model_half(M, ALS_SIDE_USERS, lambda, st), "iterate (users)");
      ALS_TRY(model_half(M, ALS_SIDE_ITEMS, lambda, st), "iterate (items)");
    }
    return ALS_OK;
  }
  if (!M->graph || M->graph_lambda != lambda) {
    if (M->graph) { cudaGraphExecDestroy(M->graph); M->graph = nullptr; }
    cudaGraph_t g;
    ALS_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t e1 = model_half(M, ALS_SIDE_USERS, lambda, st);
    cudaError_t e2 = e1 == cudaSuccess ? model_half(M, ALS_SIDE_ITEMS, lambda, st) : e1;
    cudaError_t e3 = cudaStreamEndCapture(st, &g);
    if (e2 != cudaSuccess) return cuda_fail(e2, "capture");
    if (e3 != cudaSuccess) return cuda_fail(e3, "end capture");
    cudaError_t e4 = cudaGraphInstantiate(&M->graph, g, 0);
    cudaGraphDestroy(g);
    if (e4 != cudaSuccess) return cuda_fail(e4, "instantiate");
    M->graph_lambda = lambda;
  }
  for (int it = 0; it < iters; ++it) ALS_TRY(cudaGraphLaunch(M->graph, st), "graph launch");
  return ALS_OK;
}

int als_model_factors(als_model *M, float **x, float **t) {
  if (!M) return fail(ALS_ERR_INVALID, "null model");
  if (x) *x = M->X;
  if (t) *t = M->T;
  return ALS_OK;
}

int als_model_row_flags(als_model *M, int32_t side, const uint32_t **flags) {
  if (!M || !flags || (side != 0 && side != 1)) return fail(ALS_ERR_INVALID, "bad args");
  *flags = M->side[side].flags;
  return ALS_OK;
}

int als_model_stats(als_model *M, als_stats *out, int32_t reset) {
  if (!M || !out) return fail(ALS_ERR_INVALID, "bad args");
  Counters c{};
  ALS_TRY(cudaMemcpy(&c, M->ctr, sizeof(c), cudaMemcpyDeviceToHost), "stats");
  std::memset(out, 0, sizeof(*out));
  out->rows_solved = c.rows;
  out->rows_refined = c.refined;
  out->rows_not_spd = c.not_spd;
  out->cg_steps = c.cg_steps;
  out->cg_fallbacks = c.cg_fallback;
  out->kernel_errors = (uint64_t)(c.error != 0);
  out->cg_r0_micro = c.r0_micro;
  out->solver_groups[0] = (uint32_t)M->tuned[0];
  out->solver_groups[1] = (uint32_t)M->tuned[1];
  if (reset) ALS_TRY(cudaMemset(M->ctr, 0, sizeof(Counters)), "stats reset");
  return ALS_OK;
}

int als_model_rmse(als_model *M, int64_t nt, const int32_t *u, const int32_t *i, const float *r,
                   double *out, cudaStream_t st) {
  if (!M || !out || nt < 0 || (nt > 0 && (!u || !i || !r))) return fail(ALS_ERR_INVALID, "bad args");
  ALS_TRY(launch_rmse(nt, u, i, r, M->X, M->f, M->T, M->f, M->f, M->rmse_dev, M->rmse_work, st),
          "rmse");
  ALS_TRY(cudaMemcpyAsync(out, M->rmse_dev, sizeof(double), cudaMemcpyDeviceToHost, st), "rmse copy");
  ALS_TRY(cudaStreamSynchronize(st), "rmse sync");
  return ALS_OK;
}

struct als_mlp {
  void *net = nullptr;
  int f = 0;
};

int als_mlp_create(als_mlp **out, int32_t f, int64_t cap, uint64_t seed, cudaStream_t st) {
  if (!out || f <= 0 || f > 128 || cap < 64) return fail(ALS_ERR_INVALID, "bad MLP arguments");
  als_mlp *p = new als_mlp();
  p->f = f;
  cudaError_t e = mlp_create(&p->net, f, cap, seed, st);
  if (e != cudaSuccess) { delete p; return cuda_fail(e, "als_mlp_create"); }
  *out = p;
  return ALS_OK;
}
void als_mlp_destroy(als_mlp *p) {
  if (!p) return;
  mlp_destroy(p->net);
  delete p;
}
int als_mlp_feature_stride(const als_mlp *p) { return p ? mlp_ldf(p->net) : 0; }
int64_t als_mlp_param_count(int32_t f) { return f > 0 ? mlp_param_count(f) : 0; }
int als_mlp_get_params(als_mlp *p, float *host, cudaStream_t st) {
  if (!p || !host) return fail(ALS_ERR_INVALID, "bad args");
  ALS_TRY(mlp_io(p->net, host, 0, nullptr, st), "als_mlp_get_params");
  return ALS_OK;
}
int als_mlp_set_params(als_mlp *p, const float *host, cudaStream_t st) {
  if (!p || !host) return fail(ALS_ERR_INVALID, "bad args");
  ALS_TRY(mlp_io(p->net, const_cast<float *>(host), 2, nullptr, st), "als_mlp_set_params");
  return ALS_OK;
}
int als_mlp_gradients(als_mlp *p, int64_t B, const void *F, const float *T, int32_t ldt,
                      float *host, double *loss, cudaStream_t st) {
  if (!p || !F || !T || !host || B < 64 || B % 64 || ldt < p->f) return fail(ALS_ERR_INVALID, "bad args");
  ALS_TRY(mlp_gradients(p->net, B, F, T, ldt, st), "als_mlp_gradients");
  ALS_TRY(mlp_io(p->net, host, 1, loss, st), "als_mlp_gradients: copy");
  return ALS_OK;
}
int als_mlp_train_step(als_mlp *p, int64_t B, const void *F, const float *T, int32_t ldt, float lr,
                       cudaStream_t st) {
  if (!p || !F || !T || B < 64 || B % 64 || ldt < p->f) return fail(ALS_ERR_INVALID, "bad args");
  ALS_TRY(mlp_step(p->net, B, F, T, ldt, lr, st), "als_mlp_train_step");
  return ALS_OK;
}
int als_mlp_forward(als_mlp *p, int64_t rows, const void *F, float *out, int32_t ldo,
                    cudaStream_t st) {
  if (!p || !F || !out || rows < 0 || ldo < p->f) return fail(ALS_ERR_INVALID, "bad args");
  ALS_TRY(mlp_infer(p->net, rows, F, out, ldo, st), "als_mlp_forward");
  return ALS_OK;
}
int als_features(int64_t m, int32_t f, const int64_t *ptr, const int32_t *col, const float *val,
                 const void *src, int32_t ld_src, int32_t prec, void *F, int32_t ldf,
                 cudaStream_t st) {
  if (m < 0 || f <= 0 || f > 128 || !ptr || !src || !F || ld_src < f || ldf < 2 * f + 1)
    return fail(ALS_ERR_INVALID, "bad args");
  const int kind = lp_kind_of(prec);
  if (m > 0 && kind != kLpNone && ld_src % 8 == 0) {
    // the model's path: a work plan over the rows (long rows split), then the plan kernel
    WsPlan plan;
    void *mem = nullptr;
    const size_t bytes = plan_ws_bytes(m, device_sm_count(), 128);
    cudaError_t e = cudaMalloc(&mem, bytes);
    if (e == cudaSuccess)
      e = plan_ws(ptr, 0, m, device_sm_count(), 128, 0, mem, bytes, &plan, nullptr, st);
    if (e == cudaSuccess) e = mlp_features_plan(plan, f, col, val, src, ld_src, kind, F, ldf, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(mem);
    if (e != cudaErrorNotSupported) {
      ALS_TRY(e, "als_features");
      return ALS_OK;
    }
  }
  ALS_TRY(mlp_features(m, f, ptr, col, val, src, ld_src, kind, F, ldf, st), "als_features");
  return ALS_OK;
}

size_t als_half_step_work_bytes(int64_t m) {
  return align_up(sizeof(int32_t) * (size_t)(m > 0 ? m : 0), 256) +
         align_up(sizeof(unsigned) * (1 + 3 * kOrderBins), 256) + align_up(sizeof(Counters), 256);
}

int als_half_step(int64_t m, int64_t n, int32_t f, const int64_t *ptr, const int32_t *col,
                  const float *val, const float *src, int32_t ld_src, float *dst, int32_t ld_dst,
                  float lambda, const als_options *opt, void *work, size_t work_bytes,
                  cudaStream_t st) {
  if (m < 0 || n <= 0 || f <= 0 || m > INT32_MAX) return fail(ALS_ERR_INVALID, "bad sizes");
  if (m == 0) return ALS_OK;
  if (!ptr || !src || !dst || !work || ld_src < f || ld_dst < f)
    return fail(ALS_ERR_INVALID, "bad pointers or strides");
  if (work_bytes < als_half_step_work_bytes(m)) return fail(ALS_ERR_INVALID, "workspace too small");
  als_options o;
  als_default_options(&o);
  if (opt) o = *opt;
  if (o.precision != ALS_PREC_FP32)
    return fail(ALS_ERR_UNSUPPORTED, "als_half_step takes FP32 factors; use a model for BF16/FP16");
  int rc = check_options(o, f);
  if (rc != ALS_OK) return rc;
  char *b = static_cast<char *>(work);
  Side s;
  s.rows = m; s.cols = n; s.ptr = ptr; s.idx = col; s.val = val;
  s.order = (int32_t *)b;
  s.queue = (unsigned *)(b + align_up(sizeof(int32_t) * m, 256));
  Counters *ctr = (Counters *)((char *)s.queue + align_up(sizeof(unsigned) * (1 + 3 * kOrderBins), 256));
  ALS_TRY(cudaMemsetAsync(ctr, 0, sizeof(Counters), st), "half step");
  ALS_TRY(launch_degree_order(ptr, m, s.order, s.queue + 1, st), "degree order");
  RowsArgs a{};
  a.m = m; a.f = f; a.lambda = lambda; a.row_ptr = ptr; a.col = col; a.val = val;
  a.src = src; a.ld_src = ld_src; a.dst = dst; a.ld_dst = ld_dst;
  a.order = s.order; a.queue = s.queue; a.counters = ctr; a.refine_tol = o.refine_tol;
  ALS_TRY(cudaMemsetAsync(s.queue, 0, sizeof(unsigned), st), "half step");
  ALS_TRY(launch_rows_fp32(a, kLpNone, device_sm_count(), st), "half step");
  return ALS_OK;
}

size_t als_rmse_work_bytes(void) { return rmse_work_bytes() + 256; }

int als_rmse(int64_t nt, const int32_t *u, const int32_t *i, const float *r, const float *x,
             int32_t ldx, const float *t, int32_t ldt, int32_t f, double *out, void *work,
             size_t work_bytes, cudaStream_t st) {
  if (!out || !work || nt < 0 || f <= 0 || ldx < f || ldt < f) return fail(ALS_ERR_INVALID, "bad args");
  if (work_bytes < als_rmse_work_bytes()) return fail(ALS_ERR_INVALID, "workspace too small");
  double *dev = (double *)((char *)work + rmse_work_bytes());
  ALS_TRY(launch_rmse(nt, u, i, r, x, ldx, t, ldt, f, dev, work, st), "rmse");
  ALS_TRY(cudaMemcpyAsync(out, dev, sizeof(double), cudaMemcpyDeviceToHost, st), "rmse copy");
  ALS_TRY(cudaStreamSynchronize(st), "rmse sync");
  return ALS_OK;
}

int als_predict(int64_t nt, const int32_t *u, const int32_t *i, const float *x, int32_t ldx,
                const float *t, int32_t ldt, int32_t f, float *out, cudaStream_t st) {
  if (nt < 0 || f <= 0 || ldx < f || ldt < f || (nt > 0 && (!u || !i || !x || !t || !out)))
    return fail(ALS_ERR_INVALID, "bad args");
  ALS_TRY(launch_predict(nt, u, i, x, ldx, t, ldt, f, out, st), "predict");
  return ALS_OK;
}

int als_topk(int64_t nq, const int32_t *users, const float *x, int32_t ldx, const float *t,
             int32_t ldt, int64_t n, int32_t f, int32_t k, const int64_t *seen_ptr,
             const int32_t *seen_col, int32_t *items, float *scores, cudaStream_t st) {
  if (nq < 0 || n < 0 || f < 1 || f > 128 || k < 1 || k > 256 || ldx < f || ldt < f ||
      n > INT32_MAX - 1 || (nq > 0 && (!users || !x || !t || !items || !scores)) ||
      ((seen_ptr == nullptr) != (seen_col == nullptr)))
    return fail(ALS_ERR_INVALID, "als_topk: bad args (1 <= k <= 256, 1 <= f <= 128)");
  ALS_TRY(launch_topk(nq, users, x, ldx, t, ldt, n, f, k, seen_ptr, seen_col, items, scores, st),
          "als_topk");
  return ALS_OK;
}

int als_csr_to_csc(int64_t m, int64_t n, int64_t nnz, const int64_t *ptr, const int32_t *col,
                   const float *val, int64_t *cptr, int32_t *crow, float *cval, cudaStream_t st) {
  if (m < 0 || n < 0 || nnz < 0 || m > INT32_MAX || n > INT32_MAX || !ptr || !cptr ||
      (nnz > 0 && (!col || !val || !crow || !cval)))
    return fail(ALS_ERR_INVALID, "als_csr_to_csc: bad args");
  ALS_TRY(csr_to_csc(m, n, nnz, ptr, col, val, cptr, crow, cval, st), "als_csr_to_csc");
  return ALS_OK;
}

int als_train(const int64_t *csr_ptr, const int32_t *csr_col, const float *csr_val,
              const int64_t *csc_ptr, const int32_t *csc_row, const float *csc_val, int64_t m,
              int64_t n, int32_t f, int64_t nnz, float lambda, int32_t iterations,
              const als_options *opt, float *X_out, float *theta_inout, als_stats *stats) {
  if (!csr_ptr || !csc_ptr || !X_out || !theta_inout || m <= 0 || n <= 0 || f <= 0 || nnz < 0)
    return fail(ALS_ERR_INVALID, "bad args");
  if (csr_ptr[m] != nnz || csc_ptr[n] != nnz) return fail(ALS_ERR_INVALID, "nnz does not match pointers");
  cudaStream_t st = 0;
  char *d = nullptr;
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t p = off; off = align_up(off + bytes, 256); return p; };
  const size_t o1 = take(8 * (m + 1)), o2 = take(4 * nnz), o3 = take(4 * nnz), o4 = take(8 * (n + 1)),
               o5 = take(4 * nnz), o6 = take(4 * nnz), o7 = take(4ull * n * f);
  ALS_TRY(cudaMalloc(&d, off), "als_train: cudaMalloc");
  auto cleanup = [&]() { cudaFree(d); };
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMemcpy(d + o1, csr_ptr, 8 * (m + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nnz) e = cudaMemcpy(d + o2, csr_col, 4 * nnz, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nnz) e = cudaMemcpy(d + o3, csr_val, 4 * nnz, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o4, csc_ptr, 8 * (n + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nnz) e = cudaMemcpy(d + o5, csc_row, 4 * nnz, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nnz) e = cudaMemcpy(d + o6, csc_val, 4 * nnz, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o7, theta_inout, 4ull * n * f, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { cleanup(); return cuda_fail(e, "als_train: upload"); }
  als_model *M = nullptr;
  int rc = als_model_create(&M, m, n, f, nnz, (int64_t *)(d + o1), (int32_t *)(d + o2),
                            (float *)(d + o3), (int64_t *)(d + o4), (int32_t *)(d + o5),
                            (float *)(d + o6), opt, st);
  if (rc == ALS_OK) rc = als_model_set_theta(M, (float *)(d + o7), f, st);
  if (rc == ALS_OK) rc = als_model_iterate(M, lambda, iterations, st);
  if (rc == ALS_OK) {
    e = cudaMemcpy(X_out, M->X, 4ull * m * f, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(theta_inout, M->T, 4ull * n * f, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = cuda_fail(e, "als_train: download");
  }
  if (rc == ALS_OK && stats) rc = als_model_stats(M, stats, 0);
  als_model_destroy(M);
  cleanup();
  return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Drop-in entry points of the reference.
// ---------------------------------------------------------------------------
namespace {
// Cache of device blocks behind mallocBest / freeBest and the drop-in
// half-step's workspace. The Spark flow allocates and frees the three CSR
// arrays and the half-step's scratch on every call (hundreds of MB each at the
// Netflix shape): cudaMalloc / cudaFree of such blocks take milliseconds each,
// and cudaFree synchronises the device. A freed block is kept for its device
// (at most kCacheMax bytes per device; the largest blocks are released first
// beyond that) and handed out again to a request of at least half its size.
// When cudaMalloc fails, the device's cached blocks are released and the
// allocation is tried once more before mallocBest falls back to mapped host
// memory. The cache is never destroyed: static destructors run after the CUDA
// runtime may already be gone, and the driver reclaims the memory at exit.
constexpr size_t kBlockGranule = 2u << 20;
constexpr size_t kCacheMax = 8ull << 30;
constexpr int kCacheDevices = 64;

struct BlockCache {
  std::mutex mu;
  std::multimap<size_t, void *> idle[kCacheDevices];  // capacity -> block
  size_t idle_bytes[kCacheDevices] = {};
  std::unordered_map<void *, std::pair<int, size_t>> live;  // block -> (device, capacity)
};

BlockCache &block_cache() {
  static BlockCache *c = new BlockCache();
  return *c;
}

// cudaFree of every idle block of device `dev` (the caller holds the lock).
void release_idle(BlockCache &c, int dev) {
  for (auto &kv : c.idle[dev]) cudaFree(kv.second);
  c.idle[dev].clear();
  c.idle_bytes[dev] = 0;
}

// A device block of at least `bytes` on the current device.
cudaError_t block_alloc(void **out, size_t bytes) {
  *out = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const size_t cap = (std::max<size_t>(bytes, 1) + kBlockGranule - 1) / kBlockGranule * kBlockGranule;
  BlockCache &c = block_cache();
  if (dev >= 0 && dev < kCacheDevices) {
    std::lock_guard<std::mutex> lk(c.mu);
    auto it = c.idle[dev].lower_bound(cap);
    if (it != c.idle[dev].end() && it->first / 2 <= cap) {
      *out = it->second;
      c.live[it->second] = {dev, it->first};
      c.idle_bytes[dev] -= it->first;
      c.idle[dev].erase(it);
      return cudaSuccess;
    }
  }
  void *p = nullptr;
  e = cudaMalloc(&p, cap);
  if (e == cudaErrorMemoryAllocation && dev >= 0 && dev < kCacheDevices) {
    cudaGetLastError();
    {
      std::lock_guard<std::mutex> lk(c.mu);
      release_idle(c, dev);
    }
    e = cudaMalloc(&p, cap);
  }
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < kCacheDevices) {
    std::lock_guard<std::mutex> lk(c.mu);
    c.live[p] = {dev, cap};
  }
  *out = p;
  return cudaSuccess;
}

// Return a block of block_alloc to the cache. false: not such a block. With
// sync_device, the block's device is synchronised first, as cudaFree would
// do, so work still queued on it cannot race a later owner.
bool block_release(void *p, bool sync_device) {
  BlockCache &c = block_cache();
  int dev = -1;
  size_t cap = 0;
  {
    std::lock_guard<std::mutex> lk(c.mu);
    auto it = c.live.find(p);
    if (it == c.live.end()) return false;
    dev = it->second.first;
    cap = it->second.second;
    c.live.erase(it);
  }
  if (sync_device) {
    int cur = 0;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != dev) {
      cudaSetDevice(dev);
      cudaDeviceSynchronize();
      cudaSetDevice(cur);
    } else {
      cudaDeviceSynchronize();
    }
  }
  std::lock_guard<std::mutex> lk(c.mu);
  c.idle[dev].insert({cap, p});
  c.idle_bytes[dev] += cap;
  while (c.idle_bytes[dev] > kCacheMax && !c.idle[dev].empty()) {
    auto big = std::prev(c.idle[dev].end());
    cudaFree(big->second);
    c.idle_bytes[dev] -= big->first;
    c.idle[dev].erase(big);
  }
  return true;
}

cudaError_t free_best(void *devPtr, bool sync_device) {
  if (!devPtr) return cudaSuccess;
  if (block_release(devPtr, sync_device)) return cudaSuccess;
  cudaPointerAttributes attr;
  cudaError_t e = cudaPointerGetAttributes(&attr, devPtr);
  if (e != cudaSuccess) return e;
  if (attr.type == cudaMemoryTypeDevice) return cudaFree(devPtr);
  // mapped host memory: free through its host address
  return cudaFreeHost(attr.hostPointer ? attr.hostPointer : devPtr);
}
}  // namespace

// C++ linkage, as the reference's utilities.h:36-41 declares them.
cudaError_t mallocBest(void **devPtr, size_t size) {
  if (!devPtr) return cudaErrorInvalidValue;
  if (block_alloc(devPtr, size) == cudaSuccess) return cudaSuccess;
  cudaGetLastError();  // clear the allocation failure
  void *h = nullptr;
  cudaError_t e = cudaHostAlloc(&h, size, cudaHostAllocMapped | cudaHostAllocWriteCombined);
  if (e != cudaSuccess) return e;
  return cudaHostGetDevicePointer(devPtr, h, 0);
}

cudaError_t freeBest(void *devPtr) { return free_best(devPtr, true); }

extern "C" {

cudaError_t als_malloc_best(void **devPtr, size_t size) { return mallocBest(devPtr, size); }
cudaError_t als_free_best(void *devPtr) { return freeBest(devPtr); }

int get_gpu(void) {
  static std::once_flag once;
  static int count = 0;
  static std::atomic<int> next{0};
  std::call_once(once, []() {
    if (cudaGetDeviceCount(&count) != cudaSuccess || count < 0) {
      cudaGetLastError();
      count = 0;
    }
  });
  if (count <= 0) return -1;
  if (count == 1) return 0;
  return next.fetch_add(1) % count;
}

}  // extern "C"

static void throw_cuda(cudaError_t e, const char *where) {
  std::fprintf(stderr, "CUDA Error: %s: %s\n", where, cudaGetErrorString(e));
  throw thrust::system_error(e, thrust::cuda_category(), cudaGetErrorString(e));
}

namespace als {
bool debug_take_withhold() { return debug_withhold().exchange(false); }

// The drop-in call's check of the kernels' error word after a half-step:
// results of a half-step whose kernel gave up a bounded wait (bit 1), or whose
// work plan was rejected for malformed row pointers (bit 2), are incomplete,
// so the call throws like any other CUDA failure instead of returning them.
void dropin_raise_on_kernel_error(int error_word) {
  if (error_word == 0) return;
  const char *what = (error_word & 1)
                         ? "doALSWithCSR: a kernel gave up a bounded wait (bounded wait timed out); "
                           "the half-step's rows are incomplete"
                         : "doALSWithCSR: malformed CSR row pointers; the half-step was not run";
  std::fprintf(stderr, "CUDA Error: %s\n", what);
  throw thrust::system_error(cudaErrorLaunchFailure, thrust::cuda_category(), what);
}
}  // namespace als

namespace {
// Host <-> device copies of the drop-in's theta and X. Callers (the JNI shim,
// Python) usually pass pageable host memory, which the DMA engines reach only
// through the driver's small bounce buffers: 4-11 GB/s measured at 192 MB on
// a B200 box. Large pageable copies therefore go through pinned staging:
// kStageWorkers host threads each own two kStageChunk halves and take every
// kStageWorkers-th chunk, so the host-side copies (and the first-touch page
// faults of a fresh destination) run in parallel while the DMAs, all issued
// on the caller's stream, run back to back. Each worker's host copy of one
// chunk overlaps the DMA of its other half. The halves are allocated once per
// process (portable, so any device can use them) and shared by calls under a
// mutex; pinned or device memory is copied directly.
constexpr size_t kStageChunk = 8u << 20;
constexpr int kStageWorkers = 4;
constexpr size_t kStageMin = 32u << 20;  // smaller copies go directly
std::mutex g_stage_mu;
char *g_stage = nullptr;

bool pageable(const void *p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return at.type == cudaMemoryTypeUnregistered;
}

// Worker w: chunks w, w + W, w + 2W, ... of the copy through its two halves.
// A new thread starts on device 0: it selects the caller's device first, so
// its events and the legacy default stream (st == 0) are the caller's.
cudaError_t stage_worker(int w, int dev, char *d, const char *s, size_t bytes, bool to_device,
                         cudaStream_t st) {
  const cudaMemcpyKind kind = to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
  char *halves = g_stage + (size_t)w * 2 * kStageChunk;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaError_t e = cudaSetDevice(dev);
  for (int h = 0; h < 2 && e == cudaSuccess; ++h)
    e = cudaEventCreateWithFlags(&ev[h], cudaEventDisableTiming);
  size_t prev_off = 0, prev_len = 0;
  int prev_h = 0;
  const size_t step = (size_t)kStageWorkers * kStageChunk;
  size_t j = 0;
  for (size_t off = (size_t)w * kStageChunk; e == cudaSuccess && off < bytes; off += step, ++j) {
    const int h = (int)(j & 1);
    const size_t len = std::min(kStageChunk, bytes - off);
    char *half = halves + h * kStageChunk;
    if (to_device) {
      if (j >= 2 && (e = cudaEventSynchronize(ev[h])) != cudaSuccess) break;  // half free again
      std::memcpy(half, s + off, len);
      if ((e = cudaMemcpyAsync(d + off, half, len, kind, st)) != cudaSuccess) break;
      e = cudaEventRecord(ev[h], st);
    } else {
      if ((e = cudaMemcpyAsync(half, s + off, len, kind, st)) != cudaSuccess) break;
      if ((e = cudaEventRecord(ev[h], st)) != cudaSuccess) break;
      if (prev_len) {  // the previous chunk has landed in the other half: hand it over
        if ((e = cudaEventSynchronize(ev[prev_h])) != cudaSuccess) break;
        std::memcpy(d + prev_off, halves + prev_h * kStageChunk, prev_len);
      }
      prev_off = off;
      prev_len = len;
      prev_h = h;
    }
  }
  // wait for this worker's last DMAs (the halves are then free), hand over the last chunk
  for (int h = 0; h < 2; ++h)
    if (ev[h]) {
      const cudaError_t e2 = cudaEventSynchronize(ev[h]);
      if (e == cudaSuccess) e = e2;
    }
  if (e == cudaSuccess && !to_device && prev_len)
    std::memcpy(d + prev_off, halves + prev_h * kStageChunk, prev_len);
  for (int h = 0; h < 2; ++h)
    if (ev[h]) cudaEventDestroy(ev[h]);
  return e;
}

cudaError_t staged_copy(void *dst, const void *src, size_t bytes, bool to_device, cudaStream_t st) {
  const cudaMemcpyKind kind = to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
  if (bytes < kStageMin || !pageable(to_device ? src : dst))
    return cudaMemcpyAsync(dst, src, bytes, kind, st);
  std::lock_guard<std::mutex> lk(g_stage_mu);
  if (!g_stage && cudaHostAlloc((void **)&g_stage, 2 * kStageChunk * kStageWorkers,
                                cudaHostAllocPortable) != cudaSuccess) {
    g_stage = nullptr;
    cudaGetLastError();
    return cudaMemcpyAsync(dst, src, bytes, kind, st);  // no pinned memory: copy directly
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return cudaGetLastError();
  cudaError_t err[kStageWorkers];
  auto work = [&](int w) {
    err[w] = stage_worker(w, dev, static_cast<char *>(dst), static_cast<const char *>(src), bytes,
                          to_device, st);
  };
  std::vector<std::thread> pool;
  pool.reserve(kStageWorkers - 1);
  try {
    for (int w = 1; w < kStageWorkers; ++w) pool.emplace_back(work, w);
  } catch (...) {  // no thread: this one takes the chunks of the workers never started
    for (int w = 1 + (int)pool.size(); w < kStageWorkers; ++w) work(w);
  }
  work(0);
  for (auto &t : pool) t.join();
  for (int w = 0; w < kStageWorkers; ++w)
    if (err[w] != cudaSuccess) return err[w];
  return cudaSuccess;
}

// The drop-in call's workspace, leased from the block cache and given back
// when the call ends; on an exception the stream is synchronised first, so no
// queued kernel still uses the block when the next caller gets it.
struct WorkspaceLease {
  char *d = nullptr;
  cudaStream_t st;
  explicit WorkspaceLease(cudaStream_t s) : st(s) {}
  ~WorkspaceLease() {
    if (!d) return;
    if (std::uncaught_exceptions() > 0) {
      cudaStreamSynchronize(st);
      cudaGetLastError();
    }
    block_release(d, false);
  }
};

// The CSR arrays the call owns (reference als.cu:1058, 1101-1102): freed on
// the normal path with their errors checked, and on an exception too (errors
// ignored) so a failed call does not leak them.
struct CsrOwnership {
  void *p[3];
  cudaStream_t st;
  bool done = false;
  ~CsrOwnership() {
    if (done) return;
    cudaStreamSynchronize(st);
    cudaGetLastError();
    for (void *q : p) free_best(q, false);
    cudaGetLastError();
  }
};
}  // namespace

#define DROPIN_CALL(call, where)           \
  do {                                     \
    cudaError_t e_ = (call);               \
    if (e_ != cudaSuccess) throw_cuda(e_, where); \
  } while (0)

extern "C" void doALSWithCSR(cudaStream_t st, int *csrRowIndex, int *csrColIndex, float *csrVal,
                             float *thetaTHost, float *XTHost, const int m, const int n,
                             const int f, const long nnz, const float lambda, const int X_BATCH) {
  (void)X_BATCH;
  CsrOwnership csr{{csrVal, csrRowIndex, csrColIndex}, st};
  als_options o;
  als_get_dropin_options(&o);
  if (o.warm_start == ALS_WARM_PREVIOUS) o.warm_start = ALS_WARM_ZERO;  // no previous X here
  if (m < 0 || n <= 0 || f <= 0 || nnz < 0) throw_cuda(cudaErrorInvalidValue, "doALSWithCSR: sizes");
  if (check_options(o, f) != ALS_OK) throw_cuda(cudaErrorInvalidValue, als_last_error());
  const int kind = lp_kind_of(o.precision);
  const int ldp = kind ? tc_padded_ld(f) : 0;
  const int sms = device_sm_count();
  const bool ws = kind != kLpNone && tc_ws_takes(f, o.solver, o.cg_jacobi) && m > 0;
  // device buffers: theta (+ low-precision copy), X, widened row pointers,
  // order/queue/counters, the work plan of the warp-specialised kernel
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t p = off; off = align_up(off + bytes, 256); return p; };
  const size_t oT = take(sizeof(float) * (size_t)n * f), oX = take(sizeof(float) * (size_t)m * f + 4),
               oP = take(sizeof(int64_t) * ((size_t)m + 1)), oW = take(als_half_step_work_bytes(m)),
               oL = take(kind ? 2ull * n * ldp : 0),
               oPl = take(ws ? plan_ws_bytes(m, sms, tc_ws_np(f)) : 0);
  WorkspaceLease lease(st);
  void *blk = nullptr;
  DROPIN_CALL(block_alloc(&blk, off), "doALSWithCSR: workspace");
  lease.d = static_cast<char *>(blk);
  char *d = lease.d;
  DROPIN_CALL(staged_copy(d + oT, thetaTHost, sizeof(float) * (size_t)n * f, true, st),
              "doALSWithCSR: theta upload");
  DROPIN_CALL(launch_widen_ptr(csrRowIndex, (int64_t)m + 1, (int64_t *)(d + oP), st),
              "doALSWithCSR: row pointers");
  int kernel_error = 0;
  if (m > 0 && kind == kLpNone) {
    int rc = als_half_step(m, n, f, (const int64_t *)(d + oP), csrColIndex, csrVal,
                           (const float *)(d + oT), f, (float *)(d + oX), f, lambda, &o, d + oW,
                           als_half_step_work_bytes(m), st);
    if (rc != ALS_OK) {
      cudaError_t e = cudaGetLastError();
      throw_cuda(e != cudaSuccess ? e : cudaErrorInvalidValue, als_last_error());
    }
  } else if (m > 0) {
    // tensor-core form: low-precision copy of theta, a work plan built on the
    // device, one launch
    DROPIN_CALL(launch_convert_lp((const float *)(d + oT), n, f, f, d + oL, ldp, kind, st),
                "doALSWithCSR: theta copy");
    Side S;
    S.rows = m; S.cols = n; S.active = m; S.ptr = (const int64_t *)(d + oP);
    S.idx = csrColIndex; S.val = csrVal;
    char *w = d + oW;
    S.order = (int32_t *)w;
    S.queue = (unsigned *)(w + align_up(sizeof(int32_t) * m, 256));
    Counters *ctr = (Counters *)((char *)S.queue + align_up(sizeof(unsigned) * (1 + 3 * kOrderBins), 256));
    DROPIN_CALL(cudaMemsetAsync(ctr, 0, sizeof(Counters), st), "doALSWithCSR: counters");
    DROPIN_CALL(launch_degree_order(S.ptr, m, S.order, S.queue + 1, st), "doALSWithCSR: order");
    if (ws) {
      DROPIN_CALL(plan_ws(S.ptr, 0, m, sms, tc_ws_np(f), n, d + oPl, plan_ws_bytes(m, sms, tc_ws_np(f)),
                          &S.plan, &ctr->error, st),
                  "doALSWithCSR: plan");
      S.has_plan = true;
    }
    DROPIN_CALL(run_rows(S, f, lambda, o, (const float *)(d + oT), f, d + oL, ldp, (float *)(d + oX),
                         nullptr, ctr, nullptr, false, sms, st),
                "doALSWithCSR: tensor-core half-step");
    DROPIN_CALL(cudaMemcpyAsync(&kernel_error, &ctr->error, sizeof(int), cudaMemcpyDeviceToHost, st),
                "doALSWithCSR: error word");
  }
  if (m > 0)
    DROPIN_CALL(staged_copy(XTHost, d + oX, sizeof(float) * (size_t)m * f, false, st),
                "doALSWithCSR: X download");
  DROPIN_CALL(cudaStreamSynchronize(st), "doALSWithCSR: sync");
  dropin_raise_on_kernel_error(kernel_error);
  // The callee owns and frees the CSR arrays (reference als.cu:1058, 1101-1102).
  csr.done = true;
  DROPIN_CALL(free_best(csrVal, false), "doALSWithCSR: free csrVal");
  DROPIN_CALL(free_best(csrRowIndex, false), "doALSWithCSR: free csrRowIndex");
  DROPIN_CALL(free_best(csrColIndex, false), "doALSWithCSR: free csrColIndex");
}

// ---------------------------------------------------------------------------
// als_half_step_host: the drop-in half-step on HOST CSR arrays, i.e. the whole
// path of the Spark JNI call, which uploads the three arrays into mallocBest
// memory (CuMFJNIInterface.cpp:93-118) before doALSWithCSR uploads theta,
// solves and downloads X, each transfer waiting for the one before. Here the
// ratings cross PCIe in row ranges by rating count on a copy
// stream; each range is planned and solved on the caller's stream as soon as
// it has landed, and its rows of X go back on a third stream while the next
// range is solved. At the Netflix shape a side's ratings (0.8 GB) take about
// as long to upload as the users side takes to solve, so the half-step costs
// about the longer of the two instead of their sum.
// ---------------------------------------------------------------------------
namespace {
constexpr int kHostChunksMax = 16;
// Automatic range counts. A side of short rows (more than one row per 1,000
// ratings: the users side of the benchmark matrices) is bound by its solve,
// and finer ranges hide more of the upload behind it (Netflix shape, users
// half-step: 17.7 ms with 8 ranges, 17.1 with 12); a side of long rows is
// bound by its upload, where more ranges only add their overhead (items
// half-step: 18.9 ms with 8, 19.2 with 12).
constexpr long kHostChunkRatings = 12500000;       // about this many ratings a range
constexpr long kHostChunkRatingsShort = 8300000;   // the same for sides of short rows

// The streams, events and workspace of one call. The destructor waits for all
// three streams before the workspace goes back to the cache, on every path.
struct HostPipe {
  cudaStream_t st, up = nullptr, dn = nullptr;
  std::vector<cudaEvent_t> ev;
  char *d = nullptr;
  explicit HostPipe(cudaStream_t s) : st(s) {}
  cudaError_t init(int events) {
    cudaError_t e = cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&dn, cudaStreamNonBlocking);
    for (int i = 0; i < events && e == cudaSuccess; ++i) {
      cudaEvent_t x = nullptr;
      e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
      if (e == cudaSuccess) ev.push_back(x);
    }
    return e;
  }
  HostPipe(const HostPipe &) = delete;
  HostPipe &operator=(const HostPipe &) = delete;
  ~HostPipe() {
    if (up) cudaStreamSynchronize(up);
    cudaStreamSynchronize(st);
    if (dn) cudaStreamSynchronize(dn);
    if (d) block_release(d, false);
    for (cudaEvent_t x : ev) cudaEventDestroy(x);
    if (up) cudaStreamDestroy(up);
    if (dn) cudaStreamDestroy(dn);
  }
};

// Row ranges [b[c], b[c + 1]) by rating count, the first and the last half
// the size of the others: nothing can be solved before the first range has
// landed, and the last range's solve and download follow the last upload, so
// those two are the parts of the pipeline that do not overlap. Empty ranges
// are dropped; the row pointers are non-decreasing and end at nnz.
std::vector<int> host_ranges(const int *row_ptr, int m, long nnz, int chunks) {
  std::vector<int> b{0};
  for (int c = 1; c < chunks; ++c) {
    const int target = (int)(nnz * (2L * c - 1) / (2L * (chunks - 1)));
    const int r = (int)(std::lower_bound(row_ptr, row_ptr + m + 1, target) - row_ptr);
    if (r > b.back() && r < m) b.push_back(r);
  }
  b.push_back(m);
  return b;
}
}  // namespace

extern "C" int als_half_step_host(cudaStream_t st, const int *h_row_ptr, const int *h_col,
                                  const float *h_val, const float *thetaTHost, float *XTHost,
                                  int m, int n, int f, long nnz, float lambda, int chunks) {
  if (!h_row_ptr || !thetaTHost || m < 0 || n <= 0 || f <= 0 || nnz < 0 || nnz > INT32_MAX ||
      (m > 0 && !XTHost) || (nnz > 0 && (!h_col || !h_val)) || chunks < 0 ||
      chunks > kHostChunksMax)
    return fail(ALS_ERR_INVALID, "als_half_step_host: bad arguments");
  if (h_row_ptr[0] != 0 || (long)h_row_ptr[m] != nnz)
    return fail(ALS_ERR_INVALID, "als_half_step_host: the row pointers do not span nnz ratings");
  for (int i = 0; i < m; ++i)
    if (h_row_ptr[i + 1] < h_row_ptr[i])
      return fail(ALS_ERR_INVALID, "als_half_step_host: decreasing row pointer");
  als_options o;
  als_get_dropin_options(&o);
  if (o.warm_start == ALS_WARM_PREVIOUS) o.warm_start = ALS_WARM_ZERO;  // no previous X here
  if (int rc = check_options(o, f); rc != ALS_OK) return rc;
  if (m == 0) return ALS_OK;
  const bool short_rows = (long)m * 1000 > nnz;
  const long per = short_rows ? kHostChunkRatingsShort : kHostChunkRatings;
  const int K = chunks ? chunks
                       : (int)std::min<long>(short_rows ? 12 : 8,
                                             std::max<long>(1, (nnz + per - 1) / per));
  const std::vector<int> rb = host_ranges(h_row_ptr, m, nnz, K);
  const int nch = (int)rb.size() - 1;
  const int kind = lp_kind_of(o.precision);
  const int ldp = kind ? tc_padded_ld(f) : 0;
  const int sms = device_sm_count();
  const bool ws = kind != kLpNone && tc_ws_takes(f, o.solver, o.cg_jacobi);
  const int np = ws ? tc_ws_np(f) : 0;
  // the drop-in's workspace, then the CSR arrays
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t p = off; off = align_up(off + bytes, 256); return p; };
  const size_t oT = take(sizeof(float) * (size_t)n * f), oX = take(sizeof(float) * (size_t)m * f + 4),
               oP = take(sizeof(int64_t) * ((size_t)m + 1)), oW = take(als_half_step_work_bytes(m)),
               oL = take(kind ? 2ull * n * ldp : 0), oPl = take(ws ? plan_ws_bytes(m, sms, np) : 0),
               oR = take(sizeof(int) * ((size_t)m + 1)),
               oC = take(sizeof(int) * (size_t)std::max<long>(nnz, 1)),
               oV = take(sizeof(float) * (size_t)std::max<long>(nnz, 1));
  HostPipe p(st);
  ALS_TRY(p.init(1 + 2 * nch), "als_half_step_host: streams");
  void *blk = nullptr;
  ALS_TRY(block_alloc(&blk, off), "als_half_step_host: workspace");
  p.d = static_cast<char *>(blk);
  char *d = p.d;
  int *d_row = reinterpret_cast<int *>(d + oR), *d_col = reinterpret_cast<int *>(d + oC);
  float *d_val = reinterpret_cast<float *>(d + oV), *d_x = reinterpret_cast<float *>(d + oX);
  // row pointers and theta first: every range needs them
  ALS_TRY(cudaMemcpyAsync(d_row, h_row_ptr, sizeof(int) * ((size_t)m + 1), cudaMemcpyHostToDevice, p.up),
          "als_half_step_host: row pointers");
  ALS_TRY(staged_copy(d + oT, thetaTHost, sizeof(float) * (size_t)n * f, true, p.up),
          "als_half_step_host: theta upload");
  ALS_TRY(cudaEventRecord(p.ev[0], p.up), "als_half_step_host: event");
  ALS_TRY(cudaStreamWaitEvent(st, p.ev[0], 0), "als_half_step_host: event");
  ALS_TRY(launch_widen_ptr(d_row, (int64_t)m + 1, reinterpret_cast<int64_t *>(d + oP), st),
          "als_half_step_host: row pointers");
  if (kind != kLpNone)
    ALS_TRY(launch_convert_lp(reinterpret_cast<const float *>(d + oT), n, f, f, d + oL, ldp, kind, st),
            "als_half_step_host: theta copy");
  Side S;
  S.rows = m; S.cols = n; S.ptr = reinterpret_cast<const int64_t *>(d + oP);
  S.idx = d_col; S.val = d_val;
  char *w = d + oW;
  S.order = reinterpret_cast<int32_t *>(w);
  S.queue = reinterpret_cast<unsigned *>(w + align_up(sizeof(int32_t) * m, 256));
  Counters *ctr = reinterpret_cast<Counters *>(reinterpret_cast<char *>(S.queue) +
                                               align_up(sizeof(unsigned) * (1 + 3 * kOrderBins), 256));
  ALS_TRY(cudaMemsetAsync(ctr, 0, sizeof(Counters), st), "als_half_step_host: counters");
  // X goes back range by range when the caller's buffer is pinned; a pageable
  // one is written at the end through the pinned staging (a copy into
  // pageable memory holds the host thread until it is done, which would keep
  // the next range's upload from being issued)
  const bool x_pinned = !pageable(XTHost);
  for (int c = 0; c < nch; ++c) {
    const int r0 = rb[c], r1 = rb[c + 1];
    const size_t k0 = (size_t)h_row_ptr[r0], kn = (size_t)h_row_ptr[r1] - k0;
    if (kn) {
      ALS_TRY(staged_copy(d_col + k0, h_col + k0, sizeof(int) * kn, true, p.up),
              "als_half_step_host: ratings upload");
      ALS_TRY(staged_copy(d_val + k0, h_val + k0, sizeof(float) * kn, true, p.up),
              "als_half_step_host: ratings upload");
    }
    ALS_TRY(cudaEventRecord(p.ev[1 + 2 * c], p.up), "als_half_step_host: event");
    ALS_TRY(cudaStreamWaitEvent(st, p.ev[1 + 2 * c], 0), "als_half_step_host: event");
    S.begin = r0;
    S.active = r1 - r0;
    ALS_TRY(launch_degree_order(S.ptr, S.active, S.order, S.queue + 1, st, r0),
            "als_half_step_host: order");
    if (ws) {
      ALS_TRY(plan_ws(S.ptr, r0, S.active, sms, np, n, d + oPl, plan_ws_bytes(m, sms, np), &S.plan,
                      &ctr->error, st),
              "als_half_step_host: plan");
      S.has_plan = true;
    }
    ALS_TRY(run_rows(S, f, lambda, o, reinterpret_cast<const float *>(d + oT), f, d + oL, ldp, d_x,
                     nullptr, ctr, nullptr, false, sms, st),
            "als_half_step_host: half-step");
    if (x_pinned) {
      ALS_TRY(cudaEventRecord(p.ev[2 + 2 * c], st), "als_half_step_host: event");
      ALS_TRY(cudaStreamWaitEvent(p.dn, p.ev[2 + 2 * c], 0), "als_half_step_host: event");
      ALS_TRY(cudaMemcpyAsync(XTHost + (size_t)r0 * f, d_x + (size_t)r0 * f,
                              sizeof(float) * (size_t)(r1 - r0) * f, cudaMemcpyDeviceToHost, p.dn),
              "als_half_step_host: X download");
    }
  }
  int kernel_error = 0;
  ALS_TRY(cudaMemcpyAsync(&kernel_error, &ctr->error, sizeof(int), cudaMemcpyDeviceToHost, st),
          "als_half_step_host: error word");
  if (!x_pinned)
    ALS_TRY(staged_copy(XTHost, d_x, sizeof(float) * (size_t)m * f, false, st),
            "als_half_step_host: X download");
  ALS_TRY(cudaStreamSynchronize(st), "als_half_step_host: sync");
  ALS_TRY(cudaStreamSynchronize(p.dn), "als_half_step_host: sync");
  if (kernel_error)
    return fail(ALS_ERR_CUDA, (kernel_error & 1)
                                  ? "als_half_step_host: a kernel gave up a bounded wait (bounded "
                                    "wait timed out); the half-step's rows are incomplete"
                                  : "als_half_step_host: malformed CSR row pointers");
  return ALS_OK;
}

// ---------------------------------------------------------------------------
// als_half_step_static: the stand-alone FP32 half-step with its scratch (the
// degree-binned visiting order, the row-queue head and the counters) in a
// file-scope device array, so that a call allocates nothing. It serves callers
// that cannot call cudaMalloc: their device memory belongs to another
// allocator's pool, or they must not take the synchronisation that
// cudaMalloc/cudaFree can cause.
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kStaticQueueOff = (sizeof(int32_t) * (size_t)ALS_STATIC_MAX_ROWS + 255) / 256 * 256;
constexpr size_t kStaticCtrOff =
    kStaticQueueOff + (sizeof(unsigned) * (1 + 3 * (size_t)kOrderBins) + 255) / 256 * 256;
constexpr size_t kStaticBytes = kStaticCtrOff + (sizeof(Counters) + 255) / 256 * 256;
}  // namespace

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

namespace {
constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mu;
struct StaticScratchEntry {
  void *ptr = nullptr;
  unsigned long long ctx = 0;  // context the address belongs to (0: unknown)
};
StaticScratchEntry g_static[kStaticMaxDevices];

// ID of the calling thread's current context (cuCtxGetId, unique within the
// process), or 0 when it cannot be read. The driver functions are reached
// through the runtime's entry-point query, so the library needs no link to
// the driver library.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext *);
  using GetId = CUresult (*)(CUcontext, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 12000, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(fn);
    fn = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &fn, 12000, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(fn);
    cudaGetLastError();
  });
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&c) == CUDA_SUCCESS && c && get_id(c, &id) == CUDA_SUCCESS)
    return id;
  return 0;
}

// Device address of the scratch array in the current device's context,
// looked up with cudaGetSymbolAddress the first time a call runs in that
// context. A device reset (or a released and re-created primary context)
// reloads the module at a new address; the context ID tells the cached
// address apart from the new one, so the lookup is repeated then.
int static_scratch(void **out) {
  int dev = 0;
  ALS_TRY(cudaGetDevice(&dev), "als_half_step_static: cudaGetDevice");
  if (dev < 0 || dev >= kStaticMaxDevices)
    return fail(ALS_ERR_UNSUPPORTED, "als_half_step_static: device ordinal above 63");
  std::lock_guard<std::mutex> lk(g_static_mu);
  StaticScratchEntry &ent = g_static[dev];
  const unsigned long long ctx = current_context_id();
  if (!ent.ptr || ctx == 0 || ctx != ent.ctx) {
    void *p = nullptr;
    ALS_TRY(cudaGetSymbolAddress(&p, g_static_scratch), "als_half_step_static: cudaGetSymbolAddress");
    ent.ptr = p;
    ent.ctx = current_context_id();  // the lookup has made the context current
  }
  *out = ent.ptr;
  return ALS_OK;
}
}  // namespace

int als_half_step_static(int64_t m, int64_t n, int32_t f, const int64_t *ptr, const int32_t *col,
                         const float *val, const float *src, int32_t ld_src, float *dst,
                         int32_t ld_dst, float lambda, const als_options *opt, cudaStream_t st) {
  if (m < 0 || n <= 0 || f <= 0) return fail(ALS_ERR_INVALID, "bad sizes");
  if (m > ALS_STATIC_MAX_ROWS)
    return fail(ALS_ERR_INVALID, "als_half_step_static: " + std::to_string(m) +
                                     " rows exceed the static scratch limit of " +
                                     std::to_string(ALS_STATIC_MAX_ROWS) +
                                     " rows; use als_half_step with a caller workspace");
  if (m == 0) return ALS_OK;
  if (!ptr || !src || !dst || ld_src < f || ld_dst < f)
    return fail(ALS_ERR_INVALID, "bad pointers or strides");
  als_options o;
  als_default_options(&o);
  if (opt) o = *opt;
  if (o.precision != ALS_PREC_FP32)
    return fail(ALS_ERR_UNSUPPORTED, "als_half_step_static takes FP32 factors");
  int rc = check_options(o, f);
  if (rc != ALS_OK) return rc;
  void *scratch = nullptr;
  if ((rc = static_scratch(&scratch)) != ALS_OK) return rc;
  char *b = static_cast<char *>(scratch);
  int32_t *order = reinterpret_cast<int32_t *>(b);
  unsigned *queue = reinterpret_cast<unsigned *>(b + kStaticQueueOff);
  Counters *ctr = reinterpret_cast<Counters *>(b + kStaticCtrOff);
  // Zeroed on every call: the counters and the row-queue head. The degree
  // histogram behind queue + 1 is cleared by launch_degree_order itself, and
  // every entry of the order it reads is written before it is read.
  ALS_TRY(cudaMemsetAsync(ctr, 0, sizeof(Counters), st), "als_half_step_static: counters");
  ALS_TRY(cudaMemsetAsync(queue, 0, sizeof(unsigned), st), "als_half_step_static: queue");
  ALS_TRY(launch_degree_order(ptr, m, order, queue + 1, st), "als_half_step_static: degree order");
  RowsArgs a{};
  a.m = m; a.f = f; a.lambda = lambda; a.row_ptr = ptr; a.col = col; a.val = val;
  a.src = src; a.ld_src = ld_src; a.dst = dst; a.ld_dst = ld_dst;
  a.order = order; a.queue = queue; a.counters = ctr; a.refine_tol = o.refine_tol;
  ALS_TRY(launch_rows_fp32(a, kLpNone, device_sm_count(), st), "als_half_step_static");
  return ALS_OK;
}
