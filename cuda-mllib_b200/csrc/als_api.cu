// C ABI of the engine: resident model, half-step dispatch, the drop-in
// doALSWithCSR / utilities entry points, and host-buffer training.
#include <thrust/system/cuda/error.h>
#include <thrust/system_error.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/als_b200.h"
#include "als_internal.h"

using namespace als;

namespace {

thread_local std::string g_last_error;

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
};

// Dispatch one half-step: rows of `s` solved against factor `src`.
cudaError_t run_rows(const Side &s, int f, float lambda, const als_options &o, const float *src32,
                     int ld_src32, const void *src_lp, int ld_lp, float *dst32, void *dst_lp,
                     Counters *ctr, const float *x0, int num_sms, cudaStream_t st) {
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
  return launch_rows_tc(a, kind, o.solver, o.cg_max_steps, o.cg_tol, x0, num_sms, st);
}

}  // namespace

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
};

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
}

const char *als_last_error(void) { return g_last_error.c_str(); }
const char *als_version(void) { return "als_b200 1.0 (sm_100a)"; }

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
  *out = M;
  return ALS_OK;
}

void als_model_destroy(als_model *M) {
  if (!M) return;
  if (M->graph) cudaGraphExecDestroy(M->graph);
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
  const float *x0 = (M->opt.warm_start == ALS_WARM_PREVIOUS) ? dst32 : nullptr;
  return run_rows(M->side[side], M->f, lambda, M->opt, src32, M->f, src_lp, M->lp_ld, dst32,
                  dst_lp, M->ctr, x0, M->num_sms, st);
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
  if (!M->opt.use_graph || st == 0) {
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

// ---------------------------------------------------------------------------
// Drop-in entry points of the reference.
// ---------------------------------------------------------------------------

cudaError_t mallocBest(void **devPtr, size_t size) {
  if (cudaMalloc(devPtr, size) == cudaSuccess) return cudaSuccess;
  cudaGetLastError();  // clear the allocation failure
  void *h = nullptr;
  cudaError_t e = cudaHostAlloc(&h, size, cudaHostAllocMapped | cudaHostAllocWriteCombined);
  if (e != cudaSuccess) return e;
  return cudaHostGetDevicePointer(devPtr, h, 0);
}

cudaError_t freeBest(void *devPtr) {
  if (!devPtr) return cudaSuccess;
  cudaPointerAttributes attr;
  cudaError_t e = cudaPointerGetAttributes(&attr, devPtr);
  if (e != cudaSuccess) return e;
  if (attr.type == cudaMemoryTypeDevice) return cudaFree(devPtr);
  // mapped host memory: free through its host address
  return cudaFreeHost(attr.hostPointer ? attr.hostPointer : devPtr);
}

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

#define DROPIN_CALL(call, where)           \
  do {                                     \
    cudaError_t e_ = (call);               \
    if (e_ != cudaSuccess) throw_cuda(e_, where); \
  } while (0)

extern "C" void doALSWithCSR(cudaStream_t st, int *csrRowIndex, int *csrColIndex, float *csrVal,
                             float *thetaTHost, float *XTHost, const int m, const int n,
                             const int f, const long nnz, const float lambda, const int X_BATCH) {
  (void)X_BATCH;
  if (m < 0 || n <= 0 || f <= 0 || nnz < 0) throw_cuda(cudaErrorInvalidValue, "doALSWithCSR: sizes");
  if (fp32_padded_rank(f) < 0) throw_cuda(cudaErrorInvalidValue, "doALSWithCSR: rank f must be 1..128");
  // device buffers: theta, X, widened row pointers, half-step workspace
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t p = off; off = align_up(off + bytes, 256); return p; };
  const size_t oT = take(sizeof(float) * (size_t)n * f), oX = take(sizeof(float) * (size_t)m * f + 4),
               oP = take(sizeof(int64_t) * ((size_t)m + 1)), oW = take(als_half_step_work_bytes(m));
  char *d = nullptr;
  DROPIN_CALL(cudaMalloc(&d, off), "doALSWithCSR: cudaMalloc");
  DROPIN_CALL(cudaMemcpyAsync(d + oT, thetaTHost, sizeof(float) * (size_t)n * f,
                              cudaMemcpyHostToDevice, st), "doALSWithCSR: theta upload");
  DROPIN_CALL(launch_widen_ptr(csrRowIndex, (int64_t)m + 1, (int64_t *)(d + oP), st),
              "doALSWithCSR: row pointers");
  als_options o;
  als_default_options(&o);
  if (m > 0) {
    int rc = als_half_step(m, n, f, (const int64_t *)(d + oP), csrColIndex, csrVal,
                           (const float *)(d + oT), f, (float *)(d + oX), f, lambda, &o, d + oW,
                           als_half_step_work_bytes(m), st);
    if (rc != ALS_OK) {
      cudaError_t e = cudaGetLastError();
      throw_cuda(e != cudaSuccess ? e : cudaErrorInvalidValue, als_last_error());
    }
    DROPIN_CALL(cudaMemcpyAsync(XTHost, d + oX, sizeof(float) * (size_t)m * f,
                                cudaMemcpyDeviceToHost, st), "doALSWithCSR: X download");
  }
  DROPIN_CALL(cudaStreamSynchronize(st), "doALSWithCSR: sync");
  DROPIN_CALL(cudaFree(d), "doALSWithCSR: cudaFree");
  // The callee owns and frees the CSR arrays (reference als.cu:1058, 1101-1102).
  DROPIN_CALL(freeBest(csrVal), "doALSWithCSR: free csrVal");
  DROPIN_CALL(freeBest(csrRowIndex), "doALSWithCSR: free csrRowIndex");
  DROPIN_CALL(freeBest(csrColIndex), "doALSWithCSR: free csrColIndex");
}
