/*
 * als_oracle.c -- CPU restatement of cuMF's ALS half-step.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA engine and
 * the timed CPU baseline ("port"); nothing in the product links or calls it.
 *
 * What it restates (paths within IBMSparkGPU/CUDA-MLlib):
 *   - A_u = sum_{i in R(u)} theta_i theta_i^T + lambda * n_u * I
 *       get_hermitian100 / get_hermitianT10, als/src/cuda/als.cu:478-912 and
 *       als.cu:52-470; the weighted-lambda diagonal term is als.cu:905-909.
 *   - b_u = sum_{i in R(u)} r_ui theta_i
 *       cusparseScsrmm2 + cublasSgeam, als/src/cuda/als.cu:1041-1059.
 *   - x_u = A_u^{-1} b_u
 *       updateX, als/src/cuda/als.cu:939-997 (batched FP64 LU, no pivoting).
 *   - the half-step contract (m rows of X from n rows of theta, row-major)
 *       doALSWithCSR, als/src/cuda/als.cu:1001-1115.
 *
 * Two modes of the FP64 half-step:
 *   ORC_EXACT   the mathematics the reference intends: symmetric A_u, Cholesky,
 *               x_u = 0 for rows with no ratings. The engine is checked against this mode.
 *   ORC_REFEMU  reproduces the reference bit for bit where that is defined:
 *               A_u accumulated in FP32 with fused multiply-adds in CSR order
 *               (as the per-thread accumulators temp0..temp99 do), the store
 *               defect in every 10x10 tile (element (x+4, y) receives temp0
 *               instead of temp40, als.cu:275 and als.cu:718), the lower
 *               triangle mirrored correctly (als.cu:391, als.cu:834), then FP64
 *               LU without pivoting. Requires f % 10 == 0. Used only to pin
 *               this oracle against the reference's own kernels.
 *
 * Rows are processed by a small pthread pool pulling chunks from an atomic
 * counter; results do not depend on the thread count.
 */
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define ORC_EXACT 0
#define ORC_REFEMU 1

typedef struct {
  int64_t m;
  int32_t f;
  const int64_t *row_ptr;
  const int32_t *col;
  const float *val;
  const void *src;
  double lambda;
  void *dst;
  int32_t mode;
  int32_t single; /* 1: FP32 port */
  atomic_llong next;
  atomic_llong fails;
} job_t;

static int resolve_threads(int32_t t) {
  if (t > 0) return t;
  long h = sysconf(_SC_NPROCESSORS_ONLN);
  return h > 0 ? (int)h : 1;
}

/* ---------------- FP64: exact mathematics ---------------- */

static int chol_solve_f64(double *A, double *b, int f) {
  /* A row-major f x f, lower triangle used; overwritten by L. */
  for (int j = 0; j < f; ++j) {
    double d = A[j * f + j];
    for (int k = 0; k < j; ++k) d -= A[j * f + k] * A[j * f + k];
    if (!(d > 0.0)) return -1;
    d = sqrt(d);
    A[j * f + j] = d;
    for (int i = j + 1; i < f; ++i) {
      double s = A[i * f + j];
      for (int k = 0; k < j; ++k) s -= A[i * f + k] * A[j * f + k];
      A[i * f + j] = s / d;
    }
  }
  for (int i = 0; i < f; ++i) { /* L y = b */
    double s = b[i];
    for (int k = 0; k < i; ++k) s -= A[i * f + k] * b[k];
    b[i] = s / A[i * f + i];
  }
  for (int i = f - 1; i >= 0; --i) { /* L^T x = y */
    double s = b[i];
    for (int k = i + 1; k < f; ++k) s -= A[k * f + i] * b[k];
    b[i] = s / A[i * f + i];
  }
  return 0;
}

static void row_exact_f64(job_t *J, int64_t u, double *A, double *b) {
  const int f = J->f;
  const double *src = (const double *)J->src;
  double *x = (double *)J->dst + (size_t)u * f;
  const int64_t s = J->row_ptr[u], e = J->row_ptr[u + 1];
  if (e == s) {
    memset(x, 0, sizeof(double) * (size_t)f);
    return;
  }
  memset(A, 0, sizeof(double) * (size_t)f * f);
  memset(b, 0, sizeof(double) * (size_t)f);
  for (int64_t q = s; q < e; ++q) {
    const double *t = src + (size_t)J->col[q] * f;
    const double r = (double)J->val[q];
    for (int i = 0; i < f; ++i) {
      const double ti = t[i];
      double *Ai = A + (size_t)i * f;
      for (int j = 0; j <= i; ++j) Ai[j] += ti * t[j];
      b[i] += r * ti;
    }
  }
  const double reg = J->lambda * (double)(e - s);
  for (int i = 0; i < f; ++i) A[i * f + i] += reg;
  if (chol_solve_f64(A, b, f) != 0) {
    atomic_fetch_add(&J->fails, 1);
    memset(x, 0, sizeof(double) * (size_t)f);
    return;
  }
  memcpy(x, b, sizeof(double) * (size_t)f);
}

/* ---------------- FP64: reference emulation ---------------- */

/* The reference's store of the accumulated tiles into the column-major
 * system tt: upper tiles element by element (with the defect at (x+4, y)),
 * mirrored lower tiles, then lambda * n_u added on the diagonal tiles. */
static void refemu_store(const float *acc, int f, int64_t n_u, double lambda, double *tt) {
  const int T = 10, N = f / 10;
  for (int ti = 0; ti < N; ++ti)
    for (int tj = ti; tj < N; ++tj) {
      const int x0 = ti * T, y0 = tj * T;
      for (int r = 0; r < T; ++r)
        for (int c = 0; c < T; ++c) {
          float v = acc[(x0 + r) * f + (y0 + c)];
          if (r == 4 && c == 0) v = acc[x0 * f + y0]; /* the defective store */
          tt[(x0 + r) + (size_t)(y0 + c) * f] = (double)v;
          if (x0 != y0) tt[(y0 + c) + (size_t)(x0 + r) * f] = (double)acc[(x0 + r) * f + (y0 + c)];
        }
      if (x0 == y0)
        for (int k = 0; k < T; ++k)
          tt[(size_t)(x0 + k) * (1 + f)] += (double)((float)n_u * (float)lambda);
    }
}

static void row_refemu(job_t *J, int64_t u, double *tt, double *b, float *acc) {
  const int f = J->f;
  const double *src = (const double *)J->src;
  double *x = (double *)J->dst + (size_t)u * f;
  const int64_t s = J->row_ptr[u], e = J->row_ptr[u + 1];
  /* FP32 accumulation of theta theta^T in CSR order, one fused multiply-add
   * per item, per output element (the temp registers of the kernels). */
  memset(acc, 0, sizeof(float) * (size_t)f * f);
  memset(b, 0, sizeof(double) * (size_t)f);
  for (int64_t q = s; q < e; ++q) {
    const double *t = src + (size_t)J->col[q] * f;
    for (int i = 0; i < f; ++i) {
      const float ti = (float)t[i];
      for (int j = 0; j < f; ++j) acc[i * f + j] = fmaf(ti, (float)t[j], acc[i * f + j]);
    }
  }
  /* b = R theta, FP32 products summed in CSR order (cuSPARSE's order is not
   * specified; the tolerance of the pin absorbs the difference). */
  for (int64_t q = s; q < e; ++q) {
    const double *t = src + (size_t)J->col[q] * f;
    for (int i = 0; i < f; ++i) b[i] = (double)fmaf(J->val[q], (float)t[i], (float)b[i]);
  }
  refemu_store(acc, f, e - s, J->lambda, tt);
  /* LU without pivoting on the column-major matrix, then two triangular solves. */
  for (int k = 0; k < f; ++k) {
    const double p = tt[k + (size_t)k * f];
    for (int i = k + 1; i < f; ++i) tt[i + (size_t)k * f] /= p;
    for (int j = k + 1; j < f; ++j) {
      const double ukj = tt[k + (size_t)j * f];
      for (int i = k + 1; i < f; ++i) tt[i + (size_t)j * f] -= tt[i + (size_t)k * f] * ukj;
    }
  }
  for (int i = 0; i < f; ++i)
    for (int k = 0; k < i; ++k) b[i] -= tt[i + (size_t)k * f] * b[k];
  for (int i = f - 1; i >= 0; --i) {
    for (int k = i + 1; k < f; ++k) b[i] -= tt[i + (size_t)k * f] * b[k];
    b[i] /= tt[i + (size_t)i * f];
  }
  memcpy(x, b, sizeof(double) * (size_t)f);
}

/* ---------------- FP32 port (the timed CPU baseline) ---------------- */

static int chol_solve_f32(float *A, float *b, int f) {
  for (int j = 0; j < f; ++j) {
    float d = A[j * f + j];
    for (int k = 0; k < j; ++k) d -= A[j * f + k] * A[j * f + k];
    if (!(d > 0.0f)) return -1;
    d = sqrtf(d);
    A[j * f + j] = d;
    const float inv = 1.0f / d;
    for (int i = j + 1; i < f; ++i) {
      float s = A[i * f + j];
      for (int k = 0; k < j; ++k) s -= A[i * f + k] * A[j * f + k];
      A[i * f + j] = s * inv;
    }
  }
  for (int i = 0; i < f; ++i) {
    float s = b[i];
    for (int k = 0; k < i; ++k) s -= A[i * f + k] * b[k];
    b[i] = s / A[i * f + i];
  }
  for (int i = f - 1; i >= 0; --i) {
    float s = b[i];
    for (int k = i + 1; k < f; ++k) s -= A[k * f + i] * b[k];
    b[i] = s / A[i * f + i];
  }
  return 0;
}

static void row_f32(job_t *J, int64_t u, float *A, float *b) {
  const int f = J->f;
  const float *src = (const float *)J->src;
  float *x = (float *)J->dst + (size_t)u * f;
  const int64_t s = J->row_ptr[u], e = J->row_ptr[u + 1];
  if (e == s) {
    memset(x, 0, sizeof(float) * (size_t)f);
    return;
  }
  memset(A, 0, sizeof(float) * (size_t)f * f);
  memset(b, 0, sizeof(float) * (size_t)f);
  for (int64_t q = s; q < e; ++q) {
    const float *t = src + (size_t)J->col[q] * f;
    const float r = J->val[q];
    for (int i = 0; i < f; ++i) {
      const float ti = t[i];
      float *Ai = A + (size_t)i * f;
      for (int j = 0; j <= i; ++j) Ai[j] += ti * t[j];
      b[i] += r * ti;
    }
  }
  const float reg = (float)J->lambda * (float)(e - s);
  for (int i = 0; i < f; ++i) A[i * f + i] += reg;
  if (chol_solve_f32(A, b, f) != 0) {
    atomic_fetch_add(&J->fails, 1);
    memset(x, 0, sizeof(float) * (size_t)f);
    return;
  }
  memcpy(x, b, sizeof(float) * (size_t)f);
}

static void *worker(void *arg) {
  job_t *J = (job_t *)arg;
  const int f = J->f;
  void *A = malloc(sizeof(double) * (size_t)f * f);
  void *b = malloc(sizeof(double) * (size_t)f);
  float *acc = (J->mode == ORC_REFEMU) ? (float *)malloc(sizeof(float) * (size_t)f * f) : NULL;
  for (;;) {
    int64_t r0 = atomic_fetch_add(&J->next, 64);
    if (r0 >= J->m) break;
    int64_t r1 = r0 + 64 < J->m ? r0 + 64 : J->m;
    for (int64_t u = r0; u < r1; ++u) {
      if (J->single) row_f32(J, u, (float *)A, (float *)b);
      else if (J->mode == ORC_REFEMU) row_refemu(J, u, (double *)A, (double *)b, acc);
      else row_exact_f64(J, u, (double *)A, (double *)b);
    }
  }
  free(A);
  free(b);
  free(acc);
  return NULL;
}

static int64_t run(job_t *J, int32_t threads) {
  int T = resolve_threads(threads);
  if ((int64_t)T * 64 > J->m) T = (int)((J->m + 63) / 64);
  if (T < 1) T = 1;
  atomic_init(&J->next, 0);
  atomic_init(&J->fails, 0);
  pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)T);
  for (int t = 0; t < T; ++t) pthread_create(&th[t], NULL, worker, J);
  for (int t = 0; t < T; ++t) pthread_join(th[t], NULL);
  free(th);
  return (int64_t)atomic_load(&J->fails);
}

/* FP64 half-step. src: n x f row-major, dst: m x f row-major.
 * Returns the number of rows whose system was not positive definite (their
 * x_u is set to 0), or -1 on bad arguments. */
int64_t orc_half_step_f64(int64_t m, int32_t f, const int64_t *row_ptr, const int32_t *col,
                          const float *val, const double *src, double lambda, double *dst,
                          int32_t mode, int32_t threads) {
  if (m < 0 || f <= 0 || !row_ptr || !dst) return -1;
  if (mode == ORC_REFEMU && f % 10 != 0) return -1;
  job_t J = {m, f, row_ptr, col, val, src, lambda, dst, mode, 0};
  return run(&J, threads);
}

/* FP32 half-step with the same algorithm in single precision (CPU baseline). */
int64_t orc_half_step_f32(int64_t m, int32_t f, const int64_t *row_ptr, const int32_t *col,
                          const float *val, const float *src, float lambda, float *dst,
                          int32_t threads) {
  if (m < 0 || f <= 0 || !row_ptr || !dst) return -1;
  job_t J = {m, f, row_ptr, col, val, src, lambda, dst, ORC_EXACT, 1};
  return run(&J, threads);
}

/* Test RMSE, FP64 accumulation: sqrt(sum (r - x_u . theta_i)^2 / nt). */
double orc_rmse(int64_t nt, const int32_t *u, const int32_t *i, const float *r, const double *X,
                const double *T, int32_t f) {
  if (nt <= 0) return 0.0;
  double acc = 0.0;
  for (int64_t q = 0; q < nt; ++q) {
    const double *x = X + (size_t)u[q] * f, *t = T + (size_t)i[q] * f;
    double p = 0.0;
    for (int k = 0; k < f; ++k) p += x[k] * t[k];
    const double e = (double)r[q] - p;
    acc += e * e;
  }
  return sqrt(acc / (double)nt);
}

/* Sum-of-squares objective of the weighted-lambda ALS problem (FP64):
 * sum_(u,i) (r - x_u.theta_i)^2 + lambda * (sum_u n_u |x_u|^2 + sum_i n_i |theta_i|^2).
 * Each half-step must not increase it; tests use that as a size-independent
 * property. row_ptr is the CSR over users, ncols_of_item the item degrees. */
double orc_objective(int64_t m, int64_t n, int32_t f, const int64_t *row_ptr, const int32_t *col,
                     const float *val, const double *X, const double *T, double lambda) {
  double loss = 0.0, reg = 0.0;
  for (int64_t uu = 0; uu < m; ++uu) {
    const double *x = X + (size_t)uu * f;
    double nx = 0.0;
    for (int k = 0; k < f; ++k) nx += x[k] * x[k];
    reg += (double)(row_ptr[uu + 1] - row_ptr[uu]) * nx;
    for (int64_t q = row_ptr[uu]; q < row_ptr[uu + 1]; ++q) {
      const double *t = T + (size_t)col[q] * f;
      double p = 0.0;
      for (int k = 0; k < f; ++k) p += x[k] * t[k];
      const double e = (double)val[q] - p;
      loss += e * e;
    }
  }
  int64_t *deg = (int64_t *)calloc((size_t)n, sizeof(int64_t));
  for (int64_t q = 0; q < row_ptr[m]; ++q) deg[col[q]]++;
  for (int64_t j = 0; j < n; ++j) {
    const double *t = T + (size_t)j * f;
    double nt = 0.0;
    for (int k = 0; k < f; ++k) nt += t[k] * t[k];
    reg += (double)deg[j] * nt;
  }
  free(deg);
  return loss + lambda * reg;
}

/* The system the reference builds for one row, column-major f x f, from the
 * row's gathered factor rows (d x f, row-major): FP32 fused accumulation,
 * the tile store map with its defect, the weighted-lambda diagonal.
 * Exposed so tests can inspect exactly which entries differ from A_u. */
int orc_refemu_system(int32_t f, int64_t d, const double *rows, double lambda, double *tt) {
  if (f <= 0 || f % 10 != 0 || d < 0) return -1;
  float *acc = (float *)calloc((size_t)f * f, sizeof(float));
  if (!acc) return -1;
  for (int64_t q = 0; q < d; ++q) {
    const double *t = rows + (size_t)q * f;
    for (int i = 0; i < f; ++i)
      for (int j = 0; j < f; ++j) acc[i * f + j] = fmaf((float)t[i], (float)t[j], acc[i * f + j]);
  }
  refemu_store(acc, f, d, lambda, tt);
  free(acc);
  return 0;
}
