// Shared device-side pieces of the ALS engine: argument block, the degree-ordered
// work queue, and the in-CTA SPD solver used by every hermitian kernel.
//
// Layout conventions (all row-major):
//   src   n x ld_src   fixed factor matrix (theta when solving users)
//   dst   m x ld_dst   factors being solved (X when solving users)
//   CSR   row_ptr[m+1] int64, col[nnz] int32, val[nnz] float32
// A_u lives in shared memory as S[FP][FP+1] floats: after factorisation the
// lower triangle holds L (A = L L^T), the strict upper triangle still holds the
// original A_u and dg[] its original diagonal, which is what the refinement
// residual needs.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace als {

// Per-row status bits written to ws.row_flags (when non-null).
enum RowFlag : uint32_t {
  kRowEmpty = 1u,        // n_u == 0: x_u defined as 0
  kRowNotSPD = 2u,       // non-positive pivot: x_u set to 0
  kRowRefinedF64 = 4u,   // relative residual > 1e-5: FP64-residual refinement ran
  kRowCgFallback = 8u,   // CG did not converge: Cholesky fallback ran
};

// Counters accumulated by the kernels (device memory, zeroed by the host).
struct Counters {
  unsigned long long rows;
  unsigned long long refined;
  unsigned long long not_spd;
  unsigned long long cg_steps;
  unsigned long long cg_fallback;
  unsigned long long r0_micro;  // sum over CG rows of |b - A x0| / |b| (after scaling), x 1e6
  int error;             // sticky kernel error bits (1: a bounded wait timed out,
                         // 2: row pointers malformed beyond the work plan's bounds)
  int pad;
};

struct RowsArgs {
  int64_t m;                 // rows to solve
  int32_t f;                 // rank
  int32_t ld_src;            // row stride of src (elements)
  int32_t ld_dst;            // row stride of dst (elements)
  float lambda;
  const int64_t *row_ptr;
  const int32_t *col;
  const float *val;
  const void *src;           // float / bf16 / fp16 by kernel
  float *dst;                // FP32 result
  void *dst_lp;              // optional low-precision copy of the result (ld = ld_dst_lp)
  int32_t ld_dst_lp;
  const int32_t *order;      // row visiting order (heaviest first); null = identity
  unsigned int *queue;       // work-queue head, zeroed before launch
  uint32_t *row_flags;       // optional per-row status
  Counters *counters;        // optional
  float refine_tol;          // relative residual that triggers FP64 refinement
  int *error;                // sticky error word (device), may be null
  const int *m_dev;          // optional: the number of rows, read from device memory
                             // (m is then only an upper bound for launch sizing)
};

// A group of threads that synchronise together: the whole CTA (id 0) or a
// warpgroup on its own named barrier. tid is the thread's index in the group.
struct Bar {
  int id, n, tid;
  __device__ __forceinline__ void sync() const {
    if (id == 0) __syncthreads();
    else asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
  }
  // barrier that also returns whether `pred` held on every thread of the group
  __device__ __forceinline__ bool all(bool pred) const {
    if (id == 0) return __syncthreads_and(pred);
    uint32_t r;
    asm volatile(
        "{\n.reg .pred p, q;\nsetp.ne.u32 p, %1, 0;\n"
        "bar.red.and.pred q, %2, %3, p;\nselp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(n)
        : "memory");
    return r != 0;
  }
};

__device__ __forceinline__ Bar cta_bar() { return Bar{0, (int)blockDim.x, (int)threadIdx.x}; }

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Next row index from the device work queue; every thread of the CTA gets it.
__device__ __forceinline__ int64_t next_row(const RowsArgs &a, int *slot) {
  __syncthreads();
  if (threadIdx.x == 0) *slot = (int)atomicAdd(a.queue, 1u);
  __syncthreads();
  const int64_t i = *slot;
  if (i >= (a.m_dev ? (int64_t)*a.m_dev : a.m)) return -1;
  return a.order ? (int64_t)a.order[i] : i;
}

// ---------------------------------------------------------------------------
// Triangular solves with L stored in the lower triangle of S (ld = LDS).
// One warp; lane owns entries i = lane + 32*s. Vector v in shared memory.
// ---------------------------------------------------------------------------
template <int FP, int LDS>
__device__ __forceinline__ void warp_forward(const float *S, float *v, int f) {
  constexpr int NS = (FP + 31) / 32;
  const int lane = threadIdx.x & 31;
  float y[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) y[s] = (lane + 32 * s < f) ? v[lane + 32 * s] : 0.f;
  for (int j = 0; j < f; ++j) {
    const int sj = j >> 5, lj = j & 31;
    float yj = 0.f;
#pragma unroll
    for (int s = 0; s < NS; ++s)
      if (s == sj) yj = __shfl_sync(0xffffffffu, y[s], lj);
    yj = yj / S[j * LDS + j];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const int i = lane + 32 * s;
      if (i == j) y[s] = yj;
      else if (i > j && i < f) y[s] = fmaf(-S[i * LDS + j], yj, y[s]);
    }
  }
#pragma unroll
  for (int s = 0; s < NS; ++s)
    if (lane + 32 * s < f) v[lane + 32 * s] = y[s];
  __syncwarp();
}

template <int FP, int LDS>
__device__ __forceinline__ void warp_backward(const float *S, float *v, int f) {
  constexpr int NS = (FP + 31) / 32;
  const int lane = threadIdx.x & 31;
  float y[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) y[s] = (lane + 32 * s < f) ? v[lane + 32 * s] : 0.f;
  for (int j = f - 1; j >= 0; --j) {
    const int sj = j >> 5, lj = j & 31;
    float yj = 0.f;
#pragma unroll
    for (int s = 0; s < NS; ++s)
      if (s == sj) yj = __shfl_sync(0xffffffffu, y[s], lj);
    yj = yj / S[j * LDS + j];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const int i = lane + 32 * s;
      // L^T x = y: x_j known, y_i -= L[j][i] x_j for i < j
      if (i == j) y[s] = yj;
      else if (i < j) y[s] = fmaf(-S[j * LDS + i], yj, y[s]);
    }
  }
#pragma unroll
  for (int s = 0; s < NS; ++s)
    if (lane + 32 * s < f) v[lane + 32 * s] = y[s];
  __syncwarp();
}

// ---------------------------------------------------------------------------
// In-CTA blocked Cholesky on 8x8 register tiles.
//
// Thread t < NTILES owns lower-triangle tile (ti, tj), ti >= tj, whose current
// value is in acc[8][8] (A_u restricted to the tile). At block step kb:
//   1. the owner of (kb,kb) stores it, warp 0 factors the 8x8 block in smem;
//   2. owners of (ti,kb), ti > kb, solve X D^T = tile and store L(ti,kb);
//   3. owners of (ti,tj), tj > kb, subtract L(ti,kb) L(tj,kb)^T in registers.
// On exit the lower triangle of S holds L. Rows/cols >= f must be an identity
// block on entry (the caller sets the padding diagonal to 1).
// Returns false (for all threads) if a pivot was not positive.
// ---------------------------------------------------------------------------
template <int FP, int LDS, int NT>
__device__ bool tile_cholesky(float (&acc)[8][8], int ti, int tj, bool owner, float *S,
                              int *bad, const Bar &B) {
  constexpr int T8 = FP / 8;
  if (B.tid == 0) *bad = 0;
  B.sync();
  for (int kb = 0; kb < T8; ++kb) {
    // 1. diagonal block
    if (owner && ti == kb && tj == kb) {
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c <= r; ++c) S[(8 * kb + r) * LDS + 8 * kb + c] = acc[r][c];
    }
    B.sync();
    if (B.tid < 32) {
      const int lane = B.tid;
      float *D = S + (8 * kb) * LDS + 8 * kb;
      for (int j = 0; j < 8; ++j) {
        const float d = D[j * LDS + j];
        const float p = sqrtf(fmaxf(d, 0.f));
        __syncwarp();
        if (lane == 0) {
          if (!(d > 0.f)) *bad = 1;
          D[j * LDS + j] = p;
        }
        const float inv = (p > 0.f) ? 1.f / p : 0.f;
        __syncwarp();
        if (lane > j && lane < 8) D[lane * LDS + j] *= inv;
        __syncwarp();
        // update the trailing part of the 8x8 block: (i, c) with j < c <= i < 8
        for (int e = lane; e < 64; e += 32) {
          const int i = e >> 3, c = e & 7;
          if (c > j && c <= i) D[i * LDS + c] = fmaf(-D[i * LDS + j], D[c * LDS + j], D[i * LDS + c]);
        }
        __syncwarp();
      }
    }
    B.sync();
    // 2. panel: L(ti,kb) = tile * D^{-T}
    if (owner && tj == kb && ti > kb) {
      const float *D = S + (8 * kb) * LDS + 8 * kb;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const float inv = 1.f / D[c * LDS + c];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          float x = acc[r][c];
#pragma unroll
          for (int k = 0; k < c; ++k) x = fmaf(-acc[r][k], D[c * LDS + k], x);
          acc[r][c] = x * inv;
        }
      }
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) S[(8 * ti + r) * LDS + 8 * kb + c] = acc[r][c];
    }
    B.sync();
    // 3. trailing update
    if (owner && tj > kb) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        float a[8], b[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) a[r] = S[(8 * ti + r) * LDS + 8 * kb + k];
#pragma unroll
        for (int c = 0; c < 8; ++c) b[c] = S[(8 * tj + c) * LDS + 8 * kb + k];
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
          for (int c = 0; c < 8; ++c) acc[r][c] = fmaf(-a[r], b[c], acc[r][c]);
      }
    }
  }
  B.sync();
  return *bad == 0;
}

// Map a lower-triangle tile index t to (ti, tj), ti >= tj.
__device__ __forceinline__ void tile_of(int t, int &ti, int &tj) {
  int r = 0;
  while ((r + 1) * (r + 2) / 2 <= t) ++r;
  ti = r;
  tj = t - r * (r + 1) / 2;
}

// ---------------------------------------------------------------------------
// Solve with the factor in S, then one FP64-residual refinement step when the
// FP32 relative residual exceeds tol. Uses the original A_u kept in the strict
// upper triangle of S plus dg[]. x: on entry b, on exit the solution. Every
// thread of the group B calls; red is 64 floats of group-private scratch.
// ---------------------------------------------------------------------------
template <int FP, int LDS, int NT>
__device__ void solve_and_refine(const float *S, const float *dg, const float *b, float *x,
                                 double *rd, float *tmp, int f, float tol, bool *refined,
                                 float *red, const Bar &B) {
  const int tid = B.tid;
  if (tid < 32) {
    warp_forward<FP, LDS>(S, x, f);
    warp_backward<FP, LDS>(S, x, f);
  }
  B.sync();
  // FP32 residual norm vs |b|
  float rr = 0.f, bb = 0.f;
  for (int i = tid; i < f; i += NT) {
    float s = b[i] - dg[i] * x[i];
    for (int k = 0; k < i; ++k) s = fmaf(-S[k * LDS + i], x[k], s);
    for (int k = i + 1; k < f; ++k) s = fmaf(-S[i * LDS + k], x[k], s);
    rr = fmaf(s, s, rr);
    bb = fmaf(b[i], b[i], bb);
  }
  rr = warp_sum(rr);
  bb = warp_sum(bb);
  if ((tid & 31) == 0) { red[tid >> 5] = rr; red[32 + (tid >> 5)] = bb; }
  B.sync();
  float ra = 0.f, rc = 0.f;
  for (int w = 0; w < (NT + 31) / 32; ++w) { ra += red[w]; rc += red[32 + w]; }
  const bool need = ra > tol * tol * rc;
  B.sync();
  *refined = need;
  if (!need) return;
  // FP64 residual r = b - A x, then L L^T d = r in FP32, x += d.
  for (int i = tid; i < f; i += NT) {
    double s = (double)b[i] - (double)dg[i] * (double)x[i];
    for (int k = 0; k < i; ++k) s -= (double)S[k * LDS + i] * (double)x[k];
    for (int k = i + 1; k < f; ++k) s -= (double)S[i * LDS + k] * (double)x[k];
    rd[i] = s;
    tmp[i] = (float)s;
  }
  B.sync();
  if (tid < 32) {
    warp_forward<FP, LDS>(S, tmp, f);
    warp_backward<FP, LDS>(S, tmp, f);
  }
  B.sync();
  for (int i = tid; i < f; i += NT) x[i] += tmp[i];
  B.sync();
}

}  // namespace als
