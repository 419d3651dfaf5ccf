// Learned CG warm start: a 3-layer MLP (2f+1 -> 256 -> 256 -> f, GELU,
// BF16 weights and activations, FP32 accumulation) that maps a row's
// features [b_u / n_u, diag(A_u) / n_u, log1p(n_u) / 8] to a starting point
// x0 for the conjugate-gradient solve. Forward, backward and Adam run as this
// file's kernels; every product is one tcgen05 GEMM.
//
// GEMM: C[M x N] = A[M x K] * B[K x N], one CTA per 128-row tile, N <= 256 in
// one tile, K streamed in 64-wide chunks through two shared-memory stages.
// Each operand is either K-major (A[m][k] at m*lda + k; B[k][n] at n*ldb + k)
// or MN-major (A[m][k] at k*lda + m; B[k][n] at k*ldb + n), staged into the
// matching 128B-swizzled canonical layout, so one kernel serves
//   forward      Z = X W^T + b         (X K-major, W [out][in] K-major)
//   backward dX  dH = dZ W             (dZ K-major, W [out][in] MN-major)
//   backward dW  G = dZ^T X            (both MN-major; K = batch)
// Epilogues: + bias, GELU, or multiply by GELU'(pre-activation).
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "als_common.cuh"
#include "als_internal.h"
#include "als_tcgen05.cuh"

namespace als {

namespace mlp {

constexpr int kThreads = 128;
constexpr int kKC = 64;          // K per stage
constexpr int kABytes = 16384;   // 128 x 64 bf16
constexpr int kBBytes = 32768;   // up to 256 x 64 bf16
constexpr int kStage = kABytes + kBBytes;

enum Act { kActNone = 0, kActGelu = 1, kActGeluGrad = 2 };

struct GemmArgs {
  int M, N, K;
  const __nv_bfloat16 *A;
  int lda, a_mn;
  const __nv_bfloat16 *B;
  int ldb, b_mn;
  const float *bias;  // [N] or null
  int act;
  const float *aux;   // pre-activation for kActGeluGrad (M x N, ld ldaux)
  int ldaux;
  float *C32;         // optional FP32 output
  int ldc32, accumulate;
  __nv_bfloat16 *C16;  // optional BF16 output
  int ldc16;
  float *Z;           // optional pre-activation output
  int ldz;
  int *error;
};

__device__ __forceinline__ float gelu(float z) {
  return 0.5f * z * (1.f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.f + erff(z * 0.70710678118654752f)) +
         z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// K-major SW128: 8-row groups of 128 B rows at 1024 B; LBO field 1 (16 B).
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// Stage one 64-wide K chunk of an operand with `rows` MN entries.
//   K-major: row r (an M or N index) holds 64 K values (128 B), rows in 8-row groups.
//   MN-major: K row k holds MN values in 64-element atoms (8 KB apart).
__device__ __forceinline__ void stage_operand(unsigned char *dst, const __nv_bfloat16 *src,
                                              int ld, int mn_major, int r0, int rows_tile,
                                              int rows_total, int k0, int K) {
  const int tid = threadIdx.x;
  if (!mn_major) {
    for (int q = tid; q < rows_tile * 8; q += kThreads) {
      const int r = q >> 3, c = q & 7;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (r0 + r < rows_total && k0 + 8 * c < K)
        v = *reinterpret_cast<const uint4 *>(src + (int64_t)(r0 + r) * ld + k0 + 8 * c);
      *reinterpret_cast<uint4 *>(dst + (r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4)) = v;
    }
  } else {
    const int chunks = rows_tile / 8;
    for (int q = tid; q < kKC * chunks; q += kThreads) {
      const int k = q / chunks, j = q - k * chunks;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (k0 + k < K && r0 + 8 * j < rows_total)
        v = *reinterpret_cast<const uint4 *>(src + (int64_t)(k0 + k) * ld + r0 + 8 * j);
      const int atom = j >> 3, cc = j & 7, kg = k >> 3, kr = k & 7;
      *reinterpret_cast<uint4 *>(dst + atom * 8192 + kg * 1024 + kr * 128 + ((cc ^ kr) << 4)) = v;
    }
  }
}

__global__ void __launch_bounds__(kThreads) gemm_kernel(GemmArgs g, int np, uint32_t idesc,
                                                         int tmem_cols) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *base = smem_raw + ((1024 - (tc::smem_u32(smem_raw) & 1023)) & 1023);
  uint64_t *bars = reinterpret_cast<uint64_t *>(base + 2 * kStage);
  int *misc = reinterpret_cast<int *>(bars + 4);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.x * 128;
  if (tid == 0) {
    for (int i = 0; i < 3; ++i) tc::mbar_init(&bars[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32(&misc[0])),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = (uint32_t)misc[0];
  const int nk = (g.K + kKC - 1) / kKC;
  unsigned uses0 = 0, uses1 = 0;
  bool ok = true;
  for (int kc = 0; kc < nk; ++kc) {
    const int buf = kc & 1;
    const unsigned used = buf ? uses1 : uses0;
    const bool okw = kc < 2 || tc::mbar_wait(&bars[buf], (used - 1) & 1);
    unsigned char *sa = base + buf * kStage, *sb = sa + kABytes;
    if (okw) {
      stage_operand(sa, g.A, g.lda, g.a_mn, m0, 128, g.M, kc * kKC, g.K);
      stage_operand(sb, g.B, g.ldb, g.b_mn, 0, np, g.N, kc * kKC, g.K);
    }
    tc::fence_proxy_async();
    if (!__syncthreads_and(okw)) { ok = false; break; }
    if (tid == 0) {
      tc::tc_fence_after();
      const uint32_t a0 = tc::smem_u32(sa), b0 = tc::smem_u32(sb);
      for (int kk = 0; kk < kKC / 16; ++kk) {
        const uint64_t ad = g.a_mn ? tc::make_desc(a0 + kk * 2048, 8192, 1024) : desc_kmajor(a0 + kk * 32);
        const uint64_t bd = g.b_mn ? tc::make_desc(b0 + kk * 2048, 8192, 1024) : desc_kmajor(b0 + kk * 32);
        tc::mma_f16(tmem, ad, bd, idesc, (kc > 0 || kk > 0) ? 1u : 0u);
      }
      tc::mma_commit(&bars[buf]);
      if (kc == nk - 1) tc::mma_commit(&bars[2]);
    }
    if (buf) ++uses1; else ++uses0;
  }
  const bool oka = ok && tc::mbar_wait(&bars[2], 0);
  if (!__syncthreads_and(oka)) {
    if (tid == 0 && g.error) atomicCAS(g.error, 0, 1);
    if (tid == 0) tc::mma_commit(&bars[3]);
    tc::mbar_wait(&bars[3], 0);
  } else {
    tc::tc_fence_after();
    const int m = m0 + tid;
    for (int c0 = 0; c0 < np; c0 += 16) {
      float v[16];
      tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
      if (m < g.M) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int n = c0 + q;
          if (n >= g.N) break;
          float z = v[q];
          if (g.bias) z += g.bias[n];
          if (g.Z) g.Z[(int64_t)m * g.ldz + n] = z;
          float y = z;
          if (g.act == kActGelu) y = gelu(z);
          else if (g.act == kActGeluGrad) y = z * gelu_grad(g.aux[(int64_t)m * g.ldaux + n]);
          if (g.C32) {
            float *o = g.C32 + (int64_t)m * g.ldc32 + n;
            *o = g.accumulate ? *o + y : y;
          }
          if (g.C16) g.C16[(int64_t)m * g.ldc16 + n] = __float2bfloat16(y);
        }
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(tmem_cols));
  }
}

cudaError_t gemm(const GemmArgs &g, cudaStream_t st) {
  if (g.N > 256 && g.M > 0 && g.K > 0 && g.N % 8 == 0) {
    // One accumulator holds at most 256 columns: split N into near-equal
    // blocks of a multiple of 8 columns (the first-layer weight gradient at
    // f = 128 has N = 264) and run one GEMM per block.
    const int nb = (g.N + 255) / 256, w = ((g.N + nb - 1) / nb + 7) / 8 * 8;
    for (int n0 = 0; n0 < g.N; n0 += w) {
      GemmArgs h = g;
      h.N = std::min(w, g.N - n0);
      h.B = g.b_mn ? g.B + n0 : g.B + (int64_t)n0 * g.ldb;
      if (g.bias) h.bias = g.bias + n0;
      if (g.aux) h.aux = g.aux + n0;
      if (g.C32) h.C32 = g.C32 + n0;
      if (g.C16) h.C16 = g.C16 + n0;
      if (g.Z) h.Z = g.Z + n0;
      const cudaError_t e = gemm(h, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  if (g.N <= 0 || g.N > 256 || g.M <= 0 || g.K <= 0) return cudaErrorInvalidValue;
  if (g.K % 8 || g.lda % 8 || g.ldb % 8) return cudaErrorInvalidValue;
  if ((g.a_mn && g.M % 8) || (g.b_mn && g.N % 8)) return cudaErrorInvalidValue;
  const int np = (g.N + 15) / 16 * 16;
  const int tmem_cols = np <= 32 ? 32 : np <= 64 ? 64 : np <= 128 ? 128 : 256;
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)g.a_mn << 15) |
                         ((uint32_t)g.b_mn << 16) | ((uint32_t)(np >> 3) << 17) |
                         ((uint32_t)(128 >> 4) << 24);
  const size_t smem = 1024 + 2 * kStage + 4 * 8 + 16;
  cudaError_t e = cudaFuncSetAttribute(gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  const unsigned grid = (unsigned)((g.M + 127) / 128);
  gemm_kernel<<<grid, kThreads, smem, st>>>(g, np, idesc, tmem_cols);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------

// Features of row u from the low-precision source factors: one block per row
// (grid-stride), its 8 warps striding the row's ratings, then a shared-memory
// reduction over the warps, so long rows do not serialise on one warp.
template <typename LP>
__global__ void __launch_bounds__(256) features_kernel(int64_t m, int f, const int64_t *row_ptr,
                                                       const int32_t *col, const float *val,
                                                       const LP *src, int ld_src,
                                                       __nv_bfloat16 *F, int ldf) {
  constexpr int MAXE = 4;  // f <= 128
  __shared__ float part[8][2][128];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int64_t u = blockIdx.x; u < m; u += gridDim.x) {
    const int64_t s = row_ptr[u], e = row_ptr[u + 1];
    float b[MAXE] = {0.f, 0.f, 0.f, 0.f}, d[MAXE] = {0.f, 0.f, 0.f, 0.f};
    for (int64_t q = s + w; q < e; q += 8) {
      const LP *t = src + (int64_t)col[q] * ld_src;
      const float r = val[q];
#pragma unroll
      for (int j = 0; j < MAXE; ++j) {
        const int i = lane + 32 * j;
        if (i < f) {
          const float v = (float)t[i];
          b[j] = fmaf(r, v, b[j]);
          d[j] = fmaf(v, v, d[j]);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < MAXE; ++j) {
      part[w][0][lane + 32 * j] = b[j];
      part[w][1][lane + 32 * j] = d[j];
    }
    __syncthreads();
    const float n = (float)(e - s), inv = n > 0.f ? 1.f / n : 0.f;
    __nv_bfloat16 *o = F + u * ldf;
    for (int i = threadIdx.x; i < ldf; i += blockDim.x) {
      float v = 0.f;
      if (i < 2 * f) {
        const int h = i < f ? 0 : 1, c = i < f ? i : i - f;
        for (int k = 0; k < 8; ++k) v += part[k][h][c];
        v *= inv;
      } else if (i == 2 * f) {
        v = log1pf(n) * 0.125f;
      }
      o[i] = __float2bfloat16(v);
    }
    __syncthreads();
  }
}

// The same features from a 16-bit factor copy (row stride ld a multiple of 8):
// each half-warp takes one rating, its lanes one 16-byte piece (8 elements)
// of the rated factor row each; a warp takes 32 ratings per round, their
// column indices and ratings read in one coalesced load and handed out by
// shuffles, so sixteen factor-row loads can be in flight per warp.
template <typename LP>
__global__ void __launch_bounds__(256) features_lp_kernel(int64_t m, int f, const int64_t *row_ptr,
                                                          const int32_t *col, const float *val,
                                                          const LP *src, int ld_src,
                                                          __nv_bfloat16 *F, int ldf) {
  __shared__ float part[8][2][128];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, h = lane >> 4, j = lane & 15;
  const int nj = ld_src / 8;
  for (int64_t u = blockIdx.x; u < m; u += gridDim.x) {
    const int64_t S0 = row_ptr[u], E0 = row_ptr[u + 1];
    float b[8], d[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) b[q] = d[q] = 0.f;
    for (int64_t q0 = S0 + 32 * w; q0 < E0; q0 += 256) {
      const int64_t q = q0 + lane;
      const int cl = q < E0 ? col[q] : -1;
      const float rl = q < E0 ? val[q] : 0.f;
#pragma unroll 8
      for (int k = 0; k < 32; k += 2) {
        const int ci = __shfl_sync(0xffffffffu, cl, k + h);
        const float ri = __shfl_sync(0xffffffffu, rl, k + h);
        if (ci >= 0 && j < nj) {
          const uint4 raw = __ldg(reinterpret_cast<const uint4 *>(src + (size_t)ci * ld_src) + j);
          const LP *v = reinterpret_cast<const LP *>(&raw);
#pragma unroll
          for (int t = 0; t < 8; ++t) {
            const float x = (float)v[t];
            b[t] = fmaf(ri, x, b[t]);
            d[t] = fmaf(x, x, d[t]);
          }
        }
      }
    }
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      b[t] += __shfl_xor_sync(0xffffffffu, b[t], 16);
      d[t] += __shfl_xor_sync(0xffffffffu, d[t], 16);
    }
    if (h == 0) {
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        part[w][0][8 * j + t] = b[t];
        part[w][1][8 * j + t] = d[t];
      }
    }
    __syncthreads();
    const float n = (float)(E0 - S0), inv = n > 0.f ? 1.f / n : 0.f;
    __nv_bfloat16 *o = F + u * ldf;
    for (int i = threadIdx.x; i < ldf; i += blockDim.x) {
      float v = 0.f;
      if (i < 2 * f) {
        const int hh = i < f ? 0 : 1, c = i < f ? i : i - f;
        for (int k = 0; k < 8; ++k) v += part[k][hh][c];
        v *= inv;
      } else if (i == 2 * f) {
        v = log1pf(n) * 0.125f;
      }
      o[i] = __float2bfloat16(v);
    }
    __syncthreads();
  }
}

// Features driven by a side's work plan: one block per work item (a row, or
// a chunk of a row too long for one block), largest first. A chunk stores its
// sums in its partial slot; the chunk that finishes last adds the row's slots
// in chunk order (deterministic) and writes the features.
template <typename LP>
__global__ void __launch_bounds__(256) features_plan_kernel(WsPlan plan, int f, const int32_t *col,
                                                            const float *val, const LP *src,
                                                            int ld_src, __nv_bfloat16 *F, int ldf) {
  __shared__ float part[8][2][128];
  __shared__ float tot[256];
  __shared__ int last;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, h = lane >> 4, j = lane & 15;
  // 16-byte pieces that hold columns below f (at most 16 for f <= 128; the
  // stride may have one more piece of padding, which the features never read)
  const int nj = min(ld_src / 8, (f + 7) / 8);
  const int64_t nitems = plan.nitems_dev ? *plan.nitems_dev : plan.nitems;
  for (int64_t idx = blockIdx.x; idx < nitems; idx += gridDim.x) {
    const WorkItem it = plan.items[idx];
    const int64_t S0 = it.s, E0 = it.e;
    float b[8], d[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) b[q] = d[q] = 0.f;
    for (int64_t q0 = S0 + 32 * w; q0 < E0; q0 += 256) {
      const int64_t q = q0 + lane;
      const int cl = q < E0 ? col[q] : -1;
      const float rl = q < E0 ? val[q] : 0.f;
#pragma unroll 8
      for (int k = 0; k < 32; k += 2) {
        const int ci = __shfl_sync(0xffffffffu, cl, k + h);
        const float ri = __shfl_sync(0xffffffffu, rl, k + h);
        if (ci >= 0 && j < nj) {
          const uint4 raw = __ldg(reinterpret_cast<const uint4 *>(src + (size_t)ci * ld_src) + j);
          const LP *v = reinterpret_cast<const LP *>(&raw);
#pragma unroll
          for (int t = 0; t < 8; ++t) {
            const float x = (float)v[t];
            b[t] = fmaf(ri, x, b[t]);
            d[t] = fmaf(x, x, d[t]);
          }
        }
      }
    }
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      b[t] += __shfl_xor_sync(0xffffffffu, b[t], 16);
      d[t] += __shfl_xor_sync(0xffffffffu, d[t], 16);
    }
    if (h == 0) {
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        part[w][0][8 * j + t] = b[t];
        part[w][1][8 * j + t] = d[t];
      }
    }
    __syncthreads();
    {
      const int i = threadIdx.x, hh = i >> 7, c = i & 127;
      float v = 0.f;
      for (int k = 0; k < 8; ++k) v += part[k][hh][c];
      tot[i] = v;
    }
    __syncthreads();
    if (it.part >= 0) {
      float *P = plan.partial + (size_t)it.part * 128 * plan.part_ld;
      __stcg(P + threadIdx.x, tot[threadIdx.x]);
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) {
        const unsigned done = atomicAdd(&plan.heavy_count[it.heavy], 1u) + 1;
        last = done == (unsigned)plan.heavy_nchunks[it.heavy] ? 1 : 0;
      }
      __syncthreads();
      if (!last) continue;
      __threadfence();
      const int base = plan.heavy_base[it.heavy], nch = plan.heavy_nchunks[it.heavy];
      float v = 0.f;
      for (int ch = 0; ch < nch; ++ch)
        v += __ldcg(plan.partial + (size_t)(base + ch) * 128 * plan.part_ld + threadIdx.x);
      __syncthreads();
      tot[threadIdx.x] = v;
      if (threadIdx.x == 0) plan.heavy_count[it.heavy] = 0;  // ready for the next use
      __syncthreads();
    }
    const float n = (float)it.deg, inv = n > 0.f ? 1.f / n : 0.f;
    __nv_bfloat16 *o = F + (size_t)it.u * ldf;
    for (int i = threadIdx.x; i < ldf; i += blockDim.x) {
      float v = 0.f;
      if (i < 2 * f) v = (i < f ? tot[i] : tot[128 + i - f]) * inv;
      else if (i == 2 * f) v = log1pf(n) * 0.125f;
      o[i] = __float2bfloat16(v);
    }
    __syncthreads();
  }
}

// dY = 2 (Y - T) / (B f) for the loss mean_b |Y_b - T_b|^2 / f; loss partials in FP64.
__global__ void loss_grad_kernel(int64_t B, int f, const float *Y, int ldy, const float *T,
                                 int ldt, __nv_bfloat16 *dY, float *dY32, int lddy,
                                 double *loss) {
  const double scale = 1.0 / ((double)B * f);
  double acc = 0.0;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < B * lddy;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = q / lddy;
    const int j = (int)(q - b * lddy);
    float g = 0.f;
    if (j < f) {
      const float e = Y[b * ldy + j] - T[b * ldt + j];
      acc += (double)e * e;
      g = (float)(2.0 * scale) * e;
    }
    dY[b * lddy + j] = __float2bfloat16(g);
    dY32[b * lddy + j] = g;
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, acc * scale);
}

// out[n] (+)= sum_m X[m][n]
__global__ void colsum_kernel(int M, int N, const float *X, int ld, float *out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int m = 0; m < M; ++m) s += X[(int64_t)m * ld + n];
  out[n] = s;
}

__global__ void adam_kernel(int64_t n, float *w, float *mo, float *ve, const float *g, float lr,
                            float b1, float b2, float eps, float c1, float c2,
                            __nv_bfloat16 *w16) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float m = b1 * mo[i] + (1.f - b1) * gi;
    const float v = b2 * ve[i] + (1.f - b2) * gi * gi;
    mo[i] = m;
    ve[i] = v;
    const float wi = w[i] - lr * (m * c1) / (sqrtf(v * c2) + eps);
    w[i] = wi;
    if (w16) w16[i] = __float2bfloat16(wi);
  }
}

__global__ void to_bf16_kernel(int64_t n, const float *x, __nv_bfloat16 *y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16(x[i]);
}

// Gather rows idx[0..B) of features (bf16, ldf) and targets (fp32, ldt).
__global__ void gather_rows_kernel(int64_t B, const int32_t *idx, const __nv_bfloat16 *F, int ldf,
                                   const float *T, int ldt, int f, __nv_bfloat16 *Fo,
                                   float *To) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < B * ldf;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = q / ldf;
    const int j = (int)(q - b * ldf);
    const int64_t r = idx[b];
    Fo[q] = F[r * ldf + j];
    if (j < f) To[b * f + j] = T[r * ldt + j];
  }
}

}  // namespace mlp
}  // namespace als

// ---------------------------------------------------------------------------
// host side: parameters, Adam state, activations
// ---------------------------------------------------------------------------
namespace als {
namespace mlp {

struct Net {
  int f = 0, din = 0, ldf = 0, fp = 0, hid = 256;
  int64_t cap = 0;  // rows per GEMM pass
  int step = 0;
  // FP32 master parameters, then their Adam moments and gradients (same layout)
  float *P = nullptr, *Mo = nullptr, *Ve = nullptr, *G = nullptr;
  int64_t nparam = 0;
  float *W1, *b1, *W2, *b2, *W3, *b3;        // views into P
  float *gW1, *gb1, *gW2, *gb2, *gW3, *gb3;  // views into G
  __nv_bfloat16 *W16 = nullptr;              // BF16 copy of P (weights used by the GEMMs)
  __nv_bfloat16 *W1h, *W2h, *W3h;
  // activations for `cap` rows
  float *Z1, *Z2, *Y, *dY32, *dZ32;
  __nv_bfloat16 *H1, *H2, *dY16, *dZ2h, *dZ1h, *Fb;
  float *Tb;
  int32_t *idx;
  double *loss;
  int *error;
  void *block = nullptr;
};

static size_t al(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace mlp
}  // namespace als

namespace als {
namespace mlp {

static uint64_t mix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// He-normal weights (std sqrt(2 / fan_in)), zero biases; padding rows stay zero.
static void init_params(Net &n, uint64_t seed, std::vector<float> &h) {
  h.assign((size_t)n.nparam, 0.f);
  auto fill = [&](size_t off, int rows, int cols, int ld, int fan_in, uint64_t stream) {
    const double sd = std::sqrt(2.0 / fan_in);
    for (int r = 0; r < rows; ++r)
      for (int c = 0; c < cols; ++c) {
        uint64_t k = mix(seed ^ (stream << 40) ^ ((uint64_t)r << 20) ^ (uint64_t)c);
        double u1 = ((k >> 11) + 1) * 0x1.0p-53;
        double u2 = ((mix(k) >> 11) + 1) * 0x1.0p-53;
        h[off + (size_t)r * ld + c] =
            (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
      }
  };
  fill(n.W1 - n.P, n.hid, n.din, n.ldf, n.din, 1);
  fill(n.W2 - n.P, n.hid, n.hid, n.hid, n.hid, 2);
  fill(n.W3 - n.P, n.f, n.hid, n.hid, n.hid, 3);
}

static cudaError_t create(Net *&out, int f, int64_t cap, uint64_t seed, cudaStream_t st) {
  Net *n = new Net();
  n->f = f;
  n->din = 2 * f + 1;
  n->ldf = (n->din + 7) / 8 * 8;
  n->fp = (f + 7) / 8 * 8;
  n->cap = (cap + 127) / 128 * 128;
  const int H = n->hid;
  const int64_t sW1 = (int64_t)H * n->ldf, sW2 = (int64_t)H * H, sW3 = (int64_t)n->fp * H;
  n->nparam = sW1 + H + sW2 + H + sW3 + n->fp;
  const int64_t C = n->cap;
  size_t off = 0;
  auto take = [&](size_t b) { size_t p = off; off = al(off + b); return p; };
  const size_t oP = take(4 * n->nparam), oM = take(4 * n->nparam), oV = take(4 * n->nparam),
               oG = take(4 * n->nparam), oW16 = take(2 * n->nparam);
  const size_t oZ1 = take(4 * C * H), oZ2 = take(4 * C * H), oY = take(4 * C * n->fp),
               oDY32 = take(4 * C * n->fp), oDZ32 = take(4 * C * H);
  const size_t oH1 = take(2 * C * H), oH2 = take(2 * C * H), oDY16 = take(2 * C * n->fp),
               oDZ2 = take(2 * C * H), oDZ1 = take(2 * C * H), oFb = take(2 * C * n->ldf),
               oTb = take(4 * C * f), oIdx = take(4 * C), oLoss = take(8), oErr = take(4);
  cudaError_t e = cudaMalloc(&n->block, off);
  if (e != cudaSuccess) { delete n; return e; }
  char *b = (char *)n->block;
  n->P = (float *)(b + oP); n->Mo = (float *)(b + oM); n->Ve = (float *)(b + oV);
  n->G = (float *)(b + oG); n->W16 = (__nv_bfloat16 *)(b + oW16);
  n->W1 = n->P; n->b1 = n->W1 + sW1; n->W2 = n->b1 + H; n->b2 = n->W2 + sW2; n->W3 = n->b2 + H;
  n->b3 = n->W3 + sW3;
  n->gW1 = n->G; n->gb1 = n->gW1 + sW1; n->gW2 = n->gb1 + H; n->gb2 = n->gW2 + sW2;
  n->gW3 = n->gb2 + H; n->gb3 = n->gW3 + sW3;
  n->W1h = n->W16; n->W2h = n->W1h + sW1 + H; n->W3h = n->W2h + sW2 + H;
  n->Z1 = (float *)(b + oZ1); n->Z2 = (float *)(b + oZ2); n->Y = (float *)(b + oY);
  n->dY32 = (float *)(b + oDY32); n->dZ32 = (float *)(b + oDZ32);
  n->H1 = (__nv_bfloat16 *)(b + oH1); n->H2 = (__nv_bfloat16 *)(b + oH2);
  n->dY16 = (__nv_bfloat16 *)(b + oDY16); n->dZ2h = (__nv_bfloat16 *)(b + oDZ2);
  n->dZ1h = (__nv_bfloat16 *)(b + oDZ1); n->Fb = (__nv_bfloat16 *)(b + oFb);
  n->Tb = (float *)(b + oTb); n->idx = (int32_t *)(b + oIdx); n->loss = (double *)(b + oLoss);
  n->error = (int *)(b + oErr);
  std::vector<float> h;
  init_params(*n, seed, h);
  e = cudaMemsetAsync(n->block, 0, off, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(n->P, h.data(), 4 * n->nparam, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    to_bf16_kernel<<<256, 256, 0, st>>>(n->nparam, n->P, n->W16);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // h goes out of scope
  if (e != cudaSuccess) { cudaFree(n->block); delete n; return e; }
  out = n;
  return cudaSuccess;
}

static GemmArgs gargs() {
  GemmArgs g;
  std::memset(&g, 0, sizeof(g));
  return g;
}

// Forward over B <= cap rows of features F (ld ldf). Keeps Z1, Z2 when `train`.
static cudaError_t forward(Net &n, int64_t B, const __nv_bfloat16 *F, bool train, float *Yout,
                           int ldy, cudaStream_t st) {
  const int H = n.hid;
  GemmArgs g = gargs();
  g.M = (int)B; g.N = H; g.K = n.ldf; g.A = F; g.lda = n.ldf; g.B = n.W1h; g.ldb = n.ldf;
  g.bias = n.b1; g.act = kActGelu; g.C16 = n.H1; g.ldc16 = H; g.error = n.error;
  if (train) { g.Z = n.Z1; g.ldz = H; }
  cudaError_t e = gemm(g, st);
  if (e != cudaSuccess) return e;
  g = gargs();
  g.M = (int)B; g.N = H; g.K = H; g.A = n.H1; g.lda = H; g.B = n.W2h; g.ldb = H;
  g.bias = n.b2; g.act = kActGelu; g.C16 = n.H2; g.ldc16 = H; g.error = n.error;
  if (train) { g.Z = n.Z2; g.ldz = H; }
  if ((e = gemm(g, st)) != cudaSuccess) return e;
  g = gargs();
  g.M = (int)B; g.N = n.f; g.K = H; g.A = n.H2; g.lda = H; g.B = n.W3h; g.ldb = H;
  g.bias = n.b3; g.C32 = Yout; g.ldc32 = ldy; g.error = n.error;
  return gemm(g, st);
}

// Loss and gradients for B rows (features Fb, targets Tb, ld f), into n.G.
static cudaError_t backward(Net &n, int64_t B, const __nv_bfloat16 *F, const float *T, int ldt,
                            cudaStream_t st) {
  const int H = n.hid, fp = n.fp;
  cudaError_t e = forward(n, B, F, true, n.Y, fp, st);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(n.loss, 0, sizeof(double), st)) != cudaSuccess) return e;
  loss_grad_kernel<<<256, 256, 0, st>>>(B, n.f, n.Y, fp, T, ldt, n.dY16, n.dY32, fp, n.loss);
  colsum_kernel<<<(fp + 127) / 128, 128, 0, st>>>((int)B, fp, n.dY32, fp, n.gb3);
  GemmArgs g = gargs();
  // G3 = dY^T H2   [fp x H], K = B
  g.M = fp; g.N = H; g.K = (int)B; g.A = n.dY16; g.lda = fp; g.a_mn = 1; g.B = n.H2; g.ldb = H;
  g.b_mn = 1; g.C32 = n.gW3; g.ldc32 = H; g.error = n.error;
  if ((e = gemm(g, st)) != cudaSuccess) return e;
  // dZ2 = (dY W3) * gelu'(Z2)
  g = gargs();
  g.M = (int)B; g.N = H; g.K = fp; g.A = n.dY16; g.lda = fp; g.B = n.W3h; g.ldb = H; g.b_mn = 1;
  g.act = kActGeluGrad; g.aux = n.Z2; g.ldaux = H; g.C16 = n.dZ2h; g.ldc16 = H; g.C32 = n.dZ32;
  g.ldc32 = H; g.error = n.error;
  if ((e = gemm(g, st)) != cudaSuccess) return e;
  colsum_kernel<<<(H + 127) / 128, 128, 0, st>>>((int)B, H, n.dZ32, H, n.gb2);
  // G2 = dZ2^T H1  [H x H]
  g = gargs();
  g.M = H; g.N = H; g.K = (int)B; g.A = n.dZ2h; g.lda = H; g.a_mn = 1; g.B = n.H1; g.ldb = H;
  g.b_mn = 1; g.C32 = n.gW2; g.ldc32 = H; g.error = n.error;
  if ((e = gemm(g, st)) != cudaSuccess) return e;
  // dZ1 = (dZ2 W2) * gelu'(Z1)
  g = gargs();
  g.M = (int)B; g.N = H; g.K = H; g.A = n.dZ2h; g.lda = H; g.B = n.W2h; g.ldb = H; g.b_mn = 1;
  g.act = kActGeluGrad; g.aux = n.Z1; g.ldaux = H; g.C16 = n.dZ1h; g.ldc16 = H; g.C32 = n.dZ32;
  g.ldc32 = H; g.error = n.error;
  if ((e = gemm(g, st)) != cudaSuccess) return e;
  colsum_kernel<<<(H + 127) / 128, 128, 0, st>>>((int)B, H, n.dZ32, H, n.gb1);
  // G1 = dZ1^T F  [H x ldf]
  g = gargs();
  g.M = H; g.N = n.ldf; g.K = (int)B; g.A = n.dZ1h; g.lda = H; g.a_mn = 1; g.B = F; g.ldb = n.ldf;
  g.b_mn = 1; g.C32 = n.gW1; g.ldc32 = n.ldf; g.error = n.error;
  if ((e = gemm(g, st)) != cudaSuccess) return e;
  return cudaGetLastError();
}

// Rows for a training batch: B seeded draws from [0, m).
__global__ void sample_rows_kernel(int64_t B, int64_t m, uint64_t seed, int32_t *idx) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < B;
       b += (int64_t)gridDim.x * blockDim.x) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ULL * (uint64_t)(b + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    idx[b] = (int32_t)(z % (uint64_t)m);
  }
}

static cudaError_t adam(Net &n, float lr, cudaStream_t st) {
  ++n.step;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f / (1.f - std::pow(b1, (float)n.step));
  const float c2 = 1.f / (1.f - std::pow(b2, (float)n.step));
  adam_kernel<<<512, 256, 0, st>>>(n.nparam, n.P, n.Mo, n.Ve, n.G, lr, b1, b2, eps, c1, c2, n.W16);
  return cudaGetLastError();
}

// One Adam step on a batch of B <= cap rows (features ld ldf, targets ld ldt).
static cudaError_t train_step(Net &n, int64_t B, const __nv_bfloat16 *F, const float *T, int ldt,
                              float lr, cudaStream_t st) {
  cudaError_t e = backward(n, B, F, T, ldt, st);
  if (e != cudaSuccess) return e;
  return adam(n, lr, st);
}

// Sample B rows of (features, targets) and take one Adam step on them.
static cudaError_t train_sampled(Net &n, int64_t m, int64_t B, const __nv_bfloat16 *F,
                                 const float *T, int ldt, float lr, uint64_t seed,
                                 cudaStream_t st) {
  if (B > n.cap) B = n.cap;
  B = B / 64 * 64;
  if (B <= 0 || m <= 0) return cudaSuccess;
  sample_rows_kernel<<<64, 256, 0, st>>>(B, m, seed, n.idx);
  gather_rows_kernel<<<512, 256, 0, st>>>(B, n.idx, F, n.ldf, T, ldt, n.f, n.Fb, n.Tb);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return train_step(n, B, n.Fb, n.Tb, n.f, lr, st);
}

// x0 for rows [0, m): forward in chunks of cap rows.
static cudaError_t infer(Net &n, int64_t m, const __nv_bfloat16 *F, float *X0, int ldx,
                         cudaStream_t st) {
  for (int64_t r0 = 0; r0 < m; r0 += n.cap) {
    const int64_t B = m - r0 < n.cap ? m - r0 : n.cap;
    cudaError_t e = forward(n, B, F + r0 * n.ldf, false, X0 + r0 * ldx, ldx, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace mlp
}  // namespace als

// ---------------------------------------------------------------------------
// entry points used by the engine and the C ABI
// ---------------------------------------------------------------------------
namespace als {

cudaError_t mlp_create(void **out, int f, int64_t cap, uint64_t seed, cudaStream_t st) {
  mlp::Net *n = nullptr;
  cudaError_t e = mlp::create(n, f, cap, seed, st);
  *out = n;
  return e;
}
void mlp_destroy(void *p) {
  mlp::Net *n = (mlp::Net *)p;
  if (!n) return;
  cudaFree(n->block);
  delete n;
}
int mlp_ldf(const void *p) { return ((const mlp::Net *)p)->ldf; }
int64_t mlp_nparam(const void *p) { return ((const mlp::Net *)p)->nparam; }
int *mlp_error(const void *p) { return ((const mlp::Net *)p)->error; }

cudaError_t mlp_features_plan(const WsPlan &plan, int f, const int32_t *col, const float *val,
                              const void *src, int ld_src, int lp_kind, void *F, int ldf,
                              cudaStream_t st) {
  if (plan.nitems <= 0) return cudaSuccess;
  if (f > 128 || ld_src % 8 != 0 || ld_src < f || (reinterpret_cast<uintptr_t>(src) & 15) != 0 ||
      plan.part_ld * 128 < 256 || (lp_kind != kLpBf16 && lp_kind != kLpFp16))
    return cudaErrorNotSupported;
  const unsigned grid = (unsigned)std::min<int64_t>(plan.nitems, (int64_t)device_sm_count() * 8);
  if (lp_kind == kLpBf16)
    mlp::features_plan_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(
        plan, f, col, val, (const __nv_bfloat16 *)src, ld_src, (__nv_bfloat16 *)F, ldf);
  else
    mlp::features_plan_kernel<__half><<<grid, 256, 0, st>>>(
        plan, f, col, val, (const __half *)src, ld_src, (__nv_bfloat16 *)F, ldf);
  return cudaGetLastError();
}

cudaError_t mlp_features(int64_t m, int f, const int64_t *row_ptr, const int32_t *col,
                         const float *val, const void *src, int ld_src, int lp_kind, void *F,
                         int ldf, cudaStream_t st) {
  if (m <= 0) return cudaSuccess;
  if (f > 128) return cudaErrorInvalidValue;
  const unsigned grid = (unsigned)std::min<int64_t>(m, 148 * 8);
  const bool pieces = ld_src % 8 == 0 && ld_src <= 128 &&
                      (reinterpret_cast<uintptr_t>(src) & 15) == 0;
  if (lp_kind == kLpBf16 && pieces)
    mlp::features_lp_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(
        m, f, row_ptr, col, val, (const __nv_bfloat16 *)src, ld_src, (__nv_bfloat16 *)F, ldf);
  else if (lp_kind == kLpFp16 && pieces)
    mlp::features_lp_kernel<__half><<<grid, 256, 0, st>>>(m, f, row_ptr, col, val,
                                                          (const __half *)src, ld_src,
                                                          (__nv_bfloat16 *)F, ldf);
  else if (lp_kind == kLpBf16)
    mlp::features_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(
        m, f, row_ptr, col, val, (const __nv_bfloat16 *)src, ld_src, (__nv_bfloat16 *)F, ldf);
  else if (lp_kind == kLpFp16)
    mlp::features_kernel<__half><<<grid, 256, 0, st>>>(m, f, row_ptr, col, val,
                                                       (const __half *)src, ld_src,
                                                       (__nv_bfloat16 *)F, ldf);
  else
    mlp::features_kernel<float><<<grid, 256, 0, st>>>(m, f, row_ptr, col, val, (const float *)src,
                                                      ld_src, (__nv_bfloat16 *)F, ldf);
  return cudaGetLastError();
}

cudaError_t mlp_infer(void *p, int64_t m, const void *F, float *X0, int ldx, cudaStream_t st) {
  return mlp::infer(*(mlp::Net *)p, m, (const __nv_bfloat16 *)F, X0, ldx, st);
}

cudaError_t mlp_train(void *p, int64_t m, int64_t batch, int steps, const void *F, const float *T,
                      int ldt, float lr, uint64_t seed, cudaStream_t st) {
  mlp::Net &n = *(mlp::Net *)p;
  for (int s = 0; s < steps; ++s) {
    cudaError_t e = mlp::train_sampled(n, m, batch, (const __nv_bfloat16 *)F, T, ldt, lr,
                                       seed * 1000003ULL + (uint64_t)s, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Loss and gradients (no update) on B rows; gradients stay in the net's G.
cudaError_t mlp_gradients(void *p, int64_t B, const void *F, const float *T, int ldt,
                          cudaStream_t st) {
  return mlp::backward(*(mlp::Net *)p, B, (const __nv_bfloat16 *)F, T, ldt, st);
}

cudaError_t mlp_step(void *p, int64_t B, const void *F, const float *T, int ldt, float lr,
                     cudaStream_t st) {
  return mlp::train_step(*(mlp::Net *)p, B, (const __nv_bfloat16 *)F, T, ldt, lr, st);
}

// Copy parameters (what = 0), gradients (1) to host, or set parameters (2) from host,
// unpadded: W1 [256 x (2f+1)], b1 [256], W2 [256 x 256], b2 [256], W3 [f x 256], b3 [f].
cudaError_t mlp_io(void *p, float *host, int what, double *loss, cudaStream_t st) {
  mlp::Net &n = *(mlp::Net *)p;
  const int H = n.hid;
  struct Blk { float *dev; int rows, cols, ld; };
  float *base = what == 1 ? n.G : n.P;
  const Blk blks[6] = {{base + (n.W1 - n.P), H, n.din, n.ldf}, {base + (n.b1 - n.P), 1, H, H},
                       {base + (n.W2 - n.P), H, H, H},        {base + (n.b2 - n.P), 1, H, H},
                       {base + (n.W3 - n.P), n.f, H, H},      {base + (n.b3 - n.P), 1, n.f, n.fp}};
  size_t off = 0;
  cudaError_t e = cudaSuccess;
  for (const Blk &b : blks) {
    if (what == 2)
      e = cudaMemcpy2DAsync(b.dev, 4 * b.ld, host + off, 4 * b.cols, 4 * b.cols, b.rows,
                            cudaMemcpyHostToDevice, st);
    else
      e = cudaMemcpy2DAsync(host + off, 4 * b.cols, b.dev, 4 * b.ld, 4 * b.cols, b.rows,
                            cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    off += (size_t)b.rows * b.cols;
  }
  if (what == 2) {
    mlp::to_bf16_kernel<<<256, 256, 0, st>>>(n.nparam, n.P, n.W16);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (loss && what == 1) e = cudaMemcpyAsync(loss, n.loss, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(st);
}

int64_t mlp_param_count(int f) {
  const int64_t din = 2 * f + 1, H = 256;
  return H * din + H + H * H + H + (int64_t)f * H + f;
}

}  // namespace als
