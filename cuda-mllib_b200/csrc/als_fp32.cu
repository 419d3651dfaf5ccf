// FP32 form of the ALS half-step: one CTA per CSR row, persistent over a
// degree-ordered work queue. Per row:
//   gather   theta rows of the row's items into shared memory, KC at a time
//            (float4 loads when the row stride allows);
//   hermitian A_u = sum theta_i theta_i^T on CUDA cores, one 8x8 lower-triangle
//            register tile per thread, b_u = sum r_ui theta_i on the diagonal
//            tiles' threads, + lambda * n_u on the diagonal;
//   solve    register-tile blocked Cholesky, two triangular solves, one
//            FP64-residual refinement step for rows whose FP32 relative
//            residual exceeds the tolerance.
// A_u never leaves the SM (the reference writes f*f doubles per row to HBM,
// als/src/cuda/als.cu:1069-1081, then runs cuBLAS batched LU on them,
// als.cu:939-997).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "als_common.cuh"
#include "als_internal.h"

namespace als {

template <int FP>
struct Fp32Cfg {
  static constexpr int T8 = FP / 8;
  static constexpr int NTILES = T8 * (T8 + 1) / 2;
  static constexpr int NT = ((NTILES + 31) / 32) * 32;
  static constexpr int KC = 32;       // items staged per chunk
  // CTAs per SM the register allocation must allow (at most ~168 registers a
  // thread), so the staged loads do not cost occupancy
  static constexpr int kMinBlocks = 65536 / (NT * 168) > 0 ? 65536 / (NT * 168) : 1;
  static constexpr int LDS = FP + 1;  // row stride of S (odd: conflict-free columns)
  static constexpr size_t kStage = (size_t)KC * FP * 4 + (size_t)KC * 8;
  static constexpr size_t kS = (size_t)FP * LDS * 4;
  static constexpr size_t kMain = ((kStage > kS ? kStage : kS) + 15) / 16 * 16;
  // dg, bv, xv, tmp (floats) + rd (doubles) + misc ints
  static constexpr size_t kSmem = kMain + 4 * FP * 4 + FP * 8 + 64;
};

template <typename T>
__device__ __forceinline__ void store_lp(void *p, int64_t idx, float v) {
  reinterpret_cast<T *>(p)[idx] = T(v);
}

template <int FP, bool VEC>
__global__ void __launch_bounds__(Fp32Cfg<FP>::NT, Fp32Cfg<FP>::kMinBlocks)
rows_fp32_kernel(RowsArgs a, int lp_kind) {
  using C = Fp32Cfg<FP>;
  constexpr int KC = C::KC, LDS = C::LDS, NT = C::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float *S = reinterpret_cast<float *>(smem_raw);
  float *th = S;                                        // KC x FP (aliases S)
  float *rv = th + KC * FP;                             // KC
  int *colk = reinterpret_cast<int *>(rv + KC);         // KC
  float *dg = reinterpret_cast<float *>(smem_raw + C::kMain);
  float *bv = dg + FP, *xv = bv + FP, *tmp = xv + FP;
  double *rd = reinterpret_cast<double *>(tmp + FP);
  int *misc = reinterpret_cast<int *>(rd + FP);

  __shared__ float red64[64];
  const int tid = threadIdx.x;
  const int f = a.f;
  int ti = 0, tj = 0;
  const bool owner = tid < C::NTILES;
  if (owner) tile_of(tid, ti, tj);
  const float *src = reinterpret_cast<const float *>(a.src);
  unsigned long long n_rows = 0, n_ref = 0, n_bad = 0;

  for (;;) {
    const int64_t u = next_row(a, &misc[0]);
    if (u < 0) break;
    const int64_t s = a.row_ptr[u], e = a.row_ptr[u + 1];
    const int64_t d = e - s;
    ++n_rows;
    if (d == 0) {
      for (int i = tid; i < f; i += NT) {
        a.dst[u * a.ld_dst + i] = 0.f;
        if (a.dst_lp) {
          if (lp_kind == 1) store_lp<__nv_bfloat16>(a.dst_lp, u * a.ld_dst_lp + i, 0.f);
          else store_lp<__half>(a.dst_lp, u * a.ld_dst_lp + i, 0.f);
        }
      }
      if (a.row_flags && tid == 0) a.row_flags[u] = kRowEmpty;
      continue;
    }
    float acc[8][8], bacc[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      bacc[r] = 0.f;
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[r][c] = 0.f;
    }
    for (int64_t k0 = s; k0 < e; k0 += KC) {
      const int kc = (int)(e - k0 < KC ? e - k0 : KC);
      __syncthreads();
      if (tid < KC) {
        colk[tid] = tid < kc ? a.col[k0 + tid] : 0;
        rv[tid] = tid < kc ? a.val[k0 + tid] : 0.f;
      }
      __syncthreads();
      if (VEC) {
        // A thread's float4 loads of the chunk go out kB at a time, each
        // batch issued before any of it is stored, so the chunk costs about
        // kV / kB memory latencies per thread rather than kV (kB is kept small
        // so the batch fits beside the 8x8 accumulator tile in registers).
        constexpr int C4 = FP / 4, kV = (KC * C4 + NT - 1) / NT, kB = 3;
#pragma unroll
        for (int i0 = 0; i0 < kV; i0 += kB) {
          float4 v[kB];
#pragma unroll
          for (int i = 0; i < kB; ++i) {
            const int q = tid + (i0 + i) * NT, k = q / C4, c4 = q - k * C4;
            v[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (i0 + i < kV && q < KC * C4 && k < kc && 4 * c4 < f)
              v[i] = __ldg(reinterpret_cast<const float4 *>(src + (int64_t)colk[k] * a.ld_src) + c4);
          }
#pragma unroll
          for (int i = 0; i < kB; ++i) {
            const int q = tid + (i0 + i) * NT;
            if (i0 + i < kV && q < KC * C4) reinterpret_cast<float4 *>(th)[q] = v[i];
          }
        }
      } else {
        for (int q = tid; q < KC * FP; q += NT) {
          const int k = q / FP, c = q - k * FP;
          float v = 0.f;
          if (k < kc && c < f) v = __ldg(src + (int64_t)colk[k] * a.ld_src + c);
          th[q] = v;
        }
      }
      __syncthreads();
      if (owner) {
        const float4 *t4 = reinterpret_cast<const float4 *>(th);
#pragma unroll 2
        for (int k = 0; k < kc; ++k) {
          const float4 a0 = t4[k * (FP / 4) + 2 * ti], a1 = t4[k * (FP / 4) + 2 * ti + 1];
          const float4 b0 = t4[k * (FP / 4) + 2 * tj], b1 = t4[k * (FP / 4) + 2 * tj + 1];
          const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
          const float bw[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
          for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int c = 0; c < 8; ++c) acc[r][c] = fmaf(av[r], bw[c], acc[r][c]);
          if (ti == tj) {
            const float rk = rv[k];
#pragma unroll
            for (int r = 0; r < 8; ++r) bacc[r] = fmaf(rk, av[r], bacc[r]);
          }
        }
      }
    }
    __syncthreads();  // staging area becomes S
    const float reg = a.lambda * (float)d;
    if (owner) {
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const int i = 8 * ti + r, j = 8 * tj + c;
          if (i > j) S[j * LDS + i] = acc[r][c];
          else if (i < j) S[i * LDS + j] = acc[r][c];
          else {
            const float v = acc[r][c] + (i < f ? reg : 1.f);
            acc[r][c] = v;
            dg[i] = v;
          }
        }
      if (ti == tj)
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          const float bvv = (8 * ti + r < f) ? bacc[r] : 0.f;
          bv[8 * ti + r] = bvv;
          xv[8 * ti + r] = bvv;
        }
    }
    const bool ok = tile_cholesky<FP, LDS, NT>(acc, ti, tj, owner, S, &misc[1], cta_bar());
    uint32_t flags = 0;
    if (!ok) {
      for (int i = tid; i < f; i += NT) xv[i] = 0.f;
      flags |= kRowNotSPD;
      ++n_bad;
      __syncthreads();
    } else {
      bool refined = false;
      solve_and_refine<FP, LDS, NT>(S, dg, bv, xv, rd, tmp, f, a.refine_tol, &refined, red64,
                                      cta_bar());
      if (refined) { flags |= kRowRefinedF64; ++n_ref; }
    }
    for (int i = tid; i < f; i += NT) {
      const float v = xv[i];
      a.dst[u * a.ld_dst + i] = v;
      if (a.dst_lp) {
        if (lp_kind == 1) store_lp<__nv_bfloat16>(a.dst_lp, u * a.ld_dst_lp + i, v);
        else store_lp<__half>(a.dst_lp, u * a.ld_dst_lp + i, v);
      }
    }
    if (a.row_flags && tid == 0) a.row_flags[u] = flags;
  }
  if (a.counters && tid == 0) {
    atomicAdd(&a.counters->rows, n_rows);
    if (n_ref) atomicAdd(&a.counters->refined, n_ref);
    if (n_bad) atomicAdd(&a.counters->not_spd, n_bad);
  }
}

template <int FP>
static cudaError_t launch_fp32_fp(const RowsArgs &a, int lp_kind, bool vec, int num_sms,
                                  cudaStream_t st) {
  using C = Fp32Cfg<FP>;
  auto kern = vec ? rows_fp32_kernel<FP, true> : rows_fp32_kernel<FP, false>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)C::kSmem);
  if (err != cudaSuccess) return err;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::NT, C::kSmem);
  if (err != cudaSuccess) return err;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int64_t grid = (int64_t)num_sms * per_sm;
  if (grid > a.m) grid = a.m > 0 ? a.m : 1;
  kern<<<(unsigned)grid, C::NT, C::kSmem, st>>>(a, lp_kind);
  return cudaGetLastError();
}

int fp32_padded_rank(int f) {
  if (f <= 16) return 16;
  if (f <= 32) return 32;
  if (f <= 64) return 64;
  if (f <= 104) return 104;
  if (f <= 128) return 128;
  return -1;
}

cudaError_t launch_rows_fp32(const RowsArgs &a, int lp_kind, int num_sms, cudaStream_t st) {
  const bool vec = (a.f % 4 == 0) && (a.ld_src % 4 == 0) &&
                   ((reinterpret_cast<uintptr_t>(a.src) & 15) == 0);
  switch (fp32_padded_rank(a.f)) {
    case 16: return launch_fp32_fp<16>(a, lp_kind, vec, num_sms, st);
    case 32: return launch_fp32_fp<32>(a, lp_kind, vec, num_sms, st);
    case 64: return launch_fp32_fp<64>(a, lp_kind, vec, num_sms, st);
    case 104: return launch_fp32_fp<104>(a, lp_kind, vec, num_sms, st);
    case 128: return launch_fp32_fp<128>(a, lp_kind, vec, num_sms, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace als
