// Tensor-core form of the ALS half-step (sm_100a, tcgen05 + TMEM).
//
// Per CSR row u (one CTA per row, persistent over the degree-ordered queue):
//
//   gather   the row's item factors (BF16 or FP16 copy, row stride LDP) are
//            loaded 16 B at a time and stored into a 128B-swizzled MN-major
//            shared-memory tile: item k is "K row" k, its f factor values run
//            along M/N. The rating r_uk is patched into element f of the row,
//            so column f of the product is b_u.
//   hermitian one elected thread issues tcgen05.mma.kind::f16 with
//            A = tile^T (M = 128), B = tile (N = NP = roundup16(f+1)), K = 16
//            per instruction, FP32 accumulation in TMEM:
//                D[m][n] = sum_k theta_k[m] * [theta_k | r_k][n]
//            i.e. D[:, :f] = sum theta theta^T and D[:, f] = b_u. Stages of 64
//            items are double-buffered: tcgen05.commit on a per-buffer mbarrier
//            releases a buffer once its MMAs completed, while the CTA gathers
//            the next stage into the other buffer.
//   solve    D is read back with tcgen05.ld (warp w reads TMEM lanes 32w..),
//            written to shared memory, and solved by the same register-tile
//            blocked Cholesky + FP64-residual refinement as the FP32 form.
//
// Every mbarrier wait is bounded: on timeout the kernel records an error code
// and the CTA stops taking rows (no spin is unbounded).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "als_common.cuh"
#include "als_internal.h"
#include "als_tcgen05.cuh"

namespace als {



// v with its 16-bit element pos (0..7) replaced by bits, by selects (no
// dynamic indexing, so v stays in registers)
__device__ __forceinline__ uint4 patch16(uint4 v, int pos, uint16_t bits) {
  const int sh = (pos & 1) * 16, w = pos >> 1;
  const uint32_t keep = ~(0xFFFFu << sh), put = (uint32_t)bits << sh;
  v.x = w == 0 ? (v.x & keep) | put : v.x;
  v.y = w == 1 ? (v.y & keep) | put : v.y;
  v.z = w == 2 ? (v.z & keep) | put : v.z;
  v.w = w == 3 ? (v.w & keep) | put : v.w;
  return v;
}

template <int FP>
struct TcCfg {
  static constexpr int T8 = FP / 8;
  static constexpr int NTILES = T8 * (T8 + 1) / 2;
  static constexpr int NT = ((NTILES + 31) / 32) * 32 < 128 ? 128 : ((NTILES + 31) / 32) * 32;
  static constexpr int LDS = FP + 1;
  static constexpr size_t kS = (size_t)FP * LDS * 4;
};

// Runtime geometry shared by host and device.
struct TcGeom {
  int np;        // MMA N
  int ldp;       // global row stride of the low-precision factors (elements)
  int chunks;    // 16 B chunks per global row = ldp / 8
  int atoms;     // MN atoms of 64 elements in the staged tile
  int stage_bytes;
  int tmem_cols;
};

__host__ __device__ inline TcGeom tc_geom(int f) {
  TcGeom g;
  g.np = ((f + 1 + 15) / 16) * 16;
  g.ldp = ((f + 1 + 7) / 8) * 8;
  g.chunks = g.ldp / 8;
  const int mn = g.np > 128 ? g.np : 128;
  g.atoms = (mn + 63) / 64;
  g.stage_bytes = g.atoms * (tc::KS / 8) * 1024;
  g.tmem_cols = g.np <= 32 ? 32 : g.np <= 64 ? 64 : g.np <= 128 ? 128 : 256;
  return g;
}



// Sum over the CTA of one value per thread; two slot sets alternate so one
// barrier per reduction suffices.
template <int NT>
__device__ __forceinline__ float cta_sum(float v, float *red, int &slot) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[slot * 8 + (threadIdx.x >> 5)] = v;
  __syncthreads();
  float s = 0.f;
#pragma unroll
  for (int w = 0; w < NT / 32; ++w) s += red[slot * 8 + w];
  slot ^= 1;
  return s;
}

template <int FP, int NP, typename LP>
__global__ void __launch_bounds__(TcCfg<FP>::NT)
rows_tc_kernel(RowsArgs a, TcGeom g, uint32_t idesc, TcSolve sv) {
  using C = TcCfg<FP>;
  constexpr int LDS = C::LDS, NT = C::NT;
  // 16-byte pieces per thread and stage: a stage holds KS rows of at most
  // (FP + 8) / 8 pieces (row stride roundup8(f + 1) <= FP + 8)
  constexpr int kQ = (tc::KS * ((FP + 8) / 8) + NT - 1) / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // 1024-aligned base for the swizzled stages
  unsigned char *base = smem_raw + ((1024 - (tc::smem_u32(smem_raw) & 1023)) & 1023);
  const size_t stages_bytes = (size_t)tc::kStages * g.stage_bytes;
  const size_t main_bytes = ((stages_bytes > C::kS ? stages_bytes : C::kS) + 15) / 16 * 16;
  float *S = reinterpret_cast<float *>(base);   // aliases the stages after the MMAs
  float *dg = reinterpret_cast<float *>(base + main_bytes);
  float *bv = dg + FP, *xv = bv + FP, *tmp = xv + FP;
  float *ps = tmp + FP;                                    // CG direction, NP entries
  float *red = ps + NP;                                    // 2 x 8 reduction slots
  double *rd = reinterpret_cast<double *>(red + 16);
  uint64_t *bars = reinterpret_cast<uint64_t *>(rd + FP);  // [0,1] stages, [2] acc, [3] drain
  int *misc = reinterpret_cast<int *>(bars + 4);          // slot, bad, tmem base, abort

  __shared__ float red64[64];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int f = a.f;
  const LP *src = reinterpret_cast<const LP *>(a.src);

  if (tid == 0) {
    for (int i = 0; i < 4; ++i) tc::mbar_init(&bars[i], 1);
    misc[3] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32(&misc[2])),
                 "r"(g.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  for (int q = tid; q < (int)(stages_bytes / 16); q += NT)
    reinterpret_cast<uint4 *>(base)[q] = make_uint4(0, 0, 0, 0);
  for (int q = tid; q < NP; q += NT) ps[q] = 0.f;
  tc::fence_proxy_async();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = (uint32_t)misc[2];

  int ti = 0, tj = 0;
  const bool owner = tid < C::NTILES;
  if (owner) tile_of(tid, ti, tj);
  unsigned uses0 = 0, uses1 = 0;  // commits issued per stage buffer
  unsigned acc_phase = 0;
  int rslot = 0;
  unsigned long long n_rows = 0, n_ref = 0, n_bad = 0, n_steps = 0, n_fb = 0, n_r0 = 0;
  const uint32_t lbo = (tc::KS / 8) * 1024, sbo = 1024;
  const uint32_t stage0 = tc::smem_u32(base);
  const int rchunk = f >> 3, rpos = f & 7;
  const int m = tid;                       // this thread's row of A_u (TMEM lane)
  const bool lane_row = warp < 4;          // warps 0-3 own TMEM lanes 0..127
  const bool live = lane_row && m < f;

  for (;;) {
    const int64_t u = next_row(a, &misc[0]);
    if (u < 0 || misc[3]) break;
    const int64_t s = a.row_ptr[u], e = a.row_ptr[u + 1];
    const int64_t d = e - s;
    ++n_rows;
    if (d == 0) {
      for (int i = tid; i < f; i += NT) {
        a.dst[u * a.ld_dst + i] = 0.f;
        if (a.dst_lp) reinterpret_cast<LP *>(a.dst_lp)[u * a.ld_dst_lp + i] = LP(0.f);
      }
      if (a.row_flags && tid == 0) a.row_flags[u] = kRowEmpty;
      continue;
    }
    // ---------------- gather + MMA over stages ----------------
    const int nstage = (int)((d + tc::KS - 1) / tc::KS);
    bool aborted = false;
    for (int gi = 0; gi < nstage; ++gi) {
      const int buf = gi & 1;
      const unsigned used = buf ? uses1 : uses0;
      // the MMAs of stage gi-2 read this buffer; wait for their commit
      const bool okw = gi < 2 || tc::mbar_wait(&bars[buf], (used - 1) & 1);
      const int64_t k0 = s + (int64_t)gi * tc::KS;
      const int kc = (int)(e - k0 < tc::KS ? e - k0 : tc::KS);
      const int krows = (kc + 15) & ~15;
      unsigned char *stg = base + (size_t)buf * g.stage_bytes;
      if (okw) {
        // Each thread copies up to kQ 16-byte pieces of the stage. The column
        // indices and ratings are read first and the factor pieces are then
        // loaded back to back, so a thread waits on two memory latencies per
        // stage instead of two per piece.
        const int total = krows * g.chunks;
        int64_t item[kQ];
        float rv[kQ];
#pragma unroll
        for (int i = 0; i < kQ; ++i) {
          const int q = tid + i * NT, k = q / g.chunks, j = q - k * g.chunks;
          const bool in = q < total && k < kc;
          item[i] = in ? (int64_t)a.col[k0 + k] : 0;
          rv[i] = (in && j == rchunk) ? a.val[k0 + k] : 0.f;
        }
        uint4 v[kQ];
#pragma unroll
        for (int i = 0; i < kQ; ++i) {
          const int q = tid + i * NT, k = q / g.chunks, j = q - k * g.chunks;
          v[i] = make_uint4(0, 0, 0, 0);
          if (q < total && k < kc) v[i] = __ldg(reinterpret_cast<const uint4 *>(src + item[i] * a.ld_src) + j);
        }
#pragma unroll
        for (int i = 0; i < kQ; ++i) {
          const int q = tid + i * NT, k = q / g.chunks, j = q - k * g.chunks;
          if (q < total) {
            if (k < kc && j == rchunk) v[i] = patch16(v[i], rpos, tc::to_bits<LP>(rv[i]));
            const int atom = j >> 3, c = j & 7, kg = k >> 3, kr = k & 7;
            *reinterpret_cast<uint4 *>(stg + atom * lbo + kg * 1024 + kr * 128 + ((c ^ kr) << 4)) = v[i];
          }
        }
        // pieces beyond kQ per thread (none while ld <= FP + 8): one at a time
        for (int q = tid + kQ * NT; q < total; q += NT) {
          const int k = q / g.chunks, j = q - k * g.chunks;
          uint4 w = make_uint4(0, 0, 0, 0);
          if (k < kc) {
            const int64_t it = a.col[k0 + k];
            w = __ldg(reinterpret_cast<const uint4 *>(src + it * a.ld_src) + j);
            if (j == rchunk) reinterpret_cast<uint16_t *>(&w)[rpos] = tc::to_bits<LP>(a.val[k0 + k]);
          }
          const int atom = j >> 3, c = j & 7, kg = k >> 3, kr = k & 7;
          *reinterpret_cast<uint4 *>(stg + atom * lbo + kg * 1024 + kr * 128 + ((c ^ kr) << 4)) = w;
        }
      }
      tc::fence_proxy_async();
      if (!__syncthreads_and(okw)) { aborted = true; break; }
      if (tid == 0) {
        tc::tc_fence_after();
        const uint32_t sa = stage0 + buf * g.stage_bytes;
        for (int kk = 0; kk < krows / 16; ++kk) {
          const uint64_t desc = tc::make_desc(sa + kk * 2 * sbo, lbo, sbo);
          tc::mma_f16(tmem, desc, desc, idesc, (gi > 0 || kk > 0) ? 1u : 0u);
        }
        tc::mma_commit(&bars[buf]);
        if (gi == nstage - 1) tc::mma_commit(&bars[2]);
      }
      if (buf) ++uses1; else ++uses0;
    }
    const bool oka = !aborted && tc::mbar_wait(&bars[2], acc_phase);
    acc_phase ^= 1;
    if (!__syncthreads_and(oka)) {
      if (tid == 0) { atomicCAS(a.error, 0, 1); misc[3] = 1; }
      break;
    }
    tc::tc_fence_after();
    // ---------------- TMEM -> registers: thread m holds row m ----------------
    float arow[NP];
#pragma unroll
    for (int c = 0; c < NP; ++c) arow[c] = 0.f;
    if (lane_row) {
#pragma unroll
      for (int c0 = 0; c0 < NP; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
#pragma unroll
        for (int q = 0; q < 16; ++q) arow[c0 + q] = v[q];
      }
    }
    tc::tc_fence_before();
    float bm = 0.f;  // b_u[m] sits in column f
#pragma unroll
    for (int c = 0; c < NP; ++c) {
      if (c == f) bm = arow[c];
      if (c >= f || !live) arow[c] = 0.f;
    }
    if (!live) bm = 0.f;
    const float reg = a.lambda * (float)d;
    uint32_t flags = 0;
    bool solved = false;
    float xm = 0.f;
    if (sv.solver == 1) {
      // ---------------- CG on A_u = arow + reg * I, all in registers ----------------
      float x = (live && sv.x0) ? sv.x0[u * sv.ld_x0 + m] : 0.f;
      if (!isfinite(x)) x = 0.f;
      if (live) ps[m] = x;
      __syncthreads();
      float q = reg * x;
#pragma unroll
      for (int k = 0; k < NP; k += 4) {
        const float4 p4 = *reinterpret_cast<const float4 *>(ps + k);
        q = fmaf(arow[k], p4.x, q);
        q = fmaf(arow[k + 1], p4.y, q);
        q = fmaf(arow[k + 2], p4.z, q);
        q = fmaf(arow[k + 3], p4.w, q);
      }
      if (sv.scale_x0) {
        // Scale the warm start along its own direction: alpha = x0.b / x0.A x0
        // minimises the A-norm error of alpha * x0, so no start is worse than zero.
        const float xb = cta_sum<NT>(x * bm, red, rslot);
        const float xq = cta_sum<NT>(x * q, red, rslot);
        float sc = xb / xq;
        if (!(sc > 0.f) || !isfinite(sc)) sc = 0.f;
        x *= sc;
        q *= sc;
      }
      float r = live ? bm - q : 0.f;
      float p = r;
      float rr = cta_sum<NT>(r * r, red, rslot);
      const float bb = cta_sum<NT>(bm * bm, red, rslot);
      const float target = sv.cg_tol2 * bb;
      if (tid == 0 && bb > 0.f) n_r0 += (unsigned long long)(1e6f * sqrtf(rr / bb));
      int it = 0;
      bool conv = rr <= target;
      while (!conv && it < sv.cg_max_steps) {
        if (live) ps[m] = p;
        __syncthreads();
        float w = reg * p;
#pragma unroll
        for (int k = 0; k < NP; k += 4) {
          const float4 p4 = *reinterpret_cast<const float4 *>(ps + k);
          w = fmaf(arow[k], p4.x, w);
          w = fmaf(arow[k + 1], p4.y, w);
          w = fmaf(arow[k + 2], p4.z, w);
          w = fmaf(arow[k + 3], p4.w, w);
        }
        const float pq = cta_sum<NT>(p * w, red, rslot);
        if (!(pq > 0.f)) break;  // not positive definite along p: fall back
        const float alpha = rr / pq;
        x = fmaf(alpha, p, x);
        r = fmaf(-alpha, w, r);
        const float rr2 = cta_sum<NT>(r * r, red, rslot);
        ++it;
        conv = rr2 <= target;
        p = fmaf(rr2 / rr, p, r);
        rr = rr2;
      }
      n_steps += it;
      if (conv) {
        solved = true;
        xm = x;
      } else {
        flags |= kRowCgFallback;
        ++n_fb;
      }
      __syncthreads();  // ps reads done before the next row (or S) reuses memory
    }
    if (!solved) {
      // ---------------- register-tile Cholesky + FP64-residual refinement ----------------
      if (lane_row && m < FP) {
#pragma unroll
        for (int c = 0; c < FP; ++c) {
          const float v = c < NP ? arow[c] : 0.f;
          S[m * LDS + c] = (m < f && c < f) ? v : (m == c ? 1.f : 0.f);
        }
        bv[m] = bm;
      }
      __syncthreads();
      float acc[8][8];
      if (owner) {
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            const int i = 8 * ti + r, j = 8 * tj + c;
            float v = S[i * LDS + j];
            if (i == j && i < f) v += reg;
            acc[r][c] = v;
          }
      }
      __syncthreads();
      if (owner && ti == tj) {
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          const int i = 8 * ti + r;
          dg[i] = acc[r][r];
          xv[i] = bv[i];
        }
      }
      const bool ok = tile_cholesky<FP, LDS, NT>(acc, ti, tj, owner, S, &misc[1], cta_bar());
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
      if (live) xm = xv[m];
    }
    if (live) {
      a.dst[u * a.ld_dst + m] = xm;
      if (a.dst_lp) reinterpret_cast<LP *>(a.dst_lp)[u * a.ld_dst_lp + m] = LP(xm);
    }
    if (a.row_flags && tid == 0) a.row_flags[u] = flags | sv.flags_or;
    // the next row's gather overwrites S (the stages): make sure all reads are done
    __syncthreads();
  }
  if (a.counters && tid == 0) {
    atomicAdd(&a.counters->rows, n_rows);
    if (n_ref) atomicAdd(&a.counters->refined, n_ref);
    if (n_bad) atomicAdd(&a.counters->not_spd, n_bad);
    if (n_steps) atomicAdd(&a.counters->cg_steps, n_steps);
    if (n_fb) atomicAdd(&a.counters->cg_fallback, n_fb);
    if (n_r0) atomicAdd(&a.counters->r0_micro, n_r0);
  }
  __syncthreads();
  if (misc[3]) {  // aborted: drain any MMA still in flight before freeing TMEM
    if (tid == 0) tc::mma_commit(&bars[3]);
    tc::mbar_wait(&bars[3], 0);
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(g.tmem_cols));
  }
}

bool tc_supported(int f) { return f >= 16 && f <= 128; }
int tc_padded_ld(int f) { return tc_geom(f).ldp; }

template <int FP, int NP, typename LP>
static cudaError_t launch_tc_fp(const RowsArgs &a, int lp_kind, const TcSolve &sv, int num_sms,
                                cudaStream_t st) {
  using C = TcCfg<FP>;
  const TcGeom g = tc_geom(a.f);
  if (g.np != NP) return cudaErrorInvalidValue;
  const size_t stages = (size_t)tc::kStages * g.stage_bytes;
  const size_t main_bytes = ((stages > C::kS ? stages : C::kS) + 15) / 16 * 16;
  const size_t smem = 1024 + main_bytes + 4 * FP * 4 + NP * 4 + 16 * 4 + FP * 8 + 4 * 8 + 64;
  auto kern = rows_tc_kernel<FP, NP, LP>;
  cudaError_t err =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::NT, smem);
  if (err != cudaSuccess) return err;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  per_sm = per_sm < 512 / g.tmem_cols ? per_sm : 512 / g.tmem_cols;  // TMEM columns per SM
  int64_t grid = (int64_t)num_sms * per_sm;
  if (grid > a.m) grid = a.m > 0 ? a.m : 1;
  const uint32_t idesc = tc::make_idesc(lp_kind == kLpBf16 ? 1 : 0, g.np);
  kern<<<(unsigned)grid, C::NT, smem, st>>>(a, g, idesc, sv);
  return cudaGetLastError();
}

template <int FP, int NP>
static cudaError_t launch_tc_np(const RowsArgs &a, int lp_kind, const TcSolve &sv, int num_sms,
                                cudaStream_t st) {
  return lp_kind == kLpBf16 ? launch_tc_fp<FP, NP, __nv_bfloat16>(a, lp_kind, sv, num_sms, st)
                            : launch_tc_fp<FP, NP, __half>(a, lp_kind, sv, num_sms, st);
}

cudaError_t launch_rows_tc(const RowsArgs &a, int lp_kind, int solver, int cg_max_steps,
                           float cg_tol, int cg_jacobi, int groups, const float *x0,
                           int scale_x0, const WsPlan *plan, int num_sms, cudaStream_t st) {
  if (!tc_supported(a.f)) return cudaErrorNotSupported;
  if (a.ld_src != tc_padded_ld(a.f) || !a.error) return cudaErrorInvalidValue;
  if ((reinterpret_cast<uintptr_t>(a.src) & 15) != 0) return cudaErrorInvalidValue;
  TcSolve sv{solver, cg_max_steps, cg_tol * cg_tol, x0, a.ld_dst, x0 && scale_x0 ? 1 : 0,
             cg_jacobi, groups >= 1 && groups <= 3 ? groups : 2, 0, 0u};
  RowsArgs ap = a;
  if (plan && tc_ws_takes(a.f, solver, cg_jacobi)) {
    const bool post = a.f > 112;
    if (post) {
      if (!plan->fb_rows || !plan->fb_count) return cudaErrorInvalidValue;
      cudaError_t e = cudaMemsetAsync(plan->fb_count, 0, 2 * sizeof(int), st);
      if (e != cudaSuccess) return e;
    }
    // The split rows' chunk counters start at zero: the kernel's last chunk
    // resets its row's counter, but a launch that gave up a bounded wait may
    // have left some part-way.
    if (plan->heavy_count && plan->ctas > 0) {
      cudaError_t e = cudaMemsetAsync(plan->heavy_count, 0, sizeof(unsigned) * ((size_t)kPlanSplitDiv * plan->ctas + 1), st);
      if (e != cudaSuccess) return e;
    }
    sv.withhold_first = debug_take_withhold() ? 1 : 0;
    cudaError_t e = launch_rows_tc_ws(a, lp_kind, sv, *plan, num_sms, st);
    if (e != cudaSuccess || !post || sv.prepare) return e;
    // The post-pass: the rows CG did not finish (listed by the warp-specialised
    // kernel, count in device memory), solved here by Cholesky with
    // FP64-residual refinement; their status words carry the CG fallback bit.
    ap.order = plan->fb_rows;
    ap.m_dev = plan->fb_count;
    ap.queue = reinterpret_cast<unsigned *>(plan->fb_count + 1);
    ap.m = plan->rows > 0 ? plan->rows : a.m;
    sv.solver = 0;
    sv.flags_or = kRowCgFallback;
  }
  const RowsArgs &a2 = ap;
  const int f = a2.f, np = tc_geom(f).np;
  // (FP, NP): FP >= f is the Cholesky tile extent, NP = roundup16(f + 1) the MMA N
  if (np == 32) return launch_tc_np<32, 32>(a2, lp_kind, sv, num_sms, st);
  if (np == 48) return launch_tc_np<64, 48>(a2, lp_kind, sv, num_sms, st);
  if (np == 64) return launch_tc_np<64, 64>(a2, lp_kind, sv, num_sms, st);
  if (np == 80) return launch_tc_np<104, 80>(a2, lp_kind, sv, num_sms, st);
  if (np == 96) return launch_tc_np<104, 96>(a2, lp_kind, sv, num_sms, st);
  if (np == 112 && f <= 104) return launch_tc_np<104, 112>(a2, lp_kind, sv, num_sms, st);
  if (np == 112) return launch_tc_np<128, 112>(a2, lp_kind, sv, num_sms, st);
  if (np == 128) return launch_tc_np<128, 128>(a2, lp_kind, sv, num_sms, st);
  if (np == 144) return launch_tc_np<128, 144>(a2, lp_kind, sv, num_sms, st);
  return cudaErrorNotSupported;
}

}  // namespace als
