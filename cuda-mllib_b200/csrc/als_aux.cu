// Auxiliary kernels: degree-binned row ordering, pointer widening, factor
// down-conversion, the fused RMSE / predict gather, and top-k recommendation.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "als_internal.h"

namespace als {

int device_sm_count() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  return sms;
}

__device__ __forceinline__ int degree_bin(int64_t d) {
  const int b = d <= 0 ? 0 : 64 - __clzll((unsigned long long)d);  // 1 + floor(log2 d)
  return b < kOrderBins ? b : kOrderBins - 1;
}

// Rows [row_begin, row_begin + m) of the CSR; order[] receives absolute row ids.
__global__ void order_hist_kernel(const int64_t *row_ptr, int64_t m, unsigned *hist) {
  __shared__ unsigned h[kOrderBins];
  for (int i = threadIdx.x; i < kOrderBins; i += blockDim.x) h[i] = 0;
  __syncthreads();
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < m;
       u += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&h[degree_bin(row_ptr[u + 1] - row_ptr[u])], 1u);
  __syncthreads();
  for (int i = threadIdx.x; i < kOrderBins; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], h[i]);
}

// Heaviest bin first: offsets are an exclusive scan over bins in descending order.
__global__ void order_scan_kernel(const unsigned *hist, unsigned *offs) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    unsigned acc = 0;
    for (int b = kOrderBins - 1; b >= 0; --b) {
      offs[b] = acc;
      acc += hist[b];
    }
  }
}

__global__ void order_scatter_kernel(const int64_t *row_ptr, int64_t m, unsigned *offs,
                                     int32_t *order, int64_t row_begin) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < m;
       u += (int64_t)gridDim.x * blockDim.x) {
    const unsigned p = atomicAdd(&offs[degree_bin(row_ptr[u + 1] - row_ptr[u])], 1u);
    order[p] = (int32_t)(u + row_begin);
  }
}

cudaError_t launch_degree_order(const int64_t *row_ptr, int64_t m, int32_t *order,
                                unsigned *work, cudaStream_t st, int64_t row_begin) {
  row_ptr += row_begin;
  if (m <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(work, 0, sizeof(unsigned) * 2 * kOrderBins, st);
  if (e != cudaSuccess) return e;
  const int sms = device_sm_count();
  const unsigned grid = (unsigned)std::min<int64_t>((m + 255) / 256, (int64_t)sms * 8);
  order_hist_kernel<<<grid, 256, 0, st>>>(row_ptr, m, work);
  order_scan_kernel<<<1, 32, 0, st>>>(work, work + kOrderBins);
  order_scatter_kernel<<<grid, 256, 0, st>>>(row_ptr, m, work + kOrderBins, order, row_begin);
  return cudaGetLastError();
}

__global__ void widen_kernel(const int32_t *in, int64_t count, int64_t *out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int64_t)in[i];
}

cudaError_t launch_widen_ptr(const int32_t *in, int64_t count, int64_t *out, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)std::min<int64_t>((count + 255) / 256, 4096);
  widen_kernel<<<grid, 256, 0, st>>>(in, count, out);
  return cudaGetLastError();
}

template <typename T>
__global__ void convert_kernel(const float *src, int64_t rows, int f, int ld_src, T *dst,
                               int ld_dst) {
  const int64_t total = rows * ld_dst;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = q / ld_dst;
    const int c = (int)(q - r * ld_dst);
    dst[q] = T(c < f ? src[r * ld_src + c] : 0.f);
  }
}

cudaError_t launch_convert_lp(const float *src, int64_t rows, int f, int ld_src, void *dst,
                              int ld_dst, int kind, cudaStream_t st) {
  if (rows <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)std::min<int64_t>((rows * ld_dst + 255) / 256, 8192);
  if (kind == kLpBf16)
    convert_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(src, rows, f, ld_src,
                                                        (__nv_bfloat16 *)dst, ld_dst);
  else if (kind == kLpFp16)
    convert_kernel<__half><<<grid, 256, 0, st>>>(src, rows, f, ld_src, (__half *)dst, ld_dst);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// RMSE / predict: one warp per test entry, lanes stride the rank; the squared
// errors are summed in FP64 per warp, per block, then across blocks by a
// single-block pass (fixed order: the result is bit-reproducible).
// ---------------------------------------------------------------------------
constexpr int kRmseBlocks = 1184;  // 8 x 148 SMs
constexpr int kRmseThreads = 256;

size_t rmse_work_bytes() { return sizeof(double) * kRmseBlocks; }

__device__ __forceinline__ float dot_warp(const float *x, const float *t, int f) {
  float s = 0.f;
  for (int k = threadIdx.x & 31; k < f; k += 32) s = fmaf(x[k], t[k], s);
  return warp_sum(s);
}

__global__ void __launch_bounds__(kRmseThreads)
rmse_partial_kernel(int64_t nt, const int32_t *u, const int32_t *i, const float *r,
                    const float *X, int ldx, const float *T, int ldt, int f, double *part) {
  const int warps = kRmseThreads / 32, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double acc = 0.0;
  for (int64_t q = blockIdx.x * (int64_t)warps + w; q < nt; q += (int64_t)gridDim.x * warps) {
    const float p = dot_warp(X + (int64_t)u[q] * ldx, T + (int64_t)i[q] * ldt, f);
    const double e = (double)r[q] - (double)p;
    acc += e * e;
  }
  __shared__ double red[kRmseThreads / 32];
  if (lane == 0) red[w] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < warps; ++k) s += red[k];
    part[blockIdx.x] = s;
  }
}

// out = sqrt(sum / nt), or the sum itself with `root` unset (a shard's share)
__global__ void rmse_final_kernel(const double *part, int nblocks, int64_t nt, int root,
                                  double *out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int k = threadIdx.x; k < nblocks; k += blockDim.x) s += part[k];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = !root ? red[0] : nt > 0 ? sqrt(red[0] / (double)nt) : 0.0;
}

cudaError_t launch_rmse(int64_t nt, const int32_t *u, const int32_t *i, const float *r,
                        const float *X, int ldx, const float *T, int ldt, int f, double *out_dev,
                        void *work, cudaStream_t st) {
  double *part = reinterpret_cast<double *>(work);
  rmse_partial_kernel<<<kRmseBlocks, kRmseThreads, 0, st>>>(nt, u, i, r, X, ldx, T, ldt, f, part);
  rmse_final_kernel<<<1, 256, 0, st>>>(part, kRmseBlocks, nt, 1, out_dev);
  return cudaGetLastError();
}

cudaError_t launch_rmse_sum(int64_t nt, const int32_t *u, const int32_t *i, const float *r,
                            const float *X, int ldx, const float *T, int ldt, int f,
                            double *sum_dev, void *work, cudaStream_t st) {
  double *part = reinterpret_cast<double *>(work);
  rmse_partial_kernel<<<kRmseBlocks, kRmseThreads, 0, st>>>(nt, u, i, r, X, ldx, T, ldt, f, part);
  rmse_final_kernel<<<1, 256, 0, st>>>(part, kRmseBlocks, nt, 0, sum_dev);
  return cudaGetLastError();
}

__global__ void predict_kernel(int64_t nt, const int32_t *u, const int32_t *i, const float *X,
                               int ldx, const float *T, int ldt, int f, float *out) {
  const int warps = blockDim.x / 32, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t q = blockIdx.x * (int64_t)warps + w; q < nt; q += (int64_t)gridDim.x * warps) {
    const float p = dot_warp(X + (int64_t)u[q] * ldx, T + (int64_t)i[q] * ldt, f);
    if (lane == 0) out[q] = p;
  }
}

cudaError_t launch_predict(int64_t nt, const int32_t *u, const int32_t *i, const float *X, int ldx,
                           const float *T, int ldt, int f, float *out, cudaStream_t st) {
  if (nt <= 0) return cudaSuccess;
  predict_kernel<<<kRmseBlocks, kRmseThreads, 0, st>>>(nt, u, i, X, ldx, T, ldt, f, out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// top-k recommendation: for each query user, the k items of largest x_u . theta_i,
// leaving out the items the user has already rated (its row of the training
// CSR, columns ascending). One block per query: a tile of 256 item scores at a
// time joins the running top list in shared memory through a bitonic sort of
// 512 (score descending, item ascending) pairs; tiles with no score above the
// current k-th are skipped after one block vote.
// ---------------------------------------------------------------------------
constexpr int kTopThreads = 256;

__device__ __forceinline__ bool top_before(float sa, int ia, float sb, int ib) {
  return sa > sb || (sa == sb && ia < ib);
}

__device__ __forceinline__ bool seen_by(const int32_t *cols, int64_t s, int64_t e, int item) {
  while (s < e) {  // binary search in the ascending columns [s, e)
    const int64_t mid = (s + e) >> 1;
    const int c = cols[mid];
    if (c == item) return true;
    if (c < item) s = mid + 1;
    else e = mid;
  }
  return false;
}

__global__ void __launch_bounds__(kTopThreads) topk_kernel(
    int64_t nq, const int32_t *users, const float *X, int ldx, const float *T, int ldt, int64_t n,
    int f, int k, const int64_t *seen_ptr, const int32_t *seen_col, int32_t *out_items,
    float *out_scores) {
  __shared__ float xs[128];
  __shared__ float sc[2 * kTopThreads];
  __shared__ int id[2 * kTopThreads];
  const int t = threadIdx.x;
  for (int64_t q = blockIdx.x; q < nq; q += gridDim.x) {
    const int64_t u = users[q];
    if (t < f) xs[t] = X[u * ldx + t];
    sc[t] = sc[t + kTopThreads] = -INFINITY;
    id[t] = id[t + kTopThreads] = INT_MAX;
    const int64_t s0 = seen_ptr ? seen_ptr[u] : 0, s1 = seen_ptr ? seen_ptr[u + 1] : 0;
    __syncthreads();
    float kth = -INFINITY;
    int kid = INT_MAX;
    for (int64_t base = 0; base < n; base += kTopThreads) {
      const int64_t i = base + t;
      float s = -INFINITY;
      int ii = INT_MAX;
      if (i < n && !seen_by(seen_col, s0, s1, (int)i)) {
        const float *th = T + i * ldt;
        float a0 = 0.f, a1 = 0.f;
        int c = 0;
        for (; c + 1 < f; c += 2) {
          a0 = fmaf(xs[c], th[c], a0);
          a1 = fmaf(xs[c + 1], th[c + 1], a1);
        }
        if (c < f) a0 = fmaf(xs[c], th[c], a0);
        s = a0 + a1;
        ii = (int)i;
      }
      if (!__syncthreads_or(ii != INT_MAX && top_before(s, ii, kth, kid))) continue;
      sc[kTopThreads + t] = s;
      id[kTopThreads + t] = ii;
      // bitonic sort of the 512 pairs, best first
      for (int size = 2; size <= 2 * kTopThreads; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
          __syncthreads();
          const int a = 2 * t - (t & (stride - 1)), b = a + stride;
          const bool best_first = (a & size) == 0;
          const float sa = sc[a], sb = sc[b];
          const int ia = id[a], ib = id[b];
          if (top_before(sb, ib, sa, ia) == best_first) {
            sc[a] = sb; sc[b] = sa;
            id[a] = ib; id[b] = ia;
          }
        }
      }
      __syncthreads();
      kth = sc[k - 1];
      kid = id[k - 1];
      __syncthreads();
    }
    for (int j = t; j < k; j += kTopThreads) {
      out_items[q * k + j] = id[j] == INT_MAX ? -1 : id[j];
      out_scores[q * k + j] = id[j] == INT_MAX ? -INFINITY : sc[j];
    }
    __syncthreads();
  }
}

cudaError_t launch_topk(int64_t nq, const int32_t *users, const float *X, int ldx, const float *T,
                        int ldt, int64_t n, int f, int k, const int64_t *seen_ptr,
                        const int32_t *seen_col, int32_t *out_items, float *out_scores,
                        cudaStream_t st) {
  if (nq <= 0) return cudaSuccess;
  if (f < 1 || f > 128 || k < 1 || k > kTopThreads || n > INT32_MAX - 1) return cudaErrorInvalidValue;
  const unsigned grid = (unsigned)std::min<int64_t>(nq, (int64_t)device_sm_count() * 8);
  topk_kernel<<<grid, kTopThreads, 0, st>>>(nq, users, X, ldx, T, ldt, n, f, k, seen_ptr, seen_col,
                                            out_items, out_scores);
  return cudaGetLastError();
}

}  // namespace als
