// Internal launchers shared by the engine's translation units.
#pragma once
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
cudaError_t launch_rows_tc(const RowsArgs &a, int lp_kind, int solver, int cg_max_steps,
                           float cg_tol, const float *x0, int num_sms, cudaStream_t st);

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
cudaError_t launch_predict(int64_t nt, const int32_t *u, const int32_t *i, const float *X, int ldx,
                           const float *T, int ldt, int f, float *out, cudaStream_t st);

int device_sm_count();

}  // namespace als
