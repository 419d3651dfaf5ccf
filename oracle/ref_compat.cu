// ref_compat.cu -- stand-in for the removed legacy cusparseScsrmm2.
//
// TEST INFRASTRUCTURE ONLY (part of the reference checker build).
//
// Semantics (legacy cuSPARSE documentation): A is m x k in 0-based CSR,
// op(B) is k x n, C is m x n column-major with leading dimension ldc.
// With transB == TRANSPOSE, B is stored column-major n x k (ldb >= n), i.e.
// op(B)(j, c) = B[c + j * ldb]. The reference calls it with transA = N,
// transB = T, B = theta stored row-major n_items x f (als.cu:1047-1049), so
// C(u, c) = sum_q val[q] * theta[col[q]][c]: the right-hand sides b_u.
// One thread per (row, column) output; products summed in CSR order.
#include "ref_compat.h"

static __global__ void csrmm_kernel(int m, int n, float alpha, const float *val, const int *ptr,
                                    const int *col, const float *B, int ldb, bool transB,
                                    float beta, float *C, int ldc) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)m * n) return;
  const int row = (int)(t % m), c = (int)(t / m);
  float acc = 0.f;
  for (int q = ptr[row]; q < ptr[row + 1]; ++q) {
    const float b = transB ? B[c + (long long)col[q] * ldb] : B[col[q] + (long long)c * ldb];
    acc = fmaf(val[q], b, acc);
  }
  float *out = C + row + (long long)c * ldc;
  *out = (beta == 0.f) ? alpha * acc : alpha * acc + beta * *out;
}

cusparseStatus_t cusparseScsrmm2(cusparseHandle_t handle, cusparseOperation_t transA,
                                 cusparseOperation_t transB, int m, int n, int k, int nnz,
                                 const float *alpha, const cusparseMatDescr_t descrA,
                                 const float *csrValA, const int *csrRowPtrA,
                                 const int *csrColIndA, const float *B, int ldb,
                                 const float *beta, float *C, int ldc) {
  (void)k; (void)nnz; (void)descrA;
  if (transA != CUSPARSE_OPERATION_NON_TRANSPOSE) return CUSPARSE_STATUS_NOT_SUPPORTED;
  cudaStream_t st = 0;
  if (cusparseGetStream(handle, &st) != CUSPARSE_STATUS_SUCCESS) return CUSPARSE_STATUS_INVALID_VALUE;
  const long long total = (long long)m * n;
  if (total == 0) return CUSPARSE_STATUS_SUCCESS;
  csrmm_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
      m, n, *alpha, csrValA, csrRowPtrA, csrColIndA, B, ldb,
      transB == CUSPARSE_OPERATION_TRANSPOSE, *beta, C, ldc);
  return cudaGetLastError() == cudaSuccess ? CUSPARSE_STATUS_SUCCESS : CUSPARSE_STATUS_EXECUTION_FAILED;
}
