// ref_harness.cu -- calls the reference's own doALSWithCSR (als/src/cuda/als.cu:1001-1115)
// the way its JNI shim does (als/src/CuMFJNIInterface.cpp:93-109): CSR uploaded to
// mallocBest memory that the callee frees, theta/X in pinned host memory.
//
// TEST INFRASTRUCTURE ONLY (part of the reference checker build).
#include <cuda_runtime.h>
#include <cstring>
#include <cstdio>

extern "C" void doALSWithCSR(cudaStream_t cuda_stream, int *csrRowIndex, int *csrColIndex,
                             float *csrVal, float *thetaTHost, float *XTHost, const int m,
                             const int n, const int f, const long nnz, const float lambda,
                             const int X_BATCH);
// utilities.h gives only get_gpu C linkage; mallocBest keeps C++ linkage.
cudaError_t mallocBest(void **devPtr, size_t size);

// Returns 0 on success. x_batch must keep batch * f * f below 2^31 (the
// reference indexes its f x f systems with int).
extern "C" int ref_half_step(int m, int n, int f, long nnz, const int *row_ptr, const int *col,
                             const float *val, const float *theta, float lambda, int x_batch,
                             float *x_out, float *elapsed_ms) {
  int *d_row = 0, *d_col = 0;
  float *d_val = 0, *th = 0, *xt = 0;
  cudaStream_t st;
  if (cudaStreamCreate(&st) != cudaSuccess) return 1;
  if (cudaMallocHost((void **)&th, sizeof(float) * (size_t)n * f) != cudaSuccess) return 2;
  if (cudaMallocHost((void **)&xt, sizeof(float) * (size_t)m * f) != cudaSuccess) return 2;
  std::memcpy(th, theta, sizeof(float) * (size_t)n * f);
  if (mallocBest((void **)&d_row, sizeof(int) * (m + 1)) != cudaSuccess) return 3;
  if (mallocBest((void **)&d_col, sizeof(int) * (nnz > 0 ? nnz : 1)) != cudaSuccess) return 3;
  if (mallocBest((void **)&d_val, sizeof(float) * (nnz > 0 ? nnz : 1)) != cudaSuccess) return 3;
  cudaMemcpy(d_row, row_ptr, sizeof(int) * (m + 1), cudaMemcpyHostToDevice);
  if (nnz > 0) {
    cudaMemcpy(d_col, col, sizeof(int) * nnz, cudaMemcpyHostToDevice);
    cudaMemcpy(d_val, val, sizeof(float) * nnz, cudaMemcpyHostToDevice);
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  doALSWithCSR(st, d_row, d_col, d_val, th, xt, m, n, f, nnz, lambda, x_batch);
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  if (elapsed_ms) cudaEventElapsedTime(elapsed_ms, e0, e1);
  std::memcpy(x_out, xt, sizeof(float) * (size_t)m * f);
  cudaFreeHost(th);
  cudaFreeHost(xt);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}
