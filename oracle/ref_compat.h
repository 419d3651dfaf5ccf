/*
 * ref_compat.h -- force-included when compiling the reference's als.cu.
 *
 * TEST INFRASTRUCTURE ONLY (builds the reference as a checker).
 *
 * Two CUDA 12 changes stop the reference from compiling as written:
 *  1. cusparseScsrmm2, which als/src/cuda/als.cu:1047-1049 calls, was removed
 *     from cuSPARSE. The declaration below keeps its legacy signature; the
 *     definition in ref_compat.cu computes the same product
 *     C = alpha * A * op(B) + beta * C with our own CSR kernel.
 *  2. cudaPointerAttributes::memoryType became ::type (see the macro below).
 * Everything else of the reference compiles unchanged for sm_100a.
 */
#pragma once
#include <cuda_runtime.h>
#include <cusparse.h>

/* CUDA 12 renamed cudaPointerAttributes::memoryType to ::type; utilities.cu:89
 * (freeBest) still reads the old member. The runtime headers are already
 * included above, so this only rewrites the reference's own uses. */
#define memoryType type

cusparseStatus_t cusparseScsrmm2(cusparseHandle_t handle, cusparseOperation_t transA,
                                 cusparseOperation_t transB, int m, int n, int k, int nnz,
                                 const float *alpha, const cusparseMatDescr_t descrA,
                                 const float *csrValA, const int *csrRowPtrA,
                                 const int *csrColIndA, const float *B, int ldb,
                                 const float *beta, float *C, int ldc);
