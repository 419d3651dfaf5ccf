// Device-side CSR -> CSC (the CSR of the transpose) for callers that hold only
// one orientation of the rating matrix on the GPU. Rows stay ascending within
// each column (a stable radix sort by column), so the result equals the host
// transpose bit for bit and the hermitian of a column sums in the same order
// as with a host-built CSC.
#include <thrust/binary_search.h>
#include <thrust/device_ptr.h>
#include <thrust/device_vector.h>
#include <thrust/execution_policy.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/zip_iterator.h>
#include <thrust/sort.h>

#include "als_internal.h"

namespace als {

// row index of every stored rating: ptr[u] <= q < ptr[u+1] -> rows[q] = u
__global__ void expand_rows_kernel(int64_t m, const int64_t *ptr, int32_t *rows) {
  for (int64_t u = blockIdx.x; u < m; u += gridDim.x)
    for (int64_t q = ptr[u] + threadIdx.x; q < ptr[u + 1]; q += blockDim.x) rows[q] = (int32_t)u;
}

cudaError_t csr_to_csc(int64_t m, int64_t n, int64_t nnz, const int64_t *ptr, const int32_t *col,
                       const float *val, int64_t *cptr, int32_t *crow, float *cval,
                       cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(cptr, 0, sizeof(int64_t), st);
  if (e != cudaSuccess || n == 0) return e;
  if (nnz == 0) return cudaMemsetAsync(cptr, 0, sizeof(int64_t) * (size_t)(n + 1), st);
  try {
    thrust::device_vector<int32_t> keys(nnz);
    auto pol = thrust::cuda::par.on(st);
    if ((e = cudaMemcpyAsync(thrust::raw_pointer_cast(keys.data()), col, sizeof(int32_t) * nnz,
                             cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
      return e;
    if ((e = cudaMemcpyAsync(cval, val, sizeof(float) * nnz, cudaMemcpyDeviceToDevice, st)) !=
        cudaSuccess)
      return e;
    if (m > 0) {
      const unsigned grid = (unsigned)std::min<int64_t>(m, 65535);
      expand_rows_kernel<<<grid, 128, 0, st>>>(m, ptr, crow);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    thrust::device_ptr<int32_t> r(crow);
    thrust::device_ptr<float> v(cval);
    thrust::stable_sort_by_key(pol, keys.begin(), keys.end(),
                               thrust::make_zip_iterator(thrust::make_tuple(r, v)));
    // cptr[c + 1] = number of ratings with column <= c
    thrust::upper_bound(pol, keys.begin(), keys.end(), thrust::counting_iterator<int32_t>(0),
                        thrust::counting_iterator<int32_t>((int32_t)n),
                        thrust::device_ptr<int64_t>(cptr + 1));
    return cudaStreamSynchronize(st);  // keys is freed on return
  } catch (const std::exception &) {
    cudaGetLastError();
    return cudaErrorMemoryAllocation;
  }
}

}  // namespace als
