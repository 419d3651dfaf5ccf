// A C++ caller of libGPUALS.so written against the reference's own
// declarations, not this library's header: utilities.h:36-41 gives C linkage
// to get_gpu only (mallocBest and freeBest keep C++ linkage), and
// als/src/cuda/als.h:96-103 declares doALSWithCSR extern "C". Linking this
// program proves that a caller built for the reference resolves every symbol
// against this library. Running it needs no GPU: it calls only the drop-in's
// error check, which must throw thrust::system_error (the type the
// reference's JNI catch block expects) for a set kernel error word.
#include <cuda_runtime_api.h>
#include <thrust/system_error.h>

#include <cstdio>
#include <cstring>

extern "C" int get_gpu();
cudaError_t mallocBest(void **devPtr, size_t size);
cudaError_t freeBest(void *devPtr);

extern "C" {
void doALSWithCSR(cudaStream_t cuda_stream, int *csrRowIndex, int *csrColIndex, float *csrVal,
                  float *thetaTHost, float *XTHost, const int m, const int n, const int f,
                  const long nnz, const float lambda, const int X_BATCH);
}

namespace als {
void dropin_raise_on_kernel_error(int error_word);
}

int main(int argc, char **) {
  // The addresses keep every call site: the linker must resolve each symbol.
  void *volatile keep[] = {(void *)&get_gpu, (void *)&mallocBest, (void *)&freeBest,
                           (void *)&doALSWithCSR};
  if (argc > 99) std::printf("%p\n", keep[0]);
  int ok = 0;
  try {
    als::dropin_raise_on_kernel_error(0);
    ok |= 1;
  } catch (...) {
  }
  try {
    als::dropin_raise_on_kernel_error(1);
  } catch (thrust::system_error &e) {
    if (std::strstr(e.what(), "bounded wait")) ok |= 2;
  }
  try {
    als::dropin_raise_on_kernel_error(2);
  } catch (thrust::system_error &e) {
    if (std::strstr(e.what(), "malformed")) ok |= 4;
  }
  std::printf("checks %d\n", ok);
  return ok == 7 ? 0 : 1;
}
