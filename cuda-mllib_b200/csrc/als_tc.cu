// Tensor-core (tcgen05) form of the half-step.
#include "als_internal.h"

namespace als {

bool tc_supported(int f) { return false; }
int tc_padded_ld(int f) { return ((f + 1 + 7) / 8) * 8; }
cudaError_t launch_rows_tc(const RowsArgs &, int, int, int, float, const float *, int, cudaStream_t) {
  return cudaErrorNotSupported;
}

}  // namespace als
