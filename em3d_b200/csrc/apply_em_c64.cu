// Instantiations of the operator passes for em, complex64.
#include "operator_passes.cuh"

namespace em3d {
template int apply<float, 3, false>(const Dims&, int, const void*, const void*, const void*, void*, void*, size_t, const int*, cudaStream_t, BatchStrides);
template int apply<float, 3, true>(const Dims&, int, const void*, const void*, const void*, void*, void*, size_t, const int*, cudaStream_t, BatchStrides);
}  // namespace em3d
