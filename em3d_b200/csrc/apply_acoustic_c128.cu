// Instantiations of the operator passes for acoustic, complex128.
#include "operator_passes.cuh"

namespace em3d {
template int apply<double, 1, false>(const Dims&, int, const void*, const void*, const void*, void*, void*, size_t, const int*, cudaStream_t, BatchStrides);
template int apply<double, 1, true>(const Dims&, int, const void*, const void*, const void*, void*, void*, size_t, const int*, cudaStream_t, BatchStrides);
}  // namespace em3d
