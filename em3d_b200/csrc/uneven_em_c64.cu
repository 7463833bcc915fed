// Instantiations of the uneven-size application for em, complex64.
#include <algorithm>

#include "uneven.cuh"

namespace em3d {
template int apply_uneven<float, 3, false>(int, int, const em3d_segment*, void*, size_t, const int*, cudaStream_t);
template int apply_uneven<float, 3, true>(int, int, const em3d_segment*, void*, size_t, const int*, cudaStream_t);
}  // namespace em3d
