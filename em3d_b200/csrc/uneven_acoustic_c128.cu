// Instantiations of the uneven-size application for acoustic, complex128.
#include <algorithm>

#include "uneven.cuh"

namespace em3d {
template int apply_uneven<double, 1, false>(int, int, const em3d_segment*, void*, size_t, const int*, cudaStream_t);
template int apply_uneven<double, 1, true>(int, int, const em3d_segment*, void*, size_t, const int*, cudaStream_t);
}  // namespace em3d
