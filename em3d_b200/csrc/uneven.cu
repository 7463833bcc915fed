// C entry points of the applications over problems of uneven grid sizes;
// the passes themselves are instantiated in uneven_{em,acoustic}_c{64,128}.cu.
#include <algorithm>

#include "uneven.cuh"

namespace em3d {

#define EM3D_UNEVEN_EXTERN(R, C, ADJ) \
  extern template int apply_uneven<R, C, ADJ>(int, int, const em3d_segment*, void*, size_t, const int*, cudaStream_t);
EM3D_UNEVEN_EXTERN(float, 3, false)
EM3D_UNEVEN_EXTERN(float, 3, true)
EM3D_UNEVEN_EXTERN(double, 3, false)
EM3D_UNEVEN_EXTERN(double, 3, true)
EM3D_UNEVEN_EXTERN(float, 1, false)
EM3D_UNEVEN_EXTERN(float, 1, true)
EM3D_UNEVEN_EXTERN(double, 1, false)
EM3D_UNEVEN_EXTERN(double, 1, true)
#undef EM3D_UNEVEN_EXTERN

template <int C, bool ADJ>
static int uneven_dispatch(int dtype, int nseg, const em3d_segment* segs, void* ws, size_t wsb, const int* skip,
                           void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == EM3D_C64) return apply_uneven<float, C, ADJ>(dtype, nseg, segs, ws, wsb, skip, st);
  if (dtype == EM3D_C128) return apply_uneven<double, C, ADJ>(dtype, nseg, segs, ws, wsb, skip, st);
  em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128");
  return EM3D_ERR_INVALID;
}

}  // namespace em3d

using namespace em3d;

extern "C" {

size_t em3d_segment_size(void) { return sizeof(em3d_segment); }

int em3d_uneven_supported(const em3d_grid* g, int kind, int dtype) {
  Dims d;
  if (check_grid(g, &d)) return 0;
  if (kind == EM3D_EM) {
    if (dtype == EM3D_C64) return uneven_grid_ok<float, 3>(d) ? 1 : 0;
    if (dtype == EM3D_C128) return uneven_grid_ok<double, 3>(d) ? 1 : 0;
  } else if (kind == EM3D_ACOUSTIC) {
    if (dtype == EM3D_C64) return uneven_grid_ok<float, 1>(d) ? 1 : 0;
    if (dtype == EM3D_C128) return uneven_grid_ok<double, 1>(d) ? 1 : 0;
  }
  return 0;
}

size_t em3d_uneven_workspace_bytes(int kind, int dtype, int nseg, const em3d_segment* segs) {
  if (nseg < 1 || nseg > kMaxSegments || !segs) return 0;
  if (kind == EM3D_EM) {
    if (dtype == EM3D_C64) return uneven_ws_bytes<float, 3>(nseg, segs, dtype);
    if (dtype == EM3D_C128) return uneven_ws_bytes<double, 3>(nseg, segs, dtype);
  } else if (kind == EM3D_ACOUSTIC) {
    if (dtype == EM3D_C64) return uneven_ws_bytes<float, 1>(nseg, segs, dtype);
    if (dtype == EM3D_C128) return uneven_ws_bytes<double, 1>(nseg, segs, dtype);
  }
  return 0;
}

int em3d_em_matvec_uneven(int dtype, int nseg, const em3d_segment* segs, void* ws, size_t wsb, const int* skip,
                          void* stream) {
  return uneven_dispatch<3, false>(dtype, nseg, segs, ws, wsb, skip, stream);
}
int em3d_em_rmatvec_uneven(int dtype, int nseg, const em3d_segment* segs, void* ws, size_t wsb, const int* skip,
                           void* stream) {
  return uneven_dispatch<3, true>(dtype, nseg, segs, ws, wsb, skip, stream);
}
int em3d_acoustic_matvec_uneven(int dtype, int nseg, const em3d_segment* segs, void* ws, size_t wsb,
                                const int* skip, void* stream) {
  return uneven_dispatch<1, false>(dtype, nseg, segs, ws, wsb, skip, stream);
}
int em3d_acoustic_rmatvec_uneven(int dtype, int nseg, const em3d_segment* segs, void* ws, size_t wsb,
                                 const int* skip, void* stream) {
  return uneven_dispatch<1, true>(dtype, nseg, segs, ws, wsb, skip, stream);
}

}  // extern "C"
