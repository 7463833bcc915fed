// Small transfers between device memory and pinned host memory done by a
// kernel on the caller's stream instead of the copy engines.
//
// A solver reads a few bytes back several times per solve (its stop flag,
// the operator's status word, its states and residual histories) and writes
// its states at the start of each cycle.  As cudaMemcpyAsync calls those
// queue on the copy engines behind whatever large transfer another stream
// has issued (a 100 MB right-hand side for the next solve, the previous
// solution going out), so one 4-byte read can wait milliseconds.  Pinned
// host memory is addressable from kernels (unified addressing), so a kernel
// on the solving stream moves such small amounts over the host link directly
// and the large transfers on other streams no longer hold up the solve.
#include <algorithm>

#include "common.cuh"

namespace em3d {

constexpr int kIoThreads = 256;

// W-byte words (16 when both addresses are 16-byte aligned: fewer, larger
// requests over the host link), then the ragged tail byte by byte.  Loads
// bypass the caches (ld.global.cv): a pinned staging buffer is rewritten by
// the host between uploads.
template <typename W>
__global__ void __launch_bounds__(kIoThreads) k_copy_small(unsigned char* dst, const unsigned char* src, size_t bytes) {
  const size_t words = bytes / sizeof(W);
  const size_t gs = (size_t)gridDim.x * blockDim.x;
  W* dw = reinterpret_cast<W*>(dst);
  const W* sw = reinterpret_cast<const W*>(src);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < words; i += gs) dw[i] = __ldcv(sw + i);
  const size_t tail = words * sizeof(W);
  if (blockIdx.x == 0 && threadIdx.x < bytes - tail) dst[tail + threadIdx.x] = __ldcv(src + tail + threadIdx.x);
}

// The address a kernel uses for p: device memory as is, pinned host memory by
// its device mapping; 0 for memory a kernel cannot reach (pageable host memory).
static const void* device_address(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return p;
  if (a.type == cudaMemoryTypeHost) return a.devicePointer;
  return nullptr;
}

}  // namespace em3d

using namespace em3d;

size_t em3d_copy_small_max_bytes(void) { return (size_t)16 << 20; }

int em3d_copy_small(void* dst, const void* src, size_t bytes, void* stream) {
  if (bytes == 0) return EM3D_OK;
  if (!dst || !src) { em3d_set_last_error("em3d_copy_small: null pointer"); return EM3D_ERR_INVALID; }
  if (bytes > em3d_copy_small_max_bytes()) {
    em3d_set_last_error("em3d_copy_small: more than em3d_copy_small_max_bytes() bytes");
    return EM3D_ERR_INVALID;
  }
  if (((uintptr_t)dst | (uintptr_t)src) & 3) {
    em3d_set_last_error("em3d_copy_small: dst and src must be 4-byte aligned");
    return EM3D_ERR_INVALID;
  }
  void* d = const_cast<void*>(device_address(dst));
  const void* s = device_address(src);
  if (!d || !s) {
    em3d_set_last_error("em3d_copy_small: dst and src must be device memory or pinned host memory");
    return EM3D_ERR_INVALID;
  }
  const bool wide = (((uintptr_t)d | (uintptr_t)s) & 15) == 0;
  const size_t words = bytes / (wide ? 16 : 4);
  const int blocks = (int)std::min<size_t>(148, std::max<size_t>(1, (words + kIoThreads - 1) / kIoThreads));
  unsigned char* dd = static_cast<unsigned char*>(d);
  const unsigned char* ss = static_cast<const unsigned char*>(s);
  if (wide) k_copy_small<uint4><<<blocks, kIoThreads, 0, (cudaStream_t)stream>>>(dd, ss, bytes);
  else k_copy_small<uint32_t><<<blocks, kIoThreads, 0, (cudaStream_t)stream>>>(dd, ss, bytes);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}
