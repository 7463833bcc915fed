// EM matvec for callers that cannot allocate device memory.
//
// em3d_em_matvec needs a workspace of em3d_apply_workspace_bytes() bytes that
// the caller allocates.  Some callers cannot do that: code that runs where
// cudaMalloc is unavailable or forbidden (a host framework that owns all
// device allocations and hands out only input/output buffers, a plugin
// sandbox, a real-time loop that must never enter the allocator).  For them
// this file provides em3d_em_matvec_static_scratch, which runs the same five
// passes with the workspace placed in a fixed device array compiled into the
// library.
//
// The array (kStaticScratchBytes = 64 MiB) is a file-scope __device__
// variable: every GPU on which the library is used holds it until the
// process exits.  Its device address is looked up once per device with
// cudaGetSymbolAddress (host code may not take the address of a __device__
// variable directly: the host-side symbol is only a stand-in).  That look-up
// happens during the first call on each device, so make that first call
// before capturing a stream into a CUDA graph.  The passes write every
// transform element before reading it; the one part that must start at zero,
// the status words at the end of this call's workspace (the count of bounded
// waits that gave up), is cleared by each call on its stream before the
// passes.  This entry point does not report that count to its caller (the
// regular entry points leave it in the caller's workspace).  All calls share the
// one array: calls that overlap on the GPU (on different streams, or from
// several host threads) race and must be serialised by the caller.
#include <mutex>

#include "common.cuh"

namespace {

constexpr size_t kStaticScratchBytes = (size_t)64 << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of g_static_scratch on the current device (looked up once).
int scratch_address(void** out) {
  int dev = -1;
  EM3D_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    em3d_set_last_error("device ordinal out of range for the static scratch table");
    return EM3D_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    EM3D_CUDA_TRY(cudaGetSymbolAddress(&p, g_static_scratch));
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return EM3D_OK;
}

}  // namespace

extern "C" {

size_t em3d_static_scratch_bytes(void) { return kStaticScratchBytes; }

int em3d_em_matvec_static_scratch(const em3d_grid* g, int dtype, const void* spectrum, const void* chi,
                                  const void* u, void* out, const int* skip, void* stream) {
  em3d_set_last_error("");
  const size_t need = em3d_apply_workspace_bytes(g, EM3D_EM, dtype, 1);
  if (need == 0) {
    if (em3d_last_error()[0] == '\0') em3d_set_last_error("invalid grid or dtype");
    return EM3D_ERR_INVALID;
  }
  if (need > kStaticScratchBytes) {
    em3d_set_last_error("grid too large for em3d_em_matvec_static_scratch: the workspace would exceed the "
                        "64 MiB static scratch; use em3d_em_matvec with a caller-allocated workspace");
    return EM3D_ERR_INVALID;
  }
  void* ws = nullptr;
  const int rc = scratch_address(&ws);
  if (rc != EM3D_OK) return rc;
  // The status words are the workspace's last 256 bytes (need - 256 into the
  // array), a place that a call on a larger grid used for transform data:
  // clear them on the caller's stream so this call starts from a zero count.
  EM3D_CUDA_TRY(cudaMemsetAsync((char*)ws + (need - 256), 0, 256, (cudaStream_t)stream));
  return em3d_em_matvec(g, dtype, 1, spectrum, chi, u, out, ws, need, skip, stream);
}

}  // extern "C"
