// Shared device helpers for the em3d B200 library: complex arithmetic on
// float2 / double2, launch checks, the skip flag used by device-resident
// solver loops.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/em3d_b200.h"

namespace em3d {

template <typename R> struct Cx;
template <> struct Cx<float> { using T = float2; };
template <> struct Cx<double> { using T = double2; };
template <typename R> using cx = typename Cx<R>::T;

template <typename R> __host__ __device__ __forceinline__ cx<R> mk(R re, R im) {
  cx<R> v; v.x = re; v.y = im; return v;
}
template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// conj(a) * b
template <typename C> __host__ __device__ __forceinline__ C cmulcj(C a, C b) {
  C r; r.x = a.x * b.x + a.y * b.y; r.y = a.x * b.y - a.y * b.x; return r;
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }

// Complex add / subtract for the FFT butterflies: one packed FP32x2
// instruction (sm_100's FADD2: two lanes per issue slot, each rounded like a
// scalar add) for complex64, the scalar pair for complex128.  Used where both
// operands are plain complex values; sums involving a value multiplied by
// +-i mix the lanes and stay scalar.
template <typename C> __device__ __forceinline__ C vadd(C a, C b) { return cadd(a, b); }
template <typename C> __device__ __forceinline__ C vsub(C a, C b) { return csub(a, b); }
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
template <> __device__ __forceinline__ float2 vadd<float2>(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <> __device__ __forceinline__ float2 vsub<float2>(float2 a, float2 b) {
  return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
#endif
template <typename C, typename S> __host__ __device__ __forceinline__ C cscale(C a, S s) { a.x *= s; a.y *= s; return a; }
// multiply by -i (forward) or +i (inverse)
template <typename C> __host__ __device__ __forceinline__ C mul_mi(C a) { C r; r.x = a.y; r.y = -a.x; return r; }
template <typename C> __host__ __device__ __forceinline__ C mul_pi(C a) { C r; r.x = -a.y; r.y = a.x; return r; }

__host__ __device__ __forceinline__ double2 to_c64(float2 a) { return make_double2(a.x, a.y); }
__host__ __device__ __forceinline__ double2 to_c64(double2 a) { return a; }
template <typename R> __host__ __device__ __forceinline__ cx<R> from_c64(double2 a);
template <> __host__ __device__ __forceinline__ float2 from_c64<float>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <> __host__ __device__ __forceinline__ double2 from_c64<double>(double2 a) { return a; }

// Per-batch-entry addressing of an application.  chi / spec: element strides
// between the entries' contrast and spectrum (zero when the whole batch shares
// one operator; non-zero for a group of operators of one grid).  done
// (nullable): entry b's stop flag at done + b * done_stride bytes (non-zero =
// that entry's solve has stopped, its work is skipped); outer: pencil groups
// per entry in the strided passes (C * Nx); status: see the field.
struct BatchStrides {
  size_t chi;
  size_t spec;
  const char* done;
  size_t done_stride;
  int outer;
  int* status;  // this application's status words (bounded waits that gave up), or null
  int chi_layout = 9;  // EM contrast components stored per cell: 9 (full), 6 (symmetric) or 1 (isotropic)
  // element stride between the entries' fields u / out (register row passes);
  // 0: back to back (C cells each)
  size_t field = 0;
  // nullable: the last pass of a matvec also writes, per CTA, the partial
  // sums |t|^2, Re and Im of vdot(t, w) of its output t = u - y (one entry),
  // w = dot_with (same element type and layout as t) or, when that is null, u
  double* dots = nullptr;
  const void* dot_with = nullptr;
};

// Index of entry (r, c) of a symmetric 3x3 contrast stored as its six
// distinct entries xx yy zz xy xz yz.
__host__ __device__ constexpr int sym_index(int r, int c) { return r == c ? r : 2 + r + c; }

__device__ __forceinline__ bool entry_done(const BatchStrides& bs, int b) {
  return bs.done != nullptr && *(volatile const int*)(bs.done + (size_t)b * bs.done_stride) != 0;
}
__device__ __forceinline__ bool entries_done(const BatchStrides& bs, int b0, int b1) {
  if (bs.done == nullptr) return false;
  for (int b = b0; b <= b1; ++b)
    if (!entry_done(bs, b)) return false;
  return true;
}

// A kernel launched inside a device-resident solver loop returns at once when
// the loop's status word says the solve has already stopped.
__device__ __forceinline__ bool skip_launch(const int* flag) {
  return flag != nullptr && *(volatile const int*)flag != 0;
}

}  // namespace em3d

#define EM3D_CUDA_TRY(expr)                                     \
  do {                                                          \
    cudaError_t _e = (expr);                                    \
    if (_e != cudaSuccess) { em3d_set_last_error(cudaGetErrorString(_e)); return EM3D_ERR_CUDA; } \
  } while (0)

#define EM3D_LAUNCH_CHECK()                                     \
  do {                                                          \
    cudaError_t _e = cudaGetLastError();                        \
    if (_e != cudaSuccess) { em3d_set_last_error(cudaGetErrorString(_e)); return EM3D_ERR_CUDA; } \
  } while (0)

void em3d_set_last_error(const char* msg);
