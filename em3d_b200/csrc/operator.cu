// Green-spectrum construction and the fused FFT-convolution operator
// A = I - B chi (EM, 3 components) and H = I - B chi (acoustic, scalar).
//
// Data path of one application (N = Nx x Ny x Nz cells, doubled axes 2N):
//   pass 1  rows along z     : read u (and chi), apply chi, zero-pad, FFT_z  -> T1 (B,C,Nx,Ny,2Nz)
//   pass 2  pencils along y  : zero-pad, FFT_y                               -> T2 (B,C,Nx,2Ny,2Nz)
//   pass 3  pencils along x  : zero-pad, FFT_x, spectrum multiply, IFFT_x,
//                              keep x < Nx                                   -> T2 (in place)
//   pass 4  pencils along y  : IFFT_y, keep y < Ny                          -> T1
//   pass 5  rows along z     : IFFT_z, keep z < Nz, out = u - y (matvec) or
//                              v - chi^H y (rmatvec)                         -> out
// The zero padding is never materialised (pruned inputs), the crop happens
// inside the inverse passes, the 1/(8N) normalisation of ifftn is folded into
// the stored spectrum, and the spectrum is stored as one symmetric octant.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <string>
#include <unordered_set>

#include "operator_passes.cuh"

namespace {
thread_local std::string g_last_error;
}

void em3d_set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

extern "C" const char* em3d_last_error(void) { return g_last_error.c_str(); }
extern "C" int em3d_abi_version(void) { return EM3D_ABI_VERSION; }

namespace em3d {

// Tuning knobs (em3d_set_tuning / em3d_get_tuning).
int g_tuning[EM3D_TUNE_COUNT] = {-1, 0, 0, 0};

// The passes are instantiated in apply_*.cu.
extern template int apply<float, 3, false>(const Dims&, int, const void*, const void*, const void*, void*, void*, size_t, const int*, cudaStream_t, BatchStrides);
extern template int apply<float, 3, true>(const Dims&, int, const void*, const void*, const void*, void*, void*, size_t, const int*, cudaStream_t, BatchStrides);
extern template int apply<float, 1, false>(const Dims&, int, const void*, const void*, const void*, void*, void*, size_t, const int*, cudaStream_t, BatchStrides);
extern template int apply<float, 1, true>(const Dims&, int, const void*, const void*, const void*, void*, void*, size_t, const int*, cudaStream_t, BatchStrides);
extern template int apply<double, 3, false>(const Dims&, int, const void*, const void*, const void*, void*, void*, size_t, const int*, cudaStream_t, BatchStrides);
extern template int apply<double, 3, true>(const Dims&, int, const void*, const void*, const void*, void*, void*, size_t, const int*, cudaStream_t, BatchStrides);
extern template int apply<double, 1, false>(const Dims&, int, const void*, const void*, const void*, void*, void*, size_t, const int*, cudaStream_t, BatchStrides);
extern template int apply<double, 1, true>(const Dims&, int, const void*, const void*, const void*, void*, void*, size_t, const int*, cudaStream_t, BatchStrides);

template <int C, bool ADJ>
static int apply_dispatch(const em3d_grid* g, int dtype, int batch, const void* spectrum, const void* chi,
                          const void* u, void* out, void* ws, size_t wsb, const int* skip, void* stream) {
  Dims d;
  int rc = check_grid(g, &d);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == EM3D_C64) return apply<float, C, ADJ>(d, batch, spectrum, chi, u, out, ws, wsb, skip, st);
  if (dtype == EM3D_C128) return apply<double, C, ADJ>(d, batch, spectrum, chi, u, out, ws, wsb, skip, st);
  em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128");
  return EM3D_ERR_INVALID;
}

// A group of operators on one grid: batch entry b has its own contrast
// (chi + b * chi_stride elements) and spectrum (spectra + b * spectrum_stride
// bytes); the twiddle tables of entry 0 serve all (they depend on the grid
// only).  entry_done: optional per-entry stop flags (see BatchStrides).
template <int C, bool ADJ>
static int apply_grouped(const em3d_grid* g, int dtype, int batch, const void* spectra, size_t spectrum_stride,
                         const void* chis, const void* u, void* out, void* ws, size_t wsb, const int* skip,
                         const void* entry_done, size_t entry_done_stride, void* stream) {
  Dims d;
  int rc = check_grid(g, &d);
  if (rc) return rc;
  if (dtype != EM3D_C64 && dtype != EM3D_C128) { em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128"); return EM3D_ERR_INVALID; }
  const int kind = C == 3 ? EM3D_EM : EM3D_ACOUSTIC;
  const size_t esz = dtype == EM3D_C64 ? sizeof(float2) : sizeof(double2);
  if (spectrum_stride < em3d_spectrum_bytes(g, kind, dtype) || spectrum_stride % esz != 0) {
    em3d_set_last_error("spectrum_stride must be >= em3d_spectrum_bytes and a multiple of the element size");
    return EM3D_ERR_INVALID;
  }
  if (entry_done && entry_done_stride < sizeof(int)) {
    em3d_set_last_error("entry_done_stride must be at least sizeof(int)");
    return EM3D_ERR_INVALID;
  }
  const size_t ncell = (size_t)d.nx * d.ny * d.nz;
  const BatchStrides bs{(C == 3 ? 9 : 1) * ncell, spectrum_stride / esz, (const char*)entry_done,
                        entry_done_stride, 0};
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == EM3D_C64) return apply<float, C, ADJ>(d, batch, spectra, chis, u, out, ws, wsb, skip, st, bs);
  return apply<double, C, ADJ>(d, batch, spectra, chis, u, out, ws, wsb, skip, st, bs);
}

// EM application with the contrast stored as 9, 6 (symmetric) or 1
// (isotropic) components per cell.
template <bool ADJ>
static int em_apply_layout(const em3d_grid* g, int dtype, int batch, const void* spectrum, int chi_layout,
                           const void* chi, const void* u, void* out, void* ws, size_t wsb, const int* skip,
                           void* stream) {
  Dims d;
  int rc = check_grid(g, &d);
  if (rc) return rc;
  if (chi_layout != EM3D_CHI_FULL && chi_layout != EM3D_CHI_SYMMETRIC && chi_layout != EM3D_CHI_ISOTROPIC) {
    em3d_set_last_error("chi_layout must be EM3D_CHI_FULL (9), EM3D_CHI_SYMMETRIC (6) or EM3D_CHI_ISOTROPIC (1)");
    return EM3D_ERR_INVALID;
  }
  BatchStrides bs{};
  bs.chi_layout = chi_layout;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == EM3D_C64) return apply<float, 3, ADJ>(d, batch, spectrum, chi, u, out, ws, wsb, skip, st, bs);
  if (dtype == EM3D_C128) return apply<double, 3, ADJ>(d, batch, spectrum, chi, u, out, ws, wsb, skip, st, bs);
  em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128");
  return EM3D_ERR_INVALID;
}

template <typename S, typename D> __global__ void k_round_copy(const S* __restrict__ src, D* __restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = from_c64<decltype(dst[0].x)>(to_c64(src[i]));
}

// Copy a prepared spectrum into another precision: the octant blocks and the
// twiddle tables are converted element by element.  A build in either
// precision computes the same FP64 values (octant samples scaled by 1/(8N);
// twiddles from sincospi) and rounds them once to the stored type, so a
// complex128 spectrum rounded to complex64 is bit-identical to a complex64
// build (the widening direction only changes the type).
template <typename RS, typename RD>
static int spectrum_convert(const Dims& d, int kind, const void* src, void* dst, cudaStream_t st) {
  SpecLayout<RS> ls(d, kind);
  SpecLayout<RD> ld(d, kind);
  const size_t noct = ls.blocks * ls.oct_elems;
  const size_t ntw = (size_t)2 * (d.nx + d.ny + d.nz);
  void* s = const_cast<void*>(src);
  const int g1 = (int)std::min<size_t>((noct + 255) / 256, (size_t)148 * 16);
  k_round_copy<<<g1, 256, 0, st>>>(ls.oct(s), ld.oct(dst), noct);
  EM3D_LAUNCH_CHECK();
  k_round_copy<<<(int)((ntw + 255) / 256), 256, 0, st>>>(ls.twx(s, d), ld.twx(dst, d), ntw);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

}  // namespace em3d

using namespace em3d;

extern "C" {

int em3d_set_tuning(int key, int value) {
  if (key < 0 || key >= EM3D_TUNE_COUNT) { em3d_set_last_error("unknown tuning key"); return EM3D_ERR_INVALID; }
  if (key == EM3D_TUNE_XPASS_VARIANT && (value < -1 || value > 10)) {
    em3d_set_last_error("x-pass variant must be -1 (automatic) or 0 .. 10");
    return EM3D_ERR_INVALID;
  }
  if (key == EM3D_TUNE_FNO_SIMT && (value < 0 || value > 3)) {
    em3d_set_last_error("FNO row-pass switch must be 0, 1, 2 or 3");
    return EM3D_ERR_INVALID;
  }
  if (key == EM3D_TUNE_FNO_CONTRACT && value != 0 && value != 2 && value != 4 && value != 8 && value != 12 &&
      value != 24) {
    em3d_set_last_error("FNO contraction blocking must be 0 (automatic), 2, 4, 8, 12 or 24");
    return EM3D_ERR_INVALID;
  }
  g_tuning[key] = value;
  return EM3D_OK;
}

int em3d_get_tuning(int key) { return (key >= 0 && key < EM3D_TUNE_COUNT) ? g_tuning[key] : -1; }

size_t em3d_spectrum_bytes(const em3d_grid* g, int kind, int dtype) {
  Dims d;
  if (check_grid(g, &d) || (kind != EM3D_EM && kind != EM3D_ACOUSTIC)) return 0;
  return dtype == EM3D_C64 ? SpecLayout<float>(d, kind).total_bytes : SpecLayout<double>(d, kind).total_bytes;
}

size_t em3d_build_workspace_bytes(const em3d_grid* g) {
  Dims d;
  if (check_grid(g, &d)) return 0;
  return build_ws_bytes(d);
}

size_t em3d_apply_workspace_bytes(const em3d_grid* g, int kind, int dtype, int batch) {
  Dims d;
  if (check_grid(g, &d) || batch < 1 || (kind != EM3D_EM && kind != EM3D_ACOUSTIC)) return 0;
  return dtype == EM3D_C64 ? apply_ws_bytes<float>(d, kind, batch) : apply_ws_bytes<double>(d, kind, batch);
}

int em3d_em_spectrum_build(const em3d_grid* g, double k, int dtype, void* spectrum, void* ws, size_t wsb, void* stream) {
  Dims d;
  int rc = check_grid(g, &d);
  if (rc) return rc;
  if (!spectrum) { em3d_set_last_error("spectrum is NULL"); return EM3D_ERR_INVALID; }
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == EM3D_C64) return em_spectrum_build<float>(g, d, k, spectrum, ws, wsb, st);
  if (dtype == EM3D_C128) return em_spectrum_build<double>(g, d, k, spectrum, ws, wsb, st);
  em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128");
  return EM3D_ERR_INVALID;
}

int em3d_acoustic_spectrum_build(const em3d_grid* g, double k0, int dtype, void* spectrum, void* ws, size_t wsb,
                                 void* stream) {
  Dims d;
  int rc = check_grid(g, &d);
  if (rc) return rc;
  if (!spectrum) { em3d_set_last_error("spectrum is NULL"); return EM3D_ERR_INVALID; }
  if (!(k0 > 0)) { em3d_set_last_error("k0 must be positive"); return EM3D_ERR_INVALID; }
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == EM3D_C64) return ac_spectrum_build<float>(g, d, k0, spectrum, ws, wsb, st);
  if (dtype == EM3D_C128) return ac_spectrum_build<double>(g, d, k0, spectrum, ws, wsb, st);
  em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128");
  return EM3D_ERR_INVALID;
}

int em3d_spectrum_convert(const em3d_grid* g, int kind, int src_dtype, const void* src, int dst_dtype, void* dst,
                          void* stream) {
  Dims d;
  int rc = check_grid(g, &d);
  if (rc) return rc;
  if (kind != EM3D_EM && kind != EM3D_ACOUSTIC) { em3d_set_last_error("kind must be EM3D_EM or EM3D_ACOUSTIC"); return EM3D_ERR_INVALID; }
  if (!src || !dst) { em3d_set_last_error("NULL spectrum"); return EM3D_ERR_INVALID; }
  if (src == dst) { em3d_set_last_error("src and dst must be different buffers"); return EM3D_ERR_INVALID; }
  cudaStream_t st = (cudaStream_t)stream;
  if (src_dtype == EM3D_C128 && dst_dtype == EM3D_C64) return spectrum_convert<double, float>(d, kind, src, dst, st);
  if (src_dtype == EM3D_C64 && dst_dtype == EM3D_C128) return spectrum_convert<float, double>(d, kind, src, dst, st);
  if (src_dtype == EM3D_C64 && dst_dtype == EM3D_C64) return spectrum_convert<float, float>(d, kind, src, dst, st);
  if (src_dtype == EM3D_C128 && dst_dtype == EM3D_C128) return spectrum_convert<double, double>(d, kind, src, dst, st);
  em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128");
  return EM3D_ERR_INVALID;
}

int em3d_em_kernel_hat_full(const em3d_grid* g, double k, int dtype, int adjoint, void* out, void* ws, size_t wsb,
                            void* stream) {
  Dims d;
  int rc = check_grid(g, &d);
  if (rc) return rc;
  if (!out) { em3d_set_last_error("out is NULL"); return EM3D_ERR_INVALID; }
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == EM3D_C64) return em_kernel_hat_full<float>(g, d, k, adjoint, out, ws, wsb, st);
  if (dtype == EM3D_C128) return em_kernel_hat_full<double>(g, d, k, adjoint, out, ws, wsb, st);
  em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128");
  return EM3D_ERR_INVALID;
}

int em3d_acoustic_kernel_hat_full(const em3d_grid* g, double k0, int dtype, int adjoint, void* out, void* ws,
                                  size_t wsb, void* stream) {
  Dims d;
  int rc = check_grid(g, &d);
  if (rc) return rc;
  if (!out) { em3d_set_last_error("out is NULL"); return EM3D_ERR_INVALID; }
  if (!(k0 > 0)) { em3d_set_last_error("k0 must be positive"); return EM3D_ERR_INVALID; }
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == EM3D_C64) return ac_kernel_hat_full<float>(g, d, k0, adjoint, out, ws, wsb, st);
  if (dtype == EM3D_C128) return ac_kernel_hat_full<double>(g, d, k0, adjoint, out, ws, wsb, st);
  em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128");
  return EM3D_ERR_INVALID;
}

int em3d_em_matvec_grouped(const em3d_grid* g, int dtype, int batch, const void* spectra, size_t spectrum_stride,
    const void* chis, const void* u, void* out, void* ws, size_t wsb, const int* skip, const void* entry_done,
    size_t entry_done_stride, void* stream) {
  return apply_grouped<3, false>(g, dtype, batch, spectra, spectrum_stride, chis, u, out, ws, wsb, skip, entry_done,
                                 entry_done_stride, stream);
}
int em3d_em_rmatvec_grouped(const em3d_grid* g, int dtype, int batch, const void* spectra, size_t spectrum_stride,
    const void* chis, const void* v, void* out, void* ws, size_t wsb, const int* skip, const void* entry_done,
    size_t entry_done_stride, void* stream) {
  return apply_grouped<3, true>(g, dtype, batch, spectra, spectrum_stride, chis, v, out, ws, wsb, skip, entry_done,
                                 entry_done_stride, stream);
}
int em3d_acoustic_matvec_grouped(const em3d_grid* g, int dtype, int batch, const void* spectra, size_t spectrum_stride,
    const void* chis, const void* u, void* out, void* ws, size_t wsb, const int* skip, const void* entry_done,
    size_t entry_done_stride, void* stream) {
  return apply_grouped<1, false>(g, dtype, batch, spectra, spectrum_stride, chis, u, out, ws, wsb, skip, entry_done,
                                 entry_done_stride, stream);
}
int em3d_acoustic_rmatvec_grouped(const em3d_grid* g, int dtype, int batch, const void* spectra, size_t spectrum_stride,
    const void* chis, const void* v, void* out, void* ws, size_t wsb, const int* skip, const void* entry_done,
    size_t entry_done_stride, void* stream) {
  return apply_grouped<1, true>(g, dtype, batch, spectra, spectrum_stride, chis, v, out, ws, wsb, skip, entry_done,
                                 entry_done_stride, stream);
}

int em3d_em_matvec_chi(const em3d_grid* g, int dtype, int batch, const void* spectrum, int chi_layout,
                       const void* chi, const void* u, void* out, void* ws, size_t wsb, const int* skip,
                       void* stream) {
  return em_apply_layout<false>(g, dtype, batch, spectrum, chi_layout, chi, u, out, ws, wsb, skip, stream);
}

int em3d_em_rmatvec_chi(const em3d_grid* g, int dtype, int batch, const void* spectrum, int chi_layout,
                        const void* chi, const void* v, void* out, void* ws, size_t wsb, const int* skip,
                        void* stream) {
  return em_apply_layout<true>(g, dtype, batch, spectrum, chi_layout, chi, v, out, ws, wsb, skip, stream);
}

int em3d_matvec_dot_parts(int kind, const em3d_grid* g, int dtype) {
  Dims d;
  if (check_grid(g, &d)) return 0;
  if (kind != EM3D_EM && kind != EM3D_ACOUSTIC) return 0;
  const bool f64 = dtype == EM3D_C128;
  if ((dtype != EM3D_C64 && !f64) || !fast_len(2 * d.nz, f64, false)) return 0;
  const int nrows = d.nx * d.ny;
  if (kind == EM3D_EM) return f64 ? rows_fast_ctas<double, 3>(2 * d.nz, nrows) : rows_fast_ctas<float, 3>(2 * d.nz, nrows);
  return f64 ? rows_fast_ctas<double, 1>(2 * d.nz, nrows) : rows_fast_ctas<float, 1>(2 * d.nz, nrows);
}

int em3d_matvec_dots(int kind, const em3d_grid* g, int dtype, const void* spectrum, int chi_layout, const void* chi,
                     const void* u, void* out, void* ws, size_t wsb, const int* skip, double* partials,
                     const void* dot_with, void* stream) {
  Dims d;
  int rc = check_grid(g, &d);
  if (rc) return rc;
  if (!partials) { em3d_set_last_error("partials is NULL"); return EM3D_ERR_INVALID; }
  BatchStrides bs{};
  bs.dots = partials;
  bs.dot_with = dot_with;
  cudaStream_t st = (cudaStream_t)stream;
  if (kind == EM3D_EM) {
    if (chi_layout != EM3D_CHI_FULL && chi_layout != EM3D_CHI_SYMMETRIC && chi_layout != EM3D_CHI_ISOTROPIC) {
      em3d_set_last_error("chi_layout must be EM3D_CHI_FULL (9), EM3D_CHI_SYMMETRIC (6) or EM3D_CHI_ISOTROPIC (1)");
      return EM3D_ERR_INVALID;
    }
    bs.chi_layout = chi_layout;
    if (dtype == EM3D_C64) return apply<float, 3, false>(d, 1, spectrum, chi, u, out, ws, wsb, skip, st, bs);
    if (dtype == EM3D_C128) return apply<double, 3, false>(d, 1, spectrum, chi, u, out, ws, wsb, skip, st, bs);
  } else if (kind == EM3D_ACOUSTIC) {
    if (dtype == EM3D_C64) return apply<float, 1, false>(d, 1, spectrum, chi, u, out, ws, wsb, skip, st, bs);
    if (dtype == EM3D_C128) return apply<double, 1, false>(d, 1, spectrum, chi, u, out, ws, wsb, skip, st, bs);
  } else {
    em3d_set_last_error("kind must be EM3D_EM or EM3D_ACOUSTIC");
    return EM3D_ERR_INVALID;
  }
  em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128");
  return EM3D_ERR_INVALID;
}

int em3d_em_matvec(const em3d_grid* g, int dtype, int batch, const void* spectrum, const void* chi, const void* u,
                   void* out, void* ws, size_t wsb, const int* skip, void* stream) {
  return apply_dispatch<3, false>(g, dtype, batch, spectrum, chi, u, out, ws, wsb, skip, stream);
}

int em3d_em_rmatvec(const em3d_grid* g, int dtype, int batch, const void* spectrum, const void* chi, const void* v,
                    void* out, void* ws, size_t wsb, const int* skip, void* stream) {
  return apply_dispatch<3, true>(g, dtype, batch, spectrum, chi, v, out, ws, wsb, skip, stream);
}

int em3d_acoustic_matvec(const em3d_grid* g, int dtype, int batch, const void* spectrum, const void* chi,
                         const void* u, void* out, void* ws, size_t wsb, const int* skip, void* stream) {
  return apply_dispatch<1, false>(g, dtype, batch, spectrum, chi, u, out, ws, wsb, skip, stream);
}

int em3d_acoustic_rmatvec(const em3d_grid* g, int dtype, int batch, const void* spectrum, const void* chi,
                          const void* v, void* out, void* ws, size_t wsb, const int* skip, void* stream) {
  return apply_dispatch<1, true>(g, dtype, batch, spectrum, chi, v, out, ws, wsb, skip, stream);
}

}  // extern "C"
