/*
 * em3d_b200 — C ABI of the B200 (sm_100a) implementation of em3d's
 * operator-and-Krylov path.
 *
 * Conventions
 *   - Every entry point returns an int status (EM3D_OK = 0).  On failure the
 *     message is available from em3d_last_error() (thread-local).
 *   - All array arguments are DEVICE pointers to C-contiguous arrays; complex
 *     values are interleaved (re, im) pairs: complex64 (EM3D_C64) or
 *     complex128 (EM3D_C128).  Field layouts follow the reference:
 *       EM field         (batch, 3, Nx, Ny, Nz)       (src/em3d/operator.py:353)
 *       EM contrast chi  (3, 3, Nx, Ny, Nz)            (src/em3d/problem.py:19)
 *       acoustic field   (batch, Nx, Ny, Nz)           (src/em3d/acoustics/operator.py:40)
 *       acoustic chi     (Nx, Ny, Nz)                  (src/em3d/acoustics/problem.py:74)
 *   - `stream` is a cudaStream_t passed as void*; every call is asynchronous
 *     on it and can be captured in a CUDA graph.  No entry point allocates
 *     device memory: the caller provides the spectrum buffer and the workspace,
 *     sized by the *_bytes queries.
 *   - `skip` (nullable) points to a device int; when it is non-zero at launch
 *     time the kernels return without work.  Device-resident solver loops use
 *     it to stop after convergence without a host round trip.
 */
#ifndef EM3D_B200_H
#define EM3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EM3D_ABI_VERSION 1

enum em3d_status {
  EM3D_OK = 0,
  EM3D_ERR_INVALID = 1,     /* bad argument (size, pointer, dtype)           */
  EM3D_ERR_CUDA = 2,        /* CUDA runtime error                            */
  EM3D_ERR_UNSUPPORTED = 3, /* grid size the FFT planner cannot factor       */
};

enum em3d_dtype { EM3D_C64 = 0, EM3D_C128 = 1 };
enum em3d_kind { EM3D_ACOUSTIC = 1, EM3D_EM = 3 };

/* Uniform Cartesian grid: cells per axis and box edge lengths. */
typedef struct em3d_grid {
  int32_t nx, ny, nz;
  double lx, ly, lz;
} em3d_grid;

int em3d_abi_version(void);
const char* em3d_last_error(void);

/* ------------------------------------------------------------------------
 * Sizes
 * ------------------------------------------------------------------------ */

/* Bytes of a prepared operator spectrum: the symmetric octant of the Green
 * spectrum (6 dyadic blocks for EM, 1 for acoustic) in `dtype`, pre-scaled by
 * 1/(8 Nx Ny Nz), followed by the FFT twiddle tables of the three axes.
 * Replaces the storage of PreparedEMKernel.kernel_hat
 * (src/em3d/operator.py:151-223) and AcousticOperator._K_hat
 * (src/em3d/acoustics/operator.py:32-33). */
size_t em3d_spectrum_bytes(const em3d_grid* g, int kind, int dtype);

/* FP64 scratch needed by the spectrum builders (two doubled-grid blocks). */
size_t em3d_build_workspace_bytes(const em3d_grid* g);

/* Scratch needed by one matvec / rmatvec over `batch` right-hand sides. */
size_t em3d_apply_workspace_bytes(const em3d_grid* g, int kind, int dtype, int batch);

/* ------------------------------------------------------------------------
 * Green-spectrum construction (FP64 sampling and FFT, stored in `dtype`)
 * ------------------------------------------------------------------------ */

/* EM dyadic kernel spectrum for wave number k.
 * Replaces PreparedEMKernel.build (src/em3d/operator.py:171-223) with
 * _kernel_geometry / _kernel_block_from_geometry (:28-84). */
int em3d_em_spectrum_build(const em3d_grid* g, double k, int dtype, void* spectrum,
                           void* build_ws, size_t build_ws_bytes, void* stream);

/* Scalar acoustic kernel spectrum k0^2 dv G with the equivalent-sphere self
 * cell.  Replaces prep_coeffs_acoustic / prep_conj_coeffs_acoustic
 * (src/em3d/acoustics/kernel.py:21-58). */
int em3d_acoustic_spectrum_build(const em3d_grid* g, double k0, int dtype, void* spectrum,
                                 void* build_ws, size_t build_ws_bytes, void* stream);

/* Full reference-layout EM spectrum (3,3,2Nx,2Ny,2Nz) in `dtype`, exactly
 * PreparedEMKernel.kernel_hat (adjoint = 0) or kernel_hat_adjoint = fftn(conj K)
 * (adjoint = 1) of src/em3d/operator.py:202-211.  Diagnostic export only; the
 * operator never reads it. */
int em3d_em_kernel_hat_full(const em3d_grid* g, double k, int dtype, int adjoint, void* out,
                            void* build_ws, size_t build_ws_bytes, void* stream);

/* Full acoustic spectrum (2Nx,2Ny,2Nz): fftn(K) or fftn(conj K). */
int em3d_acoustic_kernel_hat_full(const em3d_grid* g, double k0, int dtype, int adjoint, void* out,
                                  void* build_ws, size_t build_ws_bytes, void* stream);

/* ------------------------------------------------------------------------
 * Operator application  A = I - B chi  and its adjoint
 * ------------------------------------------------------------------------ */

/* out = u - crop(IFFT(K_hat . FFT(pad(chi u)))), for `batch` fields.
 * Replaces Operator.matvec (src/em3d/operator.py:353-363). */
int em3d_em_matvec(const em3d_grid* g, int dtype, int batch, const void* spectrum, const void* chi,
                   const void* u, void* out, void* ws, size_t ws_bytes, const int* skip, void* stream);

/* out = v - chi^H crop(IFFT(conj(K_hat) . FFT(pad v))).
 * Replaces Operator.rmatvec (src/em3d/operator.py:365-398), both adjoint storages. */
int em3d_em_rmatvec(const em3d_grid* g, int dtype, int batch, const void* spectrum, const void* chi,
                    const void* v, void* out, void* ws, size_t ws_bytes, const int* skip, void* stream);

/* Scalar versions.  Replace AcousticOperator.matvec / rmatvec
 * (src/em3d/acoustics/operator.py:40-67). */
int em3d_acoustic_matvec(const em3d_grid* g, int dtype, int batch, const void* spectrum, const void* chi,
                         const void* u, void* out, void* ws, size_t ws_bytes, const int* skip, void* stream);
int em3d_acoustic_rmatvec(const em3d_grid* g, int dtype, int batch, const void* spectrum, const void* chi,
                          const void* v, void* out, void* ws, size_t ws_bytes, const int* skip, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* EM3D_B200_H */
