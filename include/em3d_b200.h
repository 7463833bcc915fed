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
/* Storage of an EM contrast: components per cell.  FULL is the reference's
 * (3,3,Nx,Ny,Nz); SYMMETRIC keeps chi_xx, chi_yy, chi_zz, chi_xy, chi_xz,
 * chi_yz as (6,Nx,Ny,Nz) for chi = chi^T (rotated anisotropic media);
 * ISOTROPIC keeps s as (Nx,Ny,Nz) for chi = s I (isotropic media). */
enum em3d_chi_layout { EM3D_CHI_ISOTROPIC = 1, EM3D_CHI_SYMMETRIC = 6, EM3D_CHI_FULL = 9 };

/* Uniform Cartesian grid: cells per axis and box edge lengths. */
typedef struct em3d_grid {
  int32_t nx, ny, nz;
  double lx, ly, lz;
} em3d_grid;

int em3d_abi_version(void);
const char* em3d_last_error(void);

/* ------------------------------------------------------------------------
 * Tuning (process-wide; chosen by em3d_b200.tune.autotune).  No counterpart
 * in the reference, which has no native code to tune.
 * ------------------------------------------------------------------------ */
enum em3d_tune_key {
  EM3D_TUNE_XPASS_VARIANT = 0, /* x pass: -1 automatic (default: EM 6, acoustic 9 at 512 points, else 0), 0 register 256-thread, 1 register
                                   128-thread, 2 component-split, 3 persistent cp.async-pipelined 256-thread,
                                   4 the same 128-thread, 5 and 6 = 3 and 4 with the field slab loaded by
                                   TMA, 7 / 8 / 9 = 6 with register twiddles and single-barrier exchanges
                                   (component loop / inlined components / 256 threads; plans equal to their
                                   reverse), 10 = 6 with 8 elements per thread in two 256-thread CTAs per SM
                                   (complex64, power-of-two axes); a variant that does not apply or whose
                                   shared memory does not fit is replaced by the first that fits in the
                                   order 6, 4, 1, 2, 0, 5, 3 */
  EM3D_TUNE_FFT_GENERIC = 1,   /* 1 = use the generic shared-memory FFT passes for every axis length */
  EM3D_TUNE_FNO_SIMT = 2,      /* FNO row pass (bf16, width 32, Z a multiple of 32): 0 = automatic (the layer passes on
                                   tcgen05 with TMEM accumulators, the lift on mma.sync), 1 = CUDA cores everywhere,
                                   2 = the same as 0, 3 = mma.sync for the layer passes too */
  EM3D_TUNE_FNO_CONTRACT = 3,  /* FNO truncated-DFT contractions: 0 automatic, else outputs per thread (2, 4, 8, 12, 24) */
  EM3D_TUNE_COUNT = 4,
};
int em3d_set_tuning(int key, int value);
int em3d_get_tuning(int key);

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

/* Scratch needed by one matvec / rmatvec over `batch` right-hand sides.  Its
 * last 256 bytes are status words: the int at the start of them counts the
 * bounded waits inside the passes that gave up (a transfer that never
 * completed; the result is then wrong).  Zero the workspace once after
 * allocating it; the library only ever adds to that count. */
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

/* The spectrum `src` (built for grid g and operator `kind` in `src_dtype`)
 * copied into `dst` (em3d_spectrum_bytes(g, kind, dst_dtype) bytes) in
 * `dst_dtype`.  complex128 -> complex64 gives exactly the bytes of a
 * complex64 build, without sampling or transforming again: the FP32 twin of
 * an FP64 operator (PreparedEMKernel.build, src/em3d/operator.py:171-223,
 * for the same grid and k in the other precision). */
int em3d_spectrum_convert(const em3d_grid* g, int kind, int src_dtype, const void* src, int dst_dtype,
                          void* dst, void* stream);

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

/* em3d_em_matvec / em3d_em_rmatvec with the contrast in `chi_layout`
 * (em3d_chi_layout).  The symmetric and isotropic storages read 6/9 and 1/9
 * of the contrast bytes in the passes that apply chi (the first pass of a
 * matvec, the last of an rmatvec); the result is that of the full storage
 * of the same contrast.  Same operator as Operator.matvec / rmatvec
 * (src/em3d/operator.py:353-398), whose Problem keeps the full tensor
 * (src/em3d/problem.py:19-32). */
int em3d_em_matvec_chi(const em3d_grid* g, int dtype, int batch, const void* spectrum, int chi_layout,
                       const void* chi, const void* u, void* out, void* ws, size_t ws_bytes, const int* skip,
                       void* stream);
int em3d_em_rmatvec_chi(const em3d_grid* g, int dtype, int batch, const void* spectrum, int chi_layout,
                        const void* chi, const void* v, void* out, void* ws, size_t ws_bytes, const int* skip,
                        void* stream);

/* EM matvec for callers that cannot allocate device memory (no counterpart
 * in the reference).  Same result as em3d_em_matvec with batch = 1, but the
 * workspace is a fixed 64 MiB device array inside the library (held on every
 * GPU that uses the library until the process exits), so the caller passes
 * only inputs and outputs.  Grids whose workspace exceeds 64 MiB are rejected
 * with EM3D_ERR_INVALID (about 466k cells in complex64, 233k in complex128).
 * The first call on a device looks up the array's device address; make it
 * before any stream capture.  Calls share the array: calls that overlap on
 * the GPU race and must be serialised by the caller. */
int em3d_em_matvec_static_scratch(const em3d_grid* g, int dtype, const void* spectrum, const void* chi,
                                  const void* u, void* out, const int* skip, void* stream);
/* Size of that fixed workspace in bytes. */
size_t em3d_static_scratch_bytes(void);

/* Groups of operators on one grid (many problems of the same size, each with
 * its own contrast and wave number): batch entry b of u / out is applied with
 * the contrast at chis + b * (9 or 1) * Nx*Ny*Nz elements and the spectrum at
 * spectra + b * spectrum_stride bytes (each built by em3d_*_spectrum_build;
 * spectrum_stride >= em3d_spectrum_bytes, a multiple of the element size).
 * One launch per pass for the whole group; workspace as for a batch of that
 * size.  entry_done (nullable): entry b's int stop flag at entry_done +
 * b * entry_done_stride bytes; the work of entries whose flag is non-zero is
 * skipped and their out left as it was (a batched solve passes its per-entry
 * status words).  No counterpart call in the reference, which solves such
 * sets one problem at a time with src/em3d/operator.py:320-428 /
 * src/em3d/acoustics/operator.py:25-73. */
int em3d_em_matvec_grouped(const em3d_grid* g, int dtype, int batch, const void* spectra, size_t spectrum_stride,
    const void* chis, const void* u, void* out, void* workspace, size_t workspace_bytes, const int* skip,
    const void* entry_done, size_t entry_done_stride, void* stream);
int em3d_em_rmatvec_grouped(const em3d_grid* g, int dtype, int batch, const void* spectra, size_t spectrum_stride,
    const void* chis, const void* v, void* out, void* workspace, size_t workspace_bytes, const int* skip,
    const void* entry_done, size_t entry_done_stride, void* stream);
int em3d_acoustic_matvec_grouped(const em3d_grid* g, int dtype, int batch, const void* spectra, size_t spectrum_stride,
    const void* chis, const void* u, void* out, void* workspace, size_t workspace_bytes, const int* skip,
    const void* entry_done, size_t entry_done_stride, void* stream);
int em3d_acoustic_rmatvec_grouped(const em3d_grid* g, int dtype, int batch, const void* spectra, size_t spectrum_stride,
    const void* chis, const void* v, void* out, void* workspace, size_t workspace_bytes, const int* skip,
    const void* entry_done, size_t entry_done_stride, void* stream);

/* Problems of uneven grid sizes in one application: each of the five passes
 * is ONE launch over every problem of every segment (a segment = `count`
 * problems on one grid, each with its own spectrum, contrast and field); a
 * CTA finds its segment and runs the register FFT of that segment's axis
 * length.  Up to EM3D_MAX_SEGMENTS segments; every doubled axis length
 * (2 Nx, 2 Ny, 2 Nz) must be one em3d_uneven_supported accepts (32..256:
 * powers of two, 96, 160, 192, with the exceptions it reports).  All
 * strides are in bytes and multiples of the element size.  EM segments share
 * one chi_layout.  Stopped entries (entry_done) are skipped as in the grouped
 * calls; `skip` is the whole-application flag.  No counterpart call in the
 * reference, which solves such sets one problem at a time
 * (src/em3d/operator.py:320-428 per problem). */
#define EM3D_MAX_SEGMENTS 8
typedef struct em3d_segment {
  em3d_grid grid;
  int32_t count;                /* problems in this segment (>= 1)                   */
  int32_t chi_layout;           /* EM: EM3D_CHI_FULL / SYMMETRIC / ISOTROPIC; acoustic: ignored */
  const void* spectra;          /* problem j's spectrum at spectra + j * spectrum_stride */
  size_t spectrum_stride;       /* >= em3d_spectrum_bytes of this grid              */
  const void* chi;              /* problem j's contrast at chi + j * chi_stride       */
  size_t chi_stride;
  const void* u;                /* problem j's input field at u + j * field_stride    */
  void* out;                    /* problem j's output at out + j * field_stride       */
  size_t field_stride;          /* >= C * Nx*Ny*Nz elements                          */
  const void* entry_done;       /* nullable: problem j's int stop flag at entry_done + j * entry_done_stride */
  size_t entry_done_stride;
} em3d_segment;

/* sizeof(em3d_segment) as compiled into the library (ABI check). */
size_t em3d_segment_size(void);
/* 1 if a problem on grid g can join an uneven application of this kind and
 * dtype, else 0. */
int em3d_uneven_supported(const em3d_grid* g, int kind, int dtype);
/* Workspace bytes of an uneven application (each segment's two transform
 * buffers, then 256 bytes of status words as for em3d_apply_workspace_bytes);
 * only the grids, counts, layouts and strides are read (the array pointers
 * may still be NULL); 0 for invalid segments. */
size_t em3d_uneven_workspace_bytes(int kind, int dtype, int nseg, const em3d_segment* segs);
int em3d_em_matvec_uneven(int dtype, int nseg, const em3d_segment* segs, void* workspace, size_t workspace_bytes,
                          const int* skip, void* stream);
int em3d_em_rmatvec_uneven(int dtype, int nseg, const em3d_segment* segs, void* workspace, size_t workspace_bytes,
                           const int* skip, void* stream);
int em3d_acoustic_matvec_uneven(int dtype, int nseg, const em3d_segment* segs, void* workspace,
                                size_t workspace_bytes, const int* skip, void* stream);
int em3d_acoustic_rmatvec_uneven(int dtype, int nseg, const em3d_segment* segs, void* workspace,
                                 size_t workspace_bytes, const int* skip, void* stream);

/* A matvec of one right-hand side (EM with chi stored in chi_layout, or
 * acoustic) whose last pass also writes, per CTA, the partial sums of
 * |t|^2 and Re / Im of vdot(t, w) of its output t = u - A' u, three doubles
 * per CTA at partials[3 * cta]; w = dot_with (nullable; the layout and
 * element type of u), u itself when dot_with is NULL.  These are the inner
 * products BiCGStab forms right after each matvec, without reading the
 * vectors again: vdot(t, t) and vdot(t, s) after t = A s (u = s, dot_with
 * NULL; src/em3d/solvers/bicgstab.py:151-161) and vdot(r_hat, v) =
 * conj(vdot(v, r_hat)) after v = A p (u = p, dot_with = r_hat;
 * bicgstab.py:106-108).  em3d_matvec_dot_parts gives the number of CTAs
 * (partials holds 3x that many doubles); 0 when the z axis has no register
 * FFT (then this call returns EM3D_ERR_UNSUPPORTED).
 * em3d_bicgstab_omega_parts and em3d_bicgstab_alpha_parts finish omega and
 * alpha from the partials. */
int em3d_matvec_dot_parts(int kind, const em3d_grid* g, int dtype);
int em3d_matvec_dots(int kind, const em3d_grid* g, int dtype, const void* spectrum, int chi_layout, const void* chi,
                     const void* u, void* out, void* ws, size_t ws_bytes, const int* skip, double* partials,
                     const void* dot_with, void* stream);

/* Scalar versions.  Replace AcousticOperator.matvec / rmatvec
 * (src/em3d/acoustics/operator.py:40-67). */
int em3d_acoustic_matvec(const em3d_grid* g, int dtype, int batch, const void* spectrum, const void* chi,
                         const void* u, void* out, void* ws, size_t ws_bytes, const int* skip, void* stream);
int em3d_acoustic_rmatvec(const em3d_grid* g, int dtype, int batch, const void* spectrum, const void* chi,
                          const void* v, void* out, void* ws, size_t ws_bytes, const int* skip, void* stream);


/* ------------------------------------------------------------------------
 * Device-resident Krylov solvers
 *
 * The solver scalars, counters, status and residual history of one
 * right-hand side live in one device block (em3d_krylov_state followed by
 * the history and the reduction partials; size from
 * em3d_krylov_state_bytes).  A batch of `batch` right-hand sides uses
 * `batch` such blocks `state_stride` bytes apart and vectors stored batch
 * after batch, each of length n; every right-hand side keeps its own
 * scalars and stops on its own.  Inner products and norms accumulate in FP64
 * whatever the vector dtype.  Step kernels skip right-hand sides whose
 * status != 0, and the operator entry points take &state[0].batch_done as
 * their `skip` flag, so a sequence of iterations can be launched (or
 * replayed from a CUDA graph) without host round trips; the host reads
 * batch_done once per chunk of iterations.
 * ------------------------------------------------------------------------ */

enum em3d_solver_status {
  EM3D_RUNNING = 0,
  EM3D_CONVERGED = 1,
  EM3D_MAX_ITER = 2,
  EM3D_MAX_OPERATOR_ACTIONS = 3,
  EM3D_NONFINITE = 4,
  EM3D_DIVERGENCE_GUARD = 5,
  EM3D_BREAKDOWN_RHO = 6,
  EM3D_BREAKDOWN_ALPHA = 7,
  EM3D_BREAKDOWN_OMEGA = 8,
  EM3D_BREAKDOWN_T = 9,
  EM3D_BREAKDOWN_GRADIENT = 10,
};

typedef struct em3d_krylov_state {
  double rhs_norm;             /* ||f||                                        */
  double tol;                  /* max(rtol, atol / ||f||)                      */
  double guard;                /* divergence guard; < 0 disables it            */
  double gamma_re, gamma_im;   /* SIM step 1/mu                                */
  double rho_re, rho_im, rho_prev_re, rho_prev_im;
  double alpha_re, alpha_im, omega_re, omega_im;
  double t, h;                 /* TwoStep step coefficients                    */
  double last_rel;             /* last recorded relative residual              */
  double dots[4];              /* output of em3d_vec_dots (re, im pairs)       */
  int32_t status;              /* enum em3d_solver_status                      */
  int32_t iter;                /* completed updates                            */
  int32_t matvecs, rmatvecs;   /* operator actions so far                      */
  int32_t max_iter;
  int32_t max_actions;         /* < 0 disables the action budget               */
  int32_t hist_len, hist_cap;  /* residual history entries used / capacity     */
  int32_t pending;             /* BiCGStab: 1 = u += alpha p still to apply    */
  int32_t first;               /* TwoStep: 1 before the first update; BiCGStab:
                                  non-zero disables the half-step (||s||)
                                  convergence exit                              */
  uint32_t ticket;             /* last-block counter of the reductions         */
  int32_t batch_running;       /* state 0 only: right-hand sides still running */
  int32_t batch_done;          /* state 0 only: 1 once all have stopped; the
                                  operator's `skip` flag in a solve loop        */
  int32_t n_used;              /* elements of this right-hand side's n in use;
                                  the step kernels leave the rest (padding of
                                  a problem smaller than n) alone; 0: all n    */
} em3d_krylov_state;

/* sizeof(em3d_krylov_state) as compiled into the library (ABI check). */
size_t em3d_krylov_state_size(void);

/* Bytes of the state buffer: the struct (padded to 256 B), the residual
 * history (double[hist_cap]) and its action counts (int32[hist_cap]), and the
 * reduction partials. */
size_t em3d_krylov_state_bytes(int hist_cap);
/* Offsets of the history arrays inside the state buffer. */
size_t em3d_krylov_history_offset(int hist_cap);
size_t em3d_krylov_counts_offset(int hist_cap);

/* Per right-hand side b: state[b].dots[0..1] = vdot(x0_b, y0_b) and
 * state[b].dots[2..3] = vdot(x1_b, y1_b) (when x1 != NULL); FP64 accumulation.  Replaces xp.vdot / xp.linalg.norm of the
 * solvers (src/em3d/solvers/bicgstab.py:70,90). */
int em3d_vec_dots(int dtype, size_t n, int batch, const void* x0, const void* y0, const void* x1, const void* y1,
                  void* state, size_t state_stride, void* stream);
/* out = a*x + b*y (scalars rounded to the vector dtype; y may be NULL). */
int em3d_vec_axpby(int dtype, size_t n, void* out, double a_re, double a_im, const void* x, double b_re,
                   double b_im, const void* y, void* stream);
/* dst = src for a few bytes (at most em3d_copy_small_max_bytes(), both
 * 4-byte aligned) between device memory and pinned host memory, by a kernel
 * on `stream` rather than a copy engine: a small read-back or state upload
 * of a solver then never waits behind a large transfer that another stream
 * queued on the copy engines.  Pageable host memory is refused
 * (EM3D_ERR_INVALID); the copy is complete once the stream has reached it. */
size_t em3d_copy_small_max_bytes(void);
int em3d_copy_small(void* dst, const void* src, size_t bytes, void* stream);

/* Precision conversion dst = src (complex64 <-> complex128), or, with
 * accumulate = 1, dst += src. */
int em3d_vec_convert(size_t n, int src_dtype, const void* src, int dst_dtype, void* dst, int accumulate,
                     void* stream);

/* BiCGStab (src/em3d/solvers/bicgstab.py:12-211), one iteration =
 *   p -> [matvec v = A p] -> alpha -> s -> [matvec t = A s] -> omega -> update
 * The update also completes an early exit taken at s in the same iteration
 * (the reference returns u + alpha p there); em3d_bicgstab_finalize does only
 * that, for a driver that stops between s and update, and is a no-op once the
 * exit has been completed. */
int em3d_bicgstab_p(int dtype, size_t n, int batch, void* state, size_t state_stride, const void* r, void* p, const void* v, void* stream);
int em3d_bicgstab_alpha(int dtype, size_t n, int batch, void* state, size_t state_stride, const void* r_hat, const void* v, void* stream);
int em3d_bicgstab_s(int dtype, size_t n, int batch, void* state, size_t state_stride, const void* r, const void* v, void* s, void* stream);
int em3d_bicgstab_omega(int dtype, size_t n, int batch, void* state, size_t state_stride, const void* t, const void* s, void* stream);
/* The same omega step for one right-hand side from the nparts per-CTA partial
 * sums (3 doubles each) that em3d_matvec_dots wrote while forming t = A s. */
int em3d_bicgstab_omega_parts(int nparts, void* state, const double* partials, void* stream);
/* The alpha step for one right-hand side from the nparts per-CTA partial sums
 * that em3d_matvec_dots wrote while forming v = A p with dot_with = r_hat. */
int em3d_bicgstab_alpha_parts(int nparts, void* state, const double* partials, void* stream);
int em3d_bicgstab_update(int dtype, size_t n, int batch, void* state, size_t state_stride, void* u, const void* p, const void* s, const void* t,
                         void* r, const void* r_hat, void* stream);
int em3d_bicgstab_finalize(int dtype, size_t n, int batch, void* state, size_t state_stride, void* u, const void* p, void* stream);

/* SIM (src/em3d/solvers/sim.py:13-91): [matvec res = A u] -> residual -> update */
int em3d_sim_residual(int dtype, size_t n, int batch, void* state, size_t state_stride, void* res, const void* f, void* stream);
int em3d_sim_update(int dtype, size_t n, int batch, void* state, size_t state_stride, void* u, const void* res, void* stream);

/* TwoStep (src/em3d/solvers/twostep.py:16-139):
 *   [matvec r = A u] -> residual -> [rmatvec g = A* r] -> [matvec hg = A g] -> coeffs -> update */
int em3d_twostep_residual(int dtype, size_t n, int batch, void* state, size_t state_stride, void* r, const void* f, void* stream);
int em3d_twostep_coeffs(int dtype, size_t n, int batch, void* state, size_t state_stride, const void* r, const void* r_prev, const void* g,
                        const void* hg, void* stream);
int em3d_twostep_update(int dtype, size_t n, int batch, void* state, size_t state_stride, void* u, void* u_prev, const void* r, void* r_prev,
                        const void* g, void* stream);

/* ------------------------------------------------------------------------
 * Fourier-neural-operator warm start (no counterpart in the reference: the
 * learned initial guess for the solvers).  Activations/weights in `act`
 * (0 = bf16, 1 = float), FP32 accumulation; channel tensors (B, C, X, Y, Z);
 * mode-space tensors complex64.  See em3d_b200/csrc/fno.cu for the network.
 * ------------------------------------------------------------------------ */
int em3d_fno_lift(int act, int B, size_t ncell, int W, const void* chi, const void* wave, const void* P,
                  const float* pb, void* v0, void* stream);
int em3d_fno_lift_bwd(int B, size_t ncell, int W, const void* chi, const void* wave, const float* dv0, float* dP,
                      float* dpb, void* stream);
/* kind 0: real(act) -> complex; 1: complex -> complex; 2: complex -> real, += Re(.) */
int em3d_fno_contract(int kind, int act, size_t outer, int L, int J, int inner, const void* X, const void* M, void* Y,
                      void* stream);
/* The y and x truncated DFTs of a layer in one launch, one CTA per (batch x
 * channel, kz) slice.  inverse = 0: in = Vz (BW, X, Y, m), mx = the x matrix
 * (X, 2m), my = the y matrix (Y, 2m), out = V (BW, 2m, 2m, m); inverse = 1:
 * in = U (BW, 2m, 2m, m), mx = (2m, X), my = (2m, Y), out = Uxy (BW, X, Y, m).
 * Equals em3d_fno_contract along y then x (inverse: x then y) up to FP32
 * rounding.  EM3D_ERR_UNSUPPORTED when a slice does not fit in shared memory. */
/* Bounded waits of the tcgen05 row pass that gave up since the last reset (the
 * outputs of those launches are invalid); reset = 1 clears the count.  Reads a
 * device counter (synchronous); -1 when it cannot be read. */
int em3d_fno_failures(int reset);
int em3d_fno_spectral(int inverse, int BW, int m, int X, int Y, const void* in, const void* mx, const void* my,
                      void* out, void* stream);
int em3d_fno_modemix(int act, int B, int W, int nm, const void* V, const void* Wre, const void* Wim, void* U,
                     void* stream);
int em3d_fno_modemix_bwd(int act, int B, int W, int nm, const void* V, const void* dU, const void* Wre,
                         const void* Wim, void* dV, float* dWre, float* dWim, void* stream);
int em3d_fno_layer_out(int act, int B, int W, int X, int Y, int Z, int m, const void* vin, const void* Uxy,
                       const void* A, const float* a, int apply_gelu, void* pre, void* vout, void* stream);
int em3d_fno_layer_out_bwd(int act, int B, int W, int X, int Y, int Z, int m, const float* gout, const void* pre,
                           const void* A, int apply_gelu, float* gpre, float* gin, void* dUxy, void* stream);
int em3d_fno_pointwise_wgrad(int act, int B, size_t ncell, int W, const float* gpre, const void* v, float* dA,
                             float* da, void* stream);
int em3d_fno_project(int act, int B, size_t ncell, int W, const void* v, const void* Q, const float* qb,
                     const void* wave, void* u, void* stream);
int em3d_fno_project_bwd(int act, int B, size_t ncell, int W, const void* v, const void* Q, const void* du,
                         float* gv, float* dQ, float* dqb, void* stream);
int em3d_fno_loss(int B, size_t n, const void* pred, const void* target, double* terms, void* grad, void* stream);
int em3d_fno_adam(int act, size_t n, float* w, const float* g, float* m1, float* m2, float lr, float b1, float b2,
                  float eps, int step, void* wact, void* stream);
/* Fused forward z-row pass (Z <= 128, W <= 32, modes <= 16; EM3D_ERR_UNSUPPORTED
 * otherwise): lift (lift = 1: o = P feat + pb from chi, wave) or one Fourier
 * layer (o = act(A vin + a + Re IDFT_z(Uxy))), writing any of: pre (pre_out),
 * o (vout), the truncated z-DFT of o (Vz, (B,W,X,Y,m) complex) and the
 * projection u = wave + Q o + qb (u_out).  NULL outputs are skipped. */
int em3d_fno_row_forward(int act, int lift, int B, int W, int X, int Y, int Z, int m, const void* chi,
                         const void* wave, const void* vin, const void* Uxy, const void* Wt, const float* bias,
                         int apply_gelu, void* pre_out, void* vout, void* Vz, const void* Q, const float* qb,
                         void* u_out, void* stream);
/* Half-resolution evaluation of the network on an even grid: 2x2x2 cell
 * means of (C, 2nx, 2ny, 2nz) fields (complex64 or complex128) into complex64
 * (C, nx, ny, nz), and trilinear interpolation back between cell centres
 * (clamped at the faces) into complex64 or complex128 (C, 2nx, 2ny, 2nz).
 * No reference counterpart (the network is not part of the reference). */
int em3d_fno_downsample2(int in_dtype, int C, int nx, int ny, int nz, const void* in, void* out, void* stream);
int em3d_fno_upsample2(int out_dtype, int C, int nx, int ny, int nz, const void* in, void* out, void* stream);
int em3d_fno_cast(int act, size_t n, const float* src, void* dst, void* stream);
int em3d_fno_uncast(int act, size_t n, const void* src, float* dst, void* stream);

/* ------------------------------------------------------------------------
 * Input builders on the device.
 *
 * em3d_sample_ellipsoids: a scene of `count` ellipsoids sampled at cell
 * centres; replaces the host-side center_mask + sample_contrast_tensor
 * (src/em3d/geometry.py:67-93, 203-252) and eta_sphere / eta_ellipsoid
 * (src/em3d/acoustics/materials.py:44-83), extended to rotated ellipsoids and
 * to several shapes painted in order (the last shape containing a cell wins).
 *   x, y, z    DEVICE float64 cell-centre coordinates (nx, ny, nz values)
 *   shapes     DEVICE float64 array, EM3D_SHAPE_DOUBLES per shape: centre[3],
 *              radii[3], R[9] (row-major; columns = body axes, r = c + R p),
 *              eps[18] (3x3 complex row-major, re/im interleaved; acoustic
 *              uses eps[0][0] as eta)
 *   tol        inside <=> sum (p_i / a_i)^2 <= 1 + tol (the reference EM
 *              builder uses 64 eps_f64 max(1, |L|); the acoustic ones 0)
 *   background HOST float64: 18 values (EM eps tensor) or 2 (acoustic eta)
 *   out        EM: chi = eps - I (3,3,Nx,Ny,Nz); acoustic: eta (Nx,Ny,Nz)
 * em3d_plane_wave: amplitude[c] exp(i sign (k orient.r + phi0)), (3,Nx,Ny,Nz);
 * replaces flat_wave_vec (src/em3d/wave.py:9-37).  orient (3) and amplitude
 * (3 complex = 6 doubles) are HOST arrays.
 * ------------------------------------------------------------------------ */
/* ------------------------------------------------------------------------
 * Far field.
 *
 * em3d_em_farfield: F[m][c] = dv sum_q (chi u)_c(q) exp(-i k0 dirs[m] . r_q)
 * (replaces scatter_integral_direct, src/em3d/farfield/_core.py:8-71);
 * em3d_acoustic_farfield: F[m] = k0^2 dv / (4 pi) sum_q chi(q) u(q)
 * exp(-i k0 dirs[m] . r_q) (replaces farfield_amplitude,
 * src/em3d/acoustics/farfield.py:29-60).  chi and u are the operator's device
 * arrays (EM3D_C64 or EM3D_C128); x, y, z the DEVICE float64 cell-centre
 * coordinates; dirs a DEVICE float64 (M, 3) array used as given (the callers
 * normalise where the reference does); F a DEVICE complex128 (M, 3) / (M,)
 * output.  Phases and sums are FP64.  Workspace: em3d_farfield_workspace_bytes.
 * ------------------------------------------------------------------------ */
size_t em3d_farfield_workspace_bytes(const em3d_grid* g, int M);
int em3d_em_farfield(const em3d_grid* g, int dtype, const void* chi, const void* u, const double* x, const double* y,
                     const double* z, double k0, double dv, int M, const double* dirs, void* F, void* workspace,
                     size_t workspace_bytes, void* stream);
int em3d_acoustic_farfield(const em3d_grid* g, int dtype, const void* chi, const void* u, const double* x,
                           const double* y, const double* z, double k0, double dv, int M, const double* dirs, void* F,
                           void* workspace, size_t workspace_bytes, void* stream);

#define EM3D_SHAPE_DOUBLES 33
int em3d_sample_ellipsoids(int kind, int dtype, int nx, int ny, int nz, const double* x, const double* y,
                           const double* z, int count, const double* shapes, double tol, const double* background,
                           void* out, void* stream);
int em3d_plane_wave(int dtype, int nx, int ny, int nz, const double* x, const double* y, const double* z, double k,
                    const double* orient, const double* amplitude, double phi0, int sign, void* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* EM3D_B200_H */
