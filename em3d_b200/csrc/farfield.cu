// Far-field scatter integrals (reference src/em3d/farfield/_core.py:8-71 and
// src/em3d/acoustics/farfield.py:29-60):
//
//   EM:        F[m][c] = scale * sum_q (chi u)_c(q) exp(-i k0 e_m . r_q),  c = 0..2
//   acoustic:  F[m]    = scale * sum_q  chi(q) u(q) exp(-i k0 e_m . r_q)
//
// with scale = dV (EM) or k0^2 dV / (4 pi) (acoustic).  The phase factorises
// over the axes, exp(-i k0 e.r) = tx[m][x] ty[m][y] tz[m][z], so one pass
// reads the source once: a CTA stages the source of RB consecutive (x, y) rows
// in shared memory, contracts it along z with tz for every direction, applies
// tx ty, sums its rows and adds the per-direction totals into F with FP64
// atomics.  Everything after the field load is FP64.
#include <math.h>

#include "common.cuh"

namespace em3d {
namespace ff {

constexpr int kThreads = 256;
constexpr int kCells = 1024;   // RB * Nz cells staged per CTA

// t[m][i] = exp(-i k0 dir[m][axis] coord[i]) for the three axes, laid out as
// tx (M x Nx), ty (M x Ny), tz (M x Nz) back to back.
__global__ void k_tables(int M, int nx, int ny, int nz, const double* __restrict__ x, const double* __restrict__ y,
                         const double* __restrict__ z, const double* __restrict__ dirs, double k0, double2* tab) {
  const int per = nx + ny + nz;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M * per; i += gridDim.x * blockDim.x) {
    const int m = i / per, j = i - m * per;
    int axis, idx;
    double c;
    if (j < nx) { axis = 0; idx = j; c = x[idx]; }
    else if (j < nx + ny) { axis = 1; idx = j - nx; c = y[idx]; }
    else { axis = 2; idx = j - nx - ny; c = z[idx]; }
    double s, co;
    sincos(-k0 * dirs[3 * m + axis] * c, &s, &co);
    double2* out = tab + (axis == 0 ? (size_t)m * nx + idx
                          : axis == 1 ? (size_t)M * nx + (size_t)m * ny + idx
                                      : (size_t)M * (nx + ny) + (size_t)m * nz + idx);
    *out = make_double2(co, s);
  }
}

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// C = 3: EM (chi 3x3, u 3 components); C = 1: acoustic (chi, u scalar).
template <typename R, int C>
__global__ void __launch_bounds__(kThreads) k_farfield(int nx, int ny, int nz, int rb, const cx<R>* __restrict__ chi,
                                                       const cx<R>* __restrict__ u, int M,
                                                       const double2* __restrict__ tab, double scale,
                                                       double2* __restrict__ F) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* J = reinterpret_cast<double2*>(smem_raw);          // [z][row][c]
  double2* acc = J + (size_t)kCells * C;                        // [m][c]
  const size_t ncell = (size_t)nx * ny * nz;
  const int nrows = nx * ny;
  const int row0 = blockIdx.x * rb;
  const int rows = min(rb, nrows - row0);
  for (int i = threadIdx.x; i < M * C; i += blockDim.x) acc[i] = make_double2(0.0, 0.0);
  // source of the CTA's rows, J[z][r][c]
  for (int i = threadIdx.x; i < rows * nz; i += blockDim.x) {
    const int r = i / nz, zz = i - r * nz;
    const size_t cell = (size_t)(row0 + r) * nz + zz;
    if (C == 3) {
      double2 uu[3];
#pragma unroll
      for (int b = 0; b < 3; ++b) uu[b] = to_c64(u[(size_t)b * ncell + cell]);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double2 s = make_double2(0.0, 0.0);
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          const double2 e = to_c64(chi[(size_t)(c * 3 + b) * ncell + cell]);
          const double2 p = zmul(e, uu[b]);
          s.x += p.x;
          s.y += p.y;
        }
        J[((size_t)zz * rb + r) * C + c] = s;
      }
    } else {
      J[(size_t)zz * rb + r] = zmul(to_c64(chi[cell]), to_c64(u[cell]));
    }
  }
  __syncthreads();
  const double2* tx = tab;
  const double2* ty = tab + (size_t)M * nx;
  const double2* tz = tab + (size_t)M * (nx + ny);
  const int work = M * rows * C;
  for (int o = threadIdx.x; o < work; o += blockDim.x) {
    const int c = o % C;
    const int r = (o / C) % rows;
    const int m = o / (C * rows);
    const double2* tzm = tz + (size_t)m * nz;
    double sr = 0.0, si = 0.0;
    for (int zz = 0; zz < nz; ++zz) {
      const double2 j = J[((size_t)zz * rb + r) * C + c];
      const double2 t = __ldg(tzm + zz);
      sr += j.x * t.x - j.y * t.y;
      si += j.x * t.y + j.y * t.x;
    }
    const int row = row0 + r;
    const int xi = row / ny, yi = row - xi * ny;
    const double2 v = zmul(zmul(make_double2(sr, si), __ldg(tx + (size_t)m * nx + xi)), __ldg(ty + (size_t)m * ny + yi));
    atomicAdd(&acc[m * C + c].x, v.x);
    atomicAdd(&acc[m * C + c].y, v.y);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < M * C; i += blockDim.x) {
    atomicAdd(&F[i].x, scale * acc[i].x);
    atomicAdd(&F[i].y, scale * acc[i].y);
  }
}

}  // namespace ff
}  // namespace em3d

using namespace em3d;

namespace {

constexpr int kMaxDirsPerLaunch = 1024;

size_t tables_bytes(const em3d_grid* g, int M) {
  return sizeof(double2) * (size_t)M * ((size_t)g->nx + g->ny + g->nz);
}

template <typename R, int C>
int farfield_impl(const em3d_grid* g, const void* chi, const void* u, const double* x, const double* y,
                  const double* z, double k0, double scale, int M, const double* dirs, void* F, void* ws,
                  size_t ws_bytes, cudaStream_t st) {
  const int nz = g->nz;
  const int rb = nz >= ff::kCells ? 1 : ff::kCells / nz;
  const int nrows = g->nx * g->ny;
  EM3D_CUDA_TRY(cudaMemsetAsync(F, 0, sizeof(double2) * (size_t)M * C, st));
  double2* tab = (double2*)ws;
  for (int m0 = 0; m0 < M; m0 += kMaxDirsPerLaunch) {
    const int mb = M - m0 < kMaxDirsPerLaunch ? M - m0 : kMaxDirsPerLaunch;
    const int per = g->nx + g->ny + g->nz;
    const int tb = (int)(((size_t)mb * per + 255) / 256);
    ff::k_tables<<<tb < 4096 ? tb : 4096, 256, 0, st>>>(mb, g->nx, g->ny, g->nz, x, y, z, dirs + 3 * (size_t)m0, k0,
                                                        tab);
    EM3D_LAUNCH_CHECK();
    const size_t smem = sizeof(double2) * ((size_t)ff::kCells * C + (size_t)mb * C);
    auto kern = ff::k_farfield<R, C>;
    EM3D_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(nrows + rb - 1) / rb, ff::kThreads, smem, st>>>(g->nx, g->ny, nz, rb, (const cx<R>*)chi,
                                                          (const cx<R>*)u, mb, tab, scale,
                                                          (double2*)F + (size_t)m0 * C);
    EM3D_LAUNCH_CHECK();
  }
  (void)ws_bytes;
  return EM3D_OK;
}

int check_ff(const em3d_grid* g, int dtype, int M, const void* chi, const void* u, const double* x, const double* y,
             const double* z, const double* dirs, const void* F, const void* ws, size_t ws_bytes) {
  if (!g || g->nx < 1 || g->ny < 1 || g->nz < 1) { em3d_set_last_error("farfield: bad grid"); return EM3D_ERR_INVALID; }
  if (g->nz > ff::kCells) { em3d_set_last_error("farfield: Nz must be <= 1024"); return EM3D_ERR_UNSUPPORTED; }
  if (dtype != EM3D_C64 && dtype != EM3D_C128) { em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128"); return EM3D_ERR_INVALID; }
  if (M < 1) { em3d_set_last_error("farfield: need at least one direction"); return EM3D_ERR_INVALID; }
  if (!chi || !u || !x || !y || !z || !dirs || !F || !ws) { em3d_set_last_error("farfield: NULL pointer"); return EM3D_ERR_INVALID; }
  const int mb = M < kMaxDirsPerLaunch ? M : kMaxDirsPerLaunch;
  if (ws_bytes < tables_bytes(g, mb)) { em3d_set_last_error("farfield: workspace too small"); return EM3D_ERR_INVALID; }
  return EM3D_OK;
}

}  // namespace

extern "C" {

size_t em3d_farfield_workspace_bytes(const em3d_grid* g, int M) {
  if (!g || g->nx < 1 || g->ny < 1 || g->nz < 1 || M < 1) return 0;
  return tables_bytes(g, M < kMaxDirsPerLaunch ? M : kMaxDirsPerLaunch);
}

int em3d_em_farfield(const em3d_grid* g, int dtype, const void* chi, const void* u, const double* x, const double* y,
                     const double* z, double k0, double dv, int M, const double* dirs, void* F, void* workspace,
                     size_t workspace_bytes, void* stream) {
  if (int rc = check_ff(g, dtype, M, chi, u, x, y, z, dirs, F, workspace, workspace_bytes)) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == EM3D_C64)
    return farfield_impl<float, 3>(g, chi, u, x, y, z, k0, dv, M, dirs, F, workspace, workspace_bytes, st);
  return farfield_impl<double, 3>(g, chi, u, x, y, z, k0, dv, M, dirs, F, workspace, workspace_bytes, st);
}

int em3d_acoustic_farfield(const em3d_grid* g, int dtype, const void* chi, const void* u, const double* x,
                           const double* y, const double* z, double k0, double dv, int M, const double* dirs, void* F,
                           void* workspace, size_t workspace_bytes, void* stream) {
  if (int rc = check_ff(g, dtype, M, chi, u, x, y, z, dirs, F, workspace, workspace_bytes)) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const double scale = k0 * k0 * dv / (4.0 * M_PI);
  if (dtype == EM3D_C64)
    return farfield_impl<float, 1>(g, chi, u, x, y, z, k0, scale, M, dirs, F, workspace, workspace_bytes, st);
  return farfield_impl<double, 1>(g, chi, u, x, y, z, k0, scale, M, dirs, F, workspace, workspace_bytes, st);
}

}  // extern "C"
