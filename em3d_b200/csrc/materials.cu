// Device-side input builders: contrast of a scene of (rotated) ellipsoids
// sampled at cell centres, and plane-wave incident fields.
//
// Cell-centre test (reference src/em3d/geometry.py:67-93, center_mask):
//   d = r - c,  p = R^T d  (R's columns are the body axes in world
//   coordinates, so r = c + R p),  inside  <=>  sum_i (p_i / a_i)^2 <= 1 + tol.
// Every product, quotient and sum is rounded explicitly (no contraction into
// FMAs) in a fixed order, so the mask equals the float64 NumPy restatement bit
// for bit; with R = I it is the reference's own axis-aligned test.  Shapes are
// painted in order: a cell inside several takes the last one's material.
//
// EM output (3, 3, Nx, Ny, Nz): chi = eps - I with eps the shape's 3x3 tensor
// (the background tensor outside every shape), rounded as
// sample_contrast_tensor does it (src/em3d/geometry.py:203-252): eps =
// bg + (feature - bg) in float64, cast to the output type, minus I there.
// Acoustic output (Nx, Ny, Nz): the material value eta itself (the shape's
// eps[0][0], background outside), as the eta_sphere / eta_ellipsoid builders
// (src/em3d/acoustics/materials.py:44-83; those use tol = 0).
#include <math.h>

#include "common.cuh"

namespace em3d {
namespace mat {

constexpr int kShape = EM3D_SHAPE_DOUBLES;  // c[3] a[3] R[9] eps[18]

struct Background {
  double v[18];
};

__device__ __forceinline__ bool inside(const double* __restrict__ s, double x, double y, double z, double lim) {
  const double d0 = __dsub_rn(x, __ldg(s + 0));
  const double d1 = __dsub_rn(y, __ldg(s + 1));
  const double d2 = __dsub_rn(z, __ldg(s + 2));
  double acc = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const double p = __dadd_rn(__dadd_rn(__dmul_rn(__ldg(s + 6 + i), d0), __dmul_rn(__ldg(s + 9 + i), d1)),
                               __dmul_rn(__ldg(s + 12 + i), d2));
    const double q = __ddiv_rn(p, __ldg(s + 3 + i));
    acc = __dadd_rn(acc, __dmul_rn(q, q));
  }
  return acc <= lim;
}

template <typename R>
__global__ void k_sample(int kind, int nx, int ny, int nz, const double* __restrict__ xs, const double* __restrict__ ys,
                         const double* __restrict__ zs, int count, const double* __restrict__ shapes, double lim,
                         Background bg, cx<R>* __restrict__ out) {
  const size_t ncell = (size_t)nx * ny * nz;
  for (size_t cell = blockIdx.x * (size_t)blockDim.x + threadIdx.x; cell < ncell;
       cell += (size_t)gridDim.x * blockDim.x) {
    const int iz = (int)(cell % nz);
    const int iy = (int)((cell / nz) % ny);
    const int ix = (int)(cell / ((size_t)nz * ny));
    const double x = xs[ix], y = ys[iy], z = zs[iz];
    int hit = -1;
    for (int s = 0; s < count; ++s)
      if (inside(shapes + (size_t)s * kShape, x, y, z, lim)) hit = s;
    const double* e = hit >= 0 ? shapes + (size_t)hit * kShape + 15 : nullptr;
    if (kind == EM3D_ACOUSTIC) {
      const double re = e ? __ldg(e) : bg.v[0], im = e ? __ldg(e + 1) : bg.v[1];
      out[cell] = mk<R>((R)re, (R)im);
    } else {
      // eps = bg + (feature - bg) in float64, stored in R, then minus I in R
#pragma unroll
      for (int ab = 0; ab < 9; ++ab) {
        const double br = bg.v[2 * ab], bi = bg.v[2 * ab + 1];
        const double er = e ? __dadd_rn(br, __dsub_rn(__ldg(e + 2 * ab), br)) : br;
        const double ei = e ? __dadd_rn(bi, __dsub_rn(__ldg(e + 2 * ab + 1), bi)) : bi;
        R re = (R)er;
        if (ab == 0 || ab == 4 || ab == 8) re = re - (R)1;
        out[(size_t)ab * ncell + cell] = mk<R>(re, (R)ei);
      }
    }
  }
}

// out[c] = amplitude[c] * exp(i sign (k (o0 x + o1 y + o2 z) + phi0))
// (reference src/em3d/wave.py:9-37, flat_wave_vec)
template <typename R>
__global__ void k_plane_wave(int nx, int ny, int nz, const double* __restrict__ xs, const double* __restrict__ ys,
                             const double* __restrict__ zs, double k, double o0, double o1, double o2, double a0r,
                             double a0i, double a1r, double a1i, double a2r, double a2i, double phi0, int sign,
                             cx<R>* __restrict__ out) {
  const size_t ncell = (size_t)nx * ny * nz;
  for (size_t cell = blockIdx.x * (size_t)blockDim.x + threadIdx.x; cell < ncell;
       cell += (size_t)gridDim.x * blockDim.x) {
    const int iz = (int)(cell % nz);
    const int iy = (int)((cell / nz) % ny);
    const int ix = (int)(cell / ((size_t)nz * ny));
    const double dot = __dadd_rn(__dadd_rn(__dmul_rn(o0, xs[ix]), __dmul_rn(o1, ys[iy])), __dmul_rn(o2, zs[iz]));
    const double ph = sign * __dadd_rn(__dmul_rn(k, dot), phi0);
    double sn, cs;
    sincos(ph, &sn, &cs);
    out[cell] = mk<R>((R)(a0r * cs - a0i * sn), (R)(a0r * sn + a0i * cs));
    out[ncell + cell] = mk<R>((R)(a1r * cs - a1i * sn), (R)(a1r * sn + a1i * cs));
    out[2 * ncell + cell] = mk<R>((R)(a2r * cs - a2i * sn), (R)(a2r * sn + a2i * cs));
  }
}

inline int grid_blocks(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)(b > 148 * 16 ? 148 * 16 : (b == 0 ? 1 : b));
}

}  // namespace mat
}  // namespace em3d

using namespace em3d;

extern "C" {

int em3d_sample_ellipsoids(int kind, int dtype, int nx, int ny, int nz, const double* x, const double* y,
                           const double* z, int count, const double* shapes, double tol, const double* background,
                           void* out, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || !x || !y || !z || !out || !background) {
    em3d_set_last_error("sample_ellipsoids: bad grid or NULL pointer");
    return EM3D_ERR_INVALID;
  }
  if (count < 0 || (count > 0 && !shapes)) {
    em3d_set_last_error("sample_ellipsoids: count must be >= 0 and shapes non-NULL");
    return EM3D_ERR_INVALID;
  }
  if (kind != EM3D_EM && kind != EM3D_ACOUSTIC) {
    em3d_set_last_error("sample_ellipsoids: kind must be EM3D_EM or EM3D_ACOUSTIC");
    return EM3D_ERR_INVALID;
  }
  mat::Background bg;
  const int nb = kind == EM3D_EM ? 18 : 2;
  for (int i = 0; i < 18; ++i) bg.v[i] = i < nb ? background[i] : 0.0;
  const double lim = 1.0 + tol;
  const size_t n = (size_t)nx * ny * nz;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == EM3D_C64)
    mat::k_sample<float><<<mat::grid_blocks(n), 256, 0, st>>>(kind, nx, ny, nz, x, y, z, count, shapes, lim, bg,
                                                               (float2*)out);
  else if (dtype == EM3D_C128)
    mat::k_sample<double><<<mat::grid_blocks(n), 256, 0, st>>>(kind, nx, ny, nz, x, y, z, count, shapes, lim, bg,
                                                                (double2*)out);
  else {
    em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128");
    return EM3D_ERR_INVALID;
  }
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_plane_wave(int dtype, int nx, int ny, int nz, const double* x, const double* y, const double* z, double k,
                    const double* orient, const double* amplitude, double phi0, int sign, void* out, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || !x || !y || !z || !out || !orient || !amplitude) {
    em3d_set_last_error("plane_wave: bad grid or NULL pointer");
    return EM3D_ERR_INVALID;
  }
  if (sign != 1 && sign != -1) {
    em3d_set_last_error("plane_wave: sign must be 1 or -1");
    return EM3D_ERR_INVALID;
  }
  const size_t n = (size_t)nx * ny * nz;
  cudaStream_t st = (cudaStream_t)stream;
  const double* a = amplitude;
  if (dtype == EM3D_C64)
    mat::k_plane_wave<float><<<mat::grid_blocks(n), 256, 0, st>>>(nx, ny, nz, x, y, z, k, orient[0], orient[1],
                                                                   orient[2], a[0], a[1], a[2], a[3], a[4], a[5],
                                                                   phi0, sign, (float2*)out);
  else if (dtype == EM3D_C128)
    mat::k_plane_wave<double><<<mat::grid_blocks(n), 256, 0, st>>>(nx, ny, nz, x, y, z, k, orient[0], orient[1],
                                                                    orient[2], a[0], a[1], a[2], a[3], a[4], a[5],
                                                                    phi0, sign, (double2*)out);
  else {
    em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128");
    return EM3D_ERR_INVALID;
  }
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

}  // extern "C"
