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
//
// This header holds the passes and their dispatch (`apply`); its
// instantiations are compiled in apply_*.cu (one translation unit per
// precision and operator kind, built in parallel).
#pragma once

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <string>
#include <unordered_set>
#include "common.cuh"
#include "fft.cuh"
#include "passes_fast.cuh"
#include "passes_x.cuh"

namespace em3d {

constexpr int kThreads = 256;
constexpr size_t kAlign = 256;

static inline size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }
__host__ __device__ inline int odd_stride(int P) { return (P & 1) ? P : P + 1; }

// ---------------------------------------------------------------------------
// layouts
// ---------------------------------------------------------------------------

struct Dims {
  int nx, ny, nz;
  size_t cells() const { return (size_t)nx * ny * nz; }
  size_t doubled() const { return (size_t)8 * cells(); }
  size_t octant() const { return (size_t)(nx + 1) * (ny + 1) * (nz + 1); }
};

template <typename R> struct SpecLayout {
  size_t oct_elems, blocks, tw_off, total_bytes;
  SpecLayout(const Dims& d, int kind) {
    blocks = (kind == EM3D_EM) ? 6 : 1;
    oct_elems = d.octant();
    tw_off = align_up(blocks * oct_elems * sizeof(cx<R>));
    total_bytes = tw_off + align_up((size_t)2 * (d.nx + d.ny + d.nz) * sizeof(cx<R>));
  }
  cx<R>* oct(void* base) const { return (cx<R>*)base; }
  cx<R>* twx(void* base, const Dims& d) const { return (cx<R>*)((char*)base + tw_off); }
  cx<R>* twy(void* base, const Dims& d) const { return twx(base, d) + 2 * d.nx; }
  cx<R>* twz(void* base, const Dims& d) const { return twy(base, d) + 2 * d.ny; }
};

static size_t build_ws_bytes(const Dims& d) {
  return align_up(d.doubled() * sizeof(double2)) + align_up((size_t)2 * (d.nx + d.ny + d.nz) * sizeof(double2));
}

// Apply workspace: T1, T2, then 256 bytes of status words (word 0 counts the
// bounded waits that gave up; zero the workspace once after allocating it).
constexpr size_t kStatusBytes = 256;
template <typename R> static size_t apply_status_offset(const Dims& d, int C, int batch) {
  size_t t1 = (size_t)batch * C * d.nx * d.ny * 2 * d.nz;
  size_t t2 = (size_t)batch * C * d.nx * 2 * d.ny * 2 * d.nz;
  return align_up(t1 * sizeof(cx<R>)) + align_up(t2 * sizeof(cx<R>));
}
template <typename R> static size_t apply_ws_bytes(const Dims& d, int C, int batch) {
  return apply_status_offset<R>(d, C, batch) + kStatusBytes;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

template <typename R> __global__ void k_twiddles(cx<R>* tw, int L) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < L) {
    double s, c;
    sincospi(2.0 * (double)m / (double)L, &s, &c);
    tw[m] = from_c64<R>(make_double2(c, -s));  // e^{-2 pi i m / L}
  }
}

template <typename C> __device__ __forceinline__ void load_twiddles(C* tws, const C* __restrict__ twg, int L) {
  for (int i = threadIdx.x; i < L; i += blockDim.x) tws[i] = twg[i];
}

// Load / store modes of the generic row pass (see FLD_* / FST_* in passes_fast.cuh).
enum { LD_PLAIN = 0, LD_EM_CHI = 1, LD_AC_CHI = 2, LD_EM_CHI6 = 3, LD_EM_CHI1 = 4 };
enum { ST_PLAIN = 0, ST_SUB = 1, ST_EM_ADJ = 2, ST_AC_ADJ = 3, ST_EM_ADJ6 = 4, ST_EM_ADJ1 = 5 };

// Rows along the contiguous axis.  Row g of batch b, component c lives at
// ((b*C + c) * rows_pb + row) * len.
template <typename R, int C, int LD, int ST, bool INV>
__global__ void __launch_bounds__(kThreads) k_rows(const cx<R>* in, const cx<R>* __restrict__ chi,
                                                   const cx<R>* base, cx<R>* out,
                                                   const cx<R>* __restrict__ twg, AxisPlan pl, int rows_pb,
                                                   int nrows, int Lin, int Lout, int RPB, BatchStrides bs,
                                                   const int* skip) {
  using T = cx<R>;
  if (skip_launch(skip)) return;
  // stop flags of the (usually one or two) entries this CTA's rows belong to, read once
  const int gb0 = blockIdx.x * RPB, gb1 = min(gb0 + RPB, nrows) - 1;
  const int eb0 = gb0 / rows_pb, eb1 = gb1 / rows_pb;
  const bool d0 = entry_done(bs, eb0), d1 = entry_done(bs, eb1);
  if (d0 && d1 && eb1 - eb0 <= 1) return;
  auto row_done = [&](int g) {
    const int bb = g / rows_pb;
    return bb == eb0 ? d0 : (bb == eb1 ? d1 : entry_done(bs, bb));
  };
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int L = pl.L;
  const int P = C * RPB, S = odd_stride(P);
  T* A = reinterpret_cast<T*>(smem_raw);
  T* Bf = A + (size_t)L * S;
  T* tw = Bf + (size_t)L * S;
  load_twiddles(tw, twg, L);
  const int g0 = blockIdx.x * RPB;

  for (int e = threadIdx.x; e < RPB * Lin; e += blockDim.x) {
    const int rl = e / Lin, k = e - rl * Lin;
    const int g = g0 + rl;
    T v[C];
#pragma unroll
    for (int c = 0; c < C; ++c) v[c] = mk<R>(0, 0);
    if (g < nrows && !row_done(g)) {
      const int b = g / rows_pb, row = g - b * rows_pb;
      if constexpr (LD == LD_EM_CHI || LD == LD_EM_CHI6) {
        T uu[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) uu[c] = in[((size_t)(b * 3 + c) * rows_pb + row) * Lin + k];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          T acc = mk<R>(0, 0);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int ci = LD == LD_EM_CHI ? a * 3 + c : sym_index(a, c);
            acc = cadd(acc, cmul((chi + (size_t)b * bs.chi)[((size_t)ci * rows_pb + row) * Lin + k], uu[c]));
          }
          v[a] = acc;
        }
      } else if constexpr (LD == LD_EM_CHI1) {
        const T s = (chi + (size_t)b * bs.chi)[(size_t)row * Lin + k];
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = cmul(s, in[((size_t)(b * 3 + c) * rows_pb + row) * Lin + k]);
      } else if constexpr (LD == LD_AC_CHI) {
        v[0] = cmul((chi + (size_t)b * bs.chi)[(size_t)row * Lin + k], in[((size_t)b * rows_pb + row) * Lin + k]);
      } else {
#pragma unroll
        for (int c = 0; c < C; ++c) v[c] = in[((size_t)(b * C + c) * rows_pb + row) * Lin + k];
      }
    }
#pragma unroll
    for (int c = 0; c < C; ++c) A[(size_t)k * S + c * RPB + rl] = v[c];
  }
  for (int e = threadIdx.x; e < (L - Lin) * P; e += blockDim.x) {
    const int k = Lin + e / P, p = e % P;
    A[(size_t)k * S + p] = mk<R>(0, 0);
  }
  __syncthreads();
  T* Rs = smem_fft<INV>(A, Bf, tw, pl, P, S);

  for (int e = threadIdx.x; e < RPB * Lout; e += blockDim.x) {
    const int rl = e / Lout, k = e - rl * Lout;
    const int g = g0 + rl;
    if (g >= nrows || row_done(g)) continue;
    const int b = g / rows_pb, row = g - b * rows_pb;
    T y[C];
#pragma unroll
    for (int c = 0; c < C; ++c) y[c] = Rs[(size_t)k * S + c * RPB + rl];
    if constexpr (ST == ST_PLAIN) {
#pragma unroll
      for (int c = 0; c < C; ++c) out[((size_t)(b * C + c) * rows_pb + row) * Lout + k] = y[c];
    } else if constexpr (ST == ST_SUB) {
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const size_t o = ((size_t)(b * C + c) * rows_pb + row) * Lout + k;
        out[o] = csub(base[o], y[c]);
      }
    } else if constexpr (ST == ST_EM_ADJ || ST == ST_EM_ADJ6) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        T acc = mk<R>(0, 0);
#pragma unroll
        for (int c = 0; c < 3; ++c) {  // (chi^H)[a][c] = conj(chi[c][a])
          const int ci = ST == ST_EM_ADJ ? c * 3 + a : sym_index(c, a);
          acc = cadd(acc, cmulcj((chi + (size_t)b * bs.chi)[((size_t)ci * rows_pb + row) * Lout + k], y[c]));
        }
        const size_t o = ((size_t)(b * 3 + a) * rows_pb + row) * Lout + k;
        out[o] = csub(base[o], acc);
      }
    } else if constexpr (ST == ST_EM_ADJ1) {
      const T s = (chi + (size_t)b * bs.chi)[(size_t)row * Lout + k];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const size_t o = ((size_t)(b * 3 + a) * rows_pb + row) * Lout + k;
        out[o] = csub(base[o], cmulcj(s, y[a]));
      }
    } else if constexpr (ST == ST_AC_ADJ) {
      const size_t o = ((size_t)b * rows_pb + row) * Lout + k;
      out[o] = csub(base[o], cmulcj((chi + (size_t)b * bs.chi)[(size_t)row * Lout + k], y[0]));
    }
  }
}

// Pencils along a strided axis: in (outer, Lin, inner) -> out (outer, Lout, inner).
// A CTA takes P neighbouring inner indices of one outer index, so each row
// of the tile is a contiguous segment of global memory.
template <typename R, bool INV>
__global__ void __launch_bounds__(kThreads) k_strided(const cx<R>* in, cx<R>* out, const cx<R>* __restrict__ twg,
                                                      AxisPlan pl, int Lin, int Lout, int inner, int P, int ntiles,
                                                      BatchStrides bs, const int* skip) {
  using T = cx<R>;
  if (skip_launch(skip)) return;
  if (bs.done && entry_done(bs, (int)(blockIdx.x / ntiles) / bs.outer)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int L = pl.L;
  const int S = odd_stride(P);
  T* A = reinterpret_cast<T*>(smem_raw);
  T* Bf = A + (size_t)L * S;
  T* tw = Bf + (size_t)L * S;
  load_twiddles(tw, twg, L);
  const int o = blockIdx.x / ntiles;
  const int i0 = (blockIdx.x - o * ntiles) * P;
  const T* src = in + (size_t)o * Lin * inner;
  for (int e = threadIdx.x; e < Lin * P; e += blockDim.x) {
    const int k = e / P, pp = e - k * P;
    const int i = i0 + pp;
    A[(size_t)k * S + pp] = (i < inner) ? src[(size_t)k * inner + i] : mk<R>(0, 0);
  }
  for (int e = threadIdx.x; e < (L - Lin) * P; e += blockDim.x) {
    const int k = Lin + e / P, pp = e % P;
    A[(size_t)k * S + pp] = mk<R>(0, 0);
  }
  __syncthreads();
  T* Rs = smem_fft<INV>(A, Bf, tw, pl, P, S);
  T* dst = out + (size_t)o * Lout * inner;
  for (int e = threadIdx.x; e < Lout * P; e += blockDim.x) {
    const int k = e / P, pp = e - k * P;
    const int i = i0 + pp;
    if (i < inner) dst[(size_t)k * inner + i] = Rs[(size_t)k * S + pp];
  }
}

// Octant spectrum access: frequency kx in [0, 2Nx) folds to i = min(kx, 2Nx - kx);
// off-diagonal dyadic blocks are odd along their two axes, so they pick up
// the sign -1 per folded axis they are odd in.
__device__ __forceinline__ int fold(int k, int n) { return k <= n ? k : 2 * n - k; }
__device__ __forceinline__ int fsign(int k, int n) { return k <= n ? 1 : -1; }

// Pencils along x with the spectrum multiply between forward and inverse FFT.
template <typename R, int C, bool ADJ>
__global__ void __launch_bounds__(kThreads) k_xmul(cx<R>* T2, const cx<R>* __restrict__ spec,
                                                   const cx<R>* __restrict__ twg, AxisPlan pl, int Nx, int Ny,
                                                   int Nz, int Pz, int ntz, int nb, BatchStrides bs,
                                                   const int* skip) {
  using T = cx<R>;
  if (skip_launch(skip)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int L = pl.L;  // 2 Nx
  const int P = C * Pz, S = odd_stride(P);
  const int Ny2 = 2 * Ny, Nz2 = 2 * Nz;
  T* A = reinterpret_cast<T*>(smem_raw);
  T* Bf = A + (size_t)L * S;
  T* tw = Bf + (size_t)L * S;
  load_twiddles(tw, twg, L);
  int idx = blockIdx.x;
  const int b = idx % nb; idx /= nb;
  const int tile = idx % ntz;
  const int ky = idx / ntz;
  const int kz0 = tile * Pz;
  if (entry_done(bs, b)) return;
  spec += (size_t)b * bs.spec;
  const size_t xstride = (size_t)Ny2 * Nz2;

  for (int e = threadIdx.x; e < C * Nx * Pz; e += blockDim.x) {
    const int c = e / (Nx * Pz);
    const int r = e - c * Nx * Pz;
    const int x = r / Pz, zl = r - x * Pz;
    const int kz = kz0 + zl;
    T v = mk<R>(0, 0);
    if (kz < Nz2) v = T2[((size_t)(b * C + c) * Nx + x) * xstride + (size_t)ky * Nz2 + kz];
    A[(size_t)x * S + c * Pz + zl] = v;
  }
  for (int e = threadIdx.x; e < (L - Nx) * P; e += blockDim.x) {
    const int k = Nx + e / P, p = e % P;
    A[(size_t)k * S + p] = mk<R>(0, 0);
  }
  __syncthreads();
  T* Xs = smem_fft<false>(A, Bf, tw, pl, P, S);

  const size_t ostride = (size_t)(Nx + 1) * (Ny + 1) * (Nz + 1);
  const int j = fold(ky, Ny), sy = fsign(ky, Ny);
  for (int e = threadIdx.x; e < L * Pz; e += blockDim.x) {
    const int kx = e / Pz, zl = e - kx * Pz;
    const int kz = kz0 + zl;
    if (kz >= Nz2) continue;
    const int i = fold(kx, Nx), l = fold(kz, Nz);
    const size_t so = ((size_t)i * (Ny + 1) + j) * (Nz + 1) + l;
    T* px = Xs + (size_t)kx * S + zl;
    if constexpr (C == 1) {
      T kk = spec[so];
      px[0] = ADJ ? cmulcj(kk, px[0]) : cmul(kk, px[0]);
    } else {
      const int sx = fsign(kx, Nx), sz = fsign(kz, Nz);
      T kxx = spec[so], kyy = spec[ostride + so], kzz = spec[2 * ostride + so];
      T kxy = spec[3 * ostride + so], kxz = spec[4 * ostride + so], kyz = spec[5 * ostride + so];
      const R fxy = (R)(sx * sy), fxz = (R)(sx * sz), fyz = (R)(sy * sz);
      kxy = cscale(kxy, fxy); kxz = cscale(kxz, fxz); kyz = cscale(kyz, fyz);
      if (ADJ) { kxx = cconj(kxx); kyy = cconj(kyy); kzz = cconj(kzz); kxy = cconj(kxy); kxz = cconj(kxz); kyz = cconj(kyz); }
      const T X0 = px[0], X1 = px[Pz], X2 = px[2 * Pz];
      px[0] = cadd(cadd(cmul(kxx, X0), cmul(kxy, X1)), cmul(kxz, X2));
      px[Pz] = cadd(cadd(cmul(kxy, X0), cmul(kyy, X1)), cmul(kyz, X2));
      px[2 * Pz] = cadd(cadd(cmul(kxz, X0), cmul(kyz, X1)), cmul(kzz, X2));
    }
  }
  __syncthreads();
  T* other = (Xs == A) ? Bf : A;
  T* Ys = smem_fft<true>(Xs, other, tw, pl, P, S);

  for (int e = threadIdx.x; e < C * Nx * Pz; e += blockDim.x) {
    const int c = e / (Nx * Pz);
    const int r = e - c * Nx * Pz;
    const int x = r / Pz, zl = r - x * Pz;
    const int kz = kz0 + zl;
    if (kz < Nz2) T2[((size_t)(b * C + c) * Nx + x) * xstride + (size_t)ky * Nz2 + kz] = Ys[(size_t)x * S + c * Pz + zl];
  }
}

// ---- spectrum construction (FP64) ----------------------------------------

// Signed offset of doubled-grid index i: i*d for i < n, -(2n - i)*d otherwise
// (src/em3d/operator.py:16-25).
__device__ __forceinline__ double offset_of(int i, int n, double d) {
  return i < n ? (double)i * d : -((double)(2 * n - i) * d);
}

// One dyadic block (r, c) of the EM kernel on the doubled grid
// (src/em3d/operator.py:28-84).  `crop_eq` zeroes the index-N plane along the
// axes an off-diagonal block is odd in: those samples never reach the cropped
// output, and without them each block is exactly even/odd per axis.
static __global__ void k_em_sample(double2* out, int r, int c, int Nx, int Ny, int Nz, double dx, double dy, double dz,
                            double k, double dv, int crop_eq, int conj) {
  const size_t n = (size_t)8 * Nx * Ny * Nz;
  const int Ny2 = 2 * Ny, Nz2 = 2 * Nz;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int l = (int)(t % Nz2);
    const int j = (int)((t / Nz2) % Ny2);
    const int i = (int)(t / ((size_t)Nz2 * Ny2));
    const double s[3] = {offset_of(i, Nx, dx), offset_of(j, Ny, dy), offset_of(l, Nz, dz)};
    const int idx[3] = {i, j, l};
    const int nn[3] = {Nx, Ny, Nz};
    const double r2 = (s[0] * s[0] + s[1] * s[1]) + s[2] * s[2];
    double rad = sqrt(r2);
    double2 v;
    if (rad < 1e-15) {
      v = make_double2(r == c ? -1.0 / 3.0 : 0.0, 0.0);
    } else if (r != c && crop_eq && (idx[r] == nn[r] || idx[c] == nn[c])) {
      v = make_double2(0.0, 0.0);
    } else {
      const double ir = 1.0 / rad;
      double sn, cs;
      sincos(k * rad, &sn, &cs);
      const double den = 4.0 * M_PI * rad;
      const double2 wg = make_double2(cs / den * dv, sn / den * dv);
      const double2 c1 = make_double2(3.0 * ir * ir - k * k, -3.0 * k * ir);
      const double ar = s[r] * ir, ac = s[c] * ir;
      double2 blk = cmul(wg, c1);
      blk = cscale(cscale(blk, ar), ac);
      if (r == c) {
        const double2 c2 = make_double2(k * k - ir * ir, k * ir);
        blk = cadd(blk, cmul(wg, c2));
      }
      v = blk;
    }
    if (conj) v.y = -v.y;
    out[t] = v;
  }
}

// Scalar acoustic kernel k0^2 dv e^{ikR}/(4 pi R), self cell replaced
// (src/em3d/acoustics/kernel.py:21-40).
static __global__ void k_ac_sample(double2* out, int Nx, int Ny, int Nz, double dx, double dy, double dz, double k0,
                            double dv, double2 self_value, int conj) {
  const size_t n = (size_t)8 * Nx * Ny * Nz;
  const int Ny2 = 2 * Ny, Nz2 = 2 * Nz;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int l = (int)(t % Nz2);
    const int j = (int)((t / Nz2) % Ny2);
    const int i = (int)(t / ((size_t)Nz2 * Ny2));
    const double sx = offset_of(i, Nx, dx), sy = offset_of(j, Ny, dy), sz = offset_of(l, Nz, dz);
    const double R = sqrt(sx * sx + sy * sy + sz * sz);
    double2 v;
    if (R < 1e-15) {
      v = self_value;
    } else {
      double sn, cs;
      sincos(k0 * R, &sn, &cs);
      const double f = (k0 * k0) * dv / (4.0 * M_PI * R);
      v = make_double2(f * cs, f * sn);
    }
    if (conj) v.y = -v.y;
    out[t] = v;
  }
}

template <typename R>
__global__ void k_extract_octant(const double2* __restrict__ full, cx<R>* oct, int Nx, int Ny, int Nz, double scale) {
  const size_t n = (size_t)(Nx + 1) * (Ny + 1) * (Nz + 1);
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int l = (int)(t % (Nz + 1));
    const int j = (int)((t / (Nz + 1)) % (Ny + 1));
    const int i = (int)(t / ((size_t)(Nz + 1) * (Ny + 1)));
    const double2 v = full[((size_t)i * 2 * Ny + j) * 2 * Nz + l];
    oct[t] = from_c64<R>(make_double2(v.x * scale, v.y * scale));
  }
}

template <typename R> __global__ void k_store_full(const double2* __restrict__ full, cx<R>* a, cx<R>* b, size_t n) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const cx<R> v = from_c64<R>(full[t]);
    a[t] = v;
    if (b) b[t] = v;
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

static int grid_blocks(size_t n) {
  size_t b = (n + kThreads - 1) / kThreads;
  if (b > (size_t)148 * 64) b = (size_t)148 * 64;
  return (int)(b ? b : 1);
}

// Opt each kernel in to the full 227 KB of dynamic shared memory once, keyed
// by the kernel's address (its first launch happens outside any capture).
template <typename K> static cudaError_t allow_smem(K kernel) {
  static std::mutex mu;
  static std::unordered_set<const void*> done;
  const void* key = reinterpret_cast<const void*>(kernel);
  std::lock_guard<std::mutex> lock(mu);
  if (done.count(key)) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  if (e == cudaSuccess) done.insert(key);
  return e;
}

// Multiprocessor count of the current device, looked up once per device
// ordinal (host threads driving different GPUs each get their own entry).
static cudaError_t sm_count(int* out) {
  constexpr int kMaxDev = 64;
  static std::mutex mu;
  static int cache[kMaxDev] = {0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < kMaxDev && cache[dev] > 0) { *out = cache[dev]; return cudaSuccess; }
  int n = 0;
  e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < kMaxDev) cache[dev] = n;
  *out = n;
  return cudaSuccess;
}

static inline int check_grid(const em3d_grid* g, Dims* d) {
  if (!g) { em3d_set_last_error("grid is NULL"); return EM3D_ERR_INVALID; }
  if (g->nx <= 0 || g->ny <= 0 || g->nz <= 0) { em3d_set_last_error("grid sizes must be positive"); return EM3D_ERR_INVALID; }
  if (!(g->lx > 0 && g->ly > 0 && g->lz > 0)) { em3d_set_last_error("grid lengths must be positive"); return EM3D_ERR_INVALID; }
  AxisPlan p;
  if (!make_axis_plan(2 * g->nx, &p) || !make_axis_plan(2 * g->ny, &p) || !make_axis_plan(2 * g->nz, &p)) {
    em3d_set_last_error("unsupported grid size: every doubled axis must be <= 1024 with prime factors <= 61");
    return EM3D_ERR_UNSUPPORTED;
  }
  d->nx = g->nx; d->ny = g->ny; d->nz = g->nz;
  return EM3D_OK;
}

// Rows per CTA for a row pass of length L with C components.
template <typename R> static int rows_per_cta(int L, int C, size_t nrows) {
  const int target = sizeof(R) == 4 ? 6144 : 3072;
  int rpb = target / (L * C);
  if (rpb < 1) rpb = 1;
  size_t want = (nrows + 295) / 296;  // keep >= 2 CTAs per SM when the grid is small
  if (want < 1) want = 1;
  if ((size_t)rpb > want) rpb = (int)want;
  return rpb;
}

// Inner-tile width of a strided pass of length L with C components per tile.
template <typename R> static int tile_width(int L, int C) {
  const int target = sizeof(R) == 4 ? 6144 : 3072;
  const int cap = sizeof(R) == 4 ? 16 : 8;
  int p = 1;
  while (p * 2 <= cap && (p * 2) * L * C <= target) p *= 2;
  return p;
}

template <typename R, int C, int LD, int ST, bool INV>
static int launch_rows(const cx<R>* in, const cx<R>* chi, const cx<R>* base, cx<R>* out, const cx<R>* tw, int L,
                       int rows_pb, int nrows, int Lin, int Lout, const int* skip, cudaStream_t st,
                       BatchStrides bs = BatchStrides{}) {
  AxisPlan pl;
  make_axis_plan(L, &pl);
  const int rpb = rows_per_cta<R>(L, C, (size_t)nrows);
  const int P = C * rpb;
  const size_t smem = (size_t)(2 * (size_t)L * odd_stride(P) + L) * sizeof(cx<R>);
  auto kern = k_rows<R, C, LD, ST, INV>;
  EM3D_CUDA_TRY(allow_smem(kern));
  const int grid = (nrows + rpb - 1) / rpb;
  kern<<<grid, kThreads, smem, st>>>(in, chi, base, out, tw, pl, rows_pb, nrows, Lin, Lout, rpb, bs, skip);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

template <typename R, bool INV>
static int launch_strided(const cx<R>* in, cx<R>* out, const cx<R>* tw, int L, int outer, int Lin, int Lout,
                          int inner, const int* skip, cudaStream_t st, BatchStrides bs = BatchStrides{}) {
  AxisPlan pl;
  make_axis_plan(L, &pl);
  const int P = tile_width<R>(L, 1);
  const int ntiles = (inner + P - 1) / P;
  const size_t smem = (size_t)(2 * (size_t)L * odd_stride(P) + L) * sizeof(cx<R>);
  auto kern = k_strided<R, INV>;
  EM3D_CUDA_TRY(allow_smem(kern));
  const size_t grid = (size_t)outer * ntiles;
  if (grid > 0x7fffffff) { em3d_set_last_error("grid too large"); return EM3D_ERR_INVALID; }
  kern<<<(unsigned)grid, kThreads, smem, st>>>(in, out, tw, pl, Lin, Lout, inner, P, ntiles, bs, skip);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

template <typename R, int C, bool ADJ>
static int launch_xmul(cx<R>* T2, const cx<R>* spec, const cx<R>* tw, const Dims& d, int batch, const int* skip,
                       cudaStream_t st, BatchStrides bs) {
  AxisPlan pl;
  make_axis_plan(2 * d.nx, &pl);
  const int Pz = tile_width<R>(2 * d.nx, C);
  const int ntz = (2 * d.nz + Pz - 1) / Pz;
  const int P = C * Pz;
  const size_t smem = (size_t)(2 * (size_t)(2 * d.nx) * odd_stride(P) + 2 * d.nx) * sizeof(cx<R>);
  auto kern = k_xmul<R, C, ADJ>;
  EM3D_CUDA_TRY(allow_smem(kern));
  const size_t grid = (size_t)batch * 2 * d.ny * ntz;
  kern<<<(unsigned)grid, kThreads, smem, st>>>(T2, spec, tw, pl, d.nx, d.ny, d.nz, Pz, ntz, batch, bs, skip);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

// In-place forward 3D FFT of one FP64 doubled-grid block.
static int fft3d_inplace(double2* buf, const double2* twx, const double2* twy, const double2* twz, const Dims& d,
                         cudaStream_t st) {
  const int X = 2 * d.nx, Y = 2 * d.ny, Z = 2 * d.nz;
  int rc = launch_rows<double, 1, LD_PLAIN, ST_PLAIN, false>(buf, nullptr, nullptr, buf, twz, Z, X * Y, X * Y, Z, Z,
                                                             nullptr, st);
  if (rc) return rc;
  rc = launch_strided<double, false>(buf, buf, twy, Y, X, Y, Y, Z, nullptr, st);
  if (rc) return rc;
  return launch_strided<double, false>(buf, buf, twx, X, 1, X, X, Y * Z, nullptr, st);
}

template <typename R> static int init_twiddles(cx<R>* tw, int L, cudaStream_t st) {
  k_twiddles<R><<<(L + 255) / 256, 256, 0, st>>>(tw, L);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

struct BuildBufs {
  double2 *full, *twx, *twy, *twz;
};

static int build_bufs(const Dims& d, void* ws, size_t ws_bytes, cudaStream_t st, BuildBufs* b) {
  if (!ws || ws_bytes < build_ws_bytes(d)) { em3d_set_last_error("build workspace too small"); return EM3D_ERR_INVALID; }
  b->full = (double2*)ws;
  b->twx = (double2*)((char*)ws + align_up(d.doubled() * sizeof(double2)));
  b->twy = b->twx + 2 * d.nx;
  b->twz = b->twy + 2 * d.ny;
  int rc = init_twiddles<double>(b->twx, 2 * d.nx, st);
  if (!rc) rc = init_twiddles<double>(b->twy, 2 * d.ny, st);
  if (!rc) rc = init_twiddles<double>(b->twz, 2 * d.nz, st);
  return rc;
}

static const int kPairs[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};

template <typename R>
static int em_spectrum_build(const em3d_grid* g, const Dims& d, double k, void* spectrum, void* ws, size_t wsb,
                             cudaStream_t st) {
  BuildBufs b;
  int rc = build_bufs(d, ws, wsb, st, &b);
  if (rc) return rc;
  SpecLayout<R> lay(d, EM3D_EM);
  const double dx = g->lx / d.nx, dy = g->ly / d.ny, dz = g->lz / d.nz;
  const double dv = dx * dy * dz;
  const double scale = 1.0 / (double)d.doubled();
  for (int blk = 0; blk < 6; ++blk) {
    k_em_sample<<<grid_blocks(d.doubled()), kThreads, 0, st>>>(b.full, kPairs[blk][0], kPairs[blk][1], d.nx, d.ny,
                                                                d.nz, dx, dy, dz, k, dv, 1, 0);
    EM3D_LAUNCH_CHECK();
    if ((rc = fft3d_inplace(b.full, b.twx, b.twy, b.twz, d, st))) return rc;
    k_extract_octant<R><<<grid_blocks(d.octant()), kThreads, 0, st>>>(b.full, lay.oct(spectrum) + blk * lay.oct_elems,
                                                                       d.nx, d.ny, d.nz, scale);
    EM3D_LAUNCH_CHECK();
  }
  if ((rc = init_twiddles<R>(lay.twx(spectrum, d), 2 * d.nx, st))) return rc;
  if ((rc = init_twiddles<R>(lay.twy(spectrum, d), 2 * d.ny, st))) return rc;
  return init_twiddles<R>(lay.twz(spectrum, d), 2 * d.nz, st);
}

static double2 acoustic_self_value(double k0, double dv) {
  // e^{ika}(1 - ika) - 1 with a = (3 dv / 4 pi)^(1/3)  (src/em3d/acoustics/kernel.py:7-18)
  const double a = std::pow(3.0 * dv / (4.0 * M_PI), 1.0 / 3.0);
  const double ka = k0 * a;
  const double c = std::cos(ka), s = std::sin(ka);
  // (c + i s)(1 - i ka) = c + s ka + i (s - c ka)
  return make_double2(c + s * ka - 1.0, s - c * ka);
}

template <typename R>
static int ac_spectrum_build(const em3d_grid* g, const Dims& d, double k0, void* spectrum, void* ws, size_t wsb,
                             cudaStream_t st) {
  BuildBufs b;
  int rc = build_bufs(d, ws, wsb, st, &b);
  if (rc) return rc;
  SpecLayout<R> lay(d, EM3D_ACOUSTIC);
  const double dx = g->lx / d.nx, dy = g->ly / d.ny, dz = g->lz / d.nz;
  const double dv = dx * dy * dz;
  k_ac_sample<<<grid_blocks(d.doubled()), kThreads, 0, st>>>(b.full, d.nx, d.ny, d.nz, dx, dy, dz, k0, dv,
                                                              acoustic_self_value(k0, dv), 0);
  EM3D_LAUNCH_CHECK();
  if ((rc = fft3d_inplace(b.full, b.twx, b.twy, b.twz, d, st))) return rc;
  k_extract_octant<R><<<grid_blocks(d.octant()), kThreads, 0, st>>>(b.full, lay.oct(spectrum), d.nx, d.ny, d.nz,
                                                                     1.0 / (double)d.doubled());
  EM3D_LAUNCH_CHECK();
  if ((rc = init_twiddles<R>(lay.twx(spectrum, d), 2 * d.nx, st))) return rc;
  if ((rc = init_twiddles<R>(lay.twy(spectrum, d), 2 * d.ny, st))) return rc;
  return init_twiddles<R>(lay.twz(spectrum, d), 2 * d.nz, st);
}

template <typename R>
static int em_kernel_hat_full(const em3d_grid* g, const Dims& d, double k, int adjoint, void* out, void* ws, size_t wsb,
                              cudaStream_t st) {
  BuildBufs b;
  int rc = build_bufs(d, ws, wsb, st, &b);
  if (rc) return rc;
  const double dx = g->lx / d.nx, dy = g->ly / d.ny, dz = g->lz / d.nz;
  const double dv = dx * dy * dz;
  const size_t M = d.doubled();
  cx<R>* o = (cx<R>*)out;
  for (int blk = 0; blk < 6; ++blk) {
    const int r = kPairs[blk][0], c = kPairs[blk][1];
    k_em_sample<<<grid_blocks(M), kThreads, 0, st>>>(b.full, r, c, d.nx, d.ny, d.nz, dx, dy, dz, k, dv, 0, adjoint);
    EM3D_LAUNCH_CHECK();
    if ((rc = fft3d_inplace(b.full, b.twx, b.twy, b.twz, d, st))) return rc;
    k_store_full<R><<<grid_blocks(M), kThreads, 0, st>>>(b.full, o + (size_t)(r * 3 + c) * M,
                                                          r == c ? nullptr : o + (size_t)(c * 3 + r) * M, M);
    EM3D_LAUNCH_CHECK();
  }
  return EM3D_OK;
}

template <typename R>
static int ac_kernel_hat_full(const em3d_grid* g, const Dims& d, double k0, int adjoint, void* out, void* ws, size_t wsb,
                              cudaStream_t st) {
  BuildBufs b;
  int rc = build_bufs(d, ws, wsb, st, &b);
  if (rc) return rc;
  const double dx = g->lx / d.nx, dy = g->ly / d.ny, dz = g->lz / d.nz;
  const double dv = dx * dy * dz;
  const size_t M = d.doubled();
  k_ac_sample<<<grid_blocks(M), kThreads, 0, st>>>(b.full, d.nx, d.ny, d.nz, dx, dy, dz, k0, dv,
                                                    acoustic_self_value(k0, dv), adjoint);
  EM3D_LAUNCH_CHECK();
  if ((rc = fft3d_inplace(b.full, b.twx, b.twy, b.twz, d, st))) return rc;
  k_store_full<R><<<grid_blocks(M), kThreads, 0, st>>>(b.full, (cx<R>*)out, nullptr, M);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

// ---- register-FFT dispatch (doubled axes 32..512 and 96, 160, 192) -------

// Tuning knobs (em3d_set_tuning / em3d_get_tuning).  They select among
// equivalent implementations; results do not depend on them beyond rounding.
extern int g_tuning[EM3D_TUNE_COUNT];  // defined in operator.cu

static bool generic_forced() {
  const char* v = getenv("EM3D_FFT_GENERIC");
  return g_tuning[EM3D_TUNE_FFT_GENERIC] != 0 || (v && v[0] == '1');
}

// 160 (20 elements per thread) runs on the register plan in complex64 for
// every pass and in complex128 for the row and pencil passes (one pencil per
// thread); the complex128 x pass, which holds three pencils per thread, would
// spill and uses the generic passes.
static bool fast_len(int L, bool fp64, bool x_pass) {
  return !generic_forced() && (L == 32 || L == 64 || L == 128 || L == 256 || L == 512 || L == 96 || L == 192 ||
                               (L == 160 && !(fp64 && x_pass)));
}

template <typename R, int L, int C, int LD, int ST, bool INV>
static int go_rows(const cx<R>* in, const cx<R>* chi, const cx<R>* base, cx<R>* out, const cx<R>* tw, int rows_pb,
                   int nrows, const int* skip, cudaStream_t st, BatchStrides bs) {
  using G = RowsGeom<L, FastE<R, L>::E, C>;
  auto kern = kf_rows<R, L, C, LD, ST, INV>;
  EM3D_CUDA_TRY(allow_smem(kern));
  const size_t smem = (size_t)(L + C * G::RPB * G::PSTRIDE) * sizeof(cx<R>);
  const int grid = (nrows + G::RPB - 1) / G::RPB;
  kern<<<grid, G::NT, smem, st>>>(in, chi, base, out, tw, rows_pb, nrows, bs, skip);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

template <typename R, int C, int LD, int ST, bool INV>
static int launch_rows_fast(int L, const cx<R>* in, const cx<R>* chi, const cx<R>* base, cx<R>* out,
                            const cx<R>* tw, int rows_pb, int nrows, const int* skip, cudaStream_t st,
                            BatchStrides bs) {
  switch (L) {
    case 32: return go_rows<R, 32, C, LD, ST, INV>(in, chi, base, out, tw, rows_pb, nrows, skip, st, bs);
    case 64: return go_rows<R, 64, C, LD, ST, INV>(in, chi, base, out, tw, rows_pb, nrows, skip, st, bs);
    case 128: return go_rows<R, 128, C, LD, ST, INV>(in, chi, base, out, tw, rows_pb, nrows, skip, st, bs);
    case 256: return go_rows<R, 256, C, LD, ST, INV>(in, chi, base, out, tw, rows_pb, nrows, skip, st, bs);
    case 512: return go_rows<R, 512, C, LD, ST, INV>(in, chi, base, out, tw, rows_pb, nrows, skip, st, bs);
    case 96: return go_rows<R, 96, C, LD, ST, INV>(in, chi, base, out, tw, rows_pb, nrows, skip, st, bs);
    case 160:
      return go_rows<R, 160, C, LD, ST, INV>(in, chi, base, out, tw, rows_pb, nrows, skip, st, bs);
    case 192: return go_rows<R, 192, C, LD, ST, INV>(in, chi, base, out, tw, rows_pb, nrows, skip, st, bs);
  }
  em3d_set_last_error("no register FFT for this length");
  return EM3D_ERR_UNSUPPORTED;
}

template <typename R, int L, bool INV>
static int go_strided(const cx<R>* in, cx<R>* out, const cx<R>* tw, int outer, int inner, const int* skip,
                      cudaStream_t st, BatchStrides bs) {
  using G = StridedGeom<L, FastE<R, L>::E>;
  auto kern = kf_strided<R, L, INV>;
  EM3D_CUDA_TRY(allow_smem(kern));
  const int ntiles = (inner + G::P - 1) / G::P;
  const size_t smem = (size_t)(L + L * G::S) * sizeof(cx<R>);
  const size_t grid = (size_t)outer * ntiles;
  kern<<<(unsigned)grid, G::NT, smem, st>>>(in, out, tw, inner, ntiles, bs, skip);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

// CTAs of a register row pass of length L over nrows rows (the partial sums
// that FST_SUB_DOTS writes); 0 when L has no register plan.
template <typename R, int C> static int rows_fast_ctas(int L, int nrows) {
  switch (L) {
#define EM3D_CASE(LL) \
  case LL: { constexpr int RPB = RowsGeom<LL, FastE<R, LL>::E, C>::RPB; return (nrows + RPB - 1) / RPB; }
    EM3D_CASE(32) EM3D_CASE(64) EM3D_CASE(128) EM3D_CASE(256) EM3D_CASE(512) EM3D_CASE(96) EM3D_CASE(160)
    EM3D_CASE(192)
#undef EM3D_CASE
  }
  return 0;
}

template <typename R, bool INV>
static int launch_strided_fast(int L, const cx<R>* in, cx<R>* out, const cx<R>* tw, int outer, int inner,
                               const int* skip, cudaStream_t st, BatchStrides bs) {
  switch (L) {
    case 32: return go_strided<R, 32, INV>(in, out, tw, outer, inner, skip, st, bs);
    case 64: return go_strided<R, 64, INV>(in, out, tw, outer, inner, skip, st, bs);
    case 128: return go_strided<R, 128, INV>(in, out, tw, outer, inner, skip, st, bs);
    case 256: return go_strided<R, 256, INV>(in, out, tw, outer, inner, skip, st, bs);
    case 512: return go_strided<R, 512, INV>(in, out, tw, outer, inner, skip, st, bs);
    case 96: return go_strided<R, 96, INV>(in, out, tw, outer, inner, skip, st, bs);
    case 160:
      return go_strided<R, 160, INV>(in, out, tw, outer, inner, skip, st, bs);
    case 192: return go_strided<R, 192, INV>(in, out, tw, outer, inner, skip, st, bs);
  }
  em3d_set_last_error("no register FFT for this length");
  return EM3D_ERR_UNSUPPORTED;
}

template <typename R, int L, int C, bool ADJ, int E, int NTT = 256>
static int go_xmul(cx<R>* T2, const cx<R>* spec, const cx<R>* tw, const Dims& d, int batch, const int* skip,
                   cudaStream_t st, BatchStrides bs) {
  using G = XmulGeom<L, E, C, NTT>;
  auto kern = kf_xmul<R, L, C, ADJ, E, NTT>;
  EM3D_CUDA_TRY(allow_smem(kern));
  const int ntz = (2 * d.nz + G::P - 1) / G::P;
  const size_t smem = (size_t)(L + G::REGIONS * L * G::S) * sizeof(cx<R>);
  const size_t grid = (size_t)batch * 2 * d.ny * ntz;
  kern<<<(unsigned)grid, G::NT, smem, st>>>(T2, spec, tw, d.ny, d.nz, ntz, batch, bs, skip);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

template <typename R, int L, int C, bool ADJ, int E, int NTT, bool TMAF, int MINB = 1>
static int go_xpipe(cx<R>* T2, const cx<R>* spec, const cx<R>* tw, const Dims& d, int batch, const int* skip,
                    cudaStream_t st, BatchStrides bs) {
  using G = XpipeGeom<L, E, C, NTT>;
  auto kern = kf_xmul_pipe<R, L, C, ADJ, E, NTT, TMAF, MINB>;
  EM3D_CUDA_TRY(allow_smem(kern));
  const size_t smem = (size_t)G::TOTAL * sizeof(cx<R>) + G::BYTES_EXTRA;
  const int ntz = (2 * d.nz + G::P - 1) / G::P;
  // work units: (entries, jy = 0..Ny, kz tile), see kf_xmul_pipe
  const long long ntiles = (long long)(batch / xpipe_entries_per_unit(batch, bs.spec == 0)) * (d.ny + 1) * ntz;
  int sms = 0;
  EM3D_CUDA_TRY(sm_count(&sms));
  int per_sm = 0;
  EM3D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, G::NT, smem));
  if (per_sm < 1) per_sm = 1;
  const long long grid = std::min<long long>(ntiles, (long long)sms * per_sm);
  if (grid <= 0) return EM3D_OK;
  CUtensorMap fmap;
  memset(&fmap, 0, sizeof fmap);
  if constexpr (TMAF) {
    // T2 as 8-byte words: (2 Nz * W, 2 Ny, batch * C * Nx), one box of
    // P * W words x 1 x Nx per component and tile.  The row strides are
    // multiples of 16 bytes, the box's inner extent is P * 8 or P * 16 bytes
    // and every tile starts at kz0 = a multiple of P (even), so each load
    // starts on a 16-byte boundary.
    static_assert(G::P % 2 == 0 && L / 2 <= 256, "TMA field slab: even tile width, at most 256 rows per box");
    auto enc = tensor_map_encoder();
    if (enc == nullptr) { em3d_set_last_error("cuTensorMapEncodeTiled is unavailable"); return EM3D_ERR_CUDA; }
    constexpr cuuint64_t W = sizeof(cx<R>) / 8;
    const cuuint64_t dims[3] = {(cuuint64_t)2 * d.nz * W, (cuuint64_t)2 * d.ny, (cuuint64_t)batch * C * d.nx};
    const cuuint64_t strides[2] = {(cuuint64_t)2 * d.nz * sizeof(cx<R>), (cuuint64_t)4 * d.ny * d.nz * sizeof(cx<R>)};
    const cuuint32_t box[3] = {(cuuint32_t)(G::P * W), 1u, (cuuint32_t)d.nx};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    const CUresult r = enc(&fmap, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, (void*)T2, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) { em3d_set_last_error("cuTensorMapEncodeTiled rejected the field slab map"); return EM3D_ERR_CUDA; }
  }
  kern<<<(unsigned)grid, G::NT, smem, st>>>(T2, spec, tw, d.ny, d.nz, ntz, batch, bs, skip, fmap, bs.status);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

// T2 as 8-byte words (2 Nz W, 2 Ny, batch C Nx), one box of P W words x 1 x
// Nx per component and tile (see go_xpipe).
template <typename R, int C, int P>
static int encode_field_map(CUtensorMap* fmap, cx<R>* T2, const Dims& d, int batch) {
  auto enc = tensor_map_encoder();
  if (enc == nullptr) { em3d_set_last_error("cuTensorMapEncodeTiled is unavailable"); return EM3D_ERR_CUDA; }
  constexpr cuuint64_t W = sizeof(cx<R>) / 8;
  const cuuint64_t dims[3] = {(cuuint64_t)2 * d.nz * W, (cuuint64_t)2 * d.ny, (cuuint64_t)batch * C * d.nx};
  const cuuint64_t strides[2] = {(cuuint64_t)2 * d.nz * sizeof(cx<R>), (cuuint64_t)4 * d.ny * d.nz * sizeof(cx<R>)};
  const cuuint32_t box[3] = {(cuuint32_t)(P * W), 1u, (cuuint32_t)d.nx};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  memset(fmap, 0, sizeof *fmap);
  const CUresult r = enc(fmap, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, (void*)T2, dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) { em3d_set_last_error("cuTensorMapEncodeTiled rejected the field slab map"); return EM3D_ERR_CUDA; }
  return EM3D_OK;
}

template <typename R, int L, int C, bool ADJ, int E, int NTT, bool ROT>
static int go_xrot(cx<R>* T2, const cx<R>* spec, const cx<R>* tw, const Dims& d, int batch, const int* skip,
                   cudaStream_t st, BatchStrides bs) {
  using G = XrotGeom<L, E, C, NTT>;
  static_assert(G::P % 2 == 0 && L / 2 <= 256, "TMA field slab: even tile width, at most 256 rows per box");
  auto kern = kf_xmul_rot<R, L, C, ADJ, E, NTT, ROT>;
  EM3D_CUDA_TRY(allow_smem(kern));
  const size_t smem = (size_t)G::TOTAL * sizeof(cx<R>) + G::BYTES_EXTRA;
  const int ntz = (2 * d.nz + G::P - 1) / G::P;
  const long long ntiles = (long long)(batch / xpipe_entries_per_unit(batch, bs.spec == 0)) * (d.ny + 1) * ntz;
  int sms = 0;
  EM3D_CUDA_TRY(sm_count(&sms));
  int per_sm = 0;
  EM3D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, G::NT, smem));
  if (per_sm < 1) per_sm = 1;
  const long long grid = std::min<long long>(ntiles, (long long)sms * per_sm);
  if (grid <= 0) return EM3D_OK;
  CUtensorMap fmap;
  if (int rc = encode_field_map<R, C, G::P>(&fmap, T2, d, batch)) return rc;
  kern<<<(unsigned)grid, G::NT, smem, st>>>(T2, spec, tw, d.ny, d.nz, ntz, batch, bs, skip, fmap, bs.status);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

template <typename R, int L, bool ADJ, int E>
static int go_xsplit(cx<R>* T2, const cx<R>* spec, const cx<R>* tw, const Dims& d, int batch, const int* skip,
                     cudaStream_t st, BatchStrides bs) {
  using G = XsplitGeom<L, E>;
  auto kern = kf_xmul_split<R, L, ADJ, E>;
  EM3D_CUDA_TRY(allow_smem(kern));
  const int ntz = (2 * d.nz + G::PZ - 1) / G::PZ;
  const size_t smem = (size_t)(L + 3 * G::REGION) * sizeof(cx<R>);
  const size_t grid = (size_t)batch * 2 * d.ny * ntz;
  kern<<<(unsigned)grid, G::NT, smem, st>>>(T2, spec, tw, d.ny, d.nz, ntz, batch, bs, skip);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

// x-pass variant (tuning key EM3D_TUNE_XPASS_VARIANT): 0 = three components
// in registers, 256-thread CTAs; 1 = the same with 128-thread CTAs (two per
// SM); 2 = component-split threads (EM only); 3 = persistent CTAs with the
// next tile's field and spectrum prefetched by cp.async, 256 threads; 4 = the
// same with 128 threads; 5 and 6 = 3 and 4 with the field slab loaded by TMA;
// 7, 8 and 9 = 6 with register twiddles and single-barrier exchanges
// (kf_xmul_rot; plans equal to their reverse only): 7 with one copy of the
// transform code rotating the three components, 8 without, 9 = 8 with
// 256-thread CTAs; 10 = 6 with 8 elements per thread (complex64, power-of-two
// axes) in 256-thread CTAs limited to 128 registers, two per SM.  -1 (the
// default) picks, per operator kind and x length, the fastest
// measured on B200: EM 6 (both precisions; 128^3, 96^3, 80^3); acoustic 9 on
// 512-point axes (256^3: 1.35 vs 1.36-1.54 ms for variant 5 in complex64, 2.46
// vs 2.67-3.03 ms in complex128) and 0 on shorter ones (128^3).
static int xmul_variant(int C, int L) {
  const int v = g_tuning[EM3D_TUNE_XPASS_VARIANT];
  if (v >= 0) return v;
  if (C == 3) return 6;
  return L >= 512 ? 9 : 0;
}

// Shared memory of each x-pass variant; a variant that does not fit in the
// 227 KB a CTA may use (large mixed-radix plans in complex128) is replaced by
// the first that fits in the order 6, 4, 1, 2, 0, 5, 3.
constexpr size_t kSmemPerCta = 227 * 1024;

template <typename R, int L, int C, int E>
static size_t xvariant_smem(int v) {
  switch (v) {
    case 0: return (size_t)(L + XmulGeom<L, E, C, 256>::REGIONS * L * XmulGeom<L, E, C, 256>::S) * sizeof(cx<R>);
    case 1: return (size_t)(L + XmulGeom<L, E, C, 128>::REGIONS * L * XmulGeom<L, E, C, 128>::S) * sizeof(cx<R>);
    case 2: return C == 3 ? (size_t)(L + 3 * XsplitGeom<L, E>::REGION) * sizeof(cx<R>) : ~(size_t)0;
    case 3: case 5: return (size_t)XpipeGeom<L, E, C, 256>::TOTAL * sizeof(cx<R>) + 16;
    case 4: case 6: return (size_t)XpipeGeom<L, E, C, 128>::TOTAL * sizeof(cx<R>) + 16;
    case 7: case 8:
      return SymPlan<L, E>::symmetric() ? (size_t)XrotGeom<L, E, C, 128>::TOTAL * sizeof(cx<R>) + 16 : ~(size_t)0;
    case 9: return SymPlan<L, E>::symmetric() ? (size_t)XrotGeom<L, E, C, 256>::TOTAL * sizeof(cx<R>) + 16 : ~(size_t)0;
    case 10:
      return (sizeof(R) == 4 && (L & (L - 1)) == 0) ? (size_t)XpipeGeom<L, 8, C, 256>::TOTAL * sizeof(cx<R>) + 16
                                                     : ~(size_t)0;
  }
  return ~(size_t)0;
}

template <typename R, int C, bool ADJ, int L>
static int launch_xmul_len(cx<R>* T2, const cx<R>* spec, const cx<R>* tw, const Dims& d, int batch,
                           const int* skip, cudaStream_t st, BatchStrides bs) {
  constexpr int EB = FastE<R, L>::E;
  int v = xmul_variant(C, L);
  if (C == 1 && v == 2) v = 0;  // the component split is EM only
  if (xvariant_smem<R, L, C, EB>(v) > kSmemPerCta) {
    for (int alt : {6, 4, 1, 2, 0, 5, 3}) {
      if (xvariant_smem<R, L, C, EB>(alt) <= kSmemPerCta) { v = alt; break; }
    }
  }
  if constexpr (C == 3) {
    if (v == 2) return go_xsplit<R, L, ADJ, EB>(T2, spec, tw, d, batch, skip, st, bs);
  }
  if (v == 3) return go_xpipe<R, L, C, ADJ, EB, 256, false>(T2, spec, tw, d, batch, skip, st, bs);
  if (v == 4) return go_xpipe<R, L, C, ADJ, EB, 128, false>(T2, spec, tw, d, batch, skip, st, bs);
  if (v == 5) return go_xpipe<R, L, C, ADJ, EB, 256, true>(T2, spec, tw, d, batch, skip, st, bs);
  if (v == 6) return go_xpipe<R, L, C, ADJ, EB, 128, true>(T2, spec, tw, d, batch, skip, st, bs);
  if constexpr (SymPlan<L, EB>::symmetric()) {
    if (v == 7) return go_xrot<R, L, C, ADJ, EB, 128, true>(T2, spec, tw, d, batch, skip, st, bs);
    if (v == 8) return go_xrot<R, L, C, ADJ, EB, 128, false>(T2, spec, tw, d, batch, skip, st, bs);
    if (v == 9) return go_xrot<R, L, C, ADJ, EB, 256, false>(T2, spec, tw, d, batch, skip, st, bs);
  }
  if constexpr (sizeof(R) == 4 && (L & (L - 1)) == 0) {
    // 8 elements per thread, two 256-thread CTAs per SM (16 warps)
    if (v == 10) return go_xpipe<R, L, C, ADJ, 8, 256, true, 2>(T2, spec, tw, d, batch, skip, st, bs);
  }
  if (v == 1) return go_xmul<R, L, C, ADJ, EB, 128>(T2, spec, tw, d, batch, skip, st, bs);
  return go_xmul<R, L, C, ADJ, EB, 256>(T2, spec, tw, d, batch, skip, st, bs);
}

template <typename R, int C, bool ADJ>
static int launch_xmul_fast(cx<R>* T2, const cx<R>* spec, const cx<R>* tw, const Dims& d, int batch,
                            const int* skip, cudaStream_t st, BatchStrides bs) {
  switch (2 * d.nx) {
    case 32: return launch_xmul_len<R, C, ADJ, 32>(T2, spec, tw, d, batch, skip, st, bs);
    case 64: return launch_xmul_len<R, C, ADJ, 64>(T2, spec, tw, d, batch, skip, st, bs);
    case 128: return launch_xmul_len<R, C, ADJ, 128>(T2, spec, tw, d, batch, skip, st, bs);
    case 256: return launch_xmul_len<R, C, ADJ, 256>(T2, spec, tw, d, batch, skip, st, bs);
    case 512: return launch_xmul_len<R, C, ADJ, 512>(T2, spec, tw, d, batch, skip, st, bs);
    case 96: return launch_xmul_len<R, C, ADJ, 96>(T2, spec, tw, d, batch, skip, st, bs);
    case 160:
      if constexpr (sizeof(R) == 4) return launch_xmul_len<R, C, ADJ, 160>(T2, spec, tw, d, batch, skip, st, bs);
      break;
    case 192: return launch_xmul_len<R, C, ADJ, 192>(T2, spec, tw, d, batch, skip, st, bs);
  }
  em3d_set_last_error("no register FFT for this length");
  return EM3D_ERR_UNSUPPORTED;
}


// The five passes of one application.
template <typename R, int C, bool ADJ>
int apply(const Dims& d, int batch, const void* spectrum, const void* chi, const void* u, void* out, void* ws,
                 size_t wsb, const int* skip, cudaStream_t st, BatchStrides bs = BatchStrides{}) {
  if (batch < 1) { em3d_set_last_error("batch must be >= 1"); return EM3D_ERR_INVALID; }
  if (!spectrum || !chi || !u || !out) { em3d_set_last_error("NULL array argument"); return EM3D_ERR_INVALID; }
  if (!ws || wsb < apply_ws_bytes<R>(d, C, batch)) { em3d_set_last_error("apply workspace too small"); return EM3D_ERR_INVALID; }
  if (out == u) { em3d_set_last_error("out must not alias the input field"); return EM3D_ERR_INVALID; }
  using T = cx<R>;
  bs.outer = C * d.nx;
  bs.status = (int*)((char*)ws + apply_status_offset<R>(d, C, batch));
  SpecLayout<R> lay(d, C == 3 ? EM3D_EM : EM3D_ACOUSTIC);
  void* sp = const_cast<void*>(spectrum);
  const T* twx = lay.twx(sp, d);
  const T* twy = lay.twy(sp, d);
  const T* twz = lay.twz(sp, d);
  const T* oct = lay.oct(sp);
  T* T1 = (T*)ws;
  T* T2 = (T*)((char*)ws + align_up((size_t)batch * C * d.nx * d.ny * 2 * d.nz * sizeof(T)));
  const T* uu = (const T*)u;
  const T* ch = (const T*)chi;
  T* o = (T*)out;
  const int rows = d.nx * d.ny;
  const int nrows = batch * rows;
  int rc;
  const int Lz = 2 * d.nz, Ly = 2 * d.ny;
  constexpr bool F64 = sizeof(R) == 8;
  const bool fz = fast_len(Lz, F64, false), fy = fast_len(Ly, F64, false), fx = fast_len(2 * d.nx, F64, true);
  if (bs.dots && (ADJ || !fz || batch != 1)) {
    em3d_set_last_error("the fused dot products need a matvec of one right-hand side on a register-FFT z length");
    return EM3D_ERR_UNSUPPORTED;
  }
  constexpr int LDF = C == 3 ? LD_EM_CHI : LD_AC_CHI;
  constexpr int FLDF = C == 3 ? FLD_EM_CHI : FLD_AC_CHI;
  constexpr int STA = C == 3 ? ST_EM_ADJ : ST_AC_ADJ;
  constexpr int FSTA = C == 3 ? FST_EM_ADJ : FST_AC_ADJ;
  // pass 1: rows along z, chi applied on load (matvec) or plain (rmatvec);
  // an EM contrast stored as 6 or 1 components per cell has its own load mode
  const int chil = C == 3 ? bs.chi_layout : 9;
  if (fz) {
    if (ADJ) rc = launch_rows_fast<R, C, FLD_PLAIN, FST_PLAIN, false>(Lz, uu, nullptr, nullptr, T1, twz, rows, nrows, skip, st, bs);
    else if constexpr (C == 3) {
      if (chil == 6) rc = launch_rows_fast<R, C, FLD_EM_CHI6, FST_PLAIN, false>(Lz, uu, ch, nullptr, T1, twz, rows, nrows, skip, st, bs);
      else if (chil == 1) rc = launch_rows_fast<R, C, FLD_EM_CHI1, FST_PLAIN, false>(Lz, uu, ch, nullptr, T1, twz, rows, nrows, skip, st, bs);
      else rc = launch_rows_fast<R, C, FLDF, FST_PLAIN, false>(Lz, uu, ch, nullptr, T1, twz, rows, nrows, skip, st, bs);
    } else rc = launch_rows_fast<R, C, FLDF, FST_PLAIN, false>(Lz, uu, ch, nullptr, T1, twz, rows, nrows, skip, st, bs);
  } else {
    if (ADJ) rc = launch_rows<R, C, LD_PLAIN, ST_PLAIN, false>(uu, nullptr, nullptr, T1, twz, Lz, rows, nrows, d.nz, Lz, skip, st, bs);
    else if constexpr (C == 3) {
      if (chil == 6) rc = launch_rows<R, C, LD_EM_CHI6, ST_PLAIN, false>(uu, ch, nullptr, T1, twz, Lz, rows, nrows, d.nz, Lz, skip, st, bs);
      else if (chil == 1) rc = launch_rows<R, C, LD_EM_CHI1, ST_PLAIN, false>(uu, ch, nullptr, T1, twz, Lz, rows, nrows, d.nz, Lz, skip, st, bs);
      else rc = launch_rows<R, C, LDF, ST_PLAIN, false>(uu, ch, nullptr, T1, twz, Lz, rows, nrows, d.nz, Lz, skip, st, bs);
    } else rc = launch_rows<R, C, LDF, ST_PLAIN, false>(uu, ch, nullptr, T1, twz, Lz, rows, nrows, d.nz, Lz, skip, st, bs);
  }
  if (rc) return rc;
  // pass 2: (batch*C*Nx, Ny, 2Nz) -> (batch*C*Nx, 2Ny, 2Nz)
  if (fy) rc = launch_strided_fast<R, false>(Ly, T1, T2, twy, batch * C * d.nx, Lz, skip, st, bs);
  else rc = launch_strided<R, false>(T1, T2, twy, Ly, batch * C * d.nx, d.ny, Ly, Lz, skip, st, bs);
  if (rc) return rc;
  // pass 3
  if (fx) rc = launch_xmul_fast<R, C, ADJ>(T2, oct, twx, d, batch, skip, st, bs);
  else rc = launch_xmul<R, C, ADJ>(T2, oct, twx, d, batch, skip, st, bs);
  if (rc) return rc;
  // pass 4: (batch*C*Nx, 2Ny, 2Nz) -> (batch*C*Nx, Ny, 2Nz)
  if (fy) rc = launch_strided_fast<R, true>(Ly, T2, T1, twy, batch * C * d.nx, Lz, skip, st, bs);
  else rc = launch_strided<R, true>(T2, T1, twy, Ly, batch * C * d.nx, Ly, d.ny, Lz, skip, st, bs);
  if (rc) return rc;
  // pass 5: rows along z, crop and combine
  if (fz) {
    bool fused = false;
    if constexpr (!ADJ) {
      if (bs.dots) {
        rc = launch_rows_fast<R, C, FLD_PLAIN, FST_SUB_DOTS, true>(Lz, T1, nullptr, uu, o, twz, rows, nrows, skip, st, bs);
        fused = true;
      }
    }
    if (fused) {
    } else if (!ADJ) rc = launch_rows_fast<R, C, FLD_PLAIN, FST_SUB, true>(Lz, T1, nullptr, uu, o, twz, rows, nrows, skip, st, bs);
    else if constexpr (C == 3) {
      if (chil == 6) rc = launch_rows_fast<R, C, FLD_PLAIN, FST_EM_ADJ6, true>(Lz, T1, ch, uu, o, twz, rows, nrows, skip, st, bs);
      else if (chil == 1) rc = launch_rows_fast<R, C, FLD_PLAIN, FST_EM_ADJ1, true>(Lz, T1, ch, uu, o, twz, rows, nrows, skip, st, bs);
      else rc = launch_rows_fast<R, C, FLD_PLAIN, FSTA, true>(Lz, T1, ch, uu, o, twz, rows, nrows, skip, st, bs);
    } else rc = launch_rows_fast<R, C, FLD_PLAIN, FSTA, true>(Lz, T1, ch, uu, o, twz, rows, nrows, skip, st, bs);
  } else {
    if (!ADJ) rc = launch_rows<R, C, LD_PLAIN, ST_SUB, true>(T1, nullptr, uu, o, twz, Lz, rows, nrows, Lz, d.nz, skip, st, bs);
    else if constexpr (C == 3) {
      if (chil == 6) rc = launch_rows<R, C, LD_PLAIN, ST_EM_ADJ6, true>(T1, ch, uu, o, twz, Lz, rows, nrows, Lz, d.nz, skip, st, bs);
      else if (chil == 1) rc = launch_rows<R, C, LD_PLAIN, ST_EM_ADJ1, true>(T1, ch, uu, o, twz, Lz, rows, nrows, Lz, d.nz, skip, st, bs);
      else rc = launch_rows<R, C, LD_PLAIN, STA, true>(T1, ch, uu, o, twz, Lz, rows, nrows, Lz, d.nz, skip, st, bs);
    } else rc = launch_rows<R, C, LD_PLAIN, STA, true>(T1, ch, uu, o, twz, Lz, rows, nrows, Lz, d.nz, skip, st, bs);
  }
  return rc;
}


}  // namespace em3d
