// Operator passes on the register-resident FFT (power-of-two axes 32..512,
// and 96, 160, 192).
// Same data layouts and fused work as the generic passes in operator.cu:
//   kf_rows    pass 1 (z forward, chi applied on load) and pass 5 (z inverse,
//              crop, u - y or v - chi^H y on store)
//   kf_strided passes 2 and 4 (y forward with zero padding, y inverse with crop)
//   kf_xmul    pass 3 (x forward, spectrum multiply in registers, x inverse, crop)
#pragma once

#include "fft_reg.cuh"
#include "tma.cuh"

namespace em3d {

// Row-pass load modes: plain, chi u with the EM contrast stored as 9
// (full), 6 (symmetric: xx yy zz xy xz yz) or 1 (isotropic: chi = s I)
// components per cell, scalar acoustic chi u.  Store modes: plain, u - y,
// v - chi^H y for the three EM layouts, v - conj(chi) y (acoustic).
enum { FLD_PLAIN = 0, FLD_EM_CHI = 1, FLD_AC_CHI = 2, FLD_EM_CHI6 = 3, FLD_EM_CHI1 = 4 };
enum { FST_PLAIN = 0, FST_SUB = 1, FST_EM_ADJ = 2, FST_AC_ADJ = 3, FST_EM_ADJ6 = 4, FST_EM_ADJ1 = 5,
       FST_SUB_DOTS = 6 };  // u - y, and the CTA's partial sums of |t|^2 and vdot(t, w) (t = u - y; w = bs.dot_with, else u) into bs.dots

// Elements per thread: power-of-two axes 16 (complex64) or 8 (complex128);
// mixed axes 12 (3 x 2^k) or 20 (5 x 2^k).
template <typename R, int L> struct FastE {
  static constexpr int E = (L & (L - 1)) == 0 ? (sizeof(R) == 4 ? 16 : 8) : (L % 5 == 0 ? 20 : 12);
};

// NTGT: the CTA size aimed at (C * RPB * TT threads, RPB rows per CTA).
template <int L, int E, int C, int NTGT = 256> struct RowsGeom {
  static constexpr int TT = L / E;
  static constexpr int RPB = (NTGT / (C * TT)) > 0 ? (NTGT / (C * TT)) : 1;
  static constexpr int NT = C * RPB * TT;
  static constexpr int PSTRIDE = rows_pencil_stride(L);
};

// Rows along z.  Forward (INV = false): input rows of length L/2 (pruned),
// output rows of length L.  Inverse: input rows of length L, output the
// first L/2 (crop).  One thread handles one (component, row) pencil slice.
// The body works on CTA `blk` of the pass (blockIdx.x in its own launch, a
// CTA of one segment in an application over problems of uneven sizes).
// Entries' fields (the forward pass's input, the inverse pass's output and
// base) lie bs.field elements apart, or back to back when bs.field is 0.
template <typename R, int L, int C, int LD, int ST, bool INV, int NTGT>
__device__ __forceinline__ void rows_body(const cx<R>* in, const cx<R>* __restrict__ chi, const cx<R>* base,
                                          cx<R>* out, const cx<R>* __restrict__ twg, int rows_pb, int nrows,
                                          const BatchStrides& bs, const int* skip, int blk) {
  using T = cx<R>;
  constexpr int E = FastE<R, L>::E;
  using G = RowsGeom<L, E, C, NTGT>;
  using P = RegPlan<L, E>;
  constexpr int TT = G::TT, RPB = G::RPB;
  constexpr int R1 = P::first(false), RL = P::last(false);
  constexpr int M1 = L / R1, ML = L / RL;
  constexpr int LIN = INV ? L : L / 2;
  constexpr int LOUT = INV ? L / 2 : L;
  if (skip_launch(skip)) return;
  {
    const int g0 = blk * RPB, g1 = min(g0 + RPB, nrows) - 1;
    if (entries_done(bs, g0 / rows_pb, g1 / rows_pb)) return;
  }
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tw = reinterpret_cast<T*>(smem_raw);
  T* sm = tw + L;
  for (int i = threadIdx.x; i < L; i += blockDim.x) tw[i] = twg[i];
  const int t = threadIdx.x % TT;
  const int pen = threadIdx.x / TT;
  const int c = pen / RPB, rl = pen - c * RPB;
  const int g = blk * RPB + rl;
  // rows of stopped entries are treated like rows past the end (no loads, no stores)
  const bool valid = g < nrows && !entry_done(bs, g / rows_pb);
  const int b = valid ? g / rows_pb : 0;
  const int row = valid ? g - b * rows_pb : 0;
  const cx<R>* chb = chi ? chi + (size_t)b * bs.chi : nullptr;
  // element offsets of entry b's input and output
  const size_t ib = (size_t)b * ((!INV && bs.field) ? bs.field : (size_t)C * rows_pb * LIN);
  const size_t ob = (size_t)b * ((INV && bs.field) ? bs.field : (size_t)C * rows_pb * LOUT);

  T a[1][E];
#pragma unroll
  for (int q = 0; q < E / R1; ++q) {
    const int j = t + q * TT;
#pragma unroll
    for (int r = 0; r < R1; ++r) {
      const int pos = j + r * M1;
      T v = mk<R>(0, 0);
      if (valid && (INV || r < R1 / 2)) {
        if constexpr (LD == FLD_EM_CHI) {
          const size_t o = (size_t)row * LIN + pos;
          const size_t cs = (size_t)rows_pb * LIN;
          const T* ub = in + ib;
#pragma unroll
          for (int k = 0; k < 3; ++k) v = cadd(v, cmul(chb[(size_t)(c * 3 + k) * cs + o], ub[k * cs + o]));
        } else if constexpr (LD == FLD_EM_CHI6) {
          const size_t o = (size_t)row * LIN + pos;
          const size_t cs = (size_t)rows_pb * LIN;
          const T* ub = in + ib;
#pragma unroll
          for (int k = 0; k < 3; ++k) v = cadd(v, cmul(chb[(size_t)sym_index(c, k) * cs + o], ub[k * cs + o]));
        } else if constexpr (LD == FLD_EM_CHI1) {
          const size_t o = (size_t)row * LIN + pos;
          v = cmul(chb[o], in[ib + (size_t)c * rows_pb * LIN + o]);
        } else if constexpr (LD == FLD_AC_CHI) {
          v = cmul(chb[(size_t)row * LIN + pos], in[ib + (size_t)row * LIN + pos]);
        } else {
          v = in[ib + ((size_t)c * rows_pb + row) * LIN + pos];
        }
      }
      a[0][q * R1 + r] = v;
    }
  }
  // u - y (the last pass of a matvec) or v - chi^H y (of an adjoint): u or v
  // at this thread's output positions is loaded before the transform, so its
  // latency overlaps the butterflies
  constexpr bool PRE = INV && ST != FST_PLAIN;
  T pre[PRE ? E / 2 : 1];
  if constexpr (PRE) {
#pragma unroll
    for (int q = 0; q < E / RL; ++q) {
      const int j = t + q * TT;
#pragma unroll
      for (int r = 0; r < RL / 2; ++r)
        pre[q * (RL / 2) + r] = valid ? base[ob + ((size_t)c * rows_pb + row) * LOUT + j + r * ML] : mk<R>(0, 0);
    }
  }
  __syncthreads();
  const LayRows lay{pen * G::PSTRIDE, G::PSTRIDE};
  reg_fft<L, E, INV, false, 1, !INV>(a, t, sm, tw, lay);

  if constexpr (ST == FST_EM_ADJ || ST == FST_EM_ADJ6) {
    // v - chi^H y needs all three components of y at each z: stage y through
    // shared memory (the last exchange ended with a sync).
#pragma unroll
    for (int q = 0; q < E / RL; ++q) {
      const int j = t + q * TT;
#pragma unroll
      for (int r = 0; r < RL / 2; ++r) sm[lay(0, j + r * ML)] = a[0][q * RL + r];
    }
    __syncthreads();
    if (!valid) return;
    const size_t cs = (size_t)rows_pb * LOUT;
#pragma unroll
    for (int q = 0; q < E / RL; ++q) {
      const int j = t + q * TT;
#pragma unroll
      for (int r = 0; r < RL / 2; ++r) {
        const int pos = j + r * ML;
        const size_t o = (size_t)row * LOUT + pos;
        T acc = mk<R>(0, 0);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const T yk = sm[(k * RPB + rl) * G::PSTRIDE + pos + (pos >> 4)];
          const int ci = ST == FST_EM_ADJ ? k * 3 + c : sym_index(k, c);
          acc = cadd(acc, cmulcj(chb[(size_t)ci * cs + o], yk));
        }
        const size_t oo = ob + (size_t)c * cs + o;
        out[oo] = csub(pre[q * (RL / 2) + r], acc);
      }
    }
    return;
  } else if constexpr (ST == FST_SUB_DOTS) {
    // every thread takes part in the CTA's reduction (no early return); the
    // exchange buffer, free once the transform is done, holds the partials
    double d0 = 0.0, d1 = 0.0, d2 = 0.0;
    const T* wv = static_cast<const T*>(bs.dot_with);
    if (valid) {
#pragma unroll
      for (int q = 0; q < E / RL; ++q) {
        const int j = t + q * TT;
#pragma unroll
        for (int r = 0; r < RL / 2; ++r) {
          const int pos = j + r * ML;
          const size_t oo = ob + ((size_t)c * rows_pb + row) * LOUT + pos;
          const T s = pre[q * (RL / 2) + r];
          const T v = csub(s, a[0][q * RL + r]);
          out[oo] = v;
          const T w = wv ? wv[oo] : s;
          d0 += (double)v.x * v.x + (double)v.y * v.y;
          d1 += (double)v.x * w.x + (double)v.y * w.y;
          d2 += (double)v.x * w.y - (double)v.y * w.x;
        }
      }
    }
    const int nt = blockDim.x;
    double* red = reinterpret_cast<double*>(sm);  // 3 x nt doubles
    __syncthreads();  // every thread is past its last read of the exchange buffer
    red[threadIdx.x] = d0;
    red[nt + threadIdx.x] = d1;
    red[2 * nt + threadIdx.x] = d2;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
      if ((int)threadIdx.x < h && (int)threadIdx.x + h < nt) {
#pragma unroll
        for (int k = 0; k < 3; ++k) red[k * nt + threadIdx.x] += red[k * nt + threadIdx.x + h];
      }
      __syncthreads();
    }
    if (threadIdx.x < 3) bs.dots[(size_t)blk * 3 + threadIdx.x] = red[threadIdx.x * nt];
    return;
  } else {
    if (!valid) return;
#pragma unroll
    for (int q = 0; q < E / RL; ++q) {
      const int j = t + q * TT;
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        if (INV && r >= RL / 2) continue;
        const int pos = j + r * ML;
        const T y = a[0][q * RL + r];
        const size_t oo = ob + ((size_t)c * rows_pb + row) * LOUT + pos;
        if constexpr (ST == FST_PLAIN) out[oo] = y;
        else if constexpr (ST == FST_SUB) out[oo] = csub(PRE ? pre[q * (RL / 2) + r] : base[oo], y);
        else if constexpr (ST == FST_AC_ADJ || ST == FST_EM_ADJ1)  // chi^H y = conj(s) y per component
          out[oo] = csub(PRE ? pre[q * (RL / 2) + r] : base[oo], cmulcj(chb[(size_t)row * LOUT + pos], y));
      }
    }
  }
}

template <typename R, int L, int C, int LD, int ST, bool INV>
__global__ void __launch_bounds__(RowsGeom<L, FastE<R, L>::E, C>::NT)
kf_rows(const cx<R>* in, const cx<R>* __restrict__ chi, const cx<R>* base, cx<R>* out,
        const cx<R>* __restrict__ twg, int rows_pb, int nrows, BatchStrides bs, const int* skip) {
  rows_body<R, L, C, LD, ST, INV, 256>(in, chi, base, out, twg, rows_pb, nrows, bs, skip, blockIdx.x);
}

template <int L, int E> struct StridedGeom {
  static constexpr int TT = L / E;
  static constexpr int P = (256 / TT) >= 8 ? (256 / TT) : 8;
  static constexpr int NT = P * TT;
  static constexpr int S = (P & 1) ? P : P + 1;
};

// Pencils along y: in (outer, L/2 or L, inner) -> out (outer, L or L/2, inner).
// The body works on CTA `blk` of the pass (see rows_body).
template <typename R, int L, bool INV>
__device__ __forceinline__ void strided_body(const cx<R>* in, cx<R>* out, const cx<R>* __restrict__ twg, int inner,
                                             int ntiles, const BatchStrides& bs, const int* skip, int blk) {
  using T = cx<R>;
  constexpr int E = FastE<R, L>::E;
  using G = StridedGeom<L, E>;
  using PL = RegPlan<L, E>;
  constexpr int TT = G::TT, PP = G::P, S = G::S;
  constexpr int R1 = PL::first(false), RL = PL::last(false);
  constexpr int M1 = L / R1, ML = L / RL;
  constexpr int LIN = INV ? L : L / 2;
  constexpr int LOUT = INV ? L / 2 : L;
  if (skip_launch(skip)) return;
  if (bs.done && entry_done(bs, (blk / ntiles) / bs.outer)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tw = reinterpret_cast<T*>(smem_raw);
  T* sm = tw + L;
  for (int i = threadIdx.x; i < L; i += blockDim.x) tw[i] = twg[i];
  const int p = threadIdx.x % PP, t = threadIdx.x / PP;
  const int o = blk / ntiles;
  const int i = (blk - o * ntiles) * PP + p;
  const bool valid = i < inner;
  const T* src = in + (size_t)o * LIN * inner + i;
  T a[1][E];
#pragma unroll
  for (int q = 0; q < E / R1; ++q) {
    const int j = t + q * TT;
#pragma unroll
    for (int r = 0; r < R1; ++r) {
      const int pos = j + r * M1;
      a[0][q * R1 + r] = (valid && (INV || r < R1 / 2)) ? src[(size_t)pos * inner] : mk<R>(0, 0);
    }
  }
  __syncthreads();
  const LayInter lay{p, S, 0};
  reg_fft<L, E, INV, false, 1, !INV>(a, t, sm, tw, lay);
  if (!valid) return;
  T* dst = out + (size_t)o * LOUT * inner + i;
#pragma unroll
  for (int q = 0; q < E / RL; ++q) {
    const int j = t + q * TT;
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      if (INV && r >= RL / 2) continue;
      dst[(size_t)(j + r * ML) * inner] = a[0][q * RL + r];
    }
  }
}

template <typename R, int L, bool INV>
__global__ void __launch_bounds__(StridedGeom<L, FastE<R, L>::E>::NT)
kf_strided(const cx<R>* in, cx<R>* out, const cx<R>* __restrict__ twg, int inner, int ntiles, BatchStrides bs,
           const int* skip) {
  strided_body<R, L, INV>(in, out, twg, inner, ntiles, bs, skip, blockIdx.x);
}

template <int L, int E, int C, int NTT = 256> struct XmulGeom {
  static constexpr int TT = L / E;
  static constexpr int P = (NTT / TT) > 32 ? 32 : ((NTT / TT) >= 4 ? (NTT / TT) : 4);
  static constexpr int NT = P * TT;
  static constexpr int S = (P & 1) ? P : P + 1;
  // small-E plans exchange one component at a time to keep shared memory small
  static constexpr bool SEQ = (E <= 8);
  static constexpr int REGIONS = SEQ ? 1 : C;
};

template <int L, int E, int R, int NSV, int RN, int C, typename T, class Lay>
__device__ __forceinline__ void reg_exchange_seq(T (&a)[C][E], int t, T* sm, const Lay& lay) {
  constexpr int TT = L / E;
#pragma unroll
  for (int c = 0; c < C; ++c) {
#pragma unroll
    for (int q = 0; q < E / R; ++q) {
      const int j = t + q * TT;
      const int bse = (j / NSV) * NSV * R + (j % NSV);
#pragma unroll
      for (int r = 0; r < R; ++r) sm[lay(0, bse + r * NSV)] = a[c][q * R + r];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < E / RN; ++q) {
      const int j = t + q * TT;
#pragma unroll
      for (int r = 0; r < RN; ++r) a[c][q * RN + r] = sm[lay(0, j + r * (L / RN))];
    }
    __syncthreads();
  }
}

template <int L, int E, bool INV, bool REV, int S, bool HALF_IN> struct RegFFTSeq {
  template <int C, typename T, class Lay>
  __device__ __forceinline__ static void run(T (&a)[C][E], int t, T* sm, const T* __restrict__ tw, const Lay& lay) {
    using P = RegPlan<L, E>;
    constexpr int R = P::rad(REV, S);
    constexpr int NSV = P::nsb(REV, S);
    reg_stage<L, E, R, NSV, INV, C, HALF_IN && S == 0>(a, t, tw);
    if constexpr (S + 1 < P::NS) {
      constexpr int RN = P::rad(REV, S + 1);
      reg_exchange_seq<L, E, R, NSV, RN, C>(a, t, sm, lay);
      RegFFTSeq<L, E, INV, REV, S + 1, HALF_IN>::template run<C>(a, t, sm, tw, lay);
    }
  }
};

template <int L, int E, bool INV, bool REV, bool SEQ, int C, typename T, class Lay>
__device__ __forceinline__ void reg_fft_x(T (&a)[C][E], int t, T* sm, const T* __restrict__ tw, const Lay& lay) {
  if constexpr (SEQ) RegFFTSeq<L, E, INV, REV, 0, !INV>::template run<C>(a, t, sm, tw, lay);
  else reg_fft<L, E, INV, REV, C, !INV>(a, t, sm, tw, lay);
}

__device__ __forceinline__ int kfold(int k, int n) { return k <= n ? k : 2 * n - k; }

// Pencils along x for one (batch, ky, kz tile): forward FFT, spectrum multiply
// in registers, reversed-plan inverse FFT, crop to x < Nx, in place in T2.
// The body works on CTA `blk` of the pass (see rows_body).
template <typename R, int L, int C, bool ADJ, int E, int NTT>
__device__ __forceinline__ void xmul_body(cx<R>* T2, const cx<R>* __restrict__ spec, const cx<R>* __restrict__ twg,
                                          int Ny, int Nz, int ntz, int nb, const BatchStrides& bs, const int* skip,
                                          int blk) {
  using T = cx<R>;
  using G = XmulGeom<L, E, C, NTT>;
  using PL = RegPlan<L, E>;
  constexpr int TT = G::TT, PP = G::P, S = G::S;
  constexpr int Nx = L / 2;
  constexpr int R1 = PL::first(false), RL = PL::last(false);
  constexpr int M1 = L / R1, ML = L / RL;
  if (skip_launch(skip)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tw = reinterpret_cast<T*>(smem_raw);
  T* sm = tw + L;
  for (int i = threadIdx.x; i < L; i += blockDim.x) tw[i] = twg[i];
  const int p = threadIdx.x % PP, t = threadIdx.x / PP;
  // batch index fastest: consecutive CTAs share one spectrum tile in L2
  int idx = blk;
  const int b = idx % nb;
  idx /= nb;
  const int tile = idx % ntz;
  const int ky = idx / ntz;
  if (entry_done(bs, b)) return;
  const int Ny2 = 2 * Ny, Nz2 = 2 * Nz;
  const int kz = tile * PP + p;
  const bool valid = kz < Nz2;
  const size_t xstride = (size_t)Ny2 * Nz2;
  T* col = T2 + (size_t)b * C * Nx * xstride + (size_t)ky * Nz2 + kz;

  T a[C][E];
#pragma unroll
  for (int q = 0; q < E / R1; ++q) {
    const int j = t + q * TT;
#pragma unroll
    for (int r = 0; r < R1; ++r) {
      const int x = j + r * M1;
#pragma unroll
      for (int c = 0; c < C; ++c)
        a[c][q * R1 + r] = (valid && r < R1 / 2) ? col[((size_t)c * Nx + x) * xstride] : mk<R>(0, 0);
    }
  }
  __syncthreads();
  const LayInter lay{p, S, L * S};
  reg_fft_x<L, E, false, false, G::SEQ, C>(a, t, sm, tw, lay);

  // spectrum multiply on the forward outputs kx = j + r * ML
  const int jy = kfold(ky, Ny);
  const int l = kfold(valid ? kz : 0, Nz);
  const size_t ostride = (size_t)(Nx + 1) * (Ny + 1) * (Nz + 1);
  const T* sp = spec + (size_t)b * bs.spec + (size_t)jy * (Nz + 1) + l;
  const R sy = ky <= Ny ? (R)1 : (R)-1;
  const R sz = kz <= Nz ? (R)1 : (R)-1;
#pragma unroll
  for (int q = 0; q < E / RL; ++q) {
    const int j = t + q * TT;
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      const int kx = j + r * ML;
      const int ix = kfold(kx, Nx);
      const T* s0 = sp + (size_t)ix * (Ny + 1) * (Nz + 1);
      const int e = q * RL + r;
      if constexpr (C == 1) {
        const T k0 = valid ? s0[0] : mk<R>(0, 0);
        a[0][e] = ADJ ? cmulcj(k0, a[0][e]) : cmul(k0, a[0][e]);
      } else {
        const R sx = kx <= Nx ? (R)1 : (R)-1;
        T kxx = mk<R>(0, 0), kyy = kxx, kzz = kxx, kxy = kxx, kxz = kxx, kyz = kxx;
        if (valid) {
          kxx = s0[0]; kyy = s0[ostride]; kzz = s0[2 * ostride];
          kxy = cscale(s0[3 * ostride], sx * sy);
          kxz = cscale(s0[4 * ostride], sx * sz);
          kyz = cscale(s0[5 * ostride], sy * sz);
        }
        if (ADJ) { kxx = cconj(kxx); kyy = cconj(kyy); kzz = cconj(kzz); kxy = cconj(kxy); kxz = cconj(kxz); kyz = cconj(kyz); }
        const T X0 = a[0][e], X1 = a[1][e], X2 = a[2][e];
        a[0][e] = cadd(cadd(cmul(kxx, X0), cmul(kxy, X1)), cmul(kxz, X2));
        a[1][e] = cadd(cadd(cmul(kxy, X0), cmul(kyy, X1)), cmul(kyz, X2));
        a[2][e] = cadd(cadd(cmul(kxz, X0), cmul(kyz, X1)), cmul(kzz, X2));
      }
    }
  }
  reg_fft_x<L, E, true, true, G::SEQ, C>(a, t, sm, tw, lay);
  if (!valid) return;
  // reversed plan: last inverse stage has radix R1, outputs x = j + r * M1
#pragma unroll
  for (int q = 0; q < E / R1; ++q) {
    const int j = t + q * TT;
#pragma unroll
    for (int r = 0; r < R1 / 2; ++r) {
      const int x = j + r * M1;
#pragma unroll
      for (int c = 0; c < C; ++c) col[((size_t)c * Nx + x) * xstride] = a[c][q * R1 + r];
    }
  }
}

template <typename R, int L, int C, bool ADJ, int E, int NTT>
__global__ void __launch_bounds__(XmulGeom<L, E, C, NTT>::NT)
kf_xmul(cx<R>* T2, const cx<R>* __restrict__ spec, const cx<R>* __restrict__ twg, int Ny, int Nz, int ntz,
        int nb, BatchStrides bs, const int* skip) {
  xmul_body<R, L, C, ADJ, E, NTT>(T2, spec, twg, Ny, Nz, ntz, nb, bs, skip, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Pipelined x pass: a persistent CTA loops over (batch, ky, kz-tile) tiles and
// prefetches the next tile's field slab (C x Nx x P) and spectrum slab
// (6 or 1 x (Nx+1) x P, octant-folded) into shared memory with cp.async while
// it transforms the current tile, so the global loads overlap the FFTs.
//
// Per tile:  wait field(i) -> registers -> prefetch field(i+1) -> forward FFT
//            -> wait spectrum(i) -> 3x3 multiply -> prefetch spectrum(i+1)
//            -> reversed inverse FFT -> crop and store (in place; tiles are
//            disjoint, so the prefetch never reads what another tile writes).
// Exactly two cp.async groups are committed per tile (empty ones at the end),
// so "wait until at most one group is pending" always targets the right one.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void cp_async_el(void* dst, const void* src, int bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if (bytes == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// Exchange layout of the pipelined x pass: element pos of pencil p at
// pos * P + p + 2 (pos / 4).  The shift by two words every four positions
// spreads both the stage-output stores (stride R positions per thread) and
// the next stage's loads over distinct banks for the 8-pencil tiles (a plain
// odd stride P + 1 gives them two-way conflicts there).
template <int P> struct LayPipe {
  int p;
  __device__ __forceinline__ int operator()(int c, int pos) const { return pos * P + p + 2 * (pos >> 2); }
};

// Batch entries per work unit of the pipelined x pass: up to 4 when the batch
// shares one spectrum (the slab is then loaded once for up to 8 tiles), 1 for
// a group of operators.  Small units keep the CTAs' loads balanced.
__host__ __device__ inline int xpipe_entries_per_unit(int nb, bool shared) {
  return !shared ? 1 : (nb % 4 == 0 ? 4 : (nb % 2 == 0 ? 2 : 1));
}

template <int L, int E, int C, int NTT> struct XpipeGeom {
  static constexpr int TT = L / E;
  static constexpr int P = (NTT / TT) > 32 ? 32 : ((NTT / TT) >= 2 ? (NTT / TT) : 2);
  static constexpr int NT = P * TT;
  static constexpr int S = (P & 1) ? P : P + 1;
  static constexpr int NX = L / 2;
  static constexpr int NSPEC = C == 3 ? 6 : 1;
  static constexpr int TW = L;
  static constexpr int EXCH = L * P + L / 2;   // LayPipe
  static constexpr int FIELD = C * NX * P;
  static constexpr int SPEC = NSPEC * (NX + 1) * P;
  static constexpr int TOTAL = TW + EXCH + FIELD + SPEC;   // complex elements of shared memory
  static constexpr size_t BYTES_EXTRA = 16;                  // the TMA mbarrier after the slabs
};

// TMAF: the field slab arrives by TMA (one tile load per component, issued by
// thread 0 and completed on an mbarrier; `fmap` describes T2 as (kz words,
// ky, batch * C * Nx rows)) instead of per-thread cp.async copies.
// The body runs as CTA `blk` of `nblk` persistent CTAs (blockIdx.x of gridDim.x
// in its own launch; a segment's share of CTAs in an application over problems
// of uneven sizes); `fmap` points to the field map in the parameter block.
template <typename R, int L, int C, bool ADJ, int E, int NTT, bool TMAF>
__device__ __forceinline__ void xpipe_body(cx<R>* T2, const cx<R>* __restrict__ spec,
                                           const cx<R>* __restrict__ twg, int Ny, int Nz, int ntz, int nb,
                                           const BatchStrides& bs, const int* skip, const CUtensorMap* fmap,
                                           int* status, int blk, int nblk) {
  using T = cx<R>;
  using G = XpipeGeom<L, E, C, NTT>;
  using PL = RegPlan<L, E>;
  constexpr int TT = G::TT, PP = G::P, NX = G::NX;
  constexpr int R1 = PL::first(false), RL = PL::last(false);
  constexpr int M1 = L / R1, ML = L / RL;
  constexpr int EB = (int)sizeof(T);
  if (skip_launch(skip)) return;
  extern __shared__ __align__(128) unsigned char smem_pipe[];
  // the field slab first: TMA writes it at a 128-byte aligned address
  T* sfield = reinterpret_cast<T*>(smem_pipe);
  T* tw = sfield + G::FIELD;
  T* sm = tw + G::TW;
  T* sspec = sm + G::EXCH;
  uint64_t* fbar = reinterpret_cast<uint64_t*>(sspec + G::SPEC);
  for (int i = threadIdx.x; i < L; i += blockDim.x) tw[i] = twg[i];
  if constexpr (TMAF) {
    if (threadIdx.x == 0) {
      mbar_init(fbar, 1);
      mbar_init_fence();
    }
    __syncthreads();
  }
  uint32_t fphase = 0;
  const int p = threadIdx.x % PP, t = threadIdx.x / PP;
  const int Ny2 = 2 * Ny, Nz2 = 2 * Nz;
  const size_t xstride = (size_t)Ny2 * Nz2;
  const size_t ostride = (size_t)(NX + 1) * (Ny + 1) * (Nz + 1);
  // Work units (jy, kz tile) with jy = 0..Ny: the tiles ky = jy and
  // ky = 2Ny - jy (one tile when jy is 0 or Ny) fold to the same spectrum
  // rows, and when the batch shares one spectrum (bs.spec == 0) so do its
  // entries; a unit covers nbu entries, whose tiles a CTA transforms in a row
  // (entry-major, then the two ky), loading the spectrum slab once.
  const int nbu = xpipe_entries_per_unit(nb, bs.spec == 0);
  const int ngroups = nb / nbu;                 // units per (jy, kz tile)
  const int nunits = ngroups * (Ny + 1) * ntz;
  auto decode = [&](int u, int& bg, int& jy, int& kz0) {
    bg = u % ngroups;
    const int idx = u / ngroups;
    kz0 = (idx % ntz) * PP;
    jy = idx / ntz;
  };
  auto nmirror = [&](int jy) { return (jy == 0 || jy == Ny) ? 1 : 2; };
  // Prefetch loops: a thread always copies the kz lane p of its pencil and
  // steps through the rows (component x position, or spectrum component x
  // folded kx) with a constant stride, so the addresses are incremental.
  constexpr int RSTEP = G::NT / PP;
  auto issue_field = [&](int u, int sub) {
    int bg, jy, kz0;
    decode(u, bg, jy, kz0);
    const int b = bg * nbu + sub / nmirror(jy);
    const int ky = (sub % nmirror(jy)) ? Ny2 - jy : jy;
    if (entry_done(bs, b)) return;
    if constexpr (TMAF) {
      // kz words of 8 bytes: one per complex64, two per complex128; rows
      // past Nz2 (the last tile) are filled with zeros by the TMA unit
      constexpr int W = EB / 8;
      if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(fbar, (uint32_t)(C * NX * PP * EB));
#pragma unroll
        for (int c = 0; c < C; ++c) tma_load_3d(sfield + c * NX * PP, fmap, fbar, kz0 * W, ky, (b * C + c) * NX);
      }
      return;
    }
    const bool ok = kz0 + p < Nz2;
    int row = threadIdx.x / PP;                       // c * NX + x
    const T* src = T2 + (size_t)b * C * NX * xstride + (size_t)ky * Nz2 + kz0 + p + (size_t)row * xstride;
    T* dst = sfield + row * PP + p;
    for (; row < C * NX; row += RSTEP, src += (size_t)RSTEP * xstride, dst += RSTEP * PP) {
      if (ok) cp_async_el(dst, src, EB);
      else *dst = mk<R>(0, 0);
    }
  };
  auto issue_spec = [&](int u) {
    int b, jy, kz0;
    decode(u, b, jy, kz0);  // with one entry per unit, b is that entry
    if (nbu == 1 && entry_done(bs, b)) return;
    const int kz = kz0 + p;
    const bool ok = kz < Nz2;
    const T* base = spec + (size_t)b * bs.spec + (size_t)jy * (Nz + 1) + (ok ? kfold(kz, Nz) : 0);
    const size_t xs = (size_t)(Ny + 1) * (Nz + 1);
    int row = threadIdx.x / PP;                       // component * (NX + 1) + ix
    int sc = row / (NX + 1), ix = row - sc * (NX + 1);
    T* dst = sspec + row * PP + p;
    for (; row < G::SPEC / PP; row += RSTEP, dst += RSTEP * PP) {
      if (ok) cp_async_el(dst, base + sc * ostride + ix * xs, EB);
      else *dst = mk<R>(0, 0);
      ix += RSTEP;
      while (ix > NX) { ix -= NX + 1; ++sc; }
    }
  };

  int u = blk, sub = 0;
  if (u < nunits) issue_field(u, 0);
  cp_async_commit();
  if (u < nunits) issue_spec(u);
  cp_async_commit();
  const LayPipe<PP> lay{p};

  while (u < nunits) {
    int bg, jy, kz0;
    decode(u, bg, jy, kz0);
    const int b = bg * nbu + sub / nmirror(jy);
    const int ky = (sub % nmirror(jy)) ? Ny2 - jy : jy;
    const int kz = kz0 + p;
    const bool valid = kz < Nz2;
    // the next tile: the unit's next (entry, ky), else the CTA's next unit
    int nu = u, ns = sub + 1;
    if (ns >= nbu * nmirror(jy)) {
      nu = u + nblk;
      ns = 0;
    }
    // the same for every thread of the CTA, so the barriers below stay uniform
    const bool live = !entry_done(bs, b);

    cp_async_wait_one();  // this tile's field slab
    __syncthreads();
    if constexpr (TMAF) {
      if (live) {  // uniform over the CTA
        const bool arrived = mbar_wait_bounded(fbar, fphase);
        if (!__syncthreads_and(arrived)) {
          // the field slab never arrived: count it once, give the copy still in
          // flight one more bounded wait, issue nothing further and leave (the
          // host reads the count and reports the application as failed)
          if (threadIdx.x == 0 && status != nullptr) atomicAdd(status, 1);
          mbar_wait_bounded(fbar, fphase);
          cp_async_wait_all();
          return;
        }
        fphase ^= 1u;
      }
    }
    T a[C][E];
#pragma unroll
    for (int q = 0; q < E / R1; ++q) {
      const int j = t + q * TT;
#pragma unroll
      for (int r = 0; r < R1; ++r) {
        const int x = j + r * M1;
#pragma unroll
        for (int c = 0; c < C; ++c) a[c][q * R1 + r] = r < R1 / 2 ? sfield[(c * NX + x) * PP + p] : mk<R>(0, 0);
      }
    }
    if constexpr (TMAF) fence_proxy_async_smem();  // these reads before the next tile's TMA overwrite
    __syncthreads();
    if (nu < nunits) issue_field(nu, ns);
    cp_async_commit();

    if (live) reg_fft_x<L, E, false, false, true, C>(a, t, sm, tw, lay);

    cp_async_wait_one();  // this tile's spectrum slab
    __syncthreads();
    const R sy = ky <= Ny ? (R)1 : (R)-1;
    const R sz = kz <= Nz ? (R)1 : (R)-1;
#pragma unroll
    for (int q = 0; q < E / RL; ++q) {
      const int j = t + q * TT;
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int kx = j + r * ML;
        const T* s0 = sspec + kfold(kx, NX) * PP + p;
        const int e = q * RL + r;
        if constexpr (C == 1) {
          const T k0 = s0[0];
          a[0][e] = ADJ ? cmulcj(k0, a[0][e]) : cmul(k0, a[0][e]);
        } else {
          constexpr int OS = (NX + 1) * PP;
          const R sx = kx <= NX ? (R)1 : (R)-1;
          T kxx = s0[0], kyy = s0[OS], kzz = s0[2 * OS];
          T kxy = cscale(s0[3 * OS], sx * sy);
          T kxz = cscale(s0[4 * OS], sx * sz);
          T kyz = cscale(s0[5 * OS], sy * sz);
          if (ADJ) { kxx = cconj(kxx); kyy = cconj(kyy); kzz = cconj(kzz); kxy = cconj(kxy); kxz = cconj(kxz); kyz = cconj(kyz); }
          const T X0 = a[0][e], X1 = a[1][e], X2 = a[2][e];
          a[0][e] = cadd(cadd(cmul(kxx, X0), cmul(kxy, X1)), cmul(kxz, X2));
          a[1][e] = cadd(cadd(cmul(kxy, X0), cmul(kyy, X1)), cmul(kyz, X2));
          a[2][e] = cadd(cadd(cmul(kxz, X0), cmul(kyz, X1)), cmul(kzz, X2));
        }
      }
    }
    __syncthreads();
    if (nu < nunits && nu != u) issue_spec(nu);  // the mirrored tile keeps this slab
    cp_async_commit();

    if (live) reg_fft_x<L, E, true, true, true, C>(a, t, sm, tw, lay);
    if (valid && live) {
      T* col = T2 + (size_t)b * C * NX * xstride + (size_t)ky * Nz2 + kz;
#pragma unroll
      for (int q = 0; q < E / R1; ++q) {
        const int j = t + q * TT;
#pragma unroll
        for (int r = 0; r < R1 / 2; ++r) {
          const int x = j + r * M1;
#pragma unroll
          for (int c = 0; c < C; ++c) col[((size_t)c * NX + x) * xstride] = a[c][q * R1 + r];
        }
      }
    }
    u = nu;
    sub = ns;
  }
  cp_async_wait_all();
}

template <typename R, int L, int C, bool ADJ, int E, int NTT, bool TMAF, int MINB = 1>
__global__ void __launch_bounds__(XpipeGeom<L, E, C, NTT>::NT, MINB)
kf_xmul_pipe(cx<R>* T2, const cx<R>* __restrict__ spec, const cx<R>* __restrict__ twg, int Ny, int Nz, int ntz,
             int nb, BatchStrides bs, const int* skip, const __grid_constant__ CUtensorMap fmap, int* status) {
  xpipe_body<R, L, C, ADJ, E, NTT, TMAF>(T2, spec, twg, Ny, Nz, ntz, nb, bs, skip, &fmap, status, blockIdx.x,
                                          gridDim.x);
}

// ---------------------------------------------------------------------------
// Component-split x pass (EM only): each thread transforms one component
// pencil slice, so a thread holds E elements instead of 3E; the 3x3 dyadic
// multiply reads the other two components of the same frequency through
// shared memory.  Small CTAs (PZ = 8 columns) let two CTAs share an SM, so
// one CTA's loads overlap the other's transforms.
// ---------------------------------------------------------------------------
template <int L, int E> struct XsplitGeom {
  static constexpr int TT = L / E;
  static constexpr int PZ = (384 / (3 * TT)) > 16 ? 16 : ((384 / (3 * TT)) < 2 ? 2 : (384 / (3 * TT)));
  static constexpr int NT = 3 * PZ * TT;
  static constexpr int S = (PZ & 1) ? PZ : PZ + 1;
  static constexpr int REGION = L * S;
};

template <typename R, int L, bool ADJ, int E>
__global__ void __launch_bounds__(XsplitGeom<L, E>::NT, 2)
kf_xmul_split(cx<R>* T2, const cx<R>* __restrict__ spec, const cx<R>* __restrict__ twg, int Ny, int Nz, int ntz,
              int nb, BatchStrides bs, const int* skip) {
  using T = cx<R>;
  using G = XsplitGeom<L, E>;
  using PL = RegPlan<L, E>;
  constexpr int TT = G::TT, PZ = G::PZ, S = G::S;
  constexpr int Nx = L / 2;
  constexpr int R1 = PL::first(false), RL = PL::last(false);
  constexpr int M1 = L / R1, ML = L / RL;
  if (skip_launch(skip)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tw = reinterpret_cast<T*>(smem_raw);
  T* sm = tw + L;
  for (int i = threadIdx.x; i < L; i += blockDim.x) tw[i] = twg[i];
  const int c = threadIdx.x / (PZ * TT);  // uniform per warp
  const int rem = threadIdx.x - c * (PZ * TT);
  const int p = rem % PZ, t = rem / PZ;
  // batch index fastest: consecutive CTAs share one spectrum tile in L2
  int idx = blockIdx.x;
  const int b = idx % nb;
  idx /= nb;
  const int tile = idx % ntz;
  const int ky = idx / ntz;
  if (entry_done(bs, b)) return;
  const int Ny2 = 2 * Ny, Nz2 = 2 * Nz;
  const int kz = tile * PZ + p;
  const bool valid = kz < Nz2;
  const size_t xstride = (size_t)Ny2 * Nz2;
  T* col = T2 + ((size_t)(b * 3 + c) * Nx) * xstride + (size_t)ky * Nz2 + kz;

  T a[1][E];
#pragma unroll
  for (int q = 0; q < E / R1; ++q) {
    const int j = t + q * TT;
#pragma unroll
    for (int r = 0; r < R1 / 2; ++r) a[0][q * R1 + r] = valid ? col[(size_t)(j + r * M1) * xstride] : mk<R>(0, 0);
#pragma unroll
    for (int r = R1 / 2; r < R1; ++r) a[0][q * R1 + r] = mk<R>(0, 0);
  }
  __syncthreads();
  const LayInter lay{c * G::REGION + p, S, 0};
  reg_fft<L, E, false, false, 1, true>(a, t, sm, tw, lay);

  // publish this component's spectrum values, then multiply by row c of the
  // symmetric dyadic block (blocks xx yy zz xy xz yz)
#pragma unroll
  for (int q = 0; q < E / RL; ++q) {
    const int j = t + q * TT;
#pragma unroll
    for (int r = 0; r < RL; ++r) sm[lay(0, j + r * ML)] = a[0][q * RL + r];
  }
  __syncthreads();
  const int bd = c;
  const int b1 = (c == 2) ? 4 : 3;
  const int b2 = (c == 0) ? 4 : 5;
  const int r1 = ((c == 0) ? 1 : 0) * G::REGION + p;  // shared-memory base of component c1
  const int r2 = ((c == 2) ? 1 : 2) * G::REGION + p;  // and of component c2
  const R sy = ky <= Ny ? (R)1 : (R)-1;
  const R sz = kz <= Nz ? (R)1 : (R)-1;
  // sign of block (c, c1) = sx * f1; of block (c, c2) = (c == 0 ? sx * sz : sy * sz)
  const R f1 = (c == 2) ? sz : sy;
  const bool b2x = (c == 0);
  const R syz = sy * sz;
  const int jy = kfold(ky, Ny);
  const int l = kfold(valid ? kz : 0, Nz);
  const size_t ostride = (size_t)(Nx + 1) * (Ny + 1) * (Nz + 1);
  const size_t rowstride = (size_t)(Ny + 1) * (Nz + 1);
  const T* sb0 = spec + (size_t)b * bs.spec;
  const T* spd = sb0 + bd * ostride + (size_t)jy * (Nz + 1) + l;
  const T* sp1 = sb0 + b1 * ostride + (size_t)jy * (Nz + 1) + l;
  const T* sp2 = sb0 + b2 * ostride + (size_t)jy * (Nz + 1) + l;
#pragma unroll
  for (int q = 0; q < E / RL; ++q) {
    const int j = t + q * TT;
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      const int kx = j + r * ML;
      const R sx = kx <= Nx ? (R)1 : (R)-1;
      const size_t o = (size_t)kfold(kx, Nx) * rowstride;
      T kd = mk<R>(0, 0), k1 = kd, k2 = kd;
      if (valid) {
        kd = spd[o];
        k1 = cscale(sp1[o], sx * f1);
        k2 = cscale(sp2[o], b2x ? sx * sz : syz);
      }
      if (ADJ) { kd = cconj(kd); k1 = cconj(k1); k2 = cconj(k2); }
      const T X1 = sm[kx * S + r1];
      const T X2 = sm[kx * S + r2];
      const int e = q * RL + r;
      a[0][e] = cadd(cadd(cmul(kd, a[0][e]), cmul(k1, X1)), cmul(k2, X2));
    }
  }
  __syncthreads();
  reg_fft<L, E, true, true, 1>(a, t, sm, tw, lay);
  if (!valid) return;
#pragma unroll
  for (int q = 0; q < E / R1; ++q) {
    const int j = t + q * TT;
#pragma unroll
    for (int r = 0; r < R1 / 2; ++r) col[(size_t)(j + r * M1) * xstride] = a[0][q * R1 + r];
  }
}

}  // namespace em3d
