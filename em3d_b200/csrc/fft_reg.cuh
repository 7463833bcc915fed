// Register-resident Stockham FFT for power-of-two lengths 32..1024 and the
// mixed lengths 96, 160 and 192.
//
// T = L / E threads cooperate on one pencil; each holds E elements in
// registers.  A stage of radix R (a power of two dividing E) runs E / R
// butterflies per thread: butterfly j = t + q T reads positions
// j + r L/R and writes expand(j) + r Ns, Ns = product of the earlier radices.
// Between stages the elements are exchanged through shared memory (one
// write, one sync, one read, one sync); the first stage reads its inputs
// straight from global memory and the last stage's outputs go straight back,
// so a two-stage transform touches shared memory once.
//
// Position sets at the two ends (used to fuse work into the transform):
//   first stage input  : j + r (L / R_first),  j = t + q T
//   last stage output  : j + r (L / R_last),   j = t + q T   (expand(j) = j)
// A plan and its reverse therefore meet without an exchange: the forward
// transform's outputs are exactly the reversed inverse transform's inputs,
// which is how the spectrum multiply sits between the two x transforms.
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace em3d {

__host__ __device__ constexpr int ilog2c(int x) { return x <= 1 ? 0 : 1 + ilog2c(x / 2); }

// Mixed-radix plans (L = 3 or 5 times a power of two).  The first and last
// radices are even, so the zero-padded half of a forward input and the
// cropped half of an inverse output are whole register groups, exactly as in
// the power-of-two plans; every radix divides E.
__host__ __device__ constexpr int mixed_stages(int L, int E) {
  return (L == 96 && E == 12) || (L == 192 && E == 12) || (L == 160 && E == 20) ? 3 : 0;
}
__host__ __device__ constexpr int mixed_radix(int L, int E, int s) {
  return s != 1 ? 4 : (L == 96 ? 6 : L == 192 ? 12 : 10);
}

template <int L, int E> struct RegPlan {
  static constexpr bool POW2 = (L & (L - 1)) == 0 && (E & (E - 1)) == 0;
  static_assert(L >= E && E >= 2 && (POW2 || mixed_stages(L, E) > 0), "no register plan for this length");
  static constexpr int A = ilog2c(L), EB = ilog2c(E);
  static constexpr int NS = POW2 ? (A + EB - 1) / EB : mixed_stages(L, E);
  static constexpr int T = L / E;
  __host__ __device__ static constexpr int bits(int s) { return A / NS + (s < A % NS ? 1 : 0); }
  // radix of stage s in forward (REV = false) or reversed order
  __host__ __device__ static constexpr int rad(bool rev, int s) {
    return POW2 ? 1 << bits(rev ? NS - 1 - s : s) : mixed_radix(L, E, rev ? NS - 1 - s : s);
  }
  __host__ __device__ static constexpr int nsb(bool rev, int s) {
    int n = 1;
    for (int i = 0; i < s; ++i) n *= rad(rev, i);
    return n;
  }
  __host__ __device__ static constexpr int first(bool rev) { return rad(rev, 0); }
  __host__ __device__ static constexpr int last(bool rev) { return rad(rev, NS - 1); }
  __host__ __device__ static constexpr bool valid() {
    for (int s = 0; s < NS; ++s)
      if (E % rad(false, s) != 0) return false;
    return nsb(false, NS) == L && first(false) % 2 == 0 && last(false) % 2 == 0;
  }
  static_assert(valid(), "register plan: radices must divide E, multiply to L, and start and end even");
};

// Twiddle-multiply and DFT of this thread's butterflies in one stage, for C
// pencils held as a[c][E] (register index q*R + r).
template <int L, int E, int R, int NSV, bool INV, int C, bool HALF_IN = false, typename T>
__device__ __forceinline__ void reg_stage(T (&a)[C][E], int t, const T* __restrict__ tw) {
  constexpr int TT = L / E;
  constexpr int Q = E / R;
  constexpr int TS = L / (NSV * R);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int j = t + q * TT;
    const int k = j % NSV;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      T* b = &a[c][q * R];
      if constexpr (NSV > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const T w = tw[r * k * TS];
          b[r] = INV ? cmulcj(w, b[r]) : cmul(w, b[r]);
        }
      }
      if constexpr (HALF_IN) dft_fixed_half_in<R, INV>(b);
      else dft_fixed<R, INV>(b);
    }
  }
}

// Write this stage's outputs to shared memory and read the next stage's inputs.
// lay(c, pos) gives the shared-memory index of element pos of pencil c.
template <int L, int E, int R, int NSV, int RN, int C, typename T, class Lay>
__device__ __forceinline__ void reg_exchange(T (&a)[C][E], int t, T* sm, const Lay& lay) {
  constexpr int TT = L / E;
#pragma unroll
  for (int q = 0; q < E / R; ++q) {
    const int j = t + q * TT;
    const int base = (j / NSV) * NSV * R + (j % NSV);
#pragma unroll
    for (int c = 0; c < C; ++c)
#pragma unroll
      for (int r = 0; r < R; ++r) sm[lay(c, base + r * NSV)] = a[c][q * R + r];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < E / RN; ++q) {
    const int j = t + q * TT;
#pragma unroll
    for (int c = 0; c < C; ++c)
#pragma unroll
      for (int r = 0; r < RN; ++r) a[c][q * RN + r] = sm[lay(c, j + r * (L / RN))];
  }
  __syncthreads();
}

template <int L, int E, bool INV, bool REV, int S, bool HALF_IN> struct RegFFT {
  template <int C, typename T, class Lay>
  __device__ __forceinline__ static void run(T (&a)[C][E], int t, T* sm, const T* __restrict__ tw, const Lay& lay) {
    using P = RegPlan<L, E>;
    constexpr int R = P::rad(REV, S);
    constexpr int NSV = P::nsb(REV, S);
    reg_stage<L, E, R, NSV, INV, C, HALF_IN && S == 0>(a, t, tw);
    if constexpr (S + 1 < P::NS) {
      constexpr int RN = P::rad(REV, S + 1);
      reg_exchange<L, E, R, NSV, RN, C>(a, t, sm, lay);
      RegFFT<L, E, INV, REV, S + 1, HALF_IN>::template run<C>(a, t, sm, tw, lay);
    }
  }
};

// Full transform of C pencils in registers: inputs in first-stage order,
// outputs in last-stage order (see the header comment).  HALF_IN: the
// first-stage inputs with r >= R/2 are zero padding and are not read.
template <int L, int E, bool INV, bool REV, int C, bool HALF_IN = false, typename T, class Lay>
__device__ __forceinline__ void reg_fft(T (&a)[C][E], int t, T* sm, const T* __restrict__ tw, const Lay& lay) {
  RegFFT<L, E, INV, REV, 0, HALF_IN>::template run<C>(a, t, sm, tw, lay);
}

// Shared-memory layouts.
// Pencil-contiguous with one pad element per 16 (rows: threads of a pencil
// are consecutive, so the first stage's stride-R writes spread over banks).
struct LayRows {
  int base;    // this thread's first pencil
  int stride;  // elements per pencil incl. padding
  __device__ __forceinline__ int operator()(int c, int pos) const { return base + c * stride + pos + (pos >> 4); }
};
// Interleaved: element pos of pencil p at pos*S + p (strided passes: pencils
// of neighbouring threads are neighbours).
struct LayInter {
  int p;       // this thread's pencil
  int S;       // odd pencil stride
  int cstride; // offset between component pencils held by one thread
  __device__ __forceinline__ int operator()(int c, int pos) const { return pos * S + p + c * cstride; }
};

__host__ __device__ constexpr int rows_pencil_stride(int L) { return L + (L >> 4) + 1; }

}  // namespace em3d
