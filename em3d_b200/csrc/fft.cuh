// Batched mixed-radix Stockham FFT on pencils held in shared memory.
//
// A CTA holds P pencils of length L in shared memory, element k of pencil p
// at buf[k * S + p] with S = P + 1.  Interleaving the pencils makes the
// butterfly loads/stores of neighbouring threads hit neighbouring words, and
// the +1 pad keeps the transposing global<->shared copies of row-major data
// free of bank conflicts.  Each Stockham stage (radix R, Ns = product of the
// earlier radices) reads one buffer and writes the other; results come out in
// natural order, so no bit reversal pass exists.
//
// Sign convention (numpy.fft): forward X[q] = sum_n x[n] e^{-2 pi i q n / L};
// inverse is unnormalised (the 1/L of numpy's ifftn is folded into the
// operator spectrum at build time).
#pragma once

#include "common.cuh"

namespace em3d {

constexpr int kMaxStages = 12;
constexpr int kMaxLen = 1024;  // longest supported transform (doubled axis, N <= 512)

struct AxisPlan {
  int L;
  int nstages;
  int radix[kMaxStages];
};

// Factor L into Stockham stages: the power of two is split into as few radix
// 16/8/4/2 stages as possible, balanced; odd factors become radix 3 / 5
// stages or a generic odd-prime stage.  Returns false if L is unsupported.
inline bool make_axis_plan(int L, AxisPlan* pl) {
  if (L < 1 || L > kMaxLen) return false;
  pl->L = L;
  pl->nstages = 0;
  int n = L, e = 0;
  while ((n & 1) == 0) { n >>= 1; ++e; }
  int s2 = (e + 3) / 4;
  for (int i = 0; i < s2; ++i) {
    int bits = e / s2 + (i < e % s2 ? 1 : 0);
    if (pl->nstages >= kMaxStages) return false;
    pl->radix[pl->nstages++] = 1 << bits;
  }
  for (int f = 3; n > 1; f += 2) {
    while (n % f == 0) {
      if (f > 61 || pl->nstages >= kMaxStages) return false;  // generic stage bound
      pl->radix[pl->nstages++] = f;
      n /= f;
    }
  }
  return true;
}

// ---------------------------------------------------------------------------
// fixed-radix DFTs on registers
// ---------------------------------------------------------------------------

template <bool INV, typename C> __device__ __forceinline__ C rot_q(C a) {  // times w^1 of radix 4
  return INV ? mul_pi(a) : mul_mi(a);
}

// Butterfly sums use vadd / vsub (packed FP32x2 for complex64) wherever both
// operands are plain complex values; a sum with a value multiplied by -+i
// mixes real and imaginary lanes and uses the scalar cadd / csub.
template <bool INV, typename C> __device__ __forceinline__ void dft2(C& a0, C& a1) {
  C t = a0; a0 = vadd(t, a1); a1 = vsub(t, a1);
}

template <bool INV, typename C> __device__ __forceinline__ void dft4(C& a0, C& a1, C& a2, C& a3) {
  C t0 = vadd(a0, a2), t1 = vsub(a0, a2), t2 = vadd(a1, a3), t3 = rot_q<INV>(vsub(a1, a3));
  a0 = vadd(t0, t2); a2 = vsub(t0, t2); a1 = cadd(t1, t3); a3 = csub(t1, t3);
}

// radix 8 = two radix 4 on even/odd inputs, combined with w8^q
template <bool INV, typename C> __device__ __forceinline__ void dft8(C* a) {
  using R = decltype(a[0].x);
  const R h = (R)0.70710678118654752440;
  C e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6];
  C o0 = a[1], o1 = a[3], o2 = a[5], o3 = a[7];
  dft4<INV>(e0, e1, e2, e3);
  dft4<INV>(o0, o1, o2, o3);
  // w8^1 = (1 -+ i)/sqrt2, w8^2 = -+i, w8^3 = (-1 -+ i)/sqrt2
  C w1, w3;
  if (!INV) { w1 = mk<R>(h * (o1.x + o1.y), h * (o1.y - o1.x)); w3 = mk<R>(h * (o3.y - o3.x), -h * (o3.x + o3.y)); }
  else      { w1 = mk<R>(h * (o1.x - o1.y), h * (o1.y + o1.x)); w3 = mk<R>(-h * (o3.x + o3.y), h * (o3.x - o3.y)); }
  C w2 = rot_q<INV>(o2);
  a[0] = vadd(e0, o0); a[4] = vsub(e0, o0);
  a[1] = vadd(e1, w1); a[5] = vsub(e1, w1);
  a[2] = cadd(e2, w2); a[6] = csub(e2, w2);
  a[3] = vadd(e3, w3); a[7] = vsub(e3, w3);
}

// radix 16 = two radix 8 on even/odd inputs, combined with w16^q
template <bool INV, typename C> __device__ __forceinline__ void dft16(C* a) {
  using R = decltype(a[0].x);
  C e[8], o[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) { e[i] = a[2 * i]; o[i] = a[2 * i + 1]; }
  dft8<INV>(e);
  dft8<INV>(o);
  const R c1 = (R)0.92387953251128675613, s1 = (R)0.38268343236508977173;  // cos, sin of pi/8
  const R h = (R)0.70710678118654752440;
  const R cs[8] = {(R)1, c1, h, s1, (R)0, -s1, -h, -c1};
  const R sn[8] = {(R)0, s1, h, c1, (R)1, c1, h, s1};
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    // w16^q = cos(2 pi q/16) -+ i sin(2 pi q/16); q = 0 and q = 4 are exact
    C t;
    if (q == 4) {
      t = rot_q<INV>(o[4]);
      a[q] = cadd(e[q], t);
      a[q + 8] = csub(e[q], t);
      continue;
    }
    if (q == 0) t = o[0];
    else t = cmul(o[q], mk<R>(cs[q], INV ? sn[q] : -sn[q]));
    a[q] = vadd(e[q], t);
    a[q + 8] = vsub(e[q], t);
  }
}

// DFTs of length R whose inputs a[R/2 .. R-1] are zero (the zero-padded half
// of a forward transform):  y[2m] = DFT_{R/2}(a)[m],
// y[2m+1] = DFT_{R/2}(a[r] w_R^r)[m].  Only a[0 .. R/2-1] are read.
template <int RX, bool INV, typename C> __device__ __forceinline__ void dft_fixed_half_in(C* a) {
  using R = decltype(a[0].x);
  if constexpr (RX == 2) {
    a[1] = a[0];
  } else if constexpr (RX == 4) {
    C a0 = a[0], a1 = a[1];
    C w1 = rot_q<INV>(a1);
    a[0] = vadd(a0, a1); a[2] = cadd(a0, w1); a[1] = vsub(a0, a1); a[3] = csub(a0, w1);
    // natural order: y0 = E0, y1 = O0, y2 = E1, y3 = O1
    C y0 = a[0], y1 = a[2], y2 = a[1], y3 = a[3];
    a[0] = y0; a[1] = y1; a[2] = y2; a[3] = y3;
  } else if constexpr (RX == 8) {
    const R h = (R)0.70710678118654752440;
    C e0 = a[0], e1 = a[1], e2 = a[2], e3 = a[3];
    // odd half: a[r] * w8^r
    C o0 = a[0];
    C o1 = INV ? mk<R>(h * (a[1].x - a[1].y), h * (a[1].y + a[1].x)) : mk<R>(h * (a[1].x + a[1].y), h * (a[1].y - a[1].x));
    C o2 = rot_q<INV>(a[2]);
    C o3 = INV ? mk<R>(-h * (a[3].x + a[3].y), h * (a[3].x - a[3].y)) : mk<R>(h * (a[3].y - a[3].x), -h * (a[3].x + a[3].y));
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    a[0] = e0; a[1] = o0; a[2] = e1; a[3] = o1; a[4] = e2; a[5] = o2; a[6] = e3; a[7] = o3;
  } else if constexpr (RX == 16) {
    const R c1 = (R)0.92387953251128675613, s1 = (R)0.38268343236508977173;
    const R h = (R)0.70710678118654752440;
    const R cs[8] = {(R)1, c1, h, s1, (R)0, -s1, -h, -c1};
    const R sn[8] = {(R)0, s1, h, c1, (R)1, c1, h, s1};
    C e[8], o[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      e[r] = a[r];
      if (r == 0) o[r] = a[0];
      else if (r == 4) o[r] = rot_q<INV>(a[4]);
      else o[r] = cmul(a[r], mk<R>(cs[r], INV ? sn[r] : -sn[r]));
    }
    dft8<INV>(e);
    dft8<INV>(o);
#pragma unroll
    for (int m = 0; m < 8; ++m) { a[2 * m] = e[m]; a[2 * m + 1] = o[m]; }
  }
}

template <bool INV, typename C> __device__ __forceinline__ void dft3(C& a0, C& a1, C& a2) {
  using R = decltype(a0.x);
  const R s = (R)0.86602540378443864676;  // sqrt(3)/2
  C t = vadd(a1, a2), d = vsub(a1, a2);
  C m = mk<R>(a0.x - (R)0.5 * t.x, a0.y - (R)0.5 * t.y);
  a0 = vadd(a0, t);
  // forward: y1 = m - i s d, y2 = m + i s d
  C isd = mk<R>(-s * d.y, s * d.x);  // i s d
  if (!INV) { a1 = vsub(m, isd); a2 = vadd(m, isd); }
  else      { a1 = vadd(m, isd); a2 = vsub(m, isd); }
}

template <bool INV, typename C> __device__ __forceinline__ void dft5(C* a) {
  using R = decltype(a[0].x);
  const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;
  const R s1 = (R)0.95105651629515357212, s2 = (R)0.58778525229247312917;
  C t1 = vadd(a[1], a[4]), t2 = vadd(a[2], a[3]);
  C d1 = vsub(a[1], a[4]), d2 = vsub(a[2], a[3]);
  C a0 = a[0];
  C b1 = mk<R>(a0.x + c1 * t1.x + c2 * t2.x, a0.y + c1 * t1.y + c2 * t2.y);
  C b2 = mk<R>(a0.x + c2 * t1.x + c1 * t2.x, a0.y + c2 * t1.y + c1 * t2.y);
  C e1 = mk<R>(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y);
  C e2 = mk<R>(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y);
  C ie1 = mk<R>(-e1.y, e1.x), ie2 = mk<R>(-e2.y, e2.x);
  a[0] = vadd(a0, vadd(t1, t2));
  if (!INV) { a[1] = vsub(b1, ie1); a[4] = vadd(b1, ie1); a[2] = vsub(b2, ie2); a[3] = vadd(b2, ie2); }
  else      { a[1] = vadd(b1, ie1); a[4] = vsub(b1, ie1); a[2] = vadd(b2, ie2); a[3] = vsub(b2, ie2); }
}

// cos and sin of 2 pi m / n for n in {6, 10, 12} (compile-time m): the
// angles are multiples of 30 or 36 degrees, whose values are sqrt(3)/2, 1/2
// and (sqrt(5) +- 1)/4 with their complements.
__host__ __device__ constexpr double root_cos(int n, int m) {
  constexpr double h3 = 0.86602540378443864676, c36 = 0.80901699437494742410, c72 = 0.30901699437494742410;
  if (n == 6) return root_cos(12, 2 * m);
  if (n == 12) {
    constexpr double t[12] = {1.0, h3, 0.5, 0.0, -0.5, -h3, -1.0, -h3, -0.5, 0.0, 0.5, h3};
    return t[m % 12];
  }
  constexpr double t[10] = {1.0, c36, c72, -c72, -c36, -1.0, -c36, -c72, c72, c36};
  return t[m % 10];
}
__host__ __device__ constexpr double root_sin(int n, int m) {
  constexpr double h3 = 0.86602540378443864676, s36 = 0.58778525229247312917, s72 = 0.95105651629515357212;
  if (n == 6) return root_sin(12, 2 * m);
  if (n == 12) {
    constexpr double t[12] = {0.0, 0.5, h3, 1.0, h3, 0.5, 0.0, -0.5, -h3, -1.0, -h3, -0.5};
    return t[m % 12];
  }
  constexpr double t[10] = {0.0, s36, s72, s72, s36, 0.0, -s36, -s72, -s72, -s36};
  return t[m % 10];
}

template <int RX, bool INV, typename C> __device__ __forceinline__ void dft_fixed(C* a);

// Radix A*B in registers (Cooley-Tukey, n = B n1 + n2, k = k1 + A k2):
// B DFTs of length A on the inputs a[B n1 + n2], twiddles w_{AB}^{n2 k1},
// then A DFTs of length B giving X[k1 + A k2].
template <int A, int B, bool INV, typename C> __device__ __forceinline__ void dft_comp(C* a) {
  using R = decltype(a[0].x);
  constexpr int RX = A * B;
  C y[B][A];
#pragma unroll
  for (int n2 = 0; n2 < B; ++n2) {
#pragma unroll
    for (int n1 = 0; n1 < A; ++n1) y[n2][n1] = a[B * n1 + n2];
    dft_fixed<A, INV>(y[n2]);
#pragma unroll
    for (int k1 = 1; k1 < A; ++k1) {
      if (n2 == 0) continue;
      const int m = (n2 * k1) % RX;
      const R c = (R)root_cos(RX, m), s = (R)root_sin(RX, m);
      y[n2][k1] = cmul(y[n2][k1], mk<R>(c, INV ? s : -s));
    }
  }
#pragma unroll
  for (int k1 = 0; k1 < A; ++k1) {
    C z[B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) z[n2] = y[n2][k1];
    dft_fixed<B, INV>(z);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) a[k1 + A * k2] = z[k2];
  }
}

template <int RX, bool INV, typename C> __device__ __forceinline__ void dft_fixed(C* a) {
  if constexpr (RX == 2) dft2<INV>(a[0], a[1]);
  else if constexpr (RX == 3) dft3<INV>(a[0], a[1], a[2]);
  else if constexpr (RX == 4) dft4<INV>(a[0], a[1], a[2], a[3]);
  else if constexpr (RX == 5) dft5<INV>(a);
  else if constexpr (RX == 6) dft_comp<2, 3, INV>(a);
  else if constexpr (RX == 8) dft8<INV>(a);
  else if constexpr (RX == 10) dft_comp<2, 5, INV>(a);
  else if constexpr (RX == 12) dft_comp<4, 3, INV>(a);
  else if constexpr (RX == 16) dft16<INV>(a);
  else static_assert(RX == 2, "no fixed DFT for this radix");
}

// One Stockham stage with a compile-time radix.
template <int RX, bool INV, typename C>
__device__ __forceinline__ void stage_fixed(const C* __restrict__ in, C* __restrict__ out, const C* __restrict__ tw,
                                            int L, int P, int S, int Ns) {
  const int m = L / RX;
  const int twstep = L / (Ns * RX);
  const int total = m * P;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int p = t % P, j = t / P;
    const int k = j % Ns;
    C a[RX];
#pragma unroll
    for (int r = 0; r < RX; ++r) a[r] = in[(j + r * m) * S + p];
    if (k != 0) {
#pragma unroll
      for (int r = 1; r < RX; ++r) {
        C w = tw[r * k * twstep];
        a[r] = INV ? cmulcj(w, a[r]) : cmul(w, a[r]);
      }
    }
    dft_fixed<RX, INV>(a);
    const int ob = (j - k) * RX + k;
#pragma unroll
    for (int r = 0; r < RX; ++r) out[(ob + r * Ns) * S + p] = a[r];
  }
}

// Generic odd radix (prime factors without a fixed kernel): direct DFT reading
// the stage inputs from shared memory.  Only odd test sizes use it.
template <bool INV, typename C>
__device__ void stage_generic(const C* __restrict__ in, C* __restrict__ out, const C* __restrict__ tw,
                              int L, int P, int S, int Ns, int RX) {
  const int m = L / RX;
  const int twstep = L / (Ns * RX);
  const int dstep = L / RX;
  const int total = m * P;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int p = t % P, j = t / P;
    const int k = j % Ns;
    const int ob = (j - k) * RX + k;
    for (int q = 0; q < RX; ++q) {
      C acc = in[j * S + p];
      for (int r = 1; r < RX; ++r) {
        C x = in[(j + r * m) * S + p];
        C w = tw[r * k * twstep];
        x = INV ? cmulcj(w, x) : cmul(w, x);
        C d = tw[((q * r) % RX) * dstep];
        x = INV ? cmulcj(d, x) : cmul(d, x);
        acc = cadd(acc, x);
      }
      out[(ob + q * Ns) * S + p] = acc;
    }
  }
}

// Transform P pencils held in buffer a (b is scratch of the same size).
// Returns the buffer that holds the result.  Caller syncs before the call;
// the function ends with a sync.
template <bool INV, typename C>
__device__ C* smem_fft(C* a, C* b, const C* __restrict__ tw, const AxisPlan& pl, int P, int S) {
  int Ns = 1;
  const int L = pl.L;
  for (int s = 0; s < pl.nstages; ++s) {
    const int RX = pl.radix[s];
    switch (RX) {
      case 2: stage_fixed<2, INV>(a, b, tw, L, P, S, Ns); break;
      case 3: stage_fixed<3, INV>(a, b, tw, L, P, S, Ns); break;
      case 4: stage_fixed<4, INV>(a, b, tw, L, P, S, Ns); break;
      case 5: stage_fixed<5, INV>(a, b, tw, L, P, S, Ns); break;
      case 8: stage_fixed<8, INV>(a, b, tw, L, P, S, Ns); break;
      case 16: stage_fixed<16, INV>(a, b, tw, L, P, S, Ns); break;
      default: stage_generic<INV>(a, b, tw, L, P, S, Ns, RX); break;
    }
    __syncthreads();
    C* t = a; a = b; b = t;
    Ns *= RX;
  }
  return a;
}

// Shared-memory footprint of one pencil batch (two buffers + twiddles).
template <typename R> inline size_t fft_smem_bytes(int L, int P) {
  return (size_t)(2 * (size_t)L * (P + 1) + L) * sizeof(cx<R>);
}

}  // namespace em3d
