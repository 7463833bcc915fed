// x pass (pass 3) with fewer instructions per pencil, for register plans whose
// reversed order is the same plan (256 points: radix 16 x 16; 512: 8 x 8 x 8;
// 64: 8 x 8).
//
// Same work, data layout and pipeline as kf_xmul_pipe (persistent CTAs; field
// slab by TMA on an mbarrier with bounded waits; spectrum slab by cp.async one
// work unit ahead; the tiles ky and 2Ny - ky sharing one spectrum slab).  It
// differs in how the transforms are issued:
//   * the stage twiddles of every thread are loaded once into registers (the
//     forward transform and the reversed inverse transform visit the same
//     positions, so one set serves both: conjugated for the inverse);
//   * the exchange between two stages synchronises once: consecutive
//     exchanges alternate between two shared-memory buffers, so a buffer is
//     only rewritten after the next exchange's barrier, by which point every
//     thread has read it;
//   * ROT: the three field components are transformed by one copy of the
//     transform code in a loop that rotates the components through the
//     registers (a third of the instruction footprint of three inlined
//     copies, at the cost of the register moves).
#pragma once

#include "passes_fast.cuh"

namespace em3d {

template <int L, int E> struct SymPlan {
  using P = RegPlan<L, E>;
  __host__ __device__ static constexpr bool symmetric() {
    if (!P::POW2) return false;
    for (int s = 0; s < P::NS; ++s)
      if (P::rad(false, s) != P::rad(true, s)) return false;
    return true;
  }
  // index of the first register twiddle of stage s >= 1
  __host__ __device__ static constexpr int tw_offset(int s) {
    int n = 0;
    for (int i = 1; i < s; ++i) n += (E / P::rad(false, i)) * (P::rad(false, i) - 1);
    return n;
  }
  static constexpr int NW = tw_offset(P::NS) > 0 ? tw_offset(P::NS) : 1;
};

// Register twiddles of stages S..NS-1 for thread t: stage S (radix R, NSV
// earlier points per group) multiplies element r of butterfly q by
// w^{r k L/(NSV R)}, k = (t + q T) mod NSV.
template <int L, int E, int S, typename T, int NW>
__device__ __forceinline__ void load_stage_twiddles(T (&w)[NW], int t, const T* __restrict__ tw) {
  using P = RegPlan<L, E>;
  if constexpr (S < P::NS) {
    constexpr int R = P::rad(false, S), NSV = P::nsb(false, S), TT = L / E, TS = L / (NSV * R);
    constexpr int OFF = SymPlan<L, E>::tw_offset(S);
#pragma unroll
    for (int q = 0; q < E / R; ++q) {
      const int k = (t + q * TT) % NSV;
#pragma unroll
      for (int r = 1; r < R; ++r) w[OFF + q * (R - 1) + r - 1] = tw[r * k * TS];
    }
    load_stage_twiddles<L, E, S + 1>(w, t, tw);
  }
}

template <int L, int E, int S, bool INV, bool HALF_IN, typename T, int NW>
__device__ __forceinline__ void wstage(T (&a)[E], const T (&w)[NW]) {
  using P = RegPlan<L, E>;
  constexpr int R = P::rad(false, S), Q = E / R;
  constexpr int OFF = SymPlan<L, E>::tw_offset(S);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    T* b = &a[q * R];
    if constexpr (S > 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const T ww = w[OFF + q * (R - 1) + r - 1];
        b[r] = INV ? cmulcj(ww, b[r]) : cmul(ww, b[r]);
      }
    }
    if constexpr (HALF_IN) dft_fixed_half_in<R, INV>(b);
    else dft_fixed<R, INV>(b);
  }
}

// Stage S's outputs to shared memory, one barrier, stage S+1's inputs back.
template <int L, int E, int S, typename T, class Lay>
__device__ __forceinline__ void xchg_once(T (&a)[E], int t, T* sm, const Lay& lay) {
  using P = RegPlan<L, E>;
  constexpr int R = P::rad(false, S), NSV = P::nsb(false, S), RN = P::rad(false, S + 1), TT = L / E;
#pragma unroll
  for (int q = 0; q < E / R; ++q) {
    const int j = t + q * TT;
    const int base = (j / NSV) * NSV * R + (j % NSV);
#pragma unroll
    for (int r = 0; r < R; ++r) sm[lay(0, base + r * NSV)] = a[q * R + r];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < E / RN; ++q) {
    const int j = t + q * TT;
#pragma unroll
    for (int r = 0; r < RN; ++r) a[q * RN + r] = sm[lay(0, j + r * (L / RN))];
  }
}

// One pencil slice through all stages; exchange number xi uses buffer xi & 1.
template <int L, int E, bool INV, bool HALF_IN, int S = 0, typename T, int NW, class Lay>
__device__ __forceinline__ void fft_one(T (&a)[E], int t, T* xbuf, int xsize, int& xi, const T (&w)[NW],
                                        const Lay& lay) {
  wstage<L, E, S, INV, HALF_IN && S == 0>(a, w);
  if constexpr (S + 1 < RegPlan<L, E>::NS) {
    xchg_once<L, E, S>(a, t, xbuf + (xi & 1) * xsize, lay);
    ++xi;
    fft_one<L, E, INV, HALF_IN, S + 1>(a, t, xbuf, xsize, xi, w, lay);
  }
}

template <int L, int E, int C, int NTT> struct XrotGeom {
  using B = XpipeGeom<L, E, C, NTT>;
  static constexpr int TT = B::TT, P = B::P, NT = B::NT, NX = B::NX, NSPEC = B::NSPEC;
  static constexpr int TW = L, EXCH = B::EXCH, FIELD = B::FIELD, SPEC = B::SPEC;
  static constexpr int TOTAL = FIELD + TW + 2 * EXCH + SPEC;  // complex elements
  static constexpr size_t BYTES_EXTRA = 16;                     // the TMA mbarrier
};

template <typename R, int L, int C, bool ADJ, int E, int NTT, bool ROT>
__global__ void __launch_bounds__(XrotGeom<L, E, C, NTT>::NT)
kf_xmul_rot(cx<R>* T2, const cx<R>* __restrict__ spec, const cx<R>* __restrict__ twg, int Ny, int Nz, int ntz,
            int nb, BatchStrides bs, const int* skip, const __grid_constant__ CUtensorMap fmap, int* status) {
  using T = cx<R>;
  using G = XrotGeom<L, E, C, NTT>;
  using PL = RegPlan<L, E>;
  static_assert(SymPlan<L, E>::symmetric(), "kf_xmul_rot needs a plan equal to its reverse");
  constexpr int TT = G::TT, PP = G::P, NX = G::NX;
  constexpr int R1 = PL::first(false), RL = PL::last(false);
  constexpr int M1 = L / R1, ML = L / RL;
  constexpr int EB = (int)sizeof(T);
  constexpr int NW = SymPlan<L, E>::NW;
  if (skip_launch(skip)) return;
  extern __shared__ __align__(128) unsigned char smem_rot[];
  T* sfield = reinterpret_cast<T*>(smem_rot);  // TMA destination first (128-byte aligned)
  T* tw = sfield + G::FIELD;
  T* xbuf = tw + G::TW;                          // two exchange buffers of G::EXCH
  T* sspec = xbuf + 2 * G::EXCH;
  uint64_t* fbar = reinterpret_cast<uint64_t*>(sspec + G::SPEC);
  for (int i = threadIdx.x; i < L; i += blockDim.x) tw[i] = twg[i];
  if (threadIdx.x == 0) {
    mbar_init(fbar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  const int p = threadIdx.x % PP, t = threadIdx.x / PP;
  T w[NW];
  load_stage_twiddles<L, E, 1>(w, t, tw);
  uint32_t fphase = 0;
  int xi = 0;
  const int Ny2 = 2 * Ny, Nz2 = 2 * Nz;
  const size_t xstride = (size_t)Ny2 * Nz2;
  const size_t ostride = (size_t)(NX + 1) * (Ny + 1) * (Nz + 1);
  const int nbu = xpipe_entries_per_unit(nb, bs.spec == 0);
  const int ngroups = nb / nbu;
  const int nunits = ngroups * (Ny + 1) * ntz;
  auto decode = [&](int u, int& bg, int& jy, int& kz0) {
    bg = u % ngroups;
    const int idx = u / ngroups;
    kz0 = (idx % ntz) * PP;
    jy = idx / ntz;
  };
  auto nmirror = [&](int jy) { return (jy == 0 || jy == Ny) ? 1 : 2; };
  constexpr int RSTEP = G::NT / PP;
  auto issue_field = [&](int u, int sub) {
    int bg, jy, kz0;
    decode(u, bg, jy, kz0);
    const int b = bg * nbu + sub / nmirror(jy);
    const int ky = (sub % nmirror(jy)) ? Ny2 - jy : jy;
    if (entry_done(bs, b)) return;
    constexpr int W = EB / 8;
    if (threadIdx.x == 0) {
      mbar_arrive_expect_tx(fbar, (uint32_t)(C * NX * PP * EB));
#pragma unroll
      for (int c = 0; c < C; ++c) tma_load_3d(sfield + c * NX * PP, &fmap, fbar, kz0 * W, ky, (b * C + c) * NX);
    }
  };
  auto issue_spec = [&](int u) {
    int b, jy, kz0;
    decode(u, b, jy, kz0);
    if (nbu == 1 && entry_done(bs, b)) return;
    const int kz = kz0 + p;
    const bool ok = kz < Nz2;
    const T* base = spec + (size_t)b * bs.spec + (size_t)jy * (Nz + 1) + (ok ? kfold(kz, Nz) : 0);
    const size_t xs = (size_t)(Ny + 1) * (Nz + 1);
    int row = threadIdx.x / PP;
    int sc = row / (NX + 1), ix = row - sc * (NX + 1);
    T* dst = sspec + row * PP + p;
    for (; row < G::SPEC / PP; row += RSTEP, dst += RSTEP * PP) {
      if (ok) cp_async_el(dst, base + sc * ostride + ix * xs, EB);
      else *dst = mk<R>(0, 0);
      ix += RSTEP;
      while (ix > NX) { ix -= NX + 1; ++sc; }
    }
  };

  int u = blockIdx.x, sub = 0;
  if (u < nunits) issue_field(u, 0);
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
    int nu = u, ns = sub + 1;
    if (ns >= nbu * nmirror(jy)) {
      nu = u + gridDim.x;
      ns = 0;
    }
    const bool live = !entry_done(bs, b);  // uniform over the CTA

    if (live) {
      const bool arrived = mbar_wait_bounded(fbar, fphase);
      if (!__syncthreads_and(arrived)) {
        // the field slab never arrived: count it once, give the copy still in
        // flight one more bounded wait, issue nothing further and leave
        if (threadIdx.x == 0 && status != nullptr) atomicAdd(status, 1);
        mbar_wait_bounded(fbar, fphase);
        cp_async_wait_all();
        return;
      }
      fphase ^= 1u;
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
    fence_proxy_async_smem();  // these reads before the next tile's TMA overwrite
    __syncthreads();
    if (nu < nunits) issue_field(nu, ns);

    if (live) {
      if constexpr (ROT && C == 3) {
#pragma unroll 1
        for (int c = 0; c < 3; ++c) {
          fft_one<L, E, false, true>(a[0], t, xbuf, G::EXCH, xi, w, lay);
#pragma unroll
          for (int e = 0; e < E; ++e) {
            const T tmp = a[0][e];
            a[0][e] = a[1][e];
            a[1][e] = a[2][e];
            a[2][e] = tmp;
          }
        }
      } else {
#pragma unroll
        for (int c = 0; c < C; ++c) fft_one<L, E, false, true>(a[c], t, xbuf, G::EXCH, xi, w, lay);
      }
    }

    cp_async_wait_all();  // this unit's spectrum slab
    __syncthreads();
    const R sy = ky <= Ny ? (R)1 : (R)-1;
    const R sz = kz <= Nz ? (R)1 : (R)-1;
#pragma unroll
    for (int q = 0; q < E / RL; ++q) {
      const int j = t + q * TT;
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int kx = j + r * ML;
        // kx <= NX is known at compile time except where this (q, r) slot
        // straddles NX (then it depends on t < TT)
        const int lo = q * TT + r * ML, hi = lo + TT - 1;
        const bool up = hi <= NX ? true : (lo > NX ? false : kx <= NX);
        const T* s0 = sspec + (up ? kx : L - kx) * PP + p;
        const int e = q * RL + r;
        if constexpr (C == 1) {
          const T k0 = s0[0];
          a[0][e] = ADJ ? cmulcj(k0, a[0][e]) : cmul(k0, a[0][e]);
        } else {
          constexpr int OS = (NX + 1) * PP;
          const R sx = up ? (R)1 : (R)-1;
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

    if (live) {
      if constexpr (ROT && C == 3) {
#pragma unroll 1
        for (int c = 0; c < 3; ++c) {
          fft_one<L, E, true, false>(a[0], t, xbuf, G::EXCH, xi, w, lay);
#pragma unroll
          for (int e = 0; e < E; ++e) {
            const T tmp = a[0][e];
            a[0][e] = a[1][e];
            a[1][e] = a[2][e];
            a[2][e] = tmp;
          }
        }
      } else {
#pragma unroll
        for (int c = 0; c < C; ++c) fft_one<L, E, true, false>(a[c], t, xbuf, G::EXCH, xi, w, lay);
      }
    }
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

}  // namespace em3d
