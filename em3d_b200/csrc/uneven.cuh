// Applications over problems of uneven grid sizes (em3d_*_uneven).
//
// The problems are given as segments, one per grid size.  Each of the five
// passes is ONE launch: its CTAs are numbered segment after segment, a CTA
// finds the segment its index falls in (a scan of at most eight entries of
// the kernel's parameter block) and runs the register-FFT body compiled for
// that segment's axis length on its CTA index within the segment.  All
// lengths of one pass share the CTA size (rows: 192 threads for EM, 256 for
// acoustic; y pencils: 256; x pencils: 128), which is why only the plans
// whose CTA shape divides it join (uneven_*_ok below).  The dynamic shared
// memory is the largest any present segment needs.
//
// Workspace: per segment its T1 (count, C, Nx, Ny, 2Nz) and T2
// (count, C, Nx, 2Ny, 2Nz), one after the other, then the status words.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>

#include "operator_passes.cuh"

namespace em3d {

constexpr int kMaxSegments = EM3D_MAX_SEGMENTS;

template <int C> struct UnevenNT {
  static constexpr int rows = C == 3 ? 192 : 256;
  static constexpr int strided = 256;
  static constexpr int xmul = 128;
};

template <typename R, int L, int C> constexpr bool uneven_rows_ok() {
  return RowsGeom<L, FastE<R, L>::E, C, UnevenNT<C>::rows>::NT == UnevenNT<C>::rows;
}
template <typename R, int L> constexpr bool uneven_strided_ok() {
  return StridedGeom<L, FastE<R, L>::E>::NT == UnevenNT<1>::strided;
}
// (complex128 at 160 keeps three 20-element pencils per thread and spills
// part of them to local memory; it joins all the same, so that FP64
// operators over such sizes stay one launch per pass)
template <typename R, int L, int C> constexpr bool uneven_x_ok() {
  return XmulGeom<L, FastE<R, L>::E, C, 128>::NT == UnevenNT<C>::xmul;
}

// The pipelined x pass (persistent CTAs, field slab by TMA): same CTA shape
// rule, and its slabs must fit in a CTA's shared memory.
template <typename R, int L, int C> constexpr bool uneven_xpipe_ok() {
  using G = XpipeGeom<L, FastE<R, L>::E, C, 128>;
  return G::NT == UnevenNT<C>::xmul && G::P % 2 == 0 &&
         (size_t)G::TOTAL * sizeof(cx<R>) + G::BYTES_EXTRA <= kSmemPerCta;
}

#define EM3D_UNEVEN_LENGTHS(X) X(32) X(64) X(96) X(128) X(160) X(192) X(256)

// Host-side geometry of one axis length in the three pass kinds.
struct UnevenLen {
  bool rows_ok, strided_ok, x_ok;
  int rows_rpb;        // rows per CTA
  size_t rows_smem;    // bytes
  int strided_p;       // pencils per CTA
  size_t strided_smem;
  int x_p;             // kz per CTA
  size_t x_smem;
  bool xpipe_ok;       // the pipelined x pass applies
  int xpipe_p;
  size_t xpipe_smem;
};

template <typename R, int C, int L> static UnevenLen uneven_len_of() {
  constexpr int E = FastE<R, L>::E;
  using GR = RowsGeom<L, E, C, UnevenNT<C>::rows>;
  using GS = StridedGeom<L, E>;
  using GX = XmulGeom<L, E, C, 128>;
  UnevenLen u;
  u.rows_ok = uneven_rows_ok<R, L, C>();
  u.strided_ok = uneven_strided_ok<R, L>();
  u.x_ok = uneven_x_ok<R, L, C>();
  u.rows_rpb = GR::RPB;
  u.rows_smem = (size_t)(L + C * GR::RPB * GR::PSTRIDE) * sizeof(cx<R>);
  u.strided_p = GS::P;
  u.strided_smem = (size_t)(L + L * GS::S) * sizeof(cx<R>);
  u.x_p = GX::P;
  u.x_smem = (size_t)(L + GX::REGIONS * L * GX::S) * sizeof(cx<R>);
  using GP = XpipeGeom<L, E, C, 128>;
  u.xpipe_ok = uneven_xpipe_ok<R, L, C>();
  u.xpipe_p = GP::P;
  u.xpipe_smem = (size_t)GP::TOTAL * sizeof(cx<R>) + GP::BYTES_EXTRA;
  return u;
}

// The TMA map of a segment's T2 for the pipelined x pass (tile width P of its
// x length).
template <typename R, int C>
static int uneven_field_map(int L, CUtensorMap* fmap, cx<R>* T2, const Dims& d, int count) {
  switch (L) {
#define EM3D_CASE(LL)                                                                      \
  case LL:                                                                                 \
    if constexpr (uneven_xpipe_ok<R, LL, C>())                                             \
      return encode_field_map<R, C, XpipeGeom<LL, FastE<R, LL>::E, C, 128>::P>(fmap, T2, d, count); \
    break;
    EM3D_UNEVEN_LENGTHS(EM3D_CASE)
#undef EM3D_CASE
  }
  em3d_set_last_error("no pipelined x pass for this length");
  return EM3D_ERR_UNSUPPORTED;
}

template <typename R, int C> static bool uneven_len(int L, UnevenLen* out) {
  switch (L) {
#define EM3D_CASE(LL) \
  case LL: *out = uneven_len_of<R, C, LL>(); return true;
    EM3D_UNEVEN_LENGTHS(EM3D_CASE)
#undef EM3D_CASE
  }
  return false;
}

template <typename R, int C> static bool uneven_grid_ok(const Dims& d) {
  UnevenLen lz, ly, lx;
  return uneven_len<R, C>(2 * d.nz, &lz) && lz.rows_ok && uneven_len<R, C>(2 * d.ny, &ly) && ly.strided_ok &&
         uneven_len<R, C>(2 * d.nx, &lx) && lx.x_ok;
}

// ---------------------------------------------------------------------------
// kernels: per-segment arguments in the parameter block
// ---------------------------------------------------------------------------

template <typename R> struct RowsSeg {
  const cx<R>* in;
  const cx<R>* chi;
  const cx<R>* base;
  cx<R>* out;
  const cx<R>* tw;
  int rows_pb, nrows, L, block0;
  BatchStrides bs;
};
template <typename R> struct StridedSeg {
  const cx<R>* in;
  cx<R>* out;
  const cx<R>* tw;
  int inner, ntiles, L, block0;
  BatchStrides bs;
};
template <typename R> struct XSeg {
  cx<R>* T2;
  const cx<R>* spec;
  const cx<R>* tw;
  int ny, nz, ntz, nb, L, block0;
  BatchStrides bs;
};
// The map comes first: it needs 64-byte alignment in the parameter block.
template <typename R> struct XPSeg {
  CUtensorMap fmap;
  cx<R>* T2;
  const cx<R>* spec;
  const cx<R>* tw;
  int ny, nz, ntz, nb, L, block0, nblocks;
  BatchStrides bs;
};
template <class S> struct Segs {
  S s[kMaxSegments];
  int n;
};

template <class S> __device__ __forceinline__ const S& my_segment(const Segs<S>& a, int* blk) {
  int s = 0;
  while (s + 1 < a.n && (int)blockIdx.x >= a.s[s + 1].block0) ++s;
  *blk = (int)blockIdx.x - a.s[s].block0;
  return a.s[s];
}

template <typename R, int C, int LD, int ST, bool INV>
__global__ void __launch_bounds__(UnevenNT<C>::rows) ku_rows(const __grid_constant__ Segs<RowsSeg<R>> a, const int* skip) {
  int blk;
  const RowsSeg<R>& g = my_segment(a, &blk);
  switch (g.L) {
#define EM3D_CASE(LL)                                                                                           \
  case LL:                                                                                                      \
    if constexpr (uneven_rows_ok<R, LL, C>())                                                                   \
      rows_body<R, LL, C, LD, ST, INV, UnevenNT<C>::rows>(g.in, g.chi, g.base, g.out, g.tw, g.rows_pb, g.nrows, \
                                                          g.bs, skip, blk);                                     \
    break;
    EM3D_UNEVEN_LENGTHS(EM3D_CASE)
#undef EM3D_CASE
  }
}

template <typename R, bool INV>
__global__ void __launch_bounds__(256) ku_strided(const __grid_constant__ Segs<StridedSeg<R>> a, const int* skip) {
  int blk;
  const StridedSeg<R>& g = my_segment(a, &blk);
  switch (g.L) {
#define EM3D_CASE(LL)                                                                        \
  case LL:                                                                                   \
    if constexpr (uneven_strided_ok<R, LL>())                                                \
      strided_body<R, LL, INV>(g.in, g.out, g.tw, g.inner, g.ntiles, g.bs, skip, blk);       \
    break;
    EM3D_UNEVEN_LENGTHS(EM3D_CASE)
#undef EM3D_CASE
  }
}

template <typename R, int C, bool ADJ>
__global__ void __launch_bounds__(128) ku_xmul(const __grid_constant__ Segs<XSeg<R>> a, const int* skip) {
  int blk;
  const XSeg<R>& g = my_segment(a, &blk);
  switch (g.L) {
#define EM3D_CASE(LL)                                                                                        \
  case LL:                                                                                                   \
    if constexpr (uneven_x_ok<R, LL, C>())                                                                   \
      xmul_body<R, LL, C, ADJ, FastE<R, LL>::E, 128>(g.T2, g.spec, g.tw, g.ny, g.nz, g.ntz, g.nb, g.bs, skip, \
                                                     blk);                                                   \
    break;
    EM3D_UNEVEN_LENGTHS(EM3D_CASE)
#undef EM3D_CASE
  }
}

// Pipelined x pass: each segment has its own share of persistent CTAs
// (nblocks) that loop over that segment's tiles.
template <typename R, int C, bool ADJ>
__global__ void __launch_bounds__(128) ku_xpipe(const __grid_constant__ Segs<XPSeg<R>> a, const int* skip) {
  int blk;
  const XPSeg<R>& g = my_segment(a, &blk);
  switch (g.L) {
#define EM3D_CASE(LL)                                                                                          \
  case LL:                                                                                                     \
    if constexpr (uneven_xpipe_ok<R, LL, C>())                                                                 \
      xpipe_body<R, LL, C, ADJ, FastE<R, LL>::E, 128, true>(g.T2, g.spec, g.tw, g.ny, g.nz, g.ntz, g.nb, g.bs, \
                                                            skip, &g.fmap, g.bs.status, blk, g.nblocks);       \
    break;
    EM3D_UNEVEN_LENGTHS(EM3D_CASE)
#undef EM3D_CASE
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

// Checks one segment (its arrays too when `arrays`); fills its dims and the
// element strides.
template <typename R, int C>
static int uneven_check(const em3d_segment& s, int dtype, Dims* d, BatchStrides* bs, bool arrays = true) {
  int rc = check_grid(&s.grid, d);
  if (rc) return rc;
  constexpr size_t esz = sizeof(cx<R>);
  if (s.count < 1) { em3d_set_last_error("segment count must be >= 1"); return EM3D_ERR_INVALID; }
  if (arrays && (!s.spectra || !s.chi || !s.u || !s.out)) {
    em3d_set_last_error("NULL array argument in a segment");
    return EM3D_ERR_INVALID;
  }
  if (arrays && s.u == s.out) { em3d_set_last_error("out must not alias the input field"); return EM3D_ERR_INVALID; }
  if (!uneven_grid_ok<R, C>(*d)) {
    em3d_set_last_error("grid not supported by the uneven application (see em3d_uneven_supported)");
    return EM3D_ERR_UNSUPPORTED;
  }
  const int kind = C == 3 ? EM3D_EM : EM3D_ACOUSTIC;
  const size_t cells = d->cells();
  int comps = 1;
  if (C == 3) {
    if (s.chi_layout != EM3D_CHI_FULL && s.chi_layout != EM3D_CHI_SYMMETRIC && s.chi_layout != EM3D_CHI_ISOTROPIC) {
      em3d_set_last_error("chi_layout must be EM3D_CHI_FULL (9), EM3D_CHI_SYMMETRIC (6) or EM3D_CHI_ISOTROPIC (1)");
      return EM3D_ERR_INVALID;
    }
    comps = s.chi_layout;
  }
  if (s.spectrum_stride < em3d_spectrum_bytes(&s.grid, kind, dtype) || s.spectrum_stride % esz) {
    em3d_set_last_error("spectrum_stride must be >= em3d_spectrum_bytes and a multiple of the element size");
    return EM3D_ERR_INVALID;
  }
  if (s.count > 1 && (s.chi_stride < comps * cells * esz || s.chi_stride % esz)) {
    em3d_set_last_error("chi_stride must hold one contrast and be a multiple of the element size");
    return EM3D_ERR_INVALID;
  }
  if (s.count > 1 && (s.field_stride < C * cells * esz || s.field_stride % esz)) {
    em3d_set_last_error("field_stride must hold one field and be a multiple of the element size");
    return EM3D_ERR_INVALID;
  }
  if (s.entry_done && s.entry_done_stride < sizeof(int)) {
    em3d_set_last_error("entry_done_stride must be at least sizeof(int)");
    return EM3D_ERR_INVALID;
  }
  *bs = BatchStrides{};
  bs->chi = s.count > 1 ? s.chi_stride / esz : 0;
  bs->spec = s.count > 1 ? s.spectrum_stride / esz : 0;
  bs->done = (const char*)s.entry_done;
  bs->done_stride = s.entry_done_stride;
  bs->outer = C * d->nx;
  bs->chi_layout = C == 3 ? s.chi_layout : 9;
  bs->field = s.count > 1 ? s.field_stride / esz : 0;
  return EM3D_OK;
}

template <typename R, int C>
static size_t uneven_ws_bytes(int nseg, const em3d_segment* segs, int dtype, size_t* t_off = nullptr) {
  size_t off = 0;
  for (int i = 0; i < nseg; ++i) {
    Dims d;
    BatchStrides bs;
    if (uneven_check<R, C>(segs[i], dtype, &d, &bs, t_off != nullptr)) return 0;
    const size_t t1 = (size_t)segs[i].count * C * d.nx * d.ny * 2 * d.nz;
    const size_t t2 = (size_t)segs[i].count * C * d.nx * 2 * d.ny * 2 * d.nz;
    if (t_off) { t_off[2 * i] = off; t_off[2 * i + 1] = off + align_up(t1 * sizeof(cx<R>)); }
    off += align_up(t1 * sizeof(cx<R>)) + align_up(t2 * sizeof(cx<R>));
  }
  return off + kStatusBytes;
}

template <typename K, class A>
static int uneven_launch(K kern, const A& args, int blocks, int threads, size_t smem, const int* skip,
                         cudaStream_t st) {
  EM3D_CUDA_TRY(allow_smem(kern));
  kern<<<blocks, threads, smem, st>>>(args, skip);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

template <typename R, int C, bool ADJ>
int apply_uneven(int dtype, int nseg, const em3d_segment* segs, void* ws, size_t wsb, const int* skip,
                 cudaStream_t st) {
  using T = cx<R>;
  if (nseg < 1 || nseg > kMaxSegments || !segs) {
    em3d_set_last_error("nseg must be 1..EM3D_MAX_SEGMENTS with a segment array");
    return EM3D_ERR_INVALID;
  }
  size_t toff[2 * kMaxSegments];
  const size_t need = uneven_ws_bytes<R, C>(nseg, segs, dtype, toff);
  if (need == 0) return EM3D_ERR_INVALID;  // the failing check has set the message
  if (!ws || wsb < need) { em3d_set_last_error("uneven workspace too small"); return EM3D_ERR_INVALID; }
  int* status = (int*)((char*)ws + need - kStatusBytes);

  Segs<RowsSeg<R>> p1{}, p5{};
  Segs<StridedSeg<R>> p2{}, p4{};
  Segs<XSeg<R>> p3{};
  Segs<XPSeg<R>> p3p;
  memset(&p3p, 0, sizeof p3p);
  p1.n = p2.n = p3.n = p4.n = p5.n = p3p.n = nseg;
  int b1 = 0, b2 = 0, b3 = 0;
  size_t sm1 = 0, sm2 = 0, sm3 = 0, sm3p = 0;
  int layout = 0;
  // the EM x pass runs pipelined (persistent CTAs, field slab by TMA) when
  // every segment's x length allows it, unless a non-pipelined x-pass
  // variant (0..2) is selected
  const int xv = g_tuning[EM3D_TUNE_XPASS_VARIANT];
  bool pipe = C == 3 && (xv < 0 || xv >= 3);
  double work[kMaxSegments];
  long long units[kMaxSegments];
  Dims dims[kMaxSegments];
  for (int i = 0; i < nseg; ++i) {
    const em3d_segment& s = segs[i];
    Dims d;
    BatchStrides bs;
    int rc = uneven_check<R, C>(s, dtype, &d, &bs);
    if (rc) return rc;
    if (C == 3) {
      if (i == 0) layout = s.chi_layout;
      else if (s.chi_layout != layout) {
        em3d_set_last_error("every EM segment of an uneven application needs the same chi_layout");
        return EM3D_ERR_INVALID;
      }
    }
    bs.status = status;
    UnevenLen lz, ly, lx;
    uneven_len<R, C>(2 * d.nz, &lz);
    uneven_len<R, C>(2 * d.ny, &ly);
    uneven_len<R, C>(2 * d.nx, &lx);
    SpecLayout<R> lay(d, C == 3 ? EM3D_EM : EM3D_ACOUSTIC);
    void* sp = const_cast<void*>(s.spectra);
    T* T1 = (T*)((char*)ws + toff[2 * i]);
    T* T2 = (T*)((char*)ws + toff[2 * i + 1]);
    const int rows_pb = d.nx * d.ny, nrows = s.count * rows_pb;
    const int rblocks = (nrows + lz.rows_rpb - 1) / lz.rows_rpb;
    // passes 1 and 5 (rows along z)
    p1.s[i] = RowsSeg<R>{(const T*)s.u, (const T*)s.chi, nullptr, T1, lay.twz(sp, d), rows_pb, nrows, 2 * d.nz, b1, bs};
    p5.s[i] = RowsSeg<R>{T1, (const T*)s.chi, (const T*)s.u, (T*)s.out, lay.twz(sp, d), rows_pb, nrows, 2 * d.nz, b1, bs};
    b1 += rblocks;
    sm1 = std::max(sm1, lz.rows_smem);
    // passes 2 and 4 (pencils along y)
    const int inner = 2 * d.nz, ntiles = (inner + ly.strided_p - 1) / ly.strided_p;
    p2.s[i] = StridedSeg<R>{T1, T2, lay.twy(sp, d), inner, ntiles, 2 * d.ny, b2, bs};
    p4.s[i] = StridedSeg<R>{T2, T1, lay.twy(sp, d), inner, ntiles, 2 * d.ny, b2, bs};
    b2 += s.count * C * d.nx * ntiles;
    sm2 = std::max(sm2, ly.strided_smem);
    // pass 3 (pencils along x)
    const int ntz = (2 * d.nz + lx.x_p - 1) / lx.x_p;
    p3.s[i] = XSeg<R>{T2, lay.oct(sp), lay.twx(sp, d), d.ny, d.nz, ntz, s.count, 2 * d.nx, b3, bs};
    b3 += s.count * 2 * d.ny * ntz;
    sm3 = std::max(sm3, lx.x_smem);
    pipe = pipe && lx.xpipe_ok;
    {
      XPSeg<R>& q = p3p.s[i];
      q.T2 = T2;
      q.spec = lay.oct(sp);
      q.tw = lay.twx(sp, d);
      q.ny = d.ny;
      q.nz = d.nz;
      q.ntz = (2 * d.nz + lx.xpipe_p - 1) / lx.xpipe_p;
      q.nb = s.count;
      q.L = 2 * d.nx;
      q.bs = bs;
      // work units of the persistent loop (one entry per unit: every entry
      // has its own spectrum, or the segment holds one entry)
      units[i] = (long long)s.count * (d.ny + 1) * q.ntz;
      work[i] = (double)units[i] * lx.xpipe_p * (2.0 * d.nx) * std::log2(2.0 * d.nx);
      dims[i] = d;
      sm3p = std::max(sm3p, lx.xpipe_smem);
    }
  }
  int b3p = 0;
  if (pipe) {
    // Each CTA loops over U of its segment's work units (one spectrum slab, the
    // ky / 2Ny - ky tiles); the grid is several waves of such CTAs, so the
    // hardware scheduler balances the segments, and the segments with the
    // most transform work come first (their CTAs start in the first wave).
    auto kern = ku_xpipe<R, C, ADJ>;
    EM3D_CUDA_TRY(allow_smem(kern));
    int sms = 0, per_sm = 0;
    EM3D_CUDA_TRY(sm_count(&sms));
    EM3D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, UnevenNT<C>::xmul, sm3p));
    if (per_sm < 1) per_sm = 1;
    constexpr long long kWaves = 8;
    long long all_units = 0;
    for (int i = 0; i < nseg; ++i) all_units += units[i];
    const long long U = std::max(2LL, (all_units + kWaves * sms * per_sm - 1) / (kWaves * sms * per_sm));
    int order[kMaxSegments];
    for (int i = 0; i < nseg; ++i) order[i] = i;
    std::sort(order, order + nseg, [&](int a, int b) { return work[a] > work[b]; });
    Segs<XPSeg<R>> sorted;
    memset(&sorted, 0, sizeof sorted);
    sorted.n = nseg;
    for (int k = 0; k < nseg; ++k) {
      const int i = order[k];
      XPSeg<R>& q = sorted.s[k];
      q = p3p.s[i];
      q.block0 = b3p;
      q.nblocks = (int)((units[i] + U - 1) / U);
      b3p += q.nblocks;
      const int rc = uneven_field_map<R, C>(q.L, &q.fmap, q.T2, dims[i], q.nb);
      if (rc) return rc;
    }
    p3p = sorted;
  }
  constexpr int NR = UnevenNT<C>::rows;
  int rc;
  // pass 1: chi applied on load (matvec) or plain (rmatvec)
  if constexpr (ADJ) {
    rc = uneven_launch(ku_rows<R, C, FLD_PLAIN, FST_PLAIN, false>, p1, b1, NR, sm1, skip, st);
  } else if constexpr (C == 1) {
    rc = uneven_launch(ku_rows<R, C, FLD_AC_CHI, FST_PLAIN, false>, p1, b1, NR, sm1, skip, st);
  } else {
    if (layout == 6) rc = uneven_launch(ku_rows<R, C, FLD_EM_CHI6, FST_PLAIN, false>, p1, b1, NR, sm1, skip, st);
    else if (layout == 1) rc = uneven_launch(ku_rows<R, C, FLD_EM_CHI1, FST_PLAIN, false>, p1, b1, NR, sm1, skip, st);
    else rc = uneven_launch(ku_rows<R, C, FLD_EM_CHI, FST_PLAIN, false>, p1, b1, NR, sm1, skip, st);
  }
  if (rc) return rc;
  rc = uneven_launch(ku_strided<R, false>, p2, b2, UnevenNT<C>::strided, sm2, skip, st);
  if (rc) return rc;
  if (pipe) rc = uneven_launch(ku_xpipe<R, C, ADJ>, p3p, b3p, UnevenNT<C>::xmul, sm3p, skip, st);
  else rc = uneven_launch(ku_xmul<R, C, ADJ>, p3, b3, UnevenNT<C>::xmul, sm3, skip, st);
  if (rc) return rc;
  rc = uneven_launch(ku_strided<R, true>, p4, b2, UnevenNT<C>::strided, sm2, skip, st);
  if (rc) return rc;
  // pass 5: u - y (matvec) or v - chi^H y (rmatvec)
  if constexpr (!ADJ) {
    rc = uneven_launch(ku_rows<R, C, FLD_PLAIN, FST_SUB, true>, p5, b1, NR, sm1, skip, st);
  } else if constexpr (C == 1) {
    rc = uneven_launch(ku_rows<R, C, FLD_PLAIN, FST_AC_ADJ, true>, p5, b1, NR, sm1, skip, st);
  } else {
    if (layout == 6) rc = uneven_launch(ku_rows<R, C, FLD_PLAIN, FST_EM_ADJ6, true>, p5, b1, NR, sm1, skip, st);
    else if (layout == 1) rc = uneven_launch(ku_rows<R, C, FLD_PLAIN, FST_EM_ADJ1, true>, p5, b1, NR, sm1, skip, st);
    else rc = uneven_launch(ku_rows<R, C, FLD_PLAIN, FST_EM_ADJ, true>, p5, b1, NR, sm1, skip, st);
  }
  return rc;
}

}  // namespace em3d
