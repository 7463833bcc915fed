// Device-resident Krylov solvers: fused vector updates with FP64 inner
// products, and the scalar recurrences / stopping rules of the reference
// solvers evaluated on the device by the last block of each reduction.
//
// Reduction scheme: each block reduces its grid-stride share with warp
// shuffles, writes one partial per value, and takes a ticket; the block that
// draws the last ticket sums the partials in a fixed order (deterministic for
// a given grid) and runs the scalar logic.  No block ever waits for another.
#include <math.h>

#include "common.cuh"

namespace em3d {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 148 * 8;
constexpr int kPartials = 8;  // values per block
// threads of the one CTA that adds an operator pass's per-CTA partial sums
// (a few thousand values: many loads in flight, one block_sum)
constexpr int kPartsThreads = 1024;
constexpr size_t kStateHeader = 256;

static_assert(sizeof(em3d_krylov_state) <= kStateHeader, "state header too small");

inline size_t al256(size_t v) { return (v + 255) / 256 * 256; }

struct StateView {
  em3d_krylov_state* st;
  double* hist;
  int* counts;
  double* partials;
};

__host__ __device__ inline size_t hist_off(int cap) { return kStateHeader; }
__host__ __device__ inline size_t counts_off(int cap) { return kStateHeader + ((size_t)8 * cap + 255) / 256 * 256; }
__host__ __device__ inline size_t partials_off(int cap) { return counts_off(cap) + ((size_t)4 * cap + 255) / 256 * 256; }

// State of right-hand side blockIdx.y; states are `stride` bytes apart and
// state 0 also carries the batch-wide running count and done flag.
__device__ inline StateView view(void* base, size_t stride) {
  StateView v;
  v.st = (em3d_krylov_state*)((char*)base + blockIdx.y * stride);
  const int cap = v.st->hist_cap;
  char* mine = (char*)v.st;
  v.hist = (double*)(mine + hist_off(cap));
  v.counts = (int*)(mine + counts_off(cap));
  v.partials = (double*)(mine + partials_off(cap));
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum K values over the block; the result is valid in thread 0.
template <int K> __device__ void block_sum(double (&v)[K]) {
  __shared__ double sh[K][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int q = 0; q < K; ++q) v[q] = warp_sum(v[q]);
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < K; ++q) sh[q][warp] = v[q];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < K; ++q) {
      double x = lane < nw ? sh[q][lane] : 0.0;
      v[q] = warp_sum(x);
    }
  }
  __syncthreads();
}

// Publish this block's partials and report whether it is the last block.
// The last block returns with the totals in tot[] (valid in all threads).
template <int K> __device__ bool reduce_last(StateView& sv, double (&v)[K], double (&tot)[K]) {
  __shared__ bool am_last;
  __shared__ double shtot[K];
  block_sum<K>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < K; ++q) sv.partials[(size_t)blockIdx.x * kPartials + q] = v[q];
    __threadfence();
    unsigned t = atomicAdd(&sv.st->ticket, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  double acc[K];
#pragma unroll
  for (int q = 0; q < K; ++q) acc[q] = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int q = 0; q < K; ++q) acc[q] += ((volatile double*)sv.partials)[(size_t)b * kPartials + q];
  }
  block_sum<K>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < K; ++q) shtot[q] = acc[q];
    sv.st->ticket = 0u;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < K; ++q) tot[q] = shtot[q];
  return true;
}

// Elements of this right-hand side's vectors in use (n_used; the rest of its
// n is padding that the step kernels leave alone), all n when n_used is 0.
__device__ __forceinline__ size_t used_len(const em3d_krylov_state* st, size_t n) {
  return st->n_used > 0 && (size_t)st->n_used < n ? (size_t)st->n_used : n;
}

__device__ __forceinline__ bool running(const em3d_krylov_state* st) {
  return *(volatile const int*)&st->status == EM3D_RUNNING;
}

__device__ inline void record(StateView& sv, double rel, int actions) {
  em3d_krylov_state* st = sv.st;
  if (st->hist_len < st->hist_cap) {
    sv.hist[st->hist_len] = rel;
    sv.counts[st->hist_len] = actions;
    st->hist_len += 1;
  }
  st->last_rel = rel;
}

// Set a stop status for this right-hand side (once) and maintain the batch
// count; the last one to stop raises batch_done, the operator's skip flag.
__device__ inline void stop_rhs(em3d_krylov_state* st, void* base, int code) {
  if (st->status != EM3D_RUNNING || code == EM3D_RUNNING) return;
  st->status = code;
  em3d_krylov_state* b0 = (em3d_krylov_state*)base;
  __threadfence();
  if (atomicSub(&b0->batch_running, 1) == 1) b0->batch_done = 1;
}

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  // plain complex division (the magnitudes here are far from over/underflow)
  const double den = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / den, (a.y * b.x - a.x * b.y) / den);
}
__device__ __forceinline__ double cabs2(double2 a) { return hypot(a.x, a.y); }

template <typename R> __device__ __forceinline__ cx<R> cast_s(double re, double im) { return mk<R>((R)re, (R)im); }

// accumulate conj(a) * b into (re, im)
template <typename C> __device__ __forceinline__ void acc_dot(double& re, double& im, C a, C b) {
  re += (double)a.x * (double)b.x + (double)a.y * (double)b.y;
  im += (double)a.x * (double)b.y - (double)a.y * (double)b.x;
}

// ---------------------------------------------------------------------------
// generic vector kernels
// ---------------------------------------------------------------------------

template <typename R>
__global__ void __launch_bounds__(kThreads) k_dots(size_t n, const cx<R>* x0, const cx<R>* y0, const cx<R>* x1,
                                                   const cx<R>* y1, void* state, size_t sstride) {
  StateView sv = view(state, sstride);
  const size_t vo = blockIdx.y * n;
  n = used_len(sv.st, n);
  x0 += vo; y0 += vo;
  if (x1) { x1 += vo; y1 += vo; }
  double v[4] = {0, 0, 0, 0};
  const size_t gs = (size_t)gridDim.x * blockDim.x;
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (!x1) {
    for (; i + 3 * gs < n; i += 4 * gs) {
      cx<R> x[4], y[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) { x[k] = x0[i + k * gs]; y[k] = y0[i + k * gs]; }
#pragma unroll
      for (int k = 0; k < 4; ++k) acc_dot(v[0], v[1], x[k], y[k]);
    }
  }
  for (; i < n; i += gs) {
    acc_dot(v[0], v[1], x0[i], y0[i]);
    if (x1) acc_dot(v[2], v[3], x1[i], y1[i]);
  }
  double tot[4];
  if (reduce_last<4>(sv, v, tot) && threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) sv.st->dots[q] = tot[q];
  }
}

template <typename R>
__global__ void k_axpby(size_t n, cx<R>* out, cx<R> a, const cx<R>* x, cx<R> b, const cx<R>* y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    cx<R> r = cmul(a, x[i]);
    if (y) r = cadd(r, cmul(b, y[i]));
    out[i] = r;
  }
}

template <typename S, typename D>
__global__ void k_convert(size_t n, const S* src, D* dst, int accumulate) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const S s = src[i];
    D d;
    d.x = (decltype(d.x))s.x;
    d.y = (decltype(d.y))s.y;
    if (accumulate) d = cadd(dst[i], d);
    dst[i] = d;
  }
}

// ---------------------------------------------------------------------------
// BiCGStab (src/em3d/solvers/bicgstab.py:84-197)
// ---------------------------------------------------------------------------

// rho / omega checks, beta, p = r + beta (p - omega v) (p = r on the first
// iteration), then the action-budget check before the matvec v = A p.
template <typename R>
__global__ void __launch_bounds__(kThreads) k_bicg_p(size_t n, void* state, size_t sstride, const cx<R>* r, cx<R>* p, const cx<R>* v) {
  em3d_krylov_state* st = (em3d_krylov_state*)((char*)state + blockIdx.y * sstride);
  if (!running(st)) return;
  { const size_t vo = blockIdx.y * n; r += vo; p += vo; v += vo; }
  n = used_len(st, n);
  const double2 rho = make_double2(st->rho_re, st->rho_im);
  const double2 omega = make_double2(st->omega_re, st->omega_im);
  int stop = EM3D_RUNNING;
  if (cabs2(rho) == 0.0) stop = EM3D_BREAKDOWN_RHO;
  else if (st->iter > 0 && cabs2(omega) == 0.0) stop = EM3D_BREAKDOWN_OMEGA;
  if (stop != EM3D_RUNNING) {
    if (blockIdx.x == 0 && threadIdx.x == 0) stop_rhs(st, state, stop);
    return;
  }
  if (st->iter == 0) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = r[i];
  } else {
    const double2 rp = make_double2(st->rho_prev_re, st->rho_prev_im);
    const double2 al = make_double2(st->alpha_re, st->alpha_im);
    const double2 beta = cmul(cdiv(rho, rp), cdiv(al, omega));
    const cx<R> b = cast_s<R>(beta.x, beta.y), w = cast_s<R>(omega.x, omega.y);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
      p[i] = cadd(r[i], cmul(b, csub(p[i], cmul(w, v[i]))));
  }
  if (st->max_actions >= 0 && st->matvecs + 1 > st->max_actions) {
    if (blockIdx.x == 0 && threadIdx.x == 0) stop_rhs(st, state, EM3D_MAX_OPERATOR_ACTIONS);
  }
}

// alpha = rho / den with den = vdot(r_hat, v), and the breakdown check
// (src/em3d/solvers/bicgstab.py:106-112); one thread.
__device__ inline void alpha_from_dot(StateView& sv, void* state, double2 den) {
  em3d_krylov_state* st = sv.st;
  st->matvecs += 1;
  if (cabs2(den) == 0.0) { stop_rhs(st, state, EM3D_BREAKDOWN_ALPHA); return; }
  const double2 al = cdiv(make_double2(st->rho_re, st->rho_im), den);
  st->alpha_re = al.x;
  st->alpha_im = al.y;
}

// den = vdot(r_hat, v); alpha = rho / den.
template <typename R>
__global__ void __launch_bounds__(kThreads) k_bicg_alpha(size_t n, void* state, size_t sstride, const cx<R>* rh, const cx<R>* v) {
  StateView sv = view(state, sstride);
  if (!running(sv.st)) return;
  { const size_t vo = blockIdx.y * n; rh += vo; v += vo; }
  n = used_len(sv.st, n);
  double a[2] = {0, 0};
  // four strides of loads in flight per thread (this kernel only reads)
  const size_t gs = (size_t)gridDim.x * blockDim.x;
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  for (; i + 3 * gs < n; i += 4 * gs) {
    cx<R> x[4], y[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) { x[k] = rh[i + k * gs]; y[k] = v[i + k * gs]; }
#pragma unroll
    for (int k = 0; k < 4; ++k) acc_dot(a[0], a[1], x[k], y[k]);
  }
  for (; i < n; i += gs) acc_dot(a[0], a[1], rh[i], v[i]);
  double tot[2];
  if (reduce_last<2>(sv, a, tot) && threadIdx.x == 0) alpha_from_dot(sv, state, make_double2(tot[0], tot[1]));
}

// The same alpha from per-CTA partial sums (|v|^2, Re / Im of vdot(v, r_hat))
// that the operator's last pass wrote while it produced v = A p
// (em3d_matvec_dots with r_hat as the second vector): den = conj of their sum.
__global__ void __launch_bounds__(kPartsThreads) k_bicg_alpha_parts(int nparts, void* state, const double* parts) {
  StateView sv = view(state, 0);
  if (!running(sv.st)) return;
  double a[2] = {0, 0};
#pragma unroll 4
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    a[0] += parts[(size_t)3 * i + 1];
    a[1] += parts[(size_t)3 * i + 2];
  }
  block_sum<2>(a);
  if (threadIdx.x == 0) alpha_from_dot(sv, state, make_double2(a[0], -a[1]));
}

// s = r - alpha v, ||s||; stopping checks on ||s|| (the update u += alpha p
// of an early exit is applied by the finalize kernel).  state.first != 0
// turns the convergence exit here off, so a run stops on full iterations
// only (the reliable-update cycles continue the recurrence from there).
template <typename R>
__global__ void __launch_bounds__(kThreads) k_bicg_s(size_t n, void* state, size_t sstride, const cx<R>* r, const cx<R>* v, cx<R>* s) {
  StateView sv = view(state, sstride);
  if (!running(sv.st)) return;
  { const size_t vo = blockIdx.y * n; r += vo; v += vo; s += vo; }
  n = used_len(sv.st, n);
  const cx<R> al = cast_s<R>(sv.st->alpha_re, sv.st->alpha_im);
  double a[1] = {0};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const cx<R> si = csub(r[i], cmul(al, v[i]));
    s[i] = si;
    a[0] += (double)si.x * si.x + (double)si.y * si.y;
  }
  double tot[1];
  if (reduce_last<1>(sv, a, tot) && threadIdx.x == 0) {
    em3d_krylov_state* st = sv.st;
    const double srel = sqrt(tot[0]) / st->rhs_norm;
    int stop = EM3D_RUNNING;
    if (!isfinite(srel)) stop = EM3D_NONFINITE;
    else if (st->guard >= 0.0 && srel > st->guard) stop = EM3D_DIVERGENCE_GUARD;
    else if (srel < st->tol && st->first == 0) stop = EM3D_CONVERGED;
    else if (st->max_actions >= 0 && st->matvecs + 1 > st->max_actions) stop = EM3D_MAX_OPERATOR_ACTIONS;
    st->last_rel = srel;
    if (stop != EM3D_RUNNING) {
      record(sv, srel, st->matvecs);
      st->iter += 1;
      st->pending = 1;
      stop_rhs(st, state, stop);
    }
  }
}

// omega = ts / tt from tot = (tt, Re ts, Im ts), with the breakdown checks
// (src/em3d/solvers/bicgstab.py:151-168); one thread.
__device__ inline void omega_from_dots(StateView& sv, void* state, const double (&tot)[3]) {
  em3d_krylov_state* st = sv.st;
  st->matvecs += 1;
  const double tt = tot[0];
  int stop = EM3D_RUNNING;
  if (fabs(tt) < 1e-30 * st->rhs_norm * st->rhs_norm) {
    stop = EM3D_BREAKDOWN_T;
  } else {
    const double2 om = make_double2(tot[1] / tt, tot[2] / tt);
    st->omega_re = om.x;
    st->omega_im = om.y;
    if (cabs2(om) == 0.0) stop = EM3D_BREAKDOWN_OMEGA;
  }
  if (stop != EM3D_RUNNING) {
    record(sv, st->last_rel, st->matvecs);
    st->iter += 1;
    st->pending = 1;
    stop_rhs(st, state, stop);
  }
}

// tt = vdot(t, t), ts = vdot(t, s); omega = ts / tt with the breakdown checks.
template <typename R>
__global__ void __launch_bounds__(kThreads) k_bicg_omega(size_t n, void* state, size_t sstride, const cx<R>* t, const cx<R>* s) {
  StateView sv = view(state, sstride);
  if (!running(sv.st)) return;
  { const size_t vo = blockIdx.y * n; t += vo; s += vo; }
  n = used_len(sv.st, n);
  double a[3] = {0, 0, 0};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const cx<R> ti = t[i];
    a[0] += (double)ti.x * ti.x + (double)ti.y * ti.y;
    acc_dot(a[1], a[2], ti, s[i]);
  }
  double tot[3];
  if (reduce_last<3>(sv, a, tot) && threadIdx.x == 0) omega_from_dots(sv, state, tot);
}

// The same omega from per-CTA partial sums (|t|^2, Re / Im of vdot(t, s))
// that the operator's last pass wrote while it produced t = A s
// (em3d_matvec_dots): one CTA adds them in a fixed order.
__global__ void __launch_bounds__(kPartsThreads) k_bicg_omega_parts(int nparts, void* state, const double* parts) {
  StateView sv = view(state, 0);
  if (!running(sv.st)) return;
  double a[3] = {0, 0, 0};
#pragma unroll 4
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
#pragma unroll
    for (int q = 0; q < 3; ++q) a[q] += parts[(size_t)3 * i + q];
  }
  block_sum<3>(a);
  if (threadIdx.x == 0) omega_from_dots(sv, state, a);
}

// Early exits at s (converged / guard / budget / breakdown_t / breakdown_omega)
// return u + alpha p: applied once (pending 1 -> 2) by the update kernel of
// the iteration that stopped, or by k_bicg_finalize.  u, p: this right-hand
// side's vectors.
template <typename R>
__device__ __forceinline__ void bicg_finish_early(StateView& sv, size_t n, cx<R>* u, const cx<R>* p) {
  n = used_len(sv.st, n);
  const cx<R> al = cast_s<R>(sv.st->alpha_re, sv.st->alpha_im);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    u[i] = cadd(u[i], cmul(al, p[i]));
  double a[1] = {0};
  double tot[1];
  if (reduce_last<1>(sv, a, tot) && threadIdx.x == 0) sv.st->pending = 2;
}

// u = (u + alpha p) + omega s;  r = s - omega t;  ||r||, vdot(r_hat, r) for the
// next rho; stopping checks on ||r||.  A right-hand side that stopped earlier
// in this iteration with an early exit pending gets u + alpha p instead.
template <typename R>
__global__ void __launch_bounds__(kThreads) k_bicg_update(size_t n, void* state, size_t sstride, cx<R>* u, const cx<R>* p,
                                                          const cx<R>* s, const cx<R>* t, cx<R>* r,
                                                          const cx<R>* rh) {
  StateView sv = view(state, sstride);
  if (!running(sv.st)) {
    if (*(volatile int*)&sv.st->pending == 1) bicg_finish_early<R>(sv, n, u + blockIdx.y * n, p + blockIdx.y * n);
    return;
  }
  { const size_t vo = blockIdx.y * n; u += vo; p += vo; s += vo; t += vo; r += vo; rh += vo; }
  n = used_len(sv.st, n);
  const cx<R> al = cast_s<R>(sv.st->alpha_re, sv.st->alpha_im);
  const cx<R> om = cast_s<R>(sv.st->omega_re, sv.st->omega_im);
  double a[3] = {0, 0, 0};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const cx<R> si = s[i];
    const cx<R> ua = cadd(u[i], cmul(al, p[i]));
    u[i] = cadd(ua, cmul(om, si));
    const cx<R> ri = csub(si, cmul(om, t[i]));
    r[i] = ri;
    a[0] += (double)ri.x * ri.x + (double)ri.y * ri.y;
    acc_dot(a[1], a[2], rh[i], ri);
  }
  double tot[3];
  if (reduce_last<3>(sv, a, tot) && threadIdx.x == 0) {
    em3d_krylov_state* st = sv.st;
    const double rel = sqrt(tot[0]) / st->rhs_norm;
    st->iter += 1;
    record(sv, rel, st->matvecs);
    int stop = EM3D_RUNNING;
    if (!isfinite(rel)) stop = EM3D_NONFINITE;
    else if (rel < st->tol) stop = EM3D_CONVERGED;
    else if (st->guard >= 0.0 && rel > st->guard) stop = EM3D_DIVERGENCE_GUARD;
    if (stop == EM3D_RUNNING) {
      st->rho_prev_re = st->rho_re;
      st->rho_prev_im = st->rho_im;
      st->rho_re = tot[1];
      st->rho_im = tot[2];
      if (st->iter >= st->max_iter) stop = EM3D_MAX_ITER;
    }
    stop_rhs(st, state, stop);
  }
}

// The same completion of an early exit as a kernel of its own (for drivers
// that stop between the s and update steps); a no-op once it has been applied.
template <typename R>
__global__ void __launch_bounds__(kThreads) k_bicg_finalize(size_t n, void* state, size_t sstride, cx<R>* u, const cx<R>* p) {
  StateView sv = view(state, sstride);
  if (*(volatile int*)&sv.st->pending != 1) return;
  bicg_finish_early<R>(sv, n, u + blockIdx.y * n, p + blockIdx.y * n);
}

// ---------------------------------------------------------------------------
// SIM (src/em3d/solvers/sim.py:45-79)
// ---------------------------------------------------------------------------

template <typename R>
__global__ void __launch_bounds__(kThreads) k_sim_residual(size_t n, void* state, size_t sstride, cx<R>* res, const cx<R>* f) {
  StateView sv = view(state, sstride);
  if (!running(sv.st)) return;
  { const size_t vo = blockIdx.y * n; res += vo; f += vo; }
  n = used_len(sv.st, n);
  double a[1] = {0};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const cx<R> ri = csub(res[i], f[i]);
    res[i] = ri;
    a[0] += (double)ri.x * ri.x + (double)ri.y * ri.y;
  }
  double tot[1];
  if (reduce_last<1>(sv, a, tot) && threadIdx.x == 0) {
    em3d_krylov_state* st = sv.st;
    st->matvecs += 1;
    const double rel = sqrt(tot[0]) / st->rhs_norm;
    record(sv, rel, st->matvecs);
    int stop = EM3D_RUNNING;
    if (!isfinite(rel)) stop = EM3D_NONFINITE;
    else if (rel < st->tol) stop = EM3D_CONVERGED;
    else if (st->guard >= 0.0 && rel > st->guard) stop = EM3D_DIVERGENCE_GUARD;
    else if (st->max_actions >= 0 && st->matvecs >= st->max_actions) stop = EM3D_MAX_OPERATOR_ACTIONS;
    else if (st->iter >= st->max_iter) stop = EM3D_MAX_ITER;
    stop_rhs(st, state, stop);
  }
}

template <typename R>
__global__ void __launch_bounds__(kThreads) k_sim_update(size_t n, void* state, size_t sstride, cx<R>* u, const cx<R>* res) {
  StateView sv = view(state, sstride);
  if (!running(sv.st)) return;
  { const size_t vo = blockIdx.y * n; u += vo; res += vo; }
  n = used_len(sv.st, n);
  const cx<R> g = cast_s<R>(sv.st->gamma_re, sv.st->gamma_im);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    u[i] = csub(u[i], cmul(g, res[i]));
  double a[1] = {0};
  double tot[1];
  if (reduce_last<1>(sv, a, tot) && threadIdx.x == 0) sv.st->iter += 1;
}

// ---------------------------------------------------------------------------
// TwoStep (src/em3d/solvers/twostep.py:45-121)
// ---------------------------------------------------------------------------

template <typename R>
__global__ void __launch_bounds__(kThreads) k_ts_residual(size_t n, void* state, size_t sstride, cx<R>* r, const cx<R>* f) {
  StateView sv = view(state, sstride);
  if (!running(sv.st)) return;
  { const size_t vo = blockIdx.y * n; r += vo; f += vo; }
  n = used_len(sv.st, n);
  double a[1] = {0};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const cx<R> ri = csub(r[i], f[i]);
    r[i] = ri;
    a[0] += (double)ri.x * ri.x + (double)ri.y * ri.y;
  }
  double tot[1];
  if (reduce_last<1>(sv, a, tot) && threadIdx.x == 0) {
    em3d_krylov_state* st = sv.st;
    st->matvecs += 1;
    const int acts = st->matvecs + st->rmatvecs;
    const double rel = sqrt(tot[0]) / st->rhs_norm;
    record(sv, rel, acts);
    int stop = EM3D_RUNNING;
    if (!isfinite(rel)) stop = EM3D_NONFINITE;
    else if (rel < st->tol) stop = EM3D_CONVERGED;
    else if (st->guard >= 0.0 && rel > st->guard) stop = EM3D_DIVERGENCE_GUARD;
    else if (st->max_actions >= 0 && acts >= st->max_actions) stop = EM3D_MAX_OPERATOR_ACTIONS;
    else if (st->iter >= st->max_iter) stop = EM3D_MAX_ITER;
    else if (st->max_actions >= 0 && acts + 2 > st->max_actions) stop = EM3D_MAX_OPERATOR_ACTIONS;
    stop_rhs(st, state, stop);
  }
}

// a11 = Re<Hg,Hg>; first update: h = Re<g,g>/a11; later: the 2x2 minimal-residual
// system in (t, h) with dr = r - r_prev.
template <typename R>
__global__ void __launch_bounds__(kThreads) k_ts_coeffs(size_t n, void* state, size_t sstride, const cx<R>* r, const cx<R>* rp,
                                                        const cx<R>* g, const cx<R>* hg) {
  StateView sv = view(state, sstride);
  if (!running(sv.st)) return;
  { const size_t vo = blockIdx.y * n; r += vo; rp += vo; g += vo; hg += vo; }
  n = used_len(sv.st, n);
  const bool first = sv.st->first != 0;
  double a[5] = {0, 0, 0, 0, 0};  // a11, gg | a00, a01, b0, b1
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const cx<R> h = hg[i];
    a[0] += (double)h.x * h.x + (double)h.y * h.y;
    if (first) {
      const cx<R> gi = g[i];
      a[1] += (double)gi.x * gi.x + (double)gi.y * gi.y;
    } else {
      const cx<R> ri = r[i];
      const cx<R> dr = csub(ri, rp[i]);
      a[1] += (double)dr.x * dr.x + (double)dr.y * dr.y;
      a[2] += (double)dr.x * h.x + (double)dr.y * h.y;
      a[3] += (double)ri.x * dr.x + (double)ri.y * dr.y;
      a[4] += (double)ri.x * h.x + (double)ri.y * h.y;
    }
  }
  double tot[5];
  if (reduce_last<5>(sv, a, tot) && threadIdx.x == 0) {
    em3d_krylov_state* st = sv.st;
    st->rmatvecs += 1;
    st->matvecs += 1;
    const double a11 = tot[0];
    if (!isfinite(a11) || a11 <= 0.0) { stop_rhs(st, state, EM3D_BREAKDOWN_GRADIENT); return; }
    if (first) {
      st->t = 0.0;
      st->h = tot[1] / a11;
    } else {
      const double a00 = tot[1], a01 = tot[2], b0 = tot[3], b1 = tot[4];
      const double det = a00 * a11 - a01 * a01;
      const double scale = fmax(fmax(fabs(a00 * a11), fabs(a01 * a01)), 1.0);
      if (fabs(det) <= 1e-14 * scale) {
        st->t = 0.0;
        st->h = b1 / a11;
      } else {
        st->t = (b0 * a11 - b1 * a01) / det;
        st->h = (a00 * b1 - a01 * b0) / det;
      }
    }
  }
}

template <typename R>
__global__ void __launch_bounds__(kThreads) k_ts_update(size_t n, void* state, size_t sstride, cx<R>* u, cx<R>* up, const cx<R>* r,
                                                        cx<R>* rp, const cx<R>* g) {
  StateView sv = view(state, sstride);
  if (!running(sv.st)) return;
  { const size_t vo = blockIdx.y * n; u += vo; up += vo; r += vo; rp += vo; g += vo; }
  n = used_len(sv.st, n);
  const bool first = sv.st->first != 0;
  const R t = (R)sv.st->t, h = (R)sv.st->h;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const cx<R> ui = u[i];
    cx<R> nu;
    if (first) nu = csub(ui, cscale(g[i], h));
    else nu = csub(csub(ui, cscale(csub(ui, up[i]), t)), cscale(g[i], h));
    up[i] = ui;
    rp[i] = r[i];
    u[i] = nu;
  }
  double a[1] = {0};
  double tot[1];
  if (reduce_last<1>(sv, a, tot) && threadIdx.x == 0) {
    sv.st->iter += 1;
    sv.st->first = 0;
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------

inline int nblocks(size_t n) {
  size_t b = (n + kThreads - 1) / kThreads;
  if (b > (size_t)kMaxBlocks) b = kMaxBlocks;
  return (int)(b ? b : 1);
}

// CTAs per right-hand side of a batched launch: one wave of 256-thread CTAs
// for a single right-hand side; for a batch, about two waves in all (at least
// 32 per right-hand side), so that a wide batch does not launch a full wave
// for every entry (most of whose CTAs would find little to do, or nothing
// beyond a short entry's n_used).
inline int nblocks_batch(size_t n, int batch) {
  const int full = nblocks(n);
  if (batch <= 1) return full;
  int share = (2 * kMaxBlocks + batch - 1) / batch;
  if (share < 32) share = 32;
  return full < share ? full : share;
}

#define EM3D_DTYPE_DISPATCH(dtype, CALL)                                          \
  do {                                                                            \
    if ((dtype) == EM3D_C64) { using R = float; CALL; }                          \
    else if ((dtype) == EM3D_C128) { using R = double; CALL; }                   \
    else { em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128"); return EM3D_ERR_INVALID; } \
  } while (0)

inline int check_state(const void* state, size_t n) {
  if (!state) { em3d_set_last_error("state is NULL"); return EM3D_ERR_INVALID; }
  if (n == 0) { em3d_set_last_error("vector length must be positive"); return EM3D_ERR_INVALID; }
  return EM3D_OK;
}

inline int check_batch(int batch, size_t stride) {
  if (batch < 1 || batch > 65535) { em3d_set_last_error("batch must be in [1, 65535]"); return EM3D_ERR_INVALID; }
  if (batch > 1 && stride < kStateHeader) { em3d_set_last_error("state stride too small"); return EM3D_ERR_INVALID; }
  return EM3D_OK;
}

}  // namespace
}  // namespace em3d

using namespace em3d;

extern "C" {

size_t em3d_krylov_state_size(void) { return sizeof(em3d_krylov_state); }

size_t em3d_krylov_state_bytes(int hist_cap) {
  if (hist_cap < 1) return 0;
  return partials_off(hist_cap) + al256((size_t)kMaxBlocks * kPartials * sizeof(double));
}
size_t em3d_krylov_history_offset(int hist_cap) { return hist_off(hist_cap); }
size_t em3d_krylov_counts_offset(int hist_cap) { return counts_off(hist_cap); }

int em3d_vec_dots(int dtype, size_t n, int batch, const void* x0, const void* y0, const void* x1, const void* y1,
                  void* state, size_t state_stride, void* stream) {
  if (int rc = check_state(state, n)) return rc;
  if (int rc = check_batch(batch, state_stride)) return rc;
  if (!x0 || !y0 || (x1 && !y1)) { em3d_set_last_error("NULL vector"); return EM3D_ERR_INVALID; }
  cudaStream_t st = (cudaStream_t)stream;
  const dim3 grid(nblocks_batch(n, batch), batch);
  EM3D_DTYPE_DISPATCH(dtype, (k_dots<R><<<grid, kThreads, 0, st>>>(n, (const cx<R>*)x0, (const cx<R>*)y0,
                                                                     (const cx<R>*)x1, (const cx<R>*)y1, state,
                                                                     state_stride)));
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_vec_axpby(int dtype, size_t n, void* out, double a_re, double a_im, const void* x, double b_re, double b_im,
                   const void* y, void* stream) {
  if (!out || !x || n == 0) { em3d_set_last_error("bad vector arguments"); return EM3D_ERR_INVALID; }
  cudaStream_t st = (cudaStream_t)stream;
  EM3D_DTYPE_DISPATCH(dtype, (k_axpby<R><<<nblocks(n), kThreads, 0, st>>>(n, (cx<R>*)out, mk<R>((R)a_re, (R)a_im),
                                                                            (const cx<R>*)x, mk<R>((R)b_re, (R)b_im),
                                                                            (const cx<R>*)y)));
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_vec_convert(size_t n, int src_dtype, const void* src, int dst_dtype, void* dst, int accumulate, void* stream) {
  if (!src || !dst || n == 0) { em3d_set_last_error("bad vector arguments"); return EM3D_ERR_INVALID; }
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = nblocks(n);
  if (src_dtype == EM3D_C64 && dst_dtype == EM3D_C128)
    k_convert<float2, double2><<<nb, kThreads, 0, st>>>(n, (const float2*)src, (double2*)dst, accumulate);
  else if (src_dtype == EM3D_C128 && dst_dtype == EM3D_C64)
    k_convert<double2, float2><<<nb, kThreads, 0, st>>>(n, (const double2*)src, (float2*)dst, accumulate);
  else if (src_dtype == EM3D_C64 && dst_dtype == EM3D_C64)
    k_convert<float2, float2><<<nb, kThreads, 0, st>>>(n, (const float2*)src, (float2*)dst, accumulate);
  else if (src_dtype == EM3D_C128 && dst_dtype == EM3D_C128)
    k_convert<double2, double2><<<nb, kThreads, 0, st>>>(n, (const double2*)src, (double2*)dst, accumulate);
  else { em3d_set_last_error("bad dtype"); return EM3D_ERR_INVALID; }
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

#define EM3D_STEP(NAME, KERNEL, PARAMS, ARGS)                                         \
  int NAME PARAMS {                                                                   \
    if (int rc = check_state(state, n)) return rc;                                    \
    if (int rc = check_batch(batch, sstride)) return rc;                              \
    cudaStream_t st = (cudaStream_t)stream;                                           \
    const dim3 grid(nblocks_batch(n, batch), batch);                                  \
    EM3D_DTYPE_DISPATCH(dtype, (KERNEL<R><<<grid, kThreads, 0, st>>> ARGS));          \
    EM3D_LAUNCH_CHECK();                                                              \
    return EM3D_OK;                                                                   \
  }

EM3D_STEP(em3d_bicgstab_p, k_bicg_p,
          (int dtype, size_t n, int batch, void* state, size_t sstride, const void* r, void* p, const void* v, void* stream),
          (n, state, sstride, (const cx<R>*)r, (cx<R>*)p, (const cx<R>*)v))
EM3D_STEP(em3d_bicgstab_alpha, k_bicg_alpha,
          (int dtype, size_t n, int batch, void* state, size_t sstride, const void* r_hat, const void* v, void* stream),
          (n, state, sstride, (const cx<R>*)r_hat, (const cx<R>*)v))
EM3D_STEP(em3d_bicgstab_s, k_bicg_s,
          (int dtype, size_t n, int batch, void* state, size_t sstride, const void* r, const void* v, void* s, void* stream),
          (n, state, sstride, (const cx<R>*)r, (const cx<R>*)v, (cx<R>*)s))
int em3d_bicgstab_omega_parts(int nparts, void* state, const double* partials, void* stream) {
  if (int rc = check_state(state, 1)) return rc;
  if (nparts < 1 || !partials) { em3d_set_last_error("em3d_bicgstab_omega_parts: no partial sums"); return EM3D_ERR_INVALID; }
  k_bicg_omega_parts<<<1, kPartsThreads, 0, (cudaStream_t)stream>>>(nparts, state, partials);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_bicgstab_alpha_parts(int nparts, void* state, const double* partials, void* stream) {
  if (int rc = check_state(state, 1)) return rc;
  if (nparts < 1 || !partials) { em3d_set_last_error("em3d_bicgstab_alpha_parts: no partial sums"); return EM3D_ERR_INVALID; }
  k_bicg_alpha_parts<<<1, kPartsThreads, 0, (cudaStream_t)stream>>>(nparts, state, partials);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

EM3D_STEP(em3d_bicgstab_omega, k_bicg_omega,
          (int dtype, size_t n, int batch, void* state, size_t sstride, const void* t, const void* s, void* stream),
          (n, state, sstride, (const cx<R>*)t, (const cx<R>*)s))
EM3D_STEP(em3d_bicgstab_update, k_bicg_update,
          (int dtype, size_t n, int batch, void* state, size_t sstride, void* u, const void* p, const void* s, const void* t, void* r,
           const void* r_hat, void* stream),
          (n, state, sstride, (cx<R>*)u, (const cx<R>*)p, (const cx<R>*)s, (const cx<R>*)t, (cx<R>*)r, (const cx<R>*)r_hat))
EM3D_STEP(em3d_bicgstab_finalize, k_bicg_finalize,
          (int dtype, size_t n, int batch, void* state, size_t sstride, void* u, const void* p, void* stream),
          (n, state, sstride, (cx<R>*)u, (const cx<R>*)p))
EM3D_STEP(em3d_sim_residual, k_sim_residual,
          (int dtype, size_t n, int batch, void* state, size_t sstride, void* res, const void* f, void* stream),
          (n, state, sstride, (cx<R>*)res, (const cx<R>*)f))
EM3D_STEP(em3d_sim_update, k_sim_update,
          (int dtype, size_t n, int batch, void* state, size_t sstride, void* u, const void* res, void* stream),
          (n, state, sstride, (cx<R>*)u, (const cx<R>*)res))
EM3D_STEP(em3d_twostep_residual, k_ts_residual,
          (int dtype, size_t n, int batch, void* state, size_t sstride, void* r, const void* f, void* stream),
          (n, state, sstride, (cx<R>*)r, (const cx<R>*)f))
EM3D_STEP(em3d_twostep_coeffs, k_ts_coeffs,
          (int dtype, size_t n, int batch, void* state, size_t sstride, const void* r, const void* r_prev, const void* g, const void* hg,
           void* stream),
          (n, state, sstride, (const cx<R>*)r, (const cx<R>*)r_prev, (const cx<R>*)g, (const cx<R>*)hg))
EM3D_STEP(em3d_twostep_update, k_ts_update,
          (int dtype, size_t n, int batch, void* state, size_t sstride, void* u, void* u_prev, const void* r, void* r_prev, const void* g,
           void* stream),
          (n, state, sstride, (cx<R>*)u, (cx<R>*)u_prev, (const cx<R>*)r, (cx<R>*)r_prev, (const cx<R>*)g))

}  // extern "C"
