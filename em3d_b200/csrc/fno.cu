// Fourier-neural-operator warm start: forward, backward and optimiser kernels.
//
// Activations and weights are stored in ACT (bf16, or float for gradient
// checks); every product accumulates in FP32.  Layout of a channel tensor:
// (B, C, X, Y, Z), C-contiguous.  Mode-space tensors are complex FP32.
//
// Network (one layer l of L):
//   V_l   = DFT_trunc(v_l)            separable: z -> m modes, y -> 2m, x -> 2m
//   U_l   = W_l[mode] V_l[mode]       per-mode complex width x width mixing
//   s     = Re(IDFT_trunc(U_l))       weights c_kz / (X Y Z), c_0 = 1, c_kz>0 = 2
//   pre_l = A_l v_l + a_l + s
//   v_l+1 = GELU(pre_l)               (identity after the last layer)
// Lift (24 features -> width) before, projection (width -> 6) after; the
// prediction is u = f + (out_0 + i out_1, out_2 + i out_3, out_4 + i out_5).
//
// The truncated DFTs are small complex contractions along one axis,
// Y[o][j][i] = sum_l X[o][l][i] M[l][j]; the adjoint of a contraction with M
// is the contraction with conj(M)^T, so the backward pass reuses the same
// kernel with the forward/inverse matrices swapped.
#include <cuda_bf16.h>
#include <math.h>

#include "common.cuh"
#include "tma.cuh"

namespace em3d {
namespace fno {

constexpr int kMaxWidth = 32;
constexpr int kFeat = 24;

template <typename A> __device__ __forceinline__ float ld(const A* p) { return (float)(*p); }
template <> __device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16* p) { return __bfloat162float(*p); }
template <typename A> __device__ __forceinline__ A st(float v) { return (A)v; }
template <> __device__ __forceinline__ __nv_bfloat16 st<__nv_bfloat16>(float v) { return __float2bfloat16(v); }

// Row index -> batch entry: the row passes check that B X Y < 2^32, so the
// division runs in 32 bits (a 64-bit one is a long instruction sequence).
__device__ __forceinline__ size_t row_batch(size_t row, size_t XY) { return (size_t)((uint32_t)row / (uint32_t)XY); }

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// ---------------------------------------------------------------------------
// lift: 24 features per cell -> width channels
// ---------------------------------------------------------------------------

__device__ __forceinline__ void cell_features(const float2* chi, const float2* wave, size_t ncell, int b, size_t cell,
                                              float* f) {
  const float2* c = chi + (size_t)b * 9 * ncell + cell;
  const float2* w = wave + (size_t)b * 3 * ncell + cell;
#pragma unroll
  for (int i = 0; i < 9; ++i) { const float2 v = c[(size_t)i * ncell]; f[2 * i] = v.x; f[2 * i + 1] = v.y; }
#pragma unroll
  for (int i = 0; i < 3; ++i) { const float2 v = w[(size_t)i * ncell]; f[18 + 2 * i] = v.x; f[19 + 2 * i] = v.y; }
}

template <typename ACT>
__global__ void k_lift(int B, size_t ncell, int W, const float2* chi, const float2* wave, const ACT* P, const float* pb,
                       ACT* v0) {
  __shared__ float sP[kMaxWidth * kFeat], sb[kMaxWidth];
  for (int i = threadIdx.x; i < W * kFeat; i += blockDim.x) sP[i] = ld(P + i);
  for (int i = threadIdx.x; i < W; i += blockDim.x) sb[i] = pb[i];
  __syncthreads();
  const size_t total = (size_t)B * ncell;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(t / ncell);
    const size_t cell = t - (size_t)b * ncell;
    float f[kFeat];
    cell_features(chi, wave, ncell, b, cell, f);
    for (int co = 0; co < W; ++co) {
      float acc = sb[co];
#pragma unroll
      for (int k = 0; k < kFeat; ++k) acc += sP[co * kFeat + k] * f[k];
      v0[((size_t)b * W + co) * ncell + cell] = st<ACT>(acc);
    }
  }
}

// dP[co][f] += sum dv0[co] feat[f];  dpb[co] += sum dv0[co]
__global__ void k_lift_bwd(int B, size_t ncell, int W, const float2* chi, const float2* wave, const float* dv0,
                           float* dP, float* dpb) {
  __shared__ float acc[kMaxWidth * (kFeat + 1)];
  for (int i = threadIdx.x; i < W * (kFeat + 1); i += blockDim.x) acc[i] = 0.0f;
  __syncthreads();
  const size_t total = (size_t)B * ncell;
  float local[kFeat + 1];
  for (int co = 0; co < W; ++co) {
#pragma unroll
    for (int k = 0; k <= kFeat; ++k) local[k] = 0.0f;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
      const int b = (int)(t / ncell);
      const size_t cell = t - (size_t)b * ncell;
      float f[kFeat];
      cell_features(chi, wave, ncell, b, cell, f);
      const float g = dv0[((size_t)b * W + co) * ncell + cell];
#pragma unroll
      for (int k = 0; k < kFeat; ++k) local[k] += g * f[k];
      local[kFeat] += g;
    }
#pragma unroll
    for (int k = 0; k <= kFeat; ++k) {
      float v = local[k];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if ((threadIdx.x & 31) == 0) atomicAdd(&acc[co * (kFeat + 1) + k], v);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < W * (kFeat + 1); i += blockDim.x) {
    const int co = i / (kFeat + 1), k = i - co * (kFeat + 1);
    if (k < kFeat) atomicAdd(&dP[co * kFeat + k], acc[i]);
    else atomicAdd(&dpb[co], acc[i]);
  }
}

// ---------------------------------------------------------------------------
// contractions along one axis: Y[o][j][i] = sum_l X[o][l][i] M[l][j]
// ---------------------------------------------------------------------------

template <typename ACT>
__global__ void k_contract_r2c(size_t outer, int L, int J, int inner, const ACT* X, const float2* M, float2* Y) {
  const size_t total = outer * J * inner;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % inner);
    const int j = (int)((t / inner) % J);
    const size_t o = t / ((size_t)inner * J);
    const ACT* x = X + o * L * inner + i;
    float re = 0.0f, im = 0.0f;
    for (int l = 0; l < L; ++l) {
      const float v = ld(x + (size_t)l * inner);
      const float2 m = M[l * J + j];
      re += v * m.x;
      im += v * m.y;
    }
    Y[t] = make_float2(re, im);
  }
}

__global__ void k_contract_c2c(size_t outer, int L, int J, int inner, const float2* X, const float2* M, float2* Y) {
  const size_t total = outer * J * inner;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % inner);
    const int j = (int)((t / inner) % J);
    const size_t o = t / ((size_t)inner * J);
    const float2* x = X + o * L * inner + i;
    float re = 0.0f, im = 0.0f;
    for (int l = 0; l < L; ++l) {
      const float2 v = x[(size_t)l * inner];
      const float2 m = M[l * J + j];
      re += v.x * m.x - v.y * m.y;
      im += v.x * m.y + v.y * m.x;
    }
    Y[t] = make_float2(re, im);
  }
}

// Y[o][j][i] += Re(sum_l X[o][l][i] M[l][j])  (adjoint of a real-input DFT)
__global__ void k_contract_c2r_acc(size_t outer, int L, int J, int inner, const float2* X, const float2* M, float* Y) {
  const size_t total = outer * J * inner;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % inner);
    const int j = (int)((t / inner) % J);
    const size_t o = t / ((size_t)inner * J);
    const float2* x = X + o * L * inner + i;
    float re = 0.0f;
    for (int l = 0; l < L; ++l) {
      const float2 v = x[(size_t)l * inner];
      const float2 m = M[l * J + j];
      re += v.x * m.x - v.y * m.y;
    }
    Y[t] += re;
  }
}

// ---------------------------------------------------------------------------
// per-mode channel mixing; W stored (ci, co, mode) as complex ACT pairs
// ---------------------------------------------------------------------------

template <typename ACT>
__global__ void k_modemix(int B, int W, int nm, const float2* V, const ACT* Wre, const ACT* Wim, float2* U) {
  const size_t total = (size_t)B * W * nm;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int mode = (int)(t % nm);
    const int co = (int)((t / nm) % W);
    const int b = (int)(t / ((size_t)nm * W));
    float re = 0.0f, im = 0.0f;
    for (int ci = 0; ci < W; ++ci) {
      const float2 v = V[((size_t)b * W + ci) * nm + mode];
      const size_t wi = ((size_t)ci * W + co) * nm + mode;
      const float wr = ld(Wre + wi), wim = ld(Wim + wi);
      re += v.x * wr - v.y * wim;
      im += v.x * wim + v.y * wr;
    }
    U[t] = make_float2(re, im);
  }
}

// dV[b][ci][mode] = sum_co dU[b][co][mode] conj(W[ci][co][mode])
template <typename ACT>
__global__ void k_modemix_bwd_v(int B, int W, int nm, const float2* dU, const ACT* Wre, const ACT* Wim, float2* dV) {
  const size_t total = (size_t)B * W * nm;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int mode = (int)(t % nm);
    const int ci = (int)((t / nm) % W);
    const int b = (int)(t / ((size_t)nm * W));
    float re = 0.0f, im = 0.0f;
    for (int co = 0; co < W; ++co) {
      const float2 g = dU[((size_t)b * W + co) * nm + mode];
      const size_t wi = ((size_t)ci * W + co) * nm + mode;
      const float wr = ld(Wre + wi), wim = ld(Wim + wi);
      re += g.x * wr + g.y * wim;
      im += g.y * wr - g.x * wim;
    }
    dV[t] = make_float2(re, im);
  }
}

// dW[ci][co][mode] += sum_b conj(V[b][ci][mode]) dU[b][co][mode]
__global__ void k_modemix_bwd_w(int B, int W, int nm, const float2* V, const float2* dU, float* dWre, float* dWim) {
  const size_t total = (size_t)W * W * nm;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int mode = (int)(t % nm);
    const int co = (int)((t / nm) % W);
    const int ci = (int)(t / ((size_t)nm * W));
    float re = 0.0f, im = 0.0f;
    for (int b = 0; b < B; ++b) {
      const float2 v = V[((size_t)b * W + ci) * nm + mode];
      const float2 g = dU[((size_t)b * W + co) * nm + mode];
      re += v.x * g.x + v.y * g.y;
      im += v.x * g.y - v.y * g.x;
    }
    dWre[t] += re;
    dWim[t] += im;
  }
}

// ---------------------------------------------------------------------------
// inverse z transform + pointwise linear + GELU; one CTA per (b, x, y) row,
// one thread per z
// ---------------------------------------------------------------------------

template <typename ACT>
__global__ void k_layer_out(int W, int X, int Y, int Z, int m, const ACT* vin, const float2* Uxy, const ACT* A,
                            const float* a, int apply_gelu, ACT* pre_out, ACT* vout) {
  extern __shared__ float sh[];
  float* sA = sh;                                   // W*W
  float* sa = sA + W * W;                           // W
  float2* sU = reinterpret_cast<float2*>(sa + W);   // W*m
  const int row = blockIdx.x;                        // (b, x, y)
  const int y = row % Y;
  const int x = (row / Y) % X;
  const int b = row / (X * Y);
  const size_t ncell = (size_t)X * Y * Z;
  for (int i = threadIdx.x; i < W * W; i += blockDim.x) sA[i] = ld(A + i);
  for (int i = threadIdx.x; i < W; i += blockDim.x) sa[i] = a[i];
  for (int i = threadIdx.x; i < W * m; i += blockDim.x) {
    const int co = i / m, k = i - co * m;
    sU[i] = Uxy[((((size_t)b * W + co) * X + x) * Y + y) * m + k];
  }
  __syncthreads();
  const int z = threadIdx.x;
  if (z >= Z) return;
  const size_t base = (size_t)b * W * ncell + ((size_t)x * Y + y) * Z + z;
  float v[kMaxWidth];
  for (int ci = 0; ci < W; ++ci) v[ci] = ld(vin + base + (size_t)ci * ncell);
  float cs[16], sn[16];
  const float inv = 1.0f / (float)ncell;
  for (int k = 0; k < m; ++k) {
    float s, c;
    sincospif(2.0f * (float)((k * z) % Z) / (float)Z, &s, &c);
    const float w = (k == 0 ? 1.0f : 2.0f) * inv;
    cs[k] = c * w;
    sn[k] = s * w;
  }
  for (int co = 0; co < W; ++co) {
    float acc = sa[co];
    for (int ci = 0; ci < W; ++ci) acc += sA[co * W + ci] * v[ci];
    for (int k = 0; k < m; ++k) {
      const float2 u = sU[co * m + k];
      acc += u.x * cs[k] - u.y * sn[k];
    }
    pre_out[base + (size_t)co * ncell] = st<ACT>(acc);
    vout[base + (size_t)co * ncell] = st<ACT>(apply_gelu ? gelu(acc) : acc);
  }
}

// Backward of k_layer_out for one (b, x, y) row:
//   gpre = gout * GELU'(pre);  gin = A^T gpre (pointwise part);
//   dUxy[co][k] = sum_z gpre[co][z] (c_k / XYZ) e^{-2 pi i k z / Z}
template <typename ACT>
__global__ void k_layer_out_bwd(int W, int X, int Y, int Z, int m, const float* gout, const ACT* pre, const ACT* A,
                                int apply_gelu, float* gpre, float* gin, float2* dUxy) {
  extern __shared__ float sh[];
  float* sA = sh;                                         // W*W
  float* sg = sA + W * W;                                 // W*Z gpre of the row
  float2* stw = reinterpret_cast<float2*>(sg + W * Z);    // m*Z: e^{-2 pi i k z / Z}
  const int row = blockIdx.x;
  const int y = row % Y;
  const int x = (row / Y) % X;
  const int b = row / (X * Y);
  const size_t ncell = (size_t)X * Y * Z;
  for (int i = threadIdx.x; i < W * W; i += blockDim.x) sA[i] = ld(A + i);
  for (int i = threadIdx.x; i < m * Z; i += blockDim.x) {
    const int k = i / Z, zz = i - k * Z;
    float s, c;
    sincospif(2.0f * (float)((k * zz) % Z) / (float)Z, &s, &c);
    stw[i] = make_float2(c, -s);
  }
  const int z = threadIdx.x;
  const size_t base = (size_t)b * W * ncell + ((size_t)x * Y + y) * Z + z;
  if (z < Z) {
    for (int co = 0; co < W; ++co) {
      float g = gout[base + (size_t)co * ncell];
      if (apply_gelu) g *= gelu_grad(ld(pre + base + (size_t)co * ncell));
      gpre[base + (size_t)co * ncell] = g;
      sg[co * Z + z] = g;
    }
  }
  __syncthreads();
  if (z < Z) {
    for (int ci = 0; ci < W; ++ci) {
      float acc = 0.0f;
      for (int co = 0; co < W; ++co) acc += sA[co * W + ci] * sg[co * Z + z];
      gin[base + (size_t)ci * ncell] = acc;
    }
  }
  // spectral gradient of the row: W*m complex sums over z
  const float inv = 1.0f / (float)ncell;
  for (int i = threadIdx.x; i < W * m; i += blockDim.x) {
    const int co = i / m, k = i - co * m;
    float re = 0.0f, im = 0.0f;
    for (int zz = 0; zz < Z; ++zz) {
      const float2 w = stw[k * Z + zz];
      const float g = sg[co * Z + zz];
      re += g * w.x;
      im += g * w.y;
    }
    const float w = (k == 0 ? 1.0f : 2.0f) * inv;
    dUxy[((((size_t)b * W + co) * X + x) * Y + y) * m + k] = make_float2(re * w, im * w);
  }
}

// dA[co][ci] += sum_cells gpre[co] v[ci];  da[co] += sum gpre[co]
// One CTA of W*W threads per chunk of cells; tiles staged in shared memory.
template <typename ACT>
__global__ void k_pointwise_wgrad(int B, size_t ncell, int W, const float* gpre, const ACT* v, float* dA, float* da,
                                  size_t chunk) {
  constexpr int T = 32;
  __shared__ float sg[kMaxWidth][T + 1], sv[kMaxWidth][T + 1];
  const int tid = threadIdx.x;
  const int co = tid / W, ci = tid - (tid / W) * W;
  const size_t total = (size_t)B * ncell;
  const size_t begin = blockIdx.x * chunk;
  const size_t end = begin + chunk < total ? begin + chunk : total;
  float acc = 0.0f, accb = 0.0f;
  for (size_t t0 = begin; t0 < end; t0 += T) {
    for (int i = tid; i < W * T; i += blockDim.x) {
      const int c = i / T, k = i - c * T;
      const size_t t = t0 + k;
      float g = 0.0f, vv = 0.0f;
      if (t < end) {
        const int b = (int)(t / ncell);
        const size_t cell = t - (size_t)b * ncell;
        g = gpre[((size_t)b * W + c) * ncell + cell];
        vv = ld(v + ((size_t)b * W + c) * ncell + cell);
      }
      sg[c][k] = g;
      sv[c][k] = vv;
    }
    __syncthreads();
    if (tid < W * W) {
#pragma unroll 8
      for (int k = 0; k < T; ++k) acc += sg[co][k] * sv[ci][k];
      if (ci == 0)
        for (int k = 0; k < T; ++k) accb += sg[co][k];
    }
    __syncthreads();
  }
  if (tid < W * W) {
    atomicAdd(&dA[co * W + ci], acc);
    if (ci == 0) atomicAdd(&da[co], accb);
  }
}

// ---------------------------------------------------------------------------
// projection width -> 6 and u = f + out
// ---------------------------------------------------------------------------

template <typename ACT>
__global__ void k_project(int B, size_t ncell, int W, const ACT* v, const ACT* Q, const float* qb, const float2* wave,
                          float2* u) {
  __shared__ float sQ[6 * kMaxWidth], sq[6];
  for (int i = threadIdx.x; i < 6 * W; i += blockDim.x) sQ[i] = ld(Q + i);
  if (threadIdx.x < 6) sq[threadIdx.x] = qb[threadIdx.x];
  __syncthreads();
  const size_t total = (size_t)B * ncell;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(t / ncell);
    const size_t cell = t - (size_t)b * ncell;
    float o[6];
#pragma unroll
    for (int j = 0; j < 6; ++j) o[j] = sq[j];
    for (int ci = 0; ci < W; ++ci) {
      const float vv = ld(v + ((size_t)b * W + ci) * ncell + cell);
#pragma unroll
      for (int j = 0; j < 6; ++j) o[j] += sQ[j * W + ci] * vv;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t idx = ((size_t)b * 3 + c) * ncell + cell;
      const float2 f = wave[idx];
      u[idx] = make_float2(f.x + o[2 * c], f.y + o[2 * c + 1]);
    }
  }
}

// du: gradient wrt u (dL/dRe + i dL/dIm).  gv = Q^T dout; dQ += dout v; dqb += dout
template <typename ACT>
__global__ void k_project_bwd(int B, size_t ncell, int W, const ACT* v, const ACT* Q, const float2* du, float* gv,
                              float* dQ, float* dqb) {
  __shared__ float sQ[6 * kMaxWidth];
  __shared__ float acc[6 * (kMaxWidth + 1)];
  for (int i = threadIdx.x; i < 6 * W; i += blockDim.x) sQ[i] = ld(Q + i);
  for (int i = threadIdx.x; i < 6 * (W + 1); i += blockDim.x) acc[i] = 0.0f;
  __syncthreads();
  const size_t total = (size_t)B * ncell;
  float lQ[6 * (kMaxWidth + 1)];
  for (int i = 0; i < 6 * (W + 1); ++i) lQ[i] = 0.0f;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(t / ncell);
    const size_t cell = t - (size_t)b * ncell;
    float d[6];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float2 g = du[((size_t)b * 3 + c) * ncell + cell];
      d[2 * c] = g.x;
      d[2 * c + 1] = g.y;
    }
    for (int ci = 0; ci < W; ++ci) {
      const float vv = ld(v + ((size_t)b * W + ci) * ncell + cell);
      float g = 0.0f;
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        g += sQ[j * W + ci] * d[j];
        lQ[j * (W + 1) + ci] += d[j] * vv;
      }
      gv[((size_t)b * W + ci) * ncell + cell] = g;
    }
#pragma unroll
    for (int j = 0; j < 6; ++j) lQ[j * (W + 1) + W] += d[j];
  }
  for (int i = 0; i < 6 * (W + 1); ++i) {
    float val = lQ[i];
    for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&acc[i], val);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 6 * (W + 1); i += blockDim.x) {
    const int j = i / (W + 1), k = i - j * (W + 1);
    if (k < W) atomicAdd(&dQ[j * W + k], acc[i]);
    else atomicAdd(&dqb[j], acc[i]);
  }
}

// ---------------------------------------------------------------------------
// loss: mean_b ||pred_b - t_b||^2 / ||t_b||^2 and its gradient
// ---------------------------------------------------------------------------

__global__ void k_loss_terms(int B, size_t n, const float2* pred, const float2* target, double* terms) {
  // terms[2b] = ||pred_b - t_b||^2, terms[2b+1] = ||t_b||^2  (atomic FP64 accumulation)
  const int b = blockIdx.y;
  double num = 0.0, den = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float2 p = pred[(size_t)b * n + i], t = target[(size_t)b * n + i];
    const double dx = (double)p.x - t.x, dy = (double)p.y - t.y;
    num += dx * dx + dy * dy;
    den += (double)t.x * t.x + (double)t.y * t.y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    num += __shfl_xor_sync(0xffffffffu, num, o);
    den += __shfl_xor_sync(0xffffffffu, den, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&terms[2 * b], num);
    atomicAdd(&terms[2 * b + 1], den);
  }
}

__global__ void k_loss_grad(int B, size_t n, const float2* pred, const float2* target, const double* terms,
                            float2* grad) {
  const int b = blockIdx.y;
  const float s = (float)(2.0 / (terms[2 * b + 1] * B));
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float2 p = pred[(size_t)b * n + i], t = target[(size_t)b * n + i];
    grad[(size_t)b * n + i] = make_float2(s * (p.x - t.x), s * (p.y - t.y));
  }
}

// ---------------------------------------------------------------------------
// Adam on FP32 master weights, writing the ACT copy used by the kernels
// ---------------------------------------------------------------------------

template <typename ACT>
__global__ void k_adam(size_t n, float* w, const float* g, float* m1, float* m2, float lr, float b1, float b2,
                       float eps, float bc1, float bc2, ACT* wact) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float v = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = v;
    const float upd = lr * (a / bc1) / (sqrtf(v / bc2) + eps);
    const float nw = w[i] - upd;
    w[i] = nw;
    if (wact) wact[i] = st<ACT>(nw);
  }
}

template <typename ACT> __global__ void k_cast(size_t n, const float* src, ACT* dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = st<ACT>(src[i]);
}

template <typename ACT> __global__ void k_uncast(size_t n, const ACT* src, float* dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = ld(src + i);
}

// ---------------------------------------------------------------------------
// Fused z-row kernel of the forward pass (Z <= 128, W <= 32, m <= 16).
//
// One group of R = 128 / Z consecutive (b, x, y) rows per step, one thread per
// cell.  Each thread keeps its cell's channels in registers:
//   LIFT:  o = P feat + pb                              (feat: 24 per cell)
//   layer: pre = A v + a + sum_k Re(U[k] (c_k/XYZ) e^{+2 pi i k z/Z});
//          o = GELU(pre) (identity on the last layer)
// and writes what the caller asks for: pre (training), o (the next layer's
// input), the truncated z-DFT of o, Vz[k] = sum_z o[z] e^{-2 pi i k z/Z}
// (computed from a shared-memory copy of the rows, so the next layer does not
// re-read o from memory), and/or the projection u = f + Q o + qb.  o is
// rounded to the activation type before the DFT and the projection, so they
// see exactly the values a separate pass would read back.
// ---------------------------------------------------------------------------

constexpr int kMaxModes = 16;
constexpr int kRowThreads = 128;

template <typename ACT, bool LIFT>
__global__ void __launch_bounds__(kRowThreads) k_row_fwd(
    int B, int W, int X, int Y, int Z, int m, const float2* __restrict__ chi, const float2* __restrict__ wave,
    const ACT* __restrict__ vin, const float2* __restrict__ Uxy, const ACT* __restrict__ Wt,
    const float* __restrict__ bias, int apply_gelu, ACT* __restrict__ pre_out, ACT* __restrict__ vout,
    float2* __restrict__ Vz, const ACT* __restrict__ Q, const float* __restrict__ qb, float2* __restrict__ u_out) {
  constexpr int KIN = LIFT ? kFeat : kMaxWidth;
  extern __shared__ __align__(16) float sh[];
  float* sW = sh;                                        // kMaxWidth x KIN
  float* sb = sW + kMaxWidth * KIN;                      // kMaxWidth
  float* sQ = sb + kMaxWidth;                            // 6 x kMaxWidth
  float* sqb = sQ + 6 * kMaxWidth;                       // 8
  float2* stw = reinterpret_cast<float2*>(sqb + 8);      // Z x kMaxModes: e^{-2 pi i k z / Z} at [z][k]
  const int R = kRowThreads / Z;
  const int TS = ((Z + 3) & ~3) + 4;                     // tile row stride: a multiple of 4 floats (16-byte rows)
  float2* sU = stw + Z * kMaxModes;                      // R x kMaxWidth x kMaxModes
  float* tile = reinterpret_cast<float*>(sU + R * kMaxWidth * kMaxModes);  // R x kMaxWidth x TS

  const int kin = LIFT ? kFeat : W;
  for (int i = threadIdx.x; i < kMaxWidth * KIN; i += blockDim.x) {
    const int co = i / KIN, c = i - co * KIN;
    sW[i] = (co < W && c < kin) ? ld(Wt + co * kin + c) : 0.0f;
  }
  for (int i = threadIdx.x; i < kMaxWidth; i += blockDim.x) sb[i] = i < W ? bias[i] : 0.0f;
  for (int i = threadIdx.x; i < 6 * kMaxWidth; i += blockDim.x) {
    const int j = i / kMaxWidth, c = i - j * kMaxWidth;
    sQ[i] = (Q != nullptr && c < W) ? ld(Q + j * W + c) : 0.0f;
  }
  if (threadIdx.x < 8) sqb[threadIdx.x] = (qb != nullptr && threadIdx.x < 6) ? qb[threadIdx.x] : 0.0f;
  for (int i = threadIdx.x; i < Z * kMaxModes; i += blockDim.x) {
    const int zz = i / kMaxModes, k = i - zz * kMaxModes;
    float s = 0.0f, c = 0.0f;
    if (k < m) sincospif(2.0f * (float)((k * zz) % Z) / (float)Z, &s, &c);
    stw[i] = make_float2(c, -s);
  }
  __syncthreads();

  const int z = threadIdx.x % Z;
  const int rr = threadIdx.x / Z;
  const bool lane_on = rr < R;
  const size_t XY = (size_t)X * Y;
  const size_t ncell = XY * Z;
  const size_t nrows = (size_t)B * XY;
  // inverse-DFT weights of this thread's z (loop invariant; zero for k >= m)
  float cs[kMaxModes], sn[kMaxModes];
  {
    const float inv = 1.0f / (float)ncell;
#pragma unroll
    for (int k = 0; k < kMaxModes; ++k) {
      const float2 t = stw[z * kMaxModes + k];
      const float w = (k == 0 ? 1.0f : 2.0f) * inv;
      cs[k] = t.x * w;
      sn[k] = -t.y * w;
    }
  }
  const int mb = (m + 3) / 4;  // mode blocks of 4 in the DFT phase
  const size_t ngroups = (nrows + R - 1) / R;
  for (size_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
    const size_t row0 = g * R;
    if (!LIFT) {
      for (int i = threadIdx.x; i < R * kMaxWidth * kMaxModes; i += blockDim.x) {
        const int r = i / (kMaxWidth * kMaxModes), rem = i - r * (kMaxWidth * kMaxModes);
        const int co = rem / kMaxModes, k = rem - co * kMaxModes;
        const size_t row = row0 + r;
        float2 val = make_float2(0.0f, 0.0f);
        if (row < nrows && co < W && k < m) {
          const size_t b = row_batch(row, XY), xy = row - b * XY;
          val = Uxy[((b * W + co) * XY + xy) * m + k];
        }
        sU[i] = val;
      }
      __syncthreads();
    }
    const size_t row = row0 + rr;
    const bool valid = lane_on && row < nrows;
    if (valid) {
      const size_t b = row_batch(row, XY), xy = row - b * XY;
      const size_t cell = xy * Z + z;
      const size_t base = b * W * ncell + cell;
      float o[kMaxWidth];
      if (LIFT) {
        float f[kFeat];
        cell_features(chi, wave, ncell, (int)b, cell, f);
#pragma unroll
        for (int co = 0; co < kMaxWidth; ++co) {
          const float4* w4 = reinterpret_cast<const float4*>(sW + co * KIN);
          float acc = sb[co];
#pragma unroll
          for (int c4 = 0; c4 < kFeat / 4; ++c4) {
            const float4 w = w4[c4];
            acc += w.x * f[4 * c4] + w.y * f[4 * c4 + 1] + w.z * f[4 * c4 + 2] + w.w * f[4 * c4 + 3];
          }
          o[co] = acc;
        }
      } else {
        float v[kMaxWidth];
#pragma unroll
        for (int ci = 0; ci < kMaxWidth; ++ci) v[ci] = ci < W ? ld(vin + base + (size_t)ci * ncell) : 0.0f;
        const float4* u4 = reinterpret_cast<const float4*>(sU + rr * kMaxWidth * kMaxModes);
#pragma unroll
        for (int co = 0; co < kMaxWidth; ++co) {
          const float4* w4 = reinterpret_cast<const float4*>(sW + co * KIN);
          float acc = sb[co];
#pragma unroll
          for (int c4 = 0; c4 < kMaxWidth / 4; ++c4) {
            const float4 w = w4[c4];
            acc += w.x * v[4 * c4] + w.y * v[4 * c4 + 1] + w.z * v[4 * c4 + 2] + w.w * v[4 * c4 + 3];
          }
#pragma unroll
          for (int k2 = 0; k2 < kMaxModes / 2; ++k2) {
            if (2 * k2 < m) {
              const float4 uk = u4[co * (kMaxModes / 2) + k2];   // modes 2 k2 and 2 k2 + 1
              acc += uk.x * cs[2 * k2] - uk.y * sn[2 * k2] + uk.z * cs[2 * k2 + 1] - uk.w * sn[2 * k2 + 1];
            }
          }
          o[co] = acc;
        }
      }
#pragma unroll
      for (int co = 0; co < kMaxWidth; ++co) {
        if (co < W) {
          if (pre_out) pre_out[base + (size_t)co * ncell] = st<ACT>(o[co]);
          const ACT q = st<ACT>((!LIFT && apply_gelu) ? gelu(o[co]) : o[co]);
          if (vout) vout[base + (size_t)co * ncell] = q;
          o[co] = ld(&q);
        } else {
          o[co] = 0.0f;
        }
      }
      if (u_out) {
        float p[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) {
          const float4* q4 = reinterpret_cast<const float4*>(sQ + j * kMaxWidth);
          float acc = sqb[j];
#pragma unroll
          for (int c4 = 0; c4 < kMaxWidth / 4; ++c4) {
            const float4 w = q4[c4];
            acc += w.x * o[4 * c4] + w.y * o[4 * c4 + 1] + w.z * o[4 * c4 + 2] + w.w * o[4 * c4 + 3];
          }
          p[j] = acc;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const size_t idx = (b * 3 + c) * ncell + cell;
          const float2 fw = wave[idx];
          u_out[idx] = make_float2(fw.x + p[2 * c], fw.y + p[2 * c + 1]);
        }
      }
      if (Vz) {
        float* t = tile + rr * kMaxWidth * TS;
#pragma unroll
        for (int co = 0; co < kMaxWidth; ++co)
          if (co < W) t[co * TS + z] = o[co];
      }
    }
    if (Vz) {
      __syncthreads();
      // one (row, channel, block of 4 modes) per item; 4 cells per tile load
      for (int i = threadIdx.x; i < R * W * mb; i += blockDim.x) {
        const int r = i / (W * mb), rem = i - r * (W * mb), co = rem / mb, kb = rem - co * mb;
        const size_t rw = row0 + r;
        if (rw < nrows) {
          const float* t = tile + (r * kMaxWidth + co) * TS;
          float re[4] = {0.0f, 0.0f, 0.0f, 0.0f}, im[4] = {0.0f, 0.0f, 0.0f, 0.0f};
          const int z4 = Z & ~3;
          for (int zz = 0; zz < z4; zz += 4) {
            const float4 tv = *reinterpret_cast<const float4*>(t + zz);
            const float tz[4] = {tv.x, tv.y, tv.z, tv.w};
#pragma unroll
            for (int d = 0; d < 4; ++d) {
              const float4* w4 = reinterpret_cast<const float4*>(stw + (zz + d) * kMaxModes + 4 * kb);
              const float4 wa = w4[0], wb = w4[1];
              re[0] += tz[d] * wa.x; im[0] += tz[d] * wa.y;
              re[1] += tz[d] * wa.z; im[1] += tz[d] * wa.w;
              re[2] += tz[d] * wb.x; im[2] += tz[d] * wb.y;
              re[3] += tz[d] * wb.z; im[3] += tz[d] * wb.w;
            }
          }
          for (int zz = z4; zz < Z; ++zz) {
            const float tzz = t[zz];
#pragma unroll
            for (int d = 0; d < 4; ++d) {
              const float2 w = stw[zz * kMaxModes + 4 * kb + d];
              re[d] += tzz * w.x;
              im[d] += tzz * w.y;
            }
          }
          const size_t b = row_batch(rw, XY), xy = rw - b * XY;
          float2* dst = Vz + ((b * W + co) * XY + xy) * m;
#pragma unroll
          for (int d = 0; d < 4; ++d)
            if (4 * kb + d < m) dst[4 * kb + d] = make_float2(re[d], im[d]);
        }
      }
    }
    __syncthreads();
  }
}

inline size_t row_fwd_smem(bool lift, int Z, int m) {
  (void)m;
  const int KIN = lift ? kFeat : kMaxWidth;
  const int R = kRowThreads / Z;
  return sizeof(float) * (kMaxWidth * KIN + kMaxWidth + 6 * kMaxWidth + 8) + sizeof(float2) * (size_t)Z * kMaxModes +
         sizeof(float2) * (size_t)R * kMaxWidth * kMaxModes +
         sizeof(float) * (size_t)R * kMaxWidth * (((Z + 3) & ~3) + 4);
}

// ---------------------------------------------------------------------------
// Tensor-core z-row kernel (bf16 activations, width 32, Z in {32, 64, 128}).
//
// Per row the layer is two small GEMMs on mma.sync m16n8k16 (bf16 in, FP32
// accumulate), one warp per 32 cells of the row:
//   O[co][z]  = sum_ci A[co][ci] v[ci][z] + sum_j Ucat[co][j] T[j][z]
//               (Ucat = Re/Im of the row's mode coefficients, T the weighted
//                inverse-DFT cos / -sin table), + a[co], GELU
//   Vz[co][j] = sum_z O[co][z] F[z][j]   (F = cos / -sin: next layer's z-DFT)
// The second GEMM takes its A operand straight from the first one's
// accumulators (the m16n8 C layout of two neighbouring n-tiles is the m16k16 A
// layout), after rounding O to bf16, so it sees exactly the stored values.
// The lift uses the same path with A = P and the 24 cell features (padded to
// 32) in place of v.  Twiddles and the mode coefficients enter the tensor
// cores as bf16, like every other activation of the network.
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ uint32_t pack_raw(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  __nv_bfloat162 v;
  v.x = lo;
  v.y = hi;
  return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

constexpr int kTcCols = 128;  // cells per CTA step (R rows of Z)

inline size_t row_fwd_tc_smem() {
  return sizeof(__nv_bfloat16) * 2 * 32 * kTcCols   // Vs, Os
         + sizeof(float2) * 4 * 32 * kMaxModes      // sU (up to 4 rows)
         + sizeof(float) * 4 * 32 * 32              // per-warp DFT partials
         + sizeof(float) * (32 + 6 * 32 + 8);       // bias, Q, qb
}

template <bool LIFT>
__global__ void __launch_bounds__(128) k_row_fwd_tc(
    int B, int X, int Y, int Z, int m, const float2* __restrict__ chi, const float2* __restrict__ wave,
    const __nv_bfloat16* __restrict__ vin, const float2* __restrict__ Uxy, const __nv_bfloat16* __restrict__ Wt,
    const float* __restrict__ bias, int apply_gelu, __nv_bfloat16* __restrict__ pre_out,
    __nv_bfloat16* __restrict__ vout, float2* __restrict__ Vz, const __nv_bfloat16* __restrict__ Q,
    const float* __restrict__ qb, float2* __restrict__ u_out) {
  constexpr int W = 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __nv_bfloat16* Vs = reinterpret_cast<__nv_bfloat16*>(smem_raw);   // [32][kTcCols]
  __nv_bfloat16* Os = Vs + 32 * kTcCols;                            // [32][kTcCols]
  float2* sU = reinterpret_cast<float2*>(Os + 32 * kTcCols);        // [4][32][kMaxModes]
  float* red = reinterpret_cast<float*>(sU + 4 * 32 * kMaxModes);   // [4 warps][32][32]
  float* sb = red + 4 * 32 * 32;
  float* sQ = sb + 32;
  float* sqb = sQ + 6 * 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tg = lane & 3;
  const int WPR = Z / 32, R = 4 / WPR;
  const int wr = warp / WPR, zs = (warp % WPR) * 32;
  const int kin = LIFT ? kFeat : W;
  const size_t XY = (size_t)X * Y, ncell = XY * Z, nrows = (size_t)B * XY;

  for (int i = threadIdx.x; i < 32; i += blockDim.x) sb[i] = bias[i];
  for (int i = threadIdx.x; i < 6 * 32; i += blockDim.x) sQ[i] = Q ? __bfloat162float(Q[i]) : 0.0f;
  if (threadIdx.x < 8) sqb[threadIdx.x] = (qb && threadIdx.x < 6) ? qb[threadIdx.x] : 0.0f;

  // constant fragments: weights (A), inverse-DFT table (B), forward-DFT table (B)
  uint32_t Aw[2][2][4], Bt[2][4][2], Bf[2][4][2];
  {
    const __nv_bfloat16 zero = __float2bfloat16(0.0f);
    auto wv = [&](int r, int c) { return c < kin ? Wt[r * kin + c] : zero; };
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        const int r0 = mt * 16 + g, c0 = ks * 16 + tg * 2;
        Aw[mt][ks][0] = pack_raw(wv(r0, c0), wv(r0, c0 + 1));
        Aw[mt][ks][1] = pack_raw(wv(r0 + 8, c0), wv(r0 + 8, c0 + 1));
        Aw[mt][ks][2] = pack_raw(wv(r0, c0 + 8), wv(r0, c0 + 9));
        Aw[mt][ks][3] = pack_raw(wv(r0 + 8, c0 + 8), wv(r0 + 8, c0 + 9));
      }
    const float inv = 1.0f / (float)ncell;
    // T[j][z]: j = 2k -> cos(theta) w_k, j = 2k+1 -> -sin(theta) w_k; F[z][j]: cos / -sin
    auto tw = [&](int j, int z, bool weighted) {
      if (j >= 2 * m) return 0.0f;
      const int k = j >> 1;
      float sn, cs;
      sincospif(2.0f * (float)((k * z) % Z) / (float)Z, &sn, &cs);
      const float w = weighted ? (k == 0 ? 1.0f : 2.0f) * inv : 1.0f;
      return (j & 1) ? -sn * w : cs * w;
    };
#pragma unroll
    for (int ks = 0; ks < 2; ++ks)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int k0 = ks * 16 + tg * 2;
        const int z = zs + nt * 8 + g;
        Bt[ks][nt][0] = pack_bf16(tw(k0, z, true), tw(k0 + 1, z, true));
        Bt[ks][nt][1] = pack_bf16(tw(k0 + 8, z, true), tw(k0 + 9, z, true));
        // F: K = z (this warp's 32 cells, k-step ks), N = j
        const int zk = zs + ks * 16 + tg * 2, j = nt * 8 + g;
        Bf[ks][nt][0] = pack_bf16(tw(j, zk, false), tw(j, zk + 1, false));
        Bf[ks][nt][1] = pack_bf16(tw(j, zk + 8, false), tw(j, zk + 9, false));
      }
  }
  const int nt3 = (2 * m + 7) / 8;
  __syncthreads();

  const size_t ngroups = (nrows + R - 1) / R;
  for (size_t gi = blockIdx.x; gi < ngroups; gi += gridDim.x) {
    const size_t row0 = gi * R;
    // ---- stage the rows' inputs
    if (LIFT) {
      for (int i = threadIdx.x; i < R * Z; i += blockDim.x) {
        const int r = i / Z, z = i - r * Z;
        const size_t row = row0 + r;
        float f[kFeat];
        if (row < nrows) {
          const size_t b = row_batch(row, XY), xy = row - b * XY;
          cell_features(chi, wave, ncell, (int)b, xy * Z + z, f);
        } else {
#pragma unroll
          for (int c = 0; c < kFeat; ++c) f[c] = 0.0f;
        }
#pragma unroll
        for (int c = 0; c < 32; ++c) Vs[c * kTcCols + r * Z + z] = __float2bfloat16(c < kFeat ? f[c] : 0.0f);
      }
    } else {
      const int chunks = Z / 8;
      for (int i = threadIdx.x; i < R * 32 * chunks; i += blockDim.x) {
        const int r = i / (32 * chunks), rem = i - r * 32 * chunks, ci = rem / chunks, q = rem - ci * chunks;
        const size_t row = row0 + r;
        uint4 val = make_uint4(0, 0, 0, 0);
        if (row < nrows) {
          const size_t b = row_batch(row, XY), xy = row - b * XY;
          val = *reinterpret_cast<const uint4*>(vin + (b * W + ci) * ncell + xy * Z + q * 8);
        }
        *reinterpret_cast<uint4*>(Vs + ci * kTcCols + r * Z + q * 8) = val;
      }
      for (int i = threadIdx.x; i < R * 32 * kMaxModes; i += blockDim.x) {
        const int r = i / (32 * kMaxModes), rem = i - r * 32 * kMaxModes, co = rem / kMaxModes,
                  k = rem - co * kMaxModes;
        const size_t row = row0 + r;
        float2 val = make_float2(0.0f, 0.0f);
        if (row < nrows && k < m) {
          const size_t b = row_batch(row, XY), xy = row - b * XY;
          val = Uxy[((b * W + co) * XY + xy) * m + k];
        }
        sU[i] = val;
      }
    }
    __syncthreads();

    // ---- GEMM 1 (+ inverse DFT) on this warp's 32 cells
    float acc[2][4][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[mt][nt][e] = 0.0f;
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      uint32_t bv[4][2];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int col = wr * Z + zs + nt * 8 + g, k0 = ks * 16 + tg * 2;
        bv[nt][0] = pack_raw(Vs[k0 * kTcCols + col], Vs[(k0 + 1) * kTcCols + col]);
        bv[nt][1] = pack_raw(Vs[(k0 + 8) * kTcCols + col], Vs[(k0 + 9) * kTcCols + col]);
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[mt][nt], Aw[mt][ks], bv[nt]);
    }
    if (!LIFT) {
      const float2* u = sU + wr * 32 * kMaxModes;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
          const int c0 = mt * 16 + g, j0 = ks * 16 + tg * 2;   // j0 even: (Re, Im) of mode j0 / 2
          const float2 u00 = u[c0 * kMaxModes + (j0 >> 1)], u10 = u[(c0 + 8) * kMaxModes + (j0 >> 1)];
          const float2 u01 = u[c0 * kMaxModes + (j0 >> 1) + 4], u11 = u[(c0 + 8) * kMaxModes + (j0 >> 1) + 4];
          uint32_t au[4];
          au[0] = pack_bf16(u00.x, u00.y);
          au[1] = pack_bf16(u10.x, u10.y);
          au[2] = pack_bf16(u01.x, u01.y);
          au[3] = pack_bf16(u11.x, u11.y);
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[mt][nt], au, Bt[ks][nt]);
        }
      }
    }

    // ---- epilogue: bias, GELU, bf16; keep the rounded values for GEMM 2
    const size_t row = row0 + wr;
    const bool valid = row < nrows;
    const size_t b = valid ? row_batch(row, XY) : 0, xy = valid ? row - b * XY : 0;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int co = mt * 16 + g + 8 * h;
          const int z = zs + nt * 8 + tg * 2;
          float o0 = acc[mt][nt][2 * h] + sb[co], o1 = acc[mt][nt][2 * h + 1] + sb[co];
          if (pre_out && valid)
            *reinterpret_cast<uint32_t*>(pre_out + (b * W + co) * ncell + xy * Z + z) = pack_bf16(o0, o1);
          if (!LIFT && apply_gelu) { o0 = gelu(o0); o1 = gelu(o1); }
          const uint32_t q = pack_bf16(o0, o1);
          *reinterpret_cast<uint32_t*>(Os + co * kTcCols + wr * Z + z) = q;
          const __nv_bfloat162 qq = *reinterpret_cast<const __nv_bfloat162*>(&q);
          acc[mt][nt][2 * h] = __bfloat162float(qq.x);
          acc[mt][nt][2 * h + 1] = __bfloat162float(qq.y);
        }

    // ---- GEMM 2: this warp's share of the next layer's z-DFT
    if (Vz) {
      float d[2][4][4];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int e = 0; e < 4; ++e) d[mt][nt][e] = 0.0f;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks)
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
          uint32_t a[4];
          a[0] = pack_bf16(acc[mt][2 * ks][0], acc[mt][2 * ks][1]);
          a[1] = pack_bf16(acc[mt][2 * ks][2], acc[mt][2 * ks][3]);
          a[2] = pack_bf16(acc[mt][2 * ks + 1][0], acc[mt][2 * ks + 1][1]);
          a[3] = pack_bf16(acc[mt][2 * ks + 1][2], acc[mt][2 * ks + 1][3]);
#pragma unroll
          for (int nt = 0; nt < 4; ++nt)
            if (nt < nt3) mma_bf16(d[mt][nt], a, Bf[ks][nt]);
        }
      float* rw = red + warp * 32 * 32;
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int co = mt * 16 + g + (e >= 2 ? 8 : 0), j = nt * 8 + tg * 2 + (e & 1);
            rw[co * 32 + j] = d[mt][nt][e];
          }
    }
    __syncthreads();
    if (Vz) {
      for (int i = threadIdx.x; i < R * 32 * m; i += blockDim.x) {
        const int r = i / (32 * m), rem = i - r * 32 * m, co = rem / m, k = rem - co * m;
        const size_t rw = row0 + r;
        if (rw < nrows) {
          float re = 0.0f, im = 0.0f;
          for (int w = r * WPR; w < (r + 1) * WPR; ++w) {
            re += red[(w * 32 + co) * 32 + 2 * k];
            im += red[(w * 32 + co) * 32 + 2 * k + 1];
          }
          const size_t bb = row_batch(rw, XY), xyy = rw - bb * XY;
          Vz[((bb * W + co) * XY + xyy) * m + k] = make_float2(re, im);
        }
      }
    }
    if (vout) {
      const int chunks = Z / 8;
      for (int i = threadIdx.x; i < R * 32 * chunks; i += blockDim.x) {
        const int r = i / (32 * chunks), rem = i - r * 32 * chunks, co = rem / chunks, q = rem - co * chunks;
        const size_t rw = row0 + r;
        if (rw < nrows) {
          const size_t bb = row_batch(rw, XY), xyy = rw - bb * XY;
          *reinterpret_cast<uint4*>(vout + (bb * W + co) * ncell + xyy * Z + q * 8) =
              *reinterpret_cast<const uint4*>(Os + co * kTcCols + r * Z + q * 8);
        }
      }
    }
    if (u_out) {
      for (int i = threadIdx.x; i < R * Z; i += blockDim.x) {
        const int r = i / Z, z = i - r * Z;
        const size_t rw = row0 + r;
        if (rw < nrows) {
          float p[6];
#pragma unroll
          for (int j = 0; j < 6; ++j) p[j] = sqb[j];
#pragma unroll 8
          for (int co = 0; co < 32; ++co) {
            const float o = __bfloat162float(Os[co * kTcCols + r * Z + z]);
#pragma unroll
            for (int j = 0; j < 6; ++j) p[j] += sQ[j * 32 + co] * o;
          }
          const size_t bb = row_batch(rw, XY), xyy = rw - bb * XY;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const size_t idx = (bb * 3 + c) * ncell + xyy * Z + z;
            const float2 fw = wave[idx];
            u_out[idx] = make_float2(fw.x + p[2 * c], fw.y + p[2 * c + 1]);
          }
        }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Register-blocked contraction Y[o][j][i] (op)= sum_l X[o][l][i] M[l][j] with
// M (L x J) in shared memory; each thread produces JB consecutive j of one
// (o, i), so X is read once instead of once per output.
// ---------------------------------------------------------------------------

template <int JB, bool REAL_ACC>
__global__ void k_contract_blk(size_t outer, int L, int J, int inner, const float2* __restrict__ Xin,
                               const float2* __restrict__ M, void* __restrict__ Yout) {
  extern __shared__ float2 sM[];
  for (int i = threadIdx.x; i < L * J; i += blockDim.x) sM[i] = M[i];
  __syncthreads();
  const int nb = (J + JB - 1) / JB;
  const size_t total = outer * (size_t)nb * inner;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % inner);
    const int jb = (int)((t / inner) % nb);
    const size_t o = t / ((size_t)inner * nb);
    const float2* x = Xin + o * L * inner + i;
    float re[JB], im[JB];
#pragma unroll
    for (int jj = 0; jj < JB; ++jj) re[jj] = im[jj] = 0.0f;
    const int j0 = jb * JB;
    for (int l = 0; l < L; ++l) {
      const float2 v = x[(size_t)l * inner];
      const float2* mr = sM + l * J + j0;
#pragma unroll
      for (int jj = 0; jj < JB; ++jj) {
        if (j0 + jj < J) {
          const float2 mm = mr[jj];
          re[jj] += v.x * mm.x - v.y * mm.y;
          im[jj] += v.x * mm.y + v.y * mm.x;
        }
      }
    }
#pragma unroll
    for (int jj = 0; jj < JB; ++jj) {
      if (j0 + jj < J) {
        const size_t idx = (o * J + j0 + jj) * inner + i;
        if (REAL_ACC) reinterpret_cast<float*>(Yout)[idx] += re[jj];
        else reinterpret_cast<float2*>(Yout)[idx] = make_float2(re[jj], im[jj]);
      }
    }
  }
}


// ---------------------------------------------------------------------------
// The y and x truncated DFTs of one layer in one pass.  One CTA per
// (batch x channel, kz mode) slice: forward, the slice Vz[x][y] (X x Y,
// elements m apart in memory) goes to V[jx][jy] = sum_x fx[x][jx]
// sum_y Vz[x][y] fy[y][jy] (2m x 2m); inverse, U[jx][jy] goes to
// Uxy[x][y] = sum_jy iy[jy][y] sum_jx U[jx][jy] ix[jx][x].  The same sums as
// the two contractions it replaces (k_contract_blk along y, then x), with
// the intermediate in shared memory instead of global memory.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void cmac(float& re, float& im, float2 a, float2 b) {
  re += a.x * b.x - a.y * b.y;
  im += a.x * b.y + a.y * b.x;
}

// Each thread accumulates kSpecB outputs along the last index (NB apart, so
// neighbouring threads read neighbouring elements), and a value read from
// shared memory serves kSpecB products; rows of the slice are padded by one
// element so the threads of a warp (several rows) hit different banks.
constexpr int kSpecB = 4;

__global__ void __launch_bounds__(256) k_spec_fwd(int X, int Y, int m, const float2* __restrict__ Vz,
                                                  const float2* __restrict__ fy, const float2* __restrict__ fx,
                                                  float2* __restrict__ V) {
  const int J = 2 * m, NB = (J + kSpecB - 1) / kSpecB, YP = Y + 1;
  const size_t bw = blockIdx.x;
  const int k = blockIdx.y;
  extern __shared__ float2 sh2[];
  float2* S = sh2;            // X * (Y + 1)
  float2* T = S + X * YP;     // X * J
  float2* Fy = T + X * J;     // Y * J
  float2* Fx = Fy + Y * J;    // X * J
  const float2* src = Vz + bw * X * Y * m + k;
  for (int i = threadIdx.x; i < X * Y; i += blockDim.x) {
    const int x = i / Y;
    S[i + x] = src[(size_t)i * m];
  }
  for (int i = threadIdx.x; i < Y * J; i += blockDim.x) Fy[i] = fy[i];
  for (int i = threadIdx.x; i < X * J; i += blockDim.x) Fx[i] = fx[i];
  __syncthreads();
  // T[x][j] = sum_y S[x][y] Fy[y][j]
  for (int o = threadIdx.x; o < X * NB; o += blockDim.x) {
    const int x = o / NB, jb = o - x * NB;
    float re[kSpecB] = {}, im[kSpecB] = {};
    const float2* srow = S + x * YP;
#pragma unroll 4
    for (int y = 0; y < Y; ++y) {
      const float2 a = srow[y];
      const float2* f = Fy + y * J + jb;
#pragma unroll
      for (int jj = 0; jj < kSpecB; ++jj)
        if (jb + jj * NB < J) cmac(re[jj], im[jj], a, f[jj * NB]);
    }
#pragma unroll
    for (int jj = 0; jj < kSpecB; ++jj)
      if (jb + jj * NB < J) T[x * J + jb + jj * NB] = make_float2(re[jj], im[jj]);
  }
  __syncthreads();
  // V[jx][jy] = sum_x Fx[x][jx] T[x][jy]
  float2* dst = V + bw * J * J * m + k;
  for (int o = threadIdx.x; o < J * NB; o += blockDim.x) {
    const int jx = o / NB, jb = o - jx * NB;
    float re[kSpecB] = {}, im[kSpecB] = {};
#pragma unroll 4
    for (int x = 0; x < X; ++x) {
      const float2 a = Fx[x * J + jx];
      const float2* t = T + x * J + jb;
#pragma unroll
      for (int jj = 0; jj < kSpecB; ++jj)
        if (jb + jj * NB < J) cmac(re[jj], im[jj], t[jj * NB], a);
    }
#pragma unroll
    for (int jj = 0; jj < kSpecB; ++jj)
      if (jb + jj * NB < J) dst[(size_t)(jx * J + jb + jj * NB) * m] = make_float2(re[jj], im[jj]);
  }
}

__global__ void __launch_bounds__(256) k_spec_inv(int X, int Y, int m, const float2* __restrict__ U,
                                                  const float2* __restrict__ ix, const float2* __restrict__ iy,
                                                  float2* __restrict__ Uxy) {
  const int J = 2 * m, NB = (J + kSpecB - 1) / kSpecB, NYB = (Y + kSpecB - 1) / kSpecB;
  const size_t bw = blockIdx.x;
  const int k = blockIdx.y;
  extern __shared__ float2 sh2[];
  float2* Us = sh2;           // J * J
  float2* T = Us + J * J;     // X * J
  float2* Ix = T + X * J;     // J * X
  float2* Iy = Ix + J * X;    // J * Y
  const float2* src = U + bw * J * J * m + k;
  for (int i = threadIdx.x; i < J * J; i += blockDim.x) Us[i] = src[(size_t)i * m];
  for (int i = threadIdx.x; i < J * X; i += blockDim.x) Ix[i] = ix[i];
  for (int i = threadIdx.x; i < J * Y; i += blockDim.x) Iy[i] = iy[i];
  __syncthreads();
  // T[x][jy] = sum_jx Us[jx][jy] Ix[jx][x]
  for (int o = threadIdx.x; o < X * NB; o += blockDim.x) {
    const int x = o / NB, jb = o - x * NB;
    float re[kSpecB] = {}, im[kSpecB] = {};
#pragma unroll 4
    for (int jx = 0; jx < J; ++jx) {
      const float2 a = Ix[jx * X + x];
      const float2* u = Us + jx * J + jb;
#pragma unroll
      for (int jj = 0; jj < kSpecB; ++jj)
        if (jb + jj * NB < J) cmac(re[jj], im[jj], u[jj * NB], a);
    }
#pragma unroll
    for (int jj = 0; jj < kSpecB; ++jj)
      if (jb + jj * NB < J) T[x * J + jb + jj * NB] = make_float2(re[jj], im[jj]);
  }
  __syncthreads();
  // Uxy[x][y] = sum_jy T[x][jy] Iy[jy][y]
  float2* dst = Uxy + bw * X * Y * m + k;
  for (int o = threadIdx.x; o < X * NYB; o += blockDim.x) {
    const int x = o / NYB, yb = o - x * NYB;
    float re[kSpecB] = {}, im[kSpecB] = {};
#pragma unroll 4
    for (int jy = 0; jy < J; ++jy) {
      const float2 a = T[x * J + jy];
      const float2* f = Iy + jy * Y + yb;
#pragma unroll
      for (int yy = 0; yy < kSpecB; ++yy)
        if (yb + yy * NYB < Y) cmac(re[yy], im[yy], a, f[yy * NYB]);
    }
#pragma unroll
    for (int yy = 0; yy < kSpecB; ++yy)
      if (yb + yy * NYB < Y) dst[(size_t)(x * Y + yb + yy * NYB) * m] = make_float2(re[yy], im[yy]);
  }
}

// ---------------------------------------------------------------------------
// Grid resampling for evaluating the network on the half-resolution grid:
// 2x2x2 cell means down (complex64 or complex128 in, complex64 out) and
// trilinear interpolation up between cell centres (clamped at the faces, the
// align_corners = false convention), complex64 in, complex64 or complex128
// out.  Fields are (C, nx, ny, nz) on the coarse side, C stacked components.
// ---------------------------------------------------------------------------

template <typename S>
__global__ void k_down2(int C, int nx, int ny, int nz, const S* __restrict__ in, float2* __restrict__ out) {
  const size_t n = (size_t)C * nx * ny * nz;
  const size_t fy = 2 * (size_t)ny, fz = 2 * (size_t)nz;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(o % nz);
    const int y = (int)((o / nz) % ny);
    const int x = (int)((o / ((size_t)nz * ny)) % nx);
    const size_t c = o / ((size_t)nz * ny * nx);
    const S* b = in + ((c * 2 * nx + 2 * x) * fy + 2 * y) * fz + 2 * z;
    double re = 0.0, im = 0.0;
#pragma unroll
    for (int dx = 0; dx < 2; ++dx)
#pragma unroll
      for (int dy = 0; dy < 2; ++dy)
#pragma unroll
        for (int dz = 0; dz < 2; ++dz) {
          const S v = b[(dx * fy + dy) * fz + dz];
          re += (double)v.x;
          im += (double)v.y;
        }
    out[o] = make_float2((float)(0.125 * re), (float)(0.125 * im));
  }
}

// fine index j of a doubled axis -> coarse neighbours (i0, i1) and weight of i1
__device__ __forceinline__ void up_axis(int j, int n, int& i0, int& i1, float& w1) {
  const int i = j >> 1;
  if (j & 1) {  // source coordinate i + 1/4
    i0 = i;
    i1 = min(i + 1, n - 1);
    w1 = 0.25f;
  } else {      // source coordinate i - 1/4, clamped to 0 at the face
    i0 = i > 0 ? i - 1 : 0;
    i1 = i;
    w1 = i > 0 ? 0.75f : 0.0f;
  }
}

template <typename D>
__global__ void k_up2(int C, int nx, int ny, int nz, const float2* __restrict__ in, D* __restrict__ out) {
  const int Fx = 2 * nx, Fy = 2 * ny, Fz = 2 * nz;
  const size_t n = (size_t)C * Fx * Fy * Fz;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int jz = (int)(o % Fz);
    const int jy = (int)((o / Fz) % Fy);
    const int jx = (int)((o / ((size_t)Fz * Fy)) % Fx);
    const size_t c = o / ((size_t)Fz * Fy * Fx);
    int x0, x1, y0, y1, z0, z1;
    float wx, wy, wz;
    up_axis(jx, nx, x0, x1, wx);
    up_axis(jy, ny, y0, y1, wy);
    up_axis(jz, nz, z0, z1, wz);
    const float2* b = in + c * (size_t)nx * ny * nz;
    float re = 0.0f, im = 0.0f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int bb = 0; bb < 2; ++bb)
#pragma unroll
        for (int d = 0; d < 2; ++d) {
          const float w = (a ? wx : 1.0f - wx) * (bb ? wy : 1.0f - wy) * (d ? wz : 1.0f - wz);
          const float2 v = b[((size_t)(a ? x1 : x0) * ny + (bb ? y1 : y0)) * nz + (d ? z1 : z0)];
          re += w * v.x;
          im += w * v.y;
        }
    D r;
    r.x = re;
    r.y = im;
    out[o] = r;
  }
}

inline int blocks_for(size_t n, int threads = 256) {
  size_t b = (n + threads - 1) / threads;
  if (b > (size_t)148 * 32) b = (size_t)148 * 32;
  return (int)(b ? b : 1);
}

#include "fno_umma.cuh"

// Failed bounded waits of the tcgen05 row pass (read and cleared by
// em3d_fno_failures).
__device__ unsigned int g_fno_fails = 0;

}  // namespace fno
}  // namespace em3d

using namespace em3d;
using namespace em3d::fno;

enum { FNO_BF16 = 0, FNO_F32 = 1 };

#define FNO_DISPATCH(act, CALL)                                                    \
  do {                                                                             \
    if ((act) == FNO_BF16) { using ACT = __nv_bfloat16; CALL; }                   \
    else if ((act) == FNO_F32) { using ACT = float; CALL; }                       \
    else { em3d_set_last_error("act dtype must be 0 (bf16) or 1 (float)"); return EM3D_ERR_INVALID; } \
  } while (0)

// Opt a kernel in to more than 48 KB of dynamic shared memory.
static bool allow_dyn_smem(const void* fn, size_t bytes) {
  if (bytes <= 48 * 1024) return true;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) { em3d_set_last_error(cudaGetErrorString(e)); return false; }
  return true;
}

template <typename ACT>
static int launch_row_fwd(bool lift, int grid, size_t smem, cudaStream_t st, int B, int W, int X, int Y, int Z, int m,
                          const void* chi, const void* wave, const void* vin, const void* Uxy, const void* Wt,
                          const float* bias, int apply_gelu, void* pre_out, void* vout, void* Vz, const void* Q,
                          const float* qb, void* u_out) {
  if (lift) {
    if (!allow_dyn_smem((const void*)k_row_fwd<ACT, true>, smem)) return EM3D_ERR_CUDA;
    k_row_fwd<ACT, true><<<grid, kRowThreads, smem, st>>>(
        B, W, X, Y, Z, m, (const float2*)chi, (const float2*)wave, nullptr, nullptr, (const ACT*)Wt, bias, 0,
        (ACT*)pre_out, (ACT*)vout, (float2*)Vz, (const ACT*)Q, qb, (float2*)u_out);
  } else {
    if (!allow_dyn_smem((const void*)k_row_fwd<ACT, false>, smem)) return EM3D_ERR_CUDA;
    k_row_fwd<ACT, false><<<grid, kRowThreads, smem, st>>>(
        B, W, X, Y, Z, m, (const float2*)chi, (const float2*)wave, (const ACT*)vin, (const float2*)Uxy,
        (const ACT*)Wt, bias, apply_gelu, (ACT*)pre_out, (ACT*)vout, (float2*)Vz, (const ACT*)Q, qb,
        (float2*)u_out);
  }
  return EM3D_OK;
}

static int check_width(int W) {
  if (W < 1 || W > kMaxWidth) { em3d_set_last_error("FNO width must be in [1, 32]"); return EM3D_ERR_INVALID; }
  return EM3D_OK;
}

extern "C" {

int em3d_fno_lift(int act, int B, size_t ncell, int W, const void* chi, const void* wave, const void* P,
                  const float* pb, void* v0, void* stream) {
  if (int rc = check_width(W)) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  FNO_DISPATCH(act, (k_lift<ACT><<<blocks_for((size_t)B * ncell), 256, 0, st>>>(
                         B, ncell, W, (const float2*)chi, (const float2*)wave, (const ACT*)P, pb, (ACT*)v0)));
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_lift_bwd(int B, size_t ncell, int W, const void* chi, const void* wave, const float* dv0, float* dP,
                      float* dpb, void* stream) {
  if (int rc = check_width(W)) return rc;
  k_lift_bwd<<<blocks_for((size_t)B * ncell) / 8 + 1, 256, 0, (cudaStream_t)stream>>>(
      B, ncell, W, (const float2*)chi, (const float2*)wave, dv0, dP, dpb);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

// Outputs per thread of the blocked contraction: every thread reads its input
// column once per JB outputs, so a large JB saves loads, while a small JB
// gives more threads to small problems (the x contractions have outer = B W).
static int contract_jb(size_t outer, int J, size_t inner) {
  const size_t cols = outer * inner;
  if (cols * (size_t)((J + 7) / 8) < (size_t)148 * 256 * 2) return 2;
  return 8;
}

#define CONTRACT_JB_DISPATCH(jb, CALL)                                    \
  do {                                                                    \
    switch (jb) {                                                         \
      case 2: { constexpr int JB = 2; CALL; break; }                      \
      case 4: { constexpr int JB = 4; CALL; break; }                      \
      case 12: { constexpr int JB = 12; CALL; break; }                    \
      case 24: { constexpr int JB = 24; CALL; break; }                    \
      default: { constexpr int JB = 8; CALL; break; }                     \
    }                                                                     \
  } while (0)

int em3d_fno_contract(int kind, int act, size_t outer, int L, int J, int inner, const void* X, const void* M, void* Y,
                      void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = outer * (size_t)J * inner;
  if (kind == 0) {
    FNO_DISPATCH(act, (k_contract_r2c<ACT><<<blocks_for(n), 256, 0, st>>>(outer, L, J, inner, (const ACT*)X,
                                                                           (const float2*)M, (float2*)Y)));
  } else if (kind == 1 || kind == 2) {
    const size_t smem = sizeof(float2) * (size_t)L * J;
    if (smem <= 48 * 1024) {
      int jb = em3d_get_tuning(EM3D_TUNE_FNO_CONTRACT);
      if (jb == 0) jb = contract_jb(outer, J, inner);
      if (kind == 1) {
        CONTRACT_JB_DISPATCH(jb, (k_contract_blk<JB, false><<<blocks_for(outer * (size_t)((J + JB - 1) / JB) * inner),
                                                                256, smem, st>>>(outer, L, J, inner, (const float2*)X,
                                                                                 (const float2*)M, Y)));
      } else {
        CONTRACT_JB_DISPATCH(jb, (k_contract_blk<JB, true><<<blocks_for(outer * (size_t)((J + JB - 1) / JB) * inner),
                                                               256, smem, st>>>(outer, L, J, inner, (const float2*)X,
                                                                                (const float2*)M, Y)));
      }
    } else if (kind == 1) {
      k_contract_c2c<<<blocks_for(n), 256, 0, st>>>(outer, L, J, inner, (const float2*)X, (const float2*)M,
                                                    (float2*)Y);
    } else {
      k_contract_c2r_acc<<<blocks_for(n), 256, 0, st>>>(outer, L, J, inner, (const float2*)X, (const float2*)M,
                                                        (float*)Y);
    }
  } else {
    em3d_set_last_error("contract kind must be 0 (real->complex), 1 (complex), 2 (complex->real, accumulate)");
    return EM3D_ERR_INVALID;
  }
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_failures(int reset) {
  unsigned int n = 0;
  if (cudaMemcpyFromSymbol(&n, g_fno_fails, sizeof n) != cudaSuccess) {
    em3d_set_last_error("em3d_fno_failures: cannot read the counter");
    return -1;
  }
  if (reset && n) {
    const unsigned int zero = 0;
    if (cudaMemcpyToSymbol(g_fno_fails, &zero, sizeof zero) != cudaSuccess) return -1;
  }
  return (int)n;
}

int em3d_fno_spectral(int inverse, int BW, int m, int X, int Y, const void* in, const void* mx, const void* my,
                      void* out, void* stream) {
  if (BW < 1 || m < 1 || X < 2 * m || Y < 2 * m || !in || !mx || !my || !out) {
    em3d_set_last_error("em3d_fno_spectral: bad sizes or NULL arrays (need X, Y >= 2 m)");
    return EM3D_ERR_INVALID;
  }
  const size_t J = 2 * (size_t)m;
  const size_t smem = sizeof(float2) * (inverse ? J * J + 2 * (size_t)X * J + J * Y
                                                : (size_t)X * (Y + 1) + 2 * (size_t)X * J + (size_t)Y * J);
  if (smem > 227 * 1024) {
    em3d_set_last_error("em3d_fno_spectral: slice too large for shared memory (use em3d_fno_contract)");
    return EM3D_ERR_UNSUPPORTED;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const dim3 grid(BW, m);
  static bool opted = false;  // both kernels opted in to 227 KB once (first call outside any capture)
  if (!opted) {
    EM3D_CUDA_TRY(cudaFuncSetAttribute(k_spec_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    EM3D_CUDA_TRY(cudaFuncSetAttribute(k_spec_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    opted = true;
  }
  if (inverse) {
    k_spec_inv<<<grid, 256, smem, st>>>(X, Y, m, (const float2*)in, (const float2*)mx, (const float2*)my,
                                        (float2*)out);
  } else {
    k_spec_fwd<<<grid, 256, smem, st>>>(X, Y, m, (const float2*)in, (const float2*)my, (const float2*)mx,
                                        (float2*)out);
  }
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_row_forward(int act, int lift, int B, int W, int X, int Y, int Z, int m, const void* chi,
                         const void* wave, const void* vin, const void* Uxy, const void* Wt, const float* bias,
                         int apply_gelu, void* pre_out, void* vout, void* Vz, const void* Q, const float* qb,
                         void* u_out, void* stream) {
  if (int rc = check_width(W)) return rc;
  if (Z < 1 || Z > kRowThreads || m < 1 || m > kMaxModes || 2 * m > Z || X < 1 || Y < 1 || B < 1) {
    em3d_set_last_error("row_forward: needs 1 <= Z <= 128, 1 <= modes <= 16, 2 modes <= Z");
    return EM3D_ERR_UNSUPPORTED;
  }
  if ((size_t)B * X * Y >= ((size_t)1 << 32)) {
    em3d_set_last_error("row_forward: B X Y must stay below 2^32 rows");
    return EM3D_ERR_UNSUPPORTED;
  }
  if (lift ? (!chi || !wave) : (!vin || !Uxy)) {
    em3d_set_last_error("row_forward: missing input");
    return EM3D_ERR_INVALID;
  }
  if (u_out && (!Q || !qb || !wave)) {
    em3d_set_last_error("row_forward: projection needs Q, qb and wave");
    return EM3D_ERR_INVALID;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const size_t smem = row_fwd_smem(lift != 0, Z, m);
  if (smem > 200 * 1024) {
    em3d_set_last_error("row_forward: rows too short (Z < 4) for the shared-memory tile");
    return EM3D_ERR_UNSUPPORTED;
  }
  const int R = kRowThreads / Z;
  const size_t groups = ((size_t)B * X * Y + R - 1) / R;
  const int grid = (int)(groups < (size_t)148 * 12 ? groups : (size_t)148 * 12);
  const int row_mode = em3d_get_tuning(EM3D_TUNE_FNO_SIMT);  // 0 auto, 1 CUDA cores, 2 tcgen05, 3 mma.sync
  if (act == FNO_BF16 && W == 32 && Z % 32 == 0 && row_mode != 1) {
    const size_t tsm = row_fwd_tc_smem();
    const int Rt = 128 / Z;
    const size_t tgroups = ((size_t)B * X * Y + Rt - 1) / Rt;
    const int tgrid = (int)(tgroups < (size_t)148 * 8 ? tgroups : (size_t)148 * 8);
    using BF = __nv_bfloat16;
    if (!lift && row_mode != 3) {
      // the layer pass on tcgen05 (fno_umma.cuh)
      static unsigned int* fails = nullptr;
      if (fails == nullptr) EM3D_CUDA_TRY(cudaGetSymbolAddress((void**)&fails, g_fno_fails));
      const size_t usm = UmmaSmem::TOTAL;
      if (!allow_dyn_smem((const void*)k_row_fwd_umma, usm)) return EM3D_ERR_CUDA;
      const size_t tiles = ((size_t)B * X * Y + Rt - 1) / Rt;
      const int ugrid = (int)(tiles < (size_t)148 * 2 ? tiles : (size_t)148 * 2);
      k_row_fwd_umma<<<ugrid, 128, usm, st>>>(B, X, Y, Z, m, (const BF*)vin, (const float2*)Uxy, (const BF*)Wt,
                                               bias, apply_gelu, (BF*)pre_out, (BF*)vout, (float2*)Vz,
                                               (const BF*)Q, qb, (const float2*)wave, (float2*)u_out, fails);
      EM3D_LAUNCH_CHECK();
      return EM3D_OK;
    }
    if (lift) {
      if (!allow_dyn_smem((const void*)k_row_fwd_tc<true>, tsm)) return EM3D_ERR_CUDA;
      k_row_fwd_tc<true><<<tgrid, 128, tsm, st>>>(B, X, Y, Z, m, (const float2*)chi, (const float2*)wave, nullptr,
                                                    nullptr, (const BF*)Wt, bias, 0, (BF*)pre_out, (BF*)vout,
                                                    (float2*)Vz, (const BF*)Q, qb, (float2*)u_out);
    } else {
      if (!allow_dyn_smem((const void*)k_row_fwd_tc<false>, tsm)) return EM3D_ERR_CUDA;
      k_row_fwd_tc<false><<<tgrid, 128, tsm, st>>>(B, X, Y, Z, m, (const float2*)chi, (const float2*)wave,
                                                     (const BF*)vin, (const float2*)Uxy, (const BF*)Wt, bias,
                                                     apply_gelu, (BF*)pre_out, (BF*)vout, (float2*)Vz,
                                                     (const BF*)Q, qb, (float2*)u_out);
    }
    EM3D_LAUNCH_CHECK();
    return EM3D_OK;
  }
  int rc = EM3D_OK;
  FNO_DISPATCH(act, (rc = launch_row_fwd<ACT>(lift != 0, grid, smem, st, B, W, X, Y, Z, m, chi, wave, vin, Uxy, Wt,
                                              bias, apply_gelu, pre_out, vout, Vz, Q, qb, u_out)));
  if (rc != EM3D_OK) return rc;
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_modemix(int act, int B, int W, int nm, const void* V, const void* Wre, const void* Wim, void* U,
                     void* stream) {
  if (int rc = check_width(W)) return rc;
  FNO_DISPATCH(act, (k_modemix<ACT><<<blocks_for((size_t)B * W * nm), 256, 0, (cudaStream_t)stream>>>(
                         B, W, nm, (const float2*)V, (const ACT*)Wre, (const ACT*)Wim, (float2*)U)));
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_modemix_bwd(int act, int B, int W, int nm, const void* V, const void* dU, const void* Wre,
                         const void* Wim, void* dV, float* dWre, float* dWim, void* stream) {
  if (int rc = check_width(W)) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  FNO_DISPATCH(act, (k_modemix_bwd_v<ACT><<<blocks_for((size_t)B * W * nm), 256, 0, st>>>(
                         B, W, nm, (const float2*)dU, (const ACT*)Wre, (const ACT*)Wim, (float2*)dV)));
  EM3D_LAUNCH_CHECK();
  k_modemix_bwd_w<<<blocks_for((size_t)W * W * nm), 256, 0, st>>>(B, W, nm, (const float2*)V, (const float2*)dU,
                                                                   dWre, dWim);
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_layer_out(int act, int B, int W, int X, int Y, int Z, int m, const void* vin, const void* Uxy,
                       const void* A, const float* a, int apply_gelu, void* pre, void* vout, void* stream) {
  if (int rc = check_width(W)) return rc;
  if (Z > 1024 || m > 16 || m < 1) { em3d_set_last_error("FNO needs Z <= 1024 and 1 <= modes <= 16"); return EM3D_ERR_INVALID; }
  const size_t smem = (size_t)(W * W + W) * sizeof(float) + (size_t)W * m * sizeof(float2);
  const int threads = ((Z + 31) / 32) * 32;
  FNO_DISPATCH(act, (k_layer_out<ACT><<<B * X * Y, threads, smem, (cudaStream_t)stream>>>(
                         W, X, Y, Z, m, (const ACT*)vin, (const float2*)Uxy, (const ACT*)A, a, apply_gelu,
                         (ACT*)pre, (ACT*)vout)));
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_layer_out_bwd(int act, int B, int W, int X, int Y, int Z, int m, const float* gout, const void* pre,
                           const void* A, int apply_gelu, float* gpre, float* gin, void* dUxy, void* stream) {
  if (int rc = check_width(W)) return rc;
  if (Z > 1024 || m > 16 || m < 1) { em3d_set_last_error("FNO needs Z <= 1024 and 1 <= modes <= 16"); return EM3D_ERR_INVALID; }
  const size_t smem = (size_t)(W * W + W * Z) * sizeof(float) + (size_t)m * Z * sizeof(float2);
  if (smem > 200 * 1024) { em3d_set_last_error("FNO row too long for shared memory"); return EM3D_ERR_INVALID; }
  const int threads = ((Z + 31) / 32) * 32;
  if (act == FNO_BF16) {
    auto kern = k_layer_out_bwd<__nv_bfloat16>;
    EM3D_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    kern<<<B * X * Y, threads, smem, (cudaStream_t)stream>>>(W, X, Y, Z, m, gout, (const __nv_bfloat16*)pre,
                                                              (const __nv_bfloat16*)A, apply_gelu, gpre, gin,
                                                              (float2*)dUxy);
  } else if (act == FNO_F32) {
    auto kern = k_layer_out_bwd<float>;
    EM3D_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    kern<<<B * X * Y, threads, smem, (cudaStream_t)stream>>>(W, X, Y, Z, m, gout, (const float*)pre, (const float*)A,
                                                              apply_gelu, gpre, gin, (float2*)dUxy);
  } else {
    em3d_set_last_error("act dtype must be 0 (bf16) or 1 (float)");
    return EM3D_ERR_INVALID;
  }
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_pointwise_wgrad(int act, int B, size_t ncell, int W, const float* gpre, const void* v, float* dA,
                             float* da, void* stream) {
  if (int rc = check_width(W)) return rc;
  const size_t total = (size_t)B * ncell;
  const size_t chunk = 4096;
  const int grid = (int)((total + chunk - 1) / chunk);
  const int threads = ((W * W + 31) / 32) * 32;
  FNO_DISPATCH(act, (k_pointwise_wgrad<ACT><<<grid, threads, 0, (cudaStream_t)stream>>>(B, ncell, W, gpre,
                                                                                         (const ACT*)v, dA, da,
                                                                                         chunk)));
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_project(int act, int B, size_t ncell, int W, const void* v, const void* Q, const float* qb,
                     const void* wave, void* u, void* stream) {
  if (int rc = check_width(W)) return rc;
  FNO_DISPATCH(act, (k_project<ACT><<<blocks_for((size_t)B * ncell), 256, 0, (cudaStream_t)stream>>>(
                         B, ncell, W, (const ACT*)v, (const ACT*)Q, qb, (const float2*)wave, (float2*)u)));
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_project_bwd(int act, int B, size_t ncell, int W, const void* v, const void* Q, const void* du,
                         float* gv, float* dQ, float* dqb, void* stream) {
  if (int rc = check_width(W)) return rc;
  FNO_DISPATCH(act, (k_project_bwd<ACT><<<blocks_for((size_t)B * ncell) / 8 + 1, 256, 0, (cudaStream_t)stream>>>(
                         B, ncell, W, (const ACT*)v, (const ACT*)Q, (const float2*)du, gv, dQ, dqb)));
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_loss(int B, size_t n, const void* pred, const void* target, double* terms, void* grad, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  EM3D_CUDA_TRY(cudaMemsetAsync(terms, 0, sizeof(double) * 2 * B, st));
  const dim3 grid(blocks_for(n) < 296 ? blocks_for(n) : 296, B);
  k_loss_terms<<<grid, 256, 0, st>>>(B, n, (const float2*)pred, (const float2*)target, terms);
  EM3D_LAUNCH_CHECK();
  if (grad) {
    const dim3 g2(blocks_for(n), B);
    k_loss_grad<<<g2, 256, 0, st>>>(B, n, (const float2*)pred, (const float2*)target, terms, (float2*)grad);
    EM3D_LAUNCH_CHECK();
  }
  return EM3D_OK;
}

int em3d_fno_adam(int act, size_t n, float* w, const float* g, float* m1, float* m2, float lr, float b1, float b2,
                  float eps, int step, void* wact, void* stream) {
  if (step < 1) { em3d_set_last_error("adam step counts from 1"); return EM3D_ERR_INVALID; }
  const float bc1 = 1.0f - powf(b1, (float)step), bc2 = 1.0f - powf(b2, (float)step);
  FNO_DISPATCH(act, (k_adam<ACT><<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(n, w, g, m1, m2, lr, b1, b2, eps,
                                                                                  bc1, bc2, (ACT*)wact)));
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_cast(int act, size_t n, const float* src, void* dst, void* stream) {
  FNO_DISPATCH(act, (k_cast<ACT><<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(n, src, (ACT*)dst)));
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_uncast(int act, size_t n, const void* src, float* dst, void* stream) {
  FNO_DISPATCH(act, (k_uncast<ACT><<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(n, (const ACT*)src, dst)));
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_downsample2(int in_dtype, int C, int nx, int ny, int nz, const void* in, void* out, void* stream) {
  if (C < 1 || nx < 1 || ny < 1 || nz < 1 || !in || !out) { em3d_set_last_error("downsample2: bad arguments"); return EM3D_ERR_INVALID; }
  const size_t n = (size_t)C * nx * ny * nz;
  cudaStream_t st = (cudaStream_t)stream;
  if (in_dtype == EM3D_C64) k_down2<float2><<<blocks_for(n), 256, 0, st>>>(C, nx, ny, nz, (const float2*)in, (float2*)out);
  else if (in_dtype == EM3D_C128) k_down2<double2><<<blocks_for(n), 256, 0, st>>>(C, nx, ny, nz, (const double2*)in, (float2*)out);
  else { em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128"); return EM3D_ERR_INVALID; }
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

int em3d_fno_upsample2(int out_dtype, int C, int nx, int ny, int nz, const void* in, void* out, void* stream) {
  if (C < 1 || nx < 1 || ny < 1 || nz < 1 || !in || !out) { em3d_set_last_error("upsample2: bad arguments"); return EM3D_ERR_INVALID; }
  const size_t n = (size_t)C * 8 * nx * ny * nz;
  cudaStream_t st = (cudaStream_t)stream;
  if (out_dtype == EM3D_C64) k_up2<float2><<<blocks_for(n), 256, 0, st>>>(C, nx, ny, nz, (const float2*)in, (float2*)out);
  else if (out_dtype == EM3D_C128) k_up2<double2><<<blocks_for(n), 256, 0, st>>>(C, nx, ny, nz, (const float2*)in, (double2*)out);
  else { em3d_set_last_error("dtype must be EM3D_C64 or EM3D_C128"); return EM3D_ERR_INVALID; }
  EM3D_LAUNCH_CHECK();
  return EM3D_OK;
}

}  // extern "C"

