// FNO layer row pass on the fifth-generation tensor cores (tcgen05, TMEM
// accumulators).  Included by fno.cu inside namespace em3d::fno.
//
// Per tile of 128 cells (R = 128 / Z whole z-rows; Z in {32, 64, 128},
// width 32):
//   GEMM 1 (M = 128 cells, N = 32 channels, into TMEM columns 0..31)
//     O[cell][co] = sum_ci v[ci][cell] A[co][ci]                     (K = 32)
//                 + sum_(r, j) Tbd[cell][r, j] Ucat_r[co][j]          (K = 32 R)
//   where Tbd is block diagonal over the tile's rows, holding the weighted
//   inverse z-DFT table (cos / -sin, j < 2m) of each row, and Ucat_r the
//   row's mode coefficients (Re / Im); then, per cell, bias, GELU, bf16.
//   GEMM 2 (M = 128 = 32 R' rows of (row, j), N = 32 channels, K = 128
//   cells, into TMEM columns 32..63): the next layer's truncated z-DFT
//     Vz[r, j][co] = sum_cell Fbd[r, j][cell] O[cell][co]
//   with Fbd block diagonal (cos / -sin of the row's cells).
// The same products as the mma.sync kernel (k_row_fwd_tc): bf16 operands,
// FP32 accumulation, O rounded to bf16 before GEMM 2.
//
// Operands live in shared memory in the no-swizzle K-major layout of the
// tensor cores: 8-row x 16-byte core matrices of 128 contiguous bytes, the
// core matrices of one 8-row group side by side along K (leading byte
// offset 128), the groups one after another (stride byte offset K / 8 x 128).
// One thread issues the MMAs and commits them to an mbarrier; every wait on
// it is bounded (a give-up is counted in `fails`, the CTA waits once more for
// the MMAs in flight, frees its tensor memory and leaves).

constexpr int kUmmaCells = 128;

__device__ __forceinline__ uint32_t umma_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: start, leading and stride byte offsets
// (16-byte units), descriptor version 1 (bits 46-47), no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// instruction descriptor of kind::f16: D FP32 (bits 4-5 = 1), A and B bf16
// (bits 7-9 and 10-12 = 1), both K-major, N / 8 at bits 17-22, M / 16 at 24-28
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// 32 consecutive TMEM columns of this thread's lane (warp w reads lanes 32w..32w+31)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared memory of k_row_fwd_umma (bytes, regions 1024-aligned).
struct UmmaSmem {
  static constexpr uint32_t W = 0;                       // 32 x 32 bf16
  static constexpr uint32_t T = W + 2048;                 // 128 x 128 bf16 (K = 32 R used)
  static constexpr uint32_t F = T + 32768;                // 128 x 128 bf16
  static constexpr uint32_t V = F + 32768;                // 128 x 32 bf16
  static constexpr uint32_t U = V + 8192;                 // 32 x 128 bf16 (K = 32 R used)
  static constexpr uint32_t O = U + 8192;                 // 32 x 128 bf16
  static constexpr uint32_t MISC = O + 8192;              // bias, Q, qb, mbarrier, tmem slot
  static constexpr uint32_t TOTAL = MISC + 1024;
};

__global__ void __launch_bounds__(128, 1)
k_row_fwd_umma(int B, int X, int Y, int Z, int m, const __nv_bfloat16* __restrict__ vin,
               const float2* __restrict__ Uxy, const __nv_bfloat16* __restrict__ Wt, const float* __restrict__ bias,
               int apply_gelu, __nv_bfloat16* __restrict__ pre_out, __nv_bfloat16* __restrict__ vout,
               float2* __restrict__ Vz, const __nv_bfloat16* __restrict__ Q, const float* __restrict__ qb,
               const float2* __restrict__ wave, float2* __restrict__ u_out, unsigned int* __restrict__ fails) {
  constexpr int W = 32;
  using S = UmmaSmem;
  extern __shared__ __align__(1024) unsigned char smem_umma[];
  unsigned char* sm = smem_umma;
  float* sb = reinterpret_cast<float*>(sm + S::MISC);       // 32
  float* sQ = sb + 32;                                       // 6 x 32
  float* sqb = sQ + 6 * 32;                                  // 8
  uint64_t* bar = reinterpret_cast<uint64_t*>(sqb + 8);      // 8-byte aligned
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int R = kUmmaCells / Z, K1 = 32 * R;
  const size_t XY = (size_t)X * Y, ncell = XY * Z, nrows = (size_t)B * XY;
  const uint32_t base = smem_u32(sm);

  // constants: bias, projection, A (as B operand), the block-diagonal tables
  for (int i = tid; i < 32; i += blockDim.x) sb[i] = bias[i];
  for (int i = tid; i < 6 * 32; i += blockDim.x) sQ[i] = Q ? __bfloat162float(Q[i]) : 0.0f;
  if (tid < 8) sqb[tid] = (qb && tid < 6) ? qb[tid] : 0.0f;
  for (int i = tid; i < W * W; i += blockDim.x) {
    const int co = i / W, ci = i - co * W;
    *reinterpret_cast<__nv_bfloat16*>(sm + S::W + umma_off(co, ci, W)) = Wt[co * W + ci];
  }
  // the block-diagonal tables: zero both, then the twiddles cos / sin of
  // 2 pi k z / Z (k < m) once into the tile buffers, then the nonzero blocks
  {
    uint4* zt = reinterpret_cast<uint4*>(sm + S::T);
    for (int i = tid; i < (int)((S::V - S::T) / 16); i += blockDim.x) zt[i] = make_uint4(0, 0, 0, 0);
    float2* tw = reinterpret_cast<float2*>(sm + S::V);  // Z x m <= 2048 entries in V and U (16 KB)
    for (int i = tid; i < Z * m; i += blockDim.x) {
      const int z = i / m, k = i - z * m;
      float sn, cs;
      sincospif(2.0f * (float)((k * z) % Z) / (float)Z, &sn, &cs);
      tw[i] = make_float2(cs, sn);
    }
    __syncthreads();
    const float inv = 1.0f / (float)ncell;
    const int J = 2 * m;
    for (int i = tid; i < kUmmaCells * J; i += blockDim.x) {
      const int cell = i / J, j = i - cell * J;
      const int r = cell / Z, z = cell - r * Z, k = j >> 1;
      const float2 t = tw[z * m + k];
      const float w = (k == 0 ? 1.0f : 2.0f) * inv;
      const float v = (j & 1) ? -t.y : t.x;
      *reinterpret_cast<__nv_bfloat16*>(sm + S::T + umma_off(cell, r * 32 + j, K1)) = __float2bfloat16(v * w);
      *reinterpret_cast<__nv_bfloat16*>(sm + S::F + umma_off(r * 32 + j, cell, kUmmaCells)) = __float2bfloat16(v);
    }
    __syncthreads();  // the twiddles' space is the tiles' from here on
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;\n" ::"r"(smem_u32(tslot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = umma_idesc_bf16(128, 32);
  uint32_t phase = 0;
  bool failed = false;

  const size_t ntiles = (nrows + R - 1) / R;
  for (size_t tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
    const size_t row0 = tile * R;
    // ---- stage the tile: v as the A operand (cell x ci), U as a B operand (co x (r, j))
    const int chunks = Z / 8;
    for (int i = tid; i < R * W * chunks; i += blockDim.x) {
      const int r = i / (W * chunks), rem = i - r * W * chunks, ci = rem / chunks, q = rem - ci * chunks;
      const size_t row = row0 + r;
      uint4 val = make_uint4(0, 0, 0, 0);
      if (row < nrows) {
        const size_t b = row_batch(row, XY), xy = row - b * XY;
        val = *reinterpret_cast<const uint4*>(vin + (b * W + ci) * ncell + xy * Z + q * 8);
      }
      const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(&val);
#pragma unroll
      for (int t = 0; t < 8; ++t)
        *reinterpret_cast<__nv_bfloat16*>(sm + S::V + umma_off(r * Z + q * 8 + t, ci, W)) = e[t];
    }
    for (int i = tid; i < W * R * 16; i += blockDim.x) {
      const int co = i / (R * 16), rem = i - co * R * 16, r = rem >> 4, k = rem & 15;
      const size_t row = row0 + r;
      float2 u = make_float2(0.0f, 0.0f);
      if (row < nrows && k < m) {
        const size_t b = row_batch(row, XY), xy = row - b * XY;
        u = Uxy[((b * W + co) * XY + xy) * m + k];
      }
      const int col = r * 32 + 2 * k;
      *reinterpret_cast<__nv_bfloat16*>(sm + S::U + umma_off(co, col, K1)) = __float2bfloat16(u.x);
      *reinterpret_cast<__nv_bfloat16*>(sm + S::U + umma_off(co, col + 1, K1)) = __float2bfloat16(u.y);
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // ---- GEMM 1
    if (tid == 0) {
#pragma unroll
      for (int s = 0; s < 2; ++s)
        umma_bf16(tmem, umma_desc(base + S::V + s * 256, 128, 512), umma_desc(base + S::W + s * 256, 128, 512),
                  idesc, s > 0);
      const uint32_t sbo = (uint32_t)(K1 / 8) * 128;
      for (int s = 0; s < K1 / 16; ++s)
        umma_bf16(tmem, umma_desc(base + S::T + s * 256, 128, sbo), umma_desc(base + S::U + s * 256, 128, sbo),
                  idesc, 1);
      umma_commit(bar);
    }
    if (!__syncthreads_and(mbar_wait_bounded(bar, phase))) {
      failed = true;
      break;
    }
    phase ^= 1u;
    tc_fence_after();
    // ---- epilogue: bias, GELU, bf16; O kept as GEMM 2's B operand (co x cell)
    {
      float d[32];
      tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16), d);
      const int cell = tid, r = cell / Z, z = cell - r * Z;
      const size_t row = row0 + r;
      const bool valid = row < nrows;
      const size_t b = valid ? row_batch(row, XY) : 0, xy = valid ? row - b * XY : 0;
      const size_t at = xy * Z + z;
      float p[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) p[j] = sqb[j];
#pragma unroll
      for (int co = 0; co < W; ++co) {
        float o = d[co] + sb[co];
        if (pre_out && valid) pre_out[(b * W + co) * ncell + at] = __float2bfloat16(o);
        if (apply_gelu) o = gelu(o);
        const __nv_bfloat16 q = __float2bfloat16(o);
        *reinterpret_cast<__nv_bfloat16*>(sm + S::O + umma_off(co, cell, kUmmaCells)) = q;
        if (vout && valid) vout[(b * W + co) * ncell + at] = q;
        if (u_out) {
          const float qf = __bfloat162float(q);
#pragma unroll
          for (int j = 0; j < 6; ++j) p[j] += sQ[j * 32 + co] * qf;
        }
      }
      if (u_out && valid) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const size_t idx = (b * 3 + c) * ncell + at;
          const float2 fw = wave[idx];
          u_out[idx] = make_float2(fw.x + p[2 * c], fw.y + p[2 * c + 1]);
        }
      }
    }
    // ---- GEMM 2: the next layer's z-DFT of the tile's rows
    if (Vz) {
      fence_proxy_async_smem();
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      if (tid == 0) {
#pragma unroll
        for (int s = 0; s < kUmmaCells / 16; ++s)
          umma_bf16(tmem + 32, umma_desc(base + S::F + s * 256, 128, 2048),
                    umma_desc(base + S::O + s * 256, 128, 2048), idesc, s > 0);
        umma_commit(bar);
      }
      if (!__syncthreads_and(mbar_wait_bounded(bar, phase))) {
        failed = true;
        break;
      }
      phase ^= 1u;
      tc_fence_after();
      if (warp < R) {
        float e[32];
        tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + 32u, e);
        const size_t row = row0 + warp;
        const bool ok = row < nrows && (lane & 1) == 0 && (lane >> 1) < m;
        const size_t b = row < nrows ? row_batch(row, XY) : 0, xy = row < nrows ? row - b * XY : 0;
#pragma unroll
        for (int co = 0; co < W; ++co) {
          const float im = __shfl_down_sync(0xffffffffu, e[co], 1);
          if (ok) Vz[((b * W + co) * XY + xy) * m + (lane >> 1)] = make_float2(e[co], im);
        }
      }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (failed) {
    // a commit never completed: count it once, give the MMAs in flight one
    // more bounded wait, then free the tensor memory and leave
    if (tid == 0 && fails) atomicAdd(fails, 1u);
    mbar_wait_bounded(bar, phase);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;\n" ::"r"(tmem) : "memory");
}
