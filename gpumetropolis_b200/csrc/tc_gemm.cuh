// tc_gemm.cuh -- BF16 tensor-core GEMM on sm_100a with tcgen05 (5th-generation
// tensor cores, accumulators in tensor memory), for the surrogate MLP.
//
//   C[M x N] (f32) = A[M x K] (bf16, row-major) . B[N x K]^T (bf16, row-major)
//
// One CTA (256 threads) owns a 128 x BN output tile (BN in {64, 128, 256,
// 512}; 512 is two N = 256 MMAs side by side in tensor memory).  Per 64-wide
// K step the CTA copies its A and B slices into shared memory in the
// canonical K-major, no-swizzle core-matrix layout (8 rows x 16 bytes per
// core matrix), one elected thread issues the tcgen05.mma (M=128, N<=256,
// K=16) into TMEM accumulators and commits them to an mbarrier, and the CTA
// waits (bounded) before reusing shared memory; the next slice's global loads
// are in flight meanwhile.  The epilogue reads TMEM with tcgen05.ld: warp w
// owns lanes 32 (w % 4) .. 32 (w % 4) + 31 (rows) and column half w / 4, and
// applies one of the fused epilogues of the surrogate's training step
// (GemmEpi).  M, N and K must be multiples of
// 128, BN and 64 (callers pad with zeros).
// Split K (EPI_STORE only): with gridDim.z = S > 1, CTA z reduces K columns
// [z*kz, z*kz + kz) into its own partial C + z*M*N; the consumer adds the S
// partials in order, which keeps the result deterministic.
#pragma once
#include <cuda_bf16.h>

#include "device.cuh"

namespace gpum {

constexpr int kGemmBM = 128;
constexpr int kGemmBK = 64;
constexpr int kGemmThreads = 256;

enum DevErrGemm : uint32_t { DEV_ERR_MMA_TIMEOUT = 1u << 1 };

// Instruction descriptor, kind::f16: D f32, A and B bf16, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// The network's activations on the hardware 2^x and reciprocal: sigmoid(z)
// = 1 / (1 + 2^(-z log2 e)) (0 and 1 at the extremes, no division), silu(z) =
// z sigmoid(z), silu'(z) = s (1 + z (1 - s)).  Their few-ulp error is far
// below the BF16 rounding of every tensor-core operand.
__device__ __forceinline__ float sigmoidf_(float z) {
  return gm_rcp_approx(1.0f + gm_ex2_approx(-1.44269504f * z));
}
__device__ __forceinline__ float silu(float z) { return z * sigmoidf_(z); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = sigmoidf_(z);
  return s * (1.0f + z * (1.0f - s));
}

// Byte offset of element (r, k) of an R x 64 bf16 slice in the canonical
// K-major no-swizzle layout: core matrix (k/8, r/8) at ((k/8)*(R/8) + r/8)*128.
__device__ __forceinline__ uint32_t kmajor_offset(int r, int k, int R) {
  return (uint32_t)((((k >> 3) * (R >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// Column sums of a warp's 32 rows x 16 columns (v = this lane's row) by
// recursive halving: 16 shuffles instead of 16 x 5.  On return, lane l holds
// the sum of column warp_colsum16_col(l) over the 32 lanes (lanes l and l ^ 1
// hold the same column).  The addition order is fixed, so it is deterministic.
__device__ __forceinline__ int warp_colsum16_col(int lane) {
  return ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
}
__device__ __forceinline__ float warp_colsum16(const float (&v)[16], int lane) {
  float a[8], b[4], c[2];
  const bool h4 = lane & 16, h3 = lane & 8, h2 = lane & 4, h1 = lane & 2;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float mine = h4 ? v[j + 8] : v[j];
    const float give = h4 ? v[j] : v[j + 8];
    a[j] = mine + __shfl_xor_sync(0xffffffffu, give, 16);
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float mine = h3 ? a[j + 4] : a[j];
    const float give = h3 ? a[j] : a[j + 4];
    b[j] = mine + __shfl_xor_sync(0xffffffffu, give, 8);
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const float mine = h2 ? b[j + 2] : b[j];
    const float give = h2 ? b[j] : b[j + 2];
    c[j] = mine + __shfl_xor_sync(0xffffffffu, give, 4);
  }
  const float mine = h1 ? c[1] : c[0];
  const float give = h1 ? c[0] : c[1];
  const float d = mine + __shfl_xor_sync(0xffffffffu, give, 2);
  return d + __shfl_xor_sync(0xffffffffu, d, 1);
}

__device__ __forceinline__ float warp_sum(float x) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
  return x;
}

// Fused epilogues of the surrogate's training step (one thread = one row and
// one half of the tile's columns):
//   EPI_STORE  C = acc (+ bias), f32; with gridDim.z > 1 a split-K partial
//   EPI_SILU   Z = acc + bias -> C (f32); A = silu(Z) -> act (bf16, row-major)
//              and actT (bf16, transposed [N][M])
//   EPI_HEAD   needs the whole row (n0 = 0, BN = N = H): Z2 = acc + bias;
//              y = silu(Z2) . w3 + b3; r = y - t (rows < n_live), dy = 2 r /
//              n_live; dZ2 = dy w3 silu'(Z2) -> dzh (bf16 row-major) and actT
//              (bf16 transposed); per CTA the column sums of dy silu(Z2) (w3's
//              gradient) and dZ2 (b2's) -> colpart[2][gridDim.y][N], and the
//              sums of dy and r^2 -> rowpart[2][gridDim.y]; yhat (optional);
//              with unit_dy, dy = 1 (the gradient of y itself, for the
//              surrogate's input gradient)
//   EPI_DSILU  dZ1 = acc * silu'(Zprev) -> actT (bf16 transposed, optional)
//              and act (bf16 row-major, optional); per CTA the column sums
//              of dZ1 (b1's gradient) -> colpart[gridDim.y][N] (optional)
enum GemmEpi : int { EPI_STORE = 0, EPI_SILU = 1, EPI_HEAD = 2, EPI_DSILU = 3 };

struct GemmArgs {
  const __nv_bfloat16* A;
  const __nv_bfloat16* B;
  int M, N, K, kz;
  float* C;
  const float* bias;
  __nv_bfloat16* act;
  __nv_bfloat16* actT;
  const float* w3;
  const float* b3;
  const float* t;
  int n_live;
  __nv_bfloat16* dzh;
  float* colpart;
  float* rowpart;
  float* yhat;
  const float* Zprev;
  int unit_dy;
  uint32_t* err;
};

template <int BN>
constexpr size_t tc_gemm_smem() {
  // A slice | B slice | column-sum scratch [2][4 lane quarters][BN] | row
  // partials [2 halves][128] | bias, w3 [2][BN] | barrier, slot
  return (size_t)kGemmBM * kGemmBK * 2 + (size_t)BN * kGemmBK * 2 + (size_t)2 * 4 * BN * 4 +
         2 * 128 * 4 + (size_t)2 * BN * 4 + 16 + 16 + 1024;
}

// Stores 16 bf16 values of one row (32 bytes).
__device__ __forceinline__ void store_bf16x16(__nv_bfloat16* dst, const float (&v)[16]) {
  uint4 packed[2];
  uint32_t* w32 = reinterpret_cast<uint32_t*>(packed);
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const __nv_bfloat162 h2 = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
    w32[q] = *reinterpret_cast<const uint32_t*>(&h2);
  }
  uint4* a4 = reinterpret_cast<uint4*>(dst);
  a4[0] = packed[0];
  a4[1] = packed[1];
}

template <int BN, int EPI>
__global__ void __launch_bounds__(kGemmThreads, 1) tc_gemm_kernel(const GemmArgs g) {
  static_assert(BN == 64 || BN == 128 || BN == 256 || BN == 512, "BN");
  constexpr int kMmaN = BN < 256 ? BN : 256;          // N of one MMA
  constexpr int kNMma = BN / kMmaN;                   // MMAs side by side
  constexpr uint32_t kTmemCols = BN <= 32 ? 32 : (uint32_t)BN;
  extern __shared__ __align__(1024) unsigned char gsm[];
  unsigned char* sa = gsm;                                  // 128 x 64 bf16 = 16 KB
  unsigned char* sb = gsm + kGemmBM * kGemmBK * 2;          // BN x 64 bf16
  float* red = reinterpret_cast<float*>(sb + BN * kGemmBK * 2);  // [2][4][BN]
  float* ypart = red + 2 * 4 * BN;                                // [2][128]
  float* s_bias = ypart + 2 * 128;                                 // [BN]
  float* s_w3 = s_bias + BN;                                       // [BN]
  uint64_t* bar = reinterpret_cast<uint64_t*>(s_w3 + BN);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int M = g.M, N = g.N, K = g.K;
  const int m0 = blockIdx.y * kGemmBM, n0 = blockIdx.x * BN;
  const int kbeg = (int)blockIdx.z * g.kz, kend = min(kbeg + g.kz, K);
  const __nv_bfloat16* __restrict__ A = g.A;
  const __nv_bfloat16* __restrict__ B = g.B;

  if (warp == 0) tmem_alloc(tslot, kTmemCols);
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  // the epilogue's per-column operands, read by every row: staged once
  for (int i = tid; i < BN; i += kGemmThreads) {
    s_bias[i] = g.bias ? g.bias[n0 + i] : 0.0f;
    s_w3[i] = g.w3 ? g.w3[n0 + i] : 0.0f;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = umma_idesc_bf16(kGemmBM, kMmaN);
  const uint32_t sa_addr = smem_addr(sa), sb_addr = smem_addr(sb);
  const uint32_t lbo_a = (kGemmBM / 8) * 128, lbo_b = (BN / 8) * 128;
  bool ok = true;
  uint32_t fail_parity = 0;  // phase of the commit a wait gave up on

  // Staging: each thread owns kLA + kLB 16-byte chunks of a K slice.  All
  // global loads of a slice are issued back to back into registers, and the
  // next slice is loaded while the tensor core works on the current one.
  constexpr int kChunks = kGemmBK / 8;  // 16-byte chunks per row of a slice
  constexpr int kLA = kGemmBM * kChunks / kGemmThreads;
  constexpr int kLB = BN * kChunks / kGemmThreads;
  static_assert(kGemmBM * kChunks % kGemmThreads == 0 && BN * kChunks % kGemmThreads == 0, "");
  uint4 ra[kLA], rb[kLB];
  auto load_slice = [&](int k0) {
#pragma unroll
    for (int q = 0; q < kLA; ++q) {
      const int i = tid + q * kGemmThreads, r = i / kChunks, c8 = (i % kChunks) * 8;
      ra[q] = *reinterpret_cast<const uint4*>(A + (size_t)(m0 + r) * K + k0 + c8);
    }
#pragma unroll
    for (int q = 0; q < kLB; ++q) {
      const int i = tid + q * kGemmThreads, r = i / kChunks, c8 = (i % kChunks) * 8;
      rb[q] = *reinterpret_cast<const uint4*>(B + (size_t)(n0 + r) * K + k0 + c8);
    }
  };
  auto store_slice = [&]() {
#pragma unroll
    for (int q = 0; q < kLA; ++q) {
      const int i = tid + q * kGemmThreads, r = i / kChunks, c8 = (i % kChunks) * 8;
      *reinterpret_cast<uint4*>(sa + kmajor_offset(r, c8, kGemmBM)) = ra[q];
    }
#pragma unroll
    for (int q = 0; q < kLB; ++q) {
      const int i = tid + q * kGemmThreads, r = i / kChunks, c8 = (i % kChunks) * 8;
      *reinterpret_cast<uint4*>(sb + kmajor_offset(r, c8, BN)) = rb[q];
    }
  };
  if (kbeg < kend) load_slice(kbeg);

  for (int k0 = kbeg, it = 0; k0 < kend; k0 += kGemmBK, ++it) {
    store_slice();
    // Generic-proxy smem writes must be visible to the tensor core's async proxy.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int kk = 0; kk < kGemmBK / 16; ++kk) {
        const uint64_t ad = umma_smem_desc(sa_addr + 2 * kk * lbo_a, lbo_a, 128);
#pragma unroll
        for (int h = 0; h < kNMma; ++h) {
          // rows [h * 256, h * 256 + 256) of the B slice: 32 row groups further
          const uint64_t bd =
              umma_smem_desc(sb_addr + 2 * kk * lbo_b + h * (kMmaN / 8) * 128, lbo_b, 128);
          umma_bf16(tmem + (uint32_t)(h * kMmaN), ad, bd, idesc,
                    (k0 > kbeg || kk > 0) ? 1u : 0u);
        }
      }
      umma_commit(bar);
    }
    if (k0 + kGemmBK < kend) load_slice(k0 + kGemmBK);  // overlaps the MMAs
    __syncwarp();
    fail_parity = (uint32_t)(it & 1);
    if (!mbar_wait_bounded(bar, fail_parity)) {
      ok = false;
      if (lane == 0) atomicOr(g.err, DEV_ERR_MMA_TIMEOUT);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // block-uniform: a wait that gave up in any thread ends the K loop and
    // skips the epilogue in every thread
    ok = __syncthreads_and(ok) != 0;
    if (!ok) break;
  }

  // Epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (rows) and the
  // columns [cb, ce) of its half of the tile, 16 at a time.
  const int quarter = warp & 3, half = warp >> 2;
  const int row = m0 + quarter * 32 + lane;
  const uint32_t trow = tmem + ((uint32_t)(quarter * 32) << 16);
  constexpr int kHalf = BN / 2;
  const int cb = half * kHalf, ce = cb + kHalf;
  if (ok) {
    if constexpr (EPI == EPI_STORE || EPI == EPI_SILU) {
      float* C = g.C + (size_t)blockIdx.z * M * N;
#pragma unroll 1
      for (int c = cb; c < ce; c += 16) {
        float v[16];
        tmem_ld16(trow + (uint32_t)c, v);
        if (g.bias) {
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] += s_bias[c + j];
        }
        float4* c4 = reinterpret_cast<float4*>(C + (size_t)row * N + n0 + c);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          c4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        if constexpr (EPI == EPI_SILU) {
          float a[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) a[j] = silu(v[j]);
          if (g.act) store_bf16x16(g.act + (size_t)row * N + n0 + c, a);
          if (g.actT) {
#pragma unroll
            for (int j = 0; j < 16; ++j)
              g.actT[(size_t)(n0 + c + j) * M + row] = __float2bfloat16(a[j]);
          }
        }
      }
    } else if constexpr (EPI == EPI_HEAD) {
      // pass 1: the prediction of this row, its two column halves added in order
      float yp = 0.0f;
#pragma unroll 1
      for (int c = cb; c < ce; c += 16) {
        float v[16];
        tmem_ld16(trow + (uint32_t)c, v);
#pragma unroll
        for (int j = 0; j < 16; ++j) yp = fmaf(silu(v[j] + s_bias[c + j]), s_w3[c + j], yp);
      }
      ypart[half * 128 + quarter * 32 + lane] = yp;
      __syncthreads();
      const float y = (ypart[quarter * 32 + lane] + ypart[128 + quarter * 32 + lane]) + g.b3[0];
      if (g.yhat && half == 0) g.yhat[row] = y;
      const bool live = row < g.n_live;
      const float r = (live && g.t) ? y - g.t[row] : 0.0f;
      const float dy = g.unit_dy ? 1.0f : 2.0f * r / (float)g.n_live;
      // pass 2: dZ2, its two layouts and the column sums
#pragma unroll 1
      for (int c = cb; c < ce; c += 16) {
        float v[16], dz[16], wa[16];
        tmem_ld16(trow + (uint32_t)c, v);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float z = v[j] + s_bias[c + j];
          const float s = sigmoidf_(z);
          wa[j] = dy * (z * s);
          dz[j] = dy * s_w3[c + j] * (s * (1.0f + z * (1.0f - s)));
        }
        store_bf16x16(g.dzh + (size_t)row * N + c, dz);
        if (g.actT) {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            g.actT[(size_t)(c + j) * M + row] = __float2bfloat16(dz[j]);
        }
        if (g.colpart) {
          const float sw = warp_colsum16(wa, lane);
          const float sb2 = warp_colsum16(dz, lane);
          if ((lane & 1) == 0) {
            red[(0 * 4 + quarter) * BN + c + warp_colsum16_col(lane)] = sw;
            red[(1 * 4 + quarter) * BN + c + warp_colsum16_col(lane)] = sb2;
          }
        }
      }
      const float sdy = warp_sum(dy), sr2 = warp_sum(r * r);
      __syncthreads();
      if (g.colpart) {
        for (int i = tid; i < 2 * BN; i += kGemmThreads) {
          const int q = i / BN, n = i % BN;
          const float* rq = red + (size_t)q * 4 * BN;
          g.colpart[((size_t)q * gridDim.y + blockIdx.y) * N + n] =
              ((rq[n] + rq[BN + n]) + rq[2 * BN + n]) + rq[3 * BN + n];
        }
      }
      if (g.rowpart) {
        if (half == 0 && lane == 0) {
          ypart[quarter] = sdy;
          ypart[4 + quarter] = sr2;
        }
        __syncthreads();
        if (tid == 0) {
          g.rowpart[blockIdx.y] = ((ypart[0] + ypart[1]) + ypart[2]) + ypart[3];
          g.rowpart[gridDim.y + blockIdx.y] = ((ypart[4] + ypart[5]) + ypart[6]) + ypart[7];
        }
      }
    } else {  // EPI_DSILU
#pragma unroll 1
      for (int c = cb; c < ce; c += 16) {
        float v[16];
        tmem_ld16(trow + (uint32_t)c, v);
        const float4* z4 = reinterpret_cast<const float4*>(g.Zprev + (size_t)row * N + n0 + c);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 z = z4[q];
          v[4 * q] *= dsilu(z.x);
          v[4 * q + 1] *= dsilu(z.y);
          v[4 * q + 2] *= dsilu(z.z);
          v[4 * q + 3] *= dsilu(z.w);
        }
        if (g.actT) {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            g.actT[(size_t)(n0 + c + j) * M + row] = __float2bfloat16(v[j]);
        }
        if (g.act) store_bf16x16(g.act + (size_t)row * N + n0 + c, v);
        if (g.colpart) {
          const float s = warp_colsum16(v, lane);
          if ((lane & 1) == 0) red[quarter * BN + c + warp_colsum16_col(lane)] = s;
        }
      }
      if (g.colpart) {
        __syncthreads();
        for (int n = tid; n < BN; n += kGemmThreads)
          g.colpart[(size_t)blockIdx.y * N + n0 + n] =
              ((red[n] + red[BN + n]) + red[2 * BN + n]) + red[3 * BN + n];
      }
    }
  }
  // After a wait that gave up, give the MMAs in flight one more bounded wait
  // before the tensor memory is released.
  if (!ok && tid == 0) mbar_wait_bounded(bar, fail_parity);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

// out[i] = sum_z part[z*n + i], z in order.
static __global__ void tc_splitk_sum(const float* __restrict__ part, int S, size_t n,
                                     float* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float t = 0.0f;
  for (int z = 0; z < S; ++z) t += part[(size_t)z * n + i];
  out[i] = t;
}

}  // namespace gpum
