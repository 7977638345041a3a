// tc_gemm.cuh -- BF16 tensor-core GEMM on sm_100a with tcgen05 (5th-generation
// tensor cores, accumulators in tensor memory), for the surrogate MLP.
//
//   C[M x N] (f32) = A[M x K] (bf16, row-major) . B[N x K]^T (bf16, row-major)
//   optional epilogue: Z = C + bias[n] (f32 out), and act = silu(Z) (bf16 out)
//
// One CTA (128 threads) owns a 128 x BN output tile.  Per 64-wide K step the
// CTA copies its A and B slices into shared memory in the canonical K-major,
// no-swizzle core-matrix layout (8 rows x 16 bytes per core matrix), one
// elected thread issues four tcgen05.mma (M=128, N=BN, K=16) into a TMEM
// accumulator and commits them to an mbarrier, and the CTA waits (bounded)
// before reusing shared memory.  The epilogue reads TMEM with tcgen05.ld
// (warp w owns lanes 32w..32w+31 = rows), applies bias and SiLU, and stores.
// M, N and K must be multiples of 128, BN and 64 (callers pad with zeros).
// Split K: with gridDim.z = S > 1, CTA z reduces K columns [z*kz, z*kz + kz)
// into its own partial C + z*M*N (no epilogue); the caller adds the S
// partials in order (tc_splitk_sum), which keeps the result deterministic.
#pragma once
#include <cuda_bf16.h>

#include "device.cuh"

namespace gpum {

constexpr int kGemmBM = 128;
constexpr int kGemmBK = 64;
constexpr int kGemmThreads = 128;

enum DevErrGemm : uint32_t { DEV_ERR_MMA_TIMEOUT = 1u << 1 };

// Shared-memory matrix descriptor (tcgen05, sm_100): start address, leading
// byte offset (between the two 8-element K chunks of one MMA), stride byte
// offset (between 8-row groups), version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, lbo mode 0, layout type 0 (no swizzle)
}

// Instruction descriptor, kind::f16: D f32, A and B bf16, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t* smem_dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_addr(smem_dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
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

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::
                   "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }

// Byte offset of element (r, k) of an R x 64 bf16 slice in the canonical
// K-major no-swizzle layout: core matrix (k/8, r/8) at ((k/8)*(R/8) + r/8)*128.
__device__ __forceinline__ uint32_t kmajor_offset(int r, int k, int R) {
  return (uint32_t)((((k >> 3) * (R >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

template <int BN>
__global__ void __launch_bounds__(kGemmThreads, 1)
tc_gemm_kernel(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B,
               float* __restrict__ C, const float* __restrict__ bias,
               __nv_bfloat16* __restrict__ act, int M, int N, int K, int kz, uint32_t* err) {
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "BN");
  constexpr uint32_t kTmemCols = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
  extern __shared__ __align__(1024) unsigned char gsm[];
  unsigned char* sa = gsm;                                  // 128 x 64 bf16 = 16 KB
  unsigned char* sb = gsm + kGemmBM * kGemmBK * 2;          // BN x 64 bf16
  uint64_t* bar = reinterpret_cast<uint64_t*>(sb + BN * kGemmBK * 2);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * kGemmBM, n0 = blockIdx.x * BN;
  const int kbeg = (int)blockIdx.z * kz, kend = min(kbeg + kz, K);
  C += (size_t)blockIdx.z * M * N;

  if (warp == 0) tmem_alloc(tslot, kTmemCols);
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = umma_idesc_bf16(kGemmBM, BN);
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
        const uint64_t bd = umma_smem_desc(sb_addr + 2 * kk * lbo_b, lbo_b, 128);
        umma_bf16(tmem, ad, bd, idesc, (k0 > kbeg || kk > 0) ? 1u : 0u);
      }
      umma_commit(bar);
    }
    if (k0 + kGemmBK < kend) load_slice(k0 + kGemmBK);  // overlaps the MMAs
    __syncwarp();
    fail_parity = (uint32_t)(it & 1);
    if (!mbar_wait_bounded(bar, fail_parity)) {
      ok = false;
      if (lane == 0) atomicOr(err, DEV_ERR_MMA_TIMEOUT);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // block-uniform: a wait that gave up in any thread ends the K loop and
    // skips the epilogue in every thread
    ok = __syncthreads_and(ok) != 0;
    if (!ok) break;
  }

  // Epilogue: warp w reads TMEM lanes 32w..32w+31 (rows), 16 columns at a
  // time, and writes each row's 16 values with 16-byte stores.
  if (ok) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      if (bias) {
        const float4* b4 = reinterpret_cast<const float4*>(bias + n0 + c);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 b = b4[q];
          v[4 * q] += b.x;
          v[4 * q + 1] += b.y;
          v[4 * q + 2] += b.z;
          v[4 * q + 3] += b.w;
        }
      }
      float4* c4 = reinterpret_cast<float4*>(C + (size_t)row * N + n0 + c);
#pragma unroll
      for (int q = 0; q < 4; ++q) c4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      if (act) {
        uint4 packed[2];
        uint32_t* w32 = reinterpret_cast<uint32_t*>(packed);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const __nv_bfloat162 h2 = __floats2bfloat162_rn(silu(v[2 * q]), silu(v[2 * q + 1]));
          w32[q] = *reinterpret_cast<const uint32_t*>(&h2);
        }
        uint4* a4 = reinterpret_cast<uint4*>(act + (size_t)row * N + n0 + c);
        a4[0] = packed[0];
        a4[1] = packed[1];
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

template <int BN>
constexpr size_t tc_gemm_smem() {
  return (size_t)kGemmBM * kGemmBK * 2 + (size_t)BN * kGemmBK * 2 + 16 + 16 + 1024;
}

}  // namespace gpum
