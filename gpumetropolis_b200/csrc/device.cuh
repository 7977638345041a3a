// device.cuh -- sm_100a device helpers: TMA bulk-tensor loads with mbarrier
// completion (bounded waits), counter-based RNGs, compensated accumulation.
#pragma once
#ifdef __CUDACC_RTC__
// Compiled at run time by NVRTC: no host headers.
typedef unsigned int uint32_t;
typedef int int32_t;
typedef unsigned long long uint64_t;
typedef long long int64_t;
#else
#include <cuda_runtime.h>
#include <stdint.h>
#endif

namespace gpum {

// Opaque 128-byte TMA descriptor (same size and alignment as CUtensorMap);
// the host fills it with cuTensorMapEncodeTiled.
struct __align__(64) TmapDesc {
  uint64_t opaque[16];
};

// ---------------------------------------------------------------- errors
// Bits of the device error word a kernel sets instead of trapping; the host
// reads it after every run and turns it into a status code.
enum DevErr : uint32_t {
  DEV_ERR_TMA_TIMEOUT = 1u << 0,   // a tile never arrived within the wait limit
  // (1u << 1 is the tensor-core commit timeout of tc_gemm.cuh)
  DEV_ERR_WAIT_SELFTEST = 1u << 2, // the self-test's wait ran out, as it must
  DEV_ERR_TC_TIMEOUT = 1u << 3,    // a wait of the tensor-core value kernel ran out
};

// ------------------------------------------------------------- mbarrier/TMA
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Every wait is bounded: after the limit the caller records an error and
// carries on, so a lost transfer can never hang the GPU.
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Nanosecond clock of the GPU, for waits bounded in time as well as polls.
__device__ __forceinline__ uint64_t gm_globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// 16-byte shared-memory load that the compiler may not merge with an earlier
// load of the same address (a reload instead of keeping the value live).
__device__ __forceinline__ float4 gm_lds4v(const float* p) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(smem_addr(p)));
  return v;
}

// 2-D tiled TMA load (no multicast): box at (x, y) of `map` into smem `dst`,
// completion counted on `bar`.  x * elemsize must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_2d(void* dst, const TmapDesc* map, uint64_t* bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const TmapDesc* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Bulk copy without a tensor map (no multicast): `bytes` from global `src`
// to shared `dst`, completion counted on `bar`.  Both addresses 16-byte
// aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// ------------------------------------------ tcgen05 (5th-generation tensor cores)
// Shared-memory matrix descriptor: start address, leading byte offset
// (between the two K-adjacent core matrices of one MMA), stride byte offset
// (between 8-row groups), version 1, no swizzle.  A core matrix is 8 rows x
// 16 bytes (8 bf16 or 4 tf32 values of K per row).
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, lbo mode 0, layout type 0 (no swizzle)
}

// Instruction descriptor, kind::tf32: D f32, A and B tf32, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
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

// D (+)= A . B^T with tf32 operands, f32 accumulators in tensor memory.
__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive on `bar` once every tcgen05 operation this thread issued is done.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::
                   "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Generic-proxy shared-memory writes made visible to the async proxy (the
// tensor core reading an operand this thread wrote).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16 consecutive f32 columns of this thread's TMEM lane (32x32b shape: warp
// w % 4 reads lanes 32 (w % 4) .. + 31), waited for before returning.
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

// 32 consecutive f32 columns of this thread's TMEM lane, waited for.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld(uint32_t taddr, float (&v)[16]) { tmem_ld16(taddr, v); }
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float (&v)[32]) { tmem_ld32(taddr, v); }

// x rounded to the nearest tf32 value (ties away from zero), in an f32
// container: the tensor core reads tf32 operands from the top 19 bits.
__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// ------------------------------------------------------------------ RNGs
// triple32 integer hash (Wellons), the reference's stream
// (src/rust/src/cpu_native.rs:14-28, chain_kernel.rs:23-41).
__host__ __device__ __forceinline__ uint32_t triple32(uint32_t h) {
  h ^= h >> 17;
  h *= 2129725213u;
  h ^= h >> 11;
  h *= 2890025505u;
  h ^= h >> 15;
  h *= 831628273u;
  h ^= h >> 14;
  return h;
}

__device__ __forceinline__ double t32_uniform(uint32_t seedmix, uint32_t ctr) {
  return ((double)triple32(seedmix + ctr) + 0.5) / 4294967296.0;
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw; SC'11): counter-based, so a
// chain's stream is a pure function of (seed, chain, iteration, draw).
struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// 53-bit uniform in (0, 1] from two 32-bit words (the top value, 2^53 - 1/2
// over 2^53, rounds to 1).
__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
  const uint64_t m = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);
  return ((double)(m & ((1ull << 53) - 1)) + 0.5) * (1.0 / 9007199254740992.0);
}

// ------------------------------------------------------------- digamma
// Digamma by the reference's method (src/rust/src/cpu_native.rs:66-77):
// recurrence psi(x) = psi(x+1) - 1/x up past 6, then the asymptotic series
// ln x - 1/(2x) - 1/(12x^2) + 1/(120x^4) - 1/(252x^6).  It is the local
// derivative of the lgamma opcode in the adjoint.
__device__ __forceinline__ double gm_digamma(double x) {
  double r = 0.0;
  for (int i = 0; i < 64 && x < 6.0; ++i) {
    r -= 1.0 / x;
    x += 1.0;
  }
  const double f = 1.0 / (x * x);
  return r + log(x) - 1.0 / (2.0 * x) - f * (1.0 / 12.0 - f * (1.0 / 120.0 - f * (1.0 / 252.0)));
}

__device__ __forceinline__ float gm_digammaf(float x) {
  float r = 0.0f;
  for (int i = 0; i < 64 && x < 6.0f; ++i) {
    r -= 1.0f / x;
    x += 1.0f;
  }
  const float f = 1.0f / (x * x);
  return r + logf(x) - 1.0f / (2.0f * x) -
         f * (1.0f / 12.0f - f * (1.0f / 120.0f - f * (1.0f / 252.0f)));
}

// ------------------------------------------------- compensated accumulation
// Fast2Sum-compensated FP32 sum.  `s` follows plain summation exactly (so an
// infinite or NaN term propagates as in the reference's naive sum, which
// decides acceptance of non-finite proposals), and `c` collects the finite
// rounding errors; the total is s + c.
struct Comp {
  float s, c;
  __device__ __forceinline__ void init() { s = 0.f; c = 0.f; }
  __device__ __forceinline__ void add(float x) {
    const float t = s + x;
    const float e = x - (t - s);
    c += (fabsf(e) <= 3.402823466e38f) ? e : 0.f;
    s = t;
  }
  __device__ __forceinline__ double total() const {
    return isfinite(s) ? (double)s + (double)c : (double)s;
  }
};

// ------------------------------------------------------------- softplus
// softplus(a) = log(1 + e^a), which codegen substitutes for LOG(1 + EXP(a)):
//   softplus(a) = max(a, 0) + log1p(u),  u = e^(-|a|) in (0, 1],
//   u = 2^t e^r with t = fl(-|a| log2(e)) and the residual r = -|a| - t ln 2
//       (Cody & Waite reduction: ln 2 = LN2_HI + LN2_LO, two FMAs), 2^t from
//       the hardware ex2 and e^r = 1 + r (|r| < 6e-6, so r^2/2 < 2e-11);
//   log1p(u) = 2 atanh(s), s = u / (2 + u) in (0, 1/3]; with w = 2s =
//       u / (1 + u/2) and q = w^2 in [0, 4/9]:  w (1 + q P(q)), P the
//       degree-3 minimax fit (discrete Chebyshev approximation by linear
//       programming on 4001 points, weighted to the relative error of
//       log1p) of the atanh series sum_k q^(k-1) / ((2k+1) 4^k); its
//       relative error in log1p is below 5e-9.
// Unlike log(1 + exp(a)) in FP32 this keeps full relative accuracy where
// e^a underflows against 1.  NaN propagates (max.NaN); +inf -> +inf;
// -inf -> 0.
__device__ __forceinline__ float gm_ex2_approx(float t) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(t));
  return y;
}
__device__ __forceinline__ float gm_rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gm_max_nan(float a, float b) {
  float y;
  asm("max.NaN.f32 %0, %1, %2;" : "=f"(y) : "f"(a), "f"(b));
  return y;
}
__device__ __forceinline__ float gm_min_nan(float a, float b) {
  float y;
  asm("min.NaN.f32 %0, %1, %2;" : "=f"(y) : "f"(a), "f"(b));
  return y;
}

#define GM_SP_L2E 1.44269502162933349609375f        // log2(e) rounded to float
#define GM_SP_LN2_HI 0.693147182464599609375f       // ln(2) rounded to float
#define GM_SP_LN2_LO (-1.904654212125934e-09f)      // ln(2) - GM_SP_LN2_HI
#define GM_SP_P0 8.333302289e-02f
#define GM_SP_P1 1.250672713e-02f
#define GM_SP_P2 2.187641105e-03f
#define GM_SP_P3 5.471091135e-04f

// log1p(e^-|a|), the second addend of softplus(a).
__device__ __forceinline__ float gm_log1p_nexp(float a) {
  const float na = fmaxf(-fabsf(a), -126.0f);  // e^-126 underflows to 0 anyway
  const float t = na * GM_SP_L2E;
  const float r = fmaf(t, -GM_SP_LN2_LO, fmaf(t, -GM_SP_LN2_HI, na));
  const float u0 = gm_ex2_approx(t);
  const float u = fmaf(u0, r, u0);
  const float w = u * gm_rcp_approx(fmaf(u, 0.5f, 1.0f));
  const float q = w * w;
  float p = GM_SP_P3;
  p = fmaf(p, q, GM_SP_P2);
  p = fmaf(p, q, GM_SP_P1);
  p = fmaf(p, q, GM_SP_P0);
  return fmaf(w, q * p, w);
}

__device__ __forceinline__ float gm_softplus(float a) {
  return gm_max_nan(a, 0.0f) + gm_log1p_nexp(a);
}

// log(e^p + e^q) = max(p, q) + log1p(e^-|p - q|), which codegen substitutes
// for LOG(c1 EXP(a) + c2 EXP(b)) with positive parameter-only weights (p = a
// + log c1, q = b + log c2): no exponential of the terms themselves, so no
// FP32 underflow to log(0) where the reference's f64 sum is still finite.
// NaN propagates; both terms -inf gives -inf.
__device__ __forceinline__ float gm_logaddexp(float p, float q) {
  const float m = gm_max_nan(p, q);
  const float r = m + gm_log1p_nexp(p - q);
  return m < -3.402823466e38f ? m : r;  // m is -inf
}

// ------------------------------------------------- paired FP32 arithmetic
// Two observations per lane: sm_100's two-wide FP32 instructions (FADD2,
// FMUL2, FFMA2) round each half exactly like the scalar instruction.
// Subtraction and negation are FFMA2 / FMUL2 by -1, which are exact.
__device__ __forceinline__ float2 gm2(float c) { return make_float2(c, c); }
__device__ __forceinline__ float2 gm2_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 gm2_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 gm2_fma(float2 a, float2 b, float2 c) {
  return __ffma2_rn(a, b, c);
}
__device__ __forceinline__ float2 gm2_sub(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}
__device__ __forceinline__ float2 gm2_neg(float2 a) {
  return __fmul2_rn(a, make_float2(-1.0f, -1.0f));
}
__device__ __forceinline__ float2 gm2_div(float2 a, float2 b) {
  return make_float2(a.x / b.x, a.y / b.y);
}
__device__ __forceinline__ float2 gm2_exp(float2 a) { return make_float2(expf(a.x), expf(a.y)); }
__device__ __forceinline__ float2 gm2_log(float2 a) { return make_float2(logf(a.x), logf(a.y)); }
__device__ __forceinline__ float2 gm2_sqrt(float2 a) {
  return make_float2(sqrtf(a.x), sqrtf(a.y));
}
__device__ __forceinline__ float2 gm2_lgamma(float2 a) {
  return make_float2(lgammaf(a.x), lgammaf(a.y));
}
// Paired softplus (the scalar gm_softplus step for step): the reduction,
// the correction and the series on FFMA2/FMUL2/FADD2; the hardware 2^x,
// reciprocal and NaN-propagating max per half.  gm2_log1p_nexp is the
// second addend log1p(e^-|a|).
__device__ __forceinline__ float2 gm2_log1p_nexp(float2 a) {
  const float2 na = make_float2(fmaxf(-fabsf(a.x), -126.0f), fmaxf(-fabsf(a.y), -126.0f));
  const float2 t = __fmul2_rn(na, gm2(GM_SP_L2E));
  const float2 r =
      __ffma2_rn(t, gm2(-GM_SP_LN2_LO), __ffma2_rn(t, gm2(-GM_SP_LN2_HI), na));
  const float2 u0 = make_float2(gm_ex2_approx(t.x), gm_ex2_approx(t.y));
  const float2 u = __ffma2_rn(u0, r, u0);
  const float2 den = __ffma2_rn(u, gm2(0.5f), gm2(1.0f));
  const float2 w = __fmul2_rn(u, make_float2(gm_rcp_approx(den.x), gm_rcp_approx(den.y)));
  const float2 q = __fmul2_rn(w, w);
  float2 p = gm2(GM_SP_P3);
  p = __ffma2_rn(p, q, gm2(GM_SP_P2));
  p = __ffma2_rn(p, q, gm2(GM_SP_P1));
  p = __ffma2_rn(p, q, gm2(GM_SP_P0));
  return __ffma2_rn(w, __fmul2_rn(q, p), w);
}
__device__ __forceinline__ float2 gm2_softplus(float2 a) {
  const float2 m = make_float2(gm_max_nan(a.x, 0.0f), gm_max_nan(a.y, 0.0f));
  return __fadd2_rn(m, gm2_log1p_nexp(a));
}
// Paired gm_logaddexp.
__device__ __forceinline__ float2 gm2_logaddexp(float2 p, float2 q) {
  const float2 m = make_float2(gm_max_nan(p.x, q.x), gm_max_nan(p.y, q.y));
  const float2 r = __fadd2_rn(m, gm2_log1p_nexp(__ffma2_rn(q, gm2(-1.0f), p)));
  return make_float2(m.x < -3.402823466e38f ? m.x : r.x, m.y < -3.402823466e38f ? m.y : r.y);
}
// x * y - softplus(a) as FFMA2(x, y, min(-a, 0) - log1p(e^-|a|)), the NaN-
// propagating min giving -max(a, 0): one rounding fewer than the product and
// the difference apart, and no separate negation.
__device__ __forceinline__ float2 gm2_fma_nsoftplus(float2 x, float2 y, float2 a) {
  const float2 nm = make_float2(gm_min_nan(-a.x, 0.0f), gm_min_nan(-a.y, 0.0f));
  return __ffma2_rn(x, y, __ffma2_rn(gm2_log1p_nexp(a), gm2(-1.0f), nm));
}

__device__ __forceinline__ float2 gm2_digamma(float2 a) {
  return make_float2(gm_digammaf(a.x), gm_digammaf(a.y));
}
// Adjoint of a^b with respect to the exponent: G v log(a) where a > 0, else 0
// (the reference's guard, cpu_native.rs:271-274).
__device__ __forceinline__ float2 gm2_powexp_adj(float2 G, float2 v, float2 a) {
  return make_float2(a.x > 0.0f ? G.x * v.x * logf(a.x) : 0.0f,
                     a.y > 0.0f ? G.y * v.y * logf(a.y) : 0.0f);
}

__device__ __forceinline__ float2 gm2_pow(float2 a, float2 b) {
  return make_float2(powf(a.x, b.x), powf(a.y, b.y));
}

}  // namespace gpum
