// compiled.cuh -- the compiled engine's kernels, built at session creation by
// NVRTC for sm_100a together with the model functions that codegen.cpp
// generates from the bytecode (gm_data, gm_hoist, gm_value, gm_value_grad,
// gm_hoist_grad, gm_prior, gm_prior_grad; GM_NP/GM_NH/GM_ND; GM_G/GM_GG the
// chains per thread of the value and gradient kernels).
//
// Same skeleton as the interpreter engine (common.cuh); the body keeps each
// chain's parameters, hoisted parameter-only values and (for the gradient)
// the gradient accumulators in registers, so the observation loop is
// straight-line FP32 code with no dispatch.
#pragma once
#include "common.cuh"

namespace gpum {

// Per-thread sums: FP32 terms are added in blocks of kAccBlock into an FP32
// partial, and each block's partial is added into an FP64 sum.  The FP32
// error of a block is at most (kAccBlock - 1) ulp-scale of its terms and
// does not grow with the number of observations; the f32 -> f64 conversion
// and the f64 add (slow pipes) run once per block instead of per term.
constexpr int kAccBlock = 8;

struct Acc64 {
  double s;
  float part;
  __device__ __forceinline__ void init() {
    s = 0.0;
    part = 0.0f;
  }
  __device__ __forceinline__ void add(float x) { part += x; }
  __device__ __forceinline__ void flush() {
    s += (double)part;
    part = 0.0f;
  }
  __device__ __forceinline__ double total() const { return s + (double)part; }
};

template <int G, bool GRAD>
struct JitBody {
  static constexpr bool kChainLanes = false;
  static constexpr int kObsPerEval = 1;
  float p[G][GM_NP];
  float h[G][GM_NH];
  Acc64 acc[G];
  int cnt;  // terms in the open FP32 blocks
  float lastv[G];
  float gp[GRAD ? G : 1][GRAD ? GM_NP : 1];
  float gh[GRAD ? G : 1][GRAD ? GM_NH : 1];

  __device__ __forceinline__ void begin(const float* pc0, int CG) {
#pragma unroll
    for (int g = 0; g < G; ++g) {
#pragma unroll
      for (int j = 0; j < GM_NP; ++j) p[g][j] = pc0[j * CG + g];
      gm_hoist(p[g], h[g]);
      acc[g].init();
      lastv[g] = 0.0f;
    }
    cnt = 0;
    if (GRAD) {
#pragma unroll
      for (int g = 0; g < (GRAD ? G : 1); ++g) {
#pragma unroll
        for (int j = 0; j < (GRAD ? GM_NP : 1); ++j) gp[g][j] = 0.0f;
#pragma unroll
        for (int j = 0; j < (GRAD ? GM_NH : 1); ++j) gh[g][j] = 0.0f;
      }
    }
  }

  __device__ __forceinline__ void eval(const float* xo, int T, bool valid) {
    float d[GM_ND];
    gm_data(xo, T, d);
#pragma unroll
    for (int g = 0; g < G; ++g) {
      if (GRAD) {
        if (valid) {  // gradient terms of padding rows must not be accumulated
          const float v = gm_value_grad(d, p[g], h[g], gp[GRAD ? g : 0], gh[GRAD ? g : 0]);
          lastv[g] = v;
          acc[g].add(v);
        }
      } else {
        const float v = gm_value(d, p[g], h[g]);
        lastv[g] = v;
        if (valid) acc[g].add(v);
      }
    }
    if (valid && ++cnt == kAccBlock) {
      cnt = 0;
#pragma unroll
      for (int g = 0; g < G; ++g) acc[g].flush();
    }
  }

  __device__ __forceinline__ float last(int g) const { return lastv[g]; }

  __device__ __forceinline__ void end() {
    if (GRAD) {
#pragma unroll
      for (int g = 0; g < (GRAD ? G : 1); ++g) gm_hoist_grad(p[g], gh[g], gp[g]);
    }
  }

  __device__ __forceinline__ double total(int g, int w) const {
    if (w == 0) return acc[g].total();
    return (double)gp[GRAD ? g : 0][GRAD ? w - 1 : 0];
  }
};

#if GM_PAIR
// Value body over observation pairs: gm_data2 loads each column pair with one
// 64-bit shared-memory load and gm_value2 runs the model on both
// observations with two-wide FP32 instructions.  Parameters and hoisted
// values are kept as broadcast pairs (p, p) so every instruction is paired.
template <int G>
struct JitBody2 {
  static constexpr bool kChainLanes = false;
  static constexpr int kObsPerEval = 2;
  static constexpr int kTileObs = GM_T;
  float2 pp[G][GM_NP];
  float2 hh[G][GM_NH];
  double s[G];
  float2 part[G];
  float2 lastv[G];
  int cnt;  // observation pairs in the open FP32 blocks

  __device__ __forceinline__ void begin(const float* pc0, int CG) {
#pragma unroll
    for (int g = 0; g < G; ++g) {
      float p[GM_NP], h[GM_NH];
#pragma unroll
      for (int j = 0; j < GM_NP; ++j) p[j] = pc0[j * CG + g];
      gm_hoist(p, h);
#pragma unroll
      for (int j = 0; j < GM_NP; ++j) pp[g][j] = make_float2(p[j], p[j]);
#pragma unroll
      for (int j = 0; j < GM_NH; ++j) hh[g][j] = make_float2(h[j], h[j]);
      s[g] = 0.0;
      part[g] = make_float2(0.0f, 0.0f);
      lastv[g] = make_float2(0.0f, 0.0f);
    }
    cnt = 0;
  }

  // xo: the first observation of the pair (the second is xo + 1).
  __device__ __forceinline__ void eval2(const float* xo, int T, bool v0, bool v1) {
    float2 d[GM_ND];
    gm_data2(xo, T, d);
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const float2 v = gm_value2(d, pp[g], hh[g]);
      lastv[g] = v;
      if (v1) part[g] = __fadd2_rn(part[g], v);
      else if (v0) part[g].x += v.x;
    }
    if (v0 && ++cnt == kAccBlock) {
      cnt = 0;
#pragma unroll
      for (int g = 0; g < G; ++g) {
        s[g] += (double)part[g].x + (double)part[g].y;
        part[g] = make_float2(0.0f, 0.0f);
      }
    }
  }

  // A pair of a full tile outside pointwise output: no validity tests, no
  // block counter; the caller flushes once per tile.
  __device__ __forceinline__ void eval2_full(const float* xo) {
    float2 d[GM_ND];
    gm_data2(xo, GM_T, d);
#pragma unroll
    for (int g = 0; g < G; ++g) part[g] = __fadd2_rn(part[g], gm_value2(d, pp[g], hh[g]));
  }
  // Close the open FP32 blocks into the FP64 sums.
  __device__ __forceinline__ void flush() {
#pragma unroll
    for (int g = 0; g < G; ++g) {
      s[g] += (double)part[g].x + (double)part[g].y;
      part[g] = make_float2(0.0f, 0.0f);
    }
    cnt = 0;
  }

  __device__ __forceinline__ float2 last2(int g) const { return lastv[g]; }
  __device__ __forceinline__ void end() {}
  __device__ __forceinline__ double total(int g, int) const {
    return s[g] + ((double)part[g].x + (double)part[g].y);
  }
};
using ValueBody = JitBody2<GM_G>;
constexpr int kValueG = GM_G;
#elif GM_LANES
// Value body for wide models, one chain per lane: the lanes of a warp are 32
// chains, so every lane reads the same observation values (a shared-memory
// broadcast) and one 16-byte load per column serves four observations of all
// 32 chains.  Parameters come straight from the [np][C_pad] evaluation
// points; terms are added in FP32 blocks of eight observations, each block
// into an FP64 sum.
struct JitLanes {
  static constexpr bool kChainLanes = true;
  static constexpr bool kLanesAcc = false;
  static constexpr int kObsPerEval = 4;
  static constexpr int kTileObs = GM_T;
  float p[GM_NP];
  float h[GM_NH];
  double s;
  float part;
  int cnt;  // quads in the open FP32 block
  float lastv[4];

  __device__ __forceinline__ void begin_lanes(const float* pc, int C_pad) {
#pragma unroll
    for (int j = 0; j < GM_NP; ++j) p[j] = pc[(size_t)j * C_pad];
    gm_hoist(p, h);
    s = 0.0;
    part = 0.0f;
    cnt = 0;
  }

  // Observations xo .. xo + 3, of which the first nv are valid.
  __device__ __forceinline__ void eval4(const float* xo, int nv) {
    float v[4];
    gm_value4l(xo, p, h, v);
#pragma unroll
    for (int k = 0; k < 4; ++k) lastv[k] = v[k];
    if (nv == 4) {
      part = ((part + lastv[0]) + lastv[1]) + (lastv[2] + lastv[3]);
    } else {
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (k < nv) part += lastv[k];
    }
    if (++cnt == 2) {
      s += (double)part;
      part = 0.0f;
      cnt = 0;
    }
  }

  __device__ __forceinline__ float last4(int k) const { return lastv[k]; }
  __device__ __forceinline__ void end() {}
  __device__ __forceinline__ double total(int, int) const { return s + (double)part; }
};
using ValueBody = JitLanes;
constexpr int kValueG = 32;  // chains per warp group, as the host counts them
#else
using ValueBody = JitBody<GM_G, false>;
constexpr int kValueG = GM_G;
#endif

#if GM_LANESG
// Value + gradient body for wide models, one chain per lane (the chain-lane
// layout of JitLanes): gm_value_grad4l on four observations per broadcast
// load; each lane's FP32 parameter adjoints of one tile are added into its
// own FP64 row of the reduction buffer in shared memory (acc, W = 1 + np
// values, zeroed at the start), hoisted-value adjoints into FP64 registers,
// and pushed through the hoisted nodes once at the end.
struct JitLanesG {
  static constexpr bool kChainLanes = true;
  static constexpr bool kLanesAcc = true;
  static constexpr int kObsPerEval = 4;
  static constexpr int kTileObs = GM_T;
  float p[GM_NP];
  float h[GM_NH];
  float gp[GM_NP];
  float gh[GM_NH];
  double ghd[GM_NH];
  double* acc;
  double s;
  float part;
  int cnt;
  float lastv[4];

  __device__ __forceinline__ void begin_lanes_acc(const float* pc, int C_pad, double* row) {
#pragma unroll
    for (int j = 0; j < GM_NP; ++j) {
      p[j] = pc[(size_t)j * C_pad];
      gp[j] = 0.0f;
    }
    gm_hoist(p, h);
#pragma unroll
    for (int j = 0; j < GM_NH; ++j) {
      gh[j] = 0.0f;
      ghd[j] = 0.0;
    }
    acc = row;
    for (int w = 0; w < 1 + GM_NP; ++w) acc[w] = 0.0;
    s = 0.0;
    part = 0.0f;
    cnt = 0;
  }

  __device__ __forceinline__ void eval4(const float* xo, int nv) {
    float v[4];
    if (nv == 4) gm_value_grad4l(xo, 4, p, h, gp, gh, v);
    else gm_value_grad4l(xo, nv, p, h, gp, gh, v);
#pragma unroll
    for (int k = 0; k < 4; ++k) lastv[k] = v[k];
    if (nv == 4) {
      part = ((part + v[0]) + v[1]) + (v[2] + v[3]);
    } else {
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (k < nv) part += v[k];
    }
    if (++cnt == 2) {
      s += (double)part;
      part = 0.0f;
      cnt = 0;
    }
  }

  // After each tile: the tile's FP32 adjoints into the FP64 accumulators.
  __device__ __forceinline__ void flush_tile() {
#pragma unroll
    for (int j = 0; j < GM_NP; ++j) {
      acc[1 + j] += (double)gp[j];
      gp[j] = 0.0f;
    }
#pragma unroll
    for (int j = 0; j < GM_NH; ++j) {
      ghd[j] += (double)gh[j];
      gh[j] = 0.0f;
    }
  }

  __device__ __forceinline__ float last4(int k) const { return lastv[k]; }

  __device__ __forceinline__ void end() {
    flush_tile();
    float ghf[GM_NH], gx[GM_NP];
#pragma unroll
    for (int j = 0; j < GM_NH; ++j) ghf[j] = (float)ghd[j];
#pragma unroll
    for (int j = 0; j < GM_NP; ++j) gx[j] = 0.0f;
    gm_hoist_grad(p, ghf, gx);
#pragma unroll
    for (int j = 0; j < GM_NP; ++j) acc[1 + j] += (double)gx[j];
  }

  __device__ __forceinline__ double total(int, int w) const {
    return w == 0 ? s + (double)part : acc[w];
  }
};
using GradBody = JitLanesG;
constexpr int kGradG = 32;  // chains per warp group, as the host counts them
#else
using GradBody = JitBody<GM_GG, true>;
constexpr int kGradG = GM_GG;
#endif

// The generated f64 prior (value and reverse-mode gradient).
struct JitPrior {
  __device__ static double value(const ChainArgs&, int, const double* p) { return gm_prior(p); }
  __device__ static double value_grad(const ChainArgs&, int, const double* p, double* g) {
    return gm_prior_grad(p, g);
  }
};

}  // namespace gpum

// Materialized data-only operations: one thread per observation reads the
// data columns (column-major, leading dimension ld) and writes the operations'
// values into columns GM_NCOLS .. GM_NCOLS + n_mat - 1 of the same array.
extern "C" __global__ void gm_materialize(float* __restrict__ cols, long long n_obs,
                                          long long ld) {
  const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!GM_HAS_MAT || o >= n_obs) return;
  float m[GM_NMAT];
  gpum::gm_mat_obs(cols + o, ld, m);
#pragma unroll
  for (int k = 0; k < GM_NMAT; ++k) cols[(size_t)(GM_NCOLS + k) * ld + o] = m[k];
}

// The generated f64 prior at n points x[n][GM_NP], one thread per point;
// with grad != nullptr its gradient is added into grad[n][GM_NP].  Delayed
// acceptance reads these instead of interpreting the prior per chain.
extern "C" __global__ void gm_prior_batch(const double* __restrict__ x, int n,
                                          double* __restrict__ out, double* __restrict__ grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* p = x + (size_t)i * GM_NP;
  out[i] = grad ? gpum::gm_prior_grad(p, grad + (size_t)i * GM_NP) : gpum::gm_prior(p);
}

// Value-only kernel: PH_EVAL / PH_POINTWISE / RWM, DE and Cholesky steps.
// CTAs per SM the registers must allow (GM_VALUE_CTAS from the host: three
// for narrow paired models, 80 registers; two for the other paired ones).
#ifdef GM_VALUE_CTAS
#define GM_VALUE_MIN_CTAS GM_VALUE_CTAS
#elif GM_PAIR
#define GM_VALUE_MIN_CTAS 2
#else
#define GM_VALUE_MIN_CTAS 1
#endif
extern "C" __global__ void __launch_bounds__(gpum::kThreads, GM_VALUE_MIN_CTAS)
gm_iter_value(const __grid_constant__ gpum::TmapDesc tmap, gpum::EvalArgs E, gpum::ChainArgs A,
              int phase) {
  gpum::ValueBody body;
  gpum::run_iteration<gpum::kValueG, 1, gpum::ValueBody, gpum::JitPrior>(&tmap, E, A, phase,
                                                                          body);
}

// Value + gradient kernel: gradient batches and MALA steps (GM_GRAD_CTAS
// from the host: CTAs per SM the registers must allow).
#ifndef GM_GRAD_CTAS
#define GM_GRAD_CTAS 1
#endif
extern "C" __global__ void __launch_bounds__(gpum::kThreads, GM_GRAD_CTAS)
gm_iter_grad(const __grid_constant__ gpum::TmapDesc tmap, gpum::EvalArgs E, gpum::ChainArgs A,
             int phase) {
  gpum::GradBody body;
  gpum::run_iteration<gpum::kGradG, 1 + GM_NP, gpum::GradBody, gpum::JitPrior>(&tmap, E, A,
                                                                            phase,
                                                                        body);
}

#if GM_TC
// ----------------------------------------------------------------------------
// Tensor-core value kernel.  The model's linear predictor eta = sum_c
// coef_c(theta) x_c (codegen: the largest per-observation node affine in the
// data with parameter-only coefficients; an offset is the coefficient of a
// ones column) is, for the 128 chains of a CTA and a tile of GM_TC_TN
// observations, the product A (128 x K, coefficients) . B^T (TN x K, data).
// It runs on the 5th-generation tensor cores in TF32 with both operands split
// into a TF32 head and a TF32 rounding of the remainder, v = hi + lo:
// a.x ~ a_hi.x_hi + a_hi.x_lo + a_lo.x_hi, within 2^-20 of |a x| (2^-21 on
// average: the dropped a_lo.x_lo and the rounding of the lo parts), FP32
// accumulation in tensor memory.  The rest of the per-observation expression (gm_tc_tail2) runs on
// the FP32 pipes with eta read from tensor memory.
//
// Roles (GM_TC_EW epilogue warps, a multiple of four, and a control warp):
//   warps 0 .. EW-1  epilogue: warp w reads TMEM lane quarter w % 4 (chains
//                32 (w % 4) .. + 31, one chain per lane) and column part
//                w / 4 of each tile, evaluates the tail and sums its terms
//   warp EW      control, one thread: the copies (per tile of the packed
//                data, below, one bulk copy of the product columns into a
//                GM_TC_STAGES-deep operand ring and one of the tail columns
//                into a ring of four slots) and the MMAs (3 KP/8 per tile
//                into one of two accumulators of TN TMEM columns); the warp
//                allocates the tensor memory
// Barriers: bfull[s] / tfull[s] (copy landed), bempty[s] (the tile's MMAs
// are done with the operand stage: a tcgen05.commit), tempty[s] (the
// epilogue is done with the tail slot), accf[a] (accumulator a holds a tile),
// acce[a] (the epilogue has read it).  Every
// wait is bounded; one that runs out sets DEV_ERR_TC_TIMEOUT and a CTA-wide
// abort flag, the roles leave their loops, the control thread waits (bounded)
// for its MMAs and copies, and the CTA frees its tensor memory and finishes
// the chain block's bookkeeping.
//
// Packed data (gm_tc_pack, once per session): per tile of TN observations
// [hi: KP/4 chunks][TN][4] | [lo: same] | [tail: NTAIL][TN] floats, i.e. the
// canonical K-major, no-swizzle core-matrix layout of the MMA's B operand
// (core matrix (k/4, o/8) at (k/4 * TN/8 + o/8) * 128 bytes), so one
// contiguous copy fills a stage.
namespace gpum {
constexpr int kTcEpiWarps = GM_TC_EW;
constexpr int kTcThreads = 32 * (kTcEpiWarps + 1);
constexpr int kTcTN = GM_TC_TN;
constexpr int kTcKP = GM_TC_KP;
constexpr int kTcS = GM_TC_STAGES;  // operand stages (hi | lo product columns)
constexpr int kTcST = 4;            // tail-column slots
constexpr uint32_t kTcTileFloats = (uint32_t)(2 * kTcKP + GM_TC_NTAIL) * kTcTN;  // packed tile
constexpr uint32_t kTcStageFloats = (uint32_t)2 * kTcKP * kTcTN;
constexpr uint32_t kTcTailFloats = (uint32_t)GM_TC_NTAIL * kTcTN;
constexpr uint32_t kTcAFloats = (uint32_t)2 * kTcKP * kTcM;
// two accumulators, each at a power-of-two column offset (tcgen05.alloc
// takes a power of two)
constexpr uint32_t kTcAccCols = kTcTN <= 32 ? 32 : kTcTN <= 64 ? 64 : kTcTN <= 128 ? 128 : 256;
constexpr uint32_t kTcTmemCols = 2 * kTcAccCols;
constexpr int kTcParts = kTcEpiWarps / 4;  // epilogue warps per lane quarter
constexpr int kTcColsPerWarp = kTcTN / kTcParts;
// columns per TMEM load: 32 where the warp's share divides into them, else 16
constexpr int kTcChunk = kTcColsPerWarp % 32 == 0 ? 32 : 16;
static_assert(kTcKP % 8 == 0 && kTcTN % 16 == 0 && kTcTN <= 256 && kTcColsPerWarp % 16 == 0 &&
                  kTcEpiWarps % 4 == 0 && kTcParts <= 4,  // the reduction buffer holds 4 parts
              "tensor-core tile shape");
}  // namespace gpum

extern "C" __global__ void gm_tc_pack(const float* __restrict__ cols, long long n_obs,
                                      long long ld, long long n_tiles, float* __restrict__ xt,
                                      unsigned int* __restrict__ nonfinite) {
  using namespace gpum;
  const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n_tiles * kTcTN) return;
  const long long tile = o / kTcTN;
  const int r = (int)(o % kTcTN);
  float* base = xt + (size_t)tile * kTcTileFloats;
  const bool valid = o < n_obs;
  float v[GM_TC_K], t[GM_TC_NT1];
#pragma unroll
  for (int k = 0; k < GM_TC_K; ++k) v[k] = 0.0f;
#pragma unroll
  for (int k = 0; k < GM_TC_NT1; ++k) t[k] = 0.0f;
  if (valid) {
    gm_tc_colvals(cols + o, ld, v);
    gm_tc_tailvals(cols + o, ld, t);
  }
  bool bad = false;
#pragma unroll
  for (int kc = 0; kc < kTcKP / 4; ++kc) {
    float hi[4], lo[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = 4 * kc + e;
      float x = 0.0f;
      if (k < GM_TC_K) x = v[k];
      hi[e] = tf32_rna(x);
      lo[e] = isfinite(hi[e]) ? tf32_rna(x - hi[e]) : 0.0f;
      bad = bad || !isfinite(x);
    }
    *reinterpret_cast<float4*>(base + ((size_t)kc * kTcTN + r) * 4) =
        make_float4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<float4*>(base + (size_t)kTcKP * kTcTN + ((size_t)kc * kTcTN + r) * 4) =
        make_float4(lo[0], lo[1], lo[2], lo[3]);
  }
#pragma unroll
  for (int m = 0; m < GM_TC_NTAIL; ++m) base[(size_t)2 * kTcKP * kTcTN + m * kTcTN + r] = t[m];
  // a non-finite product column would turn into inf * 0 = NaN in the split
  // products: the host keeps such data on the FP32 kernel
  if (bad) atomicOr(nonfinite, 1u);
}

// eta of observation `col` of the tile on the FP32 pipe from the operands'
// hi + lo (the coefficients in shared memory, the tile's packed data in
// global memory): for a chain with an infinite coefficient, whose inf * 0
// products in the split form would be NaN where the plain product is +-inf.
__device__ __noinline__ float gm_tc_eta_fp32(const float* __restrict__ As,
                                                const float* __restrict__ xs, int cl, int col) {
  using namespace gpum;
  float e = 0.0f;
  for (int k = 0; k < kTcKP; ++k) {
    const int ao = ((((k >> 2) * (kTcM / 8) + (cl >> 3)) << 5) + ((cl & 7) << 2) + (k & 3));
    const int xo = ((((k >> 2) * (kTcTN / 8) + (col >> 3)) << 5) + ((col & 7) << 2) + (k & 3));
    const float a = As[ao] + As[kTcKP * kTcM + ao];
    const float x = xs[xo] + xs[kTcKP * kTcTN + xo];
    if (a != 0.0f) e = fmaf(a, x, e);
  }
  return e;
}

extern "C" __global__ void __launch_bounds__(gpum::kTcThreads, 1)
gm_iter_value_tc(const float* __restrict__ xt, gpum::EvalArgs E, gpum::ChainArgs A, int phase) {
  using namespace gpum;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int cb = blockIdx.x, ob = blockIdx.y, tiles_per_cta = E.tiles_per_cta;
  if (E.active) {  // delayed acceptance: geometry from the live count
    const int live = (int)*E.active;
    const int busy = (live + kTcM - 1) / kTcM;
    const int nob = da_obs_blocks(live, kTcM, (int)(gridDim.x * gridDim.y), E.ntiles,
                                  &tiles_per_cta);
    const int id = (int)(blockIdx.y * gridDim.x + blockIdx.x);
    if (busy == 0 || id >= busy * nob) return;
    cb = id % busy;
    ob = id / busy;
  }
  float* stg = reinterpret_cast<float*>(smem_raw);
  float* tls = stg + (size_t)kTcS * kTcStageFloats;            // tail slots
  float* As = tls + (size_t)kTcST * kTcTailFloats;
  double* red = reinterpret_cast<double*>(As + kTcAFloats);  // [column parts][128]
  uint32_t* inf_chain = reinterpret_cast<uint32_t*>(red + 4 * kTcM);  // [128]
  uint64_t* bfull = reinterpret_cast<uint64_t*>(inf_chain + kTcM);
  uint64_t* bempty = bfull + kTcS;
  uint64_t* tfull = bempty + kTcS;
  uint64_t* tempty = tfull + kTcST;
  uint64_t* accf = tempty + kTcST;
  uint64_t* acce = accf + 2;
  uint64_t* drain = acce + 2;
  uint32_t* misc = reinterpret_cast<uint32_t*>(drain + 1);  // TMEM base, ticket, abort
  volatile uint32_t* abort_flag = misc + 2;

  const int t0 = ob * tiles_per_cta;
  const int t1 = min(t0 + tiles_per_cta, E.ntiles);
  const int nt = max(t1 - t0, 0);
  const int chain0 = cb * kTcM;

  if (tid == 0) {
    for (int s = 0; s < kTcS; ++s) {
      mbar_init(&bfull[s], 1);
      mbar_init(&bempty[s], 1);
    }
    for (int s = 0; s < kTcST; ++s) {
      mbar_init(&tfull[s], 1);
      mbar_init(&tempty[s], kTcEpiWarps);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&accf[a], 1);
      mbar_init(&acce[a], kTcEpiWarps);
    }
    mbar_init(drain, 1);
    misc[2] = 0;
    mbar_fence_init();
  }
  if (warp == kTcEpiWarps) tmem_alloc(&misc[0], kTcTmemCols);
  // The coefficient operand, one chain per thread: [hi | lo] in the
  // canonical layout (core matrix (k/4, r/8) at (k/4 * 16 + r/8) * 128 bytes).
  if (tid < kTcM) {
    float p[GM_NP], a[GM_TC_K];
#pragma unroll
    for (int j = 0; j < GM_NP; ++j) p[j] = E.params[(size_t)j * E.C_pad + chain0 + tid];
    gm_tc_coef(p, a);
    uint32_t inf = 0;
#pragma unroll
    for (int kc = 0; kc < kTcKP / 4; ++kc) {
      float hi[4], lo[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int k = 4 * kc + e;
        float v = 0.0f;
        if (k < GM_TC_K) v = a[k];
        hi[e] = tf32_rna(v);
        lo[e] = isfinite(hi[e]) ? tf32_rna(v - hi[e]) : 0.0f;
        inf |= isinf(v) ? 1u : 0u;
      }
      const int off = ((kc * (kTcM / 8) + (tid >> 3)) << 5) + ((tid & 7) << 2);
      *reinterpret_cast<float4*>(As + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<float4*>(As + kTcKP * kTcM + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
    }
    inf_chain[tid] = inf;
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = misc[0];
  auto give_up = [&]() {
    atomicOr(E.err, DEV_ERR_TC_TIMEOUT);
    *abort_flag = 1u;
  };

  if (warp == kTcEpiWarps) {
    // ---- control: copies and MMAs
    if (lane == 0) {
      constexpr uint32_t idesc = umma_idesc_tf32(kTcM, kTcTN);
      constexpr uint32_t lbo_a = (kTcM / 8) * 128, lbo_b = (kTcTN / 8) * 128;
      const uint32_t a_hi = smem_addr(As), a_lo = a_hi + (uint32_t)kTcKP * kTcM * 4;
      auto load_b = [&](int k) {
        const int s = k % kTcS;
        mbar_expect_tx(&bfull[s], kTcStageFloats * 4);
        bulk_load(stg + (size_t)s * kTcStageFloats, xt + (size_t)(t0 + k) * kTcTileFloats,
                  kTcStageFloats * 4, &bfull[s]);
      };
      auto load_t = [&](int k) {
        const int s = k % kTcST;
        mbar_expect_tx(&tfull[s], kTcTailFloats * 4);
        bulk_load(tls + (size_t)s * kTcTailFloats,
                  xt + (size_t)(t0 + k) * kTcTileFloats + kTcStageFloats, kTcTailFloats * 4,
                  &tfull[s]);
      };
      int nb = 0, ntl = 0;  // tiles whose operands / tail columns were issued
      for (; nb < kTcS && nb < nt; ++nb) load_b(nb);
      if (GM_TC_NTAIL > 0)
        for (; ntl < kTcST && ntl < nt; ++ntl) load_t(ntl);
      for (int k = 0; k < nt; ++k) {
        if (*abort_flag) break;
        const int s = k % kTcS, acc = k & 1;
        if (!mbar_wait_bounded(&bfull[s], (uint32_t)((k / kTcS) & 1))) {
          give_up();
          break;
        }
        if (k >= 2 && !mbar_wait_bounded(&acce[acc], (uint32_t)(((k >> 1) - 1) & 1))) {
          give_up();
          break;
        }
        tc_fence_after();
        const uint32_t b_hi = smem_addr(stg + (size_t)s * kTcStageFloats);
        const uint32_t b_lo = b_hi + (uint32_t)kTcKP * kTcTN * 4;
        const uint32_t d = tmem + (uint32_t)acc * kTcAccCols;
        // the small products first: the accumulator rounds toward zero, so
        // only the KP/8 head products are added onto a large partial sum
#pragma unroll
        for (int kk = 0; kk < kTcKP / 8; ++kk) {
          const uint64_t ah = umma_smem_desc(a_hi + 2 * kk * lbo_a, lbo_a, 128);
          const uint64_t al = umma_smem_desc(a_lo + 2 * kk * lbo_a, lbo_a, 128);
          const uint64_t bh = umma_smem_desc(b_hi + 2 * kk * lbo_b, lbo_b, 128);
          const uint64_t bl = umma_smem_desc(b_lo + 2 * kk * lbo_b, lbo_b, 128);
          umma_tf32(d, ah, bl, idesc, kk > 0 ? 1u : 0u);
          umma_tf32(d, al, bh, idesc, 1u);
        }
#pragma unroll
        for (int kk = 0; kk < kTcKP / 8; ++kk)
          umma_tf32(d, umma_smem_desc(a_hi + 2 * kk * lbo_a, lbo_a, 128),
                    umma_smem_desc(b_hi + 2 * kk * lbo_b, lbo_b, 128), idesc, 1u);
        umma_commit(&accf[acc]);
        umma_commit(&bempty[s]);
        if (k >= 1) {
          // the operand stage of tile k - 1 is free once its MMAs are done
          if (nb < nt) {
            if (!mbar_wait_bounded(&bempty[(k - 1) % kTcS], (uint32_t)(((k - 1) / kTcS) & 1))) {
              give_up();
              break;
            }
            load_b(nb++);
          }
          // the tail slot of tile k - 1 once its epilogue is done (the next
          // tile's MMAs wait for that epilogue anyway)
          if (GM_TC_NTAIL > 0 && ntl < nt) {
            if (!mbar_wait_bounded(&tempty[(k - 1) % kTcST], (uint32_t)(((k - 1) / kTcST) & 1))) {
              give_up();
              break;
            }
            load_t(ntl++);
          }
        }
      }
      // every MMA has finished before the tensor memory is released, and no
      // copy is still writing into shared memory
      umma_commit(drain);
      if (!mbar_wait_bounded(drain, 0u)) give_up();
      for (int i = max(0, nb - kTcS); i < nb; ++i)
        if (!mbar_wait_bounded(&bfull[i % kTcS], (uint32_t)((i / kTcS) & 1))) give_up();
      for (int i = max(0, ntl - kTcST); i < ntl; ++i)
        if (!mbar_wait_bounded(&tfull[i % kTcST], (uint32_t)((i / kTcST) & 1))) give_up();
    }
  } else {
    // ---- epilogue
    const int q = warp & 3, part = warp >> 2;
    const int cl = q * 32 + lane;
    const int c = chain0 + cl;
    float2 pp[GM_NP], hh[GM_NH];
    {
      float p[GM_NP], h[GM_NH];
#pragma unroll
      for (int j = 0; j < GM_NP; ++j) p[j] = E.params[(size_t)j * E.C_pad + c];
      gm_hoist(p, h);
#pragma unroll
      for (int j = 0; j < GM_NP; ++j) pp[j] = make_float2(p[j], p[j]);
#pragma unroll
      for (int j = 0; j < GM_NH; ++j) hh[j] = make_float2(h[j], h[j]);
    }
    const bool inf = inf_chain[cl] != 0;
    const bool warp_inf = __any_sync(0xffffffffu, inf);
    double sum = 0.0;
    for (int k = 0; k < nt; ++k) {
      if (*abort_flag) break;
      const int st = k % kTcST, acc = k & 1;
      // warp-uniform waits: the accumulator and the tile's tail columns
      bool ok = mbar_wait_bounded(&accf[acc], (uint32_t)((k >> 1) & 1)) &&
                (GM_TC_NTAIL == 0 || mbar_wait_bounded(&tfull[st], (uint32_t)((k / kTcST) & 1)));
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) {
        if (lane == 0) give_up();
        break;
      }
      tc_fence_after();
      const float* xg = xt + (size_t)(t0 + k) * kTcTileFloats;  // the packed tile
      const float* tail = tls + (size_t)st * kTcTailFloats;
      const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) +
                             (uint32_t)acc * kTcAccCols + (uint32_t)(part * kTcColsPerWarp);
      const long long obs0 = (long long)(t0 + k) * kTcTN + part * kTcColsPerWarp;
      float2 tsum = make_float2(0.0f, 0.0f);
#pragma unroll 1
      for (int ch = 0; ch < kTcColsPerWarp / kTcChunk; ++ch) {
        float v[kTcChunk];
        tmem_ld(taddr + (uint32_t)(ch * kTcChunk), v);
        const int col0 = part * kTcColsPerWarp + ch * kTcChunk;
        if (warp_inf) {  // a chain of this warp has an infinite coefficient
#pragma unroll
          for (int j = 0; j < kTcChunk; ++j)
            if (inf) v[j] = gm_tc_eta_fp32(As, xg, cl, col0 + j);
        }
        float2 val[kTcChunk / 2];
        float4 tq[GM_TC_NT1];  // the tail columns of two pairs (a 16-byte broadcast load)
#pragma unroll
        for (int j = 0; j < kTcChunk / 2; ++j) {
          float2 t[GM_TC_NT1];
#pragma unroll
          for (int m = 0; m < GM_TC_NTAIL; ++m) {
            if ((j & 1) == 0)
              tq[m] = *reinterpret_cast<const float4*>(tail + m * kTcTN + col0 + 2 * j);
            t[m] = (j & 1) ? make_float2(tq[m].z, tq[m].w) : make_float2(tq[m].x, tq[m].y);
          }
          val[j] = gm_tc_tail2(make_float2(v[2 * j], v[2 * j + 1]), t, pp, hh);
        }
        const long long o0 = obs0 + ch * kTcChunk;
        if (o0 + kTcChunk > (long long)E.n_obs) {  // the ragged end of the last tile
#pragma unroll
          for (int j = 0; j < kTcChunk / 2; ++j) {
            if (o0 + 2 * j >= E.n_obs) val[j].x = 0.0f;
            if (o0 + 2 * j + 1 >= E.n_obs) val[j].y = 0.0f;
          }
        }
        // pairwise: the FP32 error of a chunk grows with log2 of its terms
#pragma unroll
        for (int w = kTcChunk / 4; w > 0; w >>= 1) {
#pragma unroll
          for (int j = 0; j < w; ++j) val[j] = __fadd2_rn(val[j], val[j + w]);
        }
        tsum = __fadd2_rn(tsum, val[0]);
      }
      sum += (double)tsum.x + (double)tsum.y;
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&acce[acc]);
        if (GM_TC_NTAIL > 0) mbar_arrive(&tempty[st]);
      }
    }
    red[part * kTcM + cl] = sum;
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kTcEpiWarps) tmem_dealloc(tmem, kTcTmemCols);
  // The chain's value over this observation block: the column parts in
  // order.
  if (tid < kTcM) {
    double v = red[tid];
#pragma unroll
    for (int pt = 1; pt < kTcParts; ++pt) v += red[pt * kTcM + tid];
    E.partials[(size_t)ob * E.C_pad + chain0 + tid] = v;
  }
  if (phase == PH_EVAL) return;
  finish_chain_block<1, JitPrior>(E, A, cb, kTcM, phase, &misc[1], kTcThreads);
}
#endif  // GM_TC
