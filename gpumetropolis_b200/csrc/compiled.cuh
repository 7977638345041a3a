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
