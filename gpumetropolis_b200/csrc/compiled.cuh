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

// Each observation's FP32 value is accumulated into an FP64 sum (exact per
// term, two instructions), so per-thread partial sums carry no FP32 error.
struct Acc64 {
  double s;
  __device__ __forceinline__ void init() { s = 0.0; }
  __device__ __forceinline__ void add(float x) { s += (double)x; }
  __device__ __forceinline__ double total() const { return s; }
};

template <int G, bool GRAD>
struct JitBody {
  float p[G][GM_NP];
  float h[G][GM_NH];
  Acc64 acc[G];
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

// The generated f64 prior (value and reverse-mode gradient).
struct JitPrior {
  __device__ static double value(const ChainArgs&, const double* p) { return gm_prior(p); }
  __device__ static double value_grad(const ChainArgs&, const double* p, double* g) {
    return gm_prior_grad(p, g);
  }
};

}  // namespace gpum

// Value-only kernel: PH_EVAL / PH_POINTWISE / RWM, DE and Cholesky steps.
extern "C" __global__ void __launch_bounds__(gpum::kThreads, 1)
gm_iter_value(const __grid_constant__ gpum::TmapDesc tmap, gpum::EvalArgs E, gpum::ChainArgs A,
              int phase) {
  gpum::JitBody<GM_G, false> body;
  gpum::run_iteration<GM_G, 1, gpum::JitBody<GM_G, false>, gpum::JitPrior>(&tmap, E, A, phase,
                                                                           body);
}

// Value + gradient kernel: gradient batches and MALA steps.
extern "C" __global__ void __launch_bounds__(gpum::kThreads, 1)
gm_iter_grad(const __grid_constant__ gpum::TmapDesc tmap, gpum::EvalArgs E, gpum::ChainArgs A,
             int phase) {
  gpum::JitBody<GM_GG, true> body;
  gpum::run_iteration<GM_GG, 1 + GM_NP, gpum::JitBody<GM_GG, true>, gpum::JitPrior>(
      &tmap, E, A, phase, body);
}
