// kernels.cuh -- the interpreter engine's per-iteration kernel, and helper
// kernels (data layout, points, draws layout).
//
// The evaluation body here is the register-stack interpreter (interp.cuh):
// the bytecode is whatever the session compiled, read from the constant bank.
#pragma once
#include "common.cuh"
#include "interp.cuh"

namespace gpum {

template <int G, int D>
struct InterpBody {
  const EvalProg& pg;
  const float* pc0;
  int CG;
  float s[D][G];
  Comp acc[G];
  __device__ explicit InterpBody(const EvalProg& p) : pg(p), pc0(nullptr), CG(0) {}
  __device__ __forceinline__ void begin(const float* p0, int cg) {
    pc0 = p0;
    CG = cg;
#pragma unroll
    for (int g = 0; g < G; ++g) acc[g].init();
  }
  __device__ __forceinline__ void eval(const float* xo, int T, bool valid) {
    interp_run<G, D>(pg, s, xo, T, pc0, CG);
    if (valid) {
#pragma unroll
      for (int g = 0; g < G; ++g) acc[g].add(s[0][g]);
    }
  }
  __device__ __forceinline__ float last(int g) const { return s[0][g]; }
  __device__ __forceinline__ void end() {}
  __device__ __forceinline__ double total(int g, int) const { return acc[g].total(); }
};

// f64 prior interpreted from the source bytecode; the interpreter engine has
// no gradient (MALA runs on the compiled engine).
struct InterpPrior {
  __device__ static double value(const ChainArgs& A, const double* p) {
    return prior_interp(A.prior_code, A.n_prior, A.prior_consts, p);
  }
  __device__ static double value_grad(const ChainArgs& A, const double* p, double*) {
    return prior_interp(A.prior_code, A.n_prior, A.prior_consts, p);
  }
};

template <int G, int D>
__global__ void __launch_bounds__(kThreads, 2)
iter_kernel(const __grid_constant__ EvalProg prog, const __grid_constant__ TmapDesc tmap,
            EvalArgs E, ChainArgs A, int phase) {
  InterpBody<G, D> body(prog);
  run_iteration<G, 1, InterpBody<G, D>, InterpPrior>(&tmap, E, A, phase, body);
}

// ------------------------------------------------------------- helpers
// Row-major f64 rows [r0, r0+nr) -> column-major f32 [ncols][ld].
static __global__ void convert_rows_kernel(const double* __restrict__ src, float* __restrict__ dst,
                                    int ncols, int64_t ld, int64_t r0, int64_t nr) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr * ncols) return;
  const int64_t r = i / ncols, j = i % ncols;
  dst[(int64_t)j * ld + r0 + r] = (float)src[i];
}

// f64 chain-major points [C][np] -> f32 [np][C_pad]; pad chains copy chain 0.
static __global__ void points_to_params_kernel(const double* __restrict__ pts, float* __restrict__ params,
                                        int n, int np, int C_pad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np * C_pad) return;
  const int j = i / C_pad, c = i % C_pad;
  const int src = c < n ? c : 0;
  params[i] = (float)pts[(size_t)src * np + j];
}

// Internal draws [n_iter][np][C_pad] -> the reference layout, column-major
// (n_iter, C, np): out[t + n_iter*(c + C*j)] (chain_kernel.rs:345).
static __global__ void draws_layout_kernel(const float* __restrict__ in, float* __restrict__ out,
                                    int n_iter, int np, int C, int C_pad) {
  __shared__ float tile[32][33];
  const int j = blockIdx.z;
  const int c0 = blockIdx.x * 32, t0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int t = t0 + r, c = c0 + threadIdx.x;
    if (t < n_iter && c < C) tile[r][threadIdx.x] = in[((size_t)t * np + j) * C_pad + c];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int c = c0 + r, t = t0 + threadIdx.x;
    if (t < n_iter && c < C)
      out[(size_t)t + (size_t)n_iter * ((size_t)c + (size_t)C * j)] = tile[threadIdx.x][r];
  }
}

}  // namespace gpum
