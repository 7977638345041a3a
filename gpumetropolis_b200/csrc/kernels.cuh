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
  static constexpr bool kChainLanes = false;
  static constexpr int kObsPerEval = 1;
  const EvalProg& pg;
  const float* pc0;
  int CG;
  float* hsm;
  float2 s[D][G / 2];  // chain pairs
  Comp acc[G];
  __device__ InterpBody(const EvalProg& p, float* h) : pg(p), pc0(nullptr), CG(0), hsm(h) {}
  __device__ __forceinline__ void begin(const float* p0, int cg) {
    pc0 = p0;
    CG = cg;
#pragma unroll
    for (int g = 0; g < G; ++g) acc[g].init();
  }
  __device__ __forceinline__ void eval(const float* xo, int T, bool valid) {
    interp_run<G, D>(pg, s, xo, T, pc0, CG, hsm);
    if (valid) {
#pragma unroll
      for (int h = 0; h < G / 2; ++h) {
        acc[2 * h].add(s[0][h].x);
        acc[2 * h + 1].add(s[0][h].y);
      }
    }
  }
  __device__ __forceinline__ float last(int g) const {
    return (g & 1) ? s[0][g >> 1].y : s[0][g >> 1].x;
  }
  __device__ __forceinline__ void end() {}
  __device__ __forceinline__ double total(int g, int) const { return acc[g].total(); }
};

// f64 prior interpreted from the source bytecode; its gradient (MALA on the
// interpreter engine) by the reverse-mode tape over chain c's scratch.
struct InterpPrior {
  __device__ static double value(const ChainArgs& A, int, const double* p) {
    return prior_interp(A.prior_code, A.n_prior, A.prior_consts, p);
  }
  __device__ static double value_grad(const ChainArgs& A, int c, const double* p, double* g) {
    const size_t n = (size_t)(A.n_prior > 0 ? A.n_prior : 1);
    double* tv = A.ptape + (size_t)c * 2 * n;
    uint32_t* ti = A.ptape_i + (size_t)c * 2 * n;
    return prior_value_grad_tape(A.prior_code, A.n_prior, A.prior_consts, p, g, tv, tv + n, ti,
                                 ti + n);
  }
};

// The widest variants (sixteen chains per thread over a six-deep stack, eight
// over eight: 96 and 64 stack registers) keep their stacks in registers at one
// CTA per SM; the others fit two.
template <int G, int D>
__global__ void __launch_bounds__(kThreads, (G >= 8 ? 1 : 2))
iter_kernel(const __grid_constant__ EvalProg prog, const __grid_constant__ TmapDesc tmap,
            EvalArgs E, ChainArgs A, int phase) {
  static_assert(kThreads == kInterpThreads, "the operand scratch is laid out per thread");
  __shared__ float hsm[2 * G * kInterpThreads];
  InterpBody<G, D> body(prog, hsm + threadIdx.x);
  run_iteration<G, 1, InterpBody<G, D>, InterpPrior>(&tmap, E, A, phase, body);
}

// ------------------------------------------------------- failure self-test
// The device-failure path end to end: an mbarrier that expects one arrival
// and gets none, polled by every thread at most `polls` times and for at
// most `max_ns` nanoseconds; the wait runs out, thread 0 sets the error word
// the host reads after every run, and the kernel returns (no copy or MMA is
// in flight, nothing hangs).
static __global__ void selftest_wait_kernel(uint32_t* err, uint32_t polls, uint64_t max_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  const uint64_t t0 = gm_globaltimer();
  bool done = false;
  for (uint32_t i = 0; i < polls && !done; ++i) {
    done = mbar_try_wait(&bar, 0u);
    if (gm_globaltimer() - t0 > max_ns) break;
  }
  if (__syncthreads_or(done ? 0 : 1) && threadIdx.x == 0) atomicOr(err, DEV_ERR_WAIT_SELFTEST);
}

// ------------------------------------------ gradient in the interpreter engine
// The node program of compile_grad_program (program.hpp) in the constant bank.
struct __align__(16) GradProg {
  uint32_t n_nodes, root, has_root, np;
  uint32_t node[kMaxGradNodes];
  float cst[kMaxConsts];
};

// Value and parameter gradient per observation by a reverse sweep over a tape
// of the observation's node values (cpu_native.rs:148-279 in FP32, with the
// compiled engine's local derivatives: POW's exponent term only where the
// base is positive, LGAMMA's the digamma, an exponent of constant 2 as a
// square).  One chain per thread, lanes over observations (G = 1); the tape
// and the adjoints live in the thread's local memory.  W = 1 + the largest
// parameter count the instantiation serves; entries past np stay 0.
template <int W>
struct InterpGradBody {
  static constexpr bool kChainLanes = false;
  static constexpr int kObsPerEval = 1;
  static constexpr int kNp = W - 1;
  const GradProg& pg;
  const float* pc0;
  int CG;
  float vals[kMaxGradNodes];
  float adj[kMaxGradNodes];
  float gp[kNp];
  double gpd[kNp];
  double s;
  float part, lastv;
  int cnt;
  __device__ explicit InterpGradBody(const GradProg& p) : pg(p), pc0(nullptr), CG(0) {}

  __device__ __forceinline__ void begin(const float* p0, int cg) {
    pc0 = p0;
    CG = cg;
    for (int j = 0; j < kNp; ++j) {
      gp[j] = 0.0f;
      gpd[j] = 0.0;
    }
    s = 0.0;
    part = 0.0f;
    lastv = 0.0f;
    cnt = 0;
  }
  __device__ __forceinline__ float fetch(uint32_t r, const float* xo, int T) const {
    const uint32_t t = r & 3u, i = r >> 2;
    return t == GREF_NODE ? vals[i]
         : t == GREF_CONST ? pg.cst[i]
         : t == GREF_PARAM ? pc0[(size_t)i * CG]
                           : xo[(size_t)i * T];
  }
  __device__ __forceinline__ void sink(uint32_t r, float x) {
    const uint32_t t = r & 3u, i = r >> 2;
    if (t == GREF_NODE) adj[i] += x;
    else if (t == GREF_PARAM) gp[i] += x;
  }
  __device__ __forceinline__ void flush() {
    s += (double)part;
    part = 0.0f;
    for (uint32_t j = 0; j < pg.np; ++j) {
      gpd[j] += (double)gp[j];
      gp[j] = 0.0f;
    }
    cnt = 0;
  }
  __device__ void eval(const float* xo, int T, bool valid) {
    if (!valid) {  // padding rows add neither value nor gradient
      lastv = 0.0f;
      return;
    }
    const uint32_t n = pg.n_nodes;
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t w = pg.node[i], op = w & 15u;
      const uint32_t ra = (w >> 4) & 0x3FFFu, rb = w >> 18;
      const float a = fetch(ra, xo, T);
      float v;
      if (op == 7) v = -a;
      else if (op == 8) v = expf(a);
      else if (op == 9) v = logf(a);
      else if (op == 10) v = sqrtf(a);
      else if (op == 12) v = lgammaf(a);
      else {
        const float b = fetch(rb, xo, T);
        if (op == 3) v = a + b;
        else if (op == 4) v = a - b;
        else if (op == 5) v = a * b;
        else if (op == 6) v = a / b;
        else v = ((rb & 3u) == GREF_CONST && b == 2.0f) ? a * a : powf(a, b);
      }
      vals[i] = v;
    }
    const float val = pg.has_root ? fetch(pg.root, xo, T) : 0.0f;
    lastv = val;
    part += val;
    if (pg.has_root) {
      if ((pg.root & 3u) == GREF_NODE) {
        for (uint32_t i = 0; i < n; ++i) adj[i] = 0.0f;
        adj[pg.root >> 2] = 1.0f;
        for (int i = (int)n - 1; i >= 0; --i) {
          const float g = adj[i];
          if (g == 0.0f) continue;
          const uint32_t w = pg.node[i], op = w & 15u;
          const uint32_t ra = (w >> 4) & 0x3FFFu, rb = w >> 18;
          const float a = fetch(ra, xo, T), v = vals[i];
          switch (op) {
            case 3: sink(ra, g); sink(rb, g); break;
            case 4: sink(ra, g); sink(rb, -g); break;
            case 5: {
              const float b = fetch(rb, xo, T);
              sink(ra, g * b);
              sink(rb, g * a);
              break;
            }
            case 6: {
              const float b = fetch(rb, xo, T);
              sink(ra, g / b);
              sink(rb, -g * v / b);
              break;
            }
            case 7: sink(ra, -g); break;
            case 8: sink(ra, g * v); break;
            case 9: sink(ra, g / a); break;
            case 10: sink(ra, g * 0.5f / v); break;
            case 12: sink(ra, g * gm_digammaf(a)); break;
            default: {
              const float b = fetch(rb, xo, T);
              if ((rb & 3u) == GREF_CONST && b == 2.0f) {
                sink(ra, g * 2.0f * a);
              } else {
                sink(ra, g * b * powf(a, b - 1.0f));
                sink(rb, a > 0.0f ? g * v * logf(a) : 0.0f);
              }
              break;
            }
          }
        }
      } else if ((pg.root & 3u) == GREF_PARAM) {
        gp[pg.root >> 2] += 1.0f;
      }
    }
    if (++cnt == 8) flush();
  }
  __device__ __forceinline__ float last(int) const { return lastv; }
  __device__ __forceinline__ void end() { flush(); }
  __device__ __forceinline__ double total(int, int w) const {
    if (w == 0) return s + (double)part;
    return w - 1 < (int)pg.np ? gpd[w - 1] : 0.0;
  }
};

template <int W>
__global__ void __launch_bounds__(kThreads, 1)
iter_kernel_grad(const __grid_constant__ GradProg prog, const __grid_constant__ TmapDesc tmap,
                 EvalArgs E, ChainArgs A, int phase) {
  InterpGradBody<W> body(prog);
  run_iteration<1, W, InterpGradBody<W>, InterpPrior>(&tmap, E, A, phase, body);
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

// ===================================================== delayed acceptance
// Two-stage Metropolis-Hastings (Christen & Fox 2005) with the surrogate
// log-likelihood s() as stage 1 and the exact log-likelihood l() as stage 2:
//   stage 1: accept y with min(1, exp([s(y)+p(y) - s(x)-p(x)] / T) q(x|y)/q(y|x))
//   stage 2: accept with min(1, exp([(l(y)-l(x)) - (s(y)-s(x))] / T))
// (p = prior, which cancels in stage 2, as does the proposal ratio: the
// stage-1 acceptance of the reverse move carries its inverse).  The product
// of the two acceptance probabilities satisfies detailed balance for the
// exact tempered posterior, so the target is unchanged; only stage-1
// survivors are evaluated exactly.  The proposal is the random walk, DE, or
// a Langevin move whose drift is the surrogate log-posterior gradient (so no
// exact gradient is ever needed).
namespace gpum {

// ------------------------------------------------- draw moments (adaptation)
// Moments of the draws of iterations [t0, t0 + n) in the internal layout
// [n_iter][np][C_pad], all in f64 and in a fixed order: per chain and
// parameter the mean and the sum of squared deviations (two passes), the
// pooled mean per parameter, and the pooled sums of cross deviations.
static __global__ void moments_chain_kernel(const float* __restrict__ draws, int np, int C,
                                            int C_pad, int t0, int n, double* __restrict__ mean,
                                            double* __restrict__ m2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np * C) return;
  const int j = i / C, c = i % C;  // consecutive threads: consecutive chains
  double sm = 0.0;
  for (int t = 0; t < n; ++t) sm += (double)draws[((size_t)(t0 + t) * np + j) * C_pad + c];
  const double mu = sm / n;
  double q = 0.0;
  for (int t = 0; t < n; ++t) {
    const double dv = (double)draws[((size_t)(t0 + t) * np + j) * C_pad + c] - mu;
    q += dv * dv;
  }
  mean[(size_t)c * np + j] = mu;
  m2[(size_t)c * np + j] = q;
}

// One block per parameter: pooled mean of the n x C values (fixed-order
// strided sums, then a fixed shared-memory tree).
static __global__ void moments_pool_mean_kernel(const float* __restrict__ draws, int np, int C,
                                                int C_pad, int t0, int n,
                                                double* __restrict__ pmean) {
  __shared__ double red[256];
  const int j = blockIdx.x;
  const size_t total = (size_t)n * C;
  double sm = 0.0;
  for (size_t k = threadIdx.x; k < total; k += blockDim.x) {
    const size_t t = k / C, c = k % C;
    sm += (double)draws[((t0 + t) * np + j) * C_pad + c];
  }
  red[threadIdx.x] = sm;
  __syncthreads();
  for (int off = 128; off > 0; off >>= 1) {
    if ((int)threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) pmean[j] = red[0] / (double)total;
}

// One block per (j, k >= j): pooled sum of (x_j - m_j)(x_k - m_k).
static __global__ void moments_pool_m2_kernel(const float* __restrict__ draws, int np, int C,
                                              int C_pad, int t0, int n,
                                              const double* __restrict__ pmean,
                                              double* __restrict__ pm2) {
  __shared__ double red[256];
  const int j = blockIdx.x / np, k = blockIdx.x % np;
  if (k < j) return;  // uniform per block
  const size_t total = (size_t)n * C;
  const double mj = pmean[j], mk = pmean[k];
  double sm = 0.0;
  for (size_t q = threadIdx.x; q < total; q += blockDim.x) {
    const size_t t = q / C, c = q % C;
    const double a = (double)draws[((t0 + t) * np + j) * C_pad + c] - mj;
    const double b = (double)draws[((t0 + t) * np + k) * C_pad + c] - mk;
    sm += a * b;
  }
  red[threadIdx.x] = sm;
  __syncthreads();
  for (int off = 128; off > 0; off >>= 1) {
    if ((int)threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    pm2[(size_t)j * np + k] = red[0];
    pm2[(size_t)k * np + j] = red[0];
  }
}

// ------------------------------------------------------ parallel tempering
// Replica exchange on the device (the reference swaps on the host between
// batches, R/adaptive.R:272-413): after every `every`-th iteration, the
// adjacent pairs (i, i + 1) of each ladder -- contiguous groups of K chains
// with the temperatures along the group -- of one parity (alternating from
// exchange to exchange, starting with the even pairs) exchange states with
// probability min(1, exp(delta)), delta = (lp[i+1] - lp[i]) (1/T[i] - 1/T[i+1])
// on the untempered log posteriors.  The proposals already drawn for the
// next iteration were centred on the old states, so both chains of an
// exchanged pair draw new ones.  Uniforms: Philox keyed by (seed, exchange,
// pair).  One thread per pair; the pairs of one parity are disjoint.
struct PtArgs {
  int K;               // ladder length
  int every;           // iterations between exchanges
  const uint32_t* iter;  // [1] iterations done (the step's or the DA loop's counter)
  double* sll_x;       // [C] delayed acceptance: surrogate value at the state, or null
  double* prior_x;     // [C] delayed acceptance: prior at the state, or null
  uint32_t* n_swaps;   // [1] exchanges done
  uint32_t* att;       // [C] attempts of pair (c, c + 1)
  uint32_t* acc;       // [C] accepted exchanges of pair (c, c + 1)
  float* params;       // [np][C_pad] evaluation points of the next iteration
  int C_pad;
};

static __global__ void pt_exchange_kernel(ChainArgs A, PtArgs P) {
  const uint32_t t = P.iter[0];  // iterations done (all chain blocks agree here)
  if (t == 0 || t % (uint32_t)P.every != 0 || t >= A.n_iter) return;
  const uint32_t s = t / (uint32_t)P.every;  // exchange number, from 1
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int C = A.n_chains, np = A.np;
  if (i == 0) P.n_swaps[0] = s;
  if (i + 1 >= C || (i % P.K) == P.K - 1) return;     // not a pair of one ladder
  if (((i % P.K) & 1) != (int)((s + 1) & 1)) return;  // odd exchanges: even pairs
  const double lpa = A.cur[i], lpb = A.cur[i + 1];
  const double delta = (lpb - lpa) * (1.0 / A.temp[i] - 1.0 / A.temp[i + 1]);
  const U4 r = philox4x32_10(U4{(uint32_t)i, s, 0x50545357u, 0u}, A.seed, 0x3C6EF372u);
  const double u = u53(r.x, r.y);
  P.att[i] += 1;
  if (!(isfinite(delta) && log(u) < delta)) return;
  P.acc[i] += 1;
  double* xa = A.state + (size_t)i * np;
  double* xb = A.state + (size_t)(i + 1) * np;
  for (int j = 0; j < np; ++j) {
    const double tmp = xa[j];
    xa[j] = xb[j];
    xb[j] = tmp;
  }
  A.cur[i] = lpb;
  A.cur[i + 1] = lpa;
  if (P.sll_x) {  // the two-stage loop's cached values follow their states
    const double s0 = P.sll_x[i], p0 = P.prior_x[i];
    P.sll_x[i] = P.sll_x[i + 1];
    P.prior_x[i] = P.prior_x[i + 1];
    P.sll_x[i + 1] = s0;
    P.prior_x[i + 1] = p0;
  }
  if (A.mode == MODE_MALA) {  // the cached gradients belong to the states
    double* ga = A.gx + (size_t)i * np;
    double* gb = A.gx + (size_t)(i + 1) * np;
    for (int j = 0; j < np; ++j) {
      const double tmp = ga[j];
      ga[j] = gb[j];
      gb[j] = tmp;
    }
  }
  for (int c = i; c <= i + 1; ++c) {
    Stream rs = make_stream(A, c);
    rs.it = t;
    rs.k = 0x40000000u;  // counters apart from the iteration's own proposal
    propose(A, c, rs, P.params, P.C_pad);
    A.ctr[c] = rs.ctr;
  }
}

// Path-B DE proposals of generation A.iter[0] for every chain (one thread per
// chain), between the previous generation's accepts and this generation's
// evaluation.  All chain blocks have the same iteration count here.
static __global__ void desync_propose_kernel(ChainArgs A, float* params, int C_pad) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.n_chains) return;
  const uint32_t t = A.iter[0];
  if (t >= A.n_iter) return;
  Stream rs = make_stream(A, c);
  rs.it = t;
  rs.k = 0;
  propose_desync(A, c, rs, params, C_pad);
  A.ctr[c] = rs.ctr;
}

struct DaArgs {
  double* sll_x;     // [C] surrogate log-likelihood at the state
  double* sll_y;     // [C] surrogate log-likelihood at the proposal
  double* prior_x;   // [C] prior at the state
  double* prior_y;   // [C] prior at the proposal
  uint32_t* flag;    // [C] stage 1 accepted this iteration
  uint32_t* slot;    // [C] position in the compacted evaluation
  uint32_t* active;  // [1] stage-1 acceptances this iteration
  uint32_t* iter;    // [1] iterations done
  uint32_t* stage1;  // [C] stage-1 acceptance counts
  float* params;     // [np][C_pad] compacted evaluation points
  float* full;       // [np][C_pad] scratch for propose()
  int C_pad;
  // Langevin proposal (MALA): the surrogate's data-term gradient at the
  // proposals (at the states during set-up), and the prior tape's scratch
  double* gs;        // [C][np]
  double* tvals;     // [C][n_prior]
  double* tadj;      // [C][n_prior]
  uint32_t* tlhs;    // [C][n_prior]
  uint32_t* trhs;    // [C][n_prior]
  // 1: the compiled engine's prior kernel has already written prior_x (set-up)
  // or prior_y (each iteration) and, with the Langevin proposal, added the
  // prior's gradient into gs; 0: the kernels interpret the prior themselves
  int prior_ready;
};

// Surrogate log-posterior gradient at theta: the surrogate's data-term
// gradient gs plus the f64 prior's gradient (tape); returns the prior.
__device__ __forceinline__ double da_post_grad(const ChainArgs& A, const DaArgs& D, int c,
                                               const double* theta, const double* gs,
                                               double* g) {
  const int np = A.np, n = A.n_prior;
  for (int j = 0; j < np; ++j) g[j] = gs[j];
  const size_t o = (size_t)c * (size_t)(n > 0 ? n : 1);
  return prior_value_grad_tape(A.prior_code, n, A.prior_consts, theta, g, D.tvals + o,
                               D.tadj + o, D.tlhs + o, D.trhs + o);
}

__device__ __forceinline__ double da_uniform(Stream& rs, uint32_t t, uint32_t k) {
  if (rs.kind == RNG_TRIPLE32) return rs.next();
  rs.it = t;
  rs.k = k;
  return rs.next();
}

// After the exact start (PH_INIT): the prior at each state, zero counters.
// With the Langevin proposal (A.mode == MODE_MALA; the start ran with a
// symmetric mode) also the surrogate log-posterior gradient at each state
// (D.gs holds the surrogate's data-term gradient there), and every chain
// draws its first proposal again, now with that drift.
static __global__ void da_setup_kernel(ChainArgs A, DaArgs D) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c == 0) D.iter[0] = 0;
  if (c >= A.n_chains) return;
  const double* x = A.state + (size_t)c * A.np;
  if (A.mode == MODE_MALA) {
    if (D.prior_ready) {
      for (int j = 0; j < A.np; ++j) A.gx[(size_t)c * A.np + j] = D.gs[(size_t)c * A.np + j];
    } else {
      D.prior_x[c] =
          da_post_grad(A, D, c, x, D.gs + (size_t)c * A.np, A.gx + (size_t)c * A.np);
    }
    if (A.n_iter > 0) {
      Stream rs = make_stream(A, c);
      rs.it = 0;
      rs.k = 0x20000000u;  // counters apart from the start's own proposal
      propose(A, c, rs, D.full, D.C_pad);
      A.ctr[c] = rs.ctr;
    }
  } else if (!D.prior_ready) {
    D.prior_x[c] = InterpPrior::value(A, c, x);
  }
  D.stage1[c] = 0;
}

// Stage 1 on the surrogate.  With the Langevin proposal the ratio carries
// q(x | y) / q(y | x) of the surrogate-driven drift (the reverse drift from
// the surrogate log-posterior gradient at y, capped as the forward one;
// cpu_native.rs:704-710 for the exact-gradient form), and the surrogate
// log posterior at y must be finite (cpu_native.rs:713-714).
static __global__ void da_stage1_kernel(ChainArgs A, DaArgs D) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.n_chains) return;
  const uint32_t t = D.iter[0];
  const int np = A.np;
  const double* y = A.prop + (size_t)c * np;
  double py, lqd = 0.0;
  if (A.mode == MODE_MALA) {
    double* gy = A.gy + (size_t)c * np;
    if (D.prior_ready) {
      py = D.prior_y[c];
      for (int j = 0; j < np; ++j) gy[j] = D.gs[(size_t)c * np + j];
    } else {
      py = da_post_grad(A, D, c, y, D.gs + (size_t)c * np, gy);
    }
    const double* sd = A.sd + (size_t)c * np;
    const double* L = A.L ? A.L + (size_t)c * np * np : nullptr;
    double* my = A.my + (size_t)c * np;
    double* tmp = A.vbuf + (size_t)c * np;
    half_m_times(np, sd, L, gy, my, tmp);
    for (int j = 0; j < np; ++j) my[j] += y[j];
    lqd = log_q(np, sd, L, A.state + (size_t)c * np, my, tmp) -
          log_q(np, sd, L, y, A.mx + (size_t)c * np, tmp);
  } else {
    py = D.prior_ready ? D.prior_y[c] : InterpPrior::value(A, c, y);
  }
  D.prior_y[c] = py;
  Stream rs = make_stream(A, c);
  const double u = da_uniform(rs, t, 0xFFFF0001u);
  const double a1 = ((D.sll_y[c] + py) - (D.sll_x[c] + D.prior_x[c])) / A.temp[c] + lqd;
  const bool finite = A.mode != MODE_MALA || isfinite(D.sll_y[c] + py);
  D.flag[c] = (finite && log(u) < a1) ? 1u : 0u;
  A.ctr[c] = rs.ctr;
}

// Deterministic compaction: one block scans the flags in chain order.
static __global__ void da_compact_kernel(ChainArgs A, DaArgs D) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < A.n_chains; base += blockDim.x) {
    const int c = base + tid;
    const uint32_t f = c < A.n_chains ? D.flag[c] : 0u;
    uint32_t incl = f;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += v;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const int nw = blockDim.x >> 5;
      uint32_t ws = lane < nw ? warp_sums[lane] : 0u;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, ws, off);
        if (lane >= off) ws += v;
      }
      if (lane < nw) warp_sums[lane] = ws;  // inclusive warp prefix
    }
    __syncthreads();
    const uint32_t before = carry + (warp > 0 ? warp_sums[warp - 1] : 0u) + incl - f;
    if (c < A.n_chains) D.slot[c] = before;
    __syncthreads();
    if (tid == blockDim.x - 1) carry += warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
  }
  if (tid == 0) D.active[0] = carry;
}

// Stage-1 survivors' proposals into the compacted f32 evaluation array.
static __global__ void da_pack_kernel(ChainArgs A, DaArgs D) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)A.n_chains * A.np) return;
  const int c = (int)(i / A.np), j = (int)(i % A.np);
  if (!D.flag[c]) return;
  D.params[(size_t)j * D.C_pad + D.slot[c]] = (float)A.prop[i];
}

// The i-th uniform (i >= 1) a chain's stream `rs` would return from its
// current position, without advancing it: both streams are counter-based, so
// the lanes of a warp can draw a chain's normals in parallel.
__device__ __forceinline__ double stream_at(const Stream& rs, uint32_t i) {
  if (rs.kind == RNG_TRIPLE32) return t32_uniform(rs.seedmix, rs.ctr + i);
  const U4 r = philox4x32_10(U4{rs.k + i - 1u, rs.it, rs.chain, 0xB2000001u}, rs.seed,
                             0x6A09E667u);
  return u53(r.x, r.y);
}
__device__ __forceinline__ double stream_normal_at(const Stream& rs, uint32_t i0, int j) {
  const double u1 = stream_at(rs, i0 + 2u * (uint32_t)j + 1u);
  const double u2 = stream_at(rs, i0 + 2u * (uint32_t)j + 2u);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

// propose() for chain c by the 32 lanes of a warp: the same draws, the same
// arithmetic per coordinate (each lane runs one coordinate's loops in the
// serial order; the drift norm is summed by lane 0 in coordinate order), so
// the proposal equals the serial one bit for bit.  `sm` is this warp's
// scratch of 2 np doubles.  Returns the stream advanced past the draws.
__device__ inline Stream propose_warp(const ChainArgs& A, int c, Stream rs, float* params,
                                      int C_pad, int lane, double* sm) {
  const int np = A.np;
  const double* x = A.state + (size_t)c * np;
  double* y = A.prop + (size_t)c * np;
  const double* sd = A.sd + (size_t)c * np;
  const double* L = A.L ? A.L + (size_t)c * np * np : nullptr;
  uint32_t used = 2u * (uint32_t)np;
  if (A.mode == MODE_RWM) {
    for (int j = lane; j < np; j += 32) y[j] = x[j] + sd[j] * stream_normal_at(rs, 0, j);
  } else if (A.mode == MODE_CHOL || A.mode == MODE_MALA) {
    double* z = sm;
    double* base = sm + np;
    if (A.mode == MODE_MALA) {
      // mean = x + f (1/2) M g (half_m_times, cpu_native.rs:617-651)
      const double* gx = A.gx + (size_t)c * np;
      double* tmp = z;  // reused for z below, after the mean is built
      for (int j = lane; j < np; j += 32) {
        double acc = 0.0;
        if (!L) {
          tmp[j] = 0.5 * sd[j] * gx[j];
        } else {
          for (int k = j; k < np; ++k) acc += L[(size_t)k * np + j] * gx[k];
          tmp[j] = 0.5 * acc;
        }
      }
      __syncwarp();
      double f = 1.0;
      if (lane == 0) {
        double ss = 0.0;
        for (int j = 0; j < np; ++j) ss += tmp[j] * tmp[j];
        const double norm = sqrt(ss), dmax = 2.0 * sqrt((double)np);
        f = norm > dmax ? dmax / norm : 1.0;
      }
      f = __shfl_sync(0xffffffffu, f, 0);
      double* mx = A.mx + (size_t)c * np;
      for (int k = lane; k < np; k += 32) {
        double out;
        if (!L) {
          out = f * sd[k] * tmp[k];
        } else {
          double acc = 0.0;
          for (int j = 0; j <= k; ++j) acc += L[(size_t)k * np + j] * tmp[j];
          out = f * acc;
        }
        mx[k] = out + x[k];
        base[k] = mx[k];
      }
    } else {
      for (int k = lane; k < np; k += 32) base[k] = x[k];
    }
    __syncwarp();
    for (int j = lane; j < np; j += 32) z[j] = stream_normal_at(rs, 0, j);
    __syncwarp();
    for (int k = lane; k < np; k += 32) {
      if (L) {
        double acc = base[k];
        for (int j = 0; j <= k; ++j) acc += L[(size_t)k * np + j] * z[j];
        y[k] = acc;
      } else {
        y[k] = base[k] + sd[k] * z[k];
      }
    }
  } else {  // DE on the snapshot
    const int n = A.n_chains;
    int a = (int)(stream_at(rs, 1) * (double)n);
    if (a >= n) a = n - 1;
    int b = (int)(stream_at(rs, 2) * (double)n);
    if (b >= n) b = n - 1;
    if (b == a) b = (b + 1) % n;
    const double g = stream_at(rs, 3) < 0.1 ? 1.0 : A.gamma;
    const double* pa = A.snap + (size_t)a * np;
    const double* pb = A.snap + (size_t)b * np;
    for (int j = lane; j < np; j += 32) {
      const double zj = stream_normal_at(rs, 3, j);
      const double diff = pa[j] - pb[j];
      y[j] = x[j] + g * diff + A.de_noise * sd[j] * zj;
    }
    used += 3u;
  }
  for (int j = lane; j < np; j += 32) params[(size_t)j * C_pad + c] = (float)y[j];
  __syncwarp();
  if (rs.kind == RNG_TRIPLE32) rs.ctr += used;
  else rs.k += used;
  return rs;
}

// Stage 2 for the survivors, the draw for every chain, the next proposal.
// One warp per chain: the lanes add the chain's observation-block partials in
// a fixed lane-strided order and a fixed shuffle tree (deterministic), lane 0
// takes the decision, and the lanes copy, record and propose in parallel.
static __global__ void da_finalize_kernel(ChainArgs A, DaArgs D, const double* __restrict__ partials,
                                          int CG, int total, int ntiles, int C_pad_eval) {
  const int c = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= A.n_chains) return;
  const bool live = D.flag[c] != 0;
  double ll = 0.0;
  if (live) {
    int tpc = 0;
    const int nob = da_obs_blocks((int)D.active[0], CG, total, ntiles, &tpc);
    const uint32_t k = D.slot[c];
    for (int o = lane; o < nob; o += 32) ll += partials[(size_t)o * C_pad_eval + k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) ll += __shfl_xor_sync(0xffffffffu, ll, off);
  }
  extern __shared__ double fin_sm[];  // [warps per block][2 np]
  const int np = A.np;
  const uint32_t t = D.iter[0];
  double* x = A.state + (size_t)c * np;
  const double* y = A.prop + (size_t)c * np;
  Stream rs = make_stream(A, c);
  int take = 0;
  if (live) {
    if (lane == 0) {
      const double plp = ll + D.prior_y[c];
      A.last_eval[c] = plp;
      const double u = da_uniform(rs, t, 0xFFFF0002u);
      const double llx = A.cur[c] - D.prior_x[c];
      const double a2 = ((ll - llx) - (D.sll_y[c] - D.sll_x[c])) / A.temp[c];
      take = log(u) < a2 ? 1 : 0;
      if (take) {
        A.cur[c] = plp;
        D.sll_x[c] = D.sll_y[c];
        D.prior_x[c] = D.prior_y[c];
        A.accepts[c] += 1;
      }
      D.stage1[c] += 1;
    } else if (rs.kind == RNG_TRIPLE32) {
      rs.ctr += 1;  // the stage-2 uniform lane 0 drew
    }
    take = __shfl_sync(0xffffffffu, take, 0);
    if (take) {
      for (int j = lane; j < np; j += 32) x[j] = y[j];
      if (A.mode == MODE_MALA) {  // the drift of the new state
        double* gx = A.gx + (size_t)c * np;
        const double* gy = A.gy + (size_t)c * np;
        for (int j = lane; j < np; j += 32) gx[j] = gy[j];
      }
    }
    __syncwarp();
  }
  if (t < A.n_iter)
    for (int j = lane; j < np; j += 32) A.draws[((size_t)t * np + j) * D.C_pad + c] = (float)x[j];
  __syncwarp();
  if (t + 1 < A.n_iter) {
    rs.it = t + 1;
    rs.k = 0;
    rs = propose_warp(A, c, rs, D.full, D.C_pad, lane, fin_sm + (size_t)(threadIdx.x >> 5) * 2 * np);
  }
  if (lane == 0) A.ctr[c] = rs.ctr;
}

static __global__ void da_tick_kernel(DaArgs D) {
  if (threadIdx.x == 0 && blockIdx.x == 0) D.iter[0] += 1;
}

}  // namespace gpum
