// kernels.cuh -- the B200 hot path: the fused per-iteration evaluation +
// accept/propose kernel, and its helpers.
//
// One launch of `iter_kernel` is one Metropolis iteration for every chain
// (the reference runs the whole chain inside one CTA per chain,
// src/rust/src/chain_kernel.rs:123-357; here the data sum of every chain is
// spread over the whole GPU instead):
//   grid.x = observation blocks, grid.y = chain blocks of CG chains;
//   each CTA streams its observation tiles through shared memory with TMA
//   (double-buffered, mbarrier completion) and runs the interpreter for its
//   CG chains on every observation, so one tile read serves CG chains;
//   per-thread compensated FP32 sums -> FP64 warp-shuffle tree -> FP64 CTA
//   sum in fixed order -> FP64 partial per (obs block, chain);
//   the last CTA of a chain block to finish (atomic ticket, no spinning) sums
//   the partials in fixed obs-block order, adds the f64 prior, makes the
//   tempered f64 accept decision, records the draw and draws the next
//   proposal (diagonal / Cholesky RWM, DE).  Results are deterministic.
#pragma once
#include "interp.cuh"

namespace gpum {

constexpr int kWarps = 8;              // warps per CTA
constexpr int kThreads = kWarps * 32;

enum Phase : int { PH_EVAL = 0, PH_INIT = 1, PH_STEP = 2, PH_POINTWISE = 3 };
enum RngKind : int { RNG_TRIPLE32 = 0, RNG_PHILOX = 1 };

// Chain state of a run, all device pointers.
struct ChainArgs {
  int n_chains, np;
  double* state;        // [C][np]
  double* prop;         // [C][np]
  double* cur;          // [C]   current log posterior (untempered)
  double* last_eval;    // [C]   log posterior of the latest evaluated point
  uint32_t* ctr;        // [C]   triple32 counters
  uint32_t* accepts;    // [C]
  uint32_t* iter;       // [NCB] iterations done, per chain block
  const double* sd;     // [C][np]
  const double* temp;   // [C]
  const double* L;      // [C][np][np] row-major lower factors, or nullptr
  const double* snap;   // [C][np] DE pool snapshot (batch start states)
  float* draws;         // [n_iter][np][C_pad] internal layout
  uint32_t n_iter;
  uint32_t seed;
  int mode;             // 0 diag RWM, 1 DE, 2 Cholesky RWM
  int rng;              // RngKind
  double gamma, de_noise;
  const uint32_t* prior_code;   // f64-interpreted prior (validated)
  const double* prior_consts;
  int n_prior;
  double* zbuf;         // [C][np] scratch for the Cholesky proposal
};

struct EvalArgs {
  int n_obs, ncols, T, ntiles, tiles_per_cta, CG, WC, C_pad, np;
  const float* params;  // [np][C_pad] evaluation points (f32)
  double* partials;     // [NOB][C_pad]
  double* pointwise;    // [C][n_obs] (PH_POINTWISE)
  int n_points;         // chains/points that are real (rest padding)
  uint32_t* tickets;    // [NCB]
  uint32_t* err;        // device error word
};

// ---------------------------------------------------------- f64 prior
// The prior is a handful of ops once per chain per iteration; it is
// interpreted in f64 from the source bytecode (semantics of
// src/rust/src/cpu_native.rs:80-107) so the prior term carries no f32 error.
__device__ inline double prior_eval(const uint32_t* __restrict__ code, int n,
                                    const double* __restrict__ cst,
                                    const double* __restrict__ p) {
  if (n == 0) return 0.0;
  double st[kMaxStack];
  int sp = 0;
  for (int pc = 0; pc < n; ++pc) {
    const uint32_t op = code[2 * pc], a = code[2 * pc + 1];
    switch (op) {
      case 0: st[sp++] = cst[a]; break;
      case 1: st[sp++] = p[a]; break;
      case 2: st[sp++] = 0.0; break;  // rejected by validation
      case 3: st[sp - 2] += st[sp - 1]; --sp; break;
      case 4: st[sp - 2] -= st[sp - 1]; --sp; break;
      case 5: st[sp - 2] *= st[sp - 1]; --sp; break;
      case 6: st[sp - 2] /= st[sp - 1]; --sp; break;
      case 7: st[sp - 1] = -st[sp - 1]; break;
      case 8: st[sp - 1] = exp(st[sp - 1]); break;
      case 9: st[sp - 1] = log(st[sp - 1]); break;
      case 10: st[sp - 1] = sqrt(st[sp - 1]); break;
      case 12: st[sp - 1] = lgamma(st[sp - 1]); break;
      default: st[sp - 2] = pow(st[sp - 2], st[sp - 1]); --sp; break;
    }
  }
  return st[0];
}

// ------------------------------------------------------- uniform streams
struct Stream {
  int kind;
  uint32_t seedmix;     // triple32: hash(seed) + chain * 2654435761
  uint32_t ctr;         // triple32 counter
  uint32_t seed, chain, it, k;  // philox counter fields
  __device__ __forceinline__ double next() {
    if (kind == RNG_TRIPLE32) {
      ctr += 1;
      return t32_uniform(seedmix, ctr);
    }
    const U4 r = philox4x32_10(U4{k++, it, chain, 0xB2000001u}, seed, 0x6A09E667u);
    return u53(r.x, r.y);
  }
  __device__ __forceinline__ double normal() {
    const double u1 = next();
    const double u2 = next();
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  }
};

// Draw the next proposal of chain c into prop (f64) and params (f32).
// Diagonal RWM chain_kernel.rs:212-223 / cpu_native.rs:726-735; Cholesky
// RWM :224-249 / :736-753; DE on the frozen snapshot :250-295 / :754-784.
__device__ inline void propose(const ChainArgs& A, int c, Stream& rs, float* params,
                               int C_pad) {
  const int np = A.np;
  const double* x = A.state + (size_t)c * np;
  double* y = A.prop + (size_t)c * np;
  const double* sd = A.sd + (size_t)c * np;
  if (A.mode == 0) {
    for (int j = 0; j < np; ++j) y[j] = x[j] + sd[j] * rs.normal();
  } else if (A.mode == 2) {
    double* z = A.zbuf + (size_t)c * np;
    for (int j = 0; j < np; ++j) z[j] = rs.normal();
    const double* L = A.L + (size_t)c * np * np;
    for (int k = 0; k < np; ++k) {
      double acc = x[k];
      for (int j = 0; j <= k; ++j) acc += L[(size_t)k * np + j] * z[j];
      y[k] = acc;
    }
  } else {
    const int n = A.n_chains;
    int a = (int)(rs.next() * (double)n);
    if (a >= n) a = n - 1;
    int b = (int)(rs.next() * (double)n);
    if (b >= n) b = n - 1;
    if (b == a) b = (b + 1) % n;
    const double g = rs.next() < 0.1 ? 1.0 : A.gamma;
    const double* pa = A.snap + (size_t)a * np;
    const double* pb = A.snap + (size_t)b * np;
    for (int j = 0; j < np; ++j) {
      const double z = rs.normal();
      const double diff = pa[j] - pb[j];
      y[j] = x[j] + g * diff + A.de_noise * sd[j] * z;
    }
  }
  for (int j = 0; j < np; ++j) params[(size_t)j * C_pad + c] = (float)y[j];
}

// Accept/reject + record + propose for chain c with data-term sum `ll`.
__device__ inline void finalize_chain(const ChainArgs& A, int c, int cb, double ll, int phase,
                                      float* params, int C_pad) {
  const int np = A.np;
  const uint32_t t = A.iter[cb];
  Stream rs;
  rs.kind = A.rng;
  rs.seedmix = triple32(A.seed) + (uint32_t)c * 2654435761u;
  rs.ctr = A.ctr[c];
  rs.seed = A.seed;
  rs.chain = (uint32_t)c;
  if (phase == PH_INIT) {
    const double lp = ll + prior_eval(A.prior_code, A.n_prior, A.prior_consts,
                                      A.state + (size_t)c * np);
    A.cur[c] = lp;
    A.last_eval[c] = lp;
    if (A.n_iter > 0) {
      rs.it = 0;
      rs.k = 0;
      propose(A, c, rs, params, C_pad);
    }
  } else {
    const double* y = A.prop + (size_t)c * np;
    double* x = A.state + (size_t)c * np;
    const double plp = ll + prior_eval(A.prior_code, A.n_prior, A.prior_consts, y);
    A.last_eval[c] = plp;
    double u;
    if (A.rng == RNG_TRIPLE32) {
      u = rs.next();
    } else {
      rs.it = t;
      rs.k = 0xFFFF0000u;
      u = rs.next();
    }
    // Tempered acceptance on the f64 totals (chain_kernel.rs:334,
    // cpu_native.rs:792): ln u < (plp - cur) / T.
    if (log(u) < (plp - A.cur[c]) / A.temp[c]) {
      for (int j = 0; j < np; ++j) x[j] = y[j];
      A.cur[c] = plp;
      A.accepts[c] += 1;
    }
    if (t < A.n_iter) {
      for (int j = 0; j < np; ++j)
        A.draws[((size_t)t * np + j) * C_pad + c] = (float)x[j];
    }
    if (t + 1 < A.n_iter) {
      rs.it = t + 1;
      rs.k = 0;
      propose(A, c, rs, params, C_pad);
    }
  }
  A.ctr[c] = rs.ctr;
}

// ------------------------------------------------------------ the kernel
template <int G, int D>
__global__ void __launch_bounds__(kThreads, 2)
iter_kernel(const __grid_constant__ EvalProg prog, const __grid_constant__ CUtensorMap tmap,
            EvalArgs E, ChainArgs A, int phase) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int CG = E.CG, T = E.T, ncols = E.ncols, np = E.np;
  const int cb = blockIdx.y, ob = blockIdx.x;
  const int WO = kWarps / E.WC;
  const int wc = warp % E.WC, wo = warp / E.WC;

  // Shared-memory carve-up (smem_bytes() on the host must agree):
  // 2 data stages | params [np][CG] | reduction [8][G] f64 | 2 mbarriers | ticket.
  const size_t stage_floats = (size_t)T * ncols;
  float* xs = reinterpret_cast<float*>(smem_raw);
  float* psm = xs + 2 * stage_floats;
  double* red = reinterpret_cast<double*>(psm + (((size_t)np * CG + 3) & ~(size_t)3));
  uint64_t* bars = reinterpret_cast<uint64_t*>(red + kWarps * G);
  uint32_t* s_ticket = reinterpret_cast<uint32_t*>(bars + 2);

  // Parameters of this CTA's chains (coalesced rows of the [np][C_pad] array).
  for (int i = tid; i < np * CG; i += kThreads) {
    const int p = i / CG, cl = i % CG;
    psm[i] = E.params[(size_t)p * E.C_pad + (size_t)cb * CG + cl];
  }

  const int t0 = ob * E.tiles_per_cta;
  const int t1 = min(t0 + E.tiles_per_cta, E.ntiles);
  const int nt = max(t1 - t0, 0);
  const uint32_t tile_bytes = (uint32_t)(stage_floats * sizeof(float));
  // No tiles (or no data columns): the tensor map is never touched.
  const bool staged = ncols > 0 && nt > 0;
  if (tid == 0 && staged) {
    tma_prefetch_desc(&tmap);
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0 && staged) {
    for (int s = 0; s < 2 && s < nt; ++s) {
      mbar_expect_tx(&bars[s], tile_bytes);
      tma_load_2d(xs + s * stage_floats, &tmap, &bars[s], (t0 + s) * T, 0);
    }
  }

  Comp acc[G];
#pragma unroll
  for (int g = 0; g < G; ++g) acc[g].init();
  const float* pc0 = psm + wc * G;
  float s[D][G];

  for (int k = 0; k < nt; ++k) {
    const int st = k & 1;
    const float* tile = xs + st * stage_floats;
    if (staged && !mbar_wait_bounded(&bars[st], (uint32_t)((k >> 1) & 1))) {
      if (lane == 0) atomicOr(E.err, DEV_ERR_TMA_TIMEOUT);
    }
    const int obs0 = (t0 + k) * T;
    for (int ol = lane + 32 * wo; ol < T; ol += 32 * WO) {
      const int obs = obs0 + ol;
      interp_run<G, D>(prog, s, tile + ol, T, pc0, CG);
      if (phase == PH_POINTWISE) {
        if (obs < E.n_obs) {
#pragma unroll
          for (int g = 0; g < G; ++g) {
            const int c = cb * CG + wc * G + g;
            if (c < E.n_points) E.pointwise[(size_t)c * E.n_obs + obs] = (double)s[0][g];
          }
        }
      } else if (obs < E.n_obs) {
#pragma unroll
        for (int g = 0; g < G; ++g) acc[g].add(s[0][g]);
      }
    }
    __syncthreads();  // every warp is done with this stage
    if (tid == 0 && staged && k + 2 < nt) {
      mbar_expect_tx(&bars[st], tile_bytes);
      tma_load_2d(xs + st * stage_floats, &tmap, &bars[st], (t0 + k + 2) * T, 0);
    }
  }
  if (phase == PH_POINTWISE) return;

  // FP64 fixed-order reduction: lanes (shuffle tree), then the WO warps that
  // share a chain group, in warp order.
  double tot[G];
#pragma unroll
  for (int g = 0; g < G; ++g) tot[g] = acc[g].total();
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int g = 0; g < G; ++g) tot[g] += __shfl_down_sync(0xffffffffu, tot[g], off);
  }
  if (lane == 0) {
#pragma unroll
    for (int g = 0; g < G; ++g) red[warp * G + g] = tot[g];
  }
  __syncthreads();
  if (tid < CG) {
    const int wcc = tid / G, g = tid % G;
    double v = 0.0;
    for (int o = 0; o < WO; ++o) v += red[(o * E.WC + wcc) * G + g];
    E.partials[(size_t)ob * E.C_pad + (size_t)cb * CG + tid] = v;
  }
  if (phase == PH_EVAL) return;

  // Last CTA of this chain block (ticket) finishes the iteration.
  __threadfence();
  __syncthreads();
  if (tid == 0) *s_ticket = atomicAdd(&E.tickets[cb], 1u);
  __syncthreads();
  const uint32_t nob = gridDim.x;
  if (*s_ticket != nob - 1) return;
  __threadfence();
  for (int cl = tid; cl < CG; cl += kThreads) {
    const int c = cb * CG + cl;
    if (c >= A.n_chains) continue;
    double ll = 0.0;
    for (uint32_t o = 0; o < nob; ++o)
      ll += __ldcg(&E.partials[(size_t)o * E.C_pad + c]);
    finalize_chain(A, c, cb, ll, phase, const_cast<float*>(E.params), E.C_pad);
  }
  __syncthreads();
  if (tid == 0) {
    E.tickets[cb] = 0;
    if (phase == PH_STEP) A.iter[cb] += 1;
  }
}

// ------------------------------------------------------------- helpers
// Row-major f64 rows [r0, r0+nr) -> column-major f32 [ncols][ld].
__global__ void convert_rows_kernel(const double* __restrict__ src, float* __restrict__ dst,
                                    int ncols, int64_t ld, int64_t r0, int64_t nr) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr * ncols) return;
  const int64_t r = i / ncols, j = i % ncols;
  dst[(int64_t)j * ld + r0 + r] = (float)src[i];
}

// f64 chain-major points [C][np] -> f32 [np][C_pad]; pad chains copy chain 0.
__global__ void points_to_params_kernel(const double* __restrict__ pts, float* __restrict__ params,
                                        int n, int np, int C_pad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np * C_pad) return;
  const int j = i / C_pad, c = i % C_pad;
  const int src = c < n ? c : 0;
  params[i] = (float)pts[(size_t)src * np + j];
}

// Fixed-order sum of the partials of each point.
__global__ void reduce_partials_kernel(const double* __restrict__ partials, double* __restrict__ out,
                                       int nob, int C_pad, int n) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  double v = 0.0;
  for (int o = 0; o < nob; ++o) v += partials[(size_t)o * C_pad + c];
  out[c] = v;
}

// Internal draws [n_iter][np][C_pad] -> the reference layout, column-major
// (n_iter, C, np): out[t + n_iter*(c + C*j)] (chain_kernel.rs:345).
__global__ void draws_layout_kernel(const float* __restrict__ in, float* __restrict__ out,
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
    if (t < n_iter && c < C) out[(size_t)t + (size_t)n_iter * ((size_t)c + (size_t)C * j)] =
        tile[threadIdx.x][r];
  }
}

}  // namespace gpum
