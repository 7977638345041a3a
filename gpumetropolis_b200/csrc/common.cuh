// common.cuh -- the per-iteration kernel skeleton shared by the interpreter
// and the compiled (NVRTC) evaluation bodies, plus the accept/propose logic.
//
// One launch = one Metropolis iteration for every chain (the reference runs
// a whole chain inside one CTA, src/rust/src/chain_kernel.rs:123-357; here
// the data sum of every chain is spread over the whole GPU):
//   grid.x = chain blocks of CG chains, grid.y = observation blocks;
//   each CTA streams its observation tiles through shared memory with TMA
//   (double-buffered, mbarrier completion, bounded waits) and evaluates its
//   CG chains on every observation, so one tile read serves CG chains;
//   per-thread compensated FP32 sums -> FP64 warp-shuffle tree -> FP64 sum
//   over warps in fixed order -> FP64 partial per (obs block, chain, value);
//   the last CTA of a chain block (atomic ticket, no spinning) sums the
//   partials in obs-block order, adds the f64 prior, makes the tempered f64
//   accept decision, records the draw and draws the next proposal.
// Results are deterministic for a given launch geometry.
#pragma once
#include "device.cuh"

namespace gpum {

constexpr int kWarps = 8;  // warps per CTA
constexpr int kThreads = kWarps * 32;
// The tensor-core value kernel (gm_iter_value_tc): 128 chains per CTA (the
// MMA's M); its epilogue warps (a multiple of four, GenModel::tc_warps) and
// one control warp.
constexpr int kTcM = 128;
constexpr int kMaxStackF64 = 32;

enum Phase : int { PH_EVAL = 0, PH_INIT = 1, PH_STEP = 2, PH_POINTWISE = 3 };
enum RngKind : int { RNG_TRIPLE32 = 0, RNG_PHILOX = 1 };
enum ModeKind : int { MODE_RWM = 0, MODE_DE = 1, MODE_CHOL = 2, MODE_MALA = 3, MODE_DESYNC = 4 };

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
  int mode;             // ModeKind
  int rng;              // RngKind
  double gamma, de_noise;
  const uint32_t* prior_code;   // f64-interpreted prior (validated)
  const double* prior_consts;
  int n_prior;
  double* zbuf;         // [C][np] scratch: normals
  // MALA (mode 3)
  double* gx;           // [C][np] gradient of the log posterior at `state`
  double* gy;           // [C][np] gradient at `prop`
  double* mx;           // [C][np] proposal mean from `state`
  double* my;           // [C][np] proposal mean from `prop`
  double* vbuf;         // [C][np] scratch
  // Training pairs for the surrogate: every exactly evaluated proposal's
  // (theta, data-term log-likelihood), slot rec_base + t*C + c (< rec_cap).
  float* rec_theta;     // [rec_cap][np] or nullptr
  double* rec_ll;       // [rec_cap]
  uint64_t rec_base, rec_cap;
  // Power posteriors (thermodynamic integration): chain c targets
  // beta[c] * loglik + prior; nullptr means beta = 1.
  const double* beta;
  // The interpreted prior's gradient (MALA on the interpreter engine): per
  // chain a tape of n_prior values, adjoints and operand indices.
  double* ptape;        // [C][2][n_prior]
  uint32_t* ptape_i;    // [C][2][n_prior]
};

struct EvalArgs {
  int n_obs, ncols, T, ntiles, tiles_per_cta, CG, WC, C_pad, np;
  int width;            // values per (chain, obs block): 1, or 1 + np with the gradient
  const float* params;  // [np][C_pad] evaluation points (f32)
  double* partials;     // [NOB][C_pad][width]
  double* pointwise;    // [C][n_obs] (PH_POINTWISE)
  int n_points;         // chains/points that are real (rest padding)
  uint32_t* tickets;    // [NCB]
  uint32_t* err;        // device error word
  const uint32_t* active;  // if set: only the first *active points are live
};

// Delayed acceptance evaluates the first `live` points of the compacted array
// with a fixed 1-D grid of `total` CTAs, whose split into chain blocks x
// observation blocks is decided on the device from `live`, so the GPU stays
// full whatever stage 1 accepted.  Returns the observation blocks used (0 if
// nothing is live) and the tiles per CTA.
__host__ __device__ inline int da_obs_blocks(int live, int CG, int total, int ntiles, int* tpc) {
  const int busy = (live + CG - 1) / CG;
  if (busy <= 0) {
    *tpc = 0;
    return 0;
  }
  if (ntiles <= 0) {
    *tpc = 0;
    return 1;
  }
  int nob = total / busy;
  nob = nob < 1 ? 1 : (nob > ntiles ? ntiles : nob);
  *tpc = (ntiles + nob - 1) / nob;
  return (ntiles + *tpc - 1) / *tpc;
}

// ------------------------------------------------------ f64 prior, interpreted
// The prior is a handful of ops once per chain per iteration; it is
// interpreted in f64 from the source bytecode (semantics of
// src/rust/src/cpu_native.rs:80-107) so the prior term carries no f32 error.
__device__ inline double prior_interp(const uint32_t* __restrict__ code, int n,
                                      const double* __restrict__ cst,
                                      const double* __restrict__ p) {
  if (n == 0) return 0.0;
  double st[kMaxStackF64];
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
      // x^2 squared exactly: the correctly rounded x*x, which is what the
      // host libm's pow returns for an exponent of 2
      default: {
        const double a = st[sp - 2], b = st[sp - 1];
        st[sp - 2] = b == 2.0 ? a * a : pow(a, b);
        --sp;
        break;
      }
    }
  }
  return st[0];
}

// Value and gradient of the f64 prior by a reverse-mode tape over its
// bytecode (the reference's tape AD, cpu_native.rs:148-279, for a program
// that reads no data): forward pass recording each instruction's value and
// operands, then adjoints in reverse order with the reference's local
// derivatives (POW's exponent term only where the base is positive; LGAMMA's
// derivative the digamma).  The gradient is added into g.  vals/adj/lhs/rhs
// are this chain's scratch of n entries each.  Used by delayed acceptance
// with the Langevin proposal, whose drift needs the prior's gradient in
// either evaluation engine.
__device__ inline double prior_value_grad_tape(const uint32_t* __restrict__ code, int n,
                                               const double* __restrict__ cst,
                                               const double* __restrict__ p, double* g,
                                               double* vals, double* adj, uint32_t* lhs,
                                               uint32_t* rhs) {
  if (n == 0) return 0.0;
  uint32_t ist[kMaxStackF64];
  int sp = 0;
  for (int pc = 0; pc < n; ++pc) {
    const uint32_t op = code[2 * pc], a = code[2 * pc + 1];
    if (op <= 2) {
      vals[pc] = op == 0 ? cst[a] : (op == 1 ? p[a] : 0.0);
      lhs[pc] = 0xFFFFFFFFu;
      ist[sp++] = (uint32_t)pc;
    } else if ((op >= 7 && op <= 10) || op == 12) {
      const uint32_t l = ist[sp - 1];
      const double x = vals[l];
      vals[pc] = op == 7 ? -x : op == 8 ? exp(x) : op == 9 ? log(x) : op == 10 ? sqrt(x)
                                                                                  : lgamma(x);
      lhs[pc] = l;
      rhs[pc] = 0xFFFFFFFFu;
      ist[sp - 1] = (uint32_t)pc;
    } else {
      const uint32_t r = ist[sp - 1], l = ist[sp - 2];
      const double a0 = vals[l], b0 = vals[r];
      vals[pc] = op == 3 ? a0 + b0 : op == 4 ? a0 - b0 : op == 5 ? a0 * b0 : op == 6 ? a0 / b0
                                                      : (b0 == 2.0 ? a0 * a0 : pow(a0, b0));
      lhs[pc] = l;
      rhs[pc] = r;
      ist[sp - 2] = (uint32_t)pc;
      --sp;
    }
  }
  const int root = n - 1;
  for (int i = 0; i < n; ++i) adj[i] = 0.0;
  adj[root] = 1.0;
  for (int k = n - 1; k >= 0; --k) {
    const double gk = adj[k];
    if (gk == 0.0) continue;
    const uint32_t op = code[2 * k], arg = code[2 * k + 1];
    const uint32_t l = lhs[k], r = rhs[k];
    switch (op) {
      case 0: case 2: break;
      case 1: g[arg] += gk; break;
      case 3: adj[l] += gk; adj[r] += gk; break;
      case 4: adj[l] += gk; adj[r] -= gk; break;
      case 5: adj[l] += gk * vals[r]; adj[r] += gk * vals[l]; break;
      case 6:
        adj[l] += gk / vals[r];
        adj[r] -= gk * vals[k] / vals[r];
        break;
      case 7: adj[l] -= gk; break;
      case 8: adj[l] += gk * vals[k]; break;
      case 9: adj[l] += gk / vals[l]; break;
      case 10: adj[l] += gk * 0.5 / vals[k]; break;
      case 12: adj[l] += gk * gm_digamma(vals[l]); break;
      default: {
        const double a0 = vals[l], b0 = vals[r];
        adj[l] += gk * b0 * pow(a0, b0 - 1.0);
        if (a0 > 0.0) adj[r] += gk * vals[k] * log(a0);
        break;
      }
    }
  }
  return vals[ist[0]];  // stack slot 0, as the value interpreter returns
}

// ------------------------------------------------------- uniform streams
struct Stream {
  int kind;
  uint32_t seedmix;             // triple32: hash(seed) + chain * 2654435761
  uint32_t ctr;                 // triple32 counter
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

__device__ __forceinline__ Stream make_stream(const ChainArgs& A, int c) {
  Stream rs;
  rs.kind = A.rng;
  rs.seedmix = triple32(A.seed) + (uint32_t)c * 2654435761u;
  rs.ctr = A.ctr[c];
  rs.seed = A.seed;
  rs.chain = (uint32_t)c;
  rs.it = 0;
  rs.k = 0;
  return rs;
}

// -------------------------------------------------------------- MALA helpers
// out = f * (1/2) M g, M = Ls Ls' (or diag sd^2), the whitened drift capped at
// 2 sqrt(d) (MALTA; cpu_native.rs:617-651).
__device__ inline void half_m_times(int np, const double* sd, const double* L, const double* g,
                                    double* out, double* tmp) {
  const double dmax = 2.0 * sqrt((double)np);
  if (!L) {
    for (int j = 0; j < np; ++j) tmp[j] = 0.5 * sd[j] * g[j];
  } else {
    for (int j = 0; j < np; ++j) {
      double acc = 0.0;
      for (int k = j; k < np; ++k) acc += L[(size_t)k * np + j] * g[k];
      tmp[j] = 0.5 * acc;
    }
  }
  double ss = 0.0;
  for (int j = 0; j < np; ++j) ss += tmp[j] * tmp[j];
  const double norm = sqrt(ss);
  const double f = norm > dmax ? dmax / norm : 1.0;
  if (!L) {
    for (int j = 0; j < np; ++j) out[j] = f * sd[j] * tmp[j];
  } else {
    for (int k = 0; k < np; ++k) {
      double acc = 0.0;
      for (int j = 0; j <= k; ++j) acc += L[(size_t)k * np + j] * tmp[j];
      out[k] = f * acc;
    }
  }
}

// -1/2 |Ls^{-1}(v - m)|^2 by forward substitution (cpu_native.rs:655-673).
__device__ inline double log_q(int np, const double* sd, const double* L, const double* v,
                               const double* m, double* tmp) {
  double q = 0.0;
  if (!L) {
    for (int j = 0; j < np; ++j) {
      const double r = (v[j] - m[j]) / sd[j];
      q -= 0.5 * r * r;
    }
  } else {
    for (int k = 0; k < np; ++k) {
      double acc = v[k] - m[k];
      for (int j = 0; j < k; ++j) acc -= L[(size_t)k * np + j] * tmp[j];
      tmp[k] = acc / L[(size_t)k * np + k];
      q -= 0.5 * tmp[k] * tmp[k];
    }
  }
  return q;
}

// ------------------------------------------------------------- proposals
// Next proposal of chain c into prop (f64) and params (f32).
// Diagonal RWM chain_kernel.rs:212-223 / cpu_native.rs:726-735; Cholesky
// RWM :224-249 / :736-753; DE on the frozen snapshot :250-295 / :754-784;
// MALA :681-703 (mean from the cached gradient, then L z or sd * z).
__device__ inline void propose(const ChainArgs& A, int c, Stream& rs, float* params, int C_pad) {
  const int np = A.np;
  const double* x = A.state + (size_t)c * np;
  double* y = A.prop + (size_t)c * np;
  const double* sd = A.sd + (size_t)c * np;
  const double* L = A.L ? A.L + (size_t)c * np * np : nullptr;
  if (A.mode == MODE_RWM) {
    for (int j = 0; j < np; ++j) y[j] = x[j] + sd[j] * rs.normal();
  } else if (A.mode == MODE_CHOL || A.mode == MODE_MALA) {
    double* z = A.zbuf + (size_t)c * np;
    const double* base = x;
    if (A.mode == MODE_MALA) {
      double* mx = A.mx + (size_t)c * np;
      half_m_times(np, sd, L, A.gx + (size_t)c * np, mx, A.vbuf + (size_t)c * np);
      for (int j = 0; j < np; ++j) mx[j] += x[j];
      base = mx;
    }
    for (int j = 0; j < np; ++j) z[j] = rs.normal();
    if (L) {
      for (int k = 0; k < np; ++k) {
        double acc = base[k];
        for (int j = 0; j <= k; ++j) acc += L[(size_t)k * np + j] * z[j];
        y[k] = acc;
      }
    } else {
      for (int j = 0; j < np; ++j) y[j] = base[j] + sd[j] * z[j];
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

// Synchronous per-generation DE (path B, cpu_native.rs:400-506): the
// difference vector comes from the current population, so this runs in its
// own kernel after every chain's previous accept.  Partners a != c and
// b != c, a (cpu_native.rs:430-440); g = 1 with probability 0.1, else gamma.
__device__ inline void propose_desync(const ChainArgs& A, int c, Stream& rs, float* params,
                                      int C_pad) {
  const int n = A.n_chains, np = A.np;
  int a = (int)(rs.next() * (double)n);
  if (a >= n) a = n - 1;
  if (a == c) a = (a + 1) % n;
  int b = (int)(rs.next() * (double)n);
  if (b >= n) b = n - 1;
  while (b == c || b == a) b = (b + 1) % n;  // n >= 3 is checked by the host
  const double g = rs.next() < 0.1 ? 1.0 : A.gamma;
  const double* x = A.state + (size_t)c * np;
  const double* pa = A.state + (size_t)a * np;
  const double* pb = A.state + (size_t)b * np;
  const double* sd = A.sd + (size_t)c * np;
  double* y = A.prop + (size_t)c * np;
  for (int j = 0; j < np; ++j) {
    const double z = rs.normal();
    y[j] = x[j] + g * (pa[j] - pb[j]) + A.de_noise * sd[j] * z;
    params[(size_t)j * C_pad + c] = (float)y[j];
  }
}

// Accept/reject + record + propose for chain c.  `ll` is the data-term sum;
// with MALA the data-term gradient has been summed into A.gy (STEP) or A.gx
// (INIT).  Prior::value(A, c, p) and Prior::value_grad(A, c, p, g) give the
// f64 prior of chain c's point p (value_grad accumulates into g).
template <class Prior>
__device__ inline void finalize_chain(const ChainArgs& A, int c, int cb, double ll, int phase,
                                      float* params, int C_pad) {
  const int np = A.np;
  const uint32_t t = A.iter[cb];
  Stream rs = make_stream(A, c);
  const bool mala = A.mode == MODE_MALA;
  double* x = A.state + (size_t)c * np;
  const double bl = A.beta ? A.beta[c] * ll : ll;  // likelihood power
  if (phase == PH_INIT) {
    const double lp = bl + (mala ? Prior::value_grad(A, c, x, A.gx + (size_t)c * np)
                                 : Prior::value(A, c, x));
    A.cur[c] = lp;
    A.last_eval[c] = lp;
    if (A.n_iter > 0 && A.mode != MODE_DESYNC) {  // path B proposes in its own kernel
      rs.it = 0;
      propose(A, c, rs, params, C_pad);
    }
  } else {
    const double* y = A.prop + (size_t)c * np;
    const double plp = bl + (mala ? Prior::value_grad(A, c, y, A.gy + (size_t)c * np)
                                  : Prior::value(A, c, y));
    A.last_eval[c] = plp;
    if (A.rec_ll) {
      const uint64_t slot = A.rec_base + (uint64_t)t * A.n_chains + c;
      if (slot < A.rec_cap) {
        for (int j = 0; j < np; ++j) A.rec_theta[slot * np + j] = (float)y[j];
        A.rec_ll[slot] = ll;
      }
    }
    double lqd = 0.0;
    if (mala) {
      // q(x | y) - q(y | x) with the truncated drift at y (cpu_native.rs:704-710)
      const double* sd = A.sd + (size_t)c * np;
      const double* L = A.L ? A.L + (size_t)c * np * np : nullptr;
      double* my = A.my + (size_t)c * np;
      double* tmp = A.vbuf + (size_t)c * np;
      half_m_times(np, sd, L, A.gy + (size_t)c * np, my, tmp);
      for (int j = 0; j < np; ++j) my[j] += y[j];
      lqd = log_q(np, sd, L, x, my, tmp) - log_q(np, sd, L, y, A.mx + (size_t)c * np, tmp);
    }
    double u;
    if (A.rng == RNG_TRIPLE32) {
      u = rs.next();
    } else {
      rs.it = t;
      rs.k = 0xFFFF0000u;
      u = rs.next();
    }
    // Tempered acceptance on the f64 totals (chain_kernel.rs:334,
    // cpu_native.rs:792); MALA adds the proposal ratio and requires a
    // finite proposal log density (cpu_native.rs:713-714).
    const bool take = mala ? (isfinite(plp) && log(u) < (plp - A.cur[c]) / A.temp[c] + lqd)
                           : (log(u) < (plp - A.cur[c]) / A.temp[c]);
    if (take) {
      for (int j = 0; j < np; ++j) x[j] = y[j];
      if (mala) {
        double* gx = A.gx + (size_t)c * np;
        const double* gy = A.gy + (size_t)c * np;
        for (int j = 0; j < np; ++j) gx[j] = gy[j];
      }
      A.cur[c] = plp;
      A.accepts[c] += 1;
    }
    if (t < A.n_iter)
      for (int j = 0; j < np; ++j) A.draws[((size_t)t * np + j) * C_pad + c] = (float)x[j];
    if (t + 1 < A.n_iter && A.mode != MODE_DESYNC) {
      rs.it = t + 1;
      rs.k = 0;
      propose(A, c, rs, params, C_pad);
    }
  }
  A.ctr[c] = rs.ctr;
}

// The last CTA of chain block cb to write its partials (an atomic ticket, no
// spinning) finishes the iteration for the block's CG chains: the partials
// summed in observation-block order, then accept/reject, record and
// propose.  Every one of the CTA's nthreads threads calls it.
template <int W, class Prior>
__device__ __forceinline__ void finish_chain_block(const EvalArgs& E, const ChainArgs& A, int cb,
                                                   int CG, int phase, uint32_t* s_ticket,
                                                   int nthreads) {
  const int tid = threadIdx.x, np = E.np;
  __threadfence();
  __syncthreads();
  if (tid == 0) *s_ticket = atomicAdd(&E.tickets[cb], 1u);
  __syncthreads();
  const uint32_t nob = gridDim.y;
  if (*s_ticket != nob - 1) return;
  __threadfence();
  for (int cl = tid; cl < CG; cl += nthreads) {
    const int c = cb * CG + cl;
    if (c >= A.n_chains) continue;
    double ll = 0.0;
    for (uint32_t o = 0; o < nob; ++o) ll += __ldcg(&E.partials[((size_t)o * E.C_pad + c) * W]);
    if (A.mode == MODE_MALA) {
      double* gsum = (phase == PH_INIT ? A.gx : A.gy) + (size_t)c * np;
      const double b = A.beta ? A.beta[c] : 1.0;
      for (int j = 0; j < np; ++j) {
        double v = 0.0;
        for (uint32_t o = 0; o < nob; ++o)
          v += __ldcg(&E.partials[((size_t)o * E.C_pad + c) * W + 1 + j]);
        gsum[j] = b * v;
      }
    }
    finalize_chain<Prior>(A, c, cb, ll, phase, const_cast<float*>(E.params), E.C_pad);
  }
  __syncthreads();
  if (tid == 0) {
    E.tickets[cb] = 0;
    if (phase == PH_STEP) A.iter[cb] += 1;
  }
}

// --------------------------------------------------------- kernel skeleton
// Shared-memory carve-up (the host's smem_bytes() must agree):
//   2 data stages [ncols][T] f32 | params [np][CG] f32 (rounded to 4; none
//   for chain-lane bodies, whose lanes read their parameters from global
//   memory) | reduction [kWarps][G][width] f64 | 2 mbarriers | ticket.
__host__ __device__ inline size_t skel_param_floats(int np, int CG, bool lanes) {
  return lanes ? 0 : (((size_t)np * CG + 3) & ~(size_t)3);
}
__host__ __device__ inline size_t skel_smem_bytes(int T, int ncols, int np, int CG, int G,
                                                  int width, bool lanes = false) {
  return 2 * (size_t)T * ncols * 4 + skel_param_floats(np, CG, lanes) * 4 +
         (size_t)kWarps * G * width * 8 + 2 * 8 + 16;
}

// Body contract (G chains per thread):
//   bool kChainLanes                       false: lanes are observations (below);
//                                          true: lanes are chains, G = 32 counts
//                                          the chains of a warp, and the body has
//                                          begin_lanes(pc, C_pad), eval4(xo, nv),
//                                          last4(k) instead of begin/eval/last
//   bool kLanesAcc (chain lanes)           true: the body accumulates values
//                                          1 .. W-1 in its own row of the
//                                          reduction buffer (begin_lanes_acc(pc,
//                                          C_pad, row), flush_tile() after each
//                                          tile); only value 0 is written here
//   void begin(const float* pc0, int CG)   pc0 = this thread's first chain in
//                                          the [np][CG] parameter tile
//   void eval(const float* xo, int T, bool valid)  one observation
//   float last(int g)                      value of the last eval (pointwise)
//   void end()                             after the last observation
//   double total(int g, int w)             w = 0 value, 1.. gradient entries
//   W (compile time) = E.width values reduced per chain
template <int G, int W, class Body, class Prior>
__device__ __forceinline__ void run_iteration(const TmapDesc* tmap, const EvalArgs& E,
                                              const ChainArgs& A, int phase, Body& body) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int CG = E.CG, T = E.T, ncols = E.ncols, np = E.np;
  // Chain blocks vary fastest, so the CTAs that share an observation tile
  // run in the same wave and read it through L2 once.
  int cb = blockIdx.x, ob = blockIdx.y, tiles_per_cta = E.tiles_per_cta;
  if (E.active) {  // delayed acceptance: geometry from the live count
    const int live = (int)*E.active;
    const int busy = (live + CG - 1) / CG;
    const int nob = da_obs_blocks(live, CG, (int)(gridDim.x * gridDim.y), E.ntiles,
                                  &tiles_per_cta);
    const int id = (int)(blockIdx.y * gridDim.x + blockIdx.x);
    if (busy == 0 || id >= busy * nob) return;
    cb = id % busy;
    ob = id / busy;
  }
  const int WO = kWarps / E.WC;
  const int wc = warp % E.WC, wo = warp / E.WC;

  const size_t stage_floats = (size_t)T * ncols;
  float* xs = reinterpret_cast<float*>(smem_raw);
  constexpr bool kLanes = Body::kChainLanes;
  float* psm = xs + 2 * stage_floats;
  double* red = reinterpret_cast<double*>(psm + skel_param_floats(np, CG, kLanes));
  uint64_t* bars = reinterpret_cast<uint64_t*>(red + (size_t)kWarps * G * W);
  uint32_t* s_ticket = reinterpret_cast<uint32_t*>(bars + 2);

  if constexpr (!kLanes) {
    for (int i = tid; i < np * CG; i += kThreads) {
      const int p = i / CG, cl = i % CG;
      psm[i] = E.params[(size_t)p * E.C_pad + (size_t)cb * CG + cl];
    }
  }

  const int t0 = ob * tiles_per_cta;
  const int t1 = min(t0 + tiles_per_cta, E.ntiles);
  const int nt = max(t1 - t0, 0);
  const uint32_t tile_bytes = (uint32_t)(stage_floats * sizeof(float));
  // No tiles (or no data columns): the tensor map is never touched.
  const bool staged = ncols > 0 && nt > 0;
  if (tid == 0 && staged) {
    tma_prefetch_desc(tmap);
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0 && staged) {
    for (int s = 0; s < 2 && s < nt; ++s) {
      mbar_expect_tx(&bars[s], tile_bytes);
      tma_load_2d(xs + s * stage_floats, tmap, &bars[s], (t0 + s) * T, 0);
    }
  }
  if constexpr (kLanes) {
    const float* pc = E.params + (size_t)cb * CG + (size_t)wc * 32 + lane;
    if constexpr (Body::kLanesAcc)
      body.begin_lanes_acc(pc, E.C_pad, red + ((size_t)warp * G + lane) * W);
    else
      body.begin_lanes(pc, E.C_pad);
  } else {
    body.begin(psm + wc * G, CG);
  }

  for (int k = 0; k < nt; ++k) {
    const int st = k & 1;
    const float* tile = xs + st * stage_floats;
    int gave_up = 0;
    if (staged && !mbar_wait_bounded(&bars[st], (uint32_t)((k >> 1) & 1))) {
      gave_up = 1;
      if (lane == 0) atomicOr(E.err, DEV_ERR_TMA_TIMEOUT);
    }
    const int obs0 = (t0 + k) * T;
    if constexpr (kLanes) {
      // quads of observations (o .. o + 3), the WO warps of a chain group
      // taking every WO-th quad; all lanes read the same addresses
      for (int o = 4 * wo; o < T; o += 4 * WO) {
        const long long left = (long long)E.n_obs - (obs0 + o);
        if (left <= 0) break;
        const int nv = left >= 4 ? 4 : (int)left;
        body.eval4(tile + o, nv);
        if (phase == PH_POINTWISE) {
          const int c = cb * CG + wc * 32 + lane;
          if (c < E.n_points) {
#pragma unroll
            for (int q = 0; q < 4; ++q)  // constant indices keep the values in registers
              if (q < nv) E.pointwise[(size_t)c * E.n_obs + obs0 + o + q] = (double)body.last4(q);
          }
        }
      }
      if constexpr (Body::kLanesAcc) body.flush_tile();
    } else if constexpr (Body::kObsPerEval == 2) {
      // observation pairs (2 pi, 2 pi + 1); T is even, so each pair is
      // 8-byte aligned in every column of the tile
      auto pair = [&](int pi) {
        const int obs = obs0 + 2 * pi;
        const bool v0 = obs < E.n_obs, v1 = obs + 1 < E.n_obs;
        body.eval2(tile + 2 * pi, T, v0, v1);
        if (phase == PH_POINTWISE && v0) {
#pragma unroll
          for (int g = 0; g < G; ++g) {
            const int c = cb * CG + wc * G + g;
            if (c < E.n_points) {
              const float2 lv = body.last2(g);
              E.pointwise[(size_t)c * E.n_obs + obs] = (double)lv.x;
              if (v1) E.pointwise[(size_t)c * E.n_obs + obs + 1] = (double)lv.y;
            }
          }
        }
      };
      constexpr int kT = Body::kTileObs;  // compile-time tile height, or 0
      if (kT > 0 && kT % 64 == 0 && WO == 1) {
        // every warp covers the tile: a fixed trip count, unrolled so the
        // compiler can overlap one pair's loads with another's arithmetic
        bool done = false;
        if constexpr (kT > 0) {
          if (phase != PH_POINTWISE && obs0 + kT <= E.n_obs) {  // a full tile
#pragma unroll
            for (int it = 0; it < kT / 64; ++it) body.eval2_full(tile + 2 * (lane + 32 * it));
            body.flush();
            done = true;
          }
        }
        if (!done) {
#pragma unroll
          for (int it = 0; it < (kT > 0 ? kT : 64) / 64; ++it) pair(lane + 32 * it);
        }
      } else {
        for (int pi = lane + 32 * wo; 2 * pi < T; pi += 32 * WO) pair(pi);
      }
    } else {
      for (int ol = lane + 32 * wo; ol < T; ol += 32 * WO) {
        const int obs = obs0 + ol;
        const bool valid = obs < E.n_obs;
        body.eval(tile + ol, T, valid);
        if (phase == PH_POINTWISE && valid) {
#pragma unroll
          for (int g = 0; g < G; ++g) {
            const int c = cb * CG + wc * G + g;
            if (c < E.n_points) E.pointwise[(size_t)c * E.n_obs + obs] = (double)body.last(g);
          }
        }
      }
    }
    // Every warp is done with this stage.  A wait that gave up anywhere in
    // the CTA (the error bit is set) stops the tile loop for the whole CTA:
    // no more loads are issued, thread 0 waits (bounded) for the loads still
    // in flight into this CTA's stages, and the CTA goes on to the reduction
    // and the ticket so the chain block's bookkeeping stays consistent.
    if (__syncthreads_or(gave_up)) {
      if (tid == 0 && staged) {
        mbar_wait_bounded(&bars[st], (uint32_t)((k >> 1) & 1));
        if (k + 1 < nt) mbar_wait_bounded(&bars[st ^ 1], (uint32_t)(((k + 1) >> 1) & 1));
      }
      __syncthreads();
      break;
    }
    if (tid == 0 && staged && k + 2 < nt) {
      mbar_expect_tx(&bars[st], tile_bytes);
      tma_load_2d(xs + st * stage_floats, tmap, &bars[st], (t0 + k + 2) * T, 0);
    }
  }
  if (phase == PH_POINTWISE) return;
  body.end();

  // FP64 fixed-order reduction of each of the W values: lanes (shuffle
  // tree), then the WO warps that share a chain group, in warp order.
#pragma unroll
  for (int w = 0; w < W; ++w) {
    if constexpr (kLanes) {  // each lane holds its own chain's sum (G == 32)
      if (!Body::kLanesAcc || w == 0) red[((size_t)warp * G + lane) * W + w] = body.total(0, w);
    } else {
      double tot[G];
#pragma unroll
      for (int g = 0; g < G; ++g) tot[g] = body.total(g, w);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
        for (int g = 0; g < G; ++g) tot[g] += __shfl_down_sync(0xffffffffu, tot[g], off);
      }
      if (lane == 0) {
#pragma unroll
        for (int g = 0; g < G; ++g) red[((size_t)warp * G + g) * W + w] = tot[g];
      }
    }
  }
  __syncthreads();
  for (int i = tid; i < CG * W; i += kThreads) {
    const int cl = i / W, w = i % W;
    const int wcc = cl / G, g = cl % G;
    double v = 0.0;
    for (int o = 0; o < WO; ++o) v += red[((size_t)(o * E.WC + wcc) * G + g) * W + w];
    E.partials[((size_t)ob * E.C_pad + (size_t)cb * CG + cl) * W + w] = v;
  }
  if (phase == PH_EVAL) return;
  finish_chain_block<W, Prior>(E, A, cb, CG, phase, s_ticket, kThreads);
}

// Fixed-order sum of the partials of each point: out[p*W + w].
static __global__ void reduce_partials_kernel(const double* __restrict__ partials,
                                       double* __restrict__ out, int nob, int C_pad, int n,
                                       int W) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * W) return;
  const int c = i / W, w = i % W;
  double v = 0.0;
  for (int o = 0; o < nob; ++o) v += partials[((size_t)o * C_pad + c) * W + w];
  out[i] = v;
}

}  // namespace gpum
