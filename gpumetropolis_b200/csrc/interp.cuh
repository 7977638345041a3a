// interp.cuh -- the warp-uniform register-stack bytecode interpreter.
//
// Replaces the reference's per-thread `vm_eval` (src/rust/src/chain_kernel.rs
// :63-120), whose `stack[32]` lives in local memory and whose opcode dispatch
// is an if-chain executed once per (chain, observation).  Here:
//   * the micro-op stream sits in the constant bank (a __grid_constant__
//     kernel parameter), read at a warp-uniform pc, so the dispatch is a
//     uniform indirect branch with no divergence;
//   * every case names its stack slot at compile time, so the operand stack
//     `s[D][G/2]` (chain pairs) is an array of registers (never local
//     memory), and the arithmetic runs on two-wide FP32 instructions;
//   * each thread carries G chains through the same instruction, amortising
//     one dispatch over G chain-observations; the 32 lanes of a warp take 32
//     consecutive observations of the shared-memory tile;
//   * expensive ops (divide, pow, lgamma) share one code block per kind
//     instead of being inlined per slot.
#pragma once
#include "device.cuh"
#include "program.hpp"

namespace gpum {

constexpr int kInterpThreads = 256;  // threads per interpreter CTA

struct __align__(16) EvalProg {
  uint32_t n_uops;
  uint32_t pad_[3];
  uint32_t uop[kMaxUops];
  uint32_t term[kMaxTerms];  // K_DOT terms: param | column << 11
  float cst[kMaxConsts];
};

enum HeavyKind : int { H_NONE = -1, H_DIV = 0, H_POW = 1, H_LGAMMA = 2 };

// The G parameters of this thread's chains for one parameter index, as G/2
// pairs: one broadcast 16- or 8-byte shared load per 4 or 2 chains.
template <int G>
__device__ __forceinline__ void load_params2(const float* __restrict__ p,
                                             float2 (&v)[G / 2]) {
  if constexpr (G % 4 == 0) {
#pragma unroll
    for (int g = 0; g < G; g += 4) {
      const float4 q = *reinterpret_cast<const float4*>(p + g);
      v[g / 2] = make_float2(q.x, q.y);
      v[g / 2 + 1] = make_float2(q.z, q.w);
    }
  } else {
#pragma unroll
    for (int g = 0; g < G; g += 2) v[g / 2] = *reinterpret_cast<const float2*>(p + g);
  }
}

// acc += sum over n terms of param[p_k] * x[col_k] for the G chains, in term
// order (one FFMA2 per chain pair and term).  The narrower variants load two
// terms ahead of their multiply-adds to overlap the loads' latency.
template <int G>
__device__ __forceinline__ void gpum_dot(float2 (&acc)[G / 2], const uint32_t* __restrict__ tm,
                                         uint32_t n, const float* __restrict__ xo, int T,
                                         const float* __restrict__ pc0, int CG) {
  constexpr int H = G / 2;
  uint32_t k = 0;
  if constexpr (H <= 4) {
    for (; k + 2 <= n; k += 2) {
      const uint32_t ta = tm[k], tb = tm[k + 1];
      const float2 va = gm2(xo[(size_t)(ta >> 11) * T]), vb = gm2(xo[(size_t)(tb >> 11) * T]);
      float2 pa[H], pb[H];
      load_params2<G>(pc0 + (size_t)(ta & 0x7FFu) * CG, pa);
      load_params2<G>(pc0 + (size_t)(tb & 0x7FFu) * CG, pb);
#pragma unroll
      for (int h = 0; h < H; ++h) acc[h] = gm2_fma(pa[h], va, acc[h]);
#pragma unroll
      for (int h = 0; h < H; ++h) acc[h] = gm2_fma(pb[h], vb, acc[h]);
    }
  }
  for (; k < n; ++k) {
    const uint32_t tw = tm[k];
    const float2 v = gm2(xo[(size_t)(tw >> 11) * T]);
    float2 pv[H];
    load_params2<G>(pc0 + (size_t)(tw & 0x7FFu) * CG, pv);
#pragma unroll
    for (int h = 0; h < H; ++h) acc[h] = gm2_fma(pv[h], v, acc[h]);
  }
}

// Interpret the program once for G chains at one observation.  The stack
// holds the chains as pairs, so the arithmetic runs on sm_100's two-wide
// FP32 instructions (FADD2, FMUL2, FFMA2; subtraction and negation as exact
// FFMA2 / FMUL2 by -1), which round each half exactly like the scalar
// instruction: the values are those of one chain per instruction.
//   s  : slot S, chains 2h and 2h+1 in s[S][h]
//   xo : this lane's observation inside the tile; column j is at xo[j*T]
//   pc0: this thread's first chain in the param tile; param p, chain g at
//        pc0[p*CG + g]  (16-byte aligned; G is a multiple of 2)
//   hsm: this thread's operand scratch for the shared expensive ops, 2*G
//        floats at a stride of kInterpThreads (the block's thread count)
template <int G, int D>
__device__ __forceinline__ void interp_run(const EvalProg& pg, float2 (&s)[D][G / 2],
                                           const float* __restrict__ xo, int T,
                                           const float* __restrict__ pc0, int CG,
                                           float* __restrict__ hsm) {
  static_assert(G % 2 == 0, "chains are processed in pairs");
  constexpr int H = G / 2;
  const uint32_t n = pg.n_uops;
  // Saved subtrees (K_SAVEk / K_LOADk): registers, since every case names
  // its save index at compile time.  The sixteen-chain variant keeps one, the
  // deep-stack variants none (the compiler saves nothing for stacks deeper
  // than kMaxSavedDepth).
  constexpr int NS = D > kMaxSavedDepth ? 0 : (G >= 16 ? 1 : kMaxSaves);
  float2 sv[NS > 0 ? NS : 1][H];
  uint32_t wnext = n > 0 ? pg.uop[0] : 0u;
  for (uint32_t pc = 0; pc < n; ++pc) {
    const uint32_t w = wnext;
    wnext = pc + 1 < n ? pg.uop[pc + 1] : 0u;  // in flight while this one runs
    const uint32_t a0 = (w >> kCaseBits) & 0x7FFu;
    const uint32_t a1 = w >> 22;
    int hk = H_NONE, hs = 0;

#define GPUM_XD(a) xo[(size_t)(a) * T]
#define GPUM_HA(g) hsm[(g) * kInterpThreads]
#define GPUM_HB(g) hsm[(G + (g)) * kInterpThreads]
#define GPUM_UN(S, EXPR)                                                               \
  if constexpr (S < D) {                                                               \
    _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = EXPR;                      \
  }                                                                                    \
  break;
#define GPUM_UN1(S, EXPR)                                                              \
  if constexpr (S + 1 < D) {                                                           \
    _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = EXPR;                      \
  }                                                                                    \
  break;
#define GPUM_HEAVY2(S, KIND, BX, BY)                                                   \
  if constexpr (S < D) {                                                               \
    _Pragma("unroll") for (int h = 0; h < H; ++h) {                                    \
      GPUM_HA(2 * h) = s[S][h].x;                                                      \
      GPUM_HA(2 * h + 1) = s[S][h].y;                                                  \
      GPUM_HB(2 * h) = BX;                                                             \
      GPUM_HB(2 * h + 1) = BY;                                                         \
    }                                                                                  \
    hk = KIND;                                                                         \
    hs = S;                                                                            \
  }                                                                                    \
  break;
#define GPUM_SLOT(S)                                                                   \
  case S * NKIND + K_PUSH_C: GPUM_UN(S, gm2(pg.cst[a0]))                               \
  case S * NKIND + K_PUSH_P:                                                           \
    if constexpr (S < D) load_params2<G>(pc0 + (size_t)a0 * CG, s[S]);                 \
    break;                                                                             \
  case S * NKIND + K_PUSH_D: GPUM_UN(S, gm2(GPUM_XD(a0)))                              \
  case S * NKIND + K_ADD:                                                              \
    if constexpr (S + 1 < D) {                                                         \
      _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = gm2_add(s[S][h], s[S + 1][h]); \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SUB:                                                              \
    if constexpr (S + 1 < D) {                                                         \
      _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = gm2_sub(s[S][h], s[S + 1][h]); \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_MUL:                                                              \
    if constexpr (S + 1 < D) {                                                         \
      _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = gm2_mul(s[S][h], s[S + 1][h]); \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_DIV:                                                              \
    if constexpr (S + 1 < D) { GPUM_HEAVY2(S, H_DIV, s[S + 1][h].x, s[S + 1][h].y) }   \
    break;                                                                             \
  case S * NKIND + K_POW:                                                              \
    if constexpr (S + 1 < D) { GPUM_HEAVY2(S, H_POW, s[S + 1][h].x, s[S + 1][h].y) }   \
    break;                                                                             \
  case S * NKIND + K_ADD_C: GPUM_UN(S, gm2_add(s[S][h], gm2(pg.cst[a0])))              \
  case S * NKIND + K_SUB_C: GPUM_UN(S, gm2_sub(s[S][h], gm2(pg.cst[a0])))              \
  case S * NKIND + K_MUL_C: GPUM_UN(S, gm2_mul(s[S][h], gm2(pg.cst[a0])))              \
  case S * NKIND + K_DIV_C: GPUM_HEAVY2(S, H_DIV, pg.cst[a0], pg.cst[a0])              \
  case S * NKIND + K_POW_C: GPUM_HEAVY2(S, H_POW, pg.cst[a0], pg.cst[a0])              \
  case S * NKIND + K_ADD_P:                                                            \
    if constexpr (S < D) {                                                             \
      float2 pv[H];                                                                    \
      load_params2<G>(pc0 + (size_t)a0 * CG, pv);                                      \
      _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = gm2_add(s[S][h], pv[h]); \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SUB_P:                                                            \
    if constexpr (S < D) {                                                             \
      float2 pv[H];                                                                    \
      load_params2<G>(pc0 + (size_t)a0 * CG, pv);                                      \
      _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = gm2_sub(s[S][h], pv[h]); \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_MUL_P:                                                            \
    if constexpr (S < D) {                                                             \
      float2 pv[H];                                                                    \
      load_params2<G>(pc0 + (size_t)a0 * CG, pv);                                      \
      _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = gm2_mul(s[S][h], pv[h]); \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_DIV_P:                                                            \
  case S * NKIND + K_POW_P:                                                            \
    if constexpr (S < D) {                                                             \
      const float* pp = pc0 + (size_t)a0 * CG;                                         \
      _Pragma("unroll") for (int h = 0; h < H; ++h) {                                  \
        GPUM_HA(2 * h) = s[S][h].x;                                                    \
        GPUM_HA(2 * h + 1) = s[S][h].y;                                                \
        GPUM_HB(2 * h) = pp[2 * h];                                                    \
        GPUM_HB(2 * h + 1) = pp[2 * h + 1];                                            \
      }                                                                                \
      hk = ((w & kCaseMask) == S * NKIND + K_DIV_P) ? H_DIV : H_POW;                   \
      hs = S;                                                                          \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_ADD_D: GPUM_UN(S, gm2_add(s[S][h], gm2(GPUM_XD(a0))))             \
  case S * NKIND + K_SUB_D: GPUM_UN(S, gm2_sub(s[S][h], gm2(GPUM_XD(a0))))             \
  case S * NKIND + K_MUL_D: GPUM_UN(S, gm2_mul(s[S][h], gm2(GPUM_XD(a0))))             \
  case S * NKIND + K_DIV_D: GPUM_HEAVY2(S, H_DIV, GPUM_XD(a0), GPUM_XD(a0))            \
  case S * NKIND + K_POW_D: GPUM_HEAVY2(S, H_POW, GPUM_XD(a0), GPUM_XD(a0))            \
  case S * NKIND + K_NEG: GPUM_UN(S, gm2_neg(s[S][h]))                                 \
  case S * NKIND + K_EXP: GPUM_UN(S, gm2_exp(s[S][h]))                                 \
  case S * NKIND + K_LOG: GPUM_UN(S, gm2_log(s[S][h]))                                 \
  case S * NKIND + K_SQRT: GPUM_UN(S, gm2_sqrt(s[S][h]))                               \
  case S * NKIND + K_LGAMMA: GPUM_HEAVY2(S, H_LGAMMA, 0.0f, 0.0f)                      \
  case S * NKIND + K_SQR: GPUM_UN(S, gm2_mul(s[S][h], s[S][h]))                        \
  case S * NKIND + K_FMA_PD:                                                           \
    if constexpr (S < D) {                                                             \
      const float2 v = gm2(GPUM_XD(a1));                                               \
      float2 pv[H];                                                                    \
      load_params2<G>(pc0 + (size_t)a0 * CG, pv);                                      \
      _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = gm2_fma(pv[h], v, s[S][h]); \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_DOTP:                                                             \
    if constexpr (S < D) load_params2<G>(pc0 + (size_t)(pg.term[a0] & 0x7FFu) * CG, s[S]); \
    [[fallthrough]];                                                                   \
  case S * NKIND + K_DOT:                                                              \
    if constexpr (S < D) {                                                             \
      const uint32_t t0 = a0 + ((w & kCaseMask) == S * NKIND + K_DOTP ? 1u : 0u);      \
      gpum_dot<G>(s[S], pg.term + t0, a1 & kDotCount, xo, T, pc0, CG);                 \
      if (a1 & kDotSave) {                                                             \
        if constexpr (NS > 0) {                                                        \
          _Pragma("unroll") for (int h = 0; h < H; ++h) sv[0][h] = s[S][h];            \
        }                                                                              \
      }                                                                                \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SOFTPLUS_SV:                                                      \
    if constexpr (S < D && NS > 0) {                                                   \
      _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = gm2_softplus(sv[0][h]);  \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_ADD_C1: GPUM_UN1(S, gm2_add(gm2(pg.cst[a0]), s[S + 1][h]))       \
  case S * NKIND + K_SUB_C1: GPUM_UN1(S, gm2_sub(gm2(pg.cst[a0]), s[S + 1][h]))       \
  case S * NKIND + K_MUL_C1: GPUM_UN1(S, gm2_mul(gm2(pg.cst[a0]), s[S + 1][h]))       \
  case S * NKIND + K_ADD_D1: GPUM_UN1(S, gm2_add(gm2(GPUM_XD(a0)), s[S + 1][h]))      \
  case S * NKIND + K_SUB_D1: GPUM_UN1(S, gm2_sub(gm2(GPUM_XD(a0)), s[S + 1][h]))      \
  case S * NKIND + K_MUL_D1: GPUM_UN1(S, gm2_mul(gm2(GPUM_XD(a0)), s[S + 1][h]))      \
  case S * NKIND + K_ADD_P1:                                                           \
  case S * NKIND + K_SUB_P1:                                                           \
  case S * NKIND + K_MUL_P1:                                                           \
    if constexpr (S + 1 < D) {                                                         \
      float2 pv[H];                                                                    \
      load_params2<G>(pc0 + (size_t)a0 * CG, pv);                                      \
      const uint32_t kd = (w & kCaseMask) - S * NKIND;                                 \
      if (kd == K_ADD_P1) {                                                            \
        _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = gm2_add(pv[h], s[S + 1][h]); \
      } else if (kd == K_SUB_P1) {                                                     \
        _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = gm2_sub(pv[h], s[S + 1][h]); \
      } else {                                                                         \
        _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = gm2_mul(pv[h], s[S + 1][h]); \
      }                                                                                \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_EXP_SV:                                                           \
    if constexpr (S < D && NS > 0) {                                                   \
      _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = gm2_exp(sv[0][h]);       \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SAVE0:                                                            \
    if constexpr (S < D && NS > 0) {                                                   \
      _Pragma("unroll") for (int h = 0; h < H; ++h) sv[0][h] = s[S][h];                \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_LOAD0:                                                            \
    if constexpr (S < D && NS > 0) {                                                   \
      _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = sv[0][h];                \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SAVE1:                                                            \
    if constexpr (S < D && NS > 1) {                                                   \
      _Pragma("unroll") for (int h = 0; h < H; ++h) sv[NS - 1][h] = s[S][h];           \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_LOAD1:                                                            \
    if constexpr (S < D && NS > 1) {                                                   \
      _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = sv[NS - 1][h];           \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SOFTPLUS: GPUM_UN(S, gm2_softplus(s[S][h]))                       \
  case S * NKIND + K_SOFTPLUS1:                                                        \
    if constexpr (S + 1 < D) {                                                         \
      _Pragma("unroll") for (int h = 0; h < H; ++h) s[S][h] = gm2_softplus(s[S + 1][h]); \
    }                                                                                  \
    break;

    // Only the labels a variant can reach (slot < D) are emitted, so each
    // variant's switch is dense from 0 and compiles to one indexed branch.
#define GPUM_SLOTS_8 GPUM_SLOT(0) GPUM_SLOT(1) GPUM_SLOT(2) GPUM_SLOT(3) \
  GPUM_SLOT(4) GPUM_SLOT(5) GPUM_SLOT(6) GPUM_SLOT(7)
#define GPUM_SLOTS_16 GPUM_SLOTS_8 GPUM_SLOT(8) GPUM_SLOT(9) GPUM_SLOT(10) GPUM_SLOT(11) \
  GPUM_SLOT(12) GPUM_SLOT(13) GPUM_SLOT(14) GPUM_SLOT(15)
#define GPUM_SLOTS_32 GPUM_SLOTS_16 GPUM_SLOT(16) GPUM_SLOT(17) GPUM_SLOT(18) \
  GPUM_SLOT(19) GPUM_SLOT(20) GPUM_SLOT(21) GPUM_SLOT(22) GPUM_SLOT(23) GPUM_SLOT(24) \
  GPUM_SLOT(25) GPUM_SLOT(26) GPUM_SLOT(27) GPUM_SLOT(28) GPUM_SLOT(29) GPUM_SLOT(30) \
  GPUM_SLOT(31)
    if constexpr (D <= 8) {
      switch (w & kCaseMask) {
        GPUM_SLOTS_8
        default: break;
      }
    } else if constexpr (D <= 16) {
      switch (w & kCaseMask) {
        GPUM_SLOTS_16
        default: break;
      }
    } else {
      switch (w & kCaseMask) {
        GPUM_SLOTS_32
        default: break;
      }
    }
#undef GPUM_SLOTS_8
#undef GPUM_SLOTS_16
#undef GPUM_SLOTS_32
#undef GPUM_SLOT
#undef GPUM_UN
#undef GPUM_UN1
#undef GPUM_HEAVY2
#undef GPUM_XD

    if (hk != H_NONE) {  // warp-uniform
      // One copy of the expensive function for every slot and chain: the
      // operands went through shared memory, so this loop stays rolled.
#pragma unroll 1
      for (int g = 0; g < G; ++g) {
        const float x = GPUM_HA(g);
        GPUM_HA(g) = hk == H_DIV ? x / GPUM_HB(g)
                                 : (hk == H_POW ? powf(x, GPUM_HB(g)) : lgammaf(x));
      }
      // Write back to the slot named by the case (a second uniform switch).
#define GPUM_WB(S)                                                              \
  case S:                                                                       \
    if constexpr (S < D) {                                                      \
      _Pragma("unroll") for (int h = 0; h < H; ++h)                             \
        s[S][h] = make_float2(GPUM_HA(2 * h), GPUM_HA(2 * h + 1));              \
    }                                                                           \
    break;
      switch (hs) {
        GPUM_WB(0) GPUM_WB(1) GPUM_WB(2) GPUM_WB(3) GPUM_WB(4) GPUM_WB(5) GPUM_WB(6)
        GPUM_WB(7) GPUM_WB(8) GPUM_WB(9) GPUM_WB(10) GPUM_WB(11) GPUM_WB(12) GPUM_WB(13)
        GPUM_WB(14) GPUM_WB(15) GPUM_WB(16) GPUM_WB(17) GPUM_WB(18) GPUM_WB(19)
        GPUM_WB(20) GPUM_WB(21) GPUM_WB(22) GPUM_WB(23) GPUM_WB(24) GPUM_WB(25)
        GPUM_WB(26) GPUM_WB(27) GPUM_WB(28) GPUM_WB(29) GPUM_WB(30) GPUM_WB(31)
        default: break;
      }
#undef GPUM_WB
    }
#undef GPUM_HA
#undef GPUM_HB
  }
}

}  // namespace gpum
