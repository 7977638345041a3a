// interp.cuh -- the warp-uniform register-stack bytecode interpreter.
//
// Replaces the reference's per-thread `vm_eval` (src/rust/src/chain_kernel.rs
// :63-120), whose `stack[32]` lives in local memory and whose opcode dispatch
// is an if-chain executed once per (chain, observation).  Here:
//   * the micro-op stream sits in the constant bank (a __grid_constant__
//     kernel parameter), read at a warp-uniform pc, so the dispatch is a
//     uniform indirect branch with no divergence;
//   * every case names its stack slot at compile time, so the operand stack
//     `s[D][G]` is an array of registers (never local memory);
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

// The G parameters of this thread's chains for one parameter index: one
// broadcast 16- or 8-byte shared load per 4 or 2 chains.
template <int G>
__device__ __forceinline__ void load_params(const float* __restrict__ p, float (&v)[G]) {
  if constexpr (G % 4 == 0) {
#pragma unroll
    for (int g = 0; g < G; g += 4) {
      const float4 q = *reinterpret_cast<const float4*>(p + g);
      v[g] = q.x; v[g + 1] = q.y; v[g + 2] = q.z; v[g + 3] = q.w;
    }
  } else if constexpr (G % 2 == 0) {
#pragma unroll
    for (int g = 0; g < G; g += 2) {
      const float2 q = *reinterpret_cast<const float2*>(p + g);
      v[g] = q.x; v[g + 1] = q.y;
    }
  } else {
#pragma unroll
    for (int g = 0; g < G; ++g) v[g] = p[g];
  }
}

// Interpret the program once for G chains at one observation.
//   xo : this lane's observation inside the tile; column j is at xo[j*T]
//   pc0: this thread's first chain in the param tile; param p, chain g at
//        pc0[p*CG + g]  (16-byte aligned; G is a multiple of 2)
//   hsm: this thread's operand scratch for the shared expensive ops, 2*G
//        floats at a stride of kInterpThreads (the block's thread count)
template <int G, int D>
__device__ __forceinline__ void interp_run(const EvalProg& pg, float (&s)[D][G],
                                           const float* __restrict__ xo, int T,
                                           const float* __restrict__ pc0, int CG,
                                           float* __restrict__ hsm) {
  const uint32_t n = pg.n_uops;
  // Saved subtrees (K_SAVEk / K_LOADk): registers, since every case names
  // its save index at compile time.  The sixteen-chain variant keeps one, the
  // deep-stack variants none (the compiler saves nothing for stacks deeper
  // than kMaxSavedDepth).
  constexpr int NS = D > kMaxSavedDepth ? 0 : (G >= 16 ? 1 : kMaxSaves);
  float sv[NS > 0 ? NS : 1][G];
  for (uint32_t pc = 0; pc < n; ++pc) {
    const uint32_t w = pg.uop[pc];
    const uint32_t a0 = (w >> kCaseBits) & 0x7FFu;
    const uint32_t a1 = w >> 22;
    int hk = H_NONE, hs = 0;

#define GPUM_PL(g) pv[g]
#define GPUM_XD(a) xo[(size_t)(a) * T]
#define GPUM_HA(g) hsm[(g) * kInterpThreads]
#define GPUM_HB(g) hsm[(G + (g)) * kInterpThreads]
#define GPUM_SLOT(S)                                                                   \
  case S * NKIND + K_PUSH_C:                                                           \
    if constexpr (S < D) {                                                             \
      const float v = pg.cst[a0];                                                      \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = v;                       \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_PUSH_P:                                                           \
    if constexpr (S < D) {                                                             \
      float pv[G];                                                                     \
      load_params<G>(pc0 + (size_t)a0 * CG, pv);                                       \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = GPUM_PL(g);              \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_PUSH_D:                                                           \
    if constexpr (S < D) {                                                             \
      const float v = GPUM_XD(a0);                                                     \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = v;                       \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_ADD:                                                              \
    if constexpr (S + 1 < D) {                                                         \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = s[S][g] + s[S + 1][g];   \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SUB:                                                              \
    if constexpr (S + 1 < D) {                                                         \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = s[S][g] - s[S + 1][g];   \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_MUL:                                                              \
    if constexpr (S + 1 < D) {                                                         \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = s[S][g] * s[S + 1][g];   \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_DIV:                                                              \
  case S * NKIND + K_POW:                                                              \
    if constexpr (S + 1 < D) {                                                         \
      _Pragma("unroll") for (int g = 0; g < G; ++g) {                                  \
        GPUM_HA(g) = s[S][g];                                                          \
        GPUM_HB(g) = s[S + 1][g];                                                      \
      }                                                                                \
      hk = ((w & kCaseMask) == S * NKIND + K_DIV) ? H_DIV : H_POW;                         \
      hs = S;                                                                          \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_ADD_C:                                                            \
    if constexpr (S < D) {                                                             \
      const float v = pg.cst[a0];                                                      \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = s[S][g] + v;             \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SUB_C:                                                            \
    if constexpr (S < D) {                                                             \
      const float v = pg.cst[a0];                                                      \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = s[S][g] - v;             \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_MUL_C:                                                            \
    if constexpr (S < D) {                                                             \
      const float v = pg.cst[a0];                                                      \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = s[S][g] * v;             \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_DIV_C:                                                            \
  case S * NKIND + K_POW_C:                                                            \
    if constexpr (S < D) {                                                             \
      const float v = pg.cst[a0];                                                      \
      _Pragma("unroll") for (int g = 0; g < G; ++g) {                                  \
        GPUM_HA(g) = s[S][g];                                                          \
        GPUM_HB(g) = v;                                                                \
      }                                                                                \
      hk = ((w & kCaseMask) == S * NKIND + K_DIV_C) ? H_DIV : H_POW;                       \
      hs = S;                                                                          \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_ADD_P:                                                            \
    if constexpr (S < D) {                                                             \
      float pv[G];                                                                     \
      load_params<G>(pc0 + (size_t)a0 * CG, pv);                                       \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = s[S][g] + GPUM_PL(g);    \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SUB_P:                                                            \
    if constexpr (S < D) {                                                             \
      float pv[G];                                                                     \
      load_params<G>(pc0 + (size_t)a0 * CG, pv);                                       \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = s[S][g] - GPUM_PL(g);    \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_MUL_P:                                                            \
    if constexpr (S < D) {                                                             \
      float pv[G];                                                                     \
      load_params<G>(pc0 + (size_t)a0 * CG, pv);                                       \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = s[S][g] * GPUM_PL(g);    \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_DIV_P:                                                            \
  case S * NKIND + K_POW_P:                                                            \
    if constexpr (S < D) {                                                             \
      float pv[G];                                                                     \
      load_params<G>(pc0 + (size_t)a0 * CG, pv);                                       \
      _Pragma("unroll") for (int g = 0; g < G; ++g) {                                  \
        GPUM_HA(g) = s[S][g];                                                          \
        GPUM_HB(g) = GPUM_PL(g);                                                       \
      }                                                                                \
      hk = ((w & kCaseMask) == S * NKIND + K_DIV_P) ? H_DIV : H_POW;                       \
      hs = S;                                                                          \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_ADD_D:                                                            \
    if constexpr (S < D) {                                                             \
      const float v = GPUM_XD(a0);                                                     \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = s[S][g] + v;             \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SUB_D:                                                            \
    if constexpr (S < D) {                                                             \
      const float v = GPUM_XD(a0);                                                     \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = s[S][g] - v;             \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_MUL_D:                                                            \
    if constexpr (S < D) {                                                             \
      const float v = GPUM_XD(a0);                                                     \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = s[S][g] * v;             \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_DIV_D:                                                            \
  case S * NKIND + K_POW_D:                                                            \
    if constexpr (S < D) {                                                             \
      const float v = GPUM_XD(a0);                                                     \
      _Pragma("unroll") for (int g = 0; g < G; ++g) {                                  \
        GPUM_HA(g) = s[S][g];                                                          \
        GPUM_HB(g) = v;                                                                \
      }                                                                                \
      hk = ((w & kCaseMask) == S * NKIND + K_DIV_D) ? H_DIV : H_POW;                       \
      hs = S;                                                                          \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_NEG:                                                              \
    if constexpr (S < D) {                                                             \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = -s[S][g];                \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_EXP:                                                              \
    if constexpr (S < D) {                                                             \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = expf(s[S][g]);           \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_LOG:                                                              \
    if constexpr (S < D) {                                                             \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = logf(s[S][g]);           \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SQRT:                                                             \
    if constexpr (S < D) {                                                             \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = sqrtf(s[S][g]);          \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_LGAMMA:                                                           \
    if constexpr (S < D) {                                                             \
      _Pragma("unroll") for (int g = 0; g < G; ++g) GPUM_HA(g) = s[S][g];              \
      hk = H_LGAMMA;                                                                   \
      hs = S;                                                                          \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SQR:                                                              \
    if constexpr (S < D) {                                                             \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = s[S][g] * s[S][g];       \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_FMA_PD:                                                           \
    if constexpr (S < D) {                                                             \
      const float v = GPUM_XD(a1);                                                     \
      float pv[G];                                                                     \
      load_params<G>(pc0 + (size_t)a0 * CG, pv);                                       \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = fmaf(GPUM_PL(g), v, s[S][g]); \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_DOT:                                                              \
    if constexpr (S < D) {                                                             \
      for (uint32_t k = 0; k < a1; ++k) {                                              \
        const uint32_t tw = pg.term[a0 + k];                                           \
        const float v = GPUM_XD(tw >> 11);                                             \
        float pv[G];                                                                   \
        load_params<G>(pc0 + (size_t)(tw & 0x7FFu) * CG, pv);                          \
        _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = fmaf(GPUM_PL(g), v, s[S][g]); \
      }                                                                                \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SAVE0:                                                            \
    if constexpr (S < D && NS > 0) {                                                   \
      _Pragma("unroll") for (int g = 0; g < G; ++g) sv[0][g] = s[S][g];                \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_LOAD0:                                                            \
    if constexpr (S < D && NS > 0) {                                                   \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = sv[0][g];                \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SAVE1:                                                            \
    if constexpr (S < D && NS > 1) {                                                   \
      _Pragma("unroll") for (int g = 0; g < G; ++g) sv[NS - 1][g] = s[S][g];           \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_LOAD1:                                                            \
    if constexpr (S < D && NS > 1) {                                                   \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = sv[NS - 1][g];           \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SOFTPLUS:                                                         \
    if constexpr (S < D) {                                                             \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = gm_softplus(s[S][g]);    \
    }                                                                                  \
    break;                                                                             \
  case S * NKIND + K_SOFTPLUS1:                                                        \
    if constexpr (S + 1 < D) {                                                         \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = gm_softplus(s[S + 1][g]); \
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
#undef GPUM_PL
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
#define GPUM_WB(S)                                                        \
  case S:                                                                 \
    if constexpr (S < D) {                                                \
      _Pragma("unroll") for (int g = 0; g < G; ++g) s[S][g] = GPUM_HA(g); \
    }                                                                     \
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
