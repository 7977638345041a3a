// program.hpp -- host-side compiler from gpumetropolis bytecode to the
// register-slot micro-op stream the B200 interpreter executes.
//
// Input format (R/dsl.R:13-17, emitted as (opcode, arg) u32 pairs):
//   0 PUSH_CONST, 1 PUSH_PARAM, 2 PUSH_DATA, 3 ADD, 4 SUB, 5 MUL, 6 DIV,
//   7 NEG, 8 EXP, 9 LOG, 10 SQRT, 11 POW, 12 LGAMMA.
// Semantics follow the reference interpreter (src/rust/src/cpu_native.rs:80-107
// and chain_kernel.rs:63-120): an empty program evaluates to 0, the result is
// stack slot 0, and every opcode outside {0..10,12} acts as POW.  Unlike the
// reference (which validates only in R, dsl.R:115-119, and otherwise panics on
// an out-of-range index), this compiler rejects malformed programs with an
// error before anything reaches the GPU.
//
// Output: one 32-bit word per micro-op,
//   bits  0..10  case id = slot * NKIND + kind   (slot = stack index of the
//                 result, a compile-time register index in the kernel)
//   bits 11..21  a0 (const / param / column index)
//   bits 22..31  a1 (second index for two-operand fused forms, < 1024)
// plus an f32 constant pool.  Peephole fusion folds a push into the binary op
// that consumes it, `p*x + acc` patterns into one multiply-add, and a run of
// such multiply-adds into the same slot (a linear predictor) into one K_DOT
// micro-op over a term table, so the dispatch is paid once per run.  A
// subtree of at least kMinSaved instructions that the program computes again
// later (the logistic and Poisson likelihoods write their linear predictor
// twice) is kept after its first evaluation (K_SAVEk) and every later copy
// becomes one K_LOADk: the same FP32 value, computed once.  A push whose
// value waits on the stack while a subtree above it is evaluated, and then
// meets it in an add, subtract or multiply, is not pushed: the operation
// reads the operand directly (K_ADD_D1 and the like).  A last pass
// folds micro-op pairs that always meet into one dispatch: a parameter push
// that starts a K_DOT (K_DOTP), a K_SAVE0 of a K_DOT's result (a flag of the
// K_DOT), and a K_LOAD0 whose value only feeds a softplus or an exponential
// (K_SOFTPLUS_SV, K_EXP_SV).  LOG(1 + EXP(a))
// (either operand order of the ADD) becomes one K_SOFTPLUS of a, evaluated
// as max(a, 0) + log1p(e^-|a|): more accurate than the two calls in FP32
// (no rounding of 1 + e^a to 1 where e^a < 2^-24) and about half the work.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace gpum {

enum Kind : uint32_t {
  K_PUSH_C = 0, K_PUSH_P, K_PUSH_D,
  K_ADD, K_SUB, K_MUL, K_DIV, K_POW,            // s[t] = s[t] op s[t+1]
  K_ADD_C, K_SUB_C, K_MUL_C, K_DIV_C, K_POW_C,  // s[t] = s[t] op const
  K_ADD_P, K_SUB_P, K_MUL_P, K_DIV_P, K_POW_P,  // s[t] = s[t] op param
  K_ADD_D, K_SUB_D, K_MUL_D, K_DIV_D, K_POW_D,  // s[t] = s[t] op data
  K_NEG, K_EXP, K_LOG, K_SQRT, K_LGAMMA,        // s[t] = f(s[t])
  K_SQR,                                        // s[t] = s[t]*s[t]  (x^2)
  K_FMA_PD,                                     // s[t] += param[a0]*data[a1]
  K_DOT,                                        // s[t] += sum over terms[a0 .. a0+a1)
                                                //   of param[p_k]*data[x_k], in order
  K_SAVE0, K_SAVE1,                             // saved[k] = s[t]
  K_LOAD0, K_LOAD1,                             // s[t] = saved[k]
  K_SOFTPLUS,                                   // s[t] = log(1 + exp(s[t]))
  K_SOFTPLUS1,                                  // s[t] = log(1 + exp(s[t+1]))
  K_DOTP,                                       // s[t] = param[terms[a0]], then
                                                //   the terms a0+1 .. a0+count as K_DOT
  K_SOFTPLUS_SV,                                // s[t] = log(1 + exp(saved[0]))
  K_EXP_SV,                                     // s[t] = exp(saved[0])
  K_ADD_C1, K_SUB_C1, K_MUL_C1,                 // s[t] = const op s[t+1]
  K_ADD_P1, K_SUB_P1, K_MUL_P1,                 // s[t] = param op s[t+1]
  K_ADD_D1, K_SUB_D1, K_MUL_D1,                 // s[t] = data op s[t+1]
  NKIND
};
constexpr int kMaxSaves = 2;       // saved subtrees per program
constexpr uint32_t kDotCount = 0x1FFu;  // K_DOT / K_DOTP a1: term count (bits 0-8)
constexpr uint32_t kDotSave = 0x200u;   //   and bit 9: also keep the result as saved[0]
constexpr int kMinSaved = 8;       // smallest subtree worth saving (instructions)
constexpr int kMaxSavedDepth = 8;  // programs with deeper stacks save nothing
constexpr int kCaseBits = 11;
constexpr uint32_t kCaseMask = (1u << kCaseBits) - 1u;

constexpr int kMaxStack = 32;      // reference limit (R/dsl.R:20)
constexpr int kMaxUops = 1024;     // micro-ops per program (constant bank)
constexpr int kMaxConsts = 512;    // f32 constants per program
constexpr int kMaxIndex = 2047;    // 11-bit a0 field
constexpr int kMaxA1 = 1023;       // 10-bit a1 field
constexpr int kMaxSlots = 32;      // deepest interpreter variant
constexpr int kMaxTerms = 1024;    // (param, column) terms of K_DOT micro-ops

struct UProg {
  std::vector<uint32_t> uops;
  std::vector<uint32_t> terms;  // K_DOT terms: param | column << 11
  std::vector<float> consts;
  int depth = 0;          // peak stack depth of the source program
  int n_saves = 0;        // saved subtrees (K_SAVEk / K_LOADk pairs)
  int n_src = 0;          // source instructions
  bool uses_data = false;
  bool empty() const { return n_src == 0; }
};

inline uint32_t uop_word(uint32_t kind, uint32_t slot, uint32_t a0, uint32_t a1) {
  return (slot * NKIND + kind) | (a0 << kCaseBits) | (a1 << 22);
}
static_assert(kMaxSlots * NKIND <= (1 << kCaseBits), "case ids must fit their field");

// The interpreter engine's gradient program: the source bytecode as a list
// of its non-push instructions ("nodes"), each naming its operands directly
// -- another node, a constant, a parameter or a data column -- so a thread
// can keep one observation's forward values in a tape of nodes and sweep it
// backwards (the reference's tape AD, cpu_native.rs:148-279).
//   node word: op (4 bits: 3..12, unknown opcodes as POW 11) | refA << 4 |
//              refB << 18;  ref = type (2 bits) | index << 2, type 0 node,
//              1 constant, 2 parameter, 3 data column (index < 4096)
//   root: the ref of the program's result (slot 0)
enum GradRef : uint32_t { GREF_NODE = 0, GREF_CONST = 1, GREF_PARAM = 2, GREF_DATA = 3 };
constexpr int kMaxGradNodes = 512;   // tape entries per observation
constexpr int kMaxGradParams = 128;  // parameters of the interpreted gradient

struct UGradProg {
  std::vector<uint32_t> nodes;
  uint32_t root = 0;   // a ref; meaningful when has_root
  bool has_root = false;
};

// Builds the gradient program; 1 with *err when the program is beyond the
// interpreted gradient's limits (the compiled engine has none of them).
int compile_grad_program(const uint32_t* code, size_t n_code, uint32_t n_params,
                         UGradProg* out, std::string* err);

// Validates and compiles.  Returns 0 or an error message in *err.
int compile_program(const uint32_t* code, size_t n_code, const double* consts,
                    size_t n_consts, uint32_t n_params, uint32_t n_cols,
                    bool allow_data, UProg* out, std::string* err);

// Validation only (stack discipline, operand ranges, depth), for programs
// that are interpreted in f64 directly from the source bytecode (the prior).
int validate_program(const uint32_t* code, size_t n_code, size_t n_consts,
                     uint32_t n_params, uint32_t n_cols, bool allow_data,
                     int* depth, std::string* err);

// Observations per shared-memory tile for a data set of n_cols columns: a
// multiple of 32 (one per lane), at most 256 (the TMA box limit) and at most
// 32 KB per stage.  The compiled engine bakes it into the generated loads.
inline int tile_obs(uint32_t n_cols) {
  if (n_cols == 0) return 256;
  const int T = (int)((8192 / n_cols) / 32 * 32);
  return T < 32 ? 32 : (T > 256 ? 256 : T);
}

}  // namespace gpum
