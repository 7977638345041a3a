// codegen.hpp -- translate gpumetropolis bytecode into straight-line CUDA C
// for the compiled tier (NVRTC, sm_100a).
//
// The GPU analogue of the reference's Cranelift JIT (src/rust/src/jit.rs:
// compile_loglik :441-631, compile_grad :97-436): the stack program becomes
// SSA values; here additionally
//   * identical subexpressions are computed once (hash-consing), so e.g. the
//     linear predictor that a logistic log-likelihood spells twice is one sum;
//   * constant subexpressions are folded in f64;
//   * parameter-only subexpressions (exp(log_sigma), 1/(1+exp(-lw)), ...) are
//     hoisted out of the observation loop and computed once per chain;
//   * the reverse-mode gradient is unrolled (local derivatives of
//     cpu_native.rs:217-277, including the POW exponent guard a > 0 and the
//     digamma derivative of lgamma), with parameter-only nodes receiving
//     accumulated adjoints that are pushed to the parameters once per chain.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace gpum {

struct GenModel {
  std::string source;     // device functions gm_* (see codegen.cpp)
  int np = 0;             // parameters
  int n_hoist = 0;        // per-chain hoisted values
  int n_data = 0;         // per-observation data registers
  int n_fwd = 0;          // per-observation forward nodes
  int n_mat = 0;          // data-only operations materialized as extra columns
  bool has_grad = false;
  // Linear predictor on the tensor cores (gm_iter_value_tc): product
  // columns (data, materialized, and a ones column for the offset), padded
  // to a multiple of 8, tail data columns, observations per tile, stages.
  // tc_warps: epilogue warps (8, 12 or 16; GPUM_B200_TC_WARPS, default 16),
  // the kernel adds one control warp.
  bool tc = false;
  int tc_k = 0, tc_kp = 0, tc_ntail = 0, tc_tn = 0, tc_stages = 0, tc_warps = 8;
};

// Dynamic shared memory of the tensor-core value kernel: `stages` stages of
// [hi | lo] product columns (kp, a multiple of 8) for tn observations, four
// slots of the nt tail columns, the coefficient operand [hi | lo] x 128
// chains, the FP64 reduction buffer [4][128], per-chain flags [128] and the
// barriers.
inline size_t tc_smem_bytes(int kp, int nt, int tn, int stages) {
  return (size_t)stages * 2 * kp * tn * 4 + (size_t)4 * nt * tn * 4 +
         (size_t)2 * kp * 128 * 4 + 4 * 128 * 8 + 128 * 4 + 512;
}

// Builds the model functions for the log-likelihood program (f32 per
// observation) and the prior program (f64, parameters only).  Returns 0, or
// 1 with a message.  The programs must already be validated.
int generate_model(const uint32_t* code, size_t n_code, const double* consts,
                   const uint32_t* prior_code, size_t n_prior, const double* prior_consts,
                   uint32_t n_params, uint32_t n_cols, GenModel* out, std::string* err);

}  // namespace gpum
