// jit.hpp -- the compiled engine's run-time build: NVRTC (loaded with dlopen,
// so the library has no link-time dependency on it) compiles the generated
// model functions with the kernel headers for sm_100a; the cubin is loaded
// with cudaLibraryLoadData.  Builds are cached per generated source for the
// life of the process.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "codegen.hpp"

namespace gpum {

struct CompiledModel {
  cudaKernel_t k_value = nullptr;   // gm_iter_value
  cudaKernel_t k_grad = nullptr;    // gm_iter_grad
  cudaKernel_t k_mat = nullptr;     // gm_materialize (extra data columns)
  cudaKernel_t k_prior = nullptr;   // gm_prior_batch (f64 prior, optional gradient)
  int n_mat = 0;                    // materialized data-only operations
  int G = 1, GG = 1;                // chains per thread of each kernel
  bool pair = false;                // value kernel evaluates observation pairs
  bool lanes = false;               // value kernel: one chain per lane (G counts 32)
  bool lanes_grad = false;          // gradient kernel: one chain per lane
  int np = 0;
  double compile_seconds = 0.0;
  // Linear predictor on the tensor cores (GenModel::tc): the value kernel
  // gm_iter_value_tc and the packing kernel gm_tc_pack, with their shapes.
  bool tc = false;
  cudaKernel_t k_value_tc = nullptr;
  cudaKernel_t k_tc_pack = nullptr;
  int tc_kp = 0, tc_ntail = 0, tc_tn = 0, tc_stages = 0, tc_threads = 0;
};

// Chains per thread for the value and gradient kernels, and whether the
// value kernel uses the paired-observation body, by parameter and hoisted
// value counts.
void jit_chains_per_thread(int np, int nh, int* G, int* GG, bool* pair);

// Whether the value kernel maps chains to lanes (wide models: every lane
// reads the same observation values, broadcast): models the paired body does
// not take, with parameters + hoisted values that fit the registers (data-only
// operations are materialized columns, so no lane repeats them).
bool jit_value_lanes(const GenModel& gm, bool pair);

// Whether the gradient kernel maps chains to lanes: models whose parameters
// + hoisted values (values and adjoints in registers) stay within 100; wider
// ones take the scalar body (GG chains per thread, lanes over observations).
bool jit_grad_lanes(const GenModel& gm);

// Returns 0 and a loaded model, or 1 with a message (NVRTC missing, compile
// error, load error).
int jit_compile(const GenModel& gm, CompiledModel* out, std::string* err);

// The full NVRTC source a model compiles from (for tests and diagnostics).
std::string jit_source(const GenModel& gm, int G, int GG, bool pair);

// Compile only (no GPU needed): returns 0 and the cubin size, or 1 + message.
int jit_compile_check(const GenModel& gm, size_t* cubin_bytes, std::string* err);

}  // namespace gpum
