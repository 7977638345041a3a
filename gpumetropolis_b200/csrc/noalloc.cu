// noalloc.cu -- log-likelihood batches for callers that cannot allocate.
//
// Some embedding hosts own all device memory themselves (a pool managed by
// their own allocator, a memory budget fixed before the sampler is loaded,
// or code that must not call cudaMalloc/cudaFree at all).  This entry point
// evaluates the summed log-likelihood at a batch of points on buffers the
// caller already owns, and allocates nothing: no cudaMalloc, no cudaFree, no
// host heap.  Its scratch (the f32 parameter tile and the per-block partial
// sums of the interpreter kernel) lives in one file-scope __device__ array of
// kScratchBytes, which every GPU that loads this library holds until the
// process exits.
//
// The array is shared by every call on a device and keeps the last call's
// contents; each call rewrites all it reads and clears its error word first.
// Calls whose GPU work overlaps (different streams, or host threads racing)
// race on the array and give wrong results: serialise them.  The first call
// on a device looks up the array's device address (cudaGetSymbolAddress);
// make that first call before any stream capture.  Each call waits for its
// stream before returning, so it reports device-side failures.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/gpum_b200.h"
#include "kernels.cuh"
#include "program.hpp"

using namespace gpum;

namespace {

constexpr size_t kScratchBytes = 16u << 20;  // 16 MiB per device
constexpr int kMaxDevicesNoAlloc = 64;
constexpr int kMaxSrcInstr = kMaxUops;       // one micro-op per source instruction

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevicesNoAlloc];

int fail(char* err, size_t len, int code, const char* msg) {
  if (err && len) std::snprintf(err, len, "%s", msg);
  return code;
}

// Device address of the scratch array for the current device, looked up
// once per device (the first call on a device does this).
int scratch_for_device(void** out, char* err, size_t len) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevicesNoAlloc)
    return fail(err, len, GPUM_ERR_NODEVICE, "no usable current CUDA device");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      if (err && len)
        std::snprintf(err, len,
                      "cudaGetSymbolAddress of the scratch array failed (%s); the 16 MiB "
                      "array is placed when the library's device code first loads",
                      cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? GPUM_ERR_NOMEM : GPUM_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return GPUM_OK;
}

// Validate and emit one micro-op per source instruction (no fusion) into a
// caller-provided program, using stack storage only.
int emit_plain(const uint32_t* code, size_t n_code, const double* consts, size_t n_consts,
               uint32_t np, uint32_t ncols, EvalProg* prog, int* depth, char* err, size_t len) {
  if (n_code % 2 != 0) return fail(err, len, GPUM_ERR_INVALID, "bytecode length must be even");
  const size_t n = n_code / 2;
  if (n > (size_t)kMaxSrcInstr)
    return fail(err, len, GPUM_ERR_UNSUPPORTED, "program longer than 1024 instructions");
  if (n_consts > (size_t)kMaxConsts)
    return fail(err, len, GPUM_ERR_UNSUPPORTED, "more than 512 constants");
  if ((n > 0 && !code) || (n_consts > 0 && !consts))
    return fail(err, len, GPUM_ERR_INVALID, "bytecode or constant pointer is NULL");
  int sp = 0, maxd = 0;
  for (size_t pc = 0; pc < n; ++pc) {
    uint32_t op = code[2 * pc];
    const uint32_t arg = code[2 * pc + 1];
    if (!(op <= 10 || op == 12)) op = 11;  // unknown opcodes act as POW
    uint32_t kind = 0;
    int slot = 0;
    if (op <= 2) {
      const bool ok = (op == 0 && arg < n_consts) || (op == 1 && arg < np) ||
                      (op == 2 && arg < ncols);
      if (!ok) return fail(err, len, GPUM_ERR_INVALID, "operand index out of range");
      kind = op == 0 ? K_PUSH_C : (op == 1 ? K_PUSH_P : K_PUSH_D);
      slot = sp++;
    } else if ((op >= 7 && op <= 10) || op == 12) {
      if (sp < 1) return fail(err, len, GPUM_ERR_INVALID, "stack underflow");
      kind = op == 7 ? K_NEG : op == 8 ? K_EXP : op == 9 ? K_LOG : op == 10 ? K_SQRT : K_LGAMMA;
      slot = sp - 1;
    } else {
      if (sp < 2) return fail(err, len, GPUM_ERR_INVALID, "stack underflow");
      kind = op == 3 ? K_ADD : op == 4 ? K_SUB : op == 5 ? K_MUL : op == 6 ? K_DIV : K_POW;
      slot = sp - 2;
      --sp;
    }
    if (sp > maxd) maxd = sp;
    if (maxd > kMaxStack) return fail(err, len, GPUM_ERR_INVALID, "stack deeper than 32");
    prog->uop[pc] = uop_word(kind, (uint32_t)slot, op <= 2 ? arg : 0u, 0u);
  }
  if (n > 0 && sp < 1) return fail(err, len, GPUM_ERR_INVALID, "program leaves an empty stack");
  prog->n_uops = (uint32_t)n;
  for (size_t i = 0; i < n_consts; ++i) prog->cst[i] = (float)consts[i];
  *depth = maxd;
  return GPUM_OK;
}

}  // namespace

extern "C" int gpum_b200_loglik_batch_noalloc(
    const uint32_t* code, size_t n_code, const double* consts, size_t n_consts,
    uint32_t n_params, const float* d_data, uint64_t ld, uint32_t n_cols, uint64_t n_obs,
    const double* d_points, size_t n_points, double* d_out, void* stream, char* err,
    size_t err_len) {
  if (err && err_len) err[0] = '\0';
  if (n_params < 1 || n_params > 256)
    return fail(err, err_len, GPUM_ERR_INVALID, "n_params must be in 1..256");
  if (n_cols > 256) return fail(err, err_len, GPUM_ERR_UNSUPPORTED, "more than 256 columns");
  if (n_obs >= (1ull << 31) - 1024)
    return fail(err, err_len, GPUM_ERR_UNSUPPORTED, "more than 2^31 observations");
  if (n_points == 0) return GPUM_OK;
  if (!d_points || !d_out) return fail(err, err_len, GPUM_ERR_INVALID, "NULL points or out");
  // A model with no data columns still adds its per-observation term once
  // per observation (n_obs times); only then is no data pointer needed.
  const bool has_data = n_cols > 0 && n_obs > 0;
  if (has_data) {
    if (!d_data) return fail(err, err_len, GPUM_ERR_INVALID, "NULL data pointer");
    if (ld < n_obs || ld % 4 != 0 || ((uintptr_t)d_data & 15u) != 0)
      return fail(err, err_len, GPUM_ERR_INVALID,
                  "data must be column-major f32 with ld >= n_obs, ld % 4 == 0, "
                  "and 16-byte aligned");
  }
  EvalProg prog;  // about 6 KB of host stack
  std::memset(&prog, 0, sizeof prog);
  int depth = 0;
  int rc = emit_plain(code, n_code, consts, n_consts, n_params, n_cols, &prog, &depth, err,
                      err_len);
  if (rc != GPUM_OK) return rc;
  void* scratch = nullptr;
  rc = scratch_for_device(&scratch, err, err_len);
  if (rc != GPUM_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned char* base = static_cast<unsigned char*>(scratch);
  uint32_t* d_err = reinterpret_cast<uint32_t*>(base);
  if (prog.n_uops == 0 || n_obs == 0) {
    // empty program or no observations: every sum is zero
    if (cudaMemsetAsync(d_out, 0, sizeof(double) * n_points, st) != cudaSuccess)
      return fail(err, err_len, GPUM_ERR_CUDA, "cudaMemsetAsync on the output failed");
    return GPUM_OK;
  }

  // Launch geometry, as the session's interpreter engine chooses it.
  const int G = depth <= 8 ? 8 : (depth <= 16 ? 4 : 2);
  const void* fn = depth <= 8 ? (const void*)iter_kernel<8, 8>
                              : (depth <= 16 ? (const void*)iter_kernel<4, 16>
                                             : (const void*)iter_kernel<2, 32>);
  const int T = n_cols > 0 ? std::max(32, std::min(256, (int)((8192 / n_cols) / 32 * 32)))
                           : 256;
  const int n = (int)std::min<size_t>(n_points, 1u << 24);
  if ((size_t)n != n_points) return fail(err, err_len, GPUM_ERR_UNSUPPORTED, "too many points");
  const int groups = (n + G - 1) / G;
  int WC = 1;
  while (WC < kWarps && WC < groups) WC *= 2;
  const int CG = WC * G, NCB = (n + CG - 1) / CG, C_pad = NCB * CG;
  const int ntiles = (int)((n_obs + T - 1) / T);
  const size_t smem = skel_smem_bytes(T, (int)n_cols, (int)n_params, CG, G, 1);
  int occ = 1, sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncAttributes fa{};  // the interpreter's static operand scratch counts too
  if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess)
    return fail(err, err_len, GPUM_ERR_CUDA, "cudaFuncGetAttributes failed");
  if (smem + fa.sharedSizeBytes > 48 * 1024 &&
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
    return fail(err, err_len, GPUM_ERR_UNSUPPORTED, "shared memory request refused");
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kThreads, smem);
  occ = std::max(occ, 1);
  // Scratch: [error word | params f32 np x C_pad | partials f64 NOB x C_pad].
  const size_t off_params = 256;
  const size_t param_bytes = (((size_t)n_params * C_pad * 4) + 255) & ~(size_t)255;
  const size_t off_part = off_params + param_bytes;
  if (off_part >= kScratchBytes)
    return fail(err, err_len, GPUM_ERR_UNSUPPORTED,
                "n_params x points exceeds the 16 MiB scratch of this entry point");
  const size_t max_nob = (kScratchBytes - off_part) / ((size_t)C_pad * 8);
  if (max_nob < 1)
    return fail(err, err_len, GPUM_ERR_UNSUPPORTED,
                "too many points for the 16 MiB scratch of this entry point");
  int nob = std::max(1, (4 * sms * occ) / NCB);
  nob = std::min<int>(nob, std::max(1, ntiles));
  nob = std::min<int>(nob, (int)std::min<size_t>(max_nob, 1u << 20));
  const int tiles_per_cta = (ntiles + nob - 1) / nob;
  nob = (ntiles + tiles_per_cta - 1) / tiles_per_cta;

  // Without data columns the kernel stages no tiles and never reads the map.
  CUtensorMap tm;
  std::memset(&tm, 0, sizeof tm);
  if (has_data) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
      return fail(err, err_len, GPUM_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    auto enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    cuuint64_t gdim[2] = {(cuuint64_t)n_obs, (cuuint64_t)n_cols};
    cuuint64_t gstride[1] = {(cuuint64_t)ld * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)T, (cuuint32_t)n_cols};
    cuuint32_t estr[2] = {1, 1};
    if (enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(d_data), gdim, gstride,
            box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return fail(err, err_len, GPUM_ERR_INVALID, "cuTensorMapEncodeTiled rejected the data");
  }
  TmapDesc tmap;
  std::memcpy(&tmap, &tm, sizeof tm);

  float* d_params = reinterpret_cast<float*>(base + off_params);
  double* d_part = reinterpret_cast<double*>(base + off_part);
  EvalArgs E{};
  E.n_obs = (int)n_obs;
  E.ncols = (int)n_cols;
  E.T = T;
  E.ntiles = ntiles;
  E.tiles_per_cta = tiles_per_cta;
  E.CG = CG;
  E.WC = WC;
  E.C_pad = C_pad;
  E.np = (int)n_params;
  E.width = 1;
  E.params = d_params;
  E.partials = d_part;
  E.n_points = n;
  E.tickets = nullptr;  // PH_EVAL takes no ticket
  E.err = d_err;
  ChainArgs A{};

  if (cudaMemsetAsync(d_err, 0, sizeof(uint32_t), st) != cudaSuccess)
    return fail(err, err_len, GPUM_ERR_CUDA, "clearing the scratch error word failed");
  const int total = (int)(n_params * C_pad);
  points_to_params_kernel<<<(total + 255) / 256, 256, 0, st>>>(d_points, d_params, n,
                                                               (int)n_params, C_pad);
  const dim3 grid(NCB, nob);
  switch (G) {
    case 8: iter_kernel<8, 8><<<grid, kThreads, smem, st>>>(prog, tmap, E, A, PH_EVAL); break;
    case 4: iter_kernel<4, 16><<<grid, kThreads, smem, st>>>(prog, tmap, E, A, PH_EVAL); break;
    default: iter_kernel<2, 32><<<grid, kThreads, smem, st>>>(prog, tmap, E, A, PH_EVAL); break;
  }
  reduce_partials_kernel<<<(n + 255) / 256, 256, 0, st>>>(d_part, d_out, nob, C_pad, n, 1);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    if (err && err_len) std::snprintf(err, err_len, "launch failed: %s", cudaGetErrorString(e));
    return GPUM_ERR_CUDA;
  }
  // The call returns once the results are in d_out, so that a device-side
  // failure recorded in the scratch error word is reported here.
  uint32_t dev_err = 0;
  e = cudaMemcpyAsync(&dev_err, d_err, sizeof dev_err, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    if (err && err_len) std::snprintf(err, err_len, "stream failed: %s", cudaGetErrorString(e));
    return GPUM_ERR_CUDA;
  }
  if (dev_err) {
    if (err && err_len)
      std::snprintf(err, err_len, "a kernel reported a device-side failure (code %u)", dev_err);
    return GPUM_ERR_DEVICE;
  }
  return GPUM_OK;
}
