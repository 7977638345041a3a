// capi.cu -- host side of the B200 backend: sessions (model + data resident
// in HBM), the two evaluation engines, launch geometry, CUDA-graph replay of
// the iteration loop, and the extern "C" entry points of include/gpum_b200.h.
//
// Replaces the reference's per-call CubeCL client + upload + launch +
// readback (src/rust/src/chain_kernel.rs:372-463) and its backend dispatch
// (chain_kernel.rs:469-532).  No entry point throws across the ABI: every
// failure becomes a status code and a message.
//
// Engines:
//   interpreter -- the register-stack bytecode interpreter (interp.cuh), the
//                  micro-op stream in the constant bank; compiled ahead of
//                  time, works for every valid program;
//   compiled    -- the program translated to straight-line CUDA C
//                  (codegen.cpp) and built by NVRTC for sm_100a at session
//                  creation (jit.cpp); required for gradients (MALA,
//                  grad_batch).
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/gpum_b200.h"
#include "codegen.hpp"
#include "jit.hpp"
#include "kernels.cuh"
#include "program.hpp"

using namespace gpum;

namespace gpum {
// Surrogate inference on device parameters (mlp.cu).
int mlp_infer(gpum_b200_mlp* m, const double* theta, int n, int d, double* out, cudaStream_t st,
              std::string* err);
int mlp_infer_launches(const gpum_b200_mlp* m, int n);
int mlp_infer_grad(gpum_b200_mlp* m, const double* theta, int n, int d, double* out_val,
                   double* out_grad, cudaStream_t st, std::string* err);
int mlp_infer_grad_launches(const gpum_b200_mlp* m, int n);
int mlp_train_device(gpum_b200_mlp* m, const float* dth, const double* dll, size_t n_pairs,
                     uint32_t n_stages, const uint32_t* steps, const double* lrs,
                     float* out_loss, std::string* err);
int mlp_input_width(const gpum_b200_mlp* m);
}  // namespace gpum

static_assert(sizeof(CUtensorMap) == sizeof(TmapDesc), "tensor map size");

namespace {

struct Failure {
  int code;
  std::string msg;
};

void set_err(char* err, size_t len, const std::string& m) {
  if (err && len) {
    const size_t n = std::min(len - 1, m.size());
    std::memcpy(err, m.data(), n);
    err[n] = '\0';
  }
}

#define GPUM_CK(call)                                                                 \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      throw Failure{e_ == cudaErrorMemoryAllocation ? GPUM_ERR_NOMEM : GPUM_ERR_CUDA, \
                    std::string(#call) + ": " + cudaGetErrorString(e_)};             \
  } while (0)

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  void ensure(size_t count) {
    if (count <= n && p) return;
    release();
    if (count == 0) count = 1;
    GPUM_CK(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DBuf() { release(); }
};

using EncodeTiledFn = PFN_cuTensorMapEncodeTiled_v12000;

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
      throw Failure{GPUM_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable"};
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// Static shared memory of a kernel (the interpreter's operand scratch): with
// it, a dynamic request below 48 KB can still need the opt-in attribute.
size_t static_smem(const void* fn) {
  cudaFuncAttributes fa{};
  return cudaFuncGetAttributes(&fa, fn) == cudaSuccess ? fa.sharedSizeBytes : 0;
}

// Interpreter variants by peak stack depth: registers go to depth or to
// chains per thread.
enum Variant { V8x8 = 0, V4x16 = 1, V2x32 = 2, V16x6 = 3 };
int variant_G(int v) { return v == V16x6 ? 16 : v == V8x8 ? 8 : (v == V4x16 ? 4 : 2); }
int choose_variant(const UProg& p) {
  if (p.depth <= 6 && p.n_saves <= 1) return V16x6;
  return p.depth <= 8 ? V8x8 : (p.depth <= 16 ? V4x16 : V2x32);
}

const void* interp_kernel(int v) {
  switch (v) {
    case V16x6: return (const void*)iter_kernel<16, 6>;
    case V8x8: return (const void*)iter_kernel<8, 8>;
    case V4x16: return (const void*)iter_kernel<4, 16>;
    default: return (const void*)iter_kernel<2, 32>;
  }
}

void launch_interp(int v, dim3 grid, size_t smem, cudaStream_t st, const EvalProg& prog,
                   const TmapDesc& tmap, const EvalArgs& E, const ChainArgs& A, int phase) {
  switch (v) {
    case V16x6: iter_kernel<16, 6><<<grid, kThreads, smem, st>>>(prog, tmap, E, A, phase); break;
    case V8x8: iter_kernel<8, 8><<<grid, kThreads, smem, st>>>(prog, tmap, E, A, phase); break;
    case V4x16: iter_kernel<4, 16><<<grid, kThreads, smem, st>>>(prog, tmap, E, A, phase); break;
    default: iter_kernel<2, 32><<<grid, kThreads, smem, st>>>(prog, tmap, E, A, phase); break;
  }
  GPUM_CK(cudaGetLastError());
}

// Interpreter gradient kernels by width (1 + parameters, rounded up).
int grad_width(uint32_t np) {
  const int w = 1 + (int)np;
  return w <= 9 ? 9 : (w <= 17 ? 17 : (w <= 33 ? 33 : (w <= 65 ? 65 : 129)));
}

const void* interp_grad_kernel(int W) {
  switch (W) {
    case 9: return (const void*)iter_kernel_grad<9>;
    case 17: return (const void*)iter_kernel_grad<17>;
    case 33: return (const void*)iter_kernel_grad<33>;
    case 65: return (const void*)iter_kernel_grad<65>;
    default: return (const void*)iter_kernel_grad<129>;
  }
}

void launch_interp_grad(int W, dim3 grid, size_t smem, cudaStream_t st, const GradProg& prog,
                        const TmapDesc& tmap, const EvalArgs& E, const ChainArgs& A, int phase) {
  switch (W) {
    case 9: iter_kernel_grad<9><<<grid, kThreads, smem, st>>>(prog, tmap, E, A, phase); break;
    case 17: iter_kernel_grad<17><<<grid, kThreads, smem, st>>>(prog, tmap, E, A, phase); break;
    case 33: iter_kernel_grad<33><<<grid, kThreads, smem, st>>>(prog, tmap, E, A, phase); break;
    case 65: iter_kernel_grad<65><<<grid, kThreads, smem, st>>>(prog, tmap, E, A, phase); break;
    default: iter_kernel_grad<129><<<grid, kThreads, smem, st>>>(prog, tmap, E, A, phase); break;
  }
  GPUM_CK(cudaGetLastError());
}

int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// Which kernel evaluates the current run or batch.
struct KernelChoice {
  bool compiled = false;
  const void* fn = nullptr;  // __global__ pointer or cudaKernel_t
  int G = 8;                 // chains per thread (per warp for a chain-lane body)
  int W = 1;                 // values per chain (1, or 1 + np with the gradient)
  bool lanes = false;        // chain-lane body: G = 32 chains per warp group
  bool grad_interp = false;  // the interpreter engine's gradient (tape) kernel
  bool tc = false;           // the compiled engine's tensor-core value kernel
  int threads = kThreads;    // threads per CTA
};

struct Geometry {
  int G, WC, CG, NCB, C_pad, NOB, tiles_per_cta, ntiles;
  size_t smem;
};


}  // namespace

// Tensor map of column-major f32 data (n_cols columns of leading dimension
// ld >= n_obs, a multiple of 4): boxes of T observations x all columns.
void encode_cols_tmap(float* base, uint64_t n_obs, uint32_t n_cols, int64_t ld, int T,
                      TmapDesc* out) {
  CUtensorMap tm;
  cuuint64_t gdim[2] = {(cuuint64_t)n_obs, (cuuint64_t)n_cols};
  cuuint64_t gstride[1] = {(cuuint64_t)ld * sizeof(float)};
  cuuint32_t box[2] = {(cuuint32_t)T, (cuuint32_t)n_cols};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, gdim, gstride, box,
                           estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    throw Failure{GPUM_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(r) + ")"};
  std::memcpy(out, &tm, sizeof tm);
}

struct gpum_b200_session {
  cudaStream_t stream = nullptr;
  UProg ll;
  std::unique_ptr<EvalProg> prog;
  // the interpreter engine's gradient program (or why there is none)
  std::unique_ptr<GradProg> gprog;
  std::string gprog_err;
  GenModel gm;
  CompiledModel cm;
  bool cm_ready = false;
  std::string cm_error;
  int engine = GPUM_ENGINE_AUTO;
  std::vector<uint32_t> prior_code;
  std::vector<double> prior_consts;
  uint32_t np = 0, ncols = 0;
  uint64_t n_obs = 0;
  int variant = V8x8;
  int T = 256;
  int64_t ld = 0;
  DBuf<float> data;
  TmapDesc tmap;
  // The compiled engine's data when its model materializes data-only
  // operations (cm.n_mat > 0): the data columns, then one column per
  // operation, with its own tile height and tensor map.
  DBuf<float> data_c;
  TmapDesc tmap_c;
  int T_c = 256;
  uint32_t ncols_c = 0;
  // The compiled engine's tensor-core value path (cm.tc): the data packed
  // as [hi | lo | tail] tiles once per session; off when a product column
  // holds a non-finite value or GPUM_B200_TENSOR_CORES=0.
  DBuf<float> tc_data;
  DBuf<uint32_t> tc_flag;
  bool tc_ok = false;
  DBuf<uint32_t> d_prior_code;
  DBuf<double> d_prior_consts;
  DBuf<uint32_t> d_err;
  // run state
  KernelChoice kc;
  Geometry geo{};
  int n_chains = 0;
  uint32_t max_iter = 0, n_done = 0;
  bool prepared = false;
  DBuf<double> state, prop, cur, last_eval, sd, temp, L, snap, zbuf, partials, pointwise,
      points, out64, gx, gy, mx, my, vbuf;
  DBuf<float> params, draws, draws_out;
  DBuf<uint32_t> ctr, accepts, iter, tickets, ptape_i;
  DBuf<double> ptape;
  EvalArgs E{};
  ChainArgs A{};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int graph_len = 0;
  uint64_t graph_launches = 0;  // kernel nodes per graph replay
  uint64_t launches = 0;
  // Training pairs for the surrogate (exact runs only).
  DBuf<float> rec_theta;
  DBuf<double> rec_ll;
  uint64_t rec_cap = 0, rec_count = 0;
  // Delayed acceptance.
  DBuf<double> sll_x, sll_y, prior_x, prior_y, da_partials, da_gs, da_tvals, da_tadj;
  DBuf<uint32_t> da_flag, da_slot, da_active, da_iter, da_stage1, da_tlhs, da_trhs;
  DBuf<float> da_params;
  Geometry geo_da{};
  EvalArgs E_da{};
  DaArgs D{};
  gpum_b200_mlp* da_mlp = nullptr;
  int da_mlp_launches = 0;  // kernel launches per surrogate call
  DBuf<double> mom;  // draw moments scratch
  // Replica exchange on the device (0 = off).
  int pt_K = 0, pt_every = 0;
  DBuf<uint32_t> pt_att, pt_acc, pt_n;
  // Per-chain likelihood powers for later runs (power posteriors).
  DBuf<double> beta;
  size_t n_beta = 0;

  ~gpum_b200_session() {
    drop_graph();
    if (stream) cudaStreamDestroy(stream);
  }

  void drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    gexec = nullptr;
    graph = nullptr;
  }

  // Builds the compiled engine once; false (with cm_error) when NVRTC is
  // unavailable or the build fails.
  bool compiled_available() {
    if (cm_ready) return true;
    if (!cm_error.empty()) return false;
    std::string e;
    if (jit_compile(gm, &cm, &e)) {
      cm_error = e.empty() ? "compiled engine unavailable" : e;
      return false;
    }
    if (cm.n_mat > 0 && ncols > 0 && n_obs > 0) materialize();
    if (cm.tc && n_obs > 0 && tensor_cores_enabled()) {
      // Without room for the packed copy the session keeps the FP32 kernel.
      try {
        pack_tc();
      } catch (const Failure& f) {
        if (f.code != GPUM_ERR_NOMEM) throw;
        cudaGetLastError();  // an allocation failure is not sticky
        tc_data.release();
        tc_ok = false;
      }
    }
    cm_ready = true;
    return true;
  }

  static bool tensor_cores_enabled() {
    const char* e = std::getenv("GPUM_B200_TENSOR_CORES");
    return !(e && e[0] == '0');
  }

  // The tensor-core value kernel's operand B, once per session: every tile
  // of tc_tn observations as [hi | lo] product columns in the MMA's
  // core-matrix layout and the tail columns (gm_tc_pack).
  void pack_tc() {
    const long long tn = cm.tc_tn;
    long long ntl = (long long)((n_obs + (uint64_t)tn - 1) / (uint64_t)tn);
    const size_t stage = (size_t)(2 * cm.tc_kp + cm.tc_ntail) * (size_t)tn;
    tc_data.ensure(stage * (size_t)ntl);
    tc_flag.ensure(1);
    GPUM_CK(cudaMemsetAsync(tc_flag.p, 0, sizeof(uint32_t), stream));
    const float* cols = cm.n_mat > 0 ? data_c.p : data.p;
    long long nobs = (long long)n_obs, lld = (long long)ld;
    float* xt = tc_data.p;
    uint32_t* flag = tc_flag.p;
    void* args[] = {(void*)&cols, (void*)&nobs, (void*)&lld, (void*)&ntl, (void*)&xt,
                    (void*)&flag};
    GPUM_CK(cudaLaunchKernel((const void*)cm.k_tc_pack,
                             dim3((unsigned)((ntl * tn + 255) / 256)), dim3(256), args, 0,
                             stream));
    ++launches;
    uint32_t bad = 0;
    GPUM_CK(cudaMemcpyAsync(&bad, tc_flag.p, sizeof bad, cudaMemcpyDeviceToHost, stream));
    GPUM_CK(cudaStreamSynchronize(stream));
    tc_ok = bad == 0;
    if (!tc_ok) tc_data.release();
  }

  // Extra columns for the compiled model's data-only operations, computed
  // once on the device by the model's own gm_materialize.
  void materialize() {
    ncols_c = ncols + (uint32_t)cm.n_mat;
    T_c = tile_obs(ncols_c);
    data_c.ensure((size_t)ld * ncols_c);
    GPUM_CK(cudaMemcpyAsync(data_c.p, data.p, sizeof(float) * (size_t)ld * ncols,
                            cudaMemcpyDeviceToDevice, stream));
    float* cols = data_c.p;
    long long nobs = (long long)n_obs, lld = (long long)ld;
    void* args[] = {(void*)&cols, (void*)&nobs, (void*)&lld};
    GPUM_CK(cudaLaunchKernel((const void*)cm.k_mat, dim3((unsigned)((n_obs + 255) / 256)),
                             dim3(256), args, 0, stream));
    ++launches;
    encode_cols_tmap(data_c.p, n_obs, ncols_c, ld, T_c, &tmap_c);
    GPUM_CK(cudaStreamSynchronize(stream));
  }
  bool ext(const KernelChoice& k) const { return k.compiled && cm.n_mat > 0; }

  // `pointwise`: per-observation output, which the tensor-core value kernel
  // does not write.
  KernelChoice choose(bool need_grad, bool pointwise = false) {
    KernelChoice k;
    // Gradients: the compiled engine's adjoint unless the interpreter engine
    // was chosen or NVRTC cannot build the model; then the interpreted tape.
    if (need_grad && (engine == GPUM_ENGINE_INTERP ||
                      (engine == GPUM_ENGINE_AUTO && !compiled_available()))) {
      if (!gprog)
        throw Failure{GPUM_ERR_UNSUPPORTED,
                      "the interpreter engine's gradient is unavailable (" + gprog_err +
                          ")" + (cm_error.empty() ? "" : "; compiled engine: " + cm_error)};
      k.compiled = false;
      k.grad_interp = true;
      k.W = grad_width(np);
      k.fn = interp_grad_kernel(k.W);
      k.G = 1;
      return k;
    }
    const bool want_compiled =
        need_grad || engine == GPUM_ENGINE_COMPILED ||
        (engine == GPUM_ENGINE_AUTO && compiled_available());
    if (want_compiled) {
      if (!compiled_available())
        throw Failure{GPUM_ERR_UNSUPPORTED,
                      std::string(need_grad ? "gradients need" : "engine=compiled needs") +
                          " the compiled engine: " + cm_error};
      k.compiled = true;
      k.fn = need_grad ? (const void*)cm.k_grad : (const void*)cm.k_value;
      k.lanes = need_grad ? cm.lanes_grad : cm.lanes;
      k.G = k.lanes ? 32 : (need_grad ? cm.GG : cm.G);
      k.W = need_grad ? 1 + (int)np : 1;
      if (!need_grad && !pointwise && tc_ok) {
        k.tc = true;
        k.fn = (const void*)cm.k_value_tc;
        k.lanes = false;
        k.G = kTcM;
        k.threads = cm.tc_threads;
      }
    } else {
      k.compiled = false;
      k.fn = interp_kernel(variant);
      k.G = variant_G(variant);
      k.W = 1;
    }
    return k;
  }

  Geometry geometry(int n, const KernelChoice& k) const {
    Geometry g{};
    g.G = k.G;
    const int groups = (n + g.G - 1) / g.G;
    g.WC = 1;
    while (!k.tc && g.WC < kWarps && g.WC < groups) g.WC *= 2;
    g.CG = g.WC * g.G;
    g.NCB = (n + g.CG - 1) / g.CG;
    g.C_pad = g.NCB * g.CG;
    const int Tk = k.tc ? cm.tc_tn : (ext(k) ? T_c : T);
    g.ntiles = (int)((n_obs + Tk - 1) / Tk);
    g.smem = k.tc ? tc_smem_bytes(cm.tc_kp, cm.tc_ntail, cm.tc_tn, cm.tc_stages)
                  : skel_smem_bytes(Tk, (int)(ext(k) ? ncols_c : ncols), (int)np, g.CG, g.G,
                                    k.W, k.lanes);
    int occ = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k.fn, k.threads, g.smem);
    if (occ < 1) occ = 1;
    const int slots = num_sms() * occ;
    int nob = std::max(1, (4 * slots) / g.NCB);
    nob = std::min(nob, std::max(1, g.ntiles));
    g.tiles_per_cta = g.ntiles > 0 ? (g.ntiles + nob - 1) / nob : 0;
    g.NOB = g.ntiles > 0 ? (g.ntiles + g.tiles_per_cta - 1) / g.tiles_per_cta : 1;
    return g;
  }

  void check_device_error() {
    uint32_t e = 0;
    GPUM_CK(cudaMemcpyAsync(&e, d_err.p, sizeof e, cudaMemcpyDeviceToHost, stream));
    GPUM_CK(cudaStreamSynchronize(stream));
    if (e) {
      GPUM_CK(cudaMemsetAsync(d_err.p, 0, sizeof(uint32_t), stream));
      throw Failure{GPUM_ERR_DEVICE, "a kernel reported a device-side failure (code " +
                                         std::to_string(e) + ")"};
    }
  }

  // Evaluation-argument block for `n` points (params in `params`).
  void setup_eval(int n, bool need_grad, bool pointwise = false) {
    kc = choose(need_grad, pointwise);
    geo = geometry(n, kc);
    if (geo.smem + static_smem(kc.fn) > 48 * 1024)
      GPUM_CK(cudaFuncSetAttribute(kc.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)geo.smem));
    params.ensure((size_t)np * geo.C_pad);
    partials.ensure((size_t)geo.NOB * geo.C_pad * kc.W);
    tickets.ensure(geo.NCB);
    GPUM_CK(cudaMemsetAsync(tickets.p, 0, sizeof(uint32_t) * geo.NCB, stream));
    E = EvalArgs{};
    E.n_obs = (int)n_obs;
    E.ncols = (int)(ext(kc) ? ncols_c : ncols);
    E.T = kc.tc ? cm.tc_tn : (ext(kc) ? T_c : T);
    E.ntiles = geo.ntiles;
    E.tiles_per_cta = geo.tiles_per_cta;
    E.CG = geo.CG;
    E.WC = geo.WC;
    E.C_pad = geo.C_pad;
    E.np = (int)np;
    E.width = kc.W;
    E.params = params.p;
    E.partials = partials.p;
    E.n_points = n;
    E.tickets = tickets.p;
    E.err = d_err.p;
  }

  void upload_points(const double* pts, int n) {
    points.ensure((size_t)n * np);
    GPUM_CK(cudaMemcpyAsync(points.p, pts, sizeof(double) * n * np, cudaMemcpyHostToDevice,
                            stream));
    const int total = (int)(np * geo.C_pad);
    points_to_params_kernel<<<(total + 255) / 256, 256, 0, stream>>>(points.p, params.p, n,
                                                                     (int)np, geo.C_pad);
    GPUM_CK(cudaGetLastError());
    ++launches;
  }

  void launch(int phase) { launch_with(geo, E, phase); }

  // One Metropolis iteration: for path-B DE the proposals of the generation
  // come first, in their own kernel (every chain reads the population).
  void step() {
    if (A.mode == MODE_DESYNC) {
      desync_propose_kernel<<<(unsigned)((n_chains + 127) / 128), 128, 0, stream>>>(
          A, params.p, geo.C_pad);
      GPUM_CK(cudaGetLastError());
      ++launches;
    }
    launch(PH_STEP);
    if (pt_K > 0) {
      PtArgs P{pt_K, pt_every, A.iter, nullptr, nullptr, pt_n.p, pt_att.p, pt_acc.p,
               params.p, geo.C_pad};
      pt_exchange_kernel<<<(unsigned)((n_chains + 127) / 128), 128, 0, stream>>>(A, P);
      GPUM_CK(cudaGetLastError());
      ++launches;
    }
  }

  void launch_with(const Geometry& g, EvalArgs& e, int phase) {
    const dim3 grid(g.NCB, g.NOB);
    if (kc.tc) {
      void* args[] = {(void*)&tc_data.p, (void*)&e, (void*)&A, (void*)&phase};
      GPUM_CK(cudaLaunchKernel(kc.fn, grid, dim3(kc.threads), args, g.smem, stream));
    } else if (kc.compiled) {
      void* args[] = {(void*)(ext(kc) ? &tmap_c : &tmap), (void*)&e, (void*)&A, (void*)&phase};
      GPUM_CK(cudaLaunchKernel(kc.fn, grid, dim3(kThreads), args, g.smem, stream));
    } else if (kc.grad_interp) {
      launch_interp_grad(kc.W, grid, g.smem, stream, *gprog, tmap, e, A, phase);
    } else {
      launch_interp(variant, grid, g.smem, stream, *prog, tmap, e, A, phase);
    }
    ++launches;
  }

  // Pairs recorded so far, after `n_done` iterations of the prepared run.
  void settle_recording() {
    if (A.rec_ll && prepared)
      rec_count = std::min<uint64_t>(rec_cap, A.rec_base + (uint64_t)n_done * n_chains);
  }
};

namespace {

// Runs `body`, converting every failure into a status code and message.
int guard(char* err, size_t len, const std::function<void()>& body) {
  try {
    body();
    set_err(err, len, "");
    return GPUM_OK;
  } catch (const Failure& f) {
    set_err(err, len, f.msg);
    return f.code;
  } catch (const std::bad_alloc&) {
    set_err(err, len, "host allocation failed");
    return GPUM_ERR_NOMEM;
  } catch (...) {
    set_err(err, len, "unexpected internal error");
    return GPUM_ERR_CUDA;
  }
}

void require(bool ok, const std::string& m, int code = GPUM_ERR_INVALID) {
  if (!ok) throw Failure{code, m};
}

void require_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
    cudaGetLastError();
    throw Failure{GPUM_ERR_NODEVICE, "no CUDA device is visible"};
  }
  int dev = 0, major = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (major != 10)
    throw Failure{GPUM_ERR_NODEVICE,
                  "the b200 backend needs an sm_100 (B200) GPU; found compute capability " +
                      std::to_string(major) + ".x"};
}

// Validation and code generation shared by sessions and the compile check.
void check_model(const uint32_t* code, size_t n_code, const double* consts, size_t n_consts,
                 const uint32_t* prior_code, size_t n_prior, const double* prior_consts,
                 size_t n_prior_consts, uint32_t n_params, uint32_t n_cols, UProg* ll,
                 GenModel* gm) {
  require(n_params >= 1, "n_params must be at least 1");
  require(n_params <= 256, "more than 256 parameters", GPUM_ERR_UNSUPPORTED);
  require(n_cols <= 256, "more than 256 data columns", GPUM_ERR_UNSUPPORTED);
  std::string msg;
  if (compile_program(code, n_code, consts, n_consts, n_params, n_cols, true, ll, &msg))
    throw Failure{GPUM_ERR_INVALID, "log-likelihood bytecode: " + msg};
  int pdepth = 0;
  if (validate_program(prior_code, n_prior, n_prior_consts, n_params, 0, false, &pdepth, &msg))
    throw Failure{GPUM_ERR_INVALID, "prior bytecode: " + msg};
  require(n_prior_consts == 0 || prior_consts != nullptr, "prior constant pointer is NULL");
  if (generate_model(code, n_code, consts, prior_code, n_prior, prior_consts, n_params, n_cols,
                     gm, &msg))
    throw Failure{GPUM_ERR_INVALID, "code generation: " + msg};
}

gpum_b200_session* create_session(const uint32_t* code, size_t n_code, const double* consts,
                                  size_t n_consts, const uint32_t* prior_code, size_t n_prior,
                                  const double* prior_consts, size_t n_prior_consts,
                                  uint32_t n_params, const double* data, uint32_t n_cols,
                                  uint64_t n_obs) {
  require(n_obs < (1ull << 31) - 1024, "more than 2^31 observations", GPUM_ERR_UNSUPPORTED);
  require(n_obs == 0 || n_cols == 0 || data != nullptr, "data pointer is NULL");
  std::unique_ptr<gpum_b200_session> s(new gpum_b200_session());
  check_model(code, n_code, consts, n_consts, prior_code, n_prior, prior_consts, n_prior_consts,
              n_params, n_cols, &s->ll, &s->gm);
  require_device();

  s->np = n_params;
  s->ncols = n_cols;
  s->n_obs = n_obs;
  s->variant = choose_variant(s->ll);
  s->prog.reset(new EvalProg());
  std::memset(s->prog.get(), 0, sizeof(EvalProg));
  s->prog->n_uops = (uint32_t)s->ll.uops.size();
  std::copy(s->ll.uops.begin(), s->ll.uops.end(), s->prog->uop);
  std::copy(s->ll.terms.begin(), s->ll.terms.end(), s->prog->term);
  std::copy(s->ll.consts.begin(), s->ll.consts.end(), s->prog->cst);
  {
    UGradProg gp;
    std::string ge;
    if (compile_grad_program(code, n_code, n_params, &gp, &ge) == 0) {
      s->gprog.reset(new GradProg());
      std::memset(s->gprog.get(), 0, sizeof(GradProg));
      s->gprog->n_nodes = (uint32_t)gp.nodes.size();
      s->gprog->root = gp.root;
      s->gprog->has_root = gp.has_root ? 1u : 0u;
      s->gprog->np = n_params;
      std::copy(gp.nodes.begin(), gp.nodes.end(), s->gprog->node);
      std::copy(s->ll.consts.begin(),
                s->ll.consts.begin() + std::min<size_t>(n_consts, (size_t)kMaxConsts),
                s->gprog->cst);
    } else {
      s->gprog_err = ge;
    }
  }
  s->prior_code.assign(prior_code, prior_code + n_prior);
  s->prior_consts.assign(prior_consts, prior_consts + n_prior_consts);

  GPUM_CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  s->d_err.ensure(1);
  GPUM_CK(cudaMemsetAsync(s->d_err.p, 0, sizeof(uint32_t), s->stream));
  s->d_prior_code.ensure(std::max<size_t>(n_prior, 2));
  s->d_prior_consts.ensure(std::max<size_t>(n_prior_consts, 1));
  if (n_prior)
    GPUM_CK(cudaMemcpyAsync(s->d_prior_code.p, prior_code, n_prior * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, s->stream));
  if (n_prior_consts)
    GPUM_CK(cudaMemcpyAsync(s->d_prior_consts.p, prior_consts, n_prior_consts * sizeof(double),
                            cudaMemcpyHostToDevice, s->stream));

  // Observations per tile: a multiple of 32 (one per lane), <= 256 (TMA box
  // limit), with a stage of at most 32 KB.
  if (n_cols > 0) {
    s->T = tile_obs(n_cols);
  } else {
    s->T = 256;
  }
  std::memset(&s->tmap, 0, sizeof s->tmap);
  if (n_cols > 0 && n_obs > 0) {
    // Column-major f32 in HBM: each column contiguous, leading dimension
    // padded to 4 floats so every TMA row stride is a multiple of 16 bytes.
    s->ld = (int64_t)((n_obs + 3) & ~3ull);
    s->data.ensure((size_t)s->ld * n_cols);
    // f64 rows through a 16 MB staging buffer (2M values per chunk; the
    // copy of a chunk follows the conversion of the previous one on the
    // stream), so a session does not allocate a second full copy.
    const int64_t rows_per_chunk = std::max<int64_t>(1, (int64_t)(2u << 20) / n_cols);
    DBuf<double> stage;
    stage.ensure((size_t)std::min<int64_t>(rows_per_chunk, (int64_t)n_obs) * n_cols);
    for (int64_t r0 = 0; r0 < (int64_t)n_obs; r0 += rows_per_chunk) {
      const int64_t nr = std::min<int64_t>(rows_per_chunk, (int64_t)n_obs - r0);
      GPUM_CK(cudaMemcpyAsync(stage.p, data + r0 * n_cols, sizeof(double) * nr * n_cols,
                              cudaMemcpyHostToDevice, s->stream));
      const int64_t tot = nr * n_cols;
      convert_rows_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s->stream>>>(
          stage.p, s->data.p, (int)n_cols, s->ld, r0, nr);
      GPUM_CK(cudaGetLastError());
    }
    GPUM_CK(cudaStreamSynchronize(s->stream));
    encode_cols_tmap(s->data.p, n_obs, n_cols, s->ld, s->T, &s->tmap);
  }
  return s.release();
}

void prepare(gpum_b200_session* s, const double* init, const double* sd, const double* temps,
             uint32_t C, uint32_t max_iter, uint32_t seed, uint32_t mode, double gamma,
             double de_noise, const double* L, size_t n_l, int rng) {
  require(s != nullptr, "session is NULL");
  require(C >= 1, "n_chains must be at least 1");
  require(init && sd && temps, "init, proposal_sd and temperatures must be non-NULL");
  require(mode <= 4,
          "proposal_mode must be 0 (rwm), 1 (de), 2 (cholesky), 3 (mala) or 4 (de_sync)");
  require(mode != 4 || C >= 3, "de_sync needs at least 3 chains (two distinct partners)");
  require(rng == GPUM_RNG_TRIPLE32 || rng == GPUM_RNG_PHILOX, "rng must be 0 or 1");
  const size_t np = s->np;
  const bool mala = mode == 3;
  const bool use_L = mode == 2 || (mala && L != nullptr && n_l > 0);
  if (mode == 2)
    require(L != nullptr && n_l == (size_t)C * np * np,
            "proposal_mode 2 needs proposal_l of n_chains*n_params^2 values");
  if (mala && use_L)
    require(n_l == (size_t)C * np * np, "proposal_l must hold n_chains*n_params^2 values");
  require(C <= (1u << 24), "more than 2^24 chains", GPUM_ERR_UNSUPPORTED);
  require((uint64_t)max_iter * np * C <= (1ull << 33), "draw storage above 32 GiB",
          GPUM_ERR_UNSUPPORTED);

  s->settle_recording();
  s->drop_graph();
  s->prepared = false;
  s->n_chains = (int)C;
  s->setup_eval((int)C, mala);
  const Geometry& g = s->geo;
  s->state.ensure(C * np);
  s->prop.ensure(C * np);
  s->snap.ensure(C * np);
  s->sd.ensure(C * np);
  s->zbuf.ensure(C * np);
  s->temp.ensure(C);
  s->cur.ensure(C);
  s->last_eval.ensure(C);
  s->ctr.ensure(C);
  s->accepts.ensure(C);
  s->iter.ensure(g.NCB);
  s->draws.ensure(std::max<size_t>(1, (size_t)max_iter * np * g.C_pad));
  if (use_L) s->L.ensure((size_t)C * np * np);
  if (mala) {
    s->gx.ensure(C * np);
    s->gy.ensure(C * np);
    s->mx.ensure(C * np);
    s->my.ensure(C * np);
    s->vbuf.ensure(C * np);
    if (!s->kc.compiled) {  // the interpreted prior's gradient tape
      const size_t npr = std::max<size_t>(s->prior_code.size() / 2, 1);
      s->ptape.ensure((size_t)C * 2 * npr);
      s->ptape_i.ensure((size_t)C * 2 * npr);
    }
  }
  cudaStream_t st = s->stream;
  GPUM_CK(cudaMemcpyAsync(s->state.p, init, sizeof(double) * C * np, cudaMemcpyHostToDevice, st));
  GPUM_CK(cudaMemcpyAsync(s->snap.p, s->state.p, sizeof(double) * C * np,
                          cudaMemcpyDeviceToDevice, st));
  GPUM_CK(cudaMemcpyAsync(s->sd.p, sd, sizeof(double) * C * np, cudaMemcpyHostToDevice, st));
  GPUM_CK(cudaMemcpyAsync(s->temp.p, temps, sizeof(double) * C, cudaMemcpyHostToDevice, st));
  if (use_L)
    GPUM_CK(cudaMemcpyAsync(s->L.p, L, sizeof(double) * C * np * np, cudaMemcpyHostToDevice, st));
  GPUM_CK(cudaMemsetAsync(s->ctr.p, 0, sizeof(uint32_t) * C, st));
  GPUM_CK(cudaMemsetAsync(s->accepts.p, 0, sizeof(uint32_t) * C, st));
  GPUM_CK(cudaMemsetAsync(s->iter.p, 0, sizeof(uint32_t) * g.NCB, st));
  const int total = (int)(np * g.C_pad);
  points_to_params_kernel<<<(total + 255) / 256, 256, 0, st>>>(s->state.p, s->params.p, (int)C,
                                                               (int)np, g.C_pad);
  GPUM_CK(cudaGetLastError());
  ++s->launches;

  ChainArgs& A = s->A;
  A = ChainArgs{};
  A.n_chains = (int)C;
  A.np = (int)np;
  A.state = s->state.p;
  A.prop = s->prop.p;
  A.cur = s->cur.p;
  A.last_eval = s->last_eval.p;
  A.ctr = s->ctr.p;
  A.accepts = s->accepts.p;
  A.iter = s->iter.p;
  A.sd = s->sd.p;
  A.temp = s->temp.p;
  A.L = use_L ? s->L.p : nullptr;
  A.snap = s->snap.p;
  A.draws = s->draws.p;
  A.n_iter = max_iter;
  A.seed = seed;
  A.mode = mode == 0 ? MODE_RWM
         : mode == 2 ? MODE_CHOL
         : mala      ? MODE_MALA
         : mode == 4 ? MODE_DESYNC
                     : MODE_DE;
  A.rng = rng;
  A.gamma = gamma;
  A.de_noise = de_noise;
  A.prior_code = s->d_prior_code.p;
  A.prior_consts = s->d_prior_consts.p;
  A.n_prior = (int)(s->prior_code.size() / 2);
  A.zbuf = s->zbuf.p;
  if (mala) {
    A.gx = s->gx.p;
    A.gy = s->gy.p;
    A.mx = s->mx.p;
    A.my = s->my.p;
    A.vbuf = s->vbuf.p;
    if (!s->kc.compiled) {
      A.ptape = s->ptape.p;
      A.ptape_i = s->ptape_i.p;
    }
  }
  if (s->n_beta > 0) {
    require(s->n_beta == C, "likelihood powers were set for " + std::to_string(s->n_beta) +
                                " chains, the run has " + std::to_string(C));
    A.beta = s->beta.p;
  }
  if (s->pt_K > 0) {
    require(C % (uint32_t)s->pt_K == 0,
            "n_chains must be a multiple of the ladder length for device exchanges");
    require(mode != 4, "device exchanges are not available with de_sync");
    s->pt_att.ensure(C);
    s->pt_acc.ensure(C);
    s->pt_n.ensure(1);
    GPUM_CK(cudaMemsetAsync(s->pt_att.p, 0, sizeof(uint32_t) * C, st));
    GPUM_CK(cudaMemsetAsync(s->pt_acc.p, 0, sizeof(uint32_t) * C, st));
    GPUM_CK(cudaMemsetAsync(s->pt_n.p, 0, sizeof(uint32_t), st));
  }
  if (s->rec_cap > 0) {
    A.rec_theta = s->rec_theta.p;
    A.rec_ll = s->rec_ll.p;
    A.rec_base = s->rec_count;
    A.rec_cap = s->rec_cap;
  }
  s->launch(PH_INIT);
  s->max_iter = max_iter;
  s->n_done = 0;
  s->prepared = true;
}

void advance(gpum_b200_session* s, uint32_t n) {
  require(s && s->prepared, "session has no prepared run");
  require((uint64_t)s->n_done + n <= s->max_iter, "advance beyond the prepared max_iter");
  if (n == 0) return;
  constexpr int kGraphLen = 32;
  if (n >= (uint32_t)kGraphLen && !s->gexec) {
    GPUM_CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    const uint64_t before = s->launches;
    try {
      for (int i = 0; i < kGraphLen; ++i) s->step();
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(s->stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    s->graph_launches = s->launches - before;  // counted per replay below
    s->launches = before;
    GPUM_CK(cudaStreamEndCapture(s->stream, &s->graph));
    GPUM_CK(cudaGraphInstantiate(&s->gexec, s->graph, 0));
    s->graph_len = kGraphLen;
  }
  uint32_t left = n;
  while (s->gexec && left >= (uint32_t)s->graph_len) {
    GPUM_CK(cudaGraphLaunch(s->gexec, s->stream));
    s->launches += s->graph_launches;
    left -= s->graph_len;
  }
  for (; left > 0; --left) s->step();
  s->n_done += n;
}

void fetch(gpum_b200_session* s, float* out_draws, float* out_accept, double* out_last,
           uint32_t* n_done) {
  require(s && s->prepared, "session has no prepared run");
  s->check_device_error();
  const uint32_t n = s->n_done;
  const int C = s->n_chains;
  const size_t np = s->np;
  if (n_done) *n_done = n;
  cudaStream_t st = s->stream;
  if (out_draws && n > 0) {
    s->draws_out.ensure((size_t)n * C * np);
    dim3 grid((C + 31) / 32, (n + 31) / 32, (unsigned)np);
    draws_layout_kernel<<<grid, dim3(32, 8), 0, st>>>(s->draws.p, s->draws_out.p, (int)n,
                                                      (int)np, C, s->geo.C_pad);
    GPUM_CK(cudaGetLastError());
    ++s->launches;
    GPUM_CK(cudaMemcpyAsync(out_draws, s->draws_out.p, sizeof(float) * n * C * np,
                            cudaMemcpyDeviceToHost, st));
  }
  std::vector<uint32_t> acc(C);
  GPUM_CK(cudaMemcpyAsync(acc.data(), s->accepts.p, sizeof(uint32_t) * C,
                          cudaMemcpyDeviceToHost, st));
  if (out_last)
    GPUM_CK(cudaMemcpyAsync(out_last, s->cur.p, sizeof(double) * C, cudaMemcpyDeviceToHost, st));
  GPUM_CK(cudaStreamSynchronize(st));
  if (out_accept)
    for (int c = 0; c < C; ++c) out_accept[c] = n == 0 ? 0.0f : (float)acc[c] / (float)n;
}

enum BatchKind { B_SUM = 0, B_POINTWISE = 1, B_GRAD = 2 };

void batch(gpum_b200_session* s, const double* pts, size_t n_points, double* out, int kind) {
  require(s != nullptr, "session is NULL");
  require(out != nullptr || n_points == 0, "output pointer is NULL");
  require(pts != nullptr || n_points == 0, "points pointer is NULL");
  if (n_points == 0) return;
  require(n_points <= (1u << 24), "more than 2^24 points", GPUM_ERR_UNSUPPORTED);
  s->settle_recording();
  s->prepared = false;  // the evaluation buffers are reused
  s->drop_graph();
  const size_t np = s->np;
  size_t chunk = n_points;
  if (kind == B_POINTWISE && s->n_obs > 0)
    chunk = std::max<size_t>(1, std::min<size_t>(n_points, (size_t)(1ull << 27) / s->n_obs));
  for (size_t p0 = 0; p0 < n_points; p0 += chunk) {
    const int n = (int)std::min(chunk, n_points - p0);
    s->setup_eval(n, kind == B_GRAD, kind == B_POINTWISE);
    s->upload_points(pts + p0 * np, n);
    s->A = ChainArgs{};
    if (kind == B_POINTWISE) {
      if (s->n_obs == 0) continue;
      s->pointwise.ensure((size_t)n * s->n_obs);
      s->E.pointwise = s->pointwise.p;
      if (s->ll.empty()) {
        GPUM_CK(cudaMemsetAsync(s->pointwise.p, 0, sizeof(double) * n * s->n_obs, s->stream));
      } else {
        s->launch(PH_POINTWISE);
      }
      GPUM_CK(cudaMemcpyAsync(out + p0 * s->n_obs, s->pointwise.p,
                              sizeof(double) * n * s->n_obs, cudaMemcpyDeviceToHost, s->stream));
    } else {
      const int W = s->kc.W;
      s->out64.ensure((size_t)n * W);
      if (s->ll.empty()) {
        GPUM_CK(cudaMemsetAsync(s->out64.p, 0, sizeof(double) * n * W, s->stream));
      } else {
        s->launch(PH_EVAL);
        reduce_partials_kernel<<<(n * W + 255) / 256, 256, 0, s->stream>>>(
            s->partials.p, s->out64.p, s->geo.NOB, s->geo.C_pad, n, W);
        GPUM_CK(cudaGetLastError());
        ++s->launches;
      }
      if (kind == B_GRAD) {
        std::vector<double> tmp((size_t)n * W);
        GPUM_CK(cudaMemcpyAsync(tmp.data(), s->out64.p, sizeof(double) * n * W,
                                cudaMemcpyDeviceToHost, s->stream));
        GPUM_CK(cudaStreamSynchronize(s->stream));
        for (int p = 0; p < n; ++p)
          for (size_t j = 0; j < np; ++j) out[(p0 + p) * np + j] = tmp[(size_t)p * W + 1 + j];
      } else {
        GPUM_CK(cudaMemcpyAsync(out + p0, s->out64.p, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                s->stream));
      }
    }
    s->check_device_error();
  }
}

// ------------------------------------------------------ delayed acceptance
// Exact start as prepare() (PH_INIT), then per iteration: surrogate at the
// proposals (tcgen05 MLP) -> stage-1 decision -> compaction of the
// survivors -> exact evaluation of the compacted prefix only (CTAs of dead
// chain blocks exit at once) -> stage-2 decision, draw, next proposal.
// The loop is captured in a CUDA graph of kDaGraphLen iterations.
// The compiled engine's f64 prior at the chains' points (state or proposal)
// into out; with the Langevin proposal its gradient is added into D.gs (the
// surrogate's data-term gradient there).
void launch_prior(gpum_b200_session* s, double* pts, double* out) {
  int n = s->n_chains;
  double* grad = s->A.mode == MODE_MALA ? s->D.gs : nullptr;
  void* args[] = {(void*)&pts, (void*)&n, (void*)&out, (void*)&grad};
  GPUM_CK(cudaLaunchKernel((const void*)s->cm.k_prior, dim3((unsigned)((n + 127) / 128)),
                           dim3(128), args, 0, s->stream));
  ++s->launches;
}

void da_step(gpum_b200_session* s) {
  const int C = s->n_chains, np = (int)s->np;
  std::string e;
  const int rc = s->A.mode == MODE_MALA
                     ? mlp_infer_grad(s->da_mlp, s->prop.p, C, np, s->sll_y.p, s->D.gs,
                                      s->stream, &e)
                     : mlp_infer(s->da_mlp, s->prop.p, C, np, s->sll_y.p, s->stream, &e);
  if (rc != GPUM_OK) throw Failure{rc, "surrogate: " + e};
  cudaStream_t st = s->stream;
  if (s->D.prior_ready) launch_prior(s, s->prop.p, s->prior_y.p);
  // 64-thread blocks spread the per-chain f64 work (prior, proposal) over
  // more SMs; finalize runs one warp per chain.
  const unsigned cb = (unsigned)((C + 63) / 64);
  da_stage1_kernel<<<cb, 64, 0, st>>>(s->A, s->D);
  da_compact_kernel<<<1, 1024, 0, st>>>(s->A, s->D);
  da_pack_kernel<<<(unsigned)(((size_t)C * np + 255) / 256), 256, 0, st>>>(s->A, s->D);
  GPUM_CK(cudaGetLastError());
  s->launch_with(s->geo_da, s->E_da, PH_EVAL);
  da_finalize_kernel<<<(unsigned)((C + 7) / 8), 256, (size_t)8 * 2 * np * sizeof(double), st>>>(
      s->A, s->D, s->da_partials.p, s->geo_da.CG, s->geo_da.NCB * s->geo_da.NOB,
      s->geo_da.ntiles, s->geo_da.C_pad);
  da_tick_kernel<<<1, 32, 0, st>>>(s->D);
  GPUM_CK(cudaGetLastError());
  s->launches += 5 + (uint64_t)s->da_mlp_launches;  // launch_prior counts itself
  if (s->pt_K > 0) {  // exchanges on the exact log posteriors, caches swapped along
    PtArgs P{s->pt_K,   s->pt_every,  s->D.iter, s->D.sll_x, s->D.prior_x,
             s->pt_n.p, s->pt_att.p, s->pt_acc.p, s->D.full,  s->D.C_pad};
    pt_exchange_kernel<<<(unsigned)((C + 127) / 128), 128, 0, st>>>(s->A, P);
    GPUM_CK(cudaGetLastError());
    ++s->launches;
  }
}

void run_da(gpum_b200_session* s, gpum_b200_mlp* mlp, const double* init, const double* sd,
            const double* temps, uint32_t C, uint32_t n_iter, uint32_t seed, uint32_t mode,
            double gamma, double de_noise, const double* L, size_t n_l, int rng, float* out_draws,
            float* out_accept, double* out_last, uint32_t* out_exact) {
  require(s != nullptr, "session is NULL");
  require(mlp != nullptr, "surrogate is NULL");
  require(mode <= 3, "delayed acceptance takes proposal mode 0 (rwm), 1 (de), 2 (cholesky) or "
                     "3 (mala: a Langevin move driven by the surrogate's gradient)");
  require(s->n_beta == 0, "delayed acceptance does not support likelihood powers");
  // The Langevin proposal's drift is the surrogate log-posterior gradient, so
  // the exact start evaluates values only (as the random walk with the same
  // preconditioner), and the chains draw their first proposals again below.
  const bool lang = mode == 3;
  const bool lang_L = lang && L != nullptr && n_l > 0;
  const uint64_t keep_cap = s->rec_cap;
  s->rec_cap = 0;  // stage-1 rejections leave no exact pair to record
  try {
    prepare(s, init, sd, temps, C, n_iter, seed, lang ? (lang_L ? 2u : 0u) : mode, gamma,
            de_noise, L, n_l, rng);
  } catch (...) {
    s->rec_cap = keep_cap;
    throw;
  }
  s->rec_cap = keep_cap;
  const int np = (int)s->np;
  cudaStream_t st = s->stream;
  const Geometry& g = s->geo;
  if (lang) {
    for (auto* b : {&s->gx, &s->gy, &s->mx, &s->my, &s->vbuf, &s->da_gs}) b->ensure((size_t)C * np);
    const size_t nt = (size_t)C * std::max<size_t>(s->prior_code.size() / 2, 1);
    s->da_tvals.ensure(nt);
    s->da_tadj.ensure(nt);
    s->da_tlhs.ensure(nt);
    s->da_trhs.ensure(nt);
    s->A.mode = MODE_MALA;
    s->A.gx = s->gx.p;
    s->A.gy = s->gy.p;
    s->A.mx = s->mx.p;
    s->A.my = s->my.p;
    s->A.vbuf = s->vbuf.p;
  }
  s->sll_x.ensure(C);
  s->sll_y.ensure(C);
  s->prior_x.ensure(C);
  s->prior_y.ensure(C);
  s->da_flag.ensure(C);
  s->da_slot.ensure(C);
  s->da_stage1.ensure(C);
  s->da_active.ensure(1);
  s->da_iter.ensure(1);
  s->da_params.ensure((size_t)np * g.C_pad);
  // The exact evaluation runs a fixed 1-D grid of one CTA per resident slot
  // (at least one per chain block); the kernel splits it into (live chain
  // blocks x observation blocks) from the stage-1 survivor count on the
  // device (da_obs_blocks).
  s->geo_da = g;
  {
    int occ = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, s->kc.fn, s->kc.threads, g.smem);
    // one wave of resident CTAs: with few survivors each CTA then takes many
    // tiles, so the per-CTA set-up is paid once per SM slot
    s->geo_da.NCB = std::max(num_sms() * std::max(occ, 1), g.NCB);
    s->geo_da.NOB = 1;
  }
  const int max_nob = std::max(1, std::min(s->geo_da.NCB, std::max(g.ntiles, 1)));
  s->da_partials.ensure((size_t)max_nob * s->geo_da.C_pad);
  GPUM_CK(cudaMemsetAsync(s->da_params.p, 0, sizeof(float) * np * g.C_pad, st));
  s->E_da = s->E;
  s->E_da.params = s->da_params.p;
  s->E_da.partials = s->da_partials.p;
  s->E_da.active = s->da_active.p;
  DaArgs& D = s->D;
  D.sll_x = s->sll_x.p;
  D.sll_y = s->sll_y.p;
  D.prior_x = s->prior_x.p;
  D.prior_y = s->prior_y.p;
  D.flag = s->da_flag.p;
  D.slot = s->da_slot.p;
  D.active = s->da_active.p;
  D.iter = s->da_iter.p;
  D.stage1 = s->da_stage1.p;
  D.params = s->da_params.p;
  D.full = s->params.p;
  D.C_pad = g.C_pad;
  D.gs = lang ? s->da_gs.p : nullptr;
  D.tvals = lang ? s->da_tvals.p : nullptr;
  D.tadj = lang ? s->da_tadj.p : nullptr;
  D.tlhs = lang ? s->da_tlhs.p : nullptr;
  D.trhs = lang ? s->da_trhs.p : nullptr;
  s->da_mlp = mlp;
  s->da_mlp_launches = 0;
  std::string e;
  int rc = lang ? mlp_infer_grad(mlp, s->state.p, (int)C, np, s->sll_x.p, D.gs, st, &e)
                : mlp_infer(mlp, s->state.p, (int)C, np, s->sll_x.p, st, &e);
  if (rc != GPUM_OK) throw Failure{rc, "surrogate: " + e};
  s->da_mlp_launches = lang ? mlp_infer_grad_launches(mlp, (int)C)
                            : mlp_infer_launches(mlp, (int)C);
  // With the compiled engine the prior is its generated f64 code, one kernel
  // over all chains, instead of an interpreted prior per chain thread.
  D.prior_ready = s->kc.compiled && s->cm.k_prior ? 1 : 0;
  if (D.prior_ready) launch_prior(s, s->state.p, s->prior_x.p);
  s->launches += (uint64_t)s->da_mlp_launches;
  da_setup_kernel<<<(C + 255) / 256, 256, 0, st>>>(s->A, D);
  GPUM_CK(cudaGetLastError());
  ++s->launches;

  constexpr uint32_t kDaGraphLen = 16;
  uint32_t left = n_iter;
  if (n_iter >= kDaGraphLen) {
    GPUM_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const uint64_t before = s->launches;
    try {
      for (uint32_t i = 0; i < kDaGraphLen; ++i) da_step(s);
    } catch (...) {
      cudaGraph_t gr = nullptr;
      cudaStreamEndCapture(st, &gr);
      if (gr) cudaGraphDestroy(gr);
      throw;
    }
    const uint64_t per_graph = s->launches - before;
    s->launches = before;
    GPUM_CK(cudaStreamEndCapture(st, &s->graph));
    GPUM_CK(cudaGraphInstantiate(&s->gexec, s->graph, 0));
    while (left >= kDaGraphLen) {
      GPUM_CK(cudaGraphLaunch(s->gexec, st));
      s->launches += per_graph;
      left -= kDaGraphLen;
    }
    s->drop_graph();
  }
  for (; left > 0; --left) da_step(s);
  s->n_done = n_iter;
  s->A.rec_ll = nullptr;
  fetch(s, out_draws, out_accept, out_last, nullptr);
  if (out_exact) {
    GPUM_CK(cudaMemcpyAsync(out_exact, s->da_stage1.p, sizeof(uint32_t) * C,
                            cudaMemcpyDeviceToHost, st));
    GPUM_CK(cudaStreamSynchronize(st));
  }
  s->prepared = false;  // the DA state is not resumable through advance()
}

}  // namespace

// =================================================================== C ABI
extern "C" {

int gpum_b200_available(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
    cudaGetLastError();
    return 0;
  }
  int dev = 0, major = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (major != 10) return 0;
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, interp_kernel(V8x8)) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return 1;
}

const char* gpum_b200_version(void) { return "gpum_b200 0.2.0 sm_100a"; }

int gpum_b200_validate_program(const uint32_t* code, size_t n_code, size_t n_consts,
                               uint32_t n_params, uint32_t n_cols, int allow_data, int* depth,
                               char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    int d = 0;
    std::string m;
    if (validate_program(code, n_code, n_consts, n_params, n_cols, allow_data != 0, &d, &m))
      throw Failure{GPUM_ERR_INVALID, m};
    if (depth) *depth = d;
  });
}

int gpum_b200_compile_check(const uint32_t* code, size_t n_code, const double* consts,
                            size_t n_consts, const uint32_t* prior_code, size_t n_prior,
                            const double* prior_consts, size_t n_prior_consts,
                            uint32_t n_params, uint32_t n_cols, size_t* cubin_bytes, char* err,
                            size_t err_len) {
  return guard(err, err_len, [&] {
    UProg ll;
    GenModel gm;
    check_model(code, n_code, consts, n_consts, prior_code, n_prior, prior_consts,
                n_prior_consts, n_params, n_cols, &ll, &gm);
    std::string m;
    if (jit_compile_check(gm, cubin_bytes, &m)) throw Failure{GPUM_ERR_UNSUPPORTED, m};
  });
}

int gpum_b200_session_create(const uint32_t* code, size_t n_code, const double* consts,
                             size_t n_consts, const uint32_t* prior_code, size_t n_prior,
                             const double* prior_consts, size_t n_prior_consts,
                             uint32_t n_params, const double* data, uint32_t n_cols,
                             uint64_t n_obs, gpum_b200_session** out, char* err,
                             size_t err_len) {
  return guard(err, err_len, [&] {
    require(out != nullptr, "output session pointer is NULL");
    *out = nullptr;
    *out = create_session(code, n_code, consts, n_consts, prior_code, n_prior, prior_consts,
                          n_prior_consts, n_params, data, n_cols, n_obs);
  });
}

int gpum_b200_session_set_engine(gpum_b200_session* s, int engine, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    require(s != nullptr, "session is NULL");
    require(engine == GPUM_ENGINE_INTERP || engine == GPUM_ENGINE_COMPILED ||
                engine == GPUM_ENGINE_AUTO,
            "engine must be 0 (interpreter), 1 (compiled) or 2 (auto)");
    if (engine == GPUM_ENGINE_COMPILED && !s->compiled_available())
      throw Failure{GPUM_ERR_UNSUPPORTED, "compiled engine unavailable: " + s->cm_error};
    s->engine = engine;
    s->drop_graph();
    s->prepared = false;
  });
}

int gpum_b200_session_engine(gpum_b200_session* s) {
  if (!s) return -1;
  if (s->engine == GPUM_ENGINE_AUTO)
    return s->compiled_available() ? GPUM_ENGINE_COMPILED : GPUM_ENGINE_INTERP;
  return s->engine;
}

int gpum_b200_session_tensor_cores(gpum_b200_session* s) {
  if (!s) return -1;
  return gpum_b200_session_engine(s) == GPUM_ENGINE_COMPILED && s->tc_ok ? 1 : 0;
}

void gpum_b200_session_destroy(gpum_b200_session* s) {
  if (!s) return;
  if (s->stream) cudaStreamSynchronize(s->stream);
  delete s;
}

uint64_t gpum_b200_session_launches(const gpum_b200_session* s) { return s ? s->launches : 0; }

void* gpum_b200_session_stream(const gpum_b200_session* s) {
  return s ? (void*)s->stream : nullptr;
}

int gpum_b200_session_prepare(gpum_b200_session* s, const double* init, const double* sd,
                              const double* temps, uint32_t n_chains, uint32_t max_iter,
                              uint32_t seed, uint32_t mode, double gamma, double de_noise,
                              const double* L, size_t n_l, int rng, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    prepare(s, init, sd, temps, n_chains, max_iter, seed, mode, gamma, de_noise, L, n_l, rng);
  });
}

int gpum_b200_session_advance(gpum_b200_session* s, uint32_t n, char* err, size_t err_len) {
  return guard(err, err_len, [&] { advance(s, n); });
}

int gpum_b200_session_sync(gpum_b200_session* s, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    require(s != nullptr, "session is NULL");
    GPUM_CK(cudaStreamSynchronize(s->stream));
  });
}

int gpum_b200_session_fetch(gpum_b200_session* s, float* out_draws, float* out_accept,
                            double* out_last, uint32_t* n_done, char* err, size_t err_len) {
  return guard(err, err_len, [&] { fetch(s, out_draws, out_accept, out_last, n_done); });
}

int gpum_b200_session_run(gpum_b200_session* s, const double* init, const double* sd,
                          const double* temps, uint32_t n_chains, uint32_t n_iter, uint32_t seed,
                          uint32_t mode, double gamma, double de_noise, const double* L,
                          size_t n_l, int rng, float* out_draws, float* out_accept,
                          double* out_last, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    prepare(s, init, sd, temps, n_chains, n_iter, seed, mode, gamma, de_noise, L, n_l, rng);
    advance(s, n_iter);
    fetch(s, out_draws, out_accept, out_last, nullptr);
  });
}

int gpum_b200_session_loglik_batch(gpum_b200_session* s, const double* points, size_t n_points,
                                   double* out, char* err, size_t err_len) {
  return guard(err, err_len, [&] { batch(s, points, n_points, out, B_SUM); });
}

int gpum_b200_session_loglik_pointwise(gpum_b200_session* s, const double* points,
                                       size_t n_points, double* out, char* err, size_t err_len) {
  return guard(err, err_len, [&] { batch(s, points, n_points, out, B_POINTWISE); });
}

int gpum_b200_session_grad_batch(gpum_b200_session* s, const double* points, size_t n_points,
                                 double* out, char* err, size_t err_len) {
  return guard(err, err_len, [&] { batch(s, points, n_points, out, B_GRAD); });
}

int gpum_b200_run(const uint32_t* code, size_t n_code, const double* consts, size_t n_consts,
                  const uint32_t* prior_code, size_t n_prior, const double* prior_consts,
                  size_t n_prior_consts, uint32_t n_params, const double* data, uint32_t n_cols,
                  uint64_t n_obs, const double* init, const double* sd, const double* temps,
                  uint32_t n_chains, uint32_t n_iter, uint32_t seed, uint32_t mode, double gamma,
                  double de_noise, const double* L, size_t n_l, float* out_draws,
                  float* out_accept, double* out_last, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    std::unique_ptr<gpum_b200_session> s(create_session(code, n_code, consts, n_consts,
                                                        prior_code, n_prior, prior_consts,
                                                        n_prior_consts, n_params, data, n_cols,
                                                        n_obs));
    prepare(s.get(), init, sd, temps, n_chains, n_iter, seed, mode, gamma, de_noise, L, n_l,
            GPUM_RNG_TRIPLE32);
    advance(s.get(), n_iter);
    fetch(s.get(), out_draws, out_accept, out_last, nullptr);
  });
}

static int one_shot_batch(const uint32_t* code, size_t n_code, const double* consts,
                          size_t n_consts, uint32_t n_params, const double* data, uint32_t n_cols,
                          uint64_t n_obs, const double* points, size_t n_points, double* out,
                          char* err, size_t err_len, int kind) {
  return guard(err, err_len, [&] {
    std::unique_ptr<gpum_b200_session> s(create_session(
        code, n_code, consts, n_consts, nullptr, 0, nullptr, 0, n_params, data, n_cols, n_obs));
    batch(s.get(), points, n_points, out, kind);
  });
}

int gpum_b200_loglik_batch(const uint32_t* code, size_t n_code, const double* consts,
                           size_t n_consts, uint32_t n_params, const double* data, uint32_t n_cols,
                           uint64_t n_obs, const double* points, size_t n_points, double* out,
                           char* err, size_t err_len) {
  return one_shot_batch(code, n_code, consts, n_consts, n_params, data, n_cols, n_obs, points,
                        n_points, out, err, err_len, B_SUM);
}

int gpum_b200_loglik_pointwise(const uint32_t* code, size_t n_code, const double* consts,
                               size_t n_consts, uint32_t n_params, const double* data,
                               uint32_t n_cols, uint64_t n_obs, const double* points,
                               size_t n_points, double* out, char* err, size_t err_len) {
  return one_shot_batch(code, n_code, consts, n_consts, n_params, data, n_cols, n_obs, points,
                        n_points, out, err, err_len, B_POINTWISE);
}

int gpum_b200_grad_batch(const uint32_t* code, size_t n_code, const double* consts,
                         size_t n_consts, uint32_t n_params, const double* data, uint32_t n_cols,
                         uint64_t n_obs, const double* points, size_t n_points, double* out,
                         char* err, size_t err_len) {
  return one_shot_batch(code, n_code, consts, n_consts, n_params, data, n_cols, n_obs, points,
                        n_points, out, err, err_len, B_GRAD);
}

int gpum_b200_session_run_de_sync(gpum_b200_session* s, const double* init, const double* sd,
                                  uint32_t n_chains, uint32_t n_iter, uint32_t seed,
                                  double gamma, double de_noise, int rng, float* out_draws,
                                  float* out_accept, double* out_last, char* err,
                                  size_t err_len) {
  return guard(err, err_len, [&] {
    require(n_chains >= 1, "n_chains must be at least 1");
    const std::vector<double> temps(n_chains, 1.0);  // path B is untempered
    prepare(s, init, sd, temps.data(), n_chains, n_iter, seed, 4, gamma, de_noise, nullptr, 0,
            rng);
    advance(s, n_iter);
    fetch(s, out_draws, out_accept, out_last, nullptr);
  });
}

int gpum_b200_run_de_sync(const uint32_t* code, size_t n_code, const double* consts,
                          size_t n_consts, uint32_t n_params, const double* data,
                          uint32_t n_cols, uint64_t n_obs, const uint32_t* prior_code,
                          size_t n_prior, const double* prior_consts, size_t n_prior_consts,
                          const double* init, const double* sd, uint32_t n_chains,
                          uint32_t n_iter, uint32_t seed, double gamma, double de_noise,
                          float* out_draws, float* out_accept, double* out_last, char* err,
                          size_t err_len) {
  return guard(err, err_len, [&] {
    require(n_chains >= 1, "n_chains must be at least 1");
    std::unique_ptr<gpum_b200_session> s(create_session(code, n_code, consts, n_consts,
                                                        prior_code, n_prior, prior_consts,
                                                        n_prior_consts, n_params, data, n_cols,
                                                        n_obs));
    const std::vector<double> temps(n_chains, 1.0);
    prepare(s.get(), init, sd, temps.data(), n_chains, n_iter, seed, 4, gamma, de_noise,
            nullptr, 0, GPUM_RNG_TRIPLE32);
    advance(s.get(), n_iter);
    fetch(s.get(), out_draws, out_accept, out_last, nullptr);
  });
}

int gpum_b200_session_set_exchange(gpum_b200_session* s, uint32_t ladder_len,
                                   uint32_t swap_every, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    require(s != nullptr, "session is NULL");
    require(ladder_len == 0 || (ladder_len >= 2 && swap_every >= 1),
            "ladder_len must be 0 (off) or >= 2, with swap_every >= 1");
    s->drop_graph();
    s->prepared = false;
    s->pt_K = (int)ladder_len;
    s->pt_every = ladder_len ? (int)swap_every : 0;
  });
}

int gpum_b200_session_exchange_stats(gpum_b200_session* s, uint32_t* attempts,
                                     uint32_t* accepted, uint32_t* n_exchanges, char* err,
                                     size_t err_len) {
  return guard(err, err_len, [&] {
    require(s != nullptr, "session is NULL");
    require(s->pt_K > 0, "device exchanges are off");
    const size_t C = (size_t)s->n_chains;
    require(C > 0 && s->pt_att.p && s->pt_att.n >= C,
            "no run with device exchanges since they were set");
    if (attempts)
      GPUM_CK(cudaMemcpyAsync(attempts, s->pt_att.p, sizeof(uint32_t) * C,
                              cudaMemcpyDeviceToHost, s->stream));
    if (accepted)
      GPUM_CK(cudaMemcpyAsync(accepted, s->pt_acc.p, sizeof(uint32_t) * C,
                              cudaMemcpyDeviceToHost, s->stream));
    if (n_exchanges)
      GPUM_CK(cudaMemcpyAsync(n_exchanges, s->pt_n.p, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                              s->stream));
    GPUM_CK(cudaStreamSynchronize(s->stream));
  });
}

int gpum_b200_session_draw_moments(gpum_b200_session* s, uint32_t t0, uint32_t n,
                                   double* chain_mean, double* chain_m2, double* pool_mean,
                                   double* pool_m2, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    require(s && s->prepared, "session has no prepared run");
    require(n >= 1 && (uint64_t)t0 + n <= s->n_done, "iterations beyond those advanced");
    require(chain_mean && chain_m2 && pool_mean && pool_m2, "output pointers are NULL");
    const int C = s->n_chains, np = (int)s->np;
    cudaStream_t st = s->stream;
    s->mom.ensure((size_t)2 * C * np + np + (size_t)np * np);
    double* dmean = s->mom.p;
    double* dm2 = dmean + (size_t)C * np;
    double* pmean = dm2 + (size_t)C * np;
    double* pm2 = pmean + np;
    const int CP = s->geo.C_pad;
    moments_chain_kernel<<<(unsigned)(((size_t)C * np + 255) / 256), 256, 0, st>>>(
        s->draws.p, np, C, CP, (int)t0, (int)n, dmean, dm2);
    moments_pool_mean_kernel<<<np, 256, 0, st>>>(s->draws.p, np, C, CP, (int)t0, (int)n, pmean);
    moments_pool_m2_kernel<<<np * np, 256, 0, st>>>(s->draws.p, np, C, CP, (int)t0, (int)n,
                                                    pmean, pm2);
    GPUM_CK(cudaGetLastError());
    s->launches += 3;
    GPUM_CK(cudaMemcpyAsync(chain_mean, dmean, sizeof(double) * C * np, cudaMemcpyDeviceToHost,
                            st));
    GPUM_CK(cudaMemcpyAsync(chain_m2, dm2, sizeof(double) * C * np, cudaMemcpyDeviceToHost, st));
    GPUM_CK(cudaMemcpyAsync(pool_mean, pmean, sizeof(double) * np, cudaMemcpyDeviceToHost, st));
    GPUM_CK(cudaMemcpyAsync(pool_m2, pm2, sizeof(double) * np * np, cudaMemcpyDeviceToHost, st));
    GPUM_CK(cudaStreamSynchronize(st));
  });
}

int gpum_b200_session_state(gpum_b200_session* s, double* out_state, char* err,
                            size_t err_len) {
  return guard(err, err_len, [&] {
    require(s && s->prepared, "session has no prepared run");
    require(out_state != nullptr, "output pointer is NULL");
    GPUM_CK(cudaMemcpyAsync(out_state, s->state.p, sizeof(double) * s->n_chains * s->np,
                            cudaMemcpyDeviceToHost, s->stream));
    GPUM_CK(cudaStreamSynchronize(s->stream));
  });
}

int gpum_b200_session_set_likelihood_powers(gpum_b200_session* s, const double* beta,
                                            size_t n_chains, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    require(s != nullptr, "session is NULL");
    s->drop_graph();
    s->prepared = false;
    if (beta == nullptr || n_chains == 0) {
      s->n_beta = 0;
      s->beta.release();
      return;
    }
    for (size_t c = 0; c < n_chains; ++c)
      require(std::isfinite(beta[c]) && beta[c] >= 0.0,
              "likelihood powers must be finite and non-negative");
    s->beta.ensure(n_chains);
    GPUM_CK(cudaMemcpyAsync(s->beta.p, beta, sizeof(double) * n_chains, cudaMemcpyHostToDevice,
                            s->stream));
    GPUM_CK(cudaStreamSynchronize(s->stream));
    s->n_beta = n_chains;
  });
}

int gpum_b200_session_record(gpum_b200_session* s, uint64_t capacity, char* err,
                             size_t err_len) {
  return guard(err, err_len, [&] {
    require(s != nullptr, "session is NULL");
    require(capacity <= (1ull << 28), "more than 2^28 recorded pairs", GPUM_ERR_UNSUPPORTED);
    s->settle_recording();
    s->drop_graph();
    s->prepared = false;
    s->rec_count = 0;
    s->rec_cap = capacity;
    if (capacity == 0) {
      s->rec_theta.release();
      s->rec_ll.release();
      return;
    }
    s->rec_theta.ensure((size_t)capacity * s->np);
    s->rec_ll.ensure((size_t)capacity);
  });
}

}  // extern "C"

namespace {

// ----------------------------------------- surrogate fit from device pairs
// Pair i of the recording is held out when holdout_every > 0 and
// i % holdout_every == 0; a pair with a non-finite log-likelihood or
// parameter is dropped.  One CTA scans the flags in pair order, so the
// positions (and the training set's order) are deterministic:
//   pos[i] = training position | kHeldOut for a held-out position |
//            kDropped.
constexpr int kSplitThreads = 1024;
constexpr uint32_t kHeldOut = 0x80000000u, kDropped = 0xFFFFFFFFu;

__global__ void __launch_bounds__(kSplitThreads)
pairs_split_kernel(const float* __restrict__ th, const double* __restrict__ ll, uint32_t n,
                   int np, uint32_t every, uint32_t* __restrict__ pos,
                   uint32_t* __restrict__ counts) {
  __shared__ uint32_t wsum[2][32], tot[2], base[2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) base[0] = base[1] = 0;
  __syncthreads();
  for (uint32_t i0 = 0; i0 < n; i0 += kSplitThreads) {
    const uint32_t i = i0 + tid;
    bool ok = false, hold = false;
    if (i < n) {
      ok = isfinite(ll[i]);
      for (int j = 0; j < np && ok; ++j) ok = isfinite(th[(size_t)i * np + j]);
      hold = every > 0 && i % every == 0;
    }
    const bool ft = ok && !hold, fh = ok && hold;
    const uint32_t bt = __ballot_sync(0xffffffffu, ft), bh = __ballot_sync(0xffffffffu, fh);
    const uint32_t below = (1u << lane) - 1u;
    if (lane == 0) {
      wsum[0][warp] = __popc(bt);
      wsum[1][warp] = __popc(bh);
    }
    __syncthreads();
    if (warp == 0) {  // exclusive prefix over the warps, and the totals
      const uint32_t a0 = wsum[0][lane], b0 = wsum[1][lane];
      uint32_t a = a0, b = b0;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, a, o);
        const uint32_t y = __shfl_up_sync(0xffffffffu, b, o);
        if (lane >= o) {
          a += x;
          b += y;
        }
      }
      wsum[0][lane] = a - a0;
      wsum[1][lane] = b - b0;
      if (lane == 31) {
        tot[0] = a;
        tot[1] = b;
      }
    }
    __syncthreads();
    if (i < n)
      pos[i] = ft   ? base[0] + wsum[0][warp] + __popc(bt & below)
               : fh ? kHeldOut | (base[1] + wsum[1][warp] + __popc(bh & below))
                    : kDropped;
    __syncthreads();
    if (tid == 0) {
      base[0] += tot[0];
      base[1] += tot[1];
    }
    __syncthreads();
  }
  if (tid == 0) {
    counts[0] = base[0];
    counts[1] = base[1];
  }
}

// Training pairs keep the f32 parameters the gather reads; held-out pairs
// become the f64 rows the inference path takes.
__global__ void pairs_scatter_kernel(const float* __restrict__ th, const double* __restrict__ ll,
                                     uint32_t n, int np, const uint32_t* __restrict__ pos,
                                     float* __restrict__ tr_th, double* __restrict__ tr_ll,
                                     double* __restrict__ ho_th, double* __restrict__ ho_ll) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = pos[i];
  if (p == kDropped) return;
  const float* src = th + (size_t)i * np;
  if (p & kHeldOut) {
    const uint32_t q = p & ~kHeldOut;
    for (int j = 0; j < np; ++j) ho_th[(size_t)q * np + j] = (double)src[j];
    ho_ll[q] = ll[i];
  } else {
    for (int j = 0; j < np; ++j) tr_th[(size_t)p * np + j] = src[j];
    tr_ll[p] = ll[i];
  }
}

// Shifted f64 sums over the training pairs (shift: the first pair, so the
// sums of squares do not cancel): accumulator a < d is sum x_j, d <= a <
// d + d(d+1)/2 is sum x_j x_k over the row-major upper triangle (j <= k),
// then sum y and sum y^2.  Block (c, g) sums rows of chunk c into
// accumulator g * blockDim.x + threadIdx.x, in row order.
constexpr int kMomRows = 32;
__global__ void pairs_moments_kernel(const float* __restrict__ th, const double* __restrict__ ll,
                                     uint32_t n, int d, uint32_t chunk,
                                     double* __restrict__ part) {
  extern __shared__ double xs[];  // [kMomRows][d + 1]
  const int NA = d + d * (d + 1) / 2 + 2;
  const int a = blockIdx.y * blockDim.x + threadIdx.x;
  int kind = 3, j = 0, k = 0;
  if (a < d) {
    kind = 0;
    j = a;
  } else if (a < NA - 2) {
    int p = a - d;
    while (p >= d - j) {
      p -= d - j;
      ++j;
    }
    k = j + p;
    kind = 1;
  } else if (a == NA - 2) {
    kind = 2;
  }
  const uint32_t r0 = blockIdx.x * chunk, r1 = min(n, r0 + chunk);
  double acc = 0.0;
  for (uint32_t rb = r0; rb < r1; rb += kMomRows) {
    const int rows = (int)min((uint32_t)kMomRows, r1 - rb);
    __syncthreads();
    for (int e = threadIdx.x; e < rows * (d + 1); e += blockDim.x) {
      const int r = e / (d + 1), c = e % (d + 1);
      xs[e] = c < d ? (double)th[(size_t)(rb + r) * d + c] - (double)th[c]
                    : ll[rb + r] - ll[0];
    }
    __syncthreads();
    if (a < NA) {
      for (int r = 0; r < rows; ++r) {
        const double* x = xs + r * (d + 1);
        acc += kind == 0 ? x[j] : kind == 1 ? x[j] * x[k] : kind == 2 ? x[d] : x[d] * x[d];
      }
    }
  }
  if (a < NA) part[(size_t)blockIdx.x * NA + a] = acc;
}

// Lower Cholesky factor of the d x d matrix A (row-major) and its inverse;
// false when a pivot is not positive.
bool cholesky_inverse(int d, const std::vector<double>& A, std::vector<double>* Linv) {
  std::vector<double> L((size_t)d * d, 0.0);
  for (int i = 0; i < d; ++i)
    for (int j = 0; j <= i; ++j) {
      double v = A[(size_t)i * d + j];
      for (int k = 0; k < j; ++k) v -= L[(size_t)i * d + k] * L[(size_t)j * d + k];
      if (i == j) {
        if (!(v > 0.0) || !std::isfinite(v)) return false;
        L[(size_t)i * d + i] = std::sqrt(v);
      } else {
        L[(size_t)i * d + j] = v / L[(size_t)j * d + j];
      }
    }
  Linv->assign((size_t)d * d, 0.0);
  for (int c = 0; c < d; ++c)  // forward substitution, column c of the inverse
    for (int i = c; i < d; ++i) {
      double v = i == c ? 1.0 : 0.0;
      for (int k = c; k < i; ++k) v -= L[(size_t)i * d + k] * (*Linv)[(size_t)k * d + c];
      (*Linv)[(size_t)i * d + c] = v / L[(size_t)i * d + i];
    }
  return true;
}

}  // namespace

extern "C" {

int gpum_b200_session_train_surrogate(gpum_b200_session* s, gpum_b200_mlp* m,
                                      uint32_t holdout_every, int whiten, uint32_t n_stages,
                                      const uint32_t* steps, const double* lrs,
                                      float* out_loss, double* out_info, char* err,
                                      size_t err_len) {
  return guard(err, err_len, [&] {
    require(s != nullptr && m != nullptr, "session or surrogate is NULL");
    require(mlp_input_width(m) == (int)s->np,
            "surrogate input width does not match the model's parameter count");
    require(holdout_every != 1, "holdout_every = 1 would hold out every pair");
    s->settle_recording();
    const uint64_t n64 = s->rec_count;
    require(n64 >= 2 && s->rec_ll.p, "fewer than two recorded pairs");
    require(n64 < kHeldOut, "too many recorded pairs", GPUM_ERR_UNSUPPORTED);
    const uint32_t n = (uint32_t)n64;
    const int d = (int)s->np;
    s->check_device_error();
    cudaStream_t st = s->stream;
    DBuf<uint32_t> pos, counts;
    pos.ensure(n);
    counts.ensure(2);
    pairs_split_kernel<<<1, kSplitThreads, 0, st>>>(s->rec_theta.p, s->rec_ll.p, n, d,
                                                    holdout_every, pos.p, counts.p);
    GPUM_CK(cudaGetLastError());
    uint32_t cnt[2] = {0, 0};
    GPUM_CK(cudaMemcpyAsync(cnt, counts.p, sizeof cnt, cudaMemcpyDeviceToHost, st));
    GPUM_CK(cudaStreamSynchronize(st));
    const uint32_t n_tr = cnt[0], n_ho = cnt[1];
    require(n_tr >= 2, "fewer than two finite training pairs");
    DBuf<float> tr_th;
    DBuf<double> tr_ll, ho_th, ho_ll;
    tr_th.ensure((size_t)n_tr * d);
    tr_ll.ensure(n_tr);
    ho_th.ensure((size_t)std::max<uint32_t>(n_ho, 1) * d);
    ho_ll.ensure(std::max<uint32_t>(n_ho, 1));
    pairs_scatter_kernel<<<(n + 255) / 256, 256, 0, st>>>(s->rec_theta.p, s->rec_ll.p, n, d,
                                                           pos.p, tr_th.p, tr_ll.p, ho_th.p,
                                                           ho_ll.p);
    GPUM_CK(cudaGetLastError());

    // Moments of the training pairs (f64, fixed order) -> the normaliser.
    const int NA = d + d * (d + 1) / 2 + 2;
    const uint32_t nchunk = std::max<uint32_t>(1, std::min<uint32_t>(64, n_tr / 2048));
    const uint32_t chunk = (n_tr + nchunk - 1) / nchunk;
    const size_t msmem = (size_t)kMomRows * (d + 1) * sizeof(double);
    if (msmem > 48 * 1024)
      GPUM_CK(cudaFuncSetAttribute(pairs_moments_kernel,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msmem));
    DBuf<double> part;
    part.ensure((size_t)nchunk * NA);
    pairs_moments_kernel<<<dim3(nchunk, (NA + 255) / 256), 256, msmem, st>>>(
        tr_th.p, tr_ll.p, n_tr, d, chunk, part.p);
    GPUM_CK(cudaGetLastError());
    std::vector<double> hp((size_t)nchunk * NA);
    std::vector<float> x0(d);
    double y0 = 0.0;
    GPUM_CK(cudaMemcpyAsync(hp.data(), part.p, hp.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
    GPUM_CK(cudaMemcpyAsync(x0.data(), tr_th.p, d * sizeof(float), cudaMemcpyDeviceToHost, st));
    GPUM_CK(cudaMemcpyAsync(&y0, tr_ll.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    GPUM_CK(cudaStreamSynchronize(st));
    std::vector<double> S(NA, 0.0);
    for (uint32_t c = 0; c < nchunk; ++c)
      for (int a = 0; a < NA; ++a) S[a] += hp[(size_t)c * NA + a];
    const double N = (double)n_tr;
    std::vector<double> mean(d), cov((size_t)d * d);
    for (int j = 0; j < d; ++j) mean[j] = (double)x0[j] + S[j] / N;
    for (int j = 0, a = d; j < d; ++j)
      for (int k = j; k < d; ++k, ++a) {
        const double c = (S[a] - S[j] * S[k] / N) / (N - 1.0);
        cov[(size_t)j * d + k] = cov[(size_t)k * d + j] = c;
      }
    const double sy = S[NA - 2], syy = S[NA - 1];
    const double ymean = y0 + sy / N;
    const double yvar = (syy - sy * sy / N) / N;
    const double ysd = yvar > 0.0 && std::isfinite(yvar) ? std::sqrt(yvar) : 1.0;
    char merr[512];
    bool whitened = false;
    if (whiten && d > 1) {
      double md = 0.0;
      for (int j = 0; j < d; ++j) md += cov[(size_t)j * d + j];
      md = std::max(md / d, 1e-300);
      std::vector<double> cj = cov, Linv;
      for (int j = 0; j < d; ++j) cj[(size_t)j * d + j] += 1e-10 * md;
      if (cholesky_inverse(d, cj, &Linv)) {
        const int rc = gpum_b200_mlp_set_whitening(m, mean.data(), Linv.data(), ymean, ysd,
                                                   merr, sizeof merr);
        if (rc != GPUM_OK) throw Failure{rc, merr};
        whitened = true;
      }
    }
    if (!whitened) {
      std::vector<double> sd(d);
      for (int j = 0; j < d; ++j) {
        const double v = cov[(size_t)j * d + j] * (N - 1.0) / N;
        sd[j] = v > 0.0 && std::isfinite(v) ? std::sqrt(v) : 1.0;
      }
      const int rc = gpum_b200_mlp_set_normalizer(m, mean.data(), sd.data(), ymean, ysd, merr,
                                                  sizeof merr);
      if (rc != GPUM_OK) throw Failure{rc, merr};
    }

    std::string e;
    int rc = mlp_train_device(m, tr_th.p, tr_ll.p, n_tr, n_stages, steps, lrs, out_loss, &e);
    if (rc != GPUM_OK) throw Failure{rc, e};

    double resid_sd = std::nan("");
    if (n_ho > 0) {  // residual spread of the trained network on the held-out pairs
      DBuf<double> pred;
      pred.ensure(n_ho);
      rc = mlp_infer(m, ho_th.p, (int)n_ho, d, pred.p, st, &e);
      if (rc != GPUM_OK) throw Failure{rc, e};
      std::vector<double> hpred(n_ho), hll(n_ho);
      GPUM_CK(cudaMemcpyAsync(hpred.data(), pred.p, n_ho * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
      GPUM_CK(cudaMemcpyAsync(hll.data(), ho_ll.p, n_ho * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
      GPUM_CK(cudaStreamSynchronize(st));
      double mr = 0.0, m2 = 0.0;
      for (uint32_t i = 0; i < n_ho; ++i) mr += hpred[i] - hll[i];
      mr /= n_ho;
      for (uint32_t i = 0; i < n_ho; ++i) {
        const double r = hpred[i] - hll[i] - mr;
        m2 += r * r;
      }
      resid_sd = std::sqrt(m2 / n_ho);
    }
    if (out_info) {
      out_info[0] = (double)n;
      out_info[1] = (double)n_tr;
      out_info[2] = (double)n_ho;
      out_info[3] = resid_sd;
      out_info[4] = whitened ? 1.0 : 0.0;
    }
  });
}

int gpum_b200_session_recorded(gpum_b200_session* s, float* out_theta, double* out_ll,
                               uint64_t max_pairs, uint64_t* n_pairs, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    require(s != nullptr, "session is NULL");
    s->settle_recording();
    const uint64_t n = std::min<uint64_t>(s->rec_count, max_pairs);
    if (n_pairs) *n_pairs = s->rec_count;
    if (n == 0) return;
    require(out_theta && out_ll, "output pointers are NULL");
    s->check_device_error();
    GPUM_CK(cudaMemcpyAsync(out_theta, s->rec_theta.p, sizeof(float) * n * s->np,
                            cudaMemcpyDeviceToHost, s->stream));
    GPUM_CK(cudaMemcpyAsync(out_ll, s->rec_ll.p, sizeof(double) * n, cudaMemcpyDeviceToHost,
                            s->stream));
    GPUM_CK(cudaStreamSynchronize(s->stream));
  });
}

int gpum_b200_session_selftest_wait(gpum_b200_session* s, uint32_t polls, char* err,
                                    size_t err_len) {
  return guard(err, err_len, [&] {
    require(s != nullptr, "session is NULL");
    require(polls >= 1 && polls <= (1u << 20), "polls must be in 1..2^20");
    selftest_wait_kernel<<<1, 32, 0, s->stream>>>(s->d_err.p, polls, 50000000ull);
    GPUM_CK(cudaGetLastError());
    ++s->launches;
    s->check_device_error();
  });
}

int gpum_b200_session_run_da(gpum_b200_session* s, gpum_b200_mlp* surrogate, const double* init,
                             const double* sd, const double* temps, uint32_t n_chains,
                             uint32_t n_iter, uint32_t seed, uint32_t mode, double gamma,
                             double de_noise, const double* L, size_t n_l, int rng,
                             float* out_draws, float* out_accept, double* out_last,
                             uint32_t* out_exact, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    run_da(s, surrogate, init, sd, temps, n_chains, n_iter, seed, mode, gamma, de_noise, L, n_l,
           rng, out_draws, out_accept, out_last, out_exact);
  });
}

}  // extern "C"
