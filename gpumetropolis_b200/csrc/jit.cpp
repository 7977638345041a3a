// jit.cpp -- NVRTC build of the compiled engine (see jit.hpp).
#include "jit.hpp"

#include <dlfcn.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <vector>

namespace gpum {

namespace {

// The kernel headers, embedded at build time (build.py writes _embedded.inc
// from device.cuh, common.cuh and compiled.cuh).
#include "_embedded.inc"

typedef int nvrtcResult_;
typedef struct _nvrtcProgram* nvrtcProgram_;

struct Nvrtc {
  void* h = nullptr;
  nvrtcResult_ (*create)(nvrtcProgram_*, const char*, const char*, int, const char* const*,
                         const char* const*) = nullptr;
  nvrtcResult_ (*compile)(nvrtcProgram_, int, const char* const*) = nullptr;
  nvrtcResult_ (*log_size)(nvrtcProgram_, size_t*) = nullptr;
  nvrtcResult_ (*log)(nvrtcProgram_, char*) = nullptr;
  nvrtcResult_ (*cubin_size)(nvrtcProgram_, size_t*) = nullptr;
  nvrtcResult_ (*cubin)(nvrtcProgram_, char*) = nullptr;
  nvrtcResult_ (*destroy)(nvrtcProgram_*) = nullptr;
  const char* (*errstr)(nvrtcResult_) = nullptr;
  std::string load_error;

  bool load() {
    if (h) return true;
    const char* names[] = {"libnvrtc.so.12", "libnvrtc.so",
                           "/usr/local/cuda/lib64/libnvrtc.so.12"};
    for (const char* n : names) {
      h = dlopen(n, RTLD_NOW | RTLD_LOCAL);
      if (h) break;
    }
    if (!h) {
      load_error = "NVRTC (libnvrtc.so.12) cannot be loaded";
      return false;
    }
    auto sym = [&](const char* s) { return dlsym(h, s); };
    create = (decltype(create))sym("nvrtcCreateProgram");
    compile = (decltype(compile))sym("nvrtcCompileProgram");
    log_size = (decltype(log_size))sym("nvrtcGetProgramLogSize");
    log = (decltype(log))sym("nvrtcGetProgramLog");
    cubin_size = (decltype(cubin_size))sym("nvrtcGetCUBINSize");
    cubin = (decltype(cubin))sym("nvrtcGetCUBIN");
    destroy = (decltype(destroy))sym("nvrtcDestroyProgram");
    errstr = (decltype(errstr))sym("nvrtcGetErrorString");
    if (!create || !compile || !log_size || !log || !cubin_size || !cubin || !destroy ||
        !errstr) {
      load_error = "NVRTC is missing entry points";
      dlclose(h);
      h = nullptr;
      return false;
    }
    return true;
  }
};

Nvrtc& nvrtc() {
  static Nvrtc n;
  return n;
}

std::mutex g_mu;

struct CacheEntry {
  cudaLibrary_t lib = nullptr;
  CompiledModel model;
};

std::map<size_t, CacheEntry>& cache() {
  static std::map<size_t, CacheEntry> c;
  return c;
}

// On-disk cubin cache: $GPUM_B200_CACHE, else a _jit_cache directory next to
// this shared library.  A missing or unwritable cache only costs rebuilds.
std::string cache_dir() {
  const char* env = std::getenv("GPUM_B200_CACHE");
  if (env && *env) return env;
  Dl_info info;
  if (dladdr((void*)&cache_dir, &info) && info.dli_fname) {
    std::string p = info.dli_fname;
    const size_t k = p.rfind('/');
    if (k != std::string::npos) return p.substr(0, k) + "/_jit_cache";
  }
  return "";
}

bool cache_read(const std::string& path, std::vector<char>* out) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  bool ok = n > 0;
  if (ok) {
    out->resize((size_t)n);
    ok = std::fread(out->data(), 1, (size_t)n, f) == (size_t)n;
  }
  std::fclose(f);
  return ok;
}

void cache_write(const std::string& dir, const std::string& path, const std::vector<char>& c) {
  mkdir(dir.c_str(), 0755);
  const std::string tmp = path + ".tmp" + std::to_string((long)getpid());
  FILE* f = std::fopen(tmp.c_str(), "wb");
  if (!f) return;
  const bool ok = std::fwrite(c.data(), 1, c.size(), f) == c.size();
  std::fclose(f);
  if (ok) std::rename(tmp.c_str(), path.c_str());
  else std::remove(tmp.c_str());
}

int build_cubin_uncached(const std::string& src, std::vector<char>* out, std::string* err);

int build_cubin(const std::string& src, std::vector<char>* out, std::string* err) {
  const std::string dir = cache_dir();
  char key[32];
  std::snprintf(key, sizeof key, "%016zx", std::hash<std::string>()(src + kEmbeddedDevice +
                                                                    kEmbeddedCommon +
                                                                    kEmbeddedCompiled));
  const std::string path = dir.empty() ? "" : dir + "/gm_" + key + ".cubin";
  if (!path.empty() && cache_read(path, out)) return 0;
  if (build_cubin_uncached(src, out, err)) return 1;
  if (!path.empty()) cache_write(dir, path, *out);
  return 0;
}

int build_cubin_uncached(const std::string& src, std::vector<char>* out, std::string* err) {
  Nvrtc& nv = nvrtc();
  if (!nv.load()) {
    *err = nv.load_error;
    return 1;
  }
  const char* hdr_src[] = {kEmbeddedDevice, kEmbeddedCommon, kEmbeddedCompiled};
  const char* hdr_name[] = {"device.cuh", "common.cuh", "compiled.cuh"};
  nvrtcProgram_ prog = nullptr;
  int r = nv.create(&prog, src.c_str(), "gm_model.cu", 3, hdr_src, hdr_name);
  if (r != 0) {
    *err = std::string("nvrtcCreateProgram: ") + nv.errstr(r);
    return 1;
  }
  const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo",
                        "--fmad=true", "-DGPUM_NVRTC=1"};
  r = nv.compile(prog, 5, opts);
  if (r != 0) {
    size_t n = 0;
    nv.log_size(prog, &n);
    std::string log(n, '\0');
    if (n) nv.log(prog, &log[0]);
    *err = std::string("NVRTC compile failed: ") + nv.errstr(r) + "\n" + log;
    nv.destroy(&prog);
    return 1;
  }
  size_t n = 0;
  nv.cubin_size(prog, &n);
  out->resize(n);
  nv.cubin(prog, out->data());
  nv.destroy(&prog);
  return 0;
}

}  // namespace

void jit_chains_per_thread(int np, int nh, int* G, int* GG, bool* pair) {
  // The paired body keeps G x (parameters + hoisted values) broadcast pairs
  // in registers: use it while that stays within 96 registers.
  const int w = np + std::max(nh, 1);
  *pair = w <= 48;
  if (*pair) *G = w <= 24 ? 2 : 1;
  else *G = np <= 24 ? 4 : (np <= 48 ? 2 : 1);
  // Chains per thread of the scalar gradient body (models too wide for the
  // chain-lane gradient body).
  *GG = np <= 16 ? 2 : 1;
}

bool jit_value_lanes(const GenModel& gm, bool pair) {
  return !pair && gm.np + std::max(gm.n_hoist, 1) <= 160;
}

bool jit_grad_lanes(const GenModel& gm) { return gm.np + std::max(gm.n_hoist, 1) <= 100; }

std::string jit_source(const GenModel& gm, int G, int GG, bool pair) {
  const bool lanes = jit_value_lanes(gm, pair);
  const bool lanes_grad = jit_grad_lanes(gm);
  std::string s;
  s += "#include \"device.cuh\"\n";
  s += "#define GM_LANES " + std::string(lanes ? "1" : "0") + "\n";
  s += "#define GM_LANESG " + std::string(lanes_grad ? "1" : "0") + "\n";
  s += "#define GM_PAIR " + std::string(pair ? "1" : "0") + "\n";
  s += "#define GM_G " + std::to_string(G) + "\n";
  s += "#define GM_GG " + std::to_string(GG) + "\n";
  // Narrow paired models with two chains per thread (2 x (parameters +
  // hoisted values) <= 40 broadcast pairs) fit in 80 registers without
  // spills: three CTAs, 24 warps per SM.
  const int w = gm.np + std::max(gm.n_hoist, 1);
  // Paired gradient body of at most 25 parameters + hoisted values: two CTAs.
  s += "#define GM_GRAD_CTAS 1\n";  // the gradient bodies keep up to 255 registers
  // Chain lanes: two CTAs while parameters + hoisted values stay within 80.
  s += "#define GM_VALUE_CTAS " +
       std::to_string(pair ? (G == 2 && G * w <= 40 ? 3 : 2) : (lanes && w <= 80 ? 2 : 1)) +
       "\n";
  s += "namespace gpum {\n";
  s += gm.source;
  s += "}  // namespace gpum\nusing namespace gpum;\n";
  s += "#include \"compiled.cuh\"\n";
  return s;
}

int jit_compile_check(const GenModel& gm, size_t* cubin_bytes, std::string* err) {
  int G = 1, GG = 1;
  bool pair = false;
  jit_chains_per_thread(gm.np, gm.n_hoist, &G, &GG, &pair);
  std::vector<char> cubin;
  if (build_cubin(jit_source(gm, G, GG, pair), &cubin, err)) return 1;
  if (cubin_bytes) *cubin_bytes = cubin.size();
  return 0;
}

int jit_compile(const GenModel& gm, CompiledModel* out, std::string* err) {
  int G = 1, GG = 1;
  bool pair = false;
  jit_chains_per_thread(gm.np, gm.n_hoist, &G, &GG, &pair);
  const std::string src = jit_source(gm, G, GG, pair);
  const size_t key = std::hash<std::string>()(src);
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = cache().find(key);
  if (it != cache().end()) {
    *out = it->second.model;
    return 0;
  }
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<char> cubin;
  if (build_cubin(src, &cubin, err)) return 1;
  CacheEntry e;
  cudaError_t ce = cudaLibraryLoadData(&e.lib, cubin.data(), nullptr, nullptr, 0, nullptr,
                                       nullptr, 0);
  if (ce != cudaSuccess) {
    *err = std::string("cudaLibraryLoadData: ") + cudaGetErrorString(ce);
    return 1;
  }
  if (cudaLibraryGetKernel(&e.model.k_value, e.lib, "gm_iter_value") != cudaSuccess ||
      cudaLibraryGetKernel(&e.model.k_grad, e.lib, "gm_iter_grad") != cudaSuccess ||
      cudaLibraryGetKernel(&e.model.k_mat, e.lib, "gm_materialize") != cudaSuccess ||
      cudaLibraryGetKernel(&e.model.k_prior, e.lib, "gm_prior_batch") != cudaSuccess) {
    *err = "compiled model is missing its kernels";
    cudaLibraryUnload(e.lib);
    return 1;
  }
  if (gm.tc && (cudaLibraryGetKernel(&e.model.k_value_tc, e.lib, "gm_iter_value_tc") !=
                    cudaSuccess ||
                cudaLibraryGetKernel(&e.model.k_tc_pack, e.lib, "gm_tc_pack") != cudaSuccess)) {
    *err = "compiled model is missing its tensor-core kernels";
    cudaLibraryUnload(e.lib);
    return 1;
  }
  e.model.tc = gm.tc;
  e.model.tc_kp = gm.tc_kp;
  e.model.tc_ntail = gm.tc_ntail;
  e.model.tc_tn = gm.tc_tn;
  e.model.tc_stages = gm.tc_stages;
  e.model.tc_threads = 32 * (gm.tc_warps + 1);
  e.model.G = G;
  e.model.GG = GG;
  e.model.pair = pair;
  e.model.lanes = jit_value_lanes(gm, pair);
  e.model.lanes_grad = jit_grad_lanes(gm);
  e.model.n_mat = gm.n_mat;
  e.model.np = gm.np;
  e.model.compile_seconds =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  cache()[key] = e;
  *out = e.model;
  return 0;
}

}  // namespace gpum
