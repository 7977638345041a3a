// mlp.cu -- the surrogate of the log-likelihood: a d-H-H-1 MLP with SiLU,
// trained and evaluated on the GPU with the tcgen05 GEMM (tc_gemm.cuh).
// No reference counterpart: the surrogate and delayed acceptance are new.
//
// Inputs are standardised parameters (per-coordinate mean and sd of the
// training pairs), the target is the standardised exact log-likelihood, the
// loss is the mean squared error.  Weights live in f32 (master) with Adam
// moments; BF16 copies feed the tensor cores.  All reductions are fixed-order
// (no atomics), so training is bitwise repeatable for a given seed.
//
// Per training step, for a batch of B rows (B, H multiples of 128; the input
// width is padded to dp, a multiple of 64):
//   Z1 = X W1^T + b1, A1 = silu(Z1)          tcgen05 GEMM, fused epilogue
//   Z2 = A1 W2^T + b2, A2 = silu(Z2)         tcgen05 GEMM, fused epilogue
//   yhat = A2 w3 + b3; r = yhat - t          row kernel (warp per row)
//   dZ2 = (2r/B) w3 * silu'(Z2)              row kernel
//   dW2 = dZ2^T A1                           tcgen05 GEMM (K = B)
//   dA1 = dZ2 W2                             tcgen05 GEMM (K = H)
//   dZ1 = dA1 * silu'(Z1); dW1 = dZ1^T X     elementwise + tcgen05 GEMM
//   biases / w3: fixed-order column sums; Adam on every parameter.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "../../include/gpum_b200.h"
#include "tc_gemm.cuh"

using namespace gpum;
typedef __nv_bfloat16 bf16;

namespace {

struct MlpFail {
  int code;
  std::string msg;
};

#define MLP_CK(call)                                                                   \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      throw MlpFail{e_ == cudaErrorMemoryAllocation ? GPUM_ERR_NOMEM : GPUM_ERR_CUDA,  \
                    std::string(#call) + ": " + cudaGetErrorString(e_)};              \
  } while (0)

template <class T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    if (p) cudaFree(p);
    p = nullptr;
    MLP_CK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    n = count;
  }
  ~Buf() {
    if (p) cudaFree(p);
  }
};

// ----------------------------------------------------------------- kernels
__device__ __forceinline__ float sigmoidf_(float z) { return 1.0f / (1.0f + expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = sigmoidf_(z);
  return s * (1.0f + z * (1.0f - s));
}

// Deterministic uniform index for (seed, step, row): Philox counter.
__device__ __forceinline__ uint32_t pick(uint32_t seed, uint32_t step, uint32_t row, uint32_t n) {
  const U4 r = philox4x32_10(U4{row, step, 0x4D4C5031u, 0u}, seed, 0x2545F491u);
  return (uint32_t)(((uint64_t)r.x * n) >> 32);
}

// Input transform of one row into Xh (bf16, zero padded to dp):
//   per coordinate  v_j = (theta_j - xmean_j) * xinv_j            (xw == nullptr)
//   whitening       v_j = sum_k xw[j][k] (theta_k - xmean_k)      (xw: d x d)
// `cen` is block-shared scratch of d floats.  Called by every thread.
template <class Src>
__device__ __forceinline__ void mlp_input_row(Src theta_at, bool live, int d, int dp,
                                              const float* __restrict__ xmean,
                                              const float* __restrict__ xinv,
                                              const float* __restrict__ xw, float* cen,
                                              bf16* __restrict__ out) {
  if (xw) {
    for (int k = threadIdx.x; k < d; k += blockDim.x) cen[k] = live ? theta_at(k) - xmean[k] : 0.0f;
    __syncthreads();
  }
  for (int j = threadIdx.x; j < dp; j += blockDim.x) {
    float v = 0.0f;
    if (live && j < d) {
      if (xw) {
        const float* wr = xw + (size_t)j * d;
        for (int k = 0; k < d; ++k) v = fmaf(wr[k], cen[k], v);
      } else {
        v = (theta_at(j) - xmean[j]) * xinv[j];
      }
    }
    out[j] = __float2bfloat16(v);
  }
}

// Batch rows: transformed inputs (bf16, padded with zeros) and targets.
// idx_mode 0: rows 0..n-1 in order (inference / gradient check);
//          1: Philox-random rows of the training set.
__global__ void mlp_gather(const float* __restrict__ theta, const double* __restrict__ ll,
                           size_t n, int d, int dp, int B, int idx_mode, uint32_t seed,
                           uint32_t step, const float* __restrict__ xmean,
                           const float* __restrict__ xinv, const float* __restrict__ xw,
                           float ymean, float yinv, bf16* __restrict__ Xh,
                           float* __restrict__ t) {
  __shared__ float cen[256];
  const int row = blockIdx.x;
  if (row >= B) return;
  size_t src = idx_mode ? pick(seed, step, (uint32_t)row, (uint32_t)n) : (size_t)row;
  const bool live = src < n;
  if (!live) src = 0;
  const float* th = theta + src * d;
  mlp_input_row([&](int k) { return th[k]; }, live, d, dp, xmean, xinv, xw, cen,
                Xh + (size_t)row * dp);
  if (threadIdx.x == 0 && t) t[row] = live && ll ? (float)((ll[src] - ymean) * yinv) : 0.0f;
}

// Output layer, loss and dZ2 for one row per warp (fixed lane-order sums).
//   yhat = silu(Z2) . w3 + b3; r = yhat - t; loss row = r^2
//   dZ2 = (2 r / B) w3 * silu'(Z2)  (f32 and bf16, and bf16 transposed)
__global__ void mlp_head(const float* __restrict__ Z2, const float* __restrict__ w3,
                         const float* __restrict__ b3, const float* __restrict__ t, int B,
                         int H, int n_live, float* __restrict__ yhat, float* __restrict__ rsq,
                         float* __restrict__ dyhat, bf16* __restrict__ dZ2h,
                         bf16* __restrict__ dZ2Th, int backward) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= B) return;
  const float* z = Z2 + (size_t)warp * H;
  float acc = 0.0f;
  for (int j = lane; j < H; j += 32) acc += silu(z[j]) * w3[j];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  const float y = acc + b3[0];
  if (lane == 0 && yhat) yhat[warp] = y;
  if (!backward) return;
  const bool live = warp < n_live;
  const float r = live ? y - t[warp] : 0.0f;
  if (lane == 0) {
    rsq[warp] = r * r;
    dyhat[warp] = 2.0f * r / (float)n_live;
  }
  const float g = 2.0f * r / (float)n_live;
  for (int j = lane; j < H; j += 32) {
    const float dz = g * w3[j] * dsilu(z[j]);
    dZ2h[(size_t)warp * H + j] = __float2bfloat16(dz);
    dZ2Th[(size_t)j * B + warp] = __float2bfloat16(dz);
  }
}

// dZ1 = dA1 * silu'(Z1) -> bf16 transposed [H][B] and f32 [B][H] for db1.
__global__ void mlp_dz1(const float* __restrict__ dA1, const float* __restrict__ Z1, int B, int H,
                        float* __restrict__ dZ1, bf16* __restrict__ dZ1Th) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)B * H) return;
  const size_t b = i / H, j = i % H;
  const float v = dA1[i] * dsilu(Z1[i]);
  dZ1[i] = v;
  dZ1Th[j * B + b] = __float2bfloat16(v);
}

// bf16 [R][Cc] -> [Cc][R]
__global__ void mlp_transpose(const bf16* __restrict__ in, bf16* __restrict__ out, int R, int Cc) {
  __shared__ bf16 tile[32][34];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = r0 + y, c = c0 + threadIdx.x;
    if (r < R && c < Cc) tile[y][threadIdx.x] = in[(size_t)r * Cc + c];
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int c = c0 + y, r = r0 + threadIdx.x;
    if (r < R && c < Cc) out[(size_t)c * R + r] = tile[threadIdx.x][y];
  }
}

// Column sums out[j] = scale_j * sum_b f(M[b][j]) * (s ? s[b] : 1) with
// f = identity, silu or silu' (mode 0/1/2), in two fixed-order passes: blocks
// of 32 columns x kColRows rows (8 warps, each a fixed row stride, then the
// warps in order) write partials[chunk][j]; the second pass adds the chunks
// in order.  Deterministic, and parallel over rows.
constexpr int kColRows = 128;

__global__ void mlp_colsum_part(const float* __restrict__ M, const float* __restrict__ s, int B,
                                int H, int mode, float* __restrict__ part) {
  __shared__ float red[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int j = blockIdx.x * 32 + lane;
  const int b0 = blockIdx.y * kColRows, b1 = min(b0 + kColRows, B);
  float acc = 0.0f;
  if (j < H) {
    for (int b = b0 + w; b < b1; b += 8) {
      float v = M[(size_t)b * H + j];
      v = mode == 1 ? silu(v) : (mode == 2 ? dsilu(v) : v);
      acc += s ? v * s[b] : v;
    }
  }
  red[w][lane] = acc;
  __syncthreads();
  if (w == 0 && j < H) {
    float t = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) t += red[k][lane];
    part[(size_t)blockIdx.y * H + j] = t;
  }
}

__global__ void mlp_colsum_fin(const float* __restrict__ part, int nchunk, int H,
                               const float* __restrict__ scale, float* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= H) return;
  float t = 0.0f;
  for (int c = 0; c < nchunk; ++c) t += part[(size_t)c * H + j];
  out[j] = scale ? t * scale[j] : t;
}

// out[0] = sum of v[0..n), fixed order: 256 strided per-thread sums, then a
// fixed shared-memory tree.  One block of 256 threads.
__global__ void mlp_sum(const float* __restrict__ v, int n, float* __restrict__ out) {
  __shared__ float red[256];
  float t = 0.0f;
  for (int i = threadIdx.x; i < n; i += 256) t += v[i];
  red[threadIdx.x] = t;
  __syncthreads();
  for (int off = 128; off > 0; off >>= 1) {
    if ((int)threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0];
}

// Adam (Kingma & Ba) with bias correction; also refreshes the bf16 copy and,
// when `wt` is set, the transposed bf16 copy of an R x Cc weight.
__global__ void mlp_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                         const float* __restrict__ g, size_t n, float lr, float b1, float b2,
                         float c1, float c2, float eps, bf16* __restrict__ wh,
                         bf16* __restrict__ wt, int R, int Cc) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wh) wh[i] = __float2bfloat16(wi);
  if (wt) wt[(i % Cc) * R + i / Cc] = __float2bfloat16(wi);
}

__global__ void mlp_init_weights(float* __restrict__ w, size_t n, int fan_in, int cols_live,
                                 int cols, uint32_t seed, uint32_t tag) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int col = (int)(i % cols);
  const U4 r = philox4x32_10(U4{(uint32_t)i, tag, 0x57494E49u, 0u}, seed, 0x9E3779B9u);
  const float u = ((float)(r.x >> 8) + 0.5f) * (1.0f / 16777216.0f);
  const float bound = sqrtf(6.0f / (float)fan_in);  // He-uniform style for SiLU
  w[i] = col < cols_live ? (2.0f * u - 1.0f) * bound : 0.0f;
}

__global__ void mlp_to_bf16(const float* __restrict__ w, bf16* __restrict__ wh,
                            bf16* __restrict__ wt, size_t n, int R, int Cc) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  wh[i] = __float2bfloat16(w[i]);
  if (wt) wt[(i % Cc) * R + i / Cc] = __float2bfloat16(w[i]);
}

unsigned blocks(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// Inference gather from f64 chain-major parameters [n][d].
__global__ void mlp_gather64(const double* __restrict__ theta, int n, int d, int dp, int B,
                             const float* __restrict__ xmean, const float* __restrict__ xinv,
                             const float* __restrict__ xw, bf16* __restrict__ Xh) {
  __shared__ float cen[256];
  const int row = blockIdx.x;
  if (row >= B) return;
  const bool live = row < n;
  const double* th = theta + (size_t)(live ? row : 0) * d;
  mlp_input_row([&](int k) { return (float)th[k]; }, live, d, dp, xmean, xinv, xw, cen,
                Xh + (size_t)row * dp);
}

__global__ void mlp_unscale(const float* __restrict__ y, int n, float ysd, float ymean,
                            double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (double)y[i] * ysd + ymean;
}

// Fused inference for 128 rows per CTA, for d <= 64 (dp = 64) and H in
// {128, 256}, with 512 threads: warp w serves TMEM lane quarter w % 4 (rows
// 32 (w % 4) + lane) and hidden-column quarter w / 4, so both epilogues are
// spread over 16 warps.
//   X = transform(theta) -> shared (bf16, K-major core matrices)
//   Z1 = X W1^T  (tcgen05, M = 128, N = H, K = 64, accumulators in TMEM)
//   A1 = silu(Z1 + b1) -> shared (bf16, the K-major A operand of layer 2)
//   Z2 = A1 W2^T (tcgen05, K = H in 64-wide slices; each W2 slice staged in
//        shared memory, the next one prefetched into registers meanwhile)
//   y  = silu(Z2 + b2) . w3 + b3 (four column-quarter partials added in
//        order);  out = y * ysd + ymean   (f64)
// Shared memory: X 16 KB | W1 H x 64 | A1 (H / 64) x 16 KB | W2 slice H x 64.
// The whitening scratch (centred inputs, 128 x 64 f32) and the head
// partials live in A1's space when it is free.  Waits are bounded; a timeout
// sets the error word and skips the epilogues.
constexpr int kInfRows = 128;
constexpr int kInfThreads = 512;

__host__ __device__ constexpr size_t mlp_infer_smem(int H) {
  return (size_t)kInfRows * 64 * 2 + (size_t)H * 64 * 2 + (size_t)(H / 64) * kInfRows * 64 * 2 +
         (size_t)H * 64 * 2 + 64;
}

__global__ void __launch_bounds__(kInfThreads, 1)
mlp_infer_fused(const double* __restrict__ theta, int n, int d, int H,
                const float* __restrict__ xmean, const float* __restrict__ xinv,
                const float* __restrict__ xw, const bf16* __restrict__ W1h,
                const float* __restrict__ b1, const bf16* __restrict__ W2h,
                const float* __restrict__ b2, const float* __restrict__ w3,
                const float* __restrict__ b3, float ysd, float ymean, double* __restrict__ out,
                uint32_t* err) {
  extern __shared__ __align__(1024) unsigned char fsm[];
  constexpr int kSlice = kInfRows * 64 * 2;  // one 128 x 64 bf16 slice
  unsigned char* sx = fsm;
  unsigned char* sw1 = sx + kSlice;
  unsigned char* sa1 = sw1 + (size_t)H * 128;
  unsigned char* sw2 = sa1 + (size_t)(H / 64) * kSlice;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sw2 + (size_t)H * 128);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int rloc = (warp & 3) * 32 + lane;  // this thread's TMEM lane = row
  const int quarter = warp >> 2;            // hidden-column quarter
  const int row0 = blockIdx.x * kInfRows;
  const int KH = H / 64;

  if (warp == 0) tmem_alloc(tslot, 256);
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }

  // Inputs: row rloc, input columns [16 quarter, 16 quarter + 16).  The
  // centred values go to a swizzled scratch (conflict-free column access).
  float* cen = reinterpret_cast<float*>(sa1);
  {
    const int row = row0 + rloc;
    const bool live = row < n;
    const double* th = theta + (size_t)(live ? row : 0) * d;
    for (int j = quarter; j < d; j += 4)
      cen[rloc * 64 + ((j + rloc) & 63)] = live ? (float)th[j] - xmean[j] : 0.0f;
    __syncthreads();
    for (int k8 = quarter * 16; k8 < quarter * 16 + 16; k8 += 8) {
      __align__(16) bf16 v8[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int k = k8 + q;
        float v = 0.0f;
        if (live && k < d) {
          if (xw) {
            const float* wr = xw + (size_t)k * d;
            for (int j = 0; j < d; ++j) v = fmaf(wr[j], cen[rloc * 64 + ((j + rloc) & 63)], v);
          } else {
            v = cen[rloc * 64 + ((k + rloc) & 63)] * xinv[k];
          }
        }
        v8[q] = __float2bfloat16(v);
      }
      *reinterpret_cast<uint4*>(sx + kmajor_offset(rloc, k8, kInfRows)) =
          *reinterpret_cast<const uint4*>(v8);
    }
  }
  // W1 (H x 64) into its K-major layout.
  for (int i = tid; i < H * 8; i += kInfThreads) {
    const int r = i >> 3, c8 = (i & 7) * 8;
    *reinterpret_cast<uint4*>(sw1 + kmajor_offset(r, c8, H)) =
        *reinterpret_cast<const uint4*>(W1h + (size_t)r * 64 + c8);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma_idesc_bf16(kInfRows, H);
  const uint32_t lbo_x = (kInfRows / 8) * 128, lbo_h = (uint32_t)(H / 8) * 128;
  if (tid == 0) {
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
      umma_bf16(tmem, umma_smem_desc(smem_addr(sx) + 2 * kk * lbo_x, lbo_x, 128),
                umma_smem_desc(smem_addr(sw1) + 2 * kk * lbo_h, lbo_h, 128), idesc,
                kk > 0 ? 1u : 0u);
    umma_commit(bar);
  }
  // W2 slice prefetch into registers while layer 1 runs (H x 64 per slice).
  constexpr int kMaxPf = 256 * 8 / kInfThreads;  // 4 chunks per thread at H = 256
  uint4 pf[kMaxPf];
  const int npf = H * 8 / kInfThreads;
  auto load_w2 = [&](int s) {
#pragma unroll
    for (int q = 0; q < kMaxPf; ++q) {
      if (q < npf) {
        const int i = tid + q * kInfThreads, r = i >> 3, c8 = (i & 7) * 8;
        pf[q] = *reinterpret_cast<const uint4*>(W2h + (size_t)r * H + s * 64 + c8);
      }
    }
  };
  auto store_w2 = [&]() {
#pragma unroll
    for (int q = 0; q < kMaxPf; ++q) {
      if (q < npf) {
        const int i = tid + q * kInfThreads, r = i >> 3, c8 = (i & 7) * 8;
        *reinterpret_cast<uint4*>(sw2 + kmajor_offset(r, c8, H)) = pf[q];
      }
    }
  };
  load_w2(0);
  int ok = mbar_wait_bounded(bar, 0u) ? 1 : 0;
  ok = __syncthreads_and(ok);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  const int cq = H / 4;  // hidden columns per quarter (64 or 32)
  const uint32_t trow = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  if (ok) {
    // Layer-1 epilogue: A1 = silu(Z1 + b1) as bf16 into the layer-2 A operand.
    for (int c = quarter * cq; c < quarter * cq + cq; c += 16) {
      float v[16];
      tmem_ld16(trow + (uint32_t)c, v);
      __align__(16) bf16 a8[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) a8[j] = __float2bfloat16(silu(v[j] + b1[c + j]));
      unsigned char* base = sa1 + (size_t)(c / 64) * kSlice;
      *reinterpret_cast<uint4*>(base + kmajor_offset(rloc, c % 64, kInfRows)) =
          *reinterpret_cast<const uint4*>(a8);
      *reinterpret_cast<uint4*>(base + kmajor_offset(rloc, c % 64 + 8, kInfRows)) =
          *reinterpret_cast<const uint4*>(a8 + 8);
    }
  }
  // Layer 2 over the K slices of A1 / W2.
  for (int s = 0; s < KH && ok; ++s) {
    store_w2();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        umma_bf16(tmem,
                  umma_smem_desc(smem_addr(sa1 + (size_t)s * kSlice) + 2 * kk * lbo_x, lbo_x, 128),
                  umma_smem_desc(smem_addr(sw2) + 2 * kk * lbo_h, lbo_h, 128), idesc,
                  (s > 0 || kk > 0) ? 1u : 0u);
      umma_commit(bar);
    }
    if (s + 1 < KH) load_w2(s + 1);
    ok = mbar_wait_bounded(bar, (uint32_t)((s + 1) & 1)) ? 1 : 0;
    ok = __syncthreads_and(ok);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  // Head: partial dot products per column quarter, added in quarter order.
  // A1's space is free once the last layer-2 MMA has completed.
  float* part = reinterpret_cast<float*>(sa1);
  if (ok) {
    float acc = 0.0f;
    for (int c = quarter * cq; c < quarter * cq + cq; c += 16) {
      float v[16];
      tmem_ld16(trow + (uint32_t)c, v);
#pragma unroll
      for (int j = 0; j < 16; ++j) acc = fmaf(silu(v[j] + b2[c + j]), w3[c + j], acc);
    }
    part[quarter * kInfRows + rloc] = acc;
  } else if (tid == 0) {
    atomicOr(err, DEV_ERR_MMA_TIMEOUT);
  }
  __syncthreads();
  if (ok && quarter == 0) {
    const int row = row0 + rloc;
    const float y = ((part[rloc] + part[kInfRows + rloc]) + part[2 * kInfRows + rloc]) +
                    part[3 * kInfRows + rloc];
    if (row < n) out[row] = (double)(y + b3[0]) * ysd + ymean;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 256);
}

}  // namespace

struct gpum_b200_mlp {
  int d = 0, dp = 0, H = 0, B = 0;
  uint32_t seed = 0;
  uint32_t step = 0;
  cudaStream_t st = nullptr;
  // parameters (f32 master), Adam moments, gradients
  Buf<float> W1, b1, W2, b2, w3, b3;
  Buf<float> mW1, mb1, mW2, mb2, mw3, mb3, vW1, vb1, vW2, vb2, vw3, vb3;
  Buf<float> gW1, gb1, gW2, gb2, gw3, gb3;
  Buf<bf16> W1h, W2h, W2Th;
  // activations and work buffers (batch rows)
  Buf<bf16> Xh, XTh, A1h, A1Th, A2h, dZ2h, dZ2Th, dZ1Th;
  Buf<float> Z1, Z2, t, yhat, rsq, dyhat, dA1, dZ1, loss, scratch;
  Buf<float> colpart;  // [B / kColRows][H] column-sum partials
  Buf<float> splitk;   // split-K GEMM partials
  // normaliser
  Buf<float> xmean, xinv, xw;  // xw: d x d whitening, used when `whiten`
  bool whiten = false;
  const float* xw_or_null() const { return whiten ? xw.p : nullptr; }
  float ymean = 0.0f, yinv = 1.0f, ysd = 1.0f;
  Buf<uint32_t> err;
  int adam_t = 0;
  bool smem_set[2] = {false, false};
  bool infer_smem_set = false;

  // The fused inference kernel covers d <= 64 and H in {128, 256}.
  bool fused_inference() const { return dp == 64 && (H == 128 || H == 256); }

  ~gpum_b200_mlp() {
    if (st) cudaStreamDestroy(st);
  }

  template <int BN>
  void gemm(const bf16* A, const bf16* Bm, float* C, const float* bias, bf16* act, int M, int N,
            int K) {
    const size_t smem = tc_gemm_smem<BN>();
    // Set once, so later launches (possibly under stream capture) make no
    // non-stream API calls.
    if (!smem_set[BN == 128]) {
      MLP_CK(cudaFuncSetAttribute(tc_gemm_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
      smem_set[BN == 128] = true;
    }
    // Long-K products with few output tiles (the weight gradients, K = batch)
    // split K across CTAs so the GPU is not left with a handful of CTAs.
    int S = 1;
    if (!bias && !act) {
      const int tiles = (N / BN) * (M / kGemmBM);
      while (S < 32 && tiles * S < 128 && K % (2 * S * kGemmBK) == 0 &&
             (size_t)2 * S * M * N <= splitk.n)
        S *= 2;
    }
    dim3 grid(N / BN, M / kGemmBM, S);
    tc_gemm_kernel<BN><<<grid, kGemmThreads, smem, st>>>(A, Bm, S > 1 ? splitk.p : C, bias, act,
                                                         M, N, K, K / S, err.p);
    if (S > 1)
      tc_splitk_sum<<<blocks((size_t)M * N), 256, 0, st>>>(splitk.p, S, (size_t)M * N, C);
    MLP_CK(cudaGetLastError());
  }

  void gemm_any(const bf16* A, const bf16* Bm, float* C, const float* bias, bf16* act, int M,
                int N, int K) {
    if (N % 128 == 0) gemm<128>(A, Bm, C, bias, act, M, N, K);
    else gemm<64>(A, Bm, C, bias, act, M, N, K);
  }

  // Forward of the first `rows` rows already gathered into Xh.
  void forward(int rows) {
    gemm_any(Xh.p, W1h.p, Z1.p, b1.p, A1h.p, rows, H, dp);
    gemm_any(A1h.p, W2h.p, Z2.p, b2.p, A2h.p, rows, H, H);
  }

  // Gradients for the gathered batch (n_live real rows of B).
  void backward(int n_live) {
    mlp_head<<<blocks((size_t)B * 32), 256, 0, st>>>(Z2.p, w3.p, b3.p, t.p, B, H, n_live, yhat.p,
                                                     rsq.p, dyhat.p, dZ2h.p, dZ2Th.p, 1);
    MLP_CK(cudaGetLastError());
    // w3 and b3: dw3[j] = sum_b dyhat[b] silu(Z2[b][j]); db3 = sum dyhat
    colsum(Z2.p, dyhat.p, 1, nullptr, gw3.p);
    mlp_sum<<<1, 256, 0, st>>>(dyhat.p, B, gb3.p);
    mlp_sum<<<1, 256, 0, st>>>(rsq.p, B, loss.p);
    // db2 = column sums of dZ2 (from its bf16 transpose would lose bits: use
    // the f32 row kernel output through dA1's buffer as scratch)
    mlp_transpose<<<dim3(H / 32, B / 32), dim3(32, 8), 0, st>>>(A1h.p, A1Th.p, B, H);
    gemm_any(dZ2Th.p, A1Th.p, gW2.p, nullptr, nullptr, H, H, B);  // dW2 = dZ2^T A1
    gemm_any(dZ2h.p, W2Th.p, dA1.p, nullptr, nullptr, B, H, H);   // dA1 = dZ2 W2
    // db2 = sum_b dZ2[b][j]: recompute in f32 from Z2 and dyhat
    db2_from_head();
    mlp_dz1<<<blocks((size_t)B * H), 256, 0, st>>>(dA1.p, Z1.p, B, H, dZ1.p, dZ1Th.p);
    colsum(dZ1.p, nullptr, 0, nullptr, gb1.p);
    mlp_transpose<<<dim3(dp / 32, B / 32), dim3(32, 8), 0, st>>>(Xh.p, XTh.p, B, dp);
    gemm_any(dZ1Th.p, XTh.p, gW1.p, nullptr, nullptr, H, dp, B);  // dW1 = dZ1^T X
    MLP_CK(cudaGetLastError());
  }

  // db2[j] = w3[j] sum_b dyhat[b] silu'(Z2[b][j]), fixed order over b.
  void db2_from_head() { colsum(Z2.p, dyhat.p, 2, w3.p, gb2.p); }

  // Column sums of a B x H row-major matrix (mlp_colsum_part / _fin).
  void colsum(const float* M, const float* sc, int mode, const float* scale, float* out) {
    const int nchunk = (B + kColRows - 1) / kColRows;
    mlp_colsum_part<<<dim3((H + 31) / 32, nchunk), 256, 0, st>>>(M, sc, B, H, mode, colpart.p);
    mlp_colsum_fin<<<blocks(H), 256, 0, st>>>(colpart.p, nchunk, H, scale, out);
    MLP_CK(cudaGetLastError());
  }

  void adam(float lr) {
    ++adam_t;
    const float bb1 = 0.9f, bb2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.0f - std::pow(bb1, (float)adam_t), c2 = 1.0f - std::pow(bb2, (float)adam_t);
    auto go = [&](Buf<float>& w, Buf<float>& m, Buf<float>& v, Buf<float>& g, bf16* wh, bf16* wt,
                  int R, int Cc) {
      mlp_adam<<<blocks(w.n), 256, 0, st>>>(w.p, m.p, v.p, g.p, w.n, lr, bb1, bb2, c1, c2, eps,
                                            wh, wt, R, Cc);
    };
    go(W1, mW1, vW1, gW1, W1h.p, nullptr, H, dp);
    go(b1, mb1, vb1, gb1, nullptr, nullptr, 1, H);
    go(W2, mW2, vW2, gW2, W2h.p, W2Th.p, H, H);
    go(b2, mb2, vb2, gb2, nullptr, nullptr, 1, H);
    go(w3, mw3, vw3, gw3, nullptr, nullptr, 1, H);
    go(b3, mb3, vb3, gb3, nullptr, nullptr, 1, 1);
    MLP_CK(cudaGetLastError());
  }

  void check_err() {
    uint32_t e = 0;
    MLP_CK(cudaMemcpyAsync(&e, err.p, sizeof e, cudaMemcpyDeviceToHost, st));
    MLP_CK(cudaStreamSynchronize(st));
    if (e) {
      MLP_CK(cudaMemsetAsync(err.p, 0, sizeof(uint32_t), st));
      throw MlpFail{GPUM_ERR_DEVICE, "a tensor-core kernel reported a device-side failure"};
    }
  }
};

namespace {

int mlp_guard(char* err, size_t len, const std::function<void()>& body) {
  try {
    body();
    if (err && len) err[0] = '\0';
    return GPUM_OK;
  } catch (const MlpFail& f) {
    if (err && len) std::snprintf(err, len, "%s", f.msg.c_str());
    return f.code;
  } catch (const std::bad_alloc&) {
    if (err && len) std::snprintf(err, len, "host allocation failed");
    return GPUM_ERR_NOMEM;
  } catch (...) {
    if (err && len) std::snprintf(err, len, "unexpected internal error");
    return GPUM_ERR_CUDA;
  }
}

void need(bool ok, const char* msg, int code = GPUM_ERR_INVALID) {
  if (!ok) throw MlpFail{code, msg};
}

}  // namespace

namespace {

// Upload host pairs (theta f64 -> f32, ll f64) into device buffers.
void upload_pairs(gpum_b200_mlp* m, const double* theta, const double* ll, size_t n,
                  Buf<float>& dth, Buf<double>& dll) {
  std::vector<float> th((size_t)n * m->d);
  for (size_t i = 0; i < th.size(); ++i) th[i] = (float)theta[i];
  dth.alloc(th.size());
  MLP_CK(cudaMemcpyAsync(dth.p, th.data(), th.size() * sizeof(float), cudaMemcpyHostToDevice,
                         m->st));
  if (ll) {
    dll.alloc(n);
    MLP_CK(cudaMemcpyAsync(dll.p, ll, n * sizeof(double), cudaMemcpyHostToDevice, m->st));
  }
  MLP_CK(cudaStreamSynchronize(m->st));
}

}  // namespace

namespace gpum {

// Kernel launches one mlp_infer call of n rows makes.
int mlp_infer_launches(const gpum_b200_mlp* m, int n) {
  return m->fused_inference() ? 1 : 5 * ((n + m->B - 1) / m->B);
}

// Surrogate log-likelihood of n f64 parameter vectors (device, chain-major)
// into out (device), enqueued on `st`.  Used by the delayed-acceptance loop.
int mlp_infer(gpum_b200_mlp* m, const double* theta, int n, int d, double* out, cudaStream_t st,
              std::string* err) {
  if (!m || d != m->d) {
    *err = "surrogate input width does not match the model's parameter count";
    return GPUM_ERR_INVALID;
  }
  cudaStream_t keep = m->st;
  m->st = st;
  int rc = GPUM_OK;
  try {
    if (m->fused_inference()) {
      const size_t smem = mlp_infer_smem(m->H);
      if (!m->infer_smem_set) {
        MLP_CK(cudaFuncSetAttribute(mlp_infer_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
        m->infer_smem_set = true;
      }
      if (n > 0) {
        mlp_infer_fused<<<(unsigned)((n + kInfRows - 1) / kInfRows), kInfThreads, smem, st>>>(
            theta, n, d, m->H, m->xmean.p, m->xinv.p, m->xw_or_null(), m->W1h.p, m->b1.p,
            m->W2h.p, m->b2.p, m->w3.p, m->b3.p, m->ysd, m->ymean, out, m->err.p);
        MLP_CK(cudaGetLastError());
      }
      m->st = keep;
      return GPUM_OK;
    }
    for (int r0 = 0; r0 < n; r0 += m->B) {
      const int rows = std::min(m->B, n - r0);
      const int Mi = (rows + kGemmBM - 1) / kGemmBM * kGemmBM;  // rows padded to the tile
      mlp_gather64<<<Mi, 128, 0, st>>>(theta + (size_t)r0 * d, rows, d, m->dp, Mi, m->xmean.p,
                                       m->xinv.p, m->xw_or_null(), m->Xh.p);
      m->forward(Mi);
      mlp_head<<<blocks((size_t)Mi * 32), 256, 0, st>>>(m->Z2.p, m->w3.p, m->b3.p, nullptr, Mi,
                                                       m->H, Mi, m->yhat.p, nullptr, nullptr,
                                                       nullptr, nullptr, 0);
      mlp_unscale<<<blocks(rows), 256, 0, st>>>(m->yhat.p, rows, m->ysd, m->ymean, out + r0);
      MLP_CK(cudaGetLastError());
    }
  } catch (const MlpFail& f) {
    *err = f.msg;
    rc = f.code;
  }
  m->st = keep;
  return rc;
}

}  // namespace gpum

extern "C" {

int gpum_b200_mlp_create(uint32_t d, uint32_t hidden, uint32_t batch, uint32_t seed,
                         gpum_b200_mlp** out, char* err, size_t err_len) {
  return mlp_guard(err, err_len, [&] {
    need(out != nullptr, "output pointer is NULL");
    *out = nullptr;
    need(d >= 1 && d <= 256, "input width must be in 1..256");
    need(hidden >= 128 && hidden <= 1024 && hidden % 128 == 0,
         "hidden width must be a multiple of 128 in 128..1024");
    need(batch >= 128 && batch <= 65536 && batch % 128 == 0,
         "batch must be a multiple of 128 in 128..65536");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
      cudaGetLastError();
      throw MlpFail{GPUM_ERR_NODEVICE, "no CUDA device is visible"};
    }
    std::unique_ptr<gpum_b200_mlp> m(new gpum_b200_mlp());
    m->d = (int)d;
    m->dp = (int)((d + 63) / 64 * 64);
    m->H = (int)hidden;
    m->B = (int)batch;
    m->seed = seed;
    MLP_CK(cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking));
    const int H = m->H, dp = m->dp, B = m->B;
    for (auto* b : {&m->W1, &m->mW1, &m->vW1, &m->gW1}) b->alloc((size_t)H * dp);
    for (auto* b : {&m->W2, &m->mW2, &m->vW2, &m->gW2}) b->alloc((size_t)H * H);
    for (auto* b : {&m->b1, &m->mb1, &m->vb1, &m->gb1, &m->b2, &m->mb2, &m->vb2, &m->gb2, &m->w3,
                    &m->mw3, &m->vw3, &m->gw3})
      b->alloc(H);
    for (auto* b : {&m->b3, &m->mb3, &m->vb3, &m->gb3}) b->alloc(1);
    m->W1h.alloc((size_t)H * dp);
    m->W2h.alloc((size_t)H * H);
    m->W2Th.alloc((size_t)H * H);
    m->Xh.alloc((size_t)B * dp);
    m->XTh.alloc((size_t)dp * B);
    for (auto* b : {&m->A1h, &m->A2h, &m->dZ2h}) b->alloc((size_t)B * H);
    for (auto* b : {&m->A1Th, &m->dZ2Th, &m->dZ1Th}) b->alloc((size_t)H * B);
    for (auto* b : {&m->Z1, &m->Z2, &m->dA1, &m->dZ1}) b->alloc((size_t)B * H);
    for (auto* b : {&m->t, &m->yhat, &m->rsq, &m->dyhat}) b->alloc(B);
    m->loss.alloc(1);
    m->colpart.alloc((size_t)((B + kColRows - 1) / kColRows) * H);
    m->splitk.alloc((size_t)32 * H * std::max(H, dp));
    m->xmean.alloc(d);
    m->xinv.alloc(d);
    m->xw.alloc((size_t)d * d);
    m->err.alloc(1);
    MLP_CK(cudaMemsetAsync(m->err.p, 0, sizeof(uint32_t), m->st));
    // zero moments and padded rows
    for (auto* b : {&m->mW1, &m->vW1, &m->mW2, &m->vW2, &m->mb1, &m->vb1, &m->mb2, &m->vb2,
                    &m->mw3, &m->vw3, &m->mb3, &m->vb3, &m->b1, &m->b2, &m->b3})
      MLP_CK(cudaMemsetAsync(b->p, 0, b->n * sizeof(float), m->st));
    mlp_init_weights<<<blocks((size_t)H * dp), 256, 0, m->st>>>(m->W1.p, (size_t)H * dp, (int)d,
                                                                (int)d, dp, seed, 1);
    mlp_init_weights<<<blocks((size_t)H * H), 256, 0, m->st>>>(m->W2.p, (size_t)H * H, H, H, H,
                                                               seed, 2);
    mlp_init_weights<<<blocks(H), 256, 0, m->st>>>(m->w3.p, H, H, H, H, seed, 3);
    mlp_to_bf16<<<blocks((size_t)H * dp), 256, 0, m->st>>>(m->W1.p, m->W1h.p, nullptr,
                                                           (size_t)H * dp, H, dp);
    mlp_to_bf16<<<blocks((size_t)H * H), 256, 0, m->st>>>(m->W2.p, m->W2h.p, m->W2Th.p,
                                                          (size_t)H * H, H, H);
    MLP_CK(cudaGetLastError());
    std::vector<float> ones(d, 1.0f);
    MLP_CK(cudaMemsetAsync(m->xmean.p, 0, d * sizeof(float), m->st));
    MLP_CK(cudaMemcpyAsync(m->xinv.p, ones.data(), d * sizeof(float), cudaMemcpyHostToDevice,
                           m->st));
    MLP_CK(cudaStreamSynchronize(m->st));
    *out = m.release();
  });
}

void gpum_b200_mlp_destroy(gpum_b200_mlp* m) {
  if (!m) return;
  if (m->st) cudaStreamSynchronize(m->st);
  delete m;
}

int gpum_b200_mlp_set_normalizer(gpum_b200_mlp* m, const double* xmean, const double* xsd,
                                 double ymean, double ysd, char* err, size_t err_len) {
  return mlp_guard(err, err_len, [&] {
    need(m && xmean && xsd, "NULL argument");
    need(std::isfinite(ymean) && ysd > 0 && std::isfinite(ysd), "ysd must be positive");
    std::vector<float> mu(m->d), inv(m->d);
    for (int j = 0; j < m->d; ++j) {
      need(xsd[j] > 0 && std::isfinite(xsd[j]) && std::isfinite(xmean[j]), "xsd must be positive");
      mu[j] = (float)xmean[j];
      inv[j] = (float)(1.0 / xsd[j]);
    }
    MLP_CK(cudaMemcpyAsync(m->xmean.p, mu.data(), m->d * sizeof(float), cudaMemcpyHostToDevice,
                           m->st));
    MLP_CK(cudaMemcpyAsync(m->xinv.p, inv.data(), m->d * sizeof(float), cudaMemcpyHostToDevice,
                           m->st));
    MLP_CK(cudaStreamSynchronize(m->st));
    m->whiten = false;
    m->ymean = (float)ymean;
    m->ysd = (float)ysd;
    m->yinv = (float)(1.0 / ysd);
  });
}

int gpum_b200_mlp_set_whitening(gpum_b200_mlp* m, const double* xmean, const double* xw,
                                double ymean, double ysd, char* err, size_t err_len) {
  return mlp_guard(err, err_len, [&] {
    need(m && xmean && xw, "NULL argument");
    need(std::isfinite(ymean) && ysd > 0 && std::isfinite(ysd), "ysd must be positive");
    const int d = m->d;
    std::vector<float> mu(d), w((size_t)d * d);
    for (int j = 0; j < d; ++j) {
      need(std::isfinite(xmean[j]), "xmean must be finite");
      mu[j] = (float)xmean[j];
    }
    for (size_t i = 0; i < (size_t)d * d; ++i) {
      need(std::isfinite(xw[i]), "the whitening matrix must be finite");
      w[i] = (float)xw[i];
    }
    MLP_CK(cudaMemcpyAsync(m->xmean.p, mu.data(), d * sizeof(float), cudaMemcpyHostToDevice,
                           m->st));
    MLP_CK(cudaMemcpyAsync(m->xw.p, w.data(), (size_t)d * d * sizeof(float),
                           cudaMemcpyHostToDevice, m->st));
    MLP_CK(cudaStreamSynchronize(m->st));
    m->whiten = true;
    m->ymean = (float)ymean;
    m->ysd = (float)ysd;
    m->yinv = (float)(1.0 / ysd);
  });
}

int gpum_b200_mlp_train(gpum_b200_mlp* m, const double* theta, const double* ll, size_t n_pairs,
                        uint32_t steps, double lr, float* out_loss, char* err, size_t err_len) {
  return mlp_guard(err, err_len, [&] {
    need(m && theta && ll, "NULL argument");
    need(n_pairs >= 1 && n_pairs <= (1u << 28), "n_pairs must be in 1..2^28");
    Buf<float> dth;
    Buf<double> dll;
    upload_pairs(m, theta, ll, n_pairs, dth, dll);
    std::vector<float> losses(steps);
    for (uint32_t s = 0; s < steps; ++s) {
      mlp_gather<<<m->B, 128, 0, m->st>>>(dth.p, dll.p, n_pairs, m->d, m->dp, m->B, 1, m->seed,
                                          m->step++, m->xmean.p, m->xinv.p, m->xw_or_null(),
                                          m->ymean, m->yinv,
                                          m->Xh.p, m->t.p);
      m->forward(m->B);
      m->backward(m->B);
      m->adam((float)lr);
      if (out_loss)
        MLP_CK(cudaMemcpyAsync(&losses[s], m->loss.p, sizeof(float), cudaMemcpyDeviceToHost,
                               m->st));
    }
    m->check_err();
    if (out_loss)
      for (uint32_t s = 0; s < steps; ++s) out_loss[s] = losses[s] / (float)m->B;
  });
}

int gpum_b200_mlp_predict(gpum_b200_mlp* m, const double* theta, size_t n, double* out, char* err,
                          size_t err_len) {
  return mlp_guard(err, err_len, [&] {
    need(m && theta && out, "NULL argument");
    need(n <= (1u << 24), "more than 2^24 points");
    if (n == 0) return;
    // The same device path as the delayed-acceptance loop (mlp_infer).
    Buf<double> dth, dout;
    dth.alloc(n * m->d);
    dout.alloc(n);
    MLP_CK(cudaMemcpyAsync(dth.p, theta, n * m->d * sizeof(double), cudaMemcpyHostToDevice,
                           m->st));
    std::string e;
    const int rc = gpum::mlp_infer(m, dth.p, (int)n, m->d, dout.p, m->st, &e);
    if (rc != GPUM_OK) throw MlpFail{rc, e};
    MLP_CK(cudaMemcpyAsync(out, dout.p, n * sizeof(double), cudaMemcpyDeviceToHost, m->st));
    MLP_CK(cudaStreamSynchronize(m->st));
    m->check_err();
  });
}

int gpum_b200_mlp_gradients(gpum_b200_mlp* m, const double* theta, const double* ll, size_t n,
                            float* out_grads, float* out_loss, char* err, size_t err_len) {
  return mlp_guard(err, err_len, [&] {
    need(m && theta && ll && out_grads, "NULL argument");
    need(n >= 1 && n <= (size_t)m->B, "n must be in 1..batch");
    Buf<float> dth;
    Buf<double> dll;
    upload_pairs(m, theta, ll, n, dth, dll);
    mlp_gather<<<m->B, 128, 0, m->st>>>(dth.p, dll.p, n, m->d, m->dp, m->B, 0, 0, 0, m->xmean.p,
                                        m->xinv.p, m->xw_or_null(), m->ymean, m->yinv, m->Xh.p,
                                        m->t.p);
    m->forward(m->B);
    m->backward((int)n);
    const int H = m->H, dp = m->dp;
    size_t off = 0;
    auto cp = [&](const float* src, size_t cnt) {
      MLP_CK(cudaMemcpyAsync(out_grads + off, src, cnt * sizeof(float), cudaMemcpyDeviceToHost,
                             m->st));
      off += cnt;
    };
    cp(m->gW1.p, (size_t)H * dp);
    cp(m->gb1.p, H);
    cp(m->gW2.p, (size_t)H * H);
    cp(m->gb2.p, H);
    cp(m->gw3.p, H);
    cp(m->gb3.p, 1);
    float l = 0.0f;
    MLP_CK(cudaMemcpyAsync(&l, m->loss.p, sizeof l, cudaMemcpyDeviceToHost, m->st));
    m->check_err();
    if (out_loss) *out_loss = l / (float)n;
  });
}

int gpum_b200_mlp_get_params(gpum_b200_mlp* m, float* out, char* err, size_t err_len) {
  return mlp_guard(err, err_len, [&] {
    need(m && out, "NULL argument");
    const int H = m->H, dp = m->dp;
    size_t off = 0;
    auto cp = [&](const float* src, size_t cnt) {
      MLP_CK(cudaMemcpyAsync(out + off, src, cnt * sizeof(float), cudaMemcpyDeviceToHost, m->st));
      off += cnt;
    };
    cp(m->W1.p, (size_t)H * dp);
    cp(m->b1.p, H);
    cp(m->W2.p, (size_t)H * H);
    cp(m->b2.p, H);
    cp(m->w3.p, H);
    cp(m->b3.p, 1);
    MLP_CK(cudaStreamSynchronize(m->st));
  });
}

int gpum_b200_mlp_gemm_check(uint32_t M, uint32_t N, uint32_t K, const float* A, const float* B,
                             float* C, char* err, size_t err_len) {
  return mlp_guard(err, err_len, [&] {
    need(A && B && C, "NULL argument");
    need(M % 128 == 0 && K % 64 == 0 && (N % 128 == 0 || N % 64 == 0) && M && N && K,
         "M, N, K must be multiples of 128, 64 and 64");
    std::vector<bf16> ah((size_t)M * K), bh((size_t)N * K);
    for (size_t i = 0; i < ah.size(); ++i) ah[i] = __float2bfloat16(A[i]);
    for (size_t i = 0; i < bh.size(); ++i) bh[i] = __float2bfloat16(B[i]);
    gpum_b200_mlp tmp;
    MLP_CK(cudaStreamCreateWithFlags(&tmp.st, cudaStreamNonBlocking));
    Buf<bf16> da, db;
    Buf<float> dc;
    da.alloc(ah.size());
    db.alloc(bh.size());
    dc.alloc((size_t)M * N);
    tmp.err.alloc(1);
    tmp.splitk.alloc(std::min<size_t>((size_t)32 * M * N, (size_t)1 << 26));
    MLP_CK(cudaMemsetAsync(tmp.err.p, 0, sizeof(uint32_t), tmp.st));
    MLP_CK(cudaMemcpyAsync(da.p, ah.data(), ah.size() * 2, cudaMemcpyHostToDevice, tmp.st));
    MLP_CK(cudaMemcpyAsync(db.p, bh.data(), bh.size() * 2, cudaMemcpyHostToDevice, tmp.st));
    tmp.gemm_any(da.p, db.p, dc.p, nullptr, nullptr, (int)M, (int)N, (int)K);
    MLP_CK(cudaMemcpyAsync(C, dc.p, (size_t)M * N * 4, cudaMemcpyDeviceToHost, tmp.st));
    tmp.check_err();
  });
}

}  // extern "C"
