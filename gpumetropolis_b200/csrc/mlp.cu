// mlp.cu -- the surrogate of the log-likelihood: a d-H-H-1 MLP with SiLU,
// trained and evaluated on the GPU with the tcgen05 GEMM (tc_gemm.cuh).
// No reference counterpart: the surrogate and delayed acceptance are new.
//
// Inputs are standardised (or whitened) parameters, the target is the
// standardised exact log-likelihood, the loss is the mean squared error.
// Weights live in f32 (master) with Adam moments, all in one flat vector
// [W1 | b1 | W2 | b2 | w3 | b3]; BF16 copies feed the tensor cores.  All
// reductions are fixed-order (no atomics on values), so training is bitwise
// repeatable for a given seed.
//
// One training step on a batch of B rows (B, H multiples of 128, H <= 512;
// the input width padded to dp, a multiple of 64) is seven kernels, captured
// once per train() call as a CUDA graph and replayed:
//   gather   X (bf16, row-major and transposed), targets t
//   GEMM1    Z1 = X W1^T + b1; A1 = silu(Z1) (row-major and transposed)
//   GEMM2    Z2 = A1 W2^T + b2 with the head fused into its epilogue (one
//            CTA holds whole rows): y = silu(Z2) w3 + b3, r = y - t, dy =
//            2r/B, dZ2 = dy w3 silu'(Z2) (both layouts); per-CTA column sums
//            for w3's and b2's gradients, row sums for b3's and the loss
//   GEMM3    dW2 = dZ2^T A1, split K into fixed partials
//   GEMM4    dZ1 = (dZ2 W2) * silu'(Z1) (transposed); per-CTA sums for b1's
//   GEMM5    dW1 = dZ1^T X, split K into fixed partials
//   adam     every gradient from its partials in a fixed order, then Adam
//            (Kingma & Ba, bias-corrected) and the BF16 copies; the last
//            block advances the device step counter the gather reads.
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
// Deterministic uniform index for (seed, step, row): Philox counter.
__device__ __forceinline__ uint32_t pick(uint32_t seed, uint32_t step, uint32_t row, uint32_t n) {
  const U4 r = philox4x32_10(U4{row, step, 0x4D4C5031u, 0u}, seed, 0x2545F491u);
  return (uint32_t)(((uint64_t)r.x * n) >> 32);
}

// Input transform of one row into out (bf16, zero padded to dp):
//   per coordinate  v_j = (theta_j - xmean_j) * xinv_j            (xw == nullptr)
//   whitening       v_j = sum_k xw[j][k] (theta_k - xmean_k)      (xw: d x d)
// and, when outT is set, the same values into column `row` of the
// transposed copy outT[j * ldT + row].  `cen` is block-shared scratch of d
// floats.  Called by every thread.
template <class Src>
__device__ __forceinline__ void mlp_input_row(Src theta_at, bool live, int d, int dp,
                                              const float* __restrict__ xmean,
                                              const float* __restrict__ xinv,
                                              const float* __restrict__ xw, float* cen,
                                              bf16* __restrict__ out, bf16* __restrict__ outT,
                                              int row, int ldT) {
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
    const bf16 h = __float2bfloat16(v);
    out[j] = h;
    if (outT) outT[(size_t)j * ldT + row] = h;
  }
}

// Batch rows: transformed inputs (bf16, padded with zeros; row-major and
// transposed) and standardised targets, one warp per row, kGatherRows rows
// per block.
// idx_mode 0: rows 0..n-1 in order (inference / gradient check);
//          1: Philox-random rows of the training set at step ctr[0].
constexpr int kGatherRows = 8;

__global__ void mlp_gather(const float* __restrict__ theta, const double* __restrict__ ll,
                           size_t n, int d, int dp, int B, int idx_mode, uint32_t seed,
                           const uint32_t* __restrict__ ctr, const float* __restrict__ xmean,
                           const float* __restrict__ xinv, const float* __restrict__ xw,
                           float ymean, float yinv, bf16* __restrict__ Xh,
                           bf16* __restrict__ XTh, float* __restrict__ t) {
  __shared__ float cen[kGatherRows][256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * kGatherRows + warp;
  if (row >= B) return;  // whole warps leave; no block-wide barrier follows
  size_t src = idx_mode ? pick(seed, ctr[0], (uint32_t)row, (uint32_t)n) : (size_t)row;
  const bool live = src < n;
  if (!live) src = 0;
  const float* th = theta + src * d;
  if (xw) {
    for (int k = lane; k < d; k += 32) cen[warp][k] = live ? th[k] - xmean[k] : 0.0f;
    __syncwarp();
  }
  for (int j = lane; j < dp; j += 32) {
    float v = 0.0f;
    if (live && j < d) {
      if (xw) {
        const float* wr = xw + (size_t)j * d;
        for (int k = 0; k < d; ++k) v = fmaf(wr[k], cen[warp][k], v);
      } else {
        v = (th[j] - xmean[j]) * xinv[j];
      }
    }
    const bf16 h = __float2bfloat16(v);
    Xh[(size_t)row * dp + j] = h;
    XTh[(size_t)j * B + row] = h;
  }
  if (lane == 0 && t) t[row] = live && ll ? (float)((ll[src] - ymean) * yinv) : 0.0f;
}

// Offsets of the flat parameter vector [W1 | b1 | W2 | b2 | w3 | b3].
struct MlpLayout {
  size_t oW1, ob1, oW2, ob2, ow3, ob3, n;
  int H, dp;
};

// Sources of one step's gradients: split-K partials of the two weight
// gradients, per-CTA column partials of the bias / head gradients, per-CTA
// row partials of b3's gradient and of the loss.
struct GradParts {
  const float* pW1;      // [S1][H][dp]
  int S1;
  const float* pW2;      // [S2][H][H]
  int S2;
  const float* colhead;  // [2][nct][H]: w3's, then b2's
  const float* colb1;    // [nct][H]
  const float* rowpart;  // [2][nct]: b3's, then sum r^2
  int nct;
};

// Every gradient from its partials (fixed order) into G; with `apply`, Adam
// (learning rate *lr_p, device memory, so a captured step serves every stage
// of a schedule) at step ctr[0] + 1 on the master weights and their BF16 copies (W1h, W2h
// and the transposed W1Th, W2Th), the loss of the step into
// loss_hist[ctr[0] - loss_base]; mlp_step_done then advances ctr[0].
__global__ void mlp_reduce_adam(MlpLayout L, GradParts Gp, float* __restrict__ P,
                                float* __restrict__ Mm, float* __restrict__ V,
                                float* __restrict__ G, bf16* __restrict__ W1h,
                                bf16* __restrict__ W1Th, bf16* __restrict__ W2h,
                                bf16* __restrict__ W2Th, const float* __restrict__ lr_p,
                                int apply, uint32_t* __restrict__ ctr, float* __restrict__ loss,
                                uint32_t loss_base, uint32_t loss_cap) {
  const uint32_t step = *reinterpret_cast<volatile const uint32_t*>(ctr);
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int H = L.H, dp = L.dp;
  if (i < L.n) {
    float g = 0.0f;
    if (i < L.ob1) {
      for (int z = 0; z < Gp.S1; ++z) g += Gp.pW1[(size_t)z * H * dp + i];
    } else if (i < L.oW2) {
      const size_t j = i - L.ob1;
      for (int c = 0; c < Gp.nct; ++c) g += Gp.colb1[(size_t)c * H + j];
    } else if (i < L.ob2) {
      const size_t k = i - L.oW2;
      for (int z = 0; z < Gp.S2; ++z) g += Gp.pW2[(size_t)z * H * H + k];
    } else if (i < L.ow3) {
      const size_t j = i - L.ob2;
      for (int c = 0; c < Gp.nct; ++c) g += Gp.colhead[((size_t)Gp.nct + c) * H + j];
    } else if (i < L.ob3) {
      const size_t j = i - L.ow3;
      for (int c = 0; c < Gp.nct; ++c) g += Gp.colhead[(size_t)c * H + j];
    } else {
      for (int c = 0; c < Gp.nct; ++c) g += Gp.rowpart[c];
    }
    G[i] = g;
    if (apply) {
      const float lr = *lr_p;
      const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
      const float t = (float)(step + 1);
      const float c1 = 1.0f - powf(b1, t), c2 = 1.0f - powf(b2, t);
      const float mi = b1 * Mm[i] + (1.0f - b1) * g;
      const float vi = b2 * V[i] + (1.0f - b2) * g * g;
      Mm[i] = mi;
      V[i] = vi;
      const float wi = P[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
      P[i] = wi;
      if (i < L.ob1) {
        W1h[i] = __float2bfloat16(wi);
        W1Th[(i % dp) * H + i / dp] = __float2bfloat16(wi);
      } else if (i >= L.oW2 && i < L.ob2) {
        const size_t k = i - L.oW2;
        W2h[k] = __float2bfloat16(wi);
        W2Th[(k % H) * H + k / H] = __float2bfloat16(wi);
      }
    }
  }
  if (i == 0 && loss) {
    float s = 0.0f;
    for (int c = 0; c < Gp.nct; ++c) s += Gp.rowpart[Gp.nct + c];
    const uint32_t slot = step - loss_base;
    if (slot < loss_cap) loss[slot] = s;
  }
}

// The step counter advances after the reduction (a kernel of its own: every
// block of the reduction has read the counter by then).
__global__ void mlp_step_done(uint32_t* __restrict__ ctr) {
  if (threadIdx.x == 0) ctr[0] += 1;
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
                Xh + (size_t)row * dp, nullptr, row, B);
}

__global__ void mlp_unscale(const float* __restrict__ y, int n, float ysd, float ymean,
                            double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (double)y[i] * ysd + ymean;
}

// Gradient of the surrogate log-likelihood with respect to the parameters,
// from dX = dy/dx (rows x dp, f32) of the network input x: through the input
// transform (whitening x = xw (theta - xmean), or per coordinate x_j =
// (theta_j - xmean_j) xinv_j) and the target's scale ysd.  One warp per row.
__global__ void mlp_input_grad(const float* __restrict__ dX, int n, int d, int dp,
                               const float* __restrict__ xinv, const float* __restrict__ xw,
                               float ysd, double* __restrict__ out) {
  const int row = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (row >= n) return;
  const float* g = dX + (size_t)row * dp;
  for (int j = lane; j < d; j += 32) {
    float v;
    if (xw) {
      v = 0.0f;
      for (int k = 0; k < d; ++k) v = fmaf(g[k], xw[(size_t)k * d + j], v);
    } else {
      v = g[j] * xinv[j];
    }
    out[(size_t)row * d + j] = (double)v * ysd;
  }
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
  uint32_t steps_done = 0;  // host mirror of the device step counter
  cudaStream_t st = nullptr;
  // second stream and events: the dW2 GEMM runs beside the dZ1 -> dW1 chain
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  MlpLayout L{};
  // parameters (f32 master), Adam moments, gradients: flat [W1|b1|W2|b2|w3|b3]
  Buf<float> P, Mm, V, G;
  Buf<bf16> W1h, W1Th, W2h, W2Th;
  // batch work buffers
  Buf<bf16> Xh, XTh, A1h, A1Th, dZ2h, dZ2Th, dZ1Th;
  Buf<float> Z1, t, yhat, dX;
  // gradient partials: split K (weights), per-CTA columns / rows (biases, head, loss)
  Buf<float> pW1, pW2, colhead, colb1, rowpart;
  int S1 = 1, S2 = 1;
  Buf<uint32_t> ctr;   // [step, unused]
  Buf<float> lr;       // [1] the current learning rate
  Buf<float> losses;   // per-step sums of squared residuals of one train() call
  // normaliser
  Buf<float> xmean, xinv, xw;  // xw: d x d whitening, used when `whiten`
  bool whiten = false;
  const float* xw_or_null() const { return whiten ? xw.p : nullptr; }
  float ymean = 0.0f, yinv = 1.0f, ysd = 1.0f;
  Buf<uint32_t> err;
  bool infer_smem_set = false;
  bool gemm_smem_set[16] = {};  // per (BN, epilogue) instantiation

  float* W1p() const { return P.p + L.oW1; }
  float* b1p() const { return P.p + L.ob1; }
  float* W2p() const { return P.p + L.oW2; }
  float* b2p() const { return P.p + L.ob2; }
  float* w3p() const { return P.p + L.ow3; }
  float* b3p() const { return P.p + L.ob3; }

  // The fused inference kernel covers d <= 64 and H in {128, 256}.
  bool fused_inference() const { return dp == 64 && (H == 128 || H == 256); }

  ~gpum_b200_mlp() {
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (st2) cudaStreamDestroy(st2);
    if (st) cudaStreamDestroy(st);
  }

  template <int BN, int EPI>
  void gemm(const GemmArgs& a, int S) {
    const size_t smem = tc_gemm_smem<BN>();
    // Set once per instantiation, so later launches (possibly under stream
    // capture) make no non-stream API calls.
    constexpr int slot = (BN == 64 ? 0 : BN == 128 ? 1 : BN == 256 ? 2 : 3) * 4 + EPI;
    if (!gemm_smem_set[slot]) {
      MLP_CK(cudaFuncSetAttribute(tc_gemm_kernel<BN, EPI>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      gemm_smem_set[slot] = true;
    }
    dim3 grid(a.N / BN, a.M / kGemmBM, S);
    tc_gemm_kernel<BN, EPI><<<grid, kGemmThreads, smem, st>>>(a);
    MLP_CK(cudaGetLastError());
  }

  GemmArgs args(const bf16* A, const bf16* Bm, int M, int N, int K) const {
    GemmArgs a{};
    a.A = A;
    a.B = Bm;
    a.M = M;
    a.N = N;
    a.K = K;
    a.kz = K;
    a.err = err.p;
    return a;
  }

  // Layer 1 (SiLU epilogue) and layer 2 with the head, for `rows` rows in Xh;
  // targets in t for the first n_live rows (nullptr: inference, r = 0).
  void forward(int rows, int n_live, const float* targets, int unit_dy = 0) {
    GemmArgs a1 = args(Xh.p, W1h.p, rows, H, dp);
    a1.C = Z1.p;
    a1.bias = b1p();
    a1.act = A1h.p;
    a1.actT = targets ? A1Th.p : nullptr;
    gemm<128, EPI_SILU>(a1, 1);
    GemmArgs a2 = args(A1h.p, W2h.p, rows, H, H);
    a2.bias = b2p();
    a2.w3 = w3p();
    a2.b3 = b3p();
    a2.t = targets;
    a2.n_live = n_live;
    a2.dzh = dZ2h.p;
    a2.colpart = targets ? colhead.p : nullptr;
    a2.rowpart = targets ? rowpart.p : nullptr;
    a2.actT = targets ? dZ2Th.p : nullptr;
    a2.unit_dy = unit_dy;
    a2.yhat = yhat.p;
    if (H == 128) gemm<128, EPI_HEAD>(a2, 1);
    else if (H == 256) gemm<256, EPI_HEAD>(a2, 1);
    else gemm<512, EPI_HEAD>(a2, 1);
  }

  // Weight gradients and b1's (after forward() with targets), then the
  // reduction of every gradient into G, with Adam when `apply`.
  void backward_and_update(int apply, float* loss_hist, uint32_t loss_base,
                           uint32_t loss_cap) {
    GemmArgs g3 = args(dZ2Th.p, A1Th.p, H, H, B);  // dW2 = dZ2^T A1
    g3.C = pW2.p;
    g3.kz = B / S2;
    // dW2 on the second stream, concurrent with dZ1 and dW1 (both only read
    // dZ2); the reduction waits for both.  Under stream capture the fork and
    // join become graph edges.
    const bool fork = st2 != nullptr;
    if (fork) {
      MLP_CK(cudaEventRecord(ev_fork, st));
      MLP_CK(cudaStreamWaitEvent(st2, ev_fork, 0));
      cudaStream_t keep = st;
      st = st2;
      try {
        gemm<64, EPI_STORE>(g3, S2);
      } catch (...) {
        st = keep;
        throw;
      }
      st = keep;
      MLP_CK(cudaEventRecord(ev_join, st2));
    } else {
      gemm<64, EPI_STORE>(g3, S2);
    }
    GemmArgs g4 = args(dZ2h.p, W2Th.p, B, H, H);   // dZ1 = (dZ2 W2) * silu'(Z1)
    g4.Zprev = Z1.p;
    g4.actT = dZ1Th.p;
    g4.colpart = colb1.p;
    gemm<128, EPI_DSILU>(g4, 1);
    GemmArgs g5 = args(dZ1Th.p, XTh.p, H, dp, B);  // dW1 = dZ1^T X
    g5.C = pW1.p;
    g5.kz = B / S1;
    gemm<64, EPI_STORE>(g5, S1);
    if (fork) MLP_CK(cudaStreamWaitEvent(st, ev_join, 0));
    GradParts gp{pW1.p, S1, pW2.p, S2, colhead.p, colb1.p, rowpart.p, B / kGemmBM};
    mlp_reduce_adam<<<blocks(L.n), 256, 0, st>>>(L, gp, P.p, Mm.p, V.p, G.p, W1h.p, W1Th.p,
                                                  W2h.p, W2Th.p, lr.p, apply, ctr.p, loss_hist,
                                                  loss_base, loss_cap);
    if (apply) mlp_step_done<<<1, 32, 0, st>>>(ctr.p);
    MLP_CK(cudaGetLastError());
  }

  // Value and parameter gradient of the surrogate log-likelihood for `rows`
  // rows in Xh (after the gather): layer 1, layer 2 with the head at dy = 1,
  // then back through both layers to the input (dZ1 row-major in A1Th's
  // space, dX = dZ1 W1), and through the input transform.
  void value_grad(int rows, int n, int d_in, double* out_val, double* out_grad) {
    forward(rows, rows, nullptr, /*unit_dy=*/1);
    mlp_unscale<<<blocks(n), 256, 0, st>>>(yhat.p, n, ysd, ymean, out_val);
    GemmArgs g4 = args(dZ2h.p, W2Th.p, rows, H, H);  // dZ1 = (dZ2 W2) * silu'(Z1)
    g4.Zprev = Z1.p;
    g4.act = A1Th.p;
    gemm<128, EPI_DSILU>(g4, 1);
    GemmArgs g5 = args(A1Th.p, W1Th.p, rows, dp, H);  // dX = dZ1 W1
    g5.C = dX.p;
    gemm<64, EPI_STORE>(g5, 1);
    mlp_input_grad<<<blocks((size_t)n * 32), 256, 0, st>>>(dX.p, n, d_in, dp, xinv.p,
                                                           xw_or_null(), ysd, out_grad);
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

// Split-K factor of a B-deep weight-gradient GEMM with `tiles` output tiles:
// the largest power of two up to `cap` that keeps at least one 64-wide K
// slice per CTA and at most about two waves of CTAs (each split is one
// partial of the weight's size that the reduction reads back).
int split_k(int B, int tiles, int sms, int cap) {
  int S = 1;
  while (S < cap && (B / (2 * S)) % kGemmBK == 0 && B / (2 * S) >= kGemmBK &&
         tiles * 2 * S <= 2 * sms)
    S *= 2;
  return S;
}

}  // namespace

namespace gpum {

// Kernel launches one mlp_infer call of n rows makes.
int mlp_infer_launches(const gpum_b200_mlp* m, int n) {
  return m->fused_inference() ? 1 : 4 * ((n + m->B - 1) / m->B);
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
            theta, n, d, m->H, m->xmean.p, m->xinv.p, m->xw_or_null(), m->W1h.p, m->b1p(),
            m->W2h.p, m->b2p(), m->w3p(), m->b3p(), m->ysd, m->ymean, out, m->err.p);
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
      m->forward(Mi, Mi, nullptr);
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

// Surrogate log-likelihood and its gradient with respect to the parameters
// at n f64 parameter vectors (device, chain-major), into out_val[n] and
// out_grad[n][d] (device), enqueued on `st`: the drift of the
// delayed-acceptance Langevin proposal.
int mlp_infer_grad(gpum_b200_mlp* m, const double* theta, int n, int d, double* out_val,
                   double* out_grad, cudaStream_t st, std::string* err) {
  if (!m || d != m->d) {
    *err = "surrogate input width does not match the model's parameter count";
    return GPUM_ERR_INVALID;
  }
  cudaStream_t keep = m->st;
  m->st = st;
  int rc = GPUM_OK;
  try {
    for (int r0 = 0; r0 < n; r0 += m->B) {
      const int rows = std::min(m->B, n - r0);
      const int Mi = (rows + kGemmBM - 1) / kGemmBM * kGemmBM;
      mlp_gather64<<<Mi, 128, 0, st>>>(theta + (size_t)r0 * d, rows, d, m->dp, Mi, m->xmean.p,
                                       m->xinv.p, m->xw_or_null(), m->Xh.p);
      MLP_CK(cudaGetLastError());
      m->value_grad(Mi, rows, d, out_val + r0, out_grad + (size_t)r0 * d);
    }
  } catch (const MlpFail& f) {
    *err = f.msg;
    rc = f.code;
  }
  m->st = keep;
  return rc;
}

// Kernel launches one mlp_infer_grad call of n rows makes.
int mlp_infer_grad_launches(const gpum_b200_mlp* m, int n) {
  return 7 * ((n + m->B - 1) / m->B);
}

}  // namespace gpum

extern "C" {

int gpum_b200_mlp_create(uint32_t d, uint32_t hidden, uint32_t batch, uint32_t seed,
                         gpum_b200_mlp** out, char* err, size_t err_len) {
  return mlp_guard(err, err_len, [&] {
    need(out != nullptr, "output pointer is NULL");
    *out = nullptr;
    need(d >= 1 && d <= 256, "input width must be in 1..256");
    need(hidden == 128 || hidden == 256 || hidden == 512, "hidden width must be 128, 256 or 512");
    need(batch >= 128 && batch <= 65536 && batch % 128 == 0,
         "batch must be a multiple of 128 in 128..65536");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
      cudaGetLastError();
      throw MlpFail{GPUM_ERR_NODEVICE, "no CUDA device is visible"};
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    std::unique_ptr<gpum_b200_mlp> m(new gpum_b200_mlp());
    m->d = (int)d;
    m->dp = (int)((d + 63) / 64 * 64);
    m->H = (int)hidden;
    m->B = (int)batch;
    m->seed = seed;
    MLP_CK(cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking));
    MLP_CK(cudaStreamCreateWithFlags(&m->st2, cudaStreamNonBlocking));
    MLP_CK(cudaEventCreateWithFlags(&m->ev_fork, cudaEventDisableTiming));
    MLP_CK(cudaEventCreateWithFlags(&m->ev_join, cudaEventDisableTiming));
    const int H = m->H, dp = m->dp, B = m->B;
    MlpLayout& L = m->L;
    L.H = H;
    L.dp = dp;
    L.oW1 = 0;
    L.ob1 = L.oW1 + (size_t)H * dp;
    L.oW2 = L.ob1 + H;
    L.ob2 = L.oW2 + (size_t)H * H;
    L.ow3 = L.ob2 + H;
    L.ob3 = L.ow3 + H;
    L.n = L.ob3 + 1;
    for (auto* b : {&m->P, &m->Mm, &m->V, &m->G}) b->alloc(L.n);
    m->W1h.alloc((size_t)H * dp);
    m->W1Th.alloc((size_t)dp * H);
    m->W2h.alloc((size_t)H * H);
    m->W2Th.alloc((size_t)H * H);
    m->Xh.alloc((size_t)B * dp);
    m->XTh.alloc((size_t)dp * B);
    for (auto* b : {&m->A1h, &m->dZ2h}) b->alloc((size_t)B * H);
    for (auto* b : {&m->A1Th, &m->dZ2Th, &m->dZ1Th}) b->alloc((size_t)H * B);
    m->Z1.alloc((size_t)B * H);
    m->t.alloc(B);
    m->yhat.alloc(B);
    m->dX.alloc((size_t)B * dp);
    m->S2 = split_k(B, (H / 128) * (H / 64), sms, 16);
    m->S1 = split_k(B, (H / 128) * (dp / 64), sms, 64);
    m->pW2.alloc((size_t)m->S2 * H * H);
    m->pW1.alloc((size_t)m->S1 * H * dp);
    const int nct = B / kGemmBM;
    m->colhead.alloc((size_t)2 * nct * H);
    m->colb1.alloc((size_t)nct * H);
    m->rowpart.alloc((size_t)2 * nct);
    m->ctr.alloc(2);
    m->lr.alloc(1);
    m->xmean.alloc(d);
    m->xinv.alloc(d);
    m->xw.alloc((size_t)d * d);
    m->err.alloc(1);
    MLP_CK(cudaMemsetAsync(m->err.p, 0, sizeof(uint32_t), m->st));
    MLP_CK(cudaMemsetAsync(m->ctr.p, 0, 2 * sizeof(uint32_t), m->st));
    // zero moments, biases and the (padded) batch buffers
    for (auto* b : {&m->P, &m->Mm, &m->V, &m->G})
      MLP_CK(cudaMemsetAsync(b->p, 0, b->n * sizeof(float), m->st));
    mlp_init_weights<<<blocks((size_t)H * dp), 256, 0, m->st>>>(m->W1p(), (size_t)H * dp, (int)d,
                                                                (int)d, dp, seed, 1);
    mlp_init_weights<<<blocks((size_t)H * H), 256, 0, m->st>>>(m->W2p(), (size_t)H * H, H, H, H,
                                                               seed, 2);
    mlp_init_weights<<<blocks(H), 256, 0, m->st>>>(m->w3p(), H, H, H, H, seed, 3);
    mlp_to_bf16<<<blocks((size_t)H * dp), 256, 0, m->st>>>(m->W1p(), m->W1h.p, m->W1Th.p,
                                                           (size_t)H * dp, H, dp);
    mlp_to_bf16<<<blocks((size_t)H * H), 256, 0, m->st>>>(m->W2p(), m->W2h.p, m->W2Th.p,
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

}  // extern "C"

namespace {

// Checks a learning-rate schedule; returns its total step count.
uint64_t schedule_steps(uint32_t n_stages, const uint32_t* steps, const double* lrs) {
  need(n_stages == 0 || (steps && lrs), "NULL argument");
  uint64_t total = 0;
  for (uint32_t k = 0; k < n_stages; ++k) {
    need(std::isfinite(lrs[k]) && lrs[k] >= 0.0, "learning rates must be finite and >= 0");
    total += steps[k];
  }
  need(total <= (1u << 24), "more than 2^24 steps");
  return total;
}

// Adam on n_pairs device-resident pairs (theta f32 [n][d], ll f64 [n]) with
// a learning-rate schedule of `total` steps; out_loss (may be NULL) receives
// every step's mean squared error.
void train_on_device(gpum_b200_mlp* m, const float* dth, const double* dll, size_t n_pairs,
                     uint32_t n_stages, const uint32_t* steps, const double* lrs, uint64_t total,
                     float* out_loss) {
  m->losses.alloc(total);
  const uint32_t base = m->steps_done;
  // One step: its kernels read the step from the device counter the
  // reduction advances and the learning rate from device memory, so one
  // captured CUDA graph serves all steps of all stages.
  auto one_step = [&] {
    mlp_gather<<<m->B / kGatherRows, 32 * kGatherRows, 0, m->st>>>(
        dth, dll, n_pairs, m->d, m->dp, m->B, 1, m->seed, m->ctr.p, m->xmean.p,
        m->xinv.p, m->xw_or_null(), m->ymean, m->yinv, m->Xh.p, m->XTh.p, m->t.p);
    MLP_CK(cudaGetLastError());
    m->forward(m->B, m->B, m->t.p);
    m->backward_and_update(1, m->losses.p, base, (uint32_t)total);
  };
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool first = true;
  cudaError_t le = cudaSuccess;
  for (uint32_t k = 0; k < n_stages && le == cudaSuccess; ++k) {
    if (steps[k] == 0) continue;
    const float lr_f = (float)lrs[k];
    MLP_CK(cudaMemcpyAsync(m->lr.p, &lr_f, sizeof lr_f, cudaMemcpyHostToDevice, m->st));
    MLP_CK(cudaStreamSynchronize(m->st));  // lr_f is a stack value
    uint32_t left = steps[k];
    if (first) {
      one_step();  // eagerly: sets every kernel attribute outside capture
      first = false;
      --left;
    }
    if (left > 0 && !exec) {
      MLP_CK(cudaStreamBeginCapture(m->st, cudaStreamCaptureModeThreadLocal));
      try {
        one_step();
      } catch (...) {
        cudaGraph_t g2 = nullptr;
        cudaStreamEndCapture(m->st, &g2);
        if (g2) cudaGraphDestroy(g2);
        throw;
      }
      MLP_CK(cudaStreamEndCapture(m->st, &graph));
      const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
      if (ie != cudaSuccess) {
        cudaGraphDestroy(graph);
        MLP_CK(ie);
      }
    }
    for (; left > 0 && le == cudaSuccess; --left) le = cudaGraphLaunch(exec, m->st);
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  MLP_CK(le);
  m->steps_done += (uint32_t)total;
  std::vector<float> losses(total);
  MLP_CK(cudaMemcpyAsync(losses.data(), m->losses.p, total * sizeof(float),
                         cudaMemcpyDeviceToHost, m->st));
  m->check_err();
  if (out_loss)
    for (uint64_t s = 0; s < total; ++s) out_loss[s] = losses[s] / (float)m->B;
}

}  // namespace

namespace gpum {
int mlp_input_width(const gpum_b200_mlp* m) { return m ? m->d : 0; }

// Training from pairs already on the device (the session's recorded pairs).
int mlp_train_device(gpum_b200_mlp* m, const float* dth, const double* dll, size_t n_pairs,
                     uint32_t n_stages, const uint32_t* steps, const double* lrs,
                     float* out_loss, std::string* err) {
  char buf[512];
  const int rc = mlp_guard(buf, sizeof buf, [&] {
    need(m && dth && dll, "NULL argument");
    need(n_pairs >= 1 && n_pairs <= (1u << 28), "n_pairs must be in 1..2^28");
    const uint64_t total = schedule_steps(n_stages, steps, lrs);
    if (total > 0) train_on_device(m, dth, dll, n_pairs, n_stages, steps, lrs, total, out_loss);
  });
  if (rc != GPUM_OK && err) *err = buf;
  return rc;
}
}  // namespace gpum

extern "C" {

int gpum_b200_mlp_train_stages(gpum_b200_mlp* m, const double* theta, const double* ll,
                               size_t n_pairs, uint32_t n_stages, const uint32_t* steps,
                               const double* lrs, float* out_loss, char* err, size_t err_len) {
  return mlp_guard(err, err_len, [&] {
    need(m && theta && ll, "NULL argument");
    need(n_pairs >= 1 && n_pairs <= (1u << 28), "n_pairs must be in 1..2^28");
    const uint64_t total = schedule_steps(n_stages, steps, lrs);
    if (total == 0) return;
    // The pairs are uploaded once for every stage.
    Buf<float> dth;
    Buf<double> dll;
    upload_pairs(m, theta, ll, n_pairs, dth, dll);
    train_on_device(m, dth.p, dll.p, n_pairs, n_stages, steps, lrs, total, out_loss);
  });
}

int gpum_b200_mlp_train(gpum_b200_mlp* m, const double* theta, const double* ll, size_t n_pairs,
                        uint32_t steps, double lr, float* out_loss, char* err, size_t err_len) {
  return gpum_b200_mlp_train_stages(m, theta, ll, n_pairs, 1, &steps, &lr, out_loss, err,
                                    err_len);
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

int gpum_b200_mlp_predict_grad(gpum_b200_mlp* m, const double* theta, size_t n, double* out,
                               double* out_grad, char* err, size_t err_len) {
  return mlp_guard(err, err_len, [&] {
    need(m && theta && out && out_grad, "NULL argument");
    need(n <= (1u << 24), "more than 2^24 points");
    if (n == 0) return;
    // The same device path as the delayed-acceptance Langevin loop.
    Buf<double> dth, dout, dgrad;
    dth.alloc(n * m->d);
    dout.alloc(n);
    dgrad.alloc(n * m->d);
    MLP_CK(cudaMemcpyAsync(dth.p, theta, n * m->d * sizeof(double), cudaMemcpyHostToDevice,
                           m->st));
    std::string e;
    const int rc = gpum::mlp_infer_grad(m, dth.p, (int)n, m->d, dout.p, dgrad.p, m->st, &e);
    if (rc != GPUM_OK) throw MlpFail{rc, e};
    MLP_CK(cudaMemcpyAsync(out, dout.p, n * sizeof(double), cudaMemcpyDeviceToHost, m->st));
    MLP_CK(cudaMemcpyAsync(out_grad, dgrad.p, n * m->d * sizeof(double), cudaMemcpyDeviceToHost,
                           m->st));
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
    Buf<float> loss1;
    loss1.alloc(1);
    mlp_gather<<<m->B / kGatherRows, 32 * kGatherRows, 0, m->st>>>(
        dth.p, dll.p, n, m->d, m->dp, m->B, 0, 0, m->ctr.p,
                                        m->xmean.p, m->xinv.p, m->xw_or_null(), m->ymean,
                                        m->yinv, m->Xh.p, m->XTh.p, m->t.p);
    MLP_CK(cudaGetLastError());
    m->forward(m->B, (int)n, m->t.p);
    // loss slot: the device step counter is not advanced without `apply`
    uint32_t step = 0;
    MLP_CK(cudaMemcpyAsync(&step, m->ctr.p, sizeof step, cudaMemcpyDeviceToHost, m->st));
    MLP_CK(cudaStreamSynchronize(m->st));
    m->backward_and_update(0, loss1.p, step, 1);
    MLP_CK(cudaMemcpyAsync(out_grads, m->G.p, m->L.n * sizeof(float), cudaMemcpyDeviceToHost,
                           m->st));
    float l = 0.0f;
    MLP_CK(cudaMemcpyAsync(&l, loss1.p, sizeof l, cudaMemcpyDeviceToHost, m->st));
    m->check_err();
    if (out_loss) *out_loss = l / (float)n;
  });
}

int gpum_b200_mlp_get_params(gpum_b200_mlp* m, float* out, char* err, size_t err_len) {
  return mlp_guard(err, err_len, [&] {
    need(m && out, "NULL argument");
    MLP_CK(cudaMemcpyAsync(out, m->P.p, m->L.n * sizeof(float), cudaMemcpyDeviceToHost, m->st));
    MLP_CK(cudaStreamSynchronize(m->st));
  });
}

int gpum_b200_mlp_gemm_check(uint32_t M, uint32_t N, uint32_t K, const float* A, const float* B,
                             float* C, char* err, size_t err_len) {
  return mlp_guard(err, err_len, [&] {
    need(A && B && C, "NULL argument");
    need(M % 128 == 0 && K % 64 == 0 && N % 64 == 0 && M && N && K,
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
    MLP_CK(cudaMemsetAsync(tmp.err.p, 0, sizeof(uint32_t), tmp.st));
    MLP_CK(cudaMemcpyAsync(da.p, ah.data(), ah.size() * 2, cudaMemcpyHostToDevice, tmp.st));
    MLP_CK(cudaMemcpyAsync(db.p, bh.data(), bh.size() * 2, cudaMemcpyHostToDevice, tmp.st));
    GemmArgs a = tmp.args(da.p, db.p, (int)M, (int)N, (int)K);
    a.C = dc.p;
    if (N % 512 == 0) tmp.gemm<512, EPI_STORE>(a, 1);
    else if (N % 256 == 0) tmp.gemm<256, EPI_STORE>(a, 1);
    else if (N % 128 == 0) tmp.gemm<128, EPI_STORE>(a, 1);
    else tmp.gemm<64, EPI_STORE>(a, 1);
    MLP_CK(cudaMemcpyAsync(C, dc.p, (size_t)M * N * 4, cudaMemcpyDeviceToHost, tmp.st));
    tmp.check_err();
  });
}

}  // extern "C"
