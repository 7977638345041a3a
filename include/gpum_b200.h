/*
 * gpum_b200.h -- C ABI of the B200 (sm_100a) backend for gpumetropolis.
 *
 * Plain pointers and sizes only; no function throws, aborts or exits.  Every
 * compute entry point returns GPUM_OK (0) or a GPUM_ERR_* code and, when `err`
 * is non-NULL, writes a NUL-terminated message of at most err_len bytes.
 *
 * Layouts follow the reference's FFI (src/rust/src/lib.rs):
 *   code        u32 (opcode, arg) pairs, length n_code (even)   R/dsl.R:13-17
 *   consts      f64 constant pool
 *   data        f64 row-major n_obs x n_cols                     R/api.R:281-294
 *   init, proposal_sd   f64 chain-major n_chains x n_params      R/api.R:297-346
 *   proposal_l  f64 n_chains x n_params x n_params, row-major lower factors,
 *               or NULL / n_l == 0                               chain_kernel.rs:224-249
 *   out_draws   f32 n_iter*n_chains*n_params, column-major (n_iter, n_chains,
 *               n_params): draws[t + n_iter*(c + n_chains*j)]     chain_kernel.rs:345
 *   points      f64 point-major n_points x n_params              lib.rs:131-207
 *
 * Arithmetic: the per-observation bytecode runs in FP32 on the GPU with
 * compensated FP32 partial sums; totals, the prior, proposals and the
 * acceptance ratio are FP64.
 */
#ifndef GPUM_B200_H
#define GPUM_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GPUM_API __attribute__((visibility("default")))
#else
#define GPUM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define GPUM_OK 0
#define GPUM_ERR_INVALID 1      /* bad argument or malformed bytecode          */
#define GPUM_ERR_CUDA 2         /* CUDA runtime / driver failure               */
#define GPUM_ERR_NOMEM 3        /* device or host allocation failed            */
#define GPUM_ERR_UNSUPPORTED 4  /* valid input beyond this backend's limits    */
#define GPUM_ERR_NODEVICE 5     /* no sm_100 GPU visible                       */
#define GPUM_ERR_DEVICE 6       /* a kernel reported a device-side failure     */

/* proposal_mode values (lib.rs:85; chain_kernel.rs:212-295; cpu_native.rs:573-784) */
#define GPUM_MODE_RWM 0         /* diagonal Gaussian random walk               */
#define GPUM_MODE_DE 1          /* differential evolution on the init snapshot */
#define GPUM_MODE_CHOL 2        /* random walk with per-chain Cholesky factor  */
#define GPUM_MODE_MALA 3        /* Metropolis-adjusted Langevin                */
#define GPUM_MODE_DE_SYNC 4     /* per-generation DE, path B (sessions only;   *
                                 * cpu_native.rs:400-506)                      */

/* evaluation engines (gpum_b200_session_set_engine) */
#define GPUM_ENGINE_INTERP 0    /* register-stack bytecode interpreter          */
#define GPUM_ENGINE_COMPILED 1  /* bytecode -> CUDA C -> NVRTC (sm_100a)        */
#define GPUM_ENGINE_AUTO 2      /* compiled when NVRTC builds it, else interp.  */

/* rng values for the session API */
#define GPUM_RNG_TRIPLE32 0     /* the reference's counter hash stream         */
#define GPUM_RNG_PHILOX 1       /* Philox4x32-10 counter-based stream          */

/* 1 if an sm_100 device is visible and the kernels load, else 0.
 * Replaces rust_available_backends()'s feature probe (lib.rs:51-61). */
GPUM_API int gpum_b200_available(void);

/* Library version string, e.g. "gpum_b200 0.1.0 sm_100a". */
GPUM_API const char* gpum_b200_version(void);

/* Check a program without touching the GPU: opcode/argument ranges, stack
 * discipline, depth <= 32 (R/dsl.R:115-119).  allow_data = 0 for a prior.
 * Writes the peak stack depth to *depth (may be NULL). */
GPUM_API int gpum_b200_validate_program(const uint32_t* code, size_t n_code, size_t n_consts,
                               uint32_t n_params, uint32_t n_cols, int allow_data,
                               int* depth, char* err, size_t err_len);

/* Whole sampler, one call per batch, inputs and outputs in host memory.
 * Replaces rust_gpu_metropolis -> gpu_metropolis_chain (lib.rs:69-123,
 * chain_kernel.rs:469-532).  Uses the reference's triple32 stream, so with
 * the same seed the b200 chains follow the CPU backend's chains up to FP32
 * evaluation differences in the data sum. */
GPUM_API int gpum_b200_run(const uint32_t* code, size_t n_code, const double* consts, size_t n_consts,
                  const uint32_t* prior_code, size_t n_prior, const double* prior_consts,
                  size_t n_prior_consts, uint32_t n_params, const double* data, uint32_t n_cols,
                  uint64_t n_obs, const double* init, const double* proposal_sd,
                  const double* temperatures, uint32_t n_chains, uint32_t n_iter, uint32_t seed,
                  uint32_t proposal_mode, double gamma, double de_noise,
                  const double* proposal_l, size_t n_l, float* out_draws, float* out_accept,
                  double* out_last_logpost, char* err, size_t err_len);

/* Summed log-likelihood at each point, out[n_points] f64
 * (rust_loglik_batch, lib.rs:131-151). */
GPUM_API int gpum_b200_loglik_batch(const uint32_t* code, size_t n_code, const double* consts,
                           size_t n_consts, uint32_t n_params, const double* data,
                           uint32_t n_cols, uint64_t n_obs, const double* points,
                           size_t n_points, double* out, char* err, size_t err_len);

/* Gradient of the summed log-likelihood (data term) at each point,
 * point-major out[p*n_params + j] f64, by the compiled engine's reverse-mode
 * adjoint, or, on the interpreter engine (chosen, or when NVRTC cannot build
 * the model), by a reverse sweep over a per-observation tape of the
 * interpreted program (at most 128 parameters and 512 operations)
 * (rust_grad_batch, lib.rs:158-179; cpu_native.rs:306-329). */
GPUM_API int gpum_b200_grad_batch(const uint32_t* code, size_t n_code, const double* consts,
                         size_t n_consts, uint32_t n_params, const double* data,
                         uint32_t n_cols, uint64_t n_obs, const double* points,
                         size_t n_points, double* out, char* err, size_t err_len);

/* Build the compiled engine's kernels for a model with NVRTC without touching
 * a GPU; *cubin_bytes (may be NULL) receives the module size.  No reference
 * counterpart: the reference's JIT (jit.rs) is CPU-only. */
GPUM_API int gpum_b200_compile_check(const uint32_t* code, size_t n_code, const double* consts,
                            size_t n_consts, const uint32_t* prior_code, size_t n_prior,
                            const double* prior_consts, size_t n_prior_consts,
                            uint32_t n_params, uint32_t n_cols, size_t* cubin_bytes,
                            char* err, size_t err_len);

/* Per-observation log-likelihood, out[p*n_obs + i] f64
 * (rust_loglik_pointwise, lib.rs:187-207). */
GPUM_API int gpum_b200_loglik_pointwise(const uint32_t* code, size_t n_code, const double* consts,
                               size_t n_consts, uint32_t n_params, const double* data,
                               uint32_t n_cols, uint64_t n_obs, const double* points,
                               size_t n_points, double* out, char* err, size_t err_len);

/* Summed log-likelihood at each point for callers that cannot allocate
 * device memory (their memory is owned by another allocator or budget).  No
 * counterpart in the reference.  Allocates nothing: inputs and outputs are
 * the caller's DEVICE buffers -- data column-major f32 d_data[j*ld + i]
 * (ld >= n_obs, ld % 4 == 0, 16-byte aligned), points f64 n_points x
 * n_params, out f64 n_points -- and the scratch is a fixed 16 MiB
 * __device__ array per GPU, held until process exit from the moment the
 * library's device code is loaded on that GPU (at the first call that uses
 * it under CUDA's default lazy loading, at library load with
 * CUDA_MODULE_LOADING=EAGER; a GPU without 16 MiB free fails that first
 * call with GPUM_ERR_NOMEM); inputs needing more (n_params x points beyond
 * it) are rejected with GPUM_ERR_UNSUPPORTED.  With n_cols == 0 (a
 * per-observation term that reads no data) d_data may be NULL.  Work is enqueued on `stream` (a cudaStream_t, NULL
 * for the legacy stream) and the call waits for it.  Calls share the scratch:
 * calls that overlap on the GPU race.  The first call on a device sets up
 * the scratch address; make it before any stream capture.  The program is
 * interpreted one micro-op per instruction (at most 1024 instructions). */
GPUM_API int gpum_b200_loglik_batch_noalloc(const uint32_t* code, size_t n_code,
                                            const double* consts, size_t n_consts,
                                            uint32_t n_params, const float* d_data, uint64_t ld,
                                            uint32_t n_cols, uint64_t n_obs,
                                            const double* d_points, size_t n_points,
                                            double* d_out, void* stream, char* err,
                                            size_t err_len);

/* Synchronous per-generation differential evolution (path B): every
 * proposal of generation t reads the population after generation t-1;
 * untempered; proposal_sd is the jitter base; needs n_chains >= 3.  Same
 * arguments and outputs as rust_gpu_metropolis_de_sync (lib.rs:215-259,
 * cpu_native.rs:400-506), in this header's layouts, with the reference's
 * triple32 stream. */
GPUM_API int gpum_b200_run_de_sync(const uint32_t* code, size_t n_code, const double* consts,
                                   size_t n_consts, uint32_t n_params, const double* data,
                                   uint32_t n_cols, uint64_t n_obs, const uint32_t* prior_code,
                                   size_t n_prior, const double* prior_consts,
                                   size_t n_prior_consts, const double* init,
                                   const double* proposal_sd, uint32_t n_chains,
                                   uint32_t n_iter, uint32_t seed, double gamma,
                                   double de_noise, float* out_draws, float* out_accept,
                                   double* out_last_logpost, char* err, size_t err_len);

/* ------------------------------------------------------------- sessions --
 * A session keeps the model and the data resident on the GPU, so batches of a
 * host-orchestrated run (adaptive warmup, PT, DE snapshots) do not re-upload
 * the data each call as the reference does (chain_kernel.rs:391-413). */
typedef struct gpum_b200_session gpum_b200_session;

GPUM_API int gpum_b200_session_create(const uint32_t* code, size_t n_code, const double* consts,
                             size_t n_consts, const uint32_t* prior_code, size_t n_prior,
                             const double* prior_consts, size_t n_prior_consts,
                             uint32_t n_params, const double* data, uint32_t n_cols,
                             uint64_t n_obs, gpum_b200_session** out, char* err,
                             size_t err_len);

/* Same contract as gpum_b200_run on a session; rng selects the stream. */
GPUM_API int gpum_b200_session_run(gpum_b200_session* s, const double* init, const double* proposal_sd,
                          const double* temperatures, uint32_t n_chains, uint32_t n_iter,
                          uint32_t seed, uint32_t proposal_mode, double gamma, double de_noise,
                          const double* proposal_l, size_t n_l, int rng, float* out_draws,
                          float* out_accept, double* out_last_logpost, char* err,
                          size_t err_len);

/* gpum_b200_run_de_sync on a session; rng selects the stream. */
GPUM_API int gpum_b200_session_run_de_sync(gpum_b200_session* s, const double* init,
                                           const double* proposal_sd, uint32_t n_chains,
                                           uint32_t n_iter, uint32_t seed, double gamma,
                                           double de_noise, int rng, float* out_draws,
                                           float* out_accept, double* out_last_logpost,
                                           char* err, size_t err_len);

/* Select the evaluation engine (GPUM_ENGINE_*); the default is AUTO.
 * Gradients (MALA, grad_batch) use the engine too: the compiled engine's
 * generated adjoint, or the interpreter's tape (up to 128 parameters and 512
 * operations; AUTO falls back to it when NVRTC cannot build the model). */
GPUM_API int gpum_b200_session_set_engine(gpum_b200_session* s, int engine, char* err,
                                          size_t err_len);
/* The engine plain evaluations use (GPUM_ENGINE_INTERP or _COMPILED). */
GPUM_API int gpum_b200_session_engine(gpum_b200_session* s);
/* 1 when the session's log-likelihood sums and value-only sampler steps
 * (rwm, pt, de, cholesky; delayed acceptance's exact stage) run the
 * compiled engine's tensor-core value kernel: the model's linear predictor
 * (the largest per-observation subexpression that is affine in the data
 * with parameter-only coefficients, at least 6 data columns) as a TF32
 * tensor-core product with a three-term split, the rest of each term on the
 * FP32 pipes.  0 otherwise: no such predictor, a non-finite value in one of
 * its data columns, no device memory for its packed copy of those columns
 * (8 bytes per column per observation), the interpreter engine, or
 * GPUM_B200_TENSOR_CORES=0 in the environment at the session's first
 * compiled evaluation.  Pointwise
 * output and gradients keep the FP32 kernels.  No counterpart in the
 * reference (src/rust/src/chain_kernel.rs:305-321 evaluates the bytecode
 * per chain and observation). */
GPUM_API int gpum_b200_session_tensor_cores(gpum_b200_session* s);

/* loglik_batch / loglik_pointwise / grad_batch on a session. */
GPUM_API int gpum_b200_session_loglik_batch(gpum_b200_session* s, const double* points, size_t n_points,
                                   double* out, char* err, size_t err_len);
GPUM_API int gpum_b200_session_loglik_pointwise(gpum_b200_session* s, const double* points,
                                       size_t n_points, double* out, char* err,
                                       size_t err_len);
GPUM_API int gpum_b200_session_grad_batch(gpum_b200_session* s, const double* points,
                                          size_t n_points, double* out, char* err,
                                          size_t err_len);

/* Device-resident stepping, for callers that keep chain state on the GPU
 * between calls: prepare() uploads the batch-start state and evaluates it,
 * advance() runs n more iterations entirely on the device (CUDA graph),
 * fetch() copies results out.  Draw storage is reserved for max_iter
 * iterations at prepare(). */
GPUM_API int gpum_b200_session_prepare(gpum_b200_session* s, const double* init,
                              const double* proposal_sd, const double* temperatures,
                              uint32_t n_chains, uint32_t max_iter, uint32_t seed,
                              uint32_t proposal_mode, double gamma, double de_noise,
                              const double* proposal_l, size_t n_l, int rng, char* err,
                              size_t err_len);
GPUM_API int gpum_b200_session_advance(gpum_b200_session* s, uint32_t n_iter, char* err, size_t err_len);
GPUM_API int gpum_b200_session_sync(gpum_b200_session* s, char* err, size_t err_len);
/* Copies draws of the iterations advanced so far (n_done <= max_iter) in the
 * reference layout with n_iter = n_done, accept rates over n_done, last
 * log posteriors.  Any output pointer may be NULL. */
GPUM_API int gpum_b200_session_fetch(gpum_b200_session* s, float* out_draws, float* out_accept,
                            double* out_last_logpost, uint32_t* n_done, char* err,
                            size_t err_len);

/* Replica exchange on the device for later runs: chains form ladders of
 * ladder_len consecutive chains (their temperatures along the ladder, n_chains
 * a multiple of ladder_len); after every swap_every-th iteration the adjacent
 * pairs of one parity (alternating, even pairs first) exchange states with
 * the reference's probability min(1, exp((lp[i+1] - lp[i]) (1/T[i] -
 * 1/T[i+1]))) (R/adaptive.R:362-387, there between host batches); exchanged
 * chains draw fresh proposals.  Philox uniforms.  ladder_len 0 turns it off. */
GPUM_API int gpum_b200_session_set_exchange(gpum_b200_session* s, uint32_t ladder_len,
                                            uint32_t swap_every, char* err, size_t err_len);
/* Per pair (c, c+1) the attempted and accepted exchanges of the last run
 * (prepared, run or run_da; n_chains entries each; entries that are no pair
 * stay 0) and the number of exchange steps.  In a delayed-acceptance run the
 * exchanges use the exact log posteriors, and the surrogate value and prior
 * cached for each state move with it.  Any output pointer may be NULL. */
GPUM_API int gpum_b200_session_exchange_stats(gpum_b200_session* s, uint32_t* attempts,
                                              uint32_t* accepted, uint32_t* n_exchanges,
                                              char* err, size_t err_len);

/* Moments of the draws of iterations [t0, t0 + n) of the prepared run, for
 * adaptive warmup without copying the draws (R/adaptive.R:101-254 only uses
 * these): per chain the mean and the sum of squared deviations of each
 * parameter (chain-major n_chains x n_params), the pooled mean (n_params) and
 * the pooled sums of cross deviations (n_params x n_params) over the
 * n x n_chains draws; f64, fixed summation order.  No reference counterpart
 * (the reference returns every draw to R). */
GPUM_API int gpum_b200_session_draw_moments(gpum_b200_session* s, uint32_t t0, uint32_t n,
                                            double* chain_mean, double* chain_m2,
                                            double* pool_mean, double* pool_m2, char* err,
                                            size_t err_len);
/* The current chain states (n_chains x n_params, f64). */
GPUM_API int gpum_b200_session_state(gpum_b200_session* s, double* out_state, char* err,
                                     size_t err_len);

/* The device-failure path, exercised without a fault: a one-warp kernel on
 * the session's stream waits on an mbarrier that nothing arrives on, gives
 * up after `polls` polls (1..2^20) or 50 ms, sets the session's device error
 * word and returns; the call then reports GPUM_ERR_DEVICE exactly as a run
 * whose bounded TMA or tensor-core wait ran out does, clears the word, and
 * the session stays usable.  No counterpart in the reference (its kernels
 * have no bounded waits); for tests of failure detection. */
GPUM_API int gpum_b200_session_selftest_wait(gpum_b200_session* s, uint32_t polls, char* err,
                                             size_t err_len);

/* The session's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events with the session's launches. */
GPUM_API void* gpum_b200_session_stream(const gpum_b200_session* s);

/* Kernel launches issued by this session so far (every node of a replayed
 * graph counts once per replay). */
GPUM_API uint64_t gpum_b200_session_launches(const gpum_b200_session* s);

GPUM_API void gpum_b200_session_destroy(gpum_b200_session* s);

/* ------------------------------------------------------- surrogate MLP --
 * A d-H-H-1 SiLU network approximating the log-likelihood over the
 * parameters, trained and evaluated on the GPU with BF16 tcgen05 tensor-core
 * GEMMs (f32 accumulation in tensor memory), f32 master weights and Adam.
 * No counterpart in the reference: it is the first stage of delayed
 * acceptance.  hidden is 128, 256 or 512; batch a multiple of 128; d <= 256.
 * A training step is seven kernels (input gather, two forward GEMMs with
 * the head fused into the second one's epilogue, three gradient GEMMs, one
 * fixed-order gradient reduction with Adam), replayed as a CUDA graph. */
typedef struct gpum_b200_mlp gpum_b200_mlp;

GPUM_API int gpum_b200_mlp_create(uint32_t d, uint32_t hidden, uint32_t batch, uint32_t seed,
                                  gpum_b200_mlp** out, char* err, size_t err_len);
GPUM_API void gpum_b200_mlp_destroy(gpum_b200_mlp* m);
/* Standardisation of inputs (per coordinate) and of the target. */
GPUM_API int gpum_b200_mlp_set_normalizer(gpum_b200_mlp* m, const double* xmean,
                                          const double* xsd, double ymean, double ysd, char* err,
                                          size_t err_len);
/* Whitening instead of per-coordinate scaling: the network sees
 * xw (theta - xmean), xw a d x d row-major matrix (e.g. the inverse Cholesky
 * factor of the training parameters' covariance). */
GPUM_API int gpum_b200_mlp_set_whitening(gpum_b200_mlp* m, const double* xmean, const double* xw,
                                         double ymean, double ysd, char* err, size_t err_len);
/* `steps` Adam steps on random batches of the pairs (host arrays theta
 * n_pairs x d, ll n_pairs); out_loss (may be NULL) receives each step's mean
 * squared error in standardised units. */
GPUM_API int gpum_b200_mlp_train(gpum_b200_mlp* m, const double* theta, const double* ll,
                                 size_t n_pairs, uint32_t steps, double lr, float* out_loss,
                                 char* err, size_t err_len);
/* A learning-rate schedule in one call: steps[k] Adam steps at lrs[k] for
 * k < n_stages, the pairs uploaded once; out_loss (may be NULL) receives
 * sum(steps) losses. */
GPUM_API int gpum_b200_mlp_train_stages(gpum_b200_mlp* m, const double* theta, const double* ll,
                                        size_t n_pairs, uint32_t n_stages,
                                        const uint32_t* steps, const double* lrs,
                                        float* out_loss, char* err, size_t err_len);
/* Predicted log-likelihood at n points (host arrays). */
GPUM_API int gpum_b200_mlp_predict(gpum_b200_mlp* m, const double* theta, size_t n, double* out,
                                   char* err, size_t err_len);
/* Predicted log-likelihood and its gradient with respect to the parameters
 * (out_grad n x d, row-major) at n points (host arrays): the drift of the
 * Langevin proposal in session_run_da, through the same device path. */
GPUM_API int gpum_b200_mlp_predict_grad(gpum_b200_mlp* m, const double* theta, size_t n,
                                        double* out, double* out_grad, char* err,
                                        size_t err_len);
/* Gradients of the batch loss at the first n <= batch pairs, without an
 * update: out = [dW1 (H x dp) | db1 (H) | dW2 (H x H) | db2 (H) | dw3 (H) |
 * db3 (1)], dp = d rounded up to 64; *out_loss = mean squared error. */
GPUM_API int gpum_b200_mlp_gradients(gpum_b200_mlp* m, const double* theta, const double* ll,
                                     size_t n, float* out_grads, float* out_loss, char* err,
                                     size_t err_len);
/* Master weights in the same order as the gradients. */
GPUM_API int gpum_b200_mlp_get_params(gpum_b200_mlp* m, float* out, char* err, size_t err_len);
/* C[M x N] = bf16(A)[M x K] . bf16(B)[N x K]^T through the tcgen05 GEMM
 * (host f32 arrays; M % 128 == 0, K % 64 == 0, N % 64 == 0). */
GPUM_API int gpum_b200_mlp_gemm_check(uint32_t M, uint32_t N, uint32_t K, const float* A,
                                      const float* B, float* C, char* err, size_t err_len);

/* Power posteriors for thermodynamic integration: later runs on this session
 * target beta[c] * log-likelihood + log-prior for chain c (the prior is not
 * tempered; the acceptance temperature still applies).  The reference builds
 * one "power model" per rung (R/bayes.R:266-277) and runs the rungs one after
 * another; here all rungs run as chains of one batch.  NULL / 0 clears; runs
 * must then have exactly n_chains chains.  Not available with run_da. */
GPUM_API int gpum_b200_session_set_likelihood_powers(gpum_b200_session* s, const double* beta,
                                                     size_t n_chains, char* err,
                                                     size_t err_len);

/* ------------------------------------------------- delayed acceptance --
 * No counterpart in the reference.  Training pairs come from exact runs:
 * with recording on, every proposal an exact step (session_run / advance)
 * evaluates is stored as (theta as f32, data-term log-likelihood), up to
 * `capacity` pairs; capacity 0 turns recording off and frees the store.
 * Calling record() again restarts the store. */
GPUM_API int gpum_b200_session_record(gpum_b200_session* s, uint64_t capacity, char* err,
                                      size_t err_len);
/* Copies the first min(recorded, max_pairs) pairs (theta row-major
 * n x n_params, ll n); *n_pairs = pairs recorded so far. */
GPUM_API int gpum_b200_session_recorded(gpum_b200_session* s, float* out_theta, double* out_ll,
                                        uint64_t max_pairs, uint64_t* n_pairs, char* err,
                                        size_t err_len);
/* Fits the surrogate to the pairs this session recorded without copying them
 * to the host.  Pair i is held out when holdout_every > 0 and i %
 * holdout_every == 0 (holdout_every = 1 is refused); pairs with a non-finite
 * value are dropped.  The normaliser comes from the training pairs' f64
 * moments: with `whiten` (and n_params > 1) inputs are whitened by the
 * inverse Cholesky factor of their covariance (ddof 1, diagonal jitter
 * 1e-10 x its mean), else standardised per coordinate; the target is
 * standardised (ddof 0).  Then Adam with the learning-rate schedule of
 * mlp_train_stages.  out_loss (may be NULL) receives sum(steps) losses;
 * out_info (may be NULL) receives 5 values: pairs recorded, training pairs,
 * held-out pairs, the held-out residual standard deviation of the trained
 * network (NaN without held-out pairs), 1 if the inputs were whitened. */
GPUM_API int gpum_b200_session_train_surrogate(gpum_b200_session* s, gpum_b200_mlp* m,
                                               uint32_t holdout_every, int whiten,
                                               uint32_t n_stages, const uint32_t* steps,
                                               const double* lrs, float* out_loss,
                                               double* out_info, char* err, size_t err_len);
/* Two-stage Metropolis-Hastings (Christen & Fox): the surrogate screens each
 * proposal (stage 1) and only survivors are evaluated exactly (stage 2), so
 * the chains target the exact tempered posterior.  Same arguments and
 * outputs as session_run for proposal modes 0, 1 and 2; mode 3 is a
 * Langevin proposal whose drift is the surrogate log-posterior gradient
 * (the surrogate's input gradient plus the f64 prior's), preconditioned and
 * capped as MALA (cpu_native.rs:617-651), with q(x|y)/q(y|x) in stage 1 --
 * no exact gradient is evaluated, so it runs on either engine.  out_exact
 * (may be NULL) receives per chain the number of exact evaluations (stage-1
 * acceptances).  The surrogate must have d = n_params.  Device exchanges
 * (session_set_exchange) run as in session_run. */
GPUM_API int gpum_b200_session_run_da(gpum_b200_session* s, gpum_b200_mlp* surrogate,
                                      const double* init, const double* proposal_sd,
                                      const double* temperatures, uint32_t n_chains,
                                      uint32_t n_iter, uint32_t seed, uint32_t proposal_mode,
                                      double gamma, double de_noise, const double* proposal_l,
                                      size_t n_l, int rng, float* out_draws, float* out_accept,
                                      double* out_last_logpost, uint32_t* out_exact, char* err,
                                      size_t err_len);

#ifdef __cplusplus
}
#endif
#endif /* GPUM_B200_H */
