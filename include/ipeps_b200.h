/*
 * libipeps_b200 — C ABI of the B200 CTMRG engine (drop-in for the CTMRG hot
 * path of iPEPS.jl).
 *
 * The reference has no FFI: its hot path sits behind the Julia functions
 * listed beside each entry point (paths relative to the iPEPS.jl source
 * tree).  A Julia binding calls these through `ccall`; the Python binding in
 * ipeps.jl_b200/host.py calls them through ctypes.
 *
 * Conventions
 *  - Every function returns an int status (IPEPS_OK, or one of the codes
 *    below); the message of the last failure is ipeps_last_error(ctx).
 *  - Host arrays are column-major (Julia layout).  Real data is double;
 *    complex data is interleaved (re, im) double pairs (ComplexF64).
 *  - Hamiltonian bond matrices (d^2 x d^2) are always passed as complex.
 *  - The library owns all device memory behind opaque handles.  Each context
 *    owns one CUDA stream; calls are synchronous on return; a handle is not
 *    thread-safe (use one context per host thread).
 */
#ifndef IPEPS_B200_H
#define IPEPS_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define IPEPS_API __attribute__((visibility("default")))
#else
#define IPEPS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define IPEPS_OK 0
#define IPEPS_ENOTCONV 1   /* an iteration cap was hit (CTMRG or Jacobi) */
#define IPEPS_ENONFINITE 2 /* NaN/Inf detected in a result */
#define IPEPS_EOOM 3       /* device allocation failed */
#define IPEPS_EINVAL 4     /* bad argument / shape */
#define IPEPS_ECUDA 5      /* other CUDA error */

#define IPEPS_PREC_FP64 0  /* every contraction in FP64 */
#define IPEPS_PREC_MIXED 1 /* contractions as 3xTF32 on tcgen05, FP64 SVD/normalisation/energy */

#define IPEPS_CONV_ENERGY 0   /* run_ctm with conv_fun = get_gs_energy (ctmrg.jl:21-28) */
#define IPEPS_CONV_SPECTRUM 1 /* run_ctm without conv_fun: left-move spectrum (ctmrg.jl:29-31) */
#define IPEPS_CONV_ES 2       /* conv_fun = get_es_energy / get_all_norm (optim_es.jl:175) */

typedef struct ipeps_ctx ipeps_ctx;
typedef struct ipeps_env ipeps_env;
typedef struct ipeps_mlp ipeps_mlp;

typedef struct {
  uint64_t launches[8]; /* per kernel family: permute, gemm_f64, gemm_tf32x3, reduce, elementwise, small_linalg, jacobi */
  double flops[8];
  double bytes[8];
  uint64_t moves;       /* directional moves done by all envs of this context */
  double move_seconds;  /* host wall time inside moves (synchronous) */
  uint64_t projector_calls; /* truncated-SVD projectors computed */
  uint64_t jacobi_sweeps;   /* one-sided Jacobi sweeps summed over those projectors */
  uint64_t extra_passes;    /* extra power iterations triggered by the residual check */
  uint64_t series_cap_hits; /* projector adjoints whose Chebyshev expansion of the broadened
                               resolvent hit its 160-term cap before its 1e-11 tolerance
                               (gradient possibly inexact) */
  uint64_t series_terms;    /* Chebyshev terms summed over all projector adjoints */
  uint64_t series_retries;  /* expansions redone over a wider interval because the resolvent
                               check ((x^2 + eta) f(x) = x on the result) failed */
  uint64_t resid_misses;    /* projectors whose kept triplets stayed above the residual tolerance
                               (the extra power iterations stopped converging or ran out) */
} ipeps_stats_t;

/* ---- context (no reference counterpart: the reference is one CPU process) */
IPEPS_API int ipeps_ctx_create(int device, ipeps_ctx** out);
IPEPS_API int ipeps_ctx_destroy(ipeps_ctx* ctx);
IPEPS_API const char* ipeps_last_error(ipeps_ctx* ctx);
IPEPS_API int ipeps_ctx_set_precision(ipeps_ctx* ctx, int precision);
IPEPS_API int ipeps_ctx_set_seed(ipeps_ctx* ctx, uint64_t seed);
IPEPS_API int ipeps_stats(ipeps_ctx* ctx, ipeps_stats_t* out);
IPEPS_API int ipeps_stats_reset(ipeps_ctx* ctx);
/* the context's CUDA stream (cudaStream_t), for callers that time or order work on it */
IPEPS_API int ipeps_ctx_stream(ipeps_ctx* ctx, void** stream);
/* per-kernel-family CUDA-event timing: enable, then query ms / launches /
 * credited flops / bytes per family since enabling (query clears the window) */
IPEPS_API int ipeps_prof_enable(ipeps_ctx* ctx, int on);
IPEPS_API int ipeps_prof_query(ipeps_ctx* ctx, double* ms, uint64_t* launches, double* flops, double* bytes);
/* While profiling is enabled: wall ms of the E+grad pullback's phases since the last call
 * (ms[5]: checkpoint iterations, energy tape, recorded recomputation of the iterations, their
 * backward, the projector adjoints inside that backward), then cleared. */
IPEPS_API int ipeps_prof_phases(ipeps_ctx* ctx, double* ms);

/* ---- contraction operator: tcon(ind_xs, ind_y, A, B) (src/utility/wrapper.jl:15-23).
 * la/lb: labels per leg (positive = summed, negative -1..-n = output order).
 * out receives the result (capacity out_cap elements), out_dims/out_nd its shape.
 * is_complex applies to A, B and out. */
IPEPS_API int ipeps_tcon(ipeps_ctx* ctx, int is_complex, const double* A, int nA, const int64_t* dimsA, const int* la,
               const double* B, int nB, const int64_t* dimsB, const int* lb, double* out, int64_t out_cap,
               int64_t* out_dims, int* out_nd);
/* ---- projector: get_projector(R1, R2, chi) (ctmrg.jl:254-265) for real R1 (N1 x K1) and
 * R2 (K1 x N2), column-major.  P1 (K1 x n) and P2 (n x K1) need capacity K1*(chi+1); s capacity
 * chi+1; *n = kept count (at most min(chi, K1) + 1, by the degenerate-pair rule of cutoff_matrix). */
IPEPS_API int ipeps_projector(ipeps_ctx* ctx, const double* R1, const double* R2, int64_t N1, int64_t K1, int64_t N2,
                    int chi, double* P1, double* P2, double* s, int* n);
/* The same for ComplexF64 R1, R2 (interleaved re, im): P1 = R2 V S^-1/2, P2 = S^-1/2 U' R1
 * with U' the conjugate transpose (ctmrg.jl:262-263); P1, P2 complex, s real. */
IPEPS_API int ipeps_projector_c(ipeps_ctx* ctx, const double* R1, const double* R2, int64_t N1, int64_t K1,
                      int64_t N2, int chi, double* P1, double* P2, double* s, int* n);

/* ---- orthonormal basis of range(Y) for Y (N x k, column-major, real, N >= k): the
 * projector's range-finder step (it stands in for the Q factor of the reference's full SVD,
 * ctmrg.jl:257).  passes CholeskyQR passes, the first one shifted (passes = 3: sCholQR3):
 * Q (N x k) with Q^T Q = I, and, when R is not NULL, R (k x k upper triangular, column-major)
 * with Q R = Y. */
IPEPS_API int ipeps_orth(ipeps_ctx* ctx, const double* Y, int64_t N, int k, int passes, double* Q, double* R);

/* ---- environment state: CTMTensors (src/ctm/ctm_tensor.jl:3-18, ctors :57-69) */
IPEPS_API int ipeps_env_create(ipeps_ctx* ctx, int D, int d, int chi, int is_complex, ipeps_env** out);
IPEPS_API int ipeps_env_destroy(ipeps_env* env);
/* Params Dict keys chi/min_iter/max_iter/ad_max_iter/rg_tol (default_config.toml:9-17) */
IPEPS_API int ipeps_env_set_params(ipeps_env* env, int chi, int min_iter, int max_iter, int ad_max_iter, double rg_tol);
/* rg_step runs the left and right moves concurrently, then the top and bottom
 * moves (each pair reads and writes disjoint slots, ctmrg.jl:122-252), on two
 * streams from two host threads; on = 0 runs the four moves one after another
 * on one stream (same results up to the projectors' random sketches).
 * Default on.  No counterpart in the reference (sequential moves). */
IPEPS_API int ipeps_env_set_parallel(ipeps_env* env, int on);
/* projector sketch: k = n+1 + max(min_over, (n+1)*num/den); power iterations cold/warm;
 * a posteriori check ||M v_i - s_i u_i|| <= resid_tol * s_1 with up to max_extra
 * further power iterations; inter_passes CholeskyQR passes for intermediate sketches;
 * seed_older: seed from the vectors of two calls back (period-2 cycles) */
IPEPS_API int ipeps_env_set_svd_params(ipeps_env* env, int over_num, int over_den, int min_over, int power_iters,
                                       int power_iters_warm, int warm_start, double resid_tol, int max_extra,
                                       int inter_passes, int seed_older);
/* mixed form (IPEPS_PREC_MIXED contexts only): run_ctm switches to FP64 for the
 * last polish_iters iterations, or once the change per iteration drops below
 * polish_tol * rg_tol (default 100: close to the requested convergence; with
 * rg_tol = 0 only the last iterations), and accepts convergence only after
 * polish_iters FP64 iterations
 * (0 = stay in the mixed form).  No counterpart in the reference (FP64 only). */
IPEPS_API int ipeps_env_set_mixed(ipeps_env* env, int polish_iters, double polish_tol);
/* A (D,D,D,D,d); Ad = NULL means conj(A) (CTMTensors(A, cfg), ctm_tensor.jl:63) */
IPEPS_API int ipeps_env_set_A(ipeps_env* env, const double* A, const double* Ad);
/* init_ctm1 (ctm_tensor.jl:97-130) */
IPEPS_API int ipeps_env_init(ipeps_env* env);
/* C_k (chi_a x chi_b) and E_k (chi_a, chi_b, D, D), k = 1..4 (ts.Cs[k], ts.Es[k]).
 * Pass NULL data pointers to query the dims only. */
IPEPS_API int ipeps_env_get_CT(ipeps_env* env, int k, double* C, int64_t* C_dims, double* E, int64_t* E_dims);
IPEPS_API int ipeps_env_set_CT(ipeps_env* env, int k, const double* C, const int64_t* C_dims, const double* E,
                     const int64_t* E_dims);

/* ---- moves: left_rg/right_rg/top_rg/bottom_rg (ctmrg.jl:66-120), dir 0..3.
 * s_out (capacity *s_len on entry) receives the kept singular values of the
 * projector; *s_len is set to their count. */
IPEPS_API int ipeps_ctm_move(ipeps_env* env, int dir, double* s_out, int* s_len);
/* rg_step (ctmrg.jl:57-64): left, right, top, bottom; s of the left move */
IPEPS_API int ipeps_ctm_step(ipeps_env* env, double* s_out, int* s_len);
/* run_ctm (ctmrg.jl:1-55).  Hh/Hv complex d2 x d2 (needed for the energy
 * and es modes).  Returns IPEPS_OK also when not converged (the reference only
 * prints "Not Converged"); *converged reports it. */
IPEPS_API int ipeps_ctm_run(ipeps_env* env, int conv_mode, const double* Hh, const double* Hv, int d2, int* iters,
                  double* last_diff, int* converged);
/* per-iteration log of the last run: 4 doubles per iteration (diff, obj_re, obj_im, chi) */
IPEPS_API int ipeps_ctm_log(ipeps_env* env, double* out, int* n_iters);

/* ---- observables (src/graph/evaluation.jl) */
/* get_gs_energy (evaluation.jl:15-29): E and Na complex (re, im) */
IPEPS_API int ipeps_energy(ipeps_env* env, const double* Hh, const double* Hv, int d2, double* E, double* Na);
/* get_gs_norm (evaluation.jl:47-59) */
IPEPS_API int ipeps_gs_norm(ipeps_env* env, double* nrm);
/* ndm_Ad of get_tangent_basis (optim_es.jl:247-251): get_single_dm contracted
 * with Ad, shape (D,D,D,D,d), dtype of A */
IPEPS_API int ipeps_single_dm_Ad(ipeps_env* env, double* out);

/* ---- energy + gradient: the pullback of run_gs (optim_gs.jl:133-143) as
 * used by fg! (optim_gs.jl:53-91).  Starting from the environment currently
 * held (normally converged by ipeps_ctm_run), runs ad_iters CTMRG iterations
 * with A as the variable, then get_gs_energy; returns real(E) and dE/dA
 * (D,D,D,D,d, real A only; A and Ad = conj(A) both contribute).  The
 * environment is advanced by those iterations.  C/T are checkpointed per
 * iteration and the moves recomputed in the backward pass. */
IPEPS_API int ipeps_energy_grad(ipeps_env* env, const double* Hh, const double* Hv, int d2, int ad_iters, double* E,
                                double* dA);

/* ---- nested-tensor (excited-state) move, optim_es (src/optimize/optim_es.jl:167-210) */
/* setproperties(ts, B=B, Bd=conj(B)) + Params px, py (in radians); B complex (D,D,D,D,d).
 * Clears the B/Bd/BB environment slots (EmptyT). */
IPEPS_API int ipeps_nested_set_B(ipeps_env* env, const double* B, double px, double py);
/* get_es_energy (evaluation.jl:31-45) */
IPEPS_API int ipeps_es_energy(ipeps_env* env, const double* Hh, const double* Hv, int d2, double* E);
/* get_all_norm (evaluation.jl:61-77): Nb (complex) and envB (complex, size of A) */
IPEPS_API int ipeps_all_norm(ipeps_env* env, double* Nb, double* envB);
/* pullback of run_es (optim_es.jl:184-188) from the nested environment held by
 * env: runs ad_iters nested iterations, returns E = get_es_energy and
 * gH = dE/dB (complex (D,D,D,D,d), convention dE/dRe B + i dE/dIm B).
 * The environment is advanced by those iterations (get_all_norm afterwards
 * gives gN = envB as in get_es_grad, optim_es.jl:189). */
IPEPS_API int ipeps_es_energy_grad(ipeps_env* env, const double* Hh, const double* Hv, int d2, int ad_iters,
                                   double* E, double* gB);

/* ---- plaquette (4x4 cluster) observables of the h4 drivers (src/graph/evaluation.jl:339-398,
 * 443-518; src/optimize/optim_gs_h4.jl, optim_es_h4.jl).  The plaquette Hamiltonian is the
 * MPO [s1, s2, s3, s4] of get_local_h (src/model/local_h.jl:1-31): s1 (d,d,a), s2 (a,d,d,b),
 * s3 (b,d,d,c), s4 (c,d,d), each a complex128 column-major array. */
typedef struct {
  const double* data; /* interleaved (re, im) */
  int nd;
  int64_t dims[4];
} ipeps_ctensor_t;
/* nested = 0: get_gs_energy_4x4 (evaluation.jl:339-356); nested = 1: get_es_energy_4x4
 * (evaluation.jl:358-398, needs B).  E receives the complex value (2 doubles). */
IPEPS_API int ipeps_energy_4x4(ipeps_env* env, const ipeps_ctensor_t* H4, int nested, double* E);
/* run_ctm with conv_fun = get_gs_energy_4x4 (nested = 0) or get_es_energy_4x4 / get_all_norm
 * (nested = 1) (optim_es_h4.jl:33,139); as ipeps_ctm_run otherwise. */
IPEPS_API int ipeps_ctm_run_4x4(ipeps_env* env, const ipeps_ctensor_t* H4, int nested, int* iters,
                                double* last_diff, int* converged);
/* Pullback of run_gs_h4 w.r.t. A (the fg! of optim_gs_h4, optim_gs_h4.jl:53-91,113-123):
 * ad_iters CTMRG iterations from the current environment with the plaquette energy as
 * convergence value, E = real(get_gs_energy_4x4), dA real (D,D,D,D,d); real A only. */
IPEPS_API int ipeps_energy_grad_4x4(ipeps_env* env, const ipeps_ctensor_t* H4, int ad_iters, double* E,
                                    double* dA);
/* Pullback of run_es_h4 w.r.t. B (get_es_grad_h4, optim_es_h4.jl:133-168): as
 * ipeps_es_energy_grad with the plaquette energy; E = real(get_es_energy_4x4). */
/* The unit of optim_wp (get_wp_grad / run_wp, optim_wp.jl:195-238): in the environment held
 * by env (no CTMRG), the plaquette operator given as the MPO wp4 = [s1, s2, s3, s4] of
 * get_local_h and the norm of the 2x2 cluster whose site `site` (Params["wp"], 1..4) holds
 * B (ComplexF64, the shape of A) and the others A (energy_norm_4x4, evaluation.jl:435-441).
 * wp_norm[4] = (re, im) of the operator value, then of the norm; gH, gN (ComplexF64, the
 * shape of A): the gradients of their real parts w.r.t. B (Zygote's back((1, nothing)) and
 * back((nothing, 1))). */
IPEPS_API int ipeps_wp_grad(ipeps_env* env, const ipeps_ctensor_t* wp4, int site, const double* B, double* wp_norm,
                            double* gH, double* gN);
IPEPS_API int ipeps_es_energy_grad_4x4(ipeps_env* env, const ipeps_ctensor_t* H4, int ad_iters, double* E,
                                       double* gB);

/* ---- learned warm start (no counterpart in the reference: its CTMRG always starts
 * from init_ctm1, ctm_tensor.jl:97-130).  A 3-layer perceptron n_in -> n_hidden ->
 * n_hidden -> n_out (GELU) whose matrix products run on BF16 tensor-core GEMMs
 * with FP32 accumulation; FP32 parameters, mean-squared error, Adam.  Host arrays
 * are float32, column-major with the batch as rows (X: B x n_in, T/Y: B x n_out).
 * Parameters are one flat vector W1 (n_in x n_hidden), b1, W2, b2, W3 (n_hidden x
 * n_out), b3.  ipeps_gemm_bf16 exposes the GEMM on host buffers (C = alpha op(A)
 * op(B) + beta C, operands rounded to BF16) for its parity test. */
IPEPS_API int ipeps_gemm_bf16(ipeps_ctx* ctx, char opA, char opB, int64_t m, int64_t n, int64_t k, float alpha,
                    const float* A, int64_t lda, const float* B, int64_t ldb, float beta, float* C, int64_t ldc);
IPEPS_API int ipeps_mlp_create(ipeps_ctx* ctx, int n_in, int n_hidden, int n_out, int max_batch, uint64_t seed,
                     ipeps_mlp** out);
IPEPS_API int ipeps_mlp_destroy(ipeps_mlp* mlp);
IPEPS_API int ipeps_mlp_num_params(ipeps_mlp* mlp, int64_t* n);
IPEPS_API int ipeps_mlp_get_params(ipeps_mlp* mlp, float* params);
IPEPS_API int ipeps_mlp_set_params(ipeps_mlp* mlp, const float* params);
IPEPS_API int ipeps_mlp_forward(ipeps_mlp* mlp, const float* X, int B, float* Y);
/* loss and gradient (flat, like the parameters) of the mean-squared error, no update */
IPEPS_API int ipeps_mlp_grad(ipeps_mlp* mlp, const float* X, const float* T, int B, double* loss, float* grads);
/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the batch; *loss = the batch loss before the step */
IPEPS_API int ipeps_mlp_train_step(ipeps_mlp* mlp, const float* X, const float* T, int B, float lr, double* loss);

/* ---- FP64 GEMM of the engine (the DMMA kernel every real FP64 contraction of
 * tcon, the projector and the adjoint runs on; no counterpart in the reference,
 * where these products are BLAS calls inside TensorOperations).  Host buffers:
 * C = alpha*op(A)*op(B) + beta*C, column-major, op in {'N','T'}; the product is
 * computed `reps` times from the same input C (for timing; the result is that
 * of one product). */
IPEPS_API int ipeps_gemm_f64(ipeps_ctx* ctx, char opA, char opB, int64_t m, int64_t n, int64_t k, double alpha,
                             const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                             int64_t ldc, int reps);

/* ---- 3xTF32 GEMM on the tcgen05 tensor cores (no counterpart in the reference: the
 * contraction kernel of the mixed form, exposed for tests and kernel timing).
 * C = alpha*op(A)*op(B) + beta*C, column-major FP64 host arrays, op in {'N','T'}: each
 * operand is split into TF32 hi/lo planes, the products lo*hi + hi*lo + hi*hi accumulate
 * in FP32 in tensor memory, split-K partial sums in FP64.  The product runs `reps` times
 * from the same input C; *ms_per_rep (optional) receives the device time of one product
 * (splits included; the first repetition is excluded when reps > 1). */
IPEPS_API int ipeps_gemm_tf32x3(ipeps_ctx* ctx, char opA, char opB, int64_t m, int64_t n, int64_t k, double alpha,
                                const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                                int64_t ldc, int reps, double* ms_per_rep);

/* ---- allocation-free FP64 GEMM (no counterpart in the reference).
 * C = alpha*op(A)*op(B) + beta*C, column-major, op in {'N','T'}; A, B, C are
 * DEVICE pointers and the work is enqueued on `stream` (a cudaStream_t; NULL =
 * the legacy default stream); the call returns without synchronising.
 * For callers that cannot call cudaMalloc (device memory owned by a host
 * framework's pool, or sections where cudaMalloc/cudaFree are not allowed):
 * its split-K partial sums live in a fixed 4 MiB device array (524288
 * doubles) instead of an allocation.  The split is capped so that the partial
 * sums fit; outputs above 262144 elements (m*n) run unsplit and use no
 * scratch.  Shapes beyond the kernel grid (n > 65535*64) are rejected with
 * IPEPS_EINVAL and a message on stderr.  The first call on a device sets up
 * the array's address (make it before any stream capture).  All calls share
 * the array: calls that overlap on the GPU race. */
IPEPS_API int ipeps_gemm_f64_noalloc(char opA, char opB, int64_t m, int64_t n, int64_t k, double alpha,
                                     const double* A, int64_t lda, const double* B, int64_t ldb, double beta,
                                     double* C, int64_t ldc, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IPEPS_B200_H */
