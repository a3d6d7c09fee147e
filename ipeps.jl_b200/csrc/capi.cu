// extern "C" boundary of libipeps_b200 (declared in include/ipeps_b200.h).
#include "../../include/ipeps_b200.h"
#include "ctm.cuh"
#include "mlp.cuh"

#include <cstring>

struct ipeps_ctx {
  ipeps::Ctx* c = nullptr;
  std::string err;
  uint64_t moves_done = 0;
  double move_seconds = 0;
};

struct ipeps_env {
  ipeps_ctx* owner = nullptr;
  ipeps::Env e;
};

struct ipeps_mlp {
  ipeps_ctx* owner = nullptr;
  std::unique_ptr<ipeps::Mlp> m;
};

namespace {

using ipeps::DType;
using ipeps::Tensor;

template <typename F>
int guarded(ipeps_ctx* ctx, F&& f) {
  if (!ctx) return IPEPS_EINVAL;
  try {
    ctx->err.clear();
    if (ctx->c) IPEPS_CUDA(cudaMemsetAsync(ctx->c->d_status, 0, sizeof(int), ctx->c->stream));
    int st = f();
    if (ctx->c) {
      // status bits: 2 non-finite value, 4 Jacobi sweep cap hit, 8 tensor-core pipeline wait timed out,
      // 16 projector-adjoint resolvent series stopped at its term cap (counted in ipeps_stats_t)
      int dev_status = 0;
      IPEPS_CUDA(cudaMemcpyAsync(&dev_status, ctx->c->d_status, sizeof(int), cudaMemcpyDeviceToHost,
                                 ctx->c->stream));
      IPEPS_CUDA(cudaStreamSynchronize(ctx->c->stream));
      if (st == IPEPS_OK && (dev_status & 8)) {
        ctx->err = "tensor-core GEMM pipeline wait timed out (results invalid)";
        st = IPEPS_ECUDA;
      } else if (st == IPEPS_OK && (dev_status & 2)) {
        ctx->err = "non-finite value detected";
        st = IPEPS_ENONFINITE;
      }
    }
    return st;
  } catch (const ipeps::Error& e) {
    ctx->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    ctx->err = e.what();
    return IPEPS_ECUDA;
  }
}

Tensor upload(ipeps::Ctx& c, const double* h, DType dt, const std::vector<int64_t>& dims) {
  Tensor t = c.alloc(dt, dims);
  IPEPS_CUDA(cudaMemcpyAsync(t.data(), h, t.bytes(), cudaMemcpyHostToDevice, c.stream));
  return t;
}

void download(ipeps::Ctx& c, double* h, const Tensor& t) {
  IPEPS_CUDA(cudaMemcpyAsync(h, t.data(), t.bytes(), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
}

Tensor upload_H(ipeps::Ctx& c, const double* H, int d2) {
  IPEPS_CHECK(H != nullptr && d2 > 0, "Hamiltonian required");
  return upload(c, H, DType::C128, {d2, d2});
}

void account(ipeps_env* env, uint64_t m0, double s0) {
  env->owner->moves_done += env->e.moves - m0;
  env->owner->move_seconds += env->e.move_seconds - s0;
}

}  // namespace

extern "C" {

int ipeps_ctx_create(int device, ipeps_ctx** out) {
  if (!out) return IPEPS_EINVAL;
  *out = nullptr;
  auto* h = new ipeps_ctx();
  try {
    h->c = new ipeps::Ctx(device);
  } catch (const ipeps::Error& e) {
    int code = e.code;
    delete h;
    return code;
  }
  *out = h;
  return IPEPS_OK;
}

int ipeps_ctx_destroy(ipeps_ctx* ctx) {
  if (!ctx) return IPEPS_EINVAL;
  delete ctx->c;
  delete ctx;
  return IPEPS_OK;
}

const char* ipeps_last_error(ipeps_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int ipeps_ctx_set_precision(ipeps_ctx* ctx, int precision) {
  return guarded(ctx, [&] {
    IPEPS_CHECK(precision == IPEPS_PREC_FP64 || precision == IPEPS_PREC_MIXED, "bad precision");
    ctx->c->precision = precision;
    return IPEPS_OK;
  });
}

int ipeps_ctx_set_seed(ipeps_ctx* ctx, uint64_t seed) {
  return guarded(ctx, [&] {
    ctx->c->rng_seed = seed;
    ctx->c->rng_counter = 0;
    return IPEPS_OK;
  });
}

int ipeps_stats(ipeps_ctx* ctx, ipeps_stats_t* out) {
  return guarded(ctx, [&] {
    IPEPS_CHECK(out, "null stats");
    std::memset(out, 0, sizeof(*out));
    for (int i = 0; i < int(ipeps::KFam::Count) && i < 8; ++i) {
      out->launches[i] = ctx->c->stats[i].launches;
      out->flops[i] = ctx->c->stats[i].flops;
      out->bytes[i] = ctx->c->stats[i].bytes;
    }
    out->moves = ctx->moves_done;
    out->move_seconds = ctx->move_seconds;
    out->projector_calls = ctx->c->projector_calls;
    out->jacobi_sweeps = ctx->c->jacobi_sweeps;
    out->extra_passes = ctx->c->projector_extra_passes;
    out->series_cap_hits = ctx->c->series_cap_hits;
    out->series_terms = ctx->c->series_terms;
    out->series_retries = ctx->c->series_retries;
    out->resid_misses = ctx->c->resid_misses;
    return IPEPS_OK;
  });
}

int ipeps_stats_reset(ipeps_ctx* ctx) {
  return guarded(ctx, [&] {
    for (auto& s : ctx->c->stats) s = ipeps::KStat{};
    ctx->moves_done = 0;
    ctx->move_seconds = 0;
    ctx->c->projector_calls = 0;
    ctx->c->jacobi_sweeps = 0;
    ctx->c->projector_extra_passes = 0;
    ctx->c->series_cap_hits = 0;
    ctx->c->series_terms = 0;
    ctx->c->series_retries = 0;
    ctx->c->resid_misses = 0;
    return IPEPS_OK;
  });
}

int ipeps_ctx_stream(ipeps_ctx* ctx, void** stream) {
  return guarded(ctx, [&] {
    IPEPS_CHECK(stream, "null stream out");
    *stream = reinterpret_cast<void*>(ctx->c->stream);
    return IPEPS_OK;
  });
}

int ipeps_prof_enable(ipeps_ctx* ctx, int on) {
  return guarded(ctx, [&] {
    ctx->c->prof_collect();
    ctx->c->prof = on != 0;
    for (auto& s : ctx->c->prof_stats) s = ipeps::KStat{};
    return IPEPS_OK;
  });
}

int ipeps_prof_query(ipeps_ctx* ctx, double* ms, uint64_t* launches, double* flops, double* bytes) {
  return guarded(ctx, [&] {
    auto t = ctx->c->prof_collect();
    for (int i = 0; i < int(ipeps::KFam::Count) && i < 8; ++i) {
      if (ms) ms[i] = t[i];
      if (launches) launches[i] = ctx->c->prof_stats[i].launches;
      if (flops) flops[i] = ctx->c->prof_stats[i].flops;
      if (bytes) bytes[i] = ctx->c->prof_stats[i].bytes;
    }
    for (auto& s : ctx->c->prof_stats) s = ipeps::KStat{};
    return IPEPS_OK;
  });
}

int ipeps_prof_phases(ipeps_ctx* ctx, double* ms) {
  return guarded(ctx, [&] {
    IPEPS_CHECK(ms, "null output");
    for (int i = 0; i < 5; ++i) ms[i] = ctx->c->ad_phase_ms[size_t(i)];
    ctx->c->ad_phase_ms = {};
    return IPEPS_OK;
  });
}

int ipeps_tcon(ipeps_ctx* ctx, int is_complex, const double* A, int nA, const int64_t* dimsA, const int* la,
               const double* B, int nB, const int64_t* dimsB, const int* lb, double* out, int64_t out_cap,
               int64_t* out_dims, int* out_nd) {
  return guarded(ctx, [&] {
    IPEPS_CHECK(A && B && dimsA && dimsB && la && lb && nA >= 0 && nB >= 0, "bad tcon arguments");
    auto& c = *ctx->c;
    DType dt = is_complex ? DType::C128 : DType::F64;
    Tensor ta = upload(c, A, dt, std::vector<int64_t>(dimsA, dimsA + nA));
    Tensor tb = upload(c, B, dt, std::vector<int64_t>(dimsB, dimsB + nB));
    Tensor r = ipeps::tcon(c, ta, std::vector<int>(la, la + nA), tb, std::vector<int>(lb, lb + nB));
    if (out_nd) *out_nd = r.nd;
    if (out_dims) for (int i = 0; i < r.nd; ++i) out_dims[i] = r.dims[i];
    IPEPS_CHECK(r.numel() <= out_cap, "tcon: output capacity too small");
    if (out) download(c, out, r);
    return IPEPS_OK;
  });
}

int ipeps_projector(ipeps_ctx* ctx, const double* R1, const double* R2, int64_t N1, int64_t K1, int64_t N2, int chi,
                     double* P1, double* P2, double* s, int* n) {
  return guarded(ctx, [&] {
    IPEPS_CHECK(R1 && R2 && N1 > 0 && K1 > 0 && N2 > 0 && chi > 0 && n, "bad projector arguments");
    auto& c = *ctx->c;
    ipeps::MatRef r1{upload(c, R1, DType::F64, {N1, K1}), false};
    ipeps::MatRef r2{upload(c, R2, DType::F64, {K1, N2}), false};
    ipeps::SvdParams sp;
    ipeps::ProjResult pr = ipeps::get_projector(c, r1, r2, chi, sp, nullptr);
    *n = pr.n;
    if (P1) download(c, P1, pr.P1);
    if (P2) download(c, P2, pr.P2);
    if (s) for (int i = 0; i < pr.n; ++i) s[i] = pr.s_host[i];
    return IPEPS_OK;
  });
}

int ipeps_projector_c(ipeps_ctx* ctx, const double* R1, const double* R2, int64_t N1, int64_t K1, int64_t N2, int chi,
                       double* P1, double* P2, double* s, int* n) {
  return guarded(ctx, [&] {
    IPEPS_CHECK(R1 && R2 && N1 > 0 && K1 > 0 && N2 > 0 && chi > 0 && n, "bad projector arguments");
    auto& c = *ctx->c;
    ipeps::MatRef r1{upload(c, R1, DType::C128, {N1, K1}), false};
    ipeps::MatRef r2{upload(c, R2, DType::C128, {K1, N2}), false};
    ipeps::SvdParams sp;
    ipeps::ProjResult pr = ipeps::get_projector(c, r1, r2, chi, sp, nullptr);
    *n = pr.n;
    if (P1) download(c, P1, pr.P1);
    if (P2) download(c, P2, pr.P2);
    if (s) for (int i = 0; i < pr.n; ++i) s[i] = pr.s_host[i];
    return IPEPS_OK;
  });
}

int ipeps_orth(ipeps_ctx* ctx, const double* Y, int64_t N, int k, int passes, double* Q, double* R) {
  return guarded(ctx, [&] {
    IPEPS_CHECK(Y && Q && N > 0 && k > 0 && N >= k && passes >= 1, "bad orth arguments");
    auto& c = *ctx->c;
    Tensor y = upload(c, Y, DType::F64, {N, k});
    Tensor r;
    Tensor q = ipeps::orth(c, y, passes, R ? &r : nullptr);
    download(c, Q, q);
    if (R) download(c, R, r);
    return IPEPS_OK;
  });
}

int ipeps_env_create(ipeps_ctx* ctx, int D, int d, int chi, int is_complex, ipeps_env** out) {
  return guarded(ctx, [&] {
    IPEPS_CHECK(out && D > 0 && d > 0 && chi > 0, "bad env arguments");
    auto* h = new ipeps_env();
    h->owner = ctx;
    h->e.ctx = ctx->c;
    h->e.D = D;
    h->e.d = d;
    h->e.dt = is_complex ? DType::C128 : DType::F64;
    h->e.prm.chi = chi;
    *out = h;
    return IPEPS_OK;
  });
}

int ipeps_env_destroy(ipeps_env* env) {
  if (!env) return IPEPS_EINVAL;
  delete env;  // buffers are released in stream order (they keep the stream alive)
  return IPEPS_OK;
}

int ipeps_env_set_params(ipeps_env* env, int chi, int min_iter, int max_iter, int ad_max_iter, double rg_tol) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(chi > 0 && min_iter >= 0 && max_iter >= 0 && ad_max_iter >= 0, "bad params");
    env->e.prm.chi = chi;
    env->e.prm.min_iter = min_iter;
    env->e.prm.max_iter = max_iter;
    env->e.prm.ad_max_iter = ad_max_iter;
    env->e.prm.rg_tol = rg_tol;
    return IPEPS_OK;
  });
}

int ipeps_env_set_parallel(ipeps_env* env, int on) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    env->e.parallel_moves = on != 0;
    return IPEPS_OK;
  });
}

int ipeps_env_set_svd_params(ipeps_env* env, int over_num, int over_den, int min_over, int power_iters,
                             int power_iters_warm, int warm_start, double resid_tol, int max_extra,
                             int inter_passes, int seed_older) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(over_num >= 0 && over_den > 0 && min_over >= 0 && power_iters >= 0 && power_iters_warm >= 0 &&
                    resid_tol >= 0 && max_extra >= 0 && inter_passes >= 1,
                "bad svd params");
    env->e.prm.svd.resid_tol = resid_tol;
    env->e.prm.svd.max_extra_passes = max_extra;
    env->e.prm.svd.inter_passes = inter_passes;
    env->e.prm.svd.seed_older = seed_older != 0;
    auto& s = env->e.prm.svd;
    s.oversample_num = over_num;
    s.oversample_den = over_den;
    s.min_oversample = min_over;
    s.power_iters = power_iters;
    s.power_iters_warm = power_iters_warm;
    s.warm_start = warm_start != 0;
    return IPEPS_OK;
  });
}

int ipeps_env_set_A(ipeps_env* env, const double* A, const double* Ad) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(A, "null A");
    auto& c = *env->e.ctx;
    const int64_t D = env->e.D;
    std::vector<int64_t> dims{D, D, D, D, env->e.d};
    env->e.A = upload(c, A, env->e.dt, dims);
    env->e.Ad = Ad ? upload(c, Ad, env->e.dt, dims) : ipeps::conj(c, env->e.A);
    ipeps::check_finite(c, env->e.A);
    return IPEPS_OK;
  });
}

int ipeps_env_init(ipeps_env* env) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(!env->e.A.empty(), "set A first");
    ipeps::init_ctm1(env->e);
    env->e.nested = false;
    return IPEPS_OK;
  });
}

int ipeps_env_get_CT(ipeps_env* env, int k, double* C, int64_t* C_dims, double* E, int64_t* E_dims) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(k >= 1 && k <= 4, "k must be 1..4");
    const Tensor& Ct = env->e.Cs[k - 1];
    const Tensor& Et = env->e.Es[k - 1];
    IPEPS_CHECK(!Ct.empty() && !Et.empty(), "environment not initialised");
    if (C_dims) for (int i = 0; i < 2; ++i) C_dims[i] = Ct.dims[i];
    if (E_dims) for (int i = 0; i < 4; ++i) E_dims[i] = Et.dims[i];
    if (C) download(*env->e.ctx, C, Ct);
    if (E) download(*env->e.ctx, E, Et);
    return IPEPS_OK;
  });
}

int ipeps_env_set_CT(ipeps_env* env, int k, const double* C, const int64_t* C_dims, const double* E,
                     const int64_t* E_dims) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(k >= 1 && k <= 4 && C && C_dims && E && E_dims, "bad set_CT arguments");
    auto& c = *env->e.ctx;
    IPEPS_CHECK(E_dims[2] == env->e.D && E_dims[3] == env->e.D, "E must be (chi_a, chi_b, D, D)");
    env->e.Cs[k - 1] = upload(c, C, env->e.dt, {C_dims[0], C_dims[1]});
    env->e.Es[k - 1] = upload(c, E, env->e.dt, {E_dims[0], E_dims[1], E_dims[2], E_dims[3]});
    for (auto& cc : env->e.cache) cc = ipeps::ProjCache();
    return IPEPS_OK;
  });
}

int ipeps_ctm_move(ipeps_env* env, int dir, double* s_out, int* s_len) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(dir >= 0 && dir < 4, "dir must be 0..3");
    uint64_t m0 = env->e.moves;
    double s0 = env->e.move_seconds;
    std::vector<double> s = ipeps::ctm_move(env->e, dir);
    account(env, m0, s0);
    if (s_len) {
      int cap = *s_len;
      *s_len = int(s.size());
      if (s_out) for (int i = 0; i < std::min<int>(cap, int(s.size())); ++i) s_out[i] = s[i];
    }
    return IPEPS_OK;
  });
}

int ipeps_ctm_step(ipeps_env* env, double* s_out, int* s_len) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    uint64_t m0 = env->e.moves;
    double s0 = env->e.move_seconds;
    std::vector<double> s = ipeps::rg_step(env->e);
    account(env, m0, s0);
    if (s_len) {
      int cap = *s_len;
      *s_len = int(s.size());
      if (s_out) for (int i = 0; i < std::min<int>(cap, int(s.size())); ++i) s_out[i] = s[i];
    }
    return IPEPS_OK;
  });
}

int ipeps_ctm_run(ipeps_env* env, int conv_mode, const double* Hh, const double* Hv, int d2, int* iters,
                  double* last_diff, int* converged) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    auto& c = *env->e.ctx;
    Tensor th, tv;
    if (conv_mode != IPEPS_CONV_SPECTRUM) {
      th = upload_H(c, Hh, d2);
      tv = upload_H(c, Hv, d2);
    }
    uint64_t m0 = env->e.moves;
    double s0 = env->e.move_seconds;
    bool conv = false;
    double diff = 0;
    int it = ipeps::run_ctm(env->e, conv_mode, &th, &tv, &diff, &conv);
    account(env, m0, s0);
    if (iters) *iters = it;
    if (last_diff) *last_diff = diff;
    if (converged) *converged = conv ? 1 : 0;
    return IPEPS_OK;
  });
}

int ipeps_ctm_log(ipeps_env* env, double* out, int* n_iters) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(n_iters, "null n_iters");
    int cap = *n_iters;
    *n_iters = int(env->e.log.size());
    if (out)
      for (int i = 0; i < std::min<int>(cap, int(env->e.log.size())); ++i) {
        out[4 * i] = env->e.log[i].diff;
        out[4 * i + 1] = env->e.log[i].obj_re;
        out[4 * i + 2] = env->e.log[i].obj_im;
        out[4 * i + 3] = env->e.log[i].chi_left;
      }
    return IPEPS_OK;
  });
}

int ipeps_energy(ipeps_env* env, const double* Hh, const double* Hv, int d2, double* E, double* Na) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    auto& c = *env->e.ctx;
    Tensor th = upload_H(c, Hh, d2), tv = upload_H(c, Hv, d2);
    std::complex<double> e, na;
    ipeps::gs_energy(env->e, th, tv, &e, &na);
    if (E) { E[0] = e.real(); E[1] = e.imag(); }
    if (Na) { Na[0] = na.real(); Na[1] = na.imag(); }
    return IPEPS_OK;
  });
}

int ipeps_gs_norm(ipeps_env* env, double* nrm) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    std::complex<double> n = ipeps::gs_norm(env->e);
    if (nrm) { nrm[0] = n.real(); nrm[1] = n.imag(); }
    return IPEPS_OK;
  });
}

int ipeps_nested_set_B(ipeps_env* env, const double* B, double px, double py) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(B, "null B");
    auto& c = *env->e.ctx;
    const int64_t D = env->e.D;
    env->e.B = upload(c, B, DType::C128, {D, D, D, D, env->e.d});
    env->e.Bd = ipeps::conj(c, env->e.B);
    env->e.px = px;
    env->e.py = py;
    env->e.nested = true;
    for (int i = 0; i < 4; ++i) {
      env->e.B_Cs[i] = env->e.Bd_Cs[i] = env->e.BB_Cs[i] = Tensor();
      env->e.B_Es[i] = env->e.Bd_Es[i] = env->e.BB_Es[i] = Tensor();
    }
    return IPEPS_OK;
  });
}

int ipeps_es_energy(ipeps_env* env, const double* Hh, const double* Hv, int d2, double* E) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    auto& c = *env->e.ctx;
    Tensor th = upload_H(c, Hh, d2), tv = upload_H(c, Hv, d2);
    double e = ipeps::es_energy(env->e, th, tv);
    if (E) *E = e;
    return IPEPS_OK;
  });
}

int ipeps_all_norm(ipeps_env* env, double* Nb, double* envB) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    Tensor eb;
    std::complex<double> nb = ipeps::all_norm(env->e, envB ? &eb : nullptr);
    if (Nb) { Nb[0] = nb.real(); Nb[1] = nb.imag(); }
    if (envB) download(*env->e.ctx, envB, eb);
    return IPEPS_OK;
  });
}

}  // extern "C"

#include "ad.cuh"

extern "C" int ipeps_energy_grad(ipeps_env* env, const double* Hh, const double* Hv, int d2, int ad_iters, double* E,
                                 double* dA) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(ad_iters >= 1, "ad_iters must be >= 1");
    auto& c = *env->e.ctx;
    Tensor th = upload_H(c, Hh, d2), tv = upload_H(c, Hv, d2);
    uint64_t m0 = env->e.moves;
    double s0 = env->e.move_seconds;
    Tensor g;
    double e = ipeps::energy_grad(env->e, th, tv, ad_iters, &g);
    account(env, m0, s0);
    if (E) *E = e;
    if (dA) download(c, dA, g);
    return IPEPS_OK;
  });
}

extern "C" int ipeps_env_set_mixed(ipeps_env* env, int polish_iters, double polish_tol) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(polish_iters >= 0 && polish_tol >= 0, "bad mixed-form parameters");
    env->e.prm.polish_iters = polish_iters;
    env->e.prm.polish_tol = polish_tol;
    return IPEPS_OK;
  });
}

extern "C" int ipeps_es_energy_grad(ipeps_env* env, const double* Hh, const double* Hv, int d2, int ad_iters,
                                    double* E, double* gB) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(ad_iters >= 1, "ad_iters must be >= 1");
    auto& c = *env->e.ctx;
    Tensor th = upload_H(c, Hh, d2), tv = upload_H(c, Hv, d2);
    uint64_t m0 = env->e.moves;
    double s0 = env->e.move_seconds;
    Tensor g;
    double e = ipeps::es_energy_grad(env->e, th, tv, ad_iters, &g);
    account(env, m0, s0);
    if (E) *E = e;
    if (gB) download(c, gB, g);
    return IPEPS_OK;
  });
}

namespace {

ipeps::H4 upload_H4(ipeps::Ctx& c, const ipeps_ctensor_t* H) {
  IPEPS_CHECK(H != nullptr, "plaquette Hamiltonian required");
  static const int want_nd[4] = {3, 4, 4, 3};
  ipeps::H4 h;
  for (int k = 0; k < 4; ++k) {
    IPEPS_CHECK(H[k].data && H[k].nd == want_nd[k], "plaquette MPO factor " + std::to_string(k + 1) +
                                                        ": expected a " + std::to_string(want_nd[k]) + "-d tensor");
    std::vector<int64_t> dims(H[k].dims, H[k].dims + H[k].nd);
    for (int64_t d : dims) IPEPS_CHECK(d > 0, "plaquette MPO factor with an empty dimension");
    h[k] = upload(c, H[k].data, DType::C128, dims);
  }
  IPEPS_CHECK(h[0].dims[2] == h[1].dims[0] && h[1].dims[3] == h[2].dims[0] && h[2].dims[3] == h[3].dims[0],
              "plaquette MPO bond dimensions do not chain");
  return h;
}

}  // namespace

extern "C" int ipeps_energy_4x4(ipeps_env* env, const ipeps_ctensor_t* H4, int nested, double* E) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    ipeps::H4 h = upload_H4(*env->e.ctx, H4);
    std::complex<double> v = nested ? ipeps::es_energy_4x4(env->e, h) : ipeps::gs_energy_4x4(env->e, h);
    if (E) { E[0] = v.real(); E[1] = v.imag(); }
    return IPEPS_OK;
  });
}

extern "C" int ipeps_ctm_run_4x4(ipeps_env* env, const ipeps_ctensor_t* H4, int nested, int* iters,
                                 double* last_diff, int* converged) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    ipeps::H4 h = upload_H4(*env->e.ctx, H4);
    uint64_t m0 = env->e.moves;
    double s0 = env->e.move_seconds;
    bool conv = false;
    double diff = 0;
    int it = ipeps::run_ctm(env->e, nested ? ipeps::kConvEs4x4 : ipeps::kConvEnergy4x4, nullptr, nullptr, &diff,
                            &conv, &h);
    account(env, m0, s0);
    if (iters) *iters = it;
    if (last_diff) *last_diff = diff;
    if (converged) *converged = conv ? 1 : 0;
    return IPEPS_OK;
  });
}

extern "C" int ipeps_energy_grad_4x4(ipeps_env* env, const ipeps_ctensor_t* H4, int ad_iters, double* E,
                                     double* dA) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(ad_iters >= 1, "ad_iters must be >= 1");
    auto& c = *env->e.ctx;
    ipeps::H4 h = upload_H4(c, H4);
    uint64_t m0 = env->e.moves;
    double s0 = env->e.move_seconds;
    Tensor g, none;
    double e = ipeps::energy_grad(env->e, none, none, ad_iters, &g, &h);
    account(env, m0, s0);
    if (E) *E = e;
    if (dA) download(c, dA, g);
    return IPEPS_OK;
  });
}

extern "C" int ipeps_es_energy_grad_4x4(ipeps_env* env, const ipeps_ctensor_t* H4, int ad_iters, double* E,
                                        double* gB) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(ad_iters >= 1, "ad_iters must be >= 1");
    auto& c = *env->e.ctx;
    ipeps::H4 h = upload_H4(c, H4);
    uint64_t m0 = env->e.moves;
    double s0 = env->e.move_seconds;
    Tensor g, none;
    double e = ipeps::es_energy_grad(env->e, none, none, ad_iters, &g, &h);
    account(env, m0, s0);
    if (E) *E = e;
    if (gB) download(c, gB, g);
    return IPEPS_OK;
  });
}

extern "C" int ipeps_wp_grad(ipeps_env* env, const ipeps_ctensor_t* wp4, int site, const double* B,
                             double* wp_norm, double* gH, double* gN) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(B && site >= 1 && site <= 4, "ipeps_wp_grad: B and site 1..4 required");
    auto& c = *env->e.ctx;
    ipeps::H4 h = upload_H4(c, wp4);
    Tensor b = upload(c, B, DType::C128, env->e.A.shape());
    std::complex<double> w, n;
    Tensor gh, gn;
    ipeps::wp_grad(env->e, h, site, b, &w, &n, &gh, &gn);
    if (wp_norm) {
      wp_norm[0] = w.real();
      wp_norm[1] = w.imag();
      wp_norm[2] = n.real();
      wp_norm[3] = n.imag();
    }
    if (gH) download(c, gH, gh);
    if (gN) download(c, gN, gn);
    return IPEPS_OK;
  });
}

extern "C" int ipeps_single_dm_Ad(ipeps_env* env, double* out) {
  if (!env) return IPEPS_EINVAL;
  return guarded(env->owner, [&] {
    IPEPS_CHECK(out, "null output");
    Tensor t = ipeps::single_dm_Ad(env->e);
    download(*env->e.ctx, out, t);
    return IPEPS_OK;
  });
}

// ------------------------------------------------------------ warm-start network
namespace {

void h2d(ipeps::Ctx& c, void* d, const void* h, size_t bytes) {
  IPEPS_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, c.stream));
}
void d2h(ipeps::Ctx& c, void* h, const void* d, size_t bytes) {
  IPEPS_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, c.stream));
}

}  // namespace

int ipeps_gemm_bf16(ipeps_ctx* ctx, char opA, char opB, int64_t m, int64_t n, int64_t k, float alpha, const float* A,
                    int64_t lda, const float* B, int64_t ldb, float beta, float* C, int64_t ldc) {
  return guarded(ctx, [&] {
    IPEPS_CHECK(A && B && C && m > 0 && n > 0 && k > 0, "bad gemm_bf16 arguments");
    auto& c = *ctx->c;
    const int64_t acols = (opA == 'N') ? k : m, bcols = (opB == 'N') ? n : k;
    IPEPS_CHECK(lda >= ((opA == 'N') ? m : k) && ldb >= ((opB == 'N') ? k : n) && ldc >= m, "bad leading dimension");
    ipeps::DBuf dA(size_t(lda * acols) * 4, c.sh), dB(size_t(ldb * bcols) * 4, c.sh), dC(size_t(ldc * n) * 4, c.sh);
    h2d(c, dA.p, A, dA.bytes);
    h2d(c, dB.p, B, dB.bytes);
    h2d(c, dC.p, C, dC.bytes);
    ipeps::gemm_bf16(c, opA, opB, m, n, k, alpha, static_cast<float*>(dA.p), lda, static_cast<float*>(dB.p), ldb,
                     beta, static_cast<float*>(dC.p), ldc);
    d2h(c, C, dC.p, dC.bytes);
    c.sync();
    return IPEPS_OK;
  });
}

int ipeps_gemm_f64(ipeps_ctx* ctx, char opA, char opB, int64_t m, int64_t n, int64_t k, double alpha,
                   const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc,
                   int reps) {
  return guarded(ctx, [&] {
    IPEPS_CHECK(A && B && C && m > 0 && n > 0 && k > 0 && reps >= 1, "bad gemm_f64 arguments");
    IPEPS_CHECK((opA == 'N' || opA == 'T') && (opB == 'N' || opB == 'T'), "gemm_f64: op must be 'N' or 'T'");
    auto& c = *ctx->c;
    const int64_t acols = (opA == 'N') ? k : m, bcols = (opB == 'N') ? n : k;
    IPEPS_CHECK(lda >= ((opA == 'N') ? m : k) && ldb >= ((opB == 'N') ? k : n) && ldc >= m, "bad leading dimension");
    ipeps::DBuf dA(size_t(lda * acols) * 8, c.sh), dB(size_t(ldb * bcols) * 8, c.sh), dC(size_t(ldc * n) * 8, c.sh),
        dC0(size_t(ldc * n) * 8, c.sh);
    h2d(c, dA.p, A, dA.bytes);
    h2d(c, dB.p, B, dB.bytes);
    h2d(c, dC0.p, C, dC0.bytes);
    for (int r = 0; r < reps; ++r) {
      IPEPS_CUDA(cudaMemcpyAsync(dC.p, dC0.p, dC.bytes, cudaMemcpyDeviceToDevice, c.stream));
      ipeps::gemm_f64_dmma(c, opA, opB, m, n, k, alpha, static_cast<double*>(dA.p), lda, static_cast<double*>(dB.p),
                           ldb, beta, static_cast<double*>(dC.p), ldc);
    }
    d2h(c, C, dC.p, dC.bytes);
    c.sync();
    return IPEPS_OK;
  });
}

int ipeps_gemm_tf32x3(ipeps_ctx* ctx, char opA, char opB, int64_t m, int64_t n, int64_t k, double alpha,
                      const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                      int64_t ldc, int reps, double* ms_per_rep) {
  return guarded(ctx, [&] {
    IPEPS_CHECK(A && B && C && m > 0 && n > 0 && k > 0 && reps >= 1, "bad gemm_tf32x3 arguments");
    IPEPS_CHECK((opA == 'N' || opA == 'T') && (opB == 'N' || opB == 'T'), "gemm_tf32x3: op must be 'N' or 'T'");
    auto& c = *ctx->c;
    const int64_t acols = (opA == 'N') ? k : m, bcols = (opB == 'N') ? n : k;
    IPEPS_CHECK(lda >= ((opA == 'N') ? m : k) && ldb >= ((opB == 'N') ? k : n) && ldc >= m, "bad leading dimension");
    ipeps::DBuf dA(size_t(lda * acols) * 8, c.sh), dB(size_t(ldb * bcols) * 8, c.sh), dC(size_t(ldc * n) * 8, c.sh),
        dC0(size_t(ldc * n) * 8, c.sh);
    h2d(c, dA.p, A, dA.bytes);
    h2d(c, dB.p, B, dB.bytes);
    h2d(c, dC0.p, C, dC0.bytes);
    cudaEvent_t e0 = c.take_event(), e1 = c.take_event();
    float total = 0;
    for (int r = 0; r < reps; ++r) {
      IPEPS_CUDA(cudaMemcpyAsync(dC.p, dC0.p, dC.bytes, cudaMemcpyDeviceToDevice, c.stream));
      IPEPS_CUDA(cudaEventRecord(e0, c.stream));
      ipeps::gemm_tf32x3(c, opA, opB, m, n, k, alpha, static_cast<double*>(dA.p), lda, static_cast<double*>(dB.p),
                         ldb, beta, static_cast<double*>(dC.p), ldc);
      IPEPS_CUDA(cudaEventRecord(e1, c.stream));
      IPEPS_CUDA(cudaEventSynchronize(e1));
      float t = 0;
      IPEPS_CUDA(cudaEventElapsedTime(&t, e0, e1));
      if (r > 0 || reps == 1) total += t;
    }
    c.ev_pool.push_back(e0);
    c.ev_pool.push_back(e1);
    if (ms_per_rep) *ms_per_rep = double(total) / double(reps > 1 ? reps - 1 : 1);
    d2h(c, C, dC.p, dC.bytes);
    c.sync();
    return IPEPS_OK;
  });
}

int ipeps_mlp_create(ipeps_ctx* ctx, int n_in, int n_hidden, int n_out, int max_batch, uint64_t seed,
                     ipeps_mlp** out) {
  return guarded(ctx, [&] {
    IPEPS_CHECK(out, "null output handle");
    auto* h = new ipeps_mlp();
    h->owner = ctx;
    try {
      h->m.reset(new ipeps::Mlp(*ctx->c, n_in, n_hidden, n_out, max_batch, seed));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return IPEPS_OK;
  });
}

int ipeps_mlp_destroy(ipeps_mlp* h) {
  // touches no context: the network's buffers hold their own reference to the
  // stream they are freed on (stream-ordered), so this is safe in any order
  if (!h) return IPEPS_EINVAL;
  delete h;
  return IPEPS_OK;
}

int ipeps_mlp_num_params(ipeps_mlp* h, int64_t* n) {
  if (!h || !n) return IPEPS_EINVAL;
  *n = h->m->np;
  return IPEPS_OK;
}

int ipeps_mlp_get_params(ipeps_mlp* h, float* p) {
  if (!h) return IPEPS_EINVAL;
  return guarded(h->owner, [&] {
    IPEPS_CHECK(p, "null buffer");
    d2h(h->m->c, p, h->m->params->p, size_t(h->m->np) * 4);
    h->m->c.sync();
    return IPEPS_OK;
  });
}

int ipeps_mlp_set_params(ipeps_mlp* h, const float* p) {
  if (!h) return IPEPS_EINVAL;
  return guarded(h->owner, [&] {
    IPEPS_CHECK(p, "null buffer");
    h2d(h->m->c, h->m->params->p, p, size_t(h->m->np) * 4);
    return IPEPS_OK;
  });
}

int ipeps_mlp_forward(ipeps_mlp* h, const float* X, int B, float* Y) {
  if (!h) return IPEPS_EINVAL;
  return guarded(h->owner, [&] {
    auto& m = *h->m;
    IPEPS_CHECK(X && Y && B > 0 && B <= m.cap, "bad mlp_forward arguments");
    h2d(m.c, m.X->p, X, size_t(B) * m.n_in * 4);
    m.forward(B);
    d2h(m.c, Y, m.Y->p, size_t(B) * m.n_out * 4);
    m.c.sync();
    return IPEPS_OK;
  });
}

int ipeps_mlp_grad(ipeps_mlp* h, const float* X, const float* T, int B, double* loss, float* grads) {
  if (!h) return IPEPS_EINVAL;
  return guarded(h->owner, [&] {
    auto& m = *h->m;
    IPEPS_CHECK(X && T && B > 0 && B <= m.cap, "bad mlp_grad arguments");
    h2d(m.c, m.X->p, X, size_t(B) * m.n_in * 4);
    h2d(m.c, m.T->p, T, size_t(B) * m.n_out * 4);
    m.forward(B);
    const double l = m.loss_and_grad(B);
    if (loss) *loss = l;
    if (grads) {
      d2h(m.c, grads, m.grads->p, size_t(m.np) * 4);
      m.c.sync();
    }
    return IPEPS_OK;
  });
}

int ipeps_mlp_train_step(ipeps_mlp* h, const float* X, const float* T, int B, float lr, double* loss) {
  if (!h) return IPEPS_EINVAL;
  return guarded(h->owner, [&] {
    auto& m = *h->m;
    IPEPS_CHECK(X && T && B > 0 && B <= m.cap && lr > 0, "bad mlp_train_step arguments");
    h2d(m.c, m.X->p, X, size_t(B) * m.n_in * 4);
    h2d(m.c, m.T->p, T, size_t(B) * m.n_out * 4);
    m.forward(B);
    const double l = m.loss_and_grad(B);
    m.adam(lr);
    if (loss) *loss = l;
    return IPEPS_OK;
  });
}
