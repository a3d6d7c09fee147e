// CTMRG engine: nested-tensor algebra, the four directional moves, the
// energy and run_ctm.  The contraction sequences live in moves.cuh
// (reference labels verbatim); this file instantiates them on NT tensors
// (plain or 4-component nested) and adds the projector, max-abs
// renormalisation, the phase shift of the nested move and the run loop.
#include "ctm.cuh"
#include "linalg.cuh"
#include "moves.cuh"

#include <chrono>
#include <exception>
#include <thread>
#include <cmath>

namespace ipeps {

// ------------------------------------------------------------ nested algebra
namespace {

void add_into(Ctx& c, Tensor& acc, const Tensor& t) {
  if (t.empty()) return;
  if (acc.empty()) {
    acc = t;
    return;
  }
  if (acc.dt == DType::F64 && t.dt == DType::C128) acc = to_complex(c, acc);
  axpy(c, cplx(1), t, acc);  // real into complex handled by axpy_rc
}

}  // namespace

// nested_tensor.jl:77-92 (product rule), emptyT.jl:24-26 (EmptyT absorbs)
NT ntcon(Ctx& c, const NT& A, const std::vector<int>& la, const NT& B, const std::vector<int>& lb) {
  if (!A.nested && !B.nested) return NT(tcon(c, A.c[0], la, B.c[0], lb));
  NT r;
  r.nested = true;
  if (A.nested && B.nested) {
    static const int pairs[4][4][2] = {{{0, 0}, {-1, -1}, {-1, -1}, {-1, -1}},
                                       {{0, 1}, {1, 0}, {-1, -1}, {-1, -1}},
                                       {{0, 2}, {2, 0}, {-1, -1}, {-1, -1}},
                                       {{0, 3}, {3, 0}, {1, 2}, {2, 1}}};
    for (int o = 0; o < 4; ++o)
      for (int p = 0; p < 4; ++p) {
        int i = pairs[o][p][0], j = pairs[o][p][1];
        if (i < 0 || !A.has(i) || !B.has(j)) continue;
        add_into(c, r.c[o], tcon(c, A.c[i], la, B.c[j], lb));
      }
  } else if (A.nested) {
    for (int i = 0; i < 4; ++i)
      if (A.has(i)) r.c[i] = tcon(c, A.c[i], la, B.c[0], lb);
  } else {
    for (int i = 0; i < 4; ++i)
      if (B.has(i)) r.c[i] = tcon(c, A.c[0], la, B.c[i], lb);
  }
  return r;
}

NT nreshape(const NT& A, const std::vector<int64_t>& s) {
  NT r = A;
  for (int i = 0; i < 4; ++i)
    if (A.has(i)) r.c[i] = A.c[i].reshape(s);
  return r;
}

NT npermute(Ctx& c, const NT& A, const std::vector<int>& perm) {
  NT r = A;
  for (int i = 0; i < 4; ++i)
    if (A.has(i)) r.c[i] = permute(c, A.c[i], perm);
  return r;
}

// nested_tensor.jl:43-44 (componentwise product with a plain matrix)
NT nmatmul(Ctx& c, const NT& A, char opA, const NT& B, char opB) {
  IPEPS_CHECK(!(A.nested && B.nested), "nmatmul: nested x nested");
  NT r;
  r.nested = A.nested || B.nested;
  if (A.nested) {
    for (int i = 0; i < 4; ++i)
      if (A.has(i)) r.c[i] = matmul(c, A.c[i], opA, B.c[0], opB);
  } else if (B.nested) {
    for (int i = 0; i < 4; ++i)
      if (B.has(i)) r.c[i] = matmul(c, A.c[0], opA, B.c[i], opB);
  } else {
    r.c[0] = matmul(c, A.c[0], opA, B.c[0], opB);
  }
  return r;
}

// nested_tensor.jl:65: [A1, A2 e^{i phi}, A3 e^{-i phi}, A4]
NT nshift(Ctx& c, const NT& A, double phi) {
  if (!A.nested) return A;
  NT r = A;
  const double cs = std::cos(phi), sn = std::sin(phi);
  if (A.has(1)) {
    r.c[1] = clone(c, to_complex(c, A.c[1]));
    scale(c, r.c[1], cplx(cs, sn));
  }
  if (A.has(2)) {
    r.c[2] = clone(c, to_complex(c, A.c[2]));
    scale(c, r.c[2], cplx(cs, -sn));
  }
  return r;
}

// wrapper.jl:57 / nested_tensor.jl:70-75: divide by max|component 1|
void nrenormalize(Ctx& c, NT& A) {
  double* d_m = reinterpret_cast<double*>(c.scal->p) + 16;
  maxabs(c, A.c[0], d_m);
  for (int i = 0; i < 4; ++i)
    if (A.has(i)) {
      A.c[i] = A.c[i].buf.use_count() > 1 ? clone(c, A.c[i]) : A.c[i];
      scale_inv(c, A.c[i], d_m);
    }
}

// Forward policy for moves.cuh on NT tensors
struct NTPolicy {
  using T = NT;
  Ctx& c;
  T tc(const T& a, const std::vector<int>& la, const T& b, const std::vector<int>& lb) { return ntcon(c, a, la, b, lb); }
  T rs(const T& a, const std::vector<int64_t>& s) { return nreshape(a, s); }
  T pm(const T& a, const std::vector<int>& perm) { return npermute(c, a, perm); }
  T mm(const T& a, const T& b) { return nmatmul(c, a, 'N', b, 'N'); }
  int64_t dim(const T& a, int i) const { return a.c[0].dims[i]; }
};

// ------------------------------------------------------------ environment
NT Env::all_A() const {  // ctm_tensor.jl:20-27
  if (!nested) return NT(A);
  NT r;
  r.nested = true;
  r.c[0] = A;
  r.c[1] = B;
  return r;
}
NT Env::all_Ad() const {  // ctm_tensor.jl:29-36
  if (!nested) return NT(Ad);
  NT r;
  r.nested = true;
  r.c[0] = Ad;
  r.c[2] = Bd;
  return r;
}
NT Env::all_C(int i) const {  // ctm_tensor.jl:38-45
  if (!nested) return NT(Cs[i]);
  NT r;
  r.nested = true;
  r.c = {Cs[i], B_Cs[i], Bd_Cs[i], BB_Cs[i]};
  return r;
}
NT Env::all_E(int i) const {  // ctm_tensor.jl:47-55
  if (!nested) return NT(Es[i]);
  NT r;
  r.nested = true;
  r.c = {Es[i], B_Es[i], Bd_Es[i], BB_Es[i]};
  return r;
}

// ctm_tensor.jl:97-130
void init_ctm1(Env& e) {
  Ctx& c = *e.ctx;
  const int64_t D = e.D, D2 = int64_t(D) * D;
  auto mk = [&](const std::vector<int>& la, const std::vector<int>& lb, std::vector<int64_t> shape) {
    NT t(tcon(c, e.A, la, e.Ad, lb).reshape(shape));
    nrenormalize(c, t);
    return t.c[0];
  };
  e.Cs[0] = mk({1, 2, -1, -3, 3}, {1, 2, -2, -4, 3}, {D2, D2});
  e.Cs[1] = mk({1, -1, -3, 2, 3}, {1, -2, -4, 2, 3}, {D2, D2});
  e.Cs[2] = mk({-1, -3, 1, 2, 3}, {-2, -4, 1, 2, 3}, {D2, D2});
  e.Cs[3] = mk({-1, 1, 2, -3, 3}, {-2, 1, 2, -4, 3}, {D2, D2});
  e.Es[0] = mk({1, -1, -5, -3, 2}, {1, -2, -6, -4, 2}, {D2, D2, D, D});
  e.Es[1] = mk({-1, -5, -3, 1, 2}, {-2, -6, -4, 1, 2}, {D2, D2, D, D});
  e.Es[2] = mk({-5, -1, 1, -3, 2}, {-6, -2, 1, -4, 2}, {D2, D2, D, D});
  e.Es[3] = mk({-1, 1, -3, -5, 2}, {-2, 1, -4, -6, 2}, {D2, D2, D, D});
  for (int i = 0; i < 4; ++i) e.cache[i] = ProjCache();
}

// One directional move: *_rg (ctmrg.jl:66-120) = projector + proj_* +
// renormalize + up_*.
std::vector<double> ctm_move(Env& e, int dir, ProjResult* keep) {
  Ctx& c = *e.ctx;
  auto t0 = std::chrono::steady_clock::now();
  NTPolicy p{c};
  Arr4<NTPolicy> Cs0, Es0;
  for (int i = 0; i < 4; ++i) {
    Cs0[i] = NT(e.Cs[i]);
    Es0[i] = NT(e.Es[i]);
  }
  ProjResult pr;
  {
    QuarterPair<NTPolicy> q = quarters(p, dir, Cs0, Es0, NT(e.A), NT(e.Ad));
    MatRef R1{q.R1.c[0], q.t1}, R2{q.R2.c[0], q.t2};
    pr = get_projector(c, R1, R2, e.prm.chi, e.prm.svd, &e.cache[dir], keep != nullptr && e.keep_adjoint);
  }
  Arr4<NTPolicy> Cs, Es;
  for (int i = 0; i < 4; ++i) {
    Cs[i] = e.all_C(i);
    Es[i] = e.all_E(i);
  }
  Projected<NTPolicy> np = project(p, dir, Cs, Es, e.all_A(), e.all_Ad(), NT(pr.P1), NT(pr.P2));
  nrenormalize(c, np.Ca);
  nrenormalize(c, np.E);
  nrenormalize(c, np.Cb);
  int ia, ib, ie;
  move_slots(dir, &ia, &ib, &ie);
  if (e.nested) {
    const double phi = (dir == 0) ? -e.px : (dir == 1) ? e.px : (dir == 2) ? -e.py : e.py;
    np.Ca = nshift(c, np.Ca, phi);
    np.Cb = nshift(c, np.Cb, phi);
    np.E = nshift(c, np.E, phi);
    e.B_Cs[ia] = np.Ca.c[1]; e.Bd_Cs[ia] = np.Ca.c[2]; e.BB_Cs[ia] = np.Ca.c[3];
    e.B_Cs[ib] = np.Cb.c[1]; e.Bd_Cs[ib] = np.Cb.c[2]; e.BB_Cs[ib] = np.Cb.c[3];
    e.B_Es[ie] = np.E.c[1]; e.Bd_Es[ie] = np.E.c[2]; e.BB_Es[ie] = np.E.c[3];
  }
  e.Cs[ia] = np.Ca.c[0];
  e.Cs[ib] = np.Cb.c[0];
  e.Es[ie] = np.E.c[0];
  e.moves++;
  auto t1 = std::chrono::steady_clock::now();
  e.move_seconds += std::chrono::duration<double>(t1 - t0).count();
  std::vector<double> s = pr.s_host;
  if (keep) *keep = std::move(pr);
  return s;
}

namespace {

void rehome(Tensor& t, const std::shared_ptr<StreamHolder>& sh) {
  if (t.buf && t.buf->sh != sh) t.buf->sh = sh;
}

// Moves `da` (on e's context) and `db` (on the auxiliary context) at the same
// time.  The pairs (left, right) and (top, bottom) touch disjoint slots: left
// reads C1 C4 E1 E3 E4 and writes C1 E4 C4, right reads C2 C3 E1 E2 E3 and
// writes C2 E2 C3 (ctmrg.jl:122-186); top reads C1 C2 E1 E2 E4 and writes
// C1 E1 C2, bottom reads C3 C4 E2 E3 E4 and writes C3 E3 C4 (ctmrg.jl:188-252).
// Each move runs from its own host thread (the projector reads singular values
// back, so one thread could not keep both streams busy) on a shallow copy of
// the environment; afterwards the streams are joined both ways, the second
// move's slots and projector cache are copied back, and every long-lived
// tensor is re-homed to the main stream, so later frees are ordered after all
// work of both streams.  Until then `keep` holds every tensor either move may
// drop, so no buffer is freed while the other stream may still read it.
std::vector<double> move_pair(Env& e, int da, int db, ProjResult* ka, ProjResult* kb) {
  Ctx& c1 = *e.ctx;
  if (!e.aux) {
    e.aux = std::make_shared<Ctx>(c1.device);
    e.aux->rng_seed = c1.rng_seed ^ 0x9e3779b97f4a7c15ULL;
  }
  Ctx& c2 = *e.aux;
  c2.precision = c1.precision;
  c2.prof = c1.prof;
  c2.d_status = c1.d_status;  // device-side problems of either stream reach the caller's status word
  const Env keep = e;
  Env eb = e;
  eb.ctx = &c2;
  eb.aux.reset();
  cudaEvent_t ev0 = c1.take_event(), ev1 = c1.take_event(), ev2 = c1.take_event();
  IPEPS_CUDA(cudaEventRecord(ev0, c1.stream));
  IPEPS_CUDA(cudaStreamWaitEvent(c2.stream, ev0, 0));
  std::exception_ptr err_a, err_b;
  std::vector<double> s;
  std::thread tb([&] {
    try {
      IPEPS_CUDA(cudaSetDevice(c2.device));
      ctm_move(eb, db, kb);
    } catch (...) {
      err_b = std::current_exception();
    }
  });
  try {
    s = ctm_move(e, da, ka);
  } catch (...) {
    err_a = std::current_exception();
  }
  tb.join();
  IPEPS_CUDA(cudaEventRecord(ev1, c2.stream));
  IPEPS_CUDA(cudaStreamWaitEvent(c1.stream, ev1, 0));
  IPEPS_CUDA(cudaEventRecord(ev2, c1.stream));
  IPEPS_CUDA(cudaStreamWaitEvent(c2.stream, ev2, 0));
  c1.ev_pool.push_back(ev0);
  c1.ev_pool.push_back(ev1);
  c1.ev_pool.push_back(ev2);
  // counters and timing records of the auxiliary context go to the main one
  for (int f = 0; f < int(KFam::Count); ++f) {
    c1.stats[f].launches += c2.stats[f].launches;
    c1.stats[f].flops += c2.stats[f].flops;
    c1.stats[f].bytes += c2.stats[f].bytes;
    c1.prof_stats[f].launches += c2.prof_stats[f].launches;
    c1.prof_stats[f].flops += c2.prof_stats[f].flops;
    c1.prof_stats[f].bytes += c2.prof_stats[f].bytes;
  }
  c2.stats = {};
  c2.prof_stats = {};
  c1.jacobi_sweeps += c2.jacobi_sweeps;
  c1.projector_calls += c2.projector_calls;
  c1.projector_extra_passes += c2.projector_extra_passes;
  c1.series_cap_hits += c2.series_cap_hits;
  c1.series_terms += c2.series_terms;
  c1.series_retries += c2.series_retries;
  c1.resid_misses += c2.resid_misses;
  c2.jacobi_sweeps = c2.projector_calls = c2.projector_extra_passes = c2.series_cap_hits = 0;
  c2.series_terms = c2.series_retries = c2.resid_misses = 0;
  for (auto& r : c2.prof_rec) c1.prof_rec.push_back(r);
  c2.prof_rec.clear();
  if (err_a) std::rethrow_exception(err_a);
  if (err_b) std::rethrow_exception(err_b);
  int ia, ib, ie;
  move_slots(db, &ia, &ib, &ie);
  e.Cs[ia] = eb.Cs[ia];
  e.Cs[ib] = eb.Cs[ib];
  e.Es[ie] = eb.Es[ie];
  using Slots = std::array<Tensor, 4> Env::*;
  if (e.nested) {
    for (Slots a : {&Env::B_Cs, &Env::Bd_Cs, &Env::BB_Cs}) {
      (e.*a)[ia] = (eb.*a)[ia];
      (e.*a)[ib] = (eb.*a)[ib];
    }
    for (Slots a : {&Env::B_Es, &Env::Bd_Es, &Env::BB_Es}) (e.*a)[ie] = (eb.*a)[ie];
  }
  e.cache[db] = eb.cache[db];
  e.moves += eb.moves - keep.moves;
  e.move_seconds += eb.move_seconds - keep.move_seconds;
  for (int i = 0; i < 4; ++i) {
    for (Slots a : {&Env::Cs, &Env::Es, &Env::B_Cs, &Env::Bd_Cs, &Env::BB_Cs, &Env::B_Es, &Env::Bd_Es, &Env::BB_Es})
      rehome((e.*a)[i], c1.sh);
    rehome(e.cache[i].V, c1.sh);
    rehome(e.cache[i].Vold, c1.sh);
  }
  if (kb)
    for (Tensor* t : {&kb->P1, &kb->P2, &kb->S, &kb->Ur, &kb->Vr, &kb->Sr}) rehome(*t, c1.sh);
  return s;
}

}  // namespace

std::vector<double> ctm_moves4(Env& e, ProjResult* keep) {
  ProjResult* k[4] = {nullptr, nullptr, nullptr, nullptr};
  if (keep)
    for (int d = 0; d < 4; ++d) k[d] = keep + d;
  std::vector<double> s;
  if (e.parallel_moves) {
    s = move_pair(e, 0, 1, k[0], k[1]);
    move_pair(e, 2, 3, k[2], k[3]);
  } else {
    s = ctm_move(e, 0, k[0]);
    for (int d = 1; d < 4; ++d) ctm_move(e, d, k[d]);
  }
  return s;
}

// ctmrg.jl:57-64
std::vector<double> rg_step(Env& e) {
  std::vector<double> s = ctm_moves4(e, nullptr);
  e.last_s = s;
  return s;
}

// ------------------------------------------------------------ observables
namespace {

// out[0..1] = tr(H rho) (complex), out[2..3] = tr(rho) (complex); FP64
__global__ void dm_trace_kernel(const double* rho, int rho_complex, const double2* H, int n, double* out) {
  double hr = 0, hi = 0, tr = 0, ti = 0;
  for (int t = threadIdx.x; t < n * n; t += 32) {
    int i = t % n, j = t / n;  // tr(H rho) = sum_ij H[i,j] rho[j,i]
    double rr, ri;
    int64_t idx = int64_t(j) + int64_t(i) * n;
    if (rho_complex) { rr = rho[2 * idx]; ri = rho[2 * idx + 1]; }
    else { rr = rho[idx]; ri = 0; }
    double2 h = H[i + int64_t(j) * n];
    hr += h.x * rr - h.y * ri;
    hi += h.x * ri + h.y * rr;
    if (i == j) { tr += rr; ti += ri; }
  }
  for (int o = 16; o; o >>= 1) {
    hr += __shfl_xor_sync(0xffffffffu, hr, o);
    hi += __shfl_xor_sync(0xffffffffu, hi, o);
    tr += __shfl_xor_sync(0xffffffffu, tr, o);
    ti += __shfl_xor_sync(0xffffffffu, ti, o);
  }
  if (threadIdx.x == 0) { out[0] = hr; out[1] = hi; out[2] = tr; out[3] = ti; }
}

}  // namespace

// traces of several (rho, H) pairs in one host round trip
std::vector<Traces> dm_traces(Ctx& c, const std::vector<std::pair<Tensor, Tensor>>& items) {
  const int n = int(items.size());
  double* d_out = reinterpret_cast<double*>(c.scal->p) + 64;
  IPEPS_CHECK(n * 4 <= 256, "dm_traces: too many items");
  for (int i = 0; i < n; ++i) {
    const Tensor& rho = items[i].first;
    const Tensor& H = items[i].second;
    int d2 = int(rho.dims[0]);
    IPEPS_CHECK(H.dims[0] == d2 && H.dt == DType::C128, "dm_traces: H must be complex d^2 x d^2");
    dm_trace_kernel<<<1, 32, 0, c.stream>>>(rho.f64(), rho.dt == DType::C128, static_cast<const double2*>(H.data()),
                                            d2, d_out + 4 * i);
    IPEPS_LAUNCH_CHECK();
    c.count(KFam::Reduce);
  }
  std::vector<double> h(4 * n);
  IPEPS_CUDA(cudaMemcpyAsync(h.data(), d_out, h.size() * 8, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  std::vector<Traces> r(n);
  for (int i = 0; i < n; ++i) {
    r[i].trH = {h[4 * i], h[4 * i + 1]};
    r[i].tr = {h[4 * i + 2], h[4 * i + 3]};
  }
  return r;
}

// evaluation.jl:15-29 with get_dms (only_gs) evaluation.jl:124-156
void gs_energy(Env& e, const Tensor& Hh, const Tensor& Hv, std::complex<double>* E, std::complex<double>* Na,
               bool ctx_precision) {
  // FP64 contractions unless the caller asks for the context's precision (the
  // mixed form's convergence energies of its 3xTF32 iterations); the traces are FP64
  const int prec = e.ctx->precision;
  Fp64Scope fp64(*e.ctx);
  if (ctx_precision) e.ctx->precision = prec;
  Ctx& c = *e.ctx;
  NTPolicy p{c};
  NT C1(e.Cs[0]), C2(e.Cs[1]), C3(e.Cs[2]), C4(e.Cs[3]);
  NT E1(e.Es[0]), E2(e.Es[1]), E3(e.Es[2]), E4(e.Es[3]);
  NT A(e.A), Ad(e.Ad);
  NT roh = get_dm_h(p, C1, C2, C3, C4, E1, E1, E2, E3, E3, E4, A, A, Ad, Ad);
  NT rov = get_dm_v(p, C1, C2, C3, C4, E1, E2, E2, E3, E4, E4, A, A, Ad, Ad);
  auto t = dm_traces(c, {{roh.c[0], Hh}, {rov.c[0], Hv}});
  const std::complex<double> Nh = t[0].tr, Nv = t[1].tr;
  *Na = (Nh + Nv) / 2.0;
  *E = t[0].trH / Nh + t[1].trH / Nv;
}

// evaluation.jl:31-45 (get_dms with only_gs = false)
double es_energy(Env& e, const Tensor& Hh, const Tensor& Hv) {
  Fp64Scope fp64(*e.ctx);
  Ctx& c = *e.ctx;
  IPEPS_CHECK(e.nested, "es_energy: no B set");
  NTPolicy p{c};
  NT C1 = e.all_C(0), C2 = e.all_C(1), C3 = e.all_C(2), C4 = e.all_C(3);
  NT E1 = e.all_E(0), E2 = e.all_E(1), E3 = e.all_E(2), E4 = e.all_E(3);
  NT A = e.all_A(), Ad = e.all_Ad();
  const double px = e.px, py = e.py;
  NT roh = get_dm_h(p, C1, nshift(c, C2, px), nshift(c, C3, px), C4, E1, nshift(c, E1, px), nshift(c, E2, px), E3,
                    nshift(c, E3, px), E4, A, nshift(c, A, px), Ad, nshift(c, Ad, px));
  NT rov = get_dm_v(p, C1, C2, nshift(c, C3, py), nshift(c, C4, py), E1, E2, nshift(c, E2, py), nshift(c, E3, py),
                    E4, nshift(c, E4, py), A, nshift(c, A, py), Ad, nshift(c, Ad, py));
  std::vector<std::pair<Tensor, Tensor>> items;
  std::vector<int> which;
  for (int i = 0; i < 4; ++i)
    if (roh.has(i)) { items.push_back({roh.c[i], Hh}); which.push_back(i); }
  for (int i = 0; i < 4; ++i)
    if (rov.has(i)) { items.push_back({rov.c[i], Hv}); which.push_back(4 + i); }
  auto t = dm_traces(c, items);
  std::complex<double> trHh[4] = {}, trHv[4] = {}, trh0 = 0, trv0 = 0;
  for (size_t i = 0; i < items.size(); ++i) {
    int w = which[i];
    if (w < 4) { trHh[w] = t[i].trH; if (w == 0) trh0 = t[i].tr; }
    else { trHv[w - 4] = t[i].trH; if (w == 4) trv0 = t[i].tr; }
  }
  const double Nh = trh0.real(), Nv = trv0.real();
  std::complex<double> E4v = trHh[3] / Nh + trHv[3] / Nv;
  return E4v.real();
}

static std::complex<double> scalar_of(Ctx& c, const Tensor& t) {
  double h[2] = {0, 0};
  IPEPS_CUDA(cudaMemcpyAsync(h, t.data(), t.dt == DType::F64 ? 8 : 16, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  return {h[0], t.dt == DType::F64 ? 0.0 : h[1]};
}

// ndm_Ad of get_tangent_basis (optim_es.jl:247-251): get_single_dm contracted with Ad
Tensor single_dm_Ad(Env& e) {
  Fp64Scope fp64(*e.ctx);
  Ctx& c = *e.ctx;
  NTPolicy p{c};
  NT n_dm = get_single_dm(p, NT(e.Cs[0]), NT(e.Cs[1]), NT(e.Cs[2]), NT(e.Cs[3]), NT(e.Es[0]), NT(e.Es[1]),
                          NT(e.Es[2]), NT(e.Es[3]));
  return tcon(c, n_dm.c[0], {-1, -2, -3, -4, 1, 2, 3, 4}, e.Ad, {1, 2, 3, 4, -5});
}

// evaluation.jl:47-59
std::complex<double> gs_norm(Env& e) {
  Fp64Scope fp64(*e.ctx);
  Ctx& c = *e.ctx;
  NTPolicy p{c};
  NT n_dm = get_single_dm(p, NT(e.Cs[0]), NT(e.Cs[1]), NT(e.Cs[2]), NT(e.Cs[3]), NT(e.Es[0]), NT(e.Es[1]),
                          NT(e.Es[2]), NT(e.Es[3]));
  Tensor ndm_Ad = tcon(c, n_dm.c[0], {-1, -2, -3, -4, 1, 2, 3, 4}, e.Ad, {1, 2, 3, 4, -5});
  Tensor nrm0 = tcon(c, ndm_Ad, {1, 2, 3, 4, 5}, e.A, {1, 2, 3, 4, 5});
  return scalar_of(c, nrm0);
}

// evaluation.jl:61-77
std::complex<double> all_norm(Env& e, Tensor* envB) {
  Fp64Scope fp64(*e.ctx);
  Ctx& c = *e.ctx;
  IPEPS_CHECK(e.nested, "all_norm: no B set");
  NTPolicy p{c};
  NT n_dm = get_single_dm(p, e.all_C(0), e.all_C(1), e.all_C(2), e.all_C(3), e.all_E(0), e.all_E(1), e.all_E(2),
                          e.all_E(3));
  NT ndm_A = ntcon(c, n_dm, {1, 2, 3, 4, -1, -2, -3, -4}, e.all_A(), {1, 2, 3, 4, -5});
  NT all = ntcon(c, ndm_A, {1, 2, 3, 4, 5}, e.all_Ad(), {1, 2, 3, 4, 5});
  std::complex<double> n1 = scalar_of(c, all.c[0]);
  IPEPS_CHECK(ndm_A.has(1), "all_norm: empty B slot");
  if (envB) {
    *envB = clone(c, to_complex(c, ndm_A.c[1]));
    scale(c, *envB, cplx((1.0 / n1).real(), (1.0 / n1).imag()));
  }
  Tensor Nb = tcon(c, ndm_A.c[1], {1, 2, 3, 4, 5}, e.Bd, {1, 2, 3, 4, 5});
  return scalar_of(c, Nb) / n1;
}

// evaluation.jl:339-356 (get_gs_energy_4x4): <H_plaquette> / <1> of the
// 2 x 2 cluster, H given as the MPO [s1, s2, s3, s4] of get_local_h
std::complex<double> gs_energy_4x4(Env& e, const H4& h) {
  Fp64Scope fp64(*e.ctx);
  Ctx& c = *e.ctx;
  NTPolicy p{c};
  Arr4<NTPolicy> s{NT(h[0]), NT(h[1]), NT(h[2]), NT(h[3])};
  NT A(e.A), Ad(e.Ad);
  Arr4<NTPolicy> As{A, A, A, A}, Ads{Ad, Ad, Ad, Ad};
  Arr4<NTPolicy> op = get_op_Ad4(p, s, Ads);
  NT C1(e.Cs[0]), C2(e.Cs[1]), C3(e.Cs[2]), C4(e.Cs[3]);
  NT E1(e.Es[0]), E2(e.Es[1]), E3(e.Es[2]), E4(e.Es[3]);
  auto en = energy_norm_4x4(p, C1, C2, C3, C4, E1, E1, E2, E2, E3, E3, E4, E4, As, Ads, op);
  return scalar_of(c, en[0].c[0]) / scalar_of(c, en[1].c[0]);
}

// evaluation.jl:358-398 (get_es_energy_4x4): component 4 of the nested
// plaquette energy over component 1 of the norm
std::complex<double> es_energy_4x4(Env& e, const H4& h) {
  Fp64Scope fp64(*e.ctx);
  Ctx& c = *e.ctx;
  IPEPS_CHECK(e.nested, "es_energy_4x4: no B set");
  NTPolicy p{c};
  Arr4<NTPolicy> s{NT(h[0]), NT(h[1]), NT(h[2]), NT(h[3])};
  Arr4<NTPolicy> C{e.all_C(0), e.all_C(1), e.all_C(2), e.all_C(3)};
  Arr4<NTPolicy> E{e.all_E(0), e.all_E(1), e.all_E(2), e.all_E(3)};
  auto sh = [&](const NT& x, double ph) { return nshift(c, x, ph); };
  auto en = es_plaquette(p, sh, s, e.all_A(), e.all_Ad(), C, E, e.px, e.py);
  IPEPS_CHECK(en[0].has(3), "es_energy_4x4: empty fourth component");
  return scalar_of(c, en[0].c[3]) / scalar_of(c, en[1].c[0]);
}

namespace {

// Moves the counters and timing records of `from` into `to`.
void merge_stats(Ctx& to, Ctx& from) {
  for (int f = 0; f < int(KFam::Count); ++f) {
    to.stats[f].launches += from.stats[f].launches;
    to.stats[f].flops += from.stats[f].flops;
    to.stats[f].bytes += from.stats[f].bytes;
    to.prof_stats[f].launches += from.prof_stats[f].launches;
    to.prof_stats[f].flops += from.prof_stats[f].flops;
    to.prof_stats[f].bytes += from.prof_stats[f].bytes;
  }
  from.stats = {};
  from.prof_stats = {};
  to.jacobi_sweeps += from.jacobi_sweeps;
  to.projector_calls += from.projector_calls;
  to.projector_extra_passes += from.projector_extra_passes;
  to.series_cap_hits += from.series_cap_hits;
  to.series_terms += from.series_terms;
  to.series_retries += from.series_retries;
  to.resid_misses += from.resid_misses;
  from.jacobi_sweeps = from.projector_calls = from.projector_extra_passes = from.series_cap_hits = 0;
  from.series_terms = from.series_retries = from.resid_misses = 0;
  for (auto& r : from.prof_rec) to.prof_rec.push_back(r);
  from.prof_rec.clear();
}

// The convergence value of run_ctm: get_gs_energy (mode 0) or
// get_es_energy / get_all_norm (mode 2).
std::complex<double> conv_value(Env& e, int conv_mode, const Tensor* Hh, const Tensor* Hv, const H4* h4) {
  if (conv_mode == kConvEnergy) {
    std::complex<double> E, Na;
    gs_energy(e, *Hh, *Hv, &E, &Na, true);
    return E;
  }
  if (conv_mode == kConvEnergy4x4) return gs_energy_4x4(e, *h4);
  if (conv_mode == kConvEs4x4) return es_energy_4x4(e, *h4) / all_norm(e, nullptr);
  return es_energy(e, *Hh, *Hv) / all_norm(e, nullptr);
}

// One convergence evaluation in flight on the evaluation context, from its own
// host thread, on a snapshot of the environment after iteration `iter`.  The
// snapshot also keeps every tensor the evaluation reads alive until finish().
struct PendingConv {
  Env& e;
  int conv_mode;
  const Tensor* Hh;
  const Tensor* Hv;
  const H4* h4;
  bool active = false;
  std::thread th;
  std::complex<double> val;
  std::exception_ptr err;
  Env snap;
  std::vector<double> s;
  uint64_t rng1 = 0, rng2 = 0;
  int iter = 0;

  PendingConv(Env& env, int mode, const Tensor* hh, const Tensor* hv, const H4* h)
      : e(env), conv_mode(mode), Hh(hh), Hv(hv), h4(h) {}
  ~PendingConv() {
    if (th.joinable()) th.join();
  }
  void launch(int it, const std::vector<double>& sp) {
    Ctx& c1 = *e.ctx;
    if (!e.aux_eval) e.aux_eval = std::make_shared<Ctx>(c1.device);
    Ctx& c3 = *e.aux_eval;
    c3.prof = c1.prof;
    c3.d_status = c1.d_status;
    c3.precision = c1.precision;  // the energy of an iteration in that iteration's precision
    snap = e;
    s = sp;
    iter = it;
    err = nullptr;
    rng1 = c1.rng_counter;
    rng2 = e.aux ? e.aux->rng_counter : 0;
    Env ev = e;
    ev.ctx = &c3;
    ev.aux.reset();
    ev.aux_eval.reset();
    cudaEvent_t ev0 = c1.take_event();
    IPEPS_CUDA(cudaEventRecord(ev0, c1.stream));
    IPEPS_CUDA(cudaStreamWaitEvent(c3.stream, ev0, 0));
    c1.ev_pool.push_back(ev0);
    active = true;
    th = std::thread([this, &c3, ev]() mutable {
      try {
        IPEPS_CUDA(cudaSetDevice(c3.device));
        val = conv_value(ev, conv_mode, Hh, Hv, h4);
      } catch (...) {
        err = std::current_exception();
      }
    });
  }
  std::complex<double> finish() {
    Ctx& c1 = *e.ctx;
    Ctx& c3 = *e.aux_eval;
    th.join();
    active = false;
    // later frees of the snapshot's buffers (main stream) follow the evaluation's reads
    cudaEvent_t ev1 = c1.take_event();
    IPEPS_CUDA(cudaEventRecord(ev1, c3.stream));
    IPEPS_CUDA(cudaStreamWaitEvent(c1.stream, ev1, 0));
    c1.ev_pool.push_back(ev1);
    merge_stats(c1, c3);
    if (err) std::rethrow_exception(err);
    return val;
  }
  // back to the environment the evaluation saw (drops a speculative iteration)
  void roll_back() {
    e.Cs = snap.Cs;
    e.Es = snap.Es;
    e.B_Cs = snap.B_Cs;
    e.Bd_Cs = snap.Bd_Cs;
    e.BB_Cs = snap.BB_Cs;
    e.B_Es = snap.B_Es;
    e.Bd_Es = snap.Bd_Es;
    e.BB_Es = snap.BB_Es;
    for (int d = 0; d < 4; ++d) e.cache[d] = snap.cache[d];
    e.last_s = snap.last_s;
    e.ctx->rng_counter = rng1;
    if (e.aux) e.aux->rng_counter = rng2;
  }
};

}  // namespace

// ctmrg.jl:1-55
int run_ctm(Env& e, int conv_mode, const Tensor* Hh, const Tensor* Hv, double* last_diff, bool* converged,
            const H4* h4) {
  const bool by_value = conv_mode != kConvSpectrum;
  IPEPS_CHECK(!by_value || ((conv_mode == kConvEnergy4x4 || conv_mode == kConvEs4x4) ? h4 != nullptr
                                                                                    : (Hh && Hv)),
              "run_ctm: Hamiltonian missing for the convergence criterion");
  std::vector<double> diffs{1.0};
  std::complex<double> conv = 1.0;
  std::vector<double> conv_s{1.0};
  e.log.clear();
  int i = 1;
  bool done = false;
  // Mixed form: 3xTF32 contractions while the environment is still moving, then
  // FP64 for the last polish_iters iterations (or from the point where the
  // change per iteration drops below polish_tol * rg_tol, i.e. close to the
  // requested convergence), and convergence is accepted only after that many
  // FP64 iterations.  The CTMRG map contracts errors, so the FP32-level errors
  // of the mixed iterations decay in the FP64 ones.  With rg_tol = 0 (a fixed
  // number of iterations) only the last polish_iters iterations run in FP64.
  // With a tolerance, the switch also happens when the mixed iterations stall
  // close to convergence: the change per iteration is below 1e-6 of the
  // objective and has not halved against either of the two iterations before
  // (the FP32-level floor of the 3xTF32 products can sit above
  // polish_tol * rg_tol, and the run would reach max_iter unconverged).
  auto stalled = [&]() {
    const size_t n = diffs.size();
    return e.prm.rg_tol > 0 && n >= 4 && diffs[n - 1] < 1e-6 * std::max(std::abs(conv), 1e-12) &&
           diffs[n - 1] > 0.5 * std::min(diffs[n - 2], diffs[n - 3]);
  };
  Ctx& c = *e.ctx;
  const int prec0 = c.precision;
  const bool polish = (prec0 == kPrecMixed) && e.prm.polish_iters > 0;
  const int polish_start = polish ? std::max(1, e.prm.max_iter - e.prm.polish_iters + 1) : 1 << 30;
  int fp64_done = 0;
  struct Restore {
    Ctx& c;
    int p;
    ~Restore() { c.precision = p; }
  } restore{c, prec0};
  if (by_value && e.parallel_moves) {
    // Pipelined: the energy of iteration i is evaluated while iteration i+1
    // runs.  When iteration i turns out converged, iteration i+1 is rolled
    // back, so the returned environment and log are those of the sequential
    // loop.  In the mixed form the switch to FP64 sees the change per
    // iteration one iteration later than the sequential loop does.
    PendingConv pc(e, conv_mode, Hh, Hv, h4);
    std::vector<int> fp64_upto(size_t(std::max(e.prm.max_iter, 0)) + 2, 0);
    auto record = [&](std::complex<double> v) {
      const std::complex<double> old = conv;
      conv = v;
      diffs.push_back(std::abs(conv - old));
      CtmLogEntry le{pc.iter, diffs.back(), conv.real(), conv.imag(), int(pc.s.size())};
      e.log.push_back(le);
      return pc.iter >= e.prm.min_iter && diffs.back() < e.prm.rg_tol &&
             (!polish || fp64_upto[pc.iter] >= e.prm.polish_iters);
    };
    int last = 0;
    for (; i <= e.prm.max_iter; ++i) {
      if (polish && c.precision != kPrecFP64 &&
          (i >= polish_start || diffs.back() < e.prm.polish_tol * e.prm.rg_tol || stalled()))
        c.precision = kPrecFP64;
      std::vector<double> s = rg_step(e);
      if (polish && c.precision == kPrecFP64) fp64_done++;
      fp64_upto[i] = fp64_done;
      if (pc.active && record(pc.finish())) {
        pc.roll_back();
        done = true;
        last = pc.iter;
        break;
      }
      pc.launch(i, s);
    }
    if (!done && pc.active) {
      done = record(pc.finish());
      last = pc.iter;
    }
    if (last_diff) *last_diff = diffs.back();
    if (converged) *converged = done;
    return done ? last : e.prm.max_iter;
  }
  for (; i <= e.prm.max_iter; ++i) {
    if (polish && c.precision != kPrecFP64 &&
        (i >= polish_start || diffs.back() < e.prm.polish_tol * e.prm.rg_tol || (by_value && stalled())))
      c.precision = kPrecFP64;
    std::vector<double> s = rg_step(e);
    if (polish && c.precision == kPrecFP64) fp64_done++;
    CtmLogEntry le{i, 0, 0, 0, int(s.size())};
    if (by_value) {
      std::complex<double> old = conv;
      conv = conv_value(e, conv_mode, Hh, Hv, h4);
      diffs.push_back(std::abs(conv - old));
      le.obj_re = conv.real();
      le.obj_im = conv.imag();
    } else {
      std::vector<double> old = conv_s;
      conv_s = s;
      if (conv_s.size() == old.size()) {
        double acc = 0;
        for (size_t j = 0; j < s.size(); ++j) acc += (conv_s[j] - old[j]) * (conv_s[j] - old[j]);
        diffs.push_back(std::sqrt(acc));
      }
    }
    le.diff = diffs.back();
    e.log.push_back(le);
    if (i >= e.prm.min_iter && diffs.back() < e.prm.rg_tol && (!polish || fp64_done >= e.prm.polish_iters)) {
      done = true;
      break;
    }
  }
  if (last_diff) *last_diff = diffs.back();
  if (converged) *converged = done;
  return done ? i : e.prm.max_iter;
}

}  // namespace ipeps
