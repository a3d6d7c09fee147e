// Pullback of the nested (excited-state) CTMRG with respect to B:
// get_es_grad / run_es (src/optimize/optim_es.jl:167-210).
//
// In the nested move the projectors are built from the plain environment
// (ctmrg.jl:122-134), which does not depend on B, and the renormalisation
// factor is max|component 1| (nested_tensor.jl:70-75), also independent of B.
// Both are therefore constants of the B-pullback: only the product-rule
// contractions (nested_tensor.jl:77-92), the phase shifts (nested_tensor.jl:65)
// and get_es_energy (evaluation.jl:31-45) are differentiated.  Complex
// cotangents follow the convention dL/dRe + i dL/dIm (Zygote's); B enters as
// B and Bd = conj(B), so gH = g_B + conj(g_Bd).
#include "ad.cuh"
#include "linalg.cuh"
#include "moves.cuh"

#include <cmath>

namespace ipeps {
namespace {

__global__ void real_part_kernel(const double2* x, double* y, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[i] = x[i].x;
}

unsigned gridn(Ctx& c, int64_t n) {
  return unsigned(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, int64_t(c.sm_count) * 8)));
}

Tensor real_part(Ctx& c, const Tensor& x) {
  if (x.dt == DType::F64) return x;
  Tensor y = c.alloc(DType::F64, x.shape());
  real_part_kernel<<<gridn(c, x.numel()), 256, 0, c.stream>>>(static_cast<const double2*>(x.data()), y.f64(),
                                                              x.numel());
  IPEPS_LAUNCH_CHECK();
  return y;
}

// cotangent of a tensor of dtype `dt` from a possibly complex gradient
Tensor as_dtype(Ctx& c, const Tensor& g, DType dt) {
  if (g.dt == dt) return g;
  return dt == DType::F64 ? real_part(c, g) : to_complex(c, g);
}

AV ad_add(Tape& tp, const AV& a, const AV& b) {
  Ctx& c = tp.ctx();
  if (a.t.empty()) return b;
  if (b.t.empty()) return a;
  DType dt = (a.t.dt == DType::C128 || b.t.dt == DType::C128) ? DType::C128 : DType::F64;
  AV out{clone(c, a.t.dt == dt ? a.t : to_complex(c, a.t)), -1};
  axpy(c, cplx(1), b.t, out.t);
  if (a.id < 0 && b.id < 0) return out;
  out.id = tp.newid();
  const int ia = a.id, ib = b.id, io = out.id;
  const DType da = a.t.dt, db = b.t.dt;
  const std::vector<int64_t> sa = a.t.shape(), sb = b.t.shape();
  tp.push([&tp, ia, ib, io, da, db, sa, sb]() {
    const Tensor& g = tp.grad(io);
    if (g.empty()) return;
    Ctx& c = tp.ctx();
    if (ia >= 0) tp.acc(ia, as_dtype(c, g, da).reshape(sa));
    if (ib >= 0) tp.acc(ib, as_dtype(c, g, db).reshape(sb));
  });
  return out;
}

// y = s x (s complex constant); dx = conj(s) dy
AV ad_scale_c(Tape& tp, const AV& a, double re, double im) {
  Ctx& c = tp.ctx();
  if (a.t.empty()) return a;
  AV out{clone(c, to_complex(c, a.t)), -1};
  scale(c, out.t, cplx(re, im));
  if (a.id < 0) return out;
  out.id = tp.newid();
  const int ia = a.id, io = out.id;
  const DType da = a.t.dt;
  tp.push([&tp, ia, io, re, im, da]() {
    const Tensor& g = tp.grad(io);
    if (g.empty()) return;
    Ctx& c = tp.ctx();
    Tensor gx = clone(c, to_complex(c, g));
    scale(c, gx, cplx(re, -im));
    tp.acc(ia, as_dtype(c, gx, da));
  });
  return out;
}

// y = x / m with m a device scalar that does not depend on the variables
AV ad_div_const(Tape& tp, const AV& a, const Tensor& m) {
  Ctx& c = tp.ctx();
  if (a.t.empty()) return a;
  AV out{clone(c, a.t), -1};
  scale_inv(c, out.t, m.f64());
  if (a.id < 0) return out;
  out.id = tp.newid();
  const int ia = a.id, io = out.id;
  tp.push([&tp, ia, io, m]() {
    const Tensor& g = tp.grad(io);
    if (g.empty()) return;
    Ctx& c = tp.ctx();
    Tensor gx = clone(c, g);
    scale_inv(c, gx, m.f64());
    tp.acc(ia, gx);
  });
  return out;
}

// value of a one-element (0-d) tensor on the host
std::complex<double> host_scalar(Ctx& c, const Tensor& t) {
  double h[2] = {0, 0};
  IPEPS_CUDA(cudaMemcpyAsync(h, t.data(), t.dt == DType::F64 ? 8 : 16, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  return {h[0], t.dt == DType::F64 ? 0.0 : h[1]};
}

// nested autodiff value: 4 components, an empty tensor is EmptyT
struct NAV {
  std::array<AV, 4> c;
  bool nested = false;
  bool has(int i) const { return !c[i].t.empty(); }
};

struct NADPolicy {
  using T = NAV;
  Tape& tp;
  T tc(const T& a, const std::vector<int>& la, const T& b, const std::vector<int>& lb) {
    T r;
    if (!a.nested && !b.nested) {
      r.c[0] = ad_tcon(tp, a.c[0], la, b.c[0], lb);
      return r;
    }
    r.nested = true;
    if (a.nested && b.nested) {  // nested_tensor.jl:77-88
      static const int pairs[4][4][2] = {{{0, 0}, {-1, -1}, {-1, -1}, {-1, -1}},
                                         {{0, 1}, {1, 0}, {-1, -1}, {-1, -1}},
                                         {{0, 2}, {2, 0}, {-1, -1}, {-1, -1}},
                                         {{0, 3}, {3, 0}, {1, 2}, {2, 1}}};
      for (int o = 0; o < 4; ++o)
        for (int p = 0; p < 4; ++p) {
          const int i = pairs[o][p][0], j = pairs[o][p][1];
          if (i < 0 || !a.has(i) || !b.has(j)) continue;
          r.c[o] = ad_add(tp, r.c[o], ad_tcon(tp, a.c[i], la, b.c[j], lb));
        }
    } else if (a.nested) {
      for (int i = 0; i < 4; ++i)
        if (a.has(i)) r.c[i] = ad_tcon(tp, a.c[i], la, b.c[0], lb);
    } else {
      for (int i = 0; i < 4; ++i)
        if (b.has(i)) r.c[i] = ad_tcon(tp, a.c[0], la, b.c[i], lb);
    }
    return r;
  }
  T rs(const T& a, const std::vector<int64_t>& s) {
    T r = a;
    for (int i = 0; i < 4; ++i)
      if (a.has(i)) r.c[i] = ad_reshape(tp, a.c[i], s);
    return r;
  }
  T pm(const T& a, const std::vector<int>& perm) {
    T r = a;
    for (int i = 0; i < 4; ++i)
      if (a.has(i)) r.c[i] = ad_permute(tp, a.c[i], perm);
    return r;
  }
  T mm(const T& a, const T& b) { return tc(a, {-1, 1}, b, {1, -2}); }
  int64_t dim(const T& a, int i) const { return a.c[0].t.dims[i]; }
};

// nested_tensor.jl:65
NAV nav_shift(Tape& tp, const NAV& a, double phi) {
  if (!a.nested) return a;
  NAV r = a;
  const double cs = std::cos(phi), sn = std::sin(phi);
  if (a.has(1)) r.c[1] = ad_scale_c(tp, a.c[1], cs, sn);
  if (a.has(2)) r.c[2] = ad_scale_c(tp, a.c[2], cs, -sn);
  return r;
}

// nested_tensor.jl:70-75 with the factor max|component 1| held constant
NAV nav_renorm(Tape& tp, const NAV& a) {
  Ctx& c = tp.ctx();
  Tensor m = c.alloc(DType::F64, {1});
  maxabs(c, a.c[0].t, m.f64());
  NAV r = a;
  for (int i = 0; i < 4; ++i)
    if (a.has(i)) r.c[i] = ad_div_const(tp, a.c[i], m);
  return r;
}

struct EsCk {
  std::array<std::array<Tensor, 4>, 4> C, E;  // [slot][component]
  std::array<Tensor, 4> P1, P2;               // per direction
};

NAV leaf_nav(Tape& tp, const std::array<Tensor, 4>& comps) {
  NAV r;
  r.nested = true;
  r.c[0] = tp.constant(comps[0]);  // the plain environment does not depend on B
  for (int i = 1; i < 4; ++i)
    if (!comps[i].empty()) r.c[i] = tp.leaf(comps[i]);
  return r;
}

}  // namespace

double es_energy_grad(Env& e, const Tensor& Hh, const Tensor& Hv, int ad_iters, Tensor* gB, const H4* h4) {
  Ctx& c = *e.ctx;
  Fp64Scope fp64_all(c);  // the pullback in FP64 in both forms, as in energy_grad
  IPEPS_CHECK(e.nested, "es_energy_grad: no B set");
  // the checkpointed moves keep P1/P2 only (no projector adjoint: the projectors are B-independent)
  struct KeepAdj {
    Env& e;
    bool v;
    ~KeepAdj() { e.keep_adjoint = v; }
  } keep_adj{e, e.keep_adjoint};
  e.keep_adjoint = false;
  auto conv_of = [&]() {
    return h4 ? es_energy_4x4(e, *h4) / all_norm(e, nullptr) : es_energy(e, Hh, Hv) / all_norm(e, nullptr);
  };
  auto slots = [&](std::array<std::array<Tensor, 4>, 4>& C, std::array<std::array<Tensor, 4>, 4>& E) {
    for (int s = 0; s < 4; ++s) {
      C[s] = {e.Cs[s], e.B_Cs[s], e.Bd_Cs[s], e.BB_Cs[s]};
      E[s] = {e.Es[s], e.B_Es[s], e.Bd_Es[s], e.BB_Es[s]};
    }
  };
  // forward: ad_iters nested iterations, checkpointing every slot and the projectors
  std::vector<EsCk> ck;
  {
    std::complex<double> conv = 1.0;
    for (int i = 1; i <= ad_iters; ++i) {
      EsCk k;
      slots(k.C, k.E);
      std::array<ProjResult, 4> pr;
      ctm_moves4(e, pr.data());
      for (int d = 0; d < 4; ++d) {
        k.P1[d] = pr[d].P1;
        k.P2[d] = pr[d].P2;
      }
      ck.push_back(std::move(k));
      // run_ctm's early exit with conv_fun = get_es_energy / get_all_norm (optim_es.jl:200)
      if (e.prm.min_iter < ad_iters && i < ad_iters) {
        std::complex<double> v = conv_of();
        const double diff = std::abs(v - conv);
        conv = v;
        if (i >= e.prm.min_iter && diff < e.prm.rg_tol) break;
      }
    }
  }
  std::array<std::array<Tensor, 4>, 4> gC, gE;  // [slot][component]
  Tensor gBacc, gBdacc;
  double Eres = 0;
  auto add_to = [&](Tensor& acc, const Tensor& g) {
    if (g.empty()) return;
    if (acc.empty()) acc = clone(c, to_complex(c, g));
    else axpy(c, cplx(1), to_complex(c, g), acc);
  };
  // get_es_energy on a tape (evaluation.jl:31-45): real part of component 4
  {
    Fp64Scope fp64(c);  // the energy and its seed in FP64 in both forms
    Tape tp(c);
    NADPolicy p{tp};
    std::array<std::array<Tensor, 4>, 4> Cn, En;
    slots(Cn, En);
    NAV C[4], E[4], leafC[4], leafE[4];
    for (int s = 0; s < 4; ++s) {
      leafC[s] = C[s] = leaf_nav(tp, Cn[s]);
      leafE[s] = E[s] = leaf_nav(tp, En[s]);
    }
    NAV A, Ad;
    A.nested = Ad.nested = true;
    A.c[0] = tp.constant(e.A);
    AV Bl = tp.leaf(e.B);
    A.c[1] = Bl;
    Ad.c[0] = tp.constant(e.Ad);
    AV Bdl = tp.leaf(e.Bd);
    Ad.c[2] = Bdl;
    const double px = e.px, py = e.py;
    auto sh = [&](const NAV& x, double ph) { return nav_shift(tp, x, ph); };
    if (h4) {
      // get_es_energy_4x4 (evaluation.jl:358-398): Re(e4 / n1); n1 (the plain
      // norm) does not depend on B, so the seed of e4 is conj(1 / n1)
      Arr4<NADPolicy> sv, Cv{C[0], C[1], C[2], C[3]}, Ev{E[0], E[1], E[2], E[3]};
      for (int k = 0; k < 4; ++k) sv[k].c[0] = tp.constant((*h4)[k]);
      auto en = es_plaquette(p, sh, sv, A, Ad, Cv, Ev, px, py);
      IPEPS_CHECK(en[0].has(3) && en[1].has(0), "es_energy_grad: empty plaquette component");
      const std::complex<double> e4 = host_scalar(c, en[0].c[3].t), n1 = host_scalar(c, en[1].c[0].t);
      Eres = (e4 / n1).real();
      const std::complex<double> w = std::conj(1.0 / n1);
      Tensor sd = c.alloc(DType::C128, en[0].c[3].t.shape());
      const double hw[2] = {w.real(), w.imag()};
      IPEPS_CUDA(cudaMemcpyAsync(sd.data(), hw, 16, cudaMemcpyHostToDevice, c.stream));
      c.sync();
      tp.acc(en[0].c[3].id, as_dtype(c, sd, en[0].c[3].t.dt));
    } else {
    NAV roh = get_dm_h(p, C[0], sh(C[1], px), sh(C[2], px), C[3], E[0], sh(E[0], px), sh(E[1], px), E[2],
                       sh(E[2], px), E[3], A, sh(A, px), Ad, sh(Ad, px));
    NAV rov = get_dm_v(p, C[0], C[1], sh(C[2], py), sh(C[3], py), E[0], E[1], sh(E[1], py), sh(E[2], py), E[3],
                       sh(E[3], py), A, sh(A, py), Ad, sh(Ad, py));
    IPEPS_CHECK(roh.has(3) && rov.has(3), "es_energy_grad: empty fourth component");
    auto t = dm_traces(c, {{roh.c[0].t, Hh}, {rov.c[0].t, Hv}, {roh.c[3].t, Hh}, {rov.c[3].t, Hv}});
    const double Nh = t[0].tr.real(), Nv = t[1].tr.real();
    Eres = (t[2].trH / Nh + t[3].trH / Nv).real();
    // seed: d Re tr(H rho4) / d rho4 = conj(H)^T (cotangent convention), divided by N
    auto seed = [&](const Tensor& H, const AV& rho, double N) {
      const int d2 = int(H.dims[0]);
      std::vector<double> hH(size_t(d2) * d2 * 2), g(size_t(d2) * d2 * 2);
      IPEPS_CUDA(cudaMemcpyAsync(hH.data(), H.data(), hH.size() * 8, cudaMemcpyDeviceToHost, c.stream));
      c.sync();
      for (int a = 0; a < d2; ++a)
        for (int b = 0; b < d2; ++b) {
          // g[a,b] = conj(H[b,a]) / N
          g[2 * (a + size_t(b) * d2)] = hH[2 * (b + size_t(a) * d2)] / N;
          g[2 * (a + size_t(b) * d2) + 1] = -hH[2 * (b + size_t(a) * d2) + 1] / N;
        }
      Tensor gt = c.alloc(DType::C128, {d2, d2});
      IPEPS_CUDA(cudaMemcpyAsync(gt.data(), g.data(), g.size() * 8, cudaMemcpyHostToDevice, c.stream));
      return as_dtype(c, gt, rho.t.dt);
    };
    tp.acc(roh.c[3].id, seed(Hh, roh.c[3], Nh));
    tp.acc(rov.c[3].id, seed(Hv, rov.c[3], Nv));
    }
    tp.backward();
    for (int s = 0; s < 4; ++s)
      for (int i = 1; i < 4; ++i) {
        gC[s][i] = leafC[s].c[i].id >= 0 ? tp.grad(leafC[s].c[i].id) : Tensor();
        gE[s][i] = leafE[s].c[i].id >= 0 ? tp.grad(leafE[s].c[i].id) : Tensor();
      }
    add_to(gBacc, tp.grad(Bl.id));
    add_to(gBdacc, tp.grad(Bdl.id));
  }
  // reverse over the iterations; projectors and normalisations are constants
  for (int it = int(ck.size()) - 1; it >= 0; --it) {
    Tape tp(c);
    NADPolicy p{tp};
    Arr4<NADPolicy> C, E;
    NAV leafC[4], leafE[4];
    for (int s = 0; s < 4; ++s) {
      leafC[s] = C[s] = leaf_nav(tp, ck[it].C[s]);
      leafE[s] = E[s] = leaf_nav(tp, ck[it].E[s]);
    }
    NAV A, Ad;
    A.nested = Ad.nested = true;
    A.c[0] = tp.constant(e.A);
    AV Bl = tp.leaf(e.B);
    A.c[1] = Bl;
    Ad.c[0] = tp.constant(e.Ad);
    AV Bdl = tp.leaf(e.Bd);
    Ad.c[2] = Bdl;
    for (int d = 0; d < 4; ++d) {
      NAV P1, P2;
      P1.c[0] = tp.constant(ck[it].P1[d]);
      P2.c[0] = tp.constant(ck[it].P2[d]);
      Projected<NADPolicy> np = project(p, d, C, E, A, Ad, P1, P2);
      int ia, ib, ie;
      move_slots(d, &ia, &ib, &ie);
      const double phi = (d == 0) ? -e.px : (d == 1) ? e.px : (d == 2) ? -e.py : e.py;
      C[ia] = nav_shift(tp, nav_renorm(tp, np.Ca), phi);
      C[ib] = nav_shift(tp, nav_renorm(tp, np.Cb), phi);
      E[ie] = nav_shift(tp, nav_renorm(tp, np.E), phi);
    }
    for (int s = 0; s < 4; ++s)
      for (int i = 1; i < 4; ++i) {
        if (C[s].has(i) && C[s].c[i].id >= 0) tp.acc(C[s].c[i].id, gC[s][i]);
        if (E[s].has(i) && E[s].c[i].id >= 0) tp.acc(E[s].c[i].id, gE[s][i]);
      }
    tp.backward();
    for (int s = 0; s < 4; ++s)
      for (int i = 1; i < 4; ++i) {
        gC[s][i] = leafC[s].c[i].id >= 0 ? tp.grad(leafC[s].c[i].id) : Tensor();
        gE[s][i] = leafE[s].c[i].id >= 0 ? tp.grad(leafE[s].c[i].id) : Tensor();
      }
    add_to(gBacc, tp.grad(Bl.id));
    add_to(gBdacc, tp.grad(Bdl.id));
  }
  // B enters as B and Bd = conj(B): gH = g_B + conj(g_Bd)
  Tensor g = gBacc.empty() ? c.zeros(DType::C128, e.B.shape()) : gBacc;
  if (!gBdacc.empty()) axpy(c, cplx(1), conj(c, gBdacc), g);
  *gB = g;
  return Eres;
}

void wp_grad(Env& e, const std::array<Tensor, 4>& wp, int site, const Tensor& B, std::complex<double>* wp_value,
             std::complex<double>* norm, Tensor* gH, Tensor* gN) {
  Ctx& c = *e.ctx;
  IPEPS_CHECK(site >= 1 && site <= 4, "wp_grad: site must be 1..4");
  IPEPS_CHECK(B.shape() == e.A.shape(), "wp_grad: B must have the shape of A");
  Fp64Scope fp64(c);
  auto cx = [&](const Tensor& t) { return t.dt == DType::C128 ? t : to_complex(c, t); };
  const Tensor Ac = cx(e.A), Adc = conj(c, Ac), Bc = cx(B), Bdc = conj(c, Bc);
  std::array<Tensor, 4> Cc, Ec, sc;
  for (int k = 0; k < 4; ++k) {
    Cc[k] = cx(e.Cs[k]);
    Ec[k] = cx(e.Es[k]);
    sc[k] = cx(wp[k]);
  }
  // one tape per seed: the operator value (gH), then the norm (gN)
  for (int pass = 0; pass < 2; ++pass) {
    Tape tp(c);
    ADPolicy p{tp};
    AV Bl = tp.leaf(Bc), Bdl = tp.leaf(Bdc);
    Arr4<ADPolicy> As, Ads, sv;
    for (int k = 0; k < 4; ++k) {
      As[k] = tp.constant(Ac);
      Ads[k] = tp.constant(Adc);
      sv[k] = tp.constant(sc[k]);
    }
    As[site - 1] = Bl;
    Ads[site - 1] = Bdl;
    AV C[4], E[4];
    for (int k = 0; k < 4; ++k) {
      C[k] = tp.constant(Cc[k]);
      E[k] = tp.constant(Ec[k]);
    }
    Arr4<ADPolicy> op = get_op_Ad4(p, sv, Ads);
    auto en = energy_norm_4x4(p, C[0], C[1], C[2], C[3], E[0], E[0], E[1], E[1], E[2], E[2], E[3], E[3], As, Ads, op);
    if (pass == 0) {
      if (wp_value) *wp_value = host_scalar(c, en[0].t);
      if (norm) *norm = host_scalar(c, en[1].t);
    }
    // L = Re(y): the cotangent of y is 1
    Tensor sd = c.alloc(DType::C128, en[pass].t.shape());
    const double one[2] = {1.0, 0.0};
    IPEPS_CUDA(cudaMemcpyAsync(sd.data(), one, 16, cudaMemcpyHostToDevice, c.stream));
    c.sync();
    tp.acc(en[pass].id, as_dtype(c, sd, en[pass].t.dt));
    tp.backward();
    // B enters as B and conj(B): the gradient is g_B + conj(g_Bd)
    Tensor g = tp.grad(Bl.id).empty() ? c.zeros(DType::C128, B.shape()) : clone(c, cx(tp.grad(Bl.id)));
    if (!tp.grad(Bdl.id).empty()) axpy(c, cplx(1), conj(c, cx(tp.grad(Bdl.id))), g);
    (pass == 0 ? *gH : *gN) = g;
  }
}

}  // namespace ipeps
