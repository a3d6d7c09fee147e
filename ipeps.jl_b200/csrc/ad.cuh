// Reverse-mode differentiation of the CTMRG move and the energy.
//
// A Tape records the engine's primitives (tcon, reshape, permutedims, matrix
// product, max-abs renormalisation, projector) with their backward rules;
// moves.cuh runs the same contraction sequences on AV values through
// ADPolicy.  The projector's backward is the reference's broadened full-SVD
// adjoint (autodiff.jl:41-74) restricted to the truncated SVD it feeds.
#pragma once
#include "ctm.cuh"

#include <functional>

namespace ipeps {

// autodiff value: tensor + tape slot (-1: constant)
struct AV {
  Tensor t;
  int id = -1;
};

class Tape {
 public:
  explicit Tape(Ctx& c) : c_(c) {}
  Ctx& ctx() { return c_; }
  AV leaf(const Tensor& t) { return AV{t, newid()}; }
  AV constant(const Tensor& t) { return AV{t, -1}; }
  int newid() {
    g_.emplace_back();
    return int(g_.size()) - 1;
  }
  void push(std::function<void()> f) { ops_.push_back(std::move(f)); }
  // g[id] += gt (reshaped to gt's own numel; shapes must agree in element count)
  void acc(int id, const Tensor& gt);
  const Tensor& grad(int id) const { return g_[id]; }
  void backward();

 private:
  Ctx& c_;
  std::vector<Tensor> g_;
  std::vector<std::function<void()>> ops_;
};

AV ad_tcon(Tape& tp, const AV& a, const std::vector<int>& la, const AV& b, const std::vector<int>& lb);
AV ad_reshape(Tape& tp, const AV& a, const std::vector<int64_t>& s);
AV ad_permute(Tape& tp, const AV& a, const std::vector<int>& perm);
AV ad_renorm(Tape& tp, const AV& a);

struct ADPolicy {
  using T = AV;
  Tape& tp;
  T tc(const T& a, const std::vector<int>& la, const T& b, const std::vector<int>& lb) {
    return ad_tcon(tp, a, la, b, lb);
  }
  T rs(const T& a, const std::vector<int64_t>& s) { return ad_reshape(tp, a, s); }
  T pm(const T& a, const std::vector<int>& perm) { return ad_permute(tp, a, perm); }
  T mm(const T& a, const T& b) { return ad_tcon(tp, a, {-1, 1}, b, {1, -2}); }
  int64_t dim(const T& a, int i) const { return a.t.dims[i]; }
};

// Projector from stored factors (U, S, V of the forward move) on the tape:
// P1 = R2 V S^-1/2, P2 = S^-1/2 U^T R1, backward through the truncated SVD.
void ad_projector(Tape& tp, const AV& R1, bool t1, const AV& R2, bool t2, const ProjResult& pr, AV* P1, AV* P2);

// Energy + gradient: E+grad unit of fg! (optim_gs.jl:53-91, run_gs :133-143).
// From the current (converged) environment, run ad_iters CTMRG iterations
// with A as the variable, evaluate get_gs_energy and return real(E) and
// dE/dA (real A only).  C/T are checkpointed per iteration and each
// iteration is recomputed on a tape in the backward pass.
// h4 (optional): the plaquette energy get_gs_energy_4x4 (run_gs_h4,
// optim_gs_h4.jl:113-123) instead of the bond energies; Hh, Hv unused then.
double energy_grad(Env& e, const Tensor& Hh, const Tensor& Hv, int ad_iters, Tensor* gA,
                   const std::array<Tensor, 4>* h4 = nullptr);

// Pullback of run_es (optim_es.jl:196-210) with respect to B from the nested
// environment held by e: runs ad_iters nested iterations, returns
// get_es_energy and gH = dE/dB (complex, convention dE/dRe + i dE/dIm).
// h4 (optional): the plaquette energy get_es_energy_4x4 instead of the bond
// energies (run_es_h4 / get_es_grad_h4, optim_es_h4.jl:133-168); Hh, Hv unused then
double es_energy_grad(Env& e, const Tensor& Hh, const Tensor& Hv, int ad_iters, Tensor* gB,
                      const std::array<Tensor, 4>* h4 = nullptr);

// The unit of optim_wp (get_wp_grad / run_wp, optim_wp.jl:195-238): in the
// environment held by e (no CTMRG iterations), the plaquette operator given
// as the MPO wp = [s1, s2, s3, s4] (get_local_h) and the norm of the 2x2
// cluster whose site `site` (1..4, Params["wp"]) holds B and the other three
// A (energy_norm_4x4, evaluation.jl:435-441).  Returns both values and their
// gradients w.r.t. B, gH of the real part of the operator value and gN of the
// real part of the norm (Zygote's back((1, nothing)) / back((nothing, 1)):
// dRe/dRe(B) + i dRe/dIm(B)); complex.
void wp_grad(Env& e, const std::array<Tensor, 4>& wp, int site, const Tensor& B, std::complex<double>* wp_value,
             std::complex<double>* norm, Tensor* gH, Tensor* gN);

}  // namespace ipeps
