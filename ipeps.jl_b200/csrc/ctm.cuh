// CTMRG environment and moves (src/ctm/ctmrg.jl, src/ctm/ctm_tensor.jl,
// src/graph/evaluation.jl, src/nested_tensor/*.jl of the reference).
#pragma once
#include "projector.cuh"

#include <array>
#include <complex>

namespace ipeps {

// Nested tensor: component 0 is the plain tensor; 1..3 are the B, Bd, BB
// slots (empty tensor == EmptyT).  A plain tensor has nested == false.
struct NT {
  std::array<Tensor, 4> c;
  bool nested = false;
  NT() = default;
  NT(const Tensor& t) { c[0] = t; }  // NOLINT: implicit plain -> NT
  bool has(int i) const { return !c[i].empty(); }
};

NT ntcon(Ctx& c, const NT& A, const std::vector<int>& la, const NT& B, const std::vector<int>& lb);
NT nreshape(const NT& A, const std::vector<int64_t>& s);
NT npermute(Ctx& c, const NT& A, const std::vector<int>& perm);
NT nmatmul(Ctx& c, const NT& A, char opA, const NT& B, char opB);
NT nshift(Ctx& c, const NT& A, double phi);
void nrenormalize(Ctx& c, NT& A);

struct CtmParams {
  int chi = 32;
  int min_iter = 4;
  int max_iter = 20;
  int ad_max_iter = 4;
  double rg_tol = 1e-6;
  // mixed form: FP64 for the last polish_iters iterations (0 = stay mixed), or
  // from the iteration whose change drops below polish_tol * rg_tol
  int polish_iters = 4;
  double polish_tol = 100.0;
  SvdParams svd;
};

struct CtmLogEntry {
  int iter;
  double diff;
  double obj_re, obj_im;
  int chi_left;
};

struct Env {
  Ctx* ctx = nullptr;
  int D = 0, d = 0;
  DType dt = DType::F64;   // dtype of A
  CtmParams prm;
  Tensor A, Ad;
  std::array<Tensor, 4> Cs, Es;
  // nested (excited-state) slots
  bool nested = false;
  Tensor B, Bd;
  std::array<Tensor, 4> B_Cs, Bd_Cs, BB_Cs, B_Es, Bd_Es, BB_Es;
  double px = 0, py = 0;
  ProjCache cache[4];
  std::vector<double> last_s;  // spectrum of the last left move
  std::vector<CtmLogEntry> log;
  // statistics
  uint64_t moves = 0;
  double move_seconds = 0;
  // rg_step runs left || right, then top || bottom: each pair reads and writes
  // disjoint environment slots.  The second move of a pair runs on `aux`, a
  // context with its own stream (created on first use).
  bool parallel_moves = true;
  // moves that keep their projector (keep != nullptr) also keep the resolved
  // singular triplets for the projector adjoint; the nested pullback needs
  // P1/P2 only (complex environments have no projector adjoint)
  bool keep_adjoint = true;
  std::shared_ptr<Ctx> aux;
  // run_ctm evaluates the convergence criterion of iteration i on `aux_eval`
  // (a third stream, its own host thread) while iteration i+1 runs; a
  // speculative iteration after convergence is rolled back (FP64 form,
  // energy criteria; on with parallel_moves)
  std::shared_ptr<Ctx> aux_eval;

  NT all_A() const;
  NT all_Ad() const;
  NT all_C(int i) const;
  NT all_E(int i) const;
};

void init_ctm1(Env& e);
// one directional move; dir 0=left 1=right 2=top 3=bottom; returns s (host).
// keep (optional) receives the projector with its resolved singular triplets.
std::vector<double> ctm_move(Env& e, int dir, ProjResult* keep = nullptr);

struct Traces {
  std::complex<double> trH, tr;
};
// tr(H rho) and tr(rho) of several (rho, H) pairs (FP64, one host round trip)
std::vector<Traces> dm_traces(Ctx& c, const std::vector<std::pair<Tensor, Tensor>>& items);
std::vector<double> rg_step(Env& e);
// the four moves of rg_step (left || right, then top || bottom when
// e.parallel_moves); keep (optional, 4 entries, by direction) receives the
// projectors with their resolved triplets.  Returns the left-move spectrum.
std::vector<double> ctm_moves4(Env& e, ProjResult* keep);
// energy (evaluation.jl:15-29): E (complex) and Na (complex)
// (ctx_precision: contractions in the context's precision instead of FP64; traces FP64)
void gs_energy(Env& e, const Tensor& Hh, const Tensor& Hv, std::complex<double>* E, std::complex<double>* Na,
               bool ctx_precision = false);
// nested energy (evaluation.jl:31-45): real(E[4])
double es_energy(Env& e, const Tensor& Hh, const Tensor& Hv);
// get_all_norm (evaluation.jl:61-77): returns Nb, writes envB (complex, size of A)
std::complex<double> all_norm(Env& e, Tensor* envB);
// get_gs_norm (evaluation.jl:47-59)
std::complex<double> gs_norm(Env& e);
// get_single_dm contracted with Ad (optim_es.jl:247-251), shape of A
Tensor single_dm_Ad(Env& e);
// plaquette Hamiltonian as the MPO [s1, s2, s3, s4] of get_local_h (local_h.jl:1-31):
// s1 (d, d, a), s2 (a, d, d, b), s3 (b, d, d, c), s4 (c, d, d)
using H4 = std::array<Tensor, 4>;
// get_gs_energy_4x4 (evaluation.jl:339-356)
std::complex<double> gs_energy_4x4(Env& e, const H4& h);
// get_es_energy_4x4 (evaluation.jl:358-398)
std::complex<double> es_energy_4x4(Env& e, const H4& h);

enum ConvMode : int {
  kConvEnergy = 0,     // get_gs_energy (optim_gs.jl:121)
  kConvSpectrum = 1,   // left-move spectrum (ctmrg.jl:29-31)
  kConvEs = 2,         // get_es_energy / get_all_norm (optim_es.jl:175)
  kConvEnergy4x4 = 3,  // get_gs_energy_4x4 (optim_es_h4.jl:33)
  kConvEs4x4 = 4,      // get_es_energy_4x4 / get_all_norm (optim_es_h4.jl:139)
};
// run_ctm (ctmrg.jl:1-55) with the convergence criterion of conv_mode
// (Hh, Hv for the bond energies, h4 for the plaquette ones).
// Returns iterations done; *last_diff = diffs[end]; *converged.
int run_ctm(Env& e, int conv_mode, const Tensor* Hh, const Tensor* Hv, double* last_diff, bool* converged,
            const H4* h4 = nullptr);

}  // namespace ipeps
