// Truncated-SVD projector of the enlarged corners (ctmrg.jl:254-265 and
// wrapper.jl:25-55), computed without forming R1*R2.
#pragma once
#include "ctx.cuh"

namespace ipeps {

// A logical matrix: t (2-D) or its transpose.
struct MatRef {
  Tensor t;
  bool trans = false;
  int64_t rows() const { return trans ? t.dims[1] : t.dims[0]; }
  int64_t cols() const { return trans ? t.dims[0] : t.dims[1]; }
};

struct SvdParams {
  int oversample_num = 1;   // k = want + max(min_oversample, want*num/den)
  int oversample_den = 1;
  int min_oversample = 16;
  int power_iters = 3;      // cold start
  int power_iters_warm = 2; // when the previous V of this direction seeds the sketch
  int max_extra_passes = 6; // extra power iterations while the residual check fails
  int inter_passes = 1;     // CholeskyQR passes for the intermediate power-iteration sketches
  bool seed_older = true;   // seed from the call before the previous one (period-2 cycles)
  // ||M v_i - s_i u_i|| <= resid_tol * s_1 for the kept triplets.  On slowly
  // decaying spectra each extra pass lowers the residual only ~7x.  Measured
  // against exact-SVD trajectories (30 iterations, Heisenberg D=4 chi=64): the
  // last-iteration energy error is 5e-14 at 1e-11, 4e-11 at 3e-10 and 1.4e-9 at
  // 1e-9; 1e-10 keeps the 1e-10 bar with a margin and saves ~1/4 of the passes.
  double resid_tol = 1e-10;
  // the same check in the mixed form, whose 3xTF32 products carry FP32-level
  // errors (~1e-6 of s_1 in the residual itself)
  double resid_tol_mixed = 1e-6;
  bool warm_start = true;
  int jacobi_max_sweeps = 40;
  double jacobi_tol = 0.0;  // <= 0: m * eps (rounding level of the column dot products)
  // the Jacobi SVD's tolerance in the mixed form's 3xTF32 iterations, whose
  // products carry ~1e-7 relative errors: the last sweep or two that take the
  // column angles from 1e-10 to the rounding level buy nothing there (the
  // FP64 iterations at the end of a run use jacobi_tol)
  double jacobi_tol_mixed = 1e-10;
};

// Resolved right vectors of the last two calls of one direction (warm start).
// The sketch is seeded from the older one: a CTMRG run that has settled into
// a period-2 cycle returns to the same environment every second iteration,
// and for a converging run both are equally close to the fixed point.
struct ProjCache {
  Tensor V;      // previous call
  Tensor Vold;   // the call before
  // the last truncation of this direction was set by the 1e-12 cutoff rather
  // than by chi: the next sketch keeps its small directions (sCholQR3 throughout)
  bool cutoff_limited = true;
  // power iterations added to the next call's sketch: raised by the extra
  // passes a call needed, lowered by one after a call that needed none
  int qbonus = 0;
  // residual (relative to s_1) the call that produced V (Vold) reached
  double tol = 1.0, tol_old = 1.0;
  const Tensor& seed(bool older) const { return (older && !Vold.empty()) ? Vold : V; }
  double seed_tol(bool older) const { return (older && !Vold.empty()) ? tol_old : tol; }
};

struct ProjResult {
  Tensor P1;  // N x n   (P  in the reference)
  Tensor P2;  // n x N   (Pd in the reference)
  Tensor S;   // n (device)
  std::vector<double> s_host;  // n singular values, descending
  int n = 0;
  int k = 0;
  int sweeps = 0;
  // resolved singular triplets of the sketch (kept ones first), for the
  // adjoint: r columns with s_a > 1e-13 s_1
  int r = 0;
  Tensor Ur, Vr, Sr;  // N x r, N x r, r
  std::vector<double> sr_host;
  // upper estimate of the largest singular value outside the resolved set
  // (the next sketch value, or the smallest resolved one when the sketch is
  // exhausted): bounds the spectrum the adjoint's resolvent expansion sees
  double s_next = 0;
};

// Returns P1 = R2 V S^-1/2, P2 = S^-1/2 U^T R1 with (U,S,V) the truncated
// SVD of R1*R2 following wrap_svd/cutoff_matrix (keep min(chi, #{s/smax >
// 1e-12}), plus one when |s[n+1]-s[n]| < 1e-10).
ProjResult get_projector(Ctx& c, const MatRef& R1, const MatRef& R2, int chi, const SvdParams& sp,
                         ProjCache* cache, bool keep_factors = false);

// op(R)*X with R a MatRef; op in {'N','T'}
Tensor apply(Ctx& c, const MatRef& R, char op, const Tensor& X);
// X^T * op(R)   (returns X^T op(R))
Tensor apply_left_T(Ctx& c, const Tensor& X, const MatRef& R, char op);
// TF32 hi/lo planes of one enlarged-corner matrix, split on first use (mixed form)
struct PlaneCache {
  Planes row, col;
};
// the same products; in the mixed form R's planes are taken from (or added to) pc
Tensor apply(Ctx& c, const MatRef& R, char op, const Tensor& X, PlaneCache* pc);
Tensor apply_left_T(Ctx& c, const Tensor& X, const MatRef& R, char op, PlaneCache* pc);

// Orthonormalise the columns of Y (N x k) by shifted CholeskyQR; if Rout is
// non-null it receives R with Y = Q R.
Tensor orth(Ctx& c, const Tensor& Y, int passes, Tensor* Rout);

}  // namespace ipeps
