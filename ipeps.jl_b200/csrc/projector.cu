// Projector of the directional CTMRG move (real and complex enlarged corners).
//
// The reference forms M = R1*R2 (N x N, N = chi*D^2) and takes its full LAPACK
// SVD (ctmrg.jl:254-265, wrapper.jl:25-55).  Here M is never formed: a
// randomized range finder with power iterations works on R1 (R2 X) and
// R2^T (R1^T X) (all GEMMs), the sketches are orthonormalised by shifted
// CholeskyQR in FP64, and the projected k x k matrix is diagonalised by a
// one-sided Jacobi SVD in FP64 (k = n+1 plus oversampling).  Accuracy is
// checked a posteriori: the residual ||M v_i - s_i u_i|| of every kept
// triplet (the part of M v_i outside the sketch) must be below
// resid_tol * s_1, otherwise one more power iteration runs, warm-started from
// the current vectors.  The resolved right vectors of the last call of the
// same direction seed the next sketch, which near the CTMRG fixed point makes
// one pass sufficient.  Sorting, the relative cutoff 1e-12 and the
// degenerate-pair rule follow cutoff_matrix exactly.
#include "linalg.cuh"
#include "projector.cuh"

#include <algorithm>
#include <cmath>

namespace ipeps {

namespace {

// TF32 hi/lo planes of an enlarged-corner matrix Rt (r0 x c0, column-major)
// for the mixed form, split once per projector call and shared by all its
// products: `row` holds Rt itself as the A operand (rows r0, K = c0), `col`
// holds Rt^T (rows c0, K = r0), which is also Rt as a B operand.
const Planes& planes_row(Ctx& c, const Tensor& Rt, PlaneCache* pc) {
  if (pc->row.empty()) pc->row = split_kmajor(c, Rt.f64(), Rt.dims[0], false, Rt.dims[0], Rt.dims[1]);
  return pc->row;
}
const Planes& planes_col(Ctx& c, const Tensor& Rt, PlaneCache* pc) {
  if (pc->col.empty()) pc->col = split_kmajor(c, Rt.f64(), Rt.dims[0], true, Rt.dims[1], Rt.dims[0]);
  return pc->col;
}

bool use_planes(const Ctx& c, const MatRef& R, const PlaneCache* pc) {
  return pc && c.precision == kPrecMixed && R.t.dt == DType::F64;
}

}  // namespace

Tensor apply(Ctx& c, const MatRef& R, char op, const Tensor& X, PlaneCache* pc) {
  if (use_planes(c, R, pc)) {
    const bool t = (op == 'T') != R.trans;
    const int64_t m = (op == 'N') ? R.rows() : R.cols();
    const int64_t kk = (op == 'N') ? R.cols() : R.rows();
    IPEPS_CHECK(X.dims[0] == kk, "apply: shape mismatch");
    const int64_t n = X.nd > 1 ? X.dims[1] : 1;
    Tensor Y = c.alloc(DType::F64, {m, n});
    const Planes& PA = t ? planes_col(c, R.t, pc) : planes_row(c, R.t, pc);
    const Planes PB = split_kmajor(c, X.f64(), X.dims[0], true, n, kk);
    gemm_tf32x3_planes(c, PA, PB, m, n, kk, 1.0, 0.0, Y.f64(), m);
    return Y;
  }
  return apply(c, R, op, X);
}

Tensor apply_left_T(Ctx& c, const Tensor& X, const MatRef& R, char op, PlaneCache* pc) {
  if (use_planes(c, R, pc)) {
    const bool t = (op == 'T') != R.trans;
    const int64_t kk = (op == 'N') ? R.rows() : R.cols();
    const int64_t n = (op == 'N') ? R.cols() : R.rows();
    IPEPS_CHECK(X.dims[0] == kk, "apply_left_T: shape mismatch");
    const int64_t m = X.dims[1];
    Tensor Y = c.alloc(DType::F64, {m, n});
    const Planes PA = split_kmajor(c, X.f64(), X.dims[0], true, m, kk);
    const Planes& PB = t ? planes_row(c, R.t, pc) : planes_col(c, R.t, pc);
    gemm_tf32x3_planes(c, PA, PB, m, n, kk, 1.0, 0.0, Y.f64(), m);
    return Y;
  }
  return apply_left_T(c, X, R, op);
}

Tensor apply(Ctx& c, const MatRef& R, char op, const Tensor& X) {
  // op(R) * X
  bool t = (op == 'T') != R.trans;
  int64_t m = (op == 'N') ? R.rows() : R.cols();
  int64_t kk = (op == 'N') ? R.cols() : R.rows();
  IPEPS_CHECK(X.dims[0] == kk, "apply: shape mismatch");
  int64_t n = X.nd > 1 ? X.dims[1] : 1;
  Tensor Y = c.alloc(DType::F64, {m, n});
  gemm(c, DType::F64, t ? 'T' : 'N', 'N', m, n, kk, cplx(1), R.t.data(), R.t.dims[0], X.data(), X.dims[0],
       cplx(0), Y.data(), m);
  return Y;
}

Tensor apply_left_T(Ctx& c, const Tensor& X, const MatRef& R, char op) {
  // X^T * op(R): X is (kk x m) -> result (m x ncols)
  bool t = (op == 'T') != R.trans;
  int64_t kk = (op == 'N') ? R.rows() : R.cols();
  int64_t n = (op == 'N') ? R.cols() : R.rows();
  IPEPS_CHECK(X.dims[0] == kk, "apply_left_T: shape mismatch");
  int64_t m = X.dims[1];
  Tensor Y = c.alloc(DType::F64, {m, n});
  gemm(c, DType::F64, 'T', t ? 'T' : 'N', m, n, kk, cplx(1), X.data(), X.dims[0], R.t.data(), R.t.dims[0],
       cplx(0), Y.data(), m);
  return Y;
}

Tensor orth(Ctx& c, const Tensor& Y0, int passes, Tensor* Rout) {
  const int64_t N = Y0.dims[0];
  const int k = int(Y0.dims[1]);
  Tensor Y = Y0;
  Tensor G = c.alloc(DType::F64, {k, k});
  Tensor Ri = c.alloc(DType::F64, {k, k});
  Tensor Racc;
  double* d_tr = reinterpret_cast<double*>(c.scal->p) + 8;
  const double u = 1.1102230246251565e-16;
  const bool blocked = chol_fits(k) && trsm_fits(k);
  Tensor Rrow = blocked ? c.alloc(DType::F64, {int64_t(k) * (k + 1) / 2}) : Tensor();
  for (int pass = 0; pass < passes; ++pass) {
    // G = Y^T Y  (FP64 always: the Gram matrix is where precision is lost)
    gemm(c, DType::F64, 'T', 'N', k, k, N, cplx(1), Y.data(), N, Y.data(), N, cplx(0), G.data(), k, true);
    // shifted CholeskyQR: the first pass adds 11 (N k + k (k+1)) u trace(G) to the diagonal
    const double sf = (pass == 0) ? 11.0 * (double(N) * k + double(k) * (k + 1)) * u : 0.0;
    Tensor Yn = c.alloc(DType::F64, {N, k});
    if (blocked) {
      chol_blocked(c, G.f64(), k, k, sf, Rrow.f64());
      trsm_right_upper(c, Y.f64(), N, N, k, G.f64(), k, Yn.f64(), N, Rrow.f64());
    } else {
      if (pass == 0) {
        trace(c, G.f64(), k, k, d_tr);
        chol_upper(c, G.f64(), k, k, d_tr, sf);
      } else {
        chol_upper(c, G.f64(), k, k, nullptr, 0.0);
      }
      triinv_upper(c, G.f64(), k, k, Ri.f64(), k);
      gemm(c, DType::F64, 'N', 'N', N, k, k, cplx(1), Y.data(), N, Ri.data(), k, cplx(0), Yn.data(), N, true);
    }
    Y = Yn;
    if (Rout) {
      if (pass == 0) {
        Racc = clone(c, G);
      } else {
        Tensor Rn = c.alloc(DType::F64, {k, k});
        gemm(c, DType::F64, 'N', 'N', k, k, k, cplx(1), G.data(), k, Racc.data(), k, cplx(0), Rn.data(), k, true);
        Racc = Rn;
      }
    }
  }
  if (Rout) *Rout = Racc;
  return Y;
}

namespace {

// out[j] = ||X[:, j]|| for j < nc (FP64, one warp per column)
__global__ void colnorms_kernel(const double* X, int64_t m, int nc, double* out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nc) return;
  double s = 0;
  for (int64_t i = lane; i < m; i += 32) s = fma(X[i + warp * m], X[i + warp * m], s);
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) out[warp] = sqrt(s);
}

// max over columns j < nc of ||X[:, j]|| (FP64, one warp per column)
__global__ void colnorm_max_kernel(const double* X, int64_t m, int nc, unsigned long long* out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nc) return;
  double s = 0;
  for (int64_t i = lane; i < m; i += 32) s = fma(X[i + warp * m], X[i + warp * m], s);
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(sqrt(s))));
}

// ------------------------------------------------------------------ backends
// The projector logic below is written once over two backends: real (FP64)
// and complex (complex128) enlarged corners.  M = R1 R2 is N1 x N2 with
// R1 (N1 x K1), R2 (K1 x N2); it is rectangular while the corner dimensions of
// an environment still differ (first iterations from init_ctm1).  words is the
// number of doubles per element, so that the gathers and column scalings can
// treat a complex column as a real column of twice the height.

struct RealOps {
  Ctx& c;
  const MatRef& R1;
  const MatRef& R2;
  PlaneCache pc1, pc2;  // mixed form: TF32 planes of R1, R2
  static constexpr DType dt = DType::F64;
  static constexpr int words = 1;
  int64_t N1() const { return R1.rows(); }
  int64_t K1() const { return R1.cols(); }
  int64_t N2() const { return R2.cols(); }
  Tensor M(const Tensor& X) { return apply(c, R1, 'N', apply(c, R2, 'N', X, &pc2), &pc1); }   // M X
  Tensor MH(const Tensor& X) { return apply(c, R2, 'T', apply(c, R1, 'T', X, &pc1), &pc2); }  // M^T X
  Tensor orth_(const Tensor& Y, int passes) { return orth(c, Y, passes, nullptr); }
  // X = Bh^H Q2 (k x k) for Bh = M^H Q (N2 x k)
  Tensor small(const Tensor& Bh, const Tensor& Q2, int k) {
    Tensor X = c.alloc(dt, {k, k});
    gemm(c, dt, 'T', 'N', k, k, N2(), cplx(1), Bh.data(), N2(), Q2.data(), N2(), cplx(0), X.data(), k, true);
    return X;
  }
  void jacobi(Tensor& X, Tensor& J, Tensor& S, int k, const SvdParams& sp, int* d_sweeps) {
    const double tol = (c.precision == kPrecMixed) ? std::max(sp.jacobi_tol, sp.jacobi_tol_mixed) : sp.jacobi_tol;
    jacobi_svd_auto(c, X.f64(), k, k, k, J.f64(), k, S.f64(), sp.jacobi_max_sweeps, tol, d_sweeps);
  }
  // sketch width: 128 columns when that still oversamples by want/2 (the
  // Jacobi then rotates all of its 64 pairs in one pass of its 8-lane groups),
  // else at most 160 (the widest sketch whose Jacobi fits in shared memory)
  int width(int want, int kw, const SvdParams& sp) const {
    if (kw > 128 && want + std::max(sp.min_oversample, want / 2) <= 128) return 128;
    if (kw > 160 && want + sp.min_oversample <= 160) return 160;
    return kw;
  }
  Tensor P1(const Tensor& V) { return apply(c, R2, 'N', V, &pc2); }          // R2 V      (K1 x n)
  Tensor P2(const Tensor& U) { return apply_left_T(c, U, R1, 'N', &pc1); }   // U^T R1    (n x K1)
};

Tensor cmm(Ctx& c, char oa, char ob, int64_t m, int64_t n, int64_t k, const Tensor& A, int64_t lda, const Tensor& B,
           int64_t ldb) {
  Tensor Y = c.alloc(DType::C128, {m, n});
  gemm(c, DType::C128, oa, ob, m, n, k, cplx(1), A.data(), lda, B.data(), ldb, cplx(0), Y.data(), m, true);
  return Y;
}

Tensor orth_c(Ctx& c, const Tensor& Y0, int passes) {
  const int64_t N = Y0.dims[0];
  const int k = int(Y0.dims[1]);
  Tensor Y = Y0;
  Tensor G = c.alloc(DType::C128, {k, k});
  const double u = 1.1102230246251565e-16;
  for (int pass = 0; pass < passes; ++pass) {
    gemm(c, DType::C128, 'C', 'N', k, k, N, cplx(1), Y.data(), N, Y.data(), N, cplx(0), G.data(), k, true);
    const double sf = (pass == 0) ? 11.0 * (double(N) * k + double(k) * (k + 1)) * u : 0.0;
    chol_c(c, G.data(), k, k, sf);
    Tensor Yn = c.alloc(DType::C128, {N, k});
    trsm_c(c, Y.data(), N, N, k, G.data(), k, Yn.data(), N);
    Y = Yn;
  }
  return Y;
}

struct ComplexOps {
  Ctx& c;
  Tensor R1, R2;  // materialised (untransposed) complex128
  static constexpr DType dt = DType::C128;
  static constexpr int words = 2;
  ComplexOps(Ctx& cc, const MatRef& a, const MatRef& b)
      : c(cc),
        R1(to_complex(cc, a.trans ? permute(cc, a.t, {1, 0}) : a.t)),
        R2(to_complex(cc, b.trans ? permute(cc, b.t, {1, 0}) : b.t)) {}
  int64_t N1() const { return R1.dims[0]; }
  int64_t K1() const { return R1.dims[1]; }
  int64_t N2() const { return R2.dims[1]; }
  Tensor M(const Tensor& X) {
    const int64_t n = X.dims[1];
    return cmm(c, 'N', 'N', N1(), n, K1(), R1, N1(), cmm(c, 'N', 'N', K1(), n, N2(), R2, K1(), X, N2()), K1());
  }
  Tensor MH(const Tensor& X) {
    const int64_t n = X.dims[1];
    return cmm(c, 'C', 'N', N2(), n, K1(), R2, K1(), cmm(c, 'C', 'N', K1(), n, N1(), R1, N1(), X, N1()), K1());
  }
  Tensor orth_(const Tensor& Y, int passes) { return orth_c(c, Y, passes); }
  Tensor small(const Tensor& Bh, const Tensor& Q2, int k) { return cmm(c, 'C', 'N', k, k, N2(), Bh, N2(), Q2, N2()); }
  void jacobi(Tensor& X, Tensor& J, Tensor& S, int k, const SvdParams& sp, int* d_sweeps) {
    jacobi_c_svd(c, X.data(), k, k, k, J.data(), k, S.f64(), sp.jacobi_max_sweeps, sp.jacobi_tol, d_sweeps);
  }
  int width(int want, int kw, const SvdParams& sp) const {
    while (kw > want + sp.min_oversample && !complex_small_fits(kw, kw)) --kw;
    IPEPS_CHECK(complex_small_fits(kw, kw), "get_projector: complex sketch too wide for the shared-memory kernels");
    return kw;
  }
  Tensor P1(const Tensor& V) { return cmm(c, 'N', 'N', K1(), V.dims[1], N2(), R2, K1(), V, N2()); }
  Tensor P2(const Tensor& U) { return cmm(c, 'C', 'N', U.dims[1], K1(), N1(), U, N1(), R1, N1()); }
};

// One sketch pass: range finder with q power iterations from Omega, Rayleigh-Ritz, Jacobi.
struct Sketch {
  Tensor Q, Q2, X, J, Ss;  // Q: N1 x k, Q2: N2 x k; X = W (k x k); J (k x k); Ss sorted S (k)
  Tensor perm;             // int[k] stored in a double buffer
  int sweeps = 0;
};

// inter: CholeskyQR passes of the intermediate sketches.  One shifted pass
// suppresses directions below ~sqrt(shift) ~ 1e-6 s_1, which over the power
// iterations then decay away; three passes (sCholQR3) keep them, as needed
// when the truncation reaches down to the 1e-12 relative cutoff.
template <class Ops>
Sketch sketch_pass(Ctx& c, Ops& o, const Tensor& Om, int q, const SvdParams& sp, int inter) {
  const int k = int(Om.dims[1]);
  Sketch s;
  Tensor Y = o.M(Om);
  for (int it = 0; it < q; ++it) {
    Tensor Q = o.orth_(Y, inter);
    Tensor Z = o.orth_(o.MH(Q), inter);
    Y = o.M(Z);
  }
  s.Q = o.orth_(Y, 3);
  // B^H = M^H Q (N2 x k), Q2 = orth(B^H).  The Rayleigh-Ritz matrix is formed
  // explicitly, X = B = (M^H Q)^H Q2, rather than taken as R^H from B^H = Q2 R:
  // when M is numerically rank deficient the shifted first CholeskyQR pass
  // leaves sqrt(shift)-sized entries in R for the null directions, which the
  // later passes cannot normalise, and R^H would show them as spurious
  // singular values far above the 1e-12 cutoff.
  Tensor Bh = o.MH(s.Q);
  s.Q2 = o.orth_(Bh, 3);
  s.X = o.small(Bh, s.Q2, k);
  // one-sided Jacobi: X J = W = Ux S  =>  U = Q Ux, V = Q2 J
  s.J = c.alloc(Ops::dt, {k, k});
  Tensor S = c.alloc(DType::F64, {k});
  int* d_sweeps = reinterpret_cast<int*>(static_cast<char*>(c.scal->p) + 3900);
  o.jacobi(s.X, s.J, S, k, sp, d_sweeps);
  s.Ss = c.alloc(DType::F64, {k});
  s.perm = c.alloc(DType::F64, {(k + 1) / 2});
  sort_desc(c, S.f64(), k, s.Ss.f64(), static_cast<int*>(s.perm.data()));
  IPEPS_CUDA(cudaMemcpyAsync(&s.sweeps, d_sweeps, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  return s;
}

void copy_cols(Ctx& c, Tensor& dst, const Tensor& src, int64_t rows, int ncols, int words) {
  IPEPS_CUDA(cudaMemcpyAsync(dst.data(), src.data(), size_t(rows) * ncols * 8 * words, cudaMemcpyDeviceToDevice,
                             c.stream));
}

template <class Ops>
ProjResult projector_impl(Ctx& c, Ops& o, int chi, const SvdParams& sp, ProjCache* cache, bool keep_factors) {
  constexpr DType dt = Ops::dt;
  constexpr int w = Ops::words;
  const int64_t N1 = o.N1(), K1 = o.K1(), N2 = o.N2(), Nmin = std::min(N1, N2);
  const int new_chi = int(std::min<int64_t>(chi, K1));
  const int want = int(std::min<int64_t>(Nmin, new_chi + 1));
  const int over = std::max(sp.min_oversample, want * sp.oversample_num / std::max(sp.oversample_den, 1));
  const int k = o.width(want, int(std::min<int64_t>(Nmin, int64_t(want) + over)), sp);

  // Sketch Omega (N2 x k): resolved right vectors of an earlier call first,
  // then Gaussian columns.  No seeds when k = min(N1, N2): a Gaussian Omega
  // then spans the domain and one pass is exact, which seed vectors (possibly
  // confined to a few symmetry sectors of M) would not guarantee.  After a
  // cutoff-limited truncation at least min_oversample columns stay Gaussian,
  // so that directions absent from the seeds can enter; in the chi-limited
  // regime the seeds may fill the sketch.
  Tensor Om = c.alloc(dt, {N2, k});
  randn(c, Om);
  bool warm = false;
  const bool room = !cache || cache->cutoff_limited;
  const int seed_cap = room ? std::max(0, k - std::max(sp.min_oversample, 1)) : k;
  if (k < Nmin && seed_cap > 0 && sp.warm_start && cache && !cache->seed(sp.seed_older).empty() &&
      cache->seed(sp.seed_older).dims[0] == N2 && cache->seed(sp.seed_older).dt == dt) {
    const Tensor& Vs = cache->seed(sp.seed_older);
    copy_cols(c, Om, Vs, N2, int(std::min<int64_t>(Vs.dims[1], seed_cap)), w);
    warm = true;
  }
  int q = (k == Nmin) ? 0 : (warm ? sp.power_iters_warm : sp.power_iters);
  int inter = sp.inter_passes;
  if (!warm || !cache || cache->cutoff_limited) inter = std::max(inter, 3);
  // power iterations this direction's recent calls needed beyond q (each
  // extra pass below costs a Rayleigh-Ritz step, two sCholQR3 and a Jacobi SVD
  // on top of its power iteration; doing the iterations up front is cheaper).
  // Only with sCholQR3 intermediates: a single shifted pass drops directions
  // below ~sqrt(shift) s_1 at every iteration, so more iterations would lose them.
  // residual tolerance of this call (the mixed form's 3xTF32 iterations settle
  // for the FP32-level floor of their products)
  const double rtol = (c.precision == kPrecMixed && dt == DType::F64) ? std::max(sp.resid_tol, sp.resid_tol_mixed)
                                                                       : sp.resid_tol;
  // seeds resolved to a looser tolerance than this call's (the first FP64
  // iterations after the mixed form's 3xTF32 ones, the adjoint's checkpoint
  // iterations at 1e-12): one power iteration per factor ~7 of the residual,
  // done up front with sCholQR3 intermediates, instead of as extra passes
  if (warm && q > 0 && cache->seed_tol(sp.seed_older) > 10.0 * rtol) {
    inter = std::max(inter, 3);
    q += std::min(6, int(std::ceil(std::log(cache->seed_tol(sp.seed_older) / rtol) / std::log(7.0))));
  }
  const bool adapt = q > 0 && cache && inter >= 3;
  if (adapt) q += cache->qbonus;
  int extra = 0;
  double res_final = 1.0;

  ProjResult r;
  r.k = k;
  Sketch sk;
  std::vector<double> all(k);
  int n = 0, n_above_last = 0;
  Tensor Ux, Vk;
  int* d_perm = nullptr;
  double* d_res = reinterpret_cast<double*>(c.scal->p) + 48;
  double prev_res = 1e300;
  for (int attempt = 0;; ++attempt) {
    sk = sketch_pass(c, o, Om, q, sp, inter);
    d_perm = static_cast<int*>(sk.perm.data());
    IPEPS_CUDA(cudaMemcpyAsync(all.data(), sk.Ss.data(), size_t(k) * 8, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    c.jacobi_sweeps += uint64_t(sk.sweeps);
    // cutoff_matrix (wrapper.jl:37-55)
    const double smax = all[0];
    int n_above = 0;
    for (int i = 0; i < k; ++i)
      if (smax > 0 && all[i] / smax > 1e-12) n_above++;
    n_above_last = n_above;
    if (n_above < new_chi && inter < 3 && q > 0) {
      // cutoff-limited after cheap intermediates: small directions may be missing; redo cold with sCholQR3
      inter = 3;
      Om = c.alloc(dt, {N2, k});
      randn(c, Om);
      q = sp.power_iters;
      --attempt;
      continue;
    }
    n = std::min(new_chi, n_above);
    IPEPS_CHECK(n >= 1, "get_projector: no singular value above the cutoff (zero enlarged corner?)");
    // the reference's s has length min(N1, N2) (full SVD); ours is the top-k part
    if (Nmin > n && k > n) {
      if (std::fabs(all[n] - all[n - 1]) < 1e-10) n = n + 1;
    }
    IPEPS_CHECK(n <= k, "get_projector: truncation beyond the sketch");
    // Ux[:, j] = W[:, perm[j]] / S_sorted[j] (kept + one), Vk = Q2 J[:, perm]
    const int nc = std::min(n + 1, k);
    Ux = c.alloc(dt, {k, nc});
    gather_cols(c, sk.X.f64(), w * k, w * k, d_perm, nc, sk.Ss.f64(), 2, Ux.f64(), w * k);
    Tensor Js = c.alloc(dt, {k, k});
    gather_cols(c, sk.J.f64(), w * k, w * k, d_perm, k, nullptr, 0, Js.f64(), w * k);
    Vk = c.alloc(dt, {N2, k});
    gemm(c, dt, 'N', 'N', N2, k, k, cplx(1), sk.Q2.data(), N2, Js.data(), k, cplx(0), Vk.data(), N2, true);
    if (q == 0 && k == Nmin) {  // the sketch spans a whole side of M: exact
      res_final = 0.0;
      break;
    }
    // residual of the kept triplets and the next one: ||M v_i - s_i u_i|| <= resid_tol * s_1.
    // For the adjoint (keep_factors) also the tail down to 0.8 s_n: the adjoint
    // sums those triplets exactly, and the interval of its expansion of the
    // rest of the spectrum, and with it the number of terms, is set by the
    // first triplet it does not resolve.
    int nr = nc;
    if (keep_factors)
      while (nr < k && all[nr] >= 0.8 * all[n - 1]) ++nr;
    Tensor Vc = c.alloc(dt, {N2, nr});
    copy_cols(c, Vc, Vk, N2, nr, w);
    Tensor Res = o.M(Vc);
    Tensor Us = c.alloc(dt, {k, nr});
    gather_cols(c, sk.X.f64(), w * k, w * k, d_perm, nr, nullptr, 0, Us.f64(), w * k);  // W = Ux S
    gemm(c, dt, 'N', 'N', N1, nr, k, cplx(-1), sk.Q.data(), N1, Us.data(), k, cplx(1), Res.data(), N1, true);
    IPEPS_CUDA(cudaMemsetAsync(d_res, 0, 8, c.stream));
    colnorm_max_kernel<<<(nr * 32 + 255) / 256, 256, 0, c.stream>>>(Res.f64(), w * N1, nr,
                                                                    reinterpret_cast<unsigned long long*>(d_res));
    IPEPS_LAUNCH_CHECK();
    double res = 0;
    IPEPS_CUDA(cudaMemcpyAsync(&res, d_res, 8, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    // done when below tolerance, or when it stopped decreasing (the FP64 floor of
    // R1 (R2 v), ~eps ||R1|| ||R2||, can sit above resid_tol * s_1)
    res_final = smax > 0 ? res / smax : 1.0;
    if (res <= rtol * smax) break;
    if (res > 0.5 * prev_res || attempt >= sp.max_extra_passes) {
      c.resid_misses++;
      break;
    }
    prev_res = res;
    // not converged: one more power iteration from the current right vectors
    Om = Vk;
    q = 1;
    c.projector_extra_passes++;
    ++extra;
  }
  r.sweeps = sk.sweeps;
  c.projector_calls++;
  r.n = n;
  r.s_host.assign(all.begin(), all.begin() + n);

  Tensor U = c.alloc(dt, {N1, n});
  gemm(c, dt, 'N', 'N', N1, n, k, cplx(1), sk.Q.data(), N1, Ux.data(), k, cplx(0), U.data(), N1, true);
  Tensor V = c.alloc(dt, {N2, n});
  copy_cols(c, V, Vk, N2, n, w);
  // resolved part of the sketch: s_a > 1e-13 s_1 (W/s is accurate there)
  int rr = 0;
  while (rr < k && all[rr] > 1e-13 * all[0]) ++rr;
  rr = std::max(rr, n);
  if (cache) {
    // seed for the next call of this direction: the resolved right vectors only
    // (near-null directions of this M say nothing about the next one)
    Tensor Vc = c.alloc(dt, {N2, rr});
    copy_cols(c, Vc, Vk, N2, rr, w);
    cache->Vold = cache->V;
    cache->V = Vc;
    cache->tol_old = cache->tol;
    cache->tol = std::max(res_final, 1e-15);  // the residual these vectors reached
    cache->cutoff_limited = n_above_last < new_chi;
    if (adapt)
      cache->qbonus = extra > 0 ? std::min(cache->qbonus + extra, sp.max_extra_passes) : std::max(cache->qbonus - 1, 0);
  }
  if (keep_factors) {
    IPEPS_CHECK(dt == DType::F64, "get_projector: the projector adjoint is real-only");
    // The adjoint sums the resolved triplets exactly and expands the rest of the
    // spectrum on their complement, which is exact only if the resolved vectors
    // span an invariant subspace: keep just the leading triplets whose residual
    // ||M v_a - s_a u_a|| is at most 1e-10 s_1 (the sketch's oversampled tail is
    // less accurate and goes to the expansion instead).
    if (rr > n) {
      Tensor Vall = c.alloc(dt, {N2, rr});
      copy_cols(c, Vall, Vk, N2, rr, w);
      Tensor Res = o.M(Vall);
      Tensor Wall = c.alloc(dt, {k, rr});
      gather_cols(c, sk.X.f64(), k, k, d_perm, rr, nullptr, 0, Wall.f64(), k);
      gemm(c, dt, 'N', 'N', N1, rr, k, cplx(-1), sk.Q.data(), N1, Wall.data(), k, cplx(1), Res.data(), N1, true);
      Tensor rn = c.alloc(DType::F64, {rr});
      colnorms_kernel<<<(rr * 32 + 255) / 256, 256, 0, c.stream>>>(Res.f64(), N1, rr, rn.f64());
      IPEPS_LAUNCH_CHECK();
      std::vector<double> rh(rr);
      IPEPS_CUDA(cudaMemcpyAsync(rh.data(), rn.data(), size_t(rr) * 8, cudaMemcpyDeviceToHost, c.stream));
      c.sync();
      int acc = n;
      while (acc < rr && rh[acc] <= 1e-10 * all[0]) ++acc;
      rr = acc;
    }
    r.r = rr;
    r.sr_host.assign(all.begin(), all.begin() + rr);
    r.s_next = (rr < k) ? all[rr] : all[k - 1];
    Tensor Uxr = c.alloc(dt, {k, rr});
    gather_cols(c, sk.X.f64(), k, k, d_perm, rr, sk.Ss.f64(), 2, Uxr.f64(), k);
    r.Ur = c.alloc(dt, {N1, rr});
    gemm(c, dt, 'N', 'N', N1, rr, k, cplx(1), sk.Q.data(), N1, Uxr.data(), k, cplx(0), r.Ur.data(), N1, true);
    r.Vr = c.alloc(dt, {N2, rr});
    copy_cols(c, r.Vr, Vk, N2, rr, w);
    r.Sr = c.alloc(DType::F64, {rr});
    IPEPS_CUDA(cudaMemcpyAsync(r.Sr.data(), sk.Ss.data(), size_t(rr) * 8, cudaMemcpyDeviceToDevice, c.stream));
  }

  r.S = c.alloc(DType::F64, {n});
  IPEPS_CUDA(cudaMemcpyAsync(r.S.data(), sk.Ss.data(), size_t(n) * 8, cudaMemcpyDeviceToDevice, c.stream));
  // P1 = R2 V S^-1/2 ; P2 = S^-1/2 U^H R1
  scale_cols(c, V.f64(), w * N2, w * N2, n, r.S.f64(), 1);
  scale_cols(c, U.f64(), w * N1, w * N1, n, r.S.f64(), 1);
  r.P1 = o.P1(V);
  r.P2 = o.P2(U);
  return r;
}

}  // namespace

ProjResult get_projector(Ctx& c, const MatRef& R1, const MatRef& R2, int chi, const SvdParams& sp,
                         ProjCache* cache, bool keep_factors) {
  IPEPS_CHECK(R1.cols() == R2.rows(), "get_projector: inner dimensions of R1*R2 differ");
  if (R1.t.dt == DType::C128 || R2.t.dt == DType::C128) {
    ComplexOps o(c, R1, R2);
    return projector_impl(c, o, chi, sp, cache, keep_factors);
  }
  RealOps o{c, R1, R2, {}, {}};
  return projector_impl(c, o, chi, sp, cache, keep_factors);
}

}  // namespace ipeps
