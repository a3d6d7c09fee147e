// Projector of the directional CTMRG move.
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
  for (int pass = 0; pass < passes; ++pass) {
    // G = Y^T Y  (FP64 always: the Gram matrix is where precision is lost)
    gemm(c, DType::F64, 'T', 'N', k, k, N, cplx(1), Y.data(), N, Y.data(), N, cplx(0), G.data(), k, true);
    // shifted CholeskyQR: the first pass adds 11 (N k + k (k+1)) u trace(G) to the diagonal
    const double sf = (pass == 0) ? 11.0 * (double(N) * k + double(k) * (k + 1)) * u : 0.0;
    Tensor Yn = c.alloc(DType::F64, {N, k});
    if (blocked) {
      chol_blocked(c, G.f64(), k, k, sf);
      trsm_right_upper(c, Y.f64(), N, N, k, G.f64(), k, Yn.f64(), N);
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

// max over columns j < nc of ||X[:, j]|| (FP64, one warp per column)
__global__ void colnorm_max_kernel(const double* X, int64_t m, int nc, unsigned long long* out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nc) return;
  double s = 0;
  for (int64_t i = lane; i < m; i += 32) s = fma(X[i + warp * m], X[i + warp * m], s);
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(sqrt(s))));
}

// One sketch pass: range finder with q power iterations from Omega, Rayleigh-Ritz, Jacobi.
struct Sketch {
  Tensor Q, Q2, X, J, Ss;  // Q, Q2: N x k; X = W (k x k); J (k x k); Ss sorted S (k)
  Tensor perm;             // int[k] stored in a double buffer
  int sweeps = 0;
};

Sketch sketch_pass(Ctx& c, const MatRef& R1, const MatRef& R2, const Tensor& Om, int q, const SvdParams& sp) {
  const int64_t N = R1.rows();
  const int k = int(Om.dims[1]);
  Sketch s;
  Tensor Y = apply(c, R1, 'N', apply(c, R2, 'N', Om));
  for (int it = 0; it < q; ++it) {
    Tensor Q = orth(c, Y, sp.inter_passes, nullptr);
    Tensor Z = orth(c, apply(c, R2, 'T', apply(c, R1, 'T', Q)), sp.inter_passes, nullptr);
    Y = apply(c, R1, 'N', apply(c, R2, 'N', Z));
  }
  s.Q = orth(c, Y, 3, nullptr);
  // B^T = M^T Q (N x k);  B^T = Q2 R  =>  B = R^T Q2^T
  Tensor Bt = apply(c, R2, 'T', apply(c, R1, 'T', s.Q));
  Tensor Rm;
  s.Q2 = orth(c, Bt, 3, &Rm);
  // X = R^T ; one-sided Jacobi: X J = W = Ux S  =>  U = Q Ux, V = Q2 J
  s.X = permute(c, Rm, {1, 0});
  s.J = c.alloc(DType::F64, {k, k});
  Tensor S = c.alloc(DType::F64, {k});
  int* d_sweeps = reinterpret_cast<int*>(static_cast<char*>(c.scal->p) + 3900);
  jacobi_svd_auto(c, s.X.f64(), k, k, k, s.J.f64(), k, S.f64(), sp.jacobi_max_sweeps, sp.jacobi_tol, d_sweeps);
  s.Ss = c.alloc(DType::F64, {k});
  s.perm = c.alloc(DType::F64, {(k + 1) / 2});
  sort_desc(c, S.f64(), k, s.Ss.f64(), static_cast<int*>(s.perm.data()));
  IPEPS_CUDA(cudaMemcpyAsync(&s.sweeps, d_sweeps, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  (void)N;
  return s;
}

}  // namespace

ProjResult get_projector(Ctx& c, const MatRef& R1, const MatRef& R2, int chi, const SvdParams& sp,
                         ProjCache* cache, bool keep_factors) {
  const int64_t N = R1.rows();
  IPEPS_CHECK(R1.cols() == R2.rows() && R2.cols() == N, "get_projector: R1*R2 must be square");
  IPEPS_CHECK(R1.t.dt == DType::F64 && R2.t.dt == DType::F64, "get_projector: real operands expected");
  const int new_chi = int(std::min<int64_t>(chi, R1.cols()));
  const int want = int(std::min<int64_t>(N, new_chi + 1));
  int over = std::max(sp.min_oversample, want * sp.oversample_num / std::max(sp.oversample_den, 1));
  int kw = int(std::min<int64_t>(N, int64_t(want) + over));
  // at most 128 columns when the minimum oversampling allows it: the Jacobi
  // then rotates all of its pairs (64) in one pass of its 64 half-warps
  if (kw > 128 && want + sp.min_oversample <= 128) kw = 128;
  const int k = kw;

  // sketch Omega (N x k): resolved right vectors of the previous call first, then Gaussian columns
  Tensor Om = c.alloc(DType::F64, {N, k});
  randn(c, Om);
  bool warm = false;
  if (sp.warm_start && cache && !cache->seed(sp.seed_older).empty() && cache->seed(sp.seed_older).dims[0] == N) {
    const Tensor& Vs = cache->seed(sp.seed_older);
    int nv = int(std::min<int64_t>(Vs.dims[1], k));
    IPEPS_CUDA(cudaMemcpyAsync(Om.data(), Vs.data(), size_t(N) * nv * 8, cudaMemcpyDeviceToDevice, c.stream));
    warm = true;
  }
  int q = (k == N) ? 0 : (warm ? sp.power_iters_warm : sp.power_iters);

  ProjResult r;
  r.k = k;
  Sketch sk;
  std::vector<double> all(k);
  int n = 0;
  Tensor Ux, Vk;
  int* d_perm = nullptr;
  double* d_res = reinterpret_cast<double*>(c.scal->p) + 48;
  double prev_res = 1e300;
  for (int attempt = 0;; ++attempt) {
    sk = sketch_pass(c, R1, R2, Om, q, sp);
    d_perm = static_cast<int*>(sk.perm.data());
    IPEPS_CUDA(cudaMemcpyAsync(all.data(), sk.Ss.data(), size_t(k) * 8, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    c.jacobi_sweeps += uint64_t(sk.sweeps);
    // cutoff_matrix (wrapper.jl:37-55)
    const double smax = all[0];
    int n_above = 0;
    for (int i = 0; i < k; ++i)
      if (smax > 0 && all[i] / smax > 1e-12) n_above++;
    n = std::min(new_chi, n_above);
    IPEPS_CHECK(n >= 1, "get_projector: no singular value above the cutoff (zero enlarged corner?)");
    // the reference's s has length N (full SVD); ours is the top-k part, k > n whenever N > n
    if (int64_t(N) > n && k > n) {
      if (std::fabs(all[n] - all[n - 1]) < 1e-10) n = n + 1;
    }
    IPEPS_CHECK(n <= k, "get_projector: truncation beyond the sketch");
    // Ux[:, j] = W[:, perm[j]] / S_sorted[j] (kept + one), Vk = Q2 J[:, perm]
    const int nc = std::min(n + 1, k);
    Ux = c.alloc(DType::F64, {k, nc});
    gather_cols(c, sk.X.f64(), k, k, d_perm, nc, sk.Ss.f64(), 2, Ux.f64(), k);
    Tensor Js = c.alloc(DType::F64, {k, k});
    gather_cols(c, sk.J.f64(), k, k, d_perm, k, nullptr, 0, Js.f64(), k);
    Vk = c.alloc(DType::F64, {N, k});
    gemm(c, DType::F64, 'N', 'N', N, k, k, cplx(1), sk.Q2.data(), N, Js.data(), k, cplx(0), Vk.data(), N, true);
    if (q == 0 && k == N) break;  // the sketch spans everything: exact
    if (attempt >= sp.max_extra_passes) break;
    // residual of the kept triplets: ||M v_i - s_i u_i|| <= resid_tol * s_1
    Tensor Vc = c.alloc(DType::F64, {N, nc});
    IPEPS_CUDA(cudaMemcpyAsync(Vc.data(), Vk.data(), size_t(N) * nc * 8, cudaMemcpyDeviceToDevice, c.stream));
    Tensor Res = apply(c, R1, 'N', apply(c, R2, 'N', Vc));
    Tensor Us = c.alloc(DType::F64, {k, nc});
    gather_cols(c, sk.X.f64(), k, k, d_perm, nc, nullptr, 0, Us.f64(), k);  // W = Ux S
    gemm(c, DType::F64, 'N', 'N', N, nc, k, cplx(-1), sk.Q.data(), N, Us.data(), k, cplx(1), Res.data(), N, true);
    IPEPS_CUDA(cudaMemsetAsync(d_res, 0, 8, c.stream));
    colnorm_max_kernel<<<(nc * 32 + 255) / 256, 256, 0, c.stream>>>(Res.f64(), N, nc,
                                                                    reinterpret_cast<unsigned long long*>(d_res));
    IPEPS_LAUNCH_CHECK();
    double res = 0;
    IPEPS_CUDA(cudaMemcpyAsync(&res, d_res, 8, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    // done when below tolerance, or when it stopped decreasing (the FP64 floor of
    // R1 (R2 v), ~eps ||R1|| ||R2||, can sit above resid_tol * s_1)
    if (res <= sp.resid_tol * smax || res > 0.5 * prev_res) break;
    prev_res = res;
    // not converged: one more power iteration from the current right vectors
    Om = Vk;
    q = 1;
    c.projector_extra_passes++;
  }
  r.sweeps = sk.sweeps;
  c.projector_calls++;
  r.n = n;
  r.s_host.assign(all.begin(), all.begin() + n);

  Tensor U = c.alloc(DType::F64, {N, n});
  gemm(c, DType::F64, 'N', 'N', N, n, k, cplx(1), sk.Q.data(), N, Ux.data(), k, cplx(0), U.data(), N, true);
  Tensor V = c.alloc(DType::F64, {N, n});
  IPEPS_CUDA(cudaMemcpyAsync(V.data(), Vk.data(), size_t(N) * n * 8, cudaMemcpyDeviceToDevice, c.stream));
  // resolved part of the sketch: s_a > 1e-13 s_1 (W/s is accurate there)
  int rr = 0;
  while (rr < k && all[rr] > 1e-13 * all[0]) ++rr;
  rr = std::max(rr, n);
  if (cache) {
    // seed for the next call of this direction: the resolved right vectors only
    // (near-null directions of this M say nothing about the next one)
    Tensor Vc = c.alloc(DType::F64, {N, rr});
    IPEPS_CUDA(cudaMemcpyAsync(Vc.data(), Vk.data(), size_t(N) * rr * 8, cudaMemcpyDeviceToDevice, c.stream));
    cache->Vold = cache->V;
    cache->V = Vc;
  }
  if (keep_factors) {
    r.r = rr;
    r.sr_host.assign(all.begin(), all.begin() + rr);
    Tensor Uxr = c.alloc(DType::F64, {k, rr});
    gather_cols(c, sk.X.f64(), k, k, d_perm, rr, sk.Ss.f64(), 2, Uxr.f64(), k);
    r.Ur = c.alloc(DType::F64, {N, rr});
    gemm(c, DType::F64, 'N', 'N', N, rr, k, cplx(1), sk.Q.data(), N, Uxr.data(), k, cplx(0), r.Ur.data(), N, true);
    r.Vr = c.alloc(DType::F64, {N, rr});
    IPEPS_CUDA(cudaMemcpyAsync(r.Vr.data(), Vk.data(), size_t(N) * rr * 8, cudaMemcpyDeviceToDevice, c.stream));
    r.Sr = c.alloc(DType::F64, {rr});
    IPEPS_CUDA(cudaMemcpyAsync(r.Sr.data(), sk.Ss.data(), size_t(rr) * 8, cudaMemcpyDeviceToDevice, c.stream));
  }

  r.S = c.alloc(DType::F64, {n});
  IPEPS_CUDA(cudaMemcpyAsync(r.S.data(), sk.Ss.data(), size_t(n) * 8, cudaMemcpyDeviceToDevice, c.stream));
  // P1 = R2 V S^-1/2 ; P2 = S^-1/2 U^T R1
  scale_cols(c, V.f64(), N, N, n, r.S.f64(), 1);
  scale_cols(c, U.f64(), N, N, n, r.S.f64(), 1);
  r.P1 = apply(c, R2, 'N', V);
  r.P2 = apply_left_T(c, U, R1, 'N');
  return r;
}

}  // namespace ipeps
