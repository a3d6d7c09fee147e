// Reverse-mode tape, backward rules, the truncated-SVD projector adjoint and
// the energy + gradient driver.
#include "ad.cuh"
#include "linalg.cuh"
#include "moves.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>

namespace ipeps {


constexpr double kSvdEta = 1e-12;  // broadening of svd_back (autodiff.jl:41-48)

// ------------------------------------------------------------------ kernels
namespace {

unsigned gridn(Ctx& c, int64_t n) {
  return unsigned(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, int64_t(c.sm_count) * 8)));
}

__device__ __forceinline__ double wsum(double v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// out[0] = sum x*y (deterministic: fixed grid, then one block)
__global__ void dot_partial_kernel(const double* x, const double* y, int64_t n, double* part) {
  double s = 0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    s = fma(x[i], y[i], s);
  s = wsum(s);
  __shared__ double sm[32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t += sm[w];
    part[blockIdx.x] = t;
  }
}

__global__ void sum_kernel(const double* part, int n, double* out) {
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  s = wsum(s);
  __shared__ double sm[32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t += sm[w];
    *out = t;
  }
}

// smallest index with |x_i| == m
__global__ void argmax_kernel(const double* x, int64_t n, const double* m, unsigned long long* idx) {
  const double mv = *m;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    if (fabs(x[i]) == mv) atomicMin(idx, static_cast<unsigned long long>(i));
}

// dx = dy/m - (dot/m^2) sign(x_k) e_k
__global__ void renorm_back_kernel(const double* dy, const double* x, int64_t n, const double* m,
                                   const unsigned long long* idx, const double* dot, double* dx) {
  const double mv = *m, inv = 1.0 / mv;
  const int64_t k = int64_t(*idx);
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double v = dy[i] * inv;
    if (i == k) v -= (*dot) * inv * inv * copysign(1.0, x[i]);
    dx[i] = v;
  }
}

// X[:, j] *= f(s[j]); mode 0: s, 1: 1/sqrt(s), 2: sqrt(s), 3: 1/s.  The inverse
// of a kept s of exactly 0 is taken as 0 (its projector column is zero).
__global__ void colscale_kernel(double* X, int64_t ld, int64_t m, int ncols, const double* s, int mode) {
  const int64_t tot = m * ncols;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < tot; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = t % m;
    const int j = int(t / m);
    const double v = s[j];
    const double f = mode == 0 ? v : mode == 2 ? sqrt(v) : v > 0.0 ? (mode == 1 ? 1.0 / sqrt(v) : 1.0 / v) : 0.0;
    X[i + j * ld] *= f;
  }
}

// out (N x n) = transpose of in (n x N) with columns scaled by 1/sqrt(s)
__global__ void transpose_scale_kernel(const double* in, int n, int64_t N, const double* s, double* out) {
  const int64_t tot = int64_t(n) * N;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < tot; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t a = t % N;
    const int i = int(t / N);
    out[a + i * N] = s[i] > 0.0 ? in[i + a * n] / sqrt(s[i]) : 0.0;
  }
}

// dS_i = -1/(2 s_i) (sum_a dP1[a,i] P1[a,i] + sum_j dP2[i,j] P2[i,j]); one warp per i
__global__ void dS_kernel(int n, int64_t N, const double* dP1, const double* P1, const double* dP2, const double* P2,
                          const double* s, double* dS) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int i = warp;
  double acc = 0;
  if (dP1)
    for (int64_t a = lane; a < N; a += 32) acc = fma(dP1[a + i * N], P1[a + i * N], acc);
  if (dP2)
    for (int64_t j = lane; j < N; j += 32) acc = fma(dP2[i + j * n], P2[i + j * n], acc);
  acc = wsum(acc);
  if (lane == 0) dS[i] = s[i] > 0.0 ? -0.5 * acc / s[i] : 0.0;
}

__device__ __forceinline__ double Fb(double x, double eta) { return x / (x * x + eta); }

// A_tt[i,j] = (J_ij + J_ji) s_j + s_i (K_ij + K_ji) + delta_ij dS_i,
// J = F o C1, K = F o C2, F_ij = f(s_j^2 - s_i^2)
__global__ void att_kernel(int n, const double* C1, const double* C2, const double* s, const double* dS, double eta,
                           double* A) {
  const int64_t tot = int64_t(n) * n;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < tot; t += int64_t(gridDim.x) * blockDim.x) {
    const int i = int(t % n), j = int(t / n);
    const double si = s[i], sj = s[j];
    const double Fij = Fb(sj * sj - si * si, eta), Fji = Fb(si * si - sj * sj, eta);
    const double J = (C1 ? Fij * C1[i + j * n] + Fji * C1[j + i * n] : 0.0);
    const double K = (C2 ? Fij * C2[i + j * n] + Fji * C2[j + i * n] : 0.0);
    A[i + j * n] = J * sj + si * K + (i == j ? dS[i] : 0.0);
  }
}

// G[a,i] = f(s_t[i]^2 - s_in[a]^2) C[a,i]  (a in-sketch discarded, i kept)
__global__ void fin_kernel(int nin, int n, const double* C, const double* s_in, const double* s_t, double eta,
                           double* G) {
  const int64_t tot = int64_t(nin) * n;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < tot; t += int64_t(gridDim.x) * blockDim.x) {
    const int a = int(t % nin), i = int(t / nin);
    G[a + int64_t(i) * nin] = Fb(s_t[i] * s_t[i] - s_in[a] * s_in[a], eta) * C[a + int64_t(i) * nin];
  }
}

// Chebyshev coefficient a_m(i) of the broadened resolvent on [0, b]:
// Re[1 / (s_i^2 - i sqrt(eta) - t)] = Re[(2/b) / (z - x)], x = 2t/b - 1,
// z = 2 (s_i^2 - i sqrt(eta)) / b - 1, and 1/(z - x) = sum_m e_m w^m T_m(x) / q
// with q = sqrt(z^2 - 1), w = z - q (|w| < 1), e_0 = 1, e_m = 2.
__device__ __forceinline__ double cheb_coef(double si, double eta, double b, int m) {
  const double zr = 2.0 * si * si / b - 1.0, zi = -2.0 * sqrt(eta) / b;
  // q = sqrt(z^2 - 1) (principal), then the root with |z - q| < 1
  const double ar = zr * zr - zi * zi - 1.0, ai = 2.0 * zr * zi;
  const double mod = hypot(ar, ai);
  double qr = sqrt(0.5 * (mod + ar)), qi = copysign(sqrt(fmax(0.0, 0.5 * (mod - ar))), ai);
  // w = z - q = 1 / (z + q), formed from the larger of |z + q|, |z - q| (no cancellation)
  double sr = zr + qr, si2 = zi + qi;
  const double dr = zr - qr, di = zi - qi;
  if (sr * sr + si2 * si2 < dr * dr + di * di) {
    qr = -qr;
    qi = -qi;
    sr = dr;
    si2 = di;
  }
  const double sd = sr * sr + si2 * si2;
  const double wr = sr / sd, wi = -si2 / sd;
  // (2/b) e_m w^m / q
  const double rw = hypot(wr, wi), tw = atan2(wi, wr);
  const double pm = pow(rw, double(m)), cr = pm * cos(m * tw), ci = pm * sin(m * tw);
  const double qq = qr * qr + qi * qi;
  const double re = (cr * qr + ci * qi) / qq;  // Re(w^m / q)
  return (m == 0 ? 1.0 : 2.0) * (2.0 / b) * re;
}

// X[:, i] += a_m(i) T[:, i]
__global__ void cheb_acc_kernel(double* X, const double* T, int64_t N, int n, const double* s, double eta, double b,
                                int m) {
  const int64_t tot = N * n;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < tot; t += int64_t(gridDim.x) * blockDim.x) {
    const int i = int(t / N);
    X[t] = fma(cheb_coef(s[i], eta, b, m), T[t], X[t]);
  }
}

__global__ void cheb_coef_max_kernel(const double* s, int n, double eta, double b, int m, double* out) {
  double mx = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) mx = fmax(mx, fabs(cheb_coef(s[i], eta, b, m)));
  for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (threadIdx.x == 0) *out = mx;
}

// Check of X[:, i] = f(s_i^2 - B) Y[:, i] through (x^2 + eta) f(x) = x:
//   rhs = s_i^2 Y - BY,   res = (s_i^4 + eta) X - 2 s_i^2 BX + B^2 X - rhs
__global__ void resolvent_check_kernel(const double* X, const double* BX, const double* BBX, const double* Y,
                                       const double* BY, const double* s, double eta, int64_t N, int n, double* res,
                                       double* rhs) {
  const int64_t tot = N * n;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < tot; t += int64_t(gridDim.x) * blockDim.x) {
    const double s2 = s[t / N] * s[t / N];
    const double r = fma(s2, Y[t], -BY[t]);
    rhs[t] = r;
    res[t] = fma(fma(s2, s2, eta), X[t], fma(-2.0 * s2, BX[t], BBX[t])) - r;
  }
}

// out[i] = sum_j X[i + j N]
__global__ void rowsum_kernel(const double* X, int64_t N, int n, double* out) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += int64_t(gridDim.x) * blockDim.x) {
    double a = 0;
    for (int j = 0; j < n; ++j) a += X[i + j * N];
    out[i] = a;
  }
}

// y = alpha * x + beta * y (elementwise over n doubles)
__global__ void axpby_kernel(double alpha, const double* x, double beta, double* y, int64_t n) {
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x)
    y[t] = fma(alpha, x[t], beta * y[t]);
}

}  // namespace

// ------------------------------------------------------------------ helpers
namespace {

double dot_host(Ctx& c, const Tensor& x, const Tensor& y) {
  const int64_t n = x.numel();
  const int blocks = int(std::min<int64_t>((n + 255) / 256, 1024));
  double* part = static_cast<double*>(c.workspace(size_t(std::max(blocks, 1)) * 8 + 64));
  double* out = reinterpret_cast<double*>(c.scal->p) + 32;
  dot_partial_kernel<<<std::max(blocks, 1), 256, 0, c.stream>>>(x.f64(), y.f64(), n, part);
  sum_kernel<<<1, 256, 0, c.stream>>>(part, std::max(blocks, 1), out);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Reduce, 2.0 * n, 16.0 * n);
  double h = 0;
  IPEPS_CUDA(cudaMemcpyAsync(&h, out, 8, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  return h;
}

// *out = sum x*y on the device (stream ordered, no host round trip)
void dot_dev(Ctx& c, const Tensor& x, const Tensor& y, double* out) {
  const int64_t n = x.numel();
  const int blocks = int(std::min<int64_t>((n + 255) / 256, 1024));
  double* part = static_cast<double*>(c.workspace(size_t(std::max(blocks, 1)) * 8 + 64));
  dot_partial_kernel<<<std::max(blocks, 1), 256, 0, c.stream>>>(x.f64(), y.f64(), n, part);
  sum_kernel<<<1, 256, 0, c.stream>>>(part, std::max(blocks, 1), out);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Reduce, 2.0 * n, 16.0 * n);
}

void colscale(Ctx& c, Tensor& X, const double* s, int ncols, int mode) {
  colscale_kernel<<<gridn(c, X.dims[0] * ncols), 256, 0, c.stream>>>(X.f64(), X.dims[0], X.dims[0], ncols, s, mode);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Elementwise, 0, 16.0 * X.dims[0] * ncols);
}

// view of columns [j0, j0+nc) of a column-major matrix
Tensor cols(const Tensor& X, int64_t j0, int64_t nc) {
  Tensor v = X;
  v.offset = X.offset + size_t(j0) * X.dims[0] * dtype_size(X.dt);
  v.nd = 2;
  v.dims[1] = nc;
  return v;
}

Tensor vec_view(const Tensor& s, int64_t i0, int64_t n) {
  Tensor v = s;
  v.offset = s.offset + size_t(i0) * 8;
  v.nd = 1;
  v.dims[0] = n;
  return v;
}

// C (m x n) = alpha op(A) op(B) + beta C on 2-D tensors (fresh output when C empty)
Tensor mm(Ctx& c, const Tensor& A, char oa, const Tensor& B, char ob, bool fp64 = false) {
  const int64_t m = (oa == 'N') ? A.dims[0] : A.dims[1];
  const int64_t k = (oa == 'N') ? A.dims[1] : A.dims[0];
  const int64_t n = (ob == 'N') ? B.dims[1] : B.dims[0];
  IPEPS_CHECK(((ob == 'N') ? B.dims[0] : B.dims[1]) == k, "ad mm: inner dimension mismatch");
  Tensor C = c.alloc(DType::F64, {m, n});
  gemm(c, DType::F64, oa, ob, m, n, k, cplx(1), A.data(), A.dims[0], B.data(), B.dims[0], cplx(0), C.data(), m, fp64);
  return C;
}

// op(R) X with R logical = t or t^T
Tensor Rapply(Ctx& c, const Tensor& Rt, bool rtrans, char op, const Tensor& X) {
  const bool t = (op == 'T') != rtrans;
  return mm(c, Rt, t ? 'T' : 'N', X, 'N');
}

Tensor hcat(Ctx& c, const Tensor& X, const Tensor& Y) {
  IPEPS_CHECK(X.dims[0] == Y.dims[0], "hcat: rows differ");
  const int64_t N = X.dims[0], a = X.numel() / N, b = Y.numel() / N;
  Tensor Z = c.alloc(DType::F64, {N, a + b});
  IPEPS_CUDA(cudaMemcpyAsync(Z.data(), X.data(), X.bytes(), cudaMemcpyDeviceToDevice, c.stream));
  IPEPS_CUDA(cudaMemcpyAsync(static_cast<char*>(Z.data()) + X.bytes(), Y.data(), Y.bytes(), cudaMemcpyDeviceToDevice,
                             c.stream));
  return Z;
}

// Y - U (U^T Y)
Tensor project_out(Ctx& c, const Tensor& U, const Tensor& Y) {
  Tensor Z = clone(c, Y);
  Tensor C = mm(c, U, 'T', Y, 'N', true);
  gemm(c, DType::F64, 'N', 'N', Z.dims[0], Z.dims[1], U.dims[1], cplx(-1), U.data(), U.dims[0], C.data(), C.dims[0],
       cplx(1), Z.data(), Z.dims[0], true);
  return Z;
}

int findl(const std::vector<int>& l, int x) {
  for (size_t i = 0; i < l.size(); ++i)
    if (l[i] == x) return int(i);
  return -1;
}

}  // namespace

// ------------------------------------------------------------------ tape
void Tape::acc(int id, const Tensor& gt0) {
  if (id < 0 || gt0.empty()) return;
  Tensor gt = gt0;
  Tensor& G = g_[id];
  if (G.empty()) {
    G = gt;
    return;
  }
  IPEPS_CHECK(G.numel() == gt.numel(), "tape: gradient size mismatch");
  if (G.buf.use_count() > 1) G = clone(c_, G);
  if (G.dt == DType::F64 && gt.dt == DType::C128) G = to_complex(c_, G);
  axpy(c_, cplx(1), gt, G);
}

void Tape::backward() {
  for (int i = int(ops_.size()) - 1; i >= 0; --i) ops_[i]();
  ops_.clear();
}

AV ad_tcon(Tape& tp, const AV& a, const std::vector<int>& la, const AV& b, const std::vector<int>& lb) {
  Ctx& c = tp.ctx();
  AV out{tcon(c, a.t, la, b.t, lb), -1};
  if (a.id < 0 && b.id < 0) return out;
  out.id = tp.newid();
  const int nout = out.t.nd;
  // dA = tcon(dC, lcA, B, lbA): output in A's leg order; B's free labels are summed
  std::vector<int> lcA(nout), lbA(lb.size()), lcB(nout), laB(la.size());
  for (int j = 0; j < nout; ++j) {
    const int l = -(j + 1);
    const int p = findl(la, l), q = findl(lb, l);
    lcA[j] = (p >= 0) ? -(p + 1) : 1000 + (j + 1);
    lcB[j] = (q >= 0) ? -(q + 1) : 2000 + (j + 1);
  }
  for (size_t q = 0; q < lb.size(); ++q) lbA[q] = (lb[q] > 0) ? -(findl(la, lb[q]) + 1) : 1000 - lb[q];
  for (size_t p = 0; p < la.size(); ++p) laB[p] = (la[p] > 0) ? -(findl(lb, la[p]) + 1) : 2000 - la[p];
  Tensor at = a.t, bt = b.t;
  const int ia = a.id, ib = b.id, io = out.id;
  tp.push([&tp, at, bt, ia, ib, io, lcA, lbA, lcB, laB]() {
    const Tensor& g = tp.grad(io);
    if (g.empty()) return;
    Ctx& c = tp.ctx();
    if (ia >= 0) tp.acc(ia, tcon(c, g, lcA, bt.dt == DType::C128 ? conj(c, bt) : bt, lbA));
    if (ib >= 0) tp.acc(ib, tcon(c, at.dt == DType::C128 ? conj(c, at) : at, laB, g, lcB));
  });
  return out;
}

AV ad_reshape(Tape& tp, const AV& a, const std::vector<int64_t>& s) {
  AV out{a.t.reshape(s), -1};
  if (a.id < 0) return out;
  out.id = tp.newid();
  const int ia = a.id, io = out.id;
  const std::vector<int64_t> shape = a.t.shape();
  tp.push([&tp, ia, io, shape]() {
    const Tensor& g = tp.grad(io);
    if (!g.empty()) tp.acc(ia, g.reshape(shape));
  });
  return out;
}

AV ad_permute(Tape& tp, const AV& a, const std::vector<int>& perm) {
  Ctx& c = tp.ctx();
  AV out{permute(c, a.t, perm), -1};
  if (a.id < 0) return out;
  out.id = tp.newid();
  std::vector<int> inv(perm.size());
  for (size_t i = 0; i < perm.size(); ++i) inv[perm[i]] = int(i);
  const int ia = a.id, io = out.id;
  tp.push([&tp, ia, io, inv]() {
    const Tensor& g = tp.grad(io);
    if (!g.empty()) tp.acc(ia, permute(tp.ctx(), g, inv));
  });
  return out;
}

// wrapper.jl:57: y = x / max|x|, differentiated through the maximum as Zygote does
AV ad_renorm(Tape& tp, const AV& a) {
  Ctx& c = tp.ctx();
  IPEPS_CHECK(a.t.dt == DType::F64, "ad_renorm: real tensors only");
  Tensor mk = c.alloc(DType::F64, {2});  // [0] = max|x|, [1] = argmax (as uint64 bits)
  double* d_m = mk.f64();
  maxabs(c, a.t, d_m);
  unsigned long long* d_k = reinterpret_cast<unsigned long long*>(d_m + 1);
  IPEPS_CUDA(cudaMemsetAsync(d_k, 0xff, 8, c.stream));
  const int64_t n = a.t.numel();
  argmax_kernel<<<gridn(c, n), 256, 0, c.stream>>>(a.t.f64(), n, d_m, d_k);
  IPEPS_LAUNCH_CHECK();
  AV out{clone(c, a.t), -1};
  scale_inv(c, out.t, d_m);
  if (a.id < 0) return out;
  out.id = tp.newid();
  const int ia = a.id, io = out.id;
  Tensor xt = a.t;
  tp.push([&tp, ia, io, xt, mk]() {
    const Tensor& g = tp.grad(io);
    if (g.empty()) return;
    Ctx& c = tp.ctx();
    const int64_t n = xt.numel();
    const int blocks = int(std::min<int64_t>((n + 255) / 256, 1024));
    double* part = static_cast<double*>(c.workspace(size_t(std::max(blocks, 1)) * 8 + 64));
    Tensor dot = c.alloc(DType::F64, {1});
    dot_partial_kernel<<<std::max(blocks, 1), 256, 0, c.stream>>>(g.f64(), xt.f64(), n, part);
    sum_kernel<<<1, 256, 0, c.stream>>>(part, std::max(blocks, 1), dot.f64());
    Tensor dx = c.alloc(DType::F64, xt.shape());
    renorm_back_kernel<<<gridn(c, n), 256, 0, c.stream>>>(
        g.f64(), xt.f64(), n, mk.f64(), reinterpret_cast<const unsigned long long*>(mk.f64() + 1), dot.f64(),
        dx.f64());
    IPEPS_LAUNCH_CHECK();
    c.count(KFam::Elementwise, 0, 24.0 * n);
    tp.acc(ia, dx);
  });
  return out;
}

// ------------------------------------------------------------------ projector
namespace {

// Backward of P1 = R2 V S^-1/2, P2 = S^-1/2 U^T R1 through (U, S, V) = the
// truncated SVD of M = R1 R2.  The reference differentiates the full SVD of M
// (svd_back, autodiff.jl:41-74) with zero cotangents on discarded columns:
//   dM = U_t A_tt V_t^T + sum_{i kept} [u_i a_i^T + b_i v_i^T]
//   a_i = M^T R_i du_i + s_i R'_i dv_i,   b_i = s_i R_i du_i + M R'_i dv_i
// with R_i = sum_{a discarded} f(s_i^2 - s_a^2) u_a u_a^T, f(x) = x/(x^2+eta)
// (R'_i the same with v_a).  Discarded pairs resolved by the sketch (a <= r)
// are summed exactly; the rest of the spectrum (s_a <= s_{r+1}) enters through
// the Taylor series of f in M M^T (resp. M^T M) on the complement of the
// resolved vectors, which converges like (s_{r+1}/s_i)^2.
void projector_backward(Ctx& c, const Tensor& R1t, bool t1, const Tensor& R2t, bool t2, const ProjResult& pr,
                        const Tensor& P1, const Tensor& P2, const Tensor& dP1in, const Tensor& dP2in, Tensor* dR1t,
                        Tensor* dR2t) {
  // R1: N1 x K1, R2: K1 x N2 (rectangular when the boundaries' bond
  // dimensions differ); U: N1 x n, V: N2 x n, P1: K1 x n, P2: n x K1
  const int n = pr.n, r = pr.r;
  const int64_t N1 = pr.Ur.dims[0], N2 = pr.Vr.dims[0], K1 = P1.dims[0];
  IPEPS_CHECK(P2.dims[1] == K1, "projector_backward: P1/P2 shapes differ");
  Tensor Ut = cols(pr.Ur, 0, n), Vt = cols(pr.Vr, 0, n);
  Tensor s = vec_view(pr.Sr, 0, n);
  Tensor dP1 = dP1in.empty() ? c.zeros(DType::F64, {K1, n}) : dP1in.reshape({K1, n});
  Tensor dP2 = dP2in.empty() ? c.zeros(DType::F64, {n, K1}) : dP2in.reshape({n, K1});
  // dU_t = R1 dP2^T S^-1/2,  dV_t = R2^T dP1 S^-1/2
  Tensor dUt = c.alloc(DType::F64, {N1, n});
  gemm(c, DType::F64, t1 ? 'T' : 'N', 'T', N1, n, K1, cplx(1), R1t.data(), R1t.dims[0], dP2.data(), n, cplx(0),
       dUt.data(), N1);
  colscale(c, dUt, s.f64(), n, 1);
  Tensor dVt = Rapply(c, R2t, t2, 'T', dP1);
  colscale(c, dVt, s.f64(), n, 1);
  // dS
  Tensor dS = c.alloc(DType::F64, {n});
  dS_kernel<<<(n * 32 + 255) / 256, 256, 0, c.stream>>>(n, K1, dP1.f64(), P1.f64(), dP2.f64(), P2.f64(), s.f64(),
                                                         dS.f64());
  IPEPS_LAUNCH_CHECK();
  // kept x kept block
  Tensor C1 = mm(c, Ut, 'T', dUt, 'N', true), C2 = mm(c, Vt, 'T', dVt, 'N', true);
  Tensor Att = c.alloc(DType::F64, {n, n});
  att_kernel<<<gridn(c, int64_t(n) * n), 256, 0, c.stream>>>(n, C1.f64(), C2.f64(), s.f64(), dS.f64(), kSvdEta,
                                                             Att.f64());
  IPEPS_LAUNCH_CHECK();
  // W1 = V_t A_tt^T ; Acol, Bcol accumulate the discarded couplings
  Tensor W1 = mm(c, Vt, 'N', Att, 'T', true);
  Tensor Bcol = c.zeros(DType::F64, {N1, n});
  Tensor VinGv_plus_Xv = c.zeros(DType::F64, {N2, n});  // (V_in G_v + X_v), later scaled by s_t
  Tensor UinGu_plus_Xu = c.zeros(DType::F64, {N1, n});  // (U_in G_u + X_u), later scaled by s_t
  if (r > n) {
    const int nin = r - n;
    Tensor Uin = cols(pr.Ur, n, nin), Vin = cols(pr.Vr, n, nin);
    Tensor sin = vec_view(pr.Sr, n, nin);
    Tensor Cu = mm(c, Uin, 'T', dUt, 'N', true), Cv = mm(c, Vin, 'T', dVt, 'N', true);
    Tensor Gu = c.alloc(DType::F64, {nin, n}), Gv = c.alloc(DType::F64, {nin, n});
    fin_kernel<<<gridn(c, int64_t(nin) * n), 256, 0, c.stream>>>(nin, n, Cu.f64(), sin.f64(), s.f64(), kSvdEta,
                                                                 Gu.f64());
    fin_kernel<<<gridn(c, int64_t(nin) * n), 256, 0, c.stream>>>(nin, n, Cv.f64(), sin.f64(), s.f64(), kSvdEta,
                                                                 Gv.f64());
    IPEPS_LAUNCH_CHECK();
    // Acol += V_in diag(s_in) G_u ; Bcol += U_in diag(s_in) G_v
    Tensor sGu = clone(c, Gu), sGv = clone(c, Gv);
    scale_rows(c, sGu.f64(), nin, nin, n, sin.f64(), 0);
    scale_rows(c, sGv.f64(), nin, nin, n, sin.f64(), 0);
    gemm(c, DType::F64, 'N', 'N', N2, n, nin, cplx(1), Vin.data(), N2, sGu.data(), nin, cplx(1), W1.data(), N2, true);
    gemm(c, DType::F64, 'N', 'N', N1, n, nin, cplx(1), Uin.data(), N1, sGv.data(), nin, cplx(1), Bcol.data(), N1, true);
    gemm(c, DType::F64, 'N', 'N', N2, n, nin, cplx(1), Vin.data(), N2, Gv.data(), nin, cplx(0), VinGv_plus_Xv.data(),
         N2, true);
    gemm(c, DType::F64, 'N', 'N', N1, n, nin, cplx(1), Uin.data(), N1, Gu.data(), nin, cplx(0), UinGu_plus_Xu.data(),
         N1, true);
  }
  // complement of the resolved vectors: Chebyshev expansion of the broadened
  // resolvent f_i(t) = Re[1 / (s_i^2 - i sqrt(eta) - t)] over the unresolved
  // spectrum t in [0, b] of B = P M M^T P (resp. P' M^T M P').  The
  // coefficients decay like |w_i|^m with w_i set by s_i^2 / b alone; the
  // recursion T_{m+1} = 2 B~ T_m - T_{m-1} (B~ = (2/b) B - 1) keeps
  // |T_m| <= |T_0| while the spectrum lies in [0, b].  b must bound the
  // spectrum: the sketch's estimate of the first unresolved singular value is a
  // Ritz value, i.e. a lower bound, so b also covers a power-iteration estimate
  // of the top of B, and every result is checked through the identity
  // (x^2 + eta) f(x) = x, i.e. ((s_i^2 - B)^2 + eta) X_i = (s_i^2 - B) Y_i;
  // a failed check redoes the expansion over a wider interval.
  {
    Tensor Ur = pr.Ur, Vr = pr.Vr;
    const Tensor Yu0 = project_out(c, Ur, dUt), Yv0 = project_out(c, Vr, dVt);
    double* d_cmax = reinterpret_cast<double*>(c.scal->p) + 40;
    constexpr int kMaxTerms = 160;
    constexpr double kTol = 1e-11;
    constexpr double kCheckTol = 1e-10;
    constexpr int kCheckEvery = 4;
    const double ny0 = std::sqrt(dot_host(c, Yu0, Yu0) + dot_host(c, Yv0, Yv0));
    Tensor Xu = c.zeros(DType::F64, {N1, n}), Xv = c.zeros(DType::F64, {N2, n});
    // M = R1 R2 formed once (N1 x N2): each application of M M^T or M^T M is
    // then two products instead of four
    Tensor Mx = c.alloc(DType::F64, {N1, N2});
    gemm(c, DType::F64, t1 ? 'T' : 'N', t2 ? 'T' : 'N', N1, N2, K1, cplx(1), R1t.data(), R1t.dims[0], R2t.data(),
         R2t.dims[0], cplx(0), Mx.data(), N1);
    // M_P = (1 - U_r U_r^T) M (1 - V_r V_r^T), formed once.  For vectors in the
    // complement, P M M^T P = M_P M_P^T + (P M V_r)(P M V_r)^T, and P M V_r is
    // the resolved triplets' residual (<= 1e-10 s_1 each), so B = M_P M_P^T
    // (resp. M_P^T M_P) up to ~1e-20 s_1^2 and keeps the complement by
    // construction: the expansion's terms need no projection.
    Tensor MP = clone(c, Mx);
    {
      const int64_t rr = Ur.dims[1];
      Tensor C1 = mm(c, Ur, 'T', Mx, 'N', true);  // rr x N2
      gemm(c, DType::F64, 'N', 'N', N1, N2, rr, cplx(-1), Ur.data(), N1, C1.data(), rr, cplx(1), MP.data(), N1,
           true);
      Tensor C2 = mm(c, MP, 'N', Vr, 'N', true);  // N1 x rr
      gemm(c, DType::F64, 'N', 'T', N1, N2, rr, cplx(-1), C2.data(), N1, Vr.data(), N2, cplx(1), MP.data(), N1,
           true);
    }
    auto Bu_of = [&](const Tensor& T) { return mm(c, MP, 'N', mm(c, MP, 'T', T, 'N', true), 'N', true); };
    auto Bv_of = [&](const Tensor& T) { return mm(c, MP, 'T', mm(c, MP, 'N', T, 'N', true), 'N', true); };
    bool series_done = (ny0 == 0.0);
    if (!series_done) {
      // b: above the sketch's s_next^2 and a power-iteration estimate of the
      // top of B (six steps on the sum of the u-side cotangent columns), kept
      // below the smallest kept s_n^2 so that every resolvent's pole lies outside [0, b]
      const double lam = pr.s_next * pr.s_next, sn2 = pr.sr_host[n - 1] * pr.sr_host[n - 1];
      double est = 0;
      {
        Tensor t = c.alloc(DType::F64, {N1, 1});
        rowsum_kernel<<<gridn(c, N1), 256, 0, c.stream>>>(Yu0.f64(), N1, n, t.f64());
        IPEPS_LAUNCH_CHECK();
        double nt = std::sqrt(dot_host(c, t, t));
        for (int it = 0; it < 6 && nt > 0; ++it) {
          Tensor bt = Bu_of(t);
          const double nb = std::sqrt(dot_host(c, bt, bt));
          est = nb / nt;
          t = bt;
          nt = nb;
        }
      }
      // b is at least the rounding level of B (~eps s_1^2): below it the
      // recursion would amplify rounding noise.  Kept s_n^2 under that floor
      // are far inside the broadening (f(x) ~ x / eta there, the pole
      // sqrt(eta) off the real axis), so the expansion converges all the same.
      const double s1 = pr.sr_host[0], bfloor = 1e-14 * s1 * s1;
      const double top = std::max(lam, est);
      double b = std::max({1.25 * lam, 1.2 * est, bfloor});
      if (b >= sn2 && sn2 > bfloor) b = std::max(top < sn2 ? 0.5 * (top + sn2) : top, bfloor);
      // One term's products with M, the u and v sides batched into two GEMMs of
      // 2n columns: W1 = M^T [T_u | M T_v] = [M^T T_u | M^T M T_v], then, with the
      // next v-side vector T_v' formed from the second half,
      // W2 = M [M^T T_u | T_v'] = [M M^T T_u | M T_v'], whose second half feeds the
      // next term (with M_P in place of M).  B~ T = (2/b) B T - T,
      // T_{m+1} = 2 B~ T_m - T_{m-1}.
      Tensor W1 = c.alloc(DType::F64, {N2, 2 * int64_t(n)}), W2 = c.alloc(DType::F64, {N1, 2 * int64_t(n)});
      Tensor BYu, BYv;
      auto next_T = [&](Tensor& B, const Tensor& T, const Tensor& Tprev, int m) {
        axpby_kernel<<<gridn(c, B.numel()), 256, 0, c.stream>>>(-1.0, T.f64(), 2.0 / b, B.f64(), B.numel());
        if (m > 0) axpby_kernel<<<gridn(c, B.numel()), 256, 0, c.stream>>>(-1.0, Tprev.f64(), 2.0, B.f64(), B.numel());
        IPEPS_LAUNCH_CHECK();
      };
      auto apply_B = [&](const Tensor& Tu, const Tensor& Tv, const Tensor& Pu, const Tensor& Pv, int m, Tensor* Bu,
                         Tensor* Bv) {
        IPEPS_CUDA(cudaMemcpyAsync(W2.data(), Tu.data(), size_t(N1) * n * 8, cudaMemcpyDeviceToDevice, c.stream));
        gemm(c, DType::F64, 'T', 'N', N2, 2 * n, N1, cplx(1), MP.data(), N1, W2.data(), N1, cplx(0), W1.data(), N2,
             true);
        // the next v-side vector in place (it feeds the second product), and a copy to keep
        Tensor zv = cols(W1, n, n);
        if (m == 0) BYv = clone(c, zv);  // B Y_0 on the v side, for the resolvent check
        next_T(zv, Tv, Pv, m);
        *Bv = clone(c, zv);
        gemm(c, DType::F64, 'N', 'N', N1, 2 * n, N2, cplx(1), MP.data(), N1, W1.data(), N2, cplx(0), W2.data(), N1,
             true);
        *Bu = clone(c, cols(W2, 0, n));
        if (m == 0) BYu = clone(c, *Bu);  // B Y_0 on the u side
        next_T(*Bu, Tu, Pu, m);
      };
      // relative residual of ((s_i^2 - B)^2 + eta) X_i = (s_i^2 - B) Y_i over all columns of one side
      auto check = [&](const Tensor& X, const Tensor& Y, const Tensor& BY, bool u_side) {
        auto B = [&](const Tensor& T) { return u_side ? Bu_of(T) : Bv_of(T); };
        const Tensor BX = B(X), BBX = B(BX);
        Tensor res = c.alloc(DType::F64, X.shape()), rhs = c.alloc(DType::F64, X.shape());
        resolvent_check_kernel<<<gridn(c, X.numel()), 256, 0, c.stream>>>(
            X.f64(), BX.f64(), BBX.f64(), Y.f64(), BY.f64(), s.f64(), kSvdEta, X.dims[0], n, res.f64(), rhs.f64());
        IPEPS_LAUNCH_CHECK();
        const double nr = dot_host(c, rhs, rhs);
        return nr > 0 ? std::sqrt(dot_host(c, res, res) / nr) : 0.0;
      };
      for (int attempt = 0; attempt < 6; ++attempt) {
        Xu = c.zeros(DType::F64, {N1, n});
        Xv = c.zeros(DType::F64, {N2, n});
        Tensor Pu = Yu0, Pv = Yv0;  // T_{m-1}
        Tensor Tu = Yu0, Tv = Yv0;  // T_m
        bool blew_up = false, converged = false;
        // M_P T_v of the first term, in the second half of W2
        gemm(c, DType::F64, 'N', 'N', N1, n, N2, cplx(1), MP.data(), N1, Tv.data(), N2, cplx(0),
             cols(W2, n, n).data(), N1, true);
        for (int m = 0; m < kMaxTerms; ++m) {
          cheb_acc_kernel<<<gridn(c, N1 * n), 256, 0, c.stream>>>(Xu.f64(), Tu.f64(), N1, n, s.f64(), kSvdEta, b, m);
          cheb_acc_kernel<<<gridn(c, N2 * n), 256, 0, c.stream>>>(Xv.f64(), Tv.f64(), N2, n, s.f64(), kSvdEta, b, m);
          IPEPS_LAUNCH_CHECK();
          c.series_terms++;
          // the stopping tests read back five device scalars every kCheckEvery terms
          // (one host round trip instead of five per term)
          if (m % kCheckEvery == kCheckEvery - 1 || m == kMaxTerms - 1) {
            cheb_coef_max_kernel<<<1, 32, 0, c.stream>>>(s.f64(), n, kSvdEta, b, m + 1, d_cmax);
            IPEPS_LAUNCH_CHECK();
            dot_dev(c, Tu, Tu, d_cmax + 1);
            dot_dev(c, Tv, Tv, d_cmax + 2);
            dot_dev(c, Xu, Xu, d_cmax + 3);
            dot_dev(c, Xv, Xv, d_cmax + 4);
            double h[5];
            IPEPS_CUDA(cudaMemcpyAsync(h, d_cmax, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
            c.sync();
            if (std::sqrt(h[1] + h[2]) > 8.0 * ny0) {
              blew_up = true;  // spectrum beyond b
              break;
            }
            // |T_m| <= |T_0| on [0, b]: the remaining terms are bounded by the coefficient tail
            if (h[0] * ny0 <= kTol * std::sqrt(h[3] + h[4])) {
              converged = true;
              break;
            }
          }
          Tensor Bu, Bv;
          apply_B(Tu, Tv, Pu, Pv, m, &Bu, &Bv);
          Pu = Tu;
          Pv = Tv;
          Tu = Bu;
          Tv = Bv;
        }
        if (converged && std::max(check(Xu, Yu0, BYu, true), check(Xv, Yv0, BYv, false)) <= kCheckTol) {
          series_done = true;
          break;
        }
        if (!converged && !blew_up) break;  // term cap: counted below
        // the spectrum reaches beyond b: widen the interval, still below s_n^2
        c.series_retries++;
        const double sn2w = sn2 > b ? sn2 : 2.0 * b;
        b = (2.0 * b < sn2w) ? 2.0 * b : 0.5 * (b + sn2w);
      }
    }
    // the expansion stopped at its term cap or never passed its check: the
    // discarded spectrum's share of the gradient is left out (counted in
    // ipeps_stats_t, bit 16 of the status word) rather than taken from a
    // diverging partial sum
    if (!series_done) {
      c.series_cap_hits++;
      flag_status(c, 16);
      Xu = c.zeros(DType::F64, {N1, n});
      Xv = c.zeros(DType::F64, {N2, n});
    }
    // Acol += M^T X_u ; Bcol += M X_v ; and the s_t-scaled terms
    Tensor MtXu = mm(c, Mx, 'T', Xu, 'N');
    axpy(c, cplx(1), MtXu, W1);
    Tensor MXv = mm(c, Mx, 'N', Xv, 'N');
    axpy(c, cplx(1), MXv, Bcol);
    axpy(c, cplx(1), Xv, VinGv_plus_Xv);
    axpy(c, cplx(1), Xu, UinGu_plus_Xu);
  }
  colscale(c, VinGv_plus_Xv, s.f64(), n, 0);
  colscale(c, UinGu_plus_Xu, s.f64(), n, 0);
  axpy(c, cplx(1), VinGv_plus_Xv, W1);    // W1 = V_t A_tt^T + Acol
  axpy(c, cplx(1), UinGu_plus_Xu, Bcol);  // Bcol complete
  // dR1 = U_t [ (R2 W1)^T + S^-1/2 dP2 ] + Bcol (R2 V_t)^T,   R2 V_t = P1 S^1/2
  Tensor Z = Rapply(c, R2t, t2, 'N', W1);
  Tensor dP2T = c.alloc(DType::F64, {K1, n});
  transpose_scale_kernel<<<gridn(c, K1 * n), 256, 0, c.stream>>>(dP2.f64(), n, K1, s.f64(), dP2T.f64());
  IPEPS_LAUNCH_CHECK();
  axpy(c, cplx(1), dP2T, Z);
  Tensor BcolS = clone(c, Bcol);
  colscale(c, BcolS, s.f64(), n, 2);
  Tensor L1 = hcat(c, Ut, BcolS), Rm1 = hcat(c, Z, P1);
  // dR2 = (P2^T S^1/2) W1^T + (R1^T Bcol + dP1 S^-1/2) V_t^T
  Tensor P2T = permute(c, P2, {1, 0});
  colscale(c, P2T, s.f64(), n, 2);
  Tensor Y2 = Rapply(c, R1t, t1, 'T', Bcol);
  Tensor dP1s = clone(c, dP1);
  colscale(c, dP1s, s.f64(), n, 1);
  axpy(c, cplx(1), dP1s, Y2);
  Tensor L2 = hcat(c, P2T, Y2), Rm2 = hcat(c, W1, Vt);
  // gradients of the stored tensors (logical R = t^T when transposed)
  *dR1t = t1 ? mm(c, Rm1, 'N', L1, 'T') : mm(c, L1, 'N', Rm1, 'T');
  *dR2t = t2 ? mm(c, Rm2, 'N', L2, 'T') : mm(c, L2, 'N', Rm2, 'T');
}

}  // namespace

void ad_projector(Tape& tp, const AV& R1, bool t1, const AV& R2, bool t2, const ProjResult& pr, AV* P1, AV* P2) {
  Ctx& c = tp.ctx();
  const int n = pr.n;
  Tensor Ut = cols(pr.Ur, 0, n), Vt = cols(pr.Vr, 0, n);
  Tensor s = vec_view(pr.Sr, 0, n);
  Tensor Vs = clone(c, Vt), Us = clone(c, Ut);
  colscale(c, Vs, s.f64(), n, 1);
  colscale(c, Us, s.f64(), n, 1);
  P1->t = Rapply(c, R2.t, t2, 'N', Vs);
  P2->t = mm(c, Us, 'T', R1.t, t1 ? 'T' : 'N');
  P1->id = tp.newid();
  P2->id = tp.newid();
  const int i1 = R1.id, i2 = R2.id, o1 = P1->id, o2 = P2->id;
  Tensor R1t = R1.t, R2t = R2.t, P1t = P1->t, P2t = P2->t;
  ProjResult prc = pr;
  tp.push([&tp, R1t, t1, R2t, t2, prc, P1t, P2t, i1, i2, o1, o2]() {
    const Tensor &g1 = tp.grad(o1), &g2 = tp.grad(o2);
    if (g1.empty() && g2.empty()) return;
    Tensor dR1, dR2;
    Ctx& cx = tp.ctx();
    if (cx.prof) cx.sync();
    const auto t0 = std::chrono::steady_clock::now();
    projector_backward(cx, R1t, t1, R2t, t2, prc, P1t, P2t, g1, g2, &dR1, &dR2);
    if (cx.prof) {
      cx.sync();
      cx.ad_phase_ms[4] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    tp.acc(i1, dR1);
    tp.acc(i2, dR2);
  });
}

// ------------------------------------------------------------------ driver
namespace {

struct IterCk {
  std::array<Tensor, 4> Cs, Es;
  std::array<ProjResult, 4> proj;
};

}  // namespace

namespace {

__global__ void real_part_kernel(const double2* x, double* y, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[i] = x[i].x;
}

// the cotangent of a real variable from a possibly complex one: its real part
Tensor real_of(Ctx& c, const Tensor& x) {
  if (x.empty() || x.dt == DType::F64) return x;
  Tensor y = c.alloc(DType::F64, x.shape());
  const int64_t n = x.numel();
  const unsigned g = unsigned(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, int64_t(c.sm_count) * 8)));
  real_part_kernel<<<g, 256, 0, c.stream>>>(static_cast<const double2*>(x.data()), y.f64(), n);
  IPEPS_LAUNCH_CHECK();
  return y;
}

std::complex<double> scalar_host(Ctx& c, const Tensor& t) {
  double h[2] = {0, 0};
  IPEPS_CUDA(cudaMemcpyAsync(h, t.data(), t.dt == DType::F64 ? 8 : 16, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  return {h[0], t.dt == DType::F64 ? 0.0 : h[1]};
}

// a one-element cotangent of dtype dt with value v (the real part when dt is real)
Tensor scalar_seed(Ctx& c, const Tensor& like, std::complex<double> v) {
  Tensor g = c.alloc(like.dt, like.shape());
  const double h[2] = {v.real(), v.imag()};
  IPEPS_CUDA(cudaMemcpyAsync(g.data(), h, like.dt == DType::F64 ? 8 : 16, cudaMemcpyHostToDevice, c.stream));
  c.sync();
  return g;
}

}  // namespace

namespace {
// wall-clock phase timer of the pullback, active only while profiling (it
// synchronises the stream at each mark)
struct PhaseClock {
  Ctx& c;
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  explicit PhaseClock(Ctx& cc) : c(cc) {
    if (c.prof) c.sync();
    t = std::chrono::steady_clock::now();
  }
  void mark(int phase) {
    if (!c.prof) return;
    c.sync();
    const auto t1 = std::chrono::steady_clock::now();
    c.ad_phase_ms[size_t(phase)] += std::chrono::duration<double, std::milli>(t1 - t).count();
    t = t1;
  }
};
}  // namespace

double energy_grad(Env& e, const Tensor& Hh, const Tensor& Hv, int ad_iters, Tensor* gA, const H4* h4) {
  Ctx& c = *e.ctx;
  PhaseClock clock(c);
  IPEPS_CHECK(e.dt == DType::F64 && !e.nested, "energy_grad: real single-site A only");
  // The pullback runs in FP64 in both forms.  Measured at Heisenberg D=5
  // chi=100: with 3xTF32 contractions in the tape's backward (checkpoints and
  // projector adjoint in FP64) the gradient moves by 2.5e-5 relative, with the
  // whole pullback in 3xTF32 by 3.3e-5, against a 1e-6 requirement; FP32-level
  // cotangent errors reach the gradient through the adjoint's 1/(s_i^2 - s_j^2)
  // terms.  The mixed form gains its speed in the iterations before this call.
  Fp64Scope fp64_all(c);
  // forward: ad_iters iterations with checkpoints of C/T and the projector
  // factors; the singular triplets the adjoint uses are resolved to a residual
  // of 1e-12 s_1 (the gradient of the reference's exact SVD is reproduced to
  // ~1e-7 instead of the ~1e-6 a 1e-10 residual leaves)
  std::vector<IterCk> ck;
  const double resid_tol0 = e.prm.svd.resid_tol;
  struct RestoreTol {
    Env& e;
    double v;
    ~RestoreTol() { e.prm.svd.resid_tol = v; }
  } restore_tol{e, resid_tol0};
  e.prm.svd.resid_tol = std::min(resid_tol0, 1e-12);
  const int max_extra0 = e.prm.svd.max_extra_passes;
  struct RestoreExtra {
    Env& e;
    int v;
    ~RestoreExtra() { e.prm.svd.max_extra_passes = v; }
  } restore_extra{e, max_extra0};
  e.prm.svd.max_extra_passes = std::max(max_extra0, 12);
  {
    std::complex<double> conv = 1.0;
    for (int i = 1; i <= ad_iters; ++i) {
      IterCk k;
      k.Cs = e.Cs;
      k.Es = e.Es;
      ctm_moves4(e, k.proj.data());
      ck.push_back(std::move(k));
      // run_ctm's early exit (ctmrg.jl:44) can only trigger once i >= min_iter
      auto energy_now = [&]() {
        if (h4) return gs_energy_4x4(e, *h4);
        std::complex<double> E, Na;
        gs_energy(e, Hh, Hv, &E, &Na);
        return E;
      };
      if (i >= e.prm.min_iter && i < ad_iters) {
        const std::complex<double> E = energy_now();
        const double diff = std::abs(E - conv);
        conv = E;
        if (diff < e.prm.rg_tol) break;
      } else if (i < ad_iters && e.prm.min_iter < ad_iters) {
        conv = energy_now();
      }
    }
  }
  e.prm.svd.resid_tol = resid_tol0;
  e.prm.svd.max_extra_passes = max_extra0;
  clock.mark(0);
  // energy on a tape (evaluation.jl:15-29)
  std::array<Tensor, 4> gC, gE;
  Tensor gAcc, gAdc;
  double Ere = 0;
  {
    Tape tp(c);
    const int prec_bw = c.precision;
    c.precision = kPrecFP64;  // the energy and its seed in FP64 in both forms
    ADPolicy p{tp};
    AV C[4], E[4];
    for (int i = 0; i < 4; ++i) {
      C[i] = tp.leaf(e.Cs[i]);
      E[i] = tp.leaf(e.Es[i]);
    }
    AV A = tp.leaf(e.A), Ad = tp.leaf(e.Ad);
    if (h4) {
      // get_gs_energy_4x4 (evaluation.jl:339-356): Re(en / nrm), both on the
      // tape; seeds conj(1 / nrm) and conj(-en / nrm^2)
      Arr4<ADPolicy> sv, As{A, A, A, A}, Ads{Ad, Ad, Ad, Ad};
      for (int k = 0; k < 4; ++k) sv[k] = tp.constant((*h4)[k]);
      Arr4<ADPolicy> op = get_op_Ad4(p, sv, Ads);
      auto en = energy_norm_4x4(p, C[0], C[1], C[2], C[3], E[0], E[0], E[1], E[1], E[2], E[2], E[3], E[3], As,
                                Ads, op);
      const std::complex<double> ev = scalar_host(c, en[0].t), nv = scalar_host(c, en[1].t);
      Ere = (ev / nv).real();
      tp.acc(en[0].id, scalar_seed(c, en[0].t, std::conj(1.0 / nv)));
      tp.acc(en[1].id, scalar_seed(c, en[1].t, std::conj(-ev / (nv * nv))));
      c.precision = prec_bw;
      tp.backward();
      // every variable is real: the real parts of the cotangents
      for (int i = 0; i < 4; ++i) {
        gC[i] = real_of(c, tp.grad(C[i].id));
        gE[i] = real_of(c, tp.grad(E[i].id));
      }
      gAcc = real_of(c, tp.grad(A.id));
      gAdc = real_of(c, tp.grad(Ad.id));
    } else {
    AV roh = get_dm_h(p, C[0], C[1], C[2], C[3], E[0], E[0], E[1], E[2], E[2], E[3], A, A, Ad, Ad);
    AV rov = get_dm_v(p, C[0], C[1], C[2], C[3], E[0], E[1], E[1], E[2], E[3], E[3], A, A, Ad, Ad);
    auto t = dm_traces(c, {{roh.t, Hh}, {rov.t, Hv}});
    const std::complex<double> Eh = t[0].trH / t[0].tr, Ev = t[1].trH / t[1].tr;
    Ere = (Eh + Ev).real();
    // seed: d Re(E_x) / d rho = (Re H^T - Re(E_x) I) / tr(rho)   (rho real)
    auto seed = [&](const Tensor& H, const Tensor& rho, std::complex<double> Ex, double Nx) {
      const int d2 = int(rho.dims[0]);
      std::vector<double> hH(size_t(d2) * d2 * 2), g(size_t(d2) * d2);
      IPEPS_CUDA(cudaMemcpyAsync(hH.data(), H.data(), hH.size() * 8, cudaMemcpyDeviceToHost, c.stream));
      c.sync();
      for (int a = 0; a < d2; ++a)
        for (int b = 0; b < d2; ++b)
          g[a + size_t(b) * d2] = (hH[2 * (b + size_t(a) * d2)] - (a == b ? Ex.real() : 0.0)) / Nx;
      Tensor gt = c.alloc(DType::F64, {d2, d2});
      IPEPS_CUDA(cudaMemcpyAsync(gt.data(), g.data(), g.size() * 8, cudaMemcpyHostToDevice, c.stream));
      return gt;
    };
    IPEPS_CHECK(roh.t.dt == DType::F64, "energy_grad: real density matrices expected");
    tp.acc(roh.id, seed(Hh, roh.t, Eh, t[0].tr.real()));
    tp.acc(rov.id, seed(Hv, rov.t, Ev, t[1].tr.real()));
    c.precision = prec_bw;
    tp.backward();
    for (int i = 0; i < 4; ++i) {
      gC[i] = tp.grad(C[i].id);
      gE[i] = tp.grad(E[i].id);
    }
    gAcc = tp.grad(A.id);
    gAdc = tp.grad(Ad.id);
    }
  }
  clock.mark(1);
  // reverse over the iterations, recomputing each on a tape
  for (int it = int(ck.size()) - 1; it >= 0; --it) {
    Tape tp(c);
    ADPolicy p{tp};
    Arr4<ADPolicy> C, E;
    AV leafC[4], leafE[4];
    for (int i = 0; i < 4; ++i) {
      leafC[i] = C[i] = tp.leaf(ck[it].Cs[i]);
      leafE[i] = E[i] = tp.leaf(ck[it].Es[i]);
    }
    AV A = tp.leaf(e.A), Ad = tp.leaf(e.Ad);
    for (int d = 0; d < 4; ++d) {
      QuarterPair<ADPolicy> q = quarters(p, d, C, E, A, Ad);
      AV P1, P2;
      ad_projector(tp, q.R1, q.t1, q.R2, q.t2, ck[it].proj[d], &P1, &P2);
      Projected<ADPolicy> np = project(p, d, C, E, A, Ad, P1, P2);
      int ia, ib, ie;
      move_slots(d, &ia, &ib, &ie);
      C[ia] = ad_renorm(tp, np.Ca);
      C[ib] = ad_renorm(tp, np.Cb);
      E[ie] = ad_renorm(tp, np.E);
    }
    for (int i = 0; i < 4; ++i) {
      tp.acc(C[i].id, gC[i]);
      tp.acc(E[i].id, gE[i]);
    }
    clock.mark(2);
    tp.backward();
    clock.mark(3);
    for (int i = 0; i < 4; ++i) {
      gC[i] = tp.grad(leafC[i].id);
      gE[i] = tp.grad(leafE[i].id);
    }
    if (!tp.grad(A.id).empty()) {
      if (gAcc.empty()) gAcc = clone(c, tp.grad(A.id));
      else axpy(c, cplx(1), tp.grad(A.id), gAcc);
    }
    if (!tp.grad(Ad.id).empty()) {
      if (gAdc.empty()) gAdc = clone(c, tp.grad(Ad.id));
      else axpy(c, cplx(1), tp.grad(Ad.id), gAdc);
    }
  }
  // A enters as A and Ad = conj(A) = A (real)
  Tensor g = gAcc.empty() ? c.zeros(DType::F64, e.A.shape()) : clone(c, gAcc);
  if (!gAdc.empty()) axpy(c, cplx(1), gAdc, g);
  *gA = g;
  return Ere;
}

}  // namespace ipeps
