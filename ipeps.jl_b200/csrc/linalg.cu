// Small dense FP64 linear algebra on the device (k x k, k <= a few hundred):
//   * guarded Cholesky (G = R^T R, upper R) for shifted CholeskyQR,
//   * inverse of an upper-triangular matrix,
//   * one-sided (Hestenes) Jacobi SVD with round-robin parallel ordering,
//   * descending sort of singular values with the permutation.
// Each runs as one CTA of 1024 threads; every loop is bounded and a
// non-converged Jacobi sets a bit in the context status word instead of
// spinning.
#include "linalg.cuh"

namespace ipeps {
namespace {

constexpr int kThreads = 1024;

// G (k x k, col-major, ldg) symmetric positive semi-definite; on exit R (upper
// triangle of G's storage) with G = R^T R.  Pivots <= tiny*trace are replaced
// by 1 with a zero row (the matching column of Q = Y R^-1 then stays a
// residual of size ~0 instead of blowing up).  shift is added to the diagonal.
__global__ void __launch_bounds__(kThreads) chol_kernel(double* G, int k, int64_t ldg, double shift,
                                                        int* status) {
  __shared__ double s_piv;
  __shared__ double s_tr;
  if (threadIdx.x == 0) {
    double tr = 0;
    for (int i = 0; i < k; ++i) tr += fabs(G[i + i * ldg]);
    s_tr = tr + shift * k;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < k; i += blockDim.x) G[i + i * ldg] += shift;
  __syncthreads();
  const double tiny = 1e-300 + 1e-32 * s_tr;
  for (int j = 0; j < k; ++j) {
    if (threadIdx.x == 0) {
      double d = G[j + j * ldg];
      s_piv = (d > tiny) ? sqrt(d) : 0.0;
      G[j + j * ldg] = (s_piv > 0) ? s_piv : 1.0;
    }
    __syncthreads();
    const double piv = s_piv;
    // row j of R: R[j, l] = G[j, l] / piv (upper part stored in G[j + l*ldg])
    for (int l = j + 1 + threadIdx.x; l < k; l += blockDim.x) G[j + l * ldg] = (piv > 0) ? G[j + l * ldg] / piv : 0.0;
    __syncthreads();
    // trailing update: G[i,l] -= R[j,i]*R[j,l] for j < i <= l
    const int rem = k - j - 1;
    const int64_t tot = int64_t(rem) * rem;
    for (int64_t t = threadIdx.x; t < tot; t += blockDim.x) {
      int i = j + 1 + int(t % rem), l = j + 1 + int(t / rem);
      if (i <= l) G[i + l * ldg] -= G[j + i * ldg] * G[j + l * ldg];
    }
    __syncthreads();
  }
  // zero the strict lower triangle so the buffer holds exactly R
  for (int64_t t = threadIdx.x; t < int64_t(k) * k; t += blockDim.x) {
    int i = int(t % k), l = int(t / k);
    if (i > l) G[i + l * ldg] = 0.0;
  }
}

// Rinv = R^-1 for upper-triangular R (k x k).  Row sweep from the bottom:
// X[i, j] = -(sum_{l=i+1..j} R[i,l] X[l,j]) / R[i,i], X[i,i] = 1/R[i,i].
__global__ void __launch_bounds__(kThreads) triinv_kernel(const double* R, int k, int64_t ldr, double* X,
                                                          int64_t ldx) {
  for (int64_t t = threadIdx.x; t < int64_t(k) * k; t += blockDim.x) {
    int i = int(t % k), j = int(t / k);
    X[i + j * ldx] = (i == j) ? 1.0 / R[i + i * ldr] : 0.0;
  }
  __syncthreads();
  for (int i = k - 2; i >= 0; --i) {
    const double rii = R[i + i * ldr];
    for (int j = i + 1 + threadIdx.x; j < k; j += blockDim.x) {
      double s = 0;
      for (int l = i + 1; l <= j; ++l) s = fma(R[i + l * ldr], X[l + j * ldx], s);
      X[i + j * ldx] = -s / rii;
    }
    __syncthreads();
  }
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One-sided Jacobi: orthogonalise the columns of X (m x k) by plane
// rotations accumulated into J (k x k, starts as identity).  On exit the
// columns of X are mutually orthogonal, S[j] = ||X[:,j]||.
__global__ void __launch_bounds__(kThreads) jacobi_kernel(double* X, int m, int k, int64_t ldx, double* J,
                                                          int64_t ldj, double* S, int max_sweeps, double tol,
                                                          int* status, int* sweeps_out) {
  __shared__ double s_off;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  for (int64_t t = threadIdx.x; t < int64_t(k) * k; t += blockDim.x) {
    int i = int(t % k), j = int(t / k);
    J[i + j * ldj] = (i == j) ? 1.0 : 0.0;
  }
  const int kk = (k + 1) & ~1;  // even player count (k odd: one idle slot)
  int sweep = 0;
  bool converged = (k < 2);
  for (; sweep < max_sweeps && !converged; ++sweep) {
    if (threadIdx.x == 0) s_off = 0.0;
    __syncthreads();
    for (int r = 0; r < kk - 1; ++r) {
      for (int pi = warp; pi < kk / 2; pi += nwarps) {
        int p = (pi == 0) ? 0 : 1 + (pi - 1 + r) % (kk - 1);
        int q = 1 + (kk - 2 - pi + r) % (kk - 1);
        if (p >= k || q >= k) continue;
        if (p > q) { int t = p; p = q; q = t; }
        double a = 0, b = 0, cc = 0;
        for (int i = lane; i < m; i += 32) {
          double xp = X[i + p * ldx], xq = X[i + q * ldx];
          a = fma(xp, xp, a);
          b = fma(xq, xq, b);
          cc = fma(xp, xq, cc);
        }
        a = warp_sum(a);
        b = warp_sum(b);
        cc = warp_sum(cc);
        if (cc == 0.0 || a == 0.0 || b == 0.0) continue;
        const double rel = fabs(cc) / sqrt(a * b);
        if (rel <= tol) continue;
        if (lane == 0) {
          // block-wide max of the off-diagonal measure (non-negative doubles order like ints)
          atomicMax(reinterpret_cast<unsigned long long*>(&s_off),
                    static_cast<unsigned long long>(__double_as_longlong(rel)));
        }
        const double zeta = (b - a) / (2.0 * cc);
        const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
        for (int i = lane; i < m; i += 32) {
          double xp = X[i + p * ldx], xq = X[i + q * ldx];
          X[i + p * ldx] = cs * xp - sn * xq;
          X[i + q * ldx] = sn * xp + cs * xq;
        }
        for (int i = lane; i < k; i += 32) {
          double jp = J[i + p * ldj], jq = J[i + q * ldj];
          J[i + p * ldj] = cs * jp - sn * jq;
          J[i + q * ldj] = sn * jp + cs * jq;
        }
      }
      __syncthreads();
    }
    converged = (s_off <= tol);
    __syncthreads();
  }
  // column norms
  for (int j = warp; j < k; j += nwarps) {
    double a = 0;
    for (int i = lane; i < m; i += 32) a = fma(X[i + j * ldx], X[i + j * ldx], a);
    a = warp_sum(a);
    if (lane == 0) S[j] = sqrt(a);
  }
  if (threadIdx.x == 0) {
    if (!converged) atomicOr(status, 4);
    if (sweeps_out) *sweeps_out = sweep;
  }
}

// Descending sort of S (length k <= 4096) with permutation; ties keep the
// later index first (the reference reverses an ascending stable sortperm).
__global__ void sort_desc_kernel(const double* S, int k, double* S_out, int* perm) {
  extern __shared__ unsigned char sm_raw[];
  double* v = reinterpret_cast<double*>(sm_raw);
  for (int i = threadIdx.x; i < k; i += blockDim.x) v[i] = S[i];
  __syncthreads();
  // rank sort: position = #{j : v[j] > v[i]} + #{j > i : v[j] == v[i]}
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    double x = v[i];
    int pos = 0;
    for (int j = 0; j < k; ++j) {
      double y = v[j];
      pos += (y > x) || (y == x && j > i);
    }
    S_out[pos] = x;
    perm[pos] = i;
  }
}

// out[:, j] = in[:, perm[j]] * (scale ? scale[j] : 1), j < ncols
__global__ void gather_cols_kernel(const double* in, int64_t ldi, int64_t m, const int* perm, int ncols,
                                   const double* scale_v, int scale_mode, double* out, int64_t ldo) {
  int64_t tot = m * ncols;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < tot; t += int64_t(gridDim.x) * blockDim.x) {
    int64_t i = t % m;
    int j = int(t / m);
    double s = 1.0;
    if (scale_mode == 1) s = scale_v[j];
    else if (scale_mode == 2) s = scale_v[j] != 0.0 ? 1.0 / scale_v[j] : 0.0;  // a null column stays zero
    out[i + j * ldo] = in[i + int64_t(perm[j]) * ldi] * s;
  }
}

// y[:, j] *= f(s[j]), f: 1 -> 1/sqrt(s)
__global__ void scale_cols_kernel(double* X, int64_t ldx, int64_t m, int ncols, const double* s, int mode) {
  int64_t tot = m * ncols;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < tot; t += int64_t(gridDim.x) * blockDim.x) {
    int64_t i = t % m;
    int j = int(t / m);
    // a kept s of exactly 0 (the degenerate-pair rule of the cutoff can keep one
    // past the 1e-12 cutoff) gets a zero column instead of an infinite one
    double f = (mode == 1) ? (s[j] > 0.0 ? 1.0 / sqrt(s[j]) : 0.0) : s[j];
    X[i + j * ldx] *= f;
  }
}

__global__ void scale_rows_kernel(double* X, int64_t ldx, int64_t m, int64_t ncols, const double* s, int mode) {
  int64_t tot = m * ncols;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < tot; t += int64_t(gridDim.x) * blockDim.x) {
    int64_t i = t % m, j = t / m;
    double f = (mode == 1) ? (s[i] > 0.0 ? 1.0 / sqrt(s[i]) : 0.0) : s[i];
    X[i + j * ldx] *= f;
  }
}

// trace of G (k x k) -> out
__global__ void trace_kernel(const double* G, int k, int64_t ldg, double* out) {
  double s = 0;
  for (int i = threadIdx.x; i < k; i += blockDim.x) s += G[i + i * ldg];
  s = warp_sum(s);
  __shared__ double sm[32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t += sm[w];
    *out = t;
  }
}

__global__ void shift_diag_kernel(double* G, int k, int64_t ldg, const double* tr, double factor) {
  const double sft = factor * (*tr);
  for (int i = threadIdx.x; i < k; i += blockDim.x) G[i + i * ldg] += sft;
}

unsigned grid_for(Ctx& c, int64_t n) {
  return unsigned(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, int64_t(c.sm_count) * 8)));
}

}  // namespace

void chol_upper(Ctx& c, double* G, int k, int64_t ldg, const double* d_trace_shift, double shift_factor) {
  if (d_trace_shift) {
    shift_diag_kernel<<<1, 256, 0, c.stream>>>(G, k, ldg, d_trace_shift, shift_factor);
    IPEPS_LAUNCH_CHECK();
  }
  ProfScope ps(c, KFam::SmallLinalg);
  chol_kernel<<<1, kThreads, 0, c.stream>>>(G, k, ldg, 0.0, c.d_status);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::SmallLinalg, double(k) * k * k / 3.0);
}

void triinv_upper(Ctx& c, const double* R, int k, int64_t ldr, double* X, int64_t ldx) {
  ProfScope ps(c, KFam::SmallLinalg);
  triinv_kernel<<<1, kThreads, 0, c.stream>>>(R, k, ldr, X, ldx);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::SmallLinalg, double(k) * k * k / 3.0);
}

void trace(Ctx& c, const double* G, int k, int64_t ldg, double* d_out) {
  trace_kernel<<<1, 256, 0, c.stream>>>(G, k, ldg, d_out);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Reduce);
}

void jacobi_svd(Ctx& c, double* X, int m, int k, int64_t ldx, double* J, int64_t ldj, double* S,
                int max_sweeps, double tol, int* d_sweeps) {
  ProfScope ps(c, KFam::Jacobi);
  jacobi_kernel<<<1, kThreads, 0, c.stream>>>(X, m, k, ldx, J, ldj, S, max_sweeps, tol, c.d_status, d_sweeps);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Jacobi, 6.0 * double(m + k) * k * k / 2.0);
}

void sort_desc(Ctx& c, const double* S, int k, double* S_out, int* perm) {
  IPEPS_CHECK(k <= 4096, "sort_desc: k too large");
  sort_desc_kernel<<<1, 1024, size_t(k) * sizeof(double), c.stream>>>(S, k, S_out, perm);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::SmallLinalg);
}

void gather_cols(Ctx& c, const double* in, int64_t ldi, int64_t m, const int* perm, int ncols,
                 const double* scale_v, int scale_mode, double* out, int64_t ldo) {
  gather_cols_kernel<<<grid_for(c, m * ncols), 256, 0, c.stream>>>(in, ldi, m, perm, ncols, scale_v, scale_mode,
                                                                   out, ldo);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Elementwise, 0, 16.0 * m * ncols);
}

void scale_cols(Ctx& c, double* X, int64_t ldx, int64_t m, int ncols, const double* s, int mode) {
  scale_cols_kernel<<<grid_for(c, m * ncols), 256, 0, c.stream>>>(X, ldx, m, ncols, s, mode);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Elementwise, 0, 16.0 * m * ncols);
}

void scale_rows(Ctx& c, double* X, int64_t ldx, int64_t m, int64_t ncols, const double* s, int mode) {
  scale_rows_kernel<<<grid_for(c, m * ncols), 256, 0, c.stream>>>(X, ldx, m, ncols, s, mode);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Elementwise, 0, 16.0 * m * ncols);
}

}  // namespace ipeps
