// Complex (complex128) versions of the projector's k x k kernels, for
// complex iPEPS tensors (e.g. the honeycomb models of src/model/*.jl, whose
// environments are ComplexF64).  Same algorithms as the real kernels in
// smallmat.cu, written for the modest sketch widths these models use
// (k <= ~118, one CTA):
//
//   chol_c           G = R^H R (G Hermitian), right-looking, one column per step
//   trsm_c           Q = Y R^-1, one warp per row of Y
//   jacobi_c_svd     one-sided Jacobi; the pair (p, q) with c = x_p^H x_q =
//                    |c| e^{i phi} is rotated as the real pair (x_p, e^{-i phi} x_q),
//                    i.e. [x_p x_q] <- [x_p x_q] [[cs, sn], [-sn e^{-i phi}, cs e^{-i phi}]]
//                    (unitary); the rotations are logged and applied to J row-parallel.
#include "linalg.cuh"

#include <atomic>

namespace ipeps {
namespace {

constexpr unsigned kFullC = 0xffffffffu;
constexpr size_t kSmemMaxC = 226 * 1024;

__device__ __forceinline__ int pkc(int i, int j) { return ((j * (j + 1)) >> 1) + i; }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconjmul(double2 a, double2 b) {  // conj(a) * b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

constexpr int kCholCThreads = 256;

// Guarded Cholesky of a Hermitian positive semi-definite G (upper triangle
// read): the same shift and pivot guard as the real kernel.  G <- R.
__global__ void __launch_bounds__(kCholCThreads) chol_c_kernel(double2* G, int k, int64_t ldg, double shift_factor) {
  extern __shared__ __align__(16) double2 Pc[];
  double2* rowj = Pc + (k * (k + 1)) / 2;
  __shared__ double s_red[kCholCThreads / 32];
  __shared__ double s_tr;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = kCholCThreads / 32;
  for (int j = warp; j < k; j += nw)
    for (int i = lane; i <= j; i += 32) Pc[pkc(i, j)] = G[i + int64_t(j) * ldg];
  __syncthreads();
  double t = 0;
  for (int i = tid; i < k; i += kCholCThreads) t += fabs(Pc[pkc(i, i)].x);
  for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(kFullC, t, o);
  if (lane == 0) s_red[warp] = t;
  __syncthreads();
  if (tid == 0) {
    double s = 0;
    for (int w = 0; w < nw; ++w) s += s_red[w];
    s_tr = s;
  }
  __syncthreads();
  const double shift = shift_factor > 0 ? shift_factor * s_tr : 0.0;
  if (shift > 0)
    for (int i = tid; i < k; i += kCholCThreads) Pc[pkc(i, i)].x += shift;
  const double tiny = 1e-300 + 1e-32 * (s_tr + shift * k);
  __syncthreads();
  for (int j = 0; j < k; ++j) {
    const double d = Pc[pkc(j, j)].x;
    const bool ok = d > tiny;
    const double rs = ok ? rsqrt(d) : 0.0;
    __syncthreads();
    for (int l = j + 1 + tid; l < k; l += kCholCThreads) {
      const double2 v = make_double2(Pc[pkc(j, l)].x * rs, Pc[pkc(j, l)].y * rs);
      Pc[pkc(j, l)] = v;
      rowj[l] = v;
    }
    if (tid == 0) Pc[pkc(j, j)] = make_double2(ok ? d * rs : 1.0, 0.0);
    __syncthreads();
    // P[i][l] -= conj(R[j][i]) R[j][l], j < i <= l
    for (int l = j + 1 + tid; l < k; l += kCholCThreads) {
      const double2 rl = rowj[l];
      double2* col = Pc + (l * (l + 1)) / 2;
      for (int i = j + 1; i <= l; ++i) {
        const double2 u = cconjmul(rowj[i], rl);
        col[i].x -= u.x;
        col[i].y -= u.y;
      }
    }
    __syncthreads();
  }
  for (int j = warp; j < k; j += nw)
    for (int i = lane; i < k; i += 32) G[i + int64_t(j) * ldg] = (i <= j) ? Pc[pkc(i, j)] : make_double2(0.0, 0.0);
}

constexpr int kTrsmCRows = 8;

// Q = Y R^-1 (R upper, real positive diagonal): x R = y row by row, the row
// in shared memory, x_j = (y_j - sum_{l<j} x_l R[l][j]) / R[j][j].
__global__ void __launch_bounds__(kTrsmCRows * 32) trsm_c_kernel(const double2* Y, int64_t ldy, int64_t N, int k,
                                                                 const double2* R, int64_t ldr, double2* Q,
                                                                 int64_t ldq) {
  extern __shared__ __align__(16) double2 smc[];
  double2* Rs = smc;                                                // column-major packed upper, k(k+1)/2
  double2* rows = Rs + (k * (k + 1)) / 2;                           // kTrsmCRows x k
  double* rinv = reinterpret_cast<double*>(rows + kTrsmCRows * k);  // 1 / R[j][j]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int nthr = kTrsmCRows * 32;
  const int64_t i0 = int64_t(blockIdx.x) * kTrsmCRows;
  for (int l = warp; l < k; l += kTrsmCRows)
    for (int j = lane; j <= l; j += 32) Rs[pkc(j, l)] = R[j + int64_t(l) * ldr];
  for (int j = tid; j < k; j += nthr) rinv[j] = 1.0 / R[j + int64_t(j) * ldr].x;
  for (int t = tid; t < kTrsmCRows * k; t += nthr) {
    const int r = t % kTrsmCRows, l = t / kTrsmCRows;
    rows[r * k + l] = (i0 + r < N) ? Y[(i0 + r) + int64_t(l) * ldy] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2* row = rows + warp * k;
  for (int j = 0; j < k; ++j) {
    const double2 yj = row[j];
    const double2 xj = make_double2(yj.x * rinv[j], yj.y * rinv[j]);
    __syncwarp();
    if (lane == 0) row[j] = xj;
    for (int l = j + 1 + lane; l < k; l += 32) {
      const double2 u = cmul(xj, Rs[pkc(j, l)]);
      row[l].x -= u.x;
      row[l].y -= u.y;
    }
    __syncwarp();
  }
  __syncthreads();
  for (int t = tid; t < kTrsmCRows * k; t += nthr) {
    const int r = t % kTrsmCRows, l = t / kTrsmCRows;
    if (i0 + r < N) Q[(i0 + r) + int64_t(l) * ldq] = rows[r * k + l];
  }
}

__device__ __forceinline__ bool rr_pair_c(int pi, int r, int kk, int k, int& p, int& q) {
  const int n1 = kk - 1;
  int a = pi - 1 + r;
  if (a >= n1) a -= n1;
  int b = kk - 2 - pi + r;
  if (b >= n1) b -= n1;
  p = (pi == 0) ? 0 : 1 + a;
  q = 1 + b;
  if (p > q) {
    const int t = p;
    p = q;
    q = t;
  }
  return p < k && q < k;
}

__device__ __forceinline__ double hsum16c(double v) {
  for (int o = 8; o; o >>= 1) v += __shfl_xor_sync(kFullC, v, o);
  return v;
}

// One-sided complex Jacobi on X (m x k) in shared memory, one half-warp per
// column pair.  Log entry e of round r in sweep s: rot[2 e] = (cs, sn),
// rot[2 e + 1] = e^{-i phi} ((1, 0), (1, 0) when skipped).
__global__ void __launch_bounds__(1024) jacobi_c_kernel(double2* Xg, int m, int k, int64_t ldx, double2* rot,
                                                        int max_sweeps, double tol, double* S, int* status,
                                                        int* sweeps_out) {
  extern __shared__ __align__(16) double2 Xc[];
  double* nrm = reinterpret_cast<double*>(Xc + int64_t(m) * k);
  __shared__ int s_rot;
  const int tid = threadIdx.x, grp = tid >> 4, l16 = tid & 15, ngrp = blockDim.x >> 4;
  const int warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
  for (int j = warp; j < k; j += nwarps)
    for (int i = lane; i < m; i += 32) Xc[i + j * m] = Xg[i + int64_t(j) * ldx];
  __syncthreads();
  const int kk = (k + 1) & ~1, np = kk / 2;
  const double tol2 = tol * tol;
  int sweep = 0;
  bool converged = (k < 2);
  for (; sweep < max_sweeps && !converged; ++sweep) {
    for (int j = warp; j < k; j += nwarps) {
      double a = 0;
      for (int i = lane; i < m; i += 32) {
        const double2 x = Xc[i + j * m];
        a = fma(x.x, x.x, fma(x.y, x.y, a));
      }
      for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(kFullC, a, o);
      if (lane == 0) nrm[j] = a;
    }
    if (tid == 0) s_rot = 0;
    __syncthreads();
    for (int r = 0; r < kk - 1; ++r) {
      double2* rr = rot + (size_t(sweep) * (kk - 1) + r) * np * 2;
      for (int base = 0; base < np; base += ngrp) {
        const int pi = base + grp;
        int p = 0, q = 0;
        const bool valid = pi < np && rr_pair_c(pi, r, kk, k, p, q);
        double cr = 0, ci = 0;
        if (valid)
          for (int i = l16; i < m; i += 16) {
            const double2 u = cconjmul(Xc[i + p * m], Xc[i + q * m]);
            cr += u.x;
            ci += u.y;
          }
        cr = hsum16c(cr);
        ci = hsum16c(ci);
        double cs = 1.0, sn = 0.0;
        double2 eb = make_double2(1.0, 0.0);
        if (valid) {
          const double a = nrm[p], b = nrm[q];
          const double mag2 = cr * cr + ci * ci;
          if (mag2 > 0.0 && a > 0.0 && b > 0.0 && mag2 > tol2 * (a * b)) {
            const double im = rsqrt(mag2), mag = mag2 * im;
            eb = make_double2(cr * im, -ci * im);  // e^{-i phi}
            const double d = b - a;
            const double rho = rsqrt(fma(d, d, 4.0 * mag2));
            const double c2 = fabs(d) * rho, s2 = copysign(1.0, d) * (2.0 * mag * rho);
            const double uu = 0.5 * (1.0 + c2);
            const double ru = rsqrt(uu);
            cs = uu * ru;
            sn = 0.5 * s2 * ru;
            for (int i = l16; i < m; i += 16) {
              const double2 xp = Xc[i + p * m];
              const double2 yq = cmul(eb, Xc[i + q * m]);
              Xc[i + p * m] = make_double2(cs * xp.x - sn * yq.x, cs * xp.y - sn * yq.y);
              Xc[i + q * m] = make_double2(sn * xp.x + cs * yq.x, sn * xp.y + cs * yq.y);
            }
            if (l16 == 0) {
              const double tc = 0.5 * s2 * mag * (ru * ru);
              nrm[p] = a - tc;
              nrm[q] = b + tc;
              s_rot = 1;
            }
          }
        }
        if (pi < np && l16 == 0) {
          rr[2 * pi] = make_double2(cs, sn);
          rr[2 * pi + 1] = eb;
        }
      }
      __syncthreads();
    }
    converged = (s_rot == 0);
    __syncthreads();
  }
  for (int j = warp; j < k; j += nwarps) {
    double a = 0;
    for (int i = lane; i < m; i += 32) {
      const double2 x = Xc[i + j * m];
      a = fma(x.x, x.x, fma(x.y, x.y, a));
      Xg[i + int64_t(j) * ldx] = x;
    }
    for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(kFullC, a, o);
    if (lane == 0) S[j] = sqrt(a);
  }
  if (tid == 0) {
    if (!converged) atomicOr(status, 4);
    *sweeps_out = sweep;
  }
}

constexpr int kApplyCRows = 8;

// J = product of the logged unitary column transforms, one warp per row of J.
__global__ void __launch_bounds__(kApplyCRows * 32) jacobi_c_apply_kernel(const double2* rot, int k,
                                                                         const int* d_sweeps, double2* J,
                                                                         int64_t ldj) {
  extern __shared__ __align__(16) double2 rowc[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * kApplyCRows + warp;
  if (i >= k) return;
  double2* row = rowc + warp * k;
  for (int j = lane; j < k; j += 32) row[j] = make_double2(j == i ? 1.0 : 0.0, 0.0);
  __syncwarp();
  const int kk = (k + 1) & ~1, np = kk / 2;
  const int nsw = *d_sweeps;
  for (int s = 0; s < nsw; ++s)
    for (int r = 0; r < kk - 1; ++r) {
      const double2* rr = rot + (size_t(s) * (kk - 1) + r) * np * 2;
      for (int pi = lane; pi < np; pi += 32) {
        const double2 g = rr[2 * pi];
        if (g.y == 0.0) continue;
        int p, q;
        if (!rr_pair_c(pi, r, kk, k, p, q)) continue;
        const double2 eb = rr[2 * pi + 1];
        const double2 jp = row[p], jq = cmul(eb, row[q]);
        row[p] = make_double2(g.x * jp.x - g.y * jq.x, g.x * jp.y - g.y * jq.y);
        row[q] = make_double2(g.y * jp.x + g.x * jq.x, g.y * jp.y + g.x * jq.y);
      }
      __syncwarp();
    }
  for (int j = lane; j < k; j += 32) J[i + int64_t(j) * ldj] = row[j];
}

SmemAttrOnce g_cholc_attr, g_trsmc_attr, g_jacc_attr, g_appc_attr;

size_t cholc_smem(int k) { return (size_t(k) * (k + 1) / 2 + size_t(k)) * 16; }
size_t trsmc_smem(int k) { return (size_t(k) * (k + 1) / 2 + size_t(kTrsmCRows) * k) * 16 + size_t(k) * 8; }
size_t jacc_smem(int m, int k) { return size_t(m) * k * 16 + size_t(k) * 8; }

}  // namespace

bool complex_small_fits(int m, int k) {
  return k >= 1 && cholc_smem(k) <= kSmemMaxC && trsmc_smem(k) <= kSmemMaxC && jacc_smem(m, k) <= kSmemMaxC;
}

void chol_c(Ctx& c, void* G, int k, int64_t ldg, double shift_factor) {
  IPEPS_CHECK(cholc_smem(k) <= kSmemMaxC, "chol_c: k too large for shared memory");
  g_cholc_attr.ensure(chol_c_kernel, int(kSmemMaxC));
  ProfScope ps(c, KFam::SmallLinalg);
  chol_c_kernel<<<1, kCholCThreads, cholc_smem(k), c.stream>>>(static_cast<double2*>(G), k, ldg, shift_factor);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::SmallLinalg, 8.0 * double(k) * k * k / 6.0);
}

void trsm_c(Ctx& c, const void* Y, int64_t ldy, int64_t N, int k, const void* R, int64_t ldr, void* Q, int64_t ldq) {
  IPEPS_CHECK(trsmc_smem(k) <= kSmemMaxC, "trsm_c: k too large for shared memory");
  if (N == 0) return;
  g_trsmc_attr.ensure(trsm_c_kernel, int(kSmemMaxC));
  ProfScope ps(c, KFam::SmallLinalg);
  const unsigned grid = unsigned((N + kTrsmCRows - 1) / kTrsmCRows);
  trsm_c_kernel<<<grid, kTrsmCRows * 32, trsmc_smem(k), c.stream>>>(static_cast<const double2*>(Y), ldy, N, k,
                                                                    static_cast<const double2*>(R), ldr,
                                                                    static_cast<double2*>(Q), ldq);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::SmallLinalg, 4.0 * double(N) * k * k);
}

void jacobi_c_svd(Ctx& c, void* X, int m, int k, int64_t ldx, void* J, int64_t ldj, double* S, int max_sweeps,
                  double tol, int* d_sweeps) {
  IPEPS_CHECK(jacc_smem(m, k) <= kSmemMaxC, "jacobi_c_svd: sketch too wide for shared memory");
  if (tol <= 0) tol = double(m) * 2.220446049250313e-16;
  g_jacc_attr.ensure(jacobi_c_kernel, int(kSmemMaxC));
  const int kk = (k + 1) & ~1;
  // two double2 per pair slot: (cs, sn) and e^{-i phi}
  Tensor rot = c.alloc(DType::F64, {int64_t(max_sweeps) * (kk - 1) * kk * 2});
  double2* rp = reinterpret_cast<double2*>(rot.data());
  {
    ProfScope ps(c, KFam::Jacobi);
    jacobi_c_kernel<<<1, 1024, jacc_smem(m, k), c.stream>>>(static_cast<double2*>(X), m, k, ldx, rp, max_sweeps, tol,
                                                            S, c.d_status, d_sweeps);
    IPEPS_LAUNCH_CHECK();
    c.count(KFam::Jacobi, 24.0 * double(m) * k * k / 2.0);
  }
  {
    ProfScope ps(c, KFam::Jacobi);
    const size_t smem = size_t(kApplyCRows) * k * 16;
    g_appc_attr.ensure(jacobi_c_apply_kernel, int(kSmemMaxC));
    const unsigned grid = unsigned((k + kApplyCRows - 1) / kApplyCRows);
    jacobi_c_apply_kernel<<<grid, kApplyCRows * 32, smem, c.stream>>>(rp, k, d_sweeps, static_cast<double2*>(J), ldj);
    IPEPS_LAUNCH_CHECK();
    c.count(KFam::Jacobi, 24.0 * double(k) * k * k / 2.0);
  }
}

}  // namespace ipeps
