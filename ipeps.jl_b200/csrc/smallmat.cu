// Shared-memory kernels for the projector's k x k problems (k ~ chi + oversampling):
//
//   chol_blocked      G = R^T R in one CTA, 32-column panels: one warp factors the
//                     diagonal block in registers, the block's rows of R are solved
//                     column-parallel, the trailing update is a register-tiled SYRK.
//   chol_ldl          the same for k <= 160 with the upper triangle in registers: one
//                     barrier per elimination step.
//   trsm_right_upper  Q = Y R^-1, two rows of Y per warp (the rows are independent), at
//                     most one CTA per SM, R staged row-major in each CTA's shared memory.
//   jacobi_svd_auto   one-sided Jacobi with only X in shared memory; every rotation is
//                     logged, and J = product of the rotations is formed afterwards by a
//                     row-parallel kernel (each row of J sees the same rotation sequence).
//
// These replace, for the sizes that fit, the reference's LAPACK calls behind
// svd(R1*R2) (src/utility/wrapper.jl:25-35) in the randomized projector.
#include "linalg.cuh"

#include <atomic>

namespace ipeps {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kPanel = 32;
constexpr int kCholThreads = 256;
// opt-in limit per block is 227 KB including static shared memory
constexpr size_t kSmemMax = 226 * 1024;

__device__ __forceinline__ int pku(int i, int j) { return ((j * (j + 1)) >> 1) + i; }  // packed upper, i <= j
// row-major packed upper triangle: row j (columns j..k-1) starts at rowoff(j)
__device__ __forceinline__ int rowoff(int j, int k) { return j * k - ((j * (j - 1)) >> 1); }

size_t chol_smem_doubles(int k) {
  const size_t npk = (size_t(k) * (k + 1) / 2 + 1) & ~size_t(1);  // even: W below is 16-byte aligned
  return npk + size_t(kPanel) * size_t(k + 2) + 8 + size_t(k + (k & 1)) + 34;
}

// Guarded blocked Cholesky.  On entry G (k x k, upper triangle read) is
// symmetric positive semi-definite; shift_factor > 0 first adds
// shift_factor * trace(G) to the diagonal (shifted CholeskyQR).  A pivot at or
// below 1e-32 * trace leaves R[j][j] = 1 and row j zero, so R stays
// invertible.  On exit G holds R (strict lower triangle zeroed) and, when
// Rrow is given, Rrow holds R's upper triangle packed row by row (the layout
// the row-parallel triangular solve stages with contiguous copies).
__global__ void __launch_bounds__(kCholThreads) chol_blocked_kernel(double* G, int k, int64_t ldg,
                                                                    double shift_factor, double* Rrow) {
  extern __shared__ __align__(16) double sm[];
  const int npk = ((k * (k + 1)) / 2 + 1) & ~1;
  double* P = sm;                                     // packed upper triangle
  double* W = P + npk;                                // rows of R right of the diagonal block: 32 x ldw (+8 pad)
  double* rsv = W + size_t(kPanel) * (k + 2) + 8;     // 1 / R[j][j] as used for the row scaling (0: failed pivot)
  double* rowb = rsv + (k + (k & 1));                 // pivot row of the diagonal block (32) + pivot (1), 16-byte aligned
  __shared__ double s_red[kCholThreads / 32];
  __shared__ double s_tr;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = kCholThreads / 32;

  {
    // the upper triangle, four independent loads in flight per thread
    const int kk2 = k * k;
    for (int t0 = tid; t0 < kk2; t0 += 4 * kCholThreads) {
      double v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int t = t0 + u * kCholThreads, i = t % k, j = t / k;
        v[u] = (t < kk2 && i <= j) ? G[i + int64_t(j) * ldg] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int t = t0 + u * kCholThreads, i = t % k, j = t / k;
        if (t < kk2 && i <= j) P[pku(i, j)] = v[u];
      }
    }
  }
  __syncthreads();
  double t = 0;
  for (int i = tid; i < k; i += kCholThreads) t += fabs(P[pku(i, i)]);
  for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(kFull, t, o);
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
    for (int i = tid; i < k; i += kCholThreads) P[pku(i, i)] += shift;
  const double tiny = 1e-300 + 1e-32 * (s_tr + shift * k);
  __syncthreads();

  for (int j0 = 0; j0 < k; j0 += kPanel) {
    const int jb = min(kPanel, k - j0), j1 = j0 + jb, nt = k - j1;
    const int ldw = (nt + 1) & ~1;
    // (A) warp 0: right-looking Cholesky of the diagonal block, lane l holding column j0 + l.
    // A partial last block is padded with the identity, so the 32 steps run without branches;
    // the pivot row goes through shared memory (one broadcast load per two entries).
    if (warp == 0) {
      double a[kPanel];
#pragma unroll
      for (int i = 0; i < kPanel; ++i)
        a[i] = (i <= lane && lane < jb) ? P[pku(j0 + i, j0 + lane)] : (i == lane ? 1.0 : 0.0);
#pragma unroll
      for (int jj = 0; jj < kPanel; ++jj) {
        if (lane == jj) rowb[32] = a[jj];
        __syncwarp();
        const double d = rowb[32];
        const bool ok = d > tiny;
        const double rs = ok ? rsqrt(d) : 0.0;
        if (lane == jj) {
          a[jj] = ok ? d * rs : 1.0;
          if (jj < jb) rsv[j0 + jj] = rs;
        } else if (lane > jj) {
          a[jj] *= rs;
        }
        const double v = a[jj];
        rowb[lane] = v;
        __syncwarp();
        double rv[kPanel];
#pragma unroll
        for (int i = ((jj + 1) & ~1); i < kPanel; i += 2) {
          const double2 t2 = *reinterpret_cast<const double2*>(rowb + i);
          rv[i] = t2.x;
          rv[i + 1] = t2.y;
        }
#pragma unroll
        for (int i = jj + 1; i < kPanel; ++i)
          if (lane >= i) a[i] = fma(-rv[i], v, a[i]);
        __syncwarp();
      }
#pragma unroll
      for (int i = 0; i < kPanel; ++i)
        if (i <= lane && lane < jb) P[pku(j0 + i, j0 + lane)] = a[i];
    }
    __syncthreads();
    if (nt == 0) break;
    // (B) rows j0..j1 of R beyond the block: R_pp^T X = A12, four columns per warp step
    {
      const double rsl = lane < jb ? rsv[j0 + lane] : 0.0;
      double rp[kPanel];  // R_pp[m][lane], m < lane
#pragma unroll
      for (int m = 0; m < kPanel; ++m) rp[m] = (m < lane && lane < jb) ? P[pku(j0 + m, j0 + lane)] : 0.0;
      for (int c0 = j1 + 4 * warp; c0 < k; c0 += 4 * nw) {
        double x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = (lane < jb && c0 + u < k) ? P[pku(j0 + lane, c0 + u)] : 0.0;
#pragma unroll
        for (int m = 0; m < kPanel; ++m) {  // rows m >= jb carry zeros (rsl = 0 there)
          const double rsm = __shfl_sync(kFull, rsl, m);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const double xm = __shfl_sync(kFull, x[u], m) * rsm;
            if (lane > m) x[u] = fma(-rp[m], xm, x[u]);
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (lane < jb && c0 + u < k) W[lane * ldw + (c0 + u - j1)] = x[u] * rsl;
      }
    }
    __syncthreads();
    // (C) trailing update P[i][j] -= sum_l W[l][i] W[l][j] (j1 <= i <= j), 32 rows x 8 columns per warp
    // unit; the block's rows of R are copied back from W
    {
      const int nrb = (nt + 31) >> 5, ncg = (nt + 7) >> 3;
      for (int u = warp; u < nrb * ncg; u += nw) {
        const int rb = u % nrb, cg = u / nrb;
        if (rb * 32 > cg * 8 + 7) continue;  // the whole row block lies below the diagonal
        const int ir = rb * 32 + lane;       // row relative to j1
        double acc[8];
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[v] = 0.0;
        for (int l = 0; l < jb; ++l) {
          const double* wl = W + l * ldw;
          const double wi = ir < nt ? wl[ir] : 0.0;
          const double2* wj = reinterpret_cast<const double2*>(wl + cg * 8);
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            const double2 w2 = wj[v];
            acc[2 * v] = fma(wi, w2.x, acc[2 * v]);
            acc[2 * v + 1] = fma(wi, w2.y, acc[2 * v + 1]);
          }
        }
#pragma unroll
        for (int v = 0; v < 8; ++v) {
          const int jc = cg * 8 + v;
          if (ir < nt && jc < nt && ir <= jc) {
            double* pp = P + pku(j1 + ir, j1 + jc);
            *pp -= acc[v];
          }
        }
      }
      for (int t2 = tid; t2 < jb * nt; t2 += kCholThreads) {
        const int l = t2 % jb, cc = t2 / jb;
        P[pku(j0 + l, j1 + cc)] = W[l * ldw + cc];
      }
    }
    __syncthreads();
  }
  __syncthreads();
  for (int j = warp; j < k; j += nw)
    for (int i = lane; i < k; i += 32) G[i + int64_t(j) * ldg] = (i <= j) ? P[pku(i, j)] : 0.0;
  if (Rrow)
    for (int i = warp; i < k; i += nw)
      for (int jj = lane; jj < k - i; jj += 32) Rrow[rowoff(i, k) + jj] = P[pku(i, i + jj)];
}

// Register-resident Cholesky for k <= 32 NBB (NBB <= 5), same contract as
// chol_blocked_kernel.  The right-looking elimination is written as
// G = U^T D U (U unit upper): step j subtracts a[j][r] a[j][c] / a[j][j] from
// every a[r][c] with c >= r > j, and R = D^1/2 U at the end.  512 threads
// hold the upper triangle in registers, thread (w, l) of warp w and lane l the
// entries (w + 16 a, l + 32 b) (slots a <= 2b + 1 can reach the triangle), so a
// step costs one barrier: the warp owning row j publishes the row and the row
// divided by the pivot in shared memory (double-buffered by the parity of j),
// and every thread updates its slots from two broadcast loads per row and
// one load per column block.
constexpr int kLdlThreads = 512;

size_t chol_ldl_smem_doubles(int k) {
  const size_t npk = (size_t(k) * (k + 1) / 2 + 1) & ~size_t(1);
  return npk + 4 * 160 + 2 * 160 + 8;
}

// Publishes row j (16 JB <= j < 16 JB + 16, held in slot a = JB of the calling
// warp): a[j][c] (c >= j) into rw, a[j][c] / a[j][j] (c > j) into sc, the
// pivot into dd[j] (0 for a failed pivot).
template <int NBB, int JB>
__device__ __forceinline__ void ldl_publish(const double (&v)[2 * NBB][NBB], int j, int k, int lane, double* rw,
                                            double* sc, double* dd, double tiny) {
  constexpr int B0 = JB / 2;
  // the pivot a[j][j] sits in column block JB / 2 of lane j mod 32
  const double d = __shfl_sync(kFull, v[JB][B0], j & 31);
  const bool ok = d > tiny;
  const double inv = ok ? __drcp_rn(d) : 0.0;
#pragma unroll
  for (int b = B0; b < NBB; ++b) {
    const int c = lane + 32 * b;
    if (c >= j && c < k) {
      rw[c] = v[JB][b];
      if (c > j) sc[c] = v[JB][b] * inv;
    }
  }
  if (lane == 0) dd[j] = ok ? d : 0.0;
}

// Elimination steps j = 16 JB .. 16 JB + 15 of chol_ldl_kernel, then the next
// block of 16 (JB is a compile-time constant, so the slots of rows that are
// finished, a < JB, and of column blocks left of every pivot of the block,
// 32 b + 31 <= 16 JB, drop out of the code instead of being tested per step).
// Step j: the warp holding row j (warp j mod 16, slot a = JB) publishes it in
// shared memory, double-buffered by the parity of j, and after the barrier
// every slot of a row r > j takes a[r][c] -= a[j][r] (a[j][c] / a[j][j]).
// Slots left of the diagonal take stale buffer entries and are never read.
// (Publishing row j + 1 during step j, as soon as its warp has updated it,
// measured no faster: the steps are bound by the barrier and the shared-memory
// broadcasts, not by the pivot's reciprocal.)
template <int NBB, int JB>
__device__ __forceinline__ void ldl_steps(double (&v)[2 * NBB][NBB], int k, int warp, int lane, double* raw,
                                          double* scl, double* dd, double tiny) {
  constexpr int NBA = 2 * NBB, KP = 32 * NBB, B0 = JB / 2;
  const int tmax = min(16, k - 16 * JB);
  for (int t = 0; t < tmax; ++t) {
    const int j = 16 * JB + t;
    double* rw = raw + (t & 1) * KP;
    double* sc = scl + (t & 1) * KP;
    if (warp == t) ldl_publish<NBB, JB>(v, j, k, lane, rw, sc, dd, tiny);
    __syncthreads();
    double s[NBB];
#pragma unroll
    for (int b = B0; b < NBB; ++b) s[b] = sc[lane + 32 * b];
    if (warp > t) {  // slot a = JB holds row 16 JB + warp > j
      const double ra = rw[16 * JB + warp];
#pragma unroll
      for (int b = B0; b < NBB; ++b) v[JB][b] = fma(-ra, s[b], v[JB][b]);
    }
#pragma unroll
    for (int a = JB + 1; a < NBA; ++a) {
      const double ra = rw[warp + 16 * a];
#pragma unroll
      for (int b = B0; b < NBB; ++b) {
        if (a > 2 * b + 1) continue;
        v[a][b] = fma(-ra, s[b], v[a][b]);
      }
    }
  }
  if constexpr (JB + 1 < NBA) ldl_steps<NBB, JB + 1>(v, k, warp, lane, raw, scl, dd, tiny);
}

template <int NBB>
__global__ void __launch_bounds__(kLdlThreads, 1) chol_ldl_kernel(double* G, int k, int64_t ldg, double shift_factor,
                                                                double* Rrow) {
  constexpr int NBA = 2 * NBB, KP = 32 * NBB;
  extern __shared__ __align__(16) double sm[];
  const int npk = ((k * (k + 1)) / 2 + 1) & ~1;
  double* P = sm;             // packed upper triangle, column by column
  double* raw = P + npk;      // [2][KP]: row j of the eliminated matrix
  double* scl = raw + 2 * KP; // [2][KP]: the same divided by the pivot (0 for a failed pivot)
  double* dd = scl + 2 * KP;  // pivots (0: failed)
  double* rs = dd + KP;       // 1 / sqrt(pivot), 0 for a failed pivot
  __shared__ double s_red[kLdlThreads / 32];
  __shared__ double s_tr;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  {
    constexpr int kU = 4;
    const int kk2 = k * k;
    for (int t0 = tid; t0 < kk2; t0 += kU * kLdlThreads) {
      double v[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int t = t0 + u * kLdlThreads, i = t % k, j = t / k;
        v[u] = (t < kk2 && i <= j) ? G[i + int64_t(j) * ldg] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int t = t0 + u * kLdlThreads, i = t % k, j = t / k;
        if (t < kk2 && i <= j) P[pku(i, j)] = v[u];
      }
    }
    for (int t = tid; t < 4 * KP; t += kLdlThreads) raw[t] = 0.0;  // raw and scl, rows >= k stay 0
  }
  __syncthreads();
  double t = 0;
  for (int i = tid; i < k; i += kLdlThreads) t += fabs(P[pku(i, i)]);
  for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(kFull, t, o);
  if (lane == 0) s_red[warp] = t;
  __syncthreads();
  if (tid == 0) {
    double s = 0;
    for (int w = 0; w < kLdlThreads / 32; ++w) s += s_red[w];
    s_tr = s;
  }
  __syncthreads();
  const double shift = shift_factor > 0 ? shift_factor * s_tr : 0.0;
  const double tiny = 1e-300 + 1e-32 * (s_tr + shift * k);

  double v[NBA][NBB];
#pragma unroll
  for (int a = 0; a < NBA; ++a)
#pragma unroll
    for (int b = 0; b < NBB; ++b) {
      if (a > 2 * b + 1) continue;
      const int r = warp + 16 * a, c = lane + 32 * b;
      double x = (r <= c && c < k) ? P[pku(r, c)] : 0.0;
      if (r == c) x += shift;
      v[a][b] = x;
    }

  ldl_steps<NBB, 0>(v, k, warp, lane, raw, scl, dd, tiny);
  for (int i = tid; i < k; i += kLdlThreads) rs[i] = dd[i] > 0.0 ? rsqrt(dd[i]) : 0.0;
  __syncthreads();
  // R = D^1/2 U into P; a failed pivot gives R[j][j] = 1 and row j zero
#pragma unroll
  for (int a = 0; a < NBA; ++a)
#pragma unroll
    for (int b = 0; b < NBB; ++b) {
      if (a > 2 * b + 1) continue;
      const int r = warp + 16 * a, c = lane + 32 * b;
      if (r <= c && c < k) {
        const double q = rs[r];
        P[pku(r, c)] = (r == c) ? (q > 0.0 ? dd[r] * q : 1.0) : v[a][b] * q;
      }
    }
  __syncthreads();
  for (int j = warp; j < k; j += kLdlThreads / 32)
    for (int i = lane; i < k; i += 32) G[i + int64_t(j) * ldg] = (i <= j) ? P[pku(i, j)] : 0.0;
  if (Rrow)
    for (int i = warp; i < k; i += kLdlThreads / 32)
      for (int jj = lane; jj < k - i; jj += 32) Rrow[rowoff(i, k) + jj] = P[pku(i, i + jj)];
}

// Q = Y R^-1 for R (k x k) upper triangular: row y of Y solves x R = y by
// forward substitution, x_j = (y_j - sum_{l<j} x_l R[l][j]) / R[j][j].  Each
// warp carries two rows at once (two independent substitution chains), a CTA
// takes 2 x warps rows per pass over a grid of at most one CTA per SM, so R is
// staged into shared memory once per SM rather than once per handful of rows.
constexpr int kTrsmRPW = 2;  // rows per warp and pass

template <int NS>
__global__ void __launch_bounds__(512, 1) trsm_rows_kernel(const double* Y, int64_t ldy, int64_t N, int k,
                                                           const double* R, int64_t ldr, const double* Rrow,
                                                           double* Q, int64_t ldq) {
  extern __shared__ __align__(16) double sm[];
  const int kp = k | 1;
  const int nthr = blockDim.x, nwarp = nthr >> 5, rows = nwarp * kTrsmRPW;
  double* Rs = sm;                        // k(k+1)/2, row-major packed
  double* rinv = Rs + (k * (k + 1)) / 2;  // k
  double* Yt = rinv + k;                  // rows x kp
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int npk = (k * (k + 1)) / 2;
  if (Rrow) {
    // R already packed row by row: contiguous 16-byte copies (both bases are 16-byte aligned)
    const double2* src = reinterpret_cast<const double2*>(Rrow);
    double2* dst = reinterpret_cast<double2*>(Rs);
    for (int t = tid; t < npk / 2; t += nthr) dst[t] = src[t];
    if ((npk & 1) && tid == 0) Rs[npk - 1] = Rrow[npk - 1];
    __syncthreads();
    for (int j = tid; j < k; j += nthr) rinv[j] = 1.0 / Rs[rowoff(j, k)];
  } else {
    for (int l = warp; l < k; l += nwarp)
      for (int j = lane; j <= l; j += 32) Rs[rowoff(j, k) + (l - j)] = R[j + int64_t(l) * ldr];
    for (int j = tid; j < k; j += nthr) rinv[j] = 1.0 / R[j + int64_t(j) * ldr];
  }
  for (int64_t i0 = int64_t(blockIdx.x) * rows; i0 < N; i0 += int64_t(gridDim.x) * rows) {
    __syncthreads();  // R staged; the previous pass's Yt written out
    for (int t = tid; t < rows * k; t += nthr) {
      const int r = t % rows, l = t / rows;
      Yt[r * kp + l] = (i0 + r < N) ? Y[(i0 + r) + int64_t(l) * ldy] : 0.0;
    }
    __syncthreads();
    double b0[NS], b1[NS];
    const double* y0 = Yt + (kTrsmRPW * warp) * kp;
    const double* y1 = y0 + kp;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const int l = 32 * s + lane;
      b0[s] = l < k ? y0[l] : 0.0;
      b1[s] = l < k ? y1[l] : 0.0;
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) {
#pragma unroll 8
      for (int o = 0; o < 32; ++o) {
        const int j = 32 * s + o;
        if (j >= k) break;
        const double rj_inv = rinv[j];
        const double x0 = __shfl_sync(kFull, b0[s], o) * rj_inv;
        const double x1 = __shfl_sync(kFull, b1[s], o) * rj_inv;
        const double* rj = Rs + rowoff(j, k) - j;  // rj[l] = R[j][l], l >= j
#pragma unroll
        for (int t = 0; t < NS; ++t) {
          if (t < s) continue;
          const int l = 32 * t + lane;
          if (l > j && l < k) {
            const double rv = rj[l];
            b0[t] = fma(-x0, rv, b0[t]);
            b1[t] = fma(-x1, rv, b1[t]);
          }
        }
      }
    }
    __syncthreads();  // every warp has read its rows of Yt
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const int l = 32 * s + lane;
      if (l < k) {
        Yt[(kTrsmRPW * warp) * kp + l] = b0[s] * rinv[l];
        Yt[(kTrsmRPW * warp + 1) * kp + l] = b1[s] * rinv[l];
      }
    }
    __syncthreads();
    for (int t = tid; t < rows * k; t += nthr) {
      const int r = t % rows, l = t / rows;
      if (i0 + r < N) Q[(i0 + r) + int64_t(l) * ldq] = Yt[r * kp + l];
    }
  }
}

size_t trsm_smem_bytes(int k, int warps) {
  return (size_t(k) * (k + 1) / 2 + size_t(k) + size_t(kTrsmRPW) * warps * (k | 1)) * 8;
}
// warps per CTA: 16 when their rows fit next to R, else fewer (at least 4)
int trsm_warps(int k) {
  int w = 16;
  while (w > 4 && trsm_smem_bytes(k, w) > kSmemMax) w /= 2;
  return w;
}

// round-robin pair pi of round r over kk (even) slots; p < q, valid when both < k.
// Both sums are below 2 (kk - 1), so one conditional subtraction replaces the modulo.
__device__ __forceinline__ bool rr_pair(int pi, int r, int kk, int k, int& p, int& q) {
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

constexpr int kJacThreads = 512;  // 64 groups of 8 lanes, one column pair each per round
// sketch width from which the Jacobi SVD runs on a cluster of 8 CTAs
constexpr int kClusterJacobiMinK = 96;

// One-sided Jacobi on X (m x k, rows zero-padded to 16 NV) held in shared
// memory.  Each 8-lane group takes one column pair per round: it reads both
// columns once into registers (two rows per lane and 16-byte access), forms
// the dot product, and writes the rotated columns back only when it rotates.
// The squared column norms are carried in shared memory (recomputed every
// sweep).  The rotation of pair slot pi in round r of sweep s is stored as
// (cos, sin) in rot[(s (kk-1) + r) kk/2 + pi] ((1, 0) when skipped).  The
// angle comes from rsqrt only: with d = b - a and h = sqrt(d^2 + 4c^2),
// cos 2t = |d|/h, sin 2t = 2c sgn(d)/h, cos t = sqrt((1 + cos 2t)/2),
// sin t = sin 2t / (2 cos t); (cos t, sin t) is orthonormal to rounding
// whatever the accuracy of the angle.
template <int NV>
__global__ void __launch_bounds__(kJacThreads) jacobi_log_kernel(double* Xg, int m, int k, int64_t ldx, double2* rot,
                                                                 int max_sweeps, double tol, double* S, int* status,
                                                                 int* sweeps_out) {
  extern __shared__ __align__(16) double X[];
  constexpr int mp = 16 * NV;
  double* nrm = X + int64_t(mp) * k;
  __shared__ int s_rot;
  const int tid = threadIdx.x, grp = tid >> 3, l8 = tid & 7;
  constexpr int ngrp = kJacThreads / 8;
  const int warp = tid >> 5, lane = tid & 31;
  constexpr int nwarps = kJacThreads / 32;
  for (int j = warp; j < k; j += nwarps)
    for (int i = lane; i < mp; i += 32) X[i + j * mp] = i < m ? Xg[i + int64_t(j) * ldx] : 0.0;
  __syncthreads();
  const int kk = (k + 1) & ~1, np = kk / 2;
  const double tol2 = tol * tol;
  int sweep = 0;
  bool converged = (k < 2);
  for (; sweep < max_sweeps && !converged; ++sweep) {
    for (int j = warp; j < k; j += nwarps) {
      double a = 0;
      for (int i = lane; i < mp; i += 32) a = fma(X[i + j * mp], X[i + j * mp], a);
      for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(kFull, a, o);
      if (lane == 0) nrm[j] = a;
    }
    if (tid == 0) s_rot = 0;
    __syncthreads();
    for (int r = 0; r < kk - 1; ++r) {
      double2* rr = rot + (size_t(sweep) * (kk - 1) + r) * np;
      // every lane runs the same trip count (the group shuffles use the full mask)
      for (int base = 0; base < np; base += ngrp) {
        const int pi = base + grp;
        int p = 0, q = 0;
        const bool valid = pi < np && rr_pair(pi, r, kk, k, p, q);
        double2* xp2 = reinterpret_cast<double2*>(X + p * mp) + l8;
        double2* xq2 = reinterpret_cast<double2*>(X + q * mp) + l8;
        double2 u[NV], v[NV];
        double c0 = 0, c1 = 0;
        if (valid) {
#pragma unroll
          for (int t = 0; t < NV; ++t) {
            u[t] = xp2[8 * t];
            v[t] = xq2[8 * t];
          }
#pragma unroll
          for (int t = 0; t < NV; ++t) {
            c0 = fma(u[t].x, v[t].x, c0);
            c1 = fma(u[t].y, v[t].y, c1);
          }
        }
        double cc = c0 + c1;
        cc += __shfl_xor_sync(kFull, cc, 1);
        cc += __shfl_xor_sync(kFull, cc, 2);
        cc += __shfl_xor_sync(kFull, cc, 4);
        double cs = 1.0, sn = 0.0;
        if (valid) {
          const double a = nrm[p], b = nrm[q];
          if (cc != 0.0 && a > 0.0 && b > 0.0 && cc * cc > tol2 * (a * b)) {
            const double d = b - a;
            const double rho = rsqrt(fma(d, d, 4.0 * cc * cc));
            const double c2 = fabs(d) * rho, s2 = copysign(1.0, d) * (2.0 * cc * rho);
            const double uu = 0.5 * (1.0 + c2);
            const double ru = rsqrt(uu);
            cs = uu * ru;
            sn = 0.5 * s2 * ru;
#pragma unroll
            for (int t = 0; t < NV; ++t) {
              xp2[8 * t] = make_double2(cs * u[t].x - sn * v[t].x, cs * u[t].y - sn * v[t].y);
              xq2[8 * t] = make_double2(sn * u[t].x + cs * v[t].x, sn * u[t].y + cs * v[t].y);
            }
            if (l8 == 0) {
              const double tc = 0.5 * s2 * cc * (ru * ru);  // tan(t) * c
              nrm[p] = a - tc;
              nrm[q] = b + tc;
              s_rot = 1;
            }
          }
        }
        if (pi < np && l8 == 0) rr[pi] = make_double2(cs, sn);
      }
      __syncthreads();
    }
    converged = (s_rot == 0);
    __syncthreads();
  }
  for (int j = warp; j < k; j += nwarps) {
    double a = 0;
    for (int i = lane; i < m; i += 32) {
      const double x = X[i + j * mp];
      a = fma(x, x, a);
      Xg[i + int64_t(j) * ldx] = x;
    }
    for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(kFull, a, o);
    if (lane == 0) S[j] = sqrt(a);
  }
  if (tid == 0) {
    if (!converged) atomicOr(status, 4);
    *sweeps_out = sweep;
  }
}

constexpr int kApplyRows = 8;  // rows of J per CTA, one warp each
constexpr int kChunk = 16;     // rounds of the log staged per step
constexpr int kMaxPairs = 128; // kk/2 <= 128 (k <= 256)

size_t apply_smem_bytes(int k) {
  const int np = ((k + 1) & ~1) / 2;
  return (size_t(2) * 2 * kChunk * np + size_t(kApplyRows) * k) * 8;
}

// J = product of the logged rotations, one warp per row of J (rows are
// independent: each sees the same sequence of column rotations).  The log
// streams through shared memory in chunks of kChunk rounds shared by the
// CTA's warps; the next chunk is loaded into registers while this one is
// applied.
__global__ void __launch_bounds__(kApplyRows * 32) jacobi_apply_kernel(const double2* rot, int k, const int* d_sweeps,
                                                                     double* J, int64_t ldj) {
  extern __shared__ __align__(16) double sm2[];
  const int kk = (k + 1) & ~1, np = kk / 2;
  double2* logb = reinterpret_cast<double2*>(sm2);  // 2 x kChunk x np
  double* rowbuf = sm2 + size_t(2) * 2 * kChunk * np;
  constexpr int nthr = kApplyRows * 32;
  constexpr int npre = (kChunk * kMaxPairs) / nthr;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int i = blockIdx.x * kApplyRows + warp;
  double* row = rowbuf + warp * k;
  for (int j = lane; j < k; j += 32) row[j] = (j == i) ? 1.0 : 0.0;
  const int nr = (*d_sweeps) * (kk - 1);
  const int nch = (nr + kChunk - 1) / kChunk;
  const int per = kChunk * np;
  for (int t = tid; t < per; t += nthr) logb[t] = (t / np < nr) ? rot[t] : make_double2(1.0, 0.0);
  __syncthreads();
  int r = 0;
  for (int ch = 0; ch < nch; ++ch) {
    const double2* cur = logb + (ch & 1) * per;
    double2* nxt = logb + ((ch + 1) & 1) * per;
    double2 pre[npre];
    const size_t base = size_t(ch + 1) * per;
#pragma unroll
    for (int s = 0; s < npre; ++s) {
      const int t = tid + nthr * s;
      pre[s] = (t < per && (ch + 1) * kChunk + t / np < nr) ? rot[base + t] : make_double2(1.0, 0.0);
    }
    if (i < k) {
      const int nrc = min(kChunk, nr - ch * kChunk);
      for (int c = 0; c < nrc; ++c) {
        const double2* g = cur + c * np;
        for (int pi = lane; pi < np; pi += 32) {
          const double2 gg = g[pi];
          int p, q;
          if (gg.y != 0.0 && rr_pair(pi, r, kk, k, p, q)) {
            const double jp = row[p], jq = row[q];
            row[p] = gg.x * jp - gg.y * jq;
            row[q] = gg.y * jp + gg.x * jq;
          }
        }
        __syncwarp();
        if (++r == kk - 1) r = 0;
      }
    }
#pragma unroll
    for (int s = 0; s < npre; ++s) {
      const int t = tid + nthr * s;
      if (t < per) nxt[t] = pre[s];
    }
    __syncthreads();
  }
  if (i < k)
    for (int j = lane; j < k; j += 32) J[i + int64_t(j) * ldj] = row[j];
}

// shared-memory opt-in, once per kernel and device
SmemAttrOnce g_chol_attr, g_ldl_attr[6], g_trsm_attr[9], g_jlog_attr[11], g_apply_attr;

template <int NBB>
void launch_ldl(Ctx& c, double* G, int k, int64_t ldg, double shift_factor, double* Rrow) {
  const size_t smem = chol_ldl_smem_doubles(k) * 8;
  g_ldl_attr[NBB].ensure(chol_ldl_kernel<NBB>, int(kSmemMax));
  chol_ldl_kernel<NBB><<<1, kLdlThreads, smem, c.stream>>>(G, k, ldg, shift_factor, Rrow);
}

template <int NV>
void launch_jacobi(Ctx& c, double* X, int m, int k, int64_t ldx, double2* rot, int max_sweeps, double tol, double* S,
                   int* d_sweeps, size_t smem) {
  g_jlog_attr[NV].ensure(jacobi_log_kernel<NV>, int(kSmemMax));
  jacobi_log_kernel<NV><<<1, kJacThreads, smem, c.stream>>>(X, m, k, ldx, rot, max_sweeps, tol, S, c.d_status, d_sweeps);
  IPEPS_LAUNCH_CHECK();
}

template <int NS>
void launch_trsm(Ctx& c, const double* Y, int64_t ldy, int64_t N, int k, const double* R, int64_t ldr,
                 const double* Rrow, double* Q, int64_t ldq) {
  const int warps = trsm_warps(k);
  const size_t smem = trsm_smem_bytes(k, warps);
  g_trsm_attr[NS].ensure(trsm_rows_kernel<NS>, int(kSmemMax));
  const int64_t rows = int64_t(warps) * kTrsmRPW;
  const unsigned grid = unsigned(std::min<int64_t>((N + rows - 1) / rows, std::max(c.sm_count, 1)));
  trsm_rows_kernel<NS><<<grid, warps * 32, smem, c.stream>>>(Y, ldy, N, k, R, ldr, Rrow, Q, ldq);
  IPEPS_LAUNCH_CHECK();
}

}  // namespace

bool chol_fits(int k) { return k >= 1 && chol_smem_doubles(k) * 8 <= kSmemMax; }

void chol_blocked(Ctx& c, double* G, int k, int64_t ldg, double shift_factor, double* Rrow) {
  IPEPS_CHECK(chol_fits(k), "chol_blocked: k too large for shared memory");
  ProfScope ps(c, KFam::SmallLinalg);
  if (k <= 160 && chol_ldl_smem_doubles(k) * 8 <= kSmemMax) {
    switch ((k + 31) / 32) {
      case 1: launch_ldl<1>(c, G, k, ldg, shift_factor, Rrow); break;
      case 2: launch_ldl<2>(c, G, k, ldg, shift_factor, Rrow); break;
      case 3: launch_ldl<3>(c, G, k, ldg, shift_factor, Rrow); break;
      case 4: launch_ldl<4>(c, G, k, ldg, shift_factor, Rrow); break;
      default: launch_ldl<5>(c, G, k, ldg, shift_factor, Rrow); break;
    }
  } else {
    g_chol_attr.ensure(chol_blocked_kernel, int(kSmemMax));
    chol_blocked_kernel<<<1, kCholThreads, chol_smem_doubles(k) * 8, c.stream>>>(G, k, ldg, shift_factor, Rrow);
  }
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::SmallLinalg, double(k) * k * k / 3.0);
}

bool trsm_fits(int k) { return k >= 1 && k <= 256 && trsm_smem_bytes(k, trsm_warps(k)) <= kSmemMax; }

void trsm_right_upper(Ctx& c, const double* Y, int64_t ldy, int64_t N, int k, const double* R, int64_t ldr, double* Q,
                      int64_t ldq, const double* Rrow) {
  IPEPS_CHECK(trsm_fits(k), "trsm_right_upper: k too large for shared memory");
  if (N == 0) return;
  ProfScope ps(c, KFam::SmallLinalg);
  switch ((k + 31) / 32) {
    case 1: launch_trsm<1>(c, Y, ldy, N, k, R, ldr, Rrow, Q, ldq); break;
    case 2: launch_trsm<2>(c, Y, ldy, N, k, R, ldr, Rrow, Q, ldq); break;
    case 3: launch_trsm<3>(c, Y, ldy, N, k, R, ldr, Rrow, Q, ldq); break;
    case 4: launch_trsm<4>(c, Y, ldy, N, k, R, ldr, Rrow, Q, ldq); break;
    case 5: launch_trsm<5>(c, Y, ldy, N, k, R, ldr, Rrow, Q, ldq); break;
    case 6: launch_trsm<6>(c, Y, ldy, N, k, R, ldr, Rrow, Q, ldq); break;
    case 7: launch_trsm<7>(c, Y, ldy, N, k, R, ldr, Rrow, Q, ldq); break;
    default: launch_trsm<8>(c, Y, ldy, N, k, R, ldr, Rrow, Q, ldq); break;
  }
  c.count(KFam::SmallLinalg, double(N) * k * k);
}

void jacobi_svd_auto(Ctx& c, double* X, int m, int k, int64_t ldx, double* J, int64_t ldj, double* S,
                     int max_sweeps, double tol, int* d_sweeps) {
  if (tol <= 0) tol = double(m) * 2.220446049250313e-16;  // rounding level of the column dot products
  if (k >= kClusterJacobiMinK && jacobi_cluster_fits(m, k)) {
    jacobi_svd_cluster(c, X, m, k, ldx, J, ldj, S, max_sweeps, tol, d_sweeps);
    return;
  }
  const int nv = (m + 15) / 16;
  const size_t smem = (size_t(16) * nv * k + k) * 8;
  if (k < 2 || nv > 10 || k > 2 * kMaxPairs || smem > kSmemMax || apply_smem_bytes(k) > kSmemMax) {
    jacobi_svd(c, X, m, k, ldx, J, ldj, S, max_sweeps, tol, d_sweeps);
    return;
  }
  const int kk = (k + 1) & ~1;
  Tensor rot = c.alloc(DType::F64, {int64_t(max_sweeps) * (kk - 1) * kk});  // double2 per pair slot
  double2* rp = reinterpret_cast<double2*>(rot.data());
  {
    ProfScope ps(c, KFam::Jacobi);
    switch (nv) {
      case 1: launch_jacobi<1>(c, X, m, k, ldx, rp, max_sweeps, tol, S, d_sweeps, smem); break;
      case 2: launch_jacobi<2>(c, X, m, k, ldx, rp, max_sweeps, tol, S, d_sweeps, smem); break;
      case 3: launch_jacobi<3>(c, X, m, k, ldx, rp, max_sweeps, tol, S, d_sweeps, smem); break;
      case 4: launch_jacobi<4>(c, X, m, k, ldx, rp, max_sweeps, tol, S, d_sweeps, smem); break;
      case 5: launch_jacobi<5>(c, X, m, k, ldx, rp, max_sweeps, tol, S, d_sweeps, smem); break;
      case 6: launch_jacobi<6>(c, X, m, k, ldx, rp, max_sweeps, tol, S, d_sweeps, smem); break;
      case 7: launch_jacobi<7>(c, X, m, k, ldx, rp, max_sweeps, tol, S, d_sweeps, smem); break;
      case 8: launch_jacobi<8>(c, X, m, k, ldx, rp, max_sweeps, tol, S, d_sweeps, smem); break;
      case 9: launch_jacobi<9>(c, X, m, k, ldx, rp, max_sweeps, tol, S, d_sweeps, smem); break;
      default: launch_jacobi<10>(c, X, m, k, ldx, rp, max_sweeps, tol, S, d_sweeps, smem); break;
    }
    c.count(KFam::Jacobi, 6.0 * double(m) * k * k / 2.0);
  }
  {
    ProfScope ps(c, KFam::Jacobi);
    g_apply_attr.ensure(jacobi_apply_kernel, int(kSmemMax));
    const unsigned grid = unsigned((k + kApplyRows - 1) / kApplyRows);
    jacobi_apply_kernel<<<grid, kApplyRows * 32, apply_smem_bytes(k), c.stream>>>(rp, k, d_sweeps, J, ldj);
    IPEPS_LAUNCH_CHECK();
    c.count(KFam::Jacobi, 6.0 * double(k) * k * k / 2.0);
  }
}

}  // namespace ipeps
