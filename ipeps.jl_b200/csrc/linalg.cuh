// Small dense FP64 linear algebra (single-CTA kernels) used by the projector.
#pragma once
#include "ctx.cuh"

namespace ipeps {

// In-place guarded Cholesky of a k x k SPD matrix: G = R^T R (upper R,
// strict lower triangle zeroed).  If d_trace_shift is given, shift_factor *
// (*d_trace_shift) is first added to the diagonal (shifted CholeskyQR).
void chol_upper(Ctx& c, double* G, int k, int64_t ldg, const double* d_trace_shift, double shift_factor);
// X = R^-1 (R upper triangular)
void triinv_upper(Ctx& c, const double* R, int k, int64_t ldr, double* X, int64_t ldx);
// d_out = trace(G)
void trace(Ctx& c, const double* G, int k, int64_t ldg, double* d_out);
// One-sided Jacobi on the m x k matrix X: X <- X J with orthogonal columns,
// J accumulated (k x k), S = column norms (unsorted).
void jacobi_svd(Ctx& c, double* X, int m, int k, int64_t ldx, double* J, int64_t ldj, double* S,
                int max_sweeps, double tol, int* d_sweeps);
// Blocked guarded Cholesky in shared memory (packed upper triangle, 32-column
// panels): G <- R with G = R^T R after adding shift_factor * trace(G) to the
// diagonal when shift_factor > 0; a pivot at or below 1e-32 trace(G) gives
// R[j][j] = 1 and a zero row.  Requires chol_fits(k).
bool chol_fits(int k);
// Rrow (optional, k(k+1)/2 doubles, 16-byte aligned): R packed row by row, for trsm_right_upper.
void chol_blocked(Ctx& c, double* G, int k, int64_t ldg, double shift_factor, double* Rrow = nullptr);
// Q = Y R^-1 (Y: N x k, R: k x k upper triangular), one warp per row of Y.
// Requires trsm_fits(k).
bool trsm_fits(int k);
// Rrow (optional): the same R packed row by row as written by chol_blocked.
void trsm_right_upper(Ctx& c, const double* Y, int64_t ldy, int64_t N, int k, const double* R, int64_t ldr,
                      double* Q, int64_t ldq, const double* Rrow = nullptr);
// jacobi_svd with X held in shared memory and J formed from the logged
// rotations when it fits; tol <= 0 means m * eps
void jacobi_svd_auto(Ctx& c, double* X, int m, int k, int64_t ldx, double* J, int64_t ldj, double* S,
                     int max_sweeps, double tol, int* d_sweeps);
// The same SVD on a cluster of 8 CTAs (J carried with X, distributed shared
// memory between rounds); jacobi_cluster_fits says whether (m, k) fits.
bool jacobi_cluster_fits(int m, int k);
void jacobi_svd_cluster(Ctx& c, double* X, int m, int k, int64_t ldx, double* J, int64_t ldj, double* S,
                        int max_sweeps, double tol, int* d_sweeps);
// Complex (complex128) counterparts for complex iPEPS tensors, one CTA each;
// complex_small_fits(m, k) says whether all three fit in shared memory.
bool complex_small_fits(int m, int k);
void chol_c(Ctx& c, void* G, int k, int64_t ldg, double shift_factor);
void trsm_c(Ctx& c, const void* Y, int64_t ldy, int64_t N, int k, const void* R, int64_t ldr, void* Q, int64_t ldq);
void jacobi_c_svd(Ctx& c, void* X, int m, int k, int64_t ldx, void* J, int64_t ldj, double* S, int max_sweeps,
                  double tol, int* d_sweeps);
// Descending sort with permutation (ties: later index first)
void sort_desc(Ctx& c, const double* S, int k, double* S_out, int* perm);
// out[:, j] = in[:, perm[j]] * f(scale[j]); scale_mode 0: 1, 1: scale, 2: 1/scale
void gather_cols(Ctx& c, const double* in, int64_t ldi, int64_t m, const int* perm, int ncols,
                 const double* scale_v, int scale_mode, double* out, int64_t ldo);
// X[:, j] *= f(s[j]); mode 1: 1/sqrt(s), 0: s
void scale_cols(Ctx& c, double* X, int64_t ldx, int64_t m, int ncols, const double* s, int mode);
// X[i, :] *= f(s[i]); mode 1: 1/sqrt(s), 0: s
void scale_rows(Ctx& c, double* X, int64_t ldx, int64_t m, int64_t ncols, const double* s, int mode);

}  // namespace ipeps
