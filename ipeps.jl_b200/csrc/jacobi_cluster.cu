// One-sided Jacobi SVD of the projector's k x k Rayleigh-Ritz matrix on a
// thread-block cluster of 8 CTAs (8 SMs) instead of one CTA.
//
// The columns of [X; J] (J starts as the identity and accumulates the
// rotations, so no separate pass forms it) are cut into 16 blocks of b
// columns; each CTA holds two blocks in shared memory.  A sweep is the
// block round robin of 15 rounds (the circle method over 16 block
// positions): in round 0 each CTA also orthogonalises the column pairs
// inside its two blocks, and in every round all b x b pairs between its two
// blocks, b disjoint pairs at a time (one warp per pair; the first block's
// column stays in the warp's registers for the whole round).  Between rounds
// every CTA writes its two blocks into the shared memory of the CTAs that
// hold those block positions next (distributed shared memory, double
// buffered), and the cluster barrier orders the exchange.  Every pair of
// columns meets exactly once per sweep, as in the cyclic Jacobi method.  The
// sweep loop ends when no CTA rotated (an all-to-all flag exchange) or at
// max_sweeps (status bit 4).  The rotation (angle from rsqrt only, as the
// single-CTA kernel) and the threshold |x_p.x_q| > tol |x_p| |x_q| are those
// of the single-CTA kernel, so the result is the same SVD up to rounding.
#include "linalg.cuh"

#include <cooperative_groups.h>

namespace ipeps {
namespace {

namespace cg = cooperative_groups;

constexpr int kJP = 8;                 // CTAs per cluster (portable cluster size)
constexpr int kJBlocks = 2 * kJP;      // column blocks
constexpr int kJWarps = 16;            // warps per CTA (>= b)
constexpr int kJMaxRowsPerLane = 16;   // H <= 512
constexpr size_t kJSmemMax = 200 * 1024;

struct JcArgs {
  const double* X;
  int64_t ldx;
  int m, k, b, H;  // rows of X, columns, block width (even), padded height of [X; J]
  int max_sweeps;
  double tol2;
  double* Xout;
  double* J;
  int64_t ldj;
  double* S;
  int* status;
  int* sweeps_out;
};

// circle-method pair w of round t among n (even) players
__device__ __forceinline__ void circle_pair(int w, int t, int n, int& p, int& q) {
  const int n1 = n - 1;
  int a = w - 1 + t;
  a %= n1;
  int c = n - 2 - w + t;
  c %= n1;
  p = (w == 0) ? 0 : 1 + a;
  q = 1 + c;
}

// position p of the block round robin -> (cluster rank, slot)
__device__ __forceinline__ void pos_owner(int p, int& rank, int& slot) {
  if (p < kJP) {
    rank = p;
    slot = 0;
  } else {
    rank = kJBlocks - 1 - p;
    slot = 1;
  }
}

// rotate columns u (registers) and the shared column y; returns true when it rotated
__device__ __forceinline__ bool rotate_pair(double (&u)[kJMaxRowsPerLane], double* y, int m, int H, int lane,
                                            double tol2) {
  double v[kJMaxRowsPerLane];
  double a = 0, bb = 0, c = 0;
#pragma unroll
  for (int j = 0; j < kJMaxRowsPerLane; ++j) {
    const int r = lane + 32 * j;
    v[j] = (r < H) ? y[r] : 0.0;
    if (r < m) {
      a = fma(u[j], u[j], a);
      bb = fma(v[j], v[j], bb);
      c = fma(u[j], v[j], c);
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    bb += __shfl_xor_sync(0xffffffffu, bb, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if (!(c != 0.0 && a > 0.0 && bb > 0.0 && c * c > tol2 * (a * bb))) return false;
  const double d = bb - a;
  const double rho = rsqrt(fma(d, d, 4.0 * c * c));
  const double c2 = fabs(d) * rho, s2 = copysign(1.0, d) * (2.0 * c * rho);
  const double uu = 0.5 * (1.0 + c2);
  const double ru = rsqrt(uu);
  const double cs = uu * ru, sn = 0.5 * s2 * ru;
#pragma unroll
  for (int j = 0; j < kJMaxRowsPerLane; ++j) {
    const int r = lane + 32 * j;
    const double up = cs * u[j] - sn * v[j], vq = sn * u[j] + cs * v[j];
    u[j] = up;
    if (r < H) y[r] = vq;
  }
  return true;
}

__device__ __forceinline__ void load_col(double (&u)[kJMaxRowsPerLane], const double* x, int H, int lane) {
#pragma unroll
  for (int j = 0; j < kJMaxRowsPerLane; ++j) {
    const int r = lane + 32 * j;
    u[j] = (r < H) ? x[r] : 0.0;
  }
}

__device__ __forceinline__ void store_col(const double (&u)[kJMaxRowsPerLane], double* x, int H, int lane) {
#pragma unroll
  for (int j = 0; j < kJMaxRowsPerLane; ++j) {
    const int r = lane + 32 * j;
    if (r < H) x[r] = u[j];
  }
}

__global__ void __cluster_dims__(kJP, 1, 1) __launch_bounds__(kJWarps * 32, 1) jacobi_cluster_kernel(JcArgs a) {
  extern __shared__ __align__(16) double jsm[];
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = int(cluster.block_rank());
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int b = a.b, H = a.H, m = a.m;
  const size_t slot_sz = size_t(b) * H;
  // buf[cur][slot] columns, then the block ids of the slots per buffer, then the flags
  double* buf = jsm;
  int* blk = reinterpret_cast<int*>(jsm + 4 * slot_sz);  // [2 buffers][2 slots]
  int* flags = blk + 4;                                   // [kJP]
  __shared__ int s_rot;

  int cur = 0;
  if (tid < 2) blk[tid] = (tid == 0) ? rank : kJBlocks - 1 - rank;
  __syncthreads();
  // load [X; I] columns of both blocks (columns >= k are zero)
  for (int s = 0; s < 2; ++s) {
    double* dst = buf + (0 * 2 + s) * slot_sz;
    const int b0 = blk[s] * b;
    for (int j = warp; j < b; j += kJWarps) {
      const int col = b0 + j;
      for (int r = lane; r < H; r += 32) {
        double v = 0.0;
        if (col < a.k) {
          if (r < m) v = a.X[r + int64_t(col) * a.ldx];
          else if (r - m == col) v = 1.0;
        }
        dst[j * H + r] = v;
      }
    }
  }
  cluster.sync();

  int sweep = 0;
  bool converged = false;
  for (; sweep < a.max_sweeps && !converged; ++sweep) {
    if (tid == 0) s_rot = 0;
    __syncthreads();
    bool rot = false;
    for (int round = 0; round < kJBlocks - 1; ++round) {
      double* A = buf + (cur * 2 + 0) * slot_sz;
      double* B = buf + (cur * 2 + 1) * slot_sz;
      if (round == 0) {
        // pairs inside each block: b - 1 sub-rounds of b/2 pairs per block
        for (int t = 0; t < b - 1; ++t) {
          for (int w = warp; w < b; w += kJWarps) {
            double* base = (w < b / 2) ? A : B;
            int p, q;
            circle_pair(w % (b / 2), t, b, p, q);
            double u[kJMaxRowsPerLane];
            load_col(u, base + size_t(p) * H, H, lane);
            if (rotate_pair(u, base + size_t(q) * H, m, H, lane, a.tol2)) {
              store_col(u, base + size_t(p) * H, H, lane);
              rot = true;
            }
          }
          __syncthreads();
        }
      }
      // pairs between the two blocks: warp i keeps column A_i, meets B_{(i+t) % b}
      for (int i = warp; i < b; i += kJWarps) {
        double u[kJMaxRowsPerLane];
        load_col(u, A + size_t(i) * H, H, lane);
        bool any = false;
        for (int t = 0; t < b; ++t) {
          // B columns are touched by one warp per sub-round: sync the warps that share them
          if (rotate_pair(u, B + size_t((i + t) % b) * H, m, H, lane, a.tol2)) any = true;
          asm volatile("bar.sync 1, %0;" ::"r"(((b + 0) < kJWarps ? b : kJWarps) * 32) : "memory");
        }
        if (any) {
          store_col(u, A + size_t(i) * H, H, lane);
          rot = true;
        }
      }
      __syncthreads();
      // hand both blocks to the CTAs that hold their next positions
      const int nxt = cur ^ 1;
      for (int s = 0; s < 2; ++s) {
        const int pos = (s == 0) ? rank : kJBlocks - 1 - rank;
        const int np = (pos == 0) ? 0 : (pos == kJBlocks - 1 ? 1 : pos + 1);
        int drank, dslot;
        pos_owner(np, drank, dslot);
        double* src = buf + (cur * 2 + s) * slot_sz;
        double* dst = cluster.map_shared_rank(buf + (nxt * 2 + dslot) * slot_sz, drank);
        for (size_t e = tid; e < slot_sz; e += kJWarps * 32) dst[e] = src[e];
        if (tid == 0) *cluster.map_shared_rank(blk + nxt * 2 + dslot, drank) = blk[cur * 2 + s];
      }
      cluster.sync();
      cur = nxt;
    }
    // did any CTA rotate in this sweep?
    if (rot) s_rot = 1;
    __syncthreads();
    if (tid < kJP) *cluster.map_shared_rank(flags + rank, tid) = s_rot;
    cluster.sync();
    int any = 0;
    for (int r = 0; r < kJP; ++r) any |= flags[r];
    converged = (any == 0);
    cluster.sync();  // flags are rewritten only after every CTA has read them
  }

  // write back W = X J columns, J, and the column norms of W
  for (int s = 0; s < 2; ++s) {
    const double* src = buf + (cur * 2 + s) * slot_sz;
    const int b0 = blk[cur * 2 + s] * b;
    for (int j = warp; j < b; j += kJWarps) {
      const int col = b0 + j;
      if (col >= a.k) continue;
      double nn = 0;
      for (int r = lane; r < H; r += 32) {
        const double v = src[j * H + r];
        if (r < m) {
          a.Xout[r + int64_t(col) * a.ldx] = v;
          nn = fma(v, v, nn);
        } else if (r - m < a.k) {
          a.J[(r - m) + int64_t(col) * a.ldj] = v;
        }
      }
#pragma unroll
      for (int o = 16; o; o >>= 1) nn += __shfl_xor_sync(0xffffffffu, nn, o);
      if (lane == 0) a.S[col] = sqrt(nn);
    }
  }
  if (rank == 0 && tid == 0) {
    if (!converged) atomicOr(a.status, 4);
    *a.sweeps_out = sweep;
  }
  cluster.sync();
}

SmemAttrOnce g_jc_attr;

}  // namespace

bool jacobi_cluster_fits(int m, int k) {
  if (m < 1 || k < 2 || k > 2 * kJBlocks * 16) return false;
  const int kk = (k + 1) & ~1;
  int b = (kk + kJBlocks - 1) / kJBlocks;
  b += b & 1;
  const int H = ((m + k + 31) / 32) * 32;
  return b <= kJWarps && H <= 32 * kJMaxRowsPerLane && (size_t(4) * b * H + 64) * 8 <= kJSmemMax;
}

void jacobi_svd_cluster(Ctx& c, double* X, int m, int k, int64_t ldx, double* J, int64_t ldj, double* S,
                        int max_sweeps, double tol, int* d_sweeps) {
  IPEPS_CHECK(jacobi_cluster_fits(m, k), "jacobi_svd_cluster: problem does not fit");
  if (tol <= 0) tol = double(m) * 2.220446049250313e-16;
  const int kk = (k + 1) & ~1;
  int b = (kk + kJBlocks - 1) / kJBlocks;
  b += b & 1;
  JcArgs a{};
  a.X = X;
  a.ldx = ldx;
  a.m = m;
  a.k = k;
  a.b = b;
  a.H = ((m + k + 31) / 32) * 32;
  a.max_sweeps = max_sweeps;
  a.tol2 = tol * tol;
  a.Xout = X;
  a.J = J;
  a.ldj = ldj;
  a.S = S;
  a.status = c.d_status;
  a.sweeps_out = d_sweeps;
  const size_t smem = (size_t(4) * b * a.H + 64) * 8;
  g_jc_attr.ensure(jacobi_cluster_kernel, int(kJSmemMax));
  ProfScope ps(c, KFam::Jacobi);
  jacobi_cluster_kernel<<<kJP, kJWarps * 32, smem, c.stream>>>(a);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Jacobi, 6.0 * double(m + k) * k * k / 2.0);
}

}  // namespace ipeps
