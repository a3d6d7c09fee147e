// Real FP64 GEMM on the FP64 tensor-core path (DMMA, mma.sync m8n8k4 .f64).
//
// tcgen05 has no FP64 kind, so FP64 matrix products on sm_100a go through the
// warp-level DMMA instruction.  Its point over a DFMA kernel is operand reuse:
// one m8n8k4 takes one A and one B value per lane and does 256 FMAs per warp,
// so a warp tile of 64x32 (or 32x32) reads shared memory at a quarter of the
// rate a register-tiled DFMA kernel needs for the same FMAs; the DFMA kernel
// was bound by shared-memory bandwidth (16 doubles per SM cycle for 64 FMAs).
//
//   C = alpha op(A) op(B) + beta C, column-major, op in {N, T}
//
// Tiles BM x BN x 16, staged by cp.async (16-byte chunks when the operand is
// 16-byte aligned with an even leading dimension, else 8-byte) through a
// three-stage shared-memory ring.  Each operand keeps its global contiguity in
// shared memory: k-contiguous operands as [mn][16 + 4], mn-contiguous ones as
// [16][BMN + 4]; both paddings make the fragment loads of a warp (8 rows x 4
// columns of doubles) conflict-free.  Out-of-range elements are zero-filled by
// the copy (src-size 0 or 8), so tiles at the edges need no special path.
// Skinny problems use a deterministic split-K: the partial products of each
// K chunk go to a workspace and are summed in a fixed order.
#include "ctx.cuh"

#include <atomic>

#include <algorithm>

namespace ipeps {
namespace {

constexpr int kBK = 16;
constexpr int kStages = 3;
constexpr int kPad = 4;

__device__ __forceinline__ unsigned su32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ int64_t imin(int64_t a, int64_t b) { return a < b ? a : b; }
__device__ __forceinline__ int64_t imax(int64_t a, int64_t b) { return a > b ? a : b; }

template <int VEC>
__device__ __forceinline__ void cp_async(double* dst, const double* src, int bytes) {
  if constexpr (VEC == 2) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(su32(dst)), "l"(src), "r"(bytes));
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(su32(dst)), "l"(src), "r"(bytes));
  }
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Shared-memory geometry of one operand tile (BMN rows of the m or n index).
template <int BMN, bool KMAJ>
struct Tile {
  static constexpr int ld = KMAJ ? (kBK + kPad) : (BMN + kPad);  // doubles per stored row
  static constexpr int size = KMAJ ? BMN * ld : kBK * ld;         // doubles per stage
  // element (mn, k) of the tile
  static __device__ __forceinline__ int at(int mn, int k) { return KMAJ ? mn * ld + k : k * ld + mn; }
};

// Copy the operand tile [mn0, mn0 + BMN) x [k0, k0 + 16) into shared memory.
// Global layout: KMAJ: element (mn, k) at P[k + mn * ld]; else at P[mn + k * ld].
template <int BMN, bool KMAJ, int VEC, int NT>
__device__ __forceinline__ void load_tile(double* s, const double* __restrict__ P, int64_t ldp, int64_t MN,
                                          int64_t mn0, int64_t k0, int64_t ke, int tid) {
  using T = Tile<BMN, KMAJ>;
  constexpr int inner = KMAJ ? kBK : BMN;  // contiguous extent
  constexpr int outer = KMAJ ? BMN : kBK;
  constexpr int chunks = inner / VEC * outer;
  static_assert(chunks % NT == 0, "tile chunks must divide evenly over the threads");
#pragma unroll
  for (int r = 0; r < chunks / NT; ++r) {
    const int e = tid + r * NT;
    const int i = (e % (inner / VEC)) * VEC, o = e / (inner / VEC);
    const int mn = KMAJ ? o : i, k = KMAJ ? i : o;
    const int64_t gmn = mn0 + mn, gk = k0 + k;
    int64_t valid;
    const double* src;
    if (KMAJ) {
      valid = (gmn < MN) ? imin(VEC, imax(0, ke - gk)) : 0;
      src = P + gk + gmn * ldp;
    } else {
      valid = (gk < ke) ? imin(VEC, imax(0, MN - gmn)) : 0;
      src = P + gmn + gk * ldp;
    }
    if (valid == 0) src = P;  // any valid address; nothing is read
    cp_async<VEC>(s + T::at(mn, k), src, int(valid) * 8);
  }
}

template <int BM, int BN, int WGM, int WGN, bool AK, bool BK_, int VEC>
__global__ void __launch_bounds__(WGM * WGN * 32)
    dmma_gemm_kernel(int64_t M, int64_t N, int64_t K, int64_t kchunk, double alpha, const double* __restrict__ A,
                     int64_t lda, const double* __restrict__ B, int64_t ldb, double beta, double* __restrict__ C,
                     int64_t ldc, double* __restrict__ partial) {
  constexpr int NT = WGM * WGN * 32;
  constexpr int WM = BM / WGM, WN = BN / WGN;  // warp tile
  constexpr int TI = WM / 8, TJ = WN / 8;      // 8x8 DMMA tiles per warp
  using TA = Tile<BM, AK>;
  using TB = Tile<BN, BK_>;
  extern __shared__ __align__(16) double smem[];
  double* sA = smem;
  double* sB = smem + kStages * TA::size;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm0 = (warp % WGM) * WM, wn0 = (warp / WGM) * WN;
  const int64_t m0 = int64_t(blockIdx.x) * BM, n0 = int64_t(blockIdx.y) * BN;
  const int64_t kb = int64_t(blockIdx.z) * kchunk;
  const int64_t ke = imin(K, kb + kchunk);
  const int nk = ke > kb ? int((ke - kb + kBK - 1) / kBK) : 0;

  double acc[TI][TJ][2];
#pragma unroll
  for (int i = 0; i < TI; ++i)
#pragma unroll
    for (int j = 0; j < TJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  // B is consumed as (k, n): its "mn" index is n and it is k-contiguous when op(B) = N
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nk) {
      load_tile<BM, AK, VEC, NT>(sA + s * TA::size, A, lda, M, m0, kb + s * kBK, ke, tid);
      load_tile<BN, BK_, VEC, NT>(sB + s * TB::size, B, ldb, N, n0, kb + s * kBK, ke, tid);
    }
    cp_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_wait<kStages - 2>();
    __syncthreads();
    const int pf = kt + kStages - 1;
    if (pf < nk) {
      const int st = pf % kStages;
      load_tile<BM, AK, VEC, NT>(sA + st * TA::size, A, lda, M, m0, kb + int64_t(pf) * kBK, ke, tid);
      load_tile<BN, BK_, VEC, NT>(sB + st * TB::size, B, ldb, N, n0, kb + int64_t(pf) * kBK, ke, tid);
    }
    cp_commit();
    const double* a_s = sA + (kt % kStages) * TA::size;
    const double* b_s = sB + (kt % kStages) * TB::size;
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 4) {
      double a[TI], b[TJ];
#pragma unroll
      for (int i = 0; i < TI; ++i) a[i] = a_s[TA::at(wm0 + i * 8 + g, kk + t)];
#pragma unroll
      for (int j = 0; j < TJ; ++j) b[j] = b_s[TB::at(wn0 + j * 8 + g, kk + t)];
#pragma unroll
      for (int i = 0; i < TI; ++i)
#pragma unroll
        for (int j = 0; j < TJ; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
  }
  cp_wait<0>();

  // epilogue: lane holds rows g, columns 2t and 2t+1 of each 8x8 tile
#pragma unroll
  for (int i = 0; i < TI; ++i) {
    const int64_t gm = m0 + wm0 + i * 8 + g;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < TJ; ++j) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t gn = n0 + wn0 + j * 8 + 2 * t + e;
        if (gn >= N) continue;
        if (partial) {
          partial[int64_t(blockIdx.z) * M * N + gm + gn * M] = acc[i][j][e];
        } else {
          double v = alpha * acc[i][j][e];
          if (beta != 0.0) v = fma(beta, C[gm + gn * ldc], v);
          C[gm + gn * ldc] = v;
        }
      }
    }
  }
}

// Sum of the S split-K partial products (in split order, so the result does
// not depend on the launch).  Contiguous C (ldc == M) takes two elements per
// thread with 16-byte loads; the general case one element per thread.
__global__ void dmma_splitk_reduce(int64_t M, int64_t N, int S, const double* __restrict__ partial, double alpha,
                                   double beta, double* __restrict__ C, int64_t ldc) {
  const int64_t tot = M * N;
  if (ldc == M && (tot & 1) == 0 && (reinterpret_cast<uintptr_t>(C) & 15) == 0) {
    const int64_t i2 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, idx = 2 * i2;
    if (idx >= tot) return;
    double2 acc = *reinterpret_cast<const double2*>(partial + idx);
    for (int z = 1; z < S; ++z) {
      const double2 p = *reinterpret_cast<const double2*>(partial + int64_t(z) * tot + idx);
      acc.x += p.x;
      acc.y += p.y;
    }
    double2 v = make_double2(alpha * acc.x, alpha * acc.y);
    if (beta != 0.0) {
      const double2 c = *reinterpret_cast<const double2*>(C + idx);
      v.x = fma(beta, c.x, v.x);
      v.y = fma(beta, c.y, v.y);
    }
    *reinterpret_cast<double2*>(C + idx) = v;
    return;
  }
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= tot) return;
  const int64_t gn = idx / M, gm = idx - gn * M;
  double s = partial[idx];
  for (int z = 1; z < S; ++z) s += partial[int64_t(z) * tot + idx];
  double v = alpha * s;
  if (beta != 0.0) v = fma(beta, C[gm + gn * ldc], v);
  C[gm + gn * ldc] = v;
}

template <int BM, int BN, int WGM, int WGN, bool AK, bool BK_, int VEC>
void launch_cfg(Ctx& c, int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda,
                const double* B, int64_t ldb, double beta, double* C, int64_t ldc) {
  constexpr int NT = WGM * WGN * 32;
  constexpr size_t smem = size_t(kStages) * (Tile<BM, AK>::size + Tile<BN, BK_>::size) * sizeof(double);
  auto kern = dmma_gemm_kernel<BM, BN, WGM, WGN, AK, BK_, VEC>;
  static SmemAttrOnce attr;
  attr.ensure(kern, int(smem));
  const int64_t gx = (m + BM - 1) / BM, gy = (n + BN - 1) / BN;
  IPEPS_CHECK(gy <= 65535, "gemm: n too large for grid");
  const int64_t tiles = gx * gy;
  int S = 1;
  // split K when the output grid covers well under four CTAs per SM and K is
  // long: up to four per SM in total (a 64 x 64 output with K ~ 1e5, the
  // gradient of A, would otherwise run on a few dozen SMs; finer splits also
  // even out the last wave), at least 8 K blocks per split
  const int64_t target = 4LL * c.sm_count;
  if (tiles < target && k >= 16 * kBK) {
    const int64_t want = (target + tiles - 1) / tiles;
    const int64_t maxs = k / (8 * kBK);
    S = int(std::max<int64_t>(1, std::min<int64_t>(want, maxs)));
  }
  int64_t kchunk = (k + S - 1) / S;
  kchunk = ((kchunk + kBK - 1) / kBK) * kBK;
  S = int((k + kchunk - 1) / kchunk);
  if (S < 1) S = 1;
  double* partial = nullptr;
  if (S > 1) partial = static_cast<double*>(c.workspace(size_t(S) * m * n * sizeof(double)));
  dim3 grid{unsigned(gx), unsigned(gy), unsigned(S)};
  kern<<<grid, NT, smem, c.stream>>>(m, n, k, kchunk, alpha, A, lda, B, ldb, beta, C, ldc, partial);
  IPEPS_LAUNCH_CHECK();
  if (S > 1) {
    const int64_t tot = m * n;
    const bool pairs = ldc == m && (tot & 1) == 0 && (reinterpret_cast<uintptr_t>(C) & 15) == 0;
    const int64_t threads = pairs ? tot / 2 : tot;
    dmma_splitk_reduce<<<unsigned((threads + 255) / 256), 256, 0, c.stream>>>(m, n, S, partial, alpha, beta, C, ldc);
    IPEPS_LAUNCH_CHECK();
    c.count(KFam::Reduce, 0, double(S + 2) * tot * sizeof(double));
  }
}

template <int BM, int BN, int WGM, int WGN, int VEC>
void launch_ops(Ctx& c, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
                int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc) {
  // A is k-contiguous when op(A) = T; B is k-contiguous when op(B) = N
  if (ta && !tb)
    launch_cfg<BM, BN, WGM, WGN, true, true, VEC>(c, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  else if (ta && tb)
    launch_cfg<BM, BN, WGM, WGN, true, false, VEC>(c, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  else if (!ta && !tb)
    launch_cfg<BM, BN, WGM, WGN, false, true, VEC>(c, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  else
    launch_cfg<BM, BN, WGM, WGN, false, false, VEC>(c, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

}  // namespace

void gemm_f64_dmma(Ctx& c, char opA, char opB, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
                   int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc) {
  if (m <= 0 || n <= 0) return;
  IPEPS_CHECK(k > 0, "gemm: k == 0 is not supported");
  const bool ta = (opA == 'T' || opA == 't'), tb = (opB == 'T' || opB == 't');
  IPEPS_CHECK(ta || opA == 'N' || opA == 'n', "gemm: bad op");
  IPEPS_CHECK(tb || opB == 'N' || opB == 'n', "gemm: bad op");
  ProfScope ps(c, KFam::GemmF64);
  const bool vec = (reinterpret_cast<uintptr_t>(A) % 16 == 0) && (reinterpret_cast<uintptr_t>(B) % 16 == 0) &&
                   lda % 2 == 0 && ldb % 2 == 0;
  const int64_t big_tiles = ((m + 127) / 128) * ((n + 127) / 128);
  // one narrow side (<= 64, e.g. a leg of D^2 d = 50 in the contractions with
  // A): 128x64 / 64x128 tiles, so that half of a 128x128 tile is not wasted
  if (n <= 64 && ((m + 127) / 128) >= c.sm_count) {
    if (vec)
      launch_ops<128, 64, 4, 2, 2>(c, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else
      launch_ops<128, 64, 4, 2, 1>(c, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  } else if (m <= 64 && ((n + 127) / 128) >= c.sm_count) {
    if (vec)
      launch_ops<64, 128, 2, 4, 2>(c, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else
      launch_ops<64, 128, 2, 4, 1>(c, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  } else if (k <= 256 && ((m + 127) / 128) * ((n + 63) / 64) >= 2 * c.sm_count) {
    // short K (e.g. a bond of chi = 100): the 128x64 tiles hold two CTAs per SM
    // (<= 128 registers, 92 KB of shared memory), which hides the load latency
    // of the few K steps better than one 128x128 CTA
    if (vec)
      launch_ops<128, 64, 4, 2, 2>(c, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else
      launch_ops<128, 64, 4, 2, 1>(c, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  } else if (big_tiles >= c.sm_count) {
    if (vec)
      launch_ops<128, 128, 2, 4, 2>(c, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else
      launch_ops<128, 128, 2, 4, 1>(c, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  } else {
    if (vec)
      launch_ops<64, 64, 2, 2, 2>(c, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else
      launch_ops<64, 64, 2, 2, 1>(c, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  }
  c.count(KFam::GemmF64, 2.0 * double(m) * double(n) * double(k));
}

}  // namespace ipeps
