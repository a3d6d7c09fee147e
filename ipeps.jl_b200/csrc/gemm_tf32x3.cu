// 3xTF32 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// C = alpha*op(A)*op(B) + beta*C with FP64 operands in global memory
// (column-major, op in {N, T}).  Each FP64 value a is split into
//   a_hi = tf32(a),  a_lo = tf32(a - a_hi)
// and the product is accumulated in FP32 in tensor memory as
//   a_lo*b_hi + a_hi*b_lo + a_hi*b_hi,
// which carries ~22 mantissa bits per product (FP32-equivalent accuracy).
//
// CTA tile 128 x 128, K-step 32, 3-stage shared-memory ring.  Warp roles:
//   warps 0-3  producers: FP64 global loads, split into hi/lo TF32, stores
//              into the 128B-swizzled K-major layout the UMMA descriptors
//              describe (no TMA, so any leading dimension / alignment works);
//              then the epilogue (tcgen05.ld of their 32 TMEM lanes each)
//   warp 4     TMEM allocation and the single-thread tcgen05.mma issue.
// Stage hand-off uses mbarriers: producers arrive on full[s] after a
// fence.proxy.async; the MMA thread commits (tcgen05.commit) to empty[s] and,
// after the last K-step, to the accumulator barrier.  Every wait is bounded:
// on timeout the kernel records bit 8 in the status word and drains.
#include "umma.cuh"

#include <atomic>

#include <algorithm>

namespace ipeps {
namespace {

constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3;
constexpr int TILE_BYTES = BM * BK * 4;            // 16 KB per operand tile (A or B, hi or lo)
constexpr int STAGE_BYTES = 4 * TILE_BYTES;        // A_hi, A_lo, B_hi, B_lo
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
constexpr int NTHREADS = 160;
constexpr uint32_t TMEM_COLS = 128;

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// instruction descriptor: D = F32, A = B = TF32, both K-major, M = 128, N = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(BN >> 3) << 17) |
                           (uint32_t(BM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem), "l"(da), "l"(db), "r"(IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

struct Args {
  int64_t M, N, K, kchunk;
  int opA, opB;  // 0 = N, 1 = T
  const double* A;
  int64_t lda;
  const double* B;
  int64_t ldb;
  double alpha, beta;
  double* C;
  int64_t ldc;
  double* partial;
  int* status;
};

// Load a 128 x 32 logical tile X(row, k) (rows [row0, row0+128), k [k0, k0+32))
// split into hi/lo TF32 swizzled tiles.  rowc: rows are contiguous in memory
// (X(row,k) = P[row + k*ld]); otherwise k is contiguous (X(row,k) = P[k + row*ld]).
__device__ __forceinline__ void load_split(const double* __restrict__ P, int64_t ld, bool rowc, int64_t row0,
                                           int64_t nrows, int64_t k0, int64_t kend, char* hi, char* lo, int t) {
  if (rowc) {
    // thread t owns row t; 8 chunks of 4 k each
    const int r = t;
    const int64_t gr = row0 + r;
#pragma unroll 2
    for (int c = 0; c < 8; ++c) {
      uint32_t h[4], l[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int64_t gk = k0 + 4 * c + i;
        double v = (gr < nrows && gk < kend) ? __ldg(P + gr + gk * ld) : 0.0;
        h[i] = to_tf32(float(v));
        l[i] = to_tf32(float(v - double(__uint_as_float(h[i]))));
      }
      const uint32_t off = sw128(r, c);
      *reinterpret_cast<uint4*>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
  } else {
    // thread t owns chunk t%8 of rows t/8 + 16j
    const int c = t & 7;
#pragma unroll 2
    for (int j = 0; j < 8; ++j) {
      const int r = (t >> 3) + 16 * j;
      const int64_t gr = row0 + r;
      uint32_t h[4], l[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int64_t gk = k0 + 4 * c + i;
        double v = (gr < nrows && gk < kend) ? __ldg(P + gk + gr * ld) : 0.0;
        h[i] = to_tf32(float(v));
        l[i] = to_tf32(float(v - double(__uint_as_float(h[i]))));
      }
      const uint32_t off = sw128(r, c);
      *reinterpret_cast<uint4*>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
  }
}

__global__ void __launch_bounds__(NTHREADS, 1) gemm_tf32x3_kernel(Args a) {
  extern __shared__ unsigned char smem_raw[];
  char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  // bars[0..S-1] full, bars[S..2S-1] empty, bars[2S] accumulator ready
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 1);
  int* s_err = reinterpret_cast<int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t m0 = int64_t(blockIdx.x) * BM, n0 = int64_t(blockIdx.y) * BN;
  const int64_t kb = int64_t(blockIdx.z) * a.kchunk;
  const int64_t ke = min(a.K, kb + a.kchunk);
  const int nkb = int((ke - kb + BK - 1) / BK);

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(smem_u32(&bars[s]), 4);              // one arrive per producer warp
      mbar_init(smem_u32(&bars[STAGES + s]), 1);     // tcgen05.commit
    }
    mbar_init(smem_u32(&bars[2 * STAGES]), 1);
    *s_err = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 4) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const bool a_rowc = (a.opA == 0);  // A(m,k) = A[m + k*lda]
  const bool b_rowc = (a.opB == 1);  // B(k,n) = B[n + k*ldb] -> rows (n) contiguous

  if (warp < 4) {
    // ------------------------------------------------------------ producers
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      const uint32_t ph = uint32_t(i / STAGES) & 1u;
      if (!mbar_wait(smem_u32(&bars[STAGES + s]), ph ^ 1u)) {
        atomicOr(s_err, 1);
        break;
      }
      char* st = smem + s * STAGE_BYTES;
      const int64_t k0 = kb + int64_t(i) * BK;
      load_split(a.A, a.lda, a_rowc, m0, a.M, k0, ke, st, st + TILE_BYTES, tid);
      load_split(a.B, a.ldb, b_rowc, n0, a.N, k0, ke, st + 2 * TILE_BYTES, st + 3 * TILE_BYTES, tid);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&bars[s]));
    }
  } else if (lane == 0) {
    // ------------------------------------------------------------ MMA issue
    const uint32_t sbase = smem_u32(smem);
    bool ok = true;
    for (int i = 0; i < nkb && ok; ++i) {
      const int s = i % STAGES;
      const uint32_t ph = uint32_t(i / STAGES) & 1u;
      if (!mbar_wait(smem_u32(&bars[s]), ph)) {
        atomicOr(s_err, 2);
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t st = sbase + s * STAGE_BYTES;
      const uint64_t dah = make_desc(st), dal = make_desc(st + TILE_BYTES);
      const uint64_t dbh = make_desc(st + 2 * TILE_BYTES), dbl = make_desc(st + 3 * TILE_BYTES);
#pragma unroll
      for (int kk = 0; kk < BK / 8; ++kk) {
        const uint64_t adv = uint64_t(kk * 2);  // 8 TF32 = 32 B = 2 x 16 B inside the swizzle atom
        mma_tf32(tmem, dal + adv, dbh + adv, (i > 0 || kk > 0) ? 1u : 0u);
        mma_tf32(tmem, dah + adv, dbl + adv, 1u);
        mma_tf32(tmem, dah + adv, dbh + adv, 1u);
      }
      mma_commit(smem_u32(&bars[STAGES + s]));  // stage s free once these MMAs have read it
    }
    mma_commit(smem_u32(&bars[2 * STAGES]));    // accumulator complete (all prior MMAs)
  }

  // ---------------------------------------------------------------- epilogue
  if (warp < 4) {
    const bool ready = mbar_wait(smem_u32(&bars[2 * STAGES]), 0u);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int64_t row = m0 + warp * 32 + lane;
    const bool bad = !ready || (*s_err != 0);
    for (int c0 = 0; c0 < BN; c0 += 32) {
      uint32_t v[32];
      const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
          "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
          "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
            "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
            "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
            "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (bad || row >= a.M) continue;
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int64_t col = n0 + c0 + j;
        if (col >= a.N) break;
        const double acc = double(__uint_as_float(v[j]));
        if (a.partial) {
          a.partial[int64_t(blockIdx.z) * a.M * a.N + row + col * a.M] = acc;
        } else {
          double* cp = a.C + row + col * a.ldc;
          *cp = (a.beta != 0.0) ? fma(a.alpha, acc, a.beta * *cp) : a.alpha * acc;
        }
      }
    }
    if (bad && warp == 0 && lane == 0) atomicOr(a.status, 8);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 4) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

__global__ void splitk_reduce_f64(int64_t M, int64_t N, int S, const double* __restrict__ partial, double alpha,
                                  double beta, double* __restrict__ C, int64_t ldc) {
  int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= M * N) return;
  int64_t gm = idx % M, gn = idx / M;
  double s = partial[idx];
  for (int z = 1; z < S; ++z) s += partial[int64_t(z) * M * N + idx];
  double* cp = C + gm + gn * ldc;
  *cp = (beta != 0.0) ? fma(alpha, s, beta * *cp) : alpha * s;
}

std::atomic<bool> g_attr_set{false};

}  // namespace

void gemm_tf32x3(Ctx& c, char opA, char opB, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
                 int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc) {
  if (m <= 0 || n <= 0) return;
  IPEPS_CHECK(k > 0, "gemm_tf32x3: k == 0");
  IPEPS_CHECK((opA == 'N' || opA == 'T') && (opB == 'N' || opB == 'T'), "gemm_tf32x3: op must be N or T");
  if (!g_attr_set) {
    IPEPS_CUDA(cudaFuncSetAttribute(gemm_tf32x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
    g_attr_set = true;
  }
  const int64_t gx = (m + BM - 1) / BM, gy = (n + BN - 1) / BN;
  IPEPS_CHECK(gy <= 65535, "gemm_tf32x3: n too large for grid");
  const int64_t tiles = gx * gy;
  int S = 1;
  if (tiles < c.sm_count && k >= 4 * BK) {
    int64_t want = (c.sm_count + tiles - 1) / tiles;
    int64_t maxs = k / (4 * BK);
    S = int(std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(want, maxs), 32)));
  }
  int64_t kchunk = (k + S - 1) / S;
  kchunk = ((kchunk + BK - 1) / BK) * BK;
  S = int((k + kchunk - 1) / kchunk);
  Args a{};
  a.M = m;
  a.N = n;
  a.K = k;
  a.kchunk = kchunk;
  a.opA = (opA == 'T');
  a.opB = (opB == 'T');
  a.A = A;
  a.lda = lda;
  a.B = B;
  a.ldb = ldb;
  a.alpha = alpha;
  a.beta = beta;
  a.C = C;
  a.ldc = ldc;
  a.partial = (S > 1) ? static_cast<double*>(c.workspace(size_t(S) * m * n * sizeof(double))) : nullptr;
  a.status = c.d_status;
  ProfScope ps(c, KFam::GemmTF32x3);
  dim3 grid{unsigned(gx), unsigned(gy), unsigned(S)};
  gemm_tf32x3_kernel<<<grid, NTHREADS, SMEM_BYTES, c.stream>>>(a);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::GemmTF32x3, 2.0 * double(m) * double(n) * double(k));
  if (S > 1) {
    const int64_t tot = m * n;
    splitk_reduce_f64<<<unsigned((tot + 255) / 256), 256, 0, c.stream>>>(m, n, S, a.partial, alpha, beta, C, ldc);
    IPEPS_LAUNCH_CHECK();
    c.count(KFam::Reduce, 0, double(S + 2) * tot * 8);
  }
}

}  // namespace ipeps
