// BF16 GEMM on the 5th-generation tensor cores (tcgen05.mma kind::f16, sm_100a)
// for the warm-start network: C = alpha*op(A)*op(B) + beta*C with FP32
// operands and result in global memory (column-major, op in {N, T}); the
// operands are rounded to BF16 while they are staged, the products accumulate
// in FP32 in tensor memory.
//
// CTA tile 128 x 128, K-step 64 (one 128-byte swizzled row of BF16), 4-stage
// shared-memory ring.  Warp roles as in the 3xTF32 kernel: warps 0-3 load,
// convert and store the swizzled K-major tiles, then run the epilogue
// (tcgen05.ld of their 32 TMEM lanes); warp 4 allocates TMEM and one of its
// threads issues the MMAs.  Every mbarrier wait is bounded; on timeout the
// kernel records bit 8 in the status word and drains.
#include "umma.cuh"

#include <atomic>

#include <algorithm>

namespace ipeps {
namespace {

constexpr int BM = 128, BN = 128, BK = 64, STAGES = 4;
constexpr int TILE_BYTES = BM * BK * 2;      // 16 KB per operand tile
constexpr int STAGE_BYTES = 2 * TILE_BYTES;  // A, B
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
constexpr int NTHREADS = 160;
constexpr uint32_t TMEM_COLS = 128;

// instruction descriptor: D = F32, A = B = BF16, both K-major, M = 128, N = 128
constexpr uint32_t IDESC_BF16 = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(BN >> 3) << 17) |
                                (uint32_t(BM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem), "l"(da), "l"(db), "r"(IDESC_BF16), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

// two FP32 values -> packed BF16 pair (first value in the low half: the lower address)
__device__ __forceinline__ uint32_t pack_bf16(float first, float second) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(second), "f"(first));
  return r;
}

struct ArgsB {
  int64_t M, N, K;
  int opA, opB;  // 0 = N, 1 = T
  const float* A;
  int64_t lda;
  const float* B;
  int64_t ldb;
  float alpha, beta;
  float* C;
  int64_t ldc;
  int* status;
};

// Load the 128 x 64 logical tile X(row, k) into one BF16 swizzled tile.
// rowc: X(row,k) = P[row + k*ld]; otherwise X(row,k) = P[k + row*ld].
__device__ __forceinline__ void load_bf16(const float* __restrict__ P, int64_t ld, bool rowc, int64_t row0,
                                          int64_t nrows, int64_t k0, int64_t kend, char* tile, int t) {
  if (rowc) {
    const int r = t;  // thread t owns row t: 8 chunks of 8 k
    const int64_t gr = row0 + r;
#pragma unroll 2
    for (int c = 0; c < 8; ++c) {
      float v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int64_t gk = k0 + 8 * c + i;
        v[i] = (gr < nrows && gk < kend) ? __ldg(P + gr + gk * ld) : 0.0f;
      }
      *reinterpret_cast<uint4*>(tile + sw128(r, c)) =
          make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
    }
  } else {
    const int c = t & 7;  // thread t owns chunk t%8 of rows t/8 + 16j
#pragma unroll 2
    for (int j = 0; j < 8; ++j) {
      const int r = (t >> 3) + 16 * j;
      const int64_t gr = row0 + r;
      float v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int64_t gk = k0 + 8 * c + i;
        v[i] = (gr < nrows && gk < kend) ? __ldg(P + gk + gr * ld) : 0.0f;
      }
      *reinterpret_cast<uint4*>(tile + sw128(r, c)) =
          make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
    }
  }
}

__global__ void __launch_bounds__(NTHREADS, 1) gemm_bf16_kernel(ArgsB a) {
  extern __shared__ unsigned char smem_raw[];
  char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 1);
  int* s_err = reinterpret_cast<int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t m0 = int64_t(blockIdx.x) * BM, n0 = int64_t(blockIdx.y) * BN;
  const int nkb = int((a.K + BK - 1) / BK);

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(smem_u32(&bars[s]), 4);           // one arrive per producer warp
      mbar_init(smem_u32(&bars[STAGES + s]), 1);  // tcgen05.commit
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
  const bool b_rowc = (a.opB == 1);  // B(k,n) = B[n + k*ldb]

  if (warp < 4) {
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      const uint32_t ph = uint32_t(i / STAGES) & 1u;
      if (!mbar_wait(smem_u32(&bars[STAGES + s]), ph ^ 1u)) {
        atomicOr(s_err, 1);
        break;
      }
      char* st = smem + s * STAGE_BYTES;
      const int64_t k0 = int64_t(i) * BK;
      load_bf16(a.A, a.lda, a_rowc, m0, a.M, k0, a.K, st, tid);
      load_bf16(a.B, a.ldb, b_rowc, n0, a.N, k0, a.K, st + TILE_BYTES, tid);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&bars[s]));
    }
  } else if (lane == 0) {
    const uint32_t sbase = smem_u32(smem);
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      const uint32_t ph = uint32_t(i / STAGES) & 1u;
      if (!mbar_wait(smem_u32(&bars[s]), ph)) {
        atomicOr(s_err, 2);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t st = sbase + s * STAGE_BYTES;
      const uint64_t da = make_desc(st), db = make_desc(st + TILE_BYTES);
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) {
        const uint64_t adv = uint64_t(kk * 2);  // 16 BF16 = 32 B = 2 x 16 B inside the swizzle atom
        mma_bf16(tmem, da + adv, db + adv, (i > 0 || kk > 0) ? 1u : 0u);
      }
      mma_commit(smem_u32(&bars[STAGES + s]));
    }
    mma_commit(smem_u32(&bars[2 * STAGES]));
  }

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
        float* cp = a.C + row + col * a.ldc;
        const float acc = __uint_as_float(v[j]);
        *cp = (a.beta != 0.0f) ? fmaf(a.alpha, acc, a.beta * *cp) : a.alpha * acc;
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

SmemAttrOnce g_bf16_attr;

}  // namespace

void gemm_bf16(Ctx& c, char opA, char opB, int64_t m, int64_t n, int64_t k, float alpha, const float* A, int64_t lda,
               const float* B, int64_t ldb, float beta, float* C, int64_t ldc) {
  if (m <= 0 || n <= 0) return;
  IPEPS_CHECK(k > 0, "gemm_bf16: k == 0");
  IPEPS_CHECK((opA == 'N' || opA == 'T') && (opB == 'N' || opB == 'T'), "gemm_bf16: op must be N or T");
  g_bf16_attr.ensure(gemm_bf16_kernel, SMEM_BYTES);
  const int64_t gx = (m + BM - 1) / BM, gy = (n + BN - 1) / BN;
  IPEPS_CHECK(gy <= 65535, "gemm_bf16: n too large for grid");
  ArgsB a{};
  a.M = m;
  a.N = n;
  a.K = k;
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
  a.status = c.d_status;
  ProfScope ps(c, KFam::GemmTF32x3);
  gemm_bf16_kernel<<<dim3{unsigned(gx), unsigned(gy), 1u}, NTHREADS, SMEM_BYTES, c.stream>>>(a);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::GemmTF32x3, 2.0 * double(m) * double(n) * double(k));
}

}  // namespace ipeps
