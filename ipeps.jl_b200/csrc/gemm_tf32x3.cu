// 3xTF32 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// C = alpha*op(A)*op(B) + beta*C with FP64 operands (column-major, op in
// {N, T}).  Each FP64 value a is split once into
//   a_hi = tf32(a),  a_lo = tf32(a - a_hi)
// (split_kmajor: one HBM pass that also transposes to the K-major layout the
// UMMA descriptors read), and the product is accumulated in FP32 in tensor
// memory as a_lo*b_hi + a_hi*b_lo + a_hi*b_hi (~22 mantissa bits per
// product, FP32-equivalent accuracy).  Split-K partial sums are added in FP64.
//
// Operand planes: rows x Kp FP32, K contiguous, Kp = K rounded up to 32 (zero
// padded), the lo plane stacked under the hi plane (rows..2*rows-1).  One
// 2-D TMA tensor map per operand loads 128-byte-swizzled boxes of 32 K x
// {128 | BN} rows straight into the SW128 K-major layout of the UMMA shared
// memory descriptors.  Rows past the end of an operand only feed rows or
// columns of C outside the result, which the epilogue never stores.
//
// Kernel: persistent, one CTA per SM, warp-specialised.
//   warp 0   TMA producer (one lane): stage ring of STAGES x {A_hi, A_lo, B_hi, B_lo}
//   warp 1   TMEM allocation (512 or 256 columns) and the MMA issue (one lane):
//            12 tcgen05.mma (kind::tf32, M=128, N=BN, K=8) per 32-wide K block
//   warps 2-5 epilogue: tcgen05.ld of the accumulator (warp w reads TMEM lanes
//            32*(w%4)..+31), FP64 alpha/beta scaling and coalesced stores
//            (or FP32 split-K partials)
// Two accumulator buffers in TMEM let the epilogue of one work unit overlap
// the main loop of the next.  A work unit is (M tile, N tile, K split).
// Every mbarrier wait is bounded: on a timeout the kernel records bit 8 in
// the status word, every role leaves its loop, the producer waits (bounded)
// for its own copies in flight, the MMA thread for its own MMAs, and TMEM is
// freed.
#include "umma.cuh"

#include <cuda.h>

#include <algorithm>
#include <mutex>

namespace ipeps {
namespace {

constexpr int BM = 128, BK = 32;
constexpr int A_TILE = BM * BK * 4;      // 16 KB per plane
constexpr int NTHREADS = 192;            // 6 warps
constexpr int SMEM_BUDGET = 227 * 1024;  // opt-in maximum per CTA
constexpr int MAX_STAGES = 8;

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// ------------------------------------------------------------------ split
// P_hi[r*Kp + k] and P_lo[(rows + r)*Kp + k] from X(r, k); k in [K, Kp) is 0.
// k contiguous: X(r, k) = X[k + r*ld]; each thread converts 4 consecutive k
__global__ void split_kc_kernel(const double* __restrict__ X, int64_t ld, int64_t rows, int64_t K, int64_t Kp,
                                float* __restrict__ P) {
  const int64_t q = Kp / 4;
  const int64_t n = rows * q;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = i / q, k0 = (i - r * q) * 4;
    uint32_t h[4], l[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const double v = (k0 + j < K) ? __ldg(X + r * ld + k0 + j) : 0.0;
      h[j] = to_tf32(float(v));
      l[j] = to_tf32(float(v - double(__uint_as_float(h[j]))));
    }
    *reinterpret_cast<uint4*>(P + r * Kp + k0) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(P + (rows + r) * Kp + k0) = make_uint4(l[0], l[1], l[2], l[3]);
  }
}

// rows contiguous: X(r, k) = X[r + k*ld]; 32 x 32 tiles through shared memory
__global__ void split_tr_kernel(const double* __restrict__ X, int64_t ld, int64_t rows, int64_t K, int64_t Kp,
                                float* __restrict__ P) {
  __shared__ double t[32][33];
  const int64_t r0 = int64_t(blockIdx.x) * 32, k0 = int64_t(blockIdx.y) * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
#pragma unroll
  for (int j = 0; j < 32; j += 8) {
    const int64_t r = r0 + tx, k = k0 + ty + j;
    t[ty + j][tx] = (r < rows && k < K) ? __ldg(X + r + k * ld) : 0.0;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 32; j += 8) {
    const int64_t r = r0 + ty + j, k = k0 + tx;
    if (r < rows && k < Kp) {
      const double v = t[tx][ty + j];
      const uint32_t h = to_tf32(float(v));
      const uint32_t l = to_tf32(float(v - double(__uint_as_float(h))));
      P[r * Kp + k] = __uint_as_float(h);
      P[(rows + r) * Kp + k] = __uint_as_float(l);
    }
  }
}

// ------------------------------------------------------------------ GEMM
struct Args {
  int M, N, BN, stages;
  int tiles_m, tiles_n, splits, nkb, kb_per_split;
  int units;
  double alpha, beta;
  double* C;
  int64_t ldc;
  float* partial;  // splits > 1: [split] column-major M x N FP32 partial sums
  int* status;
};

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(NTHREADS, 1)
    tf32x3_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, Args a) {
  extern __shared__ unsigned char smem_raw[];
  char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int BN = a.BN, S = a.stages;
  const int b_tile = BN * BK * 4;
  const int stage_bytes = 2 * A_TILE + 2 * b_tile;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S * stage_bytes);
  // bars: full[S], empty[S], acc_full[2], acc_empty[2], drain
  uint64_t* full = bars;
  uint64_t* empty = bars + S;
  uint64_t* acc_full = bars + 2 * S;
  uint64_t* acc_empty = bars + 2 * S + 2;
  uint64_t* drain = bars + 2 * S + 4;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 5);
  volatile int* s_err = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const uint32_t tmem_cols = (2 * BN > 256) ? 512u : 256u;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&acc_full[b]), 1);
      mbar_init(smem_u32(&acc_empty[b]), 4);
    }
    mbar_init(smem_u32(drain), 1);
    *s_err = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapA)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapB)) : "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  // unit u -> (tile_m, tile_n, split): M tiles fastest, then splits, then N tiles
  auto unit_coords = [&](int u, int& tm, int& tn, int& sp) {
    tm = u % a.tiles_m;
    const int r = u / a.tiles_m;
    sp = r % a.splits;
    tn = r / a.splits;
  };

  if (warp == 0) {
    if (lane == 0) {
      // ------------------------------------------------------------ producer
      int it = 0;
      int last_phase[MAX_STAGES];
      for (int s = 0; s < MAX_STAGES; ++s) last_phase[s] = -1;
      for (int u = blockIdx.x; u < a.units && !*s_err; u += gridDim.x) {
        int tm, tn, sp;
        unit_coords(u, tm, tn, sp);
        const int kb0 = sp * a.kb_per_split, kb1 = min(a.nkb, kb0 + a.kb_per_split);
        bool ok = true;
        for (int kb = kb0; kb < kb1; ++kb, ++it) {
          const int s = it % S;
          const uint32_t ph = uint32_t(it / S) & 1u;
          if (!mbar_wait(smem_u32(&empty[s]), ph ^ 1u)) {
            *s_err = 1;
            ok = false;
            break;
          }
          const uint32_t st = smem_u32(smem + s * stage_bytes);
          const uint32_t fb = smem_u32(&full[s]);
          mbar_expect_tx(fb, uint32_t(stage_bytes));
          const int x = kb * BK;
          tma_load_2d(st, &mapA, x, tm * BM, fb);
          tma_load_2d(st + A_TILE, &mapA, x, a.M + tm * BM, fb);
          tma_load_2d(st + 2 * A_TILE, &mapB, x, tn * BN, fb);
          tma_load_2d(st + 2 * A_TILE + b_tile, &mapB, x, a.N + tn * BN, fb);
          last_phase[s] = int(ph);
        }
        if (!ok) break;
      }
      // the CTA may exit only after its own copies have landed
      for (int s = 0; s < S; ++s)
        if (last_phase[s] >= 0 && !mbar_wait(smem_u32(&full[s]), uint32_t(last_phase[s]))) *s_err = 1;
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ------------------------------------------------------------ MMA issue
      const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(BN >> 3) << 17) |
                             (uint32_t(BM >> 4) << 24);
      const uint32_t sbase = smem_u32(smem);
      int it = 0, t = 0;
      for (int u = blockIdx.x; u < a.units && !*s_err; u += gridDim.x, ++t) {
        int tm, tn, sp;
        unit_coords(u, tm, tn, sp);
        const int kb0 = sp * a.kb_per_split, kb1 = min(a.nkb, kb0 + a.kb_per_split);
        const int b = t & 1;
        const uint32_t aph = uint32_t(t >> 1) & 1u;
        if (!mbar_wait(smem_u32(&acc_empty[b]), aph ^ 1u)) {
          *s_err = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t dacc = tmem + uint32_t(b * BN);
        bool ok = true;
        for (int kb = kb0; kb < kb1; ++kb, ++it) {
          const int s = it % S;
          const uint32_t ph = uint32_t(it / S) & 1u;
          if (!mbar_wait(smem_u32(&full[s]), ph)) {
            *s_err = 1;
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t st = sbase + s * stage_bytes;
          const uint64_t dah = make_desc(st), dal = make_desc(st + A_TILE);
          const uint64_t dbh = make_desc(st + 2 * A_TILE), dbl = make_desc(st + 2 * A_TILE + b_tile);
#pragma unroll
          for (int kk = 0; kk < BK / 8; ++kk) {
            const uint64_t adv = uint64_t(kk * 2);  // 8 TF32 = 32 B = 2 x 16 B inside the swizzle atom
            mma_tf32(dacc, dal + adv, dbh + adv, idesc, (kb > kb0 || kk > 0) ? 1u : 0u);
            mma_tf32(dacc, dah + adv, dbl + adv, idesc, 1u);
            mma_tf32(dacc, dah + adv, dbh + adv, idesc, 1u);
          }
          mma_commit(smem_u32(&empty[s]));  // stage s free once these MMAs have read it
        }
        if (!ok) break;
        mma_commit(smem_u32(&acc_full[b]));  // accumulator b complete
      }
      // every MMA this thread issued has completed before TMEM can be freed
      mma_commit(smem_u32(drain));
      if (!mbar_wait(smem_u32(drain), 0u)) *s_err = 1;
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3;  // TMEM lane quadrant this warp may access
    int t = 0;
    for (int u = blockIdx.x; u < a.units; u += gridDim.x, ++t) {
      // warp-uniform control flow: tcgen05.ld is .sync.aligned
      if (__shfl_sync(0xffffffffu, *s_err, 0)) break;
      int tm, tn, sp;
      unit_coords(u, tm, tn, sp);
      const int b = t & 1;
      const uint32_t aph = uint32_t(t >> 1) & 1u;
      if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(&acc_full[b]), aph))) {
        *s_err = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int row = tm * BM + q * 32 + lane;
      const bool rok = row < a.M;
      for (int c0 = 0; c0 < BN; c0 += 32) {
        uint32_t v[32];
        tmem_ld32(tmem + (uint32_t(q * 32) << 16) + uint32_t(b * BN + c0), v);
        if (c0 + 32 >= BN) {
          // the accumulator buffer may be reused once every load of it has completed
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) mbar_arrive(smem_u32(&acc_empty[b]));
        }
        if (!rok) continue;
        const int col0 = tn * BN + c0;
        if (a.partial) {
          float* p = a.partial + int64_t(sp) * a.M * a.N + row;
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (col0 + j < a.N) p[int64_t(col0 + j) * a.M] = __uint_as_float(v[j]);
        } else {
          double* cp = a.C + row;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            if (col0 + j < a.N) {
              double* d = cp + int64_t(col0 + j) * a.ldc;
              const double acc = double(__uint_as_float(v[j]));
              *d = (a.beta != 0.0) ? fma(a.alpha, acc, a.beta * *d) : a.alpha * acc;
            }
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (threadIdx.x == 0 && *s_err) atomicOr(a.status, 8);
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols) : "memory");
  }
}

// C = alpha * sum_z partial[z] + beta * C, FP64 sums of the FP32 partials
__global__ void splitk_reduce_kernel(int M, int N, int S, const float* __restrict__ partial, double alpha,
                                     double beta, double* __restrict__ C, int64_t ldc) {
  const int64_t tot = int64_t(M) * N;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < tot; i += int64_t(gridDim.x) * blockDim.x) {
    double s = 0;
    for (int z = 0; z < S; ++z) s += double(partial[int64_t(z) * tot + i]);
    const int64_t m = i % M, n = i / M;
    double* cp = C + m + n * ldc;
    *cp = (beta != 0.0) ? fma(alpha, s, beta * *cp) : alpha * s;
  }
}

// ------------------------------------------------------------------ host
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static std::once_flag once;
  static EncodeTiled fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  IPEPS_CHECK(fn != nullptr, "gemm_tf32x3: cuTensorMapEncodeTiled unavailable");
  return fn;
}

// 2-D map over the stacked hi/lo planes: inner extent Kp (FP32), 2*rows rows
CUtensorMap plane_map(const Planes& p, int box_rows) {
  CUtensorMap m;
  const cuuint64_t dims[2] = {cuuint64_t(p.Kp), cuuint64_t(2 * p.rows)};
  const cuuint64_t strides[1] = {cuuint64_t(p.Kp) * 4};
  const cuuint32_t box[2] = {cuuint32_t(BK), cuuint32_t(box_rows)};
  const cuuint32_t es[2] = {1, 1};
  CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, p.buf.data(), dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  IPEPS_CHECK(r == CUDA_SUCCESS, "gemm_tf32x3: cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
  return m;
}

SmemAttrOnce g_attr;

// N tile: one tile of round_up(n, 32) up to 256, else the width in
// {256, 224, 192, 160, 128} with the least padding
int pick_bn(int64_t n) {
  if (n <= 256) return int((n + 31) / 32) * 32;
  int best = 256;
  int64_t best_pad = ((n + 255) / 256) * 256;
  for (int bn : {224, 192, 160, 128}) {
    const int64_t pad = ((n + bn - 1) / bn) * bn;
    if (pad < best_pad) {
      best = bn;
      best_pad = pad;
    }
  }
  return best;
}

}  // namespace

Planes split_kmajor(Ctx& c, const double* X, int64_t ld, bool kcontig, int64_t rows, int64_t K) {
  IPEPS_CHECK(rows > 0 && K > 0, "split_kmajor: empty operand");
  IPEPS_CHECK(2 * rows < (int64_t(1) << 31), "split_kmajor: too many rows for a TMA coordinate");
  Planes p;
  p.rows = rows;
  p.K = K;
  p.Kp = ((K + BK - 1) / BK) * BK;
  p.buf = c.alloc(DType::F64, {rows * p.Kp});  // 2 * rows * Kp FP32
  float* P = reinterpret_cast<float*>(p.buf.data());
  ProfScope ps(c, KFam::Permute);
  if (kcontig) {
    const int64_t n = rows * (p.Kp / 4);
    const int grid = int(std::min<int64_t>((n + 255) / 256, int64_t(c.sm_count) * 16));
    split_kc_kernel<<<grid, 256, 0, c.stream>>>(X, ld, rows, K, p.Kp, P);
  } else {
    IPEPS_CHECK(p.Kp / 32 <= 65535, "split_kmajor: K too large for the grid");
    dim3 grid{unsigned((rows + 31) / 32), unsigned(p.Kp / 32)};
    split_tr_kernel<<<grid, dim3{32, 8}, 0, c.stream>>>(X, ld, rows, K, p.Kp, P);
  }
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Permute, 0, double(rows) * K * 8 + double(rows) * p.Kp * 8);
  return p;
}

void gemm_tf32x3_planes(Ctx& c, const Planes& PA, const Planes& PB, int64_t m, int64_t n, int64_t k, double alpha,
                        double beta, double* C, int64_t ldc) {
  if (m <= 0 || n <= 0) return;
  IPEPS_CHECK(PA.rows == m && PB.rows == n && PA.K == k && PB.K == k && PA.Kp == PB.Kp,
              "gemm_tf32x3: operand planes do not match the product shape");
  IPEPS_CHECK(m < (int64_t(1) << 30) && n < (int64_t(1) << 30), "gemm_tf32x3: dimension too large");
  const int BN = pick_bn(n);
  const int b_tile = BN * BK * 4;
  const int stage_bytes = 2 * A_TILE + 2 * b_tile;
  const int stages = std::min(MAX_STAGES, (SMEM_BUDGET - 1024 - 256) / stage_bytes);
  IPEPS_CHECK(stages >= 2, "gemm_tf32x3: tile does not fit in shared memory");
  const int smem = 1024 + stages * stage_bytes + 256;
  // the attribute is set once per device, so to the largest size any tile width uses
  g_attr.ensure(tf32x3_kernel, SMEM_BUDGET);

  Args a{};
  a.M = int(m);
  a.N = int(n);
  a.BN = BN;
  a.stages = stages;
  a.tiles_m = int((m + BM - 1) / BM);
  a.tiles_n = int((n + BN - 1) / BN);
  a.nkb = int(PA.Kp / BK);
  const int tiles = a.tiles_m * a.tiles_n;
  // split K when the tiles alone leave SMs idle (at least 4 K blocks per split)
  int S = 1;
  if (tiles < c.sm_count && a.nkb >= 8) S = std::max(1, std::min({(c.sm_count + tiles - 1) / tiles, a.nkb / 4, 16}));
  a.kb_per_split = (a.nkb + S - 1) / S;
  S = (a.nkb + a.kb_per_split - 1) / a.kb_per_split;
  a.splits = S;
  a.units = tiles * S;
  a.alpha = alpha;
  a.beta = beta;
  a.C = C;
  a.ldc = ldc;
  a.partial = (S > 1) ? static_cast<float*>(c.workspace(size_t(S) * m * n * sizeof(float))) : nullptr;
  a.status = c.d_status;
  const CUtensorMap mA = plane_map(PA, BM), mB = plane_map(PB, BN);
  const int grid = std::min(a.units, c.sm_count);
  ProfScope ps(c, KFam::GemmTF32x3);
  tf32x3_kernel<<<grid, NTHREADS, smem, c.stream>>>(mA, mB, a);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::GemmTF32x3, 2.0 * double(m) * double(n) * double(k));
  if (S > 1) {
    const int64_t tot = m * n;
    const int rg = int(std::min<int64_t>((tot + 255) / 256, int64_t(c.sm_count) * 8));
    splitk_reduce_kernel<<<rg, 256, 0, c.stream>>>(int(m), int(n), S, a.partial, alpha, beta, C, ldc);
    IPEPS_LAUNCH_CHECK();
    c.count(KFam::Reduce, 0, double(S) * tot * 4 + double(beta != 0.0 ? 2 : 1) * tot * 8);
  }
}

// A(m, k) = op(A): op N -> A[m + k*lda] (rows contiguous), op T -> A[k + m*lda];
// B(k, n) = op(B): op N -> B[k + n*ldb] (k contiguous),    op T -> B[n + k*ldb]
void gemm_tf32x3(Ctx& c, char opA, char opB, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
                 int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc) {
  if (m <= 0 || n <= 0) return;
  IPEPS_CHECK(k > 0, "gemm_tf32x3: k == 0");
  IPEPS_CHECK((opA == 'N' || opA == 'T') && (opB == 'N' || opB == 'T'), "gemm_tf32x3: op must be N or T");
  const Planes PA = split_kmajor(c, A, lda, opA == 'T', m, k);
  const Planes PB = split_kmajor(c, B, ldb, opB == 'N', n, k);
  gemm_tf32x3_planes(c, PA, PB, m, n, k, alpha, beta, C, ldc);
}

}  // namespace ipeps
