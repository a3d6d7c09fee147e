// Complex128 GEMM for sm_100a (and the real FP64 kernel of the allocation-free
// entry point): register-tiled SIMT FMA kernel.  Real FP64 products of the
// engine go to the DMMA kernel (gemm_dmma.cu).  Tiles:
//   real     64x64x16, 4x4 outputs per thread (allocation-free entry point)
//   complex  64x64x8,  4x4 outputs per thread
// Operands are staged through shared memory with one register prefetch stage.
// Skinny problems (few output tiles, long K) use a deterministic split-K:
// partial products go to a workspace and are summed in a fixed order.
#include "ctx.cuh"

#include <algorithm>

namespace ipeps {
namespace {

__device__ __forceinline__ double cj(double x) { return x; }
__device__ __forceinline__ cuDoubleComplex cj(cuDoubleComplex x) { return cuConj(x); }
__device__ __forceinline__ void fma_acc(double& acc, double a, double b) { acc = fma(a, b, acc); }
__device__ __forceinline__ void fma_acc(cuDoubleComplex& acc, cuDoubleComplex a, cuDoubleComplex b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
template <typename T> __device__ __forceinline__ T zero();
template <> __device__ __forceinline__ double zero<double>() { return 0.0; }
template <> __device__ __forceinline__ cuDoubleComplex zero<cuDoubleComplex>() {
  return make_cuDoubleComplex(0, 0);
}
__device__ __forceinline__ double mulS(double a, cuDoubleComplex s) { return a * s.x; }
__device__ __forceinline__ cuDoubleComplex mulS(cuDoubleComplex a, cuDoubleComplex s) {
  return cuCmul(a, s);
}
__device__ __forceinline__ double addv(double a, double b) { return a + b; }
__device__ __forceinline__ cuDoubleComplex addv(cuDoubleComplex a, cuDoubleComplex b) {
  return cuCadd(a, b);
}
__device__ __forceinline__ bool is_zero(cuDoubleComplex s) { return s.x == 0.0 && s.y == 0.0; }

// op codes: 0 = N, 1 = T, 2 = C (conjugate transpose)
template <typename T, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
    gemm_kernel(int opA, int opB, int64_t M, int64_t N, int64_t K, int64_t kchunk,
                cuDoubleComplex alpha, const T* __restrict__ A, int64_t lda,
                const T* __restrict__ B, int64_t ldb, cuDoubleComplex beta, T* __restrict__ C,
                int64_t ldc, T* __restrict__ partial) {
  constexpr int NT = (BM / TM) * (BN / TN);
  constexpr int TX = BM / TM;  // threads along m
  constexpr int A_PER = BM * BK / NT;
  constexpr int B_PER = BN * BK / NT;
  static_assert(A_PER >= 1 && B_PER >= 1, "tile too small");
  __shared__ T As[2][BK][BM + 1];
  __shared__ T Bs[2][BK][BN + 1];

  const int tid = threadIdx.x;
  const int tx = tid % TX, ty = tid / TX;
  const int64_t m0 = int64_t(blockIdx.x) * BM;
  const int64_t n0 = int64_t(blockIdx.y) * BN;
  const int64_t kb = int64_t(blockIdx.z) * kchunk;
  const int64_t ke = min(K, kb + kchunk);

  T acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = zero<T>();

  T ra[A_PER], rb[B_PER];

  auto load_a = [&](int64_t k0) {
#pragma unroll
    for (int r = 0; r < A_PER; ++r) {
      int e = tid + r * NT;
      int mi, ki;
      if (opA == 0) { mi = e % BM; ki = e / BM; }
      else { ki = e % BK; mi = e / BK; }
      int64_t gm = m0 + mi, gk = k0 + ki;
      T v = zero<T>();
      if (gm < M && gk < ke) {
        v = (opA == 0) ? A[gm + gk * lda] : A[gk + gm * lda];
        if (opA == 2) v = cj(v);
      }
      ra[r] = v;
    }
  };
  auto load_b = [&](int64_t k0) {
#pragma unroll
    for (int r = 0; r < B_PER; ++r) {
      int e = tid + r * NT;
      int ni, ki;
      if (opB == 0) { ki = e % BK; ni = e / BK; }
      else { ni = e % BN; ki = e / BN; }
      int64_t gn = n0 + ni, gk = k0 + ki;
      T v = zero<T>();
      if (gn < N && gk < ke) {
        v = (opB == 0) ? B[gk + gn * ldb] : B[gn + gk * ldb];
        if (opB == 2) v = cj(v);
      }
      rb[r] = v;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int r = 0; r < A_PER; ++r) {
      int e = tid + r * NT;
      int mi, ki;
      if (opA == 0) { mi = e % BM; ki = e / BM; }
      else { ki = e % BK; mi = e / BK; }
      As[buf][ki][mi] = ra[r];
    }
#pragma unroll
    for (int r = 0; r < B_PER; ++r) {
      int e = tid + r * NT;
      int ni, ki;
      if (opB == 0) { ki = e % BK; ni = e / BK; }
      else { ni = e % BN; ki = e / BN; }
      Bs[buf][ki][ni] = rb[r];
    }
  };

  int buf = 0;
  if (kb < ke) {
    load_a(kb);
    load_b(kb);
    store(0);
  }
  __syncthreads();
  for (int64_t k0 = kb; k0 < ke; k0 += BK) {
    const bool more = k0 + BK < ke;
    if (more) {
      load_a(k0 + BK);
      load_b(k0 + BK);
    }
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      T a[TM], b[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) a[i] = As[buf][kk][tx + i * TX];
#pragma unroll
      for (int j = 0; j < TN; ++j) b[j] = Bs[buf][kk][ty + j * (BN / TN)];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) fma_acc(acc[i][j], a[i], b[j]);
    }
    if (more) {
      store(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }
  }

  // epilogue
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    int64_t gm = m0 + tx + i * TX;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      int64_t gn = n0 + ty + j * (BN / TN);
      if (gn >= N) continue;
      if (partial) {
        partial[int64_t(blockIdx.z) * M * N + gm + gn * M] = acc[i][j];
      } else {
        T v = mulS(acc[i][j], alpha);
        if (!is_zero(beta)) v = addv(v, mulS(C[gm + gn * ldc], beta));
        C[gm + gn * ldc] = v;
      }
    }
  }
}

template <typename T>
__global__ void splitk_reduce(int64_t M, int64_t N, int S, const T* __restrict__ partial,
                              cuDoubleComplex alpha, cuDoubleComplex beta, T* __restrict__ C,
                              int64_t ldc) {
  int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= M * N) return;
  int64_t gm = idx % M, gn = idx / M;
  T s = partial[idx];
  for (int z = 1; z < S; ++z) s = addv(s, partial[int64_t(z) * M * N + idx]);
  T v = mulS(s, alpha);
  if (!is_zero(beta)) v = addv(v, mulS(C[gm + gn * ldc], beta));
  C[gm + gn * ldc] = v;
}

int opcode(char o) {
  switch (o) {
    case 'N': case 'n': return 0;
    case 'T': case 't': return 1;
    case 'C': case 'c': return 2;
  }
  throw Error(kEInval, "gemm: bad op");
}

template <typename T, int BM, int BN, int BK, int TM, int TN>
void launch(Ctx& c, int oa, int ob, int64_t m, int64_t n, int64_t k, cuDoubleComplex alpha,
            const void* A, int64_t lda, const void* B, int64_t ldb, cuDoubleComplex beta, void* C,
            int64_t ldc) {
  constexpr int NT = (BM / TM) * (BN / TN);
  int64_t gx = (m + BM - 1) / BM, gy = (n + BN - 1) / BN;
  IPEPS_CHECK(gy <= 65535, "gemm: n too large for grid");
  int64_t tiles = gx * gy;
  int S = 1;
  // split K when the output grid covers well under two waves and K is long
  const int64_t target = 2LL * c.sm_count;
  if (tiles < target && k >= 8 * BK * 2) {
    int64_t want = (target + tiles - 1) / tiles;
    int64_t maxs = k / (8 * BK);
    S = int(std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(want, maxs), 64)));
  }
  int64_t kchunk = (k + S - 1) / S;
  kchunk = ((kchunk + BK - 1) / BK) * BK;
  S = int((k + kchunk - 1) / kchunk);
  if (S < 1) S = 1;
  ProfScope ps(c, KFam::GemmF64);
  T* partial = nullptr;
  if (S > 1) partial = static_cast<T*>(c.workspace(size_t(S) * m * n * sizeof(T)));
  dim3 grid{unsigned(gx), unsigned(gy), unsigned(S)};
  gemm_kernel<T, BM, BN, BK, TM, TN><<<grid, NT, 0, c.stream>>>(
      oa, ob, m, n, k, kchunk, alpha, static_cast<const T*>(A), lda, static_cast<const T*>(B),
      ldb, beta, static_cast<T*>(C), ldc, partial);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::GemmF64, (sizeof(T) == 8 ? 2.0 : 8.0) * double(m) * double(n) * double(k));
  if (S > 1) {
    int64_t tot = m * n;
    splitk_reduce<T><<<unsigned((tot + 255) / 256), 256, 0, c.stream>>>(
        m, n, S, partial, alpha, beta, static_cast<T*>(C), ldc);
    IPEPS_LAUNCH_CHECK();
    c.count(KFam::Reduce, 0, double(S + 2) * tot * sizeof(T));
  }
}

}  // namespace

void gemm_f64(Ctx& c, DType dt, char opA, char opB, int64_t m, int64_t n, int64_t k,
              cuDoubleComplex alpha, const void* A, int64_t lda, const void* B, int64_t ldb,
              cuDoubleComplex beta, void* C, int64_t ldc) {
  if (m <= 0 || n <= 0) return;
  int oa = opcode(opA), ob = opcode(opB);
  IPEPS_CHECK(k > 0, "gemm: k == 0 is not supported");
  if (dt == DType::F64) {
    IPEPS_CHECK(oa != 2 && ob != 2, "gemm: conjugate op on real data");
    gemm_f64_dmma(c, opA, opB, m, n, k, alpha.x, static_cast<const double*>(A), lda, static_cast<const double*>(B),
                  ldb, beta.x, static_cast<double*>(C), ldc);
  } else {
    launch<cuDoubleComplex, 64, 64, 8, 4, 4>(c, oa, ob, m, n, k, alpha, A, lda, B, ldb, beta, C,
                                             ldc);
  }
}

}  // namespace ipeps

// ---------------------------------------------------------------------------
// Allocation-free variant of the split-K FP64 GEMM.
//
// Some callers cannot call cudaMalloc: a host framework that owns every byte
// of device memory through its own pool (a Julia CUDA.jl session, a plugin
// host with a fixed budget), or a latency-critical section where
// cudaMalloc/cudaFree, which may synchronise the device, are not allowed.
// For them the split-K partial sums live in this fixed device array
// (4 MiB = 524288 doubles; every GPU that loads the library holds it until
// the process exits).  The caller passes device pointers for A, B and C and a
// stream.  The split factor S is capped so that S*m*n partial sums fit in the
// array; an output of more than 262144 elements therefore runs unsplit and
// touches no scratch at all.  Requests the kernel grid cannot cover
// (ceil(n/64) > 65535) are rejected with IPEPS_EINVAL and a message on stderr.
//
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress (with that device current); make that first call
// before any stream capture.  Every call shares the array: calls that overlap
// on the GPU (different streams, or threads without ordering) race on it.
// Each call overwrites all the partial sums it reads, so nothing needs
// clearing between calls.
// ---------------------------------------------------------------------------
#include <mutex>

#include "../../include/ipeps_b200.h"

namespace ipeps {
namespace {

constexpr int64_t kNoAllocScratchDoubles = int64_t(1) << 19;  // 4 MiB of FP64 partial sums
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_splitk_scratch[kNoAllocScratchDoubles];

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device (set-up once per device).
cudaError_t noalloc_scratch(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_splitk_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

}  // namespace
}  // namespace ipeps

extern "C" int ipeps_gemm_f64_noalloc(char opA, char opB, int64_t m, int64_t n, int64_t k, double alpha,
                                      const double* A, int64_t lda, const double* B, int64_t ldb, double beta,
                                      double* C, int64_t ldc, void* stream) {
  using namespace ipeps;
  if (!A || !B || !C || m <= 0 || n <= 0 || k <= 0) return IPEPS_EINVAL;
  int oa, ob;
  try {
    oa = opcode(opA);
    ob = opcode(opB);
  } catch (...) {
    return IPEPS_EINVAL;
  }
  if (oa == 2 || ob == 2) return IPEPS_EINVAL;  // real data: 'C' is not meaningful
  if (lda < ((oa == 0) ? m : k) || ldb < ((ob == 0) ? k : n) || ldc < m) return IPEPS_EINVAL;
  constexpr int BM = 64, BN = 64, BK = 16, TM = 4, TN = 4, NT = (BM / TM) * (BN / TN);
  const int64_t gx = (m + BM - 1) / BM, gy = (n + BN - 1) / BN;
  if (gy > 65535 || gx > int64_t(0x7fffffff)) {
    std::fprintf(stderr, "ipeps_gemm_f64_noalloc: m = %lld, n = %lld exceed the kernel grid (n <= %lld)\n",
                 static_cast<long long>(m), static_cast<long long>(n), 65535LL * BN);
    return IPEPS_EINVAL;
  }
  double* scratch = nullptr;
  if (noalloc_scratch(&scratch) != cudaSuccess) return IPEPS_ECUDA;
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // same split heuristic as the allocating path, capped by the scratch size
  const int64_t tiles = gx * gy, target = 2LL * sms;
  int64_t S = 1;
  if (tiles < target && k >= 8 * BK * 2) S = std::min<int64_t>(std::min<int64_t>((target + tiles - 1) / tiles, k / (8 * BK)), 64);
  // cap by the scratch: S * m * n partial sums at most (S = 1 uses none)
  S = std::max<int64_t>(1, std::min<int64_t>(S, kNoAllocScratchDoubles / (m * n)));
  int64_t kchunk = (k + S - 1) / S;
  kchunk = ((kchunk + BK - 1) / BK) * BK;
  S = (k + kchunk - 1) / kchunk;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const cuDoubleComplex a = make_cuDoubleComplex(alpha, 0), b = make_cuDoubleComplex(beta, 0);
  dim3 grid{unsigned(gx), unsigned(gy), unsigned(S)};
  gemm_kernel<double, BM, BN, BK, TM, TN><<<grid, NT, 0, st>>>(oa, ob, m, n, k, kchunk, a, A, lda, B, ldb, b, C, ldc,
                                                                S > 1 ? scratch : nullptr);
  if (cudaGetLastError() != cudaSuccess) return IPEPS_ECUDA;
  if (S > 1) {
    const int64_t tot = m * n;
    splitk_reduce<double><<<unsigned((tot + 255) / 256), 256, 0, st>>>(m, n, int(S), scratch, a, b, C, ldc);
    if (cudaGetLastError() != cudaSuccess) return IPEPS_ECUDA;
  }
  return IPEPS_OK;
}
