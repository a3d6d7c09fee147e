// Engine context: one CUDA stream per context, a stream-ordered memory pool,
// per-kernel-family launch/flop counters and the small helpers every
// contraction uses.
#pragma once

#include "common.cuh"

#include <array>
#include <atomic>
#include <map>
#include <tuple>

namespace ipeps {

enum class KFam : int {
  Permute = 0,
  GemmF64,
  GemmTF32x3,
  Reduce,
  Elementwise,
  SmallLinalg,
  Jacobi,
  Count
};

struct KStat {
  uint64_t launches = 0;
  double flops = 0;   // algorithmic flops credited (2*M*N*K per real GEMM, 8*M*N*K complex)
  double bytes = 0;   // algorithmic bytes moved (permutes, reductions)
};

enum Precision : int { kPrecFP64 = 0, kPrecMixed = 1 };

struct Ctx {
  int device = 0;
  std::shared_ptr<StreamHolder> sh;
  cudaStream_t stream = nullptr;
  int sm_count = 148;
  int precision = kPrecFP64;
  uint64_t rng_seed = 0x1234abcdULL;
  uint64_t rng_counter = 0;
  std::string last_error;
  std::array<KStat, int(KFam::Count)> stats{};
  uint64_t jacobi_sweeps = 0;
  uint64_t projector_calls = 0;
  uint64_t projector_extra_passes = 0;
  // projector adjoints whose resolvent expansion stopped at its term cap before
  // reaching its tolerance (the gradient may be inexact)
  uint64_t series_cap_hits = 0;
  // Chebyshev terms summed over all projector adjoints, and expansions redone
  // over a wider interval after the resolvent check failed
  uint64_t series_terms = 0;
  uint64_t series_retries = 0;
  // projectors whose kept triplets ended above the residual tolerance (the
  // extra passes stopped converging or ran out)
  uint64_t resid_misses = 0;
  // split-K partial sums live here (grown on demand, stream ordered)
  std::shared_ptr<DBuf> ws;
  // small device scalars (max-abs, traces, status words)
  std::shared_ptr<DBuf> scal;
  int* d_status = nullptr;
  // per-kernel-family CUDA-event timing (enabled by ipeps_prof_enable)
  bool prof = false;
  // with prof: wall ms of the E+grad pullback's phases (checkpoint iterations,
  // energy tape, recorded recomputation of the iterations, their backward,
  // and the projector adjoints inside that backward), stream-synchronised
  std::array<double, 5> ad_phase_ms{};
  std::array<KStat, int(KFam::Count)> prof_stats{};
  std::vector<std::tuple<int, cudaEvent_t, cudaEvent_t>> prof_rec;
  std::vector<cudaEvent_t> ev_pool;
  cudaEvent_t take_event();
  // returns ms per family and clears the records
  std::array<double, int(KFam::Count)> prof_collect();

  explicit Ctx(int dev);
  ~Ctx();

  Tensor alloc(DType dt, const std::vector<int64_t>& dims);
  Tensor zeros(DType dt, const std::vector<int64_t>& dims);
  void* workspace(size_t bytes);
  void sync() { IPEPS_CUDA(cudaStreamSynchronize(stream)); }
  void count(KFam f, double flops = 0, double bytes = 0) {
    auto& s = stats[int(f)];
    s.launches++;
    s.flops += flops;
    s.bytes += bytes;
    if (prof) {
      auto& p = prof_stats[int(f)];
      p.launches++;
      p.flops += flops;
      p.bytes += bytes;
    }
  }
};

// Brackets the launches of one kernel family with CUDA events on the
// context stream while profiling is enabled.
// FP64 contractions for the lifetime of the scope, whatever the context's
// precision: the observables (energies, norms, density matrices) are
// evaluated in FP64 in both forms.
struct Fp64Scope {
  Ctx& c;
  int prev;
  explicit Fp64Scope(Ctx& cc) : c(cc), prev(cc.precision) { c.precision = kPrecFP64; }
  ~Fp64Scope() { c.precision = prev; }
  Fp64Scope(const Fp64Scope&) = delete;
  Fp64Scope& operator=(const Fp64Scope&) = delete;
};

// The dynamic shared-memory limit of a kernel is a per-function, per-device
// attribute: set it once on every device the kernel is launched on.
struct SmemAttrOnce {
  static constexpr int kMaxDevices = 64;
  std::atomic<bool> done[kMaxDevices] = {};
  template <class K>
  void ensure(K kern, int bytes) {
    int dev = 0;
    IPEPS_CUDA(cudaGetDevice(&dev));
    if (dev < kMaxDevices && done[dev].load()) return;
    IPEPS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    if (dev < kMaxDevices) done[dev].store(true);
  }
};

struct ProfScope {
  Ctx& c;
  int fam;
  cudaEvent_t a = nullptr;
  ProfScope(Ctx& cc, KFam f) : c(cc), fam(int(f)) {
    if (c.prof) {
      a = c.take_event();
      cudaEventRecord(a, c.stream);
    }
  }
  ~ProfScope() {
    if (a) {
      cudaEvent_t b = c.take_event();
      cudaEventRecord(b, c.stream);
      c.prof_rec.emplace_back(fam, a, b);
    }
  }
};

// ---------------------------------------------------------------- kernels
// permute: out = permutedims(in, perm) (0-based perm, Julia semantics:
// size(out,i) = size(in, perm[i])).
Tensor permute(Ctx& c, const Tensor& in, const std::vector<int>& perm);
// out = in (copy) into a fresh contiguous tensor
Tensor clone(Ctx& c, const Tensor& in);

// C = alpha*op(A)*op(B) + beta*C, column-major, op in {'N','T','C'}.
// Dispatches on c.precision for real operands (FP64 DMMA or 3xTF32 tcgen05).
void gemm(Ctx& c, DType dt, char opA, char opB, int64_t m, int64_t n, int64_t k,
          cuDoubleComplex alpha, const void* A, int64_t lda, const void* B, int64_t ldb,
          cuDoubleComplex beta, void* C, int64_t ldc, bool force_fp64 = false);
// FP64 GEMM: DMMA for real operands, register-tiled SIMT for complex128
void gemm_f64(Ctx& c, DType dt, char opA, char opB, int64_t m, int64_t n, int64_t k,
              cuDoubleComplex alpha, const void* A, int64_t lda, const void* B, int64_t ldb,
              cuDoubleComplex beta, void* C, int64_t ldc);
// real FP64 GEMM on the DMMA (FP64 tensor-core) path, op in {N, T}
void gemm_f64_dmma(Ctx& c, char opA, char opB, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
                   int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc);
// 3xTF32 tcgen05 GEMM for real operands (FP32-accumulated split products)
// BF16 operands (rounded from FP32 while staged), FP32 accumulation and result; op in {N, T}
void gemm_bf16(Ctx& c, char opA, char opB, int64_t m, int64_t n, int64_t k, float alpha, const float* A, int64_t lda,
               const float* B, int64_t ldb, float beta, float* C, int64_t ldc);
// An FP64 operand split once into TF32 hi/lo planes for the 3xTF32 GEMM:
// rows x Kp FP32 each, K contiguous (K-major), Kp = K rounded up to 32 with
// zero padding, the lo plane stacked after the hi plane.
struct Planes {
  Tensor buf;
  int64_t rows = 0, K = 0, Kp = 0;
  bool empty() const { return buf.empty(); }
};
// X(r, k) = kcontig ? X[k + r*ld] : X[r + k*ld], r < rows, k < K
Planes split_kmajor(Ctx& c, const double* X, int64_t ld, bool kcontig, int64_t rows, int64_t K);
// C = alpha * A B + beta * C with A given as m x k planes and B as n x k planes (B^T rows)
void gemm_tf32x3_planes(Ctx& c, const Planes& A, const Planes& B, int64_t m, int64_t n, int64_t k, double alpha,
                        double beta, double* C, int64_t ldc);
void gemm_tf32x3(Ctx& c, char opA, char opB, int64_t m, int64_t n, int64_t k, double alpha,
                 const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                 int64_t ldc);

inline cuDoubleComplex cplx(double r, double i = 0) { return make_cuDoubleComplex(r, i); }

// Matrix product helpers on 2-D tensors: returns op(A)*op(B)
Tensor matmul(Ctx& c, const Tensor& A, char opA, const Tensor& B, char opB);

// tcon: contraction with the reference's label convention (positive labels
// are summed, negative labels -1,-2,... give the output order).
Tensor tcon(Ctx& c, const Tensor& A, const std::vector<int>& la, const Tensor& B,
            const std::vector<int>& lb);
// out += tcon(...) (out must have the output shape)
void tcon_acc(Ctx& c, Tensor& out, const Tensor& A, const std::vector<int>& la, const Tensor& B,
              const std::vector<int>& lb);

// ------------------------------------------------------------ reductions
// d_out[0] = max |x| (device scalar)
void maxabs(Ctx& c, const Tensor& x, double* d_out);
// x *= 1/d_s[0] (x real or complex), in place
void scale_inv(Ctx& c, Tensor& x, const double* d_s);
// x *= s (complex scalar), in place
void scale(Ctx& c, Tensor& x, cuDoubleComplex s);
// y += a*x
void axpy(Ctx& c, cuDoubleComplex a, const Tensor& x, Tensor& y);
// conj copy (returns new tensor; real input -> plain copy)
Tensor conj(Ctx& c, const Tensor& x);
// convert real tensor to complex128
Tensor to_complex(Ctx& c, const Tensor& x);
// ORs `bits` into the status word on the context stream (host-detected
// conditions that the caller reads with the device-side ones)
void flag_status(Ctx& c, int bits);
// nonfinite scan: sets bit in c.d_status
void check_finite(Ctx& c, const Tensor& x);
// fill with N(0,1) (counter-based hash RNG, reproducible)
void randn(Ctx& c, Tensor& x);

}  // namespace ipeps
