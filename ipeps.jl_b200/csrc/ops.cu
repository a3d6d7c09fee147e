// Memory-bound kernels: index permutation (coalesced on both sides through a
// shared-memory tile when the fastest index moves), max-abs reduction,
// scaling, axpy, conj, RNG, and the context / allocator plumbing.
#include "ctx.cuh"

#include <algorithm>
#include <cstdlib>
#include <atomic>
#include <numeric>

namespace ipeps {

std::string shape_str(const Tensor& t) {
  std::string s = "(";
  for (int i = 0; i < t.nd; ++i) s += std::to_string(t.dims[i]) + (i + 1 < t.nd ? "," : "");
  return s + ")";
}

// ------------------------------------------------------------------ context
Ctx::Ctx(int dev) : device(dev) {
  IPEPS_CUDA(cudaSetDevice(dev));
  sh = std::make_shared<StreamHolder>();
  sh->device = dev;
  IPEPS_CUDA(cudaStreamCreateWithFlags(&sh->s, cudaStreamNonBlocking));
  stream = sh->s;
  IPEPS_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev));
  // keep freed blocks in the pool (no release back to the driver)
  cudaMemPool_t pool;
  IPEPS_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t thr = UINT64_MAX;
  IPEPS_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  // Once per device: grow the pool by a block of min(8 GiB, a quarter of the
  // free memory) and hand it back, so that steady-state allocations (up to a
  // few GB at D=5 chi=100, from up to three streams) are served from reserved
  // memory instead of mapping new memory in the middle of a CTMRG step.
  // IPEPS_POOL_RESERVE_MB overrides the 8 GiB (0: no reservation, e.g. for
  // processes that share the GPU or run under a kernel profiler).
  static std::atomic<bool> reserved[64];
  if (dev >= 0 && dev < 64 && !reserved[dev].exchange(true)) {
    size_t free_b = 0, total_b = 0;
    size_t cap = size_t(8) << 30;
    if (const char* env = std::getenv("IPEPS_POOL_RESERVE_MB")) cap = size_t(std::strtoull(env, nullptr, 10)) << 20;
    if (cap > 0 && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
      const size_t want = std::min<size_t>(cap, free_b / 4);
      void* p = nullptr;
      if (want > 0 && cudaMallocAsync(&p, want, stream) == cudaSuccess) {
        IPEPS_CUDA(cudaFreeAsync(p, stream));
        IPEPS_CUDA(cudaStreamSynchronize(stream));
      } else {
        (void)cudaGetLastError();  // not fatal: the pool then grows on demand
      }
    }
  }
  scal = std::make_shared<DBuf>(4096, sh);
  IPEPS_CUDA(cudaMemsetAsync(scal->p, 0, 4096, stream));
  d_status = reinterpret_cast<int*>(static_cast<char*>(scal->p) + 4000);
}

cudaEvent_t Ctx::take_event() {
  if (!ev_pool.empty()) {
    cudaEvent_t e = ev_pool.back();
    ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  IPEPS_CUDA(cudaEventCreate(&e));
  return e;
}

std::array<double, int(KFam::Count)> Ctx::prof_collect() {
  std::array<double, int(KFam::Count)> ms{};
  sync();
  for (auto& r : prof_rec) {
    float t = 0;
    IPEPS_CUDA(cudaEventElapsedTime(&t, std::get<1>(r), std::get<2>(r)));
    ms[std::get<0>(r)] += t;
    ev_pool.push_back(std::get<1>(r));
    ev_pool.push_back(std::get<2>(r));
  }
  prof_rec.clear();
  return ms;
}

Ctx::~Ctx() {
  for (auto& r : prof_rec) {
    cudaEventDestroy(std::get<1>(r));
    cudaEventDestroy(std::get<2>(r));
  }
  for (auto e : ev_pool) cudaEventDestroy(e);
  ws.reset();
  scal.reset();
  sh.reset();  // the stream goes when the last buffer that uses it is released
}

Tensor Ctx::alloc(DType dt, const std::vector<int64_t>& dims) {
  Tensor t;
  t.dt = dt;
  t.nd = int(dims.size());
  IPEPS_CHECK(t.nd <= kMaxDims, "too many dims");
  for (int i = 0; i < t.nd; ++i) t.dims[i] = dims[i];
  t.buf = std::make_shared<DBuf>(std::max<size_t>(t.bytes(), 16), sh);
  return t;
}

Tensor Ctx::zeros(DType dt, const std::vector<int64_t>& dims) {
  Tensor t = alloc(dt, dims);
  IPEPS_CUDA(cudaMemsetAsync(t.data(), 0, t.bytes(), stream));
  return t;
}

void* Ctx::workspace(size_t bytes) {
  if (!ws || ws->bytes < bytes) ws = std::make_shared<DBuf>(std::max<size_t>(bytes, 1 << 20), sh);
  return ws->p;
}

// ------------------------------------------------------------------ permute
namespace {

struct PermArgs {
  int nd;
  int64_t odims[kMaxDims];    // output dims
  int64_t istride[kMaxDims];  // input stride of output dim i
};

template <typename T>
__global__ void permute_simple(PermArgs a, int64_t total, const T* __restrict__ in, T* __restrict__ out) {
  for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    int64_t r = idx, off = 0;
#pragma unroll
    for (int i = 0; i < kMaxDims; ++i) {
      if (i >= a.nd) break;
      int64_t q = r / a.odims[i];
      off += (r - q * a.odims[i]) * a.istride[i];
      r = q;
    }
    out[idx] = in[off];
  }
}

// perm[0] == 0 with a long first dimension: every output "row" (n0
// consecutive elements) is a contiguous run of the input too.  One warp per
// row; the mixed-radix decomposition of the row index (integer divisions) is
// done once per row instead of once per element.
struct RowArgs {
  int nd;                     // output dims after the first
  int64_t n0;                 // row length (extent of the shared first dim)
  int64_t odims[kMaxDims];    // output dims 1.. (innermost first)
  int64_t istride[kMaxDims];  // their input strides
};

// A warp copies one chunk of up to kPermChunk consecutive elements of one
// row, so that a few very long rows still spread over the whole GPU and many
// short rows take one warp each.
constexpr int64_t kPermChunk = 2048;

// SMALL: the unit count and every output dim fit in 32 bits, so the row
// index is decomposed with 32-bit divisions (a 64-bit division is several
// times the instructions, and the decomposition is most of the work of a
// short row).
template <typename T, bool SMALL>
__global__ void permute_rows(RowArgs a, int64_t rows, int64_t nchunk, const T* __restrict__ in, T* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const int64_t units = rows * nchunk;
  for (int64_t u = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; u < units; u += nwarps) {
    int64_t r, c0, off = 0;
    if constexpr (SMALL) {
      const uint32_t uu = uint32_t(u), nc = uint32_t(nchunk);
      uint32_t q = uu / nc;
      r = q;
      c0 = int64_t(uu - q * nc) * kPermChunk;
      for (int i = 0; i < a.nd; ++i) {
        const uint32_t od = uint32_t(a.odims[i]);
        const uint32_t t = q / od;
        off += int64_t(q - t * od) * a.istride[i];
        q = t;
      }
    } else {
      r = u / nchunk;
      c0 = (u - r * nchunk) * kPermChunk;
      int64_t q = r;
      for (int i = 0; i < a.nd; ++i) {
        const int64_t t = q / a.odims[i];
        off += (q - t * a.odims[i]) * a.istride[i];
        q = t;
      }
    }
    const T* src = in + off;
    T* dst = out + r * a.n0;
    const int64_t c1 = min(a.n0, c0 + kPermChunk);
    if (sizeof(T) == 8 && ((off | a.n0 | c0) & 1) == 0 &&
        ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) == 0) {
      // both runs 16-byte aligned: two doubles per load and store
      const double2* s2 = reinterpret_cast<const double2*>(src);
      double2* d2 = reinterpret_cast<double2*>(dst);
#pragma unroll 4
      for (int64_t i = (c0 >> 1) + lane; i < (c1 >> 1); i += 32) d2[i] = s2[i];
      if ((c1 & 1) && lane == 0) dst[c1 - 1] = src[c1 - 1];
    } else {
#pragma unroll 4
      for (int64_t i = c0 + lane; i < c1; i += 32) dst[i] = src[i];
    }
  }
}

struct TileArgs {
  int64_t n0, nq;        // extent of input dim 0 and of input dim q (= output dim 0)
  int64_t in_q_stride;   // input stride of dim q
  int64_t out_p_stride;  // output stride of input dim 0
  int nrest;
  int64_t rdims[kMaxDims];
  int64_t rin[kMaxDims];
  int64_t rout[kMaxDims];
  int64_t rest_total;
};

template <typename T>
__global__ void permute_tiled(TileArgs a, const T* __restrict__ in, T* __restrict__ out) {
  __shared__ T tile[32][33];
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  const int64_t x0 = int64_t(blockIdx.x) * 32, y0 = int64_t(blockIdx.y) * 32;
  for (int64_t rest = blockIdx.z; rest < a.rest_total; rest += gridDim.z) {
    int64_t r = rest, oin = 0, oout = 0;
    for (int i = 0; i < a.nrest; ++i) {
      int64_t q = r / a.rdims[i];
      int64_t v = r - q * a.rdims[i];
      oin += v * a.rin[i];
      oout += v * a.rout[i];
      r = q;
    }
    // load: coalesced along input dim 0
    for (int j = ty; j < 32; j += 8) {
      int64_t i0 = x0 + tx, iq = y0 + j;
      if (i0 < a.n0 && iq < a.nq) tile[j][tx] = in[oin + i0 + iq * a.in_q_stride];
    }
    __syncthreads();
    // store: coalesced along output dim 0 (= input dim q)
    for (int j = ty; j < 32; j += 8) {
      int64_t iq = y0 + tx, i0 = x0 + j;
      if (i0 < a.n0 && iq < a.nq) out[oout + iq + i0 * a.out_p_stride] = tile[tx][j];
    }
    __syncthreads();
  }
}

template <typename T>
void permute_impl(Ctx& c, const Tensor& in, const std::vector<int>& perm, Tensor& out) {
  const int nd = in.nd;
  int64_t istr[kMaxDims], ostr[kMaxDims];
  istr[0] = 1;
  for (int i = 1; i < nd; ++i) istr[i] = istr[i - 1] * in.dims[i - 1];
  ostr[0] = 1;
  for (int i = 1; i < nd; ++i) ostr[i] = ostr[i - 1] * out.dims[i - 1];
  const int64_t total = in.numel();
  const T* ip = static_cast<const T*>(in.data());
  T* op = static_cast<T*>(out.data());
  if (perm[0] == 0 && in.dims[0] >= 16 && nd > 1) {
    RowArgs a{};
    a.nd = nd - 1;
    a.n0 = in.dims[0];
    for (int i = 1; i < nd; ++i) {
      a.odims[i - 1] = out.dims[i];
      a.istride[i - 1] = istr[perm[i]];
    }
    const int64_t rows = total / a.n0;
    const int64_t nchunk = (a.n0 + kPermChunk - 1) / kPermChunk;
    const int64_t blocks = std::min<int64_t>((rows * nchunk + 7) / 8, int64_t(c.sm_count) * 16);
    bool small = rows * nchunk <= int64_t(UINT32_MAX);
    for (int i = 0; i < a.nd; ++i) small = small && a.odims[i] <= int64_t(UINT32_MAX);
    if (small)
      permute_rows<T, true><<<unsigned(std::max<int64_t>(blocks, 1)), 256, 0, c.stream>>>(a, rows, nchunk, ip, op);
    else
      permute_rows<T, false><<<unsigned(std::max<int64_t>(blocks, 1)), 256, 0, c.stream>>>(a, rows, nchunk, ip, op);
  } else if (perm[0] == 0 || in.dims[0] == 1 || out.dims[0] == 1) {
    PermArgs a{};
    a.nd = nd;
    for (int i = 0; i < nd; ++i) {
      a.odims[i] = out.dims[i];
      a.istride[i] = istr[perm[i]];
    }
    int64_t blocks = std::min<int64_t>((total + 255) / 256, int64_t(c.sm_count) * 16);
    permute_simple<T><<<unsigned(std::max<int64_t>(blocks, 1)), 256, 0, c.stream>>>(a, total, ip, op);
  } else {
    const int q = perm[0];
    int p = 0;
    for (int i = 0; i < nd; ++i)
      if (perm[i] == 0) p = i;
    TileArgs a{};
    a.n0 = in.dims[0];
    a.nq = in.dims[q];
    a.in_q_stride = istr[q];
    a.out_p_stride = ostr[p];
    a.nrest = 0;
    a.rest_total = 1;
    for (int i = 0; i < nd; ++i) {  // remaining input dims
      if (i == 0 || i == q) continue;
      int oi = 0;
      for (int t = 0; t < nd; ++t)
        if (perm[t] == i) oi = t;
      a.rdims[a.nrest] = in.dims[i];
      a.rin[a.nrest] = istr[i];
      a.rout[a.nrest] = ostr[oi];
      a.nrest++;
      a.rest_total *= in.dims[i];
    }
    dim3 grid(unsigned((a.n0 + 31) / 32), unsigned((a.nq + 31) / 32),
              unsigned(std::min<int64_t>(a.rest_total, 65535)));
    IPEPS_CHECK(grid.x <= 2147483647u && grid.y <= 65535u, "permute: grid too large");
    permute_tiled<T><<<grid, dim3(32, 8), 0, c.stream>>>(a, ip, op);
  }
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Permute, 0, 2.0 * double(total) * sizeof(T));
}

}  // namespace

Tensor permute(Ctx& c, const Tensor& in, const std::vector<int>& perm) {
  IPEPS_CHECK(int(perm.size()) == in.nd, "permute: rank mismatch");
  std::vector<int64_t> od(in.nd);
  std::vector<bool> seen(in.nd, false);
  for (int i = 0; i < in.nd; ++i) {
    IPEPS_CHECK(perm[i] >= 0 && perm[i] < in.nd && !seen[perm[i]], "permute: bad permutation");
    seen[perm[i]] = true;
    od[i] = in.dims[perm[i]];
  }
  Tensor out = c.alloc(in.dt, od);
  if (in.numel() == 0) return out;
  // identity (ignoring unit dims) -> plain copy
  std::vector<int> nz;
  for (int i = 0; i < in.nd; ++i)
    if (in.dims[perm[i]] != 1) nz.push_back(perm[i]);
  if (std::is_sorted(nz.begin(), nz.end())) {
    IPEPS_CUDA(cudaMemcpyAsync(out.data(), in.data(), in.bytes(), cudaMemcpyDeviceToDevice, c.stream));
    return out;
  }
  // drop unit dims for the kernel (keeps index arithmetic short)
  Tensor in2 = in, out2 = out;
  std::vector<int> keep;
  for (int i = 0; i < in.nd; ++i)
    if (in.dims[i] != 1) keep.push_back(i);
  std::vector<int> rank(in.nd, -1);
  for (size_t r = 0; r < keep.size(); ++r) rank[keep[r]] = int(r);
  std::vector<int> p2;
  for (int i = 0; i < in.nd; ++i)
    if (in.dims[perm[i]] != 1) p2.push_back(rank[perm[i]]);
  // merge runs of input dims that stay adjacent (and in order) in the output:
  // fewer dims, longer contiguous runs, shorter index arithmetic
  std::vector<int64_t> kd(keep.size());
  for (size_t r = 0; r < keep.size(); ++r) kd[r] = in.dims[keep[r]];
  std::vector<int> gstart;  // output-ordered groups: first input dim of each
  std::vector<int64_t> gsize;
  for (size_t t = 0; t < p2.size(); ++t) {
    if (t > 0 && p2[t] == p2[t - 1] + 1) {
      gsize.back() *= kd[p2[t]];
    } else {
      gstart.push_back(p2[t]);
      gsize.push_back(kd[p2[t]]);
    }
  }
  std::vector<int> order(gstart.size());  // groups sorted by input position
  for (size_t g = 0; g < order.size(); ++g) order[g] = int(g);
  std::sort(order.begin(), order.end(), [&](int x, int y) { return gstart[x] < gstart[y]; });
  std::vector<int> gpos(gstart.size());
  for (size_t r = 0; r < order.size(); ++r) gpos[order[r]] = int(r);
  in2.nd = int(order.size());
  for (size_t r = 0; r < order.size(); ++r) in2.dims[r] = gsize[order[r]];
  p2.assign(gstart.size(), 0);
  for (size_t g = 0; g < gstart.size(); ++g) p2[g] = gpos[g];
  out2.nd = int(p2.size());
  for (size_t r = 0; r < p2.size(); ++r) out2.dims[r] = in2.dims[p2[r]];
  ProfScope ps(c, KFam::Permute);
  if (in.dt == DType::F64) permute_impl<double>(c, in2, p2, out2);
  else permute_impl<double2>(c, in2, p2, out2);
  return out;
}

Tensor clone(Ctx& c, const Tensor& in) {
  Tensor out = c.alloc(in.dt, in.shape());
  IPEPS_CUDA(cudaMemcpyAsync(out.data(), in.data(), in.bytes(), cudaMemcpyDeviceToDevice, c.stream));
  return out;
}

// --------------------------------------------------------------- reductions
namespace {

__device__ __forceinline__ double absval(double x) { return fabs(x); }
__device__ __forceinline__ double absval(double2 x) { return hypot(x.x, x.y); }

template <typename T>
__global__ void maxabs_kernel(const T* __restrict__ x, int64_t n, unsigned long long* out) {
  double m = 0.0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    m = fmax(m, absval(x[i]));
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double sm[32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = (threadIdx.x < (blockDim.x >> 5)) ? sm[threadIdx.x] : 0.0;
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    // non-negative doubles order like their bit patterns
    if (threadIdx.x == 0) atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(m)));
  }
}

__global__ void scale_inv_kernel(double* __restrict__ x, int64_t n, const double* __restrict__ s) {
  const double inv = 1.0 / s[0];
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    x[i] *= inv;
}

__global__ void scale_c_kernel(double2* __restrict__ x, int64_t n, double2 s) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double2 v = x[i];
    x[i] = make_double2(v.x * s.x - v.y * s.y, v.x * s.y + v.y * s.x);
  }
}

__global__ void scale_r_kernel(double* __restrict__ x, int64_t n, double s) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    x[i] *= s;
}

__global__ void axpy_r_kernel(double a, const double* __restrict__ x, double* __restrict__ y, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[i] = fma(a, x[i], y[i]);
}

__global__ void axpy_c_kernel(double2 a, const double2* __restrict__ x, double2* __restrict__ y, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double2 v = x[i], w = y[i];
    w.x += a.x * v.x - a.y * v.y;
    w.y += a.x * v.y + a.y * v.x;
    y[i] = w;
  }
}

__global__ void axpy_rc_kernel(double2 a, const double* __restrict__ x, double2* __restrict__ y, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double v = x[i];
    double2 w = y[i];
    w.x += a.x * v;
    w.y += a.y * v;
    y[i] = w;
  }
}

__global__ void conj_kernel(const double2* __restrict__ x, double2* __restrict__ y, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double2 v = x[i];
    y[i] = make_double2(v.x, -v.y);
  }
}

__global__ void to_complex_kernel(const double* __restrict__ x, double2* __restrict__ y, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[i] = make_double2(x[i], 0.0);
}

__global__ void flag_status_kernel(int* status, int bits) { atomicOr(status, bits); }

__global__ void finite_kernel(const double* __restrict__ x, int64_t n, int* status) {
  bool bad = false;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    bad |= !isfinite(x[i]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(status, 2);
}

// counter-based RNG: splitmix64 -> Box-Muller
__device__ __forceinline__ uint64_t splitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

__global__ void randn_kernel(double* __restrict__ x, int64_t n, uint64_t seed) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    uint64_t a = splitmix(seed ^ (2 * uint64_t(i)));
    uint64_t b = splitmix(seed ^ (2 * uint64_t(i) + 1));
    double u1 = (double((a >> 11) + 1)) * (1.0 / 9007199254740993.0);  // (0,1]
    double u2 = double(b >> 11) * (1.0 / 9007199254740992.0);
    x[i] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  }
}

unsigned grid_for(Ctx& c, int64_t n) {
  return unsigned(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, int64_t(c.sm_count) * 8)));
}

}  // namespace

void maxabs(Ctx& c, const Tensor& x, double* d_out) {
  IPEPS_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double), c.stream));
  const int64_t n = x.numel();
  if (x.dt == DType::F64)
    maxabs_kernel<double><<<grid_for(c, n), 256, 0, c.stream>>>(x.f64(), n, reinterpret_cast<unsigned long long*>(d_out));
  else
    maxabs_kernel<double2><<<grid_for(c, n), 256, 0, c.stream>>>(static_cast<const double2*>(x.data()), n,
                                                                  reinterpret_cast<unsigned long long*>(d_out));
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Reduce, 0, double(x.bytes()));
}

void scale_inv(Ctx& c, Tensor& x, const double* d_s) {
  const int64_t n = x.numel() * (x.dt == DType::F64 ? 1 : 2);
  scale_inv_kernel<<<grid_for(c, n), 256, 0, c.stream>>>(x.f64(), n, d_s);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Elementwise, 0, 2.0 * double(x.bytes()));
}

void scale(Ctx& c, Tensor& x, cuDoubleComplex s) {
  const int64_t n = x.numel();
  if (x.dt == DType::F64) {
    IPEPS_CHECK(s.y == 0.0, "scale: complex factor on real tensor");
    scale_r_kernel<<<grid_for(c, n), 256, 0, c.stream>>>(x.f64(), n, s.x);
  } else {
    scale_c_kernel<<<grid_for(c, n), 256, 0, c.stream>>>(static_cast<double2*>(x.data()), n, make_double2(s.x, s.y));
  }
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Elementwise, 0, 2.0 * double(x.bytes()));
}

void axpy(Ctx& c, cuDoubleComplex a, const Tensor& x, Tensor& y) {
  IPEPS_CHECK(x.numel() == y.numel(), "axpy: size mismatch " + shape_str(x) + " vs " + shape_str(y));
  const int64_t n = x.numel();
  if (y.dt == DType::F64) {
    IPEPS_CHECK(x.dt == DType::F64 && a.y == 0.0, "axpy: complex into real");
    axpy_r_kernel<<<grid_for(c, n), 256, 0, c.stream>>>(a.x, x.f64(), y.f64(), n);
  } else if (x.dt == DType::C128) {
    axpy_c_kernel<<<grid_for(c, n), 256, 0, c.stream>>>(make_double2(a.x, a.y), static_cast<const double2*>(x.data()),
                                                         static_cast<double2*>(y.data()), n);
  } else {
    axpy_rc_kernel<<<grid_for(c, n), 256, 0, c.stream>>>(make_double2(a.x, a.y), x.f64(), static_cast<double2*>(y.data()), n);
  }
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Elementwise, 0, 3.0 * double(y.bytes()));
}

Tensor conj(Ctx& c, const Tensor& x) {
  if (x.dt == DType::F64) return clone(c, x);
  Tensor y = c.alloc(x.dt, x.shape());
  conj_kernel<<<grid_for(c, x.numel()), 256, 0, c.stream>>>(static_cast<const double2*>(x.data()),
                                                           static_cast<double2*>(y.data()), x.numel());
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Elementwise, 0, 2.0 * double(x.bytes()));
  return y;
}

Tensor to_complex(Ctx& c, const Tensor& x) {
  if (x.dt == DType::C128) return x;
  Tensor y = c.alloc(DType::C128, x.shape());
  to_complex_kernel<<<grid_for(c, x.numel()), 256, 0, c.stream>>>(x.f64(), static_cast<double2*>(y.data()), x.numel());
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Elementwise, 0, 3.0 * double(x.bytes()));
  return y;
}

void check_finite(Ctx& c, const Tensor& x) {
  const int64_t n = x.numel() * (x.dt == DType::F64 ? 1 : 2);
  finite_kernel<<<grid_for(c, n), 256, 0, c.stream>>>(x.f64(), n, c.d_status);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Reduce, 0, double(x.bytes()));
}

void flag_status(Ctx& c, int bits) {
  flag_status_kernel<<<1, 1, 0, c.stream>>>(c.d_status, bits);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Reduce);
}

void randn(Ctx& c, Tensor& x) {
  const int64_t n = x.numel() * (x.dt == DType::F64 ? 1 : 2);
  uint64_t seed = c.rng_seed * 0x2545F4914F6CDD1DULL + (c.rng_counter++);
  randn_kernel<<<grid_for(c, n), 256, 0, c.stream>>>(x.f64(), n, seed);
  IPEPS_LAUNCH_CHECK();
  c.count(KFam::Elementwise, 0, double(x.bytes()));
}

}  // namespace ipeps
