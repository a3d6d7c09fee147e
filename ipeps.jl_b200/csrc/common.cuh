// Core types for the B200 CTMRG engine: column-major device tensors (the
// layout Julia hands over through ccall), a stream-ordered allocator and the
// error plumbing shared by every translation unit.
#pragma once

#include <cuda_runtime.h>
#include <cuComplex.h>

#include <cstdint>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace ipeps {

enum class DType : int { F64 = 0, C128 = 1 };

inline size_t dtype_size(DType t) { return t == DType::F64 ? 8 : 16; }

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// status codes shared with include/ipeps_b200.h
constexpr int kOk = 0;
constexpr int kENotConv = 1;
constexpr int kENonFinite = 2;
constexpr int kEOOM = 3;
constexpr int kEInval = 4;
constexpr int kECuda = 5;

#define IPEPS_CUDA(call)                                                              \
  do {                                                                                \
    cudaError_t _e = (call);                                                          \
    if (_e != cudaSuccess) {                                                          \
      int _c = (_e == cudaErrorMemoryAllocation) ? ::ipeps::kEOOM : ::ipeps::kECuda;   \
      throw ::ipeps::Error(_c, std::string(#call) + ": " + cudaGetErrorString(_e) +    \
                                   " at " + __FILE__ + ":" + std::to_string(__LINE__)); \
    }                                                                                 \
  } while (0)

#define IPEPS_CHECK(cond, msg)                                               \
  do {                                                                       \
    if (!(cond)) throw ::ipeps::Error(::ipeps::kEInval, std::string(msg));   \
  } while (0)

#define IPEPS_LAUNCH_CHECK() IPEPS_CUDA(cudaGetLastError())

// Owner of a context's CUDA stream; every buffer keeps it alive, so a
// buffer that outlives its context is still released in stream order.
struct StreamHolder {
  cudaStream_t s = nullptr;
  int device = 0;
  ~StreamHolder() {
    if (s) {
      cudaSetDevice(device);
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};

// A device buffer released on its stream (stream-ordered, pool-backed).
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  std::shared_ptr<StreamHolder> sh;
  DBuf(size_t n, std::shared_ptr<StreamHolder> h) : bytes(n), sh(std::move(h)) {
    if (n) IPEPS_CUDA(cudaMallocAsync(&p, n, sh->s));
  }
  ~DBuf() {
    if (p) cudaFreeAsync(p, sh->s);
  }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
};

constexpr int kMaxDims = 10;

// Column-major dense tensor on the device (dims[0] is the fastest index).
struct Tensor {
  std::shared_ptr<DBuf> buf;
  size_t offset = 0;  // bytes
  int nd = 0;
  int64_t dims[kMaxDims] = {0};
  DType dt = DType::F64;

  bool empty() const { return buf == nullptr; }
  int64_t numel() const {
    int64_t n = 1;
    for (int i = 0; i < nd; ++i) n *= dims[i];
    return n;
  }
  size_t bytes() const { return size_t(numel()) * dtype_size(dt); }
  void* data() const { return static_cast<char*>(buf->p) + offset; }
  double* f64() const { return static_cast<double*>(data()); }
  int64_t dim(int i) const { return i < nd ? dims[i] : 1; }
  std::vector<int64_t> shape() const { return std::vector<int64_t>(dims, dims + nd); }
  // Julia-style reshape: free for column-major storage.
  Tensor reshape(const std::vector<int64_t>& s) const {
    Tensor t = *this;
    int64_t n = 1, neg = -1;
    for (size_t i = 0; i < s.size(); ++i) {
      if (s[i] < 0) neg = int64_t(i);
      else n *= s[i];
    }
    t.nd = int(s.size());
    for (size_t i = 0; i < s.size(); ++i) t.dims[i] = s[i];
    if (neg >= 0) t.dims[neg] = n ? numel() / n : 0;
    IPEPS_CHECK(t.numel() == numel(), "reshape: element count mismatch");
    return t;
  }
};

std::string shape_str(const Tensor& t);

}  // namespace ipeps
