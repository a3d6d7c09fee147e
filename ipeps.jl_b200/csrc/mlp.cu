// The warm-start network: a 3-layer perceptron n_in -> n_h -> n_h -> n_out
// with GELU on the hidden layers, trained by mean-squared error and Adam.
// Every matrix product of the forward and backward pass runs on the BF16
// tcgen05 GEMM (operands rounded to BF16, FP32 accumulation); parameters,
// activations, gradients and the Adam moments are FP32.  Matrices are
// column-major with the batch as the row index: X (B x n_in), W1 (n_in x n_h),
// Z1 = X W1 + b1, H1 = gelu(Z1), ..., Y = H2 W3 + b3 (B x n_out).
#include "mlp.cuh"

#include <cmath>

namespace ipeps {
namespace {

// GELU, tanh form (Hendrycks & Gimpel): 0.5 x (1 + tanh(c (x + 0.044715 x^3))), c = sqrt(2/pi)
constexpr float kGeluC = 0.7978845608028654f;

__device__ __forceinline__ float gelu(float x) {
  return 0.5f * x * (1.0f + tanhf(kGeluC * (x + 0.044715f * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float u = kGeluC * (x + 0.044715f * x * x * x);
  const float t = tanhf(u);
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * kGeluC * (1.0f + 3.0f * 0.044715f * x * x);
}

// Z (B x n) += b[col]; H = gelu(Z) when H is given (Z keeps the pre-activation)
__global__ void bias_act_kernel(float* Z, const float* b, int64_t B, int64_t n, float* H) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= B * n) return;
  const float z = Z[t] + b[t / B];
  Z[t] = z;
  if (H) H[t] = gelu(z);
}

// dZ = dH * gelu'(Z)
__global__ void act_back_kernel(const float* dH, const float* Z, int64_t n, float* dZ) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < n) dZ[t] = dH[t] * gelu_grad(Z[t]);
}

// db[j] = sum_i dZ[i, j] (one warp per column)
__global__ void colsum_kernel(const float* dZ, int64_t B, int64_t n, float* db) {
  const int64_t col = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (col >= n) return;
  float s = 0.0f;
  for (int64_t i = lane; i < B; i += 32) s += dZ[i + col * B];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) db[col] = s;
}

// mean-squared error over B x n: loss += sum (Y - T)^2 / (B n), dY = 2 (Y - T) / (B n)
__global__ void mse_kernel(const float* Y, const float* T, int64_t n, float inv, float* dY, double* loss) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double e2 = 0.0;
  if (t < n) {
    const float e = Y[t] - T[t];
    dY[t] = 2.0f * inv * e;
    e2 = double(e) * e * inv;
  }
  for (int o = 16; o; o >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, o);
  if ((threadIdx.x & 31) == 0 && e2 != 0.0) atomicAdd(loss, e2);
}

// Adam (Kingma & Ba) with bias correction
__global__ void adam_kernel(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gt = g[t];
  const float mt = b1 * m[t] + (1.0f - b1) * gt;
  const float vt = b2 * v[t] + (1.0f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  p[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
}

// N(0, s^2) from a counter hash (splitmix64) and the Box-Muller transform
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
__global__ void randn_f32_kernel(float* x, int64_t n, uint64_t seed, float s) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint64_t h1 = mix64(seed ^ (uint64_t(t) * 2 + 1)), h2 = mix64(seed + uint64_t(t) * 2 + 7);
  const double u1 = (double(h1 >> 11) + 1.0) * (1.0 / 9007199254740993.0);
  const double u2 = double(h2 >> 11) * (1.0 / 9007199254740992.0);
  x[t] = float(s * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
}

unsigned blocks(int64_t n) { return unsigned((n + 255) / 256); }

}  // namespace

Mlp::Mlp(Ctx& cc, int n_in_, int n_h_, int n_out_, int max_batch, uint64_t seed)
    : c(cc), n_in(n_in_), n_h(n_h_), n_out(n_out_), cap(max_batch) {
  IPEPS_CHECK(n_in > 0 && n_h > 0 && n_out > 0 && cap > 0, "mlp: bad sizes");
  off[0] = 0;                                // W1
  off[1] = off[0] + int64_t(n_in) * n_h;     // b1
  off[2] = off[1] + n_h;                     // W2
  off[3] = off[2] + int64_t(n_h) * n_h;      // b2
  off[4] = off[3] + n_h;                     // W3
  off[5] = off[4] + int64_t(n_h) * n_out;    // b3
  np = off[5] + n_out;
  auto mk = [&](int64_t n) { return std::make_shared<DBuf>(size_t(n) * 4, c.sh); };
  params = mk(np);
  grads = mk(np);
  m1 = mk(np);
  m2 = mk(np);
  const int64_t B = cap;
  X = mk(B * n_in);
  T = mk(B * n_out);
  Z1 = mk(B * n_h);
  H1 = mk(B * n_h);
  Z2 = mk(B * n_h);
  H2 = mk(B * n_h);
  Y = mk(B * n_out);
  dY = mk(B * n_out);
  dH = mk(B * n_h);
  dZ = mk(B * n_h);
  loss = mk(2);
  // He-style initialisation N(0, 1/fan_in) for the weights, zero biases and moments
  IPEPS_CUDA(cudaMemsetAsync(params->p, 0, size_t(np) * 4, c.stream));
  IPEPS_CUDA(cudaMemsetAsync(m1->p, 0, size_t(np) * 4, c.stream));
  IPEPS_CUDA(cudaMemsetAsync(m2->p, 0, size_t(np) * 4, c.stream));
  const int64_t wn[3] = {int64_t(n_in) * n_h, int64_t(n_h) * n_h, int64_t(n_h) * n_out};
  const int fan[3] = {n_in, n_h, n_h};
  for (int l = 0; l < 3; ++l) {
    randn_f32_kernel<<<blocks(wn[l]), 256, 0, c.stream>>>(p(2 * l), wn[l], seed * 3 + uint64_t(l) + 1,
                                                         float(1.0 / std::sqrt(double(fan[l]))));
    IPEPS_LAUNCH_CHECK();
  }
}

float* Mlp::f(const std::shared_ptr<DBuf>& b) { return static_cast<float*>(b->p); }

void Mlp::forward(int B) {
  IPEPS_CHECK(B > 0 && B <= cap, "mlp: batch larger than the capacity");
  const float* x = f(X);
  gemm_bf16(c, 'N', 'N', B, n_h, n_in, 1.0f, x, B, p(0), n_in, 0.0f, f(Z1), B);
  bias_act_kernel<<<blocks(int64_t(B) * n_h), 256, 0, c.stream>>>(f(Z1), p(1), B, n_h, f(H1));
  IPEPS_LAUNCH_CHECK();
  gemm_bf16(c, 'N', 'N', B, n_h, n_h, 1.0f, f(H1), B, p(2), n_h, 0.0f, f(Z2), B);
  bias_act_kernel<<<blocks(int64_t(B) * n_h), 256, 0, c.stream>>>(f(Z2), p(3), B, n_h, f(H2));
  IPEPS_LAUNCH_CHECK();
  gemm_bf16(c, 'N', 'N', B, n_out, n_h, 1.0f, f(H2), B, p(4), n_h, 0.0f, f(Y), B);
  bias_act_kernel<<<blocks(int64_t(B) * n_out), 256, 0, c.stream>>>(f(Y), p(5), B, n_out, nullptr);
  IPEPS_LAUNCH_CHECK();
}

void Mlp::backward(int B) {
  float* g = f(grads);
  // layer 3: dW3 = H2^T dY, db3 = colsum(dY), dH2 = dY W3^T
  gemm_bf16(c, 'T', 'N', n_h, n_out, B, 1.0f, f(H2), B, f(dY), B, 0.0f, g + off[4], n_h);
  colsum_kernel<<<blocks(int64_t(n_out) * 32), 256, 0, c.stream>>>(f(dY), B, n_out, g + off[5]);
  IPEPS_LAUNCH_CHECK();
  gemm_bf16(c, 'N', 'T', B, n_h, n_out, 1.0f, f(dY), B, p(4), n_h, 0.0f, f(dH), B);
  act_back_kernel<<<blocks(int64_t(B) * n_h), 256, 0, c.stream>>>(f(dH), f(Z2), int64_t(B) * n_h, f(dZ));
  IPEPS_LAUNCH_CHECK();
  // layer 2
  gemm_bf16(c, 'T', 'N', n_h, n_h, B, 1.0f, f(H1), B, f(dZ), B, 0.0f, g + off[2], n_h);
  colsum_kernel<<<blocks(int64_t(n_h) * 32), 256, 0, c.stream>>>(f(dZ), B, n_h, g + off[3]);
  IPEPS_LAUNCH_CHECK();
  gemm_bf16(c, 'N', 'T', B, n_h, n_h, 1.0f, f(dZ), B, p(2), n_h, 0.0f, f(dH), B);
  act_back_kernel<<<blocks(int64_t(B) * n_h), 256, 0, c.stream>>>(f(dH), f(Z1), int64_t(B) * n_h, f(dZ));
  IPEPS_LAUNCH_CHECK();
  // layer 1 (no input gradient)
  gemm_bf16(c, 'T', 'N', n_in, n_h, B, 1.0f, f(X), B, f(dZ), B, 0.0f, g + off[0], n_in);
  colsum_kernel<<<blocks(int64_t(n_h) * 32), 256, 0, c.stream>>>(f(dZ), B, n_h, g + off[1]);
  IPEPS_LAUNCH_CHECK();
}

double Mlp::loss_and_grad(int B) {
  double* d_loss = static_cast<double*>(loss->p);
  IPEPS_CUDA(cudaMemsetAsync(d_loss, 0, 8, c.stream));
  const int64_t n = int64_t(B) * n_out;
  mse_kernel<<<blocks(n), 256, 0, c.stream>>>(f(Y), f(T), n, float(1.0 / double(n)), f(dY), d_loss);
  IPEPS_LAUNCH_CHECK();
  backward(B);
  double h = 0;
  IPEPS_CUDA(cudaMemcpyAsync(&h, d_loss, 8, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  return h;
}

void Mlp::adam(float lr) {
  ++step;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = float(1.0 - std::pow(double(b1), step)), c2 = float(1.0 - std::pow(double(b2), step));
  adam_kernel<<<blocks(np), 256, 0, c.stream>>>(p(0), f(grads), f(m1), f(m2), np, lr, b1, b2, 1e-8f, c1, c2);
  IPEPS_LAUNCH_CHECK();
}

}  // namespace ipeps
