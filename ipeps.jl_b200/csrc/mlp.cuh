// The warm-start network (see mlp.cu).
#pragma once
#include "ctx.cuh"

namespace ipeps {

struct Mlp {
  Ctx& c;
  int n_in, n_h, n_out, cap;
  int64_t off[6] = {0};  // W1, b1, W2, b2, W3, b3 in the flat parameter vector
  int64_t np = 0;
  int step = 0;
  std::shared_ptr<DBuf> params, grads, m1, m2;
  std::shared_ptr<DBuf> X, T, Z1, H1, Z2, H2, Y, dY, dH, dZ, loss;

  Mlp(Ctx& cc, int n_in, int n_h, int n_out, int max_batch, uint64_t seed);
  float* p(int i) { return static_cast<float*>(params->p) + off[i]; }
  static float* f(const std::shared_ptr<DBuf>& b);
  // Y = net(X) for the first B rows of the X buffer
  void forward(int B);
  // with Y from forward(B) and targets in T: mean-squared error; gradients into grads
  double loss_and_grad(int B);
  void backward(int B);
  void adam(float lr);
};

}  // namespace ipeps
