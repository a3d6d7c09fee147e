// 3xTF32 tcgen05 GEMM (mixed-precision form): not built yet.
#include "ctx.cuh"

namespace ipeps {

void gemm_tf32x3(Ctx&, char, char, int64_t, int64_t, int64_t, double, const double*, int64_t, const double*,
                 int64_t, double, double*, int64_t) {
  throw Error(kEInval, "mixed precision (3xTF32) GEMM is not available in this build");
}

}  // namespace ipeps
