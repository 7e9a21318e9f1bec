// tc_gemm.cu -- tensor-core Schur-complement update (3xTF32) for the mixed factor.
#include "tc_gemm.cuh"

namespace jfg {
namespace tc {

bool schur_update_tf32x3(const int32_t*, int, const int32_t*, const int32_t*, const int64_t*, const int64_t*,
                         float*, float*, int, int, cudaStream_t) {
  return false;
}

}  // namespace tc
}  // namespace jfg
