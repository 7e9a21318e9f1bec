// tc_gemm.cuh -- tensor-core Schur-complement update for the mixed factor.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace jfg {
namespace tc {

// U -= L21 L21^T for every front of a level in 3xTF32 split precision on the
// sm_100a tensor cores.  Returns false when the tensor-core path is not
// applicable, in which case the caller runs the SIMT FP32 kernel.
bool schur_update_tf32x3(const int32_t* list, int count, const int32_t* first, const int32_t* mrows,
                         const int64_t* Lptr, const int64_t* Uptr, float* L, float* U, int max_r,
                         int max_c, cudaStream_t st);

}  // namespace tc
}  // namespace jfg
