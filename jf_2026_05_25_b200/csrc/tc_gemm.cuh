// tc_gemm.cuh -- tensor-core Schur-complement update for the mixed factor.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "jfg_internal.h"

namespace jfg {
namespace tc {

// U = -L21 L21^T for every front of a level in 3xTF32 split precision on the
// sm_100a tensor cores (tcgen05.mma, accumulator in tensor memory).  Returns
// false when the tensor-core path is switched off (it runs only with the
// environment variable JFG_TENSOR_CORES=1, read at every call) or could not
// be launched, in which case the caller runs the SIMT FP32 kernel.  A bounded
// wait that expires records EE_TC_TIMEOUT in *err.
bool schur_update_tf32x3(const int32_t* list, int count, const int32_t* first, const int32_t* mrows,
                         const int64_t* Lptr, const int64_t* Uptr, float* L, float* U, int max_r,
                         int max_c, DevError* err, cudaStream_t st);

// Whether the tensor-core path is switched on (JFG_TENSOR_CORES=1).
bool enabled();

}  // namespace tc
}  // namespace jfg
