// tc_gemm.cuh -- tensor-core (3xTF32) front updates of the mixed factor.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "jfg_internal.h"

namespace jfg {
namespace tc {

// C -= A B^T on the tensor cores for one level of the mixed factor, the same
// geometry as the SIMT front update (mode 0: panel columns [min(kend, c),
// min(cend, c)) with K = [kbeg, min(kend, c)); mode 1: U = -L21 L21^T).
// Llo holds rn19(v - trunc19(v)) for every FP32 factor entry written by the
// panel triangular solve.  max_rows / max_cols bound the output of any front
// of the level.  Returns false when switched off or not launched, in which
// case the caller runs the SIMT kernel.  A bounded wait that expires records
// EE_TC_TIMEOUT in *err.
bool front_update_tf32x3(const int32_t* list, int count, const int32_t* first, const int32_t* mrows,
                         const int64_t* Lptr, const int64_t* Uptr, float* L, const float* Llo, float* U, int mode,
                         int kbeg, int kend, int cend, int max_rows, int max_cols, DevError* err, cudaStream_t st);

// JFG_TENSOR_CORES, read at every call: 1 = on, 0 = off, -1 = not set (the
// caller picks: on for solid-only models, off where shells are present).
int setting();

// Whether the tensor-core update may run at all (not switched off).
bool enabled();

}  // namespace tc
}  // namespace jfg
