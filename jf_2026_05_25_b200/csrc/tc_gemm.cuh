// tc_gemm.cuh -- tensor-core (3xTF32) front updates of the mixed factor.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "jfg_internal.h"

namespace jfg {
namespace tc {

// output tile (rows and columns) of the tensor-core front update
constexpr int TILE_M = 128;

// C -= A B^T on the tensor cores for one level of the mixed factor, the same
// geometry as the SIMT front update (mode 0: panel columns [min(kend, c),
// min(cend, c)) with K = [kbeg, min(kend, c)); mode 1: U = -L21 L21^T).
// Phi / Plo hold hi = rn19(v) and lo = rn19(v - hi) of every FP32 factor
// entry written by the panel triangular solve, packed per front (offset
// PKptr[s] floats) in 512-byte atoms of 8 rows x 16 columns: atom (sb, rg)
// (columns 16 sb.., rows 8 rg..) at PKptr[s] + (sb * ceil(m/8) + rg) * 128,
// row i of the atom at i * 16 floats, its 4-column chunk q at chunk position
// q ^ ((i >> 1) & 3) (the 64-byte-swizzled K-major image); padding zeroed.
// zero points at 8 KB of zeros.  tiles lists the n_tiles lower 128 x 128
// output tiles with work, (position in list, tile index ti * ntj + tj of the
// front's grid, which starts at the output origin rounded down to a multiple
// of 8 rows).  Returns false when switched off or not launched, in which case
// the caller runs the SIMT kernel.  A bounded wait that expires records
// EE_TC_TIMEOUT in *err.
bool front_update_tf32x3(const int32_t* list, const int2* tiles, int n_tiles, const int32_t* first,
                         const int32_t* mrows, const int64_t* Lptr, const int64_t* Uptr, float* L, const float* Phi,
                         const float* Plo, const int64_t* PKptr, const float* zero, float* U, int mode, int kbeg,
                         int kend, int cend, int drain, DevError* err, cudaStream_t st);

// JFG_TENSOR_CORES, read at every call: 1 = on, 0 = off, -1 = not set (on).
int setting();

// K-slices of 16 columns the tensor core sums per accumulator use before the
// FP32 register drain: JFG_TC_DRAIN when set (1..16), else `dflt`.
int drain_slices(int dflt);

// Whether the tensor-core update may run at all (not switched off).
bool enabled();

}  // namespace tc
}  // namespace jfg
