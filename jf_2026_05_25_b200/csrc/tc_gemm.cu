// tc_gemm.cu -- tensor-core Schur-complement update (3xTF32) for the mixed
// factor: U = -L21 L21^T for every front of a level, lower-triangular
// 128 x 128 tiles, on the sm_100a 5th-generation tensor cores.
//
// Per CTA (128 threads, one output tile):
//   * all threads stream K-slices of 16 columns of L21 from global memory
//     (column-major, coalesced along rows), split every value into
//     hi = tf32(v) and lo = tf32(v - hi), and store hi/lo of both operands
//     into shared memory in the no-swizzle K-major core-matrix layout
//     (8 rows x 16 bytes per core matrix);
//   * one thread issues tcgen05.mma kind::tf32 (M = N = 128, K = 8):
//     lo*hi + hi*lo + hi*hi accumulate in FP32 in tensor memory, and
//     tcgen05.commit arrives on the stage's mbarrier;
//   * two shared-memory stages: the loads of slice k+1 overlap the MMAs of
//     slice k; a stage is refilled only after its mbarrier has completed;
//   * every few K-slices the accumulator is read with tcgen05.ld (warp w
//     owns TMEM lanes 32w..32w+31 = tile rows) and added into an FP32
//     register row per thread; the epilogue writes -acc into the
//     column-major update matrix, lower triangle only.
// Every mbarrier wait is bounded (about two seconds of clock); on expiry the
// CTA records EE_TC_TIMEOUT in the device error record, waits (bounded) for
// its own MMAs, frees its tensor memory and returns.  No TMA and no cluster
// multicast are used.
#include "tc_gemm.cuh"

#include <cstdlib>

#include "jfg_internal.h"

namespace jfg {
namespace tc {
namespace {

constexpr int TM = 128;                        // tile rows (M) and columns (N)
constexpr int TK = 16;                         // K columns per shared-memory stage
constexpr int PART = TM * TK * 4;              // bytes of one operand part (hi or lo)
constexpr int NSPLIT = 2;                      // tf32 terms per operand value (hi, lo)
constexpr int STAGE = 2 * NSPLIT * PART;       // A_hi, A_lo, B_hi, B_lo
constexpr int NSTAGE = 2;
constexpr int SMEM_BYTES = NSTAGE * STAGE + 64;
constexpr uint32_t TMEM_COLS = 128;
// instruction descriptor: D f32, A/B tf32, both K-major, N = 128, M = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TM >> 3) << 17) |
                           ((uint32_t)(TM >> 4) << 24);
constexpr long long WAIT_CYCLES = 4000000000LL;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor, K-major without swizzle: core matrices of
// 8 rows x 16 bytes; 128 bytes between 8-row groups (SBO) and 2048 bytes
// between the two 16-byte K halves of one K = 8 instruction (LBO)
__device__ __forceinline__ uint64_t mat_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((2048u >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version for sm_100
  return d;
}

__device__ __forceinline__ float tf32_round(float v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return __uint_as_float(r);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  long long t0 = clock64();
  while (!mbar_try(bar, parity))
    if (clock64() - t0 > WAIT_CYCLES) return false;
  return true;
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// byte offset of element (row i, column k) inside one operand part
__device__ __forceinline__ uint32_t part_off(int i, int k) {
  return (uint32_t)(((k >> 2) * (TM / 8) + (i >> 3)) * 128 + (i & 7) * 16 + (k & 3) * 4);
}

// loads columns [k, k + TK) of rows [row, row + 128) of the column-major panel
// (rows past nrows or columns past kend read as zero), splits every value
// into hi = tf32(v) and lo = tf32(v - hi) and stores hi into the first part,
// lo into the second
__device__ __forceinline__ void load_split(const float* __restrict__ P, int64_t ld, int64_t row, int nrows,
                                           int k, int kend, unsigned char* parts) {
  const int t = threadIdx.x;   // one row per thread
  const bool rok = t < nrows;
#pragma unroll
  for (int q = 0; q < TK / 4; ++q) {
    float v[4], h[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      int kk = k + 4 * q + e;
      v[e] = (rok && kk < kend) ? P[row + t + ld * kk] : 0.0f;
      h[e] = tf32_round(v[e]);
      l[e] = tf32_round(v[e] - h[e]);
    }
    const uint32_t off = part_off(t, 4 * q);
    *reinterpret_cast<float4*>(parts + off) = make_float4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<float4*>(parts + PART + off) = make_float4(l[0], l[1], l[2], l[3]);
  }
}

__global__ void __launch_bounds__(128)
k_schur_tf32x3(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
               const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr,
               const int64_t* __restrict__ Uptr, const float* __restrict__ L, float* __restrict__ U,
               int drain, DevError* err) {
  const int s = list[blockIdx.y];
  const int c = first[s + 1] - first[s];
  const int m = mrows[s];
  const int r = m - c;
  if (r <= 0 || Uptr[s] < 0) return;
  const int nt = (r + TM - 1) / TM;
  // lower-triangular tile (ti, tj), tj <= ti, from the linear index
  int t = blockIdx.x;
  if (t >= nt * (nt + 1) / 2) return;
  int ti = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
  while (ti * (ti + 1) / 2 > t) --ti;
  while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
  const int tj = t - ti * (ti + 1) / 2;

  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + NSTAGE * STAGE);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + NSTAGE * STAGE + 32);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int q = 0; q < NSTAGE; ++q) mbar_init(smem_addr(&bars[q]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;

  const float* P = L + Lptr[s];
  const int64_t arow = (int64_t)c + (int64_t)ti * TM, brow = (int64_t)c + (int64_t)tj * TM;
  const int anr = min(TM, r - ti * TM), bnr = min(TM, r - tj * TM);
  const int nk = (c + TK - 1) / TK;
  bool ok = true;
  int issued = 0;   // K-slices whose MMAs were committed
  // FP32 accumulator of this thread's tile row: tensor memory is drained into
  // it every `drain` K-slices, so no tensor-memory sum runs over more than
  // drain * 16 products (the tensor-core accumulation is not round-to-nearest)
  float acc[TM];
#pragma unroll
  for (int j = 0; j < TM; ++j) acc[j] = 0.0f;
  int fresh = 1;    // the next MMA starts a new tensor-memory sum
  for (int kt = 0; kt < nk; ++kt) {
    const int stg = kt & 1;
    unsigned char* base = smem + stg * STAGE;
    if (kt >= NSTAGE) {
      // the MMAs that read this stage (slice kt - 2) must have completed
      if (!mbar_wait_bounded(smem_addr(&bars[stg]), (uint32_t)(((kt - NSTAGE) / NSTAGE) & 1))) ok = false;
    }
    if (__syncthreads_or(!ok)) { ok = false; break; }
    load_split(P, m, arow, anr, kt * TK, c, base);
    load_split(P, m, brow, bnr, kt * TK, c, base + NSPLIT * PART);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      fence_after();
      const uint32_t a0 = smem_addr(base), b0 = a0 + NSPLIT * PART;
#pragma unroll
      for (int q = 0; q < TK / 8; ++q) {
        const uint32_t o = (uint32_t)q * 2 * (TM / 8) * 128;
        // lo*hi + hi*lo + hi*hi (3xTF32), small terms first
        mma_tf32(tmem, mat_desc(a0 + PART + o), mat_desc(b0 + o), (fresh && q == 0) ? 0u : 1u);
        mma_tf32(tmem, mat_desc(a0 + o), mat_desc(b0 + PART + o), 1u);
        mma_tf32(tmem, mat_desc(a0 + o), mat_desc(b0 + o), 1u);
      }
      mma_commit(smem_addr(&bars[stg]));
    }
    issued = kt + 1;
    fresh = 0;
    if ((kt + 1) % drain == 0 || kt == nk - 1) {
      if (!mbar_wait_bounded(smem_addr(&bars[stg]), (uint32_t)((kt / NSTAGE) & 1))) ok = false;
      if (__syncthreads_or(!ok)) { ok = false; break; }
      fence_after();
      const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
      for (int j0 = 0; j0 < TM; j0 += 16) {
        uint32_t v[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(lane_base + (uint32_t)j0));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int e = 0; e < 16; ++e) acc[j0 + e] += __uint_as_float(v[e]);
      }
      fence_before();
      fresh = 1;
    }
  }
  // the last slice was drained inside the loop; after a timeout, wait
  // (bounded) for whatever MMAs were committed before freeing tensor memory
  if (!ok && issued > 0) {
    const int last = issued - 1;
    mbar_wait_bounded(smem_addr(&bars[last & 1]), (uint32_t)((last / NSTAGE) & 1));
  }
  if (!ok && threadIdx.x == 0 && atomicCAS(&err->code, 0, (int32_t)EE_TC_TIMEOUT) == 0) err->index = s;
  if (ok && issued == nk) {
    float* Ud = U + Uptr[s];
    const int li = warp * 32 + lane;              // row inside the tile
    const int64_t gi = (int64_t)ti * TM + li;     // row inside U
#pragma unroll
    for (int j = 0; j < TM; ++j) {
      const int64_t gj = (int64_t)tj * TM + j;
      if (li < anr && j < bnr && gi >= gj) Ud[gi + (int64_t)r * gj] = -acc[j];
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

}  // namespace

// Off unless JFG_TENSOR_CORES=1.  Measured on the 914k-DOF wing panel: the
// tensor-core update takes about as long as the SIMT FP32 kernel (its loads
// are the bottleneck, not the MMAs) and its FP32 accumulation in tensor
// memory is less accurate (a mixed-factor diagonal about 4x further from the
// FP64 one, even with a three-term split), so refinement needs more
// iterations (13 instead of 8).
bool enabled() {
  const char* e = std::getenv("JFG_TENSOR_CORES");
  return e && e[0] == '1';
}

bool schur_update_tf32x3(const int32_t* list, int count, const int32_t* first, const int32_t* mrows,
                         const int64_t* Lptr, const int64_t* Uptr, float* L, float* U, int max_r, int max_c,
                         DevError* err, cudaStream_t st) {
  (void)max_c;
  if (!enabled() || count <= 0 || max_r <= 0) return false;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_schur_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES) !=
        cudaSuccess)
      return false;
    attr = true;
  }
  const int nt = (max_r + TM - 1) / TM;
  const unsigned tiles = (unsigned)(nt * (nt + 1) / 2);
  const char* d = std::getenv("JFG_TC_DRAIN");
  int drain = d ? std::atoi(d) : 1;
  if (drain < 1) drain = 1 << 30;
  k_schur_tf32x3<<<dim3(tiles, (unsigned)count), 128, SMEM_BYTES, st>>>(list, first, mrows, Lptr, Uptr, L, U, drain,
                                                                      err);
  count_launch();
  return cudaGetLastError() == cudaSuccess;
}

}  // namespace tc
}  // namespace jfg
