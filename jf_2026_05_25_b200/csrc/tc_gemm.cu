// tc_gemm.cu -- tensor-core (tcgen05, kind::tf32) front updates of the
// mixed-precision supernodal factor: C -= A B^T on 128 x 128 tiles of the
// panel columns of a front (mode 0) and U = -L21 L21^T (mode 1), in 3xTF32
// split precision with FP32 accumulation.  Operands (packed hi/lo images
// written by the panel trsm) are streamed with bulk asynchronous copies
// (cp.async.bulk, global -> shared, no tensor maps, no cluster multicast)
// into a shared-memory ring; accumulators live in tensor memory and are
// drained into FP32 registers every K-slice.  Every wait is bounded.
#include "tc_gemm.cuh"

#include <cstdlib>

#include "jfg_internal.h"

namespace jfg {
namespace tc {
namespace {

constexpr long long WAIT_CYCLES = 4000000000LL;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
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


__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---------------------------------------------------------------------------
// Front updates of the mixed factor on the tensor cores.  The trsm kernel
// writes every FP32 panel value v a second time as hi = rn19(v) and
// lo = rn19(v - hi) into two packed operand arrays laid out as the shared-
// memory image the tensor core reads: per front, 512-byte atoms of 8 rows x
// 16 columns in the 64-byte-swizzled K-major layout, slice-block major, so
// that 128 rows of one 16-column K-slice are 8 KB of contiguous memory.
//
// One CTA per 128 x 128 output tile, warp-specialised:
//   * warps 0-7 (drain): warp w reads TMEM lanes 32(w%4).. +32 (tile rows)
//     and columns 64(w/4).. +64; every UDR K-slices of 16 columns are
//     accumulated by the tensor core into one of USL TMEM accumulators
//     (round robin, so the MMAs run up to USL - 1 uses ahead of the drain) and
//     added here into FP32 registers once complete, so the tensor core never
//     sums more than 16 UDR columns of products; the epilogue writes
//     C -= acc (mode 0, panel columns of the front) or C = -acc (mode 1,
//     the update matrix U), all loads of a column group before its stores;
//   * warp 8 (one thread): per K-slice 4 bulk copies (cp.async.bulk, no
//     multicast) of 8 KB (A hi, A lo, B hi, B lo) into a UST-stage ring,
//     completion counted in bytes on the stage's mbarrier;
//   * warp 9 (one thread): waits for a full stage and a free accumulator,
//     issues lo*hi + hi*lo + hi*hi (kind::tf32, M = N = 128, K = 8) and
//     commits to the stage's "empty" and the accumulator's "full" barriers.
// Tile origins are multiples of 8 rows: mode 1 (origin c) starts the tile
// grid c mod 8 rows early and stores nothing above row c.  Rows past the
// front come from stale shared memory or zeroed padding and reach only output
// rows that are not stored; columns past the K range are zeroed padding of
// the packed arrays (or an 8 KB zero page).
// Every wait is bounded (about two seconds of clock) and also gives up as
// soon as another warp has given up; the CTA then records EE_TC_TIMEOUT,
// waits (bounded) for its own copies and MMAs and frees its tensor memory.
constexpr int UM = TILE_M;
constexpr int UK = 16;
#ifndef JFG_TC_STAGES
#define JFG_TC_STAGES 4
#endif
constexpr int UST = JFG_TC_STAGES;
constexpr int UDW = 8;                          // drain warps: 4 lane quarters x 2 column halves
constexpr int UTHREADS = (UDW + 2) * 32;        // + producer warp + MMA warp
#ifndef JFG_TC_SLOTS
#define JFG_TC_SLOTS 4
#endif
constexpr int USL = JFG_TC_SLOTS;               // TMEM accumulators of 128 columns
constexpr uint32_t UTMEM = USL * UM;
// K-major, 64-byte swizzle: an 8-row x 16-column atom of 512 bytes, row i at
// i*64, its 16-byte chunk c (4 columns) at chunk position c ^ ((i >> 1) & 3);
// 16 atoms (128 rows) stacked 512 bytes apart (SBO) form one operand part
// of a K-slice.  The two K = 8 halves of a slice start 32 bytes apart.
constexpr int UPART = UM * UK * 4;
constexpr uint32_t U_LBO = 16, U_SBO = 512, U_KSTEP = 32;
constexpr uint64_t U_SWIZZLE_64B = 4;
constexpr int USTAGE = 4 * UPART;               // A hi, A lo, B hi, B lo
constexpr int UBAR = UST * USTAGE;
constexpr int USMEM = UBAR + 8 * (2 * UST + 2 * USL + 1) + 16;
constexpr uint32_t UIDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(UM >> 3) << 17) |
                            ((uint32_t)(UM >> 4) << 24);

__device__ __forceinline__ uint64_t u_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((U_LBO >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((U_SBO >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= U_SWIZZLE_64B << 61;
  return d;
}

__device__ __forceinline__ void u_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(UIDESC), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const float* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// bounded wait that also gives up once another warp has set *abort
__device__ __forceinline__ bool u_wait(uint32_t bar, uint32_t parity, volatile int* abort) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (*abort) return false;
    if (clock64() - t0 > WAIT_CYCLES) { *abort = 1; return false; }
  }
  return true;
}

__global__ void __launch_bounds__(UTHREADS, 1)
k_update_tf32x3(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
                const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr,
                const int64_t* __restrict__ Uptr, float* __restrict__ L, const float* __restrict__ Phi,
                const float* __restrict__ Plo, const int64_t* __restrict__ PKptr, const float* __restrict__ zero,
                float* __restrict__ U, int mode, int kbeg, int kend, int cend, int terms, int udr, DevError* err,
                const int2* __restrict__ tiles) {
  const int UDR = udr;   // K-slices of 16 summed by the tensor core per accumulator use
  int tq, tb;
  tile_of(tiles, tq, tb);
  const int s = list[tq];
  const int c = first[s + 1] - first[s];
  const int m = mrows[s];
  int row0, col0, nrow, ncol, kb, ke;
  float* C;
  int64_t ldc;
  if (mode == 0) {
    int k1 = min(kend, c);
    int ce = min(cend, c);
    if (kbeg >= c || k1 >= ce) return;
    row0 = k1; col0 = k1; nrow = m - k1; ncol = ce - k1; kb = kbeg; ke = k1;
    C = L + Lptr[s] + row0 + (int64_t)m * col0;
    ldc = m;
  } else {
    int r = m - c;
    if (r <= 0 || Uptr[s] < 0) return;
    row0 = c; col0 = c; nrow = r; ncol = r; kb = 0; ke = c;
    C = U + Uptr[s];
    ldc = r;
  }
  // tile grid from a row origin that is a multiple of 8 (row0 == col0)
  const int sh = row0 & 7;
  const int row0e = row0 - sh, col0e = col0 - sh, nrowe = nrow + sh, ncole = ncol + sh;
  const int ntj = (ncole + UM - 1) / UM, nti = (nrowe + UM - 1) / UM;
  const int t = tb;
  if (t >= nti * ntj) return;
  const int ti = t / ntj, tj = t % ntj;
  if (ti * UM + UM - 1 + row0e < tj * UM + col0e) return;   // strictly upper tile
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + UBAR);
  uint64_t* empty = full + UST;
  uint64_t* accfull = empty + UST;
  uint64_t* accempty = accfull + USL;
  uint64_t* spare = accempty + USL;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(spare + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int q = 0; q < UST; ++q) {
      mbar_init(smem_addr(&full[q]), 1);
      mbar_init(smem_addr(&empty[q]), 1);
    }
    mbar_init(smem_addr(spare), 1);
    for (int q = 0; q < USL; ++q) {
      mbar_init(smem_addr(&accfull[q]), 1);
      mbar_init(smem_addr(&accempty[q]), UDW * 32);
    }
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(UTMEM)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  const int nk = (ke - kb + UK - 1) / UK;
  const uint32_t sbase = smem_addr(smem);

  if (warp == UDW) {
    // ---------------------------------------------------------- producer
    if (lane == 0) {
      const int64_t pk = PKptr[s], nrg = (m + 7) / 8;
      const int64_t rga = (row0e + (int64_t)ti * UM) >> 3, rgb = (col0e + (int64_t)tj * UM) >> 3;
      const uint32_t na = (uint32_t)min((int64_t)16, nrg - rga) * 512u;
      const uint32_t nb = (uint32_t)min((int64_t)16, nrg - rgb) * 512u;
      int issued = 0;
      for (int j = 0; j < nk; ++j) {
        const int st = j % UST, n = j / UST;
        if (n >= 1 && !u_wait(smem_addr(&empty[st]), (uint32_t)((n - 1) & 1), abort)) break;
        const uint32_t dst = sbase + (uint32_t)(st * USTAGE), bar = smem_addr(&full[st]);
        const int64_t sb = (kb + j * UK) >> 4;   // 16-column slice block
        if (16 * sb < ke) {
          const int64_t oa = pk + (sb * nrg + rga) * 128, ob = pk + (sb * nrg + rgb) * 128;
          mbar_expect_tx(bar, 2 * (na + nb));
          bulk_load(dst, Phi + oa, na, bar);
          bulk_load(dst + UPART, Plo + oa, na, bar);
          bulk_load(dst + 2 * UPART, Phi + ob, nb, bar);
          bulk_load(dst + 3 * UPART, Plo + ob, nb, bar);
        } else {   // columns past the K range: zeros
          mbar_expect_tx(bar, 4 * UPART);
#pragma unroll
          for (int q = 0; q < 4; ++q) bulk_load(dst + q * UPART, zero, UPART, bar);
        }
        issued = j + 1;
      }
      if (issued < nk && issued > 0) {
        // gave up: let every copy still in flight land before the CTA exits.
        // The last UST issued slices are the latest use of each stage; wait
        // for each at its own phase (bounded; a phase already complete
        // returns at once)
        for (int l = max(0, issued - UST); l < issued; ++l) {
          const long long t0 = clock64();
          while (!mbar_try(smem_addr(&full[l % UST]), (uint32_t)((l / UST) & 1)) && clock64() - t0 < WAIT_CYCLES) {
          }
        }
      }
    }
    __syncwarp();
  } else if (warp == UDW + 1) {
    // ---------------------------------------------------------- MMA issue
    if (lane == 0) {
      int issued = 0;
      for (int j = 0; j < nk; ++j) {
        const int st = j % UST, n = j / UST, use = j / UDR, slot = use % USL, q = use / USL;
        const bool first_of_use = (j % UDR) == 0, last_of_use = (j % UDR) == UDR - 1 || j == nk - 1;
        if (!u_wait(smem_addr(&full[st]), (uint32_t)(n & 1), abort)) break;
        if (first_of_use && q >= 1 && !u_wait(smem_addr(&accempty[slot]), (uint32_t)((q - 1) & 1), abort)) break;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        fence_after();
        const uint32_t a_hi = sbase + (uint32_t)(st * USTAGE), a_lo = a_hi + UPART;
        const uint32_t b_hi = a_hi + 2 * UPART, b_lo = a_hi + 3 * UPART;
        const uint32_t d = tmem + (uint32_t)(slot * UM);
#pragma unroll
        for (int kq = 0; kq < UK / 8; ++kq) {
          const uint32_t o = (uint32_t)kq * U_KSTEP;
          u_mma(d, u_desc(a_lo + o), u_desc(b_hi + o), (first_of_use && kq == 0) ? 0u : 1u);
          u_mma(d, u_desc(a_hi + o), u_desc(b_lo + o), 1u);
          u_mma(d, u_desc(a_hi + o), u_desc(b_hi + o), 1u);
          if (terms > 3) u_mma(d, u_desc(a_lo + o), u_desc(b_lo + o), 1u);
        }
        mma_commit(smem_addr(&empty[st]));
        if (last_of_use) mma_commit(smem_addr(&accfull[slot]));
        issued = j + 1;
      }
      if (issued < nk && issued > 0) {
        // gave up: let the MMAs already issued finish before TMEM is freed
        mma_commit(smem_addr(spare));
        const long long t0 = clock64();
        while (!mbar_try(smem_addr(spare), 0u) && clock64() - t0 < WAIT_CYCLES) {
        }
      }
    }
    __syncwarp();
  } else {
    // ---------------------------------------------------------- drain + epilogue
    constexpr int HC = UM / 2;
    float acc[HC];
#pragma unroll
    for (int jj = 0; jj < HC; ++jj) acc[jj] = 0.0f;
    const uint32_t tlane = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)((warp >> 2) * HC);
    const int nuse = (nk + UDR - 1) / UDR;
    int drained = 0;
    for (int u = 0; u < nuse; ++u) {
      const int slot = u % USL, q = u / USL;
      bool ok = lane == 0 ? u_wait(smem_addr(&accfull[slot]), (uint32_t)(q & 1), abort) : true;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      fence_after();
      const uint32_t tb = tlane + (uint32_t)(slot * UM);
#pragma unroll
      for (int j0 = 0; j0 < HC; j0 += 32) {
        uint32_t v[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(tb + (uint32_t)j0));
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
              "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
            : "r"(tb + (uint32_t)(j0 + 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int e = 0; e < 32; ++e) acc[j0 + e] += __uint_as_float(v[e]);
      }
      fence_before();
      mbar_arrive(smem_addr(&accempty[slot]));
      drained = u + 1;
    }
    if (drained == nuse && nk > 0) {
      // this thread's row of the tile and columns j0g .. j0g + HC - 1 (front
      // coordinates relative to C); stored are rows in [0, nrow) and columns
      // in [0, ncol) on or below the front's diagonal.  All loads of a
      // 16-column group are issued before its stores.
      const int64_t gi = (int64_t)ti * UM + (warp & 3) * 32 + lane - sh;
      const int64_t j0g = (int64_t)tj * UM + (warp >> 2) * HC - sh;
      const int64_t jfirst = -j0g;
      const int64_t jlast = min((int64_t)ncol - 1, row0 + gi - col0) - j0g;
      if (gi >= 0 && gi < nrow && jlast >= 0) {
#pragma unroll
        for (int h = 0; h < HC; h += 16) {
          if (mode == 0) {
            float cv[16];
#pragma unroll
            for (int e = 0; e < 16; ++e)
              cv[e] = (h + e >= jfirst && h + e <= jlast) ? C[gi + ldc * (j0g + h + e)] : 0.0f;
#pragma unroll
            for (int e = 0; e < 16; ++e)
              if (h + e >= jfirst && h + e <= jlast) C[gi + ldc * (j0g + h + e)] = cv[e] - acc[h + e];
          } else {
#pragma unroll
            for (int e = 0; e < 16; ++e)
              if (h + e >= jfirst && h + e <= jlast) C[gi + ldc * (j0g + h + e)] = -acc[h + e];
          }
        }
      }
    }
  }
  fence_before();
  __syncthreads();
  if (tid == 0 && *abort && atomicCAS(&err->code, 0, (int32_t)EE_TC_TIMEOUT) == 0) err->index = s;
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(UTMEM) : "memory");
  }
}

}  // namespace

int setting() {
  const char* e = std::getenv("JFG_TENSOR_CORES");
  if (!e || !e[0]) return -1;
  return e[0] == '0' ? 0 : 1;
}

bool enabled() { return setting() != 0; }

int drain_slices(int dflt) {
  const char* de = std::getenv("JFG_TC_DRAIN");
  int v = de ? std::atoi(de) : dflt;
  return v < 1 ? 1 : (v > 16 ? 16 : v);
}

bool front_update_tf32x3(const int32_t* list, const int2* tiles, int n_tiles, const int32_t* first,
                         const int32_t* mrows, const int64_t* Lptr, const int64_t* Uptr, float* L, const float* Phi,
                         const float* Plo, const int64_t* PKptr, const float* zero, float* U, int mode, int kbeg,
                         int kend, int cend, int drain, DevError* err, cudaStream_t st) {
  if (!enabled() || !Phi || !Plo || !PKptr || !zero || !tiles) return false;
  if (n_tiles <= 0) return true;   // no front of the level has output here
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_update_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize, USMEM) != cudaSuccess)
      return false;
    attr = true;
  }
  const char* te = std::getenv("JFG_TC_TERMS");   // 4: add lo*lo
  const int terms = (te && te[0] == '4') ? 4 : 3;
  const int udr = drain < 1 ? 1 : (drain > 16 ? 16 : drain);
  k_update_tf32x3<<<(unsigned)n_tiles, UTHREADS, USMEM, st>>>(
      list, first, mrows, Lptr, Uptr, L, Phi, Plo, PKptr, zero, U, mode, kbeg, kend, cend, terms, udr, err, tiles);
  count_launch();
  return cudaGetLastError() == cudaSuccess;
}

}  // namespace tc
}  // namespace jfg
