// factor.cu -- supernodal multifrontal Cholesky of K_ff on the device,
// level-scheduled triangular solves and FP64 iterative refinement.
//
// Replaces cholesky(Symmetric(K_ff)) and F \ f of
// src/solver/boundary_conditions.jl:1656-1714 (and the cached re-solve
// :1418-1477).  Fronts are processed one elimination-tree level at a time,
// leaves first; every front of a level is factored by the same sequence of
// batched kernels (diagonal-block Cholesky, panel triangular solve, panel
// update, Schur-complement update).  Children hand their update matrices to
// the parent by an extend-add launched once per child rank, so no two writers
// ever touch one entry: the factor is bitwise deterministic.
//
// Precision: FP64 (plain path) or FP32 storage with symmetric diagonal
// scaling (mixed path); the mixed factor is the preconditioner of an FP64
// iterative refinement on the FP64 CSC matrix.
#include <algorithm>
#include <climits>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>

#include "jfg_internal.h"
#include "tc_gemm.cuh"

struct NumericFactor {
  // symbolic arrays on the device
  int32_t *first = nullptr, *mrows = nullptr, *level_sn = nullptr, *ea_child = nullptr, *rel = nullptr,
          *rows = nullptr, *parent = nullptr, *perm_dof = nullptr, *amap_src = nullptr,
          *amap_pr = nullptr, *amap_pc = nullptr;
  int64_t *Lptr = nullptr, *Uptr = nullptr, *rows_ptr = nullptr, *relptr = nullptr, *amap_dst = nullptr;
  int64_t n_amap = 0;
  const int32_t* level_sn_cur = nullptr;   // the level the factor loop is on
  // CUDA graphs of the factorisation (per precision) and of one preconditioner
  // application (per precision and right-hand-side count 1..32)
  cudaGraphExec_t factor_graph[2] = {nullptr, nullptr};
  int64_t factor_graph_nodes[2] = {0, 0};
  int factor_calls[2] = {0, 0};
  cudaGraphExec_t solve_graph[2][33] = {};
  int64_t solve_graph_nodes[2][33] = {};
  // host launch metadata
  struct Level {
    int32_t off, count;
    int32_t max_c, max_m, max_r;
    std::vector<std::pair<int32_t, int32_t>> ea;   // (offset into ea_child, count), per child rank
    int32_t ea_max_r;
    double schur_flops;   // sum over fronts of r(r+1) c (lower SYRK, 2 flops per FMA)
    int64_t pk_len = 0;   // floats of the packed tensor-core operand images of the level's fronts
    int64_t nnz = 0;      // factor entries of the level's fronts (sum of m c)
    // the level's fronts are listed by decreasing width: cs[i] is the width
    // of the i-th, pm[i] the largest row count among the first i + 1
    std::vector<int32_t> cs, pm;
    // fronts wider than kmin (a prefix of the list)
    int active(int kmin) const {
      return (int)(std::upper_bound(cs.begin(), cs.end(), kmin, std::greater<int32_t>()) - cs.begin());
    }
    int maxm(int na) const { return na > 0 ? pm[na - 1] : 0; }
    // tile lists (offset, count into NumericFactor::tiles) of the level's launches
    struct Span { int64_t off = 0; int32_t cnt = 0; };
    std::vector<Span> ea_f, ea_s;     // factor / solve extend-add, per child-rank segment
    std::vector<Span> trsm;           // panel trsm, per 64-column step
    struct StripSpans { Span diag, upd32, upd128, bwd; };
    std::vector<StripSpans> strips;   // solve sweeps, per 256-column strip
    // front updates: lower output tiles of 64 (SIMT / DMMA) and of 128
    // (tensor cores), as (position, ti * ntj + tj) of each front's grid
    struct UpdSpans { Span t64, t128; };
    std::vector<UpdSpans> upd_step;    // inside the super-panel, per 64-column step
    std::vector<UpdSpans> upd_trail;   // after the super-panel, per super-panel
    UpdSpans schur;                    // U = -L21 L21^T
  };
  std::vector<Level> levels;
  int2* tiles = nullptr;      // every level launch's work tiles (see tile_of)
  int64_t n_tiles = 0;
  // factor storage
  double* L64 = nullptr;
  double* U64 = nullptr;
  float* L32 = nullptr;
  // tensor-core operand copies of L32 (mixed factor with tcgen05 updates):
  // hi = rn19(v), lo = rn19(v - hi), packed per front (offset PKptr[s]) in
  // 512-byte 64-byte-swizzled atoms of 8 rows x 16 columns, slice-block
  // major.  The images are only read by the updates of the front's own level,
  // so one workspace sized for the largest level serves every level: PKptr[s]
  // is the front's offset inside its level's region, which is zeroed (the
  // padding must read as zero) before the level's panels write it.
  // tc_zero: 8 KB of zeros.
  float *Phi = nullptr, *Plo = nullptr, *tc_zero = nullptr;
  int64_t* PKptr = nullptr;
  int64_t pk_len = 0;
  int tc_drain = 1;           // K-slices per tensor-memory accumulator use
  float* U32 = nullptr;
  double* scale = nullptr;    // n, symmetric diagonal scaling of the mixed factor
  // inverse diagonal blocks of the strip solve
  int64_t dinv_len = 0, part_len = 0;
  int64_t *Dptr = nullptr, *part_off = nullptr;
  double* Dinv64 = nullptr;
  float* Dinv32 = nullptr;
  // inverses of the 256-column strip diagonal blocks (solve only)
  int64_t sinv_len = 0, n_inv_items = 0;
  int64_t* Sptr = nullptr;
  int32_t *inv_sn = nullptr, *inv_kb = nullptr, *inv_jb = nullptr;
  double* Sinv64 = nullptr;
  float* Sinv32 = nullptr;
  double* part = nullptr;
  bool have64 = false, have32 = false;
  bool prefer_mixed = false;   // solve with the mixed factor when both exist
  // solve workspace
  int nrhs_cap = 0;
  double *xp = nullptr, *tt = nullptr, *V = nullptr, *dF = nullptr, *dU = nullptr, *dR = nullptr, *dD = nullptr;
  double *dZ = nullptr, *dP = nullptr, *dQ = nullptr;
  uint8_t* free_mask = nullptr;
  double *norms = nullptr;
  int64_t v_total = 0;
  jfg::DevError* err = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

#define JFG_CUDA_VOID(x) (void)(x)

namespace jfg {
namespace {

// fine-grained per-kernel-class event brackets (profiling level 2, or
// JFG_FINE_PROFILE=1 with profiling on)
inline bool fine_prof() {
  static int v = -1;
  if (v < 0) v = std::getenv("JFG_FINE_PROFILE") ? 1 : 0;
  return profiling_level() >= 2 || (v == 1 && profiling_enabled());
}

// Launch-bound sequences (the level loop of the factorisation, the level and
// strip loop of a preconditioner application) are captured once into a CUDA
// graph and replayed: one graph launch instead of hundreds of kernel launches.
// JFG_GRAPHS=0 or kernel-class profiling runs them eagerly.
inline bool graphs_enabled() {
  const char* e = std::getenv("JFG_GRAPHS");
  return !(e && e[0] == '0') && !profiling_enabled();
}

template <typename Fn>
jfg_status run_graph(cudaGraphExec_t& ge, int64_t& nodes, cudaStream_t st, Fn&& body) {
  if (!ge) {
    const int64_t c0 = launch_count();
    cudaGraph_t g = nullptr;
    JFG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    jfg_status s = body();
    cudaError_t e = cudaStreamEndCapture(st, &g);
    const int64_t k = launch_count() - c0;
    count_launch(-(int)k);   // nothing ran while capturing
    if (s != JFG_OK || e != cudaSuccess || g == nullptr) {
      if (g) cudaGraphDestroy(g);
      (void)cudaGetLastError();
      return body();          // run eagerly instead
    }
    e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      ge = nullptr;
      (void)cudaGetLastError();
      return body();
    }
    nodes = k;
  }
  JFG_CUDA(cudaGraphLaunch(ge, st));
  count_launch((int)nodes);
  return JFG_OK;
}

void drop_solve_graphs(NumericFactor* F) {
  for (auto& row : F->solve_graph)
    for (auto& g : row)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

constexpr int NB = 64;       // panel block width
constexpr int MAXR = 32;     // right-hand sides per solve sweep (one read of the factor serves all)
constexpr int TILE = 64;     // Schur-update tile
// super-panel width of the blocked front factorisation (multiple of NB):
// JFG_PANEL_WIDTH, default 256
inline int panel_width() {
  static int v = -1;
  if (v < 0) {
    const char* e = std::getenv("JFG_PANEL_WIDTH");
    int w = e ? std::atoi(e) : 256;
    w = std::max(64, std::min(2048, (w / 64) * 64));
    v = w;
  }
  return v;
}


__device__ inline void rec_err(DevError* e, int32_t code, int64_t idx) {
  if (atomicCAS(&e->code, 0, code) == 0) e->index = idx;
}

template <typename T>
__global__ void k_scatter_A(int64_t na, const int32_t* __restrict__ src, const int64_t* __restrict__ dst,
                            const int32_t* __restrict__ pr, const int32_t* __restrict__ pc,
                            const double* __restrict__ nzval, const double* __restrict__ scale, T* __restrict__ L) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= na) return;
  double v = nzval[src[k]];
  if (scale) v = v * scale[pr[k]] * scale[pc[k]];
  L[dst[k]] = (T)v;
}

// (permuted row, permuted column) of each K_ff entry's front slot d: the
// owning supernode s is the last with Lptr[s] <= d; the slot is row
// (d - Lptr[s]) mod m_s, column (d - Lptr[s]) div m_s of its front
__global__ void k_amap_rowcol(int64_t na, int64_t ns, const int64_t* __restrict__ dst, const int64_t* __restrict__ Lptr,
                              const int32_t* __restrict__ mrows, const int64_t* __restrict__ rows_ptr,
                              const int32_t* __restrict__ rows, const int32_t* __restrict__ first,
                              int32_t* __restrict__ pr, int32_t* __restrict__ pc) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= na) return;
  const int64_t d = dst[q];
  int64_t lo = 0, hi = ns;   // upper_bound(Lptr[0..ns], d) - 1
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (Lptr[mid] <= d) lo = mid + 1; else hi = mid;
  }
  const int64_t s = lo - 1;
  const int64_t mm = mrows[s], off = d - Lptr[s];
  pr[q] = rows[rows_ptr[s] + off % mm];
  pc[q] = first[s] + (int32_t)(off / mm);
}

__global__ void k_diag_scale(int64_t n, const int32_t* __restrict__ perm_dof, const int64_t* __restrict__ diag_pos,
                             const double* __restrict__ nzval, double* __restrict__ scale) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int64_t p = diag_pos[perm_dof[k]];
  double d = p >= 0 ? fabs(nzval[p]) : 0.0;
  scale[k] = d > 0.0 ? 1.0 / sqrt(d) : 1.0;
}

// Extend-add of child update matrices into their parents' fronts.  One launch
// covers the children of one rank, so each parent receives one child.
template <typename T>
__global__ void k_extend_add(const int32_t* __restrict__ child, const int32_t* __restrict__ first,
                             const int32_t* __restrict__ mrows, const int32_t* __restrict__ parent,
                             const int64_t* __restrict__ Lptr, const int64_t* __restrict__ Uptr,
                             const int64_t* __restrict__ relptr, const int32_t* __restrict__ rel,
                             T* __restrict__ L, T* __restrict__ U, int pass, const int2* __restrict__ tiles) {
  int tq, tb;
  tile_of(tiles, tq, tb);
  int ch = child[tq];
  int64_t uc = Uptr[ch];
  if (uc < 0) return;
  int rc = mrows[ch] - (first[ch + 1] - first[ch]);
  int cb = tb * 8 + (threadIdx.x >> 5);   // one warp per child column
  if (cb >= rc) return;
  int lane = threadIdx.x & 31;
  int p = parent[ch];
  int cp = first[p + 1] - first[p];
  int mp = mrows[p];
  int rp = mp - cp;
  const int32_t* rl = rel + relptr[ch];
  int rb = rl[cb];
  if ((pass == 0) != (rb < cp)) return;
  const T* src = U + uc + (int64_t)rc * cb;
  T* dst = rb < cp ? L + Lptr[p] + (int64_t)mp * rb : U + Uptr[p] + (int64_t)rp * (rb - cp) - cp;
  // groups of 8 entries per lane: every load of a group (map, source,
  // destination) is issued before its stores
  for (int a0 = cb + lane; a0 < rc; a0 += 32 * 8) {
    int idx[8];
    T sv[8], dv[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      int a = a0 + 32 * u;
      idx[u] = a < rc ? rl[a] : -1;
      sv[u] = a < rc ? src[a] : (T)0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) dv[u] = idx[u] >= 0 ? dst[idx[u]] : (T)0;
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (idx[u] >= 0) dst[idx[u]] = dv[u] + sv[u];
  }
}

// 32 x 32 Cholesky of A[o..o+31][o..o+31] and its inverse into B, by one warp
// (warp-synchronous, no block barrier).  Lane i holds row o+i in registers;
// the factor runs on unscaled columns (a_ik -= a_ij a_kj / a_jj, the L D L^T
// form) and scales column k by 1/sqrt(a_kk) at the end.  The inverse is
// right-looking by rows with lane j holding column o+j of X = L^{-1}.
// Pivots that are not positive and finite are replaced by 1 and the smallest
// such column index is recorded in *bad_idx.
// Not inlined: the two calls of k_potrf_diag share one copy of this long,
// fully unrolled body (the kernel runs one CTA per front and is bound by
// its serial chain, where instruction-cache misses showed as stalls).
template <typename T>
__device__ __noinline__ void chol32_inv(T (*A)[NB + 1], T (*B)[NB + 1], T* sv, T* pv, int o, int kn,
                                        int* bad_idx) {
  const int lane = threadIdx.x & 31;
  const int gi = o + lane;
  T a[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) a[k] = (k <= lane) ? A[gi][o + k] : (T)0;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    T d = __shfl_sync(0xffffffffu, a[j], j);
    T* s = sv + (j & 1) * 32;
    s[lane] = a[j];
    if (lane == 0) pv[j] = d;
    bool bad = !(d > (T)0) || !isfinite((double)d);
    T rd = bad ? (T)1 : (T)1 / d;
    T lj = (lane > j) ? a[j] * rd : (T)0;
    __syncwarp();
#pragma unroll
    for (int k = j + 1; k < 32; ++k) a[k] = fma(-lj, s[k], a[k]);
  }
  __syncwarp();
  {
    T p = pv[lane];
    bool bad = !(p > (T)0) || !isfinite((double)p);
    if (bad && gi < kn) atomicMin(bad_idx, gi);
    T sq = bad ? (T)1 : sqrt(p);
    sv[lane] = (T)1 / sq;
    sv[32 + lane] = sq;
  }
  __syncwarp();
#pragma unroll
  for (int k = 0; k < 32; ++k) A[gi][o + k] = (k < lane) ? a[k] * sv[k] : (k == lane ? sv[32 + k] : (T)0);
  __syncwarp();
  T x[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) x[i] = (i == lane) ? (T)1 : (T)0;
#pragma unroll
  for (int l = 0; l < 32; ++l) {
    x[l] = x[l] * sv[l];
#pragma unroll
    for (int i = l + 1; i < 32; ++i) x[i] = fma(-A[o + i][o + l], x[l], x[i]);
  }
#pragma unroll
  for (int i = 0; i < 32; ++i) B[o + i][gi] = (i >= lane) ? x[i] : (T)0;
}

template <typename T>
constexpr int potrf_smem() { return (2 * NB * (NB + 1) + 2 * NB) * (int)sizeof(T); }

// Cholesky of the NB x NB diagonal block at column k0 of every front of the
// level, and the inverse of the factor block (kept for the panel triangular
// solve and for the forward/backward solves).  The block is split 2 x 2 into
// 32 x 32 tiles: L11 and X11 = L11^{-1} by one warp, L21 = A21 X11^T and
// A22 -= L21 L21^T by the whole CTA, L22 and X22 by one warp, then
// X21 = -X22 (L21 X11).  Rows and columns past the front's width are padded
// with the identity so the tiles are always full.
template <typename T>
__global__ void __launch_bounds__(256)
k_potrf_diag(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
             const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr,
             const int64_t* __restrict__ Dptr, T* __restrict__ L, T* __restrict__ Dinv, int k0, DevError* err) {
  int s = list[blockIdx.x];
  int c = first[s + 1] - first[s];
  if (k0 >= c) return;
  int m = mrows[s];
  int kn = min(NB, c - k0);
  extern __shared__ unsigned char smem_raw[];
  T (*A)[NB + 1] = reinterpret_cast<T (*)[NB + 1]>(smem_raw);
  T (*B)[NB + 1] = A + NB;
  T* sv = reinterpret_cast<T*>(B + NB);  // 64 entries of broadcast scratch
  T* pv = sv + 64;                       // 32 pivots
  __shared__ int bad_idx;
  T* P = L + Lptr[s] + k0 + (int64_t)m * k0;
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  if (t == 0) bad_idx = NB;
  // 256 threads: all 16 loads of a thread in flight together
#pragma unroll
  for (int u = 0; u < NB * NB / 256; ++u) {
    int e = t + 256 * u;
    int i = e & (NB - 1), j = e >> 6;
    A[i][j] = (i < kn && j < kn) ? (i >= j ? P[i + (int64_t)m * j] : (T)0) : (i == j ? (T)1 : (T)0);
  }
  __syncthreads();
  if (w == 0) chol32_inv<T>(A, B, sv, pv, 0, kn, &bad_idx);
  __syncthreads();
  if (kn > 32) {
    const int i = 32 + lane;
    T acc[4] = {0, 0, 0, 0};
    // L21 = A21 X11^T  (thread: row i, columns w + 8q)
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
      T av = A[i][k];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fma(av, B[w + 8 * q][k], acc[q]);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) A[i][w + 8 * q] = acc[q];
    __syncthreads();
    // A22 -= L21 L21^T, lower triangle
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = 0;
#pragma unroll 8
    for (int j = 0; j < 32; ++j) {
      T lv = A[i][j];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fma(lv, A[32 + w + 8 * q][j], acc[q]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int k = 32 + w + 8 * q;
      if (k <= i) A[i][k] -= acc[q];
    }
    __syncthreads();
    if (w == 0) chol32_inv<T>(A, B, sv, pv, 32, kn, &bad_idx);
    __syncthreads();
    // Tm = L21 X11 into the unused upper-right tile of B
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = 0;
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
      T lv = A[i][k];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fma(lv, B[k][w + 8 * q], acc[q]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) B[lane][32 + w + 8 * q] = acc[q];
    __syncthreads();
    // X21 = -X22 Tm
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = 0;
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
      T xv = B[i][32 + k];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fma(xv, B[k][32 + w + 8 * q], acc[q]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) B[i][w + 8 * q] = -acc[q];
    __syncthreads();
  }
  if (t == 0 && bad_idx < kn) rec_err(err, EE_PIVOT, (int64_t)first[s] + k0 + bad_idx);
  T* Dv = Dinv + Dptr[s] + (int64_t)(k0 / NB) * NB * NB;
  for (int e = t; e < NB * NB; e += blockDim.x) {
    int i = e & (NB - 1), j = e >> 6;
    bool in = i < kn && j < kn && i >= j;
    if (in) P[i + (int64_t)m * j] = A[i][j];
    Dv[i + NB * j] = in ? B[i][j] : (T)0;
  }
}

// Cholesky of the NB x NB diagonal block at column k0 of every front of the
// level and the inverse of its factor, with the whole CTA on both serial
// chains.  Each thread owns up to 9 entries of the 64 x 64 lower triangle.
// Factor: right-looking on unscaled columns (a_ik -= a_ij a_kj / a_jj for
// j < k <= i, the L D L^T form), one block barrier per column, and the
// columns scaled by 1/sqrt(a_jj) at the end.  Inverse: X = L^{-1} by rows,
// right-looking on the residual R (R_iq -= L_ij R_jq / L_jj for q <= j < i),
// one barrier per row, X_iq = R_iq / L_ii at the end.  Both chains stop at
// the block's width kn.  Pivots that are not positive and finite are
// replaced by 1 and the smallest such column is recorded; rows and columns
// past the front's width are the identity.
template <typename T>
__global__ void __launch_bounds__(256, 2)
k_potrf_cta(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
            const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr,
            const int64_t* __restrict__ Dptr, T* __restrict__ L, T* __restrict__ Dinv, int k0, DevError* err) {
  int s = list[blockIdx.x];
  int c = first[s + 1] - first[s];
  if (k0 >= c) return;
  int m = mrows[s];
  int kn = min(NB, c - k0);
  extern __shared__ unsigned char smem_raw[];
  T (*A)[NB + 1] = reinterpret_cast<T (*)[NB + 1]>(smem_raw);
  T (*B)[NB + 1] = A + NB;
  T* sv = reinterpret_cast<T*>(B + NB);   // 64 entries: sqrt of the pivots
  __shared__ int bad_idx;
  T* P = L + Lptr[s] + k0 + (int64_t)m * k0;
  const int t = threadIdx.x;
  if (t == 0) bad_idx = NB;
#pragma unroll
  for (int u = 0; u < NB * NB / 256; ++u) {
    int e = t + 256 * u;
    int i = e & (NB - 1), j = e >> 6;
    A[i][j] = (i < kn && j < kn) ? (i >= j ? P[i + (int64_t)m * j] : (T)0) : (i == j ? (T)1 : (T)0);
    B[i][j] = (i == j) ? (T)1 : (T)0;
  }
  // this thread's lower-triangle entries (row-major enumeration, 2080 in all)
  constexpr int NE = 9;
  int ei[NE], ek[NE];
#pragma unroll
  for (int u = 0; u < NE; ++u) {
    int e = t + 256 * u;
    if (e < NB * (NB + 1) / 2) {
      int i = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
      while ((i + 1) * (i + 2) / 2 <= e) ++i;
      while (i * (i + 1) / 2 > e) --i;
      ei[u] = i;
      ek[u] = e - i * (i + 1) / 2;
    }
    if (e >= NB * (NB + 1) / 2 || ei[u] >= kn) {
      // no entry, or one of the identity rows past the block's width (they
      // never change): every predicate below is false for (-1, -1)
      ei[u] = -1;
      ek[u] = -1;
    }
  }
  // factor.  Each thread keeps its entries in registers; an entry reaches
  // shared memory when its column becomes the next pivot column (final after
  // the update by the column before it), so a step reads only final values
  // and all its loads are independent of its stores (they issue together).
  T av[NE];
  __syncthreads();
#pragma unroll
  for (int u = 0; u < NE; ++u) av[u] = ei[u] >= 0 ? A[ei[u]][ek[u]] : (T)0;
  for (int j = 0; j < kn; ++j) {
    __syncthreads();   // column j final in shared memory
    T d = A[j][j];
    const bool bad = !(d > (T)0) || !isfinite((double)d);
    if (bad) {
      if (t == 0) atomicMin(&bad_idx, j);
      d = (T)1;
    }
    const T rd = (T)1 / d;
    T lij[NE], lkj[NE];
#pragma unroll
    for (int u = 0; u < NE; ++u)
      if (ek[u] > j) { lij[u] = A[ei[u]][j]; lkj[u] = A[ek[u]][j]; }
#pragma unroll
    for (int u = 0; u < NE; ++u)
      if (ek[u] > j) av[u] = fma(-lij[u] * rd, lkj[u], av[u]);
#pragma unroll
    for (int u = 0; u < NE; ++u)
      if (ek[u] == j + 1) A[ei[u]][j + 1] = av[u];
  }
  __syncthreads();
  if (t < NB) {
    T d = A[t][t];
    const bool bad = !(d > (T)0) || !isfinite((double)d);
    sv[t] = bad ? (T)1 : sqrt(d);
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < NE; ++u) {
    const int i = ei[u], k = ek[u];
    if (i >= 0) A[i][k] = (i == k) ? sv[k] : A[i][k] / sv[k];
  }
  // inverse of the factor, the same way: a row of B reaches shared memory
  // when it becomes final (after the step of the row before it)
  T bv[NE];
#pragma unroll
  for (int u = 0; u < NE; ++u) bv[u] = (ei[u] >= 0 && ei[u] == ek[u]) ? (T)1 : (T)0;
  for (int j = 0; j < kn; ++j) {
    __syncthreads();   // row j of B final; the scaled factor visible
    const T rl = (T)1 / A[j][j];
    T lij[NE], bjq[NE];
#pragma unroll
    for (int u = 0; u < NE; ++u)
      if (ek[u] <= j && ei[u] > j) { lij[u] = A[ei[u]][j]; bjq[u] = B[j][ek[u]]; }
#pragma unroll
    for (int u = 0; u < NE; ++u)
      if (ek[u] <= j && ei[u] > j) bv[u] = fma(-lij[u] * rl, bjq[u], bv[u]);
#pragma unroll
    for (int u = 0; u < NE; ++u)
      if (ei[u] == j + 1 && ek[u] <= j + 1) B[j + 1][ek[u]] = bv[u];
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < NE; ++u) {
    const int i = ei[u], q = ek[u];
    if (i >= 0) B[i][q] = B[i][q] / A[i][i];
  }
  __syncthreads();
  if (t == 0 && bad_idx < kn) rec_err(err, EE_PIVOT, (int64_t)first[s] + k0 + bad_idx);
  T* Dv = Dinv + Dptr[s] + (int64_t)(k0 / NB) * NB * NB;
  for (int e = t; e < NB * NB; e += blockDim.x) {
    int i = e & (NB - 1), j = e >> 6;
    bool in = i < kn && j < kn && i >= j;
    if (in) P[i + (int64_t)m * j] = A[i][j];
    Dv[i + NB * j] = in ? B[i][j] : (T)0;
  }
}

// JFG_POTRF=1 selects the earlier diagonal-block kernel (one warp per 32 x 32
// tile); the default runs the CTA-wide chains above
inline bool potrf_cta() {
  static int v = -1;
  if (v < 0) {
    const char* e = std::getenv("JFG_POTRF");
    v = (e && e[0] == '1') ? 0 : 1;
  }
  return v == 1;
}

// rows [k1, m) of panel columns [k0, k1):  X := X * L_D^{-T} = X * Dinv^T,
// 64 rows per CTA, both operands staged in shared memory.
template <typename T>
__global__ void __launch_bounds__(256)
k_trsm_panel(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
             const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr, const int64_t* __restrict__ Dptr,
             T* __restrict__ L, const T* __restrict__ Dinv, int k0, float* __restrict__ Phi,
             float* __restrict__ Plo, const int64_t* __restrict__ PKptr, const int2* __restrict__ tiles) {
  int tq, tb;
  tile_of(tiles, tq, tb);
  int s = list[tq];
  int c = first[s + 1] - first[s];
  if (k0 >= c) return;
  int m = mrows[s];
  int k1 = min(k0 + NB, c), kn = k1 - k0;
  int row0 = k1 + tb * 64;
  if (row0 >= m) return;
  extern __shared__ unsigned char smem_raw[];
  T (*Di)[NB + 1] = reinterpret_cast<T (*)[NB + 1]>(smem_raw);
  T (*X)[NB + 1] = Di + NB;
  const T* Dv = Dinv + Dptr[s] + (int64_t)(k0 / NB) * NB * NB;
  T* P = L + Lptr[s];
  // 256 threads: all 32 loads of a thread in flight together
#pragma unroll
  for (int u = 0; u < NB * NB / 256; ++u) {
    int e = threadIdx.x + 256 * u;
    int i = e % NB, j = e / NB;
    Di[i][j] = Dv[i + NB * j];
    int row = row0 + i;
    X[i][j] = (row < m && j < kn) ? P[row + (int64_t)m * (k0 + j)] : (T)0;
  }
  __syncthreads();
  int r = threadIdx.x & 63, g = threadIdx.x >> 6;   // row, group of 16 output columns
  int row = row0 + r;
  T acc[16];
#pragma unroll
  for (int t = 0; t < 16; ++t) acc[t] = (T)0;
  for (int q = 0; q < kn; ++q) {
    T xq = X[r][q];
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      int l = g * 16 + t;
      acc[t] += (q <= l) ? xq * Di[l][q] : (T)0;
    }
  }
  if (row < m) {
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      int l = g * 16 + t;
      if (l < kn) P[row + (int64_t)m * (k0 + l)] = acc[t];
    }
    if constexpr (sizeof(T) == 4) {
      // packed tensor-core operands: hi = rn19(v), lo = rn19(v - hi), in the
      // 64-byte-swizzled atoms of 8 rows x 16 columns (this thread's 16
      // columns are one slice block; its row is 64 contiguous bytes)
      if (Phi) {
        const int64_t nrg = (m + 7) / 8;
        const int ri = row & 7, sw = (ri >> 1) & 3;
        const int64_t base = PKptr[s] + ((int64_t)((k0 + 16 * g) >> 4) * nrg + (row >> 3)) * 128 + ri * 16;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float h[4], l[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const float v = acc[4 * q + e];
            h[e] = __uint_as_float((__float_as_uint(v) + 0x1000u) & 0xFFFFE000u);
            const float rem = v - h[e];
            l[e] = __uint_as_float((__float_as_uint(rem) + 0x1000u) & 0xFFFFE000u);
          }
          const int l0 = g * 16 + 4 * q;                   // first panel column of the chunk
          const int64_t off = base + (int64_t)((q ^ sw) * 4);
          if (l0 + 3 < kn) {
            *reinterpret_cast<float4*>(Phi + off) = make_float4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<float4*>(Plo + off) = make_float4(l[0], l[1], l[2], l[3]);
          } else {
#pragma unroll
            for (int e = 0; e < 4; ++e)
              if (l0 + e < kn) { Phi[off + e] = h[e]; Plo[off + e] = l[e]; }
          }
        }
      }
    }
  }
}

// Tile update C -= A_rows * B_rows^T (lower part).  mode 0: trailing panel
// columns after block k0; mode 1: Schur complement U -= L21 L21^T.
template <typename T>
__global__ void __launch_bounds__(256)
k_front_update(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
               const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr,
               const int64_t* __restrict__ Uptr, T* __restrict__ L, T* __restrict__ U, int mode, int kbeg,
               int kend, int cend, const int2* __restrict__ tiles) {
  int tq, tb;
  tile_of(tiles, tq, tb);
  int s = list[tq];
  int c = first[s + 1] - first[s];
  int m = mrows[s];
  const T* P = L + Lptr[s];
  int row0, col0, nrow, ncol, kb, ke;
  T* C;
  int64_t ldc;
  if (mode == 0) {
    // columns [k1, min(cend, c)) and rows [k1, m) of the front, K = [kbeg, k1)
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
  int ntj = (ncol + TILE - 1) / TILE, nti = (nrow + TILE - 1) / TILE;
  int t = tb;
  if (t >= nti * ntj) return;
  int ti = t / ntj, tj = t % ntj;
  if (ti * TILE + TILE - 1 + row0 < tj * TILE + col0) return;   // strictly upper tile
  __shared__ T As[16][TILE + 1];
  __shared__ T Bs[16][TILE + 1];
  int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = (T)0;
  int lr = threadIdx.x & 63, lk = threadIdx.x >> 6;   // loader: 64 rows x 4 k
  int64_t arow = row0 + (int64_t)ti * TILE + lr, brow = col0 + (int64_t)tj * TILE + lr;
  bool aok = ti * TILE + lr < nrow, bok = tj * TILE + lr < ncol;
  for (int k = kb; k < ke; k += 16) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int kk = lk + 4 * q;
      int kg = k + kk;
      As[kk][lr] = (aok && kg < ke) ? P[arow + (int64_t)m * kg] : (T)0;
      Bs[kk][lr] = (bok && kg < ke) ? P[brow + (int64_t)m * kg] : (T)0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      T av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = As[kk][ty + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = Bs[kk][tx + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] += av[a] * bv[b];
    }
    __syncthreads();
  }
  // epilogue; for mode 0 every load of C is issued before the first store.
  // Mode 1 writes U = -L21 L21^T; the children are added after.
  auto inside = [&](int i, int j) { return i < nrow && j < ncol && row0 + i >= col0 + j; };
  if (mode == 0) {
    T cv[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        int i = ti * TILE + ty + 16 * a, j = tj * TILE + tx + 16 * b;
        cv[a][b] = inside(i, j) ? C[i + ldc * j] : (T)0;
      }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        int i = ti * TILE + ty + 16 * a, j = tj * TILE + tx + 16 * b;
        if (inside(i, j)) C[i + ldc * j] = cv[a][b] - acc[a][b];
      }
  } else {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        int i = ti * TILE + ty + 16 * a, j = tj * TILE + tx + 16 * b;
        if (inside(i, j)) C[i + ldc * j] = -acc[a][b];
      }
  }
}

// FP64 tensor-core (DMMA, mma.sync m8n8k4 f64) version of k_front_update for
// the FP64 factor: the same 64 x 64 tiles and modes, 4 warps per CTA, each
// warp a 32 x 32 block of 4 x 4 m8n8 accumulators; K in slices of 16 staged
// through double-buffered shared memory (row stride 68 doubles keeps the
// fragment loads free of bank conflicts).  tcgen05 has no FP64 kind, so this
// is the tensor-core route for FP64.
__device__ __forceinline__ void dmma_884(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

constexpr int DM_LD = TILE + 4;

__global__ void __launch_bounds__(128)
k_front_update_dmma(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
                    const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr,
                    const int64_t* __restrict__ Uptr, double* __restrict__ L, double* __restrict__ U, int mode,
                    int kbeg, int kend, int cend, const int2* __restrict__ tiles) {
  int tq, tb;
  tile_of(tiles, tq, tb);
  int s = list[tq];
  int c = first[s + 1] - first[s];
  int m = mrows[s];
  const double* P = L + Lptr[s];
  int row0, col0, nrow, ncol, kb, ke;
  double* C;
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
  int ntj = (ncol + TILE - 1) / TILE, nti = (nrow + TILE - 1) / TILE;
  int t = tb;
  if (t >= nti * ntj) return;
  int ti = t / ntj, tj = t % ntj;
  if (ti * TILE + TILE - 1 + row0 < tj * TILE + col0) return;   // strictly upper tile
  __shared__ double As[2][16][DM_LD];
  __shared__ double Bs[2][16][DM_LD];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wr = warp >> 1, wc = warp & 1;
  const int g = lane >> 2, q = lane & 3;
  // loader: element e = tid + 128 j -> row e & 63, k (e >> 6) in [0, 16)
  const int64_t abase = row0 + (int64_t)ti * TILE, bbase = col0 + (int64_t)tj * TILE;
  double ra[8], rb[8];
  auto gload = [&](int k) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      int e = tid + 128 * j, r = e & 63, kk = e >> 6;
      int kg = k + kk;
      bool kok = kg < ke;
      ra[j] = (kok && ti * TILE + r < nrow) ? P[abase + r + (int64_t)m * kg] : 0.0;
      rb[j] = (kok && tj * TILE + r < ncol) ? P[bbase + r + (int64_t)m * kg] : 0.0;
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      int e = tid + 128 * j, r = e & 63, kk = e >> 6;
      As[buf][kk][r] = ra[j];
      Bs[buf][kk][r] = rb[j];
    }
  };
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  gload(kb);
  sstore(0);
  __syncthreads();
  int buf = 0;
  for (int k = kb; k < ke; k += 16) {
    const bool more = k + 16 < ke;
    if (more) gload(k + 16);
#pragma unroll
    for (int k4 = 0; k4 < 16; k4 += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) af[a] = As[buf][k4 + q][wr * 32 + a * 8 + g];
#pragma unroll
      for (int b = 0; b < 4; ++b) bf[b] = Bs[buf][k4 + q][wc * 32 + b * 8 + g];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dmma_884(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
    }
    if (more) sstore(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }
  // epilogue; for mode 0 every load of C is issued before the first store
  auto inside = [&](int i, int j) { return i < nrow && j < ncol && row0 + i >= col0 + j; };
  if (mode == 0) {
    double cv[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          int i = ti * TILE + wr * 32 + a * 8 + g, j = tj * TILE + wc * 32 + b * 8 + 2 * q + h;
          cv[a][b][h] = inside(i, j) ? C[i + ldc * j] : 0.0;
        }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          int i = ti * TILE + wr * 32 + a * 8 + g, j = tj * TILE + wc * 32 + b * 8 + 2 * q + h;
          if (inside(i, j)) C[i + ldc * j] = cv[a][b][h] - acc[a][b][h];
        }
  } else {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          int i = ti * TILE + wr * 32 + a * 8 + g, j = tj * TILE + wc * 32 + b * 8 + 2 * q + h;
          if (inside(i, j)) C[i + ldc * j] = -acc[a][b][h];
        }
  }
}

// FP64 panel triangular solve on the FP64 tensor cores: rows [k1 + 64 tb,
// +64) of panel columns [k0, k1) become X Dinv^T, a 64 x kn x kn product
// (Dinv is stored with zeros above its diagonal, so the dense product is
// the triangular one).  Same tiles as k_trsm_panel; 4 warps, each 32 rows x
// 32 columns of the 64 x 64 output, K in slices of 16 double-buffered in
// shared memory (the layout of k_front_update_dmma: As[k][row],
// Bs[k][col] with Bs[q][l] = Dinv[l][q]).  Every read of the CTA's rows
// happens before the barrier that ends the K loop, so the result is
// written in place.
__global__ void __launch_bounds__(128)
k_trsm_panel_dmma(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
                  const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr,
                  const int64_t* __restrict__ Dptr, double* __restrict__ L, const double* __restrict__ Dinv,
                  int k0, const int2* __restrict__ tiles) {
  int tq, tb;
  tile_of(tiles, tq, tb);
  const int s = list[tq];
  const int c = first[s + 1] - first[s];
  if (k0 >= c) return;
  const int m = mrows[s];
  const int k1 = min(k0 + NB, c), kn = k1 - k0;
  const int row0 = k1 + tb * 64;
  if (row0 >= m) return;
  const int nrow = min(64, m - row0);
  __shared__ double As[2][16][DM_LD];
  __shared__ double Bs[2][16][DM_LD];
  const double* Dv = Dinv + Dptr[s] + (int64_t)(k0 / NB) * NB * NB;
  double* X = L + Lptr[s] + row0 + (int64_t)m * k0;   // X[r + m q], r < nrow, q < kn
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wr = warp >> 1, wc = warp & 1;
  const int g = lane >> 2, q4 = lane & 3;
  double ra[8], rb[8];
  // loader: element e = tid + 128 j -> row / column e & 63, k (e >> 6) in [0, 16)
  auto gload = [&](int k) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int e = tid + 128 * j, r = e & 63, kk = k + (e >> 6);
      ra[j] = (kk < kn && r < nrow) ? X[r + (int64_t)m * kk] : 0.0;
      rb[j] = (kk < kn && r < kn) ? Dv[r + NB * kk] : 0.0;
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int e = tid + 128 * j, r = e & 63, kk = e >> 6;
      As[buf][kk][r] = ra[j];
      Bs[buf][kk][r] = rb[j];
    }
  };
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  gload(0);
  sstore(0);
  __syncthreads();
  int buf = 0;
  for (int k = 0; k < kn; k += 16) {
    const bool more = k + 16 < kn;
    if (more) gload(k + 16);
#pragma unroll
    for (int k4 = 0; k4 < 16; k4 += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) af[a] = As[buf][k4 + q4][wr * 32 + a * 8 + g];
#pragma unroll
      for (int b = 0; b < 4; ++b) bf[b] = Bs[buf][k4 + q4][wc * 32 + b * 8 + g];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dmma_884(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
    }
    if (more) sstore(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = wr * 32 + a * 8 + g, j = wc * 32 + b * 8 + 2 * q4 + h;
        if (i < nrow && j < kn) X[i + (int64_t)m * j] = acc[a][b][h];
      }
}

// smallest level output (rows) handed to the tensor-core update kernel
inline int tc_min_dim() {
  const char* e = std::getenv("JFG_TC_MIN");
  return e ? std::max(1, std::atoi(e)) : 256;
}

inline bool dmma_enabled() {
  const char* e = std::getenv("JFG_DMMA");
  return !(e && e[0] == '0');
}

// FP64 panel triangular solves on the FP64 tensor cores (JFG_DMMA_TRSM=0:
// the SIMT kernel)
inline bool dmma_trsm() {
  static int v = -1;
  if (v < 0) {
    const char* e = std::getenv("JFG_DMMA_TRSM");
    v = (e && e[0] == '0') ? 0 : (dmma_enabled() ? 1 : 0);
  }
  return v == 1;
}

// one launch of the front update for a level: DMMA for the FP64 factor,
// SIMT tiles otherwise (and for the FP64 factor with JFG_DMMA=0)
template <typename T>
void launch_front_update(const int2* tiles, int n_tiles, NumericFactor* F, T* Lf, T* Uf, int mode, int kbeg,
                         int kend, int cend, cudaStream_t st) {
  if constexpr (sizeof(T) == 8) {
    if (dmma_enabled()) {
      k_front_update_dmma<<<(unsigned)n_tiles, 128, 0, st>>>(F->level_sn_cur, F->first, F->mrows, F->Lptr, F->Uptr,
                                                             Lf, Uf, mode, kbeg, kend, cend, tiles);
      count_launch();
      return;
    }
  }
  k_front_update<T><<<(unsigned)n_tiles, 256, 0, st>>>(F->level_sn_cur, F->first, F->mrows, F->Lptr, F->Uptr, Lf, Uf,
                                                       mode, kbeg, kend, cend, tiles);
  count_launch();
}

// ---------------------------------------------------------------- solves
// Vectors: xp (n x nr, ld n, permuted order); V arena of update vectors
// (r_s x nr per supernode, ld r_s, offset relptr[s]*nr).

__global__ void k_zero_V(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
                         const int32_t* __restrict__ mrows, const int64_t* __restrict__ relptr, int nr,
                         double* __restrict__ V) {
  int s = list[blockIdx.x];
  int64_t r = mrows[s] - (first[s + 1] - first[s]);
  double* v = V + relptr[s] * nr;
  for (int64_t q = threadIdx.x; q < r * nr; q += blockDim.x) v[q] = 0.0;
}

template <int NRC>
__global__ void k_vec_extend_add(const int32_t* __restrict__ child, const int32_t* __restrict__ first,
                                 const int32_t* __restrict__ mrows, const int32_t* __restrict__ parent,
                                 const int64_t* __restrict__ relptr, const int32_t* __restrict__ rel, int nr,
                                 int64_t n, double* __restrict__ xp, double* __restrict__ V, const int2* __restrict__ tiles) {
  int tq, tb;
  tile_of(tiles, tq, tb);
  int ch = child[tq];
  int rc = mrows[ch] - (first[ch + 1] - first[ch]);
  int p = parent[ch];
  int cp = first[p + 1] - first[p];
  int rp = mrows[p] - cp;
  const int32_t* rl = rel + relptr[ch];
  const double* src = V + relptr[ch] * nr;
  double* vp = V + relptr[p] * nr;
  // the tile's block is a chunk of 256 update rows; children of one launch have
  // distinct parents, and distinct rows of a child map to distinct targets
  int a = tb * 256 + threadIdx.x;
  if (a >= rc) return;
  int ra = rl[a];
  double* dst = (ra < cp) ? xp + first[p] + ra : vp + (ra - cp);
  const int64_t ld = (ra < cp) ? n : (int64_t)rp;
  double v[NRC], d[NRC];
#pragma unroll
  for (int k = 0; k < NRC; ++k) v[k] = k < nr ? src[a + (int64_t)rc * k] : 0.0;
#pragma unroll
  for (int k = 0; k < NRC; ++k) d[k] = k < nr ? dst[ld * k] : 0.0;
#pragma unroll
  for (int k = 0; k < NRC; ++k)
    if (k < nr) dst[ld * k] = d[k] + v[k];
}

// ---------------------------------------------------------------- strip solves
// The solve sweeps every front of a level in strips of SW = 256 columns.  The
// inverse X of each strip's diagonal block (kw x kw, kw = min(256, width
// left)) is formed once per factorisation (k_strip_inverse), so the diagonal
// part of a strip is one dense matrix-vector product per CTA; the rows below
// the strip are updated (forward) or dotted (backward) by wide, coalesced
// kernels over many CTAs.
constexpr int SB = 64;
constexpr int SW = 256;

// Strip inverses from the 64 x 64 inverse blocks D_i of the factor: block
// column jb of X = L_strip^{-1} is X_jj = D_jb and, for i > jb,
// X_ij = -D_i * sum_{jb <= k < i} L_ik X_kj  (block forward substitution).
// One CTA per (front, strip, block column); X is column-major with ld kw.
template <typename T>
__global__ void __launch_bounds__(256)
k_strip_inverse(const int32_t* __restrict__ it_sn, const int32_t* __restrict__ it_kb,
                const int32_t* __restrict__ it_jb, const int32_t* __restrict__ first,
                const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr,
                const int64_t* __restrict__ Dptr, const int64_t* __restrict__ Sptr, const T* __restrict__ L,
                const T* __restrict__ Dinv, T* __restrict__ Sinv) {
  const int s = it_sn[blockIdx.x], kb = it_kb[blockIdx.x], jb = it_jb[blockIdx.x];
  const int c = first[s + 1] - first[s], m = mrows[s];
  const int j0 = kb * SW, kw = min(SW, c - j0), nblk = (kw + SB - 1) / SB;
  const T* P = L + Lptr[s];
  const T* Dv = Dinv + Dptr[s] + (int64_t)(kb * (SW / SB)) * SB * SB;
  T* X = Sinv + Sptr[s] + (int64_t)kb * SW * SW;
  extern __shared__ unsigned char smem_raw[];
  T (*As)[SB + 1] = reinterpret_cast<T (*)[SB + 1]>(smem_raw);
  T (*Bs)[SB + 1] = As + SB;
  const int t = threadIdx.x, tr = t & 15, tc = t >> 4;
  // X_jj = D_jb
  for (int e = t; e < SB * SB; e += blockDim.x) {
    int r = e & (SB - 1), q = e >> 6;
    int gr = SB * jb + r, gq = SB * jb + q;
    if (gr < kw && gq < kw) X[gr + (int64_t)kw * gq] = Dv[(int64_t)jb * SB * SB + r + SB * q];
  }
  __syncthreads();
  for (int i = jb + 1; i < nblk; ++i) {
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    for (int k = jb; k < i; ++k) {
      for (int e = t; e < SB * SB; e += blockDim.x) {
        int r = e & (SB - 1), q = e >> 6;
        int ar = SB * i + r, aq = SB * k + q, br = SB * k + r, bq = SB * jb + q;
        As[r][q] = (ar < kw && aq < kw) ? P[(j0 + ar) + (int64_t)m * (j0 + aq)] : (T)0;
        Bs[r][q] = (br < kw && bq < kw) ? X[br + (int64_t)kw * bq] : (T)0;
      }
      __syncthreads();
#pragma unroll 8
      for (int q = 0; q < SB; ++q) {
        double av[4], bv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) av[a] = (double)As[tr + 16 * a][q];
#pragma unroll
        for (int b = 0; b < 4; ++b) bv[b] = (double)Bs[q][tc + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] += av[a] * bv[b];
      }
      __syncthreads();
    }
    // X_ij = -D_i * acc
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) Bs[tr + 16 * a][tc + 16 * b] = (T)acc[a][b];
    for (int e = t; e < SB * SB; e += blockDim.x) {
      int r = e & (SB - 1), q = e >> 6;
      As[r][q] = Dv[(int64_t)i * SB * SB + r + SB * q];
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
#pragma unroll 8
    for (int q = 0; q < SB; ++q) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = (double)As[tr + 16 * a][q];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = (double)Bs[q][tc + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] += av[a] * bv[b];
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        int gr = SB * i + tr + 16 * a, gq = SB * jb + tc + 16 * b;
        if (gr < kw && gq < kw) X[gr + (int64_t)kw * gq] = (T)(-acc[a][b]);
      }
    __syncthreads();   // X_ij visible to the CTA before it is read as an operand
  }
}

// The diagonal product of a strip is spread over ceil(kw / 32) CTAs, each
// owning 32 rows (forward) or 32 output columns (backward).  The forward
// reads b from xp and writes y to the vector tt; the backward reads y from tt
// and writes x to xp.  No CTA overwrites values another CTA of the same
// launch reads, and at the end of the backward sweep xp holds the solution.
// forward (a): y = X b on the rows of strip kb; CTA (g, front) owns rows
// [32g, 32g + 32) and its 8 warps split the columns j (stride 8)
template <int NRC>
constexpr int fwd_sdiag_smem() { return (SW * NRC + 8 * 32 * (NRC + 1)) * (int)sizeof(double); }

template <typename T, int NRC>
__global__ void __launch_bounds__(256)
k_fwd_sdiag(const int32_t* __restrict__ list, const int32_t* __restrict__ first, const int64_t* __restrict__ Sptr,
            const T* __restrict__ Sinv, int kb, int nr, int64_t n, const double* __restrict__ xp,
            double* __restrict__ tt, const int2* __restrict__ tiles) {
  int tq, tb;
  tile_of(tiles, tq, tb);
  int s = list[tq];
  int f = first[s], c = first[s + 1] - f;
  int j0 = kb * SW;
  if (j0 >= c) return;
  int kw = min(SW, c - j0);
  int g = tb, r0 = 32 * g;
  if (r0 >= kw) return;
  const T* X = Sinv + Sptr[s] + (int64_t)kb * SW * SW;
  int rmax = min(kw, r0 + 32);          // columns j < rmax can touch the slab
  extern __shared__ double sdyn[];
  double (*bs)[NRC] = reinterpret_cast<double (*)[NRC]>(sdyn);
  double (*red)[32][NRC + 1] = reinterpret_cast<double (*)[32][NRC + 1]>(sdyn + SW * NRC);
  for (int e = threadIdx.x; e < rmax * NRC; e += blockDim.x) {
    int l = e % rmax, k = e / rmax;
    bs[l][k] = k < nr ? xp[f + j0 + l + n * k] : 0.0;
  }
  __syncthreads();
  int lane = threadIdx.x & 31, cg = threadIdx.x >> 5;
  int r = r0 + lane;
  double acc[NRC];
#pragma unroll
  for (int k = 0; k < NRC; ++k) acc[k] = 0.0;
  if (r < kw) {
    const T* xr = X + r;
#pragma unroll 4
    for (int j = cg; j <= r; j += 8) {
      double x = (double)xr[(int64_t)kw * j];
#pragma unroll
      for (int k = 0; k < NRC; ++k) acc[k] += x * bs[j][k];
    }
  }
#pragma unroll
  for (int k = 0; k < NRC; ++k) red[cg][lane][k] = acc[k];
  __syncthreads();
  for (int e = threadIdx.x; e < 32 * NRC; e += blockDim.x) {
    int l = e & 31, k = e >> 5;
    if (r0 + l < kw && k < nr) {
      double v = 0.0;
#pragma unroll
      for (int w = 0; w < 8; ++w) v += red[w][l][k];
      tt[f + j0 + r0 + l + n * k] = v;
    }
  }
}

// forward (b): rows below strip kb, 32 rows x SW columns per CTA
template <typename T>
__global__ void __launch_bounds__(256)
k_fwd_supdate(const int32_t* __restrict__ list, const int32_t* __restrict__ first, const int32_t* __restrict__ mrows,
              const int64_t* __restrict__ Lptr, const int64_t* __restrict__ relptr, const T* __restrict__ L, int kb,
              int nr, int64_t n, const double* __restrict__ tt, double* __restrict__ xp,
              double* __restrict__ V, const int2* __restrict__ tiles) {
  int tq, tb;
  tile_of(tiles, tq, tb);
  int s = list[tq];
  int f = first[s], c = first[s + 1] - f, m = mrows[s], r = m - c;
  int j0 = kb * SW;
  if (j0 >= c) return;
  int kw = min(SW, c - j0);
  int row0 = j0 + kw + tb * 32;
  if (row0 >= m) return;
  __shared__ double ys[SW][8];
  __shared__ double red[8][32][9];
  // only the strip's kw columns and nr right-hand sides are read below (the
  // accumulators of right-hand sides past nr are never stored)
  for (int e = threadIdx.x; e < kw * nr; e += blockDim.x) {
    int l = e % kw, k = e / kw;
    ys[l][k] = tt[f + j0 + l + n * k];
  }
  __syncthreads();
  int rr = threadIdx.x & 31, g = threadIdx.x >> 5;   // row, column group of SW/8
  int i = row0 + rr;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (i < m) {
    const T* P = L + Lptr[s] + i;
    // the strip's kw columns split evenly over the 8 warps (narrow fronts
    // would otherwise leave most warps without columns)
    const int cw = (kw + 7) / 8;
    int l0 = g * cw, l1 = min(l0 + cw, kw);
#pragma unroll 8
    for (int l = l0; l < l1; ++l) {
      double lv = (double)P[(int64_t)m * (j0 + l)];
#pragma unroll
      for (int k = 0; k < 8; ++k) acc[k] += lv * ys[l][k];
    }
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) red[g][rr][k] = acc[k];
  __syncthreads();
  if (threadIdx.x < 32 * 8) {
    int row = threadIdx.x & 31, k = threadIdx.x >> 5;
    int ii = row0 + row;
    if (ii < m && k < nr) {
      double t = 0.0;
      for (int gg = 0; gg < 8; ++gg) t += red[gg][row][k];
      if (ii < c) xp[f + ii + n * k] -= t;
      else V[relptr[s] * nr + (ii - c) + (int64_t)r * k] -= t;
    }
  }
}

// forward (b), 16 or 32 right-hand sides: one thread per row below the
// strip, 128 rows per CTA, the strip's columns in tiles of 64 (y staged in
// shared memory); every factor entry is read once for all right-hand sides
template <typename T, int NRC>
__global__ void __launch_bounds__(128)
k_fwd_supdate_wide(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
                   const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr,
                   const int64_t* __restrict__ relptr, const T* __restrict__ L, int kb, int nr, int64_t n,
                   const double* __restrict__ tt, double* __restrict__ xp, double* __restrict__ V, const int2* __restrict__ tiles) {
  int tq, tb;
  tile_of(tiles, tq, tb);
  int s = list[tq];
  int f = first[s], c = first[s + 1] - f, m = mrows[s], r = m - c;
  int j0 = kb * SW;
  if (j0 >= c) return;
  int kw = min(SW, c - j0);
  int row0 = j0 + kw + tb * 128;
  if (row0 >= m) return;
  __shared__ double ys[64][NRC];
  const int i = row0 + threadIdx.x;
  double acc[NRC];
#pragma unroll
  for (int k = 0; k < NRC; ++k) acc[k] = 0.0;
  const T* P = L + Lptr[s] + i;
  for (int l0 = 0; l0 < kw; l0 += 64) {
    const int lw = min(64, kw - l0);
    __syncthreads();
    for (int e = threadIdx.x; e < lw * NRC; e += 128) {
      int l = e % lw, k = e / lw;
      ys[l][k] = k < nr ? tt[f + j0 + l0 + l + n * k] : 0.0;
    }
    __syncthreads();
    if (i < m) {
#pragma unroll 8
      for (int l = 0; l < lw; ++l) {
        const double lv = (double)P[(int64_t)m * (j0 + l0 + l)];
#pragma unroll
        for (int k = 0; k < NRC; ++k) acc[k] += lv * ys[l][k];
      }
    }
  }
  if (i < m) {
#pragma unroll
    for (int k = 0; k < NRC; ++k) {
      if (k >= nr) break;
      if (i < c) xp[f + i + n * k] -= acc[k];
      else V[relptr[s] * nr + (i - c) + (int64_t)r * k] -= acc[k];
    }
  }
}

// Sums each of v[0..NRC-1] over the 32 lanes of a warp by halving: every
// step hands half of the remaining components to the partner lane (log2 NRC
// exchanges), the rest is a plain butterfly.  Lane L ends with the total of
// component L >> (5 - log2 NRC) (the other lanes of its group hold the same).
template <int NRC>
__device__ __forceinline__ double warp_sum_scatter(const double (&v)[NRC], int lane) {
  constexpr int H = NRC >= 32 ? 5 : NRC >= 16 ? 4 : 3;
  const unsigned full = 0xffffffffu;
  double a[NRC];
#pragma unroll
  for (int k = 0; k < NRC; ++k) a[k] = v[k];
#pragma unroll
  for (int step = 0; step < H; ++step) {
    const int off = 16 >> step;
    const int half = NRC >> (step + 1);
    const bool hi = lane & off;
#pragma unroll
    for (int k = 0; k < half; ++k) {
      const double keep = hi ? a[k + half] : a[k], send = hi ? a[k] : a[k + half];
      a[k] = keep + __shfl_xor_sync(full, send, off);
    }
  }
  double c = a[0];
#pragma unroll
  for (int off = 16 >> H; off > 0; off >>= 1) c += __shfl_xor_sync(full, c, off);
  return c;
}

// backward (a): partial dots for the SW columns of strip kb over a tile of
// 256 rows x 32 columns below the strip (8 warps x 4 columns)
template <int NRC>
constexpr int bwd_spartial_smem() { return NRC * 256 * (int)sizeof(double); }

template <typename T, int NRC>
__global__ void __launch_bounds__(256)
k_bwd_spartial(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
               const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr,
               const int64_t* __restrict__ rows_ptr, const int32_t* __restrict__ rows,
               const int64_t* __restrict__ part_off, const T* __restrict__ L, int kb, int nr, int64_t n,
               const double* __restrict__ xp, double* __restrict__ part, const int2* __restrict__ tiles) {
  int tq, tb;
  tile_of(tiles, tq, tb);
  int s = list[tq];
  int c = first[s + 1] - first[s], m = mrows[s];
  int j0 = kb * SW;
  if (j0 >= c) return;
  int kw = min(SW, c - j0);
  int nrb = (m - (j0 + kw) + 255) / 256;
  int rb = tb / (SW / 32), cg = tb % (SW / 32);
  if (rb >= nrb || cg * 32 >= kw) return;
  int row0 = j0 + kw + rb * 256;
  // right-hand-side major, so that lanes reading consecutive rows hit
  // consecutive banks
  extern __shared__ double sdyn[];
  double (*xs)[256] = reinterpret_cast<double (*)[256]>(sdyn);
  const int32_t* R = rows + rows_ptr[s];
  for (int e = threadIdx.x; e < 256 * NRC; e += blockDim.x) {
    int ii = e & 255, k = e >> 8;
    int i = row0 + ii;
    xs[k][ii] = (i < m && k < nr) ? xp[(int64_t)R[i] + n * k] : 0.0;
  }
  __syncthreads();
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* out = part + part_off[tq] + (int64_t)rb * SW * MAXR;
  constexpr int GRP = 32 / NRC;   // lanes sharing one reduced component
  for (int q = 0; q < 4; ++q) {
    int jj = cg * 32 + warp * 4 + q;
    double acc[NRC];
#pragma unroll
    for (int k = 0; k < NRC; ++k) acc[k] = 0.0;
    if (jj < kw) {
      const T* col = L + Lptr[s] + (int64_t)m * (j0 + jj);
      double lv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {   // all eight loads in flight
        int i = row0 + lane + 32 * u;
        lv[u] = i < m ? (double)col[i] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int k = 0; k < NRC; ++k) acc[k] += lv[u] * xs[k][lane + 32 * u];
    }
    double v = warp_sum_scatter<NRC>(acc, lane);
    if ((lane % GRP) == 0 && jj < SW) out[jj * MAXR + lane / GRP] = v;
  }
}

// backward (b): x = X^T (b - sum of the partial dots) on the rows of strip kb;
// CTA (g, front) owns outputs [32g, 32g + 32), a warp per output with lanes
// along column i of X
template <int NRC>
constexpr int bwd_sdiag_smem() { return NRC * SW * (int)sizeof(double); }

template <typename T, int NRC>
__global__ void __launch_bounds__(256)
k_bwd_sdiag(const int32_t* __restrict__ list, const int32_t* __restrict__ first, const int32_t* __restrict__ mrows,
            const int64_t* __restrict__ Sptr, const int64_t* __restrict__ part_off, const T* __restrict__ Sinv,
            int kb, int nr, int64_t n, const double* __restrict__ part, const double* __restrict__ tt,
            double* __restrict__ xp, const int2* __restrict__ tiles) {
  int tq, tb;
  tile_of(tiles, tq, tb);
  int s = list[tq];
  int f = first[s], c = first[s + 1] - f, m = mrows[s];
  int j0 = kb * SW;
  if (j0 >= c) return;
  int kw = min(SW, c - j0);
  int g = tb, i0 = 32 * g;
  if (i0 >= kw) return;
  int nrb = (m - (j0 + kw) + 255) / 256;
  const double* pp = part + part_off[tq];
  const T* X = Sinv + Sptr[s] + (int64_t)kb * SW * SW;
  extern __shared__ double sdyn[];
  double (*bs)[SW] = reinterpret_cast<double (*)[SW]>(sdyn);   // right-hand-side major
  for (int e = threadIdx.x; e < (kw - i0) * NRC; e += blockDim.x) {
    int l = i0 + e / NRC, k = e % NRC;
    double v = 0.0;
    if (k < nr) {
      // independent partial sums: four loads in flight per step
      double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
      const double* q = pp + l * MAXR + k;
      int rb = 0;
      for (; rb + 4 <= nrb; rb += 4) {
        a0 += q[(int64_t)rb * SW * MAXR];
        a1 += q[(int64_t)(rb + 1) * SW * MAXR];
        a2 += q[(int64_t)(rb + 2) * SW * MAXR];
        a3 += q[(int64_t)(rb + 3) * SW * MAXR];
      }
      for (; rb < nrb; ++rb) a0 += q[(int64_t)rb * SW * MAXR];
      v = tt[f + j0 + l + n * k] - ((a0 + a1) + (a2 + a3));
    }
    bs[k][l] = v;
  }
  __syncthreads();
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int GRP = 32 / NRC;
  for (int i = i0 + warp; i < min(kw, i0 + 32); i += 8) {
    double acc[NRC];
#pragma unroll
    for (int k = 0; k < NRC; ++k) acc[k] = 0.0;
    const T* col = X + (int64_t)kw * i;
    double x[SW / 32];
#pragma unroll
    for (int u = 0; u < SW / 32; ++u) {   // all loads in flight
      int j = i + lane + 32 * u;
      x[u] = j < kw ? (double)col[j] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < SW / 32; ++u) {
      int j = i + lane + 32 * u;   // bs holds columns [i0, kw) only
      if (j < kw) {
#pragma unroll
        for (int k = 0; k < NRC; ++k) acc[k] += x[u] * bs[k][j];
      }
    }
    double v = warp_sum_scatter<NRC>(acc, lane);
    int k = lane / GRP;
    if ((lane % GRP) == 0 && k < nr) xp[f + j0 + i + n * k] = v;
  }
}

__global__ void k_gather_perm(int64_t n, int nr, const int32_t* __restrict__ perm_dof,
                              const double* __restrict__ scale, const double* __restrict__ src, int64_t ldsrc,
                              double* __restrict__ xp, double sign) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int64_t g = perm_dof[k];
  double sc = scale ? scale[k] : 1.0;
  for (int q = 0; q < nr; ++q) xp[k + n * q] = sign * src[g + ldsrc * q] * sc;
}

__global__ void k_scatter_add_perm(int64_t n, int nr, const int32_t* __restrict__ perm_dof,
                                   const double* __restrict__ scale, const double* __restrict__ xp,
                                   double* __restrict__ dst, int64_t lddst) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int64_t g = perm_dof[k];
  double sc = scale ? scale[k] : 1.0;
  for (int q = 0; q < nr; ++q) dst[g + lddst * q] += xp[k + n * q] * sc;
}

// Second level of the per-column dot products: the nb partial sums of each
// column added in a fixed order (deterministic two-level tree).
__global__ void k_colnorm2_final(int nb, int nr, const double* __restrict__ part, double* __restrict__ out) {
  int q = threadIdx.x;
  if (q >= nr) return;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += part[q * nb + b];
  out[q] = s;
}

struct CoefR { double v[MAXR]; };

__global__ void k_axpy_cols(int64_t len, int nr, CoefR a, const double* __restrict__ x, double* __restrict__ y) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= len) return;
  for (int k = 0; k < nr; ++k) y[i + len * k] += a.v[k] * x[i + len * k];
}
__global__ void k_xpby_cols(int64_t len, int nr, CoefR b, const double* __restrict__ z, double* __restrict__ p) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= len) return;
  for (int k = 0; k < nr; ++k) p[i + len * k] = z[i + len * k] + b.v[k] * p[i + len * k];
}
__global__ void k_mask_free(int64_t len, int nr, const uint8_t* __restrict__ free_mask, double* __restrict__ v) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= len || free_mask[i]) return;
  for (int k = 0; k < nr; ++k) v[i + len * k] = 0.0;
}
// per-column dot products of two len x nr blocks (deterministic two-level tree)
__global__ void k_coldot_partial(int64_t len, int nr, const double* __restrict__ a, const double* __restrict__ b,
                                 double* __restrict__ part) {
  __shared__ double sh[256];
  int q = blockIdx.y;
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
    s += a[i + len * q] * b[i + len * q];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[q * gridDim.x + blockIdx.x] = sh[0];
}

__global__ void k_diag_of_factor64(int64_t ns, const int32_t* first, const int32_t* mrows, const int64_t* Lptr,
                                   const double* L, double* out) {
  int64_t s = (int64_t)blockIdx.x;
  if (s >= ns) return;
  int f = first[s], c = first[s + 1] - f, m = mrows[s];
  for (int j = threadIdx.x; j < c; j += blockDim.x) out[f + j] = L[Lptr[s] + j + (int64_t)m * j];
}
__global__ void k_diag_of_factor32(int64_t ns, const int32_t* first, const int32_t* mrows, const int64_t* Lptr,
                                   const float* L, const double* scale, double* out) {
  int64_t s = (int64_t)blockIdx.x;
  if (s >= ns) return;
  int f = first[s], c = first[s + 1] - f, m = mrows[s];
  for (int j = threadIdx.x; j < c; j += blockDim.x)
    out[f + j] = (double)L[Lptr[s] + j + (int64_t)m * j] / scale[f + j];
}

template <typename T, typename A>
void upload(const std::vector<T, A>& h, T** d, jfg_ctx* c, jfg_status& st) {
  if (st != JFG_OK) return;
  size_t bytes = sizeof(T) * std::max<size_t>(h.size(), 1);
  st = dev_alloc(c, (void**)d, bytes);
  if (st != JFG_OK) return;
  if (!h.empty() && cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    set_error("cudaMemcpy failed uploading symbolic arrays");
    st = JFG_CUDA_ERROR;
  }
}

// tc: the FP32 factor's updates go to the tensor-core kernel (where the
// level's output is large enough); the trsm then also writes the packed
// operand copies F->Phi / F->Plo
template <typename T>
jfg_status factor_levels(jfg_model* m, NumericFactor* F, T* Lf, T* Uf, T* Dvf, bool tc, cudaStream_t st) {
  static bool attr_set = false;
  if (!attr_set) {
    int bytes = 2 * NB * (NB + 1) * (int)sizeof(T);
    JFG_CUDA(cudaFuncSetAttribute(k_potrf_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, potrf_smem<T>()));
    JFG_CUDA(cudaFuncSetAttribute(k_potrf_cta<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, potrf_smem<T>()));
    JFG_CUDA(cudaFuncSetAttribute(k_trsm_panel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    attr_set = true;
  }
  const Symbolic& S = m->sym();
  const int tc_min = tc_min_dim();
  for (const auto& lv : F->levels) {
    const int32_t* list = F->level_sn + lv.off;
    F->level_sn_cur = list;
    if (sizeof(T) == 4 && tc && lv.pk_len > 0) {
      // fresh zero padding for this level's operand images
      JFG_CUDA(cudaMemsetAsync(F->Phi, 0, sizeof(float) * lv.pk_len, st));
      JFG_CUDA(cudaMemsetAsync(F->Plo, 0, sizeof(float) * lv.pk_len, st));
    }
    // one front update of the level: the tensor-core 3xTF32 kernel for the
    // FP32 factor when its low parts exist and the level's output is large
    // enough for 128 x 128 tiles, else the SIMT / DMMA tiles
    using UpdSpans = NumericFactor::Level::UpdSpans;
    auto update = [&](int mode, int kbeg, int kend, int cend, int max_rows, int max_cols, const UpdSpans& u) {
      if constexpr (sizeof(T) == 4) {
        if (tc && max_rows >= tc_min && max_cols >= tc_min / 2 &&
            tc::front_update_tf32x3(list, F->tiles + u.t128.off, u.t128.cnt, F->first, F->mrows, F->Lptr, F->Uptr,
                                    Lf, F->Phi, F->Plo, F->PKptr, F->tc_zero, Uf, mode, kbeg, kend, cend,
                                    F->tc_drain, F->err, st))
          return;
      }
      if (u.t64.cnt > 0)
        launch_front_update<T>(F->tiles + u.t64.off, u.t64.cnt, F, Lf, Uf, mode, kbeg, kend, cend, st);
    };
    // extend-add, pass 0: children columns that land in this level's panels
    for (size_t si = 0; si < lv.ea.size(); ++si) {
      const auto& seg = lv.ea[si];
      const auto& tsp = lv.ea_f[si];
      if (seg.second == 0 || tsp.cnt == 0) continue;
      { int ps_ = fine_prof() ? prof_start(st) : -1; { k_extend_add<T><<<(unsigned)tsp.cnt, 256, 0, st>>>(F->ea_child + seg.first, F->first, F->mrows,
                                                            F->parent, F->Lptr, F->Uptr, F->relptr, F->rel, Lf, Uf, 0,
                                                            F->tiles + tsp.off);
        count_launch(); } prof_end(ps_, st, KS_F_EA, 0.0); }
    }
    // algorithmic flops of the level's diagonal-block, trsm and panel-update
    // launches (kernel-class statistics only): fronts i < n of the level,
    // widths lv.cs[i], rows sn_m
    const bool count_work = fine_prof();
    auto front_m = [&](int i) -> double { return (double)S.sn_m[S.level_sn[lv.off + i]]; };
    auto potrf_flops = [&](int n, int k0) {
      double f = 0;
      for (int i = 0; count_work && i < n; ++i) {
        const double kn = std::min(NB, lv.cs[i] - k0);
        f += (2.0 / 3.0) * kn * kn * kn;   // Cholesky and inverse of the block
      }
      return f;
    };
    auto trsm_flops = [&](int n, int k0) {
      double f = 0;
      for (int i = 0; count_work && i < n; ++i) {
        const double kn = std::min(NB, lv.cs[i] - k0);
        f += 2.0 * kn * kn * std::max(0.0, front_m(i) - k0 - kn);
      }
      return f;
    };
    // C -= A B^T on the lower trapezoid rows r0.., columns r0..ce of K columns
    auto update_flops = [&](int n, int kb, int ke, int r0, int cend) {
      double f = 0;
      for (int i = 0; count_work && i < n; ++i) {
        const double K = std::min(ke, lv.cs[i]) - kb;
        const double rows = front_m(i) - r0, cols = std::min(cend, lv.cs[i]) - r0;
        if (K > 0 && rows > 0 && cols > 0) f += 2.0 * K * (rows * cols - cols * (cols - 1.0) / 2.0);
      }
      return f;
    };
    // blocked partial factorisation of every front of the level, in
    // super-panels of PW columns: inside a super-panel the 64-column steps
    // update only the super-panel's own later columns; the columns after it
    // take one update with K = PW, so the trailing part of a wide front is
    // read and written once per PW columns instead of once per 64
    const int PW = panel_width();
    for (int P0 = 0; P0 < lv.max_c; P0 += PW) {
      const int P1 = P0 + PW;
      for (int k0 = P0; k0 < std::min(P1, lv.max_c); k0 += NB) {
        const int na = lv.active(k0);   // fronts wider than k0: a prefix of the list
        { int ps_ = fine_prof() ? prof_start(st) : -1; { if (potrf_cta())
            k_potrf_cta<T><<<na, 256, potrf_smem<T>(), st>>>(list, F->first, F->mrows, F->Lptr, F->Dptr, Lf, Dvf, k0,
                                                              F->err);
          else
            k_potrf_diag<T><<<na, 256, potrf_smem<T>(), st>>>(list, F->first, F->mrows, F->Lptr,
                                                               F->Dptr, Lf, Dvf, k0, F->err);
          count_launch(); } prof_end(ps_, st, KS_F_POTRF, potrf_flops(na, k0)); }
        int rows_max = lv.maxm(na) - k0 - 1;
        if (rows_max <= 0) continue;
        const auto& tsp = lv.trsm[k0 / NB];
        if (tsp.cnt > 0) { int ps_ = fine_prof() ? prof_start(st) : -1; {
          if constexpr (sizeof(T) == 8) {
            if (dmma_trsm())
              k_trsm_panel_dmma<<<(unsigned)tsp.cnt, 128, 0, st>>>(list, F->first, F->mrows, F->Lptr, F->Dptr,
                                                                   reinterpret_cast<double*>(Lf),
                                                                   reinterpret_cast<const double*>(Dvf), k0,
                                                                   F->tiles + tsp.off);
            else
              k_trsm_panel<T><<<(unsigned)tsp.cnt, 256, 2 * NB * (NB + 1) * sizeof(T), st>>>(
                  list, F->first, F->mrows, F->Lptr, F->Dptr, Lf, Dvf, k0, nullptr, F->Plo, F->PKptr,
                  F->tiles + tsp.off);
          } else {
            k_trsm_panel<T><<<(unsigned)tsp.cnt, 256, 2 * NB * (NB + 1) * sizeof(T), st>>>(
                list, F->first, F->mrows, F->Lptr, F->Dptr, Lf, Dvf, k0, tc ? F->Phi : nullptr, F->Plo, F->PKptr,
                F->tiles + tsp.off);
          }
          count_launch(); } prof_end(ps_, st, KS_F_TRSM, trsm_flops(na, k0)); }
        const int nu = lv.active(k0 + NB);   // fronts with columns after this block
        int nrow = lv.maxm(nu) - k0 - NB, ncol = std::min(P1, lv.max_c) - k0 - NB;
        if (nu > 0 && nrow > 0 && ncol > 0) {
          { int ps_ = fine_prof() ? prof_start(st) : -1;
            update(0, k0, k0 + NB, P1, nrow, ncol, lv.upd_step[k0 / NB]);
            prof_end(ps_, st, KS_F_PANEL, update_flops(nu, k0, k0 + NB, k0 + NB, P1)); }
        }
      }
      const int nt = lv.active(P1);   // fronts with columns after the super-panel
      int nrow = lv.maxm(nt) - P1, ncol = lv.max_c - P1;
      if (nt > 0 && nrow > 0 && ncol > 0) {
        { int ps_ = fine_prof() ? prof_start(st) : -1;
          update(0, P0, P1, INT_MAX, nrow, ncol, lv.upd_trail[P0 / PW]);
          prof_end(ps_, st, KS_F_PANEL, update_flops(nt, P0, P1, P1, INT_MAX)); }
      }
    }
    if (lv.max_r > 0) {
      int ps = prof_start(st);
      update(1, 0, 0, 0, lv.max_r, lv.max_r, lv.schur);
      prof_end(ps, st, KS_SCHUR, lv.schur_flops);
    }
    // extend-add, pass 1: children columns that land in the U of this level
    for (size_t si = 0; si < lv.ea.size(); ++si) {
      const auto& seg = lv.ea[si];
      const auto& tsp = lv.ea_f[si];
      if (seg.second == 0 || tsp.cnt == 0) continue;
      { int ps_ = fine_prof() ? prof_start(st) : -1; { k_extend_add<T><<<(unsigned)tsp.cnt, 256, 0, st>>>(F->ea_child + seg.first, F->first, F->mrows,
                                                            F->parent, F->Lptr, F->Uptr, F->relptr, F->rel, Lf, Uf, 1,
                                                            F->tiles + tsp.off);
        count_launch(); } prof_end(ps_, st, KS_F_EA, 0.0); }
    }
    JFG_CUDA(cudaGetLastError());
  }
  (void)S;
  return JFG_OK;
}

// Inverses of every strip's diagonal block, one launch over all fronts once
// the factor is complete (the blocks are independent of each other).
template <typename T>
jfg_status strip_inverses(NumericFactor* F, const T* Lf, const T* Dvf, T* Svf, cudaStream_t st) {
  if (F->n_inv_items == 0) return JFG_OK;
  static bool attr_set = false;
  const int bytes = 2 * SB * (SB + 1) * (int)sizeof(T);
  if (!attr_set) {
    JFG_CUDA(cudaFuncSetAttribute(k_strip_inverse<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    attr_set = true;
  }
  int ps = fine_prof() ? prof_start(st) : -1;
  { k_strip_inverse<T><<<(unsigned)F->n_inv_items, 256, bytes, st>>>(F->inv_sn, F->inv_kb, F->inv_jb, F->first,
                                                                  F->mrows, F->Lptr, F->Dptr, F->Sptr, Lf, Dvf, Svf);
    count_launch(); }
  prof_end(ps, st, KS_F_POTRF, 0.0);
  JFG_CUDA(cudaGetLastError());
  return JFG_OK;
}

template <typename T, int NRC>
void solve_inner_n(jfg_model* m, NumericFactor* F, const T* Lf, const T* Sv, int nr, cudaStream_t st) {
  const Symbolic& S = m->sym();
  int64_t n = S.n;
  int ps = prof_start(st);
  // forward, leaves first
  for (size_t li = 0; li < F->levels.size(); ++li) {
    const auto& lv = F->levels[li];
    const int32_t* list = F->level_sn + lv.off;
    const int pl = (fine_prof() && li < (size_t)KS_MAX_LEVELS) ? prof_start(st) : -1;
    { int ps_ = fine_prof() ? prof_start(st) : -1; { k_zero_V<<<lv.count, 256, 0, st>>>(list, F->first, F->mrows, F->relptr, nr, F->V); count_launch(); } prof_end(ps_, st, KS_S_VEC, 0.0); }
    for (size_t si = 0; si < lv.ea.size(); ++si) {
      const auto& seg = lv.ea[si];
      const auto& tsp = lv.ea_s[si];
      if (seg.second > 0 && tsp.cnt > 0)
        { int ps_ = fine_prof() ? prof_start(st) : -1; { k_vec_extend_add<NRC><<<(unsigned)tsp.cnt, 256, 0, st>>>(F->ea_child + seg.first, F->first, F->mrows, F->parent,
                                                     F->relptr, F->rel, nr, n, F->xp, F->V, F->tiles + tsp.off); count_launch(); } prof_end(ps_, st, KS_S_VEC, 0.0); }
    }
    int nstrip = (lv.max_c + SW - 1) / SW;
    for (int kb = 0; kb < nstrip; ++kb) {
      const auto& ts = lv.strips[kb];
      if (ts.diag.cnt > 0) { int ps_ = fine_prof() ? prof_start(st) : -1; { k_fwd_sdiag<T, NRC><<<(unsigned)ts.diag.cnt, 256, fwd_sdiag_smem<NRC>(), st>>>(list, F->first, F->Sptr, Sv, kb, nr, n, F->xp, F->tt, F->tiles + ts.diag.off);
        count_launch(); } prof_end(ps_, st, KS_S_FDIAG, 0.0); }
      const bool narrow = NRC == 8;
      const auto& tu = narrow ? ts.upd32 : ts.upd128;
      if (tu.cnt > 0) {
        int ps_ = fine_prof() ? prof_start(st) : -1;
        if (narrow) {
          k_fwd_supdate<T><<<(unsigned)tu.cnt, 256, 0, st>>>(list, F->first, F->mrows, F->Lptr, F->relptr, Lf, kb,
                                                              nr, n, F->tt, F->xp, F->V, F->tiles + tu.off);
        } else {
          k_fwd_supdate_wide<T, NRC><<<(unsigned)tu.cnt, 128, 0, st>>>(list, F->first, F->mrows, F->Lptr, F->relptr, Lf,
                                                                        kb, nr, n, F->tt, F->xp, F->V,
                                                                        F->tiles + tu.off);
        }
        count_launch();
        prof_end(ps_, st, KS_S_FUPD, 0.0);
      }
    }
    prof_end(pl, st, KS_LEVEL_FWD + (int)li, (double)sizeof(T) * (double)lv.nnz);
  }
  // backward, root first
  for (size_t li = F->levels.size(); li-- > 0;) {
    const auto& lv = F->levels[li];
    const int32_t* list = F->level_sn + lv.off;
    const int64_t* poff = F->part_off + lv.off;
    const int pl = (fine_prof() && li < (size_t)KS_MAX_LEVELS) ? prof_start(st) : -1;
    int nstrip = (lv.max_c + SW - 1) / SW;
    for (int kb = nstrip - 1; kb >= 0; --kb) {
      const auto& ts = lv.strips[kb];
      if (ts.bwd.cnt > 0) {
        { int ps_ = fine_prof() ? prof_start(st) : -1; { k_bwd_spartial<T, NRC><<<(unsigned)ts.bwd.cnt, 256, bwd_spartial_smem<NRC>(), st>>>(list, F->first, F->mrows, F->Lptr, F->rows_ptr, F->rows,
                                                               poff, Lf, kb, nr, n, F->xp, F->part, F->tiles + ts.bwd.off); count_launch(); } prof_end(ps_, st, KS_S_BPART, 0.0); }
      }
      if (ts.diag.cnt > 0) { int ps_ = fine_prof() ? prof_start(st) : -1; { k_bwd_sdiag<T, NRC><<<(unsigned)ts.diag.cnt, 256, bwd_sdiag_smem<NRC>(), st>>>(list, F->first, F->mrows, F->Sptr, poff, Sv, kb, nr, n,
                                                 F->part, F->tt, F->xp, F->tiles + ts.diag.off); count_launch(); } prof_end(ps_, st, KS_S_BDIAG, 0.0); }
    }
    prof_end(pl, st, KS_LEVEL_BWD + (int)li, (double)sizeof(T) * (double)lv.nnz);
  }
  // algorithmic bytes: the factor read twice (forward and backward) plus the
  // permuted vectors read and written in each sweep
  prof_end(ps, st, KS_SOLVE, 2.0 * sizeof(T) * (double)S.nnz_L + 4.0 * 8.0 * n * nr);
}

// One application of the factor for nr <= MAXR right-hand sides: the
// kernels are instantiated for 8, 16 and 32 columns (the smallest that holds nr).
template <typename T>
void solve_inner(jfg_model* m, NumericFactor* F, const T* Lf, const T* Sv, int nr, cudaStream_t st) {
  if (nr <= 8) solve_inner_n<T, 8>(m, F, Lf, Sv, nr, st);
  else if (nr <= 16) solve_inner_n<T, 16>(m, F, Lf, Sv, nr, st);
  else solve_inner_n<T, 32>(m, F, Lf, Sv, nr, st);
}

// Dynamic shared-memory limits of the solve kernels that need more than the
// default 48 KB (set once, outside any stream capture).
template <typename T, int NRC>
jfg_status solve_attributes_n() {
  JFG_CUDA(cudaFuncSetAttribute(k_fwd_sdiag<T, NRC>, cudaFuncAttributeMaxDynamicSharedMemorySize, fwd_sdiag_smem<NRC>()));
  JFG_CUDA(cudaFuncSetAttribute(k_bwd_spartial<T, NRC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                bwd_spartial_smem<NRC>()));
  JFG_CUDA(cudaFuncSetAttribute(k_bwd_sdiag<T, NRC>, cudaFuncAttributeMaxDynamicSharedMemorySize, bwd_sdiag_smem<NRC>()));
  return JFG_OK;
}

jfg_status solve_attributes() {
  static bool done = false;
  if (done) return JFG_OK;
  JFG_TRY((solve_attributes_n<double, 8>())); JFG_TRY((solve_attributes_n<double, 16>()));
  JFG_TRY((solve_attributes_n<double, 32>())); JFG_TRY((solve_attributes_n<float, 8>()));
  JFG_TRY((solve_attributes_n<float, 16>())); JFG_TRY((solve_attributes_n<float, 32>()));
  done = true;
  return JFG_OK;
}

jfg_status ensure_workspace(jfg_model* m, NumericFactor* F, int nrhs) {
  if (nrhs <= F->nrhs_cap) return JFG_OK;
  jfg_ctx* c = m->ctx;
  auto fr = [&](double*& p, int64_t len) {
    if (p) dev_free(c, p, sizeof(double) * len);
    p = nullptr;
  };
  int64_t n = m->sym().n, ndof = m->ndof;
  drop_solve_graphs(F);
  if (F->nrhs_cap > 0) {
    // the old work arrays go back to the pool: work enqueued on the model's
    // stream (an asynchronous application) may still read them
    JFG_CUDA(cudaStreamSynchronize(m->stream));
    int oc = F->nrhs_cap;
    fr(F->xp, n * oc); fr(F->tt, n * oc); fr(F->V, F->v_total * oc); fr(F->dF, ndof * oc); fr(F->dU, ndof * oc);
    fr(F->dR, ndof * oc); fr(F->dD, n * oc); fr(F->dZ, ndof * oc); fr(F->dP, ndof * oc); fr(F->dQ, ndof * oc);
  }
  int cap = std::max(nrhs, 8);
  JFG_TRY(dev_alloc(c, (void**)&F->xp, sizeof(double) * n * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->tt, sizeof(double) * n * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->V, sizeof(double) * std::max<int64_t>(F->v_total, 1) * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->dF, sizeof(double) * ndof * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->dU, sizeof(double) * ndof * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->dR, sizeof(double) * ndof * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->dD, sizeof(double) * n * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->dZ, sizeof(double) * ndof * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->dP, sizeof(double) * ndof * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->dQ, sizeof(double) * ndof * cap));
  F->nrhs_cap = cap;
  return JFG_OK;
}

jfg_status check_err(NumericFactor* F, const char* what) {
  DevError h{};
  JFG_CUDA(cudaMemcpy(&h, F->err, sizeof(DevError), cudaMemcpyDeviceToHost));
  if (h.code == EE_PIVOT) {
    set_error(std::string(what) + ": non-positive pivot in permuted column " + std::to_string(h.index), h.index);
    JFG_CUDA(cudaMemset(F->err, 0, sizeof(DevError)));
    return JFG_NOT_SPD;
  }
  if (h.code == EE_TC_TIMEOUT) {
    set_error(std::string(what) + ": tensor-core pipeline wait expired (front " + std::to_string(h.index) + ")",
              h.index);
    JFG_CUDA(cudaMemset(F->err, 0, sizeof(DevError)));
    return JFG_TIMEOUT;
  }
  return JFG_OK;
}

jfg_status coldot(NumericFactor* F, int64_t len, int nr, const double* a, const double* b, double* out_host,
                  cudaStream_t st) {
  const int nb = 256;
  { k_coldot_partial<<<dim3(nb, nr), 256, 0, st>>>(len, nr, a, b, F->norms); count_launch(); }
  { k_colnorm2_final<<<1, 64, 0, st>>>(nb, nr, F->norms, F->norms + nb * 64); count_launch(); }
  JFG_CUDA(cudaMemcpyAsync(out_host, F->norms + nb * 64, sizeof(double) * nr, cudaMemcpyDeviceToHost, st));
  JFG_CUDA(cudaStreamSynchronize(st));
  return JFG_OK;
}

}  // namespace

// Fronts of a level by decreasing width (then by index), so that the fronts
// still active at a column step are a prefix of the level's list and each
// step launches only them.
static void sort_levels(const Symbolic& S, std::vector<int32_t>& level_sn) {
  if (S.n_levels == 0) return;
  for (int64_t l = 0; l < S.n_levels; ++l)
    std::sort(level_sn.begin() + S.level_ptr[l], level_sn.begin() + S.level_ptr[l + 1], [&](int32_t x, int32_t y) {
      const int32_t cx = S.sn_first[x + 1] - S.sn_first[x], cy = S.sn_first[y + 1] - S.sn_first[y];
      return cx != cy ? cx > cy : x < y;
    });
}

void sort_level_lists(Symbolic& S) {
  std::vector<int32_t> lsn = S.level_sn;
  sort_levels(S, lsn);
  S.level_sn.swap(lsn);
}

// Host launch metadata of every level and the tile lists of its launches
// (only blocks with work).  level_sn holds the level lists, each sorted by
// decreasing width.
static void build_levels(const Symbolic& S, const std::vector<int32_t>& level_sn,
                         std::vector<NumericFactor::Level>& levels, std::vector<int2>& tl) {
  levels.assign(S.n_levels, NumericFactor::Level());
  for (int64_t l = 0; l < S.n_levels; ++l) {
    auto& lv = levels[l];
    lv.off = S.level_ptr[l];
    lv.count = S.level_ptr[l + 1] - S.level_ptr[l];
    lv.max_c = lv.max_m = lv.max_r = 0;
    lv.cs.clear();
    lv.pm.clear();
    lv.nnz = 0;
    for (int32_t q = lv.off; q < lv.off + lv.count; ++q) {
      int32_t s = level_sn[q];
      int32_t cc = S.sn_first[s + 1] - S.sn_first[s];
      lv.max_c = std::max(lv.max_c, cc);
      lv.max_m = std::max(lv.max_m, S.sn_m[s]);
      if (S.sn_parent[s] >= 0) lv.max_r = std::max(lv.max_r, S.sn_m[s] - cc);
      lv.cs.push_back(cc);
      lv.pm.push_back(lv.max_m);
      lv.nnz += (int64_t)S.sn_m[s] * cc;
    }
    lv.schur_flops = 0;
    for (int32_t q = lv.off; q < lv.off + lv.count; ++q) {
      int32_t s = level_sn[q];
      double cc = S.sn_first[s + 1] - S.sn_first[s];
      double rr = S.sn_parent[s] >= 0 ? S.sn_m[s] - cc : 0.0;
      lv.schur_flops += rr * (rr + 1) * cc;
    }
    lv.ea_max_r = 0;
    for (int32_t k = S.ea_level_ptr[l]; k < S.ea_level_ptr[l + 1]; ++k) {
      int32_t a = S.ea_ptr[k], b = S.ea_ptr[k + 1];
      lv.ea.push_back({a, b - a});
      for (int32_t q = a; q < b; ++q) {
        int32_t ch = S.ea_child[q];
        lv.ea_max_r = std::max(lv.ea_max_r, S.sn_m[ch] - (S.sn_first[ch + 1] - S.sn_first[ch]));
      }
    }
  }
  // work tiles of every level launch (only blocks with work)
  {
    using Span = NumericFactor::Level::Span;
    auto span = [&](auto&& gen) {
      Span sp;
      sp.off = (int64_t)tl.size();
      gen();
      sp.cnt = (int32_t)((int64_t)tl.size() - sp.off);
      return sp;
    };
    for (int64_t l = 0; l < S.n_levels; ++l) {
      auto& lv = levels[l];
      const int cnt = lv.count;
      auto mq = [&](int q) { return (int64_t)S.sn_m[level_sn[lv.off + q]]; };
      // extend-add segments: children of one rank
      for (const auto& seg : lv.ea) {
        auto rc_of = [&](int q) {
          const int32_t ch = S.ea_child[seg.first + q];
          return (int64_t)S.sn_m[ch] - (S.sn_first[ch + 1] - S.sn_first[ch]);
        };
        lv.ea_f.push_back(span([&] {
          for (int q = 0; q < seg.second; ++q)
            for (int64_t b = 0; b * 8 < rc_of(q); ++b) tl.push_back(make_int2(q, (int)b));
        }));
        lv.ea_s.push_back(span([&] {
          for (int q = 0; q < seg.second; ++q)
            for (int64_t b = 0; b * 256 < rc_of(q); ++b) tl.push_back(make_int2(q, (int)b));
        }));
      }
      // panel trsm of every 64-column step
      for (int k0 = 0; k0 < lv.max_c; k0 += NB) {
        lv.trsm.push_back(span([&] {
          for (int q = 0; q < cnt && lv.cs[q] > k0; ++q) {
            const int64_t rows = mq(q) - std::min(k0 + NB, lv.cs[q]);
            for (int64_t b = 0; b * 64 < rows; ++b) tl.push_back(make_int2(q, (int)b));
          }
        }));
      }
      // solve strips
      for (int kb = 0; kb * SW < lv.max_c; ++kb) {
        NumericFactor::Level::StripSpans ss;
        auto kw_of = [&](int q) { return (int64_t)std::min(SW, lv.cs[q] - kb * SW); };
        auto rows_of = [&](int q) { return mq(q) - kb * SW - kw_of(q); };
        ss.diag = span([&] {
          for (int q = 0; q < cnt && lv.cs[q] > kb * SW; ++q)
            for (int64_t g = 0; g * 32 < kw_of(q); ++g) tl.push_back(make_int2(q, (int)g));
        });
        ss.upd32 = span([&] {
          for (int q = 0; q < cnt && lv.cs[q] > kb * SW; ++q)
            for (int64_t b = 0; b * 32 < rows_of(q); ++b) tl.push_back(make_int2(q, (int)b));
        });
        ss.upd128 = span([&] {
          for (int q = 0; q < cnt && lv.cs[q] > kb * SW; ++q)
            for (int64_t b = 0; b * 128 < rows_of(q); ++b) tl.push_back(make_int2(q, (int)b));
        });
        ss.bwd = span([&] {
          for (int q = 0; q < cnt && lv.cs[q] > kb * SW; ++q) {
            const int64_t nrb = (rows_of(q) + 255) / 256, ncg = (kw_of(q) + 31) / 32;
            for (int64_t rb = 0; rb < nrb; ++rb)
              for (int64_t cg = 0; cg < ncg; ++cg) tl.push_back(make_int2(q, (int)(rb * (SW / 32) + cg)));
          }
        });
        lv.strips.push_back(ss);
      }
      // front updates, with the kernels' own geometry: mode 0 writes columns
      // [k1, min(cend, c)) and rows [k1, m) (k1 = min(kend, c)), mode 1 the
      // r x r update matrix; the 128-tile grid starts at the output origin
      // rounded down to a multiple of 8 rows
      auto upd = [&](int mode, int kbeg, int kend, int cend) {
        auto gen = [&](int tile, bool align8) {
          for (int q = 0; q < cnt; ++q) {
            const int32_t s = level_sn[lv.off + q];
            const int c = S.sn_first[s + 1] - S.sn_first[s], m = S.sn_m[s];
            int row0, nrow, ncol;
            if (mode == 0) {
              const int k1 = std::min(kend, c), ce = std::min(cend, c);
              if (kbeg >= c || k1 >= ce) continue;
              row0 = k1; nrow = m - k1; ncol = ce - k1;
            } else {
              if (m - c <= 0 || S.sn_Uptr[s] < 0) continue;
              row0 = c; nrow = ncol = m - c;
            }
            if (align8) { nrow += row0 & 7; ncol += row0 & 7; }
            const int ntj = (ncol + tile - 1) / tile, nti = (nrow + tile - 1) / tile;
            for (int ti = 0; ti < nti; ++ti)
              for (int tj = 0; tj <= ti && tj < ntj; ++tj) tl.push_back(make_int2(q, ti * ntj + tj));
          }
        };
        NumericFactor::Level::UpdSpans u;
        u.t64 = span([&] { gen(TILE, false); });
        u.t128 = span([&] { gen(tc::TILE_M, true); });
        return u;
      };
      const int PW = panel_width();
      for (int k0 = 0; k0 < lv.max_c; k0 += NB) {
        const int P1 = (k0 / PW) * PW + PW;
        lv.upd_step.push_back(upd(0, k0, k0 + NB, P1));
      }
      for (int P0 = 0; P0 < lv.max_c; P0 += PW) lv.upd_trail.push_back(upd(0, P0, P0 + PW, INT_MAX));
      lv.schur = upd(1, 0, 0, 0);
    }
  }
}

jfg_status numeric_create(jfg_model* m) {
  numeric_destroy(m);
  JFG_TRY(solve_attributes());
  NumericFactor* F = new NumericFactor();
  m->num = F;
  const Symbolic& S = m->sym();   // level lists sorted by sort_level_lists
  jfg_ctx* c = m->ctx;
  jfg_status st = JFG_OK;
  upload(S.sn_first, &F->first, c, st);
  upload(S.sn_m, &F->mrows, c, st);
  upload(S.level_sn, &F->level_sn, c, st);
  upload(S.ea_child, &F->ea_child, c, st);
  upload(S.rel, &F->rel, c, st);
  upload(S.rows, &F->rows, c, st);
  upload(S.sn_parent, &F->parent, c, st);
  upload(S.perm_dof, &F->perm_dof, c, st);
  upload(S.amap_src, &F->amap_src, c, st);
  upload(S.sn_Lptr, &F->Lptr, c, st);
  upload(S.sn_Uptr, &F->Uptr, c, st);
  upload(S.sn_rows_ptr, &F->rows_ptr, c, st);
  upload(S.sn_relptr, &F->relptr, c, st);
  upload(S.amap_dst, &F->amap_dst, c, st);
  // the pageable copies above run on the legacy stream and may still be in
  // flight when cudaMemcpy returns: finish them before the model's own
  // (non-blocking) stream reads the arrays
  if (st == JFG_OK && cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess) {
    set_error("uploading symbolic arrays failed");
    st = JFG_CUDA_ERROR;
  }
  // permuted (row, col) of every scattered entry, for the mixed scaling:
  // decoded on the device from the front slot through its supernode
  if (st == JFG_OK) {
    const int64_t na = (int64_t)S.amap_dst.size();
    if ((st = dev_alloc(c, (void**)&F->amap_pr, sizeof(int32_t) * std::max<int64_t>(na, 1))) == JFG_OK &&
        (st = dev_alloc(c, (void**)&F->amap_pc, sizeof(int32_t) * std::max<int64_t>(na, 1))) == JFG_OK && na > 0) {
      k_amap_rowcol<<<(unsigned)((na + 255) / 256), 256, 0, m->stream>>>(na, S.ns, F->amap_dst, F->Lptr, F->mrows,
                                                                       F->rows_ptr, F->rows, F->first, F->amap_pr,
                                                                       F->amap_pc);
      count_launch();
      if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(m->stream) != cudaSuccess) {
        set_error("decoding the scatter map failed");
        st = JFG_CUDA_ERROR;
      }
    }
  }
  if (st != JFG_OK) return st;
  F->n_amap = (int64_t)S.amap_dst.size();
  F->v_total = S.sn_relptr[S.ns];
  // levels and the tile lists of their launches
  {
    std::vector<int2> tl;
    build_levels(S, S.level_sn, F->levels, tl);
    F->n_tiles = (int64_t)tl.size();
    upload(tl, &F->tiles, c, st);
    if (st != JFG_OK) return st;
  }
  // strip metadata: 64-block inverse offsets, 256-strip inverse offsets with
  // their work items (front, strip, block column), per-level partial offsets
  {
    std::vector<int64_t> dptr(S.ns, 0), sptr(S.ns, 0), poff(S.ns, 0);
    std::vector<int32_t> isn, ikb, ijb;
    int64_t dl = 0, sl = 0;
    for (int64_t sn = 0; sn < S.ns; ++sn) {
      int64_t cc = S.sn_first[sn + 1] - S.sn_first[sn];
      int64_t nb = (cc + 63) / 64;
      dptr[sn] = dl;
      dl += nb * 64 * 64;
      sptr[sn] = sl;
      for (int64_t kb = 0; kb * 256 < cc; ++kb) {
        int64_t kw = std::min<int64_t>(256, cc - 256 * kb);
        sl += (kw == 256) ? 256 * 256 : kw * kw;
        for (int64_t jb = 0; jb * 64 < kw; ++jb) {
          isn.push_back((int32_t)sn); ikb.push_back((int32_t)kb); ijb.push_back((int32_t)jb);
        }
      }
    }
    int64_t pmax = 0;
    for (int64_t l = 0; l < S.n_levels; ++l) {
      int64_t acc = 0;
      for (int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
        int32_t sn = S.level_sn[q];
        int64_t cc = S.sn_first[sn + 1] - S.sn_first[sn];
        int64_t kw0 = std::min<int64_t>(256, cc);
        int64_t nrb0 = (S.sn_m[sn] - kw0 + 255) / 256;
        poff[q] = acc;
        acc += nrb0 * 256 * MAXR;
      }
      pmax = std::max(pmax, acc);
    }
    F->dinv_len = std::max<int64_t>(dl, 1);
    F->sinv_len = std::max<int64_t>(sl, 1);
    F->n_inv_items = (int64_t)isn.size();
    F->part_len = std::max<int64_t>(pmax, 1);
    upload(dptr, &F->Dptr, c, st);
    upload(sptr, &F->Sptr, c, st);
    upload(isn, &F->inv_sn, c, st);
    upload(ikb, &F->inv_kb, c, st);
    upload(ijb, &F->inv_jb, c, st);
    upload(poff, &F->part_off, c, st);
    if (st != JFG_OK) return st;
    JFG_TRY(dev_alloc(c, (void**)&F->part, sizeof(double) * F->part_len));
  }
  JFG_TRY(dev_alloc(c, (void**)&F->err, sizeof(DevError)));
  JFG_CUDA(cudaMemset(F->err, 0, sizeof(DevError)));
  {
    std::vector<uint8_t> mask(m->ndof);
    for (int64_t d = 0; d < m->ndof; ++d) mask[d] = S.gdof_to_perm[d] >= 0 ? 1 : 0;
    upload(mask, &F->free_mask, c, st);
    if (st != JFG_OK) return st;
  }
  JFG_TRY(dev_alloc(c, (void**)&F->norms, sizeof(double) * (256 * 64 + 64)));
  JFG_CUDA(cudaEventCreate(&F->ev0));
  JFG_CUDA(cudaEventCreate(&F->ev1));
  JFG_CUDA(cudaStreamSynchronize(cudaStreamLegacy));   // the pageable uploads and memsets above
  return JFG_OK;
}

void numeric_destroy(jfg_model* m) {
  NumericFactor* F = m->num;
  if (!F) return;
  jfg_ctx* c = m->ctx;
  // the factor's arrays go back to the pool: nothing on the model's stream
  // may still use them
  if (m->aev_out) cudaEventSynchronize(m->aev_out);
  cudaStreamSynchronize(m->stream);
  const Symbolic& S = m->sym();
  auto fr = [&](void* p, size_t b) { if (p) dev_free(c, p, b); };
  fr(F->first, 4 * (S.ns + 1)); fr(F->mrows, 4 * S.ns); fr(F->level_sn, 4 * S.ns);
  fr(F->ea_child, 4 * std::max<size_t>(S.ea_child.size(), 1)); fr(F->rel, 4 * std::max<size_t>(S.rel.size(), 1));
  fr(F->rows, 4 * S.rows.size()); fr(F->parent, 4 * S.ns); fr(F->perm_dof, 4 * S.n);
  fr(F->amap_src, 4 * S.amap_src.size()); fr(F->Lptr, 8 * (S.ns + 1)); fr(F->Uptr, 8 * S.ns);
  fr(F->rows_ptr, 8 * (S.ns + 1)); fr(F->relptr, 8 * (S.ns + 1)); fr(F->amap_dst, 8 * S.amap_dst.size());
  fr(F->amap_pr, 4 * S.amap_dst.size()); fr(F->amap_pc, 4 * S.amap_dst.size());
  fr(F->L64, 8 * S.nnz_L); fr(F->U64, 8 * std::max<int64_t>(S.u_arena, 1));
  fr(F->L32, 4 * S.nnz_L); fr(F->Phi, 4 * F->pk_len); fr(F->Plo, 4 * F->pk_len);
  fr(F->PKptr, 8 * (S.ns + 1)); fr(F->tc_zero, 8192); fr(F->U32, 4 * std::max<int64_t>(S.u_arena, 1));
  fr(F->scale, 8 * S.n);
  int oc = F->nrhs_cap;
  if (oc > 0) {
    fr(F->xp, 8 * S.n * oc); fr(F->tt, 8 * S.n * oc); fr(F->V, 8 * std::max<int64_t>(F->v_total, 1) * oc);
    fr(F->dF, 8 * m->ndof * oc); fr(F->dU, 8 * m->ndof * oc); fr(F->dR, 8 * m->ndof * oc);
    fr(F->dD, 8 * S.n * oc); fr(F->dZ, 8 * m->ndof * oc); fr(F->dP, 8 * m->ndof * oc); fr(F->dQ, 8 * m->ndof * oc);
  }
  fr(F->free_mask, m->ndof);
  fr(F->Dptr, 8 * S.ns); fr(F->Sptr, 8 * S.ns); fr(F->part_off, 8 * S.ns);
  fr(F->tiles, sizeof(int2) * std::max<int64_t>(F->n_tiles, 1));
  int64_t ni = std::max<int64_t>(F->n_inv_items, 1);
  fr(F->inv_sn, 4 * ni); fr(F->inv_kb, 4 * ni); fr(F->inv_jb, 4 * ni);
  fr(F->Dinv64, 8 * F->dinv_len); fr(F->Dinv32, 4 * F->dinv_len); fr(F->part, 8 * F->part_len);
  fr(F->Sinv64, 8 * F->sinv_len); fr(F->Sinv32, 4 * F->sinv_len);
  fr(F->err, sizeof(DevError));
  fr(F->norms, 8 * (256 * 64 + 64));
  if (F->ev0) cudaEventDestroy(F->ev0);
  if (F->ev1) cudaEventDestroy(F->ev1);
  drop_solve_graphs(F);
  for (auto& g : F->factor_graph)
    if (g) cudaGraphExecDestroy(g);
  delete F;
  m->num = nullptr;
}

jfg_status numeric_factor(jfg_model* m, int precision) {
  JFG_TRY(numeric_factor_enqueue(m, precision));
  return numeric_factor_finish(m, precision);
}

// Everything of the factorisation that goes on the model's stream; the
// first factorisation of a precision also allocates (and so synchronises).
jfg_status numeric_factor_enqueue(jfg_model* m, int precision) {
  NumericFactor* F = m->num;
  if (!F || !m->sym_ready) { set_error("factor before symbolic analysis"); return JFG_NOT_READY; }
  if (!m->values_ready) { set_error("factor before assembly"); return JFG_NOT_READY; }
  const Symbolic& S = m->sym();
  jfg_ctx* c = m->ctx;
  cudaStream_t st = m->stream;
  int64_t ublk = std::max<int64_t>(S.u_arena, 1);
  unsigned ga = (unsigned)((F->n_amap + 255) / 256);
  JFG_CUDA(cudaEventRecord(F->ev0, st));
  if (precision == JFG_PREC_FP64) {
    if (!F->L64) {
      JFG_TRY(dev_alloc(c, (void**)&F->L64, sizeof(double) * S.nnz_L));
      JFG_TRY(dev_alloc(c, (void**)&F->U64, sizeof(double) * ublk));
    }
    JFG_CUDA(cudaMemsetAsync(F->L64, 0, sizeof(double) * S.nnz_L, st));
    if (F->n_amap > 0)
      { k_scatter_A<double><<<ga, 256, 0, st>>>(F->n_amap, F->amap_src, F->amap_dst, F->amap_pr, F->amap_pc,
                                              m->d_nzval, nullptr, F->L64); count_launch(); }
    F->have64 = false;
    if (!F->Dinv64) JFG_TRY(dev_alloc(c, (void**)&F->Dinv64, sizeof(double) * F->dinv_len));
    if (!F->Sinv64) JFG_TRY(dev_alloc(c, (void**)&F->Sinv64, sizeof(double) * F->sinv_len));
    auto body = [&]() -> jfg_status {
      JFG_TRY(factor_levels<double>(m, F, F->L64, F->U64, F->Dinv64, false, st));
      return strip_inverses<double>(F, F->L64, F->Dinv64, F->Sinv64, st);
    };
    // the first factorisation runs eagerly (one-time kernel attributes);
    // later ones replay its graph
    if (F->factor_calls[0]++ > 0 && graphs_enabled())
      JFG_TRY(run_graph(F->factor_graph[0], F->factor_graph_nodes[0], st, body));
    else
      JFG_TRY(body());
  } else if (precision == JFG_PREC_MIXED) {
    if (!F->L32) {
      JFG_TRY(dev_alloc(c, (void**)&F->L32, sizeof(float) * S.nnz_L));
      JFG_TRY(dev_alloc(c, (void**)&F->U32, sizeof(float) * ublk));
      JFG_TRY(dev_alloc(c, (void**)&F->scale, sizeof(double) * S.n));
    }
    // symmetric diagonal scaling s_k = 1/sqrt(|K_kk|)
    JFG_CUDA(cudaMemsetAsync(F->L32, 0, sizeof(float) * S.nnz_L, st));
    { k_diag_scale<<<(unsigned)((S.n + 255) / 256), 256, 0, st>>>(S.n, F->perm_dof, m->d_diag_pos,
                                                              m->d_nzval, F->scale); count_launch(); }
    if (F->n_amap > 0)
      { k_scatter_A<float><<<ga, 256, 0, st>>>(F->n_amap, F->amap_src, F->amap_dst, F->amap_pr, F->amap_pc,
                                             m->d_nzval, F->scale, F->L32); count_launch(); }
    F->have32 = false;
    // tensor-core 3xTF32 updates for every model (JFG_TENSOR_CORES=0: FP32
    // SIMT).  The tensor core's own sums carry one-sided errors (truncating
    // accumulation in tensor memory, no lo*lo term), so their length is
    // chosen by model: shell models (thin-shell and drilling stiffness)
    // drain every 16-column K-slice into FP32 registers -- 9 refinement steps
    // on the 914k-DOF wing panel against 8 with the SIMT updates and 13 with
    // 64-column sums -- while solid-only models let the tensor core sum 64
    // columns (4 steps on the CTETRA10 block either way)
    const int tcs = tc::setting();
    const bool use_tc = tcs != 0;
    F->tc_drain = tc::drain_slices(m->n_q4 + m->n_q8 > 0 ? 1 : 4);
    if (use_tc && !F->Phi) {
      // packed operand images: ceil(c/16) x ceil(m/8) atoms of 128 floats per
      // front, offsets relative to the front's level region
      std::vector<int64_t> pk(S.ns + 1, 0);
      int64_t wmax = 0;
      for (auto& lv : F->levels) {
        int64_t acc = 0;
        for (int32_t q = lv.off; q < lv.off + lv.count; ++q) {
          const int32_t s = S.level_sn[q];
          const int64_t cs = S.sn_first[s + 1] - S.sn_first[s], ms = S.sn_m[s];
          pk[s] = acc;
          acc += ((cs + 15) / 16) * ((ms + 7) / 8) * 128;
        }
        lv.pk_len = acc;
        wmax = std::max(wmax, acc);
      }
      F->pk_len = std::max<int64_t>(wmax, 128);
      JFG_TRY(dev_alloc(c, (void**)&F->PKptr, sizeof(int64_t) * (S.ns + 1)));
      JFG_TRY(dev_alloc(c, (void**)&F->Phi, sizeof(float) * F->pk_len));
      JFG_TRY(dev_alloc(c, (void**)&F->Plo, sizeof(float) * F->pk_len));
      JFG_TRY(dev_alloc(c, (void**)&F->tc_zero, 8192));
      JFG_CUDA(cudaMemcpyAsync(F->PKptr, pk.data(), sizeof(int64_t) * (S.ns + 1), cudaMemcpyHostToDevice, st));
      JFG_CUDA(cudaMemsetAsync(F->tc_zero, 0, 8192, st));
      JFG_CUDA(cudaStreamSynchronize(st));   // pk is a host temporary
    }
    if (!F->Dinv32) JFG_TRY(dev_alloc(c, (void**)&F->Dinv32, sizeof(float) * F->dinv_len));
    if (!F->Sinv32) JFG_TRY(dev_alloc(c, (void**)&F->Sinv32, sizeof(float) * F->sinv_len));
    auto body = [&]() -> jfg_status {
      JFG_TRY(factor_levels<float>(m, F, F->L32, F->U32, F->Dinv32, use_tc, st));
      return strip_inverses<float>(F, F->L32, F->Dinv32, F->Sinv32, st);
    };
    if (F->factor_calls[1]++ > 0 && graphs_enabled())
      JFG_TRY(run_graph(F->factor_graph[1], F->factor_graph_nodes[1], st, body));
    else
      JFG_TRY(body());
  } else {
    set_error("unknown precision");
    return JFG_BAD_INPUT;
  }
  JFG_CUDA(cudaEventRecord(F->ev1, st));
  return JFG_OK;
}

// Device bytes of the numeric part of a model: `now` as allocated, `peak`
// once a factorisation at `precision` and a solve with `nrhs` right-hand
// sides have run (each allocation mirrored from numeric_create,
// numeric_factor_enqueue and ensure_workspace).
void numeric_bytes(jfg_model* m, int precision, int nrhs, int64_t* now, int64_t* peak) {
  const Symbolic& S = m->sym();
  NumericFactor* F = m->num;
  const int64_t ns = S.ns, n = S.n, ndof = m->ndof, na = (int64_t)S.amap_dst.size();
  int64_t base = 4 * (ns + 1) + 4 * ns + 4 * ns + 4 * std::max<int64_t>((int64_t)S.ea_child.size(), 1) +
                 4 * std::max<int64_t>((int64_t)S.rel.size(), 1) + 4 * (int64_t)S.rows.size() + 4 * ns + 4 * n +
                 4 * na + 8 * (ns + 1) + 8 * ns + 8 * (ns + 1) + 8 * (ns + 1) + 8 * na + 8 * na + 3 * 8 * ns +
                 8 * (256 * 64 + 64) + ndof + (int64_t)sizeof(DevError);
  int64_t items = 0, dl = 0, sl = 0;
  for (int64_t s = 0; s < ns; ++s) {
    const int64_t cc = S.sn_first[s + 1] - S.sn_first[s];
    dl += ((cc + 63) / 64) * 64 * 64;
    for (int64_t kb = 0; kb * 256 < cc; ++kb) {
      const int64_t kw = std::min<int64_t>(256, cc - 256 * kb);
      sl += kw * kw;
      items += (kw + 63) / 64;
    }
  }
  base += 12 * std::max<int64_t>(items, 1);
  const int64_t ublk = std::max<int64_t>(S.u_arena, 1);
  int64_t part = F ? F->part_len : 0;
  int64_t n_tiles = F ? F->n_tiles : 0;
  if (!F && S.ns > 0) {   // the tile lists numeric_create will build
    std::vector<int32_t> lsn = S.level_sn;
    sort_levels(S, lsn);
    std::vector<NumericFactor::Level> lv;
    std::vector<int2> tl;
    build_levels(S, lsn, lv, tl);
    n_tiles = (int64_t)tl.size();
  }
  base += 8 * part + 8 * std::max<int64_t>(n_tiles, 1);
  auto fp64 = [&]() { return 8 * S.nnz_L + 8 * ublk + 8 * std::max<int64_t>(dl, 1) + 8 * std::max<int64_t>(sl, 1); };
  auto mixed = [&]() {
    int64_t pk = 0;
    for (int64_t l = 0; l < S.n_levels; ++l) {
      int64_t acc = 0;
      for (int32_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
        const int32_t s = S.level_sn[q];
        acc += ((S.sn_first[s + 1] - S.sn_first[s] + 15) / 16) * ((S.sn_m[s] + 7) / 8) * 128;
      }
      pk = std::max(pk, acc);
    }
    return 4 * S.nnz_L + 4 * ublk + 8 * n + 4 * std::max<int64_t>(dl, 1) + 4 * std::max<int64_t>(sl, 1) +
           2 * 4 * std::max<int64_t>(pk, 128) + 8 * (ns + 1) + 8192;
  };
  auto work = [&](int cap) {
    const int64_t vt = std::max<int64_t>(S.sn_relptr.empty() ? 0 : S.sn_relptr[ns], 1);
    return 8 * cap * (3 * n + vt + 6 * ndof);
  };
  int64_t cur = base;
  if (F) {
    if (F->L64) cur += fp64();
    if (F->L32) cur += mixed();
    if (F->nrhs_cap > 0) cur += work(F->nrhs_cap);
  }
  const int cap = std::max(std::min(std::max(nrhs, 1), MAXR), F ? std::max(F->nrhs_cap, 8) : 8);
  int64_t pk = base + (precision == JFG_PREC_FP64 ? fp64() : mixed()) + work(cap);
  if (F && precision == JFG_PREC_FP64 && F->L32) pk += mixed();
  if (F && precision == JFG_PREC_MIXED && F->L64) pk += fp64();
  *now = cur;
  *peak = std::max(pk, cur);
}

// Precision of the factor a solve would use (-1: none).
int numeric_current_precision(jfg_model* m) {
  NumericFactor* F = m->num;
  if (!F) return -1;
  if (F->have32 && (!F->have64 || F->prefer_mixed)) return JFG_PREC_MIXED;
  return F->have64 ? JFG_PREC_FP64 : -1;
}

// Waits for the enqueued factorisation and reads its device error record.
jfg_status numeric_factor_finish(jfg_model* m, int precision) {
  NumericFactor* F = m->num;
  if (!F) { set_error("no factor"); return JFG_NOT_READY; }
  JFG_CUDA(cudaEventSynchronize(F->ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, F->ev0, F->ev1);
  m->t_factor = ms * 1e-3;
  prof_flush();
  JFG_TRY(check_err(F, "factorisation"));
  if (precision == JFG_PREC_FP64) F->have64 = true; else F->have32 = true;
  F->prefer_mixed = precision == JFG_PREC_MIXED;
  return JFG_OK;
}

// U = K_ff^{-1} F by one application of the factor (forward and backward
// sweeps, no refinement), F and U in device memory (ndof x nrhs, column-
// major, global DOF space; U is zero at fixed DOFs).  Enqueued on the
// model's stream; `precision` names the factor to use.
jfg_status numeric_apply(jfg_model* m, int nrhs, const double* Fd, double* Ud, int precision) {
  NumericFactor* F = m->num;
  if (!F) { set_error("apply before symbolic analysis"); return JFG_NOT_READY; }
  if (nrhs <= 0) { set_error("nrhs must be positive"); return JFG_BAD_INPUT; }
  const bool use32 = precision == JFG_PREC_MIXED;
  if ((use32 && !F->L32) || (!use32 && !F->L64)) { set_error("apply before factorisation"); return JFG_NOT_READY; }
  const Symbolic& S = m->sym();
  cudaStream_t st = m->stream;
  const int64_t n = S.n, ndof = m->ndof;
  const unsigned gn = (unsigned)((n + 255) / 256);
  for (int done = 0; done < nrhs;) {
    const int nr = std::min(MAXR, nrhs - done);
    JFG_TRY(ensure_workspace(m, F, nr));
    const double* sc = use32 ? F->scale : nullptr;
    { k_gather_perm<<<gn, 256, 0, st>>>(n, nr, F->perm_dof, sc, Fd + ndof * done, ndof, F->xp, 1.0); count_launch(); }
    auto body = [&]() -> jfg_status {
      if (use32) solve_inner<float>(m, F, F->L32, F->Sinv32, nr, st);
      else solve_inner<double>(m, F, F->L64, F->Sinv64, nr, st);
      return JFG_OK;
    };
    if (graphs_enabled()) JFG_TRY(run_graph(F->solve_graph[use32][nr], F->solve_graph_nodes[use32][nr], st, body));
    else JFG_TRY(body());
    JFG_CUDA(cudaMemsetAsync(Ud + ndof * done, 0, sizeof(double) * ndof * nr, st));
    { k_scatter_add_perm<<<gn, 256, 0, st>>>(n, nr, F->perm_dof, sc, F->xp, Ud + ndof * done, ndof); count_launch(); }
    done += nr;
  }
  return JFG_OK;
}

jfg_status numeric_factor_diag(jfg_model* m, double* out) {
  NumericFactor* F = m->num;
  if (!F || !(F->have64 || F->have32)) { set_error("no factor"); return JFG_NOT_READY; }
  const Symbolic& S = m->sym();
  cudaStream_t st = m->stream;
  double* d = nullptr;
  JFG_TRY(dev_alloc(m->ctx, (void**)&d, sizeof(double) * std::max<int64_t>(S.n, 1)));
  if (F->have64)
    { k_diag_of_factor64<<<(unsigned)S.ns, 128, 0, st>>>(S.ns, F->first, F->mrows, F->Lptr, F->L64, d); count_launch(); }
  else
    { k_diag_of_factor32<<<(unsigned)S.ns, 128, 0, st>>>(S.ns, F->first, F->mrows, F->Lptr, F->L32, F->scale, d); count_launch(); }
  JFG_CUDA(cudaMemcpyAsync(out, d, sizeof(double) * S.n, cudaMemcpyDeviceToHost, st));
  JFG_CUDA(cudaStreamSynchronize(st));
  dev_free(m->ctx, d, sizeof(double) * std::max<int64_t>(S.n, 1));
  return JFG_OK;
}

// Preconditioned conjugate gradients on K_ff in FP64 with the Cholesky factor
// (FP64, or the scaled mixed factor) as the preconditioner.  With the FP64
// factor the first iterate is the direct solution and one or two further
// steps polish it; with the mixed factor CG recovers FP64 accuracy.  Vectors
// live in the global DOF space with fixed DOFs held at zero; the matrix-vector
// product uses the FP64 CSC matrix.  Stagnation of the mixed preconditioner
// switches to the FP64 factor (restart from the current iterate).
jfg_status numeric_solve(jfg_model* m, int nrhs, const double* hF, double* hU, double tol, int max_ir,
                         jfg_solve_report* rep, bool device_io) {
  NumericFactor* F = m->num;
  if (!F || !(F->have64 || F->have32)) { set_error("solve before factor"); return JFG_NOT_READY; }
  if (nrhs <= 0) { set_error("nrhs must be positive"); return JFG_BAD_INPUT; }
  if (tol <= 0) tol = 1e-10;
  if (max_ir < 0) max_ir = 30;
  const Symbolic& S = m->sym();
  jfg_ctx* c = m->ctx;
  cudaStream_t st = m->stream;
  const int64_t n = S.n, ndof = m->ndof;
  const bool trace = std::getenv("JFG_IR_TRACE") != nullptr;
  JFG_CUDA(cudaEventRecord(F->ev0, st));
  jfg_solve_report R{};
  bool prefer32 = F->have32 && (!F->have64 || F->prefer_mixed);
  R.precision = prefer32 ? JFG_PREC_MIXED : JFG_PREC_FP64;
  const unsigned gn = (unsigned)((n + 255) / 256), gd = (unsigned)((ndof + 255) / 256);
  int done_rhs = 0;
  while (done_rhs < nrhs) {
    int nr = std::min(MAXR, nrhs - done_rhs);
    JFG_TRY(ensure_workspace(m, F, nr));
    double *X = F->dU, *Rv = F->dR, *Z = F->dZ, *Pv = F->dP, *Q = F->dQ;
    const double* srcF = hF + ndof * done_rhs;
    JFG_CUDA(cudaMemcpyAsync(F->dF, srcF, sizeof(double) * ndof * nr,
                             device_io ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    bool use32 = prefer32;
    auto precond = [&](const double* rin, double* zout) -> jfg_status {
      const double* sc = use32 ? F->scale : nullptr;
      { k_gather_perm<<<gn, 256, 0, st>>>(n, nr, F->perm_dof, sc, rin, ndof, F->xp, 1.0); count_launch(); }
      auto body = [&]() -> jfg_status {
        if (use32) solve_inner<float>(m, F, F->L32, F->Sinv32, nr, st);
        else solve_inner<double>(m, F, F->L64, F->Sinv64, nr, st);
        return JFG_OK;
      };
      if (graphs_enabled()) JFG_TRY(run_graph(F->solve_graph[use32][nr], F->solve_graph_nodes[use32][nr], st, body));
      else JFG_TRY(body());
      JFG_CUDA(cudaMemsetAsync(zout, 0, sizeof(double) * ndof * nr, st));
      { k_scatter_add_perm<<<gn, 256, 0, st>>>(n, nr, F->perm_dof, sc, F->xp, zout, ndof); count_launch(); }
      return JFG_OK;
    };
    auto matvec = [&](const double* x, double* y) {
      spmv_csc_sym(m, nr, x, ndof, y, ndof, st);
      { k_mask_free<<<gd, 256, 0, st>>>(ndof, nr, F->free_mask, y); count_launch(); }
    };
    // b = F restricted to the free DOFs
    JFG_CUDA(cudaMemcpyAsync(Rv, F->dF, sizeof(double) * ndof * nr, cudaMemcpyDeviceToDevice, st));
    { k_mask_free<<<gd, 256, 0, st>>>(ndof, nr, F->free_mask, Rv); count_launch(); }
    double bn[MAXR], rz[MAXR], pq[MAXR], rr[MAXR], rzn[MAXR];
    JFG_TRY(coldot(F, ndof, nr, Rv, Rv, bn, st));
    JFG_CUDA(cudaMemsetAsync(X, 0, sizeof(double) * ndof * nr, st));
    int it = 0, restarts = 0, stall = 0;
    double last_true = 1e300;
    double worst = 1.0, best = 1e300;
    bool fresh = true;
    for (;;) {
      if (fresh) {
        JFG_TRY(precond(Rv, Z));
        JFG_CUDA(cudaMemcpyAsync(Pv, Z, sizeof(double) * ndof * nr, cudaMemcpyDeviceToDevice, st));
        JFG_TRY(coldot(F, ndof, nr, Rv, Z, rz, st));
        fresh = false;
      }
      matvec(Pv, Q);
      JFG_TRY(coldot(F, ndof, nr, Pv, Q, pq, st));
      CoefR al{}, nal{};
      for (int k = 0; k < nr; ++k) {
        al.v[k] = (pq[k] > 0.0 && rz[k] > 0.0) ? rz[k] / pq[k] : 0.0;
        nal.v[k] = -al.v[k];
      }
      { k_axpy_cols<<<gd, 256, 0, st>>>(ndof, nr, al, Pv, X); count_launch(); }
      { k_axpy_cols<<<gd, 256, 0, st>>>(ndof, nr, nal, Q, Rv); count_launch(); }
      ++it;
      JFG_TRY(coldot(F, ndof, nr, Rv, Rv, rr, st));
      worst = 0.0;
      for (int k = 0; k < nr; ++k) worst = std::max(worst, bn[k] > 0 ? std::sqrt(rr[k] / bn[k]) : std::sqrt(rr[k]));
      if (trace)
        std::fprintf(stderr, "[jfg] pcg step %d (%s preconditioner): max recursive relative residual %.3e\n", it,
                     use32 ? "mixed" : "fp64", worst);
      bool conv = worst <= 0.5 * tol;
      stall = worst > 0.7 * best ? stall + 1 : 0;
      best = std::min(best, worst);
      if (conv || it >= max_ir || stall >= 3) {
        // true residual F - K x on the free DOFs (compensated)
        residual_dd(m, nr, X, F->dF, Rv, st);
        { k_mask_free<<<gd, 256, 0, st>>>(ndof, nr, F->free_mask, Rv); count_launch(); }
        JFG_TRY(coldot(F, ndof, nr, Rv, Rv, rr, st));
        worst = 0.0;
        for (int k = 0; k < nr; ++k) worst = std::max(worst, bn[k] > 0 ? std::sqrt(rr[k] / bn[k]) : std::sqrt(rr[k]));
        if (trace) std::fprintf(stderr, "[jfg] pcg true relative residual %.3e after %d steps\n", worst, it);
        if (worst <= tol || it >= max_ir || restarts >= 3 || worst > 0.9 * last_true) break;
        last_true = worst;
        // restart from the current iterate; a stalled mixed preconditioner is
        // replaced by the FP64 factor
        if (stall >= 3 && use32) {
          if (!F->have64) JFG_TRY(numeric_factor(m, JFG_PREC_FP64));
          use32 = false;
          R.fallback_used = 1;
          R.precision = JFG_PREC_FP64;
        }
        ++restarts;
        stall = 0;
        best = 1e300;
        fresh = true;
        continue;
      }
      JFG_TRY(precond(Rv, Z));
      JFG_TRY(coldot(F, ndof, nr, Rv, Z, rzn, st));
      CoefR be{};
      for (int k = 0; k < nr; ++k) be.v[k] = rz[k] > 0.0 ? rzn[k] / rz[k] : 0.0;
      { k_xpby_cols<<<gd, 256, 0, st>>>(ndof, nr, be, Z, Pv); count_launch(); }
      for (int k = 0; k < nr; ++k) rz[k] = rzn[k];
    }
    R.ir_iters = std::max(R.ir_iters, it);
    R.rel_residual = std::max(R.rel_residual, worst);
    double* dstU = hU + ndof * done_rhs;
    JFG_CUDA(cudaMemcpyAsync(dstU, X, sizeof(double) * ndof * nr,
                             device_io ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    done_rhs += nr;
  }
  JFG_CUDA(cudaEventRecord(F->ev1, st));
  JFG_CUDA(cudaEventSynchronize(F->ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, F->ev0, F->ev1);
  m->t_solve = ms * 1e-3;
  prof_flush();
  if (rep) *rep = R;
  if (R.rel_residual > tol) {
    set_error("refinement did not reach the tolerance", 0);
    return JFG_IR_STALLED;
  }
  return JFG_OK;
}

}  // namespace jfg
