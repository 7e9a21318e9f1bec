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
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "jfg_internal.h"
#include "tc_gemm.cuh"

struct NumericFactor {
  // symbolic arrays on the device
  int32_t *first = nullptr, *mrows = nullptr, *level_sn = nullptr, *ea_child = nullptr, *rel = nullptr,
          *rows = nullptr, *parent = nullptr, *perm_dof = nullptr, *amap_src = nullptr,
          *amap_pr = nullptr, *amap_pc = nullptr;
  int64_t *Lptr = nullptr, *Uptr = nullptr, *rows_ptr = nullptr, *relptr = nullptr, *amap_dst = nullptr;
  int64_t n_amap = 0;
  // host launch metadata
  struct Level {
    int32_t off, count;
    int32_t max_c, max_m, max_r;
    std::vector<std::pair<int32_t, int32_t>> ea;   // (offset into ea_child, count), per child rank
    int32_t ea_max_r;
    double schur_flops;   // sum over fronts of r(r+1) c (lower SYRK, 2 flops per FMA)
  };
  std::vector<Level> levels;
  // factor storage
  double* L64 = nullptr;
  double* U64 = nullptr;
  float* L32 = nullptr;
  float* U32 = nullptr;
  double* scale = nullptr;    // n, symmetric diagonal scaling of the mixed factor
  bool have64 = false, have32 = false;
  bool prefer_mixed = false;   // solve with the mixed factor when both exist
  // solve workspace
  int nrhs_cap = 0;
  double *xp = nullptr, *V = nullptr, *dF = nullptr, *dU = nullptr, *dR = nullptr, *dD = nullptr;
  double *norms = nullptr;
  int64_t v_total = 0;
  jfg::DevError* err = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace jfg {
namespace {

constexpr int NB = 32;       // panel block width
constexpr int TILE = 64;     // Schur-update tile

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

__global__ void k_diag_scale(int64_t n, const int32_t* __restrict__ perm_dof, const int64_t* __restrict__ diag_pos,
                             const double* __restrict__ nzval, double* __restrict__ scale) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int64_t p = diag_pos[perm_dof[k]];
  double d = p >= 0 ? fabs(nzval[p]) : 0.0;
  scale[k] = d > 0.0 ? 1.0 / sqrt(d) : 1.0;
}

template <typename T>
__global__ void k_zero_U(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
                         const int32_t* __restrict__ mrows, const int64_t* __restrict__ Uptr, T* __restrict__ U) {
  int s = list[blockIdx.y];
  int64_t up = Uptr[s];
  if (up < 0) return;
  int64_t r = mrows[s] - (first[s + 1] - first[s]);
  int64_t tot = r * r;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x)
    U[up + q] = (T)0;
}

// Extend-add of child update matrices into their parents' fronts.  One launch
// covers the children of one rank, so each parent receives one child.
template <typename T>
__global__ void k_extend_add(const int32_t* __restrict__ child, const int32_t* __restrict__ first,
                             const int32_t* __restrict__ mrows, const int32_t* __restrict__ parent,
                             const int64_t* __restrict__ Lptr, const int64_t* __restrict__ Uptr,
                             const int64_t* __restrict__ relptr, const int32_t* __restrict__ rel,
                             T* __restrict__ L, T* __restrict__ U) {
  int ch = child[blockIdx.y];
  int64_t uc = Uptr[ch];
  if (uc < 0) return;
  int rc = mrows[ch] - (first[ch + 1] - first[ch]);
  int cb = blockIdx.x * 8 + (threadIdx.x >> 5);   // one warp per child column
  if (cb >= rc) return;
  int lane = threadIdx.x & 31;
  int p = parent[ch];
  int cp = first[p + 1] - first[p];
  int mp = mrows[p];
  int rp = mp - cp;
  const int32_t* rl = rel + relptr[ch];
  int rb = rl[cb];
  const T* src = U + uc + (int64_t)rc * cb;
  if (rb < cp) {
    T* dst = L + Lptr[p] + (int64_t)mp * rb;
    for (int a = cb + lane; a < rc; a += 32) dst[rl[a]] += src[a];
  } else {
    T* dst = U + Uptr[p] + (int64_t)rp * (rb - cp) - cp;
    for (int a = cb + lane; a < rc; a += 32) dst[rl[a]] += src[a];
  }
}

template <typename T>
__global__ void k_potrf_diag(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
                             const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr,
                             T* __restrict__ L, int k0, DevError* err) {
  int s = list[blockIdx.x];
  int c = first[s + 1] - first[s];
  if (k0 >= c) return;
  int m = mrows[s];
  int kn = min(NB, c - k0);
  __shared__ T A[NB][NB + 1];
  int tx = threadIdx.x, ty = threadIdx.y;
  T* P = L + Lptr[s] + k0 + (int64_t)m * k0;
  A[ty][tx] = (ty < kn && tx < kn && ty >= tx) ? P[ty + (int64_t)m * tx] : (T)0;
  for (int j = 0; j < kn; ++j) {
    __syncthreads();
    if (tx == 0 && ty == 0) {
      T d = A[j][j];
      if (!(d > (T)0) || !isfinite((double)d)) {
        rec_err(err, EE_PIVOT, (int64_t)first[s] + k0 + j);
        d = (T)1;
      }
      A[j][j] = sqrt(d);
    }
    __syncthreads();
    if (tx == j && ty > j && ty < kn) A[ty][j] /= A[j][j];
    __syncthreads();
    if (tx > j && ty >= tx && ty < kn) A[ty][tx] -= A[ty][j] * A[tx][j];
  }
  __syncthreads();
  if (ty < kn && tx < kn && ty >= tx) P[ty + (int64_t)m * tx] = A[ty][tx];
}

// rows [k1, m) of panel columns [k0, k1):  X := X * L_D^{-T}
template <typename T>
__global__ void k_trsm_panel(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
                             const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr,
                             T* __restrict__ L, int k0) {
  int s = list[blockIdx.y];
  int c = first[s + 1] - first[s];
  if (k0 >= c) return;
  int m = mrows[s];
  int k1 = min(k0 + NB, c), kn = k1 - k0;
  __shared__ T D[NB][NB + 1];
  T* P = L + Lptr[s];
  for (int q = threadIdx.x; q < NB * NB; q += blockDim.x) {
    int i = q % NB, j = q / NB;
    D[i][j] = (i < kn && j < kn && i >= j) ? P[(k0 + i) + (int64_t)m * (k0 + j)] : (T)0;
  }
  __syncthreads();
  int i = k1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  T x[NB];
#pragma unroll
  for (int l = 0; l < NB; ++l) x[l] = l < kn ? P[i + (int64_t)m * (k0 + l)] : (T)0;
#pragma unroll
  for (int l = 0; l < NB; ++l) {
    if (l < kn) {
      T v = x[l];
#pragma unroll
      for (int q = 0; q < NB; ++q)
        if (q < l) v -= x[q] * D[l][q];
      x[l] = v / D[l][l];
    }
  }
#pragma unroll
  for (int l = 0; l < NB; ++l)
    if (l < kn) P[i + (int64_t)m * (k0 + l)] = x[l];
}

// Tile update C -= A_rows * B_rows^T (lower part).  mode 0: trailing panel
// columns after block k0; mode 1: Schur complement U -= L21 L21^T.
template <typename T>
__global__ void __launch_bounds__(256)
k_front_update(const int32_t* __restrict__ list, const int32_t* __restrict__ first,
               const int32_t* __restrict__ mrows, const int64_t* __restrict__ Lptr,
               const int64_t* __restrict__ Uptr, T* __restrict__ L, T* __restrict__ U, int mode, int k0) {
  int s = list[blockIdx.y];
  int c = first[s + 1] - first[s];
  int m = mrows[s];
  const T* P = L + Lptr[s];
  int row0, col0, nrow, ncol, kb, ke;
  T* C;
  int64_t ldc;
  if (mode == 0) {
    int k1 = min(k0 + NB, c);
    if (k0 >= c || k1 >= c) return;
    row0 = k1; col0 = k1; nrow = m - k1; ncol = c - k1; kb = k0; ke = k1;
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
  int t = blockIdx.x;
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
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      int i = ti * TILE + ty + 16 * a, j = tj * TILE + tx + 16 * b;
      if (i < nrow && j < ncol && row0 + i >= col0 + j) C[i + ldc * j] -= acc[a][b];
    }
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

__global__ void k_vec_extend_add(const int32_t* __restrict__ child, const int32_t* __restrict__ first,
                                 const int32_t* __restrict__ mrows, const int32_t* __restrict__ parent,
                                 const int64_t* __restrict__ relptr, const int32_t* __restrict__ rel, int nr,
                                 int64_t n, double* __restrict__ xp, double* __restrict__ V) {
  int ch = child[blockIdx.x];
  int rc = mrows[ch] - (first[ch + 1] - first[ch]);
  int p = parent[ch];
  int cp = first[p + 1] - first[p];
  int rp = mrows[p] - cp;
  const int32_t* rl = rel + relptr[ch];
  const double* src = V + relptr[ch] * nr;
  double* vp = V + relptr[p] * nr;
  for (int q = threadIdx.x; q < rc * nr; q += blockDim.x) {
    int a = q % rc, k = q / rc;
    int ra = rl[a];
    double v = src[a + (int64_t)rc * k];
    if (ra < cp) xp[first[p] + ra + n * k] += v;
    else vp[(ra - cp) + (int64_t)rp * k] += v;
  }
}

template <typename T>
__global__ void __launch_bounds__(256)
k_fwd(const int32_t* __restrict__ list, const int32_t* __restrict__ first, const int32_t* __restrict__ mrows,
      const int64_t* __restrict__ Lptr, const int64_t* __restrict__ relptr, const T* __restrict__ L, int nr,
      int64_t n, double* __restrict__ xp, double* __restrict__ V) {
  int s = list[blockIdx.x];
  int f = first[s], c = first[s + 1] - f, m = mrows[s], r = m - c;
  const T* P = L + Lptr[s];
  double* v = V + relptr[s] * nr;
  __shared__ double ys[NB][8];
  for (int jb = 0; jb < c; jb += NB) {
    int kn = min(NB, c - jb);
    if (threadIdx.x < 32) {
      int k = threadIdx.x;
      if (k < nr) {
        double y[NB];
#pragma unroll
        for (int l = 0; l < NB; ++l) y[l] = l < kn ? xp[f + jb + l + n * k] : 0.0;
#pragma unroll
        for (int l = 0; l < NB; ++l) {
          if (l < kn) {
            double t = y[l];
            for (int q = 0; q < l; ++q) t -= (double)P[(jb + l) + (int64_t)m * (jb + q)] * y[q];
            y[l] = t / (double)P[(jb + l) + (int64_t)m * (jb + l)];
            ys[l][k] = y[l];
            xp[f + jb + l + n * k] = y[l];
          }
        }
      }
    }
    __syncthreads();
    for (int i = jb + kn + threadIdx.x; i < m; i += blockDim.x) {
      double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int l = 0; l < kn; ++l) {
        double lv = (double)P[i + (int64_t)m * (jb + l)];
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] += lv * ys[l][k];
      }
      if (i < c) {
        for (int k = 0; k < nr; ++k) xp[f + i + n * k] -= acc[k];
      } else {
        for (int k = 0; k < nr; ++k) v[(i - c) + (int64_t)r * k] -= acc[k];
      }
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(256)
k_bwd(const int32_t* __restrict__ list, const int32_t* __restrict__ first, const int32_t* __restrict__ mrows,
      const int64_t* __restrict__ Lptr, const int64_t* __restrict__ rows_ptr, const int32_t* __restrict__ rows,
      const T* __restrict__ L, int nr, int64_t n, double* __restrict__ xp) {
  int s = list[blockIdx.x];
  int f = first[s], c = first[s + 1] - f, m = mrows[s];
  const T* P = L + Lptr[s];
  const int32_t* R = rows + rows_ptr[s];
  __shared__ double tsum[NB][8];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int nblk = (c + NB - 1) / NB;
  for (int bi = nblk - 1; bi >= 0; --bi) {
    int jb = bi * NB, kn = min(NB, c - jb);
    // t_l = sum_{i >= jb+kn} L[i, jb+l] x_i
    for (int l = warp; l < kn; l += 8) {
      double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      const T* col = P + (int64_t)m * (jb + l);
      for (int i = jb + kn + lane; i < m; i += 32) {
        double lv = (double)col[i];
        int64_t gi = R[i];
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if (k < nr) acc[k] += lv * xp[gi + n * k];
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) tsum[l][k] = v;
      }
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      int k = threadIdx.x;
      if (k < nr) {
        double x[NB];
        for (int l = kn - 1; l >= 0; --l) {
          double t = xp[f + jb + l + n * k] - tsum[l][k];
          for (int q = l + 1; q < kn; ++q) t -= (double)P[(jb + q) + (int64_t)m * (jb + l)] * x[q];
          x[l] = t / (double)P[(jb + l) + (int64_t)m * (jb + l)];
          xp[f + jb + l + n * k] = x[l];
        }
      }
    }
    __syncthreads();
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

// Per-column sums of squares of an n x nr block (deterministic two-level tree).
__global__ void k_colnorm2_partial(int64_t n, int nr, const double* __restrict__ x, double* __restrict__ part) {
  __shared__ double sh[256];
  int q = blockIdx.y;
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = x[i + n * q];
    s += v * v;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[q * gridDim.x + blockIdx.x] = sh[0];
}
__global__ void k_colnorm2_final(int nb, int nr, const double* __restrict__ part, double* __restrict__ out) {
  int q = threadIdx.x;
  if (q >= nr) return;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += part[q * nb + b];
  out[q] = s;
}

__global__ void k_copy_scale(int64_t n, int nr, const double* __restrict__ src, const double* __restrict__ scale,
                             double* __restrict__ dst) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double sc = scale ? scale[k] : 1.0;
  for (int q = 0; q < nr; ++q) dst[k + n * q] = src[k + n * q] * sc;
}

__global__ void k_axpy_sub(int64_t len, const double* __restrict__ a, const double* __restrict__ b,
                           double* __restrict__ out) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < len) out[k] = a[k] - b[k];
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

template <typename T>
void upload(std::vector<T>& h, T** d, jfg_ctx* c, jfg_status& st) {
  if (st != JFG_OK) return;
  size_t bytes = sizeof(T) * std::max<size_t>(h.size(), 1);
  st = dev_alloc(c, (void**)d, bytes);
  if (st != JFG_OK) return;
  if (!h.empty() && cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    set_error("cudaMemcpy failed uploading symbolic arrays");
    st = JFG_CUDA_ERROR;
  }
}

template <typename T>
jfg_status factor_levels(jfg_model* m, NumericFactor* F, T* Lf, T* Uf, cudaStream_t st) {
  const Symbolic& S = m->sym;
  for (const auto& lv : F->levels) {
    const int32_t* list = F->level_sn + lv.off;
    // zero the update matrices of this level's fronts
    if (lv.max_r > 0) {
      int64_t mx = (int64_t)lv.max_r * lv.max_r;
      unsigned gx = (unsigned)std::min<int64_t>((mx + 255) / 256, 4096);
      { k_zero_U<T><<<dim3(gx, lv.count), 256, 0, st>>>(list, F->first, F->mrows, F->Uptr, Uf); count_launch(); }
    }
    // extend-add children, one launch per child rank
    for (const auto& seg : lv.ea) {
      if (seg.second == 0) continue;
      unsigned gx = (unsigned)((lv.ea_max_r + 7) / 8);
      if (gx == 0) continue;
      { k_extend_add<T><<<dim3(gx, seg.second), 256, 0, st>>>(F->ea_child + seg.first, F->first, F->mrows,
                                                            F->parent, F->Lptr, F->Uptr, F->relptr, F->rel, Lf, Uf); count_launch(); }
    }
    // blocked partial factorisation of every front of the level
    for (int k0 = 0; k0 < lv.max_c; k0 += NB) {
      { k_potrf_diag<T><<<lv.count, dim3(NB, NB), 0, st>>>(list, F->first, F->mrows, F->Lptr, Lf, k0, F->err); count_launch(); }
      int rows_max = lv.max_m - k0 - 1;
      if (rows_max > 0) {
        unsigned gx = (unsigned)((rows_max + 127) / 128);
        { k_trsm_panel<T><<<dim3(gx, lv.count), 128, 0, st>>>(list, F->first, F->mrows, F->Lptr, Lf, k0); count_launch(); }
        int nrow = lv.max_m - k0 - NB, ncol = lv.max_c - k0 - NB;
        if (nrow > 0 && ncol > 0) {
          int64_t tiles = (int64_t)((nrow + TILE - 1) / TILE) * ((ncol + TILE - 1) / TILE);
          { k_front_update<T><<<dim3((unsigned)tiles, lv.count), 256, 0, st>>>(list, F->first, F->mrows, F->Lptr,
                                                                          F->Uptr, Lf, Uf, 0, k0); count_launch(); }
        }
      }
    }
    if (lv.max_r > 0) {
      int64_t nt = (lv.max_r + TILE - 1) / TILE;
      int64_t tiles = nt * nt;
      bool done = false;
      int ps = prof_start(st);
      if constexpr (sizeof(T) == 4) {
        done = tc::schur_update_tf32x3(list, lv.count, F->first, F->mrows, F->Lptr, F->Uptr, Lf, Uf,
                                       lv.max_r, lv.max_c, st);
      }
      if (!done)
        { k_front_update<T><<<dim3((unsigned)tiles, lv.count), 256, 0, st>>>(list, F->first, F->mrows, F->Lptr,
                                                                        F->Uptr, Lf, Uf, 1, 0); count_launch(); }
      prof_end(ps, st, KS_SCHUR, lv.schur_flops);
    }
    JFG_CUDA(cudaGetLastError());
  }
  (void)S;
  return JFG_OK;
}

template <typename T>
void solve_inner(jfg_model* m, NumericFactor* F, const T* Lf, int nr, cudaStream_t st) {
  const Symbolic& S = m->sym;
  int64_t n = S.n;
  int ps = prof_start(st);
  // forward, leaves first
  for (size_t li = 0; li < F->levels.size(); ++li) {
    const auto& lv = F->levels[li];
    const int32_t* list = F->level_sn + lv.off;
    { k_zero_V<<<lv.count, 256, 0, st>>>(list, F->first, F->mrows, F->relptr, nr, F->V); count_launch(); }
    for (const auto& seg : lv.ea)
      if (seg.second > 0)
        { k_vec_extend_add<<<seg.second, 256, 0, st>>>(F->ea_child + seg.first, F->first, F->mrows, F->parent,
                                                     F->relptr, F->rel, nr, n, F->xp, F->V); count_launch(); }
    { k_fwd<T><<<lv.count, 256, 0, st>>>(list, F->first, F->mrows, F->Lptr, F->relptr, Lf, nr, n, F->xp, F->V); count_launch(); }
  }
  // backward, root first
  for (size_t li = F->levels.size(); li-- > 0;) {
    const auto& lv = F->levels[li];
    const int32_t* list = F->level_sn + lv.off;
    { k_bwd<T><<<lv.count, 256, 0, st>>>(list, F->first, F->mrows, F->Lptr, F->rows_ptr, F->rows, Lf, nr, n,
                                       F->xp); count_launch(); }
  }
  // algorithmic bytes: the factor read twice (forward and backward) plus the
  // permuted vectors read and written in each sweep
  prof_end(ps, st, KS_SOLVE, 2.0 * sizeof(T) * (double)S.nnz_L + 4.0 * 8.0 * n * nr);
}

jfg_status ensure_workspace(jfg_model* m, NumericFactor* F, int nrhs) {
  if (nrhs <= F->nrhs_cap) return JFG_OK;
  jfg_ctx* c = m->ctx;
  auto fr = [&](double*& p, int64_t len) {
    if (p) dev_free(c, p, sizeof(double) * len);
    p = nullptr;
  };
  int64_t n = m->sym.n, ndof = m->ndof;
  if (F->nrhs_cap > 0) {
    int oc = F->nrhs_cap;
    fr(F->xp, n * oc); fr(F->V, F->v_total * oc); fr(F->dF, ndof * oc); fr(F->dU, ndof * oc);
    fr(F->dR, ndof * oc); fr(F->dD, n * oc);
  }
  int cap = std::max(nrhs, 8);
  JFG_TRY(dev_alloc(c, (void**)&F->xp, sizeof(double) * n * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->V, sizeof(double) * std::max<int64_t>(F->v_total, 1) * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->dF, sizeof(double) * ndof * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->dU, sizeof(double) * ndof * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->dR, sizeof(double) * ndof * cap));
  JFG_TRY(dev_alloc(c, (void**)&F->dD, sizeof(double) * n * cap));
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
  return JFG_OK;
}

// per-RHS squared norms of the n x nr block x (result on host)
jfg_status colnorm2(NumericFactor* F, int64_t n, int nr, const double* x, double* out_host, cudaStream_t st) {
  const int nb = 256;
  { k_colnorm2_partial<<<dim3(nb, nr), 256, 0, st>>>(n, nr, x, F->norms); count_launch(); }
  { k_colnorm2_final<<<1, 64, 0, st>>>(nb, nr, F->norms, F->norms + nb * 64); count_launch(); }
  JFG_CUDA(cudaMemcpyAsync(out_host, F->norms + nb * 64, sizeof(double) * nr, cudaMemcpyDeviceToHost, st));
  JFG_CUDA(cudaStreamSynchronize(st));
  return JFG_OK;
}

}  // namespace

jfg_status numeric_create(jfg_model* m) {
  numeric_destroy(m);
  NumericFactor* F = new NumericFactor();
  m->num = F;
  Symbolic& S = m->sym;
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
  // permuted (row, col) of every scattered entry, for the mixed scaling
  {
    std::vector<int32_t> pr(S.amap_dst.size()), pc(S.amap_dst.size());
    std::vector<int32_t> col_of(S.n);
    for (int64_t s = 0; s < S.ns; ++s)
      for (int64_t k = S.sn_first[s]; k < S.sn_first[s + 1]; ++k) col_of[k] = (int32_t)s;
    // decode dst -> (front row, front col) through the supernode that owns it
    std::vector<int64_t> Lp = S.sn_Lptr;
    for (size_t q = 0; q < S.amap_dst.size(); ++q) {
      int64_t d = S.amap_dst[q];
      int64_t s = std::upper_bound(Lp.begin(), Lp.end(), d) - Lp.begin() - 1;
      int64_t mm = S.sn_m[s];
      int64_t off = d - Lp[s];
      int64_t ri = off % mm, cj = off / mm;
      pr[q] = S.rows[S.sn_rows_ptr[s] + ri];
      pc[q] = S.sn_first[s] + (int32_t)cj;
    }
    upload(pr, &F->amap_pr, c, st);
    upload(pc, &F->amap_pc, c, st);
  }
  if (st != JFG_OK) return st;
  F->n_amap = (int64_t)S.amap_dst.size();
  F->v_total = S.sn_relptr[S.ns];
  // levels
  F->levels.resize(S.n_levels);
  for (int64_t l = 0; l < S.n_levels; ++l) {
    auto& lv = F->levels[l];
    lv.off = S.level_ptr[l];
    lv.count = S.level_ptr[l + 1] - S.level_ptr[l];
    lv.max_c = lv.max_m = lv.max_r = 0;
    for (int32_t q = lv.off; q < lv.off + lv.count; ++q) {
      int32_t s = S.level_sn[q];
      int32_t cc = S.sn_first[s + 1] - S.sn_first[s];
      lv.max_c = std::max(lv.max_c, cc);
      lv.max_m = std::max(lv.max_m, S.sn_m[s]);
      if (S.sn_parent[s] >= 0) lv.max_r = std::max(lv.max_r, S.sn_m[s] - cc);
    }
    lv.schur_flops = 0;
    for (int32_t q = lv.off; q < lv.off + lv.count; ++q) {
      int32_t s = S.level_sn[q];
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
  JFG_TRY(dev_alloc(c, (void**)&F->err, sizeof(DevError)));
  JFG_CUDA(cudaMemset(F->err, 0, sizeof(DevError)));
  JFG_TRY(dev_alloc(c, (void**)&F->norms, sizeof(double) * (256 * 64 + 64)));
  JFG_CUDA(cudaEventCreate(&F->ev0));
  JFG_CUDA(cudaEventCreate(&F->ev1));
  return JFG_OK;
}

void numeric_destroy(jfg_model* m) {
  NumericFactor* F = m->num;
  if (!F) return;
  jfg_ctx* c = m->ctx;
  const Symbolic& S = m->sym;
  auto fr = [&](void* p, size_t b) { if (p) dev_free(c, p, b); };
  fr(F->first, 4 * (S.ns + 1)); fr(F->mrows, 4 * S.ns); fr(F->level_sn, 4 * S.ns);
  fr(F->ea_child, 4 * std::max<size_t>(S.ea_child.size(), 1)); fr(F->rel, 4 * std::max<size_t>(S.rel.size(), 1));
  fr(F->rows, 4 * S.rows.size()); fr(F->parent, 4 * S.ns); fr(F->perm_dof, 4 * S.n);
  fr(F->amap_src, 4 * S.amap_src.size()); fr(F->Lptr, 8 * (S.ns + 1)); fr(F->Uptr, 8 * S.ns);
  fr(F->rows_ptr, 8 * (S.ns + 1)); fr(F->relptr, 8 * (S.ns + 1)); fr(F->amap_dst, 8 * S.amap_dst.size());
  fr(F->amap_pr, 4 * S.amap_dst.size()); fr(F->amap_pc, 4 * S.amap_dst.size());
  fr(F->L64, 8 * S.nnz_L); fr(F->U64, 8 * std::max<int64_t>(S.u_arena, 1));
  fr(F->L32, 4 * S.nnz_L); fr(F->U32, 4 * std::max<int64_t>(S.u_arena, 1));
  fr(F->scale, 8 * S.n);
  int oc = F->nrhs_cap;
  if (oc > 0) {
    fr(F->xp, 8 * S.n * oc); fr(F->V, 8 * std::max<int64_t>(F->v_total, 1) * oc);
    fr(F->dF, 8 * m->ndof * oc); fr(F->dU, 8 * m->ndof * oc); fr(F->dR, 8 * m->ndof * oc);
    fr(F->dD, 8 * S.n * oc);
  }
  fr(F->err, sizeof(DevError));
  fr(F->norms, 8 * (256 * 64 + 64));
  if (F->ev0) cudaEventDestroy(F->ev0);
  if (F->ev1) cudaEventDestroy(F->ev1);
  delete F;
  m->num = nullptr;
}

jfg_status numeric_factor(jfg_model* m, int precision) {
  NumericFactor* F = m->num;
  if (!F || !m->sym_ready) { set_error("factor before symbolic analysis"); return JFG_NOT_READY; }
  if (!m->values_ready) { set_error("factor before assembly"); return JFG_NOT_READY; }
  const Symbolic& S = m->sym;
  jfg_ctx* c = m->ctx;
  cudaStream_t st = c->stream;
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
    JFG_TRY(factor_levels<double>(m, F, F->L64, F->U64, st));
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
    JFG_TRY(factor_levels<float>(m, F, F->L32, F->U32, st));
  } else {
    set_error("unknown precision");
    return JFG_BAD_INPUT;
  }
  JFG_CUDA(cudaEventRecord(F->ev1, st));
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

jfg_status numeric_factor_diag(jfg_model* m, double* out) {
  NumericFactor* F = m->num;
  if (!F || !(F->have64 || F->have32)) { set_error("no factor"); return JFG_NOT_READY; }
  const Symbolic& S = m->sym;
  cudaStream_t st = m->ctx->stream;
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

jfg_status numeric_solve(jfg_model* m, int nrhs, const double* hF, double* hU, double tol, int max_ir,
                         jfg_solve_report* rep, bool device_io) {
  NumericFactor* F = m->num;
  if (!F || !(F->have64 || F->have32)) { set_error("solve before factor"); return JFG_NOT_READY; }
  if (nrhs <= 0) { set_error("nrhs must be positive"); return JFG_BAD_INPUT; }
  if (tol <= 0) tol = 1e-10;
  if (max_ir < 0) max_ir = 10;
  const Symbolic& S = m->sym;
  jfg_ctx* c = m->ctx;
  cudaStream_t st = c->stream;
  int64_t n = S.n, ndof = m->ndof;
  JFG_CUDA(cudaEventRecord(F->ev0, st));
  int done_rhs = 0;
  jfg_solve_report R{};
  R.precision = F->have32 && !F->have64 ? JFG_PREC_MIXED : JFG_PREC_FP64;
  bool prefer32 = F->have32 && (!F->have64 || F->prefer_mixed);
  if (prefer32) R.precision = JFG_PREC_MIXED;
  while (done_rhs < nrhs) {
    int nr = std::min(8, nrhs - done_rhs);
    JFG_TRY(ensure_workspace(m, F, nr));
    const double* srcF = hF + ndof * done_rhs;
    JFG_CUDA(cudaMemcpyAsync(F->dF, srcF, sizeof(double) * ndof * nr,
                             device_io ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    JFG_CUDA(cudaMemsetAsync(F->dU, 0, sizeof(double) * ndof * nr, st));
    unsigned gn = (unsigned)((n + 255) / 256);
    // r = F_ff (u = 0), permuted, and ||F_ff||
    { k_gather_perm<<<gn, 256, 0, st>>>(n, nr, F->perm_dof, nullptr, F->dF, ndof, F->dD, 1.0); count_launch(); }
    double fn[8], rn[8], prev[8];
    JFG_TRY(colnorm2(F, n, nr, F->dD, fn, st));
    bool use32 = prefer32;
    int it = 0, stall_count = 0;
    double rn_max_prev = 1e300;
    double worst = 0;
    for (int q = 0; q < nr; ++q) prev[q] = 1e300;
    for (;;) {
      const double* sc = use32 ? F->scale : nullptr;
      int64_t len = n * nr;
      { k_copy_scale<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, nr, F->dD, sc, F->xp); count_launch(); }
      if (use32) solve_inner<float>(m, F, F->L32, nr, st);
      else solve_inner<double>(m, F, F->L64, nr, st);
      { k_scatter_add_perm<<<gn, 256, 0, st>>>(n, nr, F->perm_dof, sc, F->xp, F->dU, ndof); count_launch(); }
      // R = F - K u over all DOFs; its free part is the next right-hand side
      spmv_csc_sym(m, nr, F->dU, ndof, F->dR, ndof, st);
      int64_t lg = ndof * nr;
      { k_axpy_sub<<<(unsigned)((lg + 255) / 256), 256, 0, st>>>(lg, F->dF, F->dR, F->dR); count_launch(); }
      { k_gather_perm<<<gn, 256, 0, st>>>(n, nr, F->perm_dof, nullptr, F->dR, ndof, F->dD, 1.0); count_launch(); }
      (void)len;
      JFG_TRY(colnorm2(F, n, nr, F->dD, rn, st));
      worst = 0;
      for (int q = 0; q < nr; ++q) {
        double rel = fn[q] > 0 ? sqrt(rn[q] / fn[q]) : sqrt(rn[q]);
        rn[q] = rel;
        worst = std::max(worst, rel);
      }
      if (std::getenv("JFG_IR_TRACE"))
        std::fprintf(stderr, "[jfg] ir step %d (%s factor): max relative residual %.3e\n", it,
                     use32 ? "mixed" : "fp64", worst);
      if (worst <= tol || it >= max_ir) break;
      // stagnation: a step that does not reduce some unconverged residual by
      // at least 10 % counts as stalled; two stalled steps in a row end the
      // refinement (after a switch to the FP64 factor for the mixed path)
      bool stalled = false;
      for (int q = 0; q < nr; ++q)
        if (rn[q] > tol && rn[q] > 0.9 * prev[q]) stalled = true;
      stall_count = stalled ? stall_count + 1 : 0;
      if (stall_count >= 2 || (stalled && use32 && rn_max_prev < worst)) {
        if (use32) {
          // refinement with the mixed factor stalls: FP64 factor fallback
          if (!F->have64) JFG_TRY(numeric_factor(m, JFG_PREC_FP64));
          use32 = false;
          stall_count = 0;
          R.fallback_used = 1;
          R.precision = JFG_PREC_FP64;
        } else {
          break;
        }
      }
      rn_max_prev = worst;
      for (int q = 0; q < nr; ++q) prev[q] = rn[q];
      ++it;
    }
    R.ir_iters = std::max(R.ir_iters, it);
    R.rel_residual = std::max(R.rel_residual, worst);
    double* dstU = hU + ndof * done_rhs;
    JFG_CUDA(cudaMemcpyAsync(dstU, F->dU, sizeof(double) * ndof * nr,
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
    set_error("iterative refinement did not reach the tolerance", 0);
    return JFG_IR_STALLED;
  }
  return JFG_OK;
}

}  // namespace jfg
