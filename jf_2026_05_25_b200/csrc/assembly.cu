// assembly.cu -- global CSC pattern, triplet slot map and the device assembly.
//
// Semantics of K = sparse(I,J,V,ndof,ndof) (src/solver/assembly.jl:5942):
// pattern = every (I,J) emitted by an element (explicit zeros kept); values =
// duplicates combined left to right in triplet order (:5963-5974).  The
// triplet order is the element order: all CQUAD4 (positional slots
// (ei-1)*576, :3506-3508), then the CTETRA10 (900 each, :5882-5884).
//
// The pattern is built once per mesh on the host from the node-pair blocks of
// the connectivity.  The device assembly is a gather: every CSC entry sums its
// own contributions, in triplet order, from the element value buffer -- no
// atomics, bitwise deterministic, and the same summation order as Julia.
#include <omp.h>

#include <algorithm>

#include <cstring>

#include "jfg_internal.h"

namespace jfg {
namespace {

constexpr uint64_t MASK_Q4 = (1ull << 36) - 1;   // all 6x6 component pairs
uint64_t mask_t10() {
  uint64_t m = 0;
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) m |= 1ull << (i + 6 * j);
  return m;
}

struct ElemRef {
  int64_t e;        // global element order: Q4 first, then T10, then Q8
  int8_t local;     // local index of the column node in the element
};

__global__ void k_assemble(int64_t nnz, const int32_t* __restrict__ nzptr,
                           const int32_t* __restrict__ trip, const double* __restrict__ ev,
                           double* __restrict__ nzval) {
  int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nnz) return;
  int32_t a = nzptr[q], b = nzptr[q + 1];
  double v = ev[trip[a]];
  for (int32_t k = a + 1; k < b; ++k) v = v + ev[trip[k]];
  nzval[q] = v;
}

// y = K x with K in CSC and a structurally symmetric pattern: row i of K is
// gathered through the transpose positions (one warp per row).
__global__ void k_spmv(int64_t n, const int64_t* __restrict__ colptr, const int32_t* __restrict__ rowval,
                       const int64_t* __restrict__ tpos, const double* __restrict__ nzval, int nrhs,
                       const double* __restrict__ x, int64_t ldx, double* __restrict__ y, int64_t ldy) {
  int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (row >= n) return;
  int64_t a = colptr[row], b = colptr[row + 1];
  for (int r0 = 0; r0 < nrhs; r0 += 8) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int nr = min(8, nrhs - r0);
    for (int64_t p = a + lane; p < b; p += 32) {
      double kv = nzval[tpos[p]];
      int64_t col = rowval[p];
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (k < nr) acc[k] += kv * x[col + ldx * (r0 + k)];
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      double v = acc[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0 && k < nr) y[row + ldy * (r0 + k)] = v;
    }
  }
}

// r = F - K x with error-free transformations (FMA product error + two-sum)
// per row: the residual carries no rounding from the cancelling row sums of
// the stiffness matrix, only the final rounding.
__global__ void k_residual_dd(int64_t n, const int64_t* __restrict__ colptr, const int32_t* __restrict__ rowval,
                              const int64_t* __restrict__ tpos, const double* __restrict__ nzval, int nrhs,
                              const double* __restrict__ x, const double* __restrict__ f, int64_t ld,
                              double* __restrict__ r) {
  int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (row >= n) return;
  int64_t a = colptr[row], b = colptr[row + 1];
  for (int k = 0; k < nrhs; ++k) {
    double hi = 0.0, lo = 0.0;
    for (int64_t p = a + lane; p < b; p += 32) {
      double kv = nzval[tpos[p]];
      double xv = x[rowval[p] + ld * k];
      double prod = kv * xv;
      double perr = fma(kv, xv, -prod);
      double s = hi + prod;
      double bp = s - hi;
      double serr = (hi - (s - bp)) + (prod - bp);
      hi = s;
      lo += serr + perr;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double h2 = __shfl_down_sync(0xffffffffu, hi, o);
      double l2 = __shfl_down_sync(0xffffffffu, lo, o);
      double s = hi + h2;
      double bp = s - hi;
      double serr = (hi - (s - bp)) + (h2 - bp);
      hi = s;
      lo += l2 + serr;
    }
    if (lane == 0) {
      // f - (hi + lo) in two-sum form
      double fv = f[row + ld * k];
      double s = fv - hi;
      double bp = s - fv;
      double serr = (fv - (s - bp)) + (-hi - bp);
      r[row + ld * k] = s + (serr - lo);
    }
  }
}

}  // namespace

namespace {

__global__ void k_gather_diag(int64_t ndof, const int64_t* __restrict__ diag_pos, const double* __restrict__ nzval,
                              double* __restrict__ out) {
  const int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (d < ndof) out[d] = diag_pos[d] >= 0 ? nzval[diag_pos[d]] : 0.0;
}

// max |v| over n values: per-thread maxima, a warp reduction, one atomic
// per warp on the bit pattern (non-negative doubles order like their bits)
__global__ void k_absmax(int64_t n, const double* __restrict__ v, unsigned long long* __restrict__ out) {
  double mx = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    mx = fmax(mx, fabs(v[i]));
  for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(mx));
}

// the 3 x 3 translational and rotational diagonal blocks of every grid:
// thread (node, entry) finds its row in its column by bisection
__global__ void k_node_blocks(int64_t n_nodes, const int64_t* __restrict__ colptr, const int32_t* __restrict__ rowval,
                              const double* __restrict__ nzval, double* __restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 18 * n_nodes) return;
  const int64_t n = t / 18;
  const int k = (int)(t - 18 * n), off = k / 9, a = k % 3, b = (k % 9) / 3;
  const int64_t col = 6 * n + 3 * off + b, row = 6 * n + 3 * off + a;
  int64_t lo = colptr[col], hi = colptr[col + 1];
  double val = 0.0;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    const int32_t r = rowval[mid];
    if (r == row) { val = nzval[mid]; break; }
    if (r < row) lo = mid + 1; else hi = mid;
  }
  out[t] = val;
}

}  // namespace

jfg_status device_diag(jfg_model* m, double* diag, double* max_elem_stiff) {
  cudaStream_t st = m->stream;
  double* d = nullptr;
  unsigned long long* mx = nullptr;
  JFG_TRY(dev_alloc(m->ctx, (void**)&d, sizeof(double) * std::max<int64_t>(m->ndof, 1) + 64));
  mx = reinterpret_cast<unsigned long long*>(d + std::max<int64_t>(m->ndof, 1));
  jfg_status s = JFG_OK;
  if (cudaMemsetAsync(mx, 0, sizeof(unsigned long long), st) != cudaSuccess) s = JFG_CUDA_ERROR;
  if (s == JFG_OK && diag) {
    k_gather_diag<<<(unsigned)((m->ndof + 255) / 256), 256, 0, st>>>(m->ndof, m->d_diag_pos, m->d_nzval, d);
    count_launch();
  }
  if (s == JFG_OK && max_elem_stiff && m->n_ev > 0) {
    const int64_t blocks = std::min<int64_t>((m->n_ev + 255) / 256, 148 * 16);
    k_absmax<<<(unsigned)blocks, 256, 0, st>>>(m->n_ev, m->d_ev, mx);
    count_launch();
  }
  unsigned long long bits = 0;
  if (s == JFG_OK && (cudaGetLastError() != cudaSuccess ||
                      (diag && cudaMemcpyAsync(diag, d, sizeof(double) * m->ndof, cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
                      cudaMemcpyAsync(&bits, mx, sizeof(bits), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                      cudaStreamSynchronize(st) != cudaSuccess))
    s = JFG_CUDA_ERROR;
  dev_free(m->ctx, d, sizeof(double) * std::max<int64_t>(m->ndof, 1) + 64);
  if (s != JFG_OK) { set_error("device diagonal / element maximum failed"); return s; }
  if (max_elem_stiff) {
    double v;
    std::memcpy(&v, &bits, sizeof v);
    *max_elem_stiff = v;
  }
  return JFG_OK;
}

jfg_status device_node_blocks(jfg_model* m, double* blocks) {
  cudaStream_t st = m->stream;
  const int64_t len = 18 * m->n_nodes;
  double* d = nullptr;
  JFG_TRY(dev_alloc(m->ctx, (void**)&d, sizeof(double) * std::max<int64_t>(len, 1)));
  k_node_blocks<<<(unsigned)((len + 255) / 256), 256, 0, st>>>(m->n_nodes, m->d_colptr, m->d_rowval, m->d_nzval, d);
  count_launch();
  jfg_status s = JFG_OK;
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(blocks, d, sizeof(double) * len, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    s = JFG_CUDA_ERROR;
  dev_free(m->ctx, d, sizeof(double) * std::max<int64_t>(len, 1));
  if (s != JFG_OK) set_error("device node blocks failed");
  return s;
}

void residual_dd(const jfg_model* m, int nrhs, const double* x, const double* f, double* r, cudaStream_t st) {
  int64_t threads = m->ndof * 32;
  int64_t blocks = (threads + 255) / 256;
  { k_residual_dd<<<(unsigned)blocks, 256, 0, st>>>(m->ndof, m->d_colptr, m->d_rowval, m->d_tpos, m->d_nzval, nrhs, x,
                                                   f, m->ndof, r); count_launch(); }
}

jfg_status build_pattern(jfg_model* m) {
  const int64_t nn = m->n_nodes, ndof = m->ndof;
  const int64_t nq4 = m->n_q4, nt10 = m->n_t10, nq8 = m->n_q8, nt3 = m->n_t3;
  const uint64_t mt10 = mask_t10();
  // CQUAD8 emits only its nonzero entries (assembly.jl:5912-5916), so its
  // part of the pattern depends on the element values computed just before:
  // per element and node pair a 6x6 component mask, per column a 48-bit row
  // mask and the number of nonzeros in the earlier columns.
  std::vector<uint64_t> q8pair(64 * nq8), q8col(48 * nq8);
  std::vector<int32_t> q8pref(49 * nq8);
  std::vector<int64_t> q8off(nq8 + 1, 0);
  if (nq8 > 0) {
    std::vector<double> v(2304 * nq8);
    JFG_CUDA(cudaMemcpy(v.data(), m->d_ev + m->ev_q8_off, sizeof(double) * v.size(), cudaMemcpyDeviceToHost));
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < nq8; ++e) {
      const double* K = v.data() + 2304 * e;
      int32_t run = 0;
      for (int cc = 0; cc < 48; ++cc) {
        q8pref[49 * e + cc] = run;
        uint64_t rm = 0;
        for (int rr = 0; rr < 48; ++rr)
          if (K[rr + 48 * cc] != 0.0) {
            rm |= 1ull << rr;
            ++run;
            q8pair[64 * e + 8 * (rr / 6) + cc / 6] |= 1ull << ((rr % 6) + 6 * (cc % 6));
          }
        q8col[48 * e + cc] = rm;
      }
      q8pref[49 * e + 48] = run;
    }
    for (int64_t e = 0; e < nq8; ++e) q8off[e + 1] = q8off[e] + q8pref[49 * e + 48];
  }
  // global element order = the reference's triplet order: CQUAD4, CTRIA3,
  // CTETRA10, CQUAD8
  const int64_t g3 = nq4, g10 = nq4 + nt3;
  const int64_t g8 = g10 + nt10;   // first global index of the CQUAD8 elements
  // node -> incident elements (ascending global order)
  std::vector<int64_t> iptr(nn + 1, 0);
  for (int64_t e = 0; e < nq4; ++e)
    for (int k = 0; k < 4; ++k) iptr[m->h_q4n[4 * e + k] + 1]++;
  for (int64_t e = 0; e < nt3; ++e)
    for (int k = 0; k < 3; ++k) iptr[m->h_t3n[3 * e + k] + 1]++;
  for (int64_t e = 0; e < nt10; ++e)
    for (int k = 0; k < 10; ++k) iptr[m->h_t10n[10 * e + k] + 1]++;
  for (int64_t e = 0; e < nq8; ++e)
    for (int k = 0; k < 8; ++k) iptr[m->h_q8n[8 * e + k] + 1]++;
  for (int64_t v = 0; v < nn; ++v) iptr[v + 1] += iptr[v];
  std::vector<ElemRef> inc(iptr[nn]);
  {
    std::vector<int64_t> pos(iptr.begin(), iptr.end() - 1);
    for (int64_t e = 0; e < nq4; ++e)
      for (int k = 0; k < 4; ++k) inc[pos[m->h_q4n[4 * e + k]]++] = {e, (int8_t)k};
    for (int64_t e = 0; e < nt3; ++e)
      for (int k = 0; k < 3; ++k) inc[pos[m->h_t3n[3 * e + k]]++] = {g3 + e, (int8_t)k};
    for (int64_t e = 0; e < nt10; ++e)
      for (int k = 0; k < 10; ++k) inc[pos[m->h_t10n[10 * e + k]]++] = {g10 + e, (int8_t)k};
    for (int64_t e = 0; e < nq8; ++e)
      for (int k = 0; k < 8; ++k) inc[pos[m->h_q8n[8 * e + k]]++] = {g8 + e, (int8_t)k};
  }
  auto enodes = [&](int64_t ge, int& nnd) -> const int32_t* {
    if (ge < nq4) { nnd = 4; return m->h_q4n.data() + 4 * ge; }
    if (ge < g10) { nnd = 3; return m->h_t3n.data() + 3 * (ge - g3); }
    if (ge < g8) { nnd = 10; return m->h_t10n.data() + 10 * (ge - g10); }
    nnd = 8;
    return m->h_q8n.data() + 8 * (ge - g8);
  };
  // 6x6 component mask of the (row node la, column node lb) block of element ge
  auto pmask = [&](int64_t ge, int la, int lb) -> uint64_t {
    if (ge < g10) return MASK_Q4;   // CQUAD4 and CTRIA3: dense 6 x 6 blocks
    if (ge < g8) return mt10;
    return q8pair[64 * (ge - g8) + 8 * la + lb];
  };
  // per column node: sorted (row node, mask)
  struct Blk { int32_t a; uint64_t mask; };
  auto node_blocks = [&](int64_t b, std::vector<Blk>& out) {
    out.clear();
    for (int64_t p = iptr[b]; p < iptr[b + 1]; ++p) {
      int nnd;
      const int32_t* en = enodes(inc[p].e, nnd);
      for (int k = 0; k < nnd; ++k) out.push_back({en[k], pmask(inc[p].e, k, inc[p].local)});
    }
    std::sort(out.begin(), out.end(), [](const Blk& x, const Blk& y) { return x.a < y.a; });
    size_t w = 0;
    for (size_t r = 0; r < out.size(); ++r) {
      if (w > 0 && out[w - 1].a == out[r].a) out[w - 1].mask |= out[r].mask;
      else out[w++] = out[r];
    }
    out.resize(w);
  };
  // pass 1: column counts
  m->pat->colptr.assign(ndof + 1, 0);
#pragma omp parallel
  {
    std::vector<Blk> blk;
#pragma omp for schedule(dynamic, 256)
    for (int64_t b = 0; b < nn; ++b) {
      node_blocks(b, blk);
      for (int j = 0; j < 6; ++j) {
        int64_t cnt = 0;
        for (auto& x : blk)
          for (int i = 0; i < 6; ++i) cnt += (x.mask >> (i + 6 * j)) & 1;
        m->pat->colptr[6 * b + j + 1] = cnt;
      }
    }
  }
  for (int64_t j = 0; j < ndof; ++j) m->pat->colptr[j + 1] += m->pat->colptr[j];
  const int64_t nnz = m->pat->colptr[ndof];
  m->nnz = nnz;
  m->pat->rowval.resize(nnz);
  m->pat->diag_pos.assign(ndof, -1);
  m->n_trip = 576 * nq4 + 324 * nt3 + 900 * nt10 + q8off[nq8];
  if (m->n_trip >= (int64_t)INT32_MAX || m->n_ev >= (int64_t)INT32_MAX) {
    set_error("triplet count exceeds the 32-bit slot-map range");
    return JFG_UNSUPPORTED;
  }
  std::vector<int32_t> cnt(nnz + 1, 0);
  // Passes 2 and 3 walk, per column node b, its incident elements in global
  // element order (the reference's triplet order): every (element node a,
  // component pair) contribution lands in CSC entry q = start[a's block][j]
  // + (rows of that block in column j above i).  Column nodes own disjoint
  // entries, so they run in parallel; pass 2 writes the rows and counts the
  // contributions per entry, pass 3 fills them in order with the slot map.
  struct ColNode {
    std::vector<Blk> blk;
    std::vector<int64_t> start;   // (block, j) -> first CSC position of its rows in column 6b+j
  };
  auto prepare_col = [&](int64_t b, ColNode& cn, std::vector<int32_t>& where) {
    node_blocks(b, cn.blk);
    const size_t nb = cn.blk.size();
    cn.start.resize(6 * nb);
    for (int j = 0; j < 6; ++j) {
      int64_t q = m->pat->colptr[6 * b + j];
      for (size_t k = 0; k < nb; ++k) {
        cn.start[6 * k + j] = q;
        q += __builtin_popcountll((cn.blk[k].mask >> (6 * j)) & 0x3Full);
      }
    }
    for (size_t k = 0; k < nb; ++k) where[cn.blk[k].a] = (int32_t)k;
  };
  // calls f(q, t, src) for every contribution of column node b, in order
  auto for_contribs = [&](int64_t b, const ColNode& cn, const std::vector<int32_t>& where, auto&& f) {
    for (int64_t p = iptr[b]; p < iptr[b + 1]; ++p) {
      const int64_t ge = inc[p].e;
      const int lb = inc[p].local;
      int nnd;
      const int32_t* en = enodes(ge, nnd);
      for (int la = 0; la < nnd; ++la) {
        const int k = where[en[la]];
        const uint64_t em = pmask(ge, la, lb);
        const uint64_t bm = cn.blk[k].mask;
        for (int j = 0; j < 6; ++j) {
          const uint64_t ecol = (em >> (6 * j)) & 0x3Full;
          if (!ecol) continue;
          const uint64_t bcol = (bm >> (6 * j)) & 0x3Full;
          for (int i = 0; i < 6; ++i) {
            if (!((ecol >> i) & 1)) continue;
            const int64_t q = cn.start[6 * k + j] + __builtin_popcountll(bcol & ((1ull << i) - 1));
            // t: the triplet's position in the reference's triplet order;
            // src: the element value it reads
            int64_t t, src;
            if (ge < nq4) {
              const int rr = 6 * la + i, cc = 6 * lb + j;
              t = src = 576 * ge + rr + 24 * cc;
            } else if (ge < g10) {
              const int rr = 6 * la + i, cc = 6 * lb + j;
              t = 576 * nq4 + 324 * (ge - g3) + rr + 18 * cc;
              src = m->ev_t3_off + 324 * (ge - g3) + rr + 18 * cc;
            } else if (ge < g8) {
              const int rr = 3 * la + i, cc = 3 * lb + j;
              t = 576 * nq4 + 324 * nt3 + 900 * (ge - g10) + rr + 30 * cc;
              src = m->ev_t10_off + 900 * (ge - g10) + rr + 30 * cc;
            } else {
              const int64_t e8 = ge - g8;
              const int rr = 6 * la + i, cc = 6 * lb + j;
              const uint64_t below = q8col[48 * e8 + cc] & ((1ull << rr) - 1);
              t = 576 * nq4 + 324 * nt3 + 900 * nt10 + q8off[e8] + q8pref[49 * e8 + cc] +
                  __builtin_popcountll(below);
              src = m->ev_q8_off + 2304 * e8 + rr + 48 * cc;
            }
            f(q, t, src);
          }
        }
      }
    }
  };
  // pass 2: rows, diagonal positions and contribution counts
#pragma omp parallel
  {
    ColNode cn;
    std::vector<int32_t> where(nn, -1);
#pragma omp for schedule(dynamic, 256)
    for (int64_t b = 0; b < nn; ++b) {
      prepare_col(b, cn, where);
      for (size_t k = 0; k < cn.blk.size(); ++k)
        for (int j = 0; j < 6; ++j) {
          int64_t q = cn.start[6 * k + j];
          for (int i = 0; i < 6; ++i) {
            if (!((cn.blk[k].mask >> (i + 6 * j)) & 1)) continue;
            m->pat->rowval[q] = 6 * cn.blk[k].a + i;
            if (cn.blk[k].a == b && i == j) m->pat->diag_pos[6 * b + j] = q;
            ++q;
          }
        }
      for_contribs(b, cn, where, [&](int64_t q, int64_t, int64_t) { cnt[q + 1]++; });
      for (auto& x : cn.blk) where[x.a] = -1;
    }
  }
  for (int64_t q = 0; q < nnz; ++q) cnt[q + 1] += cnt[q];
  if (cnt[nnz] != m->n_trip) {
    set_error("internal: slot-map contribution count mismatch");
    return JFG_BAD_INPUT;
  }
  // both filled completely by pass 3 (the counts above match the triplets)
  std::vector<int32_t, UninitAlloc<int32_t>> trip(m->n_trip);
  m->pat->slot.resize(m->n_trip);
  // pass 3: contributions in triplet (element) order, and the slot map
#pragma omp parallel
  {
    ColNode cn;
    std::vector<int32_t> where(nn, -1);
    std::vector<int32_t> fill;
#pragma omp for schedule(dynamic, 256)
    for (int64_t b = 0; b < nn; ++b) {
      prepare_col(b, cn, where);
      const int64_t q0 = m->pat->colptr[6 * b], q1 = m->pat->colptr[6 * b + 6];
      fill.assign(cnt.begin() + q0, cnt.begin() + q1);   // next free position of each entry
      for_contribs(b, cn, where, [&](int64_t q, int64_t t, int64_t src) {
        trip[fill[q - q0]++] = (int32_t)src;
        m->pat->slot[t] = (int32_t)q;
      });
      for (auto& x : cn.blk) where[x.a] = -1;
    }
  }
  // transpose positions (row i of the symmetric pattern through column i)
  std::vector<int64_t, UninitAlloc<int64_t>> tpos(nnz);
  int asym = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(| : asym)
  for (int64_t j = 0; j < ndof; ++j)
    for (int64_t p = m->pat->colptr[j]; p < m->pat->colptr[j + 1]; ++p) {
      int64_t i = m->pat->rowval[p];
      const int32_t* beg = m->pat->rowval.data() + m->pat->colptr[i];
      const int32_t* end = m->pat->rowval.data() + m->pat->colptr[i + 1];
      const int32_t* f = std::lower_bound(beg, end, (int32_t)j);
      const bool hit = f != end && *f == j;
      tpos[p] = hit ? m->pat->colptr[i] + (f - beg) : -1;
      asym |= hit ? 0 : 1;
    }
  if (asym) {
    set_error("pattern is not structurally symmetric");
    return JFG_BAD_INPUT;
  }
  jfg_ctx* c = m->ctx;
  JFG_TRY(dev_alloc(c, (void**)&m->d_colptr, sizeof(int64_t) * (ndof + 1)));
  JFG_TRY(dev_alloc(c, (void**)&m->d_rowval, sizeof(int32_t) * nnz));
  JFG_TRY(dev_alloc(c, (void**)&m->d_nzptr, sizeof(int32_t) * (nnz + 1)));
  JFG_TRY(dev_alloc(c, (void**)&m->d_trip, sizeof(int32_t) * m->n_trip));
  JFG_TRY(dev_alloc(c, (void**)&m->d_tpos, sizeof(int64_t) * nnz));
  JFG_TRY(dev_alloc(c, (void**)&m->d_nzval, sizeof(double) * nnz));
  JFG_CUDA(cudaMemcpy(m->d_colptr, m->pat->colptr.data(), sizeof(int64_t) * (ndof + 1), cudaMemcpyHostToDevice));
  JFG_CUDA(cudaMemcpy(m->d_rowval, m->pat->rowval.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice));
  JFG_CUDA(cudaMemcpy(m->d_nzptr, cnt.data(), sizeof(int32_t) * (nnz + 1), cudaMemcpyHostToDevice));
  JFG_CUDA(cudaMemcpy(m->d_trip, trip.data(), sizeof(int32_t) * m->n_trip, cudaMemcpyHostToDevice));
  JFG_CUDA(cudaMemcpy(m->d_tpos, tpos.data(), sizeof(int64_t) * nnz, cudaMemcpyHostToDevice));
  m->pattern_built = true;
  return JFG_OK;
}

jfg_status launch_assembly(jfg_model* m, cudaStream_t st) {
  int64_t blocks = (m->nnz + 255) / 256;
  int ps = prof_start(st);
  { k_assemble<<<(unsigned)blocks, 256, 0, st>>>(m->nnz, m->d_nzptr, m->d_trip, m->d_ev, m->d_nzval); count_launch(); }
  // algorithmic bytes: each triplet's index + value read once, each entry's
  // pointer read and value written once
  prof_end(ps, st, KS_ASSEMBLY, (double)m->n_trip * 12 + (double)m->nnz * 12);
  JFG_CUDA(cudaGetLastError());
  return JFG_OK;
}

void spmv_csc_sym(const jfg_model* m, int nrhs, const double* x, int64_t ldx, double* y, int64_t ldy,
                  cudaStream_t st) {
  int64_t threads = m->ndof * 32;
  int64_t blocks = (threads + 255) / 256;
  { k_spmv<<<(unsigned)blocks, 256, 0, st>>>(m->ndof, m->d_colptr, m->d_rowval, m->d_tpos, m->d_nzval, nrhs,
                                           x, ldx, y, ldy); count_launch(); }
}

// The slot-map gather of launch_assembly reading element values from `ev`
// and writing the nnz values to `nzval`; no profiling events.
jfg_status launch_gather_into(const jfg_model* m, cudaStream_t st, const double* ev, double* nzval) {
  int64_t blocks = (m->nnz + 255) / 256;
  { k_assemble<<<(unsigned)blocks, 256, 0, st>>>(m->nnz, m->d_nzptr, m->d_trip, ev, nzval); count_launch(); }
  JFG_CUDA(cudaGetLastError());
  return JFG_OK;
}

}  // namespace jfg
