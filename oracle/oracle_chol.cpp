// oracle_chol.cpp -- CPU FP64 supernodal multifrontal Cholesky of K_ff.
// TEST INFRASTRUCTURE ONLY (the FP64 checker and the timed CPU baseline).
//
// Restates what the reference obtains from cholesky(Symmetric(K_ff)) and
// F \ f (src/solver/boundary_conditions.jl:1656-1714): an LL^T factor of the
// upper triangle of K_ff, then forward/back substitution one right-hand side
// at a time.  The dense kernels are OpenBLAS (dpotrf/dtrsm/dsyrk/dgemm), the
// same library version as the reference's OpenBLAS_jll 0.3.30, loaded at run
// time from SciPy's wheel.  The elimination order is an input.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>
#include <algorithm>
#include <chrono>
#include <dlfcn.h>

namespace {

using dgemm_t = void (*)(const char*, const char*, const int*, const int*, const int*, const double*,
                         const double*, const int*, const double*, const int*, const double*, double*,
                         const int*);
using dsyrk_t = void (*)(const char*, const char*, const int*, const int*, const double*, const double*,
                         const int*, const double*, double*, const int*);
using dtrsm_t = void (*)(const char*, const char*, const char*, const char*, const int*, const int*,
                         const double*, const double*, const int*, double*, const int*);
using dpotrf_t = void (*)(const char*, const int*, double*, const int*, int*);
using setthreads_t = void (*)(int);

struct Blas {
  dgemm_t gemm = nullptr;
  dsyrk_t syrk = nullptr;
  dtrsm_t trsm = nullptr;
  dpotrf_t potrf = nullptr;
  setthreads_t set_threads = nullptr;
  bool ok = false;
};

Blas& blas() {
  static Blas b;
  static bool tried = false;
  if (tried) return b;
  tried = true;
  const char* path = std::getenv("JFEM_ORACLE_OPENBLAS");
  std::vector<std::string> cands;
  if (path) cands.push_back(path);
  void* h = nullptr;
  for (auto& c : cands) {
    h = dlopen(c.c_str(), RTLD_NOW | RTLD_LOCAL);
    if (h) break;
  }
  if (!h) return b;
  b.gemm = (dgemm_t)dlsym(h, "scipy_dgemm_");
  b.syrk = (dsyrk_t)dlsym(h, "scipy_dsyrk_");
  b.trsm = (dtrsm_t)dlsym(h, "scipy_dtrsm_");
  b.potrf = (dpotrf_t)dlsym(h, "scipy_dpotrf_");
  b.set_threads = (setthreads_t)dlsym(h, "scipy_openblas_set_num_threads");
  b.ok = b.gemm && b.syrk && b.trsm && b.potrf;
  return b;
}

// Fallback dense kernels (used when OpenBLAS is not found): plain loops.
void potrf_lower(int n, double* A, int lda, int* info) {
  Blas& b = blas();
  if (b.ok) { char L = 'L'; b.potrf(&L, &n, A, &lda, info); return; }
  *info = 0;
  for (int j = 0; j < n; ++j) {
    double d = A[j + (int64_t)lda * j];
    for (int k = 0; k < j; ++k) d -= A[j + (int64_t)lda * k] * A[j + (int64_t)lda * k];
    if (!(d > 0)) { *info = j + 1; return; }
    d = std::sqrt(d);
    A[j + (int64_t)lda * j] = d;
    for (int i = j + 1; i < n; ++i) {
      double s = A[i + (int64_t)lda * j];
      for (int k = 0; k < j; ++k) s -= A[i + (int64_t)lda * k] * A[j + (int64_t)lda * k];
      A[i + (int64_t)lda * j] = s / d;
    }
  }
}
// B (m x n) := B * L^{-T}, L n x n lower
void trsm_rlt(int m, int n, const double* L, int ldl, double* B, int ldb) {
  Blas& b = blas();
  if (b.ok) {
    char R = 'R', Lo = 'L', T = 'T', N = 'N';
    double one = 1.0;
    b.trsm(&R, &Lo, &T, &N, &m, &n, &one, L, &ldl, B, &ldb);
    return;
  }
  for (int j = 0; j < n; ++j) {
    for (int k = 0; k < j; ++k) {
      double l = L[j + (int64_t)ldl * k];
      for (int i = 0; i < m; ++i) B[i + (int64_t)ldb * j] -= B[i + (int64_t)ldb * k] * l;
    }
    double d = L[j + (int64_t)ldl * j];
    for (int i = 0; i < m; ++i) B[i + (int64_t)ldb * j] /= d;
  }
}
// C (n x n lower) -= A A^T, A n x k
void syrk_ln(int n, int k, const double* A, int lda, double* C, int ldc) {
  Blas& b = blas();
  if (b.ok) {
    char L = 'L', N = 'N';
    double m1 = -1.0, one = 1.0;
    b.syrk(&L, &N, &n, &k, &m1, A, &lda, &one, C, &ldc);
    return;
  }
  for (int j = 0; j < n; ++j)
    for (int l = 0; l < k; ++l) {
      double a = A[j + (int64_t)lda * l];
      for (int i = j; i < n; ++i) C[i + (int64_t)ldc * j] -= A[i + (int64_t)lda * l] * a;
    }
}

// Permuted lower triangle of Symmetric(K_ff, :U) (lp/li/lv, CSC by column),
// Liu's elimination tree and the column counts of L by row subtrees.
// Returns 0, or -1 for a bad permutation.
int symbolic_counts(int64_t n, const int64_t* colptr, const int32_t* rowval, const double* nzval,
                    const int32_t* perm, std::vector<int64_t>& lp, std::vector<int32_t>& li,
                    std::vector<double>& lv, std::vector<int32_t>& parent, std::vector<int64_t>& cc) {
  std::vector<int32_t> iperm(n);
  for (int64_t k = 0; k < n; ++k) {
    if (perm[k] < 0 || perm[k] >= n) return -1;
    iperm[perm[k]] = (int32_t)k;
  }
  // permuted lower triangle, CSC by column
  lp.assign(n + 1, 0);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) {
      int64_t i = rowval[p];
      if (i > j) continue;
      int64_t a = iperm[i], b = iperm[j];
      lp[std::min(a, b) + 1]++;
    }
  for (int64_t j = 0; j < n; ++j) lp[j + 1] += lp[j];
  li.assign(lp[n], 0);
  lv.assign(nzval ? lp[n] : 0, 0.0);
  {
    std::vector<int64_t> pos(lp.begin(), lp.end() - 1);
    for (int64_t j = 0; j < n; ++j)
      for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) {
        int64_t i = rowval[p];
        if (i > j) continue;
        int64_t a = iperm[i], b = iperm[j];
        int64_t c = std::min(a, b), r = std::max(a, b);
        li[pos[c]] = (int32_t)r;
        if (nzval) lv[pos[c]] = nzval[p];
        pos[c]++;
      }
  }
  // elimination tree (Liu) from the row structure: for column j, the rows
  // i > j with A(i,j) != 0 give, for each i, an edge j -> (subtree of i).
  // Build row lists of the lower triangle (i.e. for each row i, columns j < i).
  std::vector<int64_t> rp(n + 1, 0);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t p = lp[j]; p < lp[j + 1]; ++p) rp[li[p] + 1]++;
  for (int64_t i = 0; i < n; ++i) rp[i + 1] += rp[i];
  std::vector<int32_t> rj(rp[n]);
  {
    std::vector<int64_t> pos(rp.begin(), rp.end() - 1);
    for (int64_t j = 0; j < n; ++j)
      for (int64_t p = lp[j]; p < lp[j + 1]; ++p) rj[pos[li[p]]++] = (int32_t)j;
  }
  parent.assign(n, -1);
  std::vector<int32_t> anc(n, -1);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t p = rp[i]; p < rp[i + 1]; ++p) {
      int64_t j = rj[p];
      if (j >= i) continue;
      while (j != -1 && j < i) {
        int64_t next = anc[j];
        anc[j] = (int32_t)i;
        if (next == -1) { parent[j] = (int32_t)i; break; }
        j = next;
      }
    }
  // column counts via row subtrees
  cc.assign(n, 1);
  std::vector<int64_t> mark(n, -1);
  for (int64_t i = 0; i < n; ++i) {
    mark[i] = i;
    for (int64_t p = rp[i]; p < rp[i + 1]; ++p) {
      int64_t j = rj[p];
      if (j >= i) continue;
      while (j != -1 && mark[j] != i) {
        cc[j]++;
        mark[j] = i;
        j = parent[j];
      }
    }
  }
  return 0;
}

struct CholFactor {
  int64_t n = 0, ns = 0;
  std::vector<int32_t> perm;
  std::vector<int64_t> sfirst;
  std::vector<std::vector<int32_t>> srows;
  std::vector<std::vector<double>> panel;
  double nnzL = 0, flops = 0;
};

// Symbolic analysis and numeric multifrontal factorisation into C.
// Returns 0, -1 (bad input) or k+1 (first non-positive pivot in column k).
int factor_into(CholFactor& C, int64_t n, const int64_t* colptr, const int32_t* rowval, const double* nzval,
                const int32_t* perm, int32_t nthreads) {
  Blas& bl = blas();
  if (bl.ok && bl.set_threads) bl.set_threads(nthreads > 0 ? nthreads : 1);
  std::vector<int64_t> lp, cc;
  std::vector<int32_t> li, parent;
  std::vector<double> lv;
  if (symbolic_counts(n, colptr, rowval, nzval, perm, lp, li, lv, parent, cc) != 0) return -1;
  std::vector<int32_t> nchild(n, 0);
  for (int64_t j = 0; j < n; ++j)
    if (parent[j] >= 0) nchild[parent[j]]++;
  // fundamental supernodes
  std::vector<int64_t>& sfirst = C.sfirst;
  sfirst.clear();
  for (int64_t j = 0; j < n; ++j) {
    bool merge = j > 0 && parent[j - 1] == j && cc[j - 1] == cc[j] + 1 && nchild[j] == 1;
    if (!merge) sfirst.push_back(j);
  }
  int64_t ns = (int64_t)sfirst.size();
  sfirst.push_back(n);
  std::vector<int32_t> col2sn(n);
  for (int64_t s = 0; s < ns; ++s)
    for (int64_t j = sfirst[s]; j < sfirst[s + 1]; ++j) col2sn[j] = (int32_t)s;
  std::vector<int32_t> sparent(ns, -1);
  for (int64_t s = 0; s < ns; ++s) {
    int64_t l = sfirst[s + 1] - 1;
    if (parent[l] >= 0) sparent[s] = col2sn[parent[l]];
  }
  std::vector<std::vector<int32_t>> schildren(ns);
  for (int64_t s = 0; s < ns; ++s)
    if (sparent[s] >= 0) schildren[sparent[s]].push_back((int32_t)s);
  // supernode row structures (rows below the supernode), bottom-up
  std::vector<std::vector<int32_t>>& srows = C.srows;
  srows.assign(ns, {});
  std::vector<int64_t> fmark(n, -1);
  double flops = 0;
  int64_t nnzL = 0;
  for (int64_t s = 0; s < ns; ++s) {
    int64_t f = sfirst[s], l = sfirst[s + 1] - 1;
    std::vector<int32_t>& R = srows[s];
    for (int64_t j = f; j <= l; ++j)
      for (int64_t p = lp[j]; p < lp[j + 1]; ++p) {
        int64_t i = li[p];
        if (i > l && fmark[i] != s) { fmark[i] = s; R.push_back((int32_t)i); }
      }
    for (int32_t c : schildren[s])
      for (int32_t i : srows[c])
        if (i > l && fmark[i] != s) { fmark[i] = s; R.push_back(i); }
    std::sort(R.begin(), R.end());
    int64_t c = l - f + 1, r = (int64_t)R.size();
    for (int64_t k = 0; k < c; ++k) {
      double cj = (double)(c - k + r);
      flops += cj * cj;
    }
    nnzL += c * (c + 1) / 2 + c * r;
  }
  // numeric multifrontal
  std::vector<std::vector<double>>& panel = C.panel;   // m x c, ld = m
  panel.assign(ns, {});
  std::vector<std::vector<double>> upd(ns);     // r x r
  std::vector<int64_t> rowpos(n, -1);
  for (int64_t s = 0; s < ns; ++s) {
    int64_t f = sfirst[s], l = sfirst[s + 1] - 1;
    int64_t c = l - f + 1;
    const std::vector<int32_t>& R = srows[s];
    int64_t r = (int64_t)R.size(), m = c + r;
    for (int64_t k = 0; k < c; ++k) rowpos[f + k] = k;
    for (int64_t k = 0; k < r; ++k) rowpos[R[k]] = c + k;
    std::vector<double> front((size_t)(m * m), 0.0);
    for (int64_t j = f; j <= l; ++j)
      for (int64_t p = lp[j]; p < lp[j + 1]; ++p)
        front[rowpos[li[p]] + m * (j - f)] += lv[p];
    for (int32_t ch : schildren[s]) {
      const std::vector<int32_t>& Rc = srows[ch];
      int64_t rc = (int64_t)Rc.size();
      std::vector<double>& Uc = upd[ch];
      for (int64_t b = 0; b < rc; ++b) {
        int64_t cb = rowpos[Rc[b]];
        for (int64_t a = b; a < rc; ++a) {
          int64_t ra = rowpos[Rc[a]];
          front[ra + m * cb] += Uc[a + rc * b];
        }
      }
      std::vector<double>().swap(Uc);
    }
    int info_p = 0;
    int ci = (int)c, mi = (int)m, ri = (int)r;
    potrf_lower(ci, front.data(), mi, &info_p);
    if (info_p != 0) {
      return (int)(f + info_p);
    }
    if (r > 0) {
      trsm_rlt(ri, ci, front.data(), mi, front.data() + c, mi);
      syrk_ln(ri, ci, front.data() + c, mi, front.data() + c + m * c, mi);
      std::vector<double>& Us = upd[s];
      Us.resize((size_t)(r * r));
      for (int64_t b = 0; b < r; ++b)
        for (int64_t a = b; a < r; ++a) Us[a + r * b] = front[(c + a) + m * (c + b)];
    }
    panel[s].assign(front.begin(), front.begin() + m * c);
  }
  C.n = n;
  C.ns = ns;
  C.perm.assign(perm, perm + n);
  C.nnzL = (double)nnzL;
  C.flops = flops;
  return 0;
}

// Forward and backward substitution with C, one right-hand side at a time
// (boundary_conditions.jl:1714).
void solve_with(const CholFactor& C, int32_t nrhs, const double* F, double* U) {
  const int64_t n = C.n, ns = C.ns;
  const int32_t* perm = C.perm.data();
  const std::vector<int64_t>& sfirst = C.sfirst;
  const std::vector<std::vector<int32_t>>& srows = C.srows;
  const std::vector<std::vector<double>>& panel = C.panel;
  std::vector<double> x(n);
  for (int32_t q = 0; q < nrhs; ++q) {
    for (int64_t k = 0; k < n; ++k) x[k] = F[(int64_t)q * n + perm[k]];
    for (int64_t s = 0; s < ns; ++s) {
      int64_t f = sfirst[s], c = sfirst[s + 1] - f;
      const std::vector<int32_t>& R = srows[s];
      int64_t r = (int64_t)R.size(), m = c + r;
      const double* P = panel[s].data();
      for (int64_t j = 0; j < c; ++j) {
        double v = x[f + j] / P[j + m * j];
        x[f + j] = v;
        for (int64_t i = j + 1; i < c; ++i) x[f + i] -= P[i + m * j] * v;
        for (int64_t k = 0; k < r; ++k) x[R[k]] -= P[(c + k) + m * j] * v;
      }
    }
    for (int64_t s = ns - 1; s >= 0; --s) {
      int64_t f = sfirst[s], c = sfirst[s + 1] - f;
      const std::vector<int32_t>& R = srows[s];
      int64_t r = (int64_t)R.size(), m = c + r;
      const double* P = panel[s].data();
      for (int64_t j = c - 1; j >= 0; --j) {
        double v = x[f + j];
        for (int64_t k = 0; k < r; ++k) v -= P[(c + k) + m * j] * x[R[k]];
        for (int64_t i = j + 1; i < c; ++i) v -= P[i + m * j] * x[f + i];
        x[f + j] = v / P[j + m * j];
      }
    }
    for (int64_t k = 0; k < n; ++k) U[(int64_t)q * n + perm[k]] = x[k];
  }
}

}  // namespace

extern "C" {

// n: order of K_ff.  CSC (colptr, rowval, nzval) of K_ff; only entries with
// row <= col are read (Symmetric(K_ff, :U)).  perm[k] = unknown eliminated
// k-th.  F, U: n x nrhs column-major.  info[0..3] = factor seconds, solve
// seconds, nnz(L), flops (sum c_j^2).  Returns 0, or -1 (bad input), or
// k+1 (first non-positive pivot in permuted column k).
// Symbolic counts of the factor of Symmetric(K_ff) in the elimination order
// perm: info[0] = nnz(L) (incl. diagonal), info[1] = flops (sum_j c_j^2),
// info[2] = nnz of the lower triangle of K_ff.  Returns 0 or -1.
int or_chol_counts(int64_t n, const int64_t* colptr, const int32_t* rowval, const int32_t* perm, double* info) {
  std::vector<int64_t> lp, cc;
  std::vector<int32_t> li, parent;
  std::vector<double> lv;
  if (symbolic_counts(n, colptr, rowval, nullptr, perm, lp, li, lv, parent, cc) != 0) return -1;
  double nnzL = 0, flops = 0;
  for (int64_t j = 0; j < n; ++j) { nnzL += (double)cc[j]; flops += (double)cc[j] * (double)cc[j]; }
  info[0] = nnzL;
  info[1] = flops;
  info[2] = (double)lp[n];
  return 0;
}

int or_chol_factor_solve(int64_t n, const int64_t* colptr, const int32_t* rowval,
                         const double* nzval, const int32_t* perm, int32_t nrhs,
                         const double* F, double* U, int32_t nthreads, double* info) {
  using clk = std::chrono::steady_clock;
  auto t0 = clk::now();
  CholFactor C;
  int st = factor_into(C, n, colptr, rowval, nzval, perm, nthreads);
  auto t1 = clk::now();
  info[0] = std::chrono::duration<double>(t1 - t0).count();
  if (st != 0) return st;
  solve_with(C, nrhs, F, U);
  auto t2 = clk::now();
  info[1] = std::chrono::duration<double>(t2 - t1).count();
  info[2] = C.nnzL;
  info[3] = C.flops;
  return 0;
}

// Factor once, solve many times (the checker's iterative refinement).
int or_chol_factor(int64_t n, const int64_t* colptr, const int32_t* rowval, const double* nzval,
                   const int32_t* perm, int32_t nthreads, void** handle) {
  CholFactor* C = new CholFactor();
  int st = factor_into(*C, n, colptr, rowval, nzval, perm, nthreads);
  if (st != 0) { delete C; *handle = nullptr; return st; }
  *handle = C;
  return 0;
}
int or_chol_solve(void* handle, int32_t nrhs, const double* F, double* U) {
  if (!handle) return -1;
  solve_with(*static_cast<CholFactor*>(handle), nrhs, F, U);
  return 0;
}
void or_chol_free(void* handle) { delete static_cast<CholFactor*>(handle); }

}  // extern "C"
