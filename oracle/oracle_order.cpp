// oracle_order.cpp -- fill-reducing orderings owned by the CPU oracle.
// TEST INFRASTRUCTURE ONLY: the orderings of the CPU checker and of the timed
// CPU baseline, so that neither loads the device library or calls its
// symbolic analysis.
//
// The reference gets its ordering from CHOLMOD (SuiteSparse_jll 7.10.1 via
// cholesky(Symmetric(K_ff)), src/solver/boundary_conditions.jl:1660), whose
// default tries approximate minimum degree and, when that ordering is poor,
// METIS nested dissection, keeping the one with the smaller factor.  Neither
// library is in this image, so both methods are restated here from their
// published descriptions:
//   * or_amd_order: approximate minimum degree on the quotient graph
//     (Amestoy, Davis & Duff, "An approximate minimum degree ordering
//     algorithm", SIAM J. Matrix Anal. Appl. 17(4), 1996): element absorption,
//     the approximate external degree bound, aggressive absorption,
//     indistinguishable-variable detection by hashing, mass elimination;
//   * or_nd_order: nested dissection by recursive coordinate bisection with a
//     vertex separator (George 1973; geometric partitioning), the separator
//     ordered last, small parts ordered by approximate minimum degree.
// Both order the grid-point graph (one vertex per grid with free DOFs,
// weighted by its number of free DOFs); the DOFs of a grid are consecutive.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <vector>

namespace {

struct Graph {
  int n = 0;
  std::vector<int64_t> ptr;
  std::vector<int32_t> adj;
};

// Approximate minimum degree on the subgraph `verts` (local ids 0..m-1 map to
// global vertices verts[k]); appends the elimination order (global ids) to out.
void amd_order(const Graph& G, const std::vector<int32_t>& wt, const std::vector<int32_t>& verts,
               std::vector<int32_t>& out) {
  const int m = (int)verts.size();
  if (m == 0) return;
  std::vector<int32_t> loc(G.n, -1);
  for (int k = 0; k < m; ++k) loc[verts[k]] = k;
  // quotient graph
  std::vector<std::vector<int32_t>> A(m), E(m), L(m);   // variable adjacency / element adjacency / element members
  std::vector<int64_t> nv(m), deg(m, 0);
  std::vector<uint8_t> is_elem(m, 0), dead(m, 0);        // dead: absorbed element or merged variable
  std::vector<std::vector<int32_t>> merged(m);            // variables merged into a principal variable
  int64_t total = 0;
  for (int k = 0; k < m; ++k) {
    nv[k] = wt[verts[k]];
    total += nv[k];
    const int v = verts[k];
    for (int64_t p = G.ptr[v]; p < G.ptr[v + 1]; ++p) {
      const int j = loc[G.adj[p]];
      if (j >= 0 && j != k) A[k].push_back(j);
    }
  }
  for (int k = 0; k < m; ++k)
    for (int j : A[k]) deg[k] += nv[j];
  // degree buckets (doubly linked lists)
  const int64_t maxd = total + 1;
  std::vector<int32_t> head(maxd + 1, -1), nxt(m, -1), prv(m, -1);
  int64_t mind = 0;
  auto bucket_insert = [&](int i) {
    int64_t d = std::min(deg[i], maxd);
    nxt[i] = head[d];
    prv[i] = -1;
    if (head[d] >= 0) prv[head[d]] = i;
    head[d] = i;
    mind = std::min(mind, d);
  };
  auto bucket_remove = [&](int i) {
    int64_t d = std::min(deg[i], maxd);
    if (prv[i] >= 0) nxt[prv[i]] = nxt[i]; else head[d] = nxt[i];
    if (nxt[i] >= 0) prv[nxt[i]] = prv[i];
    nxt[i] = prv[i] = -1;
  };
  for (int k = 0; k < m; ++k) bucket_insert(k);
  std::vector<int64_t> mark(m, -1), wmark(m, -1), w(m, 0);
  int64_t tag = 0;
  int64_t remaining = total;
  std::vector<int32_t> Lp;
  std::vector<std::pair<uint64_t, int32_t>> hashes;
  auto emit = [&](int i) {
    // a principal variable and every variable merged into it, recursively
    std::vector<int32_t> stack{i};
    while (!stack.empty()) {
      int v = stack.back();
      stack.pop_back();
      out.push_back(verts[v]);
      for (int c : merged[v]) stack.push_back(c);
    }
  };
  int eliminated = 0;
  while (eliminated < m) {
    while (mind <= maxd && head[mind] < 0) ++mind;
    if (mind > maxd) break;
    const int p = head[mind];
    bucket_remove(p);
    // ---- the new element p: L_p = (A_p u U_{e in E_p} L_e) \ {p}
    ++tag;
    mark[p] = tag;
    Lp.clear();
    for (int e : E[p]) {
      if (dead[e]) continue;
      for (int i : L[e])
        if (!dead[i] && !is_elem[i] && mark[i] != tag) { mark[i] = tag; Lp.push_back(i); }
      dead[e] = 1;                 // absorbed into p
      std::vector<int32_t>().swap(L[e]);
    }
    for (int i : A[p])
      if (!dead[i] && !is_elem[i] && mark[i] != tag) { mark[i] = tag; Lp.push_back(i); }
    std::vector<int32_t>().swap(A[p]);
    std::vector<int32_t>().swap(E[p]);
    is_elem[p] = 1;
    remaining -= nv[p];
    emit(p);
    eliminated += 1 + (int)merged[p].size();
    int64_t degp = 0;
    for (int i : Lp) { degp += nv[i]; bucket_remove(i); }
    // ---- prune the adjacency of every i in L_p
    for (int i : Lp) {
      auto& Ei = E[i];
      size_t q = 0;
      for (int e : Ei) if (!dead[e] && e != p) Ei[q++] = e;
      Ei.resize(q);
      Ei.push_back(p);
      auto& Ai = A[i];
      q = 0;
      for (int j : Ai) if (!dead[j] && !is_elem[j] && mark[j] != tag) Ai[q++] = j;
      Ai.resize(q);
    }
    // ---- |L_e \ L_p| (weighted) for every element adjacent to L_p
    for (int i : Lp)
      for (int e : E[i]) {
        if (e == p) continue;
        if (wmark[e] != tag) {
          wmark[e] = tag;
          auto& Le = L[e];
          size_t q = 0;
          int64_t s = 0;
          for (int j : Le) if (!dead[j] && !is_elem[j]) { Le[q++] = j; s += nv[j]; }
          Le.resize(q);
          w[e] = s;
        }
        w[e] -= nv[i];
      }
    // ---- approximate external degrees, aggressive absorption
    for (int i : Lp) {
      auto& Ei = E[i];
      int64_t de = 0;
      size_t q = 0;
      for (int e : Ei) {
        if (e == p) { Ei[q++] = e; continue; }
        if (w[e] <= 0) { dead[e] = 1; std::vector<int32_t>().swap(L[e]); continue; }   // L_e inside L_p
        de += w[e];
        Ei[q++] = e;
      }
      Ei.resize(q);
      for (int j : A[i]) de += nv[j];
      const int64_t lp_ext = degp - nv[i];
      int64_t d = std::min(deg[i] + lp_ext, de + lp_ext);
      d = std::min(d, remaining - nv[i]);
      deg[i] = std::max<int64_t>(d, 0);
    }
    // ---- indistinguishable variables (same A and E): merge into one
    hashes.clear();
    for (int i : Lp) {
      std::sort(A[i].begin(), A[i].end());
      std::sort(E[i].begin(), E[i].end());
      uint64_t h = 1469598103934665603ull;
      for (int j : A[i]) h = (h ^ (uint64_t)(j + 1)) * 1099511628211ull;
      h = (h ^ 0x9e3779b97f4a7c15ull) * 1099511628211ull;
      for (int e : E[i]) h = (h ^ (uint64_t)(e + 1)) * 1099511628211ull;
      hashes.push_back({h, i});
    }
    std::sort(hashes.begin(), hashes.end());
    for (size_t a = 0; a < hashes.size();) {
      size_t b = a;
      while (b < hashes.size() && hashes[b].first == hashes[a].first) ++b;
      for (size_t x = a; x < b; ++x) {
        const int i = hashes[x].second;
        if (dead[i]) continue;
        for (size_t y = x + 1; y < b; ++y) {
          const int j = hashes[y].second;
          if (dead[j] || A[i] != A[j] || E[i] != E[j]) continue;
          nv[i] += nv[j];
          deg[i] = std::max<int64_t>(deg[i] - nv[j], 0);
          dead[j] = 1;
          merged[i].push_back(j);
          std::vector<int32_t>().swap(A[j]);
          std::vector<int32_t>().swap(E[j]);
        }
      }
      a = b;
    }
    // ---- mass elimination and reinsertion; the element keeps its live members
    std::vector<int32_t> keep;
    keep.reserve(Lp.size());
    for (int i : Lp) {
      if (dead[i]) continue;
      if (A[i].empty() && E[i].size() == 1 && E[i][0] == p) {
        is_elem[i] = 1;
        dead[i] = 1;
        remaining -= nv[i];
        emit(i);
        eliminated += 1 + (int)merged[i].size();
        std::vector<int32_t>().swap(E[i]);
        continue;
      }
      keep.push_back(i);
    }
    for (int i : keep) bucket_insert(i);
    L[p] = keep;
  }
}

// Nested dissection by recursive coordinate bisection.  A part is split at
// the median of its widest coordinate; the vertices of the lower half with a
// neighbour in the upper half form the separator, ordered after both halves.
void nd_recurse(const Graph& G, const std::vector<int32_t>& wt, const double* xyz, std::vector<int32_t> verts,
                int leaf, std::vector<int32_t>& out, std::vector<int32_t>& side) {
  if ((int)verts.size() <= leaf) {
    amd_order(G, wt, verts, out);
    return;
  }
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int v : verts)
    for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], xyz[3 * v + a]); hi[a] = std::max(hi[a], xyz[3 * v + a]); }
  int ax = 0;
  for (int a = 1; a < 3; ++a) if (hi[a] - lo[a] > hi[ax] - lo[ax]) ax = a;
  std::vector<int32_t> sorted = verts;
  const size_t mid = sorted.size() / 2;
  std::nth_element(sorted.begin(), sorted.begin() + mid, sorted.end(),
                   [&](int a, int b) { return xyz[3 * a + ax] < xyz[3 * b + ax] ||
                                              (xyz[3 * a + ax] == xyz[3 * b + ax] && a < b); });
  const double cut = xyz[3 * sorted[mid] + ax];
  // side: 1 lower, 2 upper (vertices at the cut coordinate go to the lower side)
  for (int v : verts) side[v] = xyz[3 * v + ax] <= cut ? 1 : 2;
  std::vector<int32_t> a, b, sep;
  for (int v : verts) {
    if (side[v] == 2) { b.push_back(v); continue; }
    bool touches = false;
    for (int64_t p = G.ptr[v]; p < G.ptr[v + 1] && !touches; ++p) touches = side[G.adj[p]] == 2;
    (touches ? sep : a).push_back(v);
  }
  for (int v : verts) side[v] = 0;
  if (a.empty() || b.empty()) {   // no useful split (degenerate geometry)
    amd_order(G, wt, verts, out);
    return;
  }
  nd_recurse(G, wt, xyz, std::move(a), leaf, out, side);
  nd_recurse(G, wt, xyz, std::move(b), leaf, out, side);
  amd_order(G, wt, sep, out);
}

Graph make_graph(int32_t n, const int64_t* ptr, const int32_t* adj) {
  Graph G;
  G.n = n;
  G.ptr.assign(ptr, ptr + n + 1);
  G.adj.assign(adj, adj + ptr[n]);
  return G;
}

}  // namespace

extern "C" {

// Grid-point graph (CSR ptr/adj over n vertices, symmetric, no self loops),
// vertex weights wt (free DOFs per grid).  order[k] = k-th eliminated vertex.
int or_amd_order(int32_t n, const int64_t* ptr, const int32_t* adj, const int32_t* wt, int32_t* order) {
  Graph G = make_graph(n, ptr, adj);
  std::vector<int32_t> w(wt, wt + n), verts(n), out;
  std::iota(verts.begin(), verts.end(), 0);
  out.reserve(n);
  amd_order(G, w, verts, out);
  if ((int)out.size() != n) return 1;
  std::copy(out.begin(), out.end(), order);
  return 0;
}

// Same graph plus grid coordinates xyz (n x 3, row per vertex); parts of at
// most `leaf` vertices are ordered by approximate minimum degree.
int or_nd_order(int32_t n, const int64_t* ptr, const int32_t* adj, const int32_t* wt, const double* xyz,
                int32_t leaf, int32_t* order) {
  Graph G = make_graph(n, ptr, adj);
  std::vector<int32_t> w(wt, wt + n), verts(n), out, side(n, 0);
  std::iota(verts.begin(), verts.end(), 0);
  out.reserve(n);
  nd_recurse(G, w, xyz, verts, std::max(leaf, 8), out, side);
  if ((int)out.size() != n) return 1;
  std::copy(out.begin(), out.end(), order);
  return 0;
}

}  // extern "C"
