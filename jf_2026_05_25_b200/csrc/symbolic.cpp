// symbolic.cpp -- host symbolic analysis for the device multifrontal Cholesky.
//
// The reference obtains ordering, elimination tree and supernodes from
// CHOLMOD inside cholesky(Symmetric(K_ff)) (src/solver/boundary_conditions.jl:1660).
// Here the analysis runs once per mesh on the host, on the NODE graph (the
// free DOFs of one GRID always share a sparsity pattern), and produces the
// flat arrays the device kernels consume.
#include "symbolic.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <functional>
#include <stack>

namespace jfg {

namespace {

struct NodeGraph {
  std::vector<int64_t> ptr;
  std::vector<int32_t> adj;
};

// Minimum-degree order of one nested-dissection leaf.  The leaf's nodes
// are eliminated before every node outside it, so the elimination graph is
// built over the leaf plus its halo (outside neighbours, never eliminated
// here) and a node's degree counts both: the exact external degree of the
// elimination graph, kept as bitsets (at most 512 vertices; larger leaves
// keep their given order).  Ties go to the earlier node.
void order_leaf(const NodeGraph& g, const std::vector<int32_t>& nodes, std::vector<int32_t>& mark,
                std::vector<int32_t>& pos, int32_t* out) {
  const int nl = (int)nodes.size();
  constexpr int MAXV = 512, W = MAXV / 64;
  std::vector<int32_t> verts(nodes.begin(), nodes.end());
  for (int k = 0; k < nl; ++k) { mark[verts[k]] = 1; pos[verts[k]] = k; }
  for (int k = 0; k < nl && (int)verts.size() <= MAXV; ++k) {
    const int32_t v = verts[k];
    for (int64_t p = g.ptr[v]; p < g.ptr[v + 1]; ++p) {
      const int32_t w = g.adj[p];
      if (mark[w] < 0) { mark[w] = 2; pos[w] = (int32_t)verts.size(); verts.push_back(w); }
    }
  }
  const int nv = (int)verts.size();
  if (nv > MAXV) {
    for (int k = 0; k < nl; ++k) out[k] = nodes[k];
  } else {
    std::vector<uint64_t> adj((size_t)nv * W, 0);
    for (int k = 0; k < nl; ++k) {
      const int32_t v = verts[k];
      for (int64_t p = g.ptr[v]; p < g.ptr[v + 1]; ++p) {
        const int j = pos[g.adj[p]];
        if (j == k) continue;
        adj[(size_t)k * W + j / 64] |= 1ull << (j % 64);
        adj[(size_t)j * W + k / 64] |= 1ull << (k % 64);
      }
    }
    std::vector<uint8_t> done(nl, 0);
    for (int step = 0; step < nl; ++step) {
      int best = -1, bd = 1 << 30;
      for (int k = 0; k < nl; ++k) {
        if (done[k]) continue;
        int d = 0;
        for (int w = 0; w < W; ++w) d += __builtin_popcountll(adj[(size_t)k * W + w]);
        if (d < bd) { bd = d; best = k; }
      }
      out[step] = verts[best];
      done[best] = 1;
      // eliminate best: its neighbours become a clique
      const uint64_t* nb = &adj[(size_t)best * W];
      for (int w = 0; w < W; ++w) {
        uint64_t bits = nb[w];
        while (bits) {
          const int j = w * 64 + __builtin_ctzll(bits);
          bits &= bits - 1;
          uint64_t* aj = &adj[(size_t)j * W];
          for (int x = 0; x < W; ++x) aj[x] |= nb[x];
          aj[j / 64] &= ~(1ull << (j % 64));
          aj[best / 64] &= ~(1ull << (best % 64));
        }
      }
      for (int x = 0; x < W; ++x) adj[(size_t)best * W + x] = 0;
    }
  }
  for (int32_t v : verts) { mark[v] = -1; pos[v] = -1; }
}

// Nested dissection by recursive coordinate bisection with a one-sided vertex
// separator: split the node set at the median of its longest bounding-box
// axis, take as separator the nodes of one half that touch the other half
// (the smaller of the two candidates), order [left, right, separator].
void nested_dissection(const NodeGraph& g, const double* xyz, const std::vector<int32_t>& active,
                       int leaf, std::vector<int32_t>& order) {
  int64_t n_nodes = (int64_t)g.ptr.size() - 1;
  order.assign(active.size(), -1);
  std::vector<int64_t> tag(n_nodes, -1);
  std::vector<int32_t> mark(n_nodes, -1), halo_pos(n_nodes, -1);
  struct Task { int64_t lo, hi; std::vector<int32_t> nodes; };
  std::vector<Task> st;
  st.push_back({0, (int64_t)active.size(), active});
  int64_t next_tag = 0;
  std::vector<std::pair<double, int32_t>> key;
  while (!st.empty()) {
    Task t = std::move(st.back());
    st.pop_back();
    int64_t sz = (int64_t)t.nodes.size();
    if (sz <= leaf) {
      order_leaf(g, t.nodes, mark, halo_pos, order.data() + t.lo);
      continue;
    }
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int32_t v : t.nodes)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], xyz[3 * (int64_t)v + a]);
        hi[a] = std::max(hi[a], xyz[3 * (int64_t)v + a]);
      }
    int ax = 0;
    for (int a = 1; a < 3; ++a)
      if (hi[a] - lo[a] > hi[ax] - lo[ax]) ax = a;
    key.resize(sz);
    for (int64_t k = 0; k < sz; ++k) key[k] = {xyz[3 * (int64_t)t.nodes[k] + ax], t.nodes[k]};
    int64_t mid = sz / 2;
    std::nth_element(key.begin(), key.begin() + mid, key.end());
    // the cut keeps every node at the median coordinate on one side, so a
    // grid line of a structured mesh is never split between the halves (a
    // split line would make a jagged, larger separator)
    // (ties at the median go to the lower half, or to the upper half when
    // the median is the largest coordinate; a split that leaves a half empty
    // falls back to splitting by rank)
    const double cut = key[mid].first;
    int64_t n_le = 0, n_lt = 0;
    for (int64_t k = 0; k < sz; ++k) { n_le += key[k].first <= cut; n_lt += key[k].first < cut; }
    const int split_mode = (n_le < sz) ? 0 : (n_lt > 0 ? 1 : 2);
    auto in_a = [&](int64_t k) {
      return split_mode == 0 ? key[k].first <= cut : split_mode == 1 ? key[k].first < cut : k < mid;
    };
    int64_t tA = next_tag++, tB = next_tag++;
    for (int64_t k = 0; k < sz; ++k) tag[key[k].second] = in_a(k) ? tA : tB;
    std::vector<int32_t> sepA, sepB, A, B;
    for (int64_t k = 0; k < sz; ++k) {
      int32_t v = key[k].second;
      bool isA = in_a(k);
      int64_t other = isA ? tB : tA;
      bool touch = false;
      for (int64_t p = g.ptr[v]; p < g.ptr[v + 1]; ++p)
        if (tag[g.adj[p]] == other) { touch = true; break; }
      if (isA) { A.push_back(v); if (touch) sepA.push_back(v); }
      else { B.push_back(v); if (touch) sepB.push_back(v); }
    }
    bool useA = sepA.size() <= sepB.size();
    std::vector<int32_t>& sep = useA ? sepA : sepB;
    if ((int64_t)sep.size() >= sz) {  // degenerate split: treat as a leaf
      for (int64_t k = 0; k < sz; ++k) order[t.lo + k] = t.nodes[k];
      continue;
    }
    // mark separator nodes to remove them from their half
    int64_t tS = next_tag++;
    for (int32_t v : sep) tag[v] = tS;
    std::vector<int32_t> A2, B2;
    for (int32_t v : A) if (tag[v] != tS) A2.push_back(v);
    for (int32_t v : B) if (tag[v] != tS) B2.push_back(v);
    // order the separator along its own longest axis (locality only)
    int64_t pos = t.hi - (int64_t)sep.size();
    for (size_t k = 0; k < sep.size(); ++k) order[pos + k] = sep[k];
    int64_t la = (int64_t)A2.size();
    Task ta{t.lo, t.lo + la, std::move(A2)};
    Task tb{t.lo + la, pos, std::move(B2)};
    st.push_back(std::move(tb));
    st.push_back(std::move(ta));
  }
}

}  // namespace

SymbolicOptions SymbolicOptions::from_env() {
  SymbolicOptions o;
  if (const char* v = std::getenv("JFG_ND_LEAF")) o.leaf_nodes = std::max(2, std::atoi(v));
  if (const char* v = std::getenv("JFG_RELAX_COLS"))
    std::sscanf(v, "%d,%d,%d", &o.relax_cols[0], &o.relax_cols[1], &o.relax_cols[2]);
  if (const char* v = std::getenv("JFG_RELAX_ZEROS"))
    std::sscanf(v, "%lf,%lf,%lf", &o.relax_zeros[0], &o.relax_zeros[1], &o.relax_zeros[2]);
  return o;
}

std::string analyze(int64_t ndof, const int64_t* colptr, const int32_t* rowval, int64_t n_free,
                    const int32_t* free_dofs, const double* xyz, const SymbolicOptions& opt,
                    Symbolic& S) {
  auto t0 = std::chrono::steady_clock::now();
  if (ndof % 6 != 0) return "ndof must be 6*n_nodes";
  int64_t n_nodes = ndof / 6;
  S = Symbolic();
  S.ndof = ndof;
  S.n = n_free;
  S.n_nodes = n_nodes;
  std::vector<int32_t> free_pos(ndof, -1);
  for (int64_t k = 0; k < n_free; ++k) {
    int32_t d = free_dofs[k];
    if (d < 0 || d >= ndof) return "free DOF out of range";
    if (k > 0 && d <= free_dofs[k - 1]) return "free DOFs must be strictly ascending";
    free_pos[d] = (int32_t)k;
  }
  std::vector<int8_t> nfree(n_nodes, 0);
  for (int64_t k = 0; k < n_free; ++k) nfree[free_dofs[k] / 6]++;
  // ---- node graph over nodes with free DOFs
  NodeGraph g;
  g.ptr.assign(n_nodes + 1, 0);
  {
    // two passes (count, fill) over the nodes; each node writes only its
    // own count and adjacency segment, so nodes run in parallel with a
    // thread-local mark array
    for (int pass = 0; pass < 2; ++pass) {
      if (pass == 1) {
        for (int64_t b = 0; b < n_nodes; ++b) g.ptr[b + 1] += g.ptr[b];
        g.adj.resize(g.ptr[n_nodes]);
      }
#pragma omp parallel
      {
        std::vector<int64_t> mark(n_nodes, -1);
#pragma omp for schedule(dynamic, 1024)
        for (int64_t b = 0; b < n_nodes; ++b) {
          if (!nfree[b]) continue;
          int64_t cnt = 0, at = pass == 1 ? g.ptr[b] : 0;
          for (int c = 0; c < 6; ++c) {
            int64_t j = 6 * b + c;
            if (free_pos[j] < 0) continue;
            for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) {
              int64_t i = rowval[p];
              if (free_pos[i] < 0) continue;
              int64_t a = i / 6;
              if (a == b || mark[a] == b) continue;
              mark[a] = b;
              if (pass == 0) ++cnt;
              else g.adj[at++] = (int32_t)a;
            }
          }
          if (pass == 0) g.ptr[b + 1] = cnt;
        }
      }
    }
  }
  std::vector<int32_t> active;
  for (int64_t v = 0; v < n_nodes; ++v)
    if (nfree[v]) active.push_back((int32_t)v);
  int64_t na = (int64_t)active.size();
  // ---- nested dissection
  std::vector<int32_t> order;
  nested_dissection(g, xyz, active, opt.leaf_nodes, order);
  std::vector<int32_t> ipos(n_nodes, -1);
  for (int64_t p = 0; p < na; ++p) ipos[order[p]] = (int32_t)p;
  // ---- elimination tree (Liu) on the node graph in ND order
  std::vector<int32_t> parent(na, -1), anc(na, -1);
  for (int64_t i = 0; i < na; ++i) {
    int32_t v = order[i];
    for (int64_t p = g.ptr[v]; p < g.ptr[v + 1]; ++p) {
      int64_t j = ipos[g.adj[p]];
      if (j >= i) continue;
      while (j != -1 && j < i) {
        int64_t nx = anc[j];
        anc[j] = (int32_t)i;
        if (nx == -1) { parent[j] = (int32_t)i; break; }
        j = nx;
      }
    }
  }
  // ---- postorder
  std::vector<int32_t> post;
  post.reserve(na);
  {
    std::vector<int32_t> head(na, -1), nxt(na, -1);
    for (int64_t j = na - 1; j >= 0; --j)
      if (parent[j] >= 0) { nxt[j] = head[parent[j]]; head[parent[j]] = (int32_t)j; }
    std::vector<int32_t> stk;
    for (int64_t r = 0; r < na; ++r) {
      if (parent[r] >= 0) continue;
      stk.push_back((int32_t)r);
      while (!stk.empty()) {
        int32_t v = stk.back();
        if (head[v] >= 0) {
          int32_t c = head[v];
          head[v] = nxt[c];
          stk.push_back(c);
        } else {
          stk.pop_back();
          post.push_back(v);
        }
      }
    }
  }
  {
    std::vector<int32_t> order2(na), newpos(na);
    for (int64_t k = 0; k < na; ++k) { order2[k] = order[post[k]]; newpos[post[k]] = (int32_t)k; }
    std::vector<int32_t> parent2(na, -1);
    for (int64_t j = 0; j < na; ++j)
      if (parent[j] >= 0) parent2[newpos[j]] = newpos[parent[j]];
    order.swap(order2);
    parent.swap(parent2);
    for (int64_t p = 0; p < na; ++p) ipos[order[p]] = (int32_t)p;
  }
  // ---- node column counts (struct sizes) via row subtrees, DOF weighted
  std::vector<int64_t> cnt(na, 0), wbelow(na, 0);
  {
    std::vector<int64_t> mark(na, -1);
    for (int64_t i = 0; i < na; ++i) {
      mark[i] = i;
      int32_t v = order[i];
      for (int64_t p = g.ptr[v]; p < g.ptr[v + 1]; ++p) {
        int64_t j = ipos[g.adj[p]];
        if (j >= i) continue;
        while (j != -1 && mark[j] != i) {
          cnt[j]++;
          wbelow[j] += nfree[v];
          mark[j] = i;
          j = parent[j];
        }
      }
    }
  }
  std::vector<int32_t> nchild(na, 0);
  for (int64_t j = 0; j < na; ++j)
    if (parent[j] >= 0) nchild[parent[j]]++;
  // ---- fundamental supernodes
  std::vector<int32_t> ffirst;
  for (int64_t j = 0; j < na; ++j) {
    bool merge = j > 0 && parent[j - 1] == j && cnt[j - 1] == cnt[j] + 1 && nchild[j] == 1;
    if (!merge) ffirst.push_back((int32_t)j);
  }
  int64_t nf = (int64_t)ffirst.size();
  ffirst.push_back((int32_t)na);
  std::vector<int32_t> node2f(na);
  for (int64_t s = 0; s < nf; ++s)
    for (int64_t j = ffirst[s]; j < ffirst[s + 1]; ++j) node2f[j] = (int32_t)s;
  std::vector<int32_t> fparent(nf, -1);
  for (int64_t s = 0; s < nf; ++s) {
    int64_t l = ffirst[s + 1] - 1;
    if (parent[l] >= 0) fparent[s] = node2f[parent[l]];
  }
  // ---- relaxed amalgamation (DOF-weighted, CHOLMOD-style thresholds)
  std::vector<int64_t> fcols(nf, 0), fbelow(nf, 0), fnz(nf, 0);
  auto entries = [](int64_t c, int64_t b) { return c * (c + 1) / 2 + c * b; };
  for (int64_t s = 0; s < nf; ++s) {
    for (int64_t j = ffirst[s]; j < ffirst[s + 1]; ++j) fcols[s] += nfree[order[j]];
    fbelow[s] = wbelow[ffirst[s + 1] - 1];
    fnz[s] = entries(fcols[s], fbelow[s]);
  }
  std::vector<int32_t> rep(nf);
  std::iota(rep.begin(), rep.end(), 0);
  std::function<int32_t(int32_t)> find = [&](int32_t x) {
    while (rep[x] != x) { rep[x] = rep[rep[x]]; x = rep[x]; }
    return x;
  };
  {
    std::vector<std::vector<int32_t>> fch(nf);
    for (int64_t s = 0; s < nf; ++s)
      if (fparent[s] >= 0) fch[fparent[s]].push_back((int32_t)s);
    for (int64_t p = 0; p < nf; ++p) {
      // merge smaller children first
      std::vector<int32_t> ch = fch[p];
      std::sort(ch.begin(), ch.end(), [&](int32_t a, int32_t b) { return fcols[a] < fcols[b]; });
      for (int32_t c : ch) {
        int64_t nc = fcols[c] + fcols[p];
        int64_t ne = entries(nc, fbelow[p]);
        int64_t tr = fnz[c] + fnz[p];
        double frac = ne > 0 ? double(ne - tr) / double(ne) : 0.0;
        bool merge = nc <= opt.relax_cols[0] ||
                     (nc <= opt.relax_cols[1] && frac < opt.relax_zeros[0]) ||
                     (nc <= opt.relax_cols[2] && frac < opt.relax_zeros[1]) ||
                     frac < opt.relax_zeros[2];
        if (merge) {
          rep[c] = (int32_t)p;
          fcols[p] = nc;
          fnz[p] = tr;
        }
      }
    }
  }
  // ---- final supernodes: members, tree, postorder
  std::vector<int32_t> fid(nf, -1);
  std::vector<int32_t> final_rep;
  for (int64_t s = 0; s < nf; ++s)
    if (find((int32_t)s) == s) { fid[s] = (int32_t)final_rep.size(); final_rep.push_back((int32_t)s); }
  int64_t ns = (int64_t)final_rep.size();
  std::vector<std::vector<int32_t>> members(ns);  // node positions (old), increasing
  for (int64_t s = 0; s < nf; ++s) {
    int32_t F = fid[find((int32_t)s)];
    for (int64_t j = ffirst[s]; j < ffirst[s + 1]; ++j) members[F].push_back((int32_t)j);
  }
  std::vector<int32_t> sp(ns, -1);
  for (int64_t F = 0; F < ns; ++F) {
    int32_t r = final_rep[F];
    if (fparent[r] >= 0) sp[F] = fid[find(fparent[r])];
  }
  std::vector<int32_t> spost;
  {
    std::vector<int32_t> head(ns, -1), nxt(ns, -1);
    for (int64_t j = ns - 1; j >= 0; --j)
      if (sp[j] >= 0) { nxt[j] = head[sp[j]]; head[sp[j]] = (int32_t)j; }
    std::vector<int32_t> stk;
    for (int64_t r = 0; r < ns; ++r) {
      if (sp[r] >= 0) continue;
      stk.push_back((int32_t)r);
      while (!stk.empty()) {
        int32_t v = stk.back();
        if (head[v] >= 0) { int32_t c = head[v]; head[v] = nxt[c]; stk.push_back(c); }
        else { stk.pop_back(); spost.push_back(v); }
      }
    }
  }
  // new node positions
  std::vector<int32_t> npos(na);       // old position -> new position
  std::vector<int32_t> nnode(na);      // new position -> node id
  std::vector<int32_t> sfirst(ns + 1);  // new node positions per final supernode (postordered)
  std::vector<int32_t> snew(ns);        // old F -> new index
  {
    int64_t p = 0;
    for (int64_t k = 0; k < ns; ++k) {
      int32_t F = spost[k];
      snew[F] = (int32_t)k;
      sfirst[k] = (int32_t)p;
      for (int32_t j : members[F]) { npos[j] = (int32_t)p; nnode[p] = order[j]; ++p; }
    }
    sfirst[ns] = (int32_t)p;
  }
  std::vector<int32_t> sparent(ns, -1);
  for (int64_t F = 0; F < ns; ++F)
    if (sp[F] >= 0) sparent[snew[F]] = snew[sp[F]];
  for (int64_t v = 0; v < n_nodes; ++v) ipos[v] = -1;
  for (int64_t p = 0; p < na; ++p) ipos[nnode[p]] = (int32_t)p;
  // ---- node-level structures of final supernodes (positions > last member)
  std::vector<std::vector<int32_t>> schildren(ns);
  for (int64_t s = 0; s < ns; ++s)
    if (sparent[s] >= 0) schildren[sparent[s]].push_back((int32_t)s);
  std::vector<std::vector<int32_t>> sstruct(ns);
  {
    std::vector<int64_t> mark(na, -1);
    for (int64_t s = 0; s < ns; ++s) {
      int64_t l = sfirst[s + 1] - 1;
      std::vector<int32_t>& R = sstruct[s];
      for (int64_t p = sfirst[s]; p <= l; ++p) {
        int32_t v = nnode[p];
        for (int64_t q = g.ptr[v]; q < g.ptr[v + 1]; ++q) {
          int64_t u = ipos[g.adj[q]];
          if (u > l && mark[u] != s) { mark[u] = s; R.push_back((int32_t)u); }
        }
      }
      for (int32_t c : schildren[s])
        for (int32_t u : sstruct[c])
          if (u > l && mark[u] != s) { mark[u] = s; R.push_back(u); }
      std::sort(R.begin(), R.end());
    }
  }
  // ---- DOF expansion
  std::vector<int64_t> dfirst(na + 1, 0);
  for (int64_t p = 0; p < na; ++p) dfirst[p + 1] = dfirst[p] + nfree[nnode[p]];
  if (dfirst[na] != n_free) return "internal: free DOF count mismatch";
  S.perm_dof.resize(n_free);
  S.perm_free.resize(n_free);
  S.gdof_to_perm.assign(ndof, -1);
  for (int64_t p = 0; p < na; ++p) {
    int32_t v = nnode[p];
    int64_t k = dfirst[p];
    for (int c = 0; c < 6; ++c) {
      int64_t d = 6 * (int64_t)v + c;
      if (free_pos[d] < 0) continue;
      S.perm_dof[k] = (int32_t)d;
      S.perm_free[k] = free_pos[d];
      S.gdof_to_perm[d] = (int32_t)k;
      ++k;
    }
  }
  S.ns = ns;
  S.sn_first.resize(ns + 1);
  S.sn_parent = sparent;
  S.sn_m.resize(ns);
  S.sn_rows_ptr.assign(ns + 1, 0);
  S.sn_Lptr.assign(ns + 1, 0);
  for (int64_t s = 0; s < ns; ++s) {
    S.sn_first[s] = (int32_t)dfirst[sfirst[s]];
    int64_t c = dfirst[sfirst[s + 1]] - dfirst[sfirst[s]];
    int64_t r = 0;
    for (int32_t u : sstruct[s]) r += nfree[nnode[u]];
    S.sn_m[s] = (int32_t)(c + r);
    S.sn_rows_ptr[s + 1] = S.sn_rows_ptr[s] + c + r;
    S.sn_Lptr[s + 1] = S.sn_Lptr[s] + (c + r) * c;
    S.max_front = std::max<int64_t>(S.max_front, c + r);
    S.max_c = std::max<int64_t>(S.max_c, c);
    for (int64_t k = 0; k < c; ++k) {
      double cj = double(c - k + r);
      S.flops += cj * cj;
    }
  }
  S.sn_first[ns] = (int32_t)n_free;
  S.nnz_L = S.sn_Lptr[ns];
  S.rows.resize(S.sn_rows_ptr[ns]);
  for (int64_t s = 0; s < ns; ++s) {
    int64_t q = S.sn_rows_ptr[s];
    for (int64_t k = S.sn_first[s]; k < S.sn_first[s + 1]; ++k) S.rows[q++] = (int32_t)k;
    for (int32_t u : sstruct[s])
      for (int64_t k = dfirst[u]; k < dfirst[u + 1]; ++k) S.rows[q++] = (int32_t)k;
  }
  std::vector<std::vector<int32_t>>().swap(sstruct);
  // ---- child relative maps and the A scatter map
  S.sn_relptr.assign(ns + 1, 0);
  for (int64_t s = 0; s < ns; ++s)
    S.sn_relptr[s + 1] = S.sn_relptr[s] + (S.sn_m[s] - (S.sn_first[s + 1] - S.sn_first[s]));
  S.rel.assign(S.sn_relptr[ns], -1);
  // lower-permuted CSC of K_ff: bucket c (permuted column c, global DOF
  // perm_dof[c]) holds its entries of permuted row >= c, each with the
  // position of its upper-triangle copy in K (row <= column); the pattern is
  // structurally symmetric, so column perm_dof[c] lists them all.  Buckets
  // are independent: both passes run in parallel over the columns.
  const int32_t* g2p = S.gdof_to_perm.data();
  std::vector<int64_t> lp(n_free + 1, 0);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t c = 0; c < n_free; ++c) {
    const int64_t j = S.perm_dof[c];
    int64_t cnt = 0;
    for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p)
      if (g2p[rowval[p]] >= c) ++cnt;
    lp[c + 1] = cnt;
  }
  for (int64_t k = 0; k < n_free; ++k) lp[k + 1] += lp[k];
  std::vector<int32_t, UninitAlloc<int32_t>> lrow(lp[n_free]);
  std::vector<int32_t> lsrc(lp[n_free]);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t c = 0; c < n_free; ++c) {
    const int64_t j = S.perm_dof[c];
    int64_t q = lp[c];
    for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) {
      const int64_t i = rowval[p];
      const int32_t pi = g2p[i];
      if (pi < c) continue;
      int64_t src = p;
      if (i > j) {   // the upper-triangle copy is entry (j, i), in column i
        const int32_t* b0 = rowval + colptr[i];
        const int32_t* b1 = rowval + colptr[i + 1];
        src = colptr[i] + (std::lower_bound(b0, b1, (int32_t)j) - b0);
      }
      lrow[q] = pi;
      lsrc[q] = (int32_t)src;
      ++q;
    }
  }
  // scatter map (slot of every bucket entry in its supernode's front) and the
  // child -> parent row maps, in parallel over supernodes; entry p of the
  // buckets is entry p of the map, since supernodes own consecutive columns
  S.amap_dst.resize(lp[n_free]);
  int bad = 0;
#pragma omp parallel
  {
    std::vector<int32_t> rowidx(n_free, -1);
#pragma omp for schedule(dynamic, 8) reduction(| : bad)
    for (int64_t s = 0; s < ns; ++s) {
      int64_t m = S.sn_m[s];
      const int32_t* R = S.rows.data() + S.sn_rows_ptr[s];
      for (int64_t k = 0; k < m; ++k) rowidx[R[k]] = (int32_t)k;
      int64_t f = S.sn_first[s];
      for (int64_t j = f; j < S.sn_first[s + 1]; ++j)
        for (int64_t p = lp[j]; p < lp[j + 1]; ++p) {
          int32_t ri = rowidx[lrow[p]];
          if (ri < 0 || ri >= m || R[ri] != lrow[p]) { bad |= 1; continue; }
          S.amap_dst[p] = S.sn_Lptr[s] + ri + m * (j - f);
        }
      for (int32_t ch : schildren[s]) {
        int64_t cc = S.sn_first[ch + 1] - S.sn_first[ch];
        const int32_t* Rc = S.rows.data() + S.sn_rows_ptr[ch];
        int64_t mc = S.sn_m[ch];
        for (int64_t k = cc; k < mc; ++k) {
          int32_t ri = rowidx[Rc[k]];
          if (ri < 0 || ri >= m || R[ri] != Rc[k]) { bad |= 2; continue; }
          S.rel[S.sn_relptr[ch] + (k - cc)] = ri;
        }
      }
      for (int64_t k = 0; k < m; ++k) rowidx[R[k]] = -1;
    }
  }
  S.amap_src.swap(lsrc);   // entry p's source is bucket entry p's
  if (bad & 1) return "internal: A entry outside its front";
  if (bad & 2) return "internal: child row outside its parent front";
  // ---- levels
  S.sn_level.assign(ns, 0);
  for (int64_t s = 0; s < ns; ++s)
    if (sparent[s] >= 0) S.sn_level[sparent[s]] = std::max(S.sn_level[sparent[s]], S.sn_level[s] + 1);
  int64_t nl = 0;
  for (int64_t s = 0; s < ns; ++s) nl = std::max<int64_t>(nl, S.sn_level[s] + 1);
  S.n_levels = nl;
  S.level_ptr.assign(nl + 1, 0);
  for (int64_t s = 0; s < ns; ++s) S.level_ptr[S.sn_level[s] + 1]++;
  for (int64_t l = 0; l < nl; ++l) S.level_ptr[l + 1] += S.level_ptr[l];
  S.level_sn.resize(ns);
  {
    std::vector<int32_t> pos(S.level_ptr.begin(), S.level_ptr.end() - 1);
    for (int64_t s = 0; s < ns; ++s) S.level_sn[pos[S.sn_level[s]]++] = (int32_t)s;
  }
  // extend-add segments: (level, child rank)
  S.ea_level_ptr.assign(nl + 1, 0);
  S.ea_ptr.clear();
  S.ea_child.clear();
  for (int64_t l = 0; l < nl; ++l) {
    int64_t maxr = 0;
    for (int64_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q)
      maxr = std::max<int64_t>(maxr, (int64_t)schildren[S.level_sn[q]].size());
    S.ea_level_ptr[l] = (int32_t)S.ea_ptr.size();
    for (int64_t k = 0; k < maxr; ++k) {
      S.ea_ptr.push_back((int32_t)S.ea_child.size());
      for (int64_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
        const auto& ch = schildren[S.level_sn[q]];
        if ((int64_t)ch.size() > k) S.ea_child.push_back(ch[k]);
      }
    }
  }
  S.ea_level_ptr[nl] = (int32_t)S.ea_ptr.size();
  S.ea_ptr.push_back((int32_t)S.ea_child.size());
  // ---- update arena: U(s) lives from level(s) to level(parent(s)); first fit
  S.sn_Uptr.assign(ns, -1);
  {
    struct Blk { int64_t off, size; };
    std::vector<Blk> freel;  // sorted by offset
    int64_t top = 0;
    auto alloc = [&](int64_t size) -> int64_t {
      for (size_t k = 0; k < freel.size(); ++k)
        if (freel[k].size >= size) {
          int64_t off = freel[k].off;
          freel[k].off += size;
          freel[k].size -= size;
          if (freel[k].size == 0) freel.erase(freel.begin() + k);
          return off;
        }
      // extend: merge with a free block at the top if present
      if (!freel.empty() && freel.back().off + freel.back().size == top) {
        int64_t off = freel.back().off;
        top = off + size;
        freel.pop_back();
        return off;
      }
      int64_t off = top;
      top += size;
      return off;
    };
    auto release = [&](int64_t off, int64_t size) {
      Blk b{off, size};
      auto it = std::lower_bound(freel.begin(), freel.end(), b,
                                 [](const Blk& x, const Blk& y) { return x.off < y.off; });
      it = freel.insert(it, b);
      size_t k = it - freel.begin();
      if (k + 1 < freel.size() && freel[k].off + freel[k].size == freel[k + 1].off) {
        freel[k].size += freel[k + 1].size;
        freel.erase(freel.begin() + k + 1);
      }
      if (k > 0 && freel[k - 1].off + freel[k - 1].size == freel[k].off) {
        freel[k - 1].size += freel[k].size;
        freel.erase(freel.begin() + k);
      }
    };
    auto usize = [&](int64_t s) {
      int64_t r = S.sn_m[s] - (S.sn_first[s + 1] - S.sn_first[s]);
      return r * r;
    };
    for (int64_t l = 0; l < nl; ++l) {
      for (int64_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
        int32_t s = S.level_sn[q];
        int64_t sz = usize(s);
        if (sz > 0 && sparent[s] >= 0) S.sn_Uptr[s] = alloc(sz);
      }
      for (int64_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q)
        for (int32_t ch : schildren[S.level_sn[q]])
          if (S.sn_Uptr[ch] >= 0) release(S.sn_Uptr[ch], usize(ch));
    }
    S.u_arena = top;
  }
  S.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return "";
}

}  // namespace jfg
