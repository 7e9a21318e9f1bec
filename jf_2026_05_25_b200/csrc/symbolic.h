// symbolic.h -- host-side symbolic analysis of K_ff for the supernodal
// multifrontal Cholesky (nested dissection, elimination tree, supernodes,
// front index maps, level schedule, update-matrix arena).
#pragma once
#include <cstdint>
#include <string>
#include <memory>
#include <utility>
#include <vector>

namespace jfg {

// Allocator whose value-initialising resize leaves the elements
// uninitialised: for arrays that a parallel loop fills completely (the
// zeroing pass of std::vector would run on one thread and touch every page)
template <class T>
struct UninitAlloc : std::allocator<T> {
  template <class U>
  struct rebind { using other = UninitAlloc<U>; };
  UninitAlloc() = default;
  template <class U>
  UninitAlloc(const UninitAlloc<U>&) {}
  template <class U>
  void construct(U* p) { ::new ((void*)p) U; }
  template <class U, class... Args>
  void construct(U* p, Args&&... args) { ::new ((void*)p) U(std::forward<Args>(args)...); }
};

struct SymbolicOptions {
  int leaf_nodes = 24;          // nested-dissection leaf size (nodes)
  int relax_cols[3] = {24, 64, 192};    // amalgamation column thresholds (DOFs)
  double relax_zeros[3] = {0.6, 0.15, 0.05};  // zero-fraction thresholds
  // Overrides from JFG_ND_LEAF, JFG_RELAX_COLS="a,b,c", JFG_RELAX_ZEROS="x,y,z"
  // (used by the tile/amalgamation autotuner).
  static SymbolicOptions from_env();
};

struct Symbolic {
  // problem
  int64_t ndof = 0;             // global DOFs (6 per node)
  int64_t n = 0;                // free DOFs (order of K_ff)
  int64_t n_nodes = 0;
  // permutation: perm_dof[k] = global DOF eliminated k-th; free position of it
  std::vector<int32_t> perm_dof;        // n
  std::vector<int32_t> perm_free;       // n  (position in free_dofs)
  std::vector<int32_t> gdof_to_perm;    // ndof, -1 if fixed
  // supernodes (postordered: children before parents)
  int64_t ns = 0;
  std::vector<int32_t> sn_first;        // ns+1 (permuted column ranges)
  std::vector<int32_t> sn_parent;       // ns
  std::vector<int32_t> sn_m;            // rows (cols + update rows)
  std::vector<int64_t> sn_rows_ptr;     // ns+1 into rows
  std::vector<int32_t> rows;            // permuted row indices per supernode
  std::vector<int64_t> sn_Lptr;         // ns+1, offsets into the factor (m*c each)
  std::vector<int64_t> sn_Uptr;         // ns, offsets into the update arena (r*r)
  std::vector<int64_t> sn_relptr;       // ns+1 into rel (r entries per supernode)
  std::vector<int32_t> rel;             // child update row -> parent front row
  std::vector<int32_t> sn_level;        // ns
  int64_t n_levels = 0;
  std::vector<int32_t> level_ptr;       // n_levels+1 into level_sn
  std::vector<int32_t> level_sn;        // supernodes grouped by level
  // extend-add launches: for each level, children grouped by rank so that
  // one launch never has two children of the same parent.
  std::vector<int32_t> ea_ptr;          // per (level, rank) segment start into ea_child
  std::vector<int32_t> ea_level_ptr;    // n_levels+1 into ea_ptr segments
  std::vector<int32_t> ea_child;
  // A scatter: K CSC position -> factor offset (upper triangle of K_ff)
  std::vector<int32_t> amap_src;
  std::vector<int64_t, UninitAlloc<int64_t>> amap_dst;   // filled in parallel: no zeroing pass
  int64_t nnz_L = 0;                    // sum m*c
  int64_t u_arena = 0;                  // update arena size (entries)
  int64_t max_front = 0;
  int64_t max_c = 0;
  double flops = 0;                     // sum over columns of c_j^2
  double seconds = 0;
};

// Build the symbolic analysis.  colptr/rowval: CSC pattern of the global K
// (ndof = 6*n_nodes); free_dofs ascending; xyz: n_nodes x 3 (row per node).
// Returns an empty string on success, or an error message.
std::string analyze(int64_t ndof, const int64_t* colptr, const int32_t* rowval,
                    int64_t n_free, const int32_t* free_dofs, const double* xyz,
                    const SymbolicOptions& opt, Symbolic& out);

}  // namespace jfg
