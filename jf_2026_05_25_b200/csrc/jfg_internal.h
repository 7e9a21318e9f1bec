// jfg_internal.h -- shared internals of libjfemgpu (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/jfemgpu.h"
#include "symbolic.h"

namespace jfg {

void set_error(const std::string& msg, int64_t detail = 0);

// Launch accounting (one increment per kernel launch of this library) and
// per-kernel device-time statistics for the roofline report.
void count_launch(int n = 1);
int64_t launch_count();

enum KernelStat : int { KS_SCHUR = 0, KS_Q4 = 1, KS_ASSEMBLY = 2, KS_SOLVE = 3, KS_T10 = 4,
                        KS_F_EA = 5, KS_F_POTRF = 6, KS_F_TRSM = 7, KS_F_PANEL = 8, KS_S_VEC = 9,
                        KS_S_FDIAG = 10, KS_S_FUPD = 11, KS_S_BPART = 12, KS_S_BDIAG = 13,
                        // per elimination-tree level of a solve sweep (profiling level 2):
                        // forward level l at KS_LEVEL_FWD + l, backward at KS_LEVEL_BWD + l
                        KS_LEVEL_FWD = 14, KS_LEVEL_BWD = 14 + 48, KS_COUNT = 14 + 96 };
constexpr int KS_MAX_LEVELS = 48;
struct KernelStats {
  int64_t launches[KS_COUNT] = {0};
  double ms[KS_COUNT] = {0};
  double units[KS_COUNT] = {0};   // algorithmic flops (SCHUR) or bytes (others)
};
KernelStats& kernel_stats();
bool profiling_enabled();
int profiling_level();
void set_profiling(int level);
// Event brackets around instrumented launches (no-ops when profiling is off).
int prof_start(cudaStream_t st);
void prof_end(int slot, cudaStream_t st, int kind, double units);
void prof_flush();   // call after the stream has been synchronised

#define JFG_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      ::jfg::set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) +   \
                       " at " __FILE__ ":" + std::to_string(__LINE__));         \
      return JFG_CUDA_ERROR;                                                    \
    }                                                                           \
  } while (0)

#define JFG_TRY(call)                 \
  do {                                \
    jfg_status s_ = (call);           \
    if (s_ != JFG_OK) return s_;      \
  } while (0)

// Device buffer with byte accounting against the context budget.
struct DevMem {
  void* p = nullptr;
  size_t bytes = 0;
};

#ifdef __CUDACC__
// Work tiles of a level launch: with a tile list, CTA x takes tile tiles[x]
// = (position of the front in the level's list, block of that front); the
// list holds only blocks that have work, so a level of fronts of very
// different sizes launches no empty CTAs.  Without one the grid is
// (blocks, fronts).
__device__ __forceinline__ void tile_of(const int2* __restrict__ tiles, int& q, int& b) {
  if (tiles) {
    const int2 t = tiles[blockIdx.x];
    q = t.x;
    b = t.y;
  } else {
    q = blockIdx.y;
    b = blockIdx.x;
  }
}
#endif

// Error record written by device kernels (first failing element / pivot).
// doubles per CQUAD4 of the scratch record passed from the thread-per-element
// pass to the warp-per-element pass of the element kernel
constexpr int Q4_PREP_STRIDE = 210;
// CQUAD4 prep record (k_q4_prep, one per element): local corner coordinates,
// element frame rows v1 v2 v3, rotated section Cm Cb Cs, the shape law,
// centre Jacobian determinant and inverse, k6rot, h, the shear flag, the
// MacNeal shear operator D (4 x 12) and Z^-1 D, internal-mode blocks, status.
constexpr int Q4P_LC = 0, Q4P_V = 8, Q4P_CM = 17, Q4P_CB = 26, Q4P_CS = 35, Q4P_SHP = 39, Q4P_DETJC = 40,
              Q4P_IJC = 41, Q4P_K6 = 45, Q4P_H = 46, Q4P_SHEAR = 47, Q4P_D = 48, Q4P_SOL = 96, Q4P_CI = 144,
              Q4P_KBB = 176, Q4P_KBBB = 192, Q4P_STATUS = 208;
static_assert(Q4P_STATUS < Q4_PREP_STRIDE, "CQUAD4 prep record layout");

struct DevError {
  int32_t code;        // 0 = none
  int32_t pad;
  int64_t index;       // element index or permuted column
};

// Element-kernel status codes written to DevError::code.
enum ElemErr : int32_t {
  EE_NONE = 0,
  EE_NOT_FLAT = 100,
  EE_FLAGS = 101,
  EE_JACOBIAN = 1,
  EE_SHEAR = 11,
  EE_ENRICH = 20,
  EE_T10_JAC = 200,
  EE_T10_MAT = 202,
  EE_Q8_SHAPE = 300,
  EE_Q8_DREF = 301,
  EE_Q8_SINGULAR = 302,
  EE_T3_FLEX = 400,      // CTRIA3 residual bending flexibility not positive
  EE_PIVOT = 500,
  EE_TC_TIMEOUT = 600,   // a bounded tensor-core pipeline wait expired
};

}  // namespace jfg

// ---- opaque ABI objects -----------------------------------------------------
struct jfg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t astream = nullptr;   // device allocations and frees (stream-ordered, otherwise idle)
  int64_t budget = 0;
  int64_t used = 0;
};

struct NumericFactor;   // defined in factor.cu

namespace jfg {
// CSC pattern and slot map on the host (built once per mesh)
struct HostPattern {
  std::vector<int64_t> colptr;
  std::vector<int32_t> rowval;
  std::vector<int32_t, UninitAlloc<int32_t>> slot;   // triplet -> nz position (every entry written)
  std::vector<int64_t> diag_pos;    // ndof, -1 when structurally absent
};
}  // namespace jfg

struct jfg_model {
  jfg_ctx* ctx = nullptr;
  // the model's own stream: models of one context may be driven from
  // different host threads (and captured into graphs) independently
  cudaStream_t stream = nullptr;
  int64_t n_nodes = 0, n_q4 = 0, n_q8 = 0, n_t10 = 0, n_t3 = 0, ndof = 0;
  // host copies of the inputs (pattern build, element capture)
  std::vector<double> h_xyz, h_R, h_q4s, h_q8s, h_t10m, h_t3s;
  std::vector<int32_t> h_q4n, h_q8n, h_t10n, h_t3n;
  // device inputs
  double *d_xyz = nullptr, *d_R = nullptr, *d_q4s = nullptr, *d_q8s = nullptr, *d_t10m = nullptr, *d_t3s = nullptr;
  int32_t *d_q4n = nullptr, *d_q8n = nullptr, *d_t10n = nullptr, *d_t3n = nullptr;
  // element values: Q4 576 / T10 900 / Q8 2304 doubles per element
  int64_t ev_t10_off = 0, ev_q8_off = 0, ev_t3_off = 0, n_ev = 0;
  double* d_ev = nullptr;
  double* d_q4prep = nullptr;   // n_q4 x Q4_PREP_STRIDE scratch between the two CQUAD4 passes
  jfg::DevError* d_err = nullptr;
  // pattern + slot map (built once)
  bool pattern_built = false;
  int64_t nnz = 0, n_trip = 0;
  // host pattern: shared (read-only once built) by the models of one mesh
  std::shared_ptr<jfg::HostPattern> pat = std::make_shared<jfg::HostPattern>();
  int64_t* d_diag_pos = nullptr;
  int64_t* d_colptr = nullptr;
  int32_t* d_rowval = nullptr;
  int32_t* d_nzptr = nullptr;       // nnz+1, into d_trip
  int32_t* d_trip = nullptr;        // element-value index of each triplet, triplet order
  int64_t* d_tpos = nullptr;        // CSC position of the transposed entry
  double* d_nzval = nullptr;
  bool values_ready = false;
  // symbolic
  bool sym_ready = false;
  // the analysis (read-only once made; shared by the models of one mesh and
  // free set)
  std::shared_ptr<const jfg::Symbolic> symp = std::make_shared<jfg::Symbolic>();
  const jfg::Symbolic& sym() const { return *symp; }
  // analysis of the same mesh taken over from another model
  // (jfg_model_share_structure): used by jfg_set_free_dofs when its free set
  // is the one this analysis was made for
  std::vector<int32_t> sym_cache_free;
  std::shared_ptr<const jfg::Symbolic> sym_cache;
  bool has_sym_cache = false;
  NumericFactor* num = nullptr;
  // asynchronous calls (jfg_*_async): the caller's stream waits on aev_out;
  // async_factor is the precision of a factorisation not yet checked (-1 none)
  cudaEvent_t aev_in = nullptr, aev_out = nullptr;
  int async_factor = -1;
  int async_prec = -1;              // precision of the last factorisation enqueued
  // timings of the last calls (seconds, device events)
  double t_elements = 0, t_assembly = 0, t_factor = 0, t_solve = 0;
};

namespace jfg {

// elements.cu
jfg_status launch_elements(jfg_model* m, cudaStream_t st);
// assembly.cu: diag(K), max |element entry| and the grids' 3 x 3 diagonal
// blocks, computed on the device (host outputs)
jfg_status device_diag(jfg_model* m, double* diag, double* max_elem_stiff);
jfg_status device_node_blocks(jfg_model* m, double* blocks);
// factor.cu: fronts of each level listed by decreasing width (then index),
// as the level launches expect; done once, right after the analysis
void sort_level_lists(Symbolic& S);
jfg_status launch_q4_prep(const jfg_model* m, cudaStream_t st);
jfg_status launch_elements_into(const jfg_model* m, cudaStream_t st, double* ev, double* q4prep, DevError* err);
// CTRIA3 element matrices (324 doubles each, column-major) into ev
jfg_status launch_t3(const jfg_model* m, cudaStream_t st, double* ev, DevError* err);
// assembly.cu
jfg_status build_pattern(jfg_model* m);
jfg_status launch_assembly(jfg_model* m, cudaStream_t st);
jfg_status launch_gather_into(const jfg_model* m, cudaStream_t st, const double* ev, double* nzval);
void spmv_csc_sym(const jfg_model* m, int nrhs, const double* x, int64_t ldx, double* y,
                  int64_t ldy, cudaStream_t st);
void residual_dd(const jfg_model* m, int nrhs, const double* x, const double* f, double* r, cudaStream_t st);
// factor.cu
jfg_status numeric_create(jfg_model* m);
void numeric_destroy(jfg_model* m);
jfg_status numeric_factor(jfg_model* m, int precision);
jfg_status numeric_factor_enqueue(jfg_model* m, int precision);
jfg_status numeric_factor_finish(jfg_model* m, int precision);
jfg_status numeric_apply(jfg_model* m, int nrhs, const double* Fd, double* Ud, int precision);
int numeric_current_precision(jfg_model* m);
void numeric_bytes(jfg_model* m, int precision, int nrhs, int64_t* now, int64_t* peak);
jfg_status numeric_solve(jfg_model* m, int nrhs, const double* hF, double* hU, double tol,
                         int max_ir, jfg_solve_report* rep, bool device_io);
jfg_status numeric_factor_diag(jfg_model* m, double* out);
// stress.cu
jfg_status recover_t10_stresses(jfg_model* m, int nrhs, const double* U_dev, double* out_dev, cudaStream_t st);
jfg_status recover_q4_stresses(jfg_model* m, int nrhs, const double* U_dev, double* out_dev, cudaStream_t st);
// memory
jfg_status dev_alloc(jfg_ctx* c, void** p, size_t bytes);
void dev_free(jfg_ctx* c, void* p, size_t bytes);

}  // namespace jfg
