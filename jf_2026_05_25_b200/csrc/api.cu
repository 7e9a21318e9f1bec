// api.cu -- the extern "C" entry points of libjfemgpu.so (include/jfemgpu.h).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "jfg_internal.h"

namespace jfg {

static std::atomic<int64_t> g_launches{0};
static KernelStats g_stats;
static int g_prof = 0;   // 0 off, 1 coarse kernel classes, 2 every class
void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
int64_t launch_count() { return g_launches.load(); }
KernelStats& kernel_stats() { return g_stats; }
bool profiling_enabled() { return g_prof > 0; }
int profiling_level() { return g_prof; }
void set_profiling(int level) { g_prof = level < 0 ? 0 : (level > 2 ? 2 : level); }

struct ProfSlot { cudaEvent_t a = nullptr, b = nullptr; int kind = 0; double units = 0; bool live = false; };
static std::vector<ProfSlot> g_slots;
int prof_start(cudaStream_t st) {
  if (!g_prof) return -1;
  int idx = -1;
  for (size_t k = 0; k < g_slots.size(); ++k)
    if (!g_slots[k].live) { idx = (int)k; break; }
  if (idx < 0) {
    g_slots.emplace_back();
    idx = (int)g_slots.size() - 1;
    cudaEventCreate(&g_slots[idx].a);
    cudaEventCreate(&g_slots[idx].b);
  }
  g_slots[idx].live = true;
  cudaEventRecord(g_slots[idx].a, st);
  return idx;
}
void prof_end(int slot, cudaStream_t st, int kind, double units) {
  if (slot < 0) return;
  cudaEventRecord(g_slots[slot].b, st);
  g_slots[slot].kind = kind;
  g_slots[slot].units = units;
}
void prof_flush() {
  for (auto& sl : g_slots) {
    if (!sl.live) continue;
    cudaEventSynchronize(sl.b);
    float ms = 0;
    cudaEventElapsedTime(&ms, sl.a, sl.b);
    g_stats.launches[sl.kind] += 1;
    g_stats.ms[sl.kind] += ms;
    g_stats.units[sl.kind] += sl.units;
    sl.live = false;
  }
}

static thread_local std::string g_err;
static thread_local int64_t g_err_detail = 0;

void set_error(const std::string& msg, int64_t detail) {
  g_err = msg;
  g_err_detail = detail;
}

// Device memory comes from one memory pool per device, owned by the
// library, by stream-ordered allocation on the context's allocation stream
// (an otherwise idle stream).  cudaFree synchronises the whole device: with
// several models driven from several host threads, one model's free (a
// temporary buffer, an evicted model) waited for every other model's kernels
// -- a factorisation step of a large front runs for up to a second -- and
// held the other threads' CUDA calls meanwhile.  A free ordered on the idle
// allocation stream waits for nothing.  Every free site has first
// synchronised the stream that used the memory (the model's stream), so the
// memory is idle when it goes back to the pool.  The pool's release
// threshold stays 0: freed memory returns to the device at the next
// synchronisation, as after cudaFree, so the device's free-memory figure
// keeps its meaning for other users of the GPU.
namespace {
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pools[kMaxPoolDevices] = {};

cudaError_t device_pool(int dev, cudaMemPool_t* out) {
  if (dev < 0 || dev >= kMaxPoolDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    g_pools[dev] = pool;
  }
  *out = g_pools[dev];
  return cudaSuccess;
}
}  // namespace

jfg_status dev_alloc(jfg_ctx* c, void** p, size_t bytes) {
  if (bytes == 0) bytes = 8;
  if (c->budget > 0 && c->used + (int64_t)bytes > c->budget) {
    set_error("device-memory budget exceeded (" + std::to_string(c->used + bytes) + " > " +
              std::to_string(c->budget) + " bytes)");
    return JFG_OOM_BUDGET;
  }
  cudaMemPool_t pool = nullptr;
  cudaError_t e = device_pool(c->device, &pool);
  if (e == cudaSuccess) e = cudaMallocFromPoolAsync(p, bytes, pool, c->astream);
  // the allocation is ordered on the allocation stream: once that stream has
  // reached it, any stream may use the memory
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->astream);
  if (e != cudaSuccess) {
    set_error(std::string("device allocation of ") + std::to_string(bytes) + " bytes failed: " +
              cudaGetErrorString(e));
    return JFG_OOM_BUDGET;
  }
  c->used += (int64_t)bytes;
  return JFG_OK;
}

// The caller has synchronised every stream that used p.
void dev_free(jfg_ctx* c, void* p, size_t bytes) {
  if (!p) return;
  if (bytes == 0) bytes = 8;
  cudaFreeAsync(p, c->astream);
  c->used -= (int64_t)bytes;
}

}  // namespace jfg

using namespace jfg;

namespace {

jfg_status check_model(jfg_model* m) {
  if (!m) { set_error("null model"); return JFG_BAD_INPUT; }
  return JFG_OK;
}

template <typename T>
jfg_status up(jfg_ctx* c, const std::vector<T>& h, T** d) {
  JFG_TRY(dev_alloc(c, (void**)d, sizeof(T) * std::max<size_t>(h.size(), 1)));
  if (!h.empty()) JFG_CUDA(cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return JFG_OK;
}

jfg_status read_elem_error(jfg_model* m) {
  DevError h{};
  JFG_CUDA(cudaMemcpy(&h, m->d_err, sizeof(DevError), cudaMemcpyDeviceToHost));
  if (h.code == 0) return JFG_OK;
  JFG_CUDA(cudaMemset(m->d_err, 0, sizeof(DevError)));
  std::string what;
  jfg_status st = JFG_BAD_INPUT;
  switch (h.code) {
    case EE_NOT_FLAT: what = "CQUAD4 is warped (only flat elements are on the device path)"; st = JFG_UNSUPPORTED; break;
    case EE_FLAGS: what = "CQUAD4 section flags are not the default SOL101 path"; st = JFG_UNSUPPORTED; break;
    case EE_JACOBIAN: what = "CQUAD4 has a degenerate Jacobian"; break;
    case EE_ENRICH: what = "CQUAD4 internal-mode block is singular"; break;
    case EE_T10_JAC: what = "CTETRA10 has a nonpositive Jacobian at an integration point"; break;
    case EE_T10_MAT: what = "CTETRA10 needs finite E > 0 and -1 < nu < 0.5"; break;
    case EE_Q8_SHAPE: what = "CQUAD8 is not a flat parallelogram with mid-side nodes at the edge midpoints"; st = JFG_UNSUPPORTED; break;
    case EE_Q8_DREF: what = "CQUAD8 bending section needs a positive reference stiffness D11"; break;
    case EE_Q8_SINGULAR: what = "CQUAD8 transverse-shear flexibility is singular"; break;
    case EE_T3_FLEX: what = "CTRIA3 residual normal bending flexibility is not positive"; break;
    default:
      if (h.code >= EE_SHEAR && h.code < EE_SHEAR + 10) what = "CQUAD4 MacNeal shear block is degenerate";
      else what = "element kernel error " + std::to_string(h.code);
  }
  set_error(what + " (element " + std::to_string(h.index) + ")", h.index);
  return st;
}

}  // namespace

extern "C" {

const char* jfg_last_error(void) { return g_err.c_str(); }
int64_t jfg_last_error_detail(void) { return g_err_detail; }

jfg_status jfg_create(jfg_ctx** out, const jfg_config* cfg) {
  if (!out) { set_error("null output"); return JFG_BAD_INPUT; }
  jfg_ctx* c = new jfg_ctx();
  c->device = cfg ? cfg->device : 0;
  c->budget = cfg ? cfg->hbm_budget_bytes : 0;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) {
    set_error(std::string("cudaSetDevice failed: ") + cudaGetErrorString(e));
    delete c;
    return JFG_CUDA_ERROR;
  }
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->astream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    set_error(std::string("cudaStreamCreate failed: ") + cudaGetErrorString(e));
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return JFG_CUDA_ERROR;
  }
  *out = c;
  return JFG_OK;
}

jfg_status jfg_destroy(jfg_ctx* c) {
  if (!c) return JFG_OK;
  if (c->astream) {
    cudaStreamSynchronize(c->astream);   // the frees ordered on it
    cudaStreamDestroy(c->astream);
  }
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return JFG_OK;
}

jfg_status jfg_model_upload(jfg_ctx* c, int64_t n_nodes, const double* xyz, const double* node_R, int64_t n_q4,
                            const int32_t* q4_nodes, const double* q4_sect, int64_t n_q8, const int32_t* q8_nodes,
                            const double* q8_sect, int64_t n_t10, const int32_t* t10_nodes, const double* t10_mat,
                            jfg_model** out) {
  if (!c || !out) { set_error("null context/output"); return JFG_BAD_INPUT; }
  if (n_nodes <= 0 || n_q4 < 0 || n_q8 < 0 || n_t10 < 0 || !xyz) { set_error("bad sizes"); return JFG_BAD_INPUT; }
  if ((n_q4 && (!q4_nodes || !q4_sect)) || (n_q8 && (!q8_nodes || !q8_sect)) || (n_t10 && (!t10_nodes || !t10_mat))) {
    set_error("missing element arrays");
    return JFG_BAD_INPUT;
  }
  if (6 * n_nodes >= (int64_t)INT32_MAX) { set_error("too many nodes for 32-bit DOF indices"); return JFG_UNSUPPORTED; }
  for (int64_t i = 0; i < 3 * n_nodes; ++i)
    if (!std::isfinite(xyz[i])) { set_error("non-finite coordinate", i / 3); return JFG_BAD_INPUT; }
  auto chk = [&](const int32_t* a, int64_t len) {
    for (int64_t i = 0; i < len; ++i)
      if (a[i] < 0 || a[i] >= n_nodes) return i;
    return (int64_t)-1;
  };
  int64_t bad;
  if ((bad = chk(q4_nodes, 4 * n_q4)) >= 0) { set_error("CQUAD4 node index out of range", bad / 4); return JFG_BAD_INPUT; }
  if ((bad = chk(q8_nodes, 8 * n_q8)) >= 0) { set_error("CQUAD8 node index out of range", bad / 8); return JFG_BAD_INPUT; }
  if ((bad = chk(t10_nodes, 10 * n_t10)) >= 0) { set_error("CTETRA10 node index out of range", bad / 10); return JFG_BAD_INPUT; }
  cudaSetDevice(c->device);
  jfg_model* m = new jfg_model();
  m->ctx = c;
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete m;
    set_error("cudaStreamCreate failed for the model's stream");
    return JFG_CUDA_ERROR;
  }
  m->n_nodes = n_nodes; m->n_q4 = n_q4; m->n_q8 = n_q8; m->n_t10 = n_t10;
  m->ndof = 6 * n_nodes;
  m->h_xyz.assign(xyz, xyz + 3 * n_nodes);
  if (node_R) m->h_R.assign(node_R, node_R + 9 * n_nodes);
  else {
    m->h_R.assign(9 * n_nodes, 0.0);
    for (int64_t i = 0; i < n_nodes; ++i) m->h_R[9 * i] = m->h_R[9 * i + 4] = m->h_R[9 * i + 8] = 1.0;
  }
  m->h_q4n.assign(q4_nodes, q4_nodes + 4 * n_q4);
  m->h_q4s.assign(q4_sect, q4_sect + JFG_Q4_SECT_STRIDE * n_q4);
  m->h_q8n.assign(q8_nodes, q8_nodes + 8 * n_q8);
  m->h_q8s.assign(q8_sect, q8_sect + JFG_Q8_SECT_STRIDE * n_q8);
  m->h_t10n.assign(t10_nodes, t10_nodes + 10 * n_t10);
  m->h_t10m.assign(t10_mat, t10_mat + 2 * n_t10);
  jfg_status st = JFG_OK;
  if ((st = up(c, m->h_xyz, &m->d_xyz)) || (st = up(c, m->h_R, &m->d_R)) || (st = up(c, m->h_q4n, &m->d_q4n)) ||
      (st = up(c, m->h_q4s, &m->d_q4s)) || (st = up(c, m->h_q8n, &m->d_q8n)) || (st = up(c, m->h_q8s, &m->d_q8s)) ||
      (st = up(c, m->h_t10n, &m->d_t10n)) || (st = up(c, m->h_t10m, &m->d_t10m))) {
    jfg_model_free(m);
    return st;
  }
  m->ev_t10_off = 576 * n_q4;
  m->ev_q8_off = m->ev_t10_off + 900 * n_t10;
  m->n_ev = m->ev_q8_off + 2304 * n_q8;
  if ((st = dev_alloc(c, (void**)&m->d_ev, sizeof(double) * std::max<int64_t>(m->n_ev, 1))) ||
      (st = dev_alloc(c, (void**)&m->d_q4prep, sizeof(double) * Q4_PREP_STRIDE * std::max<int64_t>(n_q4, 1))) ||
      (st = dev_alloc(c, (void**)&m->d_err, sizeof(DevError)))) {
    jfg_model_free(m);
    return st;
  }
  cudaMemset(m->d_err, 0, sizeof(DevError));
  // pageable copies and memsets run on the legacy stream; the model's own
  // stream does not wait for it, so they finish here
  if (cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess) {
    jfg_model_free(m);
    set_error("uploading the model failed");
    return JFG_CUDA_ERROR;
  }
  *out = m;
  return JFG_OK;
}

jfg_status jfg_model_add_tria3(jfg_model* m, int64_t n_t3, const int32_t* t3_nodes, const double* t3_sect) {
  JFG_TRY(check_model(m));
  if (n_t3 < 0 || (n_t3 > 0 && (!t3_nodes || !t3_sect))) { set_error("bad CTRIA3 arrays"); return JFG_BAD_INPUT; }
  if (m->pattern_built || m->n_t3 > 0) {
    set_error("CTRIA3 elements are added once, before the first assembly");
    return JFG_BAD_INPUT;
  }
  for (int64_t i = 0; i < 3 * n_t3; ++i)
    if (t3_nodes[i] < 0 || t3_nodes[i] >= m->n_nodes) { set_error("CTRIA3 node index out of range", i / 3); return JFG_BAD_INPUT; }
  if (n_t3 == 0) return JFG_OK;
  jfg_ctx* c = m->ctx;
  cudaSetDevice(c->device);
  m->h_t3n.assign(t3_nodes, t3_nodes + 3 * n_t3);
  m->h_t3s.assign(t3_sect, t3_sect + JFG_Q4_SECT_STRIDE * n_t3);
  jfg_status st = JFG_OK;
  if ((st = up(c, m->h_t3n, &m->d_t3n)) || (st = up(c, m->h_t3s, &m->d_t3s))) return st;
  // the element values grow by 324 per triangle, after the others
  double* ev = nullptr;
  const int64_t n_ev = m->n_ev + 324 * n_t3;
  if ((st = dev_alloc(c, (void**)&ev, sizeof(double) * n_ev))) return st;
  dev_free(c, m->d_ev, 8 * std::max<int64_t>(m->n_ev, 1));
  m->d_ev = ev;
  m->ev_t3_off = m->n_ev;
  m->n_ev = n_ev;
  m->n_t3 = n_t3;
  JFG_CUDA(cudaStreamSynchronize(cudaStreamLegacy));   // the pageable uploads above
  return JFG_OK;
}

jfg_status jfg_model_free(jfg_model* m) {
  if (!m) return JFG_OK;
  jfg_ctx* c = m->ctx;
  if (m->aev_out) cudaEventSynchronize(m->aev_out);
  if (m->stream) cudaStreamSynchronize(m->stream);
  if (m->aev_in) cudaEventDestroy(m->aev_in);
  if (m->aev_out) cudaEventDestroy(m->aev_out);
  m->aev_in = m->aev_out = nullptr;
  numeric_destroy(m);
  dev_free(c, m->d_xyz, 8 * m->h_xyz.size()); dev_free(c, m->d_R, 8 * m->h_R.size());
  dev_free(c, m->d_q4n, 4 * m->h_q4n.size()); dev_free(c, m->d_q4s, 8 * m->h_q4s.size());
  dev_free(c, m->d_q8n, 4 * m->h_q8n.size()); dev_free(c, m->d_q8s, 8 * m->h_q8s.size());
  dev_free(c, m->d_t10n, 4 * m->h_t10n.size()); dev_free(c, m->d_t10m, 8 * m->h_t10m.size());
  dev_free(c, m->d_t3n, 4 * m->h_t3n.size()); dev_free(c, m->d_t3s, 8 * m->h_t3s.size());
  dev_free(c, m->d_ev, 8 * std::max<int64_t>(m->n_ev, 1)); dev_free(c, m->d_err, sizeof(DevError));
  dev_free(c, m->d_q4prep, 8 * Q4_PREP_STRIDE * std::max<int64_t>(m->n_q4, 1));
  if (m->pattern_built) {
    dev_free(c, m->d_colptr, 8 * (m->ndof + 1)); dev_free(c, m->d_rowval, 4 * m->nnz);
    dev_free(c, m->d_nzptr, 4 * (m->nnz + 1)); dev_free(c, m->d_trip, 4 * m->n_trip);
    dev_free(c, m->d_tpos, 8 * m->nnz); dev_free(c, m->d_nzval, 8 * m->nnz);
    dev_free(c, m->d_diag_pos, 8 * m->ndof);
  }
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return JFG_OK;
}

jfg_status jfg_get_memory(jfg_model* m, int32_t precision, int32_t nrhs, int64_t* now, int64_t* peak) {
  JFG_TRY(check_model(m));
  if (precision != JFG_PREC_FP64 && precision != JFG_PREC_MIXED) { set_error("unknown precision"); return JFG_BAD_INPUT; }
  // inputs, element values and the CQUAD4 prep records
  int64_t own = 8 * (int64_t)(m->h_xyz.size() + m->h_R.size() + m->h_q4s.size() + m->h_q8s.size() + m->h_t10m.size() +
                             m->h_t3s.size()) +
                4 * (int64_t)(m->h_q4n.size() + m->h_q8n.size() + m->h_t10n.size() + m->h_t3n.size()) +
                8 * std::max<int64_t>(m->n_ev, 1) +
                8 * Q4_PREP_STRIDE * std::max<int64_t>(m->n_q4, 1) + (int64_t)sizeof(DevError);
  if (m->pattern_built)
    own += 8 * (m->ndof + 1) + 4 * m->nnz + 4 * (m->nnz + 1) + 4 * m->n_trip + 8 * m->nnz + 8 * m->nnz + 8 * m->ndof;
  int64_t num_now = 0, num_peak = 0;
  if (m->sym_ready) numeric_bytes(m, precision, nrhs, &num_now, &num_peak);
  if (now) *now = own + num_now;
  if (peak) *peak = own + num_peak;
  return JFG_OK;
}

jfg_status jfg_assemble(jfg_model* m) {
  JFG_TRY(check_model(m));
  cudaStream_t st = m->stream;
  cudaEvent_t e0, e1, e2;
  JFG_CUDA(cudaEventCreate(&e0)); JFG_CUDA(cudaEventCreate(&e1)); JFG_CUDA(cudaEventCreate(&e2));
  JFG_CUDA(cudaEventRecord(e0, st));
  JFG_TRY(launch_elements(m, st));
  JFG_CUDA(cudaEventRecord(e1, st));
  if (!m->pattern_built) {
    JFG_CUDA(cudaStreamSynchronize(st));
    JFG_TRY(read_elem_error(m));
    JFG_TRY(build_pattern(m));
    JFG_TRY(up(m->ctx, m->pat->diag_pos, &m->d_diag_pos));
    JFG_CUDA(cudaStreamSynchronize(cudaStreamLegacy));   // the pattern's pageable uploads
  }
  JFG_TRY(launch_assembly(m, st));
  JFG_CUDA(cudaEventRecord(e2, st));
  JFG_CUDA(cudaEventSynchronize(e2));
  float a = 0, b = 0;
  cudaEventElapsedTime(&a, e0, e1);
  cudaEventElapsedTime(&b, e1, e2);
  m->t_elements = a * 1e-3;
  m->t_assembly = b * 1e-3;
  cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
  prof_flush();
  JFG_TRY(read_elem_error(m));
  m->values_ready = true;
  return JFG_OK;
}

jfg_status jfg_get_sizes(jfg_model* m, int64_t* ndof, int64_t* nnz, int64_t* n_triplets) {
  JFG_TRY(check_model(m));
  if (ndof) *ndof = m->ndof;
  if (nnz) *nnz = m->pattern_built ? m->nnz : -1;
  if (n_triplets) *n_triplets = m->pattern_built ? m->n_trip : -1;
  return JFG_OK;
}

jfg_status jfg_get_pattern(jfg_model* m, int64_t* colptr, int32_t* rowval) {
  JFG_TRY(check_model(m));
  if (!m->pattern_built) { set_error("pattern not built: call jfg_assemble first"); return JFG_NOT_READY; }
  if (colptr) std::memcpy(colptr, m->pat->colptr.data(), sizeof(int64_t) * (m->ndof + 1));
  if (rowval) std::memcpy(rowval, m->pat->rowval.data(), sizeof(int32_t) * m->nnz);
  return JFG_OK;
}

jfg_status jfg_get_values(jfg_model* m, double* nzval) {
  JFG_TRY(check_model(m));
  if (!m->values_ready) { set_error("values not assembled"); return JFG_NOT_READY; }
  JFG_CUDA(cudaMemcpy(nzval, m->d_nzval, sizeof(double) * m->nnz, cudaMemcpyDeviceToHost));
  return JFG_OK;
}

jfg_status jfg_get_slot_map(jfg_model* m, int64_t* slot) {
  JFG_TRY(check_model(m));
  if (!m->pattern_built) { set_error("pattern not built"); return JFG_NOT_READY; }
  const int32_t* src = m->pat->slot.data();
#pragma omp parallel for schedule(static)
  for (int64_t t = 0; t < m->n_trip; ++t) slot[t] = src[t];
  return JFG_OK;
}

jfg_status jfg_get_diag(jfg_model* m, double* diag, double* max_elem_stiff) {
  JFG_TRY(check_model(m));
  if (!m->values_ready) { set_error("values not assembled"); return JFG_NOT_READY; }
  // gathered and reduced on the device: only ndof + 1 values cross to the host
  return device_diag(m, diag, max_elem_stiff);
}

jfg_status jfg_get_node_blocks(jfg_model* m, double* blocks) {
  JFG_TRY(check_model(m));
  if (!m->values_ready) { set_error("values not assembled"); return JFG_NOT_READY; }
  if (!blocks) { set_error("null output"); return JFG_BAD_INPUT; }
  return device_node_blocks(m, blocks);
}

jfg_status jfg_get_element_matrix(jfg_model* m, int32_t kind, int64_t elem, double* Ke) {
  JFG_TRY(check_model(m));
  if (!m->values_ready) { set_error("values not assembled"); return JFG_NOT_READY; }
  int64_t off, len;
  if (kind == 0 && elem >= 0 && elem < m->n_q4) { off = 576 * elem; len = 576; }
  else if (kind == 2 && elem >= 0 && elem < m->n_t10) { off = m->ev_t10_off + 900 * elem; len = 900; }
  else if (kind == 1 && elem >= 0 && elem < m->n_q8) { off = m->ev_q8_off + 2304 * elem; len = 2304; }
  else if (kind == 3 && elem >= 0 && elem < m->n_t3) { off = m->ev_t3_off + 324 * elem; len = 324; }
  else { set_error("element kind/index out of range"); return JFG_BAD_INPUT; }
  JFG_CUDA(cudaMemcpy(Ke, m->d_ev + off, sizeof(double) * len, cudaMemcpyDeviceToHost));
  return JFG_OK;
}

jfg_status jfg_set_free_dofs(jfg_model* m, int64_t n_free, const int32_t* free_dofs) {
  JFG_TRY(check_model(m));
  if (!m->pattern_built) { set_error("set_free_dofs before the first assembly"); return JFG_NOT_READY; }
  if (n_free <= 0 || !free_dofs) { set_error("empty free set"); return JFG_BAD_INPUT; }
  numeric_destroy(m);
  m->sym_ready = false;
  if (m->has_sym_cache && (int64_t)m->sym_cache_free.size() == n_free &&
      std::equal(m->sym_cache_free.begin(), m->sym_cache_free.end(), free_dofs)) {
    // the shared analysis of this mesh and free set
    m->symp = std::move(m->sym_cache);
    m->sym_cache.reset();
    m->has_sym_cache = false;
    std::vector<int32_t>().swap(m->sym_cache_free);
  } else {
    SymbolicOptions opt = SymbolicOptions::from_env();
    auto S = std::make_shared<Symbolic>();
    std::string e =
        analyze(m->ndof, m->pat->colptr.data(), m->pat->rowval.data(), n_free, free_dofs, m->h_xyz.data(), opt, *S);
    if (!e.empty()) { set_error(e); return JFG_BAD_INPUT; }
    sort_level_lists(*S);   // the analysis is read-only from here on
    m->symp = std::move(S);
  }
  JFG_TRY(numeric_create(m));
  m->sym_ready = true;
  return JFG_OK;
}

jfg_status jfg_model_share_structure(jfg_model* dst, const jfg_model* src) {
  JFG_TRY(check_model(dst));
  if (!src) { set_error("null source model"); return JFG_BAD_INPUT; }
  if (!src->pattern_built) { set_error("source model has no pattern: call jfg_assemble on it first"); return JFG_NOT_READY; }
  if (dst->pattern_built) { set_error("destination model already has a pattern"); return JFG_BAD_INPUT; }
  if (dst->n_q8 > 0 || src->n_q8 > 0) {
    set_error("CQUAD8 patterns depend on the element values and are not shared");
    return JFG_UNSUPPORTED;
  }
  if (dst->n_nodes != src->n_nodes || dst->h_q4n != src->h_q4n || dst->h_t10n != src->h_t10n ||
      dst->h_t3n != src->h_t3n) {
    set_error("models do not share a mesh (grid count or element connectivity differ)");
    return JFG_BAD_INPUT;
  }
  jfg_ctx* c = dst->ctx;
  const int64_t ndof = dst->ndof, nnz = src->nnz;
  dst->nnz = nnz;
  dst->n_trip = src->n_trip;
  dst->pat = src->pat;   // read-only once built: shared, not copied
  JFG_TRY(dev_alloc(c, (void**)&dst->d_colptr, sizeof(int64_t) * (ndof + 1)));
  JFG_TRY(dev_alloc(c, (void**)&dst->d_rowval, sizeof(int32_t) * nnz));
  JFG_TRY(dev_alloc(c, (void**)&dst->d_nzptr, sizeof(int32_t) * (nnz + 1)));
  JFG_TRY(dev_alloc(c, (void**)&dst->d_trip, sizeof(int32_t) * dst->n_trip));
  JFG_TRY(dev_alloc(c, (void**)&dst->d_tpos, sizeof(int64_t) * nnz));
  JFG_TRY(dev_alloc(c, (void**)&dst->d_nzval, sizeof(double) * nnz));
  JFG_TRY(up(c, dst->pat->diag_pos, &dst->d_diag_pos));
  JFG_CUDA(cudaStreamSynchronize(cudaStreamLegacy));   // the pageable upload above
  cudaStream_t st = dst->stream;
  JFG_CUDA(cudaMemcpyAsync(dst->d_colptr, src->d_colptr, sizeof(int64_t) * (ndof + 1), cudaMemcpyDeviceToDevice, st));
  JFG_CUDA(cudaMemcpyAsync(dst->d_rowval, src->d_rowval, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice, st));
  JFG_CUDA(cudaMemcpyAsync(dst->d_nzptr, src->d_nzptr, sizeof(int32_t) * (nnz + 1), cudaMemcpyDeviceToDevice, st));
  JFG_CUDA(cudaMemcpyAsync(dst->d_trip, src->d_trip, sizeof(int32_t) * dst->n_trip, cudaMemcpyDeviceToDevice, st));
  JFG_CUDA(cudaMemcpyAsync(dst->d_tpos, src->d_tpos, sizeof(int64_t) * nnz, cudaMemcpyDeviceToDevice, st));
  JFG_CUDA(cudaStreamSynchronize(st));
  dst->pattern_built = true;
  if (src->sym_ready) {
    dst->sym_cache = src->symp;
    dst->sym_cache_free.clear();
    dst->sym_cache_free.reserve(src->sym().n);
    for (int64_t d = 0; d < ndof; ++d)
      if (src->sym().gdof_to_perm[d] >= 0) dst->sym_cache_free.push_back((int32_t)d);
    dst->has_sym_cache = true;
  }
  return JFG_OK;
}

jfg_status jfg_get_symbolic_info(jfg_model* m, jfg_symbolic_info* info) {
  JFG_TRY(check_model(m));
  if (!m->sym_ready) { set_error("no symbolic analysis"); return JFG_NOT_READY; }
  info->n_supernodes = m->sym().ns;
  info->n_levels = m->sym().n_levels;
  info->nnz_L = m->sym().nnz_L;
  info->flops = m->sym().flops;
  info->factor_bytes = 8 * m->sym().nnz_L;
  info->max_front = m->sym().max_front;
  return JFG_OK;
}

jfg_status jfg_get_perm(jfg_model* m, int32_t* perm) {
  JFG_TRY(check_model(m));
  if (!m->sym_ready) { set_error("no symbolic analysis"); return JFG_NOT_READY; }
  std::memcpy(perm, m->sym().perm_free.data(), sizeof(int32_t) * m->sym().n);
  return JFG_OK;
}

jfg_status jfg_factor(jfg_model* m, int32_t precision) {
  JFG_TRY(check_model(m));
  if (m->async_factor >= 0) JFG_TRY(jfg_wait(m));
  m->async_prec = -1;
  return numeric_factor(m, precision);
}

namespace {
// the model's stream waits for the work the caller has already put on `user`
jfg_status async_begin(jfg_model* m, cudaStream_t user) {
  if (!m->aev_in) {
    JFG_CUDA(cudaEventCreateWithFlags(&m->aev_in, cudaEventDisableTiming));
    JFG_CUDA(cudaEventCreateWithFlags(&m->aev_out, cudaEventDisableTiming));
  }
  JFG_CUDA(cudaEventRecord(m->aev_in, user));
  JFG_CUDA(cudaStreamWaitEvent(m->stream, m->aev_in, 0));
  return JFG_OK;
}
// `user` waits for the work just put on the model's stream
jfg_status async_end(jfg_model* m, cudaStream_t user) {
  JFG_CUDA(cudaEventRecord(m->aev_out, m->stream));
  JFG_CUDA(cudaStreamWaitEvent(user, m->aev_out, 0));
  return JFG_OK;
}
}  // namespace

jfg_status jfg_factor_async(jfg_model* m, int32_t precision, void* stream) {
  JFG_TRY(check_model(m));
  if (precision != JFG_PREC_FP64 && precision != JFG_PREC_MIXED) { set_error("unknown precision"); return JFG_BAD_INPUT; }
  if (m->async_factor >= 0) JFG_TRY(jfg_wait(m));     // one unchecked factorisation at a time
  cudaStream_t user = static_cast<cudaStream_t>(stream);
  JFG_TRY(async_begin(m, user));
  JFG_TRY(numeric_factor_enqueue(m, precision));
  m->async_factor = precision;
  m->async_prec = precision;
  return async_end(m, user);
}

jfg_status jfg_apply_factor_async(jfg_model* m, int32_t nrhs, const double* F_dev, double* U_dev, void* stream) {
  JFG_TRY(check_model(m));
  if (!F_dev || !U_dev) { set_error("null F/U"); return JFG_BAD_INPUT; }
  const int prec = m->async_prec >= 0 ? m->async_prec : numeric_current_precision(m);
  if (prec < 0) { set_error("apply before factorisation"); return JFG_NOT_READY; }
  cudaStream_t user = static_cast<cudaStream_t>(stream);
  JFG_TRY(async_begin(m, user));
  JFG_TRY(numeric_apply(m, nrhs, F_dev, U_dev, prec));
  return async_end(m, user);
}

jfg_status jfg_wait(jfg_model* m) {
  JFG_TRY(check_model(m));
  if (m->aev_out) JFG_CUDA(cudaEventSynchronize(m->aev_out));
  JFG_CUDA(cudaStreamSynchronize(m->stream));
  if (m->async_factor >= 0) {
    const int p = m->async_factor;
    m->async_factor = -1;
    JFG_TRY(numeric_factor_finish(m, p));
  }
  return JFG_OK;
}

jfg_status jfg_get_factor_diag(jfg_model* m, double* Ldiag) {
  JFG_TRY(check_model(m));
  if (m->async_factor >= 0) JFG_TRY(jfg_wait(m));
  return numeric_factor_diag(m, Ldiag);
}

jfg_status jfg_solve(jfg_model* m, int32_t nrhs, const double* F, double* U, double tol, int32_t max_ir,
                     jfg_solve_report* report) {
  JFG_TRY(check_model(m));
  if (m->async_factor >= 0) JFG_TRY(jfg_wait(m));
  if (!F || !U) { set_error("null F/U"); return JFG_BAD_INPUT; }
  return numeric_solve(m, nrhs, F, U, tol, max_ir, report, false);
}

jfg_status jfg_solve_device(jfg_model* m, int32_t nrhs, const double* F, double* U, double tol, int32_t max_ir,
                            jfg_solve_report* report) {
  JFG_TRY(check_model(m));
  if (m->async_factor >= 0) JFG_TRY(jfg_wait(m));
  if (!F || !U) { set_error("null F/U"); return JFG_BAD_INPUT; }
  return numeric_solve(m, nrhs, F, U, tol, max_ir, report, true);
}

jfg_status jfg_residual(jfg_model* m, int32_t nrhs, const double* U, const double* F, double* R) {
  JFG_TRY(check_model(m));
  if (!m->values_ready) { set_error("values not assembled"); return JFG_NOT_READY; }
  if (nrhs <= 0) { set_error("nrhs must be positive"); return JFG_BAD_INPUT; }
  int64_t len = m->ndof * (int64_t)nrhs;
  double *dU = nullptr, *dR = nullptr;
  JFG_TRY(dev_alloc(m->ctx, (void**)&dU, 8 * len));
  jfg_status st = dev_alloc(m->ctx, (void**)&dR, 8 * len);
  if (st) { dev_free(m->ctx, dU, 8 * len); return st; }
  cudaStream_t s = m->stream;
  cudaMemcpyAsync(dU, U, 8 * len, cudaMemcpyHostToDevice, s);
  spmv_csc_sym(m, nrhs, dU, m->ndof, dR, m->ndof, s);
  cudaError_t e = cudaMemcpyAsync(R, dR, 8 * len, cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  dev_free(m->ctx, dU, 8 * len);
  dev_free(m->ctx, dR, 8 * len);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return JFG_CUDA_ERROR; }
  if (F)
    for (int64_t i = 0; i < len; ++i) R[i] -= F[i];
  return JFG_OK;
}

jfg_status jfg_recover_stresses(jfg_model* m, int32_t kind, int32_t nrhs, const double* U, double* out) {
  JFG_TRY(check_model(m));
  if (nrhs <= 0 || !U || !out) { set_error("nrhs must be positive and U, out non-null"); return JFG_BAD_INPUT; }
  if (kind != 0 && kind != 2) {
    set_error("stress recovery is available for CQUAD4 (kind 0) and CTETRA10 (kind 2)");
    return JFG_UNSUPPORTED;
  }
  const int64_t len = m->ndof * (int64_t)nrhs;
  const int64_t olen = kind == 0 ? 31 * m->n_q4 * (int64_t)nrhs : 13 * m->n_t10 * (int64_t)nrhs;
  if (olen == 0) return JFG_OK;
  double *dU = nullptr, *dO = nullptr;
  JFG_TRY(dev_alloc(m->ctx, (void**)&dU, 8 * len));
  jfg_status st = dev_alloc(m->ctx, (void**)&dO, 8 * olen);
  if (st) { dev_free(m->ctx, dU, 8 * len); return st; }
  cudaStream_t s = m->stream;
  cudaError_t e = cudaMemcpyAsync(dU, U, 8 * len, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    st = kind == 0 ? recover_q4_stresses(m, nrhs, dU, dO, s) : recover_t10_stresses(m, nrhs, dU, dO, s);
  if (e == cudaSuccess && st == JFG_OK) e = cudaMemcpyAsync(out, dO, 8 * olen, cudaMemcpyDeviceToHost, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  dev_free(m->ctx, dU, 8 * len);
  dev_free(m->ctx, dO, 8 * olen);
  if (st != JFG_OK) return st;
  if (e != cudaSuccess || e2 != cudaSuccess) {
    set_error(cudaGetErrorString(e != cudaSuccess ? e : e2));
    return JFG_CUDA_ERROR;
  }
  return read_elem_error(m);
}

jfg_status jfg_update_q4_sections(jfg_model* m, int64_t n, const int32_t* elems, const double* sect) {
  JFG_TRY(check_model(m));
  for (int64_t k = 0; k < n; ++k) {
    int64_t e = elems[k];
    if (e < 0 || e >= m->n_q4) { set_error("element index out of range", k); return JFG_BAD_INPUT; }
    std::memcpy(m->h_q4s.data() + JFG_Q4_SECT_STRIDE * e, sect + JFG_Q4_SECT_STRIDE * k, 8 * JFG_Q4_SECT_STRIDE);
  }
  // one upload of the whole section table keeps this call simple and ordered
  JFG_CUDA(cudaMemcpyAsync(m->d_q4s, m->h_q4s.data(), 8 * m->h_q4s.size(), cudaMemcpyHostToDevice, m->stream));
  JFG_CUDA(cudaStreamSynchronize(m->stream));
  m->values_ready = false;
  return JFG_OK;
}

jfg_status jfg_get_timings(jfg_model* m, double* s4) {
  JFG_TRY(check_model(m));
  s4[0] = m->t_elements; s4[1] = m->t_assembly; s4[2] = m->t_factor; s4[3] = m->t_solve;
  return JFG_OK;
}

int64_t jfg_launch_count(void) { return launch_count(); }

jfg_status jfg_set_profiling(int32_t on) {
  set_profiling(on);
  return JFG_OK;
}

jfg_status jfg_get_kernel_stats(int32_t which, double* out3) {
  if (which < 0 || which >= KS_COUNT || !out3) { set_error("bad kernel-stat index"); return JFG_BAD_INPUT; }
  out3[0] = (double)kernel_stats().launches[which];
  out3[1] = kernel_stats().ms[which];
  out3[2] = kernel_stats().units[which];
  return JFG_OK;
}

jfg_status jfg_reset_kernel_stats(void) {
  kernel_stats() = KernelStats();
  return JFG_OK;
}

jfg_status jfg_symbolic_dry_run(int64_t ndof, const int64_t* colptr, const int32_t* rowval, int64_t n_free,
                                const int32_t* free_dofs, const double* xyz, jfg_symbolic_info* info, int32_t* perm) {
  Symbolic S;
  SymbolicOptions opt = SymbolicOptions::from_env();
  std::string e = analyze(ndof, colptr, rowval, n_free, free_dofs, xyz, opt, S);
  if (!e.empty()) { set_error(e); return JFG_BAD_INPUT; }
  if (info) {
    info->n_supernodes = S.ns; info->n_levels = S.n_levels; info->nnz_L = S.nnz_L; info->flops = S.flops;
    info->factor_bytes = 8 * S.nnz_L; info->max_front = S.max_front;
  }
  if (perm) std::memcpy(perm, S.perm_free.data(), sizeof(int32_t) * S.n);
  return JFG_OK;
}

}  // extern "C"
