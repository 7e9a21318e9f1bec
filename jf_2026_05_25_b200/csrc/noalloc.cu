// noalloc.cu -- jfg_assemble_values_noalloc: re-assembly of K's values into
// a caller-owned device buffer with no device allocation at all.
//
// Who needs it: callers that cannot call cudaMalloc between solves -- a host
// application whose device memory is owned by another framework's caching
// pool (the pool holds the free memory, so a cudaMalloc from this library can
// fail or force the pool to release and re-grow), and design loops that
// re-assemble after every section change while other streams are busy (a
// cudaMalloc/cudaFree may synchronise the whole device and stall them).  The
// regular jfg_assemble keeps its element matrices in a model-sized device
// buffer allocated at upload; this variant instead keeps them in one fixed,
// file-scope device array, so the call itself allocates nothing.
//
// Limits and sharing:
//   * the scratch array holds at most kScratchBytes (16 MiB); a model whose
//     element matrices and CQUAD4 prep records need more (roughly 2,600
//     CQUAD4 or 2,300 CTETRA10 elements) is rejected with JFG_BAD_INPUT
//     before any launch;
//   * every GPU that loads the library holds the 16 MiB array until the
//     process exits;
//   * every call on a device shares the same array and it keeps the previous
//     call's contents.  The element-error record at its head must start at
//     zero and is cleared by each call (cudaMemsetAsync); the element
//     matrices and prep records are overwritten in full by each call.  Calls whose work
//     overlaps on the same GPU (two host threads, or two contexts on
//     different streams) race on the array: serialise them;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current; with lazy module
//     loading this is also when the 16 MiB are taken); make that first call
//     before any stream capture is started on that device.  The address is
//     looked up again if the device's context has been re-created since.
#include <mutex>
#include <string>

#include "jfg_internal.h"

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;
constexpr size_t kHeaderBytes = 256;  // DevError record, then the element matrices
constexpr int kMaxDevices = 64;

// In host code this name is only a host-side stand-in for the device array;
// kernels get the device address from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// The array's address is looked up once per device and context.  A context
// that is destroyed and created again (cudaDeviceReset, or the primary
// context released and retained) reloads the module, which can move the
// array, so each cached address is tagged with the id of the context it was
// taken in (cuCtxGetId: unique for the life of the process) and looked up
// again when the current context's id differs.
using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn = int (*)(void*, unsigned long long*);

struct ScratchAddr {
  unsigned long long ctx_id = 0;
  void* ptr = nullptr;
};

std::mutex g_addr_mu;
ScratchAddr g_addr[kMaxDevices];

// Id of the calling thread's current context, 0 when it cannot be read (the
// address is then looked up again on every call, which is still allocation-free).
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, nullptr) == cudaSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, nullptr) == cudaSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
  });
  if (!get_current || !get_id) return 0;
  void* ctx = nullptr;
  if (get_current(&ctx) != 0 || !ctx) return 0;
  unsigned long long id = 0;
  if (get_id(ctx, &id) != 0) return 0;
  return id;
}

jfg_status scratch_address(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) {
    jfg::set_error("device ordinal out of range for the no-allocation scratch");
    return JFG_BAD_INPUT;
  }
  const unsigned long long ctx_id = current_context_id();
  std::lock_guard<std::mutex> lk(g_addr_mu);
  ScratchAddr& a = g_addr[dev];
  if (!a.ptr || ctx_id == 0 || a.ctx_id != ctx_id) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      jfg::set_error(std::string("cudaGetSymbolAddress of the no-allocation scratch failed: ") +
                     cudaGetErrorString(e));
      return JFG_CUDA_ERROR;
    }
    a.ptr = p;
    a.ctx_id = ctx_id;
  }
  *out = static_cast<unsigned char*>(a.ptr);
  return JFG_OK;
}

jfg_status element_error(const jfg::DevError& h) {
  if (h.code == 0) return JFG_OK;
  bool unsupported = h.code == jfg::EE_NOT_FLAT || h.code == jfg::EE_FLAGS;
  jfg::set_error("element kernel error " + std::to_string(h.code) + " (element " + std::to_string(h.index) + ")",
                 h.index);
  return unsupported ? JFG_UNSUPPORTED : JFG_BAD_INPUT;
}

// Runs on the model's device; restores the caller's current device on return.
struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    ok = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" {

jfg_status jfg_assemble_values_noalloc(jfg_model* m, double* nzval_dev) {
  using namespace jfg;
  if (!m || !m->ctx) { set_error("null model"); return JFG_BAD_INPUT; }
  if (!nzval_dev) { set_error("null output buffer"); return JFG_BAD_INPUT; }
  if (!m->pattern_built) {
    set_error("pattern not built: call jfg_assemble once before the no-allocation variant");
    return JFG_NOT_READY;
  }
  const size_t ev_bytes = (sizeof(double) * (size_t)m->n_ev + 255) / 256 * 256;
  const size_t need = kHeaderBytes + ev_bytes + sizeof(double) * Q4_PREP_STRIDE * (size_t)m->n_q4;
  if (need > kScratchBytes) {
    set_error("model needs " + std::to_string(need) + " bytes of element scratch; the no-allocation path holds " +
              std::to_string(kScratchBytes) + " bytes (use jfg_assemble)", (int64_t)need);
    return JFG_BAD_INPUT;
  }
  DeviceGuard g(m->ctx->device);
  if (!g.ok) { set_error("cudaSetDevice failed for the model's device"); return JFG_CUDA_ERROR; }
  unsigned char* base = nullptr;
  JFG_TRY(scratch_address(m->ctx->device, &base));
  DevError* err = reinterpret_cast<DevError*>(base);
  double* ev = reinterpret_cast<double*>(base + kHeaderBytes);
  double* q4prep = reinterpret_cast<double*>(base + kHeaderBytes + ev_bytes);
  cudaStream_t st = m->stream;
  JFG_CUDA(cudaMemsetAsync(err, 0, sizeof(DevError), st));
  JFG_TRY(launch_elements_into(m, st, ev, q4prep, err));
  JFG_TRY(launch_gather_into(m, st, ev, nzval_dev));
  DevError h{};
  JFG_CUDA(cudaMemcpyAsync(&h, err, sizeof(DevError), cudaMemcpyDeviceToHost, st));
  JFG_CUDA(cudaStreamSynchronize(st));
  return element_error(h);
}

}  // extern "C"
