// no_alloc.cu -- the chunked mixed-precision window without caller workspace.
//
// Some callers cannot hand the engine a device workspace: applications whose
// device memory is owned by their own fixed-size pool and may not be
// enlarged behind their back, plugins loaded into a host program that forbids
// them from calling cudaMalloc, or runtimes where a device allocation at run
// time is too slow or may fail at a point they cannot recover from.  For them
// this file keeps the scratch in a file-scope device array of
// kStaticWorkspaceBytes (32 MiB).  Every GPU that loads the library's module
// holds it until the process exits (or the context is destroyed).  Nothing
// here calls cudaMalloc, cudaFree or any allocating routine.
//
// When the 32 MiB is reserved: with CUDA's default lazy module loading
// (CUDA_MODULE_LOADING=LAZY) the module that holds the array is loaded by the
// first call on a device, inside the cudaGetSymbolAddress of the set-up below,
// so that first call is where the reservation happens and where it can fail
// (out of memory when the caller's pool already owns the device).  With
// CUDA_MODULE_LOADING=EAGER it happens when the context is created.  The
// set-up runs on the first call per device and context, so that first call
// should come before any stream capture.
#include <cudaTypedefs.h>

#include <mutex>

#include "common.cuh"

namespace ftle {

constexpr int64_t kStaticWorkspaceBytes = 32ll << 20;  // 32 MiB

static __device__ __align__(256) unsigned char g_static_workspace[kStaticWorkspaceBytes];

constexpr int kMaxDevices = 64;

// Cached device address of g_static_workspace per device, valid for one context:
// after cudaDeviceReset (or a release and re-creation of the primary context) the
// module is loaded again, possibly at another address, so an entry is used only
// while the context it was looked up in (its unique id) is still the current one.
struct WorkspaceEntry {
  unsigned long long ctx_id;
  void *addr;
};
static WorkspaceEntry g_workspace[kMaxDevices] = {};
static std::mutex g_workspace_mutex;

static PFN_cuCtxGetCurrent_v4000 g_ctx_get_current = nullptr;
static PFN_cuCtxGetId_v12000 g_ctx_get_id = nullptr;

// Unique id of the calling thread's current context (0 when none is current or the
// driver cannot say).  The driver entry points come through the runtime, so the
// library needs no link against libcuda.
static unsigned long long current_ctx_id() {
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f);
  });
  if (!g_ctx_get_current || !g_ctx_get_id) return 0;
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  unsigned long long id = 0;
  if (g_ctx_get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of g_static_workspace on the current device.  In host code the
// array's name only stands in for the symbol, so the address is looked up with the
// device current and cached for that device and context.
static int static_workspace(void **out, int *dev_out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("cudaGetDevice: %s", cudaGetErrorString(e));
    return FTLE_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) return fail_invalid("device ordinal %d not supported", dev);
  *dev_out = dev;
  std::lock_guard<std::mutex> lock(g_workspace_mutex);
  const unsigned long long id = current_ctx_id();
  WorkspaceEntry &ent = g_workspace[dev];
  if (id != 0 && ent.addr && ent.ctx_id == id) {
    *out = ent.addr;
    return FTLE_OK;
  }
  void *p = nullptr;
  e = cudaGetSymbolAddress(&p, g_static_workspace);
  if (e != cudaSuccess || !p) {
    ent.addr = nullptr;
    ent.ctx_id = 0;
    set_error("cudaGetSymbolAddress(static workspace): %s", cudaGetErrorString(e));
    return FTLE_ERR_CUDA;
  }
  // the lookup made the runtime's context current if none was: key on it now
  ent.ctx_id = id != 0 ? id : current_ctx_id();
  ent.addr = ent.ctx_id != 0 ? p : nullptr;  // unknown context: look up again next time
  *out = p;
  return FTLE_OK;
}

static void forget_workspace(int dev) {
  std::lock_guard<std::mutex> lock(g_workspace_mutex);
  g_workspace[dev].addr = nullptr;
  g_workspace[dev].ctx_id = 0;
}

}  // namespace ftle

using namespace ftle;

extern "C" int ftle_window_run_mixed_chunked_static(const ftle_window *w, int32_t chunk_steps,
                                                    int32_t sort_every, void *stream) {
  const int64_t need = ftle_window_workspace_bytes(w);
  if (need < 0) return fail_invalid("invalid window descriptor");
  if (need > kStaticWorkspaceBytes)
    return fail_invalid(
        "window needs %lld bytes of workspace, the built-in workspace holds %lld bytes "
        "(use ftle_window_run_mixed_chunked with a caller workspace)",
        (long long)need, (long long)kStaticWorkspaceBytes);
  void *ws = nullptr;
  int dev = 0;
  int rc = static_workspace(&ws, &dev);
  if (rc) return rc;
  rc = ftle_window_run_mixed_chunked(w, ws, kStaticWorkspaceBytes, chunk_steps, sort_every,
                                     stream);
  if (rc == FTLE_ERR_CUDA) forget_workspace(dev);  // look the address up afresh next call
  return rc;
}
