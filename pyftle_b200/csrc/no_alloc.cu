// no_alloc.cu -- the chunked mixed-precision window without caller workspace.
//
// Some callers cannot hand the engine a device workspace: applications whose
// device memory is owned by their own fixed-size pool and may not be
// enlarged behind their back, plugins loaded into a host program that forbids
// them from calling cudaMalloc, or runtimes where a device allocation at run
// time is too slow or may fail at a point they cannot recover from.  For them
// this file keeps the scratch in a file-scope device array that the driver
// reserves when the library's module is loaded; every GPU that loads the
// library holds kStaticWorkspaceBytes (32 MiB) of device memory until the
// process exits.  Nothing here calls cudaMalloc, cudaFree or any allocating
// routine.
#include <mutex>

#include "common.cuh"

namespace ftle {

constexpr int64_t kStaticWorkspaceBytes = 32ll << 20;  // 32 MiB

static __device__ __align__(256) unsigned char g_static_workspace[kStaticWorkspaceBytes];

constexpr int kMaxDevices = 64;
static void *g_workspace_addr[kMaxDevices] = {};
static std::mutex g_workspace_mutex;

// Device address of g_static_workspace on the current device.  In host code the
// array's name only stands in for the symbol, so the address is looked up once
// per device (with that device current) and cached.
static int static_workspace(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("cudaGetDevice: %s", cudaGetErrorString(e));
    return FTLE_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) return fail_invalid("device ordinal %d not supported", dev);
  std::lock_guard<std::mutex> lock(g_workspace_mutex);
  if (!g_workspace_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_workspace);
    if (e != cudaSuccess || !p) {
      set_error("cudaGetSymbolAddress(static workspace): %s", cudaGetErrorString(e));
      return FTLE_ERR_CUDA;
    }
    g_workspace_addr[dev] = p;
  }
  *out = g_workspace_addr[dev];
  return FTLE_OK;
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
  const int rc = static_workspace(&ws);
  if (rc) return rc;
  return ftle_window_run_mixed_chunked(w, ws, kStaticWorkspaceBytes, chunk_steps, sort_every,
                                       stream);
}
