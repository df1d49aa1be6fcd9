// api.cu -- C ABI plumbing: error reporting, argument validation, packing dispatch.
#include <stdarg.h>
#include <stdio.h>

#include "common.cuh"

namespace ftle {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int fail_invalid(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return FTLE_ERR_INVALID;
}

int check_launch(const char *what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return FTLE_ERR_CUDA;
  }
  return FTLE_OK;
}

int grid_from_abi(const ftle_grid *g, GridK *out) {
  if (!g) return fail_invalid("grid descriptor is NULL");
  if (g->dim != 2 && g->dim != 3) return fail_invalid("grid dim must be 2 or 3, got %d", g->dim);
  long long nodes = 1;
  for (int a = 0; a < 3; ++a) {
    if (a < g->dim) {
      if (g->n[a] < 2) return fail_invalid("grid axis %d needs at least 2 nodes", a);
      if (!(g->spacing[a] > 0.0) && !(g->spacing[a] < 0.0))
        return fail_invalid("grid spacing on axis %d must be non-zero", a);
      out->n[a] = g->n[a];
      out->origin[a] = g->origin[a];
      out->spacing[a] = g->spacing[a];
      nodes *= g->n[a];
    } else {
      out->n[a] = 1;
      out->origin[a] = 0.0;
      out->spacing[a] = 1.0;
    }
  }
  if (nodes > (1LL << 40)) return fail_invalid("grid too large");
  out->periodic = g->periodic ? 1 : 0;
  out->nodes = nodes;
  return FTLE_OK;
}

int window_to_kernel(const ftle_window *w, WinK *k) {
  if (!w) return fail_invalid("window descriptor is NULL");
  int rc = grid_from_abi(&w->grid, &k->g);
  if (rc) return rc;
  if (w->num_groups < 0) return fail_invalid("num_groups must be >= 0");
  if (!w->snapshots) return fail_invalid("snapshots are required");
  if (!w->positions && w->num_groups > 0) return fail_invalid("positions are required");
  if (w->num_steps < 0) return fail_invalid("num_steps must be >= 0");
  if (w->integrator < FTLE_EULER || w->integrator > FTLE_RK4)
    return fail_invalid("unknown integrator %d", w->integrator);
  if (w->time_mode != FTLE_HOLD && w->time_mode != FTLE_BLEND)
    return fail_invalid("unknown time mode %d", w->time_mode);
  if (w->num_snapshots < 1) return fail_invalid("need at least one snapshot");
  if (w->time_mode == FTLE_HOLD) {
    if (w->first_snapshot < 0 || w->first_snapshot >= w->num_snapshots)
      return fail_invalid("first_snapshot out of range");
    if (!w->periodic_time && (int64_t)w->first_snapshot + w->num_steps > w->num_snapshots)
      return fail_invalid("HOLD window needs first_snapshot + num_steps <= num_snapshots");
  } else {
    if (w->num_snapshots < 2) return fail_invalid("BLEND needs at least two snapshots");
    if (!(w->snapshot_dt > 0.0) && !(w->snapshot_dt < 0.0))
      return fail_invalid("snapshot_dt must be non-zero");
  }
  if (w->ftle && !(w->map_period > 0.0) && !(w->map_period < 0.0))
    return fail_invalid("map_period must be non-zero");
  if (reinterpret_cast<uintptr_t>(w->snapshots) % 16 != 0)
    return fail_invalid("packed snapshots must be 16-byte aligned");
  k->snaps = w->snapshots;
  k->num_snaps = w->num_snapshots;
  k->periodic_time = w->periodic_time;
  k->first_snapshot = w->first_snapshot;
  k->num_steps = w->num_steps;
  k->snap_t0 = w->snapshot_t0;
  k->snap_dt = w->snapshot_dt;
  k->t0 = w->t0;
  k->h = w->h;
  k->map_period = w->map_period;
  k->positions = w->positions;
  k->N = w->num_groups;
  k->ftle = w->ftle;
  k->keep_positions = (w->flags & FTLE_KEEP_POSITIONS) ? 1 : 0;
  return FTLE_OK;
}

}  // namespace ftle

using namespace ftle;

extern "C" {

int ftle_version(void) { return 10000; }

const char *ftle_last_error(void) { return g_err; }

int ftle_stream_synchronize(void *stream) {
  const cudaError_t e = cudaStreamSynchronize(as_stream(stream));
  if (e != cudaSuccess) {
    set_error("cudaStreamSynchronize: %s", cudaGetErrorString(e));
    return FTLE_ERR_CUDA;
  }
  return FTLE_OK;
}

int64_t ftle_packed_snapshot_bytes(int32_t dim, int64_t nodes, int32_t num_snapshots,
                                   int32_t storage) {
  if ((dim != 2 && dim != 3) || nodes < 0 || num_snapshots < 0) return -1;
  if (storage == FTLE_F64) return (int64_t)(2 * dim * 8) * nodes * num_snapshots;
  if (storage == FTLE_F16 || storage == FTLE_BF16 || storage == FTLE_FX15 || storage == FTLE_FX16) {
    // 256-byte decode header, then 4 or 8 16-bit values per record (3D pads each half to 4)
    const int64_t rec = dim == 2 ? 8 : 16;
    return 256 + rec * nodes * num_snapshots;
  }
  return -1;
}

int ftle_pack_snapshots(int32_t dim, int64_t nodes, int32_t num_snapshots, int32_t periodic_time,
                        const double *src, int32_t storage, void *dst, void *stream) {
  if (dim != 2 && dim != 3) return fail_invalid("dim must be 2 or 3");
  if (nodes < 0 || num_snapshots < 0) return fail_invalid("sizes must be >= 0");
  if (nodes == 0 || num_snapshots == 0) return FTLE_OK;
  if (!src || !dst) return fail_invalid("null pointer");
  if (reinterpret_cast<uintptr_t>(dst) % 16 != 0) return fail_invalid("dst must be 16-byte aligned");
  if (storage == FTLE_F64)
    return pack_snapshots_f64(dim, nodes, num_snapshots, periodic_time, src,
                              static_cast<double *>(dst), stream);
  if (storage == FTLE_F16 || storage == FTLE_BF16 || storage == FTLE_FX15 || storage == FTLE_FX16)
    return pack_snapshots_16(dim, nodes, num_snapshots, periodic_time, src, storage, dst, stream);
  return fail_invalid("unknown storage %d", storage);
}

}  // extern "C"
