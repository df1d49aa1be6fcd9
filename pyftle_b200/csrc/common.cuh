// common.cuh -- shared host/device helpers of the FTLE engine (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pyftle_b200.h"

namespace ftle {

// ---------------------------------------------------------------------------
// host-side error plumbing (no exceptions cross the C ABI)
// ---------------------------------------------------------------------------
void set_error(const char *fmt, ...);
int fail_invalid(const char *fmt, ...);
int check_launch(const char *what);

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr int kNumSMs = 148;  // B200

// Grid constants passed by value to kernels.
struct GridK {
  int n[3];
  double origin[3];
  double spacing[3];
  int periodic;
  long long nodes;
};

int grid_from_abi(const ftle_grid *g, GridK *out);

// Window constants passed by value to the window kernels.
struct WinK {
  GridK g;
  const void *snaps;  // packed records (layout depends on the storage type)
  int num_snaps, periodic_time, first_snapshot, num_steps;
  double snap_t0, snap_dt, t0, h, map_period;
  double *positions;
  long long N;
  double *ftle;
  int keep_positions;  // FTLE_KEEP_POSITIONS: do not write final positions
};

// Validates an ftle_window and converts it to kernel constants.
int window_to_kernel(const ftle_window *w, WinK *k);

int pack_snapshots_f64(int32_t dim, int64_t nodes, int32_t num_snapshots, int32_t periodic_time,
                       const double *src, double *dst, void *stream);
int pack_snapshots_16(int32_t dim, int64_t nodes, int32_t num_snapshots, int32_t periodic_time,
                      const double *src, int32_t storage, void *dst, void *stream);

// Blocks for a grid-stride launch over n work items.
inline unsigned grid_blocks(int64_t n, int threads, int per_sm = 8) {
  int64_t b = (n + threads - 1) / threads;
  int64_t cap = (int64_t)kNumSMs * per_sm * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------

// Wrap a cell index into [0, n) for periodic grids.
__device__ __forceinline__ int wrap_index(int q, int n) {
  int r = q % n;
  return r < 0 ? r + n : r;
}

// Node id of (i, j) / (i, j, k) in the reference's meshgrid-"xy" flattening.
__device__ __forceinline__ long long node2(const GridK &g, int i, int j) {
  return (long long)j * g.n[0] + i;
}
__device__ __forceinline__ long long node3(const GridK &g, int i, int j, int k) {
  return ((long long)j * g.n[0] + i) * g.n[2] + k;
}

}  // namespace ftle
