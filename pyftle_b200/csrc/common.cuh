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

// Largest eigenvalue of a symmetric 3x3 matrix by cyclic Jacobi rotations (FP64);
// the mixed-precision window epilogue and the 3D surrogate's FTLE use it.
static __device__ __noinline__ double lmax3_sym(double a00, double a01, double a02, double a11,
                                                double a12, double a22) {
  double a[3][3] = {{a00, a01, a02}, {a01, a11, a12}, {a02, a12, a22}};
  for (int sweep = 0; sweep < 32; ++sweep) {
    const double off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
    const double diag = fabs(a[0][0]) + fabs(a[1][1]) + fabs(a[2][2]);
    if (off == 0.0 || off <= 1e-300 || off < 1e-18 * diag) break;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
#pragma unroll
      for (int q = p + 1; q < 3; ++q) {
        const double apq = a[p][q];
        if (apq == 0.0) continue;
        const double app = a[p][p], aqq = a[q][q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0);
        const double s = t * c;
        a[p][p] = app - t * apq;
        a[q][q] = aqq + t * apq;
        a[p][q] = 0.0;
        a[q][p] = 0.0;
        const int r = 3 - p - q;
        const double arp = a[r][p], arq = a[r][q];
        const double nrp = c * arp - s * arq;
        const double nrq = s * arp + c * arq;
        a[r][p] = nrp;
        a[p][r] = nrp;
        a[r][q] = nrq;
        a[q][r] = nrq;
      }
    }
  }
  double mx = a[0][0];
  if (a[1][1] > mx) mx = a[1][1];
  if (a[2][2] > mx) mx = a[2][2];
  return mx;
}

}  // namespace ftle
