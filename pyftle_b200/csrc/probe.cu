// probe.cu -- measured gather ceilings for the roofline of the window kernels.
//
// The window kernels gather 16-byte snapshot records (8 cell corners per
// interpolation) from a working set that lives in L1/L2: one time interval of
// the 128^3 FX15 series is 33.5 MB, and cell-sorted groups reuse each other's
// corners.  Their bound is therefore the on-chip gather rate, not HBM.  This
// kernel measures that rate on the same hardware in the same process: every
// thread issues independent 16-byte read-only loads (ld.global.nc.v4) at
// pseudo-random records of a region of `region_bytes`:
//   * a region of a few KB per block is L1-resident (the L1 gather ceiling);
//   * one region of ~32 MB shared by all blocks is L2-resident (the L2 ceiling).
// `lane_span_bytes` sets how far apart the lanes of one warp load: the whole
// region (every lane its own random line: the worst case of scattered
// particles) or a few records (a coherent, cell-sorted warp).
#include "common.cuh"

namespace ftle {

constexpr int kProbeThreads = 128;
constexpr int kProbeUnroll = 8;

__global__ void __launch_bounds__(kProbeThreads)
    gather_probe_kernel(const uint4 *__restrict__ buf, long long total_recs, unsigned region_mask,
                        unsigned span_mask, int per_block_region, int iters, unsigned seed,
                        unsigned *sink) {
  const long long region_recs = (long long)region_mask + 1;
  long long base = 0;
  if (per_block_region) {
    const long long slots = total_recs / region_recs;  // >= 1 (checked on the host)
    base = ((long long)blockIdx.x % slots) * region_recs;
  }
  const unsigned lane = threadIdx.x & 31;
  const unsigned warp = blockIdx.x * (kProbeThreads / 32) + (threadIdx.x >> 5);
  // LCGs: one warp-uniform (where the warp loads), one per lane (where in that window)
  unsigned xw = seed * 747796405u + warp * 2891336453u + 1u;
  unsigned xl = (seed ^ 0x9e3779b9u) * 747796405u + (warp * 32u + lane) * 2654435761u + 7u;
  unsigned acc = 0;
  for (int i = 0; i < iters; ++i) {
    uint4 v[kProbeUnroll];
#pragma unroll
    for (int u = 0; u < kProbeUnroll; ++u) {
      xw = xw * 1664525u + 1013904223u;
      xl = xl * 1664525u + 1013904223u;
      const unsigned r = (((xw >> 7) & ~span_mask) | ((xl >> 7) & span_mask)) & region_mask;
      v[u] = __ldg(buf + base + r);
    }
#pragma unroll
    for (int u = 0; u < kProbeUnroll; ++u) acc ^= v[u].x ^ v[u].y ^ v[u].z ^ v[u].w;
  }
  // keeps the loads alive; never taken for a zero-filled buffer (acc stays 0)
  if (acc == 0x5eed5eedu) sink[0] = acc;
}

static bool pow2(long long x) { return x > 0 && (x & (x - 1)) == 0; }

}  // namespace ftle

using namespace ftle;

extern "C" int ftle_gather_probe(const void *buf, int64_t buf_bytes, int64_t region_bytes,
                                 int64_t lane_span_bytes, int32_t per_block_region,
                                 int32_t blocks, int32_t iters, uint32_t seed, void *sink,
                                 void *stream) {
  if (!buf || !sink) return fail_invalid("probe buffer and sink must be device pointers");
  if (reinterpret_cast<uintptr_t>(buf) % 16 != 0) return fail_invalid("buffer must be 16-byte aligned");
  if (!pow2(region_bytes) || region_bytes < 16 || region_bytes > buf_bytes ||
      region_bytes > (512ll << 20))
    return fail_invalid("region_bytes must be a power of two in [16, min(buffer, 512 MiB)]");
  if (!pow2(lane_span_bytes) || lane_span_bytes < 16 || lane_span_bytes > region_bytes)
    return fail_invalid("lane_span_bytes must be a power of two in [16, region_bytes]");
  if (blocks < 1 || iters < 1) return fail_invalid("blocks and iters must be >= 1");
  const long long total = buf_bytes / 16;
  const unsigned region_mask = (unsigned)(region_bytes / 16 - 1);
  const unsigned span_mask = (unsigned)(lane_span_bytes / 16 - 1);
  gather_probe_kernel<<<blocks, kProbeThreads, 0, as_stream(stream)>>>(
      static_cast<const uint4 *>(buf), total, region_mask, span_mask, per_block_region ? 1 : 0,
      iters, seed, static_cast<unsigned *>(sink));
  return check_launch("gather_probe_kernel");
}

extern "C" int64_t ftle_gather_probe_loads(int32_t blocks, int32_t iters) {
  return (int64_t)blocks * kProbeThreads * iters * kProbeUnroll;
}
