// mlp_fused.cu -- fused surrogate inference: seeds -> FTLE in one persistent kernel.
//
// Network (fixed shape): 32 Fourier frequencies (64 features of (x, y, t0)),
// 4 hidden layers of 256 SiLU units, 2 outputs (the displacement / out_scale).
// The FTLE of the surrogate flow map x0 -> x0 + s*y(x0) needs y and its Jacobian,
// so every seed carries three rows through the network: the primal activations
// and the forward-mode tangents d/dx0, d/dy0 (the tangent of a SiLU layer is the
// pre-activation tangent times silu'(z) of the primal row).
//
// Tile = 40 seeds = 128 tensor-core rows.  TMEM lane quadrant q (rows 32q..32q+31)
// holds seeds 10q..10q+9 as rows [10 primal | 10 d/dx | 10 d/dy | 2 zero], so the
// epilogue hands silu'(z) from a primal lane to its two tangent lanes with warp
// shuffles.
//
// Warp roles (17 warps):
//   * warp 16, one thread: streams the pre-packed weight chunks (17 per tile, each
//     already in the K-major core-matrix smem layout) by 1D bulk copies into a
//     3-stage ring (full barrier: bytes landed; empty barrier: the MMAs reading the
//     stage completed, via tcgen05.commit) and issues the tcgen05.mma chains
//     (M = 128, N = 256 or 16, K = 64 per chunk).  Layers alternate between two
//     TMEM accumulators (2 x 256 columns), and the MMAs of K chunk c of layer l+1
//     start as soon as chunk c of layer l's output is in shared memory, so the
//     tensor core works on layer l+1 while the epilogue still finishes layer l.
//   * warps 0..15: warp w reads TMEM lane quadrant w%4, columns 64c + 16(w/4) + [0,16)
//     of every K chunk c (chunks in order, TMEM loads software-pipelined), applies
//     bias, SiLU and the tangent rule, writes the BF16 A operand of the next layer
//     in place and arrives on that chunk's barrier (16 arrivals); at the output
//     layer warps 0..3 form F = I + s*J, C = F^T F and the FTLE in FP64 (as
//     ftle_mlp_jacobian_ftle).  They also compute the next tile's features.
// Every wait is bounded; on timeout the kernel flags the error word, stops both
// roles, waits (bounded) for its copies and MMAs in flight, frees TMEM, returns.
#include <cuda_bf16.h>

#include "common.cuh"
#include "umma.cuh"

namespace ftle {
namespace mlp {

constexpr int kEpiWarps = 16;
constexpr int kFThreads = (kEpiWarps + 1) * 32;
constexpr int kSeedsPerQuad = 10;
constexpr int kSeedsPerTile = 4 * kSeedsPerQuad;
constexpr int kHid = 256;
constexpr int kFreq = 32;
constexpr int kOutRows = 16;
constexpr int kChunksPerPass = 17;  // 1 (64 -> 256) + 3 x 4 (256 -> 256) + 4 (256 -> 16)
constexpr int kWStages = 3;
constexpr int kWStageBytes = kHid * kChunkK * 2;     // 32 KB
constexpr int kAChunkBytes = 128 * kChunkK * 2;      // 16 KB
constexpr int kABytes = 4 * kAChunkBytes;            // 64 KB (K = 256)
constexpr int kOutChunkBytes = kOutRows * kChunkK * 2;
constexpr long long kPackedBytes = 13LL * kWStageBytes + 4LL * kOutChunkBytes;
constexpr int kBiasFloats = 4 * kHid + kOutRows;
constexpr size_t kFusedSmem = (size_t)kABytes + (size_t)kWStages * kWStageBytes;
constexpr uint32_t kTmemCols = 512;

struct SurrogateArgs {
  const double *points;  // n x 2 seed positions
  long long n;
  double t0;
  const unsigned char *wpack;
  const float *bias;     // kBiasFloats
  const float4 *freq;    // kFreq x (kx, ky, kt, phase)
  double out_scale;
  double inv_T;
  double *ftle;          // n, may be null
  double *end_pos;       // n x 2, may be null
  int *err;
};

// Chunk i of a pass: layer, K chunk index, bytes and offset in the packed image.
__host__ __device__ inline void chunk_info(int i, int &layer, int &kc, uint32_t &bytes,
                                           long long &off) {
  if (i == 0) {
    layer = 0, kc = 0, bytes = kWStageBytes, off = 0;
  } else if (i <= 12) {
    layer = 1 + (i - 1) / 4, kc = (i - 1) % 4, bytes = kWStageBytes, off = (long long)i * kWStageBytes;
  } else {
    layer = 4, kc = i - 13, bytes = kOutChunkBytes;
    off = 13LL * kWStageBytes + (long long)(i - 13) * kOutChunkBytes;
  }
}

struct FusedShared {
  unsigned long long full_bar[kWStages];
  unsigned long long empty_bar[kWStages];
  unsigned long long acc_full[2];
  unsigned long long a_ready[4];
  unsigned long long drain_bar;
  uint32_t tmem_slot;
  int abort_flag;
  float bias[kBiasFloats];
  float4 freq[kFreq];
};

__device__ __forceinline__ bool aborted(const FusedShared &S) {
  return *reinterpret_cast<const volatile int *>(&S.abort_flag) != 0;
}

// ---- producer: weight ring + MMA issue (one thread) ---------------------------------
__device__ void fused_producer(const SurrogateArgs &a, FusedShared &S, uint32_t sA_u,
                               uint32_t sW_u, uint32_t tmem, long long num_tiles) {
  const long long my_tiles =
      (long long)blockIdx.x < num_tiles ? (num_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const long long total = my_tiles * kChunksPerPass;
  long long issued = 0, consumed = 0;
  uint32_t ready_cnt[4] = {0u, 0u, 0u, 0u};
  auto issue = [&](long long j) {
    int layer, kc;
    uint32_t bytes;
    long long off;
    chunk_info((int)(j % kChunksPerPass), layer, kc, bytes, off);
    const int s = (int)(j % kWStages);
    mbar_expect_tx(smem_u32(&S.full_bar[s]), bytes);
    bulk_g2s(sW_u + s * kWStageBytes, a.wpack + off, bytes, smem_u32(&S.full_bar[s]));
  };
  for (; issued < total && issued < kWStages - 1; ++issued) issue(issued);
  bool ok = true;
  long long L = 0;
  for (long long t = blockIdx.x; ok && t < num_tiles; t += gridDim.x) {
    for (int l = 0; l < 5; ++l, ++L) {
      const uint32_t acc = tmem + (uint32_t)(L & 1) * 256u;
      const int nk = l == 0 ? 1 : 4;
      const uint32_t idesc = idesc_bf16(128, l < 4 ? kHid : kOutRows);
      for (int c = 0; c < nk && ok; ++c) {
        // chunk c of this layer's input is in shared memory
        ok = mbar_wait(smem_u32(&S.a_ready[c]), ready_cnt[c] & 1u) && !aborted(S);
        ++ready_cnt[c];
        const long long j = consumed;
        const int s = (int)(j % kWStages);
        ok = ok && mbar_wait(smem_u32(&S.full_bar[s]), (uint32_t)((j / kWStages) & 1));
        if (!ok) break;
        fence_after_sync();
#pragma unroll
        for (int kk = 0; kk < kChunkK / 16; ++kk) {
          const uint64_t ad = smem_desc(sA_u + c * kAChunkBytes + kk * 256, 128, kChunkK * 16);
          const uint64_t bd = smem_desc(sW_u + s * kWStageBytes + kk * 256, 128, kChunkK * 16);
          umma(acc, ad, bd, idesc, (c > 0 || kk > 0) ? 1u : 0u);
        }
        umma_commit(smem_u32(&S.empty_bar[s]));
        ++consumed;
        // refill the stage chunk j-1 used with chunk j + kWStages - 1
        const long long nxt = j + kWStages - 1;
        if (nxt < total && nxt == issued) {
          if (j >= 1 && !mbar_wait(smem_u32(&S.empty_bar[(j - 1) % kWStages]),
                                   (uint32_t)(((j - 1) / kWStages) & 1))) {
            ok = false;
            break;
          }
          issue(issued);
          ++issued;
        }
      }
      if (!ok) break;
      umma_commit(smem_u32(&S.acc_full[L & 1]));
    }
  }
  if (!ok) {
    *reinterpret_cast<volatile int *>(&S.abort_flag) = 1;
    atomicExch(a.err, 1);
    // MMAs in flight complete, and copies in flight land, before the CTA exits
    umma_commit(smem_u32(&S.drain_bar));
    mbar_wait(smem_u32(&S.drain_bar), 0);
    for (long long j = consumed; j < issued; ++j)
      mbar_wait(smem_u32(&S.full_bar[j % kWStages]), (uint32_t)((j / kWStages) & 1));
  }
}

// ---- epilogue warps -------------------------------------------------------------------
__device__ __forceinline__ void hidden_part(const uint32_t (&r)[16], const float *bias,
                                            int role, int sl, unsigned char *chunk_base,
                                            int row, int kcol) {
  // Branch-free: every lane evaluates the SiLU of its own value (lanes of a warp
  // issue together, so a role branch would cost the same slots); tangent lanes take
  // silu'(z) from their seed's primal lane (lane sl).  Zero rows stay zero (v = 0).
  uint32_t p[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    float o[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const float v = __uint_as_float(r[2 * i + e]);
      const float z = v + bias[2 * i + e];
      const float sg = sigmoidf_(z);
      const float h = z * sg;
      const float d = dsilu_from(h, sg);
      const float dd = __shfl_sync(0xFFFFFFFFu, d, sl);
      o[e] = role == 0 ? h : v * dd;
    }
    const __nv_bfloat162 hh = __floats2bfloat162_rn(o[0], o[1]);
    p[i] = *reinterpret_cast<const uint32_t *>(&hh);
  }
  *reinterpret_cast<uint4 *>(chunk_base + kmaj_off(row, kcol)) = make_uint4(p[0], p[1], p[2], p[3]);
  *reinterpret_cast<uint4 *>(chunk_base + kmaj_off(row, kcol + 8)) =
      make_uint4(p[4], p[5], p[6], p[7]);
}

__device__ void fused_epilogue(const SurrogateArgs &a, FusedShared &S, unsigned char *sA,
                               uint32_t tmem, long long num_tiles, int warp, int lane) {
  const int quad = warp & 3, part = warp >> 2;
  const int role = lane < 3 * kSeedsPerQuad ? lane / kSeedsPerQuad : 3;  // 0 primal, 1 d/dx, 2 d/dy
  const int sl = lane % kSeedsPerQuad;
  const int row = 32 * quad + lane;
  const int etid = warp * 32 + lane;
  uint32_t acc_cnt[2] = {0u, 0u};
  long long L = 0;
  for (long long t = blockIdx.x; t < num_tiles; t += gridDim.x) {
    // ---- layer-0 operand: features and their tangents (A chunk 0) -------------------
    for (int e = etid; e < kSeedsPerTile * kFreq; e += kEpiWarps * 32) {
      const int st = e / kFreq, f = e - st * kFreq;
      const int q = st / kSeedsPerQuad, s = st - q * kSeedsPerQuad;
      const int r0 = 32 * q + s;
      const long long g = t * kSeedsPerTile + st;
      float sn = 0.f, cs = 0.f;
      const float4 k = S.freq[f];
      if (g < a.n) {
        // the phase is formed and reduced in FP64, as in the feature kernel of training
        const double ph = (double)k.x * a.points[2 * g] + (double)k.y * a.points[2 * g + 1] +
                          (double)k.z * a.t0 + (double)k.w;
        const double two_pi = 6.283185307179586;
        sincosf((float)(ph - two_pi * floor(ph / two_pi)), &sn, &cs);
      }
      const float vals[3][2] = {{sn, cs}, {k.x * cs, -k.x * sn}, {k.y * cs, -k.y * sn}};
#pragma unroll
      for (int rr = 0; rr < 3; ++rr) {
        const int r = r0 + rr * kSeedsPerQuad;
        *reinterpret_cast<__nv_bfloat16 *>(sA + kmaj_off(r, f)) = __float2bfloat16_rn(vals[rr][0]);
        *reinterpret_cast<__nv_bfloat16 *>(sA + kmaj_off(r, kFreq + f)) =
            __float2bfloat16_rn(vals[rr][1]);
      }
    }
    if (etid < 64) {  // the 2 zero rows of each quadrant, 8 x 16 B each
      const int pr = etid >> 3, c = etid & 7;
      const int r = 32 * (pr >> 1) + 30 + (pr & 1);
      *reinterpret_cast<uint4 *>(sA + kmaj_off(r, 8 * c)) = make_uint4(0u, 0u, 0u, 0u);
    }
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_u32(&S.a_ready[0]));

    for (int l = 0; l < 5; ++l, ++L) {
      const int ab = (int)(L & 1);
      const bool ok = mbar_wait(smem_u32(&S.acc_full[ab]), acc_cnt[ab] & 1u);
      ++acc_cnt[ab];
      if (!ok) *reinterpret_cast<volatile int *>(&S.abort_flag) = 1;
      if (__any_sync(0xFFFFFFFFu, !ok || aborted(S))) return;  // warp-uniform exit
      fence_after_sync();
      const uint32_t trow = tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)ab * 256u;
      if (l < 4) {
        const float *b = S.bias + l * kHid;
        uint32_t r0[16], r1[16];
        tmem_ld16_start(trow + (uint32_t)(16 * part), r0);
        tmem_wait16(r0);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int col = 64 * c + 16 * part;
          if (c < 3) tmem_ld16_start(trow + (uint32_t)(col + 64), (c & 1) ? r0 : r1);
          hidden_part((c & 1) ? r1 : r0, b + col, role, sl, sA + c * kAChunkBytes, row, 16 * part);
          if (c < 3) tmem_wait16((c & 1) ? r0 : r1);
          fence_before_sync();
          fence_proxy_async_smem();
          __syncwarp();
          if (lane == 0) mbar_arrive(smem_u32(&S.a_ready[c]));
        }
      } else {
        if (part == 0) {
          uint32_t rr[16];
          tmem_ld16_start(trow, rr);
          tmem_wait16(rr);
          const float y0 = __uint_as_float(rr[0]), y1 = __uint_as_float(rr[1]);
          const float jx0 = __shfl_sync(0xFFFFFFFFu, y0, sl + kSeedsPerQuad);
          const float jx1 = __shfl_sync(0xFFFFFFFFu, y1, sl + kSeedsPerQuad);
          const float jy0 = __shfl_sync(0xFFFFFFFFu, y0, sl + 2 * kSeedsPerQuad);
          const float jy1 = __shfl_sync(0xFFFFFFFFu, y1, sl + 2 * kSeedsPerQuad);
          const long long g = t * kSeedsPerTile + quad * kSeedsPerQuad + lane;
          if (role == 0 && g < a.n) {
            const double s = a.out_scale;
            if (a.ftle) {
              const double fa = 1.0 + s * (double)jx0, fb = s * (double)jy0;
              const double fc = s * (double)jx1, fd = 1.0 + s * (double)jy1;
              const double c11 = fa * fa + fc * fc, c12 = fa * fb + fc * fd;
              const double c22 = fb * fb + fd * fd;
              const double tr = 0.5 * (c11 + c22), df = 0.5 * (c11 - c22);
              a.ftle[g] = log(sqrt(tr + sqrt(df * df + c12 * c12))) * a.inv_T;
            }
            if (a.end_pos) {
              a.end_pos[2 * g] = a.points[2 * g] + s * (double)(y0 + S.bias[4 * kHid]);
              a.end_pos[2 * g + 1] = a.points[2 * g + 1] + s * (double)(y1 + S.bias[4 * kHid + 1]);
            }
          }
        }
        fence_before_sync();
      }
    }
  }
}

__global__ void __launch_bounds__(kFThreads, 1) surrogate_ftle_kernel(SurrogateArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) FusedShared S;
  unsigned char *sA = smem;
  unsigned char *sW = smem + kABytes;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long num_tiles = (a.n + kSeedsPerTile - 1) / kSeedsPerTile;

  if (warp == 0) tmem_alloc(smem_u32(&S.tmem_slot), kTmemCols);
  if (tid == 32) {
    for (int s = 0; s < kWStages; ++s) {
      mbar_init(smem_u32(&S.full_bar[s]), 1);
      mbar_init(smem_u32(&S.empty_bar[s]), 1);
    }
    for (int i = 0; i < 2; ++i) mbar_init(smem_u32(&S.acc_full[i]), 1);
    for (int i = 0; i < 4; ++i) mbar_init(smem_u32(&S.a_ready[i]), kEpiWarps);
    mbar_init(smem_u32(&S.drain_bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    S.abort_flag = 0;
  }
  for (int i = tid; i < kBiasFloats; i += kFThreads) S.bias[i] = a.bias[i];
  for (int i = tid; i < kFreq; i += kFThreads) S.freq[i] = a.freq[i];
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = S.tmem_slot;

  if (warp == kEpiWarps) {
    if (lane == 0) fused_producer(a, S, smem_u32(sA), smem_u32(sW), tmem, num_tiles);
    __syncwarp();
  } else {
    fused_epilogue(a, S, sA, tmem, num_tiles, warp, lane);
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

// Packs the five BF16 weight matrices (row-major out x in: 256x64, 3 x 256x256,
// and the first 16 rows of the output layer, 256 columns) into the chunk images.
__global__ void surrogate_pack_kernel(const __nv_bfloat16 *__restrict__ w0,
                                      const __nv_bfloat16 *__restrict__ w1,
                                      const __nv_bfloat16 *__restrict__ w2,
                                      const __nv_bfloat16 *__restrict__ w3,
                                      const __nv_bfloat16 *__restrict__ w4,
                                      unsigned char *__restrict__ out) {
  const long long total = 13LL * kHid * kChunkK + 4LL * kOutRows * kChunkK;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int chunk;
    long long q;
    if (e < 13LL * kHid * kChunkK) {
      chunk = (int)(e / (kHid * kChunkK));
      q = e - (long long)chunk * kHid * kChunkK;
    } else {
      const long long e2 = e - 13LL * kHid * kChunkK;
      chunk = 13 + (int)(e2 / (kOutRows * kChunkK));
      q = e2 - (long long)(chunk - 13) * kOutRows * kChunkK;
    }
    int layer, kc;
    uint32_t bytes;
    long long off;
    chunk_info(chunk, layer, kc, bytes, off);
    const int r = (int)(q / kChunkK), k = (int)(q % kChunkK);
    const __nv_bfloat16 *w = layer == 0 ? w0 : layer == 1 ? w1 : layer == 2 ? w2 : layer == 3 ? w3 : w4;
    const int ld = layer == 0 ? 2 * kFreq : kHid;
    *reinterpret_cast<__nv_bfloat16 *>(out + off + kmaj_off(r, k)) = w[(long long)r * ld + kc * kChunkK + k];
  }
}

}  // namespace mlp
}  // namespace ftle

using namespace ftle;
using namespace ftle::mlp;

extern "C" {

int64_t ftle_surrogate_packed_bytes(void) { return kPackedBytes; }

int ftle_surrogate_pack(const void *w0, const void *w1, const void *w2, const void *w3,
                        const void *w4, void *packed, void *stream) {
  if (!w0 || !w1 || !w2 || !w3 || !w4 || !packed) return fail_invalid("null pointer");
  if (reinterpret_cast<uintptr_t>(packed) % 16) return fail_invalid("packed must be 16-byte aligned");
  surrogate_pack_kernel<<<(int)kNumSMs * 4, 256, 0, as_stream(stream)>>>(
      static_cast<const __nv_bfloat16 *>(w0), static_cast<const __nv_bfloat16 *>(w1),
      static_cast<const __nv_bfloat16 *>(w2), static_cast<const __nv_bfloat16 *>(w3),
      static_cast<const __nv_bfloat16 *>(w4), static_cast<unsigned char *>(packed));
  return check_launch("surrogate_pack_kernel");
}

int ftle_surrogate_ftle(const double *points, int64_t n, double t0, const void *packed,
                        const float *bias, const float *freq, double out_scale, double T,
                        double *ftle, double *end_positions, int32_t *error_word, void *stream) {
  if (n < 0) return fail_invalid("n must be >= 0");
  if (n == 0) return FTLE_OK;
  if (!points || !packed || !bias || !freq || !error_word) return fail_invalid("null pointer");
  if (!ftle && !end_positions) return fail_invalid("nothing to compute");
  if (T == 0.0) return fail_invalid("T must be non-zero");
  if (reinterpret_cast<uintptr_t>(packed) % 16 || reinterpret_cast<uintptr_t>(freq) % 16)
    return fail_invalid("packed weights and freq must be 16-byte aligned");
  SurrogateArgs a;
  a.points = points;
  a.n = n;
  a.t0 = t0;
  a.wpack = static_cast<const unsigned char *>(packed);
  a.bias = bias;
  a.freq = reinterpret_cast<const float4 *>(freq);
  a.out_scale = out_scale;
  a.inv_T = 1.0 / fabs(T);
  a.ftle = ftle;
  a.end_pos = end_positions;
  a.err = error_word;
  const long long tiles = (n + kSeedsPerTile - 1) / kSeedsPerTile;
  const int grid = (int)(tiles < kNumSMs ? tiles : kNumSMs);
  cudaFuncSetAttribute(surrogate_ftle_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kFusedSmem);
  surrogate_ftle_kernel<<<grid, kFThreads, kFusedSmem, as_stream(stream)>>>(a);
  return check_launch("surrogate_ftle_kernel");
}

}  // extern "C"
