// mlp.cu -- BF16 tensor-core (tcgen05 / TMEM) kernels of the flow-map surrogate MLP.
//
// GEMM: C[M x N] (+)= A[M x K] * B[N x K]^T, BF16 operands, FP32 accumulation in
// tensor memory.  One CTA (4 warps) owns a 128 x NT tile (NT <= 128) of C:
//   * operands are staged in shared memory as no-swizzle core matrices (8 x 16 B) by
//     TMA (cp.async.bulk.tensor 2D boxes, 16 bytes wide, no multicast): an operand
//     stored row-major (K contiguous) as K-major tiles, an operand stored transposed
//     (its M/N index contiguous) as MN-major tiles with the descriptor's major bit set,
//     so neither needs a transposition; every product of training (X W^T, dZ W, dZ^T X)
//     and of the Jacobian tangents runs through this one kernel; rows past M (or N) lie
//     outside the tensor maps and arrive as zeros;
//   * one elected thread is both the TMA producer and the tensor-core issuer: a 3-stage
//     ring with a full barrier (TMA bytes) and an empty barrier (tcgen05.commit) per
//     stage, so chunks c+1 and c+2 are in flight while the tensor core works on chunk c;
//     it issues tcgen05.mma (kind::f16, M = 128, N = NT, K = 16 per instruction);
//   * the epilogue reads the accumulator back with tcgen05.ld (warp w owns TMEM
//     lanes 32w..32w+31 = tile rows) and applies one of the fused epilogues:
//       EPI_F32        store (or, split-K, atomically add) FP32 C
//       EPI_BIAS_SILU  z = acc + b: store z (FP32) and h = silu(z) (BF16)
//       EPI_DSILU      g = acc * silu'(z_in): store g (BF16), column sums of g
//                      (the bias gradient) atomically into colsum
//       EPI_BIAS_F32   store acc + b (FP32)
// Every mbarrier wait is bounded; on timeout the kernel records an error in the
// caller's error word, waits (bounded) for its copies and MMAs in flight, skips
// the epilogue, frees its TMEM and returns.
//
// Element-wise kernels of the surrogate: Fourier features (+ their x/y tangents),
// the MSE loss gradient, Adam, and the FTLE of the network's flow-map Jacobian.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <mutex>

#include "common.cuh"
#include "umma.cuh"

namespace ftle {
namespace mlp {

constexpr int kTileM = 128;
constexpr int kStages = 3;
constexpr int kMaxNT = 128;

enum { EPI_F32 = 0, EPI_BIAS_SILU = 1, EPI_DSILU = 2, EPI_BIAS_F32 = 3 };

struct Epi {
  int mode;
  int ldc;
  float *c;              // EPI_F32 / EPI_BIAS_F32 output (FP32)
  const float *bias;     // EPI_BIAS_SILU / EPI_BIAS_F32
  const float *zin;      // EPI_DSILU pre-activations
  int ldzin;
  float *zout;           // EPI_BIAS_SILU pre-activations out (optional)
  int ldzout;
  __nv_bfloat16 *hout;   // EPI_BIAS_SILU / EPI_DSILU BF16 output
  int ldh;
  float *colsum;         // EPI_DSILU column sums (optional)
  int accumulate;        // EPI_F32: atomically add into c
};

// Operand staging by TMA (cp.async.bulk.tensor, no multicast: every tile is this GPU's
// own memory).  Each operand has a 2D tensor map over its BF16 matrix; the boxes are
// 16 bytes wide so the shared-memory tiles come out in the no-swizzle core-matrix
// layouts the tensor core reads:
//   K-major operand (element (r, k) at src[r*ld + k]): kChunkK/8 boxes of 8 k x R rows,
//     tile layout [k/8][r][16 B]: core matrices 128 B apart along the rows (SBO) and
//     R*16 B apart along K (LBO);
//   MN-major operand (element (r, k) at src[k*ld + r]): R/8 boxes of 8 r x kChunkK k,
//     tile layout [r/8][k][16 B]: core matrices 128 B apart along K (LBO) and
//     kChunkK*16 B apart along the rows (SBO).
// Rows past M (or N) lie outside the tensor map and arrive as zeros.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y,
                                            uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}

template <bool TRANS>
__device__ __forceinline__ void tma_operand(const CUtensorMap *map, uint32_t tile, int r0, int R,
                                            int k0, uint32_t mbar) {
  if constexpr (!TRANS) {
#pragma unroll
    for (int j = 0; j < kChunkK / 8; ++j) tma_load_2d(tile + j * R * 16, map, k0 + 8 * j, r0, mbar);
  } else {
    for (int g = 0; g < R / 8; ++g) tma_load_2d(tile + g * kChunkK * 16, map, r0 + 8 * g, k0, mbar);
  }
}

// Descriptor of the K = 16 slice j of an operand tile with R rows (see the layouts above).
template <bool TRANS>
__device__ __forceinline__ uint64_t operand_desc(uint32_t tile, int R, int j) {
  if constexpr (!TRANS) return smem_desc(tile + j * 2 * R * 16, R * 16, 128);
  else return smem_desc(tile + j * 256, 128, kChunkK * 16);
}

constexpr int kPStages = 3;    // TMA -> tensor-core stage ring (2 CTAs fit an SM)
constexpr int kEpiWarps = 8;   // epilogue warps: two per TMEM lane quarter
constexpr int kGemmThreads = 64 + 32 * kEpiWarps;  // producer warp, MMA warp, epilogue warps
constexpr uint32_t kAccCols = 2 * kMaxNT;          // two accumulators of up to 128 columns

// Named barrier of the 128 epilogue threads (the producer and MMA warps never join it).
__device__ __forceinline__ void epi_barrier() {
  asm volatile("bar.sync 1, %0;" ::"n"(32 * kEpiWarps) : "memory");
}

// The fused epilogues on 8 consecutive columns [n, n+8) of one tile row.
__device__ __forceinline__ void epilogue8(const Epi &epi, float *v, int row, bool row_ok, int n,
                                          int lane, float *colsum8) {
  if (epi.mode == EPI_F32 || epi.mode == EPI_BIAS_F32) {
    if (epi.mode == EPI_BIAS_F32) {
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] += epi.bias[n + i];
    }
    if (row_ok) {
      float *dst = epi.c + (long long)row * epi.ldc + n;
      if (epi.accumulate) {
#pragma unroll
        for (int i = 0; i < 8; ++i) atomicAdd(dst + i, v[i]);
      } else {
        reinterpret_cast<float4 *>(dst)[0] = make_float4(v[0], v[1], v[2], v[3]);
        reinterpret_cast<float4 *>(dst)[1] = make_float4(v[4], v[5], v[6], v[7]);
      }
    }
  } else if (epi.mode == EPI_BIAS_SILU) {
    if (row_ok) {
      float z[8];
      uint32_t packed[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) z[i] = v[i] + epi.bias[n + i];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const __nv_bfloat162 hh = __floats2bfloat162_rn(z[2 * i] * sigmoidf_(z[2 * i]),
                                                        z[2 * i + 1] * sigmoidf_(z[2 * i + 1]));
        packed[i] = *reinterpret_cast<const uint32_t *>(&hh);
      }
      *reinterpret_cast<uint4 *>(epi.hout + (long long)row * epi.ldh + n) =
          make_uint4(packed[0], packed[1], packed[2], packed[3]);
      if (epi.zout) {
        float *zd = epi.zout + (long long)row * epi.ldzout + n;
        reinterpret_cast<float4 *>(zd)[0] = make_float4(z[0], z[1], z[2], z[3]);
        reinterpret_cast<float4 *>(zd)[1] = make_float4(z[4], z[5], z[6], z[7]);
      }
    }
  } else {  // EPI_DSILU
    float g[8];
    if (row_ok) {
      const float *zs = epi.zin + (long long)row * epi.ldzin + n;
      const float4 za = reinterpret_cast<const float4 *>(zs)[0];
      const float4 zb = reinterpret_cast<const float4 *>(zs)[1];
      const float z[8] = {za.x, za.y, za.z, za.w, zb.x, zb.y, zb.z, zb.w};
      uint32_t packed[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const float sg = sigmoidf_(z[i]);
        g[i] = v[i] * dsilu_from(z[i] * sg, sg);
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const __nv_bfloat162 hh = __floats2bfloat162_rn(g[2 * i], g[2 * i + 1]);
        packed[i] = *reinterpret_cast<const uint32_t *>(&hh);
        // the bias gradient sums the values the next GEMM consumes
        g[2 * i] = __low2float(hh);
        g[2 * i + 1] = __high2float(hh);
      }
      *reinterpret_cast<uint4 *>(epi.hout + (long long)row * epi.ldh + n) =
          make_uint4(packed[0], packed[1], packed[2], packed[3]);
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) g[i] = 0.0f;
    }
    if (colsum8) {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        float s = g[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
        if (lane == 0) atomicAdd(&colsum8[i], s);
      }
    }
  }
}

template <bool A_T, bool B_T>
__global__ void __launch_bounds__(kGemmThreads, 2)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     int M, int N, int K, int NT, int k_per_split, int tiles_m, int splits,
                     int total, Epi epi, int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) unsigned long long fullb[kPStages];
  __shared__ __align__(8) unsigned long long emptyb[kPStages];
  __shared__ __align__(8) unsigned long long tfull[2];
  __shared__ __align__(8) unsigned long long tempty[2];
  __shared__ __align__(8) unsigned long long drainb;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int s_abort;      // set by any role on a timed-out wait
  __shared__ volatile int s_epi_abort;  // set and read by the epilogue warps only
  __shared__ float colsum_s[kMaxNT];
  const int tile_bytes = (kTileM + NT) * kChunkK * 2;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t smem0 = smem_u32(smem);

  if (warp == 1) tmem_alloc(smem_u32(&tmem_slot), kAccCols);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kPStages; ++s) {
      mbar_init(smem_u32(&fullb[s]), 1);
      mbar_init(smem_u32(&emptyb[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&tfull[b]), 1);
      mbar_init(smem_u32(&tempty[b]), kEpiWarps);
    }
    mbar_init(smem_u32(&drainb), 1);
    s_abort = 0;
    s_epi_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_slot;

  // work unit u -> (k split, m tile, n tile); consecutive units share the n tile's B
  auto unit = [&](int u, int &m0, int &n0, int &kbeg, int &nch) {
    const int s = u % splits;
    const int t = u / splits;
    m0 = (t % tiles_m) * kTileM;
    n0 = (t / tiles_m) * NT;
    kbeg = s * k_per_split;
    const int kend = min(K, kbeg + k_per_split);
    nch = kend > kbeg ? (kend - kbeg) / kChunkK : 0;
  };
  auto fail = [&]() {
    s_abort = 1;
    atomicExch(err, 1);
  };

  if (warp == 0) {
    // ---- TMA producer: every chunk of every unit of this CTA into the stage ring
    if (lane == 0) {
      int g = 0;
      for (int u = blockIdx.x; u < total && !s_abort; u += gridDim.x) {
        int m0, n0, kbeg, nch;
        unit(u, m0, n0, kbeg, nch);
        for (int c = 0; c < nch; ++c, ++g) {
          const int st = g % kPStages;
          if (!mbar_wait(smem_u32(&emptyb[st]), (uint32_t)(((g / kPStages) & 1) ^ 1)) ||
              s_abort) {
            fail();
            break;
          }
          const uint32_t sA = smem0 + st * tile_bytes;
          const uint32_t sB = sA + kTileM * kChunkK * 2;
          const uint32_t fb = smem_u32(&fullb[st]);
          mbar_expect_tx(fb, (uint32_t)tile_bytes);
          tma_operand<A_T>(&tmA, sA, m0, kTileM, kbeg + c * kChunkK, fb);
          tma_operand<B_T>(&tmB, sB, n0, NT, kbeg + c * kChunkK, fb);
        }
      }
      // no load may land after the shared memory is released: wait for the last ones
      for (int j = max(0, g - kPStages); j < g; ++j)
        mbar_wait(smem_u32(&fullb[j % kPStages]), (uint32_t)((j / kPStages) & 1));
    }
  } else if (warp == 1) {
    // ---- tensor-core issuer: unit j accumulates into TMEM buffer j & 1
    if (lane == 0) {
      const uint32_t idesc =
          idesc_bf16(kTileM, NT) | (A_T ? (1u << 15) : 0u) | (B_T ? (1u << 16) : 0u);
      int g = 0, j = 0;
      for (int u = blockIdx.x; u < total && !s_abort; u += gridDim.x, ++j) {
        int m0, n0, kbeg, nch;
        unit(u, m0, n0, kbeg, nch);
        const int b = j & 1;
        if (!mbar_wait(smem_u32(&tempty[b]), (uint32_t)(((j >> 1) & 1) ^ 1))) {
          fail();
          break;
        }
        fence_after_sync();
        const uint32_t acc = tmem + (uint32_t)(b * kMaxNT);
        bool ok = true;
        for (int c = 0; c < nch; ++c, ++g) {
          const int st = g % kPStages;
          if (!(ok = mbar_wait(smem_u32(&fullb[st]), (uint32_t)((g / kPStages) & 1)))) break;
          fence_after_sync();
          const uint32_t sA = smem0 + st * tile_bytes;
          const uint32_t sB = sA + kTileM * kChunkK * 2;
#pragma unroll
          for (int q = 0; q < kChunkK / 16; ++q)
            umma(acc, operand_desc<A_T>(sA, kTileM, q), operand_desc<B_T>(sB, NT, q), idesc,
                 (c > 0 || q > 0) ? 1u : 0u);
          umma_commit(smem_u32(&emptyb[st]));  // the stage is free once these MMAs are done
        }
        if (!ok) {
          fail();
          break;
        }
        umma_commit(smem_u32(&tfull[b]));  // the accumulator is ready once they are done
      }
      // every MMA issued above has completed before TMEM is released
      umma_commit(smem_u32(&drainb));
      mbar_wait(smem_u32(&drainb), 0u);
    }
  } else {
    // ---- epilogue warps: TMEM lanes 32q..32q+31 (q = warp % 4) are tile rows; the two
    // warps of a lane quarter take one half of the tile's columns each
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int et = threadIdx.x - 64;  // 0..255 among the epilogue threads
    int j = 0;
    for (int u = blockIdx.x; u < total; u += gridDim.x, ++j) {
      int m0, n0, kbeg, nch;
      unit(u, m0, n0, kbeg, nch);
      const int b = j & 1;
      const bool dsum = epi.mode == EPI_DSILU && epi.colsum;
      if (dsum) {
        for (int i = et; i < kMaxNT; i += 32 * kEpiWarps) colsum_s[i] = 0.0f;
        epi_barrier();
      }
      const bool ready = !s_epi_abort && mbar_wait(smem_u32(&tfull[b]), (uint32_t)((j >> 1) & 1));
      if (!__all_sync(0xffffffffu, ready) && lane == 0) {
        s_epi_abort = 1;
        fail();
      }
      // the epilogue warps agree before any of them leaves (they share named barriers)
      epi_barrier();
      if (s_epi_abort) break;
      fence_after_sync();
      const int row = m0 + 32 * q + lane;
      const bool row_ok = row < M;
      const uint32_t tbase = tmem + (uint32_t)(b * kMaxNT) + ((uint32_t)(32 * q) << 16);
      const int cw = NT / 2;  // columns per warp (a multiple of 8)
      for (int c = half * cw; c < (half + 1) * cw; c += 8) {
        float v[8];
        tmem_ld8(tbase + (uint32_t)c, v);
        const int n = n0 + c;
        if (n >= N) continue;  // uniform across the warp
        epilogue8(epi, v, row, row_ok, n, lane, dsum ? &colsum_s[c] : nullptr);
      }
      // the accumulator is drained: the issuer may reuse it
      fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&tempty[b]));
      if (dsum) {
        epi_barrier();
        for (int i = et; i < NT && n0 + i < N; i += 32 * kEpiWarps)
          atomicAdd(epi.colsum + n0 + i, colsum_s[i]);
        epi_barrier();
      }
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 1) tmem_dealloc(tmem, kAccCols);
}

// ---------------------------------------------------------------------------
// Element-wise kernels
// ---------------------------------------------------------------------------

// phase_f = kx_f x + ky_f y + kt_f t + c_f;  features [sin(phase) | cos(phase)] (BF16),
// optional tangents d/dx, d/dy of the features (BF16).  points: n x 3 FP64 (x, y, t).
__global__ void features_kernel(const double *__restrict__ pts, long long n,
                                const float4 *__restrict__ freq, int F,
                                __nv_bfloat16 *__restrict__ feat, __nv_bfloat16 *__restrict__ tx,
                                __nv_bfloat16 *__restrict__ ty) {
  const long long total = n * F;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long p = e / F;
    const int f = (int)(e - p * F);
    const float4 k = freq[f];
    // the phase is formed and reduced in FP64 so large coordinates keep precision
    const double ph = (double)k.x * pts[3 * p] + (double)k.y * pts[3 * p + 1] +
                      (double)k.z * pts[3 * p + 2] + (double)k.w;
    const double two_pi = 6.283185307179586;
    const float r = (float)(ph - two_pi * floor(ph / two_pi));
    float s, c;
    sincosf(r, &s, &c);
    const long long row = p * (2 * F);
    feat[row + f] = __float2bfloat16_rn(s);
    feat[row + F + f] = __float2bfloat16_rn(c);
    if (tx) {
      tx[row + f] = __float2bfloat16_rn(k.x * c);
      tx[row + F + f] = __float2bfloat16_rn(-k.x * s);
    }
    if (ty) {
      ty[row + f] = __float2bfloat16_rn(k.y * c);
      ty[row + F + f] = __float2bfloat16_rn(-k.y * s);
    }
  }
}

// Loss = sum over rows and the `outs` used columns of (y - target)^2 / n;
// dY = 2 (y - target) / n in BF16 (padded columns zero); the output layer's bias
// gradient (column sums of the BF16 dY) and the loss are added atomically.
__global__ void mse_grad_kernel(const float *__restrict__ y, int ldy,
                                const float *__restrict__ target, int outs, long long n,
                                float inv_n, __nv_bfloat16 *__restrict__ dy, int lddy,
                                float *__restrict__ dbias, float *__restrict__ loss) {
  __shared__ float part[8][5];
  float acc_loss = 0.0f;
  float acc_g[4] = {0.f, 0.f, 0.f, 0.f};
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    for (int c = 0; c < lddy; ++c) {
      float g = 0.0f;
      if (c < outs) {
        const float d = y[r * ldy + c] - target[r * outs + c];
        acc_loss += d * d;
        g = 2.0f * d * inv_n;
      }
      const __nv_bfloat16 gb = __float2bfloat16_rn(g);
      dy[r * lddy + c] = gb;
      if (c < outs) acc_g[c] += __bfloat162float(gb);
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    acc_loss += __shfl_xor_sync(0xFFFFFFFFu, acc_loss, o);
#pragma unroll
    for (int c = 0; c < 4; ++c) acc_g[c] += __shfl_xor_sync(0xFFFFFFFFu, acc_g[c], o);
  }
  if (lane == 0) {
    part[warp][0] = acc_loss;
    for (int c = 0; c < 4; ++c) part[warp][1 + c] = acc_g[c];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float l = 0.f, g[4] = {0.f, 0.f, 0.f, 0.f};
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      l += part[w][0];
      for (int c = 0; c < 4; ++c) g[c] += part[w][1 + c];
    }
    atomicAdd(loss, l * inv_n);
    for (int c = 0; c < outs; ++c) atomicAdd(dbias + c, g[c]);
  }
}

// Adam (decoupled weight decay) on FP32 master parameters; refreshes the BF16
// copy the GEMMs read and zeroes the gradient for the next step's accumulation.
__global__ void adam_kernel(float *__restrict__ w, float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, __nv_bfloat16 *__restrict__ wb, long long n,
                            float lr, float b1, float b2, float eps, float c1, float c2,
                            float weight_decay) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / c1, vh = vi / c2;
    const float wi = w[i] - lr * (mh / (sqrtf(vh) + eps) + weight_decay * w[i]);
    w[i] = wi;
    wb[i] = __float2bfloat16_rn(wi);
    g[i] = 0.0f;
  }
}

// FTLE of x -> x + s * net(x): F = I + s [dY/dx dY/dy], C = F^T F, lambda_max of the
// 2x2 symmetric C in closed form, ftle = log(sqrt(lambda)) / |T| (FP64).
__global__ void jacobian_ftle_kernel(const float *__restrict__ jx, const float *__restrict__ jy,
                                     int ld, long long n, double scale, double inv_T,
                                     double *__restrict__ ftle) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double a = 1.0 + scale * (double)jx[i * ld];      // d x_T / d x0
    const double b = scale * (double)jy[i * ld];            // d x_T / d y0
    const double c = scale * (double)jx[i * ld + 1];        // d y_T / d x0
    const double d = 1.0 + scale * (double)jy[i * ld + 1];  // d y_T / d y0
    const double c11 = a * a + c * c, c12 = a * b + c * d, c22 = b * b + d * d;
    const double tr = 0.5 * (c11 + c22), df = 0.5 * (c11 - c22);
    const double lam = tr + sqrt(df * df + c12 * c12);
    ftle[i] = log(sqrt(lam)) * inv_T;
  }
}

// Predicted end positions: out[i] = x0[i] + s * y[i] (FP64, n x 2).
__global__ void apply_displacement_kernel(const double *__restrict__ pts,
                                          const float *__restrict__ y, int ldy, long long n,
                                          double scale, double *__restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    out[2 * i] = pts[3 * i] + scale * (double)y[i * ldy];
    out[2 * i + 1] = pts[3 * i + 1] + scale * (double)y[i * ldy + 1];
  }
}

// 3D features: points n x 4 FP64 (x, y, z, t); freq rows of 8 FP32
// (kx, ky, kz, kt, phase, 0, 0, 0); tangents d/dx, d/dy, d/dz (each may be null).
__global__ void features3_kernel(const double *__restrict__ pts, long long n,
                                 const float4 *__restrict__ freq, int F,
                                 __nv_bfloat16 *__restrict__ feat, __nv_bfloat16 *__restrict__ tx,
                                 __nv_bfloat16 *__restrict__ ty, __nv_bfloat16 *__restrict__ tz) {
  const long long total = n * F;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long p = e / F;
    const int f = (int)(e - p * F);
    const float4 k = freq[2 * f];
    const float ph0 = freq[2 * f + 1].x;
    const double ph = (double)k.x * pts[4 * p] + (double)k.y * pts[4 * p + 1] +
                      (double)k.z * pts[4 * p + 2] + (double)k.w * pts[4 * p + 3] + (double)ph0;
    const double two_pi = 6.283185307179586;
    const float r = (float)(ph - two_pi * floor(ph / two_pi));
    float sn, cs;
    sincosf(r, &sn, &cs);
    const long long row = p * (2 * F);
    feat[row + f] = __float2bfloat16_rn(sn);
    feat[row + F + f] = __float2bfloat16_rn(cs);
    __nv_bfloat16 *t[3] = {tx, ty, tz};
    const float kk[3] = {k.x, k.y, k.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (t[a]) {
        t[a][row + f] = __float2bfloat16_rn(kk[a] * cs);
        t[a][row + F + f] = __float2bfloat16_rn(-kk[a] * sn);
      }
    }
  }
}

// 3D FTLE of x -> x + s * net(x): F[r][j] = delta_rj + s * dY_r/dx_j (tangent j's
// column r), C = F^T F, lambda_max by Jacobi rotations, ftle = log(sqrt(lambda))/|T|.
__global__ void jacobian_ftle3_kernel(const float *__restrict__ jx, const float *__restrict__ jy,
                                      const float *__restrict__ jz, int ld, long long n,
                                      double scale, double inv_T, double *__restrict__ ftle) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float *J[3] = {jx + i * ld, jy + i * ld, jz + i * ld};
    double F[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int j = 0; j < 3; ++j) F[r][j] = (r == j ? 1.0 : 0.0) + scale * (double)J[j][r];
    double C[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) C[a][b] = F[0][a] * F[0][b] + F[1][a] * F[1][b] + F[2][a] * F[2][b];
    const double lam = lmax3_sym(C[0][0], C[0][1], C[0][2], C[1][1], C[1][2], C[2][2]);
    ftle[i] = log(sqrt(lam)) * inv_T;
  }
}

// 3D predicted end positions: out[i] = x0[i] + s * y[i] (FP64, n x 3; points n x 4).
__global__ void apply_displacement3_kernel(const double *__restrict__ pts,
                                           const float *__restrict__ y, int ldy, long long n,
                                           double scale, double *__restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int a = 0; a < 3; ++a) out[3 * i + a] = pts[4 * i + a] + scale * (double)y[i * ldy + a];
  }
}

inline int ew_blocks(long long n) {
  const long long b = (n + 255) / 256;
  const long long cap = (long long)kNumSMs * 16;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace mlp
}  // namespace ftle

using namespace ftle;
using namespace ftle::mlp;

namespace {

// cuTensorMapEncodeTiled through the runtime's driver entry point (the library does
// not link against libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  });
  return fn;
}

// 2D tensor map of a BF16 operand with `rows` rows (M or N) and K columns, read in the
// boxes gemm_bf16_kernel issues: K-major (element (r, k) at src[r*ld + k]) boxes of 8 k x
// R rows, MN-major (element (r, k) at src[k*ld + r]) boxes of 8 r x kChunkK k.
int operand_map(CUtensorMap *map, const void *src, bool trans, int rows, int K, int ld, int R) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return FTLE_ERR_CUDA;
  }
  cuuint64_t dims[2], strides[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2], elem[2] = {1, 1};
  if (!trans) {
    dims[0] = (cuuint64_t)K;
    dims[1] = (cuuint64_t)rows;
    box[0] = 8;
    box[1] = (cuuint32_t)R;
  } else {
    dims[0] = (cuuint64_t)rows;
    dims[1] = (cuuint64_t)K;
    box[0] = 8;
    box[1] = (cuuint32_t)kChunkK;
  }
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(src), dims,
                         strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d) for a %s operand of %d x %d, ld %d", (int)r,
              trans ? "MN-major" : "K-major", rows, K, ld);
    return FTLE_ERR_CUDA;
  }
  return FTLE_OK;
}

int gemm_launch(const void *A, int lda, int a_trans, const void *B, int ldb, int b_trans, int M,
                int N, int K, int splits, const Epi &epi, int32_t *error_word, void *stream) {
  if (!A || !B || !error_word) return fail_invalid("null operand");
  if (M <= 0 || N <= 0 || K <= 0) return fail_invalid("GEMM sizes must be positive");
  if (M % 8 || N % 8) return fail_invalid("M and N must be multiples of 8");
  if (K % kChunkK) return fail_invalid("K must be a multiple of 64");
  if (lda % 8 || ldb % 8) return fail_invalid("leading dimensions must be multiples of 8");
  if (reinterpret_cast<uintptr_t>(A) % 16 || reinterpret_cast<uintptr_t>(B) % 16)
    return fail_invalid("A and B must be 16-byte aligned");
  if (!a_trans && lda < K) return fail_invalid("lda < K");
  if (a_trans && lda < M) return fail_invalid("lda < M");
  if (!b_trans && ldb < K) return fail_invalid("ldb < K");
  if (b_trans && ldb < N) return fail_invalid("ldb < N");
  switch (epi.mode) {
    case EPI_F32:
    case EPI_BIAS_F32:
      if (!epi.c || epi.ldc < N || epi.ldc % 4 || reinterpret_cast<uintptr_t>(epi.c) % 16)
        return fail_invalid("C must be 16-byte aligned with ldc >= N and ldc %% 4 == 0");
      if (epi.mode == EPI_BIAS_F32 && !epi.bias) return fail_invalid("bias required");
      break;
    case EPI_BIAS_SILU:
      if (!epi.bias || !epi.hout) return fail_invalid("bias and activation output required");
      if (epi.zout && (epi.ldzout < N || epi.ldzout % 4 ||
                       reinterpret_cast<uintptr_t>(epi.zout) % 16))
        return fail_invalid("Z must be 16-byte aligned with ldz >= N and ldz %% 4 == 0");
      break;
    case EPI_DSILU:
      if (!epi.zin || !epi.hout) return fail_invalid("pre-activations and output required");
      if (epi.ldzin < N || epi.ldzin % 4 || reinterpret_cast<uintptr_t>(epi.zin) % 16)
        return fail_invalid("Z must be 16-byte aligned with ldz >= N and ldz %% 4 == 0");
      break;
    default:
      return fail_invalid("unknown epilogue %d", epi.mode);
  }
  if ((epi.mode == EPI_BIAS_SILU || epi.mode == EPI_DSILU) &&
      (epi.ldh < N || epi.ldh % 8 || reinterpret_cast<uintptr_t>(epi.hout) % 16))
    return fail_invalid("BF16 output must be 16-byte aligned with ldh >= N, ldh %% 8 == 0");
  const int NT = N >= kMaxNT ? kMaxNT : ((N + 15) / 16) * 16;
  const int kchunks = K / kChunkK;
  if (splits < 1) splits = 1;
  if (epi.mode != EPI_F32 && splits > 1) return fail_invalid("split-K needs the FP32 epilogue");
  if (splits > kchunks) splits = kchunks;
  const int k_per_split = ((kchunks + splits - 1) / splits) * kChunkK;
  splits = (K + k_per_split - 1) / k_per_split;
  Epi e = epi;
  if (splits > 1) e.accumulate = 1;
  const size_t smem = (size_t)kPStages * (kTileM + NT) * kChunkK * 2;
  const int tiles_m = (M + kTileM - 1) / kTileM, tiles_n = (N + NT - 1) / NT;
  const int total = tiles_m * tiles_n * splits;
  const int grid = total < 2 * kNumSMs ? total : 2 * kNumSMs;  // persistent: two CTAs per SM
  cudaStream_t st = as_stream(stream);
  CUtensorMap tmA, tmB;
  int rc = operand_map(&tmA, A, a_trans != 0, M, K, lda, kTileM);
  if (rc) return rc;
  rc = operand_map(&tmB, B, b_trans != 0, N, K, ldb, NT);
  if (rc) return rc;
#define GL(AT, BT)                                                                              \
  do {                                                                                          \
    cudaFuncSetAttribute(gemm_bf16_kernel<AT, BT>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                         (int)smem);                                                            \
    gemm_bf16_kernel<AT, BT>                                                                    \
        <<<grid, kGemmThreads, smem, st>>>(tmA, tmB, M, N, K, NT, k_per_split, tiles_m, splits, \
                                           total, e, error_word);                               \
  } while (0)
  if (!a_trans && !b_trans)
    GL(false, false);
  else if (!a_trans && b_trans)
    GL(false, true);
  else if (a_trans && !b_trans)
    GL(true, false);
  else
    GL(true, true);
#undef GL
  return check_launch("gemm_bf16_kernel");
}

}  // namespace

extern "C" {

int ftle_mlp_gemm(const void *A, int32_t lda, int32_t a_trans, const void *B, int32_t ldb,
                  int32_t b_trans, float *C, int32_t ldc, int32_t M, int32_t N, int32_t K,
                  int32_t splits, int32_t accumulate, int32_t *error_word, void *stream) {
  Epi e{};
  e.mode = EPI_F32;
  e.c = C;
  e.ldc = ldc;
  e.accumulate = accumulate;
  return gemm_launch(A, lda, a_trans, B, ldb, b_trans, M, N, K, splits, e, error_word, stream);
}

int ftle_mlp_linear(const void *X, int32_t ldx, const void *W, int32_t ldw, const float *bias,
                    int32_t M, int32_t N, int32_t K, int32_t activation, float *Z, int32_t ldz,
                    void *H, int32_t ldh, int32_t *error_word, void *stream) {
  Epi e{};
  if (activation) {
    e.mode = EPI_BIAS_SILU;
    e.bias = bias;
    e.zout = Z;
    e.ldzout = ldz;
    e.hout = static_cast<__nv_bfloat16 *>(H);
    e.ldh = ldh;
  } else {
    e.mode = EPI_BIAS_F32;
    e.bias = bias;
    e.c = Z;
    e.ldc = ldz;
  }
  return gemm_launch(X, ldx, 0, W, ldw, 0, M, N, K, 1, e, error_word, stream);
}

int ftle_mlp_gemm_dsilu(const void *A, int32_t lda, int32_t a_trans, const void *B, int32_t ldb,
                        int32_t b_trans, int32_t M, int32_t N, int32_t K, const float *Zin,
                        int32_t ldz, void *G, int32_t ldg, float *colsum, int32_t *error_word,
                        void *stream) {
  Epi e{};
  e.mode = EPI_DSILU;
  e.zin = Zin;
  e.ldzin = ldz;
  e.hout = static_cast<__nv_bfloat16 *>(G);
  e.ldh = ldg;
  e.colsum = colsum;
  return gemm_launch(A, lda, a_trans, B, ldb, b_trans, M, N, K, 1, e, error_word, stream);
}

int ftle_mlp_features(const double *points, int64_t n, const float *freq, int32_t num_freq,
                      void *features, void *tangent_x, void *tangent_y, void *stream) {
  if (n < 0 || num_freq <= 0) return fail_invalid("bad sizes");
  if (n == 0) return FTLE_OK;
  if (!points || !freq || !features) return fail_invalid("null pointer");
  if (reinterpret_cast<uintptr_t>(freq) % 16) return fail_invalid("freq must be 16-byte aligned");
  features_kernel<<<ew_blocks(n * num_freq), 256, 0, as_stream(stream)>>>(
      points, n, reinterpret_cast<const float4 *>(freq), num_freq,
      static_cast<__nv_bfloat16 *>(features), static_cast<__nv_bfloat16 *>(tangent_x),
      static_cast<__nv_bfloat16 *>(tangent_y));
  return check_launch("features_kernel");
}

int ftle_mlp_mse_grad(const float *y, int32_t ldy, const float *target, int32_t outs, int64_t n,
                      void *dy, int32_t lddy, float *dbias, float *loss, void *stream) {
  if (n <= 0 || outs <= 0 || outs > 4 || lddy < outs || ldy < outs)
    return fail_invalid("bad sizes");
  if (!y || !target || !dy || !dbias || !loss) return fail_invalid("null pointer");
  mse_grad_kernel<<<ew_blocks(n), 256, 0, as_stream(stream)>>>(
      y, ldy, target, outs, n, 1.0f / (float)n, static_cast<__nv_bfloat16 *>(dy), lddy, dbias,
      loss);
  return check_launch("mse_grad_kernel");
}

int ftle_mlp_adam(float *w, float *g, float *m, float *v, void *w_bf16, int64_t n, float lr,
                  float beta1, float beta2, float eps, int32_t step, float weight_decay,
                  void *stream) {
  if (n <= 0 || step < 1) return fail_invalid("bad sizes");
  if (!w || !g || !m || !v || !w_bf16) return fail_invalid("null pointer");
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  adam_kernel<<<ew_blocks(n), 256, 0, as_stream(stream)>>>(
      w, g, m, v, static_cast<__nv_bfloat16 *>(w_bf16), n, lr, beta1, beta2, eps, c1, c2,
      weight_decay);
  return check_launch("adam_kernel");
}

int ftle_mlp_jacobian_ftle(const float *jx, const float *jy, int32_t ld, int64_t n, double scale,
                           double T, double *ftle, void *stream) {
  if (n < 0 || ld < 2 || T == 0.0) return fail_invalid("bad sizes");
  if (n == 0) return FTLE_OK;
  if (!jx || !jy || !ftle) return fail_invalid("null pointer");
  jacobian_ftle_kernel<<<ew_blocks(n), 256, 0, as_stream(stream)>>>(jx, jy, ld, n, scale,
                                                                     1.0 / fabs(T), ftle);
  return check_launch("jacobian_ftle_kernel");
}

int ftle_mlp_apply_displacement(const double *points, const float *y, int32_t ldy, int64_t n,
                                double scale, double *out, void *stream) {
  if (n < 0 || ldy < 2) return fail_invalid("bad sizes");
  if (n == 0) return FTLE_OK;
  if (!points || !y || !out) return fail_invalid("null pointer");
  apply_displacement_kernel<<<ew_blocks(n), 256, 0, as_stream(stream)>>>(points, y, ldy, n, scale,
                                                                          out);
  return check_launch("apply_displacement_kernel");
}

int ftle_mlp_features3(const double *points, int64_t n, const float *freq, int32_t num_freq,
                       void *features, void *tangent_x, void *tangent_y, void *tangent_z,
                       void *stream) {
  if (n < 0 || num_freq <= 0) return fail_invalid("bad sizes");
  if (n == 0) return FTLE_OK;
  if (!points || !freq || !features) return fail_invalid("null pointer");
  if (reinterpret_cast<uintptr_t>(freq) % 16) return fail_invalid("freq must be 16-byte aligned");
  features3_kernel<<<ew_blocks(n * num_freq), 256, 0, as_stream(stream)>>>(
      points, n, reinterpret_cast<const float4 *>(freq), num_freq,
      static_cast<__nv_bfloat16 *>(features), static_cast<__nv_bfloat16 *>(tangent_x),
      static_cast<__nv_bfloat16 *>(tangent_y), static_cast<__nv_bfloat16 *>(tangent_z));
  return check_launch("features3_kernel");
}

int ftle_mlp_jacobian_ftle3(const float *jx, const float *jy, const float *jz, int32_t ld,
                            int64_t n, double scale, double T, double *ftle, void *stream) {
  if (n < 0 || ld < 3 || T == 0.0) return fail_invalid("bad sizes");
  if (n == 0) return FTLE_OK;
  if (!jx || !jy || !jz || !ftle) return fail_invalid("null pointer");
  jacobian_ftle3_kernel<<<ew_blocks(n), 256, 0, as_stream(stream)>>>(jx, jy, jz, ld, n, scale,
                                                                      1.0 / fabs(T), ftle);
  return check_launch("jacobian_ftle3_kernel");
}

int ftle_mlp_apply_displacement3(const double *points, const float *y, int32_t ldy, int64_t n,
                                 double scale, double *out, void *stream) {
  if (n < 0 || ldy < 3) return fail_invalid("bad sizes");
  if (n == 0) return FTLE_OK;
  if (!points || !y || !out) return fail_invalid("null pointer");
  apply_displacement3_kernel<<<ew_blocks(n), 256, 0, as_stream(stream)>>>(points, y, ldy, n,
                                                                           scale, out);
  return check_launch("apply_displacement3_kernel");
}

}  // extern "C"
