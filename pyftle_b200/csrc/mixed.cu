// mixed.cu -- mixed-precision FTLE window (sm_100a).
//
// Storage: 16-bit "pair records": record (s, node) holds the velocity of
// snapshot s and of its successor, so one 8-byte (2D) or 16-byte (3D) load per
// cell corner serves a time-blended gather.  Three encodings:
//   FTLE_F16 / FTLE_BF16  IEEE half / bfloat16 velocities;
//   FTLE_FX15             15-bit fixed point per component over the series'
//                         value range: one byte permute turns a value into the
//                         FP32 0.5 + q/65536, and u = scale*f + offset.
// A 256-byte header in front of the records holds scale/offset per component.
//
// Work unit: one thread advects one neighbour group in the split
// representation
//   centroid c           FP64 -> its cell index and in-cell fraction are exact
//   offsets  d_k = x_k-c FP32, advected with velocity differences u(c+d_k)-u(c)
// so x_R - x_L never cancels in FP32.  Per RK4 stage the thread gathers the
// centroid's cell once, turns its (time-blended) corners into the cell's
// multilinear polynomial, and evaluates every neighbour inside that cell as an
// exact polynomial *difference* p(f+delta) - p(f) (no FP32 cancellation).
// Neighbours that left the cell go through one shared gather loop.  The stage
// loop is a runtime loop so the kernel body stays small (instruction-cache
// resident).  Jacobian -> Cauchy-Green -> lambda_max runs in FP64
// (ftle.py:9-233 restated).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <math.h>

#include "common.cuh"

namespace ftle {

constexpr int kHeaderBytes = 256;
constexpr int kFxMax = 32767;  // 15-bit fixed point

struct Header16 {
  float scale[4];
  float offset[4];
  float vmin[4];
  float vmax[4];
};

// ---------------------------------------------------------------------------
// decoding two 16-bit values held in one 32-bit word
// ---------------------------------------------------------------------------
template <int STORAGE>
struct Dec;

template <>
struct Dec<FTLE_F16> {
  static __device__ __forceinline__ float lo(unsigned w) {
    return __half2float(__ushort_as_half((unsigned short)(w & 0xffffu)));
  }
  static __device__ __forceinline__ float hi(unsigned w) {
    return __half2float(__ushort_as_half((unsigned short)(w >> 16)));
  }
  static __device__ __forceinline__ unsigned short enc(double x, const Header16 &) {
    return __half_as_ushort(__double2half(x));
  }
};

template <>
struct Dec<FTLE_BF16> {
  static __device__ __forceinline__ float lo(unsigned w) { return __uint_as_float(w << 16); }
  static __device__ __forceinline__ float hi(unsigned w) {
    return __uint_as_float(w & 0xffff0000u);
  }
  static __device__ __forceinline__ unsigned short enc(double x, const Header16 &) {
    return __bfloat16_as_ushort(__double2bfloat16(x));
  }
};

// bits 0x3F000000 | q << 8 is the float 0.5 + q/65536 for q < 2^15
template <>
struct Dec<FTLE_FX15> {
  static __device__ __forceinline__ float lo(unsigned w) {
    return __uint_as_float(__byte_perm(w, 0x3F000000u, 0x7104));
  }
  static __device__ __forceinline__ float hi(unsigned w) {
    return __uint_as_float(__byte_perm(w, 0x3F000000u, 0x7324));
  }
  static __device__ __forceinline__ unsigned short enc(double x, const Header16 &h) = delete;
};

// ---------------------------------------------------------------------------
// packing (S, dim, nodes) float64 -> header + pair records
// ---------------------------------------------------------------------------

// Float min/max through integer atomics: a float with the sign bit clear orders like
// its bits as a signed int, one with the sign bit set orders reversed as unsigned.
// The branch tests the sign BIT, so -0.0 takes the negative path (as a signed int its
// bits are INT_MIN and would replace any true negative minimum).
__device__ __forceinline__ void atomic_min_f(float *a, float v) {
  if (__float_as_int(v) >= 0)
    atomicMin(reinterpret_cast<int *>(a), __float_as_int(v));
  else
    atomicMax(reinterpret_cast<unsigned *>(a), __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_f(float *a, float v) {
  if (__float_as_int(v) >= 0)
    atomicMax(reinterpret_cast<int *>(a), __float_as_int(v));
  else
    atomicMin(reinterpret_cast<unsigned *>(a), __float_as_uint(v));
}

__global__ void header_init_kernel(Header16 *h) {
  const int c = threadIdx.x;
  if (c < 4) {
    h->scale[c] = 1.0f;
    h->offset[c] = 0.0f;
    h->vmin[c] = __int_as_float(0x7f800000);   // +inf
    h->vmax[c] = __int_as_float(0xff800000);   // -inf
  }
}

// per-component min / max over every snapshot and node
template <int DIM>
__global__ void minmax_kernel(const double *__restrict__ src, long long nodes, int S, Header16 *h) {
  float mn[DIM], mx[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    mn[c] = __int_as_float(0x7f800000);
    mx[c] = __int_as_float(0xff800000);
  }
  const long long total = nodes * S;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long s = i / nodes, p = i - s * nodes;
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      const double v = src[(s * DIM + c) * nodes + p];
      mn[c] = fminf(mn[c], __double2float_rd(v));
      mx[c] = fmaxf(mx[c], __double2float_ru(v));
    }
  }
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    for (int o = 16; o > 0; o >>= 1) {
      mn[c] = fminf(mn[c], __shfl_xor_sync(0xffffffffu, mn[c], o));
      mx[c] = fmaxf(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomic_min_f(&h->vmin[c], mn[c]);
      atomic_max_f(&h->vmax[c], mx[c]);
    }
  }
}

// u = scale * (0.5 + q/65536) + offset  with  q = (v - vmin) / step,  step = range / 32767
__global__ void fx_finalize_kernel(Header16 *h, int dim) {
  const int c = threadIdx.x;
  if (c < dim) {
    const double range = (double)h->vmax[c] - (double)h->vmin[c];
    const double step = range > 0.0 ? range / kFxMax : 0.0;
    const double S = 65536.0 * step;
    h->scale[c] = (float)S;
    h->offset[c] = (float)((double)h->vmin[c] - 0.5 * S);
  }
}

// FX16: the FX15 decoder's byte permute turns the full 16-bit code q into
//   f(q) = 0.5 + q/65536             for q <= 32768
//   f(q) = 1 + (q - 32768)/32768     for q >= 32768  (bit 15 of q lands on the exponent)
// so the range [vmin, vmax] maps onto [0.5, kFx16Top] with u = scale*f + offset.
constexpr double kFx16Top = 2.0 - 1.0 / 32768.0;

__global__ void fx16_finalize_kernel(Header16 *h, int dim) {
  const int c = threadIdx.x;
  if (c < dim) {
    const double range = (double)h->vmax[c] - (double)h->vmin[c];
    const double S = range > 0.0 ? range / (kFx16Top - 0.5) : 0.0;
    h->scale[c] = (float)S;
    h->offset[c] = (float)((double)h->vmin[c] - 0.5 * S);
  }
}

template <int STORAGE>
__device__ __forceinline__ unsigned short encode(double v, const Header16 &h, int c) {
  if constexpr (STORAGE == FTLE_FX16) {
    // the code whose decoded value (with the header's FP32 scale / offset) is nearest
    const double S = (double)h.scale[c];
    if (!(S > 0.0)) return 0;
    const double f = (v - (double)h.offset[c]) / S;
    double q = f <= 1.0 ? rint((f - 0.5) * 65536.0) : 32768.0 + rint((f - 1.0) * 32768.0);
    q = q < 0.0 ? 0.0 : (q > 65535.0 ? 65535.0 : q);
    return (unsigned short)q;
  } else if constexpr (STORAGE == FTLE_FX15) {
    const double range = (double)h.vmax[c] - (double)h.vmin[c];
    double q = range > 0.0 ? rint((v - (double)h.vmin[c]) * (kFxMax / range)) : 0.0;
    q = q < 0.0 ? 0.0 : (q > kFxMax ? kFxMax : q);
    return (unsigned short)q;
  } else {
    return Dec<STORAGE>::enc(v, h);
  }
}

template <int DIM, int STORAGE>
__global__ void pack16_kernel(const double *__restrict__ src, long long nodes, int S,
                              int periodic_time, const Header16 *__restrict__ hdr,
                              unsigned char *recs) {
  const Header16 h = *hdr;
  const long long total = nodes * S;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(i / nodes);
    const long long p = i - (long long)s * nodes;
    const int s1 = (s + 1 < S) ? s + 1 : (periodic_time ? 0 : s);
    unsigned short a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      a[c] = encode<STORAGE>(src[((long long)s * DIM + c) * nodes + p], h, c);
      b[c] = encode<STORAGE>(src[((long long)s1 * DIM + c) * nodes + p], h, c);
    }
    if constexpr (DIM == 2) {
      uint2 v;
      v.x = (unsigned)a[0] | ((unsigned)a[1] << 16);
      v.y = (unsigned)b[0] | ((unsigned)b[1] << 16);
      reinterpret_cast<uint2 *>(recs)[i] = v;
    } else {
      uint4 v;
      v.x = (unsigned)a[0] | ((unsigned)a[1] << 16);
      v.y = (unsigned)a[2];
      v.z = (unsigned)b[0] | ((unsigned)b[1] << 16);
      v.w = (unsigned)b[2];
      reinterpret_cast<uint4 *>(recs)[i] = v;
    }
  }
}

template <int DIM, int STORAGE>
static int pack16(int64_t nodes, int32_t S, int32_t periodic_time, const double *src, void *dst,
                  cudaStream_t st) {
  Header16 *h = static_cast<Header16 *>(dst);
  unsigned char *recs = static_cast<unsigned char *>(dst) + kHeaderBytes;
  header_init_kernel<<<1, 32, 0, st>>>(h);
  if constexpr (STORAGE == FTLE_FX15 || STORAGE == FTLE_FX16) {
    minmax_kernel<DIM><<<grid_blocks(nodes * S, 256), 256, 0, st>>>(src, nodes, S, h);
    if constexpr (STORAGE == FTLE_FX15)
      fx_finalize_kernel<<<1, 32, 0, st>>>(h, DIM);
    else
      fx16_finalize_kernel<<<1, 32, 0, st>>>(h, DIM);
  }
  pack16_kernel<DIM, STORAGE><<<grid_blocks(nodes * S, 256), 256, 0, st>>>(src, nodes, S,
                                                                           periodic_time, h, recs);
  return check_launch("pack16_kernel");
}

int pack_snapshots_16(int32_t dim, int64_t nodes, int32_t num_snapshots, int32_t periodic_time,
                      const double *src, int32_t storage, void *dst, void *stream) {
  cudaStream_t st = as_stream(stream);
#define P16(D, S) return pack16<D, S>(nodes, num_snapshots, periodic_time, src, dst, st)
  if (dim == 2) {
    if (storage == FTLE_F16) P16(2, FTLE_F16);
    if (storage == FTLE_BF16) P16(2, FTLE_BF16);
    if (storage == FTLE_FX16) P16(2, FTLE_FX16);
    P16(2, FTLE_FX15);
  } else {
    if (storage == FTLE_F16) P16(3, FTLE_F16);
    if (storage == FTLE_BF16) P16(3, FTLE_BF16);
    if (storage == FTLE_FX16) P16(3, FTLE_FX16);
    P16(3, FTLE_FX15);
  }
#undef P16
}

// ---------------------------------------------------------------------------
// window kernel
// ---------------------------------------------------------------------------

constexpr int kBlock = 128;

struct MixK {
  WinK w;
  double inv_sp[3];   // 1/spacing
  double org_sp[3];   // origin/spacing: p = x*inv_sp - org_sp
  double period[3];   // n*spacing (periodic grids)
  float inv_spf[3];
  int stride[3];      // node-index stride per axis (2D: 1, nx; 3D: nz, nx*nz, 1)
  double inv_dt;
  double inv_S;       // 1/num_snapshots
};

// Per-window values (one window: taken from MixK; a batch: one entry per window).
struct WinVar {
  double t0, h, map_period;
  double *positions;
  double *ftle;
  long long N;
  int num_steps, first_snapshot;
  int keep_positions;
  int reserved;
};

__device__ __forceinline__ WinVar winvar_of(const MixK &m) {
  WinVar v;
  v.t0 = m.w.t0;
  v.h = m.w.h;
  v.map_period = m.w.map_period;
  v.positions = m.w.positions;
  v.ftle = m.w.ftle;
  v.N = m.w.N;
  v.num_steps = m.w.num_steps;
  v.first_snapshot = m.w.first_snapshot;
  v.keep_positions = m.w.keep_positions;
  v.reserved = 0;
  return v;
}

__device__ __forceinline__ float lerpf(float a, float b, float t) { return fmaf(t, b - a, a); }

// Wrap a cell index into [0, n): one conditional step covers every index
// within one period of the grid (the centroid is kept in the primary period).
__device__ __forceinline__ int wrap_near(int q, int n) {
  if (q < 0)
    q += n;
  else if (q >= n)
    q -= n;
  if ((unsigned)q >= (unsigned)n) q = wrap_index(q, n);
  return q;
}

// ---------------------------------------------------------------------------
// packed FP32 (sm_100 FFMA2 / FADD2 / FMUL2): two lanes of one 64-bit register pair
// per instruction, each lane rounded exactly like the scalar fmaf / add / mul, so
// a pair computes the same bits as two scalar operations.  Pairs are the (u, v)
// velocity components of a corner or polynomial, or the same component of two
// neighbours of a group (neighbours 2p and 2p+1, which share the centroid's cell).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  return __fadd2_rn(a, make_float2(-b.x, -b.y));  // a + (-b) rounds as a - b
}
__device__ __forceinline__ float2 lerp2(float2 a, float2 b, float2 t) { return fma2(t, sub2(b, a), a); }

__device__ __forceinline__ float vsub(float a, float b) { return a - b; }
__device__ __forceinline__ float2 vsub(float2 a, float2 b) { return sub2(a, b); }
__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return fma2(a, b, c); }

// Time-blended corner values of one cell, corner q = x + 2y (+ 4z): (u, v) paired, w apart.
template <int DIM>
struct CellVals {
  float2 uv[1 << DIM];
  float w[DIM == 3 ? 8 : 1];
};

// Corner values of the cell whose lower corner is `cell`; false if the cell is
// outside a non-periodic grid.
template <int DIM, int STORAGE, bool BLEND>
__device__ __forceinline__ bool cell_values(const MixK &m, const unsigned char *__restrict__ recs,
                                            float alpha, const int *cell, CellVals<DIM> &v) {
  const GridK &g = m.w.g;
  int base = 0, step[DIM];
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    int lo = cell[a];
    step[a] = m.stride[a];
    if (g.periodic) {
      lo = wrap_near(lo, g.n[a]);
      if (lo + 1 == g.n[a]) step[a] = -(g.n[a] - 1) * m.stride[a];
    } else if (lo < 0 || lo > g.n[a] - 2) {
      return false;
    }
    base += lo * m.stride[a];
  }
  const float2 a2 = bc2(alpha);
#pragma unroll
  for (int q = 0; q < (1 << DIM); ++q) {
    int idx = base;
    if (q & 1) idx += step[0];
    if (q & 2) idx += step[1];
    if constexpr (DIM == 3) {
      if (q & 4) idx += step[2];
    }
    if constexpr (DIM == 2) {
      const uint2 r = __ldg(reinterpret_cast<const uint2 *>(recs) + idx);
      const float2 f0 = make_float2(Dec<STORAGE>::lo(r.x), Dec<STORAGE>::hi(r.x));
      if constexpr (BLEND) {
        v.uv[q] = lerp2(f0, make_float2(Dec<STORAGE>::lo(r.y), Dec<STORAGE>::hi(r.y)), a2);
      } else {
        v.uv[q] = f0;
      }
    } else {
      const uint4 r = __ldg(reinterpret_cast<const uint4 *>(recs) + idx);
      const float2 f0 = make_float2(Dec<STORAGE>::lo(r.x), Dec<STORAGE>::hi(r.x));
      const float w0 = Dec<STORAGE>::lo(r.y);
      if constexpr (BLEND) {
        v.uv[q] = lerp2(f0, make_float2(Dec<STORAGE>::lo(r.z), Dec<STORAGE>::hi(r.z)), a2);
        v.w[q] = lerpf(w0, Dec<STORAGE>::lo(r.w), alpha);
      } else {
        v.uv[q] = f0;
        v.w[q] = w0;
      }
    }
  }
  return true;
}

// multilinear interpolation by lerps (x, then y, then z) of the (u, v) pair
template <int DIM>
__device__ __forceinline__ float2 interp_lerp_uv(const float2 *v, const float *f) {
  const float2 f0 = bc2(f[0]), f1 = bc2(f[1]);
  const float2 x0 = lerp2(v[0], v[1], f0);
  const float2 x1 = lerp2(v[2], v[3], f0);
  const float2 y0 = lerp2(x0, x1, f1);
  if constexpr (DIM == 2) {
    return y0;
  } else {
    const float2 x2 = lerp2(v[4], v[5], f0);
    const float2 x3 = lerp2(v[6], v[7], f0);
    return lerp2(y0, lerp2(x2, x3, f1), bc2(f[2]));
  }
}

// ... and of a single component (w in 3D)
__device__ __forceinline__ float interp_lerp3(const float *v, const float *f) {
  const float x0 = lerpf(v[0], v[1], f[0]);
  const float x1 = lerpf(v[2], v[3], f[0]);
  const float y0 = lerpf(x0, x1, f[1]);
  const float x2 = lerpf(v[4], v[5], f[0]);
  const float x3 = lerpf(v[6], v[7], f[0]);
  return lerpf(y0, lerpf(x2, x3, f[1]), f[2]);
}

// p(x) = a0 + a1 x + a2 y (+ a3 z) + a4 xy + a5 xz + a6 yz + a7 xyz  (2D: a0 a1 a2 a3=xy),
// for one component (T = float) or the (u, v) pair (T = float2)
template <int DIM, typename T>
__device__ __forceinline__ void poly_setup(const T *v, T *A) {
  if constexpr (DIM == 2) {
    A[0] = v[0];
    A[1] = vsub(v[1], v[0]);
    A[2] = vsub(v[2], v[0]);
    A[3] = vsub(vsub(v[3], v[2]), vsub(v[1], v[0]));
  } else {
    A[0] = v[0];
    A[1] = vsub(v[1], v[0]);
    A[2] = vsub(v[2], v[0]);
    A[3] = vsub(v[4], v[0]);
    A[4] = vsub(vsub(v[3], v[1]), A[2]);
    A[5] = vsub(vsub(v[5], v[1]), A[3]);
    A[6] = vsub(vsub(v[6], v[2]), A[3]);
    A[7] = vsub(vsub(vsub(v[7], v[6]), vsub(v[5], v[4])), vsub(vsub(v[3], v[2]), vsub(v[1], v[0])));
  }
}

// p(f), with f given per axis as T (a pair holds the same coordinate twice)
template <int DIM, typename T>
__device__ __forceinline__ T poly_eval(const T *A, const T *f) {
  if constexpr (DIM == 2) {
    return vfma(f[0], vfma(f[1], A[3], A[1]), vfma(f[1], A[2], A[0]));
  } else {
    const T x = f[0], y = f[1], z = f[2];
    const T t1 = vfma(z, A[7], A[4]);
    const T t3 = vfma(z, A[5], vfma(y, t1, A[1]));
    const T t4 = vfma(z, A[6], A[2]);
    return vfma(z, A[3], vfma(y, t4, vfma(x, t3, A[0])));
  }
}

// p(f + d) - p(f) of one component for two neighbours at once (F = f + d), written
// so that no large terms cancel.  `g` is the part that depends on the centroid's f
// only: 3D gz = x (a7 y + a5) + a6 y + a3, 2D gy = a3 x + a2.
//   3D: dx (a1 + a4 Y + a5 Z + a7 Y Z) + dy (a2 + a4 x + a6 Z + a7 x Z) + dz gz
//   2D: dx (a1 + a3 Y) + dy gy
template <int DIM>
__device__ __forceinline__ float2 poly_diff_pair(const float *A, float x, float g, const float2 *F,
                                                 const float2 *d) {
  if constexpr (DIM == 2) {
    return fma2(d[0], fma2(bc2(A[3]), F[1], bc2(A[1])), mul2(d[1], bc2(g)));
  } else {
    const float2 Y = F[1], Z = F[2];
    const float2 t = fma2(bc2(A[7]), Z, bc2(A[4]));
    const float2 gx = fma2(Y, t, fma2(bc2(A[5]), Z, bc2(A[1])));
    const float2 gy = fma2(bc2(x), t, fma2(bc2(A[6]), Z, bc2(A[2])));
    return fma2(d[0], gx, fma2(d[1], gy, mul2(d[2], bc2(g))));
  }
}

template <int DIM, int MODE>
__device__ __forceinline__ const unsigned char *record_set(const MixK &m, int first_snapshot,
                                                           int step, double t, float &alpha) {
  const long long rec_bytes = DIM == 2 ? 8 : 16;
  const unsigned char *base = static_cast<const unsigned char *>(m.w.snaps) + kHeaderBytes;
  int s;
  if constexpr (MODE == FTLE_HOLD) {
    s = first_snapshot + step;
    if (m.w.periodic_time) s %= m.w.num_snaps;
    alpha = 0.0f;
  } else {
    double tau = (t - m.w.snap_t0) * m.inv_dt;
    const int S = m.w.num_snaps;
    if (m.w.periodic_time) {
      tau = tau - (double)S * floor(tau * m.inv_S);
      s = (int)floor(tau);
      s = s >= S ? S - 1 : (s < 0 ? 0 : s);
      alpha = (float)(tau - (double)s);
    } else if (!(tau > 0.0)) {
      s = 0;
      alpha = 0.0f;
    } else if (tau >= (double)(S - 1)) {
      s = S - 2;
      alpha = 1.0f;
    } else {
      s = (int)floor(tau);
      alpha = (float)(tau - (double)s);
    }
  }
  return base + (long long)s * m.w.g.nodes * rec_bytes;
}

__device__ __forceinline__ int plus_r(int j) { return j == 0 ? 1 : 2 * j; }
__device__ __forceinline__ int minus_r(int j) { return j == 0 ? 0 : 2 * j + 1; }

__device__ __forceinline__ double lmax2(double F00, double F01, double F10, double F11) {
  const double A = F00 * F00 + F10 * F10;
  const double B = F00 * F01 + F10 * F11;
  const double C = F01 * F00 + F11 * F10;
  const double D = F01 * F01 + F11 * F11;
  const double trace = A + D;
  const double det = A * D - B * C;
  const double s = sqrt(trace * trace - 4.0 * det);
  const double l1 = 0.5 * (trace + s);
  const double l2 = 0.5 * (trace - s);
  return (l2 > l1) ? l2 : l1;
}


// Off-cell neighbour work items of one warp.  An item is the slot index of the
// owning thread's neighbour (its in-cell coordinates F relative to the owner's
// centroid cell wait in that slot); the owners' centroid cells sit beside it.
template <int DIM>
struct WarpQueue {
  static constexpr int kCap = 32 * 2 * DIM;
  int dst[kCap];
  int ci[DIM][32];  // centroid cell of each lane's group
};

// Per stage: centroid velocity uc and, in place of the previous stage's kd, the
// differences kd[p][a] = u(c + d_k + as*kd_k) - uc for the neighbour pair
// k = 2p, 2p+1 (lanes .x, .y).  Neighbours inside the centroid's cell use the
// cell polynomial; the others are queued per warp and gathered 32 at a time, so
// no lane idles in a divergent loop.  `dpl`: this thread's offsets in shared
// memory, float2 planes (neighbour pair p, axis a) at stride kBlock.
template <int DIM, int STORAGE, bool BLEND>
__device__ __forceinline__ void eval_group(const MixK &m, const Header16 &hd,
                                           const unsigned char *__restrict__ recs, float alpha,
                                           const double *cs, const float2 *dpl,
                                           float2 (*kd)[DIM], float as, float *uc,
                                           float *slots_base, WarpQueue<DIM> &wq, int lane) {
  constexpr int K = 2 * DIM;
  constexpr int NC = 1 << DIM;
  constexpr bool FX = STORAGE == FTLE_FX15;
  float *slots = slots_base + threadIdx.x;
  int ci[DIM];
  float fc[DIM];
  bool ok = true;
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    const double p = fma(cs[a], m.inv_sp[a], -m.org_sp[a]);
    const double fl = floor(p);
    ok = ok && fabs(fl) < 1.0e9;
    ci[a] = ok ? (int)fl : 0;
    fc[a] = ok ? (float)(p - fl) : 0.0f;
  }
  float2 fcb[DIM];
#pragma unroll
  for (int a = 0; a < DIM; ++a) fcb[a] = bc2(fc[a]);
  // the centroid cell's polynomial: (u, v) paired, w apart
  float2 Auv[NC];
  float Aw[NC];  // w (3D only)
  bool cin;
  {
    CellVals<DIM> v;
    cin = ok && cell_values<DIM, STORAGE, BLEND>(m, recs, alpha, ci, v);
    poly_setup<DIM>(v.uv, Auv);
    if constexpr (DIM == 3) poly_setup<DIM>(v.w, Aw);
  }
  {
    float2 puv = poly_eval<DIM>(Auv, fcb);
    if constexpr (FX)
      puv = fma2(make_float2(hd.scale[0], hd.scale[1]), puv,
                 make_float2(hd.offset[0], hd.offset[1]));
    uc[0] = cin ? puv.x : 0.0f;
    uc[1] = cin ? puv.y : 0.0f;
    if constexpr (DIM == 3) {
      const float pw = poly_eval<DIM>(Aw, fc);
      uc[2] = cin ? (FX ? fmaf(hd.scale[2], pw, hd.offset[2]) : pw) : 0.0f;
    }
  }
  // the part of p(f + d) - p(f) that depends on the centroid only, per component
  float g[DIM];
  if constexpr (DIM == 2) {
    const float2 gp = fma2(Auv[3], fcb[0], Auv[2]);
    g[0] = gp.x;
    g[1] = gp.y;
  } else {
    const float2 gp = fma2(fcb[0], fma2(Auv[7], fcb[1], Auv[5]), fma2(Auv[6], fcb[1], Auv[3]));
    g[0] = gp.x;
    g[1] = gp.y;
    g[2] = fmaf(fc[0], fmaf(Aw[7], fc[1], Aw[5]), fmaf(Aw[6], fc[1], Aw[3]));
  }
  // pass 1: every neighbour through the cell polynomial, two at a time; flag those
  // outside the cell
  unsigned off = 0;
  const float2 as2 = bc2(as);
#pragma unroll
  for (int p = 0; p < DIM; ++p) {
    float2 dl[DIM], F[DIM];
    bool same0 = true, same1 = true;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      // explicit roundings: the cell test and the polynomial use the same F and dl
      dl[a] = mul2(fma2(as2, kd[p][a], dpl[(p * DIM + a) * kBlock]), bc2(m.inv_spf[a]));
      F[a] = add2(fcb[a], dl[a]);
      same0 = same0 && F[a].x >= 0.0f && F[a].x < 1.0f;
      same1 = same1 && F[a].y >= 0.0f && F[a].y < 1.0f;
    }
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      float Ac[NC];
#pragma unroll
      for (int i = 0; i < NC; ++i) Ac[i] = c == 0 ? Auv[i].x : (c == 1 ? Auv[i].y : Aw[i]);
      float2 dp = poly_diff_pair<DIM>(Ac, fc[0], g[c], F, dl);
      if constexpr (FX) dp = mul2(bc2(hd.scale[c]), dp);
      kd[p][c] = make_float2(cin ? dp.x : 0.0f, cin ? dp.y : 0.0f);
    }
    const int k0 = 2 * p, k1 = 2 * p + 1;
    // 2D stores every neighbour's F without a branch (most warps have an off-cell
    // neighbour in most stages); 3D stores only the off-cell ones (measured faster)
    if constexpr (DIM == 2) {
      off |= (!same0 && ok) ? 1u << k0 : 0u;
      off |= (!same1 && ok) ? 1u << k1 : 0u;
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        slots[(k0 * DIM + a) * kBlock] = F[a].x;
        slots[(k1 * DIM + a) * kBlock] = F[a].y;
      }
    } else {
      if (!same0 && ok) {
        off |= 1u << k0;
#pragma unroll
        for (int a = 0; a < DIM; ++a) slots[(k0 * DIM + a) * kBlock] = F[a].x;
      }
      if (!same1 && ok) {
        off |= 1u << k1;
#pragma unroll
        for (int a = 0; a < DIM; ++a) slots[(k1 * DIM + a) * kBlock] = F[a].y;
      }
    }
  }
  if constexpr (DIM == 2) {
    if (!__any_sync(0xffffffffu, off != 0u)) return;
  }
  // pass 2: queue the off-cell neighbours of the whole warp.  2D queues them neighbour
  // by neighbour (every lane's neighbour 0, then every lane's neighbour 1, ...: the
  // same neighbour of Morton-adjacent groups mostly lies in the same cell, so a gather
  // pass's loads share lines; measured +2.3 % on the 2D batch), 3D lane by lane (the
  // neighbour order measured 0.5 % slower there).  Same items either way, same bits.
  int total;
  if constexpr (DIM == 2) {
    const unsigned lt = (1u << lane) - 1u;
    unsigned bal[K];
    int start[K];
    total = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      bal[k] = __ballot_sync(0xffffffffu, (off >> k) & 1u);
      start[k] = total;
      total += __popc(bal[k]);
    }
    if (total == 0) return;  // warp-uniform
    __syncwarp();  // every lane has read its slots of the previous stage
#pragma unroll
    for (int a = 0; a < DIM; ++a) wq.ci[a][lane] = ci[a];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (off & (1u << k))
        wq.dst[start[k] + __popc(bal[k] & lt)] = k * DIM * kBlock + (int)threadIdx.x;
    }
  } else {
    const int cnt = __popc(off);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) return;  // warp-uniform
    __syncwarp();  // every lane has read its slots of the previous stage
    int pos = incl - cnt;
#pragma unroll
    for (int a = 0; a < DIM; ++a) wq.ci[a][lane] = ci[a];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (off & (1u << k)) wq.dst[pos++] = k * DIM * kBlock + (int)threadIdx.x;
    }
  }
  __syncwarp();
  // pass 3: 32 queued gathers at a time (a group whose centroid is not finite queues
  // nothing, so every item belongs to a valid group)
  for (int b = 0; b < total; b += 32) {
    const int it = b + lane;
    if (it < total) {
      const int dst = wq.dst[it];
      const int owner = dst & 31;  // the owner's lane (blocks are whole warps)
      int cell[DIM];
      float q[DIM];
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        const float F = slots_base[dst + a * kBlock];
        const float fo = floorf(F);
        cell[a] = wq.ci[a][owner] + (int)fo;
        q[a] = F - fo;
      }
      CellVals<DIM> v;
      const bool kin = cell_values<DIM, STORAGE, BLEND>(m, recs, alpha, cell, v);
      float2 puv = interp_lerp_uv<DIM>(v.uv, q);
      if constexpr (FX)
        puv = fma2(make_float2(hd.scale[0], hd.scale[1]), puv,
                   make_float2(hd.offset[0], hd.offset[1]));
      slots_base[dst] = kin ? puv.x : 0.0f;
      slots_base[dst + kBlock] = kin ? puv.y : 0.0f;
      if constexpr (DIM == 3) {
        const float pw = interp_lerp3(v.w, q);
        slots_base[dst + 2 * kBlock] = kin ? (FX ? fmaf(hd.scale[2], pw, hd.offset[2]) : pw) : 0.0f;
      }
    }
  }
  __syncwarp();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if constexpr (DIM == 2) {
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        const float sv = slots[(k * DIM + c) * kBlock] - uc[c];
        float &r = (k & 1) ? kd[k >> 1][c].y : kd[k >> 1][c].x;
        r = (off & (1u << k)) ? sv : r;
      }
    } else if (off & (1u << k)) {
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        float &r = (k & 1) ? kd[k >> 1][c].y : kd[k >> 1][c].x;
        r = slots[(k * DIM + c) * kBlock] - uc[c];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// per-group state and the step loop
// ---------------------------------------------------------------------------

template <int DIM>
struct GroupState {
  double c[DIM];            // centroid (periodic grids: inside the primary period)
  int wraps[DIM];           // periods removed from the centroid
  float d[2 * DIM][DIM];    // neighbour offsets (in shared memory during the step loop)
  float kcp[DIM];           // AB2: previous centroid velocity
  float kdp[2 * DIM][DIM];  // AB2: previous velocity differences
};

// Centroid = mean of the K neighbours (particles.py:235-236); offsets relative to it.
template <int DIM>
__device__ __forceinline__ void group_from_positions(const MixK &m, const WinVar &v, long long g,
                                                     GroupState<DIM> &st) {
  constexpr int K = 2 * DIM;
  const long long N = v.N;
  double X[K][DIM];
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int a = 0; a < DIM; ++a) X[k][a] = v.positions[((long long)k * N + g) * DIM + a];
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    double s = X[0][a];
#pragma unroll
    for (int k = 1; k < K; ++k) s += X[k][a];
    st.c[a] = s / (double)K;
  }
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      st.d[k][a] = (float)(X[k][a] - st.c[a]);
      st.kdp[k][a] = 0.0f;
    }
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    st.kcp[a] = 0.0f;
    st.wraps[a] = 0;
    if (m.w.g.periodic) {
      const double w = floor((st.c[a] - m.w.g.origin[a]) / m.period[a]);
      if (fabs(w) < 1.0e9) {
        st.wraps[a] = (int)w;
        st.c[a] -= w * m.period[a];
      }
    }
  }
}

// Advect one group through steps [i0, i1) of the window.  The neighbour offsets
// (dpl) and the RK4 accumulators (accp) live in this thread's shared-memory
// columns as float2 planes (neighbour pair p = k/2, axis a) at stride kBlock.
template <int DIM, int MODE, int INTEG, int STORAGE>
__device__ __forceinline__ void group_advect(const MixK &m, const WinVar &v, const Header16 &hd,
                                             GroupState<DIM> &st, int i0, int i1,
                                             float *smem_slots, float2 *accp, float2 *dpl,
                                             WarpQueue<DIM> &wq, int lane) {
  constexpr bool BLEND = MODE == FTLE_BLEND;
  const bool periodic = m.w.g.periodic != 0;
  const double h = v.h;
  const float hf = (float)h;
  float kc[DIM], accc[DIM];
  float2 kd[DIM][DIM];  // [pair][axis]
#pragma unroll
  for (int a = 0; a < DIM; ++a) kc[a] = 0.0f;
#pragma unroll
  for (int p = 0; p < DIM; ++p)
#pragma unroll
    for (int a = 0; a < DIM; ++a) kd[p][a] = make_float2(0.0f, 0.0f);
  // the offsets live in shared memory during the step loop, which frees 3*K
  // registers (the kernel then fits 4 blocks per SM)
#pragma unroll
  for (int p = 0; p < DIM; ++p)
#pragma unroll
    for (int a = 0; a < DIM; ++a)
      dpl[(p * DIM + a) * kBlock] = make_float2(st.d[2 * p][a], st.d[2 * p + 1][a]);

  constexpr int NST = INTEG == FTLE_RK4 ? 4 : 1;
  for (int i = i0; i < i1; ++i) {
    const double t = v.t0 + (double)i * h;
#pragma unroll 1
    for (int s = 0; s < NST; ++s) {
      // RK4 tableau: stage point x + a*k_prev, weight w, time t + tc*h
      const float tc = (s == 0) ? 0.0f : (s == 3 ? 1.0f : 0.5f);
      const float as = tc * hf;
      const float ws = (s == 0 || s == 3) ? 1.0f : 2.0f;
      float alpha;
      const unsigned char *recs =
          record_set<DIM, MODE>(m, v.first_snapshot, i, t + (double)tc * h, alpha);
      double cs[DIM];
#pragma unroll
      for (int a = 0; a < DIM; ++a) cs[a] = fma((double)tc * h, (double)kc[a], st.c[a]);
      float uc[DIM];
      eval_group<DIM, STORAGE, BLEND>(m, hd, recs, alpha, cs, dpl, kd, as, uc, smem_slots, wq,
                                      lane);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        kc[a] = uc[a];
        accc[a] = s == 0 ? uc[a] : fmaf(ws, uc[a], accc[a]);
      }
      if constexpr (INTEG == FTLE_RK4) {
        // stages 1-3 keep the running sum in shared memory; the last stage's k4 goes
        // straight into the step update below (no store and reload of the sum)
        if (s < 3) {
          const float2 ws2 = bc2(ws);
#pragma unroll
          for (int p = 0; p < DIM; ++p)
#pragma unroll
            for (int a = 0; a < DIM; ++a) {
              float2 &r = accp[(p * DIM + a) * kBlock];
              r = s == 0 ? kd[p][a] : fma2(ws2, kd[p][a], r);
            }
        }
      }
    }
    if constexpr (INTEG == FTLE_RK4) {
      const double h6 = h / 6.0;
      const float2 h6f = bc2((float)h6);
      const float2 one = bc2(1.0f);
#pragma unroll
      for (int a = 0; a < DIM; ++a) st.c[a] = fma(h6, (double)accc[a], st.c[a]);
#pragma unroll
      for (int p = 0; p < DIM; ++p)
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          const int o = (p * DIM + a) * kBlock;
          // k1 + 2k2 + 2k3 + k4, rounded as the in-loop fma(1, k4, sum) would
          dpl[o] = fma2(h6f, fma2(one, kd[p][a], accp[o]), dpl[o]);
        }
    } else if constexpr (INTEG == FTLE_EULER) {
#pragma unroll
      for (int a = 0; a < DIM; ++a) st.c[a] = fma(h, (double)kc[a], st.c[a]);
#pragma unroll
      for (int p = 0; p < DIM; ++p)
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          const int o = (p * DIM + a) * kBlock;
          dpl[o] = fma2(bc2(hf), kd[p][a], dpl[o]);
        }
    } else {  // AB2, Euler on the first step (integrate.py:240-246)
      if (i == 0) {
#pragma unroll
        for (int a = 0; a < DIM; ++a) st.c[a] = fma(h, (double)kc[a], st.c[a]);
#pragma unroll
        for (int p = 0; p < DIM; ++p)
#pragma unroll
          for (int a = 0; a < DIM; ++a) {
            const int o = (p * DIM + a) * kBlock;
            dpl[o] = fma2(bc2(hf), kd[p][a], dpl[o]);
          }
      } else {
#pragma unroll
        for (int a = 0; a < DIM; ++a)
          st.c[a] = fma(h, 1.5 * (double)kc[a] - 0.5 * (double)st.kcp[a], st.c[a]);
#pragma unroll
        for (int p = 0; p < DIM; ++p)
#pragma unroll
          for (int a = 0; a < DIM; ++a) {
            const int o = (p * DIM + a) * kBlock;
            const float2 prev = make_float2(st.kdp[2 * p][a], st.kdp[2 * p + 1][a]);
            dpl[o] = fma2(bc2(hf), fma2(bc2(1.5f), kd[p][a], mul2(bc2(-0.5f), prev)), dpl[o]);
          }
      }
#pragma unroll
      for (int a = 0; a < DIM; ++a) st.kcp[a] = kc[a];
#pragma unroll
      for (int p = 0; p < DIM; ++p)
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          st.kdp[2 * p][a] = kd[p][a].x;
          st.kdp[2 * p + 1][a] = kd[p][a].y;
        }
    }
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      kc[a] = 0.0f;  // next step's first stage starts at c
      if (periodic) {  // one period at most per step
        const double lo = m.w.g.origin[a], hi = lo + m.period[a];
        if (st.c[a] < lo) {
          st.c[a] += m.period[a];
          --st.wraps[a];
        } else if (st.c[a] >= hi) {
          st.c[a] -= m.period[a];
          ++st.wraps[a];
        }
      }
    }
  }
#pragma unroll
  for (int p = 0; p < DIM; ++p)
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      const float2 dv = dpl[(p * DIM + a) * kBlock];
      st.d[2 * p][a] = dv.x;
      st.d[2 * p + 1][a] = dv.y;
    }
}

// Final positions x_k = c + wraps*period + d_k and the FP64 FTLE epilogue.
template <int DIM>
__device__ __forceinline__ void group_finish(const MixK &m, const WinVar &v, long long g,
                                             GroupState<DIM> &st) {
  constexpr int K = 2 * DIM;
  const long long N = v.N;
  double c[DIM];
#pragma unroll
  for (int a = 0; a < DIM; ++a)
    c[a] = m.w.g.periodic ? st.c[a] + (double)st.wraps[a] * m.period[a] : st.c[a];
  // initial diagonal separations (Jacobian denominators), read from the seeds before
  // this group's final positions overwrite them
  double id[DIM];
#pragma unroll
  for (int j = 0; j < DIM; ++j)
    id[j] = v.positions[((long long)plus_r(j) * N + g) * DIM + j] -
            v.positions[((long long)minus_r(j) * N + g) * DIM + j];
  if (!v.keep_positions) {
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int a = 0; a < DIM; ++a)
        v.positions[((long long)k * N + g) * DIM + a] = c[a] + (double)st.d[k][a];
  }
  if (v.ftle != nullptr) {
    double J[DIM][DIM];
#pragma unroll
    for (int i = 0; i < DIM; ++i)
#pragma unroll
      for (int j = 0; j < DIM; ++j)
        J[i][j] = ((double)st.d[plus_r(j)][i] - (double)st.d[minus_r(j)][i]) / id[j];
    double lam;
    if constexpr (DIM == 2) {
      lam = lmax2(J[0][0], J[0][1], J[1][0], J[1][1]);
    } else {
      double C[3][3];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k)
          C[i][k] = J[i][0] * J[k][0] + J[i][1] * J[k][1] + J[i][2] * J[k][2];
      lam = lmax3_sym(C[0][0], C[0][1], C[0][2], C[1][1], C[1][2], C[2][2]);
    }
    v.ftle[g] = (1.0 / v.map_period) * log(sqrt(lam));
  }
}

// ---------------------------------------------------------------------------
// chunk state (structure of arrays over N slots) and cell sort
// ---------------------------------------------------------------------------

struct ChunkBuf {
  double *c;      // DIM x N
  int *wraps;     // DIM x N
  float *d;       // K*DIM x N
  float *hist;    // (DIM + K*DIM) x N, AB2 only
  long long *idx; // N: original group index
};

template <int DIM>
__device__ __forceinline__ void state_load(const ChunkBuf &b, long long N, long long j,
                                           GroupState<DIM> &st, bool ab2) {
  constexpr int K = 2 * DIM;
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    st.c[a] = b.c[a * N + j];
    st.wraps[a] = b.wraps[a * N + j];
    st.kcp[a] = ab2 ? b.hist[a * N + j] : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      st.d[k][a] = b.d[(k * DIM + a) * N + j];
      st.kdp[k][a] = ab2 ? b.hist[(DIM + k * DIM + a) * N + j] : 0.0f;
    }
}

template <int DIM>
__device__ __forceinline__ void state_store(const ChunkBuf &b, long long N, long long j,
                                            const GroupState<DIM> &st, bool ab2) {
  constexpr int K = 2 * DIM;
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    b.c[a * N + j] = st.c[a];
    b.wraps[a * N + j] = st.wraps[a];
    if (ab2) b.hist[a * N + j] = st.kcp[a];
  }
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      b.d[(k * DIM + a) * N + j] = st.d[k][a];
      if (ab2) b.hist[(DIM + k * DIM + a) * N + j] = st.kdp[k][a];
    }
}

// Interleave the low `bits` bits of x with stride dim (bits*dim <= 30).
__device__ __forceinline__ unsigned spread_bits(unsigned x, int dim, int bits) {
  unsigned r = 0;
  for (int b = 0; b < bits; ++b) r |= ((x >> b) & 1u) << (b * dim);
  return r;
}

// Morton key of the coarse cell holding the centroid (2^bits cells per axis).
template <int DIM>
__device__ __forceinline__ int cell_key(const MixK &m, const GroupState<DIM> &st, int bits) {
  unsigned key = 0;
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    const double p = fma(st.c[a], m.inv_sp[a], -m.org_sp[a]);
    const int n = m.w.g.n[a];
    double fl = floor(p);
    fl = fl < 0.0 ? 0.0 : (fl > (double)(n - 1) ? (double)(n - 1) : fl);  // NaN -> n-1 side
    if (!(fl >= 0.0)) fl = 0.0;
    const unsigned cc = (unsigned)(((long long)fl << bits) / n);
    key |= spread_bits(cc, DIM, bits) << a;
  }
  return (int)(key & ((1u << (bits * DIM)) - 1u));  // always a valid bin
}

__global__ void sort_hist_kernel(const int *__restrict__ keys, long long N, int *hist) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < N;
       j += (long long)gridDim.x * blockDim.x)
    atomicAdd(hist + keys[j], 1);
}

// in-place exclusive scan of nbins counters (one block of 1024 threads)
__global__ void sort_scan_kernel(int *bins, int nbins) {
  __shared__ int part[1024];
  const int per = (nbins + 1023) / 1024;
  const int b0 = threadIdx.x * per;
  int s = 0;
  for (int i = 0; i < per; ++i)
    if (b0 + i < nbins) s += bins[b0 + i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = part[threadIdx.x] - s;  // exclusive prefix of this thread's bins
  for (int i = 0; i < per; ++i)
    if (b0 + i < nbins) {
      const int c = bins[b0 + i];
      bins[b0 + i] = run;
      run += c;
    }
}

template <int DIM>
__global__ void sort_scatter_kernel(const int *__restrict__ keys, long long N, int *cursor,
                                    ChunkBuf in, ChunkBuf out, int ab2) {
  constexpr int K = 2 * DIM;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < N;
       j += (long long)gridDim.x * blockDim.x) {
    const long long p = atomicAdd(cursor + keys[j], 1);
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      out.c[a * N + p] = in.c[a * N + j];
      out.wraps[a * N + p] = in.wraps[a * N + j];
    }
#pragma unroll
    for (int q = 0; q < K * DIM; ++q) out.d[q * N + p] = in.d[q * N + j];
    if (ab2)
      for (int q = 0; q < DIM + K * DIM; ++q) out.hist[q * N + p] = in.hist[q * N + j];
    out.idx[p] = in.idx[j];
  }
}

// ---------------------------------------------------------------------------
// window kernels
// ---------------------------------------------------------------------------

// One launch advances every group through steps [i0, i1).  first: the state
// comes from the role-blocked positions (slot = group index); last: final
// positions and FTLE are written at the group's original index; otherwise
// the state goes back to `buf` (and its cell key to `keys` when given).
// Shared memory of a block (dynamic): per-thread columns of the off-cell slots, the
// RK4 accumulators and the offsets (K*DIM floats each, stride kBlock), then one
// gather queue per warp.
// Blocks of kBlock threads resident per SM that the register budget is sized for
// (measured on B200): 4 in 3D; in 2D the persistent batched kernel runs 8 (the
// turbulence windows keep most neighbours in their cell and gain from latency
// hiding), the single-window kernel 4 (long, strongly stretching windows gather
// per neighbour and need the L1 that a larger shared-memory carve-out takes).
template <int DIM>
constexpr int kMinBlocks = 4;
template <int DIM>
constexpr int kMinBlocksPersistent = DIM == 2 ? 8 : 4;

template <int DIM>
struct BlockSmem {
  static constexpr int kCol = 2 * DIM * DIM * kBlock;
  static constexpr size_t kBytes = 3 * kCol * sizeof(float) + (kBlock / 32) * sizeof(WarpQueue<DIM>);
  float *slots, *acc, *d;
  WarpQueue<DIM> *queue;
  __device__ explicit BlockSmem(unsigned char *base) {
    float *f = reinterpret_cast<float *>(base);
    slots = f;
    acc = f + kCol;
    d = f + 2 * kCol;
    queue = reinterpret_cast<WarpQueue<DIM> *>(f + 3 * kCol);
  }
};

template <int DIM, int MODE, int INTEG, int STORAGE>
__global__ void __launch_bounds__(kBlock, kMinBlocks<DIM>)
    window_mixed_kernel(const MixK m, const ChunkBuf buf, int i0, int i1, int first, int last,
                        int *keys, int key_bits) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  const BlockSmem<DIM> sm(dyn_smem);
  float *smem_slots = sm.slots;
  float2 *acc = reinterpret_cast<float2 *>(sm.acc) + threadIdx.x;
  float2 *dsm = reinterpret_cast<float2 *>(sm.d) + threadIdx.x;
  const int lane = threadIdx.x & 31;
  WarpQueue<DIM> &wq = sm.queue[threadIdx.x >> 5];
  const long long N = m.w.N;
  const long long j_raw = (long long)blockIdx.x * kBlock + threadIdx.x;
  // lanes past the end mirror the last slot (warp-wide shuffles need every lane) but write nothing
  const bool active = j_raw < N;
  const long long j = active ? j_raw : N - 1;
  const Header16 hd = *reinterpret_cast<const Header16 *>(m.w.snaps);
  constexpr bool AB2 = INTEG == FTLE_AB2;

  const WinVar v = winvar_of(m);
  GroupState<DIM> st;
  long long g;
  if (first) {
    g = j;
    group_from_positions<DIM>(m, v, g, st);
  } else {
    g = buf.idx[j];
    state_load<DIM>(buf, N, j, st, AB2);
  }
  group_advect<DIM, MODE, INTEG, STORAGE>(m, v, hd, st, i0, i1, smem_slots, acc, dsm, wq, lane);
  if (!active) return;
  if (last) {
    group_finish<DIM>(m, v, g, st);
  } else {
    state_store<DIM>(buf, N, j, st, AB2);
    buf.idx[j] = g;
    if (keys) keys[j] = cell_key<DIM>(m, st, key_bits);
  }
}

// ---------------------------------------------------------------------------
// many windows in one persistent launch
// ---------------------------------------------------------------------------

// A work item: kBlock consecutive groups of one window.
struct BatchItem {
  int window;
  int reserved;
  long long g0;
};

// Plan layout (host-built, copied to the device once):
//   PlanHeader | WinVar[num_windows] | BatchItem[num_items] | int counter
struct PlanHeader {
  int num_windows, num_items, order, reserved;
};

static int64_t align256_(int64_t x) { return (x + 255) & ~int64_t(255); }
static int64_t plan_offset_wins() { return 256; }
static int64_t plan_offset_items(int nw) { return align256_(256 + (int64_t)nw * sizeof(WinVar)); }
static int64_t plan_offset_counter(int nw, int64_t ni) {
  return align256_(plan_offset_items(nw) + ni * (int64_t)sizeof(BatchItem));
}
static int64_t plan_total(int nw, int64_t ni) { return plan_offset_counter(nw, ni) + 256; }

// Persistent CTAs take work items from a global counter until the list is empty;
// every thread of an item advects one group of that item's window.
template <int DIM, int MODE, int INTEG, int STORAGE>
__global__ void __launch_bounds__(kBlock, kMinBlocksPersistent<DIM>)
    windows_persistent_kernel(const MixK m, const WinVar *__restrict__ wins,
                              const BatchItem *__restrict__ items, int num_items, int *counter) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  const BlockSmem<DIM> sm(dyn_smem);
  __shared__ int s_item;
  float *smem_slots = sm.slots;
  float2 *acc = reinterpret_cast<float2 *>(sm.acc) + threadIdx.x;
  float2 *dsm = reinterpret_cast<float2 *>(sm.d) + threadIdx.x;
  const int lane = threadIdx.x & 31;
  WarpQueue<DIM> &wq = sm.queue[threadIdx.x >> 5];
  const Header16 hd = *reinterpret_cast<const Header16 *>(m.w.snaps);
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();  // every thread has read s_item before thread 0 overwrites it
    if (it >= num_items) return;
    const BatchItem bi = items[it];
    const WinVar v = wins[bi.window];
    const long long j_raw = bi.g0 + threadIdx.x;
    const bool active = j_raw < v.N;
    const long long j = active ? j_raw : v.N - 1;
    GroupState<DIM> st;
    group_from_positions<DIM>(m, v, j, st);
    group_advect<DIM, MODE, INTEG, STORAGE>(m, v, hd, st, 0, v.num_steps, smem_slots, acc, dsm,
                                            wq, lane);
    if (active) group_finish<DIM>(m, v, j, st);
  }
}

// Allow the kernel's dynamic shared memory (31.5 KB for a 3D block, 15 KB in 2D, under
// the 48 KB default today; set anyway so a larger layout needs no other change);
// called once per kernel instance.
template <typename Kernel>
static bool set_smem_attr(Kernel kernel, size_t bytes) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  return true;
}

template <int DIM, int MODE, int STORAGE>
static void launch_persistent(const MixK &m, int integ, const WinVar *wins,
                              const BatchItem *items, int num_items, int *counter, int ctas,
                              cudaStream_t st) {
#define LP(I)                                                                              \
  do {                                                                                     \
    static const bool attr_set = set_smem_attr(windows_persistent_kernel<DIM, MODE, I, STORAGE>, \
                                               BlockSmem<DIM>::kBytes);                    \
    (void)attr_set;                                                                        \
    windows_persistent_kernel<DIM, MODE, I, STORAGE>                                       \
        <<<ctas, kBlock, BlockSmem<DIM>::kBytes, st>>>(m, wins, items, num_items, counter); \
  } while (0)
  if (integ == FTLE_EULER)
    LP(FTLE_EULER);
  else if (integ == FTLE_AB2)
    LP(FTLE_AB2);
  else
    LP(FTLE_RK4);
#undef LP
}

static void launch_persistent_any(const MixK &m, int dim, int mode, int integ, int storage,
                                  const WinVar *wins, const BatchItem *items, int num_items,
                                  int *counter, int ctas, cudaStream_t st) {
#define LPS(D, M)                                                                            \
  do {                                                                                       \
    if (storage == FTLE_F16)                                                                 \
      launch_persistent<D, M, FTLE_F16>(m, integ, wins, items, num_items, counter, ctas, st); \
    else if (storage == FTLE_BF16)                                                           \
      launch_persistent<D, M, FTLE_BF16>(m, integ, wins, items, num_items, counter, ctas, st); \
    else                                                                                     \
      launch_persistent<D, M, FTLE_FX15>(m, integ, wins, items, num_items, counter, ctas, st); \
  } while (0)
  if (dim == 2) {
    if (mode == FTLE_HOLD)
      LPS(2, FTLE_HOLD);
    else
      LPS(2, FTLE_BLEND);
  } else {
    if (mode == FTLE_HOLD)
      LPS(3, FTLE_HOLD);
    else
      LPS(3, FTLE_BLEND);
  }
#undef LPS
}

template <int DIM, int MODE, int STORAGE>
static void launch_mixed(const MixK &m, int integ, const ChunkBuf &buf, int i0, int i1,
                         int first, int last, int *keys, int key_bits, cudaStream_t st) {
  const unsigned blocks = (unsigned)((m.w.N + kBlock - 1) / kBlock);
#define LM(I)                                                                            \
  do {                                                                                   \
    static const bool attr_set =                                                         \
        set_smem_attr(window_mixed_kernel<DIM, MODE, I, STORAGE>, BlockSmem<DIM>::kBytes); \
    (void)attr_set;                                                                      \
    window_mixed_kernel<DIM, MODE, I, STORAGE><<<blocks, kBlock, BlockSmem<DIM>::kBytes, st>>>( \
        m, buf, i0, i1, first, last, keys, key_bits);                                    \
  } while (0)
  if (integ == FTLE_EULER)
    LM(FTLE_EULER);
  else if (integ == FTLE_AB2)
    LM(FTLE_AB2);
  else
    LM(FTLE_RK4);
#undef LM
}

static void launch_any(const MixK &m, int dim, int mode, int integ, int storage,
                       const ChunkBuf &buf, int i0, int i1, int first, int last, int *keys,
                       int key_bits, cudaStream_t st) {
#define LS(D, M)                                                                         \
  do {                                                                                   \
    if (storage == FTLE_F16)                                                             \
      launch_mixed<D, M, FTLE_F16>(m, integ, buf, i0, i1, first, last, keys, key_bits, st); \
    else if (storage == FTLE_BF16)                                                       \
      launch_mixed<D, M, FTLE_BF16>(m, integ, buf, i0, i1, first, last, keys, key_bits, st); \
    else                                                                                 \
      launch_mixed<D, M, FTLE_FX15>(m, integ, buf, i0, i1, first, last, keys, key_bits, st); \
  } while (0)
  if (dim == 2) {
    if (mode == FTLE_HOLD)
      LS(2, FTLE_HOLD);
    else
      LS(2, FTLE_BLEND);
  } else {
    if (mode == FTLE_HOLD)
      LS(3, FTLE_HOLD);
    else
      LS(3, FTLE_BLEND);
  }
#undef LS
}

static int mixed_setup(const ftle_window *w, MixK &m) {
  int rc = window_to_kernel(w, &m.w);
  if (rc) return rc;
  if (w->storage != FTLE_F16 && w->storage != FTLE_BF16 && w->storage != FTLE_FX15 &&
      w->storage != FTLE_FX16)
    return fail_invalid(
        "the mixed-precision window needs FTLE_F16, FTLE_BF16, FTLE_FX15 or FTLE_FX16 storage");
  if (m.w.g.nodes >= (1LL << 31))
    return fail_invalid("the mixed-precision window supports grids below 2^31 nodes");
  for (int a = 0; a < 3; ++a) {
    m.inv_sp[a] = 1.0 / m.w.g.spacing[a];
    m.org_sp[a] = m.w.g.origin[a] / m.w.g.spacing[a];
    m.inv_spf[a] = (float)m.inv_sp[a];
    m.period[a] = (double)m.w.g.n[a] * m.w.g.spacing[a];
  }
  if (w->grid.dim == 2) {
    m.stride[0] = 1;
    m.stride[1] = m.w.g.n[0];
    m.stride[2] = 0;
  } else {
    m.stride[0] = m.w.g.n[2];
    m.stride[1] = m.w.g.n[0] * m.w.g.n[2];
    m.stride[2] = 1;
  }
  m.inv_dt = 1.0 / (w->snapshot_dt != 0.0 ? w->snapshot_dt : 1.0);
  m.inv_S = 1.0 / (double)m.w.num_snaps;
  return FTLE_OK;
}

// Workspace carve-up: two state buffers, keys, bins.
struct WsLayout {
  int64_t state_bytes, keys_off, bins_off, total;
  int key_bits, nbins;
};

static int64_t align256(int64_t x) { return (x + 255) & ~int64_t(255); }

static WsLayout ws_layout(int dim, int integ, int64_t N) {
  const int K = 2 * dim;
  WsLayout L;
  int64_t per = 0;
  per += align256(8 * dim * N);                 // c
  per += align256(4 * dim * N);                 // wraps
  per += align256(4 * K * dim * N);             // d
  per += integ == FTLE_AB2 ? align256(4 * (dim + K * dim) * N) : 0;  // AB2 history
  per += align256(8 * N);                       // idx
  L.state_bytes = per;
  L.keys_off = 2 * per;
  L.bins_off = L.keys_off + align256(4 * N);
  L.key_bits = dim == 2 ? 8 : 5;
  L.nbins = 1 << (L.key_bits * dim);
  L.total = L.bins_off + align256(4 * (int64_t)L.nbins);
  return L;
}

static ChunkBuf carve(unsigned char *base, int dim, int integ, int64_t N) {
  const int K = 2 * dim;
  ChunkBuf b;
  unsigned char *p = base;
  b.c = reinterpret_cast<double *>(p);
  p += align256(8 * dim * N);
  b.wraps = reinterpret_cast<int *>(p);
  p += align256(4 * dim * N);
  b.d = reinterpret_cast<float *>(p);
  p += align256(4 * K * dim * N);
  if (integ == FTLE_AB2) {
    b.hist = reinterpret_cast<float *>(p);
    p += align256(4 * (dim + K * dim) * N);
  } else {
    b.hist = nullptr;
  }
  b.idx = reinterpret_cast<long long *>(p);
  return b;
}

}  // namespace ftle

using namespace ftle;

extern "C" {

int ftle_window_run_mixed(const ftle_window *w, void *stream) {
  MixK m;
  int rc = mixed_setup(w, m);
  if (rc) return rc;
  if (m.w.N == 0) return FTLE_OK;
  ChunkBuf none{};
  launch_any(m, w->grid.dim, w->time_mode, w->integrator, w->storage, none, 0, w->num_steps, 1, 1,
             nullptr, 0, as_stream(stream));
  return check_launch("window_mixed_kernel");
}

int64_t ftle_window_workspace_bytes(const ftle_window *w) {
  if (!w || (w->grid.dim != 2 && w->grid.dim != 3) || w->num_groups < 0) return -1;
  return ws_layout(w->grid.dim, w->integrator, w->num_groups).total;
}

int ftle_window_run_mixed_chunked(const ftle_window *w, void *workspace, int64_t workspace_bytes,
                                  int32_t chunk_steps, int32_t sort_every, void *stream) {
  MixK m;
  int rc = mixed_setup(w, m);
  if (rc) return rc;
  if (m.w.N == 0) return FTLE_OK;
  if (chunk_steps < 1) return fail_invalid("chunk_steps must be >= 1");
  const int dim = w->grid.dim;
  const WsLayout L = ws_layout(dim, w->integrator, m.w.N);
  if (!workspace || workspace_bytes < L.total)
    return fail_invalid("workspace too small: need %lld bytes", (long long)L.total);
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
    return fail_invalid("workspace must be 256-byte aligned");
  cudaStream_t st = as_stream(stream);
  unsigned char *ws = static_cast<unsigned char *>(workspace);
  ChunkBuf cur = carve(ws, dim, w->integrator, m.w.N);
  ChunkBuf nxt = carve(ws + L.state_bytes, dim, w->integrator, m.w.N);
  int *keys = reinterpret_cast<int *>(ws + L.keys_off);
  int *bins = reinterpret_cast<int *>(ws + L.bins_off);
  const int steps = w->num_steps;
  int chunk = 0;
  for (int i0 = 0;; i0 += chunk_steps, ++chunk) {
    const int i1 = i0 + chunk_steps < steps ? i0 + chunk_steps : steps;
    const int first = i0 == 0, last = i1 == steps;
    const bool sort_now = !last && sort_every > 0 && (chunk + 1) % sort_every == 0;
    launch_any(m, dim, w->time_mode, w->integrator, w->storage, cur, i0, i1, first, last,
               sort_now ? keys : nullptr, L.key_bits, st);
    if ((rc = check_launch("window_mixed_kernel"))) return rc;
    if (last) break;
    if (sort_now) {
      if (cudaMemsetAsync(bins, 0, 4 * (size_t)L.nbins, st) != cudaSuccess)
        return check_launch("cudaMemsetAsync");
      const unsigned b = grid_blocks(m.w.N, 256);
      sort_hist_kernel<<<b, 256, 0, st>>>(keys, m.w.N, bins);
      sort_scan_kernel<<<1, 1024, 0, st>>>(bins, L.nbins);
      if (dim == 2)
        sort_scatter_kernel<2><<<b, 256, 0, st>>>(keys, m.w.N, bins, cur, nxt,
                                                  w->integrator == FTLE_AB2);
      else
        sort_scatter_kernel<3><<<b, 256, 0, st>>>(keys, m.w.N, bins, cur, nxt,
                                                  w->integrator == FTLE_AB2);
      if ((rc = check_launch("sort kernels"))) return rc;
      const ChunkBuf t = cur;
      cur = nxt;
      nxt = t;
    }
  }
  return FTLE_OK;
}

// ---- many windows in one launch ------------------------------------------

static int check_batch(const ftle_window *windows, int32_t count) {
  if (!windows || count < 1) return fail_invalid("need at least one window");
  const ftle_window &a = windows[0];
  for (int i = 1; i < count; ++i) {
    const ftle_window &b = windows[i];
    if (b.snapshots != a.snapshots || b.num_snapshots != a.num_snapshots ||
        b.storage != a.storage || b.time_mode != a.time_mode ||
        b.periodic_time != a.periodic_time || b.snapshot_t0 != a.snapshot_t0 ||
        b.snapshot_dt != a.snapshot_dt || b.integrator != a.integrator ||
        b.grid.dim != a.grid.dim || b.grid.periodic != a.grid.periodic)
      return fail_invalid("window %d does not share window 0's snapshot series and integrator", i);
    for (int ax = 0; ax < 3; ++ax)
      if (b.grid.n[ax] != a.grid.n[ax] || b.grid.origin[ax] != a.grid.origin[ax] ||
          b.grid.spacing[ax] != a.grid.spacing[ax])
        return fail_invalid("window %d does not share window 0's grid", i);
  }
  for (int i = 0; i < count; ++i) {
    MixK m;
    int rc = mixed_setup(&windows[i], m);
    if (rc) return rc;
  }
  return FTLE_OK;
}

static int64_t batch_items(const ftle_window *windows, int32_t count) {
  int64_t n = 0;
  for (int i = 0; i < count; ++i) n += (windows[i].num_groups + kBlock - 1) / kBlock;
  return n;
}

int64_t ftle_windows_plan_bytes(const ftle_window *windows, int32_t count) {
  if (!windows || count < 1) return -1;
  return plan_total(count, batch_items(windows, count));
}

int ftle_windows_plan(const ftle_window *windows, int32_t count, int32_t order, void *host_plan,
                      int64_t plan_bytes) {
  int rc = check_batch(windows, count);
  if (rc) return rc;
  const int64_t ni = batch_items(windows, count);
  if (ni > 0x7fffffff) return fail_invalid("too many work items");
  if (!host_plan || plan_bytes < plan_total(count, ni))
    return fail_invalid("plan buffer too small: need %lld bytes", (long long)plan_total(count, ni));
  unsigned char *p = static_cast<unsigned char *>(host_plan);
  PlanHeader *hdr = reinterpret_cast<PlanHeader *>(p);
  hdr->num_windows = count;
  hdr->num_items = (int)ni;
  hdr->order = order;
  hdr->reserved = 0;
  WinVar *wins = reinterpret_cast<WinVar *>(p + plan_offset_wins());
  for (int i = 0; i < count; ++i) {
    const ftle_window &w = windows[i];
    wins[i].t0 = w.t0;
    wins[i].h = w.h;
    wins[i].map_period = w.map_period;
    wins[i].positions = w.positions;
    wins[i].ftle = w.ftle;
    wins[i].N = w.num_groups;
    wins[i].num_steps = w.num_steps;
    wins[i].first_snapshot = w.first_snapshot;
    wins[i].keep_positions = (w.flags & FTLE_KEEP_POSITIONS) ? 1 : 0;
    wins[i].reserved = 0;
  }
  // order 1: longest windows first (work items of long windows are scheduled before short
  // ones so the tail of the persistent launch is short); order 2: by the start of the
  // window's time range (items resident together then read nearby snapshot intervals,
  // which share L2); order 0: as given.  Insertion sorts, stable.
  int *perm = new int[count];
  for (int i = 0; i < count; ++i) perm[i] = i;
  auto t_first = [&](int i) {
    const ftle_window &w = windows[i];
    const double t_end = w.t0 + w.num_steps * w.h;
    return w.t0 < t_end ? w.t0 : t_end;
  };
  if (order == 1 || order == 2) {
    for (int i = 1; i < count; ++i) {
      const int x = perm[i];
      int k = i - 1;
      while (k >= 0 && (order == 1 ? windows[perm[k]].num_steps < windows[x].num_steps
                                   : t_first(perm[k]) > t_first(x))) {
        perm[k + 1] = perm[k];
        --k;
      }
      perm[k + 1] = x;
    }
  }
  BatchItem *items = reinterpret_cast<BatchItem *>(p + plan_offset_items(count));
  int64_t q = 0;
  for (int r = 0; r < count; ++r) {
    const int i = perm[r];
    for (int64_t g0 = 0; g0 < windows[i].num_groups; g0 += kBlock) {
      items[q].window = i;
      items[q].reserved = 0;
      items[q].g0 = g0;
      ++q;
    }
  }
  delete[] perm;
  *reinterpret_cast<int *>(p + plan_offset_counter(count, ni)) = 0;
  return FTLE_OK;
}

int ftle_windows_run_mixed(const ftle_window *windows, int32_t count, void *device_plan,
                           int64_t plan_bytes, int32_t ctas_per_sm, void *stream) {
  int rc = check_batch(windows, count);
  if (rc) return rc;
  const int64_t ni = batch_items(windows, count);
  if (!device_plan || plan_bytes < plan_total(count, ni))
    return fail_invalid("plan buffer too small: need %lld bytes", (long long)plan_total(count, ni));
  if (reinterpret_cast<uintptr_t>(device_plan) % 256 != 0)
    return fail_invalid("plan must be 256-byte aligned");
  if (ctas_per_sm < 1 || ctas_per_sm > 8) return fail_invalid("ctas_per_sm must be 1 to 8");
  if (ni == 0) return FTLE_OK;
  MixK m;
  mixed_setup(&windows[0], m);
  unsigned char *p = static_cast<unsigned char *>(device_plan);
  int *counter = reinterpret_cast<int *>(p + plan_offset_counter(count, ni));
  cudaStream_t st = as_stream(stream);
  if (cudaMemsetAsync(counter, 0, sizeof(int), st) != cudaSuccess)
    return check_launch("cudaMemsetAsync");
  launch_persistent_any(m, windows[0].grid.dim, windows[0].time_mode, windows[0].integrator,
                        windows[0].storage, reinterpret_cast<const WinVar *>(p + plan_offset_wins()),
                        reinterpret_cast<const BatchItem *>(p + plan_offset_items(count)), (int)ni,
                        counter, ctas_per_sm * kNumSMs, st);
  return check_launch("windows_persistent_kernel");
}

}  // extern "C"
