// mixed.cu -- mixed-precision FTLE window (sm_100a).
//
// Snapshots are stored as FP16 or BF16 "pair records": record (s, node) holds
// the velocity of snapshot s and of its successor, so one 8-byte (2D) or
// 16-byte (3D) load per cell corner serves a time-blended gather.
//
// Each thread advects one neighbour group in the split representation:
//   centroid c            FP64 (its cell index and in-cell fraction are exact)
//   offsets  d_k = x_k-c  FP32, advected with velocity differences u(x_k)-u(c)
// so the finite differences x_R - x_L never cancel in FP32.  Velocities are
// FP32 (blend in time at the corners, then bi/trilinear).  The 8 (3D) or 4
// (2D) corner values of the centroid's cell stay in registers and serve every
// neighbour that sits in the same cell, which is nearly all of them while the
// group is smaller than a cell.  The Jacobian -> Cauchy-Green -> lambda_max
// epilogue runs in FP64 (ftle.py:9-233 restated).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <math.h>

#include "common.cuh"

namespace ftle {

// ---------------------------------------------------------------------------
// 16-bit storage traits
// ---------------------------------------------------------------------------
template <int STORAGE>
struct Half2;  // unpack two 16-bit values packed in a 32-bit word

template <>
struct Half2<FTLE_F16> {
  static __device__ __forceinline__ float2 unpack(unsigned w) {
    __half2 h;
    memcpy(&h, &w, 4);
    return __half22float2(h);
  }
  static __device__ __forceinline__ unsigned short from_double(double x) {
    __half h = __double2half(x);
    unsigned short b;
    memcpy(&b, &h, 2);
    return b;
  }
};

template <>
struct Half2<FTLE_BF16> {
  static __device__ __forceinline__ float2 unpack(unsigned w) {
    return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
  }
  static __device__ __forceinline__ unsigned short from_double(double x) {
    __nv_bfloat16 h = __double2bfloat16(x);
    unsigned short b;
    memcpy(&b, &h, 2);
    return b;
  }
};

// ---------------------------------------------------------------------------
// packing: (S, dim, nodes) float64 -> pair records
// ---------------------------------------------------------------------------
template <int DIM, int STORAGE>
__global__ void pack16_kernel(const double *__restrict__ src, long long nodes, int S,
                              int periodic_time, unsigned short *dst) {
  constexpr int W = DIM == 2 ? 4 : 8;  // 16-bit values per record
  const long long total = nodes * S;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(i / nodes);
    const long long p = i - (long long)s * nodes;
    const int s1 = (s + 1 < S) ? s + 1 : (periodic_time ? 0 : s);
    unsigned short r[W];
    const int half = W / 2;
#pragma unroll
    for (int c = 0; c < half; ++c) {
      r[c] = c < DIM ? Half2<STORAGE>::from_double(src[((long long)s * DIM + c) * nodes + p]) : 0;
      r[half + c] =
          c < DIM ? Half2<STORAGE>::from_double(src[((long long)s1 * DIM + c) * nodes + p]) : 0;
    }
    if constexpr (DIM == 2) {
      uint2 v;
      v.x = (unsigned)r[0] | ((unsigned)r[1] << 16);
      v.y = (unsigned)r[2] | ((unsigned)r[3] << 16);
      reinterpret_cast<uint2 *>(dst)[i] = v;
    } else {
      uint4 v;
      v.x = (unsigned)r[0] | ((unsigned)r[1] << 16);
      v.y = (unsigned)r[2] | ((unsigned)r[3] << 16);
      v.z = (unsigned)r[4] | ((unsigned)r[5] << 16);
      v.w = (unsigned)r[6] | ((unsigned)r[7] << 16);
      reinterpret_cast<uint4 *>(dst)[i] = v;
    }
  }
}

int pack_snapshots_16(int32_t dim, int64_t nodes, int32_t num_snapshots, int32_t periodic_time,
                      const double *src, int32_t storage, void *dst, void *stream) {
  const int64_t total = nodes * num_snapshots;
  const unsigned b = grid_blocks(total, 256);
  cudaStream_t st = as_stream(stream);
  unsigned short *d = static_cast<unsigned short *>(dst);
  if (dim == 2) {
    if (storage == FTLE_F16)
      pack16_kernel<2, FTLE_F16><<<b, 256, 0, st>>>(src, nodes, num_snapshots, periodic_time, d);
    else
      pack16_kernel<2, FTLE_BF16><<<b, 256, 0, st>>>(src, nodes, num_snapshots, periodic_time, d);
  } else {
    if (storage == FTLE_F16)
      pack16_kernel<3, FTLE_F16><<<b, 256, 0, st>>>(src, nodes, num_snapshots, periodic_time, d);
    else
      pack16_kernel<3, FTLE_BF16><<<b, 256, 0, st>>>(src, nodes, num_snapshots, periodic_time, d);
  }
  return check_launch("pack16_kernel");
}

// ---------------------------------------------------------------------------
// gathers
// ---------------------------------------------------------------------------

struct MixK {
  WinK w;
  double inv_sp[3];   // 1/spacing (FP64, centroid cell)
  float inv_spf[3];   // 1/spacing (FP32, neighbour offsets)
  double inv_dt;      // 1/snapshot_dt
};

__device__ __forceinline__ float lerpf(float a, float b, float t) { return fmaf(t, b - a, a); }

// Blended corner velocities of cell (i0) -> v[corner][comp], corner order
// x0y0(z0) x1y0 x0y1 x1y1 (then the same at z1).
template <int DIM, bool BLEND, int STORAGE>
__device__ __forceinline__ void gather_cell(const GridK &g, const void *__restrict__ base,
                                            float alpha, const int *i0, float (*v)[DIM]) {
  int lo[DIM], hi[DIM];
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    lo[a] = i0[a];
    hi[a] = i0[a] + 1;
    if (g.periodic) {
      lo[a] = wrap_index(lo[a], g.n[a]);
      hi[a] = lo[a] + 1 == g.n[a] ? 0 : lo[a] + 1;
    }
  }
  if constexpr (DIM == 2) {
    const uint2 *rec = static_cast<const uint2 *>(base);
    long long nd[4] = {node2(g, lo[0], lo[1]), node2(g, hi[0], lo[1]), node2(g, lo[0], hi[1]),
                       node2(g, hi[0], hi[1])};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint2 r = __ldg(rec + nd[q]);
      const float2 a = Half2<STORAGE>::unpack(r.x);
      if constexpr (BLEND) {
        const float2 b = Half2<STORAGE>::unpack(r.y);
        v[q][0] = lerpf(a.x, b.x, alpha);
        v[q][1] = lerpf(a.y, b.y, alpha);
      } else {
        v[q][0] = a.x;
        v[q][1] = a.y;
      }
    }
  } else {
    const uint4 *rec = static_cast<const uint4 *>(base);
    long long nd[8] = {node3(g, lo[0], lo[1], lo[2]), node3(g, hi[0], lo[1], lo[2]),
                       node3(g, lo[0], hi[1], lo[2]), node3(g, hi[0], hi[1], lo[2]),
                       node3(g, lo[0], lo[1], hi[2]), node3(g, hi[0], lo[1], hi[2]),
                       node3(g, lo[0], hi[1], hi[2]), node3(g, hi[0], hi[1], hi[2])};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const uint4 r = __ldg(rec + nd[q]);
      const float2 a = Half2<STORAGE>::unpack(r.x);
      const float2 aw = Half2<STORAGE>::unpack(r.y);
      if constexpr (BLEND) {
        const float2 b = Half2<STORAGE>::unpack(r.z);
        const float2 bw = Half2<STORAGE>::unpack(r.w);
        v[q][0] = lerpf(a.x, b.x, alpha);
        v[q][1] = lerpf(a.y, b.y, alpha);
        v[q][2] = lerpf(aw.x, bw.x, alpha);
      } else {
        v[q][0] = a.x;
        v[q][1] = a.y;
        v[q][2] = aw.x;
      }
    }
  }
}

template <int DIM>
__device__ __forceinline__ void interp_cell(const float (*v)[DIM], const float *f, float *u) {
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    const float x0 = lerpf(v[0][c], v[1][c], f[0]);
    const float x1 = lerpf(v[2][c], v[3][c], f[0]);
    const float y0 = lerpf(x0, x1, f[1]);
    if constexpr (DIM == 2) {
      u[c] = y0;
    } else {
      const float x2 = lerpf(v[4][c], v[5][c], f[0]);
      const float x3 = lerpf(v[6][c], v[7][c], f[0]);
      const float y1 = lerpf(x2, x3, f[1]);
      u[c] = lerpf(y0, y1, f[2]);
    }
  }
}

template <int DIM>
__device__ __forceinline__ bool cell_inside(const GridK &g, const int *i0) {
  if (g.periodic) return true;
  bool in = true;
#pragma unroll
  for (int a = 0; a < DIM; ++a) in = in && i0[a] >= 0 && i0[a] <= g.n[a] - 2;
  return in;
}

// Velocity of the centroid (uc) and velocity differences du[k] = u(c + d_k) - u(c).
template <int DIM, bool BLEND, int STORAGE>
__device__ __forceinline__ void eval_group(const MixK &m, const void *base, float alpha,
                                           const double *cs, const float (*ds)[DIM], float *uc,
                                           float (*du)[DIM]) {
  constexpr int K = 2 * DIM;
  const GridK &g = m.w.g;
  int ci[DIM];
  float fc[DIM];
  bool finite = true;
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    const double p = (cs[a] - g.origin[a]) * m.inv_sp[a];
    const double fl = floor(p);
    finite = finite && fabs(fl) < 1.0e9;
    ci[a] = finite ? (int)fl : 0;
    fc[a] = finite ? (float)(p - fl) : 0.0f;
  }
  if (!finite) {  // far outside or NaN: the whole group stands still
#pragma unroll
    for (int a = 0; a < DIM; ++a) uc[a] = 0.0f;
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int a = 0; a < DIM; ++a) du[k][a] = 0.0f;
    return;
  }
  float v[1 << DIM][DIM];
  const bool cin = cell_inside<DIM>(g, ci);
  if (cin) {
    gather_cell<DIM, BLEND, STORAGE>(g, base, alpha, ci, v);
    interp_cell<DIM>(v, fc, uc);
  } else {
#pragma unroll
    for (int a = 0; a < DIM; ++a) uc[a] = 0.0f;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    float q[DIM];
    int o[DIM];
    bool same = true;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      const float qa = fmaf(ds[k][a], m.inv_spf[a], fc[a]);
      const float fo = floorf(qa);
      o[a] = (int)fo;
      q[a] = qa - fo;
      same = same && o[a] == 0;
    }
    float uk[DIM];
    if (same) {
      if (cin) {
        interp_cell<DIM>(v, q, uk);
      } else {
#pragma unroll
        for (int a = 0; a < DIM; ++a) uk[a] = 0.0f;
      }
    } else {
      int ck[DIM];
#pragma unroll
      for (int a = 0; a < DIM; ++a) ck[a] = ci[a] + o[a];
      if (cell_inside<DIM>(g, ck)) {
        float vk[1 << DIM][DIM];
        gather_cell<DIM, BLEND, STORAGE>(g, base, alpha, ck, vk);
        interp_cell<DIM>(vk, q, uk);
      } else {
#pragma unroll
        for (int a = 0; a < DIM; ++a) uk[a] = 0.0f;
      }
    }
#pragma unroll
    for (int a = 0; a < DIM; ++a) du[k][a] = uk[a] - uc[a];
  }
}

template <int DIM, int MODE>
__device__ __forceinline__ const void *record_set(const MixK &m, int step, double t,
                                                  float &alpha) {
  const long long rec_bytes = DIM == 2 ? 8 : 16;
  const char *base = static_cast<const char *>(m.w.snaps);
  const long long set_bytes = m.w.g.nodes * rec_bytes;
  int s;
  if constexpr (MODE == FTLE_HOLD) {
    s = m.w.first_snapshot + step;
    if (m.w.periodic_time) s %= m.w.num_snaps;
    alpha = 0.0f;
  } else {
    double tau = (t - m.w.snap_t0) * m.inv_dt;
    const int S = m.w.num_snaps;
    if (m.w.periodic_time) {
      tau = tau - (double)S * floor(tau / (double)S);
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
  return base + (long long)s * set_bytes;
}

// ---------------------------------------------------------------------------
// FP64 epilogue (same formulas as the plain path)
// ---------------------------------------------------------------------------
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

__device__ __forceinline__ double lmax3_sym(double a00, double a01, double a02, double a11,
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

__device__ __forceinline__ int plus_r(int j) { return j == 0 ? 1 : 2 * j; }
__device__ __forceinline__ int minus_r(int j) { return j == 0 ? 0 : 2 * j + 1; }

// ---------------------------------------------------------------------------
// the window kernel: one thread per neighbour group
// ---------------------------------------------------------------------------
template <int DIM, int MODE, int INTEG, int STORAGE>
__global__ void __launch_bounds__(128) window_mixed_kernel(const MixK m) {
  constexpr int K = 2 * DIM;
  constexpr bool BLEND = MODE == FTLE_BLEND;
  const long long N = m.w.N;
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= N) return;

  double c[DIM];
  float d[K][DIM];
  double id[DIM];
  {
    double X[K][DIM];
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int a = 0; a < DIM; ++a) X[k][a] = m.w.positions[((long long)k * N + g) * DIM + a];
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      double s = X[0][a];
#pragma unroll
      for (int k = 1; k < K; ++k) s += X[k][a];
      c[a] = s / (double)K;  // particles.py:235-236 (mean of the neighbours)
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int a = 0; a < DIM; ++a) d[k][a] = (float)(X[k][a] - c[a]);
#pragma unroll
    for (int j = 0; j < DIM; ++j) id[j] = X[plus_r(j)][j] - X[minus_r(j)][j];
  }

  const double h = m.w.h;
  const float hf = (float)h;
  float ucp[DIM], dup[K][DIM];  // AB2 history
  for (int i = 0; i < m.w.num_steps; ++i) {
    const double t = m.w.t0 + (double)i * h;
    float uc[DIM], du[K][DIM];
    float alpha;
    if constexpr (INTEG == FTLE_EULER || INTEG == FTLE_AB2) {
      const void *base = record_set<DIM, MODE>(m, i, t, alpha);
      eval_group<DIM, BLEND, STORAGE>(m, base, alpha, c, d, uc, du);
      if (INTEG == FTLE_EULER || i == 0) {
#pragma unroll
        for (int a = 0; a < DIM; ++a) c[a] += h * (double)uc[a];
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
          for (int a = 0; a < DIM; ++a) d[k][a] = fmaf(hf, du[k][a], d[k][a]);
      } else {
#pragma unroll
        for (int a = 0; a < DIM; ++a) c[a] += h * (1.5 * (double)uc[a] - 0.5 * (double)ucp[a]);
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
          for (int a = 0; a < DIM; ++a)
            d[k][a] = fmaf(hf, fmaf(1.5f, du[k][a], -0.5f * dup[k][a]), d[k][a]);
      }
      if constexpr (INTEG == FTLE_AB2) {
#pragma unroll
        for (int a = 0; a < DIM; ++a) ucp[a] = uc[a];
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
          for (int a = 0; a < DIM; ++a) dup[k][a] = du[k][a];
      }
    } else {
      const double hh = 0.5 * h;
      const float hhf = (float)hh;
      double cs[DIM], accc[DIM];
      float ds[K][DIM], accd[K][DIM];
      // stage 1
      const void *b0 = record_set<DIM, MODE>(m, i, t, alpha);
      eval_group<DIM, BLEND, STORAGE>(m, b0, alpha, c, d, uc, du);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        accc[a] = (double)uc[a];
        cs[a] = c[a] + hh * (double)uc[a];
      }
#pragma unroll
      for (int k = 0; k < K; ++k)
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          accd[k][a] = du[k][a];
          ds[k][a] = fmaf(hhf, du[k][a], d[k][a]);
        }
      // stage 2
      float alpha_h;
      const void *bh = record_set<DIM, MODE>(m, i, t + hh, alpha_h);
      eval_group<DIM, BLEND, STORAGE>(m, bh, alpha_h, cs, ds, uc, du);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        accc[a] += 2.0 * (double)uc[a];
        cs[a] = c[a] + hh * (double)uc[a];
      }
#pragma unroll
      for (int k = 0; k < K; ++k)
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          accd[k][a] = fmaf(2.0f, du[k][a], accd[k][a]);
          ds[k][a] = fmaf(hhf, du[k][a], d[k][a]);
        }
      // stage 3
      eval_group<DIM, BLEND, STORAGE>(m, bh, alpha_h, cs, ds, uc, du);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        accc[a] += 2.0 * (double)uc[a];
        cs[a] = c[a] + h * (double)uc[a];
      }
#pragma unroll
      for (int k = 0; k < K; ++k)
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          accd[k][a] = fmaf(2.0f, du[k][a], accd[k][a]);
          ds[k][a] = fmaf(hf, du[k][a], d[k][a]);
        }
      // stage 4
      float alpha_f;
      const void *bf = record_set<DIM, MODE>(m, i, t + h, alpha_f);
      eval_group<DIM, BLEND, STORAGE>(m, bf, alpha_f, cs, ds, uc, du);
      const double h6 = h / 6.0;
      const float h6f = (float)h6;
#pragma unroll
      for (int a = 0; a < DIM; ++a) c[a] += h6 * (accc[a] + (double)uc[a]);
#pragma unroll
      for (int k = 0; k < K; ++k)
#pragma unroll
        for (int a = 0; a < DIM; ++a) d[k][a] = fmaf(h6f, accd[k][a] + du[k][a], d[k][a]);
    }
  }

  // final positions x_k = c + d_k (FP64)
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int a = 0; a < DIM; ++a)
      m.w.positions[((long long)k * N + g) * DIM + a] = c[a] + (double)d[k][a];

  if (m.w.ftle != nullptr) {
    double J[DIM][DIM];
#pragma unroll
    for (int i = 0; i < DIM; ++i)
#pragma unroll
      for (int j = 0; j < DIM; ++j)
        J[i][j] = ((double)d[plus_r(j)][i] - (double)d[minus_r(j)][i]) / id[j];
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
    m.w.ftle[g] = (1.0 / m.w.map_period) * log(sqrt(lam));
  }
}

template <int DIM, int MODE, int STORAGE>
static void launch_mixed(const MixK &m, int integ, cudaStream_t st) {
  const unsigned blocks = (unsigned)((m.w.N + 127) / 128);
  if (integ == FTLE_EULER)
    window_mixed_kernel<DIM, MODE, FTLE_EULER, STORAGE><<<blocks, 128, 0, st>>>(m);
  else if (integ == FTLE_AB2)
    window_mixed_kernel<DIM, MODE, FTLE_AB2, STORAGE><<<blocks, 128, 0, st>>>(m);
  else
    window_mixed_kernel<DIM, MODE, FTLE_RK4, STORAGE><<<blocks, 128, 0, st>>>(m);
}

template <int DIM, int MODE>
static void launch_mixed_s(const MixK &m, int integ, int storage, cudaStream_t st) {
  if (storage == FTLE_F16)
    launch_mixed<DIM, MODE, FTLE_F16>(m, integ, st);
  else
    launch_mixed<DIM, MODE, FTLE_BF16>(m, integ, st);
}

}  // namespace ftle

using namespace ftle;

extern "C" int ftle_window_run_mixed(const ftle_window *w, void *stream) {
  MixK m;
  int rc = window_to_kernel(w, &m.w);
  if (rc) return rc;
  if (w->storage != FTLE_F16 && w->storage != FTLE_BF16)
    return fail_invalid("ftle_window_run_mixed needs FTLE_F16 or FTLE_BF16 storage");
  if (m.w.N == 0) return FTLE_OK;
  for (int a = 0; a < 3; ++a) {
    m.inv_sp[a] = 1.0 / m.w.g.spacing[a];
    m.inv_spf[a] = (float)m.inv_sp[a];
  }
  m.inv_dt = 1.0 / (w->snapshot_dt != 0.0 ? w->snapshot_dt : 1.0);
  cudaStream_t st = as_stream(stream);
  if (w->grid.dim == 2) {
    if (w->time_mode == FTLE_HOLD)
      launch_mixed_s<2, FTLE_HOLD>(m, w->integrator, w->storage, st);
    else
      launch_mixed_s<2, FTLE_BLEND>(m, w->integrator, w->storage, st);
  } else {
    if (w->time_mode == FTLE_HOLD)
      launch_mixed_s<3, FTLE_HOLD>(m, w->integrator, w->storage, st);
    else
      launch_mixed_s<3, FTLE_BLEND>(m, w->integrator, w->storage, st);
  }
  return check_launch("window_mixed_kernel");
}
