// plain_f64.cu -- FP64 kernels with the reference's arithmetic (sm_100a).
//
// Compiled with -fmad=false: every multiply and add rounds on its own, as in
// pyFTLE's numpy / numba / generic-x86-64 C++ code, so HOLD-mode positions
// are bit-exact with the reference and BLEND-mode positions bit-exact with
// the CPU oracle.  Division and sqrt are IEEE (CUDA's FP64 defaults).
//
// Reference operations restated here (paths inside pyFTLE):
//   physical -> index  grid_interp.py:76-81, 163-168   ((x - min) / delta)
//   bilinear           GridInterp.cpp:93-142           (operand order :136-137)
//   trilinear          GridInterp.cpp:15-91            (lerp x, then y, then z)
//   Euler / AB2 / RK4  integrate.py:16-109, 177-342
//   Jacobian           cauchy_green.py:15-76, 79-153
//   CG, lambda, FTLE   ftle.py:9-233
#include <math.h>

#include "common.cuh"

namespace ftle {

// ---------------------------------------------------------------------------
// cell location and interpolation (bit-exact with the reference)
// ---------------------------------------------------------------------------

template <int DIM>
struct Cell64 {
  int i0[DIM], i1[DIM];
  double f[DIM];
};

// (x - origin)/spacing per axis, then GridInterp.cpp's floor and "x0 >= 0 &&
// x0+1 < n" test, written as 0 <= p < n-1 (equal for every finite p, and it
// also rejects NaN / inf, which the reference rejects through the INT_MIN its
// float->int conversion returns).  Periodic grids wrap the cell instead.
template <int DIM>
__device__ __forceinline__ bool locate64(const GridK &g, const double *x, Cell64<DIM> &c) {
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    const double p = (x[a] - g.origin[a]) / g.spacing[a];
    if (g.periodic) {
      const double fl = floor(p);
      if (!(fabs(fl) < 1.0e9)) return false;
      c.f[a] = p - fl;
      const int q = wrap_index((int)fl, g.n[a]);
      c.i0[a] = q;
      c.i1[a] = (q + 1 == g.n[a]) ? 0 : q + 1;
    } else {
      if (!(p >= 0.0 && p < (double)(g.n[a] - 1))) return false;
      const int q = (int)floor(p);
      c.i0[a] = q;
      c.i1[a] = q + 1;
      c.f[a] = p - (double)q;
    }
  }
  return true;
}

// Corner node ids in the reference's operand order:
//   2D v00 v10 v01 v11;  3D x0y0z0 x1y0z0 x0y0z1 x1y0z1 x0y1z0 x1y1z0 x0y1z1 x1y1z1
template <int DIM>
__device__ __forceinline__ void corners(const GridK &g, const Cell64<DIM> &c,
                                        long long *nd) {
  if constexpr (DIM == 2) {
    nd[0] = node2(g, c.i0[0], c.i0[1]);
    nd[1] = node2(g, c.i1[0], c.i0[1]);
    nd[2] = node2(g, c.i0[0], c.i1[1]);
    nd[3] = node2(g, c.i1[0], c.i1[1]);
  } else {
    nd[0] = node3(g, c.i0[0], c.i0[1], c.i0[2]);
    nd[1] = node3(g, c.i1[0], c.i0[1], c.i0[2]);
    nd[2] = node3(g, c.i0[0], c.i0[1], c.i1[2]);
    nd[3] = node3(g, c.i1[0], c.i0[1], c.i1[2]);
    nd[4] = node3(g, c.i0[0], c.i1[1], c.i0[2]);
    nd[5] = node3(g, c.i1[0], c.i1[1], c.i0[2]);
    nd[6] = node3(g, c.i0[0], c.i1[1], c.i1[2]);
    nd[7] = node3(g, c.i1[0], c.i1[1], c.i1[2]);
  }
}

__device__ __forceinline__ double bilinear(double v00, double v10, double v01, double v11,
                                           double xd, double yd) {
  return v00 * (1.0 - xd) * (1.0 - yd) + v10 * xd * (1.0 - yd) + v01 * (1.0 - xd) * yd +
         v11 * xd * yd;
}

__device__ __forceinline__ double trilinear(const double *v, double xd, double yd, double zd) {
  const double c00 = v[0] * (1.0 - xd) + v[1] * xd;
  const double c01 = v[2] * (1.0 - xd) + v[3] * xd;
  const double c10 = v[4] * (1.0 - xd) + v[5] * xd;
  const double c11 = v[6] * (1.0 - xd) + v[7] * xd;
  const double c0 = c00 * (1.0 - yd) + c10 * yd;
  const double c1 = c01 * (1.0 - yd) + c11 * yd;
  return c0 * (1.0 - zd) + c1 * zd;
}

template <int DIM>
__device__ __forceinline__ double interp_corners(const double *v, const double *f) {
  if constexpr (DIM == 2)
    return bilinear(v[0], v[1], v[2], v[3], f[0], f[1]);
  else
    return trilinear(v, f[0], f[1], f[2]);
}

// Velocity from one reference-layout (dim, nodes) snapshot.
template <int DIM>
__device__ __forceinline__ void velocity_planar(const GridK &g, const double *__restrict__ snap,
                                                const double *x, double *u) {
  Cell64<DIM> c;
  if (!locate64<DIM>(g, x, c)) {
#pragma unroll
    for (int a = 0; a < DIM; ++a) u[a] = 0.0;
    return;
  }
  long long nd[1 << DIM];
  corners<DIM>(g, c, nd);
#pragma unroll
  for (int comp = 0; comp < DIM; ++comp) {
    const double *s = snap + (long long)comp * g.nodes;
    double v[1 << DIM];
#pragma unroll
    for (int q = 0; q < (1 << DIM); ++q) v[q] = __ldg(s + nd[q]);
    u[comp] = interp_corners<DIM>(v, c.f);
  }
}

// ---------------------------------------------------------------------------
// packed FP64 snapshot records: record (s, node) = [snapshot s | successor]
// ---------------------------------------------------------------------------

// HOLD: only the first half is read.  2D record = 4 doubles, 3D = 6 doubles
// (48 bytes, so every record is 16-byte aligned).
template <int DIM, bool BLEND>
__device__ __forceinline__ void velocity_packed(const GridK &g, const double *__restrict__ rec,
                                                double alpha, const double *x, double *u) {
  Cell64<DIM> c;
  if (!locate64<DIM>(g, x, c)) {
#pragma unroll
    for (int a = 0; a < DIM; ++a) u[a] = 0.0;
    return;
  }
  long long nd[1 << DIM];
  corners<DIM>(g, c, nd);
  double v[DIM][1 << DIM];
  const double oma = 1.0 - alpha;
#pragma unroll
  for (int q = 0; q < (1 << DIM); ++q) {
    const double *r = rec + nd[q] * (2 * DIM);
    if constexpr (DIM == 2) {
      const double2 a = __ldg(reinterpret_cast<const double2 *>(r));
      if constexpr (BLEND) {
        const double2 b = __ldg(reinterpret_cast<const double2 *>(r) + 1);
        v[0][q] = a.x * oma + b.x * alpha;
        v[1][q] = a.y * oma + b.y * alpha;
      } else {
        v[0][q] = a.x;
        v[1][q] = a.y;
      }
    } else {
      const double2 a = __ldg(reinterpret_cast<const double2 *>(r));
      if constexpr (BLEND) {
        const double2 m = __ldg(reinterpret_cast<const double2 *>(r) + 1);
        const double2 b = __ldg(reinterpret_cast<const double2 *>(r) + 2);
        v[0][q] = a.x * oma + m.y * alpha;
        v[1][q] = a.y * oma + b.x * alpha;
        v[2][q] = m.x * oma + b.y * alpha;
      } else {
        v[0][q] = a.x;
        v[1][q] = a.y;
        v[2][q] = __ldg(r + 2);
      }
    }
  }
#pragma unroll
  for (int comp = 0; comp < DIM; ++comp) u[comp] = interp_corners<DIM>(v[comp], c.f);
}

// ---------------------------------------------------------------------------
// time lookup (BLEND)
// ---------------------------------------------------------------------------

// Snapshot record and blend weight at time t (record s pairs s with its successor).
__device__ __forceinline__ void time_pair(const WinK &w, double t, int &s0, double &alpha) {
  double tau = (t - w.snap_t0) / w.snap_dt;
  const int S = w.num_snaps;
  if (w.periodic_time) {
    tau = tau - (double)S * floor(tau / (double)S);
    int s = (int)floor(tau);
    s = s >= S ? S - 1 : (s < 0 ? 0 : s);
    s0 = s;
    alpha = tau - (double)s;
  } else if (!(tau > 0.0)) {
    s0 = 0;
    alpha = 0.0;
  } else if (tau >= (double)(S - 1)) {
    s0 = S - 2;
    alpha = 1.0;
  } else {
    const int s = (int)floor(tau);
    s0 = s;
    alpha = tau - (double)s;
  }
}

template <int DIM, int MODE>
__device__ __forceinline__ void field(const WinK &w, int step, double t, const double *x,
                                      double *u) {
  const long long rec_set = w.g.nodes * (2 * DIM);
  if constexpr (MODE == FTLE_HOLD) {
    int s = w.first_snapshot + step;
    if (w.periodic_time) s %= w.num_snaps;
    velocity_packed<DIM, false>(w.g, static_cast<const double *>(w.snaps) + (long long)s * rec_set, 0.0, x, u);
  } else {
    int s0;
    double alpha;
    time_pair(w, t, s0, alpha);
    velocity_packed<DIM, true>(w.g, static_cast<const double *>(w.snaps) + (long long)s0 * rec_set, alpha, x, u);
  }
}

// One particle through the whole window (integrate.py restated step by step).
template <int DIM, int MODE, int INTEG>
__device__ __forceinline__ void advect(const WinK &w, double *x) {
  const double h = w.h;
  double vprev[DIM];
  for (int i = 0; i < w.num_steps; ++i) {
    const double t = w.t0 + (double)i * h;
    if constexpr (INTEG == FTLE_EULER) {
      double v[DIM];
      field<DIM, MODE>(w, i, t, x, v);
#pragma unroll
      for (int a = 0; a < DIM; ++a) x[a] = x[a] + h * v[a];
    } else if constexpr (INTEG == FTLE_AB2) {
      double v[DIM];
      field<DIM, MODE>(w, i, t, x, v);
      if (i == 0) {
#pragma unroll
        for (int a = 0; a < DIM; ++a) x[a] = x[a] + h * v[a];
      } else {
#pragma unroll
        for (int a = 0; a < DIM; ++a) x[a] = x[a] + h * (1.5 * v[a] - 0.5 * vprev[a]);
      }
#pragma unroll
      for (int a = 0; a < DIM; ++a) vprev[a] = v[a];
    } else {
      const double hh = 0.5 * h;
      const double th = t + 0.5 * h, tf = t + h;
      double k[DIM], acc[DIM], tmp[DIM];
      field<DIM, MODE>(w, i, t, x, k);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        acc[a] = k[a];
        tmp[a] = x[a] + hh * k[a];
      }
      field<DIM, MODE>(w, i, th, tmp, k);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        acc[a] = acc[a] + 2.0 * k[a];
        tmp[a] = x[a] + hh * k[a];
      }
      field<DIM, MODE>(w, i, th, tmp, k);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        acc[a] = acc[a] + 2.0 * k[a];
        tmp[a] = x[a] + h * k[a];
      }
      field<DIM, MODE>(w, i, tf, tmp, k);
      const double h6 = h / 6.0;
#pragma unroll
      for (int a = 0; a < DIM; ++a) x[a] = x[a] + h6 * (acc[a] + k[a]);
    }
  }
}

// ---------------------------------------------------------------------------
// FTLE epilogue
// ---------------------------------------------------------------------------

// ftle.py:122-163 on C = F^T F (ftle.py:62-67).
__device__ __forceinline__ double lambda_max_2x2(double F00, double F01, double F10, double F11) {
  const double A = F00 * F00 + F10 * F10;
  const double B = F00 * F01 + F10 * F11;
  const double C = F01 * F00 + F11 * F10;
  const double D = F01 * F01 + F11 * F11;
  const double trace = A + D;
  const double det = A * D - B * C;
  const double l1 = 0.5 * (trace + sqrt(trace * trace - 4.0 * det));
  const double l2 = 0.5 * (trace - sqrt(trace * trace - 4.0 * det));
  return (l2 > l1) ? l2 : l1;
}

// Largest eigenvalue of a symmetric 3x3 matrix by cyclic Jacobi rotations
// (the reference takes max(np.linalg.eigvals(C)), ftle.py:118-119).
__device__ __forceinline__ double sym3_lambda_max(double a00, double a01, double a02,
                                                  double a11, double a12, double a22) {
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
  double m = a[0][0];
  if (a[1][1] > m) m = a[1][1];
  if (a[2][2] > m) m = a[2][2];
  return m;
}

// C = F F^T (ftle.py:96) then lambda_max.
__device__ __forceinline__ double lambda_max_3x3(const double J[3][3]) {
  double C[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      C[i][k] = J[i][0] * J[k][0] + J[i][1] * J[k][1] + J[i][2] * J[k][2];
  return sym3_lambda_max(C[0][0], C[0][1], C[0][2], C[1][1], C[1][2], C[2][2]);
}

__device__ __forceinline__ double ftle_value(double lambda, double map_period) {
  return (1.0 / map_period) * log(sqrt(lambda));
}

// Role pairs of the Jacobian columns: (right, left), (top, bottom), (front, back).
__device__ __forceinline__ int plus_role(int j) { return j == 0 ? 1 : 2 * j; }
__device__ __forceinline__ int minus_role(int j) { return j == 0 ? 0 : 2 * j + 1; }

// FTLE of one group from its K final positions P[role][a] and initial diagonal
// separations id[j] (right-left x, top-bottom y, front-back z).
template <int DIM>
__device__ __forceinline__ double group_ftle(const double (*P)[DIM], const double *id,
                                             double map_period) {
  double J[DIM][DIM];
#pragma unroll
  for (int i = 0; i < DIM; ++i)
#pragma unroll
    for (int j = 0; j < DIM; ++j) J[i][j] = (P[plus_role(j)][i] - P[minus_role(j)][i]) / id[j];
  if constexpr (DIM == 2)
    return ftle_value(lambda_max_2x2(J[0][0], J[0][1], J[1][0], J[1][1]), map_period);
  else
    return ftle_value(lambda_max_3x3(J), map_period);
}

// ---------------------------------------------------------------------------
// fused window kernel: one thread per particle, G groups per block
// ---------------------------------------------------------------------------
template <int DIM, int MODE, int INTEG, int G>
__device__ __forceinline__ void window_f64_body(const WinK &w) {
  constexpr int K = 2 * DIM;
  const int tid = threadIdx.x;
  // role-minor: a warp holds every neighbour of a few groups, whose gathers mostly read
  // the same cell's records, so a load touches a few lines instead of 32 (a warp of one
  // role over 32 groups ran 1.36x slower in 3D BLEND, 1.24x in 2D HOLD); the
  // per-particle arithmetic is the same either way
  const int role = tid % K, gl = tid / K;
  const long long g = (long long)blockIdx.x * G + gl;
  const bool active = g < w.N;
  const long long row = (long long)role * w.N + g;
  double x[DIM], x0[DIM];
#pragma unroll
  for (int a = 0; a < DIM; ++a) x[a] = x0[a] = 0.0;
  if (active) {
#pragma unroll
    for (int a = 0; a < DIM; ++a) x[a] = x0[a] = w.positions[row * DIM + a];
    advect<DIM, MODE, INTEG>(w, x);
    if (!w.keep_positions) {
#pragma unroll
      for (int a = 0; a < DIM; ++a) w.positions[row * DIM + a] = x[a];
    }
  }
  if (w.ftle != nullptr) {  // uniform across the block
    __shared__ double sx[K][G][DIM];
    __shared__ double sx0[K][G][DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      sx[role][gl][a] = x[a];
      sx0[role][gl][a] = x0[a];
    }
    __syncthreads();
    if (tid < G) {
      const long long gg = (long long)blockIdx.x * G + tid;
      if (gg < w.N) {
        double P[K][DIM];
        double id[DIM];
#pragma unroll
        for (int r = 0; r < K; ++r)
#pragma unroll
          for (int a = 0; a < DIM; ++a) P[r][a] = sx[r][tid][a];
#pragma unroll
        for (int j = 0; j < DIM; ++j) id[j] = sx0[plus_role(j)][tid][j] - sx0[minus_role(j)][tid][j];
        w.ftle[gg] = group_ftle<DIM>(P, id, w.map_period);
      }
    }
  }
}

template <int DIM, int MODE, int INTEG, int G>
__global__ void __launch_bounds__(2 * DIM * G) window_f64_kernel(const WinK w) {
  window_f64_body<DIM, MODE, INTEG, G>(w);
}

// 2D HOLD (the reference's own semantics) with the register budget of 5 blocks per SM:
// 1.08x faster there than the compiler's own choice; the other instantiations spill at a
// tighter budget (2D BLEND 1.14x and 3D BLEND 1.01x slower at 5 / 4 blocks), so they keep
// theirs.
template <int INTEG, int G>
__global__ void __launch_bounds__(4 * G, 5) window_f64_hold2d_kernel(const WinK w) {
  window_f64_body<2, FTLE_HOLD, INTEG, G>(w);
}

// ---------------------------------------------------------------------------
// closed-form velocity fields (the "analytical" interpolator on the device)
// ---------------------------------------------------------------------------

struct FlowK {
  int kind;
  double p[8];
};

// Double gyre, in the operand order of pyFTLE's example velocity_fn:
//   f = eps sin(wt) x^2 + (1 - 2 eps sin(wt)) x,  u = -pi A sin(pi f) cos(pi y),
//   v = pi A cos(pi f) sin(pi y) df/dx.
// Time-periodic ABC: A(t) = A + a sin(w t), u = A(t) sin z + C cos y,
//   v = B sin x + A(t) cos z, w = C sin y + B cos x.
template <int DIM>
__device__ __forceinline__ void flow_velocity(const FlowK &f, double t, const double *x,
                                              double *u) {
  if constexpr (DIM == 2) {
    const double A = f.p[0], eps = f.p[1], om = f.p[2];
    const double s = sin(om * t);
    const double xx = x[0], yy = x[1];
    const double ff = eps * s * (xx * xx) + (1.0 - 2.0 * eps * s) * xx;
    const double dfdx = 2.0 * eps * s * xx + (1.0 - 2.0 * eps * s);
    const double pi = 3.141592653589793;
    u[0] = -pi * A * sin(pi * ff) * cos(pi * yy);
    u[1] = pi * A * cos(pi * ff) * sin(pi * yy) * dfdx;
  } else {
    const double At = f.p[0] + f.p[3] * sin(f.p[4] * t);
    const double B = f.p[1], C = f.p[2];
    u[0] = At * sin(x[2]) + C * cos(x[1]);
    u[1] = B * sin(x[0]) + At * cos(x[2]);
    u[2] = C * sin(x[1]) + B * cos(x[0]);
  }
}

template <int DIM, int INTEG>
__device__ __forceinline__ void advect_analytic(const FlowK &f, double t0, double h, int steps,
                                                int freeze, double *x) {
  double vprev[DIM];
  for (int i = 0; i < steps; ++i) {
    const double t = freeze ? 0.0 : t0 + (double)i * h;
    if constexpr (INTEG == FTLE_EULER || INTEG == FTLE_AB2) {
      double v[DIM];
      flow_velocity<DIM>(f, t, x, v);
      if (INTEG == FTLE_EULER || i == 0) {
#pragma unroll
        for (int a = 0; a < DIM; ++a) x[a] = x[a] + h * v[a];
      } else {
#pragma unroll
        for (int a = 0; a < DIM; ++a) x[a] = x[a] + h * (1.5 * v[a] - 0.5 * vprev[a]);
      }
#pragma unroll
      for (int a = 0; a < DIM; ++a) vprev[a] = v[a];
    } else {
      const double hh = 0.5 * h;
      const double th = freeze ? 0.0 : t + 0.5 * h, tf = freeze ? 0.0 : t + h;
      double k[DIM], acc[DIM], tmp[DIM];
      flow_velocity<DIM>(f, t, x, k);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        acc[a] = k[a];
        tmp[a] = x[a] + hh * k[a];
      }
      flow_velocity<DIM>(f, th, tmp, k);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        acc[a] = acc[a] + 2.0 * k[a];
        tmp[a] = x[a] + hh * k[a];
      }
      flow_velocity<DIM>(f, th, tmp, k);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        acc[a] = acc[a] + 2.0 * k[a];
        tmp[a] = x[a] + h * k[a];
      }
      flow_velocity<DIM>(f, tf, tmp, k);
      const double h6 = h / 6.0;
#pragma unroll
      for (int a = 0; a < DIM; ++a) x[a] = x[a] + h6 * (acc[a] + k[a]);
    }
  }
}

template <int DIM, int INTEG, int G>
__global__ void __launch_bounds__(2 * DIM * G)
    analytic_window_kernel(const FlowK f, double t0, double h, int steps, int freeze,
                           double *positions, long long N, double map_period, double *ftle) {
  constexpr int K = 2 * DIM;
  const int tid = threadIdx.x;
  const int role = tid / G, gl = tid % G;
  const long long g = (long long)blockIdx.x * G + gl;
  const bool active = g < N;
  const long long row = (long long)role * N + g;
  double x[DIM], x0[DIM];
#pragma unroll
  for (int a = 0; a < DIM; ++a) x[a] = x0[a] = 0.0;
  if (active) {
#pragma unroll
    for (int a = 0; a < DIM; ++a) x[a] = x0[a] = positions[row * DIM + a];
    advect_analytic<DIM, INTEG>(f, t0, h, steps, freeze, x);
#pragma unroll
    for (int a = 0; a < DIM; ++a) positions[row * DIM + a] = x[a];
  }
  if (ftle != nullptr) {
    __shared__ double sx[K][G][DIM];
    __shared__ double sx0[K][G][DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      sx[role][gl][a] = x[a];
      sx0[role][gl][a] = x0[a];
    }
    __syncthreads();
    if (tid < G) {
      const long long gg = (long long)blockIdx.x * G + tid;
      if (gg < N) {
        double P[K][DIM];
        double id[DIM];
#pragma unroll
        for (int r = 0; r < K; ++r)
#pragma unroll
          for (int a = 0; a < DIM; ++a) P[r][a] = sx[r][tid][a];
#pragma unroll
        for (int j = 0; j < DIM; ++j)
          id[j] = sx0[plus_role(j)][tid][j] - sx0[minus_role(j)][tid][j];
        ftle[gg] = group_ftle<DIM>(P, id, map_period);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// per-step kernels (compatibility path of the Integrator / Interpolator API)
// ---------------------------------------------------------------------------

__global__ void interp2d_kernel(const double *__restrict__ v, int nx, int ny,
                                const double *__restrict__ pts, long long n, double *out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double px = pts[i * 2 + 0], py = pts[i * 2 + 1];
    double c = 0.0;
    if (px >= 0.0 && px < (double)(nx - 1) && py >= 0.0 && py < (double)(ny - 1)) {
      const int x0 = (int)floor(px), y0 = (int)floor(py);
      const double xd = px - (double)x0, yd = py - (double)y0;
      const long long b = (long long)x0 * ny + y0;
      c = bilinear(__ldg(v + b), __ldg(v + b + ny), __ldg(v + b + 1), __ldg(v + b + ny + 1), xd,
                   yd);
    }
    out[i] = c;
  }
}

__global__ void interp3d_kernel(const double *__restrict__ v, int X, int Y, int Z,
                                const double *__restrict__ pts, long long n, double *out) {
  const long long YZ = (long long)Y * Z;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double px = pts[i * 3 + 0], py = pts[i * 3 + 1], pz = pts[i * 3 + 2];
    double c = 0.0;
    if (px >= 0.0 && px < (double)(X - 1) && py >= 0.0 && py < (double)(Y - 1) && pz >= 0.0 &&
        pz < (double)(Z - 1)) {
      const int x0 = (int)floor(px), y0 = (int)floor(py), z0 = (int)floor(pz);
      const double xd = px - (double)x0, yd = py - (double)y0, zd = pz - (double)z0;
      const long long b = (long long)x0 * YZ + (long long)y0 * Z + z0;
      double vv[8];
      vv[0] = __ldg(v + b);                // x0y0z0
      vv[1] = __ldg(v + b + YZ);           // x1y0z0
      vv[2] = __ldg(v + b + 1);            // x0y0z1
      vv[3] = __ldg(v + b + YZ + 1);       // x1y0z1
      vv[4] = __ldg(v + b + Z);            // x0y1z0
      vv[5] = __ldg(v + b + YZ + Z);       // x1y1z0
      vv[6] = __ldg(v + b + Z + 1);        // x0y1z1
      vv[7] = __ldg(v + b + YZ + Z + 1);   // x1y1z1
      c = trilinear(vv, xd, yd, zd);
    }
    out[i] = c;
  }
}

template <int DIM>
__global__ void grid_interpolate_kernel(const GridK g, const double *__restrict__ snap,
                                        const double *__restrict__ pts, long long m,
                                        double *out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x) {
    double x[DIM], u[DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a) x[a] = pts[i * DIM + a];
    velocity_planar<DIM>(g, snap, x, u);
#pragma unroll
    for (int a = 0; a < DIM; ++a) out[i * DIM + a] = u[a];
  }
}

template <int DIM, int INTEG>
__global__ void grid_step_kernel(const GridK g, const double *__restrict__ snap, double h,
                                 double *pos, long long m, double *hist, int hist_valid) {
  // RK4 with m = K*N (role-blocked neighbour groups): work item j takes role j mod K of
  // group j / K, so a warp holds every neighbour of a few groups and their four stages'
  // gathers share cells (3D 2.95x, 2D 1.31x faster); each particle is still advected
  // once, by the same arithmetic.  Euler / AB2 evaluate once per step and are bound by
  // streaming positions (and history), which that order makes strided (3D 1.5x slower),
  // so they keep the particle order.
  constexpr int K = 2 * DIM;
  const long long ng = (INTEG == FTLE_RK4 && m % K == 0) ? m / K : 0;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < m;
       j += (long long)gridDim.x * blockDim.x) {
    const long long i = ng ? (j % K) * ng + j / K : j;
    double x[DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a) x[a] = pos[i * DIM + a];
    if constexpr (INTEG == FTLE_EULER) {
      double v[DIM];
      velocity_planar<DIM>(g, snap, x, v);
#pragma unroll
      for (int a = 0; a < DIM; ++a) x[a] = x[a] + h * v[a];
    } else if constexpr (INTEG == FTLE_AB2) {
      double v[DIM];
      velocity_planar<DIM>(g, snap, x, v);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        if (hist_valid)
          x[a] = x[a] + h * (1.5 * v[a] - 0.5 * hist[i * DIM + a]);
        else
          x[a] = x[a] + h * v[a];
        hist[i * DIM + a] = v[a];
      }
    } else {
      const double hh = 0.5 * h;
      double k[DIM], acc[DIM], tmp[DIM];
      velocity_planar<DIM>(g, snap, x, k);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        acc[a] = k[a];
        tmp[a] = x[a] + hh * k[a];
      }
      velocity_planar<DIM>(g, snap, tmp, k);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        acc[a] = acc[a] + 2.0 * k[a];
        tmp[a] = x[a] + hh * k[a];
      }
      velocity_planar<DIM>(g, snap, tmp, k);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        acc[a] = acc[a] + 2.0 * k[a];
        tmp[a] = x[a] + h * k[a];
      }
      velocity_planar<DIM>(g, snap, tmp, k);
      const double h6 = h / 6.0;
#pragma unroll
      for (int a = 0; a < DIM; ++a) x[a] = x[a] + h6 * (acc[a] + k[a]);
    }
#pragma unroll
    for (int a = 0; a < DIM; ++a) pos[i * DIM + a] = x[a];
  }
}

__global__ void axpy_kernel(double *out, const double *x, double a, const double *k, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = x[i] + a * k[i];
}

__global__ void ab2_kernel(double *x, double h, const double *v, const double *vp, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = x[i] + h * (1.5 * v[i] - 0.5 * vp[i]);
}

__global__ void rk4_kernel(double *x, double h6, const double *k1, const double *k2,
                           const double *k3, const double *k4, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = x[i] + h6 * (((k1[i] + 2.0 * k2[i]) + 2.0 * k3[i]) + k4[i]);
}

// ---------------------------------------------------------------------------
// FTLE building blocks
// ---------------------------------------------------------------------------

template <int DIM>
__global__ void jacobian_kernel(const double *__restrict__ pos, const double *__restrict__ idl,
                                long long N, double *J) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < N;
       g += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int i = 0; i < DIM; ++i)
#pragma unroll
      for (int j = 0; j < DIM; ++j) {
        const double d = pos[((long long)plus_role(j) * N + g) * DIM + i] -
                         pos[((long long)minus_role(j) * N + g) * DIM + i];
        J[(g * DIM + i) * DIM + j] = d / idl[((long long)j * N + g) * DIM + j];
      }
  }
}

template <int DIM>
__global__ void cauchy_green_kernel(const double *__restrict__ J, long long n, double *C) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n;
       g += (long long)gridDim.x * blockDim.x) {
    const double *F = J + g * DIM * DIM;
    double *c = C + g * DIM * DIM;
    if constexpr (DIM == 2) {  // C = F^T F, ftle.py:62-67
      c[0] = F[0] * F[0] + F[2] * F[2];
      c[1] = F[0] * F[1] + F[2] * F[3];
      c[2] = F[1] * F[0] + F[3] * F[2];
      c[3] = F[1] * F[1] + F[3] * F[3];
    } else {  // C = F F^T, ftle.py:96
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k)
          c[i * 3 + k] = F[i * 3 + 0] * F[k * 3 + 0] + F[i * 3 + 1] * F[k * 3 + 1] +
                         F[i * 3 + 2] * F[k * 3 + 2];
    }
  }
}

template <int DIM>
__global__ void max_eigenvalue_kernel(const double *__restrict__ C, long long n, double *out) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n;
       g += (long long)gridDim.x * blockDim.x) {
    const double *c = C + g * DIM * DIM;
    if constexpr (DIM == 2) {  // ftle.py:146-161 on (A, B, C, D)
      const double trace = c[0] + c[3];
      const double det = c[0] * c[3] - c[1] * c[2];
      const double l1 = 0.5 * (trace + sqrt(trace * trace - 4.0 * det));
      const double l2 = 0.5 * (trace - sqrt(trace * trace - 4.0 * det));
      out[g] = (l2 > l1) ? l2 : l1;
    } else {  // symmetric part (exact for a symmetric C)
      out[g] = sym3_lambda_max(c[0], 0.5 * (c[1] + c[3]), 0.5 * (c[2] + c[6]), c[4],
                               0.5 * (c[5] + c[7]), c[8]);
    }
  }
}

template <int DIM>
__global__ void ftle_from_jacobian_kernel(const double *__restrict__ J, long long n,
                                          double map_period, double *out) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n;
       g += (long long)gridDim.x * blockDim.x) {
    const double *F = J + g * DIM * DIM;
    if constexpr (DIM == 2) {
      out[g] = ftle_value(lambda_max_2x2(F[0], F[1], F[2], F[3]), map_period);
    } else {
      double M[3][3];
#pragma unroll
      for (int i = 0; i < 9; ++i) M[i / 3][i % 3] = F[i];
      out[g] = ftle_value(lambda_max_3x3(M), map_period);
    }
  }
}

template <int DIM>
__global__ void ftle_from_positions_kernel(const double *__restrict__ pos,
                                           const double *__restrict__ idl, long long N,
                                           double map_period, double *out) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < N;
       g += (long long)gridDim.x * blockDim.x) {
    double P[2 * DIM][DIM];
    double id[DIM];
#pragma unroll
    for (int r = 0; r < 2 * DIM; ++r)
#pragma unroll
      for (int a = 0; a < DIM; ++a) P[r][a] = pos[((long long)r * N + g) * DIM + a];
#pragma unroll
    for (int j = 0; j < DIM; ++j) id[j] = idl[((long long)j * N + g) * DIM + j];
    out[g] = group_ftle<DIM>(P, id, map_period);
  }
}

// ---------------------------------------------------------------------------
// FP64 snapshot packing: (S, dim, nodes) -> records (S, nodes, 2*dim)
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void pack_f64_kernel(const double *__restrict__ src, long long nodes, int S,
                                int periodic_time, double *dst) {
  const long long total = nodes * S;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(i / nodes);
    const long long p = i - (long long)s * nodes;
    const int s1 = (s + 1 < S) ? s + 1 : (periodic_time ? 0 : s);
    double *r = dst + i * (2 * DIM);
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      r[c] = src[((long long)s * DIM + c) * nodes + p];
      r[DIM + c] = src[((long long)s1 * DIM + c) * nodes + p];
    }
  }
}

// ---------------------------------------------------------------------------
// host entry points
// ---------------------------------------------------------------------------

template <int DIM, int MODE, int INTEG>
static void launch_window(const WinK &w, cudaStream_t st) {
  constexpr int G = DIM == 2 ? 64 : 32;
  const long long blocks = (w.N + G - 1) / G;
  if constexpr (DIM == 2 && MODE == FTLE_HOLD)
    window_f64_hold2d_kernel<INTEG, G><<<(unsigned)blocks, 2 * DIM * G, 0, st>>>(w);
  else
    window_f64_kernel<DIM, MODE, INTEG, G><<<(unsigned)blocks, 2 * DIM * G, 0, st>>>(w);
}

template <int DIM, int MODE>
static void launch_window_i(const WinK &w, int integ, cudaStream_t st) {
  if (integ == FTLE_EULER)
    launch_window<DIM, MODE, FTLE_EULER>(w, st);
  else if (integ == FTLE_AB2)
    launch_window<DIM, MODE, FTLE_AB2>(w, st);
  else
    launch_window<DIM, MODE, FTLE_RK4>(w, st);
}

}  // namespace ftle

using namespace ftle;

extern "C" {

int ftle_window_run_f64(const ftle_window *w, void *stream) {
  WinK k;
  int rc = window_to_kernel(w, &k);
  if (rc) return rc;
  if (w->storage != FTLE_F64) return fail_invalid("ftle_window_run_f64 needs FTLE_F64 storage");
  if (k.N == 0) return FTLE_OK;
  cudaStream_t st = as_stream(stream);
  const int dim = w->grid.dim;
  if (dim == 2) {
    if (w->time_mode == FTLE_HOLD)
      launch_window_i<2, FTLE_HOLD>(k, w->integrator, st);
    else
      launch_window_i<2, FTLE_BLEND>(k, w->integrator, st);
  } else {
    if (w->time_mode == FTLE_HOLD)
      launch_window_i<3, FTLE_HOLD>(k, w->integrator, st);
    else
      launch_window_i<3, FTLE_BLEND>(k, w->integrator, st);
  }
  return check_launch("window_f64_kernel");
}

int ftle_interp2d_vec_inplace(const double *v, int32_t nx, int32_t ny, const double *points,
                              int64_t n, double *out, void *stream) {
  if (n < 0) return fail_invalid("n must be >= 0");
  if (n == 0) return FTLE_OK;
  if (!v || !points || !out) return fail_invalid("null pointer");
  if (nx < 1 || ny < 1) return fail_invalid("v must be 2D with positive extents");
  interp2d_kernel<<<grid_blocks(n, 256), 256, 0, as_stream(stream)>>>(v, nx, ny, points, n, out);
  return check_launch("interp2d_kernel");
}

int ftle_interp3d_vec_inplace(const double *v, int32_t X, int32_t Y, int32_t Z,
                              const double *points, int64_t n, double *out, void *stream) {
  if (n < 0) return fail_invalid("n must be >= 0");
  if (n == 0) return FTLE_OK;
  if (!v || !points || !out) return fail_invalid("null pointer");
  if (X < 1 || Y < 1 || Z < 1) return fail_invalid("v must be 3D with positive extents");
  interp3d_kernel<<<grid_blocks(n, 256), 256, 0, as_stream(stream)>>>(v, X, Y, Z, points, n,
                                                                       out);
  return check_launch("interp3d_kernel");
}

int ftle_grid_interpolate(const ftle_grid *grid, const double *snapshot, const double *points,
                          int64_t m, double *out, void *stream) {
  GridK g;
  int rc = grid_from_abi(grid, &g);
  if (rc) return rc;
  if (m < 0) return fail_invalid("m must be >= 0");
  if (m == 0) return FTLE_OK;
  if (!snapshot || !points || !out) return fail_invalid("null pointer");
  cudaStream_t st = as_stream(stream);
  if (grid->dim == 2)
    grid_interpolate_kernel<2><<<grid_blocks(m, 256), 256, 0, st>>>(g, snapshot, points, m, out);
  else
    grid_interpolate_kernel<3><<<grid_blocks(m, 256), 256, 0, st>>>(g, snapshot, points, m, out);
  return check_launch("grid_interpolate_kernel");
}

int ftle_grid_step(const ftle_grid *grid, const double *snapshot, int32_t integrator, double h,
                   double *positions, int64_t m, double *history, int32_t history_valid,
                   void *stream) {
  GridK g;
  int rc = grid_from_abi(grid, &g);
  if (rc) return rc;
  if (m < 0) return fail_invalid("m must be >= 0");
  if (integrator < FTLE_EULER || integrator > FTLE_RK4)
    return fail_invalid("unknown integrator %d", integrator);
  if (integrator == FTLE_AB2 && !history && m > 0) return fail_invalid("AB2 needs a history buffer");
  if (m == 0) return FTLE_OK;
  if (!snapshot || !positions) return fail_invalid("null pointer");
  cudaStream_t st = as_stream(stream);
  const unsigned b = grid_blocks(m, 128);
#define STEP(D, I) grid_step_kernel<D, I><<<b, 128, 0, st>>>(g, snapshot, h, positions, m, history, history_valid)
  if (grid->dim == 2) {
    if (integrator == FTLE_EULER) STEP(2, FTLE_EULER);
    else if (integrator == FTLE_AB2) STEP(2, FTLE_AB2);
    else STEP(2, FTLE_RK4);
  } else {
    if (integrator == FTLE_EULER) STEP(3, FTLE_EULER);
    else if (integrator == FTLE_AB2) STEP(3, FTLE_AB2);
    else STEP(3, FTLE_RK4);
  }
#undef STEP
  return check_launch("grid_step_kernel");
}

int ftle_axpy(double *out, const double *x, double a, const double *k, int64_t n, void *stream) {
  if (n < 0) return fail_invalid("n must be >= 0");
  if (n == 0) return FTLE_OK;
  if (!out || !x || !k) return fail_invalid("null pointer");
  axpy_kernel<<<grid_blocks(n, 256), 256, 0, as_stream(stream)>>>(out, x, a, k, n);
  return check_launch("axpy_kernel");
}

int ftle_ab2_update(double *x, double h, const double *v, const double *v_prev, int64_t n,
                    void *stream) {
  if (n < 0) return fail_invalid("n must be >= 0");
  if (n == 0) return FTLE_OK;
  if (!x || !v || !v_prev) return fail_invalid("null pointer");
  ab2_kernel<<<grid_blocks(n, 256), 256, 0, as_stream(stream)>>>(x, h, v, v_prev, n);
  return check_launch("ab2_kernel");
}

int ftle_rk4_update(double *x, double h, const double *k1, const double *k2, const double *k3,
                    const double *k4, int64_t n, void *stream) {
  if (n < 0) return fail_invalid("n must be >= 0");
  if (n == 0) return FTLE_OK;
  if (!x || !k1 || !k2 || !k3 || !k4) return fail_invalid("null pointer");
  rk4_kernel<<<grid_blocks(n, 256), 256, 0, as_stream(stream)>>>(x, h / 6.0, k1, k2, k3, k4, n);
  return check_launch("rk4_kernel");
}

#define DIM_DISPATCH(dim, KERNEL, ...)                         \
  do {                                                         \
    if ((dim) == 2)                                            \
      KERNEL<2><<<b, 256, 0, as_stream(stream)>>>(__VA_ARGS__); \
    else                                                       \
      KERNEL<3><<<b, 256, 0, as_stream(stream)>>>(__VA_ARGS__); \
  } while (0)

int ftle_flow_map_jacobian(int32_t dim, const double *positions, const double *initial_deltas,
                           int64_t num_groups, double *jacobian, void *stream) {
  if (dim != 2 && dim != 3) return fail_invalid("dim must be 2 or 3");
  if (num_groups < 0) return fail_invalid("num_groups must be >= 0");
  if (num_groups == 0) return FTLE_OK;
  if (!positions || !initial_deltas || !jacobian) return fail_invalid("null pointer");
  const unsigned b = grid_blocks(num_groups, 256);
  DIM_DISPATCH(dim, jacobian_kernel, positions, initial_deltas, num_groups, jacobian);
  return check_launch("jacobian_kernel");
}

int ftle_cauchy_green(int32_t dim, const double *jacobian, int64_t n, double *cauchy_green,
                      void *stream) {
  if (dim != 2 && dim != 3) return fail_invalid("dim must be 2 or 3");
  if (n < 0) return fail_invalid("n must be >= 0");
  if (n == 0) return FTLE_OK;
  if (!jacobian || !cauchy_green) return fail_invalid("null pointer");
  const unsigned b = grid_blocks(n, 256);
  DIM_DISPATCH(dim, cauchy_green_kernel, jacobian, n, cauchy_green);
  return check_launch("cauchy_green_kernel");
}

int ftle_max_eigenvalue(int32_t dim, const double *cauchy_green, int64_t n, double *out,
                        void *stream) {
  if (dim != 2 && dim != 3) return fail_invalid("dim must be 2 or 3");
  if (n < 0) return fail_invalid("n must be >= 0");
  if (n == 0) return FTLE_OK;
  if (!cauchy_green || !out) return fail_invalid("null pointer");
  const unsigned b = grid_blocks(n, 256);
  DIM_DISPATCH(dim, max_eigenvalue_kernel, cauchy_green, n, out);
  return check_launch("max_eigenvalue_kernel");
}

int ftle_from_jacobian(int32_t dim, const double *jacobian, int64_t n, double map_period,
                       double *out, void *stream) {
  if (dim != 2 && dim != 3) return fail_invalid("dim must be 2 or 3");
  if (n < 0) return fail_invalid("n must be >= 0");
  if (!(map_period != 0.0)) return fail_invalid("map_period must be non-zero");
  if (n == 0) return FTLE_OK;
  if (!jacobian || !out) return fail_invalid("null pointer");
  const unsigned b = grid_blocks(n, 256);
  DIM_DISPATCH(dim, ftle_from_jacobian_kernel, jacobian, n, map_period, out);
  return check_launch("ftle_from_jacobian_kernel");
}

int ftle_from_positions(int32_t dim, const double *positions, const double *initial_deltas,
                        int64_t num_groups, double map_period, double *out, void *stream) {
  if (dim != 2 && dim != 3) return fail_invalid("dim must be 2 or 3");
  if (num_groups < 0) return fail_invalid("num_groups must be >= 0");
  if (!(map_period != 0.0)) return fail_invalid("map_period must be non-zero");
  if (num_groups == 0) return FTLE_OK;
  if (!positions || !initial_deltas || !out) return fail_invalid("null pointer");
  const unsigned b = grid_blocks(num_groups, 256);
  DIM_DISPATCH(dim, ftle_from_positions_kernel, positions, initial_deltas, num_groups,
               map_period, out);
  return check_launch("ftle_from_positions_kernel");
}

int ftle_analytic_window_run(const ftle_flow *flow, int32_t integrator, double t0, double h,
                             int32_t num_steps, int32_t freeze_time, double *positions,
                             int64_t num_groups, double map_period, double *ftle, void *stream) {
  if (!flow) return fail_invalid("flow descriptor is NULL");
  int dim;
  if (flow->kind == FTLE_FLOW_DOUBLE_GYRE)
    dim = 2;
  else if (flow->kind == FTLE_FLOW_ABC)
    dim = 3;
  else
    return fail_invalid("unknown flow kind %d", flow->kind);
  if (integrator < FTLE_EULER || integrator > FTLE_RK4)
    return fail_invalid("unknown integrator %d", integrator);
  if (num_steps < 0 || num_groups < 0) return fail_invalid("sizes must be >= 0");
  if (ftle && !(map_period > 0.0) && !(map_period < 0.0))
    return fail_invalid("map_period must be non-zero");
  if (num_groups == 0) return FTLE_OK;
  if (!positions) return fail_invalid("positions are required");
  FlowK f;
  f.kind = flow->kind;
  for (int i = 0; i < 8; ++i) f.p[i] = flow->params[i];
  cudaStream_t st = as_stream(stream);
#define AN(D, I, G)                                                                       \
  analytic_window_kernel<D, I, G><<<(unsigned)((num_groups + G - 1) / G), 2 * D * G, 0, st>>>( \
      f, t0, h, num_steps, freeze_time, positions, num_groups, map_period, ftle)
  if (dim == 2) {
    if (integrator == FTLE_EULER) AN(2, FTLE_EULER, 64);
    else if (integrator == FTLE_AB2) AN(2, FTLE_AB2, 64);
    else AN(2, FTLE_RK4, 64);
  } else {
    if (integrator == FTLE_EULER) AN(3, FTLE_EULER, 32);
    else if (integrator == FTLE_AB2) AN(3, FTLE_AB2, 32);
    else AN(3, FTLE_RK4, 32);
  }
#undef AN
  return check_launch("analytic_window_kernel");
}

}  // extern "C"

namespace ftle {

int pack_snapshots_f64(int32_t dim, int64_t nodes, int32_t num_snapshots, int32_t periodic_time,
                       const double *src, double *dst, void *stream) {
  const int64_t total = nodes * num_snapshots;
  const unsigned b = grid_blocks(total, 256);
  DIM_DISPATCH(dim, pack_f64_kernel, src, nodes, num_snapshots, periodic_time, dst);
  return check_launch("pack_f64_kernel");
}

}  // namespace ftle

