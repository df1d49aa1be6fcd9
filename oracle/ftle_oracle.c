/*
 * ftle_oracle.c -- CPU restatement of pyFTLE's FTLE hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA engine is
 * checked against.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference legs may load it; the product path never does.
 *
 * Pinned against the reference: tests/test_oracle.py checks every function
 * here against golden vectors produced by running the reference package
 * itself (tests/golden/make_golden.py) -- bit-exact for the interpolator and
 * for HOLD-mode windows, rtol 1e-12 for the FTLE.
 *
 * What it restates (reference file:line, paths inside the pyFTLE project):
 *   - bilinear gather        src/pyftle/grid_interp/GridInterp.cpp:93-142
 *   - trilinear gather       src/pyftle/grid_interp/GridInterp.cpp:15-91
 *   - physical -> index      src/pyftle/grid_interp/grid_interp.py:30-38,76-81,112-121,163-168
 *   - grid layout / axes     src/pyftle/interpolate.py:342-425 (meshgrid 'xy' flattening)
 *   - Euler / AB2 / RK4      src/pyftle/integrate.py:16-109,177-196,223-257,291-342
 *   - window driver          src/pyftle/ftle_solver.py:68-161
 *   - flow-map Jacobian      src/pyftle/cauchy_green.py:15-76,79-153
 *   - Cauchy-Green, lambda   src/pyftle/ftle.py:9-69,72-96,122-163,166-233
 *
 * Two time modes:
 *   HOLD  (reference semantics): step i holds snapshot first+i frozen for all
 *         RK4 stages; h is the snapshot spacing.
 *   BLEND (no reference counterpart): velocity at time t is the linear blend
 *         of the two snapshots bracketing t; stage times t, t+h/2, t+h.
 * Plus an optional periodic-space wrap (no reference counterpart; the
 * reference returns 0 outside the grid, GridInterp.cpp:126,58).
 *
 * Build with -ffp-contract=off so no FMA contraction changes the rounding
 * (the reference's own build is generic x86-64 -O3, which has no FMA).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

enum { OR_EULER = 0, OR_AB2 = 1, OR_RK4 = 2 };
enum { OR_HOLD = 0, OR_BLEND = 1 };

/* ------------------------------------------------------------------------- */
/* Reference index-space gathers (GridInterp.cpp)                            */
/* ------------------------------------------------------------------------- */

/* GridInterp.cpp:93-142 -- v is (nx, ny) row-major, index x*ny + y. */
void oracle_interp2d(const double *v, int nx, int ny, const double *pts, int64_t n,
                     double *out) {
  for (int64_t i = 0; i < n; ++i) {
    const double px = pts[i * 2 + 0];
    const double py = pts[i * 2 + 1];
    double c = 0.0;
    /* floor(px) in [0, nx-2]  <=>  0 <= px < nx-1 (also rejects NaN/inf,
       which the reference rejects through cvttsd2si's INT_MIN result). */
    if (px >= 0.0 && px < (double)(nx - 1) && py >= 0.0 && py < (double)(ny - 1)) {
      const int x0 = (int)floor(px), y0 = (int)floor(py);
      const double xd = px - x0, yd = py - y0;
      const double v00 = v[(int64_t)x0 * ny + y0];
      const double v10 = v[(int64_t)(x0 + 1) * ny + y0];
      const double v01 = v[(int64_t)x0 * ny + y0 + 1];
      const double v11 = v[(int64_t)(x0 + 1) * ny + y0 + 1];
      c = v00 * (1.0 - xd) * (1.0 - yd) + v10 * xd * (1.0 - yd) + v01 * (1.0 - xd) * yd +
          v11 * xd * yd;
    }
    out[i] = c;
  }
}

/* GridInterp.cpp:15-91 -- v is (X, Y, Z) row-major, index x*Y*Z + y*Z + z. */
void oracle_interp3d(const double *v, int X, int Y, int Z, const double *pts, int64_t n,
                     double *out) {
  const int64_t YZ = (int64_t)Y * Z;
  for (int64_t i = 0; i < n; ++i) {
    const double px = pts[i * 3 + 0], py = pts[i * 3 + 1], pz = pts[i * 3 + 2];
    double c = 0.0;
    if (px >= 0.0 && px < (double)(X - 1) && py >= 0.0 && py < (double)(Y - 1) && pz >= 0.0 &&
        pz < (double)(Z - 1)) {
      const int x0 = (int)floor(px), y0 = (int)floor(py), z0 = (int)floor(pz);
      const double xd = px - x0, yd = py - y0, zd = pz - z0;
#define V3(a, b, cc) v[(int64_t)(a) * YZ + (int64_t)(b) * Z + (cc)]
      const double c00 = V3(x0, y0, z0) * (1.0 - xd) + V3(x0 + 1, y0, z0) * xd;
      const double c01 = V3(x0, y0, z0 + 1) * (1.0 - xd) + V3(x0 + 1, y0, z0 + 1) * xd;
      const double c10 = V3(x0, y0 + 1, z0) * (1.0 - xd) + V3(x0 + 1, y0 + 1, z0) * xd;
      const double c11 = V3(x0, y0 + 1, z0 + 1) * (1.0 - xd) + V3(x0 + 1, y0 + 1, z0 + 1) * xd;
#undef V3
      const double c0 = c00 * (1.0 - yd) + c10 * yd;
      const double c1 = c01 * (1.0 - yd) + c11 * yd;
      c = c0 * (1.0 - zd) + c1 * zd;
    }
    out[i] = c;
  }
}

/* ------------------------------------------------------------------------- */
/* Velocity field on the flattened snapshot layout                           */
/* ------------------------------------------------------------------------- */

/* A snapshot is the reference's (dim, N) array (interpolate.py:342-425):
 *   2D node (i, j)    -> p = j*nx + i            (meshgrid 'xy', F-order reshape)
 *   3D node (i, j, k) -> p = (j*nx + i)*nz + k   (reshape + transpose(0,2,1,3);
 *                                                 identical to the reference when nx == ny)
 * Component c of node p lives at snap[c*N + p]. */
typedef struct {
  int dim;
  int n[3];
  double gmin[3];
  double gdelta[3];
  int periodic;
  int64_t nodes;
} or_grid;

typedef struct {
  int64_t p[8]; /* corner node ids, order matches the reference's operand order */
  double f[3];  /* fractional offsets xd, yd, zd */
  int inside;
} or_cell;

/* grid_interp.py:76-81 / :163-168 then GridInterp.cpp's floor and bounds test. */
static void locate(const or_grid *g, const double *x, or_cell *cell) {
  int i0[3], i1[3];
  cell->inside = 1;
  for (int a = 0; a < g->dim; ++a) {
    const double p = (x[a] - g->gmin[a]) / g->gdelta[a];
    if (g->periodic) {
      const double fl = floor(p);
      cell->f[a] = p - fl;
      /* cells beyond 1e9 (and NaN / inf) count as outside: velocity 0 */
      if (!(fabs(fl) < 1.0e9)) { cell->inside = 0; return; }
      int q = (int)fl % g->n[a];
      if (q < 0) q += g->n[a];
      i0[a] = q;
      i1[a] = (i0[a] + 1 == g->n[a]) ? 0 : i0[a] + 1;
    } else {
      if (!(p >= 0.0 && p < (double)(g->n[a] - 1))) { cell->inside = 0; return; }
      i0[a] = (int)floor(p);
      i1[a] = i0[a] + 1;
      cell->f[a] = p - i0[a];
    }
  }
  if (g->dim == 2) {
    const int64_t nx = g->n[0];
    cell->p[0] = (int64_t)i0[1] * nx + i0[0]; /* v00 */
    cell->p[1] = (int64_t)i0[1] * nx + i1[0]; /* v10 */
    cell->p[2] = (int64_t)i1[1] * nx + i0[0]; /* v01 */
    cell->p[3] = (int64_t)i1[1] * nx + i1[0]; /* v11 */
  } else {
    const int64_t nx = g->n[0], nz = g->n[2];
#define P3(a, b, c) (((int64_t)(b) * nx + (a)) * nz + (c))
    cell->p[0] = P3(i0[0], i0[1], i0[2]); /* x0y0z0 */
    cell->p[1] = P3(i1[0], i0[1], i0[2]); /* x1y0z0 */
    cell->p[2] = P3(i0[0], i0[1], i1[2]); /* x0y0z1 */
    cell->p[3] = P3(i1[0], i0[1], i1[2]); /* x1y0z1 */
    cell->p[4] = P3(i0[0], i1[1], i0[2]); /* x0y1z0 */
    cell->p[5] = P3(i1[0], i1[1], i0[2]); /* x1y1z0 */
    cell->p[6] = P3(i0[0], i1[1], i1[2]); /* x0y1z1 */
    cell->p[7] = P3(i1[0], i1[1], i1[2]); /* x1y1z1 */
#undef P3
  }
}

/* Blend the corner values of component c (weights 1-alpha / alpha) and apply
 * the reference's bi/trilinear expression.  snap1 == NULL means HOLD. */
static double corner_blend(const double *s0, const double *s1, double a, double oma, int64_t idx) {
  if (!s1) return s0[idx];
  return s0[idx] * oma + s1[idx] * a;
}

static void velocity(const or_grid *g, const double *s0, const double *s1, double alpha,
                     const double *x, double *u) {
  or_cell cell;
  locate(g, x, &cell);
  if (!cell.inside) {
    for (int c = 0; c < g->dim; ++c) u[c] = 0.0;
    return;
  }
  const double oma = 1.0 - alpha;
  for (int c = 0; c < g->dim; ++c) {
    const int64_t off = (int64_t)c * g->nodes;
    if (g->dim == 2) {
      const double xd = cell.f[0], yd = cell.f[1];
      const double v00 = corner_blend(s0, s1, alpha, oma, off + cell.p[0]);
      const double v10 = corner_blend(s0, s1, alpha, oma, off + cell.p[1]);
      const double v01 = corner_blend(s0, s1, alpha, oma, off + cell.p[2]);
      const double v11 = corner_blend(s0, s1, alpha, oma, off + cell.p[3]);
      u[c] = v00 * (1.0 - xd) * (1.0 - yd) + v10 * xd * (1.0 - yd) + v01 * (1.0 - xd) * yd +
             v11 * xd * yd;
    } else {
      const double xd = cell.f[0], yd = cell.f[1], zd = cell.f[2];
      double v[8];
      for (int q = 0; q < 8; ++q) v[q] = corner_blend(s0, s1, alpha, oma, off + cell.p[q]);
      const double c00 = v[0] * (1.0 - xd) + v[1] * xd;
      const double c01 = v[2] * (1.0 - xd) + v[3] * xd;
      const double c10 = v[4] * (1.0 - xd) + v[5] * xd;
      const double c11 = v[6] * (1.0 - xd) + v[7] * xd;
      const double c0 = c00 * (1.0 - yd) + c10 * yd;
      const double c1 = c01 * (1.0 - yd) + c11 * yd;
      u[c] = c0 * (1.0 - zd) + c1 * zd;
    }
  }
}

/* BLEND time lookup: snapshot pair and weight for time t. */
typedef struct {
  int num_snaps;
  double t0, dt;
  int periodic_time;
} or_time;

static void time_pair(const or_time *tm, double t, int *s0, int *s1, double *alpha) {
  double tau = (t - tm->t0) / tm->dt;
  const int S = tm->num_snaps;
  if (tm->periodic_time) {
    tau = tau - (double)S * floor(tau / (double)S);
    int s = (int)floor(tau);
    if (s >= S) s = S - 1;
    if (s < 0) s = 0;
    *s0 = s;
    *s1 = (s + 1 == S) ? 0 : s + 1;
    *alpha = tau - (double)s;
  } else {
    if (!(tau > 0.0)) { *s0 = 0; *s1 = 1; *alpha = 0.0; return; }
    if (tau >= (double)(S - 1)) { *s0 = S - 2; *s1 = S - 1; *alpha = 1.0; return; }
    const int s = (int)floor(tau);
    *s0 = s;
    *s1 = s + 1;
    *alpha = tau - (double)s;
  }
}

typedef struct {
  const or_grid *g;
  const double *snaps; /* num_snaps x dim x nodes */
  int time_mode;
  int hold_snapshot;
  or_time tm;
} or_field;

static void field_eval(const or_field *F, double t, const double *x, double *u) {
  const int64_t ssz = (int64_t)F->g->dim * F->g->nodes;
  if (F->time_mode == OR_HOLD) {
    velocity(F->g, F->snaps + (int64_t)F->hold_snapshot * ssz, NULL, 0.0, x, u);
  } else {
    int s0, s1;
    double a;
    time_pair(&F->tm, t, &s0, &s1, &a);
    velocity(F->g, F->snaps + (int64_t)s0 * ssz, F->snaps + (int64_t)s1 * ssz, a, x, u);
  }
}

/* ------------------------------------------------------------------------- */
/* FTLE epilogue (cauchy_green.py, ftle.py)                                  */
/* ------------------------------------------------------------------------- */

/* ftle.py:122-163 (closed-form 2x2 eigenvalue) and ftle.py:9-69 (C = F^T F). */
static double lambda_max_2x2(const double J[2][2]) {
  const double A = J[0][0] * J[0][0] + J[1][0] * J[1][0];
  const double B = J[0][0] * J[0][1] + J[1][0] * J[1][1];
  const double C = J[0][1] * J[0][0] + J[1][1] * J[1][0];
  const double D = J[0][1] * J[0][1] + J[1][1] * J[1][1];
  const double trace = A + D;
  const double det = A * D - B * C;
  const double l1 = 0.5 * (trace + sqrt(trace * trace - 4.0 * det));
  const double l2 = 0.5 * (trace - sqrt(trace * trace - 4.0 * det));
  return (l2 > l1) ? l2 : l1;
}

/* Largest eigenvalue of the symmetric 3x3 C by cyclic Jacobi rotations.
 * The reference (ftle.py:99-119) calls LAPACK dgeev on C = F F^T; for a
 * symmetric matrix both give lambda_max to a few ulp of ||C||. */
double oracle_sym3_lambda_max(const double Cin[3][3]) {
  double a[3][3];
  memcpy(a, Cin, sizeof(a));
  for (int sweep = 0; sweep < 32; ++sweep) {
    const double off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
    const double diag = fabs(a[0][0]) + fabs(a[1][1]) + fabs(a[2][2]);
    if (off == 0.0 || off <= 1e-300 || off < 1e-18 * diag) break;
    for (int p = 0; p < 2; ++p) {
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
        a[p][q] = a[q][p] = 0.0;
        const int r = 3 - p - q;
        const double arp = a[r][p], arq = a[r][q];
        a[r][p] = a[p][r] = c * arp - s * arq;
        a[r][q] = a[q][r] = s * arp + c * arq;
      }
    }
  }
  double m = a[0][0];
  if (a[1][1] > m) m = a[1][1];
  if (a[2][2] > m) m = a[2][2];
  return m;
}

/* cauchy_green.py:140-151 then ftle.py:72-96 (C = F F^T). */
static double lambda_max_3x3(const double J[3][3]) {
  double C[3][3];
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) C[i][k] = J[i][0] * J[k][0] + J[i][1] * J[k][1] + J[i][2] * J[k][2];
  return oracle_sym3_lambda_max((const double(*)[3])C);
}

/* ftle_solver.py:151-161 over role-blocked positions (particles.py:153-237):
 * rows [L(N); R(N); T(N); B(N) (; F(N); Bk(N))]. */
static double group_ftle(int dim, const double *pos, const double *pos0, int64_t N, int64_t g,
                         double map_period) {
#define ROW(arr, role) ((arr) + ((int64_t)(role) * N + g) * dim)
  if (dim == 2) {
    const double *L = ROW(pos, 0), *R = ROW(pos, 1), *T = ROW(pos, 2), *B = ROW(pos, 3);
    const double *L0 = ROW(pos0, 0), *R0 = ROW(pos0, 1), *T0 = ROW(pos0, 2), *B0 = ROW(pos0, 3);
    const double irl = R0[0] - L0[0], itb = T0[1] - B0[1];
    double J[2][2];
    J[0][0] = (R[0] - L[0]) / irl;
    J[0][1] = (T[0] - B[0]) / itb;
    J[1][0] = (R[1] - L[1]) / irl;
    J[1][1] = (T[1] - B[1]) / itb;
    return (1.0 / map_period) * log(sqrt(lambda_max_2x2((const double(*)[2])J)));
  } else {
    const double *P[6], *P0[6];
    for (int r = 0; r < 6; ++r) { P[r] = ROW(pos, r); P0[r] = ROW(pos0, r); }
    const double irl = P0[1][0] - P0[0][0], itb = P0[2][1] - P0[3][1], ifb = P0[4][2] - P0[5][2];
    double J[3][3];
    for (int i = 0; i < 3; ++i) {
      J[i][0] = (P[1][i] - P[0][i]) / irl;
      J[i][1] = (P[2][i] - P[3][i]) / itb;
      J[i][2] = (P[4][i] - P[5][i]) / ifb;
    }
    return (1.0 / map_period) * log(sqrt(lambda_max_3x3((const double(*)[3])J)));
  }
#undef ROW
}

/* compute_ftle_2x2 / compute_ftle_3x3 from a stack of Jacobians (ftle.py:166-233). */
void oracle_ftle_from_jacobians(int dim, const double *J, int64_t n, double map_period,
                                double *out) {
  for (int64_t i = 0; i < n; ++i) {
    if (dim == 2) {
      const double *j = J + i * 4;
      double M[2][2] = {{j[0], j[1]}, {j[2], j[3]}};
      out[i] = (1.0 / map_period) * log(sqrt(lambda_max_2x2((const double(*)[2])M)));
    } else {
      const double *j = J + i * 9;
      double M[3][3] = {{j[0], j[1], j[2]}, {j[3], j[4], j[5]}, {j[6], j[7], j[8]}};
      out[i] = (1.0 / map_period) * log(sqrt(lambda_max_3x3((const double(*)[3])M)));
    }
  }
}

/* ------------------------------------------------------------------------- */
/* Whole window (ftle_solver.py:68-120) in FP64                              */
/* ------------------------------------------------------------------------- */

static void advect_particle(const or_field *F0, int integrator, double t0, double h,
                            int num_steps, int first_snapshot, int dim, double *x) {
  or_field F = *F0;
  double k1[3], k2[3], k3[3], k4[3], tmp[3], vprev[3];
  int have_prev = 0;
  for (int i = 0; i < num_steps; ++i) {
    F.hold_snapshot = first_snapshot + i;
    const double t = t0 + (double)i * h;
    if (integrator == OR_EULER) {
      field_eval(&F, t, x, k1);
      for (int c = 0; c < dim; ++c) x[c] = x[c] + h * k1[c];
    } else if (integrator == OR_AB2) {
      field_eval(&F, t, x, k1);
      if (!have_prev) {
        for (int c = 0; c < dim; ++c) x[c] = x[c] + h * k1[c];
      } else {
        for (int c = 0; c < dim; ++c) x[c] = x[c] + h * (1.5 * k1[c] - 0.5 * vprev[c]);
      }
      for (int c = 0; c < dim; ++c) vprev[c] = k1[c];
      have_prev = 1;
    } else {
      const double hh = 0.5 * h;
      const double th = t + 0.5 * h, tf = t + h;
      field_eval(&F, t, x, k1);
      for (int c = 0; c < dim; ++c) tmp[c] = x[c] + hh * k1[c];
      field_eval(&F, th, tmp, k2);
      for (int c = 0; c < dim; ++c) tmp[c] = x[c] + hh * k2[c];
      field_eval(&F, th, tmp, k3);
      for (int c = 0; c < dim; ++c) tmp[c] = x[c] + h * k3[c];
      field_eval(&F, tf, tmp, k4);
      const double h6 = h / 6.0;
      for (int c = 0; c < dim; ++c)
        x[c] = x[c] + h6 * (((k1[c] + 2.0 * k2[c]) + 2.0 * k3[c]) + k4[c]);
    }
  }
}

/*
 * Advect every particle of a window and compute the FTLE per group.
 *   grid_n[3], gmin[3], gdelta[3]: grid nodes, origin and spacing
 *   snaps: num_snaps reference-layout snapshots (dim x nodes each)
 *   HOLD: step i uses snapshot first_snapshot + i
 *   BLEND: times t0 + i*h, snapshot s at snap_t0 + s*snap_dt
 *   positions: (K*N, dim) role-blocked, updated in place
 *   ftle_out: N values, or NULL to skip the epilogue
 * Returns 0, or -1 on invalid arguments.
 */
int oracle_window_f64(int dim, const int *grid_n, const double *gmin, const double *gdelta,
                      int periodic_space, const double *snaps, int num_snaps, int time_mode,
                      double snap_t0, double snap_dt, int periodic_time, int first_snapshot,
                      double t0, double h, int num_steps, int integrator, double *positions,
                      int64_t num_groups, double map_period, double *ftle_out, int nthreads) {
  if (dim != 2 && dim != 3) return -1;
  if (time_mode == OR_HOLD && first_snapshot + num_steps > num_snaps) return -1;
  if (time_mode == OR_BLEND && num_snaps < 2) return -1;
  or_grid g;
  memset(&g, 0, sizeof(g));
  g.dim = dim;
  g.nodes = 1;
  for (int a = 0; a < dim; ++a) {
    g.n[a] = grid_n[a];
    g.gmin[a] = gmin[a];
    g.gdelta[a] = gdelta[a];
    g.nodes *= grid_n[a];
  }
  g.periodic = periodic_space;
  or_field F;
  F.g = &g;
  F.snaps = snaps;
  F.time_mode = time_mode;
  F.hold_snapshot = first_snapshot;
  F.tm.num_snaps = num_snaps;
  F.tm.t0 = snap_t0;
  F.tm.dt = snap_dt;
  F.tm.periodic_time = periodic_time;

  const int K = 2 * dim;
  const int64_t M = (int64_t)K * num_groups;
  double *pos0 = NULL;
  if (ftle_out) {
    pos0 = (double *)malloc(sizeof(double) * M * dim);
    if (!pos0) return -1;
    memcpy(pos0, positions, sizeof(double) * M * dim);
  }
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
#endif
  for (int64_t p = 0; p < M; ++p)
    advect_particle(&F, integrator, t0, h, num_steps, first_snapshot, dim, positions + p * dim);

  if (ftle_out) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t gi = 0; gi < num_groups; ++gi)
      ftle_out[gi] = group_ftle(dim, positions, pos0, num_groups, gi, map_period);
    free(pos0);
  }
  (void)nthreads;
  return 0;
}

/* FTLE of role-blocked final positions against role-blocked initial positions. */
void oracle_ftle_from_positions(int dim, const double *positions, const double *initial,
                                int64_t num_groups, double map_period, double *out) {
  for (int64_t gi = 0; gi < num_groups; ++gi)
    out[gi] = group_ftle(dim, positions, initial, num_groups, gi, map_period);
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
