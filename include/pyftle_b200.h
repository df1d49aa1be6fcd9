/*
 * pyftle_b200.h -- C ABI of the B200 (sm_100a) FTLE engine.
 *
 * Plain C types only: device pointers, sizes, a CUDA stream passed as void*
 * (a cudaStream_t; NULL = legacy default stream).  Every entry point
 * returns an int status (FTLE_OK = 0) and never throws; on error,
 * ftle_last_error() returns a message for the calling thread.  The caller
 * owns every buffer; no pointer is retained after a call returns.  Kernels
 * are enqueued on `stream` and run asynchronously: synchronise the stream
 * (or call ftle_stream_synchronize) before reading results on the host.
 *
 * Layouts (shared with pyFTLE):
 *   positions  (K*N, dim) float64 row-major, role-blocked rows
 *              [left(N); right(N); top(N); bottom(N) (; front(N); back(N))],
 *              K = 2*dim neighbours per group (particles.py:153-237).
 *   snapshot   (dim, nodes) float64, node (i,j) at j*nx+i in 2D and
 *              (i,j,k) at (j*nx+i)*nz+k in 3D (meshgrid "xy" flattening,
 *              the layout interpolate.py:359-401 un-flattens).
 *   grid       origin = min coordinate per axis, spacing = (max-min)/(n-1)
 *              computed on the host exactly as grid_interp.py:32-35 does.
 */
#ifndef PYFTLE_B200_H
#define PYFTLE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  FTLE_OK = 0,
  FTLE_ERR_INVALID = 1,     /* bad argument: null pointer, shape, unsupported combination */
  FTLE_ERR_CUDA = 2,        /* a CUDA runtime call or launch failed */
  FTLE_ERR_DEVICE = 3,      /* a kernel reported an error through its error word */
  FTLE_ERR_UNSUPPORTED = 4  /* valid request this build does not implement */
};

enum { FTLE_EULER = 0, FTLE_AB2 = 1, FTLE_RK4 = 2 };    /* integrate.py:372-376 keys */
enum { FTLE_HOLD = 0, FTLE_BLEND = 1 };                 /* time modes */
enum { FTLE_KEEP_POSITIONS = 1 };                       /* ftle_window.flags */
/* Snapshot storage.  FTLE_FX15: 15-bit fixed point per component over the
 * series' value range (uniform absolute error range/65534; decoded by one
 * byte permute into an FP32 in [0.5, 1)).  FTLE_FX16: all 65,536 codes of the
 * same decoder, whose byte permute maps code q to 0.5 + q/65536 for q <= 32768
 * and 1 + (q - 32768)/32768 above (two slopes, continuous): the series' range
 * maps onto [0.5, 2 - 2^-15], absolute error range/196,600 over the lower third
 * of the range and range/98,300 above; same records, same kernels, same speed. */
enum { FTLE_F64 = 0, FTLE_F16 = 1, FTLE_BF16 = 2, FTLE_FX15 = 3, FTLE_FX16 = 4 };

/* Regular grid of the "grid" interpolator (interpolate.py:342-425,
 * grid_interp.py:30-38, 112-121). */
typedef struct ftle_grid {
  int32_t dim;         /* 2 or 3 */
  int32_t n[3];        /* nodes per axis; n[2] ignored in 2D */
  double origin[3];    /* grid_x[0], grid_y[0] (, grid_z[0]) */
  double spacing[3];   /* (x[-1]-x[0])/(n-1) per axis */
  int32_t periodic;    /* 0: velocity is 0 outside the grid (GridInterp.cpp:58,126);
                          1: periodic wrap, node n == node 0 (no reference counterpart) */
  int32_t reserved;
} ftle_grid;

/* One FTLE window: advect every particle, then Jacobian -> Cauchy-Green ->
 * lambda_max -> FTLE per group.  Replaces FTLESolver.run
 * (ftle_solver.py:68-120) with one launch. */
typedef struct ftle_window {
  ftle_grid grid;
  const void *snapshots;   /* packed by ftle_pack_snapshots, num_snapshots records */
  int32_t num_snapshots;
  int32_t storage;         /* FTLE_F64 for ftle_window_run_f64; FTLE_F16/BF16/FX15/FX16 for _mixed */
  int32_t time_mode;       /* FTLE_HOLD: step i holds snapshot first_snapshot+i (reference);
                              FTLE_BLEND: linear blend of the snapshots around each stage time */
  int32_t periodic_time;   /* BLEND/HOLD: snapshot index wraps modulo num_snapshots */
  double snapshot_t0;      /* BLEND: time of snapshot 0 */
  double snapshot_dt;      /* BLEND: spacing of the snapshots */
  int32_t first_snapshot;  /* HOLD: snapshot used by step 0 */
  int32_t integrator;      /* FTLE_EULER / FTLE_AB2 / FTLE_RK4 */
  double t0;               /* BLEND: time of step 0 */
  double h;                /* step; negative for backward time */
  int32_t num_steps;
  int32_t flags;           /* FTLE_KEEP_POSITIONS: read the seeds, do not write final
                              positions back (windows may then share one seed buffer) */
  double *positions;       /* (K*N, dim) in/out, role-blocked */
  int64_t num_groups;      /* N */
  double map_period;       /* T in FTLE = log(sqrt(lambda_max))/T; reference: (steps-1)*|dt| */
  double *ftle;            /* N outputs, or NULL to skip the epilogue */
} ftle_window;

/* ---- library ----------------------------------------------------------- */
int ftle_version(void);
const char *ftle_last_error(void);
int ftle_stream_synchronize(void *stream);

/* ---- index-space gathers ------------------------------------------------
 * Replace pyftle.ginterp.interp2d_vec_inplace / interp3d_vec_inplace
 * (GridInterp.cpp:93-142 and :15-91, bound at :144-150): v is (nx, ny) or
 * (X, Y, Z) C-contiguous, points (n, dim) in index space, out (n,).
 * Bit-exact with the reference, including 0 outside the grid. */
int ftle_interp2d_vec_inplace(const double *v, int32_t nx, int32_t ny, const double *points,
                              int64_t n, double *out, void *stream);
int ftle_interp3d_vec_inplace(const double *v, int32_t X, int32_t Y, int32_t Z,
                              const double *points, int64_t n, double *out, void *stream);

/* ---- grid interpolator --------------------------------------------------
 * Replaces HighPerfInterpolator.interpolate (interpolate.py:475-543) together
 * with Interp2D/3D.__call__ (grid_interp.py:40-85, 123-172): physical points
 * (m, dim) -> velocities (m, dim) from one (dim, nodes) snapshot. */
int ftle_grid_interpolate(const ftle_grid *grid, const double *snapshot, const double *points,
                          int64_t m, double *out, void *stream);

/* ---- one integrator step with the grid interpolator ---------------------
 * Replaces EulerIntegrator / AdamsBashforth2Integrator /
 * RungeKutta4Integrator.integrate (integrate.py:177-196, 223-257, 291-342)
 * when the interpolator is the "grid" one: positions (m, dim) advance by h in
 * place on the frozen snapshot.  AB2 only: `history` (m, dim) holds the
 * previous velocity when history_valid != 0 (else the step is Euler) and
 * receives this step's velocity. */
int ftle_grid_step(const ftle_grid *grid, const double *snapshot, int32_t integrator, double h,
                   double *positions, int64_t m, double *history, int32_t history_valid,
                   void *stream);

/* ---- integrator arithmetic for any interpolator --------------------------
 * Bit-exact with the numpy / numba updates of integrate.py:
 *   ftle_axpy:       out = x + a*k          (:327-339 stage points, :44 Euler)
 *   ftle_ab2_update: x = x + h*(1.5*v - 0.5*v_prev)        (:78)
 *   ftle_rk4_update: x = x + (h/6)*(k1 + 2k2 + 2k3 + k4)   (:109)
 * n counts doubles. */
int ftle_axpy(double *out, const double *x, double a, const double *k, int64_t n, void *stream);
int ftle_ab2_update(double *x, double h, const double *v, const double *v_prev, int64_t n,
                    void *stream);
int ftle_rk4_update(double *x, double h, const double *k1, const double *k2, const double *k3,
                    const double *k4, int64_t n, void *stream);

/* ---- FTLE building blocks (cauchy_green.py, ftle.py) ---------------------
 * initial_deltas: (dim, N, dim) = [right-left; top-bottom (; front-back)] at
 * t0 (particles.py:85-100); only the diagonal entries are used
 * (cauchy_green.py:70-74, 140-151).  J and C are (n, dim, dim). */
int ftle_flow_map_jacobian(int32_t dim, const double *positions, const double *initial_deltas,
                           int64_t num_groups, double *jacobian, void *stream);
int ftle_cauchy_green(int32_t dim, const double *jacobian, int64_t n, double *cauchy_green,
                      void *stream);
int ftle_max_eigenvalue(int32_t dim, const double *cauchy_green, int64_t n, double *out,
                        void *stream);
int ftle_from_jacobian(int32_t dim, const double *jacobian, int64_t n, double map_period,
                       double *out, void *stream);
/* Jacobian -> C -> lambda_max -> FTLE in one pass (ftle_solver.py:122-161). */
int ftle_from_positions(int32_t dim, const double *positions, const double *initial_deltas,
                        int64_t num_groups, double map_period, double *out, void *stream);

/* ---- fused windows -------------------------------------------------------
 * Snapshots are first packed on the device: `src` is num_snapshots
 * reference-layout snapshots back to back ((S, dim, nodes) float64);
 * `dst` needs ftle_packed_snapshot_bytes(dim, nodes, S, storage) bytes and
 * 16-byte alignment.  Record s holds snapshot s and its successor
 * (s+1, or 0 when periodic_time, or s itself for the last one).  The 16-bit
 * storages start with a 256-byte header (per-component decode scale and
 * offset) followed by the records. */
int64_t ftle_packed_snapshot_bytes(int32_t dim, int64_t nodes, int32_t num_snapshots,
                                   int32_t storage);
int ftle_pack_snapshots(int32_t dim, int64_t nodes, int32_t num_snapshots,
                        int32_t periodic_time, const double *src, int32_t storage, void *dst,
                        void *stream);

/* Plain FP64 window (storage FTLE_F64): reference arithmetic, one thread per
 * particle, FTLE epilogue in the same kernel.  HOLD mode is bit-exact with
 * pyFTLE's positions; FTLE within 1e-10 relative. */
int ftle_window_run_f64(const ftle_window *w, void *stream);

/* Mixed-precision window (storage FTLE_F16, FTLE_BF16, FTLE_FX15 or FTLE_FX16): FP32 advection of
 * each group as an FP64 centroid plus FP32 neighbour offsets (split
 * representation), FP64 Jacobian -> Cauchy-Green -> lambda_max.  Writes
 * FP64 positions = centroid + offset. */
int ftle_window_run_mixed(const ftle_window *w, void *stream);

/* Bytes of device workspace ftle_window_run_mixed_chunked needs for `w`
 * (two group-state buffers, sort keys and bins); -1 for an invalid descriptor. */
int64_t ftle_window_workspace_bytes(const ftle_window *w);

/* The mixed-precision window in launches of `chunk_steps` steps: between
 * launches each group's state (FP64 centroid, FP32 offsets) lives in the
 * caller's `workspace` (256-byte aligned, >= ftle_window_workspace_bytes),
 * and every `sort_every` chunks (0 = never) the groups are reordered by the
 * Morton code of their centroid's cell, so that each block advects
 * neighbouring groups and their gathers share cached snapshot records.
 * Per-group arithmetic is unchanged: results equal ftle_window_run_mixed. */
int ftle_window_run_mixed_chunked(const ftle_window *w, void *workspace,
                                  int64_t workspace_bytes, int32_t chunk_steps,
                                  int32_t sort_every, void *stream);

/* ---- closed-form velocity fields -----------------------------------------
 * The "analytical" interpolator on the device (interpolate.py:765-829 with a
 * closed-form velocity_fn): FP64 advection of every particle plus the FTLE
 * epilogue in one launch, with the stage times t0 + i*h (+ h/2, + h).
 * freeze_time != 0 evaluates the field at t = 0 throughout, which is what
 * pyFTLE's AnalyticalSolver computes (its interpolator's time never advances,
 * data_source.py:274-285, interpolate.py:788,812). */
enum { FTLE_FLOW_DOUBLE_GYRE = 0, FTLE_FLOW_ABC = 1 };
typedef struct ftle_flow {
  int32_t kind;       /* FTLE_FLOW_DOUBLE_GYRE (2D) or FTLE_FLOW_ABC (3D) */
  int32_t reserved;
  double params[8];   /* double gyre: A, eps, omega; ABC: A, B, C, a, w (A(t) = A + a sin wt) */
} ftle_flow;
int ftle_analytic_window_run(const ftle_flow *flow, int32_t integrator, double t0, double h,
                             int32_t num_steps, int32_t freeze_time, double *positions,
                             int64_t num_groups, double map_period, double *ftle, void *stream);

/* ---- many windows in one persistent launch -------------------------------
 * Windows that share one packed snapshot series, grid, storage, time mode and
 * integrator, but differ in seed set, start time t0, step h, length and
 * map_period, run as one launch: persistent CTAs take work items (128 groups of
 * one window) from a counter until all are done.  Replaces the reference's
 * one-process-per-window ParallelExecutor (parallel.py:171-271) for the hot
 * path.  Build the plan once on the host (ftle_windows_plan: window table plus
 * work list; order 1 = longest windows first, 2 = by the start of each window's
 * time range, 0 = as given), copy it to a
 * 256-byte aligned device buffer, then run it any number of times; the plan
 * holds the windows' device pointers.  The run only issues a memset of the
 * plan's counter and one kernel on `stream` (ctas_per_sm x 148 persistent CTAs,
 * ctas_per_sm in 1..8; 4 blocks per SM are resident in 3D, 8 in 2D). */
int64_t ftle_windows_plan_bytes(const ftle_window *windows, int32_t count);
int ftle_windows_plan(const ftle_window *windows, int32_t count, int32_t order,
                      void *host_plan, int64_t plan_bytes);
int ftle_windows_run_mixed(const ftle_window *windows, int32_t count, void *device_plan,
                           int64_t plan_bytes, int32_t ctas_per_sm, void *stream);

/* ftle_window_run_mixed_chunked for callers that cannot provide or allocate
 * device memory (a host program owning all device memory through its own
 * pool, a plugin barred from calling cudaMalloc): the workspace is a 32 MiB
 * array built into the library, reserved on every GPU that loads it until
 * the process exits.  No counterpart in the reference.  Windows needing more
 * than 32 MiB (ftle_window_workspace_bytes) are rejected with
 * FTLE_ERR_INVALID.  The first call on a device (and again after the device's
 * context was reset) looks up the array's device address; under CUDA's
 * default lazy module loading that first call is also where the 32 MiB is
 * reserved, and where it fails with FTLE_ERR_CUDA if the device has no room
 * left.  Make that first call before any stream capture.  All calls share the
 * one array, which keeps the last call's contents: calls that overlap on the
 * GPU (other streams, other threads) race and must be serialised by the
 * caller. */
int ftle_window_run_mixed_chunked_static(const ftle_window *w, int32_t chunk_steps,
                                         int32_t sort_every, void *stream);

/* ---- flow-map surrogate MLP ------------------------------------------------
 * Kernels of the learned flow-map surrogate (Fourier features of (x0, y0, t0)
 * -> SiLU MLP -> displacement over a fixed T), which replaces advection for
 * sliding windows, with RK4 (ftle_window_run_*) as its judge and fallback.
 * No counterpart in the reference (it has no learned path); the nearest
 * interface is the advection it replaces, ftle_solver.py:116-149.
 * All matrices are row-major BF16 (2 bytes per element) unless named FP32;
 * a "transposed" operand stores element (r, k) at src[k*ld + r].
 * M, N multiples of 8, K a multiple of 64, operands 16-byte aligned,
 * leading dimensions multiples of 8.  `error_word` (device int32) is set to 1
 * when a tensor-core wait times out; the call's status reports launch errors. */

/* C[M x N] (+)= A[M x K] * B[N x K]^T, FP32 C; splits > 1 splits K (C accumulated). */
int ftle_mlp_gemm(const void *A, int32_t lda, int32_t a_trans, const void *B, int32_t ldb,
                  int32_t b_trans, float *C, int32_t ldc, int32_t M, int32_t N, int32_t K,
                  int32_t splits, int32_t accumulate, int32_t *error_word, void *stream);
/* Z = X W^T + b; activation != 0: Z (FP32, may be NULL) and H = silu(Z) (BF16);
 * activation == 0: Z = X W^T + b only (FP32). */
int ftle_mlp_linear(const void *X, int32_t ldx, const void *W, int32_t ldw, const float *bias,
                    int32_t M, int32_t N, int32_t K, int32_t activation, float *Z, int32_t ldz,
                    void *H, int32_t ldh, int32_t *error_word, void *stream);
/* G = (A B^T) * silu'(Zin) (BF16); colsum (FP32, may be NULL) += column sums of G. */
int ftle_mlp_gemm_dsilu(const void *A, int32_t lda, int32_t a_trans, const void *B, int32_t ldb,
                        int32_t b_trans, int32_t M, int32_t N, int32_t K, const float *Zin,
                        int32_t ldz, void *G, int32_t ldg, float *colsum, int32_t *error_word,
                        void *stream);
/* Features of points (n x 3 FP64: x, y, t) for freq (num_freq x 4 FP32: kx, ky,
 * kt, phase): [sin | cos] (n x 2*num_freq BF16), and their d/dx, d/dy (may be NULL). */
int ftle_mlp_features(const double *points, int64_t n, const float *freq, int32_t num_freq,
                      void *features, void *tangent_x, void *tangent_y, void *stream);
/* MSE loss over `outs` (<= 4) columns: dy = 2 (y - target) / n (BF16, lddy columns,
 * padding zero), dbias += column sums of dy, *loss += mean squared error. */
int ftle_mlp_mse_grad(const float *y, int32_t ldy, const float *target, int32_t outs, int64_t n,
                      void *dy, int32_t lddy, float *dbias, float *loss, void *stream);
/* Adam step `step` (1-based) with decoupled weight decay on FP32 w; writes the
 * BF16 copy w_bf16 and zeroes g. */
int ftle_mlp_adam(float *w, float *g, float *m, float *v, void *w_bf16, int64_t n, float lr,
                  float beta1, float beta2, float eps, int32_t step, float weight_decay,
                  void *stream);
/* FTLE (FP64) of x -> x + scale * y(x) from the tangents jx = dy/dx0, jy = dy/dy0
 * (FP32 rows, columns 0 and 1), as ftle_from_jacobian for 2D. */
int ftle_mlp_jacobian_ftle(const float *jx, const float *jy, int32_t ld, int64_t n, double scale,
                           double T, double *ftle, void *stream);
/* out (n x 2 FP64) = points[:, :2] + scale * y[:, :2]. */
int ftle_mlp_apply_displacement(const double *points, const float *y, int32_t ldy, int64_t n,
                                double scale, double *out, void *stream);
/* 3D forms: points n x 4 FP64 (x, y, z, t); freq num_freq rows of 8 FP32
 * (kx, ky, kz, kt, phase, 0, 0, 0); tangents d/dx, d/dy, d/dz (each may be NULL);
 * the FTLE from the three tangents (columns 0..2) with lambda_max of the 3x3
 * Cauchy-Green tensor by Jacobi rotations; end positions n x 3. */
int ftle_mlp_features3(const double *points, int64_t n, const float *freq, int32_t num_freq,
                       void *features, void *tangent_x, void *tangent_y, void *tangent_z,
                       void *stream);
int ftle_mlp_jacobian_ftle3(const float *jx, const float *jy, const float *jz, int32_t ld,
                            int64_t n, double scale, double T, double *ftle, void *stream);
int ftle_mlp_apply_displacement3(const double *points, const float *y, int32_t ldy, int64_t n,
                                 double scale, double *out, void *stream);

/* Fused surrogate inference for the fixed shape 32 frequencies (64 features) ->
 * 4 x 256 SiLU -> 2 outputs: one persistent launch evaluates the network and its
 * two Jacobian tangents per seed and writes the FTLE (as ftle_mlp_jacobian_ftle)
 * and/or the predicted end positions.  Weights are first packed into the
 * kernel's chunk images (ftle_surrogate_packed_bytes() bytes, 16-byte aligned)
 * from the BF16 matrices w0 (256 x 64), w1..w3 (256 x 256) and w4 (>= 16 rows x
 * 256; rows 2..15 zero).  bias: 4*256 + 16 FP32 (hidden layers, then the output
 * layer padded to 16).  points: n x 2 FP64 seed positions, all at start time t0.
 * No counterpart in the reference (it stands for ftle_solver.py:116-161). */
int64_t ftle_surrogate_packed_bytes(void);
int ftle_surrogate_pack(const void *w0, const void *w1, const void *w2, const void *w3,
                        const void *w4, void *packed, void *stream);
int ftle_surrogate_ftle(const double *points, int64_t n, double t0, const void *packed,
                        const float *bias, const float *freq, double out_scale, double T,
                        double *ftle, double *end_positions, int32_t *error_word, void *stream);

/* ---- measurement -----------------------------------------------------------
 * Gather-rate probe for the roofline of the window kernels (no counterpart in
 * the reference).  `blocks` blocks of 128 threads each issue iters x 8
 * independent 16-byte read-only loads (ftle_gather_probe_loads() in total) at
 * pseudo-random records of a region of `region_bytes` (a power of two, at most
 * 512 MiB and buf_bytes): one region per block when per_block_region != 0
 * (a few KB: L1-resident), else one region shared by all blocks (~32 MB:
 * L2-resident).  The lanes of a warp load within a random window of
 * lane_span_bytes (power of two: 16 .. region_bytes).  buf: 16-byte aligned,
 * zero-filled; sink: one device uint32 (written only if the loads XOR to a
 * magic word, never for zeros).  Time it with events on `stream`. */
int ftle_gather_probe(const void *buf, int64_t buf_bytes, int64_t region_bytes,
                      int64_t lane_span_bytes, int32_t per_block_region, int32_t blocks,
                      int32_t iters, uint32_t seed, void *sink, void *stream);
int64_t ftle_gather_probe_loads(int32_t blocks, int32_t iters);

#ifdef __cplusplus
}
#endif
#endif /* PYFTLE_B200_H */
