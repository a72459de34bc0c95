/*
 * ccfv.h -- C ABI of the B200 T2S4 CC-CFV split-step solver and its
 * Parareal engine.
 *
 * This is the drop-in boundary for the solver of T2S4_Parareal.cu.  The
 * reference exposes no library interface; its in-process entry points are
 * the C++ functions GpuOneStep / CoarsePropagator / FinePropagator operating
 * on a GPUContext, and main()'s Parareal section.  Each entry point below
 * names the reference function it replaces.
 *
 * Conventions
 *  - Every function returns an int status (CCFV_OK = 0); ccfv_strerror()
 *    gives its text.  No C++ exception crosses this boundary.
 *  - Fields are FP64, nx*ny values, laid out like the reference:
 *    C[i*ny + j], i = x index (slow), j = y index (fast).
 *  - Device pointers are caller-owned cudaMalloc memory on the context's
 *    device.  Functions taking a `mem` flag also accept host pointers.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *    stream).  Work is stream-ordered; functions that return results to the
 *    host synchronise the stream.
 *  - A context may be used by one host thread at a time.
 */
#ifndef CCFV_H
#define CCFV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
enum {
  CCFV_OK = 0,
  CCFV_ERR_INVALID = 1,     /* bad argument or configuration              */
  CCFV_ERR_CUDA = 2,        /* CUDA runtime error                          */
  CCFV_ERR_NOMEM = 3,       /* device allocation failed                    */
  CCFV_ERR_UNSUPPORTED = 4, /* combination not supported                   */
  CCFV_ERR_HALO = 5,        /* a characteristic foot left the staged halo  */
  CCFV_ERR_BUDGET = 6,      /* request exceeds the HBM budget              */
  CCFV_ERR_NOT_FOUND = 7,   /* unknown ticket                              */
  CCFV_ERR_CANCELLED = 8,   /* request cancelled                           */
  CCFV_ERR_TIMEOUT = 9      /* a bounded wait gave up                      */
};

/* ---- problem description --------------------------------------------- */
enum ccfv_bc {
  CCFV_BC_COMPAT = 0,   /* reference boundaries: extrapolated ghosts, zero
                           inflow, non-cyclic tridiagonal (T2S4:275-286,
                           322-324, 657-719)                                 */
  CCFV_BC_PERIODIC = 1  /* periodic cells, cyclic tridiagonal              */
};

enum ccfv_velocity {
  CCFV_VEL_REF_ROT4 = 0, /* Vx = -4y, Vy = 4x (T2S4_Parareal.cu:44-45)      */
  CCFV_VEL_CONST = 1,    /* (p0, p1)                                        */
  CCFV_VEL_ROTATION = 2, /* u = -p0 (y - p2), v = p0 (x - p1)               */
  CCFV_VEL_SWIRL = 3     /* u = sin^2(pi x) sin(2 pi y) cos(pi t / p0),
                            v = -sin^2(pi y) sin(2 pi x) cos(pi t / p0)     */
};

/* Which field the third sweep differentiates at the characteristic feet. */
enum ccfv_scheme {
  CCFV_SCHEME_REFERENCE = 0,  /* the remapped field, as the reference does
                                 (dcdx_bar_on_gpu(v_d_Cnphf_bar_x, ...),
                                 T2S4_Parareal.cu:929-932): bit-compatible
                                 with the reference, first order in time    */
  CCFV_SCHEME_CONSISTENT = 1  /* the sweep input, like the first two sweeps
                                 (T2S4:834-837, 882-885): 4th order in space,
                                 2nd order in time                          */
};

enum ccfv_precision { CCFV_FP64 = 0, CCFV_FP32 = 1 };
enum ccfv_mem { CCFV_MEM_DEVICE = 0, CCFV_MEM_HOST = 1 };
enum ccfv_form {
  CCFV_FORM_STANDARD = 0, /* U+ = G(U+) + F(U) - G(U)  (T2S4:1326-1329)    */
  CCFV_FORM_DELTA = 1     /* U+ = F(U) + G(U+ - U)  (linear scheme)         */
};

/* Grid and physics.  Replaces the compile-time macros and GPUContext fields
 * of the reference (T2S4_Parareal.cu:27-33, 724-768). */
/* Source term f(x, y, t) of c_t + div(V c) = K lap c + f.  The reference
 * keeps the whole source path in its step (get_source_term_on_gpu and the
 * remapped f in x_b_RHS_on_gpu / y_b_RHS_on_gpu, T2S4_Parareal.cu:142-165,
 * 564-613, 839-951) with f identically zero (T2S4_Parareal.cu:58-61).
 * GAUSSIAN: f = p0 exp(-((x-p1)^2 + (y-p2)^2) / p3) cos(p4 t), p3 > 0, as 3x3
 * Simpson cell averages; f(t_a) is remapped like C and f(t_b) added, with
 * weight 0.5 Dt per sub-step in the reference scheme (which therefore adds
 * 2 dt of source per step) and 0.25 Dt in the consistent scheme. */
enum ccfv_source { CCFV_SRC_NONE = 0, CCFV_SRC_GAUSSIAN = 1 };

typedef struct ccfv_grid {
  int nx, ny;                  /* cells; the reference forces ny = nx      */
  double x_min, x_max;         /* reference: -1, 1                         */
  double y_min, y_max;         /* reference: -1, 1                         */
  int bc;                      /* enum ccfv_bc                             */
  int velocity;                /* enum ccfv_velocity                       */
  double vel_params[4];        /* see enum ccfv_velocity                   */
  double K;                    /* diffusivity (reference config key "K")   */
  int scheme;                  /* enum ccfv_scheme (0 = reference)         */
  int source;                  /* enum ccfv_source (0 = the reference's f=0) */
  double source_params[5];     /* GAUSSIAN: amplitude, xc, yc, width, omega */
} ccfv_grid;

typedef struct ccfv_ctx ccfv_ctx;

/* ---- context --------------------------------------------------------- */
/* Creates a solver context on `device` (replaces the GPUContext set-up of
 * main(), T2S4_Parareal.cu:1057-1221).  The context owns its scratch. */
int ccfv_create(ccfv_ctx **out, const ccfv_grid *grid, int device);
int ccfv_destroy(ccfv_ctx *ctx);
const char *ccfv_strerror(int status);

/* Reads and clears the device-side status word of the context (a foot that
 * left the staged halo sets CCFV_ERR_HALO).  Synchronises `stream`. */
int ccfv_check(ccfv_ctx *ctx, void *stream);

/* ---- time stepping --------------------------------------------------- */
/* One T2S4 step x(dt/2) y(dt) x(dt/2), in place on d_C.
 * Replaces GpuOneStep(GPUContext&, tn, dt) (T2S4_Parareal.cu:785-968). */
int ccfv_step(ccfv_ctx *ctx, double *d_C, double tn, double dt, void *stream);

/* J steps of DT/J from tn, in place.
 * Replaces FinePropagator(GPUContext&, tn, DT, J) (T2S4_Parareal.cu:977-984). */
int ccfv_fine(ccfv_ctx *ctx, double *d_C, double tn, double DT, int J, void *stream);

/* m steps of DT/m from tn, in place, computed in FP64 or FP32.  With m = 1
 * and CCFV_FP64 replaces CoarsePropagator(GPUContext&, tn, DT)
 * (T2S4_Parareal.cu:971-974). */
int ccfv_coarse(ccfv_ctx *ctx, double *d_C, double tn, double DT, int m, int precision,
                void *stream);

/* ccfv_coarse with the coarse steps' implicit diffusion weight `theta`
 * (ccfv_parareal_opts::coarse_theta: 0 or 0.5 Crank-Nicolson, a value in
 * (0.5, 1], or CCFV_COARSE_THETA_AUTO, resolved for steps of DT/m): the
 * coarse propagator of the slice-distributed drivers.  No counterpart in the
 * reference. */
int ccfv_coarse_ex(ccfv_ctx *ctx, double *d_C, double tn, double DT, int m, int precision,
                   double theta, void *stream);

/* nsteps serial steps of dt from t0 on `C` (device or host memory).  The
 * reference's serial fine run (T2S4_Parareal.cu:1224-1247). */
int ccfv_run(ccfv_ctx *ctx, double *C, int mem, double t0, double dt, int nsteps, void *stream);

/* ---- Parareal -------------------------------------------------------- */
typedef struct ccfv_parareal_opts {
  double t0, t1;       /* horizon (reference: T_min, T_max)                 */
  int nt_fine;         /* fine steps over [t0,t1] (reference: Nt)           */
  int n_slices;        /* time slices (reference: 40)                       */
  int coarse_ratio;    /* coarse dt / fine dt; must divide nt_fine/n_slices;
                          0 = one coarse step per slice (reference)         */
  double tol;          /* stop when the max relative L2 slice update < tol;
                          0 = always run kmax iterations (reference)        */
  int kmax;            /* iteration cap (reference: 8)                      */
  int coarse_precision;/* CCFV_FP64 or CCFV_FP32                            */
  int form;            /* CCFV_FORM_STANDARD or CCFV_FORM_DELTA; FP32 coarse
                          requires DELTA                                    */
  int mem;             /* where C0 / C_T live: CCFV_MEM_DEVICE or _HOST      */
  const double *d_ref; /* optional device field (e.g. the serial fine solution
                          at t1): stats.err_* get ||U_k(t1) - ref|| after
                          every iteration, the reference's diagnostic
                          (T2S4_Parareal.cu:1333-1346); NULL = off          */
  double coarse_theta; /* implicit weight of the coarse propagator's
                          diffusion sub-steps: 0 or 0.5 = Crank-Nicolson as
                          in the fine steps (reference); a value in (0.5, 1]
                          (1 = backward Euler); or CCFV_COARSE_THETA_AUTO.
                          With K dtc/h^2 >> 1 Crank-Nicolson keeps the stiff
                          modes at amplification near -1 per coarse step,
                          and Parareal amplifies their rounding from slice
                          to slice (binomially in the iteration count), so
                          it stalls; a larger theta damps them.  The
                          converged result is the fine solution whatever
                          G is.                                             */
} ccfv_parareal_opts;

/* coarse_theta: the smallest theta >= 0.5 whose coarse sub-steps damp the
 * grid-scale mode by at least 1/5 (0.5 when Crank-Nicolson already does,
 * i.e. K dtc/h^2 below ~0.58; ~0.8 for stiff diffusion). */
#define CCFV_COARSE_THETA_AUTO (-1.0)

/* The coarse diffusion weight a Parareal run with these options uses on this
 * grid (CCFV_COARSE_THETA_AUTO resolved); no device work.  Introspection, no
 * counterpart in the reference. */
int ccfv_coarse_theta(const ccfv_grid *grid, const ccfv_parareal_opts *opts, double *theta);

#define CCFV_MAX_ITERS 128

typedef struct ccfv_stats {
  int iterations;                        /* Parareal iterations performed  */
  int converged;                         /* 1 if tol was reached           */
  double update[CCFV_MAX_ITERS];         /* max relative L2 slice update   */
  double fine_cell_updates;              /* executed fine cell-updates     */
  double coarse_cell_updates;            /* executed coarse cell-updates   */
  double ms;                             /* device time of the solve       */
  double fine_ms;                        /* device time of the F phases    */
  double coarse_ms;                      /* device time of the G phases    */
  long long fine_sweep_launches;         /* sweep launches in the F phases */
  long long fine_sweep_cells;            /* cells swept in the F phases    */
  double err_max[CCFV_MAX_ITERS];        /* max |U_k(t1) - d_ref| (d_ref)  */
  double err_l2[CCFV_MAX_ITERS];         /* relative L2 of the same        */
} ccfv_stats;

/* Parareal solve of C0 over [t0,t1]; the final state goes to C_T.
 * Replaces the Parareal section of main() (T2S4_Parareal.cu:1249-1355):
 * n_slices = 40, coarse_ratio = 0, tol = 0, kmax = 8, FP64, STANDARD
 * reproduces its schedule (without the duplicated k = 0 coarse sweep and
 * with G(U_k) cached instead of recomputed; both change no value). */
int ccfv_parareal(ccfv_ctx *ctx, const ccfv_parareal_opts *opts, const double *C0, double *C_T,
                  ccfv_stats *stats, void *stream);

/* ---- Parareal building blocks (slice-distributed drivers) -------------- */
/* FinePropagator (T2S4_Parareal.cu:977-984) on n contiguous fields at once:
 * field i starts at t0 + i*slice_dt and takes J steps of DT/J; all fields
 * advance in the same sweep launches.  Synchronises `stream`. */
int ccfv_fine_slices(ccfv_ctx *ctx, double *d_fields, int n, double t0, double slice_dt,
                     double DT, int J, void *stream);

/* Parareal correction of one slice (parareal_correction_kernel,
 * T2S4_Parareal.cu:771-782) fused with its update norms.
 *   STANDARD: U <- W + (F - Gold), Gold <- W          (W = G(U+ of the previous slice))
 *   DELTA:    U <- F + W,          W <- U_new - U_old  (W = G(increment))
 * *sq_update = sum (U_new - U_old)^2, *sq_state = sum U_new^2.
 * Synchronises `stream`. */
int ccfv_correct(ccfv_ctx *ctx, int form, double *d_U, const double *d_F, double *d_Gold,
                 double *d_W, double *sq_update, double *sq_state, void *stream);

/* ---- batched solves ---------------------------------------------------- */
/* One Parareal problem of a batch: its own grid, physics, options and
 * initial / final fields (device or host memory per opts.mem). */
typedef struct ccfv_problem {
  ccfv_grid grid;
  ccfv_parareal_opts opts;
  const double *C0;
  double *C_T;
} ccfv_problem;

/* Solves n independent Parareal problems of different sizes, velocities and
 * diffusivities together on `device`: the fine propagators of every active
 * slice of every problem advance in the same sweep launches, and the
 * sequential coarse sweeps of all problems advance slice by slice in shared
 * launches.  stats[i] (optional, n entries) receives problem i's iterations,
 * updates and executed cell-updates; stats[i].ms is the batch's device time.
 * No counterpart in the reference (one instance, one slice at a time). */
int ccfv_batch_solve(int n, const ccfv_problem *problems, ccfv_stats *stats, int device,
                     void *stream);

/* ---- serving ----------------------------------------------------------- */
/* A request loop with continuous batching: requests of different sizes are
 * admitted in arrival order while their resident slice states fit
 * hbm_budget_bytes (and max_active, if > 0; a request of N^2 cells and S
 * slices holds (3S + 4) N^2 doubles, plus (S + 1) N^2 in the standard form:
 * U, F and the out-of-place partner of F, and two coarse work fields);
 * every epoch all resident
 * requests advance by one Parareal iteration in shared launches, new
 * requests join at the next epoch boundary, finished ones return their result
 * to the caller's C_T and release their memory.  The caller keeps C0 / C_T
 * alive until the request completes.  No counterpart in the reference. */
typedef struct ccfv_server ccfv_server;

typedef struct ccfv_server_opts {
  int device;
  size_t hbm_budget_bytes;  /* device memory for resident request states     */
  int max_active;           /* max resident requests (0 = budget only)        */
} ccfv_server_opts;

enum ccfv_request_state {
  CCFV_REQ_QUEUED = 0,
  CCFV_REQ_RUNNING = 1,
  CCFV_REQ_DONE = 2,
  CCFV_REQ_FAILED = 3,
  CCFV_REQ_CANCELLED = 4
};

int ccfv_server_create(ccfv_server **out, const ccfv_server_opts *opts);
/* Queues a problem; CCFV_ERR_BUDGET if its states exceed the whole budget. */
int ccfv_server_submit(ccfv_server *s, const ccfv_problem *problem, uint64_t *ticket);
/* Non-blocking state query; stats / latency (submit to completion, ms) are
 * filled once the request has completed. */
int ccfv_server_poll(ccfv_server *s, uint64_t ticket, int *state, ccfv_stats *stats,
                     double *latency_ms);
/* Blocks until the request completes (timeout_s <= 0: no limit;
 * CCFV_ERR_TIMEOUT when the wait gives up). */
int ccfv_server_wait(ccfv_server *s, uint64_t ticket, double timeout_s, ccfv_stats *stats,
                     double *latency_ms);
/* Cancels a queued request, or a running one at the next epoch boundary. */
int ccfv_server_cancel(ccfv_server *s, uint64_t ticket);
/* Resident bytes, running and queued request counts. */
int ccfv_server_info(ccfv_server *s, size_t *used_bytes, int *active, int *queued);
/* Finishes running requests, cancels queued ones, stops the loop. */
int ccfv_server_destroy(ccfv_server *s);

/* ---- fields and diagnostics -------------------------------------------- */
/* 3x3 Simpson cell averages of the reference's exact solution (the rotated,
 * diffused Gaussian C_Exact, x0 = -0.35, sigma = 0.005, rotation rate 4) at
 * time t on the context's grid; t = 0 is the reference's initial condition.
 * Replaces get_exact_solution_on_gpu (T2S4_Parareal.cu:118-140). */
int ccfv_exact_ref(ccfv_ctx *ctx, double *d_C, double t, void *stream);

/* 3x3 Simpson cell averages of sum_q amp_q exp(-((x-cx_q)^2+(y-cy_q)^2)/den_q),
 * params = n x (cx, cy, den, amp), with the periodic images of the domain
 * box over [-images, images]^2 (0..4).  Synthetic initial fields. */
int ccfv_gaussians(ccfv_ctx *ctx, double *d_C, int n, const double *params, int images,
                   void *stream);

/* Relative L2 norm ||a-b||/||b|| and max |a-b| of two device fields on the
 * device (the reference computes the max norm on the host,
 * T2S4_Parareal.cu:1333-1346).  Synchronises `stream`. */
int ccfv_error_norms(ccfv_ctx *ctx, const double *d_a, const double *d_b, double *rel_l2,
                     double *max_abs, void *stream);

/* ---- allocation-free step ---------------------------------------------- */
/* One split step like ccfv_step, for callers that cannot allocate device
 * memory (inside another framework's memory pool, services that forbid
 * allocation after start-up, hosts that budget device memory up front).  No
 * counterpart in the reference.  Needs no context and calls no cudaMalloc,
 * cudaFree or allocating library routine: its scratch (solver factors, sweep
 * descriptors, status word) is a fixed file-scope device array of about
 * 340 KB that every GPU loading the library holds until exit.  Limit:
 * nx, ny <= 4096, else CCFV_ERR_UNSUPPORTED.  The first call on a device
 * looks up the array's address with that device current: make it before any
 * stream capture (and do not call it on a device after cudaDeviceReset of
 * that device: the cached address would be stale).  All calls share the
 * array: calls that overlap on the GPU race.  Synchronises `stream` before
 * returning.  Unlike ccfv_step, which leaves a foot that left the staged halo
 * in the context's status word for ccfv_check, this call returns
 * CCFV_ERR_HALO itself; d_C has been updated (with the out-of-halo reads
 * taken as zero) when it does. */
int ccfv_step_noalloc(const ccfv_grid *grid, double *d_C, double tn, double dt, void *stream);

/* ---- tuning ------------------------------------------------------------ */
/* Autotunes the line-tile shape of the sweeps for this context's grid: times
 * the candidate segment lengths (cells per CTA along a line: the tile height,
 * which also sets the recurrence chunk length) of one step of dt in the given
 * precision and keeps the fastest for every later plan with these line
 * lengths (process-wide).  *segment (optional) receives the choice. */
int ccfv_autotune(ccfv_ctx *ctx, double dt, int precision, int *segment, void *stream);

/* Which sweep kernel each sub-step of a step of dt runs in ccfv_step /
 * ccfv_run and the Parareal engines (introspection; no counterpart in the
 * reference): variant[s] for s = x(dt/2), y(dt), x(dt/2)
 * is CCFV_SWEEP_GENERAL (per-cell feet), CCFV_SWEEP_UNIFORM (shared-foot
 * stencil with exact chunked scans), CCFV_SWEEP_FILTER (shared-foot stencil
 * with the factored cyclic solve), CCFV_SWEEP_SOURCE (per-cell, with the
 * source term) or CCFV_SWEEP_FILTER_EXACT (the factored solve with the
 * periodic closure taken exactly across a line's segments: strong
 * diffusion), CCFV_SWEEP_CELL / CCFV_SWEEP_CELL_EXACT (the two factored forms
 * with a per-cell right-hand side: velocity fields whose feet differ from
 * edge to edge), CCFV_SWEEP_CELL_COMPAT (the factored solve of the
 * reference's non-cyclic system with its boundaries); segment[s] = cells per
 * CTA along a line (either may be NULL).  No device work. */
enum { CCFV_SWEEP_GENERAL = 0, CCFV_SWEEP_UNIFORM = 1, CCFV_SWEEP_FILTER = 2,
       CCFV_SWEEP_SOURCE = 3, CCFV_SWEEP_FILTER_EXACT = 4, CCFV_SWEEP_CELL = 5,
       CCFV_SWEEP_CELL_EXACT = 6, CCFV_SWEEP_CELL_COMPAT = 7 };
int ccfv_sweep_plan(ccfv_ctx *ctx, double dt, int precision, int variant[3], int segment[3]);

/* ---- library info ---------------------------------------------------- */
/* Number of kernels this library launched since load (all contexts). */
uint64_t ccfv_kernel_launches(void);

/* Text of the last error recorded on `ctx` ("" if none). */
const char *ccfv_last_error(ccfv_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* CCFV_H */
