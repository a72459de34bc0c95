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
typedef struct ccfv_grid {
  int nx, ny;                  /* cells; the reference forces ny = nx      */
  double x_min, x_max;         /* reference: -1, 1                         */
  double y_min, y_max;         /* reference: -1, 1                         */
  int bc;                      /* enum ccfv_bc                             */
  int velocity;                /* enum ccfv_velocity                       */
  double vel_params[4];        /* see enum ccfv_velocity                   */
  double K;                    /* diffusivity (reference config key "K")   */
  int scheme;                  /* enum ccfv_scheme (0 = reference)         */
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
} ccfv_parareal_opts;

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
} ccfv_stats;

/* Parareal solve of C0 over [t0,t1]; the final state goes to C_T.
 * Replaces the Parareal section of main() (T2S4_Parareal.cu:1249-1355):
 * n_slices = 40, coarse_ratio = 0, tol = 0, kmax = 8, FP64, STANDARD
 * reproduces its schedule (without the duplicated k = 0 coarse sweep and
 * with G(U_k) cached instead of recomputed; both change no value). */
int ccfv_parareal(ccfv_ctx *ctx, const ccfv_parareal_opts *opts, const double *C0, double *C_T,
                  ccfv_stats *stats, void *stream);

/* ---- allocation-free step ---------------------------------------------- */
/* One split step like ccfv_step, for callers that cannot allocate device
 * memory (inside another framework's memory pool, services that forbid
 * allocation after start-up, hosts that budget device memory up front).  No
 * counterpart in the reference.  Needs no context and calls no cudaMalloc,
 * cudaFree or allocating library routine: its scratch (solver factors, sweep
 * descriptors, status word) is a fixed file-scope device array of about
 * 200 KB that every GPU loading the library holds until exit.  Limit:
 * nx, ny <= 4096, else CCFV_ERR_UNSUPPORTED.  The first call on a device
 * looks up the array's address with that device current: make it before any
 * stream capture.  All calls share the array: calls that overlap on the GPU
 * race.  Synchronises `stream` before returning. */
int ccfv_step_noalloc(const ccfv_grid *grid, double *d_C, double tn, double dt, void *stream);

/* ---- library info ---------------------------------------------------- */
/* Number of kernels this library launched since load (all contexts). */
uint64_t ccfv_kernel_launches(void);

/* Text of the last error recorded on `ctx` ("" if none). */
const char *ccfv_last_error(ccfv_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* CCFV_H */
