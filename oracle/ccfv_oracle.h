/*
 * ccfv_oracle.h -- CPU restatement of the T2S4 CC-CFV split step and its
 * Parareal driver.  TEST INFRASTRUCTURE ONLY: this library is the checker
 * that the CUDA path is compared against (tests, smoke check, the CPU
 * baseline leg of the benchmark).  Nothing in the product links it.
 *
 * Every function follows the reference T2S4_Parareal.cu operation for
 * operation in "compat" mode (reference domain handling, reference quirks),
 * and extends it with a periodic mode and other velocity fields using the
 * same scheme.  Field layout is the reference's: C[i*ny + j], i = x index.
 */
#ifndef CCFV_ORACLE_H
#define CCFV_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_BC_COMPAT = 0, OR_BC_PERIODIC = 1 };
enum { OR_VEL_REF_ROT4 = 0, OR_VEL_CONST = 1, OR_VEL_ROTATION = 2, OR_VEL_SWIRL = 3 };
enum { OR_FORM_STANDARD = 0, OR_FORM_DELTA = 1 };
/* REFERENCE: the third sweep takes the foot derivative of the remapped
 * field, as T2S4_Parareal.cu:929-932 does; CONSISTENT: every sweep takes it
 * of its input (the first two sweeps of the reference do this). */
enum { OR_SCHEME_REFERENCE = 0, OR_SCHEME_CONSISTENT = 1 };
/* Source term f(x,y,t): NONE is the reference's f = 0 (T2S4_Parareal.cu:58-61);
 * GAUSSIAN is sp0 exp(-((x-sp1)^2 + (y-sp2)^2) / sp3) cos(sp4 t). */
enum { OR_SRC_NONE = 0, OR_SRC_GAUSSIAN = 1 };

typedef struct or_grid {
  int nx, ny;
  double x_min, x_max, y_min, y_max;
  int bc;            /* OR_BC_*                                             */
  int vel;           /* OR_VEL_*                                            */
  double vp[4];      /* CONST: (u,v); ROTATION: (omega,xc,yc); SWIRL: (T)   */
  double K;          /* diffusivity                                         */
  int quirks;        /* compat: reproduce the y-remap neighbour-row read    */
  int threads;       /* OpenMP threads for the line loops (<=0: 1)          */
  int scheme;        /* OR_SCHEME_REFERENCE or OR_SCHEME_CONSISTENT         */
  int src;           /* OR_SRC_NONE or OR_SRC_GAUSSIAN                      */
  double sp[5];      /* GAUSSIAN: (amplitude, xc, yc, width, omega)         */
  double theta;      /* implicit weight of the diffusion sub-steps (<=0: 0.5,
                        the reference's Crank-Nicolson; 1: backward Euler)   */
} or_grid;

typedef struct or_parareal_opts {
  double t0, t1;
  int nt_fine;       /* fine steps over [t0,t1]                             */
  int n_slices;
  int coarse_steps;  /* coarse steps per slice (reference: 1)               */
  double tol;        /* stop when max relative slice update < tol (0: off)  */
  int kmax;
  int form;          /* OR_FORM_STANDARD (reference) or OR_FORM_DELTA       */
  double coarse_theta;  /* diffusion weight of every coarse step: 0 -> 0.5;
                           -1: the smallest theta >= 0.5 whose sub-steps
                           damp the grid-scale mode by 1/5 or more          */
} or_parareal_opts;

/* One full split step x(dt/2) y(dt) x(dt/2), in place (GpuOneStep). */
int or_step(const or_grid *g, double *C, double tn, double dt);
/* nsteps serial steps of dt starting at t0 (the reference's serial fine run). */
int or_run(const or_grid *g, double *C, double t0, double dt, int nsteps);
/* FinePropagator: J steps of DT/J from tn. */
int or_fine(const or_grid *g, double *C, double tn, double DT, int J);
/* Generalised CoarsePropagator: m steps of DT/m (m = 1 is the reference). */
int or_coarse(const or_grid *g, double *C, double tn, double DT, int m);
/* The automatic coarse diffusion weight for coarse steps of dtc: the
 * smallest theta >= 0.5 whose sub-steps damp the grid-scale mode by 1/5. */
double or_auto_theta(const or_grid *g, double dtc);

/* The reference's Parareal schedule (40 slices, fixed kmax, duplicated
 * k=0 coarse sweep, G(U_k) recomputed).  err[k] = max|U_k(T) - Uref| when
 * Uref != NULL.  UT receives the last iterate at T. */
int or_parareal_ref(const or_grid *g, const double *C0, double T_min,
                    double T_max, int Nt, int n_slices, int kmax,
                    const double *Uref, double *err, double *UT);

/* Generalised Parareal.  upd[k] = max over slices of the relative L2
 * update of iteration k+1; returns iterations done via *iters. */
int or_parareal(const or_grid *g, const or_parareal_opts *o,
                const double *C0, double *UT, int *iters, double *upd);

/* Reference initial condition / exact solution: 3x3 Simpson cell average of
 * the rotated diffused Gaussian (get_exact_solution_on_gpu, C_Exact). */
void or_exact_ref(const or_grid *g, double t, double *C);

/* Simpson 3x3 cell averages of a sum of Gaussians
 * amp * exp(-((x-cx)^2+(y-cy)^2)/den), periodic images summed over
 * [-img, img]^2 shifts when img > 0. */
void or_gaussians(const or_grid *g, int n, const double *cx, const double *cy,
                  const double *den, const double *amp, int img, double *C);

double or_sum_kahan(const double *v, long n);

#ifdef __cplusplus
}
#endif
#endif
