/*
 * ccfv_oracle.c -- CPU restatement of the T2S4 CC-CFV split step and of
 * the Parareal driver of the reference (T2S4_Parareal.cu).
 *
 * TEST INFRASTRUCTURE (the checker).  Only the tests, the smoke check and
 * the CPU-baseline leg of the benchmark load this library.  It is never on
 * the product path.
 *
 * Parity: compat mode (OR_BC_COMPAT) reproduces the reference operation for
 * operation, including its boundary quirks, so that its results agree with
 * the reference binary to rounding (checked against golden vectors produced
 * by running the reference itself).  Periodic mode and the extra velocity
 * fields have no reference counterpart; they use the same formulas with
 * wrapped indices and a cyclic tridiagonal solve.
 *
 * Plain C99 with optional OpenMP over lines.  Build: see oracle/Makefile.
 */
#include "ccfv_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---------------------------------------------------------------------- */
/* velocity fields.  REF_ROT4 is Vx = -4y, Vy = 4x (T2S4_Parareal.cu:44-45). */

static double vel_u(const or_grid *g, double x, double y, double t) {
  switch (g->vel) {
  case OR_VEL_REF_ROT4: return -4 * y;
  case OR_VEL_CONST: return g->vp[0];
  case OR_VEL_ROTATION: return -g->vp[0] * (y - g->vp[2]);
  case OR_VEL_SWIRL: {
    double s = sin(M_PI * x);
    return s * s * sin(2.0 * M_PI * y) * cos(M_PI * t / g->vp[0]);
  }
  }
  return 0.0;
}

static double vel_v(const or_grid *g, double x, double y, double t) {
  switch (g->vel) {
  case OR_VEL_REF_ROT4: return 4 * x;
  case OR_VEL_CONST: return g->vp[1];
  case OR_VEL_ROTATION: return g->vp[0] * (x - g->vp[1]);
  case OR_VEL_SWIRL: {
    double s = sin(M_PI * y);
    return -s * s * sin(2.0 * M_PI * x) * cos(M_PI * t / g->vp[0]);
  }
  }
  return 0.0;
}

static int nthreads(const or_grid *g) { return g->threads > 0 ? g->threads : 1; }

/* ---------------------------------------------------------------------- */
/* Source term.  The reference's f is identically zero (T2S4_Parareal.cu:
 * 58-61) but its step keeps the full source path; GAUSSIAN exercises it. */

static double src_f(const or_grid *g, double x, double y, double t) {
  if (g->src != OR_SRC_GAUSSIAN) return 0.0;
  const double dx = x - g->sp[1], dy = y - g->sp[2];
  return g->sp[0] * exp(-(dx * dx + dy * dy) / g->sp[3]) * cos(g->sp[4] * t);
}

/* 3x3 Simpson cell averages of f at time t (get_source_term_on_gpu,
 * T2S4_Parareal.cu:142-165). */
static void source_cells(const or_grid *g, double t, double *out) {
  const int nx = g->nx, ny = g->ny;
  const double dx = (g->x_max - g->x_min) / nx, dy = (g->y_max - g->y_min) / ny;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++) {
      const double x_i = g->x_min + (i + 0.5) * dx, y_j = g->y_min + (j + 0.5) * dy;
      const double xm = x_i - 0.5 * dx, xp = x_i + 0.5 * dx;
      const double ym = y_j - 0.5 * dy, yp = y_j + 0.5 * dy;
      out[(size_t)i * ny + j] =
          1.0 / 36.0 *
          (src_f(g, xm, ym, t) + src_f(g, xp, ym, t) + src_f(g, xm, yp, t) + src_f(g, xp, yp, t) +
           4.0 * (src_f(g, xm, y_j, t) + src_f(g, xp, y_j, t) + src_f(g, x_i, ym, t) +
                  src_f(g, x_i, yp, t)) +
           16.0 * src_f(g, x_i, y_j, t));
    }
}

/* ---------------------------------------------------------------------- */
/* Characteristic feet.
 * Corner feet by one Heun step backwards over Dt (get_Lagrange_points_on_gpu,
 * T2S4_Parareal.cu:203-229): x* = x - Dt u(x,tb); xbar = x - Dt/2 (u(x,tb) +
 * u(x*,ta)).  For the reference's time-independent field Dt = dt/2 gives the
 * reference's 0.5*dt and 0.25*dt factors bit for bit.
 * Edge-midpoint feet are the mean of the two corner feet of the edge
 * (intersection_point_vert_x / _hori_y, T2S4_Parareal.cu:231-258). */

/* x feet of vertical edges: out[ip*ny + j], ip = 0..nx, j = 0..ny-1 */
static void feet_x(const or_grid *g, double Dt, double ta, double tb, double *out) {
  const int nx = g->nx, ny = g->ny;
  const double dx = (g->x_max - g->x_min) / nx, dy = (g->y_max - g->y_min) / ny;
  double *bar = (double *)malloc(sizeof(double) * (size_t)(nx + 1) * (ny + 1));
  for (int ip = 0; ip <= nx; ip++)
    for (int jp = 0; jp <= ny; jp++) {
      double xh = g->x_min + dx * ip, yh = g->y_min + dy * jp;
      double u0 = vel_u(g, xh, yh, tb);
      double xs = xh - Dt * u0;
      bar[(size_t)ip * (ny + 1) + jp] = xh - 0.5 * Dt * (u0 + vel_u(g, xs, yh, ta));
    }
  for (int ip = 0; ip <= nx; ip++)
    for (int j = 0; j < ny; j++) {
      size_t ind = (size_t)ip * (ny + 1) + j;
      out[(size_t)ip * ny + j] = 0.5 * (bar[ind] + bar[ind + 1]);
    }
  free(bar);
}

/* y feet of horizontal edges: out[i*(ny+1) + jp], i = 0..nx-1, jp = 0..ny */
static void feet_y(const or_grid *g, double Dt, double ta, double tb, double *out) {
  const int nx = g->nx, ny = g->ny;
  const double dx = (g->x_max - g->x_min) / nx, dy = (g->y_max - g->y_min) / ny;
  double *bar = (double *)malloc(sizeof(double) * (size_t)(nx + 1) * (ny + 1));
  for (int ip = 0; ip <= nx; ip++)
    for (int jp = 0; jp <= ny; jp++) {
      double xh = g->x_min + dx * ip, yh = g->y_min + dy * jp;
      double v0 = vel_v(g, xh, yh, tb);
      double ys = yh - Dt * v0;
      bar[(size_t)ip * (ny + 1) + jp] = yh - 0.5 * Dt * (v0 + vel_v(g, xh, ys, ta));
    }
  for (int i = 0; i < nx; i++)
    for (int jp = 0; jp <= ny; jp++) {
      size_t ind = (size_t)i * (ny + 1) + jp, nxt = (size_t)(i + 1) * (ny + 1) + jp;
      out[ind] = 0.5 * (bar[ind] + bar[nxt]);
    }
  free(bar);
}

/* ---------------------------------------------------------------------- */
/* One line of a sweep. */

typedef struct line_par {
  int L;
  double s_min, s_max, h;
  double K, Dt;
  int bc;
  double eps_remap; /* x: 1e-15 (T2S4:323-324), y: 1e-16 (T2S4:414-415) */
  int deriv_of_remap; /* derivative taken of the remapped field (3rd sweep) */
  double src_w;       /* RHS weight of (remapped f(t_a) + f(t_b))           */
  double theta;       /* implicit diffusion weight (0.5: Crank-Nicolson)    */
} line_par;

/* PPM antiderivative in cell units (d_intC_ppm4th, T2S4_Parareal.cu:63-65). */
static double ppm_int(double C6, double DltC, double CL, double xi) {
  return -1.0 / 3 * C6 * pow(xi, 3) + 0.5 * (DltC + C6) * pow(xi, 2) + CL * xi;
}

/* Compat ghost cells C_N, C_{N+1}, C_{-1}, C_{-2} (T2S4_Parareal.cu:275-286). */
static void ghosts_compat(const double *c, int L, double *CN, double *CNp1,
                          double *Cm1, double *Cm2) {
  const double one_eleventh = 1.0 / 11.0;
  *CN = one_eleventh * (-c[L - 3] + 3 * c[L - 2] + 9 * c[L - 1]);
  *CNp1 = one_eleventh * (-15 * c[L - 3] + 56 * c[L - 2] - 30 * c[L - 1]);
  *Cm1 = one_eleventh * (-c[2] + 3 * c[1] + 9 * c[0]);
  *Cm2 = one_eleventh * (-15 * c[2] + 56 * c[1] - 30 * c[0]);
}

static inline int wrap(int k, int L) { k %= L; return k < 0 ? k + L : k; }

/* PPM coefficients of every cell (x_step_ppm_coef_on_gpu, T2S4:260-304). */
static void ppm_coefs(const line_par *p, const double *c, double *CL, double *DltC, double *C6) {
  const int L = p->L;
  const double one_twelfth = 1.0 / 12.0, seven_twelfths = 7.0 / 12.0;
  double CN = 0, CNp1 = 0, Cm1 = 0, Cm2 = 0;
  if (p->bc == OR_BC_COMPAT) ghosts_compat(c, L, &CN, &CNp1, &Cm1, &Cm2);
  for (int i = 0; i < L; i++) {
    double Ci = c[i], Cip1, Cip2, Cim1, Cim2;
    if (p->bc == OR_BC_COMPAT) {
      Cip1 = (i == L - 1) ? CN : c[i + 1];
      Cip2 = (i >= L - 2) ? ((i == L - 2) ? CN : CNp1) : c[i + 2];
      Cim1 = (i == 0) ? Cm1 : c[i - 1];
      Cim2 = (i <= 1) ? ((i == 1) ? Cm1 : Cm2) : c[i - 2];
    } else {
      Cip1 = c[wrap(i + 1, L)];
      Cip2 = c[wrap(i + 2, L)];
      Cim1 = c[wrap(i - 1, L)];
      Cim2 = c[wrap(i - 2, L)];
    }
    double cl = seven_twelfths * (Ci + Cim1) - one_twelfth * (Cip1 + Cim2);
    double cr = seven_twelfths * (Cip1 + Ci) - one_twelfth * (Cip2 + Cim1);
    CL[i] = cl;
    DltC[i] = cr - cl;
    C6[i] = 6.0 * (Ci - 0.5 * (cl + cr));
  }
}

/* Coefficients of cell 0 of a line, compat mode (for the y-remap quirk). */
static void cell0_coefs_compat(const double *c, int L, double *CL, double *DltC, double *C6) {
  const double one_twelfth = 1.0 / 12.0, seven_twelfths = 7.0 / 12.0;
  double CN, CNp1, Cm1, Cm2;
  ghosts_compat(c, L, &CN, &CNp1, &Cm1, &Cm2);
  double Ci = c[0], Cip1 = c[1], Cip2 = c[2], Cim1 = Cm1, Cim2 = Cm2;
  double cl = seven_twelfths * (Ci + Cim1) - one_twelfth * (Cip1 + Cim2);
  double cr = seven_twelfths * (Cip1 + Ci) - one_twelfth * (Cip2 + Cim1);
  *CL = cl;
  *DltC = cr - cl;
  *C6 = 6.0 * (Ci - 0.5 * (cl + cr));
}

/* Neumaier-compensated sum of cells lo..hi (inclusive), wrapped. */
static double sum_cells(const double *c, int L, int lo, int hi, int periodic) {
  double s = 0.0, comp = 0.0;
  for (int k = lo; k <= hi; k++) {
    double v = periodic ? c[wrap(k, L)] : c[k];
    double t = s + v;
    if (fabs(s) >= fabs(v)) comp += (s - t) + v; else comp += (v - t) + s;
    s = t;
  }
  return s + comp;
}

/* Plain left-to-right sum (d_x_sum / d_y_sum, T2S4:76-90). */
static double sum_cells_plain(const double *c, int lo, int hi) {
  double s = 0.0;
  for (int k = lo; k <= hi; k++) s += c[k];
  return s;
}

/* Conservative remap of every cell (x_step_intC_ppm_on_gpu T2S4:306-347,
 * y_step_intC_ppm_on_gpu T2S4:396-438).  nextc0: coefficients of the next
 * line's first cell, read by the reference's y-remap when its right foot is
 * clamped onto the top edge (jR == Ny); NULL where there is none. */
static void remap(const line_par *p, const double *c, const double *foot, const double *CL,
                  const double *DltC, const double *C6, const double *nextc0, double *IntC) {
  const int L = p->L;
  const double smin = p->s_min, smax = p->s_max, h = p->h;
  for (int k = 0; k < L; k++) {
    double xbL = foot[k], xbR = foot[k + 1];
    double r = 0.0;
    if (p->bc == OR_BC_COMPAT) {
      if (!(xbL > smax || xbR < smin || xbL == xbR)) {
        double ixL = fmax(xbL, smin + p->eps_remap);
        double ixR = fmin(xbR, smax - p->eps_remap);
        int iL = (int)floor((ixL - smin) / h);
        int iR = (int)floor((ixR - smin) / h);
        double xL = (ixL - (smin + h * iL)) / h;
        double xR = (ixR - (smin + h * iR)) / h;
        /* coefficients of cell iR: the reference reads one past the line
         * when iR == L (y only); iL == L cannot occur except for a foot
         * exactly on the top edge, treated as a zero contribution. */
        double rC6 = 0, rD = 0, rCL = 0, lC6 = 0, lD = 0, lCL = 0;
        if (iR >= 0 && iR < L) { rC6 = C6[iR]; rD = DltC[iR]; rCL = CL[iR]; }
        else if (iR == L && nextc0) { rCL = nextc0[0]; rD = nextc0[1]; rC6 = nextc0[2]; }
        if (iL >= 0 && iL < L) { lC6 = C6[iL]; lD = DltC[iL]; lCL = CL[iL]; }
        if (iR == iL) {
          r = ppm_int(rC6, rD, rCL, xR) - ppm_int(lC6, lD, lCL, xL);
        } else {
          double IntCL = ppm_int(lC6, lD, lCL, 1.0) - ppm_int(lC6, lD, lCL, xL);
          double IntCR = ppm_int(rC6, rD, rCL, xR);
          int hi = iR - 1 < L - 1 ? iR - 1 : L - 1;
          double IntCM = sum_cells_plain(c, iL + 1, hi);
          r = IntCL + IntCM + IntCR;
        }
      }
    } else {
      double uL = (xbL - smin) / h, uR = (xbR - smin) / h;
      double fkL = floor(uL), fkR = floor(uR);
      int kL = (int)fkL, kR = (int)fkR;
      double xL = uL - fkL, xR = uR - fkR;
      int wL = wrap(kL, L), wR = wrap(kR, L);
      if (kR == kL) {
        r = ppm_int(C6[wR], DltC[wR], CL[wR], xR) - ppm_int(C6[wL], DltC[wL], CL[wL], xL);
      } else if (kR > kL) {
        r = sum_cells(c, L, kL, kR - 1, 1) + ppm_int(C6[wR], DltC[wR], CL[wR], xR) -
            ppm_int(C6[wL], DltC[wL], CL[wL], xL);
      } else {
        r = -(sum_cells(c, L, kR, kL - 1, 1) + ppm_int(C6[wL], DltC[wL], CL[wL], xL) -
              ppm_int(C6[wR], DltC[wR], CL[wR], xR));
      }
    }
    IntC[k] = r;
  }
}

/* Fourth-order derivative at every edge foot (dcdx_bar_on_gpu T2S4:440-494,
 * dcdy_bar_on_gpu T2S4:496-547), including the reference's ghost selection
 * at iL = L-2 and iL = 1 in compat mode. */
static void foot_derivative(const line_par *p, const double *c, const double *foot, double *D) {
  const int L = p->L;
  const double smin = p->s_min, smax = p->s_max, h = p->h;
  double CN = 0, CNp1 = 0, Cm1 = 0, Cm2 = 0;
  if (p->bc == OR_BC_COMPAT) ghosts_compat(c, L, &CN, &CNp1, &Cm1, &Cm2);
  for (int e = 0; e <= L; e++) {
    double xb = foot[e];
    double Ci, Cip1, Cip2, Cim1, Cim2, xi;
    if (p->bc == OR_BC_COMPAT) {
      if (!(xb >= smin && xb <= smax)) { D[e] = 0.0; continue; }
      double ixb = fmin(fmax(xb, smin + 1e-15), smax - 1e-15);
      int iL = (int)floor((ixb - smin) / h);
      xi = (ixb - (smin + h * iL)) / h;
      Ci = c[iL];
      Cip1 = (iL > L - 2) ? CN : c[iL + 1];
      Cip2 = (iL > L - 3) ? CNp1 : ((iL == L - 2) ? CN : c[iL + 2]);
      Cim1 = (iL < 1) ? Cm1 : c[iL - 1];
      Cim2 = (iL < 2) ? Cm2 : ((iL == 1) ? Cm1 : c[iL - 2]);
    } else {
      double u = (xb - smin) / h, fk = floor(u);
      int k = (int)fk;
      xi = u - fk;
      Ci = c[wrap(k, L)];
      Cip1 = c[wrap(k + 1, L)];
      Cip2 = c[wrap(k + 2, L)];
      Cim1 = c[wrap(k - 1, L)];
      Cim2 = c[wrap(k - 2, L)];
    }
    double xi2 = xi * xi, xi3 = xi2 * xi;
    D[e] = 1.0 / (12.0 * h) *
           ((2.0 * xi3 - 6.0 * xi2 + 3.0 * xi + 1.0) * Cim2 +
            (-8.0 * xi3 + 18.0 * xi2 + 6.0 * xi - 15.0) * Cim1 +
            (12.0 * xi3 - 18.0 * xi2 - 24.0 * xi + 15.0) * Ci +
            (-8.0 * xi3 + 6.0 * xi2 + 18.0 * xi - 1.0) * Cip1 + (2.0 * xi3 - 3.0 * xi) * Cip2);
  }
}

/* Thomas algorithm with a uniform off-diagonal and a per-row diagonal, in
 * the reference's operation order (x_Thomas_on_gpu, T2S4:657-686). */
static void thomas(int L, double coA, const double *coB, double coC, const double *r,
                   double *x, double *pw, double *qw) {
  pw[0] = coC / coB[0];
  qw[0] = r[0] / coB[0];
  for (int k = 1; k < L; k++) {
    double denom = 1.0 / (coB[k] - pw[k - 1] * coA);
    pw[k] = coC * denom;
    qw[k] = (r[k] - qw[k - 1] * coA) * denom;
  }
  x[L - 1] = qw[L - 1];
  for (int k = L - 2; k >= 0; k--) x[k] = qw[k] - pw[k] * x[k + 1];
}

/* Full line: remap + foot derivative + RHS + compact mass matrix + solve. */
static void sweep_line(const line_par *p, const double *c, const double *foot,
                       const double *nextc0, const double *s0, const double *s1,
                       const double *nexts0, double *out, double *wk) {
  const int L = p->L;
  double *CL = wk, *DltC = wk + L, *C6 = wk + 2 * L, *IntC = wk + 3 * L;
  double *D = wk + 4 * L;          /* L+1 */
  double *b = wk + 5 * L + 1, *Mb = wk + 6 * L + 1, *diag = wk + 7 * L + 1;
  double *pw = wk + 8 * L + 1, *qw = wk + 9 * L + 1, *z = wk + 10 * L + 1, *u = wk + 11 * L + 1;
  ppm_coefs(p, c, CL, DltC, C6);
  remap(p, c, foot, CL, DltC, C6, nextc0, IntC);
  /* The reference's third sweep evaluates the foot derivative on the
   * remapped field: dcdx_bar_on_gpu(v_d_Cnphf_bar_x, ...) (T2S4:929-932),
   * the first two on the sweep input (T2S4:834-837, 882-885). */
  foot_derivative(p, p->deriv_of_remap ? IntC : c, foot, D);
  /* RHS (x_b_RHS_on_gpu T2S4:564-580 / y_b_RHS_on_gpu T2S4:596-613):
   * b = remap(C) + w (remap(f(t_a)) + f(t_b)) + 0.5 K Dt/h (D_{k+1} - D_k);
   * f(t_a) is remapped by the same PPM integral as C (T2S4:846-853,
   * 893-900, 944-951).  The reference's w is 0.25 dt for the x half-steps
   * and 0.5 dt for the y step, i.e. 0.5 Dt of the sub-step.  A theta-weighted
   * diffusion (theta = 0.5 above) takes (1 - theta) K Dt/h here and theta in
   * the LHS. */
  const double rinv = p->Dt / p->h;
  double *F0b = u; /* remapped f(t_a); u is free until the cyclic solve */
  if (s0) {
    ppm_coefs(p, s0, CL, DltC, C6);
    remap(p, s0, foot, CL, DltC, C6, nexts0, F0b);
  }
  for (int k = 0; k < L; k++) {
    const double fs = s0 ? p->src_w * (F0b[k] + s1[k]) : 0.0;
    b[k] = IntC[k] + fs + (1.0 - p->theta) * p->K * rinv * (D[k + 1] - D[k]);
  }
  /* compact mass matrix (x_b_rhs_compact_on_gpu T2S4:616-634) */
  if (p->bc == OR_BC_COMPAT) {
    for (int k = 0; k < L; k++) {
      if (k == 0) Mb[k] = (10.0 * b[k] + b[k + 1]) / 12.0;
      else if (k == L - 1) Mb[k] = (10.0 * b[k] + b[k - 1]) / 12.0;
      else Mb[k] = (b[k + 1] + 10.0 * b[k] + b[k - 1]) / 12.0;
    }
  } else {
    for (int k = 0; k < L; k++)
      Mb[k] = (b[wrap(k + 1, L)] + 10.0 * b[k] + b[wrap(k - 1, L)]) / 12.0;
  }
  /* constant LHS (x_A_LHS_on_gpu T2S4:550-561 / y_A_LHS_on_gpu T2S4:583-594) */
  const double r2 = p->Dt / (p->h * p->h);
  const double coA = 1.0 / 12 - p->theta * p->K * r2;
  const double coB = 10.0 / 12 + 2.0 * p->theta * p->K * r2;
  const double coC = coA;
  if (p->bc == OR_BC_COMPAT) {
    for (int k = 0; k < L; k++) diag[k] = coB;
    thomas(L, coA, diag, coC, Mb, out, pw, qw);
  } else {
    /* cyclic: Sherman-Morrison with gamma = -b (corner entries = coA). */
    const double gam = -coB;
    for (int k = 0; k < L; k++) { diag[k] = coB; u[k] = 0.0; }
    diag[0] = coB - gam;
    diag[L - 1] = coB - coA * coC / gam;
    u[0] = gam;
    u[L - 1] = coC;
    thomas(L, coA, diag, coC, Mb, out, pw, qw);
    thomas(L, coA, diag, coC, u, z, pw, qw);
    double fac = (out[0] + coA * out[L - 1] / gam) / (1.0 + z[0] + coA * z[L - 1] / gam);
    for (int k = 0; k < L; k++) out[k] -= fac * z[k];
  }
}

/* Sweep along x (lines j, cells i, stride ny) or y (lines i, contiguous). */
/* S0, S1: cell averages of f at the sub-step's start (remapped) and end;
 * NULL when there is no source. */
static void sweep(const or_grid *g, int dir, const double *in, double *outp, const double *feet,
                  double Dt, int deriv_of_remap, const double *S0, const double *S1) {
  const int nx = g->nx, ny = g->ny;
  line_par p;
  p.K = g->K;
  p.Dt = Dt;
  p.theta = g->theta > 0 ? g->theta : 0.5;
  p.bc = g->bc;
  p.deriv_of_remap = deriv_of_remap;
  /* the reference's 0.5 Dt adds the source twice over a full split step
   * (x/2 + y + x/2); the consistent scheme weighs it 0.25 Dt */
  p.src_w = g->scheme == OR_SCHEME_REFERENCE ? 0.5 * Dt : 0.25 * Dt;
  if (dir == 0) {
    p.L = nx; p.s_min = g->x_min; p.s_max = g->x_max; p.h = (g->x_max - g->x_min) / nx;
    p.eps_remap = 1e-15;
  } else {
    p.L = ny; p.s_min = g->y_min; p.s_max = g->y_max; p.h = (g->y_max - g->y_min) / ny;
    p.eps_remap = 1e-16;
  }
  const int L = p.L, M = dir == 0 ? ny : nx;
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads(g))
#endif
  {
    double *wk = (double *)malloc(sizeof(double) * (size_t)(12 * L + 8));
    double *c = (double *)malloc(sizeof(double) * (size_t)L);
    double *o = (double *)malloc(sizeof(double) * (size_t)L);
    double *f = (double *)malloc(sizeof(double) * (size_t)(L + 1));
    double *l0 = (double *)malloc(sizeof(double) * (size_t)L);
    double *l1 = (double *)malloc(sizeof(double) * (size_t)L);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
    for (int line = 0; line < M; line++) {
      double nc[3], ns[3];
      const double *nextc0 = NULL, *nexts0 = NULL;
      if (dir == 0) {
        for (int i = 0; i < L; i++) c[i] = in[(size_t)i * ny + line];
        for (int e = 0; e <= L; e++) f[e] = feet[(size_t)e * ny + line];
        if (S0)
          for (int i = 0; i < L; i++) {
            l0[i] = S0[(size_t)i * ny + line];
            l1[i] = S1[(size_t)i * ny + line];
          }
      } else {
        memcpy(c, in + (size_t)line * ny, sizeof(double) * L);
        memcpy(f, feet + (size_t)line * (ny + 1), sizeof(double) * (L + 1));
        if (S0) {
          memcpy(l0, S0 + (size_t)line * ny, sizeof(double) * L);
          memcpy(l1, S1 + (size_t)line * ny, sizeof(double) * L);
        }
        if (g->bc == OR_BC_COMPAT && g->quirks && line + 1 < nx) {
          cell0_coefs_compat(in + (size_t)(line + 1) * ny, L, &nc[0], &nc[1], &nc[2]);
          nextc0 = nc;
          if (S0) {
            cell0_coefs_compat(S0 + (size_t)(line + 1) * ny, L, &ns[0], &ns[1], &ns[2]);
            nexts0 = ns;
          }
        }
      }
      sweep_line(&p, c, f, nextc0, S0 ? l0 : NULL, S0 ? l1 : NULL, nexts0, o, wk);
      if (dir == 0) {
        for (int i = 0; i < L; i++) outp[(size_t)i * ny + line] = o[i];
      } else {
        memcpy(outp + (size_t)line * ny, o, sizeof(double) * L);
      }
    }
    free(wk); free(c); free(o); free(f); free(l0); free(l1);
  }
}

/* ---------------------------------------------------------------------- */
/* GpuOneStep (T2S4_Parareal.cu:785-968): x(dt/2), y(dt), x(dt/2). */

int or_step(const or_grid *g, double *C, double tn, double dt) {
  const int nx = g->nx, ny = g->ny;
  if (nx < 3 || ny < 3) return 1;
  const size_t NN = (size_t)nx * ny;
  double *fx1 = (double *)malloc(sizeof(double) * (size_t)(nx + 1) * ny);
  double *fy2 = (double *)malloc(sizeof(double) * (size_t)nx * (ny + 1));
  double *fx3 = (double *)malloc(sizeof(double) * (size_t)(nx + 1) * ny);
  double *t1 = (double *)malloc(sizeof(double) * NN);
  double *t2 = (double *)malloc(sizeof(double) * NN);
  const double tnphf = tn + 0.5 * dt, tnp1 = tn + dt;
  feet_x(g, 0.5 * dt, tn, tnphf, fx1);
  feet_y(g, dt, tn, tnp1, fy2);
  feet_x(g, 0.5 * dt, tnphf, tnp1, fx3);
  double *fa = NULL, *fh = NULL, *fe = NULL;
  if (g->src != OR_SRC_NONE) {
    /* f(t_n) remapped + f(t_n+1/2) in the first sweep (T2S4:839-853),
     * f(t_n) remapped + f(t_n+1) in the second (T2S4:887-900), f(t_n+1)
     * remapped + f(t_n+1) in the third (T2S4:934-951) */
    fa = (double *)malloc(sizeof(double) * NN);
    fh = (double *)malloc(sizeof(double) * NN);
    fe = (double *)malloc(sizeof(double) * NN);
    source_cells(g, tn, fa);
    source_cells(g, tnphf, fh);
    source_cells(g, tnp1, fe);
  }
  sweep(g, 0, C, t1, fx1, 0.5 * dt, 0, fa, fh);
  sweep(g, 1, t1, t2, fy2, dt, 0, fa, fe);
  sweep(g, 0, t2, C, fx3, 0.5 * dt, g->scheme == OR_SCHEME_REFERENCE, fe, fe);
  free(fx1); free(fy2); free(fx3); free(t1); free(t2);
  free(fa); free(fh); free(fe);
  return 0;
}

int or_run(const or_grid *g, double *C, double t0, double dt, int nsteps) {
  for (int n = 0; n < nsteps; ++n) {
    int rc = or_step(g, C, t0 + n * dt, dt);
    if (rc) return rc;
  }
  return 0;
}

/* FinePropagator (T2S4_Parareal.cu:977-984). */
int or_fine(const or_grid *g, double *C, double tn, double DT, int J) {
  double dt = DT / (double)J;
  for (int j = 0; j < J; ++j) {
    int rc = or_step(g, C, tn + j * dt, dt);
    if (rc) return rc;
  }
  return 0;
}

/* CoarsePropagator (T2S4_Parareal.cu:971-974), generalised to m steps. */
int or_coarse(const or_grid *g, double *C, double tn, double DT, int m) {
  if (m <= 1) return or_step(g, C, tn, DT);
  return or_fine(g, C, tn, DT, m);
}

/* ---------------------------------------------------------------------- */
/* Parareal, reference schedule (T2S4_Parareal.cu:1249-1355). */

int or_parareal_ref(const or_grid *g, const double *C0, double T_min, double T_max, int Nt,
                    int n_slices, int kmax, const double *Uref, double *err, double *UT) {
  const size_t NN = (size_t)g->nx * g->ny;
  const int S = n_slices;
  const double DT = (T_max - T_min) / S;
  const int J = Nt / S;
  double *Uk = (double *)malloc(sizeof(double) * NN * (S + 1));
  double *Uk1 = (double *)malloc(sizeof(double) * NN * (S + 1));
  double *Gk = (double *)malloc(sizeof(double) * NN);
  double *Gk1 = (double *)malloc(sizeof(double) * NN);
  double *F = (double *)malloc(sizeof(double) * NN);
  memcpy(Uk, C0, sizeof(double) * NN);
  for (int pass = 0; pass < 2; ++pass) /* the reference runs this sweep twice */
    for (int n = 0; n < S; ++n) {
      double tn = T_min + n * DT;
      memcpy(Uk + (n + 1) * NN, Uk + n * NN, sizeof(double) * NN);
      or_step(g, Uk + (n + 1) * NN, tn, DT);
    }
  for (int k = 0; k < kmax; ++k) {
    memcpy(Uk1, Uk, sizeof(double) * NN);
    for (int n = 0; n < S; ++n) {
      double tn = T_min + n * DT;
      memcpy(Gk1, Uk1 + n * NN, sizeof(double) * NN);
      or_step(g, Gk1, tn, DT);
      memcpy(Gk, Uk + n * NN, sizeof(double) * NN);
      or_step(g, Gk, tn, DT);
      memcpy(F, Uk + n * NN, sizeof(double) * NN);
      or_fine(g, F, tn, DT, J);
      double *dst = Uk1 + (n + 1) * NN;
      for (size_t i = 0; i < NN; ++i) dst[i] = Gk1[i] + (F[i] - Gk[i]);
    }
    if (err && Uref) {
      double e = 0.0;
      for (size_t i = 0; i < NN; ++i) {
        double d = fabs(Uk1[S * NN + i] - Uref[i]);
        if (d > e) e = d;
      }
      err[k] = e;
    }
    memcpy(Uk, Uk1, sizeof(double) * NN * (S + 1));
  }
  if (UT) memcpy(UT, Uk + S * NN, sizeof(double) * NN);
  free(Uk); free(Uk1); free(Gk); free(Gk1); free(F);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Generalised Parareal: n_slices, m coarse steps per slice, tolerance.
 * STANDARD form: U+[n+1] = G(U+[n]) + F(U[n]) - G(U[n]) with G(U[n]) kept
 * from the previous iteration (the reference recomputes it; the values are
 * identical).  DELTA form: U+[n+1] = F(U[n]) + G(U+[n] - U[n]), equal in
 * exact arithmetic because every operator of the scheme is linear in C. */

/* Automatic coarse diffusion weight: the grid-scale mode of a theta-weighted
 * sub-step with nu = K Dt/h^2 is multiplied by
 * (2/3 - 32/9 (1-theta) nu) / (2/3 + 4 theta nu) (mass matrix 8/12, LHS
 * second difference 4, RHS difference of the fourth-order edge derivatives
 * 16/3); theta is the smallest value >= 1/2 that makes its magnitude at most
 * 1/5 at the largest nu of a coarse step (x sub-steps dtc/2, y dtc). */
double or_auto_theta(const or_grid *g, double dtc) {
  const double hx = (g->x_max - g->x_min) / g->nx, hy = (g->y_max - g->y_min) / g->ny;
  double nu = 0.5 * dtc / (hx * hx);
  if (dtc / (hy * hy) > nu) nu = dtc / (hy * hy);
  nu *= g->K;
  if (!(nu > 0)) return 0.5;
  const double rho = 0.2;
  double th = (32.0 / 9.0 * nu - 2.0 / 3.0 * (1.0 + rho)) / (nu * (32.0 / 9.0 + 4.0 * rho));
  return th < 0.5 ? 0.5 : (th > 1.0 ? 1.0 : th);
}

static double l2(const double *a, size_t n) {
  double s = 0.0;
  for (size_t i = 0; i < n; ++i) s += a[i] * a[i];
  return sqrt(s);
}

int or_parareal(const or_grid *g, const or_parareal_opts *o, const double *C0, double *UT,
                int *iters, double *upd) {
  const size_t NN = (size_t)g->nx * g->ny;
  const int S = o->n_slices;
  if (S < 1 || o->nt_fine % S) return 1;
  const int J = o->nt_fine / S;
  const int m = o->coarse_steps < 1 ? 1 : o->coarse_steps;
  const double DT = (o->t1 - o->t0) / S;
  /* every coarse step, the first sweep included, uses the coarse weight */
  or_grid gc = *g;
  gc.theta = o->coarse_theta > 0 ? o->coarse_theta
             : o->coarse_theta == -1.0 ? or_auto_theta(g, DT / m) : 0.5;
  double *U = (double *)malloc(sizeof(double) * NN * (S + 1));
  double *F = (double *)malloc(sizeof(double) * NN * (S + 1));
  double *Gold = (double *)malloc(sizeof(double) * NN * (S + 1));
  double *w = (double *)malloc(sizeof(double) * NN);
  double *e = (double *)malloc(sizeof(double) * NN);
  memcpy(U, C0, sizeof(double) * NN);
  for (int n = 0; n < S; ++n) {
    memcpy(U + (n + 1) * NN, U + n * NN, sizeof(double) * NN);
    or_coarse(&gc, U + (n + 1) * NN, o->t0 + n * DT, DT, m);
    memcpy(Gold + (n + 1) * NN, U + (n + 1) * NN, sizeof(double) * NN);
  }
  int k;
  for (k = 1; k <= o->kmax; ++k) {
    for (int n = 0; n < S; ++n) {
      memcpy(F + (n + 1) * NN, U + n * NN, sizeof(double) * NN);
      or_fine(g, F + (n + 1) * NN, o->t0 + n * DT, DT, J);
    }
    double worst = 0.0;
    memset(e, 0, sizeof(double) * NN);
    for (int n = 0; n < S; ++n) {
      double tn = o->t0 + n * DT;
      double *Un1 = U + (n + 1) * NN;
      if (o->form == OR_FORM_STANDARD) {
        /* U+[n] is already in U[n] (updated in place in slice order) */
        memcpy(w, U + n * NN, sizeof(double) * NN);
        or_coarse(&gc, w, tn, DT, m);
        double *Fn = F + (n + 1) * NN, *Go = Gold + (n + 1) * NN;
        for (size_t i = 0; i < NN; ++i) {
          double nv = w[i] + (Fn[i] - Go[i]);
          e[i] = nv - Un1[i];
          Un1[i] = nv;
        }
        memcpy(Go, w, sizeof(double) * NN);
      } else {
        /* e = U+[n] - U[n] goes through the linear part of G (without the
         * source term), so G(0) = 0 */
        or_grid gh = gc;
        gh.src = OR_SRC_NONE;
        memcpy(w, e, sizeof(double) * NN);
        or_coarse(&gh, w, tn, DT, m);
        double *Fn = F + (n + 1) * NN;
        for (size_t i = 0; i < NN; ++i) {
          double nv = Fn[i] + w[i];
          e[i] = nv - Un1[i];
          Un1[i] = nv;
        }
      }
      double nu = l2(Un1, NN), ne = l2(e, NN);
      double rel = nu > 0 ? ne / nu : ne;
      if (rel > worst) worst = rel;
    }
    if (upd) upd[k - 1] = worst;
    if (o->tol > 0 && worst < o->tol) break;
  }
  if (iters) *iters = k > o->kmax ? o->kmax : k;
  if (UT) memcpy(UT, U + S * NN, sizeof(double) * NN);
  free(U); free(F); free(Gold); free(w); free(e);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Initial condition / exact solution. */

/* C_Exact (T2S4_Parareal.cu:51-56) with x0 = -0.35, y0 = 0, sigma = 0.005. */
static double c_exact_ref(double x, double y, double t, double K) {
  const double gx0 = -0.35, gy0 = 0.0, sg = 0.005;
  double xs = x * cos(4 * t) + y * sin(4 * t);
  double ys = -x * sin(4 * t) + y * cos(4 * t);
  return sg / (sg + 4 * K * t) *
         exp(-(pow((xs - gx0), 2) + pow((ys - gy0), 2)) / (sg + 4 * K * t));
}

/* get_exact_solution_on_gpu (T2S4_Parareal.cu:118-140). */
void or_exact_ref(const or_grid *g, double t, double *C) {
  const int nx = g->nx, ny = g->ny;
  const double dx = (g->x_max - g->x_min) / nx, dy = (g->y_max - g->y_min) / ny;
  const double K = g->K;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++) {
      double x_i = g->x_min + (i + 0.5) * dx, y_j = g->y_min + (j + 0.5) * dy;
      double xm = x_i - 0.5 * dx, xp = x_i + 0.5 * dx, ym = y_j - 0.5 * dy, yp = y_j + 0.5 * dy;
      C[(size_t)i * ny + j] =
          1.0 / 36.0 *
          (c_exact_ref(xm, ym, t, K) + c_exact_ref(xp, ym, t, K) + c_exact_ref(xm, yp, t, K) +
           c_exact_ref(xp, yp, t, K) +
           4.0 * (c_exact_ref(xm, y_j, t, K) + c_exact_ref(xp, y_j, t, K) +
                  c_exact_ref(x_i, ym, t, K) + c_exact_ref(x_i, yp, t, K)) +
           16.0 * c_exact_ref(x_i, y_j, t, K));
    }
}

static double gauss_sum(int n, const double *cx, const double *cy, const double *den,
                        const double *amp, int img, double Lx, double Ly, double x, double y) {
  double s = 0.0;
  for (int q = 0; q < n; ++q)
    for (int a = -img; a <= img; ++a)
      for (int b = -img; b <= img; ++b) {
        double dxg = x - cx[q] + a * Lx, dyg = y - cy[q] + b * Ly;
        s += amp[q] * exp(-(dxg * dxg + dyg * dyg) / den[q]);
      }
  return s;
}

void or_gaussians(const or_grid *g, int n, const double *cx, const double *cy, const double *den,
                  const double *amp, int img, double *C) {
  const int nx = g->nx, ny = g->ny;
  const double Lx = g->x_max - g->x_min, Ly = g->y_max - g->y_min;
  const double dx = Lx / nx, dy = Ly / ny;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++) {
      double x_i = g->x_min + (i + 0.5) * dx, y_j = g->y_min + (j + 0.5) * dy;
      double xm = x_i - 0.5 * dx, xp = x_i + 0.5 * dx, ym = y_j - 0.5 * dy, yp = y_j + 0.5 * dy;
#define GS(X, Y) gauss_sum(n, cx, cy, den, amp, img, Lx, Ly, X, Y)
      C[(size_t)i * ny + j] =
          1.0 / 36.0 *
          (GS(xm, ym) + GS(xp, ym) + GS(xm, yp) + GS(xp, yp) +
           4.0 * (GS(xm, y_j) + GS(xp, y_j) + GS(x_i, ym) + GS(x_i, yp)) + 16.0 * GS(x_i, y_j));
#undef GS
    }
}

double or_sum_kahan(const double *v, long n) {
  double s = 0.0, comp = 0.0;
  for (long i = 0; i < n; ++i) {
    double t = s + v[i];
    if (fabs(s) >= fabs(v[i])) comp += (s - t) + v[i]; else comp += (v[i] - t) + s;
    s = t;
  }
  return s + comp;
}
