// sweep_math.cuh -- characteristic feet and the shared-foot stencil of one
// line, used by the sweep kernels (sweep.cu) and the resident coarse
// propagator (coarse.cu).
#pragma once

#include "ccfv_internal.h"

namespace ccfv {

// ---------------------------------------------------------------------------
// velocity component along the sweep: x-sweep u(x=s, y=tau), y-sweep v(x=tau, y=s)
__device__ __forceinline__ double vel_along(const SweepField &f, double s, double tau, double t) {
  switch (f.vel) {
    case VEL_REF_ROT4:  // Vx = -4y, Vy = 4x (T2S4_Parareal.cu:44-45)
      return f.dir == 0 ? -4 * tau : 4 * tau;
    case VEL_CONST:
      return f.dir == 0 ? f.vp[0] : f.vp[1];
    case VEL_ROTATION:
      return f.dir == 0 ? -f.vp[0] * (tau - f.vp[2]) : f.vp[0] * (tau - f.vp[1]);
    case VEL_SWIRL: {
      double ss = sinpi(s);
      double w = ss * ss * sinpi(2.0 * tau) * cospi(t / f.vp[0]);
      return f.dir == 0 ? w : -w;
    }
  }
  return 0.0;
}

// Heun foot of a cell corner (get_Lagrange_points_on_gpu, T2S4:203-229):
// s* = s - Dt w(s, tb); foot = s - Dt/2 (w(s, tb) + w(s*, ta)).
__device__ __forceinline__ double corner_foot(const SweepField &f, double s, double tau, double ta,
                                              double tb) {
  double w0 = vel_along(f, s, tau, tb);
  double xs = s - f.Dt * w0;
  return s - 0.5 * f.Dt * (w0 + vel_along(f, xs, tau, ta));
}

// Foot of edge e of a line = mean of its two corner feet
// (intersection_point_vert_x / _hori_y, T2S4:231-258).
__device__ __forceinline__ double edge_foot(const SweepField &f, int e, double tau0, double tau1,
                                            double ta, double tb) {
  double s = f.s_min + f.h * e;
  return 0.5 * (corner_foot(f, s, tau0, ta, tb) + corner_foot(f, s, tau1, ta, tb));
}

// Edge feet of one line.  The swirling field factors as
// sin^2(pi s) g(tau) h(t): its line factors g(tau0), g(tau1) and time factors
// h(ta), h(tb) are computed once per line, and sin^2(pi s) at the edge is
// shared by both corners, so an edge foot costs three sinpi instead of
// twelve transcendental calls.  Other fields use edge_foot.
struct LineFeet {
  double tau0, tau1, ta, tb;
  bool swirl;
  double a0a = 0, a0b = 0, a1a = 0, a1b = 0;  // along-line speed factors: corner line, time
  __device__ __forceinline__ LineFeet(const SweepField &f, double tau0_, double tau1_, double ta_,
                                      double tb_)
      : tau0(tau0_), tau1(tau1_), ta(ta_), tb(tb_), swirl(f.vel == VEL_SWIRL) {
    if (swirl) {
      const double sg = f.dir == 0 ? 1.0 : -1.0;
      const double ca = cospi(ta / f.vp[0]), cb = cospi(tb / f.vp[0]);
      const double g0 = sg * sinpi(2.0 * tau0), g1 = sg * sinpi(2.0 * tau1);
      a0a = g0 * ca;
      a0b = g0 * cb;
      a1a = g1 * ca;
      a1b = g1 * cb;
    }
  }
  __device__ __forceinline__ double foot(const SweepField &f, int e) const {
    if (!swirl) return edge_foot(f, e, tau0, tau1, ta, tb);
    const double s = f.s_min + f.h * e;
    const double ss = sinpi(s), s2 = ss * ss;
    const double w0 = a0b * s2, w1 = a1b * s2;  // speed at the corners at tb
    const double q0 = sinpi(s - f.Dt * w0), q1 = sinpi(s - f.Dt * w1);
    const double c0 = s - 0.5 * f.Dt * (w0 + a0a * q0 * q0);
    const double c1 = s - 0.5 * f.Dt * (w1 + a1a * q1 * q1);
    return 0.5 * (c0 + c1);
  }
};

// Stencil of line gl's w input: w_k = sum_{m=-3..4} om[m+3] C_{k+n0+m} - mu
// w_{k-1}, i.e. (1/c) M b with b the remap + foot-derivative stencil of the
// shared foot -sigma = n0 + xi and M b_k = (b_{k-1} + 10 b_k + b_{k+1}) / 12.
template <typename T>
__device__ __forceinline__ void filter_line_stencil(const SweepField &F, long long gl,
                                                    double toff, T *om, int *n0) {
  const double tau0 = F.t_min + F.ht * (double)gl;
  const double tau1 = F.t_min + F.ht * (double)(gl + 1);
  const double f0 = edge_foot(F, 0, tau0, tau1, toff + F.ta_rel, toff + F.tb_rel);
  const double u = (f0 - F.s_min) / F.h;
  const double fl = floor(u);
  *n0 = (int)fl;
  const double x = u - fl, x2 = x * x, x3 = x2 * x;
  const double A = x - 2.0 * x2 + x3, B = x3 - x2, Cc = 3.0 * x2 - 2.0 * x3;
  const double kq = F.kb * F.inv12h;
  const double pm2 = 2.0 * x3 - 6.0 * x2 + 3.0 * x + 1.0;
  const double pm1 = -8.0 * x3 + 18.0 * x2 + 6.0 * x - 15.0;
  const double pz = 12.0 * x3 - 18.0 * x2 - 24.0 * x + 15.0;
  const double pp1 = -8.0 * x3 + 6.0 * x2 + 18.0 * x - 1.0;
  const double pp2 = 2.0 * x3 - 3.0 * x;
  double o[6];  // b_k = sum_{j<6} o_j C_{k+n0-2+j}
  o[0] = A / 12.0 - kq * pm2;
  o[1] = (B - 8.0 * A) / 12.0 + kq * (pm2 - pm1);
  o[2] = 1.0 - Cc - 2.0 * B / 3.0 + kq * (pm1 - pz);
  o[3] = Cc + 2.0 * A / 3.0 + kq * (pz - pp1);
  o[4] = (8.0 * B - A) / 12.0 + kq * (pp1 - pp2);
  o[5] = -B / 12.0 + kq * pp2;
  const double icw = F.sm_inv_den / 12.0;
#pragma unroll
  for (int m = 0; m < 8; ++m) {  // tap m - 3
    const double from_bm = m < 6 ? o[m] : 0.0;                  // b_{k-1}
    const double from_bc = (m >= 1 && m < 7) ? o[m - 1] : 0.0;  // b_k
    const double from_bp = m >= 2 ? o[m - 2] : 0.0;             // b_{k+1}
    om[m] = T(icw * (from_bm + 10.0 * from_bc + from_bp));
  }
}

}  // namespace ccfv
