// sweep.cu -- the fused T2S4 CC-CFV sweep for sm_100a.
//
// One launch performs one directional sub-step (an x(dt/2) or y(dt) sweep of
// GpuOneStep, T2S4_Parareal.cu:824-963) for any number of fields.  Per line
// of cells it fuses what the reference spreads over ~11 kernels and ~40
// N^2-sized global arrays:
//   characteristic feet of the cell edges     (T2S4:203-258)
//   PPM reconstruction + conservative remap   (T2S4:260-438)
//   4th-order derivative at the edge feet     (T2S4:440-547)
//   Crank-Nicolson RHS + compact mass matrix  (T2S4:550-654)
//   tridiagonal solve                         (T2S4:657-719)
// Each cell is read once from HBM and written once.
//
// Work decomposition.  A tile is LPG = 16 neighbouring lines.  A cluster of
// cs CTAs covers the whole length of the tile's lines, each CTA a run of up
// to LC_MAX consecutive positions plus a halo on both sides (loaded from
// global memory; in place is safe because every store happens after a
// cluster-wide barrier that follows all loads).  The shared tile is
// [position][line] with an odd pitch: for x-sweeps global rows of 16
// doubles (128 B) land in shared rows; for y-sweeps each line is a
// contiguous global run written down a shared column.
//
// Thread mapping: lane % 16 = line, each thread owns a chunk of consecutive
// positions of its line.  The constant-coefficient tridiagonal system is
// solved as two first-order linear recurrences (LU forward / backward) with
// line-invariant factors alpha_k, g_k precomputed per (L, dt, K): every
// chunk runs its recurrence locally from a zero carry, the chunk maps
// (prod alpha, local value) are composed across the CTA (shared memory) and
// across the cluster (distributed shared memory), and a fix-up pass adds the
// carried-in value times the running product.  The periodic (cyclic) system
// adds a Sherman-Morrison rank-one correction with a line-invariant vector.
#include <cooperative_groups.h>

#include <atomic>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "ccfv_internal.h"
#include "sweep_math.cuh"

namespace cg = cooperative_groups;

namespace ccfv {

namespace {

// Field of tile `tile` (fields sorted by group0): binary search on the
// launch's compact group0 index when it has one (batched launches of
// thousands of fields: a few cache lines instead of one descriptor line per
// probe), else on the descriptors.
__device__ __forceinline__ int find_field(const SweepField *__restrict__ fields,
                                          const int *__restrict__ g0idx, int nfields, int tile) {
  int lo = 0, hi = nfields - 1;
  if (g0idx) {
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(g0idx + mid) <= tile) lo = mid; else hi = mid - 1;
    }
  } else {
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(&fields[mid].group0) <= tile) lo = mid; else hi = mid - 1;
    }
  }
  return lo;
}

// A field's launch time offset (field_active, ccfv_internal.h, says whether
// it takes part in a batched launch).
__device__ __forceinline__ double field_time(const SweepField &f, double toff, int jstep,
                                             int nslice) {
  return toff + jstep * f.t_step + (f.slice < 0 ? nslice * f.t_slice : 0.0);
}

// Input and output of a field in a launch (SweepField::pp): in place, or the
// ping-pong pair of an out-of-place sweep sequence.  Out of place, no CTA
// reads what another CTA of the launch writes.
__device__ __forceinline__ void field_io(const SweepField &f, int jstep, const void **src,
                                         void **dst) {
  if (!f.pp) {
    *src = f.data;
    *dst = f.data;
    return;
  }
  const int s = 3 * jstep + f.kind;
  const bool toA = ((s + f.par) & 1) != 0;
  *dst = toA ? f.data : f.data2;
  *src = s == 0 ? f.in0 : (toA ? f.data2 : f.data);
}

// Bounds-checked view of one line in the shared tile, indexed by position.
template <typename T>
struct LineView {
  const T *cs;
  int base;   // row of position 0 = H - p0
  int nrows;
  unsigned *status;
  __device__ __forceinline__ T operator()(int pos) const {
    int row = pos + base;
    if (row < 0 || row >= nrows) {
      atomicOr(status, STATUS_HALO);
      return T(0);
    }
    return cs[row * PITCH];
  }
};

template <typename T>
struct Ppm {
  T CL, D, C6;
};

// PPM coefficients of cell i (x_step_ppm_coef_on_gpu, T2S4:260-304); ghost
// cells are already in the tile (compat) or it holds wrapped cells (periodic).
template <typename T>
__device__ __forceinline__ Ppm<T> ppm(const LineView<T> &v, int i) {
  const T one_twelfth = T(1.0 / 12.0), seven_twelfths = T(7.0 / 12.0);
  T cm2 = v(i - 2), cm1 = v(i - 1), c0 = v(i), cp1 = v(i + 1), cp2 = v(i + 2);
  T cl = seven_twelfths * (c0 + cm1) - one_twelfth * (cp1 + cm2);
  T cr = seven_twelfths * (cp1 + c0) - one_twelfth * (cp2 + cm1);
  Ppm<T> p;
  p.CL = cl;
  p.D = cr - cl;
  p.C6 = T(6.0) * (c0 - T(0.5) * (cl + cr));
  return p;
}

// PPM antiderivative in cell units (d_intC_ppm4th, T2S4:63-65).
template <typename T>
__device__ __forceinline__ T ppm_int(const Ppm<T> &p, T xi) {
  T xi2 = xi * xi;
  return T(-1.0 / 3) * p.C6 * (xi2 * xi) + T(0.5) * (p.D + p.C6) * xi2 + p.CL * xi;
}

// Neumaier-compensated sum of cells lo..hi.
template <typename T>
__device__ __forceinline__ T sum_cells(const LineView<T> &v, int lo, int hi) {
  T s = T(0), comp = T(0);
  for (int k = lo; k <= hi; ++k) {
    T x = v(k);
    T t = s + x;
    comp += (fabs(s) >= fabs(x)) ? ((s - t) + x) : ((x - t) + s);
    s = t;
  }
  return s + comp;
}

// Conservative remap of one cell over its departure interval [fL, fR].
// compat: x_step_intC_ppm_on_gpu / y_step_intC_ppm_on_gpu (T2S4:306-438):
// zero inflow from outside the domain, feet clamped by eps_remap.  The
// reference's y-remap reads the next row's first cell when its right foot
// is clamped onto the top edge (jR == Ny, an O(2^-53 * Ny) contribution);
// here that term is zero.
template <typename T>
__device__ __forceinline__ T remap_cell(const SweepField &f, const LineView<T> &v, double fL,
                                        double fR) {
  const int L = f.L;
  if (f.bc == BC_COMPAT) {
    if (fL > f.s_max || fR < f.s_min || fL == fR) return T(0);
    double xL = fmax(fL, f.s_min + f.eps_remap);
    double xR = fmin(fR, f.s_max - f.eps_remap);
    int iL = (int)floor((xL - f.s_min) / f.h);
    int iR = (int)floor((xR - f.s_min) / f.h);
    T xiL = (T)((xL - (f.s_min + f.h * iL)) / f.h);
    T xiR = (T)((xR - (f.s_min + f.h * iR)) / f.h);
    Ppm<T> z{T(0), T(0), T(0)};
    Ppm<T> pL = (iL >= 0 && iL < L) ? ppm(v, iL) : z;
    if (iR == iL) return ppm_int(pL, xiR) - ppm_int(pL, xiL);
    Ppm<T> pR = (iR >= 0 && iR < L) ? ppm(v, iR) : z;
    T IntCL = ppm_int(pL, T(1)) - ppm_int(pL, xiL);
    T IntCR = ppm_int(pR, xiR);
    T IntCM = T(0);
    int hi = iR - 1 < L - 1 ? iR - 1 : L - 1;
    for (int k = iL + 1; k <= hi; ++k) IntCM += v(k);
    return IntCL + IntCM + IntCR;
  } else {
    double uL = (fL - f.s_min) / f.h, uR = (fR - f.s_min) / f.h;
    double fkL = floor(uL), fkR = floor(uR);
    int kL = (int)fkL, kR = (int)fkR;
    T xiL = (T)(uL - fkL), xiR = (T)(uR - fkR);
    Ppm<T> pL = ppm(v, kL);
    if (kR == kL) return ppm_int(pL, xiR) - ppm_int(pL, xiL);
    if (abs(kR - kL) > v.nrows) {  // cannot happen within the staged halo
      atomicOr(v.status, STATUS_HALO);
      return T(0);
    }
    Ppm<T> pR = ppm(v, kR);
    if (kR > kL) return sum_cells(v, kL, kR - 1) + ppm_int(pR, xiR) - ppm_int(pL, xiL);
    return -(sum_cells(v, kR, kL - 1) + ppm_int(pL, xiL) - ppm_int(pR, xiR));
  }
}

// Fourth-order derivative at a foot (dcdx_bar_on_gpu / dcdy_bar_on_gpu,
// T2S4:440-547).  compat keeps the reference's ghost selection at iL = L-2
// (+2 tap reads C_{N+1}) and iL = 1 (-2 tap reads C_{-2}).
template <typename T>
__device__ __forceinline__ T foot_derivative(const SweepField &f, const LineView<T> &v, double fb) {
  const int L = f.L;
  int iL, pm2, pp2;
  T xi;
  if (f.bc == BC_COMPAT) {
    if (!(fb >= f.s_min && fb <= f.s_max)) return T(0);
    double ixb = fmin(fmax(fb, f.s_min + 1e-15), f.s_max - 1e-15);
    iL = (int)floor((ixb - f.s_min) / f.h);
    xi = (T)((ixb - (f.s_min + f.h * iL)) / f.h);
    pm2 = (iL == 1) ? -2 : iL - 2;
    pp2 = (iL == L - 2) ? L + 1 : iL + 2;
  } else {
    double u = (fb - f.s_min) / f.h, fk = floor(u);
    iL = (int)fk;
    xi = (T)(u - fk);
    pm2 = iL - 2;
    pp2 = iL + 2;
  }
  T Cim2 = v(pm2), Cim1 = v(iL - 1), Ci = v(iL), Cip1 = v(iL + 1), Cip2 = v(pp2);
  T xi2 = xi * xi, xi3 = xi2 * xi;
  return T(f.inv12h) * ((T(2.0) * xi3 - T(6.0) * xi2 + T(3.0) * xi + T(1.0)) * Cim2 +
                        (T(-8.0) * xi3 + T(18.0) * xi2 + T(6.0) * xi - T(15.0)) * Cim1 +
                        (T(12.0) * xi3 - T(18.0) * xi2 - T(24.0) * xi + T(15.0)) * Ci +
                        (T(-8.0) * xi3 + T(6.0) * xi2 + T(18.0) * xi - T(1.0)) * Cip1 +
                        (T(2.0) * xi3 - T(3.0) * xi) * Cip2);
}

// Compat ghost cells C_{-2}, C_{-1}, C_N, C_{N+1} of one line of a tile
// (3-point extrapolation, T2S4:275-286), written where the tile's rows
// [lo, hi) cover them.  base = row of position 0.
template <typename T>
__device__ __forceinline__ void compat_ghosts(T *c, int base, int lo, int hi, int L) {
  const T one_eleventh = T(1.0 / 11.0);
  if (lo <= -2 && hi > 2) {
    T c0 = c[(base + 0) * PITCH], c1 = c[(base + 1) * PITCH], c2 = c[(base + 2) * PITCH];
    c[(base - 1) * PITCH] = one_eleventh * (-c2 + T(3) * c1 + T(9) * c0);
    c[(base - 2) * PITCH] = one_eleventh * (T(-15) * c2 + T(56) * c1 - T(30) * c0);
  }
  if (hi >= L + 2 && lo <= L - 3) {
    T a = c[(base + L - 3) * PITCH], b = c[(base + L - 2) * PITCH], d = c[(base + L - 1) * PITCH];
    c[(base + L) * PITCH] = one_eleventh * (-a + T(3) * b + T(9) * d);
    c[(base + L + 1) * PITCH] = one_eleventh * (T(-15) * a + T(56) * b - T(30) * d);
  }
}

// Source f(x, y, t) (the reference's f is identically zero, T2S4:58-61;
// Gaussian: sp0 exp(-((x-sp1)^2 + (y-sp2)^2) / sp3) cos(sp4 t)).
__device__ __forceinline__ double src_f(const SweepField &f, double x, double y, double t) {
  const double dx = x - f.sp[1], dy = y - f.sp[2];
  return f.sp[0] * exp(-(dx * dx + dy * dy) / f.sp[3]) * cos(f.sp[4] * t);
}

// 3x3 Simpson cell average of f over cell `pos` of line `gl` at time t
// (get_source_term_on_gpu, T2S4:142-165).
__device__ double src_cell(const SweepField &f, int pos, long long gl, double t) {
  const double s = f.s_min + (pos + 0.5) * f.h, tau = f.t_min + (gl + 0.5) * f.ht;
  const double x_i = f.dir == 0 ? s : tau, y_j = f.dir == 0 ? tau : s;
  const double dx = f.dir == 0 ? f.h : f.ht, dy = f.dir == 0 ? f.ht : f.h;
  const double xm = x_i - 0.5 * dx, xp = x_i + 0.5 * dx, ym = y_j - 0.5 * dy, yp = y_j + 0.5 * dy;
  return 1.0 / 36.0 *
         (src_f(f, xm, ym, t) + src_f(f, xp, ym, t) + src_f(f, xm, yp, t) + src_f(f, xp, yp, t) +
          4.0 * (src_f(f, xm, y_j, t) + src_f(f, xp, y_j, t) + src_f(f, x_i, ym, t) +
                 src_f(f, x_i, yp, t)) +
          16.0 * src_f(f, x_i, y_j, t));
}

// Uniform displacement: every edge foot of a line sits at e - sigma
// (position units), -sigma = n0 + xi0 from the foot f0 of edge 0.  Remap,
// foot derivative and RHS then reduce to fixed 6-tap stencils whose weights
// depend on xi0 only:
//   remap_k = sum_t w_t C_{k+n0+t},  kb (D_{k+1}-D_k) = sum_t q_t C_{k+n0+t}
// (t = -2..3; q includes (1-theta) K Dt/h and 1/(12h)), the same PPM integral
// and cubic derivative weights as the per-cell formulas (T2S4:63-65,
// 440-547), so the stencil and per-cell paths agree to rounding.
template <typename T>
__device__ __forceinline__ void uniform_weights(const SweepField &F, double f0, T w[6], T qd[6],
                                                int *n0) {
  const double u = (f0 - F.s_min) / F.h;
  const double fl = floor(u);
  *n0 = (int)fl;
  const double x = u - fl, x2 = x * x, x3 = x2 * x;
  const double A = x - 2.0 * x2 + x3, B = x3 - x2, Cc = 3.0 * x2 - 2.0 * x3;
  w[0] = T(A / 12.0);
  w[1] = T((B - 8.0 * A) / 12.0);
  w[2] = T(1.0 - Cc - 2.0 * B / 3.0);
  w[3] = T(Cc + 2.0 * A / 3.0);
  w[4] = T((8.0 * B - A) / 12.0);
  w[5] = T(-B / 12.0);
  const double pm2 = 2.0 * x3 - 6.0 * x2 + 3.0 * x + 1.0;
  const double pm1 = -8.0 * x3 + 18.0 * x2 + 6.0 * x - 15.0;
  const double pz = 12.0 * x3 - 18.0 * x2 - 24.0 * x + 15.0;
  const double pp1 = -8.0 * x3 + 6.0 * x2 + 18.0 * x - 1.0;
  const double pp2 = 2.0 * x3 - 3.0 * x;
  const double kq = F.kb * F.inv12h;
  qd[0] = T(kq * -pm2);
  qd[1] = T(kq * (pm2 - pm1));
  qd[2] = T(kq * (pm1 - pz));
  qd[3] = T(kq * (pz - pp1));
  qd[4] = T(kq * (pp1 - pp2));
  qd[5] = T(kq * pp2);
}

// Shared-memory carve-up of the sweep kernel.
template <typename T>
struct Smem {
  T *C;      // [(lc_max + 2H) * PITCH]  tile 0: the input cells
  T *B;      // [(lc_max + 2H) * PITCH]  tile 1
  // Both tiles are indexed by row = position - p0 + H.  Derivative of the
  // input: b -> tile 1, q/x -> tile 0.  Derivative of the remapped field:
  // remap -> tile 1, b -> tile 0, q/x -> tile 1.
  T *tA;     // [lc_max]  alpha_k
  T *tG;     // [lc_max]  g_k
  T *tZ;     // [lc_max]  z_k (periodic)
  T *aggA;   // [NCH * LPG] chunk products
  T *aggF;   // [NCH * LPG] chunk forward values
  T *aggR;   // [NCH * LPG] chunk backward values
  T *xch;    // [8 * LPG] cluster exchange: fwdA fwdB bwdA bwdB y0 yL
  T *Fs;     // [(lc_max + 2H) * PITCH] source cell averages at t_a (source variant only)
  SweepField *fd;
};

template <typename T>
__device__ __forceinline__ Smem<T> carve(unsigned char *raw, int lc_max, int H) {
  Smem<T> s;
  s.fd = reinterpret_cast<SweepField *>(raw);
  T *p = reinterpret_cast<T *>(raw + FD_BYTES);
  s.C = p;
  p += (lc_max + 2 * H) * PITCH;
  s.B = p;
  p += (lc_max + 2 * H) * PITCH;
  s.tA = p;
  p += lc_max;
  s.tG = p;
  p += lc_max;
  s.tZ = p;
  p += lc_max;
  s.aggA = p;
  p += NCH * LPG;
  s.aggF = p;
  p += NCH * LPG;
  s.aggR = p;
  p += NCH * LPG;
  s.xch = p;
  p += 8 * LPG;
  s.Fs = p;
  return s;
}

template <typename T>
__global__ void __launch_bounds__(NTH, 2) sweep_kernel(const SweepField *__restrict__ fields,
                                                    int nfields, int group_base, double toff,
                                                    void *data_override, int lc_max, int H,
                                                    unsigned *status, int jstep, int nslice,
                                                    const int *nlo, const int *g0idx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cg::cluster_group cluster = cg::this_cluster();
  const int cs = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const int tile = blockIdx.x / cs + group_base;
  Smem<T> S = carve<T>(smem_raw, lc_max, H);

  // ---- descriptor of this tile's field (binary search on group0) ----
  if (threadIdx.x == 0) {
    *S.fd = fields[find_field(fields, g0idx, nfields, tile)];
    if (data_override) {
      S.fd->data = data_override;
      if (S.fd->pp) S.fd->in0 = data_override;
    }
  }
  __syncthreads();
  const SweepField &F = *S.fd;
  if (!field_active(F, jstep, nslice, nlo)) return;  // uniform over the cluster
  toff = field_time(F, toff, jstep, nslice);
  const int L = F.L;
  const int g = tile - F.group0;
  const long long line0 = (long long)g * LPG;
  const int Lc = (L + cs - 1) / cs;
  const int p0 = min(L, rank * Lc);
  const int p1 = min(L, p0 + Lc);
  const int np = p1 - p0;
  const int nrows = np + 2 * H;
  const bool periodic = F.bc == BC_PERIODIC;
  const T *gsrc;
  T *gdst;
  {
    const void *vs;
    void *vd;
    field_io(F, jstep, &vs, &vd);
    gsrc = reinterpret_cast<const T *>(vs);
    gdst = reinterpret_cast<T *>(vd);
  }

  // ---- phase 0: stage the tile (+halo) and the solver factors ----
  {
    const int total = nrows * LPG;
    const bool xs = (F.s_line == 1);
    for (int e = threadIdx.x; e < total; e += NTH) {
      int row, ln;
      if (xs) { row = e / LPG; ln = e - row * LPG; }
      else { ln = e / nrows; row = e - ln * nrows; }
      int pos = p0 - H + row;
      long long gl = line0 + ln;
      T val = T(0);
      if (gl < F.M) {
        bool ok = true;
        if (pos < 0 || pos >= L) {
          if (periodic) { pos %= L; if (pos < 0) pos += L; }
          else ok = false;
        }
        if (ok) val = gsrc[(long long)pos * F.s_pos + gl * F.s_line];
      }
      S.C[row * PITCH + ln] = val;
    }
    const T *tab = reinterpret_cast<const T *>(F.tab);
    for (int k = threadIdx.x; k < np; k += NTH) {
      S.tA[k] = tab[p0 + k];
      S.tG[k] = tab[L + p0 + k];
      S.tZ[k] = periodic ? tab[2 * L + p0 + k] : T(0);
    }
  }
  __syncthreads();
  if (!periodic && threadIdx.x < LPG) compat_ghosts(S.C + threadIdx.x, H - p0, p0 - H, p1 + H, L);
  // source: f(t_a) (f(t_b) in the third sub-step) on the staged rows, remapped
  // like C (T2S4:846-853, 893-900, 944-951); f(t_b) enters unremapped
  const double t_src0 = toff + (F.src_tb ? F.tb_rel : F.ta_rel);
  const double t_src1 = toff + F.tb_rel;
  if (F.src) {
    for (int e = threadIdx.x; e < nrows * LPG; e += NTH) {
      const int row = e / LPG, l = e - row * LPG;
      int pos = p0 - H + row;
      T val = T(0);
      if (periodic) {
        pos %= L;
        if (pos < 0) pos += L;
        val = T(src_cell(F, pos, line0 + l, t_src0));
      } else if (pos >= 0 && pos < L) {
        val = T(src_cell(F, pos, line0 + l, t_src0));
      }
      S.Fs[row * PITCH + l] = val;
    }
    __syncthreads();
    if (!periodic && threadIdx.x < LPG) compat_ghosts(S.Fs + threadIdx.x, H - p0, p0 - H, p1 + H, L);
  }
  __syncthreads();

  // ---- thread -> (line, chunk) ----
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ln = lane % LPG;
  const int c = warp * CPW + lane / LPG;
  const long long gl = line0 + ln;
  const int m = (np + NCH - 1) / NCH;
  const int s = min(p1, p0 + c * m);
  const int e = min(p1, s + m);
  const int clast = (np - 1) / m;  // last non-empty chunk
  LineView<T> v{S.C + ln, H - p0, nrows, status};

  // ---- phase 1: feet, remap, foot derivative, RHS b ----
  // b_k = remap_k + w (remap(f)_k + f_k) + 0.5 K Dt/h (D_{k+1} - D_k)
  // (x_b_RHS_on_gpu / y_b_RHS_on_gpu, T2S4:564-613); w = src_w, 0 without a
  // source (the reference's f is identically zero, T2S4:58-61).
  T *bArr, *qArr;
  {
    const LineView<T> vf{S.Fs + ln, H - p0, nrows, status};  // read only when F.src
    const T srcw = T(F.src_w);
    auto src_term = [&](int k, double fa, double fb) -> T {
      int kk = k;
      if (periodic) { kk %= L; if (kk < 0) kk += L; }
      return srcw * (remap_cell(F, vf, fa, fb) + T(src_cell(F, kk, line0 + ln, t_src1)));
    };
    // the shared-foot stencils cover C only; with a source every cell takes
    // the per-cell path
    const bool stencil = F.uniform && !F.src;
    int kb = s, ke = e;
    if (c == 0 && (periodic || p0 > 0)) kb = p0 - 1;
    if (c == clast && (periodic || p1 < L)) ke = p1 + 1;
    const double tau0 = F.t_min + F.ht * (double)gl;
    const double tau1 = F.t_min + F.ht * (double)(gl + 1);
    const double ta = toff + F.ta_rel, tb = toff + F.tb_rel;
    const LineFeet lf(F, tau0, tau1, ta, tb);
    const T kbc = T(F.kb);
    // uniform displacement: shared-foot stencils (uniform_weights)
    int n0 = 0, klo = 1, khi = 0;
    T w[6], qd[6];
    if (stencil) {
      uniform_weights<T>(F, lf.foot(F, 0), w, qd, &n0);
      if (periodic) { klo = INT_MIN; khi = INT_MAX; }
      else { klo = 2 - n0; khi = L - 4 - n0; }  // clear of clamps and ghost quirks
    }
    if (F.dsrc == 0) {
      bArr = S.B;
      qArr = S.C;
      if (stencil) {
        for (int k = kb; k < ke; ++k) {
          T bk;
          if (k >= klo && k <= khi) {
            const int r = k + n0 + H - p0 - 2;
            const T *cp = S.C + r * PITCH + ln;
            if (r < 0 || r + 5 >= nrows) { atomicOr(status, STATUS_HALO); bk = T(0); }
            else {
              bk = T(0);
#pragma unroll
              for (int t = 0; t < 6; ++t) bk += (w[t] + qd[t]) * cp[t * PITCH];
            }
          } else {
            double fa = lf.foot(F, k);
            double fb = lf.foot(F, k + 1);
            bk = remap_cell(F, v, fa, fb) + kbc * (foot_derivative(F, v, fb) - foot_derivative(F, v, fa));
          }
          bArr[(k - p0 + H) * PITCH + ln] = bk;
        }
      } else if (kb < ke) {
        double fprev = lf.foot(F, kb);
        T dprev = foot_derivative(F, v, fprev);
        for (int k = kb; k < ke; ++k) {
          double fnext = lf.foot(F, k + 1);
          T dnext = foot_derivative(F, v, fnext);
          T ic = remap_cell(F, v, fprev, fnext);
          T bk = ic + kbc * (dnext - dprev);
          if (F.src) bk += src_term(k, fprev, fnext);
          bArr[(k - p0 + H) * PITCH + ln] = bk;
          fprev = fnext;
          dprev = dnext;
        }
      }
    } else {
      // The reference's third sweep differentiates the remapped field
      // (dcdx_bar_on_gpu(v_d_Cnphf_bar_x, ...), T2S4:929-932): remap the
      // cells p0-hd .. p1+hd-1 into tile 1 first, then differentiate it.
      T *R = S.B;
      int q0 = p0 - F.hd, q1 = p1 + F.hd;
      if (!periodic) { q0 = max(q0, 0); q1 = min(q1, L); }
      const int m1 = (q1 - q0 + NCH - 1) / NCH;
      const int r0 = q0 + c * m1, r1 = min(q1, r0 + m1);
      for (int k = r0; k < r1; ++k) {
        T ik;
        if (stencil && k >= klo && k <= khi) {
          const int r = k + n0 + H - p0 - 2;
          const T *cp = S.C + r * PITCH + ln;
          if (r < 0 || r + 5 >= nrows) { atomicOr(status, STATUS_HALO); ik = T(0); }
          else {
            ik = T(0);
#pragma unroll
            for (int t = 0; t < 6; ++t) ik += w[t] * cp[t * PITCH];
          }
        } else {
          double fa = lf.foot(F, k);
          double fb = lf.foot(F, k + 1);
          ik = remap_cell(F, v, fa, fb);
        }
        R[(k - p0 + H) * PITCH + ln] = ik;
      }
      __syncthreads();
      if (!periodic && threadIdx.x < LPG) compat_ghosts(R + threadIdx.x, H - p0, q0 - 2, q1 + 2, L);
      __syncthreads();
      LineView<T> vr{R + ln, H - p0, nrows, status};
      bArr = S.C;
      qArr = S.B;
      for (int k = kb; k < ke; ++k) {
        T bk;
        if (stencil && k >= klo && k <= khi) {
          const int r = k + n0 + H - p0 - 2;
          const T *rp = R + r * PITCH + ln;
          if (r < 0 || r + 5 >= nrows) { atomicOr(status, STATUS_HALO); bk = T(0); }
          else {
            T acc = T(0);
#pragma unroll
            for (int t = 0; t < 6; ++t) acc += qd[t] * rp[t * PITCH];
            bk = vr(k) + acc;
          }
        } else {
          double fa = lf.foot(F, k);
          double fb = lf.foot(F, k + 1);
          bk = vr(k) + kbc * (foot_derivative(F, vr, fb) - foot_derivative(F, vr, fa));
          if (F.src) bk += src_term(k, fa, fb);
        }
        bArr[(k - p0 + H) * PITCH + ln] = bk;
      }
    }
  }
  __syncthreads();

  // ---- phase 2: compact mass matrix + local forward recurrence ----
  T *Cl = qArr + ln;
  const int rb = H - p0;  // row of position 0 in both tiles
  {
    T A = T(1), q = T(0);
    if (s < e) {
      const T *Bl = bArr + ln;
      T bm = Bl[(s - 1 + rb) * PITCH], bc = Bl[(s + rb) * PITCH];
      for (int k = s; k < e; ++k) {
        T bp = Bl[(k + 1 + rb) * PITCH];
        T mb;
        if (!periodic && k == 0) mb = (T(10.0) * bc + bp) / T(12.0);
        else if (!periodic && k == L - 1) mb = (T(10.0) * bc + bm) / T(12.0);
        else mb = (bp + T(10.0) * bc + bm) / T(12.0);
        const T a = S.tA[k - p0];
        q = S.tG[k - p0] * mb + a * q;
        A *= a;
        Cl[(k + rb) * PITCH] = q;
        bm = bc;
        bc = bp;
      }
    }
    S.aggA[c * LPG + ln] = A;
    S.aggF[c * LPG + ln] = q;
  }
  __syncthreads();

  // ---- phase 3: forward carries (CTA prefix, then cluster prefix) ----
  {
    T PA = T(1), PB = T(0);  // composite of chunks 0..c-1
    for (int j = 0; j < c; ++j) {
      T a = S.aggA[j * LPG + ln], b = S.aggF[j * LPG + ln];
      PB = a * PB + b;
      PA = a * PA;
    }
    T cin = T(0);
    if (cs > 1) {
      T *xA = S.xch, *xB = S.xch + LPG;
      if (c == NCH - 1) {
        T a = S.aggA[c * LPG + ln], b = S.aggF[c * LPG + ln];
        xA[ln] = a * PA;
        xB[ln] = a * PB + b;
      }
      cluster.sync();
      for (int r = 0; r < rank; ++r) {
        const T *ra = cluster.map_shared_rank(xA, r);
        const T *rbv = cluster.map_shared_rank(xB, r);
        cin = ra[ln] * cin + rbv[ln];
      }
    }
    const T carry = PA * cin + PB;
    T P = T(1);
    for (int k = s; k < e; ++k) {
      P *= S.tA[k - p0];
      Cl[(k + rb) * PITCH] += P * carry;
    }
    // ---- phase 4: local backward recurrence ----
    T x = T(0);
    for (int k = e - 1; k >= s; --k) {
      x = Cl[(k + rb) * PITCH] + S.tA[k - p0] * x;
      Cl[(k + rb) * PITCH] = x;
    }
    S.aggR[c * LPG + ln] = x;
  }
  __syncthreads();

  // ---- phase 5: backward carries (CTA suffix, then cluster suffix) ----
  {
    T SA = T(1), SB = T(0);  // composite of chunks NCH-1 .. c+1
    for (int j = NCH - 1; j > c; --j) {
      T a = S.aggA[j * LPG + ln], b = S.aggR[j * LPG + ln];
      SB = b + a * SB;
      SA = a * SA;
    }
    T cin = T(0);
    if (cs > 1) {
      T *xA = S.xch + 2 * LPG, *xB = S.xch + 3 * LPG;
      if (c == 0) {
        T a = S.aggA[ln], b = S.aggR[ln];
        xA[ln] = a * SA;
        xB[ln] = b + a * SB;
      }
      cluster.sync();
      for (int r = cs - 1; r > rank; --r) {
        const T *ra = cluster.map_shared_rank(xA, r);
        const T *rbv = cluster.map_shared_rank(xB, r);
        cin = rbv[ln] + ra[ln] * cin;
      }
    }
    const T carry = SB + SA * cin;
    T P = T(1);
    for (int k = e - 1; k >= s; --k) {
      P *= S.tA[k - p0];
      Cl[(k + rb) * PITCH] += P * carry;
    }
  }

  // ---- phase 6: periodic rank-one (Sherman-Morrison) correction ----
  if (periodic) {
    T *y0 = S.xch + 4 * LPG, *yL = S.xch + 5 * LPG;
    __syncthreads();
    if (rank == 0 && threadIdx.x < LPG) y0[threadIdx.x] = qArr[(H)*PITCH + threadIdx.x];
    if (rank == cs - 1 && threadIdx.x < LPG) yL[threadIdx.x] = qArr[(H + np - 1) * PITCH + threadIdx.x];
    T a0, aL;
    if (cs > 1) {
      cluster.sync();
      a0 = cluster.map_shared_rank(y0, 0)[ln];
      aL = cluster.map_shared_rank(yL, cs - 1)[ln];
    } else {
      __syncthreads();
      a0 = y0[ln];
      aL = yL[ln];
    }
    const T fct = (a0 + T(F.sm_fac) * aL) * T(F.sm_inv_den);
    for (int k = s; k < e; ++k) Cl[(k + rb) * PITCH] -= fct * S.tZ[k - p0];
  }
  __syncthreads();

  // ---- phase 7: store ----
  {
    const int total = np * LPG;
    const bool xs = (F.s_line == 1);
    for (int q = threadIdx.x; q < total; q += NTH) {
      int row, l2;
      if (xs) { row = q / LPG; l2 = q - row * LPG; }
      else { l2 = q / np; row = q - l2 * np; }
      long long gl2 = line0 + l2;
      if (gl2 < F.M)
        gdst[(long long)(p0 + row) * F.s_pos + gl2 * F.s_line] = qArr[(row + H) * PITCH + l2];
    }
  }
  if (cs > 1) cluster.sync();  // keep shared memory alive for remote readers
}


// ---------------------------------------------------------------------------
// Fast path: uniform displacement + periodic cells, derivative of the input.
// Every cell of a line uses the same 6-tap RHS stencil, so phase 1 and the
// forward recurrence fuse into one walk with a sliding register window (one
// shared-memory read per cell).  The chunk prefix / suffix products of
// alpha_k are line-invariant and kept once per chunk, which lets the forward
// fix-up and the backward recurrence fuse into a single reverse walk, and the
// backward fix-up, the Sherman-Morrison correction and the store into a final
// walk.

__device__ __forceinline__ void cp_async8(void *sdst, const void *gsrc) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async4(void *sdst, const void *gsrc) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all_committed() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

static_assert(sizeof(SweepField) % 8 == 0, "descriptor slot");

template <typename T>
struct FastSmem {
  T *C;      // [(lc_max + 2H) * PITCH]
  T *Q;      // [lc_max * PITCH]   q, then x (row = position - p0)
  T *tA, *tG, *tZ, *tP, *tS;  // [lc_max] factors and chunk prefix/suffix products
  T *aggA;   // [NCH]        chunk products (line-invariant)
  T *PA;     // [NCH + 1]    CTA-local exclusive prefix products of the chunks
  T *aggF;   // [NCH * LPG]  chunk forward values
  T *aggR;   // [NCH * LPG]  chunk backward values
  T *om;     // [6 * LPG]    per-line stencil weights
  T *cin;    // [2 * LPG]    per-line carries from the other CTAs of the cluster
  T *xch;    // [8 * LPG]    cluster exchange
  int *n0;   // [LPG]        per-line foot offset
  SweepField *fd;
};

template <typename T>
__device__ __forceinline__ FastSmem<T> carve_fast(unsigned char *raw, int lc_max, int H) {
  FastSmem<T> s;
  s.fd = reinterpret_cast<SweepField *>(raw);
  s.n0 = reinterpret_cast<int *>(raw + FD_BYTES);
  T *p = reinterpret_cast<T *>(raw + FD_BYTES + 64 * sizeof(int));
  s.C = p; p += (lc_max + 2 * H) * PITCH;
  s.Q = p; p += lc_max * PITCH;
  s.tA = p; p += lc_max;
  s.tG = p; p += lc_max;
  s.tZ = p; p += lc_max;
  s.tP = p; p += lc_max;
  s.tS = p; p += lc_max;
  s.aggA = p; p += NCH;
  s.PA = p; p += NCH + 1;
  s.aggF = p; p += NCH * LPG;
  s.aggR = p; p += NCH * LPG;
  s.om = p; p += 6 * LPG;
  s.cin = p; p += 2 * LPG;
  s.xch = p;
  return s;
}

template <typename T>
__global__ void __launch_bounds__(NTH, 2)
    sweep_fast_kernel(const SweepField *__restrict__ fields, int nfields, int group_base,
                      double toff, void *data_override, int lc_max, int H, unsigned *status,
                      int jstep, int nslice, const int *nlo, const int *g0idx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cg::cluster_group cluster = cg::this_cluster();
  const int cs = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const int tile = blockIdx.x / cs + group_base;
  FastSmem<T> S = carve_fast<T>(smem_raw, lc_max, H);
  {
    // every thread finds the field; the descriptor is copied cooperatively
    const int lo = find_field(fields, g0idx, nfields, tile);
    constexpr int NW8 = (int)(sizeof(SweepField) / 8);
    if (threadIdx.x < NW8)
      reinterpret_cast<long long *>(S.fd)[threadIdx.x] =
          __ldg(reinterpret_cast<const long long *>(&fields[lo]) + threadIdx.x);
  }
  __syncthreads();
  if (threadIdx.x == 0 && data_override) {
    S.fd->data = data_override;
    if (S.fd->pp) S.fd->in0 = data_override;
  }
  __syncthreads();
  const SweepField &F = *S.fd;
  if (!field_active(F, jstep, nslice, nlo)) return;  // uniform over the cluster
  toff = field_time(F, toff, jstep, nslice);
  const int L = F.L;
  const long long line0 = (long long)(tile - F.group0) * LPG;
  const int Lc = (L + cs - 1) / cs;
  const int p0 = min(L, rank * Lc);
  const int p1 = min(L, p0 + Lc);
  const int np = p1 - p0;
  const int nrows = np + 2 * H;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  const T *gsrc;
  T *gdst;
  {
    const void *vs;
    void *vd;
    field_io(F, jstep, &vs, &vd);
    gsrc = reinterpret_cast<const T *>(vs);
    gdst = reinterpret_cast<T *>(vd);
  }
  // ---- stage the tile (cp.async, no integer division) ----
  {
    const T *gdata = gsrc;
    if (F.s_line == 1) {
      // x-sweep: a warp copies two rows of 16 consecutive doubles per step
      const int ln = lane & (LPG - 1);
      const long long gl = line0 + ln;
      const bool okl = gl < F.M;
      for (int row = warp * 2 + (lane >> 4); row < nrows; row += 2 * NW) {
        int pos = p0 - H + row;
        if (pos < 0 || pos >= L) { pos %= L; if (pos < 0) pos += L; }
        T *dst = S.C + row * PITCH + ln;
        if (okl) {
          const T *src = gdata + (long long)pos * F.s_pos + gl;
          if (sizeof(T) == 8) cp_async8(dst, src); else cp_async4(dst, src);
        } else {
          *dst = T(0);
        }
      }
    } else {
      // y-sweep: a warp copies 32 consecutive cells of one line per step
      for (int ln = warp; ln < LPG; ln += NW) {
        const long long gl = line0 + ln;
        const bool okl = gl < F.M;
        const T *lbase = gdata + gl * F.s_line;
        for (int row = lane; row < nrows; row += 32) {
          int pos = p0 - H + row;
          if (pos < 0 || pos >= L) { pos %= L; if (pos < 0) pos += L; }
          T *dst = S.C + row * PITCH + ln;
          if (okl) {
            if (sizeof(T) == 8) cp_async8(dst, lbase + pos); else cp_async4(dst, lbase + pos);
          } else {
            *dst = T(0);
          }
        }
      }
    }
    cp_async_commit();
    // solver factors and chunk products of this CTA's positions
    const T *tab = reinterpret_cast<const T *>(F.tab);
    for (int k = threadIdx.x; k < np; k += NTH) {
      S.tA[k] = tab[p0 + k];
      S.tG[k] = tab[L + p0 + k];
      S.tZ[k] = tab[2 * L + p0 + k];
      S.tP[k] = tab[3 * L + p0 + k];
      S.tS[k] = tab[4 * L + p0 + k];
    }
    if (threadIdx.x < NCH) S.aggA[threadIdx.x] = tab[5 * L + rank * NCH + threadIdx.x];
    if (threadIdx.x <= NCH)
      S.PA[threadIdx.x] = tab[5 * L + cs * NCH + rank * (NCH + 1) + threadIdx.x];
    // per-line stencil: b_k = sum_t om_t C_{k+n0+t}, t = -2..3 (see sweep_kernel)
    if (threadIdx.x < LPG) {
      const int l = threadIdx.x;
      const long long gl = line0 + l;
      const double tau0 = F.t_min + F.ht * (double)gl;
      const double tau1 = F.t_min + F.ht * (double)(gl + 1);
      const double f0 = edge_foot(F, 0, tau0, tau1, toff + F.ta_rel, toff + F.tb_rel);
      const double u = (f0 - F.s_min) / F.h;
      const double fl = floor(u);
      S.n0[l] = (int)fl;
      const double x = u - fl, x2 = x * x, x3 = x2 * x;
      const double A = x - 2.0 * x2 + x3, B = x3 - x2, Cc = 3.0 * x2 - 2.0 * x3;
      const double kq = F.kb * F.inv12h;
      const double pm2 = 2.0 * x3 - 6.0 * x2 + 3.0 * x + 1.0;
      const double pm1 = -8.0 * x3 + 18.0 * x2 + 6.0 * x - 15.0;
      const double pz = 12.0 * x3 - 18.0 * x2 - 24.0 * x + 15.0;
      const double pp1 = -8.0 * x3 + 6.0 * x2 + 18.0 * x - 1.0;
      const double pp2 = 2.0 * x3 - 3.0 * x;
      T *om = S.om + 6 * l;
      om[0] = T(A / 12.0 - kq * pm2);
      om[1] = T((B - 8.0 * A) / 12.0 + kq * (pm2 - pm1));
      om[2] = T(1.0 - Cc - 2.0 * B / 3.0 + kq * (pm1 - pz));
      om[3] = T(Cc + 2.0 * A / 3.0 + kq * (pz - pp1));
      om[4] = T((8.0 * B - A) / 12.0 + kq * (pp1 - pp2));
      om[5] = T(-B / 12.0 + kq * pp2);
    }
    cp_async_wait_all_committed();
  }
  __syncthreads();

  const int ln = lane % LPG;
  const int c = warp * CPW + lane / LPG;
  const long long gl = line0 + ln;
  const int m = (np + NCH - 1) / NCH;
  const int s = min(p1, p0 + c * m);
  const int e = min(p1, s + m);

  // ---- fused RHS + compact mass matrix + local forward recurrence ----
  {
    T q = T(0);
    if (s < e) {
      const int n0 = S.n0[ln];
      const int r0 = (s - 1) + n0 - 2 - p0 + H;   // row of tap -2 of cell s-1
      const int rlast = e + n0 + 3 - p0 + H;       // row of tap +3 of cell e
      if (r0 < 0 || rlast >= nrows) {
        atomicOr(status, STATUS_HALO);
      } else {
        const T *omp = S.om + 6 * ln;
        const T o0 = omp[0], o1 = omp[1], o2 = omp[2], o3 = omp[3], o4 = omp[4], o5 = omp[5];
        const T *cp = S.C + r0 * PITCH + ln;
        T w0 = cp[0], w1 = cp[PITCH], w2 = cp[2 * PITCH], w3 = cp[3 * PITCH],
          w4 = cp[4 * PITCH], w5 = cp[5 * PITCH];
        T bm = o0 * w0 + o1 * w1 + o2 * w2 + o3 * w3 + o4 * w4 + o5 * w5;
        w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = cp[6 * PITCH];
        T bc = o0 * w0 + o1 * w1 + o2 * w2 + o3 * w3 + o4 * w4 + o5 * w5;
        const T *nxt = cp + 7 * PITCH;
        T *qp = S.Q + (s - p0) * PITCH + ln;
        const T *ta = S.tA + (s - p0), *tg = S.tG + (s - p0);
        const int n = e - s;
#pragma unroll 4
        for (int i = 0; i < n; ++i) {
          w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = nxt[i * PITCH];
          const T bp = o0 * w0 + o1 * w1 + o2 * w2 + o3 * w3 + o4 * w4 + o5 * w5;
          const T mb = (bp + T(10.0) * bc + bm) * T(1.0 / 12.0);
          q = tg[i] * mb + ta[i] * q;
          qp[i * PITCH] = q;
          bm = bc;
          bc = bp;
        }
      }
    }
    S.aggF[c * LPG + ln] = q;
  }
  __syncthreads();

  // ---- forward carries: CTA prefix (this line) + cluster prefix ----
  T carry;
  {
    T PB = T(0);
    for (int j = 0; j < c; ++j) PB = S.aggA[j] * PB + S.aggF[j * LPG + ln];
    if (cs > 1) {
      T *xB = S.xch + LPG;
      if (c == NCH - 1) xB[ln] = S.aggA[c] * PB + S.aggF[c * LPG + ln];
      cluster.sync();
      if (threadIdx.x < LPG) {  // compose the preceding CTAs once per line
        const T *tab = reinterpret_cast<const T *>(F.tab);
        const T *PAg = tab + 5 * L + cs * NCH;
        T cin = T(0);
        for (int r = 0; r < rank; ++r) {
          const T *rb = cluster.map_shared_rank(xB, r);
          cin = PAg[r * (NCH + 1) + NCH] * cin + rb[threadIdx.x];
        }
        S.cin[threadIdx.x] = cin;
      }
      __syncthreads();
      carry = S.PA[c] * S.cin[ln] + PB;
    } else {
      carry = PB;
    }
  }
  // ---- fused forward fix-up + local backward recurrence (reverse walk) ----
  {
    T x = T(0);
    const int n = e - s;
    T *qp = S.Q + (s - p0) * PITCH + ln;
    const T *ta = S.tA + (s - p0), *tp = S.tP + (s - p0);
#pragma unroll 4
    for (int i = n - 1; i >= 0; --i) {
      x = (qp[i * PITCH] + tp[i] * carry) + ta[i] * x;
      qp[i * PITCH] = x;
    }
    S.aggR[c * LPG + ln] = x;
  }
  __syncthreads();
  // ---- backward carries: CTA suffix + cluster suffix ----
  T carry2;
  {
    T SB = T(0), SA = T(1);
    for (int j = NCH - 1; j > c; --j) {
      const T a = S.aggA[j];
      SB = S.aggR[j * LPG + ln] + a * SB;
      SA = a * SA;
    }
    if (cs > 1) {
      T *xB = S.xch + 3 * LPG;
      if (c == 0) xB[ln] = S.aggR[ln] + S.aggA[0] * SB;
      cluster.sync();
      if (threadIdx.x < LPG) {
        const T *tab = reinterpret_cast<const T *>(F.tab);
        const T *PAg = tab + 5 * L + cs * NCH;
        T cin = T(0);
        for (int r = cs - 1; r > rank; --r) {
          const T *rb = cluster.map_shared_rank(xB, r);
          cin = rb[threadIdx.x] + PAg[r * (NCH + 1) + NCH] * cin;
        }
        S.cin[LPG + threadIdx.x] = cin;
      }
      __syncthreads();
      carry2 = SB + SA * S.cin[LPG + ln];
    } else {
      carry2 = SB;
    }
  }
  // ---- cyclic correction (Sherman-Morrison): needs y_0 and y_{L-1} ----
  T fct;
  {
    T *y0 = S.xch + 4 * LPG, *yL = S.xch + 5 * LPG;
    if (p0 == 0 && s == p0 && s < e) y0[ln] = S.Q[ln] + S.tS[0] * carry2;
    if (p1 == L && e == p1 && s < e) yL[ln] = S.Q[(np - 1) * PITCH + ln] + S.tS[np - 1] * carry2;
    if (cs > 1) {
      cluster.sync();
      if (threadIdx.x < LPG) {
        S.cin[threadIdx.x] = cluster.map_shared_rank(y0, 0)[threadIdx.x];
        S.cin[LPG + threadIdx.x] = cluster.map_shared_rank(yL, cs - 1)[threadIdx.x];
      }
      __syncthreads();
      fct = (S.cin[ln] + T(F.sm_fac) * S.cin[LPG + ln]) * T(F.sm_inv_den);
    } else {
      __syncthreads();
      fct = (y0[ln] + T(F.sm_fac) * yL[ln]) * T(F.sm_inv_den);
    }
  }
  // ---- backward fix-up + correction + store ----
  T *gdata = gdst;
  {
    const int n = e - s;
    T *qp = S.Q + (s - p0) * PITCH + ln;
    const T *ts = S.tS + (s - p0), *tz = S.tZ + (s - p0);
    if (F.s_line == 1) {
      // x-sweep: a half-warp writes 16 consecutive doubles of one row
      if (gl < F.M) {
        T *gp = gdata + (long long)s * F.s_pos + gl;
#pragma unroll 4
        for (int i = 0; i < n; ++i) gp[i * F.s_pos] = qp[i * PITCH] + ts[i] * carry2 - fct * tz[i];
      }
    } else {
#pragma unroll 4
      for (int i = 0; i < n; ++i) qp[i * PITCH] = qp[i * PITCH] + ts[i] * carry2 - fct * tz[i];
      __syncthreads();
      for (int l2 = warp; l2 < LPG; l2 += NW) {
        const long long gl2 = line0 + l2;
        if (gl2 >= F.M) continue;
        T *lbase = gdata + gl2 * F.s_line + p0;
        for (int row = lane; row < np; row += 32) lbase[row] = S.Q[row * PITCH + l2];
      }
    }
  }
  if (cs > 1) cluster.sync();  // keep shared memory alive for remote readers
}

// ---------------------------------------------------------------------------
// Filter path: uniform displacement + periodic cells + derivative of the
// sweep input, for diffusion numbers where |mu| (below) is small enough.
//
// The cyclic constant system a x_{k-1} + b x_k + a x_{k+1} = r_k factors as
// c (1 + mu S^-1)(1 + mu S) x = r with |mu| < 1, mu / (1 + mu^2) = a / b,
// c = a / mu, so it is solved exactly by two first-order recurrences,
//   w_k = r_k / c - mu w_{k-1},   x_k = w_k - mu x_{k+1},
// whose periodic wrap-around needs no correction term.  A recurrence started
// from zero J positions early agrees with the exact one to |mu|^J, and J is
// chosen on the host so that |mu|^J is below the rounding of T.
//
// A CTA owns a segment [p0, p1) of 16 lines.  The 16 lanes of a half-warp
// own one line: lane c holds FCH consecutive positions in registers.  The
// forward recurrence runs over [p0 - J, p1 + J) (zero start J cells early),
// the backward one over [p0, p1 + J) (zero start at its end); inside a line
// the chunks are joined exactly by a 4-step shuffle scan of the chunk maps
// x -> (-mu)^FCH x + e, so only the segment ends are warmed up.  Every phase
// of a line stays inside its half-warp: the only CTA barriers are after the
// staging and before the cooperative store.

constexpr int FCH = 17;  // positions per lane (odd: conflict-free shared-memory columns)
constexpr int FLANES = 16;
// Longest segment for a recurrence warm-up J: 16 * FCH >= np + 2J.
__host__ __device__ constexpr int filter_seg_max(int J) { return FLANES * FCH - 2 * J; }

// Rows of the staged tile: enough for the longest chunk walk, so the solve
// loops need no bounds predicates (rows past the staged ones are only read
// by lanes whose positions lie past the range; their values are masked).
__host__ __device__ inline int filter_tile_rows(int lc_max, int H) {
  return (lc_max > FLANES * FCH ? lc_max : FLANES * FCH) + 2 * H + 8;
}

// Exact (cluster) form: powers (-mu)^e for e = 0 .. FPW - 1 (a segment of at
// most FLANES * FCH cells needs exponents up to FLANES * FCH).
constexpr int FPW = FLANES * FCH + 8;
// Wide stencil form (the reference scheme's third sweep, whose right-hand
// side differentiates the remapped field): 13 taps, a table row of 16.
constexpr int WIDE_TAPS = 13;
constexpr int WIDE_TAPS_PAD = 16;

template <typename T>
struct FiltSmem {
  T *C;      // [filter_tile_rows * PITCH]  input cells, then w, then x
  T *B;      // per-cell form: [filter_tile_rows * PITCH]  b of every position
  T *om;     // [8 * LPG]  weights of w's input (1/c) M b as an 8-tap stencil of C
  T *pwt;    // [32]       (-mu)^(i+1), i = 0 .. FCH-1
  T *pwa;    // exact form: [FPW] (-mu)^e
  T *ex;     // exact form: [2 * LPG] this segment's forward end / backward start per line
  double *et;  // per-cell form: [FPW] sin^2(pi s) of the tile's edges (swirling field)
  int *n0;   // [LPG]
  SweepField *fd;
  int rows;
};

template <typename T, bool EXACT, bool CELL, bool WIDE>
__device__ __forceinline__ FiltSmem<T> carve_filt(unsigned char *raw, int lc_max, int H) {
  FiltSmem<T> s;
  s.fd = reinterpret_cast<SweepField *>(raw);
  s.n0 = reinterpret_cast<int *>(raw + FD_BYTES);
  T *p = reinterpret_cast<T *>(raw + FD_BYTES + 64 * sizeof(int));
  s.om = p; p += (WIDE ? WIDE_TAPS_PAD : 8) * LPG;
  s.pwt = p; p += 32;
  s.pwa = nullptr;
  s.ex = nullptr;
  if (EXACT) {
    s.pwa = p; p += FPW;
    s.ex = p; p += 2 * LPG;
  }
  s.C = p;
  s.rows = filter_tile_rows(lc_max, H);
  s.B = CELL ? p + (size_t)s.rows * PITCH : nullptr;
  s.et = nullptr;
  if (CELL) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(s.B + (size_t)s.rows * PITCH);
    s.et = reinterpret_cast<double *>((a + 7) & ~uintptr_t(7));
  }
  return s;
}

// x^n (n >= 0) by binary powering, in FP64.
__device__ __forceinline__ double powi(double x, int n) {
  double r = 1.0;
  while (n > 0) {
    if (n & 1) r *= x;
    x *= x;
    n >>= 1;
  }
  return r;
}

// Per-cell right-hand side of the filter kernel (velocity fields whose feet
// differ from edge to edge, periodic cells, derivative of the sweep input).
// One edge e of a line: its foot's cell kf and offset xi, the PPM
// antiderivative of cell kf at xi (I(xi), d_intC_ppm4th, T2S4:63-65) and the
// fourth-order derivative at the foot (dcdx_bar_on_gpu, T2S4:440-547).  The
// remap of cell k is then I_{k+1} - I_k plus the whole cells between the two
// feet (x_step_intC_ppm_on_gpu, T2S4:306-347), so every foot, PPM
// reconstruction and derivative is evaluated once per edge instead of twice
// per cell.
template <typename T>
struct CellEdge {
  int kf;
  T phi, d;
};

template <typename T>
__device__ __forceinline__ CellEdge<T> cell_edge_at(const SweepField &F, double f,
                                                    const T *ccol, int rb, int nrows,
                                                    unsigned *status) {
  const double u = (f - F.s_min) / F.h;
  const double fk = floor(u);
  CellEdge<T> r;
  r.kf = (int)fk;
  const T xi = T(u - fk);
  const int row = r.kf + rb;
  if (row < 2 || row + 2 >= nrows) {  // cannot happen within the staged halo
    atomicOr(status, STATUS_HALO);
    r.phi = T(0);
    r.d = T(0);
    return r;
  }
  const T *cp = ccol + (row - 2) * PITCH;
  const T cm2 = cp[0], cm1 = cp[PITCH], c0 = cp[2 * PITCH], cp1 = cp[3 * PITCH],
          cp2 = cp[4 * PITCH];
  // PPM edge values and curvature of cell kf (x_step_ppm_coef_on_gpu, T2S4:260-304)
  const T cl = T(7.0 / 12.0) * (c0 + cm1) - T(1.0 / 12.0) * (cp1 + cm2);
  const T cr = T(7.0 / 12.0) * (cp1 + c0) - T(1.0 / 12.0) * (cp2 + cm1);
  const T D = cr - cl;
  const T C6 = T(6.0) * (c0 - T(0.5) * (cl + cr));
  const T xi2 = xi * xi, xi3 = xi2 * xi;
  r.phi = T(-1.0 / 3) * C6 * xi3 + T(0.5) * (D + C6) * xi2 + cl * xi;
  r.d = T(F.inv12h) * ((T(2.0) * xi3 - T(6.0) * xi2 + T(3.0) * xi + T(1.0)) * cm2 +
                       (T(-8.0) * xi3 + T(18.0) * xi2 + T(6.0) * xi - T(15.0)) * cm1 +
                       (T(12.0) * xi3 - T(18.0) * xi2 - T(24.0) * xi + T(15.0)) * c0 +
                       (T(-8.0) * xi3 + T(6.0) * xi2 + T(18.0) * xi - T(1.0)) * cp1 +
                       (T(2.0) * xi3 - T(3.0) * xi) * cp2);
  return r;
}

template <typename T>
__device__ __forceinline__ CellEdge<T> cell_edge(const SweepField &F, const LineFeet &lf,
                                                 const T *ccol, int rb, int nrows, int e,
                                                 unsigned *status) {
  return cell_edge_at<T>(F, lf.foot(F, e), ccol, rb, nrows, status);
}

// b of the cell between edges l and l+1: remap + (1-theta) K Dt/h (D_r - D_l)
// (x_b_RHS_on_gpu, T2S4:564-613, source-free); the whole cells between the
// feet are summed with Neumaier compensation (periodic remap of sweep_kernel).
template <typename T>
__device__ __forceinline__ T cell_rhs(const CellEdge<T> &l, const CellEdge<T> &r, const T *ccol,
                                      int rb, int nrows, T kbc, unsigned *status) {
  T remap;
  if (r.kf == l.kf) {
    remap = r.phi - l.phi;
  } else {
    const int lo = min(l.kf, r.kf), hi = max(l.kf, r.kf) - 1;
    T s = T(0), comp = T(0);
    if (lo + rb < 0 || hi + rb >= nrows) {
      atomicOr(status, STATUS_HALO);
    } else {
      for (int k = lo; k <= hi; ++k) {
        const T x = ccol[(k + rb) * PITCH];
        const T t = s + x;
        comp += (fabs(s) >= fabs(x)) ? ((s - t) + x) : ((x - t) + s);
        s = t;
      }
    }
    s += comp;
    remap = r.kf > l.kf ? (s + r.phi) - l.phi : -((s + l.phi) - r.phi);
  }
  return remap + kbc * (r.d - l.d);
}

// Compat boundaries (the reference's): an edge whose foot lies inside
// [s_min + eps, s_max - eps] is "normal" (its remap clamps are no-ops); cells
// next to an edge that is not, or whose feet cross, take the reference's
// per-cell remap with its clamps and zero inflow (remap_cell, T2S4:306-438).
// The foot derivative keeps the reference's ghost selection (foot_derivative).
template <typename T>
struct CompatEdge {
  double f;
  int kf;
  bool normal;
  T phi, d;
};

template <typename T>
__device__ __forceinline__ CompatEdge<T> compat_edge(const SweepField &F, const LineFeet &lf,
                                                     const LineView<T> &vc,
                                                     const LineView<T> &vd, int e) {
  CompatEdge<T> r;
  r.f = lf.foot(F, e);
  r.normal = r.f >= F.s_min + F.eps_remap && r.f <= F.s_max - F.eps_remap;
  r.kf = 0;
  r.phi = T(0);
  if (r.normal) {
    const double u = (r.f - F.s_min) / F.h;
    const double fk = floor(u);
    r.kf = (int)fk;
    r.phi = ppm_int(ppm(vc, r.kf), T(u - fk));
  }
  r.d = foot_derivative(F, vd, r.f);
  return r;
}

template <typename T>
__device__ __forceinline__ T compat_remap(const SweepField &F, const CompatEdge<T> &l,
                                          const CompatEdge<T> &r, const LineView<T> &vc) {
  if (l.normal && r.normal && r.kf >= l.kf && l.f != r.f) {
    T s = T(0);
    for (int k = l.kf; k < r.kf; ++k) s += vc(k);
    return (s + r.phi) - l.phi;
  }
  return remap_cell(F, vc, l.f, r.f);
}

// The per-line stencil table of one field (one thread per line).  Wide
// (the reference scheme's third sweep, uniform displacement): b_k = R_k +
// sum_t wq_t R_{k+n0-2+t} with R_j = sum_s wr_s C_{j+n0-2+s} (the compat
// form's interior formulas) composes into 11 taps from C_{k+2n0-4}, valid for
// n0 in [-3, 2]; with the mass matrix 13 taps from C_{k+2n0-5}, stored with
// the shift 2n0-2 so that the kernel's first tap row is k + shift - 3.
template <typename T>
__global__ void filter_weights_kernel(const SweepField *__restrict__ f, T *__restrict__ wt,
                                      int *__restrict__ nt, int lines, int wide) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= lines) return;
  const SweepField F = *f;
  if (wide) {
    double om[WIDE_TAPS_PAD];
    for (int m = 0; m < WIDE_TAPS_PAD; ++m) om[m] = 0.0;
    int shift = 0;
    if (l < F.M) {
      const double tau0 = F.t_min + F.ht * (double)l;
      const double f0 = edge_foot(F, 0, tau0, tau0 + F.ht, F.ta_rel, F.tb_rel);
      double wr[6], wq[6];
      int n0 = 0;
      uniform_weights<double>(F, f0, wr, wq, &n0);
      double bt[11];
      for (int j = 0; j < 11; ++j) bt[j] = 0.0;
      for (int sidx = 0; sidx < 6; ++sidx) {
        const int j = sidx - n0 + 2;
        if (j >= 0 && j < 11) bt[j] += wr[sidx];
      }
      for (int t = 0; t < 6; ++t)
        for (int sidx = 0; sidx < 6; ++sidx) bt[t + sidx] += wq[t] * wr[sidx];
      const double icw = F.sm_inv_den / 12.0;
      for (int m = 0; m < WIDE_TAPS; ++m) {
        const double bm = m < 11 ? bt[m] : 0.0;                       // b_{k-1}
        const double bc = (m >= 1 && m < 12) ? bt[m - 1] : 0.0;       // b_k
        const double bp = m >= 2 ? bt[m - 2] : 0.0;                   // b_{k+1}
        om[m] = icw * (bm + 10.0 * bc + bp);
      }
      shift = 2 * n0 - 2;
    }
    for (int m = 0; m < WIDE_TAPS_PAD; ++m) wt[(size_t)l * WIDE_TAPS_PAD + m] = T(om[m]);
    nt[l] = shift;
    return;
  }
  if (l < F.M) {
    T om[8];
    int n0 = 0;
    filter_line_stencil<T>(F, l, 0.0, om, &n0);
    for (int m = 0; m < 8; ++m) wt[(size_t)l * 8 + m] = om[m];
    nt[l] = n0;
  } else {
    for (int m = 0; m < 8; ++m) wt[(size_t)l * 8 + m] = T(0);
    nt[l] = 0;
  }
}

// Four CTAs per SM (at most 64 registers a thread; shared memory allows no
// more): the kernel is latency bound, and each added CTA was worth more than
// the few registers it spills (2 -> 3 -> 4 CTAs: fine phase 1498 -> 1207 ->
// 1105 us per launch on the 2048^2 x 63-slice bench).
//
// EXACT (out of place, any diffusion number): a line's cs segments form one
// thread-block cluster and no recurrence is warmed up.  Each segment runs
// both filters from a zero start over its own cells only; a segment maps its
// incoming carry linearly, w_end = (-mu)^np w_in + E (forward) and
// x_start = (-mu)^np x_in + X (backward), so after the segments publish E (X)
// in shared memory the periodic closure over the cluster gives every carry
// exactly: w_{L-1} = E_total / (1 - (-mu)^L), then carries segment by
// segment; each cell adds carry * (-mu)^distance from a power table.  The
// field, its activity and the segment length are uniform over a cluster, so
// every CTA of a cluster reaches every cluster barrier.
//
// CELL (velocity fields whose feet differ from edge to edge): the staged
// cells first give every position's b (per-edge feet, PPM antiderivatives and
// foot derivatives, cell_edge / cell_rhs) in a second tile, each line's
// half-warp filling its own column; the forward filter then takes w's input
// as the mass-matrix stencil (1/12c)(b_{k-1} + 10 b_k + b_{k+1}).  Two tiles
// and the per-edge arithmetic: two CTAs per SM.
// COMPAT (per-cell form only): the reference's boundaries, a separate
// instantiation so that the periodic per-cell form carries none of their code.
template <typename T, bool EXACT, bool CELL, bool COMPAT, bool WIDE = false>
__global__ void __launch_bounds__(NTH, (CELL || WIDE) ? 2 : 4)
    sweep_filter_kernel(const SweepField *__restrict__ fields, int nfields, int group_base,
                        double toff, void *data_override, int lc_max, int H, unsigned *status,
                        int jstep, int nslice, const int *nlo, int cs, int clustered,
                        const int *g0idx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // Programmatic dependent launch: nothing is read before the previous grid
  // of the stream has completed (a no-op when launched without the
  // attribute), and the next grid may be scheduled onto the SMs this grid's
  // CTAs free.
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  // CTA -> (field, tile of LPG lines, segment).  The launch's clusters are the
  // cs segments of one tile; fields carry their first CTA and halo, so fields
  // of different segment lengths share one launch (lc_max and H size the
  // shared memory only)
  const int cta = (int)blockIdx.x + group_base;
  FiltSmem<T> S = carve_filt<T, EXACT, CELL, WIDE>(smem_raw, lc_max, H);
  {
    // a field's CTAs start at cta0 = group0 * cs (cs is uniform over a launch);
    // only the threads that copy the descriptor search for it
    constexpr int NW8 = (int)(sizeof(SweepField) / 8);
    if (threadIdx.x < NW8) {
      const int lo = find_field(fields, g0idx, nfields, cta / cs);
      reinterpret_cast<long long *>(S.fd)[threadIdx.x] =
          __ldg(reinterpret_cast<const long long *>(&fields[lo]) + threadIdx.x);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && data_override) {
    S.fd->data = data_override;
    if (S.fd->pp) S.fd->in0 = data_override;
  }
  __syncthreads();
  const SweepField &F = *S.fd;
  if (!field_active(F, jstep, nslice, nlo)) return;
  toff = field_time(F, toff, jstep, nslice);
  const int L = F.L;
  H = F.halo_f;
  const int q = cta - F.cta0;
  const int rank = q % cs;
  const long long line0 = (long long)(q / cs) * LPG;
  // exact form: segments of a whole walk (FLANES * FCH cells) and a shorter
  // last one when cs is the least count that covers the line (full segments
  // need no masking, and their forward end is the scan's carry-out)
  int Lc = (L + cs - 1) / cs;
  if (EXACT && (cs - 1) * (FLANES * FCH) < L && cs * (FLANES * FCH) >= L) Lc = FLANES * FCH;
  const int p0 = min(L, rank * Lc);
  const int p1 = min(L, p0 + Lc);
  const int np = p1 - p0;
  const int nrows = np + 2 * H;
  // compat lines split between two launches (SweepField::hyb): each launch
  // keeps its own segments (uniform over the CTA, before any barrier)
  if (!EXACT && F.hyb > 0 && !clustered) {
    const bool interior = p0 >= F.hyb && p1 + F.hyb <= L;
    if (CELL ? interior : !interior) return;
  }
  const int J = EXACT ? 0 : F.jf;
  const T mu = T(F.sm_fac), ic = T(F.sm_inv_den);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const T *gsrc;
  T *gdst;
  {
    const void *vs;
    void *vd;
    field_io(F, jstep, &vs, &vd);
    gsrc = reinterpret_cast<const T *>(vs);
    gdst = reinterpret_cast<T *>(vd);
  }

  // Descriptor fields used in the loops live in registers: the descriptor is
  // in shared memory, and the copies' memory clobbers and the generic-pointer
  // stores would otherwise make the compiler reload it every iteration.
  const long long s_pos = F.s_pos, s_line = F.s_line, M = F.M;
  const bool xsweep = s_line == 1;
  // compat boundaries (per-cell form only): zero outside the line, ghost
  // cells, non-cyclic solve
  constexpr bool compat = CELL && COMPAT;

  // ---- stage rows p0-H .. p1+H-1 (periodic wrap) ----
  // Rows whose position lies inside the line ([rlo, rhi)) take pointer-stepped
  // copies; only the halo rows outside it wrap (periodic) or are zero (compat).
  {
    const int rlo = max(0, H - p0), rhi = min(nrows, H - p0 + L);
    auto halo_row = [&](T *dcol, const T *lbase, long long step, int row) {
      int pos = p0 - H + row;
      if (compat) {
        dcol[row * PITCH] = T(0);
        return;
      }
      pos %= L;
      if (pos < 0) pos += L;
      const T *src = lbase + (long long)pos * step;
      if (sizeof(T) == 8) cp_async8(dcol + row * PITCH, src); else cp_async4(dcol + row * PITCH, src);
    };
    if (xsweep) {
      // a warp copies two rows of 16 consecutive values (128 B for FP64) per step
      const int ln = lane & (LPG - 1);
      const long long gl = line0 + ln;
      T *dcol = S.C + ln;
      int row = warp * 2 + (lane >> 4);
      if (gl < M) {
        const T *gcol = gsrc + gl;
        for (; row < rlo; row += 2 * NW) halo_row(dcol, gcol, s_pos, row);
        const T *src = gcol + (long long)(p0 - H + row) * s_pos;
        T *dst = dcol + row * PITCH;
        const long long gstep = 2LL * NW * s_pos;
#pragma unroll 4
        for (; row < rhi; row += 2 * NW, src += gstep, dst += 2 * NW * PITCH) {
          if (sizeof(T) == 8) cp_async8(dst, src); else cp_async4(dst, src);
        }
        for (; row < nrows; row += 2 * NW) halo_row(dcol, gcol, s_pos, row);
      } else {
        for (; row < nrows; row += 2 * NW) dcol[row * PITCH] = T(0);
      }
    } else {
      // a warp copies 32 consecutive values of one line per step
      for (int ln = warp; ln < LPG; ln += NW) {
        const long long gl = line0 + ln;
        T *dcol = S.C + ln;
        int row = lane;
        if (gl < M) {
          const T *lbase = gsrc + gl * s_line;
          for (; row < rlo; row += 32) halo_row(dcol, lbase, 1, row);
          const T *src = lbase + (p0 - H + row);
          T *dst = dcol + row * PITCH;
#pragma unroll 4
          for (; row < rhi; row += 32, src += 32, dst += 32 * PITCH) {
            if (sizeof(T) == 8) cp_async8(dst, src); else cp_async4(dst, src);
          }
          for (; row < nrows; row += 32) halo_row(dcol, lbase, 1, row);
        } else {
          for (; row < nrows; row += 32) dcol[row * PITCH] = T(0);
        }
      }
    }
  }
  if (CELL) {
    // per-cell form: no per-line stencil (b is computed per cell below)
  } else if (WIDE) {  // wide stencil rows (WIDE_TAPS_PAD per line) and shifts
    static_assert(WIDE_TAPS_PAD * LPG == NTH, "one table entry per thread");
    const T *src = reinterpret_cast<const T *>(F.wt) + line0 * WIDE_TAPS_PAD + threadIdx.x;
    if (sizeof(T) == 8) cp_async8(S.om + threadIdx.x, src); else cp_async4(S.om + threadIdx.x, src);
    if (threadIdx.x < LPG) cp_async4(S.n0 + threadIdx.x, F.nt + line0 + threadIdx.x);
  } else if (F.wt) {  // per-line stencil from the plan's table, copied with the cells
    if (threadIdx.x < 8 * LPG) {
      const T *src = reinterpret_cast<const T *>(F.wt) + line0 * 8 + threadIdx.x;
      if (sizeof(T) == 8) cp_async8(S.om + threadIdx.x, src); else cp_async4(S.om + threadIdx.x, src);
    } else if (threadIdx.x < 9 * LPG) {
      const int l = threadIdx.x - 8 * LPG;
      cp_async4(S.n0 + l, F.nt + line0 + l);
    }
  }
  cp_async_commit();
  if (!CELL && !WIDE && !F.wt && threadIdx.x < LPG) {
    filter_line_stencil<T>(F, line0 + threadIdx.x, toff, S.om + 8 * threadIdx.x,
                           S.n0 + threadIdx.x);
  } else if (threadIdx.x == 9 * LPG) {
    const T mmu = T(-F.sm_fac);
    T pk = mmu;
    for (int i = 0; i < FCH; ++i) {
      S.pwt[i] = pk;
      pk *= mmu;
    }
  }
  if (EXACT && warp == 0) {
    // powers (-mu)^e, e < FPW, by doubling: [s, 2s) = [0, s) * (-mu)^s
    T xs = T(-F.sm_fac);
    if (lane == 0) S.pwa[0] = T(1);
    __syncwarp();
    for (int s = 1; s < FPW; s <<= 1) {
      for (int t = lane; t < s && s + t < FPW; t += 32) S.pwa[s + t] = S.pwa[t] * xs;
      __syncwarp();
      xs *= xs;
    }
  }
  cp_async_wait_all_committed();
  __syncthreads();
  if (compat) {  // extrapolated ghost cells C_{-2}, C_{-1}, C_L, C_{L+1} (T2S4:275-286)
    if (threadIdx.x < LPG) compat_ghosts(S.C + threadIdx.x, H - p0, p0 - H, p1 + H, L);
    __syncthreads();
  }
  // In place, the segments of a line are read (halo) by the neighbouring CTAs
  // of its cluster: this CTA's reads are complete here, and no CTA of the
  // cluster stores before every CTA has arrived.  Out of place (ping-pong),
  // the launch has no clusters and needs no barrier.
  if (clustered) asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");

  // ---- one line per half-warp, FCH positions per lane ----
  // (exact form: Lc bounds every segment of the cluster, so all its CTAs
  // leave here together, before any cluster barrier)
  if (EXACT ? Lc > FLANES * FCH : np + 2 * J > FLANES * FCH) {
    // the host keeps segments within filter_seg_max(J) (exact: FLANES * FCH)
    if (threadIdx.x == 0) atomicOr(status, STATUS_HALO);
    return;
  }
  {
    const int c = lane & (FLANES - 1);
    const int ln = warp * 2 + (lane >> 4);
    const unsigned fm = 0xffffffffu;  // the warp is converged at every shuffle
    const int rb = H - p0;            // row of position 0
    const T mmu = -mu;
    const T pw = S.pwt[FCH - 1];      // (-mu)^FCH

    if (CELL) {
      // b of positions [p0 - J - 1, p0 - J + FLANES * FCH + 1) into this
      // line's column of the second tile: every row the forward walk reads
      // (zero past p1 + J + 1, where the walk's values are masked); lane c
      // takes a contiguous run and carries the previous edge
      const long long gl = line0 + ln;
      const int kb = p0 - J - 1;
      const int kw = p0 - J + FLANES * FCH + 1;
      const int kv = min(kw, p1 + J + 1);
      const int mm = (kw - kb + FLANES - 1) / FLANES;
      const int s0 = kb + c * mm, s1 = min(kw, s0 + mm);
      const double tau0 = F.t_min + F.ht * (double)gl;
      const T *ccol = S.C + ln;
      const T kbc = T(F.kb);
      bool swirl_done = false;
      if constexpr (sizeof(T) == 8 && !compat) {
        if (F.vel == VEL_SWIRL) {
          // Swirling field: the corner feet of the tile's LPG + 1 corner
          // lines at the edges [kb, kw] once each (a corner is shared by the
          // lines on either side), sin^2(pi s) of an edge shared by all of
          // them (the LineFeet factorisation: g(tau) h(t) per corner line and
          // time), into the second tile as [edge row][corner line]; then
          // each line's edge feet (the mean of its two corners) in place,
          // and the right-hand side below reads them back per edge.
          double *cf = S.B;
          const int ne = kw - kb + 1;
          if (threadIdx.x <= LPG) {
            const double sg = F.dir == 0 ? 1.0 : -1.0;
            const double g =
                sg * sinpi(2.0 * (F.t_min + F.ht * (double)(line0 + (long long)threadIdx.x)));
            S.om[threadIdx.x] = g * cospi((toff + F.ta_rel) / F.vp[0]);
            S.om[LPG + 1 + threadIdx.x] = g * cospi((toff + F.tb_rel) / F.vp[0]);
          }
          for (int i = threadIdx.x; i < ne; i += NTH) {
            const double ss = sinpi(F.s_min + F.h * (kb + i));
            S.et[i] = ss * ss;
          }
          __syncthreads();
          for (int i = threadIdx.x; i < ne * (LPG + 1); i += NTH) {
            const int ei = i / (LPG + 1), j = i - ei * (LPG + 1);
            const double sp = F.s_min + F.h * (kb + ei);
            const double w = S.om[LPG + 1 + j] * S.et[ei];  // speed at tb
            const double q = sinpi(sp - F.Dt * w);
            cf[(kb + ei + rb) * PITCH + j] = sp - 0.5 * F.Dt * (w + S.om[j] * q * q);
          }
          __syncthreads();
          for (int i = threadIdx.x; i < ne; i += NTH) {
            double *row = cf + (kb + i + rb) * PITCH;
            double c0 = row[0];
#pragma unroll
            for (int j = 0; j < LPG; ++j) {
              const double c1 = row[j + 1];
              row[j] = 0.5 * (c0 + c1);
              c0 = c1;
            }
          }
          __syncthreads();
          // lane c's last edge is the next lane's first: read before any write
          const double fend = s0 < s1 ? cf[(s1 + rb) * PITCH + ln] : 0.0;
          __syncwarp(fm);
          T *bcol = S.B + ln;
          if (s0 < s1) {
            CellEdge<T> el{0, T(0), T(0)};
            if (s0 < kv) el = cell_edge_at<T>(F, cf[(s0 + rb) * PITCH + ln], ccol, rb, nrows, status);
            for (int k = s0; k < s1; ++k) {
              T b = T(0);
              if (k < kv) {
                const double f1 = k + 1 < s1 ? cf[(k + 1 + rb) * PITCH + ln] : fend;
                const CellEdge<T> er = cell_edge_at<T>(F, f1, ccol, rb, nrows, status);
                b = cell_rhs<T>(el, er, ccol, rb, nrows, kbc, status);
                el = er;
              }
              bcol[(k + rb) * PITCH] = b;
            }
          }
          swirl_done = true;
        }
      }
      if (!swirl_done) {
      const LineFeet lf(F, tau0, tau0 + F.ht, toff + F.ta_rel, toff + F.tb_rel);
      if (!compat) {
        T *bcol = S.B + ln;
        if (s0 < s1) {
          CellEdge<T> el{0, T(0), T(0)};
          if (s0 < kv) el = cell_edge<T>(F, lf, ccol, rb, nrows, s0, status);
          for (int k = s0; k < s1; ++k) {
            T b = T(0);
            if (k < kv) {
              const CellEdge<T> er = cell_edge<T>(F, lf, ccol, rb, nrows, k + 1, status);
              b = cell_rhs<T>(el, er, ccol, rb, nrows, kbc, status);
              el = er;
            }
            bcol[(k + rb) * PITCH] = b;
          }
        }
      } else {
        // b = 0 outside the line (the compact mass matrix's zero ghosts).
        // Uniform displacement (the reference's rotation, constant, rotation):
        // cells clear of the clamps and ghost selections take the
        // shared-foot stencils, the rest the per-cell formulas of the
        // reference (remap_cell, foot_derivative); other velocity fields the
        // per-edge path (compat_edge)
        const int ka = max(s0, 0), kz = min(min(s1, kv), L);
        const LineView<T> vc{S.C + ln, rb, nrows, status};
        const bool uni = F.uniform != 0;
        T wr[6], wq[6];
        int n0 = 0, klo = 1, khi = 0;
        if (uni) {
          uniform_weights<T>(F, lf.foot(F, 0), wr, wq, &n0);
          klo = 2 - n0;
          khi = L - 4 - n0;
        }
        if (!F.dsrc) {
          T *bcol = S.B + ln;
          if (uni) {
            // the lane's run in three ranges: the cells clear of the clamps
            // and ghost selections [i0, i1) take the stencil with no
            // per-cell branches, the others the reference's formulas (or 0
            // outside the line)
            auto edge_cell = [&](int k) {
              T b = T(0);
              if (k >= ka && k < kz) {
                const double fa = lf.foot(F, k), fb = lf.foot(F, k + 1);
                b = remap_cell(F, vc, fa, fb) +
                    kbc * (foot_derivative(F, vc, fb) - foot_derivative(F, vc, fa));
              }
              bcol[(k + rb) * PITCH] = b;
            };
            const int i0 = max(s0, max(ka, klo)), i1 = max(i0, min(s1, min(kz, khi + 1)));
            const int ia = min(i0, s1);
            for (int k = i0; k < i1; ++k) {
              const T *cp = S.C + (k + n0 - 2 + rb) * PITCH + ln;
              T b = T(0);
#pragma unroll
              for (int t = 0; t < 6; ++t) b += (wr[t] + wq[t]) * cp[t * PITCH];
              bcol[(k + rb) * PITCH] = b;
            }
            for (int k = s0; k < s1; ++k) {  // the rest, skipping [i0, i1)
              if (k == ia) k = max(ia, i1);
              if (k >= s1) break;
              edge_cell(k);
            }
          } else {
            if (ka < kz) {
              CompatEdge<T> el = compat_edge<T>(F, lf, vc, vc, ka);
              for (int k = ka; k < kz; ++k) {
                const CompatEdge<T> er = compat_edge<T>(F, lf, vc, vc, k + 1);
                bcol[(k + rb) * PITCH] = compat_remap<T>(F, el, er, vc) + kbc * (er.d - el.d);
                el = er;
              }
            }
            for (int k = s0; k < s1; ++k)
              if (k < ka || k >= kz) bcol[(k + rb) * PITCH] = T(0);
          }
        } else {
          // the reference's third sweep differentiates the remapped field
          // (dcdx_bar_on_gpu(v_d_Cnphf_bar_x, ...), T2S4:929-932): remap the
          // cells [ra0, ra1) into the second tile, its ghosts, then
          // b = R + kbc (D_R(f_{k+1}) - D_R(f_k)) into the first tile (this
          // line's cells are no longer read)
          const int ra0 = max(0, kb - F.hd), ra1 = min(L, kv + F.hd);
          const int m1 = (ra1 - ra0 + FLANES - 1) / FLANES;
          const int q0 = ra0 + c * m1, q1 = min(ra1, q0 + m1);
          T *rcol = S.B + ln;
          if (uni) {
            auto edge_remap = [&](int k) {
              rcol[(k + rb) * PITCH] = remap_cell(F, vc, lf.foot(F, k), lf.foot(F, k + 1));
            };
            const int j0 = max(q0, klo), j1 = max(j0, min(q1, khi + 1));
            const int ja = min(j0, q1);
            for (int k = j0; k < j1; ++k) {
              const T *cp = S.C + (k + n0 - 2 + rb) * PITCH + ln;
              T r = T(0);
#pragma unroll
              for (int t = 0; t < 6; ++t) r += wr[t] * cp[t * PITCH];
              rcol[(k + rb) * PITCH] = r;
            }
            for (int k = q0; k < q1; ++k) {  // the rest, skipping [j0, j1)
              if (k == ja) k = max(ja, j1);
              if (k >= q1) break;
              edge_remap(k);
            }
          } else if (q0 < q1) {
            CompatEdge<T> el = compat_edge<T>(F, lf, vc, vc, q0);
            for (int k = q0; k < q1; ++k) {
              const CompatEdge<T> er = compat_edge<T>(F, lf, vc, vc, k + 1);
              rcol[(k + rb) * PITCH] = compat_remap<T>(F, el, er, vc);
              el = er;
            }
          }
          __syncwarp(fm);
          if (c == 0) compat_ghosts(rcol, rb, ra0 - 2, ra1 + 2, L);
          __syncwarp(fm);
          const LineView<T> vr{rcol, rb, nrows, status};
          T *bcol = S.C + ln;
          auto edge_cell = [&](int k) {
            T b = T(0);
            if (k >= ka && k < kz) {
              const double fa = lf.foot(F, k), fb = lf.foot(F, k + 1);
              b = vr(k) + kbc * (foot_derivative(F, vr, fb) - foot_derivative(F, vr, fa));
            }
            bcol[(k + rb) * PITCH] = b;
          };
          // interior cells of a uniform displacement [i0, i1): the stencil
          // (empty range for other fields: klo > khi)
          const int i0 = max(s0, max(ka, klo)), i1 = max(i0, min(s1, min(kz, khi + 1)));
          const int ia = min(i0, s1);
          for (int k = i0; k < i1; ++k) {
            const T *rp = rcol + (k + n0 - 2 + rb) * PITCH;
            T acc = T(0);
#pragma unroll
            for (int t = 0; t < 6; ++t) acc += wq[t] * rp[t * PITCH];
            bcol[(k + rb) * PITCH] = rcol[(k + rb) * PITCH] + acc;
          }
          for (int k = s0; k < s1; ++k) {  // the rest, skipping [i0, i1)
            if (k == ia) k = max(ia, i1);
            if (k >= s1) break;
            edge_cell(k);
          }
        }
      }
      }
      __syncwarp(fm);
    }

    // forward: w_k = (1/c) M b_k - mu w_{k-1} over [p0 - J, qb), qb = p1 + J.
    // Lanes past qb walk stage rows that are allocated but not staged: their
    // values only flow further right and are masked by the backward load.
    const int qb = p1 + J;
    const int k0 = p0 - J + c * FCH;
    const int r0 = CELL ? k0 - 1 + rb : k0 + S.n0[ln] - 3 + rb;  // row of the first tap
    const bool ok = r0 >= 0 && r0 + FCH + (CELL ? 2 : WIDE ? WIDE_TAPS - 1 : 7) <= S.rows;
    if (!ok) atomicOr(status, STATUS_HALO);
    T v[FCH];
    if (CELL) {
      // w_k = (1/12c)(b_{k-1} + 10 b_k + b_{k+1}) - mu w_{k-1}; compat: zero
      // input outside the line (non-cyclic system, exact zero start at 0)
      const T icw = T(F.sm_inv_den / 12.0);
      const T *bp = ((compat && F.dsrc) ? S.C : S.B) + (ok ? r0 : 0) * PITCH + ln;
      T b0 = bp[0], b1 = bp[PITCH];
      T w = T(0);
#pragma unroll
      for (int i = 0; i < FCH; ++i) {
        const T b2 = bp[(2 + i) * PITCH];
        T in = icw * ((b0 + b2) + T(10.0) * b1);
        if (compat && (unsigned)(k0 + i) >= (unsigned)L) in = T(0);
        w = in + mmu * w;
        v[i] = w;
        b0 = b1;
        b1 = b2;
      }
    } else if constexpr (WIDE) {
      // w_k = sum of WIDE_TAPS taps of the cells from row r0 - mu w_{k-1}
      const T *omp = S.om + WIDE_TAPS_PAD * ln;
      T o[WIDE_TAPS], wv[WIDE_TAPS];
#pragma unroll
      for (int m = 0; m < WIDE_TAPS; ++m) o[m] = omp[m];
      const T *cp = S.C + (ok ? r0 : 0) * PITCH + ln;
#pragma unroll
      for (int m = 0; m < WIDE_TAPS - 1; ++m) wv[m] = cp[m * PITCH];
      T w = T(0);
#pragma unroll
      for (int i = 0; i < FCH; ++i) {
        wv[WIDE_TAPS - 1] = cp[(WIDE_TAPS - 1 + i) * PITCH];
        T mb = o[0] * wv[0];
#pragma unroll
        for (int m = 1; m < WIDE_TAPS; ++m) mb += o[m] * wv[m];
        w = mb + mmu * w;
        v[i] = w;
#pragma unroll
        for (int m = 0; m < WIDE_TAPS - 1; ++m) wv[m] = wv[m + 1];
      }
    } else {
      const T *omp = S.om + 8 * ln;
      const T o0 = omp[0], o1 = omp[1], o2 = omp[2], o3 = omp[3], o4 = omp[4], o5 = omp[5],
              o6 = omp[6], o7 = omp[7];
      const T *cp = S.C + (ok ? r0 : 0) * PITCH + ln;
      T w0 = cp[0], w1 = cp[PITCH], w2 = cp[2 * PITCH], w3 = cp[3 * PITCH], w4 = cp[4 * PITCH],
        w5 = cp[5 * PITCH], w6 = cp[6 * PITCH];
      T w = T(0);
#pragma unroll
      for (int i = 0; i < FCH; ++i) {
        const T w7 = cp[(7 + i) * PITCH];
        const T mb = o0 * w0 + o1 * w1 + o2 * w2 + o3 * w3 + o4 * w4 + o5 * w5 + o6 * w6 + o7 * w7;
        w = mb + mmu * w;
        v[i] = w;
        w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6; w6 = w7;
      }
    }
    T fwd_out;  // exact form, full segment: the forward value at p1 - 1
    {
      // carries: chunk map x -> pw x + e_c, inclusive scan over the line's lanes
      T sa = pw, sb = v[FCH - 1];
#pragma unroll
      for (int d = 1; d < FLANES; d <<= 1) {
        const T pa = __shfl_up_sync(fm, sa, d, FLANES);
        const T pb = __shfl_up_sync(fm, sb, d, FLANES);
        if (c >= d) {
          sb = sa * pb + sb;
          sa = sa * pa;
        }
      }
      T cin = __shfl_up_sync(fm, sb, 1, FLANES);
      if (c == 0) cin = T(0);
      fwd_out = __shfl_sync(fm, sb, FLANES - 1, FLANES);
      // + cin (-mu)^(i+1), the powers by a running product (no table loads)
#pragma unroll
      for (int i = 0; i < FCH; ++i) {
        cin *= mmu;
        v[i] += cin;
      }
    }
    // The backward filter runs on the same positions k0 .. k0+FCH-1 of each
    // lane (w stays in registers); positions left of p0 are warm-up values
    // whose x is discarded, positions from qb on start it from zero.
    const int k1 = k0;
    // positions of this lane inside the backward range (compat: the zero
    // start is at the line's end, x_L = 0)
    const int nb = (compat ? min(qb, L) : qb) - k1;
    T e_fwd = T(0);
    if (EXACT) {
      // forward end of the segment from a zero carry (position p1 - 1)
      if (np == FLANES * FCH) {
        e_fwd = fwd_out;
      } else {
        const int cend = (np - 1) / FCH, iend = (np - 1) - cend * FCH;
#pragma unroll
        for (int i = 0; i < FCH; ++i) e_fwd = (c == cend && i == iend) ? v[i] : e_fwd;
        e_fwd = __shfl_sync(fm, e_fwd, cend, FLANES);
      }
    }
    // zero from qb on; a backward range that covers every lane's positions
    // needs none (uniform over the CTA)
    if ((compat ? min(qb, L) : qb) - (p0 - J) < FLANES * FCH) {
#pragma unroll
      for (int i = 0; i < FCH; ++i) v[i] = (i < nb) ? v[i] : T(0);
    }

    // backward: x over [k0, qb), zero start at qb
    {
      T x = T(0);
#pragma unroll
      for (int i = FCH - 1; i >= 0; --i) {
        x = v[i] + mmu * x;
        v[i] = x;
      }
      T sa = pw, sb = v[0];
#pragma unroll
      for (int d = 1; d < FLANES; d <<= 1) {
        const T pa = __shfl_down_sync(fm, sa, d, FLANES);
        const T pb = __shfl_down_sync(fm, sb, d, FLANES);
        if (c + d < FLANES) {
          sb = sa * pb + sb;
          sa = sa * pa;
        }
      }
      T cin = __shfl_down_sync(fm, sb, 1, FLANES);
      if (c == FLANES - 1) cin = T(0);
#pragma unroll
      for (int i = FCH - 1; i >= 0; --i) {
        cin *= mmu;  // cin (-mu)^(FCH - i)
        v[i] += cin;
      }
    }
    if (EXACT) {
      // Both periodic closures after one cluster barrier.  From zero carries
      // the segment gives w_zs (forward end E) and x_zs (backward start X).
      // The forward carry cr into the segment adds cr (-mu)^(k-p0+1) to w,
      // which the (linear) backward filter turns into cr h_k with
      //   h_k = (-mu)^(k-p0+1) (1 - mu^(2(p1-k))) / (1 - mu^2),
      // and the backward carry d from the right adds d (-mu)^(p1-k).  So
      // the segment's backward map is x_start = (-mu)^np x_in + X + cr h_p0.
      const T xs = __shfl_sync(fm, v[0], 0, FLANES);
      if (c == 0) {
        S.ex[ln] = e_fwd;
        S.ex[LPG + ln] = xs;
      }
      cg::this_cluster().sync();
      const T inv1m = T(1) / (T(1) - mu * mu);
      T cr, d;
      {
        // lane r (< cs) loads segment r's E_r and X_r
        T sa = T(1), sb = T(0), xr = T(0), pr = T(1);
        if (c < cs) {
          const int a0 = min(L, c * Lc), a1 = min(L, a0 + Lc);
          pr = S.pwa[a1 - a0];
          sa = pr;
          const T *rex = cg::this_cluster().map_shared_rank(S.ex, c);
          sb = rex[ln];
          xr = rex[LPG + ln];
        }
        // forward: compose w -> (-mu)^np_r w + E_r left to right, close the
        // line periodically, carry into every segment
#pragma unroll
        for (int dd = 1; dd < FLANES; dd <<= 1) {
          const T pa = __shfl_up_sync(fm, sa, dd, FLANES);
          const T pb = __shfl_up_sync(fm, sb, dd, FLANES);
          if (c >= dd) {
            sb = sa * pb + sb;
            sa = sa * pa;
          }
        }
        const T at = __shfl_sync(fm, sa, FLANES - 1, FLANES);  // lanes >= cs: identity
        const T et = __shfl_sync(fm, sb, FLANES - 1, FLANES);
        const T c0 = et / (T(1) - at);
        const T ea = __shfl_up_sync(fm, sa, 1, FLANES);
        const T eb = __shfl_up_sync(fm, sb, 1, FLANES);
        const T cr_c = c > 0 ? ea * c0 + eb : c0;  // carry into segment c
        cr = __shfl_sync(fm, cr_c, rank, FLANES);
        // backward: compose x -> (-mu)^np_r x + X_r + cr_r h_p0 right to left
        T ba = pr, bb = c < cs ? xr + cr_c * (S.pwa[1] * (T(1) - pr * pr) * inv1m) : T(0);
#pragma unroll
        for (int dd = 1; dd < FLANES; dd <<= 1) {
          const T pa = __shfl_down_sync(fm, ba, dd, FLANES);
          const T pb = __shfl_down_sync(fm, bb, dd, FLANES);
          if (c + dd < FLANES) {
            bb = ba * pb + bb;
            ba = ba * pa;
          }
        }
        const T at2 = __shfl_sync(fm, ba, 0, FLANES);
        const T xt = __shfl_sync(fm, bb, 0, FLANES);
        const bool last = rank + 1 >= cs;
        const T da = __shfl_sync(fm, ba, last ? 0 : rank + 1, FLANES);
        const T db = __shfl_sync(fm, bb, last ? 0 : rank + 1, FLANES);
        const T x0 = xt / (T(1) - at2);
        d = last ? x0 : da * x0 + db;
      }
      // this CTA's reads of the cluster's shared memory are done; it waits
      // for the others' before it exits (non-aligned forms: the wait follows
      // the divergent store loops)
      asm volatile("barrier.cluster.arrive;\n" ::: "memory");
      // x_k += cr h_k + d (-mu)^(p1-k), with cr h_k = A (-mu)^(k-p0+1) -
      // A (-mu)^(np+1) (-mu)^(p1-k), A = cr / (1 - mu^2): one power series
      // rising from the segment start, one from its end (running products;
      // positions from p1 on are not stored)
      {
        const T A = cr * inv1m;
        const T Bc = d - A * S.pwa[np + 1];
        T t1 = A * S.pwa[c * FCH + 1];  // A (-mu)^(k0-p0+1)
#pragma unroll
        for (int i = 0; i < FCH; ++i) {
          v[i] += t1;
          t1 *= mmu;
        }
        const int i0 = min(nb, FCH) - 1;  // this lane's last position before p1
        T t3 = i0 >= 0 ? Bc * S.pwa[nb - i0] : T(0);
#pragma unroll
        for (int i = FCH - 1; i >= 0; --i)
          if (i <= i0) {
            v[i] += t3;
            t3 *= mmu;
          }
      }
    }
    if (compat && p0 == 0) {
      // non-cyclic system: A = c (1 + mu S^-1)(1 + mu S) + c mu^2 e_0 e_0^T,
      // so x = y - y_0 g with g_k = mu^2 ((-mu)^k - (-mu)^(2L-k)) /
      // (1 - mu^(2L+2)) (Sherman-Morrison); y_0 is this segment's x at 0
      const int c0 = J / FCH, i0 = J - c0 * FCH;
      T y0 = T(0);
#pragma unroll
      for (int i = 0; i < FCH; ++i) y0 = (i == i0) ? v[i] : y0;
      y0 = __shfl_sync(fm, y0, c0, FLANES);
      const double q = -F.sm_fac;
      const double A = q * q / (1.0 - powi(q * q, L + 1));
      const bool tail = powi(fabs(q), L) >= 0x1p-60;  // (-mu)^(2L-k) still matters
      double qk = powi(q, max(k0, 0));
#pragma unroll
      for (int i = 0; i < FCH; ++i) {
        const int k = k0 + i;
        if (k >= 0 && k < L) {
          const double gk = A * (tail ? qk - powi(q, 2 * L - k) : qk);
          v[i] -= y0 * T(gk);
          qk *= q;
        }
      }
    }
    __syncwarp(fm);
    {
      T *xp = S.C + (k1 + rb) * PITCH + ln;
#pragma unroll
      for (int i = 0; i < FCH; ++i) xp[i * PITCH] = v[i];
    }
  }
  __syncthreads();
  if (clustered) asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory");

  // ---- cooperative store of rows H .. H+np-1 ----
  if (xsweep) {
    const int l = lane & (LPG - 1);
    const long long gl = line0 + l;
    if (gl < M) {
      const int row0 = warp * 2 + (lane >> 4);
      T *gp = gdst + (long long)(p0 + row0) * s_pos + gl;
      const T *sp = S.C + (row0 + H) * PITCH + l;
      const long long gstep = 2LL * NW * s_pos;
      for (int row = row0; row < np; row += 2 * NW) {
        *gp = *sp;
        gp += gstep;
        sp += 2 * NW * PITCH;
      }
    }
  } else {
    for (int l2 = warp; l2 < LPG; l2 += NW) {
      const long long gl2 = line0 + l2;
      if (gl2 >= M) continue;
      T *lbase = gdst + gl2 * s_line + p0;
      const T *scol = S.C + H * PITCH + l2;
      for (int row = lane; row < np; row += 32) lbase[row] = scol[row * PITCH];
    }
  }
  if (EXACT) asm volatile("barrier.cluster.wait;\n" ::: "memory");
}

}  // namespace

size_t sweep_smem_bytes(int lc_max, int halo, bool fp64, bool source) {
  size_t el = fp64 ? 8 : 4;
  size_t n = (source ? 3 : 2) * (size_t)(lc_max + 2 * halo) * PITCH +
             3 * (size_t)lc_max + 3 * (size_t)NCH * LPG + 8 * (size_t)LPG;
  return FD_BYTES + n * el;
}

size_t sweep_filter_smem_bytes(int lc_max, int halo, bool fp64, bool exact, bool cell,
                               bool wide) {
  size_t el = fp64 ? 8 : 4;
  return FD_BYTES + 64 * sizeof(int) +
         ((wide ? WIDE_TAPS_PAD : 8) * (size_t)LPG + 32 + (exact ? (size_t)FPW + 2 * LPG : 0) +
          (cell ? 2 : 1) * (size_t)filter_tile_rows(lc_max, halo) * PITCH) * el +
         (cell ? 8 * (size_t)FPW + 8 : 0);
}

int filter_segment_max(int J) { return filter_seg_max(J); }

cudaError_t launch_filter_weights(bool fp64, const SweepField *d_field, void *wt, int *nt,
                                  int lines, cudaStream_t stream, bool wide) {
  const int bt = 128, grid = (lines + bt - 1) / bt;
  count_launch();
  if (fp64)
    filter_weights_kernel<double><<<grid, bt, 0, stream>>>(d_field, static_cast<double *>(wt), nt,
                                                           lines, wide ? 1 : 0);
  else
    filter_weights_kernel<float><<<grid, bt, 0, stream>>>(d_field, static_cast<float *>(wt), nt,
                                                          lines, wide ? 1 : 0);
  return cudaGetLastError();
}

size_t sweep_fast_smem_bytes(int lc_max, int halo, bool fp64) {
  size_t el = fp64 ? 8 : 4;
  size_t n = (size_t)(lc_max + 2 * halo) * PITCH + (size_t)lc_max * PITCH + 5 * (size_t)lc_max +
             2 * (size_t)NCH + 1 + 2 * (size_t)NCH * LPG + 16 * (size_t)LPG;
  return FD_BYTES + 64 * sizeof(int) + n * el;
}

template <typename T>
using FilterKernelT = void (*)(const SweepField *, int, int, double, void *, int, int, unsigned *,
                               int, int, const int *, int, int, const int *);

// The filter kernel's instantiation of a variant.
template <typename T>
static FilterKernelT<T> filter_kernel_for(int variant) {
  switch (variant) {
    case SWEEP_FILTER_EXACT: return sweep_filter_kernel<T, true, false, false>;
    case SWEEP_CELL: return sweep_filter_kernel<T, false, true, false>;
    case SWEEP_CELL_EXACT: return sweep_filter_kernel<T, true, true, false>;
    case SWEEP_CELL_COMPAT: return sweep_filter_kernel<T, false, true, true>;
    case SWEEP_FILTER_WIDE: return sweep_filter_kernel<T, false, false, false, true>;
    default: return sweep_filter_kernel<T, false, false, false>;
  }
}

template <typename T>
static cudaError_t launch_impl(int variant, const SweepField *d_fields, int nfields,
                               int group_base, int groups_total, int cs, int lc_max, int halo,
                               double toff, void *data, unsigned *d_status, int jstep,
                               int nslice, const int *nlo, bool inplace, cudaStream_t stream,
                               const int *g0idx, bool pdl_ok) {
  const bool fast = (variant == SWEEP_FAST);
  const bool cell = cell_filter_variant(variant);
  const bool exact = exact_filter_variant(variant);
  const bool filt = filter_variant(variant);
  const bool src = (variant == SWEEP_GENERAL_SRC);
  const size_t smem = filt ? sweep_filter_smem_bytes(lc_max, halo, sizeof(T) == 8, exact, cell,
                                                     variant == SWEEP_FILTER_WIDE)
                      : fast ? sweep_fast_smem_bytes(lc_max, halo, sizeof(T) == 8)
                             : sweep_smem_bytes(lc_max, halo, sizeof(T) == 8, src);
  {
    // Function attributes apply to the device that is current when they are
    // set: configure each device once (contexts, batches, servers and the
    // allocation-free step may run on different devices of one process, from
    // several host threads).
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
    static std::atomic<bool> configured[MAX_DEVICES];
    static std::mutex config_mu;
    if (!configured[dev].load(std::memory_order_acquire)) {
      std::lock_guard<std::mutex> lk(config_mu);
      if (!configured[dev].load(std::memory_order_relaxed)) {
        for (const void *fn :
             {(const void *)sweep_kernel<T>, (const void *)sweep_fast_kernel<T>,
              (const void *)filter_kernel_for<T>(SWEEP_FILTER),
              (const void *)filter_kernel_for<T>(SWEEP_FILTER_EXACT),
              (const void *)filter_kernel_for<T>(SWEEP_CELL),
              (const void *)filter_kernel_for<T>(SWEEP_CELL_EXACT),
              (const void *)filter_kernel_for<T>(SWEEP_CELL_COMPAT),
              (const void *)filter_kernel_for<T>(SWEEP_FILTER_WIDE)}) {
          err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     227 * 1024);
          if (err != cudaSuccess) return err;
          err = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
          if (err != cudaSuccess) return err;
        }
        configured[dev].store(true, std::memory_order_release);
      }
    }
  }
  if (groups_total <= 0) return cudaSuccess;
  if (exact && inplace) return cudaErrorInvalidValue;  // the exact form sweeps out of place
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(groups_total * cs), 1, 1);
  cfg.blockDim = dim3(NTH, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  count_launch();
  if (filt) {
    // whole lines per CTA, or out of place: no cluster (exact form: one
    // cluster per tile, the cs segments of its lines)
    int clustered = 0;
    cudaLaunchAttribute fattr[2];
    unsigned na = 0;
    if (exact || !(cs == 1 || !inplace)) {
      fattr[na++] = attr[0];
      clustered = exact ? 0 : 1;
    }
    // programmatic dependent launch (the kernel waits for its predecessor
    // before reading anything) for the single-instance engine's launches:
    // 1.4 % on the 2048^2 Parareal solve, while the batched engine's
    // back-to-back class launches lost 14 % of their fine phase with it.
    // CCFV_PDL=0 turns it off.
    static const bool pdl = [] {
      const char *e = std::getenv("CCFV_PDL");
      return !(e && e[0] == '0');
    }();
    if (pdl && pdl_ok) {
      fattr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      fattr[na].val.programmaticStreamSerializationAllowed = 1;
      ++na;
    }
    cfg.attrs = fattr;
    cfg.numAttrs = na;
    FilterKernelT<T> fn = filter_kernel_for<T>(variant);
    return cudaLaunchKernelEx(&cfg, fn, d_fields, nfields, group_base * cs, toff, data, lc_max,
                              halo, d_status, jstep, nslice, nlo, cs, clustered, g0idx);
  }
  if (fast)
    return cudaLaunchKernelEx(&cfg, sweep_fast_kernel<T>, d_fields, nfields, group_base, toff,
                              data, lc_max, halo, d_status, jstep, nslice, nlo, g0idx);
  return cudaLaunchKernelEx(&cfg, sweep_kernel<T>, d_fields, nfields, group_base, toff, data,
                            lc_max, halo, d_status, jstep, nslice, nlo, g0idx);
}

template <typename T>
cudaError_t launch_sweep(int variant, const SweepField *d_fields, int nfields, int group_base,
                         int groups_total, int cs, int lc_max, int halo, double toff, void *data,
                         unsigned *d_status, cudaStream_t stream, int jstep, bool inplace) {
  return launch_impl<T>(variant, d_fields, nfields, group_base, groups_total, cs, lc_max, halo,
                        toff, data, d_status, jstep, 0, nullptr, inplace, stream, nullptr, true);
}

template <typename T>
cudaError_t launch_sweep_batch(int variant, const SweepField *d_fields, int nfields,
                               int group_base, int groups_total, int cs, int lc_max, int halo,
                               const BatchStep &bs, unsigned *d_status, cudaStream_t stream) {
  return launch_impl<T>(variant, d_fields, nfields, group_base, groups_total, cs, lc_max, halo,
                        0.0, nullptr, d_status, bs.jstep, bs.nslice, bs.nlo, bs.inplace, stream,
                        bs.g0idx, false);
}

template cudaError_t launch_sweep<double>(int, const SweepField *, int, int, int, int, int, int,
                                          double, void *, unsigned *, cudaStream_t, int, bool);
template cudaError_t launch_sweep<float>(int, const SweepField *, int, int, int, int, int, int,
                                         double, void *, unsigned *, cudaStream_t, int, bool);
template cudaError_t launch_sweep_batch<double>(int, const SweepField *, int, int, int, int, int,
                                                int, const BatchStep &, unsigned *, cudaStream_t);
template cudaError_t launch_sweep_batch<float>(int, const SweepField *, int, int, int, int, int,
                                               int, const BatchStep &, unsigned *, cudaStream_t);

}  // namespace ccfv
