// coarse.cu -- the resident coarse propagator of the batched engine.
//
// The G phase of a Parareal iteration is sequential over the slices
// (CoarsePropagator T2S4:971-974, run slice after slice at T2S4:1306-1317,
// then parareal_correction_kernel T2S4:771-782).  For an instance whose
// coarse field fits in one SM's shared memory, one CTA runs that whole phase:
// for every slice s from the first active one, m coarse steps (x, y, x
// sweeps) on the increment field held in shared memory, then the delta-form
// correction U+[s+1] = F[s+1] + G(e_s) fused with the slice's update norms,
// whose new increment e_{s+1} = U+[s+1] - U[s+1] stays in shared memory for
// the next slice.  The field never goes to HBM between coarse sweeps; only
// F[s+1] and U[s+1] are read and U[s+1] written once per slice.  One launch
// per iteration serves every resident instance (one CTA each), on a stream
// beside the shared launches of the other instances.
//
// Each sweep solves a whole periodic line in one half-warp (at most 272
// cells): lane c holds positions 17c .. 17c+16; the factored filters
// w_k = r_k/c - mu w_{k-1}, x_k = w_k - mu x_{k+1} run from zero carries
// with shuffle-scan chunk joins, and the periodic closure is exact
// (w_{L-1} = E / (1 - (-mu)^L), x_0 = X / (1 - (-mu)^L)), so no recurrence
// is warmed up at any diffusion number.  The right-hand side is the
// shared-foot 8-tap stencil for uniform-displacement velocity fields and the
// per-edge remap / foot derivative for the others, with periodic indices.
#include <climits>

#include "ccfv_internal.h"
#include "sweep_math.cuh"

namespace ccfv {

namespace {

constexpr int RG_LANES = 16;           // lanes per line
constexpr int RG_CH = 17;              // positions per lane
constexpr int RG_LINE = RG_LANES * RG_CH;  // longest line (272)
constexpr int RG_POW = RG_LINE + 8;    // powers (-mu)^0 .. (-mu)^(RG_POW-1)

__device__ __forceinline__ int wrapi(int q, int L) {
  q %= L;
  return q < 0 ? q + L : q;
}

// One edge of a periodic line for the per-cell right-hand side: foot cell,
// PPM antiderivative at the foot (T2S4:63-65, 260-304) and the fourth-order
// derivative at the foot (T2S4:440-547).
template <typename T>
struct RgEdge {
  int kf;
  T phi, d;
};

template <typename T>
__device__ __forceinline__ RgEdge<T> rg_edge(const SweepField &F, const T *line, int sp, int L,
                                             double f) {
  const double u = (f - F.s_min) / F.h;
  const double fk = floor(u);
  RgEdge<T> r;
  r.kf = (int)fk;
  const T xi = T(u - fk);
  const int q = wrapi(r.kf - 2, L);
  T c[5];
#pragma unroll
  for (int t = 0, p = q; t < 5; ++t, p = (p + 1 == L) ? 0 : p + 1) c[t] = line[p * sp];
  const T cl = T(7.0 / 12.0) * (c[2] + c[1]) - T(1.0 / 12.0) * (c[3] + c[0]);
  const T cr = T(7.0 / 12.0) * (c[3] + c[2]) - T(1.0 / 12.0) * (c[4] + c[1]);
  const T D = cr - cl;
  const T C6 = T(6.0) * (c[2] - T(0.5) * (cl + cr));
  const T xi2 = xi * xi, xi3 = xi2 * xi;
  r.phi = T(-1.0 / 3) * C6 * xi3 + T(0.5) * (D + C6) * xi2 + cl * xi;
  r.d = T(F.inv12h) * ((T(2.0) * xi3 - T(6.0) * xi2 + T(3.0) * xi + T(1.0)) * c[0] +
                       (T(-8.0) * xi3 + T(18.0) * xi2 + T(6.0) * xi - T(15.0)) * c[1] +
                       (T(12.0) * xi3 - T(18.0) * xi2 - T(24.0) * xi + T(15.0)) * c[2] +
                       (T(-8.0) * xi3 + T(6.0) * xi2 + T(18.0) * xi - T(1.0)) * c[3] +
                       (T(2.0) * xi3 - T(3.0) * xi) * c[4]);
  return r;
}

// remap + (1-theta) K Dt/h (D_r - D_l) of the cell between two edges, whole
// cells between the feet summed with Neumaier compensation.
template <typename T>
__device__ __forceinline__ T rg_rhs(const RgEdge<T> &l, const RgEdge<T> &r, const T *line, int sp,
                                    int L, T kbc) {
  T remap;
  if (r.kf == l.kf) {
    remap = r.phi - l.phi;
  } else {
    const int lo = min(l.kf, r.kf), hi = max(l.kf, r.kf) - 1;
    T s = T(0), comp = T(0);
    for (int k = lo, p = wrapi(lo, L); k <= hi; ++k, p = (p + 1 == L) ? 0 : p + 1) {
      const T x = line[p * sp];
      const T t = s + x;
      comp += (fabs(s) >= fabs(x)) ? ((s - t) + x) : ((x - t) + s);
      s = t;
    }
    s += comp;
    remap = r.kf > l.kf ? (s + r.phi) - l.phi : -((s + l.phi) - r.phi);
  }
  return remap + kbc * (r.d - l.d);
}

// One sweep of the resident field E ([nx][P], P odd) for every line.
template <typename T>
__device__ void rg_sweep(const SweepField &F, T *E, int P, const T *pwa, T *bscr, double toff) {
  const int L = F.L, M = F.M;
  const int sp = F.dir == 0 ? P : 1, sl = F.dir == 0 ? 1 : P;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = lane & (RG_LANES - 1);
  const int hw = warp * 2 + (lane >> 4);
  const unsigned fm = 0xffffffffu;
  const T mu = T(F.sm_fac), mmu = -mu;
  const T pw = pwa[RG_CH];  // (-mu)^17
  const bool cell = !F.uniform;
  const int nh = (blockDim.x / 32) * 2;  // half-warps (lines per round)
  for (int r = 0; r * nh < M; ++r) {
    const int gl = r * nh + hw;
    const bool act = gl < M;
    const int g = act ? gl : M - 1;
    T *line = E + (size_t)g * sl;
    const int k0 = c * RG_CH;
    T v[RG_CH];
    const double tau0 = F.t_min + F.ht * (double)g;
    if (!cell) {
      T om[8];
      int n0 = 0;
      filter_line_stencil<T>(F, g, toff, om, &n0);
      int q = wrapi(k0 + n0 - 3, L);
      T win[8];
#pragma unroll
      for (int m = 0; m < 7; ++m) {
        win[m] = line[q * sp];
        q = (q + 1 == L) ? 0 : q + 1;
      }
      T w = T(0);
#pragma unroll
      for (int i = 0; i < RG_CH; ++i) {
        win[7] = line[q * sp];
        q = (q + 1 == L) ? 0 : q + 1;
        T in = T(0);
#pragma unroll
        for (int m = 0; m < 8; ++m) in += om[m] * win[m];
        if (k0 + i >= L) in = T(0);
        w = in + mmu * w;
        v[i] = w;
#pragma unroll
        for (int m = 0; m < 7; ++m) win[m] = win[m + 1];
      }
    } else {
      // b of this line's cells into the half-warp's scratch row (contiguous
      // runs per lane, carrying the previous edge), then the mass-matrix
      // stencil (1/12c)(b_{k-1} + 10 b_k + b_{k+1}) as w's input
      T *bl = bscr + hw * RG_LINE;
      const int mm = (L + RG_LANES - 1) / RG_LANES;
      const int s0 = c * mm, s1 = min(L, s0 + mm);
      const T kbc = T(F.kb);
      const LineFeet lf(F, tau0, tau0 + F.ht, toff + F.ta_rel, toff + F.tb_rel);
      if (s0 < s1) {
        RgEdge<T> el = rg_edge<T>(F, line, sp, L, lf.foot(F, s0));
        for (int k = s0; k < s1; ++k) {
          const RgEdge<T> er = rg_edge<T>(F, line, sp, L, lf.foot(F, k + 1));
          bl[k] = rg_rhs<T>(el, er, line, sp, L, kbc);
          el = er;
        }
      }
      __syncwarp(fm);
      const T icw = T(F.sm_inv_den / 12.0);
      T w = T(0);
#pragma unroll
      for (int i = 0; i < RG_CH; ++i) {
        const int k = k0 + i;
        T in = T(0);
        if (k < L) in = icw * ((bl[k == 0 ? L - 1 : k - 1] + bl[k + 1 == L ? 0 : k + 1]) +
                               T(10.0) * bl[k]);
        w = in + mmu * w;
        v[i] = w;
      }
    }
    // forward chunks joined by a shuffle scan of x -> pw x + e_c
    {
      T sa = pw, sb = v[RG_CH - 1];
#pragma unroll
      for (int d = 1; d < RG_LANES; d <<= 1) {
        const T pa = __shfl_up_sync(fm, sa, d, RG_LANES);
        const T pb = __shfl_up_sync(fm, sb, d, RG_LANES);
        if (c >= d) {
          sb = sa * pb + sb;
          sa = sa * pa;
        }
      }
      T cin = __shfl_up_sync(fm, sb, 1, RG_LANES);
      if (c == 0) cin = T(0);
#pragma unroll
      for (int i = 0; i < RG_CH; ++i) {
        cin *= mmu;
        v[i] += cin;
      }
    }
    // periodic closure of the forward filter: w_{-1} = w_{L-1} = E / (1 - (-mu)^L)
    {
      const int ce = (L - 1) / RG_CH, ie = (L - 1) - ce * RG_CH;
      T e = T(0);
#pragma unroll
      for (int i = 0; i < RG_CH; ++i) e = (c == ce && i == ie) ? v[i] : e;
      e = __shfl_sync(fm, e, ce, RG_LANES);
      const T wl = e / (T(1) - pwa[L]);
#pragma unroll
      for (int i = 0; i < RG_CH; ++i) {
        const int k = k0 + i;
        v[i] = k < L ? v[i] + wl * pwa[k + 1] : T(0);
      }
    }
    // backward filter from a zero start at L
    {
      T x = T(0);
#pragma unroll
      for (int i = RG_CH - 1; i >= 0; --i) {
        x = v[i] + mmu * x;
        v[i] = x;
      }
      T sa = pw, sb = v[0];
#pragma unroll
      for (int d = 1; d < RG_LANES; d <<= 1) {
        const T pa = __shfl_down_sync(fm, sa, d, RG_LANES);
        const T pb = __shfl_down_sync(fm, sb, d, RG_LANES);
        if (c + d < RG_LANES) {
          sb = sa * pb + sb;
          sa = sa * pa;
        }
      }
      T cin = __shfl_down_sync(fm, sb, 1, RG_LANES);
      if (c == RG_LANES - 1) cin = T(0);
#pragma unroll
      for (int i = RG_CH - 1; i >= 0; --i) {
        cin *= mmu;
        v[i] += cin;
      }
    }
    // periodic closure of the backward filter: x_L = x_0 = X / (1 - (-mu)^L)
    {
      const T X = __shfl_sync(fm, v[0], 0, RG_LANES);
      const T x0 = X / (T(1) - pwa[L]);
      __syncwarp(fm);  // every read of this line is done
      if (act) {
#pragma unroll
        for (int i = 0; i < RG_CH; ++i) {
          const int k = k0 + i;
          if (k < L) line[k * sp] = v[i] + x0 * pwa[L - k];
        }
      }
      __syncwarp(fm);
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256)
    resident_g_kernel(const ResidentG *__restrict__ rg, const int *__restrict__ nlo) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ SweepField fd[3];
  __shared__ double red[2][8];
  const ResidentG &R = rg[blockIdx.x];
  constexpr int NW8 = (int)(sizeof(SweepField) / 8);
  for (int i = threadIdx.x; i < 3 * NW8; i += blockDim.x)
    reinterpret_cast<long long *>(fd)[i] = reinterpret_cast<const long long *>(R.f)[i];
  const int lo = nlo[R.inst];
  const int S = R.S, m = R.m, nx = R.nx, ny = R.ny, P = R.pitch;
  const long long NN = (long long)nx * ny;
  if (lo < 0 || lo >= S) return;  // uniform over the CTA
  T *E = reinterpret_cast<T *>(smem_raw);
  T *pwx = E + (size_t)nx * P;
  T *pwy = pwx + RG_POW;
  T *bscr = pwy + RG_POW;
  __syncthreads();
  {
    const double mx = -fd[0].sm_fac, my = -fd[1].sm_fac;
    for (int e = threadIdx.x; e < RG_POW; e += blockDim.x) {
      double px = 1.0, py = 1.0, bx = mx, by = my;  // binary powering
      for (int n = e; n > 0; n >>= 1) {
        if (n & 1) {
          px *= bx;
          py *= by;
        }
        bx *= bx;
        by *= by;
      }
      pwx[e] = T(px);
      pwy[e] = T(py);
    }
    for (long long i = threadIdx.x; i < (long long)nx * P; i += blockDim.x) E[i] = T(0);
  }
  __syncthreads();
  for (int s = lo; s < S; ++s) {
    if (s > lo) {  // G(e_s): m coarse steps of the increment (G(0) = 0 at s = lo)
      for (int j = 0; j < m; ++j)
        for (int kind = 0; kind < 3; ++kind) {
          const SweepField &F = fd[kind];
          rg_sweep<T>(F, E, P, F.dir == 0 ? pwx : pwy, bscr, j * F.t_step + s * F.t_slice);
          __syncthreads();
        }
    }
    // U+[s+1] = F[s+1] + G(e_s); e_{s+1} = U+[s+1] - U[s+1]; update norms
    const double *Fs = R.F + (long long)(s + 1) * NN;
    double *Us = R.U + (long long)(s + 1) * NN;
    double se = 0.0, su = 0.0;
    for (long long idx = threadIdx.x; idx < NN; idx += blockDim.x) {
      const int i = (int)(idx / ny), jj = (int)(idx - (long long)i * ny);
      T &e = E[(size_t)i * P + jj];
      const double un = Fs[idx] + (s > lo ? (double)e : 0.0);
      const double d = un - Us[idx];
      Us[idx] = un;
      e = T(d);
      se += d * d;
      su += un * un;
    }
    for (int o = 16; o > 0; o >>= 1) {
      se += __shfl_down_sync(0xffffffffu, se, o);
      su += __shfl_down_sync(0xffffffffu, su, o);
    }
    if ((threadIdx.x & 31) == 0) {
      red[0][threadIdx.x >> 5] = se;
      red[1][threadIdx.x >> 5] = su;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0, b = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        a += red[0][w];
        b += red[1][w];
      }
      R.norms[2 * (s + 1)] = a;
      R.norms[2 * (s + 1) + 1] = b;
    }
    __syncthreads();
  }
}

}  // namespace

size_t resident_g_smem_bytes(int nx, int ny, bool fp64, bool cell) {
  const size_t el = fp64 ? 8 : 4;
  const int P = ny | 1;
  return el * ((size_t)nx * P + 2 * (size_t)RG_POW + (cell ? 16 * (size_t)RG_LINE : 0)) + 16;
}

bool resident_g_fits(int nx, int ny, bool fp64, bool cell) {
  return nx <= RG_LINE && ny <= RG_LINE && nx >= 4 && ny >= 4 &&
         resident_g_smem_bytes(nx, ny, fp64, cell) <= 200 * 1024;
}

cudaError_t launch_resident_g(bool fp64, const ResidentG *d_rg, int n, size_t smem,
                              const int *nlo, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const void *fn = fp64 ? (const void *)resident_g_kernel<double>
                        : (const void *)resident_g_kernel<float>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  count_launch();
  if (fp64)
    resident_g_kernel<double><<<n, 256, smem, st>>>(d_rg, nlo);
  else
    resident_g_kernel<float><<<n, 256, smem, st>>>(d_rg, nlo);
  return cudaGetLastError();
}

}  // namespace ccfv
