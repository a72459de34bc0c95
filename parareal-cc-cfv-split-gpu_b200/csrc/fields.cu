// fields.cu -- device kernels around the solve: the reference's initial
// condition / exact solution, Gaussian-sum initial fields and error norms.
#include <cmath>

#include "engine.h"

namespace ccfv {
namespace {

// C_Exact (T2S4_Parareal.cu:51-56): the rotated, diffused Gaussian of the
// reference (x0 = -0.35, y0 = 0, sigma = 0.005, rotation rate 4).
__device__ __forceinline__ double c_exact_ref(double x, double y, double t, double K) {
  const double gx0 = -0.35, gy0 = 0.0, sg = 0.005;
  const double xs = x * cos(4 * t) + y * sin(4 * t);
  const double ys = -x * sin(4 * t) + y * cos(4 * t);
  const double d = sg + 4 * K * t;
  return sg / d * exp(-((xs - gx0) * (xs - gx0) + (ys - gy0) * (ys - gy0)) / d);
}

// 3x3 Simpson cell average of C_Exact (get_exact_solution_on_gpu,
// T2S4_Parareal.cu:118-140), one thread per cell.
__global__ void exact_ref_kernel(double *C, int nx, int ny, double x_min, double y_min, double dx,
                                 double dy, double t, double K) {
  const long long n = (long long)nx * ny;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < n;
       id += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(id / ny), j = (int)(id - (long long)i * ny);
    const double xi = x_min + (i + 0.5) * dx, yj = y_min + (j + 0.5) * dy;
    const double xm = xi - 0.5 * dx, xp = xi + 0.5 * dx, ym = yj - 0.5 * dy, yp = yj + 0.5 * dy;
    C[id] = 1.0 / 36.0 *
            (c_exact_ref(xm, ym, t, K) + c_exact_ref(xp, ym, t, K) + c_exact_ref(xm, yp, t, K) +
             c_exact_ref(xp, yp, t, K) +
             4.0 * (c_exact_ref(xm, yj, t, K) + c_exact_ref(xp, yj, t, K) +
                    c_exact_ref(xi, ym, t, K) + c_exact_ref(xi, yp, t, K)) +
             16.0 * c_exact_ref(xi, yj, t, K));
  }
}

// 3x3 Simpson cell averages of sum_q amp_q exp(-r_q^2 / den_q) with the
// periodic images of a (Lx, Ly) box over [-img, img]^2.
__global__ void gaussians_kernel(double *C, int nx, int ny, double x_min, double y_min, double dx,
                                 double dy, int ng, const double *__restrict__ par, int img) {
  const long long n = (long long)nx * ny;
  const double Lx = dx * nx, Ly = dy * ny;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < n;
       id += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(id / ny), j = (int)(id - (long long)i * ny);
    const double xi = x_min + (i + 0.5) * dx, yj = y_min + (j + 0.5) * dy;
    double acc = 0.0;
    for (int a = -1; a <= 1; ++a)
      for (int b = -1; b <= 1; ++b) {
        const double w = (a == 0 ? 4.0 : 1.0) * (b == 0 ? 4.0 : 1.0);
        const double x = xi + 0.5 * dx * a, y = yj + 0.5 * dy * b;
        double v = 0.0;
        for (int q = 0; q < ng; ++q) {
          const double cx = par[4 * q], cy = par[4 * q + 1], den = par[4 * q + 2], amp = par[4 * q + 3];
          for (int ix = -img; ix <= img; ++ix)
            for (int iy = -img; iy <= img; ++iy) {
              const double ex = x - cx + ix * Lx, ey = y - cy + iy * Ly;
              v += amp * exp(-(ex * ex + ey * ey) / den);
            }
        }
        acc += w * v;
      }
    C[id] = acc / 36.0;
  }
}

constexpr int NT = 256;
constexpr int NB = 592;

// Sum of squares of a-b, sum of squares of b, max |a-b| (fixed-order block
// partials, last block finishes: deterministic).
__global__ void __launch_bounds__(NT) norms_kernel(const double *__restrict__ a,
                                                   const double *__restrict__ b, long long n,
                                                   double *__restrict__ partial,
                                                   unsigned *__restrict__ counter,
                                                   double *__restrict__ out) {
  double se = 0.0, sb = 0.0, mx = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double d = a[i] - b[i];
    se += d * d;
    sb += b[i] * b[i];
    mx = fmax(mx, fabs(d));
  }
  for (int o = 16; o > 0; o >>= 1) {
    se += __shfl_down_sync(0xffffffffu, se, o);
    sb += __shfl_down_sync(0xffffffffu, sb, o);
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  __shared__ double red[3][NT / 32];
  __shared__ bool last;
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { red[0][w] = se; red[1][w] = sb; red[2][w] = mx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0, y = 0, z = 0;
    for (int k = 0; k < NT / 32; ++k) { x += red[0][k]; y += red[1][k]; z = fmax(z, red[2][k]); }
    partial[3 * blockIdx.x] = x;
    partial[3 * blockIdx.x + 1] = y;
    partial[3 * blockIdx.x + 2] = z;
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double x = 0, y = 0, z = 0;
    for (unsigned k = 0; k < gridDim.x; ++k) {
      x += ((volatile double *)partial)[3 * k];
      y += ((volatile double *)partial)[3 * k + 1];
      z = fmax(z, ((volatile double *)partial)[3 * k + 2]);
    }
    out[0] = x;
    out[1] = y;
    out[2] = z;
    *counter = 0;
  }
}

int blocks_for(long long n) {
  long long b = (n + NT - 1) / NT;
  return (int)(b < 1 ? 1 : (b > NB ? NB : b));
}

}  // namespace

int exact_ref(ccfv_ctx *ctx, double *d_C, double t, cudaStream_t st) {
  const ccfv_grid &g = ctx->grid;
  const double dx = (g.x_max - g.x_min) / g.nx, dy = (g.y_max - g.y_min) / g.ny;
  const long long n = (long long)g.nx * g.ny;
  count_launch();
  exact_ref_kernel<<<blocks_for(n), NT, 0, st>>>(d_C, g.nx, g.ny, g.x_min, g.y_min, dx, dy, t, g.K);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CCFV_OK : set_error(ctx, CCFV_ERR_CUDA, cudaGetErrorString(e));
}

int gaussians(ccfv_ctx *ctx, double *d_C, int ng, const double *params, int img, cudaStream_t st) {
  const ccfv_grid &g = ctx->grid;
  const double dx = (g.x_max - g.x_min) / g.nx, dy = (g.y_max - g.y_min) / g.ny;
  const long long n = (long long)g.nx * g.ny;
  if (ctx->io.alloc(sizeof(double) * 4 * (size_t)ng) != cudaSuccess)
    return set_error(ctx, CCFV_ERR_NOMEM, "gaussian parameters");
  cudaError_t e = cudaMemcpyAsync(ctx->io.p, params, sizeof(double) * 4 * ng,
                                  cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return set_error(ctx, CCFV_ERR_CUDA, cudaGetErrorString(e));
  count_launch();
  gaussians_kernel<<<blocks_for(n), NT, 0, st>>>(d_C, g.nx, g.ny, g.x_min, g.y_min, dx, dy, ng,
                                                 ctx->io.as<double>(), img);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // parameters buffer is reused
  return e == cudaSuccess ? CCFV_OK : set_error(ctx, CCFV_ERR_CUDA, cudaGetErrorString(e));
}

int norms(ccfv_ctx *ctx, const double *a, const double *b, double *rel_l2, double *max_abs,
          cudaStream_t st) {
  const ccfv_grid &g = ctx->grid;
  const long long n = (long long)g.nx * g.ny;
  double *out = ctx->aux.as<double>();
  count_launch();
  norms_kernel<<<blocks_for(n), NT, 0, st>>>(a, b, n, ctx->partial.as<double>(),
                                             ctx->counter.as<unsigned>(), out);
  double h[3] = {0, 0, 0};
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_error(ctx, CCFV_ERR_CUDA, cudaGetErrorString(e));
  if (rel_l2) *rel_l2 = h[1] > 0 ? std::sqrt(h[0] / h[1]) : std::sqrt(h[0]);
  if (max_abs) *max_abs = h[2];
  return CCFV_OK;
}

}  // namespace ccfv
