// api.cu -- the extern "C" boundary of libccfv (declared in include/ccfv.h).
#include <cstring>
#include <new>

#include "engine.h"

using namespace ccfv;

namespace {

bool grid_ok(const ccfv_grid *g) {
  if (!g) return false;
  if (g->nx < 4 || g->ny < 4) return false;
  if (!(g->x_max > g->x_min) || !(g->y_max > g->y_min)) return false;
  if (g->bc != CCFV_BC_COMPAT && g->bc != CCFV_BC_PERIODIC) return false;
  if (g->velocity < CCFV_VEL_REF_ROT4 || g->velocity > CCFV_VEL_SWIRL) return false;
  if (g->velocity == CCFV_VEL_SWIRL && g->vel_params[0] == 0.0) return false;
  if (g->scheme != CCFV_SCHEME_REFERENCE && g->scheme != CCFV_SCHEME_CONSISTENT) return false;
  if (!(g->K >= 0.0)) return false;
  if (g->source != CCFV_SRC_NONE && g->source != CCFV_SRC_GAUSSIAN) return false;
  if (g->source == CCFV_SRC_GAUSSIAN && !(g->source_params[3] > 0.0)) return false;
  return true;
}

int use_device(ccfv_ctx *ctx) {
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return set_error(ctx, CCFV_ERR_CUDA, cudaGetErrorString(e));
  return CCFV_OK;
}

int last_launch(ccfv_ctx *ctx) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(ctx, CCFV_ERR_CUDA, cudaGetErrorString(e));
  return CCFV_OK;
}

}  // namespace

extern "C" {

const char *ccfv_strerror(int status) {
  switch (status) {
    case CCFV_OK: return "ok";
    case CCFV_ERR_INVALID: return "invalid argument";
    case CCFV_ERR_CUDA: return "CUDA error";
    case CCFV_ERR_NOMEM: return "out of device memory";
    case CCFV_ERR_UNSUPPORTED: return "unsupported configuration";
    case CCFV_ERR_HALO: return "characteristic foot outside the staged halo";
    case CCFV_ERR_BUDGET: return "request exceeds the HBM budget";
    case CCFV_ERR_NOT_FOUND: return "unknown ticket";
    case CCFV_ERR_CANCELLED: return "cancelled";
    case CCFV_ERR_TIMEOUT: return "timed out";
  }
  return "unknown status";
}

int ccfv_create(ccfv_ctx **out, const ccfv_grid *grid, int device) {
  if (!out) return CCFV_ERR_INVALID;
  *out = nullptr;
  if (!grid_ok(grid)) return CCFV_ERR_INVALID;
  ccfv_ctx *ctx = new (std::nothrow) ccfv_ctx();
  if (!ctx) return CCFV_ERR_NOMEM;
  ctx->grid = *grid;
  ctx->device = device;
  int rc = use_device(ctx);
  if (rc) { delete ctx; return rc; }
  if (ctx->status.alloc(sizeof(unsigned) * 4) != cudaSuccess ||
      ctx->partial.alloc(sizeof(double) * 3 * RED_BLOCKS_MAX) != cudaSuccess ||
      ctx->counter.alloc(sizeof(unsigned) * 4) != cudaSuccess ||
      ctx->aux.alloc(sizeof(double) * 64) != cudaSuccess) {
    delete ctx;
    return CCFV_ERR_NOMEM;
  }
  if (cudaMemset(ctx->status.p, 0, sizeof(unsigned) * 4) != cudaSuccess ||
      cudaMemset(ctx->counter.p, 0, sizeof(unsigned) * 4) != cudaSuccess) {
    delete ctx;
    return CCFV_ERR_CUDA;
  }
  *out = ctx;
  return CCFV_OK;
}

int ccfv_destroy(ccfv_ctx *ctx) {
  if (!ctx) return CCFV_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  delete ctx;
  return CCFV_OK;
}

int ccfv_check(ccfv_ctx *ctx, void *stream) {
  if (!ctx) return CCFV_ERR_INVALID;
  int rc = use_device(ctx);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned flag = 0;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaMemcpy(&flag, ctx->status.p, sizeof(unsigned), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_error(ctx, CCFV_ERR_CUDA, cudaGetErrorString(e));
  if (flag) {
    cudaMemset(ctx->status.p, 0, sizeof(unsigned));
    return set_error(ctx, CCFV_ERR_HALO, "a characteristic foot left the staged halo");
  }
  return CCFV_OK;
}

int ccfv_step(ccfv_ctx *ctx, double *d_C, double tn, double dt, void *stream) {
  if (!ctx || !d_C) return CCFV_ERR_INVALID;
  int rc = use_device(ctx);
  if (rc) return rc;
  rc = steps(ctx, d_C, true, tn, dt, 1, (cudaStream_t)stream);
  return rc ? rc : last_launch(ctx);
}

int ccfv_fine(ccfv_ctx *ctx, double *d_C, double tn, double DT, int J, void *stream) {
  if (!ctx || !d_C || J < 1) return CCFV_ERR_INVALID;
  int rc = use_device(ctx);
  if (rc) return rc;
  // FinePropagator: dt = DT / J, t_local = tn + j * dt (T2S4:979-982)
  rc = steps(ctx, d_C, true, tn, DT / (double)J, J, (cudaStream_t)stream);
  return rc ? rc : last_launch(ctx);
}

int ccfv_coarse(ccfv_ctx *ctx, double *d_C, double tn, double DT, int m, int precision,
                void *stream) {
  if (!ctx || !d_C || m < 1) return CCFV_ERR_INVALID;
  if (precision != CCFV_FP64 && precision != CCFV_FP32) return CCFV_ERR_INVALID;
  int rc = use_device(ctx);
  if (rc) return rc;
  if (precision == CCFV_FP64)
    rc = steps(ctx, d_C, true, tn, DT / (double)m, m, (cudaStream_t)stream);
  else
    rc = coarse_fp32(ctx, d_C, tn, DT, m, (cudaStream_t)stream);
  return rc ? rc : last_launch(ctx);
}

int ccfv_coarse_ex(ccfv_ctx *ctx, double *d_C, double tn, double DT, int m, int precision,
                   double theta, void *stream) {
  if (!ctx || !d_C || m < 1 || !(DT > 0.0)) return CCFV_ERR_INVALID;
  if (precision != CCFV_FP64 && precision != CCFV_FP32) return CCFV_ERR_INVALID;
  if (!coarse_theta_ok(theta)) return CCFV_ERR_INVALID;
  ccfv_parareal_opts o;
  std::memset(&o, 0, sizeof(o));
  o.coarse_theta = theta;
  const double th = coarse_theta(o, ctx->grid, DT / (double)m);
  int rc = use_device(ctx);
  if (rc) return rc;
  if (precision == CCFV_FP64)
    rc = steps(ctx, d_C, true, tn, DT / (double)m, m, (cudaStream_t)stream, th);
  else
    rc = coarse_fp32(ctx, d_C, tn, DT, m, (cudaStream_t)stream, th);
  return rc ? rc : last_launch(ctx);
}

int ccfv_coarse_theta(const ccfv_grid *grid, const ccfv_parareal_opts *opts, double *theta) {
  if (!grid || !opts || !theta || !grid_ok(grid)) return CCFV_ERR_INVALID;
  const ccfv_parareal_opts &o = *opts;
  if (o.n_slices < 1 || o.nt_fine < o.n_slices || o.nt_fine % o.n_slices || !(o.t1 > o.t0))
    return CCFV_ERR_INVALID;
  const int J = o.nt_fine / o.n_slices;
  if (o.coarse_ratio < 0 || (o.coarse_ratio > 0 && J % o.coarse_ratio)) return CCFV_ERR_INVALID;
  if (!coarse_theta_ok(o.coarse_theta)) return CCFV_ERR_INVALID;
  const int m = o.coarse_ratio > 0 ? J / o.coarse_ratio : 1;
  *theta = coarse_theta(o, *grid, (o.t1 - o.t0) / o.n_slices / (double)m);
  return CCFV_OK;
}

int ccfv_run(ccfv_ctx *ctx, double *C, int mem, double t0, double dt, int nsteps, void *stream) {
  if (!ctx || !C || nsteps < 0) return CCFV_ERR_INVALID;
  if (mem != CCFV_MEM_DEVICE && mem != CCFV_MEM_HOST) return CCFV_ERR_INVALID;
  int rc = use_device(ctx);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t bytes = sizeof(double) * (size_t)ctx->grid.nx * ctx->grid.ny;
  double *d = C;
  if (mem == CCFV_MEM_HOST) {
    if (ctx->io.alloc(bytes) != cudaSuccess) return set_error(ctx, CCFV_ERR_NOMEM, "io buffer");
    d = ctx->io.as<double>();
    cudaError_t e = cudaMemcpyAsync(d, C, bytes, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return set_error(ctx, CCFV_ERR_CUDA, cudaGetErrorString(e));
  }
  rc = steps(ctx, d, true, t0, dt, nsteps, st);
  if (rc) return rc;
  if (mem == CCFV_MEM_HOST) {
    cudaError_t e = cudaMemcpyAsync(C, d, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_error(ctx, CCFV_ERR_CUDA, cudaGetErrorString(e));
  }
  return last_launch(ctx);
}

int ccfv_parareal(ccfv_ctx *ctx, const ccfv_parareal_opts *opts, const double *C0, double *C_T,
                  ccfv_stats *stats, void *stream) {
  if (!ctx) return CCFV_ERR_INVALID;
  int rc = use_device(ctx);
  if (rc) return rc;
  return parareal(ctx, opts, C0, C_T, stats, (cudaStream_t)stream);
}

int ccfv_exact_ref(ccfv_ctx *ctx, double *d_C, double t, void *stream) {
  if (!ctx || !d_C) return CCFV_ERR_INVALID;
  int rc = use_device(ctx);
  return rc ? rc : exact_ref(ctx, d_C, t, (cudaStream_t)stream);
}

int ccfv_gaussians(ccfv_ctx *ctx, double *d_C, int n, const double *params, int images,
                   void *stream) {
  if (!ctx || !d_C || n < 1 || !params || images < 0 || images > 4) return CCFV_ERR_INVALID;
  for (int q = 0; q < n; ++q)
    if (!(params[4 * q + 2] > 0.0)) return CCFV_ERR_INVALID;
  int rc = use_device(ctx);
  return rc ? rc : gaussians(ctx, d_C, n, params, images, (cudaStream_t)stream);
}

int ccfv_error_norms(ccfv_ctx *ctx, const double *d_a, const double *d_b, double *rel_l2,
                     double *max_abs, void *stream) {
  if (!ctx || !d_a || !d_b) return CCFV_ERR_INVALID;
  int rc = use_device(ctx);
  return rc ? rc : norms(ctx, d_a, d_b, rel_l2, max_abs, (cudaStream_t)stream);
}

int ccfv_batch_solve(int n, const ccfv_problem *problems, ccfv_stats *stats, int device,
                     void *stream) {
  if (n < 1 || !problems) return CCFV_ERR_INVALID;
  for (int i = 0; i < n; ++i)
    if (!grid_ok(&problems[i].grid) || !problems[i].C0 || !problems[i].C_T) return CCFV_ERR_INVALID;
  std::string err;
  return batch_solve(n, problems, stats, device, (cudaStream_t)stream, &err);
}

int ccfv_fine_slices(ccfv_ctx *ctx, double *d_fields, int n, double t0, double slice_dt,
                     double DT, int J, void *stream) {
  if (!ctx || !d_fields || n < 1 || J < 1) return CCFV_ERR_INVALID;
  int rc = use_device(ctx);
  return rc ? rc : fine_slices(ctx, d_fields, n, t0, slice_dt, DT, J, (cudaStream_t)stream);
}

int ccfv_correct(ccfv_ctx *ctx, int form, double *d_U, const double *d_F, double *d_Gold,
                 double *d_W, double *sq_update, double *sq_state, void *stream) {
  if (!ctx || !d_U || !d_F || !d_W) return CCFV_ERR_INVALID;
  if (form != CCFV_FORM_STANDARD && form != CCFV_FORM_DELTA) return CCFV_ERR_INVALID;
  if (form == CCFV_FORM_STANDARD && !d_Gold) return CCFV_ERR_INVALID;
  int rc = use_device(ctx);
  return rc ? rc : correct(ctx, form, d_U, d_F, d_Gold, d_W, sq_update, sq_state, (cudaStream_t)stream);
}

int ccfv_autotune(ccfv_ctx *ctx, double dt, int precision, int *segment, void *stream) {
  if (!ctx || !(dt > 0.0) || (precision != CCFV_FP64 && precision != CCFV_FP32))
    return CCFV_ERR_INVALID;
  int rc = use_device(ctx);
  return rc ? rc : autotune(ctx, dt, precision == CCFV_FP64, (cudaStream_t)stream, segment);
}

int ccfv_sweep_plan(ccfv_ctx *ctx, double dt, int precision, int variant[3], int segment[3]) {
  if (!ctx || !(dt > 0.0) || (precision != CCFV_FP64 && precision != CCFV_FP32))
    return CCFV_ERR_INVALID;
  for (int kind = 0; kind < 3; ++kind) {
    const int dir = kind == 1 ? 1 : 0;
    const double Dt = kind == 1 ? dt : 0.5 * dt;
    const int dsrc = (kind == 2 && ctx->grid.scheme == CCFV_SCHEME_REFERENCE) ? 1 : 0;
    // as ccfv_step/ccfv_run and the Parareal engines sweep: out of place
    const LaunchGeom G = step_geom(ctx->grid, dir, Dt, dsrc, precision == CCFV_FP64, false);
    if (variant)
      variant[kind] = (ctx->force_general && G.variant != SWEEP_GENERAL_SRC) ? SWEEP_GENERAL : G.variant;
    if (segment) {
      // the cluster form runs whole-walk segments (and a shorter last one)
      // when its segment count is the least that covers the line
      const int L = dir == 0 ? ctx->grid.nx : ctx->grid.ny, walk = filter_segment_max(0);
      const bool whole = exact_filter_variant(G.variant) && (G.cs - 1) * walk < L &&
                         G.cs * walk >= L;
      segment[kind] = whole ? walk : G.lc_max;
    }
  }
  return CCFV_OK;
}

uint64_t ccfv_kernel_launches(void) { return launches(); }

const char *ccfv_last_error(ccfv_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

}  // extern "C"
