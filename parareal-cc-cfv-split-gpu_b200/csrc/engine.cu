// engine.cu -- solver context, line-invariant tridiagonal factors, step plans,
// propagators and the Parareal engine of libccfv.
#include "engine.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>

namespace ccfv {

static std::atomic<uint64_t> g_launches{0};
void count_launch(uint64_t n) { g_launches += n; }
uint64_t launches() { return g_launches.load(); }

cudaError_t DevBuf::alloc(size_t b) {
  if (p && bytes >= b) return cudaSuccess;
  if (p) {
    cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  if (b == 0) return cudaSuccess;
  cudaError_t e = cudaMalloc(&p, b);
  if (e == cudaSuccess) bytes = b;
  else p = nullptr;
  return e;
}

int set_error(ccfv_ctx *ctx, int code, const std::string &msg) {
  if (ctx) ctx->last_error = msg;
  return code;
}

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return set_error(ctx, e_ == cudaErrorMemoryAllocation ? CCFV_ERR_NOMEM : CCFV_ERR_CUDA, \
                       std::string(#call) + ": " + cudaGetErrorString(e_));            \
  } while (0)

// ---------------------------------------------------------------------------
// Line-invariant factors of the constant tridiagonal system
//   a x_{k-1} + b x_k + a x_{k+1} = r_k,  a = 1/12 - 0.5 K Dt/h^2,
//   b = 10/12 + K Dt/h^2  (x_A_LHS_on_gpu / y_A_LHS_on_gpu, T2S4:550-594).
// LU in the reference's Thomas order (x_Thomas_on_gpu, T2S4:666-676):
//   g_k = 1/(b_k - p_{k-1} a), p_k = a g_k, alpha_k = -a g_k,
// so that forward q_k = g_k r_k + alpha_k q_{k-1} and backward
// x_k = q_k + alpha_k x_{k+1}.  Periodic: Sherman-Morrison with gamma = -b,
// b_0 -> b - gamma, b_{L-1} -> b - a^2/gamma, z = A'^{-1} (gamma,0..0,a).
template <typename T>
static void build_table(int L, double coA, double coB, int bc, std::vector<T> &out,
                        double &sm_fac, double &sm_inv_den) {
  const double coC = coA, gam = -coB;
  std::vector<double> diag(L, coB), g(L), p(L), z(L, 0.0);
  if (bc == BC_PERIODIC) {
    diag[0] = coB - gam;
    diag[L - 1] = coB - coA * coC / gam;
  }
  g[0] = 1.0 / diag[0];
  p[0] = coC / diag[0];
  for (int k = 1; k < L; ++k) {
    g[k] = 1.0 / (diag[k] - p[k - 1] * coA);
    p[k] = coC * g[k];
  }
  out.assign(table_len(L), T(0));
  for (int k = 0; k < L; ++k) {
    out[k] = T(-coA * g[k]);
    out[L + k] = T(g[k]);
  }
  sm_fac = 0.0;
  sm_inv_den = 0.0;
  if (bc == BC_PERIODIC) {
    std::vector<double> q(L);
    for (int k = 0; k < L; ++k) {
      double u = (k == 0) ? gam : (k == L - 1 ? coC : 0.0);
      q[k] = g[k] * u + (k ? (-coA * g[k]) * q[k - 1] : 0.0);
    }
    z[L - 1] = q[L - 1];
    for (int k = L - 2; k >= 0; --k) z[k] = q[k] - p[k] * z[k + 1];
    for (int k = 0; k < L; ++k) out[2 * (size_t)L + k] = T(z[k]);
    sm_fac = coA / gam;
    sm_inv_den = 1.0 / (1.0 + z[0] + sm_fac * z[L - 1]);
  }
  fill_chunk_products(L, out.data());
}

template <typename T>
void fill_chunk_products(int L, T *tab) {
  const int cs = table_cs(L), Lc = (L + cs - 1) / cs;
  const T *alpha = tab;
  T *tP = tab + 3 * (size_t)L, *tS = tab + 4 * (size_t)L;
  T *aggA = tab + 5 * (size_t)L, *PA = aggA + (size_t)cs * NCH;
  for (int r = 0; r < cs; ++r) {
    const int p0 = std::min(L, r * Lc), p1 = std::min(L, p0 + Lc), np = p1 - p0;
    const int m = np > 0 ? (np + NCH - 1) / NCH : 1;
    double pre = 1.0;
    for (int c = 0; c < NCH; ++c) {
      const int s0 = std::min(p1, p0 + c * m), e0 = std::min(p1, s0 + m);
      double a = 1.0;
      for (int k = s0; k < e0; ++k) {
        a *= (double)alpha[k];
        tP[k] = T(a);
      }
      double b = 1.0;
      for (int k = e0 - 1; k >= s0; --k) {
        b *= (double)alpha[k];
        tS[k] = T(b);
      }
      aggA[(size_t)r * NCH + c] = T(a);
      PA[(size_t)r * (NCH + 1) + c] = T(pre);
      pre *= a;
    }
    PA[(size_t)r * (NCH + 1) + NCH] = T(pre);
  }
}
template void fill_chunk_products<double>(int, double *);
template void fill_chunk_products<float>(int, float *);

static double spacing(const ccfv_grid &g, int dir) {
  return dir == 0 ? (g.x_max - g.x_min) / g.nx : (g.y_max - g.y_min) / g.ny;
}

const SolverTable *get_table(ccfv_ctx *ctx, int dir, double Dt, bool fp64, int *status,
                             double theta) {
  auto key = std::make_tuple(dir, Dt, fp64 ? 1 : 0, theta);
  auto it = ctx->tables.find(key);
  if (it != ctx->tables.end()) return it->second.get();
  const ccfv_grid &g = ctx->grid;
  const int L = dir == 0 ? g.nx : g.ny;
  const double h = spacing(g, dir);
  const double r2 = Dt / (h * h);
  // x_A_LHS / y_A_LHS (T2S4:550-594) at theta = 1/2
  const double coA = 1.0 / 12 - theta * g.K * r2;
  const double coB = 10.0 / 12 + 2.0 * theta * g.K * r2;
  auto tab = std::make_unique<SolverTable>();
  size_t bytes = table_len(L) * (fp64 ? 8 : 4);
  if (tab->buf.alloc(bytes) != cudaSuccess) {
    *status = set_error(ctx, CCFV_ERR_NOMEM, "solver table allocation failed");
    return nullptr;
  }
  cudaError_t e;
  if (fp64) {
    std::vector<double> h_tab;
    build_table(L, coA, coB, g.bc, h_tab, tab->sm_fac, tab->sm_inv_den);
    e = cudaMemcpy(tab->buf.p, h_tab.data(), bytes, cudaMemcpyHostToDevice);
  } else {
    std::vector<float> h_tab;
    build_table(L, coA, coB, g.bc, h_tab, tab->sm_fac, tab->sm_inv_den);
    e = cudaMemcpy(tab->buf.p, h_tab.data(), bytes, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    *status = set_error(ctx, CCFV_ERR_CUDA, cudaGetErrorString(e));
    return nullptr;
  }
  const SolverTable *res = tab.get();
  ctx->tables[key] = std::move(tab);
  return res;
}

// Automatic coarse diffusion weight.  For the grid-scale (checkerboard) mode
// a theta-weighted sub-step of diffusion number nu = K Dt/h^2 multiplies the
// field by
//   a(theta, nu) = (2/3 - (32/9)(1 - theta) nu) / (2/3 + 4 theta nu):
// the compact mass matrix (1,10,1)/12 gives 2/3, the LHS second difference
// 4 theta nu, and the RHS difference of fourth-order edge derivatives
// (C_{i-1} - 15 C_i + 15 C_{i+1} - C_{i+2}) / 12h gives (16/3) nu under the
// mass matrix.  Crank-Nicolson (theta = 1/2) tends to -8/9 as nu grows; the
// rule takes the smallest theta >= 1/2 with |a| <= rho = 1/5 at the largest
// nu of the coarse step's sub-steps (x: dtc/2, y: dtc).  Measured against the
// Parareal iteration count on stiff cases (nu from 2 to 26), the optimum
// theta sits at |a| of 0.2 - 0.25.
double coarse_theta(const ccfv_parareal_opts &o, const ccfv_grid &g, double dtc) {
  if (o.coarse_theta > 0) return o.coarse_theta;
  if (o.coarse_theta != CCFV_COARSE_THETA_AUTO) return 0.5;
  const double hx = spacing(g, 0), hy = spacing(g, 1);
  const double nu = g.K * std::max(0.5 * dtc / (hx * hx), dtc / (hy * hy));
  const double rho = 0.2;
  if (!(nu > 0)) return 0.5;
  const double th = (32.0 / 9.0 * nu - 2.0 / 3.0 * (1.0 + rho)) / (nu * (32.0 / 9.0 + 4.0 * rho));
  return std::min(1.0, std::max(0.5, th));
}

// Largest |velocity component along the sweep| over the domain (bounds the
// characteristic displacement, hence the staged halo).
static double wmax(const ccfv_grid &g, int dir) {
  const double *p = g.vel_params;
  switch (g.velocity) {
    case CCFV_VEL_REF_ROT4:
      return dir == 0 ? 4 * std::max(std::fabs(g.y_min), std::fabs(g.y_max))
                      : 4 * std::max(std::fabs(g.x_min), std::fabs(g.x_max));
    case CCFV_VEL_CONST: return std::fabs(dir == 0 ? p[0] : p[1]);
    case CCFV_VEL_ROTATION:
      return dir == 0 ? std::fabs(p[0]) * std::max(std::fabs(g.y_min - p[2]), std::fabs(g.y_max - p[2]))
                      : std::fabs(p[0]) * std::max(std::fabs(g.x_min - p[1]), std::fabs(g.x_max - p[1]));
    case CCFV_VEL_SWIRL: return 1.0;
  }
  return 0.0;
}

static int shift_cells(const ccfv_grid &g, int dir, double Dt) {
  double s = std::fabs(Dt) * wmax(g, dir) / spacing(g, dir);
  return (int)std::ceil(s + 1e-9);
}

SweepField make_field(const ccfv_grid &g, int dir, double Dt, double ta_rel, double tb_rel,
                      void *data, const SolverTable *tab, int dsrc, double theta) {
  SweepField f;
  std::memset(&f, 0, sizeof(f));
  const double dx = (g.x_max - g.x_min) / g.nx, dy = (g.y_max - g.y_min) / g.ny;
  if (dir == 0) {
    f.L = g.nx; f.M = g.ny; f.s_pos = g.ny; f.s_line = 1;
    f.s_min = g.x_min; f.s_max = g.x_max; f.h = dx; f.t_min = g.y_min; f.ht = dy;
    f.eps_remap = 1e-15;  // T2S4:323-324
  } else {
    f.L = g.ny; f.M = g.nx; f.s_pos = 1; f.s_line = g.ny;
    f.s_min = g.y_min; f.s_max = g.y_max; f.h = dy; f.t_min = g.x_min; f.ht = dx;
    f.eps_remap = 1e-16;  // T2S4:414-415
  }
  f.data = data;
  f.dir = dir;
  f.bc = g.bc;
  f.vel = g.velocity;
  for (int i = 0; i < 4; ++i) f.vp[i] = g.vel_params[i];
  f.Dt = Dt;
  f.ta_rel = ta_rel;
  f.tb_rel = tb_rel;
  f.kb = (1.0 - theta) * g.K * (Dt / f.h);  // explicit diffusion weight (theta = 1: none)
  f.theta = theta;
  f.src = g.source;
  for (int i = 0; i < 5; ++i) f.sp[i] = g.source_params[i];
  f.src_w = g.source ? (g.scheme == CCFV_SCHEME_REFERENCE ? 0.5 : 0.25) * Dt : 0.0;
  f.src_tb = 0;  // 1 for the third sub-step (f(t_n+1) remapped): set by the caller
  f.inv12h = 1.0 / (12.0 * f.h);
  f.tab = tab->buf.p;
  f.sm_fac = tab->sm_fac;
  f.sm_inv_den = tab->sm_inv_den;
  f.groups = (f.M + LPG - 1) / LPG;
  f.dsrc = dsrc;
  f.hd = dsrc ? shift_cells(g, dir, Dt) + 4 : 0;
  f.uniform = (g.velocity == CCFV_VEL_REF_ROT4 || g.velocity == CCFV_VEL_CONST ||
               g.velocity == CCFV_VEL_ROTATION) ? 1 : 0;
  return f;
}

// Factorisation of the cyclic constant system used by the filter kernel:
// a z^-1 + b + a z = c (1 + mu z^-1)(1 + mu z), |mu| < 1; J = warm-up length
// with |mu|^J below the rounding of the precision.  Returns false when the
// warm-up would exceed FILTER_JMAX (strong diffusion: exact-scan kernels).
bool filter_params(const ccfv_grid &g, int dir, double Dt, bool fp64, double *mu, double *ic,
                   int *J, double theta) {
  const double h = spacing(g, dir);
  const double r2 = Dt / (h * h);
  const double a = 1.0 / 12 - theta * g.K * r2, b = 10.0 / 12 + 2.0 * theta * g.K * r2;
  const double r = a / b;  // |r| < 1/2 (diagonal dominance)
  const double m = 2.0 * r / (1.0 + std::sqrt(std::max(0.0, 1.0 - 4.0 * r * r)));
  const double c = b / (1.0 + m * m);
  const double eps = fp64 ? std::ldexp(1.0, -56) : std::ldexp(1.0, -27);
  int j = 1;
  if (std::fabs(m) > 1e-300) j = std::max(1, (int)std::ceil(std::log(eps) / std::log(std::fabs(m))));
  if (mu) *mu = m;
  if (ic) *ic = 1.0 / c;
  if (J) *J = j;
  return j <= FILTER_JMAX;
}

// Autotuned segment length (cells per CTA) of the filter kernel, per line
// length and precision (ccfv_autotune), and per line-length class (the next
// power of two, tuned by the batched engine on the first problem of each
// class); the default until either is measured.
static std::mutex g_tune_mu;
static std::map<std::pair<int, int>, int> g_filter_lc;        // (L, fp64)
static std::map<std::pair<int, int>, int> g_filter_lc_class;  // (class, fp64)
static thread_local int g_lc_override = 0;

int line_class(int L) {
  int c = 64;
  while (c < L) c *= 2;
  return c;
}

int filter_lc(int L, bool fp64) {
  if (g_lc_override > 0) return g_lc_override;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_filter_lc.find({L, fp64 ? 1 : 0});
  if (it != g_filter_lc.end()) return it->second;
  auto ic = g_filter_lc_class.find({line_class(L), fp64 ? 1 : 0});
  return ic == g_filter_lc_class.end() ? LC_MAX : ic->second;
}

bool class_tuned(int L, bool fp64) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  return g_filter_lc_class.count({line_class(L), fp64 ? 1 : 0}) > 0;
}

LaunchGeom step_geom(const ccfv_grid &g, int dir, double Dt, int dsrc, bool fp64, bool inplace,
                     double theta) {
  LaunchGeom G;
  const int L = dir == 0 ? g.nx : g.ny;
  G.cs = (L + LC_MAX - 1) / LC_MAX;
  G.lc_max = (L + G.cs - 1) / G.cs;
  const int sh = shift_cells(g, dir, Dt);
  G.halo = dsrc ? (sh + 4) + sh + 5 : sh + 5;
  const bool uniform = g.velocity == CCFV_VEL_REF_ROT4 || g.velocity == CCFV_VEL_CONST ||
                       g.velocity == CCFV_VEL_ROTATION;
  G.variant = g.source ? SWEEP_GENERAL_SRC : SWEEP_GENERAL;
  if (!g.source && g.bc == CCFV_BC_PERIODIC && dsrc == 0) {
    // periodic, derivative of the sweep input: the filter kernel, with the
    // per-line stencil (uniform displacement) or the per-cell right-hand side
    const LaunchGeom general = G;
    int J = 0;
    const bool warm = filter_params(g, dir, Dt, fp64, nullptr, nullptr, &J, theta) && L > 2 * J;
    const int seg_exact = filter_segment_max(0);  // cells per CTA without warm-up
    if (!warm && !inplace && (L + seg_exact - 1) / seg_exact <= MAX_CLUSTER) {
      // strong diffusion, out of place: the filter kernel's cluster form
      // (exact periodic closure across the segments, no warm-up)
      const int lc = std::min(seg_exact, std::max({32, (L + MAX_CLUSTER - 1) / MAX_CLUSTER,
                                                   std::min(L, filter_lc(L, fp64))}));
      G.variant = uniform ? SWEEP_FILTER_EXACT : SWEEP_CELL_EXACT;
      G.cs = (L + lc - 1) / lc;
      G.lc_max = (L + G.cs - 1) / G.cs;
      G.halo = sh + 6;
    } else if (warm) {
      G.variant = uniform ? SWEEP_FILTER : SWEEP_CELL;
      G.halo = J + sh + 6;
      // segment length from the tuner; the segments of a line form one
      // cluster (at most MAX_CLUSTER CTAs)
      const int lc = std::min(filter_segment_max(J),
                              std::max({32, (L + MAX_CLUSTER - 1) / MAX_CLUSTER,
                                        std::min(L, filter_lc(L, fp64))}));
      G.cs = (L + lc - 1) / lc;
      G.lc_max = (L + G.cs - 1) / G.cs;
      if (inplace && G.cs > MAX_CLUSTER) {  // in place, a line's segments form one cluster
        G = general;
        if (uniform) G.variant = SWEEP_FAST;
      }
    } else if (uniform) {
      G.variant = SWEEP_FAST;
    }
    if (cell_filter_variant(G.variant) &&
        sweep_filter_smem_bytes(G.lc_max, G.halo, fp64, exact_filter_variant(G.variant), true) >
            227 * 1024)
      G = general;  // the per-cell form's two tiles do not fit: per-cell scan kernel
  } else if (!g.source && g.bc == CCFV_BC_COMPAT) {
    // the reference's boundaries: the filter kernel's per-cell form with the
    // non-cyclic closure.  A line of at most one segment is solved exactly
    // (the recurrences start at its ends, no warm-up, any diffusion number);
    // longer lines need the warm-up between segments.
    const LaunchGeom general = G;
    const int extra = dsrc ? (sh + 4) + sh + 4 : sh + 6;  // foot + stencil (+ remapped field)
    int J = 0;
    const bool jok = filter_params(g, dir, Dt, fp64, nullptr, nullptr, &J, theta) && L > 2 * J;
    if (L <= filter_segment_max(0)) {
      G.variant = SWEEP_CELL_COMPAT;
      G.cs = 1;
      G.lc_max = L;
      G.halo = extra;
    } else if (jok) {
      G.variant = SWEEP_CELL_COMPAT;
      G.halo = J + extra;
      const int lc = std::min(filter_segment_max(J),
                              std::max({32, (L + MAX_CLUSTER - 1) / MAX_CLUSTER,
                                        std::min(L, filter_lc(L, fp64))}));
      G.cs = (L + lc - 1) / lc;
      G.lc_max = (L + G.cs - 1) / G.cs;
      if (inplace && G.cs > MAX_CLUSTER) G = general;
    }
    if (G.variant == SWEEP_CELL_COMPAT &&
        sweep_filter_smem_bytes(G.lc_max, G.halo, fp64, false, true) > 227 * 1024)
      G = general;
  }
  return G;
}

// Times the filter kernel's candidate segment lengths on this grid (x and y
// sweeps of one step of dt on a scratch field) and keeps the fastest.
int autotune(ccfv_ctx *ctx, double dt, bool fp64, cudaStream_t st, int *chosen, bool for_class) {
  const ccfv_grid &g = ctx->grid;
  const size_t el = fp64 ? 8 : 4;
  const size_t NN = (size_t)g.nx * g.ny;
  if (!ctx->status.p) {  // contexts of the batched engine's problems have none
    CK(ctx->status.alloc(sizeof(unsigned) * 4));
    CK(cudaMemsetAsync(ctx->status.p, 0, sizeof(unsigned) * 4, st));
  }
  // timed as the Parareal engines run it: out of place over buffer pairs.
  // For a line-length class (the batched engine) the launch holds copies of
  // the field up to about 2^24 cells, so the timing is that of a launch that
  // fills the GPU, as the batched launches do (a lone small field favours
  // short segments, whose warm-up costs more once the GPU is full).
  const size_t nf = for_class ? std::max<size_t>(1, ((size_t)1 << 24) / NN) : 1;
  CK(ctx->io.alloc(2 * el * NN * nf));
  CK(cudaMemsetAsync(ctx->io.p, 0, 2 * el * NN * nf, st));
  std::vector<PlanField> pf(nf);
  for (size_t i = 0; i < nf; ++i) {
    unsigned char *base = static_cast<unsigned char *>(ctx->io.p) + 2 * el * NN * i;
    pf[i].A = base;
    pf[i].B = base + el * NN;
    pf[i].in0 = base;
  }
  static const int cand[] = {64, 96, 128, 192, 256, 384, 512};
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  float best = 1e30f;
  int best_lc = LC_MAX;
  for (int lc : cand) {
    if (lc > std::max(g.nx, g.ny) && lc != cand[0]) break;
    g_lc_override = lc;
    StepPlan plan;
    int rc = build_step_plan(ctx, &plan, dt, fp64, pf);
    if (rc == CCFV_OK && !warm_filter_variant(plan.geom[0].variant) &&
        !warm_filter_variant(plan.geom[1].variant)) {
      g_lc_override = 0;
      break;  // nothing to tune: this grid does not use the filter kernel
    }
    if (rc == CCFV_OK) rc = run_step_plan(ctx, plan, fp64, 0, (int)nf, 0.0, nullptr, st, 0);
    if (rc == CCFV_OK) {
      cudaEventRecord(a, st);
      for (int r = 0; r < 5 && rc == CCFV_OK; ++r)
        rc = run_step_plan(ctx, plan, fp64, 0, (int)nf, 0.0, nullptr, st, r);
      cudaEventRecord(b, st);
      cudaEventSynchronize(b);
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      if (rc == CCFV_OK && ms < best) {
        best = ms;
        best_lc = lc;
      }
    }
    g_lc_override = 0;
    if (rc != CCFV_OK && rc != CCFV_ERR_UNSUPPORTED) {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      return rc;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (for_class) {  // the class of each line length, unless tuned already
      g_filter_lc_class.insert({{line_class(g.nx), fp64 ? 1 : 0}, best_lc});
      g_filter_lc_class.insert({{line_class(g.ny), fp64 ? 1 : 0}, best_lc});
    } else {
      g_filter_lc[{g.nx, fp64 ? 1 : 0}] = best_lc;
      g_filter_lc[{g.ny, fp64 ? 1 : 0}] = best_lc;
    }
  }
  ctx->step_plans.clear();  // plans built with the old geometry
  ctx->fine_plan.reset();
  if (for_class) ctx->io.release();  // scratch of the timing runs only
  if (chosen) *chosen = best_lc;
  return CCFV_OK;
}

// Fills the filter-kernel constants of a field (its variant must be FILTER).
void filter_field(const ccfv_grid &g, SweepField &f, bool fp64) {
  double mu = 0, ic = 0;
  int J = 0;
  filter_params(g, f.dir, f.Dt, fp64, &mu, &ic, &J, f.theta);
  f.sm_fac = mu;
  f.sm_inv_den = ic;
  // compat lines of one segment: the non-cyclic recurrences start exactly at
  // the line's ends (no warm-up)
  f.jf = (g.bc == CCFV_BC_COMPAT && f.L <= filter_segment_max(0)) ? 0 : J;
}

// Sub-steps of one split step: x(dt/2) over [t, t+dt/2], y(dt) over
// [t, t+dt], x(dt/2) over [t+dt/2, t+dt] (GpuOneStep, T2S4:785-968).
static void sweep_kind(int kind, double dt, int *dir, double *Dt, double *ta, double *tb) {
  if (kind == 0) { *dir = 0; *Dt = 0.5 * dt; *ta = 0.0; *tb = 0.5 * dt; }
  else if (kind == 1) { *dir = 1; *Dt = dt; *ta = 0.0; *tb = dt; }
  else { *dir = 0; *Dt = 0.5 * dt; *ta = 0.5 * dt; *tb = dt; }
}

int build_step_plan(ccfv_ctx *ctx, StepPlan *plan, double dt, bool fp64,
                    const std::vector<std::pair<void *, double>> &fields, bool homogeneous,
                    double theta) {
  std::vector<PlanField> pf(fields.size());
  for (size_t i = 0; i < fields.size(); ++i) {
    pf[i].A = fields[i].first;
    pf[i].t0 = fields[i].second;
  }
  return build_step_plan(ctx, plan, dt, fp64, pf, homogeneous, theta);
}

int build_step_plan(ccfv_ctx *ctx, StepPlan *plan, double dt, bool fp64,
                    const std::vector<PlanField> &fields, bool homogeneous, double theta) {
  ccfv_grid g = ctx->grid;
  if (homogeneous) g.source = CCFV_SRC_NONE;
  const int nf = (int)fields.size();
  std::vector<SweepField> h(3 * (size_t)nf);
  for (int kind = 0; kind < 3; ++kind) {
    int dir;
    double Dt, ta, tb;
    sweep_kind(kind, dt, &dir, &Dt, &ta, &tb);
    const int dsrc = (kind == 2 && g.scheme == CCFV_SCHEME_REFERENCE) ? 1 : 0;
    int st = CCFV_OK;
    const SolverTable *tab = get_table(ctx, dir, Dt, fp64, &st, theta);
    if (!tab) return st;
    const bool plan_pp = !fields.empty() && fields[0].B != nullptr;
    LaunchGeom G = step_geom(g, dir, Dt, dsrc, fp64, !plan_pp, theta);
    if (ctx->force_general && G.variant != SWEEP_GENERAL_SRC) G.variant = SWEEP_GENERAL;
    if (G.cs > MAX_CLUSTER && !(warm_filter_variant(G.variant) && plan_pp))
      return set_error(ctx, CCFV_ERR_UNSUPPORTED, "line longer than 4096 cells");
    if (std::max({sweep_smem_bytes(G.lc_max, G.halo, fp64, g.source != 0),
                  sweep_fast_smem_bytes(G.lc_max, G.halo, fp64),
                  sweep_filter_smem_bytes(G.lc_max, G.halo, fp64, true,
                                          cell_filter_variant(G.variant))}) > 227 * 1024)
      return set_error(ctx, CCFV_ERR_UNSUPPORTED, "time step too large for the staged halo");
    for (int i = 0; i < nf; ++i) {
      const PlanField &pfi = fields[i];
      SweepField f = make_field(g, dir, Dt, ta + pfi.t0, tb + pfi.t0, pfi.A, tab, dsrc, theta);
      f.kind = kind;
      if (pfi.B) {
        f.pp = 1;
        f.data2 = pfi.B;
        f.in0 = pfi.in0;
        f.par = pfi.par;
      }
      if (filter_variant(G.variant)) filter_field(g, f, fp64);
      f.src_tb = kind == 2 ? 1 : 0;
      f.group0 = i * f.groups;
      f.cta0 = f.group0 * G.cs;
      f.halo_f = G.halo;
      h[(size_t)kind * nf + i] = f;
      plan->groups_per_field[kind] = f.groups;
    }
    plan->geom[kind] = G;
    // Compat lines, out of place: segments at least a halo from both line
    // ends see no boundary (no clamps or ghosts, and the non-cyclic
    // correction has decayed within the warm-up), so they run the stencil
    // form (one tile) in a second launch and the compat form keeps the
    // segments at the ends.  The reference scheme's third sweep, which
    // differentiates the remapped field, takes the 13-tap stencil form
    // (displacements of at most two cells).
    plan->hyb[kind] = false;
    plan->wide[kind] = false;
    static const bool split_on = [] {
      const char *e = std::getenv("CCFV_COMPAT_SPLIT");
      return !(e && e[0] == '0');
    }();
    const bool uniform = g.velocity == CCFV_VEL_REF_ROT4 || g.velocity == CCFV_VEL_CONST ||
                         g.velocity == CCFV_VEL_ROTATION;
    int Jc = 0;
    const int shc = shift_cells(g, dir, Dt);
    if (split_on && plan_pp && uniform && g.bc == CCFV_BC_COMPAT && !g.source &&
        G.variant == SWEEP_CELL_COMPAT && G.cs >= 3 && (dsrc == 0 || shc <= 2) &&
        filter_params(g, dir, Dt, fp64, nullptr, nullptr, &Jc, theta) && Jc > 0) {
      const int L = dir == 0 ? g.nx : g.ny;
      const bool wide = dsrc != 0;
      LaunchGeom G2 = G;
      G2.variant = wide ? SWEEP_FILTER_WIDE : SWEEP_FILTER;
      G2.halo = wide ? Jc + 2 * shc + 12 : Jc + shc + 6;
      if ((L + G.cs - 1) / G.cs >= G2.halo &&
          sweep_filter_smem_bytes(G2.lc_max, G2.halo, fp64, false, false, wide) <= 227 * 1024) {
        plan->hyb[kind] = true;
        plan->wide[kind] = wide;
        plan->geom2[kind] = G2;
        for (int i = 0; i < nf; ++i) h[(size_t)kind * nf + i].hyb = G2.halo;
      }
    }
  }
  std::vector<SweepField> h2(h);  // the stencil launches' descriptors
  for (int kind = 0; kind < 3; ++kind)
    if (plan->hyb[kind])
      for (int i = 0; i < nf; ++i) h2[(size_t)kind * nf + i].halo_f = plan->geom2[kind].halo;
  plan->nf = nf;
  plan->pp = nf > 0 && fields[0].B != nullptr;
  // filter sub-steps: one per-line stencil table per kind, shared by the
  // plan's fields (same grid and sub-step; the velocity fields of the filter
  // kernel do not depend on time)
  int lines[3] = {0, 0, 0};
  bool any_hyb = false;
  for (int kind = 0; kind < 3 && nf > 0; ++kind) {
    if (!stencil_filter_variant(plan->geom[kind].variant) && !plan->hyb[kind]) continue;
    any_hyb = any_hyb || plan->hyb[kind];
    lines[kind] = h[(size_t)kind * nf].groups * LPG;
    CK(plan->wt[kind].alloc((fp64 ? 8 : 4) * (plan->wide[kind] ? 16 : 8) * (size_t)lines[kind]));
    CK(plan->nt[kind].alloc(sizeof(int) * (size_t)lines[kind]));
    for (int i = 0; i < nf; ++i) {
      for (std::vector<SweepField> *hv : {&h, &h2}) {
        (*hv)[(size_t)kind * nf + i].wt = plan->wt[kind].p;
        (*hv)[(size_t)kind * nf + i].nt = plan->nt[kind].as<int>();
      }
    }
  }
  CK(plan->fields.alloc(sizeof(SweepField) * h.size()));
  CK(cudaMemcpy(plan->fields.p, h.data(), sizeof(SweepField) * h.size(), cudaMemcpyHostToDevice));
  if (any_hyb) {
    CK(plan->fields2.alloc(sizeof(SweepField) * h2.size()));
    CK(cudaMemcpy(plan->fields2.p, h2.data(), sizeof(SweepField) * h2.size(),
                  cudaMemcpyHostToDevice));
  }
  for (int kind = 0; kind < 3; ++kind)
    if (lines[kind])
      CK(launch_filter_weights(fp64,
                               (plan->hyb[kind] ? plan->fields2 : plan->fields).as<SweepField>() +
                                   (size_t)kind * nf,
                               plan->wt[kind].p, plan->nt[kind].as<int>(), lines[kind], 0,
                               plan->wide[kind]));
  CK(cudaStreamSynchronize(0));
  return CCFV_OK;
}

int run_step_plan(ccfv_ctx *ctx, const StepPlan &plan, bool fp64, int first, int count,
                  double toff, void *data_override, cudaStream_t st, int jstep) {
  const SweepField *base = plan.fields.as<SweepField>();
  unsigned *status = ctx->status.as<unsigned>();
  for (int kind = 0; kind < 3; ++kind) {
    const LaunchGeom &G = plan.geom[kind];
    const int gpf = plan.groups_per_field[kind];
    const SweepField *fk = base + (size_t)kind * plan.nf;
    cudaError_t e =
        fp64 ? launch_sweep<double>(G.variant, fk, plan.nf, first * gpf, count * gpf, G.cs,
                                    G.lc_max, G.halo, toff, data_override, status, st, jstep,
                                    !plan.pp)
             : launch_sweep<float>(G.variant, fk, plan.nf, first * gpf, count * gpf, G.cs,
                                   G.lc_max, G.halo, toff, data_override, status, st, jstep,
                                   !plan.pp);
    CK(e);
    if (plan.hyb[kind]) {  // the interior segments of compat lines: stencil form
      const LaunchGeom &G2 = plan.geom2[kind];
      const SweepField *f2 = plan.fields2.as<SweepField>() + (size_t)kind * plan.nf;
      e = fp64 ? launch_sweep<double>(G2.variant, f2, plan.nf, first * gpf, count * gpf, G2.cs,
                                      G2.lc_max, G2.halo, toff, data_override, status, st, jstep,
                                      !plan.pp)
               : launch_sweep<float>(G2.variant, f2, plan.nf, first * gpf, count * gpf, G2.cs,
                                     G2.lc_max, G2.halo, toff, data_override, status, st, jstep,
                                     !plan.pp);
      CK(e);
    }
  }
  return CCFV_OK;
}

// Plan of one field for the single-field calls: an out-of-place sequence
// between the caller's field (passed per launch) and a context scratch field.
static StepPlan *single_plan(ccfv_ctx *ctx, double dt, bool fp64, int *status, double theta) {
  auto key = std::make_tuple(dt, fp64 ? 1 : 0, 0, theta);
  auto it = ctx->step_plans.find(key);
  if (it != ctx->step_plans.end()) return it->second.get();
  const size_t el = fp64 ? sizeof(double) : sizeof(float);
  DevBuf &scratch = fp64 ? ctx->pp64 : ctx->pp32;
  const size_t bytes = el * (size_t)ctx->grid.nx * ctx->grid.ny;
  if (!scratch.p) {
    cudaError_t e = scratch.alloc(bytes);
    if (e != cudaSuccess) {
      *status = set_error(ctx, CCFV_ERR_NOMEM, cudaGetErrorString(e));
      return nullptr;
    }
  }
  auto plan = std::make_unique<StepPlan>();
  std::vector<PlanField> f(1);
  f[0].B = scratch.p;  // A and in0: the caller's field (launch override)
  int st = build_step_plan(ctx, plan.get(), dt, fp64, f, false, theta);
  if (st != CCFV_OK) {
    *status = st;
    return nullptr;
  }
  StepPlan *res = plan.get();
  ctx->step_plans[key] = std::move(plan);
  return res;
}

// nsteps split steps on one field: 3 nsteps sweeps alternating between the
// field and the scratch field; an odd count ends in the scratch field and is
// copied back.
int steps(ccfv_ctx *ctx, void *d_C, bool fp64, double t0, double dt, int nsteps, cudaStream_t st,
          double theta) {
  int status = CCFV_OK;
  StepPlan *plan = single_plan(ctx, dt, fp64, &status, theta);
  if (!plan) return status;
  for (int n = 0; n < nsteps; ++n) {
    int rc = run_step_plan(ctx, *plan, fp64, 0, 1, t0 + n * dt, d_C, st, n);
    if (rc) return rc;
  }
  if ((3 * nsteps) & 1) {
    const size_t el = fp64 ? sizeof(double) : sizeof(float);
    CK(cudaMemcpyAsync(d_C, (fp64 ? ctx->pp64 : ctx->pp32).p,
                       el * (size_t)ctx->grid.nx * ctx->grid.ny, cudaMemcpyDeviceToDevice, st));
  }
  return CCFV_OK;
}

// ---------------------------------------------------------------------------
// Element-wise kernels: precision conversion and the fused Parareal correction.

template <typename S, typename D>
__global__ void convert_kernel(const S *__restrict__ src, D *__restrict__ dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = (D)src[i];
}

constexpr int RED_THREADS = 256;
constexpr int RED_BLOCKS = 592;  // 4 x 148 SMs

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// U+[n+1] = G + (F - Gold)  (STANDARD; parareal_correction_kernel, T2S4:771-782)
// U+[n+1] = F + G(e)        (DELTA)
// fused with the update norms sum (U+ - U)^2 and sum U+^2, reduced
// deterministically (fixed-order block partials, last block finishes).
// STANDARD stores G into Gold; DELTA stores the new increment into Wd.  G is
// read from Wg (the buffer the coarse sweep sequence ended in; Wg may be Wd).
template <typename TG>
__global__ void __launch_bounds__(RED_THREADS)
    correction_kernel(int form, long long n, double *__restrict__ U, const double *__restrict__ Fv,
                      double *__restrict__ Gold, const TG *Wg, TG *Wd,
                      double *__restrict__ partial, unsigned *__restrict__ counter,
                      double *__restrict__ out) {
  double se = 0.0, su = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double uo = U[i];
    const double gw = (double)Wg[i];
    double un;
    if (form == CCFV_FORM_STANDARD) {
      un = gw + (Fv[i] - Gold[i]);
      Gold[i] = gw;
    } else {
      un = Fv[i] + gw;
    }
    const double d = un - uo;
    U[i] = un;
    if (form != CCFV_FORM_STANDARD) Wd[i] = (TG)d;
    se += d * d;
    su += un * un;
  }
  __shared__ double red[2][RED_THREADS / 32];
  __shared__ bool last;
  se = warp_sum(se);
  su = warp_sum(su);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { red[0][w] = se; red[1][w] = su; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int k = 0; k < RED_THREADS / 32; ++k) { a += red[0][k]; b += red[1][k]; }
    partial[2 * blockIdx.x] = a;
    partial[2 * blockIdx.x + 1] = b;
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double a = 0, b = 0;
    for (unsigned k = 0; k < gridDim.x; ++k) {
      a += ((volatile double *)partial)[2 * k];
      b += ((volatile double *)partial)[2 * k + 1];
    }
    out[0] = a;
    out[1] = b;
    *counter = 0;
  }
}

static int grid_for(long long n) {
  long long b = (n + RED_THREADS - 1) / RED_THREADS;
  return (int)std::max(1LL, std::min<long long>(b, RED_BLOCKS));
}

template <typename S, typename D>
static int convert(ccfv_ctx *ctx, const S *src, D *dst, long long n, cudaStream_t st) {
  count_launch();
  convert_kernel<S, D><<<grid_for(n), RED_THREADS, 0, st>>>(src, dst, n);
  CK(cudaGetLastError());
  return CCFV_OK;
}

template <typename TG>
static int correction(ccfv_ctx *ctx, int form, long long n, double *U, const double *Fv,
                      double *Gold, const TG *Wg, TG *Wd, double *out, cudaStream_t st) {
  count_launch();
  correction_kernel<TG><<<grid_for(n), RED_THREADS, 0, st>>>(
      form, n, U, Fv, Gold, Wg, Wd, ctx->partial.as<double>(), ctx->counter.as<unsigned>(), out);
  CK(cudaGetLastError());
  return CCFV_OK;
}

// ---------------------------------------------------------------------------
// Parareal (T2S4_Parareal.cu:1249-1355, generalised).
//
// Slice states U[0..S], fine results F[1..S] (F[n+1] = F(U[n])), coarse work
// field W in the coarse precision.  Iteration k (1-based) leaves slices
// n < k exact, so only slices n >= k-1 are propagated and corrected.
//   F-phase: all active slices advance J fine steps together, one launch per
//            sweep over every slice (3 J launches).
//   G-phase: sequential over slices, m coarse steps of the single field W,
//            then the fused correction + norm kernel.

template <typename TG>
static int parareal_impl(ccfv_ctx *ctx, const ccfv_parareal_opts *o, const double *C0,
                         double *C_T, ccfv_stats *stats, cudaStream_t st) {
  const ccfv_grid &g = ctx->grid;
  const bool g64 = sizeof(TG) == 8;
  const long long NN = (long long)g.nx * g.ny;
  const int S = o->n_slices;
  const int J = o->nt_fine / S;
  const int m = o->coarse_ratio > 0 ? J / o->coarse_ratio : 1;
  const double DT = (o->t1 - o->t0) / S;
  const double dt = DT / (double)J;  // FinePropagator: dt = DT / J (T2S4:979)
  const double dtc = DT / (double)m;
  const size_t fb = sizeof(double) * NN;

  CK(ctx->U.alloc(fb * (S + 1)));
  CK(ctx->F.alloc(fb * (S + 1)));
  if (o->form == CCFV_FORM_STANDARD) CK(ctx->Gold.alloc(fb * (S + 1)));
  CK(ctx->FS.alloc(fb * S));
  CK(ctx->W.alloc(sizeof(TG) * NN));
  CK(ctx->W2.alloc(sizeof(TG) * NN));
  CK(ctx->norms.alloc(sizeof(double) * 2 * (S + 1)));
  double *U = ctx->U.as<double>(), *F = ctx->F.as<double>(), *FS = ctx->FS.as<double>();
  double *Gold = o->form == CCFV_FORM_STANDARD ? ctx->Gold.as<double>() : nullptr;
  TG *W = ctx->W.as<TG>(), *W2 = ctx->W2.as<TG>();
  double *norms = ctx->norms.as<double>();

  // Fine plan over all slices, out of place: slice n's J steps run from U[n]
  // through the pair F[n+1] / FS[n] and end in F[n+1] (no copy U -> F, no
  // CTA reads what another CTA of its launch writes); time origin t0 + n DT.
  const double key[4] = {dt, o->t0, DT, (double)S};
  const void *bufs[3] = {U, F, FS};
  if (!ctx->fine_plan || std::memcmp(key, ctx->fine_plan_key, sizeof(key)) != 0 ||
      ctx->fine_plan_slices != S || std::memcmp(bufs, ctx->fine_plan_bufs, sizeof(bufs)) != 0) {
    auto plan = std::make_unique<StepPlan>();
    std::vector<PlanField> fl(S);
    for (int n = 0; n < S; ++n) {
      fl[n].A = F + (size_t)(n + 1) * NN;
      fl[n].t0 = o->t0 + n * DT;
      fl[n].B = FS + (size_t)n * NN;
      fl[n].in0 = U + (size_t)n * NN;
      fl[n].par = pp_parity(J);
    }
    int rc = build_step_plan(ctx, plan.get(), dt, true, fl);
    if (rc) return rc;
    ctx->fine_plan = std::move(plan);
    std::memcpy(ctx->fine_plan_key, key, sizeof(key));
    std::memcpy(ctx->fine_plan_bufs, bufs, sizeof(bufs));
    ctx->fine_plan_slices = S;
  }
  // The first coarse sweep moves whole states and always runs in FP64: FP32
  // rounding there would seed every wavenumber at ~1e-7 |U|, and Parareal
  // amplifies the high-wavenumber error modes of advection (and of
  // Crank-Nicolson coarse steps with K Dt/h^2 >> 1) from one iteration to the
  // next.  In the iterations FP32 rounding is relative to the increments.
  // Coarse sweeps of the iterations: m steps out of place over W / W2,
  // starting from W; the result is in W2 when 3m is odd.  The delta form
  // propagates increments: the linear part of G (no source).
  // Every coarse step (first sweep included) uses the run's coarse diffusion
  // weight, so the standard form's cached G(U_k) is the iterations' G.
  const double th = coarse_theta(*o, g, dtc);
  StepPlan cplan, hplan;
  {
    std::vector<PlanField> f(1);
    f[0].A = W;
    f[0].B = W2;
    f[0].in0 = W;
    int rc = build_step_plan(ctx, &cplan, dtc, g64, f, false, th);
    if (!rc && o->form == CCFV_FORM_DELTA && g.source != CCFV_SRC_NONE)
      rc = build_step_plan(ctx, &hplan, dtc, g64, f, true, th);
    if (rc) return rc;
  }
  const StepPlan *dplan =
      (o->form == CCFV_FORM_DELTA && g.source != CCFV_SRC_NONE) ? &hplan : &cplan;
  const TG *Wres = ((3 * m) & 1) ? W2 : W;

  cudaEvent_t ev0, ev1;
  CK(cudaEventCreate(&ev0));
  CK(cudaEventCreate(&ev1));
  CK(cudaEventRecord(ev0, st));
  const cudaMemcpyKind k_in = o->mem == CCFV_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  CK(cudaMemcpyAsync(U, C0, fb, k_in, st));

  auto coarse_on_W = [&](int n, const StepPlan *plan) -> int {
    for (int i = 0; i < m; ++i) {
      int rc = run_step_plan(ctx, *plan, g64, 0, 1, o->t0 + n * DT + i * dtc, nullptr, st, i);
      if (rc) return rc;
    }
    return CCFV_OK;
  };

  // k = 0: coarse sweep U[n+1] = G(U[n])  (T2S4:1271-1280), FP64
  for (int n = 0; n < S; ++n) {
    double *un1 = U + (size_t)(n + 1) * NN;
    CK(cudaMemcpyAsync(un1, U + (size_t)n * NN, fb, cudaMemcpyDeviceToDevice, st));
    int rc = steps(ctx, un1, true, o->t0 + n * DT, dtc, m, st, th);
    if (rc) return rc;
    if (Gold) CK(cudaMemcpyAsync(Gold + (size_t)(n + 1) * NN, un1, fb, cudaMemcpyDeviceToDevice, st));
  }

  std::vector<double> hn(2 * (size_t)(S + 1));
  int iters = 0, converged = 0;
  double fine_cu = 0, coarse_cu = (double)S * m * NN;
  double fine_ms = 0, coarse_ms = 0;
  long long fine_launches = 0, fine_cells = 0;
  cudaEvent_t fa, fb_, gb;
  CK(cudaEventCreate(&fa));
  CK(cudaEventCreate(&fb_));
  CK(cudaEventCreate(&gb));
  for (int k = 1; k <= o->kmax; ++k) {
    const int nlo = k - 1;
    const int act = S - nlo;
    // F-phase: F[n+1] = F(U[n]) for every active slice, out of place
    CK(cudaEventRecord(fa, st));
    for (int j = 0; j < J; ++j) {
      int rc = run_step_plan(ctx, *ctx->fine_plan, true, nlo, act, j * dt, nullptr, st, j);
      if (rc) return rc;
    }
    CK(cudaEventRecord(fb_, st));
    fine_cu += (double)act * J * NN;
    fine_launches += 3LL * J;
    fine_cells += 3LL * J * act * NN;
    // G-phase + correction
    CK(cudaMemsetAsync(norms, 0, sizeof(double) * 2 * (S + 1), st));
    for (int n = nlo; n < S; ++n) {
      int rc;
      const TG *Gn = Wres;  // where this slice's G value ends up
      if (o->form == CCFV_FORM_STANDARD) {
        CK(cudaMemcpyAsync(W, U + (size_t)n * NN, fb, cudaMemcpyDeviceToDevice, st));
        if ((rc = coarse_on_W(n, &cplan))) return rc;
        coarse_cu += (double)m * NN;
      } else if (n == nlo) {
        CK(cudaMemsetAsync(W, 0, sizeof(TG) * NN, st));  // G(0) = 0
        Gn = W;
      } else {
        if ((rc = coarse_on_W(n, dplan))) return rc;
        coarse_cu += (double)m * NN;
      }
      if ((rc = correction<TG>(ctx, o->form, NN, U + (size_t)(n + 1) * NN,
                               F + (size_t)(n + 1) * NN,
                               Gold ? Gold + (size_t)(n + 1) * NN : nullptr, Gn, W,
                               norms + 2 * (n + 1), st)))
        return rc;
    }
    CK(cudaEventRecord(gb, st));
    if (o->d_ref && stats && k - 1 < CCFV_MAX_ITERS) {
      int rc = ccfv::norms(ctx, U + (size_t)S * NN, o->d_ref, &stats->err_l2[k - 1],
                           &stats->err_max[k - 1], st);
      if (rc) return rc;
    }
    CK(cudaMemcpyAsync(hn.data(), norms, sizeof(double) * 2 * (S + 1), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    {
      float a = 0, b = 0;
      cudaEventElapsedTime(&a, fa, fb_);
      cudaEventElapsedTime(&b, fb_, gb);
      fine_ms += a;
      coarse_ms += b;
    }
    double worst = 0.0;
    for (int n = nlo + 1; n <= S; ++n) {
      double e = std::sqrt(hn[2 * n]), u = std::sqrt(hn[2 * n + 1]);
      double r = u > 0 ? e / u : e;
      worst = std::max(worst, r);
    }
    iters = k;
    if (stats && k - 1 < CCFV_MAX_ITERS) stats->update[k - 1] = worst;
    if (o->tol > 0 && worst < o->tol) {
      converged = 1;
      break;
    }
  }
  const cudaMemcpyKind k_out = o->mem == CCFV_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  CK(cudaMemcpyAsync(C_T, U + (size_t)S * NN, fb, k_out, st));
  CK(cudaEventRecord(ev1, st));
  CK(cudaStreamSynchronize(st));
  float ms = 0;
  cudaEventElapsedTime(&ms, ev0, ev1);
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  cudaEventDestroy(fa);
  cudaEventDestroy(fb_);
  cudaEventDestroy(gb);
  if (stats) {
    stats->fine_ms = fine_ms;
    stats->coarse_ms = coarse_ms;
    stats->fine_sweep_launches = fine_launches;
    stats->fine_sweep_cells = fine_cells;
    stats->iterations = iters;
    stats->converged = converged;
    stats->fine_cell_updates = fine_cu;
    stats->coarse_cell_updates = coarse_cu;
    stats->ms = ms;
  }
  return CCFV_OK;
}

int parareal(ccfv_ctx *ctx, const ccfv_parareal_opts *o, const double *C0, double *C_T,
             ccfv_stats *stats, cudaStream_t st) {
  if (!o || !C0 || !C_T) return set_error(ctx, CCFV_ERR_INVALID, "null argument");
  if (o->n_slices < 1 || o->nt_fine < o->n_slices || o->nt_fine % o->n_slices)
    return set_error(ctx, CCFV_ERR_INVALID, "nt_fine must be a positive multiple of n_slices");
  const int J = o->nt_fine / o->n_slices;
  if (o->coarse_ratio < 0 || (o->coarse_ratio > 0 && J % o->coarse_ratio))
    return set_error(ctx, CCFV_ERR_INVALID, "coarse_ratio must divide nt_fine / n_slices");
  if (o->kmax < 1 || o->kmax > CCFV_MAX_ITERS)
    return set_error(ctx, CCFV_ERR_INVALID, "kmax out of range");
  if (o->form != CCFV_FORM_STANDARD && o->form != CCFV_FORM_DELTA)
    return set_error(ctx, CCFV_ERR_INVALID, "unknown Parareal form");
  if (o->coarse_precision == CCFV_FP32 && o->form != CCFV_FORM_DELTA)
    return set_error(ctx, CCFV_ERR_INVALID, "an FP32 coarse propagator needs the DELTA form");
  if (!coarse_theta_ok(o->coarse_theta))
    return set_error(ctx, CCFV_ERR_INVALID,
                     "coarse_theta must be 0 (Crank-Nicolson), in [0.5, 1] or CCFV_COARSE_THETA_AUTO");
  if (stats) std::memset(stats, 0, sizeof(*stats));
  int rc = o->coarse_precision == CCFV_FP32 ? parareal_impl<float>(ctx, o, C0, C_T, stats, st)
                                            : parareal_impl<double>(ctx, o, C0, C_T, stats, st);
  if (rc) return rc;
  unsigned flag = 0;
  CK(cudaMemcpy(&flag, ctx->status.p, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (flag) {
    CK(cudaMemset(ctx->status.p, 0, sizeof(unsigned)));
    return set_error(ctx, CCFV_ERR_HALO, "a characteristic foot left the staged halo");
  }
  return CCFV_OK;
}

// F over n contiguous fields (field i starts at t0 + i * slice_dt): J steps of
// DT/J each, every field advancing in the same launches (the F phase).
int fine_slices(ccfv_ctx *ctx, double *d_fields, int n, double t0, double slice_dt, double DT,
                int J, cudaStream_t st) {
  const long long NN = (long long)ctx->grid.nx * ctx->grid.ny;
  const double dt = DT / (double)J;
  StepPlan plan;
  std::vector<std::pair<void *, double>> fl;
  for (int i = 0; i < n; ++i) fl.push_back({d_fields + (size_t)i * NN, t0 + i * slice_dt});
  int rc = build_step_plan(ctx, &plan, dt, true, fl);
  if (rc) return rc;
  for (int j = 0; j < J; ++j)
    if ((rc = run_step_plan(ctx, plan, true, 0, n, j * dt, nullptr, st))) return rc;
  CK(cudaStreamSynchronize(st));  // the plan's descriptors are released on return
  return CCFV_OK;
}

// Stand-alone Parareal correction of one slice with its update norms (the
// building block of the slice-distributed driver).
int correct(ccfv_ctx *ctx, int form, double *U, const double *Fv, double *Gold, double *W,
            double *sq_update, double *sq_state, cudaStream_t st) {
  const long long NN = (long long)ctx->grid.nx * ctx->grid.ny;
  double *out = ctx->aux.as<double>() + 8;
  int rc = correction<double>(ctx, form, NN, U, Fv, Gold, W, W, out, st);
  if (rc) return rc;
  double h[2];
  CK(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (sq_update) *sq_update = h[0];
  if (sq_state) *sq_state = h[1];
  return CCFV_OK;
}

int coarse_fp32(ccfv_ctx *ctx, double *d_C, double tn, double DT, int m, cudaStream_t st,
                double theta) {
  const long long NN = (long long)ctx->grid.nx * ctx->grid.ny;
  CK(ctx->C32.alloc(sizeof(float) * NN));
  float *w = ctx->C32.as<float>();
  int rc = convert(ctx, d_C, w, NN, st);
  if (rc) return rc;
  const double dtc = DT / (double)m;
  if ((rc = steps(ctx, w, false, tn, dtc, m, st, theta))) return rc;
  return convert(ctx, w, d_C, NN, st);
}

}  // namespace ccfv
