// noalloc.cu -- one split step for callers that cannot allocate memory.
//
// Some callers of this solver cannot call cudaMalloc: code that runs inside
// another framework's memory pool or allocator hook, long-running services
// that forbid allocation after start-up, or hosts that budget every byte of
// device memory up front.  ccfv_step_noalloc performs the same split step as
// ccfv_step without creating a context: the sweep kernels' scratch (three
// sweep descriptors, the line-invariant solver factors of the x and y
// systems and the status word) lives in the file-scope device array below,
// and the host-side staging buffers are file-scope static arrays, so the call
// allocates nothing on the device or on the host heap.
//
// Limits and rules (also stated in include/ccfv.h):
//  - nx, ny <= NOALLOC_MAX_LINE (4096); larger grids are rejected with
//    CCFV_ERR_UNSUPPORTED before any device work.
//  - Every GPU that loads this library holds the array (about 340 KB) until
//    the process exits.
//  - The first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture.  The address is cached per device ordinal:
//    after cudaDeviceReset of a device the module is reloaded and the cached
//    address is stale, so the call must not be used on that device again.
//  - A foot that left the staged halo is returned as CCFV_ERR_HALO (the
//    context path leaves it in the status word for ccfv_check); the field has
//    been updated, with the out-of-halo reads taken as zero, when it is.
//  - All calls share the array, which keeps the last call's contents: calls
//    that overlap on the GPU (different streams, or host threads) race.  The
//    call synchronises its stream before returning.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "engine.h"

namespace ccfv {
namespace {

constexpr int NOALLOC_MAX_LINE = 4096;
constexpr size_t NOALLOC_HDR = 2048;  // status word + 3 sweep descriptors
// solver table of one direction (layout of table_len(): factors, chunk products)
constexpr size_t NOALLOC_TAB_LEN =
    5 * (size_t)NOALLOC_MAX_LINE + (size_t)MAX_CLUSTER * NCH + (size_t)MAX_CLUSTER * (NCH + 1);
constexpr size_t NOALLOC_TAB = NOALLOC_TAB_LEN * sizeof(double);
constexpr size_t NOALLOC_BYTES = NOALLOC_HDR + 2 * NOALLOC_TAB;
static_assert(sizeof(SweepField) * 3 + 256 <= NOALLOC_HDR, "descriptor area too small");

// Device scratch of ccfv_step_noalloc (layout: status | descriptors | x table | y table).
__device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

// Host staging (static, never heap-allocated).
double h_tab[2][NOALLOC_TAB_LEN];
SweepField h_fields[3];

void *g_dev_ptr[MAX_DEVICES] = {};
std::mutex g_mu;

// LU factors of the constant tridiagonal system, the same arithmetic as the
// context path (engine.cu build_table) without heap temporaries.
void table_static(int L, double coA, double coB, int bc, double *out, double *sm_fac,
                  double *sm_inv_den) {
  const double coC = coA, gam = -coB;
  auto diag = [&](int k) {
    if (bc == BC_PERIODIC && k == 0) return coB - gam;
    if (bc == BC_PERIODIC && k == L - 1) return coB - coA * coC / gam;
    return coB;
  };
  double pprev = 0.0;
  for (int k = 0; k < L; ++k) {
    const double d = diag(k);
    const double g = k == 0 ? 1.0 / d : 1.0 / (d - pprev * coA);
    pprev = k == 0 ? coC / d : coC * g;
    out[k] = -coA * g;
    out[L + k] = g;
  }
  *sm_fac = 0.0;
  *sm_inv_den = 0.0;
  if (bc == BC_PERIODIC) {
    double *z = out + 2 * (size_t)L;
    double q = 0.0;
    for (int k = 0; k < L; ++k) {
      const double u = (k == 0) ? gam : (k == L - 1 ? coC : 0.0);
      q = out[L + k] * u + (k ? out[k] * q : 0.0);
      z[k] = q;
    }
    for (int k = L - 2; k >= 0; --k) {
      const double p = k == 0 ? coC / diag(0) : coC * out[L + k];
      z[k] = z[k] - p * z[k + 1];
    }
    *sm_fac = coA / gam;
    *sm_inv_den = 1.0 / (1.0 + z[0] + *sm_fac * z[L - 1]);
  }
  fill_chunk_products(L, out);
}

int shift_of(const ccfv_grid &g, int dir, double Dt) {
  const double *p = g.vel_params;
  double w = 0.0;
  switch (g.velocity) {
    case CCFV_VEL_REF_ROT4:
      w = dir == 0 ? 4 * std::max(std::fabs(g.y_min), std::fabs(g.y_max))
                   : 4 * std::max(std::fabs(g.x_min), std::fabs(g.x_max));
      break;
    case CCFV_VEL_CONST: w = std::fabs(dir == 0 ? p[0] : p[1]); break;
    case CCFV_VEL_ROTATION:
      w = dir == 0 ? std::fabs(p[0]) * std::max(std::fabs(g.y_min - p[2]), std::fabs(g.y_max - p[2]))
                   : std::fabs(p[0]) * std::max(std::fabs(g.x_min - p[1]), std::fabs(g.x_max - p[1]));
      break;
    case CCFV_VEL_SWIRL: w = 1.0; break;
  }
  const double h = dir == 0 ? (g.x_max - g.x_min) / g.nx : (g.y_max - g.y_min) / g.ny;
  return (int)std::ceil(std::fabs(Dt) * w / h + 1e-9);
}

bool grid_valid(const ccfv_grid *g) {
  return g && g->nx >= 4 && g->ny >= 4 && g->x_max > g->x_min && g->y_max > g->y_min &&
         (g->bc == CCFV_BC_COMPAT || g->bc == CCFV_BC_PERIODIC) &&
         g->velocity >= CCFV_VEL_REF_ROT4 && g->velocity <= CCFV_VEL_SWIRL &&
         !(g->velocity == CCFV_VEL_SWIRL && g->vel_params[0] == 0.0) &&
         (g->scheme == CCFV_SCHEME_REFERENCE || g->scheme == CCFV_SCHEME_CONSISTENT) &&
         g->K >= 0.0 &&
         (g->source == CCFV_SRC_NONE ||
          (g->source == CCFV_SRC_GAUSSIAN && g->source_params[3] > 0.0));
}

}  // namespace
}  // namespace ccfv

using namespace ccfv;

extern "C" int ccfv_step_noalloc(const ccfv_grid *grid, double *d_C, double tn, double dt,
                                 void *stream) {
  if (!grid_valid(grid) || !d_C || !(dt > 0.0)) return CCFV_ERR_INVALID;
  const ccfv_grid &g = *grid;
  if (g.nx > NOALLOC_MAX_LINE || g.ny > NOALLOC_MAX_LINE) return CCFV_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_mu);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return CCFV_ERR_CUDA;
  if (!g_dev_ptr[dev]) {
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr)
      return CCFV_ERR_CUDA;
    g_dev_ptr[dev] = ptr;
  }
  unsigned char *base = static_cast<unsigned char *>(g_dev_ptr[dev]);
  unsigned *d_status = reinterpret_cast<unsigned *>(base);
  SweepField *d_fields = reinterpret_cast<SweepField *>(base + 256);
  double *d_tab[2] = {reinterpret_cast<double *>(base + NOALLOC_HDR),
                      reinterpret_cast<double *>(base + NOALLOC_HDR + NOALLOC_TAB)};
  cudaStream_t st = (cudaStream_t)stream;

  // solver factors and sweep descriptors of x(dt/2), y(dt), x(dt/2)
  LaunchGeom geom[3];
  for (int kind = 0; kind < 3; ++kind) {
    const int dir = kind == 1 ? 1 : 0;
    const double Dt = kind == 1 ? dt : 0.5 * dt;
    const double ta = kind == 2 ? 0.5 * dt : 0.0;
    const double tb = kind == 0 ? 0.5 * dt : dt;
    const int L = dir == 0 ? g.nx : g.ny;
    const double h = dir == 0 ? (g.x_max - g.x_min) / g.nx : (g.y_max - g.y_min) / g.ny;
    const double r2 = Dt / (h * h);
    double sm_fac = 0, sm_inv = 0;
    if (kind < 2)
      table_static(L, 1.0 / 12 - 0.5 * g.K * r2, 10.0 / 12 + g.K * r2, g.bc, h_tab[dir], &sm_fac,
                   &sm_inv);
    else {
      sm_fac = h_fields[0].sm_fac;
      sm_inv = h_fields[0].sm_inv_den;
    }
    const int dsrc = (kind == 2 && g.scheme == CCFV_SCHEME_REFERENCE) ? 1 : 0;
    SolverTable view;  // borrowed pointer: released before the view goes out of scope
    view.buf.p = d_tab[dir];
    view.sm_fac = sm_fac;
    view.sm_inv_den = sm_inv;
    h_fields[kind] = make_field(g, dir, Dt, ta, tb, d_C, &view, dsrc);
    view.buf.p = nullptr;
    h_fields[kind].group0 = 0;
    h_fields[kind].src_tb = kind == 2 ? 1 : 0;
    LaunchGeom &G = geom[kind];
    G.cs = (L + LC_MAX - 1) / LC_MAX;
    G.lc_max = (L + G.cs - 1) / G.cs;
    const int sh = shift_of(g, dir, Dt);
    G.halo = dsrc ? (sh + 4) + sh + 5 : sh + 5;
    const bool uniform = g.velocity == CCFV_VEL_REF_ROT4 || g.velocity == CCFV_VEL_CONST ||
                         g.velocity == CCFV_VEL_ROTATION;
    G.variant = g.source ? SWEEP_GENERAL_SRC
                : (uniform && g.bc == CCFV_BC_PERIODIC && dsrc == 0) ? SWEEP_FAST : SWEEP_GENERAL;
    h_fields[kind].cta0 = 0;
    h_fields[kind].halo_f = G.halo;
    if (std::max(sweep_smem_bytes(G.lc_max, G.halo, true, g.source != 0),
                 sweep_fast_smem_bytes(G.lc_max, G.halo, true)) > 227 * 1024)
      return CCFV_ERR_UNSUPPORTED;
  }
  cudaError_t e = cudaMemsetAsync(d_status, 0, sizeof(unsigned), st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_tab[0], h_tab[0], sizeof(double) * table_len(g.nx),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_tab[1], h_tab[1], sizeof(double) * table_len(g.ny),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_fields, h_fields, sizeof(h_fields), cudaMemcpyHostToDevice, st);
  for (int kind = 0; kind < 3 && e == cudaSuccess; ++kind) {
    const LaunchGeom &G = geom[kind];
    e = launch_sweep<double>(G.variant, d_fields + kind, 1, 0, h_fields[kind].groups, G.cs,
                             G.lc_max, G.halo, tn, nullptr, d_status, st);
  }
  unsigned flag = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&flag, d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? CCFV_ERR_NOMEM : CCFV_ERR_CUDA;
  return flag ? CCFV_ERR_HALO : CCFV_OK;
}
