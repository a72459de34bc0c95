// engine.h -- host-side solver context, plans and Parareal engine of libccfv.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/ccfv.h"
#include "ccfv_internal.h"

namespace ccfv {

// Device memory owned by the library; freed on destruction.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t b);
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T> T *as() const { return reinterpret_cast<T *>(p); }
};

// Line-invariant LU factors of one constant tridiagonal system (device, T[3L]).
struct SolverTable {
  DevBuf buf;
  double sm_fac = 0, sm_inv_den = 0;
};

// Launch geometry shared by all fields of one sweep launch.
struct LaunchGeom {
  int cs = 1, lc_max = 0, halo = 0, groups = 0, variant = 0;
};

// Three sweep launches (x dt/2, y dt, x dt/2) of one step over a set of fields.
struct StepPlan {
  DevBuf fields;          // SweepField[3][nf]
  int nf = 0;
  int groups_per_field[3] = {0, 0, 0};
  LaunchGeom geom[3];
  bool pp = false;        // out-of-place sequence (SweepField::pp)
  DevBuf wt[3], nt[3];    // filter kernel: per-line stencil tables per sub-step kind
  // compat lines split between two launches (SweepField::hyb): the second
  // launch's descriptors (stencil form) and geometry per sub-step kind
  DevBuf fields2;         // SweepField[3][nf]
  LaunchGeom geom2[3];
  bool hyb[3] = {false, false, false};
  bool wide[3] = {false, false, false};  // the stencil launch is the 13-tap form
};

// One field of a plan: swept in place on A (B == nullptr), or an out-of-place
// sequence of steps over the pair A/B that starts from in0 and, with parity
// offset par, ends in A (SweepField::pp).  t0: the field's time origin.
struct PlanField {
  void *A = nullptr;
  double t0 = 0.0;
  void *B = nullptr;
  const void *in0 = nullptr;
  int par = 0;
};
// Parity offset that makes a sequence of `steps` split steps (3 sweeps each)
// end in buffer A.
inline int pp_parity(int steps) { return (3 * steps) & 1; }

}  // namespace ccfv

struct ccfv_ctx {
  ccfv_grid grid;
  int device = 0;
  ccfv::DevBuf status;  // unsigned status word + partial-sum scratch
  // keyed by (dir, sub-step, FP64, diffusion theta) / (dt, FP64, 0, theta)
  std::map<std::tuple<int, double, int, double>, std::unique_ptr<ccfv::SolverTable>> tables;
  std::map<std::tuple<double, int, int, double>, std::unique_ptr<ccfv::StepPlan>> step_plans;
  // Parareal slice states and scratch
  ccfv::DevBuf U, F, Gold, W, C64, C32, norms, partial, counter, io, aux;
  ccfv::DevBuf FS, W2;  // ping-pong partners of the fine slices and the coarse work field
  ccfv::DevBuf pp64, pp32;  // ping-pong partner of single-field calls (FP64, FP32)
  size_t slices_cap = 0;
  std::unique_ptr<ccfv::StepPlan> fine_plan;
  double fine_plan_key[4] = {0, 0, 0, 0};
  const void *fine_plan_bufs[3] = {nullptr, nullptr, nullptr};
  int fine_plan_slices = 0;
  std::string last_error;
  bool force_general = false;  // test hook: route every sweep through the per-cell kernel
};

namespace ccfv {

int set_error(ccfv_ctx *ctx, int code, const std::string &msg);
// `theta` is the implicit weight of the diffusion sub-step: 0.5 is the
// reference's Crank-Nicolson; 1 is backward Euler (L-stable), which the
// coarse propagator may use (ccfv_parareal_opts::coarse_theta).
const SolverTable *get_table(ccfv_ctx *ctx, int dir, double Dt, bool fp64, int *status,
                             double theta = 0.5);
SweepField make_field(const ccfv_grid &g, int dir, double Dt, double ta_rel, double tb_rel,
                      void *data, const SolverTable *tab, int dsrc, double theta = 0.5);
// inplace: the sweep overwrites its input (the filter kernel's segments of a
// line then form one cluster, at most MAX_CLUSTER CTAs).
LaunchGeom step_geom(const ccfv_grid &g, int dir, double Dt, int dsrc, bool fp64,
                     bool inplace = true, double theta = 0.5);
// Diffusion weight of a Parareal run's coarse propagator of step dtc
// (ccfv_parareal_opts::coarse_theta; 0 selects 0.5).
double coarse_theta(const ccfv_parareal_opts &o, const ccfv_grid &g, double dtc);
// Whether coarse_theta holds an accepted value.
inline bool coarse_theta_ok(double th) {
  return th == 0.0 || th == CCFV_COARSE_THETA_AUTO || (th >= 0.5 && th <= 1.0);
}
void filter_field(const ccfv_grid &g, SweepField &f, bool fp64);
// for_class: keep the choice for the line-length classes of this grid (the
// batched engine) instead of its exact line lengths (ccfv_autotune).
int autotune(ccfv_ctx *ctx, double dt, bool fp64, cudaStream_t st, int *chosen,
             bool for_class = false);
// Whether the line-length class of L has a tuned segment length.
bool class_tuned(int L, bool fp64);
// The next power of two >= L (at least 64): the batched engine's tuning class.
int line_class(int L);
int batch_solve(int n, const ccfv_problem *probs, ccfv_stats *stats, int device,
                cudaStream_t st, std::string *errmsg);
// homogeneous: the source term is left out (the linear part of the step,
// which the delta form of Parareal applies to slice increments).
int build_step_plan(ccfv_ctx *ctx, StepPlan *plan, double dt, bool fp64,
                    const std::vector<std::pair<void *, double>> &fields,
                    bool homogeneous = false, double theta = 0.5);
int build_step_plan(ccfv_ctx *ctx, StepPlan *plan, double dt, bool fp64,
                    const std::vector<PlanField> &fields, bool homogeneous = false,
                    double theta = 0.5);
// jstep: the step's index in an out-of-place sequence (selects the buffers).
int run_step_plan(ccfv_ctx *ctx, const StepPlan &plan, bool fp64, int first, int count,
                  double toff, void *data_override, cudaStream_t st, int jstep = 0);
int steps(ccfv_ctx *ctx, void *d_C, bool fp64, double t0, double dt, int nsteps, cudaStream_t st,
          double theta = 0.5);
int coarse_fp32(ccfv_ctx *ctx, double *d_C, double tn, double DT, int m, cudaStream_t st,
                double theta = 0.5);
int fine_slices(ccfv_ctx *ctx, double *d_fields, int n, double t0, double slice_dt, double DT,
                int J, cudaStream_t st);
int correct(ccfv_ctx *ctx, int form, double *U, const double *Fv, double *Gold, double *W,
            double *sq_update, double *sq_state, cudaStream_t st);
int parareal(ccfv_ctx *ctx, const ccfv_parareal_opts *o, const double *C0, double *C_T,
             ccfv_stats *stats, cudaStream_t st);
int exact_ref(ccfv_ctx *ctx, double *d_C, double t, cudaStream_t st);
int gaussians(ccfv_ctx *ctx, double *d_C, int ng, const double *params, int img, cudaStream_t st);
int norms(ccfv_ctx *ctx, const double *a, const double *b, double *rel_l2, double *max_abs,
          cudaStream_t st);
constexpr int RED_BLOCKS_MAX = 592;

}  // namespace ccfv
