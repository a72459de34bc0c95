// multi.h -- incremental multi-problem Parareal engine (batched solves and the
// serving loop).
#pragma once

#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "engine.h"

namespace ccfv {

// Per-line stencil table of the filter kernel for one (sub-step kind, level,
// precision) of a problem; `cls`/`idx` locate a descriptor that uses it in
// the launch classes of the rebuild that first needs it (the weights are
// computed once, then kept while the problem lives).
struct FilterTable {
  DevBuf wt, nt;
  int lines = 0;
  bool fp64 = true;
  bool ready = false;
  int level = 0;  // 0: fine class, 1: coarse class
  std::tuple<int, int, int, int, int> cls;
  size_t idx = 0;
};
using FilterTables = std::map<std::tuple<int, int, int>, FilterTable>;  // kind, level, fp64

// A sweep descriptor of a problem, prepared once (launch geometry, filter
// constants, stencil table); a rebuild only places it into its launch class.
struct PreparedField {
  std::tuple<int, int, int, int, int> key;  // launch class
  int level = 0;                            // 0: fine, 1: coarse
  LaunchGeom G;
  FilterTable *T = nullptr;                 // filter kernel: its stencil table
  SweepField f;
};

// One live problem.  Its slice states stay resident on the device from
// admission until it finishes.
struct Problem {
  ccfv_grid g;
  ccfv_parareal_opts o;
  const double *C0 = nullptr;
  double *C_T = nullptr;
  int S = 0, J = 0, m = 0;
  double DT = 0, dt = 0, dtc = 0;
  double theta = 0.5;        // diffusion weight of the coarse steps
  long long NN = 0;
  bool g64 = true;
  void *mem = nullptr;       // cudaMallocAsync arena: U, F, FS, Gold, W, W2
  size_t bytes = 0;
  double *U = nullptr, *F = nullptr, *Gold = nullptr;
  double *FS = nullptr;      // ping-pong partner of F[1..S] (out-of-place fine sweeps)
  void *W = nullptr, *W2 = nullptr;  // coarse work field and its ping-pong partner
  std::unique_ptr<ccfv_ctx> ctx;  // owns the solver tables of this grid
  // fine x, fine y, coarse x, coarse y (coarse precision), coarse x, y in
  // FP64 (the first coarse sweep, which always runs in FP64)
  const SolverTable *tab[6] = {};
  FilterTables ftab;         // stencil tables of its filter-kernel fields
  std::vector<PreparedField> prep;  // its sweep descriptors (built at the first rebuild)
  bool prepared = false;
  // resident coarse propagator (coarse.cu): its G phase runs in one CTA with
  // the field in shared memory; rgf = its coarse sweep descriptors of the
  // iterations (not placed in the launch classes)
  bool resident = false;
  SweepField rgf[3];
  enum { NEW, RUNNING, DONE } state = NEW;
  int k = 0;                 // iterations done
  int converged = 0;
  double upd[CCFV_MAX_ITERS] = {};
  double fine_cu = 0, coarse_cu = 0;
};

// Fills the public stats of a finished problem (ms: caller-defined time).
void fill_stats(const Problem &P, ccfv_stats *s, double ms);
// Device bytes a problem keeps resident (slice states and work field).
size_t problem_bytes(const ccfv_grid &g, const ccfv_parareal_opts &o);
// Validates options and fills the derived sizes; no device work.
int problem_setup(Problem &P, const ccfv_problem &p, std::string *err);

// A launch class: its descriptors sit at `off` in the engine's descriptor
// buffer and their group0 values at `ioff` in its index buffer (one
// grow-only allocation and one upload each for all classes).  Fields are
// sorted by their step bound (SweepField::jmax, 0 = none) in descending
// order, so the fields active at step j form a prefix: a launch covers only
// that prefix's tiles.
struct SweepClass {
  int kind = 0, variant = 0, cs = 1, lc_max = 0, halo = 0, fp64 = 1;
  std::vector<SweepField> h;
  size_t off = 0, ioff = 0;
  int groups = 0;
  std::vector<int> bound;  // step bound per field (jmax, 0 -> INT_MAX), descending
  std::vector<int> gpre;   // gpre[i]: tiles of fields [0, i)
  // slice bound over the fields (0: some field has none): a launch with
  // nslice >= smax_all has no active field
  int smax_all = -1;
};

class MultiEngine {
 public:
  MultiEngine(int device, cudaStream_t st) : device_(device), st_(st) {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;  // keep released problem states cached in the pool
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
  }
  ~MultiEngine();
  // Admits a problem (allocates its states stream-ordered, uploads C0).
  int add(const ccfv_problem &p, int *slot);
  // Copies the final state of a finished problem into its C_T (stream-ordered).
  int finish(int slot);
  // Releases a problem's device memory.
  void remove(int slot);
  // One engine step: the first coarse sweep of newly admitted problems, then
  // one Parareal iteration of every running problem.  `finished` receives the
  // slots whose problems converged or reached kmax in this step.
  int iterate(std::vector<int> *finished);
  Problem *get(int slot) { return slot >= 0 && slot < (int)slots_.size() ? slots_[slot].get() : nullptr; }
  int live() const;
  const std::string &error() const { return err_; }
  double device_ms() const { return ms_; }
  // device time of the F phases (the rest of device_ms is coarse sweeps,
  // corrections and norms)
  double fine_ms() const { return fine_ms_; }

 private:
  int rebuild();
  int push_nlo();
  int elem(int op, int slice);
  bool elem_active(int op, int slice) const;
  int sweeps(std::map<std::tuple<int, int, int, int, int>, SweepClass> &cls, int kind, int jstep,
             int nslice);
  int coarse_slice(int s, int mmax);
  int fail(int code, const std::string &msg) {
    err_ = msg;
    return code;
  }

  int device_;
  cudaStream_t st_;
  std::vector<std::unique_ptr<Problem>> slots_;
  bool dirty_ = true;
  std::map<std::tuple<int, int, int, int, int>, SweepClass> fine_, coarse_;
  DevBuf classbuf_, idxbuf_;  // SweepField descriptors and group0 indices of every class
  std::vector<SweepField> hclass_;
  std::vector<int> hidx_;
  DevBuf elems_, nlo_d_, partial_, counters_, status_, norms_d_;
  std::vector<int> nlo_;
  std::vector<size_t> norm_off_;
  std::vector<double> hnorms_;
  std::string err_;
  double ms_ = 0, fine_ms_ = 0;
  // resident coarse propagators: descriptors per coarse precision (FP32,
  // FP64), their shared memory, and the side stream they run on beside the
  // shared coarse launches of the other problems
  DevBuf rgbuf_[2];
  int rgn_[2] = {0, 0};
  size_t rgsmem_[2] = {0, 0};
  cudaStream_t side_ = nullptr;
  cudaEvent_t side_ev_[2] = {nullptr, nullptr};
  long long allocs_ = 0;  // problem allocations attempted (fault injection counts them)
};

}  // namespace ccfv
