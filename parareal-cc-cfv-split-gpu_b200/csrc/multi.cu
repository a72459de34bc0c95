// multi.cu -- many Parareal solves of different sizes, velocities and
// diffusivities advanced together (batched solves and the serving loop).
//
// Every instance keeps its slice states resident on the device.  All fine
// propagators of all instances (every active slice) advance in the same sweep
// launches, and the sequential coarse sweeps of all instances advance slice by
// slice in shared launches, so a launch covers hundreds of fields and fills
// the GPU even when each instance alone cannot.  Fields are grouped into
// launch classes (kernel variant, precision, cluster size, segment length);
// instances that have converged, slices that are already exact and instances
// with fewer steps or slices drop out on the device (per-instance `nlo`
// array, SweepField::jmax/smax), and the host, which holds the same `nlo`,
// skips every launch in which no field or instance would take part.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "multi.h"

namespace ccfv {
namespace {

// Per-instance element-wise work of one batched launch.
struct BElem {
  double *U, *F, *Gold;
  void *W;        // coarse input (first sweep: FP64 state; iterations: increment)
  void *Wres;     // where the coarse sweep sequence ends (W or its partner)
  long long NN;
  int S, form, g64, pad;
  double *norms;  // [2*(S+1)]
};

enum { OP_LOAD_W = 0, OP_STORE_W = 1, OP_CORRECT = 3, OP_LOAD_W_STD = 4 };

constexpr int BT = 256;

__device__ __forceinline__ double wload(const BElem &b, long long i) {
  return b.g64 ? reinterpret_cast<const double *>(b.Wres)[i]
               : (double)reinterpret_cast<const float *>(b.Wres)[i];
}
__device__ __forceinline__ void wstore(const BElem &b, long long i, double v) {
  if (b.g64) reinterpret_cast<double *>(b.W)[i] = v;
  else reinterpret_cast<float *>(b.W)[i] = (float)v;
}

// blockIdx.y = instance.  OP_CORRECT reduces the update norms of slice n+1
// per instance with fixed-order block partials (deterministic).
__global__ void __launch_bounds__(BT)
    batch_elem_kernel(int op, const BElem *__restrict__ d, int n, const int *__restrict__ nlo,
                      double *__restrict__ partial, unsigned *__restrict__ counters) {
  const int inst = blockIdx.y;
  const BElem b = d[inst];
  const int lo = nlo[inst];
  const long long cnt = b.NN;
  if (op == OP_LOAD_W_STD) {  // G-phase: only the standard form restarts G from U
    if (b.form != CCFV_FORM_STANDARD) return;
    op = OP_LOAD_W;
  }
  switch (op) {
    case OP_LOAD_W:
    case OP_STORE_W:
    case OP_CORRECT:
      if (n >= b.S || n < lo) return;
      break;
  }
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long first = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double se = 0.0, su = 0.0;
  if (op == OP_LOAD_W) {  // FP64 W: the first coarse sweep, standard-form G
    const double *src = b.U + (long long)n * b.NN;
    double *w = reinterpret_cast<double *>(b.W);
    for (long long i = first; i < cnt; i += stride) w[i] = src[i];
  } else if (op == OP_STORE_W) {
    double *dst = b.U + (long long)(n + 1) * b.NN;
    double *gd = b.Gold ? b.Gold + (long long)(n + 1) * b.NN : nullptr;
    const double *w = reinterpret_cast<const double *>(b.Wres);
    for (long long i = first; i < cnt; i += stride) {
      const double v = w[i];
      dst[i] = v;
      if (gd) gd[i] = v;
    }
  } else {
    double *U = b.U + (long long)(n + 1) * b.NN;
    const double *Fv = b.F + (long long)(n + 1) * b.NN;
    double *Go = b.Gold ? b.Gold + (long long)(n + 1) * b.NN : nullptr;
    if (b.pad) return;  // resident coarse propagator: corrected in its own kernel
    const bool zero_g = (b.form == CCFV_FORM_DELTA && n == lo);  // G(0) = 0
    // G is read from Wres; the new increment goes to W (elementwise, so the
    // two may be the same buffer)
    for (long long i = first; i < cnt; i += stride) {
      const double uo = U[i];
      const double gw = zero_g ? 0.0 : wload(b, i);
      double un;
      if (b.form == CCFV_FORM_STANDARD) {
        un = gw + (Fv[i] - Go[i]);  // parareal_correction_kernel, T2S4:771-782
        Go[i] = gw;
      } else {
        un = Fv[i] + gw;
        wstore(b, i, un - uo);
      }
      const double dd = un - uo;
      U[i] = un;
      se += dd * dd;
      su += un * un;
    }
    for (int o = 16; o > 0; o >>= 1) {
      se += __shfl_down_sync(0xffffffffu, se, o);
      su += __shfl_down_sync(0xffffffffu, su, o);
    }
    __shared__ double red[2][BT / 32];
    __shared__ bool last;
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = se; red[1][w] = su; }
    __syncthreads();
    double *part = partial + (size_t)inst * 2 * gridDim.x;
    if (threadIdx.x == 0) {
      double a = 0, c = 0;
      for (int k = 0; k < BT / 32; ++k) { a += red[0][k]; c += red[1][k]; }
      part[2 * blockIdx.x] = a;
      part[2 * blockIdx.x + 1] = c;
      __threadfence();
      last = (atomicAdd(&counters[inst], 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
      __threadfence();
      double a = 0, c = 0;
      for (unsigned k = 0; k < gridDim.x; ++k) {
        a += ((volatile double *)part)[2 * k];
        c += ((volatile double *)part)[2 * k + 1];
      }
      b.norms[2 * (n + 1)] = a;
      b.norms[2 * (n + 1) + 1] = c;
      counters[inst] = 0;
    }
  }
}

}  // namespace

using KKey = std::tuple<int, int, int, int, int>;  // kind, variant, cs, lc bucket, fp64

// Launch classes: fields of one sub-step kind, kernel variant, precision and
// cluster size (segments per line).  Filter-kernel fields carry their own
// segment length and halo, so they share a class across segment lengths; the
// scan kernels also group by segment-length bucket.
static void prepare_field(std::vector<PreparedField> &out, int kind, const ccfv_grid &g,
                          const SweepField &f0, bool fp64, FilterTables *tabs,
                          std::tuple<int, int, int> tkey) {
  PreparedField pf;
  pf.G = step_geom(g, f0.dir, f0.Dt, f0.dsrc, fp64, /*inplace=*/false, f0.theta);
  const bool filt = filter_variant(pf.G.variant);
  const int bucket = filt ? 0 : (pf.G.lc_max + 63) / 64;  // segment-length bucket bounds the tile
  pf.key = KKey{kind, pf.G.variant, pf.G.cs, bucket, fp64 ? 1 : 0};
  pf.level = std::get<1>(tkey);
  pf.f = f0;
  pf.f.halo_f = pf.G.halo;
  if (filt) filter_field(g, pf.f, fp64);
  if (stencil_filter_variant(pf.G.variant)) {
    FilterTable &T = (*tabs)[tkey];  // shared by every field of this key
    if (!T.lines) {
      T.lines = pf.f.groups * LPG;
      T.fp64 = fp64;
      T.level = pf.level;
      T.wt.alloc((fp64 ? 8 : 4) * 8 * (size_t)T.lines);
      T.nt.alloc(sizeof(int) * (size_t)T.lines);
    }
    pf.f.wt = T.wt.p;
    pf.f.nt = T.nt.as<int>();
    pf.T = &T;
  }
  out.push_back(pf);
}

static void place_field(std::map<KKey, SweepClass> &classes, const PreparedField &pf,
                        std::vector<FilterTable *> *pending) {
  SweepClass &K = classes[pf.key];
  K.kind = std::get<0>(pf.key);
  K.variant = pf.G.variant;
  K.cs = pf.G.cs;
  K.fp64 = std::get<4>(pf.key);
  K.lc_max = std::max(K.lc_max, pf.G.lc_max);
  K.halo = std::max(K.halo, pf.G.halo);
  FilterTable *T = pf.T;
  if (T && !T->ready && (pending->empty() || pending->back() != T) &&
      std::find(pending->begin(), pending->end(), T) == pending->end()) {
    T->cls = pf.key;  // T->idx is set once the class is sorted
    pending->push_back(T);
  }
  const int sm = pf.f.slice >= 0 ? 0 : pf.f.smax;  // fixed-slice fields: no slice bound
  K.smax_all = (K.smax_all < 0 || sm == 0 || K.smax_all == 0) ? (K.smax_all < 0 ? sm : 0)
                                                              : std::max(K.smax_all, sm);
  K.h.push_back(pf.f);
}

static int step_bound(const SweepField &f) { return f.jmax > 0 ? f.jmax : INT_MAX; }

// Sorts a class by step bound (descending, stable: problem and slice order
// kept within a bound) and numbers its tiles.
static void finish_class(SweepClass &K) {
  std::stable_sort(K.h.begin(), K.h.end(), [](const SweepField &a, const SweepField &b) {
    return step_bound(a) > step_bound(b);
  });
  K.groups = 0;
  K.bound.resize(K.h.size());
  K.gpre.assign(K.h.size() + 1, 0);
  for (size_t i = 0; i < K.h.size(); ++i) {
    SweepField &f = K.h[i];
    f.group0 = K.groups;
    f.cta0 = K.groups * K.cs;
    K.groups += f.groups;
    K.bound[i] = step_bound(f);
    K.gpre[i + 1] = K.groups;
  }
}

size_t problem_bytes(const ccfv_grid &g, const ccfv_parareal_opts &o) {
  const size_t fb = sizeof(double) * (size_t)g.nx * g.ny;
  const size_t S = (size_t)std::max(o.n_slices, 1);
  const bool g64 = o.coarse_precision != CCFV_FP32;
  (void)g64;  // W holds FP64 states in the first coarse sweep whatever the coarse precision
  // U, F and F's ping-pong partner, Gold (standard form), W and its partner
  return fb * (S + 1) * 2 + fb * S + (o.form == CCFV_FORM_STANDARD ? fb * (S + 1) : 0) + 2 * fb +
         6 * 256;
}

int problem_setup(Problem &P, const ccfv_problem &p, std::string *err) {
  P.g = p.grid;
  P.o = p.opts;
  P.C0 = p.C0;
  P.C_T = p.C_T;
  const ccfv_parareal_opts &o = P.o;
  if (o.n_slices < 1 || o.nt_fine < o.n_slices || o.nt_fine % o.n_slices || o.kmax < 1 ||
      o.kmax > CCFV_MAX_ITERS || (o.coarse_precision == CCFV_FP32 && o.form != CCFV_FORM_DELTA) ||
      (o.form != CCFV_FORM_STANDARD && o.form != CCFV_FORM_DELTA) ||
      !coarse_theta_ok(o.coarse_theta)) {
    if (err) *err = "invalid Parareal options";
    return CCFV_ERR_INVALID;
  }
  P.S = o.n_slices;
  P.J = o.nt_fine / P.S;
  if (o.coarse_ratio < 0 || (o.coarse_ratio > 0 && P.J % o.coarse_ratio)) {
    if (err) *err = "coarse_ratio must divide nt_fine / n_slices";
    return CCFV_ERR_INVALID;
  }
  P.m = o.coarse_ratio > 0 ? P.J / o.coarse_ratio : 1;
  P.DT = (o.t1 - o.t0) / P.S;
  P.dt = P.DT / (double)P.J;
  P.dtc = P.DT / (double)P.m;
  P.NN = (long long)P.g.nx * P.g.ny;
  P.g64 = o.coarse_precision != CCFV_FP32;
  P.theta = coarse_theta(o, P.g, P.dtc);
  P.bytes = problem_bytes(P.g, o);
  return CCFV_OK;
}

#define MCK(call)                                                                      \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(e_ == cudaErrorMemoryAllocation ? CCFV_ERR_NOMEM : CCFV_ERR_CUDA,    \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                 \
  } while (0)

MultiEngine::~MultiEngine() {
  cudaSetDevice(device_);
  if (side_) {
    cudaStreamSynchronize(side_);
    cudaStreamDestroy(side_);
  }
  for (cudaEvent_t e : side_ev_)
    if (e) cudaEventDestroy(e);
  cudaStreamSynchronize(st_);
  for (auto &p : slots_)
    if (p && p->mem) cudaFreeAsync(p->mem, st_);
  cudaStreamSynchronize(st_);
}

int MultiEngine::live() const {
  int n = 0;
  for (const auto &p : slots_) n += p ? 1 : 0;
  return n;
}

// Host-side fault injection for tests: with CCFV_INJECT_ALLOC_FAIL=k in the
// environment, the k-th problem allocation of every engine reports an
// allocation failure instead of allocating (nothing reaches the device).
static bool inject_alloc_failure(long long nth) {
  const char *e = std::getenv("CCFV_INJECT_ALLOC_FAIL");
  if (!e || !*e) return false;
  const long long k = std::atoll(e);
  return k > 0 && nth == k;
}

static bool autotune_enabled() {
  const char *e = std::getenv("CCFV_AUTOTUNE");
  return !(e && e[0] == '0');
}

int MultiEngine::add(const ccfv_problem &pr, int *slot) {
  auto P = std::make_unique<Problem>();
  std::string e;
  int rc = problem_setup(*P, pr, &e);
  if (rc) return fail(rc, e);
  P->ctx = std::make_unique<ccfv_ctx>();
  P->ctx->grid = P->g;
  P->ctx->device = device_;
  const double th = P->theta;  // fine tables: the reference's 0.5
  for (int t = 0; t < 6; ++t) {
    const int dir = t & 1;
    const double Dt = (t < 2 ? P->dt : P->dtc) * (dir == 0 ? 0.5 : 1.0);
    P->tab[t] = get_table(P->ctx.get(), dir, Dt, (t < 2 || t >= 4) ? true : P->g64, &rc,
                          t < 2 ? 0.5 : th);
    if (!P->tab[t]) return fail(rc, P->ctx->last_error);
  }
  // line-tile shape: the filter kernel's segment length is tuned once per
  // line-length class and precision (fine FP64 steps, coarse steps in the
  // coarse precision) on the first problem of the class, before its plans
  // are built (CCFV_AUTOTUNE=0 keeps the default)
  if (autotune_enabled()) {
    const bool fps[2] = {true, P->g64};
    const double dts[2] = {P->dt, P->dtc};
    for (int lv = 0; lv < 2; ++lv)
      if (!class_tuned(P->g.nx, fps[lv]) || !class_tuned(P->g.ny, fps[lv])) {
        rc = autotune(P->ctx.get(), dts[lv], fps[lv], st_, nullptr, /*for_class=*/true);
        if (rc) return fail(rc, P->ctx->last_error);
      }
  }
  for (int kind = 0; kind < 3; ++kind)
    for (int level = 0; level < 2; ++level) {
      const int dir = kind == 1 ? 1 : 0;
      const double Dt = (level == 0 ? P->dt : P->dtc) * (dir == 0 ? 0.5 : 1.0);
      const int dsrc = (kind == 2 && P->g.scheme == CCFV_SCHEME_REFERENCE) ? 1 : 0;
      const LaunchGeom G = step_geom(P->g, dir, Dt, dsrc, level == 0 || P->g64, false,
                                     level == 0 ? 0.5 : th);
      if (!warm_filter_variant(G.variant) && G.cs > MAX_CLUSTER)
        return fail(CCFV_ERR_UNSUPPORTED, "line longer than 4096 cells");
      if (std::max({sweep_smem_bytes(G.lc_max, G.halo, true, P->g.source != 0),
                    sweep_fast_smem_bytes(G.lc_max, G.halo, true),
                    sweep_filter_smem_bytes(G.lc_max, G.halo, true, true,
                                            cell_filter_variant(G.variant))}) > 227 * 1024)
        return fail(CCFV_ERR_UNSUPPORTED, "time step too large for the staged halo");
    }
  if (inject_alloc_failure(++allocs_))
    return fail(CCFV_ERR_NOMEM, "injected allocation failure (CCFV_INJECT_ALLOC_FAIL)");
  MCK(cudaMallocAsync(&P->mem, P->bytes, st_));
  unsigned char *q = static_cast<unsigned char *>(P->mem);
  auto take = [&](size_t b) {
    unsigned char *r = q;
    q += (b + 255) & ~size_t(255);
    return r;
  };
  const size_t fb = sizeof(double) * P->NN;
  P->U = reinterpret_cast<double *>(take(fb * (P->S + 1)));
  P->F = reinterpret_cast<double *>(take(fb * (P->S + 1)));
  P->FS = reinterpret_cast<double *>(take(fb * P->S));
  P->Gold = P->o.form == CCFV_FORM_STANDARD ? reinterpret_cast<double *>(take(fb * (P->S + 1))) : nullptr;
  P->W = take(fb);
  P->W2 = take(fb);
  MCK(cudaMemcpyAsync(P->U, P->C0, fb,
                      P->o.mem == CCFV_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st_));
  int s = -1;
  for (int i = 0; i < (int)slots_.size(); ++i)
    if (!slots_[i]) { s = i; break; }
  if (s < 0) {
    s = (int)slots_.size();
    slots_.emplace_back();
  }
  slots_[s] = std::move(P);
  dirty_ = true;
  if (slot) *slot = s;
  return CCFV_OK;
}

int MultiEngine::finish(int slot) {
  Problem *P = get(slot);
  if (!P) return fail(CCFV_ERR_NOT_FOUND, "no such problem");
  MCK(cudaMemcpyAsync(P->C_T, P->U + (size_t)P->S * P->NN, sizeof(double) * P->NN,
                      P->o.mem == CCFV_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, st_));
  return CCFV_OK;
}

void MultiEngine::remove(int slot) {
  Problem *P = get(slot);
  if (!P) return;
  if (P->mem) cudaFreeAsync(P->mem, st_);
  slots_[slot].reset();
  dirty_ = true;
}

// Rebuilds the launch classes, element-wise descriptors and norm offsets
// after problems joined or left.
int MultiEngine::rebuild() {
  fine_.clear();
  coarse_.clear();
  std::vector<FilterTable *> pending;  // stencil tables not computed yet
  const int n = (int)slots_.size();
  std::vector<BElem> he(n);
  norm_off_.assign(n, 0);
  size_t noff = 0;
  // finished problems keep their slot (their stats are read later) but leave
  // the launch classes and the element-wise launches
  auto live = [&](const Problem *P) { return P && P->state != Problem::DONE; };
  for (int i = 0; i < n; ++i) {
    Problem *P = slots_[i].get();
    if (!live(P)) {
      std::memset(&he[i], 0, sizeof(BElem));
      continue;
    }
    norm_off_[i] = noff;
    noff += 2 * (size_t)(P->S + 1);
  }
  MCK(norms_d_.alloc(sizeof(double) * std::max<size_t>(noff, 2)));
  hnorms_.assign(std::max<size_t>(noff, 2), 0.0);
  for (int i = 0; i < n; ++i) {
    Problem *P = slots_[i].get();
    if (!live(P)) continue;
    const ccfv_grid &g = P->g;
    // coarse sequences start in W and end in W2 when 3m is odd
    he[i] = BElem{P->U, P->F, P->Gold, P->W, ((3 * P->m) & 1) ? P->W2 : P->W, P->NN, P->S,
                  P->o.form, P->g64 ? 1 : 0, 0, norms_d_.as<double>() + norm_off_[i]};
    // resident coarse propagator: delta form, periodic, the coarse field in
    // one SM's shared memory (CCFV_RESIDENT_G=0 keeps every problem in the
    // shared launches)
    const char *rge = std::getenv("CCFV_RESIDENT_G");
    const bool want_rg = !P->prepared && !(rge && rge[0] == '0') &&
                         P->o.form == CCFV_FORM_DELTA && g.bc == CCFV_BC_PERIODIC &&
                         resident_g_fits(g.nx, g.ny, P->g64,
                                         g.velocity == CCFV_VEL_SWIRL);
    std::vector<PreparedField> rg_prep;  // its iterations' coarse fields, if resident
    for (int kind = 0; kind < 3 && !P->prepared; ++kind) {
      const int dir = kind == 1 ? 1 : 0;
      const int dsrc = (kind == 2 && g.scheme == CCFV_SCHEME_REFERENCE) ? 1 : 0;
      {  // fine: field s = F[s+1], time t0 + s DT (+ j dt per launch step)
        const double Dt = kind == 1 ? P->dt : 0.5 * P->dt;
        const double ta = kind == 2 ? 0.5 * P->dt : 0.0, tb = kind == 0 ? 0.5 * P->dt : P->dt;
        for (int s = 0; s < P->S; ++s) {
          SweepField f = make_field(g, dir, Dt, ta + P->o.t0 + s * P->DT, tb + P->o.t0 + s * P->DT,
                                    P->F + (size_t)(s + 1) * P->NN, P->tab[dir], dsrc);
          f.inst = i;
          f.slice = s;
          f.src_tb = kind == 2 ? 1 : 0;
          f.jmax = P->J;
          f.t_step = P->dt;
          // out of place: U[s] -> ... -> F[s+1] through the pair F[s+1] / FS[s]
          f.kind = kind;
          f.pp = 1;
          f.data2 = P->FS + (size_t)s * P->NN;
          f.in0 = P->U + (size_t)s * P->NN;
          f.par = pp_parity(P->J);
          prepare_field(P->prep, kind, g, f, true, &P->ftab, std::make_tuple(kind, 0, 1));
        }
      }
      {  // coarse: the work field W, slice from the launch (t0 + n DT + i dtc)
        const double Dt = kind == 1 ? P->dtc : 0.5 * P->dtc;
        const double ta = kind == 2 ? 0.5 * P->dtc : 0.0, tb = kind == 0 ? 0.5 * P->dtc : P->dtc;
        auto coarse_field = [&](const ccfv_grid &gg, const SolverTable *tab, int phase) {
          SweepField f = make_field(gg, dir, Dt, ta + P->o.t0, tb + P->o.t0, P->W, tab, dsrc,
                                    P->theta);
          f.inst = i;
          f.slice = -1;
          f.jmax = P->m;
          f.smax = P->S;
          f.gskip = P->o.form == CCFV_FORM_DELTA ? 1 : 0;
          f.t_step = P->dtc;
          f.t_slice = P->DT;
          f.phase = phase;
          f.src_tb = kind == 2 ? 1 : 0;
          f.kind = kind;
          f.pp = 1;  // W -> ... -> W or W2 through the pair W / W2
          f.data2 = P->W2;
          f.in0 = P->W;
          f.par = 0;
          return f;
        };
        const bool delta_src = g.source != CCFV_SRC_NONE && P->o.form == CCFV_FORM_DELTA;
        if (P->g64 && !delta_src && !want_rg) {
          prepare_field(P->prep, kind, g, coarse_field(g, P->tab[2 + dir], 0), true, &P->ftab,
                        std::make_tuple(kind, 1, 1));
        } else {
          // the first sweep moves states: FP64, with the source; the
          // iterations move increments in the coarse precision (delta form:
          // with the linear part of G, without the source)
          prepare_field(P->prep, kind, g, coarse_field(g, P->tab[4 + dir], 1), true, &P->ftab,
                        std::make_tuple(kind, 1, 1));
          ccfv_grid gh = g;
          if (P->o.form == CCFV_FORM_DELTA) gh.source = CCFV_SRC_NONE;
          prepare_field(want_rg ? rg_prep : P->prep, kind, gh, coarse_field(gh, P->tab[2 + dir], 2),
                        P->g64, &P->ftab, std::make_tuple(kind, 1, P->g64 ? 1 : 0));
        }
      }
    }
    if (want_rg) {
      // resident only if every coarse sweep of the iterations runs a filter
      // form (their constants mu and 1/c are then in the descriptors)
      bool ok = rg_prep.size() == 3;
      for (const PreparedField &pf : rg_prep) ok = ok && filter_variant(pf.G.variant);
      if (ok) {
        P->resident = true;
        for (int k = 0; k < 3; ++k) P->rgf[k] = rg_prep[k].f;
      } else {
        for (const PreparedField &pf : rg_prep) P->prep.push_back(pf);
      }
    }
    he[i].pad = P->resident ? 1 : 0;
    P->prepared = true;
    for (const PreparedField &pf : P->prep) place_field(pf.level == 0 ? fine_ : coarse_, pf, &pending);
  }
  hclass_.clear();
  hidx_.clear();
  for (auto *cls : {&fine_, &coarse_})
    for (auto &kv : *cls) {
      SweepClass &K = kv.second;
      finish_class(K);
      K.off = hclass_.size();
      K.ioff = hidx_.size();
      hclass_.insert(hclass_.end(), K.h.begin(), K.h.end());
      for (const SweepField &f : K.h) hidx_.push_back(f.group0);
    }
  for (FilterTable *T : pending) {  // a descriptor of each new table, after the sort
    const SweepClass &K = (T->level == 0 ? fine_ : coarse_).at(T->cls);
    size_t i = 0;
    while (i < K.h.size() && K.h[i].wt != T->wt.p) ++i;
    if (i == K.h.size()) return fail(CCFV_ERR_CUDA, "stencil table without a field");
    T->idx = i;
  }
  MCK(classbuf_.alloc(sizeof(SweepField) * std::max<size_t>(hclass_.size(), 1)));
  MCK(idxbuf_.alloc(sizeof(int) * std::max<size_t>(hidx_.size(), 1)));
  if (!hclass_.empty()) {
    MCK(cudaMemcpyAsync(classbuf_.p, hclass_.data(), sizeof(SweepField) * hclass_.size(),
                        cudaMemcpyHostToDevice, st_));
    MCK(cudaMemcpyAsync(idxbuf_.p, hidx_.data(), sizeof(int) * hidx_.size(),
                        cudaMemcpyHostToDevice, st_));
  }
  for (FilterTable *T : pending) {  // stencil tables first needed by this rebuild
    if (!T->wt.p || !T->nt.p) return fail(CCFV_ERR_NOMEM, "stencil table allocation failed");
    const SweepClass &K = (T->level == 0 ? fine_ : coarse_).at(T->cls);
    MCK(launch_filter_weights(T->fp64, classbuf_.as<SweepField>() + K.off + T->idx, T->wt.p,
                              T->nt.as<int>(), T->lines, st_));
    T->ready = true;
  }
  const int eb = 148;
  MCK(elems_.alloc(sizeof(BElem) * std::max(n, 1)));
  if (n) MCK(cudaMemcpyAsync(elems_.p, he.data(), sizeof(BElem) * n, cudaMemcpyHostToDevice, st_));
  {
    std::vector<ResidentG> hr[2];
    for (int i = 0; i < n; ++i) {
      Problem *P = slots_[i].get();
      if (!live(P) || !P->resident) continue;
      ResidentG r;
      std::memset(&r, 0, sizeof(r));
      for (int k = 0; k < 3; ++k) r.f[k] = P->rgf[k];
      r.F = P->F;
      r.U = P->U;
      r.norms = norms_d_.as<double>() + norm_off_[i];
      r.inst = i;
      r.S = P->S;
      r.m = P->m;
      r.nx = P->g.nx;
      r.ny = P->g.ny;
      r.pitch = P->g.ny | 1;
      const int q = P->g64 ? 1 : 0;
      rgsmem_[q] = std::max(rgsmem_[q], resident_g_smem_bytes(P->g.nx, P->g.ny, P->g64,
                                                              P->g.velocity == CCFV_VEL_SWIRL));
      hr[q].push_back(r);
    }
    for (int q = 0; q < 2; ++q) {
      rgn_[q] = (int)hr[q].size();
      if (rgn_[q]) {
        MCK(rgbuf_[q].alloc(sizeof(ResidentG) * hr[q].size()));
        MCK(cudaMemcpyAsync(rgbuf_[q].p, hr[q].data(), sizeof(ResidentG) * hr[q].size(),
                            cudaMemcpyHostToDevice, st_));
      }
    }
  }
  MCK(nlo_d_.alloc(sizeof(int) * std::max(n, 1)));
  MCK(partial_.alloc(sizeof(double) * 2 * eb * (size_t)std::max(n, 1)));
  if (counters_.bytes < sizeof(unsigned) * std::max(n, 1)) {
    MCK(counters_.alloc(sizeof(unsigned) * std::max(n, 1) * 2));
    MCK(cudaMemsetAsync(counters_.p, 0, counters_.bytes, st_));
  }
  if (!status_.p) {
    MCK(status_.alloc(sizeof(unsigned) * 4));
    MCK(cudaMemsetAsync(status_.p, 0, sizeof(unsigned) * 4, st_));
  }
  MCK(cudaStreamSynchronize(st_));  // host staging vectors are reused
  nlo_.assign(n, 0);
  dirty_ = false;
  return CCFV_OK;
}

int MultiEngine::push_nlo() {
  if (!nlo_.empty())
    MCK(cudaMemcpyAsync(nlo_d_.p, nlo_.data(), sizeof(int) * nlo_.size(), cudaMemcpyHostToDevice, st_));
  return CCFV_OK;
}

// Host mirror of batch_elem_kernel's per-instance guard.
bool MultiEngine::elem_active(int op, int n) const {
  for (size_t i = 0; i < slots_.size(); ++i) {
    const Problem *P = slots_[i].get();
    if (!P || P->state == Problem::DONE) continue;  // zeroed element: S = 0
    if (op == OP_LOAD_W_STD && P->o.form != CCFV_FORM_STANDARD) continue;
    if (op == OP_CORRECT && P->resident) continue;
    if (n < P->S && n >= nlo_[i]) return true;
  }
  return false;
}

int MultiEngine::elem(int op, int slice) {
  const int n = (int)slots_.size();
  if (!n || !elem_active(op, slice)) return CCFV_OK;
  count_launch();
  batch_elem_kernel<<<dim3(148, n), BT, 0, st_>>>(op, elems_.as<BElem>(), slice, nlo_d_.as<int>(),
                                                   partial_.as<double>(), counters_.as<unsigned>());
  MCK(cudaGetLastError());
  return CCFV_OK;
}

int MultiEngine::sweeps(std::map<KKey, SweepClass> &classes, int kind, int jstep, int nslice) {
  BatchStep bs;
  bs.jstep = jstep;
  bs.nslice = nslice;
  bs.nlo = nlo_d_.as<int>();
  bs.inplace = false;  // every batched field sweeps out of place
  unsigned *status = status_.as<unsigned>();
  for (auto &kv : classes) {
    SweepClass &K = kv.second;
    if (K.kind != kind) continue;
    if (K.smax_all > 0 && nslice >= K.smax_all) continue;
    // fields with a step bound above jstep: a prefix of the sorted class
    const int np = (int)(std::partition_point(K.bound.begin(), K.bound.end(),
                                              [&](int b) { return b > jstep; }) -
                         K.bound.begin());
    bool any = false;  // the kernel's own guard, evaluated here on the host copy of nlo
    for (int i = 0; i < np && !any; ++i) any = field_active(K.h[i], jstep, nslice, nlo_.data());
    if (!any) continue;
    bs.g0idx = idxbuf_.as<int>() + K.ioff;
    const SweepField *fd = classbuf_.as<SweepField>() + K.off;
    cudaError_t e =
        K.fp64 ? launch_sweep_batch<double>(K.variant, fd, np, 0, K.gpre[np], K.cs, K.lc_max,
                                            K.halo, bs, status, st_)
               : launch_sweep_batch<float>(K.variant, fd, np, 0, K.gpre[np], K.cs, K.lc_max,
                                           K.halo, bs, status, st_);
    MCK(e);
  }
  return CCFV_OK;
}

int MultiEngine::coarse_slice(int s, int mmax) {
  for (int i = 0; i < mmax; ++i)
    for (int kind = 0; kind < 3; ++kind)
      if (int rc = sweeps(coarse_, kind, i, s)) return rc;
  return CCFV_OK;
}

int MultiEngine::iterate(std::vector<int> *finished) {
  if (finished) finished->clear();
  if (dirty_)
    if (int rc = rebuild()) return rc;
  const int n = (int)slots_.size();
  cudaEvent_t e0, ef, ef2, e1;
  MCK(cudaEventCreate(&e0));
  MCK(cudaEventCreate(&ef));
  MCK(cudaEventCreate(&ef2));
  MCK(cudaEventCreate(&e1));
  MCK(cudaEventRecord(e0, st_));
  // first coarse sweep U[s+1] = G(U[s]) of newly admitted problems
  // (T2S4:1271-1280); nlo = -1: every slice active, G starts from U
  int Snew = 0, mnew = 0;
  for (int i = 0; i < n; ++i) {
    Problem *P = slots_[i].get();
    const bool fresh = P && P->state == Problem::NEW;
    nlo_[i] = fresh ? -1 : (P ? P->S : 0);
    if (fresh) {
      Snew = std::max(Snew, P->S);
      mnew = std::max(mnew, P->m);
    }
  }
  if (Snew) {
    if (int rc = push_nlo()) return rc;
    for (int s = 0; s < Snew; ++s) {
      int rc = elem(OP_LOAD_W, s);
      if (!rc) rc = coarse_slice(s, mnew);
      if (!rc) rc = elem(OP_STORE_W, s);
      if (rc) return rc;
    }
    for (auto &p : slots_)
      if (p && p->state == Problem::NEW) {
        p->state = Problem::RUNNING;
        p->coarse_cu += (double)p->S * p->m * p->NN;
      }
  }
  // one Parareal iteration of every running problem; iteration k+1 leaves
  // slices < k untouched (already exact)
  int Smax = 0, Jmax = 0, mmax = 0, running = 0, resident = 0;
  bool any_std = false;
  for (int i = 0; i < n; ++i) {
    Problem *P = slots_[i].get();
    if (P && P->state == Problem::RUNNING) {
      nlo_[i] = P->k;
      if (P->resident) {
        ++resident;
      } else {
        Smax = std::max(Smax, P->S);
        mmax = std::max(mmax, P->m);
      }
      Jmax = std::max(Jmax, P->J);
      any_std |= P->o.form == CCFV_FORM_STANDARD;
      ++running;
      P->fine_cu += (double)(P->S - P->k) * P->J * P->NN;
      P->coarse_cu += (double)(P->S - P->k - (P->o.form == CCFV_FORM_DELTA ? 1 : 0)) * P->m * P->NN;
    } else {
      nlo_[i] = P ? P->S : 0;
    }
  }
  if (running) {
    if (int rc = push_nlo()) return rc;
    // F[s+1] = F(U[s]): the fine sequences read U[s] in their first sweep
    MCK(cudaEventRecord(ef, st_));
    for (int j = 0; j < Jmax; ++j)
      for (int kind = 0; kind < 3; ++kind)
        if (int rc = sweeps(fine_, kind, j, 0)) return rc;
    MCK(cudaEventRecord(ef2, st_));
    if (resident) {
      // the resident problems' whole G phases, one CTA each, beside the
      // shared coarse launches of the others
      if (!side_) {
        MCK(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
        MCK(cudaEventCreateWithFlags(&side_ev_[0], cudaEventDisableTiming));
      }
      MCK(cudaStreamWaitEvent(side_, ef2, 0));
      for (int q = 0; q < 2; ++q)
        if (rgn_[q])
          MCK(launch_resident_g(q == 1, rgbuf_[q].as<ResidentG>(), rgn_[q], rgsmem_[q],
                                nlo_d_.as<int>(), side_));
      MCK(cudaEventRecord(side_ev_[0], side_));
    }
    for (int s = 0; s < Smax; ++s) {
      int rc = any_std ? elem(OP_LOAD_W_STD, s) : CCFV_OK;
      if (!rc) rc = coarse_slice(s, mmax);
      if (!rc) rc = elem(OP_CORRECT, s);
      if (rc) return rc;
    }
    if (resident) MCK(cudaStreamWaitEvent(st_, side_ev_[0], 0));
    MCK(cudaMemcpyAsync(hnorms_.data(), norms_d_.p, sizeof(double) * hnorms_.size(),
                        cudaMemcpyDeviceToHost, st_));
  }
  MCK(cudaEventRecord(e1, st_));
  MCK(cudaStreamSynchronize(st_));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  ms_ += ms;
  if (running) {
    float fms = 0;
    cudaEventElapsedTime(&fms, ef, ef2);
    fine_ms_ += fms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(ef);
  cudaEventDestroy(ef2);
  cudaEventDestroy(e1);
  unsigned flag = 0;
  MCK(cudaMemcpy(&flag, status_.p, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (flag) return fail(CCFV_ERR_HALO, "a characteristic foot left the staged halo");
  for (int i = 0; i < n; ++i) {
    Problem *P = slots_[i].get();
    if (!P || P->state != Problem::RUNNING) continue;
    const double *hn = hnorms_.data() + norm_off_[i];
    double worst = 0.0;
    for (int s = P->k + 1; s <= P->S; ++s) {
      const double e = std::sqrt(hn[2 * s]), u = std::sqrt(hn[2 * s + 1]);
      worst = std::max(worst, u > 0 ? e / u : e);
    }
    P->upd[P->k] = worst;
    P->k += 1;
    if (P->o.tol > 0 && worst < P->o.tol) P->converged = 1;
    if (P->converged || P->k >= P->o.kmax || P->k >= P->S) {
      // after S iterations Parareal equals the serial fine solve exactly
      P->state = Problem::DONE;
      dirty_ = true;  // drop it from the launch classes
      if (finished) finished->push_back(i);
    }
  }
  return CCFV_OK;
}

void fill_stats(const Problem &P, ccfv_stats *s, double ms) {
  std::memset(s, 0, sizeof(*s));
  s->iterations = P.k;
  s->converged = P.converged;
  for (int k = 0; k < P.k && k < CCFV_MAX_ITERS; ++k) s->update[k] = P.upd[k];
  s->fine_cell_updates = P.fine_cu;
  s->coarse_cell_updates = P.coarse_cu;
  s->ms = ms;
}

int batch_solve(int n, const ccfv_problem *probs, ccfv_stats *stats, int device, cudaStream_t st,
                std::string *errmsg) {
  if (cudaSetDevice(device) != cudaSuccess) return CCFV_ERR_CUDA;
  MultiEngine E(device, st);
  std::vector<int> slot(n, -1);
  auto bail = [&](int rc) {
    if (errmsg) *errmsg = E.error();
    return rc;
  };
  for (int i = 0; i < n; ++i)
    if (int rc = E.add(probs[i], &slot[i])) return bail(rc);
  std::vector<int> fin;
  int remaining = n;
  while (remaining > 0) {
    if (int rc = E.iterate(&fin)) return bail(rc);
    for (int sl : fin) {
      if (int rc = E.finish(sl)) return bail(rc);
      --remaining;
    }
    if (E.live() == 0) break;
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) return bail(CCFV_ERR_CUDA);
  if (stats)
    for (int i = 0; i < n; ++i) {
      fill_stats(*E.get(slot[i]), &stats[i], E.device_ms());
      // phases are shared by the whole batch: engine-wide device times
      stats[i].fine_ms = E.fine_ms();
      stats[i].coarse_ms = E.device_ms() - E.fine_ms();
    }
  return CCFV_OK;
}

}  // namespace ccfv
