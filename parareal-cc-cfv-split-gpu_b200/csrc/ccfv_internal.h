// ccfv_internal.h -- device-side data structures and launchers shared by the
// translation units of libccfv (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace ccfv {

enum { BC_COMPAT = 0, BC_PERIODIC = 1 };
enum { VEL_REF_ROT4 = 0, VEL_CONST = 1, VEL_ROTATION = 2, VEL_SWIRL = 3 };

// Device status word bits (set by kernels, read by ccfv_check).
enum : unsigned { STATUS_HALO = 1u };

// Tile geometry of the fused sweep kernel.  A CTA owns LPG lines and a run
// of consecutive cells (positions) of those lines; a thread-block cluster of
// `cs` CTAs covers whole lines.  Lines sit in the fast (lane) index of the
// shared-memory tile, positions in the slow index, so every phase of the
// kernel reads shared memory without bank conflicts in both directions.
constexpr int LPG = 16;          // lines per tile (x-sweeps: 128 B rows)
constexpr int PITCH = LPG + 1;   // odd pitch: conflict-free column access
constexpr int NW = 8;            // warps per CTA
constexpr int NTH = NW * 32;     // threads per CTA
constexpr int CPW = 32 / LPG;    // chunks per warp
constexpr int NCH = NW * CPW;    // chunks per line per CTA
constexpr int LC_MAX = 256;      // max positions per CTA
constexpr int MAX_CLUSTER = 16;  // non-portable cluster size (lines <= 4096)
constexpr int MAX_DEVICES = 64;  // device ordinals with per-device library state

// One field (one instance at one time slice) in one sweep launch.
// x-sweep: lines are columns j (s_line = 1, s_pos = ny), positions i.
// y-sweep: lines are rows i (s_line = ny, s_pos = 1), positions j.
struct SweepField {
  void *data;            // T[ny*nx]: swept in place (pp = 0), or buffer A (pp = 1)
  void *data2;           // pp = 1: buffer B
  const void *in0;       // pp = 1: input of the first sweep of the sequence
  long long s_pos;       // element stride between positions of a line
  long long s_line;      // element stride between lines
  int L;                 // cells per line
  int M;                 // lines
  int dir;               // 0: x-sweep, 1: y-sweep
  int bc;                // BC_*
  int vel;               // VEL_*
  int group0;            // first tile index of this field in the launch
  int groups;            // tiles of this field = ceil(M / LPG)
  int dsrc;              // foot derivative of: 0 the sweep input, 1 the remapped field
  int hd;                // dsrc = 1: halo (cells) of the remapped field
  int uniform;           // 1: the velocity along the sweep depends only on the
                         // transverse coordinate (every foot of a line has the
                         // same displacement): stencil fast path
  int jf;                // filter kernel: recurrence warm-up length J
  int cta0;              // filter kernel: first CTA of this field in the launch
                         // (a multiple of the launch's cluster size)
  int halo_f;            // filter kernel: staged halo (cells) of this field
  int hyb;               // > 0: the line's segments are split between two launches,
                         // those at least hyb cells from both ends run the stencil
                         // form, the others the compat form; 0: one launch
  // Batched launches (all zero for single-instance launches):
  int inst;              // instance index into the launch's `nlo` array
  int slice;             // >= 0: fixed slice of this field; -1: the launch's slice
  int jmax;              // the field takes part while jstep < jmax (0: always)
  int smax;              // slice-indexed fields: while slice < smax
  int gskip;             // slice-indexed fields: skip slice == nlo (zero increment)
  int kind;              // sub-step of the split step: 0 x(dt/2), 1 y(dt), 2 x(dt/2)
  int pp;                // 1: out-of-place sequence: sweep s = 3 jstep + kind writes A
                         // when s + par is odd, else B, and reads the other buffer
                         // (in0 for s = 0); 0: in place on `data`
  int par;               // pp = 1: parity offset (chosen so the last sweep writes A)
  int phase;             // slice-indexed fields: 0 every launch, 1 only while the
                         // instance's nlo < 0 (first coarse sweep), 2 only while
                         // nlo >= 0 (Parareal iterations)
  int src;               // source term: 0 none (the reference's f = 0), 1 Gaussian
  int src_tb;            // 1: the remapped source is f(t_b) too (third sub-step), else f(t_a)
  double sp[5];          // Gaussian source: sp0 exp(-((x-sp1)^2+(y-sp2)^2)/sp3) cos(sp4 t)
  double src_w;          // RHS weight of (remapped f(t_a or t_b) + f(t_b))
  double t_step;         // added per launch step: time = ... + jstep * t_step
  double t_slice;        // added per launch slice: time = ... + slice * t_slice
  double vp[4];          // velocity parameters
  double s_min, s_max, h;  // along-line edge coordinates: s_min + h*e
  double t_min, ht;        // transverse edges: t_min + ht*line
  double Dt;               // sub-step length
  double ta_rel, tb_rel;   // foot-tracing interval relative to the launch time
  double eps_remap;        // compat remap clamp (x: 1e-15, y: 1e-16)
  double kb;               // (1-theta)*K*(Dt/h): RHS diffusion coefficient
  double theta;            // implicit weight of the diffusion (0.5: Crank-Nicolson);
                           // host bookkeeping: the kernels read kb and the tables
  double inv12h;           // 1/(12 h)
  double sm_fac;           // periodic, scan kernels: a / gamma; filter kernel: mu
  double sm_inv_den;       // periodic, scan kernels: 1 / (1 + z0 + (a/gamma) z_{L-1});
                           // filter kernel: 1 / c
  const void *tab;         // T[3L]: alpha_k | g_k | z_k (solver factors)
  // Filter kernel: per-line stencil of w's input, computed once per plan
  // (the velocity fields it serves do not depend on time); null: computed
  // per tile.  wt: T[groups*LPG][8] taps -3..4; nt: int[groups*LPG] shifts.
  const void *wt;
  const int *nt;
};

// Whether a field takes part in a batched launch (`nlo[inst]`: the first
// active slice of every instance, -1 before the first coarse sweep; null: a
// single-instance launch, always active).  The batched engine evaluates the
// same rule on the host to skip launches in which no field is active.
__host__ __device__ inline bool field_active(const SweepField &f, int jstep, int nslice,
                                             const int *nlo) {
  if (f.jmax > 0 && jstep >= f.jmax) return false;
  if (!nlo) return true;
  const int lo = nlo[f.inst];
  if (f.slice >= 0) return f.slice >= lo;
  if ((f.phase == 1 && lo >= 0) || (f.phase == 2 && lo < 0)) return false;
  return nslice < f.smax && nslice >= lo + f.gskip;
}

// Shared-memory slot of one descriptor at the head of every sweep kernel's
// dynamic shared memory (the data behind it stays 64-byte aligned).
constexpr size_t FD_BYTES = (sizeof(SweepField) + 63) & ~size_t(63);

// Kernel variants: the per-cell kernel (any velocity / boundary / scheme) and
// the fused stencil kernel (uniform displacement, periodic, derivative of the
// sweep input).
// SWEEP_GENERAL_SRC is the per-cell kernel with the source tile staged;
// SWEEP_FILTER_EXACT the filter kernel's cluster form (any diffusion number,
// out of place).
// SWEEP_CELL / SWEEP_CELL_EXACT: the filter kernel's two forms with a
// per-cell right-hand side (feet that differ from edge to edge);
// SWEEP_CELL_COMPAT: the per-cell form with the reference's boundaries
// (non-cyclic system).
// SWEEP_FILTER_WIDE: the stencil form with the 13-tap right-hand side of the
// reference scheme's third sweep (interior segments of compat lines).
enum { SWEEP_GENERAL = 0, SWEEP_FAST = 1, SWEEP_FILTER = 2, SWEEP_GENERAL_SRC = 3,
       SWEEP_FILTER_EXACT = 4, SWEEP_CELL = 5, SWEEP_CELL_EXACT = 6, SWEEP_CELL_COMPAT = 7,
       SWEEP_FILTER_WIDE = 8 };
// Variants run by the filter kernel (factored solve).
inline bool filter_variant(int v) {
  return v == SWEEP_FILTER || v == SWEEP_FILTER_EXACT || v == SWEEP_CELL ||
         v == SWEEP_CELL_EXACT || v == SWEEP_CELL_COMPAT || v == SWEEP_FILTER_WIDE;
}
// Warm-up (segmented) forms: lines longer than MAX_CLUSTER segments are
// allowed out of place.
inline bool warm_filter_variant(int v) {
  return v == SWEEP_FILTER || v == SWEEP_CELL || v == SWEEP_CELL_COMPAT;
}
// Variants whose right-hand side is the per-line stencil table (SweepField::wt).
inline bool stencil_filter_variant(int v) { return v == SWEEP_FILTER || v == SWEEP_FILTER_EXACT; }
// Variants with the per-cell right-hand side.
inline bool cell_filter_variant(int v) {
  return v == SWEEP_CELL || v == SWEEP_CELL_EXACT || v == SWEEP_CELL_COMPAT;
}
// The filter kernel's cluster form (exact periodic closure, out of place).
inline bool exact_filter_variant(int v) { return v == SWEEP_FILTER_EXACT || v == SWEEP_CELL_EXACT; }
constexpr int FILTER_JMAX = 64;  // longest recurrence warm-up of the filter kernel

// Shared-memory bytes of the sweep kernels for a launch.
size_t sweep_smem_bytes(int lc_max, int halo, bool fp64, bool source = false);
size_t sweep_fast_smem_bytes(int lc_max, int halo, bool fp64);
size_t sweep_filter_smem_bytes(int lc_max, int halo, bool fp64, bool exact = false,
                               bool cell = false, bool wide = false);
// Longest segment (cells per CTA along a line) of the filter kernel for a
// recurrence warm-up of J cells.
int filter_segment_max(int J);
// Fills the per-line stencil table of the filter kernel for field `*d_field`
// (device descriptor): wt = T[lines][8], nt = int[lines], lines = groups*LPG
// (lines past M get zeros).
cudaError_t launch_filter_weights(bool fp64, const SweepField *d_field, void *wt, int *nt,
                                  int lines, cudaStream_t stream, bool wide = false);

// Launches one fused sweep over all fields of `d_fields` (device array,
// sorted by group0; tiles group_base .. group_base+groups_total-1).  All fields share the cluster size `cs`, their
// max positions per CTA `lc_max` and the halo `halo`.  `toff` is added to
// every field's ta_rel/tb_rel (the launch time); `data` (if non-null)
// replaces fields[0].data (single-field launches).  `jstep` is the step of an
// out-of-place sequence (SweepField::pp); `inplace` says whether any field
// sweeps in place (the filter kernel's segments of a line then form a
// cluster).
template <typename T>
cudaError_t launch_sweep(int variant, const SweepField *d_fields, int nfields, int group_base,
                         int groups_total, int cs, int lc_max, int halo, double toff, void *data,
                         unsigned *d_status, cudaStream_t stream, int jstep = 0,
                         bool inplace = true);

// Batched form: `jstep` / `nslice` select the step and slice of this launch,
// `nlo[inst]` the first active slice of every instance (see SweepField).
struct BatchStep {
  int jstep = 0, nslice = 0;
  const int *nlo = nullptr;
  bool inplace = true;
  const int *g0idx = nullptr;  // the fields' group0 values (device), or null
};
template <typename T>
cudaError_t launch_sweep_batch(int variant, const SweepField *d_fields, int nfields,
                               int group_base, int groups_total, int cs, int lc_max, int halo,
                               const BatchStep &bs, unsigned *d_status, cudaStream_t stream);

// Solver-table layout (T values): alpha[L] g[L] z[L] tP[L] tS[L]
// aggA[cs*NCH] PA[cs*(NCH+1)], where, for the chunk partition the sweep
// kernels use (cs = ceil(L/LC_MAX) CTAs per line, NCH chunks per CTA),
// tP[k] / tS[k] are the products of alpha from the chunk start to k / from k
// to the chunk end, aggA the chunk products and PA the CTA-local exclusive
// prefix products of the chunks (PA[NCH] = product over the CTA).
inline int table_cs(int L) { return (L + LC_MAX - 1) / LC_MAX; }
inline size_t table_len(int L) {
  const int cs = table_cs(L);
  return 5 * (size_t)L + (size_t)cs * NCH + (size_t)cs * (NCH + 1);
}
// Fills tP, tS, aggA, PA of a table whose alpha is already in place
// (heap-free; T = double or float, computed in double).
template <typename T>
void fill_chunk_products(int L, T *tab);

// Resident coarse propagator (coarse.cu): the whole G phase of one
// delta-form Parareal iteration of an instance whose coarse field fits in one
// SM's shared memory, one CTA per instance.  f: the instance's coarse sweep
// descriptors of the iterations (x, y, x; filter-kernel constants filled).
struct ResidentG {
  SweepField f[3];
  const double *F;  // F[0..S] fine results
  double *U;        // U[0..S] slice states (updated)
  double *norms;    // [2 (S + 1)]: sum dU^2, sum U^2 of every corrected slice
  int inst;         // index into the launch's nlo array
  int S, m, nx, ny, pitch;
};
// Dynamic shared memory of the resident kernel for an nx x ny field.
size_t resident_g_smem_bytes(int nx, int ny, bool fp64, bool cell);
// Whether an nx x ny coarse field can be resident (lines of at most 272
// cells, the field in shared memory).
bool resident_g_fits(int nx, int ny, bool fp64, bool cell);
cudaError_t launch_resident_g(bool fp64, const ResidentG *d_rg, int n, size_t smem,
                              const int *nlo, cudaStream_t st);

// Counts kernel launches made by the library.
void count_launch(uint64_t n = 1);
uint64_t launches();

}  // namespace ccfv
