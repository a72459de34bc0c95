// ref_harness.cu -- TEST INFRASTRUCTURE (the checker's pin).
//
// Compiles the reference T2S4_Parareal.cu from its own source file (found
// through -I at build time; nothing of it is copied into this repository)
// with its main() renamed, and exposes its step orchestrator, propagators
// and Parareal schedule through a small C interface so that tests can run
// the reference itself on seeded inputs and read back full FP64 results.
//
// The set-up below mirrors what the reference's main() does before its time
// loop (T2S4_Parareal.cu:1057-1221): device buffers, launch shape, Euler
// points, GPUContext.  The time loops are the reference's own functions.
#define main t2s4_reference_main
#include "T2S4_Parareal.cu"
#undef main

#include <vector>

namespace {

struct RefSetup {
  GPUContext ctx;
  std::vector<FLOAT *> bufs;
  FLOAT *alloc(size_t n) {
    FLOAT *p = nullptr;
    if (cudaMalloc((void **)&p, n * sizeof(FLOAT)) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, n * sizeof(FLOAT));
    bufs.push_back(p);
    return p;
  }
  ~RefSetup() {
    for (FLOAT *p : bufs) cudaFree(p);
  }
};

// Mirrors T2S4_Parareal.cu:1057-1221 (sizes, launch shape, buffers, geometry).
bool setup(RefSetup &s, int N, double K) {
  GPUContext &c = s.ctx;
  c.Nx = N;
  c.Ny = N;
  c.dx = (X_max - X_min) / c.Nx;
  c.dy = (Y_max - Y_min) / c.Ny;
  c.K = K;
  c.N_grid = c.Nx * c.Ny;
  c.N_points = (c.Nx + 1) * (c.Ny + 1);
  c.N_points_inter2 = c.Nx * (c.Ny + 1);
  c.N_points_inter1 = (c.Nx + 1) * c.Ny;
  const int maxThreadsPerBlock = 128;
  if (c.N_points < maxThreadsPerBlock) {
    c.threadsPerBlock = c.N_points;
    c.numBlocks = 1;
  } else {
    c.threadsPerBlock = maxThreadsPerBlock;
    c.numBlocks = (c.N_points + maxThreadsPerBlock - 1) / maxThreadsPerBlock;
  }
  const size_t G = c.N_grid, P = c.N_points, I1 = c.N_points_inter1, I2 = c.N_points_inter2;
  c.v_d_x = s.alloc(G); c.v_d_y = s.alloc(G);
  c.v_d_xhf = s.alloc(P); c.v_d_yhf = s.alloc(P);
  c.v_d_xhf_bar1 = s.alloc(P); c.v_d_yhf_bar2 = s.alloc(P); c.v_d_xhf_bar3 = s.alloc(P);
  c.v_d_x_inter1 = s.alloc(I1); c.v_d_y_inter2 = s.alloc(I2); c.v_d_x_inter3 = s.alloc(I1);
  c.v_d_Cn = s.alloc(G); c.v_d_Cnphf_x = s.alloc(G); c.v_d_Cn_bar_x = s.alloc(G);
  c.v_d_dCndx_bar = s.alloc(I1);
  c.v_d_Cn_bar_y = s.alloc(G); c.v_d_Cnp1_y = s.alloc(G); c.v_d_dCndy_bar = s.alloc(I2);
  c.v_d_C_Exact = s.alloc(G); c.v_d_Cnp1 = s.alloc(G); c.v_d_Cnphf_bar_x = s.alloc(G);
  c.v_d_dCnphfdx_bar = s.alloc(I1);
  c.v_d_CL = s.alloc(G); c.v_d_CR = s.alloc(G); c.v_d_C6 = s.alloc(G); c.v_d_DltC = s.alloc(G);
  c.p = s.alloc(G); c.q = s.alloc(G); c.v_d_b = s.alloc(G); c.v_d_Cptb = s.alloc(G);
  c.v_d_coA_x = s.alloc(G); c.v_d_coB_x = s.alloc(G); c.v_d_coC_x = s.alloc(G);
  c.v_d_coA_y = s.alloc(G); c.v_d_coB_y = s.alloc(G); c.v_d_coC_y = s.alloc(G);
  c.v_d_f1_p0 = s.alloc(G); c.v_d_f1_p1 = s.alloc(G); c.v_d_f1_p0_bar = s.alloc(G);
  c.v_d_f2_p0 = s.alloc(G); c.v_d_f2_p1 = s.alloc(G); c.v_d_f2_p0_bar = s.alloc(G);
  for (FLOAT *p : s.bufs)
    if (!p) return false;
  get_Euler_cell_center_points_on_gpu<<<c.numBlocks, c.threadsPerBlock>>>(
      c.v_d_x, c.v_d_y, c.Nx, c.Ny, c.N_grid, c.dx, c.dy);
  get_Euler_half_points_on_gpu<<<c.numBlocks, c.threadsPerBlock>>>(
      c.v_d_xhf, c.v_d_yhf, c.Nx, c.Ny, c.N_points, c.dx, c.dy);
  return cudaDeviceSynchronize() == cudaSuccess;
}

int status() { return cudaDeviceSynchronize() == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : 2; }

}  // namespace

extern "C" {

// Nsteps serial GpuOneStep calls from t0 (the reference's serial fine run,
// T2S4_Parareal.cu:1234-1236) on the seeded field C0 (host, N*N, [i*N+j]).
int ref_run(int N, double K, double t0, double dt, int nsteps, const double *C0, double *Cout) {
  RefSetup s;
  if (!setup(s, N, K)) return 3;
  const size_t bytes = sizeof(FLOAT) * s.ctx.N_grid;
  cudaMemcpy(s.ctx.v_d_Cn, C0, bytes, cudaMemcpyHostToDevice);
  for (int n = 0; n < nsteps; ++n) GpuOneStep(s.ctx, t0 + n * dt, dt);
  cudaMemcpy(Cout, s.ctx.v_d_Cn, bytes, cudaMemcpyDeviceToHost);
  return status();
}

// Same as ref_run but times the step loop with CUDA events; returns the
// elapsed milliseconds in *ms.  Used for the reference-GPU baseline.
int ref_time_run(int N, double K, double t0, double dt, int nsteps, const double *C0, double *Cout,
                 float *ms) {
  RefSetup s;
  if (!setup(s, N, K)) return 3;
  const size_t bytes = sizeof(FLOAT) * s.ctx.N_grid;
  cudaMemcpy(s.ctx.v_d_Cn, C0, bytes, cudaMemcpyHostToDevice);
  GpuOneStep(s.ctx, t0, dt);  // warm-up (not timed)
  cudaMemcpy(s.ctx.v_d_Cn, C0, bytes, cudaMemcpyHostToDevice);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaDeviceSynchronize();
  cudaEventRecord(a);
  for (int n = 0; n < nsteps; ++n) GpuOneStep(s.ctx, t0 + n * dt, dt);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  cudaEventElapsedTime(ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaMemcpy(Cout, s.ctx.v_d_Cn, bytes, cudaMemcpyDeviceToHost);
  return status();
}

// get_exact_solution_on_gpu at time t (T2S4_Parareal.cu:1147-1148).
int ref_exact(int N, double K, double t, double *Cout) {
  RefSetup s;
  if (!setup(s, N, K)) return 3;
  get_exact_solution_on_gpu<<<s.ctx.numBlocks, s.ctx.threadsPerBlock>>>(
      s.ctx.v_d_x, s.ctx.v_d_y, s.ctx.v_d_Cn, s.ctx.dx, s.ctx.dy, t, K, s.ctx.N_grid);
  cudaMemcpy(Cout, s.ctx.v_d_Cn, sizeof(FLOAT) * s.ctx.N_grid, cudaMemcpyDeviceToHost);
  return status();
}

// The reference's Parareal section (T2S4_Parareal.cu:1249-1355) with the
// slice count and iteration cap as parameters (the reference hard-codes
// 40 and 8), driven by the reference's own CoarsePropagator,
// FinePropagator and parareal_correction_kernel.  err[k] receives
// max|U_{k+1}(T) - Uref| like the reference prints; UT the last iterate.
int ref_parareal(int N, double K, double T_min, double T_max, int Nt, int n_slices, int kmax,
                 const double *C0, const double *Uref, double *err, double *UT) {
  RefSetup s;
  if (!setup(s, N, K)) return 3;
  GPUContext &ctx = s.ctx;
  const size_t NG = ctx.N_grid, bytes = sizeof(FLOAT) * NG;
  const int Nt_coarse = n_slices;
  const FLOAT DT = (T_max - T_min) / Nt_coarse;
  const int J_fine = Nt / Nt_coarse;
  FLOAT *d_Uk = s.alloc(NG * (Nt_coarse + 1)), *d_Uk1 = s.alloc(NG * (Nt_coarse + 1));
  FLOAT *d_F = s.alloc(NG), *d_Gk = s.alloc(NG), *d_Gk1 = s.alloc(NG);
  if (!d_Uk || !d_Uk1 || !d_F || !d_Gk || !d_Gk1) return 3;
  std::vector<FLOAT> hU(NG);
  cudaMemcpy(d_Uk, C0, bytes, cudaMemcpyHostToDevice);
  for (int pass = 0; pass < 2; ++pass)
    for (int n = 0; n < Nt_coarse; ++n) {
      FLOAT tn = T_min + n * DT;
      cudaMemcpy(ctx.v_d_Cn, d_Uk + n * NG, bytes, cudaMemcpyDeviceToDevice);
      CoarsePropagator(ctx, tn, DT);
      cudaMemcpy(d_Uk + (n + 1) * NG, ctx.v_d_Cn, bytes, cudaMemcpyDeviceToDevice);
    }
  for (int k = 0; k < kmax; ++k) {
    cudaMemcpy(d_Uk1, d_Uk, bytes, cudaMemcpyDeviceToDevice);
    for (int n = 0; n < Nt_coarse; ++n) {
      FLOAT tn = T_min + n * DT;
      cudaMemcpy(ctx.v_d_Cn, d_Uk1 + n * NG, bytes, cudaMemcpyDeviceToDevice);
      CoarsePropagator(ctx, tn, DT);
      cudaMemcpy(d_Gk1, ctx.v_d_Cn, bytes, cudaMemcpyDeviceToDevice);
      cudaMemcpy(ctx.v_d_Cn, d_Uk + n * NG, bytes, cudaMemcpyDeviceToDevice);
      CoarsePropagator(ctx, tn, DT);
      cudaMemcpy(d_Gk, ctx.v_d_Cn, bytes, cudaMemcpyDeviceToDevice);
      cudaMemcpy(ctx.v_d_Cn, d_Uk + n * NG, bytes, cudaMemcpyDeviceToDevice);
      FinePropagator(ctx, tn, DT, J_fine);
      cudaMemcpy(d_F, ctx.v_d_Cn, bytes, cudaMemcpyDeviceToDevice);
      parareal_correction_kernel<<<ctx.numBlocks, ctx.threadsPerBlock>>>(
          d_Gk1, d_Gk, d_F, d_Uk1 + (n + 1) * NG, NG);
    }
    if (err && Uref) {
      cudaMemcpy(hU.data(), d_Uk1 + Nt_coarse * NG, bytes, cudaMemcpyDeviceToHost);
      double e = 0.0;
      for (size_t i = 0; i < NG; ++i) {
        double d = fabs(hU[i] - Uref[i]);
        if (d > e) e = d;
      }
      err[k] = e;
    }
    cudaMemcpy(d_Uk, d_Uk1, (Nt_coarse + 1) * bytes, cudaMemcpyDeviceToDevice);
  }
  if (UT) cudaMemcpy(UT, d_Uk + Nt_coarse * NG, bytes, cudaMemcpyDeviceToHost);
  return status();
}

}  // extern "C"
