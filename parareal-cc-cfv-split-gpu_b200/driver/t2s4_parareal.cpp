// t2s4_parareal -- command-line driver with the reference executable's
// interface: `t2s4_parareal config.txt`.
//
// Reads the reference's `key:value` config keys (T2S4_Parareal.cu:1017-1055)
//   T_min, T_max, N, Nt, T_span, K
// plus optional keys of this solver
//   slices (40), kmax (8), tol (0), coarse_ratio (0 = one coarse step per
//   slice), coarse (fp64|fp32), form (standard|delta), coarse_theta (0.5 =
//   Crank-Nicolson G, 1 = backward Euler G), scheme (reference|consistent),
//   bc (compat|periodic), dump (1|0), device (0)
// and runs what the reference's main() runs: the initial condition, the
// serial fine solve with gnuplot dumps every T_span steps
// (data_T2S4_%06d.txt, T2S4:93-114), then Parareal with the per-iteration
// max-norm error against the serial solution (T2S4:1333-1346), and the
// reference's summary lines (T2S4:1357-1366).  All solver work goes through
// the C ABI of libccfv.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <string>
#include <vector>

#include "ccfv.h"

namespace {

void die(const char *what, int rc, ccfv_ctx *ctx) {
  std::fprintf(stderr, "%s failed: %s (%s)\n", what, ccfv_strerror(rc),
               ctx ? ccfv_last_error(ctx) : "");
  std::exit(2);
}

#define CHECK(call)                  \
  do {                               \
    int rc_ = (call);                \
    if (rc_) die(#call, rc_, ctx);   \
  } while (0)

// output_result (T2S4_Parareal.cu:93-114): "%.6lf %.6lf %.4e" per cell,
// a blank line after every x row.
void output_result(const std::vector<double> &v, int step, const ccfv_grid &g) {
  char name[64];
  std::snprintf(name, sizeof(name), "data_T2S4_%06d.txt", step);
  FILE *fp = std::fopen(name, "w");
  if (!fp) return;
  const double dx = (g.x_max - g.x_min) / g.nx, dy = (g.y_max - g.y_min) / g.ny;
  for (int i = 0; i < g.nx; ++i) {
    const double x = g.x_min + dx * (i + 0.5);
    for (int j = 0; j < g.ny; ++j) {
      const double y = g.y_min + dy * (j + 0.5);
      std::fprintf(fp, "%.6lf %.6lf %.4e\n", x, y, v[(size_t)i * g.ny + j]);
    }
    std::fprintf(fp, "\n");
  }
  std::fclose(fp);
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) {
    std::cout << "please input config file name" << std::endl;
    return 1;
  }
  std::ifstream cfg(argv[1]);
  if (!cfg.is_open()) {
    std::cout << "Cannot open config file!" << std::endl;
    return 1;
  }
  std::cout << "open config file ok" << std::endl;
  std::map<std::string, std::string> kv;
  std::string line;
  while (std::getline(cfg, line)) {
    if (line.empty()) continue;
    size_t pos = line.find(':');
    if (pos == std::string::npos) continue;
    std::string v = line.substr(pos + 1);
    while (!v.empty() && (v.back() == '\r' || v.back() == ' ')) v.pop_back();
    while (!v.empty() && v.front() == ' ') v.erase(v.begin());
    kv[line.substr(0, pos)] = v;
  }
  auto num = [&](const char *k, double dflt) { return kv.count(k) ? std::atof(kv[k].c_str()) : dflt; };
  auto str = [&](const char *k, const char *dflt) { return kv.count(k) ? kv[k] : std::string(dflt); };

  const double T_min = num("T_min", 0.0), T_max = num("T_max", 1.0), K = num("K", 0.0);
  const int N = (int)num("N", 64), Nt = (int)num("Nt", 100), T_span = (int)num("T_span", 0);
  const int slices = (int)num("slices", 40), kmax = (int)num("kmax", 8);
  const int ratio = (int)num("coarse_ratio", 0), device = (int)num("device", 0);
  const double tol = num("tol", 0.0);
  const bool dump = num("dump", 1.0) != 0.0 && T_span > 0;
  const bool periodic = str("bc", "compat") == "periodic";

  ccfv_grid g = {};
  g.nx = N;
  g.ny = N;  // the reference forces Ny = Nx (T2S4:1039)
  g.x_min = -1.0; g.x_max = 1.0; g.y_min = -1.0; g.y_max = 1.0;
  g.bc = periodic ? CCFV_BC_PERIODIC : CCFV_BC_COMPAT;
  g.velocity = CCFV_VEL_REF_ROT4;
  g.K = K;
  g.scheme = str("scheme", "reference") == "consistent" ? CCFV_SCHEME_CONSISTENT
                                                        : CCFV_SCHEME_REFERENCE;
  ccfv_ctx *ctx = nullptr;
  CHECK(ccfv_create(&ctx, &g, device));

  const double dx = (g.x_max - g.x_min) / N, dy = (g.y_max - g.y_min) / N;
  const double dt = (T_max - T_min) / Nt;
  const size_t NN = (size_t)N * N, bytes = NN * sizeof(double);
  double *d_C = nullptr, *d_C0 = nullptr, *d_ref = nullptr, *d_UT = nullptr;
  if (cudaMalloc(&d_C, bytes) || cudaMalloc(&d_C0, bytes) || cudaMalloc(&d_ref, bytes) ||
      cudaMalloc(&d_UT, bytes)) {
    std::fprintf(stderr, "device allocation failed\n");
    return 2;
  }
  std::vector<double> h(NN);
  auto t_start = std::chrono::steady_clock::now();

  // initial condition: the reference's Gaussian at t = 0 (T2S4:1147-1155)
  CHECK(ccfv_exact_ref(ctx, d_C, 0.0, nullptr));
  cudaMemcpy(d_C0, d_C, bytes, cudaMemcpyDeviceToDevice);
  if (dump) {
    cudaMemcpy(h.data(), d_C, bytes, cudaMemcpyDeviceToHost);
    output_result(h, 0, g);
  }
  // serial fine solve (T2S4:1224-1247)
  int done = 0;
  while (done < Nt) {
    const int chunk = (dump ? std::min(T_span - done % T_span, Nt - done) : Nt - done);
    CHECK(ccfv_run(ctx, d_C, CCFV_MEM_DEVICE, T_min + done * dt, dt, chunk, nullptr));
    done += chunk;
    if (dump && done % T_span == 0) {
      cudaMemcpy(h.data(), d_C, bytes, cudaMemcpyDeviceToHost);
      output_result(h, done, g);
    }
  }
  CHECK(ccfv_check(ctx, nullptr));
  cudaMemcpy(d_ref, d_C, bytes, cudaMemcpyDeviceToDevice);

  // Parareal (T2S4:1249-1355)
  ccfv_parareal_opts o = {};
  o.t0 = T_min;
  o.t1 = T_max;
  o.nt_fine = Nt;
  o.n_slices = slices;
  o.coarse_ratio = ratio;
  o.tol = tol;
  o.kmax = kmax;
  o.coarse_precision = str("coarse", "fp64") == "fp32" ? CCFV_FP32 : CCFV_FP64;
  o.form = str("form", o.coarse_precision == CCFV_FP32 ? "delta" : "standard") == "delta"
               ? CCFV_FORM_DELTA
               : CCFV_FORM_STANDARD;
  o.mem = CCFV_MEM_DEVICE;
  o.d_ref = d_ref;
  o.coarse_theta = num("coarse_theta", 0.5);  // 0.5: Crank-Nicolson G (reference), 1: backward Euler
  ccfv_stats st;
  CHECK(ccfv_parareal(ctx, &o, d_C0, d_UT, &st, nullptr));
  for (int k = 0; k < st.iterations && k < CCFV_MAX_ITERS; ++k)
    std::printf("Parareal iter %2d: err(T) = %.3e\n", k + 1, st.err_max[k]);

  const double secs =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  std::cout << "K:" << K << std::fixed << std::setprecision(16) << std::endl;
  std::cout << "dx:" << dx << std::endl;
  std::cout << "dy:" << dy << std::endl;
  std::cout << "dt:" << dt << std::endl;
  std::cout << "Nx:" << N << std::endl;
  std::cout << "Ny:" << N << std::endl;
  std::cout << "Nt:" << Nt << std::endl;
  std::cout << "Total time (including Parareal): " << secs << " s" << std::endl;

  cudaFree(d_C);
  cudaFree(d_C0);
  cudaFree(d_ref);
  cudaFree(d_UT);
  ccfv_destroy(ctx);
  return 0;
}
