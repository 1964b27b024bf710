// f3r_run.cpp -- command-line driver with the argument list and the CSV
// output line of the reference's experiment drivers, so a suite script that
// runs ./bin/f3r16-gpu.exe can run this program instead.
//
//   f3r-run [options] <matrix.mtx> <acc> <suite_iter> <m2> <m3> <m4> <c> <restart> [weight]
//
// positional arguments as work/src/f3r-gpu.cpp:45-57 (static.cpp:28-38 adds
// the weight); output, one line on stdout (f3r-gpu.cpp:94-103, 267-285):
//
//   Problem,Method,Prec,M2,M3,M4,W,Precond,ACC,Time,Iter,ImplRes,ExplRes
//
//   Problem   the matrix argument without its last four characters
//   Method    F3R | F3R-Static | F3 | F2 | F4 | F3H | F2H
//   Prec      __half for F3R with SDAINV (the fp16 GPU build), _Float16 for
//             the others (their CPU builds, work/Makefile:52-86)
//   W         c for F3R, the weight for F3R-Static (static.cpp:121-125)
//   Precond   SDAINV or BJILU0, then ACC as given on the command line
//   Time      mean wall time of solver.solve over suite_iter solves, seconds
//   Iter      sum(outer iterations) * m2 * m3 * m4 / suite_iter (integer); for the depth
//             ablations sum(outer iterations) * 64 / suite_iter (depth.cpp:185-186)
//   ImplRes   |Givens residual estimate| / ||b||
//   ExplRes   ||b - A x|| / ||b|| in fp64
//
// options:
//   --method F3R|F3R-Static|F3|F2|F4|F3H|F2H
//                                   default F3R; F3R-Static reads [weight]; F3 / F2 and the
//                                   fp16-vector F4 / F3H / F2H are depth.cpp's fixed nests
//   --precond SDAINV|BJILU0         default SDAINV for F3R (f3r-gpu.cpp:74),
//                                   BJILU0 for the others (static.cpp:57-58)
//   --blocks N                      block-Jacobi blocks, default 112
//   --format SELL|CSR|AUTO          matrix storage on the GPU: SELL-32 (default), CSR as the CPU
//                                   drivers store it (f3r.cpp:50; the same sums), or the layout
//                                   autotuner's choice
//   --tol EPS                       stop at ||r|| / ||b|| < EPS, default 1e-8
//   --header                        print the CSV header line first
//
// The matrix is read as given, or from ../matrix/ (where the reference's
// drivers look, f3r-gpu.cpp:45) when it does not exist as given.  b comes
// from "<stem>_b.mtx" when present, else U(0, 1) from std::mt19937_64(0).
// The fp16 GPU F3R driver (F3R with SDAINV) caps restarts at 20 whatever
// <restart> says (f3r-gpu.cpp:262); the others use <restart>.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "f3r_b200.hpp"

namespace {

int usage(const char *msg) {
  std::fprintf(stderr,
               "%s\nusage: f3r-run [--method F3R|F3R-Static|F3|F2|F4|F3H|F2H] [--precond SDAINV|BJILU0] [--blocks N] "
               "[--format SELL|CSR|AUTO] [--tol EPS] [--header] <matrix.mtx> <acc> <suite_iter> <m2> <m3> <m4> <c> "
               "<restart> [weight]\n",
               msg);
  return 2;
}

bool exists(const std::string &p) {
  FILE *f = std::fopen(p.c_str(), "rb");
  if (f) std::fclose(f);
  return f != nullptr;
}

#define CU(x)                                                                              \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess) {                                                               \
      std::fprintf(stderr, "f3r-run: %s: %s\n", #x, cudaGetErrorString(e_));               \
      return 1;                                                                            \
    }                                                                                      \
  } while (0)

}  // namespace

int main(int argc, char **argv) {
  std::string method = "F3R", precond, format = "SELL";
  int blocks = 112;
  double eps = 1e-8;
  bool header = false;
  std::vector<std::string> pos;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    auto val = [&]() -> const char * { return i + 1 < argc ? argv[++i] : nullptr; };
    if (a == "--method") {
      const char *v = val();
      if (!v) return usage("--method needs a value");
      method = v;
    } else if (a == "--precond") {
      const char *v = val();
      if (!v) return usage("--precond needs a value");
      precond = v;
    } else if (a == "--blocks") {
      const char *v = val();
      if (!v) return usage("--blocks needs a value");
      blocks = std::atoi(v);
    } else if (a == "--format") {
      const char *v = val();
      if (!v) return usage("--format needs a value");
      format = v;
      if (format != "SELL" && format != "CSR" && format != "AUTO") return usage("--format is SELL, CSR or AUTO");
    } else if (a == "--tol") {
      const char *v = val();
      if (!v) return usage("--tol needs a value");
      eps = std::atof(v);
    } else if (a == "--header") {
      header = true;
    } else if (a.size() > 2 && a.compare(0, 2, "--") == 0) {
      return usage(("unknown option " + a).c_str());
    } else {
      pos.push_back(a);
    }
  }
  const bool is_static = method == "F3R-Static";
  const bool is_depth =
      method == "F3" || method == "F2" || method == "F4" || method == "F3H" || method == "F2H";
  if (method != "F3R" && !is_static && !is_depth) return usage("unknown method");
  if (pos.size() < 8 + (is_static ? 1u : 0u)) return usage("missing arguments");
  if (precond.empty()) precond = method == "F3R" ? "SDAINV" : "BJILU0";
  if (precond != "SDAINV" && precond != "BJILU0") return usage("unknown preconditioner");

  const std::string arg_matrix = pos[0], arg_acc = pos[1];
  const double acc = std::atof(arg_acc.c_str());
  const int suite_iter = std::atoi(pos[2].c_str());
  const int m2 = std::atoi(pos[3].c_str()), m3 = std::atoi(pos[4].c_str()), m4 = std::atoi(pos[5].c_str());
  const int c = std::atoi(pos[6].c_str()), restart = std::atoi(pos[7].c_str());
  const double weight = is_static ? std::atof(pos[8].c_str()) : 0.0;
  if (suite_iter < 1) return usage("suite_iter must be >= 1");
  if (arg_matrix.size() < 4) return usage("matrix file name too short");

  std::string path = arg_matrix;
  if (!exists(path) && exists("../matrix/" + arg_matrix)) path = "../matrix/" + arg_matrix;
  const std::string name = arg_matrix.substr(0, arg_matrix.size() - 4);

  try {
    auto [data, rhs] = f3r::io::mm::read_system(path);
    if (data.nrows() != data.ncols()) {
      std::fprintf(stderr, "f3r-run: the matrix is not square\n");
      return 1;
    }
    f3r::algorithm::scaling(data);  // f3r-gpu.cpp:65
    const int n = data.nrows();

    f3r::params p;
    p.acc = acc;
    p.c = c;
    p.precond = precond == "SDAINV" ? F3R_PRECOND_SDAINV : F3R_PRECOND_ILU0_BJ;
    p.ilu_blocks = blocks;
    if (format == "CSR") p.format = F3R_FORMAT_CSR;
    if (format == "AUTO") p.sell_autotune = 1;
    const bool gpu_build = method == "F3R" && precond == "SDAINV";  // the f3r16-gpu.exe configuration
    p.max_restarts = gpu_build ? 20 : restart;
    if (is_depth) {
      // depth.cpp:122-167, M the plain preconditioner (one step of weight 1):
      //   F3  fp32 (A32, 8) / fp32 (A16, 8) / M      F2  fp32 (A32, 64) / M
      //   F4  fp32 (A32, 8) / fp32 (A16, 4) / fp16 vectors (A16, 2) / M
      //   F3H fp32 (A32, 8) / fp16 vectors (A16, 8) / M
      //   F2H fp16 vectors (A16, 64) / M
      p.m2 = method == "F2" ? 64 : method == "F2H" ? 0 : 8;
      p.m3 = method == "F3" ? 8 : method == "F4" ? 4 : 0;
      p.half_m = method == "F4" ? 2 : method == "F3H" ? 8 : method == "F2H" ? 64 : 0;
      p.m4 = 1;
      p.static_weight = 1.0;
    } else {
      p.m2 = m2;
      p.m3 = m3;
      p.m4 = m4;
      p.static_weight = weight;
    }
    f3r::Context ctx(0);
    f3r::F3R solver(ctx, data, p);

    double *db = nullptr, *dx = nullptr;
    CU(cudaMalloc(&db, sizeof(double) * n));
    CU(cudaMalloc(&dx, sizeof(double) * n));
    CU(cudaMemcpy(db, rhs.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    double nrm_b = 0;
    for (double v : rhs) nrm_b += v * v;
    nrm_b = std::sqrt(nrm_b);

    double seconds = 0;
    long long itr_sum = 0;
    f3r::solve_res_t flag;
    f3r_result detail{};
    for (int it = 0; it < suite_iter; it++) {
      CU(cudaMemset(dx, 0, sizeof(double) * n));  // x.fill(0.0), f3r-gpu.cpp:81
      CU(cudaDeviceSynchronize());
      auto cond = [&](int, double e) { return e / nrm_b < eps; };
      auto t0 = std::chrono::steady_clock::now();
      flag = solver.solve(db, dx, cond, &detail);
      auto t1 = std::chrono::steady_clock::now();
      seconds += std::chrono::duration<double>(t1 - t0).count();
      itr_sum += flag.res_iter;
    }
    CU(cudaFree(db));
    CU(cudaFree(dx));

    std::ostringstream w;  // W column: c as an int, the static weight as ostream prints a double
    if (is_static)
      w << weight;
    else
      w << c;
    if (header) std::printf("Problem,Method,Prec,M2,M3,M4,W,Precond,ACC,Time,Iter,ImplRes,ExplRes\n");
    std::printf("%s,%s,%s,%d,%d,%d,%s,%s,%s,", name.c_str(), method.c_str(), gpu_build ? "__half" : "_Float16",
                m2, m3, m4, w.str().c_str(), precond.c_str(), arg_acc.c_str());
    std::printf("%e,", seconds / suite_iter);
    const long long ww = is_depth ? 64 : (long long)m2 * m3 * m4;  // the test() lambda's ww
    std::printf("%d,%e,", (int)(itr_sum * ww / suite_iter), flag.res_nrm2 / nrm_b);
    std::printf("%e\n", detail.expl_rel_res);
  } catch (const f3r::error &e) {
    std::fprintf(stderr, "f3r-run: %s\n", e.what());
    return 1;
  }
  return 0;
}
