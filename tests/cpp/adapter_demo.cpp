// A reference-style driver written against the C++ adapter: the same steps
// as work/src/f3r-gpu.cpp:60-104 (matrix, scaling, solver, cond, solve),
// with f3r:: in place of kmm::.  Built and run by tests/test_gpu_cpp_adapter.py.
#include <cmath>
#include <cstdio>
#include <vector>

#include "f3r_b200.hpp"

int main(int argc, char **argv) {
  const int nx = argc > 1 ? std::atoi(argv[1]) : 16;
  auto data = f3r::CSR::stencil27(nx, nx, nx, 2, 0.5);  // io::mm::read_system(...)
  f3r::algorithm::scaling(data);                       // algorithm::scaling(data)
  const int n = data.nrows();
  std::vector<double> xs(n), b(n), x(n, 0.0);
  f3r_random_uniform(0, -1.0, 1.0, n, xs.data());
  data.operate(xs.data(), b.data());
  double nrm_b = 0;
  for (double v : b) nrm_b += v * v;
  nrm_b = std::sqrt(nrm_b);

  f3r::Context ctx(0);
  f3r::params p;
  p.sell_sigma = 256;
  f3r::F3R solver(ctx, data, p);
  const double eps = 1e-10;
  int calls = 0;
  auto cond = [&](int i, double e) {  // f3r-gpu.cpp:83-86
    calls++;
    return e / nrm_b < eps;
  };
  f3r_result detail{};
  f3r::solve_res_t flag = solver.solve(b.data(), x.data(), cond, &detail);
  double err = 0, nx2 = 0;
  for (int i = 0; i < n; i++) {
    err += (x[i] - xs[i]) * (x[i] - xs[i]);
    nx2 += xs[i] * xs[i];
  }
  std::printf("solved %d iters %d calls %d expl %.3e err %.3e\n", flag.is_solved ? 1 : 0, flag.res_iter, calls,
              detail.expl_rel_res, std::sqrt(err / nx2));
  // the same solve with the SDAINV factors computed here and handed over
  auto zw = f3r::algorithm::sdainv(data, 0.1, 1.0);
  f3r::F3R given(ctx, data, p, zw.first, zw.second);
  std::vector<double> x2(n, 0.0);
  f3r_result d2{};
  const f3r::solve_res_t f2 = given.solve(b.data(), x2.data(), cond, &d2);
  bool same = f2.res_iter == flag.res_iter;
  for (int i = 0; i < n && same; i++) same = x2[i] == x[i];
  std::printf("given_factors_identical %d\n", same ? 1 : 0);
  return (flag.is_solved && detail.expl_rel_res < eps && same) ? 0 : 1;
}
