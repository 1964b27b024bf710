// kmm_drop_in.cpp -- TEST: the reference driver's own solve call site run
// against this library.  The body of the driver's test() lambda
// (work/src/f3r-gpu.cpp:76-104) is not copied here: oracle/Makefile extracts
// it from the reference tree at build time into ref_test_lambda.inc, which is
// included below unchanged.  The lambda calls solver.solve(b, x, cond) on a
// kmm::Solver<host> that wraps f3r::kmm::F3R (include/f3r_b200_kmm.hpp), and
// prints "time,iterations,implicit residual,explicit residual" as the driver
// does.  Built into oracle/_ref/kmm_drop_in (it needs the reference headers);
// run by tests/test_gpu_kmm_drop_in.py.
//
// argv: system file (int32 n, int32 nnz, rptr, idx, fp64 val of the scaled
// matrix, fp64 b), sigma, c, precond (0 SDAINV, 1 block-Jacobi ILU(0)),
// ILU blocks.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "umineko-core/timer.hpp"
#include "umineko-sparse/matrix/csr.hpp"
#include "umineko-sparse/matrix/sell.hpp"
#include "umineko-sparse/models.hpp"

#include "f3r_b200_kmm.hpp"

using namespace kmm;

// the driver's stop tolerance (a global the lambda reads; 1e-8 in the driver)
const double eps = 1.e-10;

int main(int argc, char **argv) {
  if (argc < 6) {
    std::fprintf(stderr, "usage: %s system.bin sigma c precond blocks\n", argv[0]);
    return 2;
  }
  FILE *f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  int32_t n = 0, nnz = 0;
  bool ok = std::fread(&n, 4, 1, f) == 1 && std::fread(&nnz, 4, 1, f) == 1;
  auto data = CSR<double, host>(impl::shape{n, n}, nnz);
  std::vector<double> bh(n);
  ok = ok && std::fread(data.rptr.raw(), 4, n + 1, f) == (size_t)n + 1;
  ok = ok && std::fread(data.idx.raw(), 4, nnz, f) == (size_t)nnz;
  ok = ok && std::fread(data.val.raw(), 8, nnz, f) == (size_t)nnz;
  ok = ok && std::fread(bh.data(), 8, n, f) == (size_t)n;
  std::fclose(f);
  if (!ok) return 2;

  using tag = host;
  auto A = SELL<32, double, tag>(data);
  auto b = vector<double, tag>(n);
  std::memcpy(b.raw(), bh.data(), sizeof(double) * n);
  auto x = vector<double, tag>(A.nrows());
  auto r = vector<double, tag>(A.nrows());
  impl::pool<double, tag>::init(A.nrows());
  int suite_iter = 1;

#include "ref_test_lambda.inc"

  f3r_params p = f3r::kmm::default_params();
  p.sell_sigma = std::atoi(argv[2]);
  p.c = std::atoi(argv[3]);
  p.precond = std::atoi(argv[4]) ? F3R_PRECOND_ILU0_BJ : F3R_PRECOND_SDAINV;
  p.ilu_blocks = std::atoi(argv[5]);
  auto solver = Solver<tag>(f3r::kmm::F3R<tag>(data, p));
  auto t = timer();
  int itr_sum = 0;
  test(solver, b, t, true, itr_sum, 1);

  // the other in/out types of the concept: float right-hand side and solution
  auto bf = vector<float, tag>(n), xf = vector<float, tag>(n);
  for (int32_t i = 0; i < n; i++) bf[i] = (float)b[i];
  xf.fill(0.0f);
  solver.solve(bf, xf);  // no stop test: f3r_params.rel_tol (1e-8)
  double dmax = 0, xmax = 0;
  for (int32_t i = 0; i < n; i++) {
    dmax = std::max(dmax, std::abs((double)xf[i] - x[i]));
    xmax = std::max(xmax, std::abs(x[i]));
  }
  std::printf("float_solve,%e\n", dmax / xmax);
  return 0;
}
