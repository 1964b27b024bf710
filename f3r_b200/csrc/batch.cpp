// batch.cpp -- several right-hand sides per solver, and several solvers at
// once: the nrhs and batch entry points of include/f3r_b200.h.
//
// The reference solves one system per driver run (work/src/f3r-gpu.cpp:88).
// Here a solver's device objects (matrix copies, preconditioner, captured
// inner-level graphs) serve every right-hand side given to it: up to 16
// columns at once in lockstep, one block product per matrix pass
// (Solver::solve_multi, solver.cu), or column by column where the nest has
// no block form; and independent solvers run concurrently, one host thread
// per context, so that their streams overlap on the GPU while each thread
// waits for its own solves' residual checks.
#include <algorithm>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "internal.hpp"

using namespace f3r;

extern "C" {

f3r_status f3r_solver_solve_multi(f3r_solver *s, int32_t nrhs, const double *b, int64_t ldb, double *x, int64_t ldx,
                                  f3r_cond_fn cond, void *user, f3r_result *results) {
  if (!s || nrhs < 0 || (nrhs > 0 && (!b || !x))) return fail(F3R_ERROR_INVALID_VALUE, "bad argument");
  const int32_t n = solver_rows(s);
  if (ldb < n || ldx < n) return fail(F3R_ERROR_INVALID_VALUE, "leading dimension below the row count");
  return solver_solve_multi(s, nrhs, b, ldb, x, ldx, cond, user, results);
}

f3r_status f3r_solve_batch(int32_t count, f3r_solver *const *solvers, const int32_t *nrhs, const double *const *b,
                           const int64_t *ldb, double *const *x, const int64_t *ldx, f3r_cond_fn cond, void *user,
                           f3r_result *results) {
  if (count < 0 || (count > 0 && (!solvers || !nrhs || !b || !ldb || !x || !ldx)))
    return fail(F3R_ERROR_INVALID_VALUE, "bad argument");
  std::vector<int64_t> first(count + 1, 0);  // results[first[i] ...] belong to system i
  for (int32_t i = 0; i < count; i++) {
    if (!solvers[i] || nrhs[i] < 0) return fail(F3R_ERROR_INVALID_VALUE, "null solver or negative nrhs");
    first[i + 1] = first[i] + nrhs[i];
  }
  // systems sharing a context run in order on one thread; groups spread over
  // at most 128 threads
  std::map<const void *, std::vector<int32_t>> by_ctx;
  for (int32_t i = 0; i < count; i++) by_ctx[solver_context(solvers[i])].push_back(i);
  const size_t nthreads = std::min<size_t>(by_ctx.size(), 128);
  std::vector<std::vector<int32_t>> work(nthreads);
  size_t g = 0;
  for (auto &kv : by_ctx) {
    auto &w = work[g++ % std::max<size_t>(nthreads, 1)];
    w.insert(w.end(), kv.second.begin(), kv.second.end());
  }
  std::vector<f3r_status> st(count, F3R_SUCCESS);
  std::vector<std::string> msg(count);
  auto run = [&](const std::vector<int32_t> &items) {
    for (int32_t i : items) {
      st[i] = f3r_solver_solve_multi(solvers[i], nrhs[i], b[i], ldb[i], x[i], ldx[i], cond, user,
                                     results ? results + first[i] : nullptr);
      if (st[i] != F3R_SUCCESS) msg[i] = f3r_last_error_string();
    }
  };
  if (nthreads <= 1) {
    if (nthreads == 1) run(work[0]);
  } else {
    std::vector<std::thread> th;
    th.reserve(nthreads);
    for (size_t t = 0; t < nthreads; t++) th.emplace_back(run, std::cref(work[t]));
    for (auto &t : th) t.join();
  }
  for (int32_t i = 0; i < count; i++)
    if (st[i] != F3R_SUCCESS) return fail(st[i], "system " + std::to_string(i) + ": " + msg[i]);
  return F3R_SUCCESS;
}

}  // extern "C"
