// ref_depth.cpp -- TEST INFRASTRUCTURE: the depth ablations of the paper
// whose innermost FGMRES level keeps its vectors in fp16 (work/src/
// depth.cpp:122-131 "F4", :143-151 "F3H", :161-167 "F2H"), compiled from the
// reference headers in place into oracle/_ref/libf3r_ref_depth.so.
//
// Those solvers need the reference's models2.hpp (its Operator and
// CoefficientMatrix concepts also take _Float16 vectors) and gmres2.hpp, which
// share include guards with models.hpp and gmres.hpp; so, like the s-step
// library, this is a library of its own with hidden visibility.  The
// preconditioner is block-Jacobi ILU(0) applied directly (no Richardson), as
// in depth.cpp.  A must already be scaled.
// The reference headers come first, in the depth driver's order: the
// templates below must not be visible where tensor.hpp and the matrix
// headers call sqrt() on their own scalar types.
#include "umineko-sparse/models2.hpp"

#include "umineko-sparse/matrix/csr.hpp"
#include "umineko-sparse/matrix/io.hpp"
#include "umineko-sparse/preconditioner/ilu.hpp"
#include "umineko-sparse/solver/restart.hpp"
#include "umineko-sparse/trsv/bj.hpp"

#include <cmath>
#include <type_traits>

// gmres2.hpp calls unqualified abs() and sqrt() on the level's scalar type.
// For _Float16 they are evaluated in float and rounded back, which is what
// the depth driver supplies before including it (work/src/depth.cpp:17-31).
template <typename T> T abs(const T &v) {
  if constexpr (std::is_same_v<T, _Float16>) return (_Float16)std::fabs((float)v);
  else return std::abs(v);
}
template <typename T> T sqrt(const T &v) {
  if constexpr (std::is_same_v<T, _Float16>) return (_Float16)std::sqrt((float)v);
  else return std::sqrt(v);
}

#include "umineko-sparse/solver/gmres2.hpp"

#include "ref_compose.hpp"

namespace {

using namespace kmm;
using refc::h16;

// variant 0: F4, 1: F3H, 2: F2H (the level sizes are the driver's constants)
refc::solve_out depth_half(const CSR<double, host> &data, const double *b, double *x, int variant, int restarts,
                           double tol, double acc, int blocks, double *hist, int hist_cap) {
  using tag = host;
  const int32_t n = data.nrows();
  auto A = CSR<double, tag>(data);
  impl::pool<double, tag>::init(n);
  impl::pool<float, tag>::init(n);
  impl::pool<h16, tag>::init(n);
  auto bd = data.duplicate_block_diagonal(blocks, 1);
  auto [l, u] = algorithm::split(algorithm::ilup(bd, 0, acc, blocks, 1));
  auto L = trsv::l::BJ<CSR<h16, host>>(l, {blocks});
  auto U = trsv::du::BJ<CSR<h16, host>>(u, {blocks});
  auto tmp = vector<h16, tag>(n);
  auto M = Operator<tag>(data.get_shape(), [&](auto in, auto out) {
    L.solve(in, tmp);
    U.solve(tmp, out);
  });
  auto A16 = CSR<h16, tag>(A);
  auto A32 = CSR<float, tag>(A);
  if (variant == 0) {  // F4: fp64 / fp32 (A32, 8) / fp32 (A16, 4) / fp16 (A16, 2) / M
    auto FF = FGMRES<h16, tag>(A16, M, {2, false});
    auto F = FGMRES<float, tag>(A16, FF, {4, false});
    auto inner = FGMRES<float, tag>(A32, F, {8, false});
    auto solver_ = Solver<tag>(FGMRES<double, tag>(A, inner, {100, true}));
    auto solver = Restarted<double, tag>(A, solver_, {restarts});
    return refc::run_solve(solver, A, b, x, n, tol, hist, hist_cap);
  }
  if (variant == 1) {  // F3H: fp64 / fp32 (A32, 8) / fp16 (A16, 8) / M
    auto F = FGMRES<h16, tag>(A16, M, {8, false});
    auto inner = FGMRES<float, tag>(A32, F, {8, false});
    auto solver_ = Solver<tag>(FGMRES<double, tag>(A, inner, {100, true}));
    auto solver = Restarted<double, tag>(A, solver_, {restarts});
    return refc::run_solve(solver, A, b, x, n, tol, hist, hist_cap);
  }
  // F2H: fp64 / fp16 (A16, 64) / M
  auto inner = FGMRES<h16, tag>(A16, M, {64, false});
  auto solver_ = Solver<tag>(FGMRES<double, tag>(A, inner, {100, true}));
  auto solver = Restarted<double, tag>(A, solver_, {restarts});
  return refc::run_solve(solver, A, b, x, n, tol, hist, hist_cap);
}

}  // namespace

// out[0..4] = time_s, iters, impl_res, expl_res, solved; returns n_hist
extern "C" __attribute__((visibility("default"))) int ref_f3r_solve_depth_half(
    int variant, int32_t n, int32_t nnz, const int32_t *rptr, const int32_t *idx, const double *val, const double *b,
    double *x, int restarts, double tol, double acc, int blocks, double *out, double *hist, int hist_cap) {
  refc::g_stop_after = 0;
  auto a = refc::make_csr(n, nnz, rptr, idx, val);
  refc::solve_out o = depth_half(a, b, x, variant, restarts, tol, acc, blocks, hist, hist_cap);
  out[0] = o.time_s;
  out[1] = o.iters;
  out[2] = o.impl_res;
  out[3] = o.expl_res;
  out[4] = o.solved;
  return o.n_hist;
}
