// ref_compose.hpp -- TEST INFRASTRUCTURE: assembles the reference's own F3R
// solver from the reference library headers (umineko-core / umineko-sparse),
// exactly as its experiment drivers do, but with the host execution tag so
// it runs on CPU cores.  Compiled only into oracle/_ref/ (see oracle/Makefile),
// never into the product.
//
//  * f3r_sdainv_sell: the GPU configuration, work/src/f3r-gpu.cpp:210-265
//    (SELL-32 matrices, SDAINV innermost, fp16 Richardson), with the CUDA
//    __half replaced by the host _Float16 type and tag=host.
//  * f3r_bjilu_csr: the CPU configuration, work/src/f3r.cpp:195-248
//    (CSR matrices, block-Jacobi ILU(0) with 112 blocks).
//
// The solve is timed as the drivers do (only solver.solve, f3r-gpu.cpp:87-89)
// and the stop test is the drivers' cond lambda (f3r-gpu.cpp:83-86) with the
// tolerance passed in instead of the hard-coded 1e-8.
#pragma once

#include <chrono>
#include <cstring>
#include <vector>

#include "umineko-sparse/matrix/algorithm.hpp"
#include "umineko-sparse/matrix/csr.hpp"
#include "umineko-sparse/matrix/io.hpp"
#include "umineko-sparse/matrix/sell.hpp"
#include "umineko-sparse/preconditioner/ainv.hpp"
#include "umineko-sparse/preconditioner/ilu.hpp"
#include "umineko-sparse/solver/gmres.hpp"
#include "umineko-sparse/solver/restart.hpp"
#include "umineko-sparse/trsv/baj.hpp"
#include "umineko-sparse/trsv/bj.hpp"
#include "umineko-sparse/trsv/jacobi.hpp"

namespace refc {

using namespace kmm;
using h16 = _Float16;

struct solve_out {
  double time_s = 0;
  int iters = 0;        // outer FGMRES steps (solve_res_t::res_iter)
  double impl_res = 0;  // |e| / ||b||
  double expl_res = 0;  // ||b - A x|| / ||b|| in fp64
  int solved = 0;
  int n_hist = 0;
};

inline CSR<double, host> make_csr(int32_t n, int32_t nnz, const int32_t *rptr,
                                  const int32_t *idx, const double *val) {
  auto a = CSR<double, host>(impl::shape{n, n}, nnz);
  std::memcpy(a.rptr.raw(), rptr, sizeof(int32_t) * (n + 1));
  std::memcpy(a.idx.raw(), idx, sizeof(int32_t) * nnz);
  std::memcpy(a.val.raw(), val, sizeof(double) * nnz);
  return a;
}

// stop_after > 0 ends the solve after that many outer steps through the
// reference's own cond callback (a bounded sample of the solve).
inline int g_stop_after = 0;

template <class Solver, class Mat>
solve_out run_solve(const Solver &solver, const Mat &A, const double *b_in, double *x_out,
                    int32_t n, double tol, double *hist, int hist_cap) {
  auto b = vector<double, host>(n);
  std::memcpy(b.raw(), b_in, sizeof(double) * n);
  auto x = vector<double, host>(n);
  auto r = vector<double, host>(n);
  x.fill(0.0);
  scalar<double, host> nrm_b, nrm_r;
  nrm_b = nrm(b);
  solve_out o;
  int nh = 0;
  auto cond = [&, nb = nrm_b[0]](int i, double e) {
    if (i > 0) {
      if (nh < hist_cap) hist[nh] = e / nb;
      nh++;
    }
    if (g_stop_after > 0 && i >= g_stop_after) return true;
    return e / nb < tol;
  };
  auto t0 = std::chrono::steady_clock::now();
  auto flag = solver.solve(b, x, cond);
  auto t1 = std::chrono::steady_clock::now();
  o.time_s = std::chrono::duration<double>(t1 - t0).count();
  o.iters = flag.res_iter;
  o.impl_res = flag.res_nrm2 / nrm_b[0];
  o.solved = flag.is_solved ? 1 : 0;
  A.operate(x, r);
  r = b - r;
  nrm_r = nrm(r);
  o.expl_res = nrm_r[0] / nrm_b[0];
  o.n_hist = nh;
  std::memcpy(x_out, x.raw(), sizeof(double) * n);
  return o;
}

// f3r-gpu.cpp:210-265 on the host.  `data` is the already scaled matrix.
// Level2 / Level3 are the solver class templates of the two inner levels
// (FGMRES as the driver; sFGMRES of solver/gmres2.hpp:137-221 in
// ref_sstep.cpp).
template <template <class, class> class Level2, template <class, class> class Level3>
solve_out f3r_sdainv_sell_t(const CSR<double, host> &data, const double *b, double *x,
                            int m2, int m3, int m4, int c, int restarts, double tol,
                            double acc, double sdainv_tol, double *hist, int hist_cap) {
  using tag = host;
  const int32_t n = data.nrows();
  auto A = SELL<32, double, tag>(data);
  impl::pool<double, tag>::init(n);
  impl::pool<float, tag>::init(n);
  impl::pool<h16, tag>::init(n);
  auto [z, w] = algorithm::sdainv(data, sdainv_tol, acc);

  const int period = c;
  int cnt = c;
  scalar<int, tag> den;
  scalar<float, tag> dot_ar, dot_r;
  auto A16 = SELL<32, h16, tag>(A);
  auto W = SELL<32, h16, tag>(w);
  auto Z = SELL<32, h16, tag>(z);
  auto tmp = vector<h16, tag>(n);
  auto tmp2 = vector<h16, tag>(n);
  auto hin = vector<h16, tag>(n);
  auto hout = vector<h16, tag>(n);
  auto hr = vector<h16, tag>(n);
  std::vector<scalar<float, tag>> sum(m4);
  std::vector<scalar<h16, tag>> ome(m4);
  auto tof32 = [](auto v) { return static_cast<float>(v); };
  auto R = Operator<tag>(data.get_shape(), [&](auto in, auto out) {
    ++cnt;
    hin.copy(in);
    W.operate(hin, tmp);
    Z.operate(tmp, hout);
    if (cnt % period == 0) {
      A16.operate(hout, tmp);
      dot_ar = dot(wildcard(tmp, tof32), wildcard(tmp, tof32));
      dot_r = dot(wildcard(tmp, tof32), wildcard(hin, tof32));
      hout *= dot_r / dot_ar;
      sum[0] += dot_r / dot_ar;
      ome[0] = sum[0] / (den = cnt / period);
    } else {
      hout *= ome[0];
    }
    for (int k = 1; k < m4; k++) {
      A16.compute_residual(hin, hout, hr);
      W.operate(hr, tmp);
      Z.operate(tmp, tmp2);
      if (cnt % period == 0) {
        A16.operate(tmp2, tmp);
        dot_ar = dot(wildcard(tmp, tof32), wildcard(tmp, tof32));
        dot_r = dot(wildcard(tmp, tof32), wildcard(hr, tof32));
        hout += dot_r / dot_ar * tmp2;
        sum[k] += dot_r / dot_ar;
        ome[k] = sum[k] / den;
      } else {
        hout += ome[k] * tmp2;
      }
    }
    out.copy(hout);
  });
  auto A32 = SELL<32, float, tag>(A);
  auto MM = Level3<float, tag>(A16, R, {m3, false});
  auto MMM = Level2<float, tag>(A32, MM, {m2, false});
  auto inner = Solver<tag>(FGMRES<double, tag>(A, MMM, {100, true}));
  auto solver = Restarted<double, tag>(A, inner, {restarts});
  cnt = c;
  for (int k = 0; k < m4; k++) {
    sum[k] = 1.0;
    ome[k] = 1.0;
  }
  return run_solve(solver, A, b, x, n, tol, hist, hist_cap);
}

inline solve_out f3r_sdainv_sell(const CSR<double, host> &data, const double *b, double *x,
                                 int m2, int m3, int m4, int c, int restarts, double tol,
                                 double acc, double sdainv_tol, double *hist, int hist_cap) {
  return f3r_sdainv_sell_t<FGMRES, FGMRES>(data, b, x, m2, m3, m4, c, restarts, tol, acc, sdainv_tol,
                                           hist, hist_cap);
}

// f3r.cpp:195-248 (HALF) on the host: CSR, block-Jacobi ILU(0).
inline solve_out f3r_bjilu_csr(const CSR<double, host> &data, const double *b, double *x, int m2,
                               int m3, int m4, int c, int restarts, double tol, double acc,
                               int blocks, double *hist, int hist_cap) {
  using tag = host;
  const int32_t n = data.nrows();
  auto A = CSR<double, tag>(data);
  impl::pool<double, tag>::init(n);
  impl::pool<float, tag>::init(n);
  impl::pool<h16, tag>::init(n);
  auto bd = data.duplicate_block_diagonal(blocks, 1);
  auto [l, u] = algorithm::split(algorithm::ilup(bd, 0, acc, blocks, 1));

  const int period = c;
  int cnt = c;
  scalar<int, tag> den;
  scalar<float, tag> dot_ar, dot_r;
  auto A16 = CSR<h16, tag>(A);
  auto L = trsv::l::BJ<CSR<h16, host>>(l, {blocks});
  auto U = trsv::du::BJ<CSR<h16, host>>(u, {blocks});
  auto tmp = vector<h16, tag>(n);
  auto tmp2 = vector<h16, tag>(n);
  auto hin = vector<h16, tag>(n);
  auto hout = vector<h16, tag>(n);
  auto hr = vector<h16, tag>(n);
  std::vector<scalar<float, tag>> sum(m4);
  std::vector<scalar<h16, tag>> ome(m4);
  auto tof32 = [](auto v) { return static_cast<float>(v); };
  auto R = Operator<tag>(data.get_shape(), [&](auto in, auto out) {
    ++cnt;
    hin.copy(in);
    L.solve(hin, tmp);
    U.solve(tmp, hout);
    if (cnt % period == 0) {
      A16.operate(hout, tmp);
      dot_ar = dot(wildcard(tmp, tof32), wildcard(tmp, tof32));
      dot_r = dot(wildcard(tmp, tof32), wildcard(hin, tof32));
      hout *= dot_r / dot_ar;
      sum[0] += dot_r / dot_ar;
      ome[0] = sum[0] / (den = cnt / period);
    } else {
      hout *= ome[0];
    }
    for (int k = 1; k < m4; k++) {
      A16.compute_residual(hin, hout, hr);
      L.solve(hr, tmp);
      U.solve(tmp, tmp2);
      if (cnt % period == 0) {
        A16.operate(tmp2, tmp);
        dot_ar = dot(wildcard(tmp, tof32), wildcard(tmp, tof32));
        dot_r = dot(wildcard(tmp, tof32), wildcard(hr, tof32));
        hout += dot_r / dot_ar * tmp2;
        sum[k] += dot_r / dot_ar;
        ome[k] = sum[k] / den;
      } else {
        hout += ome[k] * tmp2;
      }
    }
    out.copy(hout);
  });
  auto A32 = CSR<float, tag>(A);
  auto MM = FGMRES<float, tag>(A16, R, {m3, false});
  auto MMM = FGMRES<float, tag>(A32, MM, {m2, false});
  auto inner = Solver<tag>(FGMRES<double, tag>(A, MMM, {100, true}));
  auto solver = Restarted<double, tag>(A, inner, {restarts});
  cnt = c;
  for (int k = 0; k < m4; k++) {
    sum[k] = 1.0;
    ome[k] = 1.0;
  }
  return run_solve(solver, A, b, x, n, tol, hist, hist_cap);
}

// F3R-Static (work/src/static.cpp:99-119): the fixed-weight Richardson over
// BJ-ILU(0) in fp16, CSR matrices.
inline solve_out f3r_static_bjilu_csr(const CSR<double, host> &data, const double *b, double *x, int m2, int m3,
                                      int m4, double weight, int restarts, double tol, double acc, int blocks,
                                      double *hist, int hist_cap) {
  using tag = host;
  const int32_t n = data.nrows();
  auto A = CSR<double, tag>(data);
  impl::pool<double, tag>::init(n);
  impl::pool<float, tag>::init(n);
  impl::pool<h16, tag>::init(n);
  auto bd = data.duplicate_block_diagonal(blocks, 1);
  auto [l, u] = algorithm::split(algorithm::ilup(bd, 0, acc, blocks, 1));
  auto A16 = CSR<h16, tag>(A);
  auto L = trsv::l::BJ<CSR<h16, host>>(l, {blocks});
  auto U = trsv::du::BJ<CSR<h16, host>>(u, {blocks});
  auto tmp = vector<h16, tag>(n);
  auto tmp2 = vector<h16, tag>(n);
  auto hin = vector<h16, tag>(n);
  auto hout = vector<h16, tag>(n);
  auto hr = vector<h16, tag>(n);
  scalar<h16, tag> ome;
  ome.fill(h16(weight));
  auto R = Operator<tag>(data.get_shape(), [&](auto in, auto out) {
    hin.copy(in);
    L.solve(hin, tmp);
    U.solve(tmp, hout);
    hout *= ome;
    for (int k = 1; k < m4; k++) {
      A16.compute_residual(hin, hout, hr);
      L.solve(hr, tmp);
      U.solve(tmp, tmp2);
      hout += ome * tmp2;
    }
    out.copy(hout);
  });
  auto A32 = CSR<float, tag>(A);
  auto MM = FGMRES<float, tag>(A16, R, {m3, false});
  auto MMM = FGMRES<float, tag>(A32, MM, {m2, false});
  auto inner = Solver<tag>(FGMRES<double, tag>(A, MMM, {100, true}));
  auto solver = Restarted<double, tag>(A, inner, {restarts});
  return run_solve(solver, A, b, x, n, tol, hist, hist_cap);
}

// Depth ablations with fp32 levels (work/src/depth.cpp:122-162): M is the
// fp16 BJ-ILU(0) sweep pair; depth 3 = FGMRES<float>(A32, FGMRES<float>(A16,
// M, m3), m2), depth 2 = FGMRES<float>(A32, M, m2).
inline solve_out depth_bjilu_csr(const CSR<double, host> &data, const double *b, double *x, int depth, int m2,
                                 int m3, int restarts, double tol, double acc, int blocks, double *hist,
                                 int hist_cap) {
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
  if (depth == 3) {
    auto F = FGMRES<float, tag>(A16, M, {m3, false});
    auto inner = FGMRES<float, tag>(A32, F, {m2, false});
    auto solver_ = Solver<tag>(FGMRES<double, tag>(A, inner, {100, true}));
    auto solver = Restarted<double, tag>(A, solver_, {restarts});
    return run_solve(solver, A, b, x, n, tol, hist, hist_cap);
  }
  auto inner = FGMRES<float, tag>(A32, M, {m2, false});
  auto solver_ = Solver<tag>(FGMRES<double, tag>(A, inner, {100, true}));
  auto solver = Restarted<double, tag>(A, solver_, {restarts});
  return run_solve(solver, A, b, x, n, tol, hist, hist_cap);
}

}  // namespace refc
