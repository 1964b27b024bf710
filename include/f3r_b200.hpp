// f3r_b200.hpp -- C++ adapter over the C ABI (f3r_b200.h) with the names and
// calling conventions of the reference's solver interface
// (library/umineko-sparse/models.hpp), so that a driver written against the
// reference keeps its solve call:
//
//     auto data = f3r::CSR::stencil27(192, 192, 192, 2, 0.5);   // io::mm::read_system ...
//     f3r::algorithm::scaling(data);                              // algorithm.hpp:45-59
//     f3r::Context ctx(0);
//     f3r::F3R solver(ctx, data, f3r::params{});                  // f3r-gpu.cpp:210-265
//     auto cond = [&](int i, double e) { return e / nrm_b < eps; };  // f3r-gpu.cpp:83-86
//     f3r::solve_res_t flag = solver.solve(b, x, cond);           // f3r-gpu.cpp:88
//
// Header-only; errors become f3r::error exceptions (the C ABI returns codes).
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "f3r_b200.h"

namespace f3r {

struct error : std::runtime_error {
  f3r_status status;
  error(f3r_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

inline void check(f3r_status s) {
  if (s != F3R_SUCCESS)
    throw error(s, std::string(f3r_status_string(s)) + ": " + f3r_last_error_string());
}

// kmm::solve_res_t (models.hpp:191-200)
struct solve_res_t {
  bool is_solved = false;
  int32_t res_iter = 0;
  double res_nrm2 = 0;
  void operator+=(const solve_res_t &in) {
    is_solved = is_solved || in.is_solved;
    res_iter = res_iter + in.res_iter;
    res_nrm2 = in.res_nrm2;
  }
};

// Host CSR matrix (kmm::CSR<double, host>, csr.hpp:12-30), owned.
class CSR {
 public:
  CSR() = default;
  CSR(int32_t n, int32_t m, const std::vector<int32_t> &rptr, const std::vector<int32_t> &idx,
      const std::vector<double> &val) {
    f3r_csr v{n, m, (int32_t)idx.size(), rptr.data(), idx.data(), val.data()};
    f3r_host_matrix *h = nullptr;
    check(f3r_host_matrix_from_csr(&v, &h));
    h_.reset(h, f3r_host_matrix_destroy);
  }
  static CSR stencil27(int32_t nx, int32_t ny, int32_t nz, int32_t variant = 0, double beta = 0.5) {
    f3r_host_matrix *h = nullptr;
    check(f3r_problem_stencil27(nx, ny, nz, variant, beta, &h));
    return CSR(h);
  }
  f3r_csr view() const {
    f3r_csr v{};
    check(f3r_host_matrix_view(h_.get(), &v));
    return v;
  }
  int32_t nrows() const { return view().nrows; }
  int32_t ncols() const { return view().ncols; }
  int32_t nnz() const { return view().nnz; }
  f3r_host_matrix *handle() const { return h_.get(); }
  // takes ownership of a matrix returned by the C ABI
  static CSR adopt(f3r_host_matrix *h) { return CSR(h); }
  // y = A x on the host in fp64
  void operate(const double *x, double *y) const {
    f3r_csr v = view();
    check(f3r_host_spmv(&v, x, y));
  }

 private:
  explicit CSR(f3r_host_matrix *h) : h_(h, f3r_host_matrix_destroy) {}
  std::shared_ptr<f3r_host_matrix> h_;
};

// kmm::io::mm (matrix/io.hpp:89-217): Matrix Market files either side of the solve.
namespace io {
namespace mm {
// io::mm::read_matrix + io::CSR(COO) (io.hpp:91-96, 44-60)
inline CSR read_matrix(const std::string &path) {
  f3r_host_matrix *h = nullptr;
  check(f3r_mm_read(path.c_str(), &h));
  return CSR::adopt(h);
}
// io::mm::read_system (io.hpp:104-126) with the drivers' init: b from
// "<stem>_b.mtx" when present, else U(0, 1) from std::mt19937_64(0)
inline std::pair<CSR, std::vector<double>> read_system(const std::string &path, bool *b_from_file = nullptr) {
  CSR a = read_matrix(path);
  std::vector<double> b(a.nrows());
  int32_t ff = 0;
  check(f3r_mm_read_rhs(path.c_str(), (int64_t)b.size(), b.data(), &ff));
  if (b_from_file) *b_from_file = ff != 0;
  return {std::move(a), std::move(b)};
}
inline void write(const std::string &path, const CSR &a) {
  f3r_csr v = a.view();
  check(f3r_mm_write(path.c_str(), &v));
}
inline void write_vector(const std::string &path, const std::vector<double> &x) {
  check(f3r_mm_write_vector(path.c_str(), (int64_t)x.size(), x.data()));
}
}  // namespace mm
}  // namespace io

namespace algorithm {
// kmm::algorithm::scaling (algorithm.hpp:45-59)
inline void scaling(CSR &a) { check(f3r_host_scaling(a.handle())); }
// kmm::algorithm::sdainv (preconditioner/ainv.hpp:27-65): {Z, W^T}, M r = Z (W^T r)
inline std::pair<CSR, CSR> sdainv(const CSR &a, double tol = 0.1, double acc = 1.0) {
  f3r_csr v = a.view();
  f3r_host_matrix *z = nullptr, *wt = nullptr;
  check(f3r_host_sdainv(&v, tol, acc, &z, &wt));
  return {CSR::adopt(z), CSR::adopt(wt)};
}
}  // namespace algorithm

class Context {
 public:
  explicit Context(int32_t device = 0) {
    f3r_context *c = nullptr;
    check(f3r_context_create(device, &c));
    c_.reset(c, f3r_context_destroy);
  }
  void set_stream(void *cuda_stream) { check(f3r_context_set_stream(c_.get(), cuda_stream)); }
  void synchronize() { check(f3r_context_synchronize(c_.get())); }
  f3r_context *handle() const { return c_.get(); }

 private:
  std::shared_ptr<f3r_context> c_;
};

// Device SELL-C-sigma matrix with the operate / compute_residual surface of
// kmm::CoefficientMatrix (models.hpp:128-189); vectors are device pointers.
class SELL {
 public:
  SELL(Context &ctx, const CSR &a, int32_t sigma = 1,
       int32_t dtypes = (1 << F3R_F64) | (1 << F3R_F32) | (1 << F3R_F16)) {
    f3r_csr v = a.view();
    f3r_sell *m = nullptr;
    check(f3r_sell_create(ctx.handle(), &v, 32, sigma, dtypes, &m));
    m_.reset(m, f3r_sell_destroy);
  }
  void operate(f3r_dtype val_t, f3r_dtype in_t, const void *in, f3r_dtype out_t, void *out) const {
    check(f3r_sell_operate(m_.get(), val_t, in_t, in, out_t, out));
  }
  void compute_residual(f3r_dtype val_t, f3r_dtype t, const void *rhs, const void *in, void *res) const {
    check(f3r_sell_compute_residual(m_.get(), val_t, t, rhs, t, in, t, res));
  }
  f3r_sell_info info() const {
    f3r_sell_info i{};
    check(f3r_sell_info_get(m_.get(), &i));
    return i;
  }

 private:
  std::shared_ptr<f3r_sell> m_;
};

struct params : f3r_params {
  params() { f3r_params_default(this); }
};

// The nested F3R solver; models kmm::Solver (models.hpp:202-267):
// solve(b, x, cond) -> solve_res_t with cond(i, |e|) called after every
// outer Arnoldi step.  b and x may be host or device pointers.
class F3R {
 public:
  F3R(Context &ctx, const CSR &a, const params &p) {
    f3r_csr v = a.view();
    f3r_solver *s = nullptr;
    check(f3r_solver_create(ctx.handle(), &v, &p, &s));
    s_.reset(s, f3r_solver_destroy);
  }
  // SDAINV factors given instead of computed (f3r_solver_create_factors), e.g.
  // algorithm::sdainv's with values corrected by f3r_learned_correct
  F3R(Context &ctx, const CSR &a, const params &p, const CSR &z, const CSR &wt) {
    f3r_csr v = a.view(), zv = z.view(), wv = wt.view();
    f3r_solver *s = nullptr;
    check(f3r_solver_create_factors(ctx.handle(), &v, &p, &zv, &wv, &s));
    s_.reset(s, f3r_solver_destroy);
  }
  solve_res_t solve(const double *b, double *x, const std::function<bool(int, double)> &cond,
                    f3r_result *detail = nullptr) const {
    f3r_result r{};
    if (cond) {
      auto tramp = [](int32_t i, double e, void *u) -> int {
        return (*static_cast<const std::function<bool(int, double)> *>(u))(i, e) ? 1 : 0;
      };
      check(f3r_solver_solve(s_.get(), b, x, tramp, (void *)&cond, &r));
    } else {
      check(f3r_solver_solve(s_.get(), b, x, nullptr, nullptr, &r));
    }
    if (detail) *detail = r;
    solve_res_t out;
    out.is_solved = r.is_solved != 0;
    out.res_iter = r.res_iter;
    out.res_nrm2 = r.res_nrm2;
    return out;
  }
  // Solver::solve(in, out) without a stop test: the params' rel_tol applies
  void solve(const double *b, double *x) const { solve(b, x, nullptr); }
  // nrhs systems: column k of B (b + k * ld) into column k of X (x + k * ld)
  std::vector<f3r_result> solve_multi(int32_t nrhs, const double *b, double *x, int64_t ld) const {
    std::vector<f3r_result> r(nrhs > 0 ? nrhs : 0);
    check(f3r_solver_solve_multi(s_.get(), nrhs, b, ld, x, ld, nullptr, nullptr, r.data()));
    return r;
  }
  f3r_solver *handle() const { return s_.get(); }

 private:
  std::shared_ptr<f3r_solver> s_;
};

}  // namespace f3r
