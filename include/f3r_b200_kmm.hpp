// f3r_b200_kmm.hpp -- the nested F3R solver as an object of the reference's
// own solver concept, so that a driver written against the reference keeps
// its solver call unchanged.
//
// The reference's plugin surface is kmm::Solver<L> (library/umineko-sparse/
// models.hpp:202-267): a type-erased wrapper around any object that has
//
//     solve_res_t solve(const vector<T1, L> &b, vector<T2, L> x,
//                       const std::function<bool(int, double)> &cond) const;
//     void        solve(const vector<T1, L> &b, vector<T2, L> x) const;
//     void        operate(const vector<T1, L> &in, vector<T2, L> out) const;
//     idx_t       nrows() const, ncols() const;
//
// for T1, T2 in {double, float}.  f3r::kmm::F3R<L> is such an object.  The
// drivers build their solver as Restarted<double, tag>(A, Solver<tag>(
// FGMRES<double, tag>(A, inner, {100, true})), {restart}) (work/src/
// f3r-gpu.cpp:262-265); the same driver can instead write
//
//     auto solver = kmm::Solver<tag>(f3r::kmm::F3R<tag>(data, params));
//     auto flag = solver.solve(b, x, cond);            // f3r-gpu.cpp:88, unchanged
//
// where data is the scaled kmm::CSR<double, host> the driver already holds
// (f3r-gpu.cpp:63-65).  The solve runs on the GPU through the C ABI
// (f3r_b200.h): Restarted( FGMRES<double>( A, FGMRES<float>(A32,
// FGMRES<float>(A16, R, m3), m2), m_outer), max_restarts ) with R the fp16
// adaptive-weight Richardson over SDAINV or block-Jacobi ILU(0), as
// f3r-gpu.cpp:210-265 assembles it.
//
// Include the reference headers (umineko-sparse/models.hpp, matrix/csr.hpp)
// before this file.  Vectors may live on the host (L = kmm::host) or on the
// device (L = kmm::device, CUDA device memory): double vectors are handed to
// the solver as they are, float vectors are widened through a host copy.
// cond(i, |e|) is called as the reference's FGMRES calls it: i = 0 with the
// initial residual of every restart, then after every outer Arnoldi step.
// Errors throw f3r::kmm::error (the reference prints and exits instead).
//
// Keep f3r and the reference's kmm namespace apart at the call site (no
// `using namespace f3r;` beside `using namespace kmm;`): f3r::kmm would make
// the name kmm ambiguous.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "f3r_b200.h"

#ifndef UMINEKO_SPARSE_MODELS_HPP
#error "include the reference's umineko-sparse/models.hpp and matrix/csr.hpp before f3r_b200_kmm.hpp"
#endif

namespace f3r {
namespace kmm {

struct error : std::runtime_error {
  f3r_status status;
  error(f3r_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

inline void check(f3r_status s) {
  if (s != F3R_SUCCESS) throw error(s, std::string(f3r_status_string(s)) + ": " + f3r_last_error_string());
}

inline f3r_params default_params() {
  f3r_params p;
  f3r_params_default(&p);
  return p;
}

template <class L = ::kmm::host> class F3R {
 public:
  template <typename val_t> using vec_t = ::kmm::vector<val_t, L>;

  // a: the system as solved (the drivers scale it first, f3r-gpu.cpp:65);
  // its arrays are copied to the device here, the preconditioner built here
  explicit F3R(const ::kmm::CSR<double, ::kmm::host> &a, const f3r_params &p = default_params(),
               int32_t device = 0) {
    f3r_context *c = nullptr;
    check(f3r_context_create(device, &c));
    ctx_.reset(c, f3r_context_destroy);
    const f3r_csr v{a.nrows(), a.ncols(), a.nnz(), a.rptr.raw(), a.idx.raw(), a.val.raw()};
    f3r_solver *s = nullptr;
    check(f3r_solver_create(c, &v, &p, &s));
    // the solver is released before the context it runs on
    std::shared_ptr<f3r_context> keep = ctx_;
    solver_.reset(s, [keep](f3r_solver *q) { f3r_solver_destroy(q); });
    n_ = a.nrows();
  }

  // Solver::solve(b, x, cond): x holds the initial guess and receives the
  // solution (Restarted::solve, solver/restart.hpp:26-36)
  template <typename T1, typename T2>
  ::kmm::solve_res_t solve(const vec_t<T1> &in, vec_t<T2> out, const std::function<bool(int, double)> &cond) const {
    static_assert(std::is_floating_point_v<T1> && std::is_floating_point_v<T2>, "double or float vectors");
    f3r_result r{};
    if constexpr (std::is_same_v<T1, double> && std::is_same_v<T2, double>) {
      run(in.raw(), out.raw(), cond, &r);
    } else {
      std::vector<double> b = widen(in), x = widen(out);
      run(b.data(), x.data(), cond, &r);
      narrow(x, out);
    }
    return ::kmm::solve_res_t{r.is_solved != 0, r.res_iter, r.res_nrm2};
  }

  // Solver::solve(b, x) with no stop test: f3r_params.rel_tol decides
  template <typename T1, typename T2> void solve(const vec_t<T1> &in, vec_t<T2> out) const {
    solve(in, out, std::function<bool(int, double)>());
  }

  // Solver::operate(in, out): the solver as an operator, out = A^-1 in from a
  // zero initial guess to f3r_params.rel_tol
  template <typename T1, typename T2> void operate(const vec_t<T1> &in, vec_t<T2> out) const {
    std::vector<double> b = widen(in), x(b.size(), 0.0);
    f3r_result r{};
    run(b.data(), x.data(), std::function<bool(int, double)>(), &r);
    narrow(x, out);
  }

  [[nodiscard]] ::kmm::idx_t nrows() const { return n_; }
  [[nodiscard]] ::kmm::idx_t ncols() const { return n_; }
  f3r_solver *handle() const { return solver_.get(); }

 private:
  void run(const double *b, double *x, const std::function<bool(int, double)> &cond, f3r_result *r) const {
    if (cond) {
      auto tramp = [](int32_t i, double e, void *u) -> int {
        return (*static_cast<const std::function<bool(int, double)> *>(u))(i, e) ? 1 : 0;
      };
      check(f3r_solver_solve(solver_.get(), b, x, tramp, (void *)&cond, r));
    } else {
      check(f3r_solver_solve(solver_.get(), b, x, nullptr, nullptr, r));
    }
  }
  // a vector of any element type and location as host doubles
  template <typename T> std::vector<double> widen(const vec_t<T> &v) const {
    std::vector<T> h((size_t)n_);
    ::kmm::memory<L>::template copy<::kmm::host>(v.raw(), h.data(), (size_t)n_);
    return std::vector<double>(h.begin(), h.end());
  }
  template <typename T> void narrow(const std::vector<double> &x, vec_t<T> out) const {
    std::vector<T> h(x.begin(), x.end());
    ::kmm::memory<::kmm::host>::template copy<L>(h.data(), out.raw(), (size_t)n_);
  }

  std::shared_ptr<f3r_context> ctx_;
  std::shared_ptr<f3r_solver> solver_;
  ::kmm::idx_t n_ = 0;
};

}  // namespace kmm
}  // namespace f3r
