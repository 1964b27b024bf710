// internal.hpp -- shared declarations of the f3r_b200 library (not installed).
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/f3r_b200.h"

struct f3r_host_matrix;

namespace f3r {

using Status = f3r_status;

// Records a message for f3r_last_error_string() and returns the code.
Status fail(Status code, const std::string &msg);

#define F3R_TRY(x)                    \
  do {                                \
    ::f3r::Status s_ = (x);           \
    if (s_ != F3R_SUCCESS) return s_; \
  } while (0)

struct HostCSR {
  int32_t n = 0, m = 0;
  std::vector<int32_t> rptr, idx;
  std::vector<double> val;
  HostCSR() = default;
  HostCSR(int32_t n_, int32_t m_, int64_t nnz_);
  f3r_csr view() const;
  int64_t nnz() const { return (int64_t)idx.size(); }
};

Status check_csr(const f3r_csr *a);
HostCSR *stencil27(int32_t nx, int32_t ny, int32_t nz, int32_t variant, double beta);
HostCSR *diffusion7(int32_t nx, int32_t ny, int32_t nz, double sigma, double corr_len, uint64_t seed);
void scaling(HostCSR &a);
void host_spmv(const f3r_csr &a, const double *x, double *y);
Status sdainv(const HostCSR &A, double tol, double acc, HostCSR **Z, HostCSR **Wt);
Status ilu0_bj(const HostCSR &A, int32_t blocks, double acc, HostCSR **L, HostCSR **U,
               std::vector<int32_t> *bptr);

// The context a solver runs on (solves sharing one must not overlap) and its
// row count (solver.cu).
const void *solver_context(const f3r_solver *s);
int32_t solver_rows(const f3r_solver *s);
// f3r_solver_solve_multi after its argument checks (solver.cu)
Status solver_solve_multi(f3r_solver *s, int32_t nrhs, const double *b, int64_t ldb, double *x, int64_t ldx,
                          f3r_cond_fn cond, void *user, f3r_result *results);

}  // namespace f3r

struct f3r_host_matrix {
  std::unique_ptr<f3r::HostCSR> m;
};
