// ref_lib.cpp -- TEST INFRASTRUCTURE: a C interface over the reference
// library's own templates (compiled from the reference headers in place) so
// that tests/golden/gen_golden.py can record golden vectors from the
// reference itself.  Built into oracle/_ref/libf3r_ref.so by oracle/Makefile.
#include <cstring>
#include <memory>

#include "ref_compose.hpp"

using namespace kmm;
using refc::h16;

namespace {
struct pair_t {
  CSR<double, host> a, b;
};
void copy_csr(const CSR<double, host> &m, int32_t *rptr, int32_t *idx, double *val) {
  std::memcpy(rptr, m.rptr.raw(), sizeof(int32_t) * (m.nrows() + 1));
  std::memcpy(idx, m.idx.raw(), sizeof(int32_t) * m.nnz());
  std::memcpy(val, m.val.raw(), sizeof(double) * m.nnz());
}
}  // namespace

extern "C" {

// algorithm::scaling (algorithm.hpp:45-59), in place
void ref_scaling(int32_t n, int32_t nnz, const int32_t *rptr, const int32_t *idx, double *val) {
  auto a = refc::make_csr(n, nnz, rptr, idx, val);
  algorithm::scaling(a);
  std::memcpy(val, a.val.raw(), sizeof(double) * nnz);
}

// SELL<32> construction (sell.hpp:46-49, 249-307)
void *ref_sell32_build(int32_t n, int32_t nnz, const int32_t *rptr, const int32_t *idx,
                       const double *val) {
  auto a = refc::make_csr(n, nnz, rptr, idx, val);
  return new SELL<32, double, host>(a);
}
int64_t ref_sell32_size(void *h) { return ((SELL<32, double, host> *)h)->val.size(0); }
int32_t ref_sell32_nslice(void *h) { return ((SELL<32, double, host> *)h)->sptr.size(0) - 1; }
void ref_sell32_copy(void *h, int32_t *sptr, int32_t *sidx, double *sval) {
  auto *s = (SELL<32, double, host> *)h;
  std::memcpy(sptr, s->sptr.raw(), sizeof(int32_t) * s->sptr.size(0));
  std::memcpy(sidx, s->idx.raw(), sizeof(int32_t) * s->idx.size(0));
  std::memcpy(sval, s->val.raw(), sizeof(double) * s->val.size(0));
}
void ref_sell32_free(void *h) { delete (SELL<32, double, host> *)h; }

// SELL<32>::operate / compute_residual (sell.hpp:56-89) at the types the F3R
// levels use.  kind 0: fp64 A, fp64 x -> fp64.  1: fp32 A, fp32 x -> fp32.
// 2: fp16 A, fp32 x -> fp32 (level 3).  3: fp16 A, fp16 x -> fp16 (level 4).
void ref_sell32_operate(void *h, int kind, const void *x, void *y) {
  auto *s = (SELL<32, double, host> *)h;
  const int32_t n = s->nrows();
  if (kind == 0) {
    auto xv = vector<double, host>(n), yv = vector<double, host>(n);
    std::memcpy(xv.raw(), x, 8 * n);
    s->operate(xv, yv);
    std::memcpy(y, yv.raw(), 8 * n);
  } else if (kind == 1) {
    auto a = SELL<32, float, host>(*s);
    auto xv = vector<float, host>(n), yv = vector<float, host>(n);
    std::memcpy(xv.raw(), x, 4 * n);
    a.operate(xv, yv);
    std::memcpy(y, yv.raw(), 4 * n);
  } else if (kind == 2) {
    auto a = SELL<32, h16, host>(*s);
    auto xv = vector<float, host>(n), yv = vector<float, host>(n);
    std::memcpy(xv.raw(), x, 4 * n);
    a.operate(xv, yv);
    std::memcpy(y, yv.raw(), 4 * n);
  } else {
    auto a = SELL<32, h16, host>(*s);
    auto xv = vector<h16, host>(n), yv = vector<h16, host>(n);
    std::memcpy(xv.raw(), x, 2 * n);
    a.operate(xv, yv);
    std::memcpy(y, yv.raw(), 2 * n);
  }
}
// kind 0: fp64 residual; kind 3: fp16 residual (rhs, in, res all fp16)
void ref_sell32_residual(void *h, int kind, const void *b, const void *x, void *r) {
  auto *s = (SELL<32, double, host> *)h;
  const int32_t n = s->nrows();
  if (kind == 0) {
    auto bv = vector<double, host>(n), xv = vector<double, host>(n), rv = vector<double, host>(n);
    std::memcpy(bv.raw(), b, 8 * n);
    std::memcpy(xv.raw(), x, 8 * n);
    s->compute_residual(bv, xv, rv);
    std::memcpy(r, rv.raw(), 8 * n);
  } else {
    auto a = SELL<32, h16, host>(*s);
    auto bv = vector<h16, host>(n), xv = vector<h16, host>(n), rv = vector<h16, host>(n);
    std::memcpy(bv.raw(), b, 2 * n);
    std::memcpy(xv.raw(), x, 2 * n);
    a.compute_residual(bv, xv, rv);
    std::memcpy(r, rv.raw(), 2 * n);
  }
}

// algorithm::sdainv (ainv.hpp:27-65): returns {Z, Wt}
void *ref_sdainv(int32_t n, int32_t nnz, const int32_t *rptr, const int32_t *idx,
                 const double *val, double tol, double acc) {
  auto a = refc::make_csr(n, nnz, rptr, idx, val);
  auto [z, w] = algorithm::sdainv(a, tol, acc);
  return new pair_t{z, w};
}
// block-Jacobi ILU(0) as f3r.cpp:57-58: returns {L, U}
void *ref_ilu0_bj(int32_t n, int32_t nnz, const int32_t *rptr, const int32_t *idx,
                  const double *val, int blocks, double acc) {
  auto a = refc::make_csr(n, nnz, rptr, idx, val);
  auto bd = a.duplicate_block_diagonal(blocks, 1);
  auto [l, u] = algorithm::split(algorithm::ilup(bd, 0, acc, blocks, 1));
  return new pair_t{l, u};
}
int32_t ref_pair_nnz(void *h, int which) {
  auto *p = (pair_t *)h;
  return which == 0 ? p->a.nnz() : p->b.nnz();
}
void ref_pair_copy(void *h, int which, int32_t *rptr, int32_t *idx, double *val) {
  auto *p = (pair_t *)h;
  copy_csr(which == 0 ? p->a : p->b, rptr, idx, val);
}
// BJ triangular solves in fp16 (bj.hpp:58-98) on an ILU pair
void ref_bj_solve_f16(void *h, int blocks, int upper, const uint16_t *in, uint16_t *out) {
  auto *p = (pair_t *)h;
  const int32_t n = p->a.nrows();
  auto iv = vector<h16, host>(n), ov = vector<h16, host>(n);
  std::memcpy(iv.raw(), in, 2 * n);
  if (!upper) {
    auto L = trsv::l::BJ<CSR<h16, host>>(p->a, {blocks});
    L.solve(iv, ov);
  } else {
    auto U = trsv::du::BJ<CSR<h16, host>>(p->b, {blocks});
    U.solve(iv, ov);
  }
  std::memcpy(out, ov.raw(), 2 * n);
}
void ref_pair_free(void *h) { delete (pair_t *)h; }

// Jacobi-iteration triangular solves in fp16: Jacobi on SELL<32>
// (trsv/jacobi.hpp:290-505, kind 0), BAJ on SELL<32> (trsv/baj.hpp:95-190,
// kind 1), and the same two on CSR (jacobi.hpp:27-141, baj.hpp:27-93; kinds
// 2, 3); form 0 lower (unit diagonal last), 1 lower_d (diagonal last),
// 2 d_upper (diagonal first).
void ref_jacobi_trsv_f16(int32_t n, int32_t nnz, const int32_t *rptr, const int32_t *idx, const double *val,
                         int form, int kind, int iters, double omega, const uint16_t *in, uint16_t *out) {
  auto m = refc::make_csr(n, nnz, rptr, idx, val);
  auto iv = vector<h16, host>(n), ov = vector<h16, host>(n);
  std::memcpy(iv.raw(), in, 2 * n);
  if (kind == 0) {
    if (form == 0) trsv::l::Jacobi<SELL<32, h16, host>>(m, {iters, omega}).solve(iv, ov);
    if (form == 1) trsv::ld::Jacobi<SELL<32, h16, host>>(m, {iters, omega}).solve(iv, ov);
    if (form == 2) trsv::du::Jacobi<SELL<32, h16, host>>(m, {iters, omega}).solve(iv, ov);
  } else if (kind == 1) {
    if (form == 0) trsv::l::BAJ<SELL<32, h16, host>>(m, {iters, omega}).solve(iv, ov);
    if (form == 1) trsv::ld::BAJ<SELL<32, h16, host>>(m, {iters, omega}).solve(iv, ov);
    if (form == 2) trsv::du::BAJ<SELL<32, h16, host>>(m, {iters, omega}).solve(iv, ov);
  } else if (kind == 2) {
    if (form == 0) trsv::l::Jacobi<CSR<h16, host>>(m, {iters, omega}).solve(iv, ov);
    if (form == 1) trsv::ld::Jacobi<CSR<h16, host>>(m, {iters, omega}).solve(iv, ov);
    if (form == 2) trsv::du::Jacobi<CSR<h16, host>>(m, {iters, omega}).solve(iv, ov);
  } else {
    if (form == 0) trsv::l::BAJ<CSR<h16, host>>(m, {iters, omega}).solve(iv, ov);
    if (form == 1) trsv::ld::BAJ<CSR<h16, host>>(m, {iters, omega}).solve(iv, ov);
    if (form == 2) trsv::du::BAJ<CSR<h16, host>>(m, {iters, omega}).solve(iv, ov);
  }
  std::memcpy(out, ov.raw(), 2 * n);
}

// Full F3R solves (stop_after > 0: only that many outer steps).  config 0: SDAINV + SELL-32 (f3r-gpu.cpp:210-265);
// config 1: BJ-ILU(0) + CSR (f3r.cpp:195-248); config 2: F3R-Static with
// weight `weight` over BJ-ILU(0) (static.cpp:99-119); configs 3 / 4: the
// depth-3 / depth-2 fp32 ablations over BJ-ILU(0) (depth.cpp:140-162).  A
// must already be scaled.
// out[0..4] = time_s, iters, impl_res, expl_res, solved; returns n_hist.
int ref_f3r_solve(int config, int32_t n, int32_t nnz, const int32_t *rptr, const int32_t *idx,
                  const double *val, const double *b, double *x, int m2, int m3, int m4, int c,
                  int restarts, double tol, double acc, double sdainv_tol, int blocks,
                  double *out, double *hist, int hist_cap, int stop_after, double weight) {
  refc::g_stop_after = stop_after;
  auto a = refc::make_csr(n, nnz, rptr, idx, val);
  refc::solve_out o;
  if (config == 0)
    o = refc::f3r_sdainv_sell(a, b, x, m2, m3, m4, c, restarts, tol, acc, sdainv_tol, hist, hist_cap);
  else if (config == 1)
    o = refc::f3r_bjilu_csr(a, b, x, m2, m3, m4, c, restarts, tol, acc, blocks, hist, hist_cap);
  else if (config == 2)
    o = refc::f3r_static_bjilu_csr(a, b, x, m2, m3, m4, weight, restarts, tol, acc, blocks, hist, hist_cap);
  else
    o = refc::depth_bjilu_csr(a, b, x, config == 3 ? 3 : 2, m2, m3, restarts, tol, acc, blocks, hist, hist_cap);
  out[0] = o.time_s;
  out[1] = o.iters;
  out[2] = o.impl_res;
  out[3] = o.expl_res;
  out[4] = o.solved;
  return o.n_hist;
}

}  // extern "C"
