// ref_sstep.cpp -- TEST INFRASTRUCTURE: the F3R solve of f3r-gpu.cpp with
// sFGMRES (umineko-sparse/solver/gmres2.hpp:137-221) at the inner levels,
// compiled from the reference headers in place.
//
// gmres2.hpp and gmres.hpp share one include guard and both define FGMRES,
// so this file is its own library (oracle/_ref/libf3r_ref_sstep.so, built
// with hidden visibility so its FGMRES instantiations never meet those of
// libf3r_ref.so).  <math.h> comes first so that the unqualified abs() on
// doubles inside gmres2.hpp binds to the floating-point overload.
#include <math.h>

#include "umineko-sparse/solver/gmres2.hpp"

#include "ref_compose.hpp"

extern "C" __attribute__((visibility("default"))) int ref_f3r_solve_sstep(
    int mask, int32_t n, int32_t nnz, const int32_t *rptr, const int32_t *idx, const double *val, const double *b,
    double *x, int m2, int m3, int m4, int c, int restarts, double tol, double acc, double sdainv_tol, double *out,
    double *hist, int hist_cap) {
  using namespace kmm;
  refc::g_stop_after = 0;
  auto a = refc::make_csr(n, nnz, rptr, idx, val);
  refc::solve_out o;
  // mask bit 0: level 2 is sFGMRES; bit 1: level 3 is sFGMRES
  if (mask == 1)
    o = refc::f3r_sdainv_sell_t<sFGMRES, FGMRES>(a, b, x, m2, m3, m4, c, restarts, tol, acc, sdainv_tol, hist,
                                                 hist_cap);
  else if (mask == 2)
    o = refc::f3r_sdainv_sell_t<FGMRES, sFGMRES>(a, b, x, m2, m3, m4, c, restarts, tol, acc, sdainv_tol, hist,
                                                 hist_cap);
  else if (mask == 3)
    o = refc::f3r_sdainv_sell_t<sFGMRES, sFGMRES>(a, b, x, m2, m3, m4, c, restarts, tol, acc, sdainv_tol, hist,
                                                  hist_cap);
  else
    o = refc::f3r_sdainv_sell_t<FGMRES, FGMRES>(a, b, x, m2, m3, m4, c, restarts, tol, acc, sdainv_tol, hist,
                                                hist_cap);
  out[0] = o.time_s;
  out[1] = o.iters;
  out[2] = o.impl_res;
  out[3] = o.expl_res;
  out[4] = o.solved;
  return o.n_hist;
}
