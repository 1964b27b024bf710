// trsv.cu -- Jacobi-iteration and BAJ triangular solves on SELL-32, and the
// f3r_trsv_* entry points of include/f3r_b200.h.
//
// Restates umineko-sparse/trsv/jacobi.hpp:290-505 (Jacobi<SELL<w, T, L>,
// form>) and trsv/baj.hpp:95-190 (BAJ<SELL<w, T, L>, form>) for fp16 vectors
// and fp16 factors.  Arithmetic (fp32, one rounding per stored fp16 value):
//   init    y0 = fp16(om * (in * dinv))          (dinv = 1 for FORM_LOWER)
//   Jacobi  acc = sum of N(i,j) y(j) (fma chain by increasing column, from 0)
//           y'(i) = fp16(fmaf(om, (in(i) - acc) * dinv(i), (1 - om) * y(i)))
//   BAJ     y(i) = fp16((in(i) - acc) * dinv(i)), in place, om = 1
// The reference accumulates in fp16 and forms the Jacobi update in double;
// the oracle's two arithmetic modes cover both.  Its SELL BAJ initialisation
// for d_upper pairs in(i) with the diagonal of row n-1-i (baj.hpp:161-170,
// unlike the CSR form, baj.hpp:74-77); here every form pairs in(i) with
// row i's own diagonal.
#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "trsv.hpp"

namespace f3r {

namespace {

__device__ __forceinline__ float jh2f(__half h) { return __half2float(h); }
__device__ __forceinline__ __half jf2h(float f) { return __float2half_rn(f); }

// one synchronous Jacobi sweep, folded into the SELL product over N
struct EpiJacobi {
  using Red = float;
  struct Pre {
    __half in, yold, dinv;
  };
  static constexpr int NV = 0;
  const __half *in, *yold, *dinv;  // dinv nullable (unit diagonal)
  __half *ynew;
  float om, omc;
  const __half *ome;  // nullable: final scaling
  __device__ __forceinline__ Pre load(int64_t r) const {
    return {in[r], yold[r], dinv ? dinv[r] : __float2half_rn(1.0f)};
  }
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, Acc acc, const Pre &p, Red (&)[1]) const {
    const float res = jh2f(p.in) - (float)acc;
    const float q = dinv ? res * jh2f(p.dinv) : res;
    __half h = jf2h(__fmaf_rn(om, q, omc * jh2f(p.yold)));
    if (ome) h = jf2h(jh2f(h) * jh2f(*ome));
    ynew[r] = h;
  }
  template <int W> __device__ __forceinline__ void finish(Red (&)[1]) const {}
};

__global__ void k_jac_init(const __half *__restrict__ in, const __half *__restrict__ dinv, __half *__restrict__ y,
                           float om, const __half *__restrict__ ome, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float v = jh2f(in[i]);
    if (dinv) v = v * jh2f(dinv[i]);
    __half h = jf2h(om * v);
    if (ome) h = jf2h(jh2f(h) * jh2f(*ome));
    y[i] = h;
  }
}

// One in-place BAJ sweep: a warp per slice, a lane per row.  The vector is
// read through volatile loads so that rows rewritten earlier in this sweep by
// other warps can be seen (the reference's in-place update); slices are
// visited bottom-up for the upper factor.
constexpr int kBajWarps = 8;
__global__ void __launch_bounds__(kBajWarps * 32)
    k_baj_sweep(const __half *__restrict__ val, const int32_t *__restrict__ col, const int32_t *__restrict__ sptr,
                int32_t nslices, int64_t n, const __half *__restrict__ in, const __half *__restrict__ dinv, __half *y,
                const __half *__restrict__ ome, int reverse) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t q = (int64_t)blockIdx.x * kBajWarps + warp;
  if (q >= nslices) return;
  const int64_t s = reverse ? (int64_t)nslices - 1 - q : q;
  const int64_t r = s * 32 + lane;
  const int32_t s0 = sptr[s], w = sptr[s + 1] - s0;
  const volatile unsigned short *yv = reinterpret_cast<const volatile unsigned short *>(y);
  float acc = 0.0f;
  for (int32_t k = 0; k < w; k++) {
    const int64_t e = ((int64_t)s0 + k) * 32 + lane;
    acc = __fmaf_rn(jh2f(val[e]), jh2f(__ushort_as_half(yv[col[e]])), acc);
  }
  if (r < n) {
    const float res = jh2f(in[r]) - acc;
    __half h = jf2h(dinv ? res * jh2f(dinv[r]) : res);
    if (ome) h = jf2h(jh2f(h) * jh2f(*ome));
    y[r] = h;
  }
}

__global__ void k_f64_to_f16(const double *__restrict__ a, __half *__restrict__ b, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = __double2half(a[i]);
}

}  // namespace

Status jacobi_trsv_prepare(Context &c) { return sell_attr<__half, __half, EpiJacobi>(c); }

void JacobiTrsv::release() {
  off.release();
  cudaFree(dinv);
  cudaFree(tmp);
  dinv = nullptr;
  tmp = nullptr;
}

Status JacobiTrsv::build(Context &c, const HostCSR &M, int form_, int kind_, int32_t iters_, double omega_,
                         const std::vector<int32_t> *perm) {
  if (form_ < FORM_LOWER || form_ > FORM_D_UPPER) return fail(F3R_ERROR_INVALID_VALUE, "unknown triangular form");
  if (kind_ != TRSV_JACOBI && kind_ != TRSV_BAJ) return fail(F3R_ERROR_INVALID_VALUE, "unknown trsv kind");
  if (iters_ < (kind_ == TRSV_BAJ ? 1 : 0) || iters_ > 4096)
    return fail(F3R_ERROR_INVALID_VALUE, "trsv iterations: Jacobi 0..4096, BAJ 1..4096");
  if (!(omega_ > 0.0 && omega_ <= 2.0)) return fail(F3R_ERROR_INVALID_VALUE, "Jacobi omega in (0, 2]");
  if (M.n != M.m) return fail(F3R_ERROR_INVALID_VALUE, "triangular factor must be square");
  n = M.n;
  form = form_;
  kind = kind_;
  iters = iters_;
  omega = omega_;
  reverse = (form == FORM_D_UPPER);
  if (perm && (int32_t)perm->size() != n) return fail(F3R_ERROR_INVALID_VALUE, "permutation size");
  // the strictly triangular part N in the vector order; each row keeps its
  // original column order (the order of the reference's row sums)
  std::vector<int32_t> pos(n);
  for (int32_t i = 0; i < n; i++) pos[i] = i;
  if (perm)
    for (int32_t s = 0; s < n; s++) pos[(*perm)[s]] = s;
  HostCSR N(n, n, std::max<int64_t>(M.nnz() - n, 0));
  std::vector<double> dh(form == FORM_LOWER ? 0 : n);
  int64_t k = 0;
  for (int32_t s = 0; s < n; s++) {
    const int32_t o = perm ? (*perm)[s] : s;
    const int32_t b = M.rptr[o], e = M.rptr[o + 1];
    if (e <= b) return fail(F3R_ERROR_INVALID_VALUE, "row " + std::to_string(o) + " has no diagonal entry");
    const int32_t d = form == FORM_D_UPPER ? b : e - 1;
    if (M.idx[d] != o)
      return fail(F3R_ERROR_INVALID_VALUE, "row " + std::to_string(o) + ": the diagonal must be stored " +
                                               (form == FORM_D_UPPER ? "first" : "last"));
    if (form != FORM_LOWER) {
      if (M.val[d] == 0.0) return fail(F3R_ERROR_INVALID_VALUE, "zero diagonal in row " + std::to_string(o));
      dh[s] = 1.0 / M.val[d];
    }
    for (int32_t j = b; j < e; j++) {
      if (j == d) continue;
      const bool ok = form == FORM_D_UPPER ? M.idx[j] > o : M.idx[j] < o;
      if (!ok) return fail(F3R_ERROR_INVALID_VALUE, "row " + std::to_string(o) + " is not triangular");
      if (k >= (int64_t)N.idx.size()) return fail(F3R_ERROR_INVALID_VALUE, "duplicate diagonal entries");
      N.idx[k] = pos[M.idx[j]];
      N.val[k] = M.val[j];
      k++;
    }
    N.rptr[s + 1] = (int32_t)k;
  }
  N.idx.resize(k);
  N.val.resize(k);
  SellHost sh;
  const f3r_csr nv = N.view();
  F3R_TRY(build_sell(nv, 1, false, sh));
  F3R_TRY(upload_sell(c, sh, 1 << F3R_F16, false, off));
  const size_t nn = (size_t)std::max(n, 1);
  F3R_TRY(c.alloc((void **)&tmp, nn * sizeof(__half)));
  if (form != FORM_LOWER) {
    double *t64 = nullptr;
    F3R_TRY(c.alloc((void **)&t64, nn * sizeof(double)));
    F3R_TRY(c.alloc((void **)&dinv, nn * sizeof(__half)));
    CUDA_TRY(cudaMemcpy(t64, dh.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    launch_k(c, k_f64_to_f16, c.ew_grid(n), kEwThreads, 0, c.stream, (const double *)t64, dinv, (int64_t)n);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(c.stream));
    cudaFree(t64);
  }
  return F3R_SUCCESS;
}

Status JacobiTrsv::apply(Context &c, const __half *in, __half *out, const __half *ome) {
  if (n == 0) return F3R_SUCCESS;
  if (in == out || in == tmp) return fail(F3R_ERROR_INVALID_VALUE, "trsv input must not alias its output");
  const int g = c.ew_grid(n);
  if (kind == TRSV_BAJ) {
    launch_k(c, k_jac_init, g, kEwThreads, 0, c.stream, in, (const __half *)dinv, out, 1.0f,
             iters == 1 ? ome : nullptr, (int64_t)n);
    const int gb = (int)cdiv(off.nslices, kBajWarps);
    for (int k = 1; k < iters; k++)
      launch_k(c, k_baj_sweep, gb, kBajWarps * 32, 0, c.stream, (const __half *)off.v16, (const int32_t *)off.col,
               (const int32_t *)off.sptr, off.nslices, (int64_t)n, in, (const __half *)dinv, out,
               (const __half *)nullptr, reverse ? 1 : 0);
    // the in-place sweeps read rows that other warps rewrite, so the scaling
    // follows the solve, as in the reference (hout *= ome[0], f3r.cpp:216, 229)
    if (ome && iters > 1) launch_k(c, k_half_scale, g, kEwThreads, 0, c.stream, out, ome, (int64_t)n);
  } else {
    const float om = (float)omega, omc = 1.0f - om;
    __half *a = (iters % 2 == 0) ? out : tmp, *b = (iters % 2 == 0) ? tmp : out;
    launch_k(c, k_jac_init, g, kEwThreads, 0, c.stream, in, (const __half *)dinv, a, om, iters == 0 ? ome : nullptr,
             (int64_t)n);
    for (int k = 0; k < iters; k++) {
      F3R_TRY(launch_sell(c, off.v16, off.view(), (const __half *)a,
                          EpiJacobi{in, a, dinv, b, om, omc, k == iters - 1 ? ome : nullptr}));
      std::swap(a, b);
    }
  }
  CUDA_TRY(cudaGetLastError());
  return F3R_SUCCESS;
}

}  // namespace f3r

using namespace f3r;

extern "C" {

f3r_status f3r_trsv_create(f3r_context *ctx, const f3r_csr *m, int32_t form, int32_t kind, int32_t iters,
                           double omega, f3r_trsv **out) {
  clear_stale_error();
  if (!ctx || !out) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  F3R_TRY(check_csr(m));
  CUDA_TRY(cudaSetDevice(ctx->device));
  HostCSR M(m->nrows, m->ncols, m->nnz);
  std::memcpy(M.rptr.data(), m->rptr, sizeof(int32_t) * (m->nrows + 1));
  std::memcpy(M.idx.data(), m->idx, sizeof(int32_t) * m->nnz);
  std::memcpy(M.val.data(), m->val, sizeof(double) * m->nnz);
  auto t = std::make_unique<f3r_trsv>();
  t->ctx = ctx;
  F3R_TRY(jacobi_trsv_prepare(*ctx));
  Status s = t->t.build(*ctx, M, form, kind, iters, omega, nullptr);
  if (s != F3R_SUCCESS) {
    t->t.release();
    return s;
  }
  *out = t.release();
  return F3R_SUCCESS;
}

f3r_status f3r_trsv_solve(f3r_trsv *t, const void *in, void *out) {
  clear_stale_error();
  if (!t || !in || !out) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  CUDA_TRY(cudaSetDevice(t->ctx->device));
  return t->t.apply(*t->ctx, (const __half *)in, (__half *)out, nullptr);
}

void f3r_trsv_destroy(f3r_trsv *t) {
  if (!t) return;
  if (cudaSetDevice(t->ctx->device) != cudaSuccess) return;  // runtime shutting down: left to the exit
  t->t.release();
  delete t;
}

}  // extern "C"
