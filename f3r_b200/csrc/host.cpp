// host.cpp -- host-side set-up of the F3R solver: problem generators, the
// symmetric diagonal scaling, and the two preconditioner factorisations
// (SDAINV and block-Jacobi ILU(0)).  The reference does all of these on the
// host as well; the GPU only ever sees their results.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "internal.hpp"

namespace f3r {

HostCSR::HostCSR(int32_t n_, int32_t m_, int64_t nnz_) : n(n_), m(m_), rptr(n_ + 1, 0), idx(nnz_), val(nnz_) {}

f3r_csr HostCSR::view() const {
  f3r_csr v;
  v.nrows = n;
  v.ncols = m;
  v.nnz = (int32_t)idx.size();
  v.rptr = rptr.data();
  v.idx = idx.data();
  v.val = val.data();
  return v;
}

Status check_csr(const f3r_csr *a) {
  if (!a || !a->rptr || (a->nnz > 0 && (!a->idx || !a->val)))
    return fail(F3R_ERROR_INVALID_VALUE, "null CSR pointer");
  if (a->nrows < 0 || a->ncols < 0 || a->nnz < 0) return fail(F3R_ERROR_INVALID_VALUE, "negative CSR size");
  if (a->rptr[0] != 0 || a->rptr[a->nrows] != a->nnz)
    return fail(F3R_ERROR_INVALID_VALUE, "rptr[0] must be 0 and rptr[n] must equal nnz");
  for (int32_t i = 0; i < a->nrows; i++) {
    if (a->rptr[i + 1] < a->rptr[i]) return fail(F3R_ERROR_INVALID_VALUE, "rptr not monotone");
    for (int32_t j = a->rptr[i]; j < a->rptr[i + 1]; j++) {
      if (a->idx[j] < 0 || a->idx[j] >= a->ncols) return fail(F3R_ERROR_INVALID_VALUE, "column index out of range");
      if (j > a->rptr[i] && a->idx[j] <= a->idx[j - 1])
        return fail(F3R_ERROR_INVALID_VALUE, "columns must be strictly increasing in each row");
    }
  }
  return F3R_SUCCESS;
}

// ---------------------------------------------------------------------------
// 27-point stencils.  The neighbour loop order (dz, dy, dx from -1 to 1)
// yields columns in increasing order, the order the reference's CSR build
// produces after its per-row sort (matrix/io.hpp:59-61).  Values follow
// matrix/hpcg.cpp:42-45 and matrix/hpgmp.cpp:127-137.
// ---------------------------------------------------------------------------
HostCSR *stencil27(int32_t nx, int32_t ny, int32_t nz, int32_t variant, double beta) {
  const int64_t n = (int64_t)nx * ny * nz;
  // row lengths first, so rows can be filled in parallel
  auto *a = new HostCSR((int32_t)n, (int32_t)n, 0);
  auto cnt1 = [](int32_t i, int32_t nn) { return 1 + (i > 0) + (i < nn - 1); };
  a->rptr[0] = 0;
  for (int64_t r = 0; r < n; r++) {
    int32_t i = (int32_t)(r % nx), j = (int32_t)((r / nx) % ny), k = (int32_t)(r / ((int64_t)nx * ny));
    a->rptr[r + 1] = a->rptr[r] + cnt1(i, nx) * cnt1(j, ny) * cnt1(k, nz);
  }
  const int64_t nnz = a->rptr[n];
  a->idx.resize(nnz);
  a->val.resize(nnz);
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < n; r++) {
    int32_t i = (int32_t)(r % nx), j = (int32_t)((r / nx) % ny), k = (int32_t)(r / ((int64_t)nx * ny));
    int64_t p = a->rptr[r];
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          int kk = k + dz, jj = j + dy, ii = i + dx;
          if (kk < 0 || jj < 0 || ii < 0 || kk >= nz || jj >= ny || ii >= nx) continue;
          int64_t col = (int64_t)kk * ny * nx + (int64_t)jj * nx + ii;
          double v;
          if (col == r) v = 26.0;
          else if (variant == 1) v = (dx == 0 && dy == 0) ? (dz < 0 ? -1.0 - beta : -1.0 + beta) : -1.0;
          else if (variant == 2) v = (col > r) ? -1.0 + beta : -1.0 - beta;
          else v = -1.0;
          a->idx[p] = (int32_t)col;
          a->val[p] = v;
          p++;
        }
  }
  return a;
}

// ---------------------------------------------------------------------------
// 7-point variable-coefficient diffusion with log-normal coefficients.  The
// field g is white noise smoothed by a separable Gaussian of standard
// deviation corr_len cells, applied periodically (the circular convolution an
// FFT filter computes, so g is stationary: every cell has the same variance),
// normalised to zero mean and unit variance, times sigma; k = exp(g).  Face
// coefficients are the harmonic mean of the two cells; a boundary face uses
// the cell's own k.
// ---------------------------------------------------------------------------
HostCSR *diffusion7(int32_t nx, int32_t ny, int32_t nz, double sigma, double corr_len, uint64_t seed) {
  const int64_t n = (int64_t)nx * ny * nz;
  std::vector<double> g(n), t(n);
  {
    std::mt19937_64 eng(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    for (int64_t i = 0; i < n; i++) g[i] = nd(eng);
  }
  if (corr_len > 0) {
    const int R = std::max(1, (int)std::ceil(3.0 * corr_len));
    std::vector<double> w(2 * R + 1);
    double ws = 0;
    for (int q = -R; q <= R; q++) ws += (w[q + R] = std::exp(-0.5 * (q / corr_len) * (q / corr_len)));
    for (auto &v : w) v /= ws;
    const int64_t stride[3] = {1, nx, (int64_t)nx * ny};
    const int32_t ext[3] = {nx, ny, nz};
    for (int axis = 0; axis < 3; axis++) {
#pragma omp parallel for schedule(static)
      for (int64_t r = 0; r < n; r++) {
        int32_t c = (int32_t)((r / stride[axis]) % ext[axis]);
        double s = 0;
        for (int q = -R; q <= R; q++) {
          int32_t cc = (c + q) % ext[axis];
          if (cc < 0) cc += ext[axis];
          s += w[q + R] * g[r + (int64_t)(cc - c) * stride[axis]];
        }
        t[r] = s;
      }
      std::swap(g, t);
    }
  }
  double mean = 0, var = 0;
  for (int64_t i = 0; i < n; i++) mean += g[i];
  mean /= (double)n;
  for (int64_t i = 0; i < n; i++) var += (g[i] - mean) * (g[i] - mean);
  var /= (double)n;
  const double sc = var > 0 ? sigma / std::sqrt(var) : 0.0;
  std::vector<double> kc(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) kc[i] = std::exp((g[i] - mean) * sc);

  auto *a = new HostCSR((int32_t)n, (int32_t)n, 0);
  a->rptr[0] = 0;
  for (int64_t r = 0; r < n; r++) {
    int32_t i = (int32_t)(r % nx), j = (int32_t)((r / nx) % ny), k = (int32_t)(r / ((int64_t)nx * ny));
    a->rptr[r + 1] = a->rptr[r] + 1 + (i > 0) + (i < nx - 1) + (j > 0) + (j < ny - 1) + (k > 0) + (k < nz - 1);
  }
  a->idx.resize(a->rptr[n]);
  a->val.resize(a->rptr[n]);
  const int64_t sxy = (int64_t)nx * ny;
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < n; r++) {
    int32_t i = (int32_t)(r % nx), j = (int32_t)((r / nx) % ny), k = (int32_t)(r / sxy);
    const int64_t nb[6] = {k > 0 ? r - sxy : -1, j > 0 ? r - nx : -1, i > 0 ? r - 1 : -1,
                           i < nx - 1 ? r + 1 : -1, j < ny - 1 ? r + nx : -1, k < nz - 1 ? r + sxy : -1};
    double off[6], diag = 0;
    for (int q = 0; q < 6; q++) {
      double f = nb[q] >= 0 ? 2.0 * kc[r] * kc[nb[q]] / (kc[r] + kc[nb[q]]) : kc[r];
      off[q] = f;
      diag += f;
    }
    int64_t p = a->rptr[r];
    for (int q = 0; q < 3; q++)
      if (nb[q] >= 0) { a->idx[p] = (int32_t)nb[q]; a->val[p++] = -off[q]; }
    a->idx[p] = (int32_t)r;
    a->val[p++] = diag;
    for (int q = 3; q < 6; q++)
      if (nb[q] >= 0) { a->idx[p] = (int32_t)nb[q]; a->val[p++] = -off[q]; }
  }
  return a;
}

// D^{-1/2} A D^{-1/2}, D = |diag|; a row without a diagonal keeps scale 1.
// Same operation order as matrix/algorithm.hpp:45-59: the divisor is the
// product of the two square roots.
void scaling(HostCSR &a) {
  std::vector<double> d(a.n, 1.0);
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < a.n; i++)
    for (int32_t j = a.rptr[i]; j < a.rptr[i + 1]; j++)
      if (a.idx[j] == i) d[i] = std::sqrt(std::fabs(a.val[j]));
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < a.n; i++)
    for (int32_t j = a.rptr[i]; j < a.rptr[i + 1]; j++) a.val[j] /= d[i] * d[a.idx[j]];
}

void host_spmv(const f3r_csr &a, const double *x, double *y) {
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < a.nrows; i++) {
    double t = 0;
    for (int32_t j = a.rptr[i]; j < a.rptr[i + 1]; j++) t = std::fma(a.val[j], x[a.idx[j]], t);
    y[i] = t;
  }
}

// ---------------------------------------------------------------------------
// SDAINV (stabilised, left-looking, dropped factored approximate inverse).
// Same steps as impl::left_sdainv (preconditioner/ainv.hpp:268-329) with the
// sparse accumulator of spvec.hpp:40-92, then the 1/d scaling of Z^T rows and
// the transpose (ainv.hpp:57-64).  Each sparse vector is a sorted list of
// (index, value) pairs; zero values are never stored.
// ---------------------------------------------------------------------------
namespace {
struct SpVec {
  std::vector<int32_t> i;
  std::vector<double> v;
  void push(int32_t id, double x) {
    if (x != 0) { i.push_back(id); v.push_back(x); }
  }
  double dot(const double *val, const int32_t *idx, int32_t len) const {
    double r = 0;
    size_t p = 0;
    int32_t q = 0;
    while (p < i.size() && q < len) {
      if (i[p] < idx[q]) p++;
      else if (i[p] == idx[q]) { r += v[p] * val[q]; p++; q++; }
      else q++;
    }
    return r;
  }
};
// out = alpha * x + y, entries with |.| < tol dropped
void axpy_drop(SpVec &out, double alpha, const SpVec &x, const SpVec &y, double tol) {
  out.i.clear();
  out.v.clear();
  size_t p = 0, q = 0;
  while (p < x.i.size() || q < y.i.size()) {
    int64_t xi = p < x.i.size() ? x.i[p] : INT32_MAX;
    int64_t yi = q < y.i.size() ? y.i[q] : INT32_MAX;
    double v;
    int32_t id;
    if (xi < yi) { v = x.v[p] * alpha; id = x.i[p]; p++; }
    else if (xi == yi) { v = y.v[q] + alpha * x.v[p]; id = y.i[q]; p++; q++; }
    else { v = y.v[q]; id = y.i[q]; q++; }
    if (std::fabs(v) >= tol) out.push(id, v);
  }
}
HostCSR *transpose(const HostCSR &a) {
  auto *r = new HostCSR(a.m, a.n, (int64_t)a.idx.size());
  std::vector<int32_t> cnt(a.m + 1, 0);
  for (auto c : a.idx) cnt[c]++;
  for (int32_t c = 0; c < a.m; c++) r->rptr[c + 1] = r->rptr[c] + cnt[c];
  std::fill(cnt.begin(), cnt.end(), 0);
  for (int32_t i = 0; i < a.n; i++)
    for (int32_t j = a.rptr[i]; j < a.rptr[i + 1]; j++) {
      int32_t c = a.idx[j];
      int64_t o = r->rptr[c] + cnt[c]++;
      r->idx[o] = i;
      r->val[o] = a.val[j];
    }
  return r;
}
HostCSR *rows_to_csr(const std::vector<SpVec> &z, int32_t n) {
  auto *r = new HostCSR(n, n, 0);
  for (int32_t i = 0; i < n; i++) r->rptr[i + 1] = r->rptr[i] + (int32_t)z[i].i.size();
  r->idx.resize(r->rptr[n]);
  r->val.resize(r->rptr[n]);
  for (int32_t i = 0; i < n; i++) {
    std::copy(z[i].i.begin(), z[i].i.end(), r->idx.begin() + r->rptr[i]);
    std::copy(z[i].v.begin(), z[i].v.end(), r->val.begin() + r->rptr[i]);
  }
  return r;
}
}  // namespace

Status sdainv(const HostCSR &A, double tol, double acc, HostCSR **Zout, HostCSR **Wout) {
  const int32_t n = A.n;
  if (A.m != n) return fail(F3R_ERROR_INVALID_VALUE, "SDAINV needs a square matrix");
  for (int32_t i = 0; i < n; i++) {
    bool diag = false;
    for (int32_t j = A.rptr[i]; j < A.rptr[i + 1]; j++) diag |= (A.idx[j] == i);
    if (!diag) return fail(F3R_ERROR_INVALID_VALUE, "SDAINV needs every diagonal entry stored");
  }
  std::unique_ptr<HostCSR> At(transpose(A));
  std::vector<double> d(n, 0.0);
  std::vector<SpVec> z(n), w(n);
  for (int32_t i = 0; i < n; i++) { z[i].push(i, 1.0); w[i].push(i, 1.0); }
  SpVec tmp;
  for (int32_t i = 0; i < n; i++) {
    const int32_t a_len = A.rptr[i + 1] - A.rptr[i], off = A.rptr[i];
    const int32_t at_len = At->rptr[i + 1] - At->rptr[i], coff = At->rptr[i];
    int32_t w_len = 0, z_len = 0;
    while (A.idx[off + w_len] < i) w_len++;
    while (At->idx[coff + z_len] < i) z_len++;
    for (int32_t j = 0; j < w_len; j++) {
      const int32_t col = A.idx[off + j];
      const double alpha = -z[col].dot(&A.val[off], &A.idx[off], a_len) / d[col];
      axpy_drop(tmp, alpha, w[col], w[i], tol);
      w[i] = tmp;
    }
    for (int32_t j = 0; j < z_len; j++) {
      const int32_t col = At->idx[coff + j];
      const double alpha = -w[col].dot(&At->val[coff], &At->idx[coff], at_len) / d[col];
      axpy_drop(tmp, alpha, z[col], z[i], tol);
      z[i] = tmp;
    }
    double &last = w[i].v.back();
    last *= acc;
    d[i] = w[i].dot(&At->val[coff], &At->idx[coff], at_len);
    last /= acc;
    if (d[i] == 0) d[i] = 1;
  }
  std::unique_ptr<HostCSR> Zt(rows_to_csr(z, n));
  HostCSR *Wt = rows_to_csr(w, n);
  for (int32_t i = 0; i < n; i++)
    for (int32_t j = Zt->rptr[i]; j < Zt->rptr[i + 1]; j++) Zt->val[j] /= d[i];
  *Zout = transpose(*Zt);
  *Wout = Wt;
  return F3R_SUCCESS;
}

// ---------------------------------------------------------------------------
// Block-Jacobi ILU(0): keep only entries inside the diagonal blocks
// (csr.hpp:109-155), factor each block in IKJ order with the acc diagonal
// shift (ilu.hpp:128-164), split into unit-lower L and upper U
// (algorithm.hpp:9-43).
// ---------------------------------------------------------------------------
Status ilu0_bj(const HostCSR &A, int32_t nb, double acc, HostCSR **Lout, HostCSR **Uout,
               std::vector<int32_t> *bptr_out) {
  const int32_t n = A.n;
  if (nb < 1 || nb > n) return fail(F3R_ERROR_INVALID_VALUE, "ilu_blocks must be in [1, n]");
  const int32_t bs = (n + nb - 1) / nb;
  std::vector<int32_t> bp(nb + 1);
  bp[0] = 0;
  for (int32_t b = 0; b < nb; b++) bp[b + 1] = (b != nb - 1) ? bp[b] + bs : n;
  if (bp[nb - 1] > n)
    return fail(F3R_ERROR_INVALID_VALUE,
                "ilu_blocks overruns the matrix: (blocks-1)*ceil(n/blocks) > n (the reference "
                "would read out of bounds)");
  for (int32_t i = 0; i < n; i++) {
    bool diag = false;
    for (int32_t j = A.rptr[i]; j < A.rptr[i + 1]; j++) diag |= (A.idx[j] == i);
    if (!diag) return fail(F3R_ERROR_INVALID_VALUE, "ILU(0) needs every diagonal entry stored");
  }
  HostCSR r(n, n, 0);
  for (int32_t b = 0; b < nb; b++)
    for (int32_t i = bp[b]; i < bp[b + 1]; i++) {
      for (int32_t j = A.rptr[i]; j < A.rptr[i + 1]; j++)
        if (bp[b] <= A.idx[j] && A.idx[j] < bp[b + 1]) {
          r.idx.push_back(A.idx[j]);
          r.val.push_back(A.val[j]);
        }
      r.rptr[i + 1] = (int32_t)r.idx.size();
    }
  double *val = r.val.data();
  const int32_t *c = r.idx.data(), *rp = r.rptr.data();
  val[0] *= acc;
#pragma omp parallel for schedule(dynamic, 1)
  for (int32_t b = 0; b < nb; b++) {
    const int32_t s = (b == 0) ? 1 : bp[b], e = bp[b + 1];
    for (int32_t i = s; i < e; i++) {
      int32_t d = rp[i];
      while (c[d] != i) d++;
      val[d] *= acc;
      for (int32_t pvt = rp[i]; pvt < rp[i + 1] && c[pvt] < i; pvt++) {
        const int32_t k = c[pvt];
        int32_t ref = rp[k];
        while (c[ref] != c[pvt]) ref++;
        val[pvt] = val[pvt] / val[ref];
        int32_t base = pvt + 1;
        while (base < rp[i + 1] && ref < rp[k + 1]) {
          if (c[ref] < c[base]) ref++;
          else if (c[ref] > c[base]) base++;
          else { val[base] -= val[pvt] * val[ref]; base++; ref++; }
        }
      }
    }
  }
  auto *L = new HostCSR(n, n, 0), *U = new HostCSR(n, n, 0);
  for (int32_t i = 0; i < n; i++) {
    for (int32_t j = rp[i]; j < rp[i + 1]; j++) {
      if (c[j] <= i) { L->idx.push_back(c[j]); L->val.push_back(c[j] < i ? val[j] : 1.0); }
      if (c[j] >= i) { U->idx.push_back(c[j]); U->val.push_back(val[j]); }
    }
    L->rptr[i + 1] = (int32_t)L->idx.size();
    U->rptr[i + 1] = (int32_t)U->idx.size();
  }
  *Lout = L;
  *Uout = U;
  if (bptr_out) *bptr_out = bp;
  return F3R_SUCCESS;
}

}  // namespace f3r
