/*
 * f3r_oracle.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * A plain-C, single-threaded CPU restatement of the reference F3R algorithm
 * (suzuki-hpc/F3R, header-only C++ library "umineko").  It exists only as the
 * checker for the CUDA path: tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may load it; the product library (f3r_b200/) never does.
 *
 * Every function names the reference file:line it restates.  The oracle is
 * pinned against the reference itself: oracle/ref_lib.cpp and ref_gen.cpp
 * compile the reference headers into oracle/_ref/ (oracle/Makefile),
 * tests/golden/gen_golden.py runs them and
 * commits golden vectors, and tests/test_oracle_pins.py checks this file
 * against them.
 *
 * Arithmetic modes.  ARITH_PRODUCT is the semantics of the CUDA path: fp16
 * storage, fp32 fused-multiply-add accumulation, one rounding per store.
 * ARITH_REF follows the reference expressions literally (separate multiply and
 * add, fp16 accumulation for fp16 x fp16 products as in
 * `decltype(__half * __half)` at library/umineko-sparse/matrix/sell.hpp:63).
 * Build with -ffp-contract=off so only explicit fma() calls fuse.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef _Float16 f16;

enum { DT_F64 = 0, DT_F32 = 1, DT_F16 = 2 };
enum { ARITH_PRODUCT = 0, ARITH_REF = 1 };
enum { PRECOND_SDAINV = 0, PRECOND_ILU0_BJ = 1, PRECOND_ILU0_JACOBI = 2, PRECOND_ILU0_BAJ = 3 };
enum { FORM_LOWER = 0, FORM_LOWER_D = 1, FORM_D_UPPER = 2 };

/* ------------------------------------------------------------------------ */
/* owned CSR matrix (values in fp64)                                        */
/* ------------------------------------------------------------------------ */
typedef struct {
  int32_t n, m, nnz;
  int32_t *rptr, *idx;
  double *val;
  /* block-diagonal pattern (library/umineko-sparse/matrix/base.hpp:15-43) */
  int32_t nblocks;
  int32_t *bptr;
} or_mat;

static or_mat *mat_new(int32_t n, int32_t m, int32_t nnz) {
  or_mat *a = (or_mat *)calloc(1, sizeof(or_mat));
  a->n = n; a->m = m; a->nnz = nnz;
  a->rptr = (int32_t *)calloc((size_t)n + 1, sizeof(int32_t));
  a->idx = (int32_t *)calloc(nnz > 0 ? (size_t)nnz : 1, sizeof(int32_t));
  a->val = (double *)calloc(nnz > 0 ? (size_t)nnz : 1, sizeof(double));
  return a;
}

void or_mat_free(or_mat *a) {
  if (!a) return;
  free(a->rptr); free(a->idx); free(a->val); free(a->bptr); free(a);
}
int32_t or_mat_n(const or_mat *a) { return a->n; }
int32_t or_mat_nnz(const or_mat *a) { return a->nnz; }
void or_mat_copy_out(const or_mat *a, int32_t *rptr, int32_t *idx, double *val) {
  memcpy(rptr, a->rptr, sizeof(int32_t) * ((size_t)a->n + 1));
  memcpy(idx, a->idx, sizeof(int32_t) * (size_t)a->nnz);
  memcpy(val, a->val, sizeof(double) * (size_t)a->nnz);
}
or_mat *or_mat_from(int32_t n, int32_t m, int32_t nnz, const int32_t *rptr,
                    const int32_t *idx, const double *val) {
  or_mat *a = mat_new(n, m, nnz);
  memcpy(a->rptr, rptr, sizeof(int32_t) * ((size_t)n + 1));
  memcpy(a->idx, idx, sizeof(int32_t) * (size_t)nnz);
  memcpy(a->val, val, sizeof(double) * (size_t)nnz);
  return a;
}

/* ------------------------------------------------------------------------ */
/* 27-point stencils: matrix/hpcg.cpp:13-57 and matrix/hpgmp.cpp:13-57.     */
/* variant 0: hpcg (off-diagonals -1); 1: hpgmp (only pure +-z neighbours   */
/* get -1-beta / -1+beta); 2: half-space (every neighbour whose linear      */
/* offset is positive gets -1+beta, negative gets -1-beta).  Rows sorted by */
/* column (the reference CSR build sorts, io.hpp:59-61).                    */
/* ------------------------------------------------------------------------ */
int64_t or_stencil27(int nx, int ny, int nz, int variant, double beta,
                     int32_t *rptr, int32_t *idx, double *val) {
  int64_t cnt = 0;
  int64_t n = (int64_t)nx * ny * nz;
  rptr[0] = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        int64_t row = (int64_t)k * ny * nx + (int64_t)j * nx + i;
        for (int zz = -1; zz <= 1; zz++)
          for (int yy = -1; yy <= 1; yy++)
            for (int xx = -1; xx <= 1; xx++) {
              if (k + zz < 0 || j + yy < 0 || i + xx < 0) continue;
              if (nz <= k + zz || ny <= j + yy || nx <= i + xx) continue;
              int64_t col = (int64_t)(k + zz) * ny * nx + (int64_t)(j + yy) * nx + i + xx;
              if (col < 0 || col >= n) continue;
              double v;
              if (row == col) v = 26.0;
              else if (variant == 1) {
                if (yy == 0 && xx == 0 && zz == -1) v = -1.0 - beta;
                else if (yy == 0 && xx == 0 && zz == 1) v = -1.0 + beta;
                else v = -1.0;
              } else if (variant == 2) {
                v = (col > row) ? -1.0 + beta : -1.0 - beta;
              } else v = -1.0;
              idx[cnt] = (int32_t)col;
              val[cnt] = v;
              cnt++;
            }
        rptr[row + 1] = (int32_t)cnt;
      }
  return cnt;
}

/* ------------------------------------------------------------------------ */
/* algorithm::scaling -- library/umineko-sparse/matrix/algorithm.hpp:45-59  */
/* ------------------------------------------------------------------------ */
void or_scaling(int32_t n, const int32_t *rptr, const int32_t *idx, double *val) {
  double *diag = (double *)malloc(sizeof(double) * (size_t)n);
  for (int32_t i = 0; i < n; i++) diag[i] = 1.0;
  for (int32_t i = 0; i < n; i++)
    for (int32_t j = rptr[i]; j < rptr[i + 1]; j++)
      if (idx[j] == i) diag[i] = sqrt(fabs(val[j]));
  for (int32_t i = 0; i < n; i++)
    for (int32_t j = rptr[i]; j < rptr[i + 1]; j++) val[j] /= diag[i] * diag[idx[j]];
  free(diag);
}

/* ------------------------------------------------------------------------ */
/* csr_to_sell<w, left> -- library/umineko-sparse/matrix/sell.hpp:249-307.  */
/* Reference layout: slice s starts at sptr[s]*w, column k of the slice at  */
/* +k*t_chunk, where t_chunk = w except n%w for a ragged last slice.        */
/* Padding: value 0, index = previous index in the row (0 for empty rows).  */
/* ------------------------------------------------------------------------ */
int64_t or_sell_nnz(int32_t n, const int32_t *rptr, int32_t w) {
  int64_t nnz = 0;
  int32_t nslice = (n + w - 1) / w;
  for (int32_t s = 0; s < nslice; s++) {
    int32_t i = s * w;
    int32_t tc = (n % w != 0 && s == nslice - 1) ? n % w : w;
    int32_t mx = 0;
    for (int32_t j = 0; j < tc; j++) {
      int32_t l = rptr[i + j + 1] - rptr[i + j];
      if (l > mx) mx = l;
    }
    nnz += (int64_t)mx * tc;
  }
  return nnz;
}

void or_csr_to_sell(int32_t n, const int32_t *rptr, const int32_t *idx, const double *val,
                    int32_t w, int32_t *sptr, int32_t *sidx, double *sval) {
  int32_t nslice = (n + w - 1) / w;
  sptr[0] = 0;
  for (int32_t s = 0; s < nslice; s++) {
    int32_t i = s * w;
    int32_t tc = (n % w != 0 && s == nslice - 1) ? n % w : w;
    int32_t mx = 0;
    for (int32_t j = 0; j < tc; j++) {
      int32_t l = rptr[i + j + 1] - rptr[i + j];
      if (l > mx) mx = l;
    }
    sptr[s + 1] = sptr[s] + mx;
  }
  for (int32_t s = 0; s < nslice; s++) {
    int32_t i = s * w;
    int32_t tc = (n % w != 0 && s == nslice - 1) ? n % w : w;
    int32_t mx = sptr[s + 1] - sptr[s];
    int64_t off = (int64_t)sptr[s] * w;
    for (int32_t j = 0; j < tc; j++) {
      int32_t c = 0;
      for (int32_t k = rptr[i + j]; k < rptr[i + j + 1]; k++, c++) {
        sval[off + (int64_t)c * tc + j] = val[k];
        sidx[off + (int64_t)c * tc + j] = idx[k];
      }
      for (; c < mx; c++) {
        sval[off + (int64_t)c * tc + j] = 0.0;
        sidx[off + (int64_t)c * tc + j] = (c == 0) ? 0 : sidx[off + (int64_t)(c - 1) * tc + j];
      }
    }
  }
}

/* SELL operate on the reference layout (sell.hpp:56-71), fp64 values and
 * vectors, separate multiply/add as written in the reference.             */
void or_sell_operate_f64(int32_t n, int32_t w, const int32_t *sptr, const int32_t *sidx,
                         const double *sval, const double *x, double *y) {
  for (int32_t i = 0; i < n; i++) {
    int32_t sid = i / w, my = i % w;
    int32_t s = sptr[sid], size = sptr[sid + 1] - s;
    int32_t tc = (sid != n / w) ? w : n % w;
    double t = 0.0;
    int64_t off = (int64_t)s * w + my;
    for (int32_t j = 0; j < size; j++) {
      t += sval[off] * x[sidx[off]];
      off += tc;
    }
    y[i] = t;
  }
}

/* SELL-C-sigma row order (sell.hpp:309-343): inside each window of sigma
 * rows, rows are ordered by descending length.  The reference sorts with an
 * unstable quicksort (core/sort.hpp:18-45); this restatement uses a stable
 * order, which changes only which slice a row lands in, never a row's
 * arithmetic.  perm[s] = original row stored at position s.              */
void or_sell_sigma_perm(int32_t n, const int32_t *rptr, int32_t sigma, int32_t *perm) {
  for (int32_t w0 = 0; w0 < n; w0 += sigma) {
    int32_t e = (w0 + sigma > n) ? n : w0 + sigma;
    for (int32_t i = w0; i < e; i++) perm[i] = i;
    /* insertion sort, stable, descending by length */
    for (int32_t i = w0 + 1; i < e; i++) {
      int32_t r = perm[i], lr = rptr[r + 1] - rptr[r];
      int32_t j = i - 1;
      while (j >= w0 && (rptr[perm[j] + 1] - rptr[perm[j]]) < lr) {
        perm[j + 1] = perm[j];
        j--;
      }
      perm[j + 1] = r;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Scalar type helpers                                                      */
/* ------------------------------------------------------------------------ */
static inline double ld(const void *p, int t, int64_t i) {
  switch (t) {
  case DT_F64: return ((const double *)p)[i];
  case DT_F32: return (double)((const float *)p)[i];
  default: return (double)((const f16 *)p)[i];
  }
}
static inline void st(void *p, int t, int64_t i, double v) {
  switch (t) {
  case DT_F64: ((double *)p)[i] = v; break;
  case DT_F32: ((float *)p)[i] = (float)v; break;
  default: ((f16 *)p)[i] = (f16)v; break;
  }
}
/* double -> value type, one rounding (the reference casts fp64 matrices
 * straight to the narrower type, sell.hpp:51-53 / tensor.hpp:272-277)      */
static inline double round_to(int t, double v) {
  switch (t) {
  case DT_F64: return v;
  case DT_F32: return (double)(float)v;
  default: return (double)(f16)v;
  }
}

/* ------------------------------------------------------------------------ */
/* CSR / SELL SpMV and residual -- csr.hpp:32-50 and sell.hpp:56-89.        */
/* The row sum runs over the row's stored entries in column order (SELL     */
/* keeps CSR order; padding contributes exact zeros).                       */
/*   acc: DT_F64 / DT_F32 -> fma chain in that type (CUDA path semantics);  */
/*        DT_F16 -> reference fp16 accumulation (round product, round sum). */
/*   ref_mul_add = 1: separate multiply and add (reference expression).     */
/* b == NULL: y = A x; else y = b - A x with the subtraction in the         */
/* accumulator type.                                                        */
/* ------------------------------------------------------------------------ */
void or_spmv(int32_t n, const int32_t *rptr, const int32_t *idx, const double *val, int val_t,
             const void *x, int x_t, void *y, int y_t, int acc_t, int ref_mul_add,
             const void *b, int b_t) {
  for (int32_t i = 0; i < n; i++) {
    if (acc_t == DT_F64) {
      double t = 0.0;
      for (int32_t j = rptr[i]; j < rptr[i + 1]; j++) {
        double v = round_to(val_t, val[j]);
        double xv = ld(x, x_t, idx[j]);
        t = ref_mul_add ? t + v * xv : fma(v, xv, t);
      }
      st(y, y_t, i, b ? ld(b, b_t, i) - t : t);
    } else if (acc_t == DT_F32) {
      float t = 0.0f;
      for (int32_t j = rptr[i]; j < rptr[i + 1]; j++) {
        float v = (float)round_to(val_t, val[j]);
        float xv = (float)ld(x, x_t, idx[j]);
        t = ref_mul_add ? t + v * xv : fmaf(v, xv, t);
      }
      st(y, y_t, i, b ? (double)((float)ld(b, b_t, i) - t) : (double)t);
    } else {
      f16 t = (f16)0.0f;
      for (int32_t j = rptr[i]; j < rptr[i + 1]; j++) {
        f16 v = (f16)val[j];
        f16 xv = (f16)ld(x, x_t, idx[j]);
        f16 p = (f16)((float)v * (float)xv);
        t = (f16)((float)t + (float)p);
      }
      st(y, y_t, i, b ? (double)(f16)((float)(f16)ld(b, b_t, i) - (float)t) : (double)t);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* SpVec -- library/umineko-sparse/spvec.hpp:12-92                          */
/* ------------------------------------------------------------------------ */
typedef struct { double *v; int32_t *i; int32_t size, cap; } spvec;

static void sv_init(spvec *s) { s->cap = 8; s->size = 0; s->v = malloc(8 * sizeof(double)); s->i = malloc(8 * sizeof(int32_t)); }
static void sv_free(spvec *s) { free(s->v); free(s->i); }
static void sv_push(spvec *s, double v, int32_t i) { /* spvec.hpp:16-19: zero values are not stored */
  if (v == 0) return;
  if (s->size == s->cap) { s->cap *= 2; s->v = realloc(s->v, s->cap * sizeof(double)); s->i = realloc(s->i, s->cap * sizeof(int32_t)); }
  s->v[s->size] = v; s->i[s->size] = i; s->size++;
}
/* sparse . (val, idx, len) merge -- spvec.hpp:41-58 */
static double sv_dot(const spvec *s, const double *val, const int32_t *idx, int32_t len) {
  double r = 0;
  int32_t p = 0, q = 0;
  while (p < s->size && q < len) {
    if (s->i[p] < idx[q]) p++;
    else if (s->i[p] == idx[q]) { r += s->v[p] * val[q]; p++; q++; }
    else q++;
  }
  return r;
}
/* out = alpha*x + y with drop |.| < tol -- spvec.hpp:66-92 */
static void sv_axpy(spvec *out, double alpha, const spvec *x, const spvec *y, double tol) {
  int32_t p = 0, q = 0;
  out->size = 0;
  while (p < x->size || q < y->size) {
    int64_t xi = (p < x->size) ? x->i[p] : INT32_MAX;
    int64_t yi = (q < y->size) ? y->i[q] : INT32_MAX;
    double v; int32_t id;
    if (xi < yi) { v = x->v[p] * alpha; id = x->i[p]; p++; }
    else if (xi == yi) { v = y->v[q] + alpha * x->v[p]; id = y->i[q]; p++; q++; }
    else { v = y->v[q]; id = y->i[q]; q++; }
    if (fabs(v) >= tol) sv_push(out, v, id);
  }
}
static void sv_copy(spvec *dst, const spvec *src) {
  dst->size = 0;
  for (int32_t k = 0; k < src->size; k++) sv_push(dst, src->v[k], src->i[k]);
}

/* csr_to_csc -- preconditioner/ainv.hpp:331-357 (transpose, rows kept in
 * increasing original-row order)                                           */
static or_mat *csr_to_csc(const or_mat *a) {
  or_mat *r = mat_new(a->m, a->n, a->nnz);
  int32_t *num = (int32_t *)calloc((size_t)a->m + 1, sizeof(int32_t));
  for (int32_t i = 0; i < a->n; i++)
    for (int32_t j = a->rptr[i]; j < a->rptr[i + 1]; j++) num[a->idx[j]]++;
  r->rptr[0] = 0;
  for (int32_t i = 0; i < a->m; i++) { r->rptr[i + 1] = r->rptr[i] + num[i]; num[i] = 0; }
  for (int32_t i = 0; i < a->n; i++)
    for (int32_t j = a->rptr[i]; j < a->rptr[i + 1]; j++) {
      int32_t c = a->idx[j];
      int32_t o = r->rptr[c] + num[c]++;
      r->idx[o] = i;
      r->val[o] = a->val[j];
    }
  free(num);
  return r;
}

/* convert_to_csc -- ainv.hpp:359-375: row i of the result is z[i]          */
static or_mat *spvecs_to_csr(spvec *z, int32_t n) {
  int64_t tot = 0;
  for (int32_t i = 0; i < n; i++) tot += z[i].size;
  or_mat *r = mat_new(n, n, (int32_t)tot);
  r->rptr[0] = 0;
  for (int32_t i = 0; i < n; i++) r->rptr[i + 1] = r->rptr[i] + z[i].size;
  for (int32_t i = 0; i < n; i++)
    for (int32_t k = 0; k < z[i].size; k++) {
      r->val[r->rptr[i] + k] = z[i].v[k];
      r->idx[r->rptr[i] + k] = z[i].i[k];
    }
  return r;
}

/* ------------------------------------------------------------------------ */
/* algorithm::sdainv -- ainv.hpp:27-65 with impl::left_sdainv :268-329.     */
/* Returns Z (rows of Z) and Wt (row i = w_i), so that the preconditioner   */
/* is M r = Z (Wt r) (IZW::operate, ainv.hpp:110-114).                      */
/* ------------------------------------------------------------------------ */
void or_sdainv(const or_mat *A, double tol, double acc, or_mat **Zout, or_mat **Wout) {
  int32_t n = A->n;
  or_mat *At = csr_to_csc(A);
  double *d = (double *)calloc((size_t)n, sizeof(double));
  spvec *z = (spvec *)malloc(sizeof(spvec) * (size_t)n);
  spvec *w = (spvec *)malloc(sizeof(spvec) * (size_t)n);
  for (int32_t i = 0; i < n; i++) { sv_init(&z[i]); sv_push(&z[i], 1.0, i); sv_init(&w[i]); sv_push(&w[i], 1.0, i); }
  spvec tmp; sv_init(&tmp);
  for (int32_t i = 0; i < n; i++) {
    int32_t a_len = A->rptr[i + 1] - A->rptr[i], off = A->rptr[i];
    int32_t at_len = At->rptr[i + 1] - At->rptr[i], coff = At->rptr[i];
    int32_t w_len = 0, z_len = 0;
    while (A->idx[off + w_len] < i) w_len++;
    while (At->idx[coff + z_len] < i) z_len++;
    for (int32_t j = 0; j < w_len; j++) {
      int32_t col = A->idx[off + j];
      double valu = sv_dot(&z[col], &A->val[off], &A->idx[off], a_len);
      double alpha = -valu / d[col];
      sv_axpy(&tmp, alpha, &w[col], &w[i], tol);
      sv_copy(&w[i], &tmp);
    }
    for (int32_t j = 0; j < z_len; j++) {
      int32_t col = At->idx[coff + j];
      double valu = sv_dot(&w[col], &At->val[coff], &At->idx[coff], at_len);
      double alpha = -valu / d[col];
      sv_axpy(&tmp, alpha, &z[col], &z[i], tol);
      sv_copy(&z[i], &tmp);
    }
    int32_t end = w[i].size - 1;
    w[i].v[end] *= acc;
    d[i] = sv_dot(&w[i], &At->val[coff], &At->idx[coff], at_len);
    w[i].v[end] /= acc;
    if (d[i] == 0) d[i] = 1;
  }
  or_mat *Zt = spvecs_to_csr(z, n);
  or_mat *Wt = spvecs_to_csr(w, n);
  for (int32_t i = 0; i < n; i++) { sv_free(&z[i]); sv_free(&w[i]); }
  free(z); free(w); sv_free(&tmp);
  for (int32_t i = 0; i < n; i++)
    for (int32_t j = Zt->rptr[i]; j < Zt->rptr[i + 1]; j++) Zt->val[j] /= d[i];
  *Zout = csr_to_csc(Zt);
  *Wout = Wt;
  or_mat_free(Zt);
  or_mat_free(At);
  free(d);
}

/* ------------------------------------------------------------------------ */
/* Block-Jacobi ILU(0): CSR::duplicate_block_diagonal (csr.hpp:109-155),    */
/* impl::_ilu0 (ilu.hpp:128-164), algorithm::split (algorithm.hpp:9-43).    */
/* ------------------------------------------------------------------------ */
static or_mat *block_diagonal(const or_mat *a, int32_t nb) {
  int32_t n = a->n;
  int32_t bs = (n + nb - 1) / nb;
  int32_t *bp = (int32_t *)malloc(sizeof(int32_t) * ((size_t)nb + 1));
  bp[0] = 0;
  for (int32_t b = 0; b < nb; b++) bp[b + 1] = (b != nb - 1) ? bp[b] + bs : n;
  /* The reference overruns its arrays when (nb-1)*ceil(n/nb) > n (the last
   * block pointer then falls below the previous one); reject that case.   */
  if (bp[nb - 1] > n) { free(bp); return NULL; }
  int64_t cnt = 0;
  for (int32_t b = 0; b < nb; b++)
    for (int32_t i = bp[b]; i < bp[b + 1]; i++)
      for (int32_t j = a->rptr[i]; j < a->rptr[i + 1]; j++)
        if (bp[b] <= a->idx[j] && a->idx[j] < bp[b + 1]) cnt++;
  or_mat *r = mat_new(n, a->m, (int32_t)cnt);
  r->nblocks = nb; r->bptr = bp;
  cnt = 0;
  r->rptr[0] = 0;
  for (int32_t b = 0; b < nb; b++)
    for (int32_t i = bp[b]; i < bp[b + 1]; i++) {
      for (int32_t j = a->rptr[i]; j < a->rptr[i + 1]; j++)
        if (bp[b] <= a->idx[j] && a->idx[j] < bp[b + 1]) {
          r->val[cnt] = a->val[j];
          r->idx[cnt++] = a->idx[j];
        }
      r->rptr[i + 1] = (int32_t)cnt;
    }
  return r;
}

/* Returns L (unit lower, diagonal stored as 1.0 last in each row) and U
 * (diagonal first in each row), both block-diagonal with nblocks blocks.    */
int or_ilu0_bj(const or_mat *A, int32_t nblocks, double acc, or_mat **Lout, or_mat **Uout) {
  if (nblocks < 1 || nblocks > A->n) return -1;
  or_mat *r = block_diagonal(A, nblocks);
  if (!r) return -1;
  double *val = r->val;
  int32_t *c = r->idx, *rp = r->rptr;
  val[0] *= acc;
  for (int32_t b = 0; b < r->nblocks; b++) {
    int32_t s = (b == 0) ? 1 : r->bptr[b];
    int32_t e = r->bptr[b + 1];
    for (int32_t i = s; i < e; i++) {
      int32_t d = rp[i];
      while (c[d] != i) d++;
      val[d] *= acc;
      for (int32_t pvt = rp[i]; pvt < rp[i + 1] && c[pvt] < i; pvt++) {
        int32_t k = c[pvt];
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
  /* split */
  int32_t n = r->n;
  int64_t ln = 0, un = 0;
  for (int32_t i = 0; i < n; i++)
    for (int32_t j = rp[i]; j < rp[i + 1]; j++) { if (c[j] <= i) ln++; if (c[j] >= i) un++; }
  or_mat *L = mat_new(n, n, (int32_t)ln), *U = mat_new(n, n, (int32_t)un);
  ln = un = 0;
  for (int32_t i = 0; i < n; i++) {
    for (int32_t j = rp[i]; j < rp[i + 1]; j++) {
      if (c[j] <= i) { L->val[ln] = (c[j] < i) ? val[j] : 1.0; L->idx[ln++] = c[j]; }
      if (c[j] >= i) { U->val[un] = val[j]; U->idx[un++] = c[j]; }
    }
    L->rptr[i + 1] = (int32_t)ln;
    U->rptr[i + 1] = (int32_t)un;
  }
  L->nblocks = U->nblocks = r->nblocks;
  L->bptr = (int32_t *)malloc(sizeof(int32_t) * ((size_t)r->nblocks + 1));
  U->bptr = (int32_t *)malloc(sizeof(int32_t) * ((size_t)r->nblocks + 1));
  memcpy(L->bptr, r->bptr, sizeof(int32_t) * ((size_t)r->nblocks + 1));
  memcpy(U->bptr, r->bptr, sizeof(int32_t) * ((size_t)r->nblocks + 1));
  or_mat_free(r);
  *Lout = L; *Uout = U;
  return 0;
}

/* Forward sweep with unit diagonal, trsv/bj.hpp:60-71: the last entry of
 * each row is the diagonal and is skipped.  Backward sweep, bj.hpp:84-96 on
 * the 180-degree rotated U (csr.hpp:60-86): the row's off-diagonals are
 * visited from the largest column down, then multiplied by the inverted
 * diagonal, which the reference forms in fp64 before the fp16 cast.
 * Values are used at type val_t; the working type is x_t (the vector type).
 * prod_fma = 1 uses the CUDA path's fp32 fma accumulation instead.          */
void or_trsv_lower(const or_mat *L, int val_t, const void *in, int x_t, void *out, int prod_fma) {
  for (int32_t i = 0; i < L->n; i++) {
    if (prod_fma) {
      float t = (float)ld(in, x_t, i);
      for (int32_t j = L->rptr[i]; j < L->rptr[i + 1] - 1; j++)
        t = fmaf(-(float)round_to(val_t, L->val[j]), (float)ld(out, x_t, L->idx[j]), t);
      st(out, x_t, i, t);
    } else {
      double t = ld(in, x_t, i);
      for (int32_t j = L->rptr[i]; j < L->rptr[i + 1] - 1; j++) {
        double p = round_to(x_t, round_to(val_t, L->val[j]) * ld(out, x_t, L->idx[j]));
        t = round_to(x_t, t - p);
      }
      st(out, x_t, i, t);
    }
  }
}
void or_trsv_upper(const or_mat *U, int val_t, const void *in, int x_t, void *out, int prod_fma) {
  for (int32_t i = U->n - 1; i >= 0; i--) {
    int32_t d = U->rptr[i];                 /* diagonal is first in the row */
    double dinv = round_to(val_t, 1.0 / U->val[d]);
    if (prod_fma) {
      float t = (float)ld(in, x_t, i);
      for (int32_t j = U->rptr[i + 1] - 1; j > d; j--)
        t = fmaf(-(float)round_to(val_t, U->val[j]), (float)ld(out, x_t, U->idx[j]), t);
      st(out, x_t, i, (double)(t * (float)dinv));
    } else {
      double t = ld(in, x_t, i);
      for (int32_t j = U->rptr[i + 1] - 1; j > d; j--) {
        double p = round_to(x_t, round_to(val_t, U->val[j]) * ld(out, x_t, U->idx[j]));
        t = round_to(x_t, t - p);
      }
      st(out, x_t, i, round_to(x_t, t * dinv));
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Jacobi-iteration triangular solves on fp16 vectors.                      */
/*                                                                          */
/* Jacobi (trsv/jacobi.hpp:290-505): y0 = om D^-1 in, then `iters` sweeps    */
/* y <- om D^-1 (in - N y) + (1 - om) y, N the strictly triangular part,    */
/* double-buffered.  BAJ (trsv/baj.hpp:95-190): y = D^-1 in, then iters-1   */
/* sweeps y <- D^-1 (in - N y) in place, rows in solve order (the reference */
/* on one thread; on more threads a row may see older values).  Forms       */
/* (matrix/base.hpp): LOWER unit diagonal stored last (not read), LOWER_D   */
/* diagonal stored last, D_UPPER diagonal stored first; D^-1 is the fp16    */
/* rounding of the fp64 reciprocal (CSR::inverse_last, csr.hpp:60-65).      */
/*                                                                          */
/* ARITH_PRODUCT (the CUDA path): acc = fp32 fma chain over N's entries by  */
/* increasing column from 0, r = in - acc, q = r * dinv (fp32),             */
/* y = fmaf(om, q, (1 - om) * y_old) with om = (float)omega; init           */
/* y0 = om * (in * dinv).  ARITH_REF (the reference's expressions): t = in, */
/* t -= v * x in fp16 (lower forms by increasing column, D_UPPER by         */
/* decreasing column: its 180-degree rotated copy), the update in double:   */
/* om * t * dinv + (1 - om) * y_old, one rounding to fp16.                  */
/* ------------------------------------------------------------------------ */
static void tri_parts(const or_mat *M, int form, int32_t i, int32_t *b, int32_t *e, int32_t *d) {
  if (form == FORM_D_UPPER) { *d = M->rptr[i]; *b = M->rptr[i] + 1; *e = M->rptr[i + 1]; }
  else { *d = M->rptr[i + 1] - 1; *b = M->rptr[i]; *e = M->rptr[i + 1] - 1; }
}

static double tri_sum_ref(const or_mat *M, int form, int32_t i, const f16 *in, const f16 *x) {
  int32_t b, e, d;
  tri_parts(M, form, i, &b, &e, &d);
  f16 t = in[i];
  if (form == FORM_D_UPPER) {
    for (int32_t j = e - 1; j >= b; j--) t = (f16)((float)t - (float)(f16)((float)(f16)M->val[j] * (float)x[M->idx[j]]));
  } else {
    for (int32_t j = b; j < e; j++) t = (f16)((float)t - (float)(f16)((float)(f16)M->val[j] * (float)x[M->idx[j]]));
  }
  return (double)t;
}

static float tri_sum_prod(const or_mat *M, int form, int32_t i, const f16 *in, const f16 *x) {
  int32_t b, e, d;
  tri_parts(M, form, i, &b, &e, &d);
  float acc = 0.0f;
  for (int32_t j = b; j < e; j++) acc = fmaf((float)(f16)M->val[j], (float)x[M->idx[j]], acc);
  return (float)in[i] - acc;
}

void or_jacobi_trsv(const or_mat *M, int form, int baj, int32_t iters, double omega, int arith, const f16 *in,
                    f16 *out) {
  int32_t n = M->n;
  f16 *dinv = (f16 *)malloc(sizeof(f16) * (n > 0 ? n : 1));
  for (int32_t i = 0; i < n; i++) {
    int32_t b, e, d;
    tri_parts(M, form, i, &b, &e, &d);
    dinv[i] = form == FORM_LOWER ? (f16)1.0f : (f16)(1.0 / M->val[d]);
  }
  const int has_d = form != FORM_LOWER;
  if (baj) {
    for (int32_t i = 0; i < n; i++) {
      if (arith == ARITH_REF) out[i] = has_d ? (f16)((float)in[i] * (float)dinv[i]) : in[i];
      else out[i] = has_d ? (f16)((float)in[i] * (float)dinv[i]) : in[i];
    }
    for (int32_t k = 1; k < iters; k++) {
      for (int32_t q = 0; q < n; q++) {
        int32_t i = form == FORM_D_UPPER ? n - 1 - q : q;
        if (arith == ARITH_REF) {
          f16 t = (f16)tri_sum_ref(M, form, i, in, out);
          out[i] = has_d ? (f16)((float)t * (float)dinv[i]) : t;
        } else {
          float r = tri_sum_prod(M, form, i, in, out);
          out[i] = (f16)(has_d ? r * (float)dinv[i] : r);
        }
      }
    }
    free(dinv);
    return;
  }
  f16 *y = (f16 *)malloc(sizeof(f16) * (n > 0 ? n : 1));
  f16 *z = (f16 *)malloc(sizeof(f16) * (n > 0 ? n : 1));
  const float om = (float)omega, omc = 1.0f - om;
  for (int32_t i = 0; i < n; i++) {
    if (arith == ARITH_REF)
      y[i] = (f16)(has_d ? omega * (double)in[i] * (double)dinv[i] : omega * (double)in[i]);
    else
      y[i] = (f16)(om * (has_d ? (float)in[i] * (float)dinv[i] : (float)in[i]));
  }
  for (int32_t k = 0; k < iters; k++) {
    for (int32_t i = 0; i < n; i++) {
      if (arith == ARITH_REF) {
        double t = tri_sum_ref(M, form, i, in, y);
        z[i] = (f16)(has_d ? omega * t * (double)dinv[i] + (1.0 - omega) * (double)y[i]
                           : omega * t + (1.0 - omega) * (double)y[i]);
      } else {
        float r = tri_sum_prod(M, form, i, in, y);
        float q = has_d ? r * (float)dinv[i] : r;
        z[i] = (f16)fmaf(om, q, omc * (float)y[i]);
      }
    }
    f16 *t = y; y = z; z = t;
  }
  memcpy(out, y, sizeof(f16) * n);
  free(y); free(z); free(dinv);
}

/* ------------------------------------------------------------------------ */
/* Reductions.  The reference reduces with OpenMP (host) or a three-stage   */
/* tree (device); neither order is reproducible, so the oracle sums in      */
/* blocks of 256 in the vector's arithmetic type.                           */
/* ------------------------------------------------------------------------ */
static float dotf(int32_t n, const float *a, const float *b) {
  float tot = 0.0f;
  for (int32_t s = 0; s < n; s += 256) {
    float p = 0.0f;
    int32_t e = (s + 256 < n) ? s + 256 : n;
    for (int32_t i = s; i < e; i++) p = fmaf(a[i], b[i], p);
    tot += p;
  }
  return tot;
}
static double dotd(int32_t n, const double *a, const double *b) {
  double tot = 0.0;
  for (int32_t s = 0; s < n; s += 256) {
    double p = 0.0;
    int32_t e = (s + 256 < n) ? s + 256 : n;
    for (int32_t i = s; i < e; i++) p = fma(a[i], b[i], p);
    tot += p;
  }
  return tot;
}
float or_dot_f32(int32_t n, const float *a, const float *b) { return dotf(n, a, b); }
double or_dot_f64(int32_t n, const double *a, const double *b) { return dotd(n, a, b); }

/* ------------------------------------------------------------------------ */
/* Nested F3R solve (work/src/f3r-gpu.cpp:210-265 for SDAINV + SELL,        */
/* work/src/f3r.cpp:195-248 for BJ-ILU(0) + CSR), built from FGMRES         */
/* (solver/gmres.hpp:56-135), Restarted (solver/restart.hpp:26-36) and the  */
/* adaptive-weight Richardson lambda R (f3r-gpu.cpp:229-260).               */
/* ------------------------------------------------------------------------ */
typedef struct {
  int32_t m1, restarts, m2, m3, m4, c;
  int32_t precond;     /* PRECOND_SDAINV or PRECOND_ILU0_BJ */
  int32_t arith;       /* ARITH_PRODUCT or ARITH_REF */
  int32_t half_scale_log2; /* 0: plain fp32->fp16 cast (reference); k: scale by 2^k */
  double tol;          /* stop when implicit residual / ||b|| < tol */
  double static_weight; /* > 0: F3R-Static, fixed weight (work/src/static.cpp:99-114) */
  int32_t trsv_iters;  /* PRECOND_ILU0_JACOBI / _BAJ: sweeps (max_ier / max_iter) */
  int32_t pad_;
  double trsv_omega;   /* PRECOND_ILU0_JACOBI: damping omega */
  int32_t sstep;       /* bit 0: level 2 is sFGMRES, bit 1: level 3 (solver/gmres2.hpp:137-221) */
  int32_t half_m;      /* > 0: an FGMRES level with fp16 vectors of half_m steps directly above R
                          (FGMRES<_Float16>, work/src/depth.cpp:122-167); m2 = 0: the outer level
                          calls it directly */
} or_f3r_params;

#define MAXM4 16
typedef struct {
  int32_t n;
  const or_mat *A;
  float *v32; /* A values rounded to fp32 */
  f16 *v16;   /* A values rounded to fp16 */
  const or_mat *P1, *P2; /* SDAINV: Wt, Z.  ILU: L, U */
  or_f3r_params p;
  /* Richardson state (f3r-gpu.cpp:106-107, 224-227, 277-281) */
  int64_t cnt;
  float sum[MAXM4];
  f16 ome[MAXM4];
  int32_t den;
  /* level-4 fp16 work vectors */
  f16 *hin, *hout, *tmp, *tmp2, *hr;
  int64_t r_calls;
} f3r_ctx;

static void spmv16(f3r_ctx *c, const f16 *x, f16 *y, const f16 *b) {
  /* fp16 matrix x fp16 vector.  ARITH_REF: fp16 accumulation (sell.hpp:63
   * decltype(__half*__half)); ARITH_PRODUCT: fp32 fma accumulation.       */
  const or_mat *A = c->A;
  for (int32_t i = 0; i < c->n; i++) {
    if (c->p.arith == ARITH_REF) {
      f16 t = (f16)0.0f;
      for (int32_t j = A->rptr[i]; j < A->rptr[i + 1]; j++)
        t = (f16)((float)t + (float)(f16)((float)c->v16[j] * (float)x[A->idx[j]]));
      y[i] = b ? (f16)((float)b[i] - (float)t) : t;
    } else {
      float t = 0.0f;
      for (int32_t j = A->rptr[i]; j < A->rptr[i + 1]; j++) t = fmaf((float)c->v16[j], (float)x[A->idx[j]], t);
      y[i] = b ? (f16)((float)b[i] - t) : (f16)t;
    }
  }
}

static void csr16_apply(f3r_ctx *c, const or_mat *M, const f16 *x, f16 *y) {
  for (int32_t i = 0; i < M->n; i++) {
    if (c->p.arith == ARITH_REF) {
      f16 t = (f16)0.0f;
      for (int32_t j = M->rptr[i]; j < M->rptr[i + 1]; j++)
        t = (f16)((float)t + (float)(f16)((float)(f16)M->val[j] * (float)x[M->idx[j]]));
      y[i] = t;
    } else {
      float t = 0.0f;
      for (int32_t j = M->rptr[i]; j < M->rptr[i + 1]; j++) t = fmaf((float)(f16)M->val[j], (float)x[M->idx[j]], t);
      y[i] = (f16)t;
    }
  }
}

/* preconditioner apply M: SDAINV Z(Wt x) (f3r-gpu.cpp:232-233) or
 * U^-1 L^-1 x (f3r.cpp:215-216)                                            */
static void prec_apply(f3r_ctx *c, const f16 *x, f16 *y, f16 *work) {
  if (c->p.precond == PRECOND_SDAINV) {
    csr16_apply(c, c->P1, x, work);
    csr16_apply(c, c->P2, work, y);
  } else if (c->p.precond == PRECOND_ILU0_BJ) {
    int pf = (c->p.arith == ARITH_PRODUCT);
    or_trsv_lower(c->P1, DT_F16, x, DT_F16, work, pf);
    or_trsv_upper(c->P2, DT_F16, work, DT_F16, y, pf);
  } else {
    int baj = c->p.precond == PRECOND_ILU0_BAJ;
    or_jacobi_trsv(c->P1, FORM_LOWER, baj, c->p.trsv_iters, c->p.trsv_omega, c->p.arith, x, work);
    or_jacobi_trsv(c->P2, FORM_D_UPPER, baj, c->p.trsv_iters, c->p.trsv_omega, c->p.arith, work, y);
  }
}

static float dot16(int32_t n, const f16 *a, const f16 *b) {
  /* dot(wildcard(a, tof32), wildcard(b, tof32)), f3r-gpu.cpp:236-237 */
  float tot = 0.0f;
  for (int32_t s = 0; s < n; s += 256) {
    float p = 0.0f;
    int32_t e = (s + 256 < n) ? s + 256 : n;
    for (int32_t i = s; i < e; i++) p = fmaf((float)a[i], (float)b[i], p);
    tot += p;
  }
  return tot;
}

/* Level 4: the adaptive-weight Richardson operator R (f3r-gpu.cpp:229-260),
 * on R's fp16 input c->hin; the result is left in c->hout.                 */
static void level4_core(f3r_ctx *c) {
  int32_t n = c->n;
  int ref = (c->p.arith == ARITH_REF);
  c->r_calls++;
  ++c->cnt;
  int upd = (c->p.static_weight <= 0) && (c->cnt % c->p.c == 0);
  prec_apply(c, c->hin, c->hout, c->tmp);
  if (upd) {
    spmv16(c, c->hout, c->tmp, NULL);
    float dar = dot16(n, c->tmp, c->tmp), dr = dot16(n, c->tmp, c->hin);
    float om = dr / dar;
    f16 omh = (f16)om;
    for (int32_t i = 0; i < n; i++) c->hout[i] = (f16)((float)c->hout[i] * (float)omh);
    c->sum[0] += om;
    c->den = (int32_t)(c->cnt / c->p.c);
    c->ome[0] = (f16)(c->sum[0] / (float)c->den);
  } else {
    for (int32_t i = 0; i < n; i++) c->hout[i] = (f16)((float)c->hout[i] * (float)c->ome[0]);
  }
  for (int k = 1; k < c->p.m4; k++) {
    spmv16(c, c->hout, c->hr, c->hin);
    prec_apply(c, c->hr, c->tmp2, c->tmp);
    if (upd) {
      spmv16(c, c->tmp2, c->tmp, NULL);
      float dar = dot16(n, c->tmp, c->tmp), dr = dot16(n, c->tmp, c->hr);
      float om = dr / dar;
      for (int32_t i = 0; i < n; i++) {
        if (ref) c->hout[i] = (f16)((float)c->hout[i] + (float)(f16)(om * (float)c->tmp2[i]));
        else c->hout[i] = (f16)fmaf(om, (float)c->tmp2[i], (float)c->hout[i]);
      }
      c->sum[k] += om;
      c->ome[k] = (f16)(c->sum[k] / (float)c->den);
    } else {
      for (int32_t i = 0; i < n; i++) {
        if (ref) c->hout[i] = (f16)((float)c->hout[i] + (float)(f16)((float)c->ome[k] * (float)c->tmp2[i]));
        else c->hout[i] = (f16)fmaf((float)c->ome[k], (float)c->tmp2[i], (float)c->hout[i]);
      }
    }
  }
}

static void givens_f(float *cs, float *sn, float *H, float *e, int j);
static void trsv_f(const float *U, const float *b, float *x, int h, int w);

/* R below an fp32 level: fp32 in, hin = fp16(in * sc) (f3r-gpu.cpp:231),
 * out = fp32(hout) / sc (f3r-gpu.cpp:259)                                  */
static void level4(f3r_ctx *c, const float *in, float *out) {
  float sc = ldexpf(1.0f, c->p.half_scale_log2), isc = ldexpf(1.0f, -c->p.half_scale_log2);
  for (int32_t i = 0; i < c->n; i++) c->hin[i] = (f16)(in[i] * sc);
  level4_core(c);
  for (int32_t i = 0; i < c->n; i++) out[i] = (float)c->hout[i] * isc;
}

/* R below the fp16-vector level: its fp16 vectors in and out directly      */
static void level4_h(f3r_ctx *c, const f16 *in, f16 *out) {
  memcpy(c->hin, in, sizeof(f16) * (size_t)c->n);
  level4_core(c);
  memcpy(out, c->hout, sizeof(f16) * (size_t)c->n);
}

/* fp16 arithmetic of the reference's FGMRES<_Float16> scalars and vectors,
 * one rounding per operation (ARITH_REF)                                   */
static inline f16 hmul(f16 a, f16 b) { return (f16)((float)a * (float)b); }
static inline f16 hadd(f16 a, f16 b) { return (f16)((float)a + (float)b); }
static inline f16 hsub(f16 a, f16 b) { return (f16)((float)a - (float)b); }
static inline f16 hdiv(f16 a, f16 b) { return (f16)((float)a / (float)b); }
/* dot(a, b) with an _Float16 partial sum, one thread (tensor.hpp:509-537,
 * loop.hpp exec<host>::para_reduce)                                        */
static f16 hdot(int32_t n, const f16 *a, const f16 *b) {
  f16 s = (f16)0.0f;
  for (int32_t i = 0; i < n; i++) s = hadd(s, hmul(a[i], b[i]));
  return s;
}

/* FGMRES<_Float16> in the reference's arithmetic: dots and norms summed in
 * fp16, V(j+1) -= V H(j) in fp16 (MULMV, tensor.hpp:605-623), H, Givens and
 * the back substitution in fp16 (gmres2.hpp:14-53, sqrt through float as the
 * depth driver defines it, depth.cpp:26-31), x = Z y in fp16.             */
static void level_half_ref(f3r_ctx *c, const float *in32, const double *in64, float *out32, double *out64) {
  int32_t n = c->n;
  int m = c->p.half_m;
  f16 *V = (f16 *)malloc(sizeof(f16) * (size_t)n * (m + 1));
  f16 *Z = (f16 *)malloc(sizeof(f16) * (size_t)n * m);
  f16 *H = (f16 *)calloc((size_t)(m + 1) * m, sizeof(f16));
  f16 cs[128], sn[128], e[129], y[128];
  for (int k = 0; k < 129; k++) e[k] = (f16)0.0f;
  e[0] = (f16)1.0f;
  for (int32_t i = 0; i < n; i++) V[i] = in32 ? (f16)in32[i] : (f16)in64[i];
  for (int j = 0; j < m; j++) {
    f16 *vj = V + (size_t)n * j, *zj = Z + (size_t)n * j, *w = V + (size_t)n * (j + 1);
    level4_h(c, vj, zj);
    spmv16(c, zj, w, NULL);
    f16 *Hj = H + (size_t)(m + 1) * j;
    for (int k = 0; k <= j; k++) Hj[k] = hdot(n, w, V + (size_t)n * k);
    for (int32_t i = 0; i < n; i++) {
      f16 r = hmul(V[i], Hj[0]);
      for (int k = 1; k <= j; k++) r = hadd(r, hmul(V[(size_t)n * k + i], Hj[k]));
      w[i] = hsub(w[i], r);
    }
    f16 nr = (f16)sqrtf((float)hdot(n, w, w));
    Hj[j + 1] = nr;
    f16 inv = (f16)(1.0 / (double)nr);
    for (int32_t i = 0; i < n; i++) w[i] = hmul(inv, w[i]);
    for (int i = 0; i < j; i++) {
      f16 t = Hj[i];
      Hj[i] = hadd(hmul(cs[i], t), hmul(sn[i], Hj[i + 1]));
      Hj[i + 1] = hadd(hmul((f16)(-(float)sn[i]), t), hmul(cs[i], Hj[i + 1]));
    }
    f16 t = (f16)sqrtf((float)hadd(hmul(Hj[j], Hj[j]), hmul(Hj[j + 1], Hj[j + 1])));
    cs[j] = hdiv(Hj[j], t);
    sn[j] = hdiv(Hj[j + 1], t);
    Hj[j] = t;
    Hj[j + 1] = (f16)0.0f;
    e[j + 1] = hmul((f16)(-(float)sn[j]), e[j]);
    e[j] = hmul(cs[j], e[j]);
  }
  for (int i = m - 1; i >= 0; i--) {
    f16 t = e[i];
    for (int q = m - 1; q > i; q--) t = hsub(t, hmul(H[(size_t)q * (m + 1) + i], y[q]));
    y[i] = hdiv(t, H[(size_t)i * (m + 1) + i]);
  }
  for (int32_t i = 0; i < n; i++) {
    f16 r = hmul(Z[i], y[0]);
    for (int k = 1; k < m; k++) r = hadd(r, hmul(Z[(size_t)n * k + i], y[k]));
    if (out32) out32[i] = (float)r;
    else out64[i] = (double)r;
  }
  free(V); free(Z); free(H);
}

/* The fp16-vector level FGMRES<_Float16>::kernel<true> (gmres.hpp:96-134
 * with normalize=false; instantiated at work/src/depth.cpp:122-167): V and
 * Z stored in fp16; the product's arithmetic computes w = A16 z with fp32
 * accumulation, every dot, norm and Gram-Schmidt update in fp32 (rounded
 * once when stored), H and the Givens rotations in fp32.  in32 / in64: the
 * calling level's vector (fp32 inner level, or the fp64 outer level when
 * m2 = 0); the result goes to out32 or out64.  ARITH_REF: level_half_ref.  */
static void level_half(f3r_ctx *c, const float *in32, const double *in64, float *out32, double *out64) {
  if (c->p.arith == ARITH_REF) {
    level_half_ref(c, in32, in64, out32, out64);
    return;
  }
  int32_t n = c->n;
  int m = c->p.half_m;
  f16 *V = (f16 *)malloc(sizeof(f16) * (size_t)n * (m + 1));
  f16 *Z = (f16 *)malloc(sizeof(f16) * (size_t)n * m);
  float *H = (float *)calloc((size_t)(m + 1) * m, sizeof(float));
  float *w32 = (float *)malloc(sizeof(float) * (size_t)n);
  float cs[128], sn[128], e[129], y[128];
  memset(e, 0, sizeof(e));
  e[0] = 1.0f;
  for (int32_t i = 0; i < n; i++) V[i] = in32 ? (f16)in32[i] : (f16)in64[i];
  const or_mat *A = c->A;
  for (int j = 0; j < m; j++) {
    f16 *vj = V + (size_t)n * j, *zj = Z + (size_t)n * j, *w = V + (size_t)n * (j + 1);
    level4_h(c, vj, zj);
    spmv16(c, zj, w, NULL);
    float *Hj = H + (size_t)(m + 1) * j;
    for (int k = 0; k <= j; k++) Hj[k] = dot16(n, w, V + (size_t)n * k);
    float nn = 0.0f;
    for (int32_t i = 0; i < n; i++) {
      float r = (float)V[i] * Hj[0];
      for (int k = 1; k <= j; k++) r = fmaf((float)V[(size_t)n * k + i], Hj[k], r);
      w[i] = (f16)((float)w[i] - r);
      w32[i] = (float)w[i];
    }
    nn = dotf(n, w32, w32);
    float nr = sqrtf(nn);
    Hj[j + 1] = nr;
    float inv = 1.0f / nr;
    for (int32_t i = 0; i < n; i++) w[i] = (f16)((float)w[i] * inv);
    givens_f(cs, sn, Hj, e, j);
  }
  trsv_f(H, e, y, m + 1, m);
  for (int32_t i = 0; i < n; i++) {
    float r = (float)Z[i] * y[0];
    for (int k = 1; k < m; k++) r = fmaf((float)Z[(size_t)n * k + i], y[k], r);
    if (out32) out32[i] = r;
    else out64[i] = (double)r;
  }
  free(V); free(Z); free(H); free(w32);
}

/* Givens update of Hessenberg column j (gmres.hpp:24-38) and residual
 * vector (gmres.hpp:14-21); generic over float/double by macro.            */
#define GIVENS_DEF(T, SQRT, NAME)                                              \
  static void NAME(T *cs, T *sn, T *H, T *e, int j) {                          \
    for (int i = 0; i < j; i++) {                                              \
      T t = H[i];                                                              \
      H[i] = cs[i] * t + sn[i] * H[i + 1];                                     \
      H[i + 1] = -sn[i] * t + cs[i] * H[i + 1];                                \
    }                                                                          \
    T t = SQRT(H[j] * H[j] + H[j + 1] * H[j + 1]);                             \
    cs[j] = H[j] / t;                                                          \
    sn[j] = H[j + 1] / t;                                                      \
    H[j] = t;                                                                  \
    H[j + 1] = 0;                                                              \
    e[j + 1] = -sn[j] * e[j];                                                  \
    e[j] = cs[j] * e[j];                                                       \
  }
GIVENS_DEF(float, sqrtf, givens_f)
GIVENS_DEF(double, sqrt, givens_d)

/* back substitution Blas1::trsv (gmres.hpp:41-53), H column-major ld=h   */
#define TRSV_DEF(T, NAME)                                                      \
  static void NAME(const T *U, const T *b, T *x, int h, int w) {               \
    for (int i = w - 1; i >= 0; i--) {                                         \
      T t = b[i];                                                              \
      for (int j = w - 1; j > i; j--) t -= U[j * h + i] * x[j];                \
      x[i] = t / U[i * h + i];                                                 \
    }                                                                          \
  }
TRSV_DEF(float, trsv_f)
TRSV_DEF(double, trsv_d)

/* Inner FGMRES<float>::kernel<true> with normalize=false and no cond
 * (gmres.hpp:96-134).  level 2 uses the fp32 matrix, level 3 the fp16
 * matrix with fp32 vectors (decltype(__half*float) = float).  The input is
 * given in fp32; the fp64->fp32 cast of level 2's input is done by the
 * caller (V(0).copy(rhs), gmres.hpp:102).  Output is the fp32 sum Z*y.     */
static void level_inner(f3r_ctx *c, int level, const float *in, float *out) {
  int32_t n = c->n;
  int m = (level == 2) ? c->p.m2 : c->p.m3;
  float *V = (float *)malloc(sizeof(float) * (size_t)n * (m + 1));
  float *Z = (float *)malloc(sizeof(float) * (size_t)n * m);
  float *H = (float *)calloc((size_t)(m + 1) * m, sizeof(float));
  float cs[128], sn[128], e[129], y[128];
  memset(e, 0, sizeof(e));
  e[0] = 1.0f;
  memcpy(V, in, sizeof(float) * (size_t)n);
  const or_mat *A = c->A;
  /* sFGMRES (gmres2.hpp:176-192): every M and A application first, on the
   * raw vectors W(j+1) = A M W(j); then the same classical Gram-Schmidt,
   * norms and Givens rotations over the stored W, step by step.           */
  const int sstep = (c->p.sstep >> (level - 2)) & 1;
  for (int pass = 0; pass < (sstep ? 2 : 1); pass++)
  for (int j = 0; j < m; j++) {
    float *vj = V + (size_t)n * j, *zj = Z + (size_t)n * j, *w = V + (size_t)n * (j + 1);
    if (!sstep || pass == 0) {
      if (level == 2 && c->p.m3 > 0) level_inner(c, 3, vj, zj);
      else if (c->p.half_m > 0) level_half(c, vj, NULL, zj, NULL);  /* the fp16-vector level (depth.cpp) */
      else level4(c, vj, zj);  /* level 3, or level 2 of the depth-2 form (work/src/depth.cpp:157-162) */
      for (int32_t i = 0; i < n; i++) {
        float t = 0.0f;
        if (level == 2)
          for (int32_t q = A->rptr[i]; q < A->rptr[i + 1]; q++) t = fmaf(c->v32[q], zj[A->idx[q]], t);
        else
          for (int32_t q = A->rptr[i]; q < A->rptr[i + 1]; q++) t = fmaf((float)c->v16[q], zj[A->idx[q]], t);
        w[i] = t;
      }
      if (sstep) continue;
    }
    float *Hj = H + (size_t)(m + 1) * j;
    for (int k = 0; k <= j; k++) Hj[k] = dotf(n, w, V + (size_t)n * k);
    for (int32_t i = 0; i < n; i++) {
      float r = V[i] * Hj[0];
      for (int k = 1; k <= j; k++) r = fmaf(V[(size_t)n * k + i], Hj[k], r);
      w[i] -= r;
    }
    float nr = sqrtf(dotf(n, w, w));
    Hj[j + 1] = nr;
    float inv = 1.0f / nr;
    for (int32_t i = 0; i < n; i++) w[i] *= inv;
    givens_f(cs, sn, Hj, e, j);
  }
  trsv_f(H, e, y, m + 1, m);
  for (int32_t i = 0; i < n; i++) {
    float r = Z[i] * y[0];
    for (int k = 1; k < m; k++) r = fmaf(Z[(size_t)n * k + i], y[k], r);
    out[i] = r;
  }
  free(V); free(Z); free(H);
}

/* Outer FGMRES<double> with normalize=true (gmres.hpp:85-134) inside
 * Restarted (restart.hpp:26-36).  cond(i, e) = e/||b|| < tol
 * (f3r-gpu.cpp:83-86).  hist receives e/||b|| after every outer step.     */
int or_f3r_solve(const or_mat *A, const or_mat *P1, const or_mat *P2, const double *b, double *x,
                 const or_f3r_params *p, double *hist, int32_t hist_cap, int32_t *n_hist,
                 int32_t *iters, double *impl_res, int64_t *r_calls) {
  f3r_ctx c;
  memset(&c, 0, sizeof(c));
  int32_t n = A->n;
  c.n = n; c.A = A; c.P1 = P1; c.P2 = P2; c.p = *p;
  if (p->m2 > 127 || p->m3 > 127 || p->m3 < 0 || p->m4 > MAXM4 || p->m1 > 4096 || p->half_m < 0 ||
      p->half_m > 127 || (p->m2 == 0 && p->half_m == 0))
    return -1;
  c.v32 = (float *)malloc(sizeof(float) * (size_t)A->nnz);
  c.v16 = (f16 *)malloc(sizeof(f16) * (size_t)A->nnz);
  for (int32_t q = 0; q < A->nnz; q++) { c.v32[q] = (float)A->val[q]; c.v16[q] = (f16)A->val[q]; }
  c.hin = malloc(sizeof(f16) * n); c.hout = malloc(sizeof(f16) * n); c.tmp = malloc(sizeof(f16) * n);
  c.tmp2 = malloc(sizeof(f16) * n); c.hr = malloc(sizeof(f16) * n);
  /* per-solve reset (f3r-gpu.cpp:277-281) */
  c.cnt = p->c;
  for (int k = 0; k < MAXM4; k++) {
    c.sum[k] = 1.0f;
    c.ome[k] = (f16)(p->static_weight > 0 ? (float)p->static_weight : 1.0f);
  }

  int m = p->m1;
  double *V = (double *)malloc(sizeof(double) * (size_t)n * (m + 1));
  double *Z = (double *)malloc(sizeof(double) * (size_t)n * m);
  double *H = (double *)malloc(sizeof(double) * (size_t)(m + 1) * m);
  double *cs = malloc(sizeof(double) * m), *sn = malloc(sizeof(double) * m);
  double *e = malloc(sizeof(double) * (m + 1)), *y = malloc(sizeof(double) * m);
  float *in32 = malloc(sizeof(float) * n), *out32 = malloc(sizeof(float) * n);
  double nb = sqrt(dotd(n, b, b));
  int32_t tot_iter = 0, nh = 0;
  int solved = 0;
  double last = 0;
  for (int rs = 0; rs < p->restarts && !solved; rs++) {
    memset(H, 0, sizeof(double) * (size_t)(m + 1) * m);
    memset(e, 0, sizeof(double) * (m + 1));
    /* r = b - A x (fp64, gmres.hpp:87) */
    double *r = V;
    or_spmv(n, A->rptr, A->idx, A->val, DT_F64, x, DT_F64, r, DT_F64, DT_F64, 0, b, DT_F64);
    double h = sqrt(dotd(n, r, r));
    e[0] = h;
    double inv = 1.0 / h;
    for (int32_t i = 0; i < n; i++) V[i] = inv * r[i];
    last = fabs(h);
    if (last / nb < p->tol) { solved = 1; break; }
    int j = 0;
    for (; j < m; j++) {
      double *vj = V + (size_t)n * j, *zj = Z + (size_t)n * j, *w = V + (size_t)n * (j + 1);
      if (p->m2 > 0) {
        for (int32_t i = 0; i < n; i++) in32[i] = (float)vj[i];
        level_inner(&c, 2, in32, out32);
        for (int32_t i = 0; i < n; i++) zj[i] = (double)out32[i];
      } else {
        level_half(&c, NULL, vj, NULL, zj);  /* F2H: the fp16-vector level under the outer level */
      }
      or_spmv(n, A->rptr, A->idx, A->val, DT_F64, zj, DT_F64, w, DT_F64, DT_F64, 0, NULL, DT_F64);
      double *Hj = H + (size_t)(m + 1) * j;
      for (int k = 0; k <= j; k++) Hj[k] = dotd(n, w, V + (size_t)n * k);
      for (int32_t i = 0; i < n; i++) {
        double rr = V[i] * Hj[0];
        for (int k = 1; k <= j; k++) rr = fma(V[(size_t)n * k + i], Hj[k], rr);
        w[i] -= rr;
      }
      double nr = sqrt(dotd(n, w, w));
      Hj[j + 1] = nr;
      double iv = 1.0 / nr;
      for (int32_t i = 0; i < n; i++) w[i] *= iv;
      givens_d(cs, sn, Hj, e, j);
      last = fabs(e[j + 1]);
      if (nh < hist_cap) hist[nh] = last / nb;
      nh++;
      if (last / nb < p->tol) { j++; solved = 1; break; }
    }
    trsv_d(H, e, y, m + 1, j);
    for (int32_t i = 0; i < n; i++) {
      double rr = Z[i] * y[0];
      for (int k = 1; k < j; k++) rr = fma(Z[(size_t)n * k + i], y[k], rr);
      x[i] += rr;
    }
    tot_iter += j;
  }
  *iters = tot_iter;
  *impl_res = last / nb;
  *n_hist = nh;
  if (r_calls) *r_calls = c.r_calls;
  free(V); free(Z); free(H); free(cs); free(sn); free(e); free(y); free(in32); free(out32);
  free(c.v32); free(c.v16); free(c.hin); free(c.hout); free(c.tmp); free(c.tmp2); free(c.hr);
  return solved;
}

/* Single application of level 4 with a fresh state, for kernel-level checks
 * of the Richardson operator (f3r-gpu.cpp:229-260).  cnt0 is the counter
 * value before the call; sum/ome are the running weights (in/out).         */
void or_richardson_apply(const or_mat *A, const or_mat *P1, const or_mat *P2, const or_f3r_params *p,
                         int64_t cnt0, float *sum, float *ome, const float *in, float *out) {
  f3r_ctx c;
  memset(&c, 0, sizeof(c));
  int32_t n = A->n;
  c.n = n; c.A = A; c.P1 = P1; c.P2 = P2; c.p = *p;
  c.v16 = (f16 *)malloc(sizeof(f16) * (size_t)A->nnz);
  for (int32_t q = 0; q < A->nnz; q++) c.v16[q] = (f16)A->val[q];
  c.hin = malloc(sizeof(f16) * n); c.hout = malloc(sizeof(f16) * n); c.tmp = malloc(sizeof(f16) * n);
  c.tmp2 = malloc(sizeof(f16) * n); c.hr = malloc(sizeof(f16) * n);
  c.cnt = cnt0;
  c.den = (int32_t)(cnt0 / p->c);
  for (int k = 0; k < p->m4 && k < MAXM4; k++) { c.sum[k] = sum[k]; c.ome[k] = (f16)ome[k]; }
  level4(&c, in, out);
  for (int k = 0; k < p->m4 && k < MAXM4; k++) { sum[k] = c.sum[k]; ome[k] = (float)c.ome[k]; }
  free(c.v16); free(c.hin); free(c.hout); free(c.tmp); free(c.tmp2); free(c.hr);
}

/* One inner FGMRES level (level 2 with fp32 matrix when level==2 and its
 * nested levels, or level 3 alone when level==3) with a fresh R state.    */
void or_inner_level_apply(const or_mat *A, const or_mat *P1, const or_mat *P2, const or_f3r_params *p,
                          int level, const float *in, float *out) {
  f3r_ctx c;
  memset(&c, 0, sizeof(c));
  int32_t n = A->n;
  c.n = n; c.A = A; c.P1 = P1; c.P2 = P2; c.p = *p;
  c.v32 = (float *)malloc(sizeof(float) * (size_t)A->nnz);
  c.v16 = (f16 *)malloc(sizeof(f16) * (size_t)A->nnz);
  for (int32_t q = 0; q < A->nnz; q++) { c.v32[q] = (float)A->val[q]; c.v16[q] = (f16)A->val[q]; }
  c.hin = malloc(sizeof(f16) * n); c.hout = malloc(sizeof(f16) * n); c.tmp = malloc(sizeof(f16) * n);
  c.tmp2 = malloc(sizeof(f16) * n); c.hr = malloc(sizeof(f16) * n);
  c.cnt = p->c;
  for (int k = 0; k < MAXM4; k++) { c.sum[k] = 1.0f; c.ome[k] = (f16)1.0f; }
  level_inner(&c, level, in, out);
  free(c.v32); free(c.v16); free(c.hin); free(c.hout); free(c.tmp); free(c.tmp2); free(c.hr);
}

/* fp64 -> fp16 conversion used for device uploads (checks the product's
 * own rounding routine)                                                    */
void or_f64_to_f16(int64_t n, const double *in, uint16_t *out) {
  for (int64_t i = 0; i < n; i++) {
    f16 h = (f16)in[i];
    memcpy(&out[i], &h, 2);
  }
}
