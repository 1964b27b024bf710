// ref_gen.cpp -- TEST INFRASTRUCTURE: exposes the reference's own stencil
// generators (matrix/hpcg.cpp:13-57 and matrix/hpgmp.cpp:13-57) to the
// golden-vector script.  The two generator files are compiled in from the
// reference tree (their main() renamed) and turned into a sorted CSR through
// the reference's io::CSR (library/umineko-sparse/matrix/io.hpp:47-63).
#include <cmath>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#define main ref_hpcg_unused_main
namespace ref_hpcg {
#include "matrix/hpcg.cpp"
}
#undef main
#define main ref_hpgmp_unused_main
namespace ref_hpgmp {
#include "matrix/hpgmp.cpp"
}
#undef main

#include "umineko-sparse/matrix/csr.hpp"
#include "umineko-sparse/matrix/io.hpp"

template <class COO>
static int64_t to_csr(const COO &coo, int32_t *rptr, int32_t *idx, double *val) {
  using namespace kmm;
  const int32_t n = (int32_t)coo.n, nnz = (int32_t)coo.nnz;
  auto row = vector<int32_t, host>(nnz), col = vector<int32_t, host>(nnz);
  auto v = vector<double, host>(nnz);
  for (int32_t i = 0; i < nnz; i++) {
    row[i] = (int32_t)coo.row[i] - 1;  // Matrix Market is 1-based (io.hpp:167-168)
    col[i] = (int32_t)coo.col[i] - 1;
    v[i] = coo.val[i];
  }
  auto mcoo = io::COO<double>(impl::shape{n, n}, nnz, row, col, v);
  auto csr = CSR<double, host>(io::CSR<double>(mcoo));
  std::memcpy(rptr, csr.rptr.raw(), sizeof(int32_t) * (n + 1));
  std::memcpy(idx, csr.idx.raw(), sizeof(int32_t) * nnz);
  std::memcpy(val, csr.val.raw(), sizeof(double) * nnz);
  return nnz;
}

extern "C" int64_t ref_gen27(int variant, int nx, int ny, int nz, int32_t *rptr, int32_t *idx,
                             double *val) {
  if (variant == 0) return to_csr(ref_hpcg::generate_hpcg(nx, ny, nz), rptr, idx, val);
  return to_csr(ref_hpgmp::generate_hpgmp(nx, ny, nz, 0.5), rptr, idx, val);
}

// The half-space nonsymmetric 27-point stencil of the GPU workload (every
// neighbour with a positive linear offset gets -1+beta, negative -1-beta,
// diagonal 26), generated here independently of the product library and
// converted with the reference's io::CSR so the two generators can be
// cross-checked.
struct coo_t {
  std::vector<long> row, col;
  std::vector<double> val;
  long n, nnz;
};
extern "C" int64_t ref_gen27_halfspace(int nx, int ny, int nz, double beta, int32_t *rptr,
                                       int32_t *idx, double *val) {
  coo_t c;
  c.n = (long)nx * ny * nz;
  long cnt = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        long row = (long)k * ny * nx + (long)j * nx + i;
        for (int dz = -1; dz <= 1; dz++)
          for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
              int kk = k + dz, jj = j + dy, ii = i + dx;
              if (kk < 0 || jj < 0 || ii < 0 || kk >= nz || jj >= ny || ii >= nx) continue;
              long col = (long)kk * ny * nx + (long)jj * nx + ii;
              c.row.push_back(row + 1);
              c.col.push_back(col + 1);
              c.val.push_back(row == col ? 26.0 : (col > row ? -1.0 + beta : -1.0 - beta));
              cnt++;
            }
      }
  c.nnz = cnt;
  return to_csr(c, rptr, idx, val);
}

// The reference generators' own file writer (matrix/hpcg.cpp:60-69,
// matrix/hpgmp.cpp): the .mtx files its suites read (hpcg_7_7_7.mtx, ...).
extern "C" void ref_gen27_save(int variant, int nx, int ny, int nz, const char *path) {
  if (variant == 0)
    ref_hpcg::save_matrix_market(path, ref_hpcg::generate_hpcg(nx, ny, nz));
  else
    ref_hpgmp::save_matrix_market(path, ref_hpgmp::generate_hpgmp(nx, ny, nz, 0.5));
}

// io::mm::read_system + io::CSR (matrix/io.hpp:104-126, 44-60) with the
// drivers' init (work/src/f3r-gpu.cpp:60), as a handle.
namespace {
struct mm_system {
  kmm::CSR<double, kmm::host> a;
  kmm::vector<double, kmm::host> b;
};
}  // namespace
extern "C" void *ref_mm_read_system(const char *path) {
  using namespace kmm;
  auto [coo, rhs] = io::mm::read_system(path, [](vector<double, host> v) { v.random<0, 1>(std::mt19937_64(0)); });
  return new mm_system{CSR<double, host>(io::CSR(coo)), rhs};
}
extern "C" void ref_mm_dims(void *h, int32_t *n, int32_t *nnz) {
  auto *s = (mm_system *)h;
  *n = s->a.nrows();
  *nnz = s->a.nnz();
}
extern "C" void ref_mm_copy(void *h, int32_t *rptr, int32_t *idx, double *val, double *b) {
  auto *s = (mm_system *)h;
  std::memcpy(rptr, s->a.rptr.raw(), sizeof(int32_t) * (s->a.nrows() + 1));
  std::memcpy(idx, s->a.idx.raw(), sizeof(int32_t) * s->a.nnz());
  std::memcpy(val, s->a.val.raw(), sizeof(double) * s->a.nnz());
  std::memcpy(b, s->b.raw(), sizeof(double) * s->a.nrows());
}
extern "C" void ref_mm_free(void *h) { delete (mm_system *)h; }
