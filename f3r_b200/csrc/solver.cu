// solver.cu -- device objects (context, SELL-C-sigma matrices), the nested
// F3R solver orchestration, and the C ABI of include/f3r_b200.h.
//
// Solver structure (the reference assembles the same nesting in
// work/src/f3r-gpu.cpp:210-265):
//   Restarted( FGMRES<double>(A, L2, m_outer, normalize) , max_restarts )
//   L2 = FGMRES<float>(A32, L3, m2)         fp32 matrix and vectors
//   L3 = FGMRES<float>(A16, R, m3)          fp16 matrix, fp32 vectors
//   R  = adaptive-weight Richardson(m4, c)  fp16 vectors, SDAINV / BJ-ILU(0)
// Levels 2-4 run a fixed number of steps with no host decision, so one outer
// step's call into L2 is a static sequence of kernels; it is launched
// asynchronously (optionally as a replayed CUDA graph) and the host
// synchronises once per outer Arnoldi step to evaluate cond().
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "internal.hpp"
#include "kernels.cuh"
#include "ilu.cuh"
#include "objects.cuh"
#include "trsv.hpp"

namespace f3r {

static thread_local std::string g_err;
Status fail(Status code, const std::string &msg) {
  g_err = msg;
  return code;
}

// ---------------------------------------------------------------------------
// SELL-32 construction on the host
// ---------------------------------------------------------------------------
// Re-expresses the column indices as 16-bit offsets from the smallest index
// of each slice column, if every slice column spans fewer than 65536 columns.
bool compress_index16(SellHost &s) {
  const int64_t ncolsl = s.sptr[s.nslices];
  std::vector<int32_t> base(ncolsl);
  bool ok = true;
#pragma omp parallel for schedule(static) reduction(&& : ok)
  for (int64_t c = 0; c < ncolsl; c++) {
    int32_t lo = INT32_MAX, hi = INT32_MIN;
    for (int l = 0; l < 32; l++) {
      const int32_t v = s.col[c * 32 + l];
      lo = std::min(lo, v);
      hi = std::max(hi, v);
    }
    base[c] = lo;
    ok = ok && ((int64_t)hi - lo <= 65535);
  }
  if (!ok) return false;
  s.dcol.resize(s.col.size());
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < ncolsl; c++)
    for (int l = 0; l < 32; l++) s.dcol[c * 32 + l] = (uint16_t)(s.col[c * 32 + l] - base[c]);
  // bases laid out per slice from a multiple of 4 (16-byte aligned copies)
  s.cbptr.assign(s.nslices + 1, 0);
  for (int32_t sl = 0; sl < s.nslices; sl++) s.cbptr[sl + 1] = s.cbptr[sl] + ((s.sptr[sl + 1] - s.sptr[sl] + 3) & ~3);
  s.cbase.assign((size_t)s.cbptr[s.nslices] + 4, 0);
#pragma omp parallel for schedule(static)
  for (int32_t sl = 0; sl < s.nslices; sl++)
    for (int32_t k = 0; k < s.sptr[sl + 1] - s.sptr[sl]; k++) s.cbase[s.cbptr[sl] + k] = base[s.sptr[sl] + k];
  std::vector<int32_t>().swap(s.col);
  return true;
}

// renumber = true builds P A P^T (columns mapped to storage order) for the
// solver's permuted system; false keeps original columns and scatters rows.
// Offset-aligned slices.  Per slice, D = the sorted set of offsets
// column - row over its rows (storage numbering).  A slice can be aligned when
// |D| is at most 5/4 of its packed width: slice column k then becomes offset
// D_k for every row (a zero where the row has no entry at that offset) and no
// index is stored.  Within a row the entries stay in increasing column order,
// so the product's sums are unchanged (a zero entry adds 0 x to the chain).
//  * Every slice alignable (stencil-like matrices): the fully aligned form,
//    kAllAlignedChunk-column chunks; a slice whose columns first row + D_k +
//    lane can leave [0, ncols) is flagged in bit 0 of cbptr and clamped.
//  * Otherwise the mixed form: slices that are alignable and in range are
//    aligned, the rest keep explicit indices (compact, from xoff);
//    kAlignedChunk-column chunks.
// Slice widths are padded to a multiple of 4 and each chunk stores its values
// lane-major (a lane's values contiguous), so the kernel reads them with
// vector loads.
double align_offsets(const f3r_csr &a, bool renumber, SellHost &s) {
  const int32_t n = s.n, ns = s.nslices, nc = s.ncols;
  std::vector<int32_t> iperm;
  if (renumber) {
    iperm.resize(n);
    for (int32_t i = 0; i < n; i++) iperm[s.perm[i]] = i;
  }
  auto colof = [&](int32_t q) { return renumber ? iperm[a.idx[q]] : a.idx[q]; };
  std::vector<std::vector<int32_t>> D(ns);
  std::vector<char> shape_ok(ns, 1), in_range(ns, 1);
  int64_t not_ok = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : not_ok)
  for (int32_t sl = 0; sl < ns; sl++) {
    const int32_t wstd = s.sptr[sl + 1] - s.sptr[sl];
    if (wstd == 0) continue;
    std::vector<int32_t> d;
    d.reserve((size_t)wstd * 2);
    for (int32_t l = 0; l < 32; l++) {
      const int64_t r = (int64_t)sl * 32 + l;
      if (r >= n) break;
      const int32_t o = s.perm[r];
      for (int32_t q = a.rptr[o]; q < a.rptr[o + 1]; q++) d.push_back(colof(q) - (int32_t)r);
    }
    std::sort(d.begin(), d.end());
    d.erase(std::unique(d.begin(), d.end()), d.end());
    const int64_t lo = (int64_t)sl * 32 + d.front(), hi = (int64_t)sl * 32 + d.back() + 31;
    in_range[sl] = lo >= 0 && hi < nc;
    shape_ok[sl] = (int64_t)d.size() * 4 <= (int64_t)wstd * 5;
    if (!shape_ok[sl]) not_ok++;
    D[sl] = std::move(d);
  }
  const bool all = not_ok == 0;
  const int32_t chunk = all ? kAllAlignedChunk : kAlignedChunk;
  std::vector<char> al(ns, 0);
  std::vector<int32_t> width(ns);
  for (int32_t sl = 0; sl < ns; sl++) {
    const int32_t wstd = s.sptr[sl + 1] - s.sptr[sl];
    al[sl] = wstd > 0 && shape_ok[sl] && (all || in_range[sl]);
    width[sl] = ((al[sl] ? (int32_t)D[sl].size() : wstd) + 3) & ~3;
  }
  std::vector<int32_t> sptr(ns + 1, 0), cbptr(ns + 1, 0), xoff(all ? 0 : ns, -1);
  int64_t nx = 0, na = 0;
  for (int32_t sl = 0; sl < ns; sl++) {
    if ((int64_t)sptr[sl] + width[sl] > INT32_MAX / 32) return -1.0;
    sptr[sl + 1] = sptr[sl] + width[sl];
    cbptr[sl + 1] = cbptr[sl] + (al[sl] ? width[sl] : 0);
    if (al[sl]) {
      na++;
    } else if (!all) {
      xoff[sl] = (int32_t)nx;
      nx += (int64_t)width[sl] * 32;
    }
  }
  const int64_t np = (int64_t)sptr[ns] * 32;
  std::vector<double> val(np, 0.0);
  std::vector<int32_t> col(std::max<int64_t>(nx, 1), 0), cbase((size_t)cbptr[ns] + 4, 0);
#pragma omp parallel for schedule(dynamic, 256)
  for (int32_t sl = 0; sl < ns; sl++) {
    const int32_t wp = width[sl];
    const int64_t nb = (int64_t)sptr[sl] * 32, ob = (int64_t)s.sptr[sl] * 32;
    // lane-major position of entry (k, lane) inside the slice
    auto at = [&](int32_t k, int32_t l) {
      const int32_t k0 = k / chunk * chunk, kw = std::min(chunk, wp - k0);
      return nb + (int64_t)k0 * 32 + (int64_t)l * kw + (k - k0);
    };
    if (al[sl]) {
      const std::vector<int32_t> &d = D[sl];
      // padding slots repeat the last offset (their values are zero)
      for (int32_t k = 0; k < wp; k++) cbase[cbptr[sl] + k] = sl * 32 + d[std::min<size_t>(k, d.size() - 1)];
      for (int32_t l = 0; l < 32; l++) {
        const int64_t r = (int64_t)sl * 32 + l;
        if (r >= n) break;
        const int32_t o = s.perm[r];
        for (int32_t q = a.rptr[o]; q < a.rptr[o + 1]; q++) {
          const int32_t k = (int32_t)(std::lower_bound(d.begin(), d.end(), colof(q) - (int32_t)r) - d.begin());
          val[at(k, l)] = a.val[q];
        }
      }
    } else if (wp > 0) {
      const int32_t wstd = s.sptr[sl + 1] - s.sptr[sl];
      for (int32_t k = 0; k < wp; k++)
        for (int32_t l = 0; l < 32; l++) {
          const int32_t ks = std::min(k, wstd - 1);
          col[xoff[sl] + (int64_t)k * 32 + l] = s.col[ob + (int64_t)ks * 32 + l];
          if (k < wstd) val[at(k, l)] = s.val[ob + (int64_t)k * 32 + l];
        }
    }
  }
  // the fully aligned form flags the slices to clamp in bit 0 of cbptr
  if (all)
    for (int32_t sl = 0; sl < ns; sl++)
      if (al[sl] && !in_range[sl]) cbptr[sl] |= 1;
  int32_t mw = 0;
  for (int32_t sl = 0; sl < ns; sl++) mw = std::max(mw, width[sl]);
  s.sptr = std::move(sptr);
  s.val = std::move(val);
  s.col = all ? std::vector<int32_t>() : std::move(col);
  s.cbase = std::move(cbase);
  s.cbptr = std::move(cbptr);
  s.xoff = std::move(xoff);
  s.aligned_all = all;
  s.dcol.clear();
  s.nnz_pad = np;
  s.max_width = mw;
  return ns ? (double)na / ns : 0.0;
}

Status build_sell(const f3r_csr &a, int32_t sigma, bool renumber, SellHost &s,
                  const std::vector<int32_t> *given_perm) {
  if (sigma < 1) return fail(F3R_ERROR_INVALID_VALUE, "sigma must be >= 1");
  if (renumber && a.nrows != a.ncols) return fail(F3R_ERROR_INVALID_VALUE, "symmetric permutation needs a square matrix");
  const int32_t n = a.nrows;
  s.n = n;
  s.ncols = a.ncols;
  s.sigma = sigma;
  s.nnz = a.nnz;
  s.nslices = (int32_t)cdiv(n, 32);
  s.perm.resize(n);
  std::iota(s.perm.begin(), s.perm.end(), 0);
  auto len = [&](int32_t r) { return a.rptr[r + 1] - a.rptr[r]; };
  if (given_perm) {
    s.perm = *given_perm;
  } else if (sigma > 1) {
    // rows ordered by decreasing length inside each window of sigma rows
    // (SELLsig, matrix/sell.hpp:309-343); stable for equal lengths
    for (int64_t w0 = 0; w0 < n; w0 += sigma) {
      const int64_t e = std::min<int64_t>(n, w0 + sigma);
      std::stable_sort(s.perm.begin() + w0, s.perm.begin() + e,
                       [&](int32_t x, int32_t y) { return len(x) > len(y); });
    }
  }
  std::vector<int32_t> iperm;
  if (renumber) {
    iperm.resize(n);
    for (int32_t i = 0; i < n; i++) iperm[s.perm[i]] = i;
  }
  s.sptr.assign(s.nslices + 1, 0);
  int32_t mw = 0;
  for (int32_t sl = 0; sl < s.nslices; sl++) {
    int32_t w = 0;
    for (int32_t l = 0; l < 32; l++) {
      const int64_t r = (int64_t)sl * 32 + l;
      if (r < n) w = std::max(w, len(s.perm[r]));
    }
    mw = std::max(mw, w);
    if ((int64_t)s.sptr[sl] + w > INT32_MAX / 32) return fail(F3R_ERROR_UNSUPPORTED, "padded matrix exceeds 2^31 entries");
    s.sptr[sl + 1] = s.sptr[sl] + w;
  }
  s.max_width = mw;
  s.nnz_pad = (int64_t)s.sptr[s.nslices] * 32;
  s.col.assign(s.nnz_pad, 0);
  s.val.assign(s.nnz_pad, 0.0);
#pragma omp parallel for schedule(static)
  for (int32_t sl = 0; sl < s.nslices; sl++) {
    const int64_t base = (int64_t)s.sptr[sl] * 32;
    const int32_t w = s.sptr[sl + 1] - s.sptr[sl];
    for (int32_t l = 0; l < 32; l++) {
      const int64_t r = (int64_t)sl * 32 + l;
      int32_t c = 0, prev = 0;
      if (r < n) {
        const int32_t o = s.perm[r];
        for (int32_t q = a.rptr[o]; q < a.rptr[o + 1]; q++, c++) {
          prev = renumber ? iperm[a.idx[q]] : a.idx[q];
          s.col[base + (int64_t)c * 32 + l] = prev;
          s.val[base + (int64_t)c * 32 + l] = a.val[q];
        }
      }
      for (; c < w; c++) s.col[base + (int64_t)c * 32 + l] = prev;
    }
  }
  return F3R_SUCCESS;
}

Status upload_sell(Context &c, const SellHost &h, int dtype_mask, bool scatter_perm, DeviceSell &d) {
  d.n = h.n; d.ncols = h.ncols; d.nslices = h.nslices; d.max_width = h.max_width; d.sigma = h.sigma;
  d.nnz = h.nnz; d.nnz_pad = h.nnz_pad; d.dtypes = dtype_mask;
  const size_t np = (size_t)h.nnz_pad;
  if (!h.xoff.empty() || h.aligned_all) {
    const size_t nc = h.cbase.size(), nx = h.col.size();
    F3R_TRY(c.alloc((void **)&d.cbase, nc * 4));
    F3R_TRY(c.alloc((void **)&d.cbptr, (size_t)(h.nslices + 1) * 4));
    CUDA_TRY(cudaMemcpyAsync(d.cbase, h.cbase.data(), nc * 4, cudaMemcpyHostToDevice, c.stream));
    CUDA_TRY(cudaMemcpyAsync(d.cbptr, h.cbptr.data(), (size_t)(h.nslices + 1) * 4, cudaMemcpyHostToDevice, c.stream));
    if (!h.aligned_all) {  // mixed form: the explicit slices' indices
      F3R_TRY(c.alloc((void **)&d.col, nx * 4));
      F3R_TRY(c.alloc((void **)&d.xoff, (size_t)std::max(h.nslices, 1) * 4));
      CUDA_TRY(cudaMemcpyAsync(d.col, h.col.data(), nx * 4, cudaMemcpyHostToDevice, c.stream));
      CUDA_TRY(cudaMemcpyAsync(d.xoff, h.xoff.data(), (size_t)h.nslices * 4, cudaMemcpyHostToDevice, c.stream));
    }
  } else if (!h.dcol.empty()) {
    const size_t nc = h.cbase.size();
    F3R_TRY(c.alloc((void **)&d.dcol, np * 2));
    F3R_TRY(c.alloc((void **)&d.cbase, nc * 4));
    F3R_TRY(c.alloc((void **)&d.cbptr, (size_t)(h.nslices + 1) * 4));
    CUDA_TRY(cudaMemcpyAsync(d.dcol, h.dcol.data(), np * 2, cudaMemcpyHostToDevice, c.stream));
    CUDA_TRY(cudaMemcpyAsync(d.cbase, h.cbase.data(), nc * 4, cudaMemcpyHostToDevice, c.stream));
    CUDA_TRY(cudaMemcpyAsync(d.cbptr, h.cbptr.data(), (size_t)(h.nslices + 1) * 4, cudaMemcpyHostToDevice, c.stream));
  } else {
    F3R_TRY(c.alloc((void **)&d.col, np * 4));
    CUDA_TRY(cudaMemcpyAsync(d.col, h.col.data(), np * 4, cudaMemcpyHostToDevice, c.stream));
  }
  F3R_TRY(c.alloc((void **)&d.sptr, (size_t)(h.nslices + 1) * 4));
  CUDA_TRY(cudaMemcpyAsync(d.sptr, h.sptr.data(), (size_t)(h.nslices + 1) * 4, cudaMemcpyHostToDevice, c.stream));
  if (scatter_perm && h.sigma > 1) {
    F3R_TRY(c.alloc((void **)&d.perm, (size_t)std::max(h.n, 1) * 4));
    CUDA_TRY(cudaMemcpyAsync(d.perm, h.perm.data(), (size_t)h.n * 4, cudaMemcpyHostToDevice, c.stream));
  }
  double *tmp64 = nullptr;
  F3R_TRY(c.alloc((void **)&tmp64, np * 8));
  CUDA_TRY(cudaMemcpyAsync(tmp64, h.val.data(), np * 8, cudaMemcpyHostToDevice, c.stream));
  const int g = c.ew_grid((int64_t)np);
  if (dtype_mask & (1 << F3R_F32)) {
    F3R_TRY(c.alloc((void **)&d.v32, np * 4));
    launch_k(c, k_convert_vals<float>, g, kEwThreads, 0, c.stream, tmp64, d.v32, (int64_t)np);
  }
  if (dtype_mask & (1 << F3R_F16)) {
    F3R_TRY(c.alloc((void **)&d.v16, np * 2));
    launch_k(c, k_convert_vals<__half>, g, kEwThreads, 0, c.stream, tmp64, d.v16, (int64_t)np);
  }
  CUDA_TRY(cudaGetLastError());
  if (dtype_mask & (1 << F3R_F64)) {
    d.v64 = tmp64;
  } else {
    CUDA_TRY(cudaStreamSynchronize(c.stream));
    cudaFree(tmp64);
  }
  CUDA_TRY(cudaStreamSynchronize(c.stream));
  return F3R_SUCCESS;
}

// ---------------------------------------------------------------------------
// SpMV launcher
// ---------------------------------------------------------------------------
Status upload_csr(Context &c, const f3r_csr &a, int dtype_mask, DeviceSell &d) {
  const int32_t n = a.nrows;
  const size_t nz = (size_t)a.nnz;
  d.n = n;
  d.ncols = a.ncols;
  d.nslices = (int32_t)cdiv(n, 32);
  d.sigma = 1;
  d.nnz = a.nnz;
  d.nnz_pad = a.nnz;
  d.dtypes = dtype_mask;
  int32_t mw = 0;
  for (int32_t i = 0; i < n; i++) mw = std::max(mw, a.rptr[i + 1] - a.rptr[i]);
  d.max_width = mw;
  // the kernel's 16-byte copies may read up to 15 bytes past the last entry: kCsrPad elements of padding
  const size_t na = nz + kCsrPad;
  F3R_TRY(c.alloc((void **)&d.rptr, ((size_t)n + 1) * 4));
  F3R_TRY(c.alloc((void **)&d.col, na * 4));
  CUDA_TRY(cudaMemcpyAsync(d.rptr, a.rptr, ((size_t)n + 1) * 4, cudaMemcpyHostToDevice, c.stream));
  if (nz) CUDA_TRY(cudaMemcpyAsync(d.col, a.idx, nz * 4, cudaMemcpyHostToDevice, c.stream));
  double *tmp64 = nullptr;
  F3R_TRY(c.alloc((void **)&tmp64, na * 8));
  if (nz) CUDA_TRY(cudaMemcpyAsync(tmp64, a.val, nz * 8, cudaMemcpyHostToDevice, c.stream));
  const int g = c.ew_grid((int64_t)nz);
  if (dtype_mask & (1 << F3R_F32)) {
    F3R_TRY(c.alloc((void **)&d.v32, na * 4));
    launch_k(c, k_convert_vals<float>, g, kEwThreads, 0, c.stream, tmp64, d.v32, (int64_t)nz);
  }
  if (dtype_mask & (1 << F3R_F16)) {
    F3R_TRY(c.alloc((void **)&d.v16, na * 2));
    launch_k(c, k_convert_vals<__half>, g, kEwThreads, 0, c.stream, tmp64, d.v16, (int64_t)nz);
  }
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(c.stream));
  if (dtype_mask & (1 << F3R_F64)) d.v64 = tmp64;
  else cudaFree(tmp64);
  return F3R_SUCCESS;
}

// fp16 copy of fp64 values (rounded once on the device), recorded in allocs
static Status half_upload(std::vector<void *> &allocs, __half **d, const std::vector<double> &v) {
  double *tmp = nullptr;
  const size_t nb = std::max<size_t>(v.size(), 1);
  CUDA_TRY(cudaMalloc((void **)&tmp, nb * sizeof(double)));
  cudaError_t e = cudaMalloc((void **)d, nb * sizeof(__half));
  if (e != cudaSuccess) {
    cudaFree(tmp);
    return fail(F3R_ERROR_OUT_OF_MEMORY, "ILU values");
  }
  allocs.push_back((void *)*d);
  CUDA_TRY(cudaMemcpy(tmp, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
  const int64_t n = (int64_t)v.size();
  const int g = (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, kEwThreads), 1024));
  k_convert_vals<__half><<<g, kEwThreads>>>(tmp, *d, n);
  CUDA_TRY(cudaDeviceSynchronize());
  cudaFree(tmp);
  return F3R_SUCCESS;
}
Status IluDevice::to_half(__half **d, const std::vector<double> &v) { return half_upload(allocs, d, v); }
Status IluLevel::half_copy(__half **d, const std::vector<double> &v) { return half_upload(allocs, d, v); }

}  // namespace f3r

using namespace f3r;

// ---------------------------------------------------------------------------
// solver
// ---------------------------------------------------------------------------
namespace f3r {

__global__ void k_set_slots(double **in_slot, double **out_slot, double *in, double *out) {
  *in_slot = in;
  *out_slot = out;
}

template <typename T> struct Level {
  int m = 0;
  T *V = nullptr, *Z = nullptr;  // column-major n x (m+1), n x m (level 3 V column 0 is an alias)
  T *H = nullptr, *cs = nullptr, *sn = nullptr, *e = nullptr, *y = nullptr, *inv = nullptr;
};

struct Solver {
  f3r_context *ctx = nullptr;
  f3r_params p{};
  int32_t n = 0;
  int64_t ldn = 0;  // column stride of the Krylov bases: n rounded up to 8 (64-byte aligned columns)
  DeviceSell A;
  std::vector<int32_t> perm;  // storage row -> original row (sigma > 1)
  int32_t *perm_d = nullptr;
  // preconditioner
  int precond_diag = 0;
  __half *wd = nullptr, *zd = nullptr;
  DeviceSell W, Z;    // general SDAINV factors (permuted system)
  IluDevice ilu;      // block-Jacobi ILU(0), level scheduled
  IluLevel ilul;      // global ILU(0), level scheduled over the whole GPU
  JacobiTrsv jl, ju;  // the same factors solved by Jacobi / BAJ sweeps
  // levels
  Level<double> L1;
  Level<float> L2, L3;
  double *abs_e = nullptr;
  __half *hin = nullptr, *hout = nullptr, *hout2 = nullptr, *tmp = nullptr, *tmp2 = nullptr, *hr = nullptr;
  RichState *rs = nullptr;
  double **in_slot = nullptr;
  double **out_slot = nullptr;
  double *b_d = nullptr, *x_d = nullptr, *bp_d = nullptr, *xp_d = nullptr, *r_d = nullptr;
  int64_t cnt = 0;
  int64_t r_calls = 0;
  std::vector<void *> allocs;
  std::map<std::vector<bool>, std::pair<cudaGraphExec_t, int64_t>> graphs;  // exec, kernels in it
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  Context &C() { return *ctx; }
  template <typename T> Status alloc(T **p, size_t count) {
    F3R_TRY(ctx->alloc((void **)p, count * sizeof(T)));
    allocs.push_back((void *)*p);
    return F3R_SUCCESS;
  }
  ~Solver() {
    for (auto &kv : graphs) cudaGraphExecDestroy(kv.second.first);
    for (void *q : allocs) cudaFree(q);
    A.release(); W.release(); Z.release(); ilu.release(); ilul.release(); jl.release(); ju.release();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }

  template <typename T> Status make_level(Level<T> &L, int m, bool own_v0) {
    L.m = m;
    const size_t nn = (size_t)std::max<int64_t>(ldn, 8);
    F3R_TRY(alloc(&L.V, nn * (size_t)(m + (own_v0 ? 1 : 0))));
    F3R_TRY(alloc(&L.Z, nn * (size_t)m));
    F3R_TRY(alloc(&L.H, (size_t)(m + 1) * m));
    F3R_TRY(alloc(&L.cs, (size_t)m));
    F3R_TRY(alloc(&L.sn, (size_t)m));
    F3R_TRY(alloc(&L.e, (size_t)m + 1));
    F3R_TRY(alloc(&L.y, (size_t)m));
    F3R_TRY(alloc(&L.inv, 1));
    CUDA_TRY(cudaMemset(L.H, 0, sizeof(T) * (size_t)(m + 1) * m));
    CUDA_TRY(cudaMemset(L.e, 0, sizeof(T) * (size_t)(m + 1)));
    return F3R_SUCCESS;
  }

  // ---- level 4: R(in) -> out -------------------------------------------------
  // in_inv: 1/h of the basis vector `in` when its normalisation is still
  // pending (done in place by the first kernel), else nullptr
  Status rich_apply(float *in, float *out, float *e_set, const float *in_inv) {
    const int64_t N = n;
    const int g = C().ew_grid(N);
    const int gv = C().ew_grid(cdiv(N, 4));
    cudaStream_t st = C().stream;
    ++cnt;
    ++r_calls;
    const bool upd = p.static_weight <= 0 && (cnt % p.c) == 0;  // F3R-Static never updates
    const float sc = std::ldexp(1.0f, p.half_scale_log2), isc = std::ldexp(1.0f, -p.half_scale_log2);
    const DevSell Av = A.view();
    if (precond_diag) {
      const DiagPre M{wd, zd};
      if (!upd) {
        launch_k(C(), k_rich_enter_diag<true>, gv, kEwThreads, 0, st, in, in_inv, sc, M, hin, hout, rs, e_set, N);
        __half *cur = hout, *nxt = hout2;
        for (int k = 1; k < p.m4; k++) {
          const bool last = (k == p.m4 - 1);
          EpiRichStep epi{hin, cur, M, rs, k, last ? nullptr : nxt, last ? out : nullptr, isc};
          F3R_TRY(launch_sell(C(), A.v16, Av, (const __half *)cur, epi));
          std::swap(cur, nxt);
        }
        if (p.m4 == 1) launch_k(C(), k_rich_exit, g, kEwThreads, 0, st, hout, out, isc, N);
      } else {
        launch_k(C(), k_rich_enter_diag<false>, gv, kEwThreads, 0, st, in, in_inv, sc, M, hin, hout, rs, e_set, N);
        F3R_TRY(launch_sell(C(), A.v16, Av, (const __half *)hout, EpiRichWeight{tmp, hin, C().gred(), rs, 0}));
        launch_k(C(), k_rich_scale_om, g, kEwThreads, 0, st, hout, rs, N);
        for (int k = 1; k < p.m4; k++) {
          const bool last = (k == p.m4 - 1);
          F3R_TRY(launch_sell(C(), A.v16, Av, (const __half *)hout, EpiRichResPre{hin, M, hr, tmp2}));
          F3R_TRY(launch_sell(C(), A.v16, Av, (const __half *)tmp2, EpiRichWeight{tmp, hr, C().gred(), rs, k}));
          launch_k(C(), k_rich_axpy, g, kEwThreads, 0, st, hout, tmp2, rs, k, 0, last ? out : nullptr, isc, N);
        }
        if (p.m4 == 1) launch_k(C(), k_rich_exit, g, kEwThreads, 0, st, hout, out, isc, N);
      }
    } else {
      // general preconditioner: M = Z W^T (SDAINV) or U^-1 L^-1 (ILU)
      launch_k(C(), k_rich_cast_in, g, kEwThreads, 0, st, in, in_inv, sc, hin, e_set, N);
      F3R_TRY(prec_apply(hin, hout, !upd));
      if (upd) {
        F3R_TRY(launch_sell(C(), A.v16, Av, (const __half *)hout, EpiRichWeight{tmp, hin, C().gred(), rs, 0}));
        launch_k(C(), k_rich_scale_om, g, kEwThreads, 0, st, hout, rs, N);
      }
      for (int k = 1; k < p.m4; k++) {
        const bool last = (k == p.m4 - 1);
        F3R_TRY(launch_sell(C(), A.v16, Av, (const __half *)hout, EpiResidual<__half, __half>{hin, hr, nullptr}));
        F3R_TRY(prec_apply(hr, tmp2, false));
        if (upd) F3R_TRY(launch_sell(C(), A.v16, Av, (const __half *)tmp2, EpiRichWeight{tmp, hr, C().gred(), rs, k}));
        launch_k(C(), k_rich_axpy, g, kEwThreads, 0, st, hout, tmp2, rs, k, upd ? 0 : 1, last ? out : nullptr, isc, N);
      }
      if (p.m4 == 1) launch_k(C(), k_rich_exit, g, kEwThreads, 0, st, hout, out, isc, N);
    }
    CUDA_TRY(cudaGetLastError());
    return F3R_SUCCESS;
  }

  // out = M x for the general preconditioners; scale_ome multiplies by ome[0]
  Status prec_apply(const __half *x, __half *out, bool scale_ome) {
    if (p.precond == F3R_PRECOND_SDAINV) {
      F3R_TRY(launch_sell(C(), W.v16, W.view(), x, EpiStore<__half>{tmp, nullptr}));
      F3R_TRY(launch_sell(C(), Z.v16, Z.view(), (const __half *)tmp, EpiZScale{out, rs, scale_ome ? 1 : 0}));
    } else if (p.precond == F3R_PRECOND_ILU0_BJ) {
      F3R_TRY(ilu.apply(C().stream, x, tmp, out, scale_ome ? &rs->ome[0] : nullptr));
      C().launches += 2;
    } else if (p.precond == F3R_PRECOND_ILU0_LEVEL) {
      F3R_TRY(ilul.apply(C().stream, x, tmp, out, scale_ome ? &rs->ome[0] : nullptr, C().err));
      C().launches += 2;
    } else {
      F3R_TRY(jl.apply(C(), x, tmp, nullptr));
      F3R_TRY(ju.apply(C(), tmp, out, scale_ome ? &rs->ome[0] : nullptr));
    }
    return F3R_SUCCESS;
  }

  // w = A z with H(j, 0..nv-1) = <w, V(k)> fused; the dot count picks the
  // smallest epilogue instantiation (registers)
  //
  // The dots can ride in the SpMV epilogue (one read of w less) or run as a
  // separate vectorised pass.  On B200 the SELL kernel is bound by the
  // latency of each warp's slice loop, and the fused epilogue stretches it:
  // 239 us fused against 187 + ~20 us separate for the 192^3 fp16 product, so
  // the fp16 level uses the separate pass; the fp32 level keeps the fusion
  // for up to 4 dots (its product streams more bytes per slice and hides the
  // epilogue: 244 us fused against 228 + ~20 us) and separates wider ones.
  // H(j, 0..nv-1) = <w, V(k)>, one vectorised pass
  void dots(const float *w, const Cols<float> &Vc, int nv, float *hcol) {
    const int gv = C().ew_grid(cdiv(n, 4));
    if (nv <= 4)
      launch_k(C(), k_multidot_f32<4, 8>, gv, 256, 0, C().stream, w, Vc, nv, (int64_t)n, C().gred(), hcol);
    else if (nv <= 8)
      launch_k(C(), k_multidot_f32<8, 8>, gv, 256, 0, C().stream, w, Vc, nv, (int64_t)n, C().gred(), hcol);
    else
      launch_k(C(), k_multidot_chunked<float, 8>, C().ew_grid(n), 256, 0, C().stream, w, Vc, nv, (int64_t)n,
               C().gred(), hcol);
  }

  template <typename V>
  Status spmv_dots(const V *vals, const float *z, float *w, const Cols<float> &Vc, int nv, float *hcol) {
    if (sizeof(V) == 2 || nv > 4) {
      F3R_TRY(launch_sell(C(), vals, A.view(), z, EpiStore<float>{w, nullptr}));
      dots(w, Vc, nv, hcol);
      return F3R_SUCCESS;
    }
    if (nv <= 4) return launch_sell(C(), vals, A.view(), z, EpiStoreDots<4>{w, Vc, nv, C().gred(), hcol});
    return launch_sell(C(), vals, A.view(), z, EpiStoreDots<8>{w, Vc, nv, C().gred(), hcol});
  }

  // sFGMRES's second and third loops (gmres2.hpp:181-193): classical
  // Gram-Schmidt of the stored raw vectors W(1..m) against the basis built so
  // far, with each Givens rotation fused into its step as in FGMRES (the
  // rotation of column j needs only column j).  The next step reads V(j+1)
  // through the dots and the update, so it is normalised explicitly here.
  Status sstep_orthogonalise(Level<float> &L, float *const *Vp, const Cols<float> &V) {
    const int64_t N = n;
    const int gv = C().ew_grid(cdiv(N, 4));
    for (int j = 0; j < L.m; j++) {
      float *w = Vp[j + 1];
      dots(w, V, j + 1, L.H + (size_t)j * (L.m + 1));
      GivensCtl<float> g{L.H, L.cs, L.sn, L.e, L.y, L.inv, nullptr, L.m + 1, j, j == L.m - 1, C().err};
      launch_k(C(), k_cgs_update<float, 8>, gv, 256, 0, C().stream, w, V, j + 1, N, C().gred(), g);
      if (j + 1 < L.m) launch_k(C(), k_scale<float>, gv, kEwThreads, 0, C().stream, w, (const float *)L.inv, N);
    }
    CUDA_TRY(cudaGetLastError());
    return F3R_SUCCESS;
  }

  // ---- level 3: FGMRES<float>(A16, R, m3), input V2 column, output Z2 col ----
  // The normalisation V(j+1) *= 1/h of every basis vector is deferred to the
  // first kernel that reads it next (the Richardson entry), which scales it
  // in place; the last basis vector of a level is never read again and is
  // left unscaled.  in_inv is the pending factor of `in` (nullptr if none).
  Status level3(float *in, float *out, const float *in_inv) {
    Level<float> &L = L3;
    const int64_t N = n;
    const int gv = C().ew_grid(cdiv(N, 4));
    float *Vp[kMaxCols];
    Cols<float> V{}, Zc{};
    Vp[0] = in;
    for (int k = 1; k <= L.m; k++) Vp[k] = L.V + (size_t)(k - 1) * ldn;
    for (int k = 0; k <= L.m; k++) V.p[k] = Vp[k];
    for (int k = 0; k < L.m; k++) Zc.p[k] = L.Z + (size_t)k * ldn;
    if (p.inner_sstep & 2) {
      // sFGMRES (gmres2.hpp:176-180): W(j+1) = A16 R W(j) on the raw vectors
      for (int j = 0; j < L.m; j++) {
        float *zj = L.Z + (size_t)j * ldn;
        F3R_TRY(rich_apply(Vp[j], zj, j == 0 ? L.e : nullptr, j == 0 ? in_inv : nullptr));
        F3R_TRY(launch_sell(C(), A.v16, A.view(), (const float *)zj, EpiStore<float>{Vp[j + 1], nullptr}));
      }
      F3R_TRY(sstep_orthogonalise(L, Vp, V));
    } else {
      for (int j = 0; j < L.m; j++) {
        float *zj = L.Z + (size_t)j * ldn;
        float *w = Vp[j + 1];
        F3R_TRY(rich_apply(Vp[j], zj, j == 0 ? L.e : nullptr, j == 0 ? in_inv : L.inv));
        F3R_TRY(spmv_dots(A.v16, zj, w, V, j + 1, L.H + (size_t)j * (L.m + 1)));
        GivensCtl<float> g{L.H, L.cs, L.sn, L.e, L.y, L.inv, nullptr, L.m + 1, j, j == L.m - 1, C().err};
        launch_k(C(), k_cgs_update<float, 8>, gv, 256, 0, C().stream, w, V, j + 1, N, C().gred(), g);
      }
    }
    launch_k(C(), k_zy<float, float, false>, gv, kEwThreads, 0, C().stream, Zc, L.y, L.m, out, nullptr, N);
    CUDA_TRY(cudaGetLastError());
    return F3R_SUCCESS;
  }

  // ---- level 2: FGMRES<float>(A32, L3, m2); in/out through the slots -------
  Status level2() {
    Level<float> &L = L2;
    const int64_t N = n;
    const int gv = C().ew_grid(cdiv(N, 4));
    float *Vp[kMaxCols];
    Cols<float> V{}, Zc{};
    for (int k = 0; k <= L.m; k++) V.p[k] = Vp[k] = L.V + (size_t)k * ldn;
    for (int k = 0; k < L.m; k++) Zc.p[k] = L.Z + (size_t)k * ldn;
    // normalises the outer basis vector in place (its 1/h is L1.inv) and casts it
    launch_k(C(), k_level2_enter, gv, kEwThreads, 0, C().stream, (double *const *)in_slot, (const double *)L1.inv, L.V,
             L.e, N);
    if (p.inner_sstep & 1) {
      // sFGMRES (gmres2.hpp:176-180): W(j+1) = A32 M W(j) on the raw vectors
      for (int j = 0; j < L.m; j++) {
        float *zj = L.Z + (size_t)j * ldn;
        if (p.m3 > 0) F3R_TRY(level3(Vp[j], zj, nullptr));
        else F3R_TRY(rich_apply(Vp[j], zj, nullptr, nullptr));
        F3R_TRY(launch_sell(C(), A.v32, A.view(), (const float *)zj, EpiStore<float>{Vp[j + 1], nullptr}));
      }
      F3R_TRY(sstep_orthogonalise(L, Vp, V));
    } else {
      for (int j = 0; j < L.m; j++) {
        float *zj = L.Z + (size_t)j * ldn;
        float *w = Vp[j + 1];
        if (p.m3 > 0) F3R_TRY(level3(Vp[j], zj, j == 0 ? nullptr : L.inv));
        else F3R_TRY(rich_apply(Vp[j], zj, nullptr, j == 0 ? nullptr : L.inv));  // depth 2: R directly
        F3R_TRY(spmv_dots(A.v32, zj, w, V, j + 1, L.H + (size_t)j * (L.m + 1)));
        GivensCtl<float> g{L.H, L.cs, L.sn, L.e, L.y, L.inv, nullptr, L.m + 1, j, j == L.m - 1, C().err};
        launch_k(C(), k_cgs_update<float, 8>, gv, 256, 0, C().stream, w, V, j + 1, N, C().gred(), g);
      }
    }
    launch_k(C(), k_zy<float, double, false>, gv, kEwThreads, 0, C().stream, Zc, L.y, L.m, nullptr, out_slot, N);
    CUDA_TRY(cudaGetLastError());
    return F3R_SUCCESS;
  }

  // One call into level 2 for outer column j, replayed from a CUDA graph
  // keyed by which Richardson calls inside it update their weights.
  Status level2_call(double *in, double *out) {
    // the graph reads its input and output columns from two device slots,
    // set stream-ordered by a one-thread kernel (no host staging copy)
    launch_k(C(), k_set_slots, 1, 1, 0, C().stream, in_slot, out_slot, in, out);
    // the legacy / per-thread default streams cannot be captured
    const cudaStream_t cs = C().stream;
    if (!p.use_graphs || cs == 0 || cs == cudaStreamLegacy || cs == cudaStreamPerThread) return level2();
    const int calls = p.m2 * std::max(p.m3, 1);
    std::vector<bool> key(calls);
    for (int i = 0; i < calls; i++) key[i] = ((cnt + 1 + i) % p.c) == 0;
    auto it = graphs.find(key);
    if (it == graphs.end()) {
      const int64_t cnt0 = cnt, rc0 = r_calls, l0 = C().launches;
      cudaGraph_t graph = nullptr;
      CUDA_TRY(cudaStreamBeginCapture(C().stream, cudaStreamCaptureModeThreadLocal));
      Status s = level2();
      cudaError_t ce = cudaStreamEndCapture(C().stream, &graph);
      if (s != F3R_SUCCESS) {
        if (graph) cudaGraphDestroy(graph);
        return s;
      }
      if (ce != cudaSuccess) return fail(F3R_ERROR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
      cudaGraphExec_t exec = nullptr;
      ce = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return fail(F3R_ERROR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
      it = graphs.emplace(key, std::make_pair(exec, C().launches - l0)).first;
      cnt = cnt0;  // capture advanced the counters without running anything
      r_calls = rc0;
      C().launches = l0;
    }
    CUDA_TRY(cudaGraphLaunch(it->second.first, C().stream));
    C().launches += it->second.second;
    cnt += calls;
    r_calls += calls;
    return F3R_SUCCESS;
  }

  // |e| and the device error word come back together, one synchronisation per outer step
  Status read_abs_e(double *v) {
    int *e_h = reinterpret_cast<int *>(C().pinned + 7);
    CUDA_TRY(cudaMemcpyAsync(C().pinned, abs_e, sizeof(double), cudaMemcpyDeviceToHost, C().stream));
    CUDA_TRY(cudaMemcpyAsync(e_h, C().err, sizeof(int), cudaMemcpyDeviceToHost, C().stream));
    CUDA_TRY(cudaStreamSynchronize(C().stream));
    if (*e_h != DEV_OK) return C().check_device_error();  // maps the word to a status and clears it
    *v = C().pinned[0];
    return F3R_SUCCESS;
  }

  // ---- level 1 inside Restarted (gmres.hpp:85-134, restart.hpp:26-36) -------
  Status solve(const double *b_user, double *x_user, f3r_cond_fn cond, void *user, f3r_result *res) {
    const int64_t N = n;
    cudaStream_t st = C().stream;
    const int g = C().ew_grid(N);
    auto is_dev = [&](const void *q) {
      cudaPointerAttributes a{};
      if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
      return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
    };
    const bool b_dev = is_dev(b_user), x_dev = is_dev(x_user);
    // x is updated with 16-byte vector accesses: a device x that is not
    // 16-byte aligned is worked on in an internal copy
    const bool x_direct = x_dev && (reinterpret_cast<uintptr_t>(x_user) % 16 == 0);
    const double *b = b_user;
    double *x = x_user;
    if (!b_dev) {
      CUDA_TRY(cudaMemcpyAsync(b_d, b_user, sizeof(double) * N, cudaMemcpyHostToDevice, st));
      b = b_d;
    }
    if (!x_direct) {
      CUDA_TRY(cudaMemcpyAsync(x_d, x_user, sizeof(double) * N, x_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                               st));
      x = x_d;
    }
    CUDA_TRY(cudaEventRecord(ev0, st));
    const int64_t launches0 = C().launches;
    // permuted system (SELL-C-sigma order)
    const double *bs = b;
    double *xs = x;
    if (perm_d) {
      launch_k(C(), k_permute_gather, g, kEwThreads, 0, st, b, perm_d, bp_d, N);
      launch_k(C(), k_permute_gather, g, kEwThreads, 0, st, x, perm_d, xp_d, N);
      bs = bp_d;
      xs = xp_d;
    }
    // per-solve Richardson state (f3r-gpu.cpp:277-281)
    cnt = p.c;
    r_calls = 0;
    {
      RichState h{};
      for (int k = 0; k < kMaxM4; k++) {
        h.sum[k] = 1.0f;
        // F3R-Static: the fixed weight in the reference's fp16 scalar (static.cpp:99-100)
        h.ome[k] = __float2half(p.static_weight > 0 ? (float)p.static_weight : 1.0f);
        h.om[k] = 0.0f;
      }
      h.den = 1;
      CUDA_TRY(cudaMemcpyAsync(rs, &h, sizeof(h), cudaMemcpyHostToDevice, st));
      CUDA_TRY(cudaStreamSynchronize(st));
    }
    // ||b|| for the relative stop test
    double nb = 0;
    launch_k(C(), k_dot<double, double, 8>, g, 256, 0, st, bs, bs, N, C().gred(), C().dscratch);
    CUDA_TRY(cudaMemcpyAsync(C().pinned, C().dscratch, sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    nb = std::sqrt(C().pinned[0]);
    auto stop = [&](int i, double e) -> bool {
      if (cond) return cond(i, e, user) != 0;
      return nb > 0 ? (e / nb < p.rel_tol) : (e == 0);
    };

    Level<double> &L = L1;
    Cols<double> V{}, Zc{};
    const int gv = C().ew_grid(cdiv(N, 2));
    for (int k = 0; k <= L.m; k++) V.p[k] = L.V + (size_t)k * ldn;
    for (int k = 0; k < L.m; k++) Zc.p[k] = L.Z + (size_t)k * ldn;
    f3r_result out{};
    int restarts = 0;
    double last_e = 0;
    bool solved = false;
    while (!solved && restarts < p.max_restarts) {
      restarts++;
      // r = b - A x with ||r|| fused (gmres.hpp:87, 100)
      F3R_TRY(launch_sell(C(), A.v64, A.view(), (const double *)xs,
                          EpiResidualNorm{bs, L.V, C().gred(), L.e, L.inv, abs_e}));
      double h0;
      F3R_TRY(read_abs_e(&h0));
      last_e = h0;
      if (stop(0, h0)) {
        solved = true;
        break;
      }
      // V(0) = r / ||r|| happens inside the level-2 entry kernel (in place)
      int j = 0;
      bool conv = false;
      for (; j < L.m; j++) {
        double *zj = L.Z + (size_t)j * ldn;
        double *w = L.V + (size_t)(j + 1) * ldn;
        F3R_TRY(level2_call(L.V + (size_t)j * ldn, zj));
        F3R_TRY(launch_sell(C(), A.v64, A.view(), (const double *)zj, EpiStore<double>{w, nullptr}));
        launch_k(C(), k_multidot_chunked<double, 8>, g, 256, 0, st, w, V, j + 1, N, C().gred(), L.H + (size_t)j * (L.m + 1));
        GivensCtl<double> gc{L.H, L.cs, L.sn, L.e, L.y, L.inv, abs_e, L.m + 1, j, 0, C().err};
        launch_k(C(), k_cgs_update<double, 8>, gv, 256, 0, st, w, V, j + 1, N, C().gred(), gc);
        CUDA_TRY(cudaGetLastError());
        double ej;
        F3R_TRY(read_abs_e(&ej));
        last_e = ej;
        out.res_iter++;
        if (stop(j + 1, ej)) {
          j++;
          conv = true;
          break;
        }
        // w = V(j+1) is normalised by the next step's level-2 entry kernel
      }
      launch_k(C(), k_trsv_y<double>, 1, 32, 0, st, L.H, L.e, L.y, L.m + 1, j);
      launch_k(C(), k_zy<double, double, true>, gv, kEwThreads, 0, st, Zc, L.y, j, xs, nullptr, N);
      CUDA_TRY(cudaGetLastError());
      if (conv) solved = true;
    }
    if (perm_d) launch_k(C(), k_permute_scatter, g, kEwThreads, 0, st, xs, perm_d, x, N);
    CUDA_TRY(cudaEventRecord(ev1, st));
    out.kernel_launches = C().launches - launches0;
    // explicit residual ||b - A x|| / ||b|| in fp64 (outside the timed region,
    // as the drivers, f3r-gpu.cpp:99-102)
    F3R_TRY(launch_sell(C(), A.v64, A.view(), (const double *)xs, EpiResidual<double, double>{bs, r_d, nullptr}));
    launch_k(C(), k_dot<double, double, 8>, g, 256, 0, st, r_d, r_d, N, C().gred(), C().dscratch);
    CUDA_TRY(cudaMemcpyAsync(C().pinned, C().dscratch, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (!x_direct)
      CUDA_TRY(cudaMemcpyAsync(x_user, x, sizeof(double) * N, x_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                               st));
    CUDA_TRY(cudaStreamSynchronize(st));
    F3R_TRY(C().check_device_error());
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, ev0, ev1));
    out.is_solved = solved ? 1 : 0;
    out.res_nrm2 = last_e;
    out.impl_rel_res = nb > 0 ? last_e / nb : last_e;
    out.expl_rel_res = nb > 0 ? std::sqrt(C().pinned[0]) / nb : std::sqrt(C().pinned[0]);
    out.restarts = restarts;
    out.inner_applications = r_calls;
    out.solve_seconds = ms * 1e-3;
    if (res) *res = out;
    return F3R_SUCCESS;
  }
};

// Layout autotuner (f3r_params.sell_autotune): the fp16 copy of A is built in
// every candidate layout and its fp16 x fp32 product timed on the context's
// stream (2 warm-up launches, best of 3 runs of 5, CUDA events); p takes the
// fastest layout.  Candidates that cannot be built (padding beyond 2^31
// entries) are skipped.
static Status autotune_layout(f3r_context *ctx, const f3r_csr *a, f3r_params &p) {
  struct Cand {
    int32_t format, sigma, align, index16;
  };
  const Cand cands[] = {{F3R_FORMAT_SELL, 1, 1, 0},   {F3R_FORMAT_SELL, 1, 0, 0}, {F3R_FORMAT_SELL, 1, 0, 1},
                        {F3R_FORMAT_SELL, 256, 0, 0}, {F3R_FORMAT_SELL, 256, 1, 0}, {F3R_FORMAT_CSR, 1, 0, 0}};
  Context &c = *ctx;
  const int32_t n = a->nrows;
  float *xy = nullptr;
  F3R_TRY(c.alloc((void **)&xy, sizeof(float) * 2 * (size_t)std::max(n, 1)));
  CUDA_TRY(cudaMemsetAsync(xy, 0, sizeof(float) * 2 * (size_t)std::max(n, 1), c.stream));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 0;
  int besti = -1;
  Status st = F3R_SUCCESS;
  for (int i = 0; i < (int)(sizeof(cands) / sizeof(cands[0])) && st == F3R_SUCCESS; i++) {
    const Cand &k = cands[i];
    DeviceSell d;
    if (k.format == F3R_FORMAT_CSR) {
      st = upload_csr(c, *a, 1 << F3R_F16, d);
    } else {
      SellHost h;
      st = build_sell(*a, k.sigma, true, h);
      if (st != F3R_SUCCESS) break;
      if (k.align) {
        if (align_offsets(*a, true, h) < 0) continue;  // too large padded: not a candidate
      } else if (k.index16) {
        compress_index16(h);
      }
      st = upload_sell(c, h, 1 << F3R_F16, false, d);
    }
    float ms = 0;
    if (st == F3R_SUCCESS) {
      const DevSell v = d.view();
      float run_best = 0;
      for (int w = 0; w < 2 && st == F3R_SUCCESS; w++)
        st = launch_sell(c, d.v16, v, (const float *)xy, EpiStore<float>{xy + n, nullptr});
      for (int r = 0; r < 3 && st == F3R_SUCCESS; r++) {
        cudaEventRecord(e0, c.stream);
        for (int w = 0; w < 5 && st == F3R_SUCCESS; w++)
          st = launch_sell(c, d.v16, v, (const float *)xy, EpiStore<float>{xy + n, nullptr});
        cudaEventRecord(e1, c.stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) st = fail(F3R_ERROR_CUDA, "autotune timing failed");
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        if (r == 0 || t < run_best) run_best = t;
      }
      ms = run_best;
    }
    cudaStreamSynchronize(c.stream);
    d.release();
    if (st == F3R_SUCCESS && (besti < 0 || ms < best)) {
      best = ms;
      besti = i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(xy);
  F3R_TRY(st);
  F3R_TRY(c.check_device_error());
  if (besti < 0) return fail(F3R_ERROR_UNSUPPORTED, "no candidate layout could be built");
  p.format = cands[besti].format;
  p.sell_sigma = cands[besti].sigma;
  p.sell_align = cands[besti].align;
  p.sell_index16 = cands[besti].index16;
  return F3R_SUCCESS;
}

// zf / wf: given SDAINV factors (both or neither; precond SDAINV only)
static Status make_solver(f3r_context *ctx, const f3r_csr *a, const f3r_params *pp, Solver **out,
                          const f3r_csr *zf = nullptr, const f3r_csr *wf = nullptr) {
  F3R_TRY(check_csr(a));
  if (a->nrows != a->ncols) return fail(F3R_ERROR_INVALID_VALUE, "the system matrix must be square");
  if ((zf != nullptr) != (wf != nullptr)) return fail(F3R_ERROR_INVALID_VALUE, "give both factors or neither");
  if (zf) {
    if (pp->precond != F3R_PRECOND_SDAINV)
      return fail(F3R_ERROR_INVALID_VALUE, "given factors need precond F3R_PRECOND_SDAINV");
    F3R_TRY(check_csr(zf));
    F3R_TRY(check_csr(wf));
    if (zf->nrows != a->nrows || zf->ncols != a->nrows || wf->nrows != a->nrows || wf->ncols != a->nrows)
      return fail(F3R_ERROR_INVALID_VALUE, "the factors must be square and of the matrix's size");
  }
  f3r_params p = *pp;
  if (p.m_outer < 1 || p.m_outer + 1 > kMaxCols || p.m2 < 1 || p.m2 + 1 > kMaxCols || p.m3 < 0 ||
      p.m3 + 1 > kMaxCols || p.m4 < 1 || p.m4 > kMaxM4 || p.c < 1 || p.max_restarts < 1 || p.static_weight < 0)
    return fail(F3R_ERROR_INVALID_VALUE,
                "need 1 <= m_outer, m2 <= 127, 0 <= m3 <= 127, 1 <= m4 <= 16, c >= 1, max_restarts >= 1, "
                "static_weight >= 0");
  if (p.sell_c != 32) return fail(F3R_ERROR_UNSUPPORTED, "only SELL slice height 32 is implemented");
  if (p.format != F3R_FORMAT_SELL && p.format != F3R_FORMAT_CSR) return fail(F3R_ERROR_INVALID_VALUE, "unknown format");
  if (p.format == F3R_FORMAT_CSR && (p.sell_sigma != 1 || p.sell_align || p.sell_index16))
    return fail(F3R_ERROR_INVALID_VALUE, "format CSR takes no SELL options (sigma 1, no alignment, 32-bit indices)");
  if (p.precond < F3R_PRECOND_SDAINV || p.precond > F3R_PRECOND_ILU0_LEVEL)
    return fail(F3R_ERROR_INVALID_VALUE, "unknown preconditioner");
  if (p.half_scale_log2 < 0 || p.half_scale_log2 > 20) return fail(F3R_ERROR_INVALID_VALUE, "half_scale_log2 in [0, 20]");
  if (p.inner_sstep < 0 || p.inner_sstep > 3) return fail(F3R_ERROR_INVALID_VALUE, "inner_sstep is a 2-bit mask");
  if (p.sell_autotune) {
    CUDA_TRY(cudaSetDevice(ctx->device));
    F3R_TRY(autotune_layout(ctx, a, p));
  }
  auto s = std::make_unique<Solver>();
  s->ctx = ctx;
  s->p = p;
  s->n = a->nrows;
  s->ldn = ((int64_t)a->nrows + 7) / 8 * 8;
  const int32_t n = a->nrows;
  CUDA_TRY(cudaSetDevice(ctx->device));
  // system matrix in SELL-C-sigma order with all three value copies
  const bool csr = p.format == F3R_FORMAT_CSR;
  const int all_types = (1 << F3R_F64) | (1 << F3R_F32) | (1 << F3R_F16);
  std::vector<int32_t> hperm;
  if (csr) {
    hperm.resize(n);
    for (int32_t i = 0; i < n; i++) hperm[i] = i;
    F3R_TRY(upload_csr(*ctx, *a, all_types, s->A));
  } else {
    SellHost h;
    F3R_TRY(build_sell(*a, p.sell_sigma, true, h));
    hperm = h.perm;
    if (p.sell_align) {
      if (align_offsets(*a, true, h) < 0) return fail(F3R_ERROR_UNSUPPORTED, "padded matrix exceeds 2^31 entries");
    } else if (p.sell_index16) {
      compress_index16(h);
    }
    F3R_TRY(upload_sell(*ctx, h, all_types, false, s->A));
  }  // the host copy (up to several GB) is released here
  s->perm = hperm;
  if (p.sell_sigma > 1) {
    F3R_TRY(s->alloc(&s->perm_d, (size_t)std::max(n, 1)));
    CUDA_TRY(cudaMemcpy(s->perm_d, hperm.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice));
  }
  // the preconditioner, in the permuted order as well
  HostCSR Ah(n, n, a->nnz);
  std::memcpy(Ah.rptr.data(), a->rptr, sizeof(int32_t) * (n + 1));
  std::memcpy(Ah.idx.data(), a->idx, sizeof(int32_t) * a->nnz);
  std::memcpy(Ah.val.data(), a->val, sizeof(double) * a->nnz);
  if (p.precond == F3R_PRECOND_SDAINV) {
    HostCSR *zr = nullptr, *wr = nullptr;
    if (zf) {
      auto copy = [](const f3r_csr &m) {
        HostCSR *h = new HostCSR(m.nrows, m.ncols, m.nnz);
        std::memcpy(h->rptr.data(), m.rptr, sizeof(int32_t) * (m.nrows + 1));
        std::memcpy(h->idx.data(), m.idx, sizeof(int32_t) * m.nnz);
        std::memcpy(h->val.data(), m.val, sizeof(double) * m.nnz);
        return h;
      };
      zr = copy(*zf);
      wr = copy(*wf);
    } else {
      F3R_TRY(sdainv(Ah, p.sdainv_tol, p.acc, &zr, &wr));
    }
    std::unique_ptr<HostCSR> Zh(zr), Wh(wr);
    bool diag = true;
    for (int32_t i = 0; i < n && diag; i++) {
      diag &= (Zh->rptr[i + 1] - Zh->rptr[i] == 1 && Zh->idx[Zh->rptr[i]] == i);
      diag &= (Wh->rptr[i + 1] - Wh->rptr[i] == 1 && Wh->idx[Wh->rptr[i]] == i);
    }
    if (diag) {
      s->precond_diag = 1;
      std::vector<double> wdv(n), zdv(n);
      for (int32_t i = 0; i < n; i++) {
        wdv[i] = Wh->val[Wh->rptr[hperm[i]]];
        zdv[i] = Zh->val[Zh->rptr[hperm[i]]];
      }
      double *tmp = nullptr;
      F3R_TRY(ctx->alloc((void **)&tmp, sizeof(double) * std::max(n, 1)));
      F3R_TRY(s->alloc(&s->wd, (size_t)std::max(n, 1)));
      F3R_TRY(s->alloc(&s->zd, (size_t)std::max(n, 1)));
      CUDA_TRY(cudaMemcpy(tmp, wdv.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
      launch_k(*ctx, k_convert_vals<__half>, ctx->ew_grid(n), kEwThreads, 0, ctx->stream, tmp, s->wd, n);
      CUDA_TRY(cudaStreamSynchronize(ctx->stream));
      CUDA_TRY(cudaMemcpy(tmp, zdv.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
      launch_k(*ctx, k_convert_vals<__half>, ctx->ew_grid(n), kEwThreads, 0, ctx->stream, tmp, s->zd, n);
      CUDA_TRY(cudaStreamSynchronize(ctx->stream));
      cudaFree(tmp);
    } else {
      // W^T and Z as SELL matrices of the permuted system (same sigma order), or CSR
      SellHost hw, hz;
      f3r_csr wv = Wh->view(), zv = Zh->view();
      if (csr) {
        F3R_TRY(upload_csr(*ctx, wv, 1 << F3R_F16, s->W));
        F3R_TRY(upload_csr(*ctx, zv, 1 << F3R_F16, s->Z));
      } else {
      F3R_TRY(build_sell(wv, p.sell_sigma, true, hw, &hperm));
      F3R_TRY(build_sell(zv, p.sell_sigma, true, hz, &hperm));
      if (p.sell_align) {
        if (align_offsets(wv, true, hw) < 0 || align_offsets(zv, true, hz) < 0)
          return fail(F3R_ERROR_UNSUPPORTED, "padded matrix exceeds 2^31 entries");
      } else if (p.sell_index16) {
        compress_index16(hw);
        compress_index16(hz);
      }
      F3R_TRY(upload_sell(*ctx, hw, 1 << F3R_F16, false, s->W));
      F3R_TRY(upload_sell(*ctx, hz, 1 << F3R_F16, false, s->Z));
      }
    }
  } else {
    HostCSR *lr = nullptr, *ur = nullptr;
    std::vector<int32_t> bptr;
    const bool global = p.precond == F3R_PRECOND_ILU0_LEVEL;
    F3R_TRY(ilu0_bj(Ah, global ? 1 : p.ilu_blocks, p.acc, &lr, &ur, &bptr));
    std::unique_ptr<HostCSR> Lh(lr), Uh(ur);
    if (p.precond == F3R_PRECOND_ILU0_BJ) {
      F3R_TRY(s->ilu.build(ctx->stream, *Lh, *Uh, hperm, p.sell_sigma > 1, bptr));
    } else if (global) {
      F3R_TRY(s->ilul.build(ctx->sm_count, *Lh, *Uh, hperm, p.sell_sigma > 1));
    } else {
      const int kind = p.precond == F3R_PRECOND_ILU0_BAJ ? TRSV_BAJ : TRSV_JACOBI;
      F3R_TRY(jacobi_trsv_prepare(*ctx));
      F3R_TRY(s->jl.build(*ctx, *Lh, FORM_LOWER, kind, p.trsv_iters, p.trsv_omega, p.sell_sigma > 1 ? &hperm : nullptr));
      F3R_TRY(s->ju.build(*ctx, *Uh, FORM_D_UPPER, kind, p.trsv_iters, p.trsv_omega,
                          p.sell_sigma > 1 ? &hperm : nullptr));
    }
  }
  // level storage
  F3R_TRY(s->make_level(s->L1, p.m_outer, true));
  F3R_TRY(s->make_level(s->L2, p.m2, true));
  if (p.m3 > 0) F3R_TRY(s->make_level(s->L3, p.m3, false));
  const size_t nn = (size_t)std::max(n, 1);
  F3R_TRY(s->alloc(&s->abs_e, 1));
  F3R_TRY(s->alloc(&s->hin, nn));
  F3R_TRY(s->alloc(&s->hout, nn));
  F3R_TRY(s->alloc(&s->hout2, nn));
  F3R_TRY(s->alloc(&s->tmp, nn));
  F3R_TRY(s->alloc(&s->tmp2, nn));
  F3R_TRY(s->alloc(&s->hr, nn));
  CUDA_TRY(cudaMemset(s->tmp2, 0, nn * sizeof(__half)));
  F3R_TRY(s->alloc(&s->rs, 1));
  F3R_TRY(s->alloc(&s->in_slot, 1));
  F3R_TRY(s->alloc(&s->out_slot, 1));
  F3R_TRY(s->alloc(&s->b_d, nn));
  F3R_TRY(s->alloc(&s->x_d, nn));
  F3R_TRY(s->alloc(&s->r_d, nn));
  if (s->perm_d) {
    F3R_TRY(s->alloc(&s->bp_d, nn));
    F3R_TRY(s->alloc(&s->xp_d, nn));
  }
  CUDA_TRY(cudaEventCreate(&s->ev0));
  CUDA_TRY(cudaEventCreate(&s->ev1));
  // every SpMV instantiation the solve may launch, configured before capture
  Context &cx = *ctx;
  F3R_TRY((sell_attr<double, double, EpiResidualNorm>(cx)));
  F3R_TRY((sell_attr<double, double, EpiStore<double>>(cx)));
  F3R_TRY((sell_attr<double, double, EpiResidual<double, double>>(cx)));
  F3R_TRY((sell_attr<float, float, EpiStoreDots<4>>(cx)));
  F3R_TRY((sell_attr<float, float, EpiStoreDots<8>>(cx)));
  F3R_TRY((sell_attr<float, float, EpiStoreDots<kMaxDots>>(cx)));
  F3R_TRY((sell_attr<__half, float, EpiStoreDots<4>>(cx)));
  F3R_TRY((sell_attr<__half, float, EpiStoreDots<8>>(cx)));
  F3R_TRY((sell_attr<__half, float, EpiStoreDots<kMaxDots>>(cx)));
  F3R_TRY((sell_attr<__half, __half, EpiRichStep>(cx)));
  F3R_TRY((sell_attr<__half, __half, EpiRichWeight>(cx)));
  F3R_TRY((sell_attr<__half, __half, EpiRichResPre>(cx)));
  F3R_TRY((sell_attr<__half, __half, EpiResidual<__half, __half>>(cx)));
  F3R_TRY((sell_attr<__half, __half, EpiStore<__half>>(cx)));
  F3R_TRY((sell_attr<__half, float, EpiStore<float>>(cx)));
  F3R_TRY((sell_attr<float, float, EpiStore<float>>(cx)));
  F3R_TRY((sell_attr<__half, __half, EpiZScale>(cx)));
  CUDA_TRY(cudaDeviceSynchronize());
  *out = s.release();
  return F3R_SUCCESS;
}

}  // namespace f3r

struct f3r_solver {
  f3r::Solver *s = nullptr;
};

namespace f3r {
const void *solver_context(const f3r_solver *s) { return s && s->s ? (const void *)s->s->ctx : nullptr; }
int32_t solver_rows(const f3r_solver *s) { return s && s->s ? s->s->n : 0; }
}  // namespace f3r

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char *f3r_last_error_string(void) { return f3r::g_err.c_str(); }

const char *f3r_status_string(f3r_status s) {
  switch (s) {
  case F3R_SUCCESS: return "success";
  case F3R_ERROR_INVALID_VALUE: return "invalid value";
  case F3R_ERROR_CUDA: return "CUDA error";
  case F3R_ERROR_OUT_OF_MEMORY: return "out of memory";
  case F3R_ERROR_BREAKDOWN: return "breakdown";
  case F3R_ERROR_TIMEOUT: return "device wait timed out";
  case F3R_ERROR_UNSUPPORTED: return "unsupported";
  case F3R_ERROR_NO_DEVICE: return "no CUDA device";
  }
  return "unknown status";
}

// ---- host matrices ----------------------------------------------------------
f3r_status f3r_host_matrix_from_csr(const f3r_csr *a, f3r_host_matrix **out) {
  if (!out) return fail(F3R_ERROR_INVALID_VALUE, "out is null");
  F3R_TRY(check_csr(a));
  auto *h = new f3r_host_matrix;
  h->m.reset(new HostCSR(a->nrows, a->ncols, a->nnz));
  std::memcpy(h->m->rptr.data(), a->rptr, sizeof(int32_t) * (a->nrows + 1));
  if (a->nnz) {
    std::memcpy(h->m->idx.data(), a->idx, sizeof(int32_t) * a->nnz);
    std::memcpy(h->m->val.data(), a->val, sizeof(double) * a->nnz);
  }
  *out = h;
  return F3R_SUCCESS;
}
f3r_status f3r_host_matrix_view(const f3r_host_matrix *m, f3r_csr *view) {
  if (!m || !view) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  *view = m->m->view();
  return F3R_SUCCESS;
}
void f3r_host_matrix_destroy(f3r_host_matrix *m) { delete m; }

f3r_status f3r_problem_stencil27(int32_t nx, int32_t ny, int32_t nz, int32_t variant, double beta,
                                 f3r_host_matrix **out) {
  if (!out || nx < 1 || ny < 1 || nz < 1 || variant < 0 || variant > 2)
    return fail(F3R_ERROR_INVALID_VALUE, "stencil27: grid sizes >= 1, variant in 0..2");
  if ((int64_t)nx * ny * nz * 27 > INT32_MAX) return fail(F3R_ERROR_UNSUPPORTED, "stencil27: nnz exceeds int32");
  auto *h = new f3r_host_matrix;
  h->m.reset(stencil27(nx, ny, nz, variant, beta));
  *out = h;
  return F3R_SUCCESS;
}
f3r_status f3r_problem_diffusion7(int32_t nx, int32_t ny, int32_t nz, double sigma, double corr_len, uint64_t seed,
                                  f3r_host_matrix **out) {
  if (!out || nx < 1 || ny < 1 || nz < 1 || sigma < 0 || corr_len < 0)
    return fail(F3R_ERROR_INVALID_VALUE, "diffusion7: grid sizes >= 1, sigma and corr_len >= 0");
  if ((int64_t)nx * ny * nz * 7 > INT32_MAX) return fail(F3R_ERROR_UNSUPPORTED, "diffusion7: nnz exceeds int32");
  auto *h = new f3r_host_matrix;
  h->m.reset(diffusion7(nx, ny, nz, sigma, corr_len, seed));
  *out = h;
  return F3R_SUCCESS;
}
f3r_status f3r_host_scaling(f3r_host_matrix *m) {
  if (!m) return fail(F3R_ERROR_INVALID_VALUE, "null matrix");
  scaling(*m->m);
  return F3R_SUCCESS;
}
f3r_status f3r_host_spmv(const f3r_csr *a, const double *x, double *y) {
  F3R_TRY(check_csr(a));
  if (!x || !y) return fail(F3R_ERROR_INVALID_VALUE, "null vector");
  host_spmv(*a, x, y);
  return F3R_SUCCESS;
}
f3r_status f3r_random_uniform(uint64_t seed, double lo, double hi, int64_t n, double *out) {
  if (!out || n < 0) return fail(F3R_ERROR_INVALID_VALUE, "bad output");
  std::mt19937_64 eng(seed);
  std::uniform_real_distribution<double> d(lo, hi);
  for (int64_t i = 0; i < n; i++) out[i] = d(eng);
  return F3R_SUCCESS;
}
f3r_status f3r_host_sdainv(const f3r_csr *a, double tol, double acc, f3r_host_matrix **z, f3r_host_matrix **wt) {
  F3R_TRY(check_csr(a));
  if (!z || !wt) return fail(F3R_ERROR_INVALID_VALUE, "null output");
  HostCSR A(a->nrows, a->ncols, a->nnz);
  std::memcpy(A.rptr.data(), a->rptr, sizeof(int32_t) * (a->nrows + 1));
  std::memcpy(A.idx.data(), a->idx, sizeof(int32_t) * a->nnz);
  std::memcpy(A.val.data(), a->val, sizeof(double) * a->nnz);
  HostCSR *zr = nullptr, *wr = nullptr;
  F3R_TRY(sdainv(A, tol, acc, &zr, &wr));
  *z = new f3r_host_matrix;
  (*z)->m.reset(zr);
  *wt = new f3r_host_matrix;
  (*wt)->m.reset(wr);
  return F3R_SUCCESS;
}
f3r_status f3r_host_ilu0_bj(const f3r_csr *a, int32_t blocks, double acc, f3r_host_matrix **l, f3r_host_matrix **u) {
  F3R_TRY(check_csr(a));
  if (!l || !u) return fail(F3R_ERROR_INVALID_VALUE, "null output");
  HostCSR A(a->nrows, a->ncols, a->nnz);
  std::memcpy(A.rptr.data(), a->rptr, sizeof(int32_t) * (a->nrows + 1));
  std::memcpy(A.idx.data(), a->idx, sizeof(int32_t) * a->nnz);
  std::memcpy(A.val.data(), a->val, sizeof(double) * a->nnz);
  HostCSR *lr = nullptr, *ur = nullptr;
  F3R_TRY(ilu0_bj(A, blocks, acc, &lr, &ur, nullptr));
  *l = new f3r_host_matrix;
  (*l)->m.reset(lr);
  *u = new f3r_host_matrix;
  (*u)->m.reset(ur);
  return F3R_SUCCESS;
}

// ---- context ----------------------------------------------------------------
f3r_status f3r_context_create(int32_t device, f3r_context **out) {
  if (!out) return fail(F3R_ERROR_INVALID_VALUE, "out is null");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(F3R_ERROR_NO_DEVICE, "no CUDA device is visible");
  }
  if (device < 0 || device >= count) return fail(F3R_ERROR_INVALID_VALUE, "device ordinal out of range");
  CUDA_TRY(cudaSetDevice(device));
  int major = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  if (major != 10) return fail(F3R_ERROR_UNSUPPORTED, "this library is built for sm_100a (B200) only");
  auto c = std::make_unique<f3r_context>();
  c->device = device;
  CUDA_TRY(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
  // a blocking stream: ordered with the legacy default stream, so device
  // buffers written there (e.g. by torch) are complete when our kernels run
  CUDA_TRY(cudaStreamCreate(&c->own));
  c->stream = c->own;
  F3R_TRY(c->alloc((void **)&c->err, sizeof(int)));
  // one partial sum per block and dot: at most 8 blocks per SM (ew_grid) and
  // kMaxCols dots (the outer multi-dot), in fp64
  F3R_TRY(c->alloc(&c->partials, (size_t)c->sm_count * 8 * kMaxCols * sizeof(double)));
  F3R_TRY(c->alloc((void **)&c->ticket, sizeof(unsigned int) * 4));
  F3R_TRY(c->alloc((void **)&c->dscratch, sizeof(double) * 4));
  CUDA_TRY(cudaMemset(c->err, 0, sizeof(int)));
  CUDA_TRY(cudaMemset(c->ticket, 0, sizeof(unsigned int) * 4));
  CUDA_TRY(cudaHostAlloc((void **)&c->pinned, sizeof(double) * 8, cudaHostAllocDefault));
  *out = c.release();
  return F3R_SUCCESS;
}
void f3r_context_destroy(f3r_context *ctx) {
  if (!ctx) return;
  // while the CUDA runtime shuts down (process exit) nothing can be released
  // any more: the object is left to the exit
  if (cudaSetDevice(ctx->device) != cudaSuccess) return;
  cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->err);
  cudaFree(ctx->partials);
  cudaFree(ctx->ticket);
  cudaFree(ctx->dscratch);
  cudaFreeHost(ctx->pinned);
  if (ctx->own) cudaStreamDestroy(ctx->own);
  delete ctx;
}
f3r_status f3r_context_set_stream(f3r_context *ctx, void *stream) {
  if (!ctx) return fail(F3R_ERROR_INVALID_VALUE, "null context");
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own;
  return F3R_SUCCESS;
}
f3r_status f3r_context_synchronize(f3r_context *ctx) {
  if (!ctx) return fail(F3R_ERROR_INVALID_VALUE, "null context");
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return ctx->check_device_error();
}

// ---- SELL -------------------------------------------------------------------
f3r_status f3r_sell_create(f3r_context *ctx, const f3r_csr *a, int32_t slice_height, int32_t sigma,
                           int32_t dtype_mask, f3r_sell **out) {
  if (!ctx || !out) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  if (slice_height != 32) return fail(F3R_ERROR_UNSUPPORTED, "only slice height 32 is implemented");
  if ((dtype_mask & 7) == 0 || (dtype_mask & ~(7 | F3R_SELL_INDEX16 | F3R_SELL_ALIGNED | F3R_SELL_CSR)))
    return fail(F3R_ERROR_INVALID_VALUE,
                "dtype_mask must select f64/f32/f16 (plus F3R_SELL_INDEX16, F3R_SELL_ALIGNED or F3R_SELL_CSR)");
  F3R_TRY(check_csr(a));
  CUDA_TRY(cudaSetDevice(ctx->device));
  if (dtype_mask & F3R_SELL_CSR) {
    if (sigma != 1 || (dtype_mask & (F3R_SELL_INDEX16 | F3R_SELL_ALIGNED)))
      return fail(F3R_ERROR_INVALID_VALUE, "F3R_SELL_CSR takes sigma 1 and no other layout flag");
    auto m = std::make_unique<f3r_sell>();
    m->ctx = ctx;
    Status s = upload_csr(*ctx, *a, dtype_mask & 7, m->d);
    if (s != F3R_SUCCESS) {
      m->d.release();
      return s;
    }
    *out = m.release();
    return F3R_SUCCESS;
  }
  SellHost h;
  F3R_TRY(build_sell(*a, sigma, false, h));
  if (dtype_mask & F3R_SELL_ALIGNED) {
    if (align_offsets(*a, false, h) < 0) return fail(F3R_ERROR_UNSUPPORTED, "padded matrix exceeds 2^31 entries");
  } else if (dtype_mask & F3R_SELL_INDEX16) {
    compress_index16(h);
  }
  auto m = std::make_unique<f3r_sell>();
  m->ctx = ctx;
  Status s = upload_sell(*ctx, h, dtype_mask & 7, true, m->d);
  if (s != F3R_SUCCESS) {
    m->d.release();
    return s;
  }
  *out = m.release();
  return F3R_SUCCESS;
}
f3r_status f3r_sell_info_get(const f3r_sell *m, f3r_sell_info *info) {
  if (!m || !info) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  info->nrows = m->d.n;
  info->ncols = m->d.ncols;
  info->nnz = (int32_t)m->d.nnz;
  info->slice_height = m->d.rptr ? 0 : 32;
  info->sigma = m->d.sigma;
  info->nslices = m->d.nslices;
  info->nnz_padded = m->d.nnz_pad;
  info->max_width = m->d.max_width;
  info->dtypes = m->d.dtypes;
  info->index_bits = m->d.index_bits();
  return F3R_SUCCESS;
}
void f3r_sell_destroy(f3r_sell *m) {
  if (!m) return;
  if (cudaSetDevice(m->ctx->device) != cudaSuccess) return;  // runtime shutting down: left to the exit
  cudaStreamSynchronize(m->ctx->stream);
  m->d.release();
  delete m;
}

f3r_status f3r_sell_operate(f3r_sell *m, f3r_dtype val_t, f3r_dtype in_t, const void *in, f3r_dtype out_t, void *out) {
  if (!m || !in || !out) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  Context &c = *m->ctx;
  const DeviceSell &d = m->d;
  if (!(d.dtypes & (1 << val_t))) return fail(F3R_ERROR_INVALID_VALUE, "matrix holds no copy of that value type");
  const DevSell A = d.view();
  if (val_t == F3R_F64 && in_t == F3R_F64 && out_t == F3R_F64)
    return launch_sell(c, d.v64, A, (const double *)in, EpiStore<double>{(double *)out, A.perm});
  if (val_t == F3R_F32 && in_t == F3R_F32 && out_t == F3R_F32)
    return launch_sell(c, d.v32, A, (const float *)in, EpiStore<float>{(float *)out, A.perm});
  if (val_t == F3R_F16 && in_t == F3R_F32 && out_t == F3R_F32)
    return launch_sell(c, d.v16, A, (const float *)in, EpiStore<float>{(float *)out, A.perm});
  if (val_t == F3R_F16 && in_t == F3R_F16 && out_t == F3R_F16)
    return launch_sell(c, d.v16, A, (const __half *)in, EpiStore<__half>{(__half *)out, A.perm});
  if (val_t == F3R_F16 && in_t == F3R_F16 && out_t == F3R_F32)
    return launch_sell(c, d.v16, A, (const __half *)in, EpiStore<float>{(float *)out, A.perm});
  return fail(F3R_ERROR_UNSUPPORTED, "unsupported (val, in, out) type combination");
}

f3r_status f3r_sell_compute_residual(f3r_sell *m, f3r_dtype val_t, f3r_dtype rhs_t, const void *rhs, f3r_dtype in_t,
                                     const void *in, f3r_dtype res_t, void *res) {
  if (!m || !rhs || !in || !res) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  Context &c = *m->ctx;
  const DeviceSell &d = m->d;
  if (!(d.dtypes & (1 << val_t))) return fail(F3R_ERROR_INVALID_VALUE, "matrix holds no copy of that value type");
  const DevSell A = d.view();
  if (val_t == F3R_F64 && rhs_t == F3R_F64 && in_t == F3R_F64 && res_t == F3R_F64)
    return launch_sell(c, d.v64, A, (const double *)in, EpiResidual<double, double>{(const double *)rhs, (double *)res, A.perm});
  if (val_t == F3R_F32 && rhs_t == F3R_F32 && in_t == F3R_F32 && res_t == F3R_F32)
    return launch_sell(c, d.v32, A, (const float *)in, EpiResidual<float, float>{(const float *)rhs, (float *)res, A.perm});
  if (val_t == F3R_F16 && rhs_t == F3R_F16 && in_t == F3R_F16 && res_t == F3R_F16)
    return launch_sell(c, d.v16, A, (const __half *)in, EpiResidual<__half, __half>{(const __half *)rhs, (__half *)res, A.perm});
  return fail(F3R_ERROR_UNSUPPORTED, "unsupported (val, rhs, in, res) type combination");
}

f3r_status f3r_context_wait_probe(f3r_context *ctx, int32_t set, int32_t limit_ms) {
  if (!ctx || limit_ms < 1 || limit_ms > 10000) return fail(F3R_ERROR_INVALID_VALUE, "need 1 <= limit_ms <= 10000");
  Context &c = *ctx;
  CUDA_TRY(cudaSetDevice(c.device));
  const int32_t gen = 7;
  int32_t *flag = reinterpret_cast<int32_t *>(c.dscratch);  // the context's device scalars
  CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int32_t), c.stream));
  if (set) CUDA_TRY(cudaMemcpyAsync(flag, &gen, sizeof(int32_t), cudaMemcpyHostToDevice, c.stream));
  launch_k(c, k_wait_probe, 1, 32, 0, c.stream, (const int32_t *)flag, (unsigned int)gen, c.err,
           (unsigned long long)limit_ms * 1000000ull);
  CUDA_TRY(cudaGetLastError());
  return c.check_device_error();
}

f3r_status f3r_dot(f3r_context *ctx, f3r_dtype t, int64_t n, const void *x, const void *y, double *result) {
  if (!ctx || !result || n < 0 || (n > 0 && (!x || !y))) return fail(F3R_ERROR_INVALID_VALUE, "bad argument");
  Context &c = *ctx;
  const int g = c.ew_grid(n);
  if (t == F3R_F64) {
    launch_k(c, k_dot<double, double, 8>, g, 256, 0, c.stream, (const double *)x, (const double *)y, n, c.gred(), c.dscratch);
  } else if (t == F3R_F32) {
    launch_k(c, k_dot<float, float, 8>, g, 256, 0, c.stream, (const float *)x, (const float *)y, n, c.gred(), (float *)c.dscratch);
  } else {
    launch_k(c, k_dot<__half, float, 8>, g, 256, 0, c.stream, (const __half *)x, (const __half *)y, n, c.gred(), (float *)c.dscratch);
  }
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(c.pinned, c.dscratch, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  CUDA_TRY(cudaStreamSynchronize(c.stream));
  if (t == F3R_F64) *result = c.pinned[0];
  else {
    float f;
    std::memcpy(&f, c.pinned, sizeof(float));
    *result = f;
  }
  return F3R_SUCCESS;
}

// ---- solver -----------------------------------------------------------------
void f3r_params_default(f3r_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->m_outer = 100;
  p->max_restarts = 20;
  p->m2 = 8;
  p->m3 = 4;
  p->m4 = 2;
  p->c = 64;
  p->precond = F3R_PRECOND_SDAINV;
  p->ilu_blocks = 112;
  p->sdainv_tol = 0.1;
  p->acc = 1.0;
  p->sell_c = 32;
  p->sell_sigma = 1;
  p->rel_tol = 1e-8;
  p->half_scale_log2 = 0;
  p->use_graphs = 1;
  p->trsv_iters = 2;
  p->trsv_omega = 1.0;
}

f3r_status f3r_solver_create(f3r_context *ctx, const f3r_csr *a, const f3r_params *p, f3r_solver **out) {
  if (!ctx || !a || !p || !out) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  Solver *s = nullptr;
  F3R_TRY(make_solver(ctx, a, p, &s));
  *out = new f3r_solver{s};
  return F3R_SUCCESS;
}
f3r_status f3r_solver_create_factors(f3r_context *ctx, const f3r_csr *a, const f3r_params *p, const f3r_csr *z,
                                     const f3r_csr *wt, f3r_solver **out) {
  if (!ctx || !a || !p || !z || !wt || !out) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  Solver *s = nullptr;
  F3R_TRY(make_solver(ctx, a, p, &s, z, wt));
  *out = new f3r_solver{s};
  return F3R_SUCCESS;
}
f3r_status f3r_solver_solve(f3r_solver *s, const double *b, double *x, f3r_cond_fn cond, void *user,
                            f3r_result *result) {
  if (!s || !b || !x) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  CUDA_TRY(cudaSetDevice(s->s->ctx->device));
  return s->s->solve(b, x, cond, user, result);
}
f3r_status f3r_solver_info(const f3r_solver *s, f3r_sell_info *a_info, int32_t *precond_diagonal) {
  if (!s) return fail(F3R_ERROR_INVALID_VALUE, "null solver");
  if (a_info) {
    const DeviceSell &d = s->s->A;
    a_info->nrows = d.n;
    a_info->ncols = d.ncols;
    a_info->nnz = (int32_t)d.nnz;
    a_info->slice_height = d.rptr ? 0 : 32;
    a_info->sigma = d.sigma;
    a_info->nslices = d.nslices;
    a_info->nnz_padded = d.nnz_pad;
    a_info->max_width = d.max_width;
    a_info->dtypes = d.dtypes;
    a_info->index_bits = d.index_bits();
  }
  if (precond_diagonal) *precond_diagonal = s->s->precond_diag;
  return F3R_SUCCESS;
}
f3r_status f3r_solver_operate(f3r_solver *s, f3r_dtype val_t, f3r_dtype in_t, const void *in, f3r_dtype out_t,
                              void *out) {
  if (!s || !in || !out) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  Context &c = *s->s->ctx;
  const DeviceSell &d = s->s->A;
  const DevSell A = d.view();
  if (val_t == F3R_F64 && in_t == F3R_F64 && out_t == F3R_F64)
    return launch_sell(c, d.v64, A, (const double *)in, EpiStore<double>{(double *)out, nullptr});
  if (val_t == F3R_F32 && in_t == F3R_F32 && out_t == F3R_F32)
    return launch_sell(c, d.v32, A, (const float *)in, EpiStore<float>{(float *)out, nullptr});
  if (val_t == F3R_F16 && in_t == F3R_F32 && out_t == F3R_F32)
    return launch_sell(c, d.v16, A, (const float *)in, EpiStore<float>{(float *)out, nullptr});
  if (val_t == F3R_F16 && in_t == F3R_F16 && out_t == F3R_F16)
    return launch_sell(c, d.v16, A, (const __half *)in, EpiStore<__half>{(__half *)out, nullptr});
  if (val_t == F3R_F16 && in_t == F3R_F16 && out_t == F3R_F32)
    return launch_sell(c, d.v16, A, (const __half *)in, EpiStore<float>{(float *)out, nullptr});
  return fail(F3R_ERROR_UNSUPPORTED, "unsupported (val, in, out) type combination");
}

void f3r_solver_destroy(f3r_solver *s) {
  if (!s) return;
  if (cudaSetDevice(s->s->ctx->device) != cudaSuccess) return;  // runtime shutting down: left to the exit
  cudaStreamSynchronize(s->s->ctx->stream);
  delete s->s;
  delete s;
}

}  // extern "C"
