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
#include <type_traits>
#include <vector>

#include "internal.hpp"
#include "kernels.cuh"
#include "block.cuh"
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

bool align64(const f3r_csr &a, SellHost &s) {
  const int32_t n = a.nrows, nc = a.ncols, ns = (int32_t)cdiv(n, 64);
  std::vector<std::vector<int32_t>> D(ns);
  std::vector<char> in_range(ns, 1);
  // a slice's slots are the union D of its rows' offsets; the layout is taken
  // when the slots of all slices together are at most 5/4 of the packed
  // widths (slices that straddle a plane of a small grid gain a few), and no
  // slice more than doubles its packed width
  int64_t not_ok = 0, slots = 0, packed = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : not_ok, slots, packed)
  for (int32_t sl = 0; sl < ns; sl++) {
    std::vector<int32_t> d;
    int32_t wstd = 0;
    for (int32_t q = 0; q < 64; q++) {
      const int64_t r = (int64_t)sl * 64 + q;
      if (r >= n) break;
      wstd = std::max(wstd, a.rptr[r + 1] - a.rptr[r]);
      for (int32_t e = a.rptr[r]; e < a.rptr[r + 1]; e++) d.push_back(a.idx[e] - (int32_t)r);
    }
    std::sort(d.begin(), d.end());
    d.erase(std::unique(d.begin(), d.end()), d.end());
    if (d.empty() || (int64_t)d.size() > 2 * (int64_t)wstd) {
      not_ok++;
      continue;
    }
    slots += (int64_t)d.size();
    packed += wstd;
    in_range[sl] = (int64_t)sl * 64 + d.front() >= 0 && (int64_t)sl * 64 + d.back() + 63 < nc;
    D[sl] = std::move(d);
  }
  if (not_ok || slots * 4 > packed * 5) return false;
  std::vector<int32_t> sptr(ns + 1, 0), cbptr(ns + 1, 0), width(ns);
  for (int32_t sl = 0; sl < ns; sl++) {
    width[sl] = ((int32_t)D[sl].size() + 3) & ~3;
    if ((int64_t)sptr[sl] + width[sl] > INT32_MAX / 64) return false;
    sptr[sl + 1] = sptr[sl] + width[sl];
    cbptr[sl + 1] = cbptr[sl] + width[sl];
  }
  const int64_t np = (int64_t)sptr[ns] * 64;
  std::vector<double> val(np, 0.0);
  std::vector<int32_t> cbase((size_t)cbptr[ns] + 4, 0);
#pragma omp parallel for schedule(dynamic, 256)
  for (int32_t sl = 0; sl < ns; sl++) {
    const std::vector<int32_t> &d = D[sl];
    const int32_t wp = width[sl];
    const int64_t nb = (int64_t)sptr[sl] * 64;
    for (int32_t k = 0; k < wp; k++) cbase[cbptr[sl] + k] = sl * 64 + d[std::min<size_t>(k, d.size() - 1)];
    for (int32_t q = 0; q < 64; q++) {
      const int64_t r = (int64_t)sl * 64 + q;
      if (r >= n) break;
      for (int32_t e = a.rptr[r]; e < a.rptr[r + 1]; e++) {
        const int32_t k = (int32_t)(std::lower_bound(d.begin(), d.end(), a.idx[e] - (int32_t)r) - d.begin());
        const int32_t k0 = k / kAllAlignedChunk * kAllAlignedChunk, kw = std::min(kAllAlignedChunk, wp - k0);
        val[nb + (int64_t)k0 * 64 + (int64_t)q * kw + (k - k0)] = a.val[e];
      }
    }
  }
  for (int32_t sl = 0; sl < ns; sl++)
    if (!in_range[sl]) cbptr[sl] |= 1;
  int32_t mw = 0;
  for (int32_t sl = 0; sl < ns; sl++) mw = std::max(mw, width[sl]);
  s.n = n;
  s.ncols = nc;
  s.sigma = 1;
  s.nnz = a.nnz;
  s.nslices = ns;
  s.perm.resize(n);
  std::iota(s.perm.begin(), s.perm.end(), 0);
  s.sptr = std::move(sptr);
  s.val = std::move(val);
  s.col.clear();
  s.cbase = std::move(cbase);
  s.cbptr = std::move(cbptr);
  s.xoff.clear();
  s.dcol.clear();
  s.aligned_all = true;
  s.nnz_pad = np;
  s.max_width = mw;
  s.height = 64;
  return true;
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
  d.height = h.height;
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

// Back substitution of the columns in mask (Blas1::trsv, gmres.hpp:41-53),
// one thread per column.
template <typename T, int K> __global__ void k_trsv_yK(LevelK<T> L, uint32_t mask, int w) {
  const int c = threadIdx.x;
  if (blockIdx.x != 0 || c >= K || !((mask >> c) & 1u)) return;
  back_subst(L.H + c * L.hs, L.e + c * L.vs, L.y + c * L.vs, L.ldh, w);
}

// One FGMRES level over K columns: bases (inner levels: one allocation of
// m (+1) columns of ldn * K values, column 0 of level 3 an alias of the
// caller's column) and per-column scalars, column c's at LevelK offsets.
template <typename T> struct Level {
  int m = 0;
  T *V = nullptr, *Z = nullptr;
  T *H = nullptr, *cs = nullptr, *sn = nullptr, *e = nullptr, *y = nullptr, *inv = nullptr;
  LevelK<T> view() const { return LevelK<T>{H, cs, sn, e, y, inv, (int64_t)(m + 1) * m, m + 1, m + 1}; }
};

// The fp16-vector FGMRES level (single column): fp16 bases, fp32 Hessenberg and rotations.
struct HLevel {
  int m = 0;
  __half *V = nullptr, *Z = nullptr;  // column-major n x (m+1), n x m
  float *H = nullptr, *cs = nullptr, *sn = nullptr, *e = nullptr, *y = nullptr, *inv = nullptr;
};

struct Solver;

// Device state of solves K columns wide: the levels' bases and scalars, R's
// fp16 work vectors, K Richardson states, the right-hand side / solution
// blocks, the reduction scratch and the captured level graphs.
template <int K> struct Work {
  Level<double> L1;  // outer bases in V1 / Z1 (allocated as the solve reaches them), scalars here
  Level<float> L2, L3;
  HLevel LH;         // K == 1 only
  std::vector<double *> V1, Z1;
  double *abs_e = nullptr;
  __half *hin = nullptr, *hout = nullptr, *hout2 = nullptr, *tmp = nullptr, *tmp2 = nullptr, *hr = nullptr;
  __half *Z16 = nullptr;  // level 3's Z basis in fp16 (Solver::z16)
  RichState *rs = nullptr;
  double **in_slot = nullptr, **out_slot = nullptr;
  double *b_d = nullptr, *x_d = nullptr, *bp_d = nullptr, *xp_d = nullptr, *r_d = nullptr;
  uint32_t *active = nullptr;
  double *nrm = nullptr;  // K norms read back by the host
  double *stage = nullptr;  // K host columns staged on the device (solve_multi)
  GridRed gr{};
  int64_t cnt = 0, r_calls = 0;
  std::map<std::vector<bool>, std::pair<cudaGraphExec_t, int64_t>> graphs;  // exec, kernels in it
  std::vector<void *> allocs;
  ~Work() {
    for (auto &kv : graphs) cudaGraphExecDestroy(kv.second.first);
    for (void *q : allocs) cudaFree(q);
  }
  template <typename T> Status alloc(T **q, size_t count) {
    cudaError_t e = cudaMalloc((void **)q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess)
      return fail(e == cudaErrorMemoryAllocation ? F3R_ERROR_OUT_OF_MEMORY : F3R_ERROR_CUDA,
                  std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back((void *)*q);
    return F3R_SUCCESS;
  }
  template <typename T>
  Status make_level(Level<T> &L, int m, int64_t ldn, bool own_v0, bool bases = true, bool z_basis = true) {
    L.m = m;
    const size_t nn = (size_t)std::max<int64_t>(ldn, 8) * K;
    if (bases) {
      F3R_TRY(alloc(&L.V, nn * (size_t)(m + (own_v0 ? 1 : 0))));
      if (z_basis) F3R_TRY(alloc(&L.Z, nn * (size_t)m));
    }
    F3R_TRY(alloc(&L.H, (size_t)K * (m + 1) * m));
    F3R_TRY(alloc(&L.cs, (size_t)K * (m + 1)));
    F3R_TRY(alloc(&L.sn, (size_t)K * (m + 1)));
    F3R_TRY(alloc(&L.e, (size_t)K * (m + 1)));
    F3R_TRY(alloc(&L.y, (size_t)K * (m + 1)));
    F3R_TRY(alloc(&L.inv, (size_t)K));
    CUDA_TRY(cudaMemsetAsync(L.H, 0, sizeof(T) * (size_t)K * (m + 1) * m, st));
    CUDA_TRY(cudaMemsetAsync(L.e, 0, sizeof(T) * (size_t)K * (m + 1), st));
    return F3R_SUCCESS;
  }
  // the context's stream: the set-up of a workspace is ordered on it and never
  // touches the legacy default stream, which would invalidate a graph capture
  // that a solve on another context (thread) runs meanwhile
  cudaStream_t st = nullptr;
};

template <int K> struct Engine;

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
  // every fp16 value of wd and zd is exactly 1: the kernels take the constant
  // (DiagPre with null pointers) and the two diagonals are not read
  bool diag_unit = false;
  DiagPre diag() const { return diag_unit ? DiagPre{nullptr, nullptr} : DiagPre{wd, zd}; }
  // set diag_unit from the fp16 values as stored (unless p.diag_load asks to
  // load them always); nn values each
  Status detect_unit_diag(size_t nn) {
    diag_unit = false;
    if (p.diag_load || nn == 0) return F3R_SUCCESS;
    std::vector<uint16_t> hw(nn), hz(nn);
    CUDA_TRY(cudaMemcpy(hw.data(), wd, nn * sizeof(uint16_t), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(hz.data(), zd, nn * sizeof(uint16_t), cudaMemcpyDeviceToHost));
    bool unit = true;
    for (size_t i = 0; i < nn && unit; i++) unit = hw[i] == 0x3C00u && hz[i] == 0x3C00u;
    diag_unit = unit;
    return F3R_SUCCESS;
  }
  DeviceSell W, Z;    // general SDAINV factors (permuted system)
  IluDevice ilu;      // block-Jacobi ILU(0), level scheduled
  IluLevel ilul;      // global ILU(0), level scheduled over the whole GPU
  JacobiTrsv jl, ju;  // the same factors solved by Jacobi / BAJ sweeps
  std::vector<void *> allocs;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // A batch of systems of one pattern (f3r_batch): every column of the block
  // solve is its own system; A, W^T, Z (or wd, zd) hold mm_k values per
  // entry, interleaved.  Solves run the mm_k-column engine only.
  bool mm = false;
  // Level 3 keeps its Z basis in fp16 (single-column solves).  Each z_j is R's
  // result, fp16 values written to fp32 (hout times 1 when R's input is not
  // scaled), so the fp16 copy is exact: the level-3 product and x = Z y see
  // the same values, with half the bytes.
  bool z16 = false;
  int mm_k = 0, mm_count = 0;
  Work<1> w1;  // single-column solves
  std::unique_ptr<Work<2>> w2;
  std::unique_ptr<Work<4>> w4;
  std::unique_ptr<Work<8>> w8;
  std::unique_ptr<Work<16>> w16;

  Context &C() { return *ctx; }
  template <typename T> Status alloc(T **q, size_t count) {
    F3R_TRY(ctx->alloc((void **)q, count * sizeof(T)));
    allocs.push_back((void *)*q);
    return F3R_SUCCESS;
  }
  ~Solver() {
    w2.reset(); w4.reset(); w8.reset(); w16.reset();
    for (void *q : allocs) cudaFree(q);
    A.release(); W.release(); Z.release(); ilu.release(); ilul.release(); jl.release(); ju.release();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
  // R calls per outer step (the product of the inner levels' steps)
  int calls_per_outer() const { return std::max(p.m2, 1) * std::max(p.m3, 1) * std::max(p.half_m, 1); }
  // Can the nest run K columns in lockstep?  The block product covers SDAINV
  // (diagonal, or general factors) with FGMRES levels on SELL with 32-bit or
  // no column indices; other set-ups (ILU, s-step levels, the fp16-vector
  // level, CSR or 16-bit indices) solve column by column.
  bool block_ok() const {
    auto layout_ok = [](const DeviceSell &d) { return !d.rptr && !d.dcol; };
    if (p.precond != F3R_PRECOND_SDAINV || p.inner_sstep || p.half_m > 0 || !layout_ok(A)) return false;
    return precond_diag || (layout_ok(W) && layout_ok(Z));
  }
  template <int K> Status work(Work<K> **out);
  Status solve(const double *b_user, double *x_user, f3r_cond_fn cond, void *user, f3r_result *res);
  Status solve_batch(const double *const *b, double *const *x, f3r_cond_fn cond, void *user, f3r_result *results);
  Status solve_multi(int32_t nrhs, const double *b, int64_t ldb, double *x, int64_t ldx, f3r_cond_fn cond, void *user,
                     f3r_result *results);
};

// K-column block product on the context's stream (packed int32 or fully
// aligned SELL); every instantiation raises its shared-memory limit once per
// device, before any graph capture reaches it (Engine::prepare).
template <typename V, typename X, typename Epi, int K, typename CI>
Status launch_block_one(Context &c, const V *val, const DevSell &A, const X *x, const Epi &epi, bool attr_only) {
  using Cfg = BlockCfg<V, K, CI>;
  auto kern = k_sell_block<V, X, Epi, K, Cfg::WARPS, Cfg::STAGES, Cfg::KC, CI>;
  static int done[64] = {0};
  if (!done[c.device & 63]) {
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)block_smem_bytes<V, K, CI>()));
    done[c.device & 63] = 1;
  }
  if (attr_only || A.nslices == 0) return F3R_SUCCESS;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(A.nslices, Cfg::WARPS), c.sm_count));
  launch_k(c, kern, grid, Cfg::WARPS * 32, block_smem_bytes<V, K, CI>(), c.stream, val, A, x, epi, c.err);
  CUDA_TRY(cudaGetLastError());
  return F3R_SUCCESS;
}
// the K-column product on 64-row offset-aligned slices
template <typename V, typename X, typename Epi, int K>
Status launch_block64(Context &c, const V *val, const DevSell &A, const X *x, const Epi &epi, bool attr_only) {
  constexpr int W = block64_warps<V, K>();
  auto kern = k_sell_block64<V, X, Epi, K, W, block64_stages<V, K>()>;
  static int done[64] = {0};
  if (!done[c.device & 63]) {
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)block64_smem_bytes<V, K>()));
    done[c.device & 63] = 1;
  }
  if (attr_only || A.nslices == 0) return F3R_SUCCESS;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(A.nslices, W), c.sm_count));
  launch_k(c, kern, grid, W * 32, block64_smem_bytes<V, K>(), c.stream, val, A, x, epi, c.err);
  CUDA_TRY(cudaGetLastError());
  return F3R_SUCCESS;
}
template <typename V, typename X, typename Epi, int K>
Status launch_block(Context &c, const V *val, const DevSell &A, const X *x, const Epi &epi, bool attr_only = false) {
  if (A.rptr || A.dcol) return fail(F3R_ERROR_UNSUPPORTED, "block product: SELL with 32-bit indices or aligned slices");
  if (A.height == 64) return launch_block64<V, X, Epi, K>(c, val, A, x, epi, attr_only);
  if (attr_only) {
    F3R_TRY((launch_block_one<V, X, Epi, K, int32_t>(c, val, A, x, epi, true)));
    F3R_TRY((launch_block_one<V, X, Epi, K, AlignedIdx>(c, val, A, x, epi, true)));
    return launch_block_one<V, X, Epi, K, AllAlignedIdx>(c, val, A, x, epi, true);
  }
  if (A.xoff) return launch_block_one<V, X, Epi, K, AlignedIdx>(c, val, A, x, epi, false);
  if (A.cbase) return launch_block_one<V, X, Epi, K, AllAlignedIdx>(c, val, A, x, epi, false);
  return launch_block_one<V, X, Epi, K, int32_t>(c, val, A, x, epi, false);
}

// K systems of one pattern, each column with its own values (packed int32 SELL)
template <typename V, typename X, typename Epi, int K>
Status launch_block_mm(Context &c, const V *val, const DevSell &A, const X *x, const Epi &epi, bool attr_only = false) {
  if (A.rptr || A.xoff || A.dcol || A.cbase) return fail(F3R_ERROR_UNSUPPORTED, "batched systems: packed int32 SELL only");
  using Cfg = BlockCfgMM<V, K>;
  auto kern = k_sell_block<V, X, Epi, K, Cfg::WARPS, Cfg::STAGES, Cfg::KC, int32_t, true>;
  static int done[64] = {0};
  if (!done[c.device & 63]) {
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)block_mm_smem_bytes<V, K>()));
    done[c.device & 63] = 1;
  }
  if (attr_only || A.nslices == 0) return F3R_SUCCESS;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(A.nslices, Cfg::WARPS), c.sm_count));
  launch_k(c, kern, grid, Cfg::WARPS * 32, block_mm_smem_bytes<V, K>(), c.stream, val, A, x, epi, c.err);
  CUDA_TRY(cudaGetLastError());
  return F3R_SUCCESS;
}

// The nested solve over K columns in lockstep (K = 1: the single solve).
template <int K> struct Engine {
  Solver &S;
  Work<K> &w;
  const f3r_params &p;
  const int32_t n;
  const int64_t ldn;
  Engine(Solver &s, Work<K> &wk) : S(s), w(wk), p(s.p), n(s.n), ldn(s.ldn) {}
  Context &C() { return *S.ctx; }
  int64_t lk() const { return ldn * K; }  // column stride of a K-wide basis

  // ---- products: the single-column kernel's epilogue (K = 1) or the block one
  template <typename V, typename X, typename E1, typename EK>
  Status mv(const V *vals, const DevSell &M, const X *x, const E1 &e1, const EK &ek) {
    if constexpr (K == 1) return launch_sell(C(), vals, M, x, e1);
    else if (S.mm) return launch_block_mm<V, X, EK, K>(C(), vals, M, x, ek);
    else return launch_block<V, X, EK, K>(C(), vals, M, x, ek);
  }
  template <typename V, typename X, typename Out> Status mv_store(const V *vals, const DevSell &M, const X *x, Out *y) {
    return mv(vals, M, x, EpiStore<Out>{y, nullptr}, EpiStoreK<Out, K>{y});
  }
  // raises the shared-memory limit of every block product instantiation the solve uses
  Status prepare() {
    if constexpr (K > 1) {
      const DevSell Av = S.A.view();
      const double *d = nullptr;
      const float *f = nullptr;
      const __half *h = nullptr;
      F3R_TRY((launch_block<double, double, EpiStoreK<double, K>, K>(C(), d, Av, d, {}, true)));
      F3R_TRY((launch_block<double, double, EpiResidualK<double, double, K>, K>(C(), d, Av, d, {}, true)));
      F3R_TRY((launch_block<float, float, EpiStoreK<float, K>, K>(C(), f, Av, f, {}, true)));
      F3R_TRY((launch_block<__half, float, EpiStoreK<float, K>, K>(C(), h, Av, f, {}, true)));
      F3R_TRY((launch_block<__half, __half, EpiStoreK<float, K>, K>(C(), h, Av, h, {}, true)));
      F3R_TRY((launch_block<__half, __half, EpiStoreK<__half, K>, K>(C(), h, Av, h, {}, true)));
      F3R_TRY((launch_block<__half, __half, EpiRichStepK<K>, K>(C(), h, Av, h, {}, true)));
      F3R_TRY((launch_block<__half, __half, EpiRichResPreK<K>, K>(C(), h, Av, h, {}, true)));
      F3R_TRY((launch_block<__half, __half, EpiResidualK<__half, __half, K>, K>(C(), h, Av, h, {}, true)));
      F3R_TRY((launch_block<__half, __half, EpiZScaleK<K>, K>(C(), h, Av, h, {}, true)));
      // the Gram-Schmidt update's staging tiles (above 48 KB from K = 16)
      CUDA_TRY(cudaFuncSetAttribute(k_cgs_updateK<float, 8, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)cgs_stage_bytes<float, 8, K>()));
      CUDA_TRY(cudaFuncSetAttribute(k_cgs_updateK<double, 8, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)cgs_stage_bytes<double, 8, K>()));
      if (S.mm) {
        F3R_TRY((launch_block_mm<double, double, EpiStoreK<double, K>, K>(C(), d, Av, d, {}, true)));
        F3R_TRY((launch_block_mm<double, double, EpiResidualK<double, double, K>, K>(C(), d, Av, d, {}, true)));
        F3R_TRY((launch_block_mm<float, float, EpiStoreK<float, K>, K>(C(), f, Av, f, {}, true)));
        F3R_TRY((launch_block_mm<__half, float, EpiStoreK<float, K>, K>(C(), h, Av, f, {}, true)));
        F3R_TRY((launch_block_mm<__half, __half, EpiStoreK<float, K>, K>(C(), h, Av, h, {}, true)));
        F3R_TRY((launch_block_mm<__half, __half, EpiStoreK<__half, K>, K>(C(), h, Av, h, {}, true)));
        F3R_TRY((launch_block_mm<__half, __half, EpiRichStepK<K, true>, K>(C(), h, Av, h, {}, true)));
        F3R_TRY((launch_block_mm<__half, __half, EpiRichResPreK<K, true>, K>(C(), h, Av, h, {}, true)));
        F3R_TRY((launch_block_mm<__half, __half, EpiResidualK<__half, __half, K>, K>(C(), h, Av, h, {}, true)));
        F3R_TRY((launch_block_mm<__half, __half, EpiZScaleK<K>, K>(C(), h, Av, h, {}, true)));
      }
    }
    return F3R_SUCCESS;
  }

  // ---- outer basis columns, allocated as the solve reaches them ---------------
  Status ensure_outer(int j) {
    while ((int)w.V1.size() < std::min(j + 2, p.m_outer + 1)) {
      const int add = std::min<int>(8, p.m_outer + 1 - (int)w.V1.size());
      for (int q = 0; q < add; q++) {
        double *v = nullptr;
        F3R_TRY(w.alloc(&v, (size_t)lk()));
        w.V1.push_back(v);
        if ((int)w.Z1.size() < p.m_outer) {
          double *z = nullptr;
          F3R_TRY(w.alloc(&z, (size_t)lk()));
          w.Z1.push_back(z);
        }
      }
    }
    return F3R_SUCCESS;
  }

  // ---- level 4: R(in) -> out --------------------------------------------------
  // in_inv: the K pending 1/h factors of the basis block `in` (its
  // normalisation is done in place by the first kernel), else nullptr.  K = 1
  // below the fp16-vector level: in16 / out16 are that level's fp16 columns.
  Status rich_apply(float *in, float *out, float *e_set, int64_t e_stride, const float *in_inv,
                    __half *in16 = nullptr, __half *out16 = nullptr) {
    const int64_t N = n;
    const int g = C().ew_grid(N);
    cudaStream_t st = C().stream;
    ++w.cnt;
    ++w.r_calls;
    const bool upd = p.static_weight <= 0 && (w.cnt % p.c) == 0;  // F3R-Static never updates
    const bool h16 = in16 != nullptr;
    const float sc = h16 ? 1.0f : std::ldexp(1.0f, p.half_scale_log2);
    const float isc = h16 ? 1.0f : std::ldexp(1.0f, -p.half_scale_log2);
    const __half *hi = h16 ? in16 : w.hin;              // R's fp16 input
    __half *h0 = (p.m4 == 1 && out16) ? out16 : w.hout;  // first result (the only one when m4 = 1)
    float *out_last = out16 ? nullptr : out;            // fp32 result of the last step
    const DevSell Av = S.A.view();
    const GridRed gr = w.gr;
    if (S.precond_diag) {
      if constexpr (K > 1) {
        if (S.mm) {
          F3R_TRY(rich_diag<true>(in, out, e_set, e_stride, in_inv, upd, sc, isc, hi, h0, out_last, out16));
        } else {
          F3R_TRY(rich_diag<false>(in, out, e_set, e_stride, in_inv, upd, sc, isc, hi, h0, out_last, out16));
        }
      } else {
        const DiagPre M = S.diag();
        if (h16) {
          if (!upd)
            launch_k(C(), k_rich_enter_diag<true, __half>, C().ew_grid(cdiv(N, 4)), kEwThreads, 0, st, in16, in_inv,
                     sc, M, w.hin, h0, w.rs, e_set, N);
          else
            launch_k(C(), k_rich_enter_diag<false, __half>, C().ew_grid(cdiv(N, 4)), kEwThreads, 0, st, in16, in_inv,
                     sc, M, w.hin, h0, w.rs, e_set, N);
        } else {
          if (!upd)
            launch_k(C(), k_rich_enter_diagK<true, 1>, g, kEwThreads, 0, st, in, in_inv, sc, M, w.hin, h0, w.rs, e_set,
                     e_stride, N);
          else
            launch_k(C(), k_rich_enter_diagK<false, 1>, g, kEwThreads, 0, st, in, in_inv, sc, M, w.hin, h0, w.rs,
                     e_set, e_stride, N);
        }
        if (!upd) {
          __half *cur = h0, *nxt = w.hout2;
          for (int k = 1; k < p.m4; k++) {
            const bool last = (k == p.m4 - 1);
            __half *hn = last ? out16 : nxt;
            float *fo = last ? out_last : nullptr;
            if (S.diag_unit)
              F3R_TRY(launch_sell(C(), S.A.v16, Av, (const __half *)cur, EpiRichStepUnit{hi, cur, M, w.rs, k, hn, fo, isc}));
            else
              F3R_TRY(launch_sell(C(), S.A.v16, Av, (const __half *)cur, EpiRichStep{hi, cur, M, w.rs, k, hn, fo, isc}));
            std::swap(cur, nxt);
          }
        } else {
          F3R_TRY(mv_store(S.A.v16, Av, (const __half *)h0, w.tmp));
          launch_k(C(), k_rich_weightK<8, K>, g, 256, 0, st, (const __half *)w.tmp, hi, N, gr, w.rs, 0);
          launch_k(C(), k_rich_scale_omK<K>, g, kEwThreads, 0, st, h0, (const RichState *)w.rs, N);
          for (int k = 1; k < p.m4; k++) {
            const bool last = (k == p.m4 - 1);
            F3R_TRY(launch_sell(C(), S.A.v16, Av, (const __half *)w.hout, EpiRichResPre{hi, M, w.hr, w.tmp2}));
            F3R_TRY(mv_store(S.A.v16, Av, (const __half *)w.tmp2, w.tmp));
            launch_k(C(), k_rich_weightK<8, K>, g, 256, 0, st, (const __half *)w.tmp, (const __half *)w.hr, N, gr,
                     w.rs, k);
            F3R_TRY(axpy(k, 0, last ? out_last : nullptr, last ? out16 : nullptr, isc));
          }
        }
      }
    } else {
      // general preconditioner: M = Z W^T (SDAINV) or U^-1 L^-1 (ILU, K = 1)
      if constexpr (K == 1) {
        if (h16) launch_k(C(), k_rich_cast_in<__half>, g, kEwThreads, 0, st, in16, in_inv, sc, w.hin, e_set, N);
      }
      if (!h16) launch_k(C(), k_rich_cast_inK<K>, g, kEwThreads, 0, st, in, in_inv, sc, w.hin, e_set, e_stride, N);
      F3R_TRY(prec_apply(hi, h0, !upd));
      if (upd) {
        F3R_TRY(mv_store(S.A.v16, Av, (const __half *)h0, w.tmp));
        launch_k(C(), k_rich_weightK<8, K>, g, 256, 0, st, (const __half *)w.tmp, hi, N, gr, w.rs, 0);
        launch_k(C(), k_rich_scale_omK<K>, g, kEwThreads, 0, st, h0, (const RichState *)w.rs, N);
      }
      for (int k = 1; k < p.m4; k++) {
        const bool last = (k == p.m4 - 1);
        F3R_TRY(mv(S.A.v16, Av, (const __half *)w.hout, EpiResidual<__half, __half>{hi, w.hr, nullptr},
                   EpiResidualK<__half, __half, K>{hi, w.hr}));
        F3R_TRY(prec_apply(w.hr, w.tmp2, false));
        if (upd) {
          F3R_TRY(mv_store(S.A.v16, Av, (const __half *)w.tmp2, w.tmp));
          launch_k(C(), k_rich_weightK<8, K>, g, 256, 0, st, (const __half *)w.tmp, (const __half *)w.hr, N, gr, w.rs,
                   k);
        }
        F3R_TRY(axpy(k, upd ? 0 : 1, last ? out_last : nullptr, last ? out16 : nullptr, isc));
      }
    }
    if (p.m4 == 1 && !out16) launch_k(C(), k_rich_exitK<K>, g, kEwThreads, 0, st, (const __half *)w.hout, out, isc, N);
    CUDA_TRY(cudaGetLastError());
    return F3R_SUCCESS;
  }

  // R with the diagonal SDAINV fused, K > 1 columns (MMF: one diagonal per
  // column, a batch of systems); the same steps as the single-column path
  template <bool MMF>
  Status rich_diag(float *in, float *out, float *e_set, int64_t e_stride, const float *in_inv, bool upd, float sc,
                   float isc, const __half *hi, __half *h0, float *out_last, __half *out16) {
    const int64_t N = n;
    const int g = C().ew_grid(N);
    cudaStream_t st = C().stream;
    const DiagPre M = S.diag();
    const DevSell Av = S.A.view();
    const GridRed gr = w.gr;
    if (!upd)
      launch_k(C(), k_rich_enter_diagK<true, K, MMF>, g, kEwThreads, 0, st, in, in_inv, sc, M, w.hin, h0, w.rs, e_set,
               e_stride, N);
    else
      launch_k(C(), k_rich_enter_diagK<false, K, MMF>, g, kEwThreads, 0, st, in, in_inv, sc, M, w.hin, h0, w.rs, e_set,
               e_stride, N);
    if (!upd) {
      __half *cur = h0, *nxt = w.hout2;
      for (int k = 1; k < p.m4; k++) {
        const bool last = (k == p.m4 - 1);
        F3R_TRY(mv(S.A.v16, Av, (const __half *)cur, EpiRichStep{hi, cur, M, w.rs, k, nxt, nullptr, isc},
                   EpiRichStepK<K, MMF>{hi, cur, M, w.rs, k, last && out16 ? out16 : nxt, last ? out_last : nullptr,
                                        isc}));
        std::swap(cur, nxt);
      }
    } else {
      F3R_TRY(mv_store(S.A.v16, Av, (const __half *)h0, w.tmp));
      launch_k(C(), k_rich_weightK<8, K>, g, 256, 0, st, (const __half *)w.tmp, hi, N, gr, w.rs, 0);
      launch_k(C(), k_rich_scale_omK<K>, g, kEwThreads, 0, st, h0, (const RichState *)w.rs, N);
      for (int k = 1; k < p.m4; k++) {
        const bool last = (k == p.m4 - 1);
        F3R_TRY(mv(S.A.v16, Av, (const __half *)w.hout, EpiRichResPre{hi, M, w.hr, w.tmp2},
                   EpiRichResPreK<K, MMF>{hi, M, w.hr, w.tmp2}));
        F3R_TRY(mv_store(S.A.v16, Av, (const __half *)w.tmp2, w.tmp));
        launch_k(C(), k_rich_weightK<8, K>, g, 256, 0, st, (const __half *)w.tmp, (const __half *)w.hr, N, gr, w.rs,
                 k);
        F3R_TRY(axpy(k, 0, last ? out_last : nullptr, last ? out16 : nullptr, isc));
      }
    }
    (void)out;
    return F3R_SUCCESS;
  }

  // hout = fp16(hout + om[k] t2), or the last step's result into out / out16
  Status axpy(int k, int use_ome, float *out, __half *out16, float isc) {
    const int g = C().ew_grid(n);
    if constexpr (K == 1) {
      if (out16) {
        launch_k(C(), k_rich_axpy, g, kEwThreads, 0, C().stream, w.hout, (const __half *)w.tmp2,
                 (const RichState *)w.rs, k, use_ome, (float *)nullptr, out16, isc, (int64_t)n);
        return F3R_SUCCESS;
      }
    }
    launch_k(C(), k_rich_axpyK<K>, g, kEwThreads, 0, C().stream, w.hout, (const __half *)w.tmp2,
             (const RichState *)w.rs, k, use_ome, out, isc, (int64_t)n, out16);
    return F3R_SUCCESS;
  }

  // out = M x for the general preconditioners; scale_ome multiplies by ome[0]
  Status prec_apply(const __half *x, __half *out, bool scale_ome) {
    if (p.precond == F3R_PRECOND_SDAINV) {
      F3R_TRY(mv_store(S.W.v16, S.W.view(), x, w.tmp));
      F3R_TRY(mv(S.Z.v16, S.Z.view(), (const __half *)w.tmp, EpiZScale{out, w.rs, scale_ome ? 1 : 0},
                 EpiZScaleK<K>{out, w.rs, scale_ome ? 1 : 0}));
      return F3R_SUCCESS;
    }
    if constexpr (K == 1) {
      if (p.precond == F3R_PRECOND_ILU0_BJ) {
        F3R_TRY(S.ilu.apply(C().stream, x, w.tmp, out, scale_ome ? &w.rs->ome[0] : nullptr));
        C().launches += 2;
      } else if (p.precond == F3R_PRECOND_ILU0_LEVEL) {
        F3R_TRY(S.ilul.apply(C().stream, x, w.tmp, out, scale_ome ? &w.rs->ome[0] : nullptr, C().err));
        C().launches += 2;
      } else {
        F3R_TRY(S.jl.apply(C(), x, w.tmp, nullptr));
        F3R_TRY(S.ju.apply(C(), w.tmp, out, scale_ome ? &w.rs->ome[0] : nullptr));
      }
      return F3R_SUCCESS;
    }
    return fail(F3R_ERROR_UNSUPPORTED, "block solves take SDAINV only");
  }

  // H(j, 0..nv-1) = <w, V(k)> per column, one pass over w and the basis
  void dots(const float *wv, const Cols<float> &Vc, int nv, Level<float> &L, int j) {
    float *hcol = L.H + (size_t)j * (L.m + 1);
    const int64_t hs = (int64_t)(L.m + 1) * L.m;
    if (nv <= 4)
      launch_k(C(), k_multidot_f32K<4, 8, K>, C().ew_grid(cdiv(n, 4)), 256, 0, C().stream, wv, Vc, nv, (int64_t)n,
               w.gr, hcol, hs);
    else if (nv <= 8)
      launch_k(C(), k_multidot_f32K<8, 8, K>, C().ew_grid(cdiv(n, 4)), 256, 0, C().stream, wv, Vc, nv, (int64_t)n,
               w.gr, hcol, hs);
    else
      launch_k(C(), k_multidot_chunkedK<float, 8, K>, C().ew_grid(n), 256, 0, C().stream, wv, Vc, nv, (int64_t)n,
               w.gr, hcol, hs);
  }

  // the Gram-Schmidt update, norm and Givens of step j of an inner level
  void cgs(float *wv, const Cols<float> &Vc, int nv, Level<float> &L, int j, bool last) {
    launch_k(C(), k_cgs_updateK<float, 8, K>, C().ew_grid(cdiv(n, 4)), 256, cgs_stage_bytes<float, 8, K>(),
             C().stream, wv, Vc, nv, (int64_t)n, w.gr, L.view(), j, last ? 1 : 0, (double *)nullptr,
             (const uint32_t *)w.active, C().err);
  }

  // sFGMRES's second and third loops (gmres2.hpp:181-193), K = 1: classical
  // Gram-Schmidt of the stored raw vectors W(1..m) against the basis built so
  // far, with each Givens rotation fused into its step as in FGMRES.  The next
  // step reads V(j+1) through the dots and the update, so it is normalised
  // explicitly here.
  Status sstep_orthogonalise(Level<float> &L, float *const *Vp, const Cols<float> &V) {
    const int64_t N = n;
    for (int j = 0; j < L.m; j++) {
      float *wv = Vp[j + 1];
      dots(wv, V, j + 1, L, j);
      cgs(wv, V, j + 1, L, j, j == L.m - 1);
      if (j + 1 < L.m)
        launch_k(C(), k_scale<float>, C().ew_grid(cdiv(N, 4)), kEwThreads, 0, C().stream, wv, (const float *)L.inv, N);
    }
    CUDA_TRY(cudaGetLastError());
    return F3R_SUCCESS;
  }

  // What an fp32 level calls as its preconditioner: R, or (K = 1) the
  // fp16-vector level when there is one (which then calls R).
  Status inner_apply(float *in, float *out, float *e_set, int64_t e_stride, const float *in_inv,
                     __half *out16 = nullptr) {
    if constexpr (K == 1) {
      if (p.half_m > 0) return levelh(in, in_inv, out, e_set);
    }
    return rich_apply(in, out, e_set, e_stride, in_inv, nullptr, out16);
  }

  // ---- the fp16-vector level (K = 1): FGMRES<_Float16>(A16, R, half_m) ---------
  // (work/src/depth.cpp:122-167).  in32 / out32: the calling fp32 level's
  // columns (in32_inv the pending 1/h of in32, e_parent the caller's e to set
  // on its first call); in32 = nullptr: called by the outer level, input and
  // output through the slots.
  Status levelh(float *in32, const float *in32_inv, float *out32, float *e_parent) {
    if constexpr (K != 1) {
      return fail(F3R_ERROR_UNSUPPORTED, "block solves have no fp16-vector level");
    } else {
      HLevel &L = w.LH;
      const int64_t N = n;
      const int gv = C().ew_grid(cdiv(N, 8));
      cudaStream_t st = C().stream;
      if (in32)
        launch_k(C(), k_level_enter_h<float>, gv, kEwThreads, 0, st, in32, (float *const *)nullptr, in32_inv, L.V,
                 L.e, e_parent, N);
      else
        launch_k(C(), k_level_enter_h<double>, gv, kEwThreads, 0, st, (double *)nullptr, (double *const *)w.in_slot,
                 (const double *)w.L1.inv, L.V, L.e, (float *)nullptr, N);
      Cols<__half> V{}, Zc{};
      for (int k = 0; k <= L.m; k++) V.p[k] = L.V + (size_t)k * ldn;
      for (int k = 0; k < L.m; k++) Zc.p[k] = L.Z + (size_t)k * ldn;
      for (int j = 0; j < L.m; j++) {
        __half *vj = L.V + (size_t)j * ldn, *zj = L.Z + (size_t)j * ldn, *wv = L.V + (size_t)(j + 1) * ldn;
        // R normalises V(j) in place first (its 1/h is pending from step j - 1)
        F3R_TRY(rich_apply(nullptr, nullptr, nullptr, 0, j == 0 ? nullptr : L.inv, vj, zj));
        F3R_TRY(launch_sell(C(), S.A.v16, S.A.view(), (const __half *)zj, EpiStore<__half>{wv, nullptr}));
        launch_k(C(), k_multidot_h<8>, gv, 256, 0, st, (const __half *)wv, V, j + 1, N, w.gr,
                 L.H + (size_t)j * (L.m + 1));
        GivensCtl<float> g{L.H, L.cs, L.sn, L.e, L.y, L.inv, nullptr, L.m + 1, j, j == L.m - 1, C().err};
        launch_k(C(), k_cgs_update_h<8>, gv, 256, 0, st, wv, V, j + 1, N, w.gr, g);
      }
      if (out32)
        launch_k(C(), k_zy_h<float>, gv, kEwThreads, 0, st, Zc, (const float *)L.y, L.m, out32,
                 (float *const *)nullptr, N);
      else
        launch_k(C(), k_zy_h<double>, gv, kEwThreads, 0, st, Zc, (const float *)L.y, L.m, (double *)nullptr,
                 (double *const *)w.out_slot, N);
      CUDA_TRY(cudaGetLastError());
      return F3R_SUCCESS;
    }
  }

  // ---- level 3: FGMRES<float>(A16, R, m3), input a level-2 block column, output
  // a level-2 Z column.  The normalisation V(j+1) *= 1/h of every basis vector
  // is deferred to the first kernel that reads it next (R's entry), which
  // scales it in place; the last basis vector of a level is never read again
  // and is left unscaled.  in_inv: the pending factors of `in` (nullptr if none).
  Status level3(float *in, float *out, const float *in_inv) {
    Level<float> &L = w.L3;
    float *Vp[kMaxCols];
    Cols<float> V{}, Zc{};
    Vp[0] = in;
    for (int k = 1; k <= L.m; k++) Vp[k] = L.V + (size_t)(k - 1) * lk();
    for (int k = 0; k <= L.m; k++) V.p[k] = Vp[k];
    if (L.Z)  // fp32 basis (an fp16 one lives in Work::Z16)
      for (int k = 0; k < L.m; k++) Zc.p[k] = L.Z + (size_t)k * lk();
    const int64_t es = L.m + 1;
    if ((p.inner_sstep & 2) && K == 1) {
      // sFGMRES (gmres2.hpp:176-180): W(j+1) = A16 R W(j) on the raw vectors
      for (int j = 0; j < L.m; j++) {
        float *zj = L.Z + (size_t)j * lk();
        F3R_TRY(inner_apply(Vp[j], zj, j == 0 ? L.e : nullptr, es, j == 0 ? in_inv : nullptr));
        F3R_TRY(mv_store(S.A.v16, S.A.view(), (const float *)zj, Vp[j + 1]));
      }
      F3R_TRY(sstep_orthogonalise(L, Vp, V));
    } else if (S.z16) {
      {
        Cols<__half> Z16{};
        for (int k = 0; k < L.m; k++) Z16.p[k] = w.Z16 + (size_t)k * lk();
        for (int j = 0; j < L.m; j++) {
          __half *zj = w.Z16 + (size_t)j * lk();
          float *wv = Vp[j + 1];
          F3R_TRY(inner_apply(Vp[j], nullptr, j == 0 ? L.e : nullptr, es, j == 0 ? in_inv : L.inv, zj));
          F3R_TRY(mv_store(S.A.v16, S.A.view(), (const __half *)zj, wv));
          dots(wv, V, j + 1, L, j);
          cgs(wv, V, j + 1, L, j, j == L.m - 1);
        }
        launch_k(C(), k_zyK<float, float, false, K, __half>, C().ew_grid(n), kEwThreads, 0, C().stream, Z16,
                 (const float *)L.y, (int64_t)(L.m + 1), L.m, out, (float *const *)nullptr, 0u, (int64_t)n);
        CUDA_TRY(cudaGetLastError());
        return F3R_SUCCESS;
      }
    } else {
      for (int j = 0; j < L.m; j++) {
        float *zj = L.Z + (size_t)j * lk();
        float *wv = Vp[j + 1];
        F3R_TRY(inner_apply(Vp[j], zj, j == 0 ? L.e : nullptr, es, j == 0 ? in_inv : L.inv));
        F3R_TRY(mv_store(S.A.v16, S.A.view(), (const float *)zj, wv));
        dots(wv, V, j + 1, L, j);
        cgs(wv, V, j + 1, L, j, j == L.m - 1);
      }
    }
    launch_k(C(), k_zyK<float, float, false, K>, C().ew_grid(n), kEwThreads, 0, C().stream, Zc, (const float *)L.y,
             (int64_t)(L.m + 1), L.m, out, (float *const *)nullptr, 0u, (int64_t)n);
    CUDA_TRY(cudaGetLastError());
    return F3R_SUCCESS;
  }

  // ---- level 2: FGMRES<float>(A32, L3, m2); in / out through the slots -------
  Status level2() {
    Level<float> &L = w.L2;
    float *Vp[kMaxCols];
    Cols<float> V{}, Zc{};
    for (int k = 0; k <= L.m; k++) V.p[k] = Vp[k] = L.V + (size_t)k * lk();
    for (int k = 0; k < L.m; k++) Zc.p[k] = L.Z + (size_t)k * lk();
    // normalises the outer basis block in place (its 1/h are L1.inv) and casts it
    launch_k(C(), k_level2_enterK<K>, C().ew_grid(n), kEwThreads, 0, C().stream, (double *const *)w.in_slot,
             (const double *)w.L1.inv, L.V, L.e, (int64_t)(L.m + 1), (int64_t)n);
    if ((p.inner_sstep & 1) && K == 1) {
      // sFGMRES (gmres2.hpp:176-180): W(j+1) = A32 M W(j) on the raw vectors
      for (int j = 0; j < L.m; j++) {
        float *zj = L.Z + (size_t)j * lk();
        if (p.m3 > 0) F3R_TRY(level3(Vp[j], zj, nullptr));
        else F3R_TRY(inner_apply(Vp[j], zj, nullptr, 0, nullptr));
        F3R_TRY(mv_store(S.A.v32, S.A.view(), (const float *)zj, Vp[j + 1]));
      }
      F3R_TRY(sstep_orthogonalise(L, Vp, V));
    } else {
      for (int j = 0; j < L.m; j++) {
        float *zj = L.Z + (size_t)j * lk();
        float *wv = Vp[j + 1];
        if (p.m3 > 0) F3R_TRY(level3(Vp[j], zj, j == 0 ? nullptr : L.inv));
        else F3R_TRY(inner_apply(Vp[j], zj, nullptr, 0, j == 0 ? nullptr : L.inv));  // depth 2: R directly
        F3R_TRY(mv_store(S.A.v32, S.A.view(), (const float *)zj, wv));
        dots(wv, V, j + 1, L, j);
        cgs(wv, V, j + 1, L, j, j == L.m - 1);
      }
    }
    launch_k(C(), k_zyK<float, double, false, K>, C().ew_grid(n), kEwThreads, 0, C().stream, Zc, (const float *)L.y,
             (int64_t)(L.m + 1), L.m, (double *)nullptr, (double *const *)w.out_slot, 0u, (int64_t)n);
    CUDA_TRY(cudaGetLastError());
    return F3R_SUCCESS;
  }

  // What the outer level calls for one column: level 2, or (m2 = 0) the
  // fp16-vector level with its input and output through the slots.
  Status outer_inner() { return p.m2 > 0 ? level2() : levelh(nullptr, nullptr, nullptr, nullptr); }

  // One call into level 2 for outer column j, replayed from a CUDA graph
  // keyed by which Richardson calls inside it update their weights.
  Status level2_call(double *in, double *out) {
    // the graph reads its input and output columns from two device slots,
    // set stream-ordered by a one-thread kernel (no host staging copy)
    launch_k(C(), k_set_slots, 1, 1, 0, C().stream, w.in_slot, w.out_slot, in, out);
    // the legacy / per-thread default streams cannot be captured
    const cudaStream_t cs = C().stream;
    if (!p.use_graphs || cs == 0 || cs == cudaStreamLegacy || cs == cudaStreamPerThread) return outer_inner();
    const int calls = S.calls_per_outer();
    std::vector<bool> key(calls);
    for (int i = 0; i < calls; i++) key[i] = ((w.cnt + 1 + i) % p.c) == 0;
    auto it = w.graphs.find(key);
    if (it == w.graphs.end()) {
      const int64_t cnt0 = w.cnt, rc0 = w.r_calls, l0 = C().launches;
      cudaGraph_t graph = nullptr;
      CUDA_TRY(cudaStreamBeginCapture(C().stream, cudaStreamCaptureModeThreadLocal));
      Status s = outer_inner();
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
      it = w.graphs.emplace(key, std::make_pair(exec, C().launches - l0)).first;
      w.cnt = cnt0;  // capture advanced the counters without running anything
      w.r_calls = rc0;
      C().launches = l0;
    }
    CUDA_TRY(cudaGraphLaunch(it->second.first, C().stream));
    C().launches += it->second.second;
    w.cnt += calls;
    w.r_calls += calls;
    return F3R_SUCCESS;
  }

  // the K values of `dev` (|e| of the outer step) and the device error word
  // come back together: one synchronisation per outer step
  Status read_k(const double *dev, double *host) {
    int *e_h = reinterpret_cast<int *>(C().pinned + 7);
    double *pk = C().pinned;  // up to 6 values fit beside the active word and the error word
    CUDA_TRY(cudaMemcpyAsync(e_h, C().err, sizeof(int), cudaMemcpyDeviceToHost, C().stream));
    CUDA_TRY(cudaMemcpyAsync(K <= 6 ? pk : host, dev, sizeof(double) * K, cudaMemcpyDeviceToHost, C().stream));
    CUDA_TRY(cudaStreamSynchronize(C().stream));
    if (*e_h != DEV_OK) return C().check_device_error();  // maps the word to a status and clears it
    if (K <= 6)
      for (int c = 0; c < K; c++) host[c] = pk[c];
    return F3R_SUCCESS;
  }
  Status set_active(uint32_t mask) {
    uint32_t *h = reinterpret_cast<uint32_t *>(C().pinned + 6);
    *h = mask;
    CUDA_TRY(cudaMemcpyAsync(w.active, h, sizeof(uint32_t), cudaMemcpyHostToDevice, C().stream));
    CUDA_TRY(cudaStreamSynchronize(C().stream));  // the pinned word is reused by the next call
    return F3R_SUCCESS;
  }

  // ---- level 1 inside Restarted (gmres.hpp:85-134, restart.hpp:26-36) over K
  // columns in lockstep.  b, x: device blocks of K interleaved columns in the
  // solver's storage order (x holds the initial guesses); ncols <= K columns
  // are real, the others padding (inactive from the start).  cond(i, |e|) is
  // called for every active column after every outer step, in column order.
  Status solve_block(const double *bs, double *xs, int ncols, f3r_cond_fn cond, void *user, f3r_result *res) {
    const int64_t N = n;
    cudaStream_t st = C().stream;
    const int g = C().ew_grid(N);
    CUDA_TRY(cudaEventRecord(S.ev0, st));
    const int64_t launches0 = C().launches;
    // per-solve Richardson state (f3r-gpu.cpp:277-281), one per column
    w.cnt = p.c;
    w.r_calls = 0;
    {
      RichState h[K];
      for (int c = 0; c < K; c++) {
        RichState &q = h[c];
        std::memset(&q, 0, sizeof(q));
        for (int k = 0; k < kMaxM4; k++) {
          q.sum[k] = 1.0f;
          // F3R-Static: the fixed weight in the reference's fp16 scalar (static.cpp:99-100)
          q.ome[k] = __float2half(p.static_weight > 0 ? (float)p.static_weight : 1.0f);
          q.om[k] = 0.0f;
        }
        q.den = 1;
      }
      CUDA_TRY(cudaMemcpyAsync(w.rs, h, sizeof(h), cudaMemcpyHostToDevice, st));
      CUDA_TRY(cudaStreamSynchronize(st));
    }
    uint32_t active = ncols >= 32 ? 0xffffffffu : ((1u << ncols) - 1u);
    F3R_TRY(set_active(active));
    // ||b|| per column for the relative stop test
    double nb[K];
    launch_k(C(), k_dotK<double, double, 8, K>, g, 256, 0, st, bs, bs, N, w.gr, w.nrm);
    F3R_TRY(read_k(w.nrm, nb));
    for (int c = 0; c < K; c++) nb[c] = std::sqrt(nb[c]);
    auto stop = [&](int c, int i, double e) -> bool {
      if (cond) return cond(i, e, user) != 0;
      return nb[c] > 0 ? (e / nb[c] < p.rel_tol) : (e == 0);
    };
    Level<double> &L = w.L1;
    const LevelK<double> Lv = L.view();
    f3r_result out[K];
    std::memset(out, 0, sizeof(out));
    double last_e[K] = {0}, ev[K];
    int restarts = 0;
    while (active && restarts < p.max_restarts) {
      restarts++;
      for (int c = 0; c < K; c++)
        if ((active >> c) & 1u) out[c].restarts = restarts;
      F3R_TRY(ensure_outer(0));
      // r = b - A x and ||r|| per column (gmres.hpp:87, 100)
      F3R_TRY(mv(S.A.v64, S.A.view(), (const double *)xs, EpiResidual<double, double>{bs, w.V1[0], nullptr},
                 EpiResidualK<double, double, K>{bs, w.V1[0]}));
      launch_k(C(), k_resnormK<8, K>, g, 256, 0, st, (const double *)w.V1[0], N, w.gr, Lv, w.abs_e,
               (const uint32_t *)w.active);
      F3R_TRY(read_k(w.abs_e, ev));
      for (int c = 0; c < K; c++) {
        if (!((active >> c) & 1u)) continue;
        last_e[c] = ev[c];
        if (stop(c, 0, ev[c])) {
          out[c].is_solved = 1;
          active &= ~(1u << c);
        }
      }
      if (!active) break;
      F3R_TRY(set_active(active));
      // V(0) = r / ||r|| happens inside the level-2 entry kernel (in place)
      int j = 0;
      uint32_t running = active;  // the columns of this cycle that have not converged
      for (; j < L.m && running; j++) {
        F3R_TRY(ensure_outer(j));
        Cols<double> V{};
        for (int k = 0; k <= j + 1; k++) V.p[k] = w.V1[k];
        double *zj = w.Z1[j], *wv = w.V1[j + 1];
        F3R_TRY(level2_call(w.V1[j], zj));
        F3R_TRY(mv_store(S.A.v64, S.A.view(), (const double *)zj, wv));
        launch_k(C(), k_multidot_chunkedK<double, 8, K>, g, 256, 0, st, (const double *)wv, V, j + 1, N, w.gr,
                 L.H + (size_t)j * (L.m + 1), (int64_t)(L.m + 1) * L.m);
        launch_k(C(), k_cgs_updateK<double, 8, K>, C().ew_grid(cdiv(N, 2)), 256, cgs_stage_bytes<double, 8, K>(), st,
                 wv, V, j + 1, N, w.gr, Lv, j, 0, w.abs_e, (const uint32_t *)w.active, C().err);
        CUDA_TRY(cudaGetLastError());
        F3R_TRY(read_k(w.abs_e, ev));
        uint32_t done = 0;
        for (int c = 0; c < K; c++) {
          if (!((running >> c) & 1u)) continue;
          last_e[c] = ev[c];
          out[c].res_iter++;
          if (stop(c, j + 1, ev[c])) done |= 1u << c;
        }
        if (done) {
          // x += Z y for the columns that converged at this step (gmres.hpp:121-131)
          Cols<double> Zc{};
          for (int k = 0; k <= j; k++) Zc.p[k] = w.Z1[k];
          launch_k(C(), k_trsv_yK<double, K>, 1, 32, 0, st, Lv, done, j + 1);
          launch_k(C(), k_zyK<double, double, true, K>, g, kEwThreads, 0, st, Zc, (const double *)L.y,
                   (int64_t)(L.m + 1), j + 1, xs, (double *const *)nullptr, done, N);
          for (int c = 0; c < K; c++)
            if ((done >> c) & 1u) out[c].is_solved = 1;
          running &= ~done;
          active &= ~done;
          F3R_TRY(set_active(running));
        }
        // w = V(j+1) is normalised by the next step's level-2 entry kernel
      }
      if (running) {
        // the restart length reached: x += Z y over all m columns, then restart
        Cols<double> Zc{};
        for (int k = 0; k < j; k++) Zc.p[k] = w.Z1[k];
        launch_k(C(), k_trsv_yK<double, K>, 1, 32, 0, st, Lv, running, j);
        launch_k(C(), k_zyK<double, double, true, K>, g, kEwThreads, 0, st, Zc, (const double *)L.y,
                 (int64_t)(L.m + 1), j, xs, (double *const *)nullptr, running, N);
        CUDA_TRY(cudaGetLastError());
        F3R_TRY(set_active(active));
      }
    }
    CUDA_TRY(cudaEventRecord(S.ev1, st));
    const int64_t nl = C().launches - launches0;
    // explicit residual ||b - A x|| / ||b|| in fp64 per column (outside the
    // timed region, as the drivers, f3r-gpu.cpp:99-102)
    F3R_TRY(mv(S.A.v64, S.A.view(), (const double *)xs, EpiResidual<double, double>{bs, w.r_d, nullptr},
               EpiResidualK<double, double, K>{bs, w.r_d}));
    double er[K];
    launch_k(C(), k_dotK<double, double, 8, K>, g, 256, 0, st, (const double *)w.r_d, (const double *)w.r_d, N, w.gr,
             w.nrm);
    F3R_TRY(read_k(w.nrm, er));
    F3R_TRY(C().check_device_error());
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
    for (int c = 0; c < ncols; c++) {
      f3r_result &o = out[c];
      o.res_nrm2 = last_e[c];
      o.impl_rel_res = nb[c] > 0 ? last_e[c] / nb[c] : last_e[c];
      o.expl_rel_res = nb[c] > 0 ? std::sqrt(er[c]) / nb[c] : std::sqrt(er[c]);
      o.inner_applications = w.r_calls;
      o.solve_seconds = ms * 1e-3;
      o.kernel_launches = nl;
      if (res) res[c] = o;
    }
    return F3R_SUCCESS;
  }
};

// the workspace of K-column solves, made on first use
template <int K> Status make_work(Solver &s, Work<K> &w) {
  const size_t nn = (size_t)std::max(s.n, 1) * K;
  const f3r_params &p = s.p;
  w.st = s.ctx->stream;
  F3R_TRY(w.make_level(w.L1, p.m_outer, s.ldn, true, false));
  if (p.m2 > 0) F3R_TRY(w.make_level(w.L2, p.m2, s.ldn, true));
  if (p.m3 > 0) F3R_TRY(w.make_level(w.L3, p.m3, s.ldn, false, true, !s.z16));  // fp16 Z: Work::Z16
  if (K == 1 && p.half_m > 0) {
    HLevel &L = w.LH;
    const int m = p.half_m;
    L.m = m;
    const size_t ln = (size_t)std::max<int64_t>(s.ldn, 8);
    F3R_TRY(w.alloc(&L.V, ln * (size_t)(m + 1)));
    F3R_TRY(w.alloc(&L.Z, ln * (size_t)m));
    F3R_TRY(w.alloc(&L.H, (size_t)(m + 1) * m));
    F3R_TRY(w.alloc(&L.cs, (size_t)m));
    F3R_TRY(w.alloc(&L.sn, (size_t)m));
    F3R_TRY(w.alloc(&L.e, (size_t)m + 1));
    F3R_TRY(w.alloc(&L.y, (size_t)m));
    F3R_TRY(w.alloc(&L.inv, 1));
    CUDA_TRY(cudaMemsetAsync(L.H, 0, sizeof(float) * (size_t)(m + 1) * m, w.st));
    CUDA_TRY(cudaMemsetAsync(L.e, 0, sizeof(float) * (size_t)(m + 1), w.st));
  }
  F3R_TRY(w.alloc(&w.abs_e, K));
  F3R_TRY(w.alloc(&w.nrm, K));
  F3R_TRY(w.alloc(&w.hin, nn));
  F3R_TRY(w.alloc(&w.hout, nn));
  F3R_TRY(w.alloc(&w.hout2, nn));
  if (s.z16) F3R_TRY(w.alloc(&w.Z16, (size_t)s.ldn * K * p.m3));
  F3R_TRY(w.alloc(&w.tmp, nn));
  F3R_TRY(w.alloc(&w.tmp2, nn));
  F3R_TRY(w.alloc(&w.hr, nn));
  CUDA_TRY(cudaMemsetAsync(w.tmp2, 0, nn * sizeof(__half), w.st));
  F3R_TRY(w.alloc(&w.rs, K));
  F3R_TRY(w.alloc(&w.in_slot, 1));
  F3R_TRY(w.alloc(&w.out_slot, 1));
  F3R_TRY(w.alloc(&w.b_d, nn));
  F3R_TRY(w.alloc(&w.x_d, nn));
  F3R_TRY(w.alloc(&w.r_d, nn));
  F3R_TRY(w.alloc(&w.active, 1));
  if (K > 1) F3R_TRY(w.alloc(&w.stage, nn));
  if (s.perm_d) {
    F3R_TRY(w.alloc(&w.bp_d, nn));
    F3R_TRY(w.alloc(&w.xp_d, nn));
  }
  // reduction scratch: partial sums of up to 8 blocks per SM, kMaxCols values per column
  double *part = nullptr;
  unsigned int *ticket = nullptr;
  F3R_TRY(w.alloc(&part, (size_t)s.ctx->sm_count * 8 * kMaxCols * K + 64));
  F3R_TRY(w.alloc(&ticket, 4));
  CUDA_TRY(cudaMemsetAsync(ticket, 0, 4 * sizeof(unsigned int), w.st));
  w.gr = GridRed{part, ticket};
  CUDA_TRY(cudaStreamSynchronize(w.st));
  return Engine<K>(s, w).prepare();
}

template <int K> Status Solver::work(Work<K> **out) {
  std::unique_ptr<Work<K>> *slot = nullptr;
  if constexpr (K == 2) slot = &w2;
  if constexpr (K == 4) slot = &w4;
  if constexpr (K == 8) slot = &w8;
  if constexpr (K == 16) slot = &w16;
  if (!*slot) {
    auto wk = std::make_unique<Work<K>>();
    F3R_TRY(make_work<K>(*this, *wk));
    *slot = std::move(wk);
  }
  *out = slot->get();
  return F3R_SUCCESS;
}

// Single solve: b, x host or device vectors of the original row order.
Status Solver::solve(const double *b_user, double *x_user, f3r_cond_fn cond, void *user, f3r_result *res) {
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
  Work<1> &w = w1;
  const double *b = b_user;
  double *x = x_user;
  if (!b_dev) {
    CUDA_TRY(cudaMemcpyAsync(w.b_d, b_user, sizeof(double) * N, cudaMemcpyHostToDevice, st));
    b = w.b_d;
  }
  if (!x_direct) {
    CUDA_TRY(cudaMemcpyAsync(w.x_d, x_user, sizeof(double) * N, x_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                             st));
    x = w.x_d;
  }
  // permuted system (SELL-C-sigma order)
  const double *bs = b;
  double *xs = x;
  if (perm_d) {
    launch_k(C(), k_permute_gather, g, kEwThreads, 0, st, b, perm_d, w.bp_d, N);
    launch_k(C(), k_permute_gather, g, kEwThreads, 0, st, x, perm_d, w.xp_d, N);
    bs = w.bp_d;
    xs = w.xp_d;
  }
  f3r_result out{};
  F3R_TRY(Engine<1>(*this, w).solve_block(bs, xs, 1, cond, user, &out));
  if (perm_d) launch_k(C(), k_permute_scatter, g, kEwThreads, 0, st, (const double *)xs, perm_d, x, N);
  if (!x_direct)
    CUDA_TRY(cudaMemcpyAsync(x_user, x, sizeof(double) * N, x_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                             st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (res) *res = out;
  return F3R_SUCCESS;
}

// Several right-hand sides: blocks of up to 16 columns solved in lockstep
// (the K-column engine, K the power of two at or above the block's width)
// where the nest allows it, otherwise column by column.
Status Solver::solve_multi(int32_t nrhs, const double *b, int64_t ldb, double *x, int64_t ldx, f3r_cond_fn cond,
                           void *user, f3r_result *results) {
  if (nrhs <= 1 || !block_ok()) {
    for (int32_t k = 0; k < nrhs; k++) {
      f3r_result r{};
      F3R_TRY(solve(b + (size_t)k * ldb, x + (size_t)k * ldx, cond, user, &r));
      if (results) results[k] = r;
    }
    return F3R_SUCCESS;
  }
  auto is_dev = [&](const void *q) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
  };
  const bool b_dev = is_dev(b), x_dev = is_dev(x);
  const int64_t N = n;
  cudaStream_t st = C().stream;
  const int g = C().ew_grid(N);
  Status status = F3R_SUCCESS;
  // block width: up to 16 columns, 8 on systems of 2^20 rows or more (on the
  // 192^3 system a 16-column block took 0.482 of 16 single solves' time, an
  // 8-column block 0.451 of 8); a single column left over is solved alone
  const int32_t kmax = N >= (1 << 20) ? 8 : 16;
  for (int32_t k0 = 0, nc = 0; k0 < nrhs && status == F3R_SUCCESS; k0 += nc) {
    nc = std::min<int32_t>(kmax, nrhs - k0);
    if (nc == 1) {
      f3r_result r{};
      status = solve(b + (size_t)k0 * ldb, x + (size_t)k0 * ldx, cond, user, &r);
      if (results) results[k0] = r;
      continue;
    }
    auto run = [&](auto kc) -> Status {
      constexpr int K = decltype(kc)::value;
      Work<K> *wk = nullptr;
      F3R_TRY(work<K>(&wk));
      Work<K> &w = *wk;
      double *stage = w.stage;  // host columns pass through it
      // b, x columns into the interleaved blocks (storage order)
      double *bi = perm_d ? w.bp_d : w.b_d, *xi = perm_d ? w.xp_d : w.x_d;
      const double *bsrc = b + (size_t)k0 * ldb;
      double *xsrc = x + (size_t)k0 * ldx;
      int64_t lb = ldb, lx = ldx;
      if (!b_dev) {
        for (int c = 0; c < nc; c++)
          CUDA_TRY(cudaMemcpyAsync(stage + (size_t)c * N, bsrc + (size_t)c * ldb, sizeof(double) * N,
                                   cudaMemcpyHostToDevice, st));
        bsrc = stage;
        lb = N;
      }
      launch_k(C(), k_interleave, g, kEwThreads, 0, st, bsrc, lb, nc, K, w.b_d, N);
      if (!x_dev) {
        for (int c = 0; c < nc; c++)
          CUDA_TRY(cudaMemcpyAsync(stage + (size_t)c * N, xsrc + (size_t)c * ldx, sizeof(double) * N,
                                   cudaMemcpyHostToDevice, st));
        launch_k(C(), k_interleave, g, kEwThreads, 0, st, (const double *)stage, N, nc, K, w.x_d, N);
      } else {
        launch_k(C(), k_interleave, g, kEwThreads, 0, st, (const double *)xsrc, lx, nc, K, w.x_d, N);
      }
      if (perm_d) {
        launch_k(C(), k_permute_gatherK<K>, g, kEwThreads, 0, st, (const double *)w.b_d, perm_d, bi, N);
        launch_k(C(), k_permute_gatherK<K>, g, kEwThreads, 0, st, (const double *)w.x_d, perm_d, xi, N);
      }
      F3R_TRY(Engine<K>(*this, w).solve_block(bi, xi, nc, cond, user, results ? results + k0 : nullptr));
      if (perm_d) launch_k(C(), k_permute_scatterK<K>, g, kEwThreads, 0, st, (const double *)xi, perm_d, w.x_d, N);
      if (x_dev) {
        launch_k(C(), k_deinterleave, g, kEwThreads, 0, st, (const double *)w.x_d, K, nc, xsrc, ldx, N);
      } else {
        launch_k(C(), k_deinterleave, g, kEwThreads, 0, st, (const double *)w.x_d, K, nc, stage, N, N);
        for (int c = 0; c < nc; c++)
          CUDA_TRY(cudaMemcpyAsync(xsrc + (size_t)c * ldx, stage + (size_t)c * N, sizeof(double) * N,
                                   cudaMemcpyDeviceToHost, st));
      }
      CUDA_TRY(cudaStreamSynchronize(st));
      return F3R_SUCCESS;
    };
    if (nc <= 2) status = run(std::integral_constant<int, 2>());
    else if (nc <= 4) status = run(std::integral_constant<int, 4>());
    else if (nc <= 8) status = run(std::integral_constant<int, 8>());
    else status = run(std::integral_constant<int, 16>());
  }
  return status;
}

// Layout autotuner (f3r_params.sell_autotune): the fp16 copy of A is built in
// every candidate layout and its fp16 x fp32 product timed on the context's
// stream (2 warm-up launches, best of 3 runs of 5, CUDA events); p takes the
// fastest layout.  Candidates that cannot be built (padding beyond 2^31
// entries) are skipped.
static Status autotune_layout(f3r_context *ctx, const f3r_csr *a, f3r_params &p) {
  struct Cand {
    int32_t format, sigma, align, index16, height;
  };
  const Cand cands[] = {{F3R_FORMAT_SELL, 1, 1, 0, 32},   {F3R_FORMAT_SELL, 1, 0, 0, 32},
                        {F3R_FORMAT_SELL, 1, 0, 1, 32},   {F3R_FORMAT_SELL, 256, 0, 0, 32},
                        {F3R_FORMAT_SELL, 256, 1, 0, 32}, {F3R_FORMAT_CSR, 1, 0, 0, 32},
                        {F3R_FORMAT_SELL, 1, 1, 0, 64}};
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
      if (k.height == 64) {
        if (!align64(*a, h)) continue;  // rows do not share offsets: not a candidate
      } else if (k.align) {
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
  p.sell_c = cands[besti].height;
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
  if (p.m_outer < 1 || p.m_outer + 1 > kMaxCols || p.m2 < 0 || p.m2 + 1 > kMaxCols || p.m3 < 0 ||
      p.m3 + 1 > kMaxCols || p.half_m < 0 || p.half_m + 1 > kMaxCols || p.m4 < 1 || p.m4 > kMaxM4 || p.c < 1 ||
      p.max_restarts < 1 || p.static_weight < 0)
    return fail(F3R_ERROR_INVALID_VALUE,
                "need 1 <= m_outer <= 127, 0 <= m2, m3, half_m <= 127, 1 <= m4 <= 16, c >= 1, max_restarts >= 1, "
                "static_weight >= 0");
  if (p.m2 == 0 && (p.half_m == 0 || p.m3 > 0 || (p.inner_sstep & 3)))
    return fail(F3R_ERROR_INVALID_VALUE,
                "m2 = 0 (no fp32 level) needs half_m > 0, m3 = 0 and no s-step inner level");
  if (p.sell_c != 32 && p.sell_c != 64) return fail(F3R_ERROR_UNSUPPORTED, "SELL slice height 32 or 64");
  if (p.sell_c == 64 && (p.sell_sigma != 1 || p.format != F3R_FORMAT_SELL || p.sell_index16))
    return fail(F3R_ERROR_INVALID_VALUE, "64-row slices: SELL, sigma 1, offset-aligned (no 16-bit indices)");
  if (p.format != F3R_FORMAT_SELL && p.format != F3R_FORMAT_CSR) return fail(F3R_ERROR_INVALID_VALUE, "unknown format");
  if (p.format == F3R_FORMAT_CSR && (p.sell_sigma != 1 || p.sell_align || p.sell_index16))
    return fail(F3R_ERROR_INVALID_VALUE, "format CSR takes no SELL options (sigma 1, no alignment, 32-bit indices)");
  if (p.precond < F3R_PRECOND_SDAINV || p.precond > F3R_PRECOND_ILU0_LEVEL)
    return fail(F3R_ERROR_INVALID_VALUE, "unknown preconditioner");
  if (p.half_scale_log2 < 0 || p.half_scale_log2 > 20) return fail(F3R_ERROR_INVALID_VALUE, "half_scale_log2 in [0, 20]");
  if (p.inner_sstep < 0 || p.inner_sstep > 3) return fail(F3R_ERROR_INVALID_VALUE, "inner_sstep is a 2-bit mask");
  if (p.diag_load != 0 && p.diag_load != 1) return fail(F3R_ERROR_INVALID_VALUE, "diag_load is 0 or 1");
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
    if (p.sell_c == 64) {
      if (!align64(*a, h))
        return fail(F3R_ERROR_UNSUPPORTED, "64-row slices need every 64 rows to share their column offsets");
    } else if (p.sell_align) {
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
      F3R_TRY(s->detect_unit_diag((size_t)n));
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
  CUDA_TRY(cudaEventCreate(&s->ev0));
  CUDA_TRY(cudaEventCreate(&s->ev1));
  // every SpMV instantiation the single solve may launch, configured before capture
  Context &cx = *ctx;
  F3R_TRY((sell_attr<double, double, EpiStore<double>>(cx)));
  F3R_TRY((sell_attr<double, double, EpiResidual<double, double>>(cx)));
  F3R_TRY((sell_attr<__half, __half, EpiRichStep>(cx)));
  F3R_TRY((sell_attr<__half, __half, EpiRichStepUnit>(cx)));
  F3R_TRY((sell_attr<__half, __half, EpiRichResPre>(cx)));
  F3R_TRY((sell_attr<__half, __half, EpiResidual<__half, __half>>(cx)));
  F3R_TRY((sell_attr<__half, __half, EpiStore<__half>>(cx)));
  F3R_TRY((sell_attr<__half, float, EpiStore<float>>(cx)));
  F3R_TRY((sell_attr<__half, __half, EpiStore<float>>(cx)));
  F3R_TRY((sell_attr<float, float, EpiStore<float>>(cx)));
  F3R_TRY((sell_attr<__half, __half, EpiZScale>(cx)));
  // the single-column workspace (wider ones are made by the first solve_multi that needs them)
  s->z16 = p.m3 > 0 && p.half_scale_log2 == 0 && !(p.inner_sstep & 2) && p.half_m == 0;
  F3R_TRY(make_work<1>(*s, s->w1));
  CUDA_TRY(cudaDeviceSynchronize());
  *out = s.release();
  return F3R_SUCCESS;
}

// ---------------------------------------------------------------------------
// Batches of systems of one pattern (f3r_batch_*)
// ---------------------------------------------------------------------------

// SELL position of every CSR entry of a (rows in the storage order of h, the
// packed layout build_sell makes: entry c of storage row r at
// (sptr[r / 32] + c) * 32 + r % 32)
static std::vector<int64_t> sell_positions(const f3r_csr &a, const SellHost &h) {
  std::vector<int64_t> pos((size_t)a.nnz);
#pragma omp parallel for schedule(static)
  for (int32_t r = 0; r < h.n; r++) {
    const int32_t o = h.perm[r];
    const int64_t base = (int64_t)h.sptr[r / 32] * 32 + (r % 32);
    for (int32_t q = a.rptr[o], c = 0; q < a.rptr[o + 1]; q++, c++) pos[q] = base + (int64_t)c * 32;
  }
  return pos;
}

// The packed SELL of `pattern` (rows in the order perm) holding K systems'
// values interleaved, vals[c] on the pattern's entries (count <= K systems;
// the remaining columns hold zeros), with the value copies of dtype_mask.
static Status upload_sell_mm(Context &c, const f3r_csr &pattern, const std::vector<int32_t> &perm,
                             const std::vector<const double *> &vals, int K, int dtype_mask, DeviceSell &d) {
  SellHost h;
  F3R_TRY(build_sell(pattern, 1, true, h, &perm));
  const std::vector<int64_t> pos = sell_positions(pattern, h);
  const size_t np = (size_t)h.nnz_pad;
  std::vector<double> v(np * K, 0.0);
  for (size_t s = 0; s < vals.size(); s++)
#pragma omp parallel for schedule(static)
    for (int32_t q = 0; q < pattern.nnz; q++) v[(size_t)pos[q] * K + s] = vals[s][q];
  d.n = h.n; d.ncols = h.ncols; d.nslices = h.nslices; d.max_width = h.max_width; d.sigma = 1;
  d.nnz = h.nnz; d.nnz_pad = h.nnz_pad; d.dtypes = dtype_mask;
  F3R_TRY(c.alloc((void **)&d.col, np * 4));
  F3R_TRY(c.alloc((void **)&d.sptr, (size_t)(h.nslices + 1) * 4));
  CUDA_TRY(cudaMemcpyAsync(d.col, h.col.data(), np * 4, cudaMemcpyHostToDevice, c.stream));
  CUDA_TRY(cudaMemcpyAsync(d.sptr, h.sptr.data(), (size_t)(h.nslices + 1) * 4, cudaMemcpyHostToDevice, c.stream));
  double *tmp64 = nullptr;
  F3R_TRY(c.alloc((void **)&tmp64, np * K * 8));
  CUDA_TRY(cudaMemcpyAsync(tmp64, v.data(), np * K * 8, cudaMemcpyHostToDevice, c.stream));
  const int g = c.ew_grid((int64_t)(np * K));
  if (dtype_mask & (1 << F3R_F32)) {
    F3R_TRY(c.alloc((void **)&d.v32, np * K * 4));
    launch_k(c, k_convert_vals<float>, g, kEwThreads, 0, c.stream, tmp64, d.v32, (int64_t)(np * K));
  }
  if (dtype_mask & (1 << F3R_F16)) {
    F3R_TRY(c.alloc((void **)&d.v16, np * K * 2));
    launch_k(c, k_convert_vals<__half>, g, kEwThreads, 0, c.stream, tmp64, d.v16, (int64_t)(np * K));
  }
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(c.stream));
  if (dtype_mask & (1 << F3R_F64)) d.v64 = tmp64;
  else cudaFree(tmp64);
  return F3R_SUCCESS;
}

// The union of several CSR patterns of one shape (each row's columns merged
// and sorted), and every matrix's values on it (zero where it has no entry:
// a zero entry adds 0 x to a row's sum, so the products are unchanged).
static void union_pattern(const std::vector<const HostCSR *> &m, HostCSR &u, std::vector<std::vector<double>> &vals) {
  const int32_t n = m[0]->n;
  u.n = n;
  u.m = m[0]->m;
  u.rptr.assign(n + 1, 0);
  std::vector<std::vector<int32_t>> cols(n);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t i = 0; i < n; i++) {
    std::vector<int32_t> &c = cols[i];
    for (const HostCSR *a : m)
      for (int32_t q = a->rptr[i]; q < a->rptr[i + 1]; q++) c.push_back(a->idx[q]);
    std::sort(c.begin(), c.end());
    c.erase(std::unique(c.begin(), c.end()), c.end());
  }
  for (int32_t i = 0; i < n; i++) u.rptr[i + 1] = u.rptr[i] + (int32_t)cols[i].size();
  u.idx.resize(u.rptr[n]);
  u.val.assign(u.rptr[n], 0.0);
  for (int32_t i = 0; i < n; i++) std::copy(cols[i].begin(), cols[i].end(), u.idx.begin() + u.rptr[i]);
  vals.assign(m.size(), std::vector<double>(u.rptr[n], 0.0));
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t i = 0; i < n; i++)
    for (size_t s = 0; s < m.size(); s++) {
      const HostCSR *a = m[s];
      int32_t qu = u.rptr[i];
      for (int32_t q = a->rptr[i]; q < a->rptr[i + 1]; q++) {
        while (u.idx[qu] != a->idx[q]) qu++;
        vals[s][qu] = a->val[q];
      }
    }
}

// zf / wf: given SDAINV factors per system (all or none)
static Status make_batch(f3r_context *ctx, int32_t count, const f3r_csr *const *a, const f3r_params *pp, Solver **out,
                         const f3r_csr *const *zf, const f3r_csr *const *wf) {
  if (count < 1 || count > kMaxBlock) return fail(F3R_ERROR_INVALID_VALUE, "a batch holds 1 to 16 systems");
  for (int32_t i = 0; i < count; i++) {
    if (!a[i]) return fail(F3R_ERROR_INVALID_VALUE, "null system");
    F3R_TRY(check_csr(a[i]));
  }
  const f3r_csr &a0 = *a[0];
  if (a0.nrows != a0.ncols) return fail(F3R_ERROR_INVALID_VALUE, "the system matrices must be square");
  for (int32_t i = 1; i < count; i++) {
    const f3r_csr &ai = *a[i];
    if (ai.nrows != a0.nrows || ai.ncols != a0.ncols || ai.nnz != a0.nnz ||
        std::memcmp(ai.rptr, a0.rptr, sizeof(int32_t) * (a0.nrows + 1)) != 0 ||
        (a0.nnz && std::memcmp(ai.idx, a0.idx, sizeof(int32_t) * a0.nnz) != 0))
      return fail(F3R_ERROR_INVALID_VALUE, "the systems of a batch must share one sparsity pattern");
  }
  f3r_params p = *pp;
  if (p.precond != F3R_PRECOND_SDAINV || p.inner_sstep || p.half_m > 0 || p.format != F3R_FORMAT_SELL)
    return fail(F3R_ERROR_UNSUPPORTED, "a batch takes SDAINV, FGMRES levels and SELL storage");
  if (p.m_outer < 1 || p.m_outer + 1 > kMaxCols || p.m2 < 1 || p.m2 + 1 > kMaxCols || p.m3 < 0 || p.m3 + 1 > kMaxCols ||
      p.m4 < 1 || p.m4 > kMaxM4 || p.c < 1 || p.max_restarts < 1 || p.static_weight < 0 || p.sell_sigma < 1)
    return fail(F3R_ERROR_INVALID_VALUE, "need 1 <= m_outer, m2 <= 127, 0 <= m3 <= 127, 1 <= m4 <= 16, c >= 1");
  if (p.half_scale_log2 < 0 || p.half_scale_log2 > 20) return fail(F3R_ERROR_INVALID_VALUE, "half_scale_log2 in [0, 20]");
  if (p.diag_load != 0 && p.diag_load != 1) return fail(F3R_ERROR_INVALID_VALUE, "diag_load is 0 or 1");
  p.sell_align = 0;  // packed layout with per-column values
  p.sell_index16 = 0;
  p.sell_autotune = 0;
  const int K = count <= 2 ? 2 : count <= 4 ? 4 : count <= 8 ? 8 : 16;
  CUDA_TRY(cudaSetDevice(ctx->device));
  auto s = std::make_unique<Solver>();
  s->ctx = ctx;
  s->p = p;
  s->n = a0.nrows;
  s->ldn = ((int64_t)a0.nrows + 7) / 8 * 8;
  s->mm = true;
  s->mm_k = K;
  s->mm_count = count;
  s->z16 = p.m3 > 0 && p.half_scale_log2 == 0 && !(p.inner_sstep & 2) && p.half_m == 0;
  const int32_t n = a0.nrows;
  const int all_types = (1 << F3R_F64) | (1 << F3R_F32) | (1 << F3R_F16);
  // the row order of sigma-sorting (row lengths are the pattern's: one order for all)
  std::vector<int32_t> hperm;
  {
    SellHost h;
    F3R_TRY(build_sell(a0, p.sell_sigma, true, h));
    hperm = h.perm;
  }
  std::vector<const double *> av;
  for (int32_t i = 0; i < count; i++) av.push_back(a[i]->val);
  F3R_TRY(upload_sell_mm(*ctx, a0, hperm, av, K, all_types, s->A));
  s->A.sigma = p.sell_sigma;
  s->perm = hperm;
  if (p.sell_sigma > 1) {
    F3R_TRY(s->alloc(&s->perm_d, (size_t)std::max(n, 1)));
    CUDA_TRY(cudaMemcpy(s->perm_d, hperm.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice));
  }
  // every system's SDAINV factors (given, or computed here)
  std::vector<std::unique_ptr<HostCSR>> Zs, Ws;
  auto copy = [](const f3r_csr &m) {
    HostCSR *h = new HostCSR(m.nrows, m.ncols, m.nnz);
    std::memcpy(h->rptr.data(), m.rptr, sizeof(int32_t) * (m.nrows + 1));
    std::memcpy(h->idx.data(), m.idx, sizeof(int32_t) * m.nnz);
    std::memcpy(h->val.data(), m.val, sizeof(double) * m.nnz);
    return h;
  };
  for (int32_t i = 0; i < count; i++) {
    if (zf) {
      if (!zf[i] || !wf[i]) return fail(F3R_ERROR_INVALID_VALUE, "give the factors of every system or of none");
      F3R_TRY(check_csr(zf[i]));
      F3R_TRY(check_csr(wf[i]));
      if (zf[i]->nrows != n || zf[i]->ncols != n || wf[i]->nrows != n || wf[i]->ncols != n)
        return fail(F3R_ERROR_INVALID_VALUE, "the factors must be square and of the matrix's size");
      Zs.emplace_back(copy(*zf[i]));
      Ws.emplace_back(copy(*wf[i]));
    } else {
      std::unique_ptr<HostCSR> Ah(copy(*a[i]));
      HostCSR *zr = nullptr, *wr = nullptr;
      F3R_TRY(sdainv(*Ah, p.sdainv_tol, p.acc, &zr, &wr));
      Zs.emplace_back(zr);
      Ws.emplace_back(wr);
    }
  }
  bool diag = true;
  for (int32_t i = 0; i < count && diag; i++)
    for (int32_t r = 0; r < n && diag; r++) {
      diag &= (Zs[i]->rptr[r + 1] - Zs[i]->rptr[r] == 1 && Zs[i]->idx[Zs[i]->rptr[r]] == r);
      diag &= (Ws[i]->rptr[r + 1] - Ws[i]->rptr[r] == 1 && Ws[i]->idx[Ws[i]->rptr[r]] == r);
    }
  if (diag) {
    // one diagonal value per row and system, interleaved, storage order
    s->precond_diag = 1;
    std::vector<double> wdv((size_t)n * K, 0.0), zdv((size_t)n * K, 0.0);
    for (int32_t i = 0; i < count; i++)
      for (int32_t r = 0; r < n; r++) {
        wdv[(size_t)r * K + i] = Ws[i]->val[Ws[i]->rptr[hperm[r]]];
        zdv[(size_t)r * K + i] = Zs[i]->val[Zs[i]->rptr[hperm[r]]];
      }
    double *tmp = nullptr;
    const size_t nn = (size_t)std::max(n, 1) * K;
    F3R_TRY(ctx->alloc((void **)&tmp, sizeof(double) * nn));
    F3R_TRY(s->alloc(&s->wd, nn));
    F3R_TRY(s->alloc(&s->zd, nn));
    CUDA_TRY(cudaMemcpy(tmp, wdv.data(), sizeof(double) * nn, cudaMemcpyHostToDevice));
    launch_k(*ctx, k_convert_vals<__half>, ctx->ew_grid((int64_t)nn), kEwThreads, 0, ctx->stream, tmp, s->wd,
             (int64_t)nn);
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(cudaMemcpy(tmp, zdv.data(), sizeof(double) * nn, cudaMemcpyHostToDevice));
    launch_k(*ctx, k_convert_vals<__half>, ctx->ew_grid((int64_t)nn), kEwThreads, 0, ctx->stream, tmp, s->zd,
             (int64_t)nn);
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    cudaFree(tmp);
    F3R_TRY(s->detect_unit_diag(nn));
  } else {
    // W^T and Z of every system on the union of their patterns, rows in the storage order
    for (int which = 0; which < 2; which++) {
      std::vector<const HostCSR *> ms;
      for (int32_t i = 0; i < count; i++) ms.push_back(which == 0 ? Ws[i].get() : Zs[i].get());
      HostCSR u;
      std::vector<std::vector<double>> uv;
      union_pattern(ms, u, uv);
      std::vector<const double *> pv;
      for (auto &vv : uv) pv.push_back(vv.data());
      F3R_TRY(upload_sell_mm(*ctx, u.view(), hperm, pv, K, 1 << F3R_F16, which == 0 ? s->W : s->Z));
    }
  }
  CUDA_TRY(cudaEventCreate(&s->ev0));
  CUDA_TRY(cudaEventCreate(&s->ev1));
  CUDA_TRY(cudaDeviceSynchronize());
  *out = s.release();
  return F3R_SUCCESS;
}

// One solve of every system of a batch: b[i], x[i] host or device vectors
// (x[i] the initial guess on entry), in the K-column engine.
Status Solver::solve_batch(const double *const *b, double *const *x, f3r_cond_fn cond, void *user,
                           f3r_result *results) {
  auto is_dev = [&](const void *q) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
  };
  const int64_t N = n;
  cudaStream_t st = C().stream;
  const int g = C().ew_grid(N);
  const int nc = mm_count;
  auto run = [&](auto kc) -> Status {
    constexpr int K = decltype(kc)::value;
    Work<K> *wk = nullptr;
    F3R_TRY(work<K>(&wk));
    Work<K> &w = *wk;
    double *bi = perm_d ? w.bp_d : w.b_d, *xi = perm_d ? w.xp_d : w.x_d;
    for (int c = 0; c < nc; c++)
      CUDA_TRY(cudaMemcpyAsync(w.stage + (size_t)c * N, b[c], sizeof(double) * N,
                               is_dev(b[c]) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    launch_k(C(), k_interleave, g, kEwThreads, 0, st, (const double *)w.stage, N, nc, K, w.b_d, N);
    for (int c = 0; c < nc; c++)
      CUDA_TRY(cudaMemcpyAsync(w.stage + (size_t)c * N, x[c], sizeof(double) * N,
                               is_dev(x[c]) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    launch_k(C(), k_interleave, g, kEwThreads, 0, st, (const double *)w.stage, N, nc, K, w.x_d, N);
    if (perm_d) {
      launch_k(C(), k_permute_gatherK<K>, g, kEwThreads, 0, st, (const double *)w.b_d, perm_d, bi, N);
      launch_k(C(), k_permute_gatherK<K>, g, kEwThreads, 0, st, (const double *)w.x_d, perm_d, xi, N);
    }
    F3R_TRY(Engine<K>(*this, w).solve_block(bi, xi, nc, cond, user, results));
    if (perm_d) launch_k(C(), k_permute_scatterK<K>, g, kEwThreads, 0, st, (const double *)xi, perm_d, w.x_d, N);
    launch_k(C(), k_deinterleave, g, kEwThreads, 0, st, (const double *)w.x_d, K, nc, w.stage, N, N);
    for (int c = 0; c < nc; c++)
      CUDA_TRY(cudaMemcpyAsync(x[c], w.stage + (size_t)c * N, sizeof(double) * N,
                               is_dev(x[c]) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return F3R_SUCCESS;
  };
  switch (mm_k) {
    case 2: return run(std::integral_constant<int, 2>());
    case 4: return run(std::integral_constant<int, 4>());
    case 8: return run(std::integral_constant<int, 8>());
    default: return run(std::integral_constant<int, 16>());
  }
}

}  // namespace f3r

struct f3r_solver {
  f3r::Solver *s = nullptr;
};

namespace f3r {
const void *solver_context(const f3r_solver *s) { return s && s->s ? (const void *)s->s->ctx : nullptr; }
int32_t solver_rows(const f3r_solver *s) { return s && s->s ? s->s->n : 0; }
Status solver_solve_multi(f3r_solver *s, int32_t nrhs, const double *b, int64_t ldb, double *x, int64_t ldx,
                          f3r_cond_fn cond, void *user, f3r_result *results) {
  clear_stale_error();
  CUDA_TRY(cudaSetDevice(s->s->ctx->device));
  return s->s->solve_multi(nrhs, b, ldb, x, ldx, cond, user, results);
}
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
  clear_stale_error();
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
  clear_stale_error();
  if (!ctx || !out) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  if (slice_height != 32 && slice_height != 64) return fail(F3R_ERROR_UNSUPPORTED, "slice height 32 or 64");
  if (slice_height == 64 && (sigma != 1 || (dtype_mask & (F3R_SELL_INDEX16 | F3R_SELL_CSR))))
    return fail(F3R_ERROR_INVALID_VALUE, "slice height 64: sigma 1, offset-aligned slices");
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
  if (slice_height == 64) {
    if (!align64(*a, h)) return fail(F3R_ERROR_UNSUPPORTED, "64-row slices need every 64 rows to share their offsets");
  } else if (dtype_mask & F3R_SELL_ALIGNED) {
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
  info->slice_height = m->d.rptr ? 0 : m->d.height;
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
  clear_stale_error();
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
  clear_stale_error();
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
  clear_stale_error();
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
  clear_stale_error();
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
  clear_stale_error();
  if (!ctx || !a || !p || !out) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  Solver *s = nullptr;
  F3R_TRY(make_solver(ctx, a, p, &s));
  *out = new f3r_solver{s};
  return F3R_SUCCESS;
}
f3r_status f3r_solver_create_factors(f3r_context *ctx, const f3r_csr *a, const f3r_params *p, const f3r_csr *z,
                                     const f3r_csr *wt, f3r_solver **out) {
  clear_stale_error();
  if (!ctx || !a || !p || !z || !wt || !out) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  Solver *s = nullptr;
  F3R_TRY(make_solver(ctx, a, p, &s, z, wt));
  *out = new f3r_solver{s};
  return F3R_SUCCESS;
}
f3r_status f3r_solver_solve(f3r_solver *s, const double *b, double *x, f3r_cond_fn cond, void *user,
                            f3r_result *result) {
  clear_stale_error();
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
    a_info->slice_height = d.rptr ? 0 : d.height;
    a_info->sigma = d.sigma;
    a_info->nslices = d.nslices;
    a_info->nnz_padded = d.nnz_pad;
    a_info->max_width = d.max_width;
    a_info->dtypes = d.dtypes;
    a_info->index_bits = d.index_bits();
  }
  if (precond_diagonal) *precond_diagonal = s->s->precond_diag ? (s->s->diag_unit ? 2 : 1) : 0;
  return F3R_SUCCESS;
}
f3r_status f3r_solver_operate(f3r_solver *s, f3r_dtype val_t, f3r_dtype in_t, const void *in, f3r_dtype out_t,
                              void *out) {
  clear_stale_error();
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

f3r_status f3r_batch_create(f3r_context *ctx, int32_t count, const f3r_csr *const *a, const f3r_params *p,
                            const f3r_csr *const *z, const f3r_csr *const *wt, f3r_batch **out) {
  clear_stale_error();
  if (!ctx || !a || !p || !out || (z != nullptr) != (wt != nullptr)) return fail(F3R_ERROR_INVALID_VALUE, "bad argument");
  Solver *s = nullptr;
  F3R_TRY(make_batch(ctx, count, a, p, &s, z, wt));
  *out = reinterpret_cast<f3r_batch *>(new f3r_solver{s});
  return F3R_SUCCESS;
}
f3r_status f3r_batch_solve(f3r_batch *bt, const double *const *b, double *const *x, f3r_cond_fn cond, void *user,
                           f3r_result *results) {
  clear_stale_error();
  f3r_solver *s = reinterpret_cast<f3r_solver *>(bt);
  if (!s || !b || !x) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  for (int i = 0; i < s->s->mm_count; i++)
    if (!b[i] || !x[i]) return fail(F3R_ERROR_INVALID_VALUE, "null vector");
  CUDA_TRY(cudaSetDevice(s->s->ctx->device));
  return s->s->solve_batch(b, x, cond, user, results);
}
f3r_status f3r_batch_info(const f3r_batch *bt, int32_t *count, int32_t *width, int32_t *precond_diagonal) {
  const f3r_solver *s = reinterpret_cast<const f3r_solver *>(bt);
  if (!s) return fail(F3R_ERROR_INVALID_VALUE, "null batch");
  if (count) *count = s->s->mm_count;
  if (width) *width = s->s->mm_k;
  if (precond_diagonal) *precond_diagonal = s->s->precond_diag ? (s->s->diag_unit ? 2 : 1) : 0;
  return F3R_SUCCESS;
}
void f3r_batch_destroy(f3r_batch *bt) { f3r_solver_destroy(reinterpret_cast<f3r_solver *>(bt)); }

void f3r_solver_destroy(f3r_solver *s) {
  if (!s) return;
  if (cudaSetDevice(s->s->ctx->device) != cudaSuccess) return;  // runtime shutting down: left to the exit
  cudaStreamSynchronize(s->s->ctx->stream);
  delete s->s;
  delete s;
}

}  // extern "C"
