// objects.cuh -- device-side objects shared by the translation units of the
// library: the context (device, stream, reduction scratch), the device SELL
// matrix, the counting kernel launcher and the SELL SpMV launcher.
#pragma once

#include <algorithm>
#include <string>
#include <vector>

#include "internal.hpp"
#include "csr.cuh"
#include "sell.cuh"

namespace f3r {

#define CUDA_TRY(x)                                                                               \
  do {                                                                                            \
    cudaError_t e_ = (x);                                                                         \
    if (e_ != cudaSuccess)                                                                        \
      return fail(e_ == cudaErrorMemoryAllocation ? F3R_ERROR_OUT_OF_MEMORY : F3R_ERROR_CUDA,     \
                  std::string(#x) + ": " + cudaGetErrorString(e_));                               \
  } while (0)

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Entry points that run CUDA work start here: the runtime keeps the last
// non-sticky error of any earlier call on this thread (the caller's, another
// library's) until someone reads it, and the launch checks below read it, so
// it is cleared first.  A sticky error (a lost context) is returned by every
// later call anyway.
inline void clear_stale_error() { (void)cudaGetLastError(); }

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------

struct Context {
  int device = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  int sm_count = 148;
  int *err = nullptr;          // device error word (DevError)
  void *partials = nullptr;    // grid-reduction partial sums
  unsigned int *ticket = nullptr;
  double *pinned = nullptr;    // host-pinned scalars for D2H reads
  double *dscratch = nullptr;  // device scalars for f3r_dot
  int64_t launches = 0;        // kernels issued through this context
  std::vector<void *> allocs;

  Status alloc(void **p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess)
      return fail(e == cudaErrorMemoryAllocation ? F3R_ERROR_OUT_OF_MEMORY : F3R_ERROR_CUDA,
                  std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    return F3R_SUCCESS;
  }
  GridRed gred() const { return GridRed{partials, ticket}; }
  // grid for the elementwise / reduction kernels: up to 8 blocks of 256 per SM
  // (full thread occupancy); partial-sum buffers are sized for this bound
  int ew_grid(int64_t n) const { return (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, kEwThreads), (int64_t)sm_count * 8)); }
  // checks the device error word.  Stream-ordered on this context's stream
  // (no legacy-stream call), so it may run while another thread captures a
  // graph on its own context.
  Status check_device_error() {
    int *e_h = reinterpret_cast<int *>(pinned + 7);
    CUDA_TRY(cudaMemcpyAsync(e_h, err, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaStreamSynchronize(stream));
    const int e = *e_h;
    if (e == DEV_OK) return F3R_SUCCESS;
    CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), stream));
    CUDA_TRY(cudaStreamSynchronize(stream));
    if (e == DEV_TIMEOUT_SPMV) return fail(F3R_ERROR_TIMEOUT, "a bulk-copy wait in the SpMV kernel exceeded its bound");
    if (e == DEV_TIMEOUT_TRSV)
      return fail(F3R_ERROR_TIMEOUT, "a dependency wait in the level-scheduled ILU solve exceeded its bound");
    if (e == DEV_TIMEOUT_MMA)
      return fail(F3R_ERROR_TIMEOUT, "a tensor-core completion wait in the MLP inference exceeded its bound");
    return fail(F3R_ERROR_BREAKDOWN, "zero or non-finite norm in an Arnoldi step");
  }
};


// Launches a kernel on the context's bookkeeping (every launch is counted,
// so a solve can report how many kernels of this library it ran).
template <typename... KP, typename... A>
inline void launch_k(Context &c, void (*k)(KP...), dim3 grid, int block, size_t smem, cudaStream_t st,
                            A &&...args) {
  k<<<grid, block, smem, st>>>(std::forward<A>(args)...);
  c.launches++;
}


struct DeviceSell {
  int32_t n = 0, ncols = 0, nslices = 0, max_width = 0, sigma = 1;
  int64_t nnz = 0, nnz_pad = 0;
  int32_t *col = nullptr, *sptr = nullptr, *perm = nullptr, *cbase = nullptr, *cbptr = nullptr;
  int32_t *xoff = nullptr;  // mixed aligned form: per slice, -1 or the explicit indices' offset
  int32_t *rptr = nullptr;  // CSR storage (col = CSR indices, values unpadded), else nullptr
  int32_t height = 32;      // slice height: 32, or 64 (64-row aligned slices)
  uint16_t *dcol = nullptr;
  double *v64 = nullptr;
  float *v32 = nullptr;
  __half *v16 = nullptr;
  int dtypes = 0;
  // 32, 16, or 0 (offset-aligned slices, mixed with explicit ones or not)
  int index_bits() const { return (xoff || (cbase && !dcol)) ? 0 : dcol ? 16 : 32; }
  DevSell view() const { return DevSell{col, dcol, cbase, cbptr, xoff, sptr, perm, n, ncols, nslices, rptr, height}; }
  void release() {
    cudaFree(col); cudaFree(sptr); cudaFree(perm); cudaFree(cbase); cudaFree(cbptr); cudaFree(dcol);
    cudaFree(xoff);
    cudaFree(rptr);
    cbptr = nullptr;
    xoff = nullptr;
    rptr = nullptr;
    cudaFree(v64); cudaFree(v32); cudaFree(v16);
    col = sptr = perm = cbase = nullptr; dcol = nullptr; v64 = nullptr; v32 = nullptr; v16 = nullptr;
  }
};


template <typename V, typename X, typename Epi, typename CI>
inline Status sell_attr_one() {
  using Cfg = SellCfg<V, CI>;
  CUDA_TRY(cudaFuncSetAttribute(k_sell_cfg<V, X, Epi, Cfg::WARPS, Cfg::STAGES, Cfg::KC, CI>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sell_smem_bytes<V, CI>()));
  return F3R_SUCCESS;
}

// Raises the kernel's dynamic shared memory limit once per device, for every
// index form.  Called before any graph capture for every instantiation the
// solver uses.
template <typename V, typename X, typename Epi>
inline Status sell_attr(Context &c) {
  static int attr_done[64] = {0};
  if (!attr_done[c.device & 63]) {
    F3R_TRY((sell_attr_one<V, X, Epi, int32_t>()));
    F3R_TRY((sell_attr_one<V, X, Epi, uint16_t>()));
    F3R_TRY((sell_attr_one<V, X, Epi, AlignedIdx>()));
    F3R_TRY((sell_attr_one<V, X, Epi, AllAlignedIdx>()));
    CUDA_TRY(cudaFuncSetAttribute(k_csr_cfg<V, X, Epi, SellCfg<V, int32_t>::WARPS>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csr_smem_bytes<V>()));
    using C64 = Sell64Cfg<V>;
    CUDA_TRY(cudaFuncSetAttribute(k_sell64<V, X, Epi, C64::WARPS, C64::STAGES, C64::KC>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sell64_smem_bytes<V>()));
    attr_done[c.device & 63] = 1;
  }
  return F3R_SUCCESS;
}

template <typename V, typename X, typename Epi, typename CI>
inline void launch_sell_one(Context &c, const V *val, const DevSell &A, const X *x, const Epi &epi) {
  using Cfg = SellCfg<V, CI>;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(A.nslices, Cfg::WARPS), c.sm_count));
  launch_k(c, k_sell_cfg<V, X, Epi, Cfg::WARPS, Cfg::STAGES, Cfg::KC, CI>, grid, Cfg::WARPS * 32,
           sell_smem_bytes<V, CI>(), c.stream, val, A, x, epi, c.err);
}

template <typename V, typename X, typename Epi>
inline Status launch_sell(Context &c, const V *val, const DevSell &A, const X *x, const Epi &epi) {
  if (A.nslices == 0) return F3R_SUCCESS;
  F3R_TRY((sell_attr<V, X, Epi>(c)));
  if (A.height == 64) {
    using C64 = Sell64Cfg<V>;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(A.nslices, C64::WARPS), c.sm_count));
    launch_k(c, k_sell64<V, X, Epi, C64::WARPS, C64::STAGES, C64::KC>, grid, C64::WARPS * 32, sell64_smem_bytes<V>(),
             c.stream, val, A, x, epi, c.err);
  } else if (A.rptr) {
    // the packed kernel's geometry (rows per thread, CTAs), so sums and partials match it
    constexpr int W = SellCfg<V, int32_t>::WARPS;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(A.nslices, W), c.sm_count));
    launch_k(c, k_csr_cfg<V, X, Epi, W>, grid, W * 32, csr_smem_bytes<V>(), c.stream, val, A, x, epi, c.err);
  } else if (A.xoff) launch_sell_one<V, X, Epi, AlignedIdx>(c, val, A, x, epi);
  else if (A.cbase && !A.dcol) launch_sell_one<V, X, Epi, AllAlignedIdx>(c, val, A, x, epi);
  else if (A.dcol) launch_sell_one<V, X, Epi, uint16_t>(c, val, A, x, epi);
  else launch_sell_one<V, X, Epi, int32_t>(c, val, A, x, epi);
  CUDA_TRY(cudaGetLastError());
  return F3R_SUCCESS;
}

// ---------------------------------------------------------------------------
// SELL-32 construction on the host (solver.cu)
// ---------------------------------------------------------------------------
struct SellHost {
  int32_t n = 0, ncols = 0, nslices = 0, max_width = 0, sigma = 1;
  int64_t nnz = 0, nnz_pad = 0;
  std::vector<int32_t> sptr, col, perm;  // perm: storage row -> original row
  std::vector<double> val;
  std::vector<uint16_t> dcol;            // 16-bit offsets (when they fit)
  std::vector<int32_t> cbase;            // base of each slice column, slice s from cbptr[s]
  std::vector<int32_t> cbptr;            // nslices + 1, multiples of 4 (aligned forms: bit 0 = clamp)
  std::vector<int32_t> xoff;             // mixed aligned form: per slice, -1 or explicit offset
  bool aligned_all = false;              // fully aligned form (no explicit index at all)
  int32_t height = 32;                   // slice height (64: align64's 64-row slices)
};

// Rows sorted by decreasing length in windows of sigma (renumber: columns
// mapped to the storage order too, P A P^T); given_perm fixes the order.
Status build_sell(const f3r_csr &a, int32_t sigma, bool renumber, SellHost &s,
                  const std::vector<int32_t> *given_perm = nullptr);
// 16-bit column offsets when every slice column fits a 65536 window
bool compress_index16(SellHost &s);
// Re-lays a packed SellHost out offset-aligned: the fully aligned form when
// every slice's rows share their column offsets (offset set at most 5/4 of
// the slice's width), otherwise the mixed form.  Returns the fraction of
// slices aligned, or -1 when the padded matrix would exceed 2^31 entries.
double align_offsets(const f3r_csr &a, bool renumber, SellHost &s);
// 64-row fully aligned slices of a (rows in their natural order): true when
// every 64-row slice's rows share their column offsets (offset set at most
// 5/4 of the slice's width), false otherwise (s untouched).
bool align64(const f3r_csr &a, SellHost &s);
// Uploads the value copies selected by dtype_mask (bit 1 << f3r_dtype).
Status upload_sell(Context &c, const SellHost &h, int dtype_mask, bool scatter_perm, DeviceSell &d);
// CSR storage with the same value copies (the kernels' CSR path; sigma 1)
Status upload_csr(Context &c, const f3r_csr &a, int dtype_mask, DeviceSell &d);

}  // namespace f3r

struct f3r_context : f3r::Context {};

struct f3r_sell {
  f3r_context *ctx = nullptr;
  f3r::DeviceSell d;
};
