// tune.cu -- the launch-shape autotuner of the SELL SpMV.
//
// The SELL kernel's speed on B200 depends on how many warps per SM consume
// slices at once (registers), how many bulk-copy stages each warp keeps in
// flight and how many columns one copy carries.  f3r_sell_tune times the
// product out = A x on a given matrix at every launch shape compiled here and
// returns the timings, fastest first; the library's default shapes
// (SellCfg in sell.cuh) are the fastest ones this tuner found on the
// 192^3 27-point benchmark matrix.
#include <algorithm>
#include <vector>

#include "objects.cuh"

namespace f3r {
namespace {

template <typename V, typename X, typename Y, int W, int S, int KC, typename CI>
void time_shape_run(Context &c, const DeviceSell &d, const V *val, const X *x, Y *y, int reps,
                    std::vector<f3r_tune_entry> &out) {
  auto k = k_sell_cfg<V, X, EpiStore<Y>, W, S, KC, CI>;
  const size_t smem = sell_smem_bytes_cfg<V, CI, W, S, KC>();
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device) != cudaSuccess ||
      smem > (size_t)optin)
    return;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return;
  const DevSell A = d.view();
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(A.nslices, W), c.sm_count));
  const EpiStore<Y> epi{y, A.perm};
  for (int i = 0; i < 2; i++) k<<<grid, W * 32, smem, c.stream>>>(val, A, x, epi, c.err);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c.stream);
  for (int i = 0; i < reps; i++) k<<<grid, W * 32, smem, c.stream>>>(val, A, x, epi, c.err);
  cudaEventRecord(e1, c.stream);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (cudaGetLastError() != cudaSuccess) return;
  f3r_tune_entry t{};
  t.warps = W;
  t.stages = S;
  t.kc = KC;
  t.index_bits = IdxForm<CI>::mode >= 2 ? 0 : IdxForm<CI>::mode == 1 ? 16 : 32;
  t.is_default = (W == SellCfg<V, CI>::WARPS && S == SellCfg<V, CI>::STAGES && KC == SellCfg<V, CI>::KC) ? 1 : 0;
  t.microseconds = ms * 1e3 / reps;
  const double nnz = (double)d.nnz, n = (double)d.n;
  t.gbs_algorithmic = (nnz * (sizeof(V) + 4) + 4 * (n + 1) + n * sizeof(X) + n * sizeof(Y)) / (t.microseconds * 1e3);
  out.push_back(t);
}

// the 64-row aligned kernel (k_sell64) at one launch shape
template <typename V, typename X, typename Y, int W, int S>
void time_shape64(Context &c, const DeviceSell &d, const V *val, const X *x, Y *y, int reps,
                  std::vector<f3r_tune_entry> &out) {
  auto k = k_sell64<V, X, EpiStore<Y>, W, S, kAllAlignedChunk>;
  const size_t smem = sell64_smem_bytes_cfg<V, W, S, kAllAlignedChunk>();
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device) != cudaSuccess ||
      smem > (size_t)optin)
    return;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return;
  const DevSell A = d.view();
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(A.nslices, W), c.sm_count));
  const EpiStore<Y> epi{y, A.perm};
  for (int i = 0; i < 2; i++) k<<<grid, W * 32, smem, c.stream>>>(val, A, x, epi, c.err);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c.stream);
  for (int i = 0; i < reps; i++) k<<<grid, W * 32, smem, c.stream>>>(val, A, x, epi, c.err);
  cudaEventRecord(e1, c.stream);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (cudaGetLastError() != cudaSuccess) return;
  f3r_tune_entry t{};
  t.warps = W;
  t.stages = S;
  t.kc = kAllAlignedChunk;
  t.index_bits = 0;
  t.is_default = (W == Sell64Cfg<V>::WARPS && S == Sell64Cfg<V>::STAGES) ? 1 : 0;
  t.microseconds = ms * 1e3 / reps;
  const double nnz = (double)d.nnz, n = (double)d.n;
  t.gbs_algorithmic = (nnz * (sizeof(V) + 4) + 4 * (n + 1) + n * sizeof(X) + n * sizeof(Y)) / (t.microseconds * 1e3);
  out.push_back(t);
}

template <typename V, typename X, typename Y>
void sweep64(Context &c, const DeviceSell &d, const V *val, const X *x, Y *y, int reps,
             std::vector<f3r_tune_entry> &out) {
  time_shape64<V, X, Y, 32, 2>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 28, 2>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 24, 2>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 24, 3>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 20, 2>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 16, 2>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 16, 3>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 12, 2>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 10, 2>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 8, 2>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 6, 2>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 4, 3>(c, d, val, x, y, reps, out);
  // one stage a warp: twice the warps in the same shared memory
  time_shape64<V, X, Y, 32, 1>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 24, 1>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 16, 1>(c, d, val, x, y, reps, out);
  time_shape64<V, X, Y, 12, 1>(c, d, val, x, y, reps, out);
}

// the aligned forms' value layouts are built for one chunk width each
template <typename V, typename X, typename Y, int W, int S, int KC, typename CI>
void time_shape(Context &c, const DeviceSell &d, const V *val, const X *x, Y *y, int reps,
                std::vector<f3r_tune_entry> &out) {
  if constexpr ((IdxForm<CI>::mode == 2 && KC != kAlignedChunk) || (IdxForm<CI>::mode == 3 && KC != kAllAlignedChunk))
    return;
  else
    time_shape_run<V, X, Y, W, S, KC, CI>(c, d, val, x, y, reps, out);
}

template <typename V, typename X, typename Y, typename CI>
void sweep(Context &c, const DeviceSell &d, const V *val, const X *x, Y *y, int reps, std::vector<f3r_tune_entry> &out) {
  if constexpr (IdxForm<CI>::mode == 3) {
    time_shape<V, X, Y, 32, 3, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 32, 2, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 28, 3, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 28, 2, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 24, 4, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 24, 3, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 24, 2, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 20, 2, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 16, 4, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 16, 2, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 12, 3, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 12, 2, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 8, 4, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 8, 2, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 32, 1, 32, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 24, 1, 32, CI>(c, d, val, x, y, reps, out);
  } else {
    time_shape<V, X, Y, 24, 2, 16, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 20, 2, 16, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 20, 3, 16, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 16, 2, 16, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 16, 3, 16, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 12, 4, 16, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 32, 2, 8, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 24, 3, 8, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 8, 4, 16, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 32, 1, 16, CI>(c, d, val, x, y, reps, out);
    time_shape<V, X, Y, 24, 1, 16, CI>(c, d, val, x, y, reps, out);
  }
}

template <typename V, typename X, typename Y>
Status run(Context &c, const DeviceSell &d, const V *val, int reps, std::vector<f3r_tune_entry> &out) {
  X *x = nullptr;
  Y *y = nullptr;
  F3R_TRY(c.alloc((void **)&x, sizeof(X) * std::max<int64_t>(d.ncols, 1)));
  Status s = c.alloc((void **)&y, sizeof(Y) * std::max<int64_t>(d.n, 1));
  if (s != F3R_SUCCESS) {
    cudaFree(x);
    return s;
  }
  cudaMemsetAsync(x, 0, sizeof(X) * d.ncols, c.stream);
  if (d.height == 64) sweep64<V, X, Y>(c, d, val, x, y, reps, out);
  else if (d.xoff) sweep<V, X, Y, AlignedIdx>(c, d, val, x, y, reps, out);
  else if (d.cbase && !d.dcol) sweep<V, X, Y, AllAlignedIdx>(c, d, val, x, y, reps, out);
  else if (d.dcol) sweep<V, X, Y, uint16_t>(c, d, val, x, y, reps, out);
  else sweep<V, X, Y, int32_t>(c, d, val, x, y, reps, out);
  cudaStreamSynchronize(c.stream);
  cudaFree(x);
  cudaFree(y);
  return F3R_SUCCESS;
}

}  // namespace
}  // namespace f3r

using namespace f3r;

extern "C" f3r_status f3r_sell_tune(f3r_sell *m, f3r_dtype val_t, int32_t reps, f3r_tune_entry *out, int32_t cap,
                                    int32_t *count) {
  clear_stale_error();
  if (!m || !out || !count || cap < 1 || reps < 1) return fail(F3R_ERROR_INVALID_VALUE, "bad argument");
  const DeviceSell &d = m->d;
  if (!(d.dtypes & (1 << val_t))) return fail(F3R_ERROR_INVALID_VALUE, "matrix holds no copy of that value type");
  if (d.rptr) return fail(F3R_ERROR_UNSUPPORTED, "the launch shapes tuned are the SELL kernel's; this matrix is CSR");
  std::vector<f3r_tune_entry> res;
  Context &c = *m->ctx;
  if (val_t == F3R_F16) F3R_TRY((run<__half, float, float>(c, d, d.v16, reps, res)));
  else if (val_t == F3R_F32) F3R_TRY((run<float, float, float>(c, d, d.v32, reps, res)));
  else F3R_TRY((run<double, double, double>(c, d, d.v64, reps, res)));
  std::sort(res.begin(), res.end(),
            [](const f3r_tune_entry &a, const f3r_tune_entry &b) { return a.microseconds < b.microseconds; });
  const int32_t k = std::min<int32_t>(cap, (int32_t)res.size());
  for (int32_t i = 0; i < k; i++) out[i] = res[i];
  *count = k;
  return F3R_SUCCESS;
}
