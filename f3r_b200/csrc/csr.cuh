// csr.cuh -- CSR SpMV with the SELL kernel's epilogues (the format = CSR
// option of the solver and F3R_SELL_CSR matrices).  The reference's CSR
// operate is matrix/csr.hpp's; its GPU drivers use SELL<32>.
//
// The launch geometry is the packed SELL kernel's: WARPS warps per CTA, one
// CTA per SM at most, warp w of CTA b takes the 32-row groups b*WARPS + w,
// + gridDim*WARPS, ...; lane l owns row 32 g + l.  Each warp stages the
// contiguous CSR range of its 32 rows through shared memory in tiles of
// kCsrTile entries (coalesced loads, all issued before any is used), and each
// lane sums its own row sequentially in column order.  So every row's sum,
// every thread's partial dot products and every CTA's partials are the
// packed sigma = 1 SELL kernel's, bit for bit (SELL's padding adds exact
// zeros).
#pragma once

#include "sell.cuh"

namespace f3r {

constexpr int kCsrTile = 512;  // entries staged per warp and tile
constexpr int kCsrBatch = 8;   // gathers in flight per lane

// streamed-once matrix data: read with the evict-first cache hint
template <typename T> __device__ __forceinline__ T ldg_stream(const T *p) { return __ldcs(p); }
template <> __device__ __forceinline__ __half ldg_stream<__half>(const __half *p) {
  return __ushort_as_half(__ldcs(reinterpret_cast<const unsigned short *>(p)));
}

template <typename V> constexpr size_t csr_smem_bytes() {
  return (size_t)SellCfg<V, int32_t>::WARPS * kCsrTile * (sizeof(V) + sizeof(int32_t));
}

template <typename V, typename X, typename Epi, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 1)
    k_csr_cfg(const V *__restrict__ val, DevSell A, const X *__restrict__ x, Epi epi, int *) {
  using Acc = typename acc_of<V>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  V *sv = reinterpret_cast<V *>(smem) + (size_t)warp * kCsrTile;
  int32_t *sc = reinterpret_cast<int32_t *>(smem + (size_t)WARPS * kCsrTile * sizeof(V)) + (size_t)warp * kCsrTile;
  typename Epi::Red dots[Epi::NV > 0 ? Epi::NV : 1];
#pragma unroll
  for (int k = 0; k < (Epi::NV > 0 ? Epi::NV : 1); k++) dots[k] = 0;
  const int TW = gridDim.x * WARPS;
  for (int cs = blockIdx.x * WARPS + warp; cs < A.nslices; cs += TW) {
    const int64_t r = (int64_t)cs * 32 + lane;
    const bool live = r < A.n;
    const int64_t rl = min((int64_t)cs * 32 + 32, (int64_t)A.n);  // end of the group's rows
    const int32_t rb = live ? A.rptr[r] : 0, re = live ? A.rptr[r + 1] : 0;
    const int32_t gb = A.rptr[(int64_t)cs * 32], ge = A.rptr[rl];
    typename Epi::Pre pre{};
    if (live) pre = epi.load(r);
    Acc acc = 0;
    for (int32_t t0 = gb; t0 < ge; t0 += kCsrTile) {
      const int cnt = min(kCsrTile, ge - t0);
      __syncwarp();
      V lv[kCsrTile / 32];
      int32_t lc[kCsrTile / 32];
#pragma unroll
      for (int u = 0; u < kCsrTile / 32; u++) {
        const int k = u * 32 + lane;
        if (k < cnt) {
          lv[u] = ldg_stream(val + t0 + k);
          lc[u] = ldg_stream(A.col + t0 + k);
        }
      }
#pragma unroll
      for (int u = 0; u < kCsrTile / 32; u++) {
        const int k = u * 32 + lane;
        if (k < cnt) {
          sv[k] = lv[u];
          sc[k] = lc[u];
        }
      }
      __syncwarp();
      // the row's terms in column order, gathers issued kCsrBatch at a time
      const int lo = max(rb, t0) - t0, hi = min(re, t0 + cnt) - t0;
      int k = lo;
      for (; k + kCsrBatch <= hi; k += kCsrBatch) {
        Acc xv[kCsrBatch];
#pragma unroll
        for (int e = 0; e < kCsrBatch; e++) xv[e] = to_acc<Acc>(__ldg(x + sc[k + e]));
#pragma unroll
        for (int e = 0; e < kCsrBatch; e++) acc = fmaT(to_acc<Acc>(sv[k + e]), xv[e], acc);
      }
      for (; k < hi; k++) acc = fmaT(to_acc<Acc>(sv[k]), to_acc<Acc>(__ldg(x + sc[k])), acc);
    }
    if (live) epi.row(r, acc, pre, dots);
  }
  epi.template finish<WARPS>(dots);
}

}  // namespace f3r
