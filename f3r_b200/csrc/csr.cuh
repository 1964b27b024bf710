// csr.cuh -- CSR SpMV with the SELL kernel's epilogues (the format = CSR
// option of the solver and F3R_SELL_CSR matrices).  The reference's CSR
// operate is matrix/csr.hpp's; its GPU drivers use SELL<32>.
//
// The launch geometry is the packed SELL kernel's: WARPS warps per CTA, one
// CTA per SM at most, warp w of CTA b takes the 32-row groups b*WARPS + w,
// + gridDim*WARPS, ...; lane l owns row 32 g + l.  Each warp streams the
// contiguous CSR range of its groups through a two-stage shared-memory ring
// in tiles of up to kCsrTile entries: the tile's byte range, widened to
// 16-byte boundaries, is copied with 16-byte cp.async (the next tile is in
// flight while the current one is summed), and each lane sums its own row
// sequentially in column order, kCsrBatch gathers at a time.  So every row's
// sum, every thread's partial dot products and every CTA's partials are the
// packed sigma = 1 SELL kernel's, bit for bit (SELL's padding adds exact
// zeros).  The value and index arrays carry kCsrPad elements of padding, so
// the widened copies stay inside their allocations.
#pragma once

#include "sell.cuh"

namespace f3r {

constexpr int kCsrTile = 512;  // entries per tile
constexpr int kCsrBatch = 8;   // gathers in flight per lane
constexpr int kCsrPad = 16;    // elements of padding after the value and index arrays

template <typename V> constexpr uint32_t csr_vstage() { return kCsrTile * sizeof(V) + 32; }
constexpr uint32_t csr_istage() { return kCsrTile * 4 + 32; }
template <typename V> constexpr size_t csr_smem_bytes() {
  return (size_t)SellCfg<V, int32_t>::WARPS * 2 * (csr_vstage<V>() + csr_istage());
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <typename V, typename X, typename Epi, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 1)
    k_csr_cfg(const V *__restrict__ val, DevSell A, const X *__restrict__ x, Epi epi, int *) {
  epi_setup(epi, 0);
  using Acc = typename acc_of<V>::type;
  constexpr uint32_t VS = csr_vstage<V>(), IS = csr_istage();
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char *vbuf = smem + (size_t)warp * 2 * (VS + IS);  // stage s: values at s * VS
  unsigned char *ibuf = vbuf + 2 * VS;                       // stage s: indices at s * IS
  typename Epi::Red dots[Epi::NV > 0 ? Epi::NV : 1];
#pragma unroll
  for (int k = 0; k < (Epi::NV > 0 ? Epi::NV : 1); k++) dots[k] = 0;
  const int TW = gridDim.x * WARPS;
  auto gend = [&](int c) { return A.rptr[min((int64_t)c * 32 + 32, (int64_t)A.n)]; };
  // first tile of the first non-empty group at or after c (stepping TW)
  auto first_from = [&](int c, int &pc, int32_t &pt) {
    for (; c < A.nslices; c += TW) {
      const int32_t b = A.rptr[(int64_t)c * 32];
      if (b < gend(c)) {
        pc = c;
        pt = b;
        return true;
      }
    }
    return false;
  };
  // copies tile (c, t0) into stage s; returns the element offsets of its first entry
  auto issue = [&](int s, int c, int32_t t0, int &voff, int &ioff) {
    const int32_t cnt = min(kCsrTile, gend(c) - t0);
    const char *vs = reinterpret_cast<const char *>(val);
    const size_t b0 = (size_t)t0 * sizeof(V), a0 = b0 & ~(size_t)15;
    const size_t a1 = ((size_t)(t0 + cnt) * sizeof(V) + 15) & ~(size_t)15;
    for (size_t k = lane; k < (a1 - a0) / 16; k += 32) cp_async16(vbuf + s * VS + k * 16, vs + a0 + k * 16);
    const char *is = reinterpret_cast<const char *>(A.col);
    const size_t c0 = (size_t)t0 * 4, d0 = c0 & ~(size_t)15, d1 = ((size_t)(t0 + cnt) * 4 + 15) & ~(size_t)15;
    for (size_t k = lane; k < (d1 - d0) / 16; k += 32) cp_async16(ibuf + s * IS + k * 16, is + d0 + k * 16);
    cp_async_commit();
    voff = (int)((b0 - a0) / sizeof(V));
    ioff = (int)((c0 - d0) / 4);
  };
  int pc = 0, stage = 0, vo0 = 0, vo1 = 0, io0 = 0, io1 = 0;  // per stage: offsets of the first entry
  int32_t pt = 0;
  // the prefetch cursor (pc, pt): the last tile issued
  if (first_from(blockIdx.x * WARPS + warp, pc, pt)) issue(0, pc, pt, vo0, io0);
  for (int cs = blockIdx.x * WARPS + warp; cs < A.nslices; cs += TW) {
    const int64_t r = (int64_t)cs * 32 + lane;
    const bool live = r < A.n;
    const int32_t rb = live ? A.rptr[r] : 0, re = live ? A.rptr[r + 1] : 0;
    const int32_t gb = A.rptr[(int64_t)cs * 32], ge = gend(cs);
    typename Epi::Pre pre{};
    if (live) pre = epi.load(r);
    Acc acc = 0;
    for (int32_t t0 = gb; t0 < ge; t0 += kCsrTile) {
      // this tile sits in `stage`; put the next one in flight in the other stage
      bool next;
      if (pt + kCsrTile < gend(pc)) {
        pt += kCsrTile;
        next = true;
      } else {
        next = first_from(pc + TW, pc, pt);
      }
      if (next) {
        if (stage) issue(0, pc, pt, vo0, io0);
        else issue(1, pc, pt, vo1, io1);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncwarp();
      const V *sv = reinterpret_cast<const V *>(vbuf + stage * VS) + (stage ? vo1 : vo0);
      const int32_t *sc = reinterpret_cast<const int32_t *>(ibuf + stage * IS) + (stage ? io1 : io0);
      const int cnt = min(kCsrTile, ge - t0);
      const int lo = max(rb, t0) - t0, hi = min(re, t0 + cnt) - t0;
      // the row's terms in column order; the last batch is masked, not reordered
      for (int k = lo; k < hi; k += kCsrBatch) {
        Acc xv[kCsrBatch];
#pragma unroll
        for (int e = 0; e < kCsrBatch; e++)
          if (k + e < hi) xv[e] = to_acc<Acc>(__ldg(x + sc[k + e]));
#pragma unroll
        for (int e = 0; e < kCsrBatch; e++)
          if (k + e < hi) acc = fmaT(to_acc<Acc>(sv[k + e]), xv[e], acc);
      }
      __syncwarp();  // every lane is done with this stage before it is refilled
      stage ^= 1;
    }
    if (live) epi.row(r, acc, pre, dots);
  }
  epi.template finish<WARPS>(dots);
}

}  // namespace f3r
