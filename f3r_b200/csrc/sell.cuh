// sell.cuh -- SELL-32 sparse matrix-vector product for sm_100a.
//
// Layout (built on the host by build_sell in solver.cu): the rows are cut into
// slices of 32; slice s holds width(s) = sptr[s+1]-sptr[s] columns, and entry
// (k, lane) of the slice sits at (sptr[s] + k) * 32 + lane in the value and
// column arrays.  A slice is therefore one contiguous, 64-byte aligned block
// of memory per array, which is what makes it a single bulk copy.  Padding
// entries hold value 0 and repeat the row's previous column, as the
// reference's csr_to_sell does (matrix/sell.hpp:281-285); unlike the
// reference, a ragged last slice is padded to 32 rows so every slice has the
// same stride.
//
// Kernel: every warp owns a private ring of STAGES shared-memory buffers and
// walks the slices blockIdx*WARPS+warp, +gridDim*WARPS, ... in chunks of at
// most KC columns.  Lane 0 issues the bulk (TMA) copies of a chunk's values
// and column indices onto the stage's mbarrier with an L2 evict-first hint
// (the matrix is streamed once per product, the gathered vector should stay
// resident in L2).  All lanes wait on the mbarrier with a time bound, copy the
// chunk into registers and hand the stage straight back to the copy engine;
// only then do they gather x, run the multiply-add chain (lane = row of the
// slice, entries in stored order) and pass the finished row to the epilogue,
// whose own operands were loaded before the chain started.  The epilogue
// stores the result and may fold in residual, preconditioner, axpy and
// dot-product work.
#pragma once

#include "device.cuh"

namespace f3r {

// Column indices come in one of two forms:
//  * col:   int32 per entry;
//  * dcol + cbase: a uint16 offset per entry from an int32 base per slice
//    column, used when every slice column's indices fit in a 65536 window --
//    2 + 4/32 bytes per entry instead of 4.  The bases of slice s start at
//    cbptr[s], a multiple of 4, so a chunk's bases are one 16-byte aligned
//    bulk copy like its values and offsets.
struct DevSell {
  const int32_t *col;     // (sptr[nslices]) * 32, or nullptr
  const uint16_t *dcol;   // (sptr[nslices]) * 32, or nullptr
  const int32_t *cbase;   // cbptr[nslices] (+ padding), with dcol
  const int32_t *cbptr;   // nslices + 1, with dcol
  const int32_t *sptr;    // nslices + 1, in units of 32 entries
  const int32_t *perm;    // storage row -> output row, or nullptr (identity)
  int32_t n;              // rows (outputs written only for storage rows < n)
  int32_t nslices;
};

// Launch shape per value type: WARPS warps per CTA, STAGES buffers per warp,
// KC columns per chunk.  One CTA per SM (the rings take most of the 227 KB).
// Chosen by a sweep on the 192^3 27-point matrix (n = 7.08M, nnz = 189M):
// fp16 values x fp32 vector 24/2/16 -> 187 us (6.5 TB/s), versus 8/4/32 ->
// 345 us; the bound is how many slices are being consumed at once, not how
// many bytes are in flight.
template <typename V> struct SellCfg;
template <> struct SellCfg<__half> { static constexpr int WARPS = 24, STAGES = 2, KC = 16; };
template <> struct SellCfg<float> { static constexpr int WARPS = 24, STAGES = 2, KC = 16; };
template <> struct SellCfg<double> { static constexpr int WARPS = 16, STAGES = 2, KC = 16; };

template <typename V, typename CI, int WARPS, int STAGES, int KC>
constexpr size_t sell_smem_bytes_cfg() {
  return (size_t)WARPS * STAGES * ((size_t)KC * 32 * (sizeof(V) + sizeof(CI)) + (sizeof(CI) == 2 ? KC * 4 : 0)) +
         (size_t)WARPS * STAGES * sizeof(uint64_t);
}
template <typename V, typename CI>
constexpr size_t sell_smem_bytes() {
  return sell_smem_bytes_cfg<V, CI, SellCfg<V>::WARPS, SellCfg<V>::STAGES, SellCfg<V>::KC>();
}

// CI: the stored index type, int32_t (col) or uint16_t (dcol + cbase).
template <typename V, typename X, typename Epi, int WARPS, int STAGES, int KC, typename CI = int32_t>
__global__ void __launch_bounds__(WARPS * 32, 1)
    k_sell_cfg(const V *__restrict__ val, DevSell A, const X *__restrict__ x, Epi epi, int *err) {
  using Acc = typename acc_of<V>::type;
  constexpr bool C16 = sizeof(CI) == 2;
  static_assert(KC % 4 == 0, "chunk width must keep the bases 16-byte aligned");
  constexpr uint32_t VB = KC * 32 * sizeof(V), CB = KC * 32 * sizeof(CI), BB = C16 ? KC * 4 : 0, SB = VB + CB + BB;
  const CI *cidx = C16 ? reinterpret_cast<const CI *>(A.dcol) : reinterpret_cast<const CI *>(A.col);
  extern __shared__ __align__(128) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char *buf = smem + (size_t)warp * STAGES * SB;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + (size_t)WARPS * STAGES * SB) + warp * STAGES;
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < STAGES; s++) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncwarp();
  const uint64_t pol = l2_evict_first_policy();
  const int TW = gridDim.x * WARPS;

  // fetch cursor (warp-uniform)
  int fs = blockIdx.x * WARPS + warp, fk = 0, fst = 0, inflight = 0;
  auto fetch = [&]() {
    while (inflight < STAGES && fs < A.nslices) {
      const int s0 = A.sptr[fs], w = A.sptr[fs + 1] - s0;
      if (w == 0) {
        fs += TW;
        fk = 0;
        continue;
      }
      const int kc = min(KC, w - fk);
      if (lane == 0) {
        const size_t off = ((size_t)s0 + fk) * 32;
        fence_proxy_async_smem();
        const uint32_t bb = C16 ? (uint32_t)((kc + 3) & ~3) * 4u : 0u;
        mbar_arrive_expect_tx(&bars[fst], (uint32_t)kc * 32u * (uint32_t)(sizeof(V) + sizeof(CI)) + bb);
        bulk_g2s(buf + (size_t)fst * SB, val + off, (uint32_t)kc * 32u * (uint32_t)sizeof(V), &bars[fst], pol);
        bulk_g2s(buf + (size_t)fst * SB + VB, cidx + off, (uint32_t)kc * 32u * (uint32_t)sizeof(CI), &bars[fst], pol);
        if (C16) bulk_g2s(buf + (size_t)fst * SB + VB + CB, A.cbase + A.cbptr[fs] + fk, bb, &bars[fst], pol);
      }
      fst = (fst + 1 == STAGES) ? 0 : fst + 1;
      inflight++;
      fk += kc;
      if (fk >= w) {
        fk = 0;
        fs += TW;
      }
    }
  };
  fetch();

  typename Epi::Red dots[Epi::NV > 0 ? Epi::NV : 1];
#pragma unroll
  for (int k = 0; k < (Epi::NV > 0 ? Epi::NV : 1); k++) dots[k] = 0;
  int cs = blockIdx.x * WARPS + warp, ck = 0, cst = 0;
  uint32_t phase = 0;
  bool ok = true;
  Acc acc = 0;
  typename Epi::Pre pre{};
  while (cs < A.nslices) {
    const int s0 = A.sptr[cs], w = A.sptr[cs + 1] - s0;
    const int64_t r = (int64_t)cs * 32 + lane;
    const bool live = r < A.n;
    if (w == 0) {
      if (live) {
        pre = epi.load(r);
        epi.row(r, Acc(0), pre, dots);
      }
      cs += TW;
      continue;
    }
    if (ck == 0 && live) pre = epi.load(r);  // epilogue operands, ahead of the chain
    const int kc = min(KC, w - ck);
    if (!mbar_wait_bounded(&bars[cst], (phase >> cst) & 1u)) {
      ok = false;
      break;
    }
    phase ^= 1u << cst;
    const V *sv = reinterpret_cast<const V *>(buf + (size_t)cst * SB);
    const CI *sc = reinterpret_cast<const CI *>(buf + (size_t)cst * SB + VB);
    const int32_t *sb = reinterpret_cast<const int32_t *>(buf + (size_t)cst * SB + VB + CB);
    V vv[KC];
    int32_t cc[KC];
#pragma unroll
    for (int k = 0; k < KC; k++) {
      if (k < kc) {
        vv[k] = sv[k * 32 + lane];
        if (C16) cc[k] = sb[k] + (int32_t)sc[k * 32 + lane];
        else cc[k] = (int32_t)sc[k * 32 + lane];
      }
    }
    // the chunk is in registers: release the stage to the copy engine now
    __syncwarp();
    inflight--;
    cst = (cst + 1 == STAGES) ? 0 : cst + 1;
    fetch();
    Acc xv[KC];
#pragma unroll
    for (int k = 0; k < KC; k++)
      if (k < kc) xv[k] = to_acc<Acc>(__ldg(x + cc[k]));
#pragma unroll
    for (int k = 0; k < KC; k++)
      if (k < kc) acc = fmaT(to_acc<Acc>(vv[k]), xv[k], acc);
    ck += kc;
    if (ck >= w) {
      if (live) epi.row(r, acc, pre, dots);
      acc = 0;
      ck = 0;
      cs += TW;
    }
  }
  if (!ok) {
    if (lane == 0) atomicExch(err, (int)DEV_TIMEOUT_SPMV);
    // let the copies still in flight into this warp's buffers land (bounded)
    for (int i = 0; i < inflight; i++) {
      mbar_wait_bounded(&bars[cst], (phase >> cst) & 1u);
      phase ^= 1u << cst;
      cst = (cst + 1 == STAGES) ? 0 : cst + 1;
    }
  }
  epi.template finish<WARPS>(dots);
}

// ---------------------------------------------------------------------------
// Epilogues.  load(r) fetches the row's own operands before the multiply-add
// chain; row(r, acc, pre, dots) finishes the row (r is the storage row, < n);
// finish(dots) runs once per thread after the slice loop (grid reductions).
// ---------------------------------------------------------------------------
struct NoPre {};

__device__ __forceinline__ int64_t out_row(const int32_t *perm, int64_t r) { return perm ? perm[r] : r; }

// y = A x
template <typename Out> struct EpiStore {
  using Red = float;
  using Pre = NoPre;
  static constexpr int NV = 0;
  Out *y;
  const int32_t *perm;
  __device__ __forceinline__ Pre load(int64_t) const { return {}; }
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, Acc acc, const Pre &, Red (&)[1]) const {
    y[out_row(perm, r)] = cvt<Out>(acc);
  }
  template <int W> __device__ __forceinline__ void finish(Red (&)[1]) const {}
};

// y = b - A x (subtraction in the accumulator type)
template <typename B, typename Out> struct EpiResidual {
  using Red = float;
  struct Pre {
    B b;
  };
  static constexpr int NV = 0;
  const B *b;
  Out *y;
  const int32_t *perm;
  __device__ __forceinline__ Pre load(int64_t r) const { return {b[out_row(perm, r)]}; }
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, Acc acc, const Pre &p, Red (&)[1]) const {
    y[out_row(perm, r)] = cvt<Out>(to_acc<Acc>(p.b) - acc);
  }
  template <int W> __device__ __forceinline__ void finish(Red (&)[1]) const {}
};

}  // namespace f3r
