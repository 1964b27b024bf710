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

#include <type_traits>

#include "device.cuh"

namespace f3r {

// Column indices come in one of four forms:
//  * col:   int32 per entry;
//  * dcol + cbase: a uint16 offset per entry from an int32 base per slice
//    column, used when every slice column's indices fit in a 65536 window --
//    2 + 4/32 bytes per entry instead of 4.  The bases of slice s start at
//    cbptr[s], a multiple of 4, so a chunk's bases are one 16-byte aligned
//    bulk copy like its values and offsets.
//  * offset-aligned: in a slice whose rows share a small set of column
//    offsets d = column - row (a stencil, a banded or block-structured
//    matrix), slice column k holds every row's entry at offset D_k, so its
//    column is cbase[k] + lane with cbase[k] = first row + D_k; rows without
//    that offset hold a zero there.  Such a slice stores no index at all,
//    4/32 bytes per entry.  In the mixed form (xoff set) a slice that does
//    not fit, or whose columns base + lane would leave [0, ncols), keeps
//    explicit int32 indices in col from entry xoff[s] (xoff[s] < 0 marks an
//    aligned slice); chunks of kAlignedChunk columns.
//  * fully aligned (cbase set, no xoff, no dcol): every slice is aligned,
//    chunks of kAllAlignedChunk columns.  Bit 0 of cbptr[s] flags a slice
//    whose columns base + lane can leave [0, ncols) -- only zero entries of
//    the matrix's first and last rows do -- and the kernel clamps those.
//  In both aligned forms the values of a chunk are stored lane-major (a lane's
//  values contiguous) and slice widths are padded to a multiple of 4, so a
//  lane reads 4 values with one vector load; explicit indices stay
//  column-major (entry (k, lane) at k * 32 + lane of the slice).
struct DevSell {
  const int32_t *col;     // explicit indices (packed layout, or the mixed form's explicit slices)
  const uint16_t *dcol;   // (sptr[nslices]) * 32, or nullptr
  const int32_t *cbase;   // per slice column: 16-bit bases, or aligned bases
  const int32_t *cbptr;   // nslices + 1 (aligned forms: slice s's bases start at cbptr[s] & ~3)
  const int32_t *xoff;    // nslices, mixed aligned form only
  const int32_t *sptr;    // nslices + 1, in units of 32 entries
  const int32_t *perm;    // storage row -> output row, or nullptr (identity)
  int32_t n;              // rows (outputs written only for storage rows < n)
  int32_t ncols;
  int32_t nslices;
  const int32_t *rptr;    // CSR storage: row pointers (col holds the CSR indices), else nullptr
  int32_t height;         // slice height: 32, or 64 (64-row aligned slices, k_sell64)
};

// Index form of a kernel instantiation.
struct AlignedIdx {};     // mixed offset-aligned / explicit slices
struct AllAlignedIdx {};  // every slice offset-aligned
template <typename CI> struct IdxForm {
  static constexpr int mode = 0;                // explicit int32
  static constexpr uint32_t bytes = 4;          // stored index bytes per entry in a stage
};
template <> struct IdxForm<uint16_t> {
  static constexpr int mode = 1;
  static constexpr uint32_t bytes = 2;
};
template <> struct IdxForm<AlignedIdx> {
  static constexpr int mode = 2;
  static constexpr uint32_t bytes = 4;          // room for an explicit slice's chunk
};
template <> struct IdxForm<AllAlignedIdx> {
  static constexpr int mode = 3;
  static constexpr uint32_t bytes = 0;          // no index in a stage
};
// Chunk widths of the aligned forms' lane-major value layouts (the builder
// and the kernel's KC must agree).
constexpr int kAlignedChunk = 16;
constexpr int kAllAlignedChunk = 32;

// 4 consecutive values of one lane (aligned forms), one or two vector loads
template <typename V> struct Vec4Load;
template <> struct Vec4Load<__half> {
  static __device__ __forceinline__ void ld(const __half *p, __half (&o)[4]) {
    const uint2 u = *reinterpret_cast<const uint2 *>(p);
    const __half2 a = *reinterpret_cast<const __half2 *>(&u.x), b = *reinterpret_cast<const __half2 *>(&u.y);
    o[0] = __low2half(a); o[1] = __high2half(a); o[2] = __low2half(b); o[3] = __high2half(b);
  }
};
template <> struct Vec4Load<float> {
  static __device__ __forceinline__ void ld(const float *p, float (&o)[4]) {
    const float4 u = *reinterpret_cast<const float4 *>(p);
    o[0] = u.x; o[1] = u.y; o[2] = u.z; o[3] = u.w;
  }
};
template <> struct Vec4Load<double> {
  static __device__ __forceinline__ void ld(const double *p, double (&o)[4]) {
    const double2 a = *reinterpret_cast<const double2 *>(p), b = *reinterpret_cast<const double2 *>(p + 2);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
  }
};

// Launch shape per value type and index form: WARPS warps per CTA, STAGES
// buffers per warp, KC columns per chunk; one CTA per SM.  Chosen by sweeps
// (f3r_sell_tune) on the 192^3 27-point matrix (n = 7.08M, nnz = 189M).  The
// packed forms are bound by the bytes in flight per SM; the fully aligned
// form streams 2 bytes per fp16 entry and is bound by the latency of its
// gathers: a 32-column chunk worked in pipelined sub-blocks fits 80 registers
// at 24 warps (fp16); fp32 is fastest at 16 warps with 16-column sub-blocks.
template <typename V, typename CI = int32_t> struct SellCfg;
template <typename CI> struct SellCfg<__half, CI> { static constexpr int WARPS = 24, STAGES = 2, KC = 16; };
template <typename CI> struct SellCfg<float, CI> { static constexpr int WARPS = 24, STAGES = 2, KC = 16; };
template <typename CI> struct SellCfg<double, CI> { static constexpr int WARPS = 16, STAGES = 2, KC = 16; };
template <> struct SellCfg<__half, AllAlignedIdx> { static constexpr int WARPS = 32, STAGES = 2, KC = 32; };
// fp32, fully aligned: one stage a warp, 32 warps (151 us at 192^3 against 161 us at 24 x 2)
template <> struct SellCfg<float, AllAlignedIdx> { static constexpr int WARPS = 32, STAGES = 1, KC = 32; };
template <> struct SellCfg<double, AllAlignedIdx> { static constexpr int WARPS = 12, STAGES = 2, KC = 32; };

template <typename V, typename CI, int WARPS, int STAGES, int KC>
constexpr size_t sell_smem_bytes_cfg() {
  return (size_t)WARPS * STAGES *
             ((size_t)KC * 32 * (sizeof(V) + IdxForm<CI>::bytes) + (IdxForm<CI>::mode != 0 ? KC * 4 : 0)) +
         (size_t)WARPS * STAGES * sizeof(uint64_t);
}
template <typename V, typename CI>
constexpr size_t sell_smem_bytes() {
  return sell_smem_bytes_cfg<V, CI, SellCfg<V, CI>::WARPS, SellCfg<V, CI>::STAGES, SellCfg<V, CI>::KC>();
}

// CI: the index form -- int32_t (col), uint16_t (dcol + cbase), AlignedIdx
// (cbase for aligned slices, col from xoff for the others) or AllAlignedIdx.
template <typename V, typename X, typename Epi, int WARPS, int STAGES, int KC, typename CI = int32_t>
__global__ void __launch_bounds__(WARPS * 32, 1)
    k_sell_cfg(const V *__restrict__ val, DevSell A, const X *__restrict__ x, Epi epi, int *err) {
  epi_setup(epi, 0);
  using Acc = typename acc_of<V>::type;
  // gathered x kept as fp16 where value and x are both fp16 (the mixed-precision FMA takes them)
  using XB = typename std::conditional<std::is_same<V, __half>::value && std::is_same<X, __half>::value, __half,
                                       Acc>::type;
  constexpr int MODE = IdxForm<CI>::mode;
  constexpr bool C16 = MODE == 1;
  using SI = typename std::conditional<C16, uint16_t, int32_t>::type;  // stored index type
  static_assert(KC % 4 == 0, "chunk width must keep the bases 16-byte aligned");
  static_assert(MODE != 2 || KC == kAlignedChunk, "aligned layout is built for kAlignedChunk columns");
  static_assert(MODE != 3 || KC == kAllAlignedChunk, "fully aligned layout is built for kAllAlignedChunk columns");
  constexpr uint32_t VB = KC * 32 * sizeof(V), CB = KC * 32 * IdxForm<CI>::bytes, BB = MODE != 0 ? KC * 4 : 0,
                     SB = VB + CB + BB;
  const SI *cidx = C16 ? reinterpret_cast<const SI *>(A.dcol) : reinterpret_cast<const SI *>(A.col);
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

  // fetch cursor (warp-uniform); the current slice's metadata is read once,
  // when the cursor enters it
  int fs = blockIdx.x * WARPS + warp, fk = 0, fst = 0, inflight = 0;
  int fs0 = 0, fw = 0, fxo = 0, fcb = 0;
  auto fetch = [&]() {
    while (inflight < STAGES && fs < A.nslices) {
      if (fk == 0) {
        fs0 = A.sptr[fs];
        fw = A.sptr[fs + 1] - fs0;
        if (MODE == 2) fxo = A.xoff[fs];
        if (MODE != 0) fcb = A.cbptr[fs] & ~3;
      }
      if (fw == 0) {
        fs += TW;
        fk = 0;
        continue;
      }
      const int kc = min(KC, fw - fk);
      if (lane == 0) {
        const size_t off = ((size_t)fs0 + fk) * 32;
        // aligned forms: a slice carries either bases (aligned) or explicit indices
        const bool want_idx = MODE == 0 || MODE == 1 || (MODE == 2 && fxo >= 0);
        const bool want_base = MODE == 1 || MODE == 3 || (MODE == 2 && fxo < 0);
        const SI *isrc = MODE == 2 ? cidx + (size_t)fxo + (size_t)fk * 32 : cidx + off;
        fence_proxy_async_smem();
        const uint32_t ib = want_idx ? (uint32_t)kc * 32u * (uint32_t)sizeof(SI) : 0u;
        const uint32_t bb = want_base ? (uint32_t)((kc + 3) & ~3) * 4u : 0u;
        mbar_arrive_expect_tx(&bars[fst], (uint32_t)kc * 32u * (uint32_t)sizeof(V) + ib + bb);
        bulk_g2s(buf + (size_t)fst * SB, val + off, (uint32_t)kc * 32u * (uint32_t)sizeof(V), &bars[fst], pol);
        if (want_idx) bulk_g2s(buf + (size_t)fst * SB + VB, isrc, ib, &bars[fst], pol);
        if (want_base) bulk_g2s(buf + (size_t)fst * SB + VB + CB, A.cbase + fcb + fk, bb, &bars[fst], pol);
      }
      fst = (fst + 1 == STAGES) ? 0 : fst + 1;
      inflight++;
      fk += kc;
      if (fk >= fw) {
        fk = 0;
        fs += TW;
      }
    }
  };
  // hands the stage just read back to the copy engine and refills the ring
  auto release = [&]() {
    __syncwarp();
    inflight--;
    fetch();
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
  int w = 0;                  // width of the consumer's current slice
  bool aligned = MODE == 3;   // the current slice is offset-aligned
  bool clampc = false;        // fully aligned form: its columns need clamping
  while (cs < A.nslices) {
    if (ck == 0) {
      w = A.sptr[cs + 1] - A.sptr[cs];
      if (MODE == 2) aligned = A.xoff[cs] < 0;
      if (MODE == 3) clampc = (A.cbptr[cs] & 1) != 0;
    }
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
    const SI *sc = reinterpret_cast<const SI *>(buf + (size_t)cst * SB + VB);
    const int32_t *sb = reinterpret_cast<const int32_t *>(buf + (size_t)cst * SB + VB + CB);
    cst = (cst + 1 == STAGES) ? 0 : cst + 1;  // the stage read now is released below
    const bool full = kc == KC;
    if constexpr (MODE == 3) {
      // Fully aligned: the 32-column chunk is worked in sub-blocks of SUB
      // columns, software-pipelined: the gathers of sub-block h + 1 are issued
      // before the multiply-adds of sub-block h, so two sub-blocks of loads
      // are in flight per warp.  SUB keeps the registers within the launch
      // bound (16 columns for fp16 at up to 24 warps and for fp32 / fp64 at up
      // to 16, 8 beyond).  The stage is
      // released after the last sub-block's shared-memory loads.
      constexpr int SUB = (WARPS > 24 || (sizeof(V) >= 4 && WARPS > 16)) ? 8 : 16, NS = KC / SUB;
      const V *lv = sv + lane * kc;  // lane-major values (kc a multiple of 4)
      const int nsub = (kc + SUB - 1) / SUB;
      V vb[2][SUB];
      XB xb[2][SUB];
      const X *xl = x + lane;  // this lane's column is base + lane
      auto load_sub = [&](int h, V (&v)[SUB], XB (&xg)[SUB]) {
#pragma unroll
        for (int g = 0; g < SUB / 4; g++) {
          const int k0 = h * SUB + g * 4;
          if (full || k0 < kc) {
            V t[4];
            Vec4Load<V>::ld(lv + k0, t);
            const int4 q = *reinterpret_cast<const int4 *>(sb + k0);
            const int32_t b[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int e = 0; e < 4; e++) v[g * 4 + e] = t[e];
            if (!clampc) {
#pragma unroll
              for (int e = 0; e < 4; e++) xg[g * 4 + e] = to_acc<XB>(__ldg(xl + b[e]));
            } else {
#pragma unroll
              for (int e = 0; e < 4; e++) xg[g * 4 + e] = to_acc<XB>(__ldg(x + min(max(b[e] + lane, 0), A.ncols - 1)));
            }
          }
        }
      };
      load_sub(0, vb[0], xb[0]);
      if (nsub == 1) release();
#pragma unroll
      for (int h = 0; h < NS; h++) {
        if (h < nsub) {
          if (h + 1 < NS && h + 1 < nsub) {
            load_sub(h + 1, vb[(h + 1) & 1], xb[(h + 1) & 1]);
            if (h + 2 == nsub) release();
          }
#pragma unroll
          for (int g = 0; g < SUB / 4; g++)
            if (full || h * SUB + g * 4 < kc) {
#pragma unroll
              for (int e = 0; e < 4; e++) acc = fma_vx<Acc>(vb[h & 1][g * 4 + e], xb[h & 1][g * 4 + e], acc);
            }
        }
      }
    } else {
      V vv[KC];
      int32_t cc[KC];
      // Straight-line code for a full chunk, guarded code for a slice's last,
      // partial one; the index form is decided once per chunk, outside the
      // unrolled loops (warp-uniform).
      if constexpr (MODE == 2) {
        const V *lv = sv + lane * kc;  // lane-major values (kc a multiple of 4)
#pragma unroll
        for (int g = 0; g < KC / 4; g++) {
          if (full || g * 4 < kc) {
            V t[4];
            Vec4Load<V>::ld(lv + g * 4, t);
            int32_t b[4];
            if (aligned) {
              const int4 q = *reinterpret_cast<const int4 *>(sb + g * 4);
              b[0] = q.x + lane; b[1] = q.y + lane; b[2] = q.z + lane; b[3] = q.w + lane;
            } else {
#pragma unroll
              for (int e = 0; e < 4; e++) b[e] = (int32_t)sc[(g * 4 + e) * 32 + lane];
            }
#pragma unroll
            for (int e = 0; e < 4; e++) {
              vv[g * 4 + e] = t[e];
              cc[g * 4 + e] = b[e];
            }
          }
        }
      } else if (full) {
#pragma unroll
        for (int k = 0; k < KC; k++) {
          vv[k] = sv[k * 32 + lane];
          cc[k] = C16 ? sb[k] + (int32_t)sc[k * 32 + lane] : (int32_t)sc[k * 32 + lane];
        }
      } else {
#pragma unroll
        for (int k = 0; k < KC; k++)
          if (k < kc) {
            vv[k] = sv[k * 32 + lane];
            cc[k] = C16 ? sb[k] + (int32_t)sc[k * 32 + lane] : (int32_t)sc[k * 32 + lane];
          }
      }
      // the chunk is in registers: release the stage to the copy engine now
      release();
      XB xv[KC];
      if (full) {
#pragma unroll
        for (int k = 0; k < KC; k++) xv[k] = to_acc<XB>(__ldg(x + cc[k]));
#pragma unroll
        for (int k = 0; k < KC; k++) acc = fma_vx<Acc>(vv[k], xv[k], acc);
      } else {
#pragma unroll
        for (int k = 0; k < KC; k++)
          if (k < kc) xv[k] = to_acc<XB>(__ldg(x + cc[k]));
#pragma unroll
        for (int k = 0; k < KC; k++)
          if (k < kc) acc = fma_vx<Acc>(vv[k], xv[k], acc);
      }
    }
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
// 64-row offset-aligned slices (slice height 64, f3r_params.sell_c = 64).
// Every slice is offset-aligned (the fully aligned form): slot k of slice s
// holds, for each of its 64 rows, the entry at column offset D_k, its column
// cbase[k] + row-in-slice; a chunk of up to kAllAlignedChunk slots stores
// each row's values contiguously (row-major over the 64 rows).  Lane l works
// rows l and l + 32 of a slice: both rows read one set of slot bases, their
// gathers share one address (the second is 32 elements further), and the
// lane keeps two independent multiply-add chains.  Sums are formed in slot
// order, the order of the 32-row aligned layout: the results are bit for bit
// those of every other layout.
// ---------------------------------------------------------------------------
template <typename V> struct Sell64Cfg;
// A stage holds a 64-row x 32-column chunk and is released as soon as the
// chunk's values and bases sit in registers, so one stage a warp keeps the
// copy engine ahead and leaves the shared memory to more warps (and to L1 for
// the x gathers).  Measured at 192^3 (f3r_sell_tune): fp16 89 us at 32 warps x
// 1 stage against 102 us at 24 x 2; fp32 130 against 155 us (24 x 1 against
// 12 x 2); fp64 267 against 355 us (12 x 1 against 6 x 2).
template <> struct Sell64Cfg<__half> { static constexpr int WARPS = 32, STAGES = 1, KC = 32; };
template <> struct Sell64Cfg<float> { static constexpr int WARPS = 24, STAGES = 1, KC = 32; };
template <> struct Sell64Cfg<double> { static constexpr int WARPS = 12, STAGES = 1, KC = 32; };

template <typename V, int WARPS, int STAGES, int KC> constexpr size_t sell64_smem_bytes_cfg() {
  return (size_t)WARPS * STAGES * ((size_t)KC * 64 * sizeof(V) + KC * 4) + (size_t)WARPS * STAGES * sizeof(uint64_t);
}
template <typename V> constexpr size_t sell64_smem_bytes() {
  return sell64_smem_bytes_cfg<V, Sell64Cfg<V>::WARPS, Sell64Cfg<V>::STAGES, Sell64Cfg<V>::KC>();
}
static_assert(sell64_smem_bytes<__half>() <= 227 * 1024 && sell64_smem_bytes<float>() <= 227 * 1024 &&
                  sell64_smem_bytes<double>() <= 227 * 1024,
              "a 64-row launch shape exceeds the shared memory of a block");

template <typename V, typename X, typename Epi, int WARPS, int STAGES, int KC>
__global__ void __launch_bounds__(WARPS * 32, 1)
    k_sell64(const V *__restrict__ val, DevSell A, const X *__restrict__ x, Epi epi, int *err) {
  epi_setup(epi, 0);
  using Acc = typename acc_of<V>::type;
  static_assert(KC == kAllAlignedChunk, "64-row aligned layout is built for kAllAlignedChunk columns");
  constexpr uint32_t VB = KC * 64 * sizeof(V), BB = KC * 4, SB = VB + BB;
  // slots per pipelined sub-block: 8, or 4 where the launch leaves under ~100 registers a thread
  constexpr int SUB = ((sizeof(V) == 2 && WARPS > 20) || (sizeof(V) >= 4 && WARPS > 16)) ? 4 : 8;
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
  int fs = blockIdx.x * WARPS + warp, fk = 0, fst = 0, inflight = 0;
  int fs0 = 0, fw = 0, fcb = 0;
  auto fetch = [&]() {
    while (inflight < STAGES && fs < A.nslices) {
      if (fk == 0) {
        fs0 = A.sptr[fs];
        fw = A.sptr[fs + 1] - fs0;
        fcb = A.cbptr[fs] & ~3;
      }
      if (fw == 0) {
        fs += TW;
        fk = 0;
        continue;
      }
      const int kc = min(KC, fw - fk);
      if (lane == 0) {
        const size_t off = ((size_t)fs0 + fk) * 64;
        fence_proxy_async_smem();
        const uint32_t vb = (uint32_t)kc * 64u * (uint32_t)sizeof(V), bb = (uint32_t)((kc + 3) & ~3) * 4u;
        mbar_arrive_expect_tx(&bars[fst], vb + bb);
        bulk_g2s(buf + (size_t)fst * SB, val + off, vb, &bars[fst], pol);
        bulk_g2s(buf + (size_t)fst * SB + VB, A.cbase + fcb + fk, bb, &bars[fst], pol);
      }
      fst = (fst + 1 == STAGES) ? 0 : fst + 1;
      inflight++;
      fk += kc;
      if (fk >= fw) {
        fk = 0;
        fs += TW;
      }
    }
  };
  auto release = [&]() {
    __syncwarp();
    inflight--;
    fetch();
  };
  fetch();

  typename Epi::Red dots[Epi::NV > 0 ? Epi::NV : 1];
#pragma unroll
  for (int k = 0; k < (Epi::NV > 0 ? Epi::NV : 1); k++) dots[k] = 0;
  int cs = blockIdx.x * WARPS + warp, ck = 0, cst = 0;
  uint32_t phase = 0;
  bool ok = true;
  Acc acc0 = 0, acc1 = 0;
  typename Epi::Pre pre0{}, pre1{};
  int w = 0;
  bool clampc = false;
  const X *xl = x + lane;
  while (cs < A.nslices) {
    if (ck == 0) {
      w = A.sptr[cs + 1] - A.sptr[cs];
      clampc = (A.cbptr[cs] & 1) != 0;
    }
    const int64_t r0 = (int64_t)cs * 64 + lane, r1 = r0 + 32;
    const bool live0 = r0 < A.n, live1 = r1 < A.n;
    if (w == 0) {
      if (live0) {
        pre0 = epi.load(r0);
        epi.row(r0, Acc(0), pre0, dots);
      }
      if (live1) {
        pre1 = epi.load(r1);
        epi.row(r1, Acc(0), pre1, dots);
      }
      cs += TW;
      continue;
    }
    if (ck == 0) {  // epilogue operands, ahead of the chains
      if (live0) pre0 = epi.load(r0);
      if (live1) pre1 = epi.load(r1);
    }
    const int kc = min(KC, w - ck);
    if (!mbar_wait_bounded(&bars[cst], (phase >> cst) & 1u)) {
      ok = false;
      break;
    }
    phase ^= 1u << cst;
    const V *sv = reinterpret_cast<const V *>(buf + (size_t)cst * SB);
    const int32_t *sb = reinterpret_cast<const int32_t *>(buf + (size_t)cst * SB + VB);
    cst = (cst + 1 == STAGES) ? 0 : cst + 1;
    const bool full = kc == KC;
    const V *lv0 = sv + lane * kc, *lv1 = sv + (lane + 32) * kc;  // the two rows' values (kc a multiple of 4)
    const int nsub = (kc + SUB - 1) / SUB;
    constexpr int NS = KC / SUB;
    // gathered x: kept as fp16 where value and x are both fp16 (the mixed FMA takes them), else widened
    using XB = typename std::conditional<std::is_same<V, __half>::value && std::is_same<X, __half>::value, __half,
                                         Acc>::type;
    V vb0[2][SUB], vb1[2][SUB];
    XB xb0[2][SUB], xb1[2][SUB];
    auto load_sub = [&](int h, V (&v0)[SUB], V (&v1)[SUB], XB (&g0)[SUB], XB (&g1)[SUB]) {
#pragma unroll
      for (int g = 0; g < SUB / 4; g++) {
        const int k0 = h * SUB + g * 4;
        if (full || k0 < kc) {
          V t0[4], t1[4];
          Vec4Load<V>::ld(lv0 + k0, t0);
          Vec4Load<V>::ld(lv1 + k0, t1);
          const int4 q = *reinterpret_cast<const int4 *>(sb + k0);
          const int32_t b[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
          for (int e = 0; e < 4; e++) {
            v0[g * 4 + e] = t0[e];
            v1[g * 4 + e] = t1[e];
          }
          if (!clampc) {
#pragma unroll
            for (int e = 0; e < 4; e++) {
              const X *px = xl + b[e];
              g0[g * 4 + e] = to_acc<XB>(__ldg(px));
              g1[g * 4 + e] = to_acc<XB>(__ldg(px + 32));
            }
          } else {
#pragma unroll
            for (int e = 0; e < 4; e++) {
              g0[g * 4 + e] = to_acc<XB>(__ldg(x + min(max(b[e] + lane, 0), A.ncols - 1)));
              g1[g * 4 + e] = to_acc<XB>(__ldg(x + min(max(b[e] + lane + 32, 0), A.ncols - 1)));
            }
          }
        }
      }
    };
    load_sub(0, vb0[0], vb1[0], xb0[0], xb1[0]);
    if (nsub == 1) release();
#pragma unroll
    for (int h = 0; h < NS; h++) {
      if (h < nsub) {
        if (h + 1 < NS && h + 1 < nsub) {
          load_sub(h + 1, vb0[(h + 1) & 1], vb1[(h + 1) & 1], xb0[(h + 1) & 1], xb1[(h + 1) & 1]);
          if (h + 2 == nsub) release();
        }
#pragma unroll
        for (int g = 0; g < SUB / 4; g++)
          if (full || h * SUB + g * 4 < kc) {
#pragma unroll
            for (int e = 0; e < 4; e++) {
              acc0 = fma_vx<Acc>(vb0[h & 1][g * 4 + e], xb0[h & 1][g * 4 + e], acc0);
              acc1 = fma_vx<Acc>(vb1[h & 1][g * 4 + e], xb1[h & 1][g * 4 + e], acc1);
            }
          }
      }
    }
    ck += kc;
    if (ck >= w) {
      if (live0) epi.row(r0, acc0, pre0, dots);
      if (live1) epi.row(r1, acc1, pre1, dots);
      acc0 = 0;
      acc1 = 0;
      ck = 0;
      cs += TW;
    }
  }
  if (!ok) {
    if (lane == 0) atomicExch(err, (int)DEV_TIMEOUT_SPMV);
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
