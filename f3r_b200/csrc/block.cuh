// block.cuh -- K right-hand sides at once: the SELL product of K vectors
// (block SpMM), and the Gram-Schmidt, Givens, Richardson and level kernels of
// the nested solver over K columns.
//
// A block vector holds K columns interleaved by row, v[row * K + c], so the
// K values a matrix entry multiplies are one contiguous 8..64-byte run: one
// gather instruction feeds several columns, and the matrix (values and
// slice metadata) is streamed once for all K.
//
// Every reduction kernel here splits rows over threads exactly as the
// single-column kernel it generalises does (same grid, same rows per thread
// and order, same warp / block / grid summation tree), and every product sums
// a row in stored column order: column c of a K-column solve is therefore the
// single-column solve of that right-hand side, bit for bit.  `active` is a
// device word with bit c set for the columns still iterating; columns whose
// bit is clear are finished (their results are final and no longer written
// where that matters: Givens breakdown flags, the outer update x += Z y).
#pragma once

#include "kernels.cuh"

namespace f3r {

constexpr int kMaxBlock = 16;  // widest block of right-hand sides
// The single-column (K = 1) BLAS-1 kernels launch 8 blocks of 256 threads per
// SM (Context::ew_grid) and declare so (__launch_bounds__(256, 8), at most 32
// registers a thread), so that the whole grid is resident in one wave.

// a VecN (an aggregate of at most 16 bytes) through the read-only path
template <typename T, int N> __device__ __forceinline__ VecN<T, N> ldg_vec(const VecN<T, N> *p) {
  if constexpr (sizeof(VecN<T, N>) == 16) {
    const int4 u = ::__ldg(reinterpret_cast<const int4 *>(p));
    return *reinterpret_cast<const VecN<T, N> *>(&u);
  } else if constexpr (sizeof(VecN<T, N>) == 8) {
    const int2 u = ::__ldg(reinterpret_cast<const int2 *>(p));
    return *reinterpret_cast<const VecN<T, N> *>(&u);
  } else if constexpr (sizeof(VecN<T, N>) == 4) {
    const int u = ::__ldg(reinterpret_cast<const int *>(p));
    return *reinterpret_cast<const VecN<T, N> *>(&u);
  } else {
    const short u = ::__ldg(reinterpret_cast<const short *>(p));
    return *reinterpret_cast<const VecN<T, N> *>(&u);
  }
}

// 32 contiguous bytes (32-byte aligned) in one 256-bit access (sm_100's
// ld / st .v8.b32): a lane's access then fills a whole 32-byte sector, where
// two 16-byte accesses per lane fill half of each sector they touch
__device__ __forceinline__ void ld32_nc(const void *p, uint32_t (&u)[8]) {
  asm volatile("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7])
               : "l"(p));
}
__device__ __forceinline__ void ld32(const void *p, uint32_t (&u)[8]) {
  asm volatile("ld.global.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7])
               : "l"(p)
               : "memory");
}
__device__ __forceinline__ void st32(void *p, const uint32_t (&u)[8]) {
  asm volatile("st.global.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "r"(u[0]), "r"(u[1]), "r"(u[2]),
               "r"(u[3]), "r"(u[4]), "r"(u[5]), "r"(u[6]), "r"(u[7])
               : "memory");
}

// ---------------------------------------------------------------------------
// K contiguous values of one row in global memory: 32-byte accesses where
// the row is a multiple of 32 bytes (rows of a block vector start on 32-byte
// boundaries: every vector this library allocates is 64-byte aligned), else
// 16-byte ones where K allows.  load_any takes any address space (the stage
// buffers in shared memory).
// ---------------------------------------------------------------------------
template <typename T, int K> struct RowK {
  static constexpr int BYTES = (int)sizeof(T) * K;
  static constexpr bool WIDE = BYTES % 32 == 0;                 // 32-byte accesses
  static constexpr int W = 32 / (int)sizeof(T);                 // elements per 32-byte access
  static constexpr int VEC = BYTES >= 16 ? 16 / (int)sizeof(T) : K;  // elements per access otherwise
  template <typename Acc> static __device__ __forceinline__ void load_any(const T *p, Acc (&o)[K]) {
#pragma unroll
    for (int q = 0; q < K / VEC; q++) {
      const VecN<T, VEC> a = *reinterpret_cast<const VecN<T, VEC> *>(p + q * VEC);
#pragma unroll
      for (int e = 0; e < VEC; e++) o[q * VEC + e] = to_acc<Acc>(a.v[e]);
    }
  }
  template <typename Acc> static __device__ __forceinline__ void load(const T *p, Acc (&o)[K]) {
    if constexpr (WIDE) {
#pragma unroll
      for (int q = 0; q < K / W; q++) {
        uint32_t u[8];
        ld32(p + q * W, u);
        const T *t = reinterpret_cast<const T *>(u);
#pragma unroll
        for (int e = 0; e < W; e++) o[q * W + e] = to_acc<Acc>(t[e]);
      }
    } else {
#pragma unroll
      for (int q = 0; q < K / VEC; q++) {
        const VecN<T, VEC> a = *reinterpret_cast<const VecN<T, VEC> *>(p + q * VEC);
#pragma unroll
        for (int e = 0; e < VEC; e++) o[q * VEC + e] = to_acc<Acc>(a.v[e]);
      }
    }
  }
  template <typename Acc> static __device__ __forceinline__ void ldg(const T *p, Acc (&o)[K]) {
    if constexpr (WIDE) {
#pragma unroll
      for (int q = 0; q < K / W; q++) {
        uint32_t u[8];
        ld32_nc(p + q * W, u);
        const T *t = reinterpret_cast<const T *>(u);
#pragma unroll
        for (int e = 0; e < W; e++) o[q * W + e] = to_acc<Acc>(t[e]);
      }
    } else {
#pragma unroll
      for (int q = 0; q < K / VEC; q++) {
        const VecN<T, VEC> a = ldg_vec(reinterpret_cast<const VecN<T, VEC> *>(p + q * VEC));
#pragma unroll
        for (int e = 0; e < VEC; e++) o[q * VEC + e] = to_acc<Acc>(a.v[e]);
      }
    }
  }
  template <typename Acc> static __device__ __forceinline__ void store(T *p, const Acc (&v)[K]) {
    if constexpr (WIDE) {
#pragma unroll
      for (int q = 0; q < K / W; q++) {
        uint32_t u[8];
        T *t = reinterpret_cast<T *>(u);
#pragma unroll
        for (int e = 0; e < W; e++) t[e] = cvt<T>(v[q * W + e]);
        st32(p + q * W, u);
      }
    } else {
#pragma unroll
      for (int q = 0; q < K / VEC; q++) {
        VecN<T, VEC> a;
#pragma unroll
        for (int e = 0; e < VEC; e++) a.v[e] = cvt<T>(v[q * VEC + e]);
        *reinterpret_cast<VecN<T, VEC> *>(p + q * VEC) = a;
      }
    }
  }
};

// N diagonal preconditioner values from p, or N ones where the diagonal is
// the identity in fp16 (DiagPre with null pointers: nothing is loaded)
template <int N, typename Acc> __device__ __forceinline__ void diag_load(const __half *p, Acc (&o)[N]) {
  if (p) {
    RowK<__half, N>::load(p, o);
  } else {
#pragma unroll
    for (int q = 0; q < N; q++) o[q] = Acc(1.0f);
  }
}

// ---------------------------------------------------------------------------
// Block SELL product: out(:, c) = A x(:, c) for c < K, one pass over A.
// Same layouts and bulk-copy ring as k_sell_cfg (sell.cuh); the index forms
// are the packed int32 one (MODE 0), the mixed offset-aligned one (MODE 2:
// aligned slices with bases, the others with explicit indices) and the fully
// offset-aligned one (MODE 3).
// Each lane owns one row of a slice and K accumulators, summing the row's
// entries in stored order with one FMA per column.
// ---------------------------------------------------------------------------
template <typename V, int K, typename CI> struct BlockCfg;
template <int K> struct BlockCfg<__half, K, int32_t> { static constexpr int WARPS = 16, STAGES = 2, KC = 16; };
template <int K> struct BlockCfg<float, K, int32_t> { static constexpr int WARPS = 16, STAGES = 2, KC = 16; };
template <int K> struct BlockCfg<double, K, int32_t> { static constexpr int WARPS = 12, STAGES = 2, KC = 16; };
template <int K> struct BlockCfg<__half, K, AllAlignedIdx> { static constexpr int WARPS = 16, STAGES = 2, KC = 32; };
template <int K> struct BlockCfg<float, K, AllAlignedIdx> { static constexpr int WARPS = 16, STAGES = 2, KC = 32; };
template <int K> struct BlockCfg<double, K, AllAlignedIdx> { static constexpr int WARPS = 12, STAGES = 2, KC = 32; };
template <int K> struct BlockCfg<__half, K, AlignedIdx> { static constexpr int WARPS = 16, STAGES = 2, KC = 16; };
template <int K> struct BlockCfg<float, K, AlignedIdx> { static constexpr int WARPS = 16, STAGES = 2, KC = 16; };
template <int K> struct BlockCfg<double, K, AlignedIdx> { static constexpr int WARPS = 12, STAGES = 2, KC = 16; };

template <typename V, int K, typename CI> constexpr size_t block_smem_bytes() {
  using Cfg = BlockCfg<V, K, CI>;
  return sell_smem_bytes_cfg<V, CI, Cfg::WARPS, Cfg::STAGES, Cfg::KC>();
}
// Systems of one pattern, each with its own values (packed int32 layout, the
// K values of an entry interleaved): chunks of at most 4 KB of values.
template <typename V, int K> struct BlockCfgMM {
  static constexpr int WARPS = sizeof(V) == 8 ? 12 : 16, STAGES = 2;
  static constexpr int KC0 = 4096 / (32 * K * (int)sizeof(V));
  static constexpr int KC = KC0 < 1 ? 1 : KC0 > 16 ? 16 : KC0;
};
template <typename V, int K> constexpr size_t block_mm_smem_bytes() {
  using Cfg = BlockCfgMM<V, K>;
  return (size_t)Cfg::WARPS * Cfg::STAGES * ((size_t)Cfg::KC * 32 * (K * sizeof(V) + 4)) +
         (size_t)Cfg::WARPS * Cfg::STAGES * sizeof(uint64_t);
}

// MM: every column has its own matrix values (systems of one pattern); the
// K values of an entry are contiguous, val[position * K + c].
template <typename V, typename X, typename Epi, int K, int WARPS, int STAGES, int KC, typename CI, bool MM = false>
__global__ void __launch_bounds__(WARPS * 32, 1)
    k_sell_block(const V *__restrict__ val, DevSell A, const X *__restrict__ x, Epi epi, int *err) {
  epi_setup(epi, 0);
  using Acc = typename acc_of<V>::type;
  constexpr int MODE = IdxForm<CI>::mode;
  static_assert(MODE == 0 || MODE == 2 || MODE == 3, "block product: packed int32 or offset-aligned slices");
  static_assert(!MM || MODE == 0, "per-column values: packed int32 layout");
  static_assert(MODE != 3 || KC == kAllAlignedChunk, "fully aligned layout is built for kAllAlignedChunk columns");
  static_assert(MODE != 2 || KC == kAlignedChunk, "aligned layout is built for kAlignedChunk columns");
  constexpr int VK = MM ? K : 1;  // values per entry
  constexpr uint32_t VB = KC * 32 * sizeof(V) * VK, CB = KC * 32 * IdxForm<CI>::bytes, BB = MODE != 0 ? KC * 4 : 0,
                     SB = VB + CB + BB;
  // entries gathered per sub-block: about 32 gathered fp32 values (16 fp64) per lane
  constexpr int SUB0 = (sizeof(Acc) == 8 ? 16 : 32) / (K * (MM ? 2 : 1));
  constexpr int SUB = SUB0 > 0 ? SUB0 : 1;
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
  int fs0 = 0, fw = 0, fcb = 0, fxo = 0;
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
        fence_proxy_async_smem();
        // mixed form: a slice carries either bases (aligned) or explicit indices (from xoff)
        const bool want_idx = MODE == 0 || (MODE == 2 && fxo >= 0);
        const bool want_base = MODE == 3 || (MODE == 2 && fxo < 0);
        const uint32_t ib = want_idx ? (uint32_t)kc * 32u * 4u : 0u;
        const uint32_t bb = want_base ? (uint32_t)((kc + 3) & ~3) * 4u : 0u;
        const uint32_t vb = (uint32_t)kc * 32u * (uint32_t)sizeof(V) * (uint32_t)VK;
        const int32_t *isrc = MODE == 2 ? A.col + (size_t)fxo + (size_t)fk * 32 : A.col + off;
        mbar_arrive_expect_tx(&bars[fst], vb + ib + bb);
        bulk_g2s(buf + (size_t)fst * SB, val + off * VK, vb, &bars[fst], pol);
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
  auto release = [&]() {
    __syncwarp();
    inflight--;
    fetch();
  };
  fetch();

  int cs = blockIdx.x * WARPS + warp, ck = 0, cst = 0;
  uint32_t phase = 0;
  bool ok = true;
  Acc acc[K];
#pragma unroll
  for (int c = 0; c < K; c++) acc[c] = 0;
  int w = 0;
  bool clampc = false;
  bool aligned = MODE == 3;  // the current slice is offset-aligned
  while (cs < A.nslices) {
    if (ck == 0) {
      w = A.sptr[cs + 1] - A.sptr[cs];
      if (MODE == 2) aligned = A.xoff[cs] < 0;
      if (MODE == 3) clampc = (A.cbptr[cs] & 1) != 0;
    }
    const int64_t r = (int64_t)cs * 32 + lane;
    const bool live = r < A.n;
    if (w == 0) {
      if (live) epi.row(r, acc);
      cs += TW;
      continue;
    }
    const int kc = min(KC, w - ck);
    if (!mbar_wait_bounded(&bars[cst], (phase >> cst) & 1u)) {
      ok = false;
      break;
    }
    phase ^= 1u << cst;
    const V *sv = reinterpret_cast<const V *>(buf + (size_t)cst * SB);
    const int32_t *sc = reinterpret_cast<const int32_t *>(buf + (size_t)cst * SB + VB);
    const int32_t *sb = reinterpret_cast<const int32_t *>(buf + (size_t)cst * SB + VB + CB);
    cst = (cst + 1 == STAGES) ? 0 : cst + 1;
    // the chunk is worked in sub-blocks of SUB entries: values and columns
    // first (then the stage goes back to the copy engine), then the gathers
    // of the sub-block, then its multiply-adds
    constexpr int NSUB = (KC + SUB - 1) / SUB;
    // fp16 values with fp16 x stay fp16 for the mixed-precision FMA, else widened
    constexpr bool H2 = std::is_same<V, __half>::value && std::is_same<X, __half>::value;
    using VB = typename std::conditional<H2, __half, Acc>::type;
    VB vv[SUB][VK];
    int32_t cc[SUB];
    const V *lv = sv + lane * kc;  // aligned form: lane-major values
    for (int h = 0; h < NSUB; h++) {
      const int k0 = h * SUB;
      if (k0 >= kc) break;
#pragma unroll
      for (int e = 0; e < SUB; e++) {
        const int k = k0 + e;
        if (k < kc) {
          if (MODE == 3 || MODE == 2) {
            vv[e][0] = to_acc<VB>(lv[k]);  // lane-major values
            if (MODE == 2 && !aligned) {
              cc[e] = sc[k * 32 + lane];
            } else {
              const int32_t b = sb[k] + lane;
              cc[e] = clampc ? min(max(b, 0), A.ncols - 1) : b;
            }
          } else {
            RowK<V, VK>::load_any(sv + ((size_t)k * 32 + lane) * VK, vv[e]);  // shared memory
            cc[e] = sc[k * 32 + lane];
          }
        }
      }
      if (k0 + SUB >= kc) release();  // last sub-block of the chunk: its shared data is in registers
      VB xg[SUB][K];
#pragma unroll
      for (int e = 0; e < SUB; e++)
        if (k0 + e < kc) RowK<X, K>::ldg(x + (size_t)cc[e] * K, xg[e]);
#pragma unroll
      for (int e = 0; e < SUB; e++)
        if (k0 + e < kc) {
#pragma unroll
          for (int c = 0; c < K; c++) acc[c] = fma_vx<Acc>(vv[e][MM ? c : 0], xg[e][c], acc[c]);
        }
    }
    ck += kc;
    if (ck >= w) {
      if (live) epi.row(r, acc);
#pragma unroll
      for (int c = 0; c < K; c++) acc[c] = 0;
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
}

// ---------------------------------------------------------------------------
// Block product on 64-row offset-aligned slices (sell_c = 64): each lane owns
// rows l and l + 32 of a slice and K accumulators for each, summing every
// row's entries in slot (column) order with one FMA per column, as the
// 32-row kernels do, so the sums are theirs bit for bit.  A chunk of up to 32
// slots holds 64 rows of values, row after row, and one base per slot; the
// two rows of a lane gather x at base + lane and base + lane + 32.
// ---------------------------------------------------------------------------
// one stage a warp (released once its chunk is in registers), the warps the
// registers allow: K accumulators for each of a lane's two rows
template <typename V, int K> constexpr int block64_warps() { return sizeof(V) == 2 ? 16 : sizeof(V) == 4 ? 12 : 8; }
template <typename V, int K> constexpr int block64_stages() { return 1; }
template <typename V, int K> constexpr size_t block64_smem_bytes() {
  constexpr size_t ws = (size_t)block64_warps<V, K>() * block64_stages<V, K>();
  return ws * ((size_t)kAllAlignedChunk * 64 * sizeof(V) + kAllAlignedChunk * 4) + ws * sizeof(uint64_t);
}

template <typename V, typename X, typename Epi, int K, int WARPS, int STAGES>
__global__ void __launch_bounds__(WARPS * 32, 1)
    k_sell_block64(const V *__restrict__ val, DevSell A, const X *__restrict__ x, Epi epi, int *err) {
  epi_setup(epi, 0);
  using Acc = typename acc_of<V>::type;
  constexpr int KC = kAllAlignedChunk;
  constexpr uint32_t VB = KC * 64 * sizeof(V), BB = KC * 4, SB = VB + BB;
  // slots gathered per sub-block: about 32 gathered fp32 values (16 fp64) per lane over its two rows
  constexpr int SUB0 = (sizeof(Acc) == 8 ? 16 : 32) / (2 * K);
  constexpr int SUB = SUB0 > 0 ? SUB0 : 1;
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

  int cs = blockIdx.x * WARPS + warp, ck = 0, cst = 0;
  uint32_t phase = 0;
  bool ok = true;
  Acc acc0[K], acc1[K];
#pragma unroll
  for (int c = 0; c < K; c++) acc0[c] = acc1[c] = 0;
  int w = 0;
  bool clampc = false;
  while (cs < A.nslices) {
    if (ck == 0) {
      w = A.sptr[cs + 1] - A.sptr[cs];
      clampc = (A.cbptr[cs] & 1) != 0;
    }
    const int64_t r0 = (int64_t)cs * 64 + lane, r1 = r0 + 32;
    if (w == 0) {
      if (r0 < A.n) epi.row(r0, acc0);
      if (r1 < A.n) epi.row(r1, acc1);
      cs += TW;
      continue;
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
    const V *lv0 = sv + lane * kc, *lv1 = sv + (lane + 32) * kc;  // the two rows' values
    // fp16 values with fp16 x stay fp16 for the mixed-precision FMA, else widened
    constexpr bool H2 = std::is_same<V, __half>::value && std::is_same<X, __half>::value;
    using VB = typename std::conditional<H2, __half, Acc>::type;
    for (int k0 = 0; k0 < kc; k0 += SUB) {
      VB v0[SUB], v1[SUB];
      int32_t c0[SUB], c1[SUB];
#pragma unroll
      for (int e = 0; e < SUB; e++) {
        const int k = k0 + e;
        if (k < kc) {
          v0[e] = to_acc<VB>(lv0[k]);
          v1[e] = to_acc<VB>(lv1[k]);
          const int32_t b = sb[k] + lane;
          c0[e] = clampc ? min(max(b, 0), A.ncols - 1) : b;
          c1[e] = clampc ? min(max(b + 32, 0), A.ncols - 1) : b + 32;
        }
      }
      if (k0 + SUB >= kc) release();  // last sub-block of the chunk: its shared data is in registers
      VB x0[SUB][K], x1[SUB][K];
#pragma unroll
      for (int e = 0; e < SUB; e++)
        if (k0 + e < kc) {
          RowK<X, K>::ldg(x + (size_t)c0[e] * K, x0[e]);
          RowK<X, K>::ldg(x + (size_t)c1[e] * K, x1[e]);
        }
#pragma unroll
      for (int e = 0; e < SUB; e++)
        if (k0 + e < kc) {
#pragma unroll
          for (int c = 0; c < K; c++) {
            acc0[c] = fma_vx<Acc>(v0[e], x0[e][c], acc0[c]);
            acc1[c] = fma_vx<Acc>(v1[e], x1[e][c], acc1[c]);
          }
        }
    }
    ck += kc;
    if (ck >= w) {
      if (r0 < A.n) epi.row(r0, acc0);
      if (r1 < A.n) epi.row(r1, acc1);
#pragma unroll
      for (int c = 0; c < K; c++) acc0[c] = acc1[c] = 0;
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
}

// ---- epilogues of the block product (one row, K columns) --------------------
// y(:, c) = A x(:, c)
template <typename Out, int K> struct EpiStoreK {
  Out *y;
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, const Acc (&acc)[K]) const {
    RowK<Out, K>::store(y + r * K, acc);
  }
};
// y(:, c) = b(:, c) - A x(:, c), the subtraction in the accumulator type
template <typename B, typename Out, int K> struct EpiResidualK {
  const B *b;
  Out *y;
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, const Acc (&acc)[K]) const {
    Acc bv[K], o[K];
    RowK<B, K>::load(b + r * K, bv);
#pragma unroll
    for (int c = 0; c < K; c++) o[c] = bv[c] - acc[c];
    RowK<Out, K>::store(y + r * K, o);
  }
};

// Richardson step without a weight update, diagonal preconditioner fused
// (EpiRichStepT, kernels.cuh, per column with the column's own weight, read
// once per thread by setup()):
// hr = fp16(hin - A hout); t2 = z (w hr); hnew = fp16(hout + ome_c[k] t2); the
// last step writes out = fp32(hnew) / sc instead.
// MM: the diagonal preconditioner has one value per row and column, w[r * K + c]
template <int K, bool MM = false> struct EpiRichStepK {
  const __half *hin, *hout;
  DiagPre M;
  const RichState *rs;  // K states
  int k;
  __half *hnext;
  float *out;
  float isc;
  float ome[K] = {};  // fp32(ome_c[k]) of every column, set by setup()
  __device__ __forceinline__ void setup() {
#pragma unroll
    for (int c = 0; c < K; c++) ome[c] = h2f(rs[c].ome[k]);
  }
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, const Acc (&acc)[K]) const {
    float hi[K], ho[K], res[K];
    __half hn[K];
    __half w[MM ? K : 1], z[MM ? K : 1];
    RowK<__half, K>::load(hin + r * K, hi);
    RowK<__half, K>::load(hout + r * K, ho);
    diag_load<MM ? K : 1>(M.w ? M.w + r * (MM ? K : 1) : nullptr, w);
    diag_load<MM ? K : 1>(M.z ? M.z + r * (MM ? K : 1) : nullptr, z);
#pragma unroll
    for (int c = 0; c < K; c++) {
      const __half hr = f2h(hi[c] - (float)acc[c]);
      const __half t2 = __hmul(z[MM ? c : 0], __hmul(w[MM ? c : 0], hr));
      hn[c] = f2h(__fmaf_rn(ome[c], h2f(t2), ho[c]));  // rounded to fp16 once, stored as it is
    }
    if (out) {
#pragma unroll
      for (int c = 0; c < K; c++) res[c] = h2f(hn[c]) * isc;
      RowK<float, K>::store(out + r * K, res);
    } else {
      RowK<__half, K>::store(hnext + r * K, hn);
    }
  }
};

// Residual step of an update call (diagonal M): hr and t2 = M hr stored
template <int K, bool MM = false> struct EpiRichResPreK {
  const __half *hin;
  DiagPre M;
  __half *hr, *t2;
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, const Acc (&acc)[K]) const {
    float hi[K], h[K], t[K], w[MM ? K : 1], z[MM ? K : 1];
    RowK<__half, K>::load(hin + r * K, hi);
    diag_load<MM ? K : 1>(M.w ? M.w + r * (MM ? K : 1) : nullptr, w);
    diag_load<MM ? K : 1>(M.z ? M.z + r * (MM ? K : 1) : nullptr, z);
#pragma unroll
    for (int c = 0; c < K; c++) {
      h[c] = h2f(f2h(hi[c] - (float)acc[c]));
      t[c] = z[MM ? c : 0] * h2f(f2h(w[MM ? c : 0] * h[c]));
    }
    RowK<__half, K>::store(hr + r * K, h);
    RowK<__half, K>::store(t2 + r * K, t);
  }
};

// General M, Z apply: hout = fp16(Z tmp), then on a call without a weight
// update hout *= ome_c[0] (EpiZScale, per column)
template <int K> struct EpiZScaleK {
  __half *hout;
  const RichState *rs;
  int scale;
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, const Acc (&acc)[K]) const {
    float o[K];
#pragma unroll
    for (int c = 0; c < K; c++) {
      float h = h2f(f2h((float)acc[c]));
      if (scale) h = h2f(rs[c].ome[0]) * h;
      o[c] = h;
    }
    RowK<__half, K>::store(hout + r * K, o);
  }
};

// ---------------------------------------------------------------------------
// Reductions over K columns.  Two final stages exist, each reproducing one of
// the single-column kernels' trees exactly:
//  * "block-strided" (grid_reduce, device.cuh): each thread adds the partial
//    sums of blocks t, t + blockDim, ... ; a warp shuffle tree; thread 0 adds
//    the warps in order;
//  * "lane-strided" (k_multidot_chunked, kernels.cuh): one warp per value,
//    lanes add blocks l, l + 32, ... ; a warp shuffle tree.
// The block stage is the same in both: warp shuffle trees, then the warps of
// the block added in order.  Partial sums are laid out [block][value].
// ---------------------------------------------------------------------------

// Per-column scalars of one FGMRES level: column c's H at H + c * hs
// (column-major (m+1) x m), its cs, sn, e, y at + c * vs, its 1/h at inv[c].
template <typename T> struct LevelK {
  T *H, *cs, *sn, *e, *y, *inv;
  int64_t hs, vs;
  int ldh;  // m + 1
  __device__ __forceinline__ GivensCtl<T> col(int c, int j, int compute_y, double *abs_e, int *err) const {
    return GivensCtl<T>{H + c * hs, cs + c * vs, sn + c * vs, e + c * vs, y + c * vs, inv + c, abs_e, ldh, j,
                        compute_y, err};
  }
};

// block stage: v[q] (q < NQ, this thread's values) -> part[blockIdx.x * nq + q]
template <typename T, int NQ, int WARPS>
__device__ __forceinline__ void block_partials(T (&v)[NQ], int nq, int q0, int ntot, T *part, T (&sred)[WARPS][NQ]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    if (q < nq) {
      const T s = warp_sum(v[q]);
      if (lane == 0) sred[warp][q] = s;
    }
  }
  __syncthreads();
  if ((int)threadIdx.x < nq) {
    T s = 0;
    for (int w = 0; w < WARPS; w++) s += sred[w][threadIdx.x];
    part[(size_t)blockIdx.x * ntot + q0 + threadIdx.x] = s;
  }
  __syncthreads();
}

// true in the last block to arrive (after every block wrote its partials)
__device__ __forceinline__ bool last_block(unsigned int *ticket) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// final stage, block-strided, for nq <= QB values at once (q0 .. q0 + nq - 1
// of ntot partials per block): value q is summed by thread t over the
// partials of blocks t, t + blockDim.x, ... in that order, then by the warp
// butterfly, then over warps 0 .. WARPS-1 in order -- a fixed order for every
// column count and launch, so that the K-column kernels' sums are the single
// column's.  The values' loads and reductions overlap instead of running one
// value after another.  Value q0 + i is returned on thread i (i < nq).
template <typename T, int WARPS, int QB>
__device__ __forceinline__ T final_block_multi(const T *part, int q0, int nq, int ntot) {
  __shared__ T sw[WARPS][QB];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T s[QB];
#pragma unroll
  for (int i = 0; i < QB; i++) s[i] = 0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    const T *pb = part + (size_t)b * ntot + q0;
#pragma unroll
    for (int i = 0; i < QB; i++)
      if (i < nq) s[i] += __ldcg(pb + i);
  }
#pragma unroll
  for (int i = 0; i < QB; i++) {
    if (i < nq) {
      s[i] = warp_sum(s[i]);
      if (lane == 0) sw[warp][i] = s[i];
    }
  }
  __syncthreads();
  T t = 0;
  if ((int)threadIdx.x < nq)
    for (int w = 0; w < WARPS; w++) t += sw[w][threadIdx.x];
  __syncthreads();
  return t;
}

// <x(:, c), y(:, c)> for c < K (kmm::dot; k_dot of kernels.cuh): one element
// per thread and grid stride, block-strided final stage
template <typename T, typename Acc, int WARPS, int K>
__global__ void __launch_bounds__(WARPS * 32) k_dotK(const T *__restrict__ x, const T *__restrict__ y, int64_t n,
                                                     GridRed gr, Acc *out) {
  __shared__ Acc sred[WARPS][K];
  Acc a[K];
#pragma unroll
  for (int c = 0; c < K; c++) a[c] = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    Acc xv[K], yv[K];
    RowK<T, K>::load(x + i * K, xv);
    RowK<T, K>::load(y + i * K, yv);
#pragma unroll
    for (int c = 0; c < K; c++) a[c] = fmaT(xv[c], yv[c], a[c]);
  }
  Acc *part = static_cast<Acc *>(gr.partials);
  block_partials<Acc, K, WARPS>(a, K, 0, K, part, sred);
  if (!last_block(gr.ticket)) return;
  const Acc t = final_block_multi<Acc, WARPS, K>(part, 0, K, K);
  if ((int)threadIdx.x < K) out[threadIdx.x] = t;
  if (threadIdx.x == 0) *gr.ticket = 0;
}

// H(j, k)(c) = <w(:, c), V(k)(:, c)>, k < nv, one element per thread and
// grid stride, lane-strided final stage (k_multidot_chunked): the outer fp64
// level and inner fp32 levels with more than 8 basis vectors.  Column c's
// values go to hcol + c * hstride.
template <typename T, int WARPS, int K>
__global__ void __launch_bounds__(WARPS * 32, K == 1 ? 8 : 1) k_multidot_chunkedK(const T *__restrict__ w, Cols<T> V, int nv,
                                                                  int64_t n, GridRed gr, T *hcol, int64_t hstride) {
  constexpr int CH = K >= 8 ? 1 : 8 / K;  // basis vectors per pass over w
  constexpr int NQ = CH * K;
  __shared__ T sred[WARPS][NQ];
  T *part = static_cast<T *>(gr.partials);
  const int ntot = nv * K;
  for (int k0 = 0; k0 < nv; k0 += CH) {
    T a[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) a[q] = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      T wv[K];
      RowK<T, K>::load(w + i * K, wv);
#pragma unroll
      for (int v = 0; v < CH; v++) {
        if (k0 + v < nv) {
          T vv[K];
          RowK<T, K>::load(V.p[k0 + v] + i * K, vv);
#pragma unroll
          for (int c = 0; c < K; c++) a[v * K + c] = fmaT(wv[c], vv[c], a[v * K + c]);
        }
      }
    }
    const int nq = min(CH, nv - k0) * K;
    block_partials<T, NQ, WARPS>(a, nq, k0 * K, ntot, part, sred);
  }
  if (!last_block(gr.ticket)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int q = warp; q < ntot; q += WARPS) {
    T t = 0;
    for (int b = lane; b < (int)gridDim.x; b += 32) t += __ldcg(&part[(size_t)b * ntot + q]);
    t = warp_sum(t);
    if (lane == 0) hcol[(q % K) * hstride + q / K] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) *gr.ticket = 0;
}

// H(j, k)(c) = <w(:, c), V(k)(:, c)> for nv <= MAXV basis vectors in fp32
// (k_multidot_f32): rows in groups of 4 per thread, block-strided final stage
template <int MAXV, int WARPS, int K>
__global__ void __launch_bounds__(WARPS * 32, K == 1 ? 8 : 1) k_multidot_f32K(const float *__restrict__ w, Cols<float> V, int nv,
                                                              int64_t n, GridRed gr, float *hcol, int64_t hstride) {
  // basis vectors per pass: single columns take at most 4 (more float4 loads in flight than 32
  // registers hold spill), K columns up to 32 values
  constexpr int CV = (MAXV * K > 32) ? (32 / K > 0 ? 32 / K : 1) : (K == 1 && MAXV > 4) ? 4 : MAXV;
  constexpr int NQ = CV * K;
  __shared__ float sred[WARPS][NQ];
  float *part = static_cast<float *>(gr.partials);
  const int ntot = nv * K;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nq4 = n / 4;
  for (int k0 = 0; k0 < nv; k0 += CV) {
    float a[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) a[q] = 0.0f;
    // the 4 rows of a thread, RG at a time as one contiguous run of RG * K values
    constexpr int RG = (4 * K <= 16) ? 4 : 1, E = RG * K;
    for (int64_t q4 = tid; q4 < nq4; q4 += stride) {
#pragma unroll
      for (int g = 0; g < 4 / RG; g++) {
        const int64_t i0 = 4 * q4 + g * RG;
        float wv[E];
        RowK<float, E>::load(w + i0 * K, wv);
#pragma unroll
        for (int v = 0; v < CV; v++) {
          if (k0 + v < nv) {
            float vv[E];
            RowK<float, E>::load(V.p[k0 + v] + i0 * K, vv);
#pragma unroll
            for (int e = 0; e < E; e++) a[v * K + e % K] = __fmaf_rn(wv[e], vv[e], a[v * K + e % K]);
          }
        }
      }
    }
    for (int64_t i = nq4 * 4 + tid; i < n; i += stride) {
      float wv[K];
      RowK<float, K>::load(w + i * K, wv);
#pragma unroll
      for (int v = 0; v < CV; v++) {
        if (k0 + v < nv) {
          float vv[K];
          RowK<float, K>::load(V.p[k0 + v] + i * K, vv);
#pragma unroll
          for (int c = 0; c < K; c++) a[v * K + c] = __fmaf_rn(wv[c], vv[c], a[v * K + c]);
        }
      }
    }
    const int nq = min(CV, nv - k0) * K;
    block_partials<float, NQ, WARPS>(a, nq, k0 * K, ntot, part, sred);
  }
  if (!last_block(gr.ticket)) return;
  constexpr int QB = NQ < 16 ? NQ : 16;
  for (int q0 = 0; q0 < ntot; q0 += QB) {
    const int nq = min(QB, ntot - q0);
    const float t = final_block_multi<float, WARPS, QB>(part, q0, nq, ntot);
    const int q = q0 + (int)threadIdx.x;
    if ((int)threadIdx.x < nq) hcol[(q % K) * hstride + q / K] = t;
  }
  if (threadIdx.x == 0) *gr.ticket = 0;
}

// shared memory of k_cgs_updateK's staging tiles: per warp 32 threads x N
// rows x K values, each thread's run padded by 16 bytes (conflict-free
// 16-byte reads)
template <typename T, int WARPS, int K> constexpr size_t cgs_stage_bytes() {
  return K == 1 ? 0 : (size_t)WARPS * 32 * (16 / sizeof(T) * K + 16 / sizeof(T)) * sizeof(T);
}

// w(:, c) -= sum_k H(j, k)(c) V(k)(:, c) (MULMV order), then ||w(:, c)||^2 ->
// Givens of column c for the columns in *active (k_cgs_update): N elements
// per thread (16 bytes of one column), block-strided final stage.
// For K > 1 a thread's N rows (the single-column kernel's, so that every
// column's partial sums are its single solve's) are N * K = 16 K contiguous
// bytes; the warp moves its 32 threads' runs, one contiguous tile, between
// global and shared memory with coalesced 16-byte accesses, and each thread
// reads its own run from shared memory (launched with cgs_stage_bytes of
// dynamic shared memory).
template <typename T, int WARPS, int K>
__global__ void __launch_bounds__(WARPS * 32, K > 1 ? 1 : 8) k_cgs_updateK(T *__restrict__ w, Cols<T> V, int nv, int64_t n,
                                                            GridRed gr, LevelK<T> L, int j, int compute_y,
                                                            double *abs_e, const uint32_t *active, int *err) {
  constexpr int N = 16 / sizeof(T);
  __shared__ T sh[K][kMaxCols];
  __shared__ T sred[WARPS][K];
  for (int t = threadIdx.x; t < nv * K; t += blockDim.x) {
    const int c = t / nv, k = t % nv;
    sh[c][k] = L.H[c * L.hs + (int64_t)j * L.ldh + k];
  }
  __syncthreads();
  T part[K];
#pragma unroll
  for (int c = 0; c < K; c++) part[c] = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nq = n / N;
  if constexpr (K > 1) {
    constexpr int S = N * K, P = S + N, TILE = 32 * S;  // values a thread, its padded pitch, a warp tile
    extern __shared__ __align__(16) unsigned char cgs_stage[];
    const int lane = threadIdx.x & 31;
    T *tile = reinterpret_cast<T *>(cgs_stage) + (size_t)(threadIdx.x >> 5) * 32 * P;
    T *mine = tile + lane * P;
    for (int64_t q0 = tid - lane; q0 < nq; q0 += stride) {
      const int64_t base = q0 * S;
      const int lim = (int)((nq - q0 < 32 ? nq - q0 : 32) * S);  // values of the tile inside the vector
      auto stage_in = [&](const T *src) {
        __syncwarp();
#pragma unroll 4
        for (int i = lane * N; i < TILE; i += 32 * N)
          if (i < lim) *reinterpret_cast<uint4 *>(tile + (i / S) * P + i % S) = *reinterpret_cast<const uint4 *>(src + base + i);
        __syncwarp();
      };
      using Vec = VecN<T, N>;  // 16 bytes of the run
      T r[S];
      stage_in(V.p[0]);
#pragma unroll
      for (int e0 = 0; e0 < S; e0 += N) {
        const Vec a = *reinterpret_cast<const Vec *>(mine + e0);
#pragma unroll
        for (int e = 0; e < N; e++) r[e0 + e] = mul_rn(a.v[e], sh[(e0 + e) % K][0]);
      }
      for (int k = 1; k < nv; k++) {
        stage_in(V.p[k]);
#pragma unroll
        for (int e0 = 0; e0 < S; e0 += N) {
          const Vec a = *reinterpret_cast<const Vec *>(mine + e0);
#pragma unroll
          for (int e = 0; e < N; e++) r[e0 + e] = fmaT(a.v[e], sh[(e0 + e) % K][k], r[e0 + e]);
        }
      }
      stage_in(w);
      const bool own = q0 + lane < nq;
      // row by row, as the single-column kernel: update, then the squared norm
#pragma unroll
      for (int e0 = 0; e0 < S; e0 += N) {
        Vec a = *reinterpret_cast<const Vec *>(mine + e0);
#pragma unroll
        for (int e = 0; e < N; e++) {
          a.v[e] = sub_rn(a.v[e], r[e0 + e]);
          if (own) part[(e0 + e) % K] = fmaT(a.v[e], a.v[e], part[(e0 + e) % K]);
        }
        *reinterpret_cast<Vec *>(mine + e0) = a;
      }
      __syncwarp();
#pragma unroll 4
      for (int i = lane * N; i < TILE; i += 32 * N)
        if (i < lim) *reinterpret_cast<uint4 *>(w + base + i) = *reinterpret_cast<const uint4 *>(tile + (i / S) * P + i % S);
    }
  }
  // the N rows of a thread, RG at a time as one contiguous run of RG * K values
  constexpr int RG = (N * K <= 16) ? N : 1, E = RG * K;
  for (int64_t q = tid; K == 1 && q < nq; q += stride) {
#pragma unroll
    for (int g = 0; g < N / RG; g++) {
      const int64_t i0 = q * N + g * RG;
      T a[E], r[E], wv[E];
      RowK<T, E>::load(V.p[0] + i0 * K, a);
#pragma unroll
      for (int e = 0; e < E; e++) r[e] = mul_rn(a[e], sh[e % K][0]);
      for (int k = 1; k < nv; k++) {
        T b[E];
        RowK<T, E>::load(V.p[k] + i0 * K, b);
#pragma unroll
        for (int e = 0; e < E; e++) r[e] = fmaT(b[e], sh[e % K][k], r[e]);
      }
      RowK<T, E>::load(w + i0 * K, wv);
      // row by row, as the single-column kernel: update, then the squared norm
#pragma unroll
      for (int e = 0; e < E; e++) {
        wv[e] = sub_rn(wv[e], r[e]);
        part[e % K] = fmaT(wv[e], wv[e], part[e % K]);
      }
      RowK<T, E>::store(w + i0 * K, wv);
    }
  }
  for (int64_t i = nq * N + tid; i < n; i += stride) {
    T a[K], r[K], wv[K];
    RowK<T, K>::load(V.p[0] + i * K, a);
#pragma unroll
    for (int c = 0; c < K; c++) r[c] = mul_rn(a[c], sh[c][0]);
    for (int k = 1; k < nv; k++) {
      T b[K];
      RowK<T, K>::load(V.p[k] + i * K, b);
#pragma unroll
      for (int c = 0; c < K; c++) r[c] = fmaT(b[c], sh[c][k], r[c]);
    }
    RowK<T, K>::load(w + i * K, wv);
#pragma unroll
    for (int c = 0; c < K; c++) {
      wv[c] = sub_rn(wv[c], r[c]);
      part[c] = fmaT(wv[c], wv[c], part[c]);
    }
    RowK<T, K>::store(w + i * K, wv);
  }
  T *parts = static_cast<T *>(gr.partials);
  block_partials<T, K, WARPS>(part, K, 0, K, parts, sred);
  if (!last_block(gr.ticket)) return;
  const uint32_t act = *active;
  // column c's norm and Givens step on thread c (each column's state is its own)
  const T t = final_block_multi<T, WARPS, K>(parts, 0, K, K);
  const int c = threadIdx.x;
  if (c < K && ((act >> c) & 1u)) givens_step<T>(L.col(c, j, compute_y, abs_e ? abs_e + c : nullptr, err), t);
  if (threadIdx.x == 0) *gr.ticket = 0;
}

// ||r(:, c)|| of the outer residual (V(0) = b - A x, stored by the product):
// e(0) = ||r||, 1/||r|| and |e(0)| for the host, per column (gmres.hpp:87,
// 100-103).  Two elements per thread (16 bytes of one column).
template <int WARPS, int K>
__global__ void __launch_bounds__(WARPS * 32) k_resnormK(const double *__restrict__ r, int64_t n, GridRed gr,
                                                         LevelK<double> L, double *abs_e, const uint32_t *active) {
  __shared__ double sred[WARPS][K];
  double part[K];
#pragma unroll
  for (int c = 0; c < K; c++) part[c] = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t i = tid; i < n; i += stride) {
    double v[K];
    RowK<double, K>::load(r + i * K, v);
#pragma unroll
    for (int c = 0; c < K; c++) part[c] = __fma_rn(v[c], v[c], part[c]);
  }
  double *parts = static_cast<double *>(gr.partials);
  block_partials<double, K, WARPS>(part, K, 0, K, parts, sred);
  if (!last_block(gr.ticket)) return;
  const uint32_t act = *active;
  const double t = final_block_multi<double, WARPS, K>(parts, 0, K, K);
  const int c = threadIdx.x;
  if (c < K && ((act >> c) & 1u)) {
    const double h = sqrt(t);
    L.e[c * L.vs] = h;
    L.inv[c] = 1.0 / h;
    abs_e[c] = fabs(h);
  }
  if (threadIdx.x == 0) *gr.ticket = 0;
}

// The Richardson weight of an update call, per column: with t = tmp(:, c)
// (fp16(A v), stored by the product) and o = other(:, c), om = <t, o> / <t, t>
// in fp32 (wildcard(., tof32), f3r-gpu.cpp:235-240 / 249-254), then the
// running mean ome[k] = fp16(sum[k] / den); k = 0 also advances den.  Rows
// in groups of 4 per thread, block-strided final stage.
template <int WARPS, int K>
__global__ void __launch_bounds__(WARPS * 32) k_rich_weightK(const __half *__restrict__ tmp,
                                                             const __half *__restrict__ other, int64_t n,
                                                             GridRed gr, RichState *rs, int k) {
  __shared__ float sred[WARPS][2 * K];
  float d[2 * K];
#pragma unroll
  for (int q = 0; q < 2 * K; q++) d[q] = 0.0f;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t i = tid; i < n; i += stride) {
    float t[K], o[K];
    RowK<__half, K>::load(tmp + i * K, t);
    RowK<__half, K>::load(other + i * K, o);
#pragma unroll
    for (int c = 0; c < K; c++) {
      d[c] = __fmaf_rn(t[c], t[c], d[c]);
      d[K + c] = __fmaf_rn(t[c], o[c], d[K + c]);
    }
  }
  float *parts = static_cast<float *>(gr.partials);
  block_partials<float, 2 * K, WARPS>(d, 2 * K, 0, 2 * K, parts, sred);
  if (!last_block(gr.ticket)) return;
  // <t, t> of column c on thread c, <t, o> on thread K + c
  __shared__ float sto[K];
  const float v = final_block_multi<float, WARPS, 2 * K>(parts, 0, 2 * K, 2 * K);
  if ((int)threadIdx.x >= K && (int)threadIdx.x < 2 * K) sto[threadIdx.x - K] = v;
  __syncthreads();
  {
    const int c = threadIdx.x;
    if (c < K) {
      const float tt = v, to = sto[c];
      RichState *s = rs + c;
      const float om = to / tt;
      s->om[k] = om;
      s->sum[k] += om;
      if (k == 0) s->den += 1;
      s->ome[k] = __float2half_rn(s->sum[k] / (float)s->den);
    }
  }
  if (threadIdx.x == 0) *gr.ticket = 0;
}

// ---------------------------------------------------------------------------
// Elementwise kernels of the levels over K columns (grid stride over rows;
// each element computed exactly as the single-column kernel computes it).
// Narrow blocks take RowsPer<K> consecutive rows per thread, so that a thread
// still moves 16 bytes of fp32 per access; the rows of a group are contiguous
// (row-major interleaving), element e of a group is column e % K.
// ---------------------------------------------------------------------------
template <int K> struct RowsPer {
  static constexpr int R = K >= 4 ? 1 : 4 / K;
};
// calls f(row0, std::integral_constant<int, ROWS>) for groups of R rows, then
// for the remaining rows one at a time
template <int R, typename F> __device__ __forceinline__ void for_row_groups(int64_t n, F f) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t ng = n / R;
  for (int64_t q = tid; q < ng; q += stride) f(q * R, std::integral_constant<int, R>());
  if constexpr (R > 1)
    for (int64_t i = ng * R + tid; i < n; i += stride) f(i, std::integral_constant<int, 1>());
}

// Level-2 entry (k_level2_enter): V1(j)(:, c) *= 1/h_c in place, then
// V2(0) = float(V1(j)); e_c(0) = 1.
template <int K>
__global__ void k_level2_enterK(double *const *__restrict__ in_slot, const double *__restrict__ inv,
                                float *__restrict__ v0, float *e, int64_t e_stride, int64_t n) {
  double *in = *in_slot;
  double s[K];
#pragma unroll
  for (int c = 0; c < K; c++) s[c] = inv[c];
  if (blockIdx.x == 0 && threadIdx.x < K) e[threadIdx.x * e_stride] = 1.0f;
  for_row_groups<RowsPer<K>::R>(n, [&](int64_t i0, auto rows) {
    constexpr int E = decltype(rows)::value * K;
    double a[E];
    float o[E];
    RowK<double, E>::load(in + i0 * K, a);
#pragma unroll
    for (int q = 0; q < E; q++) {
      a[q] *= s[q % K];
      o[q] = (float)a[q];
    }
    RowK<double, E>::store(in + i0 * K, a);
    RowK<float, E>::store(v0 + i0 * K, o);
  });
}

// x(:, c) = Z y_c (inner levels) or x(:, c) += Z y_c for the columns in mask
// (outer level), the sum in the level's type T (k_zy)
template <typename T, typename Out, bool ACCUM, int K, typename ZT = T>
__global__ void __launch_bounds__(kEwThreads, K == 1 ? 8 : 1) k_zyK(Cols<ZT> Z, const T *__restrict__ y, int64_t y_stride, int nz, Out *out_direct,
                      Out *const *out_slot, uint32_t mask, int64_t n) {
  __shared__ T sy[K][kMaxCols];
  for (int t = threadIdx.x; t < nz * K; t += blockDim.x) {
    const int c = t / nz, k = t % nz;
    sy[c][k] = y[c * y_stride + k];
  }
  __syncthreads();
  Out *out = out_slot ? *out_slot : out_direct;
  for_row_groups<RowsPer<K>::R>(n, [&](int64_t i0, auto rows) {
    constexpr int E = decltype(rows)::value * K;
    T a[E], r[E];
    RowK<ZT, E>::load(Z.p[0] + i0 * K, a);  // ZT fp16: widened exactly
#pragma unroll
    for (int q = 0; q < E; q++) r[q] = mul_rn(a[q], sy[q % K][0]);
    for (int k = 1; k < nz; k++) {
      T b[E];
      RowK<ZT, E>::load(Z.p[k] + i0 * K, b);
#pragma unroll
      for (int q = 0; q < E; q++) r[q] = fmaT(b[q], sy[q % K][k], r[q]);
    }
    if (ACCUM) {
#pragma unroll
      for (int q = 0; q < E; q++)
        if ((mask >> (q % K)) & 1u) out[i0 * K + q] = add_rn(out[i0 * K + q], (Out)r[q]);
    } else {
      Out o[E];
#pragma unroll
      for (int q = 0; q < E; q++) o[q] = (Out)r[q];
      RowK<Out, E>::store(out + i0 * K, o);
    }
  });
}

// First half of R, diagonal M (k_rich_enter_diag), per column: the pending
// normalisation of in(:, c) (in_inv[c], or none), hin = fp16(in * sc),
// hout = M hin, times ome_c[0] on a call without a weight update; e_c(0) = 1
// of the calling level when e_set is given.
template <bool SCALE_BY_OME, int K, int NR, bool MM>
__device__ __forceinline__ void rich_enter_rows(int64_t i0, float *__restrict__ in, bool normalise, const float (&s)[K],
                                                const float (&om)[K], float sc, const DiagPre &M,
                                                __half *__restrict__ hin, __half *__restrict__ hout) {
  constexpr int E = NR * K, NM = MM ? E : NR;  // diagonal values: per row, or per row and column
  float v[E], w[NM], z[NM];
  __half hi[E], ho[E];
  RowK<float, E>::load(in + i0 * K, v);
  if (normalise) {
#pragma unroll
    for (int q = 0; q < E; q++) v[q] *= s[q % K];
    RowK<float, E>::store(in + i0 * K, v);
  }
  diag_load<NM>(M.w ? M.w + i0 * (MM ? K : 1) : nullptr, w);
  diag_load<NM>(M.z ? M.z + i0 * (MM ? K : 1) : nullptr, z);
#pragma unroll
  for (int q = 0; q < E; q++) {
    hi[q] = f2h(v[q] * sc);
    const float t = h2f(f2h(w[MM ? q : q / K] * h2f(hi[q])));
    float o = h2f(f2h(z[MM ? q : q / K] * t));
    if (SCALE_BY_OME) o = h2f(f2h(o * om[q % K]));
    ho[q] = f2h(o);
  }
  RowK<__half, E>::store(hin + i0 * K, hi);
  RowK<__half, E>::store(hout + i0 * K, ho);
}

template <bool SCALE_BY_OME, int K, bool MM = false>
__global__ void __launch_bounds__(kEwThreads, K == 1 ? 8 : 1) k_rich_enter_diagK(float *__restrict__ in, const float *__restrict__ in_inv, float sc, DiagPre M,
                                   __half *__restrict__ hin, __half *__restrict__ hout,
                                   const RichState *__restrict__ rs, float *e_set, int64_t e_stride, int64_t n) {
  if (e_set && blockIdx.x == 0 && threadIdx.x < K) e_set[threadIdx.x * e_stride] = 1.0f;
  float om[K], s[K];
#pragma unroll
  for (int c = 0; c < K; c++) {
    om[c] = SCALE_BY_OME ? h2f(rs[c].ome[0]) : 1.0f;
    s[c] = in_inv ? in_inv[c] : 1.0f;
  }
  const bool normalise = in_inv != nullptr;
  constexpr int R = RowsPer<K>::R;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t ng = n / R;
  for (int64_t q = tid; q < ng; q += stride)
    rich_enter_rows<SCALE_BY_OME, K, R, MM>(q * R, in, normalise, s, om, sc, M, hin, hout);
  for (int64_t i = ng * R + tid; i < n; i += stride)
    rich_enter_rows<SCALE_BY_OME, K, 1, MM>(i, in, normalise, s, om, sc, M, hin, hout);
}

// General M: (normalise in place), hin = fp16(in * sc) (k_rich_cast_in)
template <int K>
__global__ void k_rich_cast_inK(float *__restrict__ in, const float *__restrict__ in_inv, float sc,
                                __half *__restrict__ hin, float *e_set, int64_t e_stride, int64_t n) {
  if (e_set && blockIdx.x == 0 && threadIdx.x < K) e_set[threadIdx.x * e_stride] = 1.0f;
  for_row_groups<RowsPer<K>::R>(n, [&](int64_t i0, auto rows) {
    constexpr int E = decltype(rows)::value * K;
    float v[E], h[E];
    RowK<float, E>::load(in + i0 * K, v);
    if (in_inv) {
#pragma unroll
      for (int q = 0; q < E; q++) v[q] *= in_inv[q % K];
      RowK<float, E>::store(in + i0 * K, v);
    }
#pragma unroll
    for (int q = 0; q < E; q++) h[q] = v[q] * sc;
    RowK<__half, E>::store(hin + i0 * K, h);
  });
}

// hout(:, c) = fp16(hout * fp16(om_c[0])) (k_rich_scale_om)
template <int K>
__global__ void k_rich_scale_omK(__half *__restrict__ hout, const RichState *__restrict__ rs, int64_t n) {
  float om[K];
#pragma unroll
  for (int c = 0; c < K; c++) om[c] = h2f(f2h(rs[c].om[0]));
  for_row_groups<RowsPer<K>::R>(n, [&](int64_t i0, auto rows) {
    constexpr int E = decltype(rows)::value * K;
    float h[E];
    RowK<__half, E>::load(hout + i0 * K, h);
#pragma unroll
    for (int q = 0; q < E; q++) h[q] = h[q] * om[q % K];
    RowK<__half, E>::store(hout + i0 * K, h);
  });
}

// hout(:, c) = fp16(hout + om_c[k] t2), or on the last step out = fp32(that)
// / sc (k_rich_axpy); use_ome selects ome_c[k]
template <int K>
__global__ void k_rich_axpyK(__half *__restrict__ hout, const __half *__restrict__ t2,
                             const RichState *__restrict__ rs, int k, int use_ome, float *__restrict__ out, float isc,
                             int64_t n, __half *__restrict__ out16) {
  float om[K];
#pragma unroll
  for (int c = 0; c < K; c++) om[c] = use_ome ? h2f(rs[c].ome[k]) : rs[c].om[k];
  for_row_groups<RowsPer<K>::R>(n, [&](int64_t i0, auto rows) {
    constexpr int E = decltype(rows)::value * K;
    float h[E], t[E], hn[E];
    RowK<__half, E>::load(hout + i0 * K, h);
    RowK<__half, E>::load(t2 + i0 * K, t);
#pragma unroll
    for (int q = 0; q < E; q++) hn[q] = h2f(f2h(__fmaf_rn(om[q % K], t[q], h[q])));
    if (out) {
#pragma unroll
      for (int q = 0; q < E; q++) hn[q] *= isc;
      RowK<float, E>::store(out + i0 * K, hn);
    } else {
      RowK<__half, E>::store((out16 ? out16 : hout) + i0 * K, hn);
    }
  });
}

// out = fp32(hout) / sc (k_rich_exit)
template <int K>
__global__ void k_rich_exitK(const __half *__restrict__ hout, float *__restrict__ out, float isc, int64_t n) {
  for_row_groups<RowsPer<K>::R>(n, [&](int64_t i0, auto rows) {
    constexpr int E = decltype(rows)::value * K;
    float h[E];
    RowK<__half, E>::load(hout + i0 * K, h);
#pragma unroll
    for (int q = 0; q < E; q++) h[q] *= isc;
    RowK<float, E>::store(out + i0 * K, h);
  });
}

// gather / scatter of K interleaved columns through a row permutation
template <int K>
__global__ void k_permute_gatherK(const double *__restrict__ in, const int32_t *__restrict__ perm,
                                  double *__restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
    for (int c = 0; c < K; c++) out[i * K + c] = in[(int64_t)perm[i] * K + c];
}
template <int K>
__global__ void k_permute_scatterK(const double *__restrict__ in, const int32_t *__restrict__ perm,
                                   double *__restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
    for (int c = 0; c < K; c++) out[(int64_t)perm[i] * K + c] = in[i * K + c];
}

// Columns of a host or device block (nrhs columns of stride ld) into and out
// of the interleaved layout: out[i * K + c] = in[c * ld + i] for c < ncols
// (zero for the padding columns)
__global__ void k_interleave(const double *__restrict__ in, int64_t ld, int ncols, int K, double *__restrict__ out,
                             int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    for (int c = 0; c < K; c++) out[i * K + c] = c < ncols ? in[c * ld + i] : 0.0;
}
__global__ void k_deinterleave(const double *__restrict__ in, int K, int ncols, double *__restrict__ out, int64_t ld,
                               int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    for (int c = 0; c < ncols; c++) out[c * ld + i] = in[i * K + c];
}

}  // namespace f3r
