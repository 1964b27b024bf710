// ilu.cuh -- block-Jacobi ILU(0) triangular solves on the GPU.
//
// The reference solves each block sequentially on one CPU thread
// (trsv/bj.hpp:58-98).  Here every block-Jacobi block is one CTA, and inside
// a block the rows are grouped into dependency levels (level(i) = 1 + the
// highest level among the rows it reads); a CTA sweeps its levels in order
// with one __syncthreads() between levels, one thread per row.  The blocks
// never read each other's rows, so no inter-CTA synchronisation exists.
// Arithmetic per row follows the reference's order: the forward sweep walks
// the row's off-diagonals by increasing column, the backward sweep by
// decreasing column (the reference's 180-degree rotated U, csr.hpp:60-86)
// and multiplies by the fp16-rounded inverse diagonal formed in fp64
// (CSR::inverse_last, csr.hpp:60-65).  fp16 values, fp32 accumulation.
#pragma once

#include <vector>

#include "device.cuh"
#include "internal.hpp"

namespace f3r {

struct RichState;

struct IluTri {
  // the factor laid out in (block, level) row order q, as the kernel visits it
  int4 *meta = nullptr;    // per q: vector position, first and end entry, unused
  __half *val = nullptr;   // entries of every row in processing order (diagonal excluded)
  int32_t *idx = nullptr;  // their columns, mapped to vector positions
  __half *dinv = nullptr;  // upper only: fp16(1 / u_ii), per q
  int32_t *lvl_off = nullptr;  // row ranges (in q) of the levels, all blocks
  int32_t *blk_lvl = nullptr;  // per block: first level index (nblocks + 1)
  int32_t *blk_pos = nullptr;  // per block: first vector position (nblocks + 1)
  int32_t nlevels_max = 0;
  int32_t smem_rows = 0;  // > 0: blocks occupy contiguous positions, each at most this many rows
};

// One CTA per block-Jacobi block.  The factor is stored in the order the
// kernel visits rows (level by level within a block), so a row's data is one
// int4 of metadata and a contiguous run of entries: two dependent loads,
// coalesced across the threads of a level.  When the blocks occupy
// contiguous vector positions (T.smem_rows > 0) the block's results are also
// kept in shared memory, so a row reads the rows it depends on (all in its
// block, written at earlier levels) from there instead of from L2.  The
// terms are the reference's, in its order: the forward sweep by increasing
// column, the backward sweep by decreasing column.
template <bool UPPER>
__global__ void k_trsv_bj(IluTri T, const __half *__restrict__ in, __half *__restrict__ out,
                          const __half *__restrict__ ome) {
  extern __shared__ __half sy[];
  const int b = blockIdx.x;
  const int l0 = T.blk_lvl[b], l1 = T.blk_lvl[b + 1];
  const float om = ome ? __half2float(*ome) : 1.0f;
  const bool sm = T.smem_rows > 0;
  const int32_t p0 = sm ? T.blk_pos[b] : 0;
  for (int l = l0; l < l1; l++) {
    const int r0 = T.lvl_off[l], r1 = T.lvl_off[l + 1];
    for (int q = r0 + threadIdx.x; q < r1; q += blockDim.x) {
      const int4 m = T.meta[q];
      float t = __half2float(in[m.x]);
      for (int32_t j = m.y; j < m.z; j++)
        t = __fmaf_rn(-__half2float(T.val[j]), __half2float(sm ? sy[T.idx[j] - p0] : out[T.idx[j]]), t);
      const __half h = UPPER ? __float2half_rn(t * __half2float(T.dinv[q])) : __float2half_rn(t);
      out[m.x] = h;
      if (sm) sy[m.x - p0] = h;
    }
    __syncthreads();
  }
  // the reference solves, then scales: hout *= ome[0] (work/src/f3r.cpp:216, 229)
  if (UPPER && ome) {
    for (int q = T.lvl_off[l0] + threadIdx.x; q < T.lvl_off[l1]; q += blockDim.x) {
      const int32_t p = T.meta[q].x;
      out[p] = __float2half_rn(__half2float(sm ? sy[p - p0] : out[p]) * om);
    }
  }
}

constexpr int32_t kIluSmemRows = 48 * 1024;  // fp16 results of one block in shared memory: 96 KB at most

struct IluDevice {
  IluTri L, U;
  int32_t nblocks = 0;
  std::vector<void *> allocs;

  template <typename T> cudaError_t up(T **d, const std::vector<T> &h) {
    cudaError_t e = cudaMalloc((void **)d, sizeof(T) * std::max<size_t>(h.size(), 1));
    if (e != cudaSuccess) return e;
    allocs.push_back((void *)*d);
    return cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
  }
  void release() {
    for (void *p : allocs) cudaFree(p);
    allocs.clear();
  }

  // levels of one triangular factor inside each block-Jacobi block
  static void levels(const HostCSR &M, bool upper, const std::vector<int32_t> &bptr, std::vector<int32_t> &order,
                     std::vector<int32_t> &lvl_off, std::vector<int32_t> &blk_lvl, int32_t &maxlev) {
    const int32_t n = M.n, nb = (int32_t)bptr.size() - 1;
    std::vector<int32_t> lev(n, 0);
    order.clear();
    lvl_off.assign(1, 0);
    blk_lvl.assign(1, 0);
    maxlev = 0;
    for (int32_t b = 0; b < nb; b++) {
      int32_t nl = 0;
      if (!upper) {
        for (int32_t i = bptr[b]; i < bptr[b + 1]; i++) {
          int32_t lv = 0;
          for (int32_t j = M.rptr[i]; j < M.rptr[i + 1]; j++)
            if (M.idx[j] < i) lv = std::max(lv, lev[M.idx[j]] + 1);
          lev[i] = lv;
          nl = std::max(nl, lv + 1);
        }
      } else {
        for (int32_t i = bptr[b + 1] - 1; i >= bptr[b]; i--) {
          int32_t lv = 0;
          for (int32_t j = M.rptr[i]; j < M.rptr[i + 1]; j++)
            if (M.idx[j] > i) lv = std::max(lv, lev[M.idx[j]] + 1);
          lev[i] = lv;
          nl = std::max(nl, lv + 1);
        }
      }
      // bucket the block's rows by level
      std::vector<int32_t> cnt(nl + 1, 0);
      for (int32_t i = bptr[b]; i < bptr[b + 1]; i++) cnt[lev[i] + 1]++;
      for (int32_t l = 0; l < nl; l++) cnt[l + 1] += cnt[l];
      const size_t base = order.size();
      order.resize(base + (bptr[b + 1] - bptr[b]));
      std::vector<int32_t> fill(cnt.begin(), cnt.end() - 1);
      for (int32_t i = bptr[b]; i < bptr[b + 1]; i++) order[base + fill[lev[i]]++] = i;
      for (int32_t l = 0; l < nl; l++) lvl_off.push_back((int32_t)(base + cnt[l + 1]));
      blk_lvl.push_back(blk_lvl.back() + nl);
      maxlev = std::max(maxlev, nl);
    }
  }

  Status build_tri(IluTri &T, const HostCSR &M, bool upper, const std::vector<int32_t> &bptr,
                   const std::vector<int32_t> &pos) {
    std::vector<int32_t> order, lvl_off, blk_lvl;
    levels(M, upper, bptr, order, lvl_off, blk_lvl, T.nlevels_max);
    // blocks on contiguous positions (natural order) and of at most
    // kIluSmemRows rows keep their results in shared memory
    const int32_t nb = (int32_t)bptr.size() - 1;
    std::vector<int32_t> bpos(nb + 1, 0);
    bool contiguous = true;
    int32_t maxlen = 0;
    for (int32_t b = 0; b < nb; b++) {
      bpos[b] = bptr[b] < bptr[b + 1] ? pos[bptr[b]] : 0;
      maxlen = std::max(maxlen, bptr[b + 1] - bptr[b]);
      for (int32_t i = bptr[b]; i < bptr[b + 1] && contiguous; i++) contiguous = pos[i] == bpos[b] + (i - bptr[b]);
    }
    T.smem_rows = (contiguous && maxlen <= kIluSmemRows) ? std::max(maxlen, 1) : 0;
    // the factor in visiting order: fp16 values rounded once from fp64 (the
    // reference casts CSR<double> to CSR<__half>, csr.hpp:23-25)
    const size_t nq = order.size();
    std::vector<int4> meta(nq);
    std::vector<double> v, dinv;
    std::vector<int32_t> idx;
    v.reserve(M.val.size());
    idx.reserve(M.idx.size());
    if (upper) dinv.resize(nq);
    for (size_t q = 0; q < nq; q++) {
      const int32_t i = order[q], r0 = M.rptr[i], r1 = M.rptr[i + 1];
      meta[q].x = pos[i];
      meta[q].y = (int32_t)idx.size();
      if (!upper) {
        for (int32_t j = r0; j < r1 - 1; j++) {  // last entry is the unit diagonal
          v.push_back(M.val[j]);
          idx.push_back(pos[M.idx[j]]);
        }
      } else {
        for (int32_t j = r1 - 1; j > r0; j--) {  // first entry is the diagonal
          v.push_back(M.val[j]);
          idx.push_back(pos[M.idx[j]]);
        }
        dinv[q] = 1.0 / M.val[r0];
      }
      meta[q].z = (int32_t)idx.size();
      meta[q].w = 0;
    }
    if (up(&T.meta, meta) != cudaSuccess || up(&T.idx, idx) != cudaSuccess || up(&T.lvl_off, lvl_off) != cudaSuccess ||
        up(&T.blk_lvl, blk_lvl) != cudaSuccess || up(&T.blk_pos, bpos) != cudaSuccess)
      return fail(F3R_ERROR_CUDA, "ILU upload failed");
    F3R_TRY(to_half(&T.val, v));
    if (upper) F3R_TRY(to_half(&T.dinv, dinv));
    return F3R_SUCCESS;
  }

  Status to_half(__half **d, const std::vector<double> &v);

  Status build(cudaStream_t, const HostCSR &Lh, const HostCSR &Uh, const std::vector<int32_t> &perm, bool permuted,
               const std::vector<int32_t> &bptr) {
    const int32_t n = Lh.n;
    std::vector<int32_t> pos(n);
    for (int32_t i = 0; i < n; i++) pos[i] = i;
    if (permuted)
      for (int32_t s = 0; s < n; s++) pos[perm[s]] = s;
    nblocks = (int32_t)bptr.size() - 1;
    F3R_TRY(build_tri(L, Lh, false, bptr, pos));
    F3R_TRY(build_tri(U, Uh, true, bptr, pos));
    // the attribute is the kernel's, shared by every solver: always the cap
    const int cap = (int)(kIluSmemRows * sizeof(__half));
    if (cudaFuncSetAttribute(k_trsv_bj<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap) != cudaSuccess ||
        cudaFuncSetAttribute(k_trsv_bj<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap) != cudaSuccess)
      return fail(F3R_ERROR_CUDA, "ILU shared-memory attribute");
    return F3R_SUCCESS;
  }

  // out = U^-1 L^-1 x (tmp holds L^-1 x); ome (nullable) scales the result
  Status apply(cudaStream_t st, const __half *x, __half *tmp, __half *out, const __half *ome) const {
    k_trsv_bj<false><<<nblocks, 256, (size_t)L.smem_rows * sizeof(__half), st>>>(L, x, tmp, nullptr);
    k_trsv_bj<true><<<nblocks, 256, (size_t)U.smem_rows * sizeof(__half), st>>>(U, tmp, out, ome);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(F3R_ERROR_CUDA, std::string("ILU trsv launch: ") + cudaGetErrorString(e));
    return F3R_SUCCESS;
  }
};

// ---------------------------------------------------------------------------
// Global ILU(0), level-scheduled over the whole GPU (F3R_PRECOND_ILU0_LEVEL).
//
// One factor of the global (single-block) ILU(0) is solved by one kernel
// without grid barriers.  The rows are listed level by level, every level
// padded with -1 to whole 32-row chunks, so the 32 rows of a chunk never read
// each other.  Warps take chunks in list order from an atomic counter; a row
// waits until each row it reads carries this launch's generation in its flag
// (acquire load), then computes exactly as k_trsv_bj does (same order of
// terms, same roundings) and publishes value then flag (release store).  A
// warp waits only on chunks taken before its own by running warps, and the
// lowest unfinished chunk never waits, so the solve always completes.  Every
// wait is bounded (kWaitLimitNs); the first timeout sets the device error
// word, which ends every other wait of the launch at once.  The last block to
// finish resets the counter and advances the generation, so back-to-back
// launches (and graph replays) need no host work.
struct IluLevelTri {
  // rows level by level, padded to 32-row chunks, in the order warps take them
  int4 *meta = nullptr;     // per slot: vector position (-1: padding), first and end entry
  __half *val = nullptr;    // entries in processing order (diagonal excluded)
  int32_t *idx = nullptr;   // their columns, mapped to vector positions
  __half *dinv = nullptr;   // upper only: per slot
  int32_t nchunks = 0;
  int32_t nlevels = 0;
  int32_t *flag = nullptr;                  // per vector position: generation of its last write
  unsigned int *state = nullptr;            // chunk counter, finished-block ticket, generation
};

__device__ __forceinline__ unsigned int ld_relaxed_u32(const int32_t *p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(int32_t *p, unsigned int v) {
  asm volatile("st.release.gpu.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

constexpr int kLevelBatch = 16;  // dependencies polled, then read, together

// Waits until flag[q[u]] == gen for every u < cnt (relaxed polls, then one
// fence orders the caller's later loads after them).  Bounded: after
// limit_ns of %globaltimer it records DEV_TIMEOUT_TRSV in *err and returns
// false; it also returns false at once when *err is already set (another
// wait of the launch gave up, or the solve broke down), so no wait outlives
// the first failure by more than one bound.
__device__ __forceinline__ bool wait_flags(const int32_t *flag, const int32_t (&q)[kLevelBatch], int cnt,
                                           unsigned int gen, int *err, unsigned long long limit_ns) {
  volatile int *verr = err;
  uint32_t waiting = (1u << cnt) - 1u;
  unsigned long long t0 = 0;
  int polls = 0;
  bool ok = true;
  while (true) {
#pragma unroll
    for (int u = 0; u < kLevelBatch; u++)
      if ((waiting >> u) & 1u)
        if (ld_relaxed_u32(flag + q[u]) == gen) waiting &= ~(1u << u);
    if (waiting == 0) break;
    if (*verr != 0) {
      ok = false;
      break;
    }
    if (polls++ == 0) t0 = global_ns();
    else if (global_ns() - t0 > limit_ns) {
      atomicCAS(err, 0, (int)DEV_TIMEOUT_TRSV);
      ok = false;
      break;
    }
    if (polls > 4) __nanosleep(32);
  }
  __threadfence();
  return ok;
}

template <bool UPPER>
__global__ void __launch_bounds__(256, 2) k_trsv_level(IluLevelTri T, const __half *__restrict__ in, __half *out,
                                                    int *err) {
  __shared__ unsigned int gen_s;
  if (threadIdx.x == 0) gen_s = *(volatile unsigned int *)&T.state[2] + 1u;
  __syncthreads();
  const unsigned int gen = gen_s;
  const int lane = threadIdx.x & 31;
  bool abort = false;
  while (true) {
    unsigned int c = 0;
    if (lane == 0) c = atomicAdd(&T.state[0], 1u);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= (unsigned int)T.nchunks) break;
    const size_t slot = (size_t)c * 32 + lane;
    const int4 m = T.meta[slot];
    if (m.x >= 0) {
      const int32_t p = m.x;
      float t = __half2float(in[p]);
      // the entries in processing order: lower by increasing, upper by decreasing column
      const int32_t b = m.y, ndep = m.z - m.y;
      for (int32_t base = 0; base < ndep; base += kLevelBatch) {
        const int cnt = min(kLevelBatch, ndep - base);
        int32_t q[kLevelBatch];
        float lv[kLevelBatch];
#pragma unroll
        for (int u = 0; u < kLevelBatch; u++)
          if (u < cnt) {
            const int32_t j = b + base + u;
            q[u] = T.idx[j];
            lv[u] = __half2float(T.val[j]);
          }
        // every flag of the batch polled at once; one fence orders the value loads after them
        if (!abort) abort = !wait_flags(T.flag, q, cnt, gen, err, kWaitLimitNs);
        float y[kLevelBatch];
#pragma unroll
        for (int u = 0; u < kLevelBatch; u++)
          if (u < cnt) y[u] = __half2float(__ldcg(out + q[u]));
#pragma unroll
        for (int u = 0; u < kLevelBatch; u++)
          if (u < cnt) t = __fmaf_rn(-lv[u], y[u], t);
      }
      const __half h = UPPER ? __float2half_rn(t * __half2float(T.dinv[slot])) : __float2half_rn(t);
      out[p] = h;
      __threadfence();
      st_release_u32(T.flag + p, gen);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int tk = atomicAdd(&T.state[1], 1u);
    if (tk == gridDim.x - 1) {
      T.state[0] = 0;
      T.state[1] = 0;
      __threadfence();
      atomicAdd(&T.state[2], 1u);
    }
  }
}

struct IluLevel {
  IluLevelTri L, U;
  int grid = 0, scale_grid = 1;
  int64_t n = 0;
  std::vector<void *> allocs;

  template <typename T> cudaError_t up(T **d, const std::vector<T> &h) {
    cudaError_t e = cudaMalloc((void **)d, sizeof(T) * std::max<size_t>(h.size(), 1));
    if (e != cudaSuccess) return e;
    allocs.push_back((void *)*d);
    return cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
  }
  void release() {
    for (void *p : allocs) cudaFree(p);
    allocs.clear();
  }

  Status build_tri(IluLevelTri &T, const HostCSR &M, bool upper, const std::vector<int32_t> &pos) {
    const int32_t n = M.n;
    std::vector<int32_t> order, lvl_off, blk_lvl;
    int32_t nl = 0;
    IluDevice::levels(M, upper, std::vector<int32_t>{0, n}, order, lvl_off, blk_lvl, nl);
    std::vector<int32_t> padded;
    padded.reserve(order.size() + (size_t)nl * 32);
    for (int32_t l = 0; l + 1 < (int32_t)lvl_off.size(); l++) {
      for (int32_t q = lvl_off[l]; q < lvl_off[l + 1]; q++) padded.push_back(order[q]);
      while (padded.size() % 32) padded.push_back(-1);
    }
    T.nchunks = (int32_t)(padded.size() / 32);
    T.nlevels = nl;
    // the factor in slot order; fp16 values rounded once from fp64
    std::vector<int4> meta(padded.size());
    std::vector<double> v, dinv(upper ? padded.size() : 0, 1.0);
    std::vector<int32_t> idx;
    v.reserve(M.val.size());
    idx.reserve(M.idx.size());
    for (size_t q = 0; q < padded.size(); q++) {
      const int32_t i = padded[q];
      meta[q] = make_int4(-1, 0, 0, 0);
      if (i < 0) continue;
      const int32_t r0 = M.rptr[i], r1 = M.rptr[i + 1];
      meta[q].x = pos[i];
      meta[q].y = (int32_t)idx.size();
      if (!upper) {
        for (int32_t j = r0; j < r1 - 1; j++) {  // last entry is the unit diagonal
          v.push_back(M.val[j]);
          idx.push_back(pos[M.idx[j]]);
        }
      } else {
        for (int32_t j = r1 - 1; j > r0; j--) {  // first entry is the diagonal
          v.push_back(M.val[j]);
          idx.push_back(pos[M.idx[j]]);
        }
        dinv[q] = 1.0 / M.val[r0];
      }
      meta[q].z = (int32_t)idx.size();
    }
    const std::vector<int32_t> zeros(std::max(n, 1), 0);
    const std::vector<unsigned int> st(3, 0u);
    if (up(&T.meta, meta) != cudaSuccess || up(&T.idx, idx) != cudaSuccess || up(&T.flag, zeros) != cudaSuccess ||
        up(&T.state, st) != cudaSuccess)
      return fail(F3R_ERROR_CUDA, "ILU upload failed");
    F3R_TRY(half_copy(&T.val, v));
    if (upper) F3R_TRY(half_copy(&T.dinv, dinv));
    return F3R_SUCCESS;
  }

  Status half_copy(__half **d, const std::vector<double> &v);

  Status build(int sm_count, const HostCSR &Lh, const HostCSR &Uh, const std::vector<int32_t> &perm, bool permuted) {
    const int32_t n = Lh.n;
    this->n = n;
    scale_grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count * 8));
    std::vector<int32_t> pos(n);
    for (int32_t i = 0; i < n; i++) pos[i] = i;
    if (permuted)
      for (int32_t s = 0; s < n; s++) pos[perm[s]] = s;
    F3R_TRY(build_tri(L, Lh, false, pos));
    F3R_TRY(build_tri(U, Uh, true, pos));
    // warps for about four levels' chunks at a time: the frontier has work for
    // them, and few enough are left spinning ahead of it
    const int64_t chunks = std::max(L.nchunks, U.nchunks), levels = std::max(1, std::max(L.nlevels, U.nlevels));
    const int64_t warps = 4 * ((chunks + levels - 1) / levels);
    grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sm_count * 2, (warps + 7) / 8));
    return F3R_SUCCESS;
  }

  // out = U^-1 L^-1 x (tmp holds L^-1 x); ome (nullable) scales the result
  Status apply(cudaStream_t st, const __half *x, __half *tmp, __half *out, const __half *ome, int *err) const {
    k_trsv_level<false><<<grid, 256, 0, st>>>(L, x, tmp, err);
    k_trsv_level<true><<<grid, 256, 0, st>>>(U, tmp, out, err);
    // then the scaling, as the reference: hout *= ome[0] (work/src/f3r.cpp:216, 229)
    if (ome) k_half_scale<<<scale_grid, 256, 0, st>>>(out, ome, n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(F3R_ERROR_CUDA, std::string("ILU trsv launch: ") + cudaGetErrorString(e));
    return F3R_SUCCESS;
  }
};

// The level solve's flag wait on one flag (f3r_context_wait_probe): the
// flag holds gen when set, 0 otherwise.
__global__ void k_wait_probe(const int32_t *flag, unsigned int gen, int *err, unsigned long long limit_ns) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int32_t q[kLevelBatch] = {0};
  wait_flags(flag, q, 1, gen, err, limit_ns);
}

}  // namespace f3r
