// device.cuh -- sm_100a device helpers: bulk-copy (TMA) + mbarrier PTX,
// warp reductions, deterministic last-block grid reductions, type casts.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace f3r {

// Device-side error codes written to the context's error word.
enum DevError : int { DEV_OK = 0, DEV_TIMEOUT_SPMV = 1, DEV_BREAKDOWN = 2, DEV_TIMEOUT_TRSV = 3, DEV_TIMEOUT_MMA = 4 };

// Threads per block of the elementwise / reduction kernels.
constexpr int kEwThreads = 256;

// Bound for every spin-wait on an mbarrier: ~2 s of %globaltimer.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// try_wait with a suspend-time hint: a thread whose phase has not completed
// is suspended by the hardware until the phase completes or about hint_ns
// have passed, instead of spinning through issue slots.
__device__ __forceinline__ bool mbar_try_wait_suspend(uint64_t *bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}
// Suspend hint of the bounded waits: long enough that a waiting warp leaves
// the schedulers to the working ones, short against the bound.
constexpr uint32_t kSuspendHintNs = 1000000u;
// Waits for the given phase parity with a time bound; false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait_suspend(bar, parity, kSuspendHintNs)) {
    if (global_ns() - t0 > kWaitLimitNs) return false;
  }
  return true;
}
// L2 policy for streamed-once data (matrix values and indices): evict first,
// so the gathered vector stays resident in L2.
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
// Non-tensor bulk copy global -> shared (the TMA unit), completion counted on
// an mbarrier.  dst, src 16-byte aligned; bytes a multiple of 16.  No
// multicast anywhere in this library.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                         uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

namespace {
// y = fp16(y * ome): the scaling the reference applies after a whole
// preconditioner solve (hout *= ome[0], work/src/f3r.cpp:216, 229)
__global__ void k_half_scale(__half *__restrict__ y, const __half *__restrict__ ome, int64_t n) {
  const float om = __half2float(*ome);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = __float2half_rn(__half2float(y[i]) * om);
}
}  // namespace

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---- scalar conversions -----------------------------------------------------
template <typename T> struct acc_of { using type = float; };
template <> struct acc_of<double> { using type = double; };

template <typename To> __device__ __forceinline__ To cvt(float v);
template <typename To> __device__ __forceinline__ To cvt(double v);
template <> __device__ __forceinline__ float cvt<float>(float v) { return v; }
template <> __device__ __forceinline__ double cvt<double>(float v) { return (double)v; }
template <> __device__ __forceinline__ __half cvt<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ float cvt<float>(double v) { return (float)v; }
template <> __device__ __forceinline__ double cvt<double>(double v) { return v; }
template <> __device__ __forceinline__ __half cvt<__half>(double v) { return __double2half(v); }
template <typename To> __device__ __forceinline__ To cvt(__half v);
template <> __device__ __forceinline__ __half cvt<__half>(__half v) { return v; }
template <> __device__ __forceinline__ float cvt<float>(__half v) { return __half2float(v); }

__device__ __forceinline__ float widen(float v) { return v; }
__device__ __forceinline__ double widen(double v) { return v; }
__device__ __forceinline__ float widen(__half v) { return __half2float(v); }

template <typename Acc> __device__ __forceinline__ Acc to_acc(double v) { return (Acc)v; }
template <typename Acc> __device__ __forceinline__ Acc to_acc(float v) { return (Acc)v; }
template <typename Acc> __device__ __forceinline__ Acc to_acc(__half v) { return (Acc)__half2float(v); }
template <> __device__ __forceinline__ __half to_acc<__half>(__half v) { return v; }

__device__ __forceinline__ float fmaT(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return __fma_rn(a, b, c); }

// acc + v x with one rounding.  Two fp16 operands go through sm_100's
// mixed-precision FMA (fp16 sources, fp32 addend and result): the product of
// two fp16 values is exact in fp32, so this is fmaf(float(v), float(x), acc)
// bit for bit, without the two conversions.
// Per-launch set-up of a product epilogue: an epilogue with a setup() method
// reads its loop-invariant device values there, once per thread, instead of
// once per row; the others have nothing to do.  Every kernel that takes an
// epilogue calls this first.
template <typename E> __device__ __forceinline__ auto epi_setup(E &e, int) -> decltype(e.setup(), void()) { e.setup(); }
template <typename E> __device__ __forceinline__ void epi_setup(E &, long) {}

template <typename Acc, typename V, typename X> __device__ __forceinline__ Acc fma_vx(V v, X x, Acc acc) {
  return fmaT(to_acc<Acc>(v), to_acc<Acc>(x), acc);
}
template <> __device__ __forceinline__ float fma_vx<float, __half, __half>(__half v, __half x, float acc) {
  asm("fma.rn.f32.f16 %0, %1, %2, %0;" : "+f"(acc) : "h"(__half_as_ushort(v)), "h"(__half_as_ushort(x)));
  return acc;
}


// ---- deterministic grid reduction --------------------------------------------
// Every block contributes NV partial sums; the last block to arrive adds the
// partials in block order and calls fin(totals) on thread 0.  The ticket
// counter is reset by the last block, so one counter serves back-to-back
// launches on a stream.
struct GridRed {
  void *partials;       // gridDim.x * nv elements of T
  unsigned int *ticket; // one counter per reduction site
};

template <typename T, int NV, int NWARPS, typename Fin>
__device__ __forceinline__ void grid_reduce(T (&v)[NV], int nv, GridRed gr, Fin fin) {
  __shared__ T sred[NWARPS][NV];
  __shared__ T stot[NV];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
    if (k < nv) {
      T s = warp_sum(v[k]);
      if (lane == 0) sred[warp][k] = s;
    }
  }
  __syncthreads();
  T *part = static_cast<T *>(gr.partials);
  if (threadIdx.x < nv) {
    T s = 0;
    for (int w = 0; w < NWARPS; w++) s += sred[w][threadIdx.x];
    part[(size_t)blockIdx.x * nv + threadIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int t = atomicAdd(gr.ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int k = 0; k < nv; k++) {
    T s = 0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) s += __ldcg(&part[(size_t)b * nv + k]);
    s = warp_sum(s);
    if (lane == 0) sred[warp][0] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      T t = 0;
      for (int w = 0; w < NWARPS; w++) t += sred[w][0];
      stot[k] = t;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *gr.ticket = 0;
    fin(stot);
  }
}

}  // namespace f3r
