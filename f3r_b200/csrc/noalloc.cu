// noalloc.cu -- a dot product that allocates nothing.
//
// Some callers cannot allocate device memory: code that runs inside a
// custom allocator's own bookkeeping, callers that have handed every byte of
// the device to a memory pool they do not control, and code paths that must
// not call cudaMalloc for latency or determinism reasons.  f3r_dot needs a
// context, and creating one allocates its reduction scratch.  This variant of
// the same reduction keeps that scratch in a fixed, file-scope device array
// instead: 256 bytes for the arrival counter plus 8192 partial sums (64 KB).
// Every GPU that loads the library holds that array until the process exits.
//
// The kernel gives each block a tile of 4096 elements, so one call covers at
// most 8192 * 4096 = 33,554,432 elements; larger n is rejected.  Calls share
// the array: two calls that overlap on the GPU (different streams, no
// ordering between them) race on it.  The counter is cleared at the start of
// every call; the partial sums are fully rewritten by each call.
#include <mutex>

#include <algorithm>
#include <string>

#include "device.cuh"
#include "internal.hpp"

namespace f3r {
namespace {

constexpr int64_t kNoAllocTile = 4096;   // elements reduced by one block
constexpr int64_t kNoAllocSlots = 8192;  // partial sums the scratch holds
constexpr size_t kNoAllocCounterBytes = 256;
constexpr size_t kNoAllocBytes = kNoAllocCounterBytes + kNoAllocSlots * sizeof(double);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void *g_noalloc_addr[64] = {};  // device address of the scratch, per device ordinal

// <x, y> over one 4096-element tile per block; the deterministic last-block
// reduction of device.cuh adds the per-block sums in block order and writes
// the result, widened to fp64, to the caller's device pointer.
template <typename T, typename Acc, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_dot_tiled(const T *__restrict__ x, const T *__restrict__ y, int64_t n,
                                                          GridRed gr, double *out) {
  Acc part[1] = {0};
  const int64_t base = (int64_t)blockIdx.x * kNoAllocTile;
  const int64_t end = min(base + kNoAllocTile, n);
  for (int64_t i = base + threadIdx.x; i < end; i += blockDim.x)
    part[0] = fmaT(to_acc<Acc>(x[i]), to_acc<Acc>(y[i]), part[0]);
  grid_reduce<Acc, 1, WARPS>(part, 1, gr, [out](Acc *tot) { *out = (double)tot[0]; });
}

// Device address of the scratch array for the current device.  The symbol's
// name is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, once per device, with that device current.
Status scratch_address(unsigned char **addr) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(F3R_ERROR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  void *p = (dev >= 0 && dev < 64) ? g_noalloc_addr[dev] : nullptr;
  if (!p) {
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(F3R_ERROR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    if (dev >= 0 && dev < 64) g_noalloc_addr[dev] = p;
  }
  *addr = static_cast<unsigned char *>(p);
  return F3R_SUCCESS;
}

}  // namespace
}  // namespace f3r

using namespace f3r;

extern "C" f3r_status f3r_dot_noalloc(f3r_dtype t, int64_t n, const void *x, const void *y, double *result,
                                      void *stream) {
  if (n < 0 || !result || (n > 0 && (!x || !y)))
    return fail(F3R_ERROR_INVALID_VALUE, "f3r_dot_noalloc: need n >= 0, a result pointer and, for n > 0, x and y");
  if (t != F3R_F64 && t != F3R_F32 && t != F3R_F16) return fail(F3R_ERROR_INVALID_VALUE, "f3r_dot_noalloc: bad dtype");
  const int64_t blocks = std::max<int64_t>(1, (n + kNoAllocTile - 1) / kNoAllocTile);
  if (blocks > kNoAllocSlots)
    return fail(F3R_ERROR_INVALID_VALUE,
                "f3r_dot_noalloc: n = " + std::to_string(n) + " exceeds the static scratch maximum of " +
                    std::to_string(kNoAllocSlots * kNoAllocTile) + " elements");
  unsigned char *base = nullptr;
  F3R_TRY(scratch_address(&base));
  unsigned int *ticket = reinterpret_cast<unsigned int *>(base);
  void *partials = base + kNoAllocCounterBytes;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return fail(F3R_ERROR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  const GridRed gr{partials, ticket};
  if (t == F3R_F64)
    k_dot_tiled<double, double, 8><<<(int)blocks, 256, 0, st>>>((const double *)x, (const double *)y, n, gr, result);
  else if (t == F3R_F32)
    k_dot_tiled<float, float, 8><<<(int)blocks, 256, 0, st>>>((const float *)x, (const float *)y, n, gr, result);
  else
    k_dot_tiled<__half, float, 8><<<(int)blocks, 256, 0, st>>>((const __half *)x, (const __half *)y, n, gr, result);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(F3R_ERROR_CUDA, std::string("f3r_dot_noalloc launch: ") + cudaGetErrorString(e));
  return F3R_SUCCESS;
}
