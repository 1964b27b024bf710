// learned.cu -- a learned correction to SDAINV's values on its fixed pattern
// (the f3r_learned_* entry points of include/f3r_b200.h).  The reference has
// no counterpart: its innermost preconditioner is the plain SDAINV of
// preconditioner/ainv.hpp:27-65, applied as Z (W^T r) (work/src/f3r-gpu.cpp:
// 74, 215-216).
//
// For a 7-point matrix in natural order (strides 1, nx, nx*ny) SDAINV's
// factors have, per row, Z entries at column offsets {0, +1, +nx, +nx*ny} and
// W^T entries at {0, -1, -nx, -nx*ny}.  A small MLP maps row i's seven
// coefficients (offsets 0, -1, +1, -nx, +nx, -nx*ny, +nx*ny; 0 where absent)
// to eight corrections delta_i, one per factor slot (Z slots 0..3, W^T slots
// 4..7); every entry in a slot becomes v' = v (1 + delta).  The output layer
// starts at zero, so an untrained network is plain SDAINV.
//
// Training minimises, over residual / error pairs (r_p, e_p) of one system
// (A e = r), L = 1/P sum_p ||Z' (W'^T r_p) - e_p||^2 / ||e_p||^2: M = Z' W'^T
// should map a residual to its error.  Several systems of one grid shape are
// trained together as one block-diagonal system.  Kernels (fp32 master
// weights, fp64 sparse products):
//   forward    one thread per row, the weights in shared memory
//   pairs      u = W'^T r, y = Z' u, d = dL/dy, g = Z'^T d over all pairs
//              (blockIdx.y = pair); entry gradients dZ'_ij = sum_p d_i u_j and
//              dW'^T_jk = sum_p g_j r_k, folded into per-row output gradients
//              dO[row][slot] = dv' * v
//   backward   persistent blocks of 128 threads, one row each: the block
//              recomputes its tile's activations into shared memory, forms the
//              weight gradients as sums over the tile's rows into a shared
//              accumulator, and adds that to the global gradient once
//   Adam       one thread per parameter
// Inference runs the same network in BF16 on the tensor cores with fp32
// accumulation: tcgen05.mma with TMEM accumulators, one warpgroup per 128-row
// tile, the biases inside the MMAs (the default), or mma.sync m16n8k16, one
// warp per 16-row tile, the biases added in fp32.
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include <cuda_bf16.h>

#include "objects.cuh"

namespace f3r {

namespace {

constexpr int kH = 64;     // hidden width
constexpr int kIn = 7;     // coefficients per row
constexpr int kOut = 8;    // Z slots 0..3, W^T slots 4..7
constexpr int kRows = 128; // rows per tile in the training kernels
constexpr int kLdH = kH + 1, kLdO = kOut + 1;  // padded shared-memory rows (no bank conflicts)
// flat parameter layout: W1 (kH x kIn), b1, W2 (kH x kH), b2, W3 (kOut x kH), b3; W row-major (out x in)
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kOut * kH, kParams = oB3 + kOut;
constexpr size_t kBackSmem = sizeof(float) * (2 * kParams + 2 * kRows * kLdH + kRows * kLdO);

// One (possibly block-diagonal) system on the device: A, the factors with the
// slot of every entry, Z's transposed pattern, features, outputs, and the
// training pairs.
struct SysDev {
  int32_t n = 0, npairs = 0;
  int64_t znnz = 0, wnnz = 0;
  int32_t *ar = nullptr, *ai = nullptr;
  double *av = nullptr;
  int32_t *zr = nullptr, *zi = nullptr, *zs = nullptr;
  double *zv = nullptr;
  int32_t *wr = nullptr, *wi = nullptr, *ws = nullptr;
  double *wv = nullptr;
  int32_t *tr = nullptr, *ti = nullptr, *tk = nullptr;
  float *feat = nullptr, *out = nullptr, *dout = nullptr;
  double *zc = nullptr, *wc = nullptr;
  double *r = nullptr, *e = nullptr, *u = nullptr, *y = nullptr, *d = nullptr, *g = nullptr;  // n x npairs
  std::vector<void *> allocs;
  void release() {
    for (void *p : allocs) cudaFree(p);
    allocs.clear();
    *this = SysDev();
  }
  template <typename T> Status get(Context &c, T **p, size_t count) {
    F3R_TRY(c.alloc((void **)p, sizeof(T) * std::max<size_t>(count, 1)));
    allocs.push_back((void *)*p);
    return F3R_SUCCESS;
  }
  template <typename T> Status put(Context &c, T **p, const T *h, size_t count) {
    F3R_TRY(get(c, p, count));
    if (count) CUDA_TRY(cudaMemcpyAsync(*p, h, sizeof(T) * count, cudaMemcpyHostToDevice, c.stream));
    return F3R_SUCCESS;
  }
};

__device__ __forceinline__ float relu(float x) { return x > 0.f ? x : 0.f; }

// row i's coefficients by offset (0, -1, +1, -nx, +nx, -nx*ny, +nx*ny)
__global__ void k_features(int32_t n, int32_t nx, int32_t sxy, const int32_t *__restrict__ rp,
                           const int32_t *__restrict__ ci, const double *__restrict__ v, float *__restrict__ f) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float o[kIn] = {0, 0, 0, 0, 0, 0, 0};
  const int32_t offs[kIn] = {0, -1, 1, -nx, nx, -sxy, sxy};
  for (int32_t q = rp[i]; q < rp[i + 1]; q++) {
    const int32_t dd = ci[q] - (int32_t)i;
#pragma unroll
    for (int s = 0; s < kIn; s++)
      if (dd == offs[s]) o[s] = (float)v[q];
  }
#pragma unroll
  for (int s = 0; s < kIn; s++) f[i * kIn + s] = o[s];
}

__device__ __forceinline__ void load_params(float *sp, const float *__restrict__ p) {
  for (int k = threadIdx.x; k < kParams; k += blockDim.x) sp[k] = p[k];
  __syncthreads();
}

// o = W3 relu(W2 relu(W1 f + b1) + b2) + b3, one thread per row (fp32)
__global__ void __launch_bounds__(kRows) k_mlp_forward(int32_t n, const float *__restrict__ f,
                                                      const float *__restrict__ p, float *__restrict__ o) {
  __shared__ float sp[kParams];
  load_params(sp, p);
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float x[kIn], h1[kH], acc[kOut];
#pragma unroll
  for (int c = 0; c < kIn; c++) x[c] = f[i * kIn + c];
#pragma unroll
  for (int j = 0; j < kH; j++) {
    float s = sp[oB1 + j];
#pragma unroll
    for (int c = 0; c < kIn; c++) s = fmaf(sp[oW1 + j * kIn + c], x[c], s);
    h1[j] = relu(s);
  }
#pragma unroll
  for (int t = 0; t < kOut; t++) acc[t] = sp[oB3 + t];
  for (int k = 0; k < kH; k++) {
    float s = sp[oB2 + k];
#pragma unroll
    for (int j = 0; j < kH; j++) s = fmaf(sp[oW2 + k * kH + j], h1[j], s);
    const float h2 = relu(s);
#pragma unroll
    for (int t = 0; t < kOut; t++) acc[t] = fmaf(sp[oW3 + t * kH + k], h2, acc[t]);
  }
#pragma unroll
  for (int t = 0; t < kOut; t++) o[i * kOut + t] = acc[t];
}

// v' = v (1 + delta[row][slot0 + slot]) for every entry with a slot
__global__ void k_correct(int32_t n, const int32_t *__restrict__ rp, const int32_t *__restrict__ sl,
                          const double *__restrict__ v, const float *__restrict__ o, int slot0,
                          double *__restrict__ vc) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int32_t q = rp[i]; q < rp[i + 1]; q++)
    vc[q] = sl[q] >= 0 ? v[q] * (1.0 + (double)o[i * kOut + slot0 + sl[q]]) : v[q];
}

// y_p = M x_p for a CSR matrix, every pair p = blockIdx.y (row per thread, fp64)
__global__ void k_csr_mv(int32_t n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                         const double *__restrict__ v, const double *__restrict__ x, double *__restrict__ y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t off = (int64_t)blockIdx.y * n;
  double s = 0;
  for (int32_t q = rp[i]; q < rp[i + 1]; q++) s = fma(v[q], x[off + ci[q]], s);
  y[off + i] = s;
}

// g_p = Z'^T d_p through the transposed pattern (for column j: rows ti, entries tk)
__global__ void k_csr_mv_t(int32_t n, const int32_t *__restrict__ tr, const int32_t *__restrict__ ti,
                           const int32_t *__restrict__ tk, const double *__restrict__ zc,
                           const double *__restrict__ d, double *__restrict__ g) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t off = (int64_t)blockIdx.y * n;
  double s = 0;
  for (int32_t q = tr[j]; q < tr[j + 1]; q++) s = fma(zc[tk[q]], d[off + ti[q]], s);
  g[off + j] = s;
}

// d_p = 2 w (y_p - e_p) / ||e_p||^2 and the loss w sum_p ||y_p - e_p||^2 / ||e_p||^2
// (inv_ee[p] = 1 / ||e_p||^2), reduced into *loss
__global__ void k_loss_d(int32_t n, const double *__restrict__ y, const double *__restrict__ e,
                         const double *__restrict__ inv_ee, double w, double *__restrict__ d,
                         double *__restrict__ loss) {
  __shared__ double red[256];
  const int64_t off = (int64_t)blockIdx.y * n;
  const double wp = w * inv_ee[blockIdx.y];
  double acc = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double t = y[off + i] - e[off + i];
    d[off + i] = 2.0 * wp * t;
    acc += t * t;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] * wp);
}

// per-row output gradients summed over the pairs: for a Z entry (i, j) in
// slot s, dO[i][s] = sum_p d_p[i] u_p[j] z_ij; for a W^T entry (j, k),
// dO[j][4 + s] = sum_p g_p[j] r_p[k] w_jk
__global__ void k_entry_grad(int32_t n, int32_t npairs, const int32_t *__restrict__ zr,
                             const int32_t *__restrict__ zi, const int32_t *__restrict__ zs,
                             const double *__restrict__ zv, const int32_t *__restrict__ wr,
                             const int32_t *__restrict__ wi, const int32_t *__restrict__ ws,
                             const double *__restrict__ wv, const double *__restrict__ d,
                             const double *__restrict__ u, const double *__restrict__ g,
                             const double *__restrict__ r, float *__restrict__ dout) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc[kOut] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int32_t q = zr[i]; q < zr[i + 1]; q++) {
    const int s = zs[q];
    if (s < 0) continue;
    double t = 0;
    for (int p = 0; p < npairs; p++) t = fma(d[(int64_t)p * n + i], u[(int64_t)p * n + zi[q]], t);
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (s == k) acc[k] = fma(t, zv[q], acc[k]);
  }
  for (int32_t q = wr[i]; q < wr[i + 1]; q++) {
    const int s = ws[q];
    if (s < 0) continue;
    double t = 0;
    for (int p = 0; p < npairs; p++) t = fma(g[(int64_t)p * n + i], r[(int64_t)p * n + wi[q]], t);
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (s == k) acc[4 + k] = fma(t, wv[q], acc[4 + k]);
  }
#pragma unroll
  for (int k = 0; k < kOut; k++) dout[i * kOut + k] = (float)acc[k];
}

// Backward through the MLP.  Persistent blocks of kRows threads walk tiles of
// kRows rows (thread t = row t of the tile); rows past n contribute zeros.
// Shared memory: the parameters, their gradient accumulator, H1 / H2 (the
// activations, overwritten by the pre-activation gradients) and dO.
__global__ void __launch_bounds__(kRows) k_mlp_backward(int32_t n, const float *__restrict__ f,
                                                       const float *__restrict__ p,
                                                       const float *__restrict__ dout, float *__restrict__ grad) {
  extern __shared__ float sm[];
  float *sp = sm;                   // kParams
  float *G = sp + kParams;          // kParams (gradient accumulator)
  float *H1 = G + kParams;          // kRows x kLdH
  float *H2 = H1 + kRows * kLdH;    // kRows x kLdH
  float *DO = H2 + kRows * kLdH;    // kRows x kLdO
  for (int k = threadIdx.x; k < kParams; k += blockDim.x) {
    sp[k] = p[k];
    G[k] = 0.f;
  }
  __syncthreads();
  const int t = threadIdx.x;
  const int64_t ntiles = (n + kRows - 1) / kRows;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t row0 = tile * kRows, i = row0 + t;
    const bool live = i < n;
    float x[kIn];
#pragma unroll
    for (int c = 0; c < kIn; c++) x[c] = live ? f[i * kIn + c] : 0.f;
    for (int j = 0; j < kH; j++) {
      float s = sp[oB1 + j];
#pragma unroll
      for (int c = 0; c < kIn; c++) s = fmaf(sp[oW1 + j * kIn + c], x[c], s);
      H1[t * kLdH + j] = live ? relu(s) : 0.f;
    }
    for (int k = 0; k < kH; k++) {
      float s = sp[oB2 + k];
      for (int j = 0; j < kH; j++) s = fmaf(sp[oW2 + k * kH + j], H1[t * kLdH + j], s);
      H2[t * kLdH + k] = live ? relu(s) : 0.f;
    }
#pragma unroll
    for (int s = 0; s < kOut; s++) DO[t * kLdO + s] = live ? dout[i * kOut + s] : 0.f;
    __syncthreads();
    // dW3 (kOut x kH) and db3 over the tile's rows
    for (int q = t; q < kOut * kH + kOut; q += kRows) {
      float s = 0;
      if (q < kOut * kH) {
        const int so = q / kH, k = q % kH;
        for (int rr = 0; rr < kRows; rr++) s = fmaf(DO[rr * kLdO + so], H2[rr * kLdH + k], s);
        G[oW3 + q] += s;
      } else {
        const int so = q - kOut * kH;
        for (int rr = 0; rr < kRows; rr++) s += DO[rr * kLdO + so];
        G[oB3 + so] += s;
      }
    }
    __syncthreads();
    // dh2pre = (W3^T dO) [h2 > 0], in place of h2 (own row only)
    for (int k = 0; k < kH; k++) {
      float s = 0;
#pragma unroll
      for (int so = 0; so < kOut; so++) s = fmaf(sp[oW3 + so * kH + k], DO[t * kLdO + so], s);
      H2[t * kLdH + k] = H2[t * kLdH + k] > 0.f ? s : 0.f;
    }
    __syncthreads();
    // dW2 (kH x kH) = dH2pre^T H1, db2
    for (int q = t; q < kH * kH + kH; q += kRows) {
      float s = 0;
      if (q < kH * kH) {
        const int k = q / kH, j = q % kH;
        for (int rr = 0; rr < kRows; rr++) s = fmaf(H2[rr * kLdH + k], H1[rr * kLdH + j], s);
        G[oW2 + q] += s;
      } else {
        const int k = q - kH * kH;
        for (int rr = 0; rr < kRows; rr++) s += H2[rr * kLdH + k];
        G[oB2 + k] += s;
      }
    }
    __syncthreads();
    // dh1pre = (W2^T dh2pre) [h1 > 0], in place of h1 (own row only)
    for (int j = 0; j < kH; j++) {
      float s = 0;
      for (int k = 0; k < kH; k++) s = fmaf(sp[oW2 + k * kH + j], H2[t * kLdH + k], s);
      H1[t * kLdH + j] = H1[t * kLdH + j] > 0.f ? s : 0.f;
    }
    __syncthreads();
    // dW1 (kH x kIn) = dH1pre^T X, db1 (X read again from global memory)
    for (int q = t; q < kH * kIn + kH; q += kRows) {
      float s = 0;
      if (q < kH * kIn) {
        const int j = q / kIn, c = q % kIn;
        for (int rr = 0; rr < kRows; rr++)
          if (row0 + rr < n) s = fmaf(H1[rr * kLdH + j], f[(row0 + rr) * kIn + c], s);
        G[oW1 + q] += s;
      } else {
        const int j = q - kH * kIn;
        for (int rr = 0; rr < kRows; rr++) s += H1[rr * kLdH + j];
        G[oB1 + j] += s;
      }
    }
    __syncthreads();
  }
  for (int k = threadIdx.x; k < kParams; k += blockDim.x) atomicAdd(&grad[k], G[k]);
}

__global__ void k_adam(int32_t np, float *__restrict__ p, float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float c1, float c2, float eps) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= np) return;
  const float gk = g[k];
  m[k] = b1 * m[k] + (1.f - b1) * gk;
  v[k] = b2 * v[k] + (1.f - b2) * gk * gk;
  p[k] -= lr * (m[k] / c1) / (sqrtf(v[k] / c2) + eps);
  g[k] = 0.f;
}

// ---- BF16 tensor-core inference --------------------------------------------
// mma.sync m16n8k16 (bf16 inputs, fp32 accumulation).  Fragment layout (PTX
// ISA, "Matrix Fragments for mma.m16n8k16"), g = lane / 4, c = lane % 4:
// A (16 x 16, row-major) regs (g, 2c..2c+1), (g+8, 2c..), (g, 2c+8..),
// (g+8, 2c+8..); B (16 x 8) regs (k 2c..2c+1, n g), (k 2c+8.., n g);
// C (16 x 8) c0,c1 = (g, 2c..2c+1), c2,c3 = (g+8, 2c..).  Two adjacent C
// tiles (16 columns) are the A fragment of the next layer's k-chunk, so the
// activations never leave registers.  B = W^T, so a B register is two
// consecutive entries of a row of W (out x in, row-major in shared memory).
constexpr int kLd1 = 24, kLd2 = kH + 8;  // bf16 row strides: conflict-free B-fragment reads

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t wpair(const __nv_bfloat16 *w, int ld, int row, int col) {
  return *reinterpret_cast<const uint32_t *>(w + row * ld + col);
}
// relu of two adjacent 16 x 8 C tiles as one A fragment
__device__ __forceinline__ void to_a(uint32_t (&a)[4], const float (&lo)[4], const float (&hi)[4]) {
  a[0] = pack_bf16(relu(lo[0]), relu(lo[1]));
  a[1] = pack_bf16(relu(lo[2]), relu(lo[3]));
  a[2] = pack_bf16(relu(hi[0]), relu(hi[1]));
  a[3] = pack_bf16(relu(hi[2]), relu(hi[3]));
}

__global__ void __launch_bounds__(128) k_mlp_infer_bf16(int32_t n, const float *__restrict__ f,
                                                        const float *__restrict__ p, float *__restrict__ o) {
  __shared__ __align__(16) __nv_bfloat16 w1[kH * kLd1], w2[kH * kLd2], w3[kOut * kLd2];
  __shared__ float b1s[kH], b2s[kH], b3s[kOut];
  for (int q = threadIdx.x; q < kH * kLd1; q += blockDim.x) {
    const int j = q / kLd1, c = q % kLd1;
    w1[q] = __float2bfloat16_rn(c < kIn ? p[oW1 + j * kIn + c] : 0.f);
  }
  for (int q = threadIdx.x; q < kH * kLd2; q += blockDim.x) {
    const int k = q / kLd2, j = q % kLd2;
    w2[q] = __float2bfloat16_rn(j < kH ? p[oW2 + k * kH + j] : 0.f);
  }
  for (int q = threadIdx.x; q < kOut * kLd2; q += blockDim.x) {
    const int s = q / kLd2, k = q % kLd2;
    w3[q] = __float2bfloat16_rn(k < kH ? p[oW3 + s * kH + k] : 0.f);
  }
  for (int q = threadIdx.x; q < kH; q += blockDim.x) {
    b1s[q] = p[oB1 + q];
    b2s[q] = p[oB2 + q];
  }
  if (threadIdx.x < kOut) b3s[threadIdx.x] = p[oB3 + threadIdx.x];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
  // persistent grid: the weights above are staged once per CTA, then each
  // warp walks 16-row tiles
#pragma unroll 1
  for (int64_t r0 = ((int64_t)blockIdx.x * 4 + warp) * 16; r0 < n; r0 += (int64_t)gridDim.x * 64) {
  const int64_t ra = r0 + g, rb = r0 + g + 8;
  auto fx = [&](int64_t r, int col) { return (r < n && col < kIn) ? f[r * kIn + col] : 0.f; };
  // layer 1: [16 x 16 (7 inputs, zero-padded)] x [16 x 64]
  const uint32_t a1[4] = {pack_bf16(fx(ra, 2 * c), fx(ra, 2 * c + 1)), pack_bf16(fx(rb, 2 * c), fx(rb, 2 * c + 1)),
                          pack_bf16(fx(ra, 2 * c + 8), fx(ra, 2 * c + 9)),
                          pack_bf16(fx(rb, 2 * c + 8), fx(rb, 2 * c + 9))};
  float h[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; nt++) {
    h[nt][0] = h[nt][2] = b1s[nt * 8 + 2 * c];
    h[nt][1] = h[nt][3] = b1s[nt * 8 + 2 * c + 1];
    mma_bf16(h[nt], a1, wpair(w1, kLd1, nt * 8 + g, 2 * c), wpair(w1, kLd1, nt * 8 + g, 2 * c + 8));
  }
  // layer 2: [16 x 64] x [64 x 64]
  uint32_t a[4][4];
#pragma unroll
  for (int kk = 0; kk < 4; kk++) to_a(a[kk], h[2 * kk], h[2 * kk + 1]);
#pragma unroll
  for (int nt = 0; nt < 8; nt++) {
    h[nt][0] = h[nt][2] = b2s[nt * 8 + 2 * c];
    h[nt][1] = h[nt][3] = b2s[nt * 8 + 2 * c + 1];
#pragma unroll
    for (int kk = 0; kk < 4; kk++)
      mma_bf16(h[nt], a[kk], wpair(w2, kLd2, nt * 8 + g, kk * 16 + 2 * c),
               wpair(w2, kLd2, nt * 8 + g, kk * 16 + 2 * c + 8));
  }
  // layer 3: [16 x 64] x [64 x 8]
#pragma unroll
  for (int kk = 0; kk < 4; kk++) to_a(a[kk], h[2 * kk], h[2 * kk + 1]);
  float y[4] = {b3s[2 * c], b3s[2 * c + 1], b3s[2 * c], b3s[2 * c + 1]};
#pragma unroll
  for (int kk = 0; kk < 4; kk++)
    mma_bf16(y, a[kk], wpair(w3, kLd2, g, kk * 16 + 2 * c), wpair(w3, kLd2, g, kk * 16 + 2 * c + 8));
  if (ra < n) {
    o[ra * kOut + 2 * c] = y[0];
    o[ra * kOut + 2 * c + 1] = y[1];
  }
  if (rb < n) {
    o[rb * kOut + 2 * c] = y[2];
    o[rb * kOut + 2 * c + 1] = y[3];
  }
  }
}

// ---- BF16 inference on the 5th-generation tensor cores (tcgen05) ----------
// A warpgroup (128 threads) works one 128-row tile; a CTA holds two warpgroups
// that share the staged weights and own 64 tensor-memory columns each.  Every
// layer is a tcgen05.mma chain D[128 x N] = A[128 x K] . B[K x N] issued by one
// thread, A (activations) and B (the weights, stored out x in = N x K) in
// shared memory in the K-major no-swizzle canonical layout, D (fp32) in tensor
// memory: row t of the tile is TMEM lane t, read back by thread t with
// tcgen05.ld.  Layer 1: K 16 (the 7 inputs, two bias columns, zeros), N 64;
// layer 2: K 64 + 16, N 64; layer 3: K 64 + 16, N 16 (8 outputs and 8 zero
// weight rows).  Each bias is a weight against a constant one, split into two
// bf16 parts (hi = bf16(b), lo = bf16(b - hi)), so the accumulator holds
// W x + b and the epilogue of a layer only applies relu and stores its row as
// bf16 into the next layer's A (one cvt.rn.relu.bf16x2 per two values).
//
// Canonical K-major layout without swizzle: 8 x 8 bf16 core matrices of 128
// contiguous bytes (row r % 8 at 16 r bytes); the K/8 core matrices of an
// 8-row group follow each other at LBO = 128 bytes and the 8-row groups at
// SBO = 16 K bytes.  One MMA instruction covers K = 16 (two core matrices), so
// the k-th instruction of a chain starts 256 k bytes further.
constexpr int kTcRows = 128;        // rows per tile: MMA M, TMEM lanes
constexpr int kTcGroups = 2;        // warpgroups (tiles in flight) per CTA
constexpr int kTcCols = 64;         // TMEM columns per warpgroup
constexpr int kTcK1 = 16, kTcN3 = 16, kTcKB = 16;
// bytes of the operands: weights W1 (64 x 16), W2 (64 x 64), W3 (16 x 64); the
// bias blocks WB2 (64 x 16), WB3 (16 x 16) and the constant ONES (128 x 16,
// columns 0 and 1 one); per warpgroup the activations A2 (128 x 64), whose
// first 4 KB hold layer 1's A1 (128 x 16) until layer 1's MMA has read it
constexpr uint32_t kTcW1 = kH * kTcK1 * 2, kTcW2 = kH * kH * 2, kTcW3 = kTcN3 * kH * 2;
constexpr uint32_t kTcWB2 = kH * kTcKB * 2, kTcWB3 = kTcN3 * kTcKB * 2, kTcOnes = kTcRows * kTcKB * 2;
constexpr uint32_t kTcA2 = kTcRows * kH * 2;
constexpr uint32_t kTcOffW2 = kTcW1, kTcOffW3 = kTcOffW2 + kTcW2, kTcOffWB2 = kTcOffW3 + kTcW3,
                   kTcOffWB3 = kTcOffWB2 + kTcWB2, kTcOffOnes = kTcOffWB3 + kTcWB3, kTcOffA = kTcOffOnes + kTcOnes;
constexpr uint32_t kTcOffBar = kTcOffA + kTcGroups * kTcA2;
constexpr size_t kTcSmem = kTcOffBar + kTcGroups * 8 + 16;
// Four CTAs fill the 512 TMEM columns of an SM; a fifth never fits beside them
// (shared memory), so no allocation waits on another CTA.
constexpr int kTcCtasPerSm = 4;
static_assert(kTcCtasPerSm * kTcGroups * kTcCols == 512, "TMEM columns of an SM");
static_assert(kTcCtasPerSm * (kTcSmem + 1024) <= 228 * 1024, "four CTAs fit on an SM");
static_assert((kTcCtasPerSm + 1) * (kTcSmem + 1024) > 228 * 1024, "a fifth CTA would fit on an SM");
static_assert(kTcOffA % 128 == 0 && kTcOffOnes % 128 == 0 && kTcOffWB2 % 128 == 0 && kTcOffWB3 % 128 == 0 &&
                  kTcOffBar % 8 == 0,
              "operand alignment");

// byte offset of element (r, k) of a K-major no-swizzle operand with K columns
__host__ __device__ constexpr uint32_t kmaj_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
// shared-memory matrix descriptor (tcgen05): start address, LBO, SBO (all
// >> 4), version 1 (bits 46-47), base offset 0, no swizzle (bits 61-63 = 0)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         (1ull << 46);
}
// instruction descriptor, kind::f16: fp32 D (bits 4-5 = 1), bf16 A and B (bits
// 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accum)
      : "memory");
}
// arrives once on bar when every MMA this thread issued before it completes
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// 16 consecutive fp32 columns of this thread's TMEM lane; the wait takes the
// registers as operands, so no use of them is scheduled before it
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
// barrier over one warpgroup (named barrier id) that also ANDs a flag
__device__ __forceinline__ bool group_sync_and(int id, bool ok) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.b32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, 128, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(out)
      : "r"((uint32_t)ok), "r"(id)
      : "memory");
  return out != 0;
}
// relu of two fp32 values rounded to bf16 and packed (lo in the low half) in one
// instruction: for finite values the bits of pack_bf16(relu(lo), relu(hi))
__device__ __forceinline__ uint32_t pack_relu_bf16(float lo, float hi) {
  uint32_t d;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}
// relu of 16 accumulator columns of a row (the bias is in the accumulator),
// stored as bf16 at A2 columns c0..c0+15
__device__ __forceinline__ void tc_epilogue16(unsigned char *a2, int row, int c0, const float (&v)[16]) {
  uint32_t p[8];
#pragma unroll
  for (int i = 0; i < 8; i++) p[i] = pack_relu_bf16(v[2 * i], v[2 * i + 1]);
  *reinterpret_cast<uint4 *>(a2 + kmaj_off(row, c0, kH)) = make_uint4(p[0], p[1], p[2], p[3]);
  *reinterpret_cast<uint4 *>(a2 + kmaj_off(row, c0 + 8, kH)) = make_uint4(p[4], p[5], p[6], p[7]);
}
// a bias as two bf16 parts (hi + lo carries 16 of its bits)
__device__ __forceinline__ void split_bf16(float b, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
  hi = __float2bfloat16_rn(b);
  lo = __float2bfloat16_rn(b - __bfloat162float(hi));
}

__global__ void __launch_bounds__(kTcRows * kTcGroups, kTcCtasPerSm)
    k_mlp_infer_tc(int32_t n, const float *__restrict__ f, const float *__restrict__ p, float *__restrict__ o,
                   int *err) {
  extern __shared__ __align__(1024) unsigned char tcs[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(tcs + kTcOffBar);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tcs + kTcOffBar + kTcGroups * 8);
  const int tid = threadIdx.x & (kTcRows - 1), g = threadIdx.x / kTcRows, warp = threadIdx.x >> 5;
  // weights (bf16, canonical layout; the padding rows and columns zero).  The
  // biases enter the MMAs: layer 1 through columns 7 and 8 of W1 (hi and lo
  // parts) against ones in columns 7 and 8 of A1; layers 2 and 3 through one
  // more K = 16 step, ONES x WB.
  auto bf = [](float v) { return __float2bfloat16_rn(v); };
  for (int q = threadIdx.x; q < kH * kTcK1; q += blockDim.x) {
    const int j = q / kTcK1, c = q % kTcK1;
    __nv_bfloat16 v = bf(0.f), hi, lo;
    if (c < kIn) v = bf(p[oW1 + j * kIn + c]);
    else if (c == kIn || c == kIn + 1) {
      split_bf16(p[oB1 + j], hi, lo);
      v = c == kIn ? hi : lo;
    }
    *reinterpret_cast<__nv_bfloat16 *>(tcs + kmaj_off(j, c, kTcK1)) = v;
  }
  for (int q = threadIdx.x; q < kH * kH; q += blockDim.x) {
    const int j = q / kH, c = q % kH;
    *reinterpret_cast<__nv_bfloat16 *>(tcs + kTcOffW2 + kmaj_off(j, c, kH)) = bf(p[oW2 + q]);
  }
  for (int q = threadIdx.x; q < kTcN3 * kH; q += blockDim.x) {
    const int s = q / kH, c = q % kH;
    *reinterpret_cast<__nv_bfloat16 *>(tcs + kTcOffW3 + kmaj_off(s, c, kH)) = bf(s < kOut ? p[oW3 + s * kH + c] : 0.f);
  }
  for (int q = threadIdx.x; q < kH * kTcKB; q += blockDim.x) {
    const int j = q / kTcKB, c = q % kTcKB;
    __nv_bfloat16 hi, lo;
    split_bf16(p[oB2 + j], hi, lo);
    *reinterpret_cast<__nv_bfloat16 *>(tcs + kTcOffWB2 + kmaj_off(j, c, kTcKB)) = c == 0 ? hi : c == 1 ? lo : bf(0.f);
  }
  for (int q = threadIdx.x; q < kTcN3 * kTcKB; q += blockDim.x) {
    const int s = q / kTcKB, c = q % kTcKB;
    __nv_bfloat16 hi = bf(0.f), lo = bf(0.f);
    if (s < kOut) split_bf16(p[oB3 + s], hi, lo);
    *reinterpret_cast<__nv_bfloat16 *>(tcs + kTcOffWB3 + kmaj_off(s, c, kTcKB)) = c == 0 ? hi : c == 1 ? lo : bf(0.f);
  }
  for (int q = threadIdx.x; q < kTcRows * kTcKB; q += blockDim.x) {
    const int r = q / kTcKB, c = q % kTcKB;
    *reinterpret_cast<__nv_bfloat16 *>(tcs + kTcOffOnes + kmaj_off(r, c, kTcKB)) = bf(c < 2 ? 1.f : 0.f);
  }
  // A1 (layer 1's operand) in the first 4 KB of A2: features in columns 0..6,
  // ones in 7 and 8, zeros beyond; A2 overwrites it after layer 1's MMA
  unsigned char *a2 = tcs + kTcOffA + g * kTcA2, *a1 = a2;
  const uint32_t one = pack_bf16(1.f, 0.f);
  if (threadIdx.x == 0) {
    for (int q = 0; q < kTcGroups; q++) mbar_init(&bars[q], 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTcCols * kTcGroups)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot + g * kTcCols;     // this warpgroup's columns, lane 0
  const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16);  // this warp's 32 lanes
  const uint32_t sa1 = smem_u32(a1), sa2 = smem_u32(a2), sw = smem_u32(tcs);
  const uint64_t dA1 = umma_desc(sa1, 128, kTcK1 * 16), dW1 = umma_desc(sw, 128, kTcK1 * 16);
  const uint64_t dA2 = umma_desc(sa2, 128, kH * 16), dW2 = umma_desc(sw + kTcOffW2, 128, kH * 16),
                 dW3 = umma_desc(sw + kTcOffW3, 128, kH * 16);
  const uint64_t dOnes = umma_desc(sw + kTcOffOnes, 128, kTcKB * 16), dB2 = umma_desc(sw + kTcOffWB2, 128, kTcKB * 16),
                 dB3 = umma_desc(sw + kTcOffWB3, 128, kTcKB * 16);
  constexpr uint32_t i64 = umma_idesc_bf16(kTcRows, kH), i16 = umma_idesc_bf16(kTcRows, kTcN3);
  const bool issuer = tid == 0;
  const int bar_id = 1 + g;
  uint32_t phase = 0;
  bool ok = true, pending = false;
  const int64_t ntiles = (n + kTcRows - 1) / kTcRows, stride = (int64_t)gridDim.x * kTcGroups;
  int64_t tile = (int64_t)blockIdx.x * kTcGroups + g;
  float fx[kIn];
  auto fetch = [&](int64_t t) {
    const int64_t r = t * kTcRows + tid;
#pragma unroll
    for (int c = 0; c < kIn; c++) fx[c] = (t < ntiles && r < n) ? f[r * kIn + c] : 0.f;
  };
  fetch(tile);
  // one MMA chain: issue, commit, and the warpgroup's wait for its completion
  auto chain = [&](auto issue) -> bool {
    fence_proxy_async_smem();
    tc_fence_before();
    group_sync_and(bar_id, true);
    if (issuer) {
      tc_fence_after();
      issue();
      umma_commit(&bars[g]);
    }
    pending = true;
    const bool done = mbar_wait_bounded(&bars[g], phase);
    if (!group_sync_and(bar_id, done)) return false;
    phase ^= 1u;
    pending = false;
    tc_fence_after();
    return true;
  };
#pragma unroll 1
  for (; tile < ntiles; tile += stride) {
    *reinterpret_cast<uint4 *>(a1 + kmaj_off(tid, 0, kTcK1)) =
        make_uint4(pack_bf16(fx[0], fx[1]), pack_bf16(fx[2], fx[3]), pack_bf16(fx[4], fx[5]), pack_bf16(fx[6], 1.f));
    *reinterpret_cast<uint4 *>(a1 + kmaj_off(tid, 8, kTcK1)) = make_uint4(one, 0, 0, 0);
    fetch(tile + stride);  // the next tile's rows, in flight behind this tile's chains
    if (!(ok = chain([&] { umma_bf16(tmem, dA1, dW1, i64, 0); }))) break;
#pragma unroll
    for (int q = 0; q < kH / 16; q++) {
      float v[16];
      tmem_ld16(lane_addr + q * 16, v);
      tc_epilogue16(a2, tid, q * 16, v);
    }
    if (!(ok = chain([&] {
            for (int k = 0; k < kH / 16; k++) umma_bf16(tmem, dA2 + 16 * k, dW2 + 16 * k, i64, k > 0);
            umma_bf16(tmem, dOnes, dB2, i64, 1);  // + b2
          })))
      break;
#pragma unroll
    for (int q = 0; q < kH / 16; q++) {
      float v[16];
      tmem_ld16(lane_addr + q * 16, v);
      tc_epilogue16(a2, tid, q * 16, v);
    }
    if (!(ok = chain([&] {
            for (int k = 0; k < kH / 16; k++) umma_bf16(tmem, dA2 + 16 * k, dW3 + 16 * k, i16, k > 0);
            umma_bf16(tmem, dOnes, dB3, i16, 1);  // + b3
          })))
      break;
    float y[16];
    tmem_ld16(lane_addr, y);
    const int64_t r = tile * kTcRows + tid;
    if (r < n) {
      float4 *dst = reinterpret_cast<float4 *>(o + r * kOut);
      dst[0] = make_float4(y[0], y[1], y[2], y[3]);
      dst[1] = make_float4(y[4], y[5], y[6], y[7]);
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, (int)DEV_TIMEOUT_MMA);
    if (pending) mbar_wait_bounded(&bars[g], phase);  // the chain still in flight (bounded)
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot), "r"(kTcCols * kTcGroups)
                 : "memory");
  }
}

// slot of every entry: the index of (col - row) in the factor's offset list, or -1
std::vector<int32_t> slots(const f3r_csr &m, const int32_t (&offs)[4]) {
  std::vector<int32_t> s(m.nnz, -1);
  for (int32_t i = 0; i < m.nrows; i++)
    for (int32_t q = m.rptr[i]; q < m.rptr[i + 1]; q++)
      for (int k = 0; k < 4; k++)
        if (m.idx[q] - i == offs[k]) s[q] = k;
  return s;
}

// uploads A, the factors (with slots and Z's transposed pattern) and computes
// the features; the pair buffers are left to the caller
Status load_system(Context &c, SysDev &s, const f3r_csr *a, int32_t nx, int32_t ny, const f3r_csr *z,
                   const f3r_csr *wt) {
  F3R_TRY(check_csr(a));
  F3R_TRY(check_csr(z));
  F3R_TRY(check_csr(wt));
  const int32_t n = a->nrows;
  if (a->ncols != n || z->nrows != n || wt->nrows != n || z->ncols != n || wt->ncols != n)
    return fail(F3R_ERROR_INVALID_VALUE, "the matrix and its factors must be square and of one size");
  if (nx < 1 || ny < 1 || (int64_t)nx * ny > std::max(n, 1))
    return fail(F3R_ERROR_INVALID_VALUE, "grid strides nx, ny must satisfy 1 <= nx * ny <= n");
  s.release();
  s.n = n;
  s.znnz = z->nnz;
  s.wnnz = wt->nnz;
  const int32_t sxy = nx * ny;
  const int32_t zo[4] = {0, 1, nx, sxy}, wo[4] = {0, -1, -nx, -sxy};
  const std::vector<int32_t> zs = slots(*z, zo), ws = slots(*wt, wo);
  std::vector<int32_t> tr(n + 1, 0), ti(z->nnz), tk(z->nnz);
  for (int32_t q = 0; q < z->nnz; q++) tr[z->idx[q] + 1]++;
  for (int32_t j = 0; j < n; j++) tr[j + 1] += tr[j];
  {
    std::vector<int32_t> fill(tr.begin(), tr.end() - 1);
    for (int32_t i = 0; i < n; i++)
      for (int32_t q = z->rptr[i]; q < z->rptr[i + 1]; q++) {
        const int32_t at = fill[z->idx[q]]++;
        ti[at] = i;
        tk[at] = q;
      }
  }
  F3R_TRY(s.put(c, &s.ar, a->rptr, (size_t)n + 1));
  F3R_TRY(s.put(c, &s.ai, a->idx, (size_t)a->nnz));
  F3R_TRY(s.put(c, &s.av, a->val, (size_t)a->nnz));
  F3R_TRY(s.put(c, &s.zr, z->rptr, (size_t)n + 1));
  F3R_TRY(s.put(c, &s.zi, z->idx, (size_t)z->nnz));
  F3R_TRY(s.put(c, &s.zs, zs.data(), zs.size()));
  F3R_TRY(s.put(c, &s.zv, z->val, (size_t)z->nnz));
  F3R_TRY(s.put(c, &s.wr, wt->rptr, (size_t)n + 1));
  F3R_TRY(s.put(c, &s.wi, wt->idx, (size_t)wt->nnz));
  F3R_TRY(s.put(c, &s.ws, ws.data(), ws.size()));
  F3R_TRY(s.put(c, &s.wv, wt->val, (size_t)wt->nnz));
  F3R_TRY(s.put(c, &s.tr, tr.data(), tr.size()));
  F3R_TRY(s.put(c, &s.ti, ti.data(), ti.size()));
  F3R_TRY(s.put(c, &s.tk, tk.data(), tk.size()));
  F3R_TRY(s.get(c, &s.feat, (size_t)n * kIn));
  F3R_TRY(s.get(c, &s.out, (size_t)n * kOut));
  F3R_TRY(s.get(c, &s.dout, (size_t)n * kOut));
  F3R_TRY(s.get(c, &s.zc, (size_t)z->nnz));
  F3R_TRY(s.get(c, &s.wc, (size_t)wt->nnz));
  if (n > 0)
    launch_k(c, k_features, (int)cdiv(n, 256), 256, 0, c.stream, n, nx, sxy, (const int32_t *)s.ar,
             (const int32_t *)s.ai, (const double *)s.av, s.feat);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(c.stream));  // the host vectors above go out of scope
  return F3R_SUCCESS;
}

}  // namespace

}  // namespace f3r

using namespace f3r;

struct f3r_learned {
  f3r_context *ctx = nullptr;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  double *loss = nullptr;         // device loss scalars (one per training step)
  int32_t loss_cap = 0;
  double *inv_ee = nullptr;       // 1 / ||e_p||^2 per pair
  int64_t steps = 0;
  int grid_back = 0;              // persistent grid of the backward kernel
  SysDev train;                   // the training system and its pairs
};

namespace {

// forward pass and corrected factors of a loaded system; mode 0: the fp32
// training forward pass, 1: BF16 inference on tcgen05, 2: BF16 inference on
// mma.sync
Status forward(Context &c, const float *params, SysDev &s, int mode) {
  if (s.n == 0) return F3R_SUCCESS;
  // inference: a persistent grid, each CTA staging the weights once
  if (mode == 1) {
    const int64_t tiles = cdiv(s.n, kTcRows);
    launch_k(c, k_mlp_infer_tc, (int)std::min<int64_t>(cdiv(tiles, kTcGroups), (int64_t)c.sm_count * kTcCtasPerSm),
             kTcRows * kTcGroups, kTcSmem, c.stream, s.n, (const float *)s.feat, params, s.out, c.err);
  } else if (mode == 2)
    launch_k(c, k_mlp_infer_bf16, (int)std::min<int64_t>(cdiv(s.n, 64), (int64_t)c.sm_count * 8), 128, 0, c.stream,
             s.n, (const float *)s.feat, params, s.out);
  else
    launch_k(c, k_mlp_forward, (int)cdiv(s.n, kRows), kRows, 0, c.stream, s.n, (const float *)s.feat, params, s.out);
  const int g = (int)cdiv(s.n, 256);
  launch_k(c, k_correct, g, 256, 0, c.stream, s.n, (const int32_t *)s.zr, (const int32_t *)s.zs,
           (const double *)s.zv, (const float *)s.out, 0, s.zc);
  launch_k(c, k_correct, g, 256, 0, c.stream, s.n, (const int32_t *)s.wr, (const int32_t *)s.ws,
           (const double *)s.wv, (const float *)s.out, 4, s.wc);
  CUDA_TRY(cudaGetLastError());
  return F3R_SUCCESS;
}

// one evaluation of the loss into *loss_d and (want_grad) of the gradient into L->g
Status loss_and_grad(f3r_learned *L, double *loss_d, bool want_grad) {
  Context &c = *L->ctx;
  SysDev &s = L->train;
  F3R_TRY(forward(c, L->p, s, 0));
  const int32_t n = s.n, P = s.npairs;
  const dim3 grid((unsigned)cdiv(n, 256), (unsigned)P);
  launch_k(c, k_csr_mv, grid, 256, 0, c.stream, n, (const int32_t *)s.wr, (const int32_t *)s.wi,
           (const double *)s.wc, (const double *)s.r, s.u);
  launch_k(c, k_csr_mv, grid, 256, 0, c.stream, n, (const int32_t *)s.zr, (const int32_t *)s.zi,
           (const double *)s.zc, (const double *)s.u, s.y);
  const dim3 lgrid((unsigned)std::min<int64_t>(cdiv(n, 256), 2 * c.sm_count), (unsigned)P);
  launch_k(c, k_loss_d, lgrid, 256, 0, c.stream, n, (const double *)s.y, (const double *)s.e,
           (const double *)L->inv_ee, 1.0 / P, s.d, loss_d);
  if (want_grad) {
    launch_k(c, k_csr_mv_t, grid, 256, 0, c.stream, n, (const int32_t *)s.tr, (const int32_t *)s.ti,
             (const int32_t *)s.tk, (const double *)s.zc, (const double *)s.d, s.g);
    launch_k(c, k_entry_grad, (int)cdiv(n, 256), 256, 0, c.stream, n, P, (const int32_t *)s.zr,
             (const int32_t *)s.zi, (const int32_t *)s.zs, (const double *)s.zv, (const int32_t *)s.wr,
             (const int32_t *)s.wi, (const int32_t *)s.ws, (const double *)s.wv, (const double *)s.d,
             (const double *)s.u, (const double *)s.g, (const double *)s.r, s.dout);
    launch_k(c, k_mlp_backward, (int)std::min<int64_t>(cdiv(n, kRows), L->grid_back), kRows, kBackSmem, c.stream, n,
             (const float *)s.feat, (const float *)L->p, (const float *)s.dout, L->g);
  }
  CUDA_TRY(cudaGetLastError());
  return F3R_SUCCESS;
}

}  // namespace

extern "C" {

f3r_status f3r_learned_create(f3r_context *ctx, int32_t hidden, uint64_t seed, f3r_learned **out) {
  clear_stale_error();
  if (!ctx || !out) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  if (hidden != kH) return fail(F3R_ERROR_UNSUPPORTED, "the network's hidden width is 64");
  CUDA_TRY(cudaSetDevice(ctx->device));
  auto L = std::make_unique<f3r_learned>();
  L->ctx = ctx;
  Context &c = *ctx;
  // He-normal hidden layers, zero output layer: the untrained network changes nothing
  std::vector<float> p(kParams, 0.f);
  std::mt19937_64 eng(seed);
  std::normal_distribution<float> n1(0.f, std::sqrt(2.f / kIn)), n2(0.f, std::sqrt(2.f / kH));
  for (int k = 0; k < kH * kIn; k++) p[oW1 + k] = n1(eng);
  for (int k = 0; k < kH * kH; k++) p[oW2 + k] = n2(eng);
  for (float **b : {&L->p, &L->g, &L->m, &L->v}) F3R_TRY(c.alloc((void **)b, sizeof(float) * kParams));
  CUDA_TRY(cudaMemcpy(L->p, p.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice));
  for (float *b : {L->g, L->m, L->v}) CUDA_TRY(cudaMemset(b, 0, sizeof(float) * kParams));
  CUDA_TRY(cudaFuncSetAttribute(k_mlp_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBackSmem));
  CUDA_TRY(cudaFuncSetAttribute(k_mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
  int per_sm = 0;
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mlp_backward, kRows, kBackSmem));
  L->grid_back = std::max(1, per_sm) * c.sm_count;
  *out = L.release();
  return F3R_SUCCESS;
}

void f3r_learned_destroy(f3r_learned *L) {
  if (!L) return;
  if (cudaSetDevice(L->ctx->device) != cudaSuccess) return;  // runtime shutting down: left to the exit
  cudaStreamSynchronize(L->ctx->stream);
  L->train.release();
  for (void *b : {(void *)L->p, (void *)L->g, (void *)L->m, (void *)L->v, (void *)L->loss, (void *)L->inv_ee})
    cudaFree(b);
  delete L;
}

f3r_status f3r_learned_params(f3r_learned *L, float *params, int32_t set, int64_t *count) {
  if (!L) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  if (count) *count = kParams;
  if (!params) return F3R_SUCCESS;
  CUDA_TRY(cudaSetDevice(L->ctx->device));
  CUDA_TRY(cudaStreamSynchronize(L->ctx->stream));
  if (set) {
    for (int k = 0; k < kParams; k++)
      if (!std::isfinite(params[k])) return fail(F3R_ERROR_INVALID_VALUE, "non-finite parameter");
    CUDA_TRY(cudaMemcpy(L->p, params, sizeof(float) * kParams, cudaMemcpyHostToDevice));
  } else {
    CUDA_TRY(cudaMemcpy(params, L->p, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
  }
  return F3R_SUCCESS;
}

f3r_status f3r_learned_set_data(f3r_learned *L, const f3r_csr *a, int32_t nx, int32_t ny, const f3r_csr *z,
                                const f3r_csr *wt, int32_t npairs, const double *r, const double *e) {
  clear_stale_error();
  if (!L || !a || !z || !wt || npairs < 1 || npairs > 1024 || !r || !e)
    return fail(F3R_ERROR_INVALID_VALUE, "bad argument (npairs in 1..1024)");
  CUDA_TRY(cudaSetDevice(L->ctx->device));
  Context &c = *L->ctx;
  SysDev &s = L->train;
  F3R_TRY(load_system(c, s, a, nx, ny, z, wt));
  const int32_t n = s.n;
  if (n == 0) return fail(F3R_ERROR_INVALID_VALUE, "empty training system");
  std::vector<double> inv(npairs);
  for (int32_t p = 0; p < npairs; p++) {
    double ee = 0;
    for (int32_t i = 0; i < n; i++) ee += e[(size_t)p * n + i] * e[(size_t)p * n + i];
    if (!(ee > 0) || !std::isfinite(ee)) {
      s.release();
      return fail(F3R_ERROR_INVALID_VALUE, "an error vector is zero or not finite");
    }
    inv[p] = 1.0 / ee;
  }
  s.npairs = npairs;
  const size_t nv = (size_t)n * npairs;
  F3R_TRY(s.put(c, &s.r, r, nv));
  F3R_TRY(s.put(c, &s.e, e, nv));
  for (double **b : {&s.u, &s.y, &s.d, &s.g}) F3R_TRY(s.get(c, b, nv));
  cudaFree(L->inv_ee);
  L->inv_ee = nullptr;
  F3R_TRY(c.alloc((void **)&L->inv_ee, sizeof(double) * npairs));
  CUDA_TRY(cudaMemcpyAsync(L->inv_ee, inv.data(), sizeof(double) * npairs, cudaMemcpyHostToDevice, c.stream));
  CUDA_TRY(cudaStreamSynchronize(c.stream));
  return F3R_SUCCESS;
}

f3r_status f3r_learned_evaluate(f3r_learned *L, double *loss, float *grad) {
  clear_stale_error();
  if (!L || !loss) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  if (L->train.npairs == 0) return fail(F3R_ERROR_INVALID_VALUE, "no training data set");
  CUDA_TRY(cudaSetDevice(L->ctx->device));
  Context &c = *L->ctx;
  if (L->loss_cap < 1) {
    F3R_TRY(c.alloc((void **)&L->loss, sizeof(double)));
    L->loss_cap = 1;
  }
  CUDA_TRY(cudaMemsetAsync(L->loss, 0, sizeof(double), c.stream));
  CUDA_TRY(cudaMemsetAsync(L->g, 0, sizeof(float) * kParams, c.stream));
  F3R_TRY(loss_and_grad(L, L->loss, grad != nullptr));
  CUDA_TRY(cudaMemcpyAsync(c.pinned, L->loss, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  if (grad) CUDA_TRY(cudaMemcpyAsync(grad, L->g, sizeof(float) * kParams, cudaMemcpyDeviceToHost, c.stream));
  CUDA_TRY(cudaMemsetAsync(L->g, 0, sizeof(float) * kParams, c.stream));
  CUDA_TRY(cudaStreamSynchronize(c.stream));
  *loss = c.pinned[0];
  return F3R_SUCCESS;
}

f3r_status f3r_learned_train(f3r_learned *L, int32_t steps, double lr, double *losses) {
  clear_stale_error();
  if (!L || steps < 0 || !(lr > 0)) return fail(F3R_ERROR_INVALID_VALUE, "bad argument");
  if (L->train.npairs == 0) return fail(F3R_ERROR_INVALID_VALUE, "no training data set");
  if (steps == 0) return F3R_SUCCESS;
  CUDA_TRY(cudaSetDevice(L->ctx->device));
  Context &c = *L->ctx;
  if (L->loss_cap < steps) {
    cudaFree(L->loss);
    L->loss = nullptr;
    L->loss_cap = 0;
    F3R_TRY(c.alloc((void **)&L->loss, sizeof(double) * steps));
    L->loss_cap = steps;
  }
  CUDA_TRY(cudaMemsetAsync(L->loss, 0, sizeof(double) * steps, c.stream));
  CUDA_TRY(cudaMemsetAsync(L->g, 0, sizeof(float) * kParams, c.stream));
  const float b1 = 0.9f, b2 = 0.999f;
  for (int32_t k = 0; k < steps; k++) {
    F3R_TRY(loss_and_grad(L, L->loss + k, true));
    L->steps++;
    const float c1 = 1.f - std::pow(b1, (float)L->steps), c2 = 1.f - std::pow(b2, (float)L->steps);
    launch_k(c, k_adam, (int)cdiv(kParams, 256), 256, 0, c.stream, (int32_t)kParams, L->p, L->g, L->m, L->v,
             (float)lr, b1, b2, c1, c2, 1e-8f);
  }
  CUDA_TRY(cudaGetLastError());
  if (losses) CUDA_TRY(cudaMemcpyAsync(losses, L->loss, sizeof(double) * steps, cudaMemcpyDeviceToHost, c.stream));
  CUDA_TRY(cudaStreamSynchronize(c.stream));
  return F3R_SUCCESS;
}

f3r_status f3r_learned_correct(f3r_learned *L, const f3r_csr *a, int32_t nx, int32_t ny, const f3r_csr *z,
                               const f3r_csr *wt, int32_t bf16, double *z_val, double *wt_val, float *delta) {
  clear_stale_error();
  if (!L || !a || !z || !wt || !z_val || !wt_val) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  CUDA_TRY(cudaSetDevice(L->ctx->device));
  Context &c = *L->ctx;
  SysDev s;
  Status st = load_system(c, s, a, nx, ny, z, wt);
  if (st == F3R_SUCCESS && (bf16 < 0 || bf16 > 2)) st = fail(F3R_ERROR_INVALID_VALUE, "bf16 must be 0, 1 or 2");
  if (st == F3R_SUCCESS) st = forward(c, L->p, s, bf16);
  if (st == F3R_SUCCESS && bf16 == 1) st = c.check_device_error();
  cudaError_t ce = cudaSuccess;
  if (st == F3R_SUCCESS && s.n > 0) {
    ce = cudaMemcpyAsync(z_val, s.zc, sizeof(double) * s.znnz, cudaMemcpyDeviceToHost, c.stream);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(wt_val, s.wc, sizeof(double) * s.wnnz, cudaMemcpyDeviceToHost, c.stream);
    if (ce == cudaSuccess && delta)
      ce = cudaMemcpyAsync(delta, s.out, sizeof(float) * (size_t)s.n * kOut, cudaMemcpyDeviceToHost, c.stream);
  }
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(c.stream);
  if (st == F3R_SUCCESS && ce != cudaSuccess) st = fail(F3R_ERROR_CUDA, cudaGetErrorString(ce));
  cudaStreamSynchronize(c.stream);
  s.release();
  return st;
}

f3r_status f3r_learned_time_inference(f3r_learned *L, const f3r_csr *a, int32_t nx, int32_t ny, const f3r_csr *z,
                                      const f3r_csr *wt, int32_t mode, int32_t reps, double *us) {
  clear_stale_error();
  if (!L || !a || !z || !wt || !us) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  if (mode < 0 || mode > 2 || reps < 1) return fail(F3R_ERROR_INVALID_VALUE, "mode must be 0, 1 or 2 and reps >= 1");
  CUDA_TRY(cudaSetDevice(L->ctx->device));
  Context &c = *L->ctx;
  SysDev s;
  Status st = load_system(c, s, a, nx, ny, z, wt);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (st == F3R_SUCCESS && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
    st = fail(F3R_ERROR_CUDA, "cudaEventCreate");
  // the network alone: one warm-up launch, then reps launches between events
  auto net = [&]() -> Status {
    if (s.n == 0) return F3R_SUCCESS;
    if (mode == 1) {
      const int64_t tiles = cdiv(s.n, kTcRows);
      launch_k(c, k_mlp_infer_tc, (int)std::min<int64_t>(cdiv(tiles, kTcGroups), (int64_t)c.sm_count * kTcCtasPerSm),
               kTcRows * kTcGroups, kTcSmem, c.stream, s.n, (const float *)s.feat, (const float *)L->p, s.out, c.err);
    } else if (mode == 2)
      launch_k(c, k_mlp_infer_bf16, (int)std::min<int64_t>(cdiv(s.n, 64), (int64_t)c.sm_count * 8), 128, 0,
               c.stream, s.n, (const float *)s.feat, (const float *)L->p, s.out);
    else
      launch_k(c, k_mlp_forward, (int)cdiv(s.n, kRows), kRows, 0, c.stream, s.n, (const float *)s.feat,
               (const float *)L->p, s.out);
    CUDA_TRY(cudaGetLastError());
    return F3R_SUCCESS;
  };
  if (st == F3R_SUCCESS) st = net();
  if (st == F3R_SUCCESS && cudaEventRecord(e0, c.stream) != cudaSuccess) st = fail(F3R_ERROR_CUDA, "cudaEventRecord");
  for (int32_t k = 0; st == F3R_SUCCESS && k < reps; k++) st = net();
  if (st == F3R_SUCCESS && cudaEventRecord(e1, c.stream) != cudaSuccess) st = fail(F3R_ERROR_CUDA, "cudaEventRecord");
  if (st == F3R_SUCCESS && cudaEventSynchronize(e1) != cudaSuccess) st = fail(F3R_ERROR_CUDA, "cudaEventSynchronize");
  float ms = 0.f;
  if (st == F3R_SUCCESS) {
    cudaEventElapsedTime(&ms, e0, e1);
    *us = 1e3 * ms / reps;
  }
  if (st == F3R_SUCCESS && mode == 1) st = c.check_device_error();
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaStreamSynchronize(c.stream);
  s.release();
  return st;
}

}  // extern "C"
