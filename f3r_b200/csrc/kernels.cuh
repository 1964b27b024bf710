// kernels.cuh -- the F3R level kernels: fused Gram-Schmidt reductions, the
// device-resident Givens/Hessenberg update, precision casts, and the fp16
// Richardson operator with its adaptive weights.
#pragma once

#include "sell.cuh"

namespace f3r {

constexpr int kMaxCols = 128;  // FGMRES basis columns per level (m + 1 <= 128)
constexpr int kMaxDots = 16;   // dot products fused into an inner-level SpMV
constexpr int kMaxM4 = 16;

template <typename T> struct Cols {
  const T *p[kMaxCols];
};

// 16-byte (or narrower) vector access; every vector this library allocates
// starts on a 64-byte boundary with columns padded to 8 elements.
template <typename T, int N> struct alignas(sizeof(T) * N) VecN {
  T v[N];
};
template <typename T, int N> __device__ __forceinline__ VecN<T, N> ldv(const T *p) {
  return *reinterpret_cast<const VecN<T, N> *>(p);
}
template <typename T, int N> __device__ __forceinline__ void stv(T *p, const VecN<T, N> &v) {
  *reinterpret_cast<VecN<T, N> *>(p) = v;
}

// Running state of the adaptive-weight Richardson operator
// (f3r-gpu.cpp:106-108, 224-227, 239-240, 253-254, 277-281).
struct RichState {
  float sum[kMaxM4];   // sum[k]: 1 + all weights computed so far (fp32, as the reference)
  __half ome[kMaxM4];  // ome[k]: sum[k] / den rounded to fp16 (the reference's scalar<__half>)
  float om[kMaxM4];    // weight computed by the current update call
  int den;             // cnt / period at the last update
};

// Per-level FGMRES scalars kept on the device (gmres.hpp:61-63).
template <typename T> struct GivensCtl {
  T *H;           // (m+1) x m, column-major, ld = ldh
  T *cs, *sn, *e, *y;
  T *inv;         // 1 / h_{j+1,j}
  double *abs_e;  // |e(j+1)| for the host's cond() call (outer level), or nullptr
  int ldh, j, compute_y;
  int *err;
};

// Scalar arithmetic of the Hessenberg / Givens / back-substitution updates
// with every operation rounded on its own (no FMA contraction), so that the
// result is the same in every kernel these are inlined into, as in the
// reference's unfused scalar code (gmres.hpp:14-53).
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// Blas1::trsv (gmres.hpp:41-53): y(0..w-1) from the triangular H and e
template <typename T> __device__ __forceinline__ void back_subst(const T *H, const T *e, T *y, int ldh, int w) {
  for (int i = w - 1; i >= 0; i--) {
    T s = e[i];
    for (int q = w - 1; q > i; q--) s = sub_rn(s, mul_rn(H[(size_t)q * ldh + i], y[q]));
    y[i] = s / H[(size_t)i * ldh + i];
  }
}

// full_grot + final_grot (gmres.hpp:14-38) and, after the level's last step,
// the back substitution Blas1::trsv (gmres.hpp:41-53).  One thread.
template <typename T> __device__ void givens_step(const GivensCtl<T> &g, T nrm2) {
  const int j = g.j;
  T *Hc = g.H + (size_t)j * g.ldh;
  const T h = sqrt(nrm2);
  Hc[j + 1] = h;
  *g.inv = T(1) / h;
  if (!(h > T(0)) || !isfinite(h)) atomicExch(g.err, (int)DEV_BREAKDOWN);
  for (int i = 0; i < j; i++) {
    const T t = Hc[i];
    Hc[i] = add_rn(mul_rn(g.cs[i], t), mul_rn(g.sn[i], Hc[i + 1]));
    Hc[i + 1] = add_rn(mul_rn(-g.sn[i], t), mul_rn(g.cs[i], Hc[i + 1]));
  }
  const T t = sqrt(add_rn(mul_rn(Hc[j], Hc[j]), mul_rn(Hc[j + 1], Hc[j + 1])));
  g.cs[j] = Hc[j] / t;
  g.sn[j] = Hc[j + 1] / t;
  Hc[j] = t;
  Hc[j + 1] = 0;
  g.e[j + 1] = mul_rn(-g.sn[j], g.e[j]);
  g.e[j] = mul_rn(g.cs[j], g.e[j]);
  if (g.abs_e) *g.abs_e = (double)fabs(g.e[j + 1]);
  if (g.compute_y) back_subst(g.H, g.e, g.y, g.ldh, j + 1);
}

// ---------------------------------------------------------------------------
// SpMV epilogues of the FGMRES levels
// ---------------------------------------------------------------------------

// Inner levels (fp32 vectors): w = A z stored, and H(j, k) = <w, V(k)>,
// k = 0..nv-1, fused (CGS dots all use the unmodified w, gmres.hpp:112-114).
template <int NVT, bool PREFETCH = (NVT <= 4)> struct EpiStoreDots {
  using Red = float;
  static constexpr int NV = NVT;
  // up to 4 basis values are fetched ahead of the multiply-add chain; wider
  // epilogues read them afterwards (their registers would spill)
  static constexpr bool PRE = PREFETCH;
  struct Pre {
    float v[PRE ? NVT : 1];
  };
  float *y;
  Cols<float> V;
  int nv;
  GridRed gr;
  float *hcol;
  __device__ __forceinline__ Pre load(int64_t r) const {
    Pre p;
    if (PRE) {
#pragma unroll
      for (int k = 0; k < (PRE ? NVT : 1); k++) p.v[k] = (k < nv) ? __ldg(V.p[k] + r) : 0.0f;
    }
    return p;
  }
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, Acc acc, const Pre &p, Red (&d)[NV]) const {
    const float yv = (float)acc;
    y[r] = yv;
#pragma unroll
    for (int k = 0; k < NV; k++)
      if (k < nv) d[k] = __fmaf_rn(yv, PRE ? p.v[PRE ? k : 0] : __ldg(V.p[k] + r), d[k]);
  }
  template <int W> __device__ __forceinline__ void finish(Red (&d)[NV]) const {
    float *h = hcol;
    const int m = nv;
    grid_reduce<float, NV, W>(d, nv, gr, [h, m](float *tot) {
      for (int k = 0; k < m; k++) h[k] = tot[k];
    });
  }
};

// Outer level: r = b - A x in fp64 with ||r||^2 fused; the finisher sets
// e(0) = ||r||, 1/||r|| and |e(0)| for the host (gmres.hpp:87, 100-103).
struct EpiResidualNorm {
  using Red = double;
  static constexpr int NV = 1;
  struct Pre {
    double b;
  };
  const double *b;
  double *y;
  GridRed gr;
  double *e, *inv, *abs_e;
  __device__ __forceinline__ Pre load(int64_t r) const { return {b[r]}; }
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, Acc acc, const Pre &p, Red (&d)[1]) const {
    const double v = p.b - (double)acc;
    y[r] = v;
    d[0] = __fma_rn(v, v, d[0]);
  }
  template <int W> __device__ __forceinline__ void finish(Red (&d)[1]) const {
    double *e_ = e, *inv_ = inv, *ae = abs_e;
    grid_reduce<double, 1, W>(d, 1, gr, [e_, inv_, ae](double *tot) {
      const double h = sqrt(tot[0]);
      e_[0] = h;
      *inv_ = 1.0 / h;
      *ae = fabs(h);
    });
  }
};

// ---------------------------------------------------------------------------
// Gram-Schmidt update, norm, Givens (gmres.hpp:115-119)
// ---------------------------------------------------------------------------
// w -= sum_k H(j,k) V(k)   (MULMV order: V(i,0) h0, then fma over k)
// then ||w||^2 -> h_{j+1,j}, 1/h, Givens rotation, optional back substitution.
template <typename T, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_cgs_update(T *__restrict__ w, Cols<T> V, int nv, int64_t n,
                                                           GridRed gr, GivensCtl<T> g) {
  constexpr int N = 16 / sizeof(T);
  __shared__ T sh[kMaxCols];
  const T *hcol = g.H + (size_t)g.j * g.ldh;
  for (int k = threadIdx.x; k < nv; k += blockDim.x) sh[k] = hcol[k];
  __syncthreads();
  T part[1] = {0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nq = n / N;
  for (int64_t q = tid; q < nq; q += stride) {
    const int64_t i = q * N;
    const VecN<T, N> a = ldv<T, N>(V.p[0] + i);
    T r[N];
#pragma unroll
    for (int e = 0; e < N; e++) r[e] = a.v[e] * sh[0];
#pragma unroll 4
    for (int k = 1; k < nv; k++) {
      const VecN<T, N> b = ldv<T, N>(V.p[k] + i);
      const T hk = sh[k];
#pragma unroll
      for (int e = 0; e < N; e++) r[e] = fmaT(b.v[e], hk, r[e]);
    }
    VecN<T, N> wv = ldv<T, N>(w + i);
#pragma unroll
    for (int e = 0; e < N; e++) {
      wv.v[e] -= r[e];
      part[0] = fmaT(wv.v[e], wv.v[e], part[0]);
    }
    stv<T, N>(w + i, wv);
  }
  for (int64_t i = nq * N + tid; i < n; i += stride) {
    T r = V.p[0][i] * sh[0];
    for (int k = 1; k < nv; k++) r = fmaT(V.p[k][i], sh[k], r);
    const T wi = w[i] - r;
    w[i] = wi;
    part[0] = fmaT(wi, wi, part[0]);
  }
  const GivensCtl<T> gg = g;
  grid_reduce<T, 1, WARPS>(part, 1, gr, [gg](T *tot) { givens_step<T>(gg, tot[0]); });
}

// H(j, k) = <w, V(k)> for k < nv (any nv up to kMaxCols): vectors taken in
// chunks of 8 with w re-read from L1/L2 per chunk; used by the outer fp64
// level and by inner fp32 levels with more than 8 basis vectors.
template <typename T, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_multidot_chunked(const T *__restrict__ w, Cols<T> V, int nv,
                                                                 int64_t n, GridRed gr, T *hcol) {
  constexpr int CH = 8;
  // partials laid out [block][nv]
  T *part = static_cast<T *>(gr.partials);
  __shared__ T sred[WARPS][CH];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k0 = 0; k0 < nv; k0 += CH) {
    T a[CH];
#pragma unroll
    for (int c = 0; c < CH; c++) a[c] = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      const T wi = w[i];
#pragma unroll
      for (int c = 0; c < CH; c++)
        if (k0 + c < nv) a[c] = fmaT(wi, V.p[k0 + c][i], a[c]);
    }
#pragma unroll
    for (int c = 0; c < CH; c++) {
      const T s = warp_sum(a[c]);
      if (lane == 0) sred[warp][c] = s;
    }
    __syncthreads();
    if (threadIdx.x < CH && k0 + threadIdx.x < nv) {
      T s = 0;
      for (int q = 0; q < WARPS; q++) s += sred[q][threadIdx.x];
      part[(size_t)blockIdx.x * nv + k0 + threadIdx.x] = s;
    }
    __syncthreads();
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(gr.ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int k = warp; k < nv; k += WARPS) {
    T s = 0;
    for (int b = lane; b < (int)gridDim.x; b += 32) s += __ldcg(&part[(size_t)b * nv + k]);
    s = warp_sum(s);
    if (lane == 0) hcol[k] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) *gr.ticket = 0;
}

// H(j, k) = <w, V(k)> for k < nv in fp32 (inner levels), one pass over w and
// the nv basis columns with 16-byte loads; the fp32 accumulators of a thread
// are reduced per block and then in block order by the last block.  This is
// the CGS dot phase (gmres.hpp:112-114, all dots with the unmodified w).
template <int MAXV, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_multidot_f32(const float *__restrict__ w, Cols<float> V, int nv,
                                                             int64_t n, GridRed gr, float *hcol) {
  float a[MAXV];
#pragma unroll
  for (int k = 0; k < MAXV; k++) a[k] = 0.0f;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nq = n / 4;
  for (int64_t q = tid; q < nq; q += stride) {
    const VecN<float, 4> wv = ldv<float, 4>(w + 4 * q);
#pragma unroll
    for (int k = 0; k < MAXV; k++) {
      if (k < nv) {
        const VecN<float, 4> v = ldv<float, 4>(V.p[k] + 4 * q);
#pragma unroll
        for (int e = 0; e < 4; e++) a[k] = __fmaf_rn(wv.v[e], v.v[e], a[k]);
      }
    }
  }
  for (int64_t i = nq * 4 + tid; i < n; i += stride) {
    const float wi = w[i];
#pragma unroll
    for (int k = 0; k < MAXV; k++)
      if (k < nv) a[k] = __fmaf_rn(wi, V.p[k][i], a[k]);
  }
  float *h = hcol;
  const int m = nv;
  grid_reduce<float, MAXV, WARPS>(a, nv, gr, [h, m](float *tot) {
    for (int k = 0; k < m; k++) h[k] = tot[k];
  });
}

// v *= *inv  (V(j+1) *= h.inv(), gmres.hpp:117)
template <typename T> __global__ void k_scale(T *__restrict__ v, const T *__restrict__ inv, int64_t n) {
  constexpr int N = 16 / sizeof(T);
  const T s = *inv;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nq = n / N;
  for (int64_t q = tid; q < nq; q += stride) {
    VecN<T, N> a = ldv<T, N>(v + q * N);
#pragma unroll
    for (int e = 0; e < N; e++) a.v[e] *= s;
    stv<T, N>(v + q * N, a);
  }
  for (int64_t i = nq * N + tid; i < n; i += stride) v[i] *= s;
}

// Level-2 entry.  The outer basis vector V1(j) is normalised here, in place
// (V(j+1) *= h.inv(), gmres.hpp:117; the factor 1/h was left by the outer
// level's reduction), then cast: V2(0) = float(V1(j)) (V(0).copy(rhs),
// gmres.hpp:102), with e(0) = 1 (normalize=false, gmres.hpp:100-101).  `in`
// is read through a device pointer slot so one captured graph serves every
// outer step.
__global__ void k_level2_enter(double *const *__restrict__ in_slot, const double *__restrict__ inv,
                               float *__restrict__ v0, float *e, int64_t n) {
  double *in = *in_slot;
  const double s = *inv;
  if (blockIdx.x == 0 && threadIdx.x == 0) e[0] = 1.0f;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nq = n / 4;
  for (int64_t q = tid; q < nq; q += stride) {
    VecN<double, 2> a = ldv<double, 2>(in + 4 * q), b = ldv<double, 2>(in + 4 * q + 2);
    a.v[0] *= s;
    a.v[1] *= s;
    b.v[0] *= s;
    b.v[1] *= s;
    stv<double, 2>(in + 4 * q, a);
    stv<double, 2>(in + 4 * q + 2, b);
    VecN<float, 4> o;
    o.v[0] = (float)a.v[0];
    o.v[1] = (float)a.v[1];
    o.v[2] = (float)b.v[0];
    o.v[3] = (float)b.v[1];
    stv<float, 4>(v0 + 4 * q, o);
  }
  for (int64_t i = nq * 4 + tid; i < n; i += stride) {
    const double v = in[i] * s;
    in[i] = v;
    v0[i] = (float)v;
  }
}

// x = Z y (with_init) for the inner levels, x += Z y for the outer level
// (gmres.hpp:127-131); the sum is formed in the level's type T and converted
// to the caller's type Out, as MULMV followed by T(...) in the reference.
template <typename T, typename Out, bool ACCUM>
__global__ void k_zy(Cols<T> Z, const T *__restrict__ y, int nz, Out *__restrict__ out_direct,
                     Out *const *__restrict__ out_slot, int64_t n) {
  constexpr int N = 16 / sizeof(T);
  __shared__ T sy[kMaxCols];
  for (int k = threadIdx.x; k < nz; k += blockDim.x) sy[k] = y[k];
  __syncthreads();
  Out *out = out_slot ? *out_slot : out_direct;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nq = n / N;
  for (int64_t q = tid; q < nq; q += stride) {
    const int64_t i = q * N;
    const VecN<T, N> a = ldv<T, N>(Z.p[0] + i);
    T r[N];
#pragma unroll
    for (int e = 0; e < N; e++) r[e] = a.v[e] * sy[0];
#pragma unroll 4
    for (int k = 1; k < nz; k++) {
      const VecN<T, N> b = ldv<T, N>(Z.p[k] + i);
      const T yk = sy[k];
#pragma unroll
      for (int e = 0; e < N; e++) r[e] = fmaT(b.v[e], yk, r[e]);
    }
    VecN<Out, N> o;
    if (ACCUM) o = ldv<Out, N>(out + i);
#pragma unroll
    for (int e = 0; e < N; e++) o.v[e] = ACCUM ? o.v[e] + (Out)r[e] : (Out)r[e];
    stv<Out, N>(out + i, o);
  }
  for (int64_t i = nq * N + tid; i < n; i += stride) {
    T r = Z.p[0][i] * sy[0];
    for (int k = 1; k < nz; k++) r = fmaT(Z.p[k][i], sy[k], r);
    if (ACCUM) out[i] += (Out)r;
    else out[i] = (Out)r;
  }
}

// ---------------------------------------------------------------------------
// Level 4: the fp16 Richardson operator R (f3r-gpu.cpp:229-260).  fp16
// storage, fp32 arithmetic, one rounding to fp16 per stored value.
// Diagonal SDAINV (W^T, Z both diagonal -- what tol = 0.1 leaves of a scaled
// stencil) is fused into the vector kernels; general W^T / Z run as SELL
// SpMVs with fused epilogues.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float h2f(__half h) { return __half2float(h); }
__device__ __forceinline__ __half f2h(float f) { return __float2half_rn(f); }

// Diagonal of W^T and of Z in fp16.  Both pointers are null where every fp16
// value of both diagonals is exactly 1 (a diagonally scaled matrix whose
// SDAINV keeps only the diagonal): the kernels then multiply by the constant
// 1 instead of a loaded 1 -- the same arithmetic, without 4 bytes a row.
struct DiagPre {
  const __half *w, *z;
  static __device__ __forceinline__ __half one() { return __ushort_as_half((unsigned short)0x3C00); }
  __device__ __forceinline__ __half wv(int64_t i) const { return w ? w[i] : one(); }
  __device__ __forceinline__ __half zv(int64_t i) const { return z ? z[i] : one(); }
  __device__ __forceinline__ VecN<__half, 4> w4(int64_t i) const { return w ? ldv<__half, 4>(w + i) : ones4(); }
  __device__ __forceinline__ VecN<__half, 4> z4(int64_t i) const { return z ? ldv<__half, 4>(z + i) : ones4(); }
  static __device__ __forceinline__ VecN<__half, 4> ones4() {
    VecN<__half, 4> a;
#pragma unroll
    for (int e = 0; e < 4; e++) a.v[e] = one();
    return a;
  }
  __device__ __forceinline__ float apply(int64_t i, float x) const {
    const float t = h2f(f2h(h2f(wv(i)) * x));  // tmp = W^T x
    return h2f(f2h(h2f(zv(i)) * t));           // hout = Z tmp
  }
};

// First half of R.  The caller's basis vector is normalised here, in place,
// when its 1/h factor is given (V(j+1) *= h.inv(), gmres.hpp:117 -- deferred
// from the Gram-Schmidt step to save a pass); then hin = fp16(in * sc),
// hout = M hin, and on a call without a weight update hout *= ome[0]
// (f3r-gpu.cpp:231-243).  In is float (R below an fp32 level) or __half (R
// below the fp16-vector level: the input already is R's fp16 working vector,
// so hin is `in` itself and is not written; sc is 1 there).
template <typename In> struct In4;
template <> struct In4<float> {
  static __device__ __forceinline__ void ld(const float *p, float (&v)[4]) {
    const VecN<float, 4> a = ldv<float, 4>(p);
#pragma unroll
    for (int e = 0; e < 4; e++) v[e] = a.v[e];
  }
  static __device__ __forceinline__ void st(float *p, const float (&v)[4]) {
    VecN<float, 4> a;
#pragma unroll
    for (int e = 0; e < 4; e++) a.v[e] = v[e];
    stv<float, 4>(p, a);
  }
};
template <> struct In4<__half> {
  static __device__ __forceinline__ void ld(const __half *p, float (&v)[4]) {
    const VecN<__half, 4> a = ldv<__half, 4>(p);
#pragma unroll
    for (int e = 0; e < 4; e++) v[e] = __half2float(a.v[e]);
  }
  static __device__ __forceinline__ void st(__half *p, const float (&v)[4]) {
    VecN<__half, 4> a;
#pragma unroll
    for (int e = 0; e < 4; e++) a.v[e] = __float2half_rn(v[e]);
    stv<__half, 4>(p, a);
  }
};
__device__ __forceinline__ float as_float(float v) { return v; }
__device__ __forceinline__ float as_float(__half v) { return __half2float(v); }
template <typename T> __device__ __forceinline__ T from_float(float v);
template <> __device__ __forceinline__ float from_float<float>(float v) { return v; }
template <> __device__ __forceinline__ __half from_float<__half>(float v) { return __float2half_rn(v); }

template <bool SCALE_BY_OME, typename In = float>
__global__ void k_rich_enter_diag(In *__restrict__ in, const float *__restrict__ in_inv, float sc, DiagPre M,
                                  __half *__restrict__ hin, __half *__restrict__ hout,
                                  const RichState *__restrict__ rs, float *e_set, int64_t n) {
  constexpr bool HALF_IN = std::is_same<In, __half>::value;
  if (e_set && blockIdx.x == 0 && threadIdx.x == 0) e_set[0] = 1.0f;
  const float om = SCALE_BY_OME ? h2f(rs->ome[0]) : 1.0f;
  const float s = in_inv ? *in_inv : 1.0f;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nq = n / 4;
  for (int64_t q = tid; q < nq; q += stride) {
    const int64_t i = 4 * q;
    float v[4];
    In4<In>::ld(in + i, v);
    if (in_inv) {
#pragma unroll
      for (int e = 0; e < 4; e++) v[e] *= s;
      In4<In>::st(in + i, v);
    }
    const VecN<__half, 4> w = M.w4(i), z = M.z4(i);
    VecN<__half, 4> hi, ho;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      hi.v[e] = f2h(v[e] * sc);
      const float t = h2f(f2h(h2f(w.v[e]) * h2f(hi.v[e])));
      float o = h2f(f2h(h2f(z.v[e]) * t));
      if (SCALE_BY_OME) o = h2f(f2h(o * om));
      ho.v[e] = f2h(o);
    }
    if (!HALF_IN) stv<__half, 4>(hin + i, hi);
    stv<__half, 4>(hout + i, ho);
  }
  for (int64_t i = nq * 4 + tid; i < n; i += stride) {
    float v = as_float(in[i]);
    if (in_inv) {
      v *= s;
      in[i] = from_float<In>(v);
    }
    const __half hi = f2h(v * sc);
    if (!HALF_IN) hin[i] = hi;
    float ho = M.apply(i, h2f(hi));
    if (SCALE_BY_OME) ho = h2f(f2h(ho * om));
    hout[i] = f2h(ho);
  }
}

// General preconditioner: (normalise in place), hin = fp16(in * sc) only
// (nothing but the normalisation when the input is R's fp16 vector itself).
template <typename In = float>
__global__ void k_rich_cast_in(In *__restrict__ in, const float *__restrict__ in_inv, float sc,
                               __half *__restrict__ hin, float *e_set, int64_t n) {
  constexpr bool HALF_IN = std::is_same<In, __half>::value;
  if (e_set && blockIdx.x == 0 && threadIdx.x == 0) e_set[0] = 1.0f;
  const float s = in_inv ? *in_inv : 1.0f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float v = as_float(in[i]);
    if (in_inv) {
      v *= s;
      in[i] = from_float<In>(v);
    }
    if (!HALF_IN) hin[i] = f2h(v * sc);
  }
}

// Residual step of R with the diagonal preconditioner fused (no weight
// update): hr = fp16(hin - A16 hout); t2 = M hr; hnew = fp16(hout + ome[k] t2);
// the last step writes out = fp32(hnew) / sc (out.copy(hout)).  ome[k] is read
// once per thread (setup).  UNIT: both diagonal factors are 1 in fp16, so
// t2 = 1 * (1 * hr) = hr exactly (an fp16 multiply by one returns its operand,
// a NaN as the canonical NaN the update then produces anyway); the row's own
// operands are hin and hout only, held as one half2 through the chain.
template <bool PREFETCH = true, bool UNIT = false> struct EpiRichStepT {
  using Red = float;
  static constexpr int NV = 0;
  struct PreUnit {
    __half2 io;  // hin, hout
  };
  struct PreDiag {
    __half2 io;
    __half w, z;
  };
  using Pre = typename std::conditional<UNIT, PreUnit, PreDiag>::type;
  const __half *hin, *hout;
  DiagPre M;
  const RichState *rs;
  int k;
  __half *hnext;  // next hout (steps before the last)
  float *out;     // fp32 result (last step)
  float isc;
  float ome = 0.0f;  // fp32(ome[k]), set by setup()
  __device__ __forceinline__ void setup() { ome = h2f(rs->ome[k]); }
  __device__ __forceinline__ void fetch(int64_t r, Pre &p) const {
    p.io = __halves2half2(hin[r], hout[r]);
    if constexpr (!UNIT) {
      p.w = M.wv(r);
      p.z = M.zv(r);
    }
  }
  __device__ __forceinline__ Pre load(int64_t r) const {
    Pre p{};
    if (PREFETCH) fetch(r, p);
    return p;
  }
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, Acc acc, const Pre &pp, Red (&)[1]) const {
    Pre p = pp;
    if (!PREFETCH) fetch(r, p);
    // The product of two fp16 values is exact in fp32, so the fp16 multiply
    // (one correctly rounded result) gives the bits of fp16(float(a) * float(b))
    // in one instruction; the subtraction (fp32 acc) and the fused update keep
    // their fp32 arithmetic.
    const __half hr = f2h(h2f(__low2half(p.io)) - (float)acc);
    __half t2 = hr;
    if constexpr (!UNIT) t2 = __hmul(p.z, __hmul(p.w, hr));
    // hnew is rounded to fp16 once; the fp16 store takes it as it is (widening
    // and rounding it again would give the same bits)
    const __half hn = f2h(__fmaf_rn(ome, h2f(t2), h2f(__high2half(p.io))));
    if (out) out[r] = h2f(hn) * isc;
    else hnext[r] = hn;
  }
  template <int W> __device__ __forceinline__ void finish(Red (&)[1]) const {}
};
using EpiRichStep = EpiRichStepT<true>;
using EpiRichStepUnit = EpiRichStepT<true, true>;

// Residual step of an update call (diagonal M): stores hr and t2 = M hr.
struct EpiRichResPre {
  using Red = float;
  static constexpr int NV = 0;
  struct Pre {
    __half hin, w, z;
  };
  const __half *hin;
  DiagPre M;
  __half *hr, *t2;
  __device__ __forceinline__ Pre load(int64_t r) const { return {hin[r], M.wv(r), M.zv(r)}; }
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, Acc acc, const Pre &p, Red (&)[1]) const {
    const __half h = f2h(h2f(p.hin) - (float)acc);
    hr[r] = h;
    const float t = h2f(f2h(h2f(p.w) * h2f(h)));
    t2[r] = f2h(h2f(p.z) * t);
  }
  template <int W> __device__ __forceinline__ void finish(Red (&)[1]) const {}
};

// Weight computation of an update call: tmp = fp16(A16 v) stored, and
// dot_ar = <tmp, tmp>, dot_r = <tmp, other> in fp32 (wildcard(., tof32),
// f3r-gpu.cpp:235-240 / 249-254); the finisher forms the weight and the
// running mean.  k = 0 also advances den = cnt / period.
struct EpiRichWeight {
  using Red = float;
  static constexpr int NV = 2;
  struct Pre {
    __half other;
  };
  __half *tmp;
  const __half *other;
  GridRed gr;
  RichState *rs;
  int k;
  __device__ __forceinline__ Pre load(int64_t r) const { return {other[r]}; }
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, Acc acc, const Pre &p, Red (&d)[2]) const {
    const __half t = f2h((float)acc);
    tmp[r] = t;
    const float tv = h2f(t);
    d[0] = __fmaf_rn(tv, tv, d[0]);
    d[1] = __fmaf_rn(tv, h2f(p.other), d[1]);
  }
  template <int W> __device__ __forceinline__ void finish(Red (&d)[2]) const {
    RichState *s = rs;
    const int kk = k;
    grid_reduce<float, 2, W>(d, 2, gr, [s, kk](float *tot) {
      const float om = tot[1] / tot[0];
      s->om[kk] = om;
      s->sum[kk] += om;
      if (kk == 0) s->den += 1;
      s->ome[kk] = __float2half_rn(s->sum[kk] / (float)s->den);
    });
  }
};

// hout = fp16(hout * fp16(om[0]))  (hout *= dot_r / dot_ar, f3r-gpu.cpp:238)
__global__ void k_rich_scale_om(__half *__restrict__ hout, const RichState *__restrict__ rs, int64_t n) {
  const float om = h2f(f2h(rs->om[0]));
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    hout[i] = f2h(h2f(hout[i]) * om);
}

// hout = fp16(hout + om[k] t2) (f3r-gpu.cpp:252), or on the last step out =
// fp32(that) / sc, or out16 = that (R below the fp16-vector level).  use_ome
// selects ome[k] (no-update calls, general M).
__global__ void k_rich_axpy(__half *__restrict__ hout, const __half *__restrict__ t2,
                            const RichState *__restrict__ rs, int k, int use_ome, float *__restrict__ out,
                            __half *__restrict__ out16, float isc, int64_t n) {
  const float om = use_ome ? h2f(rs->ome[k]) : rs->om[k];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float hn = h2f(f2h(__fmaf_rn(om, h2f(t2[i]), h2f(hout[i]))));
    if (out) out[i] = hn * isc;
    else if (out16) out16[i] = f2h(hn);
    else hout[i] = f2h(hn);
  }
}

// out = fp32(hout) / sc (m4 = 1: R is the preconditioner application alone)
__global__ void k_rich_exit(const __half *__restrict__ hout, float *__restrict__ out, float isc, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = h2f(hout[i]) * isc;
}

// General M, Z apply: hout = fp16(Z tmp), then (no-update calls) hout *=
// ome[0] as a second rounding, as the reference's separate statements.
struct EpiZScale {
  using Red = float;
  using Pre = NoPre;
  static constexpr int NV = 0;
  __half *hout;
  const RichState *rs;
  int scale;
  __device__ __forceinline__ Pre load(int64_t) const { return {}; }
  template <typename Acc> __device__ __forceinline__ void row(int64_t r, Acc acc, const Pre &, Red (&)[1]) const {
    __half h = f2h((float)acc);
    if (scale) h = f2h(h2f(h) * h2f(rs->ome[0]));
    hout[r] = h;
  }
  template <int W> __device__ __forceinline__ void finish(Red (&)[1]) const {}
};

// fp32 -> fp64 / fp16 / fp32 conversion of a value array (matrix copies).
template <typename To> __global__ void k_convert_vals(const double *__restrict__ in, To *__restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = cvt<To>(in[i]);
}

// gather / scatter through a row permutation (SELL-C-sigma system order)
__global__ void k_permute_gather(const double *__restrict__ in, const int32_t *__restrict__ perm,
                                 double *__restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[perm[i]];
}
__global__ void k_permute_scatter(const double *__restrict__ in, const int32_t *__restrict__ perm,
                                  double *__restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[perm[i]] = in[i];
}

// ---------------------------------------------------------------------------
// The fp16-vector FGMRES level (FGMRES<_Float16>, depth.cpp:122-167): V and Z
// stored in fp16, every dot, norm, update and Givens rotation computed in
// fp32 (the reference computes them in fp16).  Vectors of the level start on
// 16-byte boundaries (columns of ldn elements, ldn a multiple of 8), so a
// thread moves 8 values per access.
// ---------------------------------------------------------------------------

// Entry: the caller's basis vector -- an fp32 column of an inner level, or
// the outer level's fp64 column read through a slot -- is normalised in
// place when its 1/h factor is given (deferred V(j+1) *= h.inv(),
// gmres.hpp:117), then V(0) = fp16(in) (V(0).copy(rhs), gmres.hpp:102),
// e(0) = 1 (normalize = false, gmres.hpp:100-101), and the caller's own e(0)
// = 1 when e_parent is given (the caller's first inner call sets it).
__device__ __forceinline__ __half round_half(float v) { return __float2half_rn(v); }
__device__ __forceinline__ __half round_half(double v) { return __double2half(v); }  // one rounding

template <typename In>
__global__ void k_level_enter_h(In *in_direct, In *const *in_slot, const In *__restrict__ in_inv,
                                __half *__restrict__ v0, float *e, float *e_parent, int64_t n) {
  In *in = in_slot ? *in_slot : in_direct;
  const In s = in_inv ? *in_inv : In(1);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    e[0] = 1.0f;
    if (e_parent) e_parent[0] = 1.0f;
  }
  constexpr int N = 16 / sizeof(In);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n8 = n / 8;
  for (int64_t q = tid; q < n8; q += stride) {
    const int64_t i = 8 * q;
    VecN<__half, 8> o;
#pragma unroll
    for (int c = 0; c < 8 / N; c++) {
      VecN<In, N> a = ldv<In, N>(in + i + c * N);
      if (in_inv) {
#pragma unroll
        for (int e = 0; e < N; e++) a.v[e] *= s;
        stv<In, N>(in + i + c * N, a);
      }
#pragma unroll
      for (int e = 0; e < N; e++) o.v[c * N + e] = round_half(a.v[e]);
    }
    stv<__half, 8>(v0 + i, o);
  }
  for (int64_t i = n8 * 8 + tid; i < n; i += stride) {
    In v = in[i];
    if (in_inv) {
      v *= s;
      in[i] = v;
    }
    v0[i] = round_half(v);
  }
}

// H(j, k) = <w, V(k)> for k < nv, fp16 vectors, fp32 accumulation (the CGS
// dot phase, gmres.hpp:112-114): basis vectors in chunks of 8 per pass over
// w, partial sums per block, then the last block adds them in block order.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_multidot_h(const __half *__restrict__ w, Cols<__half> V, int nv,
                                                           int64_t n, GridRed gr, float *hcol) {
  constexpr int CH = 8;
  float *part = static_cast<float *>(gr.partials);
  __shared__ float sred[WARPS][CH];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n8 = n / 8;
  for (int k0 = 0; k0 < nv; k0 += CH) {
    float a[CH];
#pragma unroll
    for (int c = 0; c < CH; c++) a[c] = 0.0f;
    for (int64_t q = tid; q < n8; q += stride) {
      const VecN<__half, 8> wv = ldv<__half, 8>(w + 8 * q);
#pragma unroll
      for (int c = 0; c < CH; c++) {
        if (k0 + c < nv) {
          const VecN<__half, 8> v = ldv<__half, 8>(V.p[k0 + c] + 8 * q);
#pragma unroll
          for (int e = 0; e < 8; e++) a[c] = __fmaf_rn(__half2float(wv.v[e]), __half2float(v.v[e]), a[c]);
        }
      }
    }
    for (int64_t i = n8 * 8 + tid; i < n; i += stride) {
      const float wi = __half2float(w[i]);
#pragma unroll
      for (int c = 0; c < CH; c++)
        if (k0 + c < nv) a[c] = __fmaf_rn(wi, __half2float(V.p[k0 + c][i]), a[c]);
    }
#pragma unroll
    for (int c = 0; c < CH; c++) {
      const float t = warp_sum(a[c]);
      if (lane == 0) sred[warp][c] = t;
    }
    __syncthreads();
    if (threadIdx.x < CH && k0 + (int)threadIdx.x < nv) {
      float t = 0;
      for (int q = 0; q < WARPS; q++) t += sred[q][threadIdx.x];
      part[(size_t)blockIdx.x * nv + k0 + threadIdx.x] = t;
    }
    __syncthreads();
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(gr.ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int k = warp; k < nv; k += WARPS) {
    float t = 0;
    for (int b = lane; b < (int)gridDim.x; b += 32) t += __ldcg(&part[(size_t)b * nv + k]);
    t = warp_sum(t);
    if (lane == 0) hcol[k] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) *gr.ticket = 0;
}

// w = fp16(w - sum_k H(j,k) V(k)) (MULMV order, in fp32), then the squared
// norm of the stored fp16 w -> h_{j+1,j}, 1/h, the Givens rotation and, after
// the level's last step, the back substitution (gmres.hpp:115-121).
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_cgs_update_h(__half *__restrict__ w, Cols<__half> V, int nv,
                                                             int64_t n, GridRed gr, GivensCtl<float> g) {
  __shared__ float sh[kMaxCols];
  const float *hcol = g.H + (size_t)g.j * g.ldh;
  for (int k = threadIdx.x; k < nv; k += blockDim.x) sh[k] = hcol[k];
  __syncthreads();
  float part[1] = {0.0f};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n8 = n / 8;
  for (int64_t q = tid; q < n8; q += stride) {
    const int64_t i = q * 8;
    const VecN<__half, 8> a = ldv<__half, 8>(V.p[0] + i);
    float r[8];
#pragma unroll
    for (int e = 0; e < 8; e++) r[e] = __half2float(a.v[e]) * sh[0];
#pragma unroll 4
    for (int k = 1; k < nv; k++) {
      const VecN<__half, 8> b = ldv<__half, 8>(V.p[k] + i);
      const float hk = sh[k];
#pragma unroll
      for (int e = 0; e < 8; e++) r[e] = __fmaf_rn(__half2float(b.v[e]), hk, r[e]);
    }
    VecN<__half, 8> wv = ldv<__half, 8>(w + i);
#pragma unroll
    for (int e = 0; e < 8; e++) {
      wv.v[e] = __float2half_rn(__half2float(wv.v[e]) - r[e]);
      const float u = __half2float(wv.v[e]);
      part[0] = __fmaf_rn(u, u, part[0]);
    }
    stv<__half, 8>(w + i, wv);
  }
  for (int64_t i = n8 * 8 + tid; i < n; i += stride) {
    float r = __half2float(V.p[0][i]) * sh[0];
    for (int k = 1; k < nv; k++) r = __fmaf_rn(__half2float(V.p[k][i]), sh[k], r);
    const __half wi = __float2half_rn(__half2float(w[i]) - r);
    w[i] = wi;
    const float u = __half2float(wi);
    part[0] = __fmaf_rn(u, u, part[0]);
  }
  const GivensCtl<float> gg = g;
  grid_reduce<float, 1, WARPS>(part, 1, gr, [gg](float *tot) { givens_step<float>(gg, tot[0]); });
}

// x = Z y of the fp16-vector level (with_init, gmres.hpp:127-128): fp16 Z,
// fp32 y and sum, stored in the caller's type (fp32 column, or the outer
// level's fp64 column through a slot).
template <typename Out>
__global__ void k_zy_h(Cols<__half> Z, const float *__restrict__ y, int nz, Out *out_direct, Out *const *out_slot,
                       int64_t n) {
  __shared__ float sy[kMaxCols];
  for (int k = threadIdx.x; k < nz; k += blockDim.x) sy[k] = y[k];
  __syncthreads();
  Out *out = out_slot ? *out_slot : out_direct;
  constexpr int N = 16 / sizeof(Out);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n8 = n / 8;
  for (int64_t q = tid; q < n8; q += stride) {
    const int64_t i = q * 8;
    const VecN<__half, 8> a = ldv<__half, 8>(Z.p[0] + i);
    float r[8];
#pragma unroll
    for (int e = 0; e < 8; e++) r[e] = __half2float(a.v[e]) * sy[0];
#pragma unroll 4
    for (int k = 1; k < nz; k++) {
      const VecN<__half, 8> b = ldv<__half, 8>(Z.p[k] + i);
      const float yk = sy[k];
#pragma unroll
      for (int e = 0; e < 8; e++) r[e] = __fmaf_rn(__half2float(b.v[e]), yk, r[e]);
    }
#pragma unroll
    for (int c = 0; c < 8 / N; c++) {
      VecN<Out, N> o;
#pragma unroll
      for (int e = 0; e < N; e++) o.v[e] = (Out)r[c * N + e];
      stv<Out, N>(out + i + c * N, o);
    }
  }
  for (int64_t i = n8 * 8 + tid; i < n; i += stride) {
    float r = __half2float(Z.p[0][i]) * sy[0];
    for (int k = 1; k < nz; k++) r = __fmaf_rn(__half2float(Z.p[k][i]), sy[k], r);
    out[i] = (Out)r;
  }
}

// <x, y> with the deterministic grid reduction (kmm::dot)
template <typename T, typename Acc, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_dot(const T *__restrict__ x, const T *__restrict__ y, int64_t n,
                                                    GridRed gr, Acc *out) {
  Acc part[1] = {0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    part[0] = fmaT(to_acc<Acc>(x[i]), to_acc<Acc>(y[i]), part[0]);
  grid_reduce<Acc, 1, WARPS>(part, 1, gr, [out](Acc *tot) { *out = tot[0]; });
}

}  // namespace f3r
