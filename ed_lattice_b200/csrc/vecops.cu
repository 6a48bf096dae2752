// vecops.cu -- the fused vector passes of the Lanczos recurrence.
//
// The recurrence of sp_lanc_tridiag / sp_lanc_eigh (called from src/DIAG/HAMILTONIAN.f90:268
// and src/DIAG/DIAG.f90:216) split into three HBM passes around H x v:
//   step A : w <- Hv - b_j v_{j-1};        a_j = <v_j|w>            (reads 3 vectors, writes 1)
//   step B : w <- w - a_j v_j;             b_{j+1}^2 = <w|w>        (reads 2, writes 1)
//   scale  : v_{j+1} <- w / b_{j+1}                                   (reads 1, writes 1)
// Element arithmetic is FP64 (FP32 vectors are widened on load and rounded once on store);
// dot products accumulate in FP64 over a fixed grid of kRedBlocks blocks followed by a
// one-block pass in fixed order, so results are bit-reproducible run to run.
// Scalars (a, b) live in device memory and are read by the next kernel: no host round trip
// is needed between the passes.
#include <cstdint>

#include "common.cuh"
#include "reduce.cuh"

namespace edg {
namespace {

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[kRedThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    r = lane < kRedThreads / 32 ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  return r;  // valid in thread 0
}

// Block mode: blockIdx.y is a column of a block of vectors (vectors vstride elements apart,
// device scalars sstride apart, reduction scratch kRedSlots apart); a column whose active[c]
// is 0 is skipped. Single-vector launches pass Cols{} (gridDim.y == 1).
struct Cols {
  int64_t vstride = 0, sstride = 0;
  const int* active = nullptr;
};
__device__ __forceinline__ bool col_on(const Cols& k) { return !k.active || k.active[blockIdx.y]; }
__device__ __forceinline__ int64_t col_v(const Cols& k) { return int64_t(blockIdx.y) * k.vstride; }
__device__ __forceinline__ int64_t col_s(const Cols& k) { return int64_t(blockIdx.y) * k.sstride; }
__device__ __forceinline__ int64_t col_r(const Cols&) { return int64_t(blockIdx.y) * kRedSlots; }

// Grid-stride loops below take kUnr elements per thread per trip (indices i + u*stride, each
// coalesced across the warp) with all loads issued before the arithmetic, so that every
// thread keeps several HBM requests in flight; the order of the partial sums is fixed.
constexpr int kUnr = 4;

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_dot(const T* __restrict__ x, const T* __restrict__ y, int64_t n,
                                                     double* __restrict__ partial, double* __restrict__ out,
                                                     int do_sqrt, Cols cl) {
  if (!col_on(cl)) return;
  x += col_v(cl);
  y += col_v(cl);
  partial += col_r(cl);
  out += col_s(cl);
  const int64_t st = int64_t(gridDim.x) * blockDim.x;
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  double s = 0.0;
  for (; i + (kUnr - 1) * st < n; i += kUnr * st) {
    T xa[kUnr], ya[kUnr];
#pragma unroll
    for (int u = 0; u < kUnr; ++u) {
      xa[u] = x[i + u * st];
      ya[u] = y[i + u * st];
    }
#pragma unroll
    for (int u = 0; u < kUnr; ++u) s = __fma_rn(double(xa[u]), double(ya[u]), s);
  }
  for (; i < n; i += st) s = __fma_rn(double(x[i]), double(y[i]), s);
  s = block_sum(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  finish_in_last_block(partial, gridDim.x, out, do_sqrt);
}

// out = sum(partial) (do_sqrt: sqrt of the sum)
__global__ void __launch_bounds__(kRedThreads) k_finish(const double* __restrict__ partial, int nblk,
                                                        double* __restrict__ out, int do_sqrt) {
  double s = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) s += partial[i];
  s = block_sum(s);
  if (threadIdx.x == 0) out[0] = do_sqrt ? sqrt(s) : s;
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_step_a(T* __restrict__ w, const T* __restrict__ vprev,
                                                        const T* __restrict__ v, const double* __restrict__ bprev,
                                                        int64_t n, double* __restrict__ partial,
                                                        double* __restrict__ out, Cols cl) {
  if (!col_on(cl)) return;
  w += col_v(cl);
  vprev += col_v(cl);
  v += col_v(cl);
  bprev += col_s(cl);
  partial += col_r(cl);
  out += col_s(cl);
  const double b = *bprev;
  const int64_t st = int64_t(gridDim.x) * blockDim.x;
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  double s = 0.0;
  for (; i + (kUnr - 1) * st < n; i += kUnr * st) {
    T wa[kUnr], pa[kUnr], va[kUnr];
#pragma unroll
    for (int u = 0; u < kUnr; ++u) {
      wa[u] = w[i + u * st];
      pa[u] = vprev[i + u * st];
      va[u] = v[i + u * st];
    }
#pragma unroll
    for (int u = 0; u < kUnr; ++u) {
      const T wt = T(double(wa[u]) - b * double(pa[u]));
      w[i + u * st] = wt;
      s = __fma_rn(double(va[u]), double(wt), s);
    }
  }
  for (; i < n; i += st) {
    const T wt = T(double(w[i]) - b * double(vprev[i]));
    w[i] = wt;
    s = __fma_rn(double(v[i]), double(wt), s);
  }
  s = block_sum(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  finish_in_last_block(partial, gridDim.x, out, 0);
}

// w <- w - coef * x, returning this thread's partial sum of |w|^2
template <typename T>
__device__ __forceinline__ double axpy_norm(T* __restrict__ w, const T* __restrict__ x, double coef, int64_t n) {
  const int64_t st = int64_t(gridDim.x) * blockDim.x;
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  double s = 0.0;
  for (; i + (kUnr - 1) * st < n; i += kUnr * st) {
    T wa[kUnr], xa[kUnr];
#pragma unroll
    for (int u = 0; u < kUnr; ++u) {
      wa[u] = w[i + u * st];
      xa[u] = x[i + u * st];
    }
#pragma unroll
    for (int u = 0; u < kUnr; ++u) {
      const T wt = T(double(wa[u]) - coef * double(xa[u]));
      w[i + u * st] = wt;
      s = __fma_rn(double(wt), double(wt), s);
    }
  }
  for (; i < n; i += st) {
    const T wt = T(double(w[i]) - coef * double(x[i]));
    w[i] = wt;
    s = __fma_rn(double(wt), double(wt), s);
  }
  return s;
}

// 16-byte vector forms (float4 / double2) for arrays whose length is a multiple of K and
// whose pointers are 16-byte aligned: four times the bytes in flight per load instruction.
template <typename T>
struct V16;
template <>
struct V16<float> {
  using type = float4;
  static constexpr int K = 4;
};
template <>
struct V16<double> {
  using type = double2;
  static constexpr int K = 2;
};

template <typename T>
__device__ __forceinline__ double axpy_norm_v(T* __restrict__ w, const T* __restrict__ x, double coef, int64_t nv) {
  using V = typename V16<T>::type;
  constexpr int K = V16<T>::K;
  V* __restrict__ wv = reinterpret_cast<V*>(w);
  const V* __restrict__ xv = reinterpret_cast<const V*>(x);
  const int64_t st = int64_t(gridDim.x) * blockDim.x;
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nv; i += 2 * st) {
    V wa[2], xa[2];
    const bool two = i + st < nv;
    wa[0] = wv[i];
    xa[0] = xv[i];
    if (two) {
      wa[1] = wv[i + st];
      xa[1] = xv[i + st];
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (u == 1 && !two) break;
      T* pw = reinterpret_cast<T*>(&wa[u]);
      const T* px = reinterpret_cast<const T*>(&xa[u]);
#pragma unroll
      for (int c = 0; c < K; ++c) {
        pw[c] = T(double(pw[c]) - coef * double(px[c]));
        s = __fma_rn(double(pw[c]), double(pw[c]), s);
      }
      wv[i + u * st] = wa[u];
    }
  }
  return s;
}

template <typename T>
__device__ __forceinline__ double dot_v(const T* __restrict__ x, const T* __restrict__ y, int64_t nv) {
  using V = typename V16<T>::type;
  constexpr int K = V16<T>::K;
  const V* __restrict__ xv = reinterpret_cast<const V*>(x);
  const V* __restrict__ yv = reinterpret_cast<const V*>(y);
  const int64_t st = int64_t(gridDim.x) * blockDim.x;
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nv; i += 2 * st) {
    V xa[2], ya[2];
    const bool two = i + st < nv;
    xa[0] = xv[i];
    ya[0] = yv[i];
    if (two) {
      xa[1] = xv[i + st];
      ya[1] = yv[i + st];
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (u == 1 && !two) break;
      const T* px = reinterpret_cast<const T*>(&xa[u]);
      const T* py = reinterpret_cast<const T*>(&ya[u]);
#pragma unroll
      for (int c = 0; c < K; ++c) s = __fma_rn(double(px[c]), double(py[c]), s);
    }
  }
  return s;
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_dot_v(const T* __restrict__ x, const T* __restrict__ y, int64_t nv,
                                                       double* __restrict__ partial, double* __restrict__ out,
                                                       int do_sqrt, Cols cl) {
  if (!col_on(cl)) return;
  x += col_v(cl);
  y += col_v(cl);
  partial += col_r(cl);
  out += col_s(cl);
  double s = dot_v<T>(x, y, nv);
  s = block_sum(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  finish_in_last_block(partial, gridDim.x, out, do_sqrt);
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_step_b2_v(T* __restrict__ w, const T* __restrict__ u,
                                                           const double* __restrict__ a,
                                                           const double* __restrict__ bn, int64_t nv,
                                                           double* __restrict__ partial, double* __restrict__ out,
                                                           Cols cl) {
  if (!col_on(cl)) return;
  w += col_v(cl);
  u += col_v(cl);
  a += col_s(cl);
  bn += col_s(cl);
  partial += col_r(cl);
  out += col_s(cl);
  double s = axpy_norm_v<T>(w, u, *a / *bn, nv);
  s = block_sum(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  finish_in_last_block(partial, gridDim.x, out, 1);
}

template <typename T>
bool vec16_ok(int64_t n, const void* p, const void* q) {
  return n % V16<T>::K == 0 && (reinterpret_cast<uintptr_t>(p) % 16) == 0 && (reinterpret_cast<uintptr_t>(q) % 16) == 0;
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_step_b(T* __restrict__ w, const T* __restrict__ v,
                                                        const double* __restrict__ a, int64_t n,
                                                        double* __restrict__ partial, double* __restrict__ out,
                                                        Cols cl) {
  if (!col_on(cl)) return;
  w += col_v(cl);
  v += col_v(cl);
  a += col_s(cl);
  partial += col_r(cl);
  out += col_s(cl);
  double s = axpy_norm<T>(w, v, *a, n);
  s = block_sum(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  finish_in_last_block(partial, gridDim.x, out, 1);
}

// Fused recurrence, second half: u_{j+1} = w - (a_j / bn_j) u_j in place on w, and the
// partial sums of |u_{j+1}|^2 (bn_{j+1} after the finish pass).
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_step_b2(T* __restrict__ w, const T* __restrict__ u,
                                                         const double* __restrict__ a, const double* __restrict__ bn,
                                                         int64_t n, double* __restrict__ partial,
                                                         double* __restrict__ out, Cols cl) {
  if (!col_on(cl)) return;
  w += col_v(cl);
  u += col_v(cl);
  a += col_s(cl);
  bn += col_s(cl);
  partial += col_r(cl);
  out += col_s(cl);
  double s = axpy_norm<T>(w, u, *a / *bn, n);
  s = block_sum(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  finish_in_last_block(partial, gridDim.x, out, 1);
}

// dst[i] = T(src[i] * scale); dst and src do not overlap
template <typename TD, typename TS>
__device__ __forceinline__ void scale_copy(TD* __restrict__ dst, const TS* __restrict__ src, int64_t n, double scale) {
  const int64_t st = int64_t(gridDim.x) * blockDim.x;
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  for (; i + (kUnr - 1) * st < n; i += kUnr * st) {
    TS xa[kUnr];
#pragma unroll
    for (int u = 0; u < kUnr; ++u) xa[u] = src[i + u * st];
#pragma unroll
    for (int u = 0; u < kUnr; ++u) dst[i + u * st] = TD(double(xa[u]) * scale);
  }
  for (; i < n; i += st) dst[i] = TD(double(src[i]) * scale);
}

template <typename T>
__global__ void k_scale_into(T* __restrict__ dst, const T* __restrict__ src, const double* __restrict__ b, int64_t n,
                             Cols cl) {
  if (!col_on(cl)) return;
  dst += col_v(cl);
  src += col_v(cl);
  b += col_s(cl);
  const double bb = *b;
  scale_copy<T, T>(dst, src, n, bb != 0.0 ? 1.0 / bb : 0.0);
}

template <typename TD, typename TS>
__global__ void k_convert(TD* __restrict__ dst, const TS* __restrict__ src, int64_t n, double scale) {
  scale_copy<TD, TS>(dst, src, n, scale);
}

// dst_c = TD(src_c / sqrt(norm2[c])) for every column (zero when norm2[c] is 0)
template <typename TD, typename TS>
__global__ void k_normalise_cols(TD* __restrict__ dst, int64_t dstride, const TS* __restrict__ src, int64_t sstride_v,
                                 const double* __restrict__ norm2, int64_t sstride, int64_t n) {
  const double n2 = norm2[int64_t(blockIdx.y) * sstride];
  scale_copy<TD, TS>(dst + int64_t(blockIdx.y) * dstride, src + int64_t(blockIdx.y) * sstride_v, n,
                     n2 > 0.0 ? 1.0 / sqrt(n2) : 0.0);
}

// x[i] *= scale in place
template <typename T>
__global__ void k_scale_inplace(T* __restrict__ x, int64_t n, double scale) {
  const int64_t st = int64_t(gridDim.x) * blockDim.x;
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  for (; i + (kUnr - 1) * st < n; i += kUnr * st) {
    T xa[kUnr];
#pragma unroll
    for (int u = 0; u < kUnr; ++u) xa[u] = x[i + u * st];
#pragma unroll
    for (int u = 0; u < kUnr; ++u) x[i + u * st] = T(double(xa[u]) * scale);
  }
  for (; i < n; i += st) x[i] = T(double(x[i]) * scale);
}

template <typename TS>
__global__ void k_axpy_accum(double* __restrict__ dst, const TS* __restrict__ x, double coef, int64_t n) {
  const int64_t st = int64_t(gridDim.x) * blockDim.x;
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  for (; i + (kUnr - 1) * st < n; i += kUnr * st) {
    double da[kUnr];
    TS xa[kUnr];
#pragma unroll
    for (int u = 0; u < kUnr; ++u) {
      da[u] = dst[i + u * st];
      xa[u] = x[i + u * st];
    }
#pragma unroll
    for (int u = 0; u < kUnr; ++u) dst[i + u * st] = __fma_rn(coef, double(xa[u]), da[u]);
  }
  for (; i < n; i += st) dst[i] = __fma_rn(coef, double(x[i]), dst[i]);
}

// x[i] = sum_j z[j] * basis[j][i] in one pass over the stored FP32 Lanczos basis (z in FP64,
// j ascending: the same FMA sequence as m successive axpys, one read of each column).
__global__ void __launch_bounds__(256) k_ritz(const float* __restrict__ basis, const double* __restrict__ z, int m,
                                              int64_t n, double* __restrict__ x) {
  extern __shared__ double s_z[];
  for (int j = threadIdx.x; j < m; j += blockDim.x) s_z[j] = z[j];
  __syncthreads();
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double acc = 0.0;
    for (int j = 0; j < m; ++j) acc = __fma_rn(s_z[j], double(__ldcs(basis + int64_t(j) * n + i)), acc);
    x[i] = acc;
  }
}

// k_ritz with four consecutive elements per thread (16-byte loads; n % 4 == 0 and a 16-byte
// aligned basis) and four columns' loads issued together; each element's terms are added in
// the same order as k_ritz, so the results are the same bits.
__global__ void __launch_bounds__(256) k_ritz_v4(const float4* __restrict__ basis, const double* __restrict__ z,
                                                 int m, int64_t n4, double2* __restrict__ x) {
  extern __shared__ double s_z4[];
  for (int j = threadIdx.x; j < m; j += blockDim.x) s_z4[j] = z[j];
  __syncthreads();
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n4; i += int64_t(gridDim.x) * blockDim.x) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int j = 0;
    for (; j + 4 <= m; j += 4) {
      float4 b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) b[u] = __ldcs(basis + int64_t(j + u) * n4 + i);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double c = s_z4[j + u];
        a0 = __fma_rn(c, double(b[u].x), a0);
        a1 = __fma_rn(c, double(b[u].y), a1);
        a2 = __fma_rn(c, double(b[u].z), a2);
        a3 = __fma_rn(c, double(b[u].w), a3);
      }
    }
    for (; j < m; ++j) {
      const float4 b = __ldcs(basis + int64_t(j) * n4 + i);
      const double c = s_z4[j];
      a0 = __fma_rn(c, double(b.x), a0);
      a1 = __fma_rn(c, double(b.y), a1);
      a2 = __fma_rn(c, double(b.z), a2);
      a3 = __fma_rn(c, double(b.w), a3);
    }
    x[2 * i] = make_double2(a0, a1);
    x[2 * i + 1] = make_double2(a2, a3);
  }
}

__device__ __host__ __forceinline__ uint64_t splitmix64_d(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__global__ void k_random(double* __restrict__ dst, int64_t n, uint64_t seed) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t z = splitmix64_d(seed + uint64_t(i));
    dst[i] = double(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
  }
}

inline int grid_for(int64_t n) {
  int64_t g = (n + 255) / 256;
  return int(g < 148 * 16 ? (g < 1 ? 1 : g) : 148 * 16);
}

}  // namespace

uint64_t splitmix64(uint64_t x) { return splitmix64_d(x); }

template <typename T>
int dot_dev(cudaStream_t st, const T* x, const T* y, int64_t n, double* partial, double* out) {
  if (vec16_ok<T>(n, x, y))
    k_dot_v<T><<<kRedBlocks, kRedThreads, 0, st>>>(x, y, n / V16<T>::K, partial, out, 0, Cols{});
  else
    k_dot<T><<<kRedBlocks, kRedThreads, 0, st>>>(x, y, n, partial, out, 0, Cols{});
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

template <typename T>
int lanczos_step_a(cudaStream_t st, T* w, const T* vprev, const T* v, const double* bprev, int64_t n, double* partial,
                   double* aout) {
  k_step_a<T><<<kRedBlocks, kRedThreads, 0, st>>>(w, vprev, v, bprev, n, partial, aout, Cols{});
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

template <typename T>
int lanczos_step_b(cudaStream_t st, T* w, const T* v, const double* a, int64_t n, double* partial, double* bout) {
  k_step_b<T><<<kRedBlocks, kRedThreads, 0, st>>>(w, v, a, n, partial, bout, Cols{});
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

template <typename T>
int lanczos_step_b2(cudaStream_t st, T* w, const T* u, const double* a, const double* bn, int64_t n, double* partial,
                    double* bn_next) {
  if (vec16_ok<T>(n, w, u))
    k_step_b2_v<T><<<kRedBlocks, kRedThreads, 0, st>>>(w, u, a, bn, n / V16<T>::K, partial, bn_next, Cols{});
  else
    k_step_b2<T><<<kRedBlocks, kRedThreads, 0, st>>>(w, u, a, bn, n, partial, bn_next, Cols{});
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

int norm_dev(cudaStream_t st, const double* x, int64_t n, double* partial, double* out) {
  if (vec16_ok<double>(n, x, x))
    k_dot_v<double><<<kRedBlocks, kRedThreads, 0, st>>>(x, x, n / V16<double>::K, partial, out, 1, Cols{});
  else
    k_dot<double><<<kRedBlocks, kRedThreads, 0, st>>>(x, x, n, partial, out, 1, Cols{});
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

int red_scratch_reset(cudaStream_t st, double* partial) {
  EDG_CUDA(cudaMemsetAsync(partial + kRedBlocks, 0, sizeof(double), st));
  return EDG_OK;
}

int finish_dev(cudaStream_t st, const double* partial, int nblk, double* out, int do_sqrt) {
  k_finish<<<1, kRedThreads, 0, st>>>(partial, nblk, out, do_sqrt);
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

template <typename T>
int scale_into(cudaStream_t st, T* dst, const T* src, const double* b, int64_t n) {
  k_scale_into<T><<<grid_for(n), 256, 0, st>>>(dst, src, b, n, Cols{});
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

template <typename TD, typename TS>
int convert_dev(cudaStream_t st, TD* dst, const TS* src, int64_t n, double scale) {
  k_convert<TD, TS><<<grid_for(n), 256, 0, st>>>(dst, src, n, scale);
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

template <typename T>
int scale_inplace_dev(cudaStream_t st, T* x, int64_t n, double scale) {
  k_scale_inplace<T><<<grid_for(n), 256, 0, st>>>(x, n, scale);
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}
template int scale_inplace_dev<double>(cudaStream_t, double*, int64_t, double);
template int scale_inplace_dev<float>(cudaStream_t, float*, int64_t, double);

template <typename TS>
int axpy_accum_dev(cudaStream_t st, double* dst, const TS* x, double coef, int64_t n) {
  k_axpy_accum<TS><<<grid_for(n), 256, 0, st>>>(dst, x, coef, n);
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

int ritz_dev(cudaStream_t st, const float* basis, const double* z_dev, int m, int64_t n, double* x) {
  const size_t smem = size_t(m) * sizeof(double);
  if (smem > 48 * 1024) {
    set_error("ritz_dev: %d basis columns exceed the shared-memory coefficient cache", m);
    return EDG_ERR_ARG;
  }
  if (n % 4 == 0 && reinterpret_cast<uintptr_t>(basis) % 16 == 0 && reinterpret_cast<uintptr_t>(x) % 16 == 0)
    k_ritz_v4<<<grid_for(n / 4), 256, smem, st>>>(reinterpret_cast<const float4*>(basis), z_dev, m, n / 4,
                                                   reinterpret_cast<double2*>(x));
  else
    k_ritz<<<grid_for(n), 256, smem, st>>>(basis, z_dev, m, n, x);
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

int random_dev(cudaStream_t st, double* dst, int64_t n, uint64_t seed) {
  k_random<<<grid_for(n), 256, 0, st>>>(dst, n, seed);
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

// ---- block forms: ncols columns, vectors vstride elements apart, device scalars sstride
// apart, reduction scratch kRedSlots apart per column; inactive columns skipped
inline dim3 col_grid(int nblk, int ncols) { return dim3(nblk, ncols); }

template <typename T>
int dot_cols(cudaStream_t st, int ncols, const T* x, const T* y, int64_t n, int64_t vstride, double* partial,
             double* out, int64_t sstride, int do_sqrt) {
  Cols cl{vstride, sstride, nullptr};
  if (vec16_ok<T>(n, x, y) && vstride % V16<T>::K == 0)
    k_dot_v<T><<<col_grid(kRedBlocks, ncols), kRedThreads, 0, st>>>(x, y, n / V16<T>::K, partial, out, do_sqrt, cl);
  else
    k_dot<T><<<col_grid(kRedBlocks, ncols), kRedThreads, 0, st>>>(x, y, n, partial, out, do_sqrt, cl);
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

template <typename TD, typename TS>
int normalise_cols(cudaStream_t st, int ncols, TD* dst, int64_t dstride, const TS* src, int64_t srcstride,
                   const double* norm2, int64_t sstride, int64_t n) {
  int g = grid_for(n) / ncols;
  if (g < 1) g = 1;
  k_normalise_cols<TD, TS><<<col_grid(g, ncols), 256, 0, st>>>(dst, dstride, src, srcstride, norm2, sstride, n);
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

template <typename T>
int lanczos_step_a_cols(cudaStream_t st, int ncols, const int* active, T* w, const T* vprev, const T* v,
                        int64_t vstride, const double* bprev, double* partial, double* aout, int64_t sstride, int64_t n) {
  k_step_a<T><<<col_grid(kRedBlocks, ncols), kRedThreads, 0, st>>>(w, vprev, v, bprev, n, partial, aout,
                                                                  Cols{vstride, sstride, active});
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

template <typename T>
int lanczos_step_b_cols(cudaStream_t st, int ncols, const int* active, T* w, const T* v, int64_t vstride,
                        const double* a, double* partial, double* bout, int64_t sstride, int64_t n) {
  k_step_b<T><<<col_grid(kRedBlocks, ncols), kRedThreads, 0, st>>>(w, v, a, n, partial, bout,
                                                                  Cols{vstride, sstride, active});
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

template <typename T>
int lanczos_step_b2_cols(cudaStream_t st, int ncols, const int* active, T* w, const T* u, int64_t vstride,
                         const double* a, const double* bn, double* partial, double* bn_next, int64_t sstride,
                         int64_t n) {
  const Cols cl{vstride, sstride, active};
  if (vec16_ok<T>(n, w, u) && vstride % V16<T>::K == 0)
    k_step_b2_v<T><<<col_grid(kRedBlocks, ncols), kRedThreads, 0, st>>>(w, u, a, bn, n / V16<T>::K, partial, bn_next,
                                                                       cl);
  else
    k_step_b2<T><<<col_grid(kRedBlocks, ncols), kRedThreads, 0, st>>>(w, u, a, bn, n, partial, bn_next, cl);
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

template <typename T>
int scale_into_cols(cudaStream_t st, int ncols, const int* active, T* dst, const T* src, int64_t vstride,
                    const double* b, int64_t sstride, int64_t n) {
  int g = grid_for(n) / ncols;
  if (g < 1) g = 1;
  k_scale_into<T><<<col_grid(g, ncols), 256, 0, st>>>(dst, src, b, n, Cols{vstride, sstride, active});
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

#define EDG_INST(T)                                                                                        \
  template int dot_dev<T>(cudaStream_t, const T*, const T*, int64_t, double*, double*);                   \
  template int lanczos_step_a<T>(cudaStream_t, T*, const T*, const T*, const double*, int64_t, double*,   \
                                 double*);                                                                 \
  template int lanczos_step_b<T>(cudaStream_t, T*, const T*, const double*, int64_t, double*, double*);   \
  template int scale_into<T>(cudaStream_t, T*, const T*, const double*, int64_t);                         \
  template int lanczos_step_b2<T>(cudaStream_t, T*, const T*, const double*, const double*, int64_t,      \
                                  double*, double*);                                                      \
  template int axpy_accum_dev<T>(cudaStream_t, double*, const T*, double, int64_t);                         \
  template int dot_cols<T>(cudaStream_t, int, const T*, const T*, int64_t, int64_t, double*, double*, int64_t,  \
                           int);                                                                           \
  template int lanczos_step_a_cols<T>(cudaStream_t, int, const int*, T*, const T*, const T*, int64_t,     \
                                      const double*, double*, double*, int64_t, int64_t);                  \
  template int lanczos_step_b_cols<T>(cudaStream_t, int, const int*, T*, const T*, int64_t, const double*, \
                                      double*, double*, int64_t, int64_t);                                 \
  template int lanczos_step_b2_cols<T>(cudaStream_t, int, const int*, T*, const T*, int64_t, const double*, \
                                       const double*, double*, double*, int64_t, int64_t);                 \
  template int scale_into_cols<T>(cudaStream_t, int, const int*, T*, const T*, int64_t, const double*,     \
                                  int64_t, int64_t);                                                       \
  template int normalise_cols<T, double>(cudaStream_t, int, T*, int64_t, const double*, int64_t,           \
                                         const double*, int64_t, int64_t);
EDG_INST(float)
EDG_INST(double)
#undef EDG_INST
template int convert_dev<float, double>(cudaStream_t, float*, const double*, int64_t, double);
template int convert_dev<double, float>(cudaStream_t, double*, const float*, int64_t, double);
template int convert_dev<double, double>(cudaStream_t, double*, const double*, int64_t, double);
template int convert_dev<float, float>(cudaStream_t, float*, const float*, int64_t, double);

}  // namespace edg
