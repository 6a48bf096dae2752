// hxv.cu -- the spin-factorised Hubbard H x v on the device.
//
// Hv = diag o v + (I (x) H_up) v + (H_dw (x) I) v, with v laid out as the reference's
// i = iup + idw*DimUp: a row-major DimDw x DimUp matrix V whose rows are contiguous in iup.
//  * diag(iup,idw) = Eup[iup] + Edw[idw] + U*popcount(mup & mdw)  (src/DIAG/direct/
//    HxV_local.f90:15-95 and stored/H_local.f90:15-89, one orbital),
//  * H_up acts inside each row: a gather along iup (direct/HxV_up.f90, spMatVec :193-207),
//  * H_dw combines whole rows: row idw' += h * row jdw, coalesced along iup
//    (direct/HxV_dw.f90, spMatVec :178-191).
// Summation order per output element follows the reference form being replaced:
//  STORED (spMatVec, src/DIAG/HAMILTONIAN_STORED_HxV.f90:159-220): diag, DW, UP;
//  DIRECT (directMatVec, src/DIAG/HAMILTONIAN_DIRECT_HxV.f90:19-59): diag, UP, DW;
// inside each spin part sources are added in ascending rank, as the reference's loops do.
#include <algorithm>
#include <cstdlib>
#include <type_traits>

#include "common.cuh"
#include "reduce.cuh"

namespace edg {
namespace {

template <typename T>
struct HxvArgs {
  const T* __restrict__ v;
  T* __restrict__ hv;
  int64_t dimup, dimdw;
  const uint32_t* __restrict__ off_up;
  const uint32_t* __restrict__ src_up;
  const T* __restrict__ val_up;
  const uint32_t* __restrict__ off_dw;
  const uint32_t* __restrict__ src_dw;
  const T* __restrict__ val_dw;
  const T* __restrict__ e_up;
  const T* __restrict__ e_dw;
  const uint32_t* __restrict__ map_up;
  const uint32_t* __restrict__ map_dw;
  T U;
  // Lanczos-fused mode (v = u / bn[jstep] is applied with the scale folded into the matrix
  // elements; the step forms w = Hv - (bn[j]/bn[j-1]) uprev and the up pass the partial
  // <v, w>; lz_sub_in_dw says which pass subtracts uprev)
  const double* __restrict__ bn = nullptr;
  int jstep = 0;
  const T* __restrict__ uprev = nullptr;
  double* __restrict__ partial = nullptr;  // reduction scratch [kRedSlots]
  double* __restrict__ red_out = nullptr;  // receives <v, w>
  // Block mode (several vectors of the sector in one launch, blockIdx.y = column c): column c
  // reads v + c*vstride, writes hv + c*vstride, uses uprev + c*vstride, bn + c*sstride,
  // red_out + c*sstride and the scratch partial + c*kRedSlots; a column whose active[c] is 0
  // is skipped. ncols is the launch's gridDim.y (1 for a single vector).
  int64_t vstride = 0, sstride = 0;
  const int* __restrict__ active = nullptr;
  int ncols = 1;
  int dwv = 0, upv = 0;  // kernel choice (edg_sector_s::hxv_dw / hxv_up)
};

// Which pass of the Lanczos-fused step subtracts c * uprev. FP32: the down pass, as the start
// of its diagonal term (it runs at a fraction of HBM bandwidth, and the up pass, short of
// registers, then reads no third vector). FP64: the up pass, after all hops, which is the
// reference's order (w = Hv - b u_prev), so FP64 coefficients stay bit-exact.
template <typename T>
constexpr bool lz_sub_in_dw() { return sizeof(T) == 4; }

// Points a block-mode launch's arguments at this CTA's column; false when the column has
// stopped. A single-vector launch (gridDim.y == 1, active == nullptr) is left as it is.
template <typename T>
__device__ __forceinline__ bool select_column(HxvArgs<T>& a) {
  const int64_t c = blockIdx.y;
  if (a.active && !a.active[c]) return false;
  if (c) {
    a.v += c * a.vstride;
    a.hv += c * a.vstride;
    if (a.uprev) a.uprev += c * a.vstride;
    if (a.bn) a.bn += c * a.sstride;
    if (a.partial) a.partial += c * kRedSlots;
    if (a.red_out) a.red_out += c * a.sstride;
  }
  return true;
}

template <typename T>
__device__ __forceinline__ T fmaT(T a, T b, T c);
template <>
__device__ __forceinline__ float fmaT<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <>
__device__ __forceinline__ double fmaT<double>(double a, double b, double c) { return __fma_rn(a, b, c); }

// Row pass: one CTA per row idw (grid-stride), threads along iup. H_up gathers hit L1/L2
// (a row is DimUp*sizeof(T) bytes). FIRST: hv = diag*v + up-part; else hv += up-part.
template <typename T, bool FIRST>
__global__ void __launch_bounds__(256) k_up_rows(HxvArgs<T> a) {
  for (int64_t idw = blockIdx.x; idw < a.dimdw; idw += gridDim.x) {
    const T* __restrict__ vrow = a.v + idw * a.dimup;
    T* __restrict__ hrow = a.hv + idw * a.dimup;
    const uint32_t mdw = a.map_dw[idw];
    const T edw = a.e_dw[idw];
    for (int64_t iup = threadIdx.x; iup < a.dimup; iup += blockDim.x) {
      T acc;
      if (FIRST) {
        const T d = a.e_up[iup] + edw + a.U * T(__popc(a.map_up[iup] & mdw));
        acc = d * vrow[iup];
      } else {
        acc = hrow[iup];
      }
      const uint32_t k0 = a.off_up[iup], k1 = a.off_up[iup + 1];
      for (uint32_t k = k0; k < k1; ++k) acc = fmaT<T>(a.val_up[k], __ldg(vrow + a.src_up[k]), acc);
      hrow[iup] = acc;
    }
  }
}

// Row pass with the rows staged in shared memory. A CTA takes RT consecutive rows, stores
// them interleaved (S[jup] holds the RT values of column jup, one vector load per hop) and
// gathers H_up's sources from there instead of from L1, where random 4-byte reads cost a
// wavefront per distinct line. The table is SELL-32: the k-th entries of a warp's 32
// target columns are one coalesced 128-byte read, shared by the RT rows.
template <typename T, int RT>
struct VecT;
template <> struct VecT<float, 1> { using type = float; };
template <> struct VecT<float, 2> { using type = float2; };
template <> struct VecT<float, 4> { using type = float4; };
template <> struct VecT<double, 1> { using type = double; };
template <> struct VecT<double, 2> { using type = double2; };

template <typename T>
struct SellArgs {
  const uint32_t* __restrict__ ent;
  const uint32_t* __restrict__ off;
  const T* __restrict__ val;  // non-uniform tables only
  T h;                        // |value| with the sign of code 0 (uniform tables)
  bool v4 = false;            // a lane's slots stored four together (SpinBasis::sched_v4)
};

// acc[0..RT) += h * x[0..RT): packed FP32x2 FMAs where the pair shares h (Blackwell
// fma.rn.f32x2; each lane is an IEEE fma, identical to two scalar ones).
template <typename T, int RT>
struct Fma {
  static __device__ __forceinline__ void run(T h, const T* x, T* acc) {
#pragma unroll
    for (int r = 0; r < RT; ++r) acc[r] = fmaT<T>(h, x[r], acc[r]);
  }
};
__device__ __forceinline__ void ffma2(float h, const float* x, float* acc) {
  uint64_t d;
  const uint64_t uh = (uint64_t(__float_as_uint(h)) << 32) | __float_as_uint(h);
  const uint64_t ux = (uint64_t(__float_as_uint(x[1])) << 32) | __float_as_uint(x[0]);
  const uint64_t ua = (uint64_t(__float_as_uint(acc[1])) << 32) | __float_as_uint(acc[0]);
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(uh), "l"(ux), "l"(ua));
  acc[0] = __uint_as_float(uint32_t(d));
  acc[1] = __uint_as_float(uint32_t(d >> 32));
}
template <>
struct Fma<float, 2> {
  static __device__ __forceinline__ void run(float h, const float* x, float* acc) { ffma2(h, x, acc); }
};
template <>
struct Fma<float, 4> {
  static __device__ __forceinline__ void run(float h, const float* x, float* acc) {
    ffma2(h, x, acc);
    ffma2(h, x + 2, acc + 2);
  }
};

__device__ __forceinline__ float flip_sign(float h, uint32_t e) {
  return __uint_as_float(__float_as_uint(h) ^ (e & 0x80000000u));
}
__device__ __forceinline__ double flip_sign(double h, uint32_t e) {
  return __longlong_as_double(__double_as_longlong(h) ^ (static_cast<long long>(e & 0x80000000u) << 32));
}

// SELL entry: bit 31 = sign of the uniform value, bits 0..30 = source column (DimUp for
// padding: a zero slot after the staged rows, so padding needs no branch).
// ONE: one CTA per SM (the staged rows take more than half of shared memory); the 64
// registers per thread this allows carry the next batch of entries while the current one is
// applied.
// The FP64 Lanczos-fused form (LZ) with two CTAs per SM runs 768 threads per CTA: that
// leaves 40 registers per thread for reading uprev and the epilogue's FP64 state next to the
// batch of entries in flight. The FP32 form reads no uprev (its down pass subtracts it) and
// runs 1024 threads: 1.34 ms with uprev at 768 threads, against 2.56 ms with uprev at 1024,
// on the 4x4 half-filled sector; without uprev 1024 threads are the faster choice
// (FP32+refine E0 0.2427 -> 0.2365 s). One CTA per SM keeps 1024 threads.
template <typename T, bool LZ, bool ONE>
constexpr int up_threads() { return LZ && !ONE && !lz_sub_in_dw<T>() ? 768 : 1024; }

// E4: the table stores a lane's slots four together (sched_v4), so a batch of 8 entries is
// two 16-byte loads per lane instead of eight 4-byte ones (two CTAs per SM, uniform tables).
template <typename T, int RT, bool FIRST, bool UNIFORM, bool LZ, bool ONE, bool E4 = false>
__global__ void __launch_bounds__(up_threads<T, LZ, ONE>(), ONE ? 1 : 2) k_up_smem(HxvArgs<T> a, SellArgs<T> sl, int64_t nrowblk) {
  if (!select_column(a)) return;
  using V = typename VecT<T, RT>::type;
  extern __shared__ __align__(16) unsigned char smem_up[];
  V* S = reinterpret_cast<V*>(smem_up);
  const int64_t dimup = a.dimup;
  // Lanczos scalars 1/bn[j] and bn[j]/bn[j-1]: the epilogue reads them from shared memory,
  // so that they take no registers in the gather loop (the two-CTA FP32 form has 32)
  __shared__ double s_lz[2];
  double pa = 0.0, sc = 1.0;
  if (LZ) {
    sc = 1.0 / a.bn[a.jstep];
    if (threadIdx.x == 0) {
      s_lz[0] = sc;
      s_lz[1] = a.jstep > 0 ? a.bn[a.jstep] / a.bn[a.jstep - 1] : 0.0;
    }
  }
  const T hs = LZ ? T(double(sl.h) * sc) : sl.h;
  const double scn = UNIFORM ? 1.0 : sc;  // per-term scale of non-uniform values
  for (int zq = threadIdx.x; zq < kUpZeroSlots; zq += blockDim.x) {  // padding targets
    V z;
    T* zs = reinterpret_cast<T*>(&z);
#pragma unroll
    for (int r = 0; r < RT; ++r) zs[r] = T(0);
    S[dimup + zq] = z;
  }
  for (int64_t rb = blockIdx.x; rb < nrowblk; rb += gridDim.x) {
    const int64_t r0 = rb * RT;
    for (int64_t j = threadIdx.x; j < dimup; j += blockDim.x) {
      V x;
      T* xs = reinterpret_cast<T*>(&x);
#pragma unroll
      for (int r = 0; r < RT; ++r) xs[r] = (r0 + r < a.dimdw) ? a.v[(r0 + r) * dimup + j] : T(0);
      S[j] = x;
    }
    __syncthreads();
    for (int64_t iup = threadIdx.x; iup < dimup; iup += blockDim.x) {
      T acc[RT];
      const int64_t slice = iup >> 5;
      const int lane = int(iup & 31);
      const uint32_t o = sl.off[slice], o1 = sl.off[slice + 1];
      if (FIRST) {
        const V xc = S[iup];
        const T* xs = reinterpret_cast<const T*>(&xc);
        const T eu = a.e_up[iup];
        const uint32_t mu = a.map_up[iup];
#pragma unroll
        for (int r = 0; r < RT; ++r) {
          const int64_t row = r0 + r < a.dimdw ? r0 + r : a.dimdw - 1;
          acc[r] = (eu + a.e_dw[row] + a.U * T(__popc(mu & a.map_dw[row]))) * xs[r];
        }
      } else {
#pragma unroll
        for (int r = 0; r < RT; ++r) acc[r] = (r0 + r < a.dimdw) ? a.hv[(r0 + r) * dimup + iup] : T(0);
      }
      // entries in batches of independent loads (slice widths are whole batches; padding
      // entries read a zero column)
      constexpr int kUpBatch = kSellBatch;
      if (ONE && UNIFORM) {
        uint32_t e[kUpBatch];
        uint32_t p0 = o + lane;
        if (p0 < o1) {
#pragma unroll
          for (int u = 0; u < kUpBatch; ++u) e[u] = __ldg(sl.ent + p0 + 32u * u);
        }
        for (; p0 < o1; p0 += 32 * kUpBatch) {
          uint32_t en[kUpBatch];
          const uint32_t pn = p0 + 32 * kUpBatch;
          if (pn < o1) {
#pragma unroll
            for (int u = 0; u < kUpBatch; ++u) en[u] = __ldg(sl.ent + pn + 32u * u);
          }
#pragma unroll
          for (int u = 0; u < kUpBatch; ++u) {
            const V x = S[e[u] & 0x7fffffffu];
            Fma<T, RT>::run(flip_sign(hs, e[u]), reinterpret_cast<const T*>(&x), acc);
          }
#pragma unroll
          for (int u = 0; u < kUpBatch; ++u) e[u] = en[u];
        }
      } else if (E4 && UNIFORM) {
        static_assert(!E4 || kUpBatch == 8, "two 16-byte entry loads per batch");
        const uint4* __restrict__ ent4 = reinterpret_cast<const uint4*>(sl.ent);
        for (uint32_t q = o >> 2; q < (o1 >> 2); q += 8 * kUpBatch) {
          const uint4 x0 = __ldg(ent4 + q + lane), x1 = __ldg(ent4 + q + 32 + lane);
          const uint32_t e[kUpBatch] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
#pragma unroll
          for (int u = 0; u < kUpBatch; ++u) {
            const V x = S[e[u] & 0x7fffffffu];
            Fma<T, RT>::run(flip_sign(hs, e[u]), reinterpret_cast<const T*>(&x), acc);
          }
        }
      } else {
        for (uint32_t p0 = o + lane; p0 < o1; p0 += 32 * kUpBatch) {
          uint32_t e[kUpBatch];
          T hv_[kUpBatch];
#pragma unroll
          for (int u = 0; u < kUpBatch; ++u) {
            e[u] = __ldg(sl.ent + p0 + 32u * u);
            if (!UNIFORM) hv_[u] = __ldg(sl.val + p0 + 32u * u);
          }
#pragma unroll
          for (int u = 0; u < kUpBatch; ++u) {
            const T h = UNIFORM ? flip_sign(hs, e[u]) : (LZ ? T(double(hv_[u]) * scn) : hv_[u]);
            const V x = S[e[u] & 0x7fffffffu];
            Fma<T, RT>::run(h, reinterpret_cast<const T*>(&x), acc);
          }
        }
      }
      if (LZ) {
        // w = Hv - c * uprev (FP64 here; FP32: the down pass began from -c * uprev);
        // partial <v, w> with v = sc * u (staged in S)
        const volatile double* lz = s_lz;
        const double sc = lz[0], cc = lz_sub_in_dw<T>() ? 0.0 : lz[1];
        const V xc = S[iup];
        const T* xs = reinterpret_cast<const T*>(&xc);
#pragma unroll
        for (int r = 0; r < RT; ++r)
          if (r0 + r < a.dimdw) {
            const int64_t e = (r0 + r) * dimup + iup;
            const T wt = lz_sub_in_dw<T>() ? acc[r] : T(double(acc[r]) - cc * double(a.uprev[e]));
            pa = __fma_rn(double(xs[r]) * sc, double(wt), pa);
            __stcs(a.hv + e, wt);
          }
      } else {
#pragma unroll
        for (int r = 0; r < RT; ++r)
          if (r0 + r < a.dimdw) __stcs(a.hv + (r0 + r) * dimup + iup, acc[r]);
      }
    }
    __syncthreads();
  }
  if (LZ) {  // block partial of <v, w>, fixed order
    __shared__ double s_red[32];
    for (int o = 16; o > 0; o >>= 1) pa += __shfl_down_sync(0xffffffffu, pa, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = pa;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int q = 0; q < int(blockDim.x >> 5); ++q) t += s_red[q];
      a.partial[blockIdx.x] = t;
    }
    finish_in_last_block(a.partial, gridDim.x, a.red_out, 0);
  }
}

// FP32 up pass over the Kronecker schedule (SpinBasis::kron_*). The CTA stages RT rows
// interleaved in shared memory as k_up_smem does; thread t owns one low part (lidx) of one
// group and a run of consecutive blocks of that group, the same for every row block of the
// launch. Its LL hops are (column offset, sign) pairs loaded once into registers; the HH hops
// of a block are one short list shared by every lane on that block (the same cached words);
// only the cross hops read a per-column table, lane-interleaved per warp and step. Lanes of a
// warp hold consecutive lidx, so the reads and writes of Hv stay coalesced within a block.
struct KronArgs {
  const int4* __restrict__ thr;
  const int32_t* __restrict__ bcol;
  const uint32_t* __restrict__ hoff;
  const int32_t* __restrict__ hent;
  const int32_t* __restrict__ lent;
  const uint32_t* __restrict__ xent;
  const uint32_t* __restrict__ xoff;
  const uint32_t* __restrict__ xwid;
  int nthr, lmax;
  int nkrow, nhent;  // block rows, HH entries (staged in shared memory)
  float h;
};

constexpr int kKronX = 8;  // cross entries of a step loaded together into registers

// h with its sign flipped when bit 0 of e is set
__device__ __forceinline__ float flip_bit0(float h, uint32_t e) { return __uint_as_float(__float_as_uint(h) ^ (e << 31)); }

template <int RT, bool LZ, bool ONE>
__global__ void __launch_bounds__(kKronThreads, ONE ? 1 : 2) k_up_kron(HxvArgs<float> a, KronArgs q, int64_t nrowblk) {
  if (!select_column(a)) return;
  using V = typename VecT<float, RT>::type;
  extern __shared__ __align__(16) unsigned char smem_kr[];
  V* S = reinterpret_cast<V*>(smem_kr);
  const int64_t dimup = a.dimup;
  __shared__ double s_lz[2];  // 1/bn[j], bn[j]/bn[j-1]: read by the epilogue only
  double pa = 0.0;
  float hs = q.h;
  if (LZ) {
    const double sc = 1.0 / a.bn[a.jstep];
    if (threadIdx.x == 0) {
      s_lz[0] = sc;
      s_lz[1] = a.jstep > 0 ? a.bn[a.jstep] / a.bn[a.jstep - 1] : 0.0;
    }
    hs = float(double(q.h) * sc);
  }
  for (int zq = threadIdx.x; zq < kUpZeroSlots; zq += blockDim.x) {  // padding targets
    V z;
    float* zs = reinterpret_cast<float*>(&z);
#pragma unroll
    for (int r = 0; r < RT; ++r) zs[r] = 0.f;
    S[dimup + zq] = z;
  }
  // the per-block tables (first column, HH range, HH entries) sit after the staged rows:
  // every step reads them, and from L2 their loads were a dependent chain ahead of each gather
  int32_t* s_bcol = reinterpret_cast<int32_t*>(S + dimup + kUpZeroSlots);
  uint32_t* s_hoff = reinterpret_cast<uint32_t*>(s_bcol + q.nkrow);
  int32_t* s_hent = reinterpret_cast<int32_t*>(s_hoff + q.nkrow + 1);
  for (int i = threadIdx.x; i < q.nkrow; i += blockDim.x) s_bcol[i] = q.bcol[i];
  for (int i = threadIdx.x; i <= q.nkrow; i += blockDim.x) s_hoff[i] = q.hoff[i];
  for (int i = threadIdx.x; i < q.nhent; i += blockDim.x) s_hent[i] = q.hent[i];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int4 me = t < q.nthr ? q.thr[t] : make_int4(0, 0, 0, 0);
  const int krow0 = me.x, len = me.y, lidx = me.w;
  // this thread's LL slots, held in registers for the whole launch (the empty asm keeps
  // the compiler from reloading them from the table inside the loops)
  // (column offsets as 16-bit halves, two per register)
  uint32_t lld[kKronLL / 2];
  uint32_t lsg = 0, lval = 0;
#pragma unroll
  for (int j = 0; j < kKronLL; ++j) {
    const int32_t e = q.lent[t * kKronLL + j];
    const uint32_t d16 = uint32_t(e >> 2) & 0xffffu;
    if (j & 1) lld[j >> 1] |= d16 << 16;
    else lld[j >> 1] = d16;
    lval |= uint32_t((e >> 1) & 1) << j;
    lsg |= uint32_t(e & 1) << j;
  }
#pragma unroll
  for (int j = 0; j < kKronLL / 2; ++j) asm volatile("" : "+r"(lld[j]));
  asm volatile("" : "+r"(lval), "+r"(lsg));
  int wlen = len;  // steps of the warp: the longest run among its lanes
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) wlen = max(wlen, __shfl_xor_sync(0xffffffffu, wlen, o));
  const uint32_t xbase = q.xoff[warp];
  const uint32_t* __restrict__ xw = q.xwid + warp * q.lmax;
  for (int64_t rb = blockIdx.x; rb < nrowblk; rb += gridDim.x) {
    const int64_t r0 = rb * RT;
    for (int64_t j = threadIdx.x; j < dimup; j += blockDim.x) {
      V x;
      float* xs = reinterpret_cast<float*>(&x);
#pragma unroll
      for (int r = 0; r < RT; ++r) xs[r] = (r0 + r < a.dimdw) ? a.v[(r0 + r) * dimup + j] : 0.f;
      S[j] = x;
    }
    __syncthreads();
    uint32_t xs = xbase;
    for (int k = 0; k < wlen; ++k) {
      const int wd = int(xw[k]);
      if (k < len) {
        // the step's loads from HBM/L2 first, all in flight together: its cross entries and
        // the down pass's partial sums; the shared-memory terms then cover their latency
        uint32_t xe[kKronX];
#pragma unroll
        for (int j = 0; j < kKronX; ++j) xe[j] = j < wd ? __ldg(q.xent + size_t(xs + j) * 32 + lane) : 0u;
        const int kr = krow0 + k;
        const int c = s_bcol[kr] + lidx;
        float acc[RT];
#pragma unroll
        for (int r = 0; r < RT; ++r) acc[r] = (r0 + r < a.dimdw) ? a.hv[(r0 + r) * dimup + c] : 0.f;
#pragma unroll
        for (int j = 0; j < kKronLL; ++j) {
          if ((lval >> j) & 1u) {
            const int d = (j & 1) ? int(lld[j >> 1]) >> 16 : int(int16_t(lld[j >> 1] & 0xffffu));
            const V x = S[c + d];
            Fma<float, RT>::run(flip_bit0(hs, lsg >> j), reinterpret_cast<const float*>(&x), acc);
          }
        }
        const uint32_t h1 = s_hoff[kr + 1];
        for (uint32_t p = s_hoff[kr]; p < h1; ++p) {
          const int32_t e = s_hent[p];
          const V x = S[c + (e >> 1)];
          Fma<float, RT>::run(flip_bit0(hs, uint32_t(e)), reinterpret_cast<const float*>(&x), acc);
        }
#pragma unroll
        for (int j = 0; j < kKronX; ++j) {
          if (j < wd) {
            const V x = S[xe[j] & 0x7fffffffu];
            Fma<float, RT>::run(flip_sign(hs, xe[j]), reinterpret_cast<const float*>(&x), acc);
          }
        }
        for (int j = kKronX; j < wd; ++j) {
          const uint32_t e = __ldg(q.xent + size_t(xs + j) * 32 + lane);
          const V x = S[e & 0x7fffffffu];
          Fma<float, RT>::run(flip_sign(hs, e), reinterpret_cast<const float*>(&x), acc);
        }
        if (LZ) {
          const volatile double* lz = s_lz;
          const double sc = lz[0];
          const V xc = S[c];
          const float* xv = reinterpret_cast<const float*>(&xc);
#pragma unroll
          for (int r = 0; r < RT; ++r)
            if (r0 + r < a.dimdw) {
              const int64_t e = (r0 + r) * dimup + c;
              const float wt = acc[r];  // c * uprev: subtracted by the down pass
              pa = __fma_rn(double(xv[r]) * sc, double(wt), pa);
              __stcs(a.hv + e, wt);
            }
        } else {
#pragma unroll
          for (int r = 0; r < RT; ++r)
            if (r0 + r < a.dimdw) __stcs(a.hv + (r0 + r) * dimup + c, acc[r]);
        }
      }
      xs += uint32_t(wd);
    }
    __syncthreads();
  }
  if (LZ) {  // block partial of <v, w>, fixed order
    __shared__ double s_red[32];
    for (int o = 16; o > 0; o >>= 1) pa += __shfl_down_sync(0xffffffffu, pa, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = pa;
    __syncthreads();
    if (threadIdx.x == 0) {
      double tt = 0.0;
      for (int w = 0; w < int(blockDim.x >> 5); ++w) tt += s_red[w];
      a.partial[blockIdx.x] = tt;
    }
    finish_in_last_block(a.partial, gridDim.x, a.red_out, 0);
  }
}

// FP32 up pass over the packed 16-bit schedule (SpinBasis::p16_*). A CTA stages RT rows
// interleaved in shared memory as in k_up_smem and, when NEG, their negated copy at slot
// offset negoff, so that every term is one shared load and one FMA with the uniform hopping
// value: the entry is the slot itself (src, or negoff + src for a negative term). Without NEG
// the entry carries the sign in bit 15 and the value's sign bit is flipped per term. Entries
// come two per 32-bit word; a warp walks its slice in batches of four words (eight terms)
// with warp-uniform bounds (all 32 lanes of a warp share one slice). Slot counts are rounded
// to 2 instead of 8, and the slot order is the bank-conflict-free schedule of k_up_smem, so
// each half-warp's shared loads hit 16 distinct 8-byte bank pairs.
struct P16Args {
  const uint32_t* __restrict__ ent;
  const uint32_t* __restrict__ off;
  float h;
  uint32_t negoff;
};

__device__ __forceinline__ void ffma2_acc(uint64_t& acc, uint64_t h2, uint64_t x) {
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(h2), "l"(x));
}

template <bool NEG, bool ONE, bool LZ>
__global__ void __launch_bounds__(1024, ONE ? 1 : 2) k_up_p16(HxvArgs<float> a, P16Args q, int64_t nrowblk) {
  if (!select_column(a)) return;
  extern __shared__ __align__(16) unsigned char smem_p16[];
  float2* S = reinterpret_cast<float2*>(smem_p16);
  const uint64_t* S64 = reinterpret_cast<const uint64_t*>(smem_p16);
  const int64_t dimup = a.dimup;
  double sc = 1.0, pa = 0.0;
  if (LZ) sc = 1.0 / a.bn[a.jstep];
  const float hs = LZ ? float(double(q.h) * sc) : q.h;
  const uint64_t hh = (uint64_t(__float_as_uint(hs)) << 32) | __float_as_uint(hs);
  for (int zq = threadIdx.x; zq < kUpZeroSlots; zq += blockDim.x) {  // padding targets
    S[dimup + zq] = make_float2(0.f, 0.f);
    if (NEG) S[q.negoff + dimup + zq] = make_float2(0.f, 0.f);
  }
  for (int64_t rb = blockIdx.x; rb < nrowblk; rb += gridDim.x) {
    const int64_t r0 = rb * 2;
    const bool two = r0 + 1 < a.dimdw;
    const float* __restrict__ v0 = a.v + r0 * dimup;
    const float* __restrict__ v1 = two ? v0 + dimup : v0;
    for (int64_t j = threadIdx.x; j < dimup; j += blockDim.x) {
      const float2 x = make_float2(v0[j], two ? v1[j] : 0.f);
      S[j] = x;
      if (NEG) S[q.negoff + j] = make_float2(-x.x, -x.y);
    }
    __syncthreads();
    float* __restrict__ h0 = a.hv + r0 * dimup;
    float* __restrict__ h1 = h0 + dimup;
    for (int64_t iup = threadIdx.x; iup < dimup; iup += blockDim.x) {
      const uint32_t o1 = q.off[(iup >> 5) + 1];
      uint32_t p = q.off[iup >> 5] + uint32_t(iup & 31);
      uint64_t acc = (uint64_t(__float_as_uint(two ? h1[iup] : 0.f)) << 32) | __float_as_uint(h0[iup]);
      for (; p < o1; p += 32 * 4) {
        uint32_t w[4];  // the table carries 128 words of padding after its last slice
#pragma unroll
        for (int u = 0; u < 4; ++u) w[u] = __ldg(q.ent + p + 32u * u);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (p + 32u * u < o1) {
#pragma unroll
            for (int half = 0; half < 2; ++half) {
              const uint32_t e = half ? (w[u] >> 16) : (w[u] & 0xffffu);
              if (NEG) {
                ffma2_acc(acc, hh, S64[e]);
              } else {
                const uint64_t sb = uint64_t((e & 0x8000u) << 16);  // the term's sign, both halves
                ffma2_acc(acc, hh ^ (sb | (sb << 32)), S64[e & 0x7fffu]);
              }
            }
          }
        }
      }
      const float acc0 = __uint_as_float(uint32_t(acc)), acc1 = __uint_as_float(uint32_t(acc >> 32));
      if (LZ) {
        const float2 xc = S[iup];
        const float w0 = acc0;  // c * uprev: subtracted by the down pass
        pa = __fma_rn(double(xc.x) * sc, double(w0), pa);
        __stcs(h0 + iup, w0);
        if (two) {
          const float w1 = acc1;
          pa = __fma_rn(double(xc.y) * sc, double(w1), pa);
          __stcs(h1 + iup, w1);
        }
      } else {
        __stcs(h0 + iup, acc0);
        if (two) __stcs(h1 + iup, acc1);
      }
    }
    __syncthreads();
  }
  if (LZ) {  // block partial of <v, w>, fixed order, then the fused finish
    __shared__ double s_red[32];
    for (int o = 16; o > 0; o >>= 1) pa += __shfl_down_sync(0xffffffffu, pa, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = pa;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < int(blockDim.x >> 5); ++w) t += s_red[w];
      a.partial[blockIdx.x] = t;
    }
    finish_in_last_block(a.partial, gridDim.x, a.red_out, 0);
  }
}

// Up pass for rows too long to stage whole (FP64 rows above 227 KB): one CTA per row (grid-
// stride) stages the row one column part at a time and applies that part's entries; between
// parts the running sums of the row live in hv (the CTA's own row, just written, so L2).
// Each target column is always handled by the same thread, and the parts' entries come in
// ascending source order, so the sums are those of the whole-row kernels.
template <typename T>
struct SplitArgs {
  const uint32_t* __restrict__ ent;
  const uint32_t* __restrict__ off;
  const T* __restrict__ val;  // non-uniform tables only
  T h;
  int parts;
  int64_t nsl;
  int64_t col[SpinBasis::kMaxSplit + 1];
};

template <typename T, bool FIRST, bool UNIFORM>
__global__ void __launch_bounds__(1024, 1) k_up_split(HxvArgs<T> a, SplitArgs<T> sp) {
  extern __shared__ __align__(16) unsigned char smem_split[];
  T* S = reinterpret_cast<T*>(smem_split);
  const int64_t dimup = a.dimup;
  for (int64_t idw = blockIdx.x; idw < a.dimdw; idw += gridDim.x) {
    const T* __restrict__ vrow = a.v + idw * dimup;
    T* __restrict__ hrow = a.hv + idw * dimup;
    for (int p = 0; p < sp.parts; ++p) {
      const int64_t c0 = sp.col[p], w = sp.col[p + 1] - c0;
      for (int64_t j = threadIdx.x; j < w + kUpZeroSlots; j += blockDim.x) S[j] = j < w ? vrow[c0 + j] : T(0);
      __syncthreads();
      const uint32_t* __restrict__ offp = sp.off + int64_t(p) * (sp.nsl + 1);
      for (int64_t iup = threadIdx.x; iup < dimup; iup += blockDim.x) {
        T acc;
        if (FIRST && p == 0) {
          const T d = a.e_up[iup] + a.e_dw[idw] + a.U * T(__popc(a.map_up[iup] & a.map_dw[idw]));
          acc = d * vrow[iup];
        } else {
          acc = hrow[iup];
        }
        const uint32_t o = offp[iup >> 5], o1 = offp[(iup >> 5) + 1];
        for (uint32_t q = o + uint32_t(iup & 31); q < o1; q += 32 * kSellBatch) {
          uint32_t e[kSellBatch];
          T hv_[kSellBatch];
#pragma unroll
          for (int u = 0; u < kSellBatch; ++u) {
            e[u] = __ldg(sp.ent + q + 32u * u);
            if (!UNIFORM) hv_[u] = __ldg(sp.val + q + 32u * u);
          }
#pragma unroll
          for (int u = 0; u < kSellBatch; ++u) {
            const T h = UNIFORM ? flip_sign(sp.h, e[u]) : hv_[u];
            acc = fmaT<T>(h, S[e[u] & 0x7fffffffu], acc);
          }
        }
        hrow[iup] = acc;
      }
      __syncthreads();
    }
  }
}

// Down-spin pass, one warp per (row idw', segment of 32*VEC consecutive iup). The row's hop
// list is uniform across the warp: lanes load up to 32 (source, value) pairs in one
// coalesced read and hand them out with shuffles; the source rows are then read as
// independent VEC-wide loads, unrolled so several are in flight per thread. Segments are
// visited slab-major (all rows of a 32*VEC-column slab before the next slab) so the slab
// (DimDw * 32*VEC*sizeof(T) bytes) stays in L2 while each of its rows is read ~hops times.
template <typename T, int VEC>
struct VecLd;
template <typename T>
struct VecLd<T, 1> {
  static __device__ __forceinline__ void load(const T* p, T* x) { x[0] = __ldg(p); }
};
template <>
struct VecLd<float, 2> {
  static __device__ __forceinline__ void load(const float* p, float* x) {
    const float2 t = __ldg(reinterpret_cast<const float2*>(p));
    x[0] = t.x;
    x[1] = t.y;
  }
};
template <>
struct VecLd<double, 2> {
  static __device__ __forceinline__ void load(const double* p, double* x) {
    const double2 t = __ldg(reinterpret_cast<const double2*>(p));
    x[0] = t.x;
    x[1] = t.y;
  }
};

template <typename T, int VEC, bool FIRST>
__global__ void __launch_bounds__(256) k_dw_seg(HxvArgs<T> a, int64_t ntiles) {
  const int lane = threadIdx.x & 31;
  const int64_t wpb = blockDim.x >> 5;
  const int64_t dimup = a.dimup, dimdw = a.dimdw;
  for (int64_t tile = blockIdx.x * wpb + (threadIdx.x >> 5); tile < ntiles; tile += int64_t(gridDim.x) * wpb) {
    const int64_t slab = tile / dimdw, idw = tile - slab * dimdw;
    const int64_t col = slab * (32 * VEC) + int64_t(lane) * VEC;
    const bool active = col < dimup;
    const int64_t e0 = idw * dimup + col;
    T acc[VEC];
    if (active) {
      if (FIRST) {
        const T edw = a.e_dw[idw];
        const uint32_t mdw = a.map_dw[idw];
        T x[VEC];
        VecLd<T, VEC>::load(a.v + e0, x);
#pragma unroll
        for (int q = 0; q < VEC; ++q)
          acc[q] = (a.e_up[col + q] + edw + a.U * T(__popc(a.map_up[col + q] & mdw))) * x[q];
      } else {
#pragma unroll
        for (int q = 0; q < VEC; ++q) acc[q] = a.hv[e0 + q];
      }
    }
    const uint32_t k0 = a.off_dw[idw], k1 = a.off_dw[idw + 1];
    for (uint32_t base = k0; base < k1; base += 32) {
      const int cnt = int(k1 - base < 32u ? k1 - base : 32u);
      const uint32_t my_src = lane < cnt ? a.src_dw[base + lane] : 0u;
      const T my_val = lane < cnt ? a.val_dw[base + lane] : T(0);
      constexpr int kU = 8;
      for (int k = 0; k < cnt; k += kU) {
        T x[kU][VEC];
        T h[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          const int kk = k + u < cnt ? k + u : k;  // out-of-range slots repeat a valid row
          const uint32_t sr = __shfl_sync(0xffffffffu, my_src, kk);
          h[u] = __shfl_sync(0xffffffffu, my_val, kk);
          if (k + u >= cnt) h[u] = T(0);
          if (active) VecLd<T, VEC>::load(a.v + int64_t(sr) * dimup + col, x[u]);
        }
        if (active) {
#pragma unroll
          for (int u = 0; u < kU; ++u) {
            if (k + u < cnt) {
#pragma unroll
              for (int q = 0; q < VEC; ++q) acc[q] = fmaT<T>(h[u], x[u][q], acc[q]);
            }
          }
        }
      }
    }
    if (active) {
#pragma unroll
      for (int q = 0; q < VEC; ++q) __stcs(a.hv + e0 + q, acc[q]);  // streamed: read back only by the next pass
    }
  }
}

// Single-pass stored-form H x v for sectors whose vectors sit in L2 (D up to a few million):
// one warp per 32 consecutive columns of one row idw. The down hops of the row are the same
// for the 32 lanes (one broadcast entry each, a coalesced read of the source row's segment),
// the up hops are each lane's own CSR list (gathers inside the row, from L1/L2). Terms in the
// stored form's order, diag, DW, UP, sources ascending, so FP64 results equal the two-pass
// kernels' and the reference's bit for bit on integer-valued models. LZ: the Lanczos-fused
// step of k_up_smem (v = u / bn[j] through scaled matrix elements, w = Hv - c u_prev and the
// block partials of <v, w>), in the same single pass.
template <typename T, bool LZ>
__global__ void __launch_bounds__(256) k_hxv_fused(HxvArgs<T> a, int64_t ntiles) {
  if (!select_column(a)) return;
  const int lane = threadIdx.x & 31;
  const int64_t wpb = blockDim.x >> 5;
  const int64_t dimup = a.dimup;
  const int64_t nct = (dimup + 31) >> 5;  // column tiles per row
  double sc = 1.0, cc = 0.0, pa = 0.0;
  if (LZ) {
    sc = 1.0 / a.bn[a.jstep];
    cc = a.jstep > 0 ? a.bn[a.jstep] / a.bn[a.jstep - 1] : 0.0;
  }
  for (int64_t tile = blockIdx.x * wpb + (threadIdx.x >> 5); tile < a.dimdw * nct;
       tile += int64_t(gridDim.x) * wpb) {
    const int64_t idw = tile / nct;
    const int64_t iup = (tile - idw * nct) * 32 + lane;
    const bool act = iup < dimup;
    const int64_t cup = act ? iup : dimup - 1;  // inactive lanes read a valid column, store nothing
    const T* __restrict__ vrow = a.v + idw * dimup;
    const T d = a.e_up[cup] + a.e_dw[idw] + a.U * T(__popc(a.map_up[cup] & a.map_dw[idw]));
    T acc = (LZ ? T(double(d) * sc) : d) * vrow[cup];
    // sources in batches of 4 loads issued together, terms added in list order
    constexpr int kB = 4;
    const uint32_t k0 = a.off_dw[idw], k1 = a.off_dw[idw + 1];
    for (uint32_t k = k0; k < k1; k += kB) {
      T x[kB], h[kB];
#pragma unroll
      for (int u = 0; u < kB; ++u) {
        const uint32_t kk = k + u < k1 ? k + u : k;
        h[u] = LZ ? T(double(a.val_dw[kk]) * sc) : a.val_dw[kk];
        x[u] = a.v[int64_t(a.src_dw[kk]) * dimup + cup];
      }
#pragma unroll
      for (int u = 0; u < kB; ++u)
        if (k + u < k1) acc = fmaT<T>(h[u], x[u], acc);
    }
    const uint32_t u0 = a.off_up[cup], u1 = a.off_up[cup + 1];
    for (uint32_t k = u0; k < u1; k += kB) {
      T x[kB], h[kB];
#pragma unroll
      for (int u = 0; u < kB; ++u) {
        const uint32_t kk = k + u < u1 ? k + u : k;
        h[u] = LZ ? T(double(a.val_up[kk]) * sc) : a.val_up[kk];
        x[u] = __ldg(vrow + a.src_up[kk]);
      }
#pragma unroll
      for (int u = 0; u < kB; ++u)
        if (k + u < u1) acc = fmaT<T>(h[u], x[u], acc);
    }
    if (act) {
      const int64_t e = idw * dimup + iup;
      if (LZ) {
        const T wt = T(double(acc) - cc * double(a.uprev[e]));
        pa = __fma_rn(double(vrow[iup]) * sc, double(wt), pa);
        __stcs(a.hv + e, wt);
      } else {
        __stcs(a.hv + e, acc);
      }
    }
  }
  if (LZ) {  // block partial of <v, w>, fixed order
    __shared__ double s_red[8];
    for (int o = 16; o > 0; o >>= 1) pa += __shfl_down_sync(0xffffffffu, pa, o);
    if (lane == 0) s_red[threadIdx.x >> 5] = pa;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < int(wpb); ++w) t += s_red[w];
      a.partial[blockIdx.x] = t;
    }
    finish_in_last_block(a.partial, gridDim.x, a.red_out, 0);
  }
}

// Down-spin pass, balanced persistent form. CTA g owns the rows of group g (rows grouped on
// the host so every group carries the same total number of hops); their hop lists sit in
// shared memory. All CTAs sweep the column slabs (32*VEC columns) in the same order; inside
// a CTA the warps take the group's rows from a shared counter, and a CTA barrier closes
// each slab. Equal work per CTA keeps the whole grid within a few slabs of each other, so
// the slab being combined (DimDw rows x 32*VEC columns) stays in L2 while each of its rows
// is read once per hop; no global load of the hop list sits in the inner loop.
constexpr int kDwHops = 32;  // hop-list capacity per row held in shared memory

template <typename T, int VEC, int NSEG, int KU, bool FIRST, bool SCALED>
__global__ void __launch_bounds__(256, 4) k_dw_grp(HxvArgs<T> a, const uint32_t* __restrict__ goff,
                                                const uint32_t* __restrict__ grows, int64_t nslab) {
  if (!select_column(a)) return;
  extern __shared__ __align__(16) unsigned char smem_dw[];
  // the Lanczos scale 1/bn[j] (SCALED): folded into the hop values staged below, and read
  // from shared memory where the diagonal is formed, so that it holds no registers in the
  // slab loop (the FP64 form spilled with it)
  __shared__ double s_sc, s_cc;
  const double sc = SCALED ? 1.0 / a.bn[a.jstep] : 1.0;
  if (SCALED && threadIdx.x == 0) {
    s_sc = sc;
    s_cc = a.jstep > 0 ? a.bn[a.jstep] / a.bn[a.jstep - 1] : 0.0;
  }
  constexpr bool SUB = SCALED && lz_sub_in_dw<T>();  // this pass starts from -c * uprev
  __shared__ int s_ctr;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t gr0 = goff[blockIdx.x];
  const int nr = int(goff[blockIdx.x + 1] - gr0);
  T* s_val = reinterpret_cast<T*>(smem_dw);            // [nr][kDwHops]
  T* s_edw = s_val + size_t(nr) * kDwHops;              // [nr]
  uint32_t* s_src = reinterpret_cast<uint32_t*>(s_edw + nr);  // [nr][kDwHops]
  uint32_t* s_row = s_src + size_t(nr) * kDwHops;       // [nr]
  uint32_t* s_mdw = s_row + nr;                         // [nr]
  int* s_cnt = reinterpret_cast<int*>(s_mdw + nr);      // [nr]
  for (int rr = wib; rr < nr; rr += nw) {
    const uint32_t row = grows[gr0 + rr];
    const uint32_t k0 = a.off_dw[row];
    const int cnt = int(a.off_dw[row + 1] - k0);
    if (lane < cnt) {
      s_src[rr * kDwHops + lane] = a.src_dw[k0 + lane];
      s_val[rr * kDwHops + lane] = SCALED ? T(double(a.val_dw[k0 + lane]) * sc) : a.val_dw[k0 + lane];
    }
    if (lane == 0) {
      s_row[rr] = row;
      s_cnt[rr] = cnt;
      s_edw[rr] = a.e_dw[row];
      s_mdw[rr] = a.map_dw[row];
    }
  }
  const int64_t dimup = a.dimup;
  constexpr int SEGW = 32 * VEC;  // columns per warp-wide segment
  for (int64_t slab = 0; slab < nslab; ++slab) {
    if (threadIdx.x == 0) s_ctr = 0;
    __syncthreads();
    const int64_t col0 = slab * (SEGW * NSEG) + int64_t(lane) * VEC;
    bool act[NSEG];
#pragma unroll
    for (int g = 0; g < NSEG; ++g) act[g] = col0 + g * SEGW < dimup;
    for (;;) {
      int rr = 0;
      if (lane == 0) rr = atomicAdd(&s_ctr, 1);
      rr = __shfl_sync(0xffffffffu, rr, 0);
      if (rr >= nr) break;
      const int64_t idw = s_row[rr];
      const T* __restrict__ vrow0 = a.v + col0;   // + src*dimup per hop
      const int64_t e0 = idw * dimup + col0;
      const int cnt = s_cnt[rr];
      const uint32_t* hs = s_src + rr * kDwHops;
      const T* hvv = s_val + rr * kDwHops;
      T acc[NSEG][VEC];
#pragma unroll
      for (int g = 0; g < NSEG; ++g) {
        if (!act[g]) continue;
        const int64_t c = col0 + g * SEGW;
        if (FIRST) {
          const T edw = s_edw[rr];
          const uint32_t mdw = s_mdw[rr];
          T x[VEC], up[VEC];
          VecLd<T, VEC>::load(a.v + e0 + g * SEGW, x);
          if (SUB) VecLd<T, VEC>::load(a.uprev + e0 + g * SEGW, up);
          const double scl = SCALED ? *static_cast<volatile double*>(&s_sc) : 1.0;
#pragma unroll
          for (int r = 0; r < VEC; ++r) {
            const T d = a.e_up[c + r] + edw + a.U * T(__popc(a.map_up[c + r] & mdw));
            acc[g][r] = (SCALED ? T(double(d) * scl) : d) * x[r];
          }
          if (SUB) {
            const T ccn = T(-*static_cast<volatile double*>(&s_cc));
#pragma unroll
            for (int r = 0; r < VEC; ++r) acc[g][r] = fmaT<T>(ccn, up[r], acc[g][r]);
          }
        } else {
#pragma unroll
          for (int r = 0; r < VEC; ++r) acc[g][r] = a.hv[e0 + g * SEGW + r];
        }
      }
      for (int k = 0; k < cnt; k += KU) {
        T x[KU][NSEG][VEC];
#pragma unroll
        for (int u = 0; u < KU; ++u) {
          const int kk = k + u < cnt ? k + u : k;
          const T* __restrict__ src = vrow0 + int64_t(hs[kk]) * dimup;
#pragma unroll
          for (int g = 0; g < NSEG; ++g)
            if (act[g]) VecLd<T, VEC>::load(src + g * SEGW, x[u][g]);
        }
#pragma unroll
        for (int u = 0; u < KU; ++u) {
          if (k + u < cnt) {
            const T h = hvv[k + u];
#pragma unroll
            for (int g = 0; g < NSEG; ++g)
              if (act[g]) Fma<T, VEC>::run(h, x[u][g], acc[g]);
          }
        }
      }
#pragma unroll
      for (int g = 0; g < NSEG; ++g)
        if (act[g]) {
#pragma unroll
          for (int r = 0; r < VEC; ++r) __stcs(a.hv + e0 + g * SEGW + r, acc[g][r]);
        }
    }
    __syncthreads();
  }
}

// Down-spin pass over contiguous row blocks. CTA g owns the rows of block g (consecutive
// ranks, blocks balanced by hop count) and sweeps the column slabs (32*VEC*NSEG columns) in
// the order of k_dw_grp. For each slab it first stages its own rows' slab segments in shared
// memory; a hop whose source row lies in the block (about a third of them on square
// lattices: hops among the low-order sites keep the high-order part of the bitstring, hence
// the rank range) reads the source there, every other hop reads it from L2 as k_dw_grp does.
// The choice is per (row, hop), uniform over the warp, and the terms keep k_dw_grp's order,
// so results are bit-identical to it.
template <typename T, int VEC>
struct VecLds {  // VEC-wide shared-memory load
  static __device__ __forceinline__ void load(const T* p, T* x) {
#pragma unroll
    for (int r = 0; r < VEC; ++r) x[r] = p[r];
  }
};
template <>
struct VecLds<float, 2> {
  static __device__ __forceinline__ void load(const float* p, float* x) {
    const float2 t = *reinterpret_cast<const float2*>(p);
    x[0] = t.x;
    x[1] = t.y;
  }
};
template <>
struct VecLds<double, 2> {
  static __device__ __forceinline__ void load(const double* p, double* x) {
    const double2 t = *reinterpret_cast<const double2*>(p);
    x[0] = t.x;
    x[1] = t.y;
  }
};

template <typename T, int VEC, int NSEG, int KU, bool FIRST, bool SCALED, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) k_dw_blk(HxvArgs<T> a, const uint32_t* __restrict__ boff, int64_t nslab) {
  if (!select_column(a)) return;
  extern __shared__ __align__(16) unsigned char smem_dwb[];
  constexpr int SEGW = 32 * VEC, SLAB = SEGW * NSEG;
  const double sc = SCALED ? 1.0 / a.bn[a.jstep] : 1.0;
  constexpr bool SUB = SCALED && lz_sub_in_dw<T>();  // this pass starts from -c * uprev
  const T ccn = SUB && a.jstep > 0 ? T(-(a.bn[a.jstep] / a.bn[a.jstep - 1])) : T(0);
  __shared__ int s_ctr;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t r0 = boff[blockIdx.x];
  const int nr = int(boff[blockIdx.x + 1] - r0);
  T* tile = reinterpret_cast<T*>(smem_dwb);                 // [nr][SLAB]
  T* s_val = tile + size_t(nr) * SLAB;                      // [nr][kDwHops]
  T* s_edw = s_val + size_t(nr) * kDwHops;                  // [nr]
  uint32_t* s_src = reinterpret_cast<uint32_t*>(s_edw + nr);  // [nr][kDwHops]
  uint32_t* s_mdw = s_src + size_t(nr) * kDwHops;           // [nr]
  int* s_cnt = reinterpret_cast<int*>(s_mdw + nr);          // [nr]
  for (int rr = wib; rr < nr; rr += nw) {
    const uint32_t row = r0 + rr;
    const uint32_t k0 = a.off_dw[row];
    const int cnt = int(a.off_dw[row + 1] - k0);
    if (lane < cnt) {
      s_src[rr * kDwHops + lane] = a.src_dw[k0 + lane];
      s_val[rr * kDwHops + lane] = SCALED ? T(double(a.val_dw[k0 + lane]) * sc) : a.val_dw[k0 + lane];
    }
    if (lane == 0) {
      s_cnt[rr] = cnt;
      s_edw[rr] = a.e_dw[row];
      s_mdw[rr] = a.map_dw[row];
    }
  }
  const int64_t dimup = a.dimup;
  for (int64_t slab = 0; slab < nslab; ++slab) {
    const int64_t col0 = slab * SLAB + int64_t(lane) * VEC;
    bool act[NSEG];
#pragma unroll
    for (int g = 0; g < NSEG; ++g) act[g] = col0 + g * SEGW < dimup;
    // stage the block's own rows of this slab
    for (int rr = wib; rr < nr; rr += nw) {
      const T* __restrict__ src = a.v + int64_t(r0 + rr) * dimup + col0;
#pragma unroll
      for (int g = 0; g < NSEG; ++g)
        if (act[g]) VecLd<T, VEC>::load(src + g * SEGW, tile + size_t(rr) * SLAB + g * SEGW + lane * VEC);
    }
    if (threadIdx.x == 0) s_ctr = 0;
    __syncthreads();
    for (;;) {
      int rr = 0;
      if (lane == 0) rr = atomicAdd(&s_ctr, 1);
      rr = __shfl_sync(0xffffffffu, rr, 0);
      if (rr >= nr) break;
      const int64_t idw = r0 + rr;
      const T* __restrict__ vcol = a.v + col0;  // + src*dimup per external hop
      const T* tcol = tile + lane * VEC;
      const int64_t e0 = idw * dimup + col0;
      const int cnt = s_cnt[rr];
      const uint32_t* hs = s_src + rr * kDwHops;
      const T* hvv = s_val + rr * kDwHops;
      T acc[NSEG][VEC];
#pragma unroll
      for (int g = 0; g < NSEG; ++g) {
        if (!act[g]) continue;
        const int64_t c = col0 + g * SEGW;
        if (FIRST) {
          const T edw = s_edw[rr];
          const uint32_t mdw = s_mdw[rr];
          T x[VEC], up[VEC];
          VecLds<T, VEC>::load(tcol + size_t(rr) * SLAB + g * SEGW, x);
          if (SUB) VecLd<T, VEC>::load(a.uprev + e0 + g * SEGW, up);
#pragma unroll
          for (int r = 0; r < VEC; ++r) {
            const T d = a.e_up[c + r] + edw + a.U * T(__popc(a.map_up[c + r] & mdw));
            acc[g][r] = (SCALED ? T(double(d) * sc) : d) * x[r];
            if (SUB) acc[g][r] = fmaT<T>(ccn, up[r], acc[g][r]);
          }
        } else {
#pragma unroll
          for (int r = 0; r < VEC; ++r) acc[g][r] = a.hv[e0 + g * SEGW + r];
        }
      }
      for (int k = 0; k < cnt; k += KU) {
        T x[KU][NSEG][VEC];
#pragma unroll
        for (int u = 0; u < KU; ++u) {
          const int kk = k + u < cnt ? k + u : k;
          const uint32_t sr = hs[kk];
          const uint32_t lr = sr - r0;
          if (lr < uint32_t(nr)) {
            const T* t = tcol + size_t(lr) * SLAB;
#pragma unroll
            for (int g = 0; g < NSEG; ++g) VecLds<T, VEC>::load(t + g * SEGW, x[u][g]);
          } else {
            const T* __restrict__ src = vcol + int64_t(sr) * dimup;
#pragma unroll
            for (int g = 0; g < NSEG; ++g)
              if (act[g]) VecLd<T, VEC>::load(src + g * SEGW, x[u][g]);
          }
        }
#pragma unroll
        for (int u = 0; u < KU; ++u) {
          if (k + u < cnt) {
            const T h = hvv[k + u];
#pragma unroll
            for (int g = 0; g < NSEG; ++g)
              if (act[g]) Fma<T, VEC>::run(h, x[u][g], acc[g]);
          }
        }
      }
#pragma unroll
      for (int g = 0; g < NSEG; ++g)
        if (act[g]) {
#pragma unroll
          for (int r = 0; r < VEC; ++r) __stcs(a.hv + e0 + g * SEGW + r, acc[g][r]);
        }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- direct (on-the-fly) form
// No tables: each thread derives its hops from the bitstrings, as directMatVec does, with
// ranks from the combinatorial number system instead of binary_search. Bonds arrive
// sorted by 2^b - 2^a so that sources come out in ascending rank.
struct DirectArgsHdr {
  int nb_up, nb_dw;
  const int32_t* bonds;   // [nb_up + nb_dw][2]
  const double* bh;       // [nb_up + nb_dw]
  const uint32_t* C;      // binomial table
};

__device__ __forceinline__ uint32_t rank_of_d(uint32_t s, const uint32_t* C) {
  uint32_t r = 0;
  int i = 1;
  while (s) {
    int p = __ffs(s) - 1;
    r += C[p * kBinomN + i];
    ++i;
    s &= s - 1;
  }
  return r;
}

__device__ __forceinline__ int between_parity_d(uint32_t t, int a, int b) {
  int lo = a < b ? a : b, hi = a < b ? b : a;
  uint32_t mask = ((1u << hi) - 1u) & ~((2u << lo) - 1u);
  return __popc(t & mask) & 1;
}

template <typename T>
__global__ void __launch_bounds__(256) k_direct(HxvArgs<T> a, DirectArgsHdr d) {
  extern __shared__ unsigned char smem_raw[];
  int32_t* sb = reinterpret_cast<int32_t*>(smem_raw);
  const int nb = d.nb_up + d.nb_dw;
  T* sh = reinterpret_cast<T*>(smem_raw + ((2 * nb * sizeof(int32_t) + 15) / 16) * 16);
  __shared__ uint32_t sC[kBinomN * kBinomN];
  for (int k = threadIdx.x; k < 2 * nb; k += blockDim.x) sb[k] = d.bonds[k];
  for (int k = threadIdx.x; k < nb; k += blockDim.x) sh[k] = T(d.bh[k]);
  for (int k = threadIdx.x; k < kBinomN * kBinomN; k += blockDim.x) sC[k] = d.C[k];
  __syncthreads();
  const int64_t n = a.dimup * a.dimdw;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t idw = e / a.dimup, iup = e - idw * a.dimup;
    const uint32_t mup = a.map_up[iup], mdw = a.map_dw[idw];
    T acc = (a.e_up[iup] + a.e_dw[idw] + a.U * T(__popc(mup & mdw))) * a.v[e];
    for (int k = 0; k < d.nb_up; ++k) {
      const int ba = sb[2 * k], bb = sb[2 * k + 1];
      if (((mup >> ba) & 1u) && !((mup >> bb) & 1u)) {
        const uint32_t s = (mup & ~(1u << ba)) | (1u << bb);
        const T h = between_parity_d(mup, ba, bb) ? -sh[k] : sh[k];
        acc = fmaT<T>(h, a.v[idw * a.dimup + rank_of_d(s, sC)], acc);
      }
    }
    for (int k = d.nb_up; k < nb; ++k) {
      const int ba = sb[2 * k], bb = sb[2 * k + 1];
      if (((mdw >> ba) & 1u) && !((mdw >> bb) & 1u)) {
        const uint32_t s = (mdw & ~(1u << ba)) | (1u << bb);
        const T h = between_parity_d(mdw, ba, bb) ? -sh[k] : sh[k];
        acc = fmaT<T>(h, a.v[int64_t(rank_of_d(s, sC)) * a.dimup + iup], acc);
      }
    }
    a.hv[e] = acc;
  }
}

// Direct form by row blocks: a CTA takes kDirRows consecutive rows idw. One warp per row
// derives that row's down-spin hop list once (in bond order, kept in shared memory); each
// thread then derives the up-spin hops of its column iup once and applies them to all the
// block's rows. Per element: diagonal, up hops, down hops, each in bond order, the order
// k_direct sums them in.
constexpr int kDirRows = 8;
constexpr int kDirHops = 64;  // hop-list capacity per row (host checks the bound)

template <typename T>
__global__ void __launch_bounds__(256) k_direct_rows(HxvArgs<T> a, DirectArgsHdr d, int64_t nrb) {
  extern __shared__ unsigned char smem_raw[];
  int32_t* sb = reinterpret_cast<int32_t*>(smem_raw);
  const int nb = d.nb_up + d.nb_dw;
  T* sh = reinterpret_cast<T*>(smem_raw + ((2 * nb * sizeof(int32_t) + 15) / 16) * 16);
  __shared__ uint32_t sC[kBinomN * kBinomN];
  __shared__ uint32_t s_src[kDirRows][kDirHops];
  __shared__ T s_val[kDirRows][kDirHops];
  __shared__ int s_cnt[kDirRows];
  __shared__ uint32_t s_mdw[kDirRows];
  __shared__ T s_edw[kDirRows];
  for (int k = threadIdx.x; k < 2 * nb; k += blockDim.x) sb[k] = d.bonds[k];
  for (int k = threadIdx.x; k < nb; k += blockDim.x) sh[k] = T(d.bh[k]);
  for (int k = threadIdx.x; k < kBinomN * kBinomN; k += blockDim.x) sC[k] = d.C[k];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t dimup = a.dimup;
  for (int64_t rb = blockIdx.x; rb < nrb; rb += gridDim.x) {
    const int64_t r0 = rb * kDirRows;
    __syncthreads();
    if (warp < kDirRows) {
      const int64_t row = r0 + warp;
      int cnt = 0;
      if (row < a.dimdw) {
        const uint32_t mdw = a.map_dw[row];
        for (int k0 = d.nb_up; k0 < nb; k0 += 32) {
          const int k = k0 + lane;
          bool ok = false;
          int ba = 0, bb = 0;
          if (k < nb) {
            ba = sb[2 * k];
            bb = sb[2 * k + 1];
            ok = ((mdw >> ba) & 1u) && !((mdw >> bb) & 1u);
          }
          const unsigned ball = __ballot_sync(0xffffffffu, ok);
          if (ok) {
            const int pos = cnt + __popc(ball & ((1u << lane) - 1u));
            if (pos < kDirHops) {
              const uint32_t t = (mdw & ~(1u << ba)) | (1u << bb);
              s_src[warp][pos] = rank_of_d(t, sC);
              s_val[warp][pos] = between_parity_d(mdw, ba, bb) ? -sh[k] : sh[k];
            }
          }
          cnt += __popc(ball);
        }
        if (lane == 0) {
          s_mdw[warp] = mdw;
          s_edw[warp] = a.e_dw[row];
        }
      }
      if (lane == 0) s_cnt[warp] = cnt < kDirHops ? cnt : kDirHops;
    }
    __syncthreads();
    for (int64_t iup = threadIdx.x; iup < dimup; iup += blockDim.x) {
      const uint32_t mup = a.map_up[iup];
      const T eu = a.e_up[iup];
      T acc[kDirRows];
#pragma unroll
      for (int r = 0; r < kDirRows; ++r)
        acc[r] = r0 + r < a.dimdw
                     ? (eu + s_edw[r] + a.U * T(__popc(mup & s_mdw[r]))) * a.v[(r0 + r) * dimup + iup]
                     : T(0);
      for (int k = 0; k < d.nb_up; ++k) {
        const int ba = sb[2 * k], bb = sb[2 * k + 1];
        if (((mup >> ba) & 1u) && !((mup >> bb) & 1u)) {
          const uint32_t t = (mup & ~(1u << ba)) | (1u << bb);
          const T h = between_parity_d(mup, ba, bb) ? -sh[k] : sh[k];
          const int64_t src = rank_of_d(t, sC);
#pragma unroll
          for (int r = 0; r < kDirRows; ++r)
            if (r0 + r < a.dimdw) acc[r] = fmaT<T>(h, a.v[(r0 + r) * dimup + src], acc[r]);
        }
      }
#pragma unroll
      for (int r = 0; r < kDirRows; ++r) {
        if (r0 + r >= a.dimdw) continue;
        for (int q = 0; q < s_cnt[r]; ++q)
          acc[r] = fmaT<T>(s_val[r][q], a.v[int64_t(s_src[r][q]) * dimup + iup], acc[r]);
        a.hv[(r0 + r) * dimup + iup] = acc[r];
      }
    }
  }
}

// ---- complex Hij: vectors of complex elements stored interleaved (re, im)
template <typename T>
struct Cplx;
template <>
struct Cplx<float> {
  using type = float2;
};
template <>
struct Cplx<double> {
  using type = double2;
};

// acc += h * y for complex h = (hr, hi), y
template <typename T, typename T2>
__device__ __forceinline__ void cmad(T hr, T hi, T2 y, T& re, T& im) {
  re = fmaT<T>(hr, y.x, re);
  re = fmaT<T>(-hi, y.y, re);
  im = fmaT<T>(hr, y.y, im);
  im = fmaT<T>(hi, y.x, im);
}

// Stored form, one thread per element: the diagonal, then the down hops, then the up hops,
// each row's sources ascending (the order of the real passes and of spMatVec). Table values
// hold sign * conjg(Hij) (real parts in val_*, imaginary parts in vi_*).
template <typename T>
__global__ void __launch_bounds__(256) k_cplx_stored(HxvArgs<T> a, const T* __restrict__ vi_up,
                                                     const T* __restrict__ vi_dw) {
  using T2 = typename Cplx<T>::type;
  const T2* __restrict__ v = reinterpret_cast<const T2*>(a.v);
  T2* __restrict__ hv = reinterpret_cast<T2*>(a.hv);
  const int64_t n = a.dimup * a.dimdw;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t idw = e / a.dimup, iup = e - idw * a.dimup;
    const T d = a.e_up[iup] + a.e_dw[idw] + a.U * T(__popc(a.map_up[iup] & a.map_dw[idw]));
    const T2 x = v[e];
    T re = d * x.x, im = d * x.y;
    for (uint32_t k = a.off_dw[idw]; k < a.off_dw[idw + 1]; ++k)
      cmad(a.val_dw[k], vi_dw[k], v[int64_t(a.src_dw[k]) * a.dimup + iup], re, im);
    for (uint32_t k = a.off_up[iup]; k < a.off_up[iup + 1]; ++k)
      cmad(a.val_up[k], vi_up[k], v[idw * a.dimup + a.src_up[k]], re, im);
    T2 out;
    out.x = re;
    out.y = im;
    hv[e] = out;
  }
}

// Direct form, one thread per element, bonds in shared memory: the diagonal, then the up
// hops, then the down hops in bond order (directMatVec's order), value sign * Hij (not
// conjugated: the reference's direct and stored forms differ by conjugation here).
template <typename T>
__global__ void __launch_bounds__(256) k_cplx_direct(HxvArgs<T> a, DirectArgsHdr d, const double* __restrict__ bhi) {
  using T2 = typename Cplx<T>::type;
  extern __shared__ unsigned char smem_raw[];
  int32_t* sb = reinterpret_cast<int32_t*>(smem_raw);
  const int nb = d.nb_up + d.nb_dw;
  T* shr = reinterpret_cast<T*>(smem_raw + ((2 * nb * sizeof(int32_t) + 15) / 16) * 16);
  T* shi = shr + nb;
  __shared__ uint32_t sC[kBinomN * kBinomN];
  for (int k = threadIdx.x; k < 2 * nb; k += blockDim.x) sb[k] = d.bonds[k];
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {
    shr[k] = T(d.bh[k]);
    shi[k] = T(bhi[k]);
  }
  for (int k = threadIdx.x; k < kBinomN * kBinomN; k += blockDim.x) sC[k] = d.C[k];
  __syncthreads();
  const T2* __restrict__ v = reinterpret_cast<const T2*>(a.v);
  T2* __restrict__ hv = reinterpret_cast<T2*>(a.hv);
  const int64_t n = a.dimup * a.dimdw;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t idw = e / a.dimup, iup = e - idw * a.dimup;
    const uint32_t mup = a.map_up[iup], mdw = a.map_dw[idw];
    const T dg = a.e_up[iup] + a.e_dw[idw] + a.U * T(__popc(mup & mdw));
    const T2 x = v[e];
    T re = dg * x.x, im = dg * x.y;
    for (int k = 0; k < d.nb_up; ++k) {
      const int ba = sb[2 * k], bb = sb[2 * k + 1];
      if (((mup >> ba) & 1u) && !((mup >> bb) & 1u)) {
        const uint32_t t = (mup & ~(1u << ba)) | (1u << bb);
        const T sg = between_parity_d(mup, ba, bb) ? T(-1) : T(1);
        cmad(sg * shr[k], sg * shi[k], v[idw * a.dimup + rank_of_d(t, sC)], re, im);
      }
    }
    for (int k = d.nb_up; k < nb; ++k) {
      const int ba = sb[2 * k], bb = sb[2 * k + 1];
      if (((mdw >> ba) & 1u) && !((mdw >> bb) & 1u)) {
        const uint32_t t = (mdw & ~(1u << ba)) | (1u << bb);
        const T sg = between_parity_d(mdw, ba, bb) ? T(-1) : T(1);
        cmad(sg * shr[k], sg * shi[k], v[int64_t(rank_of_d(t, sC)) * a.dimup + iup], re, im);
      }
    }
    T2 out;
    out.x = re;
    out.y = im;
    hv[e] = out;
  }
}

template <typename T>
const T* pick(const DevBuf<double>& d, const DevBuf<float>& f);
template <>
const double* pick<double>(const DevBuf<double>& d, const DevBuf<float>&) { return d.p; }
template <>
const float* pick<float>(const DevBuf<double>&, const DevBuf<float>& f) { return f.p; }

int sm_count() {
  static int cached = 0;
  if (!cached) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&cached, cudaDevAttrMultiProcessorCount, dev);
    if (cached <= 0) cached = 148;
  }
  return cached;
}

template <typename T>
const T* pick_sell(const SpinBasis& B);
template <>
const double* pick_sell<double>(const SpinBasis& B) { return B.sell_v64.p; }
template <>
const float* pick_sell<float>(const SpinBasis& B) { return B.sell_v32.p; }

template <typename T, int RT, bool FIRST, bool UNIFORM, bool LZ>
int launch_up_smem(const HxvArgs<T>& a, const SellArgs<T>& sl, cudaStream_t st, int sms, int* grid) {
  const size_t smem = size_t(a.dimup + kUpZeroSlots) * RT * sizeof(T);
  const int per_sm = smem <= kUpSmemTwoPerSM ? 2 : 1;
  auto kern = per_sm == 2 ? k_up_smem<T, RT, FIRST, UNIFORM, LZ, false> : k_up_smem<T, RT, FIRST, UNIFORM, LZ, true>;
  if constexpr (sizeof(T) == 4 && UNIFORM) {
    if (per_sm == 2 && sl.v4) kern = k_up_smem<T, RT, FIRST, UNIFORM, LZ, false, true>;
  }
  if (smem > 48 * 1024) EDG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  const int64_t nrb = (a.dimdw + RT - 1) / RT;
  int64_t g = nrb < int64_t(sms) * per_sm ? nrb : int64_t(sms) * per_sm;
  if (LZ && g > kRedBlocks) g = kRedBlocks;  // one partial per block in the reduction scratch
  kern<<<dim3(int(g), a.ncols), per_sm == 2 ? up_threads<T, LZ, false>() : up_threads<T, LZ, true>(), smem, st>>>(a, sl, nrb);
  EDG_CUDA(cudaGetLastError());
  if (grid) *grid = int(g);
  return EDG_OK;
}

// VEC-wide loads need every row start aligned: DimUp a multiple of VEC and 2*sizeof(T)
// aligned vector pointers (always true for our own buffers; checked for callers' pointers).
// SCALED (Lanczos-fused mode) applies H to v = u / bn[jstep] by scaling the matrix elements.
template <typename T, bool FIRST, bool SCALED>
int dw_pass(const HxvArgs<T>& a, const SpinBasis& Bdw, cudaStream_t st, int sms) {
  const bool v2 = (a.dimup % 2 == 0) && (reinterpret_cast<uintptr_t>(a.v) % (2 * sizeof(T)) == 0) &&
                  (reinterpret_cast<uintptr_t>(a.hv) % (2 * sizeof(T)) == 0) &&
                  (!(SCALED && lz_sub_in_dw<T>()) || reinterpret_cast<uintptr_t>(a.uprev) % (2 * sizeof(T)) == 0);
  const int vec = v2 ? 2 : 1;
  const SpinBasis::RowBlocks* rb = (a.dwv == 1 || a.dwv == 2) ? &Bdw.rowblk[a.dwv - 1] : nullptr;
  if (rb && Bdw.max_row <= kDwHops && rb->count > 0) {
    constexpr int NSEG = sizeof(T) == 4 ? 4 : 2;
    constexpr int KU = sizeof(T) == 4 ? 3 : 4;
    const int slabw = 32 * vec * NSEG;
    const size_t smem = size_t(rb->max_rows) * (size_t(slabw) * sizeof(T) + kDwHops * (sizeof(T) + 4) + sizeof(T) + 8) + 16;
    const int nt = a.dwv == 2 ? 512 : 1024;
    if (smem <= (nt == 512 ? kUpSmemTwoPerSM : kUpSmemOnePerSM)) {
      auto kern = nt == 512 ? (v2 ? k_dw_blk<T, 2, NSEG, KU, FIRST, SCALED, 512> : k_dw_blk<T, 1, NSEG, KU, FIRST, SCALED, 512>)
                            : (v2 ? k_dw_blk<T, 2, NSEG, KU, FIRST, SCALED, 1024> : k_dw_blk<T, 1, NSEG, KU, FIRST, SCALED, 1024>);
      EDG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      const int64_t nslab = (a.dimup + slabw - 1) / slabw;
      kern<<<dim3(rb->count, a.ncols), nt, smem, st>>>(a, rb->off.p, nslab);
      EDG_CUDA(cudaGetLastError());
      return EDG_OK;
    }
  }
  if (Bdw.max_row <= kDwHops && Bdw.groups > 0) {
    // FP32: 4 float2 segments per lane (256 columns per slab); FP64: 2 double2 segments,
    // 4 hops in flight (3 in the Lanczos-scaled form, which spilled at 4 within the 64
    // registers of 4 CTAs per SM)
    constexpr int NSEG = sizeof(T) == 4 ? 4 : 2;
    constexpr int KU = sizeof(T) == 4 ? 3 : (SCALED ? 3 : 4);
    auto kern = v2 ? k_dw_grp<T, 2, NSEG, KU, FIRST, SCALED> : k_dw_grp<T, 1, NSEG, KU, FIRST, SCALED>;
    const size_t smem = size_t(Bdw.group_max) * (kDwHops * (sizeof(T) + 4) + sizeof(T) + 12) + 16;
    if (smem > 48 * 1024) EDG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const int64_t nslab = (a.dimup + 32 * vec * NSEG - 1) / (32 * vec * NSEG);
    kern<<<dim3(Bdw.groups, a.ncols), 256, smem, st>>>(a, Bdw.group_off.p, Bdw.group_rows.p, nslab);
    EDG_CUDA(cudaGetLastError());
    return EDG_OK;
  }
  if (SCALED || a.ncols > 1) {
    set_error("fused Lanczos and block H x V need the grouped down pass");
    return EDG_ERR_UNSUPPORTED;
  }
  const int64_t nslab = (a.dimup + 32 * vec - 1) / (32 * vec);
  const int64_t ntiles = nslab * a.dimdw;
  const int64_t want = (ntiles + 7) / 8;
  const int g = int(want < int64_t(sms) * 8 ? want : int64_t(sms) * 8);
  if (v2) k_dw_seg<T, 2, FIRST><<<g, 256, 0, st>>>(a, ntiles);
  else k_dw_seg<T, 1, FIRST><<<g, 256, 0, st>>>(a, ntiles);
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

// Packed-schedule FP32 up pass (k_up_p16); returns false when the sector has no packed table.
template <bool LZ>
bool launch_up_p16(const HxvArgs<float>& a, const SpinBasis& B, cudaStream_t st, int sms, int* status) {
  if (B.p16_negoff == 0 || (a.upv != 1 && a.upv != 2)) return false;
  const bool neg = a.upv == 1;
  P16Args q;
  q.ent = neg ? B.p16_ent.p : B.p16f_ent.p;
  q.off = B.p16_off.p;
  q.h = float(B.sell_h);
  q.negoff = B.p16_negoff;
  const size_t smem = neg ? size_t(B.p16_negoff + a.dimup + kUpZeroSlots) * sizeof(float2)
                          : size_t(a.dimup + kUpZeroSlots) * sizeof(float2);
  if (smem > kUpSmemOnePerSM) return false;
  const int per_sm = smem <= kUpSmemTwoPerSM ? 2 : 1;
  auto kern = neg ? (per_sm == 2 ? k_up_p16<true, false, LZ> : k_up_p16<true, true, LZ>)
                  : (per_sm == 2 ? k_up_p16<false, false, LZ> : k_up_p16<false, true, LZ>);
  *status = EDG_OK;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) {
    set_error("k_up_p16: %s", cudaGetErrorString(e));
    *status = EDG_ERR_CUDA;
    return true;
  }
  const int64_t nrb = (a.dimdw + 1) / 2;
  int64_t g = nrb < int64_t(sms) * per_sm ? nrb : int64_t(sms) * per_sm;
  if (LZ && g > kRedBlocks) g = kRedBlocks;
  kern<<<dim3(int(g), a.ncols), 1024, smem, st>>>(a, q, nrb);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("k_up_p16: %s", cudaGetErrorString(e));
    *status = EDG_ERR_CUDA;
  }
  return true;
}

// Kronecker-schedule FP32 up pass (k_up_kron); returns false when the sector has no schedule.
template <int RT, bool LZ>
int launch_up_kron_rt(const HxvArgs<float>& a, const KronArgs& q, cudaStream_t st, int sms) {
  const size_t smem = kron_smem(a.dimup, RT, q.nkrow, q.nhent);
  const int per_sm = smem <= kUpSmemTwoPerSM ? 2 : 1;
  auto kern = per_sm == 2 ? k_up_kron<RT, LZ, false> : k_up_kron<RT, LZ, true>;
  if (smem > 48 * 1024) EDG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  const int64_t nrb = (a.dimdw + RT - 1) / RT;
  int64_t g = nrb < int64_t(sms) * per_sm ? nrb : int64_t(sms) * per_sm;
  if (LZ && g > kRedBlocks) g = kRedBlocks;
  kern<<<dim3(int(g), a.ncols), kKronThreads, smem, st>>>(a, q, nrb);
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}
template <bool LZ>
bool launch_up_kron(const HxvArgs<float>& a, const SpinBasis& B, cudaStream_t st, int sms, int* status) {
  if (B.kron_m == 0 || a.upv != 3) return false;
  KronArgs q;
  q.thr = B.kron_thr.p;
  q.bcol = B.kron_bcol.p;
  q.hoff = B.kron_hoff.p;
  q.hent = B.kron_hent.p;
  q.lent = B.kron_lent.p;
  q.xent = B.kron_xent.p;
  q.xoff = B.kron_xoff.p;
  q.xwid = B.kron_xwid.p;
  q.nthr = B.kron_nthr;
  q.lmax = B.kron_lmax;
  q.nkrow = B.kron_nkrow;
  q.nhent = B.kron_nhent;
  q.h = float(B.sell_h);
  const int rt = up_rows_per_cta(a.dimup, sizeof(float));
  *status = rt == 4 ? launch_up_kron_rt<4, LZ>(a, q, st, sms)
          : rt == 2 ? launch_up_kron_rt<2, LZ>(a, q, st, sms)
                    : launch_up_kron_rt<1, LZ>(a, q, st, sms);
  return true;
}

template <typename T, bool FIRST, bool LZ>
int up_pass(const HxvArgs<T>& a, const SpinBasis& B, cudaStream_t st, int sms, int* grid) {
  if constexpr (std::is_same<T, float>::value && !FIRST) {
    int status = EDG_OK;
    if (launch_up_kron<LZ>(a, B, st, sms, &status)) return status;
    if (launch_up_p16<LZ>(a, B, st, sms, &status)) return status;
  }
  const int rt = up_rows_per_cta(a.dimup, sizeof(T));
  if (rt == 0) {
    if (LZ || a.ncols > 1) {
      set_error("fused Lanczos H x v needs the shared-memory up pass");
      return EDG_ERR_UNSUPPORTED;
    }
    if (B.split_parts > 0) {
      SplitArgs<T> sp;
      sp.ent = B.split_ent.p;
      sp.off = B.split_off.p;
      sp.val = sizeof(T) == 8 ? reinterpret_cast<const T*>(B.split_v64.p) : reinterpret_cast<const T*>(B.split_v32.p);
      sp.h = T(B.sell_h);
      sp.parts = B.split_parts;
      sp.nsl = (a.dimup + 31) / 32;
      int64_t wmax = 0;
      for (int p = 0; p <= SpinBasis::kMaxSplit; ++p) sp.col[p] = p <= B.split_parts ? B.split_col[p] : 0;
      for (int p = 0; p < B.split_parts; ++p) wmax = std::max<int64_t>(wmax, sp.col[p + 1] - sp.col[p]);
      const size_t smem = size_t(wmax + kUpZeroSlots) * sizeof(T);
      auto kern = B.sell_uniform ? k_up_split<T, FIRST, true> : k_up_split<T, FIRST, false>;
      EDG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      const int g = int(a.dimdw < int64_t(sms) ? a.dimdw : int64_t(sms));
      kern<<<g, 1024, smem, st>>>(a, sp);
      EDG_CUDA(cudaGetLastError());
      return EDG_OK;
    }
    const int g = int(a.dimdw < int64_t(sms) * 8 ? a.dimdw : int64_t(sms) * 8);
    k_up_rows<T, FIRST><<<g, 256, 0, st>>>(a);
    EDG_CUDA(cudaGetLastError());
    return EDG_OK;
  }
  SellArgs<T> sl;
  sl.ent = B.sell_ent.p;
  sl.off = B.sell_off.p;
  if (sizeof(T) == 4 && B.sched_rt == rt && B.sched_ent.p) {  // FP32: bank-conflict-free order
    sl.ent = B.sched_ent.p;
    sl.off = B.sched_off.p;
    sl.v4 = B.sched_v4;
  }
  sl.val = pick_sell<T>(B);
  sl.h = T(B.sell_h);
  constexpr int R4 = sizeof(T) == 4 ? 4 : 2;
  if (B.sell_uniform) {
    if (rt == 4) return launch_up_smem<T, R4, FIRST, true, LZ>(a, sl, st, sms, grid);
    if (rt == 2) return launch_up_smem<T, 2, FIRST, true, LZ>(a, sl, st, sms, grid);
    return launch_up_smem<T, 1, FIRST, true, LZ>(a, sl, st, sms, grid);
  }
  if (rt == 4) return launch_up_smem<T, R4, FIRST, false, LZ>(a, sl, st, sms, grid);
  if (rt == 2) return launch_up_smem<T, 2, FIRST, false, LZ>(a, sl, st, sms, grid);
  return launch_up_smem<T, 1, FIRST, false, LZ>(a, sl, st, sms, grid);
}

template <typename T>
HxvArgs<T> make_args(edg_sector_s* s, const T* v, T* hv) {
  HxvArgs<T> a;
  a.v = v;
  a.hv = hv;
  a.dimup = s->up.dim;
  a.dimdw = s->dw.dim;
  a.off_up = s->up.off.p;
  a.src_up = s->up.src.p;
  a.val_up = pick<T>(s->up.val64, s->up.val32);
  a.off_dw = s->dw.off.p;
  a.src_dw = s->dw.src.p;
  a.val_dw = pick<T>(s->dw.val64, s->dw.val32);
  a.e_up = pick<T>(s->up.e64, s->up.e32);
  a.e_dw = pick<T>(s->dw.e64, s->dw.e32);
  a.map_up = s->up.map.p;
  a.map_dw = s->dw.map.p;
  a.U = T(s->U);
  a.dwv = s->hxv_dw[sizeof(T) == 4];
  a.upv = sizeof(T) == 4 ? s->hxv_up[1] : 0;
  return a;
}

// Single-pass H x v (down-pass choice 3): one launch does the whole H x v; no up pass.
template <typename T, bool LZ>
int fused_pass(const HxvArgs<T>& a, cudaStream_t st, int sms) {
  const int64_t ntiles = a.dimdw * ((a.dimup + 31) / 32);
  const int64_t want = (ntiles + 7) / 8;
  int64_t g = want < int64_t(sms) * 8 ? want : int64_t(sms) * 8;
  if (LZ && g > kRedBlocks) g = kRedBlocks;  // one partial per block in the reduction scratch
  if (g < 1) g = 1;
  k_hxv_fused<T, LZ><<<dim3(int(g), a.ncols), 256, 0, st>>>(a, ntiles);
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

}  // namespace

template <typename T>
int hxv_apply(edg_sector_s* s, const T* v, T* hv) {
  HxvArgs<T> a = make_args<T>(s, v, hv);
  const int sms = sm_count();
  cudaStream_t st = s->stream;
  if (s->cplx) {
    const int64_t n = a.dimup * a.dimdw;
    const int64_t want = (n + 255) / 256;
    const int g = int(want < int64_t(sms) * 8 ? (want < 1 ? 1 : want) : int64_t(sms) * 8);
    if (s->form == EDG_FORM_STORED) {
      k_cplx_stored<T><<<g, 256, 0, st>>>(a, pick<T>(s->up.val64i, s->up.val32i), pick<T>(s->dw.val64i, s->dw.val32i));
    } else {
      DirectArgsHdr d;
      d.nb_up = s->bonds[0].nb;
      d.nb_dw = s->bonds[1].nb;
      d.bonds = s->bond_dev.p;
      d.bh = s->bondh_dev.p;
      d.C = s->binom.p;
      const int nb = d.nb_up + d.nb_dw;
      const size_t smem = ((2 * nb * sizeof(int32_t) + 15) / 16) * 16 + 2 * nb * sizeof(T) + 16;
      if (smem > 48 * 1024)
        EDG_CUDA(cudaFuncSetAttribute(k_cplx_direct<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      k_cplx_direct<T><<<g, 256, smem, st>>>(a, d, s->bondhi_dev.p);
    }
    EDG_CUDA(cudaGetLastError());
    return EDG_OK;
  }
  if (s->form == EDG_FORM_STORED) {
    if (a.dwv == 3) return fused_pass<T, false>(a, st, sms);
    EDG_CHECK((dw_pass<T, true, false>(a, s->dw, st, sms)));
    EDG_CHECK((up_pass<T, false, false>(a, s->up, st, sms, nullptr)));
  } else {
    DirectArgsHdr d;
    d.nb_up = s->bonds[0].nb;
    d.nb_dw = s->bonds[1].nb;
    d.bonds = s->bond_dev.p;
    d.bh = s->bondh_dev.p;
    d.C = s->binom.p;
    const int nb = d.nb_up + d.nb_dw;
    size_t smem = ((2 * nb * sizeof(int32_t) + 15) / 16) * 16 + nb * sizeof(T) + 16;
    // down hops of one configuration: at most min(directed bonds, Ndw * (Ns - Ndw))
    const int64_t hop_bound = std::min<int64_t>(d.nb_dw, int64_t(s->ndw) * (s->model.ns - s->ndw));
    if (hop_bound <= kDirHops) {
      const int64_t nrb = (a.dimdw + kDirRows - 1) / kDirRows;
      const int g = int(nrb < int64_t(sms) * 8 ? nrb : int64_t(sms) * 8);
      if (smem > 32 * 1024)
        EDG_CUDA(cudaFuncSetAttribute(k_direct_rows<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      k_direct_rows<T><<<g, 256, smem, st>>>(a, d, nrb);
    } else {
      const int64_t n = a.dimup * a.dimdw;
      const int64_t want = (n + 255) / 256;
      const int g = int(want < int64_t(sms) * 8 ? want : int64_t(sms) * 8);
      if (smem > 48 * 1024) EDG_CUDA(cudaFuncSetAttribute(k_direct<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      k_direct<T><<<g, 256, smem, st>>>(a, d);
    }
    EDG_CUDA(cudaGetLastError());
  }
  return EDG_OK;
}

template int hxv_apply<float>(edg_sector_s*, const float*, float*);
template int hxv_apply<double>(edg_sector_s*, const double*, double*);

// Slab forms of the stored H x v for vectors split over ranks by rows (the down-spin index).
// Column slab: all DimDw rows of columns [col0, col0 + ncols), row-major with row length
// ncols; hv = (diag + H_dw x I) v there, by the down pass of hxv_apply. Row slab: rows
// [row0, row0 + nrows) of length DimUp; hv += (I x H_up) v, by its up pass. The column form
// and then (after the transposes) the row form compute every element in hxv_apply's order,
// so the split H x v equals it bit for bit.
template <typename T>
int hxv_cols(edg_sector_s* s, int64_t col0, int64_t ncols, const T* v, T* hv) {
  if (s->cplx || s->form != EDG_FORM_STORED) {
    set_error("slab H x v: real stored-form sectors only");
    return EDG_ERR_UNSUPPORTED;
  }
  HxvArgs<T> a = make_args<T>(s, v, hv);
  a.dimup = ncols;
  a.e_up += col0;
  a.map_up += col0;
  if (a.dwv == 3) a.dwv = 0;  // the single pass needs whole rows
  return dw_pass<T, true, false>(a, s->dw, s->stream, sm_count());
}
template <typename T>
int hxv_rows(edg_sector_s* s, int64_t row0, int64_t nrows, const T* v, T* hv) {
  if (s->cplx || s->form != EDG_FORM_STORED) {
    set_error("slab H x v: real stored-form sectors only");
    return EDG_ERR_UNSUPPORTED;
  }
  HxvArgs<T> a = make_args<T>(s, v, hv);
  a.dimdw = nrows;
  a.e_dw += row0;
  a.map_dw += row0;
  return up_pass<T, false, false>(a, s->up, s->stream, sm_count(), nullptr);
}
template int hxv_cols<float>(edg_sector_s*, int64_t, int64_t, const float*, float*);
template int hxv_cols<double>(edg_sector_s*, int64_t, int64_t, const double*, double*);
template int hxv_rows<float>(edg_sector_s*, int64_t, int64_t, const float*, float*);
template int hxv_rows<double>(edg_sector_s*, int64_t, int64_t, const double*, double*);

// Lanczos-fused H x v (stored form): with v = u / bn[j], writes w = H v - (bn[j]/bn[j-1]) uprev
// into `w` and <v, w> into *aout (`partial`: a reduction scratch of kRedSlots doubles). Returns
// EDG_ERR_UNSUPPORTED when the sector needs one of the general kernels instead.
template <typename T>
int hxv_apply_lz(edg_sector_s* s, const T* u, const T* uprev, T* w, const double* bn, int j, double* partial,
                 double* aout) {
  if (s->cplx || s->form != EDG_FORM_STORED || up_rows_per_cta(s->up.dim, sizeof(T)) == 0 ||
      s->dw.max_row > kDwHops || s->dw.groups == 0) {
    set_error("fused Lanczos H x v not available for this sector");
    return EDG_ERR_UNSUPPORTED;
  }
  HxvArgs<T> a = make_args<T>(s, u, w);
  a.bn = bn;
  a.jstep = j;
  a.uprev = uprev;
  a.partial = partial;
  a.red_out = aout;
  const int sms = sm_count();
  if (a.dwv == 3) return fused_pass<T, true>(a, s->stream, sms);
  EDG_CHECK((dw_pass<T, true, true>(a, s->dw, s->stream, sms)));
  EDG_CHECK((up_pass<T, false, true>(a, s->up, s->stream, sms, nullptr)));
  return EDG_OK;
}
bool hxv_lz_available(const edg_sector_s* s, size_t elem) {
  return !s->cplx && s->form == EDG_FORM_STORED && up_rows_per_cta(s->up.dim, elem) > 0 &&
         s->dw.max_row <= kDwHops && s->dw.groups > 0;
}
template <typename T>
int hxv_block(edg_sector_s* s, int ncols, const int* active, const T* v, T* hv) {
  if (!hxv_lz_available(s, sizeof(T))) {
    set_error("block H x V not available for this sector");
    return EDG_ERR_UNSUPPORTED;
  }
  HxvArgs<T> a = make_args<T>(s, v, hv);
  a.vstride = s->vlen;
  a.active = active;
  a.ncols = ncols;
  const int sms = sm_count();
  if (a.dwv == 3) return fused_pass<T, false>(a, s->stream, sms);
  EDG_CHECK((dw_pass<T, true, false>(a, s->dw, s->stream, sms)));
  EDG_CHECK((up_pass<T, false, false>(a, s->up, s->stream, sms, nullptr)));
  return EDG_OK;
}

template <typename T>
int hxv_block_lz(edg_sector_s* s, int ncols, const int* active, const T* u, const T* uprev, T* w, const double* bn,
                 int64_t sstride, int j, double* partial, double* aout) {
  if (!hxv_lz_available(s, sizeof(T))) {
    set_error("block H x V not available for this sector");
    return EDG_ERR_UNSUPPORTED;
  }
  HxvArgs<T> a = make_args<T>(s, u, w);
  a.bn = bn;
  a.jstep = j;
  a.uprev = uprev;
  a.partial = partial;
  a.red_out = aout;
  a.vstride = s->vlen;
  a.sstride = sstride;
  a.active = active;
  a.ncols = ncols;
  const int sms = sm_count();
  if (a.dwv == 3) return fused_pass<T, true>(a, s->stream, sms);
  EDG_CHECK((dw_pass<T, true, true>(a, s->dw, s->stream, sms)));
  EDG_CHECK((up_pass<T, false, true>(a, s->up, s->stream, sms, nullptr)));
  return EDG_OK;
}
// Autotuner: every down-pass x up-pass pair (4 x 4 for FP32, 4 x 1 for FP64; a pair whose
// kernel does not apply to the sector falls back to the default kernel and times like it) on
// `reps` H x v of scratch vectors after one untimed application, timed with CUDA events on
// the sector's stream; the fastest pair becomes the sector's choice for precision T. Its
// arithmetic is unchanged in FP64 (every pair gives the same bits); in FP32 the packed and
// Kronecker up passes sum the terms of a row in another order.
template <typename T>
int hxv_autotune(edg_sector_s* s, int reps, double* ms, int* nc, int* best) {
  if (s->cplx || s->form != EDG_FORM_STORED) {
    set_error("edg_sector_autotune: only the real stored form has kernel variants");
    return EDG_ERR_UNSUPPORTED;
  }
  const int nup = sizeof(T) == 4 ? 4 : 1;
  const int ncand = 4 * nup;
  cudaStream_t st = s->stream;
  EDG_CHECK(sector_variant_tables(s));
  DevBuf<T> x, y;
  EDG_CHECK(x.alloc(size_t(s->vlen), st, "autotune vectors"));
  EDG_CHECK(y.alloc(size_t(s->vlen), st, "autotune vectors"));
  DevBuf<double> r;
  EDG_CHECK(r.alloc(size_t(s->vlen), st, "autotune vectors"));
  EDG_CHECK(random_dev(st, r.p, s->vlen, 12345));
  EDG_CHECK((convert_dev<T, double>(st, x.p, r.p, s->vlen, 1.0)));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  EDG_CUDA(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    set_error("edg_sector_autotune: cudaEventCreate failed");
    return EDG_ERR_CUDA;
  }
  const int keep_dw = s->hxv_dw[sizeof(T) == 4], keep_up = s->hxv_up[sizeof(T) == 4];
  int status = EDG_OK, arg = 0;
  double tbest = 1e300;
  for (int cnd = 0; cnd < ncand && status == EDG_OK; ++cnd) {
    s->hxv_dw[sizeof(T) == 4] = cnd / nup;
    s->hxv_up[sizeof(T) == 4] = cnd % nup;
    status = hxv_apply<T>(s, x.p, y.p);  // untimed: first launch of the pair
    float t = 0.f;
    if (status == EDG_OK && cudaEventRecord(e0, st) != cudaSuccess) status = EDG_ERR_CUDA;
    for (int k = 0; k < reps && status == EDG_OK; ++k) status = hxv_apply<T>(s, x.p, y.p);
    if (status == EDG_OK && (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                             cudaEventElapsedTime(&t, e0, e1) != cudaSuccess))
      status = EDG_ERR_CUDA;
    const double per = double(t) / (reps > 0 ? reps : 1);
    if (ms) ms[cnd] = per;
    if (status == EDG_OK && per < tbest) {
      tbest = per;
      arg = cnd;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status != EDG_OK) {
    s->hxv_dw[sizeof(T) == 4] = keep_dw;
    s->hxv_up[sizeof(T) == 4] = keep_up;
    if (status == EDG_ERR_CUDA) set_error("edg_sector_autotune: timing failed");
    return status;
  }
  s->hxv_dw[sizeof(T) == 4] = arg / nup;
  s->hxv_up[sizeof(T) == 4] = arg % nup;
  if (nc) *nc = ncand;
  if (best) *best = arg;
  return EDG_OK;
}
template int hxv_autotune<float>(edg_sector_s*, int, double*, int*, int*);
template int hxv_autotune<double>(edg_sector_s*, int, double*, int*, int*);

template int hxv_block<float>(edg_sector_s*, int, const int*, const float*, float*);
template int hxv_block<double>(edg_sector_s*, int, const int*, const double*, double*);
template int hxv_block_lz<float>(edg_sector_s*, int, const int*, const float*, const float*, float*, const double*,
                                 int64_t, int, double*, double*);
template int hxv_block_lz<double>(edg_sector_s*, int, const int*, const double*, const double*, double*,
                                  const double*, int64_t, int, double*, double*);

template int hxv_apply_lz<float>(edg_sector_s*, const float*, const float*, float*, const double*, int, double*,
                                 double*);
template int hxv_apply_lz<double>(edg_sector_s*, const double*, const double*, double*, const double*, int, double*,
                                  double*);

}  // namespace edg
