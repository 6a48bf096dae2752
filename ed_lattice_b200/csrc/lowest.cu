// lowest.cu -- the lowest k eigenpairs of a sector, and the dense sector matrix.
//
// edg_lowest_k stands in for the sp_eigh (ARPACK) call of ed_diag_d
// (src/DIAG/DIAG.f90:144-146,191-202): Neigen = min(dim, lanc_nstates_sector) lowest states
// of a sector for the finite-temperature state list. Method: FP64 Lanczos with full
// reorthogonalisation against the basis kept on the device (classical Gram-Schmidt whose
// second pass comes from the Gram matrix of the basis; applied twice for complex vectors), stopped when the k lowest Ritz pairs have residual b_{m+1}|z_m,i| below
// tol*max(1,|theta_i|); the Ritz vectors are then formed in one pass over the basis.
// Single-vector Lanczos resolves one vector per eigenspace, so exactly degenerate levels
// inside one sector are found only through round-off; the dense path covers small sectors.
//
// edg_sector_dense fills the dense sector Hamiltonian the way ed_buildh(Hmat) assembles it
// (src/DIAG/HAMILTONIAN_STORED_HxV.f90:81-117): diag + kron(Hdw,1) + kron(1,Hup), for the
// lapack branch of ed_diag_d (src/DIAG/DIAG.f90:229-254).
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "common.cuh"

namespace edg {
namespace {

constexpr int kMaxBasis = 1024;   // Lanczos basis columns (multi-dot coefficients in shared memory)
constexpr int kMaxK = 16;         // eigenpairs per call
constexpr int kLkThreads = 256;
constexpr int kDenseMaxDim = 16384;  // 2 GB dense matrix

// Two right-hand sides in one read of the basis: partial[j * nsplit + s] = sum over element
// stream s of Q[j][i] * w[i], and partial[(m + j) * nsplit + s] the same for x, j < m.
// blockIdx.y takes a group of G columns and stream s = blockIdx.x * 8 + warp a contiguous run
// of elements, so every warp streams G + 2 long coalesced rows; the grid spans all column
// groups at once (about 7 blocks per SM). On the 853,776-state sector this shape reads the
// basis at 5.8-6.2 TB/s for 112-224 columns (one right-hand side), where one element chunk
// per block with the column groups shared out among its warps reached 3.3 TB/s. Fixed
// summation order.
// TQ: element type of the basis and of w, x (FP64, or FP32 for the FP32-bulk phase); the
// products and sums are FP64 either way.
template <int G, typename TQ>
__global__ void __launch_bounds__(kLkThreads) k_multidot2(const TQ* __restrict__ Q, int m, int64_t n,
                                                          const TQ* __restrict__ w, const TQ* __restrict__ x,
                                                          double* __restrict__ partial) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nsplit = gridDim.x * (kLkThreads / 32);
  const int split = blockIdx.x * (kLkThreads / 32) + warp;
  int64_t chunk = (n + nsplit - 1) / nsplit;
  chunk = (chunk + 31) & ~int64_t(31);
  const int64_t i0 = split * chunk, i1 = i0 + chunk < n ? i0 + chunk : n;
  const int j0 = blockIdx.y * G;
  const TQ* __restrict__ q[G];
#pragma unroll
  for (int c = 0; c < G; ++c) q[c] = Q + int64_t(j0 + c < m ? j0 + c : m - 1) * n;
  double aw[G], ax[G];
#pragma unroll
  for (int c = 0; c < G; ++c) aw[c] = ax[c] = 0.0;
  for (int64_t i = i0 + lane; i < i1; i += 32) {
    const double wi = double(w[i]), xi = double(x[i]);
#pragma unroll
    for (int c = 0; c < G; ++c) {
      const double qi = double(q[c][i]);
      aw[c] = __fma_rn(qi, wi, aw[c]);
      ax[c] = __fma_rn(qi, xi, ax[c]);
    }
  }
#pragma unroll
  for (int c = 0; c < G; ++c) {
    double tw = aw[c], tx = ax[c];
    for (int o = 16; o > 0; o >>= 1) {
      tw += __shfl_down_sync(0xffffffffu, tw, o);
      tx += __shfl_down_sync(0xffffffffu, tx, o);
    }
    if (lane == 0 && j0 + c < m) {
      partial[int64_t(j0 + c) * nsplit + split] = tw;
      partial[int64_t(m + j0 + c) * nsplit + split] = tx;
    }
  }
}

// Gram-corrected projection of one step (m = j + 1 basis vectors, coef = [c | g] with
// c = Q^T w and g = Q^T q_j): stores g as row and column j of the Gram matrix Gm = Q^T Q
// (leading dimension ld), writes y = c - (Gm - I) c into coef[2m..3m) and a_j = c_j. One warp
// per row, fixed order (deterministic).
__global__ void k_gram_step(double* __restrict__ coef, int m, double* __restrict__ Gm, int ld,
                            double* __restrict__ a_out) {
  const int j = m - 1;
  const double* c = coef;
  const double* g = coef + m;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
    Gm[int64_t(j) * ld + k] = g[k];
    Gm[int64_t(k) * ld + j] = g[k];
  }
  // entries of row and column j are taken from g, never from Gm, so no block depends on
  // another block's writes above
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = warp; i < m; i += nwarps) {
    double t = 0.0;
    for (int k = lane; k < m; k += 32) {
      const double gik = (k == j) ? g[i] : (i == j ? g[k] : Gm[int64_t(i) * ld + k]);
      t = __fma_rn(gik - (i == k ? 1.0 : 0.0), c[k], t);
    }
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) coef[2 * m + i] = c[i] - t;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *a_out = c[j];
}

// Gm[i][j] = (i == j) for i, j < r (leading dimension ld): the Gram matrix of a freshly
// restarted basis (Ritz vectors and the residual direction, orthonormal to rounding)
__global__ void k_gram_eye(double* __restrict__ Gm, int ld, int r) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < r * r; t += gridDim.x * blockDim.x) {
    const int i = t / r, j = t - i * r;
    Gm[int64_t(i) * ld + j] = i == j ? 1.0 : 0.0;
  }
}

constexpr int kDotBlocks = 148 * 7;  // blocks per multi-dot launch, over all column groups

// Launch shape of k_multidot for m columns of n elements: column group width, blocks per
// group (each 8 element streams of at least 32 elements).
struct DotShape {
  int G, gx;
  int nsplit() const { return gx * (kLkThreads / 32); }
};
DotShape dot_shape(int m, int64_t n) {
  DotShape d;
  d.G = m >= 64 ? 8 : 4;
  const int ngrp = (m + d.G - 1) / d.G;
  int64_t gx = (kDotBlocks + ngrp - 1) / ngrp;
  const int64_t most = std::max<int64_t>(1, n / (32 * (kLkThreads / 32)));
  d.gx = int(std::min(gx, most));
  return d;
}


template <typename TQ>
int launch_multidot2(const TQ* Q, int m, int64_t n, const TQ* w, const TQ* x, double* partial, cudaStream_t st,
                     int* nsplit) {
  const DotShape d = dot_shape(m, n);
  const dim3 grid(d.gx, (m + d.G - 1) / d.G);
  if (d.G == 8)
    k_multidot2<8, TQ><<<grid, kLkThreads, 0, st>>>(Q, m, n, w, x, partial);
  else
    k_multidot2<4, TQ><<<grid, kLkThreads, 0, st>>>(Q, m, n, w, x, partial);
  *nsplit = d.nsplit();
  return EDG_OK;
}

// Complex vectors (complex-Hij sectors, elements (re, im)): c_j = <q_j|w> = sum conj(q) w,
// real parts into partial[j * nsplit + s], imaginary parts into partial[(m + j) * nsplit + s],
// one read of the basis for both. Complex Gram-Schmidt against Q is real Gram-Schmidt against
// Q and iQ in the real embedding, so the recurrence is otherwise unchanged.
template <int G>
__global__ void __launch_bounds__(kLkThreads) k_multidot_c(const double2* __restrict__ Q, int m, int64_t n,
                                                           const double2* __restrict__ w, double* __restrict__ partial) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nsplit = gridDim.x * (kLkThreads / 32);
  const int split = blockIdx.x * (kLkThreads / 32) + warp;
  int64_t chunk = (n + nsplit - 1) / nsplit;
  chunk = (chunk + 31) & ~int64_t(31);
  const int64_t i0 = split * chunk, i1 = i0 + chunk < n ? i0 + chunk : n;
  const int j0 = blockIdx.y * G;
  const double2* __restrict__ q[G];
#pragma unroll
  for (int c = 0; c < G; ++c) q[c] = Q + int64_t(j0 + c < m ? j0 + c : m - 1) * n;
  double ar[G], ai[G];
#pragma unroll
  for (int c = 0; c < G; ++c) ar[c] = ai[c] = 0.0;
  for (int64_t i = i0 + lane; i < i1; i += 32) {
    const double2 wi = w[i];
#pragma unroll
    for (int c = 0; c < G; ++c) {
      const double2 x = q[c][i];
      ar[c] = __fma_rn(x.x, wi.x, ar[c]);
      ar[c] = __fma_rn(x.y, wi.y, ar[c]);
      ai[c] = __fma_rn(x.x, wi.y, ai[c]);
      ai[c] = __fma_rn(-x.y, wi.x, ai[c]);
    }
  }
#pragma unroll
  for (int c = 0; c < G; ++c) {
    double tr = ar[c], ti = ai[c];
    for (int o = 16; o > 0; o >>= 1) {
      tr += __shfl_down_sync(0xffffffffu, tr, o);
      ti += __shfl_down_sync(0xffffffffu, ti, o);
    }
    if (lane == 0 && j0 + c < m) {
      partial[int64_t(j0 + c) * nsplit + split] = tr;
      partial[int64_t(m + j0 + c) * nsplit + split] = ti;
    }
  }
}

int launch_multidot_c(const double* Q, int m, int64_t n, const double* w, double* partial, cudaStream_t st,
                      int* nsplit) {
  const DotShape d = dot_shape(m, n);
  const dim3 grid(d.gx, (m + d.G - 1) / d.G);
  const double2* Q2 = reinterpret_cast<const double2*>(Q);
  const double2* w2 = reinterpret_cast<const double2*>(w);
  if (d.G == 8)
    k_multidot_c<8><<<grid, kLkThreads, 0, st>>>(Q2, m, n, w2, partial);
  else
    k_multidot_c<4><<<grid, kLkThreads, 0, st>>>(Q2, m, n, w2, partial);
  *nsplit = d.nsplit();
  return EDG_OK;
}

// w[i] -= sum_j (cr[j] + i ci[j]) Q[j][i] on complex elements
__global__ void __launch_bounds__(kLkThreads) k_multiaxpy_c(const double2* __restrict__ Q, const double* __restrict__ c,
                                                            int m, int64_t n, double2* __restrict__ w) {
  __shared__ double sr[kMaxBasis], si[kMaxBasis];
  for (int j = threadIdx.x; j < m; j += blockDim.x) {
    sr[j] = c[j];
    si[j] = c[m + j];
  }
  __syncthreads();
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double2 t = w[i];
#pragma unroll 4
    for (int j = 0; j < m; ++j) {
      const double2 q = Q[int64_t(j) * n + i];
      t.x = __fma_rn(-sr[j], q.x, t.x);
      t.x = __fma_rn(si[j], q.y, t.x);
      t.y = __fma_rn(-sr[j], q.y, t.y);
      t.y = __fma_rn(-si[j], q.x, t.y);
    }
    w[i] = t;
  }
}

__global__ void k_copy1(double* __restrict__ dst, const double* __restrict__ src) { *dst = *src; }

// c[j] = sum_blk partial[j * nblk + blk], one warp per column, fixed order
__global__ void k_multifinish(const double* __restrict__ partial, int nblk, int m, double* __restrict__ c) {
  const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (j >= m) return;
  double t = 0.0;
  for (int b = lane; b < nblk; b += 32) t += partial[int64_t(j) * nblk + b];
  for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  if (lane == 0) c[j] = t;
}

// w[i] -= sum_j c[j] Q[j][i] (sums in FP64, one rounding to TQ per element)
template <typename TQ>
__global__ void __launch_bounds__(kLkThreads) k_multiaxpy(const TQ* __restrict__ Q, const double* __restrict__ c,
                                                          int m, int64_t n, TQ* __restrict__ w) {
  __shared__ double sc[kMaxBasis];
  for (int j = threadIdx.x; j < m; j += blockDim.x) sc[j] = c[j];
  __syncthreads();
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double t = double(w[i]);
#pragma unroll 8
    for (int j = 0; j < m; ++j) t = __fma_rn(-sc[j], double(Q[int64_t(j) * n + i]), t);
    w[i] = TQ(t);
  }
}

// X[r][i] = sum_j Z[j*m + r] Q[j][i], r < k (Z column-major m x m, first k columns)
template <typename TQ>
__global__ void __launch_bounds__(kLkThreads) k_ritz_k(const TQ* __restrict__ Q, const double* __restrict__ Z,
                                                       int m, int k, int64_t n, double* __restrict__ X) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double acc[kMaxK];
#pragma unroll
    for (int r = 0; r < kMaxK; ++r) acc[r] = 0.0;
    for (int j = 0; j < m; ++j) {
      const double q = double(Q[int64_t(j) * n + i]);
#pragma unroll
      for (int r = 0; r < kMaxK; ++r)
        if (r < k) acc[r] = __fma_rn(Z[j + int64_t(r) * m], q, acc[r]);
    }
#pragma unroll
    for (int r = 0; r < kMaxK; ++r)
      if (r < k) X[int64_t(r) * n + i] = acc[r];
  }
}

// Dense sector matrix, column-major H[i + j*D] (W = 2: complex, interleaved, with the
// imaginary hop values vi_*): one thread per row i = iup + idw*DimUp.
template <int W>
__global__ void k_dense(const uint32_t* __restrict__ off_up, const uint32_t* __restrict__ src_up,
                        const double* __restrict__ val_up, const double* __restrict__ vi_up,
                        const uint32_t* __restrict__ off_dw, const uint32_t* __restrict__ src_dw,
                        const double* __restrict__ val_dw, const double* __restrict__ vi_dw,
                        const double* __restrict__ e_up, const double* __restrict__ e_dw,
                        const uint32_t* __restrict__ map_up, const uint32_t* __restrict__ map_dw, double U,
                        int64_t dimup, int64_t dimdw, double* __restrict__ H) {
  const int64_t D = dimup * dimdw;
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= D) return;
  const int64_t idw = i / dimup, iup = i - idw * dimup;
  H[(i + i * D) * W] += e_up[iup] + e_dw[idw] + U * double(__popc(map_up[iup] & map_dw[idw]));
  for (uint32_t k = off_up[iup]; k < off_up[iup + 1]; ++k) {
    const int64_t j = int64_t(src_up[k]) + idw * dimup;
    H[(i + j * D) * W] += val_up[k];
    if (W == 2) H[(i + j * D) * W + W - 1] += vi_up[k];
  }
  for (uint32_t k = off_dw[idw]; k < off_dw[idw + 1]; ++k) {
    const int64_t j = iup + int64_t(src_dw[k]) * dimup;
    H[(i + j * D) * W] += val_dw[k];
    if (W == 2) H[(i + j * D) * W + W - 1] += vi_dw[k];
  }
}

int grid_n(int64_t n) {
  int64_t g = (n + kLkThreads - 1) / kLkThreads;
  return int(g < 148 * 8 ? (g < 1 ? 1 : g) : 148 * 8);
}

}  // namespace

int sector_dense_dev(edg_sector_s* s, double* dH) {
  const int64_t D = s->dim;
  if (D > kDenseMaxDim) {
    set_error("edg_sector_dense: dimension %lld above %d", (long long)D, kDenseMaxDim);
    return EDG_ERR_ARG;
  }
  if (s->form != EDG_FORM_STORED) {
    set_error("edg_sector_dense: needs the stored form (hop tables)");
    return EDG_ERR_STATE;
  }
  cudaStream_t st = s->stream;
  const int W = s->cplx ? 2 : 1;
  EDG_CUDA(cudaMemsetAsync(dH, 0, size_t(D) * D * W * sizeof(double), st));
  if (W == 2)
    k_dense<2><<<int((D + 255) / 256), 256, 0, st>>>(s->up.off.p, s->up.src.p, s->up.val64.p, s->up.val64i.p,
                                                     s->dw.off.p, s->dw.src.p, s->dw.val64.p, s->dw.val64i.p,
                                                     s->up.e64.p, s->dw.e64.p, s->up.map.p, s->dw.map.p, s->U,
                                                     s->up.dim, s->dw.dim, dH);
  else
    k_dense<1><<<int((D + 255) / 256), 256, 0, st>>>(s->up.off.p, s->up.src.p, s->up.val64.p, nullptr, s->dw.off.p,
                                                     s->dw.src.p, s->dw.val64.p, nullptr, s->up.e64.p, s->dw.e64.p,
                                                     s->up.map.p, s->dw.map.p, s->U, s->up.dim, s->dw.dim, dH);
  EDG_CUDA(cudaGetLastError());
  return EDG_OK;
}

int sector_dense(edg_sector_s* s, double* H_host) {
  const int64_t D = s->dim;
  if (D > kDenseMaxDim) {
    set_error("edg_sector_dense: dimension %lld above %d", (long long)D, kDenseMaxDim);
    return EDG_ERR_ARG;
  }
  const size_t W = s->cplx ? 2 : 1;
  DevBuf<double> Hd;
  EDG_CHECK(Hd.alloc(size_t(D) * D * W, s->stream, "dense sector matrix"));
  EDG_CHECK(sector_dense_dev(s, Hd.p));
  cudaStream_t st = s->stream;
  EDG_CUDA(cudaMemcpyAsync(H_host, Hd.p, size_t(D) * D * W * sizeof(double), cudaMemcpyDeviceToHost, st));
  EDG_CUDA(cudaStreamSynchronize(st));
  return EDG_OK;
}

namespace {

// Eigenvalues of T closer than this fraction of its spectral radius get their Ritz
// coefficients from the QL eigenvector matrix (the twisted-factorisation vectors of such a
// pair are accurate to about eps / kRitzRelGap only).
constexpr double kRitzRelGap = 1e-5;
// FP32-bulk phase: Ritz pairs to this relative residual before the FP64 refinement (FP32
// vectors carry about 1e-7 relative rounding per H x v).
constexpr double kTol32 = 1e-6;

template <typename T>
int norm_vec(cudaStream_t st, const T* x, int64_t n, double* scratch, double* out) {
  return dot_cols<T>(st, 1, x, x, n, n, scratch, out, 1, 1);
}

// One Lanczos run with full reorthogonalisation in precision T (T = float only for real
// sectors): basis Q, the tridiagonal (A, B), the residual data of the last test.
template <typename T>
struct LkRun {
  DevBuf<T> Q, w;
  DevBuf<double> part, coef, nred, Gm, dab;
  std::vector<double> A, B, zlast;
  double blast = 0.0;
  int m = 0;

  // mmax basis columns at most; start: n FP64 device values (any nonzero norm)
  int run(edg_sector_s* s, int k, const double* start, int mmax, double tol) {
    const int64_t n = s->vlen;
    const int64_t ne = s->dim;
    const bool cplx = s->cplx;
    cudaStream_t st = s->stream;
    EDG_CHECK(Q.alloc(size_t(mmax) * n, st, "Lanczos basis (lowest-k)"));
    EDG_CHECK(w.alloc(n, st, "Lanczos vector"));
    size_t npart = 1;
    for (int mm = 1; mm <= mmax; ++mm)
      npart = std::max(npart, size_t(2) * mm * dot_shape(mm, cplx ? ne : n).nsplit());
    EDG_CHECK(part.alloc(npart, st, "multi-dot partials"));
    EDG_CHECK(nred.alloc(kRedSlots, st, "norm reduction scratch"));  // the norms' own scratch
    EDG_CHECK(red_scratch_reset(st, nred.p));
    EDG_CHECK(coef.alloc(3 * size_t(mmax) + 8, st, "multi-dot coefficients"));
    if (!cplx) EDG_CHECK(Gm.alloc(size_t(mmax) * mmax, st, "Gram matrix"));  // Q^T Q
    EDG_CHECK(dab.alloc(2 * size_t(mmax) + 4, st, "Lanczos scalars"));  // a_j at [j], b_{j+1} at [mmax+1+j+1]
    double* dA = dab.p;
    double* dB = dab.p + mmax + 1;
    EDG_CHECK(norm_vec<double>(st, start, n, nred.p, dB));
    double nrm = 0.0;
    EDG_CUDA(cudaMemcpyAsync(&nrm, dB, sizeof(double), cudaMemcpyDeviceToHost, st));
    EDG_CUDA(cudaStreamSynchronize(st));
    if (!(nrm > 0.0)) {
      set_error("edg_lowest_k: start vector has zero norm");
      return EDG_ERR_ARG;
    }
    EDG_CHECK((convert_dev<T, double>(st, Q.p, start, n, 1.0 / nrm)));
    // Steps are queued without waiting on the host: the scalars stay on the device (v_{j+1}
    // = w / b_{j+1} reads b from there) and the host reads them only when it tests
    // convergence, every max(1, m/32) steps past the first k (more while far from
    // convergence). Each step reorthogonalises against the whole basis: one pass of
    // classical Gram-Schmidt lost orthogonality entirely on small sectors, and the test of
    // Daniel, Gragg, Kaufman & Stewart (Math. Comp. 30 (1976) 772) asked for the second pass
    // at nearly every step (|a_j| is well above b_j for the shifted spectra of Hubbard sectors).
    std::vector<double> hA(size_t(mmax) + 1), hB(size_t(mmax) + 2);
    int next_check = k;
    m = 0;
    for (int j = 0; j < mmax; ++j) {
      T* qj = Q.p + size_t(j) * n;
      EDG_CHECK(hxv_apply<T>(s, qj, w.p));
      if constexpr (std::is_same<T, double>::value) {
        if (cplx) {
          for (int pass = 0; pass < 2; ++pass) {
            int nsplit = 0;
            const int nc = 2 * (j + 1);  // coefficients: real parts, then imaginary parts
            EDG_CHECK(launch_multidot_c(Q.p, j + 1, ne, w.p, part.p, st, &nsplit));
            k_multifinish<<<(nc + 7) / 8, 256, 0, st>>>(part.p, nsplit, nc, coef.p);
            if (pass == 0) k_copy1<<<1, 1, 0, st>>>(dA + j, coef.p + j);  // a_j = Re <q_j, H q_j>
            k_multiaxpy_c<<<grid_n(ne), kLkThreads, 0, st>>>(reinterpret_cast<const double2*>(Q.p), coef.p, j + 1,
                                                             ne, reinterpret_cast<double2*>(w.p));
          }
        }
      }
      if (!cplx) {
        // One read of the basis gives c = Q^T w and g = Q^T q_j (row j of the Gram matrix
        // G = Q^T Q); the second Gram-Schmidt pass is taken from G instead of a second read,
        // y = c - (G - I) c, and one more read applies w -= Q y. Two reads of the basis per
        // step instead of four; on the 3x4 sectors (up to D = 853,776) the basis stays as
        // orthogonal (|Q^T Q - I| below 4e-15) and the levels agree with classical
        // Gram-Schmidt applied twice to 1e-14.
        int nsplit = 0;
        const int m1 = j + 1;
        EDG_CHECK(launch_multidot2<T>(Q.p, m1, n, w.p, qj, part.p, st, &nsplit));
        k_multifinish<<<(2 * m1 + 7) / 8, 256, 0, st>>>(part.p, nsplit, 2 * m1, coef.p);
        k_gram_step<<<(m1 + 7) / 8, 256, 0, st>>>(coef.p, m1, Gm.p, mmax, dA + j);
        k_multiaxpy<T><<<grid_n(n), kLkThreads, 0, st>>>(Q.p, coef.p + 2 * m1, m1, n, w.p);
      }
      EDG_CUDA(cudaGetLastError());
      EDG_CHECK(norm_vec<T>(st, w.p, n, nred.p, dB + j + 1));
      m = j + 1;
      if ((m >= k && m >= next_check) || m == mmax || m == ne) {
        EDG_CUDA(cudaMemcpyAsync(hA.data(), dA, size_t(m) * sizeof(double), cudaMemcpyDeviceToHost, st));
        EDG_CUDA(cudaMemcpyAsync(hB.data(), dB, size_t(m + 1) * sizeof(double), cudaMemcpyDeviceToHost, st));
        EDG_CUDA(cudaStreamSynchronize(st));
        bool last = m == mmax || m == ne;
        for (int t = 0; t < m; ++t)
          if (!(hB[t + 1] >= 1e-12)) {  // invariant subspace reached at step t (or NaN)
            m = t + 1;
            last = true;
            break;
          }
        A.assign(hA.begin(), hA.begin() + m);
        B.assign(1, 0.0);
        for (int t = 1; t < m; ++t) B.push_back(hB[t]);
        const double b = hB[m];
        auto converged = [&](const std::vector<double>& th, const std::vector<double>& zl) {
          if (m < k) return false;
          for (int i = 0; i < k; ++i)
            if (b * std::fabs(zl[i]) > tol * std::max(1.0, std::fabs(th[i]))) return false;
          return true;
        };
        // the O(k m) test between steps; the QL eigenvectors confirm it before the loop stops
        std::vector<double> th(std::max(m, k)), zl(std::max(m, k));
        bool conv = false;
        double worst = 0.0;  // largest b|z_i| / (tol max(1,|theta_i|)) over the k pairs
        if (!last && tridiag_lowest_host(m, A.data(), B.data(), std::min(k, m), th.data(), zl.data()) == EDG_OK) {
          conv = converged(th, zl);
          for (int i = 0; i < std::min(k, m); ++i)
            worst = std::max(worst, b * std::fabs(zl[i]) / (tol * std::max(1.0, std::fabs(th[i]))));
        }
        if (conv || last) {
          EDG_CHECK(tridiag_eigh_host(m, A.data(), B.data(), th.data(), nullptr, nullptr, zl.data()));
          conv = converged(th, zl);
          zlast = zl;
          blast = b;
        }
        if (conv || last) break;
        // Ritz residuals fall by a modest factor per step, so far from the tolerance the
        // next few steps run without a test (steps past convergence cost less than tests)
        int gap = std::max(1, m / 32);
        if (worst > 1e6) gap = std::max(gap, 8);
        else if (worst > 1e3) gap = std::max(gap, 3);
        next_check = m + gap;
      }
      EDG_CHECK(scale_into<T>(st, Q.p + size_t(m) * n, w.p, dB + m, n));
    }
    return EDG_OK;
  }

  // Thick-restarted Lanczos (Wu & Simon, SIAM J. Matrix Anal. Appl. 22 (2000) 602; the
  // exact-shift form of the implicit restart of ARPACK, which the reference's sp_eigh calls
  // with Ncv basis vectors): real sectors. The basis holds at most ncv columns; every step
  // is reorthogonalised against all of them as in run(), and the Gram-Schmidt coefficients
  // y = Q^T H q_j are kept, column by column, as the projected matrix Hm = Q^T H Q. When the
  // basis is full, its p lowest Ritz vectors Q z_i replace it, the residual direction w / b
  // follows them, and Hm restarts as diag(theta_i) (the coupling of the residual direction
  // to the Ritz vectors, b z_{m,i}, comes back as the Gram-Schmidt coefficients of the next
  // step). The reorthogonalisation reads at most ncv columns per step instead of the whole
  // Krylov basis. Converged when the k lowest Ritz pairs satisfy b |z_{m,i}| <= tol
  // max(1, |theta_i|), as in run().
  std::vector<double> thf, zf;  // final Ritz values and the coefficients of the k lowest
  int steps = 0;
  int run_tr(edg_sector_s* s, int k, const double* start, int maxit, int ncv, int p, double tol) {
    const int64_t n = s->vlen;
    const int64_t ne = s->dim;
    cudaStream_t st = s->stream;
    if (ncv > ne) ncv = int(ne);
    if (p > ncv - 1) p = ncv - 1;
    EDG_CHECK(Q.alloc(size_t(ncv) * n, st, "Lanczos basis (lowest-k, restarted)"));
    EDG_CHECK(w.alloc(n, st, "Lanczos vector"));
    size_t npart = 1;
    for (int mm = 1; mm <= ncv; ++mm) npart = std::max(npart, size_t(2) * mm * dot_shape(mm, n).nsplit());
    EDG_CHECK(part.alloc(npart, st, "multi-dot partials"));
    EDG_CHECK(nred.alloc(kRedSlots, st, "norm reduction scratch"));
    EDG_CHECK(red_scratch_reset(st, nred.p));
    EDG_CHECK(coef.alloc(3 * size_t(ncv) + 8, st, "multi-dot coefficients"));
    EDG_CHECK(Gm.alloc(size_t(ncv) * ncv, st, "Gram matrix"));
    EDG_CHECK(dab.alloc(2 * size_t(ncv) + 4, st, "Lanczos scalars"));
    DevBuf<double> Yc, Xr, Zd;
    EDG_CHECK(Yc.alloc(size_t(ncv) * ncv, st, "projected matrix"));
    double* dA = dab.p;           // a_j of the current cycle (scratch)
    double* dB = dab.p + ncv + 1;  // b at column position t: dB[t]
    EDG_CHECK(norm_vec<double>(st, start, n, nred.p, dB));
    double nrm = 0.0;
    EDG_CUDA(cudaMemcpyAsync(&nrm, dB, sizeof(double), cudaMemcpyDeviceToHost, st));
    EDG_CUDA(cudaStreamSynchronize(st));
    if (!(nrm > 0.0)) {
      set_error("edg_lowest_k: start vector has zero norm");
      return EDG_ERR_ARG;
    }
    EDG_CHECK((convert_dev<T, double>(st, Q.p, start, n, 1.0 / nrm)));
    std::vector<double> hY(size_t(ncv) * ncv), hb(size_t(ncv) + 2), Hm, th(ncv), Zm;
    std::vector<double> lock;  // Ritz values of the kept block
    int mcur = 1, next_check = k;
    double prev_worst = 0.0;   // the last test's worst residual ratio, its step and restart
    int prev_steps = 0, prev_lock = -1;
    steps = 0;
    for (;;) {
      const int j = mcur - 1;
      T* qj = Q.p + size_t(j) * n;
      EDG_CHECK(hxv_apply<T>(s, qj, w.p));
      int nsplit = 0;
      EDG_CHECK(launch_multidot2<T>(Q.p, mcur, n, w.p, qj, part.p, st, &nsplit));
      k_multifinish<<<(2 * mcur + 7) / 8, 256, 0, st>>>(part.p, nsplit, 2 * mcur, coef.p);
      k_gram_step<<<(mcur + 7) / 8, 256, 0, st>>>(coef.p, mcur, Gm.p, ncv, dA + j);
      k_multiaxpy<T><<<grid_n(n), kLkThreads, 0, st>>>(Q.p, coef.p + 2 * mcur, mcur, n, w.p);
      EDG_CUDA(cudaGetLastError());
      EDG_CUDA(cudaMemcpyAsync(Yc.p + size_t(j) * ncv, coef.p + 2 * mcur, size_t(mcur) * sizeof(double),
                               cudaMemcpyDeviceToDevice, st));
      EDG_CHECK(norm_vec<T>(st, w.p, n, nred.p, dB + mcur));
      ++steps;
      const bool full = mcur == ncv;
      const bool last = steps >= maxit || (mcur == ne && lock.empty());
      if ((mcur >= k && steps >= next_check) || full || last) {
        const int pl = int(lock.size());
        EDG_CUDA(cudaMemcpyAsync(hY.data(), Yc.p, size_t(mcur) * ncv * sizeof(double), cudaMemcpyDeviceToHost, st));
        EDG_CUDA(cudaMemcpyAsync(hb.data(), dB, size_t(mcur + 1) * sizeof(double), cudaMemcpyDeviceToHost, st));
        EDG_CUDA(cudaStreamSynchronize(st));
        // an invariant subspace reached at column position t (b_t ~ 0, or NaN) ends the run
        int mm = mcur;
        bool brk = false;
        for (int t = pl + 1; t <= mcur; ++t)
          if (!(hb[t] >= 1e-12)) {
            mm = t;
            brk = true;
            break;
          }
        Hm.assign(size_t(mm) * mm, 0.0);
        for (int i = 0; i < pl && i < mm; ++i) Hm[i + size_t(i) * mm] = lock[i];
        for (int c = pl; c < mm; ++c)
          for (int i = 0; i <= c; ++i) Hm[i + size_t(c) * mm] = Hm[c + size_t(i) * mm] = hY[size_t(c) * ncv + i];
        const double b = brk ? 0.0 : hb[mcur];
        const int kk = std::min(k, mm);
        auto check = [&](const double* theta, const double* zend, double* worst) {
          bool ok = mm >= k || brk;
          *worst = 0.0;
          for (int i = 0; i < kk; ++i) {
            const double r = b * std::fabs(zend[i]);
            const double lim = tol * std::max(1.0, std::fabs(theta[i]));
            if (r > lim) ok = false;
            *worst = std::max(*worst, r / lim);
          }
          return ok;
        };
        double worst = 0.0;
        bool conv = false, dense = full || last || brk || pl > 0;
        if (!dense) {
          // before the first restart Hm is the Lanczos tridiagonal: the O(k m) test between
          // steps, the dense eigenproblem only to confirm
          std::vector<double> d(mm), e(mm, 0.0), zl(kk);
          for (int c = 0; c < mm; ++c) d[c] = hY[size_t(c) * ncv + c];
          for (int c = 1; c < mm; ++c) e[c] = hY[size_t(c) * ncv + c - 1];
          if (tridiag_lowest_host(mm, d.data(), e.data(), kk, th.data(), zl.data()) == EDG_OK)
            conv = check(th.data(), zl.data(), &worst);
          else
            conv = true;  // let the dense eigenproblem decide
          dense = conv;
        }
        if (dense) {
          Zm.assign(size_t(mm) * mm, 0.0);
          EDG_CHECK(sym_eigh_host(mm, Hm.data(), th.data(), Zm.data()));
          std::vector<double> zl(kk);
          for (int i = 0; i < kk; ++i) zl[i] = Zm[size_t(mm) - 1 + size_t(i) * mm];
          conv = check(th.data(), zl.data(), &worst);
        }
        if (conv || brk || last) {
          m = mm;
          blast = b;
          thf.assign(th.begin(), th.begin() + kk);
          zf.assign(Zm.begin(), Zm.begin() + size_t(mm) * kk);
          zlast.resize(kk);
          for (int i = 0; i < kk; ++i) zlast[i] = Zm[size_t(mm) - 1 + size_t(i) * mm];
          return EDG_OK;
        }
        // next test: the residuals of Lanczos fall about geometrically, so two tests give the
        // rate and the steps still needed; the next test comes at 3/4 of them (a test costs a
        // host round trip, several steps' worth on a small sector)
        int gap = std::max(1, mcur / 32);
        if (worst > 1e6) gap = std::max(gap, 8);
        else if (worst > 1e3) gap = std::max(gap, 3);
        if (prev_worst > 0.0 && worst < prev_worst && worst > 1.0 && steps > prev_steps && pl == prev_lock) {
          const double rate = std::log(prev_worst / worst) / double(steps - prev_steps);  // per step
          const double need = std::log(worst) / rate;
          gap = std::max(gap, std::min(32, int(0.75 * need)));
        }
        prev_worst = worst;
        prev_steps = steps;
        prev_lock = pl;
        next_check = steps + gap;
        if (full) {
          // restart: X = Q Z[:, 0:pp] in FP64, then the first pp columns := X, column pp :=
          // w / b, Gm := I on the leading pp + 1 columns, Hm := diag(theta) on them
          const int pp = std::min(p, mm - 1);
          EDG_CHECK(Xr.alloc(size_t(pp) * n, st, "thick-restart Ritz vectors"));
          EDG_CHECK(Zd.alloc(size_t(mm) * pp, st, "thick-restart coefficients"));
          EDG_CUDA(cudaMemcpyAsync(Zd.p, Zm.data(), size_t(mm) * pp * sizeof(double), cudaMemcpyHostToDevice, st));
          for (int r0 = 0; r0 < pp; r0 += kMaxK) {
            const int nr = std::min(kMaxK, pp - r0);
            k_ritz_k<T><<<grid_n(n), kLkThreads, 0, st>>>(Q.p, Zd.p + size_t(r0) * mm, mm, nr, n,
                                                          Xr.p + size_t(r0) * n);
          }
          EDG_CUDA(cudaGetLastError());
          for (int r = 0; r < pp; ++r)
            EDG_CHECK((convert_dev<T, double>(st, Q.p + size_t(r) * n, Xr.p + size_t(r) * n, n, 1.0)));
          EDG_CHECK(scale_into<T>(st, Q.p + size_t(pp) * n, w.p, dB + mcur, n));
          k_gram_eye<<<((pp + 1) * (pp + 1) + 255) / 256, 256, 0, st>>>(Gm.p, ncv, pp + 1);
          EDG_CUDA(cudaGetLastError());
          EDG_CUDA(cudaStreamSynchronize(st));  // Zm (host) is read by the copy above
          lock.assign(th.begin(), th.begin() + pp);
          mcur = pp + 1;
          continue;
        }
      }
      EDG_CHECK(scale_into<T>(st, Q.p + size_t(mcur) * n, w.p, dB + mcur, n));
      ++mcur;
    }
  }
  // Ritz pairs of a run_tr() run: the kk lowest values, residual estimates b |z_m,i| and
  // (X != null) the vectors X[r] = sum_j Z[j][r] q_j in FP64 on the device
  int ritz_tr(edg_sector_s* s, int kk, double* evals, double* resid, double* X) {
    cudaStream_t st = s->stream;
    const int64_t n = s->vlen;
    for (int i = 0; i < kk; ++i) {
      evals[i] = thf[i];
      if (resid) resid[i] = blast * std::fabs(zlast[i]);
    }
    if (X) {
      DevBuf<double> Zd;
      EDG_CHECK(Zd.alloc(size_t(m) * kk, st, "Ritz coefficients"));
      EDG_CUDA(cudaMemcpyAsync(Zd.p, zf.data(), size_t(m) * kk * sizeof(double), cudaMemcpyHostToDevice, st));
      k_ritz_k<T><<<grid_n(n), kLkThreads, 0, st>>>(Q.p, Zd.p, m, kk, n, X);
      EDG_CUDA(cudaGetLastError());
      EDG_CUDA(cudaStreamSynchronize(st));
    }
    return EDG_OK;
  }

  // the kk lowest Ritz values, their residual estimates, and (X != null) the Ritz vectors
  // X[r] = sum_j Z[j][r] q_j in FP64 on the device
  int ritz(edg_sector_s* s, int kk, double* evals, double* resid, double* X) {
    const int64_t n = s->vlen;
    cudaStream_t st = s->stream;
    // the kk lowest eigenvectors of T by twisted factorisation, O(kk m), when their
    // eigenvalues stand apart; the full QL eigenvector matrix, O(m^3), when two are close
    std::vector<double> th(m), Z(size_t(m) * m);
    if (tridiag_lowest_vectors(m, A.data(), B.data(), kk, kRitzRelGap, th.data(), Z.data()) != EDG_OK)
      EDG_CHECK(tridiag_eigh_host(m, A.data(), B.data(), th.data(), nullptr, Z.data()));
    for (int i = 0; i < kk; ++i) evals[i] = th[i];
    if (resid)
      for (int i = 0; i < kk; ++i) resid[i] = blast * std::fabs(zlast[i]);
    if (X) {
      DevBuf<double> Zd;
      EDG_CHECK(Zd.alloc(size_t(m) * kk, st, "Ritz coefficients"));
      EDG_CUDA(cudaMemcpyAsync(Zd.p, Z.data(), size_t(m) * kk * sizeof(double), cudaMemcpyHostToDevice, st));
      k_ritz_k<T><<<grid_n(n), kLkThreads, 0, st>>>(Q.p, Zd.p, m, kk, n, X);
      EDG_CUDA(cudaGetLastError());
      EDG_CUDA(cudaStreamSynchronize(st));  // Z (host) is read by the copy above
    }
    return EDG_OK;
  }
};

// Basis columns of precision `elem` that fit in HBM beyond a 2 GB reserve, at most mmax.
// `kept`: FP64 vectors held next to the basis at a thick restart (0 without restarts).
int basis_room(int64_t n, size_t elem, int k, int* mmax, int kept = 0) {
  size_t fr = 0, tot = 0;
  EDG_CUDA(cudaMemGetInfo(&fr, &tot));
  const size_t reserve = size_t(2) << 30, per = size_t(n) * elem;
  // Ritz, start and restart vectors
  const size_t extra = size_t(n) * sizeof(double) * (size_t(k) + 4 + size_t(kept));
  const int64_t fit = fr > reserve + extra ? int64_t((fr - reserve - extra) / per) - 2 : 0;
  if (fit < *mmax) *mmax = int(fit);
  if (*mmax < k || *mmax < 1) {
    set_error("edg_lowest_k: %lld-element basis vectors: no room for %d of them", (long long)n, k);
    return EDG_ERR_NOMEM;
  }
  return EDG_OK;
}

}  // namespace

int lowest_k(edg_sector_s* s, int k, const double* v0_host, uint64_t seed, int maxit, double tol, int mode,
             double* evals, double* evecs_host, double* resid, int* niter) {
  const int64_t n = s->vlen;   // reals per vector
  const int64_t ne = s->dim;   // elements per vector (complex ones for complex Hij)
  cudaStream_t st = s->stream;
  if (k < 1 || k > kMaxK) {
    set_error("edg_lowest_k: k=%d outside 1..%d", k, kMaxK);
    return EDG_ERR_ARG;
  }
  for (int i = 0; i < k; ++i) {
    evals[i] = NAN;
    if (resid) resid[i] = NAN;
  }
  if (k > ne) k = int(ne);
  const int mmax0 = std::max<int>(k, int(std::min<int64_t>(std::min(maxit, kMaxBasis), ne)));
  DevBuf<double> x0;  // start vector
  EDG_CHECK(x0.alloc(size_t(n), st, "start vector"));
  if (v0_host) {
    EDG_CUDA(cudaMemcpyAsync(x0.p, v0_host, n * sizeof(double), cudaMemcpyHostToDevice, st));
  } else {
    EDG_CHECK(random_dev(st, x0.p, n, seed));
  }
  int steps32 = 0;
  if (!s->cplx) {
    // Real sectors: thick-restarted runs with the reference's basis size, Ncv = 10 k
    // (lanc_ncv_factor * Neigen, src/DIAG/DIAG.f90:144-146), at least 2k + 16; a restart keeps
    // the k + (ncv - k)/4 lowest Ritz vectors. Sectors of at most 4 Ncv states keep their
    // whole Krylov basis (no restart). The H x v applications are bounded by maxit, and by
    // no fewer than 8 Ncv (a restarted run may need more steps than the dimension).
    int ncv = int(std::min<int64_t>(ne, std::max(10 * k, 2 * k + 16)));
    if (ne <= 4 * int64_t(ncv)) ncv = int(ne);
    const int steps_max = std::max({maxit, k, 8 * ncv});
    if (mode == EDG_LK_F32_REFINE) {
      // FP32-bulk phase to residuals kTol32; its k Ritz vectors, summed, start the FP64 run
      DevBuf<double> X;
      EDG_CHECK(X.alloc(size_t(k) * n, st, "FP32 Ritz vectors"));
      {
        int nc = ncv;
        EDG_CHECK(basis_room(n, sizeof(float), k, &nc, k + (nc - k) / 4));
        LkRun<float> r32;
        EDG_CHECK(r32.run_tr(s, k, x0.p, steps_max, nc, k + (nc - k) / 4, std::max(tol, kTol32)));
        steps32 = r32.steps;
        const int k32 = int(r32.thf.size());
        std::vector<double> ev(k32), rs(k32);
        EDG_CHECK(r32.ritz_tr(s, k32, ev.data(), rs.data(), X.p));
        EDG_CUDA(cudaMemsetAsync(x0.p, 0, n * sizeof(double), st));
        for (int r = 0; r < k32; ++r) EDG_CHECK(axpy_accum_dev<double>(st, x0.p, X.p + size_t(r) * n, 1.0, n));
      }  // the FP32 basis goes back to the pool before the FP64 one is taken
    }
    EDG_CHECK(basis_room(n, sizeof(double), k, &ncv, ncv < ne ? k + (ncv - k) / 4 : 0));
    LkRun<double> r64;
    EDG_CHECK(r64.run_tr(s, k, x0.p, steps_max, ncv, k + (ncv - k) / 4, tol));
    if (niter) *niter = steps32 + r64.steps;
    const int kk = int(r64.thf.size());
    DevBuf<double> X;
    if (evecs_host) EDG_CHECK(X.alloc(size_t(kk) * n, st, "Ritz vectors"));
    EDG_CHECK(r64.ritz_tr(s, kk, evals, resid, evecs_host ? X.p : nullptr));
    if (evecs_host) {
      EDG_CUDA(cudaMemcpyAsync(evecs_host, X.p, size_t(kk) * n * sizeof(double), cudaMemcpyDeviceToHost, st));
      EDG_CUDA(cudaStreamSynchronize(st));
    }
    return EDG_OK;
  }
  // complex sectors: one unrestarted run with the whole Krylov basis (Gram-Schmidt applied twice)
  int mmax = mmax0;
  EDG_CHECK(basis_room(n, sizeof(double), k, &mmax));
  LkRun<double> r64;
  EDG_CHECK(r64.run(s, k, x0.p, mmax, tol));
  if (niter) *niter = r64.m;
  const int kk = std::min(k, r64.m);
  DevBuf<double> X;
  if (evecs_host) EDG_CHECK(X.alloc(size_t(kk) * n, st, "Ritz vectors"));
  EDG_CHECK(r64.ritz(s, kk, evals, resid, evecs_host ? X.p : nullptr));
  if (evecs_host) {
    EDG_CUDA(cudaMemcpyAsync(evecs_host, X.p, size_t(kk) * n * sizeof(double), cudaMemcpyDeviceToHost, st));
    EDG_CUDA(cudaStreamSynchronize(st));
  }
  return EDG_OK;
}

}  // namespace edg
