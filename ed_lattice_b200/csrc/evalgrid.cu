// evalgrid.cu -- pole sums on frequency grids.
//
// The evaluation loops of lanc_eval_gf_electrons (src/GF/GF_ELECTRONS.f90:503-508):
// G(z_m) = sum_k w_k / (z_m - p_k) over every pole of every state, channel and chain that
// contributes to one Green's function entry, for the Matsubara axis (z = i w_n) and the real
// axis (z = w + i eps). With a few hundred thousand poles and ~10^4 frequencies this is 10^9
// complex divisions: a grid of (frequency block, pole chunk) CTAs writes per-chunk partial
// sums, and a second pass adds the chunks in fixed order (deterministic).
#include "common.cuh"

namespace edg {
namespace {

constexpr int kEvalThreads = 256;
constexpr int kEvalChunks = 64;   // pole chunks (second grid dimension)
constexpr int kEvalTile = 1024;   // poles staged in shared memory at a time

__global__ void __launch_bounds__(kEvalThreads) k_eval_poles(const double* __restrict__ poles,
                                                             const double* __restrict__ weights, int64_t npoles,
                                                             const double* __restrict__ zr,
                                                             const double* __restrict__ zi, int64_t nz,
                                                             double* __restrict__ part) {
  __shared__ double sp[kEvalTile], sw[kEvalTile];
  const int64_t m = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  const int64_t per = (npoles + gridDim.y - 1) / gridDim.y;
  const int64_t k0 = blockIdx.y * per, k1 = k0 + per < npoles ? k0 + per : npoles;
  const double x = m < nz ? zr[m] : 0.0, y = m < nz ? zi[m] : 0.0;
  double re = 0.0, im = 0.0;
  for (int64_t t0 = k0; t0 < k1; t0 += kEvalTile) {
    const int cnt = int(k1 - t0 < kEvalTile ? k1 - t0 : kEvalTile);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
      sp[q] = poles[t0 + q];
      sw[q] = weights[t0 + q];
    }
    __syncthreads();
    for (int q = 0; q < cnt; ++q) {
      const double d = x - sp[q];
      const double s = sw[q] / __fma_rn(d, d, y * y);
      re = __fma_rn(s, d, re);
      im = __fma_rn(-s, y, im);
    }
  }
  if (m < nz) {
    part[(int64_t(blockIdx.y) * nz + m) * 2] = re;
    part[(int64_t(blockIdx.y) * nz + m) * 2 + 1] = im;
  }
}

__global__ void k_eval_sum(const double* __restrict__ part, int nchunks, int64_t nz, double* __restrict__ out) {
  const int64_t m = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (m >= nz) return;
  double re = 0.0, im = 0.0;
  for (int c = 0; c < nchunks; ++c) {
    re += part[(int64_t(c) * nz + m) * 2];
    im += part[(int64_t(c) * nz + m) * 2 + 1];
  }
  out[2 * m] = re;
  out[2 * m + 1] = im;
}

}  // namespace

int eval_poles(int64_t npoles, const double* poles, const double* weights, int64_t nz, const double* z_re,
               const double* z_im, double* out_re, double* out_im) {
  if (npoles == 0 || nz == 0) return EDG_OK;
  int dev = 0;
  EDG_CUDA(cudaGetDevice(&dev));
  cudaStream_t st = nullptr;
  EDG_CUDA(pooled_stream(dev, &st));
  DevBuf<double> dp, dw, dzr, dzi, part, out;
  EDG_CHECK(dp.alloc(npoles, st, "poles"));
  EDG_CHECK(dw.alloc(npoles, st, "weights"));
  EDG_CHECK(dzr.alloc(nz, st, "frequencies"));
  EDG_CHECK(dzi.alloc(nz, st, "frequencies"));
  const int chunks = int(npoles < kEvalChunks ? npoles : kEvalChunks);
  EDG_CHECK(part.alloc(size_t(chunks) * nz * 2, st, "pole-sum partials"));
  EDG_CHECK(out.alloc(size_t(nz) * 2, st, "pole sums"));
  EDG_CUDA(cudaMemcpyAsync(dp.p, poles, npoles * sizeof(double), cudaMemcpyHostToDevice, st));
  EDG_CUDA(cudaMemcpyAsync(dw.p, weights, npoles * sizeof(double), cudaMemcpyHostToDevice, st));
  EDG_CUDA(cudaMemcpyAsync(dzr.p, z_re, nz * sizeof(double), cudaMemcpyHostToDevice, st));
  EDG_CUDA(cudaMemcpyAsync(dzi.p, z_im, nz * sizeof(double), cudaMemcpyHostToDevice, st));
  dim3 grid(unsigned((nz + kEvalThreads - 1) / kEvalThreads), unsigned(chunks));
  k_eval_poles<<<grid, kEvalThreads, 0, st>>>(dp.p, dw.p, npoles, dzr.p, dzi.p, nz, part.p);
  k_eval_sum<<<unsigned((nz + 255) / 256), 256, 0, st>>>(part.p, chunks, nz, out.p);
  EDG_CUDA(cudaGetLastError());
  std::vector<double> h(size_t(nz) * 2);
  EDG_CUDA(cudaMemcpyAsync(h.data(), out.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  EDG_CUDA(cudaStreamSynchronize(st));
  for (int64_t m = 0; m < nz; ++m) {
    out_re[m] += h[2 * m];
    out_im[m] += h[2 * m + 1];
  }
  return EDG_OK;
}

}  // namespace edg
