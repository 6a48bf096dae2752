// chains.cu -- response-function chains in blocks: k excitation vectors of one target
// sector tridiagonalised together (block H x V, tridiag_block) and their poles and weights
// computed on the device.
//
// The reference builds one chain per state x site x spin x {particle, hole} and calls
// add_to_lanczos_gf_normal / add_to_lanczos_spinChi on each (src/GF/GF_ELECTRONS.f90:202-290,
// :417-457; src/CHI/CHI_SPIN_ELECTRONS.f90:189-233, :305-366): the tridiagonal eigenproblem
// of every chain, weight norm2 * Z(1,j)^2 and pole isign * (theta_j - E_i). Here the chains of
// one sector run as one block and the eigenproblems of the block run as one launch.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace edg {
namespace {

// One thread per chain c: the implicit QL iteration with Wilkinson shifts of tridiag_eigh_host
// on (a[c][0..n), b[c][1..n)), rotating only the first row of the eigenvector matrix, then an
// insertion sort by eigenvalue; writes poles isign*(theta_j - ei) and weights
// norm2[c] * z1_j^2 in ascending theta. work: 3*nmax doubles per chain. status[c] = 0, or 1
// when an eigenvalue needed more than 200 sweeps (the chain's outputs are then unset).
__global__ void k_poles_ql(int k, int nmax, const double* __restrict__ a, const double* __restrict__ b,
                           const int* __restrict__ nsteps, const double* __restrict__ norm2, double ei, int isign,
                           double* __restrict__ work, double* __restrict__ poles, double* __restrict__ weights,
                           int* __restrict__ status) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= k) return;
  const int n = nsteps[c];
  double* dd = work + size_t(c) * 3 * nmax;
  double* sub = dd + nmax;
  double* row0 = sub + nmax;
  for (int i = 0; i < n; ++i) {
    dd[i] = a[size_t(c) * nmax + i];
    sub[i] = i + 1 < n ? b[size_t(c) * nmax + i + 1] : 0.0;
    row0[i] = i == 0 ? 1.0 : 0.0;
  }
  status[c] = 0;
  const double eps = 2.220446049250313e-16;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    for (;;) {
      int m = l;
      for (; m < n - 1; ++m) {
        const double scale = fabs(dd[m]) + fabs(dd[m + 1]);
        if (fabs(sub[m]) <= eps * scale) break;
      }
      if (m == l) break;
      if (++iter > 200) {
        status[c] = 1;
        return;
      }
      double g = (dd[l + 1] - dd[l]) / (2.0 * sub[l]);
      double r = hypot(g, 1.0);
      g = dd[m] - dd[l] + sub[l] / (g + (g >= 0 ? fabs(r) : -fabs(r)));
      double s = 1.0, cc = 1.0, p = 0.0;
      bool deflated = false;
      for (int i = m - 1; i >= l; --i) {
        const double f = s * sub[i], bb = cc * sub[i];
        r = hypot(f, g);
        sub[i + 1] = r;
        if (r == 0.0) {
          dd[i + 1] -= p;
          sub[m] = 0.0;
          deflated = true;
          break;
        }
        s = f / r;
        cc = g / r;
        g = dd[i + 1] - p;
        r = (dd[i] - g) * s + 2.0 * cc * bb;
        p = s * r;
        dd[i + 1] = g + p;
        g = cc * r - bb;
        const double t = row0[i + 1];
        row0[i + 1] = s * row0[i] + cc * t;
        row0[i] = cc * row0[i] - s * t;
      }
      if (deflated) continue;
      dd[l] -= p;
      sub[l] = g;
      sub[m] = 0.0;
    }
  }
  // stable insertion sort by eigenvalue (the order of equal values is kept)
  for (int i = 1; i < n; ++i) {
    const double x = dd[i], z = row0[i];
    int j = i - 1;
    while (j >= 0 && dd[j] > x) {
      dd[j + 1] = dd[j];
      row0[j + 1] = row0[j];
      --j;
    }
    dd[j + 1] = x;
    row0[j + 1] = z;
  }
  const double n2 = norm2[c];
  for (int j = 0; j < n; ++j) {
    poles[size_t(c) * nmax + j] = isign * (dd[j] - ei);
    weights[size_t(c) * nmax + j] = row0[j] * row0[j] * n2;
  }
}

// Poles and weights of k chains whose coefficients are on the host ([k][nlanc], the
// reference's blanc(1)-unused convention): one H2D copy, one launch, one D2H copy.
int poles_weights_block(cudaStream_t st, int k, int nlanc, const double* alanc, const double* blanc,
                        const double* norm2, const int* nsteps, double ei, int isign, double* poles,
                        double* weights) {
  if (k <= 0 || nlanc <= 0) return EDG_OK;
  const size_t kn = size_t(k) * nlanc;
  DevBuf<double> buf;
  EDG_CHECK(buf.alloc(7 * kn + k, st, "chain eigenproblems"));
  double* da = buf.p;
  double* db = da + kn;
  double* dwork = db + kn;
  double* dp = dwork + 3 * kn;
  double* dw = dp + kn;
  double* dn2 = dw + kn;
  DevBuf<int> ibuf;
  EDG_CHECK(ibuf.alloc(2 * size_t(k), st, "chain eigenproblems"));
  int* dns = ibuf.p;
  int* dstat = dns + k;
  EDG_CUDA(cudaMemcpyAsync(da, alanc, kn * sizeof(double), cudaMemcpyHostToDevice, st));
  EDG_CUDA(cudaMemcpyAsync(db, blanc, kn * sizeof(double), cudaMemcpyHostToDevice, st));
  EDG_CUDA(cudaMemcpyAsync(dn2, norm2, k * sizeof(double), cudaMemcpyHostToDevice, st));
  EDG_CUDA(cudaMemcpyAsync(dns, nsteps, k * sizeof(int), cudaMemcpyHostToDevice, st));
  k_poles_ql<<<(k + 31) / 32, 32, 0, st>>>(k, nlanc, da, db, dns, dn2, ei, isign, dwork, dp, dw, dstat);
  EDG_CUDA(cudaGetLastError());
  std::vector<int> stat(k);
  EDG_CUDA(cudaMemcpyAsync(poles, dp, kn * sizeof(double), cudaMemcpyDeviceToHost, st));
  EDG_CUDA(cudaMemcpyAsync(weights, dw, kn * sizeof(double), cudaMemcpyDeviceToHost, st));
  EDG_CUDA(cudaMemcpyAsync(stat.data(), dstat, k * sizeof(int), cudaMemcpyDeviceToHost, st));
  EDG_CUDA(cudaStreamSynchronize(st));
  for (int c = 0; c < k; ++c)
    if (stat[c]) {
      set_error("tridiagonal QL: no convergence in chain %d", c);
      return EDG_ERR_NOCONV;
    }
  return EDG_OK;
}

}  // namespace

int chains_block(edg_sector_s* to, int k, const StartFn& start, int nlanc, int precision, double ei, int isign,
                 double* poles, double* weights, double* norm2, int* nout) {
  std::vector<double> a(size_t(k) * nlanc), b(size_t(k) * nlanc);
  EDG_CHECK(tridiag_block_fn(to, k, start, nlanc, 1e-9, precision, a.data(), b.data(), norm2, nout));
  return poles_weights_block(to->stream, k, nlanc, a.data(), b.data(), norm2, nout, ei, isign, poles, weights);
}

int poles_block(cudaStream_t st, int k, int nlanc, const double* alanc, const double* blanc, const double* norm2,
                const int* nsteps, double ei, int isign, double* poles, double* weights) {
  return poles_weights_block(st, k, nlanc, alanc, blanc, norm2, nsteps, ei, isign, poles, weights);
}

}  // namespace edg
