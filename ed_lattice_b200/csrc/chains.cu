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

// One warp per chain c (the chains of a block diverge from one another, so a thread per chain
// would run them one after another inside a warp): the implicit QL iteration with Wilkinson
// shifts of tridiag_eigh_host on (a[c][0..n), b[c][1..n)), rotating only the first row of the
// eigenvector matrix, then a stable sort by eigenvalue; writes poles isign*(theta_j - ei) and
// weights norm2[c] * z1_j^2 in ascending theta. The diagonal, the off-diagonal and the first
// row sit in shared memory when 3*nmax doubles fit (else in work, 3*nmax doubles per chain).
// Lane 0 runs the rotation chase (each rotation from one reciprocal square root); the warp
// finds the deflation point 32 entries at a time and ranks the eigenvalues for the sort. status[c] = 0, or 1 when
// an eigenvalue needed more than 200 sweeps (the chain's outputs are then unset).
__global__ void __launch_bounds__(32) k_poles_ql(int k, int nmax, const double* __restrict__ a,
                                                 const double* __restrict__ b, const int* __restrict__ nsteps,
                                                 const double* __restrict__ norm2, double ei, int isign,
                                                 bool in_smem, double* __restrict__ work,
                                                 double* __restrict__ poles, double* __restrict__ weights,
                                                 int* __restrict__ status) {
  extern __shared__ double smem_ql[];
  const int c = blockIdx.x;
  const int lane = threadIdx.x;
  if (c >= k) return;
  const int n = nsteps[c];
  double* dd = in_smem ? smem_ql : work + size_t(c) * 3 * nmax;
  double* sub = dd + nmax;
  double* row0 = sub + nmax;
  for (int i = lane; i < n; i += 32) {
    dd[i] = a[size_t(c) * nmax + i];
    sub[i] = i + 1 < n ? b[size_t(c) * nmax + i + 1] : 0.0;
    row0[i] = i == 0 ? 1.0 : 0.0;
  }
  __syncwarp();
  const double eps = 2.220446049250313e-16;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    for (;;) {
      // the first m >= l with a negligible sub[m] (m = n-1 when there is none)
      int m = n - 1;
      for (int base = l; base < n - 1; base += 32) {
        const int i = base + lane;
        bool hit = false;
        if (i < n - 1) hit = fabs(sub[i]) <= eps * (fabs(dd[i]) + fabs(dd[i + 1]));
        const unsigned bal = __ballot_sync(0xffffffffu, hit);
        if (bal) {
          m = base + __ffs(bal) - 1;
          break;
        }
      }
      if (m == l) break;
      if (++iter > 200) {
        if (lane == 0) status[c] = 1;
        return;
      }
      if (lane == 0) {
        double g = (dd[l + 1] - dd[l]) / (2.0 * sub[l]);
        double r = hypot(g, 1.0);
        g = dd[m] - dd[l] + sub[l] / (g + (g >= 0 ? fabs(r) : -fabs(r)));
        double s = 1.0, cc = 1.0, p = 0.0;
        bool deflated = false;
        // Software-pipelined chase: entry i-1 is loaded before the stores of step i, and the
        // values step i+1 changed (dd[i+1] still unchanged, row0[i+1] rotated) stay in
        // registers, so only the arithmetic sits on the dependent chain.
        double d1 = dd[m], z1 = row0[m];                      // dd[i+1], row0[i+1]
        double si = sub[m - 1], di = dd[m - 1], zi = row0[m - 1];
        for (int i = m - 1; i >= l; --i) {
          double sn = 0.0, dn = 0.0, zn = 0.0;
          if (i > l) {
            sn = sub[i - 1];
            dn = dd[i - 1];
            zn = row0[i - 1];
          }
          const double f = s * si, bb = cc * si;
          // the rotation (cc, s) = (g, f) / r from one reciprocal square root (a shorter
          // dependent chain than hypot and two divisions); hypot where f^2 + g^2 leaves the
          // safe exponent range
          const double t = fma(f, f, g * g);
          double rinv;
          if (t > 1e-290 && t < 1e290) {
            rinv = rsqrt(t);
            r = t * rinv;
          } else {
            r = hypot(f, g);
            rinv = 1.0 / r;
          }
          sub[i + 1] = r;
          if (r == 0.0) {
            dd[i + 1] = d1 - p;
            row0[i + 1] = z1;
            sub[m] = 0.0;
            deflated = true;
            break;
          }
          s = f * rinv;
          cc = g * rinv;
          const double gg = d1 - p;
          r = (di - gg) * s + 2.0 * cc * bb;
          p = s * r;
          dd[i + 1] = gg + p;
          g = cc * r - bb;
          row0[i + 1] = s * zi + cc * z1;
          z1 = cc * zi - s * z1;
          d1 = di;
          si = sn;
          di = dn;
          zi = zn;
        }
        if (!deflated) {
          row0[l] = z1;
          dd[l] -= p;
          sub[l] = g;
          sub[m] = 0.0;
        }
      }
      __syncwarp();
    }
  }
  // stable sort by eigenvalue: the rank of j counts the smaller values and the equal ones
  // before j, and each lane writes its eigenvalues straight to their ranks
  const double n2 = norm2[c];
  for (int j = lane; j < n; j += 32) {
    const double x = dd[j];
    int rank = 0;
    for (int i = 0; i < n; ++i) {
      const double y = dd[i];
      rank += (y < x) || (y == x && i < j);
    }
    poles[size_t(c) * nmax + rank] = isign * (x - ei);
    weights[size_t(c) * nmax + rank] = row0[j] * row0[j] * n2;
  }
  if (lane == 0) status[c] = 0;
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
  // one warp per chain; its three arrays in shared memory up to nlanc = 9,400
  const size_t smem = size_t(3) * nlanc * sizeof(double);
  const bool in_smem = smem <= size_t(227) * 1024;
  if (in_smem && smem > 48 * 1024)
    EDG_CUDA(cudaFuncSetAttribute(k_poles_ql, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  k_poles_ql<<<k, 32, in_smem ? smem : 0, st>>>(k, nlanc, da, db, dns, dn2, ei, isign, in_smem, dwork, dp, dw,
                                                dstat);
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
