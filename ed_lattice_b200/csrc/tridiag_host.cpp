// tridiag_host.cpp -- FP64 symmetric tridiagonal eigensolver on the host.
//
// Stands in for SciFortran's eigh(diag,subdiag,Ev=Z) as called by the GF/CHI/OC builders
// (src/GF/GF_ELECTRONS.f90:447, src/CHI/CHI_SPIN_ELECTRONS.f90:330,
// src/OC/OC_ELECTRONS.f90:250). Method: implicit QL iteration with Wilkinson shifts
// (Bowdler, Martin, Reinsch & Wilkinson, Numer. Math. 11 (1968) 293), applying each plane
// rotation either to the full eigenvector matrix or only to its first row, which is all the
// pole weights Z(1,j)^2 need. Chains are at most a few hundred long, so this is cheap next to
// one H x v of any sector worth a GPU.
#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <vector>

#include "common.cuh"

namespace edg {

// d[n] diagonal, e[n] couplings with e[k] between k-1 and k (e[0] ignored).
// w[n] eigenvalues ascending; z1[n] (optional) first components; zfull[n*n] (optional)
// column-major eigenvectors, column j for w[j].
int tridiag_eigh_host(int n, const double* d, const double* e, double* w, double* z1, double* zfull, double* zn) {
  if (n <= 0) return EDG_OK;
  std::vector<double> dd(d, d + n), sub(n, 0.0);
  for (int i = 0; i + 1 < n; ++i) sub[i] = e[i + 1];
  const bool full = zfull != nullptr;
  std::vector<double> Z;
  std::vector<double> row0(n, 0.0), rowl(n, 0.0);  // first and last rows of Z
  if (full) {
    Z.assign(size_t(n) * n, 0.0);
    for (int i = 0; i < n; ++i) Z[i + size_t(i) * n] = 1.0;
  } else {
    row0[0] = 1.0;
    rowl[n - 1] = 1.0;
  }
  const double eps = std::numeric_limits<double>::epsilon();
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    for (;;) {
      int m = l;
      for (; m < n - 1; ++m) {
        const double scale = std::fabs(dd[m]) + std::fabs(dd[m + 1]);
        if (std::fabs(sub[m]) <= eps * scale) break;
      }
      if (m == l) break;
      if (++iter > 200) {
        set_error("tridiagonal QL: no convergence at index %d", l);
        return EDG_ERR_NOCONV;
      }
      double g = (dd[l + 1] - dd[l]) / (2.0 * sub[l]);
      double r = std::hypot(g, 1.0);
      g = dd[m] - dd[l] + sub[l] / (g + (g >= 0 ? std::fabs(r) : -std::fabs(r)));
      double s = 1.0, c = 1.0, p = 0.0;
      bool deflated = false;
      for (int i = m - 1; i >= l; --i) {
        const double f = s * sub[i], b = c * sub[i];
        r = std::hypot(f, g);
        sub[i + 1] = r;
        if (r == 0.0) {
          dd[i + 1] -= p;
          sub[m] = 0.0;
          deflated = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = dd[i + 1] - p;
        r = (dd[i] - g) * s + 2.0 * c * b;
        p = s * r;
        dd[i + 1] = g + p;
        g = c * r - b;
        if (full) {
          double* zi = &Z[size_t(i) * n];
          double* zj = &Z[size_t(i + 1) * n];
          for (int k = 0; k < n; ++k) {
            const double t = zj[k];
            zj[k] = s * zi[k] + c * t;
            zi[k] = c * zi[k] - s * t;
          }
        } else {
          const double t = row0[i + 1];
          row0[i + 1] = s * row0[i] + c * t;
          row0[i] = c * row0[i] - s * t;
          if (zn) {
            const double tl = rowl[i + 1];
            rowl[i + 1] = s * rowl[i] + c * tl;
            rowl[i] = c * rowl[i] - s * tl;
          }
        }
      }
      if (deflated) continue;
      dd[l] -= p;
      sub[l] = g;
      sub[m] = 0.0;
    }
  }
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return dd[a] < dd[b]; });
  for (int j = 0; j < n; ++j) {
    w[j] = dd[idx[j]];
    if (z1) z1[j] = full ? Z[0 + size_t(idx[j]) * n] : row0[idx[j]];
    if (zn) zn[j] = full ? Z[size_t(n - 1) + size_t(idx[j]) * n] : rowl[idx[j]];
    if (full)
      for (int k = 0; k < n; ++k) zfull[k + size_t(j) * n] = Z[k + size_t(idx[j]) * n];
  }
  return EDG_OK;
}

}  // namespace edg
