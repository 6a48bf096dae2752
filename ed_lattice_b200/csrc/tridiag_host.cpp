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

namespace {

constexpr int kLanes = 8;

// Number of eigenvalues below each x[p]: negative pivots of the LDL^T factorisation of
// T - x[p] I, with a pivot smaller than pivmin in magnitude replaced by -pivmin.
void sturm_counts(int n, const double* d, const double* e2, const double* x, double pivmin, int* cnt) {
  double q[kLanes];
  for (int p = 0; p < kLanes; ++p) {
    double t = d[0] - x[p];
    if (std::fabs(t) < pivmin) t = -pivmin;
    q[p] = t;
    cnt[p] = t < 0 ? 1 : 0;
  }
  for (int i = 1; i < n; ++i) {
    const double di = d[i], ei = e2[i];
    for (int p = 0; p < kLanes; ++p) {
      double t = di - x[p] - ei / q[p];
      if (std::fabs(t) < pivmin) t = -pivmin;
      q[p] = t;
      cnt[p] += t < 0 ? 1 : 0;
    }
  }
}

// Unit eigenvector z[n] of T for the eigenvalue th from a twisted factorisation of T - th I:
// top-down pivots D+ and bottom-up pivots R-, twist index r minimising
// |gamma_r| = |D+_r + R-_r - (d_r - th)|, then z_r = 1 and the two bidiagonal solves outward
// (Parlett & Dhillon, Linear Algebra Appl. 267 (1997) 247). Its error is about
// eps * |T| / gap for an eigenvalue at distance gap from the rest of the spectrum.
int twisted_vector(int n, const double* d, const double* e, const double* e2, double th, double pivmin,
                   double* dp, double* rm, double* z) {
  auto guard = [pivmin](double q) { return std::fabs(q) < pivmin ? -pivmin : q; };
  dp[0] = guard(d[0] - th);
  for (int i = 1; i < n; ++i) dp[i] = guard(d[i] - th - e2[i] / dp[i - 1]);
  rm[n - 1] = guard(d[n - 1] - th);
  for (int i = n - 2; i >= 0; --i) rm[i] = guard(d[i] - th - e2[i + 1] / rm[i + 1]);
  int r = 0;
  double gmin = std::numeric_limits<double>::infinity();
  for (int i = 0; i < n; ++i) {
    const double g = std::fabs(dp[i] + rm[i] - (d[i] - th));
    if (g < gmin) {
      gmin = g;
      r = i;
    }
  }
  z[r] = 1.0;
  for (int i = r - 1; i >= 0; --i) z[i] = -(e[i + 1] / dp[i]) * z[i + 1];
  for (int i = r + 1; i < n; ++i) z[i] = -(e[i] / rm[i]) * z[i - 1];
  double nrm = 0.0;
  for (int i = 0; i < n; ++i) nrm += z[i] * z[i];
  if (!(nrm > 0.0) || !std::isfinite(nrm)) {
    set_error("twisted factorisation overflowed at eigenvalue %.17g", th);
    return EDG_ERR_NOCONV;
  }
  const double inv = 1.0 / std::sqrt(nrm);
  for (int i = 0; i < n; ++i) z[i] *= inv;
  return EDG_OK;
}

// Lowest k eigenvalues of T (d[n], e[n] with e[i] between i-1 and i) in ascending order by
// bisection on Sturm counts, from the Gerschgorin interval down to a width of a few ulps.
// e2 receives e^2; returns pivmin through *pm and the spectral radius bound through *span.
void bisect_lowest(int n, const double* d, const double* e, int k, double* w, std::vector<double>& e2, double* pm,
                   double* span_out) {
  const double eps = std::numeric_limits<double>::epsilon();
  e2.assign(n, 0.0);
  double lo = d[0], hi = d[0], emax2 = 0.0;
  for (int i = 0; i < n; ++i) {
    const double r = (i > 0 ? std::fabs(e[i]) : 0.0) + (i + 1 < n ? std::fabs(e[i + 1]) : 0.0);
    lo = std::min(lo, d[i] - r);
    hi = std::max(hi, d[i] + r);
    if (i > 0) {
      e2[i] = e[i] * e[i];
      emax2 = std::max(emax2, e2[i]);
    }
  }
  const double pivmin = std::max(std::numeric_limits<double>::min(), emax2 * std::numeric_limits<double>::min());
  const double span = std::max(std::fabs(lo), std::fabs(hi));
  lo -= 2.0 * eps * span + pivmin;
  hi += 2.0 * eps * span + pivmin;
  // the k bisections advance together, kLanes Sturm recurrences interleaved per pass over T
  // so that their divisions overlap
  for (int j0 = 0; j0 < k; j0 += kLanes) {
    const int nl = std::min(kLanes, k - j0);
    double a[kLanes], b[kLanes], x[kLanes];
    int cnt[kLanes];
    for (int p = 0; p < kLanes; ++p) {
      a[p] = lo;
      b[p] = hi;
    }
    for (int it = 0; it < 200; ++it) {
      bool active = false;
      for (int p = 0; p < kLanes; ++p) {
        x[p] = 0.5 * (a[p] + b[p]);
        const bool open = p < nl && x[p] > a[p] && x[p] < b[p] &&
                          b[p] - a[p] > 2.0 * eps * std::max(std::fabs(a[p]), std::fabs(b[p])) + pivmin;
        if (open) active = true;
        else x[p] = b[p];  // a settled lane keeps counting, harmlessly, at its upper end
      }
      if (!active) break;
      sturm_counts(n, d, e2.data(), x, pivmin, cnt);
      for (int p = 0; p < nl; ++p) {
        if (x[p] == b[p]) continue;
        if (cnt[p] >= j0 + p + 1)
          b[p] = x[p];
        else
          a[p] = x[p];
      }
    }
    for (int p = 0; p < nl; ++p) w[j0 + p] = 0.5 * (a[p] + b[p]);
  }
  *pm = pivmin;
  *span_out = span;
}

}  // namespace

// k lowest eigenvalues ascending and |last component| of each unit eigenvector, O(k n);
// used to test Lanczos convergence on the k lowest Ritz pairs between steps.
int tridiag_lowest_host(int n, const double* d, const double* e, int k, double* w, double* zn) {
  if (n <= 0 || k <= 0) return EDG_OK;
  if (k > n) k = n;
  std::vector<double> e2;
  double pivmin = 0.0, span = 0.0;
  bisect_lowest(n, d, e, k, w, e2, &pivmin, &span);
  if (!zn) return EDG_OK;
  std::vector<double> dp(n), rm(n), z(n);
  for (int j = 0; j < k; ++j) {
    EDG_CHECK(twisted_vector(n, d, e, e2.data(), w[j], pivmin, dp.data(), rm.data(), z.data()));
    zn[j] = std::fabs(z[n - 1]);
  }
  return EDG_OK;
}

// k lowest eigenpairs: w[k] ascending, z[k][n] (column j of an n x k column-major matrix,
// leading dimension n) unit eigenvectors. Refuses (EDG_ERR_NOCONV) when one of these
// eigenvalues lies within relgap * spectral radius of another, where the vectors of a
// twisted factorisation lose orthogonality; the caller then takes the QL eigenvectors.
int tridiag_lowest_vectors(int n, const double* d, const double* e, int k, double relgap, double* w, double* z) {
  if (n <= 0 || k <= 0) return EDG_OK;
  if (k > n) k = n;
  const int kb = std::min(k + 1, n);  // one more eigenvalue for the gap above the k-th
  std::vector<double> wb(kb), e2;
  double pivmin = 0.0, span = 0.0;
  bisect_lowest(n, d, e, kb, wb.data(), e2, &pivmin, &span);
  const double mingap = relgap * std::max(span, std::numeric_limits<double>::min());
  for (int j = 0; j + 1 < kb; ++j)
    if (wb[j + 1] - wb[j] < mingap) {
      set_error("tridiag_lowest_vectors: eigenvalues %d and %d closer than %.3g", j, j + 1, mingap);
      return EDG_ERR_NOCONV;
    }
  std::vector<double> dp(n), rm(n);
  for (int j = 0; j < k; ++j) {
    w[j] = wb[j];
    EDG_CHECK(twisted_vector(n, d, e, e2.data(), w[j], pivmin, dp.data(), rm.data(), z + size_t(j) * n));
  }
  return EDG_OK;
}

// Dense symmetric eigenproblem of a small matrix (the projected matrix of a thick-restarted
// Lanczos run, n up to a few dozen): Householder reduction to tridiagonal form T = P^T A P
// (reflectors H = I - beta v v^T applied from both sides, P accumulated), the implicit QL
// above on T, then the eigenvectors P Z_T. A: column-major n x n (only symmetric use); w[n]
// ascending; Z column-major n x n.
int sym_eigh_host(int n, const double* A, double* w, double* Z) {
  if (n <= 0) return EDG_OK;
  std::vector<double> a(A, A + size_t(n) * n), P(size_t(n) * n, 0.0), v(n), pv(n), qv(n);
  for (int i = 0; i < n; ++i) P[i + size_t(i) * n] = 1.0;
  auto at = [&](int i, int j) -> double& { return a[i + size_t(j) * n]; };
  for (int kcol = 0; kcol + 2 < n; ++kcol) {
    // reflector that zeroes a[kcol+2..n-1][kcol]
    double sig = 0.0;
    for (int i = kcol + 1; i < n; ++i) sig += at(i, kcol) * at(i, kcol);
    const double x0 = at(kcol + 1, kcol);
    const double alpha = -std::copysign(std::sqrt(sig), x0);
    if (sig == 0.0 || sig - x0 * x0 == 0.0) continue;  // column already reduced
    std::fill(v.begin(), v.end(), 0.0);
    for (int i = kcol + 1; i < n; ++i) v[i] = at(i, kcol);
    v[kcol + 1] -= alpha;
    double vv = 0.0;
    for (int i = kcol + 1; i < n; ++i) vv += v[i] * v[i];
    const double beta = 2.0 / vv;
    // A <- H A H with p = beta A v, q = p - (beta/2)(v^T p) v: A <- A - v q^T - q v^T
    for (int i = 0; i < n; ++i) {
      double t = 0.0;
      for (int j = kcol + 1; j < n; ++j) t += at(i, j) * v[j];
      pv[i] = beta * t;
    }
    double vp = 0.0;
    for (int i = kcol + 1; i < n; ++i) vp += v[i] * pv[i];
    for (int i = 0; i < n; ++i) qv[i] = pv[i] - 0.5 * beta * vp * v[i];
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) at(i, j) -= v[i] * qv[j] + qv[i] * v[j];
    // P <- P H
    for (int i = 0; i < n; ++i) {
      double t = 0.0;
      for (int j = kcol + 1; j < n; ++j) t += P[i + size_t(j) * n] * v[j];
      t *= beta;
      for (int j = kcol + 1; j < n; ++j) P[i + size_t(j) * n] -= t * v[j];
    }
  }
  std::vector<double> d(n), e(n, 0.0), zt(size_t(n) * n);
  for (int i = 0; i < n; ++i) d[i] = at(i, i);
  for (int i = 1; i < n; ++i) e[i] = 0.5 * (at(i, i - 1) + at(i - 1, i));
  EDG_CHECK(tridiag_eigh_host(n, d.data(), e.data(), w, nullptr, zt.data()));
  for (int c = 0; c < n; ++c)
    for (int i = 0; i < n; ++i) {
      double t = 0.0;
      for (int j = 0; j < n; ++j) t += P[i + size_t(j) * n] * zt[j + size_t(c) * n];
      Z[i + size_t(c) * n] = t;
    }
  return EDG_OK;
}

}  // namespace edg
