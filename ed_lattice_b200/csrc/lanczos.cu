// lanczos.cu -- device Lanczos drivers.
//
// tridiag_dev : tridiag_Hv_sector (src/DIAG/HAMILTONIAN.f90:242-275) + sp_lanc_tridiag.
// ground_state: the ground-state solve of ed_diag_d with lanc_method="lanczos"
//               (src/DIAG/DIAG.f90:206-218, sp_lanc_eigh), in two modes:
//   EDG_GS_F64        plain FP64 Lanczos; the eigenvector is rebuilt by a second pass of
//                     the (bit-reproducible) recurrence;
//   EDG_GS_F32_REFINE FP32 vectors with FP64 scalars until the lowest Ritz value settles at
//                     FP32 resolution, FP32 Ritz vector accumulated in FP64 from the stored
//                     FP32 basis, then restarted FP64 Lanczos from it to the requested tol.
//
// The recurrence (w = H v_j - b_j v_{j-1}; a_j = <v_j|w>; u_{j+1} = w - a_j v_j;
// b_{j+1} = |u_{j+1}|) runs in one of two forms with identical mathematics:
//  * fused (stored-form sectors whose passes take the shared-memory/grouped kernels): the
//    vectors are kept unnormalised, u_j = b_j v_j, the scale 1/b_j is folded into the matrix
//    elements of the H x v, whose second pass also forms w and the partial <v_j|w>; one more
//    pass forms u_{j+1} and its norm. About 9 vector-lengths of traffic per step.
//  * general: H x v, then w/a, u/b and v_{j+1} = u/b as three passes (14 vector-lengths).
// Scalars a_j, b_{j+1} are written by the reduction kernels into device arrays and copied to
// the host once per step (16 bytes) for the convergence test.
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "common.cuh"

namespace edg {
namespace {

struct Scalars {
  double* partial;  // [kRedSlots]: reduction partials and the fused finish's counter
  double* a;        // [cap+2]
  double* b;        // [cap+2], b[0] = 0 (Lanczos b's)
  double* bn;       // [cap+2], norms of the unnormalised vectors, bn[0] = 1 (fused form)
  double* tmp;      // [8]
  int cap;
};

int scalars(edg_sector_s* s, int cap, Scalars* sc) {
  const size_t need = size_t(kRedSlots) + 3 * size_t(cap + 2) + 8;
  EDG_CHECK(s->red.alloc(need, s->stream, "reduction scratch"));
  sc->partial = s->red.p;
  sc->a = sc->partial + kRedSlots;
  sc->b = sc->a + cap + 2;
  sc->bn = sc->b + cap + 2;
  sc->tmp = sc->bn + cap + 2;
  sc->cap = cap;
  EDG_CUDA(cudaMemsetAsync(s->red.p, 0, need * sizeof(double), s->stream));
  const double one = 1.0;
  EDG_CUDA(cudaMemcpyAsync(sc->bn, &one, sizeof(double), cudaMemcpyHostToDevice, s->stream));
  EDG_CUDA(cudaStreamSynchronize(s->stream));  // `one` is a stack value
  return EDG_OK;
}

template <typename T>
DevBuf<T>* block_buf(edg_sector_s* s);
template <>
DevBuf<double>* block_buf<double>(edg_sector_s* s) { return &s->blk64; }
template <>
DevBuf<float>* block_buf<float>(edg_sector_s* s) { return &s->blk32; }

template <typename T>
DevBuf<T>* work(edg_sector_s* s);
template <>
DevBuf<double>* work<double>(edg_sector_s* s) { return s->w64; }
template <>
DevBuf<float>* work<float>(edg_sector_s* s) { return s->w32; }

// The Lanczos recurrence in precision T over the sector's three work vectors.
template <typename T>
struct Recurrence {
  edg_sector_s* s = nullptr;
  Scalars sc{};
  T* U = nullptr;  // current vector: v_j (general) or u_j = b_j v_j (fused)
  T* P = nullptr;  // previous vector
  T* W = nullptr;  // output of the step
  bool fused = false;
  std::vector<double> bn_host;  // norms of u_j (fused); 1 for the general form
  // Basis columns used as the recurrence's own vectors (fused form): u_j is written straight
  // into column j, so keeping the basis costs no copy. Column j then holds u_j, i.e.
  // v_j / vscale(j). Past the last column the three work vectors take over.
  T* ext = nullptr;
  int ext_cols = 0;
  T* wbuf[3] = {nullptr, nullptr, nullptr};

  // v_0 = dv0 * scale; cap = most steps this run will take; basis (optional): ncols device
  // columns of dim elements that receive u_0, u_1, ... (fused form only)
  int init(edg_sector_s* sec, const double* dv0, double scale, int cap, T* basis = nullptr, int ncols = 0) {
    s = sec;
    const int64_t n = s->vlen;
    EDG_CHECK(scalars(s, cap, &sc));
    DevBuf<T>* wb = work<T>(s);
    for (int k = 0; k < 3; ++k) {
      EDG_CHECK(wb[k].alloc(n, s->stream, "Lanczos vectors"));
      wbuf[k] = wb[k].p;
    }
    U = wb[0].p;
    P = wb[1].p;
    W = wb[2].p;
    fused = hxv_lz_available(s, sizeof(T));
    if (fused && basis && ncols >= 2) {
      ext = basis;
      ext_cols = ncols;
      U = ext;
      W = ext + n;
    }
    EDG_CHECK((convert_dev<T, double>(s->stream, U, dv0, n, scale)));
    EDG_CUDA(cudaMemsetAsync(P, 0, n * sizeof(T), s->stream));
    bn_host.assign(1, 1.0);
    return EDG_OK;
  }
  // scale that turns the current buffer U into v_j
  double vscale(int j) const { return fused ? 1.0 / bn_host[j] : 1.0; }
  // step j queued on the stream: a_j and b_{j+1} land in the device scalars only
  int step_dev(int j) {
    const int64_t n = s->vlen;
    cudaStream_t st = s->stream;
    if (fused) {
      EDG_CHECK(hxv_apply_lz<T>(s, U, P, W, sc.bn, j, sc.partial, sc.a + j));
      EDG_CHECK(lanczos_step_b2<T>(st, W, U, sc.a + j, sc.bn + j, n, sc.partial, sc.bn + j + 1));
    } else {
      EDG_CHECK(hxv_apply<T>(s, U, W));
      EDG_CHECK(lanczos_step_a<T>(st, W, P, U, sc.b + j, n, sc.partial, sc.a + j));
      EDG_CHECK(lanczos_step_b<T>(st, W, U, sc.a + j, n, sc.partial, sc.b + j + 1));
    }
    return EDG_OK;
  }
  // device array of b_{j+1} (index j+1)
  const double* b_dev() const { return fused ? sc.bn : sc.b; }
  // step j: W <- the unnormalised u_{j+1}; returns a_j and b_{j+1} on the host
  int step(int j, double* a, double* b) {
    EDG_CHECK(step_dev(j));
    return read(j, a, b);
  }
  // a_j and b_{j+1} of a queued step j, on the host (waits for step j)
  int read(int j, double* a, double* b) {
    cudaStream_t st = s->stream;
    double h[2];
    EDG_CUDA(cudaMemcpyAsync(&h[0], sc.a + j, sizeof(double), cudaMemcpyDeviceToHost, st));
    EDG_CUDA(cudaMemcpyAsync(&h[1], (fused ? sc.bn : sc.b) + j + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    EDG_CUDA(cudaStreamSynchronize(st));
    *a = h[0];
    *b = h[1];
    return EDG_OK;
  }
  // after step j with b = b_{j+1} > 0: make U hold (a multiple of) v_{j+1}
  int advance(int j, double b) {
    if (fused) {
      T* t = P;
      P = U;
      U = W;
      if (ext && j + 2 < ext_cols) {
        W = ext + size_t(j + 2) * s->vlen;
      } else if (ext) {  // out of basis columns: a work vector that is neither P nor U
        W = wbuf[0] != P && wbuf[0] != U ? wbuf[0] : (wbuf[1] != P && wbuf[1] != U ? wbuf[1] : wbuf[2]);
      } else {
        W = t;
      }
      bn_host.push_back(b);
    } else {
      EDG_CHECK(scale_into<T>(s->stream, P, W, sc.b + j + 1, s->vlen));
      T* t = P;
      P = U;
      U = t;
    }
    return EDG_OK;
  }
};

// Tridiagonalisation in precision T from the FP64 device start vector dv0.
template <typename T>
int tridiag_t(edg_sector_s* s, const double* dv0, int nlanc, double threshold, double* alanc, double* blanc,
              double* norm2, int* nsteps) {
  const int64_t n = s->vlen;
  cudaStream_t st = s->stream;
  for (int j = 0; j < nlanc; ++j) { alanc[j] = 0.0; blanc[j] = 0.0; }
  *nsteps = 0;
  Scalars sc0;
  EDG_CHECK(scalars(s, 2, &sc0));
  EDG_CHECK(dot_dev<double>(st, dv0, dv0, n, sc0.partial, sc0.tmp));
  double n2 = 0.0;
  EDG_CUDA(cudaMemcpyAsync(&n2, sc0.tmp, sizeof(double), cudaMemcpyDeviceToHost, st));
  EDG_CUDA(cudaStreamSynchronize(st));
  *norm2 = n2;
  if (n2 == 0.0 || nlanc <= 0) return EDG_OK;
  Recurrence<T> R;
  EDG_CHECK(R.init(s, dv0, 1.0 / std::sqrt(n2), nlanc + 1));
  // Steps are queued kChunk at a time with the scalars left on the device; the host reads a
  // chunk's a/b at its end and stops at the first b below threshold (the steps queued after
  // it in the same chunk are discarded). The arithmetic is that of one step at a time.
  constexpr int kChunk = 16;
  std::vector<double> ha(kChunk), hb(kChunk);
  for (int j0 = 0; j0 < nlanc; j0 += kChunk) {
    const int j1 = std::min(nlanc, j0 + kChunk);
    for (int j = j0; j < j1; ++j) {
      EDG_CHECK(R.step_dev(j));
      if (j + 1 < nlanc) EDG_CHECK(R.advance(j, 0.0));  // the fused form's host norms are unused here
    }
    EDG_CUDA(cudaMemcpyAsync(ha.data(), R.sc.a + j0, size_t(j1 - j0) * sizeof(double), cudaMemcpyDeviceToHost, st));
    EDG_CUDA(cudaMemcpyAsync(hb.data(), R.b_dev() + j0 + 1, size_t(j1 - j0) * sizeof(double), cudaMemcpyDeviceToHost,
                             st));
    EDG_CUDA(cudaStreamSynchronize(st));
    for (int j = j0; j < j1; ++j) {
      const double b = hb[j - j0];
      alanc[j] = ha[j - j0];
      *nsteps = j + 1;
      if (j + 1 < nlanc) blanc[j + 1] = b;
      if (!(b >= threshold)) {  // also stops on NaN
        if (j + 1 < nlanc) blanc[j + 1] = 0.0;
        return EDG_OK;
      }
    }
  }
  return EDG_OK;
}

// k chains in lockstep with the fused recurrence of Recurrence<T> applied to every column:
// one launch per pass for all columns (block H x V, then the per-column w/a and u/b passes).
// Column c's arithmetic is that of a single chain, so its coefficients equal
// tridiag_t<T>'s bit for bit. A column stops at its first b below threshold: the host reads
// every column's scalars once per kChunk steps and clears the column's device flag, and
// the steps queued after the stop in that chunk are discarded.
// start(c) returns column c's FP64 start vector on the device (valid until the next call).
template <typename T, typename Start>
int tridiag_block_t(edg_sector_s* s, int k, const Start& start, int nlanc, double threshold, double* alanc,
                    double* blanc, double* norm2, int* nsteps) {
  const int64_t n = s->vlen;
  cudaStream_t st = s->stream;
  const int64_t sstride = nlanc + 2;  // per-column scalar arrays a[], bn[]
  DevBuf<T>& blk = *block_buf<T>(s);
  EDG_CHECK(blk.alloc(size_t(3) * k * n, st, "block Lanczos vectors"));
  const size_t nred = size_t(k) * kRedSlots + 2 * size_t(k) * sstride + size_t(k);
  EDG_CHECK(s->blkred.alloc(nred, st, "block Lanczos scalars"));
  EDG_CHECK(s->blkact.alloc(size_t(k), st, "block Lanczos flags"));
  double* partial = s->blkred.p;
  double* A = partial + size_t(k) * kRedSlots;
  double* BN = A + size_t(k) * sstride;
  double* N2 = BN + size_t(k) * sstride;
  EDG_CUDA(cudaMemsetAsync(s->blkred.p, 0, nred * sizeof(double), st));
  for (int c = 0; c < k; ++c) {
    nsteps[c] = 0;
    for (int j = 0; j < nlanc; ++j) alanc[size_t(c) * nlanc + j] = blanc[size_t(c) * nlanc + j] = 0.0;
  }
  T* U = blk.p;
  T* P = U + size_t(k) * n;
  T* W = P + size_t(k) * n;
  // each column's norm, then v_0 = start / |start| in precision T, one column at a time (the
  // start vectors may be produced into one shared buffer)
  for (int c = 0; c < k; ++c) {
    const double* x0 = nullptr;
    EDG_CHECK(start(c, &x0));
    EDG_CHECK(dot_dev<double>(st, x0, x0, n, partial, N2 + c));
    EDG_CHECK((normalise_cols<T, double>(st, 1, U + size_t(c) * n, n, x0, n, N2 + c, 1, n)));
  }
  std::vector<double> n2(k), one(k, 1.0);
  EDG_CUDA(cudaMemcpyAsync(n2.data(), N2, k * sizeof(double), cudaMemcpyDeviceToHost, st));
  EDG_CUDA(cudaStreamSynchronize(st));
  std::vector<int> act(k);
  int nact = 0;
  for (int c = 0; c < k; ++c) {
    norm2[c] = n2[c];
    act[c] = (n2[c] > 0.0 && nlanc > 0) ? 1 : 0;
    nact += act[c];
  }
  if (nact == 0) return EDG_OK;
  EDG_CUDA(cudaMemsetAsync(P, 0, size_t(k) * n * sizeof(T), st));
  EDG_CUDA(cudaMemcpy2DAsync(BN, sstride * sizeof(double), one.data(), sizeof(double), sizeof(double), k,
                             cudaMemcpyHostToDevice, st));  // bn[c][0] = 1
  EDG_CUDA(cudaMemcpyAsync(s->blkact.p, act.data(), k * sizeof(int), cudaMemcpyHostToDevice, st));
  EDG_CUDA(cudaStreamSynchronize(st));  // host staging arrays are read by the copies above
  constexpr int kChunk = 16;
  std::vector<double> ha(size_t(k) * kChunk), hb(size_t(k) * kChunk);
  for (int j0 = 0; j0 < nlanc && nact > 0; j0 += kChunk) {
    const int j1 = std::min(nlanc, j0 + kChunk);
    for (int j = j0; j < j1; ++j) {
      EDG_CHECK(hxv_block_lz<T>(s, k, s->blkact.p, U, P, W, BN, sstride, j, partial, A + j));
      EDG_CHECK(lanczos_step_b2_cols<T>(st, k, s->blkact.p, W, U, n, A + j, BN + j, partial, BN + j + 1, sstride, n));
      T* t = P;
      P = U;
      U = W;
      W = t;
    }
    const int m = j1 - j0;
    EDG_CUDA(cudaMemcpy2DAsync(ha.data(), m * sizeof(double), A + j0, sstride * sizeof(double), m * sizeof(double), k,
                               cudaMemcpyDeviceToHost, st));
    EDG_CUDA(cudaMemcpy2DAsync(hb.data(), m * sizeof(double), BN + j0 + 1, sstride * sizeof(double),
                               m * sizeof(double), k, cudaMemcpyDeviceToHost, st));
    EDG_CUDA(cudaStreamSynchronize(st));
    bool changed = false;
    for (int c = 0; c < k; ++c) {
      if (!act[c]) continue;
      for (int j = j0; j < j1; ++j) {
        const double b = hb[size_t(c) * m + (j - j0)];
        alanc[size_t(c) * nlanc + j] = ha[size_t(c) * m + (j - j0)];
        nsteps[c] = j + 1;
        if (j + 1 < nlanc) blanc[size_t(c) * nlanc + j + 1] = b;
        if (!(b >= threshold)) {  // also stops on NaN
          if (j + 1 < nlanc) blanc[size_t(c) * nlanc + j + 1] = 0.0;
          act[c] = 0;
          --nact;
          changed = true;
          break;
        }
      }
    }
    if (changed && nact > 0) {
      EDG_CUDA(cudaMemcpyAsync(s->blkact.p, act.data(), k * sizeof(int), cudaMemcpyHostToDevice, st));
      EDG_CUDA(cudaStreamSynchronize(st));
    }
  }
  return EDG_OK;
}

// Lowest Ritz value of T(a, b) and the a-posteriori estimate of its error,
// (b_next * |z_m|)^2 / gap: b_next*|z_m| is the residual norm of the Ritz pair and
// theta_1 - E_0 <= r^2 / gap for the lowest eigenvalue (gap from the second Ritz value).
struct Ritz {
  double e0, err;
};
// `window` (relative to |theta_1|): Ritz values that close to the lowest one are taken as its
// copies (the duplicates that plain Lanczos produces once orthogonality is lost, which FP32
// vectors reach early) and skipped when the gap is measured; 0 takes the next Ritz value.
Ritz lowest_ritz(const std::vector<double>& a, const std::vector<double>& b, double b_next, double window) {
  const int m = int(a.size());
  std::vector<double> w(m), zl(m);
  tridiag_eigh_host(m, a.data(), b.data(), w.data(), nullptr, nullptr, zl.data());
  Ritz r;
  r.e0 = w[0];
  const double res = b_next * std::fabs(zl[0]);
  int i = 1;
  while (i < m && w[i] - w[0] <= window * std::fabs(w[0])) ++i;
  const double gap = i < m ? w[i] - w[0] : 0.0;
  r.err = gap > 1e-12 ? res * res / gap : res;
  return r;
}

// Plain Lanczos in precision T from the normalised FP64 device vector dv0 until the lowest
// Ritz value is converged to tol (see lowest_ritz), b underflows, or maxit. Optionally stores
// the normalised basis vectors in FP32 so the Ritz vector needs no second pass.
template <typename T>
int gs_run(edg_sector_s* s, const double* dv0, int maxit, double tol, std::vector<double>* A,
           std::vector<double>* B, float* basis, int basis_cols, std::vector<double>* colscale, double* e0) {
  const int64_t n = s->vlen;
  cudaStream_t st = s->stream;
  Recurrence<T> R;
  T* own = std::is_same<T, float>::value ? reinterpret_cast<T*>(basis) : nullptr;
  EDG_CHECK(R.init(s, dv0, 1.0, maxit + 1, own, own ? basis_cols : 0));
  A->clear();
  B->assign(1, 0.0);
  colscale->clear();
  // the basis column of step j (before the step is queued)
  auto column = [&](int j) -> int {
    if (basis && j < basis_cols) {
      if (R.ext) {
        colscale->push_back(R.vscale(j));  // column j holds u_j = v_j / vscale(j)
      } else {
        EDG_CHECK((convert_dev<float, T>(st, basis + size_t(j) * n, R.U, n, R.vscale(j))));
        colscale->push_back(1.0);
      }
    }
    return EDG_OK;
  };
  double eold = 0.0, err_prev = HUGE_VAL;
  bool queued = false;  // step j was queued by the previous iteration
  for (int j = 0; j < maxit; ++j) {
    if (!queued) {
      EDG_CHECK(column(j));
      EDG_CHECK(R.step_dev(j));
    }
    double a, b;
    EDG_CHECK(R.read(j, &a, &b));
    if (!std::isfinite(a) || !std::isfinite(b)) {
      set_error("Lanczos produced a non-finite coefficient at step %d", j);
      return EDG_ERR_NOCONV;
    }
    A->push_back(a);
    // While the last test was far from convergence (its error estimate more than 100x the
    // target 0.1 tol |E0|), step j+1 is queued before step j is tested, so the host's test
    // runs while the GPU works; near convergence the test comes first, so no step is wasted.
    queued = j + 1 < maxit && b >= 1e-14 && err_prev > 10.0 * tol * std::fabs(eold);
    if (queued) {
      EDG_CHECK(R.advance(j, b));
      EDG_CHECK(column(j + 1));
      EDG_CHECK(R.step_dev(j + 1));
    }
    // FP32 vectors lose orthogonality within tens of steps: skip the copies of E0 that follow
    const Ritz rz = lowest_ritz(*A, *B, b, sizeof(T) == 4 ? 10.0 * tol : 0.0);
    const double e = rz.e0;
    // converged when the error estimate is 10x below tol*|E0| (or, as a fallback for a
    // degenerate lowest level, when E0 stops moving), or the Krylov space is exhausted; a
    // step queued ahead is then discarded (its column lies past the Ritz vector's)
    const bool conv = (j > 0 && rz.err <= 0.1 * tol * std::fabs(e)) ||
                      (j > 0 && std::fabs(e - eold) <= 0.01 * tol * std::fabs(e)) || b < 1e-14;
    eold = e;
    err_prev = rz.err;
    B->push_back(b);
    *e0 = e;
    if (conv || j + 1 == maxit) break;
    if (!queued) EDG_CHECK(R.advance(j, b));
  }
  EDG_CUDA(cudaStreamSynchronize(st));  // a discarded step still runs on the work vectors
  return EDG_OK;
}

// Ritz vector x = sum_j z_j v_j (FP64, device) for the lowest Ritz value of (A, B):
// from the stored FP32 basis when present, else by replaying the recurrence from dv0.
template <typename T>
int ritz_vector(edg_sector_s* s, const double* dv0, const std::vector<double>& A, const std::vector<double>& B,
                const float* basis, int basis_cols, const std::vector<double>& colscale, double* x) {
  const int64_t n = s->vlen;
  cudaStream_t st = s->stream;
  const int m = int(A.size());
  std::vector<double> w(m), Z(size_t(m) * m);
  EDG_CHECK(tridiag_eigh_host(m, A.data(), B.data(), w.data(), nullptr, Z.data()));
  EDG_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), st));
  if (basis && basis_cols >= m && int(colscale.size()) >= m) {
    // one pass over the stored columns (same FMA order as m successive axpys); column j
    // holds v_j / colscale[j]
    for (int j = 0; j < m; ++j) Z[j] *= colscale[j];
    Scalars scz;
    EDG_CHECK(scalars(s, m + 1, &scz));
    EDG_CUDA(cudaMemcpyAsync(scz.a, Z.data(), size_t(m) * sizeof(double), cudaMemcpyHostToDevice, st));
    EDG_CHECK(ritz_dev(st, basis, scz.a, m, n, x));
    EDG_CUDA(cudaStreamSynchronize(st));  // Z (host) must outlive the copy
  } else {
    Recurrence<T> R;
    EDG_CHECK(R.init(s, dv0, 1.0, m + 1));
    for (int j = 0; j < m; ++j) {
      EDG_CHECK(axpy_accum_dev<T>(st, x, R.U, Z[j] * R.vscale(j), n));
      if (j + 1 == m) break;
      double a, b;
      EDG_CHECK(R.step(j, &a, &b));
      EDG_CHECK(R.advance(j, b));
    }
  }
  // normalise
  Scalars sc2;
  EDG_CHECK(scalars(s, 2, &sc2));
  EDG_CHECK(dot_dev<double>(st, x, x, n, sc2.partial, sc2.tmp));
  double nn = 0.0;
  EDG_CUDA(cudaMemcpyAsync(&nn, sc2.tmp, sizeof(double), cudaMemcpyDeviceToHost, st));
  EDG_CUDA(cudaStreamSynchronize(st));
  if (!(nn > 0.0)) {
    set_error("Ritz vector vanished");
    return EDG_ERR_NOCONV;
  }
  EDG_CHECK((scale_inplace_dev<double>(st, x, n, 1.0 / std::sqrt(nn))));
  return EDG_OK;
}

// normalise dv (FP64, device) in place
int normalise(edg_sector_s* s, double* dv) {
  Scalars sc;
  EDG_CHECK(scalars(s, 2, &sc));
  EDG_CHECK(dot_dev<double>(s->stream, dv, dv, s->vlen, sc.partial, sc.tmp));
  double nn = 0.0;
  EDG_CUDA(cudaMemcpyAsync(&nn, sc.tmp, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  EDG_CUDA(cudaStreamSynchronize(s->stream));
  if (!(nn > 0.0)) {
    set_error("start vector has zero norm");
    return EDG_ERR_ARG;
  }
  return scale_inplace_dev<double>(s->stream, dv, s->vlen, 1.0 / std::sqrt(nn));
}

}  // namespace

int tridiag_dev(edg_sector_s* s, const double* dv0, int nlanc, double threshold, int precision, double* alanc,
                double* blanc, double* norm2, int* nsteps) {
  if (precision == EDG_PREC_F32) return tridiag_t<float>(s, dv0, nlanc, threshold, alanc, blanc, norm2, nsteps);
  return tridiag_t<double>(s, dv0, nlanc, threshold, alanc, blanc, norm2, nsteps);
}

int tridiag_block_fn(edg_sector_s* s, int k, const StartFn& start, int nlanc, double threshold, int precision,
                     double* alanc, double* blanc, double* norm2, int* nsteps) {
  const size_t elem = precision == EDG_PREC_F32 ? sizeof(float) : sizeof(double);
  if (k <= 0) return EDG_OK;
  if (!hxv_lz_available(s, elem) || nlanc <= 0) {  // one chain after another
    for (int c = 0; c < k; ++c) {
      const double* x0 = nullptr;
      EDG_CHECK(start(c, &x0));
      EDG_CHECK(tridiag_dev(s, x0, nlanc, threshold, precision, alanc + size_t(c) * nlanc, blanc + size_t(c) * nlanc,
                            norm2 + c, nsteps + c));
    }
    return EDG_OK;
  }
  // columns per block: three vectors each, within the free HBM less 2 GB
  size_t fr = 0, tot = 0;
  EDG_CUDA(cudaMemGetInfo(&fr, &tot));
  const size_t per = 3 * size_t(s->vlen) * elem;
  const size_t reserve = size_t(2) << 30;
  int kb = fr > reserve ? int(std::min<size_t>(size_t(k), (fr - reserve) / per)) : 0;
  if (kb < 1) kb = 1;
  for (int c0 = 0; c0 < k; c0 += kb) {
    const int kk = std::min(kb, k - c0);
    auto sub = [&](int c, const double** x) -> int { return start(c0 + c, x); };
    double* a = alanc + size_t(c0) * nlanc;
    double* b = blanc + size_t(c0) * nlanc;
    if (precision == EDG_PREC_F32)
      EDG_CHECK(tridiag_block_t<float>(s, kk, sub, nlanc, threshold, a, b, norm2 + c0, nsteps + c0));
    else
      EDG_CHECK(tridiag_block_t<double>(s, kk, sub, nlanc, threshold, a, b, norm2 + c0, nsteps + c0));
  }
  return EDG_OK;
}

int tridiag_block(edg_sector_s* s, int k, const double* dv0, int nlanc, double threshold, int precision,
                  double* alanc, double* blanc, double* norm2, int* nsteps) {
  const int64_t n = s->vlen;
  StartFn start = [dv0, n](int c, const double** x) -> int {
    *x = dv0 + size_t(c) * n;
    return EDG_OK;
  };
  return tridiag_block_fn(s, k, start, nlanc, threshold, precision, alanc, blanc, norm2, nsteps);
}

int ground_state(edg_sector_s* s, const double* v0_host, uint64_t seed, int maxit, double tol, int mode,
                 double* e0, int* niter) {
  const int64_t n = s->vlen;
  cudaStream_t st = s->stream;
  if (maxit <= 0) maxit = 1;
  if (maxit > s->dim) maxit = int(s->dim);  // the Krylov space has at most dim (complex) dimensions
  EDG_CHECK(s->state.alloc(n, st, "eigenvector"));
  EDG_CHECK(s->w64[3].alloc(n, st, "start vector"));
  double* x0 = s->w64[3].p;
  if (v0_host) {
    EDG_CUDA(cudaMemcpyAsync(x0, v0_host, n * sizeof(double), cudaMemcpyHostToDevice, st));
  } else {
    EDG_CHECK(random_dev(st, x0, n, seed));
  }
  EDG_CHECK(normalise(s, x0));
  std::vector<double> A, B, cs;
  *niter = 0;
  s->last_n32 = s->last_n64 = 0;
  s->has_state = false;
  const bool want_vec = !(mode & EDG_GS_E0_ONLY);
  mode &= 0xff;
  if (mode == EDG_GS_F64) {
    EDG_CHECK(gs_run<double>(s, x0, maxit, tol, &A, &B, nullptr, 0, &cs, e0));
    s->last_n64 += int(A.size());
    if (want_vec) {
      EDG_CHECK(ritz_vector<double>(s, x0, A, B, nullptr, 0, cs, s->state.p));
      s->last_n64 += int(A.size()) - 1;
    }
  } else {
    // phase 1: FP32 vectors. The basis is kept for the Ritz vector (no second pass) when
    // HBM admits it: at most half the free memory, kMaxBasisCols columns, allocated once
    // per sector and reused by later calls.
    constexpr int kMaxBasisCols = 512;
    const int want_cols = std::min(maxit, kMaxBasisCols);
    if (s->basis32_cols < size_t(want_cols)) {
      size_t freeb = 0, totb = 0;
      EDG_CUDA(cudaMemGetInfo(&freeb, &totb));
      const size_t vecb = size_t(n) * sizeof(float);
      const size_t slack = (size_t(3) << 30) + 6 * vecb;
      int cols = 0;
      if (freeb > slack) cols = int(std::min<size_t>((freeb - slack) / 2 / vecb, size_t(want_cols)));
      if (size_t(cols) > s->basis32_cols) {
        s->basis32.reset();
        s->basis32_cols = 0;
        if (cols > 0 && s->basis32.alloc(size_t(cols) * n, st, "FP32 Lanczos basis") == EDG_OK) s->basis32_cols = cols;
      }
    }
    const int cols = int(s->basis32_cols);
    // FP32 phase: stop once the lowest Ritz value settles at FP32 resolution
    const double tol32 = tol > 2e-7 ? tol : 2e-7;
    double e32 = 0.0;
    EDG_CHECK(gs_run<float>(s, x0, maxit, tol32, &A, &B, s->basis32.p, cols, &cs, &e32));
    s->last_n32 += int(A.size());
    EDG_CHECK(ritz_vector<float>(s, x0, A, B, s->basis32.p, cols, cs, s->state.p));
    if (cols < int(A.size())) s->last_n32 += int(A.size()) - 1;
    // phase 2: restarted FP64 Lanczos from the FP32 Ritz vector
    EDG_CUDA(cudaMemcpyAsync(x0, s->state.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    EDG_CHECK(gs_run<double>(s, x0, maxit, tol, &A, &B, nullptr, 0, &cs, e0));
    s->last_n64 += int(A.size());
    if (want_vec) {
      EDG_CHECK(ritz_vector<double>(s, x0, A, B, nullptr, 0, cs, s->state.p));
      s->last_n64 += int(A.size()) - 1;
    }
  }
  *niter = s->last_n32 + s->last_n64;
  EDG_CUDA(cudaStreamSynchronize(st));
  s->has_state = want_vec;
  return EDG_OK;
}

}  // namespace edg
