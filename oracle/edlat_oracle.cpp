// edlat_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement (C++17 + OpenMP, FP64) of the EDlattice sector-Lanczos path, used
// by tests/ as the parity checker and by bench.py as the timed CPU baseline. Nothing in
// the product library links, loads or calls this file.
//
// Parity status: UNPINNED against reference outputs. The reference is Fortran built on
// SciFortran; neither a Fortran compiler nor SciFortran exists on this machine, and the
// reference ships no golden vectors or tests. The restatement is instead pinned against
// known answers from the mathematics (free-fermion U=0 energies, the Hubbard dimer closed
// form, the atomic limit) and against dense diagonalisation, in tests/test_oracle_*.py.
//
// Every routine cites the reference file:line whose loop structure it follows; paths are
// relative to the EDlattice project root. Indices in comments are the reference's
// 1-based ones; the C code is 0-based (state i here = reference i-1).
//
// Model restriction: one orbital (Norb=1, Nsites=[Ns]), Nspin 1 or 2, no Jx/Jp
// (Jhflag=.false., src/SETUP.f90:35-36), the same restriction as the hot path.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> zc;

extern "C" {

// Model description passed from Python (ctypes struct with the same layout).
typedef struct {
  int ns;                  // number of sites Ns (<= 30)
  int nspin;               // 1: Hij shared by both spins; 2: separate dw matrix
  const double* hij_re;    // Hij(1,:,:) row-major [io*Ns+jo], real part
  const double* hij_im;    // imaginary part or NULL
  const double* hijdw_re;  // Hij(2,:,:) when nspin==2, else NULL
  const double* hijdw_im;
  double uloc;             // Uloc(1)
  double xmu;              // xmu
  int hfmode;              // HFMODE (logical)
  int ed_filling;          // ED_FILLING (0 = grand canonical shift applied in direct form)
} orc_model;

}  // extern "C"

namespace {

zc hij(const orc_model* m, int spin, int io, int jo) {
  const double* re = (spin == 2 && m->nspin == 2) ? m->hijdw_re : m->hij_re;
  const double* im = (spin == 2 && m->nspin == 2) ? m->hijdw_im : m->hij_im;
  double r = re[io * m->ns + jo];
  double i = im ? im[io * m->ns + jo] : 0.0;
  return zc(r, i);
}

inline int btest(int64_t v, int pos0) { return (int)((v >> pos0) & 1); }

// c(pos,in,out,fsgn): src/AUX_FUNX.f90:76-88 (pos is 1-based there, 0-based here).
inline void op_c(int pos, int64_t in, int64_t* out, double* fsgn) {
  double s = 1.0;
  for (int l = 0; l < pos; ++l)
    if (btest(in, l)) s = -s;
  *fsgn = s;
  *out = in & ~(int64_t(1) << pos);
}
// cdg(pos,in,out,fsgn): src/AUX_FUNX.f90:90-102.
inline void op_cdg(int pos, int64_t in, int64_t* out, double* fsgn) {
  double s = 1.0;
  for (int l = 0; l < pos; ++l)
    if (btest(in, l)) s = -s;
  *fsgn = s;
  *out = in | (int64_t(1) << pos);
}

// binary_search(a,value): src/AUX_FUNX.f90:163-180, the recursive halving on array
// slices. Returns the 1-based position or 0 when absent.
int64_t bsearch_rec(const int32_t* a, int64_t n, int64_t value) {
  if (n == 0) return 0;
  int64_t mid = n / 2 + 1;  // 1-based
  if (a[mid - 1] > value) return bsearch_rec(a, mid - 1, value);
  if (a[mid - 1] < value) {
    int64_t r = bsearch_rec(a + mid, n - mid, value);
    return r != 0 ? mid + r : 0;
  }
  return mid;
}

// Lanczos vectors may be real or complex; helpers for both.
inline double cnj(double x) { return x; }
inline zc cnj(zc x) { return std::conj(x); }
inline double re_part(double x) { return x; }
inline double re_part(zc x) { return x.real(); }
inline double abs2(double x) { return x * x; }
inline double abs2(zc x) { return std::norm(x); }

struct Sector {
  int ns, nup, ndw;
  int64_t dimup, dimdw, dim;
  std::vector<int32_t> mup, mdw;
};

// build_sector: src/SECTOR.f90:69-115 -- ascending scan of 0..2^Ns-1 keeping popcount==N.
int64_t build_map(int ns, int n, int32_t* out) {
  int64_t dim = 0;
  for (int64_t s = 0; s < (int64_t(1) << ns); ++s) {
    if (__builtin_popcountll(s) != n) continue;
    if (out) out[dim] = (int32_t)s;
    ++dim;
  }
  return dim;
}

void make_sector(int ns, int nup, int ndw, Sector* S) {
  S->ns = ns; S->nup = nup; S->ndw = ndw;
  S->dimup = build_map(ns, nup, nullptr);
  S->dimdw = build_map(ns, ndw, nullptr);
  S->mup.resize(S->dimup); S->mdw.resize(S->dimdw);
  build_map(ns, nup, S->mup.data());
  build_map(ns, ndw, S->mdw.data());
  S->dim = S->dimup * S->dimdw;
}

// Diagonal element, direct form: src/DIAG/direct/HxV_local.f90:15-95 (Norb=1).
// The xmu and Hartree shifts apply only when ed_filling==0 (HxV_local.f90:63-92).
double diag_direct(const orc_model* m, int32_t mup, int32_t mdw) {
  const int ns = m->ns;
  double htmp = 0.0;
  for (int io = 0; io < ns; ++io)
    htmp += hij(m, 1, io, io).real() * btest(mup, io) + hij(m, 2, io, io).real() * btest(mdw, io);
  if (m->uloc != 0.0)
    for (int io = 0; io < ns; ++io) htmp += m->uloc * btest(mup, io) * btest(mdw, io);
  if (m->ed_filling == 0) {
    for (int io = 0; io < ns; ++io) htmp -= m->xmu * (btest(mup, io) + btest(mdw, io));
    if (m->hfmode && m->uloc != 0.0)
      for (int io = 0; io < ns; ++io) htmp -= 0.5 * m->uloc * (btest(mup, io) + btest(mdw, io));
  }
  return htmp;
}

// Diagonal element, stored form: src/DIAG/stored/H_local.f90:15-89. The xmu/Hartree
// shifts are applied unconditionally there (the ed_filling test is commented out, :61,90).
double diag_stored(const orc_model* m, int32_t mup, int32_t mdw) {
  const int ns = m->ns;
  double htmp = 0.0;
  for (int io = 0; io < ns; ++io)
    htmp += hij(m, 1, io, io).real() * btest(mup, io) + hij(m, 2, io, io).real() * btest(mdw, io);
  for (int io = 0; io < ns; ++io) htmp += m->uloc * btest(mup, io) * btest(mdw, io);
  for (int io = 0; io < ns; ++io) htmp -= m->xmu * (btest(mup, io) + btest(mdw, io));
  if (m->hfmode && m->uloc != 0.0)
    for (int io = 0; io < ns; ++io) htmp -= 0.5 * m->uloc * (btest(mup, io) + btest(mdw, io));
  return htmp;
}

// Row-of-vectors CSR as built by ed_buildh with sp_insert_element
// (src/SPARSE_MATRIX.f90:254-282): rows = target index, entries appended in insertion order.
struct RowCSR {
  std::vector<std::vector<int32_t>> cols;
  std::vector<std::vector<zc>> vals;
  void init(int64_t n) { cols.assign(n, {}); vals.assign(n, {}); }
  void insert(int64_t i, int64_t j, zc v) {
    auto& c = cols[i];
    for (size_t k = 0; k < c.size(); ++k)
      if (c[k] == j) { vals[i][k] += v; return; }
    c.push_back((int32_t)j);
    vals[i].push_back(v);
  }
};

// H_up / H_dw hop matrices of the stored form: src/DIAG/stored/H_up.f90:1-27 and
// H_dw.f90:1-28. Entry (target, source) = conjg(Hij(spin,io,jo))*sg1*sg2.
void build_hop_csr(const orc_model* m, int spin, const std::vector<int32_t>& map, RowCSR* H) {
  const int ns = m->ns;
  const int64_t dim = (int64_t)map.size();
  H->init(dim);
  for (int64_t jj = 0; jj < dim; ++jj) {
    const int64_t ms = map[jj];
    for (int io = 0; io < ns; ++io)
      for (int jo = 0; jo < ns; ++jo) {
        zc h = hij(m, spin, io, jo);
        if (h != zc(0.0) && btest(ms, jo) == 1 && btest(ms, io) == 0) {
          int64_t k1, k2; double sg1, sg2;
          op_c(jo, ms, &k1, &sg1);
          op_cdg(io, k1, &k2, &sg2);
          int64_t ii = bsearch_rec(map.data(), dim, k2) - 1;
          H->insert(ii, jj, std::conj(h) * sg1 * sg2);
        }
      }
  }
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- sector helpers
// binomial: src/SETUP.f90:336-358 (FP64 running product, rounded).
int orc_binomial(int n1, int n2) {
  if (n2 < 0) return 0;
  if (n2 > n1) return 0;
  if (n2 == 0) return 1;
  double xh = 1.0;
  for (int i = 1; i <= n2; ++i) xh = xh * double(n1 + 1 - i) / double(i);
  return (int)(xh + 0.5);
}

// get_Sector: src/SECTOR.f90:370-381 with QN=[Nup,Ndw], N=Ns.
int orc_get_sector(int ns, int nup, int ndw) { return 1 + nup * (ns + 1) + ndw; }
// get_Nup / get_Ndw: src/SECTOR.f90:401-424.
int orc_get_nup(int ns, int isector) { return ((isector - 1) / (ns + 1)) % (ns + 1); }
int orc_get_ndw(int ns, int isector) { return (isector - 1) % (ns + 1); }

int64_t orc_build_map(int ns, int n, int32_t* out) { return build_map(ns, n, out); }

int64_t orc_binary_search(const int32_t* a, int64_t n, int64_t value) { return bsearch_rec(a, n, value); }

void orc_c(int pos1, int64_t in, int64_t* out, double* sgn) { op_c(pos1 - 1, in, out, sgn); }
void orc_cdg(int pos1, int64_t in, int64_t* out, double* sgn) { op_cdg(pos1 - 1, in, out, sgn); }

// state2indices / indices2state: src/SECTOR.f90:443-464 (1-based in and out).
void orc_state2indices(int64_t istate, int64_t dimup, int64_t dimdw, int64_t* iup, int64_t* idw) {
  (void)dimdw;
  int64_t count = istate - 1;
  *iup = count % dimup + 1;
  *idw = count / dimup + 1;
}
int64_t orc_indices2state(int64_t iup, int64_t idw, int64_t dimup) { return iup + (idw - 1) * dimup; }

// Hop list of one spin in the stored form, exported for bit-exact comparison with the
// device-built tables: for each target row (ascending), its (source, value) entries in
// insertion order. Returns nnz; pass NULL buffers to query the size.
int64_t orc_hop_csr(const orc_model* m, int spin, int n, int64_t* rowptr, int32_t* cols, double* vals_re) {
  std::vector<int32_t> map(build_map(m->ns, n, nullptr));
  build_map(m->ns, n, map.data());
  RowCSR H;
  build_hop_csr(m, spin, map, &H);
  int64_t nnz = 0;
  for (size_t i = 0; i < H.cols.size(); ++i) {
    if (rowptr) rowptr[i] = nnz;
    for (size_t k = 0; k < H.cols[i].size(); ++k) {
      if (cols) cols[nnz] = H.cols[i][k];
      if (vals_re) vals_re[nnz] = H.vals[i][k].real();
      ++nnz;
    }
  }
  if (rowptr) rowptr[H.cols.size()] = nnz;
  return nnz;
}

// ---------------------------------------------------------------- H x v
// directMatVec: src/DIAG/HAMILTONIAN_DIRECT_HxV.f90:19-59 with the included
// direct/HxV_local.f90, HxV_up.f90, HxV_dw.f90; complex(8) vectors, serial loop order.
void orc_direct_matvec_z(const orc_model* m, int nup, int ndw, const zc* vin, zc* hv) {
  Sector S; make_sector(m->ns, nup, ndw, &S);
  const int ns = m->ns;
  const int64_t DimUp = S.dimup, DimDw = S.dimdw, Nloc = S.dim;
  for (int64_t i = 0; i < Nloc; ++i) hv[i] = 0.0;
  // local part, HxV_local.f90:1-97
  for (int64_t i = 0; i < Nloc; ++i) {
    int64_t iup = i % DimUp, idw = i / DimUp;
    hv[i] += diag_direct(m, S.mup[iup], S.mdw[idw]) * vin[i];
  }
  // up part, HxV_up.f90:1-34
  for (int64_t jdw = 0; jdw < DimDw; ++jdw)
    for (int64_t jup = 0; jup < DimUp; ++jup) {
      const int64_t mup = S.mup[jup];
      const int64_t j = jup + jdw * DimUp;
      for (int io = 0; io < ns; ++io)
        for (int jo = 0; jo < ns; ++jo) {
          zc h = hij(m, 1, io, jo);
          if (h != zc(0.0) && btest(mup, jo) == 1 && btest(mup, io) == 0) {
            int64_t k1, k2; double sg1, sg2;
            op_c(jo, mup, &k1, &sg1);
            op_cdg(io, k1, &k2, &sg2);
            int64_t iup = bsearch_rec(S.mup.data(), DimUp, k2) - 1;
            hv[iup + jdw * DimUp] += h * sg1 * sg2 * vin[j];
          }
        }
    }
  // dw part, HxV_dw.f90:1-32
  for (int64_t jup = 0; jup < DimUp; ++jup)
    for (int64_t jdw = 0; jdw < DimDw; ++jdw) {
      const int64_t mdw = S.mdw[jdw];
      const int64_t j = jup + jdw * DimUp;
      for (int io = 0; io < ns; ++io)
        for (int jo = 0; jo < ns; ++jo) {
          zc h = hij(m, 2, io, jo);
          if (h != zc(0.0) && btest(mdw, jo) == 1 && btest(mdw, io) == 0) {
            int64_t k1, k2; double sg1, sg2;
            op_c(jo, mdw, &k1, &sg1);
            op_cdg(io, k1, &k2, &sg2);
            int64_t idw = bsearch_rec(S.mdw.data(), DimDw, k2) - 1;
            hv[jup + idw * DimUp] += h * sg1 * sg2 * vin[j];
          }
        }
    }
}

// Stored-form operator (ed_buildh + spMatVec), kept alive across calls so that the
// CPU baseline times the matvec alone, as the reference does after build_Hv_sector.
struct orc_stored {
  orc_model m;
  Sector S;
  std::vector<double> d;             // spH0d: one diagonal entry per row
  RowCSR hup, hdw;                   // spH0ups(1), spH0dws(1)
  // flattened copies for the timed loop (same entry order as the row vectors)
  std::vector<int64_t> up_ptr, dw_ptr;
  std::vector<int32_t> up_col, dw_col;
  std::vector<zc> up_val, dw_val;
};

// ed_buildh: src/DIAG/HAMILTONIAN_STORED_HxV.f90:21-126 (H_local, H_up, H_dw includes).
orc_stored* orc_stored_create(const orc_model* m, int nup, int ndw) {
  orc_stored* st = new orc_stored();
  st->m = *m;
  st->m.hij_re = st->m.hij_im = st->m.hijdw_re = st->m.hijdw_im = nullptr;  // not used after build
  make_sector(m->ns, nup, ndw, &st->S);
  const int64_t DimUp = st->S.dimup;
  st->d.resize(st->S.dim);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < st->S.dim; ++i)
    st->d[i] = diag_stored(m, st->S.mup[i % DimUp], st->S.mdw[i / DimUp]);
  build_hop_csr(m, 1, st->S.mup, &st->hup);
  build_hop_csr(m, 2, st->S.mdw, &st->hdw);
  auto flat = [](const RowCSR& H, std::vector<int64_t>& p, std::vector<int32_t>& c, std::vector<zc>& v) {
    p.assign(H.cols.size() + 1, 0);
    for (size_t i = 0; i < H.cols.size(); ++i) p[i + 1] = p[i] + (int64_t)H.cols[i].size();
    c.resize(p.back()); v.resize(p.back());
    for (size_t i = 0; i < H.cols.size(); ++i)
      for (size_t k = 0; k < H.cols[i].size(); ++k) { c[p[i] + k] = H.cols[i][k]; v[p[i] + k] = H.vals[i][k]; }
  };
  flat(st->hup, st->up_ptr, st->up_col, st->up_val);
  flat(st->hdw, st->dw_ptr, st->dw_col, st->dw_val);
  return st;
}
void orc_stored_destroy(orc_stored* st) { delete st; }
int64_t orc_stored_dim(const orc_stored* st) { return st->S.dim; }

// spMatVec: src/DIAG/HAMILTONIAN_STORED_HxV.f90:159-220 -- local, then DW, then UP, each
// output accumulated in the reference's order. OpenMP splits the outer loops only, so
// every output element keeps the serial summation order.
}  // extern "C"

// The three sweeps restricted to output rows idw in [row_lo,row_hi) (the whole operator for
// [0,DimDw)): the reference's loop order, with its stride-DimUp DW sweep, so that a bounded
// sample of rows times the reference's memory-access pattern.
template <typename T>
void stored_matvec_sweeps(const orc_stored* st, const T* v, T* hv, int64_t row_lo, int64_t row_hi) {
  const int64_t DimUp = st->S.dimup;
#pragma omp parallel for schedule(static)
  for (int64_t i = row_lo * DimUp; i < row_hi * DimUp; ++i) hv[i] = st->d[i] * v[i];
#pragma omp parallel for schedule(static)
  for (int64_t iup = 0; iup < DimUp; ++iup)
    for (int64_t idw = row_lo; idw < row_hi; ++idw) {
      const int64_t i = iup + idw * DimUp;
      T acc = hv[i];
      for (int64_t jj = st->dw_ptr[idw]; jj < st->dw_ptr[idw + 1]; ++jj) {
        const int64_t j = iup + (int64_t)st->dw_col[jj] * DimUp;
        if constexpr (std::is_same<T, double>::value) acc += st->dw_val[jj].real() * v[j];
        else acc += st->dw_val[jj] * v[j];
      }
      hv[i] = acc;
    }
#pragma omp parallel for schedule(static)
  for (int64_t idw = row_lo; idw < row_hi; ++idw)
    for (int64_t iup = 0; iup < DimUp; ++iup) {
      const int64_t i = iup + idw * DimUp;
      T acc = hv[i];
      for (int64_t jj = st->up_ptr[iup]; jj < st->up_ptr[iup + 1]; ++jj) {
        const int64_t j = (int64_t)st->up_col[jj] + idw * DimUp;
        if constexpr (std::is_same<T, double>::value) acc += st->up_val[jj].real() * v[j];
        else acc += st->up_val[jj] * v[j];
      }
      hv[i] = acc;
    }
}
template <typename T>
void stored_matvec(const orc_stored* st, const T* v, T* hv) {
  stored_matvec_sweeps<T>(st, v, hv, 0, st->S.dimdw);
}
// The same arithmetic restricted to output rows idw in [row_lo,row_hi): a bounded sample of
// spMatVec for the CPU baseline. Each output element is computed exactly as above.
void stored_matvec_rows(const orc_stored* st, const double* v, double* hv, int64_t row_lo, int64_t row_hi) {
  const int64_t DimUp = st->S.dimup;
#pragma omp parallel for schedule(static)
  for (int64_t idw = row_lo; idw < row_hi; ++idw)
    for (int64_t iup = 0; iup < DimUp; ++iup) {
      const int64_t i = iup + idw * DimUp;
      double acc = st->d[i] * v[i];
      for (int64_t jj = st->dw_ptr[idw]; jj < st->dw_ptr[idw + 1]; ++jj)
        acc += st->dw_val[jj].real() * v[iup + (int64_t)st->dw_col[jj] * DimUp];
      for (int64_t jj = st->up_ptr[iup]; jj < st->up_ptr[iup + 1]; ++jj)
        acc += st->up_val[jj].real() * v[(int64_t)st->up_col[jj] + idw * DimUp];
      hv[i] = acc;
    }
}

extern "C" {

void orc_stored_matvec_rows_d(const orc_stored* st, const double* v, double* hv, int64_t row_lo, int64_t row_hi) {
  if (row_lo < 0) row_lo = 0;
  if (row_hi > st->S.dimdw) row_hi = st->S.dimdw;
  stored_matvec_rows(st, v, hv, row_lo, row_hi);
}
// Output rows [row_lo,row_hi) in the reference's three-sweep order (CPU baseline).
void orc_stored_matvec_sweeps_d(const orc_stored* st, const double* v, double* hv, int64_t row_lo, int64_t row_hi) {
  if (row_lo < 0) row_lo = 0;
  if (row_hi > st->S.dimdw) row_hi = st->S.dimdw;
  if (row_hi > row_lo) stored_matvec_sweeps<double>(st, v, hv, row_lo, row_hi);
}
int64_t orc_stored_dimdw(const orc_stored* st) { return st->S.dimdw; }

void orc_stored_matvec_z(const orc_stored* st, const zc* v, zc* hv) { stored_matvec<zc>(st, v, hv); }
// Real-vector variant (valid when Hij is real): identical loops on double vectors.
void orc_stored_matvec_d(const orc_stored* st, const double* v, double* hv) { stored_matvec<double>(st, v, hv); }

// Direct form on real vectors, OpenMP over the outer (source) loop of each part is not
// race free (scatter), so the parallel variant below splits the DW part by jup and the UP
// part by jdw -- both write disjoint output columns/rows. Loop bodies follow
// HxV_local/HxV_up/HxV_dw.f90 exactly (Ns x Ns scan, bit loops, binary search).
void orc_direct_matvec_d(const orc_model* m, int nup, int ndw, const double* vin, double* hv, int64_t row_lo, int64_t row_hi) {
  Sector S; make_sector(m->ns, nup, ndw, &S);
  const int ns = m->ns;
  const int64_t DimUp = S.dimup, DimDw = S.dimdw;
  if (row_hi < 0 || row_hi > DimDw) row_hi = DimDw;
  if (row_lo < 0) row_lo = 0;
  // restrict to the jdw rows [row_lo,row_hi): the UP part of those rows and the DW part
  // landing on them (used to time a bounded sample of the full operator).
#pragma omp parallel for schedule(static)
  for (int64_t idw = row_lo; idw < row_hi; ++idw)
    for (int64_t iup = 0; iup < DimUp; ++iup) {
      const int64_t i = iup + idw * DimUp;
      hv[i] = diag_direct(m, S.mup[iup], S.mdw[idw]) * vin[i];
    }
#pragma omp parallel for schedule(static)
  for (int64_t jdw = row_lo; jdw < row_hi; ++jdw)
    for (int64_t jup = 0; jup < DimUp; ++jup) {
      const int64_t mup = S.mup[jup];
      const int64_t j = jup + jdw * DimUp;
      for (int io = 0; io < ns; ++io)
        for (int jo = 0; jo < ns; ++jo) {
          double h = hij(m, 1, io, jo).real();
          if (h != 0.0 && btest(mup, jo) == 1 && btest(mup, io) == 0) {
            int64_t k1, k2; double sg1, sg2;
            op_c(jo, mup, &k1, &sg1);
            op_cdg(io, k1, &k2, &sg2);
            int64_t iup = bsearch_rec(S.mup.data(), DimUp, k2) - 1;
            hv[iup + jdw * DimUp] += h * sg1 * sg2 * vin[j];
          }
        }
    }
#pragma omp parallel for schedule(static)
  for (int64_t jup = 0; jup < DimUp; ++jup)
    for (int64_t jdw = 0; jdw < DimDw; ++jdw) {
      const int64_t mdw = S.mdw[jdw];
      const int64_t j = jup + jdw * DimUp;
      for (int io = 0; io < ns; ++io)
        for (int jo = 0; jo < ns; ++jo) {
          double h = hij(m, 2, io, jo).real();
          if (h != 0.0 && btest(mdw, jo) == 1 && btest(mdw, io) == 0) {
            int64_t k1, k2; double sg1, sg2;
            op_c(jo, mdw, &k1, &sg1);
            op_cdg(io, k1, &k2, &sg2);
            int64_t idw = bsearch_rec(S.mdw.data(), DimDw, k2) - 1;
            if (idw < row_lo || idw >= row_hi) continue;
            hv[jup + idw * DimUp] += h * sg1 * sg2 * vin[j];
          }
        }
    }
}

// Dense sector Hamiltonian as ed_buildh(Hmat) assembles it:
// src/DIAG/HAMILTONIAN_STORED_HxV.f90:81-117 -- diag + kron(Hdw,1) + kron(1,Hup).
// Real part only (column-major like the Fortran Hmat(i,j), i = row).
void orc_dense_h(const orc_model* m, int nup, int ndw, double* H) {
  orc_stored* st = orc_stored_create(m, nup, ndw);
  const int64_t D = st->S.dim, DimUp = st->S.dimup, DimDw = st->S.dimdw;
  std::memset(H, 0, sizeof(double) * D * D);
  for (int64_t i = 0; i < D; ++i) H[i + i * D] += st->d[i];
  for (int64_t idw = 0; idw < DimDw; ++idw)
    for (int64_t jj = st->dw_ptr[idw]; jj < st->dw_ptr[idw + 1]; ++jj)
      for (int64_t iup = 0; iup < DimUp; ++iup) {
        int64_t i = iup + idw * DimUp, j = iup + (int64_t)st->dw_col[jj] * DimUp;
        H[i + j * D] += st->dw_val[jj].real();
      }
  for (int64_t iup = 0; iup < DimUp; ++iup)
    for (int64_t jj = st->up_ptr[iup]; jj < st->up_ptr[iup + 1]; ++jj)
      for (int64_t idw = 0; idw < DimDw; ++idw) {
        int64_t i = iup + idw * DimUp, j = (int64_t)st->up_col[jj] + idw * DimUp;
        H[i + j * D] += st->up_val[jj].real();
      }
  orc_stored_destroy(st);
}

// ---------------------------------------------------------------- tridiagonal eigensolver
// Independent of the product's solver on purpose: cyclic Jacobi rotations on the dense
// symmetric tridiagonal matrix (Golub & Van Loan, Alg. 8.5.3). Eigenvalues ascending;
// Z column-major Z[i + j*n] (Z(i,j) of add_to_lanczos_gf_normal, src/GF/GF_ELECTRONS.f90:447).
// d[0..n-1] diagonal, e[1..n-1] sub-diagonal coupling (e[k] couples k-1 and k).
void orc_tridiag_eigh(int n, const double* d, const double* e, double* w, double* Z) {
  std::vector<double> A((size_t)n * n, 0.0), V((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) { A[i + i * n] = d[i]; V[i + i * n] = 1.0; }
  for (int k = 1; k < n; ++k) { A[k + (k - 1) * n] = e[k]; A[(k - 1) + k * n] = e[k]; }
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) { double a = A[i + j * n] * A[i + j * n]; tot += a; if (i != j) off += a; }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = A[p + q * n];
        if (apq == 0.0) continue;
        double app = A[p + p * n], aqq = A[q + q * n];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {  // A <- A J
          double akp = A[k + p * n], akq = A[k + q * n];
          A[k + p * n] = c * akp - s * akq;
          A[k + q * n] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // A <- J^T A
          double apk = A[p + k * n], aqk = A[q + k * n];
          A[p + k * n] = c * apk - s * aqk;
          A[q + k * n] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double vkp = V[k + p * n], vkq = V[k + q * n];
          V[k + p * n] = c * vkp - s * vkq;
          V[k + q * n] = s * vkp + c * vkq;
        }
      }
  }
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return A[a + a * n] < A[b + b * n]; });
  for (int j = 0; j < n; ++j) {
    w[j] = A[idx[j] + idx[j] * n];
    if (Z)
      for (int i = 0; i < n; ++i) Z[i + j * n] = V[i + idx[j] * n];
  }
}

}  // extern "C"

// ---------------------------------------------------------------- Lanczos
namespace {

template <typename T>
double dotre(const std::vector<T>& a, const std::vector<T>& b) {
  double s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) s += re_part(cnj(a[i]) * b[i]);
  return s;
}

// The three-term recurrence behind SciFortran's sp_lanc_tridiag / sp_lanc_eigh (called at
// src/DIAG/HAMILTONIAN.f90:268 and src/DIAG/DIAG.f90:216). SciFortran is not available, so
// the recurrence is restated from its mathematical definition:
//   w = H v_j - b_j v_{j-1};  a_j = <v_j|w>;  w -= a_j v_j;  b_{j+1} = |w|;  v_{j+1} = w/b_{j+1}
// stored as alanc(j)=a_j, blanc(j+1)=b_{j+1}, blanc(1)=0 -- the convention consumed by
// add_to_lanczos_gf_normal (src/GF/GF_ELECTRONS.f90:445-447). The chain stops early when
// b_{j+1} < threshold (absolute); the remaining coefficients stay zero.
template <typename T, typename MV>
int lanczos_tridiag(MV matvec, std::vector<T> v, int nlanc, double threshold, double* alanc, double* blanc,
                    std::vector<std::vector<T>>* basis) {
  const size_t n = v.size();
  std::vector<T> vprev(n, T(0.0)), w(n);
  for (int j = 0; j < nlanc; ++j) { alanc[j] = 0.0; blanc[j] = 0.0; }
  double b = 0.0;
  int used = 0;
  for (int j = 0; j < nlanc; ++j) {
    if (basis) basis->push_back(v);
    matvec(v.data(), w.data());
    for (size_t i = 0; i < n; ++i) w[i] -= b * vprev[i];
    double a = dotre(v, w);
    for (size_t i = 0; i < n; ++i) w[i] -= a * v[i];
    double bn = std::sqrt(dotre(w, w));
    alanc[j] = a;
    used = j + 1;
    if (j + 1 < nlanc) blanc[j + 1] = bn;
    if (bn < threshold) { if (j + 1 < nlanc) blanc[j + 1] = 0.0; break; }
    for (size_t i = 0; i < n; ++i) { vprev[i] = v[i]; v[i] = w[i] / bn; }
    b = bn;
  }
  return used;
}

}  // namespace

extern "C" {

// tridiag_Hv_sector: src/DIAG/HAMILTONIAN.f90:242-275. norm2=<v|v>, v/=sqrt(norm2),
// then the recurrence above with the stored-form operator (ed_sparse_H default .true.,
// src/INPUT_VARS.f90:151). Returns the number of steps taken.
int orc_tridiag_d(const orc_stored* st, const double* vvinit, int nlanc, double threshold,
                  double* alanc, double* blanc, double* norm2) {
  const int64_t D = st->S.dim;
  std::vector<double> v(vvinit, vvinit + D);
  double n2 = 0.0;
  for (int64_t i = 0; i < D; ++i) n2 += v[i] * v[i];
  *norm2 = n2;
  for (int j = 0; j < nlanc; ++j) { alanc[j] = 0.0; blanc[j] = 0.0; }
  if (n2 == 0.0) return 0;
  const double s = std::sqrt(n2);
  for (auto& x : v) x /= s;
  auto mv = [st](const double* a, double* b) { orc_stored_matvec_d(st, a, b); };
  return lanczos_tridiag<double>(mv, v, nlanc, threshold, alanc, blanc, nullptr);
}

// Ground-state Lanczos (contract of sp_lanc_eigh, src/DIAG/DIAG.f90:212-217): run the
// recurrence from the normalised start vector, after each step diagonalise T_j, stop when
// |E0(j)-E0(j-1)| <= tol*|E0(j)| or b_{j+1} < 1e-14 or j == maxit; the eigenvector is the
// Ritz vector sum_j Z(j,1) v_j, normalised. Returns the number of steps. The basis is kept
// only when evec is requested (E0-only runs of sectors with 1e8+ states keep three vectors);
// the vector loops run on all host threads with a static schedule, so a run is reproducible
// for a given thread count.
namespace {
double par_dot(const double* x, const double* y, int64_t n) {
  double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (int64_t i = 0; i < n; ++i) s += x[i] * y[i];
  return s;
}
}  // namespace

int orc_lanczos_gs_d(const orc_stored* st, const double* v0, int maxit, double tol, double* e0, double* evec,
                     double* alanc, double* blanc) {
  const int64_t D = st->S.dim;
  std::vector<double> v(v0, v0 + D);
  const double nv = std::sqrt(par_dot(v.data(), v.data(), D));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < D; ++i) v[i] /= nv;
  std::vector<double> vprev(D, 0.0), w(D);
  std::vector<std::vector<double>> basis;
  std::vector<double> a, b(1, 0.0);
  double eold = 0.0, enew = 0.0;
  int it = 0;
  for (it = 0; it < maxit; ++it) {
    if (evec) basis.push_back(v);
    orc_stored_matvec_d(st, v.data(), w.data());
    const double bj = b.back();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < D; ++i) w[i] -= bj * vprev[i];
    const double ai = par_dot(v.data(), w.data(), D);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < D; ++i) w[i] -= ai * v[i];
    const double bn = std::sqrt(par_dot(w.data(), w.data(), D));
    a.push_back(ai);
    const int m = (int)a.size();
    std::vector<double> ev(m);
    orc_tridiag_eigh(m, a.data(), b.data(), ev.data(), nullptr);
    enew = ev[0];
    bool conv = (it > 0 && std::fabs(enew - eold) <= tol * std::fabs(enew)) || bn < 1e-14;
    eold = enew;
    b.push_back(bn);
    if (conv) { ++it; break; }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < D; ++i) { vprev[i] = v[i]; v[i] = w[i] / bn; }
  }
  const int m = (int)a.size();
  std::vector<double> ev(m), Z((size_t)m * m);
  orc_tridiag_eigh(m, a.data(), b.data(), ev.data(), Z.data());
  *e0 = ev[0];
  if (alanc) for (int j = 0; j < m; ++j) alanc[j] = a[j];
  if (blanc) for (int j = 0; j < m; ++j) blanc[j] = b[j];
  if (evec) {
    for (int64_t i = 0; i < D; ++i) evec[i] = 0.0;
    for (int j = 0; j < m; ++j)
      for (int64_t i = 0; i < D; ++i) evec[i] += Z[j] * basis[j][i];
    double nn = 0.0;
    for (int64_t i = 0; i < D; ++i) nn += evec[i] * evec[i];
    nn = std::sqrt(nn);
    for (int64_t i = 0; i < D; ++i) evec[i] /= nn;
  }
  return m;
}

// ---------------------------------------------------------------- excitation operators
// GF excitation vector: the loops of lanc_build_gf_electrons_diag (src/GF/GF_ELECTRONS.f90:
// 241-245 for c^+, 267-271 for c) calling apply_op_CDG / apply_op_C (src/SECTOR.f90:217-268).
// op: +1 = c^+_{site,spin}, -1 = c_{site,spin}. site and spin are 1-based. The output
// vector (sector J) is overwritten; entries not reached stay zero. accumulate=1 adds
// instead (the (c_i + c_j) combination of lanc_build_gf_electrons_mix, :343-353).
void orc_apply_cop_d(int ns, int nupI, int ndwI, int op, int site, int spin, const double* psi, double* out, int accumulate) {
  Sector I, J;
  make_sector(ns, nupI, ndwI, &I);
  int nupJ = nupI + (spin == 1 ? op : 0), ndwJ = ndwI + (spin == 2 ? op : 0);
  make_sector(ns, nupJ, ndwJ, &J);
  if (!accumulate) for (int64_t j = 0; j < J.dim; ++j) out[j] = 0.0;
  const int pos = site - 1;
  for (int64_t i = 0; i < I.dim; ++i) {
    int64_t iup = i % I.dimup, idw = i / I.dimup;
    int64_t iud = spin == 1 ? I.mup[iup] : I.mdw[idw];
    if (op > 0 ? btest(iud, pos) != 0 : btest(iud, pos) != 1) continue;
    int64_t r; double sgn;
    if (op > 0) op_cdg(pos, iud, &r, &sgn); else op_c(pos, iud, &r, &sgn);
    int64_t jup = iup, jdw = idw;
    if (spin == 1) jup = bsearch_rec(J.mup.data(), J.dimup, r) - 1;
    else jdw = bsearch_rec(J.mdw.data(), J.dimdw, r) - 1;
    if (jup < 0 || jdw < 0) continue;
    int64_t j = jup + jdw * J.dimup;
    if (accumulate) out[j] += sgn * psi[i]; else out[j] = sgn * psi[i];
  }
}

// S^z_i |psi> and n_i |psi>: apply_op_Sz / apply_op_N (src/SECTOR.f90:271-341) in the loop of
// lanc_build_spinChi_diag (src/CHI/CHI_SPIN_ELECTRONS.f90:216-220). kind 0 = Sz, 1 = N.
// Sites are 1-based; site2 > 0 adds the second site (the _mix sum, :275-279).
void orc_apply_diagop_d(int ns, int nup, int ndw, int kind, int site, int site2, const double* psi, double* out) {
  Sector S; make_sector(ns, nup, ndw, &S);
  for (int64_t i = 0; i < S.dim; ++i) {
    int64_t mu = S.mup[i % S.dimup], md = S.mdw[i / S.dimup];
    auto f = [&](int s1) {
      int p = s1 - 1;
      return kind == 0 ? (btest(mu, p) - btest(md, p)) / 2.0 : double(btest(mu, p) + btest(md, p));
    };
    double sgn = f(site);
    if (site2 > 0) sgn += f(site2);
    out[i] = sgn * psi[i];
  }
}

// J|psi> of lanc_ed_build_oc (src/OC/OC_ELECTRONS.f90:139-205) for Norb=1: the bond
// (isite, isite+1) along the site chain, periodic, both spins, then the overall factor i.
// Real Hij: J|psi> = i * (real vector r); r is returned (out_im), the real part is zero.
void orc_apply_current_d(const orc_model* m, int nup, int ndw, const double* psi, double* out_im) {
  Sector S; make_sector(m->ns, nup, ndw, &S);
  const int ns = m->ns;
  for (int64_t j = 0; j < S.dim; ++j) out_im[j] = 0.0;
  for (int64_t i = 0; i < S.dim; ++i) {
    const int64_t iup = i % S.dimup, idw = i / S.dimup;
    const int64_t mup = S.mup[iup], mdw = S.mdw[idw];
    for (int isite = 0; isite < ns; ++isite) {
      int jsite = (isite + 1 == ns) ? 0 : isite + 1;
      for (int pass = 0; pass < 2; ++pass) {
        int io = pass == 0 ? isite : jsite, jo = pass == 0 ? jsite : isite;
        double pref = pass == 0 ? 1.0 : -1.0;  // + Hij c^+_i c_{i+1}  - conjg(Hij) c^+_{i+1} c_i
        double hu = hij(m, 1, io, jo).real(), hd = hij(m, 2, io, jo).real();
        if (btest(mup, jo) == 1 && btest(mup, io) == 0 && hu != 0.0) {
          int64_t k1, k2; double sg1, sg2;
          op_c(jo, mup, &k1, &sg1); op_cdg(io, k1, &k2, &sg2);
          int64_t jup = bsearch_rec(S.mup.data(), S.dimup, k2) - 1;
          out_im[jup + idw * S.dimup] += pref * hu * sg1 * sg2 * psi[i];
        }
        if (btest(mdw, jo) == 1 && btest(mdw, io) == 0 && hd != 0.0) {
          int64_t k1, k2; double sg1, sg2;
          op_c(jo, mdw, &k1, &sg1); op_cdg(io, k1, &k2, &sg2);
          int64_t jdw = bsearch_rec(S.mdw.data(), S.dimdw, k2) - 1;
          out_im[iup + jdw * S.dimup] += pref * hd * sg1 * sg2 * psi[i];
        }
      }
    }
  }
}

// ---------------------------------------------------------------- poles, weights, grids
// add_to_lanczos_gf_normal (src/GF/GF_ELECTRONS.f90:417-457), add_to_lanczos_spinChi
// (src/CHI/CHI_SPIN_ELECTRONS.f90:305-366) and add_to_lanczos_oc (src/OC/OC_ELECTRONS.f90:
// 223-263): eigh(T(a,b)), weight_j = norm2*Z(1,j)^2, pole_j = isign*(theta_j - Ei).
// GF uses isign=+1 (particle) / -1 (hole); CHI and OC use isign=+1.
void orc_poles_weights(int n, const double* alanc, const double* blanc, double norm2, double Ei, int isign,
                       double* poles, double* weights) {
  std::vector<double> w(n), Z((size_t)n * n);
  orc_tridiag_eigh(n, alanc, blanc, w.data(), Z.data());
  for (int j = 0; j < n; ++j) {
    weights[j] = Z[0 + (size_t)j * n] * Z[0 + (size_t)j * n] * norm2;
    poles[j] = isign * (w[j] - Ei);
  }
}

// Grids: allocate_grids (src/AUX_FUNX.f90:357-372).
void orc_grids(double temp, int lmats, int lreal, int ltau, double wini, double wfin, double* wm, double* vm,
               double* wr, double* vr, double* tau) {
  const double pi = 3.14159265358979323846;
  for (int i = 1; i <= lmats; ++i) wm[i - 1] = pi * temp * (2 * i - 1);
  for (int i = 0; i <= lmats; ++i) vm[i] = pi * temp * 2 * i;
  for (int i = 0; i < lreal; ++i) {
    wr[i] = lreal > 1 ? wini + (wfin - wini) * i / (lreal - 1) : wini;
    vr[i] = lreal > 1 ? 0.0 + (wfin - 0.0) * i / (lreal - 1) : 0.0;
  }
  for (int i = 0; i <= ltau; ++i) tau[i] = (1.0 / temp) * i / ltau;
}

// lanc_eval_gf_electrons inner sum (src/GF/GF_ELECTRONS.f90:503-508):
// G(iw) += p*w/(i*wm - e), G(w+i*eps) += p*w/(wr + i*eps - e). Outputs interleaved complex.
void orc_eval_gf(int npoles, const double* poles, const double* weights, double pesoBZ, int lmats, const double* wm,
                 int lreal, const double* wr, double eps, double* gmats, double* greal) {
  for (int k = 0; k < npoles; ++k) {
    const double peso = weights[k], de = poles[k];
    for (int i = 0; i < lmats; ++i) {
      zc g = pesoBZ * peso / (zc(0.0, wm[i]) - de);
      gmats[2 * i] += g.real(); gmats[2 * i + 1] += g.imag();
    }
    for (int i = 0; i < lreal; ++i) {
      zc g = pesoBZ * peso / (zc(wr[i], eps) - de);
      greal[2 * i] += g.real(); greal[2 * i + 1] += g.imag();
    }
  }
}

// lanc_eval_spinChi_electrons inner sums (src/CHI/CHI_SPIN_ELECTRONS.f90:420-446): chi(tau)
// symmetrised about beta/2 and chi(w) on vr. chi_iv evaluates the formula that the
// reference keeps commented out at :430-433 (bosonic Matsubara vm(0:lmats)).
void orc_eval_chi(int npoles, const double* poles, const double* weights, double pesoBZ, double beta, int ltau,
                  const double* tau, int lreal, const double* vr, double eps, int lmats, const double* vm,
                  double* chi_tau, double* chi_w, double* chi_iv) {
  for (int k = 0; k < npoles; ++k) {
    const double peso = weights[k] * pesoBZ, dE = poles[k];
    for (int i = 0; i <= ltau / 2 - 1; ++i) chi_tau[i] += peso * std::exp(-tau[i] * dE);
    chi_tau[ltau / 2] += peso * 0.5 * (std::exp(-tau[ltau / 2] * dE) + std::exp(-(beta - tau[ltau / 2]) * dE));
    for (int i = ltau / 2 + 1; i <= ltau; ++i) chi_tau[i] += peso * std::exp(-(beta - tau[i]) * dE);
    for (int i = 0; i < lreal; ++i) {
      zc c = -peso * (1.0 - std::exp(-beta * dE)) * (1.0 / (zc(vr[i], eps) - dE) - 1.0 / (zc(vr[i], eps) + dE));
      chi_w[2 * i] += c.real(); chi_w[2 * i + 1] += c.imag();
    }
    if (chi_iv) {
      if (beta * dE > 1e-3) chi_iv[0] += 2 * peso * (1.0 - std::exp(-beta * dE)) / dE;
      for (int i = 1; i <= lmats; ++i) chi_iv[2 * i] += peso * (1.0 - std::exp(-beta * dE)) * 2.0 * dE / (vm[i] * vm[i] + dE * dE);
    }
  }
}

// lanc_ed_eval_oc (src/OC/OC_ELECTRONS.f90:301-316): Drude sum and sigma(w) on vr with the
// reference's cutoff filters.
void orc_eval_oc(int npoles, const double* poles, const double* weights, double pesoBZ, double cutoff, int lreal,
                 const double* vr, double eps, double* drude, double* optcond) {
  for (int k = 0; k < npoles; ++k) {
    double peso = weights[k] * pesoBZ, dE = poles[k];
    double r = peso / dE;
    if (std::isnan(r) || std::isinf(r)) continue;
    if (std::fabs(dE) < cutoff) continue;
    if (std::fabs(r) < cutoff) continue;
    *drude += r;
    for (int i = 0; i < lreal; ++i) optcond[i] += r * eps / ((vr[i] - dE) * (vr[i] - dE) + eps * eps);
  }
}

// ---------------------------------------------------------------- observables
// lanc_observables inner loop (src/OBSERVABLES.f90:127-152) for one state with weight
// boltzman_weight/zeta folded into bw: dens, dens_up, dens_dw, docc, magz per site.
void orc_observables_d(int ns, int nup, int ndw, const double* psi, double bw, double* dens, double* dens_up,
                       double* dens_dw, double* docc, double* magz) {
  Sector S; make_sector(ns, nup, ndw, &S);
  for (int64_t i = 0; i < S.dim; ++i) {
    const double sw = psi[i] * psi[i];
    const int64_t mu = S.mup[i % S.dimup], md = S.mdw[i / S.dimup];
    for (int is = 0; is < ns; ++is) {
      double nu = btest(mu, is), nd = btest(md, is);
      dens[is] += (nu + nd) * sw * bw;
      dens_up[is] += nu * sw * bw;
      dens_dw[is] += nd * sw * bw;
      docc[is] += nu * nd * sw * bw;
      magz[is] += (nu - nd) * sw * bw;
    }
  }
}

// lanc_energy inner loop (src/ENERGY.f90:118-180 and :196-226, Norb=1 terms) for one real
// state with boltzman_weight/zeta folded into bw, accumulated into the outputs:
//  eknot    += sum_io Hdiag(spin,io) n_io           (ENERGY.f90:142-145)
//  ekin     += Hij(io,jo) sg1 sg2 psi(i) psi(j)      (up and down hops, :147-180)
//  epot     += Uloc n_up n_dw per site               (:182-188)
//  ehartree -= 0.5 Uloc (n_up + n_dw) when HFMODE    (:213-219)
// The caller adds ehartree to epot as ENERGY.f90:343 does.
void orc_energy_d(const orc_model* m, int nup, int ndw, const double* psi, double bw, double* ekin, double* epot,
                  double* eknot, double* ehartree) {
  const int ns = m->ns;
  Sector S; make_sector(ns, nup, ndw, &S);
  for (int64_t i = 0; i < S.dim; ++i) {
    const int64_t iup = i % S.dimup, idw = i / S.dimup;
    const int64_t mup = S.mup[iup], mdw = S.mdw[idw];
    const double sw = psi[i] * psi[i];
    for (int io = 0; io < ns; ++io) {
      *eknot += hij(m, 1, io, io).real() * btest(mup, io) * bw * sw;
      *eknot += hij(m, 2, io, io).real() * btest(mdw, io) * bw * sw;
    }
    for (int io = 0; io < ns; ++io)
      for (int jo = 0; jo < ns; ++jo) {
        if (hij(m, 1, io, jo) == zc(0.0) || !btest(mup, jo) || btest(mup, io)) continue;
        int64_t k1, k2; double sg1, sg2;
        op_c(jo, mup, &k1, &sg1);
        op_cdg(io, k1, &k2, &sg2);
        const int64_t jup = bsearch_rec(S.mup.data(), S.dimup, k2);
        const int64_t j = (jup - 1) + idw * S.dimup;
        *ekin += hij(m, 1, io, jo).real() * sg1 * sg2 * psi[i] * psi[j] * bw;
      }
    for (int io = 0; io < ns; ++io)
      for (int jo = 0; jo < ns; ++jo) {
        if (hij(m, 2, io, jo) == zc(0.0) || !btest(mdw, jo) || btest(mdw, io)) continue;
        int64_t k1, k2; double sg1, sg2;
        op_c(jo, mdw, &k1, &sg1);
        op_cdg(io, k1, &k2, &sg2);
        const int64_t jdw = bsearch_rec(S.mdw.data(), S.dimdw, k2);
        const int64_t j = iup + (jdw - 1) * S.dimup;
        *ekin += hij(m, 2, io, jo).real() * sg1 * sg2 * psi[i] * psi[j] * bw;
      }
    for (int io = 0; io < ns; ++io) *epot += m->uloc * btest(mup, io) * btest(mdw, io) * bw * sw;
    if (m->hfmode)
      for (int io = 0; io < ns; ++io) *ehartree -= 0.5 * m->uloc * (btest(mup, io) + btest(mdw, io)) * bw * sw;
  }
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
