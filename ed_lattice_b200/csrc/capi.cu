// capi.cu -- the extern "C" boundary of libedgpu.so (declared in include/edgpu.h).
//
// Every entry validates its arguments, returns an EDG_* status and never aborts: the
// reference's `stop` statements on bad input (e.g. src/DIAG/HAMILTONIAN_DIRECT_HxV.f90:30-33,
// src/GRAPH_MATRIX.f90:325) become EDG_ERR_ARG with a message in edg_last_error().
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "common.cuh"

namespace edg {
int apply_cop(const edg_sector_s* from, const edg_sector_s* to, int op, int site, int spin, double coef,
              int accumulate, const double* din, double* dout, cudaStream_t st);
int apply_diagop(const edg_sector_s* s, int kind, const double* wsite, const double* din, double* dout,
                 cudaStream_t st);
int apply_current(const edg_sector_s* s, const double* din, double* dout, cudaStream_t st);
int energy(edg_sector_s* s, const double* psi, double weight, double* ekin, double* epot, double* eknot,
           double* ehartree);
int eval_poles(int64_t npoles, const double* poles, const double* weights, int64_t nz, const double* z_re,
               const double* z_im, double* out_re, double* out_im);
int observables(const edg_sector_s* s, const double* psi, double weight, double* dens, double* dens_up,
                double* dens_dw, double* docc, double* magz, cudaStream_t st);

// Sectors draw their stream from a per-device pool created on first use and kept until
// exit. Creating and destroying a stream per sector (hundreds in a finite-temperature run)
// stalled the process for up to a second at random; with the pool, up to kStreamPool sectors
// still run concurrently on separate streams.
constexpr int kStreamPool = 16;
constexpr int kMaxDevices = 64;
cudaError_t pooled_stream(int dev, cudaStream_t* out) {
  static std::mutex mu;
  static cudaStream_t pool[kMaxDevices][kStreamPool] = {};
  static unsigned next[kMaxDevices] = {};
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  const unsigned slot = next[dev]++ % kStreamPool;
  if (!pool[dev][slot]) {
    const cudaError_t e = cudaStreamCreateWithFlags(&pool[dev][slot], cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      pool[dev][slot] = nullptr;
      return e;
    }
  }
  *out = pool[dev][slot];
  return cudaSuccess;
}

}  // namespace edg

using namespace edg;

namespace {

#define EDG_ARG(cond, ...)         \
  do {                             \
    if (!(cond)) {                 \
      set_error(__VA_ARGS__);      \
      return EDG_ERR_ARG;          \
    }                              \
  } while (0)

__global__ void k_deinterleave(const double* __restrict__ z, double* __restrict__ re, double* __restrict__ im,
                               int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    re[i] = z[2 * i];
    im[i] = z[2 * i + 1];
  }
}
__global__ void k_interleave(double* __restrict__ z, const double* __restrict__ re, const double* __restrict__ im,
                             int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    z[2 * i] = re[i];
    z[2 * i + 1] = im[i];
  }
}

int grid1(int64_t n) {
  int64_t g = (n + 255) / 256;
  return int(g < 148 * 16 ? (g < 1 ? 1 : g) : 148 * 16);
}

int check_sector(const edg_sector_s* s) {
  if (!s) {
    set_error("null sector handle");
    return EDG_ERR_ARG;
  }
  return EDG_OK;
}

// Device vectors of a complex sector hold (re, im) pairs: 2*sizeof(T)-aligned.
template <typename T>
int check_vec_align(const edg_sector_s* s, const void* p, const char* what) {
  if (s->cplx && reinterpret_cast<uintptr_t>(p) % (2 * sizeof(T)) != 0) {
    set_error("%s: complex vectors must be %zu-byte aligned", what, 2 * sizeof(T));
    return EDG_ERR_ARG;
  }
  return EDG_OK;
}

// The slab H x v entries (edg_hxv_cols_dev_*, edg_hxv_rows_dev_*): argument checks, then
// hxv_cols / hxv_rows on the sector's stream.
template <typename T>
int slab_hxv(edg_sector* s, int cols, int64_t first, int64_t count, const T* dv, T* dhv, const char* what) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(dv && dhv && dv != dhv, "%s: bad vectors", what);
  const int64_t extent = cols ? s->up.dim : s->dw.dim;
  EDG_ARG(first >= 0 && count >= 0 && first + count <= extent, "%s: slab [%lld, %lld) outside [0, %lld)", what,
          (long long)first, (long long)(first + count), (long long)extent);
  if (count == 0) return EDG_OK;
  EDG_ON_DEVICE(s->device);
  return cols ? hxv_cols<T>(s, first, count, dv, dhv) : hxv_rows<T>(s, first, count, dv, dhv);
}
}  // namespace

extern "C" {

const char* edg_last_error(void) { return get_error(); }

int edg_device_count(int* n) {
  if (!n) return EDG_ERR_ARG;
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    *n = 0;
    set_error("cudaGetDeviceCount: %s", cudaGetErrorString(e));
    return EDG_ERR_NODEVICE;
  }
  *n = c;
  return c > 0 ? EDG_OK : EDG_ERR_NODEVICE;
}

int edg_model_create(int ns, int nspin, const double* hij_re, const double* hij_im, const double* hijdw_re,
                     const double* hijdw_im, double uloc, double xmu, int hfmode, int ed_filling, edg_model** out) {
  EDG_ARG(out != nullptr, "edg_model_create: out is NULL");
  *out = nullptr;
  EDG_ARG(ns >= 1 && ns <= kMaxSites, "edg_model_create: ns=%d outside 1..%d", ns, kMaxSites);
  EDG_ARG(nspin == 1 || nspin == 2, "edg_model_create: nspin=%d (1 or 2)", nspin);
  EDG_ARG(hij_re != nullptr, "edg_model_create: hij_re is NULL");
  EDG_ARG(nspin == 1 || hijdw_re != nullptr, "edg_model_create: nspin=2 needs hijdw_re");
  EDG_ARG(std::isfinite(uloc) && std::isfinite(xmu), "edg_model_create: non-finite U or xmu");
  edg_model_s* m = new (std::nothrow) edg_model_s();
  if (!m) return EDG_ERR_NOMEM;
  m->ns = ns;
  m->nspin = nspin;
  for (int sp = 0; sp < nspin; ++sp) {
    const double* re = sp == 0 ? hij_re : hijdw_re;
    const double* im = sp == 0 ? hij_im : hijdw_im;
    m->hre[sp].assign(re, re + ns * ns);
    if (im) m->him[sp].assign(im, im + ns * ns);
    for (int k = 0; k < ns * ns; ++k) {
      if (!std::isfinite(m->hre[sp][k]) || (im && !std::isfinite(im[k]))) {
        delete m;
        set_error("edg_model_create: non-finite Hij entry");
        return EDG_ERR_ARG;
      }
      if (im && im[k] != 0.0) m->complex_hij = true;
    }
    // Hij_build's Hermiticity assertion (src/GRAPH_MATRIX.f90:324-326), tolerance 1e-6
    for (int i = 0; i < ns; ++i)
      for (int j = 0; j < ns; ++j) {
        const double dr = m->hre[sp][i * ns + j] - m->hre[sp][j * ns + i];
        const double di = im ? im[i * ns + j] + im[j * ns + i] : 0.0;
        if (std::fabs(dr) > 1e-6 || std::fabs(di) > 1e-6) {
          delete m;
          set_error("Hij_build ERROR: Hij is not Hermitian (spin %d, %d,%d)", sp + 1, i + 1, j + 1);
          return EDG_ERR_ARG;
        }
      }
  }
  m->uloc = uloc;
  m->xmu = xmu;
  m->hfmode = hfmode ? 1 : 0;
  m->ed_filling = ed_filling;
  *out = m;
  return EDG_OK;
}

int edg_model_destroy(edg_model* m) {
  delete m;
  return EDG_OK;
}

// get_Sector / get_Nup / get_Ndw: src/SECTOR.f90:370-424
int edg_get_sector(int ns, int nup, int ndw) { return 1 + nup * (ns + 1) + ndw; }
int edg_get_nup(int ns, int isector) { return ((isector - 1) / (ns + 1)) % (ns + 1); }
int edg_get_ndw(int ns, int isector) { return (isector - 1) % (ns + 1); }

// binomial: src/SETUP.f90:336-358 (FP64 running product, rounded to nearest)
int64_t edg_binomial(int n, int k) {
  if (k < 0 || k > n) return 0;
  if (k == 0) return 1;
  double xh = 1.0;
  for (int i = 1; i <= k; ++i) xh = xh * double(n + 1 - i) / double(i);
  return int64_t(xh + 0.5);
}

int edg_sector_create(const edg_model* m, int nup, int ndw, int form, edg_sector** out) {
  EDG_ARG(out != nullptr, "edg_sector_create: out is NULL");
  *out = nullptr;
  EDG_ARG(m != nullptr, "edg_sector_create: model is NULL");
  EDG_ARG(nup >= 0 && nup <= m->ns && ndw >= 0 && ndw <= m->ns, "edg_sector_create: (Nup,Ndw)=(%d,%d) outside 0..%d",
          nup, ndw, m->ns);
  EDG_ARG(form == EDG_FORM_STORED || form == EDG_FORM_DIRECT, "edg_sector_create: form=%d", form);
  int ndev = 0;
  if (edg_device_count(&ndev) != EDG_OK) return EDG_ERR_NODEVICE;
  edg_sector_s* s = new (std::nothrow) edg_sector_s();
  if (!s) return EDG_ERR_NOMEM;
  s->model = *m;
  s->cplx = m->complex_hij;
  s->nup = nup;
  s->ndw = ndw;
  s->form = form;
  cudaError_t e = cudaGetDevice(&s->device);
  if (e == cudaSuccess) e = pooled_stream(s->device, &s->stream);
  s->home_stream = s->stream;
  if (e != cudaSuccess) {
    set_error("edg_sector_create: %s", cudaGetErrorString(e));
    delete s;
    return EDG_ERR_CUDA;
  }
  s->own_stream = false;  // pooled: never destroyed with the sector
  int st = sector_build(s);
  if (st != EDG_OK) {
    edg_sector_destroy(s);
    return st;
  }
  // Default H x v of a small real stored sector: the single pass (down-pass choice 3), whose
  // vectors sit in L2; from about 500,000 states up the two-pass kernels win (measured on the
  // 3x4 and 4x4 lattices: 0.0085 against 0.0146 ms FP64 at D = 48,400, 0.0515 against 0.0474
  // at D = 853,776). edg_sector_autotune and edg_sector_set_kernels override it.
  if (!s->cplx && s->form == EDG_FORM_STORED && s->dim <= kFusedMaxDim) s->hxv_dw[0] = s->hxv_dw[1] = 3;
  *out = s;
  return EDG_OK;
}

int edg_sector_destroy(edg_sector* s) {
  if (!s) return EDG_OK;
  DeviceGuard dg;
  (void)dg.enter(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  cudaStream_t st = s->stream;
  bool own = s->own_stream;
  {
    // nothing of the sector's is in flight now; its buffers go back to the pool on the
    // library's own stream (a caller's stream set by edg_sector_set_stream may be gone)
    FreeStreamOverride on(s->home_stream);
    delete s;
  }
  if (own && st) cudaStreamDestroy(st);
  return EDG_OK;
}

int edg_release_cached_memory(void) { return pool_trim(0); }

int edg_sector_release_work(edg_sector* s) {
  EDG_CHECK(check_sector(s));
  EDG_ON_DEVICE(s->device);
  if (s->stream) EDG_CUDA(cudaStreamSynchronize(s->stream));
  for (int k = 0; k < 4; ++k) {
    s->w64[k].reset();
    s->w32[k].reset();
  }
  s->zstage.reset();
  s->basis32.reset();
  s->basis32_cols = 0;
  s->blk64.reset();
  s->blk32.reset();
  s->blkred.reset();
  s->blkact.reset();
  return EDG_OK;
}

int edg_sector_vlen(const edg_sector* s, int64_t* vlen) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(vlen, "edg_sector_vlen: NULL");
  *vlen = s->vlen;
  return EDG_OK;
}

int edg_sector_dims(const edg_sector* s, int64_t* dim, int64_t* dimup, int64_t* dimdw) {
  EDG_CHECK(check_sector(s));
  if (dim) *dim = s->dim;
  if (dimup) *dimup = s->up.dim;
  if (dimdw) *dimdw = s->dw.dim;
  return EDG_OK;
}

int edg_sector_get_maps(const edg_sector* s, int32_t* map_up, int32_t* map_dw) {
  EDG_CHECK(check_sector(s));
  EDG_ON_DEVICE(s->device);
  cudaStream_t st = s->stream;
  if (map_up)
    EDG_CUDA(cudaMemcpyAsync(map_up, s->up.map.p, s->up.dim * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  if (map_dw)
    EDG_CUDA(cudaMemcpyAsync(map_dw, s->dw.map.p, s->dw.dim * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  EDG_CUDA(cudaStreamSynchronize(st));
  return EDG_OK;
}

int edg_sector_get_hops(const edg_sector* s, int spin, int64_t* rowptr, int32_t* cols, double* vals, int64_t* nnz) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(spin == 1 || spin == 2, "edg_sector_get_hops: spin=%d", spin);
  if (s->form != EDG_FORM_STORED) {
    set_error("edg_sector_get_hops: the direct form keeps no tables");
    return EDG_ERR_STATE;
  }
  EDG_ON_DEVICE(s->device);
  const SpinBasis& B = spin == 1 ? s->up : s->dw;
  if (nnz) *nnz = B.nnz;
  cudaStream_t st = s->stream;
  std::vector<uint32_t> off(rowptr ? B.dim + 1 : 0);
  if (rowptr)
    EDG_CUDA(cudaMemcpyAsync(off.data(), B.off.p, off.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  if (cols && B.nnz)
    EDG_CUDA(cudaMemcpyAsync(cols, B.src.p, B.nnz * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  if (vals && B.nnz)
    EDG_CUDA(cudaMemcpyAsync(vals, B.val64.p, B.nnz * sizeof(double), cudaMemcpyDeviceToHost, st));
  EDG_CUDA(cudaStreamSynchronize(st));
  for (size_t i = 0; i < off.size(); ++i) rowptr[i] = off[i];
  return EDG_OK;
}

int edg_sector_set_stream(edg_sector* s, void* stream) {
  EDG_CHECK(check_sector(s));
  EDG_ON_DEVICE(s->device);
  if (s->stream) EDG_CUDA(cudaStreamSynchronize(s->stream));
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  s->stream = static_cast<cudaStream_t>(stream);
  s->own_stream = false;
  return EDG_OK;
}

int edg_sector_autotune(edg_sector* s, int precision, int reps, double* ms, int* ncand, int* best) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(precision == EDG_PREC_F64 || precision == EDG_PREC_F32, "edg_sector_autotune: precision=%d", precision);
  EDG_ARG(reps >= 1 && reps <= 1000, "edg_sector_autotune: reps=%d", reps);
  EDG_ON_DEVICE(s->device);
  return precision == EDG_PREC_F32 ? hxv_autotune<float>(s, reps, ms, ncand, best)
                                   : hxv_autotune<double>(s, reps, ms, ncand, best);
}

int edg_sector_set_kernels(edg_sector* s, int precision, int candidate) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(precision == EDG_PREC_F64 || precision == EDG_PREC_F32, "edg_sector_set_kernels: precision=%d", precision);
  const int nup = precision == EDG_PREC_F32 ? 4 : 1;
  EDG_ARG(candidate >= 0 && candidate < 4 * nup, "edg_sector_set_kernels: candidate=%d outside 0..%d", candidate,
          4 * nup - 1);
  const int f32 = precision == EDG_PREC_F32;
  if (candidate != 0) {
    EDG_ON_DEVICE(s->device);
    EDG_CHECK(sector_variant_tables(s));
  }
  s->hxv_dw[f32] = candidate / nup;
  s->hxv_up[f32] = candidate % nup;
  return EDG_OK;
}

int edg_hxv_dev_f64(edg_sector* s, const double* dv, double* dhv) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(dv && dhv && dv != dhv, "edg_hxv_dev_f64: bad vectors");
  EDG_CHECK(check_vec_align<double>(s, dv, "edg_hxv_dev_f64"));
  EDG_CHECK(check_vec_align<double>(s, dhv, "edg_hxv_dev_f64"));
  EDG_ON_DEVICE(s->device);
  return hxv_apply<double>(s, dv, dhv);
}

int edg_hxv_dev_f32(edg_sector* s, const float* dv, float* dhv) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(dv && dhv && dv != dhv, "edg_hxv_dev_f32: bad vectors");
  EDG_CHECK(check_vec_align<float>(s, dv, "edg_hxv_dev_f32"));
  EDG_CHECK(check_vec_align<float>(s, dhv, "edg_hxv_dev_f32"));
  EDG_ON_DEVICE(s->device);
  return hxv_apply<float>(s, dv, dhv);
}

int edg_hxv_cols_dev_f64(edg_sector* s, int64_t col0, int64_t ncols, const double* dv, double* dhv) {
  return slab_hxv<double>(s, 1, col0, ncols, dv, dhv, "edg_hxv_cols_dev_f64");
}
int edg_hxv_cols_dev_f32(edg_sector* s, int64_t col0, int64_t ncols, const float* dv, float* dhv) {
  return slab_hxv<float>(s, 1, col0, ncols, dv, dhv, "edg_hxv_cols_dev_f32");
}
int edg_hxv_rows_dev_f64(edg_sector* s, int64_t row0, int64_t nrows, const double* dv, double* dhv) {
  return slab_hxv<double>(s, 0, row0, nrows, dv, dhv, "edg_hxv_rows_dev_f64");
}
int edg_hxv_rows_dev_f32(edg_sector* s, int64_t row0, int64_t nrows, const float* dv, float* dhv) {
  return slab_hxv<float>(s, 0, row0, nrows, dv, dhv, "edg_hxv_rows_dev_f32");
}

int edg_hxv_d(edg_sector* s, int64_t nloc, const double* v, double* hv) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(v && hv, "edg_hxv_d: NULL vector");
  if (s->cplx) {
    set_error("edg_hxv_d: complex Hij maps real vectors to complex ones; use edg_hxv_z");
    return EDG_ERR_ARG;
  }
  EDG_ARG(nloc == s->dim, "directMatVec ERROR: Nloc != dim(isector) (%lld vs %lld)", (long long)nloc,
          (long long)s->dim);
  EDG_ON_DEVICE(s->device);
  const int64_t n = s->dim;
  EDG_CHECK(s->w64[0].alloc(n, s->stream, "H x v input"));
  EDG_CHECK(s->w64[1].alloc(n, s->stream, "H x v output"));
  EDG_CUDA(cudaMemcpyAsync(s->w64[0].p, v, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  EDG_CHECK(hxv_apply<double>(s, s->w64[0].p, s->w64[1].p));
  EDG_CUDA(cudaMemcpyAsync(hv, s->w64[1].p, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  EDG_CUDA(cudaStreamSynchronize(s->stream));
  return EDG_OK;
}

int edg_hxv_z(edg_sector* s, int64_t nloc, const double* v, double* hv) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(v && hv, "edg_hxv_z: NULL vector");
  EDG_ARG(nloc == s->dim, "directMatVec ERROR: Nloc != dim(isector) (%lld vs %lld)", (long long)nloc,
          (long long)s->dim);
  EDG_ON_DEVICE(s->device);
  const int64_t n = s->dim;
  if (s->cplx) {  // complex H x v straight on the interleaved vector
    EDG_CHECK(s->w64[0].alloc(2 * n, s->stream, "H x v input"));
    EDG_CHECK(s->w64[1].alloc(2 * n, s->stream, "H x v output"));
    EDG_CUDA(cudaMemcpyAsync(s->w64[0].p, v, 2 * n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    EDG_CHECK(hxv_apply<double>(s, s->w64[0].p, s->w64[1].p));
    EDG_CUDA(cudaMemcpyAsync(hv, s->w64[1].p, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    EDG_CUDA(cudaStreamSynchronize(s->stream));
    return EDG_OK;
  }
  for (int k = 0; k < 4; ++k) EDG_CHECK(s->w64[k].alloc(n, s->stream, "H x v work"));
  EDG_CHECK(s->zstage.alloc(size_t(2 * n), s->stream, "complex staging"));
  double* stage = s->zstage.p;
  EDG_CUDA(cudaMemcpyAsync(stage, v, 2 * n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  k_deinterleave<<<grid1(n), 256, 0, s->stream>>>(stage, s->w64[0].p, s->w64[1].p, n);
  EDG_CUDA(cudaGetLastError());
  EDG_CHECK(hxv_apply<double>(s, s->w64[0].p, s->w64[2].p));
  EDG_CHECK(hxv_apply<double>(s, s->w64[1].p, s->w64[3].p));
  k_interleave<<<grid1(n), 256, 0, s->stream>>>(stage, s->w64[2].p, s->w64[3].p, n);
  EDG_CUDA(cudaGetLastError());
  EDG_CUDA(cudaMemcpyAsync(hv, stage, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  EDG_CUDA(cudaStreamSynchronize(s->stream));
  return EDG_OK;
}

int edg_tridiag_dev_f64(edg_sector* s, const double* dvinit, int nlanc, double threshold, int precision,
                        double* alanc, double* blanc, double* norm2, int* nsteps) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(dvinit && alanc && blanc && norm2 && nsteps, "edg_tridiag: NULL argument");
  EDG_ARG(nlanc >= 0, "edg_tridiag: nlanc=%d", nlanc);
  EDG_ARG(precision == EDG_PREC_F64 || precision == EDG_PREC_F32, "edg_tridiag: precision=%d", precision);
  EDG_CHECK(check_vec_align<double>(s, dvinit, "edg_tridiag_dev_f64"));
  EDG_ON_DEVICE(s->device);
  return tridiag_dev(s, dvinit, nlanc, threshold, precision, alanc, blanc, norm2, nsteps);
}

int edg_tridiag_d(edg_sector* s, const double* vvinit, int nlanc, double threshold, int precision, double* alanc,
                  double* blanc, double* norm2, int* nsteps) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(vvinit, "edg_tridiag_d: NULL start vector");
  EDG_ON_DEVICE(s->device);
  EDG_CHECK(s->w64[3].alloc(s->vlen, s->stream, "start vector"));
  EDG_CUDA(cudaMemcpyAsync(s->w64[3].p, vvinit, s->vlen * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  return edg_tridiag_dev_f64(s, s->w64[3].p, nlanc, threshold, precision, alanc, blanc, norm2, nsteps);
}

int edg_ground_state_keep(edg_sector* s, const double* v0, uint64_t seed, int maxit, double tol, int mode, double* e0,
                          int* niter) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(e0 && niter, "edg_ground_state: NULL output");
  EDG_ARG((mode & 0xff) == EDG_GS_F64 || (mode & 0xff) == EDG_GS_F32_REFINE, "edg_ground_state: mode=%d", mode);
  EDG_ARG(tol >= 0.0, "edg_ground_state: tol < 0");
  EDG_ON_DEVICE(s->device);
  return ground_state(s, v0, seed, maxit, tol, mode, e0, niter);
}

int edg_ground_state(edg_sector* s, const double* v0, uint64_t seed, int maxit, double tol, int mode, double* e0,
                     double* evec, int* niter) {
  EDG_CHECK(edg_ground_state_keep(s, v0, seed, maxit, tol, mode, e0, niter));
  if (evec) return edg_state_get(s, evec);
  return EDG_OK;
}

int edg_lowest_k_mode(edg_sector* s, int k, const double* v0, uint64_t seed, int maxit, double tol, int mode,
                      double* evals, double* evecs, double* resid, int* niter) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(evals && niter, "edg_lowest_k: NULL output");
  EDG_ARG(k >= 1 && k <= 16, "edg_lowest_k: k=%d outside 1..16", k);
  EDG_ARG(maxit >= 1, "edg_lowest_k: maxit=%d", maxit);
  EDG_ARG(tol > 0.0 && std::isfinite(tol), "edg_lowest_k: tol must be > 0");
  EDG_ARG(mode == EDG_LK_F64 || mode == EDG_LK_F32_REFINE, "edg_lowest_k: mode=%d", mode);
  EDG_ON_DEVICE(s->device);
  return lowest_k(s, k, v0, seed, maxit, tol, mode, evals, evecs, resid, niter);
}

int edg_lowest_k(edg_sector* s, int k, const double* v0, uint64_t seed, int maxit, double tol, double* evals,
                 double* evecs, double* resid, int* niter) {
  return edg_lowest_k_mode(s, k, v0, seed, maxit, tol, EDG_LK_F64, evals, evecs, resid, niter);
}

int edg_sector_dense(edg_sector* s, double* h) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(h, "edg_sector_dense: NULL");
  EDG_ON_DEVICE(s->device);
  return sector_dense(s, h);
}

int edg_sector_dense_dev(edg_sector* s, double* dh) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(dh, "edg_sector_dense_dev: NULL");
  EDG_ON_DEVICE(s->device);
  return sector_dense_dev(s, dh);
}

int edg_ground_state_stats(const edg_sector* s, int* n_f32, int* n_f64) {
  EDG_CHECK(check_sector(s));
  if (n_f32) *n_f32 = s->last_n32;
  if (n_f64) *n_f64 = s->last_n64;
  return EDG_OK;
}

int edg_state_get(const edg_sector* s, double* evec) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(evec, "edg_state_get: NULL");
  if (!s->has_state) {
    set_error("edg_state_get: the sector holds no state");
    return EDG_ERR_STATE;
  }
  EDG_ON_DEVICE(s->device);
  EDG_CUDA(cudaMemcpyAsync(evec, s->state.p, s->vlen * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  EDG_CUDA(cudaStreamSynchronize(s->stream));
  return EDG_OK;
}

int edg_state_set(edg_sector* s, const double* evec) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(evec, "edg_state_set: NULL");
  EDG_ON_DEVICE(s->device);
  EDG_CHECK(s->state.alloc(s->vlen, s->stream, "state"));
  EDG_CUDA(cudaMemcpyAsync(s->state.p, evec, s->vlen * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  EDG_CUDA(cudaStreamSynchronize(s->stream));
  s->has_state = true;
  return EDG_OK;
}

int edg_random_vector(uint64_t seed, int64_t n, double* out) {
  EDG_ARG(out || n == 0, "edg_random_vector: NULL");
  for (int64_t i = 0; i < n; ++i) {
    const uint64_t z = splitmix64(seed + uint64_t(i));
    out[i] = double(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
  }
  return EDG_OK;
}

int edg_apply_cop_dev_f64(const edg_sector* from, const edg_sector* to, int op, int site, int spin, double coef,
                          int accumulate, const double* din, double* dout) {
  EDG_CHECK(check_sector(from));
  EDG_CHECK(check_sector(to));
  EDG_ARG(from->cplx == to->cplx, "edg_apply_cop_dev_f64: the two sectors come from models of different Hij types");
  EDG_ARG(din && dout && din != dout, "edg_apply_cop: bad vectors");
  EDG_ARG(op == 1 || op == -1, "edg_apply_cop: op=%d", op);
  EDG_ARG(spin == 1 || spin == 2, "edg_apply_cop: spin=%d", spin);
  EDG_ARG(site >= 1 && site <= from->model.ns, "edg_apply_cop: site=%d", site);
  EDG_ARG(from->model.ns == to->model.ns, "edg_apply_cop: sectors of different lattices");
  const int nupJ = from->nup + (spin == 1 ? op : 0), ndwJ = from->ndw + (spin == 2 ? op : 0);
  EDG_ARG(to->nup == nupJ && to->ndw == ndwJ, "edg_apply_cop: target sector (%d,%d) is not (%d,%d)", to->nup, to->ndw,
          nupJ, ndwJ);
  EDG_ON_DEVICE(to->device);
  return apply_cop(from, to, op, site, spin, coef, accumulate, din, dout, to->stream);
}

int edg_apply_diagop_dev_f64(const edg_sector* s, int kind, int site, int site2, const double* qcos, const double* din,
                             double* dout) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(din && dout, "edg_apply_diagop: NULL vector");
  EDG_ARG(kind == 0 || kind == 1, "edg_apply_diagop: kind=%d", kind);
  const int ns = s->model.ns;
  std::vector<double> w(ns, 0.0);
  if (qcos) {
    for (int i = 0; i < ns; ++i) w[i] = qcos[i];
  } else {
    EDG_ARG(site >= 1 && site <= ns, "edg_apply_diagop: site=%d", site);
    EDG_ARG(site2 <= ns, "edg_apply_diagop: site2=%d", site2);
    w[site - 1] += 1.0;
    if (site2 > 0) w[site2 - 1] += 1.0;
  }
  EDG_ON_DEVICE(s->device);
  return apply_diagop(s, kind, w.data(), din, dout, s->stream);
}

int edg_apply_current_dev_f64(const edg_sector* s, const double* din, double* dout) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(din && dout && din != dout, "edg_apply_current: bad vectors");
  EDG_ON_DEVICE(s->device);
  return apply_current(s, din, dout, s->stream);
}

int edg_energy(edg_sector* s, double weight, double* ekin, double* epot, double* eknot, double* ehartree) {
  EDG_CHECK(check_sector(s));
  if (!s->has_state) {
    set_error("edg_energy: the sector holds no state");
    return EDG_ERR_STATE;
  }
  EDG_ARG(std::isfinite(weight), "edg_energy: weight is not finite");
  EDG_ON_DEVICE(s->device);
  return energy(s, s->state.p, weight, ekin, epot, eknot, ehartree);
}

int edg_observables(const edg_sector* s, double weight, double* dens, double* dens_up, double* dens_dw, double* docc,
                    double* magz) {
  EDG_CHECK(check_sector(s));
  if (!s->has_state) {
    set_error("edg_observables: the sector holds no state");
    return EDG_ERR_STATE;
  }
  EDG_ON_DEVICE(s->device);
  return observables(s, s->state.p, weight, dens, dens_up, dens_dw, docc, magz, s->stream);
}

int edg_tridiag_eigh(int n, const double* d, const double* e, double* w, double* z1) {
  EDG_ARG(n >= 0 && (n == 0 || (d && e && w)), "edg_tridiag_eigh: bad arguments");
  return tridiag_eigh_host(n, d, e, w, z1, nullptr);
}

int edg_tridiag_lowest(int n, const double* d, const double* e, int k, double* w, double* zn) {
  EDG_ARG(n >= 0 && k >= 0 && (n == 0 || k == 0 || (d && e && w)), "edg_tridiag_lowest: bad arguments");
  return tridiag_lowest_host(n, d, e, k, w, zn);
}

int edg_poles_weights(int n, const double* alanc, const double* blanc, double norm2, double ei, int isign,
                      double* poles, double* weights) {
  EDG_ARG(n >= 0 && (n == 0 || (alanc && blanc && poles && weights)), "edg_poles_weights: bad arguments");
  std::vector<double> w(n), z(n);
  EDG_CHECK(tridiag_eigh_host(n, alanc, blanc, w.data(), z.data(), nullptr));
  for (int j = 0; j < n; ++j) {
    weights[j] = z[j] * z[j] * norm2;
    poles[j] = isign * (w[j] - ei);
  }
  return EDG_OK;
}

static int finish_chain(edg_sector_s* s, const double* x, int nlanc, int precision, double ei, int isign,
                        double* poles, double* weights, double* norm2, int* nout) {
  std::vector<double> a(nlanc > 0 ? nlanc : 1), b(nlanc > 0 ? nlanc : 1);
  int steps = 0;
  EDG_CHECK(tridiag_dev(s, x, nlanc, 1e-9, precision, a.data(), b.data(), norm2, &steps));
  *nout = steps;
  if (steps == 0) return EDG_OK;
  return edg_poles_weights(steps, a.data(), b.data(), *norm2, ei, isign, poles, weights);
}

int edg_gf_chain(const edg_sector* from, edg_sector* to, int op, int site, int site2, int spin, int nlanc,
                 int precision, double ei, double* poles, double* weights, double* norm2, int* nout) {
  EDG_CHECK(check_sector(from));
  EDG_CHECK(check_sector(to));
  EDG_ARG(from->cplx == to->cplx, "edg_gf_chain: the two sectors come from models of different Hij types");
  EDG_ARG(poles && weights && norm2 && nout, "edg_gf_chain: NULL output");
  if (!from->has_state) {
    set_error("edg_gf_chain: origin sector holds no state");
    return EDG_ERR_STATE;
  }
  EDG_ON_DEVICE(to->device);
  EDG_CHECK(to->w64[3].alloc(to->vlen, to->stream, "excitation vector"));
  EDG_CHECK(edg_apply_cop_dev_f64(from, to, op, site, spin, 1.0, 0, from->state.p, to->w64[3].p));
  if (site2 > 0)
    EDG_CHECK(edg_apply_cop_dev_f64(from, to, op, site2, spin, 1.0, 1, from->state.p, to->w64[3].p));
  return finish_chain(to, to->w64[3].p, nlanc, precision, ei, op, poles, weights, norm2, nout);
}

int edg_chi_chain(edg_sector* s, int kind, int site, int site2, const double* qcos, int nlanc, int precision,
                  double ei, double* poles, double* weights, double* norm2, int* nout) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(poles && weights && norm2 && nout, "edg_chi_chain: NULL output");
  if (!s->has_state) {
    set_error("edg_chi_chain: sector holds no state");
    return EDG_ERR_STATE;
  }
  EDG_ON_DEVICE(s->device);
  EDG_CHECK(s->w64[3].alloc(s->vlen, s->stream, "excitation vector"));
  EDG_CHECK(edg_apply_diagop_dev_f64(s, kind, site, site2, qcos, s->state.p, s->w64[3].p));
  return finish_chain(s, s->w64[3].p, nlanc, precision, ei, 1, poles, weights, norm2, nout);
}

int edg_oc_chain(edg_sector* s, int nlanc, int precision, double ei, double* poles, double* weights, double* norm2,
                 int* nout) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(poles && weights && norm2 && nout, "edg_oc_chain: NULL output");
  if (!s->has_state) {
    set_error("edg_oc_chain: sector holds no state");
    return EDG_ERR_STATE;
  }
  EDG_ON_DEVICE(s->device);
  EDG_CHECK(s->w64[3].alloc(s->vlen, s->stream, "excitation vector"));
  EDG_CHECK(edg_apply_current_dev_f64(s, s->state.p, s->w64[3].p));
  return finish_chain(s, s->w64[3].p, nlanc, precision, ei, 1, poles, weights, norm2, nout);
}

int edg_eval_poles(int64_t npoles, const double* poles, const double* weights, int64_t nz, const double* z_re,
                   const double* z_im, double* out_re, double* out_im) {
  EDG_ARG(npoles >= 0 && nz >= 0, "edg_eval_poles: negative size");
  EDG_ARG((npoles == 0 || (poles && weights)) && (nz == 0 || (z_re && z_im && out_re && out_im)),
          "edg_eval_poles: NULL array");
  int ndev = 0;
  if (edg_device_count(&ndev) != EDG_OK || ndev == 0) {
    set_error("edg_eval_poles: no CUDA device");
    return EDG_ERR_NODEVICE;
  }
  return eval_poles(npoles, poles, weights, nz, z_re, z_im, out_re, out_im);
}

int edg_tridiag_block_dev(edg_sector* s, int k, const double* dvinit, int nlanc, double threshold, int precision,
                          double* alanc, double* blanc, double* norm2, int* nsteps) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(k >= 1 && dvinit && alanc && blanc && norm2 && nsteps, "edg_tridiag_block_dev: bad arguments");
  EDG_ARG(nlanc >= 0, "edg_tridiag_block_dev: nlanc=%d", nlanc);
  EDG_ARG(precision == EDG_PREC_F64 || precision == EDG_PREC_F32, "edg_tridiag_block_dev: precision=%d", precision);
  EDG_CHECK(check_vec_align<double>(s, dvinit, "edg_tridiag_block_dev"));
  EDG_ON_DEVICE(s->device);
  return tridiag_block(s, k, dvinit, nlanc, threshold, precision, alanc, blanc, norm2, nsteps);
}

int edg_gf_chain_block(const edg_sector* from, edg_sector* to, int op, int k, const int* sites, const int* sites2,
                       int spin, int nlanc, int precision, double ei, double* poles, double* weights, double* norm2,
                       int* nout) {
  EDG_CHECK(check_sector(from));
  EDG_CHECK(check_sector(to));
  EDG_ARG(k >= 1 && sites && poles && weights && norm2 && nout, "edg_gf_chain_block: bad arguments");
  EDG_ARG(nlanc >= 1, "edg_gf_chain_block: nlanc=%d", nlanc);
  EDG_ARG(precision == EDG_PREC_F64 || precision == EDG_PREC_F32, "edg_gf_chain_block: precision=%d", precision);
  if (!from->has_state) {
    set_error("edg_gf_chain_block: origin sector holds no state");
    return EDG_ERR_STATE;
  }
  for (int c = 0; c < k; ++c) {
    EDG_ARG(sites[c] >= 1 && sites[c] <= from->model.ns, "edg_gf_chain_block: sites[%d]=%d", c, sites[c]);
    EDG_ARG(!sites2 || sites2[c] <= from->model.ns, "edg_gf_chain_block: sites2[%d]=%d", c, sites2[c]);
  }
  EDG_ON_DEVICE(to->device);
  // one excitation vector at a time, each normalised into the block's own vectors
  DevBuf<double> X;
  EDG_CHECK(X.alloc(size_t(to->vlen), to->stream, "excitation vector"));
  StartFn start = [&](int c, const double** x) -> int {
    EDG_CHECK(edg_apply_cop_dev_f64(from, to, op, sites[c], spin, 1.0, 0, from->state.p, X.p));
    if (sites2 && sites2[c] > 0)
      EDG_CHECK(edg_apply_cop_dev_f64(from, to, op, sites2[c], spin, 1.0, 1, from->state.p, X.p));
    *x = X.p;
    return EDG_OK;
  };
  return chains_block(to, k, start, nlanc, precision, ei, op, poles, weights, norm2, nout);
}

int edg_chi_chain_block(edg_sector* s, int kind, int k, const int* sites, const int* sites2, const double* qcos,
                        int nlanc, int precision, double ei, double* poles, double* weights, double* norm2,
                        int* nout) {
  EDG_CHECK(check_sector(s));
  EDG_ARG(k >= 1 && (sites || qcos) && poles && weights && norm2 && nout, "edg_chi_chain_block: bad arguments");
  EDG_ARG(nlanc >= 1, "edg_chi_chain_block: nlanc=%d", nlanc);
  EDG_ARG(precision == EDG_PREC_F64 || precision == EDG_PREC_F32, "edg_chi_chain_block: precision=%d", precision);
  if (!s->has_state) {
    set_error("edg_chi_chain_block: sector holds no state");
    return EDG_ERR_STATE;
  }
  EDG_ON_DEVICE(s->device);
  DevBuf<double> X;
  EDG_CHECK(X.alloc(size_t(s->vlen), s->stream, "excitation vector"));
  const int ns = s->model.ns;
  StartFn start = [&](int c, const double** x) -> int {
    EDG_CHECK(edg_apply_diagop_dev_f64(s, kind, sites ? sites[c] : 1, sites2 ? sites2[c] : 0,
                                       qcos ? qcos + size_t(c) * ns : nullptr, s->state.p, X.p));
    *x = X.p;
    return EDG_OK;
  };
  return chains_block(s, k, start, nlanc, precision, ei, 1, poles, weights, norm2, nout);
}

int edg_poles_weights_block(int k, int nlanc, const double* alanc, const double* blanc, const double* norm2,
                            const int* nsteps, double ei, int isign, double* poles, double* weights) {
  EDG_ARG(k >= 0 && nlanc >= 0, "edg_poles_weights_block: negative size");
  EDG_ARG(k == 0 || nlanc == 0 || (alanc && blanc && norm2 && nsteps && poles && weights),
          "edg_poles_weights_block: NULL array");
  for (int c = 0; c < k; ++c)
    EDG_ARG(nsteps[c] >= 0 && nsteps[c] <= nlanc, "edg_poles_weights_block: nsteps[%d]=%d", c, nsteps[c]);
  int dev = 0;
  EDG_CUDA(cudaGetDevice(&dev));
  cudaStream_t st = nullptr;
  EDG_CUDA(pooled_stream(dev, &st));
  return poles_block(st, k, nlanc, alanc, blanc, norm2, nsteps, ei, isign, poles, weights);
}

}  // extern "C"
