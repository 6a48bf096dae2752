// noalloc.cu -- edg_tridiag_dev_f64_noalloc: the tridiagonalisation of edg_tridiag_dev_f64
// for callers that must not allocate device memory.
//
// Some hosts of this library cannot call cudaMalloc: a Fortran or C code that runs inside
// a memory pool or arena owned by another runtime (it hands out device pointers, and a
// second allocator would break its accounting), or a latency-critical loop that must never
// block on the driver's allocator. They still own their inputs and outputs. This entry
// point gives them the sector tridiagonalisation with every piece of scratch (the three
// Lanczos vectors, the reduction partials and the scalar slots) taken from one file-scope
// __device__ array of fixed size, so the call itself allocates nothing.
//
// Limits and sharing:
//  - vector length (the sector dimension, or twice it for a complex sector, whose vectors
//    hold (re, im) pairs) <= kNoAllocMaxDim (2^20 reals) and nlanc <= kNoAllocMaxLanc
//    (1024); larger requests return EDG_ERR_ARG. The array is 3*2^20 + 4096 doubles (about 25 MB)
//    and every GPU that loads the library holds it until the process exits.
//  - every call on a device uses the same array, which keeps the previous call's contents;
//    the call clears what must start at zero. Two calls that overlap on the GPU (two host
//    threads, or two streams) race on the array and must be serialised by the caller.
//  - the first call on each device looks up the array's device address with
//    cudaGetSymbolAddress (that device current); make that first call before any stream
//    capture begins.
#include <cmath>
#include <mutex>

#include "common.cuh"

namespace edg {
namespace {

constexpr int64_t kNoAllocMaxDim = int64_t(1) << 20;
constexpr int kNoAllocMaxLanc = 1024;
constexpr int64_t kNoAllocScalars = 4096;  // reduction scratch [kRedSlots] + a [cap] + b [cap+1] + slots
static_assert(kRedSlots + 2 * (kNoAllocMaxLanc + 1) + 8 <= kNoAllocScalars, "scalar area too small");

// The scratch: [V | P | W] vectors of kNoAllocMaxDim doubles, then the scalar area.
__device__ __align__(256) double g_noalloc_scratch[3 * kNoAllocMaxDim + kNoAllocScalars];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array for the current device (set up once per device).
int scratch_ptr(int device, double** out) {
  if (device < 0 || device >= kMaxDevices) {
    set_error("edg_tridiag_dev_f64_noalloc: device %d out of range", device);
    return EDG_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error("cudaGetSymbolAddress(g_noalloc_scratch): %s", cudaGetErrorString(e));
      return EDG_ERR_CUDA;
    }
    g_noalloc_ptr[device] = static_cast<double*>(p);
  }
  *out = g_noalloc_ptr[device];
  return EDG_OK;
}

}  // namespace
}  // namespace edg

using namespace edg;

extern "C" int edg_tridiag_dev_f64_noalloc(edg_sector* s, const double* dvinit, int nlanc, double threshold,
                                           double* alanc, double* blanc, double* norm2, int* nsteps) {
  if (!s || !dvinit || !alanc || !blanc || !norm2 || !nsteps) {
    set_error("edg_tridiag_dev_f64_noalloc: NULL argument");
    return EDG_ERR_ARG;
  }
  if (s->vlen > kNoAllocMaxDim || nlanc < 0 || nlanc > kNoAllocMaxLanc) {
    set_error("edg_tridiag_dev_f64_noalloc: vector length %lld > %lld or nlanc %d outside 0..%d", (long long)s->vlen,
              (long long)kNoAllocMaxDim, nlanc, kNoAllocMaxLanc);
    return EDG_ERR_ARG;
  }
  if (s->cplx && reinterpret_cast<uintptr_t>(dvinit) % (2 * sizeof(double)) != 0) {
    set_error("edg_tridiag_dev_f64_noalloc: complex vectors must be 16-byte aligned");
    return EDG_ERR_ARG;
  }
  EDG_ON_DEVICE(s->device);
  double* base = nullptr;
  EDG_CHECK(scratch_ptr(s->device, &base));
  const int64_t n = s->vlen;
  cudaStream_t st = s->stream;
  double* V = base;
  double* P = base + kNoAllocMaxDim;
  double* W = base + 2 * kNoAllocMaxDim;
  double* partial = base + 3 * kNoAllocMaxDim;
  double* A = partial + kRedSlots;
  double* B = A + nlanc + 1;  // b[0] = 0, b[j+1] written by step j; B[nlanc+1] holds norm2
  for (int j = 0; j < nlanc; ++j) { alanc[j] = 0.0; blanc[j] = 0.0; }
  *nsteps = 0;
  // the array keeps the previous call's contents: clear the scalar slots read before written
  // and the reduction's arrival counter
  EDG_CUDA(cudaMemsetAsync(A, 0, size_t(2 * (nlanc + 1) + 2) * sizeof(double), st));
  EDG_CHECK(red_scratch_reset(st, partial));
  EDG_CHECK(dot_dev<double>(st, dvinit, dvinit, n, partial, B + nlanc + 1));
  double n2 = 0.0;
  EDG_CUDA(cudaMemcpyAsync(&n2, B + nlanc + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
  EDG_CUDA(cudaStreamSynchronize(st));
  *norm2 = n2;
  if (n2 == 0.0 || nlanc == 0) return EDG_OK;
  EDG_CHECK((convert_dev<double, double>(st, V, dvinit, n, 1.0 / std::sqrt(n2))));
  EDG_CUDA(cudaMemsetAsync(P, 0, size_t(n) * sizeof(double), st));  // v_0 = 0
  for (int j = 0; j < nlanc; ++j) {
    EDG_CHECK(hxv_apply<double>(s, V, W));
    EDG_CHECK(lanczos_step_a<double>(st, W, P, V, B + j, n, partial, A + j));
    EDG_CHECK(lanczos_step_b<double>(st, W, V, A + j, n, partial, B + j + 1));
    double h[2];
    EDG_CUDA(cudaMemcpyAsync(&h[0], A + j, sizeof(double), cudaMemcpyDeviceToHost, st));
    EDG_CUDA(cudaMemcpyAsync(&h[1], B + j + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    EDG_CUDA(cudaStreamSynchronize(st));
    alanc[j] = h[0];
    *nsteps = j + 1;
    if (j + 1 < nlanc) blanc[j + 1] = h[1];
    if (!(h[1] >= threshold)) {
      if (j + 1 < nlanc) blanc[j + 1] = 0.0;
      break;
    }
    if (j + 1 == nlanc) break;
    EDG_CHECK(scale_into<double>(st, P, W, B + j + 1, n));
    double* t = P;
    P = V;
    V = t;
  }
  return EDG_OK;
}
