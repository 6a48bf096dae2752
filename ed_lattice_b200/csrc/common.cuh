// common.cuh -- internal types of the sector-Lanczos engine (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <functional>
#include <string>
#include <vector>

#include "../../include/edgpu.h"

namespace edg {

constexpr int kMaxSites = 30;       // bitstrings fit int32 like the reference's `integer` maps
constexpr int kBinomN = kMaxSites + 2;

// Thread-local last-error text for edg_last_error().
void set_error(const char* fmt, ...);
const char* get_error();

#define EDG_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      ::edg::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
      return EDG_ERR_CUDA;                                                              \
    }                                                                                   \
  } while (0)

#define EDG_CHECK(expr)          \
  do {                           \
    int s_ = (expr);             \
    if (s_ != EDG_OK) return s_; \
  } while (0)

// Makes a sector's device current for the rest of the enclosing scope and gives the caller
// back its own current device on every return path: a host code that drives several GPUs
// from one thread must find its current device unchanged after any library call.
struct DeviceGuard {
  int prev = -1;
  bool switched = false;
  DeviceGuard() = default;
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
  int enter(int dev) {
    cudaError_t e = cudaGetDevice(&prev);
    if (e == cudaSuccess && prev != dev) {
      e = cudaSetDevice(dev);
      switched = e == cudaSuccess;
    }
    if (e != cudaSuccess) {
      set_error("selecting device %d: %s", dev, cudaGetErrorString(e));
      return EDG_ERR_CUDA;
    }
    return EDG_OK;
  }
  ~DeviceGuard() {
    if (switched) cudaSetDevice(prev);
  }
};
#define EDG_ON_DEVICE(dev)           \
  ::edg::DeviceGuard edg_dev_guard_; \
  EDG_CHECK(edg_dev_guard_.enter(dev))

// Stream-ordered buffers from a per-device pool that keeps freed memory for reuse; freed on
// the same stream when the owner goes out of scope. Every device buffer of the library comes
// from this pool: on a machine whose driver is busy with other processes, a plain
// cudaMalloc/cudaFree pair took up to 0.8 s, and a finite-temperature loop makes hundreds.
int pool_alloc(void** p, size_t bytes, cudaStream_t st, const char* what);
void pool_free(void* p, cudaStream_t st, size_t bytes);
int pool_trim(size_t keep);  // hand the pool's idle memory above `keep` back to the driver

// While one of these is alive on a thread, buffers released on that thread go back to the
// pool on `st` instead of the stream they were last allocated on. The sector destructor
// uses it after synchronising the sector's stream: a stream that a caller handed to the
// sector may no longer exist by then.
struct FreeStreamOverride {
  explicit FreeStreamOverride(cudaStream_t st);
  ~FreeStreamOverride();
  FreeStreamOverride(const FreeStreamOverride&) = delete;
  FreeStreamOverride& operator=(const FreeStreamOverride&) = delete;
  cudaStream_t prev;
  bool prev_set;
};
cudaStream_t free_stream(cudaStream_t recorded);

// One of a per-device set of library-owned streams, handed out round robin and never
// destroyed (creating a stream per sector stalled sector loops like cudaMalloc does).
cudaError_t pooled_stream(int dev, cudaStream_t* out);


// A device buffer that grows on demand. Allocation and release are ordered on the stream
// of the latest alloc() call: work queued on other streams must be finished (or ordered
// before that stream) when the buffer grows or is destroyed.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t st = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { reset(); }
  int alloc(size_t count, cudaStream_t stream, const char* what) {
    st = stream;
    if (n >= count && p) return EDG_OK;
    reset();
    if (count == 0) return EDG_OK;
    int s = pool_alloc(reinterpret_cast<void**>(&p), count * sizeof(T), stream, what);
    if (s == EDG_OK) n = count;
    return s;
  }
  void reset() {
    if (p) pool_free(p, free_stream(st), n * sizeof(T));
    p = nullptr;
    n = 0;
  }
};

// One spin species of a sector: basis maps, local energies and the gather hop table.
struct SpinBasis {
  int nel = 0;                  // Nup or Ndw
  int64_t dim = 0;              // C(Ns, nel)
  DevBuf<uint32_t> map;         // ascending bitstrings [dim]
  DevBuf<double> e64;           // local one-body energy of each configuration [dim]
  DevBuf<float> e32;
  // Gather hop table over target rows: row r lists (source rank, value) with
  // <r|H_sigma|src> = value, sources ascending. FORM_DIRECT keeps no table.
  DevBuf<uint32_t> off;         // [dim+1]
  DevBuf<uint32_t> src;         // [nnz]
  DevBuf<double> val64;         // [nnz]
  DevBuf<float> val32;
  DevBuf<double> val64i;        // [nnz] imaginary parts (complex Hij only)
  DevBuf<float> val32i;
  int64_t nnz = 0;
  // The same table in SELL-32 layout (slices of 32 consecutive target rows padded to the
  // slice's longest row, stored entry-major) so a warp reading the k-th entry of its 32
  // rows touches one 128-byte line.
  // Entry = src | sign << 31 (sign of hval; padding = src DimUp, a zero slot). Non-uniform
  // |values| keep a parallel value array.
  DevBuf<uint32_t> sell_ent;    // [sell_len]
  DevBuf<uint32_t> sell_off;    // [nslices+1], entry offsets, multiples of 32
  DevBuf<double> sell_v64;      // only when !sell_uniform
  DevBuf<float> sell_v32;
  bool sell_uniform = true;
  double sell_h = 0.0;
  // FP32 copy of the SELL table with each row's entries permuted so that, in every slot, the
  // lanes served together by one shared-memory wavefront read distinct banks (a bipartite
  // edge colouring of lanes x banks per lane group). Same rows and values; only the order
  // of the terms in each row's sum changes, so it is used for FP32 only. Empty when the
  // colouring would need too many slots.
  DevBuf<uint32_t> sched_ent;
  DevBuf<uint32_t> sched_off;
  int sched_rt = 0;             // rows-per-CTA of the FP32 up pass the schedule was built for
  bool sched_v4 = false;        // slots stored four per lane together (two 16-byte loads per batch)
  // Packed FP32 schedule (uniform tables, 2 * (DimUp + 32) <= 32768 slots): the conflict-free
  // slot schedule for two rows per CTA with slot counts rounded to 2 instead of 8, two 16-bit
  // entries per 32-bit word (entry 2k of a row in the low half of word k, 2k+1 in the high
  // half). An entry is the shared-memory slot of its source: src for a positive term,
  // p16_negoff + src for a negative one, where the up pass keeps the negated copy of the
  // staged rows, so no term applies a sign.
  DevBuf<uint32_t> p16_ent;     // words in SELL-32 slices, word-major
  DevBuf<uint32_t> p16_off;     // [nslices+1] word offsets, multiples of 32
  DevBuf<uint32_t> p16f_ent;    // the same words with the sign as bit 15 of each entry
  uint32_t p16_negoff = 0;      // 0: no packed schedule
  // Column-split copy of the SELL table for rows too long to stage whole in shared memory
  // (FP64 rows above 227 KB): part p lists, per slice, the entries whose source lies in
  // columns [split_col[p], split_col[p+1]), stored as source - split_col[p] (padding: the
  // part's width, a zero slot after the staged part). Concatenating the parts keeps each
  // row's sources ascending, so the summation order is that of the whole table.
  static constexpr int kMaxSplit = 8;
  int split_parts = 0;
  int64_t split_col[kMaxSplit + 1] = {};
  DevBuf<uint32_t> split_ent;   // parts concatenated
  DevBuf<uint32_t> split_off;   // [parts * (nslices + 1)]: part p's slice starts, then its end
  DevBuf<double> split_v64;     // only when !sell_uniform
  DevBuf<float> split_v32;
  int max_row = 0;              // longest hop list of any configuration
  // Down-spin pass work split: rows grouped into `groups` CTAs with near-equal total hop
  // counts (longest-processing-time-first assignment), CSR: group_off[groups+1], group_rows.
  // Contiguous row blocks for the block-staged down pass, one CTA each: block g owns rows
  // [off[g], off[g+1]), blocks balanced by hop count; rowblk[0] for 1024-thread CTAs (about
  // one per SM), rowblk[1] for 512-thread CTAs (about two per SM).
  struct RowBlocks {
    DevBuf<uint32_t> off;
    int count = 0;
    int max_rows = 0;
  };
  RowBlocks rowblk[2];
  DevBuf<uint32_t> group_off;
  DevBuf<uint32_t> group_rows;
  int groups = 0;
  int group_max = 0;            // most rows in one group
  // Kronecker schedule of the FP32 up pass (uniform real tables). The sites split at bit
  // kron_m into a low part (bits below kron_m) and a high part. Ascending order keeps the
  // configurations of one high part h together: a block of consecutive columns, one per low
  // part l. A hop inside the low part (LL) keeps h, so its source sits in the same block at
  // a column offset that depends on l only; a hop inside the high part (HH) keeps l and moves
  // to another block of the same size at an offset that depends on h only; the remaining
  // (cross) hops change both and keep a per-column list. Blocks are grouped by popcount(h)
  // ("group"), every block of a group has the same low parts, and block rows are numbered
  // group-major (krow). A thread of the up pass owns one low part l of one group and a run of
  // consecutive blocks of that group: its LL offsets stay in registers for the whole launch,
  // its HH offsets are shared with the lanes on the same block, and only its cross hops read
  // a per-column table.
  bool variants = false;          // the tables of the non-default kernels (rowblk, p16_*,
                                  // kron_*) are built (sector_variant_tables)
  int kron_m = 0;                 // 0: no Kronecker schedule
  int kron_nthr = 0;              // threads with work (of kKronThreads)
  int kron_lmax = 0;              // most blocks owned by one thread
  int kron_nkrow = 0, kron_nhent = 0;  // block rows, HH entries
  DevBuf<int4> kron_thr;          // per thread: first krow, blocks, low row (group base + lidx), lidx
  DevBuf<int32_t> kron_bcol;      // per krow: first column of the block
  DevBuf<uint32_t> kron_hoff;     // per krow: HH entry range [hoff[krow], hoff[krow+1])
  DevBuf<int32_t> kron_hent;      // HH entries: (column delta << 1) | sign
  DevBuf<int32_t> kron_lent;      // per thread: kKronLL LL slots (delta << 2) | valid << 1 | sign,
                                  // in bank-conflict-free slot order
  DevBuf<uint32_t> kron_xent;     // cross entries, warp by warp, step by step, lane-interleaved,
                                  // bank-conflict-free slot order: source column | sign << 31
                                  // (padding: a zero slot)
  DevBuf<uint32_t> kron_xoff;     // per warp: first slot
  DevBuf<uint32_t> kron_xwid;     // per warp and step (stride kron_lmax): slots
};

constexpr int64_t kFusedMaxDim = 500000;  // largest sector that defaults to the single-pass H x v
constexpr int kKronThreads = 512;  // threads per CTA of the Kronecker up pass
constexpr int kKronLL = 12;        // LL entries per low part held in registers
// Shared memory of the Kronecker up pass: rt staged rows plus the zero slots, then the block
// tables (first column and HH range per block row, HH entries).
inline size_t kron_smem(int64_t dimup, int rt, int nkrow, int nhent) {
  return size_t(dimup + 32) * rt * sizeof(float) + (size_t(2) * nkrow + 1 + nhent) * sizeof(int32_t);
}

// Directed bond list for one spin: Hij(a,b) != 0, a != b, value = matrix element used when
// an electron moves from b to a (direct form Hij(a,b), stored form conjg(Hij(a,b))).
struct BondList {
  int nb = 0;
  std::vector<int> a, b;
  std::vector<double> h, hi;  // Hij(a,b): real and imaginary parts
};

}  // namespace edg

struct edg_model_s {
  int ns = 0, nspin = 1;
  std::vector<double> hre[2], him[2];  // [spin-1][io*ns+jo]
  bool complex_hij = false;
  double uloc = 0, xmu = 0;
  int hfmode = 0, ed_filling = 0;
};

struct edg_sector_s {
  edg_model_s model;     // private copy: a sector outlives nothing it depends on
  int nup = 0, ndw = 0, form = EDG_FORM_STORED;
  int device = 0;
  int64_t dim = 0;
  edg::SpinBasis up, dw;
  edg::BondList bonds[2];
  edg::DevBuf<uint32_t> binom;    // C(n,k) table [kBinomN*kBinomN], exact integers
  edg::DevBuf<int32_t> bond_dev;  // device bond list for the direct form: [spin][a,b] packed
  edg::DevBuf<double> bondh_dev;
  edg::DevBuf<double> bondhi_dev;  // imaginary parts (complex Hij only)
  double U = 0;
  // Complex Hij: vectors are complex, stored interleaved (re, im), so every vector of the
  // sector holds vlen = 2*dim reals; the Lanczos scalars stay real (H is Hermitian).
  bool cplx = false;
  int64_t vlen = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t home_stream = nullptr;  // the library stream the sector was created on
  bool own_stream = false;
  // work space of the Lanczos drivers (grown on demand, freed with the sector)
  edg::DevBuf<double> w64[4];
  edg::DevBuf<float> w32[4];
  edg::DevBuf<double> red;        // reduction partials + device scalars
  edg::DevBuf<double> state;      // FP64 eigenvector kept on the device (ground_state_keep)
  edg::DevBuf<double> zstage;     // interleaved complex staging of the dd_sparse_HxV entry
  edg::DevBuf<float> basis32;     // FP32 Lanczos basis for Ritz vectors
  edg::DevBuf<double> blk64;      // block Lanczos: 3 blocks of k vectors (FP64 or FP32)
  edg::DevBuf<float> blk32;
  edg::DevBuf<double> blkred;     // block Lanczos scalars and reduction scratch
  edg::DevBuf<int> blkact;        // block Lanczos: active flag per column
  size_t basis32_cols = 0;
  bool has_state = false;
  int last_n32 = 0, last_n64 = 0;  // H x v applications of the last ground-state run per precision
  // H x v kernel choice per vector precision ([0] FP64, [1] FP32), set by edg_sector_autotune:
  // down pass 0 = hop-balanced row groups, 1 = block-staged (one CTA per SM), 2 = block-staged
  // (two CTAs per SM), 3 = single pass (k_hxv_fused: the whole H x v, no up pass); up pass
  // (FP32) 0 = 32-bit SELL schedule, 1 = packed 16-bit schedule with negated copies, 2 = packed
  // 16-bit schedule with sign bits, 3 = Kronecker schedule. Until tuned: 3/0 for real stored
  // sectors of at most kFusedMaxDim states, else 0/0.
  int hxv_dw[2] = {0, 0};
  int hxv_up[2] = {0, 0};
};

namespace edg {

// Rows per CTA of the shared-memory up pass for element size `elem` (4 or 8 bytes): four FP32
// rows if they fit two CTAs per SM (113 KB each), else two rows (two CTAs per SM if they fit,
// else one CTA of up to 227 KB), else one row with one CTA per SM, else 0 (the row does not
// fit; the L1-gather kernel takes over). On the 4x4 half-filled sector (DimUp 12870): FP32
// two rows with two CTAs per SM (four rows in one CTA measured 2.17 against 1.87 ms per
// H x v); FP64 two rows in one CTA (4.30 against 4.46 ms for one row with two CTAs). The
// staged rows carry 32 zero columns after DimUp (padding targets).
constexpr size_t kUpSmemTwoPerSM = 113 * 1024;
constexpr size_t kUpSmemOnePerSM = 227 * 1024;
constexpr int kUpZeroSlots = 32;
constexpr int kSellBatch = 8;  // SELL slice widths are multiples of this (entries loaded per batch)
inline int up_rows_per_cta(int64_t dimup, size_t elem) {
  const size_t row = size_t(dimup + kUpZeroSlots) * elem;
  if (elem == 4 && 4 * row <= kUpSmemTwoPerSM) return 4;
  if (2 * row <= kUpSmemOnePerSM) return 2;
  if (row <= kUpSmemOnePerSM) return 1;
  return 0;
}

// ---- basis.cu
int sector_build(edg_sector_s* s);
// builds, once, the tables of the non-default H x v kernels of a real stored sector
int sector_variant_tables(edg_sector_s* s);
uint64_t binom_host(int n, int k);

// ---- hxv.cu
template <typename T>
int hxv_apply(edg_sector_s* s, const T* v, T* hv);
template <typename T>
int hxv_cols(edg_sector_s* s, int64_t col0, int64_t ncols, const T* v, T* hv);
template <typename T>
int hxv_rows(edg_sector_s* s, int64_t row0, int64_t nrows, const T* v, T* hv);
template <typename T>
int hxv_apply_lz(edg_sector_s* s, const T* u, const T* uprev, T* w, const double* bn, int j, double* partial,
                 double* aout);
bool hxv_lz_available(const edg_sector_s* s, size_t elem);
template <typename T>
int hxv_autotune(edg_sector_s* s, int reps, double* ms, int* nc, int* best);
// Block forms over ncols vectors of the sector (column c at v + c*vlen): one launch per pass
// for all columns; columns whose device flag active[c] is 0 are skipped (active may be null).
// Available where the fused single-vector step is (hxv_lz_available).
template <typename T>
int hxv_block(edg_sector_s* s, int ncols, const int* active, const T* v, T* hv);
// Fused block step: per column, v_c = u_c / bn[c*sstride + j]; writes
// w_c = H v_c - (bn_j / bn_{j-1}) uprev_c and <v_c, w_c> into aout[c*sstride] (reduction
// scratch: partial + c*kRedSlots).
template <typename T>
int hxv_block_lz(edg_sector_s* s, int ncols, const int* active, const T* u, const T* uprev, T* w, const double* bn,
                 int64_t sstride, int j, double* partial, double* aout);

// ---- vecops.cu
constexpr int kRedBlocks = 592;  // 148 SMs x 4: fixed reduction grid (deterministic sums)
constexpr int kRedThreads = 256;
// A reduction scratch holds kRedBlocks partials and, at index kRedBlocks, the arrival counter
// of the fused finish (the last block of a reduction sums the partials and resets it to 0):
// kRedSlots doubles. The counter must be zero when the scratch is first used
// (red_scratch_reset).
constexpr int kRedSlots = kRedBlocks + 2;
int red_scratch_reset(cudaStream_t st, double* partial);
template <typename T>
int dot_dev(cudaStream_t st, const T* x, const T* y, int64_t n, double* partial, double* out);
template <typename T>
int lanczos_step_a(cudaStream_t st, T* w, const T* vprev, const T* v, const double* bprev, int64_t n,
                   double* partial, double* aout);
template <typename T>
int lanczos_step_b(cudaStream_t st, T* w, const T* v, const double* a, int64_t n, double* partial,
                   double* bout);
template <typename T>
int scale_into(cudaStream_t st, T* dst, const T* src, const double* b, int64_t n);
template <typename T>
int lanczos_step_b2(cudaStream_t st, T* w, const T* u, const double* a, const double* bn, int64_t n, double* partial,
                    double* bn_next);
int finish_dev(cudaStream_t st, const double* partial, int nblk, double* out, int do_sqrt);
// block forms (ncols columns: vectors vstride elements apart, device scalars sstride apart,
// reduction scratch kRedSlots apart; columns whose active[c] is 0 are skipped)
template <typename T>
int dot_cols(cudaStream_t st, int ncols, const T* x, const T* y, int64_t n, int64_t vstride, double* partial,
             double* out, int64_t sstride, int do_sqrt);
template <typename TD, typename TS>
int normalise_cols(cudaStream_t st, int ncols, TD* dst, int64_t dstride, const TS* src, int64_t srcstride,
                   const double* norm2, int64_t sstride, int64_t n);
template <typename T>
int lanczos_step_a_cols(cudaStream_t st, int ncols, const int* active, T* w, const T* vprev, const T* v,
                        int64_t vstride, const double* bprev, double* partial, double* aout, int64_t sstride, int64_t n);
template <typename T>
int lanczos_step_b_cols(cudaStream_t st, int ncols, const int* active, T* w, const T* v, int64_t vstride,
                        const double* a, double* partial, double* bout, int64_t sstride, int64_t n);
template <typename T>
int lanczos_step_b2_cols(cudaStream_t st, int ncols, const int* active, T* w, const T* u, int64_t vstride,
                         const double* a, const double* bn, double* partial, double* bn_next, int64_t sstride,
                         int64_t n);
template <typename T>
int scale_into_cols(cudaStream_t st, int ncols, const int* active, T* dst, const T* src, int64_t vstride,
                    const double* b, int64_t sstride, int64_t n);
// *out = |x| (FP64, fixed reduction grid; partial holds kRedBlocks values)
int norm_dev(cudaStream_t st, const double* x, int64_t n, double* partial, double* out);
// dst = TD(src * scale); dst and src must not overlap (scale_inplace_dev scales in place)
template <typename TD, typename TS>
int convert_dev(cudaStream_t st, TD* dst, const TS* src, int64_t n, double scale);
template <typename T>
int scale_inplace_dev(cudaStream_t st, T* x, int64_t n, double scale);
template <typename TD>
int axpy_accum_dev(cudaStream_t st, double* dst, const TD* x, double coef, int64_t n);
int random_dev(cudaStream_t st, double* dst, int64_t n, uint64_t seed);
int ritz_dev(cudaStream_t st, const float* basis, const double* z_dev, int m, int64_t n, double* x);
uint64_t splitmix64(uint64_t x);

// ---- lanczos.cu
int tridiag_dev(edg_sector_s* s, const double* dv0, int nlanc, double threshold, int precision,
                double* alanc, double* blanc, double* norm2, int* nsteps);
// k chains of one sector in lockstep (block H x V); start vectors dv0 + c*vlen (FP64, device);
// alanc/blanc [k][nlanc] on the host; falls back to one chain after another where the fused
// step is not available, and splits k into blocks that fit in free HBM.
int tridiag_block(edg_sector_s* s, int k, const double* dv0, int nlanc, double threshold, int precision,
                  double* alanc, double* blanc, double* norm2, int* nsteps);
// Same with the start vectors produced on demand: start(c, &x) points x at column c's FP64
// device vector, which need only stay valid until the next call (one shared buffer does).
using StartFn = std::function<int(int, const double**)>;
int tridiag_block_fn(edg_sector_s* s, int k, const StartFn& start, int nlanc, double threshold, int precision,
                     double* alanc, double* blanc, double* norm2, int* nsteps);

// ---- chains.cu
// k chains from the excitation vectors start(c) (FP64, device) of sector `to`: block
// tridiagonalisation (threshold 1e-9) and the poles isign*(theta_j - ei) / weights
// norm2*Z(1,j)^2 of each on the device; poles/weights [k][nlanc] on the host.
int chains_block(edg_sector_s* to, int k, const StartFn& start, int nlanc, int precision, double ei, int isign,
                 double* poles, double* weights, double* norm2, int* nout);
// poles and weights of k chains from host coefficients [k][nlanc] (one launch)
int poles_block(cudaStream_t st, int k, int nlanc, const double* alanc, const double* blanc, const double* norm2,
                const int* nsteps, double ei, int isign, double* poles, double* weights);
int ground_state(edg_sector_s* s, const double* v0_host, uint64_t seed, int maxit, double tol, int mode,
                 double* e0, int* niter);

// ---- lowest.cu
int lowest_k(edg_sector_s* s, int k, const double* v0_host, uint64_t seed, int maxit, double tol, int mode,
             double* evals,
             double* evecs_host, double* resid, int* niter);
int sector_dense(edg_sector_s* s, double* H_host);
int sector_dense_dev(edg_sector_s* s, double* dH);

// ---- tridiag_host.cpp
// zn (optional): last components of the eigenvectors (Ritz residual estimates b*|zn|).
int tridiag_eigh_host(int n, const double* d, const double* e, double* w, double* z1, double* zfull,
                      double* zn = nullptr);
// k lowest eigenvalues and |last eigenvector components| (bisection + twisted factorisation)
int tridiag_lowest_host(int n, const double* d, const double* e, int k, double* w, double* zn);
// k lowest eigenpairs (vectors z[k][n]) by bisection + twisted factorisation; EDG_ERR_NOCONV
// when two of the k+1 lowest eigenvalues are closer than relgap * spectral radius
int tridiag_lowest_vectors(int n, const double* d, const double* e, int k, double relgap, double* w, double* z);
// dense symmetric n x n (column-major A): eigenvalues w ascending, eigenvectors Z column-major
int sym_eigh_host(int n, const double* A, double* w, double* Z);

}  // namespace edg
