// basis.cu -- sector Fock basis, index maps and hop tables built on the device.
//
// Replaces build_sector (src/SECTOR.f90:69-115), the binary_search rank lookup
// (src/AUX_FUNX.f90:163-180) and the table construction of ed_buildh
// (src/DIAG/HAMILTONIAN_STORED_HxV.f90:21-126 with stored/H_local.f90, H_up.f90, H_dw.f90).
//
// Basis: the reference scans 0..2^Ns-1 and keeps popcount==N in ascending order. The same
// list is produced here without the 2^Ns scan: rank r -> bitstring by combinatorial
// unranking at the start of each thread's chunk, then Gosper's next-permutation step.
// Rank of a bitstring with set bits p_1<...<p_N is sum_i C(p_i, i) (the combinatorial number
// system), which equals its position in ascending order, i.e. binary_search's result - 1.
//
// Hop tables: gather form over target rows. For a target configuration t and a directed
// bond (a,b) with a occupied and b empty in t, the source is s = t - 2^a + 2^b and
// <t|H_sigma|s> = h(a,b) * (-1)^{popcount of t strictly between a and b}, which is the
// product sg1*sg2 of c(b) then cdg(a) in the reference (src/AUX_FUNX.f90:76-102).
// h(a,b) = Hij(a,b) for the direct form (direct/HxV_up.f90:24) and conjg(Hij(a,b)) for the
// stored form (stored/H_up.f90:20); both are real on the device.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <mutex>
#include <tuple>

#include "common.cuh"

namespace edg {

namespace {
thread_local char g_err[512] = "";
}

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
const char* get_error() { return g_err; }

// HBM admission: keep this many bytes free for the CUDA context, cuBLAS-free driver
// state and other users of the device.
static const size_t kReserveBytes = size_t(1) << 30;

// Stream-ordered allocations from a library-owned pool per device. The pool never hands
// memory back to the driver on its own: with a release threshold, every synchronisation
// returned the memory above it, and while one large buffer stayed alive (a sector's FP32
// basis) every solve's freed work space went back to the driver and came again through it,
// which stalls on a busy driver like cudaMalloc/cudaFree. Instead, freeing a buffer of
// kTrimBytes or more trims the pool's idle memory (beyond what is in use) to a quarter of the
// device memory (at least kPoolKeepBytes), and edg_release_cached_memory trims it on request. A request is refused
// when it would leave less than kReserveBytes of HBM free (memory held by the pool counts as
// used); the driver's free-memory query is skipped when the pool already holds enough idle
// memory for it.
namespace {
constexpr int kPoolDevices = 64;
constexpr uint64_t kPoolKeepBytes = uint64_t(8) << 30;
constexpr size_t kTrimBytes = size_t(1) << 30;
cudaMemPool_t g_pool[kPoolDevices] = {};
uint64_t g_pool_keep[kPoolDevices] = {};
std::mutex g_pool_mu;
thread_local cudaStream_t t_free_stream = nullptr;
thread_local bool t_free_override = false;
}  // namespace

FreeStreamOverride::FreeStreamOverride(cudaStream_t st) : prev(t_free_stream), prev_set(t_free_override) {
  t_free_stream = st;
  t_free_override = true;
}
FreeStreamOverride::~FreeStreamOverride() {
  t_free_stream = prev;
  t_free_override = prev_set;
}
cudaStream_t free_stream(cudaStream_t recorded) { return t_free_override ? t_free_stream : recorded; }

int pool_alloc(void** p, size_t bytes, cudaStream_t st, const char* what) {
  *p = nullptr;
  if (bytes == 0) return EDG_OK;
  int dev = 0;
  EDG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kPoolDevices) {
    set_error("%s: device %d outside the pool table (0..%d)", what, dev, kPoolDevices - 1);
    return EDG_ERR_CUDA;
  }
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pool[dev]) {
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      EDG_CUDA(cudaMemPoolCreate(&g_pool[dev], &props));
      size_t fr = 0, total = 0;
      EDG_CUDA(cudaMemGetInfo(&fr, &total));
      g_pool_keep[dev] = std::max<uint64_t>(kPoolKeepBytes, total / 4);
      uint64_t never = UINT64_MAX;
      EDG_CUDA(cudaMemPoolSetAttribute(g_pool[dev], cudaMemPoolAttrReleaseThreshold, &never));
    }
    pool = g_pool[dev];
  }
  size_t held = 0, used = 0;
  EDG_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &held));
  EDG_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
  const size_t idle = held > used ? held - used : 0;  // reusable without new device memory
  if (bytes > idle) {
    size_t freeb = 0, totalb = 0;
    EDG_CUDA(cudaMemGetInfo(&freeb, &totalb));
    if (bytes + kReserveBytes > freeb + idle) {
      set_error("HBM admission refused for %s: %zu bytes requested, %zu free", what, bytes, freeb + idle);
      return EDG_ERR_NOMEM;
    }
  }
  cudaError_t e = cudaMallocFromPoolAsync(p, bytes, pool, st);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    set_error("cudaMallocFromPoolAsync(%zu) for %s: %s", bytes, what, cudaGetErrorString(e));
    *p = nullptr;
    return EDG_ERR_NOMEM;
  }
  return EDG_OK;
}

void pool_free(void* p, cudaStream_t st, size_t bytes) {
  if (!p) return;
  cudaFreeAsync(p, st);
  if (bytes < kTrimBytes) return;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kPoolDevices) return;
  cudaMemPool_t pool = nullptr;
  uint64_t keep = 0;
  {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    pool = g_pool[dev];
    keep = g_pool_keep[dev];
  }
  if (!pool) return;
  // the trim target counts memory in use too: keep `keep` bytes idle on top of it
  size_t used = 0;
  if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess)
    cudaMemPoolTrimTo(pool, used + keep);
}

int pool_trim(size_t keep) {
  int dev = 0;
  EDG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kPoolDevices) return EDG_OK;
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    pool = g_pool[dev];
  }
  if (pool) {
    EDG_CUDA(cudaDeviceSynchronize());  // frees still queued on streams become trimmable
    EDG_CUDA(cudaMemPoolTrimTo(pool, keep));
  }
  return EDG_OK;
}

uint64_t binom_host(int n, int k) {
  if (k < 0 || k > n || n < 0) return 0;
  uint64_t r = 1;
  for (int i = 1; i <= k; ++i) r = r * uint64_t(n + 1 - i) / uint64_t(i);
  return r;
}

namespace {

struct EnergyParams {
  double eps[kMaxSites];  // Hdiag(io) - shift
};

__device__ __forceinline__ uint32_t binom_dev(const uint32_t* C, int n, int k) { return C[n * kBinomN + k]; }

__device__ __forceinline__ uint32_t rank_of(uint32_t s, const uint32_t* C) {
  uint32_t r = 0;
  int i = 1;
  while (s) {
    int p = __ffs(s) - 1;
    r += binom_dev(C, p, i);
    ++i;
    s &= s - 1;
  }
  return r;
}

__device__ __forceinline__ uint32_t unrank(uint64_t r, int k, int ns, const uint32_t* C) {
  uint32_t s = 0;
  for (int i = k; i >= 1; --i) {
    int p = i - 1;
    while (p + 1 < ns && binom_dev(C, p + 1, i) <= r) ++p;
    s |= 1u << p;
    r -= binom_dev(C, p, i);
  }
  return s;
}

__device__ __forceinline__ uint32_t gosper_next(uint32_t s) {
  uint32_t c = s & (0u - s);
  uint32_t r = s + c;
  return (((r ^ s) >> 2) / c) | r;
}

constexpr int kEnumChunk = 64;

__global__ void k_enum_map(uint32_t* map, int64_t dim, int k, int ns, const uint32_t* C) {
  int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  int64_t start = t * kEnumChunk;
  if (start >= dim) return;
  int64_t cnt = dim - start < kEnumChunk ? dim - start : kEnumChunk;
  uint32_t s = unrank(uint64_t(start), k, ns, C);
  for (int64_t j = 0; j < cnt; ++j) {
    map[start + j] = s;
    if (j + 1 < cnt) s = gosper_next(s);
  }
}

__global__ void k_local_energy(const uint32_t* map, int64_t dim, EnergyParams ep, double* e64, float* e32) {
  int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (r >= dim) return;
  uint32_t s = map[r];
  double e = 0.0;
  while (s) {
    int p = __ffs(s) - 1;
    e += ep.eps[p];
    s &= s - 1;
  }
  e64[r] = e;
  e32[r] = float(e);
}


__global__ void k_hop_count(const uint32_t* map, int64_t dim, const int32_t* bonds, int nb, uint32_t* cnt) {
  int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (r >= dim) return;
  uint32_t t = map[r];
  uint32_t c = 0;
  for (int k = 0; k < nb; ++k) {
    int a = bonds[2 * k], b = bonds[2 * k + 1];
    c += ((t >> a) & 1u) & (((t >> b) & 1u) ^ 1u);
  }
  cnt[r] = c;
}

__device__ __forceinline__ int between_parity(uint32_t t, int a, int b) {
  int lo = a < b ? a : b, hi = a < b ? b : a;
  uint32_t mask = ((hi >= 32 ? 0u : (1u << hi)) - 1u) & ~((2u << lo) - 1u);
  return __popc(t & mask) & 1;
}

// Row r of the stored hop table: sources ascending, value sign * Hij(a,b); with bhi (complex
// Hij) also the imaginary parts, stored as -sign * Im Hij(a,b): the stored form keeps
// conjg(Hij) (src/DIAG/stored/H_up.f90:19-21).
__global__ void k_hop_fill(const uint32_t* map, int64_t dim, const int32_t* bonds, const double* bh,
                           const double* bhi, int nb, const uint32_t* C, const uint32_t* off, uint32_t* src,
                           double* v64, float* v32, double* v64i, float* v32i) {
  int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (r >= dim) return;
  uint32_t t = map[r];
  uint32_t o = off[r];
  uint32_t n = 0;
  for (int k = 0; k < nb; ++k) {
    int a = bonds[2 * k], b = bonds[2 * k + 1];
    if (((t >> a) & 1u) && !((t >> b) & 1u)) {
      uint32_t s = (t & ~(1u << a)) | (1u << b);
      const bool neg = between_parity(t, a, b);
      double v = neg ? -bh[k] : bh[k];
      double vi = bhi ? (neg ? bhi[k] : -bhi[k]) : 0.0;
      uint32_t j = rank_of(s, C);
      // insertion into the row, ascending source rank (the reference's summation order)
      uint32_t pos = n;
      while (pos > 0 && src[o + pos - 1] > j) {
        src[o + pos] = src[o + pos - 1];
        v64[o + pos] = v64[o + pos - 1];
        if (bhi) v64i[o + pos] = v64i[o + pos - 1];
        --pos;
      }
      src[o + pos] = j;
      v64[o + pos] = v;
      if (bhi) v64i[o + pos] = vi;
      ++n;
    }
  }
  for (uint32_t q = 0; q < n; ++q) v32[o + q] = float(v64[o + q]);
  if (bhi)
    for (uint32_t q = 0; q < n; ++q) v32i[o + q] = float(v64i[o + q]);
}

int build_spin(edg_sector_s* s, int spin, SpinBasis& B, int nel) {
  const int ns = s->model.ns;
  B.nel = nel;
  B.dim = int64_t(binom_host(ns, nel));
  cudaStream_t st = s->stream;
  EDG_CHECK(B.map.alloc(B.dim, st, "basis map"));
  {
    int64_t nthr = (B.dim + kEnumChunk - 1) / kEnumChunk;
    int blocks = int((nthr + 255) / 256);
    k_enum_map<<<blocks, 256, 0, st>>>(B.map.p, B.dim, nel, ns, s->binom.p);
    EDG_CUDA(cudaGetLastError());
  }
  // local energies: Hdiag(io) = Re Hij(spin,io,io); the xmu / Hartree shift is applied
  // always in the stored form (stored/H_local.f90:62-89) and only for ed_filling==0 in the
  // direct form (direct/HxV_local.f90:63-92).
  const edg_model_s& m = s->model;
  const int sp = (m.nspin == 2) ? spin - 1 : 0;
  bool apply_shift = (s->form == EDG_FORM_STORED) || (m.ed_filling == 0);
  double shift = 0.0;
  if (apply_shift) {
    shift = m.xmu;
    if (m.hfmode && m.uloc != 0.0) shift += 0.5 * m.uloc;
  }
  EnergyParams ep{};
  for (int io = 0; io < ns; ++io) ep.eps[io] = m.hre[sp][io * ns + io] - shift;
  EDG_CHECK(B.e64.alloc(B.dim, st, "local energies"));
  EDG_CHECK(B.e32.alloc(B.dim, st, "local energies"));
  {
    int blocks = int((B.dim + 255) / 256);
    k_local_energy<<<blocks, 256, 0, st>>>(B.map.p, B.dim, ep, B.e64.p, B.e32.p);
    EDG_CUDA(cudaGetLastError());
  }
  // directed bond list (a created, b annihilated): Hij(a,b) != 0, a != b
  BondList& bl = s->bonds[spin - 1];
  bl = BondList();
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b < ns; ++b) {
      if (a == b) continue;
      double h = m.hre[sp][a * ns + b];
      double hi = m.him[sp].empty() ? 0.0 : m.him[sp][a * ns + b];
      if (h == 0.0 && hi == 0.0) continue;
      bl.a.push_back(a);
      bl.b.push_back(b);
      bl.h.push_back(h);
      bl.hi.push_back(hi);
    }
  bl.nb = int(bl.a.size());
  // Order bonds by d = 2^b - 2^a: the source of a hop is target + d, so this order yields
  // every row's sources in ascending rank (the reference's summation order) for free.
  std::vector<int> ord(bl.nb);
  for (int k = 0; k < bl.nb; ++k) ord[k] = k;
  std::sort(ord.begin(), ord.end(), [&](int x, int y) {
    const int64_t dx = (int64_t(1) << bl.b[x]) - (int64_t(1) << bl.a[x]);
    const int64_t dy = (int64_t(1) << bl.b[y]) - (int64_t(1) << bl.a[y]);
    return dx < dy;
  });
  BondList sorted;
  for (int k : ord) {
    sorted.a.push_back(bl.a[k]);
    sorted.b.push_back(bl.b[k]);
    sorted.h.push_back(bl.h[k]);
    sorted.hi.push_back(bl.hi[k]);
  }
  sorted.nb = bl.nb;
  bl = sorted;
  return EDG_OK;
}

int build_sell(edg_sector_s* s, SpinBasis& B);

int build_tables(edg_sector_s* s, int spin, SpinBasis& B) {
  cudaStream_t st = s->stream;
  const BondList& bl = s->bonds[spin - 1];
  const int nb = bl.nb;
  DevBuf<int32_t> bonds;
  DevBuf<double> bh, bhi;
  std::vector<int32_t> hb(2 * nb + 2);
  for (int k = 0; k < nb; ++k) { hb[2 * k] = bl.a[k]; hb[2 * k + 1] = bl.b[k]; }
  EDG_CHECK(bonds.alloc(hb.size(), st, "bond list"));
  EDG_CHECK(bh.alloc(nb + 1, st, "bond values"));
  EDG_CUDA(cudaMemcpyAsync(bonds.p, hb.data(), hb.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  if (nb) EDG_CUDA(cudaMemcpyAsync(bh.p, bl.h.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st));
  if (s->cplx) {
    EDG_CHECK(bhi.alloc(nb + 1, st, "bond values"));
    if (nb) EDG_CUDA(cudaMemcpyAsync(bhi.p, bl.hi.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  EDG_CHECK(B.off.alloc(B.dim + 1, st, "hop offsets"));
  DevBuf<uint32_t> cnt;
  EDG_CHECK(cnt.alloc(B.dim, st, "hop counts"));
  int blocks = int((B.dim + 255) / 256);
  k_hop_count<<<blocks, 256, 0, st>>>(B.map.p, B.dim, bonds.p, nb, cnt.p);
  EDG_CUDA(cudaGetLastError());
  EDG_CUDA(cudaMemsetAsync(B.off.p, 0, sizeof(uint32_t), st));
  size_t tmp_bytes = 0;
  EDG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, cnt.p, B.off.p + 1, B.dim, st));
  DevBuf<unsigned char> tmp;
  EDG_CHECK(tmp.alloc(tmp_bytes + 1, st, "scan scratch"));
  EDG_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tmp_bytes, cnt.p, B.off.p + 1, B.dim, st));
  uint32_t nnz = 0;
  EDG_CUDA(cudaMemcpyAsync(&nnz, B.off.p + B.dim, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  EDG_CUDA(cudaStreamSynchronize(st));
  B.nnz = nnz;
  EDG_CHECK(B.src.alloc(nnz + 1, st, "hop sources"));
  EDG_CHECK(B.val64.alloc(nnz + 1, st, "hop values"));
  EDG_CHECK(B.val32.alloc(nnz + 1, st, "hop values"));
  if (s->cplx) {
    EDG_CHECK(B.val64i.alloc(nnz + 1, st, "hop values"));
    EDG_CHECK(B.val32i.alloc(nnz + 1, st, "hop values"));
  }
  k_hop_fill<<<blocks, 256, 0, st>>>(B.map.p, B.dim, bonds.p, bh.p, s->cplx ? bhi.p : nullptr, nb, s->binom.p,
                                     B.off.p, B.src.p, B.val64.p, B.val32.p, B.val64i.p, B.val32i.p);
  EDG_CUDA(cudaGetLastError());
  EDG_CUDA(cudaStreamSynchronize(st));
  // the complex H x v gathers straight from this table; the SELL layouts serve the real kernels
  return s->cplx ? EDG_OK : build_sell(s, B);
}

// Proper edge colouring of a bipartite multigraph (left: lanes [0,G), right: banks [0,M))
// with max-degree colours (Konig's theorem), by the classic alternating-path recolouring:
// for edge (u,v) take colour a free at u and b free at v; if a is taken at v, swap a and b
// along the a/b path that starts at v (it cannot reach u), after which a is free at both.
// Returns the number of colours, or -1 when it would exceed kMaxColours.
static int edge_colour(int G, int M, const std::vector<std::pair<int, int>>& edges, std::vector<int>& colour) {
  constexpr int kMaxColours = 64;
  std::vector<int> dl(G, 0), db(M, 0);
  for (const auto& e : edges) { ++dl[e.first]; ++db[e.second]; }
  int D = 0;
  for (int x : dl) D = std::max(D, x);
  for (int x : db) D = std::max(D, x);
  if (D > kMaxColours) return -1;
  if (D == 0) return 0;
  std::vector<int> lc(size_t(G) * D, -1), bc(size_t(M) * D, -1);
  colour.assign(edges.size(), -1);
  std::vector<int> path;
  for (int e = 0; e < int(edges.size()); ++e) {
    const int u = edges[e].first, v = edges[e].second;
    int a = 0, b = 0;
    while (lc[size_t(u) * D + a] != -1) ++a;
    while (bc[size_t(v) * D + b] != -1) ++b;
    if (bc[size_t(v) * D + a] != -1) {
      path.clear();
      int x = v, c = a;
      bool on_bank = true;
      for (;;) {
        const int f = on_bank ? bc[size_t(x) * D + c] : lc[size_t(x) * D + c];
        if (f < 0) break;
        path.push_back(f);
        x = on_bank ? edges[f].first : edges[f].second;
        on_bank = !on_bank;
        c = (c == a) ? b : a;
      }
      for (int f : path) {
        lc[size_t(edges[f].first) * D + colour[f]] = -1;
        bc[size_t(edges[f].second) * D + colour[f]] = -1;
      }
      for (int f : path) {
        colour[f] = colour[f] == a ? b : a;
        lc[size_t(edges[f].first) * D + colour[f]] = f;
        bc[size_t(edges[f].second) * D + colour[f]] = f;
      }
    }
    colour[e] = a;
    lc[size_t(u) * D + a] = e;
    bc[size_t(v) * D + a] = e;
  }
  return D;
}

// Bank-conflict-free slot schedule of a uniform SELL table for the FP32 up pass with `rt`
// rows per CTA: a shared-memory wavefront serves G = 32/(rt) lanes reading rt*4-byte
// columns from M = G bank groups (column src sits in group src % M). Per slice and lane
// group, lanes x groups are edge-coloured; colour = slot. Lanes without an entry in a slot
// read one of the zero columns DimUp..DimUp+31 whose bank group is free in that slot.
// Slot c of lane l sits at c*32 + l of its slice, or, with v4, at (c/4)*128 + l*4 + c%4: a
// lane's slots 4i..4i+3 side by side, one 16-byte load (widths are multiples of 8).
static void build_schedule(int64_t dim, int rt, const std::vector<uint32_t>& off, const std::vector<uint32_t>& src,
                           const std::vector<uint32_t>& sgn, std::vector<uint32_t>& soff, std::vector<uint32_t>& ent,
                           bool* ok, int round_to = kSellBatch, bool v4 = false) {
  auto at = [v4](int c, int lane) -> size_t {
    return v4 ? size_t(c / 4) * 128 + size_t(lane) * 4 + size_t(c % 4) : size_t(c) * 32 + size_t(lane);
  };
  const int G = 32 / rt, M = G;
  const int64_t nsl = (dim + 31) / 32;
  soff.assign(nsl + 1, 0);
  ent.clear();
  *ok = true;
  for (int64_t sl = 0; sl < nsl; ++sl) {
    int width = 0;
    std::vector<std::vector<int>> grp_colour(32 / G);
    std::vector<std::vector<std::pair<int, int>>> grp_edges(32 / G);
    std::vector<std::vector<int>> grp_eidx(32 / G);
    for (int g = 0; g < 32 / G; ++g) {
      auto& E = grp_edges[g];
      auto& I = grp_eidx[g];
      for (int l = 0; l < G; ++l) {
        const int64_t r = sl * 32 + g * G + l;
        if (r >= dim) continue;
        for (uint32_t k = off[r]; k < off[r + 1]; ++k) {
          E.push_back({l, int(src[k] % uint32_t(M))});
          I.push_back(int(k));
        }
      }
      const int D = edge_colour(G, M, E, grp_colour[g]);
      if (D < 0) { *ok = false; return; }
      width = std::max(width, D);
    }
    const size_t base = ent.size();
    width = (width + round_to - 1) / round_to * round_to;  // whole batches: no bounds checks
    soff[sl + 1] = soff[sl] + 32u * uint32_t(width);
    ent.resize(base + size_t(32) * width, 0u);
    std::vector<char> used(size_t(width) * M);
    std::vector<char> filled(size_t(width) * 32);
    for (int g = 0; g < 32 / G; ++g) {
      std::fill(used.begin(), used.end(), 0);
      for (size_t q = 0; q < grp_edges[g].size(); ++q) {
        const int l = grp_edges[g][q].first, c = grp_colour[g][q], k = grp_eidx[g][q];
        const int lane = g * G + l;
        ent[base + at(c, lane)] = src[k] | (sgn[k] << 31);
        filled[size_t(c) * 32 + lane] = 1;
        used[size_t(c) * M + grp_edges[g][q].second] = 1;
      }
      for (int c = 0; c < width; ++c) {
        int free_bank = 0;
        while (free_bank < M && used[size_t(c) * M + free_bank]) ++free_bank;
        if (free_bank == M) free_bank = 0;  // every lane of the group has an entry: no padding here
        const uint32_t zcol = uint32_t(dim) + uint32_t((free_bank - int(dim % M) + M) % M);
        for (int l = 0; l < G; ++l)
          if (!filled[size_t(c) * 32 + g * G + l]) ent[base + at(c, g * G + l)] = zcol;
      }
    }
  }
}

// Kronecker split of one spin's gather table at bit m (SpinBasis::kron_*), planned on the
// host from the CSR rows and the basis map. Hops are classed by the two bits they move: both
// below m (LL), both at or above m (HH), else cross. Fails (returns false) when the table
// does not have the block structure the up pass relies on, or the schedule does not fit.
struct KronPlan {
  int m = 0;
  int64_t within = 0;                 // LL + HH hops
  std::vector<int4> thr;              // per thread: krow0, blocks, low row, lidx
  std::vector<int32_t> bcol;          // per krow
  std::vector<uint32_t> hoff;         // per krow + 1
  std::vector<int32_t> hent;
  std::vector<int32_t> lent;          // per thread: kKronLL slots
  std::vector<uint32_t> xent, xoff, xwid;
  int lmax = 0;
};

static bool plan_kron(int m, int rt, int64_t dim, const std::vector<uint32_t>& map, const std::vector<uint32_t>& off,
                      const std::vector<uint32_t>& src, const std::vector<uint32_t>& sgn, KronPlan& P) {
  const uint32_t mask = (1u << m) - 1u;
  // blocks of equal high part, in column order, then grouped by popcount(high part)
  std::vector<int64_t> bstart;        // per block (column order): first column
  std::vector<int> bgrp;
  for (int64_t c = 0; c < dim; ++c)
    if (c == 0 || (map[c] >> m) != (map[c - 1] >> m)) {
      bstart.push_back(c);
      bgrp.push_back(__builtin_popcount(map[c] >> m));
    }
  const int nblk = int(bstart.size());
  bstart.push_back(dim);
  const int G = 33;
  std::vector<int> gsize(G, -1), gcount(G, 0);
  for (int b = 0; b < nblk; ++b) {
    const int sz = int(bstart[b + 1] - bstart[b]);
    if (gsize[bgrp[b]] < 0) gsize[bgrp[b]] = sz;
    if (gsize[bgrp[b]] != sz) return false;  // blocks of one group must be alike
    ++gcount[bgrp[b]];
  }
  std::vector<int> gblk(G + 1, 0), glow(G + 1, 0);  // group-major bases of krow and low row
  for (int g = 0; g < G; ++g) {
    gblk[g + 1] = gblk[g] + gcount[g];
    glow[g + 1] = glow[g] + (gcount[g] ? gsize[g] : 0);
  }
  std::vector<int> krow_of(nblk), hidx_of(nblk), seen(G, 0);
  for (int b = 0; b < nblk; ++b) {
    hidx_of[b] = seen[bgrp[b]]++;
    krow_of[b] = gblk[bgrp[b]] + hidx_of[b];
  }
  const int nkrow = gblk[G], nlow = glow[G];
  P.m = m;
  P.within = 0;
  P.bcol.assign(nkrow, 0);
  std::vector<std::vector<int32_t>> hh(nkrow), ll(nlow);
  std::vector<char> hh_set(nkrow, 0), ll_set(nlow, 0);
  std::vector<std::vector<uint32_t>> cross(dim);
  for (int b = 0; b < nblk; ++b) {
    const int g = bgrp[b], kr = krow_of[b];
    P.bcol[kr] = int32_t(bstart[b]);
    for (int64_t c = bstart[b]; c < bstart[b + 1]; ++c) {
      const int lidx = int(c - bstart[b]), lr = glow[g] + lidx;
      std::vector<int32_t> myll, myhh;
      for (uint32_t k = off[c]; k < off[c + 1]; ++k) {
        const uint32_t d = map[c] ^ map[src[k]];
        const int64_t delta = int64_t(src[k]) - c;
        if ((d & mask) == d) myll.push_back(int32_t((delta << 1) | sgn[k]));
        else if ((d & mask) == 0) myhh.push_back(int32_t((delta << 1) | sgn[k]));
        else cross[c].push_back(src[k] | (sgn[k] << 31));
      }
      P.within += int64_t(myll.size() + myhh.size());
      if (!ll_set[lr]) { ll[lr] = myll; ll_set[lr] = 1; }
      else if (ll[lr] != myll) return false;
      if (!hh_set[kr]) { hh[kr] = myhh; hh_set[kr] = 1; }
      else if (hh[kr] != myhh) return false;
      if (int(myll.size()) > kKronLL) return false;
      for (int32_t e : myll)
        if ((e >> 1) < -32768 || (e >> 1) > 32767) return false;  // LL offsets are 16-bit in the up pass
    }
  }
  // thread schedule: a thread owns (group, lidx) and a run of consecutive blocks of the
  // group; runs of about equal length, the shortest length whose threads fit one CTA
  int64_t lanes = 0;
  for (int g = 0; g < G; ++g) lanes += gcount[g] ? gsize[g] : 0;
  if (lanes > kKronThreads) return false;
  int L = int((dim + kKronThreads - 1) / kKronThreads);
  for (;; ++L) {
    int64_t T = 0;
    for (int g = 0; g < G; ++g)
      if (gcount[g]) T += int64_t(gsize[g]) * ((gcount[g] + L - 1) / L);
    if (T <= kKronThreads) break;
  }
  P.thr.clear();
  P.lmax = 0;
  for (int g = 0; g < G; ++g) {
    if (!gcount[g]) continue;
    const int nch = (gcount[g] + L - 1) / L;
    for (int q = 0; q < nch; ++q) {
      const int h0 = int(int64_t(q) * gcount[g] / nch), h1 = int(int64_t(q + 1) * gcount[g] / nch);
      for (int lidx = 0; lidx < gsize[g]; ++lidx)
        P.thr.push_back(make_int4(gblk[g] + h0, h1 - h0, glow[g] + lidx, lidx));
      P.lmax = std::max(P.lmax, h1 - h0);
    }
  }
  // HH table
  P.hoff.assign(nkrow + 1, 0);
  P.hent.clear();
  for (int kr = 0; kr < nkrow; ++kr) {
    P.hent.insert(P.hent.end(), hh[kr].begin(), hh[kr].end());
    P.hoff[kr + 1] = uint32_t(P.hent.size());
  }
  P.hent.push_back(0);
  // A shared-memory wavefront of the up pass serves G = 32/rt lanes reading rt*4-byte
  // columns from M = G bank groups (column x sits in group x % M). Each thread's LL list and
  // each warp step's cross lists are put in slot order by an edge colouring of lanes x bank
  // groups (as the SELL schedule is), so that the lanes of a wavefront read distinct groups.
  const int Gl = 32 / rt, M = Gl, nwarps = kKronThreads / 32;
  const int nthr = int(P.thr.size());
  // LL: per thread, kKronLL slots of (delta << 2) | valid << 1 | sign. The group of an LL
  // source is (block start + lidx + delta) % M; lanes of one run share the block start, so
  // the colouring uses (lidx + delta) % M.
  P.lent.assign(size_t(kKronThreads) * kKronLL, 0);
  for (int w = 0; w < nwarps; ++w)
    for (int q = 0; q < 32 / Gl; ++q) {
      std::vector<std::pair<int, int>> E;
      std::vector<std::pair<int, int>> who;  // (thread, entry)
      for (int l = 0; l < Gl; ++l) {
        const int t = w * 32 + q * Gl + l;
        if (t >= nthr || P.thr[t].y == 0) continue;
        const auto& lst = ll[P.thr[t].z];
        for (int j = 0; j < int(lst.size()); ++j) {
          const int64_t col = int64_t(P.thr[t].w) + (lst[j] >> 1);
          E.push_back({l, int(((col % M) + M) % M)});
          who.push_back({t, j});
        }
      }
      std::vector<int> colour;
      const int D = E.empty() ? 0 : edge_colour(Gl, M, E, colour);
      std::vector<int> next(Gl, 0);
      for (size_t i = 0; i < who.size(); ++i) {
        const int t = who[i].first, j = who[i].second, l = t - w * 32 - q * Gl;
        const int slot = (D > 0 && D <= kKronLL) ? colour[i] : next[l]++;  // else natural order
        const int32_t e = ll[P.thr[t].z][j];
        P.lent[size_t(t) * kKronLL + slot] = ((e >> 1) << 2) | 2 | (e & 1);
      }
    }
  // cross entries, warp by warp and step by step, lane-interleaved; a lane without an entry
  // in a slot reads a zero slot dim + z whose bank group no lane of its wavefront uses there
  P.xoff.assign(nwarps + 1, 0);
  P.xwid.assign(size_t(nwarps) * P.lmax + 1, 0);
  P.xent.clear();
  for (int w = 0; w < nwarps; ++w) {
    P.xoff[w] = uint32_t(P.xent.size() / 32);
    for (int k = 0; k < P.lmax; ++k) {
      std::vector<const std::vector<uint32_t>*> mine(32, nullptr);
      for (int l = 0; l < 32; ++l) {
        const int t = w * 32 + l;
        if (t >= nthr || k >= P.thr[t].y) continue;
        mine[l] = &cross[size_t(P.bcol[P.thr[t].x + k]) + size_t(P.thr[t].w)];
      }
      std::vector<std::vector<int>> slot_of(32);
      int wd = 0;
      for (int q = 0; q < 32 / Gl; ++q) {
        std::vector<std::pair<int, int>> E;
        std::vector<std::pair<int, int>> who;
        for (int l = 0; l < Gl; ++l) {
          const int lane = q * Gl + l;
          if (!mine[lane]) continue;
          slot_of[lane].assign(mine[lane]->size(), 0);
          for (size_t j = 0; j < mine[lane]->size(); ++j) {
            E.push_back({l, int(((*mine[lane])[j] & 0x7fffffffu) % uint32_t(M))});
            who.push_back({lane, int(j)});
          }
        }
        std::vector<int> colour;
        const int D = E.empty() ? 0 : edge_colour(Gl, M, E, colour);
        if (D < 0) return false;
        for (size_t i = 0; i < who.size(); ++i) slot_of[who[i].first][who[i].second] = colour[i];
        wd = std::max(wd, D);
      }
      P.xwid[size_t(w) * P.lmax + k] = uint32_t(wd);
      const size_t base = P.xent.size();
      P.xent.resize(base + size_t(wd) * 32, 0xffffffffu);
      std::vector<char> used(size_t(wd) * 32 * M / Gl + 1, 0);  // [slot][group q][residue]
      const int ngr = 32 / Gl;
      for (int lane = 0; lane < 32; ++lane) {
        if (!mine[lane]) continue;
        for (size_t j = 0; j < mine[lane]->size(); ++j) {
          const uint32_t e = (*mine[lane])[j];
          const int sl = slot_of[lane][j];
          P.xent[base + size_t(sl) * 32 + lane] = e;
          used[(size_t(sl) * ngr + lane / Gl) * M + (e & 0x7fffffffu) % uint32_t(M)] = 1;
        }
      }
      for (int sl = 0; sl < wd; ++sl)
        for (int lane = 0; lane < 32; ++lane) {
          uint32_t& e = P.xent[base + size_t(sl) * 32 + lane];
          if (e != 0xffffffffu) continue;
          int fr = 0;
          const size_t u0 = (size_t(sl) * ngr + lane / Gl) * M;
          while (fr < M && used[u0 + fr]) ++fr;
          if (fr == M) fr = 0;
          e = uint32_t(dim) + uint32_t(((fr - int(dim % M)) % M + M) % M);
          used[u0 + fr] = 1;
        }
    }
  }
  P.xoff[nwarps] = uint32_t(P.xent.size() / 32);
  P.xent.push_back(uint32_t(dim));
  return true;
}

// Kronecker schedule of the FP32 up pass, for uniform real tables whose rows the up pass
// stages in shared memory: the split with the most hops inside a part among those that fit.
int build_kron(edg_sector_s* s, SpinBasis& B, const std::vector<uint32_t>& off, const std::vector<uint32_t>& src,
               const std::vector<uint32_t>& sgn) {
  cudaStream_t st = s->stream;
  B.kron_m = 0;
  const int ns = s->model.ns;
  const int64_t dim = B.dim;
  if (dim < 2 || B.nnz == 0 || up_rows_per_cta(dim, sizeof(float)) == 0 || ns < 2) return EDG_OK;
  std::vector<uint32_t> map(dim);
  EDG_CUDA(cudaMemcpyAsync(map.data(), B.map.p, dim * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  EDG_CUDA(cudaStreamSynchronize(st));
  const int rt = up_rows_per_cta(dim, sizeof(float));
  // Among the splits whose block tables fit in shared memory next to the staged rows: two
  // CTAs per SM when the rows alone allow it, then the most hops inside a part, then the
  // split nearer the middle. (A split near one end has blocks of one or two columns: nearly
  // every hop counts as HH, but its HH table is a per-column table again.)
  const bool two_rows_fit = size_t(dim + kUpZeroSlots) * rt * sizeof(float) <= kUpSmemTwoPerSM;
  auto score = [&](const KronPlan& P) {
    const size_t sm = kron_smem(dim, rt, int(P.bcol.size()), int(P.hent.size()));
    return std::make_tuple(int(!two_rows_fit || sm <= kUpSmemTwoPerSM), P.within, -std::abs(2 * P.m - ns));
  };
  KronPlan best, cand;
  for (int m = 1; m < ns; ++m) {
    if (!plan_kron(m, rt, dim, map, off, src, sgn, cand)) continue;
    if (kron_smem(dim, rt, int(cand.bcol.size()), int(cand.hent.size())) > kUpSmemOnePerSM) continue;
    if (best.m == 0 || score(cand) > score(best)) std::swap(best, cand);
  }
  if (best.m == 0) return EDG_OK;
  EDG_CHECK(B.kron_thr.alloc(kKronThreads, st, "Kronecker schedule"));
  std::vector<int4> thr(kKronThreads, make_int4(0, 0, 0, 0));
  std::copy(best.thr.begin(), best.thr.end(), thr.begin());
  EDG_CHECK(B.kron_bcol.alloc(best.bcol.size(), st, "Kronecker schedule"));
  EDG_CHECK(B.kron_hoff.alloc(best.hoff.size(), st, "Kronecker schedule"));
  EDG_CHECK(B.kron_hent.alloc(best.hent.size(), st, "Kronecker schedule"));
  EDG_CHECK(B.kron_lent.alloc(best.lent.size(), st, "Kronecker schedule"));
  EDG_CHECK(B.kron_xent.alloc(best.xent.size(), st, "Kronecker schedule"));
  EDG_CHECK(B.kron_xoff.alloc(best.xoff.size(), st, "Kronecker schedule"));
  EDG_CHECK(B.kron_xwid.alloc(best.xwid.size(), st, "Kronecker schedule"));
  auto up = [&](void* d, const void* h, size_t bytes) { return cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st); };
  EDG_CUDA(up(B.kron_thr.p, thr.data(), thr.size() * sizeof(int4)));
  EDG_CUDA(up(B.kron_bcol.p, best.bcol.data(), best.bcol.size() * sizeof(int32_t)));
  EDG_CUDA(up(B.kron_hoff.p, best.hoff.data(), best.hoff.size() * sizeof(uint32_t)));
  EDG_CUDA(up(B.kron_hent.p, best.hent.data(), best.hent.size() * sizeof(int32_t)));
  EDG_CUDA(up(B.kron_lent.p, best.lent.data(), best.lent.size() * sizeof(int32_t)));
  EDG_CUDA(up(B.kron_xent.p, best.xent.data(), best.xent.size() * sizeof(uint32_t)));
  EDG_CUDA(up(B.kron_xoff.p, best.xoff.data(), best.xoff.size() * sizeof(uint32_t)));
  EDG_CUDA(up(B.kron_xwid.p, best.xwid.data(), best.xwid.size() * sizeof(uint32_t)));
  EDG_CUDA(cudaStreamSynchronize(st));  // host plan goes out of scope
  B.kron_nthr = int(best.thr.size());
  B.kron_lmax = best.lmax;
  B.kron_nkrow = int(best.bcol.size());
  B.kron_nhent = int(best.hent.size());
  B.kron_m = best.m;
  return EDG_OK;
}

// Tables of the non-default H x v kernels (SpinBasis::rowblk, p16_*, kron_*), built from the
// device CSR on first use: edg_sector_autotune and edg_sector_set_kernels ask for them, the
// sector loops of a finite-temperature run (default kernels) never pay for them.
int build_variants(edg_sector_s* s, SpinBasis& B) {
  if (B.variants || s->cplx || B.dim == 0) return EDG_OK;
  cudaStream_t st = s->stream;
  const int64_t dim = B.dim;
  std::vector<uint32_t> off(dim + 1), src(B.nnz + 1);
  std::vector<double> val(B.nnz + 1);
  EDG_CUDA(cudaMemcpyAsync(off.data(), B.off.p, (dim + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  if (B.nnz) {
    EDG_CUDA(cudaMemcpyAsync(src.data(), B.src.p, B.nnz * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    EDG_CUDA(cudaMemcpyAsync(val.data(), B.val64.p, B.nnz * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  EDG_CUDA(cudaStreamSynchronize(st));
  const int64_t nsl = (dim + 31) / 32;
  const bool uniform = B.sell_uniform;
  const double hsgn = B.sell_h;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // contiguous blocks balanced by hops for the block-staged down pass, in two shapes: about
  // one block per SM (1024-thread CTAs) and two per SM (512-thread CTAs); each a multiple
  // of the SM count, enough blocks that one block's rows of a 256-column FP32 slab (1 KB per
  // row) stay within 112 KB per SM
  for (int shape = 0; shape < 2; ++shape) {
    const int per_sm = shape + 1;
    int64_t tot = 0;
    for (int64_t r = 0; r < dim; ++r) tot += 1 + int64_t(off[r + 1] - off[r]);
    int64_t CG = std::max<int64_t>(1, std::min<int64_t>(int64_t(sms) * per_sm, dim));
    std::vector<uint32_t> coff;
    int mx = 0;
    for (int iter = 0; iter < 16; ++iter) {
      coff.assign(1, 0u);
      int64_t acc = 0, g = 1;
      mx = 0;
      uint32_t start = 0;
      for (int64_t r = 0; r < dim; ++r) {
        acc += 1 + int64_t(off[r + 1] - off[r]);
        if (g < CG && acc * CG >= g * tot) {  // close block g-1 after row r
          coff.push_back(uint32_t(r + 1));
          mx = std::max<int>(mx, int(r + 1 - start));
          start = uint32_t(r + 1);
          ++g;
        }
      }
      coff.push_back(uint32_t(dim));
      mx = std::max<int>(mx, int(dim - start));
      if (mx <= 112 / per_sm || CG >= dim) break;
      CG = std::min<int64_t>(dim, CG + sms);
    }
    SpinBasis::RowBlocks& rb = B.rowblk[shape];
    rb.max_rows = mx;
    rb.count = int(coff.size() - 1);
    EDG_CHECK(rb.off.alloc(coff.size(), st, "row blocks"));
    EDG_CUDA(cudaMemcpyAsync(rb.off.p, coff.data(), coff.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    EDG_CUDA(cudaStreamSynchronize(st));
  }
  // Packed 16-bit schedule for the two-row FP32 up pass (slot counts rounded to 2)
  B.p16_negoff = 0;
  B.p16_ent.reset();
  B.p16_off.reset();
  B.p16f_ent.reset();
  {
    const uint32_t negoff = uint32_t((dim + kUpZeroSlots + 31) / 32 * 32);
    if (uniform && B.nnz > 0 && 2 * int64_t(negoff) <= 32768) {
      std::vector<uint32_t> sg(B.nnz);
      for (int64_t k = 0; k < B.nnz; ++k) sg[k] = (val[k] == hsgn) ? 0u : 1u;
      std::vector<uint32_t> qoff, qent;
      bool ok = false;
      build_schedule(dim, 2, off, src, sg, qoff, qent, &ok, 2);
      if (ok) {
        std::vector<uint32_t> woff(nsl + 1, 0), wn, wf;
        for (int64_t sl = 0; sl < nsl; ++sl) {
          const uint32_t width = (qoff[sl + 1] - qoff[sl]) / 32;  // even
          woff[sl + 1] = woff[sl] + 32 * (width / 2);
          for (uint32_t p = 0; p < width / 2; ++p)
            for (int l = 0; l < 32; ++l) {
              uint32_t en[2], ef[2];
              for (int h = 0; h < 2; ++h) {
                const uint32_t e = qent[qoff[sl] + (2 * p + h) * 32 + l];
                const uint32_t sidx = e & 0x7fffffffu, neg = e >> 31;
                en[h] = sidx + (neg ? negoff : 0u);
                ef[h] = sidx | (neg << 15);
              }
              wn.push_back(en[0] | (en[1] << 16));
              wf.push_back(ef[0] | (ef[1] << 16));
            }
        }
        wn.resize(wn.size() + 128, 0u);  // the up pass loads whole batches of 4 words past a slice's end
        wf.resize(wf.size() + 128, 0u);
        EDG_CHECK(B.p16_off.alloc(woff.size(), st, "packed schedule"));
        EDG_CHECK(B.p16_ent.alloc(wn.size(), st, "packed schedule"));
        EDG_CHECK(B.p16f_ent.alloc(wf.size(), st, "packed schedule"));
        EDG_CUDA(cudaMemcpyAsync(B.p16_off.p, woff.data(), woff.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        EDG_CUDA(cudaMemcpyAsync(B.p16_ent.p, wn.data(), wn.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        EDG_CUDA(cudaMemcpyAsync(B.p16f_ent.p, wf.data(), wf.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        EDG_CUDA(cudaStreamSynchronize(st));  // host vectors go out of scope
        B.p16_negoff = negoff;
      }
    }
  }
  if (uniform && B.nnz > 0) {
    std::vector<uint32_t> sg(B.nnz);
    for (int64_t k = 0; k < B.nnz; ++k) sg[k] = (val[k] == hsgn) ? 0u : 1u;
    EDG_CHECK(build_kron(s, B, off, src, sg));
  }
  B.variants = true;
  return EDG_OK;
}

// SELL-32 copy of a gather table, built on the host from the device CSR (the tables are
// O(DimUp) -- about 1 MB for a 4x4 lattice -- so this is a one-off of milliseconds).
int build_sell(edg_sector_s* s, SpinBasis& B) {
  cudaStream_t st = s->stream;
  const int64_t dim = B.dim;
  std::vector<uint32_t> off(dim + 1), src(B.nnz + 1);
  std::vector<double> val(B.nnz + 1);
  EDG_CUDA(cudaMemcpyAsync(off.data(), B.off.p, (dim + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  if (B.nnz) {
    EDG_CUDA(cudaMemcpyAsync(src.data(), B.src.p, B.nnz * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    EDG_CUDA(cudaMemcpyAsync(val.data(), B.val64.p, B.nnz * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  EDG_CUDA(cudaStreamSynchronize(st));
  const int64_t nsl = (dim + 31) / 32;
  B.max_row = 0;
  for (int64_t r = 0; r < dim; ++r) B.max_row = std::max<int>(B.max_row, int(off[r + 1] - off[r]));
  // LPT grouping of rows for the down-spin pass: one group per resident CTA (4 per SM)
  {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t G = std::max<int64_t>(1, std::min<int64_t>(int64_t(sms) * 4, dim));
    std::vector<int64_t> order(dim);
    for (int64_t r = 0; r < dim; ++r) order[r] = r;
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t x, int64_t y) { return off[x + 1] - off[x] > off[y + 1] - off[y]; });
    std::vector<std::pair<int64_t, int64_t>> heap;  // (load, group) min-heap
    for (int64_t g = 0; g < G; ++g) heap.push_back({0, g});
    auto cmp = [](const std::pair<int64_t, int64_t>& x, const std::pair<int64_t, int64_t>& y) { return x > y; };
    std::make_heap(heap.begin(), heap.end(), cmp);
    std::vector<std::vector<uint32_t>> members(G);
    for (int64_t r : order) {
      std::pop_heap(heap.begin(), heap.end(), cmp);
      auto& top = heap.back();
      members[top.second].push_back(uint32_t(r));
      top.first += 1 + int64_t(off[r + 1] - off[r]);  // diagonal + hops
      std::push_heap(heap.begin(), heap.end(), cmp);
    }
    std::vector<uint32_t> goff(G + 1, 0), grows;
    grows.reserve(dim);
    B.group_max = 0;
    for (int64_t g = 0; g < G; ++g) {
      std::sort(members[g].begin(), members[g].end());
      grows.insert(grows.end(), members[g].begin(), members[g].end());
      goff[g + 1] = uint32_t(grows.size());
      B.group_max = std::max<int>(B.group_max, int(members[g].size()));
    }
    B.groups = int(G);
    EDG_CHECK(B.group_off.alloc(G + 1, st, "row groups"));
    EDG_CHECK(B.group_rows.alloc(grows.size() + 1, st, "row groups"));
    EDG_CUDA(cudaMemcpyAsync(B.group_off.p, goff.data(), goff.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    EDG_CUDA(cudaMemcpyAsync(B.group_rows.p, grows.data(), grows.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    EDG_CUDA(cudaStreamSynchronize(st));
  }
  std::vector<uint32_t> soff(nsl + 1, 0);
  for (int64_t sl = 0; sl < nsl; ++sl) {
    uint32_t w = 0;
    for (int64_t r = sl * 32; r < std::min<int64_t>(dim, sl * 32 + 32); ++r) w = std::max(w, off[r + 1] - off[r]);
    w = (w + kSellBatch - 1) / kSellBatch * kSellBatch;
    soff[sl + 1] = soff[sl] + 32 * w;
  }
  double h0 = B.nnz ? std::fabs(val[0]) : 0.0;
  bool uniform = true;
  for (int64_t k = 0; k < B.nnz; ++k)
    if (std::fabs(val[k]) != h0) { uniform = false; break; }
  const double hsgn = B.nnz ? (val[0] < 0 ? -h0 : h0) : 0.0;  // value encoded by code 0
  // entry: bit 31 = sign (uniform tables), bits 0..30 = source; padding points at the
  // zero slot dim that the up pass keeps after the staged rows
  std::vector<uint32_t> ent(soff[nsl] + 1, uint32_t(dim));
  std::vector<double> sv(uniform ? 0 : soff[nsl] + 1, 0.0);
  for (int64_t r = 0; r < dim; ++r) {
    const int64_t sl = r / 32, lane = r % 32;
    for (uint32_t k = 0; k < off[r + 1] - off[r]; ++k) {
      const uint32_t e = off[r] + k;
      const size_t pos = soff[sl] + size_t(k) * 32 + lane;
      uint32_t sign = 0;
      if (uniform) sign = (val[e] == hsgn) ? 0u : 1u;
      else sv[pos] = val[e];
      ent[pos] = src[e] | (sign << 31);
    }
  }
  B.sell_uniform = uniform;
  B.sell_h = hsgn;
  // FP32 conflict-free schedule (uniform tables whose rows fit the shared-memory up pass)
  B.sched_rt = 0;
  B.sched_v4 = false;
  B.sched_ent.reset();
  B.sched_off.reset();
  const int rt32 = up_rows_per_cta(dim, sizeof(float));
  if (uniform && rt32 > 0 && B.nnz > 0) {
    std::vector<uint32_t> sg(B.nnz);
    for (int64_t k = 0; k < B.nnz; ++k) sg[k] = (val[k] == hsgn) ? 0u : 1u;
    std::vector<uint32_t> qoff, qent;
    bool ok = false;
    // the two-CTA form of the up pass loads its entries four slots at a time
    const bool v4 = size_t(dim + kUpZeroSlots) * rt32 * sizeof(float) <= kUpSmemTwoPerSM;
    build_schedule(dim, rt32, off, src, sg, qoff, qent, &ok, kSellBatch, v4);
    if (ok) {
      B.sched_v4 = v4;
      qent.push_back(uint32_t(dim));
      EDG_CHECK(B.sched_off.alloc(qoff.size(), st, "SELL schedule"));
      EDG_CHECK(B.sched_ent.alloc(qent.size(), st, "SELL schedule"));
      EDG_CUDA(cudaMemcpyAsync(B.sched_off.p, qoff.data(), qoff.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
      EDG_CUDA(cudaMemcpyAsync(B.sched_ent.p, qent.data(), qent.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
      B.sched_rt = rt32;
    }
  }
  // column-split copy for rows that do not fit shared memory whole (FP64 rows above 227 KB)
  B.split_parts = 0;
  if (up_rows_per_cta(dim, sizeof(double)) == 0 && B.nnz > 0) {
    const int64_t cap = int64_t(kUpSmemOnePerSM / sizeof(double)) - kUpZeroSlots;
    const int P = int((dim + cap - 1) / cap);
    if (P <= SpinBasis::kMaxSplit) {
      const int64_t wpart = (dim + P - 1) / P;
      for (int p = 0; p <= P; ++p) B.split_col[p] = std::min<int64_t>(dim, p * wpart);
      std::vector<uint32_t> poff(size_t(P) * (nsl + 1), 0), pent;
      std::vector<double> pval;
      std::vector<uint32_t> lo(32), hi(32);
      size_t base = 0;
      for (int p = 0; p < P; ++p) {
        const uint32_t c0 = uint32_t(B.split_col[p]), c1 = uint32_t(B.split_col[p + 1]);
        for (int64_t sl = 0; sl < nsl; ++sl) {
          poff[size_t(p) * (nsl + 1) + sl] = uint32_t(base);
          uint32_t w = 0;
          for (int l = 0; l < 32; ++l) {
            const int64_t r = sl * 32 + l;
            lo[l] = hi[l] = 0;
            if (r >= dim) continue;
            const uint32_t* b0 = src.data() + off[r];
            const uint32_t* b1 = src.data() + off[r + 1];
            lo[l] = uint32_t(std::lower_bound(b0, b1, c0) - src.data());
            hi[l] = uint32_t(std::lower_bound(b0, b1, c1) - src.data());
            w = std::max(w, hi[l] - lo[l]);
          }
          w = (w + kSellBatch - 1) / kSellBatch * kSellBatch;
          pent.resize(base + size_t(32) * w, c1 - c0);
          if (!uniform) pval.resize(base + size_t(32) * w, 0.0);
          for (int l = 0; l < 32; ++l)
            for (uint32_t k = lo[l]; k < hi[l]; ++k) {
              const size_t pos = base + size_t(k - lo[l]) * 32 + l;
              const uint32_t sign = uniform ? ((val[k] == hsgn) ? 0u : 1u) : 0u;
              pent[pos] = (src[k] - c0) | (sign << 31);
              if (!uniform) pval[pos] = val[k];
            }
          base += size_t(32) * w;
        }
        poff[size_t(p) * (nsl + 1) + nsl] = uint32_t(base);
      }
      pent.push_back(0u);
      EDG_CHECK(B.split_off.alloc(poff.size(), st, "split SELL offsets"));
      EDG_CHECK(B.split_ent.alloc(pent.size(), st, "split SELL entries"));
      EDG_CUDA(cudaMemcpyAsync(B.split_off.p, poff.data(), poff.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
      EDG_CUDA(cudaMemcpyAsync(B.split_ent.p, pent.data(), pent.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
      if (!uniform) {
        pval.push_back(0.0);
        std::vector<float> pv32(pval.begin(), pval.end());
        EDG_CHECK(B.split_v64.alloc(pval.size(), st, "split SELL values"));
        EDG_CHECK(B.split_v32.alloc(pv32.size(), st, "split SELL values"));
        EDG_CUDA(cudaMemcpyAsync(B.split_v64.p, pval.data(), pval.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        EDG_CUDA(cudaMemcpyAsync(B.split_v32.p, pv32.data(), pv32.size() * sizeof(float), cudaMemcpyHostToDevice, st));
      }
      EDG_CUDA(cudaStreamSynchronize(st));  // host staging vectors go out of scope
      B.split_parts = P;
    }
  }
  EDG_CHECK(B.sell_off.alloc(nsl + 1, st, "SELL offsets"));
  EDG_CHECK(B.sell_ent.alloc(ent.size(), st, "SELL entries"));
  EDG_CUDA(cudaMemcpyAsync(B.sell_off.p, soff.data(), soff.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  EDG_CUDA(cudaMemcpyAsync(B.sell_ent.p, ent.data(), ent.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  if (!uniform) {
    std::vector<float> sv32(sv.begin(), sv.end());
    EDG_CHECK(B.sell_v64.alloc(sv.size(), st, "SELL values"));
    EDG_CHECK(B.sell_v32.alloc(sv.size(), st, "SELL values"));
    EDG_CUDA(cudaMemcpyAsync(B.sell_v64.p, sv.data(), sv.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    EDG_CUDA(cudaMemcpyAsync(B.sell_v32.p, sv32.data(), sv32.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  }
  EDG_CUDA(cudaStreamSynchronize(st));
  return EDG_OK;
}

}  // namespace

int sector_variant_tables(edg_sector_s* s) {
  if (s->cplx || s->form != EDG_FORM_STORED) return EDG_OK;
  EDG_CHECK(build_variants(s, s->up));
  EDG_CHECK(build_variants(s, s->dw));
  return EDG_OK;
}

int sector_build(edg_sector_s* s) {
  // exact binomial table C(n,k), n,k < kBinomN
  std::vector<uint32_t> C(kBinomN * kBinomN, 0);
  for (int n = 0; n < kBinomN; ++n)
    for (int k = 0; k < kBinomN; ++k) C[n * kBinomN + k] = uint32_t(binom_host(n, k));
  EDG_CHECK(s->binom.alloc(C.size(), s->stream, "binomial table"));
  EDG_CUDA(cudaMemcpyAsync(s->binom.p, C.data(), C.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
  EDG_CHECK(build_spin(s, 1, s->up, s->nup));
  EDG_CHECK(build_spin(s, 2, s->dw, s->ndw));
  s->dim = s->up.dim * s->dw.dim;
  s->vlen = s->cplx ? 2 * s->dim : s->dim;
  s->U = s->model.uloc;
  if (s->form == EDG_FORM_STORED) {
    EDG_CHECK(build_tables(s, 1, s->up));
    EDG_CHECK(build_tables(s, 2, s->dw));
  } else {
    // direct form: bond lists only (both spins packed: [spin][k] -> a,b ; values)
    std::vector<int32_t> hb;
    std::vector<double> hv, hvi;
    for (int sp = 0; sp < 2; ++sp) {
      const BondList& bl = s->bonds[sp];
      for (int k = 0; k < bl.nb; ++k) {
        hb.push_back(bl.a[k]);
        hb.push_back(bl.b[k]);
        hv.push_back(bl.h[k]);
        hvi.push_back(bl.hi[k]);
      }
    }
    EDG_CHECK(s->bond_dev.alloc(hb.size() + 2, s->stream, "bond list"));
    EDG_CHECK(s->bondh_dev.alloc(hv.size() + 1, s->stream, "bond values"));
    if (s->cplx) EDG_CHECK(s->bondhi_dev.alloc(hvi.size() + 1, s->stream, "bond values"));
    if (!hb.empty()) {
      EDG_CUDA(cudaMemcpyAsync(s->bond_dev.p, hb.data(), hb.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s->stream));
      EDG_CUDA(cudaMemcpyAsync(s->bondh_dev.p, hv.data(), hv.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream));
      if (s->cplx)
        EDG_CUDA(cudaMemcpyAsync(s->bondhi_dev.p, hvi.data(), hvi.size() * sizeof(double), cudaMemcpyHostToDevice,
                                 s->stream));
    }
  }
  EDG_CUDA(cudaStreamSynchronize(s->stream));
  return EDG_OK;
}

}  // namespace edg
