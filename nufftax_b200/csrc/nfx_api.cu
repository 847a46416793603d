// extern "C" entry points of libnfx_b200 (declared in include/nfx.h).
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "nfx.h"
#include "nfx_spreadinterp.cuh"

namespace nfx {

// Per-dimension dispatchers, instantiated in nfx_si_{f32,f64}_{1,2,3}d.cu.
template <typename T, int DIM>
cudaError_t dispatch_spread(int ns, const PointArgs<T>& a, const void* c, void* fw, cudaStream_t st);
template <typename T, int DIM>
cudaError_t dispatch_interp(int ns, const PointArgs<T>& a, const void* fw, void* out, cudaStream_t st);
template <typename T, int DIM>
cudaError_t dispatch_grad(int ns, const PointArgs<T>& a, const void* G, const void* V, void* oi, void* dx, void* dy,
                          void* dz, cudaStream_t st);

template <typename T, int DIM>
cudaError_t dispatch_batch(int ns, bool spread, const void* items, int n, const int* prefix, int64_t max_subs,
                           size_t smem, cudaStream_t st);

#define NFX_EXTERN(T, D)                                                                                           \
  extern template cudaError_t dispatch_spread<T, D>(int, const PointArgs<T>&, const void*, void*, cudaStream_t);   \
  extern template cudaError_t dispatch_interp<T, D>(int, const PointArgs<T>&, const void*, void*, cudaStream_t);   \
  extern template cudaError_t dispatch_grad<T, D>(int, const PointArgs<T>&, const void*, const void*, void*, void*, \
                                                  void*, void*, cudaStream_t);                                     \
  extern template cudaError_t dispatch_batch<T, D>(int, bool, const void*, int, const int*, int64_t, size_t,       \
                                                   cudaStream_t);
NFX_EXTERN(float, 1)
NFX_EXTERN(float, 2)
NFX_EXTERN(float, 3)
NFX_EXTERN(double, 1)
NFX_EXTERN(double, 2)
NFX_EXTERN(double, 3)
#undef NFX_EXTERN

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

int num_sms() {
  static std::mutex mu;
  static std::map<int, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  cache[dev] = n;
  return n;
}

// ---- device status word and TMA tensor maps ----------------------------------
__device__ int g_status_word;

int* device_status_word() {
  static std::mutex mu;
  static std::map<int, int*> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_status_word) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  cache[dev] = (int*)p;
  return (int*)p;
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
    return (EncodeTiledFn)p;
  }();
  return fn;
}

bool interp_tile_map(CUtensorMap_st* map, size_t real_bytes, int dim, const Geom& g, int n_trans, const void* grid) {
  const char* env = std::getenv("NFX_INTERP_STAGING");
  if (env != nullptr && std::strcmp(env, "plain") == 0) return false;
  if (dim < 2 || n_trans < 1) return false;
  // 8-byte elements: a complex64 is one, a complex128 two, so x coordinates
  // (tile origin x * elements per complex) stay even, i.e. 16-byte aligned,
  // when the tile's x edge is even for complex64.
  const int per = (int)(2 * real_bytes / 8);
  if (per == 1 && (g.tile[0] % 2 != 0 || g.pitch % 2 != 0)) return false;
  const uint64_t row_bytes = (uint64_t)g.nf[0] * 2 * real_bytes;
  if (row_bytes % 16 != 0 || ((uintptr_t)grid & 15) != 0) return false;
  if ((int64_t)g.pitch * per > 256 || g.pad[1] > 256 || g.pad[2] > 256) return false;
  if (g.pitch > g.nf[0] || g.pad[1] > g.nf[1] || (dim == 3 && g.pad[2] > g.nf[2])) return false;
  EncodeTiledFn enc = encode_tiled();
  if (enc == nullptr) return false;
  cuuint64_t dims[4], strides[3];
  cuuint32_t box[4], estr[4] = {1, 1, 1, 1};
  int r = 0;
  dims[r] = (cuuint64_t)g.nf[0] * per, box[r++] = (cuuint32_t)(g.pitch * per);
  dims[r] = (cuuint64_t)g.nf[1], box[r++] = (cuuint32_t)g.pad[1];
  if (dim == 3) dims[r] = (cuuint64_t)g.nf[2], box[r++] = (cuuint32_t)g.pad[2];
  dims[r] = (cuuint64_t)n_trans, box[r++] = 1;
  strides[0] = row_bytes;
  strides[1] = row_bytes * (uint64_t)g.nf[1];
  if (dim == 3) strides[2] = strides[1] * (uint64_t)g.nf[2];
  const CUresult res = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, (cuuint32_t)r, const_cast<void*>(grid), dims, strides,
                           box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return res == CUDA_SUCCESS;
}

cudaError_t ensure_smem(const void* fn, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;
  if (smem <= 48 * 1024) return cudaSuccess;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto k = std::make_pair(fn, dev);
  if (done[k] >= smem) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) done[k] = smem;
  return e;
}

cudaError_t prefer_max_smem(const void* fn) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, bool> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto k = std::make_pair(fn, dev);
  if (done[k]) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e == cudaSuccess) done[k] = true;
  return e;
}

cudaError_t kernel_grid(const void* fn, int threads, size_t smem, int64_t max_work, int& grid) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, size_t, int>, int> occ;
  static std::map<std::pair<const void*, int>, size_t> smem_attr;
  int dev = 0;
  cudaGetDevice(&dev);
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_tuple(fn, dev, smem, threads);
    auto it = occ.find(key);
    if (it != occ.end()) {
      per_sm = it->second;
    } else {
      auto ak = std::make_pair(fn, dev);
      if (smem > 48 * 1024 && smem_attr[ak] < smem) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        smem_attr[ak] = smem;
      }
      cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
      if (e != cudaSuccess) return e;
      if (per_sm < 1) return cudaErrorInvalidConfiguration;
      occ[key] = per_sm;
    }
  }
  int64_t want = (int64_t)num_sms() * per_sm;
  if (max_work < 1) max_work = 1;
  grid = (int)std::min<int64_t>(want, max_work);
  return cudaSuccess;
}

// ---------------------------------------------------------------------------
// Options -> geometry and sort layout
// ---------------------------------------------------------------------------
constexpr int kMaxBins = 49152;
constexpr size_t kSmemBudget = 200 * 1024;

static size_t real_bytes(int precision) { return precision == NFX_F64 ? 8 : 4; }

// Row pitch (cells) of the shared-memory tile.  Footprints of at least 32
// cells in 2D/3D use the run-merging spread, whose flush has lane (grp, kx)
// add to footprint row rho = grp * rpl + r (2D: y = rho; 3D: z = rho / ns,
// y = rho % ns), column kx: the pitch (at most a quarter longer than the row)
// is the one that puts those 32 words in the fewest shared-memory banks per
// instruction.  Otherwise rows of one footprint are `ns` cells wide and a warp
// covers 32/ns rows: a pitch that is an odd multiple of ns (mod 32) puts those
// rows in disjoint bank ranges (at most ~12% longer).
static int flush_conflicts(int pitch, int plane, int ns, int dim) {
  const int G = run_groups(ns), rpl = run_rows_per_lane(dim, ns), nr = run_rows(dim, ns);
  int worst = 0;
  for (int r = 0; r < rpl; ++r) {
    int bank[32] = {0};
    for (int grp = 0; grp < G; ++grp) {
      const int rho = grp * rpl + r;
      if (rho >= nr) continue;
      const int base = dim == 3 ? (rho / ns) * plane + (rho % ns) * pitch : rho * pitch;
      for (int kx = 0; kx < ns; ++kx) ++bank[(base + kx) % 32];
    }
    for (int k = 0; k < 32; ++k) worst += bank[k] > 1 ? bank[k] - 1 : 0;
  }
  return worst;
}

static int choose_pitch(int pad0, int pad1, int ns, int dim) {
  if (dim >= 2 && run_slot_reals(dim, ns, 4) > 0) {
    int best = pad0, best_c = flush_conflicts(pad0, pad0 * pad1, ns, dim);
    for (int p = pad0 + 1; p <= pad0 + std::max(1, pad0 / 4) && best_c > 0; ++p) {
      const int c = flush_conflicts(p, p * pad1, ns, dim);
      if (c < best_c) {
        best = p;
        best_c = c;
      }
    }
    return best;
  }
  if (ns == 2 || ns == 4 || ns == 8 || ns == 16) {
    const int limit = pad0 + std::max(1, pad0 / 8);
    for (int p = pad0; p <= limit; ++p)
      if (p % ns == 0 && ((p / ns) % 2 == 1)) return p;
  }
  return pad0;
}

static void fill_geom(const nfx_opts* o, Geom& g) {
  g.dim = o->dim;
  for (int d = 0; d < 3; ++d) {
    bool act = d < o->dim;
    g.nf[d] = act ? o->nf[d] : 1;
    g.tile[d] = act ? o->tile[d] : 1;
    g.nb[d] = act ? (g.nf[d] + g.tile[d] - 1) / g.tile[d] : 1;
    g.pad[d] = act ? g.tile[d] + o->nspread - 1 : 1;
    g.tdiv[d] = make_fastdiv(g.tile[d]);
  }
  g.pitch = choose_pitch(g.pad[0], g.pad[1], o->nspread, o->dim);
  g.nbins = g.nb[0] * g.nb[1] * g.nb[2];
  g.prenorm = o->prenorm;
  g.spread_mode = o->spread_mode;
  g.interp_mode = o->interp_mode;
  g.t3_mode = 0;
  g.t3_isign = 0;
  g.t3_beta = g.t3_kc = 0.0;
  g.t3 = nullptr;
}

static int validate_opts(const nfx_opts* o) {
  if (o == nullptr) {
    set_error("opts is NULL");
    return NFX_ERR_INVALID;
  }
  if (o->precision != NFX_F32 && o->precision != NFX_F64) {
    set_error("precision must be NFX_F32 or NFX_F64");
    return NFX_ERR_INVALID;
  }
  if (o->dim < 1 || o->dim > 3) {
    set_error("dim must be 1, 2 or 3");
    return NFX_ERR_INVALID;
  }
  if (o->nspread < 2 || o->nspread > 16 || (o->nspread & 1)) {
    set_error("nspread must be even and in [2, 16]");
    return NFX_ERR_UNSUPPORTED;
  }
  for (int d = 0; d < o->dim; ++d) {
    if (o->nf[d] < 1 || o->nf[d] > (1 << 28)) {
      set_error("nf out of range");
      return NFX_ERR_INVALID;
    }
    if (o->tile[d] < 0) {
      set_error("tile must be >= 0");
      return NFX_ERR_INVALID;
    }
  }
  int64_t grid = 1;
  for (int d = 0; d < o->dim; ++d) grid *= o->nf[d];
  if (grid > ((int64_t)1 << 31) - 1) {
    set_error("fine grid larger than 2^31 - 1 cells");
    return NFX_ERR_UNSUPPORTED;
  }
  if (o->max_subproblem < 0) {
    set_error("max_subproblem must be >= 0");
    return NFX_ERR_INVALID;
  }
  if ((o->spread_mode != NFX_PER_POINT_AUTO && o->spread_mode != NFX_PER_POINT_WARP &&
       o->spread_mode != NFX_PER_POINT_CTA) ||
      (o->interp_mode != NFX_PER_POINT_AUTO && o->interp_mode != NFX_PER_POINT_THREAD &&
       o->interp_mode != NFX_PER_POINT_GROUP)) {
    set_error("spread_mode must be AUTO, WARP or CTA and interp_mode AUTO, THREAD or GROUP");
    return NFX_ERR_INVALID;
  }
  return NFX_OK;
}

// Resolve tile[] = 0 to defaults (max_subproblem = 0 stays "auto": the sort
// layout picks it from M), keep the bin count and
// the shared memory of every kernel within budget.
static int resolve_opts(const nfx_opts* in, nfx_opts& o) {
  int st = validate_opts(in);
  if (st != NFX_OK) return st;
  o = *in;
  const int ns = o.nspread;
  const size_t rb = real_bytes(o.precision);
  int def[3];
  if (o.dim == 1) {
    def[0] = 512;
  } else if (o.dim == 2) {
    def[0] = def[1] = 32;
  } else {
    def[0] = 16;
    def[1] = 16;
    def[2] = 8;
  }
  bool user_tiles = true;
  for (int d = 0; d < o.dim; ++d)
    if (o.tile[d] == 0) {
      user_tiles = false;
      o.tile[d] = std::min(def[d], o.nf[d]);
    }
  for (int d = o.dim; d < 3; ++d) o.tile[d] = 1;
  if (!user_tiles) {
    // Shrink the largest tile edge while a kernel's shared memory is over
    // budget; grow the edge of the axis with the most bins while there are too
    // many bins for the sort (only if the result still fits).
    for (int it = 0; it < 64; ++it) {
      Geom g;
      fill_geom(&o, g);
      const bool smem_ok = spread_smem_bytes(rb, o.dim, ns, g) <= kSmemBudget &&
                           interp_smem_bytes(rb, o.dim, ns, g) <= kSmemBudget;
      if (!smem_ok) {
        int dmax = 0;
        for (int d = 1; d < o.dim; ++d)
          if (o.tile[d] > o.tile[dmax]) dmax = d;
        if (o.tile[dmax] <= 2) break;
        o.tile[dmax] = (o.tile[dmax] + 1) / 2;
        continue;
      }
      if (g.nbins <= kMaxBins) break;
      int dmax = 0;
      for (int d = 1; d < o.dim; ++d)
        if (g.nb[d] > g.nb[dmax]) dmax = d;
      nfx_opts trial = o;
      trial.tile[dmax] = std::min(o.tile[dmax] * 2, o.nf[dmax]);
      Geom gt;
      fill_geom(&trial, gt);
      if (spread_smem_bytes(rb, o.dim, ns, gt) > kSmemBudget || interp_smem_bytes(rb, o.dim, ns, gt) > kSmemBudget)
        break;
      o = trial;
    }
  }
  Geom g;
  fill_geom(&o, g);
  if (g.nbins > kMaxBins) {
    set_error("too many bins for the sort (raise tile)");
    return NFX_ERR_UNSUPPORTED;
  }
  if (g.tile[0] * g.tile[1] * g.tile[2] > kMaxBins) {
    set_error("too many cells per tile for the sort (lower tile)");
    return NFX_ERR_UNSUPPORTED;
  }
  if (spread_smem_bytes(rb, o.dim, ns, g) > kSmemBudget || interp_smem_bytes(rb, o.dim, ns, g) > kSmemBudget) {
    set_error("tile too large for shared memory (lower tile)");
    return NFX_ERR_UNSUPPORTED;
  }
  return NFX_OK;
}

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Default subproblem size (max_subproblem = 0): 2048 points in 3D; in 1D/2D
// 1024, doubled (up to 4096) while the points still fill about two subproblems
// per resident spread CTA (148 SMs x 5), so large dense sets flush their tiles
// to the fine grid less often without starving the SMs.
static int auto_max_subproblem(int dim, int64_t M) {
  if (dim == 3) return 2048;
  constexpr int64_t kSubTarget = 1480;
  int maxsub = 1024;
  while (maxsub < 4096 && M / (2 * (int64_t)maxsub) >= kSubTarget) maxsub *= 2;
  return maxsub;
}

static void make_layout(const nfx_opts& o, const Geom& g, int64_t M, SortLayout& L) {
  L.M = M;
  L.nbins = g.nbins;
  L.ncell = g.tile[0] * g.tile[1] * g.tile[2];
  radix_plan(g.nbins, L.ncell, L.cbits, L.bits, L.npass, L.dbits);
  const int64_t B = (int64_t)1 << L.dbits;
  L.nchunks = (int)((M + radix_chunk() - 1) / radix_chunk());
  L.maxsub = o.max_subproblem > 0 ? o.max_subproblem : auto_max_subproblem(o.dim, M);
  L.max_subs = g.nbins + (M + L.maxsub - 1) / L.maxsub;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t at = off;
    off += align256(bytes);
    return at;
  };
  L.off_keys = take((size_t)M * 4);
  L.off_keys_tmp = take((size_t)M * 4);
  L.off_vals_tmp = take((size_t)M * 4);
  L.off_keys_sorted = take((size_t)M * 4);
  L.off_perm = take((size_t)M * 4);
  L.off_counts = take((size_t)L.nchunks * B * 4);
  L.off_totals = take((size_t)B * 4);
  L.off_bin_start = take((size_t)(g.nbins + 1) * 4);
  L.off_sub_bin = take((size_t)L.max_subs * 4);
  L.off_sub_start = take((size_t)L.max_subs * 4);
  L.off_nsub = take(4);
  for (int d = 0; d < 3; ++d) L.off_coord[d] = d < o.dim ? take((size_t)M * real_bytes(o.precision)) : 0;
  // float coordinates of non-type-3 points are carried through the radix passes
  const bool carry = o.precision == NFX_F32 && g.t3_mode == 0;
  for (int d = 0; d < 3; ++d) L.off_coord_tmp[d] = carry && d < o.dim ? take((size_t)M * 4) : 0;
  L.off_extra = g.t3_mode != 0 ? take((size_t)M * 2 * real_bytes(o.precision)) : 0;
  L.total = off;
}

// The composite sort key (bin << cbits | cell) must stay a non-negative int.
static bool key_fits(const SortLayout& L) {
  if (L.bits <= 30) return true;
  set_error("bins x cells per tile need " + std::to_string(L.bits) + " key bits (at most 30): use smaller tiles");
  return false;
}

static SortPtrs carve(const SortLayout& L, void* ws) {
  char* b = (char*)ws;
  SortPtrs P;
  P.keys = (int*)(b + L.off_keys);
  P.keys_tmp = (int*)(b + L.off_keys_tmp);
  P.vals_tmp = (int*)(b + L.off_vals_tmp);
  P.keys_sorted = (int*)(b + L.off_keys_sorted);
  P.perm = (int*)(b + L.off_perm);
  P.counts = (int*)(b + L.off_counts);
  P.totals = (int*)(b + L.off_totals);
  P.bin_start = (int*)(b + L.off_bin_start);
  P.sub_bin = (int*)(b + L.off_sub_bin);
  P.sub_start = (int*)(b + L.off_sub_start);
  P.nsub = (int*)(b + L.off_nsub);
  for (int d = 0; d < 3; ++d) P.coord[d] = L.off_coord[d] != 0 ? (void*)(b + L.off_coord[d]) : nullptr;
  for (int d = 0; d < 3; ++d) P.coord_tmp[d] = L.off_coord_tmp[d] != 0 ? (void*)(b + L.off_coord_tmp[d]) : nullptr;
  P.extra = L.off_extra != 0 ? (void*)(b + L.off_extra) : nullptr;
  return P;
}

static SortView view(const SortLayout& L, const void* ws) {
  SortPtrs P = carve(L, const_cast<void*>(ws));
  SortView v;
  for (int d = 0; d < 3; ++d) v.coord[d] = P.coord[d];
  v.extra = P.extra;
  v.perm = P.perm;
  v.bin_start = P.bin_start;
  v.sub_bin = P.sub_bin;
  v.sub_start = P.sub_start;
  v.nsub = P.nsub;
  v.maxsub = L.maxsub;
  v.max_subs = L.max_subs;
  return v;
}

static int cuda_fail(cudaError_t e, const char* where) {
  set_error(std::string(where) + ": " + cudaGetErrorString(e));
  return NFX_ERR_CUDA;
}

struct Prepared {
  nfx_opts o;
  Geom g;
  SortLayout L;
};

static int prepare(const nfx_opts* in, int64_t M, const void* x, const void* y, const void* z, const void* ws,
                   size_t ws_bytes, Prepared& P) {
  int st = resolve_opts(in, P.o);
  if (st != NFX_OK) return st;
  if (M < 0 || M > (int64_t)INT32_MAX - 1) {
    set_error("M must be in [0, 2^31 - 2]");
    return NFX_ERR_INVALID;
  }
  if (M > 0) {
    const void* cs[3] = {x, y, z};
    for (int d = 0; d < P.o.dim; ++d)
      if (cs[d] == nullptr) {
        set_error("coordinate pointer is NULL");
        return NFX_ERR_INVALID;
      }
  }
  fill_geom(&P.o, P.g);
  make_layout(P.o, P.g, M, P.L);
  if (!key_fits(P.L)) return NFX_ERR_UNSUPPORTED;
  if (ws == nullptr || ws_bytes < P.L.total) {
    set_error("workspace too small: need " + std::to_string(P.L.total) + " bytes");
    return NFX_ERR_WORKSPACE;
  }
  return NFX_OK;
}

// ---------------------------------------------------------------------------
// Polynomial ES weights (float path): for each q < ns / 2, Chebyshev
// interpolation of v -> phi(q - (v + ns - 1) / 2) on [-1, 1] at D + 1 nodes,
// converted to monomials in v; weight ns - 1 - q is the same polynomial at -v
// (phi is even), stored with the odd coefficients negated.  The degree is
// raised (up to the kernels' evaluation degree) until both forms the kernels
// evaluate in float (fmaf, as on the device) are within kPolyAbs + kPolyRel *
// |phi| of the double exp/sqrt value on a fine grid: Horner in v for every q,
// and the even/odd split E(v^2) +- v O(v^2) that gives weights q and ns - 1 - q
// together; two float ulps of the weight plus a small absolute floor (the
// exp/sqrt form in float carries errors of the same size).
// ---------------------------------------------------------------------------
constexpr double kPolyAbs = 3e-8;
constexpr double kPolyRel = 2.6e-7;

static double es_phi(double z, double beta, double kc) {
  const double arg = 1.0 - kc * z * z;
  return arg >= 0.0 ? std::exp(beta * (std::sqrt(arg > 0.0 ? arg : 0.0) - 1.0)) : 0.0;
}

static bool fit_es_poly_uncached(int ns, double beta, double kc, EsPoly& out, double& err_out) {
  for (int D = 4; D <= kPolyEvalDeg; ++D) {
    double worst = 0.0, worst_ratio = 0.0;
    EsPoly P = {};  // coefficients above D stay zero (the kernels run degree kPolyEvalDeg)
    P.deg = D;
    for (int q = 0; q < ns / 2; ++q) {
      const int n = D + 1;
      double cheb[kPolyMaxDeg + 1] = {0};
      for (int j = 0; j < n; ++j) {
        double acc = 0.0;
        for (int k = 0; k < n; ++k) {
          const double th = kPi * (k + 0.5) / n;
          const double v = std::cos(th);
          acc += es_phi(q - (v + ns - 1) / 2.0, beta, kc) * std::cos(j * th);
        }
        cheb[j] = (j == 0 ? 1.0 : 2.0) * acc / n;
      }
      // Chebyshev -> monomial: T_{j+1} = 2 v T_j - T_{j-1}
      double Tm[kPolyMaxDeg + 2][kPolyMaxDeg + 2] = {{0}};
      Tm[0][0] = 1.0;
      if (D >= 1) Tm[1][1] = 1.0;
      for (int j = 1; j < D; ++j)
        for (int i = 0; i <= j + 1; ++i) Tm[j + 1][i] = (i > 0 ? 2.0 * Tm[j][i - 1] : 0.0) - Tm[j - 1][i];
      double mono[kPolyMaxDeg + 1] = {0};
      for (int j = 0; j <= D; ++j)
        for (int i = 0; i <= j; ++i) mono[i] += cheb[j] * Tm[j][i];
      for (int i = 0; i <= D; ++i) {
        P.a[q][i] = (float)mono[i];
        P.a[ns - 1 - q][i] = (i % 2 == 0) ? P.a[q][i] : -P.a[q][i];
      }
    }
    auto account = [&](float h, double ref) {
      const double e = std::fabs((double)h - ref);
      const double ratio = e / (kPolyAbs + kPolyRel * std::fabs(ref));
      worst = e > worst ? e : worst;
      worst_ratio = ratio > worst_ratio ? ratio : worst_ratio;
    };
    for (int t = 0; t <= 2000; ++t) {
      const double v = -1.0 + 2.0 * t / 2000.0;
      const float fv = (float)v;
      for (int q = 0; q < ns; ++q) {  // Horner in v
        float h = P.a[q][kPolyEvalDeg];
        for (int d = kPolyEvalDeg - 1; d >= 0; --d) h = std::fmaf(h, fv, P.a[q][d]);
        account(h, es_phi(q - (v + ns - 1) / 2.0, beta, kc));
      }
      const float u = fv * fv;
      for (int q = 0; q < ns / 2; ++q) {  // even / odd split, weights q and ns - 1 - q
        float e = P.a[q][kPolyEvalDeg - 1], o = P.a[q][kPolyEvalDeg];
        for (int d = kPolyEvalDeg - 3; d >= 0; d -= 2) {
          e = std::fmaf(e, u, P.a[q][d]);
          o = std::fmaf(o, u, P.a[q][d + 1]);
        }
        account(std::fmaf(fv, o, e), es_phi(q - (v + ns - 1) / 2.0, beta, kc));
        account(std::fmaf(-fv, o, e), es_phi(ns - 1 - q - (v + ns - 1) / 2.0, beta, kc));
      }
    }
    if (worst_ratio <= 1.0) {
      out = P;
      err_out = worst;
      return true;
    }
  }
  return false;
}

static bool es_poly(int ns, double beta, double kc, EsPoly& out, double* err = nullptr) {
  static std::mutex mu;
  static std::map<std::tuple<int, double, double>, std::pair<EsPoly, double>> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto key = std::make_tuple(ns, beta, kc);
  auto it = cache.find(key);
  if (it == cache.end()) {
    EsPoly P = {};
    double e = -1.0;
    if (!fit_es_poly_uncached(ns, beta, kc, P, e)) P.deg = 0;
    it = cache.emplace(key, std::make_pair(P, e)).first;
  }
  out = it->second.first;
  if (err) *err = it->second.second;
  return out.deg > 0;
}

template <typename T>
static void attach_poly(PointArgs<T>& a, int ns, double beta, double kc) {
  a.poly.deg = 0;
  if (std::is_same<T, float>::value) es_poly(ns, beta, kc, a.poly);
}

template <typename T>
static cudaError_t spread_dim(const Prepared& P, const void* x, const void* y, const void* z, int64_t M, const void* c,
                              int n_trans, void* fw, const void* ws, cudaStream_t st) {
  PointArgs<T> a = make_args<T>(P.g, P.o.beta, P.o.kc, M, n_trans, view(P.L, ws));
  attach_poly(a, P.o.nspread, P.o.beta, P.o.kc);
  switch (P.o.dim) {
    case 1:
      return dispatch_spread<T, 1>(P.o.nspread, a, c, fw, st);
    case 2:
      return dispatch_spread<T, 2>(P.o.nspread, a, c, fw, st);
    default:
      return dispatch_spread<T, 3>(P.o.nspread, a, c, fw, st);
  }
}

template <typename T>
static cudaError_t interp_dim(const Prepared& P, const void* x, const void* y, const void* z, int64_t M,
                              const void* fw, int n_trans, void* out, const void* ws, cudaStream_t st) {
  PointArgs<T> a = make_args<T>(P.g, P.o.beta, P.o.kc, M, n_trans, view(P.L, ws));
  attach_poly(a, P.o.nspread, P.o.beta, P.o.kc);
  switch (P.o.dim) {
    case 1:
      return dispatch_interp<T, 1>(P.o.nspread, a, fw, out, st);
    case 2:
      return dispatch_interp<T, 2>(P.o.nspread, a, fw, out, st);
    default:
      return dispatch_interp<T, 3>(P.o.nspread, a, fw, out, st);
  }
}

template <typename T>
static cudaError_t grad_dim(const Prepared& P, const void* x, const void* y, const void* z, int64_t M, const void* G,
                            const void* V, int n_trans, void* oi, void* dx, void* dy, void* dz, const void* ws,
                            cudaStream_t st) {
  PointArgs<T> a = make_args<T>(P.g, P.o.beta, P.o.kc, M, n_trans, view(P.L, ws));
  switch (P.o.dim) {
    case 1:
      return dispatch_grad<T, 1>(P.o.nspread, a, G, V, oi, dx, nullptr, nullptr, st);
    case 2:
      return dispatch_grad<T, 2>(P.o.nspread, a, G, V, oi, dx, dy, nullptr, st);
    default:
      return dispatch_grad<T, 3>(P.o.nspread, a, G, V, oi, dx, dy, dz, st);
  }
}

static int64_t grid_cells(const Geom& g) { return (int64_t)g.nf[0] * g.nf[1] * g.nf[2]; }

template <typename T>
__global__ void k_batch_prefix(const BatchItem<T>* __restrict__ items, int n, int* __restrict__ prefix) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int run = 0;
  for (int p = 0; p < n; ++p) {
    prefix[p] = run;
    run += *items[p].a.s.nsub;
  }
  prefix[n] = run;
}

// Per-problem options from the shared ones (kernel, precision, dim) and the
// problem's own grid / tiling.
static int batch_problem_opts(const nfx_opts* common, const nfx_batch_problem& pb, Prepared& P) {
  nfx_opts o = *common;
  for (int d = 0; d < 3; ++d) {
    o.nf[d] = pb.nf[d];
    o.tile[d] = pb.tile[d];
  }
  o.max_subproblem = pb.max_subproblem;
  if (pb.interp_mode != NFX_PER_POINT_AUTO) o.interp_mode = pb.interp_mode;
  return prepare(&o, pb.M, pb.x, pb.y, pb.z, pb.workspace, pb.workspace_bytes, P);
}

static size_t batch_item_bytes(int precision) {
  return precision == NFX_F32 ? sizeof(BatchItem<float>) : sizeof(BatchItem<double>);
}

static size_t batch_prefix_offset(int precision, int n) { return align256(batch_item_bytes(precision) * n); }

// Workspace of one fused type 3: the type-3 scalars and their min / max
// scratch, the source sort (type-3 mode 1: rescale + pre-phase per point), the
// target sort (mode 2: rescale + output factor per point), the fine grid of the
// spread, the inner type 2's fine grid and the cuFFT work area of its FFT.
struct Nufft3Layout {
  Prepared src, tgt;
  size_t off_params, off_scratch, off_src, off_tgt, off_fw, off_fw2, off_fft, fft_bytes, total;
  int64_t fw_cells, fw2_cells;
};

static int nufft3_layout(const nfx_opts* opts, const int nf_inner[3], int64_t M, int64_t K, int n_trans,
                         Nufft3Layout& L3) {
  if (opts == nullptr || nf_inner == nullptr || n_trans < 1 || M < 0 || K < 0 || M > (int64_t)INT32_MAX - 1 ||
      K > (int64_t)INT32_MAX - 1) {
    set_error("nfx_nufft3: invalid arguments");
    return NFX_ERR_INVALID;
  }
  nfx_opts os = *opts;
  os.prenorm = 0;
  int st = resolve_opts(&os, L3.src.o);
  if (st != NFX_OK) return st;
  nfx_opts ot = *opts;
  for (int d = 0; d < 3; ++d) {
    ot.nf[d] = d < opts->dim ? nf_inner[d] : 1;
    ot.tile[d] = 0;
  }
  ot.prenorm = 1;
  ot.max_subproblem = 0;
  st = resolve_opts(&ot, L3.tgt.o);
  if (st != NFX_OK) return st;
  fill_geom(&L3.src.o, L3.src.g);
  fill_geom(&L3.tgt.o, L3.tgt.g);
  L3.src.g.t3_mode = 1;
  L3.tgt.g.t3_mode = 2;
  make_layout(L3.src.o, L3.src.g, M, L3.src.L);
  make_layout(L3.tgt.o, L3.tgt.g, K, L3.tgt.L);
  if (!key_fits(L3.src.L) || !key_fits(L3.tgt.L)) return NFX_ERR_UNSUPPORTED;
  const size_t cb = 2 * real_bytes(opts->precision);
  L3.fw_cells = grid_cells(L3.src.g);
  L3.fw2_cells = grid_cells(L3.tgt.g);
  st = nfx_fft_work_bytes(opts->precision, opts->dim, L3.tgt.o.nf, n_trans, &L3.fft_bytes);
  if (st != NFX_OK) return st;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t at = off;
    off += align256(bytes);
    return at;
  };
  L3.off_params = take(sizeof(T3Params));
  L3.off_scratch = take(t3_scratch_bytes());
  L3.off_src = take(L3.src.L.total);
  L3.off_tgt = take(L3.tgt.L.total);
  L3.off_fw = take((size_t)L3.fw_cells * n_trans * cb);
  L3.off_fw2 = take((size_t)L3.fw2_cells * n_trans * cb);
  L3.off_fft = take(L3.fft_bytes);
  L3.total = off;
  return NFX_OK;
}

template <typename T>
static int nufft3_run(Nufft3Layout& L3, double upsampfac, int isign, const void* const* src, int64_t M,
                      const void* c, int n_trans, const void* const* tgt, int64_t K, const void* fac1,
                      const void* fac2, const void* fac3, void* out, char* ws, cudaStream_t st) {
  const int dim = L3.src.o.dim;
  const int ns = L3.src.o.nspread;
  T3Params* params = (T3Params*)(ws + L3.off_params);
  cudaError_t e = launch_t3_params<T>(dim, L3.src.o.nf, upsampfac, src, M, tgt, K, params, ws + L3.off_scratch, st);
  if (e != cudaSuccess) return cuda_fail(e, "nfx_nufft3 set-up");
  for (Prepared* P : {&L3.src, &L3.tgt}) {
    P->g.t3 = params;
    P->g.t3_isign = isign;
    P->g.t3_beta = P->o.beta;
    P->g.t3_kc = P->o.kc;
  }
  const void* s3[3] = {nullptr, nullptr, nullptr};
  const void* t3[3] = {nullptr, nullptr, nullptr};
  for (int d = 0; d < dim; ++d) {
    s3[d] = src[d];
    t3[d] = tgt[d];
  }
  // spread of the pre-phased strengths at the rescaled sources (nufft3.py:271-283)
  char* src_ws = ws + L3.off_src;
  e = launch_sort<T>(L3.src.L, L3.src.g, ns, s3[0], s3[1], s3[2], M, carve(L3.src.L, src_ws), st);
  if (e != cudaSuccess) return cuda_fail(e, "nfx_nufft3 source sort");
  void* fw = ws + L3.off_fw;
  e = cudaMemsetAsync(fw, 0, (size_t)L3.fw_cells * n_trans * 2 * sizeof(T), st);
  if (e == cudaSuccess) e = spread_dim<T>(L3.src, nullptr, nullptr, nullptr, M, c, n_trans, fw, src_ws, st);
  if (e != cudaSuccess) return cuda_fail(e, "nfx_nufft3 spread");
  // inner type 2: the fine grid as modes, deconvolved and zero-padded, FFT
  // (nufft3.py:287-293, 381-387)
  void* fw2 = ws + L3.off_fw2;
  int stt = nfx_deconv_pad(L3.src.o.precision, dim, L3.tgt.o.nf, L3.src.o.nf, fac1, fac2, fac3, fw, fw2, n_trans, st);
  if (stt != NFX_OK) return stt;
  stt = nfx_fft_ws(L3.src.o.precision, dim, L3.tgt.o.nf, n_trans, fw2, isign < 0 ? -1 : 1,
                   L3.fft_bytes ? ws + L3.off_fft : nullptr, L3.fft_bytes, st);
  if (stt != NFX_OK) return stt;
  // interpolation at the rescaled targets, times phase / phihat (nufft3.py:293-299, 387-394)
  char* tgt_ws = ws + L3.off_tgt;
  e = launch_sort<T>(L3.tgt.L, L3.tgt.g, ns, t3[0], t3[1], t3[2], K, carve(L3.tgt.L, tgt_ws), st);
  if (e == cudaSuccess) e = interp_dim<T>(L3.tgt, nullptr, nullptr, nullptr, K, fw2, n_trans, out, tgt_ws, st);
  return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_nufft3 interp");
}

// Device table of one wave (nfx_wave): spread items and their subproblem
// prefix, interp items and theirs, then the zero-pad items of the type-2
// problems and the crop items of the type-1 problems.
struct WaveLayout {
  int n1 = 0, n2 = 0;
  size_t off_spread, off_prefix_s, off_interp, off_prefix_i, off_pad, off_shuffle, total;
  size_t smem_s = 0, smem_i = 0;
  int64_t subs_s = 0, subs_i = 0;
};

static int wave_layout(const nfx_opts* common, const nfx_wave_item* items, int n, WaveLayout& W,
                       std::vector<Prepared>* prep) {
  if (common == nullptr || items == nullptr || n < 1) {
    set_error("nfx_wave: invalid arguments");
    return NFX_ERR_INVALID;
  }
  const size_t rb = real_bytes(common->precision);
  for (int i = 0; i < n; ++i) {
    const nfx_wave_item& it = items[i];
    if (it.kind != 1 && it.kind != 2) {
      set_error("nfx_wave: kind must be 1 or 2");
      return NFX_ERR_INVALID;
    }
    // the item's own grid with the library's default tiles and subproblem size
    // for it (those of `common` belong to whichever grid they were chosen for)
    nfx_opts o = *common;
    for (int d = 0; d < 3; ++d) {
      o.nf[d] = it.nf[d];
      o.tile[d] = 0;
    }
    o.max_subproblem = 0;
    Prepared P;
    int st = prepare(&o, it.M, it.x, it.y, it.z, it.workspace, it.workspace_bytes, P);
    if (st != NFX_OK) return st;
    if (it.in == nullptr || it.out == nullptr || it.fw == nullptr) {
      set_error("nfx_wave: NULL in / out / fw");
      return NFX_ERR_INVALID;
    }
    if (it.kind == 1) {
      ++W.n1;
      W.smem_s = std::max(W.smem_s, spread_smem_bytes(rb, P.o.dim, P.o.nspread, P.g));
      W.subs_s += P.L.max_subs;
    } else {
      ++W.n2;
      W.smem_i = std::max(W.smem_i, tile_smem_bytes(rb, P.g));
      W.subs_i += P.L.max_subs;
    }
    if (prep) prep->push_back(P);
  }
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t at = off;
    off += align256(bytes);
    return at;
  };
  const size_t ib = batch_item_bytes(common->precision), db = deconv_item_bytes(common->precision == NFX_F64);
  W.off_spread = take(ib * W.n1);
  W.off_prefix_s = take((size_t)(W.n1 + 1) * 4);
  W.off_interp = take(ib * W.n2);
  W.off_prefix_i = take((size_t)(W.n2 + 1) * 4);
  W.off_pad = take(db * W.n2);
  W.off_shuffle = take(db * W.n1);
  W.total = off;
  return NFX_OK;
}

template <typename T>
static void wave_items(const nfx_opts* common, const nfx_wave_item* items, int n, const std::vector<Prepared>& prep,
                       const WaveLayout& W, unsigned char* host) {
  BatchItem<T>* sp = (BatchItem<T>*)(host + W.off_spread);
  BatchItem<T>* ip = (BatchItem<T>*)(host + W.off_interp);
  int a = 0, b = 0;
  std::vector<int> nf1, nm1, nf2, nm2;
  std::vector<const void*> fac1, fac2, src1, src2;
  std::vector<void*> dst1, dst2;
  for (int i = 0; i < n; ++i) {
    const nfx_wave_item& it = items[i];
    const Prepared& P = prep[i];
    BatchItem<T>& bi = it.kind == 1 ? sp[a++] : ip[b++];
    bi.a = make_args<T>(P.g, P.o.beta, P.o.kc, it.M, 1, view(P.L, it.workspace));
    attach_poly(bi.a, P.o.nspread, P.o.beta, P.o.kc);
    bi.src = it.kind == 1 ? it.in : it.fw;
    bi.dst = it.kind == 1 ? it.fw : it.out;
    auto& nf = it.kind == 1 ? nf1 : nf2;
    auto& nm = it.kind == 1 ? nm1 : nm2;
    auto& fac = it.kind == 1 ? fac1 : fac2;
    for (int d = 0; d < 3; ++d) {
      nf.push_back(d < common->dim ? it.nf[d] : 1);
      nm.push_back(d < common->dim ? it.n_modes[d] : 1);
      fac.push_back(d < common->dim ? it.fac[d] : nullptr);
    }
    if (it.kind == 1) {
      src1.push_back(it.fw);
      dst1.push_back(it.out);
    } else {
      src2.push_back(it.in);
      dst2.push_back(it.fw);
    }
  }
  const int prec = common->precision == NFX_F64 ? 1 : 0;
  if (W.n2 > 0)
    fill_deconv_items(prec, common->dim, true, nf2.data(), nm2.data(), fac2.data(), src2.data(), dst2.data(), W.n2,
                      host + W.off_pad);
  if (W.n1 > 0)
    fill_deconv_items(prec, common->dim, false, nf1.data(), nm1.data(), fac1.data(), src1.data(), dst1.data(), W.n1,
                      host + W.off_shuffle);
}

// Work units of the batched deconvolution pass over the wave's problems of
// one kind (the count fill_deconv_items gives their table).
static int64_t deconv_total(const nfx_wave_item* items, int n, int kind, int dim, bool pad) {
  int64_t t = 0;
  for (int i = 0; i < n; ++i) {
    if (items[i].kind != kind) continue;
    int nf[3], nm[3];
    for (int d = 0; d < 3; ++d) {
      nf[d] = d < dim ? items[i].nf[d] : 1;
      nm[d] = d < dim ? items[i].n_modes[d] : 1;
    }
    t += deconv_units(nf, nm, pad);
  }
  return t;
}

}  // namespace nfx

using namespace nfx;

extern "C" {

int nfx_version(void) { return 10000; }

int nfx_es_poly(int nspread, double beta, double kc, float* coeffs, int* degree, double* max_abs_err) {
  if (nspread < 2 || nspread > 16 || degree == nullptr) {
    set_error("nfx_es_poly: invalid arguments");
    return NFX_ERR_INVALID;
  }
  EsPoly P;
  double err = -1.0;
  es_poly(nspread, beta, kc, P, &err);
  *degree = P.deg;
  if (max_abs_err) *max_abs_err = err;
  if (coeffs && P.deg > 0)
    for (int q = 0; q < nspread; ++q)
      for (int d = 0; d <= P.deg; ++d) coeffs[q * (kPolyMaxDeg + 1) + d] = P.a[q][d];
  return NFX_OK;
}
const char* nfx_last_error(void) { return g_last_error.c_str(); }
int nfx_num_sms(void) { return num_sms(); }

// One CTA arms an mbarrier for 16 bytes of TMA data and issues no copy, so
// its bounded wait (tma_wait) runs out; nothing is in flight when it returns.
__global__ void k_bounded_wait_selftest(int* status) {
  __shared__ __align__(8) uint64_t mbar;
  nfx::tma_init(&mbar);
  const unsigned mb = nfx::smem_addr(&mbar);
  if (threadIdx.x == 0)
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(16u) : "memory");
  const bool landed = nfx::tma_wait(mb, 0u);
  if (!__syncthreads_and(landed) && threadIdx.x == 0) atomicOr(status, NFX_STATUS_TMA_TIMEOUT);
}

int nfx_selftest_bounded_wait(int* status) {
  using namespace nfx;
  if (status == nullptr) {
    set_error("status is NULL");
    return NFX_ERR_INVALID;
  }
  int* w = device_status_word();
  if (w == nullptr) {
    set_error("device status word unavailable");
    return NFX_ERR_CUDA;
  }
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemset(w, 0, sizeof(int));
  if (e == cudaSuccess) {
    k_bounded_wait_selftest<<<1, 32>>>(w);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_error(std::string("nfx_selftest_bounded_wait: ") + cudaGetErrorString(e));
    return NFX_ERR_CUDA;
  }
  return nfx_device_status(status);
}

int nfx_sort_kernel_count(const nfx_opts* opts, int64_t M, int type3, int* n) {
  using namespace nfx;
  if (n == nullptr || M < 0) {
    set_error("n is NULL or M < 0");
    return NFX_ERR_INVALID;
  }
  nfx_opts o;
  int st = resolve_opts(opts, o);
  if (st != NFX_OK) return st;
  Geom g;
  fill_geom(&o, g);
  g.t3_mode = type3 ? 1 : 0;
  SortLayout L;
  make_layout(o, g, M, L);
  const bool carry = L.off_coord_tmp[0] != 0;
  const bool fused_bounds = M > 0 && (int64_t)(L.npass - 1) * L.dbits == L.cbits;
  *n = M == 0 ? 2 : 1 + 2 * L.npass + (L.npass - 1) + (carry ? 0 : 1) + (fused_bounds ? 0 : 1) + 1;
  return NFX_OK;
}

int nfx_capture_id(void* stream, unsigned long long* id) {
  using namespace nfx;
  if (id == nullptr) {
    set_error("id is NULL");
    return NFX_ERR_INVALID;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  unsigned long long cid = 0;
  cudaError_t e = cudaStreamGetCaptureInfo((cudaStream_t)stream, &cap, &cid);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(std::string("nfx_capture_id: ") + cudaGetErrorString(e));
    return NFX_ERR_CUDA;
  }
  *id = cap == cudaStreamCaptureStatusActive ? cid : 0ull;
  return NFX_OK;
}

int nfx_device_status(int* status) {
  using namespace nfx;
  if (status == nullptr) {
    set_error("status is NULL");
    return NFX_ERR_INVALID;
  }
  int* w = device_status_word();
  if (w == nullptr) {
    set_error("device status word unavailable");
    return NFX_ERR_CUDA;
  }
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(status, w, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemset(w, 0, sizeof(int));
  if (e != cudaSuccess) {
    set_error(std::string("nfx_device_status: ") + cudaGetErrorString(e));
    return NFX_ERR_CUDA;
  }
  return NFX_OK;
}

int nfx_default_tiles(nfx_opts* opts) {
  nfx_opts o;
  int st = resolve_opts(opts, o);
  if (st != NFX_OK) return st;
  for (int d = 0; d < 3; ++d) opts->tile[d] = o.tile[d];
  opts->max_subproblem = o.max_subproblem;
  return NFX_OK;
}

int nfx_sort_workspace_bytes(const nfx_opts* opts, int64_t M, size_t* bytes) {
  Prepared P;
  int st = resolve_opts(opts, P.o);
  if (st != NFX_OK) return st;
  if (M < 0 || bytes == nullptr) {
    set_error("M < 0 or bytes is NULL");
    return NFX_ERR_INVALID;
  }
  fill_geom(&P.o, P.g);
  make_layout(P.o, P.g, M, P.L);
  if (!key_fits(P.L)) return NFX_ERR_UNSUPPORTED;
  *bytes = P.L.total;
  return NFX_OK;
}

int nfx_sort_points(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M, void* ws,
                    size_t ws_bytes, void* stream) {
  Prepared P;
  int st = prepare(opts, M, x, y, z, ws, ws_bytes, P);
  if (st != NFX_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  SortPtrs ptr = carve(P.L, ws);
  if (M == 0) {
    cudaError_t e = cudaMemsetAsync(ptr.bin_start, 0, (size_t)(P.g.nbins + 1) * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(ptr.nsub, 0, 4, s);
    return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_sort_points");
  }
  cudaError_t e = P.o.precision == NFX_F32 ? launch_sort<float>(P.L, P.g, P.o.nspread, x, y, z, M, ptr, s)
                                           : launch_sort<double>(P.L, P.g, P.o.nspread, x, y, z, M, ptr, s);
  return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_sort_points");
}

int nfx_sort_results(const nfx_opts* opts, int64_t M, const void* ws, size_t ws_bytes, int* keys, int* perm,
                     int* bin_start, int* nbins, void* stream) {
  Prepared P;
  int st = prepare(opts, M, (const void*)1, (const void*)1, (const void*)1, ws, ws_bytes, P);
  if (st != NFX_OK) return st;
  if (nbins) *nbins = P.g.nbins;
  cudaStream_t s = (cudaStream_t)stream;
  SortPtrs ptr = carve(P.L, const_cast<void*>(ws));
  cudaError_t e = cudaSuccess;
  if (keys && M > 0) e = bin_keys_of(P.L, ptr.keys, keys, s);
  if (e == cudaSuccess && perm && M > 0) e = cudaMemcpyAsync(perm, ptr.perm, (size_t)M * 4, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess && bin_start)
    e = cudaMemcpyAsync(bin_start, ptr.bin_start, (size_t)(P.g.nbins + 1) * 4, cudaMemcpyDeviceToDevice, s);
  return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_sort_results");
}

int nfx_spread_sorted(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M, const void* c,
                      int n_trans, void* fw, const void* ws, size_t ws_bytes, void* stream) {
  Prepared P;
  int st = prepare(opts, M, x, y, z, ws, ws_bytes, P);
  if (st != NFX_OK) return st;
  if (n_trans < 1 || fw == nullptr || (M > 0 && c == nullptr)) {
    set_error("n_trans < 1 or NULL c / fw");
    return NFX_ERR_INVALID;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const size_t cb = 2 * real_bytes(P.o.precision);
  cudaError_t e = cudaMemsetAsync(fw, 0, (size_t)grid_cells(P.g) * n_trans * cb, s);
  if (e != cudaSuccess) return cuda_fail(e, "nfx_spread_sorted memset");
  if (M == 0) return NFX_OK;
  e = P.o.precision == NFX_F32 ? spread_dim<float>(P, x, y, z, M, c, n_trans, fw, ws, s)
                               : spread_dim<double>(P, x, y, z, M, c, n_trans, fw, ws, s);
  return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_spread_sorted");
}

int nfx_interp_sorted(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M, const void* fw,
                      int n_trans, void* c_out, const void* ws, size_t ws_bytes, void* stream) {
  Prepared P;
  int st = prepare(opts, M, x, y, z, ws, ws_bytes, P);
  if (st != NFX_OK) return st;
  if (n_trans < 1 || fw == nullptr || (M > 0 && c_out == nullptr)) {
    set_error("n_trans < 1 or NULL fw / c_out");
    return NFX_ERR_INVALID;
  }
  if (M == 0) return NFX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = P.o.precision == NFX_F32 ? interp_dim<float>(P, x, y, z, M, fw, n_trans, c_out, ws, s)
                                           : interp_dim<double>(P, x, y, z, M, fw, n_trans, c_out, ws, s);
  return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_interp_sorted");
}

int nfx_spread(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M, const void* c,
               int n_trans, void* fw, void* ws, size_t ws_bytes, void* stream) {
  int st = nfx_sort_points(opts, x, y, z, M, ws, ws_bytes, stream);
  if (st != NFX_OK) return st;
  return nfx_spread_sorted(opts, x, y, z, M, c, n_trans, fw, ws, ws_bytes, stream);
}

int nfx_interp(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M, const void* fw,
               int n_trans, void* c_out, void* ws, size_t ws_bytes, void* stream) {
  int st = nfx_sort_points(opts, x, y, z, M, ws, ws_bytes, stream);
  if (st != NFX_OK) return st;
  return nfx_interp_sorted(opts, x, y, z, M, fw, n_trans, c_out, ws, ws_bytes, stream);
}

int nfx_spread_grad_sorted(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M,
                           const void* c, const void* g_grid, int n_trans, void* dc, void* dx, void* dy, void* dz,
                           const void* ws, size_t ws_bytes, void* stream) {
  Prepared P;
  int st = prepare(opts, M, x, y, z, ws, ws_bytes, P);
  if (st != NFX_OK) return st;
  if (n_trans < 1 || g_grid == nullptr || (M > 0 && c == nullptr)) {
    set_error("n_trans < 1 or NULL c / g_grid");
    return NFX_ERR_INVALID;
  }
  if (M == 0) return NFX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = P.o.precision == NFX_F32
                      ? grad_dim<float>(P, x, y, z, M, g_grid, c, n_trans, dc, dx, dy, dz, ws, s)
                      : grad_dim<double>(P, x, y, z, M, g_grid, c, n_trans, dc, dx, dy, dz, ws, s);
  return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_spread_grad_sorted");
}

int nfx_interp_grad_sorted(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M,
                           const void* fw, const void* g_pts, int n_trans, void* dx, void* dy, void* dz,
                           const void* ws, size_t ws_bytes, void* stream) {
  Prepared P;
  int st = prepare(opts, M, x, y, z, ws, ws_bytes, P);
  if (st != NFX_OK) return st;
  if (n_trans < 1 || fw == nullptr || (M > 0 && g_pts == nullptr)) {
    set_error("n_trans < 1 or NULL fw / g_pts");
    return NFX_ERR_INVALID;
  }
  if (M == 0) return NFX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = P.o.precision == NFX_F32
                      ? grad_dim<float>(P, x, y, z, M, fw, g_pts, n_trans, nullptr, dx, dy, dz, ws, s)
                      : grad_dim<double>(P, x, y, z, M, fw, g_pts, n_trans, nullptr, dx, dy, dz, ws, s);
  return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_interp_grad_sorted");
}

static int check_deconv(int precision, int dim, const int nf[3], const int nm[3], const void* fac1, const void* fac2,
                        const void* fac3, int n_trans, int nf_full[3], int nm_full[3]) {
  if ((precision != NFX_F32 && precision != NFX_F64) || dim < 1 || dim > 3 || nf == nullptr || nm == nullptr ||
      fac1 == nullptr || (dim >= 2 && fac2 == nullptr) || (dim >= 3 && fac3 == nullptr) || n_trans < 1) {
    set_error("invalid deconvolution arguments");
    return NFX_ERR_INVALID;
  }
  for (int d = 0; d < 3; ++d) {
    nf_full[d] = d < dim ? nf[d] : 1;
    nm_full[d] = d < dim ? nm[d] : 1;
    if (nf_full[d] < 1 || nm_full[d] < 0 || nm_full[d] > nf_full[d]) {
      set_error("need 0 <= n_modes <= nf per axis");
      return NFX_ERR_INVALID;
    }
  }
  return NFX_OK;
}

int nfx_nufft1(const nfx_opts* opts, const int n_modes[3], const void* x, const void* y, const void* z, int64_t M,
               const void* c, int n_trans, int fft_sign, const void* fac1, const void* fac2, const void* fac3, void* fw,
               void* f_out, void* ws, size_t ws_bytes, void* stream) {
  if (opts == nullptr || n_modes == nullptr) {
    set_error("nfx_nufft1: opts or n_modes is NULL");
    return NFX_ERR_INVALID;
  }
  int st = nfx_sort_points(opts, x, y, z, M, ws, ws_bytes, stream);
  if (st == NFX_OK) st = nfx_spread_sorted(opts, x, y, z, M, c, n_trans, fw, ws, ws_bytes, stream);
  if (st == NFX_OK) st = nfx_fft(opts->precision, opts->dim, opts->nf, n_trans, fw, fft_sign, stream);
  if (st == NFX_OK)
    st = nfx_deconv_shuffle(opts->precision, opts->dim, opts->nf, n_modes, fac1, fac2, fac3, fw, f_out, n_trans,
                            stream);
  return st;
}

int nfx_nufft2(const nfx_opts* opts, const int n_modes[3], const void* x, const void* y, const void* z, int64_t M,
               const void* f_in, int n_trans, int fft_sign, const void* fac1, const void* fac2, const void* fac3,
               void* fw, void* c_out, void* ws, size_t ws_bytes, void* stream) {
  if (opts == nullptr || n_modes == nullptr) {
    set_error("nfx_nufft2: opts or n_modes is NULL");
    return NFX_ERR_INVALID;
  }
  int st = nfx_deconv_pad(opts->precision, opts->dim, opts->nf, n_modes, fac1, fac2, fac3, f_in, fw, n_trans, stream);
  if (st == NFX_OK) st = nfx_fft(opts->precision, opts->dim, opts->nf, n_trans, fw, fft_sign, stream);
  if (st == NFX_OK) st = nfx_sort_points(opts, x, y, z, M, ws, ws_bytes, stream);
  if (st == NFX_OK) st = nfx_interp_sorted(opts, x, y, z, M, fw, n_trans, c_out, ws, ws_bytes, stream);
  return st;
}

int nfx_deconv_shuffle(int precision, int dim, const int nf[3], const int n_modes[3], const void* fac1,
                       const void* fac2, const void* fac3, const void* fw_hat, void* f_out, int n_trans,
                       void* stream) {
  int nff[3], nmf[3];
  int st = check_deconv(precision, dim, nf, n_modes, fac1, fac2, fac3, n_trans, nff, nmf);
  if (st != NFX_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = precision == NFX_F32
                      ? launch_deconv_shuffle<float>(dim, nff, nmf, (const float*)fac1, (const float*)fac2,
                                                     (const float*)fac3, fw_hat, f_out, n_trans, s)
                      : launch_deconv_shuffle<double>(dim, nff, nmf, (const double*)fac1, (const double*)fac2,
                                                      (const double*)fac3, fw_hat, f_out, n_trans, s);
  return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_deconv_shuffle");
}

int nfx_deconv_pad(int precision, int dim, const int nf[3], const int n_modes[3], const void* fac1, const void* fac2,
                   const void* fac3, const void* f_in, void* fw_hat, int n_trans, void* stream) {
  int nff[3], nmf[3];
  int st = check_deconv(precision, dim, nf, n_modes, fac1, fac2, fac3, n_trans, nff, nmf);
  if (st != NFX_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = precision == NFX_F32
                      ? launch_deconv_pad<float>(dim, nff, nmf, (const float*)fac1, (const float*)fac2,
                                                 (const float*)fac3, f_in, fw_hat, n_trans, s)
                      : launch_deconv_pad<double>(dim, nff, nmf, (const double*)fac1, (const double*)fac2,
                                                  (const double*)fac3, f_in, fw_hat, n_trans, s);
  return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_deconv_pad");
}


// ---- batched spread / interp / deconvolution --------------------------------

int nfx_batch_info_get(const nfx_opts* common, int spread, const nfx_batch_problem* probs, int nprob,
                       nfx_batch_info* info) {
  if (common == nullptr || probs == nullptr || nprob < 1 || info == nullptr) {
    set_error("nfx_batch_info_get: invalid arguments");
    return NFX_ERR_INVALID;
  }
  size_t smem = 0;
  int64_t subs = 0;
  for (int p = 0; p < nprob; ++p) {
    Prepared P;
    nfx_opts o = *common;
    for (int d = 0; d < 3; ++d) {
      o.nf[d] = probs[p].nf[d];
      o.tile[d] = probs[p].tile[d];
    }
    o.max_subproblem = probs[p].max_subproblem;
    int st = resolve_opts(&o, P.o);
    if (st != NFX_OK) return st;
    fill_geom(&P.o, P.g);
    make_layout(P.o, P.g, probs[p].M, P.L);
    const size_t rb = real_bytes(P.o.precision);
    const size_t sm = spread ? spread_smem_bytes(rb, P.o.dim, P.o.nspread, P.g) : tile_smem_bytes(rb, P.g);
    smem = sm > smem ? sm : smem;
    subs += P.L.max_subs;
  }
  info->table_bytes = batch_prefix_offset(common->precision, nprob) + align256((size_t)(nprob + 1) * 4);
  info->smem_bytes = smem;
  info->max_subs = subs;
  return NFX_OK;
}

int nfx_batch_upload(const nfx_opts* common, int spread, const nfx_batch_problem* probs, int nprob, void* dev_table,
                     size_t table_bytes, void* stream) {
  nfx_batch_info info;
  int st = nfx_batch_info_get(common, spread, probs, nprob, &info);
  if (st != NFX_OK) return st;
  if (dev_table == nullptr || table_bytes < info.table_bytes) {
    set_error("nfx_batch_upload: table too small");
    return NFX_ERR_WORKSPACE;
  }
  std::vector<unsigned char> host(batch_item_bytes(common->precision) * nprob);
  for (int p = 0; p < nprob; ++p) {
    Prepared P;
    st = batch_problem_opts(common, probs[p], P);
    if (st != NFX_OK) return st;
    if (probs[p].src == nullptr || probs[p].dst == nullptr) {
      set_error("nfx_batch_upload: NULL src / dst");
      return NFX_ERR_INVALID;
    }
    if (common->precision == NFX_F32) {
      BatchItem<float>* it = (BatchItem<float>*)host.data() + p;
      it->a = make_args<float>(P.g, P.o.beta, P.o.kc, probs[p].M, 1, view(P.L, probs[p].workspace));
      attach_poly(it->a, P.o.nspread, P.o.beta, P.o.kc);
      it->src = probs[p].src;
      it->dst = probs[p].dst;
    } else {
      BatchItem<double>* it = (BatchItem<double>*)host.data() + p;
      it->a = make_args<double>(P.g, P.o.beta, P.o.kc, probs[p].M, 1, view(P.L, probs[p].workspace));
      it->src = probs[p].src;
      it->dst = probs[p].dst;
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(dev_table, host.data(), host.size(), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_batch_upload");
}

int nfx_batch_sort(const nfx_opts* common, const nfx_batch_problem* probs, int nprob, void* stream) {
  if (common == nullptr || probs == nullptr || nprob < 1) {
    set_error("nfx_batch_sort: invalid arguments");
    return NFX_ERR_INVALID;
  }
  for (int p = 0; p < nprob; ++p) {
    nfx_opts o = *common;
    for (int d = 0; d < 3; ++d) {
      o.nf[d] = probs[p].nf[d];
      o.tile[d] = probs[p].tile[d];
    }
    o.max_subproblem = probs[p].max_subproblem;
    int st = nfx_sort_points(&o, probs[p].x, probs[p].y, probs[p].z, probs[p].M, probs[p].workspace,
                             probs[p].workspace_bytes, stream);
    if (st != NFX_OK) return st;
  }
  return NFX_OK;
}

int nfx_batch_launch(const nfx_opts* common, int spread, const void* dev_table, int nprob, const nfx_batch_info* info,
                     void* stream) {
  if (common == nullptr || dev_table == nullptr || nprob < 1 || info == nullptr) {
    set_error("nfx_batch_launch: invalid arguments");
    return NFX_ERR_INVALID;
  }
  nfx_opts o;
  nfx_opts probe = *common;
  probe.nf[0] = probe.nf[1] = probe.nf[2] = 64;
  probe.tile[0] = probe.tile[1] = probe.tile[2] = 0;
  int st = resolve_opts(&probe, o);
  if (st != NFX_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  int* prefix = (int*)((char*)dev_table + batch_prefix_offset(common->precision, nprob));
  cudaError_t e;
  if (common->precision == NFX_F32)
    k_batch_prefix<float><<<1, 32, 0, s>>>((const BatchItem<float>*)dev_table, nprob, prefix);
  else
    k_batch_prefix<double><<<1, 32, 0, s>>>((const BatchItem<double>*)dev_table, nprob, prefix);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "nfx_batch_launch prefix");
  const bool sp = spread != 0;
  const int ns = common->nspread;
  if (common->precision == NFX_F32) {
    e = common->dim == 1   ? dispatch_batch<float, 1>(ns, sp, dev_table, nprob, prefix, info->max_subs, info->smem_bytes, s)
        : common->dim == 2 ? dispatch_batch<float, 2>(ns, sp, dev_table, nprob, prefix, info->max_subs, info->smem_bytes, s)
                           : dispatch_batch<float, 3>(ns, sp, dev_table, nprob, prefix, info->max_subs, info->smem_bytes, s);
  } else {
    e = common->dim == 1   ? dispatch_batch<double, 1>(ns, sp, dev_table, nprob, prefix, info->max_subs, info->smem_bytes, s)
        : common->dim == 2 ? dispatch_batch<double, 2>(ns, sp, dev_table, nprob, prefix, info->max_subs, info->smem_bytes, s)
                           : dispatch_batch<double, 3>(ns, sp, dev_table, nprob, prefix, info->max_subs, info->smem_bytes, s);
  }
  return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_batch_launch");
}

int nfx_nufft3_workspace_bytes(const nfx_opts* opts, const int nf_inner[3], int64_t M, int64_t K, int n_trans,
                               size_t* bytes) {
  if (bytes == nullptr) {
    set_error("nfx_nufft3_workspace_bytes: bytes is NULL");
    return NFX_ERR_INVALID;
  }
  Nufft3Layout L3;
  int st = nufft3_layout(opts, nf_inner, M, K, n_trans, L3);
  if (st == NFX_OK) *bytes = L3.total;
  return st;
}

int nfx_nufft3(const nfx_opts* opts, const int nf_inner[3], double upsampfac, int isign, const void* const* src,
               int64_t M, const void* c, int n_trans, const void* const* tgt, int64_t K, const void* fac1,
               const void* fac2, const void* fac3, void* out, void* workspace, size_t workspace_bytes, void* stream) {
  Nufft3Layout L3;
  int st = nufft3_layout(opts, nf_inner, M, K, n_trans, L3);
  if (st != NFX_OK) return st;
  const int dim = opts->dim;
  if (M < 1 || src == nullptr || tgt == nullptr || c == nullptr || (K > 0 && out == nullptr) || fac1 == nullptr ||
      (dim >= 2 && fac2 == nullptr) || (dim >= 3 && fac3 == nullptr)) {
    set_error("nfx_nufft3: need M >= 1 and non-NULL sources, targets, strengths, output and factors");
    return NFX_ERR_INVALID;
  }
  for (int d = 0; d < dim; ++d)
    if (src[d] == nullptr || (K > 0 && tgt[d] == nullptr) || opts->nf[d] < 2) {
      set_error("nfx_nufft3: NULL coordinate axis or type-3 grid below 2");
      return NFX_ERR_INVALID;
    }
  if (workspace == nullptr || workspace_bytes < L3.total) {
    set_error("nfx_nufft3: workspace too small: need " + std::to_string(L3.total) + " bytes");
    return NFX_ERR_WORKSPACE;
  }
  if (K == 0) return NFX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  return opts->precision == NFX_F32
             ? nufft3_run<float>(L3, upsampfac, isign, src, M, c, n_trans, tgt, K, fac1, fac2, fac3, out,
                                 (char*)workspace, s)
             : nufft3_run<double>(L3, upsampfac, isign, src, M, c, n_trans, tgt, K, fac1, fac2, fac3, out,
                                  (char*)workspace, s);
}

int nfx_wave_table_bytes(const nfx_opts* common, const nfx_wave_item* items, int n, size_t* table_bytes) {
  if (table_bytes == nullptr) {
    set_error("nfx_wave_table_bytes: table_bytes is NULL");
    return NFX_ERR_INVALID;
  }
  WaveLayout W;
  int st = wave_layout(common, items, n, W, nullptr);
  if (st == NFX_OK) *table_bytes = W.total;
  return st;
}

int nfx_wave(const nfx_opts* common, const nfx_wave_item* items, int n, void* dev_table, void* host_staging,
             size_t table_bytes, void* stream) {
  WaveLayout W;
  std::vector<Prepared> prep;
  int st = wave_layout(common, items, n, W, &prep);
  if (st != NFX_OK) return st;
  if (dev_table == nullptr || host_staging == nullptr || table_bytes < W.total) {
    set_error("nfx_wave: table or staging buffer too small: need " + std::to_string(W.total) + " bytes");
    return NFX_ERR_WORKSPACE;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const bool f32 = common->precision == NFX_F32;
  unsigned char* host = (unsigned char*)host_staging;
  if (f32)
    wave_items<float>(common, items, n, prep, W, host);
  else
    wave_items<double>(common, items, n, prep, W, host);
  cudaError_t e = cudaMemcpyAsync(dev_table, host_staging, W.total, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return cuda_fail(e, "nfx_wave table upload");
  char* tab = (char*)dev_table;
  const int dim = common->dim;
  const int64_t tot_pad = deconv_total(items, n, 2, dim, true);
  const int64_t tot_shuffle = deconv_total(items, n, 1, dim, false);
  // type 2: deconvolve + zero-pad every grid in one launch, then the FFTs
  if (W.n2 > 0) {
    e = f32 ? launch_deconv_batch<float>(true, tab + W.off_pad, W.n2, tot_pad, s)
            : launch_deconv_batch<double>(true, tab + W.off_pad, W.n2, tot_pad, s);
    if (e != cudaSuccess) return cuda_fail(e, "nfx_wave zero-pad");
    for (int i = 0; i < n; ++i)
      if (items[i].kind == 2) {
        st = nfx_fft(common->precision, dim, items[i].nf, 1, items[i].fw, items[i].fft_sign, stream);
        if (st != NFX_OK) return st;
      }
  }
  // every problem's sort; zeroed grids for the spreads
  for (int i = 0; i < n; ++i) {
    const Prepared& P = prep[i];
    const nfx_wave_item& it = items[i];
    st = nfx_sort_points(&P.o, it.x, it.y, it.z, it.M, it.workspace, it.workspace_bytes, stream);
    if (st != NFX_OK) return st;
    if (it.kind == 1) {
      e = cudaMemsetAsync(it.fw, 0, (size_t)grid_cells(P.g) * 2 * real_bytes(common->precision), s);
      if (e != cudaSuccess) return cuda_fail(e, "nfx_wave grid zeroing");
    }
  }
  // one persistent spread over all type-1 problems, one interp over all type-2 problems
  for (int kind = 1; kind <= 2; ++kind) {
    const int np = kind == 1 ? W.n1 : W.n2;
    if (np == 0) continue;
    const void* table = tab + (kind == 1 ? W.off_spread : W.off_interp);
    int* prefix = (int*)(tab + (kind == 1 ? W.off_prefix_s : W.off_prefix_i));
    if (f32)
      k_batch_prefix<float><<<1, 32, 0, s>>>((const BatchItem<float>*)table, np, prefix);
    else
      k_batch_prefix<double><<<1, 32, 0, s>>>((const BatchItem<double>*)table, np, prefix);
    const bool sp = kind == 1;
    const int64_t subs = sp ? W.subs_s : W.subs_i;
    const size_t smem = sp ? W.smem_s : W.smem_i;
    const int ns = common->nspread;
    if (f32)
      e = dim == 1   ? dispatch_batch<float, 1>(ns, sp, table, np, prefix, subs, smem, s)
          : dim == 2 ? dispatch_batch<float, 2>(ns, sp, table, np, prefix, subs, smem, s)
                     : dispatch_batch<float, 3>(ns, sp, table, np, prefix, subs, smem, s);
    else
      e = dim == 1   ? dispatch_batch<double, 1>(ns, sp, table, np, prefix, subs, smem, s)
          : dim == 2 ? dispatch_batch<double, 2>(ns, sp, table, np, prefix, subs, smem, s)
                     : dispatch_batch<double, 3>(ns, sp, table, np, prefix, subs, smem, s);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, sp ? "nfx_wave spread" : "nfx_wave interp");
  }
  // type 1: the FFTs, then deconvolve + crop every problem in one launch
  if (W.n1 > 0) {
    for (int i = 0; i < n; ++i)
      if (items[i].kind == 1) {
        st = nfx_fft(common->precision, dim, items[i].nf, 1, items[i].fw, items[i].fft_sign, stream);
        if (st != NFX_OK) return st;
      }
    e = f32 ? launch_deconv_batch<float>(false, tab + W.off_shuffle, W.n1, tot_shuffle, s)
            : launch_deconv_batch<double>(false, tab + W.off_shuffle, W.n1, tot_shuffle, s);
    if (e != cudaSuccess) return cuda_fail(e, "nfx_wave crop");
  }
  return NFX_OK;
}

size_t nfx_batch_deconv_table_bytes(int precision, int nprob) {
  return align256(deconv_item_bytes(precision == NFX_F64 ? 1 : 0) * (size_t)(nprob > 0 ? nprob : 1));
}

int nfx_batch_deconv_upload(int precision, int dim, int pad, const int* nf, const int* n_modes,
                            const void* const* fac, const void* const* src, void* const* dst, int nprob,
                            void* dev_table, size_t table_bytes, int64_t* total, void* stream) {
  if ((precision != NFX_F32 && precision != NFX_F64) || dim < 1 || dim > 3 || nf == nullptr || n_modes == nullptr ||
      fac == nullptr || src == nullptr || dst == nullptr || nprob < 1 || dev_table == nullptr || total == nullptr) {
    set_error("nfx_batch_deconv_upload: invalid arguments");
    return NFX_ERR_INVALID;
  }
  if (table_bytes < nfx_batch_deconv_table_bytes(precision, nprob)) {
    set_error("nfx_batch_deconv_upload: table too small");
    return NFX_ERR_WORKSPACE;
  }
  for (int p = 0; p < nprob; ++p) {
    int a[3], b[3];
    int st = check_deconv(precision, dim, nf + 3 * p, n_modes + 3 * p, fac[3 * p], fac[3 * p + 1], fac[3 * p + 2], 1,
                          a, b);
    if (st != NFX_OK) return st;
    if (src[p] == nullptr || dst[p] == nullptr) {
      set_error("nfx_batch_deconv_upload: NULL src / dst");
      return NFX_ERR_INVALID;
    }
  }
  std::vector<unsigned char> host(deconv_item_bytes(precision == NFX_F64 ? 1 : 0) * nprob);
  *total = fill_deconv_items(precision == NFX_F64 ? 1 : 0, dim, pad != 0, nf, n_modes, fac, src, dst, nprob,
                             host.data());
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(dev_table, host.data(), host.size(), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_batch_deconv_upload");
}

int nfx_batch_deconv(int precision, int pad, const void* dev_table, int nprob, int64_t total, void* stream) {
  if ((precision != NFX_F32 && precision != NFX_F64) || dev_table == nullptr || nprob < 1 || total < 0) {
    set_error("nfx_batch_deconv: invalid arguments");
    return NFX_ERR_INVALID;
  }
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = precision == NFX_F32 ? launch_deconv_batch<float>(pad != 0, dev_table, nprob, total, s)
                                       : launch_deconv_batch<double>(pad != 0, dev_table, nprob, total, s);
  return e == cudaSuccess ? NFX_OK : cuda_fail(e, "nfx_batch_deconv");
}

}  // extern "C"
