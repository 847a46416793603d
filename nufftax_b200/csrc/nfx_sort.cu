// Bin sort of the non-uniform points: a stable counting sort on integer bin keys.
//
// The reference has no sort (nufftax spreads unsorted points with atomics,
// nufftax/core/pallas_spread.py:337-613).  Here every point gets the key of the
// tile that holds its footprint's left cell (i0 = ceil(fold(x) - ns/2) wrapped
// into [0, nf), divided by the tile edge, x-fastest), and the permutation is the
// STABLE counting sort of those keys, so it equals numpy.argsort(keys,
// kind="stable") bit for bit.
//
// Pass 1 (k_bin_count): one warp per chunk of consecutive points computes the
//   keys and a per-chunk histogram in shared memory; the histogram is written to
//   a bin-major matrix counts[bin][chunk].
// Pass 2 (exclusive scan of that matrix): entry (bin, chunk) becomes the global
//   position of the chunk's first point of that bin.
// Pass 3 (k_bin_scatter): the same warps walk their chunk again in order; a
//   __match_any_sync ballot ranks equal keys within each 32-point round and a
//   shared-memory running count carries the rank across rounds, so ties keep
//   their input order.
// Pass 4 (k_subproblems): bins larger than max_subproblem points are split into
//   subproblems so clustered inputs spread evenly over the SMs.
#include "nfx_internal.h"

namespace nfx {

template <typename T>
__device__ __forceinline__ int point_key(const T* __restrict__ x, const T* __restrict__ y,
                                         const T* __restrict__ z, int64_t p, const Geom& g, int ns_half) {
  int key = 0;
  int mult = 1;
  const T* cs[3] = {x, y, z};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d < g.dim) {
      T xs = scaled_coord(cs[d][p], g.nf[d], g.prenorm);
      int i0 = ceil_to_int(rn_sub(xs, (T)ns_half));
      int i0w = wrap_index(i0, g.nf[d]);
      key += (i0w / g.tile[d]) * mult;
      mult *= g.nb[d];
    }
  }
  return key;
}

template <typename T>
__global__ void k_bin_count(const T* __restrict__ x, const T* __restrict__ y, const T* __restrict__ z,
                            int64_t M, Geom g, int ns_half, int chunk, int nchunks,
                            int* __restrict__ keys, int* __restrict__ counts) {
  extern __shared__ int s_hist[];
  const int warps = blockDim.x >> 5;
  const int w = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int ch = blockIdx.x * warps + w;
  int* hist = s_hist + (size_t)w * g.nbins;
  for (int b = lane; b < g.nbins; b += 32) hist[b] = 0;
  __syncwarp();
  if (ch < nchunks) {
    const int64_t p0 = (int64_t)ch * chunk;
    const int64_t p1 = (p0 + chunk < M) ? p0 + chunk : M;
    for (int64_t p = p0 + lane; p < p1; p += 32) {
      int key = point_key(x, y, z, p, g, ns_half);
      keys[p] = key;
      atomicAdd(&hist[key], 1);
    }
    __syncwarp();
    for (int b = lane; b < g.nbins; b += 32) counts[(int64_t)b * nchunks + ch] = hist[b];
  }
}

__global__ void k_bin_scatter(const int* __restrict__ keys, int64_t M, int nbins, int chunk, int nchunks,
                              const int* __restrict__ offsets, int* __restrict__ perm) {
  extern __shared__ int s_hist[];
  const int warps = blockDim.x >> 5;
  const int w = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int ch = blockIdx.x * warps + w;
  int* hist = s_hist + (size_t)w * nbins;
  for (int b = lane; b < nbins; b += 32) hist[b] = 0;
  __syncwarp();
  if (ch >= nchunks) return;
  const int64_t p0 = (int64_t)ch * chunk;
  const int64_t p1 = (p0 + chunk < M) ? p0 + chunk : M;
  const unsigned lt_mask = (1u << lane) - 1u;
  for (int64_t base = p0; base < p1; base += 32) {
    const int64_t p = base + lane;
    const bool valid = p < p1;
    const int key = valid ? keys[p] : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int rank = __popc(peers & lt_mask);
    int before = 0;
    if (valid) before = hist[key];
    __syncwarp();
    if (valid && rank == 0) hist[key] = before + __popc(peers);
    __syncwarp();
    if (valid) perm[offsets[(int64_t)key * nchunks + ch] + before + rank] = (int)p;
  }
}

// bin_start[b] = offsets[b][0]; bin_start[nbins] = M.  Then subproblems: bin b
// gets ceil(count_b / maxsub) of them.  One block; each thread owns a
// contiguous run of bins.
__global__ void k_subproblems(const int* __restrict__ offsets, int nbins, int nchunks, int M, int maxsub,
                              int* __restrict__ bin_start, int* __restrict__ sub_bin,
                              int* __restrict__ sub_start, int* __restrict__ nsub_out) {
  __shared__ int s_warp[32];
  const int tid = threadIdx.x;
  const int nt = blockDim.x;
  const int per = (nbins + nt - 1) / nt;
  const int b0 = min(tid * per, nbins);
  const int b1 = min(b0 + per, nbins);
  int local = 0;
  for (int b = b0; b < b1; ++b) {
    int s = offsets[(int64_t)b * nchunks];
    int e = (b + 1 < nbins) ? offsets[(int64_t)(b + 1) * nchunks] : M;
    bin_start[b] = s;
    local += (e - s + maxsub - 1) / maxsub;
  }
  if (tid == 0) bin_start[nbins] = M;
  // block exclusive scan of `local`
  const int lane = tid & 31, wid = tid >> 5;
  int v = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  if (lane == 31) s_warp[wid] = v;
  __syncthreads();
  if (wid == 0) {
    int nw = nt >> 5;
    int t = lane < nw ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int n = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += n;
    }
    if (lane < nw) s_warp[lane] = t;
  }
  __syncthreads();
  int excl = v - local + (wid > 0 ? s_warp[wid - 1] : 0);
  if (tid == nt - 1) *nsub_out = excl + local;
  for (int b = b0; b < b1; ++b) {
    int s = offsets[(int64_t)b * nchunks];
    int e = (b + 1 < nbins) ? offsets[(int64_t)(b + 1) * nchunks] : M;
    for (int q = s; q < e; q += maxsub) {
      sub_bin[excl] = b;
      sub_start[excl] = q;
      ++excl;
    }
  }
}

// ---- generic exclusive scan of int32 (three kernels, scratch = block sums) ----
constexpr int kScanBlock = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* s_warp, int& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int n = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += n;
  }
  if (lane == 31) s_warp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    int t = lane < nw ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int n = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += n;
    }
    if (lane < nw) s_warp[lane] = t;
  }
  __syncthreads();
  total = s_warp[(blockDim.x >> 5) - 1];
  int res = inc - v + (wid > 0 ? s_warp[wid - 1] : 0);
  __syncthreads();
  return res;
}

__global__ void k_scan_reduce(const int* __restrict__ in, int64_t n, int* __restrict__ block_sums) {
  __shared__ int s_warp[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t idx = base + (int64_t)i * kScanBlock + threadIdx.x;
    if (idx < n) sum += in[idx];
  }
  int total;
  block_exclusive_scan(sum, s_warp, total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// Single block scans the block sums in place (nblocks <= kScanTile * something):
// loops over tiles of kScanTile carrying the running total.
__global__ void k_scan_sums(int* __restrict__ sums, int nblocks) {
  __shared__ int s_warp[32];
  int carry = 0;
  for (int base = 0; base < nblocks; base += kScanBlock) {
    int idx = base + threadIdx.x;
    int v = idx < nblocks ? sums[idx] : 0;
    int total;
    int ex = block_exclusive_scan(v, s_warp, total);
    if (idx < nblocks) sums[idx] = ex + carry;
    carry += total;
  }
}

__global__ void k_scan_apply(const int* __restrict__ in, int64_t n, const int* __restrict__ block_sums,
                             int* __restrict__ out) {
  __shared__ int s_warp[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int vals[kScanItems];
  int sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t idx = base + i;
    vals[i] = idx < n ? in[idx] : 0;
    sum += vals[i];
  }
  int total;
  int ex = block_exclusive_scan(sum, s_warp, total) + block_sums[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t idx = base + i;
    if (idx < n) out[idx] = ex;
    ex += vals[i];
  }
}

int64_t scan_blocks(int64_t n) { return (n + kScanTile - 1) / kScanTile; }

cudaError_t exclusive_scan(const int* in, int* out, int64_t n, int* block_sums, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  int64_t nb = scan_blocks(n);
  k_scan_reduce<<<(unsigned)nb, kScanBlock, 0, st>>>(in, n, block_sums);
  k_scan_sums<<<1, kScanBlock, 0, st>>>(block_sums, (int)nb);
  k_scan_apply<<<(unsigned)nb, kScanBlock, 0, st>>>(in, n, block_sums, out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------

template <typename T>
cudaError_t launch_sort(const SortLayout& L, const Geom& g, int ns, const void* x, const void* y, const void* z,
                        int64_t M, const SortPtrs& P, cudaStream_t st) {
  const int threads = L.sort_warps * 32;
  const unsigned blocks = (unsigned)((L.nchunks + L.sort_warps - 1) / L.sort_warps);
  const size_t smem = L.sort_smem;
  cudaError_t e0 = ensure_smem(reinterpret_cast<const void*>(k_bin_count<T>), smem);
  if (e0 == cudaSuccess) e0 = ensure_smem(reinterpret_cast<const void*>(k_bin_scatter), smem);
  if (e0 != cudaSuccess) return e0;
  k_bin_count<T><<<blocks, threads, smem, st>>>((const T*)x, (const T*)y, (const T*)z, M, g, ns / 2, L.chunk,
                                                L.nchunks, P.keys, P.counts);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = exclusive_scan(P.counts, P.counts, L.n_counts, P.scan_tmp, st);
  if (e != cudaSuccess) return e;
  k_bin_scatter<<<blocks, threads, smem, st>>>(P.keys, M, g.nbins, L.chunk, L.nchunks, P.counts, P.perm);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_subproblems<<<1, 1024, 0, st>>>(P.counts, g.nbins, L.nchunks, (int)M, L.maxsub, P.bin_start, P.sub_bin,
                                    P.sub_start, P.nsub);
  return cudaGetLastError();
}

template cudaError_t launch_sort<float>(const SortLayout&, const Geom&, int, const void*, const void*, const void*,
                                        int64_t, const SortPtrs&, cudaStream_t);
template cudaError_t launch_sort<double>(const SortLayout&, const Geom&, int, const void*, const void*, const void*,
                                         int64_t, const SortPtrs&, cudaStream_t);

}  // namespace nfx
