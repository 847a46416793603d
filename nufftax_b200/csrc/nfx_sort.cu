// Bin sort of the non-uniform points: a stable counting sort on integer bin keys.
//
// The reference has no sort (nufftax spreads unsorted points with atomics,
// nufftax/core/pallas_spread.py:337-613).  Here every point gets the key of the
// tile that holds its footprint's left cell (i0 = ceil(fold(x) - ns/2) wrapped
// into [0, nf), divided by the tile edge, x-fastest) and the index of that cell
// inside the tile, and the permutation is the STABLE sort by (bin, cell): it
// equals numpy.argsort(bin * cells_per_tile + cell, kind="stable") bit for bit.
// It is computed least-significant key first, as two stable counting passes
// (cell, then bin); each pass is:
//
// (1) count (k_bin_count, k_key_count): one CTA per chunk of consecutive
//     elements builds the chunk's key histogram in shared memory and writes it
//     to a key-major matrix counts[key][chunk];
// (2) an exclusive scan of that matrix: entry (key, chunk) becomes the global
//     position of the chunk's first element with that key;
// (3) scatter (k_bin_scatter): one CTA per chunk again, each warp on a
//     contiguous sub-chunk; ballots rank equal keys within each 32-element
//     round (peer_mask: one ballot per key bit) and per-warp
//     running counts (offset by the warps before it) carry the rank across
//     rounds, so ties keep their input order.
// Finally k_subproblems splits bins larger than max_subproblem points into
// subproblems so clustered inputs spread evenly over the SMs.  Points of a
// subproblem are then ordered by cell, which lets spreading merge runs of points
// that share a cell and gives interpolation near-identical addresses per warp.
#include "nfx_internal.h"

namespace nfx {

// Lanes of the warp holding the same key as this lane: one ballot per key bit.
// Keys are in [-1, nkeys); the +1 shift keeps the inactive lanes (-1) apart
// from every real key within `nbits` = bit length of nkeys.
__device__ __forceinline__ unsigned peer_mask(int key, int nbits) {
  const unsigned k = (unsigned)(key + 1);
  unsigned m = 0xffffffffu;
  for (int b = 0; b < nbits; ++b) {
    const unsigned bit = (k >> b) & 1u;
    const unsigned bal = __ballot_sync(0xffffffffu, bit);
    m &= bit ? bal : ~bal;
  }
  return m;
}

__host__ __device__ inline int key_bits(int nkeys) {
  int b = 0;
  while ((1 << b) < nkeys + 1) ++b;
  return b;
}

// Bin of the tile holding the footprint's left cell, and that cell's index
// inside the tile (both x-fastest).
template <typename T>
__device__ __forceinline__ void point_keys(const T* __restrict__ x, const T* __restrict__ y,
                                           const T* __restrict__ z, int64_t p, const Geom& g, int ns_half, int& kbin,
                                           int& kcell) {
  int kb = 0, kc = 0, mb = 1, mc = 1;
  const T* cs[3] = {x, y, z};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d < g.dim) {
      T xs = scaled_coord(cs[d][p], g.nf[d], g.prenorm);
      int i0 = ceil_to_int(rn_sub(xs, (T)ns_half));
      int i0w = wrap_index(i0, g.nf[d]);
      int bq = i0w / g.tile[d];
      kb += bq * mb;
      kc += (i0w - bq * g.tile[d]) * mc;
      mb *= g.nb[d];
      mc *= g.tile[d];
    }
  }
  kbin = kb;
  kcell = kc;
}

// Count pass of the cell sort: one CTA per chunk walks its points, 8 per thread
// per trip so the coordinate loads overlap, writes both keys of every point and
// counts the cell keys with shared-memory atomics.
template <typename T>
__global__ void k_bin_count(const T* __restrict__ x, const T* __restrict__ y, const T* __restrict__ z,
                            int64_t M, Geom g, int ns_half, int chunk, int nchunks, int ncell,
                            int* __restrict__ keys_bin, int* __restrict__ keys_cell, int* __restrict__ counts) {
  extern __shared__ int s_hist[];
  const int ch = blockIdx.x;
  for (int b = threadIdx.x; b < ncell; b += blockDim.x) s_hist[b] = 0;
  __syncthreads();
  const int64_t p0 = (int64_t)ch * chunk;
  const int64_t p1 = (p0 + chunk < M) ? p0 + chunk : M;
  constexpr int U = 8;
  for (int64_t base = p0; base < p1; base += (int64_t)U * blockDim.x) {
    int kb[U], kc[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t p = base + (int64_t)u * blockDim.x + threadIdx.x;
      kb[u] = kc[u] = -1;
      if (p < p1) point_keys(x, y, z, p, g, ns_half, kb[u], kc[u]);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t p = base + (int64_t)u * blockDim.x + threadIdx.x;
      if (kc[u] >= 0) {
        keys_bin[p] = kb[u];
        keys_cell[p] = kc[u];
        atomicAdd(&s_hist[kc[u]], 1);
      }
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < ncell; b += blockDim.x) counts[(int64_t)b * nchunks + ch] = s_hist[b];
}

// Histogram of an int key array per chunk (second pass of the sort).
__global__ void k_key_count(const int* __restrict__ keys, int64_t M, int nkeys, int chunk, int nchunks,
                            int* __restrict__ counts) {
  extern __shared__ int s_hist[];
  const int ch = blockIdx.x;
  for (int b = threadIdx.x; b < nkeys; b += blockDim.x) s_hist[b] = 0;
  __syncthreads();
  const int64_t p0 = (int64_t)ch * chunk;
  const int64_t p1 = (p0 + chunk < M) ? p0 + chunk : M;
#pragma unroll 8
  for (int64_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) atomicAdd(&s_hist[keys[p]], 1);
  __syncthreads();
  for (int b = threadIdx.x; b < nkeys; b += blockDim.x) counts[(int64_t)b * nchunks + ch] = s_hist[b];
}

// Scatter pass: one CTA per chunk; warp w owns the contiguous sub-chunk w of
// the chunk and its own histogram row hw[w][*].  (A) each warp counts its keys,
// (B) a prefix over the warps turns the rows into each warp's starting rank per
// key, (C) each warp walks its sub-chunk in order and ranks equal keys with
// peer_mask, so the result is a stable sort.  Element i goes to
// out[pos] = vals ? vals[i] : i, and aux_out[pos] = aux_in[i] carries a second
// array along.
__global__ void k_bin_scatter(const int* __restrict__ keys, const int* __restrict__ vals, const int* __restrict__ aux_in,
                              int64_t M, int nkeys, int chunk, int nchunks, const int* __restrict__ offsets,
                              int* __restrict__ out, int* __restrict__ aux_out) {
  extern __shared__ int s_hw[];
  const int W = blockDim.x >> 5;
  const int w = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int ch = blockIdx.x;
  for (int i = threadIdx.x; i < W * nkeys; i += blockDim.x) s_hw[i] = 0;
  __syncthreads();
  const int64_t p0 = (int64_t)ch * chunk;
  const int64_t p1 = (p0 + chunk < M) ? p0 + chunk : M;
  const int64_t sub = (((p1 - p0) + W - 1) / W + 31) / 32 * 32;
  const int64_t s0 = p0 + (int64_t)w * sub < p1 ? p0 + (int64_t)w * sub : p1;
  const int64_t s1 = s0 + sub < p1 ? s0 + sub : p1;
  int* hist = s_hw + (size_t)w * nkeys;
  const unsigned lt_mask = (1u << lane) - 1u;
  const int kbits = key_bits(nkeys);
  // (A) count this warp's keys (its own histogram row: order does not matter)
#pragma unroll 8
  for (int64_t p = s0 + lane; p < s1; p += 32) atomicAdd(&hist[keys[p]], 1);
  __syncthreads();
  // (B) hw[w][k] = global start of key k in this chunk + count of k in warps < w
  for (int k = threadIdx.x; k < nkeys; k += blockDim.x) {
    int run = offsets[(int64_t)k * nchunks + ch];
    for (int v = 0; v < W; ++v) {
      const int t = s_hw[(size_t)v * nkeys + k];
      s_hw[(size_t)v * nkeys + k] = run;
      run += t;
    }
  }
  __syncthreads();
  // (C) stable placement, four 32-element rounds per trip: the inputs of all four
  // are loaded first so their latencies overlap
  constexpr int R = 4;
  for (int64_t base = s0; base < s1; base += 32 * R) {
    int key[R], val[R], aux[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t p = base + 32 * r + lane;
      const bool valid = p < s1;
      key[r] = valid ? keys[p] : -1;
      val[r] = valid && vals != nullptr ? vals[p] : (int)p;
      aux[r] = valid && aux_in != nullptr ? aux_in[p] : 0;
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const unsigned peers = peer_mask(key[r], kbits);
      const int rank = __popc(peers & lt_mask);
      const bool valid = key[r] >= 0;
      int pos = 0;
      if (valid) pos = hist[key[r]];
      __syncwarp();
      if (valid && rank == 0) hist[key[r]] = pos + __popc(peers);
      __syncwarp();
      if (valid) {
        out[pos + rank] = val[r];
        if (aux_out != nullptr) aux_out[pos + rank] = aux[r];
      }
    }
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
  const int ncell = g.tile[0] * g.tile[1] * g.tile[2];
  const size_t cell_smem = (size_t)ncell * sizeof(int);
  const size_t bin_smem = (size_t)g.nbins * sizeof(int);
  cudaError_t e = ensure_smem(reinterpret_cast<const void*>(k_bin_count<T>), cell_smem);
  if (e == cudaSuccess) e = ensure_smem(reinterpret_cast<const void*>(k_key_count), bin_smem);
  if (e == cudaSuccess)
    e = ensure_smem(reinterpret_cast<const void*>(k_bin_scatter),
                    L.sort_smem > L.sort_smem_cell ? L.sort_smem : L.sort_smem_cell);
  if (e != cudaSuccess) return e;
  // pass A: stable by cell-in-tile (carrying each point's bin key along)
  k_bin_count<T><<<(unsigned)L.nchunks, 256, cell_smem, st>>>((const T*)x, (const T*)y, (const T*)z, M, g, ns / 2,
                                                              L.chunk, L.nchunks, ncell, P.keys, P.keys_cell,
                                                              P.counts);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = exclusive_scan(P.counts, P.counts, (int64_t)ncell * L.nchunks, P.scan_tmp, st);
  if (e != cudaSuccess) return e;
  k_bin_scatter<<<(unsigned)L.nchunks, L.sort_warps_cell * 32, L.sort_smem_cell, st>>>(
      P.keys_cell, nullptr, P.keys, M, ncell, L.chunk, L.nchunks, P.counts, P.perm_cell, P.keys_by_cell);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // pass B: stable by bin over the cell-ordered sequence
  k_key_count<<<(unsigned)L.nchunks, 256, bin_smem, st>>>(P.keys_by_cell, M, g.nbins, L.chunk, L.nchunks, P.counts);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = exclusive_scan(P.counts, P.counts, (int64_t)g.nbins * L.nchunks, P.scan_tmp, st);
  if (e != cudaSuccess) return e;
  k_bin_scatter<<<(unsigned)L.nchunks, L.sort_warps * 32, L.sort_smem, st>>>(
      P.keys_by_cell, P.perm_cell, nullptr, M, g.nbins, L.chunk, L.nchunks, P.counts, P.perm, nullptr);
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
