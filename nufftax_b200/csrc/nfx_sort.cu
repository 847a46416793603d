// Bin sort of the non-uniform points: a stable LSD radix sort on one composite
// integer key per point.
//
// The reference has no sort (nufftax spreads unsorted points with atomics,
// nufftax/core/pallas_spread.py:337-613).  Here every point gets the key
// K = bin << cbits | cell, where bin is the tile that holds its footprint's
// left cell (i0 = ceil(fold(x) - ns/2) wrapped into [0, nf), divided by the
// tile edge, x-fastest) and cell that cell's index inside the tile (cbits =
// bits of cells per tile); the permutation is the STABLE sort by (bin, cell),
// equal to numpy.argsort(bin * cells_per_tile + cell, kind="stable") bit for
// bit.  Work is split into chunks of 4096 consecutive elements, one CTA each:
//
// (1) k_sort_keys computes K for every point (one pass over the coordinates)
//     and each chunk's histogram of the first radix digit, written as row
//     `chunk` of a chunk-major count matrix;
// (2) per radix digit (1 to 3 digits of at most 11 bits, least significant
//     first): k_digit_count (digits after the first) fills the matrix from the
//     previous pass's output, k_col_scan turns every column into the counts of
//     the chunks before each chunk plus the digit's total, and
//     k_radix_scatter ranks equal digits stably within the chunk (one ballot
//     per digit bit inside each 32-element round, per-warp running counts
//     across rounds), stages the chunk in shared memory in digit order and
//     writes it out as contiguous runs per digit;
// (3) every point's folded coordinates in sorted order (the spread / interp /
//     gradient passes then stream them instead of gathering through the
//     permutation): float coordinates are written in input order by
//     k_sort_keys and carried through the scatter passes as payload (coalesced
//     reads, run-wise writes); double and type-3 points get them from
//     k_sorted_coords, which gathers through the permutation (and computes the
//     type-3 factor).  k_bin_bounds reads the bin starts
//     off the sorted keys, and k_subproblems splits bins larger than
//     max_subproblem points into subproblems so clustered inputs spread evenly
//     over the SMs.  Points of a subproblem are ordered by cell, which lets
//     spreading merge runs of points that share a cell and gives interpolation
//     near-identical addresses per warp.
// No CTA waits for another: every dependency is a kernel boundary.
#include <algorithm>
#include <type_traits>

#include "nfx_internal.h"

namespace nfx {

// Lanes of the warp holding the same key as this lane: one ballot per key bit.
// Keys are in [-1, 2^NB - 1); the +1 shift keeps the inactive lanes (-1) apart
// from every real key within NB bits (a compile-time count: fully unrolled).
template <int NB>
__device__ __forceinline__ unsigned peer_mask(int key) {
  const unsigned k = (unsigned)(key + 1);
  unsigned m = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const unsigned bit = (k >> b) & 1u;
    const unsigned bal = __ballot_sync(0xffffffffu, bit);
    m &= bit ? bal : ~bal;
  }
  return m;
}

// Bin of the tile holding the footprint's left cell, and that cell's index
// inside the tile (both x-fastest), from the point's coordinates.
// xs[d]: the folded, rescaled coordinate the key came from.
template <typename T, int DIM, bool T3>
__device__ __forceinline__ void cell_keys(const T (&c)[DIM], const Geom& g, int ns_half, int& kbin, int& kcell,
                                          T (&xs)[DIM]) {
  int kb = 0, kc = 0, mb = 1, mc = 1;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    xs[d] = T3 ? point_fold(c[d], d, g) : scaled_coord(c[d], g.nf[d], g.prenorm);
    const int i0w = wrap_index(ceil_to_int(rn_sub(xs[d], (T)ns_half)), g.nf[d]);
    const int bq = fast_div(i0w, g.tdiv[d]);
    kb += bq * mb;
    kc += (i0w - bq * g.tile[d]) * mc;
    mb *= g.nb[d];
    mc *= g.tile[d];
  }
  kbin = kb;
  kcell = kc;
}

// ---- block-wide exclusive scan of one int per thread ----------------------
__device__ __forceinline__ int block_exclusive_scan(int v, int* s_warp, int& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int n = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += n;
  }
  if (lane == 31) s_warp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    int t = lane < nw ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int n = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += n;
    }
    if (lane < nw) s_warp[lane] = t;
  }
  __syncthreads();
  total = s_warp[(blockDim.x >> 5) - 1];
  const int res = inc - v + (wid > 0 ? s_warp[wid - 1] : 0);
  __syncthreads();
  return res;
}


constexpr int kRadixThreads = 256;
constexpr int kRadixItems = 16;
constexpr int kRadixChunk = kRadixThreads * kRadixItems;  // elements per chunk (one CTA)

// ---- (1) composite keys + the first digit's per-chunk counts ---------------
// One CTA per chunk of kRadixChunk consecutive points: K = bin << cbits | cell
// for every point, and the chunk's histogram of digit 0 as row `chunk` of
// counts (chunk-major, so the row is one coalesced write).
// T3: the points are type-3 sources or targets (Geom::t3_mode), a separate
// instantiation so the common kernel carries no type-3 code.
// f[d] (nullptr: not wanted): every point's folded coordinates in input order,
// the payload the scatter passes then carry into sorted order.
template <typename T, int DIM, bool T3>
__global__ void __launch_bounds__(kRadixThreads) k_sort_keys(const T* __restrict__ x, const T* __restrict__ y,
                                                            const T* __restrict__ z, int M, Geom g, int ns_half,
                                                            int cbits, int dbits, int* __restrict__ K,
                                                            int* __restrict__ counts, T* __restrict__ f0,
                                                            T* __restrict__ f1, T* __restrict__ f2) {
  extern __shared__ int s_h[];
  const int B = 1 << dbits;
  const int mask = B - 1;
  for (int i = threadIdx.x; i < B; i += blockDim.x) s_h[i] = 0;
  __syncthreads();
  const int c0 = blockIdx.x * kRadixChunk;
  const T* cs[3] = {x, y, z};
  // all coordinate loads first, so they are in flight together
  T cv[kRadixItems][DIM];
#pragma unroll
  for (int u = 0; u < kRadixItems; ++u) {
    const int p = c0 + u * kRadixThreads + threadIdx.x;
#pragma unroll
    for (int d = 0; d < DIM; ++d) cv[u][d] = p < M ? cs[d][p] : (T)0;
  }
#pragma unroll
  for (int u = 0; u < kRadixItems; ++u) {
    const int p = c0 + u * kRadixThreads + threadIdx.x;
    if (p < M) {
      int kb, kc;
      T xs[DIM];
      cell_keys<T, DIM, T3>(cv[u], g, ns_half, kb, kc, xs);
      const int key = (kb << cbits) | kc;
      K[p] = key;
      atomicAdd(&s_h[key & mask], 1);
      if (f0 != nullptr) {
        f0[p] = xs[0];
        if (DIM > 1) f1[p] = xs[DIM > 1 ? 1 : 0];
        if (DIM > 2) f2[p] = xs[DIM > 2 ? 2 : 0];
      }
    }
  }
  __syncthreads();
  int* row = counts + (size_t)blockIdx.x * B;
  for (int i = threadIdx.x; i < B; i += blockDim.x) row[i] = s_h[i];
}

// Per-chunk counts of digit (K >> shift) & (B - 1), for the passes after the first.
__global__ void __launch_bounds__(kRadixThreads) k_digit_count(const int* __restrict__ kin, int M, int shift,
                                                              int dbits, int* __restrict__ counts) {
  extern __shared__ int s_h[];
  const int B = 1 << dbits;
  const int mask = B - 1;
  for (int i = threadIdx.x; i < B; i += blockDim.x) s_h[i] = 0;
  __syncthreads();
  const int c0 = blockIdx.x * kRadixChunk;
  int key[kRadixItems];
#pragma unroll
  for (int u = 0; u < kRadixItems; ++u) {
    const int p = c0 + u * kRadixThreads + threadIdx.x;
    key[u] = p < M ? kin[p] : -1;
  }
#pragma unroll
  for (int u = 0; u < kRadixItems; ++u)
    if (key[u] >= 0) atomicAdd(&s_h[(key[u] >> shift) & mask], 1);
  __syncthreads();
  int* row = counts + (size_t)blockIdx.x * B;
  for (int i = threadIdx.x; i < B; i += blockDim.x) row[i] = s_h[i];
}

// ---- (2a) column scan of the counts -----------------------------------------
// counts[chunk][d] becomes the number of digit-d elements in the chunks before
// `chunk`; totals[d] = all of them.  A block takes 8 digit columns; its 1024
// threads are 8 digits x 128 contiguous chunk groups, and warp d scans the
// 128 group sums of digit d in shared memory.
constexpr int kScanDigits = 8;
constexpr int kScanGroups = 128;
__global__ void __launch_bounds__(kScanDigits * kScanGroups) k_col_scan(int* __restrict__ counts, int nchunks, int B,
                                                                        int* __restrict__ totals) {
  __shared__ int s_sum[kScanGroups][kScanDigits + 1];
  const int dl = threadIdx.x % kScanDigits;
  const int gy = threadIdx.x / kScanDigits;
  const int d = blockIdx.x * kScanDigits + dl;
  const int per = (nchunks + kScanGroups - 1) / kScanGroups;
  const int cg0 = min(gy * per, nchunks);
  const int cg1 = min(cg0 + per, nchunks);
  int sum = 0;
  if (d < B) {
#pragma unroll 8
    for (int c = cg0; c < cg1; ++c) sum += counts[(size_t)c * B + d];
  }
  s_sum[gy][dl] = sum;
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w < kScanDigits) {  // warp w: exclusive scan of digit w's group sums, 4 groups a lane
    int v[kScanGroups / 32];
    int t = 0;
#pragma unroll
    for (int j = 0; j < kScanGroups / 32; ++j) {
      v[j] = s_sum[lane * (kScanGroups / 32) + j][w];
      t += v[j];
    }
    int inc = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int n = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += n;
    }
    int run = inc - t;
#pragma unroll
    for (int j = 0; j < kScanGroups / 32; ++j) {
      s_sum[lane * (kScanGroups / 32) + j][w] = run;
      run += v[j];
    }
    const int dw = blockIdx.x * kScanDigits + w;
    if (lane == 31 && dw < B) totals[dw] = inc;
  }
  __syncthreads();
  if (d < B) {
    int run = s_sum[gy][dl];
#pragma unroll 8
    for (int c = cg0; c < cg1; ++c) {
      const size_t i = (size_t)c * B + d;
      const int t = counts[i];
      counts[i] = run;
      run += t;
    }
  }
}

// ---- (2b) one stable scatter pass --------------------------------------------
// Shared memory: per-warp digit counts (later reused for the staged chunk), the
// chunk's digit starts and each digit's output offset.
// Shared-memory ints of the region that first holds the per-warp digit counts
// and then the staged chunk (keys, values and PD payload words per element).
__host__ __device__ constexpr int radix_region_ints(int B, int PD) {
  return (kRadixThreads / 32) * B > (2 + PD) * kRadixChunk ? (kRadixThreads / 32) * B : (2 + PD) * kRadixChunk;
}
__host__ __device__ constexpr size_t radix_smem_bytes(int B, int PD) {
  return (size_t)(radix_region_ints(B, PD) + 2 * B) * sizeof(int);
}

// Float words carried with every element through a pass (the folded
// coordinates, one array per axis): in[d][i] belongs to input element i and
// lands at out[d][j] where the element lands.
struct RadixPayload {
  const float* in[3];
  float* out[3];
};

// kin/vin: this pass's input keys and values (vin == nullptr: the values are
// the element indices); kout/vout: the output, stable by digit
// (kin >> shift) & (2^dbits - 1).  prefix[chunk][d]: digit-d elements in the
// chunks before this one; totals[d]: digit-d elements overall.  PD payload
// arrays move with the elements (pay).  bstart (not nullptr only in a last
// pass whose digit is the bin): CTA 0 writes the bin starts (the exclusive
// scan of the digit totals), bstart[0..nbins].  DB = dbits (compile time, so
// the ranking's ballots unroll); DPT = digits per thread, max(1, 2^DB / 256).
template <int DB, int PD, int DPT = (((1 << DB) + kRadixThreads - 1) / kRadixThreads)>
__global__ void __launch_bounds__(kRadixThreads, 3) k_radix_scatter(const int* __restrict__ kin,
                                                                const int* __restrict__ vin, int M, int shift,
                                                                int dbits, const int* __restrict__ prefix,
                                                                const int* __restrict__ totals,
                                                                int* __restrict__ kout, int* __restrict__ vout,
                                                                RadixPayload pay, int* __restrict__ bstart,
                                                                int nbins) {
  extern __shared__ int smem[];
  __shared__ int s_warp[32];
  constexpr int W = kRadixThreads / 32;
  constexpr int B = 1 << DB;
  constexpr int mask = B - 1;
  int* s_hw = smem;                                 // [W][B] per-warp digit counts
  int* s_key = smem;                                // [kRadixChunk] staged keys (after ranking)
  int* s_val = smem + kRadixChunk;                  // [kRadixChunk] staged values
  float* s_pay = reinterpret_cast<float*>(smem + 2 * kRadixChunk);  // [PD][kRadixChunk] staged payload
  int* s_dstart = smem + radix_region_ints(B, PD);  // [B] digit starts within the chunk
  int* s_gofs = s_dstart + B;                       // [B] output index - staged index, per digit
  for (int i = threadIdx.x; i < W * B; i += blockDim.x) s_hw[i] = 0;
  const int ch = blockIdx.x;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c0 = ch * kRadixChunk;
  const int wbase = c0 + w * (kRadixItems * 32);
  // keys now; values (and payload) only when the chunk is staged, so that the
  // unrolled ranking does not hold them in registers
  int key[kRadixItems], rk[kRadixItems];
#pragma unroll
  for (int r = 0; r < kRadixItems; ++r) {
    const int p = wbase + r * 32 + lane;
    key[r] = p < M ? kin[p] : -1;
  }
  // this thread's digits (a contiguous range): their totals and the counts of
  // the chunks before this one, fetched now so the loads overlap the ranking
  constexpr int kMaxDpt = DPT;  // ceil(2^dbits / threads)
  const int d0 = min((int)threadIdx.x * DPT, B);
  const int d1 = min(d0 + DPT, B);
  int tot_d[kMaxDpt], pre_d[kMaxDpt];
  const int* pre = prefix + (size_t)ch * B;
#pragma unroll
  for (int j = 0; j < kMaxDpt; ++j) {
    tot_d[j] = d0 + j < d1 ? totals[d0 + j] : 0;
    pre_d[j] = d0 + j < d1 ? pre[d0 + j] : 0;
  }
  __syncthreads();
  // stable rank of each element among the equal digits of its warp: the first
  // lane of each group of equal digits in a 32-element round adds the group's
  // size to the warp's running count with one returning shared atomic (a warp's
  // shared atomics complete in issue order, so rounds stay in order), and the
  // group reads the old count from that lane
  const unsigned lt = (1u << lane) - 1u;
  int* hw = s_hw + w * B;
#pragma unroll
  for (int r = 0; r < kRadixItems; ++r) {
    const int d = key[r] >= 0 ? (key[r] >> shift) & mask : -1;
    // DB + 1 bits: digits shifted by one so the invalid lanes (-1) stay apart
    const unsigned peers = peer_mask<DB + 1>(d);
    const int rank = __popc(peers & lt);
    int pos = 0;
    if (d >= 0 && rank == 0) pos = atomicAdd(&hw[d], __popc(peers));
    pos = __shfl_sync(0xffffffffu, pos, __ffs(peers) - 1);
    rk[r] = pos + rank;
  }
  __syncthreads();
  // per digit: the warps' exclusive starts, the chunk's count, and the digit's
  // global start (exclusive scan of the totals)
  int cnt_d[kMaxDpt];
  int mine = 0, tot = 0;
#pragma unroll
  for (int j = 0; j < kMaxDpt; ++j) {
    const int d = d0 + j;
    int c[W];
#pragma unroll
    for (int v = 0; v < W; ++v) c[v] = d < d1 ? s_hw[v * B + d] : 0;
    int run = 0;
#pragma unroll
    for (int v = 0; v < W; ++v) {
      if (d < d1) s_hw[v * B + d] = run;
      run += c[v];
    }
    cnt_d[j] = run;
    mine += run;
    tot += tot_d[j];
  }
  int total;
  int run = block_exclusive_scan(mine, s_warp, total);
  int gbase = block_exclusive_scan(tot, s_warp, total);
#pragma unroll
  for (int j = 0; j < kMaxDpt; ++j) {
    const int d = d0 + j;
    if (d < d1) {
      s_dstart[d] = run;
      s_gofs[d] = gbase + pre_d[j] - run;
      if (bstart != nullptr && blockIdx.x == 0 && d < nbins) bstart[d] = gbase;
    }
    run += cnt_d[j];
    gbase += tot_d[j];
  }
  if (bstart != nullptr && blockIdx.x == 0 && threadIdx.x == 0) bstart[nbins] = M;
  __syncthreads();
  // staged (digit-ordered) index of every element
#pragma unroll
  for (int r = 0; r < kRadixItems; ++r) {
    if (key[r] >= 0) {
      const int d = (key[r] >> shift) & mask;
      rk[r] += s_dstart[d] + hw[d];
    }
  }
  __syncthreads();  // the per-warp counts are dead: the region now holds the staged chunk
  {
    int val[kRadixItems];
#pragma unroll
    for (int r = 0; r < kRadixItems; ++r) {
      const int p = wbase + r * 32 + lane;
      val[r] = key[r] >= 0 ? (vin != nullptr ? vin[p] : p) : 0;
    }
#pragma unroll
    for (int r = 0; r < kRadixItems; ++r) {
      if (key[r] >= 0) {
        s_key[rk[r]] = key[r];
        s_val[rk[r]] = val[r];
      }
    }
  }
#pragma unroll
  for (int d = 0; d < PD; ++d) {
    float pv[kRadixItems];
#pragma unroll
    for (int r = 0; r < kRadixItems; ++r) {
      const int p = wbase + r * 32 + lane;
      pv[r] = p < M ? pay.in[d][p] : 0.f;
    }
#pragma unroll
    for (int r = 0; r < kRadixItems; ++r)
      if (key[r] >= 0) s_pay[d * kRadixChunk + rk[r]] = pv[r];
  }
  __syncthreads();
  const int n_here = M - c0 < kRadixChunk ? M - c0 : kRadixChunk;
  for (int i = threadIdx.x; i < n_here; i += blockDim.x) {
    const int k = s_key[i];
    const int gpos = s_gofs[(k >> shift) & mask] + i;
    if ((unsigned)gpos < (unsigned)M) {  // always: counts and keys come from the same array
      kout[gpos] = k;
      vout[gpos] = s_val[i];
#pragma unroll
      for (int d = 0; d < PD; ++d) pay.out[d][gpos] = s_pay[d * kRadixChunk + i];
    }
  }
}

// The scatter instantiation for dbits-bit digits (1..11) and PD payload arrays.
using ScatterFn = void (*)(const int*, const int*, int, int, int, const int*, const int*, int*, int*, RadixPayload,
                           int*, int);
template <int PD>
static ScatterFn scatter_for_digits(int dbits) {
  switch (dbits) {
    case 1: return k_radix_scatter<1, PD>;
    case 2: return k_radix_scatter<2, PD>;
    case 3: return k_radix_scatter<3, PD>;
    case 4: return k_radix_scatter<4, PD>;
    case 5: return k_radix_scatter<5, PD>;
    case 6: return k_radix_scatter<6, PD>;
    case 7: return k_radix_scatter<7, PD>;
    case 8: return k_radix_scatter<8, PD>;
    case 9: return k_radix_scatter<9, PD>;
    case 10: return k_radix_scatter<10, PD>;
    default: return k_radix_scatter<11, PD>;
  }
}
static ScatterFn scatter_for(int dbits, int PD) {
  return PD == 0 ? scatter_for_digits<0>(dbits)
                 : (PD == 1 ? scatter_for_digits<1>(dbits)
                            : (PD == 2 ? scatter_for_digits<2>(dbits) : scatter_for_digits<3>(dbits)));
}

// ---- (3) bin starts and subproblems ----------------------------------------
// bin_start[b] = first sorted position whose key lies in bin b (M for bins past
// the last point); position i writes the starts of every bin in
// (bin of i-1, bin of i].  Each thread takes 4 consecutive positions (one
// vector load).
__global__ void k_bin_bounds(const int* __restrict__ Ks, int M, int cbits, int nbins, int* __restrict__ bin_start) {
  const int nq = M / 4 + 1;  // quads covering positions 0..M
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nq; t += gridDim.x * blockDim.x) {
    const int i0 = 4 * t;
    int k[4];
    if (i0 + 3 < M) {
      const int4 v = *reinterpret_cast<const int4*>(Ks + i0);
      k[0] = v.x;
      k[1] = v.y;
      k[2] = v.z;
      k[3] = v.w;
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) k[j] = i0 + j < M ? Ks[i0 + j] : 0;
    }
    int bp = i0 > 0 ? min(Ks[i0 - 1] >> cbits, nbins) : -1;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int i = i0 + j;
      if (i > M) break;
      const int b = i < M ? min(k[j] >> cbits, nbins) : nbins;  // clamped: keys are in range
      for (int bb = bp + 1; bb <= b; ++bb) bin_start[bb] = i;
      bp = b;
    }
  }
}

// Bin b gets ceil(count_b / maxsub) subproblems.  One block: each thread
// counts a contiguous run of bins, a block scan gives every bin its first
// subproblem, and then (when the per-bin firsts fit in shared memory) all
// threads fill the tables together, each locating its subproblem's bin by
// binary search; otherwise each thread fills its own bins.
constexpr int kSubSmemBins = 12288;
__global__ void k_subproblems(const int* __restrict__ bin_start, int nbins, int maxsub, int max_subs,
                              int* __restrict__ sub_bin, int* __restrict__ sub_start, int* __restrict__ nsub_out) {
  __shared__ int s_warp[32];
  extern __shared__ int s_first[];  // [nbins + 1] when nbins <= kSubSmemBins
  const int tid = threadIdx.x;
  const int nt = blockDim.x;
  const int per = (nbins + nt - 1) / nt;
  const int b0 = min(tid * per, nbins);
  const int b1 = min(b0 + per, nbins);
  int local = 0;
  for (int b = b0; b < b1; ++b) local += max(bin_start[b + 1] - bin_start[b] + maxsub - 1, 0) / maxsub;
  int total;
  int excl = block_exclusive_scan(local, s_warp, total);
  const int nsub = min(total, max_subs);  // the tables hold max_subs entries (more only for corrupt bounds)
  if (tid == 0) *nsub_out = nsub;
  if (nbins <= kSubSmemBins) {
    for (int b = b0; b < b1; ++b) {
      s_first[b] = excl;
      excl += max(bin_start[b + 1] - bin_start[b] + maxsub - 1, 0) / maxsub;
    }
    if (tid == 0) s_first[nbins] = total;
    __syncthreads();
    for (int sidx = tid; sidx < nsub; sidx += nt) {
      int lo = 0, hi = nbins;  // last bin with s_first[bin] <= sidx
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (s_first[mid] <= sidx)
          lo = mid;
        else
          hi = mid;
      }
      sub_bin[sidx] = lo;
      sub_start[sidx] = bin_start[lo] + (sidx - s_first[lo]) * maxsub;
    }
  } else {
    for (int b = b0; b < b1; ++b) {
      const int e = bin_start[b + 1];
      for (int q = bin_start[b]; q < e && excl < max_subs; q += maxsub) {
        sub_bin[excl] = b;
        sub_start[excl] = q;
        ++excl;
      }
    }
  }
}

// ---- (3a) folded coordinates in sorted order ----------------------------------
// coord_d[k] = fold(x_d[perm[k]]) for every axis: the same float operations as
// the keys (so the spread / interp passes see exactly the coordinates the sort
// binned), written once in sorted order.  Each thread takes 4 consecutive
// positions: one vector load of the permutation, all gathers in flight together,
// one vector store per axis.  Type-3 sorts also write extra[k], the point's
// complex factor (Geom::t3_mode): sources the pre-phase e^{i isign sum D_d x_d}
// (nufft3.py:275-280, 368-372), targets e^{i isign sum (s_d - D_d) C_d} /
// prod_d phihat(s'_d) with phihat by the reference's trapezoid on
// [-ns/2, ns/2] (nufft3.py:176-213, 390-394), in double before one rounding.
constexpr int kMaxQuad = 32;

template <typename T>
__device__ __forceinline__ cplx_t<T> t3_factor(const T (&xr)[3], int dim, const Geom& g, int nq, double dz,
                                               const double* __restrict__ s_qw) {
  const T3Params* p = g.t3;
  double phase = 0.0, phi_prod = 1.0;
  for (int d = 0; d < dim; ++d) {
    if (g.t3_mode == 1) {
      phase += p->D[d] * (double)xr[d];
    } else {
      const double sr = (double)t3_rescaled(xr[d], d, g);
      double acc = 0.0;
      for (int q = 0; q < nq; ++q) acc += s_qw[q] * cos(sr * (-0.5 * dz * (nq - 1) + q * dz));
      phi_prod *= acc;
      phase += ((double)xr[d] - p->D[d]) * p->C[d];
    }
  }
  double sn, cs;
  sincos(phase * (double)g.t3_isign, &sn, &cs);
  cplx_t<T> f;
  f.x = (T)(cs / phi_prod);
  f.y = (T)(sn / phi_prod);
  return f;
}

__device__ __forceinline__ void store_quad(float* o, const float (&r)[4]) {
  *reinterpret_cast<float4*>(o) = make_float4(r[0], r[1], r[2], r[3]);
}
__device__ __forceinline__ void store_quad(double* o, const double (&r)[4]) {
  reinterpret_cast<double2*>(o)[0] = make_double2(r[0], r[1]);
  reinterpret_cast<double2*>(o)[1] = make_double2(r[2], r[3]);
}

constexpr int kCoordItems = 8;  // sorted positions per thread of k_sorted_coords

template <typename T, int DIM, bool T3>
__global__ void __launch_bounds__(256) k_sorted_coords(const T* __restrict__ x, const T* __restrict__ y,
                                                       const T* __restrict__ z, const int* __restrict__ perm, int M,
                                                       Geom g, int nspread, T* __restrict__ o0, T* __restrict__ o1,
                                                       T* __restrict__ o2, cplx_t<T>* __restrict__ extra) {
  constexpr int Q = kCoordItems;
  // trapezoid nodes and weights phi(z_q) w_q of the type-3 targets' phihat
  __shared__ double s_qw[kMaxQuad];
  const double j2 = nspread / 2.0;
  const int nq = min(max((int)(4 + 3.0 * j2), 20), kMaxQuad);
  const double dz = 2.0 * j2 / (nq - 1);
  if (T3 && g.t3_mode == 2) {
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
      const double zq = -j2 + q * dz;
      const double arg = 1.0 - g.t3_kc * zq * zq;
      const double phi = arg >= 0.0 ? exp(g.t3_beta * (sqrt(arg > 0.0 ? arg : 0.0) - 1.0)) : 0.0;
      s_qw[q] = phi * ((q == 0 || q == nq - 1) ? dz / 2 : dz);
    }
    __syncthreads();
  }
  const int ngroups = (M + Q - 1) / Q;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ngroups; t += gridDim.x * blockDim.x) {
    const int i0 = Q * t;
    int p[Q];
    if (i0 + Q - 1 < M) {
#pragma unroll
      for (int h = 0; h < Q / 4; ++h) {
        const int4 v = *reinterpret_cast<const int4*>(perm + i0 + 4 * h);  // 16-byte aligned
        p[4 * h] = v.x;
        p[4 * h + 1] = v.y;
        p[4 * h + 2] = v.z;
        p[4 * h + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int j = 0; j < Q; ++j) p[j] = i0 + j < M ? perm[i0 + j] : -1;
    }
    // every gather of the group in flight before any use
    T v[DIM][Q];
#pragma unroll
    for (int j = 0; j < Q; ++j) {
      v[0][j] = p[j] >= 0 ? x[p[j]] : (T)0;
      if (DIM > 1) v[DIM > 1 ? 1 : 0][j] = p[j] >= 0 ? y[p[j]] : (T)0;
      if (DIM > 2) v[DIM > 2 ? 2 : 0][j] = p[j] >= 0 ? z[p[j]] : (T)0;
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      T* od = d == 0 ? o0 : (d == 1 ? o1 : o2);
      T r[Q];
#pragma unroll
      for (int j = 0; j < Q; ++j) r[j] = T3 ? point_fold(v[d][j], d, g) : scaled_coord(v[d][j], g.nf[d], g.prenorm);
      if (i0 + Q - 1 < M) {
#pragma unroll
        for (int h = 0; h < Q / 4; ++h) {
          const T rq[4] = {r[4 * h], r[4 * h + 1], r[4 * h + 2], r[4 * h + 3]};
          store_quad(od + i0 + 4 * h, rq);  // 16-byte aligned: 256-aligned arrays, i0 % 8 == 0
        }
      } else {
#pragma unroll
        for (int j = 0; j < Q; ++j)
          if (p[j] >= 0) od[i0 + j] = r[j];
      }
    }
    if constexpr (T3) {
#pragma unroll 1
      for (int j = 0; j < Q; ++j) {
        if (p[j] < 0) continue;
        T xr[3] = {(T)0, (T)0, (T)0};
#pragma unroll
        for (int d = 0; d < DIM; ++d) xr[d] = v[d][j];
        extra[i0 + j] = t3_factor<T>(xr, DIM, g, nq, dz, s_qw);
      }
    }
  }
}

__global__ void k_keys_to_bins(const int* __restrict__ K, int64_t M, int cbits, int* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = K[i] >> cbits;
}

// ---------------------------------------------------------------------------

// Key layout (cell bits, total bits), the number of passes and the digit width.
void radix_plan(int nbins, int ncell, int& cbits, int& bits, int& npass, int& dbits) {
  cbits = 0;
  while ((1 << cbits) < ncell) ++cbits;
  int bbits = 0;
  while ((1 << bbits) < nbins) ++bbits;
  bits = cbits + bbits > 0 ? cbits + bbits : 1;
  npass = bits <= 11 ? 1 : (bits <= 22 ? 2 : 3);
  dbits = (bits + npass - 1) / npass;
}

int radix_chunk() { return kRadixChunk; }

cudaError_t bin_keys_of(const SortLayout& L, const int* K, int* out, cudaStream_t st) {
  if (L.M == 0) return cudaSuccess;
  const int grid = (int)std::min<int64_t>((L.M + 255) / 256, (int64_t)num_sms() * 8);
  k_keys_to_bins<<<grid, 256, 0, st>>>(K, L.M, L.cbits, out);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_sort(const SortLayout& L, const Geom& g, int ns, const void* x, const void* y, const void* z,
                        int64_t M, const SortPtrs& P, cudaStream_t st) {
  const int B = 1 << L.dbits;
  cudaError_t e = cudaSuccess;
  // float coordinates of non-type-3 points ride through the passes as payload
  // (the layout then holds coord_tmp); otherwise k_sorted_coords gathers them
  const bool carry = std::is_same<T, float>::value && P.coord_tmp[0] != nullptr;
  const int PD = carry ? g.dim : 0;
  if (M > 0) {
    const size_t hist_smem = (size_t)B * sizeof(int);
    // digits per thread of the scatter: 2^dbits / 256, at least 1
    const ScatterFn scatter = scatter_for(L.dbits, PD);
    e = ensure_smem(reinterpret_cast<const void*>(scatter), radix_smem_bytes(B, PD));
    if (e == cudaSuccess) e = prefer_max_smem(reinterpret_cast<const void*>(scatter));
    if (e != cudaSuccess) return e;
    const unsigned scan_grid = (unsigned)((B + kScanDigits - 1) / kScanDigits);
    auto keys = g.t3_mode != 0
                    ? (g.dim == 1 ? k_sort_keys<T, 1, true> : (g.dim == 2 ? k_sort_keys<T, 2, true> : k_sort_keys<T, 3, true>))
                    : (g.dim == 1 ? k_sort_keys<T, 1, false>
                                  : (g.dim == 2 ? k_sort_keys<T, 2, false> : k_sort_keys<T, 3, false>));
    // ping-pong so that the last pass writes (keys_sorted, perm[, coord]); the
    // keys kernel writes the input-order coordinates into the buffer the first
    // pass does not write
    void* const* cfirst = (L.npass % 2 == 0) ? P.coord : P.coord_tmp;
    keys<<<L.nchunks, kRadixThreads, hist_smem, st>>>(
        (const T*)x, (const T*)y, (const T*)z, (int)M, g, ns / 2, L.cbits, L.dbits, P.keys, P.counts,
        carry ? (T*)cfirst[0] : nullptr, carry ? (T*)cfirst[1] : nullptr, carry ? (T*)cfirst[2] : nullptr);
    const int* kin = P.keys;
    const int* vin = nullptr;
    void* const* cin = cfirst;
    for (int ps = 0; ps < L.npass; ++ps) {
      const int shift = ps * L.dbits;
      if (ps > 0) k_digit_count<<<L.nchunks, kRadixThreads, hist_smem, st>>>(kin, (int)M, shift, L.dbits, P.counts);
      k_col_scan<<<scan_grid, kScanDigits * kScanGroups, 0, st>>>(P.counts, L.nchunks, B, P.totals);
      const bool to_final = ((L.npass - 1 - ps) % 2) == 0;
      int* kout = to_final ? P.keys_sorted : P.keys_tmp;
      int* vout = to_final ? P.perm : P.vals_tmp;
      void* const* cout = to_final ? P.coord : P.coord_tmp;
      RadixPayload pay{{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
      for (int d = 0; d < PD; ++d) {
        pay.in[d] = (const float*)cin[d];
        pay.out[d] = (float*)cout[d];
      }
      // the last pass's digit is the bin when it starts at the cell bits
      int* bstart = (ps == L.npass - 1 && shift == L.cbits) ? P.bin_start : nullptr;
      scatter<<<L.nchunks, kRadixThreads, radix_smem_bytes(B, PD), st>>>(
          kin, vin, (int)M, shift, L.dbits, P.counts, P.totals, kout, vout, pay, bstart, g.nbins);
      kin = kout;
      vin = vout;
      cin = cout;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  const int bgrid = (int)std::max<int64_t>(1, std::min<int64_t>((M / 4 + 256) / 256, (int64_t)num_sms() * 8));
  if (M > 0 && !carry) {
    auto sc = g.t3_mode != 0 ? (g.dim == 1 ? k_sorted_coords<T, 1, true>
                                           : (g.dim == 2 ? k_sorted_coords<T, 2, true> : k_sorted_coords<T, 3, true>))
                             : (g.dim == 1 ? k_sorted_coords<T, 1, false>
                                           : (g.dim == 2 ? k_sorted_coords<T, 2, false> : k_sorted_coords<T, 3, false>));
    const int cgrid =
        (int)std::max<int64_t>(1, std::min<int64_t>((M / kCoordItems + 256) / 256, (int64_t)num_sms() * 8));
    sc<<<cgrid, 256, 0, st>>>((const T*)x, (const T*)y, (const T*)z, P.perm, (int)M, g, ns, (T*)P.coord[0],
                              (T*)P.coord[1], (T*)P.coord[2], (cplx_t<T>*)P.extra);
  }
  const bool fused_bounds = M > 0 && (int64_t)(L.npass - 1) * L.dbits == L.cbits;
  if (!fused_bounds) k_bin_bounds<<<bgrid, 256, 0, st>>>(P.keys_sorted, (int)M, L.cbits, g.nbins, P.bin_start);
  const int max_subs = (int)std::min<int64_t>(L.max_subs, INT32_MAX);
  const size_t sub_smem = g.nbins <= kSubSmemBins ? (size_t)(g.nbins + 1) * sizeof(int) : 0;
  k_subproblems<<<1, 1024, sub_smem, st>>>(P.bin_start, g.nbins, L.maxsub, max_subs, P.sub_bin, P.sub_start,
                                           P.nsub);
  return cudaGetLastError();
}

template cudaError_t launch_sort<float>(const SortLayout&, const Geom&, int, const void*, const void*, const void*,
                                        int64_t, const SortPtrs&, cudaStream_t);
template cudaError_t launch_sort<double>(const SortLayout&, const Geom&, int, const void*, const void*, const void*,
                                         int64_t, const SortPtrs&, cudaStream_t);

}  // namespace nfx
