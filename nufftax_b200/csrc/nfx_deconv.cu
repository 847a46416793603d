// Fused deconvolution + mode reordering around the FFT.
//
// Type 1 (nufftax/core/deconvolve.py:81-111, 174-224, 312-366): one pass reads
//   the FFT output at k mod nf for every kept mode k in CMCL order
//   (k = -N/2 .. (N-1)/2 per axis) and multiplies by the per-axis factors
//   fac_d[k] = (-1)^k / phihat_d(|k|) (deconvolve.py:27-56), outer product in the
//   reference's order (fac3 * fac2) * fac1.  Output is written coalesced along x.
// Type 2 (deconvolve.py:114-166, 227-304, 369-468): one pass writes every
//   cell of the fine grid: the deconvolved mode where the cell is a kept mode,
//   zero elsewhere (no separate memset of the grid).
#include <algorithm>
#include <type_traits>

#include "nfx_internal.h"

namespace nfx {

// Both passes go row by row (a row = one (transform, z, y) line along x, cut
// into segments of kSeg elements, one warp per segment): the row's indices
// come from one division chain per segment, so no thread divides per element.
// A lane takes kSeg / 32 elements of its segment, all loads issued before any
// store (unrolled), so every lane has that many reads in flight; segments are
// short enough that a 2D grid of 512 or 1024 rows still gives thousands of
// warps.
constexpr int kSeg = 128;
constexpr int kSegPerLane = kSeg / 32;
template <typename T>
__global__ void k_deconv_shuffle(int nf1, int nf2, int nf3, int n1, int n2, int n3, const T* __restrict__ f1,
                                 const T* __restrict__ f2, const T* __restrict__ f3,
                                 const cplx_t<T>* __restrict__ in, cplx_t<T>* __restrict__ out, int n_trans) {
  using CT = cplx_t<T>;
  const int64_t grid = (int64_t)nf1 * nf2 * nf3;
  const int nseg = (n1 + kSeg - 1) / kSeg;
  const int64_t nitems = (int64_t)n2 * n3 * n_trans * nseg;
  const int k1min = -(n1 / 2), k2min = -(n2 / 2), k3min = -(n3 / 2);
  const int nw = blockDim.x >> 5, lane = threadIdx.x & 31;
  for (int64_t item = (int64_t)blockIdx.x * nw + (threadIdx.x >> 5); item < nitems; item += (int64_t)gridDim.x * nw) {
    const int64_t row = item / nseg;
    const int x0 = (int)(item - row * nseg) * kSeg;
    const int x1 = min(x0 + kSeg, n1);
    const int64_t t = row / ((int64_t)n2 * n3);
    const int rr = (int)(row - t * n2 * n3);
    const int p2 = rr % n2;
    const int p3 = rr / n2;
    int i2 = p2 + k2min, i3 = p3 + k3min;
    if (i2 < 0) i2 += nf2;
    if (i3 < 0) i3 += nf3;
    T fac23 = (T)1;
    if (f2 != nullptr) fac23 = f3 != nullptr ? f3[p3] * f2[p2] : f2[p2];
    const CT* src = in + t * grid + ((int64_t)i3 * nf2 + i2) * nf1;
    CT* dst = out + row * n1;
    CT v[kSegPerLane];
    T f[kSegPerLane];
#pragma unroll
    for (int j = 0; j < kSegPerLane; ++j) {
      const int p1 = x0 + lane + 32 * j;
      if (p1 < x1) {
        int i1 = p1 + k1min;
        if (i1 < 0) i1 += nf1;
        v[j] = src[i1];
        f[j] = f1[p1];
      }
    }
#pragma unroll
    for (int j = 0; j < kSegPerLane; ++j) {
      const int p1 = x0 + lane + 32 * j;
      if (p1 < x1) {
        // (fac3 * fac2) * fac1, the reference's order
        const T fac = f2 != nullptr ? fac23 * f[j] : f[j];
        CT o;
        o.x = v[j].x * fac;
        o.y = v[j].y * fac;
        dst[p1] = o;
      }
    }
  }
}

template <typename T>
__global__ void k_deconv_pad(int nf1, int nf2, int nf3, int n1, int n2, int n3, const T* __restrict__ f1,
                             const T* __restrict__ f2, const T* __restrict__ f3, const cplx_t<T>* __restrict__ in,
                             cplx_t<T>* __restrict__ out, int n_trans) {
  using CT = cplx_t<T>;
  const int64_t per = (int64_t)n1 * n2 * n3;
  const int nseg = (nf1 + kSeg - 1) / kSeg;
  const int64_t nitems = (int64_t)nf2 * nf3 * n_trans * nseg;
  const int k1max = (n1 - 1) / 2, k2max = (n2 - 1) / 2, k3max = (n3 - 1) / 2;
  const int k1min = -(n1 / 2), k2min = -(n2 / 2), k3min = -(n3 / 2);
  const int nw = blockDim.x >> 5, lane = threadIdx.x & 31;
  for (int64_t item = (int64_t)blockIdx.x * nw + (threadIdx.x >> 5); item < nitems; item += (int64_t)gridDim.x * nw) {
    const int64_t row = item / nseg;
    const int x0 = (int)(item - row * nseg) * kSeg;
    const int x1 = min(x0 + kSeg, nf1);
    const int64_t t = row / ((int64_t)nf2 * nf3);
    const int rr = (int)(row - t * nf2 * nf3);
    const int c2 = rr % nf2;
    const int c3 = rr / nf2;
    // mode of this row per axis, or none
    const int k2 = c2 <= k2max ? c2 : (c2 >= nf2 + k2min ? c2 - nf2 : INT32_MIN);
    const int k3 = c3 <= k3max ? c3 : (c3 >= nf3 + k3min ? c3 - nf3 : INT32_MIN);
    CT* dst = out + row * nf1;
    const bool has = k2 != INT32_MIN && k3 != INT32_MIN;
    const int p2 = has ? k2 - k2min : 0, p3 = has ? k3 - k3min : 0;
    T fac23 = (T)1;
    if (has && f2 != nullptr) fac23 = f3 != nullptr ? f3[p3] * f2[p2] : f2[p2];
    const CT* src = in + t * per + ((int64_t)p3 * n2 + p2) * n1;
    CT v[kSegPerLane];
    T f[kSegPerLane];
    bool m[kSegPerLane];  // the cell holds a kept mode
#pragma unroll
    for (int j = 0; j < kSegPerLane; ++j) {
      const int c1 = x0 + lane + 32 * j;
      const int k1 = c1 <= k1max ? c1 : (c1 >= nf1 + k1min ? c1 - nf1 : INT32_MIN);
      v[j].x = v[j].y = (T)0;
      f[j] = (T)0;
      m[j] = c1 < x1 && has && k1 != INT32_MIN;
      if (m[j]) {
        const int p1 = k1 - k1min;
        v[j] = src[p1];
        f[j] = f1[p1];
      }
    }
#pragma unroll
    for (int j = 0; j < kSegPerLane; ++j) {
      const int c1 = x0 + lane + 32 * j;
      if (c1 < x1) {
        CT o;
        o.x = (T)0;
        o.y = (T)0;
        if (m[j]) {
          const T fac = f2 != nullptr ? fac23 * f[j] : f[j];
          o.x = v[j].x * fac;
          o.y = v[j].y * fac;
        }
        dst[c1] = o;
      }
    }
  }
}

// Batched forms: one launch over many problems of different grids.  `items`
// is a device table sorted by `start` (first global element of each problem).
template <typename T>
struct DeconvItem {
  int nf[3];
  int nm[3];
  const T* fac[3];
  const void* src;
  void* dst;
  int64_t start;
};

template <typename T>
__device__ __forceinline__ int deconv_find(const DeconvItem<T>* __restrict__ items, int n, int64_t i) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (items[mid].start <= i)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Work unit of the batched passes: one row segment (kSeg elements along x)
// of one problem, a warp each; `start` counts units.
template <typename T>
__global__ void k_deconv_shuffle_batch(const DeconvItem<T>* __restrict__ items, int n, int64_t total) {
  using CT = cplx_t<T>;
  const int nw = blockDim.x >> 5, lane = threadIdx.x & 31;
  for (int64_t u = (int64_t)blockIdx.x * nw + (threadIdx.x >> 5); u < total; u += (int64_t)gridDim.x * nw) {
    const DeconvItem<T>& it = items[deconv_find(items, n, u)];
    const int n1 = it.nm[0], n2 = it.nm[1], n3 = it.nm[2];
    const int nseg = (n1 + kSeg - 1) / kSeg;
    const int64_t local = u - it.start;
    const int row = (int)(local / nseg);
    if (row >= n2 * n3) continue;  // a total past the table's units (never, with deconv_units)
    const int x0 = (int)(local - (int64_t)row * nseg) * kSeg;
    const int x1 = min(x0 + kSeg, n1);
    const int p2 = row % n2, p3 = row / n2;
    int i2 = p2 - n2 / 2, i3 = p3 - n3 / 2;
    if (i2 < 0) i2 += it.nf[1];
    if (i3 < 0) i3 += it.nf[2];
    T fac23 = (T)1;
    if (it.fac[1] != nullptr) fac23 = it.fac[2] != nullptr ? it.fac[2][p3] * it.fac[1][p2] : it.fac[1][p2];
    const CT* src = (const CT*)it.src + ((int64_t)i3 * it.nf[1] + i2) * it.nf[0];
    CT* dst = (CT*)it.dst + (int64_t)row * n1;
    CT v[kSegPerLane];
    T f[kSegPerLane];
#pragma unroll
    for (int j = 0; j < kSegPerLane; ++j) {
      const int p1 = x0 + lane + 32 * j;
      if (p1 < x1) {
        int i1 = p1 - n1 / 2;
        if (i1 < 0) i1 += it.nf[0];
        v[j] = src[i1];
        f[j] = it.fac[0][p1];
      }
    }
#pragma unroll
    for (int j = 0; j < kSegPerLane; ++j) {
      const int p1 = x0 + lane + 32 * j;
      if (p1 < x1) {
        const T fac = it.fac[1] != nullptr ? fac23 * f[j] : f[j];
        CT o;
        o.x = v[j].x * fac;
        o.y = v[j].y * fac;
        dst[p1] = o;
      }
    }
  }
}

template <typename T>
__global__ void k_deconv_pad_batch(const DeconvItem<T>* __restrict__ items, int n, int64_t total) {
  using CT = cplx_t<T>;
  const int nw = blockDim.x >> 5, lane = threadIdx.x & 31;
  for (int64_t u = (int64_t)blockIdx.x * nw + (threadIdx.x >> 5); u < total; u += (int64_t)gridDim.x * nw) {
    const DeconvItem<T>& it = items[deconv_find(items, n, u)];
    const int nf1 = it.nf[0], nf2 = it.nf[1], nf3 = it.nf[2];
    const int n1 = it.nm[0], n2 = it.nm[1], n3 = it.nm[2];
    const int nseg = (nf1 + kSeg - 1) / kSeg;
    const int64_t local = u - it.start;
    const int row = (int)(local / nseg);
    if (row >= nf2 * nf3) continue;  // a total past the table's units (never, with deconv_units)
    const int x0 = (int)(local - (int64_t)row * nseg) * kSeg;
    const int x1 = min(x0 + kSeg, nf1);
    const int c2 = row % nf2, c3 = row / nf2;
    const int k2 = c2 <= (n2 - 1) / 2 ? c2 : (c2 >= nf2 - n2 / 2 ? c2 - nf2 : INT32_MIN);
    const int k3 = c3 <= (n3 - 1) / 2 ? c3 : (c3 >= nf3 - n3 / 2 ? c3 - nf3 : INT32_MIN);
    const bool has = k2 != INT32_MIN && k3 != INT32_MIN;
    const int p2 = has ? k2 + n2 / 2 : 0, p3 = has ? k3 + n3 / 2 : 0;
    T fac23 = (T)1;
    if (has && it.fac[1] != nullptr) fac23 = it.fac[2] != nullptr ? it.fac[2][p3] * it.fac[1][p2] : it.fac[1][p2];
    const CT* src = (const CT*)it.src + ((int64_t)p3 * n2 + p2) * n1;
    CT* dst = (CT*)it.dst + (int64_t)row * nf1;
    CT v[kSegPerLane];
    T f[kSegPerLane];
    bool m[kSegPerLane];  // the cell holds a kept mode
#pragma unroll
    for (int j = 0; j < kSegPerLane; ++j) {
      const int c1 = x0 + lane + 32 * j;
      const int k1 = c1 <= (n1 - 1) / 2 ? c1 : (c1 >= nf1 - n1 / 2 ? c1 - nf1 : INT32_MIN);
      v[j].x = v[j].y = (T)0;
      f[j] = (T)0;
      m[j] = c1 < x1 && has && k1 != INT32_MIN;
      if (m[j]) {
        const int p1 = k1 + n1 / 2;
        v[j] = src[p1];
        f[j] = it.fac[0][p1];
      }
    }
#pragma unroll
    for (int j = 0; j < kSegPerLane; ++j) {
      const int c1 = x0 + lane + 32 * j;
      if (c1 < x1) {
        CT o;
        o.x = (T)0;
        o.y = (T)0;
        if (m[j]) {
          const T fac = it.fac[1] != nullptr ? fac23 * f[j] : f[j];
          o.x = v[j].x * fac;
          o.y = v[j].y * fac;
        }
        dst[c1] = o;
      }
    }
  }
}

// CTAs for a pass of one warp per row segment over nrows segments (8 warps a
// CTA), at most 8 CTAs per SM.
static int row_grid(int64_t nrows) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((nrows + 7) / 8, (int64_t)num_sms() * 8));
}

template <typename T>
cudaError_t launch_deconv_shuffle(int dim, const int nf[3], const int nm[3], const T* f1, const T* f2, const T* f3,
                                  const void* fw_hat, void* out, int n_trans, cudaStream_t st) {
  const int64_t total = (int64_t)nm[0] * nm[1] * nm[2] * n_trans;
  if (total == 0) return cudaSuccess;
  k_deconv_shuffle<T><<<row_grid((int64_t)nm[1] * nm[2] * n_trans * ((nm[0] + kSeg - 1) / kSeg)), 256, 0, st>>>(
      nf[0], nf[1], nf[2], nm[0], nm[1], nm[2], f1, dim >= 2 ? f2 : nullptr, dim >= 3 ? f3 : nullptr,
      (const cplx_t<T>*)fw_hat, (cplx_t<T>*)out, n_trans);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_deconv_pad(int dim, const int nf[3], const int nm[3], const T* f1, const T* f2, const T* f3,
                              const void* f_in, void* fw_hat, int n_trans, cudaStream_t st) {
  const int64_t total = (int64_t)nf[0] * nf[1] * nf[2] * n_trans;
  if (total == 0) return cudaSuccess;
  k_deconv_pad<T><<<row_grid((int64_t)nf[1] * nf[2] * n_trans * ((nf[0] + kSeg - 1) / kSeg)), 256, 0, st>>>(
      nf[0], nf[1], nf[2], nm[0], nm[1], nm[2], f1,
                                                           dim >= 2 ? f2 : nullptr, dim >= 3 ? f3 : nullptr,
                                                           (const cplx_t<T>*)f_in, (cplx_t<T>*)fw_hat, n_trans);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_deconv_batch(bool pad, const void* items, int n, int64_t total, cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  if (pad)
    k_deconv_pad_batch<T><<<row_grid(total), 256, 0, st>>>((const DeconvItem<T>*)items, n, total);
  else
    k_deconv_shuffle_batch<T><<<row_grid(total), 256, 0, st>>>((const DeconvItem<T>*)items, n, total);
  return cudaGetLastError();
}

size_t deconv_item_bytes(int precision) {
  return precision == 0 ? sizeof(DeconvItem<float>) : sizeof(DeconvItem<double>);
}

int64_t deconv_units(const int nf[3], const int nm[3], bool pad) {
  const int* e = pad ? nf : nm;  // the output's extent
  return (int64_t)e[1] * e[2] * ((e[0] + kSeg - 1) / kSeg);
}

int64_t fill_deconv_items(int precision, int dim, bool pad, const int* nf, const int* nm, const void* const* fac,
                          const void* const* src, void* const* dst, int n, void* host_items) {
  int64_t start = 0;
  for (int p = 0; p < n; ++p) {
    const int* f = nf + 3 * p;
    const int* m = nm + 3 * p;
    auto fill = [&](auto* it) {
      using R = std::remove_pointer_t<decltype(it->fac[0])>;
      for (int d = 0; d < 3; ++d) {
        it->nf[d] = d < dim ? f[d] : 1;
        it->nm[d] = d < dim ? m[d] : 1;
        it->fac[d] = d < dim ? (R)fac[3 * p + d] : nullptr;
      }
      it->src = src[p];
      it->dst = dst[p];
      it->start = start;  // in work units: row segments of kSeg elements
      start += deconv_units(it->nf, it->nm, pad);
    };
    if (precision == 0)
      fill((DeconvItem<float>*)host_items + p);
    else
      fill((DeconvItem<double>*)host_items + p);
  }
  return start;
}

template cudaError_t launch_deconv_batch<float>(bool, const void*, int, int64_t, cudaStream_t);
template cudaError_t launch_deconv_batch<double>(bool, const void*, int, int64_t, cudaStream_t);
template cudaError_t launch_deconv_shuffle<float>(int, const int*, const int*, const float*, const float*,
                                                  const float*, const void*, void*, int, cudaStream_t);
template cudaError_t launch_deconv_shuffle<double>(int, const int*, const int*, const double*, const double*,
                                                   const double*, const void*, void*, int, cudaStream_t);
template cudaError_t launch_deconv_pad<float>(int, const int*, const int*, const float*, const float*, const float*,
                                              const void*, void*, int, cudaStream_t);
template cudaError_t launch_deconv_pad<double>(int, const int*, const int*, const double*, const double*,
                                               const double*, const void*, void*, int, cudaStream_t);

}  // namespace nfx
