// Tile spreading, interpolation and ES-derivative gradient kernels.
//
// Work unit: a subproblem = up to `maxsub` consecutive sorted points of one bin.
// All of a bin's footprints lie in its padded tile (tile + ns - 1 cells per
// axis, periodic wrap applied only when the tile is read from / flushed to the
// fine grid), so each CTA works entirely in shared memory:
//
//  * spread (nufftax/core/spread.py:285-339, 435-494, 596-658; Pallas twin
//    nufftax/core/pallas_spread.py:337-613): points are staged 32 at a time per
//    warp (each lane folds one point and evaluates its d*ns ES weights once);
//    the warp then walks the 32 footprints one after another.  For 2D/3D
//    footprints of at least 32 cells each lane owns one footprint column and a
//    block of rows and sums consecutive same-cell points in registers
//    (spread_subproblem_runs); smaller footprints go cell by cell with
//    shared-memory atomics (spread_subproblem_cells).  Every shared-memory
//    atomic of one instruction hits a distinct address, so clustered points do
//    not serialise.  The finished tile is flushed with one vectorised
//    `red.global.add.v2.f32` per non-zero cell, coalesced along x.
//  * interp (nufftax/core/spread.py:342-381, 497-540, 661-709): the padded tile
//    is staged into shared memory with coalesced loads, then each thread
//    evaluates one point as a separable sum (x innermost); no atomics.
//  * grad (nufftax/core/spread.py:820-1305): the same staged tile, with the ES
//    derivative weights (dphi/dx = -phi'(z) nf / 2pi) for each axis, giving the
//    interpolated value and all coordinate gradients in one pass.
#pragma once


#include <type_traits>

#include "nfx_internal.h"

namespace nfx {

template <int NS, int DIM>
struct Pow {
  static constexpr int value = NS * Pow<NS, DIM - 1>::value;
};
template <int NS>
struct Pow<NS, 0> {
  static constexpr int value = 1;
};

template <typename T>
struct PointArgs {
  const T* sc[3];  // folded coordinates in sorted order (SortView::coord); unused axes nullptr
  int64_t M;
  int n_trans;
  int64_t grid_stride;  // complex elements per transform of the fine grid
  int tma;              // 1: the interpolation stages interior tiles with the kernel's tensor map
  int* status;          // device status word (nonzero after a bounded wait gave up); set when tma = 1
  Geom g;
  T beta, kc;
  SortView s;
  EsPoly poly;
};

// The NS weights of one axis: w[q] = phi(i0 + q - xs).  float with a fitted
// polynomial: Horner in v = 2 (xs - i0) - (NS - 1) (exact in float: xs - i0 is
// exact because xs and i0 are within NS of each other and i0 is an integer),
// degree kPolyEvalDeg, each coefficient a fixed offset in the argument block
// (an operand of its FMA, no load); otherwise exp/sqrt
// (nufftax/core/kernel.py:79-111).
template <typename T, int NS>
__device__ __forceinline__ void axis_weights(const PointArgs<T>& a, int i0, T xs, T* w) {
  if (std::is_same<T, float>::value && a.poly.deg > 0) {
    // weights q and NS - 1 - q from one even / odd split of polynomial q:
    // P(+-v) = E(v^2) +- v O(v^2)  (phi is even)
    static_assert(kPolyEvalDeg % 2 == 1, "odd evaluation degree: E and O of equal length");
    const float v = 2.0f * (float)(xs - (T)i0) - (float)(NS - 1);
    const float u = v * v;
    float e[NS / 2], o[NS / 2];
#pragma unroll
    for (int q = 0; q < NS / 2; ++q) {
      e[q] = a.poly.a[q][kPolyEvalDeg - 1];
      o[q] = a.poly.a[q][kPolyEvalDeg];
    }
#pragma unroll
    for (int d = kPolyEvalDeg - 3; d >= 0; d -= 2) {
#pragma unroll
      for (int q = 0; q < NS / 2; ++q) {
        e[q] = fmaf(e[q], u, a.poly.a[q][d]);
        o[q] = fmaf(o[q], u, a.poly.a[q][d + 1]);
      }
    }
#pragma unroll
    for (int q = 0; q < NS / 2; ++q) {
      w[q] = (T)fmaf(v, o[q], e[q]);
      w[NS - 1 - q] = (T)fmaf(-v, o[q], e[q]);
    }
  } else {
#pragma unroll
    for (int q = 0; q < NS; ++q) w[q] = es_weight(rn_sub((T)(i0 + q), xs), a.beta, a.kc);
  }
}

__device__ __forceinline__ void bin_origin(const Geom& g, int b, int& o0, int& o1, int& o2) {
  int bx = b % g.nb[0];
  int r = b / g.nb[0];
  int by = r % g.nb[1];
  int bz = r / g.nb[1];
  o0 = bx * g.tile[0];
  o1 = by * g.tile[1];
  o2 = bz * g.tile[2];
}

__device__ __forceinline__ int wrap_up(int i, int n) {
  while (i >= n) i -= n;
  return i;
}

// Folded coordinate of axis d of the k-th sorted point (a coalesced read).
template <typename T>
__device__ __forceinline__ T sorted_coord(const PointArgs<T>& a, int d, int k) {
  return a.sc[d][k];
}

template <typename T>
__device__ __forceinline__ cplx_t<T> cmul(cplx_t<T> u, cplx_t<T> v) {
  cplx_t<T> r;
  r.x = u.x * v.x - u.y * v.y;
  r.y = u.x * v.y + u.y * v.x;
  return r;
}

// Type-3 sorts carry a complex factor per sorted point (SortView::extra): the
// spread multiplies it into the strength, the interpolation into its result.
template <typename T>
__device__ __forceinline__ cplx_t<T> with_extra(const PointArgs<T>& a, int k, cplx_t<T> v) {
  return a.s.extra != nullptr ? cmul<T>(v, reinterpret_cast<const cplx_t<T>*>(a.s.extra)[k]) : v;
}

// ---------------------------------------------------------------------------
// Spread
// ---------------------------------------------------------------------------

// Adds a finished padded tile (planar) into the fine grid, one vectorised red
// per non-zero cell: one warp per tile row, lanes along x (coalesced); periodic
// wrap applied here.
template <typename T>
__device__ __forceinline__ void flush_tile(const Geom& g, const int o[3], const T* s_re, const T* s_im,
                                           cplx_t<T>* __restrict__ out) {
  const int row = g.pitch;
  const int plane = g.pitch * g.pad[1];
  const int nrows = g.pad[1] * g.pad[2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int r = warp; r < nrows; r += nw) {
    const int ly = r % g.pad[1];
    const int lz = r / g.pad[1];
    const int gy = wrap_up(o[1] + ly, g.nf[1]);
    const int gz = wrap_up(o[2] + lz, g.nf[2]);
    cplx_t<T>* dst = out + ((int64_t)gz * g.nf[1] + gy) * g.nf[0];
    const T* sr = s_re + lz * plane + ly * row;
    const T* si = s_im + lz * plane + ly * row;
    for (int lx = lane; lx < g.pad[0]; lx += 32) {
      const T vr = sr[lx], vi = si[lx];
      if (vr != (T)0 || vi != (T)0) {
        cplx_t<T> v;
        v.x = vr;
        v.y = vi;
        red_add(dst + wrap_up(o[0] + lx, g.nf[0]), v);
      }
    }
  }
}

// From a point's folded coordinates xf (in [0, nf]), computes its tile offset
// and per-axis weights.  Returns false for a point outside its bin's tile (the
// folded coordinates come from the same sort as the bins, so this does not
// happen; the check keeps a corrupted workspace from indexing out of the tile).
template <typename T, int DIM, int NS>
__device__ __forceinline__ bool footprint(const PointArgs<T>& a, const T (&xf)[DIM], const int o[3], int row,
                                          int plane, int& off, T (&w)[DIM][NS]) {
  const Geom& g = a.g;
  bool inside = true;
  off = 0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const T xs = xf[d];
    const int i0 = left_cell<T, NS>(xs);
    const int l = wrap_index(i0, g.nf[d]) - o[d];
    inside = inside && (unsigned)l < (unsigned)g.tile[d];
    off += l * (d == 0 ? 1 : (d == 1 ? row : plane));
    axis_weights<T, NS>(a, i0, xs, w[d]);
  }
  return inside;
}

template <typename T, int DIM>
__device__ __forceinline__ void load_sorted(const PointArgs<T>& a, int k, T (&xf)[DIM]) {
#pragma unroll
  for (int d = 0; d < DIM; ++d) xf[d] = sorted_coord(a, d, k);
}

template <typename T, int DIM, int NS>
__device__ __forceinline__ bool point_footprint(const PointArgs<T>& a, int k, const int o[3], int row, int plane,
                                                int& off, T (&w)[DIM][NS]) {
  T xf[DIM];
  load_sorted<T, DIM>(a, k, xf);
  return footprint<T, DIM, NS>(a, xf, o, row, plane, off, w);
}

// Slot helpers of the run-merging spread: 16-byte chunks of four floats or two
// doubles (slots are 16-byte aligned, see run_slot_reals).
__device__ __forceinline__ void store16(float* p, float a, float b, float c, float d) {
  *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
}
__device__ __forceinline__ void store16(double* p, double a, double b) {
  *reinterpret_cast<double2*>(p) = make_double2(a, b);
}

// Writes one point's slot: c * w_x, then the y weights and (3D) the z
// weights; padding entries are zero.
template <typename T, int DIM, int NS>
__device__ __forceinline__ void stage_slot(T* sp, cplx_t<T> cv, const T (&w)[DIM][NS]) {
  constexpr int WY = run_wy(DIM, NS);
  constexpr int WZ = run_wz(DIM, NS);
  constexpr int YOFF = round4(2 * NS);
  constexpr int ZOFF = YOFF + WY;
  static_assert(NS % 2 == 0, "even widths only");
  if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int q = 0; q < NS; q += 2)
      store16(sp + 2 * q, cv.x * w[0][q], cv.y * w[0][q], cv.x * w[0][q + 1], cv.y * w[0][q + 1]);
#pragma unroll
    for (int q = 0; q < WY; q += 4)
      store16(sp + YOFF + q, q < NS ? w[1][q] : (T)0, q + 1 < NS ? w[1][q + 1] : (T)0,
              q + 2 < NS ? w[1][q + 2] : (T)0, q + 3 < NS ? w[1][q + 3] : (T)0);
    if constexpr (DIM == 3) {
#pragma unroll
      for (int q = 0; q < WZ; q += 4)
        store16(sp + ZOFF + q, q < NS ? w[DIM - 1][q] : (T)0, q + 1 < NS ? w[DIM - 1][q + 1] : (T)0,
                q + 2 < NS ? w[DIM - 1][q + 2] : (T)0, q + 3 < NS ? w[DIM - 1][q + 3] : (T)0);
    }
  } else {
#pragma unroll
    for (int q = 0; q < NS; ++q) store16(sp + 2 * q, cv.x * w[0][q], cv.y * w[0][q]);
#pragma unroll
    for (int q = 0; q < WY; q += 2)
      store16(sp + YOFF + q, q < NS ? w[1][q] : (T)0, q + 1 < NS ? w[1][q + 1] : (T)0);
    if constexpr (DIM == 3) {
#pragma unroll
      for (int q = 0; q < WZ; q += 2)
        store16(sp + ZOFF + q, q < NS ? w[DIM - 1][q] : (T)0, q + 1 < NS ? w[DIM - 1][q + 1] : (T)0);
    }
  }
}

// Adds one staged point to this lane's accumulators: acc[r] += w_row(r) * (c w_x),
// w_row the y weight of row grp * rpl + r (2D) or z weight * y weight (3D).
template <typename T, int DIM, int NS>
__device__ __forceinline__ void add_slot(const T* sp, int kx, int grp, cplx_t<T> (&acc)[run_rows_per_lane(DIM, NS)]) {
  using CT = cplx_t<T>;
  constexpr int RPL = run_rows_per_lane(DIM, NS);
  constexpr int WY = run_wy(DIM, NS);
  constexpr int YOFF = round4(2 * NS);
  constexpr int ZOFF = YOFF + WY;
  const CT cw = reinterpret_cast<const CT*>(sp)[kx];
  if constexpr (DIM == 2) {
    const T* wy = sp + YOFF + grp * RPL;
#pragma unroll
    for (int r = 0; r < RPL; ++r) acc[r] = fma_rc(wy[r], cw, acc[r]);
  } else if constexpr (RPL % NS == 0) {
    const T* wz = sp + ZOFF + grp * (RPL / NS);
#pragma unroll
    for (int zz = 0; zz < RPL / NS; ++zz) {
      const T z = wz[zz];
#pragma unroll
      for (int q = 0; q < NS; ++q) acc[zz * NS + q] = fma_rc(z * sp[YOFF + q], cw, acc[zz * NS + q]);
    }
  } else {
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int rho = grp * RPL + r;
      acc[r] = fma_rc(sp[ZOFF + rho / NS] * sp[YOFF + rho % NS], cw, acc[r]);
    }
  }
}

// Adds one staged point straight to the shared tile at footprint origin `off`.
// lane_cell: tile offset of this lane's first cell (row grp * rpl, column kx)
// from the origin, -1 when the lane owns no cell; rows r after the first are
// r rows further (2D), or r / ns planes and r % ns rows further (3D with rpl a
// multiple of ns: compile-time in r).
template <typename T, int DIM, int NS>
__device__ __forceinline__ void add_slot_direct(const T* sp, int kx, int grp, int off, T* s_re, T* s_im,
                                                int lane_cell, int row, int plane) {
  using CT = cplx_t<T>;
  constexpr int RPL = run_rows_per_lane(DIM, NS);
  constexpr int NR = run_rows(DIM, NS);
  constexpr int WY = run_wy(DIM, NS);
  constexpr int YOFF = round4(2 * NS);
  constexpr int ZOFF = YOFF + WY;
  if (lane_cell < 0) return;
  const CT cw = reinterpret_cast<const CT*>(sp)[kx];
  T* pr = s_re + off + lane_cell;
  T* pi = s_im + off + lane_cell;
  auto add = [&](int o, T w) {
    atomicAdd(pr + o, w * cw.x);
    atomicAdd(pi + o, w * cw.y);
  };
  if constexpr (DIM == 2) {
    const T* wy = sp + YOFF + grp * RPL;
#pragma unroll
    for (int r = 0; r < RPL; ++r)
      if (grp * RPL + r < NR) add(r * row, wy[r]);
  } else if constexpr (RPL % NS == 0) {
    const T* wz = sp + ZOFF + grp * (RPL / NS);
    T wy[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) wy[q] = sp[YOFF + q];
#pragma unroll
    for (int zz = 0; zz < RPL / NS; ++zz) {
      const T z = wz[zz];
#pragma unroll
      for (int q = 0; q < NS; ++q) add(zz * plane + q * row, z * wy[q]);
    }
  } else {
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int rho = grp * RPL + r;
      if (rho < NR) {
        const int rz = rho / NS, ry = rho - rz * NS;
        add((rz - (grp * RPL) / NS) * plane + (ry - (grp * RPL) % NS) * row, sp[ZOFF + rz] * sp[YOFF + ry]);
      }
    }
  }
}

// 3D batches of 32 points with at least this many run starts (mean run of 4
// or less) skip the register accumulation and add each point directly: a
// lane's rpl = 16 rows make a run's walk and flush cost more than the direct
// adds of a few points.  2D batches always take the walk: a float atomicAdd on
// shared memory is a compare-and-swap loop (no native float add), so a run's
// flush of rpl = 2 complex cells per lane costs about as much as adding one
// point's cells directly, and the walk measured faster than the direct path
// for batches of mean run 1 to 4 (2D ns = 8: 4M clustered points 167 -> 158
// us, 0.5M radial points unchanged).
constexpr int kSparseRuns = 8;
template <int DIM>
__device__ __forceinline__ bool direct_batch(unsigned starts) {
  return DIM == 3 && __popc(starts) >= kSparseRuns;
}

// Run-merging spread (2D/3D, footprints of at least 32 cells).  Each warp walks
// a contiguous, cell-ordered slice of the subproblem 32 points at a time: every
// lane stages one point in a shared slot (stage_slot), then the warp takes the
// 32 points one after another with lane l accumulating, in registers,
// footprint column kx = l % ns of rows grp*rpl .. grp*rpl + rpl - 1
// (grp = l / ns; add_slot).  Consecutive points in the same cell share the
// footprint, so the registers reach shared memory (atomics, distinct addresses
// within an instruction) only when the cell changes.  One ballot per batch
// marks where runs start; the walk goes run by run, each run an unrolled loop
// with no branch per point.  The next batch's point indices, coordinates and
// strengths are fetched while the current batch is walked.
template <typename T, int DIM, int NS, int NW>
__device__ __forceinline__ void spread_subproblem_runs(const PointArgs<T>& a, const cplx_t<T>* __restrict__ c,
                                                       cplx_t<T>* __restrict__ fw, int sidx, unsigned char* smem_raw) {
  using CT = cplx_t<T>;
  constexpr int G = run_groups(NS);
  constexpr int RPL = run_rows_per_lane(DIM, NS);
  constexpr int NR = run_rows(DIM, NS);
  constexpr int SLOT = run_slot_reals(DIM, NS, (int)sizeof(T));
  static_assert(SLOT > 0, "run-merging layout does not apply");
  const Geom& g = a.g;
  const int tile_cells = g.pad[2] * g.pad[1] * g.pitch;
  T* s_re = reinterpret_cast<T*>(smem_raw);
  T* s_im = s_re + tile_cells;
  // slots start 16-byte aligned after the two tile planes
  T* s_st = reinterpret_cast<T*>(smem_raw + ((2 * (size_t)tile_cells * sizeof(T) + 15) & ~(size_t)15));
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int row = g.pitch;
  const int plane = g.pitch * g.pad[1];
  // this lane's column and row group; lanes past the groups mirror the last
  // group's loads and never flush
  const int kx = lane % NS;
  const bool lane_on = lane / NS < G;
  const int grp = lane_on ? lane / NS : G - 1;
  T* my_slot = s_st + (warp * 32 + lane) * SLOT;
  const T* warp_slots = s_st + warp * 32 * SLOT;

  const int b = a.s.sub_bin[sidx];
  const int k0 = a.s.sub_start[sidx];
  const int k1 = min(k0 + a.s.maxsub, a.s.bin_start[b + 1]);
  int o[3];
  bin_origin(g, b, o[0], o[1], o[2]);
  for (int t = 0; t < a.n_trans; ++t) {
    const CT* ct = c + (int64_t)t * a.M;
    for (int i = threadIdx.x; i < 2 * tile_cells; i += blockDim.x) s_re[i] = (T)0;
    __syncthreads();
    const int per = ((k1 - k0 + NW - 1) / NW + 31) / 32 * 32;
    const int w0 = min(k0 + warp * per, k1);
    const int w1 = min(w0 + per, k1);
    // two accumulator sets (alternate points of a run) halve the FMA
    // dependency chains; flush_run adds them
    CT acc[RPL], acc2[RPL];
#pragma unroll
    for (int r = 0; r < RPL; ++r) acc[r].x = acc[r].y = acc2[r].x = acc2[r].y = (T)0;
    int run_off = -1;
    // this lane's first cell (row grp * rpl, column kx) relative to a
    // footprint's origin; -1 for lanes past the groups
    const int rho0 = grp * RPL;
    const int lane_cell = lane_on ? (DIM == 3 ? (rho0 / NS) * plane + (rho0 % NS) * row : rho0 * row) + kx : -1;
    auto flush_run = [&]() {
#pragma unroll
      for (int r = 0; r < RPL; ++r) {
        acc[r].x += acc2[r].x;
        acc[r].y += acc2[r].y;
      }
      if (lane_cell >= 0) {
        T* pr = s_re + run_off + lane_cell;
        T* pi = s_im + run_off + lane_cell;
#pragma unroll
        for (int r = 0; r < RPL; ++r) {
          const int rho = rho0 + r;
          if (rho < NR) {
            // offset of row r from this lane's first row
            int o;
            if constexpr (DIM == 2) {
              o = r * row;
            } else if constexpr (RPL % NS == 0) {
              o = (r / NS) * plane + (r % NS) * row;
            } else {
              o = (rho / NS - rho0 / NS) * plane + (rho % NS - rho0 % NS) * row;
            }
            atomicAdd(pr + o, acc[r].x);
            atomicAdd(pi + o, acc[r].y);
          }
        }
      }
#pragma unroll
      for (int r = 0; r < RPL; ++r) acc[r].x = acc[r].y = acc2[r].x = acc2[r].y = (T)0;
    };
    // software pipeline: folded coordinates and strength of this lane's point
    // in the current batch (xn, cn) and the point index of the next batch (pn)
    T xn[DIM];
    CT cn;
    cn.x = cn.y = (T)0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) xn[d] = (T)0;
    int pn = w0 + lane < w1 ? a.s.perm[w0 + lane] : -1;
    if (pn >= 0) {
      load_sorted<T, DIM>(a, w0 + lane, xn);
      cn = ct[pn];
    }
    pn = w0 + 32 + lane < w1 ? a.s.perm[w0 + 32 + lane] : -1;
    for (int kb = w0; kb < w1; kb += 32) {
      const bool valid = kb + lane < w1;
      T xv[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) xv[d] = xn[d];
      CT cv = cn;
      if (pn >= 0) {  // next batch (pn >= 0 exactly when kb + 32 + lane < w1)
        load_sorted<T, DIM>(a, kb + 32 + lane, xn);
        cn = ct[pn];
      }
      pn = kb + 64 + lane < w1 ? a.s.perm[kb + 64 + lane] : -1;
      int off = 0;
      if (valid) {
        T w[DIM][NS];
        const bool inside = footprint<T, DIM, NS>(a, xv, o, row, plane, off, w);
        cv = with_extra(a, kb + lane, cv);
        if (!inside) {
          cv.x = cv.y = (T)0;
          off = 0;
        }
        stage_slot<T, DIM, NS>(my_slot, cv, w);
      }
      // lane j starts a run when its cell differs from point j-1's
      int prev = __shfl_up_sync(0xffffffffu, off, 1);
      if (lane == 0) prev = run_off;
      const unsigned starts = __ballot_sync(0xffffffffu, valid && off != prev);
      __syncwarp();
      const int cnt = min(32, w1 - kb);
      int j = 0;
      const T* sp = warp_slots;
      if (direct_batch<DIM>(starts)) {
        // short runs: points before the first run start finish the pending
        // run; every later point is added to shared memory directly
        const int first = __ffs(starts) - 1;
        for (; j < first; ++j, sp += SLOT) add_slot<T, DIM, NS>(sp, kx, grp, acc);
        if (run_off >= 0) flush_run();
        for (; j < cnt; ++j, sp += SLOT)
          add_slot_direct<T, DIM, NS>(sp, kx, grp, __shfl_sync(0xffffffffu, off, j), s_re, s_im, lane_cell, row,
                                      plane);
        run_off = __shfl_sync(0xffffffffu, off, cnt - 1);  // accumulators are empty
        j = cnt;
      }
      while (j < cnt) {  // one run (or the rest of one) per trip
        if ((starts >> j) & 1u) {
          if (run_off >= 0) flush_run();
          run_off = __shfl_sync(0xffffffffu, off, j);
        }
        const unsigned later = j < 31 ? starts >> (j + 1) : 0u;
        const int je = later != 0u ? min(j + __ffs(later), cnt) : cnt;
        for (; j + 4 <= je; j += 4, sp += 4 * SLOT) {
          add_slot<T, DIM, NS>(sp, kx, grp, acc);
          add_slot<T, DIM, NS>(sp + SLOT, kx, grp, acc2);
          add_slot<T, DIM, NS>(sp + 2 * SLOT, kx, grp, acc);
          add_slot<T, DIM, NS>(sp + 3 * SLOT, kx, grp, acc2);
        }
        for (; j < je; ++j, sp += SLOT) add_slot<T, DIM, NS>(sp, kx, grp, acc);
      }
      __syncwarp();
    }
    if (run_off >= 0) flush_run();
    __syncthreads();
    flush_tile<T>(g, o, s_re, s_im, fw + (int64_t)t * a.grid_stride);
    __syncthreads();
  }
}

// Spread of one subproblem, footprints below 32 cells (1D, small ns) or with
// more than 16 rows a lane (3D, ns >= 9).  Points are staged 32 at a time per
// warp (weights axis-major), then walked footprint cell by footprint cell with
// shared-memory atomics on distinct addresses within each instruction.
template <typename T, int DIM, int NS, int NW>
__device__ __forceinline__ void spread_subproblem_cells(const PointArgs<T>& a, const cplx_t<T>* __restrict__ c,
                                                        cplx_t<T>* __restrict__ fw, int sidx, unsigned char* smem_raw) {
  using CT = cplx_t<T>;
  constexpr int CELLS = Pow<NS, DIM>::value;
  constexpr int SW = NW * 32 + 1;  // staging stride: odd, so both the per-lane writes and
                                   // the per-point reads across q hit distinct banks
  const Geom& g = a.g;
  const int tile_cells = g.pad[2] * g.pad[1] * g.pitch;
  T* s_re = reinterpret_cast<T*>(smem_raw);
  T* s_im = s_re + tile_cells;
  T* s_w = s_im + tile_cells;          // [DIM*NS][SW]
  T* s_cr = s_w + DIM * NS * SW;       // [NW*32]
  T* s_ci = s_cr + NW * 32;            // [NW*32]
  int* s_off = reinterpret_cast<int*>(s_ci + NW * 32);  // [NW*32]
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int row = g.pitch;
  const int plane = g.pitch * g.pad[1];
  const int b = a.s.sub_bin[sidx];
  const int k0 = a.s.sub_start[sidx];
  const int k1 = min(k0 + a.s.maxsub, a.s.bin_start[b + 1]);
  int o[3];
  bin_origin(g, b, o[0], o[1], o[2]);
  for (int t = 0; t < a.n_trans; ++t) {
    for (int i = threadIdx.x; i < 2 * tile_cells; i += blockDim.x) s_re[i] = (T)0;
    __syncthreads();
    const int per = ((k1 - k0 + NW - 1) / NW + 31) / 32 * 32;
    const int w0 = min(k0 + warp * per, k1);
    const int w1 = min(w0 + per, k1);
    for (int kb = w0; kb < w1; kb += 32) {
      const int k = kb + lane;
      const int slot = warp * 32 + lane;
      if (k < w1) {
        const int p = a.s.perm[k];
        int off;
        T w[DIM][NS];
        const bool inside = point_footprint<T, DIM, NS>(a, k, o, row, plane, off, w);
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
          for (int q = 0; q < NS; ++q) s_w[(d * NS + q) * SW + slot] = w[d][q];
        const CT cv = with_extra(a, k, c[(int64_t)t * a.M + p]);
        s_off[slot] = inside ? off : 0;
        s_cr[slot] = inside ? cv.x : (T)0;
        s_ci[slot] = inside ? cv.y : (T)0;
      }
      __syncwarp();
      const int cnt = min(32, w1 - kb);
      if constexpr (CELLS >= 32) {
        // large footprints: one point at a time, straight to shared memory
        constexpr int R = (CELLS + 31) / 32;
        for (int j = 0; j < cnt; ++j) {
          const int sj = warp * 32 + j;
          const T cr = s_cr[sj], ci = s_ci[sj];
          const int off = s_off[sj];
#pragma unroll 4
          for (int r = 0; r < R; ++r) {
            const int q = lane + 32 * r;
            if (CELLS % 32 == 0 || q < CELLS) {
              const int kx = q % NS;
              const int ky = (q / NS) % NS;
              const int kz = q / (NS * NS);
              T w;
              if (DIM == 1)
                w = s_w[kx * SW + sj];
              else if (DIM == 2)
                w = s_w[(NS + ky) * SW + sj] * s_w[kx * SW + sj];
              else
                w = (s_w[(2 * NS + kz) * SW + sj] * s_w[(NS + ky) * SW + sj]) * s_w[kx * SW + sj];
              const int addr = off + kz * plane + ky * row + kx;
              atomicAdd(&s_re[addr], cr * w);
              atomicAdd(&s_im[addr], ci * w);
            }
          }
        }
      } else {
        // small footprints: several points per instruction
        const int items = cnt * CELLS;
        for (int it = lane; it < items; it += 32) {
          const int j = it / CELLS;
          const int q = it - j * CELLS;
          const int kx = q % NS;
          const int ky = (q / NS) % NS;
          const int kz = q / (NS * NS);
          const int sj = warp * 32 + j;
          T w;
          if (DIM == 1)
            w = s_w[kx * SW + sj];
          else if (DIM == 2)
            w = s_w[(NS + ky) * SW + sj] * s_w[kx * SW + sj];
          else
            w = (s_w[(2 * NS + kz) * SW + sj] * s_w[(NS + ky) * SW + sj]) * s_w[kx * SW + sj];
          const int addr = s_off[sj] + kz * plane + ky * row + kx;
          atomicAdd(&s_re[addr], s_cr[sj] * w);
          atomicAdd(&s_im[addr], s_ci[sj] * w);
        }
      }
      __syncwarp();
    }
    __syncthreads();
    flush_tile<T>(g, o, s_re, s_im, fw + (int64_t)t * a.grid_stride);
    __syncthreads();
  }
}

template <typename T, int DIM, int NS, int NW>
__device__ __forceinline__ void spread_subproblem(const PointArgs<T>& a, const cplx_t<T>* __restrict__ c,
                                                  cplx_t<T>* __restrict__ fw, int sidx, unsigned char* smem_raw) {
  if constexpr (run_slot_reals(DIM, NS, (int)sizeof(T)) > 0)
    spread_subproblem_runs<T, DIM, NS, NW>(a, c, fw, sidx, smem_raw);
  else
    spread_subproblem_cells<T, DIM, NS, NW>(a, c, fw, sidx, smem_raw);
}

template <typename T, int DIM, int NS, int NW>
__global__ void __launch_bounds__(NW * 32) k_spread(PointArgs<T> a, const cplx_t<T>* __restrict__ c,
                                                    cplx_t<T>* __restrict__ fw) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int nsub = *a.s.nsub;
  for (int sidx = blockIdx.x; sidx < nsub; sidx += gridDim.x) spread_subproblem<T, DIM, NS, NW>(a, c, fw, sidx, smem_raw);
}

// Plane-owner spread (3D, points sparser than cells).  The CTA stages up to
// NW*32 points at a time (every thread folds one point: c * w_x, y and z
// weights, its tile origin); then warp w adds every staged point into the
// tile planes z with z % NW == w, each plane's ns x ns cells spread over the
// lanes, with plain shared-memory read-add-write: a plane belongs to one warp,
// whose lanes touch distinct cells in each instruction, so no atomics are
// needed and every cell sums its points in sorted order.  With NW = ns every
// footprint (ns consecutive planes) gives each warp exactly one plane.  Slots
// are 16-byte aligned (owner_slot_reals): staged with 16-byte stores, read with
// 8-byte loads of (c w_x re, im), (offset, z) and pairs of y weights.
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using type = float4;
};
template <>
struct Vec16<double> {
  using type = double2;
};

// The tile of the plane-owner spread holds interleaved complex cells (one
// 8- or 16-byte load and store per cell update).  Flushed like flush_tile.
template <typename T>
__device__ __forceinline__ void flush_tile_c(const Geom& g, const int o[3], const cplx_t<T>* s_tile,
                                             cplx_t<T>* __restrict__ out) {
  const int row = g.pitch;
  const int plane = g.pitch * g.pad[1];
  const int nrows = g.pad[1] * g.pad[2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int r = warp; r < nrows; r += nw) {
    const int ly = r % g.pad[1];
    const int lz = r / g.pad[1];
    const int gy = wrap_up(o[1] + ly, g.nf[1]);
    const int gz = wrap_up(o[2] + lz, g.nf[2]);
    cplx_t<T>* dst = out + ((int64_t)gz * g.nf[1] + gy) * g.nf[0];
    const cplx_t<T>* src = s_tile + lz * plane + ly * row;
    for (int lx = lane; lx < g.pad[0]; lx += 32) {
      const cplx_t<T> v = src[lx];
      if (v.x != (T)0 || v.y != (T)0) red_add(dst + wrap_up(o[0] + lx, g.nf[0]), v);
    }
  }
}

// A non-negative int carried in a real's bits (read back as the low int of the
// real's bytes).
template <typename T>
__device__ __forceinline__ T int_bits(int v) {
  if constexpr (sizeof(T) == 4)
    return __int_as_float(v);
  else
    return __longlong_as_double((long long)v);
}

// Row pitch (cells) of the plane-owner tile: at ns = 8 (complex64) lanes
// 0-15 of an update touch two rows 1 apart, so a pitch of 8 mod 16 cells puts
// their 64-byte segments in opposite halves of the banks; at ns = 4 the four
// rows of a half-warp need a pitch of 4 mod 8.  Other widths and complex128
// keep the tile's own pitch.
__host__ __device__ inline int owner_pitch(int pitch, int pad0, int ns, int real_bytes) {
  if (real_bytes != 4) return pitch;
  if (ns == 8) return pad0 + ((8 - pad0 % 16) + 16) % 16;
  if (ns == 4) return pad0 + ((4 - pad0 % 8) + 8) % 8;
  return pitch;
}

template <typename T, int NS, int NW>
__device__ __forceinline__ void spread_subproblem_owner(const PointArgs<T>& a, const cplx_t<T>* __restrict__ c,
                                                        cplx_t<T>* __restrict__ fw, int sidx,
                                                        unsigned char* smem_raw) {
  using CT = cplx_t<T>;
  using V16 = typename Vec16<T>::type;
  constexpr int R = 16 / (int)sizeof(T);  // reals per 16-byte vector
  static_assert((2 * NS) % R == 0, "c * w_x pairs fill whole vectors");
  constexpr int SLOT = owner_slot_reals((int)sizeof(T), NS);
  constexpr int YO = 2 * NS;                 // y weights
  constexpr int ZO = YO + owner_pad(NS, R);  // z weights
  constexpr int OO = ZO + owner_pad(NS, R);  // origin (offset, z) as raw int bits
  constexpr int NT = NW * 32;
  // cells of one footprint plane handled by this lane: column kx = lane % NS
  // and rows ky0 + i * LPR (i < IT): at NS = 8 one update touches rows
  // 0-3 (lanes 0-31), the next rows 4-7
  constexpr int LPR = 32 / NS;             // row blocks (lanes per column)
  constexpr int IT = (NS + LPR - 1) / LPR;  // rows per lane per plane
  // y weights in pair order (w_y[ky0], w_y[ky0 + LPR]) when a lane's two rows
  // are LPR apart and cover the NS rows exactly (NS = 8): one 8-byte load
  constexpr bool PAIRS = IT == 2 && 2 * LPR == NS;
  const Geom& g = a.g;
  const int tile_cells = g.pad[2] * g.pad[1] * g.pitch;
  CT* s_tile = reinterpret_cast<CT*>(smem_raw);
  T* s_st = reinterpret_cast<T*>(smem_raw) + owner_pad(2 * tile_cells, R);  // [NT][SLOT], 16-byte aligned
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int row = g.pitch;
  const int plane = g.pitch * g.pad[1];
  const int b = a.s.sub_bin[sidx];
  const int k0 = a.s.sub_start[sidx];
  const int k1 = min(k0 + a.s.maxsub, a.s.bin_start[b + 1]);
  int o[3];
  bin_origin(g, b, o[0], o[1], o[2]);
  const int kx = lane % NS;
  const int ky0 = lane / NS;
  const bool lane_on = ky0 < LPR;
  for (int t = 0; t < a.n_trans; ++t) {
    for (int i = threadIdx.x; i < tile_cells; i += blockDim.x) s_tile[i] = CT{(T)0, (T)0};
    for (int kb = k0; kb < k1; kb += NT) {
      const int k = kb + threadIdx.x;
      if (k < k1) {
        const int p = a.s.perm[k];
        T xv[3];
        load_sorted<T, 3>(a, k, xv);
        int off;
        T w[3][NS];
        const bool inside = footprint<T, 3, NS>(a, xv, o, row, plane, off, w);
        CT cv = with_extra(a, k, c[(int64_t)t * a.M + p]);
        if (!inside) {
          cv.x = cv.y = (T)0;
          off = 0;
        }
        T v[SLOT];
#pragma unroll
        for (int i = 0; i < SLOT; ++i) v[i] = (T)0;
#pragma unroll
        for (int q = 0; q < NS; ++q) {
          v[2 * q] = cv.x * w[0][q];
          v[2 * q + 1] = cv.y * w[0][q];
          v[ZO + q] = w[2][q];
        }
#pragma unroll
        for (int q = 0; q < NS; ++q) {
          if constexpr (PAIRS)
            v[YO + 2 * (q % LPR) + q / LPR] = w[1][q];
          else
            v[YO + q] = w[1][q];
        }
        v[OO] = int_bits<T>(off);
        v[OO + 1] = int_bits<T>(off / plane);  // z of the footprint origin in the tile
        V16* sp = reinterpret_cast<V16*>(s_st + threadIdx.x * SLOT);
#pragma unroll
        for (int i = 0; i < SLOT / R; ++i) {
          V16 u;
          if constexpr (R == 4) {
            u.x = v[4 * i];
            u.y = v[4 * i + 1];
            u.z = v[4 * i + 2];
            u.w = v[4 * i + 3];
          } else {
            u.x = v[2 * i];
            u.y = v[2 * i + 1];
          }
          sp[i] = u;
        }
      }
      __syncthreads();  // also orders the tile zeroing before the first adds
      const int cnt = min(NT, k1 - kb);
      static_assert((NW & (NW - 1)) == 0, "warps per CTA a power of two");
      // planes of each footprint this warp owns: dz0 + pl * NW < NS, at most
      // ceil(NS / NW) (exactly NS / NW when NW divides NS)
      constexpr int PLANES = (NS + NW - 1) / NW;
      for (int j = 0; j < cnt; ++j) {
        const T* sp = s_st + j * SLOT;
        int off, oz;
        if constexpr (sizeof(T) == 4) {
          const int2 so = *reinterpret_cast<const int2*>(sp + OO);  // 8-byte aligned: OO is a multiple of 4
          off = so.x;
          oz = so.y;
        } else {
          const int* so = reinterpret_cast<const int*>(sp + OO);
          off = so[0];
          oz = so[2];
        }
        const int dz0 = (warp - oz) & (NW - 1);
#pragma unroll
        for (int pl = 0; pl < PLANES; ++pl) {
          const int dz = dz0 + pl * NW;
          if (NS % NW != 0 && dz >= NS) break;
          const T wz = sp[ZO + dz];
          const int base = off + dz * plane + kx;
          const CT cx = *reinterpret_cast<const CT*>(sp + 2 * kx);  // c * w_x[kx]
          if (lane_on) {
            T wyr[IT];
            if constexpr (PAIRS) {
              const CT pr = *reinterpret_cast<const CT*>(sp + YO + 2 * ky0);
              wyr[0] = pr.x;
              wyr[1] = pr.y;
            } else {
#pragma unroll
              for (int i = 0; i < IT; ++i) wyr[i] = ky0 + i * LPR < NS ? sp[YO + ky0 + i * LPR] : (T)0;
            }
#pragma unroll
            for (int i = 0; i < IT; ++i) {
              const int ky = ky0 + i * LPR;
              if (ky < NS) {
                const T wy = wz * wyr[i];
                CT* cell = s_tile + base + ky * row;
                CT u = *cell;
                u.x += wy * cx.x;
                u.y += wy * cx.y;
                *cell = u;
              }
            }
          }
        }
      }
      __syncthreads();
    }
    flush_tile_c<T>(g, o, s_tile, fw + (int64_t)t * a.grid_stride);
    __syncthreads();
  }
}

template <typename T, int NS, int NW>
__global__ void __launch_bounds__(NW * 32) k_spread_owner(PointArgs<T> a, const cplx_t<T>* __restrict__ c,
                                                          cplx_t<T>* __restrict__ fw) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int nsub = *a.s.nsub;
  for (int sidx = blockIdx.x; sidx < nsub; sidx += gridDim.x)
    spread_subproblem_owner<T, NS, NW>(a, c, fw, sidx, smem_raw);
}

// ---------------------------------------------------------------------------
// Stage a padded tile of one transform's grid into shared memory (interleaved).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void stage_tile(const Geom& g, const int o[3], const cplx_t<T>* __restrict__ grid,
                                           cplx_t<T>* s_tile) {
  const int row = g.pitch;
  const int plane = g.pitch * g.pad[1];
  const int nrows = g.pad[1] * g.pad[2];
  // one warp per row, lanes along x: coalesced
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int r = warp; r < nrows; r += nw) {
    const int ly = r % g.pad[1];
    const int lz = r / g.pad[1];
    const int gy = wrap_up(o[1] + ly, g.nf[1]);
    const int gz = wrap_up(o[2] + lz, g.nf[2]);
    const cplx_t<T>* src = grid + ((int64_t)gz * g.nf[1] + gy) * g.nf[0];
    cplx_t<T>* dst = s_tile + lz * plane + ly * row;
    for (int lx = lane; lx < g.pad[0]; lx += 32) dst[lx] = src[wrap_up(o[0] + lx, g.nf[0])];
  }
}

// ---------------------------------------------------------------------------
// Tile staging by TMA.  The interpolation's padded tile of a bin whose padded
// extent lies inside the grid on every axis (no periodic wrap) is one box of
// the fine grid: one thread issues a cp.async.bulk.tensor load of it from the
// kernel's tensor map (this GPU's own grid, no multicast) into the tile
// buffer, completing on an mbarrier; the others wait on the barrier.  Tiles
// that wrap keep the plain loads (stage_tile).  Box (pitch, pad_y[, pad_z], 1)
// of elements of 8 bytes (complex64; complex128 as two), coordinates
// (x, y[, z], transform), so the box lands with the tile's own row pitch.
// The barrier wait is bounded (kTmaWaitPolls polls and kTmaWaitNs of the
// global timer, whichever ends first): a wait that gives up records
// NFX_STATUS_TMA_TIMEOUT in the status word (nfx_device_status) and the CTA
// stops, so a copy that never lands cannot hang the GPU.
// ---------------------------------------------------------------------------
constexpr int kTmaWaitPolls = 1 << 24;
constexpr unsigned long long kTmaWaitNs = 500000000ull;  // 0.5 s

struct TmaStage {
  const CUtensorMap* map;
  unsigned mbar;   // shared-memory address of the barrier
  unsigned phase;  // parity of the next completion
};

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_init(uint64_t* mbar) {
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool tma_wait(unsigned mbar, unsigned phase) {
  const unsigned long long t0 = global_ns();
  for (int it = 0; it < kTmaWaitPolls; ++it) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (done) return true;
    if ((it & 255) == 255 && global_ns() - t0 > kTmaWaitNs) break;
  }
  return false;
}

// Stages transform t's padded tile at origin o into s_tile: by TMA when
// allowed, the tile does not wrap and the buffer is 128-byte aligned, else with
// plain loads.  Must be called by every thread of the CTA between barriers;
// false (for every thread) when a TMA wait gave up, and the caller then stops.
template <typename T>
__device__ __forceinline__ bool stage_interp_tile(const PointArgs<T>& a, const int o[3], const cplx_t<T>* grid, int t,
                                                  cplx_t<T>* s_tile, TmaStage& ts) {
  const Geom& g = a.g;
  const bool interior = a.tma && o[0] + g.pitch <= g.nf[0] && o[1] + g.pad[1] <= g.nf[1] &&
                        (g.dim < 3 || o[2] + g.pad[2] <= g.nf[2]) && (smem_addr(s_tile) & 127u) == 0;
  if (!interior) {
    stage_tile<T>(g, o, grid + (int64_t)t * a.grid_stride, s_tile);
    return true;
  }
  if (threadIdx.x == 0) {
    const unsigned bytes = (unsigned)(sizeof(cplx_t<T>) * g.pitch * g.pad[1] * g.pad[2]);
    const int x = o[0] * (int)(sizeof(cplx_t<T>) / 8);  // in 8-byte elements
    const uint64_t map = reinterpret_cast<uint64_t>(ts.map);
    const unsigned dst = smem_addr(s_tile);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier reads of the buffer before the async write
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(ts.mbar), "r"(bytes) : "memory");
    if (g.dim == 2)
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
          "[%5];" ::"r"(dst),
          "l"(map), "r"(x), "r"(o[1]), "r"(t), "r"(ts.mbar)
          : "memory");
    else
      asm volatile(
          "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
          "%5}], [%6];" ::"r"(dst),
          "l"(map), "r"(x), "r"(o[1]), "r"(o[2]), "r"(t), "r"(ts.mbar)
          : "memory");
  }
  const bool landed = tma_wait(ts.mbar, ts.phase);
  ts.phase ^= 1u;
  if (__syncthreads_and(landed)) return true;
  if (threadIdx.x == 0) atomicOr(a.status, NFX_STATUS_TMA_TIMEOUT);
  return false;
}

// ---------------------------------------------------------------------------
// Interpolation with one lane group per point (2D and 3D).  GL lanes (the power
// of two >= NS) share a point: lane kx = lane % GL reads footprint column kx of
// every row (ky, or (ky, kz) in 3D).  The 32 / GL points of one warp
// instruction are consecutive in cell order, so their rows overlap in shared
// memory (few wavefronts; thread-per-point reads of 32 scattered footprints
// conflict on many of theirs).  Each lane computes only its own column's weight
// per axis; the other axes' weights reach the group's lanes by shuffles, and the
// group sums its columns with a butterfly of shuffles.
// ---------------------------------------------------------------------------
template <int NS>
__host__ __device__ constexpr int group_lanes() {
  return NS <= 4 ? 4 : (NS <= 8 ? 8 : 16);
}

// Weight q of one axis: the same arithmetic as axis_weights for that q (cq =
// the polynomial coefficients of q when the float polynomial is in use).
template <typename T, int NS>
__device__ __forceinline__ T axis_weight_q(const PointArgs<T>& a, const float (&cq)[kPolyEvalDeg + 1], int i0, T xs,
                                           int q) {
  if (std::is_same<T, float>::value && a.poly.deg > 0) {
    const float v = 2.0f * (float)(xs - (T)i0) - (float)(NS - 1);
    float h = cq[kPolyEvalDeg];
#pragma unroll
    for (int d = kPolyEvalDeg - 1; d >= 0; --d) h = fmaf(h, v, cq[d]);
    return (T)h;
  }
  return es_weight(rn_sub((T)(i0 + q), xs), a.beta, a.kc);
}

// Left cells and tile offset of a point with folded coordinates xv (false:
// outside its bin's tile, see footprint).
template <typename T, int DIM, int NS>
__device__ __forceinline__ bool group_point(const PointArgs<T>& a, const T (&xv)[3], const int o[3], int row,
                                            int plane, int& off, T (&xs)[3], int (&i0)[3]) {
  const Geom& g = a.g;
  bool inside = true;
  off = 0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    xs[d] = xv[d];
    i0[d] = left_cell<T, NS>(xs[d]);
    const int l = wrap_index(i0[d], g.nf[d]) - o[d];
    inside = inside && (unsigned)l < (unsigned)g.tile[d];
    off += l * (d == 0 ? 1 : (d == 1 ? row : plane));
  }
  return inside;
}

// One round of 32 points for a warp: lane L takes point kb + L (left cells,
// tile offset; off = -1 outside the tile); the lane groups then take the
// points PPW at a time by shuffles (group_take).  The loads are pipelined
// across rounds: the next round's permutation entries and folded coordinates
// (both read in sorted order) are in flight while a round is processed.
template <typename T>
struct WarpPoints {
  int p, off;
  T xs[3];
  int i0[3];
};

__device__ __forceinline__ int round_perm(const SortView& s, int kb, int k1) {
  const int k = kb + (threadIdx.x & 31);
  return k < k1 ? s.perm[k] : -1;
}

template <typename T, int DIM>
__device__ __forceinline__ void round_coords(const PointArgs<T>& a, int kb, int k1, T (&xv)[3]) {
  const int k = kb + (threadIdx.x & 31);
#pragma unroll
  for (int d = 0; d < 3; ++d) xv[d] = (d < DIM && k < k1) ? sorted_coord(a, d, k) : (T)0;
}

template <typename T, int DIM, int NS>
__device__ __forceinline__ WarpPoints<T> warp_points(const PointArgs<T>& a, int p, const T (&xv)[3], const int o[3],
                                                     int row, int plane) {
  WarpPoints<T> w;
  w.p = p >= 0 ? p : 0;
  w.off = -1;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    w.xs[d] = (T)0;
    w.i0[d] = 0;
  }
  if (p >= 0) {
    int off;
    const bool inside = group_point<T, DIM, NS>(a, xv, o, row, plane, off, w.xs, w.i0);
    w.off = inside ? off : -1;
  }
  return w;
}

template <typename T, int DIM>
__device__ __forceinline__ WarpPoints<T> group_take(const WarpPoints<T>& w, int src) {
  constexpr unsigned kAll = 0xffffffffu;
  WarpPoints<T> r;
  r.p = __shfl_sync(kAll, w.p, src);
  r.off = __shfl_sync(kAll, w.off, src);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    r.xs[d] = d < DIM ? __shfl_sync(kAll, w.xs[d], src) : (T)0;
    r.i0[d] = d < DIM ? __shfl_sync(kAll, w.i0[d], src) : 0;
  }
  return r;
}

template <typename T, int DIM, int NS, int NW>
__device__ __forceinline__ void interp_group(const PointArgs<T>& a, const cplx_t<T>* __restrict__ fw,
                                             cplx_t<T>* __restrict__ cout, int sidx, unsigned char* smem_raw,
                                             TmaStage& ts) {
  using CT = cplx_t<T>;
  constexpr int GL = group_lanes<NS>();
  constexpr int PPW = 32 / GL;
  constexpr unsigned kAll = 0xffffffffu;
  CT* s_tile = reinterpret_cast<CT*>(smem_raw);
  const Geom& g = a.g;
  const int row = g.pitch;
  const int plane = g.pitch * g.pad[1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int kx = lane % GL;
  const int leader = lane - kx;
  const bool col_on = kx < NS;
  float cq[kPolyEvalDeg + 1];  // this lane's coefficients (constant-indexed parameter reads)
#pragma unroll
  for (int d = 0; d <= kPolyEvalDeg; ++d) cq[d] = a.poly.a[0][d];
#pragma unroll
  for (int q = 1; q < NS; ++q) {
    if (kx == q) {
#pragma unroll
      for (int d = 0; d <= kPolyEvalDeg; ++d) cq[d] = a.poly.a[q][d];
    }
  }
  const int b = a.s.sub_bin[sidx];
  const int k0 = a.s.sub_start[sidx];
  const int k1 = min(k0 + a.s.maxsub, a.s.bin_start[b + 1]);
  int o[3];
  bin_origin(g, b, o[0], o[1], o[2]);
  for (int t = 0; t < a.n_trans; ++t) {
    __syncthreads();
    if (!stage_interp_tile<T>(a, o, fw, t, s_tile, ts)) return;
    __syncthreads();
    constexpr int kStep = NW * 32;
    int p_cur = round_perm(a.s, k0 + warp * 32, k1);
    T x_cur[3];
    round_coords<T, DIM>(a, k0 + warp * 32, k1, x_cur);
    for (int kb = k0 + warp * 32; kb < k1; kb += kStep) {  // warp-uniform
      const int p_next = round_perm(a.s, kb + kStep, k1);
      T x_next[3];
      round_coords<T, DIM>(a, kb + kStep, k1, x_next);
      const WarpPoints<T> wp = warp_points<T, DIM, NS>(a, p_cur, x_cur, o, row, plane);
      p_cur = p_next;
#pragma unroll
      for (int d = 0; d < 3; ++d) x_cur[d] = x_next[d];
      const int npts = min(32, k1 - kb);
      for (int j0 = 0; j0 < npts; j0 += PPW) {
        const int j = j0 + lane / GL;
        const bool valid = j < npts;
        const WarpPoints<T> pt = group_take<T, DIM>(wp, valid ? j : 0);
        const bool on = col_on && pt.off >= 0;
        const T wx = axis_weight_q<T, NS>(a, cq, pt.i0[0], pt.xs[0], kx);
        const T wyq = axis_weight_q<T, NS>(a, cq, pt.i0[1], pt.xs[1], kx);
        T wy[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) wy[q] = __shfl_sync(kAll, wyq, leader + q);
        CT s;
        s.x = s.y = (T)0;
        if constexpr (DIM == 3) {
          const T wzq = axis_weight_q<T, NS>(a, cq, pt.i0[2], pt.xs[2], kx);
          T wz[NS];
#pragma unroll
          for (int q = 0; q < NS; ++q) wz[q] = __shfl_sync(kAll, wzq, leader + q);
          if (on) {
            const CT* base = s_tile + pt.off + kx;
            // one independent accumulator per z plane: NS chains in flight
            CT acc[NS];
#pragma unroll
            for (int kz = 0; kz < NS; ++kz) acc[kz].x = acc[kz].y = (T)0;
#pragma unroll
            for (int ky = 0; ky < NS; ++ky) {
#pragma unroll
              for (int kz = 0; kz < NS; ++kz) acc[kz] = fma2(splat2(wy[ky]), base[kz * plane + ky * row], acc[kz]);
            }
#pragma unroll
            for (int kz = 0; kz < NS; ++kz) s = fma2(splat2(wz[kz]), acc[kz], s);
          }
        } else {
          if (on) {
            const CT* base = s_tile + pt.off + kx;
            CT s1;
            s1.x = s1.y = (T)0;  // two chains
#pragma unroll
            for (int ky = 0; ky < NS; ky += 2) {
              s = fma2(splat2(wy[ky]), base[ky * row], s);
              s1 = fma2(splat2(wy[ky + 1]), base[(ky + 1) * row], s1);
            }
            s.x += s1.x;
            s.y += s1.y;
          }
        }
        T sr = on ? s.x * wx : (T)0, si = on ? s.y * wx : (T)0;
#pragma unroll
        for (int m = GL / 2; m >= 1; m >>= 1) {
          sr += __shfl_xor_sync(kAll, sr, m);
          si += __shfl_xor_sync(kAll, si, m);
        }
        if (valid && kx == 0) {
          CT r;
          r.x = sr;
          r.y = si;
          cout[(int64_t)t * a.M + pt.p] = with_extra(a, kb + j, r);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Interp
// ---------------------------------------------------------------------------
// Threads per point of the interpolation: one lane group (the 3D default) or
// one thread.  MODE is the variant compiled into a kernel (NFX_PER_POINT_GROUP
// or _THREAD), or NFX_PER_POINT_AUTO to choose per problem at run time from
// Geom::interp_mode (the batched kernel).
template <int DIM>
__host__ __device__ __forceinline__ bool interp_by_group(int mode) {
  return DIM >= 2 && (mode == NFX_PER_POINT_GROUP || (mode == NFX_PER_POINT_AUTO && DIM == 3));
}

template <typename T, int DIM, int NS, int NW, int MODE = NFX_PER_POINT_AUTO>
__device__ __forceinline__ void interp_subproblem(const PointArgs<T>& a, const cplx_t<T>* __restrict__ fw,
                                                  cplx_t<T>* __restrict__ cout, int sidx, unsigned char* smem_raw,
                                                  TmaStage& ts) {
  using CT = cplx_t<T>;
  if constexpr (DIM >= 2 && MODE != NFX_PER_POINT_THREAD) {
    if (MODE == NFX_PER_POINT_GROUP || interp_by_group<DIM>(a.g.interp_mode)) {
      interp_group<T, DIM, NS, NW>(a, fw, cout, sidx, smem_raw, ts);
      return;
    }
  }
  CT* s_tile = reinterpret_cast<CT*>(smem_raw);
  const Geom& g = a.g;
  const int row = g.pitch;
  const int plane = g.pitch * g.pad[1];
  {
    const int b = a.s.sub_bin[sidx];
    const int k0 = a.s.sub_start[sidx];
    const int k1 = min(k0 + a.s.maxsub, a.s.bin_start[b + 1]);
    int o[3];
    bin_origin(g, b, o[0], o[1], o[2]);
    for (int t = 0; t < a.n_trans; ++t) {
      __syncthreads();
      if (!stage_interp_tile<T>(a, o, fw, t, s_tile, ts)) return;
      __syncthreads();
      // loads pipelined across iterations: the next iteration's permutation
      // entry and folded coordinates (both in sorted order)
      const int kStep = blockDim.x;
      int k = k0 + threadIdx.x;
      int p_cur = k < k1 ? a.s.perm[k] : 0;
      T x_cur[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) x_cur[d] = k < k1 ? sorted_coord(a, d, k) : (T)0;
      for (; k < k1; k += kStep) {
        const int p = p_cur;
        T xv[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) xv[d] = x_cur[d];
        {
          const bool more = k + kStep < k1;
          p_cur = more ? a.s.perm[k + kStep] : 0;
#pragma unroll
          for (int d = 0; d < DIM; ++d) x_cur[d] = more ? sorted_coord(a, d, k + kStep) : (T)0;
        }
        T w[DIM][NS];
        int off = 0;
        bool inside = true;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          const T xs = xv[d];
          const int i0 = left_cell<T, NS>(xs);
          const int l = wrap_index(i0, g.nf[d]) - o[d];
          inside = inside && (unsigned)l < (unsigned)g.tile[d];
          off += l * (d == 0 ? 1 : (d == 1 ? row : plane));
          axis_weights<T, NS>(a, i0, xs, w[d]);
        }
        if (!inside) {  // stale sort: see k_spread
          CT zero;
          zero.x = zero.y = (T)0;
          cout[(int64_t)t * a.M + p] = zero;
          continue;
        }
        T ar = 0, ai = 0;
        const CT* base = s_tile + off;
        CT wxp[NS];  // (w_x, w_x) pairs, built once per point
#pragma unroll
        for (int kx = 0; kx < NS; ++kx) wxp[kx] = splat2(w[0][kx]);
#pragma unroll 1
        for (int kz = 0; kz < (DIM == 3 ? NS : 1); ++kz) {
          T zr = 0, zi = 0;
#pragma unroll
          for (int ky = 0; ky < (DIM >= 2 ? NS : 1); ++ky) {
            const CT* rp = base + kz * plane + ky * row;
            CT xa;
            xa.x = xa.y = (T)0;
#pragma unroll
            for (int kx = 0; kx < NS; ++kx) xa = fma2(wxp[kx], rp[kx], xa);
            const T xr = xa.x, xi = xa.y;
            if (DIM >= 2) {
              zr += xr * w[DIM >= 2 ? 1 : 0][ky];
              zi += xi * w[DIM >= 2 ? 1 : 0][ky];
            } else {
              zr += xr;
              zi += xi;
            }
          }
          if (DIM == 3) {
            ar += zr * w[DIM - 1][kz];
            ai += zi * w[DIM - 1][kz];
          } else {
            ar += zr;
            ai += zi;
          }
        }
        CT r;
        r.x = ar;
        r.y = ai;
        cout[(int64_t)t * a.M + p] = with_extra(a, k, r);
      }
    }
  }
}

template <typename T, int DIM, int NS, int NW, int MODE>
__global__ void __launch_bounds__(NW * 32) k_interp(PointArgs<T> a, const cplx_t<T>* __restrict__ fw,
                                                    cplx_t<T>* __restrict__ cout, const __grid_constant__ CUtensorMap tmap) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t mbar;
  TmaStage ts{&tmap, smem_addr(&mbar), 0u};
  if (a.tma) tma_init(&mbar);
  const int nsub = *a.s.nsub;
  for (int sidx = blockIdx.x; sidx < nsub; sidx += gridDim.x)
    interp_subproblem<T, DIM, NS, NW, MODE>(a, fw, cout, sidx, smem_raw, ts);
}

// ---------------------------------------------------------------------------
// Batched launches: many problems (own points, grid, tiling and sort) in one
// persistent launch.  `items` is a device table; `sub_prefix[p]` is the number
// of subproblems of problems < p (k_batch_prefix), so the CTAs walk one global
// work queue of (problem, bin tile) items.
// ---------------------------------------------------------------------------
template <typename T>
struct BatchItem {
  PointArgs<T> a;
  const void* src;  // spread: strengths; interp: fine grid
  void* dst;        // spread: fine grid (zeroed by the caller); interp: values
};

__device__ __forceinline__ int batch_find(const int* __restrict__ prefix, int n, int g) {
  int lo = 0, hi = n;  // largest p with prefix[p] <= g
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= g)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

template <typename T, int DIM, int NS, int NW>
__global__ void __launch_bounds__(NW * 32) k_spread_batch(const BatchItem<T>* __restrict__ items, int nitems,
                                                          const int* __restrict__ sub_prefix) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int total = sub_prefix[nitems];
  for (int gi = blockIdx.x; gi < total; gi += gridDim.x) {
    const int p = batch_find(sub_prefix, nitems, gi);
    const BatchItem<T>& it = items[p];
    spread_subproblem<T, DIM, NS, NW>(it.a, (const cplx_t<T>*)it.src, (cplx_t<T>*)it.dst, gi - sub_prefix[p],
                                      smem_raw);
    __syncthreads();
  }
}

template <typename T, int DIM, int NS, int NW>
__global__ void __launch_bounds__(NW * 32) k_interp_batch(const BatchItem<T>* __restrict__ items, int nitems,
                                                          const int* __restrict__ sub_prefix) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int total = sub_prefix[nitems];
  TmaStage ts{nullptr, 0u, 0u};  // batched items stage with plain loads (their PointArgs have tma = 0)
  for (int gi = blockIdx.x; gi < total; gi += gridDim.x) {
    const int p = batch_find(sub_prefix, nitems, gi);
    const BatchItem<T>& it = items[p];
    interp_subproblem<T, DIM, NS, NW>(it.a, (const cplx_t<T>*)it.src, (cplx_t<T>*)it.dst, gi - sub_prefix[p],
                                      smem_raw, ts);
  }
}

// ---------------------------------------------------------------------------
// Gradient pass (see launch_grad in nfx_internal.h)
// ---------------------------------------------------------------------------
template <typename T, int DIM, int NS, int NW>
__global__ void __launch_bounds__(NW * 32) k_grad(PointArgs<T> a, const cplx_t<T>* __restrict__ G,
                                                  const cplx_t<T>* __restrict__ V, cplx_t<T>* __restrict__ out_interp,
                                                  T* __restrict__ dx, T* __restrict__ dy, T* __restrict__ dz,
                                                  const __grid_constant__ CUtensorMap tmap) {
  using CT = cplx_t<T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t mbar;
  TmaStage ts{&tmap, smem_addr(&mbar), 0u};
  if (a.tma) tma_init(&mbar);
  CT* s_tile = reinterpret_cast<CT*>(smem_raw);
  const Geom& g = a.g;
  const int row = g.pitch;
  const int plane = g.pitch * g.pad[1];
  const int nsub = *a.s.nsub;
  T* douts[3] = {dx, dy, dz};
  for (int sidx = blockIdx.x; sidx < nsub; sidx += gridDim.x) {
    const int b = a.s.sub_bin[sidx];
    const int k0 = a.s.sub_start[sidx];
    const int k1 = min(k0 + a.s.maxsub, a.s.bin_start[b + 1]);
    int o[3];
    bin_origin(g, b, o[0], o[1], o[2]);
    for (int t = 0; t < a.n_trans; ++t) {
      __syncthreads();
      if (!stage_interp_tile<T>(a, o, G, t, s_tile, ts)) return;
      __syncthreads();
      // loads pipelined across iterations: the permutation two iterations
      // ahead, folded coordinates (sorted order) and V one iteration ahead
      const int kStep = blockDim.x;
      int k = k0 + threadIdx.x;
      int p_cur = k < k1 ? a.s.perm[k] : 0;
      int p_next = k + kStep < k1 ? a.s.perm[k + kStep] : 0;
      T x_cur[DIM];
      CT v_cur;
      v_cur.x = v_cur.y = (T)0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) x_cur[d] = k < k1 ? sorted_coord(a, d, k) : (T)0;
      if (k < k1) v_cur = V[(int64_t)t * a.M + p_cur];
      for (; k < k1; k += kStep) {
        const int p = p_cur;
        T xv[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) xv[d] = x_cur[d];
        const CT vv = v_cur;
        {
          const bool more = k + kStep < k1;
          const int p_after = k + 2 * kStep < k1 ? a.s.perm[k + 2 * kStep] : 0;
#pragma unroll
          for (int d = 0; d < DIM; ++d) x_cur[d] = more ? sorted_coord(a, d, k + kStep) : (T)0;
          if (more) v_cur = V[(int64_t)t * a.M + p_next];
          p_cur = p_next;
          p_next = p_after;
        }
        T w[DIM][NS], dw[DIM][NS];
        int off = 0;
        bool inside = true;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          const T xs = xv[d];
          const int i0 = left_cell<T, NS>(xs);
          const int l = wrap_index(i0, g.nf[d]) - o[d];
          inside = inside && (unsigned)l < (unsigned)g.tile[d];
          off += l * (d == 0 ? 1 : (d == 1 ? row : plane));
          const T scale = -(T)((double)g.nf[d] / (2.0 * kPi));
#pragma unroll
          for (int q = 0; q < NS; ++q) {
            T ph, dph;
            es_weight_deriv(rn_sub((T)(i0 + q), xs), a.beta, a.kc, ph, dph);
            w[d][q] = ph;
            dw[d][q] = dph * scale;
          }
        }
        // S[0] = sum G w ; S[1+d] = sum G (w with axis d differentiated)
        T sr[1 + DIM], si[1 + DIM];
#pragma unroll
        for (int i = 0; i <= DIM; ++i) sr[i] = si[i] = (T)0;
        const CT* base = s_tile + (inside ? off : 0);
        CT wxp[NS], dwxp[NS];  // (w_x, w_x) and (w_x', w_x') pairs, built once per point
#pragma unroll
        for (int kx = 0; kx < NS; ++kx) {
          wxp[kx] = splat2(w[0][kx]);
          dwxp[kx] = splat2(dw[0][kx]);
        }
#pragma unroll 1
        for (int kz = 0; kz < (inside && DIM == 3 ? NS : (inside ? 1 : 0)); ++kz) {
          // per-z accumulators: [0] plain, [1] d/dx, [2] d/dy
          T zr0 = 0, zi0 = 0, zr1 = 0, zi1 = 0, zr2 = 0, zi2 = 0;
#pragma unroll
          for (int ky = 0; ky < (DIM >= 2 ? NS : 1); ++ky) {
            const CT* rp = base + kz * plane + ky * row;
            CT xa, xa1;
            xa.x = xa.y = xa1.x = xa1.y = (T)0;
#pragma unroll
            for (int kx = 0; kx < NS; ++kx) {
              const CT v = rp[kx];
              xa = fma2(wxp[kx], v, xa);
              xa1 = fma2(dwxp[kx], v, xa1);
            }
            const T xr = xa.x, xi = xa.y, xr1 = xa1.x, xi1 = xa1.y;
            if (DIM >= 2) {
              const T wy = w[DIM >= 2 ? 1 : 0][ky], dwy = dw[DIM >= 2 ? 1 : 0][ky];
              zr0 += xr * wy;
              zi0 += xi * wy;
              zr1 += xr1 * wy;
              zi1 += xi1 * wy;
              zr2 += xr * dwy;
              zi2 += xi * dwy;
            } else {
              zr0 += xr;
              zi0 += xi;
              zr1 += xr1;
              zi1 += xi1;
            }
          }
          if (DIM == 3) {
            // z weights by an unrolled select: a dynamic index would put w / dw in local memory
            T wz = (T)0, dwz = (T)0;
#pragma unroll
            for (int q = 0; q < NS; ++q) {
              if (q == kz) {
                wz = w[DIM - 1][q];
                dwz = dw[DIM - 1][q];
              }
            }
            sr[0] += zr0 * wz;
            si[0] += zi0 * wz;
            sr[1] += zr1 * wz;
            si[1] += zi1 * wz;
            sr[2] += zr2 * wz;
            si[2] += zi2 * wz;
            sr[DIM] += zr0 * dwz;
            si[DIM] += zi0 * dwz;
          } else {
            sr[0] += zr0;
            si[0] += zi0;
            sr[1] += zr1;
            si[1] += zi1;
            if (DIM == 2) {
              sr[DIM] += zr2;
              si[DIM] += zi2;
            }
          }
        }
        if (out_interp != nullptr) {
          CT r;
          r.x = sr[0];
          r.y = si[0];
          out_interp[(int64_t)t * a.M + p] = r;
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          if (douts[d] != nullptr) {
            // Re(conj(v) * s) = v.x s.x + v.y s.y ; accumulate over transforms
            const T val = vv.x * sr[1 + d] + vv.y * si[1 + d];
            if (t == 0)
              douts[d][p] = val;
            else
              douts[d][p] += val;
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Host-side launch helpers (per instantiation)
// ---------------------------------------------------------------------------
template <typename T, int DIM, int NS>
struct Launch {
  static constexpr int NW = warps_per_cta(sizeof(T), DIM, NS);
  static size_t tile_smem(const Geom& g) { return (size_t)g.pad[2] * g.pad[1] * g.pitch * sizeof(cplx_t<T>); }

  template <typename K>
  static cudaError_t prep(K kernel, size_t smem, int& grid, int64_t max_subs) {
    return kernel_grid(reinterpret_cast<const void*>(kernel), NW * 32, smem, max_subs, grid);
  }

  static cudaError_t spread(const PointArgs<T>& a, const cplx_t<T>* c, cplx_t<T>* fw, cudaStream_t st) {
    int grid = 0;
    if constexpr (DIM == 3 && NS >= 4) {
      // threads per point (Geom::spread_mode): the whole CTA (warps own tile
      // planes; by default when points are sparser than grid cells: runs of
      // same-cell points are rare, and the plane-owner spread needs no
      // shared-memory atomics) or one warp (lanes own footprint columns)
      const bool sparse = a.M < (int64_t)a.g.nf[0] * a.g.nf[1] * a.g.nf[2];
      if (a.g.spread_mode == NFX_PER_POINT_CTA || (a.g.spread_mode == NFX_PER_POINT_AUTO && sparse)) {
        // the tile's row pitch is this kernel's own (footprint offsets follow it)
        PointArgs<T> ao = a;
        ao.g.pitch = owner_pitch(a.g.pitch, a.g.pad[0], NS, (int)sizeof(T));
        const size_t smem = owner_smem_bytes(sizeof(T), NS, NW, ao.g);
        cudaError_t e = prep(k_spread_owner<T, NS, NW>, smem, grid, ao.s.max_subs);
        if (e != cudaSuccess) return e;
        k_spread_owner<T, NS, NW><<<grid, NW * 32, smem, st>>>(ao, c, fw);
        return cudaGetLastError();
      }
    }
    size_t smem = spread_smem_bytes(sizeof(T), DIM, NS, a.g);
    cudaError_t e = prep(k_spread<T, DIM, NS, NW>, smem, grid, a.s.max_subs);
    if (e != cudaSuccess) return e;
    k_spread<T, DIM, NS, NW><<<grid, NW * 32, smem, st>>>(a, c, fw);
    return cudaGetLastError();
  }
  template <int MODE>
  static cudaError_t interp_as(const PointArgs<T>& a0, const cplx_t<T>* fw, cplx_t<T>* out, cudaStream_t st) {
    // the interpolation only reads the tile, so its row pitch is free
    PointArgs<T> a = a0;
    CUtensorMap tmap{};
    tma_args(a, fw, &tmap);
    size_t smem = tile_smem(a.g);
    int grid = 0;
    cudaError_t e = prep(k_interp<T, DIM, NS, NW, MODE>, smem, grid, a.s.max_subs);
    if (e != cudaSuccess) return e;
    k_interp<T, DIM, NS, NW, MODE><<<grid, NW * 32, smem, st>>>(a, fw, out, tmap);
    return cudaGetLastError();
  }
  static cudaError_t interp(const PointArgs<T>& a, const cplx_t<T>* fw, cplx_t<T>* out, cudaStream_t st) {
    if constexpr (DIM >= 2) {
      if (interp_by_group<DIM>(a.g.interp_mode)) return interp_as<NFX_PER_POINT_GROUP>(a, fw, out, st);
    }
    return interp_as<NFX_PER_POINT_THREAD>(a, fw, out, st);
  }
  // The tile staging of the interpolation and gradient passes: a tensor map of
  // the grid for TMA box loads of interior tiles when the rules allow (else
  // a.tma = 0 and plain loads); a complex64 tile gets an even row pitch.
  static void tma_args(PointArgs<T>& a, const cplx_t<T>* grid, CUtensorMap* tmap) {
    a.tma = 0;
    if constexpr (DIM >= 2) {
      Geom gt = a.g;
      if (sizeof(T) == 4 && (gt.pitch & 1)) ++gt.pitch;
      if (interp_tile_map(tmap, sizeof(T), DIM, gt, a.n_trans, grid)) {
        a.status = device_status_word();
        if (a.status != nullptr) {
          a.g = gt;
          a.tma = 1;
        }
      }
    }
  }
  static cudaError_t grad(const PointArgs<T>& a0, const cplx_t<T>* G, const cplx_t<T>* V, cplx_t<T>* oi, T* dx,
                          T* dy, T* dz, cudaStream_t st) {
    PointArgs<T> a = a0;
    CUtensorMap tmap{};
    tma_args(a, G, &tmap);
    size_t smem = tile_smem(a.g);
    int grid = 0;
    cudaError_t e = prep(k_grad<T, DIM, NS, NW>, smem, grid, a.s.max_subs);
    if (e != cudaSuccess) return e;
    k_grad<T, DIM, NS, NW><<<grid, NW * 32, smem, st>>>(a, G, V, oi, dx, dy, dz, tmap);
    return cudaGetLastError();
  }
};

template <typename T, int DIM, int NS>
struct BatchLaunch {
  static constexpr int NW = warps_per_cta(sizeof(T), DIM, NS);
  static cudaError_t spread(const void* items, int n, const int* prefix, int64_t max_subs, size_t smem,
                            cudaStream_t st) {
    int grid = 0;
    cudaError_t e = kernel_grid(reinterpret_cast<const void*>(k_spread_batch<T, DIM, NS, NW>), NW * 32, smem, max_subs,
                                grid);
    if (e != cudaSuccess) return e;
    k_spread_batch<T, DIM, NS, NW><<<grid, NW * 32, smem, st>>>((const BatchItem<T>*)items, n, prefix);
    return cudaGetLastError();
  }
  static cudaError_t interp(const void* items, int n, const int* prefix, int64_t max_subs, size_t smem,
                            cudaStream_t st) {
    int grid = 0;
    cudaError_t e = kernel_grid(reinterpret_cast<const void*>(k_interp_batch<T, DIM, NS, NW>), NW * 32, smem, max_subs,
                                grid);
    if (e != cudaSuccess) return e;
    k_interp_batch<T, DIM, NS, NW><<<grid, NW * 32, smem, st>>>((const BatchItem<T>*)items, n, prefix);
    return cudaGetLastError();
  }
};

template <typename T, int DIM>
cudaError_t dispatch_batch(int ns, bool spread, const void* items, int n, const int* prefix, int64_t max_subs,
                           size_t smem, cudaStream_t st) {
  switch (ns) {
#define NFX_CASE(N)                                                                    \
  case N:                                                                              \
    return spread ? BatchLaunch<T, DIM, N>::spread(items, n, prefix, max_subs, smem, st) \
                  : BatchLaunch<T, DIM, N>::interp(items, n, prefix, max_subs, smem, st);
    NFX_CASE(2) NFX_CASE(4) NFX_CASE(6) NFX_CASE(8) NFX_CASE(10) NFX_CASE(12) NFX_CASE(14) NFX_CASE(16)
#undef NFX_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <typename T, int DIM>
cudaError_t dispatch_spread(int ns, const PointArgs<T>& a, const void* c, void* fw, cudaStream_t st) {
  using CT = cplx_t<T>;
  switch (ns) {
#define NFX_CASE(N) \
  case N:           \
    return Launch<T, DIM, N>::spread(a, (const CT*)c, (CT*)fw, st);
    NFX_CASE(2) NFX_CASE(4) NFX_CASE(6) NFX_CASE(8) NFX_CASE(10) NFX_CASE(12) NFX_CASE(14) NFX_CASE(16)
#undef NFX_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <typename T, int DIM>
cudaError_t dispatch_interp(int ns, const PointArgs<T>& a, const void* fw, void* out, cudaStream_t st) {
  using CT = cplx_t<T>;
  switch (ns) {
#define NFX_CASE(N) \
  case N:           \
    return Launch<T, DIM, N>::interp(a, (const CT*)fw, (CT*)out, st);
    NFX_CASE(2) NFX_CASE(4) NFX_CASE(6) NFX_CASE(8) NFX_CASE(10) NFX_CASE(12) NFX_CASE(14) NFX_CASE(16)
#undef NFX_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <typename T, int DIM>
cudaError_t dispatch_grad(int ns, const PointArgs<T>& a, const void* G, const void* V, void* oi, void* dx, void* dy,
                          void* dz, cudaStream_t st) {
  using CT = cplx_t<T>;
  switch (ns) {
#define NFX_CASE(N)                                                                                             \
  case N:                                                                                                       \
    return Launch<T, DIM, N>::grad(a, (const CT*)G, (const CT*)V, (CT*)oi, (T*)dx, (T*)dy, (T*)dz, st);
    NFX_CASE(2) NFX_CASE(4) NFX_CASE(6) NFX_CASE(8) NFX_CASE(10) NFX_CASE(12) NFX_CASE(14) NFX_CASE(16)
#undef NFX_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <typename T>
PointArgs<T> make_args(const Geom& g, double beta, double kc, int64_t M, int n_trans, const SortView& s) {
  PointArgs<T> a;
  for (int d = 0; d < 3; ++d) a.sc[d] = (const T*)s.coord[d];
  a.M = M;
  a.n_trans = n_trans;
  a.grid_stride = (int64_t)g.nf[0] * g.nf[1] * g.nf[2];
  a.tma = 0;
  a.status = nullptr;
  a.g = g;
  a.beta = (T)beta;
  a.kc = (T)kc;
  a.s = s;
  a.poly.deg = 0;
  return a;
}

}  // namespace nfx
