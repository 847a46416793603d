// Internal declarations shared by the nufftax_b200 CUDA translation units.
#pragma once

#include <cuda.h>  // CUtensorMap (type only; the encoder is fetched from the driver at run time)
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>

#include "nfx.h"
#include "nfx_common.cuh"

namespace nfx {

// Workspace layout of one bin sort (all offsets in bytes from the workspace
// base, each 256-byte aligned).  Derived deterministically from the options and
// M, so the sort and every later spread/interp call agree on it.
struct SortLayout {
  int64_t M;
  int nbins;
  int ncell;        // cells per tile
  int cbits;        // composite key = bin << cbits | cell
  int bits;         // bits of the composite key
  int npass;        // radix passes (digits of dbits bits, least significant first)
  int dbits;
  int nchunks;      // chunks of one radix pass
  int maxsub;       // points per subproblem
  int64_t max_subs; // upper bound on the number of subproblems
  size_t off_keys, off_keys_tmp, off_vals_tmp, off_keys_sorted, off_perm, off_counts, off_totals, off_bin_start,
      off_sub_bin, off_sub_start, off_nsub;
  size_t off_coord[3];  // folded coordinates in sorted order, one array per axis (0 = unused axis)
  size_t off_coord_tmp[3];  // float, non-type-3 sorts: ping-pong buffers of the coordinates the passes carry
  size_t off_extra;     // type 3 only: one complex factor per sorted point (0 = none)
  size_t total;
};

struct SortPtrs {
  int* keys;         // composite key per point (input order)
  int* keys_tmp;     // ping-pong buffers of the radix passes
  int* vals_tmp;
  int* keys_sorted;  // composite keys in sorted order
  int* perm;         // final (bin, cell) order
  int* counts;       // nchunks x 2^dbits digit counts, then their column prefixes
  int* totals;       // 2^dbits digit totals
  int* bin_start;
  int* sub_bin;
  int* sub_start;
  int* nsub;
  void* coord[3];  // sorted folded coordinates (working precision), nullptr for unused axes
  void* coord_tmp[3];  // the passes' second coordinate buffers (nullptr: coordinates are gathered instead)
  void* extra;     // type 3: complex factor per sorted point, else nullptr
};

// Pointers a spread / interp / gradient launch needs from a finished sort.
// coord[d][k] is the folded, rescaled coordinate fold(x_d[perm[k]]) in [0, nf_d]
// of the k-th sorted point (working precision), written by the sort so that the
// passes read coordinates in sorted order instead of gathering them.
struct SortView {
  const void* coord[3];
  // Type-3 sorts only (else nullptr): a complex factor per sorted point that
  // the spread multiplies into the strength (sources: the pre-phase) or the
  // interpolation into the value it writes (targets: phase / phihat).
  const void* extra;
  const int* perm;
  const int* bin_start;
  const int* sub_bin;
  const int* sub_start;
  const int* nsub;
  int maxsub;
  int64_t max_subs;
};

void radix_plan(int nbins, int ncell, int& cbits, int& bits, int& npass, int& dbits);
int radix_chunk();
// out[i] = bin of point i (composite key / cells per tile)
cudaError_t bin_keys_of(const SortLayout& L, const int* K, int* out, cudaStream_t st);

template <typename T>
cudaError_t launch_sort(const SortLayout& L, const Geom& g, int ns, const void* x, const void* y, const void* z,
                        int64_t M, const SortPtrs& P, cudaStream_t st);

// Type-3 set-up on the device: min / max of sources and targets per axis and
// the T3Params from them (scratch of t3_scratch_bytes()).
size_t t3_scratch_bytes();
template <typename T>
cudaError_t launch_t3_params(int dim, const int nf[3], double upsampfac, const void* const* src, int64_t M,
                             const void* const* tgt, int64_t K, T3Params* params, void* scratch, cudaStream_t st);

// Spread: fw (n_trans x prod nf, complex) must be zeroed by the caller.
template <typename T>
cudaError_t launch_spread(const Geom& g, int ns, double beta, double kc, const void* x, const void* y, const void* z,
                          int64_t M, const void* c, int n_trans, void* fw, const SortView& s, cudaStream_t st);

template <typename T>
cudaError_t launch_interp(const Geom& g, int ns, double beta, double kc, const void* x, const void* y, const void* z,
                          int64_t M, const void* fw, int n_trans, void* c_out, const SortView& s, cudaStream_t st);

// Gradient pass over points: with grid G and point values V (both n_trans deep)
//   out_interp[t][p] = sum_cells G[t] w          (if out_interp != nullptr)
//   d_axis[p]        = sum_t Re(conj(V[t][p]) * sum_cells G[t] dw_axis)   (for each non-null axis output)
template <typename T>
cudaError_t launch_grad(const Geom& g, int ns, double beta, double kc, const void* x, const void* y, const void* z,
                        int64_t M, const void* G, const void* V, int n_trans, void* out_interp, void* dx, void* dy,
                        void* dz, const SortView& s, cudaStream_t st);

template <typename T>
cudaError_t launch_deconv_shuffle(int dim, const int nf[3], const int nm[3], const T* f1, const T* f2, const T* f3,
                                  const void* fw_hat, void* out, int n_trans, cudaStream_t st);
template <typename T>
cudaError_t launch_deconv_pad(int dim, const int nf[3], const int nm[3], const T* f1, const T* f2, const T* f3,
                              const void* f_in, void* fw_hat, int n_trans, cudaStream_t st);

template <typename T>
cudaError_t launch_deconv_batch(bool pad, const void* items, int n, int64_t total, cudaStream_t st);
size_t deconv_item_bytes(int precision);
// Work units (row segments of the output) of one problem of a batched
// deconvolution pass (pad: the fine grid nf; else the modes nm).
int64_t deconv_units(const int nf[3], const int nm[3], bool pad);
// Fill a host table of batched deconvolution items; returns the total work units.
int64_t fill_deconv_items(int precision, int dim, bool pad, const int* nf, const int* nm, const void* const* fac,
                          const void* const* src, void* const* dst, int n, void* host_items);

int num_sms();
void set_error(const std::string& msg);

// Tensor map of a fine grid (n_trans x nf3 x nf2 x nf1 complex of 2 * real_bytes
// bytes) whose box is the interpolation's padded tile (pitch x pad_y [x pad_z] x 1
// elements of 8 bytes), for TMA staging.  False (no map) when TMA staging is
// off (NFX_INTERP_STAGING=plain in the environment), the driver lacks the
// encoder, or the grid or box breaks a TMA rule (16-byte strides and base,
// box edges <= 256); the caller then stages with plain loads.
bool interp_tile_map(CUtensorMap* map, size_t real_bytes, int dim, const Geom& g, int n_trans, const void* grid);

// The current device's status word (a __device__ int of this library), or
// nullptr if its address cannot be had.  Kernels OR NFX_STATUS_* bits into it;
// nfx_device_status reads and clears it.
int* device_status_word();

// Warps per CTA of the spread / interp / gradient kernels.
constexpr int warps_per_cta(size_t real_bytes, int dim, int ns) { return (real_bytes == 8 && dim == 3) ? 4 : 8; }

// Run-merging spread layout (2D/3D footprints of at least 32 cells): lane l of
// a warp owns footprint column kx = l % ns and rows (y, or z*ns + y) grp*rpl ..
// grp*rpl + rpl - 1 with grp = l / ns; the 32 / ns groups cover the ns^(dim-1)
// rows.  A staged point is one slot of reals: c * w_x (ns complex), then the y
// weights and (3D) the z weights.  Sections are padded to the rows the groups
// reach and to whole 16-byte chunks; the slot length (4 mod 8 floats, 2 mod 4
// doubles) makes the 16-byte stores of a warp (one slot per lane) hit distinct
// banks.  The walk reads the weights with scalar loads: every lane of a group
// reads the same word (one broadcast wavefront), which keeps the shared-memory
// pipe less busy than wider loads would.
// run_slot_reals is 0 when the layout does not apply (1D, small footprints,
// more than 16 rows a lane).
__host__ __device__ constexpr int run_groups(int ns) { return 32 / ns; }
__host__ __device__ constexpr int run_rows(int dim, int ns) { return dim == 3 ? ns * ns : ns; }
__host__ __device__ constexpr int run_rows_per_lane(int dim, int ns) {
  return (run_rows(dim, ns) + run_groups(ns) - 1) / run_groups(ns);
}
__host__ __device__ constexpr int round4(int n) { return (n + 3) / 4 * 4; }
// reals of the y and z sections
__host__ __device__ constexpr int run_wy(int dim, int ns) {
  return dim == 2 ? round4(run_groups(ns) * run_rows_per_lane(dim, ns)) : round4(ns);
}
__host__ __device__ constexpr int run_wz(int dim, int ns) {
  return dim == 3 ? round4((run_groups(ns) * run_rows_per_lane(dim, ns) + ns - 1) / ns) : 0;
}
__host__ __device__ constexpr int run_slot_base(int dim, int ns) {
  return round4(2 * ns) + run_wy(dim, ns) + run_wz(dim, ns);
}
__host__ __device__ constexpr int run_slot_reals(int dim, int ns, int real_bytes) {
  return (dim >= 2 && run_rows(dim, ns) * ns >= 32 && run_rows_per_lane(dim, ns) <= 16)
             ? (real_bytes == 4 ? run_slot_base(dim, ns) + (run_slot_base(dim, ns) % 8 == 0 ? 4 : 0)
                                : run_slot_base(dim, ns) + 2)
             : 0;
}

// Dynamic shared memory of the spread kernel: two planar tile planes plus the
// per-warp staging of 32 points (weights, strengths; tile offsets for the
// layout without run merging).
inline size_t spread_smem_bytes(size_t real_bytes, int dim, int ns, const Geom& g) {
  const int nw = warps_per_cta(real_bytes, dim, ns);
  const size_t tile = 2 * real_bytes * (size_t)g.pad[2] * g.pad[1] * g.pitch;
  const int slot = run_slot_reals(dim, ns, (int)real_bytes);
  if (slot > 0) return ((tile + 15) & ~(size_t)15) + (size_t)nw * 32 * slot * real_bytes;  // 16-byte aligned slots
  return tile + ((size_t)dim * ns * (nw * 32 + 1) + (size_t)2 * nw * 32) * real_bytes + (size_t)nw * 32 * sizeof(int);
}
// Dynamic shared memory of the plane-owner spread (3D, sparse points): two tile
// planes plus one slot of 4 ns + 3 reals per staged point.
// Staging slot of the plane-owner spread, in reals of real_bytes each: c * w_x
// pairs (2 ns), w_y and w_z (each padded to whole 16-byte vectors), then the
// footprint's tile offset and z (padded to a vector).  The slot is a whole, odd
// number of 16-byte vectors, so 16-byte stores of consecutive slots are
// conflict-free and every slot starts 16-byte aligned.
__host__ __device__ constexpr int owner_pad(int n, int m) { return (n + m - 1) / m * m; }
__host__ __device__ constexpr int owner_slot_raw(int real_bytes, int ns) {
  return 2 * ns + 2 * owner_pad(ns, 16 / real_bytes) + owner_pad(2, 16 / real_bytes);
}
__host__ __device__ constexpr int owner_slot_reals(int real_bytes, int ns) {
  return (owner_slot_raw(real_bytes, ns) / (16 / real_bytes)) % 2 == 0 ? owner_slot_raw(real_bytes, ns) + 16 / real_bytes
                                                                        : owner_slot_raw(real_bytes, ns);
}
inline size_t owner_smem_bytes(size_t real_bytes, int ns, int nw, const Geom& g) {
  const int r16 = 16 / (int)real_bytes;
  const size_t tile = (size_t)owner_pad(2 * g.pad[2] * g.pad[1] * g.pitch, r16);
  return real_bytes * (tile + (size_t)nw * 32 * owner_slot_reals((int)real_bytes, ns));
}
inline size_t tile_smem_bytes(size_t real_bytes, const Geom& g) {
  return 2 * real_bytes * (size_t)g.pad[2] * g.pad[1] * g.pitch;
}
inline size_t interp_smem_bytes(size_t real_bytes, int dim, int ns, const Geom& g) {
  (void)dim;
  (void)ns;
  return tile_smem_bytes(real_bytes, g);
}

// Persistent grid size for a kernel: SMs x resident CTAs (cached per device,
// kernel and shared-memory size), capped by the amount of work.
cudaError_t kernel_grid(const void* fn, int threads, size_t smem, int64_t max_work, int& grid);
// Opt a kernel in to `smem` bytes of dynamic shared memory (cached per device).
cudaError_t ensure_smem(const void* fn, size_t smem);
// Ask for the largest shared-memory carveout for a kernel (cached per device).
cudaError_t prefer_max_smem(const void* fn);

}  // namespace nfx
