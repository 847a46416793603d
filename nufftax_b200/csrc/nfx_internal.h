// Internal declarations shared by the nufftax_b200 CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>

#include "nfx_common.cuh"

namespace nfx {

// Workspace layout of one bin sort (all offsets in bytes from the workspace
// base, each 256-byte aligned).  Derived deterministically from the options and
// M, so the sort and every later spread/interp call agree on it.
struct SortLayout {
  int64_t M;
  int nbins;
  int ncell;        // cells per tile (keys of the first sort pass)
  int chunk;        // points per CTA in the counting passes
  int nchunks;
  int sort_warps;       // warps per CTA of the bin scatter pass
  size_t sort_smem;     // its dynamic shared memory
  int sort_warps_cell;  // same for the cell scatter pass
  size_t sort_smem_cell;
  int64_t n_counts; // max(nbins, ncell) * nchunks
  int64_t scan_blocks;
  int maxsub;       // points per subproblem
  int64_t max_subs; // upper bound on the number of subproblems
  size_t off_keys, off_keys_cell, off_keys_by_cell, off_perm_cell, off_perm, off_counts, off_scan, off_bin_start,
      off_sub_bin, off_sub_start, off_nsub;
  size_t total;
};

struct SortPtrs {
  int* keys;          // bin key per point (input order)
  int* keys_cell;     // cell-in-tile key per point (input order)
  int* keys_by_cell;  // bin keys in cell-sorted order
  int* perm_cell;     // cell-sorted order
  int* perm;          // final (bin, cell) order
  int* counts;
  int* scan_tmp;
  int* bin_start;
  int* sub_bin;
  int* sub_start;
  int* nsub;
};

// Pointers a spread / interp / gradient launch needs from a finished sort.
struct SortView {
  const int* perm;
  const int* bin_start;
  const int* sub_bin;
  const int* sub_start;
  const int* nsub;
  int maxsub;
  int64_t max_subs;
};

int64_t scan_blocks(int64_t n);
cudaError_t exclusive_scan(const int* in, int* out, int64_t n, int* block_sums, cudaStream_t st);

template <typename T>
cudaError_t launch_sort(const SortLayout& L, const Geom& g, int ns, const void* x, const void* y, const void* z,
                        int64_t M, const SortPtrs& P, cudaStream_t st);

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
// Fill a host table of batched deconvolution items; returns the total element count.
int64_t fill_deconv_items(int precision, int dim, bool pad, const int* nf, const int* nm, const void* const* fac,
                          const void* const* src, void* const* dst, int n, void* host_items);

int num_sms();
void set_error(const std::string& msg);

// Warps per CTA of the spread / interp / gradient kernels.
constexpr int warps_per_cta(size_t real_bytes, int dim, int ns) { return (real_bytes == 8 && dim == 3) ? 4 : 8; }

// Dynamic shared memory of the spread kernel: two planar tile planes plus the
// per-warp staging of 32 points (weights, strengths, tile offsets).
inline size_t spread_smem_bytes(size_t real_bytes, int dim, int ns, const Geom& g) {
  const int nw = warps_per_cta(real_bytes, dim, ns);
  return 2 * real_bytes * (size_t)g.pad[2] * g.pad[1] * g.pitch +
         ((size_t)dim * ns * (nw * 32 + 1) + (size_t)2 * nw * 32) * real_bytes + (size_t)nw * 32 * sizeof(int);
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

}  // namespace nfx
