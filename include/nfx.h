/*
 * nfx.h -- C ABI of the nufftax_b200 CUDA library (libnfx_b200.so, sm_100a).
 *
 * Plain C: device pointers, sizes and a CUDA stream passed as void*.  The caller
 * owns every buffer (inputs, outputs and workspace); the library owns only its
 * cuFFT plan cache.  Every entry point returns an nfx status code and never
 * aborts; nfx_last_error() gives the message of the calling thread's last
 * failure.  All work is enqueued on `stream` (NULL = legacy default stream) and
 * no entry point synchronises the device.
 *
 * Array conventions (shared with nufftax, the reference):
 *   coordinates   x, y, z: M reals (float or double per `precision`)
 *   strengths     c: n_trans x M complex (interleaved re, im), transform-major
 *   fine grid     fw: n_trans x nf3 x nf2 x nf1 complex, x fastest
 *                 (nufftax/core/spread.py:466, 653)
 *   modes         f: n_trans x n3 x n2 x n1 complex in CMCL order,
 *                 k = -n/2 .. (n-1)/2 per axis (nufftax/core/deconvolve.py:27-73)
 * Unused axes of 1D/2D problems have size 1 and NULL coordinate pointers.
 */
#ifndef NFX_H
#define NFX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  NFX_OK = 0,
  NFX_ERR_INVALID = 1,     /* bad argument (size, pointer, nspread, dim, ...) */
  NFX_ERR_WORKSPACE = 2,   /* workspace smaller than the matching *_bytes query */
  NFX_ERR_CUDA = 3,        /* a CUDA runtime call failed */
  NFX_ERR_CUFFT = 4,       /* a cuFFT call failed */
  NFX_ERR_UNSUPPORTED = 5  /* valid request outside what the kernels support */
};

enum { NFX_F32 = 0, NFX_F64 = 1 };

/* Threads per point of the spread / interpolation kernels (nfx_opts::spread_mode,
 * interp_mode).  AUTO: the library's choice (spread: the CTA in 3D when there are
 * fewer points than grid cells, else a warp; interpolation: a lane group in 3D,
 * one thread in 1D/2D).  THREAD: one thread per point (interpolation).  GROUP:
 * one lane group of the power of two >= nspread lanes per point, a lane per
 * footprint column (interpolation, 2D/3D).  WARP: one warp per point, a lane per
 * footprint column, runs of same-cell points summed in registers (spread).
 * CTA: every warp of the CTA on each point, a warp per tile z-plane, no atomics
 * (spread, 3D, nspread >= 4).  A mode that does not apply to a dimension falls
 * back to AUTO. */
enum { NFX_PER_POINT_AUTO = 0, NFX_PER_POINT_THREAD = 1, NFX_PER_POINT_GROUP = 2,
       NFX_PER_POINT_WARP = 3, NFX_PER_POINT_CTA = 4 };

/* Spreading/interpolation options: the grid, the ES kernel and the tiling.
 * nspread/beta/kc are nufftax's KernelParams (nufftax/core/kernel.py:19-25,
 * computed by compute_kernel_params, kernel.py:165-206).  tile[] = 0 and
 * max_subproblem = 0 select the library defaults (nfx_default_tiles). */
typedef struct nfx_opts {
  int precision;       /* NFX_F32 (float/complex64) or NFX_F64 (double/complex128) */
  int dim;             /* 1, 2 or 3 */
  int nf[3];           /* fine grid size per axis (x, y, z); unused axes 1 */
  int nspread;         /* kernel width, even, 2..16 */
  double beta;         /* ES shape parameter */
  double kc;           /* ES c = 4 / nspread^2 */
  int prenorm;         /* 1: apply mod(x + pi, 2 pi) - pi before folding, as the
                          transforms do (nufftax/transforms/nufft1.py:71); 0: fold
                          only, as the core spread / interp functions do */
  int tile[3];         /* bin edge per axis in cells; 0 = default */
  int max_subproblem;  /* points per subproblem; 0 = default (2048 in 3D; in 1D/2D
                          1024, doubled up to 4096 while M / (2 * size) >= 1480) */
  int spread_mode;     /* NFX_PER_POINT_AUTO, _WARP or _CTA */
  int interp_mode;     /* NFX_PER_POINT_AUTO, _THREAD or _GROUP */
} nfx_opts;

/* Library identity and last error of the calling thread. */
int nfx_version(void);
const char* nfx_last_error(void);
int nfx_num_sms(void);

/* Status bits of the current GPU that kernels set when a bounded wait gave up
 * instead of hanging: NFX_STATUS_TMA_TIMEOUT, a tile copy of the interpolation
 * (staged by TMA) did not land within 0.5 s and that CTA stopped, leaving its
 * outputs incomplete.  nfx_device_status synchronizes the device, writes the
 * bits to *status and clears them.  (No counterpart in the reference.) */
enum { NFX_STATUS_TMA_TIMEOUT = 1 };
int nfx_device_status(int* status);

/* Self-test of that bounded wait (no counterpart in the reference): one CTA
 * arms a barrier for a tile copy that is never issued, so its wait runs out
 * after the limit; the kernel records NFX_STATUS_TMA_TIMEOUT and returns with
 * nothing in flight.  Synchronizes the device (about 0.5 s) and writes the
 * status bits read (and cleared) to *status: NFX_STATUS_TMA_TIMEOUT when the
 * bound works. */
int nfx_selftest_bounded_wait(int* status);

/* Id of the CUDA graph capture the stream takes part in (cudaStreamGetCaptureInfo),
 * 0 when it is not capturing.  Lets a host layer reuse work captured earlier in the
 * same capture (a point sort shared by a type 1 and a type 2). */
int nfx_capture_id(void* stream, unsigned long long* id);

/* Polynomial form of the ES weights used by the float kernels (no counterpart
 * in the reference, which evaluates exp/sqrt): coefficients a[q][d] of
 * phi(q - (v + ns - 1) / 2) as a degree-`degree` polynomial in v in [-1, 1],
 * written to coeffs[q * 16 + d] (the polynomial of ns - 1 - q is that of q at
 * -v); max_abs_err is the worst float error of the kernels' evaluation forms
 * (Horner in v, and the even / odd split E(v^2) +- v O(v^2)) against the
 * exp/sqrt form.  A fit is used when that error stays within
 * 3e-8 + 2.6e-7 |phi| (about two float ulps); degree 0 means none was found and
 * the kernels evaluate exp/sqrt. */
int nfx_es_poly(int nspread, double beta, double kc, float* coeffs, int* degree, double* max_abs_err);

/* Fill tile[] with the defaults the library would use (max_subproblem = 0 is
 * left as is: its default depends on the number of points). */
int nfx_default_tiles(nfx_opts* opts);

/* ---- bin sort --------------------------------------------------------------
 * Bytes of workspace a sort of M points needs, and the sort itself: a stable
 * radix sort of the points by (tile of their footprint's left cell, that cell
 * within the tile).  The
 * workspace then holds the permutation and the bin/subproblem tables that every
 * *_sorted call below reads; it stays valid while the coordinates are unchanged.
 * (No counterpart in the reference, which spreads unsorted points.) */
int nfx_sort_workspace_bytes(const nfx_opts* opts, int64_t M, size_t* bytes);
int nfx_sort_points(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M, void* workspace,
                    size_t workspace_bytes, void* stream);
/* Kernels one nfx_sort_points call launches for these options and M (type3 != 0:
 * a type-3 source or target sort inside nfx_nufft3); host-only query. */
int nfx_sort_kernel_count(const nfx_opts* opts, int64_t M, int type3, int* n);
/* Copy the sort results out of a workspace (device pointers, any may be NULL):
 * keys[M] (bin of each point, input order), perm[M] (int32) and
 * bin_start[nbins + 1]. */
int nfx_sort_results(const nfx_opts* opts, int64_t M, const void* workspace, size_t workspace_bytes, int* keys,
                     int* perm, int* bin_start, int* nbins, void* stream);

/* ---- spread / interp -------------------------------------------------------
 * Replace nufftax/core/spread.py:717-758:
 *   _spread_{1,2,3}d_dispatch(x[, y[, z]], c, nf1[, nf2[, nf3]], kernel_params) -> fw
 *   _interp_{1,2,3}d_dispatch(x[, y[, z]], fw, kernel_params) -> c
 * nfx_spread / nfx_interp sort first (workspace of nfx_sort_workspace_bytes);
 * the *_sorted forms reuse a workspace already filled by nfx_sort_points.
 * nfx_spread* overwrite fw (it is zeroed on the stream first). */
int nfx_spread(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M, const void* c,
               int n_trans, void* fw, void* workspace, size_t workspace_bytes, void* stream);
int nfx_interp(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M, const void* fw,
               int n_trans, void* c_out, void* workspace, size_t workspace_bytes, void* stream);
int nfx_spread_sorted(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M, const void* c,
                      int n_trans, void* fw, const void* workspace, size_t workspace_bytes, void* stream);
int nfx_interp_sorted(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M, const void* fw,
                      int n_trans, void* c_out, const void* workspace, size_t workspace_bytes, void* stream);

/* ---- spreading without any allocation ---------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory or pass a workspace (code inside another framework's operator that
 * only receives its operand and result buffers, or code under a fixed memory
 * budget): same result as nfx_spread, with the sort scratch in a fixed array
 * of nfx_noalloc_scratch_bytes() (64 MiB) that the library holds on every GPU
 * that loads it.  Requests needing more scratch fail with NFX_ERR_UNSUPPORTED.
 * The first call on a device looks up the array's address (make it before any
 * stream capture) and keeps it for the process: it does not survive a
 * cudaDeviceReset.  Calls that overlap on the GPU race on the shared array. */
size_t nfx_noalloc_scratch_bytes(void);
int nfx_spread_noalloc(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M, const void* c,
                       int n_trans, void* fw, void* stream);

/* ---- adjoints (ES-derivative coordinate gradients) ---------------------------
 * Replace the backward rules of the core custom_vjp's
 * (nufftax/core/spread.py:766-1305; torch convention G = dL/dRe + i dL/dIm):
 *   nfx_spread_grad_sorted: given the grid cotangent g (n_trans x grid) and the
 *     forward strengths c, writes dc = interp(g) (if dc != NULL) and
 *     d{x,y,z}[j] = sum_t Re(conj(c[t,j]) * sum_cells g * dphi/d{x,y,z})
 *     (spread.py:820-858, 997-1032, 1168-1212), all in one pass over the tiles.
 *   nfx_interp_grad_sorted: given the grid fw and the point cotangent g,
 *     d{x,y,z}[j] = sum_t Re(conj(g[t,j]) * sum_cells fw * dphi/d{x,y,z})
 *     (spread.py:911-944, 1080-1114, 1261-1305); the fw cotangent is
 *     nfx_spread_sorted(g).
 * Coordinate outputs are reals of the working precision; NULL skips an axis. */
int nfx_spread_grad_sorted(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M,
                           const void* c, const void* g_grid, int n_trans, void* dc, void* dx, void* dy, void* dz,
                           const void* workspace, size_t workspace_bytes, void* stream);
int nfx_interp_grad_sorted(const nfx_opts* opts, const void* x, const void* y, const void* z, int64_t M,
                           const void* fw, const void* g_pts, int n_trans, void* dx, void* dy, void* dz,
                           const void* workspace, size_t workspace_bytes, void* stream);

/* ---- deconvolution / mode reordering ----------------------------------------
 * fac1..fac3: per-axis factors (-1)^k / phihat(|k|) in CMCL order (device arrays
 * of n_modes[d] reals; NULL for unused axes), nufftax/core/deconvolve.py:27-56.
 * nfx_deconv_shuffle replaces deconvolve_shuffle_{1,2,3}d (deconvolve.py:81-111,
 * 174-224, 312-366); nfx_deconv_pad replaces deconvolve_pad_{1,2,3}d
 * (deconvolve.py:114-166, 227-304, 369-468) and writes every grid cell. */
int nfx_deconv_shuffle(int precision, int dim, const int nf[3], const int n_modes[3], const void* fac1,
                       const void* fac2, const void* fac3, const void* fw_hat, void* f_out, int n_trans,
                       void* stream);
int nfx_deconv_pad(int precision, int dim, const int nf[3], const int n_modes[3], const void* fac1, const void* fac2,
                   const void* fac3, const void* f_in, void* fw_hat, int n_trans, void* stream);

/* ---- FFT (cuFFT, cached plans) ----------------------------------------------
 * In-place batched C2C over the last `dim` axes of n_trans grids.
 * sign = +1: sum_n v[n] e^{+2 pi i k n / nf} (nufftax's ifftn(.) * prod(nf));
 * sign = -1: e^{-...} (fftn).  nufftax/transforms/nufft1.py:81,154,232-235;
 * nufft2.py:317,383,454-457.  Calls on different streams may run concurrently,
 * also with the same plan: the cuFFT work area belongs to the stream (one per
 * device and stream handle, stream-ordered cudaMallocAsync, grown as needed). */
int nfx_fft(int precision, int dim, const int nf[3], int n_trans, void* data, int sign, void* stream);
/* The same transform on a caller-owned work area of at least nfx_fft_work_bytes
 * bytes (NULL when that is 0).  This is the form to capture in a CUDA graph:
 * nfx_fft refuses a capturing stream, since the graph would keep a work area
 * that later calls on the same stream handle reuse or replace. */
int nfx_fft_work_bytes(int precision, int dim, const int nf[3], int n_trans, size_t* bytes);
int nfx_fft_ws(int precision, int dim, const int nf[3], int n_trans, void* data, int sign, void* work,
               size_t work_bytes, void* stream);
/* Destroy the cached plans and free the streams' work areas (synchronises the devices). */
int nfx_fft_cache_clear(void);
/* Bound the plan cache (default 1024 plans); the least recently used plan is
 * destroyed, after a device synchronisation, when a new one needs room. */
int nfx_fft_cache_limit(int max_plans);

/* ---- whole transforms in one call -----------------------------------------
 * The type-1 and type-2 pipelines of nufftax/transforms/nufft1.py:47-90 and
 * nufft2.py:285-330 as one library call, for callers that want one host call
 * per transform (serving loops): nfx_nufft1 sorts the points into the
 * workspace, spreads c into fw (n_trans fine grids), runs the FFT with
 * fft_sign and deconvolves / reorders into f_out (n_trans x n_modes, CMCL
 * order); nfx_nufft2 deconvolves / zero-pads f_in into fw, runs the FFT,
 * sorts and interpolates into c_out.  fac1..fac3 are the per-axis
 * deconvolution factors (device, precision's real type; unused axes NULL),
 * n_modes[d] the modes per axis; workspace of nfx_sort_workspace_bytes.  The
 * FFT step uses the stream's cuFFT work area (nfx_fft), so these two refuse a
 * capturing stream (NFX_ERR_INVALID); capture the step-by-step calls with
 * nfx_fft_ws instead. */
int nfx_nufft1(const nfx_opts* opts, const int n_modes[3], const void* x, const void* y, const void* z, int64_t M,
               const void* c, int n_trans, int fft_sign, const void* fac1, const void* fac2, const void* fac3, void* fw,
               void* f_out, void* workspace, size_t workspace_bytes, void* stream);
int nfx_nufft2(const nfx_opts* opts, const int n_modes[3], const void* x, const void* y, const void* z, int64_t M,
               const void* f_in, int n_trans, int fft_sign, const void* fac1, const void* fac2, const void* fac3,
               void* fw, void* c_out, void* workspace, size_t workspace_bytes, void* stream);

/* ---- batching: many problems in one launch --------------------------------
 * No counterpart in the reference (nufftax vmaps one problem's strengths).
 * Each problem has its own points, fine grid, tiling and sort workspace; the
 * kernel (nspread, beta, kc), precision, dim and prenorm come from `common`.
 * nfx_batch_sort sorts every problem; nfx_batch_upload writes a device table
 * for one direction (spread: src = strengths, dst = fine grid, which the caller
 * zeroes; interp: src = fine grid, dst = values); nfx_batch_launch runs ONE
 * persistent launch over the (problem, bin tile) work queue of all problems.
 * The table stays valid while the problems' buffers do, so the launches can be
 * captured in a CUDA graph and replayed.  nfx_batch_deconv_* do the same for
 * the deconvolution passes (pad = 0: shuffle/crop after a type-1 FFT; pad = 1:
 * zero-pad before a type-2 FFT); nf / n_modes are 3 ints per problem and fac 3
 * pointers per problem; *total (work units: row segments of the problems'
 * outputs) is what nfx_batch_deconv takes. */
typedef struct nfx_batch_problem {
  int64_t M;
  const void* x;
  const void* y;
  const void* z;
  int nf[3];
  int tile[3];         /* 0 = default */
  int max_subproblem;  /* 0 = default */
  int interp_mode;     /* NFX_PER_POINT_*, this problem's interpolation (0 = common's) */
  void* workspace;     /* sort workspace of nfx_sort_workspace_bytes for this problem */
  size_t workspace_bytes;
  const void* src;
  void* dst;
} nfx_batch_problem;

typedef struct nfx_batch_info {
  size_t table_bytes;  /* device table size for nfx_batch_upload */
  size_t smem_bytes;   /* shared memory of the batched launch */
  int64_t max_subs;    /* bound on the work-queue length */
} nfx_batch_info;

int nfx_batch_info_get(const nfx_opts* common, int spread, const nfx_batch_problem* probs, int nprob,
                       nfx_batch_info* info);
int nfx_batch_upload(const nfx_opts* common, int spread, const nfx_batch_problem* probs, int nprob, void* dev_table,
                     size_t table_bytes, void* stream);
int nfx_batch_sort(const nfx_opts* common, const nfx_batch_problem* probs, int nprob, void* stream);
int nfx_batch_launch(const nfx_opts* common, int spread, const void* dev_table, int nprob, const nfx_batch_info* info,
                     void* stream);
size_t nfx_batch_deconv_table_bytes(int precision, int nprob);
int nfx_batch_deconv_upload(int precision, int dim, int pad, const int* nf, const int* n_modes,
                            const void* const* fac, const void* const* src, void* const* dst, int nprob,
                            void* dev_table, size_t table_bytes, int64_t* total, void* stream);
int nfx_batch_deconv(int precision, int pad, const void* dev_table, int nprob, int64_t total, void* stream);

/* ---- type 3 helpers (nufftax/transforms/nufft3.py:216-515) -------------------
 * nfx_t3_prepare: from source coordinates (dim arrays of M) and target
 *   frequencies (dim arrays of K) computes, on the device and without a host
 *   round trip, the centres C, D, half-widths S and scales gamma, h per axis
 *   (nufft3.py:268-281) into `params` (a device buffer of nfx_t3_params_bytes();
 *   computed in the working precision in the reference's order, so that
 *   complex64 inputs get the reference's float32 rescaled coordinates),
 *   then writes the rescaled folded sources xn_d = mod((x_d - C_d)/gamma_d + pi,
 *   2 pi) - pi, the pre-phased strengths c' = c e^{i isign sum_d D_d x_d}
 *   (n_trans x M), the rescaled folded targets sn_d = mod(h_d gamma_d (s_d - D_d)
 *   + pi, 2 pi) - pi, and the per-target output factor
 *   e^{i isign sum_d (s_d - D_d) C_d} / prod_d phihat(h_d gamma_d (s_d - D_d))
 *   (nufft3.py:176-213, 390-394).  nf[d] is the type-3 grid per axis.
 * nfx_t3_finish: out[t][k] *= factor[k]. */
/* ---- a wave of independent type-1 / type-2 transforms in one call -------------
 * No counterpart in the reference.  For serving loops: n problems of one
 * precision, dimension and kernel (`common`; its nf / tile / max_subproblem are
 * ignored, each item has its own grid), each a type 1 (in: M strengths, out:
 * n_modes modes in CMCL order) or a type 2 (in: modes, out: M values), one
 * transform each, are enqueued on `stream` as: one zero-pad launch for every
 * type-2 problem, their FFTs, every problem's sort, ONE persistent spread over
 * the bin tiles of all type-1 problems, ONE persistent interpolation over those
 * of all type-2 problems, the type-1 FFTs and one crop launch for all of them.
 * fac[d]: the problem's deconvolution factors (as nfx_deconv_*); fw: its fine
 * grid buffer; workspace: its sort workspace (nfx_sort_workspace_bytes with
 * its nf and default tiles, max_subproblem 0).  The problem table is built in `host_staging` (pinned host memory of
 * nfx_wave_table_bytes) and copied to `dev_table` asynchronously: both must stay
 * untouched until the wave's work on the stream is done.  The FFTs use the
 * stream's cuFFT work area (as nfx_fft), so a capturing stream is refused. */
typedef struct nfx_wave_item {
  int kind;              /* 1 or 2 */
  int64_t M;
  const void* x;
  const void* y;
  const void* z;
  int nf[3];             /* fine grid per axis; unused axes 1 */
  int n_modes[3];        /* modes per axis; unused axes 1 */
  int fft_sign;          /* +1 or -1, as nfx_fft */
  const void* fac[3];
  const void* in;
  void* out;
  void* fw;
  void* workspace;
  size_t workspace_bytes;
} nfx_wave_item;

int nfx_wave_table_bytes(const nfx_opts* common, const nfx_wave_item* items, int n, size_t* table_bytes);
int nfx_wave(const nfx_opts* common, const nfx_wave_item* items, int n, void* dev_table, void* host_staging,
             size_t table_bytes, void* stream);

/* ---- type 3 in one call ------------------------------------------------------
 * The whole of nufftax/transforms/nufft3.py:216-515 with its pre- and
 * post-processing fused into the passes: the source sort applies the rescaling
 * x' = mod((x - C)/gamma + pi, 2 pi) - pi on the fly and stores each point's
 * pre-phase e^{i isign sum_d D_d x_d}, which the spread multiplies into the
 * strength; the inner type 2 (deconvolve + zero-pad of the fine grid as modes,
 * FFT) follows; the target sort applies s' = (h gamma)(s - D) and stores
 * each target's factor e^{i isign sum_d (s_d - D_d) C_d} / prod_d phihat(s'_d),
 * which the interpolation multiplies into the value it writes.  The scalars
 * are computed on the device in the working precision (no host round trip).
 * opts: precision, dim, kernel (nspread, beta, kc) and nf = the type-3 grid
 * per axis (compute_type3_grid_size*); tile / max_subproblem apply to the
 * source sort; prenorm is ignored.  nf_inner[d] = the inner type 2's grid
 * (compute_grid_size(nf[d], upsampfac, nspread)); fac1..fac3 its
 * deconvolution factors for nf[d] modes on nf_inner[d] (as nfx_deconv_pad).
 * src / tgt: dim device arrays of M sources and K targets; c: n_trans x M;
 * out: n_trans x K.  The workspace (nfx_nufft3_workspace_bytes) holds
 * everything, the FFT's work area included, so the call can be captured in a
 * CUDA graph.  M >= 1. */
int nfx_nufft3_workspace_bytes(const nfx_opts* opts, const int nf_inner[3], int64_t M, int64_t K, int n_trans,
                               size_t* bytes);
int nfx_nufft3(const nfx_opts* opts, const int nf_inner[3], double upsampfac, int isign, const void* const* src,
               int64_t M, const void* c, int n_trans, const void* const* tgt, int64_t K, const void* fac1,
               const void* fac2, const void* fac3, void* out, void* workspace, size_t workspace_bytes, void* stream);

size_t nfx_t3_params_bytes(void);
int nfx_t3_prepare(int precision, int dim, const int nf[3], int nspread, double beta, double kc, double upsampfac,
                   int isign, const void* const* src, int64_t M, const void* c, int n_trans, const void* const* tgt,
                   int64_t K, void* params, void* const* src_out, void* c_out, void* const* tgt_out, void* factor,
                   void* scratch, size_t scratch_bytes, void* stream);
size_t nfx_t3_scratch_bytes(int precision, int64_t M, int64_t K);
int nfx_t3_finish(int precision, const void* factor, int64_t K, int n_trans, void* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NFX_H */
