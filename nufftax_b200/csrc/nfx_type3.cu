// Type-3 (non-uniform to non-uniform) pre/post-processing, fused per point.
//
// nufftax/transforms/nufft3.py:216-515 computes, per axis d, the source centre
// C_d, target centre D_d and half-width S_d from min/max reductions, the scale
// gamma_d = nf_d / (2 sigma S_d) and h_d = 2 pi / nf_d; it pre-phases the
// strengths, spreads at the rescaled folded sources, runs an inner type 2 at the
// rescaled folded targets and divides by phihat(s'_d) (20+-node trapezoid,
// nufft3.py:176-213) with a phase correction.  Here the reductions and the
// scalar set-up stay on the device (no host round trip, so the whole type 3 can
// be captured in a CUDA graph) and each of the per-point passes is one kernel.
#include <string>

#include "nfx.h"
#include "nfx_internal.h"

namespace nfx {

constexpr int kT3Blocks = 256;

template <typename T>
__global__ void k_minmax(const T* __restrict__ a, int64_t n, double* __restrict__ partial) {
  __shared__ double s_min[32], s_max[32];
  double mn = 1e300, mx = -1e300;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = (double)a[i];
    mn = v < mn ? v : mn;
    mx = v > mx ? v : mx;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    s_min[w] = mn;
    s_max[w] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) {
      mn = fmin(mn, s_min[i]);
      mx = fmax(mx, s_max[i]);
    }
    partial[2 * blockIdx.x] = mn;
    partial[2 * blockIdx.x + 1] = mx;
  }
}

// partial: [2*dim arrays][kT3Blocks][2]; arrays 0..dim-1 sources, dim..2dim-1 targets.
// The scalars are computed in the working type T in the reference's order
// (nufft3.py:258-268, 354-362), with the Python constants rounded to T first
// as JAX's weak typing does: C = (min + max) / 2, S = max((max - min) / 2,
// 1e-10), gamma = nf / ((2 upsampfac) S); h = 2 pi / nf stays a double (it is a
// Python float there) and is rounded to T where it meets a T array.  The mins
// and maxes are values of T, so every result is exactly the reference's.
template <typename T>
__global__ void k_t3_params(const double* __restrict__ partial, int dim, int nf0, int nf1, int nf2,
                            double upsampfac, T3Params* __restrict__ p) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int nf[3] = {nf0, nf1, nf2};
  for (int d = 0; d < dim; ++d) {
    T mn[2], mx[2];
    for (int s = 0; s < 2; ++s) {
      const double* q = partial + (size_t)(s * dim + d) * kT3Blocks * 2;
      double a = 1e300, b = -1e300;
      for (int i = 0; i < kT3Blocks; ++i) {
        a = fmin(a, q[2 * i]);
        b = fmax(b, q[2 * i + 1]);
      }
      mn[s] = (T)a;
      mx[s] = (T)b;
    }
    const T C = rn_add(mn[0], mx[0]) / (T)2.0;
    const T D = rn_add(mn[1], mx[1]) / (T)2.0;
    const T half = rn_sub(mx[1], mn[1]) / (T)2.0;
    const T S = half > (T)1e-10 ? half : (T)1e-10;
    p->C[d] = (double)C;
    p->D[d] = (double)D;
    p->S[d] = (double)S;
    p->h[d] = 2.0 * kPi / nf[d];
    p->gamma[d] = (double)((T)nf[d] / rn_mul((T)(2.0 * upsampfac), S));
  }
}

template <typename T>
__global__ void k_t3_sources(int dim, const T* __restrict__ x0, const T* __restrict__ x1, const T* __restrict__ x2,
                             int64_t M, const cplx_t<T>* __restrict__ c, int n_trans, int isign,
                             const T3Params* __restrict__ p, T* __restrict__ o0, T* __restrict__ o1,
                             T* __restrict__ o2, cplx_t<T>* __restrict__ cout) {
  const T* xs[3] = {x0, x1, x2};
  T* os[3] = {o0, o1, o2};
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < M; j += (int64_t)gridDim.x * blockDim.x) {
    double phase = 0.0;
    for (int d = 0; d < dim; ++d) {
      const T x = xs[d][j];
      // x' = (x - C) / gamma in T (nufft3.py:271, 365-366)
      const T r = rn_sub(x, (T)p->C[d]) / (T)p->gamma[d];
      os[d][j] = premod(r);
      phase += p->D[d] * (double)x;
    }
    phase *= (double)isign;
    double sn, cs;
    sincos(phase, &sn, &cs);
    for (int t = 0; t < n_trans; ++t) {
      const cplx_t<T> v = c[(int64_t)t * M + j];
      cplx_t<T> o;
      o.x = (T)((double)v.x * cs - (double)v.y * sn);
      o.y = (T)((double)v.x * sn + (double)v.y * cs);
      cout[(int64_t)t * M + j] = o;
    }
  }
}

template <typename T>
__global__ void k_t3_targets(int dim, const T* __restrict__ s0, const T* __restrict__ s1, const T* __restrict__ s2,
                             int64_t K, int isign, int nspread, double beta, double kc,
                             const T3Params* __restrict__ p, T* __restrict__ o0, T* __restrict__ o1,
                             T* __restrict__ o2, cplx_t<T>* __restrict__ factor) {
  const T* ss[3] = {s0, s1, s2};
  T* os[3] = {o0, o1, o2};
  // trapezoid nodes on [-ns/2, ns/2] (nufft3.py:198-207)
  const double j2 = nspread / 2.0;
  const int nq = max((int)(4 + 3.0 * j2), 20);
  const double dz = 2.0 * j2 / (nq - 1);
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
    double phase = 0.0, phi_prod = 1.0;
    for (int d = 0; d < dim; ++d) {
      const T s = ss[d][k];
      // s' = (h gamma) (s - D) in T, in the reference's order (nufft3.py:287, 381-382)
      const T r = rn_mul(rn_mul((T)p->h[d], (T)p->gamma[d]), rn_sub(s, (T)p->D[d]));
      os[d][k] = premod(r);
      const double sr = (double)r;
      double acc = 0.0;
      for (int q = 0; q < nq; ++q) {
        const double z = -j2 + q * dz;
        const double arg = 1.0 - kc * z * z;
        const double phi = arg >= 0.0 ? exp(beta * (sqrt(arg > 0.0 ? arg : 0.0) - 1.0)) : 0.0;
        const double w = (q == 0 || q == nq - 1) ? dz / 2 : dz;
        acc += phi * w * cos(sr * z);
      }
      phi_prod *= acc;
      phase += ((double)s - p->D[d]) * p->C[d];
    }
    phase *= (double)isign;
    double sn, cs;
    sincos(phase, &sn, &cs);
    cplx_t<T> f;
    f.x = (T)(cs / phi_prod);
    f.y = (T)(sn / phi_prod);
    factor[k] = f;
  }
}

template <typename T>
__global__ void k_t3_finish(const cplx_t<T>* __restrict__ factor, int64_t K, int n_trans, cplx_t<T>* __restrict__ out) {
  const int64_t total = K * n_trans;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const cplx_t<T> f = factor[i % K];
    const cplx_t<T> v = out[i];
    cplx_t<T> o;
    o.x = v.x * f.x - v.y * f.y;
    o.y = v.x * f.y + v.y * f.x;
    out[i] = o;
  }
}

static unsigned ew_grid(int64_t n) {
  int64_t want = (n + 255) / 256;
  int64_t cap = (int64_t)num_sms() * 8;
  return (unsigned)(want < cap ? (want > 0 ? want : 1) : cap);
}

size_t t3_scratch_bytes() { return (size_t)6 * kT3Blocks * 2 * sizeof(double); }

template <typename T>
cudaError_t launch_t3_params(int dim, const int nf[3], double upsampfac, const void* const* src, int64_t M,
                             const void* const* tgt, int64_t K, T3Params* params, void* scratch, cudaStream_t st) {
  double* partial = (double*)scratch;
  for (int d = 0; d < dim; ++d) {
    k_minmax<T><<<kT3Blocks, 256, 0, st>>>((const T*)src[d], M, partial + (size_t)d * kT3Blocks * 2);
    k_minmax<T><<<kT3Blocks, 256, 0, st>>>((const T*)tgt[d], K, partial + (size_t)(dim + d) * kT3Blocks * 2);
  }
  k_t3_params<T><<<1, 32, 0, st>>>(partial, dim, nf[0], dim > 1 ? nf[1] : 1, dim > 2 ? nf[2] : 1, upsampfac,
                                   params);
  return cudaGetLastError();
}

template cudaError_t launch_t3_params<float>(int, const int*, double, const void* const*, int64_t,
                                             const void* const*, int64_t, T3Params*, void*, cudaStream_t);
template cudaError_t launch_t3_params<double>(int, const int*, double, const void* const*, int64_t,
                                              const void* const*, int64_t, T3Params*, void*, cudaStream_t);

template <typename T>
static cudaError_t t3_prepare(int dim, const int nf[3], int nspread, double beta, double kc, double upsampfac,
                              int isign, const void* const* src, int64_t M, const void* c, int n_trans,
                              const void* const* tgt, int64_t K, void* params, void* const* src_out, void* c_out,
                              void* const* tgt_out, void* factor, void* scratch, cudaStream_t st) {
  cudaError_t e = launch_t3_params<T>(dim, nf, upsampfac, src, M, tgt, K, (T3Params*)params, scratch, st);
  if (e != cudaSuccess) return e;
  const T* s3[3] = {nullptr, nullptr, nullptr};
  const T* t3[3] = {nullptr, nullptr, nullptr};
  T* so[3] = {nullptr, nullptr, nullptr};
  T* to[3] = {nullptr, nullptr, nullptr};
  for (int d = 0; d < dim; ++d) {
    s3[d] = (const T*)src[d];
    t3[d] = (const T*)tgt[d];
    so[d] = (T*)src_out[d];
    to[d] = (T*)tgt_out[d];
  }
  if (M > 0)
    k_t3_sources<T><<<ew_grid(M), 256, 0, st>>>(dim, s3[0], s3[1], s3[2], M, (const cplx_t<T>*)c, n_trans, isign,
                                                (const T3Params*)params, so[0], so[1], so[2], (cplx_t<T>*)c_out);
  if (K > 0)
    k_t3_targets<T><<<ew_grid(K), 256, 0, st>>>(dim, t3[0], t3[1], t3[2], K, isign, nspread, beta, kc,
                                                (const T3Params*)params, to[0], to[1], to[2],
                                                (cplx_t<T>*)factor);
  return cudaGetLastError();
}

}  // namespace nfx

using namespace nfx;

extern "C" {

size_t nfx_t3_params_bytes(void) { return sizeof(T3Params); }

size_t nfx_t3_scratch_bytes(int precision, int64_t M, int64_t K) {
  (void)precision;
  (void)M;
  (void)K;
  return t3_scratch_bytes();
}

int nfx_t3_prepare(int precision, int dim, const int nf[3], int nspread, double beta, double kc, double upsampfac,
                   int isign, const void* const* src, int64_t M, const void* c, int n_trans, const void* const* tgt,
                   int64_t K, void* params, void* const* src_out, void* c_out, void* const* tgt_out, void* factor,
                   void* scratch, size_t scratch_bytes, void* stream) {
  if ((precision != NFX_F32 && precision != NFX_F64) || dim < 1 || dim > 3 || nf == nullptr || src == nullptr ||
      tgt == nullptr || src_out == nullptr || tgt_out == nullptr || params == nullptr || factor == nullptr ||
      n_trans < 1 || M < 1 || K < 0 || (c == nullptr) || c_out == nullptr) {
    set_error("invalid nfx_t3_prepare arguments");
    return NFX_ERR_INVALID;
  }
  for (int d = 0; d < dim; ++d) {
    if (nf[d] < 2 || src[d] == nullptr || tgt[d] == nullptr || src_out[d] == nullptr || tgt_out[d] == nullptr) {
      set_error("invalid nfx_t3_prepare axis arguments");
      return NFX_ERR_INVALID;
    }
  }
  if (scratch == nullptr || scratch_bytes < nfx_t3_scratch_bytes(precision, M, K)) {
    set_error("t3 scratch too small");
    return NFX_ERR_WORKSPACE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = precision == NFX_F32
                      ? t3_prepare<float>(dim, nf, nspread, beta, kc, upsampfac, isign, src, M, c, n_trans, tgt, K,
                                          params, src_out, c_out, tgt_out, factor, scratch, st)
                      : t3_prepare<double>(dim, nf, nspread, beta, kc, upsampfac, isign, src, M, c, n_trans, tgt, K,
                                           params, src_out, c_out, tgt_out, factor, scratch, st);
  if (e != cudaSuccess) {
    set_error(std::string("nfx_t3_prepare: ") + cudaGetErrorString(e));
    return NFX_ERR_CUDA;
  }
  return NFX_OK;
}

int nfx_t3_finish(int precision, const void* factor, int64_t K, int n_trans, void* out, void* stream) {
  if ((precision != NFX_F32 && precision != NFX_F64) || factor == nullptr || out == nullptr || K < 0 || n_trans < 1) {
    set_error("invalid nfx_t3_finish arguments");
    return NFX_ERR_INVALID;
  }
  if (K == 0) return NFX_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = K * n_trans;
  if (precision == NFX_F32)
    k_t3_finish<float><<<ew_grid(n), 256, 0, st>>>((const float2*)factor, K, n_trans, (float2*)out);
  else
    k_t3_finish<double><<<ew_grid(n), 256, 0, st>>>((const double2*)factor, K, n_trans, (double2*)out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("nfx_t3_finish: ") + cudaGetErrorString(e));
    return NFX_ERR_CUDA;
  }
  return NFX_OK;
}

}  // extern "C"
