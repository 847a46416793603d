// Shared device helpers for the nufftax_b200 CUDA library (sm_100a).
//
// Coordinate folding is written with explicitly rounded intrinsics so that no
// multiply-add is ever contracted: the integer cell and bin indices derived from
// it are bit-identical to a CPU evaluation of the same float operations
// (nufftax/core/spread.py:78-97 fold_rescale, nufftax/transforms/nufft1.py:71
// jnp.mod(x + pi, 2 pi) - pi, nufftax/core/spread.py:214 i0 = ceil(xs - ns/2)).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace nfx {

template <typename T> struct C2;
template <> struct C2<float> { using type = float2; };
template <> struct C2<double> { using type = double2; };
template <typename T> using cplx_t = typename C2<T>::type;

// ---- explicitly rounded arithmetic (no FMA contraction) -------------------
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float t_floor(float a) { return floorf(a); }
__device__ __forceinline__ double t_floor(double a) { return floor(a); }
__device__ __forceinline__ float t_fmod(float a, float b) { return fmodf(a, b); }
__device__ __forceinline__ double t_fmod(double a, double b) { return fmod(a, b); }
__device__ __forceinline__ int ceil_to_int(float a) { return __float2int_ru(a); }
__device__ __forceinline__ int ceil_to_int(double a) { return __double2int_ru(a); }
__device__ __forceinline__ float t_exp(float a) { return expf(a); }
__device__ __forceinline__ double t_exp(double a) { return exp(a); }
__device__ __forceinline__ float t_sqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ double t_sqrt(double a) { return sqrt(a); }

// Constants rounded to the working type the way JAX weak typing rounds Python
// floats: the double value first, then one conversion.
constexpr double kPi = 3.141592653589793;
constexpr double kTwoPi = 2.0 * 3.141592653589793;
constexpr double kInvTwoPi = 1.0 / (2.0 * 3.141592653589793);

// jnp.mod(x + pi, 2 pi) - pi: lax.rem (exact fmod) plus the sign fix of
// jnp.remainder (add the divisor when the remainder is negative and non-zero).
// For 0 <= x + pi < 2 pi the remainder is x + pi itself (fmod is exact), which
// skips the slow general fmod for the common in-range inputs.
template <typename T>
__device__ __forceinline__ T premod(T x) {
  const T pi = (T)kPi;
  const T two_pi = (T)kTwoPi;
  T a = rn_add(x, pi);
  T r;
  if (a >= (T)0 && a < two_pi) {
    r = a;
  } else {
    r = t_fmod(a, two_pi);
    if (r != (T)0 && r < (T)0) r = rn_add(r, two_pi);
  }
  return rn_sub(r, pi);
}

// fold_rescale: ((x * (1/2pi) + 0.5) - floor(.)) * nf, one rounding per op.
template <typename T>
__device__ __forceinline__ T fold_rescale(T x, int nf) {
  T t = rn_mul(x, (T)kInvTwoPi);
  t = rn_add(t, (T)0.5);
  t = rn_sub(t, t_floor(t));
  return rn_mul(t, (T)nf);
}

template <typename T>
__device__ __forceinline__ T scaled_coord(T x, int nf, int prenorm) {
  return fold_rescale(prenorm ? premod(x) : x, nf);
}

// Left cell of the footprint: i0 = ceil(xs - ns/2).
template <typename T, int NS>
__device__ __forceinline__ int left_cell(T xs) {
  return ceil_to_int(rn_sub(xs, (T)(NS / 2)));
}

// Periodic wrap of any int into [0, n); one compare-and-add for indices within
// one period of the grid (the footprint's left cell always is), % otherwise.
__device__ __forceinline__ int wrap_index(int i, int n) {
  if (i >= 0 && i < n) return i;
  if (i < 0 && i >= -n) return i + n;
  if (i >= n && i - n < n) return i - n;
  int r = i % n;
  return r < 0 ? r + n : r;
}

// ES kernel value phi(z) = exp(beta (sqrt(1 - c z^2) - 1)), zero where the
// argument is negative (nufftax/core/kernel.py:79-111; arg = 1 - (c z) z).
template <typename T>
__device__ __forceinline__ T es_weight(T z, T beta, T kc) {
  T arg = (T)1 - (kc * z) * z;
  T w = t_exp(beta * (t_sqrt(arg > (T)0 ? arg : (T)0) - (T)1));
  return arg >= (T)0 ? w : (T)0;
}

// phi and dphi/dz (nufftax/core/kernel.py:114-162; dphi masked where arg <= 1e-14).
template <typename T>
__device__ __forceinline__ void es_weight_deriv(T z, T beta, T kc, T& phi, T& dphi) {
  const T tiny = (T)1e-14;
  T arg = (T)1 - (kc * z) * z;
  T sq = t_sqrt(arg > tiny ? arg : tiny);
  T w = t_exp(beta * (sq - (T)1));
  phi = arg >= (T)0 ? w : (T)0;
  T d = -beta * kc * z / sq * phi;
  dphi = arg > tiny ? d : (T)0;
}

// Vectorised global reduction of a complex64 value (one 8-byte red).
__device__ __forceinline__ void red_add(float2* addr, float2 v) {
  asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(addr), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void red_add(double2* addr, double2 v) {
  atomicAdd(&addr->x, v.x);
  atomicAdd(&addr->y, v.y);
}

// Paired FMA: (a.x * b.x + c.x, a.y * b.y + c.y), each rounded once to
// nearest.  float uses Blackwell's fma.rn.f32x2 (one instruction, the same
// results as two fmaf) on 64-bit register pairs; the packing is plain C++ so
// the compiler can keep pairs in adjacent registers and hoist it out of loops.
// double is two fma.
__device__ __forceinline__ unsigned long long pack2(float2 v) {
  return (unsigned long long)__float_as_uint(v.x) | ((unsigned long long)__float_as_uint(v.y) << 32);
}
__device__ __forceinline__ float2 unpack2(unsigned long long v) {
  return make_float2(__uint_as_float((unsigned)v), __uint_as_float((unsigned)(v >> 32)));
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(pack2(a)), "l"(pack2(b)), "l"(pack2(c)));
  return unpack2(d);
}
__device__ __forceinline__ double2 fma2(double2 a, double2 b, double2 c) {
  double2 d;
  d.x = fma(a.x, b.x, c.x);
  d.y = fma(a.y, b.y, c.y);
  return d;
}
// c + s * v for a real s and a complex v.
__device__ __forceinline__ float2 fma_rc(float s, float2 v, float2 c) { return fma2(make_float2(s, s), v, c); }
__device__ __forceinline__ double2 fma_rc(double s, double2 v, double2 c) { return fma2(make_double2(s, s), v, c); }
// (s, s) as a complex-typed pair, for a real weight used with many values.
__device__ __forceinline__ float2 splat2(float s) { return make_float2(s, s); }
__device__ __forceinline__ double2 splat2(double s) { return make_double2(s, s); }

// Polynomial form of the ES weights of one footprint (float path).  For a point
// at scaled coordinate xs with left cell i0, every weight phi(i0 + q - xs),
// q = 0..ns-1, is a smooth function of v = 2 (xs - i0) - (ns - 1) in (-1, 1];
// a[q][d] are monomial coefficients in v fitted on the host (nfx_es_poly) to
// within about two float ulps of the exp/sqrt form; a[ns - 1 - q] is a[q] at
// -v (phi is even: odd coefficients negated).  The kernels evaluate degree
// kPolyEvalDeg (coefficients above the fitted degree are zero, which leaves
// the result unchanged), a whole footprint's weights as even / odd splits
// E(v^2) +- v O(v^2) of the first ns / 2 polynomials, single weights by
// Horner's rule; widths whose weights need a higher degree keep the exp/sqrt
// form.
constexpr int kPolyMaxDeg = 15;
constexpr int kPolyEvalDeg = 7;
struct EsPoly {
  float a[16][kPolyMaxDeg + 1];
  int deg;  // 0 = not used (exp/sqrt form)
};

// Exact division of a non-negative int n < 2^31 by a fixed divisor d >= 1 as a
// multiply-high and a shift: with p = 31 + ceil(log2 d) and m = ceil(2^p / d)
// (which fits in 32 bits), n * m / 2^p = n / d + n e / (d 2^p) for some
// 0 <= e < d, and the second term is below 1/d, so the floor is n / d.
// d = 1 is marked by shr = -1 (quotient n).
struct FastDiv {
  unsigned mul;
  int shr;  // p - 32, or -1 for d = 1
};
inline FastDiv make_fastdiv(int d) {
  FastDiv f;
  if (d <= 1) {
    f.mul = 0;
    f.shr = -1;
    return f;
  }
  int l = 0;
  while ((1ll << l) < d) ++l;
  const int p = 31 + l;
  f.mul = (unsigned)((((unsigned long long)1 << p) + (unsigned long long)d - 1) / (unsigned long long)d);
  f.shr = p - 32;
  return f;
}
__device__ __forceinline__ int fast_div(int n, FastDiv f) {
  return f.shr < 0 ? n : (int)(__umulhi((unsigned)n, f.mul) >> f.shr);
}

// Type-3 scalars per axis (nufftax/transforms/nufft3.py:258-268, 354-362),
// computed on the device: source centre C, target centre D, target half-width
// S, scale gamma = nf / (2 upsampfac S) and h = 2 pi / nf.  Values of the
// working type stored as doubles.
struct T3Params {
  double C[3], D[3], S[3], gamma[3], h[3];
};

// Grid geometry shared by the sort, spread and interp kernels (plain values).
struct Geom {
  int dim;
  int nf[3];     // fine grid per axis (x, y, z); unused axes are 1
  int tile[3];   // bin edge in cells per axis; unused axes are 1
  int nb[3];     // bins per axis
  int pad[3];    // padded tile extent (tile + ns - 1) per axis; 1 for unused
  int pitch;     // shared-memory row pitch along x (>= pad[0])
  int nbins;
  int prenorm;
  int spread_mode;  // nfx_opts::spread_mode (threads per point of the spread)
  int interp_mode;  // nfx_opts::interp_mode (threads per point of the interpolation)
  FastDiv tdiv[3];  // division by tile[d]
  // Type 3 fused into the sort (0: off).  1: the points are type-3 sources,
  // rescaled as x' = mod((x - C) / gamma + pi, 2 pi) - pi before the fold, and
  // the sort writes each point's pre-phase e^{i isign sum_d D_d x_d};
  // 2: type-3 targets, s' = (h gamma)(s - D) folded into [-pi, pi), and the
  // sort writes each point's output factor e^{i isign sum_d (s_d - D_d) C_d} /
  // prod_d phihat(s'_d).  t3 points at the device T3Params.
  int t3_mode;
  int t3_isign;
  double t3_beta, t3_kc;
  const T3Params* t3;
};

// The type-3 rescaling of one coordinate, in the working type and in the
// reference's order (nufft3.py:271-272, 287-288, 365-366, 381-384).
template <typename T>
__device__ __forceinline__ T t3_rescaled(T x, int d, const Geom& g) {
  const T3Params* p = g.t3;
  if (g.t3_mode == 1) return rn_sub(x, (T)p->C[d]) / (T)p->gamma[d];
  return rn_mul(rn_mul((T)p->h[d], (T)p->gamma[d]), rn_sub(x, (T)p->D[d]));
}

// Folded grid coordinate of axis d of a point (the value every pass and the
// bin keys use): the type-3 rescaling and its pre-normalisation when enabled,
// then the transforms' pre-normalisation (prenorm) and fold_rescale.
template <typename T>
__device__ __forceinline__ T point_fold(T x, int d, const Geom& g) {
  if (g.t3_mode != 0) x = premod(t3_rescaled(x, d, g));
  return scaled_coord(x, g.nf[d], g.prenorm);
}

}  // namespace nfx
