// init.cuh -- initial velocity fields generated on the device, so that a run
// (or every run of an ensemble) starts without moving n^3 host fields:
//
//   Taylor-Green, as tgv.py:14-27 writes it:
//     U = sin x cos y cos z,  V = -cos x sin y cos z,  W = 0,  x_i = i * (2 pi / n)
//     formed from the 1-D tables s_i = sin(x_i), c_i = cos(x_i) as
//     (s_i c_j) c_k and (-c_i s_j) c_k, the order numpy's einsum('i,j,k')
//     multiplies in, so the field is bit-identical to tgv.py's given the
//     same tables;
//   a seeded solenoidal perturbation with energy spectrum
//     E(k) ~ k^4 exp(-2 (k/k0)^2): white Gaussian noise in real space, r2c,
//     amplitude |k| exp(-(|k|/k0)^2) per mode (= sqrt(E(k)) / k), no content
//     on the Nyquist planes, projection onto k-perpendicular, c2r / n^3,
//     scaled to unit rms; added to Taylor-Green with rms = amplitude times
//     the rms of the Taylor-Green field.
//
// The noise comes from a counter-based generator, so any point of any
// stream is computed independently of the others: the SplitMix64 output
// function (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014) applied to key + (i + 1) * golden, and the
// Box-Muller transform (cosine branch) of two 53-bit uniforms per normal.
#pragma once
#include "kernels.cuh"

namespace dnsb {

constexpr unsigned long long GOLDEN64 = 0x9E3779B97F4A7C15ull;  // 2^64 / golden ratio

__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// key of the stream of velocity component `field` for a seed
__host__ __device__ __forceinline__ unsigned long long stream_key(unsigned long long seed, int field) {
  return mix64(seed * GOLDEN64 + (unsigned long long)(field + 1));
}
// standard normal number `idx` of a stream
__device__ __forceinline__ double counter_normal(unsigned long long key, unsigned long long idx) {
  const unsigned long long a = mix64(key + (2 * idx + 1) * GOLDEN64);
  const unsigned long long b = mix64(key + (2 * idx + 2) * GOLDEN64);
  const double u1 = (double)((a >> 11) + 1) * 0x1.0p-53;  // (0, 1]
  const double u2 = (double)(b >> 11) * 0x1.0p-53;        // [0, 1)
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

// Gaussian white noise into the three real slots [3][n^3] of one run
template <class R>
__global__ void k_noise3(R *__restrict__ out, long long nreal, unsigned long long seed) {
  const long long total = 3 * nreal;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(q / nreal);
    out[q] = (R)counter_normal(stream_key(seed, f), (unsigned long long)(q - f * nreal));
  }
}

// Spectral shaping of three slots in place: amplitude |k| exp(-(|k|/k0)^2),
// zero on the planes |kx| = n/2, |ky| = n/2, kz = n/2, then the projection
// u -= k (k . u) / |k|^2.  Arithmetic in FP64.
template <class C>
__global__ void k_shape_project(C *__restrict__ u, Geo g, double k0) {
  const long long per = (long long)g.n * g.n * g.nf;
  const int h = g.n / 2;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < per;
       q += (long long)gridDim.x * blockDim.x) {
    const long long row = q / g.nf;
    const int k = (int)(q - row * g.nf);
    const int i = (int)(row / g.n), j = (int)(row % g.n);
    const int ikx = kwave(i, g.n), iky = kwave(j, g.n);
    const double kx = ikx, ky = iky, kz = k;
    const double kk = __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
    const double km = sqrt(kk);
    const double r = __ddiv_rn(km, k0);
    double amp = km > 0 ? __dmul_rn(km, exp(-__dmul_rn(r, r))) : 0.0;
    if (ikx == -h || iky == -h || k == h) amp = 0.0;
    const long long l = row * g.nfp + k;
    double2 a[3];
#pragma unroll
    for (int f = 0; f < 3; f++) {
      const double2 v = to_d(u[f * g.slot + l]);
      a[f] = make_double2(__dmul_rn(v.x, amp), __dmul_rn(v.y, amp));
    }
    const double den = kk > 0 ? kk : 1.0;
    const double dr = __ddiv_rn(
        __dadd_rn(__dadd_rn(__dmul_rn(kx, a[0].x), __dmul_rn(ky, a[1].x)), __dmul_rn(kz, a[2].x)), den);
    const double di = __ddiv_rn(
        __dadd_rn(__dadd_rn(__dmul_rn(kx, a[0].y), __dmul_rn(ky, a[1].y)), __dmul_rn(kz, a[2].y)), den);
    const double kf[3] = {kx, ky, kz};
#pragma unroll
    for (int f = 0; f < 3; f++)
      u[f * g.slot + l] = from_d<C>(make_double2(__dsub_rn(a[f].x, __dmul_rn(kf[f], dr)),
                                                 __dsub_rn(a[f].y, __dmul_rn(kf[f], di))));
  }
}

// sum of squares of `count` doubles (double-double), block partials into
// partial[blockIdx.x]; k_diag_final combines them (the .z/.w pair unused)
template <int BS>
__global__ void __launch_bounds__(BS)
    k_sumsq(const double *__restrict__ x, long long count, double4 *__restrict__ partial) {
  DD e{0.0, 0.0}, o{0.0, 0.0};
  for (long long q = (long long)blockIdx.x * BS + threadIdx.x; q < count;
       q += (long long)gridDim.x * BS)
    e = dd_add_d(e, __dmul_rn(x[q], x[q]));
  dd_block_reduce<BS>(e, o, partial + blockIdx.x);
}

// Taylor-Green from the tables tab = [s_0..s_{n-1}, c_0..c_{n-1}] into the
// three real slots (storage R), optionally plus scale * delta / rms with
// delta [3][n^3] float64 (the perturbation before its unit-rms scaling)
// (out may be delta itself: each point is read before it is written)
template <class R>
__global__ void k_tgv_fill(R *out, const double *__restrict__ tab, const double *delta, double rms,
                           double scale, int n) {
  const long long nreal = (long long)n * n * n;
  const double *s = tab, *c = tab + n;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < 3 * nreal;
       q += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(q / nreal);
    const long long p = q - f * nreal;
    const int i = (int)(p / ((long long)n * n)), j = (int)((p / n) % n), k = (int)(p % n);
    double v;
    if (f == 0)
      v = __dmul_rn(__dmul_rn(s[i], c[j]), c[k]);
    else if (f == 1)
      v = __dmul_rn(__dmul_rn(-c[i], s[j]), c[k]);
    else
      v = 0.0;
    if (delta) v = __dadd_rn(v, __dmul_rn(scale, __ddiv_rn(delta[q], rms)));
    out[q] = (R)v;
  }
}

}  // namespace dnsb
