// fft_core.cuh -- register/shared-memory FFT building blocks for sm_100a.
//
// A line FFT of length L is spread over T = L/E threads; thread t holds
// E values in registers in the "strided" distribution: register e <-> line
// position t + T*e.  Each Stockham autosort stage of radix R (R divides E)
// runs E/R butterflies per thread entirely on its own registers; between
// stages the values are exchanged through shared memory.  After the last
// stage the outputs are again in the strided distribution and in natural
// order, so loads and stores to HBM use the same thread <-> position map.
//
// Conventions (FFTW's, which main.c relies on): forward = exp(-2 pi i jk/L),
// backward = exp(+2 pi i jk/L), no normalisation.
//
// Twiddles come from a table tw[k] = exp(-2 pi i k / n), k in [0, n), of the
// grid size n (generated on the host in long double and rounded once),
// regrouped per stage in shared memory (StageTw).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <utility>

namespace dnsb {

// Complex types: double2 (FP64 path) and float2 (FP32 storage of the mixed
// path).  Every routine below is a template on the complex type C.
template <class R>
struct Cx;
template <>
struct Cx<double> {
  using T = double2;
};
template <>
struct Cx<float> {
  using T = float2;
};
template <class R>
using cx = typename Cx<R>::T;
template <class C>
using sc = decltype(C::x);  // scalar of a complex type

typedef double2 cd;

template <class C>
__device__ __forceinline__ C cmk(sc<C> a, sc<C> b) {
  C r;
  r.x = a;
  r.y = b;
  return r;
}
template <class C>
__device__ __forceinline__ C czero() {
  return cmk<C>(sc<C>(0), sc<C>(0));
}
template <class C>
__device__ __forceinline__ C cadd(C a, C b) { return cmk<C>(a.x + b.x, a.y + b.y); }
template <class C>
__device__ __forceinline__ C csub(C a, C b) { return cmk<C>(a.x - b.x, a.y - b.y); }
template <class C>
__device__ __forceinline__ C cscale(C a, sc<C> s) { return cmk<C>(a.x * s, a.y * s); }
// a * b
template <class C>
__device__ __forceinline__ C cmul(C a, C b) {
  return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <class C>
__device__ __forceinline__ C cmulc(C a, C b) {
  return cmk<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// multiply by the twiddle w (forward table entry) in the given direction
template <bool FWD, class C>
__device__ __forceinline__ C twmul(C a, C w) {
  return FWD ? cmul(a, w) : cmulc(a, w);
}
// widen / narrow between the two complex types
__device__ __forceinline__ double2 to_d(double2 a) { return a; }
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }
template <class C>
__device__ __forceinline__ C from_d(double2 a) {
  return cmk<C>((sc<C>)a.x, (sc<C>)a.y);
}

// cos(2 pi m / 16) and sin(2 pi m / 16) for m in [0, 4]
__host__ __device__ constexpr double c16(int m) {
  return m == 0 ? 1.0
         : m == 1 ? 0.92387953251128675613
         : m == 2 ? 0.70710678118654752440
         : m == 3 ? 0.38268343236508977173
                  : 0.0;
}

// a * exp(-/+ 2 pi i m / 16) with exact handling of the trivial factors; the
// constants are rounded once to the scalar type from the double literals
template <int M, bool FWD, class C>
__device__ __forceinline__ C w16(C a) {
  using S = sc<C>;
  constexpr int m = M & 15;
  if constexpr (m == 0) {
    return a;
  } else if constexpr (m == 8) {
    return cmk<C>(-a.x, -a.y);
  } else if constexpr (m == 4) {  // exp(-i pi/2) = -i
    return FWD ? cmk<C>(a.y, -a.x) : cmk<C>(-a.y, a.x);
  } else if constexpr (m == 12) {  // exp(-3 i pi/2) = +i
    return FWD ? cmk<C>(-a.y, a.x) : cmk<C>(a.y, -a.x);
  } else {
    // cos/sin of 2 pi m / 16 via quadrant symmetry
    constexpr int q = m / 4, r = m % 4;
    constexpr double c0 = c16(r), s0 = c16(4 - r);
    constexpr S c = (S)(q == 0 ? c0 : q == 1 ? -s0 : q == 2 ? -c0 : s0);
    constexpr S s = (S)(q == 0 ? s0 : q == 1 ? c0 : q == 2 ? -s0 : -c0);
    // forward multiplies by (c - i s), backward by (c + i s)
    if constexpr (FWD)
      return cmk<C>(a.x * c + a.y * s, a.y * c - a.x * s);
    else
      return cmk<C>(a.x * c - a.y * s, a.y * c + a.x * s);
  }
}

template <int B, int E, class F, int... I>
__device__ __forceinline__ void static_for_impl(F &&f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, B + I>{}), ...);
}
// calls f(integral_constant<int, i>) for i in [B, E)
template <int B, int E, class F>
__device__ __forceinline__ void static_for(F &&f) {
  static_for_impl<B, E>(f, std::make_integer_sequence<int, E - B>{});
}

// In-register DFT of size R (1, 2, 4, 8, 16), natural order in and out
// (recursive radix-2 decimation in time).
template <int R, bool FWD, class C>
__device__ __forceinline__ void dft(C (&a)[R]) {
  if constexpr (R == 1) {
    return;
  } else if constexpr (R == 2) {
    C t = a[1];
    a[1] = csub(a[0], t);
    a[0] = cadd(a[0], t);
  } else {
    C e[R / 2], o[R / 2];
#pragma unroll
    for (int k = 0; k < R / 2; k++) {
      e[k] = a[2 * k];
      o[k] = a[2 * k + 1];
    }
    dft<R / 2, FWD>(e);
    dft<R / 2, FWD>(o);
    static_for<0, R / 2>([&](auto K) {
      constexpr int k = decltype(K)::value;
      C t = w16<k * (16 / R), FWD>(o[k]);
      a[k] = cadd(e[k], t);
      a[k + R / 2] = csub(e[k], t);
    });
  }
}

// Radix plans.  E = values per thread; radices multiply to L; each radix
// divides E.
template <int L>
struct Plan;
template <> struct Plan<2>   { static constexpr int E = 2,  NS = 1, R0 = 2,  R1 = 1, R2 = 1, R3 = 1; };
template <> struct Plan<4>   { static constexpr int E = 4,  NS = 1, R0 = 4,  R1 = 1, R2 = 1, R3 = 1; };
template <> struct Plan<8>   { static constexpr int E = 8,  NS = 1, R0 = 8,  R1 = 1, R2 = 1, R3 = 1; };
template <> struct Plan<16>  { static constexpr int E = 16, NS = 1, R0 = 16, R1 = 1, R2 = 1, R3 = 1; };
template <> struct Plan<32>  { static constexpr int E = 8,  NS = 2, R0 = 8,  R1 = 4, R2 = 1, R3 = 1; };
template <> struct Plan<64>  { static constexpr int E = 8,  NS = 2, R0 = 8,  R1 = 8, R2 = 1, R3 = 1; };
template <> struct Plan<128> { static constexpr int E = 16, NS = 2, R0 = 16, R1 = 8, R2 = 1, R3 = 1; };
template <> struct Plan<256> { static constexpr int E = 16, NS = 2, R0 = 16, R1 = 16, R2 = 1, R3 = 1; };
template <> struct Plan<512> { static constexpr int E = 16, NS = 3, R0 = 16, R1 = 16, R2 = 2, R3 = 1; };

// Plans for the half-length complex FFT of the z (real) axis, one warp or
// less per line: E <= 8 keeps registers free for the fused pointwise work.
template <int M>
struct ZPlan;
template <> struct ZPlan<4>   { static constexpr int E = 4, NS = 1, R0 = 4, R1 = 1, R2 = 1, R3 = 1; };
template <> struct ZPlan<8>   { static constexpr int E = 4, NS = 2, R0 = 4, R1 = 2, R2 = 1, R3 = 1; };
template <> struct ZPlan<16>  { static constexpr int E = 4, NS = 2, R0 = 4, R1 = 4, R2 = 1, R3 = 1; };
template <> struct ZPlan<32>  { static constexpr int E = 4, NS = 3, R0 = 4, R1 = 4, R2 = 2, R3 = 1; };
template <> struct ZPlan<64>  { static constexpr int E = 4, NS = 3, R0 = 4, R1 = 4, R2 = 4, R3 = 1; };
template <> struct ZPlan<128> { static constexpr int E = 4, NS = 4, R0 = 4, R1 = 4, R2 = 4, R3 = 2; };
template <> struct ZPlan<256> { static constexpr int E = 8, NS = 3, R0 = 8, R1 = 8, R2 = 4, R3 = 1; };

// Stage twiddle tables.  Stage s >= 1 of a plan (NSV = product of the
// earlier radices, R = its radix) needs W_{NSV*R}^{jm*r} for jm < NSV and
// 1 <= r < R.  They are kept in shared memory as [r-1][jm], so that lanes
// with consecutive jm read consecutive words (no bank conflicts) and lanes
// with equal jm read the same word (broadcast).
template <class P>
struct StageTw {
  static constexpr int N1 = P::R0, N2 = P::R0 * P::R1, N3 = P::R0 * P::R1 * P::R2;
  static constexpr int O1 = 0;
  static constexpr int O2 = O1 + (P::NS > 1 ? N1 * (P::R1 - 1) : 0);
  static constexpr int O3 = O2 + (P::NS > 2 ? N2 * (P::R2 - 1) : 0);
  static constexpr int SIZE = O3 + (P::NS > 3 ? N3 * (P::R3 - 1) : 0);
};

// Fill the stage tables of plan P for a line of length L from the length-n
// table twg[k] = exp(-2 pi i k / n) (global memory), threads tid of
// nthreads.  Caller syncs.
template <int L, class P, class C>
__device__ __forceinline__ void build_stage_tw(C *st, const C *__restrict__ twg, int n, int tid,
                                               int nthreads) {
  using S = StageTw<P>;
  for (int i = tid; i < S::SIZE; i += nthreads) {
    int nsv, R, loc;
    if (i < S::O2) {
      nsv = S::N1; R = P::R1; loc = i - S::O1;
    } else if (i < S::O3) {
      nsv = S::N2; R = P::R2; loc = i - S::O2;
    } else {
      nsv = S::N3; R = P::R3; loc = i - S::O3;
    }
    const int r = loc / nsv + 1, jm = loc % nsv;
    st[i] = twg[(long long)jm * r * (n / (nsv * R))];
  }
}

// One Stockham stage on the strided distribution.
//   L: line length, E: values per thread, R: radix, NSV: product of the
//   radices of the previous stages.  Butterfly j = t + T*q (q < E/R) reads
//   positions j + r*L/R (= registers q + r*E/R), applies the twiddles
//   W_{NSV*R}^{(j mod NSV)*r} (table tws, layout [r-1][jm]), runs a radix-R
//   DFT and sends output r to position (j/NSV)*NSV*R + (j mod NSV) + r*NSV.
// For the last stage (NSV*R == L) the destination is register q + r*E/R,
// so no exchange is needed.  Otherwise outputs go to xbuf via idx(pos),
// sync() is called, and the strided distribution is read back.
template <int L, int E, int R, int NSV, bool FWD, class C, class Idx, class Sync>
__device__ __forceinline__ void stage(C (&v)[E], const int t, const C *tws, C *xbuf, Idx idx,
                                      Sync sync) {
  constexpr int T = L / E;
  constexpr int Q = E / R;
  constexpr bool LAST = (NSV * R == L);
#pragma unroll
  for (int q = 0; q < Q; q++) {
    C a[R];
#pragma unroll
    for (int r = 0; r < R; r++) a[r] = v[q + r * Q];
    const int j = t + T * q;
    if constexpr (NSV > 1) {
      const int jm = j % NSV;
#pragma unroll
      for (int r = 1; r < R; r++) a[r] = twmul<FWD>(a[r], tws[(r - 1) * NSV + jm]);
    }
    dft<R, FWD>(a);
    if constexpr (LAST) {
#pragma unroll
      for (int r = 0; r < R; r++) v[q + r * Q] = a[r];
    } else {
      const int dst = (j / NSV) * NSV * R + (j % NSV);
#pragma unroll
      for (int r = 0; r < R; r++) xbuf[idx(dst + r * NSV)] = a[r];
    }
  }
  if constexpr (!LAST) {
    sync();
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = xbuf[idx(t + T * e)];
    sync();
  }
}

// Full line FFT of length L with plan P (P::E must equal E); st = the
// plan's stage twiddle tables (build_stage_tw).
template <int L, class P, bool FWD, class C, class Idx, class Sync>
__device__ __forceinline__ void line_fft(C (&v)[P::E], const int t, const C *st, C *xbuf,
                                         Idx idx, Sync sync) {
  constexpr int E = P::E;
  using S = StageTw<P>;
  stage<L, E, P::R0, 1, FWD>(v, t, st, xbuf, idx, sync);
  if constexpr (P::NS > 1) stage<L, E, P::R1, S::N1, FWD>(v, t, st + S::O1, xbuf, idx, sync);
  if constexpr (P::NS > 2) stage<L, E, P::R2, S::N2, FWD>(v, t, st + S::O2, xbuf, idx, sync);
  if constexpr (P::NS > 3) stage<L, E, P::R3, S::N3, FWD>(v, t, st + S::O3, xbuf, idx, sync);
}

// signed wavenumber of index i on an n-point axis (main.c:224-230:
// kx[i] = i for i < n/2, i - n otherwise, so kx[n/2] = -n/2)
__device__ __forceinline__ int kwave(int i, int n) { return i < n / 2 ? i : i - n; }

}  // namespace dnsb
