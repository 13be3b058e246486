// kernels.cuh -- the sm_100a kernels of one RK4 stage of the pseudo-spectral
// Navier-Stokes step (slitvinov/dns main.c:343-414), plus the initial
// forward transform (main.c:249-251), the dump transforms (main.c:270-279)
// and the energy/enstrophy reduction (main.c:257-266).
//
// HBM layout (one "slot" = one complex field on the half spectrum):
//   spectral slot  [i = kx index][j = ky index][k = kz index], k fastest,
//                  row pitch nfp = nf rounded up to 8 (nf = n/2 + 1), so that
//                  every 8-column tile row starts on a 128-byte boundary;
//                  the padding columns are never read or written.
//   real slot      [x][y][z], z fastest (the .raw layout of main.c:180-185).
// The same slot shape holds partially transformed data: after the x pass the
// first index is x instead of kx, after the y pass the second is y.
//
// One RK stage = five passes over HBM:
//   A  x backward   state (3) -> u,v,w and d/dx of v,w          (per field)
//   B  y backward   5 slots   -> u,v,w, dv/dx, dw/dx, du/dy, dw/dy (per field)
//   C  z pass       per z line: vorticity from the 7 slots, 6 c2r, u x omega
//                   in registers, 3 r2c; never touches real space in HBM
//                   except for the stale velocity of stage 0 / stage 3
//   D  y forward    3 slots, in place
//   E  x forward    + 2/3 mask, projection, viscous term and RK4 updates
// The vorticity is assembled from spectral derivatives taken on the axis a
// pass owns (x in A, y in B, z in C), so passes A, B and D work on one field
// per tile and need no cross-field staging.
#pragma once
#include "fft_core.cuh"

namespace dnsb {

// work slots of the stage
enum { SU = 0, SV = 1, SW = 2, SDVDX = 3, SDWDX = 4, SDUDY = 5, SDWDY = 6, NWORK = 7 };

struct Geo {
  int n, nf, nfp;
  int kcut;              // 2/3 rule: a wavenumber is kept iff |k| <= kcut
  long long slot;        // complex elements per spectral slot (n*n*nfp)
  long long nreal;       // n^3
};

// A column pass processes tiles of W adjacent kz columns x the full line
// along x or y.  Each block.z is one job: input slot -> output slot, and
// optionally the derivative i*k*f (k along the pass axis) -> der slot.
struct ColJobs {
  int in_slot[8];
  int out_slot[8];   // -1: no plain output
  int der_slot[8];   // -1: no derivative output
};

template <int W>
struct ColIdx {
  int p;
  __device__ __forceinline__ int operator()(int pos) const { return pos * W + p; }
};
struct BlockSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
struct WarpSync {
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
// per-line exchange buffer with one pad element per 8 to spread banks
struct PadIdx {
  __device__ __forceinline__ int operator()(int pos) const { return pos + (pos >> 3); }
};

__device__ __forceinline__ void load_tw(cd *tw, const cd *__restrict__ twg, int n) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) tw[k] = twg[k];
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Column pass along x (AXIS 0) or y (AXIS 1), forward or backward.
// grid: (nfp / W, n, njobs); block: (N / E) * W threads.
// ---------------------------------------------------------------------------
template <int N, int W, int AXIS, bool FWD>
__global__ void __launch_bounds__((N / Plan<N>::E) * W)
    k_colpass(const cd *__restrict__ in, cd *__restrict__ out, const cd *__restrict__ twg,
              Geo g, ColJobs jobs) {
  constexpr int E = Plan<N>::E, T = N / E;
  extern __shared__ cd smem[];
  cd *tw = smem;
  cd *xb = smem + N;
  load_tw(tw, twg, N);
  const int p = threadIdx.x % W, t = threadIdx.x / W;
  const int col = blockIdx.x * W + p;
  const bool ok = col < g.nf;
  const int fixed = blockIdx.y;  // j for the x pass, i for the y pass
  const int job = blockIdx.z;
  long long base, rs;
  if (AXIS == 0) {
    base = (long long)fixed * g.nfp + col;
    rs = (long long)N * g.nfp;
  } else {
    base = (long long)fixed * N * g.nfp + col;
    rs = g.nfp;
  }
  const cd *src = in + (long long)jobs.in_slot[job] * g.slot + base;
  cd v[E];
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = ok ? src[(t + T * e) * rs] : make_double2(0.0, 0.0);
  const int oslot = jobs.out_slot[job], dslot = jobs.der_slot[job];
  cd d[E];
  if (dslot >= 0) {
#pragma unroll
    for (int e = 0; e < E; e++) {
      const double k = (double)kwave(t + T * e, N);
      d[e] = make_double2(-k * v[e].y, k * v[e].x);  // i k f
    }
  }
  if (oslot >= 0) {
    line_fft<N, Plan<N>, FWD>(v, t, tw, 1, xb, ColIdx<W>{p}, BlockSync{});
    if (ok) {
      cd *dst = out + (long long)oslot * g.slot + base;
#pragma unroll
      for (int e = 0; e < E; e++) dst[(t + T * e) * rs] = v[e];
    }
  }
  if (dslot >= 0) {
    line_fft<N, Plan<N>, FWD>(d, t, tw, 1, xb, ColIdx<W>{p}, BlockSync{});
    if (ok) {
      cd *dst = out + (long long)dslot * g.slot + base;
#pragma unroll
      for (int e = 0; e < E; e++) dst[(t + T * e) * rs] = d[e];
    }
  }
}

// ---------------------------------------------------------------------------
// z lines: TZ = M / E threads per line (M = N/2), 32 / TZ lines per warp.
// ---------------------------------------------------------------------------
template <int N>
struct ZCfg {
  static constexpr int M = N / 2;
  static constexpr int E = ZPlan<M>::E;
  static constexpr int TZ = M / E;
  static constexpr int THREADS = (N * N * TZ) < 256 ? (N * N * TZ) : 256;
  static constexpr int LINES = THREADS / TZ;   // lines per block
  static constexpr int XB = M + M / 8;         // padded exchange buffer per line
};

// Partner exchange for the real-transform pre/post-processing: the value at
// position M - k for every k = t + TZ*e held by this thread.  For t > 0 it
// sits in lane (TZ - t) of the same line, register E-1-e; for t == 0 it is
// this thread's register E-e, or `m_val` (position M) for e == 0.
template <int E, int TZ>
__device__ __forceinline__ void partners(const cd (&v)[E], cd (&pp)[E], int t, int lane0,
                                         cd m_val) {
  const int src = lane0 + ((TZ - t) & (TZ - 1));
#pragma unroll
  for (int e = 0; e < E; e++) {
    cd s;
    s.x = __shfl_sync(0xffffffffu, v[E - 1 - e].x, src);
    s.y = __shfl_sync(0xffffffffu, v[E - 1 - e].y, src);
    if (t == 0) s = (e == 0) ? m_val : v[(E - e) % E];
    pp[e] = s;
  }
}

// c2r of one z line: in: X[k] at k = t + TZ*e, X[M] in xm (lane t == 0);
// out: z[m] = (x[2m], x[2m+1]) at m = t + TZ*e, unnormalised like FFTW.
// The imaginary parts of X[0] and X[M] are ignored (FFTW c2r semantics).
template <int N>
__device__ __forceinline__ void c2r_line(cd (&v)[ZCfg<N>::E], cd xm, int t, int lane0,
                                         const cd *tw, cd *xb) {
  using C = ZCfg<N>;
  constexpr int E = C::E, TZ = C::TZ;
  if (t == 0) {
    v[0].y = 0.0;
    xm.y = 0.0;
  }
  cd pp[E];
  partners<E, TZ>(v, pp, t, lane0, xm);
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int k = t + TZ * e;
    const cd a = make_double2(v[e].x + pp[e].x, v[e].y - pp[e].y);  // X + conj P
    const cd b = make_double2(v[e].x - pp[e].x, v[e].y + pp[e].y);  // X - conj P
    const cd c = cmulc(b, tw[k]);                                   // W^{-k} b
    v[e] = make_double2(a.x - c.y, a.y + c.x);                      // a + i c
  }
  line_fft<C::M, ZPlan<C::M>, false>(v, t, tw, 2, xb, PadIdx{}, WarpSync{});
}

// r2c of one z line: in: z[m] = (x[2m], x[2m+1]) at m = t + TZ*e;
// out: X[k] at k = t + TZ*e, and X[M] returned in xm (valid in lane t == 0).
template <int N>
__device__ __forceinline__ void r2c_line(cd (&v)[ZCfg<N>::E], cd &xm, int t, int lane0,
                                         const cd *tw, cd *xb) {
  using C = ZCfg<N>;
  constexpr int E = C::E, TZ = C::TZ;
  line_fft<C::M, ZPlan<C::M>, true>(v, t, tw, 2, xb, PadIdx{}, WarpSync{});
  cd pp[E];
  partners<E, TZ>(v, pp, t, lane0, v[0]);
  xm = make_double2(v[0].x - v[0].y, 0.0);
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int k = t + TZ * e;
    const cd ev = make_double2(0.5 * (v[e].x + pp[e].x), 0.5 * (v[e].y - pp[e].y));
    const cd dv = make_double2(0.5 * (v[e].x - pp[e].x), 0.5 * (v[e].y + pp[e].y));
    const cd q = cmul(tw[k], dv);
    v[e] = make_double2(ev.x + q.y, ev.y - q.x);  // ev - i q
  }
}

template <int N>
__device__ __forceinline__ void load_zline(cd (&v)[ZCfg<N>::E], cd &xm, const cd *__restrict__ src,
                                           int t, bool ok) {
  using C = ZCfg<N>;
#pragma unroll
  for (int e = 0; e < C::E; e++) v[e] = ok ? src[t + C::TZ * e] : make_double2(0.0, 0.0);
  xm = (ok && t == 0) ? src[C::M] : make_double2(0.0, 0.0);
}
template <int N>
__device__ __forceinline__ void store_zline(const cd (&v)[ZCfg<N>::E], cd xm, cd *__restrict__ dst,
                                            int t, bool ok) {
  using C = ZCfg<N>;
  if (!ok) return;
#pragma unroll
  for (int e = 0; e < C::E; e++) dst[t + C::TZ * e] = v[e];
  if (t == 0) dst[C::M] = xm;
}

// i*kz*X for the line positions held by this thread
template <int N>
__device__ __forceinline__ void ikz(const cd (&v)[ZCfg<N>::E], cd xm, cd (&o)[ZCfg<N>::E], cd &om,
                                    int t) {
  using C = ZCfg<N>;
#pragma unroll
  for (int e = 0; e < C::E; e++) {
    const double k = (double)(t + C::TZ * e);
    o[e] = make_double2(-k * v[e].y, k * v[e].x);
  }
  const double k = (double)C::M;  // kz[n/2] = +n/2 (main.c:228)
  om = make_double2(-k * xm.y, k * xm.x);
}

// ---------------------------------------------------------------------------
// Pass C: per z line, build omega, c2r u and omega, N = u x omega, r2c N.
// KIND 0: first stage, velocity from the stale real slots (main.c:344 skips
//         the back transform at rk == 0); KIND 1: middle stage;
// KIND 2: last stage, also stores the real velocity as the next stale one.
// grid: N*N / LINES blocks.
// ---------------------------------------------------------------------------
template <int N, int KIND>
__global__ void __launch_bounds__(ZCfg<N>::THREADS)
    k_zstage(cd *__restrict__ work, double *__restrict__ stale, const cd *__restrict__ twg, Geo g,
             double invn3) {
  using C = ZCfg<N>;
  constexpr int E = C::E, TZ = C::TZ;
  extern __shared__ cd smem[];
  cd *tw = smem;
  load_tw(tw, twg, N);
  const int lid = threadIdx.x / TZ;  // line within block
  const int t = threadIdx.x % TZ;
  const int lane0 = (threadIdx.x & 31) - t;
  cd *xb = smem + N + lid * C::XB;
  const long long line = (long long)blockIdx.x * C::LINES + lid;
  const bool ok = line < (long long)N * N;
  const long long off = line * g.nfp;
  const long long roff = line * N;  // real line offset

  cd u[E], vv[E], w[E];    // real velocity, pairs (x[2m], x[2m+1]) at m = t + TZ e
  cd oy[E], oym, ox[E], oxm;  // spectral omega_y, omega_x
  {
    cd a[E], am, b[E], bm;
    // omega_y = i kz u - dw/dx
    load_zline<N>(a, am, work + SU * g.slot + off, t, ok);
    load_zline<N>(b, bm, work + SDWDX * g.slot + off, t, ok);
    ikz<N>(a, am, oy, oym, t);
#pragma unroll
    for (int e = 0; e < E; e++) oy[e] = csub(oy[e], b[e]);
    oym = csub(oym, bm);
    if (KIND != 0) {
      c2r_line<N>(a, am, t, lane0, tw, xb);
#pragma unroll
      for (int e = 0; e < E; e++) u[e] = cscale(a[e], invn3);
    }
    // omega_x = dw/dy - i kz v
    load_zline<N>(a, am, work + SV * g.slot + off, t, ok);
    load_zline<N>(b, bm, work + SDWDY * g.slot + off, t, ok);
    ikz<N>(a, am, ox, oxm, t);
#pragma unroll
    for (int e = 0; e < E; e++) ox[e] = csub(b[e], ox[e]);
    oxm = csub(bm, oxm);
    if (KIND != 0) {
      c2r_line<N>(a, am, t, lane0, tw, xb);
#pragma unroll
      for (int e = 0; e < E; e++) vv[e] = cscale(a[e], invn3);
      load_zline<N>(a, am, work + SW * g.slot + off, t, ok);
      c2r_line<N>(a, am, t, lane0, tw, xb);
#pragma unroll
      for (int e = 0; e < E; e++) w[e] = cscale(a[e], invn3);
    }
  }
  if (KIND == 0) {
    const double *s = stale + roff;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int m = t + TZ * e;
      u[e] = ok ? *(const double2 *)(s + 2 * m) : make_double2(0.0, 0.0);
      vv[e] = ok ? *(const double2 *)(s + g.nreal + 2 * m) : make_double2(0.0, 0.0);
      w[e] = ok ? *(const double2 *)(s + 2 * g.nreal + 2 * m) : make_double2(0.0, 0.0);
    }
  }
  if (KIND == 2 && ok) {
    double *s = stale + roff;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int m = t + TZ * e;
      *(double2 *)(s + 2 * m) = u[e];
      *(double2 *)(s + g.nreal + 2 * m) = vv[e];
      *(double2 *)(s + 2 * g.nreal + 2 * m) = w[e];
    }
  }
  // N = u x omega  (main.c:372-377), accumulated one omega component at a time
  cd nx[E], ny[E], nz[E];
  c2r_line<N>(ox, oxm, t, lane0, tw, xb);
#pragma unroll
  for (int e = 0; e < E; e++) {
    const cd o = cscale(ox[e], invn3);
    ny[e] = make_double2(w[e].x * o.x, w[e].y * o.y);
    nz[e] = make_double2(-vv[e].x * o.x, -vv[e].y * o.y);
  }
  c2r_line<N>(oy, oym, t, lane0, tw, xb);
#pragma unroll
  for (int e = 0; e < E; e++) {
    const cd o = cscale(oy[e], invn3);
    nx[e] = make_double2(-w[e].x * o.x, -w[e].y * o.y);
    nz[e] = make_double2(nz[e].x + u[e].x * o.x, nz[e].y + u[e].y * o.y);
  }
  {
    cd a[E], am, b[E], bm;
    load_zline<N>(a, am, work + SDVDX * g.slot + off, t, ok);
    load_zline<N>(b, bm, work + SDUDY * g.slot + off, t, ok);
#pragma unroll
    for (int e = 0; e < E; e++) a[e] = csub(a[e], b[e]);  // omega_z = dv/dx - du/dy
    am = csub(am, bm);
    c2r_line<N>(a, am, t, lane0, tw, xb);
#pragma unroll
    for (int e = 0; e < E; e++) {
      const cd o = cscale(a[e], invn3);
      nx[e] = make_double2(nx[e].x + vv[e].x * o.x, nx[e].y + vv[e].y * o.y);
      ny[e] = make_double2(ny[e].x - u[e].x * o.x, ny[e].y - u[e].y * o.y);
    }
  }
  // forward z transforms of N into slots U, V, W (main.c:378-380)
  cd xm;
  r2c_line<N>(nx, xm, t, lane0, tw, xb);
  store_zline<N>(nx, xm, work + SU * g.slot + off, t, ok);
  r2c_line<N>(ny, xm, t, lane0, tw, xb);
  store_zline<N>(ny, xm, work + SV * g.slot + off, t, ok);
  r2c_line<N>(nz, xm, t, lane0, tw, xb);
  store_zline<N>(nz, xm, work + SW * g.slot + off, t, ok);
}

// z r2c of real slots (initial transform, main.c:249-251): real slot f ->
// work slot f.  grid: (N*N / LINES, nfields)
template <int N>
__global__ void __launch_bounds__(ZCfg<N>::THREADS)
    k_zr2c(const double *__restrict__ real, cd *__restrict__ work, const cd *__restrict__ twg,
           Geo g) {
  using C = ZCfg<N>;
  constexpr int E = C::E, TZ = C::TZ;
  extern __shared__ cd smem[];
  cd *tw = smem;
  load_tw(tw, twg, N);
  const int lid = threadIdx.x / TZ, t = threadIdx.x % TZ;
  const int lane0 = (threadIdx.x & 31) - t;
  cd *xb = smem + N + lid * C::XB;
  const long long line = (long long)blockIdx.x * C::LINES + lid;
  const bool ok = line < (long long)N * N;
  const double *s = real + blockIdx.y * g.nreal + line * N;
  cd v[E], xm;
#pragma unroll
  for (int e = 0; e < E; e++)
    v[e] = ok ? *(const double2 *)(s + 2 * (t + TZ * e)) : make_double2(0.0, 0.0);
  r2c_line<N>(v, xm, t, lane0, tw, xb);
  store_zline<N>(v, xm, work + blockIdx.y * g.slot + line * g.nfp, t, ok);
}

// z c2r of work slots into real slots scaled by `scale` (dump, main.c:274-277)
template <int N>
__global__ void __launch_bounds__(ZCfg<N>::THREADS)
    k_zc2r(const cd *__restrict__ work, double *__restrict__ real, const cd *__restrict__ twg,
           Geo g, double scale) {
  using C = ZCfg<N>;
  constexpr int E = C::E, TZ = C::TZ;
  extern __shared__ cd smem[];
  cd *tw = smem;
  load_tw(tw, twg, N);
  const int lid = threadIdx.x / TZ, t = threadIdx.x % TZ;
  const int lane0 = (threadIdx.x & 31) - t;
  cd *xb = smem + N + lid * C::XB;
  const long long line = (long long)blockIdx.x * C::LINES + lid;
  const bool ok = line < (long long)N * N;
  cd v[E], xm;
  load_zline<N>(v, xm, work + blockIdx.y * g.slot + line * g.nfp, t, ok);
  c2r_line<N>(v, xm, t, lane0, tw, xb);
  if (ok) {
    double *d = real + blockIdx.y * g.nreal + line * N;
#pragma unroll
    for (int e = 0; e < E; e++) *(double2 *)(d + 2 * (t + TZ * e)) = cscale(v[e], scale);
  }
}

// ---------------------------------------------------------------------------
// Pass E: x forward transform of the three N slots, then per point
// (main.c:381-413):
//   dU  = N * (mask * dt)
//   P   = kk > 0 ? (dU kx + dV ky + dW kz) / kk : 0
//   dU -= P kx + nu dt kk U_s          (same for V, W)
//   ST 0:   next = u0 + b0 dU,  acc = u0 + a0 dU      (u_s == u0)
//   ST 1,2: next = u0 + b dU,   acc += a dU
//   ST 3:   u0   = acc + a3 dU   (the state of the next step)
// grid: (nfp / W, n); block: (N / E) * W threads.
// ---------------------------------------------------------------------------
struct StageArgs {
  cd *u0;      // step start state (3 slots); ST 3 writes the new state here
  cd *us;      // stage input (3 slots)
  cd *acc;     // RK accumulator (3 slots)
  cd *next;    // next stage input (3 slots)
  cd *ph;      // pressure slot or nullptr
  double nu, dt, a, b;
};

template <int N, int W, int ST>
__global__ void __launch_bounds__((N / Plan<N>::E) * W)
    k_xfwd_update(const cd *__restrict__ work, const cd *__restrict__ twg, Geo g, StageArgs sa) {
  constexpr int E = Plan<N>::E, T = N / E;
  extern __shared__ cd smem[];
  cd *tw = smem;
  cd *res = smem + N;  // [3][N][W]
  load_tw(tw, twg, N);
  const int p = threadIdx.x % W, t = threadIdx.x / W;
  const int col = blockIdx.x * W + p;
  const bool ok = col < g.nf;
  const int j = blockIdx.y;
  const long long base = (long long)j * g.nfp + col;
  const long long rs = (long long)N * g.nfp;
#pragma unroll 1
  for (int f = 0; f < 3; f++) {
    const cd *src = work + f * g.slot + base;
    cd v[E];
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = ok ? src[(t + T * e) * rs] : make_double2(0.0, 0.0);
    cd *r = res + f * N * W;
    line_fft<N, Plan<N>, true>(v, t, tw, 1, r, ColIdx<W>{p}, BlockSync{});
#pragma unroll
    for (int e = 0; e < E; e++) r[(t + T * e) * W + p] = v[e];
  }
  if (!ok) return;
  const double ky = (double)kwave(j, N);
  const double kz = (double)col;
  const bool ky_in = (j < N / 2 ? j : N - j) <= g.kcut;  // |kwave(j)|
  const bool kz_in = col <= g.kcut;
#pragma unroll 2
  for (int e = 0; e < E; e++) {
    const int row = t + T * e;
    const int ikx = kwave(row, N);
    const double kx = (double)ikx;
    const bool kx_in = (ikx < 0 ? -ikx : ikx) <= g.kcut;
    const double md = (double)(kx_in && ky_in && kz_in) * sa.dt;
    const long long o = row * rs + base;
    // own points only: same thread wrote r[row][p] above
    cd du = cscale(res[(0 * N + row) * W + p], md);
    cd dv = cscale(res[(1 * N + row) * W + p], md);
    cd dw = cscale(res[(2 * N + row) * W + p], md);
    const double kk = kx * kx + ky * ky + kz * kz;
    cd P;
    if (kk > 0) {
      P.x = (du.x * kx + dv.x * ky + dw.x * kz) / kk;
      P.y = (du.y * kx + dv.y * ky + dw.y * kz) / kk;
    } else {
      P = make_double2(0.0, 0.0);
    }
    const double c = sa.nu * sa.dt * kk;
    const cd us0 = sa.us[o], us1 = sa.us[g.slot + o], us2 = sa.us[2 * g.slot + o];
    du = make_double2(du.x - (P.x * kx + c * us0.x), du.y - (P.y * kx + c * us0.y));
    dv = make_double2(dv.x - (P.x * ky + c * us1.x), dv.y - (P.y * ky + c * us1.y));
    dw = make_double2(dw.x - (P.x * kz + c * us2.x), dw.y - (P.y * kz + c * us2.y));
    if (sa.ph) sa.ph[o] = P;
    if (ST == 0) {
      // us == u0
      sa.next[o] = make_double2(us0.x + sa.b * du.x, us0.y + sa.b * du.y);
      sa.next[g.slot + o] = make_double2(us1.x + sa.b * dv.x, us1.y + sa.b * dv.y);
      sa.next[2 * g.slot + o] = make_double2(us2.x + sa.b * dw.x, us2.y + sa.b * dw.y);
      sa.acc[o] = make_double2(us0.x + sa.a * du.x, us0.y + sa.a * du.y);
      sa.acc[g.slot + o] = make_double2(us1.x + sa.a * dv.x, us1.y + sa.a * dv.y);
      sa.acc[2 * g.slot + o] = make_double2(us2.x + sa.a * dw.x, us2.y + sa.a * dw.y);
    } else if (ST < 3) {
      const cd z0 = sa.u0[o], z1 = sa.u0[g.slot + o], z2 = sa.u0[2 * g.slot + o];
      const cd a0 = sa.acc[o], a1 = sa.acc[g.slot + o], a2 = sa.acc[2 * g.slot + o];
      sa.next[o] = make_double2(z0.x + sa.b * du.x, z0.y + sa.b * du.y);
      sa.next[g.slot + o] = make_double2(z1.x + sa.b * dv.x, z1.y + sa.b * dv.y);
      sa.next[2 * g.slot + o] = make_double2(z2.x + sa.b * dw.x, z2.y + sa.b * dw.y);
      sa.acc[o] = make_double2(a0.x + sa.a * du.x, a0.y + sa.a * du.y);
      sa.acc[g.slot + o] = make_double2(a1.x + sa.a * dv.x, a1.y + sa.a * dv.y);
      sa.acc[2 * g.slot + o] = make_double2(a2.x + sa.a * dw.x, a2.y + sa.a * dw.y);
    } else {
      const cd a0 = sa.acc[o], a1 = sa.acc[g.slot + o], a2 = sa.acc[2 * g.slot + o];
      sa.u0[o] = make_double2(a0.x + sa.a * du.x, a0.y + sa.a * du.y);
      sa.u0[g.slot + o] = make_double2(a1.x + sa.a * dv.x, a1.y + sa.a * dv.y);
      sa.u0[2 * g.slot + o] = make_double2(a2.x + sa.a * dw.x, a2.y + sa.a * dw.y);
    }
  }
}

// ---------------------------------------------------------------------------
// Energy / enstrophy (main.c:257-266): sums over the half spectrum of
//   e = |U|^2 + |V|^2 + |W|^2   and   kk * e,
// each term rounded like the reference's double expression (no FMA), summed
// in double-double (error-free TwoSum), block partials then one final block.
// ---------------------------------------------------------------------------
struct DD {
  double hi, lo;
};
__device__ __forceinline__ DD dd_add_d(DD a, double b) {
  const double s = __dadd_rn(a.hi, b);
  const double bb = __dsub_rn(s, a.hi);
  const double err = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bb)), __dsub_rn(b, bb));
  return DD{s, __dadd_rn(a.lo, err)};
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
  const double s = __dadd_rn(a.hi, b.hi);
  const double bb = __dsub_rn(s, a.hi);
  double err = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bb)), __dsub_rn(b.hi, bb));
  err = __dadd_rn(err, __dadd_rn(a.lo, b.lo));
  const double hi = __dadd_rn(s, err);
  const double lo = __dsub_rn(err, __dsub_rn(hi, s));
  return DD{hi, lo};
}
__device__ __forceinline__ DD dd_shfl_down(DD a, int d) {
  return DD{__shfl_down_sync(0xffffffffu, a.hi, d), __shfl_down_sync(0xffffffffu, a.lo, d)};
}
__device__ __forceinline__ double cabs2_rn(cd z) {
  return __dadd_rn(__dmul_rn(z.x, z.x), __dmul_rn(z.y, z.y));
}

template <int BS>
__device__ __forceinline__ void dd_block_reduce(DD &e, DD &o, double4 *out) {
  __shared__ DD se[BS / 32], so[BS / 32];
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    e = dd_add(e, dd_shfl_down(e, d));
    o = dd_add(o, dd_shfl_down(o, d));
  }
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  if (l == 0) {
    se[w] = e;
    so[w] = o;
  }
  __syncthreads();
  if (w == 0) {
    e = l < BS / 32 ? se[l] : DD{0.0, 0.0};
    o = l < BS / 32 ? so[l] : DD{0.0, 0.0};
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      e = dd_add(e, dd_shfl_down(e, d));
      o = dd_add(o, dd_shfl_down(o, d));
    }
    if (l == 0) *out = make_double4(e.hi, e.lo, o.hi, o.lo);
  }
}

template <int BS>
__global__ void __launch_bounds__(BS)
    k_diag(const cd *__restrict__ u, Geo g, double4 *__restrict__ partial) {
  DD e{0.0, 0.0}, o{0.0, 0.0};
  const int n = g.n;
  const long long npts = (long long)n * n * g.nf;
  for (long long q = (long long)blockIdx.x * BS + threadIdx.x; q < npts;
       q += (long long)gridDim.x * BS) {
    const long long row = q / g.nf;
    const int k = (int)(q - row * g.nf);
    const int i = (int)(row / n), j = (int)(row % n);
    const long long l = row * g.nfp + k;
    const double s = __dadd_rn(__dadd_rn(cabs2_rn(u[l]), cabs2_rn(u[g.slot + l])),
                               cabs2_rn(u[2 * g.slot + l]));
    const double kx = kwave(i, n), ky = kwave(j, n), kz = k;
    const double kk = __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
    e = dd_add_d(e, s);
    o = dd_add_d(o, __dmul_rn(kk, s));
  }
  dd_block_reduce<BS>(e, o, partial + blockIdx.x);
}

template <int BS>
__global__ void __launch_bounds__(BS) k_diag_final(const double4 *__restrict__ partial, int np,
                                                   double4 *__restrict__ out) {
  DD e{0.0, 0.0}, o{0.0, 0.0};
  for (int q = threadIdx.x; q < np; q += BS) {
    const double4 v = partial[q];
    e = dd_add(e, DD{v.x, v.y});
    o = dd_add(o, DD{v.z, v.w});
  }
  dd_block_reduce<BS>(e, o, out);
}

}  // namespace dnsb
