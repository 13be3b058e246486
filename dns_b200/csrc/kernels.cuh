// kernels.cuh -- the sm_100a kernels of one RK4 stage of the pseudo-spectral
// Navier-Stokes step (slitvinov/dns main.c:343-414), plus the initial
// forward transform (main.c:249-251), the dump transforms (main.c:270-279)
// and the energy/enstrophy reduction (main.c:257-266).
//
// Every kernel is a template on the storage scalar R: double for the FP64
// path, float for the mixed path (FP32 fields and FFTs; the reductions and
// the pointwise update arithmetic stay FP64).
//
// HBM layout (one "slot" = one complex field on the half spectrum):
//   spectral slot  [i = kx index][j = ky index][k = kz index], k fastest,
//                  row pitch nfp = nf rounded up to the column tile width W
//                  (nf = n/2 + 1; W * sizeof(complex) = 128 bytes), so every
//                  tile row starts on a 128-byte boundary; the padding
//                  columns are never read or written.
//   real slot      [x][y][z], z fastest (the .raw layout of main.c:180-185).
// The same slot shape holds partially transformed data: after the x pass the
// first index is x instead of kx, after the y pass the second is y.
//
// One RK stage = six kernels:
//   A   x backward  state (3) -> u,v,w and d/dx of v,w            (per field)
//   B   y backward  5 slots -> u,v,w, omega_z = dv/dx - du/dy, dw/dx, dw/dy
//   C   z pass      per z line: vorticity from the 6 slots, u and omega to
//                   real space, N = u x omega, N back to z spectral (stored
//                   for kz <= kcut); real space touches HBM only for the
//                   stale velocity
//   D   y forward   3 slots, in place, tiles with kz <= kcut, |ky| <= kcut kept
//   E1  x forward   3 slots, in place, rows |ky| <= kcut, |kx| <= kcut kept
//   E2  update      2/3 mask, projection, viscous term, RK4 updates
// The vorticity is assembled from spectral derivatives taken on the axis a
// pass owns (x in A, y in B, z in C), so A, B, D and E1 work on one field per
// tile and need no cross-field staging.  N only enters the update through
// the 2/3 rule (main.c:381-386), so C, D and E1 move only those modes and E2
// reads N there only.
#pragma once
#include "fft_core.cuh"

namespace dnsb {

// work slots of the stage (after pass B, SOMZ holds omega_z = dv/dx - du/dy;
// after pass A it holds dv/dx).  The z pass writes N = u x omega over the
// slots SNX, SNY, SNZ (those of u, v and dw/dy), each once the line's input
// in it has been read, and D, E1 and E2 take N from there.
enum { SU = 0, SV = 1, SDWDY = 2, SOMZ = 3, SDWDX = 4, SW = 5, NWORK = 6 };
enum { SNX = 0, SNY = 1, SNZ = 2 };

struct Geo {
  int n, nf, nfp;
  int kcut;              // 2/3 rule: a wavenumber is kept iff |k| <= kcut
  long long slot;        // complex elements per spectral slot (n*n*nfp)
  long long nreal;       // n^3
  long long run_spec;    // complex elements between two runs' slot sets
  long long run_real;    // real elements between two runs' stale velocities
};

// A column pass processes tiles of W adjacent kz columns x the full line
// along x or y.  block.z = job + njobs * run: each job maps an input slot to
// an output slot and optionally the derivative i*k*f (k along the pass axis)
// to a der slot, in every run of the batch; with an add slot the derivative
// output is add - i*k*f instead (the same tile of another slot).  A masked
// pass (the forward passes of N, whose result only enters the update inside
// the 2/3 rule, main.c:381-386) is launched on the column tiles that hold
// kz <= kcut only, in the x pass also on the ky rows with |ky| <= kcut only,
// and stores only |k| <= kcut along its own axis.
struct ColJobs {
  int in_slot[8];
  int out_slot[8];   // -1: no plain output
  int der_slot[8];   // -1: no derivative output
  int add_slot[8];   // -1: none
  int njobs;
  int masked;
};

// column tile width: 128-byte tile rows (wider rows for the x passes, whose
// rows lie a kx plane apart, measured slower: fewer, heavier blocks), capped
// so that a block stays within 1024 threads
template <class R, int AXIS, int N>
struct ColW {
  static constexpr int WB = 128 / (int)sizeof(cx<R>);
  static constexpr int WT = 1024 / (N / Plan<N>::E);
  static constexpr int W = WB < WT ? WB : WT;
};
// row pitch granularity (128 bytes): every tile width divides it
template <class R>
struct PitchW {
  static constexpr int W = 128 / (int)sizeof(cx<R>);
};

template <int W>
struct ColIdx {
  int p;
  __device__ __forceinline__ int operator()(int pos) const { return pos * W + p; }
};
struct BlockSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
// barrier of a sub-block of `count` threads (a multiple of 32) with its own
// hardware barrier id (1..15): several work items share one block of the
// persistent ensemble kernel
struct NamedSync {
  int id, count;
  __device__ __forceinline__ void operator()() const {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
  }
};
// coordinates of one work item: the launch's blockIdx / threadIdx in the
// standalone kernels, a virtual block of the persistent ensemble kernel
struct Blk {
  int x, y, z;  // block index
  int tid;      // thread index within the item
  int nt;       // threads of the item
};
__device__ __forceinline__ Blk launch_blk() {
  return Blk{(int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, (int)threadIdx.x, (int)blockDim.x};
}
struct WarpSync {
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
// per-line exchange buffer with one pad element per 2^SH to spread banks
template <int SH>
struct PadShift {
  __device__ __forceinline__ int operator()(int pos) const { return pos + (pos >> SH); }
};
// exchange barrier of one line: the block's barrier when a line spans
// several warps, else the warp's
template <bool BLOCK, class BSync = BlockSync>
struct LineSync {
  BSync bsync{};
  __device__ __forceinline__ void operator()() const {
    if (BLOCK) bsync(); else __syncwarp();
  }
};

// ---------------------------------------------------------------------------
// Column pass along x (AXIS 0) or y (AXIS 1), forward or backward.
// grid: (nfp / W, n, njobs * nruns); block: (N / E) * W threads
// (W = ColW<R, AXIS, N>::W).
// ---------------------------------------------------------------------------
template <class R, int N, int AXIS, bool FWD, class Sync>
__device__ __forceinline__ void colpass_body(const cx<R> *__restrict__ in, cx<R> *__restrict__ out,
                                             const cx<R> *__restrict__ twg, const Geo &g,
                                             const ColJobs &jobs, const Blk b, Sync sync,
                                             unsigned char *smem) {
  using C = cx<R>;
  constexpr int W = ColW<R, AXIS, N>::W;
  constexpr int E = Plan<N>::E, T = N / E;
  C *st = (C *)smem;  // stage twiddles (<= N entries)
  C *xb = st + N;
  build_stage_tw<N, Plan<N>>(st, twg, N, b.tid, b.nt);
  sync();
  const int p = b.tid % W, t = b.tid / W;
  const int col = b.x * W + p;
  const bool ok = col < g.nf;
  // j for the x pass, i for the y pass; a masked x pass is launched on the
  // 2 kcut + 1 rows with |ky| <= kcut only: rows past kcut map to n - kcut..
  int fixed = b.y;
  if (AXIS == 0 && jobs.masked && fixed > g.kcut) fixed += N - (2 * g.kcut + 1);
  const int job = b.z % jobs.njobs;
  const long long rb = (long long)(b.z / jobs.njobs) * g.run_spec;
  in += rb;
  out += rb;
  long long base, rs;
  if (AXIS == 0) {
    base = (long long)fixed * g.nfp + col;
    rs = (long long)N * g.nfp;
  } else {
    base = (long long)fixed * N * g.nfp + col;
    rs = g.nfp;
  }
  const C *src = in + (long long)jobs.in_slot[job] * g.slot + base;
  const int oslot = jobs.out_slot[job], dslot = jobs.der_slot[job], aslot = jobs.add_slot[job];
  C v[E];
  // the input is read twice (the second read is an L2 hit) rather than kept
  // in a second register array: first for the derivative i k f, then for the
  // plain transform, which may overwrite the input in place
#pragma unroll
  for (int pass = 0; pass < 2; pass++) {
    const int dst_slot = pass == 0 ? dslot : oslot;
    if (dst_slot < 0) continue;
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = ok ? src[(t + T * e) * rs] : czero<C>();
    if (pass == 0 && aslot < 0) {
#pragma unroll
      for (int e = 0; e < E; e++) {
        const R k = (R)kwave(t + T * e, N);
        v[e] = cmk<C>(-k * v[e].y, k * v[e].x);  // i k f
      }
    } else if (pass == 0) {
      const C *add = in + (long long)aslot * g.slot + base;
#pragma unroll
      for (int e = 0; e < E; e++) {
        const R k = (R)kwave(t + T * e, N);
        const C a = ok ? add[(t + T * e) * rs] : czero<C>();
        v[e] = cmk<C>(a.x + k * v[e].y, a.y - k * v[e].x);  // add - i k f
      }
    }
    line_fft<N, Plan<N>, FWD>(v, t, st, xb, ColIdx<W>{p}, sync);
    if (ok) {
      C *dst = out + (long long)dst_slot * g.slot + base;
#pragma unroll
      for (int e = 0; e < E; e++) {
        const int k = kwave(t + T * e, N);
        if (!jobs.masked || (k < 0 ? -k : k) <= g.kcut) dst[(t + T * e) * rs] = v[e];
      }
    }
  }
}

template <class R, int N, int AXIS, bool FWD>
__global__ void __launch_bounds__((N / Plan<N>::E) * ColW<R, AXIS, N>::W)
    k_colpass(const cx<R> *__restrict__ in, cx<R> *__restrict__ out,
              const cx<R> *__restrict__ twg, Geo g, ColJobs jobs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  colpass_body<R, N, AXIS, FWD>(in, out, twg, g, jobs, launch_blk(), BlockSync{}, smem_raw);
}

// The same pass with its registers held so that MINB blocks fit per SM (a
// register schedule the autotuner may pick).
template <class R, int N, int AXIS, bool FWD, int MINB>
__global__ void __launch_bounds__((N / Plan<N>::E) * ColW<R, AXIS, N>::W, MINB)
    k_colpass_minb(const cx<R> *__restrict__ in, cx<R> *__restrict__ out,
                   const cx<R> *__restrict__ twg, Geo g, ColJobs jobs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  colpass_body<R, N, AXIS, FWD>(in, out, twg, g, jobs, launch_blk(), BlockSync{}, smem_raw);
}

// Register-schedule candidates of a column-pass tile of THREADS threads
// with complex values of CB bytes: a minimum of m[i] resident blocks per SM
// (0: the compiler's register choice; otherwise register caps of about 170,
// 128, 102, 85, 64; FP64 tiles stop at 80: at 64 they spill a kilobyte per
// thread).
template <int THREADS, int CB>
struct ColCands {
  static constexpr int n = 1;
  static constexpr int m[1] = {0};
};
template <>
struct ColCands<64, 16> {
  static constexpr int n = 5;
  static constexpr int m[5] = {0, 6, 8, 10, 12};
};
template <>
struct ColCands<128, 16> {
  static constexpr int n = 5;
  static constexpr int m[5] = {0, 3, 4, 5, 6};
};
template <>
struct ColCands<256, 16> {
  static constexpr int n = 3;
  static constexpr int m[3] = {0, 2, 3};
};
template <>
struct ColCands<128, 8> {
  static constexpr int n = 6;
  static constexpr int m[6] = {0, 3, 4, 5, 6, 8};
};
template <>
struct ColCands<256, 8> {
  static constexpr int n = 4;
  static constexpr int m[4] = {0, 2, 3, 4};
};
template <>
struct ColCands<512, 8> {
  static constexpr int n = 3;
  static constexpr int m[3] = {0, 1, 2};
};

// ---------------------------------------------------------------------------
// Real transforms of single z lines (initial r2c, dump c2r) through a
// half-length complex FFT: TZ = M / E threads per line (M = N/2).
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
template <int E, int TZ, class C>
__device__ __forceinline__ void partners(const C (&v)[E], C (&pp)[E], int t, int lane0, C m_val) {
  const int src = lane0 + ((TZ - t) & (TZ - 1));
#pragma unroll
  for (int e = 0; e < E; e++) {
    C s;
    s.x = __shfl_sync(0xffffffffu, v[E - 1 - e].x, src);
    s.y = __shfl_sync(0xffffffffu, v[E - 1 - e].y, src);
    if (t == 0) s = (e == 0) ? m_val : v[(E - e) % E];
    pp[e] = s;
  }
}

// c2r of one z line: in: X[k] at k = t + TZ*e, X[M] in xm (lane t == 0);
// out: z[m] = (x[2m], x[2m+1]) at m = t + TZ*e, unnormalised like FFTW.
// The imaginary parts of X[0] and X[M] are ignored (FFTW c2r semantics).
template <int N, class C>
__device__ __forceinline__ void c2r_line(C (&v)[ZCfg<N>::E], C xm, int t, int lane0, const C *tw,
                                         const C *st, C *xb) {
  using Z = ZCfg<N>;
  constexpr int E = Z::E, TZ = Z::TZ;
  if (t == 0) {
    v[0].y = 0;
    xm.y = 0;
  }
  C pp[E];
  partners<E, TZ>(v, pp, t, lane0, xm);
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int k = t + TZ * e;
    const C a = cmk<C>(v[e].x + pp[e].x, v[e].y - pp[e].y);  // X + conj P
    const C b = cmk<C>(v[e].x - pp[e].x, v[e].y + pp[e].y);  // X - conj P
    const C c = cmulc(b, tw[k]);                             // W^{-k} b
    v[e] = cmk<C>(a.x - c.y, a.y + c.x);                     // a + i c
  }
  line_fft<Z::M, ZPlan<Z::M>, false>(v, t, st, xb, PadShift<3>{}, WarpSync{});
}

// r2c of one z line: in: z[m] = (x[2m], x[2m+1]) at m = t + TZ*e;
// out: X[k] at k = t + TZ*e, and X[M] returned in xm (valid in lane t == 0).
template <int N, class C>
__device__ __forceinline__ void r2c_line(C (&v)[ZCfg<N>::E], C &xm, int t, int lane0, const C *tw,
                                         const C *st, C *xb) {
  using Z = ZCfg<N>;
  using S = sc<C>;
  constexpr int E = Z::E, TZ = Z::TZ;
  line_fft<Z::M, ZPlan<Z::M>, true>(v, t, st, xb, PadShift<3>{}, WarpSync{});
  C pp[E];
  partners<E, TZ>(v, pp, t, lane0, v[0]);
  xm = cmk<C>(v[0].x - v[0].y, S(0));
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int k = t + TZ * e;
    const C ev = cmk<C>(S(0.5) * (v[e].x + pp[e].x), S(0.5) * (v[e].y - pp[e].y));
    const C dv = cmk<C>(S(0.5) * (v[e].x - pp[e].x), S(0.5) * (v[e].y + pp[e].y));
    const C q = cmul(tw[k], dv);
    v[e] = cmk<C>(ev.x + q.y, ev.y - q.x);  // ev - i q
  }
}

// z r2c of real slots (initial transform, main.c:249-251): real slot f ->
// work slot f.  grid: (N*N / LINES, nfields)
template <class R, int N>
__global__ void __launch_bounds__(ZCfg<N>::THREADS)
    k_zr2c(const R *__restrict__ real, cx<R> *__restrict__ work, const cx<R> *__restrict__ twg,
           Geo g) {
  using C = cx<R>;
  using Z = ZCfg<N>;
  constexpr int E = Z::E, TZ = Z::TZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *tw = (C *)smem_raw;  // full table exp(-2 pi i k / N): pre/post twiddles
  C *st = tw + N;         // stage twiddles of ZPlan<N/2>
  for (int k = threadIdx.x; k < N; k += blockDim.x) tw[k] = twg[k];
  build_stage_tw<N / 2, ZPlan<N / 2>>(st, twg, N, threadIdx.x, blockDim.x);
  __syncthreads();
  const int lid = threadIdx.x / TZ, t = threadIdx.x % TZ;
  const int lane0 = (threadIdx.x & 31) - t;
  C *xb = tw + 2 * N + lid * Z::XB;
  const long long line = (long long)blockIdx.x * Z::LINES + lid;
  const bool ok = line < (long long)N * N;
  const R *s = real + blockIdx.y * g.nreal + line * N;
  C v[E], xm;
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int m = t + TZ * e;
    v[e] = ok ? cmk<C>(s[2 * m], s[2 * m + 1]) : czero<C>();
  }
  r2c_line<N>(v, xm, t, lane0, tw, st, xb);
  if (ok) {
    C *d = work + blockIdx.y * g.slot + line * g.nfp;
#pragma unroll
    for (int e = 0; e < E; e++) d[t + TZ * e] = v[e];
    if (t == 0) d[Z::M] = xm;
  }
}

// z c2r of work slots into float64 real slots scaled by `scale` (dump,
// main.c:274-277; fields handed to the host are always float64)
template <class R, int N>
__global__ void __launch_bounds__(ZCfg<N>::THREADS)
    k_zc2r(const cx<R> *__restrict__ work, double *__restrict__ real,
           const cx<R> *__restrict__ twg, Geo g, double scale) {
  using C = cx<R>;
  using Z = ZCfg<N>;
  constexpr int E = Z::E, TZ = Z::TZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *tw = (C *)smem_raw;
  C *st = tw + N;
  for (int k = threadIdx.x; k < N; k += blockDim.x) tw[k] = twg[k];
  build_stage_tw<N / 2, ZPlan<N / 2>>(st, twg, N, threadIdx.x, blockDim.x);
  __syncthreads();
  const int lid = threadIdx.x / TZ, t = threadIdx.x % TZ;
  const int lane0 = (threadIdx.x & 31) - t;
  C *xb = tw + 2 * N + lid * Z::XB;
  const long long line = (long long)blockIdx.x * Z::LINES + lid;
  const bool ok = line < (long long)N * N;
  const C *src = work + blockIdx.y * g.slot + line * g.nfp;
  C v[E];
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = ok ? src[t + TZ * e] : czero<C>();
  C xm = (ok && t == 0) ? src[Z::M] : czero<C>();
  c2r_line<N>(v, xm, t, lane0, tw, st, xb);
  if (ok) {
    double *d = real + blockIdx.y * g.nreal + line * N;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int m = t + TZ * e;
      *(double2 *)(d + 2 * m) = make_double2((double)v[e].x * scale, (double)v[e].y * scale);
    }
  }
}

// ---------------------------------------------------------------------------
// Pass C: per z line, build omega, c2r u and omega, N = u x omega, r2c N.
//
// Each real transform pair runs as ONE complex N-point FFT ("two for one"):
//   c2r: Y[k] = A_ext[k] + i B_ext[k] with the Hermitian extension
//        X_ext[k] = X[k] (k <= N/2), conj(X[N-k]) (k > N/2) and the
//        imaginary parts of X[0], X[N/2] dropped (FFTW c2r semantics, the
//        z axis being the last, real one); Re y = a, Im y = b.
//   r2c: Y = a + i b; X_a[k] = (Z[k] + conj Z[N-k]) / 2,
//        X_b[k] = -i (Z[k] - conj Z[N-k]) / 2.
// T = N/E threads per line hold E points each.  In the middle stages the
// pairs (u, omega_y), (w, omega_z), (v, omega_x) read each input slot once
// and u x omega accumulates in registers; the first and last stages stage
// the velocity and two partial sums in shared memory (each thread only
// reads back its own points).
// KIND 0: first stage, velocity from the stale real slots (main.c:344 skips
//         the back transform at rk == 0); KIND 1: middle stage;
// KIND 2: last stage, also stores the real velocity as the next stale one.
// ---------------------------------------------------------------------------
// The z pass runs the column plans: up to 16 values per thread, one exchange
// fewer per FFT than 8 values at n = 128, 256.
template <class R, int N, int KIND>
struct ZC {
  using P = Plan<N>;
  static constexpr int E = P::E;
  static constexpr int T = N / E;                 // threads per line
  static constexpr int M = N / 2;
  // FP64 with 16 values per thread (S2) and FP32: the pairs run in the
  // order (u, omega_y), (v, omega_x), (w, omega_z), so that N_z is complete
  // after the second and goes through its forward FFT and out before the
  // third; N_x and N_y are then formed in place in the FFT registers.  At
  // most two fields beyond the FFT's own values are live: FP64 keeps (u,
  // omega_y) in shared memory and (v, omega_x) in registers (128-thread
  // blocks of 8 lines, 2 per SM, which build the stage twiddles once for 8
  // lines: 1-10 % faster than 64-thread blocks at 4 per SM; capping the
  // registers for more blocks measured slower); FP32 keeps both pairs in
  // registers (128 of them; 512^3 in 256-thread blocks at 2 per SM, 10 %
  // faster there than 128-thread blocks at 4, 1 % slower at 256^3).  The
  // first stage reads the stale velocity where it needs it.
  static constexpr bool S2 = sizeof(R) == 8 && E >= 16;
  static constexpr bool F32 = sizeof(R) == 4;
  static constexpr int WANT = (F32 && N > 256) ? 256 : 128;
  static constexpr int THREADS = (N * N * T) < WANT ? (N * N * T) : WANT;
  static constexpr int LINES = THREADS / T;
  static constexpr int MINB = S2 ? 2 : F32 ? (N > 256 ? 2 : 4) : 3;  // blocks per SM
  static constexpr int PADSH = (E >= 16) ? 4 : 3;
  static constexpr int XB = N + (N >> PADSH);     // padded exchange buffer (complex)
  // stage twiddle entries held (even, so the exchange buffers stay 16-byte
  // aligned)
  static constexpr int TWN = (StageTw<P>::SIZE + 1) / 2 * 2 > 2 ? (StageTw<P>::SIZE + 1) / 2 * 2 : 2;
  // staged scalars per line: S2 none (first stage) or (u, omega_y); FP32
  // none; FP64 with 8 values per thread none (middle stage) or u, v, w,
  // N_y, N_z
  static constexpr int STASH =
      S2 ? (KIND == 0 ? 0 : 2 * N) : ((KIND == 1 || F32) ? 0 : 5 * N);
  static constexpr size_t SMEM =
      (size_t)(TWN + LINES * XB) * sizeof(cx<R>) + (size_t)LINES * STASH * sizeof(R);
};

// Hermitian-extended pair  Y[k] = A_ext[k] + i B_ext[k]  at k = t + T*e.
// Loads are issued in chunks of CH positions (an empty asm with a memory
// clobber keeps the compiler from hoisting all of them), which bounds the
// registers held by loads in flight.
template <class R, int N, int KIND, int CH = 4, class C, class FA, class FB>
__device__ __forceinline__ void ext_pair(C (&y)[ZC<R, N, KIND>::E], int t, FA fa, FB fb) {
  using Z = ZC<R, N, KIND>;
#pragma unroll
  for (int e0 = 0; e0 < Z::E; e0 += CH) {
#pragma unroll
    for (int e = e0; e < e0 + CH && e < Z::E; e++) {
      const int k = t + Z::T * e;
      const bool direct = k <= Z::M;
      const int s = direct ? k : N - k;
      C a = fa(s), b = fb(s);
      if (s == 0 || s == Z::M) {
        a.y = 0;
        b.y = 0;
      }
      if (!direct) {
        a.y = -a.y;
        b.y = -b.y;
      }
      y[e] = cmk<C>(a.x - b.y, a.y + b.x);
    }
    asm volatile("" ::: "memory");
  }
}

// Same, with one functor giving both spectra at a position, so that a field
// feeding both halves (u for u and omega_y) is loaded once.
template <class R, int N, int KIND, int CH = 4, class C, class FAB>
__device__ __forceinline__ void ext_gen(C (&y)[ZC<R, N, KIND>::E], int t, FAB fab) {
  using Z = ZC<R, N, KIND>;
#pragma unroll
  for (int e0 = 0; e0 < Z::E; e0 += CH) {
#pragma unroll
    for (int e = e0; e < e0 + CH && e < Z::E; e++) {
      const int k = t + Z::T * e;
      const bool direct = k <= Z::M;
      const int s = direct ? k : N - k;
      C a, b;
      fab(s, a, b);
      if (s == 0 || s == Z::M) {
        a.y = 0;
        b.y = 0;
      }
      if (!direct) {
        a.y = -a.y;
        b.y = -b.y;
      }
      y[e] = cmk<C>(a.x - b.y, a.y + b.x);
    }
    asm volatile("" ::: "memory");
  }
}

// The forward transforms of the z pass for one line (main.c:378-380); only
// kz <= kcut is stored (N enters the update through the 2/3 rule only).
// `row` = the line's row of work slot 0.
// (N_x, N_y) held in y as one complex line: FFT, unpack, store into SNX,
// SNY (ends with a barrier: the exchange buffer is free again)
template <class R, int N, int KIND, class Idx, class Sync>
__device__ __forceinline__ void zfwd_xy(cx<R> (&y)[ZC<R, N, KIND>::E], int t, const cx<R> *tw,
                                        cx<R> *xb, Idx idx, Sync sync, cx<R> *row, const Geo &g,
                                        bool ok) {
  using C = cx<R>;
  using Z = ZC<R, N, KIND>;
  constexpr int E = Z::E, T = Z::T, M = Z::M;
  const int KZ = g.kcut < M ? g.kcut : M;
  line_fft<N, typename Z::P, true>(y, t, tw, xb, idx, sync);
#pragma unroll
  for (int e = 0; e < E; e++) xb[idx(t + T * e)] = y[e];
  sync();
  C *oU = row + SNX * g.slot, *oV = row + SNY * g.slot;
#pragma unroll
  for (int e = 0; e <= E / 2; e++) {
    const int k = t + T * e;
    if (k <= KZ) {
      const C z = y[e], p = xb[idx((N - k) & (N - 1))];
      const C a = cmk<C>(R(0.5) * (z.x + p.x), R(0.5) * (z.y - p.y));  // (Z + conj P) / 2
      const C d = cmk<C>(R(0.5) * (z.x - p.x), R(0.5) * (z.y + p.y));  // (Z - conj P) / 2
      if (ok) {
        oU[k] = a;
        oV[k] = cmk<C>(d.y, -d.x);  // -i d
      }
    }
  }
  sync();
}
// N_z held in y as (N_z, 0): FFT, store into SNZ
template <class R, int N, int KIND, class Idx, class Sync>
__device__ __forceinline__ void zfwd_z(cx<R> (&y)[ZC<R, N, KIND>::E], int t, const cx<R> *tw,
                                       cx<R> *xb, Idx idx, Sync sync, cx<R> *row, const Geo &g,
                                       bool ok) {
  using C = cx<R>;
  using Z = ZC<R, N, KIND>;
  constexpr int E = Z::E, T = Z::T, M = Z::M;
  const int KZ = g.kcut < M ? g.kcut : M;
  line_fft<N, typename Z::P, true>(y, t, tw, xb, idx, sync);
  C *oW = row + SNZ * g.slot;
#pragma unroll
  for (int e = 0; e <= E / 2; e++) {
    const int k = t + T * e;
    if (k <= KZ && ok) oW[k] = y[e];
  }
}
// both, from N held in registers (the stages that complete N at the end)
template <class R, int N, int KIND, class Idx, class Sync>
__device__ __forceinline__ void zstage_forward(cx<R> (&y)[ZC<R, N, KIND>::E],
                                               const R (&nx)[ZC<R, N, KIND>::E],
                                               const R (&ny)[ZC<R, N, KIND>::E],
                                               const R (&nz)[ZC<R, N, KIND>::E], int t,
                                               const cx<R> *tw, cx<R> *xb, Idx idx, Sync sync,
                                               cx<R> *row, const Geo &g, bool ok) {
  using C = cx<R>;
  constexpr int E = ZC<R, N, KIND>::E;
#pragma unroll
  for (int e = 0; e < E; e++) y[e] = cmk<C>(nx[e], ny[e]);
  zfwd_xy<R, N, KIND>(y, t, tw, xb, idx, sync, row, g, ok);
#pragma unroll
  for (int e = 0; e < E; e++) y[e] = cmk<C>(nz[e], R(0));
  zfwd_z<R, N, KIND>(y, t, tw, xb, idx, sync, row, g, ok);
}

// One block of the z pass: Z::LINES lines starting at line b.x * LINES of
// run b.y (block-wide barriers through `bsync`, which lines of more than 32
// threads also use between FFT stages).  KEEP (the pair orders of S2 and
// FP32 only): also store the real velocity and vorticity the pass forms in
// keep[f][n^3], f = u, v, w, omega_x, omega_y, omega_z of the run (the
// first stage: the vorticity only), for the discrete adjoint.
template <class R, int N, int KIND, bool KEEP = false, class BSync>
__device__ __forceinline__ void zstage_body(cx<R> *__restrict__ work, R *__restrict__ stale,
                                            const cx<R> *__restrict__ twg, const Geo &g, R invn3,
                                            const Blk b, BSync bsync, unsigned char *smem,
                                            R *__restrict__ keep = nullptr) {
  using C = cx<R>;
  using Z = ZC<R, N, KIND>;
  constexpr int E = Z::E, T = Z::T;
  C *tw = (C *)smem;  // stage twiddles of the z plan (Z::TWN entries)
  build_stage_tw<N, typename Z::P>(tw, twg, N, b.tid, b.nt);
  bsync();
  const int lid = b.tid / T, t = b.tid % T;
  C *xb = tw + Z::TWN + lid * Z::XB;
  R *st = (R *)(tw + Z::TWN + Z::LINES * Z::XB) + lid * Z::STASH;
  // own points of staged field f: st[(f * E + e) * T + t]
  auto SU_ = [&](int f, int e) -> R & { return st[(f * E + e) * T + t]; };
  const long long line = (long long)b.x * Z::LINES + lid;
  const bool ok = line < (long long)N * N;
  work += (long long)b.y * g.run_spec;  // run of the batch
  stale += (long long)b.y * g.run_real;
  if constexpr (KEEP) keep += (long long)b.y * 6 * g.nreal;
  const long long off = line * g.nfp;
  const C *pU = work + SU * g.slot + off, *pV = work + SV * g.slot + off;
  const C *pW = work + SW * g.slot + off, *pOMZ = work + SOMZ * g.slot + off;
  const C *pDWDX = work + SDWDX * g.slot + off;
  const C *pDWDY = work + SDWDY * g.slot + off;
  auto ld = [&](const C *p, int s) -> C { return ok ? p[s] : czero<C>(); };
  auto f_ox = [&](int s) -> C {  // omega_x = dw/dy - i kz v
    const C a = ld(pDWDY, s), v = ld(pV, s);
    return cmk<C>(a.x + (R)s * v.y, a.y - (R)s * v.x);
  };
  auto f_oy = [&](int s) -> C {  // omega_y = i kz u - dw/dx
    const C u = ld(pU, s), b = ld(pDWDX, s);
    return cmk<C>(-(R)s * u.y - b.x, (R)s * u.x - b.y);
  };
  auto f_oz = [&](int s) -> C {  // omega_z = dv/dx - du/dy
    return ld(pOMZ, s);
  };
  auto f_zero = [&](int) -> C { return czero<C>(); };
  // L2 prefetch of a row of `bytes` starting on a 128-byte line: the next
  // pair's inputs are on their way from DRAM while this pair's FFT runs
  // (the waits on those loads were the pass's largest stall)
  auto pf = [&](const void *row, int bytes) {
    if (!ok) return;
    for (int l = t; l * 128 < bytes; l += T)
      asm volatile("prefetch.global.L2 [%0];" ::"l"((const char *)row + l * 128));
  };
  constexpr int ROWB = (N / 2 + 1) * (int)sizeof(C), REALB = N * (int)sizeof(R);
  const LineSync<(T > 32), BSync> sync{bsync};
  const PadShift<Z::PADSH> idx{};
  const long long roff = line * N;
  auto kp = [&](int f, int e, R v) {
    if constexpr (KEEP) {
      if (ok) keep[f * g.nreal + roff + t + T * e] = v;
    }
  };

  C y[E];
  if constexpr (Z::S2 || Z::F32) {
    if constexpr (KIND == 0) {
      // first stage: (omega_x, omega_y) with the stale real velocity read
      // where it is needed (L1/L2 hits the second time); N_z is complete
      // after this pair and leaves before (omega_z, 0)
      auto sv = [&](int f, int e) -> R { return ok ? stale[f * g.nreal + roff + t + T * e] : R(0); };
      R nx[E], ny[E];
      ext_pair<R, N, KIND>(y, t, f_ox, f_oy);
      pf(pOMZ, ROWB);
      pf(stale + roff, REALB);
      pf(stale + g.nreal + roff, REALB);
      pf(stale + 2 * g.nreal + roff, REALB);
      line_fft<N, typename Z::P, false>(y, t, tw, xb, idx, sync);
#pragma unroll
      for (int e = 0; e < E; e++) {
        const R ox = y[e].x * invn3, oy = y[e].y * invn3;
        const R u = sv(0, e), v = sv(1, e), w = sv(2, e);
        nx[e] = -w * oy;
        ny[e] = w * ox;
        y[e] = cmk<C>(u * oy - v * ox, R(0));  // N_z
        kp(3, e, ox);
        kp(4, e, oy);
      }
      zfwd_z<R, N, KIND>(y, t, tw, xb, idx, sync, work + off, g, ok);
      ext_pair<R, N, KIND>(y, t, f_oz, f_zero);
      line_fft<N, typename Z::P, false>(y, t, tw, xb, idx, sync);
#pragma unroll
      for (int e = 0; e < E; e++) {
        const R oz = y[e].x * invn3;
        y[e] = cmk<C>(nx[e] + sv(1, e) * oz, ny[e] - sv(0, e) * oz);  // (N_x, N_y)
        kp(5, e, oz);
      }
      zfwd_xy<R, N, KIND>(y, t, tw, xb, idx, sync, work + off, g, ok);
    } else {
      // middle and last stages: (u, omega_y), (v, omega_x): N_z = u oy - v ox
      // leaves; (w, omega_z): N_x = v oz - w oy, N_y = w ox - u oz formed in
      // place and leave.  The last stage stores the velocity as the next
      // stale one as it comes.
      R su[Z::S2 ? 1 : E], soy[Z::S2 ? 1 : E];  // FP32: (u, omega_y) in registers
      ext_gen<R, N, KIND>(y, t, [&](int s, C &a, C &b) {
        const C uu = ld(pU, s), d = ld(pDWDX, s);
        a = uu;
        b = cmk<C>(-(R)s * uu.y - d.x, (R)s * uu.x - d.y);  // i kz u - dw/dx
      });
      pf(pV, ROWB);
      pf(pDWDY, ROWB);
      line_fft<N, typename Z::P, false>(y, t, tw, xb, idx, sync);
#pragma unroll
      for (int e = 0; e < E; e++) {
        const R u = y[e].x * invn3, oy = y[e].y * invn3;
        if constexpr (Z::S2) {
          SU_(0, e) = u;
          SU_(1, e) = oy;
        } else {
          su[e] = u;
          soy[e] = oy;
        }
        if (KIND == 2 && ok) stale[roff + t + T * e] = u;
        kp(0, e, u);
        kp(4, e, oy);
      }
      auto U_ = [&](int e) -> R { if constexpr (Z::S2) return SU_(0, e); else return su[e]; };
      auto OY_ = [&](int e) -> R { if constexpr (Z::S2) return SU_(1, e); else return soy[e]; };
      ext_gen<R, N, KIND>(y, t, [&](int s, C &a, C &b) {
        const C vv = ld(pV, s), d = ld(pDWDY, s);
        a = vv;
        b = cmk<C>(d.x + (R)s * vv.y, d.y - (R)s * vv.x);  // dw/dy - i kz v
      });
      pf(pW, ROWB);
      pf(pOMZ, ROWB);
      line_fft<N, typename Z::P, false>(y, t, tw, xb, idx, sync);
      R sv_[E], sox[E];
#pragma unroll
      for (int e = 0; e < E; e++) {
        const R v = y[e].x * invn3, ox = y[e].y * invn3;
        sv_[e] = v;
        sox[e] = ox;
        const R nz = U_(e) * OY_(e);
        y[e] = cmk<C>(nz - v * ox, R(0));  // N_z
        if (KIND == 2 && ok) stale[g.nreal + roff + t + T * e] = v;
        kp(1, e, v);
        kp(3, e, ox);
      }
      zfwd_z<R, N, KIND>(y, t, tw, xb, idx, sync, work + off, g, ok);
      ext_gen<R, N, KIND>(y, t, [&](int s, C &a, C &b) {
        a = ld(pW, s);
        b = ld(pOMZ, s);
      });
      line_fft<N, typename Z::P, false>(y, t, tw, xb, idx, sync);
#pragma unroll
      for (int e = 0; e < E; e++) {
        const R w = y[e].x * invn3, oz = y[e].y * invn3;
        const R nx = -w * OY_(e), ny = -U_(e) * oz;
        y[e] = cmk<C>(nx + sv_[e] * oz, ny + w * sox[e]);  // (N_x, N_y)
        if (KIND == 2 && ok) stale[2 * g.nreal + roff + t + T * e] = w;
        kp(2, e, w);
        kp(5, e, oz);
      }
      zfwd_xy<R, N, KIND>(y, t, tw, xb, idx, sync, work + off, g, ok);
    }
  } else {
    // FP64 with 8 values per thread (n <= 64): N in registers, forward
    // transforms at the end
    R nx[E], ny[E], nz[E];
    if (KIND == 0) {
    // stale real velocity, own points m = t + T e
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int m = t + T * e;
#pragma unroll
      for (int f = 0; f < 3; f++) SU_(f, e) = ok ? stale[f * g.nreal + roff + m] : R(0);
    }
    ext_pair<R, N, KIND>(y, t, f_ox, f_oy);
    line_fft<N, typename Z::P, false>(y, t, tw, xb, idx, sync);
#pragma unroll
    for (int e = 0; e < E; e++) {
      const R ox = y[e].x * invn3, oy = y[e].y * invn3;
      const R u = SU_(0, e), v = SU_(1, e), w = SU_(2, e);
      nx[e] = -w * oy;
      ny[e] = w * ox;
      nz[e] = u * oy - v * ox;
    }
    ext_pair<R, N, KIND>(y, t, f_oz, f_zero);
    line_fft<N, typename Z::P, false>(y, t, tw, xb, idx, sync);
#pragma unroll
    for (int e = 0; e < E; e++) {
      const R oz = y[e].x * invn3;
      nx[e] += SU_(1, e) * oz;
      ny[e] -= SU_(0, e) * oz;
    }
    } else if (KIND == 1) {
    // Pairs ordered so that every input slot is read once and the cross
    // product accumulates in registers (FP32 last stage: the velocity is
    // stored as the next stale one as it comes):
    //   (u, omega_y): N_z = u oy
    //   (w, omega_z): N_x = -w oy, N_y = -u oz
    //   (v, omega_x): N_x += v oz, N_y += w ox, N_z -= v ox
    R u[E], oy[E];
    ext_gen<R, N, KIND>(y, t, [&](int s, C &a, C &b) {
      const C uu = ld(pU, s), d = ld(pDWDX, s);
      a = uu;
      b = cmk<C>(-(R)s * uu.y - d.x, (R)s * uu.x - d.y);  // i kz u - dw/dx
    });
    pf(pW, ROWB);
    pf(pOMZ, ROWB);
    line_fft<N, typename Z::P, false>(y, t, tw, xb, idx, sync);
#pragma unroll
    for (int e = 0; e < E; e++) {
      u[e] = y[e].x * invn3;
      oy[e] = y[e].y * invn3;
      nz[e] = u[e] * oy[e];
      if (KIND == 2 && ok) stale[roff + t + T * e] = u[e];
    }
    ext_gen<R, N, KIND>(y, t, [&](int s, C &a, C &b) {
      a = ld(pW, s);
      b = ld(pOMZ, s);
    });
    pf(pV, ROWB);
    pf(pDWDY, ROWB);
    line_fft<N, typename Z::P, false>(y, t, tw, xb, idx, sync);
    R w[E], oz[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      w[e] = y[e].x * invn3;
      oz[e] = y[e].y * invn3;
      nx[e] = -w[e] * oy[e];
      ny[e] = -u[e] * oz[e];
      if (KIND == 2 && ok) stale[2 * g.nreal + roff + t + T * e] = w[e];
    }
    ext_gen<R, N, KIND>(y, t, [&](int s, C &a, C &b) {
      const C vv = ld(pV, s), d = ld(pDWDY, s);
      a = vv;
      b = cmk<C>(d.x + (R)s * vv.y, d.y - (R)s * vv.x);  // dw/dy - i kz v
    });
    line_fft<N, typename Z::P, false>(y, t, tw, xb, idx, sync);
#pragma unroll
    for (int e = 0; e < E; e++) {
      const R v = y[e].x * invn3, ox = y[e].y * invn3;
      nx[e] += v * oz[e];
      ny[e] += w[e] * ox;
      nz[e] -= v * ox;
      if (KIND == 2 && ok) stale[g.nreal + roff + t + T * e] = v;
    }
    } else {
    // FP64 last stage at 8 values per thread: the velocity is also stored as
    // the next stale one, so it is staged in shared memory (the register-only
    // order above spills here)
    // (u, v)
    ext_pair<R, N, KIND>(y, t, [&](int s) { return ld(pU, s); }, [&](int s) { return ld(pV, s); });
    line_fft<N, typename Z::P, false>(y, t, tw, xb, idx, sync);
#pragma unroll
    for (int e = 0; e < E; e++) {
      SU_(0, e) = y[e].x * invn3;
      SU_(1, e) = y[e].y * invn3;
    }
    // (w, omega_x)
    ext_pair<R, N, KIND>(y, t, [&](int s) { return ld(pW, s); }, f_ox);
    line_fft<N, typename Z::P, false>(y, t, tw, xb, idx, sync);
#pragma unroll
    for (int e = 0; e < E; e++) {
      const R w = y[e].x * invn3, ox = y[e].y * invn3;
      SU_(2, e) = w;
      SU_(3, e) = w * ox;            // partial N_y
      SU_(4, e) = -SU_(1, e) * ox;   // partial N_z
    }
    // (omega_y, omega_z)
    ext_pair<R, N, KIND>(y, t, f_oy, f_oz);
    line_fft<N, typename Z::P, false>(y, t, tw, xb, idx, sync);
#pragma unroll
    for (int e = 0; e < E; e++) {
      const R oy = y[e].x * invn3, oz = y[e].y * invn3;
      const R u = SU_(0, e), v = SU_(1, e), w = SU_(2, e);
      nx[e] = v * oz - w * oy;
      ny[e] = SU_(3, e) - u * oz;
      nz[e] = SU_(4, e) + u * oy;
    }
    if (KIND == 2 && ok) {
#pragma unroll
      for (int e = 0; e < E; e++) {
        const int m = t + T * e;
#pragma unroll
        for (int f = 0; f < 3; f++) stale[f * g.nreal + roff + m] = SU_(f, e);
      }
    }
  }
    zstage_forward<R, N, KIND>(y, nx, ny, nz, t, tw, xb, idx, sync, work + off, g, ok);
  }
}

template <class R, int N, int KIND>
__global__ void __launch_bounds__(ZC<R, N, KIND>::THREADS, ZC<R, N, KIND>::MINB)
    k_zstage(cx<R> *__restrict__ work, R *__restrict__ stale, const cx<R> *__restrict__ twg, Geo g,
             R invn3) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  zstage_body<R, N, KIND>(work, stale, twg, g, invn3, launch_blk(), BlockSync{}, smem_raw);
}

// The z pass that also keeps the real velocity and vorticity (KEEP above),
// for the forward recomputation of the discrete adjoint; the pair orders of
// S2 and FP32 only.
template <class R, int N, int KIND>
__global__ void __launch_bounds__(ZC<R, N, KIND>::THREADS, ZC<R, N, KIND>::MINB)
    k_zstage_keep(cx<R> *__restrict__ work, R *__restrict__ stale, const cx<R> *__restrict__ twg,
                  Geo g, R invn3, R *__restrict__ keep) {
  static_assert(ZC<R, N, KIND>::S2 || ZC<R, N, KIND>::F32, "KEEP needs the S2 or FP32 pair order");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  zstage_body<R, N, KIND, true>(work, stale, twg, g, invn3, launch_blk(), BlockSync{}, smem_raw,
                                keep);
}

// ---------------------------------------------------------------------------
// E2: after the x forward transform of the three N slots (E1), the pointwise
// update of main.c:381-413 on the full half spectrum:
//   dU  = N * (mask * dt)
//   P   = kk > 0 ? (dU kx + dV ky + dW kz) / kk : 0
//   dU -= P kx + nu dt kk U_s          (same for V, W)
//   ST 0:   next = u0 + b0 dU,  acc = u0 + a0 dU      (u_s == u0)
//   ST 1,2: next = u0 + b dU,   acc += a dU
//   ST 3:   u0   = acc + a3 dU   (the state of the next step)
// A pure streaming kernel, one thread per half-spectrum point (two in FP32).
// The FP64 path computes in FP64; the mixed path computes in FP32 with the
// viscous coefficient nu dt |k|^2 formed in FP64 (update_point_f32).
// ---------------------------------------------------------------------------
// pointers are those of run 0; run r adds r * run_spec.  coef[2 r] = nu,
// coef[2 r + 1] = dt of run r (device memory, so a captured graph picks up
// new values without being rebuilt).
template <class R>
struct StageArgs {
  cx<R> *u0;    // step start state (3 slots); ST 3 writes the new state here
  cx<R> *us;    // stage input (3 slots)
  cx<R> *acc;   // RK accumulator (3 slots)
  cx<R> *next;  // next stage input (3 slots)
  cx<R> *ph;    // pressure slot or nullptr
  const double *coef;
  double a, b;  // RK coefficients of the stage (main.c:15-16)
};

// Inputs and results of one point.  A thread loads every input of its
// points before the first store: as far as the compiler knows the stores may
// alias later inputs, which would otherwise hold loads back behind them.
template <class R>
struct UpdIn {
  cx<R> n[3];   // N slots (E1 output)
  cx<R> us[3];  // stage input
  cx<R> z[3];   // u0 (ST 1, 2)
  cx<R> a[3];   // accumulator (ST 1, 2, 3)
};
template <class R>
struct UpdOut {
  cx<R> o1[3];  // next stage input (ST 0-2) or the new state (ST 3)
  cx<R> o2[3];  // accumulator (ST 0-2)
  cx<R> p;      // pressure
};

template <class R, int ST>
__device__ __forceinline__ void update_point(const UpdIn<R> &in, UpdOut<R> &out, const Geo &g,
                                             const StageArgs<R> &sa, double nu, double dt, int i,
                                             int j, int col) {
  using C = cx<R>;
  const int ikx = kwave(i, g.n), iky = kwave(j, g.n);
  const double kx = (double)ikx, ky = (double)iky, kz = (double)col;
  const bool inm = (ikx < 0 ? -ikx : ikx) <= g.kcut && (iky < 0 ? -iky : iky) <= g.kcut &&
                   col <= g.kcut;
  // main.c multiplies by the 0/1 mask; N is selected instead, because the
  // forward passes leave the entries outside the 2/3 rule unwritten
  const double2 zero = make_double2(0.0, 0.0);
  double2 du = inm ? cscale(to_d(in.n[0]), dt) : zero;
  double2 dv = inm ? cscale(to_d(in.n[1]), dt) : zero;
  double2 dw = inm ? cscale(to_d(in.n[2]), dt) : zero;
  const double kk = kx * kx + ky * ky + kz * kz;
  double2 P;
  if (kk > 0) {
    P.x = (du.x * kx + dv.x * ky + dw.x * kz) / kk;
    P.y = (du.y * kx + dv.y * ky + dw.y * kz) / kk;
  } else {
    P = make_double2(0.0, 0.0);
  }
  const double c = nu * dt * kk;
  const double2 us0 = to_d(in.us[0]), us1 = to_d(in.us[1]), us2 = to_d(in.us[2]);
  du = make_double2(du.x - (P.x * kx + c * us0.x), du.y - (P.y * kx + c * us0.y));
  dv = make_double2(dv.x - (P.x * ky + c * us1.x), dv.y - (P.y * ky + c * us1.y));
  dw = make_double2(dw.x - (P.x * kz + c * us2.x), dw.y - (P.y * kz + c * us2.y));
  out.p = from_d<C>(P);
  auto axpy = [](double2 x, double s, double2 y) {
    return make_double2(x.x + s * y.x, x.y + s * y.y);
  };
  const double2 d[3] = {du, dv, dw};
#pragma unroll
  for (int f = 0; f < 3; f++) {
    if (ST == 0) {  // us == u0
      const double2 u = to_d(in.us[f]);
      out.o1[f] = from_d<C>(axpy(u, sa.b, d[f]));
      out.o2[f] = from_d<C>(axpy(u, sa.a, d[f]));
    } else if (ST < 3) {
      out.o1[f] = from_d<C>(axpy(to_d(in.z[f]), sa.b, d[f]));
      out.o2[f] = from_d<C>(axpy(to_d(in.a[f]), sa.a, d[f]));
    } else {
      out.o1[f] = from_d<C>(axpy(to_d(in.a[f]), sa.a, d[f]));
    }
  }
}

// The mixed path's update: FP32 arithmetic for the projection and the RK
// axpys (the storage precision), FP64 only for the viscous coefficient
// nu dt |k|^2, which is formed in FP64 and rounded once.  |k|^2 and the
// wavenumbers are integers below 2^24, exact in FP32; dt and the RK
// coefficients are rounded once per launch (rk = (dt, a, b) as floats).
template <int ST>
__device__ __forceinline__ void update_point_f32(const UpdIn<float> &in, UpdOut<float> &out,
                                                 const Geo &g, float dtf, double nudt, float ra,
                                                 float rb, int i, int j, int col) {
  const int ikx = kwave(i, g.n), iky = kwave(j, g.n);
  const float kx = (float)ikx, ky = (float)iky, kz = (float)col;
  const bool inm = (ikx < 0 ? -ikx : ikx) <= g.kcut && (iky < 0 ? -iky : iky) <= g.kcut &&
                   col <= g.kcut;
  const float2 zero = make_float2(0.f, 0.f);
  float2 du = inm ? cscale(in.n[0], dtf) : zero;
  float2 dv = inm ? cscale(in.n[1], dtf) : zero;
  float2 dw = inm ? cscale(in.n[2], dtf) : zero;
  const int ikk = ikx * ikx + iky * iky + col * col;
  const float kk = (float)ikk;
  float2 P;
  if (ikk > 0) {
    P.x = __fdiv_rn(du.x * kx + dv.x * ky + dw.x * kz, kk);
    P.y = __fdiv_rn(du.y * kx + dv.y * ky + dw.y * kz, kk);
  } else {
    P = zero;
  }
  const float c = (float)(nudt * (double)ikk);
  du = make_float2(du.x - (P.x * kx + c * in.us[0].x), du.y - (P.y * kx + c * in.us[0].y));
  dv = make_float2(dv.x - (P.x * ky + c * in.us[1].x), dv.y - (P.y * ky + c * in.us[1].y));
  dw = make_float2(dw.x - (P.x * kz + c * in.us[2].x), dw.y - (P.y * kz + c * in.us[2].y));
  out.p = P;
  auto axpy = [](float2 x, float s, float2 y) { return make_float2(x.x + s * y.x, x.y + s * y.y); };
  const float2 d[3] = {du, dv, dw};
#pragma unroll
  for (int f = 0; f < 3; f++) {
    if (ST == 0) {  // us == u0
      out.o1[f] = axpy(in.us[f], rb, d[f]);
      out.o2[f] = axpy(in.us[f], ra, d[f]);
    } else if (ST < 3) {
      out.o1[f] = axpy(in.z[f], rb, d[f]);
      out.o2[f] = axpy(in.a[f], ra, d[f]);
    } else {
      out.o1[f] = axpy(in.a[f], ra, d[f]);
    }
  }
}

constexpr int UPD_THREADS = 128;
// adjacent points per vector access: two float2 make one 16-byte access
template <class R>
struct UpdVec;
template <>
struct UpdVec<double> {
  static constexpr int VP = 1;
  using T = double2;
  __device__ static double2 get(const T &v, int) { return v; }
  __device__ static T pack(const double2 *c) { return c[0]; }
};
template <>
struct UpdVec<float> {
  static constexpr int VP = 2;
  using T = float4;
  __device__ static float2 get(const T &v, int k) {
    return k ? make_float2(v.z, v.w) : make_float2(v.x, v.y);
  }
  __device__ static T pack(const float2 *c) { return make_float4(c[0].x, c[0].y, c[1].x, c[1].y); }
};

// grid: (ceil(n^2 nfp / VP / UPD_THREADS), nruns).  Thread = VP adjacent
// points of the padded slot (padding columns included and skipped), so that
// the row, kx and ky of a point come from divisions by compile-time constants.
// One chunk of UPD_THREADS threads: chunk b.x of run b.y.
template <class R, int N, int ST>
__device__ __forceinline__ void update_body(const cx<R> *__restrict__ nl, const Geo &g,
                                            const StageArgs<R> &sa, const Blk b) {
  using VT = UpdVec<R>;
  using V = typename VT::T;
  constexpr int VP = VT::VP;
  constexpr int NF = N / 2 + 1;
  constexpr int NFP = (NF + PitchW<R>::W - 1) / PitchW<R>::W * PitchW<R>::W;
  constexpr unsigned NPAD = (unsigned)N * N * NFP;
  static_assert(NFP % VP == 0, "vector access must not straddle rows");
  const unsigned q0 = ((unsigned)b.x * (unsigned)UPD_THREADS + (unsigned)b.tid) * VP;
  if (q0 >= NPAD) return;
  const unsigned row = q0 / NFP;
  const int col0 = (int)(q0 - row * NFP);
  if (col0 >= NF) return;
  const long long rb = (long long)b.y * g.run_spec;
  const double nu = sa.coef[2 * b.y], dt = sa.coef[2 * b.y + 1];
  const long long vo = (rb + q0) / VP, vs = g.slot / VP;  // vector index, slot stride
  const V *vn = (const V *)nl, *vus = (const V *)sa.us, *vz = (const V *)sa.u0,
          *va = (const V *)sa.acc;
  V ln[3], lus[3], lz[3], la[3];
  // N is read only where some point of the access lies inside the 2/3 rule
  const int ikx = kwave((int)(row / N), N), iky = kwave((int)(row % N), N);
  const bool need_n = (ikx < 0 ? -ikx : ikx) <= g.kcut && (iky < 0 ? -iky : iky) <= g.kcut &&
                      col0 <= g.kcut;
#pragma unroll
  for (int f = 0; f < 3; f++) {
    ln[f] = need_n ? vn[f * vs + vo] : V{};
    lus[f] = vus[f * vs + vo];
    if (ST == 1 || ST == 2) lz[f] = vz[f * vs + vo];
    if (ST != 0) la[f] = va[f * vs + vo];
  }
  UpdOut<R> res[VP];
#pragma unroll
  for (int v = 0; v < VP; v++) {
    if (col0 + v < NF) {
      UpdIn<R> in;
#pragma unroll
      for (int f = 0; f < 3; f++) {
        in.n[f] = VT::get(ln[f], v);
        in.us[f] = VT::get(lus[f], v);
        if (ST == 1 || ST == 2) in.z[f] = VT::get(lz[f], v);
        if (ST != 0) in.a[f] = VT::get(la[f], v);
      }
      if constexpr (sizeof(R) == 4)
        update_point_f32<ST>(in, res[v], g, (float)dt, nu * dt, (float)sa.a, (float)sa.b,
                             (int)(row / N), (int)(row % N), col0 + v);
      else
        update_point<R, ST>(in, res[v], g, sa, nu, dt, (int)(row / N), (int)(row % N), col0 + v);
    }
  }
  V *o1 = (V *)(ST == 3 ? sa.u0 : sa.next), *o2 = (V *)sa.acc, *vp = (V *)sa.ph;
  if (col0 + VP - 1 < NF) {
    cx<R> t1[VP], t2[VP], tp[VP];
#pragma unroll
    for (int f = 0; f < 3; f++) {
#pragma unroll
      for (int v = 0; v < VP; v++) {
        t1[v] = res[v].o1[f];
        t2[v] = res[v].o2[f];
      }
      o1[f * vs + vo] = VT::pack(t1);
      if (ST != 3) o2[f * vs + vo] = VT::pack(t2);
    }
    if (vp) {
#pragma unroll
      for (int v = 0; v < VP; v++) tp[v] = res[v].p;
      vp[vo] = VT::pack(tp);
    }
  } else {  // the row's last valid column: store its point alone
    const long long o = rb + q0;
    cx<R> *s1 = ST == 3 ? sa.u0 : sa.next;
#pragma unroll
    for (int f = 0; f < 3; f++) {
      s1[f * g.slot + o] = res[0].o1[f];
      if (ST != 3) sa.acc[f * g.slot + o] = res[0].o2[f];
    }
    if (sa.ph) sa.ph[o] = res[0].p;
  }
}

template <class R, int N, int ST>
__global__ void __launch_bounds__(UPD_THREADS)
    k_update(const cx<R> *__restrict__ nl, Geo g, StageArgs<R> sa) {
  update_body<R, N, ST>(nl, g, sa, launch_blk());
}

// ---------------------------------------------------------------------------
// Energy / enstrophy (main.c:257-266): sums over the half spectrum of
//   e = |U|^2 + |V|^2 + |W|^2   and   kk * e,
// each term rounded like the reference's double expression (no FMA), summed
// in double-double (error-free TwoSum), block partials then one final block.
// FP32 storage is widened to FP64 first.
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
__device__ __forceinline__ double cabs2_rn(double2 z) {
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

// grid: (blocks per run, nruns); partials [run][gridDim.x]
template <int BS, class C>
__global__ void __launch_bounds__(BS)
    k_diag(const C *__restrict__ u, Geo g, double4 *__restrict__ partial) {
  u += (long long)blockIdx.y * g.run_spec;
  partial += (long long)blockIdx.y * gridDim.x;
  DD e{0.0, 0.0}, o{0.0, 0.0};
  const int n = g.n;
  const long long npts = (long long)n * n * g.nf;
  for (long long q = (long long)blockIdx.x * BS + threadIdx.x; q < npts;
       q += (long long)gridDim.x * BS) {
    const long long row = q / g.nf;
    const int k = (int)(q - row * g.nf);
    const int i = (int)(row / n), j = (int)(row % n);
    const long long l = row * g.nfp + k;
    const double s = __dadd_rn(__dadd_rn(cabs2_rn(to_d(u[l])), cabs2_rn(to_d(u[g.slot + l]))),
                               cabs2_rn(to_d(u[2 * g.slot + l])));
    const double kx = kwave(i, n), ky = kwave(j, n), kz = k;
    const double kk = __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
    e = dd_add_d(e, s);
    o = dd_add_d(o, __dmul_rn(kk, s));
  }
  dd_block_reduce<BS>(e, o, partial + blockIdx.x);
}

// grid: (nruns); out[run]
template <int BS>
__global__ void __launch_bounds__(BS) k_diag_final(const double4 *__restrict__ partial, int np,
                                                   double4 *__restrict__ out) {
  partial += (long long)blockIdx.x * np;
  out += blockIdx.x;
  DD e{0.0, 0.0}, o{0.0, 0.0};
  for (int q = threadIdx.x; q < np; q += BS) {
    const double4 v = partial[q];
    e = dd_add(e, DD{v.x, v.y});
    o = dd_add(o, DD{v.z, v.w});
  }
  dd_block_reduce<BS>(e, o, out);
}

// ---------------------------------------------------------------------------
// Precision conversions for the FP32 path (host data is always float64).
// ---------------------------------------------------------------------------
template <class A, class B>
__global__ void k_real_convert(const A *__restrict__ in, B *__restrict__ out, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    out[q] = (B)in[q];
}
// spectral: nfields padded slots (type C, pitch nfp) <-> unpadded double2
// [nfields][n][n][nf]; TO_PADDED selects the direction
template <class C, bool TO_PADDED>
__global__ void k_spec_convert(C *__restrict__ padded, double2 *__restrict__ dense, Geo g,
                               int nfields) {
  const long long per = (long long)g.n * g.n * g.nf;
  const long long total = per * nfields;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const long long f = q / per, r = q - f * per;
    const long long row = r / g.nf;
    const long long l = f * g.slot + row * g.nfp + (r - row * g.nf);
    if (TO_PADDED)
      padded[l] = from_d<C>(dense[q]);
    else
      dense[q] = to_d(padded[l]);
  }
}

}  // namespace dnsb
