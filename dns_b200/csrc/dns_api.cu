// dns_api.cu -- context, launch orchestration (CUDA graphs) and the C ABI
// declared in include/dns_b200.h.
//
// Device memory of a context is one arena:
//   spectral slots, each [n][n][nfp] complex (double2 for DNS_PREC_FP64,
//   float2 for DNS_PREC_MIXED):
//     0..2   SA   state at the start of a step (U_hat, V_hat, W_hat)
//     3..5   SB   RK stage input (main.c's U_hat during stages 1-3)
//     6..8   ACC  RK accumulator (main.c's U_hat1)
//     9..15  WORK seven partially transformed fields of the stage
//     16     P    pressure of the last stage
//   stale real velocity [3][n^3] (main.c's U, V, W between steps)
//   twiddles, reduction partials.
// main.c's U_hat0 is SA itself: stage 0 reads SA and writes SB/ACC, stage 3
// writes the new state back into SA, so the copies of main.c:334-342 and
// main.c:415-420 disappear.
#include "dns_b200.h"
#include "kernels.cuh"

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

using namespace dnsb;

namespace {

thread_local std::string g_last_error;

enum { SLOT_SA = 0, SLOT_SB = 3, SLOT_ACC = 6, SLOT_WORK = 9, SLOT_P = 16, NSLOTS = 17 };
// per RK stage: A x-inverse, B y-inverse, C z fused, D y-forward,
// E1 x-forward, E2 pointwise update
enum { KERNELS_PER_STAGE = 6 };

int fail(int code, const char *what, const char *file, int line) {
  char buf[512];
  snprintf(buf, sizeof buf, "%s (%s:%d)", what, file, line);
  g_last_error = buf;
  return code;
}

#define CK(call)                                                                     \
  do {                                                                               \
    cudaError_t err_ = (call);                                                       \
    if (err_ != cudaSuccess) {                                                       \
      return fail(DNS_ERR_CUDA, cudaGetErrorString(err_), __FILE__, __LINE__);       \
    }                                                                                \
  } while (0)

// cos(2 pi k / n), sin(2 pi k / n): long double with octant reduction so that
// the symmetric values (0, +-1, sqrt(1/2)) are exact, rounded once to double.
void sincos2pi(long k, long n, double *c, double *s) {
  const long double PI_L = 3.141592653589793238462643383279502884L;
  k %= n;
  if (k < 0) k += n;
  const long q = (4 * k) / n, r = (4 * k) % n;
  long double cc, ss;
  if (r == 0) {
    cc = 1.0L;
    ss = 0.0L;
  } else if (2 * r <= n) {
    const long double x = (PI_L / 2.0L) * (long double)r / (long double)n;
    cc = cosl(x);
    ss = sinl(x);
  } else {
    const long double x = (PI_L / 2.0L) * (long double)(n - r) / (long double)n;
    cc = sinl(x);
    ss = cosl(x);
  }
  const double c0 = (double)cc, s0 = (double)ss;
  switch (q) {
    case 0: *c = c0; *s = s0; break;
    case 1: *c = -s0; *s = c0; break;
    case 2: *c = -c0; *s = -s0; break;
    default: *c = s0; *s = -c0; break;
  }
}

}  // namespace

namespace dnsb {
void set_last_error(const char *msg) { g_last_error = msg; }
}  // namespace dnsb

struct dns_ctx {
  long n = 0;
  int precision = 0;
  unsigned flags = 0;
  int device = 0;
  size_t csize = 16;      // bytes of one complex element
  size_t rsize = 8;       // bytes of one real element
  Geo g{};
  cudaStream_t stream = nullptr;
  char *arena = nullptr;
  size_t arena_bytes = 0;
  void *S = nullptr;      // spectral slots
  void *stale = nullptr;  // stale real velocity
  void *tw = nullptr;     // twiddles exp(-2 pi i k / n)
  double4 *diag_part = nullptr, *diag_out = nullptr;
  int diag_blocks = 0;
  double4 *diag_host = nullptr;  // pinned
  double *realbuf = nullptr;     // [4][n^3] float64, allocated on first dns_get_fields
  bool have_state = false;
  cudaGraphExec_t graph = nullptr;
  double graph_nu = 0, graph_dt = 0;
  int kernels_per_step = 4 * KERNELS_PER_STAGE;

  char *slot_ptr(int s) const { return (char *)S + (size_t)s * g.slot * csize; }
  // float64 staging for host transfers of the FP32 path: the work slots
  // (7 * n^2 * nfp * 8 bytes >= 3 n^3 * 8 and >= 3 n^2 nf * 16)
  double *staging() const { return (double *)slot_ptr(SLOT_WORK); }
};

namespace {

constexpr double RK_A[4] = {1 / 6.0, 1 / 3.0, 1 / 3.0, 1 / 6.0};  // main.c:15
constexpr double RK_B[3] = {0.5, 0.5, 1.0};                       // main.c:16

ColJobs jobs_empty() {
  ColJobs j;
  for (int q = 0; q < 8; q++) j.in_slot[q] = 0, j.out_slot[q] = -1, j.der_slot[q] = -1;
  return j;
}
ColJobs jobs_pass_a(int in0) {
  ColJobs j = jobs_empty();
  const int w = SLOT_WORK;
  j.in_slot[0] = in0 + 0; j.out_slot[0] = w + SU;
  j.in_slot[1] = in0 + 1; j.out_slot[1] = w + SV; j.der_slot[1] = w + SDVDX;
  j.in_slot[2] = in0 + 2; j.out_slot[2] = w + SW; j.der_slot[2] = w + SDWDX;
  return j;
}
ColJobs jobs_pass_b(bool first) {
  ColJobs j = jobs_empty();
  const int w = SLOT_WORK;
  j.in_slot[0] = w + SU; j.out_slot[0] = w + SU; j.der_slot[0] = w + SDUDY;
  j.in_slot[1] = w + SV; j.out_slot[1] = w + SV;
  // the first stage reads the stale real velocity, so W itself is not needed
  j.in_slot[2] = w + SW; j.out_slot[2] = first ? -1 : w + SW; j.der_slot[2] = w + SDWDY;
  j.in_slot[3] = w + SDVDX; j.out_slot[3] = w + SDVDX;
  j.in_slot[4] = w + SDWDX; j.out_slot[4] = w + SDWDX;
  return j;
}
ColJobs jobs_map(const int *in, const int *out, int cnt) {
  ColJobs j = jobs_empty();
  for (int q = 0; q < cnt; q++) j.in_slot[q] = in[q], j.out_slot[q] = out[q];
  return j;
}

template <class R, int N>
struct Ops {
  using C = cx<R>;
  static constexpr int W = ColW<R>::W;
  static constexpr int E = Plan<N>::E;
  static constexpr int CT = (N / E) * W;
  static constexpr size_t COL_SMEM = (size_t)(N + N * W) * sizeof(C);
  static constexpr size_t Z_SMEM = (size_t)(2 * N + ZCfg<N>::LINES * ZCfg<N>::XB) * sizeof(C);
  static constexpr size_t ZS_SMEM = ZC<R, N>::SMEM;

  template <class K>
  static cudaError_t allow(K kern, size_t smem) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  static cudaError_t setup() {
    cudaError_t e;
    if ((e = allow(k_colpass<R, N, 0, false>, COL_SMEM))) return e;
    if ((e = allow(k_colpass<R, N, 0, true>, COL_SMEM))) return e;
    if ((e = allow(k_colpass<R, N, 1, false>, COL_SMEM))) return e;
    if ((e = allow(k_colpass<R, N, 1, true>, COL_SMEM))) return e;
    if ((e = allow(k_zstage<R, N, 0>, ZS_SMEM))) return e;
    if ((e = allow(k_zstage<R, N, 1>, ZS_SMEM))) return e;
    if ((e = allow(k_zstage<R, N, 2>, ZS_SMEM))) return e;
    if ((e = allow(k_zr2c<R, N>, Z_SMEM))) return e;
    if ((e = allow(k_zc2r<R, N>, Z_SMEM))) return e;
    return cudaSuccess;
  }

  static C *S(dns_ctx *c) { return (C *)c->S; }
  static C *slot(dns_ctx *c, int s) { return S(c) + (long long)s * c->g.slot; }
  static const C *tw(dns_ctx *c) { return (const C *)c->tw; }

  template <int AXIS, bool FWD>
  static void colpass(dns_ctx *c, const ColJobs &jobs, int njobs) {
    dim3 grid(c->g.nfp / W, N, njobs);
    k_colpass<R, N, AXIS, FWD><<<grid, CT, COL_SMEM, c->stream>>>(S(c), S(c), tw(c), c->g, jobs);
  }

  static dim3 zgrid(int nfields) { return dim3((N * N) / ZCfg<N>::LINES, nfields); }
  static dim3 zsgrid() { return dim3((N * N + ZC<R, N>::LINES - 1) / ZC<R, N>::LINES); }

  // kernel `k` (0..KERNELS_PER_STAGE-1) of RK stage `s`
  static void stage_kernel(dns_ctx *c, int s, int k, double nu, double dt) {
    const Geo &g = c->g;
    C *work = slot(c, SLOT_WORK);
    R *stale = (R *)c->stale;
    const R invn3 = (R)(1.0 / (double)g.nreal);
    switch (k) {
      case 0:
        colpass<0, false>(c, jobs_pass_a(s == 0 ? SLOT_SA : SLOT_SB), 3);
        break;
      case 1:
        colpass<1, false>(c, jobs_pass_b(s == 0), 5);
        break;
      case 2:
        if (s == 0)
          k_zstage<R, N, 0><<<zsgrid(), ZC<R, N>::THREADS, ZS_SMEM, c->stream>>>(work, stale, tw(c), g, invn3);
        else if (s < 3)
          k_zstage<R, N, 1><<<zsgrid(), ZC<R, N>::THREADS, ZS_SMEM, c->stream>>>(work, stale, tw(c), g, invn3);
        else
          k_zstage<R, N, 2><<<zsgrid(), ZC<R, N>::THREADS, ZS_SMEM, c->stream>>>(work, stale, tw(c), g, invn3);
        break;
      case 3:
      case 4: {
        // D: y forward, E1: x forward (in place on the three N slots)
        const int io[3] = {SLOT_WORK + SU, SLOT_WORK + SV, SLOT_WORK + SW};
        if (k == 3)
          colpass<1, true>(c, jobs_map(io, io, 3), 3);
        else
          colpass<0, true>(c, jobs_map(io, io, 3), 3);
        break;
      }
      default: {
        StageArgs<R> sa;
        sa.u0 = slot(c, SLOT_SA);
        sa.us = slot(c, s == 0 ? SLOT_SA : SLOT_SB);
        sa.acc = slot(c, SLOT_ACC);
        sa.next = slot(c, SLOT_SB);
        sa.ph = (s == 3 && (c->flags & DNS_FLAG_PRESSURE)) ? slot(c, SLOT_P) : nullptr;
        sa.nu = nu;
        sa.dt = dt;
        sa.a = RK_A[s];
        sa.b = s < 3 ? RK_B[s] : 0.0;
        const long long npts = (long long)N * N * g.nf;
        const int per = UPD_THREADS * UPD_PER_THREAD;
        dim3 grid((unsigned)((npts + per - 1) / per));
        switch (s) {
          case 0: k_update<R, 0><<<grid, UPD_THREADS, 0, c->stream>>>(work, g, sa); break;
          case 1: k_update<R, 1><<<grid, UPD_THREADS, 0, c->stream>>>(work, g, sa); break;
          case 2: k_update<R, 2><<<grid, UPD_THREADS, 0, c->stream>>>(work, g, sa); break;
          default: k_update<R, 3><<<grid, UPD_THREADS, 0, c->stream>>>(work, g, sa); break;
        }
      }
    }
  }

  static void step(dns_ctx *c, double nu, double dt) {
    for (int s = 0; s < 4; s++)
      for (int k = 0; k < KERNELS_PER_STAGE; k++) stage_kernel(c, s, k, nu, dt);
  }

  // forward transform of the three stale real slots into SA
  static void forward(dns_ctx *c) {
    k_zr2c<R, N><<<zgrid(3), ZCfg<N>::THREADS, Z_SMEM, c->stream>>>((const R *)c->stale,
                                                                     slot(c, SLOT_WORK), tw(c), c->g);
    const int w3[3] = {SLOT_WORK + 0, SLOT_WORK + 1, SLOT_WORK + 2};
    const int sa[3] = {SLOT_SA + 0, SLOT_SA + 1, SLOT_SA + 2};
    colpass<1, true>(c, jobs_map(w3, w3, 3), 3);
    colpass<0, true>(c, jobs_map(w3, sa, 3), 3);
  }

  // c2r(X) / n^3 of SA (and P) into realbuf [4][n^3] float64
  static void backward(dns_ctx *c, int nfields) {
    const int in[4] = {SLOT_SA + 0, SLOT_SA + 1, SLOT_SA + 2, SLOT_P};
    const int w4[4] = {SLOT_WORK + 0, SLOT_WORK + 1, SLOT_WORK + 2, SLOT_WORK + 3};
    colpass<0, false>(c, jobs_map(in, w4, nfields), nfields);
    colpass<1, false>(c, jobs_map(w4, w4, nfields), nfields);
    k_zc2r<R, N><<<zgrid(nfields), ZCfg<N>::THREADS, Z_SMEM, c->stream>>>(
        slot(c, SLOT_WORK), c->realbuf, tw(c), c->g, 1.0 / (double)c->g.nreal);
  }

  static void diag(dns_ctx *c) {
    k_diag<256, C><<<c->diag_blocks, 256, 0, c->stream>>>(slot(c, SLOT_SA), c->g, c->diag_part);
    k_diag_final<256><<<1, 256, 0, c->stream>>>(c->diag_part, c->diag_blocks, c->diag_out);
  }
};

template <class F>
bool dispatch_n(int prec, long n, F &&f) {
  auto go = [&](auto r) -> bool {
    using R = decltype(r);
    switch (n) {
      case 8: f(Ops<R, 8>{}); return true;
      case 16: f(Ops<R, 16>{}); return true;
      case 32: f(Ops<R, 32>{}); return true;
      case 64: f(Ops<R, 64>{}); return true;
      case 128: f(Ops<R, 128>{}); return true;
      case 256: f(Ops<R, 256>{}); return true;
      case 512: f(Ops<R, 512>{}); return true;
      default: return false;
    }
  };
  if (prec == DNS_PREC_FP64) return go(double{});
  if (prec == DNS_PREC_MIXED) return go(float{});
  return false;
}
template <class F>
bool dispatch(dns_ctx *c, F &&f) {
  return dispatch_n(c->precision, c->n, f);
}

int check_launch(const char *file, int line) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(DNS_ERR_CUDA, cudaGetErrorString(e), file, line);
  return DNS_OK;
}
#define CKL()                                          \
  do {                                                 \
    int st_ = check_launch(__FILE__, __LINE__);        \
    if (st_ != DNS_OK) return st_;                     \
  } while (0)

int build_graph(dns_ctx *c, double nu, double dt) {
  if (c->graph && c->graph_nu == nu && c->graph_dt == dt) return DNS_OK;
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  cudaGraph_t gr;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  dispatch(c, [&](auto ops) { decltype(ops)::step(c, nu, dt); });
  cudaError_t le = cudaGetLastError();
  cudaError_t ce = cudaStreamEndCapture(c->stream, &gr);
  if (le != cudaSuccess) return fail(DNS_ERR_CUDA, cudaGetErrorString(le), __FILE__, __LINE__);
  CK(ce);
  cudaError_t ie = cudaGraphInstantiate(&c->graph, gr, 0);
  cudaGraphDestroy(gr);
  CK(ie);
  c->graph_nu = nu;
  c->graph_dt = dt;
  return DNS_OK;
}

unsigned conv_blocks(long long n) {
  long long b = (n + 255) / 256;
  return (unsigned)(b < 148 * 16 ? b : 148 * 16);
}

// host float64 [3][n^3] -> stale real slots (converted for the FP32 path)
int upload_real3(dns_ctx *c, const double *const src[3]) {
  const long long nr = c->g.nreal;
  const size_t fb = (size_t)nr * sizeof(double);
  double *dst = c->precision == DNS_PREC_FP64 ? (double *)c->stale : c->staging();
  for (int f = 0; f < 3; f++)
    CK(cudaMemcpyAsync(dst + f * nr, src[f], fb, cudaMemcpyHostToDevice, c->stream));
  if (c->precision != DNS_PREC_FP64) {
    k_real_convert<double, float><<<conv_blocks(3 * nr), 256, 0, c->stream>>>(dst, (float *)c->stale, 3 * nr);
    CKL();
  }
  return DNS_OK;
}

}  // namespace

extern "C" {

const char *dns_strerror(int status) {
  switch (status) {
    case DNS_OK: return "success";
    case DNS_ERR_ARG: return "invalid argument";
    case DNS_ERR_UNSUPPORTED: return "unsupported grid size or precision";
    case DNS_ERR_CUDA: return "CUDA error";
    case DNS_ERR_NOMEM: return "out of memory";
    case DNS_ERR_NONFINITE: return "non-finite energy or enstrophy";
    case DNS_ERR_STATE: return "call out of order";
    default: return "unknown status";
  }
}

const char *dns_last_error(void) { return g_last_error.c_str(); }

int dns_create(long n, int precision, unsigned flags, dns_ctx **out) {
  if (!out) return fail(DNS_ERR_ARG, "out is NULL", __FILE__, __LINE__);
  *out = nullptr;
  if (precision != DNS_PREC_FP64 && precision != DNS_PREC_MIXED)
    return fail(DNS_ERR_UNSUPPORTED, "precision not supported", __FILE__, __LINE__);
  cudaError_t se = cudaErrorInvalidValue;
  if (!dispatch_n(precision, n, [&](auto ops) { se = decltype(ops)::setup(); })) {
    char buf[128];
    snprintf(buf, sizeof buf, "n = %ld is not supported (powers of two 8..512)", n);
    return fail(DNS_ERR_UNSUPPORTED, buf, __FILE__, __LINE__);
  }
  CK(se);
  dns_ctx *c = new dns_ctx();
  c->n = n;
  c->precision = precision;
  c->flags = flags;
  const bool fp64 = precision == DNS_PREC_FP64;
  c->csize = fp64 ? sizeof(double2) : sizeof(float2);
  c->rsize = fp64 ? sizeof(double) : sizeof(float);
  const int W = fp64 ? ColW<double>::W : ColW<float>::W;
  cudaGetDevice(&c->device);
  Geo &g = c->g;
  g.n = (int)n;
  g.nf = (int)(n / 2 + 1);
  g.nfp = (g.nf + W - 1) / W * W;
  g.slot = (long long)n * n * g.nfp;
  g.nreal = (long long)n * n * n;
  // 2/3 rule of main.c:231-238: keep |k| < kmax with kmax = 2/3 (n/2 + 1)
  const double kmax = 2. / 3. * (n / 2 + 1);
  int kcut = -1;
  while ((double)(kcut + 1) < kmax) kcut++;
  g.kcut = kcut;
  const long long npts = (long long)n * n * g.nf;
  c->diag_blocks = (int)((npts + 255) / 256 < 1184 ? (npts + 255) / 256 : 1184);

  const size_t slot_b = (size_t)g.slot * c->csize;
  const size_t spec_b = slot_b * NSLOTS;
  const size_t stale_b = (size_t)g.nreal * 3 * c->rsize;
  const size_t tw_b = (size_t)n * c->csize;
  const size_t part_b = (size_t)c->diag_blocks * sizeof(double4) + sizeof(double4);
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  c->arena_bytes = al(spec_b) + al(stale_b) + al(tw_b) + al(part_b);
  cudaError_t e = cudaMalloc((void **)&c->arena, c->arena_bytes);
  if (e != cudaSuccess) {
    delete c;
    return fail(DNS_ERR_NOMEM, cudaGetErrorString(e), __FILE__, __LINE__);
  }
  char *p = c->arena;
  c->S = p; p += al(spec_b);
  c->stale = p; p += al(stale_b);
  c->tw = p; p += al(tw_b);
  c->diag_part = (double4 *)p;
  c->diag_out = c->diag_part + c->diag_blocks;
  int st = DNS_OK;
  do {
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking))) break;
    if ((e = cudaMallocHost((void **)&c->diag_host, sizeof(double4)))) break;
    // twiddles exp(-2 pi i k / n), generated in long double, rounded once to
    // the storage precision
    std::vector<double2> twd(n);
    std::vector<float2> twf(n);
    for (long k = 0; k < n; k++) {
      double cs, sn;
      sincos2pi(k, n, &cs, &sn);
      twd[k] = make_double2(cs, -sn);
      twf[k] = make_float2((float)cs, (float)-sn);
    }
    const void *src = fp64 ? (const void *)twd.data() : (const void *)twf.data();
    if ((e = cudaMemcpyAsync(c->tw, src, tw_b, cudaMemcpyHostToDevice, c->stream))) break;
    if ((e = cudaMemsetAsync(c->S, 0, spec_b, c->stream))) break;
    if ((e = cudaMemsetAsync(c->stale, 0, stale_b, c->stream))) break;
    if ((e = cudaStreamSynchronize(c->stream))) break;
  } while (0);
  if (e != cudaSuccess) {
    st = fail(DNS_ERR_CUDA, cudaGetErrorString(e), __FILE__, __LINE__);
    dns_destroy(c);
    return st;
  }
  *out = c;
  return DNS_OK;
}

int dns_destroy(dns_ctx *c) {
  if (!c) return DNS_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->graph) cudaGraphExecDestroy(c->graph);
  if (c->realbuf) cudaFree(c->realbuf);
  if (c->diag_host) cudaFreeHost(c->diag_host);
  if (c->arena) cudaFree(c->arena);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return DNS_OK;
}

int dns_set_velocity(dns_ctx *c, const double *U, const double *V, const double *W) {
  if (!c || !U || !V || !W) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  const double *src[3] = {U, V, W};
  int st = upload_real3(c, src);
  if (st != DNS_OK) return st;
  dispatch(c, [&](auto ops) { decltype(ops)::forward(c); });
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  c->have_state = true;
  return DNS_OK;
}

int dns_step(dns_ctx *c, double nu, double dt, long nsteps) {
  if (!c || nsteps < 0) return fail(DNS_ERR_ARG, "bad argument", __FILE__, __LINE__);
  if (!c->have_state) return fail(DNS_ERR_STATE, "no velocity set", __FILE__, __LINE__);
  if (nsteps == 0) return DNS_OK;
  int st = build_graph(c, nu, dt);
  if (st != DNS_OK) return st;
  for (long s = 0; s < nsteps; s++) CK(cudaGraphLaunch(c->graph, c->stream));
  return DNS_OK;
}

int dns_diagnostics(dns_ctx *c, double *e_hi, double *e_lo, double *om_hi, double *om_lo) {
  if (!c) return fail(DNS_ERR_ARG, "NULL context", __FILE__, __LINE__);
  dispatch(c, [&](auto ops) { decltype(ops)::diag(c); });
  CKL();
  CK(cudaMemcpyAsync(c->diag_host, c->diag_out, sizeof(double4), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const double4 r = *c->diag_host;
  if (e_hi) *e_hi = r.x;
  if (e_lo) *e_lo = r.y;
  if (om_hi) *om_hi = r.z;
  if (om_lo) *om_lo = r.w;
  if (!isfinite(r.x) || !isfinite(r.z) || !isfinite(r.y) || !isfinite(r.w))
    return fail(DNS_ERR_NONFINITE, "non-finite energy or enstrophy", __FILE__, __LINE__);
  return DNS_OK;
}

int dns_get_fields(dns_ctx *c, double *U, double *V, double *W, double *P) {
  if (!c) return fail(DNS_ERR_ARG, "NULL context", __FILE__, __LINE__);
  if (P && !(c->flags & DNS_FLAG_PRESSURE))
    return fail(DNS_ERR_ARG, "P requested without DNS_FLAG_PRESSURE", __FILE__, __LINE__);
  const size_t fb = (size_t)c->g.nreal * sizeof(double);
  if (!c->realbuf) CK(cudaMalloc((void **)&c->realbuf, 4 * fb));
  const int nf = P ? 4 : 3;
  dispatch(c, [&](auto ops) { decltype(ops)::backward(c, nf); });
  CKL();
  double *dst[4] = {U, V, W, P};
  for (int f = 0; f < nf; f++)
    if (dst[f])
      CK(cudaMemcpyAsync(dst[f], c->realbuf + f * c->g.nreal, fb, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DNS_OK;
}

int dns_get_spectral(dns_ctx *c, double *uvw) {
  if (!c || !uvw) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  const Geo &g = c->g;
  const size_t row = (size_t)g.nf * sizeof(double2);
  const size_t rows = (size_t)g.n * g.n;
  if (c->precision == DNS_PREC_FP64) {
    const size_t pitch = (size_t)g.nfp * sizeof(double2);
    for (int f = 0; f < 3; f++)
      CK(cudaMemcpy2DAsync((char *)uvw + f * rows * row, row, c->slot_ptr(SLOT_SA + f), pitch, row,
                           rows, cudaMemcpyDeviceToHost, c->stream));
  } else {
    const long long tot = 3LL * g.n * g.n * g.nf;
    k_spec_convert<float2, false><<<conv_blocks(tot), 256, 0, c->stream>>>(
        (float2 *)c->slot_ptr(SLOT_SA), (double2 *)c->staging(), g, 3);
    CKL();
    CK(cudaMemcpyAsync(uvw, c->staging(), 3 * rows * row, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return DNS_OK;
}

int dns_set_spectral(dns_ctx *c, const double *uvw) {
  if (!c || !uvw) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  const Geo &g = c->g;
  const size_t row = (size_t)g.nf * sizeof(double2);
  const size_t rows = (size_t)g.n * g.n;
  if (c->precision == DNS_PREC_FP64) {
    const size_t pitch = (size_t)g.nfp * sizeof(double2);
    for (int f = 0; f < 3; f++)
      CK(cudaMemcpy2DAsync(c->slot_ptr(SLOT_SA + f), pitch, (const char *)uvw + f * rows * row, row,
                           row, rows, cudaMemcpyHostToDevice, c->stream));
  } else {
    const long long tot = 3LL * g.n * g.n * g.nf;
    CK(cudaMemcpyAsync(c->staging(), uvw, 3 * rows * row, cudaMemcpyHostToDevice, c->stream));
    k_spec_convert<float2, true><<<conv_blocks(tot), 256, 0, c->stream>>>(
        (float2 *)c->slot_ptr(SLOT_SA), (double2 *)c->staging(), g, 3);
    CKL();
  }
  CK(cudaStreamSynchronize(c->stream));
  c->have_state = true;
  return DNS_OK;
}

int dns_get_stale(dns_ctx *c, double *uvw) {
  if (!c || !uvw) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  const long long nr = 3 * c->g.nreal;
  if (c->precision == DNS_PREC_FP64) {
    CK(cudaMemcpyAsync(uvw, c->stale, (size_t)nr * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  } else {
    k_real_convert<float, double><<<conv_blocks(nr), 256, 0, c->stream>>>((const float *)c->stale, c->staging(), nr);
    CKL();
    CK(cudaMemcpyAsync(uvw, c->staging(), (size_t)nr * sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return DNS_OK;
}

int dns_set_stale(dns_ctx *c, const double *uvw) {
  if (!c || !uvw) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  const long long nr = c->g.nreal;
  const double *src[3] = {uvw, uvw + nr, uvw + 2 * nr};
  int st = upload_real3(c, src);
  if (st != DNS_OK) return st;
  CK(cudaStreamSynchronize(c->stream));
  return DNS_OK;
}

int dns_get_info(dns_ctx *c, dns_info_t *info) {
  if (!c || !info) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  info->n = c->n;
  info->precision = c->precision;
  info->flags = c->flags;
  info->device_bytes = c->arena_bytes;
  info->slot_bytes = (size_t)c->g.slot * c->csize;
  info->kernels_per_step = c->kernels_per_step;
  return DNS_OK;
}

void *dns_get_stream(dns_ctx *c) { return c ? (void *)c->stream : nullptr; }

int dns_synchronize(dns_ctx *c) {
  if (!c) return fail(DNS_ERR_ARG, "NULL context", __FILE__, __LINE__);
  CK(cudaStreamSynchronize(c->stream));
  return DNS_OK;
}

int dns_time_kernels(dns_ctx *c, double nu, double dt, long nsteps, double *ms) {
  if (!c || !ms || nsteps <= 0) return fail(DNS_ERR_ARG, "bad argument", __FILE__, __LINE__);
  if (!c->have_state) return fail(DNS_ERR_STATE, "no velocity set", __FILE__, __LINE__);
  const int K = c->kernels_per_step;
  std::vector<cudaEvent_t> ev(K + 1);
  for (auto &e : ev) CK(cudaEventCreate(&e));
  for (int k = 0; k < K; k++) ms[k] = 0.0;
  int st = DNS_OK;
  for (long s = 0; s < nsteps && st == DNS_OK; s++) {
    CK(cudaEventRecord(ev[0], c->stream));
    for (int k = 0; k < K; k++) {
      dispatch(c, [&](auto ops) {
        decltype(ops)::stage_kernel(c, k / KERNELS_PER_STAGE, k % KERNELS_PER_STAGE, nu, dt);
      });
      CK(cudaEventRecord(ev[k + 1], c->stream));
    }
    st = check_launch(__FILE__, __LINE__);
    CK(cudaEventSynchronize(ev[K]));
    for (int k = 0; k < K; k++) {
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
      ms[k] += t;
    }
  }
  for (auto &e : ev) cudaEventDestroy(e);
  for (int k = 0; k < K; k++) ms[k] /= (double)nsteps;
  return st;
}

}  // extern "C"
