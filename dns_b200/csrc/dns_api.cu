// dns_api.cu -- context, launch orchestration (CUDA graphs) and the C ABI
// declared in include/dns_b200.h.
//
// Device memory of a context is one arena:
//   spectral slots, each [n][n][nfp] complex (double2 for DNS_PREC_FP64,
//   float2 for DNS_PREC_MIXED):
//     0..2   SA   state at the start of a step (U_hat, V_hat, W_hat)
//     3..5   SB   RK stage input (main.c's U_hat during stages 1-3)
//     6..8   ACC  RK accumulator (main.c's U_hat1)
//     9..15  WORK partially transformed fields of a stage (six used; all seven
//            are the float64 staging area of the FP32 path's host transfers)
//     16     P    pressure of the last stage
//   stale real velocity [3][n^3] (main.c's U, V, W between steps)
//   twiddles, reduction partials.
// main.c's U_hat0 is SA itself: stage 0 reads SA and writes SB/ACC, stage 3
// writes the new state back into SA, so the copies of main.c:334-342 and
// main.c:415-420 disappear.
#include "dns_b200.h"
#include "adjoint.cuh"
#include "init.cuh"
#include "kernels.cuh"
#include "persistent.cuh"

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <type_traits>
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

// Every device allocation of the library goes through here.  Fault
// injection for the tests of the error paths: with DNS_B200_FAIL_ALLOC=<k>
// (k >= 1) the k-th allocation of the process fails as an out-of-memory
// would, before cudaMalloc is called (host side only; nothing runs on the
// GPU for it).
std::atomic<long> g_alloc_count{0};
cudaError_t dev_malloc(void **p, size_t bytes) {
  static const long fail_at = [] {
    const char *e = getenv("DNS_B200_FAIL_ALLOC");
    return e ? atol(e) : 0L;
  }();
  const long k = ++g_alloc_count;
  if (fail_at > 0 && k == fail_at) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
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

// A group: nruns runs of one grid size and precision in one arena, stepped
// by the same (batched) kernel launches.  A dns_ctx is a group of one run;
// a dns_ens holds one group per distinct grid size.
struct Group {
  long n = 0;
  int precision = 0;
  unsigned flags = 0;
  int nruns = 1;
  size_t csize = 16;      // bytes of one complex element
  size_t rsize = 8;       // bytes of one real element
  Geo g{};
  char *arena = nullptr;
  size_t arena_bytes = 0;
  void *S = nullptr;      // spectral slots [nruns][NSLOTS][slot]
  void *stale = nullptr;  // stale real velocity [nruns][3][n^3]
  void *tw = nullptr;     // twiddles exp(-2 pi i k / n)
  double4 *diag_part = nullptr;  // [nruns][diag_blocks]
  double4 *diag_out = nullptr;   // [nruns]
  double *coef = nullptr;        // [nruns][2]: nu, dt
  int diag_blocks = 0;
  double *realbuf = nullptr;     // [4][n^3] float64, allocated on first field read
  // column-pass register schedules [axis][forward] picked by the autotuner
  // for this group's launches, and the run count they were timed on
  int pick[2][2] = {{0, 0}, {0, 0}};
  int tune_runs = 1;

  char *slot_ptr(int run, int s) const {
    return (char *)S + ((size_t)run * g.run_spec + (size_t)s * g.slot) * csize;
  }
  // float64 staging for host transfers of the FP32 path: the run's work
  // slots (7 * n^2 * nfp * 8 bytes >= 3 n^3 * 8 and >= 3 n^2 nf * 16)
  double *staging(int run) const { return (double *)slot_ptr(run, SLOT_WORK); }
  // the same arena seen as a batch of one run
  Group one(int run) const {
    Group v = *this;
    v.nruns = 1;
    v.S = slot_ptr(run, 0);
    v.stale = (char *)stale + (size_t)run * g.run_real * rsize;
    v.diag_part = diag_part + (size_t)run * diag_blocks;
    v.diag_out = diag_out + run;
    v.coef = coef + 2 * run;
    return v;
  }
};

struct dns_ctx {
  Group grp;
  cudaStream_t stream = nullptr;
  double4 *diag_host = nullptr;  // pinned
  bool have_state = false;
  cudaGraphExec_t graph = nullptr;
  double cur_nu = NAN, cur_dt = NAN;
  int kernels_per_step = 4 * KERNELS_PER_STAGE;
};

struct dns_ens {
  std::vector<Group> groups;
  std::vector<int> run_group, run_index;  // run -> (group, index in group)
  cudaStream_t stream = nullptr;
  std::vector<cudaStream_t> gstreams;
  std::vector<cudaEvent_t> gevents;
  cudaEvent_t fork = nullptr;
  double4 *diag_host = nullptr;  // pinned [nruns]
  std::vector<char> have_state;
  cudaGraphExec_t graph = nullptr;
  int nruns = 0;
  bool params_set = false;
  // the persistent schedule: one cooperative launch per step
  int mode = 0;                  // 0: batched launches, 1: persistent
  void *pplan = nullptr;         // device PPlan<R>
  PSync *psync = nullptr;        // device barrier state and error word
  int pgrid = 0;                 // co-resident blocks
  size_t psmem = 0;              // dynamic shared bytes per block
  cudaGraphExec_t pgraph = nullptr;
  bool pgraph_ok = false;        // the cooperative launch was captured
  float step_ms[2] = {-1.f, -1.f};  // measured ms per step of each schedule
};

namespace {

constexpr double RK_A[4] = {1 / 6.0, 1 / 3.0, 1 / 3.0, 1 / 6.0};  // main.c:15
constexpr double RK_B[3] = {0.5, 0.5, 1.0};                       // main.c:16

ColJobs jobs_empty(int njobs) {
  ColJobs j;
  for (int q = 0; q < 8; q++)
    j.in_slot[q] = 0, j.out_slot[q] = -1, j.der_slot[q] = -1, j.add_slot[q] = -1;
  j.njobs = njobs;
  j.masked = 0;
  return j;
}
ColJobs jobs_pass_a(int in0) {
  ColJobs j = jobs_empty(3);
  const int w = SLOT_WORK;
  j.in_slot[0] = in0 + 0; j.out_slot[0] = w + SU;
  j.in_slot[1] = in0 + 1; j.out_slot[1] = w + SV; j.der_slot[1] = w + SOMZ;  // dv/dx
  j.in_slot[2] = in0 + 2; j.out_slot[2] = w + SW; j.der_slot[2] = w + SDWDX;
  return j;
}
ColJobs jobs_pass_b(bool first) {
  ColJobs j = jobs_empty(4);
  const int w = SLOT_WORK;
  // u, and omega_z = dv/dx - i ky u over the dv/dx slot (same tile, same block)
  j.in_slot[0] = w + SU; j.out_slot[0] = w + SU; j.der_slot[0] = w + SOMZ; j.add_slot[0] = w + SOMZ;
  j.in_slot[1] = w + SV; j.out_slot[1] = w + SV;
  // the first stage reads the stale real velocity, so W itself is not needed
  j.in_slot[2] = w + SW; j.out_slot[2] = first ? -1 : w + SW; j.der_slot[2] = w + SDWDY;
  j.in_slot[3] = w + SDWDX; j.out_slot[3] = w + SDWDX;
  return j;
}
ColJobs jobs_map(const int *in, const int *out, int cnt) {
  ColJobs j = jobs_empty(cnt);
  for (int q = 0; q < cnt; q++) j.in_slot[q] = in[q], j.out_slot[q] = out[q];
  return j;
}

template <class R, int N>
struct Ops {
  using Real = R;
  using C = cx<R>;
  static constexpr int Nval = N;
  static constexpr int E = Plan<N>::E;
  template <int AXIS>
  static constexpr int CW = ColW<R, AXIS, N>::W;
  template <int AXIS>
  static constexpr int CT = (N / E) * CW<AXIS>;
  template <int AXIS>
  static constexpr size_t COL_SMEM = (size_t)(N + N * CW<AXIS>) * sizeof(C);
  static constexpr size_t Z_SMEM = (size_t)(2 * N + ZCfg<N>::LINES * ZCfg<N>::XB) * sizeof(C);
  template <int KIND>
  static constexpr size_t ZS_SMEM = ZC<R, N, KIND>::SMEM;
  // the z pass can keep its real velocity and vorticity (k_zstage_keep)
  static constexpr bool ZKEEP = ZC<R, N, 1>::S2 || ZC<R, N, 1>::F32;

  // Column-pass register schedules.  Candidate I of a pass is the same
  // kernel compiled with a minimum of ColCands::m[I] resident blocks per SM
  // (0: the compiler's own register choice); the candidates differ only in
  // register allocation, so every one computes bit-identical results.  The
  // autotuner (tune()) times them once per process, size and batch shape
  // (the run count it times on) and keeps the fastest; sizes below 64 have
  // the compiler's choice only.
  using ColFn = void (*)(const C *, C *, const C *, Geo, ColJobs);
  template <int AXIS>
  using Cands = ColCands<(N >= 64 ? (N / Plan<N>::E) * ColW<R, AXIS, N>::W : 0), (int)sizeof(C)>;
  template <int AXIS, bool FWD, int I>
  static ColFn col_cand() {
    constexpr int m = Cands<AXIS>::m[I];
    if constexpr (m == 0)
      return k_colpass<R, N, AXIS, FWD>;
    else
      return k_colpass_minb<R, N, AXIS, FWD, m>;
  }
  template <int AXIS, bool FWD, int I = 0>
  static ColFn col_cand_at(int i) {
    if constexpr (I + 1 < Cands<AXIS>::n) {
      if (i != I) return col_cand_at<AXIS, FWD, I + 1>(i);
    }
    return col_cand<AXIS, FWD, I>();
  }
  // chosen candidate of [AXIS][FWD] and the measured time per launch (ms)
  // of every candidate, per tuning run count
  struct TuneRec {
    int pick[2][2];
    float ms[2][2][16];
  };
  static inline std::map<int, TuneRec> tune_cache;
  static inline std::mutex tune_mu;  // guards tune_cache
  template <int AXIS, bool FWD>
  static ColFn colkern(const Group &G) {
    return col_cand_at<AXIS, FWD>(G.pick[AXIS][FWD]);
  }
  // runs a batch is tuned on: all of them up to the volume of two 256^3
  // runs, which fills the GPU like any larger batch
  static int tune_runs(int nruns) {
    long long cap = 2LL * 256 * 256 * 256 / ((long long)N * N * N);
    if (cap < 1) cap = 1;
    return (int)(nruns < cap ? nruns : cap);
  }

  template <class K>
  static cudaError_t allow(K kern, size_t smem) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  template <int AXIS, bool FWD>
  static cudaError_t allow_cands() {
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < Cands<AXIS>::n && e == cudaSuccess; i++)
      e = allow(col_cand_at<AXIS, FWD>(i), COL_SMEM<AXIS>);
    return e;
  }
  static cudaError_t setup() {
    cudaError_t e;
    if ((e = allow_cands<0, false>())) return e;
    if ((e = allow_cands<0, true>())) return e;
    if ((e = allow_cands<1, false>())) return e;
    if ((e = allow_cands<1, true>())) return e;
    if ((e = allow(k_zstage<R, N, 0>, ZS_SMEM<0>))) return e;
    if ((e = allow(k_zstage<R, N, 1>, ZS_SMEM<1>))) return e;
    if ((e = allow(k_zstage<R, N, 2>, ZS_SMEM<2>))) return e;
    if constexpr (ZKEEP) {
      if ((e = allow(k_zstage_keep<R, N, 0>, ZS_SMEM<0>))) return e;
      if ((e = allow(k_zstage_keep<R, N, 1>, ZS_SMEM<1>))) return e;
    }
    if ((e = allow(k_zr2c<R, N>, Z_SMEM))) return e;
    if ((e = allow(k_zc2r<R, N>, Z_SMEM))) return e;
    return cudaSuccess;
  }

  // ---- autotuner of the column-pass register schedules ----
  template <int AXIS, bool FWD>
  static cudaError_t time_cands(Group &Gt, cudaStream_t st, const ColJobs &jobs, cudaEvent_t e0,
                                cudaEvent_t e1, int force, int force_m, TuneRec &rec) {
    constexpr int n = Cands<AXIS>::n;
    int &pick = Gt.pick[AXIS][FWD];
    if (force_m >= 0) {  // a given register schedule: its candidate, else the compiler's
      pick = 0;
      for (int i = 0; i < n; i++)
        if (Cands<AXIS>::m[i] == force_m) pick = i;
      rec.pick[AXIS][FWD] = pick;
      return cudaSuccess;
    }
    int best = 0;
    for (int i = 0; i < n; i++) {
      pick = i;
      colpass_io<AXIS, FWD>(Gt, st, (C *)Gt.S, (C *)Gt.S, jobs, Gt.nruns);  // warm-up
      cudaError_t e = cudaEventRecord(e0, st);
      for (int r = 0; r < 3 && e == cudaSuccess; r++) {
        colpass_io<AXIS, FWD>(Gt, st, (C *)Gt.S, (C *)Gt.S, jobs, Gt.nruns);
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) e = cudaEventRecord(e1, st);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) return e;
      rec.ms[AXIS][FWD][i] = ms / 3.f;
      if (rec.ms[AXIS][FWD][i] < rec.ms[AXIS][FWD][best]) best = i;
    }
    pick = force >= 0 ? (force < n ? force : n - 1) : best;
    rec.pick[AXIS][FWD] = pick;
    return cudaSuccess;
  }
  // Time every register schedule of the four column passes of an RK stage
  // (their real job tables, batched over the group's first tune_runs(nruns)
  // runs, on their work slots, whose contents do not matter to an FFT's
  // timing) and keep the fastest of each; once per process, size and tuning
  // run count.  The group launches with the picks (G.pick).  DNS_B200_TUNE=0 keeps the compiler's schedule,
  // DNS_B200_TUNE=f<k> forces candidate k (the last where there are fewer),
  // DNS_B200_TUNE=m<a>,<b>,<c>,<d> the schedules of min blocks/SM a, b, c, d
  // for the x inverse, x forward, y inverse and y forward passes (as
  // dns_get_schedule reports them; a value that is not a candidate means
  // the compiler's).
  static cudaError_t tune(Group &G, cudaStream_t st, bool *ran) {
    std::lock_guard<std::mutex> lock(tune_mu);
    *ran = false;
    G.tune_runs = tune_runs(G.nruns);
    auto it = tune_cache.find(G.tune_runs);
    if (it != tune_cache.end()) {
      memcpy(G.pick, it->second.pick, sizeof G.pick);
      return cudaSuccess;
    }
    TuneRec rec{};
    const char *env = getenv("DNS_B200_TUNE");
    if (env && strcmp(env, "0") == 0) {
      tune_cache[G.tune_runs] = rec;
      memset(G.pick, 0, sizeof G.pick);
      return cudaSuccess;
    }
    const int force = (env && env[0] == 'f') ? atoi(env + 1) : -1;
    int fm[4] = {-1, -1, -1, -1};  // x inverse, x forward, y inverse, y forward
    if (env && env[0] == 'm') {
      const char *c = env + 1;
      for (int i = 0; i < 4 && *c; i++) {
        fm[i] = atoi(c);
        while (*c && *c != ',') c++;
        if (*c == ',') c++;
      }
    }
    Group Gt = G;  // the first tune_runs runs
    Gt.nruns = G.tune_runs;
    const int io[3] = {SLOT_WORK + SNX, SLOT_WORK + SNY, SLOT_WORK + SNZ};
    ColJobs jm = jobs_map(io, io, 3);
    jm.masked = 1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess)
      e = time_cands<0, false>(Gt, st, jobs_pass_a(SLOT_WORK), e0, e1, force, fm[0], rec);
    if (e == cudaSuccess)
      e = time_cands<1, false>(Gt, st, jobs_pass_b(false), e0, e1, force, fm[2], rec);
    if (e == cudaSuccess) e = time_cands<1, true>(Gt, st, jm, e0, e1, force, fm[3], rec);
    if (e == cudaSuccess) e = time_cands<0, true>(Gt, st, jm, e0, e1, force, fm[1], rec);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e == cudaSuccess) tune_cache[G.tune_runs] = rec;
    memcpy(G.pick, rec.pick, sizeof G.pick);
    *ran = true;
    return e;
  }
  // text description of the schedules chosen for G
  static std::string schedule(const Group &G) {
    std::string out;
    TuneRec rec{};
    memcpy(rec.pick, G.pick, sizeof rec.pick);
    {
      std::lock_guard<std::mutex> lock(tune_mu);
      auto it = tune_cache.find(G.tune_runs);
      if (it != tune_cache.end()) rec = it->second;
    }
    if (G.tune_runs > 1) out = "timed on " + std::to_string(G.tune_runs) + " runs: ";
    const char *name[2][2] = {{"x inverse", "x forward"}, {"y inverse", "y forward"}};
    char buf[160];
    for (int a = 0; a < 2; a++)
      for (int f = 0; f < 2; f++) {
        const int n = a == 0 ? Cands<0>::n : Cands<1>::n;
        const int *m = a == 0 ? Cands<0>::m : Cands<1>::m;
        const int k = rec.pick[a][f];
        snprintf(buf, sizeof buf, "%scolumn pass %s: min blocks/SM %d of {",
                 (a == 0 && f == 0) ? "" : "; ", name[a][f], m[k]);
        out += buf;
        for (int i = 0; i < n; i++) {
          snprintf(buf, sizeof buf, "%s%d: %.4f ms", i ? ", " : "", m[i], (double)rec.ms[a][f][i]);
          out += buf;
        }
        out += "}";
      }
    return out;
  }

  template <int KIND>
  static void zpass(const Group &G, cudaStream_t st, C *work, R *stale, R invn3) {
    k_zstage<R, N, KIND><<<zsgrid<KIND>(G.nruns), ZC<R, N, KIND>::THREADS, ZS_SMEM<KIND>, st>>>(
        work, stale, tw(G), G.g, invn3);
  }
  // the z pass of RK stage s of one run (the first stage's or the middle
  // stages' form), keeping the real velocity and vorticity in keep[6][n^3]
  static void zpass_keep(const Group &G, cudaStream_t st, int s, R *keep) {
    if constexpr (ZKEEP) {
      C *work = slot(G, SLOT_WORK);
      const R invn3 = (R)(1.0 / (double)G.g.nreal);
      if (s == 0)
        k_zstage_keep<R, N, 0><<<zsgrid<0>(1), ZC<R, N, 0>::THREADS, ZS_SMEM<0>, st>>>(
            work, (R *)G.stale, tw(G), G.g, invn3, keep);
      else
        k_zstage_keep<R, N, 1><<<zsgrid<1>(1), ZC<R, N, 1>::THREADS, ZS_SMEM<1>, st>>>(
            work, (R *)G.stale, tw(G), G.g, invn3, keep);
    }
  }

  static C *slot(const Group &G, int s) { return (C *)G.S + (long long)s * G.g.slot; }
  static const C *tw(const Group &G) { return (const C *)G.tw; }

  template <int AXIS, bool FWD>
  static void colpass_io(const Group &G, cudaStream_t st, const C *in, C *out, const ColJobs &jobs,
                         int nruns) {
    // a masked pass covers the tiles holding kz <= kcut and, along x, the
    // ky rows with |ky| <= kcut (kernels.cuh maps them back)
    const int tiles = jobs.masked ? G.g.kcut / CW<AXIS> + 1 : G.g.nfp / CW<AXIS>;
    const int rows = (jobs.masked && AXIS == 0) ? 2 * G.g.kcut + 1 : N;
    dim3 grid(tiles, rows, jobs.njobs * nruns);
    colkern<AXIS, FWD>(G)<<<grid, CT<AXIS>, COL_SMEM<AXIS>, st>>>(in, out, tw(G), G.g, jobs);
  }
  template <int AXIS, bool FWD>
  static void colpass(const Group &G, cudaStream_t st, const ColJobs &jobs) {
    colpass_io<AXIS, FWD>(G, st, (C *)G.S, (C *)G.S, jobs, G.nruns);
  }

  static dim3 zgrid(int nfields) { return dim3((N * N) / ZCfg<N>::LINES, nfields); }
  template <int KIND>
  static dim3 zsgrid(int nruns) {
    return dim3((N * N + ZC<R, N, KIND>::LINES - 1) / ZC<R, N, KIND>::LINES, nruns);
  }

  // Pass `k` (0..KERNELS_PER_STAGE-1) of RK stage `s` for all runs of G:
  // what it runs, its job table or stage arguments, and its work items (the
  // launch grid, threads and shared memory of one block).  The standalone
  // launches (stage_kernel) and the persistent ensemble kernel's plan are
  // both made from it.
  static PPhase<R> describe(const Group &G, int s, int k) {
    const Geo &g = G.g;
    PPhase<R> P{};
    P.gz = 1;
    if (k == 0 || k == 1 || k == 3 || k == 4) {
      P.kind = PK_COL;
      P.axis = (k == 0 || k == 4) ? 0 : 1;
      P.fwd = k >= 3;
      if (k == 0) {
        P.jobs = jobs_pass_a(s == 0 ? SLOT_SA : SLOT_SB);
      } else if (k == 1) {
        P.jobs = jobs_pass_b(s == 0);
      } else {
        // D: y forward, E1: x forward (in place on the three N slots); only
        // the modes inside the 2/3 rule are computed and stored
        const int io[3] = {SLOT_WORK + SNX, SLOT_WORK + SNY, SLOT_WORK + SNZ};
        P.jobs = jobs_map(io, io, 3);
        P.jobs.masked = 1;
      }
      constexpr int cw0 = CW<0>, cw1 = CW<1>, ct0 = CT<0>, ct1 = CT<1>;
      constexpr int sm0 = (int)COL_SMEM<0>, sm1 = (int)COL_SMEM<1>;
      const int cw = P.axis == 0 ? cw0 : cw1;
      // a masked pass covers the tiles holding kz <= kcut and, along x, the
      // ky rows with |ky| <= kcut (kernels.cuh maps them back)
      P.gx = P.jobs.masked ? g.kcut / cw + 1 : g.nfp / cw;
      P.gy = (P.jobs.masked && P.axis == 0) ? 2 * g.kcut + 1 : N;
      P.gz = P.jobs.njobs * G.nruns;
      P.tpi = P.axis == 0 ? ct0 : ct1;
      P.smem = P.axis == 0 ? sm0 : sm1;
    } else if (k == 2) {
      P.kind = PK_Z;
      P.sub = s == 0 ? 0 : s < 3 ? 1 : 2;
      const int lines = P.sub == 0 ? ZC<R, N, 0>::LINES : P.sub == 1 ? ZC<R, N, 1>::LINES
                                                                      : ZC<R, N, 2>::LINES;
      P.gx = (N * N + lines - 1) / lines;
      P.gy = G.nruns;
      P.tpi = ZC<R, N, 0>::THREADS;
      P.smem = (int)(P.sub == 0 ? ZS_SMEM<0> : P.sub == 1 ? ZS_SMEM<1> : ZS_SMEM<2>);
    } else {
      P.kind = PK_UPD;
      P.sub = s;
      StageArgs<R> &sa = P.sa;
      sa.u0 = slot(G, SLOT_SA);
      sa.us = slot(G, s == 0 ? SLOT_SA : SLOT_SB);
      sa.acc = slot(G, SLOT_ACC);
      sa.next = slot(G, SLOT_SB);
      sa.ph = (s == 3 && (G.flags & DNS_FLAG_PRESSURE)) ? slot(G, SLOT_P) : nullptr;
      sa.coef = G.coef;
      sa.a = RK_A[s];
      sa.b = s < 3 ? RK_B[s] : 0.0;
      const long long npad = (long long)N * N * g.nfp;
      const int per = UPD_THREADS * UpdVec<R>::VP;
      P.gx = (int)((npad + per - 1) / per);
      P.gy = G.nruns;
      P.tpi = UPD_THREADS;
      P.smem = 0;
    }
    return P;
  }

  // kernel `k` (0..KERNELS_PER_STAGE-1) of RK stage `s`, all runs of G
  static void stage_kernel(const Group &G, cudaStream_t st, int s, int k) {
    const Geo &g = G.g;
    C *work = slot(G, SLOT_WORK);
    R *stale = (R *)G.stale;
    const R invn3 = (R)(1.0 / (double)g.nreal);
    const PPhase<R> P = describe(G, s, k);
    const dim3 grid(P.gx, P.gy, P.gz);
    if (P.kind == PK_COL) {
      ColFn f = P.axis == 0 ? (P.fwd ? colkern<0, true>(G) : colkern<0, false>(G))
                            : (P.fwd ? colkern<1, true>(G) : colkern<1, false>(G));
      f<<<grid, P.tpi, P.smem, st>>>((C *)G.S, (C *)G.S, tw(G), g, P.jobs);
    } else if (P.kind == PK_Z) {
      if (P.sub == 0)
        zpass<0>(G, st, work, stale, invn3);
      else if (P.sub == 1)
        zpass<1>(G, st, work, stale, invn3);
      else
        zpass<2>(G, st, work, stale, invn3);
    } else {
      switch (s) {
        case 0: k_update<R, N, 0><<<grid, UPD_THREADS, 0, st>>>(work, g, P.sa); break;
        case 1: k_update<R, N, 1><<<grid, UPD_THREADS, 0, st>>>(work, g, P.sa); break;
        case 2: k_update<R, N, 2><<<grid, UPD_THREADS, 0, st>>>(work, g, P.sa); break;
        default: k_update<R, N, 3><<<grid, UPD_THREADS, 0, st>>>(work, g, P.sa); break;
      }
    }
  }

  // this group's part of the persistent ensemble kernel's plan
  static void plan_group(const Group &G, PGroup<R> &pg) {
    pg.n = N;
    pg.g = G.g;
    pg.S = (C *)G.S;
    pg.work = slot(G, SLOT_WORK);
    pg.stale = (R *)G.stale;
    pg.tw = tw(G);
    pg.invn3 = (R)(1.0 / (double)G.g.nreal);
    for (int s = 0; s < 4; s++)
      for (int k = 0; k < KERNELS_PER_STAGE; k++) pg.ph[s * KERNELS_PER_STAGE + k] = describe(G, s, k);
  }

  static void step(const Group &G, cudaStream_t st) {
    for (int s = 0; s < 4; s++)
      for (int k = 0; k < KERNELS_PER_STAGE; k++) stage_kernel(G, st, s, k);
  }

  // forward transform of the three stale real slots into SA (one run)
  static void forward(const Group &G, cudaStream_t st) {
    k_zr2c<R, N><<<zgrid(3), ZCfg<N>::THREADS, Z_SMEM, st>>>((const R *)G.stale,
                                                              slot(G, SLOT_WORK), tw(G), G.g);
    const int w3[3] = {SLOT_WORK + 0, SLOT_WORK + 1, SLOT_WORK + 2};
    const int sa[3] = {SLOT_SA + 0, SLOT_SA + 1, SLOT_SA + 2};
    colpass<1, true>(G, st, jobs_map(w3, w3, 3));
    colpass<0, true>(G, st, jobs_map(w3, sa, 3));
  }

  // c2r(X) / n^3 of SA (and P) into realbuf [4][n^3] float64 (one run)
  static void backward(const Group &G, cudaStream_t st, int nfields) {
    const int in[4] = {SLOT_SA + 0, SLOT_SA + 1, SLOT_SA + 2, SLOT_P};
    const int w4[4] = {SLOT_WORK + 0, SLOT_WORK + 1, SLOT_WORK + 2, SLOT_WORK + 3};
    colpass<0, false>(G, st, jobs_map(in, w4, nfields));
    colpass<1, false>(G, st, jobs_map(w4, w4, nfields));
    k_zc2r<R, N><<<zgrid(nfields), ZCfg<N>::THREADS, Z_SMEM, st>>>(
        slot(G, SLOT_WORK), G.realbuf, tw(G), G.g, 1.0 / (double)G.g.nreal);
  }

  // c2r of K spectral fields (in + in_slots[f] * slot) into out[f * nreal],
  // scaled (one run; uses the work slots)
  static void c2r_fields(const Group &G, cudaStream_t st, const C *in, const int *in_slots, int K,
                         double *out, double scale) {
    C *wk = slot(G, SLOT_WORK);
    ColJobs j1 = jobs_empty(K), j2 = jobs_empty(K);
    for (int f = 0; f < K; f++) {
      j1.in_slot[f] = in_slots[f];
      j1.out_slot[f] = f;
      j2.in_slot[f] = f;
      j2.out_slot[f] = f;
    }
    colpass_io<0, false>(G, st, in, wk, j1, 1);
    colpass_io<1, false>(G, st, wk, wk, j2, 1);
    k_zc2r<R, N><<<zgrid(K), ZCfg<N>::THREADS, Z_SMEM, st>>>(wk, out, tw(G), G.g, scale);
  }
  // r2c of K real fields in[f * nreal] into spectral out + out_slots[f] * slot
  static void r2c_fields(const Group &G, cudaStream_t st, const R *in, int K, C *out,
                         const int *out_slots) {
    C *wk = slot(G, SLOT_WORK);
    ColJobs j1 = jobs_empty(K), j2 = jobs_empty(K);
    for (int f = 0; f < K; f++) {
      j1.in_slot[f] = f;
      j1.out_slot[f] = out_slots[f];
      j2.in_slot[f] = f;
      j2.out_slot[f] = f;
    }
    k_zr2c<R, N><<<zgrid(K), ZCfg<N>::THREADS, Z_SMEM, st>>>(in, wk, tw(G), G.g);
    colpass_io<1, true>(G, st, wk, wk, j2, 1);
    colpass_io<0, true>(G, st, wk, out, j1, 1);
  }

  // energy / enstrophy sums of every run into diag_out[run]
  static void diag(const Group &G, cudaStream_t st) {
    k_diag<256, C><<<dim3(G.diag_blocks, G.nruns), 256, 0, st>>>(slot(G, SLOT_SA), G.g, G.diag_part);
    k_diag_final<256><<<G.nruns, 256, 0, st>>>(G.diag_part, G.diag_blocks, G.diag_out);
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
bool dispatch(const Group &G, F &&f) {
  return dispatch_n(G.precision, G.n, f);
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

unsigned conv_blocks(long long n) {
  long long b = (n + 255) / 256;
  return (unsigned)(b < 148 * 16 ? b : 148 * 16);
}

void group_free(Group &G) {
  if (G.realbuf) cudaFree(G.realbuf);
  if (G.arena) cudaFree(G.arena);
  G.realbuf = nullptr;
  G.arena = nullptr;
}

// allocate and initialise the arena of a group (synchronous on `st`)
int group_init(Group &G, long n, int precision, unsigned flags, int nruns, cudaStream_t st) {
  if (precision != DNS_PREC_FP64 && precision != DNS_PREC_MIXED)
    return fail(DNS_ERR_UNSUPPORTED, "precision not supported", __FILE__, __LINE__);
  if (nruns < 1) return fail(DNS_ERR_ARG, "nruns < 1", __FILE__, __LINE__);
  cudaError_t se = cudaErrorInvalidValue;
  if (!dispatch_n(precision, n, [&](auto ops) { se = decltype(ops)::setup(); })) {
    char buf[128];
    snprintf(buf, sizeof buf, "n = %ld is not supported (powers of two 8..512)", n);
    return fail(DNS_ERR_UNSUPPORTED, buf, __FILE__, __LINE__);
  }
  CK(se);
  G.n = n;
  G.precision = precision;
  G.flags = flags;
  G.nruns = nruns;
  const bool fp64 = precision == DNS_PREC_FP64;
  G.csize = fp64 ? sizeof(double2) : sizeof(float2);
  G.rsize = fp64 ? sizeof(double) : sizeof(float);
  const int W = fp64 ? PitchW<double>::W : PitchW<float>::W;
  Geo &g = G.g;
  g.n = (int)n;
  g.nf = (int)(n / 2 + 1);
  g.nfp = (g.nf + W - 1) / W * W;
  g.slot = (long long)n * n * g.nfp;
  g.nreal = (long long)n * n * n;
  g.run_spec = g.slot * NSLOTS;
  g.run_real = 3 * g.nreal;
  // 2/3 rule of main.c:231-238: keep |k| < kmax with kmax = 2/3 (n/2 + 1)
  const double kmax = 2. / 3. * (n / 2 + 1);
  int kcut = -1;
  while ((double)(kcut + 1) < kmax) kcut++;
  g.kcut = kcut;
  const long long npts = (long long)n * n * g.nf;
  G.diag_blocks = (int)((npts + 255) / 256 < 1184 ? (npts + 255) / 256 : 1184);

  const size_t spec_b = (size_t)g.run_spec * G.csize * nruns;
  const size_t stale_b = (size_t)g.run_real * G.rsize * nruns;
  const size_t tw_b = (size_t)n * G.csize;
  const size_t part_b = (size_t)(G.diag_blocks + 1) * nruns * sizeof(double4);
  const size_t coef_b = (size_t)2 * nruns * sizeof(double);
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  G.arena_bytes = al(spec_b) + al(stale_b) + al(tw_b) + al(part_b) + al(coef_b);
  cudaError_t e = dev_malloc((void **)&G.arena, G.arena_bytes);
  if (e != cudaSuccess) {
    G.arena = nullptr;
    return fail(DNS_ERR_NOMEM, cudaGetErrorString(e), __FILE__, __LINE__);
  }
  char *p = G.arena;
  G.S = p; p += al(spec_b);
  G.stale = p; p += al(stale_b);
  G.tw = p; p += al(tw_b);
  G.diag_part = (double4 *)p; p += al(part_b);
  G.diag_out = G.diag_part + (size_t)G.diag_blocks * nruns;
  G.coef = (double *)p;
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
  std::vector<double> coef(2 * nruns, 0.0);
  const void *src = fp64 ? (const void *)twd.data() : (const void *)twf.data();
  CK(cudaMemcpyAsync(G.tw, src, tw_b, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(G.coef, coef.data(), coef_b, cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(G.S, 0, spec_b, st));
  CK(cudaMemsetAsync(G.stale, 0, stale_b, st));
  CK(cudaStreamSynchronize(st));
  cudaError_t te = cudaSuccess;
  bool ran = false;
  dispatch(G, [&](auto ops) { te = decltype(ops)::tune(G, st, &ran); });
  CK(te);
  if (ran) {  // the tuner ran column passes on the work slots of its runs: zero them again
    for (int r = 0; r < G.tune_runs; r++)
      CK(cudaMemsetAsync(G.slot_ptr(r, SLOT_WORK), 0, (size_t)7 * g.slot * G.csize, st));
    CK(cudaStreamSynchronize(st));
  }
  return DNS_OK;
}

// host float64 [3][n^3] -> stale real slots of a one-run view
int upload_real3(const Group &G, cudaStream_t st, const double *const src[3]) {
  const long long nr = G.g.nreal;
  const size_t fb = (size_t)nr * sizeof(double);
  double *dst = G.precision == DNS_PREC_FP64 ? (double *)G.stale : G.staging(0);
  for (int f = 0; f < 3; f++)
    CK(cudaMemcpyAsync(dst + f * nr, src[f], fb, cudaMemcpyHostToDevice, st));
  if (G.precision != DNS_PREC_FP64) {
    k_real_convert<double, float><<<conv_blocks(3 * nr), 256, 0, st>>>(dst, (float *)G.stale, 3 * nr);
    CKL();
  }
  return DNS_OK;
}

// velocity of one run: upload and transform
int set_velocity_view(const Group &V, cudaStream_t st, const double *U, const double *Vv,
                      const double *W) {
  const double *src[3] = {U, Vv, W};
  int s = upload_real3(V, st, src);
  if (s != DNS_OK) return s;
  dispatch(V, [&](auto ops) { decltype(ops)::forward(V, st); });
  CKL();
  CK(cudaStreamSynchronize(st));
  return DNS_OK;
}

// 1-D tables of tgv.py:16-22: s_i = sin(i dx), c_i = cos(i dx) with
// dx = 2 pi / n in double (the C library's sin and cos)
void tgv_tables(long n, std::vector<double> &tab) {
  const double dx = 2 * 3.141592653589793 / (double)n;
  tab.resize(2 * n);
  for (long i = 0; i < n; i++) {
    tab[i] = sin(dx * (double)i);
    tab[n + i] = cos(dx * (double)i);
  }
}

// Taylor-Green of tgv.py (plus, with `perturb`, the seeded solenoidal
// perturbation of init.cuh) generated on the device into the stale slots of
// run `run` of G, then transformed like dns_set_velocity.  The perturbation
// is shaped at the storage precision (float32 FFTs in a mixed group).
int init_view(Group &G, int run, cudaStream_t st, bool perturb, unsigned long long seed,
              double amplitude) {
  const Group V = G.one(run);
  const Geo &g = V.g;
  const long n = G.n;
  const bool fp64 = G.precision == DNS_PREC_FP64;
  std::vector<double> tab;
  tgv_tables(n, tab);
  double *dtab = (double *)V.slot_ptr(0, SLOT_WORK + 6);  // free until the forward transform
  CK(cudaMemcpyAsync(dtab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  double *delta = nullptr;
  double rms = 1.0, scale = 0.0;
  const unsigned blocks = conv_blocks(3 * g.nreal);
  if (perturb) {
    if (!fp64 && !G.realbuf) CK(dev_malloc((void **)&G.realbuf, 4 * (size_t)g.nreal * sizeof(double)));
    // FP64: the stale slots hold the noise until its forward transform, then
    // the shaped field; mixed: a float64 buffer
    delta = fp64 ? (double *)V.stale : G.realbuf;
    dispatch(V, [&](auto ops) {
      using O = decltype(ops);
      using R = typename O::Real;
      k_noise3<R><<<blocks, 256, 0, st>>>((R *)V.stale, g.nreal, seed);
      O::forward(V, st);
      k_shape_project<typename O::C><<<conv_blocks((long long)n * n * g.nf), 256, 0, st>>>(
          O::slot(V, SLOT_SA), g, 4.0);
      const int f3[3] = {0, 1, 2};
      O::c2r_fields(V, st, O::slot(V, SLOT_SA), f3, 3, delta, 1.0 / (double)g.nreal);
    });
    k_sumsq<256><<<V.diag_blocks, 256, 0, st>>>(delta, 3 * g.nreal, V.diag_part);
    k_diag_final<256><<<1, 256, 0, st>>>(V.diag_part, V.diag_blocks, V.diag_out);
    CKL();
    double4 sum;
    CK(cudaMemcpyAsync(&sum, V.diag_out, sizeof sum, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    rms = sqrt((sum.x + sum.y) / (double)g.nreal);
    // rms of the Taylor-Green field: mean of U^2 + V^2 = 2 S C^2 / n^3 with
    // S = sum s_i^2, C = sum c_i^2
    long double S = 0, Cs = 0;
    for (long i = 0; i < n; i++) {
      S += (long double)tab[i] * tab[i];
      Cs += (long double)tab[n + i] * tab[n + i];
    }
    const double rms_tgv = (double)sqrtl(2.0L * S * Cs * Cs / ((long double)n * n * n));
    scale = amplitude * rms_tgv;
    if (!(rms > 0) || !isfinite(rms))
      return fail(DNS_ERR_NONFINITE, "perturbation has no energy", __FILE__, __LINE__);
  }
  dispatch(V, [&](auto ops) {
    using O = decltype(ops);
    using R = typename O::Real;
    k_tgv_fill<R><<<blocks, 256, 0, st>>>((R *)V.stale, dtab, delta, rms, scale, (int)n);
    O::forward(V, st);
  });
  CKL();
  CK(cudaStreamSynchronize(st));
  return DNS_OK;
}

int get_spectral_view(const Group &V, cudaStream_t st, double *uvw) {
  const Geo &g = V.g;
  const size_t row = (size_t)g.nf * sizeof(double2);
  const size_t rows = (size_t)g.n * g.n;
  if (V.precision == DNS_PREC_FP64) {
    const size_t pitch = (size_t)g.nfp * sizeof(double2);
    for (int f = 0; f < 3; f++)
      CK(cudaMemcpy2DAsync((char *)uvw + f * rows * row, row, V.slot_ptr(0, SLOT_SA + f), pitch, row,
                           rows, cudaMemcpyDeviceToHost, st));
  } else {
    const long long tot = 3LL * g.n * g.n * g.nf;
    k_spec_convert<float2, false><<<conv_blocks(tot), 256, 0, st>>>(
        (float2 *)V.slot_ptr(0, SLOT_SA), (double2 *)V.staging(0), g, 3);
    CKL();
    CK(cudaMemcpyAsync(uvw, V.staging(0), 3 * rows * row, cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  return DNS_OK;
}

int set_spectral_view(const Group &V, cudaStream_t st, const double *uvw) {
  const Geo &g = V.g;
  const size_t row = (size_t)g.nf * sizeof(double2);
  const size_t rows = (size_t)g.n * g.n;
  if (V.precision == DNS_PREC_FP64) {
    const size_t pitch = (size_t)g.nfp * sizeof(double2);
    for (int f = 0; f < 3; f++)
      CK(cudaMemcpy2DAsync(V.slot_ptr(0, SLOT_SA + f), pitch, (const char *)uvw + f * rows * row, row,
                           row, rows, cudaMemcpyHostToDevice, st));
  } else {
    const long long tot = 3LL * g.n * g.n * g.nf;
    CK(cudaMemcpyAsync(V.staging(0), uvw, 3 * rows * row, cudaMemcpyHostToDevice, st));
    k_spec_convert<float2, true><<<conv_blocks(tot), 256, 0, st>>>(
        (float2 *)V.slot_ptr(0, SLOT_SA), (double2 *)V.staging(0), g, 3);
    CKL();
  }
  CK(cudaStreamSynchronize(st));
  return DNS_OK;
}

// coefficients nu, dt of every run of a group (host arrays of nruns)
int set_coef(const Group &G, cudaStream_t st, const double *nu, const double *dt) {
  std::vector<double> c(2 * G.nruns);
  for (int r = 0; r < G.nruns; r++) c[2 * r] = nu[r], c[2 * r + 1] = dt[r];
  CK(cudaMemcpyAsync(G.coef, c.data(), c.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  return DNS_OK;
}


// ---------------------------------------------------------------------------
// Discrete adjoint of the RK4 step (FP64, or with the mixed path's FP32
// storage and transforms): gradient of the final energy
// E(T) = invn3^2 sum_half |U_hat(T)|^2 (main.c:257-266's definition) with
// respect to the initial velocity and nu.  Checkpoints of the step state
// (U_hat, stale velocity) follow a binomial split of the step range.
// ---------------------------------------------------------------------------
// spectral work triples (in units of slots)
// (the stage inputs U_1..U_3; two buffers for lambda of the step state, one
// holding the step output's, the other accumulating the step input's, which
// swap roles after every reversed step; lambda of dU_s; two transform triples)
enum { X_US1 = 0, X_LA = 9, X_LB = 12, X_LDU = 15, X_T1 = 18, X_T2 = 21, NX = 24 };
// real work triples (in units of n^3 fields)
enum { RE_U = 0, RE_OM = 3, RE_LN = 6, RE_LU = 9, RE_LOM = 12, RE_LSTALE = 15, NRE = 18 };

struct Adj {
  Group G;
  cudaStream_t st = nullptr;
  cudaGraphExec_t graph = nullptr;
  char *arena = nullptr;
  void *sp = nullptr;        // [NX][slot], storage complex type
  double *re = nullptr;      // [NRE][n^3] float64; LU, LOM hold the storage real type
  char *snap_sp = nullptr;   // [S][3][slot]
  char *snap_re = nullptr;   // [S][3][n^3], storage real type
  char *keep = nullptr;      // [4][6][n^3], storage real type: the real velocity and
                             // vorticity of each RK stage, where the z pass keeps them
  double4 *part = nullptr, *acc_nu = nullptr;
  int nblocks = 0;
  double nu = 0, dt = 0;
  int lhat = X_LA;  // the buffer holding lambda of the current step state
  template <class C>
  C *X(int i) const { return (C *)sp + (size_t)i * G.g.slot; }
  double *Rf(int i) const { return re + (size_t)i * G.g.nreal; }
  // a real triple seen in the storage type (3 n^3 values fit in its space)
  template <class R>
  R *Rr(int i) const { return (R *)(re + (size_t)i * G.g.nreal); }
  size_t slot3() const { return (size_t)3 * G.g.slot * G.csize; }
  size_t real3() const { return (size_t)3 * G.g.nreal * G.rsize; }
  size_t real3d() const { return (size_t)3 * G.g.nreal * sizeof(double); }
  template <class R>
  R *K(int s, int f) const { return (R *)keep + ((size_t)6 * s + f) * G.g.nreal; }
};

template <class R, int N>
struct AdjOps {
  using O = Ops<R, N>;
  using C = cx<R>;
  static int copy3(Adj &A, void *dst, const void *src, size_t bytes) {
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, A.st));
    return DNS_OK;
  }
  static unsigned pblocks(const Adj &A) { return (unsigned)A.nblocks; }

  // U_s: the step input (slot SA, untouched by the forward stages 0-2) or a
  // kept stage input
  static const C *stage_input(const Adj &A, int s) {
    return s == 0 ? (const C *)A.G.slot_ptr(0, SLOT_SA) : A.X<C>(X_US1 + 3 * (s - 1));
  }

  // adjoint of RK stage s: from lambda_dU (X_LDU) and U_s, add lambda_{U_s}
  // to lambda of U0 (lin into lout) and, for s > 0, form lambda_dU of stage
  // s - 1 in X_LDU; stage 0 also produces lambda_stale
  static int stage(Adj &A, int s, const C *lin, C *lout, const C *lacc) {
    const Group &G = A.G;
    const Geo &g = G.g;
    const double a = 1.0 / (double)g.nreal;
    const int t3[3] = {0, 1, 2};
    const C *Us = stage_input(A, s);
    const unsigned pb = pblocks(A);
    if constexpr (!O::ZKEEP) {  // the velocity and vorticity of the stage, again
      if (s > 0) O::c2r_fields(G, A.st, Us, t3, 3, A.Rf(RE_U), a);
      k_curl<C><<<pb, 256, 0, A.st>>>(Us, A.X<C>(X_T1), g);
      O::c2r_fields(G, A.st, A.X<C>(X_T1), t3, 3, A.Rf(RE_OM), a);
    }
    k_adj_lamN<C><<<pb, 256, 0, A.st>>>(A.X<C>(X_LDU), A.X<C>(X_T1), g, A.dt);
    O::c2r_fields(G, A.st, A.X<C>(X_T1), t3, 3, A.Rf(RE_LN), 1.0);
    const double *lso = s == 3 ? A.Rf(RE_LSTALE) : nullptr;
    const unsigned cb = conv_blocks(g.nreal);
    // stage 0 reads the stale velocity (main.c:344), the step's input one
    if constexpr (O::ZKEEP) {  // kept by the z pass of the forward stage
      const R *u = s > 0 ? A.K<R>(s, 0) : (const R *)G.stale;
      k_adj_cross<R, R, R><<<cb, 256, 0, A.st>>>(u, A.K<R>(s, 3), A.Rf(RE_LN), lso,
                                                 A.Rr<R>(RE_LU), A.Rr<R>(RE_LOM), g.nreal);
    } else if (s > 0) {
      k_adj_cross<double, double, R><<<cb, 256, 0, A.st>>>(
          A.Rf(RE_U), A.Rf(RE_OM), A.Rf(RE_LN), lso, A.Rr<R>(RE_LU), A.Rr<R>(RE_LOM), g.nreal);
    } else {
      k_adj_cross<R, double, R><<<cb, 256, 0, A.st>>>((const R *)G.stale, A.Rf(RE_OM),
                                                      A.Rf(RE_LN), lso, A.Rr<R>(RE_LU),
                                                      A.Rr<R>(RE_LOM), g.nreal);
    }
    O::r2c_fields(G, A.st, A.Rr<R>(RE_LOM), 3, A.X<C>(X_T1), t3);
    if (s > 0) O::r2c_fields(G, A.st, A.Rr<R>(RE_LU), 3, A.X<C>(X_T2), t3);
    k_adj_collect<256, C><<<pb, 256, 0, A.st>>>(
        A.X<C>(X_T1), s > 0 ? A.X<C>(X_T2) : nullptr, A.X<C>(X_LDU), Us, lin, lout, lacc, g, a,
        A.nu, A.dt, s > 0 ? RK_B[s - 1] : 0.0, s > 0 ? RK_A[s - 1] : 0.0, s > 0, A.part);
    k_dd_accumulate<256><<<1, 256, 0, A.st>>>(A.part, A.nblocks, A.acc_nu);
    if (s == 0)  // lambda of the step's input stale velocity, kept in float64
      k_real_convert<R, double><<<conv_blocks(3 * g.nreal), 256, 0, A.st>>>(
          A.Rr<R>(RE_LU), A.Rf(RE_LSTALE), 3 * g.nreal);
    CKL();
    return DNS_OK;
  }

  // adjoint of one step whose input state is in (SA, stale); lambda of the
  // step output in (A.lhat, RE_LSTALE) becomes lambda of its input (in the
  // other buffer, which becomes A.lhat).  The forward stages 0-2 run again
  // to recover the stage inputs U_1..U_3 (stage 3's output is not needed);
  // the step's state (SA, stale) is left in place for stage 0's adjoint.
  // Where the z pass can keep its real velocity and vorticity, every stage's
  // z pass (stage 3's too, after its A and B passes; without its stale
  // store) keeps them for the transposed stage.
  static int step(Adj &A) {
    const Group &G = A.G;
    const Geo &g = G.g;
    int r;
    for (int s = 0; s < 4; s++) {
      if (!O::ZKEEP && s == 3) break;
      for (int k = 0; k < KERNELS_PER_STAGE; k++) {
        if (s == 3 && k > 2) break;
        if (O::ZKEEP && k == 2)
          O::zpass_keep(G, A.st, s, A.K<R>(s, 0));
        else
          O::stage_kernel(G, A.st, s, k);
      }
      if (s < 3 && (r = copy3(A, A.X<C>(X_US1 + 3 * s), G.slot_ptr(0, SLOT_SB), A.slot3())))
        return r;
    }
    const int lo = A.lhat, li = A.lhat == X_LA ? X_LB : X_LA;
    const C *lacc = A.X<C>(lo);  // lambda of the accumulator: that of the step output
    // lambda_dU of stage 3 = a_3 lambda_acc
    k_lincomb3<C><<<pblocks(A), 256, 0, A.st>>>(lacc, nullptr, A.X<C>(X_LDU), g, RK_A[3], 0.0);
    // lambda of U0 = lambda of the output (through the accumulator's U0 term)
    // plus the lambda of every stage input (each U0 plus a multiple of dU)
    for (int s = 3; s >= 0; s--)
      if ((r = stage(A, s, s == 3 ? lacc : A.X<C>(li), A.X<C>(li), lacc))) return r;
    A.lhat = li;
    CKL();
    return DNS_OK;
  }
};

int adj_snap_store(Adj &A, int k) {
  CK(cudaMemcpyAsync(A.snap_sp + (size_t)k * A.slot3(), A.G.slot_ptr(0, SLOT_SA), A.slot3(),
                     cudaMemcpyDeviceToDevice, A.st));
  CK(cudaMemcpyAsync(A.snap_re + (size_t)k * A.real3(), A.G.stale, A.real3(),
                     cudaMemcpyDeviceToDevice, A.st));
  return DNS_OK;
}
int adj_snap_restore(Adj &A, int k) {
  CK(cudaMemcpyAsync(A.G.slot_ptr(0, SLOT_SA), A.snap_sp + (size_t)k * A.slot3(), A.slot3(),
                     cudaMemcpyDeviceToDevice, A.st));
  CK(cudaMemcpyAsync(A.G.stale, A.snap_re + (size_t)k * A.real3(), A.real3(),
                     cudaMemcpyDeviceToDevice, A.st));
  return DNS_OK;
}
int adj_advance(Adj &A, long m) {
  for (long q = 0; q < m; q++) CK(cudaGraphLaunch(A.graph, A.st));
  return DNS_OK;
}
int adj_step_one(Adj &A) {
  int r = DNS_OK;
  dispatch(A.G, [&](auto ops) {
    using O = decltype(ops);
    r = AdjOps<typename O::Real, O::Nval>::step(A);
  });
  return r;
}

double binom(int n, int k) {
  double r = 1.0;
  for (int q = 1; q <= k; q++) r = r * (n - k + q) / q;
  return r;
}

// binomial split of steps [a, b) with `free` spare snapshots (b - a >= 2,
// free >= 1): smallest repetition number rr with C(free + rr, free) >= l;
// the right part [m, b) gets what free - 1 snapshots reverse in rr
long adj_split(long a, long b, int free) {
  const long l = b - a;
  int rr = 0;
  while (binom(free + rr, free) < (double)l) rr++;
  const double right_cap = binom(free - 1 + rr, free - 1);
  long lr = right_cap < (double)(l - 1) ? (long)right_cap : l - 1;
  if (lr < 1) lr = 1;
  return b - lr;
}

// The checkpoint schedule below drives an executor: AdjDev runs it on the
// device, AdjCount only counts it (dns_adjoint_schedule).
struct AdjDev {
  Adj &A;
  int advance(long m) { return adj_advance(A, m); }
  int store(int k) { return adj_snap_store(A, k); }
  int restore(int k) { return adj_snap_restore(A, k); }
  int step_one() { return adj_step_one(A); }
};
struct AdjCount {
  long advanced = 0, reversed = 0;
  int used = 1;  // snapshot 0 holds the initial state
  int advance(long m) {
    advanced += m;
    return DNS_OK;
  }
  int store(int k) {
    used = k + 1 > used ? k + 1 : used;
    return DNS_OK;
  }
  int restore(int) { return DNS_OK; }
  int step_one() {
    reversed++;
    return DNS_OK;
  }
};

// forward sweep over steps [0, b) from the state in snapshot 0, storing
// the snapshots of the reverse sweep's rightmost path (the split points
// adj_reverse takes first, each with one snapshot fewer) on the way, so
// the reverse sweep need not recompute them
template <class Ex>
int adj_sweep(Ex &x, long b, int free) {
  long a = 0;
  int ka = 0, r;
  while (b - a >= 2 && free >= 1) {
    const long m = adj_split(a, b, free);
    if ((r = x.advance(m - a))) return r;
    if ((r = x.store(ka + 1))) return r;
    a = m;
    ka++;
    free--;
  }
  return x.advance(b - a);
}

// reverse steps [a, b): the state at step a is in snapshot ka; snapshots
// ka+1 .. ka+free are unused, unless `stored`: then those of the rightmost
// path of the split tree are already in place (adj_sweep)
template <class Ex>
int adj_reverse(Ex &x, long a, long b, int ka, int free, bool stored) {
  int r;
  if (b - a == 1) {
    if ((r = x.restore(ka))) return r;
    return x.step_one();
  }
  if (free == 0) {  // no snapshot to spare: recompute from a for every step
    for (long t = b - 1; t >= a; t--) {
      if ((r = x.restore(ka))) return r;
      if ((r = x.advance(t - a))) return r;
      if ((r = x.step_one())) return r;
    }
    return DNS_OK;
  }
  const long m = adj_split(a, b, free);
  if (!stored) {
    if ((r = x.restore(ka))) return r;
    if ((r = x.advance(m - a))) return r;
    if ((r = x.store(ka + 1))) return r;
  }
  if ((r = adj_reverse(x, m, b, ka + 1, free - 1, stored))) return r;
  return adj_reverse(x, a, m, ka, free, false);
}

int ctx_build_graph(dns_ctx *c) {
  if (c->graph) return DNS_OK;
  cudaGraph_t gr;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  dispatch(c->grp, [&](auto ops) { decltype(ops)::step(c->grp, c->stream); });
  cudaError_t le = cudaGetLastError();
  cudaError_t ce = cudaStreamEndCapture(c->stream, &gr);
  if (le != cudaSuccess) return fail(DNS_ERR_CUDA, cudaGetErrorString(le), __FILE__, __LINE__);
  CK(ce);
  cudaError_t ie = cudaGraphInstantiate(&c->graph, gr, 0);
  cudaGraphDestroy(gr);
  CK(ie);
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
  dns_ctx *c = new dns_ctx();
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return fail(DNS_ERR_CUDA, cudaGetErrorString(e), __FILE__, __LINE__);
  }
  int st = group_init(c->grp, n, precision, flags, 1, c->stream);
  if (st == DNS_OK && cudaMallocHost((void **)&c->diag_host, sizeof(double4)) != cudaSuccess)
    st = fail(DNS_ERR_NOMEM, "pinned host allocation failed", __FILE__, __LINE__);
  if (st != DNS_OK) {
    std::string keep = g_last_error;
    dns_destroy(c);
    g_last_error = keep;
    return st;
  }
  *out = c;
  return DNS_OK;
}

int dns_destroy(dns_ctx *c) {
  if (!c) return DNS_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->graph) cudaGraphExecDestroy(c->graph);
  group_free(c->grp);
  if (c->diag_host) cudaFreeHost(c->diag_host);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return DNS_OK;
}

int dns_set_velocity(dns_ctx *c, const double *U, const double *V, const double *W) {
  if (!c || !U || !V || !W) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  int st = set_velocity_view(c->grp, c->stream, U, V, W);
  if (st == DNS_OK) c->have_state = true;
  return st;
}

int dns_step(dns_ctx *c, double nu, double dt, long nsteps) {
  if (!c || nsteps < 0) return fail(DNS_ERR_ARG, "bad argument", __FILE__, __LINE__);
  if (!c->have_state) return fail(DNS_ERR_STATE, "no velocity set", __FILE__, __LINE__);
  if (nsteps == 0) return DNS_OK;
  if (!(nu == c->cur_nu && dt == c->cur_dt)) {
    int st = set_coef(c->grp, c->stream, &nu, &dt);
    if (st != DNS_OK) return st;
    c->cur_nu = nu;
    c->cur_dt = dt;
  }
  int st = ctx_build_graph(c);
  if (st != DNS_OK) return st;
  for (long s = 0; s < nsteps; s++) CK(cudaGraphLaunch(c->graph, c->stream));
  return DNS_OK;
}

int dns_diagnostics(dns_ctx *c, double *e_hi, double *e_lo, double *om_hi, double *om_lo) {
  if (!c) return fail(DNS_ERR_ARG, "NULL context", __FILE__, __LINE__);
  dispatch(c->grp, [&](auto ops) { decltype(ops)::diag(c->grp, c->stream); });
  CKL();
  CK(cudaMemcpyAsync(c->diag_host, c->grp.diag_out, sizeof(double4), cudaMemcpyDeviceToHost,
                     c->stream));
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

int dns_set_tgv(dns_ctx *c) {
  if (!c) return fail(DNS_ERR_ARG, "NULL context", __FILE__, __LINE__);
  int st = init_view(c->grp, 0, c->stream, false, 0, 0.0);
  if (st == DNS_OK) c->have_state = true;
  return st;
}

int dns_set_perturbed_tgv(dns_ctx *c, unsigned long long seed, double amplitude) {
  if (!c || !isfinite(amplitude)) return fail(DNS_ERR_ARG, "bad argument", __FILE__, __LINE__);
  int st = init_view(c->grp, 0, c->stream, true, seed, amplitude);
  if (st == DNS_OK) c->have_state = true;
  return st;
}

int dns_get_fields(dns_ctx *c, double *U, double *V, double *W, double *P) {
  if (!c) return fail(DNS_ERR_ARG, "NULL context", __FILE__, __LINE__);
  Group &G = c->grp;
  if (P && !(G.flags & DNS_FLAG_PRESSURE))
    return fail(DNS_ERR_ARG, "P requested without DNS_FLAG_PRESSURE", __FILE__, __LINE__);
  const size_t fb = (size_t)G.g.nreal * sizeof(double);
  if (!G.realbuf) CK(dev_malloc((void **)&G.realbuf, 4 * fb));
  const int nf = P ? 4 : 3;
  dispatch(G, [&](auto ops) { decltype(ops)::backward(G, c->stream, nf); });
  CKL();
  double *dst[4] = {U, V, W, P};
  for (int f = 0; f < nf; f++)
    if (dst[f])
      CK(cudaMemcpyAsync(dst[f], G.realbuf + f * G.g.nreal, fb, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DNS_OK;
}

int dns_get_spectral(dns_ctx *c, double *uvw) {
  if (!c || !uvw) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  return get_spectral_view(c->grp, c->stream, uvw);
}

int dns_set_spectral(dns_ctx *c, const double *uvw) {
  if (!c || !uvw) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  int st = set_spectral_view(c->grp, c->stream, uvw);
  if (st == DNS_OK) c->have_state = true;
  return st;
}

int dns_get_stale(dns_ctx *c, double *uvw) {
  if (!c || !uvw) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  const Group &G = c->grp;
  const long long nr = 3 * G.g.nreal;
  if (G.precision == DNS_PREC_FP64) {
    CK(cudaMemcpyAsync(uvw, G.stale, (size_t)nr * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  } else {
    k_real_convert<float, double><<<conv_blocks(nr), 256, 0, c->stream>>>(
        (const float *)G.stale, G.staging(0), nr);
    CKL();
    CK(cudaMemcpyAsync(uvw, G.staging(0), (size_t)nr * sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return DNS_OK;
}

int dns_set_stale(dns_ctx *c, const double *uvw) {
  if (!c || !uvw) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  const long long nr = c->grp.g.nreal;
  const double *src[3] = {uvw, uvw + nr, uvw + 2 * nr};
  int st = upload_real3(c->grp, c->stream, src);
  if (st != DNS_OK) return st;
  CK(cudaStreamSynchronize(c->stream));
  return DNS_OK;
}

int dns_get_info(dns_ctx *c, dns_info_t *info) {
  if (!c || !info) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  info->n = c->grp.n;
  info->precision = c->grp.precision;
  info->flags = c->grp.flags;
  info->device_bytes = c->grp.arena_bytes;
  info->slot_bytes = (size_t)c->grp.g.slot * c->grp.csize;
  info->kernels_per_step = c->kernels_per_step;
  return DNS_OK;
}

int dns_get_schedule(dns_ctx *c, char *buf, long len) {
  if (!c || !buf || len < 1) return fail(DNS_ERR_ARG, "bad argument", __FILE__, __LINE__);
  std::string s;
  dispatch(c->grp, [&](auto ops) { s = decltype(ops)::schedule(c->grp); });
  snprintf(buf, (size_t)len, "%s", s.c_str());
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
  if (!(nu == c->cur_nu && dt == c->cur_dt)) {
    int st = set_coef(c->grp, c->stream, &nu, &dt);
    if (st != DNS_OK) return st;
    c->cur_nu = nu;
    c->cur_dt = dt;
  }
  const int K = c->kernels_per_step;
  // destroyed on every return path, the early ones of CK included
  struct Events {
    std::vector<cudaEvent_t> v;
    ~Events() {
      for (cudaEvent_t e : v)
        if (e) cudaEventDestroy(e);
    }
  } evs;
  evs.v.assign(K + 1, nullptr);
  std::vector<cudaEvent_t> &ev = evs.v;
  for (auto &e : ev) CK(cudaEventCreate(&e));
  for (int k = 0; k < K; k++) ms[k] = 0.0;
  int st = DNS_OK;
  for (long s = 0; s < nsteps && st == DNS_OK; s++) {
    CK(cudaEventRecord(ev[0], c->stream));
    for (int k = 0; k < K; k++) {
      dispatch(c->grp, [&](auto ops) {
        decltype(ops)::stage_kernel(c->grp, c->stream, k / KERNELS_PER_STAGE, k % KERNELS_PER_STAGE);
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
  for (int k = 0; k < K; k++) ms[k] /= (double)nsteps;
  return st;
}

/* ------------------------------------------------------------------ */
/* ensemble                                                            */
/* ------------------------------------------------------------------ */

static int ens_build_graph(dns_ens *e);
extern "C++" {
// ---- the persistent schedule ----
static bool ens_persistent_supported(const dns_ens *e) {
  if (e->groups.size() > (size_t)PMAXG) return false;
  for (const Group &G : e->groups)
    if (!p_supported_n(G.n)) return false;
  return true;
}

template <class R>
static int ens_build_persistent_t(dns_ens *e) {
  PPlan<R> plan{};
  plan.ngroups = (int)e->groups.size();
  size_t smem = 0;
  for (size_t q = 0; q < e->groups.size(); q++) {
    const Group &G = e->groups[q];
    dispatch(G, [&](auto ops) {
      using O = decltype(ops);
      if constexpr (std::is_same<typename O::Real, R>::value) O::plan_group(G, plan.gr[q]);
    });
    for (const PPhase<R> &P : plan.gr[q].ph) smem = std::max(smem, (size_t)(PBS / P.tpi) * P.smem);
  }
  int dev = 0, sms = 0, per = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CK(p_prepare<R>(smem, &per));
  if (per < 1) return fail(DNS_ERR_UNSUPPORTED, "persistent ensemble kernel does not fit", __FILE__, __LINE__);
  e->pgrid = per * sms;
  e->psmem = smem;
  CK(dev_malloc(&e->pplan, sizeof plan));
  CK(dev_malloc((void **)&e->psync, sizeof(PSync)));
  CK(cudaMemcpyAsync(e->pplan, &plan, sizeof plan, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemsetAsync(e->psync, 0, sizeof(PSync), e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return DNS_OK;
}

// limit of the persistent kernel's grid-barrier waits (a phase lasts
// microseconds to milliseconds)
constexpr unsigned long long P_WAIT_NS = 2000000000ull;

template <class R>
static cudaError_t ens_launch_persistent_t(dns_ens *e, cudaStream_t st) {
  return p_launch<R>(e->pgrid, e->psmem, st, (const PPlan<R> *)e->pplan, e->psync, P_WAIT_NS);
}

static cudaError_t ens_launch_persistent(dns_ens *e, cudaStream_t st) {
  return e->groups[0].precision == DNS_PREC_FP64 ? ens_launch_persistent_t<double>(e, st)
                                                 : ens_launch_persistent_t<float>(e, st);
}

static int ens_build_persistent(dns_ens *e) {
  int st = e->groups[0].precision == DNS_PREC_FP64 ? ens_build_persistent_t<double>(e)
                                                   : ens_build_persistent_t<float>(e);
  if (st != DNS_OK) return st;
  // one step = one graph of the single cooperative launch, where the
  // runtime captures it; else the launch itself
  cudaGraph_t gr = nullptr;
  e->pgraph_ok = false;
  if (cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
    cudaError_t le = ens_launch_persistent(e, e->stream);
    cudaError_t ce = cudaStreamEndCapture(e->stream, &gr);
    if (le == cudaSuccess && ce == cudaSuccess && gr &&
        cudaGraphInstantiate(&e->pgraph, gr, 0) == cudaSuccess)
      e->pgraph_ok = true;
    if (gr) cudaGraphDestroy(gr);
  }
  cudaGetLastError();  // a refused capture leaves no error behind
  return DNS_OK;
}

static int ens_step_persistent(dns_ens *e, long nsteps) {
  for (long s = 0; s < nsteps; s++) {
    if (e->pgraph_ok)
      CK(cudaGraphLaunch(e->pgraph, e->stream));
    else
      CK(ens_launch_persistent(e, e->stream));
  }
  return DNS_OK;
}

static int ens_check_persistent(dns_ens *e) {
  if (!e->psync) return DNS_OK;
  unsigned err = 0;
  CK(cudaMemcpyAsync(&err, &e->psync->err, sizeof err, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  if (err & PERR_BARRIER_TIMEOUT)
    return fail(DNS_ERR_CUDA, "a grid-barrier wait of the persistent ensemble kernel timed out",
                __FILE__, __LINE__);
  return DNS_OK;
}

// ms per step of the current schedule: one untimed step, then 3 timed
static int ens_time_steps(dns_ens *e, float *ms) {
  cudaEvent_t a = nullptr, b = nullptr;
  CK(cudaEventCreate(&a));
  cudaError_t ce = cudaEventCreate(&b);
  int st = ce == cudaSuccess ? DNS_OK : fail(DNS_ERR_CUDA, cudaGetErrorString(ce), __FILE__, __LINE__);
  auto one = [&]() -> int {
    if (e->mode == 1) return ens_step_persistent(e, 1);
    CK(cudaGraphLaunch(e->graph, e->stream));
    return DNS_OK;
  };
  if (st == DNS_OK) st = one();
  if (st == DNS_OK && (ce = cudaEventRecord(a, e->stream)) != cudaSuccess)
    st = fail(DNS_ERR_CUDA, cudaGetErrorString(ce), __FILE__, __LINE__);
  for (int i = 0; i < 3 && st == DNS_OK; i++) st = one();
  if (st == DNS_OK && (ce = cudaEventRecord(b, e->stream)) == cudaSuccess &&
      (ce = cudaEventSynchronize(b)) == cudaSuccess)
    ce = cudaEventElapsedTime(ms, a, b);
  if (st == DNS_OK && ce != cudaSuccess) st = fail(DNS_ERR_CUDA, cudaGetErrorString(ce), __FILE__, __LINE__);
  if (st == DNS_OK) st = ens_check_persistent(e);
  *ms /= 3.f;
  cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  return st;
}

// The ensemble autotuner: time both schedules on the fresh (all-zero) state,
// which every step keeps at zero, and keep the faster; the flags can force
// either.  A persistent schedule exists when every size group is one the
// persistent kernel compiles (32, 64, 128) and there are at most PMAXG.
static int ens_choose_schedule(dns_ens *e, unsigned flags) {
  const bool can = ens_persistent_supported(e);
  if ((flags & DNS_FLAG_ENS_PERSISTENT) && !can)
    return fail(DNS_ERR_UNSUPPORTED, "no persistent schedule for these grid sizes", __FILE__, __LINE__);
  int st = DNS_OK;
  const bool want_b = !(flags & DNS_FLAG_ENS_PERSISTENT);
  const bool want_p = can && !(flags & DNS_FLAG_ENS_BATCHED);
  if (want_b) {
    e->mode = 0;
    st = ens_build_graph(e);
    if (st == DNS_OK && want_p) st = ens_time_steps(e, &e->step_ms[0]);
  }
  if (st == DNS_OK && want_p) {
    e->mode = 1;
    st = ens_build_persistent(e);
    if (st == DNS_OK && want_b) st = ens_time_steps(e, &e->step_ms[1]);
  }
  if (st == DNS_OK && want_b && want_p) e->mode = e->step_ms[1] < e->step_ms[0] ? 1 : 0;
  return st;
}

}  // extern "C++"

int dns_ens_destroy(dns_ens *e) {
  if (!e) return DNS_OK;
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  if (e->pgraph) cudaGraphExecDestroy(e->pgraph);
  if (e->pplan) cudaFree(e->pplan);
  if (e->psync) cudaFree(e->psync);
  for (auto &G : e->groups) group_free(G);
  for (auto s : e->gstreams) cudaStreamDestroy(s);
  for (auto v : e->gevents) cudaEventDestroy(v);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->diag_host) cudaFreeHost(e->diag_host);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return DNS_OK;
}

int dns_ens_create(int nruns, const long *n, int precision, unsigned flags, dns_ens **out) {
  if (!out || !n || nruns < 1) return fail(DNS_ERR_ARG, "bad argument", __FILE__, __LINE__);
  *out = nullptr;
  dns_ens *e = new dns_ens();
  e->nruns = nruns;
  e->run_group.assign(nruns, -1);
  e->run_index.assign(nruns, -1);
  e->have_state.assign(nruns, 0);
  std::vector<long> sizes;
  for (int r = 0; r < nruns; r++) {
    int gi = -1;
    for (size_t q = 0; q < sizes.size(); q++)
      if (sizes[q] == n[r]) gi = (int)q;
    if (gi < 0) {
      gi = (int)sizes.size();
      sizes.push_back(n[r]);
    }
    e->run_group[r] = gi;
  }
  std::vector<int> counts(sizes.size(), 0);
  for (int r = 0; r < nruns; r++) e->run_index[r] = counts[e->run_group[r]]++;
  int st = DNS_OK;
  cudaError_t ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming);
  if (ce == cudaSuccess) ce = cudaMallocHost((void **)&e->diag_host, sizeof(double4) * nruns);
  if (ce != cudaSuccess) st = fail(DNS_ERR_CUDA, cudaGetErrorString(ce), __FILE__, __LINE__);
  e->groups.resize(sizes.size());
  for (size_t q = 0; q < sizes.size() && st == DNS_OK; q++) {
    st = group_init(e->groups[q], sizes[q], precision, flags, counts[q], e->stream);
    cudaStream_t gs = nullptr;
    cudaEvent_t ev = nullptr;
    if (st == DNS_OK) {
      ce = cudaStreamCreateWithFlags(&gs, cudaStreamNonBlocking);
      if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (ce != cudaSuccess) st = fail(DNS_ERR_CUDA, cudaGetErrorString(ce), __FILE__, __LINE__);
      if (gs) e->gstreams.push_back(gs);
      if (ev) e->gevents.push_back(ev);
    }
  }
  if (st == DNS_OK) st = ens_choose_schedule(e, flags);
  if (st != DNS_OK) {
    std::string keep = g_last_error;
    dns_ens_destroy(e);
    g_last_error = keep;
    return st;
  }
  *out = e;
  return DNS_OK;
}

static int ens_check_run(dns_ens *e, int run) {
  if (!e || run < 0 || run >= e->nruns) return fail(DNS_ERR_ARG, "bad run index", __FILE__, __LINE__);
  return DNS_OK;
}

int dns_ens_set_velocity(dns_ens *e, int run, const double *U, const double *V, const double *W) {
  int st = ens_check_run(e, run);
  if (st != DNS_OK) return st;
  if (!U || !V || !W) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  const Group view = e->groups[e->run_group[run]].one(e->run_index[run]);
  st = set_velocity_view(view, e->stream, U, V, W);
  if (st == DNS_OK) e->have_state[run] = 1;
  return st;
}

int dns_ens_set_tgv(dns_ens *e, int run) {
  int st = ens_check_run(e, run);
  if (st != DNS_OK) return st;
  st = init_view(e->groups[e->run_group[run]], e->run_index[run], e->stream, false, 0, 0.0);
  if (st == DNS_OK) e->have_state[run] = 1;
  return st;
}

int dns_ens_set_perturbed_tgv(dns_ens *e, int run, unsigned long long seed, double amplitude) {
  int st = ens_check_run(e, run);
  if (st != DNS_OK) return st;
  if (!isfinite(amplitude)) return fail(DNS_ERR_ARG, "bad amplitude", __FILE__, __LINE__);
  st = init_view(e->groups[e->run_group[run]], e->run_index[run], e->stream, true, seed, amplitude);
  if (st == DNS_OK) e->have_state[run] = 1;
  return st;
}

int dns_ens_set_params(dns_ens *e, const double *nu, const double *dt) {
  if (!e || !nu || !dt) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  for (size_t q = 0; q < e->groups.size(); q++) {
    const Group &G = e->groups[q];
    std::vector<double> gn(G.nruns), gd(G.nruns);
    for (int r = 0; r < e->nruns; r++)
      if (e->run_group[r] == (int)q) gn[e->run_index[r]] = nu[r], gd[e->run_index[r]] = dt[r];
    int st = set_coef(G, e->stream, gn.data(), gd.data());
    if (st != DNS_OK) return st;
  }
  e->params_set = true;
  return DNS_OK;
}

// one graph: a fork per size group (its own stream), each group's 24
// batched kernels, then a join
static int ens_build_graph(dns_ens *e) {
  if (e->graph) return DNS_OK;
  cudaGraph_t gr;
  CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  cudaEventRecord(e->fork, e->stream);
  for (size_t q = 0; q < e->groups.size(); q++) {
    cudaStreamWaitEvent(e->gstreams[q], e->fork, 0);
    const Group &G = e->groups[q];
    dispatch(G, [&](auto ops) { decltype(ops)::step(G, e->gstreams[q]); });
    cudaEventRecord(e->gevents[q], e->gstreams[q]);
    cudaStreamWaitEvent(e->stream, e->gevents[q], 0);
  }
  cudaError_t le = cudaGetLastError();
  cudaError_t ce = cudaStreamEndCapture(e->stream, &gr);
  if (le != cudaSuccess) return fail(DNS_ERR_CUDA, cudaGetErrorString(le), __FILE__, __LINE__);
  CK(ce);
  cudaError_t ie = cudaGraphInstantiate(&e->graph, gr, 0);
  cudaGraphDestroy(gr);
  CK(ie);
  return DNS_OK;
}

int dns_ens_step(dns_ens *e, long nsteps) {
  if (!e || nsteps < 0) return fail(DNS_ERR_ARG, "bad argument", __FILE__, __LINE__);
  for (int r = 0; r < e->nruns; r++)
    if (!e->have_state[r]) return fail(DNS_ERR_STATE, "a run has no velocity", __FILE__, __LINE__);
  if (!e->params_set) return fail(DNS_ERR_STATE, "nu and dt not set", __FILE__, __LINE__);
  if (nsteps == 0) return DNS_OK;
  if (e->mode == 1) return ens_step_persistent(e, nsteps);
  int st = ens_build_graph(e);
  if (st != DNS_OK) return st;
  for (long s = 0; s < nsteps; s++) CK(cudaGraphLaunch(e->graph, e->stream));
  return DNS_OK;
}

int dns_ens_get_schedule(dns_ens *e, char *buf, long len) {
  if (!e || !buf || len < 1) return fail(DNS_ERR_ARG, "bad argument", __FILE__, __LINE__);
  std::string s = e->mode == 1 ? "persistent" : "batched";
  char tmp[256];
  snprintf(tmp, sizeof tmp,
           " (ms per step: batched %.4f, persistent %.4f, -1 = not timed; persistent grid %d "
           "blocks of %d threads, %zu B shared, %s)",
           (double)e->step_ms[0], (double)e->step_ms[1], e->pgrid, PBS, e->psmem,
           e->pgraph_ok ? "graph-captured" : (e->pplan ? "direct launch" : "not built"));
  s += tmp;
  for (const Group &G : e->groups) {
    std::string g;
    dispatch(G, [&](auto ops) { g = decltype(ops)::schedule(G); });
    snprintf(tmp, sizeof tmp, "; n=%ld: ", G.n);
    s += tmp + g;
  }
  snprintf(buf, (size_t)len, "%s", s.c_str());
  return DNS_OK;
}

int dns_selftest_barrier_timeout(double limit_s, int *timed_out) {
  if (!timed_out || !(limit_s > 0.0) || limit_s > 10.0)
    return fail(DNS_ERR_ARG, "limit_s must be in (0, 10]", __FILE__, __LINE__);
  *timed_out = 0;
  cudaStream_t st = nullptr;
  PSync *d = nullptr;
  PSync h{};
  CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaError_t e = dev_malloc((void **)&d, sizeof(PSync));
  if (e == cudaSuccess) e = cudaMemsetAsync(d, 0, sizeof(PSync), st);
  if (e == cudaSuccess) e = p_barrier_selftest(d, st, (unsigned long long)(limit_s * 1e9));
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (d) cudaFree(d);
  cudaStreamDestroy(st);
  if (e != cudaSuccess) return fail(DNS_ERR_CUDA, cudaGetErrorString(e), __FILE__, __LINE__);
  *timed_out = (h.err & PERR_BARRIER_TIMEOUT) ? 1 : 0;
  return DNS_OK;
}

int dns_ens_diagnostics(dns_ens *e, double *out) {
  if (!e || !out) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  size_t base = 0;
  std::vector<size_t> gbase(e->groups.size());
  for (size_t q = 0; q < e->groups.size(); q++) {
    const Group &G = e->groups[q];
    dispatch(G, [&](auto ops) { decltype(ops)::diag(G, e->stream); });
    CKL();
    gbase[q] = base;
    CK(cudaMemcpyAsync(e->diag_host + base, G.diag_out, sizeof(double4) * G.nruns,
                       cudaMemcpyDeviceToHost, e->stream));
    base += G.nruns;
  }
  CK(cudaStreamSynchronize(e->stream));
  const int pst = ens_check_persistent(e);
  if (pst != DNS_OK) return pst;
  bool finite = true;
  for (int r = 0; r < e->nruns; r++) {
    const double4 v = e->diag_host[gbase[e->run_group[r]] + e->run_index[r]];
    out[4 * r + 0] = v.x;
    out[4 * r + 1] = v.y;
    out[4 * r + 2] = v.z;
    out[4 * r + 3] = v.w;
    finite = finite && isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w);
  }
  if (!finite) return fail(DNS_ERR_NONFINITE, "non-finite energy or enstrophy", __FILE__, __LINE__);
  return DNS_OK;
}

int dns_ens_get_spectral(dns_ens *e, int run, double *uvw) {
  int st = ens_check_run(e, run);
  if (st != DNS_OK) return st;
  if (!uvw) return fail(DNS_ERR_ARG, "NULL argument", __FILE__, __LINE__);
  return get_spectral_view(e->groups[e->run_group[run]].one(e->run_index[run]), e->stream, uvw);
}

void *dns_ens_get_stream(dns_ens *e) { return e ? (void *)e->stream : nullptr; }

int dns_ens_synchronize(dns_ens *e) {
  if (!e) return fail(DNS_ERR_ARG, "NULL ensemble", __FILE__, __LINE__);
  CK(cudaStreamSynchronize(e->stream));
  return ens_check_persistent(e);
}

/* ------------------------------------------------------------------ */
/* discrete adjoint                                                    */
/* ------------------------------------------------------------------ */

int dns_adjoint_energy_prec(long n, int precision, const double *U, const double *V,
                            const double *W, double nu, double dt, long nsteps, int snapshots,
                            double *J, double *gU, double *gV, double *gW, double *gnu) {
  if (!U || !V || !W || nsteps < 1 || snapshots < 1)
    return fail(DNS_ERR_ARG, "bad argument", __FILE__, __LINE__);
  if (precision != DNS_PREC_FP64 && precision != DNS_PREC_MIXED)
    return fail(DNS_ERR_ARG, "unknown precision", __FILE__, __LINE__);
  Adj A;
  CK(cudaStreamCreateWithFlags(&A.st, cudaStreamNonBlocking));
  int r = group_init(A.G, n, precision, 0, 1, A.st);
  auto cleanup = [&]() {
    if (A.st) cudaStreamSynchronize(A.st);
    if (A.graph) cudaGraphExecDestroy(A.graph);
    if (A.arena) cudaFree(A.arena);
    group_free(A.G);
    if (A.st) cudaStreamDestroy(A.st);
  };
  const Geo &g = A.G.g;
  if (r == DNS_OK) r = set_coef(A.G, A.st, &nu, &dt);
  A.nu = nu;
  A.dt = dt;
  A.nblocks = A.G.diag_blocks;
  if (r == DNS_OK) {
    const size_t sp_b = (size_t)NX * g.slot * A.G.csize;
    const size_t re_b = (size_t)NRE * g.nreal * sizeof(double);
    const size_t ssp_b = (size_t)snapshots * A.slot3();
    const size_t sre_b = (size_t)snapshots * A.real3();
    const size_t keep_b = (size_t)24 * g.nreal * A.G.rsize;
    const size_t part_b = (size_t)(A.nblocks + 1) * sizeof(double4);
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    bool zkeep = false;
    dispatch(A.G, [&](auto ops) { zkeep = decltype(ops)::ZKEEP; });
    const size_t keep_a = zkeep ? al(keep_b) : 0;
    cudaError_t e = dev_malloc((void **)&A.arena,
                               al(sp_b) + al(re_b) + al(ssp_b) + al(sre_b) + keep_a + al(part_b));
    if (e != cudaSuccess) {
      A.arena = nullptr;
      r = fail(DNS_ERR_NOMEM, cudaGetErrorString(e), __FILE__, __LINE__);
    } else {
      char *p = A.arena;
      A.sp = p; p += al(sp_b);
      A.re = (double *)p; p += al(re_b);
      A.snap_sp = p; p += al(ssp_b);
      A.snap_re = p; p += al(sre_b);
      if (zkeep) {
        A.keep = p;
        p += keep_a;
      }
      A.part = (double4 *)p;
      A.acc_nu = A.part + A.nblocks;
      e = cudaMemsetAsync(A.arena, 0, al(sp_b) + al(re_b), A.st);
      if (e == cudaSuccess) e = cudaMemsetAsync(A.acc_nu, 0, sizeof(double4), A.st);
      if (e != cudaSuccess) r = fail(DNS_ERR_CUDA, cudaGetErrorString(e), __FILE__, __LINE__);
    }
  }
  if (r == DNS_OK) {  // graph of one forward step
    cudaGraph_t gr;
    cudaError_t e = cudaStreamBeginCapture(A.st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      dispatch(A.G, [&](auto ops) { decltype(ops)::step(A.G, A.st); });
      e = cudaStreamEndCapture(A.st, &gr);
      if (e == cudaSuccess) {
        e = cudaGraphInstantiate(&A.graph, gr, 0);
        cudaGraphDestroy(gr);
      }
    }
    if (e != cudaSuccess) r = fail(DNS_ERR_CUDA, cudaGetErrorString(e), __FILE__, __LINE__);
  }
  // J alone: the forward sweep is all it takes (no snapshots are needed
  // beyond the first, and no reverse sweep runs)
  const bool want_grad = gU || gV || gW || gnu;
  if (r == DNS_OK) r = set_velocity_view(A.G, A.st, U, V, W);
  if (r == DNS_OK) r = adj_snap_store(A, 0);
  if (r == DNS_OK)  // forward sweep to T
    r = want_grad ? [&] {
      AdjDev x{A};
      return adj_sweep(x, nsteps, snapshots - 1);
    }()
                  : adj_advance(A, nsteps);
  double4 d = make_double4(0, 0, 0, 0);
  const double invn3 = 1.0 / (double)g.nreal;
  if (r == DNS_OK) {
    dispatch(A.G, [&](auto ops) { decltype(ops)::diag(A.G, A.st); });
    cudaError_t e = cudaMemcpyAsync(&d, A.G.diag_out, sizeof(double4), cudaMemcpyDeviceToHost, A.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(A.st);
    if (e != cudaSuccess) r = fail(DNS_ERR_CUDA, cudaGetErrorString(e), __FILE__, __LINE__);
  }
  if (r == DNS_OK && !want_grad) {
    if (J) *J = (d.x + d.y) * (invn3 * invn3);
    cleanup();
    return r;
  }
  if (r == DNS_OK) {
    // lambda(T) = dE/dU_hat = 2 invn3^2 U_hat(T); the stale velocity at T
    // does not enter E
    dispatch(A.G, [&](auto ops) {
      using C = typename decltype(ops)::C;
      k_lincomb3<C><<<A.nblocks, 256, 0, A.st>>>((const C *)A.G.slot_ptr(0, SLOT_SA), nullptr,
                                                 A.X<C>(A.lhat), g, 2.0 * invn3 * invn3, 0.0);
    });
    cudaError_t e = cudaMemsetAsync(A.Rf(RE_LSTALE), 0, A.real3d(), A.st);
    if (e != cudaSuccess) r = fail(DNS_ERR_CUDA, cudaGetErrorString(e), __FILE__, __LINE__);
  }
  if (r == DNS_OK) {
    AdjDev x{A};
    r = adj_reverse(x, 0, nsteps, 0, snapshots - 1, true);
  }
  if (r == DNS_OK) {
    // dE/du0 = r2c^T(lambda_U(0)) + lambda_stale(0) = c2r(lambda / w_z) + lambda_stale
    const int t3[3] = {0, 1, 2};
    dispatch(A.G, [&](auto ops) {
      using O = decltype(ops);
      using C = typename O::C;
      k_div_wz3<C><<<A.nblocks, 256, 0, A.st>>>(A.X<C>(A.lhat), A.X<C>(X_T1), g);
      O::c2r_fields(A.G, A.st, A.X<C>(X_T1), t3, 3, A.Rf(RE_LN), 1.0);
    });
    k_add_real<<<conv_blocks(3 * g.nreal), 256, 0, A.st>>>(A.Rf(RE_LSTALE), A.Rf(RE_LN), 3 * g.nreal);
    cudaError_t e = cudaGetLastError();
    double *dst[3] = {gU, gV, gW};
    for (int f = 0; f < 3 && e == cudaSuccess; f++)
      if (dst[f])
        e = cudaMemcpyAsync(dst[f], A.Rf(RE_LN + f), (size_t)g.nreal * sizeof(double),
                            cudaMemcpyDeviceToHost, A.st);
    double4 gn = make_double4(0, 0, 0, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&gn, A.acc_nu, sizeof(double4), cudaMemcpyDeviceToHost, A.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(A.st);
    if (e != cudaSuccess) r = fail(DNS_ERR_CUDA, cudaGetErrorString(e), __FILE__, __LINE__);
    if (J) *J = (d.x + d.y) * (invn3 * invn3);
    if (gnu) *gnu = gn.x + gn.y;
  }
  cleanup();
  return r;
}

int dns_adjoint_schedule(long nsteps, int snapshots, long *forward_steps, long *recomputed_steps,
                         int *snapshots_used) {
  if (nsteps < 1 || snapshots < 1)
    return fail(DNS_ERR_ARG, "nsteps and snapshots must be >= 1", __FILE__, __LINE__);
  AdjCount x;
  adj_sweep(x, nsteps, snapshots - 1);
  const long sweep = x.advanced;
  adj_reverse(x, 0, nsteps, 0, snapshots - 1, true);
  if (forward_steps) *forward_steps = x.advanced;
  if (recomputed_steps) *recomputed_steps = x.advanced - sweep;
  if (snapshots_used) *snapshots_used = x.used;
  return DNS_OK;
}

int dns_adjoint_energy(long n, const double *U, const double *V, const double *W, double nu,
                       double dt, long nsteps, int snapshots, double *J, double *gU, double *gV,
                       double *gW, double *gnu) {
  return dns_adjoint_energy_prec(n, DNS_PREC_FP64, U, V, W, nu, dt, nsteps, snapshots, J, gU, gV,
                                 gW, gnu);
}

}  // extern "C"
