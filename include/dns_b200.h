/*
 * dns_b200.h -- C ABI of the B200 (sm_100a) pseudo-spectral RK4 stepper.
 *
 * Drop-in for the time-stepping path of slitvinov/dns main.c: the CLI
 * (dns_b200/cli/dns.c) and the tests call the same library.  The reference has
 * no library interface -- the path is inline in main() -- so every entry point
 * below names the block of main.c it replaces.
 *
 * Conventions
 *   - n is the grid size; the box is [0, 2 pi)^3 with n^3 nodes.  Supported:
 *     n a power of two, 8 <= n <= 512.
 *   - real fields are float64 [x][y][z] (z fastest), the .raw layout of
 *     main.c:180-185 / tgv.py:19-27.
 *   - spectral fields are complex float64 (re, im interleaved) on the half
 *     spectrum [kx][ky][kz], kz in [0, n/2], the FFTW r2c layout main.c uses
 *     (main.c:236); they are unnormalised like FFTW's r2c output.
 *   - host pointers are borrowed for the duration of the call only; the
 *     library owns all device memory.
 *   - every function returns a status (DNS_OK == 0); the library never exits.
 *   - a context owns one CUDA stream; it is not thread-safe, independent
 *     contexts may be driven from different host threads.
 */
#ifndef DNS_B200_H
#define DNS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  DNS_OK = 0,
  DNS_ERR_ARG = 1,        /* invalid argument (null pointer, bad size) */
  DNS_ERR_UNSUPPORTED = 2,/* grid size or precision not supported */
  DNS_ERR_CUDA = 3,       /* CUDA runtime error; see dns_last_error() */
  DNS_ERR_NOMEM = 4,      /* device or pinned host allocation failed */
  DNS_ERR_NONFINITE = 5,  /* diagnostics are NaN or Inf (main.c dies on
                             SIGFPE there, main.c:49-50) */
  DNS_ERR_STATE = 6       /* call out of order (e.g. step before velocity) */
};

/* precision of a context:
 *   DNS_PREC_FP64   everything in float64 (the reference's arithmetic);
 *   DNS_PREC_MIXED  fields, FFTs, the nonlinear term, the projection and the
 *                   RK axpys in float32 (twiddles generated in long double
 *                   and rounded once); the energy/enstrophy reductions
 *                   (double-double) and the viscous coefficient nu dt |k|^2
 *                   in float64, the latter rounded once per point.
 * Host-side arrays are float64 for both. */
enum { DNS_PREC_FP64 = 0, DNS_PREC_MIXED = 1 };

/* flags for dns_create (and dns_ens_create) */
enum {
  DNS_FLAG_PRESSURE = 1u, /* keep the pressure P_hat of the last RK stage so
                             that dns_get_fields can return P (needed by the
                             -d dump, main.c:269-279) */
  /* dns_ens_create only: force the ensemble's schedule instead of letting
   * its autotuner time both (see dns_ens_create) */
  DNS_FLAG_ENS_BATCHED = 2u,
  DNS_FLAG_ENS_PERSISTENT = 4u
};

typedef struct dns_ctx dns_ctx;

/* Allocate device state for an n^3 grid and build twiddle tables.
 * Replaces main.c:174-247 (allocations, FFTW plans, kx/kz, dealias, kk). */
int dns_create(long n, int precision, unsigned flags, dns_ctx **out);

/* Free everything owned by ctx.  Replaces main.c:424-460. */
int dns_destroy(dns_ctx *ctx);

/* Upload the initial velocity (three n^3 float64 arrays, host memory) and
 * transform it: U_hat = r2c(U) etc.  The raw input also becomes the stale
 * real-space velocity used by stage rk == 0 of step 0.
 * Replaces main.c:180-185 (after fread) and main.c:249-251. */
int dns_set_velocity(dns_ctx *ctx, const double *U, const double *V, const double *W);

/* Advance nsteps RK4 steps with viscosity nu and time step dt.
 * Replaces one iteration of main.c:334-422 per step (time and step counters,
 * printing and the t > T test of main.c:332 stay with the caller). */
int dns_step(dns_ctx *ctx, double nu, double dt, long nsteps);

/* Energy and enstrophy of the current state, as double-double pairs:
 *   E  = (e_hi + e_lo)  * invn3 * invn3,  Om = (om_hi + om_lo) * invn3 * invn3
 * where the sums run over the half spectrum exactly as main.c:257-266 (no
 * Hermitian weighting); the caller applies the scale in long double like
 * main.c:265-266.  Returns DNS_ERR_NONFINITE (values still filled) when a sum
 * is NaN or Inf. */
int dns_diagnostics(dns_ctx *ctx, double *e_hi, double *e_lo, double *om_hi, double *om_lo);

/* Real-space fields c2r(X_hat) / n^3 for X = U, V, W and (if the context was
 * created with DNS_FLAG_PRESSURE) the pressure P of the last RK stage, into
 * four n^3 float64 host arrays.  Any pointer may be NULL to skip that field.
 * Replaces the dump transform of main.c:270-279. */
int dns_get_fields(dns_ctx *ctx, double *U, double *V, double *W, double *P);

/* Initial velocity generated on the device, with no n^3 host transfer; the
 * field also becomes the stale real-space velocity of step 0, exactly as
 * after dns_set_velocity.
 *
 * dns_set_tgv: the Taylor-Green field tgv.py writes (tgv.py:14-27),
 *   U = sin x cos y cos z, V = -cos x sin y cos z, W = 0 at x_i = i 2 pi / n,
 *   bit-identical to tgv.py's .raw (same 1-D sin/cos tables, same order of
 *   the products).  Replaces `python tgv.py -l L -o f.raw` + main.c:163-185
 *   + main.c:249-251.
 * dns_set_perturbed_tgv: the same plus a seeded solenoidal perturbation with
 *   energy spectrum E(k) ~ k^4 exp(-2 (k/4)^2) and rms = amplitude times the
 *   rms of the Taylor-Green field (white Gaussian noise from a counter-based
 *   generator keyed by seed, r2c, shaped and projected per mode, c2r, scaled
 *   to unit rms).  No counterpart in the reference; it is the initial field
 *   of the ensemble configuration.  In a DNS_PREC_MIXED context the
 *   perturbation is shaped with float32 transforms. */
int dns_set_tgv(dns_ctx *ctx);
int dns_set_perturbed_tgv(dns_ctx *ctx, unsigned long long seed, double amplitude);

/* Human-readable text of a status / of the last error on this thread. */
const char *dns_strerror(int status);
const char *dns_last_error(void);

/* ---- state access (restart, parity tests) ----
 * The full step state is (U_hat, V_hat, W_hat) plus the stale real-space
 * velocity (main.c's U, V, W arrays between steps). */

/* spectral velocity as [3][n][n][n/2+1] complex float64 (2*3*n*n*(n/2+1)
 * doubles) */
int dns_get_spectral(dns_ctx *ctx, double *uvw_hat);
int dns_set_spectral(dns_ctx *ctx, const double *uvw_hat);
/* stale real-space velocity, [3][n^3] float64 */
int dns_get_stale(dns_ctx *ctx, double *uvw);
int dns_set_stale(dns_ctx *ctx, const double *uvw);

/* ---- introspection / measurement ---- */
typedef struct {
  long n;
  int precision;
  unsigned flags;
  size_t device_bytes;     /* device memory held by the context */
  size_t slot_bytes;       /* bytes of one padded spectral field */
  int kernels_per_step;    /* kernel launches in one RK4 step */
} dns_info_t;
int dns_get_info(dns_ctx *ctx, dns_info_t *info);
/* The kernel schedule the library's autotuner chose for this context's grid
 * size and precision (no counterpart in the reference): for each column
 * pass, the register schedule (minimum resident blocks per SM) picked by
 * timing every compiled candidate once per process, size, precision and
 * batch shape, with the measured times (an ensemble group is timed on its
 * own runs, up to the volume of two 256^3 runs; its schedule then starts
 * "timed on <k> runs: ").  All candidates compute bit-identical results.  The environment
 * variable DNS_B200_TUNE=0 keeps the compiler's schedule; DNS_B200_TUNE=f<k>
 * forces candidate k; DNS_B200_TUNE=m<a>,<b>,<c>,<d> the schedules of a, b,
 * c, d min blocks/SM for the x inverse, x forward, y inverse and y forward
 * passes (to reproduce a reported choice, e.g. under a profiler).  Writes a
 * NUL-terminated text of at most len bytes. */
int dns_get_schedule(dns_ctx *ctx, char *buf, long len);

/* The context's CUDA stream (a cudaStream_t), for callers that time work
 * with CUDA events on it. */
void *dns_get_stream(dns_ctx *ctx);

/* Wait for all work queued on the context's stream. */
int dns_synchronize(dns_ctx *ctx);

/* Time each kernel of the step: runs nsteps steps launch by launch with CUDA
 * events between kernels and writes the mean time in milliseconds of each of
 * the kernels_per_step launches of a step into ms[] (stage-major order:
 * stage 0 passes A..E, stage 1 ..., stage 3).  The state advances by
 * nsteps. */
int dns_time_kernels(dns_ctx *ctx, double nu, double dt, long nsteps, double *ms);

/* ---- ensemble: many independent runs stepped together ----
 * No counterpart in the reference's main loop; it generalises its
 * process-level ensembles (run.sh / hal.sh run one dns per core).  Runs of
 * any grid sizes and viscosities advance together, each following main.c's
 * step exactly (stale velocity included), under one of two schedules:
 *   batched     runs of equal n share batched kernel launches (24 per step),
 *               groups of different n run as concurrent branches of one
 *               CUDA graph launch per step;
 *   persistent  one cooperative kernel launch per step (captured in a CUDA
 *               graph) walks the 24 passes of every run of every size, the
 *               passes separated by grid-wide barriers (grid sizes 32, 64
 *               and 128, at most four distinct sizes).
 * Both give bit-identical states.  dns_ens_create times both on the fresh
 * ensemble and keeps the faster (its autotuner) unless a flag forces one:
 * DNS_FLAG_ENS_BATCHED or DNS_FLAG_ENS_PERSISTENT (DNS_ERR_UNSUPPORTED when
 * the sizes have no persistent schedule).  A barrier wait of the persistent
 * kernel that runs past its limit (2 s) makes the kernel end and the next
 * dns_ens_synchronize / dns_ens_diagnostics return DNS_ERR_CUDA. */
typedef struct dns_ens dns_ens;
/* nruns runs, run r of grid size n[r] (same precision and flags for all) */
int dns_ens_create(int nruns, const long *n, int precision, unsigned flags, dns_ens **out);
/* the schedule the ensemble runs (and the timings that chose it), text of
 * at most len bytes */
int dns_ens_get_schedule(dns_ens *e, char *buf, long len);
/* Self-test of the persistent kernel's bounded barrier wait (no counterpart
 * in the reference): a grid barrier that one block never reaches must give
 * up after limit_s seconds (0 < limit_s <= 10) and report it in the error
 * word; *timed_out = 1 when it did. */
int dns_selftest_barrier_timeout(double limit_s, int *timed_out);
int dns_ens_destroy(dns_ens *e);
/* initial velocity of one run (as dns_set_velocity) */
int dns_ens_set_velocity(dns_ens *e, int run, const double *U, const double *V, const double *W);
/* initial velocity of one run generated on the device (as dns_set_tgv /
 * dns_set_perturbed_tgv) */
int dns_ens_set_tgv(dns_ens *e, int run);
int dns_ens_set_perturbed_tgv(dns_ens *e, int run, unsigned long long seed, double amplitude);
/* viscosity and time step of every run (arrays of nruns) */
int dns_ens_set_params(dns_ens *e, const double *nu, const double *dt);
/* advance every run by nsteps RK4 steps */
int dns_ens_step(dns_ens *e, long nsteps);
/* per-run double-double sums as dns_diagnostics: out[4 r + 0..3] =
 * e_hi, e_lo, om_hi, om_lo of run r */
int dns_ens_diagnostics(dns_ens *e, double *out);
/* spectral velocity of one run, layout of dns_get_spectral */
int dns_ens_get_spectral(dns_ens *e, int run, double *uvw_hat);
void *dns_ens_get_stream(dns_ens *e);
int dns_ens_synchronize(dns_ens *e);

/* ---- discrete adjoint ----
 * No counterpart in the reference.  Gradient of the final energy
 *   J = E(T) = invn3^2 * sum over the half spectrum of |U_hat(T)|^2
 * (main.c:257-266's definition, no Hermitian weighting) after nsteps RK4
 * steps of main.c's scheme (stale first-stage velocity included) from the
 * initial velocity U, V, W (host, n^3 each), with respect to that initial
 * velocity (gU, gV, gW: host, n^3 each, dJ/du0 at every grid point) and to
 * nu (gnu).  FP64.  The transposed step is hand-written; forward states are
 * recomputed from `snapshots` stored step states (>= 1, the initial state
 * included) placed by a binomial split of the step range, so memory is
 * independent of nsteps: the snapshots (3 spectral and 3 real fields each)
 * plus a fixed work set (41 spectral and 45 real fields, the step's own
 * state included; 256^3 FP64 with 20 snapshots: about 28 GB).  Any output pointer may be NULL;
 * with all four gradient pointers NULL only the forward sweep runs (J
 * alone). */
int dns_adjoint_energy(long n, const double *U, const double *V, const double *W, double nu,
                       double dt, long nsteps, int snapshots, double *J, double *gU, double *gV,
                       double *gW, double *gnu);
/* The same with a choice of precision: DNS_PREC_FP64 (dns_adjoint_energy)
 * or DNS_PREC_MIXED, whose forward recomputation is the mixed step itself
 * (FP32 spectral storage and transforms, FP64 viscous coefficients and
 * reductions) and whose transposed step keeps the same FP32 storage and
 * transforms with its pointwise products, the nu gradient and the float64
 * host-facing gradient in FP64.  Its J is the mixed path's E(T), its
 * gradient the exact adjoint of that rounded map to within FP32 transform
 * error (about 1e-5 relative to the FP64 gradient). */
int dns_adjoint_energy_prec(long n, int precision, const double *U, const double *V,
                            const double *W, double nu, double dt, long nsteps, int snapshots,
                            double *J, double *gU, double *gV, double *gW, double *gnu);
/* The checkpoint schedule the two calls above follow for nsteps steps and
 * `snapshots` stored states, counted on the host (no GPU work; callable
 * without a GPU), to choose `snapshots` against time: forward_steps = the
 * steps of the first sweep (nsteps) plus those recomputed from snapshots
 * (recomputed_steps); each reversed step then re-runs its own stages once
 * more.  snapshots_used <= snapshots.  With snapshots >= nsteps nothing is
 * recomputed; with 1, every step is recomputed from the start (nsteps *
 * (nsteps - 1) / 2).  Any output pointer may be NULL. */
int dns_adjoint_schedule(long nsteps, int snapshots, long *forward_steps, long *recomputed_steps,
                         int *snapshots_used);

/* Energy and enstrophy of a spectral velocity held in caller-owned device
 * memory, allocating nothing.  No counterpart in the reference (main.c has
 * no library interface); this is an addition for callers that may not call
 * cudaMalloc where they need the diagnostics: work being recorded into a CUDA
 * graph, frameworks whose memory pool owns the device memory, monitoring
 * loops that must not trigger the synchronisation an allocation can cause.
 *   n       grid size, power of two in [8, 512]
 *   uvw_hat device pointer, [3][n][n][n/2+1] complex float64 (the layout of
 *           dns_get_spectral), unnormalised like FFTW's r2c
 *   out     device pointer to 4 doubles: e_hi, e_lo, om_hi, om_lo, the same
 *           double-double sums dns_diagnostics returns (scale by
 *           invn3 * invn3 as main.c:265-266 does)
 *   stream  a cudaStream_t (NULL: the legacy default stream); the call only
 *           queues work, the caller synchronises before reading out
 * Scratch is a fixed 263 KB device array inside the library (every GPU that
 * loads the library holds it until exit), sized for the n = 512 grid: larger
 * inputs (more than 67,371,008 half-spectrum points) are rejected with
 * DNS_ERR_UNSUPPORTED, as is any n outside the range.  The first call in a
 * CUDA context (on each device, and again after cudaDeviceReset or under
 * another context) looks up that array's device address and loads the
 * kernels, so make it before any stream capture.
 * Every call shares the array: calls that can overlap on the GPU (different
 * streams without ordering, or different host threads on one device) race;
 * serialise them.  Nothing in it has to start at zero (each call overwrites
 * every entry it reads). */
int dns_diagnostics_noalloc(long n, const double *uvw_hat, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
