/*
 * shim_fft.c -- project-written double precision FFT behind the FFTW-subset
 * shim (fftw3.h).  ORACLE / TEST INFRASTRUCTURE ONLY: the product never links
 * or calls this file.
 *
 * Algorithm: batched Stockham autosort FFT (radix 4, one radix-2 stage when
 * log2 n is odd) over B interleaved lines so that the innermost loop runs over
 * lines with one shared twiddle (vectorisable).  Real transforms of length n
 * go through a complex FFT of length n/2 plus the standard even/odd
 * pre/post-processing.  Twiddles are generated in long double with octant
 * reduction so that exact symmetries (0, +-1, sqrt(1/2)) hold bit for bit.
 * Lengths that are not powers of two use a direct O(n^2) DFT (tests only).
 *
 * Conventions follow FFTW3 as used by main.c (see fftw3.h).
 */
#define _GNU_SOURCE
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { BATCH = 8 };
enum { KIND_R2C = 1, KIND_C2R = 2 };

struct shim_plan_s {
  int kind;
  int rank;
  long n[3];
  double *rin;
  fftw_complex *cin;
  double *rout;
  fftw_complex *cout;
};

/* cos(2 pi k / n), sin(2 pi k / n) with octant reduction in long double. */
void shim_sincos2pi(long k, long n, double *c, double *s) {
  static const long double PI_L = 3.141592653589793238462643383279502884L;
  k %= n;
  if (k < 0)
    k += n;
  /* angle = 2 pi k / n = (q + r / n) * pi / 2 with 4k = q n + r */
  long q = (4 * k) / n;
  long r = (4 * k) % n;
  long double cc, ss;
  if (r == 0) {
    cc = 1.0L;
    ss = 0.0L;
  } else if (2 * r <= n) {
    long double x = (PI_L / 2.0L) * (long double)r / (long double)n;
    cc = cosl(x);
    ss = sinl(x);
  } else {
    long double x = (PI_L / 2.0L) * (long double)(n - r) / (long double)n;
    cc = sinl(x);
    ss = cosl(x);
  }
  double c0 = (double)cc, s0 = (double)ss;
  switch (q) {
  case 0:
    *c = c0;
    *s = s0;
    break;
  case 1:
    *c = -s0;
    *s = c0;
    break;
  case 2:
    *c = -c0;
    *s = -s0;
    break;
  default:
    *c = s0;
    *s = -c0;
    break;
  }
}

static int is_pow2(long n) { return n > 0 && (n & (n - 1)) == 0; }

/* twiddle table e^{-2 pi i k / n}, k in [0, n) */
typedef struct {
  long n;
  double *wr, *wi;
} twtab;

static void twtab_init(twtab *t, long n) {
  t->n = n;
  t->wr = malloc(sizeof(double) * (n > 0 ? n : 1));
  t->wi = malloc(sizeof(double) * (n > 0 ? n : 1));
  for (long k = 0; k < n; k++) {
    double c, s;
    shim_sincos2pi(k, n, &c, &s);
    t->wr[k] = c;
    t->wi[k] = -s;
  }
}
static void twtab_free(twtab *t) {
  free(t->wr);
  free(t->wi);
}

/*
 * In-place batched complex FFT of length n over B lines stored interleaved:
 * element m of line b at [m * B + b].  sign = -1 forward, +1 backward.
 * yr/yi: scratch of the same size.
 */
static void cfft_batch(const twtab *t, int sign, double *xr, double *xi,
                       double *yr, double *yi, int B) {
  long n = t->n;
  if (n <= 1)
    return;
  if (!is_pow2(n)) {
    /* direct DFT */
    for (long k = 0; k < n; k++)
      for (int b = 0; b < B; b++) {
        double sr = 0, si = 0;
        for (long j = 0; j < n; j++) {
          long idx = (j * k) % n;
          double wr = t->wr[idx], wi = sign < 0 ? t->wi[idx] : -t->wi[idx];
          double ar = xr[j * B + b], ai = xi[j * B + b];
          sr += ar * wr - ai * wi;
          si += ar * wi + ai * wr;
        }
        yr[k * B + b] = sr;
        yi[k * B + b] = si;
      }
    memcpy(xr, yr, sizeof(double) * n * B);
    memcpy(xi, yi, sizeof(double) * n * B);
    return;
  }
  double *sr = xr, *si = xi, *dr = yr, *di = yi;
  long Ns = 1;
  while (Ns < n) {
    int R = ((n / Ns) % 4 == 0) ? 4 : 2;
    long NR = n / R;
    long tstep = n / (Ns * R);
    for (long j = 0; j < NR; j++) {
      long jm = j % Ns;
      long idxD = (j / Ns) * Ns * R + jm;
      if (R == 4) {
        double w1r = t->wr[jm * tstep], w1i = t->wi[jm * tstep];
        double w2r = t->wr[2 * jm * tstep], w2i = t->wi[2 * jm * tstep];
        double w3r = t->wr[3 * jm * tstep], w3i = t->wi[3 * jm * tstep];
        if (sign > 0) {
          w1i = -w1i;
          w2i = -w2i;
          w3i = -w3i;
        }
        const double *a0r = sr + (j)*B, *a0i = si + (j)*B;
        const double *a1r = sr + (j + NR) * B, *a1i = si + (j + NR) * B;
        const double *a2r = sr + (j + 2 * NR) * B, *a2i = si + (j + 2 * NR) * B;
        const double *a3r = sr + (j + 3 * NR) * B, *a3i = si + (j + 3 * NR) * B;
        double *o0r = dr + (idxD)*B, *o0i = di + (idxD)*B;
        double *o1r = dr + (idxD + Ns) * B, *o1i = di + (idxD + Ns) * B;
        double *o2r = dr + (idxD + 2 * Ns) * B, *o2i = di + (idxD + 2 * Ns) * B;
        double *o3r = dr + (idxD + 3 * Ns) * B, *o3i = di + (idxD + 3 * Ns) * B;
        for (int b = 0; b < B; b++) {
          double v0r = a0r[b], v0i = a0i[b];
          double v1r = a1r[b] * w1r - a1i[b] * w1i;
          double v1i = a1r[b] * w1i + a1i[b] * w1r;
          double v2r = a2r[b] * w2r - a2i[b] * w2i;
          double v2i = a2r[b] * w2i + a2i[b] * w2r;
          double v3r = a3r[b] * w3r - a3i[b] * w3i;
          double v3i = a3r[b] * w3i + a3i[b] * w3r;
          double t0r = v0r + v2r, t0i = v0i + v2i;
          double t1r = v0r - v2r, t1i = v0i - v2i;
          double t2r = v1r + v3r, t2i = v1i + v3i;
          double t3r = v1r - v3r, t3i = v1i - v3i;
          o0r[b] = t0r + t2r;
          o0i[b] = t0i + t2i;
          o2r[b] = t0r - t2r;
          o2i[b] = t0i - t2i;
          if (sign < 0) { /* X1 = t1 - i t3, X3 = t1 + i t3 */
            o1r[b] = t1r + t3i;
            o1i[b] = t1i - t3r;
            o3r[b] = t1r - t3i;
            o3i[b] = t1i + t3r;
          } else {
            o1r[b] = t1r - t3i;
            o1i[b] = t1i + t3r;
            o3r[b] = t1r + t3i;
            o3i[b] = t1i - t3r;
          }
        }
      } else {
        double w1r = t->wr[jm * tstep], w1i = t->wi[jm * tstep];
        if (sign > 0)
          w1i = -w1i;
        const double *a0r = sr + (j)*B, *a0i = si + (j)*B;
        const double *a1r = sr + (j + NR) * B, *a1i = si + (j + NR) * B;
        double *o0r = dr + (idxD)*B, *o0i = di + (idxD)*B;
        double *o1r = dr + (idxD + Ns) * B, *o1i = di + (idxD + Ns) * B;
        for (int b = 0; b < B; b++) {
          double v0r = a0r[b], v0i = a0i[b];
          double v1r = a1r[b] * w1r - a1i[b] * w1i;
          double v1i = a1r[b] * w1i + a1i[b] * w1r;
          o0r[b] = v0r + v1r;
          o0i[b] = v0i + v1i;
          o1r[b] = v0r - v1r;
          o1i[b] = v0i - v1i;
        }
      }
    }
    double *tr = sr, *ti = si;
    sr = dr;
    si = di;
    dr = tr;
    di = ti;
    Ns *= R;
  }
  if (sr != xr) {
    memcpy(xr, sr, sizeof(double) * n * B);
    memcpy(xi, si, sizeof(double) * n * B);
  }
}

/* per-thread scratch */
typedef struct {
  double *xr, *xi, *yr, *yi;
} scratch;
static void scratch_init(scratch *s, long n) {
  size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1) * BATCH;
  s->xr = malloc(sz);
  s->xi = malloc(sz);
  s->yr = malloc(sz);
  s->yi = malloc(sz);
}
static void scratch_free(scratch *s) {
  free(s->xr);
  free(s->xi);
  free(s->yr);
  free(s->yi);
}

/*
 * complex transform along one axis of a [outer][len][inner] array of
 * complex values (line stride = inner), for all outer and inner indices.
 */
static void axis_cfft(double _Complex *a, long outer, long len, long inner,
                      int sign) {
  if (len <= 1)
    return;
  twtab t;
  twtab_init(&t, len);
  long nb = (inner + BATCH - 1) / BATCH;
  long total = outer * nb;
#pragma omp parallel
  {
    scratch s;
    scratch_init(&s, len);
#pragma omp for schedule(static)
    for (long job = 0; job < total; job++) {
      long o = job / nb;
      long i0 = (job % nb) * BATCH;
      int B = (int)((inner - i0) < BATCH ? (inner - i0) : BATCH);
      double _Complex *base = a + o * len * inner + i0;
      for (long m = 0; m < len; m++)
        for (int b = 0; b < B; b++) {
          s.xr[m * B + b] = creal(base[m * inner + b]);
          s.xi[m * B + b] = cimag(base[m * inner + b]);
        }
      cfft_batch(&t, sign, s.xr, s.xi, s.yr, s.yi, B);
      for (long m = 0; m < len; m++)
        for (int b = 0; b < B; b++)
          base[m * inner + b] = CMPLX(s.xr[m * B + b], s.xi[m * B + b]);
    }
    scratch_free(&s);
  }
  twtab_free(&t);
}

/* r2c along the last (contiguous) axis: in[lines][n] real -> out[lines][n/2+1] */
static void lastaxis_r2c(const double *in, double _Complex *out, long lines,
                         long n) {
  long nf = n / 2 + 1;
  if (n % 2 != 0 || !is_pow2(n)) {
    twtab t;
    twtab_init(&t, n);
#pragma omp parallel
    {
      scratch s;
      scratch_init(&s, n);
#pragma omp for schedule(static)
      for (long l = 0; l < lines; l++) {
        for (long m = 0; m < n; m++) {
          s.xr[m] = in[l * n + m];
          s.xi[m] = 0.0;
        }
        cfft_batch(&t, -1, s.xr, s.xi, s.yr, s.yi, 1);
        for (long k = 0; k < nf; k++)
          out[l * nf + k] = CMPLX(s.xr[k], s.xi[k]);
      }
      scratch_free(&s);
    }
    twtab_free(&t);
    return;
  }
  long M = n / 2;
  twtab t, tn;
  twtab_init(&t, M);
  twtab_init(&tn, n);
  long nb = (lines + BATCH - 1) / BATCH;
#pragma omp parallel
  {
    scratch s;
    scratch_init(&s, M);
#pragma omp for schedule(static)
    for (long job = 0; job < nb; job++) {
      long l0 = job * BATCH;
      int B = (int)((lines - l0) < BATCH ? (lines - l0) : BATCH);
      for (long m = 0; m < M; m++)
        for (int b = 0; b < B; b++) {
          s.xr[m * B + b] = in[(l0 + b) * n + 2 * m];
          s.xi[m * B + b] = in[(l0 + b) * n + 2 * m + 1];
        }
      cfft_batch(&t, -1, s.xr, s.xi, s.yr, s.yi, B);
      for (int b = 0; b < B; b++) {
        double _Complex *o = out + (l0 + b) * nf;
        double z0r = s.xr[b], z0i = s.xi[b];
        o[0] = CMPLX(z0r + z0i, 0.0);
        o[M] = CMPLX(z0r - z0i, 0.0);
        for (long k = 1; k < M; k++) {
          /* X[k] = 1/2 (Z[k] + conj Z[M-k]) - 1/2 i W^k (Z[k] - conj Z[M-k]) */
          double zr = s.xr[k * B + b], zi = s.xi[k * B + b];
          double cr = s.xr[(M - k) * B + b], ci = -s.xi[(M - k) * B + b];
          double er = 0.5 * (zr + cr), ei = 0.5 * (zi + ci);
          double dr = 0.5 * (zr - cr), di = 0.5 * (zi - ci);
          /* -i W^k d with W^k = (wr + i wi) */
          double wr = tn.wr[k], wi = tn.wi[k];
          double pr = wr * dr - wi * di, pi = wr * di + wi * dr;
          o[k] = CMPLX(er + pi, ei - pr);
        }
      }
    }
    scratch_free(&s);
  }
  twtab_free(&t);
  twtab_free(&tn);
}

/* c2r along the last axis: in[lines][n/2+1] -> out[lines][n] real.
 * The imaginary parts of in[.][0] and (even n) in[.][n/2] are ignored. */
static void lastaxis_c2r(const double _Complex *in, double *out, long lines,
                         long n) {
  long nf = n / 2 + 1;
  if (n % 2 != 0 || !is_pow2(n)) {
    twtab t;
    twtab_init(&t, n);
#pragma omp parallel
    {
      scratch s;
      scratch_init(&s, n);
#pragma omp for schedule(static)
      for (long l = 0; l < lines; l++) {
        for (long k = 0; k < n; k++) {
          double _Complex v;
          if (k < nf)
            v = in[l * nf + k];
          else
            v = conj(in[l * nf + (n - k)]);
          if (k == 0 || (n % 2 == 0 && k == n / 2))
            v = CMPLX(creal(v), 0.0);
          s.xr[k] = creal(v);
          s.xi[k] = cimag(v);
        }
        cfft_batch(&t, +1, s.xr, s.xi, s.yr, s.yi, 1);
        for (long m = 0; m < n; m++)
          out[l * n + m] = s.xr[m];
      }
      scratch_free(&s);
    }
    twtab_free(&t);
    return;
  }
  long M = n / 2;
  twtab t, tn;
  twtab_init(&t, M);
  twtab_init(&tn, n);
  long nb = (lines + BATCH - 1) / BATCH;
#pragma omp parallel
  {
    scratch s;
    scratch_init(&s, M);
#pragma omp for schedule(static)
    for (long job = 0; job < nb; job++) {
      long l0 = job * BATCH;
      int B = (int)((lines - l0) < BATCH ? (lines - l0) : BATCH);
      for (int b = 0; b < B; b++) {
        const double _Complex *x = in + (l0 + b) * nf;
        double x0 = creal(x[0]), xm = creal(x[M]);
        s.xr[b] = x0 + xm;
        s.xi[b] = x0 - xm;
        for (long k = 1; k < M; k++) {
          /* Z[k] = (X[k] + conj X[M-k]) + i W^{-k} (X[k] - conj X[M-k]) */
          double ar = creal(x[k]), ai = cimag(x[k]);
          double br = creal(x[M - k]), bi = -cimag(x[M - k]);
          double er = ar + br, ei = ai + bi;
          double dr = ar - br, di = ai - bi;
          double wr = tn.wr[k], wi = -tn.wi[k]; /* W^{-k} */
          double pr = wr * dr - wi * di, pi = wr * di + wi * dr;
          s.xr[k * B + b] = er - pi;
          s.xi[k * B + b] = ei + pr;
        }
      }
      cfft_batch(&t, +1, s.xr, s.xi, s.yr, s.yi, B);
      for (long m = 0; m < M; m++)
        for (int b = 0; b < B; b++) {
          out[(l0 + b) * n + 2 * m] = s.xr[m * B + b];
          out[(l0 + b) * n + 2 * m + 1] = s.xi[m * B + b];
        }
    }
    scratch_free(&s);
  }
  twtab_free(&t);
  twtab_free(&tn);
}

static void exec_r2c(const struct shim_plan_s *p, const double *in,
                     double _Complex *out) {
  long n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
  long nf = n2 / 2 + 1;
  lastaxis_r2c(in, out, n0 * n1, n2);
  /* axis 1 then axis 0 (complex, forward) */
  axis_cfft(out, n0, n1, nf, -1);
  axis_cfft(out, 1, n0, n1 * nf, -1);
}

static void exec_c2r(const struct shim_plan_s *p, double _Complex *in,
                     double *out) {
  long n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
  long nf = n2 / 2 + 1;
  axis_cfft(in, 1, n0, n1 * nf, +1);
  axis_cfft(in, n0, n1, nf, +1);
  lastaxis_c2r(in, out, n0 * n1, n2);
}

/* ---- FFTW-named API ---- */
static int shim_nthreads = 1;
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) {
  shim_nthreads = nthreads;
#ifdef _OPENMP
  if (nthreads > 0)
    omp_set_num_threads(nthreads);
#endif
}
void fftw_threads_set_callback(
    void (*parallel_loop)(void *(*work)(char *), char *jobdata, size_t elsize,
                          int njobs, void *data),
    void *data) {
  /* The shim parallelises with OpenMP directly, which is the pool main.c's
   * callback forwards to. */
  (void)parallel_loop;
  (void)data;
}
void fftw_cleanup_threads(void) {}
void fftw_cleanup(void) {}

void *fftw_malloc(size_t n) {
  void *p = NULL;
  if (posix_memalign(&p, 64, n ? n : 1) != 0)
    return NULL;
  return p;
}
double *fftw_alloc_real(size_t n) { return fftw_malloc(n * sizeof(double)); }
fftw_complex *fftw_alloc_complex(size_t n) {
  return fftw_malloc(n * sizeof(fftw_complex));
}
void fftw_free(void *p) { free(p); }

static fftw_plan mkplan(int kind, int n0, int n1, int n2) {
  if (n0 <= 0 || n1 <= 0 || n2 <= 0)
    return NULL;
  struct shim_plan_s *p = calloc(1, sizeof *p);
  p->kind = kind;
  p->n[0] = n0;
  p->n[1] = n1;
  p->n[2] = n2;
  return p;
}
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in,
                               fftw_complex *out, unsigned flags) {
  (void)flags;
  fftw_plan p = mkplan(KIND_R2C, n0, n1, n2);
  if (p) {
    p->rin = in;
    p->cout = out;
  }
  return p;
}
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in,
                               double *out, unsigned flags) {
  (void)flags;
  fftw_plan p = mkplan(KIND_C2R, n0, n1, n2);
  if (p) {
    p->cin = in;
    p->rout = out;
  }
  return p;
}
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out,
                               unsigned flags) {
  return fftw_plan_dft_r2c_3d(1, 1, n, in, out, flags);
}
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out,
                               unsigned flags) {
  return fftw_plan_dft_c2r_3d(1, 1, n, in, out, flags);
}
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out) {
  exec_r2c(p, in, out);
}
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out) {
  exec_c2r(p, in, out);
}
void fftw_execute(const fftw_plan p) {
  if (p->kind == KIND_R2C)
    exec_r2c(p, p->rin, p->cout);
  else
    exec_c2r(p, p->cin, p->rout);
}
void fftw_destroy_plan(fftw_plan p) { free(p); }
