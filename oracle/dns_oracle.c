/*
 * dns_oracle.c -- CPU restatement of the pseudo-spectral RK4 step of
 * slitvinov/dns main.c, as a small C library.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * product (dns_b200/csrc).  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py load it.  The product never links or calls it.
 *
 * It follows main.c step by step (citations are to main.c of the reference):
 *   - state and wavenumbers: main.c:174-247  (kx, kz, kmax, dealias, kk)
 *   - initial forward transform: main.c:249-251
 *   - diagnostics: main.c:257-266 (long double accumulators over the half
 *     spectrum, no Hermitian weighting, scaled by invn3*invn3)
 *   - time step: main.c:334-422, including the "stale velocity" behaviour:
 *     stage rk == 0 does not transform U_hat back to real space
 *     (main.c:344), so it uses the real-space velocity left over from stage
 *     rk == 3 of the previous step (or the raw input at step 0).
 *   - dump fields: main.c:270-279 (c2r(X_hat) * invn3 for U, V, W, P).
 * The FFTs are the project-written shim (fftw_shim/), which follows FFTW3's
 * conventions.  Compiled as C99 without FMA contraction, like `c99` builds
 * of main.c.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "fftw3.h"

typedef double _Complex cplx;

static const double rk_a[4] = {1 / 6.0, 1 / 3.0, 1 / 3.0, 1 / 6.0}; /* main.c:15 */
static const double rk_b[3] = {0.5, 0.5, 1.0};                       /* main.c:16 */

typedef struct dns_oracle {
  long n, nf, n3, n3f;
  double invn3;
  double *kx, *kz, *kk;
  int *mask;
  /* spectral state and work (names follow main.c:41-48) */
  cplx *uh[3], *uh0[3], *uh1[3], *du[3], *curl[3], *ph, *work;
  /* real fields: velocity (stale between steps), vorticity, product */
  double *u[3], *om[3], *nl[3];
  fftw_plan fplan, bplan;
} dns_oracle;

static double sq(cplx z) { return creal(z) * creal(z) + cimag(z) * cimag(z); }

dns_oracle *oracle_create(long n) {
  if (n < 2)
    return NULL;
  dns_oracle *o = calloc(1, sizeof *o);
  o->n = n;
  o->nf = n / 2 + 1;
  o->n3 = n * n * n;
  o->n3f = n * n * o->nf;
  o->invn3 = 1.0 / o->n3;
  for (int c = 0; c < 3; c++) {
    o->uh[c] = fftw_alloc_complex(o->n3f);
    o->uh0[c] = fftw_alloc_complex(o->n3f);
    o->uh1[c] = fftw_alloc_complex(o->n3f);
    o->du[c] = fftw_alloc_complex(o->n3f);
    o->curl[c] = fftw_alloc_complex(o->n3f);
    o->u[c] = fftw_alloc_real(o->n3);
    o->om[c] = fftw_alloc_real(o->n3);
    o->nl[c] = fftw_alloc_real(o->n3);
    memset(o->uh[c], 0, sizeof(cplx) * o->n3f);
    memset(o->u[c], 0, sizeof(double) * o->n3);
  }
  o->ph = fftw_alloc_complex(o->n3f);
  memset(o->ph, 0, sizeof(cplx) * o->n3f);
  o->work = fftw_alloc_complex(o->n3f);
  o->kx = malloc(sizeof(double) * n);
  o->kz = malloc(sizeof(double) * o->nf);
  o->kk = malloc(sizeof(double) * o->n3f);
  o->mask = malloc(sizeof(int) * o->n3f);
  o->fplan = fftw_plan_dft_r2c_3d(n, n, n, o->u[0], o->uh[0],
                                  FFTW_ESTIMATE | FFTW_PRESERVE_INPUT);
  o->bplan = fftw_plan_dft_c2r_3d(n, n, n, o->uh[0], o->u[0], FFTW_ESTIMATE);
  /* wavenumbers: main.c:224-230.  kx[n/2] = -n/2, kz[n/2] = +n/2 */
  for (long i = 0; i < n; i++)
    o->kx[i] = (i < n / 2) ? (double)i : (double)(i - n);
  for (long k = 0; k < o->nf; k++)
    o->kz[k] = (double)k;
  /* 2/3 rule mask and |k|^2: main.c:231-247 */
  double kmax = 2. / 3. * (n / 2 + 1);
  long nn = n, nf = o->nf;
#pragma omp parallel for collapse(3)
  for (long i = 0; i < nn; i++)
    for (long j = 0; j < nn; j++)
      for (long k = 0; k < nf; k++) {
        long l = (i * nn + j) * nf + k;
        o->mask[l] = (fabs(o->kx[i]) < kmax) && (fabs(o->kx[j]) < kmax) &&
                     (fabs(o->kz[k]) < kmax);
        o->kk[l] = o->kx[i] * o->kx[i] + o->kx[j] * o->kx[j] +
                   o->kz[k] * o->kz[k];
      }
  return o;
}

void oracle_destroy(dns_oracle *o) {
  if (!o)
    return;
  for (int c = 0; c < 3; c++) {
    fftw_free(o->uh[c]);
    fftw_free(o->uh0[c]);
    fftw_free(o->uh1[c]);
    fftw_free(o->du[c]);
    fftw_free(o->curl[c]);
    fftw_free(o->u[c]);
    fftw_free(o->om[c]);
    fftw_free(o->nl[c]);
  }
  fftw_free(o->ph);
  fftw_free(o->work);
  free(o->kx);
  free(o->kz);
  free(o->kk);
  free(o->mask);
  fftw_destroy_plan(o->fplan);
  fftw_destroy_plan(o->bplan);
  free(o);
}

long oracle_n(const dns_oracle *o) { return o->n; }

/* main.c:180-185 reads U, V, W from the file; main.c:249-251 transforms
 * them.  The real arrays keep the raw input: it is the stale velocity of the
 * first stage of step 0. */
void oracle_set_velocity(dns_oracle *o, const double *U, const double *V,
                         const double *W) {
  const double *src[3] = {U, V, W};
  for (int c = 0; c < 3; c++) {
    memcpy(o->u[c], src[c], sizeof(double) * o->n3);
    fftw_execute_dft_r2c(o->fplan, o->u[c], o->uh[c]);
  }
}

/* main.c:257-266 */
void oracle_diagnostics(const dns_oracle *o, long double *E, long double *Om) {
  long double e = 0.0, w = 0.0;
  long n3f = o->n3f;
  const cplx *U = o->uh[0], *V = o->uh[1], *W = o->uh[2];
  const double *kk = o->kk;
#pragma omp parallel for reduction(+ : e, w)
  for (long k = 0; k < n3f; k++) {
    e += sq(U[k]) + sq(V[k]) + sq(W[k]);
    w += kk[k] * (sq(U[k]) + sq(V[k]) + sq(W[k]));
  }
  e *= o->invn3 * o->invn3;
  w *= o->invn3 * o->invn3;
  *E = e;
  *Om = w;
}

/* c2r of a spectral field into a real one, scaled by 1/n^3; the spectral
 * input is preserved (main.c:23-30 copies into a work array first) */
static void to_real(dns_oracle *o, const cplx *hat, double *real) {
  long n3f = o->n3f, n3 = o->n3;
  cplx *wk = o->work;
#pragma omp parallel for
  for (long k = 0; k < n3f; k++)
    wk[k] = hat[k];
  fftw_execute_dft_c2r(o->bplan, wk, real);
  double s = o->invn3;
#pragma omp parallel for
  for (long k = 0; k < n3; k++)
    real[k] *= s;
}

/* one right-hand-side evaluation: dU = RK increment of stage rk
 * (main.c:344-399) */
static void rhs(dns_oracle *o, int rk, double nu, double dt) {
  long n = o->n, nf = o->nf, n3 = o->n3, n3f = o->n3f;
  const double *kx = o->kx, *kz = o->kz, *kk = o->kk;
  cplx *U = o->uh[0], *V = o->uh[1], *W = o->uh[2];
  if (rk > 0) /* main.c:344-353; skipped at rk == 0 (stale velocity) */
    for (int c = 0; c < 3; c++)
      to_real(o, o->uh[c], o->u[c]);
  /* vorticity in spectral space: main.c:354-362 */
  cplx *cx = o->curl[0], *cy = o->curl[1], *cz = o->curl[2];
#pragma omp parallel for collapse(3)
  for (long i = 0; i < n; i++)
    for (long j = 0; j < n; j++)
      for (long k = 0; k < nf; k++) {
        long l = (i * n + j) * nf + k;
        cz[l] = I * (kx[i] * V[l] - kx[j] * U[l]);
        cy[l] = I * (kz[k] * U[l] - kx[i] * W[l]);
        cx[l] = I * (kx[j] * W[l] - kz[k] * V[l]);
      }
  /* vorticity to real space (input destroyed): main.c:363-371 */
  for (int c = 0; c < 3; c++)
    fftw_execute_dft_c2r(o->bplan, o->curl[c], o->om[c]);
  double s = o->invn3;
  double *ox = o->om[0], *oy = o->om[1], *oz = o->om[2];
#pragma omp parallel for
  for (long k = 0; k < n3; k++) {
    ox[k] *= s;
    oy[k] *= s;
    oz[k] *= s;
  }
  /* u x omega: main.c:372-377 */
  const double *u = o->u[0], *v = o->u[1], *w = o->u[2];
  double *nx = o->nl[0], *ny = o->nl[1], *nz = o->nl[2];
#pragma omp parallel for
  for (long k = 0; k < n3; k++) {
    nx[k] = v[k] * oz[k] - w[k] * oy[k];
    ny[k] = w[k] * ox[k] - u[k] * oz[k];
    nz[k] = u[k] * oy[k] - v[k] * ox[k];
  }
  /* forward transform: main.c:378-380 */
  for (int c = 0; c < 3; c++)
    fftw_execute_dft_r2c(o->fplan, o->nl[c], o->du[c]);
  /* dealias * dt: main.c:381-386 */
  cplx *dU = o->du[0], *dV = o->du[1], *dW = o->du[2];
  const int *mask = o->mask;
#pragma omp parallel for
  for (long k = 0; k < n3f; k++) {
    dU[k] *= mask[k] * dt;
    dV[k] *= mask[k] * dt;
    dW[k] *= mask[k] * dt;
  }
  /* projection and viscous term: main.c:387-399 */
  cplx *P = o->ph;
#pragma omp parallel for collapse(3)
  for (long i = 0; i < n; i++)
    for (long j = 0; j < n; j++)
      for (long k = 0; k < nf; k++) {
        long l = (i * n + j) * nf + k;
        P[l] = kk[l] > 0
                   ? (dU[l] * kx[i] + dV[l] * kx[j] + dW[l] * kz[k]) / kk[l]
                   : 0.0;
        dU[l] -= P[l] * kx[i] + nu * dt * kk[l] * U[l];
        dV[l] -= P[l] * kx[j] + nu * dt * kk[l] * V[l];
        dW[l] -= P[l] * kz[k] + nu * dt * kk[l] * W[l];
      }
}

/* nsteps RK4 steps: main.c:334-422 (time and step counters are the
 * caller's, as the caller also decides when to print) */
void oracle_step(dns_oracle *o, double nu, double dt, long nsteps) {
  long n3f = o->n3f;
  for (long s = 0; s < nsteps; s++) {
    for (int c = 0; c < 3; c++) { /* main.c:334-342 */
      cplx *x = o->uh[c], *x0 = o->uh0[c], *x1 = o->uh1[c];
#pragma omp parallel for
      for (long k = 0; k < n3f; k++) {
        x0[k] = x[k];
        x1[k] = x[k];
      }
    }
    for (int rk = 0; rk < 4; rk++) {
      rhs(o, rk, nu, dt);
      for (int c = 0; c < 3; c++) {
        cplx *x = o->uh[c], *x0 = o->uh0[c], *x1 = o->uh1[c], *d = o->du[c];
        if (rk < 3) { /* main.c:400-407 */
          double bb = rk_b[rk];
#pragma omp parallel for
          for (long k = 0; k < n3f; k++)
            x[k] = x0[k] + bb * d[k];
        }
        double aa = rk_a[rk]; /* main.c:408-413 */
#pragma omp parallel for
        for (long k = 0; k < n3f; k++)
          x1[k] += aa * d[k];
      }
    }
    for (int c = 0; c < 3; c++) /* main.c:415-420 */
      memcpy(o->uh[c], o->uh1[c], sizeof(cplx) * n3f);
  }
}

/* ---- accessors used by the parity tests ---- */

/* spectral velocity, [3][n][n][nf] complex (re, im interleaved) */
void oracle_get_spectral(const dns_oracle *o, double *out) {
  for (int c = 0; c < 3; c++)
    memcpy(out + 2 * c * o->n3f, o->uh[c], sizeof(cplx) * o->n3f);
}
void oracle_set_spectral(dns_oracle *o, const double *in) {
  for (int c = 0; c < 3; c++)
    memcpy(o->uh[c], in + 2 * c * o->n3f, sizeof(cplx) * o->n3f);
}
/* real velocity arrays U, V, W: the stale velocity carried between steps */
void oracle_get_stale(const dns_oracle *o, double *out) {
  for (int c = 0; c < 3; c++)
    memcpy(out + c * o->n3, o->u[c], sizeof(double) * o->n3);
}
void oracle_set_stale(dns_oracle *o, const double *in) {
  for (int c = 0; c < 3; c++)
    memcpy(o->u[c], in + c * o->n3, sizeof(double) * o->n3);
}
/* P_hat of the last evaluated stage, [n][n][nf] complex */
void oracle_get_pressure(const dns_oracle *o, double *out) {
  memcpy(out, o->ph, sizeof(cplx) * o->n3f);
}
/* the four dump fields (main.c:270-279): c2r(X_hat) * invn3 for
 * X = U, V, W, P, written [4][n][n][n] */
void oracle_dump_fields(dns_oracle *o, double *out) {
  cplx *src[4] = {o->uh[0], o->uh[1], o->uh[2], o->ph};
  double *tmp = fftw_alloc_real(o->n3);
  for (int c = 0; c < 4; c++) {
    to_real(o, src[c], tmp);
    memcpy(out + c * o->n3, tmp, sizeof(double) * o->n3);
  }
  fftw_free(tmp);
}

/* plain FFT helpers for the FFT known-answer tests */
void oracle_r2c_3d(int n0, int n1, int n2, const double *in, double *out) {
  long nr = (long)n0 * n1 * n2;
  double *tmp = fftw_alloc_real(nr);
  memcpy(tmp, in, sizeof(double) * nr);
  fftw_plan p = fftw_plan_dft_r2c_3d(n0, n1, n2, tmp, (cplx *)out,
                                     FFTW_ESTIMATE | FFTW_PRESERVE_INPUT);
  fftw_execute_dft_r2c(p, tmp, (cplx *)out);
  fftw_destroy_plan(p);
  fftw_free(tmp);
}
void oracle_c2r_3d(int n0, int n1, int n2, const double *in, double *out) {
  long nc = (long)n0 * n1 * (n2 / 2 + 1);
  cplx *tmp = fftw_alloc_complex(nc);
  memcpy(tmp, in, sizeof(cplx) * nc);
  fftw_plan p = fftw_plan_dft_c2r_3d(n0, n1, n2, tmp, out, FFTW_ESTIMATE);
  fftw_execute_dft_c2r(p, tmp, out);
  fftw_destroy_plan(p);
  fftw_free(tmp);
}
int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0)
    omp_set_num_threads(n);
#else
  (void)n;
#endif
}
