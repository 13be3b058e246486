/*
 * dns -- command-line drop-in for slitvinov/dns main.c, stepping on the GPU
 * through the C ABI of libdns_b200 (include/dns_b200.h).
 *
 * Same surface as the reference:
 *   usage text, flags and error messages        main.c:58-150
 *   n from the file size, exact size check       main.c:163-171
 *   reading U, V, W (P ignored)                  main.c:180-185
 *   "% 10ld % .16e % .16Le % .16Le" every 10 steps, flushed   main.c:257-268
 *   -d: %08ld.raw with U, V, W, P and a.%08ld.xdmf2           main.c:269-330
 *   the loop: print, `t > T` test, step, t += dt              main.c:256-423
 * The -v lines report the CUDA device instead of the OpenMP thread count.
 * A NaN/Inf in the diagnostics ends the run with an error message and exit
 * status 1 (the reference dies on SIGFPE, main.c:49-50).
 *
 * The environment variable DNS_B200_PRECISION selects the arithmetic
 * without touching the reference's flags: "fp64" (default, the reference's)
 * or "mixed" (float32 fields and FFTs, float64 reductions).
 */
#define _GNU_SOURCE
#include <fenv.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dns_b200.h"

enum { nvars = 4 };
static const double pi = 3.141592653589793238;

static void usage(void) {
  fprintf(stderr, "Usage: dns [-v] [-d] -i <input.raw> -n <viscosity> -t "
                  "<end time> -s <time step>\n"
                  "\n"
                  "Options:\n"
                  "  -i <input.raw>    Input file\n"
                  "  -n <viscosity>    Viscosity\n"
                  "  -t <end time>     End time\n"
                  "  -s <time step>    Time step\n"
                  "  -v                Verbose output\n"
                  "  -d                Dump snapshots\n"
                  "  -h                Show this help message\n"
                  "\n"
                  "Example:\n"
                  "  dns -i tgv.raw -n 0.01 -t 1.0 -s 0.001 -v\n");
  fprintf(stderr, "\nBuild Info:\n"
                  "  CUDA (sm_100a) is enabled.\n");
}

static void die(const char *msg) {
  fprintf(stderr, "dns: error: %s\n", msg);
  exit(1);
}

static void die_status(const char *what, int st) {
  fprintf(stderr, "dns: error: %s: %s: %s\n", what, dns_strerror(st), dns_last_error());
  exit(1);
}

/* value of a numeric flag, with main.c's full-consumption check */
static double number(char *s) {
  char *end;
  double x = strtod(s, &end);
  if (*end != '\0') {
    fprintf(stderr, "dns: error: '%s' is not a number\n", s);
    exit(1);
  }
  return x;
}

static void write_dump(dns_ctx *ctx, long n, long tstep, long idump, double t,
                       double *buf) {
  char path[FILENAME_MAX];
  long n3 = n * n * n;
  double dx = 2 * pi / n;
  int st = dns_get_fields(ctx, buf, buf + n3, buf + 2 * n3, buf + 3 * n3);
  if (st != DNS_OK)
    die_status("dump", st);
  sprintf(path, "%08ld.raw", tstep);
  FILE *f = fopen(path, "w");
  if (f == NULL) {
    fprintf(stderr, "dns: error: fail to open '%s'\n", path);
    exit(1);
  }
  fwrite(buf, sizeof(double), (size_t)(nvars * n3), f);
  fclose(f);
  sprintf(path, "a.%08ld.xdmf2", idump);
  f = fopen(path, "w");
  if (f == NULL) {
    fprintf(stderr, "dns: error: fail to open '%s'\n", path);
    exit(1);
  }
  fprintf(f,
          "<Xdmf\n"
          "    Version=\"2\">\n"
          "  <Domain>\n"
          "    <Grid>\n"
          "      <Time\n"
          "          Value=\"%+.16e\"/>\n"
          "      <Topology\n"
          "          TopologyType=\"3DCoRectMesh\"\n"
          "          Dimensions=\"%ld %ld %ld\"/>\n"
          "      <Geometry\n"
          "          GeometryType=\"ORIGIn_DXDYDZ\">\n"
          "        <DataItem\n"
          "            Dimensions=\"3\">\n"
          "          0\n"
          "          0\n"
          "          0\n"
          "        </DataItem>\n"
          "        <DataItem\n"
          "            Dimensions=\"3\">\n"
          "          %.16e\n"
          "          %.16e\n"
          "          %.16e\n"
          "        </DataItem>\n"
          "      </Geometry>\n",
          t, n, n, n, dx, dx, dx);
  static const char *names[nvars] = {"U", "V", "W", "P"};
  long seek = 0;
  for (int v = 0; v < nvars; v++) {
    /* the data file is named by idump here, as in main.c:319-322 */
    fprintf(f,
            "      <Attribute\n"
            "          name=\"%s\">\n"
            "        <DataItem\n"
            "            Format=\"Binary\"\n"
            "            Seek=\"%ld\"\n"
            "            Precision=\"8\"\n"
            "            Dimensions=\"%ld %ld %ld\">\n"
            "          %08ld.raw\n"
            "        </DataItem>\n"
            "      </Attribute>\n",
            names[v], seek, n, n, n, idump);
    seek += n3 * (long)sizeof(double);
  }
  fprintf(f, "    </Grid>\n"
             "  </Domain>\n"
             "</Xdmf>\n");
  fclose(f);
}

int main(int argc, char **argv) {
  (void)argc;
  char *input_path = NULL;
  double dt = -1, T = 0, nu = -1;
  int verbose = 0, dump = 0;
  FILE *file;

  feclearexcept(FE_ALL_EXCEPT);
  feenableexcept(FE_DIVBYZERO | FE_INVALID | FE_OVERFLOW);

  while (*++argv != NULL && argv[0][0] == '-') {
    switch (argv[0][1]) {
    case 'h':
      usage();
      exit(1);
    case 'v':
      verbose = 1;
      break;
    case 'd':
      dump = 1;
      break;
    case 'i':
      if (*++argv == NULL)
        die("-i needs an argument");
      input_path = *argv;
      break;
    case 'n':
      if (*++argv == NULL)
        die("-n needs an argument");
      nu = number(*argv);
      break;
    case 's':
      if (*++argv == NULL)
        die("-s needs an argument");
      dt = number(*argv);
      break;
    case 't':
      if (*++argv == NULL)
        die("-t needs an argument");
      T = number(*argv);
      break;
    default:
      fprintf(stderr, "dns: error: unknown option '%s'\n", *argv);
      exit(1);
    }
  }
  if (T == 0)
    die("-t is not set or invalid");
  if (nu == -1)
    die("-n is not set or invalid");
  if (dt == -1)
    die("-s is not set or invalid");
  if (input_path == NULL)
    die("-i is not set");
  if ((file = fopen(input_path, "r")) == NULL) {
    fprintf(stderr, "dns: error: fail to open '%s'\n", input_path);
    exit(1);
  }

  /* n from the file size: main.c:163-171 (cube root in float, then rounded) */
  fseek(file, 0, SEEK_END);
  size_t offset = (size_t)ftell(file);
  rewind(file);
  long n = (long)(offset / sizeof(double) / nvars);
  n = lround(powf((float)n, 1.0f / 3));
  if ((size_t)(n * n * n * nvars) * sizeof(double) != offset) {
    fprintf(stderr, "dns: error: wrong file '%s'\n", input_path);
    exit(1);
  }

  int prec = DNS_PREC_FP64;
  const char *penv = getenv("DNS_B200_PRECISION");
  if (penv != NULL && *penv != '\0') {
    if (strcmp(penv, "mixed") == 0)
      prec = DNS_PREC_MIXED;
    else if (strcmp(penv, "fp64") != 0) {
      fprintf(stderr, "dns: error: DNS_B200_PRECISION='%s' is not fp64 or mixed\n", penv);
      exit(1);
    }
  }
  dns_ctx *ctx;
  int st = dns_create(n, prec, dump ? DNS_FLAG_PRESSURE : 0u, &ctx);
  if (st != DNS_OK)
    die_status("dns_create", st);
  if (verbose) {
    fprintf(stderr, "dns: device: CUDA sm_100a\n");
    fprintf(stderr, "dns: n = %ld\n", n);
  }
  long n3 = n * n * n;
  double *buf = malloc(sizeof(double) * (size_t)n3 * (dump ? nvars : 3));
  if (buf == NULL)
    die("out of host memory");
  if (fread(buf, sizeof(double), n3, file) != (size_t)n3 ||
      fread(buf + n3, sizeof(double), n3, file) != (size_t)n3 ||
      fread(buf + 2 * n3, sizeof(double), n3, file) != (size_t)n3 ||
      fclose(file) != 0) {
    fprintf(stderr, "dns: error: fail to read '%s'\n", input_path);
    exit(1);
  }
  st = dns_set_velocity(ctx, buf, buf + n3, buf + 2 * n3);
  if (st != DNS_OK)
    die_status("dns_set_velocity", st);

  double invn3 = 1.0 / n3;
  double t = 0.0;
  long tstep = 0, idump = 0;
  for (;;) {
    if (tstep % 10 == 0) {
      double eh, el, oh, ol;
      st = dns_diagnostics(ctx, &eh, &el, &oh, &ol);
      if (st == DNS_ERR_NONFINITE)
        die("non-finite energy or enstrophy (the flow diverged)");
      if (st != DNS_OK)
        die_status("dns_diagnostics", st);
      /* main.c:265-266: long double sums scaled by invn3 * invn3 */
      long double energy = (long double)eh + (long double)el;
      long double Omega = (long double)oh + (long double)ol;
      energy *= invn3 * invn3;
      Omega *= invn3 * invn3;
      printf("% 10ld % .16e % .16Le % .16Le\n", tstep, t, energy, Omega);
      fflush(stdout);
      if (dump) {
        write_dump(ctx, n, tstep, idump, t, buf);
        idump++;
      }
    }
    if (t > T)
      break;
    /* run up to the next print (or the end) in one call: the same t
     * accumulation as the reference decides where the loop stops */
    long k = 0;
    double tt = t;
    do {
      tt += dt;
      k++;
    } while ((tstep + k) % 10 != 0 && !(tt > T));
    st = dns_step(ctx, nu, dt, k);
    if (st != DNS_OK)
      die_status("dns_step", st);
    t = tt;
    tstep += k;
  }
  /* Opt-in kernel timings (no counterpart in the reference):
   * DNS_B200_TIMINGS=<k> times k more steps launch by launch after the run
   * (the printed history is complete before) and prints each kernel's mean
   * time to stderr. */
  const char *tenv = getenv("DNS_B200_TIMINGS");
  if (tenv && atol(tenv) > 0) {
    static const char *pass[6] = {"A x-inverse", "B y-inverse", "C z-fused",
                                  "D y-forward", "E1 x-forward", "E2 update"};
    dns_info_t info;
    st = dns_get_info(ctx, &info);
    if (st != DNS_OK)
      die_status("dns_get_info", st);
    double *ms = malloc(sizeof(double) * (size_t)info.kernels_per_step);
    if (!ms)
      die("out of host memory");
    st = dns_time_kernels(ctx, nu, dt, atol(tenv), ms);
    if (st != DNS_OK)
      die_status("dns_time_kernels", st);
    double sum = 0.0;
    for (int q = 0; q < info.kernels_per_step; q++) {
      fprintf(stderr, "dns: stage %d %s: %.4f ms\n", q / 6, pass[q % 6], ms[q]);
      sum += ms[q];
    }
    fprintf(stderr, "dns: step (sum of its kernels): %.4f ms over %ld steps\n", sum, atol(tenv));
    free(ms);
  }
  free(buf);
  dns_destroy(ctx);
  return 0;
}
