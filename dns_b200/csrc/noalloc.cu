// noalloc.cu -- energy/enstrophy of a caller-owned spectral velocity with no
// device allocation at all (dns_diagnostics_noalloc in include/dns_b200.h).
//
// Who needs it: callers that may not call cudaMalloc at the point where they
// want the diagnostics -- code recording work into a CUDA graph with a
// capture mode that forbids allocation, frameworks whose memory pool already
// holds the device memory they are allowed to use, and tight monitoring loops
// that cannot afford the implicit synchronisation an allocation can bring.
// They hand in device pointers for the input and the four output doubles and
// get the same double-double sums as dns_diagnostics.
//
// The reduction needs scratch for its per-block partial sums.  Here that
// scratch is a fixed file-scope device array, NOALLOC_MAX_PARTIALS entries of
// 32 bytes (263 KB), present on every GPU that loads the library until the
// process exits.  Each block reduces a fixed chunk of NOALLOC_CHUNK points,
// so the array bounds the problem size: n^2 (n/2+1) <= NOALLOC_MAX_PARTIALS *
// NOALLOC_CHUNK = 67,371,008 points, which is exactly the n = 512 grid;
// anything larger is rejected before anything is launched.
#include "dns_b200.h"
#include "kernels.cuh"

#include <cuda.h>  // CUcontext / CUresult types only; the driver is reached through the runtime

#include <mutex>
#include <stdio.h>

using namespace dnsb;

namespace dnsb {
void set_last_error(const char *msg);  // dns_api.cu: text for dns_last_error()
}

namespace {

constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_PER_THREAD = 32;
constexpr long long NOALLOC_CHUNK = (long long)NOALLOC_THREADS * NOALLOC_PER_THREAD;  // 8192
constexpr int NOALLOC_MAX_PARTIALS = 8224;  // = ceil(512^2 * 257 / NOALLOC_CHUNK)
static_assert((long long)NOALLOC_MAX_PARTIALS * NOALLOC_CHUNK >= 512LL * 512 * 257,
              "the scratch must hold one partial per block of the n = 512 grid");

// Shared by every call on a device.  Every block of a call writes its own
// entry before the final block reads it, so nothing has to start at zero; two
// calls that overlap on the GPU (different streams, no ordering) race on it.
__device__ __align__(256) double4 g_noalloc_partials[NOALLOC_MAX_PARTIALS];

// Device address of g_noalloc_partials, looked up once per CUDA context and
// cached under the context's unique id (cuCtxGetId).  Keying on the device
// index alone would go wrong after cudaDeviceReset, or under a driver-API
// context other than the device's primary one: the array then lives at a new
// address, and the cached one would point into freed or foreign memory.
// Context ids are never reused within a process.
typedef CUresult (*PfnCtxGetCurrent)(CUcontext *);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long *);
constexpr int ADDR_CACHE = 64;
struct AddrEntry {
  unsigned long long ctx_id;
  double4 *addr;
};
AddrEntry g_addr_cache[ADDR_CACHE] = {};
int g_addr_next = 0;
PfnCtxGetCurrent g_ctx_get_current = nullptr;
PfnCtxGetId g_ctx_get_id = nullptr;
std::mutex g_setup_mutex;

// id of the calling thread's current context (0: none current yet)
cudaError_t current_ctx_id(unsigned long long *id) {
  *id = 0;
  if (!g_ctx_get_current) {
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1);
    if (e == cudaSuccess) e = cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2);
    if (e != cudaSuccess) return e;
    if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
      return cudaErrorNotSupported;
    g_ctx_get_id = (PfnCtxGetId)f2;
    g_ctx_get_current = (PfnCtxGetCurrent)f1;
  }
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS) return cudaErrorUnknown;
  if (ctx && g_ctx_get_id(ctx, id) != CUDA_SUCCESS) return cudaErrorUnknown;
  return cudaSuccess;
}

// the scratch's device address in the current context (set-up on the first
// call in a context: the symbol lookup, which also loads this file's module)
cudaError_t partials_address(double4 **out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  unsigned long long id = 0;
  cudaError_t e = current_ctx_id(&id);
  if (e != cudaSuccess) return e;
  if (id) {
    for (const AddrEntry &a : g_addr_cache)
      if (a.ctx_id == id && a.addr) {
        *out = a.addr;
        return cudaSuccess;
      }
  }
  // host code only holds a stand-in for the array: ask for its device address
  void *p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_partials);
  if (e != cudaSuccess) return e;
  if (!id) {  // the lookup made the device's primary context current
    e = current_ctx_id(&id);
    if (e != cudaSuccess) return e;
  }
  if (id) {
    g_addr_cache[g_addr_next] = AddrEntry{id, (double4 *)p};
    g_addr_next = (g_addr_next + 1) % ADDR_CACHE;
  }
  *out = (double4 *)p;
  return cudaSuccess;
}

// Same terms and double-double arithmetic as k_diag, but each block reduces
// the fixed chunk [blockIdx.x * NOALLOC_CHUNK, +NOALLOC_CHUNK) of points of an
// unpadded [3][n][n][n/2+1] array.
__global__ void __launch_bounds__(NOALLOC_THREADS)
    k_diag_chunk(const cd *__restrict__ u, int n, long long npts, double4 *__restrict__ partial) {
  const int nf = n / 2 + 1;
  DD e{0.0, 0.0}, o{0.0, 0.0};
  const long long base = (long long)blockIdx.x * NOALLOC_CHUNK;
#pragma unroll 4
  for (int i = 0; i < NOALLOC_PER_THREAD; i++) {
    const long long q = base + threadIdx.x + (long long)i * NOALLOC_THREADS;
    if (q < npts) {
      const long long row = q / nf;
      const int k = (int)(q - row * nf);
      const int ii = (int)(row / n), jj = (int)(row % n);
      const double s = __dadd_rn(__dadd_rn(cabs2_rn(u[q]), cabs2_rn(u[npts + q])),
                                 cabs2_rn(u[2 * npts + q]));
      const double kx = kwave(ii, n), ky = kwave(jj, n), kz = k;
      const double kk =
          __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
      e = dd_add_d(e, s);
      o = dd_add_d(o, __dmul_rn(kk, s));
    }
  }
  dd_block_reduce<NOALLOC_THREADS>(e, o, partial + blockIdx.x);
}

int noalloc_fail(int code, const char *msg) {
  dnsb::set_last_error(msg);
  return code;
}

}  // namespace

extern "C" int dns_diagnostics_noalloc(long n, const double *uvw_hat, double *out, void *stream) {
  if (n < 8 || n > 512 || (n & (n - 1)) != 0)
    return noalloc_fail(DNS_ERR_UNSUPPORTED,
                        "dns_diagnostics_noalloc: n must be a power of two in [8, 512]");
  const long long npts = (long long)n * n * (n / 2 + 1);
  const long long nblocks = (npts + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK;
  if (nblocks > NOALLOC_MAX_PARTIALS)
    return noalloc_fail(DNS_ERR_UNSUPPORTED,
                        "dns_diagnostics_noalloc: input larger than the fixed scratch "
                        "(n^2 (n/2+1) must be <= 67371008 points, n <= 512)");
  if (!uvw_hat || !out) return noalloc_fail(DNS_ERR_ARG, "dns_diagnostics_noalloc: NULL pointer");
  double4 *partials = nullptr;
  cudaError_t e = partials_address(&partials);
  if (e != cudaSuccess) return noalloc_fail(DNS_ERR_CUDA, cudaGetErrorString(e));
  // each launch's own status (cudaLaunchKernel), so that an error left
  // pending by the caller's earlier, unrelated work is neither reported as
  // this call's failure nor cleared
  cudaStream_t s = (cudaStream_t)stream;
  const cd *u = (const cd *)uvw_hat;
  int ni = (int)n, nb = (int)nblocks;
  long long np = npts;
  double4 *res = (double4 *)out;
  void *a1[] = {(void *)&u, (void *)&ni, (void *)&np, (void *)&partials};
  e = cudaLaunchKernel((const void *)k_diag_chunk, dim3((unsigned)nblocks), dim3(NOALLOC_THREADS),
                       a1, 0, s);
  if (e != cudaSuccess) return noalloc_fail(DNS_ERR_CUDA, cudaGetErrorString(e));
  void *a2[] = {(void *)&partials, (void *)&nb, (void *)&res};
  e = cudaLaunchKernel((const void *)k_diag_final<NOALLOC_THREADS>, dim3(1), dim3(NOALLOC_THREADS),
                       a2, 0, s);
  if (e != cudaSuccess) return noalloc_fail(DNS_ERR_CUDA, cudaGetErrorString(e));
  return DNS_OK;
}
