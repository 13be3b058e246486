// adjoint.cuh -- pointwise kernels of the discrete adjoint of the RK4 step.
// Templates on the storage complex type C (double2 for the FP64 adjoint,
// float2 for the mixed one); the arithmetic is FP64 in registers, rounded
// once on store.  The forward stage of main.c:344-413 is, per RK stage s with input
// U_s (half spectrum) and, at s == 0, the stale real velocity:
//   u   = s > 0 ? a c2r(U_s) : stale          a = 1/n^3
//   w   = a c2r(D U_s)                        D U = i k x U  (curl)
//   N   = u x w
//   dU  = Pi(m dt r2c(N)) - nu dt kk U_s       Pi(X) = X - k (k.X)/kk
// Its transpose under the real inner product of the stored entries uses
//   c2r^T(y) = w_z * r2c(y),  r2c^T(Y) = c2r(Y / w_z),
//   w_z = 1 on the kz = 0 and kz = n/2 planes, 2 elsewhere,
// (c2r with FFTW's semantics is sum_k w_z Re(X e^{ik.x})); D and Pi are
// self-adjoint; (u x w)^T: lambda_u = w x lambda_N, lambda_w = lambda_N x u.
#pragma once
#include "kernels.cuh"

namespace dnsb {

// the loop over the valid half-spectrum points of one slot set
#define DNSB_FOR_POINTS(g)                                                              \
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x,                 \
                 npts_ = (long long)(g).n * (g).n * (g).nf;                             \
       q < npts_; q += (long long)gridDim.x * blockDim.x)

struct PointK {
  long long o;     // offset in a slot
  double kx, ky, kz, kk;
  int col;
  bool in;         // inside the 2/3 mask
  double wz;       // 1 on kz = 0, n/2; 2 elsewhere
};

__device__ __forceinline__ PointK point_k(const Geo &g, long long q) {
  PointK p;
  const long long row = q / g.nf;
  const int col = (int)(q - row * g.nf);
  const int i = (int)(row / g.n), j = (int)(row - (long long)i * g.n);
  p.o = row * g.nfp + col;
  const int ikx = kwave(i, g.n), iky = kwave(j, g.n);
  p.kx = ikx;
  p.ky = iky;
  p.kz = col;
  p.kk = p.kx * p.kx + p.ky * p.ky + p.kz * p.kz;
  p.col = col;
  p.in = (ikx < 0 ? -ikx : ikx) <= g.kcut && (iky < 0 ? -iky : iky) <= g.kcut && col <= g.kcut;
  p.wz = (col == 0 || col == g.n / 2) ? 1.0 : 2.0;
  return p;
}

// i k x U at one point (main.c:359-361, with kx[n/2] = -n/2)
__device__ __forceinline__ void curl_at(const PointK &p, cd u, cd v, cd w, cd &ox, cd &oy, cd &oz) {
  // i * (a) = (-a.y, a.x)
  const cd ax = make_double2(p.ky * w.x - p.kz * v.x, p.ky * w.y - p.kz * v.y);
  const cd ay = make_double2(p.kz * u.x - p.kx * w.x, p.kz * u.y - p.kx * w.y);
  const cd az = make_double2(p.kx * v.x - p.ky * u.x, p.kx * v.y - p.ky * u.y);
  ox = make_double2(-ax.y, ax.x);
  oy = make_double2(-ay.y, ay.x);
  oz = make_double2(-az.y, az.x);
}

// out = curl(in) on 3 slots
template <class C>
__global__ void k_curl(const C *__restrict__ in, C *__restrict__ out, Geo g) {
  DNSB_FOR_POINTS(g) {
    const PointK p = point_k(g, q);
    cd ox, oy, oz;
    curl_at(p, to_d(in[p.o]), to_d(in[g.slot + p.o]), to_d(in[2 * g.slot + p.o]), ox, oy, oz);
    out[p.o] = from_d<C>(ox);
    out[g.slot + p.o] = from_d<C>(oy);
    out[2 * g.slot + p.o] = from_d<C>(oz);
  }
}

// out = (m dt Pi(ldU)) / w_z : the adjoint of N_hat, divided by the c2r
// weights so that a plain c2r of `out` is r2c^T of m dt Pi(ldU)
template <class C>
__global__ void k_adj_lamN(const C *__restrict__ ldU, C *__restrict__ out, Geo g, double dt) {
  DNSB_FOR_POINTS(g) {
    const PointK p = point_k(g, q);
    cd x = to_d(ldU[p.o]), y = to_d(ldU[g.slot + p.o]), z = to_d(ldU[2 * g.slot + p.o]);
    if (p.kk > 0) {
      const double sr = (x.x * p.kx + y.x * p.ky + z.x * p.kz) / p.kk;
      const double si = (x.y * p.kx + y.y * p.ky + z.y * p.kz) / p.kk;
      x = make_double2(x.x - sr * p.kx, x.y - si * p.kx);
      y = make_double2(y.x - sr * p.ky, y.y - si * p.ky);
      z = make_double2(z.x - sr * p.kz, z.y - si * p.kz);
    }
    const double s = (p.in ? dt : 0.0) / p.wz;
    out[p.o] = from_d<C>(cscale(x, s));
    out[g.slot + p.o] = from_d<C>(cscale(y, s));
    out[2 * g.slot + p.o] = from_d<C>(cscale(z, s));
  }
}

// lu = om x lN (+ lstale_out), lom = lN x u   on [3][n^3] real arrays (u,
// om and the outputs in the precision they are kept in, the rest float64)
template <class RU, class RW, class RO>
__global__ void k_adj_cross(const RU *__restrict__ u, const RW *__restrict__ om,
                            const double *__restrict__ lN, const double *__restrict__ lstale_out,
                            RO *__restrict__ lu, RO *__restrict__ lom, long long nr) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nr;
       q += (long long)gridDim.x * blockDim.x) {
    const double ux = u[q], uy = u[nr + q], uz = u[2 * nr + q];
    const double wx = om[q], wy = om[nr + q], wz = om[2 * nr + q];
    const double lx = lN[q], ly = lN[nr + q], lz = lN[2 * nr + q];
    double ax = wy * lz - wz * ly, ay = wz * lx - wx * lz, az = wx * ly - wy * lx;
    if (lstale_out) {
      ax += lstale_out[q];
      ay += lstale_out[nr + q];
      az += lstale_out[2 * nr + q];
    }
    lu[q] = (RO)ax;
    lu[nr + q] = (RO)ay;
    lu[2 * nr + q] = (RO)az;
    lom[q] = (RO)(ly * uz - lz * uy);
    lom[nr + q] = (RO)(lz * ux - lx * uz);
    lom[2 * nr + q] = (RO)(lx * uy - ly * ux);
  }
}

// lUs = a w_z (curl(Rw) + Ru) - nu dt kk ldU       (Ru may be null: stage 0),
// the adjoint of the stage input U_s = U0 + b dU_{s-1}, consumed at once:
//   lhat_out = lhat_in + lUs                (lambda of U0, accumulated)
//   ldU      = bn lUs + an lacc             (lambda of dU_{s-1}; not at stage 0)
// with ldU overwritten in place; and the nu-gradient terms <ldU, -dt kk Us>,
// double-double block partials
template <int BS, class C>
__global__ void __launch_bounds__(BS)
    k_adj_collect(const C *__restrict__ Rw, const C *__restrict__ Ru, C *ldU,
                  const C *__restrict__ Us, const C *lhat_in, C *lhat_out,
                  const C *__restrict__ lacc, Geo g, double a, double nu, double dt, double bn,
                  double an, bool next, double4 *__restrict__ partial) {
  DD gn{0.0, 0.0}, unused{0.0, 0.0};
  DNSB_FOR_POINTS(g) {
    const PointK p = point_k(g, q);
    cd cxyz[3];
    curl_at(p, to_d(Rw[p.o]), to_d(Rw[g.slot + p.o]), to_d(Rw[2 * g.slot + p.o]), cxyz[0],
            cxyz[1], cxyz[2]);
    const double s = a * p.wz, c = nu * dt * p.kk;
    double dotp = 0.0;
#pragma unroll
    for (int f = 0; f < 3; f++) {
      const long long o = f * g.slot + p.o;
      cd cf = cxyz[f];
      if (Ru) cf = cadd(cf, to_d(Ru[o]));
      const cd l = to_d(ldU[o]), u = to_d(Us[o]);
      dotp += l.x * u.x;
      dotp += l.y * u.y;
      const cd lus = make_double2(s * cf.x - c * l.x, s * cf.y - c * l.y);
      lhat_out[o] = from_d<C>(cadd(to_d(lhat_in[o]), lus));
      if (next) ldU[o] = from_d<C>(cadd(cscale(lus, bn), cscale(to_d(lacc[o]), an)));
    }
    gn = dd_add_d(gn, -dt * p.kk * dotp);
  }
  dd_block_reduce<BS>(gn, unused, partial + blockIdx.x);
}

// acc (device double-double, .x .y) += sum of np block partials (.x .y)
template <int BS>
__global__ void __launch_bounds__(BS) k_dd_accumulate(const double4 *__restrict__ partial, int np,
                                                      double4 *__restrict__ acc) {
  DD e{0.0, 0.0}, unused{0.0, 0.0};
  for (int q = threadIdx.x; q < np; q += BS) e = dd_add(e, DD{partial[q].x, partial[q].y});
  __shared__ double4 tot;
  dd_block_reduce<BS>(e, unused, &tot);
  __syncthreads();
  if (threadIdx.x == 0) {
    const DD s = dd_add(DD{acc->x, acc->y}, DD{tot.x, tot.y});
    acc->x = s.hi;
    acc->y = s.lo;
  }
}

// out = a x + b y on 3 slots (y may be null)
template <class C>
__global__ void k_lincomb3(const C *__restrict__ x, const C *__restrict__ y, C *__restrict__ out,
                           Geo g, double a, double b) {
  DNSB_FOR_POINTS(g) {
    const long long row = q / g.nf;
    const long long o = row * g.nfp + (q - row * g.nf);
#pragma unroll
    for (int f = 0; f < 3; f++) {
      const cd xv = to_d(x[f * g.slot + o]);
      cd r = cscale(xv, a);
      if (y) r = cadd(r, cscale(to_d(y[f * g.slot + o]), b));
      out[f * g.slot + o] = from_d<C>(r);
    }
  }
}

// out = x / w_z on 3 slots (r2c^T = c2r of this)
template <class C>
__global__ void k_div_wz3(const C *__restrict__ x, C *__restrict__ out, Geo g) {
  DNSB_FOR_POINTS(g) {
    const PointK p = point_k(g, q);
#pragma unroll
    for (int f = 0; f < 3; f++)
      out[f * g.slot + p.o] = from_d<C>(cscale(to_d(x[f * g.slot + p.o]), 1.0 / p.wz));
  }
}

// y += x on n real values
__global__ void k_add_real(const double *__restrict__ x, double *__restrict__ y, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    y[q] += x[q];
}

}  // namespace dnsb
