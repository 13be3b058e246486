// persistent.cuh -- one cooperative kernel launch per RK4 step of a whole
// ensemble (dns_ens in its persistent schedule).
//
// The batched schedule steps an ensemble with 24 launches per size group
// (four RK stages of six passes), size groups as concurrent branches of a
// CUDA graph.  Here a single cooperative launch, of as many blocks as fit
// on the GPU at once, walks the same 24 phases for every run of every size:
// in each phase the work items of all groups (the blocks the standalone
// kernels would launch: column tiles, z line groups, update chunks) are
// pooled and dealt out to the blocks, which run the same pass bodies as the
// standalone kernels (kernels.cuh), so each run's state is bit-identical to
// the batched schedule's.  Phases are separated by a grid-wide barrier.
//
// A work item of fewer threads than the block (tpi < PBS) shares the block
// with PBS / tpi others, each synchronising on its own hardware barrier
// (NamedSync, ids 1..).  The grid barrier is a sense-reversing counter in
// device memory; its wait is bounded in time (%globaltimer): past the limit
// the block records PERR_BARRIER_TIMEOUT in the error word and the kernel
// ends, the host reports it at its next check and refuses further steps.
// Co-residency of all blocks, which the barrier needs, is what a
// cooperative launch guarantees (or the launch fails).
#pragma once
#include "kernels.cuh"

namespace dnsb {

constexpr int PBS = 128;        // threads per block
constexpr int PMAXG = 4;        // size groups
constexpr int PPHASES = 24;     // 4 RK stages x 6 passes
enum : unsigned { PERR_BARRIER_TIMEOUT = 1u };
enum { PK_COL = 0, PK_Z = 1, PK_UPD = 2 };

// register cap: FP64's z pass needs 255 registers (2 blocks of 128
// threads), FP32's 170 (3 blocks)
template <class R>
struct PMinB {
  static constexpr int value = sizeof(R) == 8 ? 2 : 3;
};

template <class R>
struct PPhase {
  int kind;          // PK_*
  int axis, fwd;     // column pass
  int sub;           // z-pass KIND or update stage
  int gx, gy, gz;    // work items: the grid of the standalone launch
  int tpi;           // threads per item
  int smem;          // shared bytes per item
  ColJobs jobs;
  StageArgs<R> sa;
};

template <class R>
struct PGroup {
  int n;
  Geo g;
  cx<R> *S;          // spectral slots of the group's run 0
  cx<R> *work;       // its work slots
  R *stale;
  const cx<R> *tw;
  R invn3;
  PPhase<R> ph[PPHASES];
};

template <class R>
struct PPlan {
  int ngroups;
  PGroup<R> gr[PMAXG];
};

struct PSync {
  unsigned count, gen, err, pad;
};

// grid sizes the persistent schedule compiles (every pass's work item has at
// most PBS threads; the kernel holds the passes of each size it supports)
__host__ __device__ constexpr bool p_supported_n(long n) { return n == 64 || n == 128; }

// launch entry points, defined with the kernel in ens_persistent.cu (its own
// translation unit: the kernel inlines every pass of every supported size)
template <class R>
cudaError_t p_prepare(size_t smem, int *blocks_per_sm);
template <class R>
cudaError_t p_launch(int grid, size_t smem, cudaStream_t st, const PPlan<R> *plan, PSync *sy,
                     unsigned long long wait_ns);
cudaError_t p_barrier_selftest(PSync *sy, cudaStream_t st, unsigned long long wait_ns);

#ifdef DNSB_PERSISTENT_KERNELS
__device__ __forceinline__ unsigned long long p_global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier of nblocks co-resident blocks (sense reversal: the last
// block to arrive resets the count and advances the generation).  False,
// for every thread of the block, if the wait ran past limit_ns.
__device__ __forceinline__ bool grid_barrier(PSync *sy, unsigned nblocks,
                                             unsigned long long limit_ns) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned *gen = &sy->gen;
    const unsigned g0 = *gen;
    __threadfence();  // this block's writes before its arrival
    if (atomicAdd(&sy->count, 1u) == nblocks - 1) {
      atomicExch(&sy->count, 0u);
      __threadfence();
      atomicAdd(&sy->gen, 1u);
    } else {
      const unsigned long long t0 = p_global_ns();
      while (*gen == g0) {
        if (p_global_ns() - t0 > limit_ns) {
          atomicOr(&sy->err, PERR_BARRIER_TIMEOUT);
          ok = 0;
          break;
        }
        __nanosleep(100);
      }
    }
    __threadfence();  // the other blocks' writes after the barrier
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

template <class R, int N, class Sync>
__device__ __forceinline__ void p_item_n(const PGroup<R> &G, const PPhase<R> &P, const Blk b,
                                         Sync sync, unsigned char *sm) {
  if (P.kind == PK_COL) {
    if (P.axis == 0) {
      if (P.fwd)
        colpass_body<R, N, 0, true>(G.S, G.S, G.tw, G.g, P.jobs, b, sync, sm);
      else
        colpass_body<R, N, 0, false>(G.S, G.S, G.tw, G.g, P.jobs, b, sync, sm);
    } else {
      if (P.fwd)
        colpass_body<R, N, 1, true>(G.S, G.S, G.tw, G.g, P.jobs, b, sync, sm);
      else
        colpass_body<R, N, 1, false>(G.S, G.S, G.tw, G.g, P.jobs, b, sync, sm);
    }
  } else if (P.kind == PK_Z) {
    if (P.sub == 0)
      zstage_body<R, N, 0>(G.work, G.stale, G.tw, G.g, G.invn3, b, sync, sm);
    else if (P.sub == 1)
      zstage_body<R, N, 1>(G.work, G.stale, G.tw, G.g, G.invn3, b, sync, sm);
    else
      zstage_body<R, N, 2>(G.work, G.stale, G.tw, G.g, G.invn3, b, sync, sm);
  } else {
    if (P.sub == 0)
      update_body<R, N, 0>(G.work, G.g, P.sa, b);
    else if (P.sub == 1)
      update_body<R, N, 1>(G.work, G.g, P.sa, b);
    else if (P.sub == 2)
      update_body<R, N, 2>(G.work, G.g, P.sa, b);
    else
      update_body<R, N, 3>(G.work, G.g, P.sa, b);
  }
}

template <class R, class Sync>
__device__ __forceinline__ void p_item(const PGroup<R> &G, const PPhase<R> &P, const Blk b, Sync sync,
                                       unsigned char *sm) {
  if (G.n == 64)
    p_item_n<R, 64>(G, P, b, sync, sm);
  else
    p_item_n<R, 128>(G, P, b, sync, sm);
}

// grid: the co-resident maximum (cooperative launch); block: PBS threads
template <class R>
__global__ void __launch_bounds__(PBS, PMinB<R>::value)
    k_ens_step(const PPlan<R> *__restrict__ plan, PSync *sy, unsigned long long wait_ns) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ng = plan->ngroups;
  for (int ph = 0; ph < PPHASES; ph++) {
    int nb[PMAXG], total = 0;
    for (int q = 0; q < ng; q++) {
      const PPhase<R> &P = plan->gr[q].ph[ph];
      const int per = PBS / P.tpi;
      nb[q] = (P.gx * P.gy * P.gz + per - 1) / per;
      total += nb[q];
    }
    for (int u = blockIdx.x; u < total; u += gridDim.x) {
      int q = 0, v = u;
      while (v >= nb[q]) v -= nb[q++];
      const PGroup<R> &G = plan->gr[q];
      const PPhase<R> &P = G.ph[ph];
      const int per = PBS / P.tpi;
      const int sub = (int)threadIdx.x / P.tpi;
      const int item = v * per + sub;
      if (item < P.gx * P.gy * P.gz) {
        const Blk b{item % P.gx, (item / P.gx) % P.gy, item / (P.gx * P.gy),
                    (int)threadIdx.x % P.tpi, P.tpi};
        // every item synchronises on its own barrier (one body per pass)
        p_item(G, P, b, NamedSync{1 + sub, P.tpi}, smem_raw + (size_t)sub * P.smem);
      }
      __syncthreads();  // the next item reuses the block's shared memory
    }
    if (!grid_barrier(sy, gridDim.x, wait_ns)) return;
  }
}

// Self-test of the bounded wait: a barrier of one more block than the grid
// has, which therefore never completes; the wait must give up after
// wait_ns and report PERR_BARRIER_TIMEOUT.
__global__ void k_barrier_selftest(PSync *sy, unsigned long long wait_ns) {
  grid_barrier(sy, gridDim.x + 1, wait_ns);
}
#endif  // DNSB_PERSISTENT_KERNELS

}  // namespace dnsb
