// ens_persistent.cu -- the persistent ensemble kernel (persistent.cuh) and
// its launch entry points, in a translation unit of their own: the kernel
// inlines every pass body of every grid size it supports.
#define DNSB_PERSISTENT_KERNELS
#include "persistent.cuh"

namespace dnsb {

template <class R>
cudaError_t p_prepare(size_t smem, int *blocks_per_sm) {
  cudaError_t e = cudaFuncSetAttribute(k_ens_step<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_ens_step<R>, PBS, smem);
}

// one cooperative launch (all blocks co-resident, or the launch fails)
template <class R>
cudaError_t p_launch(int grid, size_t smem, cudaStream_t st, const PPlan<R> *plan, PSync *sy,
                     unsigned long long wait_ns) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(PBS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_ens_step<R>, plan, sy, wait_ns);
}

cudaError_t p_barrier_selftest(PSync *sy, cudaStream_t st, unsigned long long wait_ns) {
  k_barrier_selftest<<<2, 32, 0, st>>>(sy, wait_ns);
  return cudaGetLastError();
}

template cudaError_t p_prepare<float>(size_t, int *);
template cudaError_t p_prepare<double>(size_t, int *);
template cudaError_t p_launch<float>(int, size_t, cudaStream_t, const PPlan<float> *, PSync *,
                                     unsigned long long);
template cudaError_t p_launch<double>(int, size_t, cudaStream_t, const PPlan<double> *, PSync *,
                                      unsigned long long);

}  // namespace dnsb
