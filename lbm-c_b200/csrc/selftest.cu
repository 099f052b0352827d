// Device-side failure-detection self-test: a wait that can never complete
// must give up after its bound and report a status, leaving the context
// usable.  Uses the same bounded mbarrier wait as the bulk-copy pipeline.
#include <cuda_runtime.h>

#include <cstdio>

#include "../../include/lbmc.h"
#include "kernels.cuh"

namespace {

__global__ void wait_never_arrives_kernel(long long limit_cycles, unsigned *flag) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x == 0) {
    lbmc::mbar_init(lbmc::smem_addr(&bar), 1);  // one arrival that nobody makes
    lbmc::mbar_fence_init();
  }
  __syncthreads();
  if (!lbmc::mbar_wait_bounded(lbmc::smem_addr(&bar), 0, limit_cycles)) atomicOr(flag, lbmc::ERROR_TIMEOUT);
}

}  // namespace

extern "C" lbmc_status lbmc_selftest_wait_timeout(int device, double seconds) {
  if (!(seconds > 0) || seconds > 10) return LBMC_ERR_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return LBMC_ERR_NO_DEVICE;
  }
  int khz = 0;
  cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, device);
  unsigned *flag = nullptr;
  if (cudaMalloc(&flag, sizeof(unsigned)) != cudaSuccess) return LBMC_ERR_ALLOC;
  cudaMemset(flag, 0, sizeof(unsigned));
  const long long limit = (long long)((khz > 0 ? khz : 2000000) * 1000.0 * seconds);
  wait_never_arrives_kernel<<<1, 32>>>(limit, flag);
  unsigned host = 0;
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(&host, flag, sizeof(host), cudaMemcpyDeviceToHost);
  cudaFree(flag);
  if (e != cudaSuccess) return LBMC_ERR_CUDA;
  return (host & lbmc::ERROR_TIMEOUT) ? LBMC_ERR_TIMEOUT : LBMC_OK;
}
