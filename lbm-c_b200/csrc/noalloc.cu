// lbmc_macro_sums_noalloc: the FP64 diagnostic sums (mass, momentum,
// kinetic energy) over caller-owned device arrays, without allocating.
//
// Why it exists: the engine's own diagnostics (LBMC_REDUCE_DIAG) and the
// reference's kinetic-energy sum (LBM-C/index.cu:338-373, which cudaMallocs
// and frees an N-double scratch on every call) both need device scratch.
// Some callers cannot allocate device memory at the point where they want
// these sums: hosts that have already handed the whole device to their own
// pool allocator (a coupled particle or structural solver that reserves HBM
// up front), processes running under a device-memory cap, and time-stepping
// loops that must not incur cudaMalloc's implicit device synchronisation.
// This entry point keeps its scratch in a fixed file-scope device array
// instead.
//
// Scratch: g_partials holds one FP64 partial per block and quantity,
// NOALLOC_MAX_BLOCKS blocks of NOALLOC_NODES_PER_BLOCK nodes, so n is
// limited to NOALLOC_MAX_NODES (2^27 = 134,217,728 nodes, a 512^3 domain);
// larger n is rejected with LBMC_ERR_INVALID_ARG.  The array (320 KiB) is
// resident on every device that loads the library, until the process exits.
// Every call overwrites the partials it then reads, so nothing has to be
// cleared between calls; calls whose kernels overlap on the GPU (different
// streams, no ordering between them) share the array and race.
//
// Set-up: the first call on a device resolves the array's device address
// with cudaGetSymbolAddress while that device is current and caches it; the
// host-side name g_partials is only a stand-in and is never passed to a
// kernel.  Make that first call on each device before any stream capture.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/lbmc.h"
#include "engine_internal.h"
#include "kernels.cuh"

namespace {

constexpr int NOALLOC_BLOCK = 256;
constexpr int NOALLOC_ITEMS = 64;  // nodes per thread
constexpr long long NOALLOC_NODES_PER_BLOCK = (long long)NOALLOC_BLOCK * NOALLOC_ITEMS;
constexpr int NOALLOC_MAX_BLOCKS = 8192;
constexpr long long NOALLOC_MAX_NODES = NOALLOC_NODES_PER_BLOCK * NOALLOC_MAX_BLOCKS;
constexpr int NOALLOC_VALUES = lbmc::DIAG_VALUES;  // mass, momentum x/y/z, kinetic energy
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_partials[NOALLOC_MAX_BLOCKS * NOALLOC_VALUES];

std::mutex g_setup_mutex;
double *g_partials_dev[NOALLOC_MAX_DEVICES] = {nullptr};

// Block sums of rho, rho*u and 0.5*rho*|u|^2 over one chunk of nodes.
__global__ void __launch_bounds__(NOALLOC_BLOCK)
    noalloc_partials_kernel(const double *rho, const double *ux, const double *uy, const double *uz,
                            long long n, double *partials) {
  const long long base = (long long)blockIdx.x * NOALLOC_NODES_PER_BLOCK;
  double v[NOALLOC_VALUES] = {0, 0, 0, 0, 0};
  for (int k = 0; k < NOALLOC_ITEMS; k++) {
    const long long i = base + (long long)k * NOALLOC_BLOCK + threadIdx.x;
    if (i >= n) break;
    const double r = rho[i];
    const double x = ux[i], y = uy ? uy[i] : 0.0, z = uz ? uz[i] : 0.0;
    v[0] += r;
    v[1] += r * x;
    v[2] += r * y;
    v[3] += r * z;
    v[4] += 0.5 * r * (x * x + y * y + z * z);
  }
  __shared__ double red[NOALLOC_BLOCK / 32][NOALLOC_VALUES];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NOALLOC_VALUES; q++) {
    double s = v[q];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (lane == 0) red[warp][q] = s;
  }
  __syncthreads();
  if (threadIdx.x < NOALLOC_VALUES) {
    double s = 0;
    for (int w = 0; w < NOALLOC_BLOCK / 32; w++) s += red[w][threadIdx.x];
    partials[(long long)blockIdx.x * NOALLOC_VALUES + threadIdx.x] = s;
  }
}

// Sums the partials of nblocks blocks in a fixed order.
__global__ void __launch_bounds__(NOALLOC_BLOCK)
    noalloc_finalize_kernel(const double *partials, int nblocks, double *out) {
  __shared__ double sh[NOALLOC_BLOCK];
  for (int q = 0; q < NOALLOC_VALUES; q++) {
    double s = 0;
    for (int b = threadIdx.x; b < nblocks; b += NOALLOC_BLOCK) s += partials[(long long)b * NOALLOC_VALUES + q];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = NOALLOC_BLOCK / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[q] = sh[0];
    __syncthreads();
  }
}

lbmc_status noalloc_fail(lbmc_status s, const std::string &what) {
  lbmc::set_last_error("lbmc_macro_sums_noalloc: " + what);
  return s;
}

// Device address of g_partials on the current device (resolved once; a
// cudaDeviceReset by the caller invalidates the cached address, so callers
// that reset a device must not use this entry point on it afterwards).
lbmc_status partials_for(int device, double **out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_partials_dev[device]) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_partials);
    if (e != cudaSuccess || !ptr) {
      cudaGetLastError();
      return noalloc_fail(LBMC_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    }
    g_partials_dev[device] = static_cast<double *>(ptr);
  }
  *out = g_partials_dev[device];
  return LBMC_OK;
}

}  // namespace

extern "C" lbmc_status lbmc_macro_sums_noalloc(int device, const double *rho, const double *ux,
                                               const double *uy, const double *uz, long long n,
                                               double *sums, void *cuda_stream) {
  if (!rho || !ux || !sums) return noalloc_fail(LBMC_ERR_INVALID_ARG, "rho, ux and sums must not be NULL");
  if (n < 1) return noalloc_fail(LBMC_ERR_INVALID_ARG, "n must be at least 1");
  if (n > NOALLOC_MAX_NODES)  // beyond the fixed scratch
    return noalloc_fail(LBMC_ERR_INVALID_ARG, "n = " + std::to_string(n) + " exceeds the fixed scratch's " +
                                                  std::to_string(NOALLOC_MAX_NODES) + " nodes");
  if (device < 0 || device >= NOALLOC_MAX_DEVICES)
    return noalloc_fail(LBMC_ERR_INVALID_ARG, "device ordinal out of range");
  // An error left pending by earlier work on this thread would otherwise be
  // reported after the launches below as if they had failed; it is reported
  // as what it is and left in place for its owner.
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess)
    return noalloc_fail(LBMC_ERR_CUDA, std::string("a CUDA error from earlier work is pending (not cleared): ") +
                                           cudaGetErrorString(pending));
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(LBMC_ERR_NO_DEVICE, "cudaSetDevice(" + std::to_string(device) + ") failed");
  }
  double *partials = nullptr;
  const lbmc_status st = partials_for(device, &partials);
  if (st != LBMC_OK) return st;
  const int nblocks = (int)((n + NOALLOC_NODES_PER_BLOCK - 1) / NOALLOC_NODES_PER_BLOCK);
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  noalloc_partials_kernel<<<nblocks, NOALLOC_BLOCK, 0, stream>>>(rho, ux, uy, uz, n, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(LBMC_ERR_CUDA, std::string("partials launch: ") + cudaGetErrorString(e));
  noalloc_finalize_kernel<<<1, NOALLOC_BLOCK, 0, stream>>>(partials, nblocks, sums);
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(LBMC_ERR_CUDA, std::string("finalize launch: ") + cudaGetErrorString(e));
  return LBMC_OK;
}
