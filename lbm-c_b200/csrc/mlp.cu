// Training and inference kernels of the learned subgrid closure (lbmc_mlp_*).
// No counterpart in the reference.
//
// Training is plain mini-batch Adam on the mean squared error, all on the
// GPU with hand-written kernels:
//   mlp_grad_kernel      one sample per thread: forward pass with the BF16
//                        weights (FP32 accumulation), backward pass, block
//                        gradient sums in shared memory, one FP32 partial
//                        per block;
//   mlp_reduce_kernel    sums the block partials in a fixed order
//                        (deterministic gradients);
//   mlp_adam_kernel      Adam on the FP32 master weights, refreshes the BF16
//                        copy the forward pass uses.
// The gradient is that of the loss as computed with the BF16-rounded
// weights, which is what the CPU check (oracle/mlp_oracle.py) reproduces.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/lbmc.h"
#include "engine_internal.h"
#include "mlp.cuh"

using namespace lbmc;

namespace {

constexpr int GRAD_BLOCK = 256;
constexpr int GRAD_SLOTS = MLP_PARAMS + 1;  // parameters + loss

lbmc_status merr(lbmc_status s, const std::string &m) {
  lbmc::set_last_error(m);
  return s;
}

__device__ __forceinline__ float sigmoidf_(float x) { return 1.0f / (1.0f + expf(-x)); }

__global__ void normalise_kernel(const float *raw, const float *y, long long n, MlpClosure c, float *xn,
                                 float *yn) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  for (int i = 0; i < MLP_IN; i++) xn[k * MLP_IN + i] = (raw[k * MLP_IN + i] - c.mean[i]) * c.inv_std[i];
  if (y) yn[k] = y[k] / c.target_scale;
}

// Gradient of sum over the batch of (y_hat - t)^2 / B with respect to the
// (BF16-rounded) parameters; idx selects the batch's samples.
__global__ void __launch_bounds__(GRAD_BLOCK)
    mlp_grad_kernel(const float *xn, const float *tn, const int *idx, int B, const __nv_bfloat16 *w,
                    float *partials) {
  __shared__ float g[GRAD_SLOTS];
  __shared__ float wf[MLP_PARAMS];
  for (int p = threadIdx.x; p < MLP_PARAMS; p += blockDim.x) {
    wf[p] = __bfloat162float(w[p]);
    g[p] = 0.f;
  }
  if (threadIdx.x == 0) g[MLP_PARAMS] = 0.f;
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < B) {
    const int k = idx ? idx[s] : s;
    float x[MLP_IN];
    for (int i = 0; i < MLP_IN; i++) x[i] = xn[(long long)k * MLP_IN + i];
    float a1[MLP_H], a2[MLP_H];
    for (int j = 0; j < MLP_H; j++) {
      float a = wf[MLP_B1 + j];
      for (int i = 0; i < MLP_IN; i++) a += wf[MLP_W1 + j * MLP_IN + i] * x[i];
      a1[j] = a;
    }
    float y = wf[MLP_B3];
    for (int j = 0; j < MLP_H; j++) {
      float a = wf[MLP_B2 + j];
      for (int i = 0; i < MLP_H; i++) a += wf[MLP_W2 + j * MLP_H + i] * silu(a1[i]);
      a2[j] = a;
      y += wf[MLP_W3 + j] * silu(a);
    }
    const float r = y - tn[k];
    const float dy = 2.0f * r / (float)B;
    atomicAdd(&g[MLP_PARAMS], r * r / (float)B);
    atomicAdd(&g[MLP_B3], dy);
    float d1[MLP_H];
    for (int i = 0; i < MLP_H; i++) d1[i] = 0.f;
    for (int j = 0; j < MLP_H; j++) {
      const float sg = sigmoidf_(a2[j]);
      const float h2 = a2[j] * sg;
      atomicAdd(&g[MLP_W3 + j], dy * h2);
      const float d2 = dy * wf[MLP_W3 + j] * (sg + a2[j] * sg * (1.0f - sg));
      atomicAdd(&g[MLP_B2 + j], d2);
      for (int i = 0; i < MLP_H; i++) {
        atomicAdd(&g[MLP_W2 + j * MLP_H + i], d2 * silu(a1[i]));
        d1[i] += d2 * wf[MLP_W2 + j * MLP_H + i];
      }
    }
    for (int i = 0; i < MLP_H; i++) {
      const float sg = sigmoidf_(a1[i]);
      const float d = d1[i] * (sg + a1[i] * sg * (1.0f - sg));
      atomicAdd(&g[MLP_B1 + i], d);
      for (int q = 0; q < MLP_IN; q++) atomicAdd(&g[MLP_W1 + i * MLP_IN + q], d * x[q]);
    }
  }
  __syncthreads();
  for (int p = threadIdx.x; p < GRAD_SLOTS; p += blockDim.x)
    partials[(long long)blockIdx.x * GRAD_SLOTS + p] = g[p];
}

__global__ void mlp_reduce_kernel(const float *partials, int nblocks, float *out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= GRAD_SLOTS) return;
  float s = 0.f;
  for (int b = 0; b < nblocks; b++) s += partials[(long long)b * GRAD_SLOTS + p];
  out[p] = s;
}

__global__ void mlp_adam_kernel(float *master, float *m, float *v, const float *grad, __nv_bfloat16 *w,
                                float lr, float b1, float b2, float eps, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= MLP_PARAMS) return;
  const float g = grad[p];
  const float mi = b1 * m[p] + (1.0f - b1) * g;
  const float vi = b2 * v[p] + (1.0f - b2) * g * g;
  m[p] = mi;
  v[p] = vi;
  const float step = lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  master[p] -= step;
  w[p] = __float2bfloat16_rn(master[p]);
}

__global__ void mlp_predict_kernel(const float *xn, long long n, const __nv_bfloat16 *w, float scale,
                                   float *out) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  float x[MLP_IN];
  for (int i = 0; i < MLP_IN; i++) x[i] = xn[k * MLP_IN + i];
  out[k] = scale * mlp_forward(w, x);
}

// The in-step evaluation (mlp_forward_warp) over a batch: 32 samples per
// warp, lanes past n feed zeros.
constexpr int STEP_PREDICT_BLOCK = 128;
__global__ void __launch_bounds__(STEP_PREDICT_BLOCK)
    mlp_predict_step_kernel(const float *raw, long long n, const MlpStep *cl, const MlpConsts kc, float *out) {
  __shared__ __align__(16) unsigned stage[STEP_PREDICT_BLOCK / 32][128];
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float x[MLP_IN];
  for (int i = 0; i < MLP_IN; i++) x[i] = k < n ? fmaf(raw[k * MLP_IN + i], kc.scale[i], kc.shift[i]) : 0.0f;
  const float y = mlp_forward_warp(cl, x, stage[threadIdx.x >> 5]) + kc.b3;
  if (k < n) out[k] = kc.target_scale * y;
}

__global__ void features_kernel(const float *S, const float *rho, long long n, float *out) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  strain_features(S + k * 6, rho ? rho[k] : 1.0f, out + k * MLP_IN);
}

}  // namespace

struct lbmc_mlp {
  int device = 0;
  MlpClosure host;  // weights (BF16) + normalisation
  std::vector<float> master;
  float *d_master = nullptr, *d_m = nullptr, *d_v = nullptr, *d_grad = nullptr;
  __nv_bfloat16 *d_w = nullptr;
  long long adam_t = 0;
  unsigned long long seed = 0;
};

namespace {

template <class T>
cudaError_t upload(T **dst, const T *src, size_t count) {
  cudaError_t e = cudaMalloc(dst, count * sizeof(T) + 16);
  if (e == cudaSuccess && src) e = cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

void sync_host_weights(lbmc_mlp *m) {
  for (int p = 0; p < MLP_PARAMS; p++) m->host.w[p] = __float2bfloat16_rn(m->master[p]);
}

}  // namespace

const MlpClosure *lbmc_mlp_closure(const lbmc_mlp *m) { return m ? &m->host : nullptr; }

namespace lbmc {

void mlp_step_layout(const MlpClosure &cl, int iterations, MlpStep &s, MlpConsts &kc) {
  memset(&s, 0, sizeof(s));
  memset(&kc, 0, sizeof(kc));
  // BF16 bit pattern of parameter p, times `scale` (1 or the exact 1/2 that
  // the in-step SiLU expects folded into layers 1 and 2).
  auto bits = [&](int p, float scale) -> unsigned {
    if (p < 0) return 0u;
    const __nv_bfloat16 v = __float2bfloat16_rn(scale * __bfloat162float(cl.w[p]));
    unsigned short b;
    memcpy(&b, &v, sizeof(b));
    return b;
  };
  auto pair = [&](int p0, int p1, float scale) -> unsigned {
    return bits(p0, scale) | (bits(p1, scale) << 16);
  };
  auto set = [](uint4 &v, int j, unsigned w) { (j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w) = w; };
  for (int lane = 0; lane < 32; lane++) {
    const int g = lane >> 2, c = lane & 3;
    for (int j = 0; j < 4; j++) {
      const int n = 8 * j + g, k = 2 * c, col = 8 * j + 2 * c;
      set(s.w1[lane], j, pair(k < MLP_IN ? MLP_W1 + n * MLP_IN + k : -1,
                              k + 1 < MLP_IN ? MLP_W1 + n * MLP_IN + k + 1 : -1, 0.5f));
      for (int kt = 0; kt < 2; kt++)
        for (int r = 0; r < 2; r++) {
          const int kk = 16 * kt + 8 * r + 2 * c;
          set(s.w2[j][lane], 2 * kt + r, pair(MLP_W2 + n * MLP_H + kk, MLP_W2 + n * MLP_H + kk + 1, 0.5f));
        }
      set(s.b1[lane], j, pair(MLP_B1 + col, MLP_B1 + col + 1, 0.5f));
      set(s.b2[lane], j, pair(MLP_B2 + col, MLP_B2 + col + 1, 0.5f));
    }
    for (int kt = 0; kt < 2; kt++)
      for (int r = 0; r < 2; r++) {
        const int kk = 16 * kt + 8 * r + 2 * c;
        set(s.w3[lane], 2 * kt + r, g == 0 ? pair(MLP_W3 + kk, MLP_W3 + kk + 1, 1.0f) : 0u);
      }
  }
  for (int i = 0; i < MLP_IN; i++) {
    kc.scale[i] = cl.inv_std[i];
    kc.shift[i] = -cl.mean[i] * cl.inv_std[i];
    kc.lo[i] = cl.lo[i];
    kc.hi[i] = cl.hi[i];
  }
  kc.b3 = __bfloat162float(cl.w[MLP_B3]);
  kc.target_scale = cl.target_scale;
  kc.iterations = iterations;
}

}  // namespace lbmc

extern "C" lbmc_status lbmc_mlp_create(int device, unsigned long long seed, lbmc_mlp **out) {
  if (!out) return merr(LBMC_ERR_INVALID_ARG, "lbmc_mlp_create: out is NULL");
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return merr(LBMC_ERR_NO_DEVICE, "lbmc_mlp_create: no such device");
  }
  lbmc_mlp *m = new lbmc_mlp();
  m->device = device;
  m->seed = seed;
  m->master.assign(MLP_PARAMS, 0.f);
  std::mt19937_64 rng(seed);
  auto xavier = [&](int off, int fan_in, int fan_out, int count) {
    const float a = std::sqrt(6.0f / (float)(fan_in + fan_out));
    std::uniform_real_distribution<float> u(-a, a);
    for (int k = 0; k < count; k++) m->master[off + k] = u(rng);
  };
  xavier(MLP_W1, MLP_IN, MLP_H, MLP_H * MLP_IN);
  xavier(MLP_W2, MLP_H, MLP_H, MLP_H * MLP_H);
  xavier(MLP_W3, MLP_H, 1, MLP_H);
  memset(&m->host, 0, sizeof(m->host));
  for (int i = 0; i < MLP_IN; i++) {
    m->host.inv_std[i] = 1.f;
    m->host.lo[i] = -1e30f;
    m->host.hi[i] = 1e30f;
  }
  m->host.target_scale = 1.f;
  m->host.iterations = 2;
  sync_host_weights(m);
  cudaError_t e = upload(&m->d_master, m->master.data(), MLP_PARAMS);
  std::vector<float> zeros(GRAD_SLOTS, 0.f);
  if (e == cudaSuccess) e = upload(&m->d_m, zeros.data(), MLP_PARAMS);
  if (e == cudaSuccess) e = upload(&m->d_v, zeros.data(), MLP_PARAMS);
  if (e == cudaSuccess) e = upload(&m->d_grad, zeros.data(), GRAD_SLOTS);
  if (e == cudaSuccess) e = upload(&m->d_w, m->host.w, MLP_PARAMS);
  if (e != cudaSuccess) {
    lbmc_mlp_destroy(m);
    return merr(LBMC_ERR_ALLOC, std::string("lbmc_mlp_create: ") + cudaGetErrorString(e));
  }
  *out = m;
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_mlp_set_normalization(lbmc_mlp *m, const float *mean, const float *std,
                                                  const float *lo, const float *hi, float target_scale) {
  if (!m || !mean || !std || !(target_scale > 0)) return merr(LBMC_ERR_INVALID_ARG, "lbmc_mlp_set_normalization");
  for (int i = 0; i < MLP_IN; i++) {
    if (!(std[i] > 0)) return merr(LBMC_ERR_INVALID_ARG, "lbmc_mlp_set_normalization: std must be > 0");
    m->host.mean[i] = mean[i];
    m->host.inv_std[i] = 1.0f / std[i];
    m->host.lo[i] = lo ? lo[i] : -1e30f;
    m->host.hi[i] = hi ? hi[i] : 1e30f;
  }
  m->host.target_scale = target_scale;
  return LBMC_OK;
}

// Normalised copies of host features / targets on the device.
static lbmc_status stage(lbmc_mlp *m, const float *features, const float *target, long long n, float **xn,
                         float **yn) {
  float *raw = nullptr, *ty = nullptr;
  cudaError_t e = upload(&raw, features, (size_t)n * MLP_IN);
  if (e == cudaSuccess && target) e = upload(&ty, target, (size_t)n);
  if (e == cudaSuccess) e = cudaMalloc(xn, (size_t)n * MLP_IN * sizeof(float));
  if (e == cudaSuccess && target) e = cudaMalloc(yn, (size_t)n * sizeof(float));
  if (e == cudaSuccess) {
    normalise_kernel<<<(unsigned)((n + 255) / 256), 256>>>(raw, ty, n, m->host, *xn, target ? *yn : nullptr);
    e = cudaDeviceSynchronize();
  }
  cudaFree(raw);
  cudaFree(ty);
  if (e != cudaSuccess) return merr(LBMC_ERR_CUDA, std::string("mlp staging: ") + cudaGetErrorString(e));
  return LBMC_OK;
}

static cudaError_t gradient(lbmc_mlp *m, const float *xn, const float *yn, const int *idx, int B,
                            float *partials) {
  const int nb = (B + GRAD_BLOCK - 1) / GRAD_BLOCK;
  mlp_grad_kernel<<<nb, GRAD_BLOCK>>>(xn, yn, idx, B, m->d_w, partials);
  mlp_reduce_kernel<<<(GRAD_SLOTS + 255) / 256, 256>>>(partials, nb, m->d_grad);
  return cudaGetLastError();
}

extern "C" lbmc_status lbmc_mlp_gradients(lbmc_mlp *m, const float *features, const float *target, long long n,
                                          float *grads, float *loss) {
  if (!m || !features || !target || n < 1 || n > (1 << 24)) return merr(LBMC_ERR_INVALID_ARG, "lbmc_mlp_gradients");
  cudaSetDevice(m->device);
  float *xn = nullptr, *yn = nullptr, *partials = nullptr;
  lbmc_status s = stage(m, features, target, n, &xn, &yn);
  if (s != LBMC_OK) return s;
  const int nb = (int)((n + GRAD_BLOCK - 1) / GRAD_BLOCK);
  cudaError_t e = cudaMalloc(&partials, (size_t)nb * GRAD_SLOTS * sizeof(float));
  if (e == cudaSuccess) e = gradient(m, xn, yn, nullptr, (int)n, partials);
  std::vector<float> out(GRAD_SLOTS);
  if (e == cudaSuccess) e = cudaMemcpy(out.data(), m->d_grad, GRAD_SLOTS * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(xn);
  cudaFree(yn);
  cudaFree(partials);
  if (e != cudaSuccess) return merr(LBMC_ERR_CUDA, std::string("lbmc_mlp_gradients: ") + cudaGetErrorString(e));
  if (grads) memcpy(grads, out.data(), MLP_PARAMS * sizeof(float));
  if (loss) *loss = out[MLP_PARAMS];
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_mlp_train(lbmc_mlp *m, const float *features, const float *target, long long n,
                                      int epochs, int batch, float lr, float *loss_history) {
  if (!m || !features || !target || n < 1 || epochs < 1 || batch < 1 || !(lr > 0))
    return merr(LBMC_ERR_INVALID_ARG, "lbmc_mlp_train");
  cudaSetDevice(m->device);
  float *xn = nullptr, *yn = nullptr, *partials = nullptr;
  int *idx = nullptr;
  lbmc_status s = stage(m, features, target, n, &xn, &yn);
  if (s != LBMC_OK) return s;
  const int nb = (batch + GRAD_BLOCK - 1) / GRAD_BLOCK;
  cudaError_t e = cudaMalloc(&partials, (size_t)nb * GRAD_SLOTS * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&idx, (size_t)n * sizeof(int));
  std::vector<int> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  std::mt19937_64 rng(m->seed ^ 0x9E3779B97F4A7C15ull);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int ep = 0; ep < epochs && e == cudaSuccess; ep++) {
    std::shuffle(perm.begin(), perm.end(), rng);
    e = cudaMemcpy(idx, perm.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice);
    double loss_sum = 0;
    long long batches = 0;
    for (long long off = 0; off + batch <= n && e == cudaSuccess; off += batch) {
      e = gradient(m, xn, yn, idx + off, batch, partials);
      m->adam_t++;
      const float c1 = 1.0f - std::pow(b1, (float)m->adam_t), c2 = 1.0f - std::pow(b2, (float)m->adam_t);
      if (e == cudaSuccess) {
        mlp_adam_kernel<<<(MLP_PARAMS + 255) / 256, 256>>>(m->d_master, m->d_m, m->d_v, m->d_grad, m->d_w, lr, b1,
                                                           b2, eps, c1, c2);
        e = cudaGetLastError();
      }
      if (loss_history && e == cudaSuccess && (batches % 16 == 0)) {
        float l = 0;
        e = cudaMemcpy(&l, m->d_grad + MLP_PARAMS, sizeof(float), cudaMemcpyDeviceToHost);
        loss_sum += l;
      }
      batches++;
    }
    if (loss_history) loss_history[ep] = (float)(loss_sum / std::max(1LL, (batches + 15) / 16));
  }
  if (e == cudaSuccess)
    e = cudaMemcpy(m->master.data(), m->d_master, MLP_PARAMS * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(xn);
  cudaFree(yn);
  cudaFree(partials);
  cudaFree(idx);
  if (e != cudaSuccess) return merr(LBMC_ERR_CUDA, std::string("lbmc_mlp_train: ") + cudaGetErrorString(e));
  sync_host_weights(m);
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_mlp_predict(lbmc_mlp *m, const float *features, long long n, float *out) {
  if (!m || !features || !out || n < 1) return merr(LBMC_ERR_INVALID_ARG, "lbmc_mlp_predict");
  cudaSetDevice(m->device);
  float *xn = nullptr, *yn = nullptr, *res = nullptr;
  lbmc_status s = stage(m, features, nullptr, n, &xn, &yn);
  if (s != LBMC_OK) return s;
  cudaError_t e = cudaMalloc(&res, (size_t)n * sizeof(float));
  if (e == cudaSuccess) {
    mlp_predict_kernel<<<(unsigned)((n + 255) / 256), 256>>>(xn, n, m->d_w, m->host.target_scale, res);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, res, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(xn);
  cudaFree(res);
  if (e != cudaSuccess) return merr(LBMC_ERR_CUDA, std::string("lbmc_mlp_predict: ") + cudaGetErrorString(e));
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_mlp_predict_step(lbmc_mlp *m, const float *features, long long n, float *out) {
  if (!m || !features || !out || n < 1) return merr(LBMC_ERR_INVALID_ARG, "lbmc_mlp_predict_step");
  cudaSetDevice(m->device);
  MlpStep hs;
  MlpConsts kc;
  mlp_step_layout(m->host, 1, hs, kc);
  float *raw = nullptr, *res = nullptr;
  MlpStep *ds = nullptr;
  cudaError_t e = upload(&raw, features, (size_t)n * MLP_IN);
  if (e == cudaSuccess) e = upload(&ds, &hs, 1);
  if (e == cudaSuccess) e = cudaMalloc(&res, (size_t)n * sizeof(float));
  if (e == cudaSuccess) {
    const long long blocks = (n + STEP_PREDICT_BLOCK - 1) / STEP_PREDICT_BLOCK;
    mlp_predict_step_kernel<<<(unsigned)blocks, STEP_PREDICT_BLOCK>>>(raw, n, ds, kc, res);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, res, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(raw);
  cudaFree(ds);
  cudaFree(res);
  if (e != cudaSuccess) return merr(LBMC_ERR_CUDA, std::string("lbmc_mlp_predict_step: ") + cudaGetErrorString(e));
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_mlp_features(int device, const float *strain6, const float *rho, long long n,
                                         float *features6) {
  if (!strain6 || !features6 || n < 1) return merr(LBMC_ERR_INVALID_ARG, "lbmc_mlp_features");
  if (cudaSetDevice(device) != cudaSuccess) return merr(LBMC_ERR_NO_DEVICE, "lbmc_mlp_features");
  float *S = nullptr, *r = nullptr, *f = nullptr;
  cudaError_t e = upload(&S, strain6, (size_t)n * 6);
  if (e == cudaSuccess && rho) e = upload(&r, rho, (size_t)n);
  if (e == cudaSuccess) e = cudaMalloc(&f, (size_t)n * MLP_IN * sizeof(float));
  if (e == cudaSuccess) {
    features_kernel<<<(unsigned)((n + 255) / 256), 256>>>(S, r, n, f);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(features6, f, (size_t)n * MLP_IN * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(S);
  cudaFree(r);
  cudaFree(f);
  if (e != cudaSuccess) return merr(LBMC_ERR_CUDA, std::string("lbmc_mlp_features: ") + cudaGetErrorString(e));
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_mlp_get_params(lbmc_mlp *m, float *params) {
  if (!m || !params) return merr(LBMC_ERR_INVALID_ARG, "lbmc_mlp_get_params");
  for (int p = 0; p < MLP_PARAMS; p++) params[p] = __bfloat162float(m->host.w[p]);
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_mlp_set_params(lbmc_mlp *m, const float *params) {
  if (!m || !params) return merr(LBMC_ERR_INVALID_ARG, "lbmc_mlp_set_params");
  cudaSetDevice(m->device);
  for (int p = 0; p < MLP_PARAMS; p++) m->master[p] = params[p];
  sync_host_weights(m);
  cudaError_t e = cudaMemcpy(m->d_master, m->master.data(), MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(m->d_w, m->host.w, MLP_PARAMS * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(m->d_m, 0, MLP_PARAMS * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(m->d_v, 0, MLP_PARAMS * sizeof(float));
  m->adam_t = 0;
  if (e != cudaSuccess) return merr(LBMC_ERR_CUDA, "lbmc_mlp_set_params");
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_mlp_destroy(lbmc_mlp *m) {
  if (!m) return LBMC_OK;
  cudaSetDevice(m->device);
  cudaFree(m->d_master);
  cudaFree(m->d_m);
  cudaFree(m->d_v);
  cudaFree(m->d_grad);
  cudaFree(m->d_w);
  delete m;
  return LBMC_OK;
}
