// Learned subgrid closure: a 6 -> 32 -> 32 -> 1 MLP with SiLU activations
// (1313 parameters), BF16 weights and FP32 accumulation, mapping six
// invariants of the local strain-rate estimate to an eddy viscosity.  No
// counterpart in the reference, whose only subgrid model is Smagorinsky
// (LBM-C/collision.cu:445-463); Smagorinsky remains the fallback wherever
// the inputs leave the range seen in training.
#pragma once

#include <cuda_bf16.h>

namespace lbmc {

constexpr int MLP_IN = 6;
constexpr int MLP_H = 32;
// Parameter layout (floats / bf16): W1[32][6], b1[32], W2[32][32], b2[32],
// W3[32], b3.
constexpr int MLP_W1 = 0;
constexpr int MLP_B1 = MLP_W1 + MLP_H * MLP_IN;
constexpr int MLP_W2 = MLP_B1 + MLP_H;
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;
constexpr int MLP_W3 = MLP_B2 + MLP_H;
constexpr int MLP_B3 = MLP_W3 + MLP_H;
constexpr int MLP_PARAMS = MLP_B3 + 1;  // 1313

// What the step kernel needs for inference (device memory).
struct MlpClosure {
  __nv_bfloat16 w[MLP_PARAMS];
  float mean[MLP_IN], inv_std[MLP_IN];  // input normalisation
  float lo[MLP_IN], hi[MLP_IN];         // normalised training range (fallback outside)
  float target_scale;                    // nu_t = max(0, target_scale * y)
  int iterations;                        // fixed-point passes for tau_eff
};

__host__ __device__ inline float silu(float x) { return x / (1.0f + expf(-x)); }

// Six invariants of a symmetric strain-rate tensor S (xx, yy, zz, xy, yz,
// xz) and the density: log|S| with |S| = sqrt(2 S:S), log of the summed
// absolute entries (the quantity Smagorinsky uses), signed log of det S,
// tr S, log of the diagonal magnitude, and rho - 1.  The same function
// prepares training data and runs inside the step kernel.
__host__ __device__ inline void strain_features(const float *S, float rho, float *f) {
  const float xx = S[0], yy = S[1], zz = S[2], xy = S[3], yz = S[4], xz = S[5];
  const float ss = xx * xx + yy * yy + zz * zz + 2.0f * (xy * xy + yz * yz + xz * xz);
  const float mag = sqrtf(2.0f * ss);
  const float sabs = fabsf(xx) + fabsf(yy) + fabsf(zz) + 2.0f * (fabsf(xy) + fabsf(yz) + fabsf(xz));
  const float det = xx * (yy * zz - yz * yz) - xy * (xy * zz - yz * xz) + xz * (xy * yz - yy * xz);
  const float diag = sqrtf(xx * xx + yy * yy + zz * zz);
  const float tiny = 1e-12f;
  f[0] = logf(tiny + mag);
  f[1] = logf(tiny + sabs);
  f[2] = copysignf(logf(1.0f + fabsf(det) * 1e9f), det);
  f[3] = (xx + yy + zz) * 1e3f;
  f[4] = logf(tiny + diag);
  f[5] = (rho - 1.0f) * 1e2f;
}

// Forward pass of one sample with BF16 weights, FP32 accumulation.
__device__ inline float mlp_forward(const __nv_bfloat16 *w, const float *x) {
  float h1[MLP_H];
#pragma unroll
  for (int j = 0; j < MLP_H; j++) {
    float a = __bfloat162float(w[MLP_B1 + j]);
#pragma unroll
    for (int i = 0; i < MLP_IN; i++) a += __bfloat162float(w[MLP_W1 + j * MLP_IN + i]) * x[i];
    h1[j] = silu(a);
  }
  float y = __bfloat162float(w[MLP_B3]);
#pragma unroll 4
  for (int j = 0; j < MLP_H; j++) {
    float a = __bfloat162float(w[MLP_B2 + j]);
#pragma unroll
    for (int i = 0; i < MLP_H; i++) a += __bfloat162float(w[MLP_W2 + j * MLP_H + i]) * h1[i];
    y += __bfloat162float(w[MLP_W3 + j]) * silu(a);
  }
  return y;
}

}  // namespace lbmc
