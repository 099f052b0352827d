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
// xz) and the density: log|S| with |S|^2 = 2 S:S, log of the summed
// absolute entries (the quantity Smagorinsky uses), signed log of det S,
// tr S, log of the diagonal magnitude, and rho - 1.  The same function
// prepares training data and runs inside the step kernel; the logarithms
// use the hardware log2 (absolute error ~1e-7, far below the BF16 inputs'
// resolution).
__host__ __device__ inline float fast_log(float x) {
#ifdef __CUDA_ARCH__
  return __logf(x);
#else
  return logf(x);
#endif
}
__host__ __device__ inline void strain_features(const float *S, float rho, float *f) {
  const float xx = S[0], yy = S[1], zz = S[2], xy = S[3], yz = S[4], xz = S[5];
  const float d2 = xx * xx + yy * yy + zz * zz;
  const float ss = d2 + 2.0f * (xy * xy + yz * yz + xz * xz);
  const float sabs = fabsf(xx) + fabsf(yy) + fabsf(zz) + 2.0f * (fabsf(xy) + fabsf(yz) + fabsf(xz));
  const float det = xx * (yy * zz - yz * yz) - xy * (xy * zz - yz * xz) + xz * (xy * yz - yy * xz);
  f[0] = 0.5f * fast_log(2.0f * ss + 1e-24f);
  f[1] = fast_log(1e-12f + sabs);
  f[2] = copysignf(fast_log(1.0f + fabsf(det) * 1e9f), det);
  f[3] = (xx + yy + zz) * 1e3f;
  f[4] = 0.5f * fast_log(d2 + 1e-24f);
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

// ------------------------------------------ in-step (tensor-core) inference
//
// Inside the step the network runs warp-wide on BF16 tensor cores
// (mma.sync m16n8k8 / m16n8k16, FP32 accumulation).  A warp's 32 nodes form
// two 16-row tiles: layer 1 is 4 N-tiles of K = 8 (6 inputs, zero padded),
// layer 2 is 4 N-tiles x 2 K-tiles, layer 3 one N-tile (output in column 0)
// x 2 K-tiles.  Each layer's A fragments are the previous layer's
// accumulators in place (the m16n8 accumulator layout is the A layout of the
// next K-tile), so activations never leave registers.  Numerics, BF16
// inference with FP32 accumulation:
//   x_b = bf16(x);  z1 = W1 x_b + b1 (FP32);  a1 = silu_b(z1);
//   z2 = W2 a1 + b2 (FP32);  a2 = silu_b(z2);  y = W3 a2 + b3 (FP32),
//   silu_b(z) = bf16(h + h tanh(h)) with h = bf16(z / 2) and the hardware
// tanh in BF16x2 (tanh.approx.bf16x2, within one BF16 step of tanh); the
// 1/2 is folded into W1, b1, W2, b2 (exact in BF16).  In the negative tail
// h + h tanh(h) cancels, so there the absolute error is ~|h| 2^-8.
// Fragment layouts: PTX ISA, "Matrix fragments for mma.m16n8k8 /
// mma.m16n8k16" (.bf16), g = lane / 4, c = lane % 4.

// The closure's scalars, passed to the step kernel as launch parameters
// (constant bank): normalisation x = raw * scale + shift with scale =
// 1/std, shift = -mean/std, the normalised training range [lo, hi], the
// output bias and scale, and the number of fixed-point passes.
struct MlpConsts {
  float scale[MLP_IN], shift[MLP_IN], lo[MLP_IN], hi[MLP_IN];
  float b3, target_scale;
  int iterations;
};

// The weights in fragment order, stored [field][lane] so that each field is
// one coalesced 128-bit load per warp.  "pair" = two BF16 values, lower
// column in the low half.
struct MlpStep {
  uint4 w1[32];      // layer 1 B fragments, N-tile j = 0..3: W1[8j+g][2c], W1[8j+g][2c+1] (halved)
  uint4 w2[4][32];   // layer 2, N-tile j: (K-tile 0 reg 0, reg 1, K-tile 1 reg 0, reg 1),
                     //   reg r of K-tile kt: W2[8j+g][16kt+8r+2c], W2[8j+g][16kt+8r+2c+1] (halved)
  uint4 w3[32];      // layer 3 (output column 0): same order, W3[16kt+8r+2c], W3[16kt+8r+2c+1]
                     //   where g == 0, zero elsewhere
  uint4 b1[32];      // pairs b1[8j+2c], b1[8j+2c+1] for j = 0..3 (halved)
  uint4 b2[32];      // the same for b2
};

// Host: the in-step form of a network (weights as BF16 bit patterns).
void mlp_step_layout(const MlpClosure &c, int iterations, MlpStep &s, MlpConsts &k);

__device__ __forceinline__ unsigned bf16x2_bits(__nv_bfloat162 v) {
  return *reinterpret_cast<const unsigned *>(&v);
}
__device__ __forceinline__ unsigned u4_get(const uint4 &v, int j) {
  return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w;
}
__device__ __forceinline__ float bf16_lo(unsigned w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(unsigned w) { return __uint_as_float(w & 0xffff0000u); }

// d = A B + C for one m16n8k8 / m16n8k16 tile, C given per column pair
// (the _c forms) or accumulated in place.
__device__ __forceinline__ void mma_bf16_k8(float (&d)[4], unsigned a0, unsigned a1, unsigned b0, float c0,
                                            float c1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%7,%8,%9,%10};"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(a0), "r"(a1), "r"(b0), "f"(c0), "f"(c1), "f"(c0), "f"(c1));
}
__device__ __forceinline__ void mma_bf16_k16_c(float (&d)[4], const unsigned (&a)[4], unsigned b0,
                                               unsigned b1, float c0, float c1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%10,%11,%12,%13};"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1), "f"(c0), "f"(c1), "f"(c0), "f"(c1));
}
__device__ __forceinline__ void mma_bf16_k16(float (&d)[4], const unsigned (&a)[4], unsigned b0,
                                             unsigned b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// A weight fragment, loaded where it is used: the asm is volatile so that
// the compiler neither hoists the load out of the fixed-point loop nor keeps
// the fragment live between the two tiles (all fragments together are 32
// registers; they come back from L1).
__device__ __forceinline__ uint4 ldg_frag(const uint4 *p) {
  uint4 v;
  asm volatile("ld.global.nc.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

// silu_b of two halved pre-activations (h = z / 2): h + h tanh(h) in BF16x2.
__device__ __forceinline__ unsigned silu_half_bf16x2(float h0, float h1) {
  const unsigned h = bf16x2_bits(__floats2bfloat162_rn(h0, h1));
  unsigned t, r;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(h));
  asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(r) : "r"(h), "r"(t));
  return r;
}

// Network output without the output bias b3 (and before target_scale) for
// the calling lane's normalised inputs.  Warp-wide: all 32 lanes call it
// together; `stage` is this warp's 128 words of shared memory.  The two
// 16-node tiles go through the whole network one after the other, so only
// one tile's activations are live at a time (the step kernel keeps its
// node state in registers meanwhile); the weight fragments of the second
// tile are re-read from L1.
__device__ __forceinline__ float mlp_forward_warp(const MlpStep *__restrict__ cl,
                                                  const float (&x)[MLP_IN], unsigned *stage) {
  const int lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
  __syncwarp();
  // Row `lane` of the input tile: pairs (x0 x1)(x2 x3)(x4 x5)(0 0).
  uint4 r4;
  r4.x = bf16x2_bits(__floats2bfloat162_rn(x[0], x[1]));
  r4.y = bf16x2_bits(__floats2bfloat162_rn(x[2], x[3]));
  r4.z = bf16x2_bits(__floats2bfloat162_rn(x[4], x[5]));
  r4.w = 0u;
  reinterpret_cast<uint4 *>(stage)[lane] = r4;
  __syncwarp();
  float out[4];  // entry 2t + h: tile t, row g + 8h
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const unsigned xa0 = stage[(16 * t + g) * 4 + c], xa1 = stage[(16 * t + 8 + g) * 4 + c];
    // Layer 1 -> silu_b -> layer 2's A fragments [K-tile][reg].
    unsigned a1[2][4];
    {
      const uint4 w1 = ldg_frag(&cl->w1[lane]), b1 = ldg_frag(&cl->b1[lane]);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const unsigned wj = u4_get(w1, j), bj = u4_get(b1, j);
        const int kt = j >> 1, r = (j & 1) * 2;  // N-tile j feeds K-tile j/2, regs r, r + 1
        float d[4];
        mma_bf16_k8(d, xa0, xa1, wj, bf16_lo(bj), bf16_hi(bj));
        a1[kt][r] = silu_half_bf16x2(d[0], d[1]);
        a1[kt][r + 1] = silu_half_bf16x2(d[2], d[3]);
      }
    }
    // Layer 2 -> silu_b -> layer 3's A fragments.
    unsigned a2[2][4];
    {
      const uint4 b2 = ldg_frag(&cl->b2[lane]);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const uint4 w2 = ldg_frag(&cl->w2[j][lane]);
        const unsigned bj = u4_get(b2, j);
        const int kt = j >> 1, r = (j & 1) * 2;
        float d[4];
        mma_bf16_k16_c(d, a1[0], w2.x, w2.y, bf16_lo(bj), bf16_hi(bj));
        mma_bf16_k16(d, a1[1], w2.z, w2.w);
        a2[kt][r] = silu_half_bf16x2(d[0], d[1]);
        a2[kt][r + 1] = silu_half_bf16x2(d[2], d[3]);
      }
    }
    // Layer 3: column 0 of the accumulator is the output; lanes with c == 0
    // hold rows g (d[0]) and g + 8 (d[2]).
    const uint4 w3 = ldg_frag(&cl->w3[lane]);
    float d[4];
    mma_bf16_k16_c(d, a2[0], w3.x, w3.y, 0.f, 0.f);
    mma_bf16_k16(d, a2[1], w3.z, w3.w);
    out[2 * t] = d[0];
    out[2 * t + 1] = d[2];
  }
  // Node m = 16t + 8h + g' is row g' + 8h of tile t: lane 4g', entry m / 8.
  const int src = 4 * (lane & 7), k = lane >> 3;
  float y = 0.f;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const float v = __shfl_sync(0xffffffffu, out[q], src);
    if (q == k) y = v;
  }
  return y;
}

}  // namespace lbmc
