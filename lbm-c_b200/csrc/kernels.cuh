// Step kernels of the engine: one fused kernel per (lattice, storage,
// collision family, forcing, diagnostics, streaming layout) performs, for
// every node, the reference's whole time step (LBM-C/solver.cu:10-136):
//
//   load f_i from its in-place shift slot (x - t e_i) mod L  (solver.cu:75-102)
//   rho, u                                                   (solver.cu:96-108)
//   macro BC, micro BC                                       (solver.cu:111-112)
//   collision or bounceback                                  (solver.cu:56-72,115)
//   write f_i back to the same slot                          (solver.cu:120-123)
//   optional rho/u store and FP64 diagnostic partial sums    (solver.cu:126-134,
//                                                             index.cu:338-373)
//
// Besides the reference's shift layout, the same step runs over the AA
// pattern (one array, even and odd index maps), plain or cut into 64-node
// tiles (see STREAM_* below); every layout holds the same state after every
// step, only the places of the values differ.
//
// Populations are held as deviations g_i = f_i - w_i in every storage format
// (FP64, FP32, FP16, BF16; stored value = g_i * scale).  All formulas below are
// the reference's with f_i = w_i + g_i substituted; since the Zou-He and
// bounceback pairings only combine populations of equal weight, those carry
// over verbatim, and rho = 1 + sum g, j = sum e g.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include <cmath>
#include <type_traits>
#include <utility>

#include "lattice.cuh"
#include "mlp.cuh"

namespace lbmc {

// Calls f(std::integral_constant<int, 0>) ... f(<N-1>): the index is a
// constant expression inside f, so lattice tables fold at compile time
// regardless of the optimiser's unrolling decisions.
template <class F, int... Is>
__device__ __forceinline__ void unroll_impl(F &&f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void unroll(F &&f) {
  unroll_impl(f, std::make_integer_sequence<int, N>{});
}

// ------------------------------------------------------------------ storage

template <class S>
struct Storage;

// Storage formats.  put() writes a population to global memory with the
// streaming (evict-first) cache hint: every slot is written once per step and
// next read one step later, after the whole population set has streamed
// through the 126 MB L2.  put_any() is a plain store for pointers that may be
// in shared memory (the bulk-copy pipeline's stages); the .cs hint is a
// global-space instruction and must never see a shared-memory address.
template <>
struct Storage<double> {
  using C = double;
  static constexpr bool SCALED = false;
  static __device__ __forceinline__ C get(const double *p) { return *p; }
  static __device__ __forceinline__ void put(double *p, C v) { __stcs(p, v); }
  static __device__ __forceinline__ void put_any(double *p, C v) { *p = v; }
};
template <>
struct Storage<float> {
  using C = float;
  static constexpr bool SCALED = false;
  static __device__ __forceinline__ C get(const float *p) { return *p; }
  static __device__ __forceinline__ void put(float *p, C v) { __stcs(p, v); }
  static __device__ __forceinline__ void put_any(float *p, C v) { *p = v; }
};
// FP16 keeps (f - w) * scale so that small deviations stay out of the
// subnormal range; BF16 has FP32's exponent range and needs no scale.
template <>
struct Storage<__half> {
  using C = float;
  static constexpr bool SCALED = true;
  static __device__ __forceinline__ C get(const __half *p) { return __half2float(*p); }
  static __device__ __forceinline__ void put(__half *p, C v) { __stcs(p, __float2half_rn(v)); }
  static __device__ __forceinline__ void put_any(__half *p, C v) { *p = __float2half_rn(v); }
};
// FP16 written with stochastic rounding (LBMC_F16_SR): the same 2-byte
// format and scale as __half, so loads are identical; the step kernels write
// their results through store_node_sr below, which rounds each value up
// with probability equal to its distance from the FP16 value below it
// (relative to the FP16 spacing there), so the rounding error has zero
// mean.  Round-to-nearest FP16 storage loses the slow flow's velocity
// signal to a rounding bias that accumulates step after step; stochastic
// rounding turns it into noise that averages out.  Single stores (initial
// upload, shared-memory copies) round to nearest.
struct __align__(2) half_sr {
  unsigned short bits;
};
template <>
struct Storage<half_sr> {
  using C = float;
  static constexpr bool SCALED = true;
  static __device__ __forceinline__ C get(const half_sr *p) { return __half2float(__ushort_as_half(p->bits)); }
  static __device__ __forceinline__ void put(half_sr *p, C v) {
    __stcs(reinterpret_cast<unsigned short *>(p), __half_as_ushort(__float2half_rn(v)));
  }
  static __device__ __forceinline__ void put_any(half_sr *p, C v) { p->bits = __half_as_ushort(__float2half_rn(v)); }
};
template <class S>
__host__ __device__ constexpr bool stochastic_storage() {
  return std::is_same<S, half_sr>::value;
}
template <>
struct Storage<__nv_bfloat16> {
  using C = float;
  static constexpr bool SCALED = false;
  static __device__ __forceinline__ C get(const __nv_bfloat16 *p) { return __bfloat162float(*p); }
  static __device__ __forceinline__ void put(__nv_bfloat16 *p, C v) { __stcs(p, __float2bfloat16_rn(v)); }
  static __device__ __forceinline__ void put_any(__nv_bfloat16 *p, C v) { *p = __float2bfloat16_rn(v); }
};

// FP16 storage scales are powers of two whose inverse is a normal FP16
// value, so a stored value times the inverse scale is exact in FP32 and
// the load below can fuse the conversion and the scaling.
inline bool f16_scale_ok(double scale) {
  int e = 0;
  const double m = std::frexp(scale, &e);  // scale = m 2^e, m in [0.5, 1)
  return m == 0.5 && scale >= 0x1p-15 && scale <= 0x1p14;
}

// Stored-value conversions with the storage scale applied only where the
// format uses one.  FP16: one mixed-precision FMA, h * (1/scale) + (-0)
// (the -0 addend keeps every product, signed zeros included, unchanged),
// equal bit for bit to converting and then multiplying.
template <class S>
__device__ __forceinline__ typename Storage<S>::C load_dev(const S *p, typename Storage<S>::C inv_scale) {
  if constexpr (std::is_same<S, __half>::value || std::is_same<S, half_sr>::value) {
    const unsigned short h = *reinterpret_cast<const unsigned short *>(p);
    const unsigned short s = __half_as_ushort(__float2half_rn(inv_scale));
    float d;
    asm("fma.rn.f32.f16 %0, %1, %2, %3;" : "=f"(d) : "h"(h), "h"(s), "f"(-0.0f));
    return d;
  } else if constexpr (Storage<S>::SCALED) {
    return Storage<S>::get(p) * inv_scale;
  } else {
    return Storage<S>::get(p);
  }
}
// Global-memory population store (streaming hint).
template <class S>
__device__ __forceinline__ void store_dev(S *p, typename Storage<S>::C v, typename Storage<S>::C scale) {
  if constexpr (Storage<S>::SCALED) Storage<S>::put(p, v * scale);
  else Storage<S>::put(p, v);
}
// Shared-memory (or generic) population store, no cache hint.
template <class S>
__device__ __forceinline__ void store_smem(S *p, typename Storage<S>::C v, typename Storage<S>::C scale) {
  if constexpr (Storage<S>::SCALED) Storage<S>::put_any(p, v * scale);
  else Storage<S>::put_any(p, v);
}

// ------------------------------------------------ stochastic rounding bits

// 32-bit integer finaliser (xor-shift and multiply rounds with the
// "lowbias32" constants of C. Wellons' hash-prospector search): every input
// bit affects every output bit.
__host__ __device__ __forceinline__ unsigned mix32(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
// Per-step seed of the stochastic rounding (the step counter t, 64-bit).
__host__ __device__ __forceinline__ unsigned sr_step_seed(long long t) {
  return mix32((unsigned)t ^ mix32((unsigned)((unsigned long long)t >> 32) + 0x9e3779b9u));
}
// Odd multipliers that turn one hashed word h into further random words
// w_k = lo(h m_k) xor hi(h m_k) of the 64-bit product ("multiply-mix": the
// xor folds the well-mixed upper half into the lower one).  The upper half
// alone is not uniform in its top bits when m_k is well below 2^32, and the
// lower half alone ties the low bits of every word to the low bits of h.
__host__ __device__ constexpr unsigned sr_multiplier(int k) {
  return k == 1 ? 0x9e3779b1u : k == 2 ? 0x85ebca77u : k == 3 ? 0xc2b2ae3du : k == 4 ? 0x27d4eb2fu
       : k == 5 ? 0x165667b1u : k == 6 ? 0xd3a2646du : 0xfd7046c5u;
}

// cvt.rs.f16x2.f32: hi goes to the upper, lo to the lower half of the
// result; the low 13 bits of each 16-bit half of rbits are the random bits
// that round the value of that half (measured on the B200: a value rounds
// up when those bits plus its 13 dropped mantissa bits reach 2^13).
__device__ __forceinline__ unsigned cvt_rs_f16x2(float hi, float lo, unsigned rbits) {
  unsigned d;
  asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
  return d;
}

__host__ __device__ __forceinline__ unsigned sr_word(unsigned h, int k) {
  const unsigned long long p = (unsigned long long)h * sr_multiplier(k);
  return (unsigned)p ^ (unsigned)(p >> 32);
}

// Writes a node's Q post-collision values with stochastic rounding, two per
// conversion: population pair (2k, 2k+1) takes random word k, word 0 being
// h = mix32(node ^ step seed) and word k > 0 sr_word(h, k).
// The bits depend only on (node, step, population), so every streaming
// layout writes the same values.  ptr(ic) is the destination of population
// ic; GLOBAL selects the streaming-hint global store (else a plain store,
// for shared memory).
template <int Q, bool GLOBAL, class Ptr>
__device__ __forceinline__ void store_node_sr(const float (&out)[Q], float scale, unsigned key, Ptr &&ptr) {
  const unsigned h = mix32(key);
  auto put16 = [](half_sr *p, unsigned short v) {
    if constexpr (GLOBAL) __stcs(reinterpret_cast<unsigned short *>(p), v);
    else p->bits = v;
  };
  unroll<(Q + 1) / 2>([&](auto pc) {
    constexpr int k = decltype(pc)::value;
    constexpr int i0 = 2 * k, i1 = 2 * k + 1;
    const unsigned r = k == 0 ? h : sr_word(h, k);
    // the pair's scale multiply as one packed FP32x2 multiply (same roundings)
    float o1 = 0.0f;
    if constexpr (i1 < Q) o1 = out[i1];
    const float2 v = __fmul2_rn(make_float2(out[i0], o1), make_float2(scale, scale));
    const unsigned d = cvt_rs_f16x2(v.y, v.x, r);
    put16(ptr(std::integral_constant<int, i0>{}), (unsigned short)(d & 0xffffu));
    if constexpr (i1 < Q) put16(ptr(std::integral_constant<int, i1>{}), (unsigned short)(d >> 16));
  });
}

// Writes a node's Q post-collision values to FP16 storage rounded to
// nearest, two per conversion: the scale multiply of a population pair is
// one packed FP32x2 multiply (mul.rn.f32x2) and the pair converts with one
// cvt.rn.f16x2.f32.  Every value is rounded exactly as the one-value path
// rounds it (v * scale, then to nearest FP16); only the instruction count
// differs.
template <int Q, class Ptr>
__device__ __forceinline__ void store_node_f16(const float (&out)[Q], float scale, Ptr &&ptr) {
  unroll<(Q + 1) / 2>([&](auto pc) {
    constexpr int k = decltype(pc)::value;
    constexpr int i0 = 2 * k, i1 = 2 * k + 1;
    auto put16 = [](auto *p, unsigned short v) { __stcs(reinterpret_cast<unsigned short *>(p), v); };
    if constexpr (i1 < Q) {
      const float2 v = __fmul2_rn(make_float2(out[i0], out[i1]), make_float2(scale, scale));
      const __half2 h = __floats2half2_rn(v.x, v.y);
      put16(ptr(std::integral_constant<int, i0>{}), __half_as_ushort(__low2half(h)));
      put16(ptr(std::integral_constant<int, i1>{}), __half_as_ushort(__high2half(h)));
    } else {
      put16(ptr(std::integral_constant<int, i0>{}), __half_as_ushort(__float2half_rn(out[i0] * scale)));
    }
  });
}

// ------------------------------------------------------------ node classes

// Per-node class byte: 0 plain fluid, 1 solid (B >= 1, full-way
// bounceback), >= 2 index into the class table below.
constexpr int CLASS_FLUID = 0;
constexpr int CLASS_SOLID = 1;
// Class-table entry bits.
constexpr unsigned ENTRY_MACRO_MASK = 0x000Fu;  // MacroBC code 0..15
constexpr unsigned ENTRY_MICRO_SHIFT = 4;       // MicroBC code 0..12
constexpr unsigned ENTRY_MICRO_MASK = 0x00F0u;
constexpr unsigned ENTRY_PARTIAL = 0x0100u;  // 0 < B < 1 with NTPOR/MRTPOR

// Compatibility bits (values of LBMC_COMPAT_* in include/lbmc.h).
constexpr unsigned COMPAT_D3Q15_MINV_ZERO = 1u << 0;
constexpr unsigned COMPAT_MEQ_INT_DIV = 1u << 1;
constexpr unsigned COMPAT_ZH_Z_UX = 1u << 2;
constexpr unsigned COMPAT_MRTPOR_INPLACE = 1u << 3;

// Collision families (template parameter).
constexpr int COL_BGK = 0;
constexpr int COL_BGK_SMAG = 1;
constexpr int COL_MRT = 2;
constexpr int COL_MRT_NC = 3;  // MRT whose rates on rho and j are zero
constexpr int COL_BGK_MLP = 4; // BGK family with the learned closure (Smagorinsky fallback)
constexpr int COL_BGK_MLP1 = 5; // the same with exactly one fixed-point pass (no pass loop to carry)
__host__ __device__ constexpr bool learned_closure(int col) { return col == COL_BGK_MLP || col == COL_BGK_MLP1; }

// rho and the momentum components (the conserved moments).
template <class L>
__host__ __device__ constexpr bool moment_conserved(int k) {
  return k == 0 || k == 3 || k == 5 || (L::Q == 15 && k == 7);
}

constexpr int DIAG_VALUES = 5;  // mass, momentum x/y/z, kinetic energy
// Two-stage reduction of the per-block diagnostic partials.
constexpr int FINALIZE_BLOCKS = 256;
constexpr int FINALIZE_THREADS = 640;  // 20 warps, a multiple of DIAG_VALUES
static_assert(FINALIZE_THREADS % DIAG_VALUES == 0, "a thread must meet one diagnostic value");
constexpr int STEP_BLOCK = 256;  // largest block of any step kernel
// Direct-load kernel: 64-thread blocks and a register cap that keeps 20 of
// them (40 warps) resident per SM; measured on B200 to beat 128/256-thread
// blocks and uncapped registers on the porous D3Q15 workload.
constexpr int DIRECT_BLOCK = 64;
constexpr int DIRECT_MIN_BLOCKS = 20;
constexpr int DIRECT_MIN_BLOCKS_SMAG = 16;  // the Smagorinsky stress needs more registers

template <class C>
struct StepArgs {
  void *f;                // population storage base
  long long pitch;        // elements between population arrays
  const uint8_t *cls;     // node class per node
  const C *B;             // Porosity per node (read at partial nodes only)
  const C *force[3];      // per-node force, or all null for a uniform force
  C force_u[3];           // uniform force
  C *rho;                 // rho - 1: prescribed input and stored output
  C *u[3];                // velocity: prescribed input and stored output
  const C *sf_buf;        // stress-free neighbour populations, Q per sf node
  const int *sf_index;    // node -> row of sf_buf
  double *diag_partials;  // DIAG_VALUES per block
  unsigned *diag_flag;    // bit 0: a non-finite rho/u was seen
  int L[3];
  int s[3];  // shift of the current step: t mod L (AA: t mod 2, wrapped by L)
  int aa;    // AA-pattern layout (lbmc_streaming)
  int tiled; // AA over 64-node tiles (Lx a multiple of 64)
  int odd;   // AA: the current step is odd
  int n;
  C tau;
  C omega;    // 1/tau
  // Guo source terms of the batched domains' uniform force F, per population
  // i, with pre = 1 - 1/(2 tau): guo_a = 9 w_i pre (e_i.F), guo_b = 3 w_i pre,
  // guo_odd = 3 w_i pre (e_i.F); the even part is guo_a (e_i.u) - guo_b (u.F)
  // (collide_fluid with GUO_UNIFORM).
  C guo_a[15], guo_b[15], guo_odd[15];
  C s_mrt[15];
  C c_smag;
  C scale, inv_scale;
  unsigned compat;
  int store;
  unsigned *error_flag;         // bit 0: a bounded device wait expired
  long long timeout_cycles;     // limit of every device-side wait
  long long rows;               // Ly * Lz (pipelined kernel)
  int stages;                   // shared-memory stages (pipelined kernel)
  const uint16_t *table;        // 256 class-table entries (device memory)
  const MlpStep *closure;       // learned closure (COL_BGK_MLP, COL_BGK_MLP1): weights
  MlpConsts mlp;                // and its scalars
  unsigned sr_seed;             // stochastic-rounding seed of this step (sr_step_seed(t))
};

constexpr unsigned ERROR_TIMEOUT = 1u;

// Fills the uniform-force Guo terms of StepArgs (host side).
template <class L, class C>
void set_uniform_guo(C (&ga)[15], C (&gb)[15], C (&godd)[15], double tau, const double *force) {
  const double pre = 1.0 - 1.0 / (2.0 * tau);
  for (int i = 0; i < 15; i++) {
    ga[i] = gb[i] = godd[i] = C(0);
    if (i >= L::Q) continue;
    double eF = 0;
    for (int d = 0; d < L::DIM; d++) eF += L::e(d, i) * force[d];
    const double w = (double)L::wn(i) / (double)L::wd;
    ga[i] = (C)(9.0 * w * pre * eF);
    gb[i] = (C)(3.0 * w * pre);
    godd[i] = (C)(3.0 * w * pre * eF);
  }
}

// ----------------------------------------------------------- index helpers

// Loop unrolling in functions that the host-side layout check compiles too.
#ifdef __CUDA_ARCH__
#define LBMC_UNROLL _Pragma("unroll")
#else
#define LBMC_UNROLL
#endif

__host__ __device__ __forceinline__ int wrap_sub(int x, int s, int L) {
  const int v = x - s;
  return v < 0 ? v + L : v;
}
__host__ __device__ __forceinline__ int wrap_add(int x, int s, int L) {
  const int v = x + s;
  return v >= L ? v - L : v;
}

__host__ __device__ constexpr int sel(int e) { return e == 0 ? 0 : (e > 0 ? 1 : 2); }

// Shift-streaming sites of one node: population i of node (x, y, z) at step
// t lives in slot ((x - t e_x) mod Lx) + Lx ((y - t e_y) mod Ly + Ly (...))
// (LBM-C/solver.cu:82-94).  Index [1] of a component is e = +1 (reads
// x - s), [2] is e = -1 (reads x + s).  The kernels launch one block row per
// (y, z), so the row offsets are uniform across the block.
// Slots are unsigned 32-bit element offsets within one population array, so
// each access is one 32x32+64 multiply-add on the population's base pointer.
struct Sites {
  unsigned x[3];
  unsigned row[3][3];  // [sel(e_y)][sel(e_z)] -> Lx * (y' + Ly * z')
  __host__ __device__ __forceinline__ void init(int cx, int cy, int cz, const int *s, const int *L) {
    x[0] = cx;
    x[1] = wrap_sub(cx, s[0], L[0]);
    x[2] = wrap_add(cx, s[0], L[0]);
    const unsigned ys[3] = {(unsigned)cy, (unsigned)wrap_sub(cy, s[1], L[1]),
                            (unsigned)wrap_add(cy, s[1], L[1])};
    const unsigned zs[3] = {(unsigned)cz, (unsigned)wrap_sub(cz, s[2], L[2]),
                            (unsigned)wrap_add(cz, s[2], L[2])};
    const unsigned lx = L[0], ly = L[1];
LBMC_UNROLL
    for (int a = 0; a < 3; a++)
LBMC_UNROLL
      for (int b = 0; b < 3; b++) row[a][b] = lx * (ys[a] + ly * zs[b]);
  }
  template <class L>
  __host__ __device__ __forceinline__ unsigned slot(int i) const {
    // i is a compile-time constant after unrolling, so sel() folds.
    return x[sel(L::e(0, i))] + row[sel(L::e(1, i))][sel(L::e(2, i))];
  }
};

// Streaming layouts of the direct step kernel.  SHIFT: population i of node
// x at step t sits in slot (i, (x - t e_i) mod L) and the result goes back
// to the same slot.  AA pattern (one array, natural node order, two index
// maps): at an even step population i of node x is read from (i, x) and
// the post-collision value of population i goes to (opp(i), x); at an odd
// step population i is read from (opp(i), x - e_i) and written to
// (i, x + e_i).  In both AA maps out[i] goes to the slot population opp(i)
// was read from, so a node writes exactly the slots it read (in place, no
// race), and the AA-odd read map is the shift map at t = 1 with the arrays
// swapped pairwise.  The state after every step is the same as SHIFT's;
// only where each value sits differs.
//
// Tiled AA (AAT, used when Lx is a multiple of 64): the same two maps over
// a layout cut into 64-node tiles along x, tile k holding its Q population
// arrays back to back: element (array r, slot m) sits at
// ((m / 64) Q + r) 64 + m mod 64.  A 64-thread block of the direct kernel
// is one tile, so at an even step a thread reaches all its values at fixed
// offsets r 64 from one base pointer, and at an odd step a neighbour's value
// is a block-uniform row pointer plus one of three small per-thread x
// offsets; no per-access address arithmetic on the population pitch.
constexpr int STREAM_SHIFT = 0, STREAM_AA_EVEN = 1, STREAM_AA_ODD = 2;
constexpr int STREAM_AAT_EVEN = 3, STREAM_AAT_ODD = 4;
constexpr int TILE = 64;
static_assert(TILE == DIRECT_BLOCK, "a direct-kernel block is one tile of the tiled AA layout");

// Element index of (array r, slot m) in the tiled AA layout.
__host__ __device__ __forceinline__ long long tiled_index(int q, long long m, int r) {
  return ((m / TILE) * q + r) * TILE + m % TILE;
}

// Tiled-AA sites of one node (x, y, z), x = 64 bx + lane: `base` is its own
// element (array 0), x[c] the x part of the index of x' = x, x - s, x + s
// (c = sel(e_x)) and row[a][b] the first element of row (y', z').
struct TiledSites {
  long long base;
  unsigned x[3];
  unsigned row[3][3];
  __host__ __device__ __forceinline__ void init_even(int bx, int lane, int cy, int cz, const int *L, int q) {
    base = ((long long)cy + (long long)L[1] * cz) * (L[0] / TILE) * q * TILE + (long long)bx * q * TILE + lane;
  }
  __host__ __device__ __forceinline__ void init_odd(int bx, int lane, int cy, int cz, const int *s, const int *L,
                                                    int q) {
    const int cx = bx * TILE + lane;
    const int xs[3] = {cx, wrap_sub(cx, s[0], L[0]), wrap_add(cx, s[0], L[0])};
LBMC_UNROLL
    for (int c = 0; c < 3; c++) x[c] = (xs[c] / TILE) * q * TILE + xs[c] % TILE;
    const int ys[3] = {cy, wrap_sub(cy, s[1], L[1]), wrap_add(cy, s[1], L[1])};
    const int zs[3] = {cz, wrap_sub(cz, s[2], L[2]), wrap_add(cz, s[2], L[2])};
    const unsigned rowlen = (unsigned)(L[0] / TILE) * q * TILE;
LBMC_UNROLL
    for (int a = 0; a < 3; a++)
LBMC_UNROLL
      for (int b = 0; b < 3; b++) row[a][b] = ((unsigned)ys[a] + (unsigned)L[1] * zs[b]) * rowlen;
  }
};

// Where the direct kernel reads population I of node n (before collision)
// and where it writes out[I], per layout.  Shared by the kernel and the
// host-side layout check, so both see one definition.
template <class L, int STREAM, int I, class T>
__host__ __device__ __forceinline__ T *read_ptr(T *f, long long pitch, int n, const Sites &st,
                                                const TiledSites &ts) {
  if constexpr (STREAM == STREAM_AA_EVEN) return f + I * pitch + n;
  else if constexpr (STREAM == STREAM_AA_ODD) return f + L::opp(I) * pitch + st.template slot<L>(I);
  else if constexpr (STREAM == STREAM_AAT_EVEN) return f + ts.base + I * TILE;
  else if constexpr (STREAM == STREAM_AAT_ODD)
    return (f + L::opp(I) * TILE) + (ts.row[sel(L::e(1, I))][sel(L::e(2, I))] + ts.x[sel(L::e(0, I))]);
  else return f + I * pitch + st.template slot<L>(I);
}
template <class L, int STREAM, int I, class T>
__host__ __device__ __forceinline__ T *write_ptr(T *f, long long pitch, int n, const Sites &st,
                                                 const TiledSites &ts) {
  if constexpr (STREAM == STREAM_SHIFT) return read_ptr<L, STREAM, I>(f, pitch, n, st, ts);
  else return read_ptr<L, STREAM, L::opp(I)>(f, pitch, n, st, ts);
}

// Array index and slot of population i of a node for the cold kernels
// (stress-free gather, fetch, upload), from the runtime layout flags.
template <class L, int I, class C>
__host__ __device__ __forceinline__ long long natural_slot(const StepArgs<C> &a, const Sites &st) {
  const int arr = (a.aa && a.odd) ? L::opp(I) : I;
  if (a.tiled) return tiled_index(L::Q, st.template slot<L>(I), arr);
  return (long long)arr * a.pitch + st.template slot<L>(I);
}

// -------------------------------------------------------------- physics

template <class L, class C>
struct Node {
  C g[L::Q];  // deviations f - w
  C drho;     // rho - 1
  C rho;
  C u[3];
};

template <class L>
__host__ __device__ constexpr double weight(int i) {
  return (double)L::wn(i) / (double)L::wd;
}

// e_I . v for a compile-time population I.
template <class L, int I, class C>
__device__ __forceinline__ C edot(const C *v) {
  C r = 0;
  if constexpr (L::e(0, I) != 0) r += C(L::e(0, I)) * v[0];
  if constexpr (L::e(1, I) != 0) r += C(L::e(1, I)) * v[1];
  if constexpr (L::DIM > 2 && L::e(2, I) != 0) r += C(L::e(2, I)) * v[2];
  return r;
}

// 1/x for the per-node reciprocals (density, local relaxation time): FP32
// uses the hardware approximation (rcp.approx.ftz.f32, at most 1 ulp from
// the rounded quotient, one instruction instead of the IEEE division's
// sequence); FP64 divides exactly.  1/tau for a uniform tau comes from the
// host in StepArgs.
template <class C>
__device__ __forceinline__ C recip(C x) {
  if constexpr (std::is_same<C, float>::value) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
  } else {
    return C(1) / x;
  }
}

// Rounded multiply and fused multiply-add with the fusion spelled out: the
// compiler fuses a multiply and an add of an expression or not depending on
// the code around it, so an expression that several kernels inline
// (different streaming layouts, the two step kernels) is written with these
// where both forms are possible, and every kernel computes the same bits.
template <class C>
__device__ __forceinline__ C mul_rn(C x, C y) {
  if constexpr (std::is_same<C, float>::value) return __fmul_rn(x, y);
  else return __dmul_rn(x, y);
}
template <class C>
__device__ __forceinline__ C fma_rn(C x, C y, C z) {
  if constexpr (std::is_same<C, float>::value) return __fmaf_rn(x, y, z);
  else return __fma_rn(x, y, z);
}

// rho = 1 + sum g, u = sum e g / rho (LBM-C/solver.cu:96-108).
template <class L, class C>
__device__ __forceinline__ void moments(Node<L, C> &nd) {
  C d = nd.g[0], jx = 0, jy = 0, jz = 0;
  unroll<L::NP>([&](auto pc) {
    constexpr int i = L::pair(decltype(pc)::value);
    constexpr int o = L::opp(i);
    const C sum = nd.g[i] + nd.g[o], dif = nd.g[i] - nd.g[o];
    d += sum;
    if constexpr (L::e(0, i) != 0) jx += C(L::e(0, i)) * dif;
    if constexpr (L::e(1, i) != 0) jy += C(L::e(1, i)) * dif;
    if constexpr (L::DIM > 2 && L::e(2, i) != 0) jz += C(L::e(2, i)) * dif;
  });
  nd.drho = d;
  nd.rho = C(1) + d;
  const C inv = recip(nd.rho);
  nd.u[0] = jx * inv;
  nd.u[1] = jy * inv;
  nd.u[2] = L::DIM > 2 ? jz * inv : C(0);
}

// macro_conditions[code - 1] (LBM-C/boundary_conditions/macro_bc.cu:12-125):
// bit 0 u_x, bit 1 u_y, bit 2 u_z, bit 3 rho, in the table's code order.
// The 16 four-bit masks are packed into one constant (code 0 in the low
// nibble) so a runtime code needs no table in memory.
__host__ __device__ constexpr unsigned macro_mask(int code) {
  return (unsigned)((0xFEDBCA9876534210ull >> (4 * code)) & 0xFull);
}

template <class L, class C>
__device__ __forceinline__ void apply_macro(Node<L, C> &nd, int code, const StepArgs<C> &a, int n) {
  const unsigned m = macro_mask(code);
  if (m & 0x8) {
    nd.drho = a.rho[n];
    nd.rho = C(1) + nd.drho;
  }
  if (m & 0x1) nd.u[0] = a.u[0][n];
  if (m & 0x2) nd.u[1] = a.u[1][n];
  if (L::DIM > 2 && (m & 0x4)) nd.u[2] = a.u[2][n];
}

// Zou-He pressure edges, D2Q9 (LBM-C/boundary_conditions/d2q9/d2q9_zh_defs.cu).
// The known populations of a face carry total weight 1, so the reference's
// 1 - (sum f)/rho becomes (drho - sum g)/rho.
template <class C>
__device__ __forceinline__ void zou_he(Node<D2Q9, C> &nd, int code, unsigned) {
  C *g = nd.g;
  const C r = nd.rho;
  if (code == 1) {
    const C G = g[0] + g[2] + g[4] + C(2) * (g[3] + g[6] + g[7]);
    nd.u[0] = (nd.drho - G) / r;
    nd.u[1] = 0;
    const C ru = r * nd.u[0];
    g[1] = g[3] + C(2.0 / 3.0) * ru;
    g[5] = g[7] - C(0.5) * (g[2] - g[4]) + C(1.0 / 6.0) * ru;
    g[8] = g[6] + C(0.5) * (g[2] - g[4]) + C(1.0 / 6.0) * ru;
  } else if (code == 2) {
    const C G = g[0] + g[2] + g[4] + C(2) * (g[1] + g[5] + g[8]);
    nd.u[0] = (G - nd.drho) / r;
    nd.u[1] = 0;
    const C ru = r * nd.u[0];
    g[3] = g[1] - C(2.0 / 3.0) * ru;
    g[6] = g[8] - C(0.5) * (g[2] - g[4]) - C(1.0 / 6.0) * ru;
    g[7] = g[5] + C(0.5) * (g[2] - g[4]) - C(1.0 / 6.0) * ru;
  }
}

// Zou-He pressure edges, D3Q15 (LBM-C/boundary_conditions/d3q15/d3q15_zh_defs.cu).
template <class C>
__device__ __forceinline__ void zou_he(Node<D3Q15, C> &nd, int code, unsigned compat) {
  C *g = nd.g;
  const C r = nd.rho;
  const C c23 = C(2.0 / 3.0), c12 = C(1.0 / 12.0), q = C(0.25);
  switch (code) {
    case 1: {  // -x face
      const C G = g[0] + g[3] + g[4] + g[5] + g[6] + C(2) * (g[2] + g[14] + g[10] + g[12] + g[8]);
      nd.u[0] = (nd.drho - G) / r;
      nd.u[1] = 0;
      nd.u[2] = 0;
      const C ru = r * nd.u[0];
      const C a = g[3] - g[4], b = g[5] - g[6];
      g[1] = g[2] + c23 * ru;
      g[7] = g[14] + c12 * ru - q * (-a + b);
      g[11] = g[10] + c12 * ru - q * (-a - b);
      g[9] = g[12] + c12 * ru - q * (a + b);
      g[13] = g[8] + c12 * ru - q * (a - b);
      break;
    }
    case 2: {  // +x face
      const C G = g[0] + g[3] + g[4] + g[5] + g[6] + C(2) * (g[1] + g[7] + g[11] + g[9] + g[13]);
      nd.u[0] = (G - nd.drho) / r;
      nd.u[1] = 0;
      nd.u[2] = 0;
      const C ru = r * nd.u[0];
      const C a = g[3] - g[4], b = g[5] - g[6];
      g[2] = g[1] - c23 * ru;
      g[14] = g[7] - c12 * ru - q * (a - b);
      g[10] = g[11] - c12 * ru - q * (a + b);
      g[12] = g[9] - c12 * ru - q * (-a + b);
      g[8] = g[13] - c12 * ru - q * (-a - b);
      break;
    }
    case 3: {  // -y face
      const C G = g[0] + g[1] + g[2] + g[5] + g[6] + C(2) * (g[4] + g[14] + g[10] + g[9] + g[13]);
      nd.u[0] = 0;
      nd.u[1] = (nd.drho - G) / r;
      nd.u[2] = 0;
      const C ru = r * nd.u[1];
      const C a = g[1] - g[2], b = g[5] - g[6];
      g[3] = g[4] + c23 * ru;
      g[7] = g[14] + c12 * ru - q * (-a + b);
      g[11] = g[10] + c12 * ru - q * (-a - b);
      g[12] = g[9] + c12 * ru - q * (a - b);
      g[8] = g[13] + c12 * ru - q * (a + b);
      break;
    }
    case 4: {  // +y face
      const C G = g[0] + g[1] + g[2] + g[5] + g[6] + C(2) * (g[3] + g[7] + g[11] + g[12] + g[8]);
      nd.u[0] = 0;
      nd.u[1] = (G - nd.drho) / r;
      nd.u[2] = 0;
      const C ru = r * nd.u[1];
      const C a = g[1] - g[2], b = g[5] - g[6];
      g[4] = g[3] - c23 * ru;
      g[14] = g[7] - c12 * ru - q * (a - b);
      g[10] = g[11] - c12 * ru - q * (a + b);
      g[9] = g[12] - c12 * ru - q * (-a + b);
      g[13] = g[8] - c12 * ru - q * (-a - b);
      break;
    }
    case 5: {  // -z face
      const C G = g[0] + g[1] + g[2] + g[3] + g[4] + C(2) * (g[6] + g[14] + g[11] + g[12] + g[13]);
      nd.u[0] = 0;
      nd.u[1] = 0;
      nd.u[2] = (nd.drho - G) / r;
      const C ru = r * nd.u[2];
      const C a = g[1] - g[2], b = g[3] - g[4];
      g[5] = g[6] + c23 * ru;
      g[7] = g[14] + c12 * ru - q * (-a + b);
      g[10] = g[11] + c12 * ru - q * (a - b);
      g[9] = g[12] + c12 * ru - q * (-a - b);
      g[8] = g[13] + c12 * ru - q * (a + b);
      break;
    }
    case 6: {  // +z face
      const C G = g[0] + g[1] + g[2] + g[3] + g[4] + C(2) * (g[5] + g[7] + g[10] + g[9] + g[8]);
      nd.u[0] = 0;
      nd.u[1] = 0;
      nd.u[2] = (G - nd.drho) / r;
      // d3q15_zh_defs.cu:87-91 use u[0] (zero) here; the fix uses u_z.
      const C ru = r * ((compat & COMPAT_ZH_Z_UX) ? nd.u[0] : nd.u[2]);
      const C a = g[1] - g[2], b = g[3] - g[4];
      g[6] = g[5] - c23 * ru;
      g[14] = g[7] - c12 * ru - q * (a - b);
      g[11] = g[10] - c12 * ru - q * (-a + b);
      g[12] = g[9] - c12 * ru - q * (a + b);
      g[13] = g[8] - c12 * ru - q * (-a - b);
      break;
    }
    default:
      break;
  }
}

// Micro BC codes: D2Q9 1-2 Zou-He x/X, 5-8 stress-free x/X/y/Y
// (micro_bc.cuh:7-8); D3Q15 1-6 Zou-He x/X/y/Y/z/Z, 7-12 stress-free
// (micro_bc.cuh:14-15).  Returns the stress-free face (0..5) or -1.
template <class L>
__device__ __forceinline__ int sf_face(int code) {
  if (L::Q == 9) return (code >= 5 && code <= 8) ? code - 5 : -1;
  return (code >= 7 && code <= 12) ? code - 7 : -1;
}
template <class L>
__host__ __device__ constexpr bool sf_unknown(int face, int i) {
  // inward populations of face (axis = face/2; low face -> +1, high -> -1)
  return L::e(face / 2, i) * ((face & 1) ? -1 : 1) > 0;
}

template <class L, class C>
__device__ __forceinline__ void apply_micro(Node<L, C> &nd, int code, const StepArgs<C> &a, int n) {
  const int face = sf_face<L>(code);
  if (face < 0) {
    zou_he(nd, code, a.compat);
    return;
  }
  const C *row = a.sf_buf + (long long)a.sf_index[n] * L::Q;
  unroll<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    bool take = false;
    unroll<2 * L::DIM>([&](auto fc) {
      if constexpr (sf_unknown<L>(decltype(fc)::value, i)) take |= (face == decltype(fc)::value);
    });
    if (take) nd.g[i] = row[i];
  });
}

// k-th MRT moment-equilibrium deviation meq_k - (M w)_k
// (LBM-C/collision.cu:465-503), with j = rho u.
template <class L, class C>
__device__ __forceinline__ C meq_dev(int k, const Node<L, C> &nd, unsigned compat) {
  const C jx = nd.rho * nd.u[0], jy = nd.rho * nd.u[1], jz = nd.rho * nd.u[2];
  if (L::Q == 9) {
    const C jj = jx * jx + jy * jy;
    switch (k) {
      case 0: return nd.drho;
      case 1: return C(-2) * nd.drho + C(3) * jj;
      case 2: return nd.drho - C(3) * jj;
      case 3: return jx;
      case 4: return -jx;
      case 5: return jy;
      case 6: return -jy;
      case 7: return jx * jx - jy * jy;
      default: return jx * jy;
    }
  }
  const C jj = jx * jx + jy * jy + jz * jz;
  // collision.cu:492-496 write (-7/3), which C evaluates to -2.
  const C c73 = (compat & COMPAT_MEQ_INT_DIV) ? C(-2) : C(-7.0 / 3.0);
  switch (k) {
    case 0: return nd.drho;
    case 1: return -nd.drho + jj;
    case 2: return nd.drho - C(5) * jj;
    case 3: return jx;
    case 4: return c73 * jx;
    case 5: return jy;
    case 6: return c73 * jy;
    case 7: return jz;
    case 8: return c73 * jz;
    case 9: return C(2) * jx * jx - (jy * jy + jz * jz);
    case 10: return jy * jy - jz * jz;
    case 11: return jx * jy;
    case 12: return jy * jz;
    case 13: return jx * jz;
    default: return C(0);
  }
}

// D3Q15 MRT relaxation with the moment transforms written as butterflies.
// With S_p = g_i + g_opp(i), D_p = g_i - g_opp(i) for the pairs
// p = 1 (x), 3 (y), 5 (z), 7 (+++), 8 (-++), 9 (+-+), 10 (--+), the rows of
// M (LBM-C/macros.cu:77-95) on the four diagonal pairs are a 4x4 Hadamard
// pattern, so M g and M^T m* each take a few dozen additions instead of the
// ~200 of the dense product.  ms[k] = (s_k / D_k)(m_k - meq_k); NC skips the
// conserved moments (0, 3, 5, 7) whose rates are zero.  acc = M^T ms.
template <class C, bool NC>
__device__ __forceinline__ void mrt_d3q15(const Node<D3Q15, C> &nd, const C *srate, unsigned compat,
                                          C (&acc)[15]) {
  const C *g = nd.g;
  const C S1 = g[1] + g[2], D1 = g[1] - g[2];
  const C S3 = g[3] + g[4], D3 = g[3] - g[4];
  const C S5 = g[5] + g[6], D5 = g[5] - g[6];
  const C S7 = g[7] + g[14], D7 = g[7] - g[14];
  const C S8 = g[8] + g[13], D8 = g[8] - g[13];
  const C S9 = g[9] + g[12], D9 = g[9] - g[12];
  const C S10 = g[10] + g[11], D10 = g[10] - g[11];
  // forward
  const C Sa = S1 + S3 + S5;
  const C bA = S7 + S8, bB = S7 - S8, bC = S9 + S10, bD = S9 - S10;
  const C Sd = bA + bC, m12 = bA - bC, m13 = bB + bD, m11 = bB - bD;
  const C da = D7 + D8, db = D7 - D8, dc = D9 + D10, dd = D9 - D10;
  const C Zd = da + dc, Yd = da - dc, Xd = db + dd, m14 = db - dd;
  const C m1 = Sd - Sa - C(2) * g[0];
  const C m2 = Sd - C(4) * Sa + C(16) * g[0];
  const C m4 = Xd - C(4) * D1;
  const C m6 = Yd - C(4) * D3;
  const C m8 = Zd - C(4) * D5;
  const C m9 = C(2) * S1 - S3 - S5;
  const C m10 = S3 - S5;
  // relaxed, scaled moment deviations
  const C ms1 = srate[1] * (m1 - meq_dev<D3Q15>(1, nd, compat));
  const C ms2 = srate[2] * (m2 - meq_dev<D3Q15>(2, nd, compat));
  const C ms4 = srate[4] * (m4 - meq_dev<D3Q15>(4, nd, compat));
  const C ms6 = srate[6] * (m6 - meq_dev<D3Q15>(6, nd, compat));
  const C ms8 = srate[8] * (m8 - meq_dev<D3Q15>(8, nd, compat));
  const C ms9 = srate[9] * (m9 - meq_dev<D3Q15>(9, nd, compat));
  const C ms10 = srate[10] * (m10 - meq_dev<D3Q15>(10, nd, compat));
  const C ms11 = srate[11] * (m11 - meq_dev<D3Q15>(11, nd, compat));
  const C ms12 = srate[12] * (m12 - meq_dev<D3Q15>(12, nd, compat));
  const C ms13 = srate[13] * (m13 - meq_dev<D3Q15>(13, nd, compat));
  const C ms14 = srate[14] * (m14 - meq_dev<D3Q15>(14, nd, compat));
  // inverse: acc = M^T ms
  C A0, K, O1, O3, O5, X, Y, Z;
  if constexpr (NC) {
    acc[0] = C(16) * ms2 - C(2) * ms1;
    A0 = -ms1 - C(4) * ms2;
    K = ms1 + ms2;
    O1 = C(-4) * ms4;
    O3 = C(-4) * ms6;
    O5 = C(-4) * ms8;
    X = ms4;
    Y = ms6;
    Z = ms8;
  } else {
    const C m0 = g[0] + Sa + Sd;
    const C m3 = D1 + Xd, m5 = D3 + Yd, m7 = D5 + Zd;
    const C ms0 = srate[0] * (m0 - meq_dev<D3Q15>(0, nd, compat));
    const C ms3 = srate[3] * (m3 - meq_dev<D3Q15>(3, nd, compat));
    const C ms5 = srate[5] * (m5 - meq_dev<D3Q15>(5, nd, compat));
    const C ms7 = srate[7] * (m7 - meq_dev<D3Q15>(7, nd, compat));
    acc[0] = ms0 - C(2) * ms1 + C(16) * ms2;
    A0 = ms0 - ms1 - C(4) * ms2;
    K = ms0 + ms1 + ms2;
    O1 = ms3 - C(4) * ms4;
    O3 = ms5 - C(4) * ms6;
    O5 = ms7 - C(4) * ms8;
    X = ms3 + ms4;
    Y = ms5 + ms6;
    Z = ms7 + ms8;
  }
  const C E1 = A0 + C(2) * ms9;
  const C T = A0 - ms9;
  const C E3 = T + ms10, E5 = T - ms10;
  acc[1] = E1 + O1;
  acc[2] = E1 - O1;
  acc[3] = E3 + O3;
  acc[4] = E3 - O3;
  acc[5] = E5 + O5;
  acc[6] = E5 - O5;
  const C P = ms12 + ms13, R = ms12 - ms13;
  const C Kp = K + ms11, Km = K - ms11;
  const C E7 = Kp + P, E10 = Kp - P, E8 = Km + R, E9 = Km - R;
  const C Zp = Z + ms14, Zm = Z - ms14, XY = X + Y, YX = Y - X;
  const C O7 = Zp + XY, O10 = Zp - XY, O8 = Zm + YX, O9 = Zm - YX;
  acc[7] = E7 + O7;
  acc[14] = E7 - O7;
  acc[8] = E8 + O8;
  acc[13] = E8 - O8;
  acc[9] = E9 + O9;
  acc[12] = E9 - O9;
  acc[10] = E10 + O10;
  acc[11] = E10 - O10;
}

// The fluid-node collision of the reference (collision_functions[2 type +
// forcing], LBM-C/collision.cu:19-421) after the macro/micro BCs
// (LBM-C/solver.cu:111-112), written with opposite-pair symmetry: for a pair
// (i, o = opp(i)), e_o = -e_i and w_o = w_i, so the equilibria, Guo terms
// and the MRT transforms split into even and odd parts computed once per
// pair.  Post-collision deviations go to out[].
// `participate` (learned closure only): false for the lanes that only
// accompany the warp-wide network evaluation (solid or out-of-range nodes).
// GUO_UNIFORM (the batched domains, whose force is always uniform): the
// Guo source from the host's per-population terms guo_a / guo_b / guo_odd.
// The single-domain kernels keep the per-node form, whose arithmetic is the
// same in every instantiation (shift and AA layouts, both step kernels).
template <class L, class C, int COL, bool FORCE, bool BLEND, bool GUO_UNIFORM = false>
__device__ __forceinline__ void collide_fluid(Node<L, C> &nd, const StepArgs<C> &a, int n,
                                              unsigned entry, C (&out)[L::Q], bool participate = true) {
  constexpr int Q = L::Q;
  C B = 0;
  if (entry) {
    const int macro = entry & ENTRY_MACRO_MASK;
    const int micro = (entry & ENTRY_MICRO_MASK) >> ENTRY_MICRO_SHIFT;
    if (macro) apply_macro(nd, macro, a, n);
    if (micro) apply_micro(nd, micro, a, n);
    if (BLEND && (entry & ENTRY_PARTIAL)) B = a.B[n];
  }
  const C tau0 = a.tau;
  C F[3] = {0, 0, 0}, pre = 0, uF = 0;
  if constexpr (FORCE) {
    if (a.force[0]) {
      F[0] = a.force[0][n];
      F[1] = a.force[1][n];
      if (L::DIM > 2) F[2] = a.force[2][n];
    } else {
      F[0] = a.force_u[0];
      F[1] = a.force_u[1];
      F[2] = a.force_u[2];
    }
    // u <- u + F/(2 rho) (collision.cu:74-78)
    const C h = recip(C(2) * nd.rho);
    nd.u[0] += h * F[0];
    nd.u[1] += h * F[1];
    if (L::DIM > 2) nd.u[2] += h * F[2];
    if constexpr (!GUO_UNIFORM) pre = C(1) - recip(C(2) * tau0);
    uF = nd.u[0] * F[0] + nd.u[1] * F[1] + (L::DIM > 2 ? nd.u[2] * F[2] : C(0));
  }
  const C omb = C(1) - B;
  // Guo source (collision.cu:82-99): F_i = w_i pre (3 (e_i.F - u.F) + 9 (e_i.u)(e_i.F)),
  // even part w pre (9 (e.u)(e.F) - 3 u.F), odd part 3 w pre e.F.
  auto guo_parts = [&](auto ic, C &even, C &odd) {
    if constexpr (FORCE && GUO_UNIFORM) {
      constexpr int i = decltype(ic)::value;
      even = fma_rn(a.guo_a[i], edot<L, i>(nd.u), -mul_rn(a.guo_b[i], uF));
      odd = a.guo_odd[i];
    } else if constexpr (FORCE) {
      constexpr int i = decltype(ic)::value;
      const C wp = C(weight<L>(i)) * pre;
      const C eF = edot<L, i>(F), eu = edot<L, i>(nd.u);
      even = wp * (C(9) * eu * eF - C(3) * uF);
      odd = wp * C(3) * eF;
    } else {
      even = 0;
      odd = 0;
    }
  };
  C ft0e, ft0o;
  guo_parts(std::integral_constant<int, 0>{}, ft0e, ft0o);

  if constexpr ((COL == COL_MRT || COL == COL_MRT_NC) && L::Q == 15) {
    // D3Q15 MRT (collision.cu:192-421) through the butterfly transforms.
    C acc[15];
    mrt_d3q15<C, COL == COL_MRT_NC>(nd, a.s_mrt, a.compat, acc);
    if (a.compat & COMPAT_D3Q15_MINV_ZERO) {
      // macros.cu:97-115: the reference's D3Q15 M_inv is all zeros.
      unroll<Q>([&](auto kc) { acc[decltype(kc)::value] = 0; });
    }
    out[0] = nd.g[0] - omb * acc[0] + omb * ft0e;
    const bool inplace = BLEND && (a.compat & COMPAT_MRTPOR_INPLACE);
    unroll<L::NP>([&](auto pc) {
      constexpr int i = L::pair(decltype(pc)::value);
      constexpr int o = L::opp(i);
      C fe, fo_;
      guo_parts(std::integral_constant<int, i>{}, fe, fo_);
      const C ft_i = fe + fo_, ft_o = fe - fo_;
      if constexpr (BLEND) {
        const C oi = nd.g[i] - omb * acc[i] + omb * ft_i + B * (nd.g[o] - nd.g[i]);
        const C partner = inplace ? oi : nd.g[i];
        out[i] = oi;
        out[o] = nd.g[o] - omb * acc[o] + omb * ft_o + B * (partner - nd.g[o]);
      } else {
        out[i] = nd.g[i] - acc[i] + ft_i;
        out[o] = nd.g[o] - acc[o] + ft_o;
      }
    });
  } else if constexpr (COL == COL_MRT || COL == COL_MRT_NC) {
    // m* = S (M g - meq) / D; f <- f - M^T m* (collision.cu:192-303).
    // s_mrt holds s_k / D_k.  COL_MRT_NC drops the moments whose rate is
    // zero (their m* is identically zero).
    C S[L::NP], D[L::NP];
    unroll<L::NP>([&](auto pc) {
      constexpr int p = decltype(pc)::value;
      constexpr int i = L::pair(p);
      S[p] = nd.g[i] + nd.g[L::opp(i)];
      D[p] = nd.g[i] - nd.g[L::opp(i)];
    });
    C ms[Q];
    unroll<Q>([&](auto kc) {
      constexpr int k = decltype(kc)::value;
      constexpr bool even = moment_even<L>(k);
      if constexpr (COL == COL_MRT_NC && moment_conserved<L>(k)) {
        ms[k] = 0;
        return;
      }
      C mk = 0;
      if constexpr (even && L::m(k, 0) != 0) mk = C(L::m(k, 0)) * nd.g[0];
      unroll<L::NP>([&](auto pc) {
        constexpr int p = decltype(pc)::value;
        constexpr int c = L::m(k, L::pair(p));
        const C v = even ? S[p] : D[p];
        if constexpr (c == 1) mk += v;
        else if constexpr (c == -1) mk -= v;
        else if constexpr (c != 0) mk += C(c) * v;
      });
      ms[k] = a.s_mrt[k] * (mk - meq_dev<L>(k, nd, a.compat));
    });
    if (Q == 15 && (a.compat & COMPAT_D3Q15_MINV_ZERO)) {
      // macros.cu:97-115: the reference's D3Q15 M_inv is all zeros.
      unroll<Q>([&](auto kc) { ms[decltype(kc)::value] = 0; });
    }
    // population 0
    {
      C acc = 0;
      unroll<Q>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        constexpr int c = L::m(k, 0);
        if constexpr (c != 0 && !(COL == COL_MRT_NC && moment_conserved<L>(k))) acc += C(c) * ms[k];
      });
      out[0] = nd.g[0] - omb * acc + omb * ft0e;
    }
    const bool inplace = BLEND && (a.compat & COMPAT_MRTPOR_INPLACE);
    unroll<L::NP>([&](auto pc) {
      constexpr int i = L::pair(decltype(pc)::value);
      constexpr int o = L::opp(i);
      C E = 0, O = 0;
      unroll<Q>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        constexpr int c = L::m(k, i);
        if constexpr (c != 0 && !(COL == COL_MRT_NC && moment_conserved<L>(k))) {
          if constexpr (moment_even<L>(k)) {
            if constexpr (c == 1) E += ms[k];
            else if constexpr (c == -1) E -= ms[k];
            else E += C(c) * ms[k];
          } else {
            if constexpr (c == 1) O += ms[k];
            else if constexpr (c == -1) O -= ms[k];
            else O += C(c) * ms[k];
          }
        }
      });
      C fe, fo_;
      guo_parts(std::integral_constant<int, i>{}, fe, fo_);
      const C acc_i = E + O, acc_o = E - O;
      const C ft_i = fe + fo_, ft_o = fe - fo_;
      if constexpr (BLEND) {
        // mrt_ntpor(_guo)_collision (collision.cu:305-421).  The reference
        // loops i upwards and reads f[opp[i]] after the lower index of the
        // pair was updated (collision.cu:340,416); COMPAT_MRTPOR_INPLACE
        // reproduces that.
        const C oi = nd.g[i] - omb * acc_i + omb * ft_i + B * (nd.g[o] - nd.g[i]);
        const C partner = inplace ? oi : nd.g[i];
        out[i] = oi;
        out[o] = nd.g[o] - omb * acc_o + omb * ft_o + B * (partner - nd.g[o]);
      } else {
        out[i] = nd.g[i] - acc_i + ft_i;
        out[o] = nd.g[o] - acc_o + ft_o;
      }
    });
  } else {
    // BGK family (collision.cu:49-190): geq_i = A + Bq, geq_o = A - Bq with
    // A = w (drho + rho (eu^2/2 - usq)), Bq = w rho eu, eu = 3 e_i.u.
    const C usq = C(1.5) * (nd.u[0] * nd.u[0] + nd.u[1] * nd.u[1] + nd.u[2] * nd.u[2]);
    const C A0 = C(weight<L>(0)) * (nd.drho - nd.rho * usq);
    C tau = tau0;
    if constexpr (COL == COL_BGK_SMAG || learned_closure(COL)) {
      // Smagorinsky (collision.cu:445-463, q_bar zeroed): q_ab = sum e_a e_b
      // (f - f_eq) is even in e, so each pair contributes e_a e_b (S - 2A).
      C q[6] = {0, 0, 0, 0, 0, 0};  // xx, yy, zz, xy, yz, xz
      unroll<L::NP>([&](auto pc) {
        constexpr int i = L::pair(decltype(pc)::value);
        const C eu = C(3) * edot<L, i>(nd.u);
        const C A = C(weight<L>(i)) * (nd.drho + nd.rho * (C(0.5) * eu * eu - usq));
        const C neq = nd.g[i] + nd.g[L::opp(i)] - C(2) * A;
        constexpr int ex = L::e(0, i), ey = L::e(1, i), ez = L::e(2, i);
        if constexpr (ex != 0) q[0] += neq;
        if constexpr (ey != 0) q[1] += neq;
        if constexpr (ez != 0) q[2] += neq;
        if constexpr (ex * ey != 0) q[3] += C(ex * ey) * neq;
        if constexpr (ey * ez != 0) q[4] += C(ey * ez) * neq;
        if constexpr (ex * ez != 0) q[5] += C(ex * ez) * neq;
      });
      const C r2 = sqrt(C(2));
      C qhat = r2 * (fabs(q[0]) + fabs(q[1]) + C(2) * fabs(q[3]));
      if (L::DIM > 2) qhat += r2 * (fabs(q[2]) + C(2) * (fabs(q[4]) + fabs(q[5])));
      const C k = C(2) * r2 * a.c_smag * a.c_smag * (C(9) * recip(nd.rho));
      const C tau_smag = tau0 + C(0.5) * (sqrt(fma_rn(k, qhat, mul_rn(tau0, tau0))) - tau0);
      if constexpr (COL == COL_BGK_SMAG) {
        tau = tau_smag;
      } else {
        // Learned closure: strain estimate S = -3 q / (2 rho tau) from the
        // non-equilibrium stress (c_s^2 = 1/3), six invariants, network ->
        // nu_t, tau = tau0 + 3 nu_t; the fixed point starts from the
        // Smagorinsky tau and takes `iterations` passes.  Outside the
        // normalised training range: Smagorinsky.  The network runs
        // warp-wide on the tensor cores, so every lane of the warp takes the
        // same number of passes (non-participating lanes feed zeros).
        __shared__ __align__(16) unsigned mlp_stage[DIRECT_BLOCK / 32][128];
        const MlpStep *cl = a.closure;
        bool in_range = participate;
        C tau_l = tau_smag;
        // One pass for COL_BGK_MLP1 is a compile-time constant: the pass
        // loop and what it carries disappear (128 registers, no spills,
        // against ~163 with the runtime loop).
        const int passes = COL == COL_BGK_MLP1 ? 1 : a.mlp.iterations;
        for (int it = 0; it < passes; it++) {
          const float ks = __fdividef(-1.5f, (float)(nd.rho * tau_l));
          float Sm[6], f[MLP_IN];
#pragma unroll
          for (int c = 0; c < 6; c++) Sm[c] = ks * (float)q[c];
          strain_features(Sm, (float)nd.rho, f);
#pragma unroll
          for (int c = 0; c < MLP_IN; c++) {
            f[c] = fmaf(f[c], a.mlp.scale[c], a.mlp.shift[c]);
            in_range = in_range && f[c] >= a.mlp.lo[c] && f[c] <= a.mlp.hi[c];
          }
#pragma unroll
          for (int c = 0; c < MLP_IN; c++) f[c] = in_range ? f[c] : 0.0f;
          const float y = mlp_forward_warp(cl, f, mlp_stage[threadIdx.x >> 5]) + a.mlp.b3;
          if (in_range) tau_l = tau0 + C(3) * C(fmaxf(0.0f, a.mlp.target_scale * y));
        }
        tau = in_range ? tau_l : tau_smag;
      }
    }
    // 1/tau: the host's value for a uniform tau, else the local one
    const C om = (COL == COL_BGK_SMAG || learned_closure(COL)) ? recip(tau) : a.omega;
    // population 0 (e = 0)
    out[0] = nd.g[0] - omb * (om * (nd.g[0] - A0)) + omb * ft0e;
    unroll<L::NP>([&](auto pc) {
      constexpr int i = L::pair(decltype(pc)::value);
      constexpr int o = L::opp(i);
      const C eu = C(3) * edot<L, i>(nd.u);
      const C w = C(weight<L>(i));
      const C A = w * (nd.drho + nd.rho * (C(0.5) * eu * eu - usq));
      const C Bq = w * nd.rho * eu;
      C fe, fo_;
      guo_parts(std::integral_constant<int, i>{}, fe, fo_);
      const C om_i = om * (nd.g[i] - (A + Bq));
      const C om_o = om * (nd.g[o] - (A - Bq));
      if constexpr (BLEND) {
        // bgk_ntpor(_guo)_collision (collision.cu:113-190)
        out[i] = nd.g[i] - omb * om_i + B * (nd.g[o] - nd.g[i]) + omb * (fe + fo_);
        out[o] = nd.g[o] - omb * om_o + B * (nd.g[i] - nd.g[o]) + omb * (fe - fo_);
      } else {
        out[i] = nd.g[i] - om_i + (fe + fo_);
        out[o] = nd.g[o] - om_o + (fe - fo_);
      }
    });
  }
}

// bounceback (LBM-C/collision.cu:423-443): f_i <- f_opp(i), rho = u = 0.
template <class L, class C>
__device__ __forceinline__ void collide_solid(Node<L, C> &nd, C (&out)[L::Q]) {
  unroll<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    out[i] = nd.g[L::opp(i)];
  });
  nd.drho = C(-1);
  nd.rho = 0;
  nd.u[0] = nd.u[1] = nd.u[2] = 0;
}

template <class L, class C>
__device__ __forceinline__ void store_and_reduce(const Node<L, C> &nd, const StepArgs<C> &a, int n,
                                                 double (&dv)[DIAG_VALUES], bool &nonfinite,
                                                 bool diag) {
  if (a.store) {
    a.rho[n] = nd.drho;
    a.u[0][n] = nd.u[0];
    a.u[1][n] = nd.u[1];
    if (L::DIM > 2) a.u[2][n] = nd.u[2];
  }
  if (diag) {
    const double rho = (double)nd.drho + 1.0;
    const double ux = nd.u[0], uy = nd.u[1], uz = nd.u[2];
    dv[0] += rho;
    dv[1] += rho * ux;
    dv[2] += rho * uy;
    dv[3] += rho * uz;
    dv[4] += 0.5 * rho * (ux * ux + uy * uy + uz * uz);
    nonfinite |= !(isfinite(rho) && isfinite(ux) && isfinite(uy) && isfinite(uz));
  }
}

// ------------------------------------------------------------ diagnostics

// Warp-shuffle + shared-memory block reduction of the FP64 sums; one partial
// per block, summed in a fixed order by the finalize kernels (engine.cu).
template <class C>
__device__ __forceinline__ void block_diag(const double (&v)[DIAG_VALUES], bool nonfinite,
                                           const StepArgs<C> &a, long long block) {
  __shared__ double red[16][DIAG_VALUES];  // up to 512 threads
  double s[DIAG_VALUES];
#pragma unroll
  for (int k = 0; k < DIAG_VALUES; k++) {
    double x = v[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    s[k] = x;
  }
  const unsigned bad = __ballot_sync(0xffffffffu, nonfinite);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < DIAG_VALUES; k++) red[warp][k] = s[k];
    if (bad) atomicOr(a.diag_flag, 1u);
  }
  __syncthreads();
  if (threadIdx.x < DIAG_VALUES) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w][threadIdx.x];
    a.diag_partials[block * DIAG_VALUES + threadIdx.x] = t;
  }
}

// ------------------------------------------------- direct-load step kernel

// Fallback for rows whose byte length is not a multiple of 16 (bulk copies
// need 16-byte granules) or that do not fit the shared-memory stages.
// Grid: blockDim (bx, 1, 1) along x, gridDim (ceil(Lx/bx), Ly, Lz).
template <class S, int COL>
constexpr int direct_min_blocks() {
  // FP64 arithmetic needs register pairs, the learned closure its hidden
  // layer: no cap beyond the 128 per thread that 8 resident blocks imply.
  if (std::is_same<S, double>::value || learned_closure(COL)) return 8;
  return COL == COL_BGK_SMAG ? DIRECT_MIN_BLOCKS_SMAG : DIRECT_MIN_BLOCKS;
}

template <class L, class S, int COL, bool FORCE, bool BLEND, bool DIAG, int STREAM>
__global__ void __launch_bounds__(DIRECT_BLOCK, (direct_min_blocks<S, COL>()))
    step_kernel(const StepArgs<typename Storage<S>::C> a) {
  using C = typename Storage<S>::C;
  constexpr int Q = L::Q;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = x < a.L[0];
  // Read slot of population i: (i, slot(i)) in the shift layout, (i, n) at
  // an AA-even step, (opp(i), slot(i)) with the t = 1 shift at an AA-odd
  // step; out[i] goes back to slot(i) (shift) or to population opp(i)'s
  // read slot (AA).
  auto read_at = [&](S *f, const Sites &st, const TiledSites &ts, int n, auto ic) -> S * {
    return read_ptr<L, STREAM, decltype(ic)::value>(f, a.pitch, n, st, ts);
  };
  auto write_at = [&](S *f, const Sites &st, const TiledSites &ts, int n, auto ic) -> S * {
    return write_ptr<L, STREAM, decltype(ic)::value>(f, a.pitch, n, st, ts);
  };
  // The AA-even map needs only n; the others their sites (one block row per
  // (y, z), so the row parts are uniform across the block).
  // `zero` is 0; a value the compiler cannot see through makes it recompute
  // the sites instead of keeping them live (the learned closure's stores).
  auto init_sites = [&](Sites &st, TiledSites &ts, int zero = 0) {
    if constexpr (STREAM == STREAM_AAT_EVEN)
      ts.init_even(blockIdx.x + zero, threadIdx.x, blockIdx.y, blockIdx.z, a.L, Q);
    else if constexpr (STREAM == STREAM_AAT_ODD)
      ts.init_odd(blockIdx.x + zero, threadIdx.x, blockIdx.y, blockIdx.z, a.s, a.L, Q);
    else if constexpr (STREAM != STREAM_AA_EVEN)
      st.init(x + zero, blockIdx.y, blockIdx.z, a.s, a.L);
  };
  double dv[DIAG_VALUES] = {0, 0, 0, 0, 0};
  bool nonfinite = false;
  if constexpr (!learned_closure(COL)) {
    if (!DIAG && !active) return;
    if (active) {
      const C inv_scale = a.inv_scale, scale = a.scale;
      Sites st;
      TiledSites ts;
      init_sites(st, ts);
      const int n = x + a.L[0] * ((int)blockIdx.y + a.L[1] * (int)blockIdx.z);
      S *f = reinterpret_cast<S *>(a.f);
      Node<L, C> nd;
      unroll<Q>([&](auto ic) { nd.g[decltype(ic)::value] = load_dev(read_at(f, st, ts, n, ic), inv_scale); });
      const int cls = a.cls[n];
      C out[Q];
      if (cls == CLASS_SOLID) {
        collide_solid(nd, out);
      } else {
        moments(nd);
        collide_fluid<L, C, COL, FORCE, BLEND>(nd, a, n, cls ? a.table[cls] : 0u, out);
      }
      // The store addresses equal the load addresses.  Recomputing them
      // from the three 32-bit x offsets is cheaper than keeping Q 64-bit
      // pointers live across the collision, which spills at this kernel's
      // register cap: 88-116 bytes in the tiled odd step (13% slower with
      // FP16/BF16 storage), 20-48 bytes in the shift and plain odd maps.
      // The 2-byte storages, bound by instruction issue, keep the spill in
      // the plain maps (the recomputation measured slower there).  The
      // empty asm hides the equality from the compiler.
      constexpr bool recompute = STREAM == STREAM_AAT_ODD ||
                                 ((STREAM == STREAM_AA_ODD || STREAM == STREAM_SHIFT) && sizeof(S) >= 4);
      auto store_all = [&](const Sites &sw, const TiledSites &tw) {
        if constexpr (stochastic_storage<S>())
          store_node_sr<Q, true>(out, scale, (unsigned)n ^ a.sr_seed,
                                 [&](auto ic) { return write_at(f, sw, tw, n, ic); });
        else if constexpr (std::is_same<S, __half>::value)
          store_node_f16<Q>(out, scale, [&](auto ic) { return write_at(f, sw, tw, n, ic); });
        else
          unroll<Q>([&](auto ic) { store_dev(write_at(f, sw, tw, n, ic), out[decltype(ic)::value], scale); });
      };
      if constexpr (recompute) {
        TiledSites tw = ts;
        Sites sw = st;
        if constexpr (STREAM == STREAM_AAT_ODD) asm("" : "+r"(tw.x[0]), "+r"(tw.x[1]), "+r"(tw.x[2]));
        else asm("" : "+r"(sw.x[0]), "+r"(sw.x[1]), "+r"(sw.x[2]));
        store_all(sw, tw);
      } else {
        store_all(st, ts);
      }
      store_and_reduce(nd, a, n, dv, nonfinite, DIAG);
    }
  } else {
    // The learned closure's network runs warp-wide: every lane of a warp
    // with an active node takes the node path, the others (solid or past the
    // edge) as non-participants that run the fluid update at rest (rho = 1,
    // u = 0, no boundary entry) and then bounce back.
    const bool run = __any_sync(0xffffffffu, active);
    if (!DIAG && !run) return;
    if (run) {
      const C inv_scale = a.inv_scale, scale = a.scale;
      Sites st;
      TiledSites ts;
      const int n = active ? x + a.L[0] * ((int)blockIdx.y + a.L[1] * (int)blockIdx.z) : 0;
      S *f = reinterpret_cast<S *>(a.f);
      Node<L, C> nd;
      if (active) {
        init_sites(st, ts);
        unroll<Q>([&](auto ic) { nd.g[decltype(ic)::value] = load_dev(read_at(f, st, ts, n, ic), inv_scale); });
      } else {
        unroll<Q>([&](auto ic) { nd.g[decltype(ic)::value] = C(0); });
      }
      const int cls = active ? a.cls[n] : CLASS_SOLID;
      const bool fluid = cls != CLASS_SOLID;
      C out[Q];
      if (fluid) {
        moments(nd);
      } else {
        nd.drho = 0;
        nd.rho = 1;
        nd.u[0] = nd.u[1] = nd.u[2] = 0;
      }
      collide_fluid<L, C, COL, FORCE, BLEND>(nd, a, n, fluid && cls ? a.table[cls] : 0u, out, fluid);
      if (!fluid) collide_solid(nd, out);
      if (active) {
        // The store sites equal the load sites; recomputing them is cheaper
        // than keeping them live across the network, which spills.
        Sites sw;
        TiledSites tw;
        int zero = 0;
        asm volatile("" : "+r"(zero));
        init_sites(sw, tw, zero);
        if constexpr (stochastic_storage<S>())
          store_node_sr<Q, true>(out, scale, (unsigned)n ^ a.sr_seed,
                                 [&](auto ic) { return write_at(f, sw, tw, n, ic); });
        else
          unroll<Q>([&](auto ic) { store_dev(write_at(f, sw, tw, n, ic), out[decltype(ic)::value], scale); });
        store_and_reduce(nd, a, n, dv, nonfinite, DIAG);
      }
    }
  }
  if (DIAG)
    block_diag<C>(dv, nonfinite, a,
                  blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z));
}

// -------------------------------------------- bulk-copy pipelined kernel

// Shared-memory staging of whole population rows with cp.async.bulk (the
// TMA engine's 1-D bulk copies) and mbarrier completion.  For the shift
// layout, the nodes of one grid row (y, z) read population i from one whole
// physical row, (y - t e_y, z - t e_z) rotated by t e_x along x, and write
// their results back to the same slots; so a row is: bulk-load Q rows,
// collide every node from shared memory, bulk-store the Q rows.  The
// persistent blocks walk rows r = blockIdx.x, blockIdx.x + gridDim.x, ...
// with `stages` rows in flight, so memory traffic is decoupled from the
// compute of the current row.  No cluster multicast is used.

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after `limit` cycles and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity, long long limit) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return false;
  }
  return true;
}
__device__ __forceinline__ void bulk_load(unsigned dst, const void *src, unsigned bytes, unsigned bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void bulk_store(void *dst, unsigned src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Global address of population i's physical row for grid row (y, z).
template <class L, class S>
__device__ __forceinline__ S *phys_row(S *f, long long pitch, int i, int y, int z, const int *s,
                                       const int *L_) {
  int yy = y, zz = z;
  const int ey = L::e(1, i), ez = L::e(2, i);
  if (ey > 0) yy = wrap_sub(y, s[1], L_[1]);
  if (ey < 0) yy = wrap_add(y, s[1], L_[1]);
  if (ez > 0) zz = wrap_sub(z, s[2], L_[2]);
  if (ez < 0) zz = wrap_add(z, s[2], L_[2]);
  return f + i * pitch + (long long)L_[0] * (yy + (long long)L_[1] * zz);
}

template <class L, class S>
__device__ __forceinline__ void issue_row_load(S *f, long long pitch, long long row, const int *s,
                                               const int *L_, S *stage_buf, unsigned bar) {
  const int y = (int)(row % L_[1]), z = (int)(row / L_[1]);
  const unsigned bytes = (unsigned)(L_[0] * sizeof(S));
  mbar_expect_tx(bar, bytes * L::Q);
#pragma unroll
  for (int i = 0; i < L::Q; i++)
    bulk_load(smem_addr(stage_buf + (long long)i * L_[0]), phys_row<L>(f, pitch, i, y, z, s, L_), bytes,
              bar);
}

template <class L, class S>
__device__ __forceinline__ void issue_row_store(S *f, long long pitch, long long row, const int *s,
                                                const int *L_, S *stage_buf) {
  const int y = (int)(row % L_[1]), z = (int)(row / L_[1]);
  const unsigned bytes = (unsigned)(L_[0] * sizeof(S));
#pragma unroll
  for (int i = 0; i < L::Q; i++)
    bulk_store(phys_row<L>(f, pitch, i, y, z, s, L_), smem_addr(stage_buf + (long long)i * L_[0]), bytes);
  bulk_commit();
}

constexpr int PIPE_MAX_STAGES = 8;
// Launch shape: consumer threads per block and the register cap (resident
// blocks per SM), with 32 KB of stages per block.  Many small blocks, each
// consumer stepping several nodes of a row, beat few large ones: on the
// porous 256^3 step, FP32 28.7 GLUPS (2 blocks of 256 consumers, 96 KB of
// stages) -> 41.0 (4 blocks, 48 KB) -> 46.6 (64 consumers, 7 blocks by
// shared memory); FP16 26.4 -> 37.6 -> 45.7 with 128 consumers (64: 44.2).
// Every shape caps registers at 56 a thread; FP64 keeps its register pairs.
template <class S>
constexpr int pipe_consumers() {
  return sizeof(S) == 2 ? 128 : 64;
}
template <class S>
constexpr int pipe_min_blocks() {
  return std::is_same<S, double>::value ? 1 : (65536 / 56) / (pipe_consumers<S>() + 32);
}

__device__ __forceinline__ void mbar_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Warp-specialised pipeline.  Warp 0 is the producer: its lane 0 issues the
// bulk loads of row k into stage k % stages (completion counted on
// full[stage]), and once the consumer warps have signalled done[stage] it
// bulk-stores the row back and reuses the stage for row k + stages.  Warps
// 1.. are consumers: they wait on full[stage], collide the row's nodes in
// shared memory, fence their writes for the async proxy and arrive on
// done[stage].  Every wait is bounded (timeout_cycles); on expiry the kernel
// records ERROR_TIMEOUT, stops issuing work, drains its own copies with
// bounded waits and returns.
// Dynamic shared memory: [stages][Q][Lx] storage elements.
template <class L, class S, int COL, bool FORCE, bool BLEND, bool DIAG>
__global__ void __launch_bounds__(pipe_consumers<S>() + 32, (pipe_min_blocks<S>()))
    step_pipelined_kernel(const StepArgs<typename Storage<S>::C> a) {
  using C = typename Storage<S>::C;
  constexpr int Q = L::Q;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long full_bar[PIPE_MAX_STAGES];
  __shared__ __align__(8) unsigned long long done_bar[PIPE_MAX_STAGES];
  __shared__ volatile int abort_flag;
  S *buf = reinterpret_cast<S *>(smem_raw);
  const int lx = a.L[0];
  const int nst = a.stages;
  const int stage_elems = Q * lx;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int consumers = (int)(blockDim.x >> 5) - 1;
  const long long rows = a.rows;
  const long long my_rows = rows > blockIdx.x ? (rows - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const long long tmo = a.timeout_cycles;

  if (threadIdx.x == 0) {
    for (int k = 0; k < nst; k++) {
      mbar_init(smem_addr(&full_bar[k]), 1);
      mbar_init(smem_addr(&done_bar[k]), consumers);
    }
    mbar_fence_init();
    abort_flag = 0;
  }
  __syncthreads();

  double dv[DIAG_VALUES] = {0, 0, 0, 0, 0};
  bool nonfinite = false;

  if (warp == 0) {
    if (lane == 0) {
      S *f = reinterpret_cast<S *>(a.f);
      long long issued = 0;  // rows whose loads were issued
      long long k = 0;
      for (; k < my_rows; k++) {
        const int st_idx = (int)(k % nst);
        if (k >= nst) {
          // Stage st_idx holds row k - nst: store it once the consumers are done.
          const long long prev = k - nst;
          if (!mbar_wait_bounded(smem_addr(&done_bar[st_idx]), (unsigned)((prev / nst) & 1), tmo)) {
            atomicOr(a.error_flag, ERROR_TIMEOUT);
            abort_flag = 1;
            break;
          }
          issue_row_store<L>(f, a.pitch, blockIdx.x + prev * gridDim.x, a.s, a.L, buf + st_idx * stage_elems);
          bulk_wait_read<0>();
        }
        if (abort_flag) break;
        issue_row_load<L>(f, a.pitch, blockIdx.x + k * gridDim.x, a.s, a.L, buf + st_idx * stage_elems,
                          smem_addr(&full_bar[st_idx]));
        issued = k + 1;
      }
      // Store the rows still resident (the last `nst` of this block).
      if (!abort_flag) {
        const long long first = my_rows > nst ? my_rows - nst : 0;
        for (long long j = first; j < my_rows; j++) {
          const int st_idx = (int)(j % nst);
          if (!mbar_wait_bounded(smem_addr(&done_bar[st_idx]), (unsigned)((j / nst) & 1), tmo)) {
            atomicOr(a.error_flag, ERROR_TIMEOUT);
            abort_flag = 1;
            break;
          }
          issue_row_store<L>(f, a.pitch, blockIdx.x + j * gridDim.x, a.s, a.L, buf + st_idx * stage_elems);
        }
      }
      bulk_wait_all();
      if (abort_flag) {
        // Loads issued but possibly never consumed: wait (bounded) for them so
        // no copy still targets this block's shared memory at exit.
        const long long first = issued > nst ? issued - nst : 0;
        for (long long j = first; j < issued; j++)
          mbar_wait_bounded(smem_addr(&full_bar[j % nst]), (unsigned)((j / nst) & 1), tmo);
      }
    }
  } else {
    const C inv_scale = a.inv_scale, scale = a.scale;
    const int ctid = threadIdx.x - 32;
    const int cstride = consumers * 32;
    for (long long k = 0; k < my_rows; k++) {
      const int st_idx = (int)(k % nst);
      if (abort_flag) break;
      if (!mbar_wait_bounded(smem_addr(&full_bar[st_idx]), (unsigned)((k / nst) & 1), tmo)) {
        atomicOr(a.error_flag, ERROR_TIMEOUT);
        abort_flag = 1;
        break;
      }
      // row = y + Ly z, so its first node is lx row (no division per row)
      const long long row = blockIdx.x + k * gridDim.x;
      S *sb = buf + st_idx * stage_elems;
      const int nrow = (int)(lx * row);
      for (int x = ctid; x < lx; x += cstride) {
        const int xp = wrap_sub(x, a.s[0], lx);  // e_x = +1 reads x - s
        const int xm = wrap_add(x, a.s[0], lx);  // e_x = -1 reads x + s
        const int n = x + nrow;
        Node<L, C> nd;
        unroll<Q>([&](auto ic) {
          constexpr int i = decltype(ic)::value;
          constexpr int ex = L::e(0, i);
          const int xs = ex > 0 ? xp : (ex < 0 ? xm : x);
          nd.g[i] = load_dev(sb + i * lx + xs, inv_scale);
        });
        const int cls = a.cls[n];
        C out[Q];
        if (cls == CLASS_SOLID) {
          collide_solid(nd, out);
        } else {
          moments(nd);
          collide_fluid<L, C, COL, FORCE, BLEND>(nd, a, n, cls ? a.table[cls] : 0u, out);
        }
        auto slot_of = [&](auto ic) {
          constexpr int i = decltype(ic)::value;
          constexpr int ex = L::e(0, i);
          const int xs = ex > 0 ? xp : (ex < 0 ? xm : x);
          return sb + i * lx + xs;
        };
        if constexpr (stochastic_storage<S>())
          store_node_sr<Q, false>(out, scale, (unsigned)n ^ a.sr_seed, slot_of);
        else
          unroll<Q>([&](auto ic) { store_smem(slot_of(ic), out[decltype(ic)::value], scale); });
        store_and_reduce(nd, a, n, dv, nonfinite, DIAG);
      }
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_addr(&done_bar[st_idx]));
    }
  }
  if (DIAG) {
    __syncthreads();
    block_diag<C>(dv, nonfinite, a, blockIdx.x);
  }
}

// Stress-free pre-pass: before the step, copy the inward populations of each
// stress-free node's interior neighbour (pre-collision, read from the
// neighbour's shift slots) into sf_buf, so the step kernel can use them
// without racing with the neighbour's in-place update.
template <class L, class S>
__global__ void sf_gather_kernel(const StepArgs<typename Storage<S>::C> a,
                                 const int *sf_nodes, const uint8_t *sf_face_of, int n_sf,
                                 typename Storage<S>::C *sf_buf) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_sf) return;
  const int n = sf_nodes[k];
  const int face = sf_face_of[k];
  const int axis = face >> 1;
  const int inward = (face & 1) ? -1 : 1;
  int c[3];
  c[0] = n % a.L[0];
  c[1] = (n / a.L[0]) % a.L[1];
  c[2] = n / (a.L[0] * a.L[1]);
  c[axis] += inward;
  if (c[axis] < 0) c[axis] += a.L[axis];
  if (c[axis] >= a.L[axis]) c[axis] -= a.L[axis];
  Sites st;
  st.init(c[0], c[1], c[2], a.s, a.L);
  const S *f = reinterpret_cast<const S *>(a.f);
  unroll<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    bool need = false;
    unroll<2 * L::DIM>([&](auto fc) {
      if constexpr (sf_unknown<L>(decltype(fc)::value, i)) need |= (face == decltype(fc)::value);
    });
    if (need)
      sf_buf[(long long)k * L::Q + i] = load_dev(f + natural_slot<L, i>(a, st), a.inv_scale);
  });
}

// Natural-layout FP64 copy of population i: out[x] = w_i + g_i(x).
// Grid as for the direct step kernel.
template <class L, class S>
__global__ void fetch_population_kernel(const StepArgs<typename Storage<S>::C> a,
                                        int i, double *out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.L[0]) return;
  Sites st;
  st.init(x, blockIdx.y, blockIdx.z, a.s, a.L);
  const int n = x + a.L[0] * ((int)blockIdx.y + a.L[1] * (int)blockIdx.z);
  const S *f = reinterpret_cast<const S *>(a.f);
  unroll<L::Q>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    if (k == i) out[n] = weight<L>(k) + (double)load_dev(f + natural_slot<L, k>(a, st), a.inv_scale);
  });
}

// Writes population i from natural-layout FP64 values into its slots for
// the current step: stored = (f - w) * scale.
template <class L, class S>
__global__ void upload_population_kernel(const StepArgs<typename Storage<S>::C> a,
                                         int i, const double *in) {
  using C = typename Storage<S>::C;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.L[0]) return;
  Sites st;
  st.init(x, blockIdx.y, blockIdx.z, a.s, a.L);
  const int n = x + a.L[0] * ((int)blockIdx.y + a.L[1] * (int)blockIdx.z);
  S *f = reinterpret_cast<S *>(a.f);
  unroll<L::Q>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    if (k == i) store_dev(f + natural_slot<L, k>(a, st), (C)(in[n] - weight<L>(k)), a.scale);
  });
}

}  // namespace lbmc
