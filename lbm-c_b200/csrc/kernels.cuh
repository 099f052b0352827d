// Step kernels of the engine: one fused kernel per (lattice, storage,
// collision family, forcing, diagnostics) performs, for every node, the
// reference's whole time step (LBM-C/solver.cu:10-136):
//
//   load f_i from its in-place shift slot (x - t e_i) mod L  (solver.cu:75-102)
//   rho, u                                                   (solver.cu:96-108)
//   macro BC, micro BC                                       (solver.cu:111-112)
//   collision or bounceback                                  (solver.cu:56-72,115)
//   write f_i back to the same slot                          (solver.cu:120-123)
//   optional rho/u store and FP64 diagnostic partial sums    (solver.cu:126-134,
//                                                             index.cu:338-373)
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

#include <type_traits>
#include <utility>

#include "lattice.cuh"

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

template <>
struct Storage<double> {
  using C = double;
  static __device__ __forceinline__ C get(const double *p) { return *p; }
  static __device__ __forceinline__ void put(double *p, C v) { *p = v; }
};
template <>
struct Storage<float> {
  using C = float;
  static __device__ __forceinline__ C get(const float *p) { return *p; }
  static __device__ __forceinline__ void put(float *p, C v) { *p = v; }
};
template <>
struct Storage<__half> {
  using C = float;
  static __device__ __forceinline__ C get(const __half *p) { return __half2float(*p); }
  static __device__ __forceinline__ void put(__half *p, C v) { *p = __float2half_rn(v); }
};
template <>
struct Storage<__nv_bfloat16> {
  using C = float;
  static __device__ __forceinline__ C get(const __nv_bfloat16 *p) { return __bfloat162float(*p); }
  static __device__ __forceinline__ void put(__nv_bfloat16 *p, C v) { *p = __float2bfloat16_rn(v); }
};

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

constexpr int DIAG_VALUES = 5;  // mass, momentum x/y/z, kinetic energy
constexpr int STEP_BLOCK = 256;

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
  int s[3];  // shift of the current step: t mod L
  int n;
  C tau;
  C s_mrt[15];
  C c_smag;
  C scale, inv_scale;
  unsigned compat;
  int store;
  uint16_t table[256];
};

// ----------------------------------------------------------- index helpers

__device__ __forceinline__ int wrap_sub(int x, int s, int L) {
  const int v = x - s;
  return v < 0 ? v + L : v;
}
__device__ __forceinline__ int wrap_add(int x, int s, int L) {
  const int v = x + s;
  return v >= L ? v - L : v;
}

__host__ __device__ constexpr int sel(int e) { return e == 0 ? 0 : (e > 0 ? 1 : 2); }

// Shift-streaming sites of one node: population i of node (x, y, z) at step
// t lives in slot ((x - t e_x) mod Lx) + Lx ((y - t e_y) mod Ly + Ly (...))
// (LBM-C/solver.cu:82-94).  Index [1] of a component is e = +1 (reads
// x - s), [2] is e = -1 (reads x + s).  The kernels launch one block row per
// (y, z), so the row offsets are uniform across the block.
struct Sites {
  int x[3];
  int row[3][3];  // [sel(e_y)][sel(e_z)] -> Lx * (y' + Ly * z')
  __device__ __forceinline__ void init(int cx, int cy, int cz, const int *s, const int *L) {
    x[0] = cx;
    x[1] = wrap_sub(cx, s[0], L[0]);
    x[2] = wrap_add(cx, s[0], L[0]);
    const int ys[3] = {cy, wrap_sub(cy, s[1], L[1]), wrap_add(cy, s[1], L[1])};
    const int zs[3] = {cz, wrap_sub(cz, s[2], L[2]), wrap_add(cz, s[2], L[2])};
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) row[a][b] = L[0] * (ys[a] + L[1] * zs[b]);
  }
  template <class L>
  __device__ __forceinline__ int slot(int i) const {
    // i is a compile-time constant after unrolling, so sel() folds.
    return x[sel(L::e(0, i))] + row[sel(L::e(1, i))][sel(L::e(2, i))];
  }
};

// -------------------------------------------------------------- physics

template <class L, class C>
struct Node {
  C g[L::Q];  // deviations f - w
  C drho;     // rho - 1
  C rho;
  C u[3];
};

template <class L>
__device__ __forceinline__ constexpr double weight(int i) {
  return (double)L::wn(i) / (double)L::wd;
}

// rho = 1 + sum g, u = sum e g / rho (LBM-C/solver.cu:96-108).
template <class L, class C>
__device__ __forceinline__ void moments(Node<L, C> &nd) {
  C d = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
  for (int i = 0; i < L::Q; i++) {
    d += nd.g[i];
    if (L::e(0, i)) jx += L::e(0, i) * nd.g[i];
    if (L::e(1, i)) jy += L::e(1, i) * nd.g[i];
    if (L::DIM > 2 && L::e(2, i)) jz += L::e(2, i) * nd.g[i];
  }
  nd.drho = d;
  nd.rho = C(1) + d;
  const C inv = C(1) / nd.rho;
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
#pragma unroll
  for (int i = 0; i < L::Q; i++) {
#pragma unroll
    for (int fc = 0; fc < 2 * L::DIM; fc++)
      if (fc == face && sf_unknown<L>(fc, i)) nd.g[i] = row[i];
  }
}

// e_i . v for a compile-time population i.
template <class L, class C>
__device__ __forceinline__ C edot(int i, const C *v) {
  C r = 0;
  if (L::e(0, i)) r += C(L::e(0, i)) * v[0];
  if (L::e(1, i)) r += C(L::e(1, i)) * v[1];
  if (L::DIM > 2 && L::e(2, i)) r += C(L::e(2, i)) * v[2];
  return r;
}

// Equilibrium deviation geq_i = f_eq_i - w_i = w_i (drho + rho (eu + eu^2/2 - usq))
// with eu = 3 e.u and usq = 1.5 u.u (LBM-C/collision.cu:53-59).
template <class L, class C>
__device__ __forceinline__ C geq_dev(int i, const Node<L, C> &nd, C usq) {
  const C eu = C(3) * edot<L>(i, nd.u);
  return C(weight<L>(i)) * (nd.drho + nd.rho * (eu + C(0.5) * eu * eu - usq));
}

// Guo source (LBM-C/collision.cu:82-99), after u <- u + F/(2 rho):
// F_i = w_i (1 - 1/(2 tau)) [3 (e_i - u) + 9 (e_i.u) e_i] . F
//     = w_i pre (3 (e_i.F - u.F) + 9 (e_i.u)(e_i.F)).
template <class L, class C>
__device__ __forceinline__ C guo_term(int i, const Node<L, C> &nd, const C *F, C pre, C uF) {
  const C eF = edot<L>(i, F);
  const C eu = edot<L>(i, nd.u);
  return C(weight<L>(i)) * pre * (C(3) * (eF - uF) + C(9) * eu * eF);
}

// Smagorinsky relaxation time (LBM-C/collision.cu:445-463, q_bar zeroed):
// q_ab = sum_i e_a e_b (f - f_eq), q_hat = sum_ab sqrt(2 q_ab^2),
// tau_eff = tau + (sqrt(tau^2 + 2 sqrt2 C^2 (9/rho) q_hat) - tau)/2.
template <class L, class C>
__device__ __forceinline__ C smagorinsky_tau(const Node<L, C> &nd, C usq, C tau, C cs) {
  C q[6] = {0, 0, 0, 0, 0, 0};  // xx, yy, zz, xy, yz, xz
#pragma unroll
  for (int i = 0; i < L::Q; i++) {
    const C neq = nd.g[i] - geq_dev<L>(i, nd, usq);
    const int ex = L::e(0, i), ey = L::e(1, i), ez = L::e(2, i);
    if (ex) q[0] += neq;
    if (ey) q[1] += neq;
    if (ez) q[2] += neq;
    if (ex * ey) q[3] += C(ex * ey) * neq;
    if (ey * ez) q[4] += C(ey * ez) * neq;
    if (ex * ez) q[5] += C(ex * ez) * neq;
  }
  const C r2 = sqrt(C(2));
  C qhat = r2 * (fabs(q[0]) + fabs(q[1]) + C(2) * fabs(q[3]));
  if (L::DIM > 2) qhat += r2 * (fabs(q[2]) + C(2) * (fabs(q[4]) + fabs(q[5])));
  const C k = C(2) * r2 * cs * cs * (C(9) / nd.rho);
  return tau + C(0.5) * (sqrt(tau * tau + k * qhat) - tau);
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

// ------------------------------------------------------------ diagnostics

template <class C>
__device__ __forceinline__ void block_diag(const double (&v)[DIAG_VALUES], bool nonfinite,
                                           const StepArgs<C> &a, long long block) {
  __shared__ double red[STEP_BLOCK / 32][DIAG_VALUES];
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

// -------------------------------------------------------------- the step

// Grid: blockDim (bx, 1, 1) along x, gridDim (ceil(Lx/bx), Ly, Lz).
// COL: COL_BGK / COL_BGK_SMAG / COL_MRT.  BLEND: Noble-Torczynski partial
// solid nodes present (ColType NTPOR/MRTPOR).  DIAG: emit FP64 partial sums.
template <class L, class S, int COL, bool FORCE, bool BLEND, bool DIAG>
__global__ void __launch_bounds__(STEP_BLOCK)
    step_kernel(const __grid_constant__ StepArgs<typename Storage<S>::C> a) {
  using C = typename Storage<S>::C;
  constexpr int Q = L::Q;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = x < a.L[0];
  if (!DIAG && !active) return;
  double dv[DIAG_VALUES] = {0, 0, 0, 0, 0};
  bool nonfinite = false;
  if (active) {
    Sites st;
    st.init(x, blockIdx.y, blockIdx.z, a.s, a.L);
    const int n = x + a.L[0] * ((int)blockIdx.y + a.L[1] * (int)blockIdx.z);
    S *f = reinterpret_cast<S *>(a.f);
    Node<L, C> nd;
#pragma unroll
    for (int i = 0; i < Q; i++)
      nd.g[i] = Storage<S>::get(f + i * a.pitch + st.template slot<L>(i)) * a.inv_scale;
    const int cls = a.cls[n];
    if (cls == CLASS_SOLID) {
      // bounceback (LBM-C/collision.cu:423-443): f_i <- f_opp(i), rho = u = 0.
#pragma unroll
      for (int i = 0; i < Q; i++)
        Storage<S>::put(f + i * a.pitch + st.template slot<L>(i), nd.g[L::opp(i)] * a.scale);
      nd.drho = C(-1);
      nd.rho = 0;
      nd.u[0] = nd.u[1] = nd.u[2] = 0;
    } else {
      moments(nd);
      const unsigned entry = cls ? a.table[cls] : 0u;
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
      if (FORCE) {
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
        const C h = C(1) / (C(2) * nd.rho);
        nd.u[0] += h * F[0];
        nd.u[1] += h * F[1];
        if (L::DIM > 2) nd.u[2] += h * F[2];
        pre = C(1) - C(1) / (C(2) * tau0);
        uF = nd.u[0] * F[0] + nd.u[1] * F[1] + (L::DIM > 2 ? nd.u[2] * F[2] : C(0));
      }
      const C omb = C(1) - B;
      if (COL == COL_MRT) {
        // m* = S (M g - meq) / D; f <- f - M^T m* (collision.cu:192-303)
        C ms[Q];
        unroll<Q>([&](auto kc) {
          constexpr int k = decltype(kc)::value;
          C mk = 0;
          unroll<Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            constexpr int mki = L::m(k, i);
            if constexpr (mki == 1) mk += nd.g[i];
            else if constexpr (mki == -1) mk -= nd.g[i];
            else if constexpr (mki != 0) mk += C(mki) * nd.g[i];
          });
          constexpr double inv_norm = 1.0 / (double)L::mnorm(k);
          ms[k] = a.s_mrt[k] * (mk - meq_dev<L>(k, nd, a.compat)) * C(inv_norm);
        });
        const bool minv_zero = Q == 15 && (a.compat & COMPAT_D3Q15_MINV_ZERO);
        const bool inplace = BLEND && (a.compat & COMPAT_MRTPOR_INPLACE);
        C keep[Q] = {};
        unroll<Q>([&](auto ic) {
          constexpr int i = decltype(ic)::value;
          constexpr int o = L::opp(i);
          C acc = 0;
          unroll<Q>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            constexpr int mki = L::m(k, i);
            if constexpr (mki == 1) acc += ms[k];
            else if constexpr (mki == -1) acc -= ms[k];
            else if constexpr (mki != 0) acc += C(mki) * ms[k];
          });
          if (minv_zero) acc = 0;
          const C ft = FORCE ? guo_term<L>(i, nd, F, pre, uF) : C(0);
          C out;
          if constexpr (BLEND) {
            // mrt_ntpor(_guo)_collision (collision.cu:305-421).  The reference
            // reads f[opp[i]] after lower indices were already updated
            // (collision.cu:340,416); COMPAT_MRTPOR_INPLACE reproduces that.
            C fo = nd.g[o];
            if constexpr (o < i) {
              if (inplace) fo = keep[o];
            }
            out = nd.g[i] - omb * acc + omb * ft + B * (fo - nd.g[i]);
            keep[i] = out;
          } else {
            out = nd.g[i] - acc + ft;
          }
          Storage<S>::put(f + i * a.pitch + st.template slot<L>(i), out * a.scale);
        });
      } else {
        const C usq = C(1.5) * (nd.u[0] * nd.u[0] + nd.u[1] * nd.u[1] + nd.u[2] * nd.u[2]);
        C tau = tau0;
        if (COL == COL_BGK_SMAG) tau = smagorinsky_tau(nd, usq, tau0, a.c_smag);
        const C om = C(1) / tau;
#pragma unroll
        for (int i = 0; i < Q; i++) {
          const C omega_i = om * (nd.g[i] - geq_dev<L>(i, nd, usq));
          const C ft = FORCE ? guo_term<L>(i, nd, F, pre, uF) : C(0);
          C out;
          if (BLEND)  // bgk_ntpor(_guo)_collision (collision.cu:113-190)
            out = nd.g[i] - omb * omega_i + B * (nd.g[L::opp(i)] - nd.g[i]) + omb * ft;
          else
            out = nd.g[i] - omega_i + ft;
          Storage<S>::put(f + i * a.pitch + st.template slot<L>(i), out * a.scale);
        }
      }
    }
    if (a.store) {
      a.rho[n] = nd.drho;
      a.u[0][n] = nd.u[0];
      a.u[1][n] = nd.u[1];
      if (L::DIM > 2) a.u[2][n] = nd.u[2];
    }
    if (DIAG) {
      const double rho = (double)nd.drho + 1.0;
      const double ux = nd.u[0], uy = nd.u[1], uz = nd.u[2];
      dv[0] = rho;
      dv[1] = rho * ux;
      dv[2] = rho * uy;
      dv[3] = rho * uz;
      dv[4] = 0.5 * rho * (ux * ux + uy * uy + uz * uz);
      nonfinite = !(isfinite(rho) && isfinite(ux) && isfinite(uy) && isfinite(uz));
    }
  }
  if (DIAG)
    block_diag<C>(dv, nonfinite, a,
                  blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z));
}

// Stress-free pre-pass: before the step, copy the inward populations of each
// stress-free node's interior neighbour (pre-collision, read from the
// neighbour's shift slots) into sf_buf, so the step kernel can use them
// without racing with the neighbour's in-place update.
template <class L, class S>
__global__ void sf_gather_kernel(const __grid_constant__ StepArgs<typename Storage<S>::C> a,
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
#pragma unroll
  for (int i = 0; i < L::Q; i++) {
    bool need = false;
#pragma unroll
    for (int fc = 0; fc < 2 * L::DIM; fc++) need |= (fc == face) && sf_unknown<L>(fc, i);
    if (need)
      sf_buf[(long long)k * L::Q + i] =
          Storage<S>::get(f + i * a.pitch + st.template slot<L>(i)) * a.inv_scale;
  }
}

// Natural-layout FP64 copy of population i: out[x] = w_i + g_i(x).
// Grid as for the step kernel.
template <class L, class S>
__global__ void fetch_population_kernel(const __grid_constant__ StepArgs<typename Storage<S>::C> a,
                                        int i, double *out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.L[0]) return;
  Sites st;
  st.init(x, blockIdx.y, blockIdx.z, a.s, a.L);
  const int n = x + a.L[0] * ((int)blockIdx.y + a.L[1] * (int)blockIdx.z);
  const S *f = reinterpret_cast<const S *>(a.f);
#pragma unroll
  for (int k = 0; k < L::Q; k++)
    if (k == i)
      out[n] = weight<L>(k) + (double)(Storage<S>::get(f + k * a.pitch + st.template slot<L>(k)) * a.inv_scale);
}

// Writes population i from natural-layout FP64 values into its slots for
// the current step: stored = (f - w) * scale.
template <class L, class S>
__global__ void upload_population_kernel(const __grid_constant__ StepArgs<typename Storage<S>::C> a,
                                         int i, const double *in) {
  using C = typename Storage<S>::C;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.L[0]) return;
  Sites st;
  st.init(x, blockIdx.y, blockIdx.z, a.s, a.L);
  const int n = x + a.L[0] * ((int)blockIdx.y + a.L[1] * (int)blockIdx.z);
  S *f = reinterpret_cast<S *>(a.f);
#pragma unroll
  for (int k = 0; k < L::Q; k++)
    if (k == i)
      Storage<S>::put(f + k * a.pitch + st.template slot<L>(k), (C)(in[n] - weight<L>(k)) * a.scale);
}

}  // namespace lbmc
