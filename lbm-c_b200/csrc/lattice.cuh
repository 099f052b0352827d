// Lattice descriptors for the step kernels.
//
// Velocity order, weights and opposites are those of LBM-C/macros.cu:19-53
// (D2Q9) and :71-119 (D3Q15), kept identical so that population indices,
// MacroBC/MicroBC codes and the Zou-He formulas of the reference map one to
// one.  The moment matrices are LBM-C's M (macros.cu:24-36, :77-95); their
// inverse is formed as M^T D^-1 with D = diag(M M^T) (the rows are
// orthogonal), which is what the reference's D3Q15 M_inv literals intend
// (macros.cu:97-115 evaluate to zero through integer division).
//
// Every table is a constexpr function so that, inside fully unrolled loops,
// nvcc folds the entries into immediates (no constant-memory or local-memory
// tables on the hot path).
#pragma once

namespace lbmc {

struct D2Q9 {
  static constexpr int Q = 9;
  static constexpr int DIM = 2;
  static constexpr int ID = 0;
  __host__ __device__ static constexpr int e(int d, int i) {
    constexpr int t[3][9] = {{0, 1, 0, -1, 0, 1, -1, -1, 1},
                             {0, 0, 1, 0, -1, 1, 1, -1, -1},
                             {0, 0, 0, 0, 0, 0, 0, 0, 0}};
    return t[d][i];
  }
  __host__ __device__ static constexpr int opp(int i) {
    constexpr int t[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
    return t[i];
  }
  // Opposite pairs (i, opp(i)) with i < opp(i); population 0 is its own.
  static constexpr int NP = 4;
  __host__ __device__ static constexpr int pair(int p) {
    constexpr int t[4] = {1, 2, 5, 6};
    return t[p];
  }
  // Weights as exact rationals w = wn / wd.
  __host__ __device__ static constexpr int wn(int i) { return i == 0 ? 16 : (i < 5 ? 4 : 1); }
  static constexpr int wd = 36;
  __host__ __device__ static constexpr int c2(int i) { return e(0, i) * e(0, i) + e(1, i) * e(1, i); }
  // M (LBM-C/macros.cu:24-36): rho, e, eps, jx, qx, jy, qy, pxx, pxy.
  __host__ __device__ static constexpr int m(int k, int i) {
    return k == 0   ? 1
           : k == 1 ? 3 * c2(i) - 4
           : k == 2 ? (c2(i) == 0 ? 4 : (c2(i) == 1 ? -2 : 1))
           : k == 3 ? e(0, i)
           : k == 4 ? e(0, i) * (c2(i) == 1 ? -2 : 1)
           : k == 5 ? e(1, i)
           : k == 6 ? e(1, i) * (c2(i) == 1 ? -2 : 1)
           : k == 7 ? e(0, i) * e(0, i) - e(1, i) * e(1, i)
                    : e(0, i) * e(1, i);
  }
  __host__ __device__ static constexpr int mnorm(int k) {
    int s = 0;
    for (int i = 0; i < Q; i++) s += m(k, i) * m(k, i);
    return s;
  }
};

struct D3Q15 {
  static constexpr int Q = 15;
  static constexpr int DIM = 3;
  static constexpr int ID = 1;
  __host__ __device__ static constexpr int e(int d, int i) {
    constexpr int t[3][15] = {{0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1},
                              {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
                              {0, 0, 0, 0, 0, 1, -1, 1, 1, 1, 1, -1, -1, -1, -1}};
    return t[d][i];
  }
  __host__ __device__ static constexpr int opp(int i) {
    constexpr int t[15] = {0, 2, 1, 4, 3, 6, 5, 14, 13, 12, 11, 10, 9, 8, 7};
    return t[i];
  }
  static constexpr int NP = 7;
  __host__ __device__ static constexpr int pair(int p) {
    constexpr int t[7] = {1, 3, 5, 7, 8, 9, 10};
    return t[p];
  }
  __host__ __device__ static constexpr int wn(int i) { return i == 0 ? 16 : (i < 7 ? 8 : 1); }
  static constexpr int wd = 72;
  __host__ __device__ static constexpr int c2(int i) {
    return e(0, i) * e(0, i) + e(1, i) * e(1, i) + e(2, i) * e(2, i);
  }
  __host__ __device__ static constexpr int fac(int i) { return c2(i) == 1 ? -4 : 1; }
  // M (LBM-C/macros.cu:77-95): rho, e, eps, jx, qx, jy, qy, jz, qz,
  // 3pxx, pww, pxy, pyz, pxz, mxyz.
  __host__ __device__ static constexpr int m(int k, int i) {
    return k == 0    ? 1
           : k == 1  ? (c2(i) == 0 ? -2 : (c2(i) == 1 ? -1 : 1))
           : k == 2  ? (c2(i) == 0 ? 16 : (c2(i) == 1 ? -4 : 1))
           : k == 3  ? e(0, i)
           : k == 4  ? e(0, i) * fac(i)
           : k == 5  ? e(1, i)
           : k == 6  ? e(1, i) * fac(i)
           : k == 7  ? e(2, i)
           : k == 8  ? e(2, i) * fac(i)
           : k == 9  ? 3 * e(0, i) * e(0, i) - c2(i)
           : k == 10 ? e(1, i) * e(1, i) - e(2, i) * e(2, i)
           : k == 11 ? e(0, i) * e(1, i)
           : k == 12 ? e(1, i) * e(2, i)
           : k == 13 ? e(0, i) * e(2, i)
                     : e(0, i) * e(1, i) * e(2, i);
  }
  __host__ __device__ static constexpr int mnorm(int k) {
    int s = 0;
    for (int i = 0; i < Q; i++) s += m(k, i) * m(k, i);
    return s;
  }
};

// A moment row is even when it takes the same value on opposite populations
// (rho, energy, stresses) and odd when it changes sign (momentum, fluxes).
template <class L>
__host__ __device__ constexpr bool moment_even(int k) {
  for (int i = 0; i < L::Q; i++)
    if (L::m(k, L::opp(i)) != L::m(k, i)) return false;
  return true;
}

}  // namespace lbmc
