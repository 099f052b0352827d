// Launchers for one (lattice, storage) pair; included once per inst_*.cu so
// that the kernel instantiations compile in parallel.
#pragma once

#include "engine_internal.h"
#include "kernels.cuh"

namespace lbmc {

template <class L, class S>
struct Launchers {
  using C = typename Storage<S>::C;

  static StepArgs<C> make_args(const DeviceState &d, long long t, bool store) {
    StepArgs<C> a;
    a.f = d.f;
    a.pitch = d.pitch;
    a.cls = d.cls;
    a.B = static_cast<const C *>(d.B);
    for (int k = 0; k < 3; k++) {
      a.force[k] = static_cast<const C *>(d.force[k]);
      a.force_u[k] = (C)d.force_u[k];
      a.u[k] = static_cast<C *>(d.u[k]);
      a.L[k] = d.L[k];
      a.s[k] = (int)(t % d.L[k]);
    }
    a.rho = static_cast<C *>(d.rho);
    a.sf_buf = static_cast<const C *>(d.sf_buf);
    a.sf_index = d.sf_index;
    a.diag_partials = d.partials;
    a.diag_flag = d.flag;
    a.n = (int)d.n;
    a.tau = (C)d.tau;
    for (int k = 0; k < 15; k++) a.s_mrt[k] = (C)d.s_mrt[k];
    a.c_smag = (C)d.c_smag;
    a.scale = (C)d.scale;
    a.inv_scale = (C)(1.0 / d.scale);
    a.compat = d.compat;
    a.store = store ? 1 : 0;
    for (int k = 0; k < 256; k++) a.table[k] = d.table[k];
    return a;
  }

  // One block row per (y, z); blocks of up to STEP_BLOCK threads along x.
  static dim3 block_dim(const DeviceState &d) {
    int bx = (d.L[0] + 31) / 32 * 32;
    return dim3(bx < STEP_BLOCK ? bx : STEP_BLOCK, 1, 1);
  }
  static dim3 grid_dim(const DeviceState &d) {
    const int bx = (int)block_dim(d).x;
    return dim3((unsigned)((d.L[0] + bx - 1) / bx), (unsigned)d.L[1], (unsigned)d.L[2]);
  }
  static long long blocks(const DeviceState &d) {
    const dim3 g = grid_dim(d);
    return (long long)g.x * g.y * g.z;
  }

  template <int COL, bool FORCE, bool BLEND, bool DIAG>
  static void launch(const StepArgs<C> &a, const DeviceState &d, cudaStream_t st) {
    step_kernel<L, S, COL, FORCE, BLEND, DIAG><<<grid_dim(d), block_dim(d), 0, st>>>(a);
  }

  template <int COL, bool BLEND>
  static void launch_fd(const StepArgs<C> &a, const DeviceState &d, bool diag, cudaStream_t st) {
    if (d.forcing) {
      if (diag) launch<COL, true, BLEND, true>(a, d, st);
      else launch<COL, true, BLEND, false>(a, d, st);
    } else {
      if (diag) launch<COL, false, BLEND, true>(a, d, st);
      else launch<COL, false, BLEND, false>(a, d, st);
    }
  }

  template <int COL>
  static void launch_col(const StepArgs<C> &a, const DeviceState &d, bool diag, cudaStream_t st) {
    if (d.blend) launch_fd<COL, true>(a, d, diag, st);
    else launch_fd<COL, false>(a, d, diag, st);
  }

  static cudaError_t step(const DeviceState &d, long long t, bool store, bool diag,
                          cudaStream_t st) {
    const StepArgs<C> a = make_args(d, t, store);
    if (d.n_sf > 0) {
      const int nb = (d.n_sf + 127) / 128;
      sf_gather_kernel<L, S><<<nb, 128, 0, st>>>(a, d.sf_nodes, d.sf_face, d.n_sf,
                                                  static_cast<C *>(d.sf_buf));
    }
    switch (d.col) {
      case COL_BGK: launch_col<COL_BGK>(a, d, diag, st); break;
      case COL_BGK_SMAG: launch_col<COL_BGK_SMAG>(a, d, diag, st); break;
      default: launch_col<COL_MRT>(a, d, diag, st); break;
    }
    return cudaGetLastError();
  }

  static cudaError_t fetch_population(const DeviceState &d, long long t, int i, double *out,
                                      cudaStream_t st) {
    const StepArgs<C> a = make_args(d, t, false);
    fetch_population_kernel<L, S><<<grid_dim(d), block_dim(d), 0, st>>>(a, i, out);
    return cudaGetLastError();
  }

  static cudaError_t upload_population(const DeviceState &d, long long t, int i, const double *in,
                                       cudaStream_t st) {
    const StepArgs<C> a = make_args(d, t, false);
    upload_population_kernel<L, S><<<grid_dim(d), block_dim(d), 0, st>>>(a, i, in);
    return cudaGetLastError();
  }

  static const LatticeStorageOps *ops() {
    static const LatticeStorageOps o = {(int)sizeof(C), (int)sizeof(S), &step, &fetch_population,
                                        &upload_population, &blocks};
    return &o;
  }
};

}  // namespace lbmc

#define LBMC_DEFINE_OPS(NAME, LAT, STORE) \
  namespace lbmc {                        \
  const LatticeStorageOps *NAME() { return Launchers<LAT, STORE>::ops(); } \
  }
