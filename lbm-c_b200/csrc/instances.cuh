// Launchers for one (lattice, storage) pair; included once per inst_*.cu so
// that the kernel instantiations compile in parallel.
#pragma once

#include "engine_internal.h"
#include "kernels.cuh"

namespace lbmc {

// Shared memory of the pipelined kernel's stages, per block (at least two
// stages of Q rows): with FP32 rows of 256 nodes, two stages, seven blocks
// per SM.
constexpr long long PIPE_STAGE_BUDGET = 32 * 1024;

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
      a.s[k] = d.aa ? (int)((t & 1) % d.L[k]) : (int)(t % d.L[k]);
    }
    a.aa = d.aa;
    a.tiled = d.tiled;
    a.odd = (int)(t & 1);
    a.rho = static_cast<C *>(d.rho);
    a.sf_buf = static_cast<const C *>(d.sf_buf);
    a.sf_index = d.sf_index;
    a.diag_partials = d.partials;
    a.diag_flag = d.flag;
    a.n = (int)d.n;
    a.tau = (C)d.tau;
    a.omega = (C)(1.0 / d.tau);
    // MRT rates pre-divided by the moment norms D_k = sum_i M_ki^2.
    for (int k = 0; k < 15; k++) a.s_mrt[k] = k < L::Q ? (C)(d.s_mrt[k] / (double)L::mnorm(k)) : C(0);
    a.c_smag = (C)d.c_smag;
    a.scale = (C)d.scale;
    a.inv_scale = (C)(1.0 / d.scale);
    a.compat = d.compat;
    a.store = store ? 1 : 0;
    a.error_flag = d.error_flag;
    a.timeout_cycles = d.timeout_cycles;
    a.rows = (long long)d.L[1] * d.L[2];
    a.stages = d.stages;
    a.table = d.table_dev;
    a.closure = static_cast<const MlpStep *>(d.closure);
    a.mlp = d.closure_consts;
    a.sr_seed = sr_step_seed(t);
    return a;
  }

  // One block row per (y, z); blocks of up to STEP_BLOCK threads along x.
  static dim3 block_dim(const DeviceState &d) {
    int bx = (d.L[0] + 31) / 32 * 32;
    return dim3(bx < DIRECT_BLOCK ? bx : DIRECT_BLOCK, 1, 1);
  }
  static dim3 grid_dim(const DeviceState &d) {
    const int bx = (int)block_dim(d).x;
    return dim3((unsigned)((d.L[0] + bx - 1) / bx), (unsigned)d.L[1], (unsigned)d.L[2]);
  }
  static long long blocks(const DeviceState &d) {
    const dim3 g = grid_dim(d);
    return (long long)g.x * g.y * g.z;
  }

  // Pipelined (bulk-copy) launch geometry: stages of Q rows in shared memory.
  static size_t stage_bytes(const DeviceState &d) { return (size_t)L::Q * d.L[0] * sizeof(S); }
  static bool pipelined_eligible(const DeviceState &d) {
    return d.pipeline && (d.L[0] * sizeof(S)) % 16 == 0 && 2 * stage_bytes(d) <= 200 * 1024;
  }
  static int pipe_stages(const DeviceState &d) {
    long long st = PIPE_STAGE_BUDGET / (long long)stage_bytes(d);
    if (st < 2) st = 2;
    if (st > PIPE_MAX_STAGES) st = PIPE_MAX_STAGES;
    return (int)st;
  }
  // One producer warp plus up to pipe_consumers<S>() / 32 consumer warps.
  static int pipe_threads(const DeviceState &d) {
    int bx = (d.L[0] + 31) / 32 * 32;
    return 32 + (bx < pipe_consumers<S>() ? bx : pipe_consumers<S>());
  }

  template <int COL, bool FORCE, bool BLEND, bool DIAG>
  static cudaError_t launch(const StepArgs<C> &a, const DeviceState &d, cudaStream_t st) {
    // The learned closure evaluates its network warp-wide, which the direct
    // kernel's converged warps allow: it never runs in the pipelined kernel.
    if constexpr (!learned_closure(COL)) {
      if (d.use_pipeline) {
        auto kern = step_pipelined_kernel<L, S, COL, FORCE, BLEND, DIAG>;
        const size_t smem = (size_t)d.stages * stage_bytes(d);
        static thread_local size_t configured = 0;  // per instantiation
        if (configured < smem) {
          cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
          if (e != cudaSuccess) return e;
          configured = smem;
        }
        kern<<<(unsigned)d.pipe_grid, pipe_threads(d), smem, st>>>(a);
        return cudaSuccess;
      }
    }
    if (!d.aa)
      step_kernel<L, S, COL, FORCE, BLEND, DIAG, STREAM_SHIFT><<<grid_dim(d), block_dim(d), 0, st>>>(a);
    else if (d.tiled && a.odd)
      step_kernel<L, S, COL, FORCE, BLEND, DIAG, STREAM_AAT_ODD><<<grid_dim(d), block_dim(d), 0, st>>>(a);
    else if (d.tiled)
      step_kernel<L, S, COL, FORCE, BLEND, DIAG, STREAM_AAT_EVEN><<<grid_dim(d), block_dim(d), 0, st>>>(a);
    else if (a.odd)
      step_kernel<L, S, COL, FORCE, BLEND, DIAG, STREAM_AA_ODD><<<grid_dim(d), block_dim(d), 0, st>>>(a);
    else
      step_kernel<L, S, COL, FORCE, BLEND, DIAG, STREAM_AA_EVEN><<<grid_dim(d), block_dim(d), 0, st>>>(a);
    return cudaSuccess;
  }

  template <int COL, bool BLEND>
  static cudaError_t launch_fd(const StepArgs<C> &a, const DeviceState &d, bool diag, cudaStream_t st) {
    if (d.forcing) {
      if (diag) return launch<COL, true, BLEND, true>(a, d, st);
      return launch<COL, true, BLEND, false>(a, d, st);
    }
    if (diag) return launch<COL, false, BLEND, true>(a, d, st);
    return launch<COL, false, BLEND, false>(a, d, st);
  }

  template <int COL>
  static cudaError_t launch_col(const StepArgs<C> &a, const DeviceState &d, bool diag, cudaStream_t st) {
    if (d.blend) return launch_fd<COL, true>(a, d, diag, st);
    return launch_fd<COL, false>(a, d, diag, st);
  }

  static cudaError_t step(const DeviceState &d, long long t, bool store, bool diag,
                          cudaStream_t st) {
    const StepArgs<C> a = make_args(d, t, store);
    if (d.n_sf > 0) {
      const int nb = (d.n_sf + 127) / 128;
      sf_gather_kernel<L, S><<<nb, 128, 0, st>>>(a, d.sf_nodes, d.sf_face, d.n_sf,
                                                  static_cast<C *>(d.sf_buf));
    }
    cudaError_t e;
    switch (d.col) {
      case COL_BGK: e = launch_col<COL_BGK>(a, d, diag, st); break;
      case COL_BGK_SMAG: e = launch_col<COL_BGK_SMAG>(a, d, diag, st); break;
      case COL_MRT_NC: e = launch_col<COL_MRT_NC>(a, d, diag, st); break;
      case COL_BGK_MLP: e = launch_col<COL_BGK_MLP>(a, d, diag, st); break;
      case COL_BGK_MLP1: e = launch_col<COL_BGK_MLP1>(a, d, diag, st); break;
      default: e = launch_col<COL_MRT>(a, d, diag, st); break;
    }
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
  }

  // Chooses the kernel and its launch geometry for a handle (called once by
  // lbmc_init after the device state is filled in).
  static cudaError_t plan(DeviceState &d) {
    // The direct-load kernel is the default; the bulk-copy pipeline runs when
    // asked for (lbmc_config.kernel) and the rows allow it.
    d.use_pipeline = (d.pipeline == 2 && !d.aa && pipelined_eligible(d)) ? 1 : 0;
    if (!d.use_pipeline) {
      d.nblocks = blocks(d);
      return cudaSuccess;
    }
    d.stages = pipe_stages(d);
    const size_t smem = (size_t)d.stages * stage_bytes(d);
    // Occupancy of the heaviest instantiation the handle can launch.
    int per_sm = 0;
    cudaError_t e;
    auto probe = [&](auto kern) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, pipe_threads(d), smem);
    };
    switch (d.col) {
      case COL_BGK: probe(step_pipelined_kernel<L, S, COL_BGK, true, true, true>); break;
      case COL_BGK_SMAG: probe(step_pipelined_kernel<L, S, COL_BGK_SMAG, true, true, true>); break;
      case COL_MRT_NC: probe(step_pipelined_kernel<L, S, COL_MRT_NC, true, true, true>); break;
      default: probe(step_pipelined_kernel<L, S, COL_MRT, true, true, true>); break;
    }
    if (e != cudaSuccess) return e;
    if (per_sm < 1) {
      d.use_pipeline = 0;
      d.nblocks = blocks(d);
      return cudaSuccess;
    }
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long rows = (long long)d.L[1] * d.L[2];
    long long grid = (long long)sms * per_sm;
    if (grid > rows) grid = rows;
    d.pipe_grid = grid;
    d.nblocks = grid;
    return cudaSuccess;
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
                                        &upload_population, &plan};
    return &o;
  }
};

}  // namespace lbmc

#define LBMC_DEFINE_OPS(NAME, LAT, STORE) \
  namespace lbmc {                        \
  const LatticeStorageOps *NAME() { return Launchers<LAT, STORE>::ops(); } \
  }
