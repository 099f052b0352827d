// Internal interface between the C-ABI engine (engine.cu) and the
// per-(lattice, storage) kernel instantiations (inst_*.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "mlp.cuh"

namespace lbmc {

// Device-side state of one handle, in the form the launchers consume.
struct DeviceState {
  int lattice, storage, q, dim;
  int L[3];
  long long n;
  void *f;  // storage type
  long long pitch;
  uint8_t *cls;
  void *B;         // compute type, N (partial nodes only)
  void *force[3];  // compute type, N each; null for a uniform force
  double force_u[3];
  void *rho;  // compute type: rho - 1
  void *u[3];
  int n_sf;
  int *sf_nodes;
  uint8_t *sf_face;
  int *sf_index;
  void *sf_buf;
  double *partials;
  unsigned *flag;
  double tau, c_smag, s_mrt[15], scale;
  unsigned compat;
  int col;  // COL_BGK / COL_BGK_SMAG / COL_MRT
  int forcing;
  int blend;  // Noble-Torczynski partial nodes present
  uint16_t table[256];
  uint16_t *table_dev;      // device copy of table
  unsigned *error_flag;     // device word, ERROR_TIMEOUT on an expired wait
  long long timeout_cycles; // bound of every device-side wait
  int aa;                   // AA-pattern layout (else the shift layout)
  int tiled;                // AA over 64-node tiles (Lx a multiple of 64)
  int pipeline;             // allow the bulk-copy pipelined kernel
  int use_pipeline;         // chosen by plan()
  int stages;               // shared-memory stages of the pipelined kernel
  long long pipe_grid;      // persistent blocks of the pipelined kernel
  long long nblocks;        // blocks of the step kernel (diagnostic partials)
  void *closure;            // device MlpStep when a learned closure is attached
  lbmc::MlpConsts closure_consts;  // its scalars, passed with each launch
};

struct LatticeStorageOps {
  int csize;  // bytes of the compute type
  int ssize;  // bytes of the storage type
  // One time step at step counter t (shift t mod L).
  cudaError_t (*step)(const DeviceState &, long long t, bool store, bool diag, cudaStream_t);
  // out[x] = f_i(x) in natural layout (FP64) at step counter t.
  cudaError_t (*fetch_population)(const DeviceState &, long long t, int i, double *out,
                                   cudaStream_t);
  // Sets population i from natural-layout FP64 values at step counter t.
  cudaError_t (*upload_population)(const DeviceState &, long long t, int i, const double *in,
                                   cudaStream_t);
  // Chooses the step kernel and launch geometry; sets nblocks.
  cudaError_t (*plan)(DeviceState &);
};

// Sets the calling thread's lbmc_last_error() message.
void set_last_error(const std::string &message);

struct MlpClosure;

const LatticeStorageOps *ops_d2q9_f32();
const LatticeStorageOps *ops_d2q9_f16();
const LatticeStorageOps *ops_d2q9_bf16();
const LatticeStorageOps *ops_d2q9_f64();
const LatticeStorageOps *ops_d3q15_f32();
const LatticeStorageOps *ops_d3q15_f16();
const LatticeStorageOps *ops_d3q15_bf16();
const LatticeStorageOps *ops_d3q15_f64();
const LatticeStorageOps *ops_d2q9_f16sr();
const LatticeStorageOps *ops_d3q15_f16sr();

}  // namespace lbmc
