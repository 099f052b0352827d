// TEST INFRASTRUCTURE ONLY — never linked into the product library.
//
// Host shim that compiles the reference's own time-step code (LBM-C
// solver.cu:10-136 iterate_kernel, collision.cu, boundary_conditions/**,
// macros.cu, data_types.cuh) as plain host C++ and runs it over every node
// with OpenMP.  The CUDA qualifiers are emptied, __syncthreads() is a no-op
// (it sits in a divergent branch in the reference, solver.cu:118, and has no
// effect on a per-node host loop), and threadIdx/blockIdx/blockDim are
// per-thread variables set by the node loop so that the kernel's own
// coordinate arithmetic (solver.cu:19-29) selects the node.
//
// The reference files are not copied into the repository: oracle/build_ref.sh
// points the include path at them (or at a patched temporary copy for the
// D2Q9 lattice selection and the documented defect fixes) and only the
// resulting shared objects are kept, under oracle/_ref/.
//
// The shift-streaming map of the reference (solver.cu:82-94) is a bijection
// per population, so every node reads and writes disjoint slots and any node
// order gives the same result.  The stress-free micro BCs are the exception
// (they read neighbour slots, d2q9_sf_defs.cu:7-12); those codes are only run
// single-threaded by the tests and are not used as a parity oracle.

#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <omp.h>

#define __device__
#define __constant__
#define __noinline__
#define __global__
#define __host__

struct shim_dim3 {
  unsigned x, y, z;
};
static shim_dim3 threadIdx, blockIdx, blockDim;
#pragma omp threadprivate(threadIdx, blockIdx, blockDim)
#define __syncthreads() ((void)0)

#include "macros.cu"
#include "data_types.cuh"
#include "solver.cu"

namespace {

struct RefState {
  int length[3];
  long n;
  Lattice lattice;
  Domain domain;
  double *f_store[Q];
  double *u_store[DIM];
  double *force_store[DIM];
  DomainConstant dc;
};

long node_count(const int *length) {
  long n = 1;
  for (int d = 0; d < DIM; d++) n *= length[d];
  return n;
}

}  // namespace

extern "C" {

int ref_q(void) { return Q; }
int ref_dim(void) { return DIM; }

// Returns the lattice tables as the reference loads them
// (model_builder.cu:69-73): e[DIM][Q] ints, omega[Q], opp[Q], M[Q][Q],
// M_inv[Q][Q].
void ref_tables(int *e, double *omega, int *opp, double *m, double *m_inv) {
  DomainConstant dc;
  memset(&dc, 0, sizeof(dc));
  LOAD_E(dc.e);
  LOAD_OMEGA(dc.omega);
  LOAD_OPP(dc.opp);
  LOAD_M(dc.M);
  LOAD_M_INV(dc.M_inv);
  memcpy(e, dc.e, sizeof(dc.e));
  memcpy(omega, dc.omega, sizeof(dc.omega));
  memcpy(opp, dc.opp, sizeof(dc.opp));
  memcpy(m, dc.M, sizeof(dc.M));
  memcpy(m_inv, dc.M_inv, sizeof(dc.M_inv));
}

// Builds one reference state.  Arrays are in the reference's natural index
// order ixd = x + y*Lx + z*Lx*Ly (solver.cu:23).  force/u are DIM*N
// (component-major), f_init is Q*N or NULL (then f = w_i, the reference's
// Init 0 state, model_builder.cu:233-248).  macro/micro codes may be NULL
// when the matching flag is off.
void *ref_create(const int *length, double tau, const double *tau_mrt,
                 double c_smag, int collision_type, int forcing, int macro_bc,
                 int micro_bc, const double *geometry, const double *force,
                 const int *macro_codes, const int *micro_codes,
                 const double *u, const double *rho, const double *f_init) {
  RefState *s = new RefState();
  memset(&s->dc, 0, sizeof(s->dc));
  for (int d = 0; d < 3; d++) s->length[d] = d < DIM ? length[d] : 1;
  s->n = node_count(length);
  const long n = s->n;
  DomainConstant &dc = s->dc;
  LOAD_E(dc.e);
  LOAD_OMEGA(dc.omega);
  LOAD_OPP(dc.opp);
  LOAD_M(dc.M);
  LOAD_M_INV(dc.M_inv);
  dc.tau = tau;
  for (int i = 0; i < Q; i++) dc.tau_mrt[i] = tau_mrt ? tau_mrt[i] : 0.0;
  for (int d = 0; d < DIM; d++) dc.length[d] = length[d];
  dc.forcing = forcing != 0;
  dc.macro_bc = macro_bc != 0;
  dc.micro_bc = micro_bc != 0;
  dc.collision_type = collision_type;
  dc.c_smag = c_smag;
  for (int i = 0; i < NUM_RESIDS; i++) dc.residual[i] = 1;

  for (int i = 0; i < Q; i++) {
    s->f_store[i] = (double *)malloc(sizeof(double) * n);
    for (long k = 0; k < n; k++)
      s->f_store[i][k] = f_init ? f_init[(long)i * n + k] : 1.0 * dc.omega[i];
  }
  for (int d = 0; d < DIM; d++) {
    s->u_store[d] = (double *)malloc(sizeof(double) * n);
    for (long k = 0; k < n; k++) s->u_store[d][k] = u ? u[(long)d * n + k] : 0.0;
    s->force_store[d] = (double *)malloc(sizeof(double) * n);
    for (long k = 0; k < n; k++)
      s->force_store[d][k] = force ? force[(long)d * n + k] : 0.0;
  }
  s->domain.rho = (double *)malloc(sizeof(double) * n);
  s->domain.geometry = (double *)malloc(sizeof(double) * n);
  s->domain.macro_bc = (int *)malloc(sizeof(int) * n);
  s->domain.micro_bc = (int *)malloc(sizeof(int) * n);
  for (long k = 0; k < n; k++) {
    s->domain.rho[k] = rho ? rho[k] : 0.0;
    s->domain.geometry[k] = geometry ? geometry[k] : 0.0;
    s->domain.macro_bc[k] = macro_codes ? macro_codes[k] : 0;
    s->domain.micro_bc[k] = micro_codes ? micro_codes[k] : 0;
  }
  s->lattice.f = s->f_store;
  s->domain.u = s->u_store;
  s->domain.force = s->force_store;
  return s;
}

// Runs nsteps reference iterations starting at time t0 (iterate(t) of
// index.cu:284 with t = t0, t0+1, ...).  store_macros applies to the last
// step only (earlier stores are overwritten by later ones in the reference).
void ref_run(void *h, int t0, int nsteps, int store_last, int nthreads) {
  RefState *s = (RefState *)h;
  domain_constants = s->dc;
  const int lx = s->length[0], ly = s->length[1], lz = s->length[2];
  if (nthreads > 0) omp_set_num_threads(nthreads);
  for (int step = 0; step < nsteps; step++) {
    const int t = t0 + step;
    const bool store = store_last && step == nsteps - 1;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < lz; z++) {
      for (int y = 0; y < ly; y++) {
        blockDim.x = 1; blockDim.y = 1; blockDim.z = 1;
        threadIdx.x = 0; threadIdx.y = 0; threadIdx.z = 0;
        blockIdx.y = y; blockIdx.z = z;
        for (int x = 0; x < lx; x++) {
          blockIdx.x = x;
          iterate_kernel(&s->lattice, &s->domain, store, t);
        }
      }
    }
  }
}

// Natural-layout populations after `t` completed steps: population i of node
// x is held in slot (x - t*e_i) mod L (solver.cu:82-94).
void ref_get_f(void *h, int t, double *out) {
  RefState *s = (RefState *)h;
  const int *L = s->length;
  const long n = s->n;
  for (int i = 0; i < Q; i++) {
    for (long k = 0; k < n; k++) {
      int c[3] = {(int)(k % L[0]), (int)((k / L[0]) % L[1]), (int)(k / ((long)L[0] * L[1]))};
      long src = 0, stride = 1;
      for (int d = 0; d < DIM; d++) {
        long v = ((long)c[d] - (long)t * s->dc.e[d][i]) % L[d];
        if (v < 0) v += L[d];
        src += v * stride;
        stride *= L[d];
      }
      out[(long)i * n + k] = s->f_store[i][src];
    }
  }
}

// The stored macroscopic fields (Domain.rho and Domain.u, written by
// solver.cu:126-134 on store steps).
void ref_get_macros(void *h, double *rho, double *u) {
  RefState *s = (RefState *)h;
  memcpy(rho, s->domain.rho, sizeof(double) * s->n);
  for (int d = 0; d < DIM; d++) memcpy(u + (long)d * s->n, s->u_store[d], sizeof(double) * s->n);
}

void ref_destroy(void *h) {
  RefState *s = (RefState *)h;
  for (int i = 0; i < Q; i++) free(s->f_store[i]);
  for (int d = 0; d < DIM; d++) {
    free(s->u_store[d]);
    free(s->force_store[d]);
  }
  free(s->domain.rho);
  free(s->domain.geometry);
  free(s->domain.macro_bc);
  free(s->domain.micro_bc);
  delete s;
}

}  // extern "C"
