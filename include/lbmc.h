/*
 * lbmc.h — C ABI of the B200 lattice Boltzmann time-step engine.
 *
 * This is the drop-in boundary for LBM-C's time-step path.  Each entry point
 * replaces one piece of the reference's host code (paths are relative to the
 * LBM-C project root):
 *
 *   lbmc_init      setup()            LBM-C/index.cu:157-186 and the
 *                  ModelBuilder       LBM-C/model_builder.cu:63-248
 *                  (constant upload, SoA allocation, field upload, Init 0)
 *   lbmc_iterate   iterate(int t)     LBM-C/index.cu:284-313 (one launch of
 *                  iterate_kernel, LBM-C/solver.cu:10-136, per time step)
 *   lbmc_fetch     output_macros      LBM-C/index.cu:196-216,
 *                  screen_mess        LBM-C/index.cu:412-432,
 *                  current_RMS        LBM-C/index.cu:338-373 (KE sum)
 *   lbmc_destroy   (none: the reference never frees its device state)
 *
 * Conventions kept from the reference:
 *   - node order ixd = x + y*Lx + z*Lx*Ly (LBM-C/solver.cu:23);
 *   - lattice velocity order, weights and opposites of LBM-C/macros.cu:19-53
 *     (D2Q9) and :71-119 (D3Q15);
 *   - ColType codes BGK=0, NTPOR=1, MRT=2, MRTPOR=3
 *     (LBM-C/infile_reader.cu:118-144);
 *   - MacroBC codes 1..15 (LBM-C/boundary_conditions/macro_bc.cu:12-17) and
 *     MicroBC codes 1..8 (D2Q9) / 1..12 (D3Q15)
 *     (LBM-C/boundary_conditions/micro_bc.cuh:7-15), used verbatim;
 *   - Porosity B >= 1 selects full-way bounceback (LBM-C/solver.cu:67-72);
 *   - the prescribed rho/u fields are also where stored macros are written
 *     (LBM-C/solver.cu:126-134 writes Domain.u/rho, which macro_bc.cu reads).
 *
 * Differences: every call returns an lbmc_status and never exits the process
 * (the reference calls exit(-1), LBM-C/cuda_util.cu:14-27); handles are
 * independent (the reference keeps one instance in file-scope globals,
 * LBM-C/index.cu:40-59); the step counter lives in the handle.
 *
 * Thread safety: calls on one handle must not overlap; separate handles may
 * be used from separate threads.
 */
#ifndef LBMC_H
#define LBMC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBMC_API_VERSION 1
#define LBMC_MAX_Q 15

typedef enum lbmc_status {
  LBMC_OK = 0,
  LBMC_ERR_INVALID_ARG = 1,  /* bad pointer, size, code or parameter */
  LBMC_ERR_UNSUPPORTED = 2,  /* valid input this build does not handle */
  LBMC_ERR_CUDA = 3,         /* CUDA runtime error; see lbmc_last_error() */
  LBMC_ERR_ALLOC = 4,        /* device or host allocation failed */
  LBMC_ERR_NAN = 5,          /* non-finite density/velocity detected */
  LBMC_ERR_TIMEOUT = 6,      /* a bounded device-side wait expired */
  LBMC_ERR_IO = 7,           /* file could not be read or parsed */
  LBMC_ERR_BUFFER_SIZE = 8,  /* destination buffer too small */
  LBMC_ERR_NO_DEVICE = 9     /* no usable CUDA device */
} lbmc_status;

typedef enum lbmc_lattice { LBMC_D2Q9 = 0, LBMC_D3Q15 = 1 } lbmc_lattice;

/* Population storage in HBM.  All formats hold f_i - w_i (deviation from the
 * rest-state weight); arithmetic is FP32, or FP64 for LBMC_F64.
 * LBMC_F16_SR is LBMC_F16 (same format and scale) whose step results are
 * written with stochastic rounding: each value rounds up with probability
 * equal to its distance from the FP16 value below it, from random bits that
 * depend only on (node, step, population), so runs are reproducible and
 * every streaming layout gives the same bits.  The initial upload rounds to
 * nearest.  Not available to the batched domains (lbmc_batch_*). */
typedef enum lbmc_storage {
  LBMC_F32 = 0,
  LBMC_F16 = 1,
  LBMC_BF16 = 2,
  LBMC_F64 = 3,
  LBMC_F16_SR = 4
} lbmc_storage;

/* ColType codes of LBM-C/infile_reader.cu:118-144. */
typedef enum lbmc_collision {
  LBMC_BGK = 0,
  LBMC_NTPOR = 1,
  LBMC_MRT = 2,
  LBMC_MRTPOR = 3
} lbmc_collision;

typedef enum lbmc_init_type {
  LBMC_INIT_STATIC = 0,      /* f = w_i (rho = 1, u = 0): the reference's Init 0 */
  LBMC_INIT_EQUILIBRIUM = 1, /* f = f_eq(rho, u) from lbmc_domain.rho / .u */
  LBMC_INIT_F = 2            /* f from lbmc_domain.f (restart / checkpoint) */
} lbmc_init_type;

typedef enum lbmc_streaming {
  LBMC_STREAM_SHIFT = 0, /* in place, population i of node x at (x - t e_i) mod L */
  LBMC_STREAM_AA = 1     /* in place, AA pattern (even/odd step index maps); over 64-node
                            tiles when Lx is a multiple of 64 (internal: lbmc_fetch and
                            LBMC_INIT_F always use natural order) */
} lbmc_streaming;

/* Reproduce documented reference defects exactly ("as-is" behaviour). */
#define LBMC_COMPAT_D3Q15_MINV_ZERO (1u << 0) /* macros.cu:97-115: D3Q15 MRT relaxes nothing */
#define LBMC_COMPAT_MEQ_INT_DIV (1u << 1)     /* collision.cu:492-496: (-7/3) evaluates to -2 */
#define LBMC_COMPAT_ZH_Z_UX (1u << 2)         /* d3q15_zh_defs.cu:87-91: -z Zou-He uses u[0] */
#define LBMC_COMPAT_MRTPOR_INPLACE (1u << 3)  /* collision.cu:340,416: blend reads updated f[opp] */
#define LBMC_COMPAT_REFERENCE_AS_IS                                              \
  (LBMC_COMPAT_D3Q15_MINV_ZERO | LBMC_COMPAT_MEQ_INT_DIV | LBMC_COMPAT_ZH_Z_UX | \
   LBMC_COMPAT_MRTPOR_INPLACE)

/* Mirrors the fields of DomainConstant (LBM-C/data_types.cuh:23-43) that the
 * input file sets, plus the engine's own choices. */
typedef struct lbmc_config {
  int lattice;          /* lbmc_lattice */
  int length[3];        /* Lx, Ly, Lz; Lz must be 1 for D2Q9 */
  double tau;           /* Tau */
  double tau_mrt[LBMC_MAX_Q]; /* TauMRT: MRT relaxation rates, first Q used */
  double c_smag;        /* C_smag; > 0 enables Smagorinsky (BGK family only) */
  int collision_type;   /* ColType, lbmc_collision */
  int forcing;          /* Force: Guo body force from lbmc_domain.force */
  int macro_bc;         /* MacroBC: per-node prescribed rho/u codes */
  int micro_bc;         /* MicroBC: per-node Zou-He / stress-free codes */
  int init_type;        /* Init, lbmc_init_type */
  double tolerance;     /* Tolerance (used by drivers, not by the step) */
  int h, dt;            /* DeltaX, DeltaT (carried, unused by the step, as in the reference) */
  int storage;          /* lbmc_storage */
  int streaming;        /* lbmc_streaming */
  unsigned compat;      /* LBMC_COMPAT_* bits */
  double storage_scale; /* stored value = (f - w) * scale; 0 selects the default (1024 for
                           FP16 and FP16_SR, 1 otherwise); FP16 and FP16_SR need a power of
                           two in [2^-15, 2^14] */
  int device;           /* CUDA device ordinal */
  int block_size;       /* reserved for tuning (0) */
  int kernel;           /* lbmc_kernel: 0 auto, 1 direct loads, 2 bulk-copy pipeline */
  int reserved[5];
} lbmc_config;

/* Step-kernel choice (lbmc_config.kernel).  AUTO and DIRECT run the
 * direct-load kernel; PIPELINED runs the bulk-copy (TMA) row pipeline, which
 * needs a population row to be a whole number of 16-byte granules and two
 * shared-memory stages of Q rows to fit (else lbmc_init fails with
 * LBMC_ERR_UNSUPPORTED). */
typedef enum lbmc_kernel {
  LBMC_KERNEL_AUTO = 0,
  LBMC_KERNEL_DIRECT = 1,
  LBMC_KERNEL_PIPELINED = 2
} lbmc_kernel;

/* Host arrays in ixd order; the caller keeps ownership, lbmc_init copies.
 * Mirrors Domain (LBM-C/data_types.cuh:13-21) plus the initial state. */
typedef struct lbmc_domain {
  const double *geometry; /* N: Porosity B in [0,1]; B >= 1 solid; NULL = all fluid */
  const double *force[3]; /* N each when forcing; NULL component = 0 */
  const int *macro_bc;    /* N MacroBC codes (0 = none) when macro_bc */
  const int *micro_bc;    /* N MicroBC codes (0 = none) when micro_bc */
  const double *u[3];     /* N each: prescribed velocity (macro BC) / initial velocity */
  const double *rho;      /* N: prescribed density (macro BC) / initial density */
  const double *f;        /* Q*N natural-layout populations for LBMC_INIT_F */
} lbmc_domain;

typedef struct lbmc_handle lbmc_handle;

/* lbmc_iterate flags. */
#define LBMC_STORE_MACROS (1u << 0) /* write rho/u on the last step of the call */
#define LBMC_REDUCE_DIAG (1u << 1)  /* FP64 mass/momentum/KE sums on the last step */
#define LBMC_SYNC (1u << 2)         /* wait for completion and report errors/NaN */

/* lbmc_fetch fields. */
typedef enum lbmc_field {
  LBMC_FIELD_RHO = 0, /* N doubles: stored density */
  LBMC_FIELD_U_X = 1, /* N doubles: stored velocity components */
  LBMC_FIELD_U_Y = 2,
  LBMC_FIELD_U_Z = 3,
  LBMC_FIELD_F = 4,   /* Q*N doubles: populations f_i in natural layout */
  LBMC_FIELD_DIAG = 5 /* one lbmc_diag */
} lbmc_field;

typedef struct lbmc_diag {
  double mass;           /* sum of rho over all nodes (solids hold rho = 0) */
  double momentum[3];    /* sum of rho*u */
  double kinetic_energy; /* sum of 0.5*rho*|u|^2, current_RMS (index.cu:338-373) */
  long long step;        /* completed steps when the sums were taken */
  int nonfinite;         /* 1 if any rho or u was NaN/Inf */
  int valid;             /* 1 once a LBMC_REDUCE_DIAG step has run */
} lbmc_diag;

/* Fills cfg with the reference's defaults for a lattice (c_smag = 0 as in
 * InfileReader::initialise, LBM-C/infile_reader.cu:20-23). */
lbmc_status lbmc_config_default(lbmc_config *cfg, int lattice);

/* Replaces setup() (LBM-C/index.cu:157-186) and ModelBuilder
 * (LBM-C/model_builder.cu:257-278).  Rejects what lbmc_validate rejects,
 * with the same status and message: configuration errors before any device
 * work, per-node input errors (codes, porosity, fields a code needs) once
 * the host's check of the arrays, which runs while rho and u upload, ends;
 * nothing is left allocated on failure. */
lbmc_status lbmc_init(const lbmc_config *cfg, const lbmc_domain *dom,
                      lbmc_handle **out);

/* Replaces nsteps calls of iterate(t) (LBM-C/index.cu:284-313).  The step
 * counter t continues across calls.  Without LBMC_SYNC the call only
 * enqueues work on the handle's stream. */
lbmc_status lbmc_iterate(lbmc_handle *h, int nsteps, unsigned flags);

/* Replaces the device-to-host copies of output_macros / screen_mess /
 * compute_residual (LBM-C/index.cu:196-216, 412-432, 387-409).  Blocks until
 * the handle's stream is idle. */
lbmc_status lbmc_fetch(lbmc_handle *h, int field, void *dst, size_t bytes);

lbmc_status lbmc_destroy(lbmc_handle *h);

/* Completed time steps (the t the next step will use). */
lbmc_status lbmc_get_step(lbmc_handle *h, long long *step);

/* Runs the handle's work on a caller stream (a cudaStream_t); NULL = the
 * handle's own stream. */
lbmc_status lbmc_set_stream(lbmc_handle *h, void *cuda_stream);

lbmc_status lbmc_synchronize(lbmc_handle *h);

const char *lbmc_status_string(lbmc_status s);

/* Failure-detection self-test: launches a kernel whose bounded wait on a
 * barrier that is never signalled gives up after `seconds` (<= 10) and
 * returns LBMC_ERR_TIMEOUT; the context stays usable.  The bulk-copy step
 * kernel uses the same bounded wait and reports LBMC_ERR_TIMEOUT from
 * lbmc_iterate(..., LBMC_SYNC) the same way.  No counterpart in the
 * reference, which has no device-side waits. */
lbmc_status lbmc_selftest_wait_timeout(int device, double seconds);

/* FP64 sums of rho, rho*u and 0.5*rho*|u|^2 (the lbmc_diag quantities) over
 * n nodes of caller-owned device arrays, written to sums[0..4] (device
 * memory: mass, momentum x/y/z, kinetic energy), ordered on cuda_stream
 * (NULL = legacy default stream).  No counterpart in the reference: it is
 * for callers that cannot allocate device memory when they need the sums
 * (an application whose own pool allocator already holds the device memory,
 * a process under a device-memory cap, a time loop that must avoid
 * cudaMalloc's implicit synchronisation).  It allocates nothing: its
 * per-block scratch is a fixed 320 KiB array in the library's device image,
 * so n is limited to 134,217,728 nodes (512^3); larger n, NULL rho/ux/sums
 * or n < 1 return LBMC_ERR_INVALID_ARG.  uy/uz may be NULL (zero).  The
 * first call on a device looks up the scratch array's address (make it
 * before any stream capture).  Calls share the scratch: calls whose kernels
 * overlap on the GPU race; stream-ordered calls do not. */
lbmc_status lbmc_macro_sums_noalloc(int device, const double *rho, const double *ux,
                                    const double *uy, const double *uz, long long n,
                                    double *sums, void *cuda_stream);

/* ---------------- batched small domains (no reference counterpart) -------
 * Thousands of independent D2Q9 domains with the same physics (BGK or
 * NTPOR + uniform Guo force, Init 0) stepped by one persistent kernel
 * replayed from a CUDA graph until every domain's max |u(t) - u(t-1)| falls
 * below a tolerance.  Each domain evolves exactly as one lbmc handle would. */
typedef struct lbmc_batch lbmc_batch;

typedef struct lbmc_batch_config {
  double tau;
  double force[2];      /* uniform Guo body force */
  int collision_type;   /* LBMC_BGK or LBMC_NTPOR */
  int storage;          /* LBMC_F32, LBMC_F16 or LBMC_BF16 */
  double storage_scale; /* 0 = default (1024 for FP16); FP16: a power of two in [2^-15, 2^14] */
  int device;
  int block_threads;    /* 0 = autotune (256/512/1024) */
  int steps_per_launch; /* 0 = autotune (check_every or 4*check_every) */
  int wide_min_nodes;   /* domains too large for shared memory with at least this many nodes
                           are stepped one step per launch over every SM, the others one block
                           per domain, K steps per launch; 0 = default (FP32: 32768;
                           FP16/BF16: none) */
  int wide_below;       /* the one-block-per-domain ones join the wide path once fewer than
                           this many of them are running; 0 = default (half the SMs), < 0 =
                           never */
  int reserved[6];
} lbmc_batch_config;

typedef struct lbmc_batch_domain {
  int length[2];            /* Lx, Ly; Lx * Ly <= 2^24 */
  const double *geometry;   /* Lx*Ly Porosity B: 0 fluid, (0,1) partial, >= 1 solid; NULL = fluid */
} lbmc_batch_domain;

typedef struct lbmc_batch_result {
  long long steps;    /* steps run */
  double delta_u;     /* last max |u(t) - u(t-1)| measured (NaN once non-finite) */
  double elapsed_ms;  /* device time from the run's start to convergence, -1 if not converged */
  int converged;      /* 1 if delta_u < tol was reached before the step cap */
  int nonfinite;      /* 1 if the domain's velocity became NaN/Inf; it was stopped there */
} lbmc_batch_result;

lbmc_status lbmc_batch_init(const lbmc_batch_config *cfg, int ndomains,
                            const lbmc_batch_domain *doms, lbmc_batch **out);
/* Runs until every domain converged (delta_u < tol, checked every
 * check_every steps), reached max_steps or became non-finite; results has
 * ndomains entries.  A domain whose velocity turns NaN/Inf is stopped at the
 * next check and flagged; the call then returns LBMC_ERR_NAN after filling
 * results (the reference's NaN exit, LBM-C/index.cu:130-133). */
lbmc_status lbmc_batch_run(lbmc_batch *b, long long max_steps, double tol, int check_every,
                           lbmc_batch_result *results);
/* LBMC_FIELD_RHO / U_X / U_Y (N doubles; u = j/rho) or LBMC_FIELD_F (9N). */
lbmc_status lbmc_batch_fetch(lbmc_batch *b, int domain, int field, void *dst, size_t bytes);
/* Launch shape chosen by the autotuner and how many domains stay in shared memory. */
lbmc_status lbmc_batch_info(lbmc_batch *b, long long *total_nodes, int *threads,
                            int *steps_per_launch, int *resident_domains);
lbmc_status lbmc_batch_destroy(lbmc_batch *b);

/* ---------------- learned subgrid closure (no reference counterpart) ------
 * A 6 -> 32 -> 32 -> 1 SiLU MLP (1313 parameters, BF16 weights, FP32
 * accumulation) maps six invariants of the local strain-rate estimate to an
 * eddy viscosity nu_t; tau_eff = tau + 3 nu_t.  Trained on the GPU by the
 * library's own forward/backward/Adam kernels.  Attached to a BGK-family
 * handle it replaces Smagorinsky (LBM-C/collision.cu:445-463), which stays
 * the fallback wherever the inputs leave the training range. */
typedef struct lbmc_mlp lbmc_mlp;

lbmc_status lbmc_mlp_create(int device, unsigned long long seed, lbmc_mlp **out);
/* Input normalisation x = (f - mean)/std, the normalised training range
 * [lo, hi] per input (NULL = unbounded) and the target scale
 * (nu_t = target_scale * output). */
lbmc_status lbmc_mlp_set_normalization(lbmc_mlp *m, const float *mean, const float *std,
                                       const float *lo, const float *hi, float target_scale);
/* Six features per sample from strain tensors S (xx, yy, zz, xy, yz, xz) and
 * densities (NULL = 1), computed by the same device function the step uses. */
lbmc_status lbmc_mlp_features(int device, const float *strain6, const float *rho, long long n,
                              float *features6);
/* Mini-batch Adam on the mean squared error between target_scale * output
 * and target; features are raw (normalised inside).  loss_history: epochs
 * floats or NULL. */
lbmc_status lbmc_mlp_train(lbmc_mlp *m, const float *features, const float *target, long long n,
                           int epochs, int batch, float lr, float *loss_history);
/* Gradient (1313 floats, parameter layout W1[32x6], b1, W2[32x32], b2, W3,
 * b3) and value of the loss over one batch of n samples. */
lbmc_status lbmc_mlp_gradients(lbmc_mlp *m, const float *features, const float *target, long long n,
                               float *grads, float *loss);
lbmc_status lbmc_mlp_predict(lbmc_mlp *m, const float *features, long long n, float *out);
/* The same prediction as the step computes it: warp-wide on the tensor
 * cores, BF16 inputs and activations, FP32 accumulation, BF16 SiLU. */
lbmc_status lbmc_mlp_predict_step(lbmc_mlp *m, const float *features, long long n, float *out);
lbmc_status lbmc_mlp_get_params(lbmc_mlp *m, float *params);
lbmc_status lbmc_mlp_set_params(lbmc_mlp *m, const float *params);
lbmc_status lbmc_mlp_destroy(lbmc_mlp *m);
/* Attaches (m != NULL) or detaches (m == NULL) the learned closure on a
 * BGK-family handle; iterations = fixed-point passes for tau_eff (1..8). */
lbmc_status lbmc_set_closure(lbmc_handle *h, const lbmc_mlp *m, int iterations);

/* Host-only helpers (no GPU needed). */

/* Checks a configuration and domain the way lbmc_init does, without touching
 * the GPU (the reference validates nothing and crashes on bad codes, e.g. the
 * NULL D2Q9 MicroBC entries 3 and 4 of micro_bc.cuh:7-8). */
lbmc_status lbmc_validate(const lbmc_config *cfg, const lbmc_domain *dom);

/* The per-node class bytes and class table lbmc_init would upload: class 0
 * plain fluid, 1 solid (Porosity >= 1), >= 2 an index into table, whose
 * entries pack MacroBC (bits 0-3), MicroBC (bits 4-7) and a partial-solid
 * bit (bit 8).  cls_out holds N bytes, table_out 256 entries. */
lbmc_status lbmc_classify(const lbmc_config *cfg, const lbmc_domain *dom, uint8_t *cls_out,
                          uint16_t *table_out, int *nclasses);

/* Lattice tables as the kernels use them: e[DIM*Q] (row per axis), w[Q],
 * opp[Q], M[Q*Q] (LBM-C/macros.cu:19-53, 71-119). */
lbmc_status lbmc_lattice_tables(int lattice, int *e, double *w, int *opp, int *m);

/* Message of the last error on the calling thread ("" if none). */
const char *lbmc_last_error(void);

/* ------------------------------------------------------------------------
 * Run control: the reference's front end (input file, model builder, output
 * handler, driver loop) around the step.
 * ------------------------------------------------------------------------ */

/* Stored macros of one node (rho, u_x, u_y, u_z) as of the last
 * LBMC_STORE_MACROS step: the single-node read of screen_mess
 * (LBM-C/index.cu:412-439). */
lbmc_status lbmc_probe(lbmc_handle *h, long long node, double out[4]);

#define LBMC_PATH_MAX 256

/* Everything an input file sets.  Replaces the reference's DomainConstant
 * fields, Timing, OutputController and ProjectStrings as filled by
 * InfileReader (LBM-C/infile_reader.cu:45-226, LBM-C/data_types.cuh:57-79). */
typedef struct lbmc_run_config {
  lbmc_config cfg;                  /* Tau, TauMRT, Lx/Ly/Lz, C_smag, ColType, Force,
                                       MicroBC, MacroBC, Tolerance, Init, DeltaX, DeltaT */
  char project_name[LBMC_PATH_MAX]; /* ProjName */
  char domain_file[LBMC_PATH_MAX];  /* DomainFile */
  char output_file[LBMC_PATH_MAX];  /* OutputFile */
  int max_t;                        /* MaxT: steps */
  int file_out;                     /* FileOut: output every n steps (0 = never) */
  int screen_mes;                   /* ScreenMes: screen line every n steps */
  int steady_check;                 /* SteadyCheck: residual every n steps */
  int output_u[3], output_rho, output_pressure; /* OutputVars */
  int screen_node[3];               /* ScreenNode */
  int interactive;                  /* Interactive (read and reported; no pauses) */
  int lz_given;                     /* an Lz line was read */
  int lattice_given;                /* a Lattice line (D2Q9 / D3Q15) was read */
  int tau_mrt_count;                /* values read from TauMRT */
} lbmc_run_config;

/* Reads an input file the way InfileReader does: for each line, the text
 * before '#' is matched against the keys in the reference's order by
 * substring (ProjName, DomainFile, OutputFile, TauMRT, Tau, Lx, Ly, Lz,
 * DeltaX, DeltaT, C_smag, ColType, Force, MicroBC, MacroBC, Tolerance, Init,
 * MaxT, FileOut, ScreenMes, SteadyCheck, OutputVars, ScreenNode,
 * Interactive); the first token is the name, the values follow.  Extension:
 * a "Lattice D2Q9|D3Q15" line; without it the lattice is D3Q15 when an Lz
 * line gives Lz > 1, else D2Q9 (the reference fixes DIM at compile time and
 * ignores Lz in 2-D builds).  `echo` (may be NULL) receives the report the
 * reference prints, "name = value" per line. */
lbmc_status lbmc_read_input(const char *path, lbmc_run_config *rc, char *echo, size_t echo_bytes);

/* Host arrays of a model, read from the domain directory named by
 * DomainFile: one NumPy .npy file per field, named as the reference's CGNS
 * fields (ModelBuilder::variable_loader, LBM-C/model_builder.cu:173-231):
 * Porosity; ForceX/ForceY/ForceZ when Force; MicroBC when MicroBC; MacroBC,
 * VelocityX/Y/Z and Rho when MacroBC; VelocityX/Y/Z and Rho for Init 1
 * (equilibrium); Populations (Q x N) for Init 2.  Arrays are float64,
 * float32, int32 or int64, C order, N = Lx Ly Lz elements in the node order
 * x + Lx (y + Ly z).  A missing Porosity file means all fluid. */
typedef struct lbmc_model lbmc_model;
lbmc_status lbmc_model_build(const lbmc_run_config *rc, lbmc_model **out);
/* Pointers into the model's arrays, valid until lbmc_model_free. */
lbmc_status lbmc_model_domain(const lbmc_model *m, lbmc_domain *dom);
void lbmc_model_free(lbmc_model *m);

/* Solution output with the structure of the reference's CGNS output
 * (CGNSOutputHandler, LBM-C/cgns/cgns_output_handler.cu:62-293): base
 * "Base", structured zone "LBM-C Output Data" with an (L+1)^dim vertex grid
 * (RealSingle CoordinateX/Y/Z), one cell-centred FlowSolution "Solution @
 * Time = N" per output with RealDouble fields, and the iteration values and
 * FlowSolutionPointers of BaseIterativeData / ZoneIterativeData.  No CGNS
 * library is available to this build, so the tree is written as a
 * directory: index.json (the tree), GridCoordinates/Coordinate?.npy and
 * "Solution @ Time = N"/<field>.npy. */
typedef struct lbmc_output lbmc_output;
lbmc_status lbmc_output_open(const char *path, int dim, const int length[3], lbmc_output **out);
lbmc_status lbmc_output_append(lbmc_output *o, long long step, int nfields, const double *const *data,
                               const char *const *labels);
/* Writes the iterative data and closes. */
lbmc_status lbmc_output_close(lbmc_output *o);

/* Result of a driver run. */
typedef struct lbmc_run_result {
  long long steps;     /* steps taken */
  int steady;          /* stopped by the steady-state test */
  int nonfinite;       /* stopped on a non-finite state (the reference exits with 1) */
  int outputs;         /* solutions written */
  double residual[3];  /* the last NUM_RESIDS residuals */
  double seconds;      /* wall clock of the time loop */
} lbmc_run_result;

/* The reference's main() (LBM-C/index.cu:61-153): read the input file,
 * build the model, run MaxT steps with output every FileOut steps, a screen
 * line every ScreenMes steps and the steady-state test every SteadyCheck
 * steps (residual = |KE - KE_prev| / SteadyCheck / KE from the fused FP64
 * kinetic-energy sum; stop when the last three are below Tolerance, with an
 * output; on a non-finite state write an output and stop).  Macros are
 * stored only on the steps that use them (the reference stores on nearly
 * every step when SteadyCheck > 0, defect Q7).  `cfg_overrides` (may be
 * NULL) supplies storage, streaming, device and kernel in place of the
 * defaults.  quiet = 1 suppresses the screen report. */
lbmc_status lbmc_run(const char *input_path, const lbmc_config *cfg_overrides, int quiet,
                     lbmc_run_result *res);

#ifdef __cplusplus
}
#endif

#endif /* LBMC_H */
