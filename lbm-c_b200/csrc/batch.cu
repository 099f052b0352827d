// Batched persistent step for many independent small D2Q9 domains
// (lbmc_batch_*).  No counterpart in the reference, which runs one domain per
// process; each domain here is stepped exactly as lbmc_iterate steps a single
// domain (the shift layout with FP32 storage and the AA pattern of
// LBMC_STREAM_AA with 2-byte storage, the same collide_fluid), so parity is
// inherited.
//
// Execution model.  Domains whose populations fit in a block's shared
// memory are stepped by one persistent kernel: blocks take whole domains
// from an atomic queue (largest first), load one, step it K times in shared
// memory (the step-to-step dependency is a __syncthreads) and write it back,
// so K steps cost one read and one write of HBM.  Larger domains are
// stepped in HBM in one of two ways, by size (wide_min_nodes):
//   - one block per domain, K steps per launch (the same persistent kernel
//     without the shared-memory copy): a domain's K steps run back to back,
//     so a 2-byte domain of moderate size is re-read from cache;
//   - over every SM, one step per launch (batch_wide_kernel: one warp per
//     segment of consecutive nodes, every listed domain in one launch),
//     followed by a one-thread-per-domain kernel (batch_wide_finish_kernel)
//     for the convergence test and step accounting.  Large domains need the
//     most steps and would otherwise finish last on one SM each.
// One CUDA graph launch holds the shared-memory kernel in one branch and the
// block-stepped kernel followed by K wide step pairs in the other.  Every C
// steps a domain compares u with its value C steps earlier (max norm) and
// freezes once below the tolerance, recording the device timer.  The host
// replays the graph until every domain converged, stopped or hit the step
// cap.  Once fewer than wide_below block-stepped domains run, they join the
// wide path; whenever a quarter of the listed wide domains have stopped,
// the segments are rebuilt and the graph re-captured, so launches stop
// visiting them.  An autotuner times the first launches with several block
// sizes and two values of K, and keeps the fastest.  The same node update
// runs in every kernel, so results do not depend on where a step ran.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/lbmc.h"
#include "engine_internal.h"
#include "kernels.cuh"

using namespace lbmc;

namespace {

struct BatchDomainDev {
  long long pop_off;   // element offset of population 0 in the pool
  long long node_off;  // offset into class / porosity / u_prev arrays
  int pitch;           // elements between populations (global)
  int lx, ly;
  int resident;        // fits in shared memory
};

struct BatchStateDev {
  long long t;                  // steps done
  float delta_u;                // last max |u(t) - u(t-1)| (NaN once non-finite)
  int converged;                // 1 converged, 2 stopped at the step cap, 3 stopped non-finite
  unsigned long long done_ns;   // device timer at convergence
};

struct BatchArgs {
  void *pool;
  const uint8_t *cls;
  const float *B;
  float2 *u_prev;
  const BatchDomainDev *dom;
  BatchStateDev *state;
  const int *order;          // this kernel's domains, largest first
  int ndomains;              // entries in order
  int *queue;                // this kernel's atomic work counter (reset before each launch)
  int *active;               // domains still running after this launch (both kernels)
  int *active_hbm;           // of which stepped in HBM
  int steps;                 // K: steps per launch per domain
  int check;                 // C: convergence check interval
  float tol;
  long long max_steps;
  float tau, force[2];
  float omega;               // 1/tau
  float guo_a[9], guo_b[9], guo_odd[9];  // uniform-force Guo terms (StepArgs)
  float scale, inv_scale;
  int blend;
  size_t smem_elems;         // capacity of the shared-memory population buffer
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// One D2Q9 node in the AA pattern (one array per population, in place;
// 2-byte storage, see batch_aa below):
// at an even step the node reads population i from its own slot of array i
// and writes out[i] to its own slot of array opp(i); at an odd step it reads
// population i from array opp(i) at x - e_i and writes out[i] to array i at
// x + e_i (periodic wrap).  A node writes exactly the slots it read, so the
// update is race-free in place, and the state after every step equals the
// shift layout's up to where the values sit (the single-domain engine's
// LBMC_STREAM_AA maps).  Collide, write back; returns u = j/rho + F/(2 rho)
// in `u` (the stored velocity of LBM-C/collision.cu:77).
template <class S, bool BLEND, bool ODD>
__device__ __forceinline__ void batch_node_aa(S *pop, long long pitch, int k, int x, int y, int lx, int ly,
                                              int cls, const StepArgs<float> &a, float &ux, float &uy) {
  using L = D2Q9;
  int xs[3] = {x, x, x}, ys[3] = {y, y, y};
  if constexpr (ODD) {
    xs[1] = wrap_sub(x, 1, lx);
    xs[2] = wrap_add(x, 1, lx);
    ys[1] = wrap_sub(y, 1, ly);
    ys[2] = wrap_add(y, 1, ly);
  }
  Node<L, float> nd;
  unroll<9>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    if constexpr (ODD) {
      const int slot = xs[sel(L::e(0, i))] + lx * ys[sel(L::e(1, i))];
      nd.g[i] = load_dev(pop + L::opp(i) * pitch + slot, a.inv_scale);
    } else {
      nd.g[i] = load_dev(pop + i * pitch + k, a.inv_scale);
    }
  });
  float out[9];
  if (cls == CLASS_SOLID) {
    collide_solid(nd, out);
  } else {
    moments(nd);
    // a.B is this domain's porosity array; only partial nodes read it.
    collide_fluid<L, float, COL_BGK, true, BLEND, true>(nd, a, k, cls == 2 ? ENTRY_PARTIAL : 0u, out);
  }
  if constexpr (ODD) {
    // The store slots equal the load slots; recomputing them from the six
    // coordinates is cheaper than keeping nine addresses live across the
    // collision (the empty asm hides the equality from the compiler).
    int xw[3] = {xs[0], xs[1], xs[2]}, yw[3] = {ys[0], ys[1], ys[2]};
    asm("" : "+r"(xw[0]), "+r"(xw[1]), "+r"(xw[2]), "+r"(yw[0]), "+r"(yw[1]), "+r"(yw[2]));
    unroll<9>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      constexpr int o = L::opp(i);
      const int slot = xw[sel(L::e(0, o))] + lx * yw[sel(L::e(1, o))];
      store_smem(pop + i * pitch + slot, out[i], a.scale);
    });
  } else {
    unroll<9>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      store_smem(pop + L::opp(i) * pitch + k, out[i], a.scale);
    });
  }
  ux = nd.u[0];
  uy = nd.u[1];
}

// One D2Q9 node: load its 9 shift slots from `pop` (pitch elements apart),
// collide, write back; returns u = j/rho + F/(2 rho) in `u` (the stored
// velocity of LBM-C/collision.cu:77).
template <class S, bool BLEND>
__device__ __forceinline__ void batch_node_shift(S *pop, long long pitch, int k, int x, int y, int lx, int ly,
                                                 int sx, int sy, int cls, const StepArgs<float> &a,
                                                 float &ux, float &uy) {
  using L = D2Q9;
  const int xs[3] = {x, wrap_sub(x, sx, lx), wrap_add(x, sx, lx)};
  const int ys[3] = {y, wrap_sub(y, sy, ly), wrap_add(y, sy, ly)};
  Node<L, float> nd;
  unroll<9>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    const int slot = xs[sel(L::e(0, i))] + lx * ys[sel(L::e(1, i))];
    nd.g[i] = load_dev(pop + i * pitch + slot, a.inv_scale);
  });
  float out[9];
  if (cls == CLASS_SOLID) {
    collide_solid(nd, out);
  } else {
    moments(nd);
    // a.B is this domain's porosity array; only partial nodes read it.
    collide_fluid<L, float, COL_BGK, true, BLEND, true>(nd, a, k, cls == 2 ? ENTRY_PARTIAL : 0u, out);
  }
  // The store slots equal the load slots; recomputing them from the six
  // coordinates is cheaper than keeping nine addresses live across the
  // collision (the empty asm hides the equality from the compiler).
  int xw[3] = {xs[0], xs[1], xs[2]}, yw[3] = {ys[0], ys[1], ys[2]};
  asm("" : "+r"(xw[0]), "+r"(xw[1]), "+r"(xw[2]), "+r"(yw[0]), "+r"(yw[1]), "+r"(yw[2]));
  unroll<9>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    const int slot = xw[sel(L::e(0, i))] + lx * yw[sel(L::e(1, i))];
    store_smem(pop + i * pitch + slot, out[i], a.scale);
  });
  ux = nd.u[0];
  uy = nd.u[1];
}

// The layout of the batched domains, per storage format.  Measured on the
// 4096-domain sweep (first 20,000 steps, one B200): 2-byte storage 80.1
// GLUPS in the shift layout, 84.9 in the AA pattern; FP32 55.4 shift, 51.1-53.9
// AA (its wide kernel, which FP16 does not use by default, holds both AA
// maps and spills or loses occupancy at its register cap).
template <class S>
__host__ __device__ constexpr bool batch_aa() {
  return sizeof(S) == 2;
}

// The step of node k at step t: shift t mod (lx, ly) or AA parity t & 1.
template <class S, bool BLEND>
__device__ __forceinline__ void batch_node(S *pop, long long pitch, int k, int x, int y, int lx, int ly,
                                           int sx, int sy, bool odd, int cls, const StepArgs<float> &a,
                                           float &ux, float &uy) {
  if constexpr (batch_aa<S>()) {
    if (odd) batch_node_aa<S, BLEND, true>(pop, pitch, k, x, y, lx, ly, cls, a, ux, uy);
    else batch_node_aa<S, BLEND, false>(pop, pitch, k, x, y, lx, ly, cls, a, ux, uy);
  } else {
    batch_node_shift<S, BLEND>(pop, pitch, k, x, y, lx, ly, sx, sy, cls, a, ux, uy);
  }
}

// The convergence measure keeps a non-finite velocity visible: fmaxf
// returns its non-NaN operand, which would let a diverged domain read as
// converged, so the maxima below propagate NaN and a non-finite velocity
// counts as NaN.
constexpr int STOP_CONVERGED = 1, STOP_CAP = 2, STOP_NONFINITE = 3;

__device__ __forceinline__ float nan_max(float a, float b) { return (b != b || b > a) ? b : a; }

__device__ __forceinline__ float node_delta(float ux, float uy, float2 p) {
  if (!(isfinite(ux) && isfinite(uy))) return __int_as_float(0x7fffffff);  // positive quiet NaN
  return fmaxf(fabsf(ux - p.x), fabsf(uy - p.y));
}

// Convergence test of one domain from its max |u(t) - u(t - C)|.
__device__ __forceinline__ int stop_code(float m, float tol) {
  if (m != m) return STOP_NONFINITE;
  return m < tol ? STOP_CONVERGED : 0;
}

__device__ __forceinline__ float block_max(float v, float *sh) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = nan_max(v, __shfl_xor_sync(0xffffffffu, v, off));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  float r = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); w++) r = nan_max(r, sh[w]);
  return r;
}

// RESIDENT: the domains of this launch fit in shared memory (one block per
// SM with the full shared-memory carve-out); otherwise they are stepped in
// HBM by several smaller blocks per SM with no dynamic shared memory.
template <class S, bool BLEND, bool RESIDENT>
__global__ void __launch_bounds__(1024) batch_kernel(const BatchArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int sh_dom;
  __shared__ float sh_red[32];
  __shared__ int sh_stop;
  S *sbuf = reinterpret_cast<S *>(smem_raw);
  S *pool = reinterpret_cast<S *>(A.pool);
  StepArgs<float> a;
  memset(&a, 0, sizeof(a));
  a.tau = A.tau;
  a.omega = A.omega;
  for (int i = 0; i < 9; i++) {
    a.guo_a[i] = A.guo_a[i];
    a.guo_b[i] = A.guo_b[i];
    a.guo_odd[i] = A.guo_odd[i];
  }
  a.force_u[0] = A.force[0];
  a.force_u[1] = A.force[1];
  a.scale = A.scale;
  a.inv_scale = A.inv_scale;
  for (;;) {
    if (threadIdx.x == 0) {
      const int q = atomicAdd(A.queue, 1);
      sh_dom = q < A.ndomains ? A.order[q] : -1;
    }
    __syncthreads();
    const int d = sh_dom;
    __syncthreads();
    if (d < 0) break;
    BatchStateDev &st = A.state[d];
    if (st.converged) continue;
    const BatchDomainDev D = A.dom[d];
    const int n = D.lx * D.ly;
    const uint8_t *cls = A.cls + D.node_off;
    a.B = A.B + D.node_off;
    float2 *up = A.u_prev + D.node_off;
    S *pop = pool + D.pop_off;
    long long pitch = D.pitch;
    if (RESIDENT) {
      for (int i = 0; i < 9; i++)
        for (int k = threadIdx.x; k < n; k += blockDim.x) sbuf[(long long)i * n + k] = pop[(long long)i * D.pitch + k];
      pop = sbuf;
      pitch = n;
      __syncthreads();
    }
    long long t = st.t;
    int stop = 0;
    for (int s = 0; s < A.steps && !stop; s++, t++) {
      const int sx = batch_aa<S>() ? 0 : (int)(t % D.lx), sy = batch_aa<S>() ? 0 : (int)(t % D.ly);
      const bool odd = t & 1;
      // Every C steps: du = max |u(t) - u(t - C)|, then u(t) is kept for the
      // next check.  Reduced-precision dynamics that settle into a fixed point
      // or a cycle whose period divides C give exactly zero.
      const bool save = (t % A.check) == 0;
      const bool test = save && t >= A.check;
      float dmax = 0;
      // (x, y) of node k advance by the block size without a division per node.
      int x = (int)threadIdx.x % D.lx, y = (int)threadIdx.x / D.lx;
      const int step_x = (int)blockDim.x % D.lx, step_y = (int)blockDim.x / D.lx;
      for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int c = cls[k];
        float ux, uy;
        batch_node<S, BLEND>(pop, pitch, k, x, y, D.lx, D.ly, sx, sy, odd, c, a, ux, uy);
        if (test) dmax = nan_max(dmax, node_delta(ux, uy, up[k]));
        if (save) up[k] = make_float2(ux, uy);
        x += step_x;
        y += step_y;
        if (x >= D.lx) {
          x -= D.lx;
          y += 1;
        }
      }
      __syncthreads();
      if (test) {
        const float m = block_max(dmax, sh_red);
        if (threadIdx.x == 0) {
          st.delta_u = m;
          sh_stop = stop_code(m, A.tol);
        }
        __syncthreads();
        stop = sh_stop;
      }
      if (t + 1 >= A.max_steps) stop = stop ? stop : STOP_CAP;
    }
    if (RESIDENT) {
      __syncthreads();
      for (int i = 0; i < 9; i++)
        for (int k = threadIdx.x; k < n; k += blockDim.x)
          Storage<S>::put_any(pool + D.pop_off + (long long)i * D.pitch + k, Storage<S>::get(sbuf + (long long)i * n + k));
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      st.t = t;
      if (stop) {
        st.converged = stop;
        st.done_ns = global_ns();
      } else {
        atomicAdd(A.active, 1);
        if (!RESIDENT) atomicAdd(A.active_hbm, 1);
      }
    }
    __syncthreads();
  }
}

__global__ void stamp_kernel(unsigned long long *out) { *out = global_ns(); }

// Wide phase: one step of the listed HBM domains per launch over every SM.
// The work is cut into segments of WIDE_ITERS x 32 consecutive nodes of a
// domain (node index k = x + lx y), one per warp, two warps per block, one
// block per two segments; a warp loads a segment's descriptors once and
// steps 32 nodes per iteration.  A segment records the (x, y) of its first
// node; a lane adds its offset to x and wraps into the next row when x
// passes lx, so no node index is divided, and only the last segment of a
// domain has idle lanes.
// The convergence test's warp maxima go to acc[domain] (non-negative
// floats compare as their bit patterns, and the positive NaN of a
// non-finite velocity is above every one of them).
constexpr int WIDE_THREADS = 64;
constexpr int WIDE_WARPS = WIDE_THREADS / 32;
constexpr int WIDE_ITERS = 1;  // a segment is WIDE_ITERS x 32 consecutive nodes, one warp's work
struct RowSegment {
  int domain, y, x0;  // first node (x0, y) of the segment
};
// What the next step of a listed domain needs, prepared once per domain and
// step (by the host when the list is built, then by the finish kernel), so
// that no warp divides the 64-bit step counter: the shift t mod (lx, ly),
// the parity of t (AA) and the flags below.
struct WideStep {
  int sx, sy;
  int flags;
};
constexpr int WIDE_RUNNING = 1, WIDE_SAVE = 2, WIDE_TEST = 4, WIDE_ODD = 8;

__host__ __device__ inline WideStep wide_step(long long t, int lx, int ly, int check, bool running) {
  WideStep w;
  w.sx = (int)(t % lx);
  w.sy = (int)(t % ly);
  const bool save = (t % check) == 0;
  w.flags = (running ? WIDE_RUNNING : 0) | (save ? WIDE_SAVE : 0) | (save && t >= check ? WIDE_TEST : 0) |
            ((t & 1) ? WIDE_ODD : 0);
  return w;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = nan_max(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}

// Resident blocks of the wide kernel per SM: the register cap of 20 blocks
// (48 registers) holds the shift step; the AA step (both maps in one kernel)
// spills 28-76 bytes there and 0-24 at 18 blocks (56 registers).
template <class S>
constexpr int wide_min_blocks() {
  return batch_aa<S>() ? 18 : 20;
}

template <class S, bool BLEND>
__global__ void __launch_bounds__(WIDE_THREADS, (wide_min_blocks<S>()))
    batch_wide_kernel(const BatchArgs A, const RowSegment *segs, int nsegs, const WideStep *steps, int *acc) {
  const int si = blockIdx.x * WIDE_WARPS + (int)(threadIdx.x >> 5);
  if (si >= nsegs) return;  // whole warps
  const RowSegment G = segs[si];
  const WideStep W = steps[G.domain];
  if (!(W.flags & WIDE_RUNNING)) return;  // warp-uniform: one domain per segment
  S *pool = reinterpret_cast<S *>(A.pool);
  StepArgs<float> a;
  memset(&a, 0, sizeof(a));
  a.tau = A.tau;
  a.omega = A.omega;
  for (int i = 0; i < 9; i++) {
    a.guo_a[i] = A.guo_a[i];
    a.guo_b[i] = A.guo_b[i];
    a.guo_odd[i] = A.guo_odd[i];
  }
  a.force_u[0] = A.force[0];
  a.force_u[1] = A.force[1];
  a.scale = A.scale;
  a.inv_scale = A.inv_scale;
  const BatchDomainDev D = A.dom[G.domain];
  const int sx = W.sx, sy = W.sy;
  const bool odd = W.flags & WIDE_ODD;
  const bool save = W.flags & WIDE_SAVE;
  const bool test = W.flags & WIDE_TEST;
  a.B = A.B + D.node_off;
  const int lane = (int)(threadIdx.x & 31);
  int x = G.x0 + lane, y = G.y;
  while (x >= D.lx) {  // at most once when lx >= 32
    x -= D.lx;
    y += 1;
  }
  float dmax = 0;
  float2 *up = A.u_prev + D.node_off;
  for (int j = 0; j < WIDE_ITERS; j++) {
    if (y >= D.ly) break;  // past the domain's last node
    const int k = x + y * D.lx;
    float ux, uy;
    batch_node<S, BLEND>(pool + D.pop_off, D.pitch, k, x, y, D.lx, D.ly, sx, sy, odd, A.cls[D.node_off + k], a,
                         ux, uy);
    if (test) dmax = nan_max(dmax, node_delta(ux, uy, up[k]));
    if (save) up[k] = make_float2(ux, uy);
    x += 32;
    while (x >= D.lx) {
      x -= D.lx;
      y += 1;
    }
  }
  if (test) {
    const float m = warp_max(dmax);
    if ((threadIdx.x & 31) == 0) atomicMax(acc + G.domain, __float_as_int(m));
  }
}

// After each tail-phase step: per domain, the convergence test of the step
// just taken (max |u(t) - u(t - C)| < tol), t + 1, the step cap; at the last
// step of a launch group the domains still running are counted.
__global__ void batch_wide_finish_kernel(const BatchArgs A, const int *wide, int nwide, WideStep *steps, int *acc,
                                         int last) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nwide) return;
  const int d = wide[i];
  BatchStateDev &st = A.state[d];
  if (st.converged) return;
  long long t = st.t;
  const bool test = steps[d].flags & WIDE_TEST;
  int stop = 0;
  if (test) {
    const float m = __int_as_float(acc[d]);
    acc[d] = 0;
    st.delta_u = m;
    stop = stop_code(m, A.tol);
  }
  t += 1;
  if (!stop && t >= A.max_steps) stop = STOP_CAP;
  st.t = t;
  const BatchDomainDev D = A.dom[d];
  steps[d] = wide_step(t, D.lx, D.ly, A.check, !stop);
  if (stop) {
    st.converged = stop;
    st.done_ns = global_ns();
  } else if (last) {
    atomicAdd(A.active, 1);
    atomicAdd(A.active_hbm, 1);
  }
}

}  // namespace

struct lbmc_batch {
  lbmc_batch_config cfg;
  int ndomains = 0;
  std::vector<BatchDomainDev> dom;
  // Domain classes, each largest first: resident (shared memory), then
  // block-stepped HBM domains (one block per domain, K steps per launch),
  // then wide HBM domains (over every SM, one step per launch).
  std::vector<int> order;
  int n_resident = 0, n_block = 0;
  long long wide_min_nodes = 0;  // HBM domains with at least this many nodes are wide
  void *pool = nullptr;
  uint8_t *cls = nullptr;
  float *B = nullptr;
  float2 *u_prev = nullptr;
  BatchDomainDev *dom_dev = nullptr;
  BatchStateDev *state = nullptr;
  int *order_dev = nullptr;
  int *counters = nullptr;  // [0] resident queue, [1] block-stepped queue, [2] active,
                            // [3] active block-stepped, [4] active wide
  int *acc = nullptr;       // tail phase: per-domain convergence maxima (float bits)
  int wide_below = 0;       // move the block-stepped domains to the wide path below this many
  unsigned long long *t0 = nullptr;
  cudaStream_t stream = nullptr;
  int ssize = 4;
  bool blend = false;
  long long total_nodes = 0;
  size_t smem_bytes = 0;
  int sms = 0;
  int threads = 0, steps = 0;  // tuned launch shape
  int hbm_blocks_per_sm[3] = {1, 1, 1};  // for 256 / 512 / 1024 threads
  cudaStream_t side = nullptr;            // second graph branch
  cudaEvent_t fork = nullptr, join = nullptr;
  double scale = 1;
};

namespace {

lbmc_status berr(lbmc_status s, const std::string &m) {
  lbmc::set_last_error(m);
  return s;
}

template <class S>
cudaError_t configure_batch(lbmc_batch *b) {
  cudaError_t e = cudaFuncSetAttribute(batch_kernel<S, true, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem_bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(batch_kernel<S, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)b->smem_bytes);
  const int th[3] = {256, 512, 1024};
  for (int k = 0; k < 3 && e == cudaSuccess; k++) {
    int nb = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &nb, b->blend ? batch_kernel<S, true, false> : batch_kernel<S, false, false>, th[k], 0);
    b->hbm_blocks_per_sm[k] = nb > 0 ? nb : 1;
  }
  return e;
}

enum DomainClass { CLASS_RESIDENT, CLASS_BLOCK, CLASS_WIDE };

BatchArgs make_args(lbmc_batch *b, int steps, int check, double tol, long long max_steps, DomainClass c) {
  BatchArgs A;
  memset(&A, 0, sizeof(A));
  A.pool = b->pool;
  A.cls = b->cls;
  A.B = b->B;
  A.u_prev = b->u_prev;
  A.dom = b->dom_dev;
  A.state = b->state;
  A.order = b->order_dev + (c == CLASS_RESIDENT ? 0 : b->n_resident);
  A.ndomains = c == CLASS_RESIDENT ? b->n_resident : (c == CLASS_BLOCK ? b->n_block : 0);
  A.queue = b->counters + (c == CLASS_RESIDENT ? 0 : 1);
  A.active = b->counters + 2;
  A.active_hbm = b->counters + (c == CLASS_WIDE ? 4 : 3);
  A.steps = steps;
  A.check = check;
  A.tol = (float)tol;
  A.max_steps = max_steps;
  A.tau = (float)b->cfg.tau;
  A.omega = (float)(1.0 / b->cfg.tau);
  {
    float ga[15], gb[15], go[15];
    set_uniform_guo<D2Q9, float>(ga, gb, go, b->cfg.tau, b->cfg.force);
    for (int i = 0; i < 9; i++) {
      A.guo_a[i] = ga[i];
      A.guo_b[i] = gb[i];
      A.guo_odd[i] = go[i];
    }
  }
  A.force[0] = (float)b->cfg.force[0];
  A.force[1] = (float)b->cfg.force[1];
  A.scale = (float)b->scale;
  A.inv_scale = (float)(1.0 / b->scale);
  A.blend = b->blend;
  A.smem_elems = c == CLASS_RESIDENT ? b->smem_bytes / b->ssize : 0;
  return A;
}

// The wide domains still running, as node segments, with their step
// descriptors (device arrays; release() frees them).
struct WideWork {
  RowSegment *segs = nullptr;
  int *wide = nullptr;
  WideStep *steps = nullptr;  // per domain (every domain, listed or not)
  int nsegs = 0, nwide = 0;
  void release() {
    if (segs) cudaFree(segs);
    if (wide) cudaFree(wide);
    if (steps) cudaFree(steps);
    segs = nullptr;
    wide = nullptr;
    steps = nullptr;
    nsegs = nwide = 0;
  }
};

// One graph launch: the resident kernel on st; on the side stream the
// block-stepped kernel (unless its domains moved to the wide path) and then
// K wide steps; joined again.
template <class S>
cudaError_t launch_round(lbmc_batch *b, const BatchArgs &res, const BatchArgs &blk, const BatchArgs &wid,
                         int threads, bool run_block, const WideWork &w, cudaStream_t st) {
  cudaError_t e = cudaEventRecord(b->fork, st);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(b->side, b->fork, 0);
  if (e != cudaSuccess) return e;
  if (res.ndomains > 0) {
    auto kr = b->blend ? batch_kernel<S, true, true> : batch_kernel<S, false, true>;
    kr<<<b->sms, threads, b->smem_bytes, st>>>(res);
  }
  if (run_block && blk.ndomains > 0) {
    const int k = threads <= 256 ? 0 : (threads <= 512 ? 1 : 2);
    auto kh = b->blend ? batch_kernel<S, true, false> : batch_kernel<S, false, false>;
    kh<<<b->sms * b->hbm_blocks_per_sm[k], threads, 0, b->side>>>(blk);
  }
  if (w.nwide > 0) {
    auto kw = b->blend ? batch_wide_kernel<S, true> : batch_wide_kernel<S, false>;
    const unsigned grid = (unsigned)((w.nsegs + WIDE_WARPS - 1) / WIDE_WARPS);
    for (int s = 0; s < wid.steps; s++) {
      kw<<<grid, WIDE_THREADS, 0, b->side>>>(wid, w.segs, w.nsegs, w.steps, b->acc);
      batch_wide_finish_kernel<<<(w.nwide + 127) / 128, 128, 0, b->side>>>(wid, w.wide, w.nwide, w.steps, b->acc,
                                                                          s == wid.steps - 1);
    }
  }
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventRecord(b->join, b->side);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(st, b->join, 0);
  return e;
}

cudaError_t enqueue_round(lbmc_batch *b, int steps, int check, double tol, long long max_steps, int threads,
                          bool run_block, const WideWork &w, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(b->counters, 0, 5 * sizeof(int), st);
  if (e != cudaSuccess) return e;
  const BatchArgs res = make_args(b, steps, check, tol, max_steps, CLASS_RESIDENT);
  const BatchArgs blk = make_args(b, steps, check, tol, max_steps, CLASS_BLOCK);
  const BatchArgs wid = make_args(b, steps, check, tol, max_steps, CLASS_WIDE);
  switch (b->cfg.storage) {
    case LBMC_F16: return launch_round<__half>(b, res, blk, wid, threads, run_block, w, st);
    case LBMC_BF16: return launch_round<__nv_bfloat16>(b, res, blk, wid, threads, run_block, w, st);
    default: return launch_round<float>(b, res, blk, wid, threads, run_block, w, st);
  }
}

// The wide domains still running (with include_block the block-stepped ones
// too), as node segments; device arrays in w (the caller releases them).
cudaError_t build_wide(lbmc_batch *b, int check, bool include_block, WideWork &w) {
  std::vector<BatchStateDev> st(b->ndomains);
  cudaError_t e = cudaMemcpy(st.data(), b->state, b->ndomains * sizeof(BatchStateDev), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return e;
  std::vector<RowSegment> segs;
  std::vector<int> wide;
  std::vector<WideStep> steps(b->ndomains, WideStep{0, 0, 0});
  for (int j = b->n_resident; j < b->ndomains; j++) {
    const int d = b->order[j];
    const BatchDomainDev &D = b->dom[d];
    const bool block_stepped = j < b->n_resident + b->n_block;
    if (st[d].converged || (block_stepped && !include_block)) continue;
    wide.push_back(d);
    steps[d] = wide_step(st[d].t, D.lx, D.ly, check, true);
    const long long n = (long long)D.lx * D.ly;
    for (long long k0 = 0; k0 < n; k0 += 32 * WIDE_ITERS) segs.push_back({d, (int)(k0 / D.lx), (int)(k0 % D.lx)});
  }
  w.nsegs = (int)segs.size();
  w.nwide = (int)wide.size();
  e = cudaMalloc(&w.segs, sizeof(RowSegment) * std::max(1, w.nsegs));
  if (e == cudaSuccess) e = cudaMalloc(&w.wide, sizeof(int) * std::max(1, w.nwide));
  if (e == cudaSuccess) e = cudaMalloc(&w.steps, sizeof(WideStep) * b->ndomains);
  if (e == cudaSuccess)
    e = cudaMemcpy(w.steps, steps.data(), sizeof(WideStep) * b->ndomains, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && w.nsegs)
    e = cudaMemcpy(w.segs, segs.data(), sizeof(RowSegment) * w.nsegs, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && w.nwide) e = cudaMemcpy(w.wide, wide.data(), sizeof(int) * w.nwide, cudaMemcpyHostToDevice);
  // Pageable copies above: make sure they landed before the side stream reads.
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return e;
}

}  // namespace

extern "C" lbmc_status lbmc_batch_init(const lbmc_batch_config *cfg, int ndomains,
                                       const lbmc_batch_domain *doms, lbmc_batch **out) {
  if (!cfg || !doms || !out || ndomains < 1) return berr(LBMC_ERR_INVALID_ARG, "lbmc_batch_init: NULL or empty");
  *out = nullptr;
  if (!(cfg->tau > 0.5) || !std::isfinite(cfg->tau)) return berr(LBMC_ERR_INVALID_ARG, "tau must be > 0.5");
  if (cfg->collision_type != LBMC_BGK && cfg->collision_type != LBMC_NTPOR)
    return berr(LBMC_ERR_UNSUPPORTED, "batched domains support ColType BGK and NTPOR");
  if (cfg->storage != LBMC_F32 && cfg->storage != LBMC_F16 && cfg->storage != LBMC_BF16)
    return berr(LBMC_ERR_UNSUPPORTED, "batched domains store FP32, FP16 or BF16");
  if (cfg->storage_scale < 0 || !std::isfinite(cfg->storage_scale) ||
      (cfg->storage == LBMC_F16 && cfg->storage_scale > 0 && !f16_scale_ok(cfg->storage_scale)))
    return berr(LBMC_ERR_INVALID_ARG, "storage_scale: >= 0, and for FP16 a power of two in [2^-15, 2^14]");
  if (cudaSetDevice(cfg->device) != cudaSuccess) {
    cudaGetLastError();
    return berr(LBMC_ERR_NO_DEVICE, "no such device");
  }
  lbmc_batch *b = new lbmc_batch();
  b->cfg = *cfg;
  b->ndomains = ndomains;
  b->ssize = cfg->storage == LBMC_F32 ? 4 : 2;
  b->scale = cfg->storage_scale > 0 ? cfg->storage_scale : (cfg->storage == LBMC_F16 ? 1024.0 : 1.0);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, cfg->device);
  int smem_optin = 0;
  cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, cfg->device);
  b->smem_bytes = (size_t)std::max(0, smem_optin - 2048);  // leave room for static shared memory
  const size_t resident_elems = b->smem_bytes / b->ssize;

  // Layout: populations padded to 64 elements per array (128-byte aligned).
  long long pop = 0, node = 0;
  b->dom.resize(ndomains);
  for (int d = 0; d < ndomains; d++) {
    const int lx = doms[d].length[0], ly = doms[d].length[1];
    if (lx < 1 || ly < 1 || (long long)lx * ly > (1LL << 24)) {
      delete b;
      return berr(LBMC_ERR_INVALID_ARG, "domain " + std::to_string(d) + " has a bad size");
    }
    const long long n = (long long)lx * ly;
    BatchDomainDev &D = b->dom[d];
    D.lx = lx;
    D.ly = ly;
    D.pitch = (int)((n + 63) / 64 * 64);
    D.pop_off = pop;
    D.node_off = node;
    D.resident = (size_t)n * 9 <= resident_elems;
    pop += 9LL * D.pitch;
    node += n;
  }
  b->total_nodes = node;
  std::vector<uint8_t> cls(node, 0);
  std::vector<float> B(node, 0.f);
  for (int d = 0; d < ndomains; d++) {
    const long long n = (long long)b->dom[d].lx * b->dom[d].ly;
    for (long long k = 0; k < n; k++) {
      const double v = doms[d].geometry ? doms[d].geometry[k] : 0.0;
      if (!std::isfinite(v)) {
        delete b;
        return berr(LBMC_ERR_INVALID_ARG, "non-finite porosity");
      }
      uint8_t c = 0;
      if (v >= 1) c = CLASS_SOLID;
      else if (v != 0 && cfg->collision_type == LBMC_NTPOR) c = 2;
      cls[b->dom[d].node_off + k] = c;
      B[b->dom[d].node_off + k] = (float)v;
      if (c == 2) b->blend = true;
    }
  }
  // HBM domains with at least wide_min_nodes nodes are stepped over every
  // SM from the start.  Defaults measured on the 4096-domain sweep (first
  // 20000 steps, aggregate GLUPS for thresholds 1 / 32768 / 65536 / 131072 /
  // none): FP32 52.3 / 55.4 / 54.1 / 52.0 / 50.3, FP16 66.1 / 71.2 / 74.7 /
  // 78.2 / 80.2 (2-byte domains stepped K times by one block stay in cache).
  // Either way the last block-stepped domains join the wide path
  // (wide_below), which shortens the time to steady state.
  b->wide_min_nodes = cfg->wide_min_nodes > 0 ? cfg->wide_min_nodes
                                              : (cfg->storage == LBMC_F32 ? 32768 : LLONG_MAX);
  auto klass = [&](int d) {
    const BatchDomainDev &D = b->dom[d];
    if (D.resident) return 0;
    return (long long)D.lx * D.ly >= b->wide_min_nodes ? 2 : 1;
  };
  b->order.resize(ndomains);
  std::iota(b->order.begin(), b->order.end(), 0);
  std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) {
    if (klass(x) != klass(y)) return klass(x) < klass(y);
    return (long long)b->dom[x].lx * b->dom[x].ly > (long long)b->dom[y].lx * b->dom[y].ly;
  });
  for (int d = 0; d < ndomains; d++) {
    b->n_resident += klass(d) == 0;
    b->n_block += klass(d) == 1;
  }
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void **p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes ? bytes : 16);
  };
  alloc(&b->pool, (size_t)pop * b->ssize);
  alloc((void **)&b->cls, node);
  alloc((void **)&b->B, node * sizeof(float));
  alloc((void **)&b->u_prev, node * sizeof(float2));
  alloc((void **)&b->dom_dev, ndomains * sizeof(BatchDomainDev));
  alloc((void **)&b->state, ndomains * sizeof(BatchStateDev));
  alloc((void **)&b->order_dev, ndomains * sizeof(int));
  alloc((void **)&b->counters, 5 * sizeof(int));
  alloc((void **)&b->acc, ndomains * sizeof(int));
  alloc((void **)&b->t0, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(b->pool, 0, (size_t)pop * b->ssize);  // f = w (Init 0)
  if (e == cudaSuccess) e = cudaMemcpy(b->cls, cls.data(), node, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->B, B.data(), node * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->u_prev, 0, node * sizeof(float2));
  if (e == cudaSuccess)
    e = cudaMemcpy(b->dom_dev, b->dom.data(), ndomains * sizeof(BatchDomainDev), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->state, 0, ndomains * sizeof(BatchStateDev));
  if (e == cudaSuccess) e = cudaMemset(b->acc, 0, ndomains * sizeof(int));
  if (e == cudaSuccess)
    e = cudaMemcpy(b->order_dev, b->order.data(), ndomains * sizeof(int), cudaMemcpyHostToDevice);
  // A host-to-device cudaMemcpy from pageable memory may return before its
  // DMA lands, and the non-blocking streams below do not wait for it.
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming);
  if (e == cudaSuccess) {
    switch (cfg->storage) {
      case LBMC_F16: e = configure_batch<__half>(b); break;
      case LBMC_BF16: e = configure_batch<__nv_bfloat16>(b); break;
      default: e = configure_batch<float>(b); break;
    }
  }
  if (e != cudaSuccess) {
    lbmc_batch_destroy(b);
    return berr(e == cudaErrorMemoryAllocation ? LBMC_ERR_ALLOC : LBMC_ERR_CUDA,
                std::string("lbmc_batch_init: ") + cudaGetErrorString(e));
  }
  b->threads = cfg->block_threads;
  b->steps = cfg->steps_per_launch;
  b->wide_below = cfg->wide_below == 0 ? b->sms / 2 : cfg->wide_below;
  *out = b;
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_batch_run(lbmc_batch *b, long long max_steps, double tol, int check_every,
                                      lbmc_batch_result *results) {
  if (!b || max_steps < 1 || check_every < 1 || !(tol >= 0))
    return berr(LBMC_ERR_INVALID_ARG, "lbmc_batch_run: bad arguments");
  if (cudaSetDevice(b->cfg.device) != cudaSuccess) return berr(LBMC_ERR_CUDA, "cudaSetDevice");
  cudaError_t e = cudaSuccess;
  stamp_kernel<<<1, 1, 0, b->stream>>>(b->t0);

  // Wide domains run over every SM from the start; the block-stepped ones
  // join them once fewer than wide_below of those are running.
  WideWork w;
  bool all_wide = false;  // the block-stepped domains moved to the wide path
  {
    std::vector<BatchStateDev> st(b->ndomains);
    e = cudaMemcpy(st.data(), b->state, b->ndomains * sizeof(BatchStateDev), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return berr(LBMC_ERR_CUDA, std::string("lbmc_batch_run: ") + cudaGetErrorString(e));
    long long block_active = 0;
    for (int j = b->n_resident; j < b->n_resident + b->n_block; j++) block_active += !st[b->order[j]].converged;
    all_wide = b->wide_below > 0 && block_active > 0 && block_active < b->wide_below;
    e = build_wide(b, check_every, all_wide, w);
    if (e != cudaSuccess) {
      w.release();
      return berr(LBMC_ERR_CUDA, std::string("lbmc_batch_run: ") + cudaGetErrorString(e));
    }
  }
  auto enqueue_any = [&](int steps, int threads) {
    return enqueue_round(b, steps, check_every, tol, max_steps, threads, !all_wide, w, b->stream);
  };

  // Autotune the launch shape on the first launches (they are real steps).
  if (b->threads <= 0 || b->steps <= 0) {
    const int cand_threads[3] = {256, 512, 1024};
    const int cand_steps[2] = {check_every, 4 * check_every};
    double best = -1;
    int bt = 512, bs = check_every;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int ti = 0; ti < 3; ti++)
      for (int si = 0; si < 2; si++) {
        const int th = b->threads > 0 ? b->threads : cand_threads[ti];
        const int sp = b->steps > 0 ? b->steps : cand_steps[si];
        cudaEventRecord(e0, b->stream);
        e = enqueue_any(sp, th);
        cudaEventRecord(e1, b->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double rate = (double)sp / ms;  // steps per ms over the whole batch
        if (rate > best) {
          best = rate;
          bt = th;
          bs = sp;
        }
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) {
      w.release();
      return berr(LBMC_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
    }
    b->threads = bt;
    b->steps = bs;
  }

  // Capture one launch (queue reset + the kernels of K steps) in a graph and
  // replay it.  Once a quarter of the listed wide domains have stopped, their
  // segments are rebuilt and the graph re-captured, so launches no longer
  // visit them; the same when the block-stepped domains join the wide path.
  auto capture = [&](cudaGraph_t &graph, cudaGraphExec_t &exec) -> cudaError_t {
    cudaError_t ec = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (ec != cudaSuccess) return ec;
    cudaError_t e2 = enqueue_any(b->steps, b->threads);
    ec = cudaStreamEndCapture(b->stream, &graph);
    if (e2 != cudaSuccess) ec = e2;
    if (ec == cudaSuccess) ec = cudaGraphInstantiate(&exec, graph, 0);
    return ec;
  };
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  auto drop_graph = [&]() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  };
  auto rebuild = [&]() -> cudaError_t {
    drop_graph();
    w.release();
    cudaError_t ew = build_wide(b, check_every, all_wide, w);
    if (ew == cudaSuccess) ew = capture(graph, exec);
    return ew;
  };
  if (e == cudaSuccess) e = capture(graph, exec);
  int counts[5] = {0, 0, 1, 0, 0};
  const long long launches_max = max_steps / std::max(1, b->steps) + 2;
  for (long long l = 0; e == cudaSuccess && counts[2] > 0 && l < launches_max; l++) {
    e = cudaGraphLaunch(exec, b->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(counts, b->counters, sizeof(counts), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess || counts[2] == 0) break;
    if (!all_wide && b->wide_below > 0 && counts[3] > 0 && counts[3] < b->wide_below) {
      all_wide = true;
      e = rebuild();
    } else if (w.nwide > 0 && 4LL * counts[4] < 3LL * w.nwide) {
      e = rebuild();
    }
  }
  drop_graph();
  w.release();
  if (e != cudaSuccess) return berr(LBMC_ERR_CUDA, std::string("lbmc_batch_run: ") + cudaGetErrorString(e));
  if (results) {
    std::vector<BatchStateDev> st(b->ndomains);
    unsigned long long t0 = 0;
    e = cudaMemcpy(st.data(), b->state, b->ndomains * sizeof(BatchStateDev), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&t0, b->t0, sizeof(t0), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return berr(LBMC_ERR_CUDA, cudaGetErrorString(e));
    int nonfinite = 0;
    for (int d = 0; d < b->ndomains; d++) {
      results[d].steps = st[d].t;
      results[d].delta_u = st[d].delta_u;
      results[d].converged = st[d].converged == STOP_CONVERGED;
      results[d].nonfinite = st[d].converged == STOP_NONFINITE;
      results[d].elapsed_ms = st[d].converged == STOP_CONVERGED ? (double)(st[d].done_ns - t0) * 1e-6 : -1.0;
      nonfinite += results[d].nonfinite;
    }
    if (nonfinite)
      return berr(LBMC_ERR_NAN, std::to_string(nonfinite) + " domain(s) became non-finite and were stopped");
  }
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_batch_info(lbmc_batch *b, long long *total_nodes, int *threads,
                                       int *steps_per_launch, int *resident_domains) {
  if (!b) return berr(LBMC_ERR_INVALID_ARG, "NULL batch");
  if (total_nodes) *total_nodes = b->total_nodes;
  if (threads) *threads = b->threads;
  if (steps_per_launch) *steps_per_launch = b->steps;
  if (resident_domains) {
    int r = 0;
    for (const auto &D : b->dom) r += D.resident;
    *resident_domains = r;
  }
  return LBMC_OK;
}

namespace {

template <class S>
__global__ void batch_fetch_kernel(const S *pop, long long pitch, int lx, int ly, long long t, float inv_scale,
                                   double *rho, double *ux, double *uy, double *f) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= lx * ly) return;
  using L = D2Q9;
  const int x = k % lx, y = k / lx;
  // Shift layout: population i of node x in array i at (x - t e_i) mod L.
  // AA pattern: after an even number of steps in array i at x; after an odd
  // number in array opp(i) at x - e_i (the next, odd step's read map).
  const bool odd = batch_aa<S>() && (t & 1);
  const int sx = batch_aa<S>() ? (odd ? 1 : 0) : (int)(t % lx);
  const int sy = batch_aa<S>() ? (odd ? 1 : 0) : (int)(t % ly);
  const int xs[3] = {x, wrap_sub(x, sx % lx, lx), wrap_add(x, sx % lx, lx)};
  const int ys[3] = {y, wrap_sub(y, sy % ly, ly), wrap_add(y, sy % ly, ly)};
  double r = 0, jx = 0, jy = 0;
  for (int i = 0; i < 9; i++) {
    const int slot = xs[sel(L::e(0, i))] + lx * ys[sel(L::e(1, i))];
    const int arr = odd ? L::opp(i) : i;
    const double v = weight<L>(i) + (double)load_dev(pop + arr * pitch + slot, inv_scale);
    if (f) f[(long long)i * lx * ly + k] = v;
    r += v;
    jx += L::e(0, i) * v;
    jy += L::e(1, i) * v;
  }
  if (rho) rho[k] = r;
  if (ux) ux[k] = jx / r;
  if (uy) uy[k] = jy / r;
}

}  // namespace

// Natural-layout fields of one domain: RHO, U_X, U_Y (N doubles; u = j/rho of
// the current populations, without the Guo half-force shift) or F (9N).
extern "C" lbmc_status lbmc_batch_fetch(lbmc_batch *b, int domain, int field, void *dst, size_t bytes) {
  if (!b || !dst || domain < 0 || domain >= b->ndomains) return berr(LBMC_ERR_INVALID_ARG, "lbmc_batch_fetch");
  const BatchDomainDev &D = b->dom[domain];
  const long long n = (long long)D.lx * D.ly;
  const size_t need = (size_t)n * 8 * (field == LBMC_FIELD_F ? 9 : 1);
  if (field != LBMC_FIELD_RHO && field != LBMC_FIELD_U_X && field != LBMC_FIELD_U_Y && field != LBMC_FIELD_F)
    return berr(LBMC_ERR_INVALID_ARG, "lbmc_batch_fetch: field");
  if (bytes < need) return berr(LBMC_ERR_BUFFER_SIZE, "lbmc_batch_fetch: buffer too small");
  cudaSetDevice(b->cfg.device);
  BatchStateDev st;
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaMemcpy(&st, b->state + domain, sizeof(st), cudaMemcpyDeviceToHost);
  double *tmp = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&tmp, need);
  if (e == cudaSuccess) {
    double *rho = field == LBMC_FIELD_RHO ? tmp : nullptr;
    double *ux = field == LBMC_FIELD_U_X ? tmp : nullptr;
    double *uy = field == LBMC_FIELD_U_Y ? tmp : nullptr;
    double *f = field == LBMC_FIELD_F ? tmp : nullptr;
    const int nb = (int)((n + 255) / 256);
    const float inv = (float)(1.0 / b->scale);
    switch (b->cfg.storage) {
      case LBMC_F16:
        batch_fetch_kernel<__half><<<nb, 256, 0, b->stream>>>(
            reinterpret_cast<const __half *>(b->pool) + D.pop_off, D.pitch, D.lx, D.ly, st.t, inv, rho, ux, uy, f);
        break;
      case LBMC_BF16:
        batch_fetch_kernel<__nv_bfloat16><<<nb, 256, 0, b->stream>>>(
            reinterpret_cast<const __nv_bfloat16 *>(b->pool) + D.pop_off, D.pitch, D.lx, D.ly, st.t, inv, rho,
            ux, uy, f);
        break;
      default:
        batch_fetch_kernel<float><<<nb, 256, 0, b->stream>>>(reinterpret_cast<const float *>(b->pool) + D.pop_off,
                                                            D.pitch, D.lx, D.ly, st.t, inv, rho, ux, uy, f);
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e == cudaSuccess) e = cudaMemcpy(dst, tmp, need, cudaMemcpyDeviceToHost);
  }
  if (tmp) cudaFree(tmp);
  if (e != cudaSuccess) return berr(LBMC_ERR_CUDA, std::string("lbmc_batch_fetch: ") + cudaGetErrorString(e));
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_batch_destroy(lbmc_batch *b) {
  if (!b) return LBMC_OK;
  cudaSetDevice(b->cfg.device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  void *ptrs[] = {b->pool, b->cls, b->B, b->u_prev, b->dom_dev, b->state, b->order_dev, b->counters, b->t0, b->acc};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (b->stream) cudaStreamDestroy(b->stream);
  if (b->side) cudaStreamDestroy(b->side);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->join) cudaEventDestroy(b->join);
  delete b;
  return LBMC_OK;
}
