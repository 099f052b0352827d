// C-ABI engine: lbmc_init / lbmc_iterate / lbmc_fetch / lbmc_destroy.
//
// Host side of the drop-in boundary for LBM-C's time-step path.  lbmc_init
// plays the role of setup() + ModelBuilder (LBM-C/index.cu:157-186,
// LBM-C/model_builder.cu:63-248): it validates the configuration, packs the
// per-node inputs (Porosity, MacroBC, MicroBC) into one class byte per node
// plus a class table, uploads the fields and sets the initial populations.
// lbmc_iterate replaces iterate(t) (LBM-C/index.cu:284-313) and enqueues one
// fused step kernel per time step on the handle's stream; lbmc_fetch replaces
// the device-to-host copies of output_macros / screen_mess /
// compute_residual (LBM-C/index.cu:196-216, 387-439).
#include <cuda_runtime.h>

#include <sys/mman.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <climits>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lbmc.h"
#include "engine_internal.h"
#include "kernels.cuh"
#include "lattice.cuh"
#include "mlp.cuh"

using namespace lbmc;

// Values per lbmc_fetch staging chunk (64 MiB of FP64).
constexpr long long FETCH_CHUNK = 1ll << 23;

namespace {

thread_local std::string g_last_error;

lbmc_status fail(lbmc_status s, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

// Reports a CUDA error as the call's status and consumes it, so that a
// non-sticky error is not left pending for the caller's later CUDA calls.
lbmc_status cuda_fail(cudaError_t e, const char *what) {
  cudaGetLastError();
  return fail(e == cudaErrorMemoryAllocation ? LBMC_ERR_ALLOC : LBMC_ERR_CUDA, "%s: %s", what,
              cudaGetErrorString(e));
}

#define CK(call, what)                          \
  do {                                          \
    cudaError_t e_ = (call);                    \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

int lattice_q(int lattice) { return lattice == LBMC_D2Q9 ? 9 : 15; }
int lattice_dim(int lattice) { return lattice == LBMC_D2Q9 ? 2 : 3; }

double lattice_w(int lattice, int i) {
  return lattice == LBMC_D2Q9 ? (double)D2Q9::wn(i) / D2Q9::wd : (double)D3Q15::wn(i) / D3Q15::wd;
}
int lattice_e(int lattice, int d, int i) {
  return lattice == LBMC_D2Q9 ? D2Q9::e(d, i) : D3Q15::e(d, i);
}

const LatticeStorageOps *select_ops(int lattice, int storage) {
  if (lattice == LBMC_D2Q9) {
    switch (storage) {
      case LBMC_F32: return ops_d2q9_f32();
      case LBMC_F16: return ops_d2q9_f16();
      case LBMC_BF16: return ops_d2q9_bf16();
      case LBMC_F64: return ops_d2q9_f64();
      case LBMC_F16_SR: return ops_d2q9_f16sr();
    }
  } else {
    switch (storage) {
      case LBMC_F32: return ops_d3q15_f32();
      case LBMC_F16: return ops_d3q15_f16();
      case LBMC_BF16: return ops_d3q15_bf16();
      case LBMC_F64: return ops_d3q15_f64();
      case LBMC_F16_SR: return ops_d3q15_f16sr();
    }
  }
  return nullptr;
}

bool is_sf_code(int lattice, int code) {
  return lattice == LBMC_D2Q9 ? (code >= 5 && code <= 8) : (code >= 7 && code <= 12);
}

// Runs body(begin, end, chunk) over [0, n) in contiguous chunks on the
// host's cores (serially for small n); chunk c covers an increasing range,
// so per-chunk results concatenated in chunk order are in node order.
template <class F>
int parallel_for(long long n, F body) {
  unsigned hw = std::thread::hardware_concurrency();
  int t = (int)(hw == 0 ? 1 : (hw > 32 ? 32 : hw));
  if (n < (1LL << 20)) t = 1;
  const long long per = (n + t - 1) / t;
  std::vector<std::thread> pool;
  for (int c = 1; c < t; c++) {
    const long long b = c * per, e = std::min(n, b + per);
    if (b < e) pool.emplace_back(body, b, e, c);
  }
  body(0LL, std::min(n, per), 0);
  for (auto &th : pool) th.join();
  return t;
}

// Host scratch of the class packing: left uninitialised, so that the
// parallel passes touch its pages first (the page faults spread over the
// cores), and 2 MB aligned with a huge-page hint, so that where the kernel
// has transparent huge pages a 16 M-node domain faults a few dozen pages
// instead of ~12,000.
template <class T>
class HostBuffer {
 public:
  HostBuffer() = default;
  HostBuffer(const HostBuffer &) = delete;
  HostBuffer &operator=(const HostBuffer &) = delete;
  ~HostBuffer() { std::free(p_); }
  bool allocate(size_t count) {
    constexpr size_t HUGE_PAGE = 2u << 20;
    const size_t bytes = (count * sizeof(T) + HUGE_PAGE - 1) / HUGE_PAGE * HUGE_PAGE;
    std::free(p_);
    p_ = static_cast<T *>(std::aligned_alloc(HUGE_PAGE, bytes ? bytes : HUGE_PAGE));
    if (p_ && bytes) madvise(p_, bytes, MADV_HUGEPAGE);
    return p_ != nullptr;
  }
  T *data() { return p_; }
  const T *data() const { return p_; }
  T &operator[](size_t k) { return p_[k]; }

 private:
  T *p_ = nullptr;
};

// Host-side packing of the per-node inputs.
struct HostClasses {
  HostBuffer<uint8_t> cls;
  uint16_t table[256];
  int nclasses = 2;
  std::vector<int> sf_nodes;
  std::vector<uint8_t> sf_face;
  bool any_partial = false;
};

}  // namespace

void lbmc::set_last_error(const std::string &message) { g_last_error = message; }

struct lbmc_handle {
  lbmc_config cfg;
  DeviceState ds;
  const LatticeStorageOps *ops = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  long long step = 0;
  long long nblocks = 0;
  double *diag_out = nullptr;  // DIAG_VALUES doubles
  long long diag_step = -1;
  double *fetch_stage = nullptr;  // FP64 staging of uploads and lbmc_fetch (allocated on first use)
  long long fetch_stage_n = 0;
  std::vector<void *> allocations;
};

// ------------------------------------------------------------ validation

extern "C" lbmc_status lbmc_config_default(lbmc_config *cfg, int lattice) {
  if (!cfg) return fail(LBMC_ERR_INVALID_ARG, "lbmc_config_default: cfg is NULL");
  if (lattice != LBMC_D2Q9 && lattice != LBMC_D3Q15)
    return fail(LBMC_ERR_INVALID_ARG, "lbmc_config_default: unknown lattice %d", lattice);
  memset(cfg, 0, sizeof(*cfg));
  cfg->lattice = lattice;
  cfg->length[0] = cfg->length[1] = 1;
  cfg->length[2] = 1;
  cfg->tau = 1.0;
  cfg->c_smag = 0.0;
  cfg->collision_type = LBMC_BGK;
  cfg->init_type = LBMC_INIT_STATIC;
  cfg->storage = LBMC_F32;
  cfg->streaming = LBMC_STREAM_SHIFT;
  cfg->compat = 0;
  cfg->storage_scale = 0.0;
  return LBMC_OK;
}

static double default_scale(int storage) {
  return storage == LBMC_F16 || storage == LBMC_F16_SR ? 1024.0 : 1.0;
}

// The configuration checks of lbmc_validate (everything but the per-node
// arrays).
static lbmc_status validate_config(const lbmc_config *cfg, const lbmc_domain *dom) {
  if (!cfg) return fail(LBMC_ERR_INVALID_ARG, "config is NULL");
  if (cfg->lattice != LBMC_D2Q9 && cfg->lattice != LBMC_D3Q15)
    return fail(LBMC_ERR_INVALID_ARG, "unknown lattice %d", cfg->lattice);
  const int dim = lattice_dim(cfg->lattice);
  long long n = 1;
  for (int d = 0; d < 3; d++) {
    if (cfg->length[d] < 1) return fail(LBMC_ERR_INVALID_ARG, "length[%d] = %d must be >= 1", d, cfg->length[d]);
    if (d < dim) n *= cfg->length[d];
  }
  if (dim == 2 && cfg->length[2] != 1)
    return fail(LBMC_ERR_INVALID_ARG, "D2Q9 needs length[2] == 1 (got %d)", cfg->length[2]);
  if (n > 0x7FFFFFFFLL - 1024)
    return fail(LBMC_ERR_UNSUPPORTED, "%lld nodes exceed the 2^31 node limit of one domain", n);
  if (cfg->length[1] > 65535 || cfg->length[2] > 65535)
    return fail(LBMC_ERR_UNSUPPORTED, "Ly and Lz are limited to 65535 (one grid row per (y, z))");
  if (!(cfg->tau > 0.0) || !std::isfinite(cfg->tau))
    return fail(LBMC_ERR_INVALID_ARG, "tau must be positive and finite (got %g)", cfg->tau);
  if (cfg->collision_type < 0 || cfg->collision_type > 3)
    return fail(LBMC_ERR_INVALID_ARG, "unknown collision type %d", cfg->collision_type);
  if (cfg->c_smag > 0 && cfg->collision_type >= LBMC_MRT)
    return fail(LBMC_ERR_UNSUPPORTED, "Smagorinsky is only defined for the BGK family (ColType BGK/NTPOR)");
  if (!(cfg->c_smag >= 0.0) || !std::isfinite(cfg->c_smag))
    return fail(LBMC_ERR_INVALID_ARG, "c_smag must be >= 0 (got %g)", cfg->c_smag);
  if (cfg->storage < LBMC_F32 || cfg->storage > LBMC_F16_SR)
    return fail(LBMC_ERR_INVALID_ARG, "unknown storage %d", cfg->storage);
  if (cfg->streaming != LBMC_STREAM_SHIFT && cfg->streaming != LBMC_STREAM_AA)
    return fail(LBMC_ERR_INVALID_ARG, "unknown streaming scheme %d", cfg->streaming);
  if (cfg->streaming == LBMC_STREAM_AA && cfg->kernel == LBMC_KERNEL_PIPELINED)
    return fail(LBMC_ERR_UNSUPPORTED, "AA-pattern streaming runs in the direct-load kernel only");
  if (cfg->init_type < 0 || cfg->init_type > 2)
    return fail(LBMC_ERR_INVALID_ARG, "unknown init type %d", cfg->init_type);
  if (cfg->compat & ~(LBMC_COMPAT_REFERENCE_AS_IS))
    return fail(LBMC_ERR_INVALID_ARG, "unknown compat bits 0x%x", cfg->compat);
  if (cfg->storage_scale < 0 || !std::isfinite(cfg->storage_scale))
    return fail(LBMC_ERR_INVALID_ARG, "storage_scale must be >= 0");
  if ((cfg->storage == LBMC_F16 || cfg->storage == LBMC_F16_SR) && cfg->storage_scale > 0 &&
      !f16_scale_ok(cfg->storage_scale))
    return fail(LBMC_ERR_INVALID_ARG, "FP16 storage_scale must be a power of two in [2^-15, 2^14] (got %g)",
                cfg->storage_scale);
  if (cfg->kernel < LBMC_KERNEL_AUTO || cfg->kernel > LBMC_KERNEL_PIPELINED)
    return fail(LBMC_ERR_INVALID_ARG, "unknown kernel choice %d", cfg->kernel);
  if (!dom) return fail(LBMC_ERR_INVALID_ARG, "domain is NULL");
  if (cfg->init_type == LBMC_INIT_F && !dom->f)
    return fail(LBMC_ERR_INVALID_ARG, "init_type LBMC_INIT_F needs domain.f");
  if (cfg->macro_bc && !dom->macro_bc)
    return fail(LBMC_ERR_INVALID_ARG, "macro_bc is on but domain.macro_bc is NULL");
  if (cfg->micro_bc && !dom->micro_bc)
    return fail(LBMC_ERR_INVALID_ARG, "micro_bc is on but domain.micro_bc is NULL");
  return LBMC_OK;
}

// The per-node checks of lbmc_validate for node k: false (and the message)
// at a bad node; needs_rho is set where a MacroBC code prescribes rho.
static bool node_ok(const lbmc_config *cfg, const lbmc_domain *dom, long long k, bool have_u, bool &needs_rho,
                    char *msg, size_t len) {
  const double B = dom->geometry ? dom->geometry[k] : 0.0;
  if (!std::isfinite(B)) {
    snprintf(msg, len, "Porosity at node %lld is not finite", k);
    return false;
  }
  if (B >= 1) return true;
  if (cfg->macro_bc) {
    const int c = dom->macro_bc[k];
    if (c < 0 || c > 15) {
      snprintf(msg, len, "MacroBC code %d at node %lld is outside 0..15", c, k);
      return false;
    }
    if (macro_mask(c) & 0x8) needs_rho = true;
    if ((macro_mask(c) & 0x7) && !have_u) {
      snprintf(msg, len, "MacroBC code %d needs the velocity fields", c);
      return false;
    }
  }
  if (cfg->micro_bc) {
    const int c = dom->micro_bc[k];
    const int maxc = cfg->lattice == LBMC_D2Q9 ? 8 : 12;
    if (c < 0 || c > maxc) {
      snprintf(msg, len, "MicroBC code %d at node %lld is outside 0..%d", c, k, maxc);
      return false;
    }
    // micro_bc.cuh:7-8 leaves D2Q9 codes 3 and 4 as NULL entries.
    if (cfg->lattice == LBMC_D2Q9 && (c == 3 || c == 4)) {
      snprintf(msg, len, "MicroBC code %d is undefined for D2Q9 (node %lld)", c, k);
      return false;
    }
  }
  return true;
}

static bool have_velocity(const lbmc_config *cfg, const lbmc_domain *dom) {
  return dom->u[0] && dom->u[1] && (lattice_dim(cfg->lattice) == 2 || dom->u[2]);
}

// The status of the per-node checks, from the first bad node in node order
// (LLONG_MAX: none) and whether some node prescribes rho.
static lbmc_status node_status(const lbmc_config *cfg, const lbmc_domain *dom, long long bad, bool needs_rho) {
  if (bad != LLONG_MAX) {
    char msg[160];
    bool unused = false;
    node_ok(cfg, dom, bad, have_velocity(cfg, dom), unused, msg, sizeof(msg));
    return fail(LBMC_ERR_INVALID_ARG, "%s", msg);
  }
  if (needs_rho && !dom->rho) return fail(LBMC_ERR_INVALID_ARG, "a MacroBC code prescribes rho but domain.rho is NULL");
  return LBMC_OK;
}

// Checks a configuration and domain without touching the GPU; the first
// failing node in node order is reported.
extern "C" lbmc_status lbmc_validate(const lbmc_config *cfg, const lbmc_domain *dom) {
  lbmc_status st = validate_config(cfg, dom);
  if (st != LBMC_OK) return st;
  long long n = 1;
  for (int d = 0; d < lattice_dim(cfg->lattice); d++) n *= cfg->length[d];
  const bool have_u = have_velocity(cfg, dom);
  struct Chunk {
    long long bad = LLONG_MAX;
    bool needs_rho = false;
  };
  std::vector<Chunk> chunks(32);
  parallel_for(n, [&](long long b, long long e, int c) {
    char msg[160];
    for (long long k = b; k < e; k++)
      if (!node_ok(cfg, dom, k, have_u, chunks[c].needs_rho, msg, sizeof(msg))) {
        chunks[c].bad = k;
        break;
      }
  });
  bool needs_rho = false;
  long long bad = LLONG_MAX;
  for (const Chunk &c : chunks) {
    needs_rho = needs_rho || c.needs_rho;
    bad = std::min(bad, c.bad);
  }
  return node_status(cfg, dom, bad, needs_rho);
}

// Packs Porosity / MacroBC / MicroBC into class bytes (host only, no GPU).
// Class ids >= 2 go to the distinct (MacroBC, MicroBC, partial) entries in
// the order of their first node; the pass runs on the host's cores.
// With `check`, the per-node checks of lbmc_validate run in the same pass
// over the input arrays (lbmc_init reads them once).
static lbmc_status build_classes(const lbmc_config *cfg, const lbmc_domain *dom, long long n,
                                 HostClasses &hc, bool check) {
  HostBuffer<uint16_t> key;
  if (!hc.cls.allocate(n) || !key.allocate(n)) return fail(LBMC_ERR_ALLOC, "host allocation of %lld node classes", n);
  memset(hc.table, 0, sizeof(hc.table));
  const bool blend = cfg->collision_type == LBMC_NTPOR || cfg->collision_type == LBMC_MRTPOR;
  constexpr int KEYS = 512;            // macro (4 bits) | micro << 4 (4 bits) | partial << 8
  constexpr uint16_t SOLID_KEY = 0xFFFF;
  struct Chunk {
    long long first[KEYS];
    bool any_partial = false;
    std::vector<int> sf_nodes;
    std::vector<uint8_t> sf_face;
    long long bad = LLONG_MAX;
    bool needs_rho = false;
  };
  const bool have_u = have_velocity(cfg, dom);
  std::vector<std::unique_ptr<Chunk>> chunks(32);
  for (auto &c : chunks) {
    c.reset(new Chunk());
    for (int k = 0; k < KEYS; k++) c->first[k] = LLONG_MAX;
  }
  parallel_for(n, [&](long long b, long long e, int ci) {
    Chunk &c = *chunks[ci];
    char msg[160];
    for (long long k = b; k < e; k++) {
      if (check && !node_ok(cfg, dom, k, have_u, c.needs_rho, msg, sizeof(msg))) {
        c.bad = k;
        break;
      }
      const double B = dom->geometry ? dom->geometry[k] : 0.0;
      if (B >= 1) {  // LBM-C/solver.cu:67-72
        key[k] = SOLID_KEY;
        continue;
      }
      const int macro = cfg->macro_bc ? dom->macro_bc[k] : 0;
      const int micro = cfg->micro_bc ? dom->micro_bc[k] : 0;
      const bool partial = blend && B != 0.0;
      const unsigned entry = (unsigned)macro | ((unsigned)micro << ENTRY_MICRO_SHIFT) | (partial ? ENTRY_PARTIAL : 0u);
      if (partial) c.any_partial = true;
      if (micro && is_sf_code(cfg->lattice, micro)) {
        c.sf_nodes.push_back((int)k);
        c.sf_face.push_back((uint8_t)(cfg->lattice == LBMC_D2Q9 ? micro - 5 : micro - 7));
      }
      key[k] = (uint16_t)entry;
      if (entry && c.first[entry] == LLONG_MAX) c.first[entry] = k;
    }
  });
  if (check) {
    bool needs_rho = false;
    long long bad = LLONG_MAX;
    for (auto &c : chunks) {
      needs_rho = needs_rho || c->needs_rho;
      bad = std::min(bad, c->bad);
    }
    const lbmc_status st = node_status(cfg, dom, bad, needs_rho);
    if (st != LBMC_OK) return st;
  }
  // Ids by first appearance, as a sequential scan would give them.
  std::vector<std::pair<long long, int>> order;
  for (int e = 1; e < KEYS; e++) {
    long long f = LLONG_MAX;
    for (auto &c : chunks) f = std::min(f, c->first[e]);
    if (f != LLONG_MAX) order.push_back({f, e});
  }
  std::sort(order.begin(), order.end());
  if ((int)order.size() > 254)
    return fail(LBMC_ERR_UNSUPPORTED, "more than 254 distinct (MacroBC, MicroBC, partial) combinations");
  uint8_t id_of[KEYS] = {0};
  hc.nclasses = 2;
  for (auto &o : order) {
    id_of[o.second] = (uint8_t)hc.nclasses;
    hc.table[hc.nclasses++] = (uint16_t)o.second;
  }
  parallel_for(n, [&](long long b, long long e, int) {
    for (long long k = b; k < e; k++)
      hc.cls[k] = key[k] == SOLID_KEY ? (uint8_t)CLASS_SOLID : id_of[key[k]];
  });
  hc.any_partial = false;
  hc.sf_nodes.clear();
  hc.sf_face.clear();
  for (auto &c : chunks) {
    hc.any_partial = hc.any_partial || c->any_partial;
    hc.sf_nodes.insert(hc.sf_nodes.end(), c->sf_nodes.begin(), c->sf_nodes.end());
    hc.sf_face.insert(hc.sf_face.end(), c->sf_face.begin(), c->sf_face.end());
  }
  return LBMC_OK;
}

// Host-only view of the class packing, for tests and tools.
extern "C" lbmc_status lbmc_classify(const lbmc_config *cfg, const lbmc_domain *dom,
                                     uint8_t *cls_out, uint16_t *table_out, int *nclasses) {
  lbmc_status s = lbmc_validate(cfg, dom);
  if (s != LBMC_OK) return s;
  long long n = 1;
  for (int d = 0; d < lattice_dim(cfg->lattice); d++) n *= cfg->length[d];
  HostClasses hc;
  s = build_classes(cfg, dom, n, hc, false);
  if (s != LBMC_OK) return s;
  if (cls_out) memcpy(cls_out, hc.cls.data(), n);
  if (table_out) memcpy(table_out, hc.table, sizeof(hc.table));
  if (nclasses) *nclasses = hc.nclasses;
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_lattice_tables(int lattice, int *e, double *w, int *opp, int *m) {
  if (lattice != LBMC_D2Q9 && lattice != LBMC_D3Q15)
    return fail(LBMC_ERR_INVALID_ARG, "unknown lattice %d", lattice);
  const int q = lattice_q(lattice), dim = lattice_dim(lattice);
  for (int i = 0; i < q; i++) {
    for (int d = 0; d < dim; d++)
      if (e) e[d * q + i] = lattice_e(lattice, d, i);
    if (w) w[i] = lattice_w(lattice, i);
    if (opp) opp[i] = lattice == LBMC_D2Q9 ? D2Q9::opp(i) : D3Q15::opp(i);
    for (int k = 0; k < q; k++)
      if (m) m[k * q + i] = lattice == LBMC_D2Q9 ? D2Q9::m(k, i) : D3Q15::m(k, i);
  }
  return LBMC_OK;
}

// ------------------------------------------------------------ allocation

template <class T>
static lbmc_status dev_alloc(lbmc_handle *h, T **p, size_t bytes, const char *what) {
  void *ptr = nullptr;
  cudaError_t e = cudaMalloc(&ptr, bytes ? bytes : 16);
  if (e != cudaSuccess) return fail(LBMC_ERR_ALLOC, "cudaMalloc(%zu) for %s: %s", bytes, what, cudaGetErrorString(e));
  h->allocations.push_back(ptr);
  *p = static_cast<T *>(ptr);
  return LBMC_OK;
}

// dst[k] = (C)(src[k] + offset), or (C)fill everywhere when src is null,
// over one chunk of a field.
template <class C>
__global__ void narrow_kernel(const double *src, C *dst, long long n, double offset, double fill) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    dst[k] = (C)(src ? src[k] + offset : fill);
}

static lbmc_status ensure_stage(lbmc_handle *h, long long chunk) {
  if (h->fetch_stage_n >= chunk) return LBMC_OK;
  double *p = nullptr;
  CK(cudaMalloc(&p, sizeof(double) * chunk), "staging buffer");
  h->allocations.push_back(p);
  h->fetch_stage = p;
  h->fetch_stage_n = chunk;
  return LBMC_OK;
}

// Uploads N doubles as the compute type (float or double): each FP64 chunk
// of the caller's array goes to the device staging buffer in one copy and
// the device adds the offset and narrows it, so the host makes no pass over
// the data and allocates no temporary.
static lbmc_status upload_compute(lbmc_handle *h, void *dst, const double *src, long long n,
                                  double offset, double fill) {
  const long long chunk = std::min(n, FETCH_CHUNK);
  if (src) {
    lbmc_status s = ensure_stage(h, chunk);
    if (s != LBMC_OK) return s;
  }
  for (long long b = 0; b < n; b += chunk) {
    const long long m = std::min(chunk, n - b);
    const unsigned grid = (unsigned)std::min<long long>((m + 255) / 256, 4096);
    if (src)
      CK(cudaMemcpyAsync(h->fetch_stage, src + b, sizeof(double) * m, cudaMemcpyHostToDevice, h->stream),
         "upload field");
    const double *stage = src ? h->fetch_stage : nullptr;
    if (h->ops->csize == 8)
      narrow_kernel<double><<<grid, 256, 0, h->stream>>>(stage, static_cast<double *>(dst) + b, m, offset, fill);
    else
      narrow_kernel<float><<<grid, 256, 0, h->stream>>>(stage, static_cast<float *>(dst) + b, m, offset, fill);
    CK(cudaGetLastError(), "upload narrow launch");
    // The staging buffer is reused by the next chunk.
    CK(cudaStreamSynchronize(h->stream), "upload field");
  }
  return LBMC_OK;
}

static void release(lbmc_handle *h) {
  if (!h) return;
  for (void *p : h->allocations) cudaFree(p);
  h->allocations.clear();
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
}

#define TRY(call)                  \
  do {                             \
    lbmc_status s_ = (call);       \
    if (s_ != LBMC_OK) {           \
      release(h);                  \
      return s_;                   \
    }                              \
  } while (0)

#define TRYCUDA(call, what)                       \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) {                      \
      lbmc_status s_ = cuda_fail(e_, what);       \
      release(h);                                 \
      return s_;                                  \
    }                                             \
  } while (0)

// SM clock of a device in kHz, queried once per device and process.
static long long device_clock_khz(int device) {
  static std::mutex mu;
  static std::vector<long long> khz_of;
  std::lock_guard<std::mutex> lock(mu);
  if (device >= (int)khz_of.size()) khz_of.resize(device + 1, 0);
  if (khz_of[device] == 0) {
    int khz = 0;
    cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, device);
    khz_of[device] = khz > 0 ? khz : 2000000;
  }
  return khz_of[device];
}

extern "C" lbmc_status lbmc_init(const lbmc_config *cfg, const lbmc_domain *dom, lbmc_handle **out) {
  if (!out) return fail(LBMC_ERR_INVALID_ARG, "lbmc_init: out is NULL");
  *out = nullptr;
  // The per-node checks run with the class packing below, on the host's
  // cores while the uploads run.
  lbmc_status st = validate_config(cfg, dom);
  if (st != LBMC_OK) return st;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(LBMC_ERR_NO_DEVICE, "no CUDA device is available");
  }
  if (cfg->device < 0 || cfg->device >= ndev)
    return fail(LBMC_ERR_INVALID_ARG, "device %d does not exist (%d devices)", cfg->device, ndev);
  CK(cudaSetDevice(cfg->device), "cudaSetDevice");

  lbmc_handle *h = new (std::nothrow) lbmc_handle();
  if (!h) return fail(LBMC_ERR_ALLOC, "host allocation failed");
  h->cfg = *cfg;
  DeviceState &d = h->ds;
  memset(&d, 0, sizeof(d));
  d.lattice = cfg->lattice;
  d.storage = cfg->storage;
  d.q = lattice_q(cfg->lattice);
  d.dim = lattice_dim(cfg->lattice);
  d.n = 1;
  for (int k = 0; k < 3; k++) {
    d.L[k] = k < d.dim ? cfg->length[k] : 1;
    d.n *= d.L[k];
  }
  h->ops = select_ops(cfg->lattice, cfg->storage);
  const long long n = d.n;
  const int q = d.q, cs = h->ops->csize, ss = h->ops->ssize;

  d.tau = cfg->tau;
  d.c_smag = cfg->c_smag;
  for (int k = 0; k < 15; k++) d.s_mrt[k] = k < q ? cfg->tau_mrt[k] : 0.0;
  d.scale = cfg->storage_scale > 0 ? cfg->storage_scale : default_scale(cfg->storage);
  d.compat = cfg->compat;
  d.col = cfg->collision_type >= LBMC_MRT ? COL_MRT : (cfg->c_smag > 0 ? COL_BGK_SMAG : COL_BGK);
  if (d.col == COL_MRT) {
    bool conserved_zero = true;
    for (int k = 0; k < q; k++)
      if ((k == 0 || k == 3 || k == 5 || (q == 15 && k == 7)) && cfg->tau_mrt[k] != 0.0) conserved_zero = false;
    if (conserved_zero) d.col = COL_MRT_NC;
  }
  d.forcing = cfg->forcing ? 1 : 0;

  TRYCUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
  h->stream = h->own_stream;

  // Every device-side wait gives up after about two seconds.
  d.timeout_cycles = device_clock_khz(cfg->device) * 1000LL * 2;
  d.aa = cfg->streaming == LBMC_STREAM_AA ? 1 : 0;
  // The tiled AA layout needs whole 64-node tiles along x (one direct-kernel
  // block each) and element indices over all Q arrays below 2^32 (its row
  // and x offsets are 32-bit); other domains keep the plain AA layout.
  d.tiled = d.aa && d.L[0] % lbmc::TILE == 0 && (long long)q * n < (1ll << 32) ? 1 : 0;
  d.pipeline = cfg->kernel == LBMC_KERNEL_PIPELINED ? 2 : 0;
  TRYCUDA(h->ops->plan(d), "kernel planning");
  if (cfg->kernel == LBMC_KERNEL_PIPELINED && !d.use_pipeline) {
    release(h);
    return fail(LBMC_ERR_UNSUPPORTED,
                "the bulk-copy pipeline needs Lx * element size to be a multiple of 16 bytes "
                "and two stages of Q rows to fit in shared memory");
  }
  h->nblocks = d.nblocks;

  // The buffers every handle holds come from one cudaMalloc, carved at
  // 256-byte boundaries: each cudaMalloc of a large buffer measured 1-5 ms
  // inside lbmc_init, about as long as the upload of a field.
  {
    // Populations: Q arrays, each padded to a 256-byte boundary.
    const long long align = 256 / ss;
    d.pitch = (n + align - 1) / align * align;
    const long long stage_n = std::min(n, FETCH_CHUNK);
    const size_t sizes[] = {(size_t)d.pitch * q * ss,                                     // populations
                            (size_t)n,                                                    // node classes
                            (size_t)n * cs, (size_t)n * cs, (size_t)n * cs,               // rho - 1, u_x, u_y
                            d.dim > 2 ? (size_t)n * cs : 0,                               // u_z
                            sizeof(double) * stage_n,                                     // FP64 staging
                            sizeof(d.table), sizeof(unsigned),                            // table, error flag
                            sizeof(double) * DIAG_VALUES * (h->nblocks + FINALIZE_BLOCKS),  // partials
                            sizeof(unsigned), sizeof(double) * DIAG_VALUES};              // flag, diagnostics
    size_t total = 0;
    for (size_t b : sizes) total += (b + 255) / 256 * 256;
    char *base = nullptr;
    TRY(dev_alloc(h, &base, total, "handle buffers"));
    size_t off = 0;
    auto take = [&](int i) {
      void *p = base + off;
      off += (sizes[i] + 255) / 256 * 256;
      return p;
    };
    d.f = take(0);
    d.cls = static_cast<uint8_t *>(take(1));
    d.rho = take(2);
    for (int k = 0; k < 3; k++) {
      void *p = take(3 + k);
      if (k < d.dim) d.u[k] = p;
    }
    if (d.dim == 2) d.u[2] = d.u[1];  // never written for D2Q9; keeps pointers valid
    h->fetch_stage = static_cast<double *>(take(6));
    h->fetch_stage_n = stage_n;
    d.table_dev = static_cast<uint16_t *>(take(7));
    d.error_flag = static_cast<unsigned *>(take(8));
    d.partials = static_cast<double *>(take(9));
    d.flag = static_cast<unsigned *>(take(10));
    h->diag_out = static_cast<double *>(take(11));
  }
  TRYCUDA(cudaMemsetAsync(d.error_flag, 0, sizeof(unsigned), h->stream), "clear error flag");
  TRYCUDA(cudaMemsetAsync(d.flag, 0, sizeof(unsigned), h->stream), "clear flag");

  // The node classes are checked and packed on the host's cores while this
  // thread uploads rho and u (DMA): the two take similar times and do not
  // depend on each other.  The packing thread
  // reads only cfg and dom; an invalid domain is reported once it has
  // joined (uploads of absent arrays fill zeros, so nothing reads past what
  // the caller passed).
  HostClasses hc;
  lbmc_status cls_status = LBMC_OK;
  std::string cls_error;
  std::thread cls_thread([&] {
    cls_status = build_classes(cfg, dom, n, hc, true);
    if (cls_status != LBMC_OK) cls_error = lbmc_last_error();
  });
  struct Joiner {
    std::thread &t;
    ~Joiner() {
      if (t.joinable()) t.join();
    }
  } joiner{cls_thread};

  // rho - 1 and u: prescribed input (macro BC) and stored output.
  TRY(upload_compute(h, d.rho, dom->rho, n, -1.0, 0.0));
  for (int k = 0; k < d.dim; k++) TRY(upload_compute(h, d.u[k], dom->u[k], n, 0.0, 0.0));

  cls_thread.join();
  if (cls_status != LBMC_OK) {
    release(h);
    set_last_error(cls_error);
    return cls_status;
  }
  memcpy(d.table, hc.table, sizeof(d.table));
  d.blend = hc.any_partial ? 1 : 0;
  TRYCUDA(cudaMemcpy(d.cls, hc.cls.data(), n, cudaMemcpyHostToDevice), "upload classes");
  TRYCUDA(cudaMemcpy(d.table_dev, d.table, sizeof(d.table), cudaMemcpyHostToDevice), "upload class table");

  if (hc.any_partial) {
    TRY(dev_alloc(h, &d.B, (size_t)n * cs, "porosity"));
    TRY(upload_compute(h, d.B, dom->geometry, n, 0.0, 0.0));
  }

  if (cfg->forcing) {
    bool uniform = true;
    for (int k = 0; k < d.dim && uniform; k++) {
      const double *F = dom->force[k];
      const double v0 = F ? F[0] : 0.0;
      d.force_u[k] = v0;
      if (F)
        for (long long j = 1; j < n; j++)
          if (F[j] != v0) {
            uniform = false;
            break;
          }
    }
    if (!uniform) {
      for (int k = 0; k < d.dim; k++) {
        TRY(dev_alloc(h, &d.force[k], (size_t)n * cs, "force"));
        TRY(upload_compute(h, d.force[k], dom->force[k], n, 0.0, 0.0));
      }
      if (d.dim == 2) d.force[2] = d.force[1];
      d.force_u[0] = d.force_u[1] = d.force_u[2] = 0;
    }
  }

  if (!hc.sf_nodes.empty()) {
    d.n_sf = (int)hc.sf_nodes.size();
    TRY(dev_alloc(h, &d.sf_nodes, sizeof(int) * d.n_sf, "sf nodes"));
    TRY(dev_alloc(h, &d.sf_face, d.n_sf, "sf faces"));
    TRY(dev_alloc(h, &d.sf_index, sizeof(int) * n, "sf index"));
    TRY(dev_alloc(h, &d.sf_buf, (size_t)cs * q * d.n_sf, "sf buffer"));
    std::vector<int> idx(n, -1);
    for (int k = 0; k < d.n_sf; k++) idx[hc.sf_nodes[k]] = k;
    TRYCUDA(cudaMemcpy(d.sf_nodes, hc.sf_nodes.data(), sizeof(int) * d.n_sf, cudaMemcpyHostToDevice), "upload sf");
    TRYCUDA(cudaMemcpy(d.sf_face, hc.sf_face.data(), d.n_sf, cudaMemcpyHostToDevice), "upload sf");
    TRYCUDA(cudaMemcpy(d.sf_index, idx.data(), sizeof(int) * n, cudaMemcpyHostToDevice), "upload sf");
    TRYCUDA(cudaMemset(d.sf_buf, 0, (size_t)cs * q * d.n_sf), "clear sf");
  }

  // Initial populations (Init: model_builder.cu:227-248 for Init 0).
  if (cfg->init_type == LBMC_INIT_STATIC) {
    TRYCUDA(cudaMemset(d.f, 0, (size_t)d.pitch * q * ss), "clear populations");
  } else {
    double *tmp = nullptr;
    TRYCUDA(cudaMalloc(&tmp, sizeof(double) * n), "init staging");
    std::vector<double> host(cfg->init_type == LBMC_INIT_F ? 0 : n);
    lbmc_status s2 = LBMC_OK;
    for (int i = 0; i < q && s2 == LBMC_OK; i++) {
      const double *src = host.data();
      if (cfg->init_type == LBMC_INIT_F) {
        src = dom->f + (size_t)i * n;  // the caller's array, valid for the whole call
      } else {
        // f_eq(rho, u) of collision.cu:58.
        const double w = lattice_w(d.lattice, i);
        parallel_for(n, [&](long long b, long long e, int) {
          for (long long k = b; k < e; k++) {
            const double rho = dom->rho ? dom->rho[k] : 1.0;
            double u[3] = {0, 0, 0}, usq = 0, eu = 0;
            for (int c = 0; c < d.dim; c++) {
              u[c] = dom->u[c] ? dom->u[c][k] : 0.0;
              usq += u[c] * u[c];
              eu += lattice_e(d.lattice, c, i) * u[c];
            }
            eu *= 3.0;
            host[k] = rho * w * (1.0 + eu + 0.5 * eu * eu - 1.5 * usq);
          }
        });
      }
      // Ordered on the handle's stream: a pageable cudaMemcpy may return
      // before its DMA lands, and the non-blocking stream would not wait.
      cudaError_t e = cudaMemcpyAsync(tmp, src, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream);
      if (e == cudaSuccess) e = h->ops->upload_population(d, 0, i, tmp, h->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
      if (e != cudaSuccess) s2 = cuda_fail(e, "upload initial populations");
    }
    cudaFree(tmp);
    if (s2 != LBMC_OK) {
      release(h);
      return s2;
    }
  }
  TRYCUDA(cudaDeviceSynchronize(), "lbmc_init");
  *out = h;
  return LBMC_OK;
}

// Sums the per-block partials in FP64 in a fixed order (deterministic: the
// order depends only on the number of step blocks).  Stage 1: block g of
// FINALIZE_BLOCKS sums a contiguous run of whole partial records with
// coalesced loads; FINALIZE_THREADS is a multiple of DIAG_VALUES, so thread
// t always meets value t mod DIAG_VALUES, and the threads of one value are
// then added in thread order.  Stage 2: one block adds the stage-1 sums in
// block order.
__global__ void __launch_bounds__(FINALIZE_THREADS)
    diag_finalize_blocks_kernel(const double *partials, long long nblocks, double *mid) {
  __shared__ double sh[FINALIZE_THREADS];
  const long long per = (nblocks + FINALIZE_BLOCKS - 1) / FINALIZE_BLOCKS;
  const long long b0 = per * blockIdx.x, b1 = b0 + per < nblocks ? b0 + per : nblocks;
  const long long end = b1 * DIAG_VALUES;
  double acc = 0;
  for (long long k = b0 * DIAG_VALUES + threadIdx.x; k < end; k += FINALIZE_THREADS) acc += partials[k];
  sh[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < DIAG_VALUES) {
    double t = 0;
    for (int k = threadIdx.x; k < FINALIZE_THREADS; k += DIAG_VALUES) t += sh[k];
    mid[blockIdx.x * DIAG_VALUES + threadIdx.x] = t;
  }
}
__global__ void diag_finalize_kernel(const double *mid, double *out) {
  if (threadIdx.x < DIAG_VALUES) {
    double t = 0;
    for (int g = 0; g < FINALIZE_BLOCKS; g++) t += mid[g * DIAG_VALUES + threadIdx.x];
    out[threadIdx.x] = t;
  }
}

extern "C" lbmc_status lbmc_iterate(lbmc_handle *h, int nsteps, unsigned flags) {
  if (!h) return fail(LBMC_ERR_INVALID_ARG, "lbmc_iterate: handle is NULL");
  if (nsteps < 0) return fail(LBMC_ERR_INVALID_ARG, "lbmc_iterate: nsteps = %d", nsteps);
  if (flags & ~(LBMC_STORE_MACROS | LBMC_REDUCE_DIAG | LBMC_SYNC))
    return fail(LBMC_ERR_INVALID_ARG, "lbmc_iterate: unknown flags 0x%x", flags);
  CK(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  for (int s = 0; s < nsteps; s++) {
    const bool last = s == nsteps - 1;
    const bool store = last && (flags & LBMC_STORE_MACROS);
    const bool diag = last && (flags & LBMC_REDUCE_DIAG);
    if (diag) CK(cudaMemsetAsync(h->ds.flag, 0, sizeof(unsigned), h->stream), "clear flag");
    CK(h->ops->step(h->ds, h->step, store, diag, h->stream), "step kernel launch");
    h->step++;
    if (diag) {
      double *mid = h->ds.partials + DIAG_VALUES * h->nblocks;
      diag_finalize_blocks_kernel<<<FINALIZE_BLOCKS, FINALIZE_THREADS, 0, h->stream>>>(h->ds.partials,
                                                                                       h->nblocks, mid);
      diag_finalize_kernel<<<1, 32, 0, h->stream>>>(mid, h->diag_out);
      CK(cudaGetLastError(), "diagnostic reduction launch");
      h->diag_step = h->step;
    }
  }
  if (flags & LBMC_SYNC) {
    CK(cudaStreamSynchronize(h->stream), "lbmc_iterate");
    unsigned err = 0;
    CK(cudaMemcpy(&err, h->ds.error_flag, sizeof(err), cudaMemcpyDeviceToHost), "read error flag");
    if (err & ERROR_TIMEOUT)
      return fail(LBMC_ERR_TIMEOUT, "a device-side wait expired (bulk-copy pipeline)");
    if ((flags & LBMC_REDUCE_DIAG) && nsteps > 0) {
      unsigned flag = 0;
      CK(cudaMemcpy(&flag, h->ds.flag, sizeof(flag), cudaMemcpyDeviceToHost), "read flag");
      if (flag) return fail(LBMC_ERR_NAN, "non-finite density or velocity at step %lld", h->step);
    }
  }
  return LBMC_OK;
}

// dst[k] = (double)src[k] + offset over one chunk of a field.
template <class C>
__global__ void widen_kernel(const C *src, double *dst, long long n, double offset) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    dst[k] = (double)src[k] + offset;
}

// A compute-type field to the caller's FP64 array: the device widens it
// (and adds the rho offset) into a staging buffer, chunk by chunk, and each
// chunk goes to the caller's array in one copy, so the host does no
// conversion pass and allocates no temporary.
static lbmc_status fetch_compute(lbmc_handle *h, const void *src, double *dst, long long n, double offset) {
  if (h->ops->csize == 8 && offset == 0) {
    CK(cudaMemcpy(dst, src, n * 8, cudaMemcpyDeviceToHost), "fetch field");
    return LBMC_OK;
  }
  const long long chunk = std::min(n, FETCH_CHUNK);
  lbmc_status s = ensure_stage(h, chunk);
  if (s != LBMC_OK) return s;
  for (long long b = 0; b < n; b += chunk) {
    const long long m = std::min(chunk, n - b);
    const unsigned grid = (unsigned)std::min<long long>((m + 255) / 256, 4096);
    if (h->ops->csize == 8)
      widen_kernel<double><<<grid, 256, 0, h->stream>>>(static_cast<const double *>(src) + b, h->fetch_stage, m, offset);
    else
      widen_kernel<float><<<grid, 256, 0, h->stream>>>(static_cast<const float *>(src) + b, h->fetch_stage, m, offset);
    CK(cudaGetLastError(), "fetch widen launch");
    CK(cudaMemcpyAsync(dst + b, h->fetch_stage, sizeof(double) * m, cudaMemcpyDeviceToHost, h->stream), "fetch field");
    CK(cudaStreamSynchronize(h->stream), "fetch field");
  }
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_fetch(lbmc_handle *h, int field, void *dst, size_t bytes) {
  if (!h) return fail(LBMC_ERR_INVALID_ARG, "lbmc_fetch: handle is NULL");
  if (!dst) return fail(LBMC_ERR_INVALID_ARG, "lbmc_fetch: dst is NULL");
  CK(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  CK(cudaStreamSynchronize(h->stream), "lbmc_fetch");
  const DeviceState &d = h->ds;
  const long long n = d.n;
  switch (field) {
    case LBMC_FIELD_RHO:
    case LBMC_FIELD_U_X:
    case LBMC_FIELD_U_Y:
    case LBMC_FIELD_U_Z: {
      if (bytes < (size_t)n * 8) return fail(LBMC_ERR_BUFFER_SIZE, "lbmc_fetch: need %lld bytes", n * 8);
      if (field == LBMC_FIELD_U_Z && d.dim == 2)
        return fail(LBMC_ERR_INVALID_ARG, "lbmc_fetch: D2Q9 has no z velocity");
      const void *src = field == LBMC_FIELD_RHO ? d.rho : d.u[field - LBMC_FIELD_U_X];
      return fetch_compute(h, src, static_cast<double *>(dst), n, field == LBMC_FIELD_RHO ? 1.0 : 0.0);
    }
    case LBMC_FIELD_F: {
      if (bytes < (size_t)n * d.q * 8)
        return fail(LBMC_ERR_BUFFER_SIZE, "lbmc_fetch: need %lld bytes", n * d.q * 8);
      double *tmp = nullptr;
      CK(cudaMalloc(&tmp, sizeof(double) * n), "fetch staging");
      cudaError_t e = cudaSuccess;
      for (int i = 0; i < d.q && e == cudaSuccess; i++) {
        e = h->ops->fetch_population(d, h->step, i, tmp, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e == cudaSuccess)
          e = cudaMemcpy(static_cast<double *>(dst) + (size_t)i * n, tmp, sizeof(double) * n, cudaMemcpyDeviceToHost);
      }
      cudaFree(tmp);
      if (e != cudaSuccess) return cuda_fail(e, "lbmc_fetch populations");
      return LBMC_OK;
    }
    case LBMC_FIELD_DIAG: {
      if (bytes < sizeof(lbmc_diag)) return fail(LBMC_ERR_BUFFER_SIZE, "lbmc_fetch: need sizeof(lbmc_diag)");
      lbmc_diag out;
      memset(&out, 0, sizeof(out));
      if (h->diag_step >= 0) {
        double v[DIAG_VALUES];
        unsigned flag = 0;
        CK(cudaMemcpy(v, h->diag_out, sizeof(v), cudaMemcpyDeviceToHost), "fetch diagnostics");
        CK(cudaMemcpy(&flag, d.flag, sizeof(flag), cudaMemcpyDeviceToHost), "fetch diagnostics");
        out.mass = v[0];
        out.momentum[0] = v[1];
        out.momentum[1] = v[2];
        out.momentum[2] = v[3];
        out.kinetic_energy = v[4];
        out.step = h->diag_step;
        out.nonfinite = flag ? 1 : 0;
        out.valid = 1;
      }
      memcpy(dst, &out, sizeof(out));
      return LBMC_OK;
    }
    default:
      return fail(LBMC_ERR_INVALID_ARG, "lbmc_fetch: unknown field %d", field);
  }
}

extern "C" lbmc_status lbmc_probe(lbmc_handle *h, long long node, double out[4]) {
  if (!h || !out) return fail(LBMC_ERR_INVALID_ARG, "lbmc_probe: NULL argument");
  const DeviceState &d = h->ds;
  if (node < 0 || node >= d.n) return fail(LBMC_ERR_INVALID_ARG, "lbmc_probe: node %lld outside the domain", node);
  CK(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  CK(cudaStreamSynchronize(h->stream), "lbmc_probe");
  const void *src[4] = {d.rho, d.u[0], d.u[1], d.dim == 3 ? d.u[2] : nullptr};
  for (int k = 0; k < 4; k++) {
    out[k] = 0.0;
    if (!src[k]) continue;
    if (h->ops->csize == 8) {
      CK(cudaMemcpy(&out[k], static_cast<const double *>(src[k]) + node, 8, cudaMemcpyDeviceToHost), "lbmc_probe");
    } else {
      float v = 0.f;
      CK(cudaMemcpy(&v, static_cast<const float *>(src[k]) + node, 4, cudaMemcpyDeviceToHost), "lbmc_probe");
      out[k] = v;
    }
  }
  out[0] += 1.0;  // stored as rho - 1
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_destroy(lbmc_handle *h) {
  if (!h) return LBMC_OK;
  cudaSetDevice(h->cfg.device);
  cudaStreamSynchronize(h->stream);
  release(h);
  return LBMC_OK;
}

// Defined in mlp.cu: the host copy of a network's closure parameters.
const MlpClosure *lbmc_mlp_closure(const lbmc_mlp *m);

extern "C" lbmc_status lbmc_set_closure(lbmc_handle *h, const lbmc_mlp *m, int iterations) {
  if (!h) return fail(LBMC_ERR_INVALID_ARG, "lbmc_set_closure: handle is NULL");
  if (h->cfg.collision_type != LBMC_BGK && h->cfg.collision_type != LBMC_NTPOR)
    return fail(LBMC_ERR_UNSUPPORTED, "the learned closure replaces Smagorinsky: BGK family only");
  CK(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  CK(cudaStreamSynchronize(h->stream), "lbmc_set_closure");
  if (!m) {  // detach: back to Smagorinsky / plain BGK
    h->ds.col = h->cfg.c_smag > 0 ? COL_BGK_SMAG : COL_BGK;
    return LBMC_OK;
  }
  if (iterations < 1 || iterations > 8) return fail(LBMC_ERR_INVALID_ARG, "iterations must be 1..8");
  if (h->ds.use_pipeline)
    return fail(LBMC_ERR_UNSUPPORTED, "the learned closure runs in the direct-load kernel (lbmc_config.kernel)");
  // The step evaluates the network warp-wide on the tensor cores, from the
  // weights in fragment order; the scalars travel with each launch.
  MlpStep c;
  mlp_step_layout(*lbmc_mlp_closure(m), iterations, c, h->ds.closure_consts);
  if (!h->ds.closure) {
    lbmc_status s = dev_alloc(h, &h->ds.closure, sizeof(MlpStep), "closure");
    if (s != LBMC_OK) return s;
  }
  CK(cudaMemcpyAsync(h->ds.closure, &c, sizeof(c), cudaMemcpyHostToDevice, h->stream), "upload closure");
  CK(cudaStreamSynchronize(h->stream), "upload closure");
  h->ds.col = iterations == 1 ? COL_BGK_MLP1 : COL_BGK_MLP;
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_get_step(lbmc_handle *h, long long *step) {
  if (!h || !step) return fail(LBMC_ERR_INVALID_ARG, "lbmc_get_step: NULL argument");
  *step = h->step;
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_set_stream(lbmc_handle *h, void *cuda_stream) {
  if (!h) return fail(LBMC_ERR_INVALID_ARG, "lbmc_set_stream: handle is NULL");
  CK(cudaStreamSynchronize(h->stream), "lbmc_set_stream");
  h->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : h->own_stream;
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_synchronize(lbmc_handle *h) {
  if (!h) return fail(LBMC_ERR_INVALID_ARG, "lbmc_synchronize: handle is NULL");
  CK(cudaStreamSynchronize(h->stream), "lbmc_synchronize");
  return LBMC_OK;
}

extern "C" const char *lbmc_status_string(lbmc_status s) {
  switch (s) {
    case LBMC_OK: return "ok";
    case LBMC_ERR_INVALID_ARG: return "invalid argument";
    case LBMC_ERR_UNSUPPORTED: return "unsupported";
    case LBMC_ERR_CUDA: return "CUDA error";
    case LBMC_ERR_ALLOC: return "allocation failed";
    case LBMC_ERR_NAN: return "non-finite value";
    case LBMC_ERR_TIMEOUT: return "timeout";
    case LBMC_ERR_IO: return "I/O error";
    case LBMC_ERR_BUFFER_SIZE: return "buffer too small";
    case LBMC_ERR_NO_DEVICE: return "no CUDA device";
  }
  return "unknown status";
}

extern "C" const char *lbmc_last_error(void) { return g_last_error.c_str(); }
