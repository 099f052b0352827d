// Host-side check of the direct step kernel's streaming maps (shift, AA,
// tiled AA), compiled from the same functions the kernel uses
// (read_ptr / write_ptr / Sites / TiledSites / natural_slot in
// lbm-c_b200/csrc/kernels.cuh).  For every node and population of a few
// small domains and steps it checks that
//   1. every read and write lands inside the population allocation,
//   2. the reads of one step touch every element exactly once,
//   3. a node writes exactly the elements it read (in place, no race),
//   4. what node n writes as population i at step t is what node n + e_i
//      reads as population i at step t + 1 (streaming),
//   5. the cold kernels' natural_slot (fetch, upload, stress-free gather)
//      finds population i of node n where the step kernel reads it.
// Prints one line per failure (up to a limit) and exits 1 on any failure.
#include <cstdio>
#include <cstring>
#include <utility>
#include <vector>

#include "../lbm-c_b200/csrc/kernels.cuh"

using namespace lbmc;

namespace {

int failures = 0;

// Compile-time loop over 0..N-1 on the host (the kernels' unroll is device-only).
template <int N, class F, int... Is>
void unroll_host_impl(F &&f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
void unroll_host(F &&f) {
  unroll_host_impl<N>(f, std::make_integer_sequence<int, N>{});
}

void fail(const char *what, const char *mode, const int *L, long long t, long long n, int i, long long got,
          long long want) {
  static const int none[3] = {0, 0, 0};
  if (!L) L = none;
  if (failures++ < 20)
    std::printf("FAIL %s mode=%s L=%dx%dx%d t=%lld node=%lld i=%d got=%lld want=%lld\n", what, mode, L[0], L[1],
                L[2], t, n, i, got, want);
}

struct Domain {
  int L[3];
  long long n, pitch;
};

// The step-t shift the launcher passes (make_args): t mod L, or for the AA
// layouts (t mod 2) mod L.
void shifts(const Domain &d, bool aa, long long t, int *s) {
  for (int k = 0; k < 3; k++) s[k] = aa ? (int)((t & 1) % d.L[k]) : (int)(t % d.L[k]);
}

template <class L, int STREAM, std::size_t... Is>
void node_maps(const Domain &d, long long t, int bx, int lane, int y, int z, std::vector<long long> &rd,
               std::vector<long long> &wr, std::index_sequence<Is...>) {
  const bool aa = STREAM != STREAM_SHIFT;
  int s[3];
  shifts(d, aa, t, s);
  const int x = bx * DIRECT_BLOCK + lane;
  const int n = x + d.L[0] * (y + d.L[1] * z);
  Sites st;
  TiledSites ts;
  std::memset(&st, 0, sizeof st);
  std::memset(&ts, 0, sizeof ts);
  if (STREAM == STREAM_AAT_EVEN) ts.init_even(bx, lane, y, z, d.L, L::Q);
  else if (STREAM == STREAM_AAT_ODD) ts.init_odd(bx, lane, y, z, s, d.L, L::Q);
  else if (STREAM != STREAM_AA_EVEN) st.init(x, y, z, s, d.L);
  float *f = nullptr;
  static std::vector<float> buf;
  buf.resize((size_t)(L::Q * d.pitch) + 1);
  f = buf.data();
  ((rd[Is] = read_ptr<L, STREAM, (int)Is>(f, d.pitch, n, st, ts) - f), ...);
  ((wr[Is] = write_ptr<L, STREAM, (int)Is>(f, d.pitch, n, st, ts) - f), ...);
}

template <class L, std::size_t... Is>
void cold_slots(const Domain &d, long long t, bool aa, bool tiled, int x, int y, int z, std::vector<long long> &out,
                std::index_sequence<Is...>) {
  StepArgs<float> a;
  std::memset(&a, 0, sizeof a);
  a.pitch = d.pitch;
  a.aa = aa;
  a.odd = (int)(t & 1);
  a.tiled = tiled;
  shifts(d, aa, t, a.s);
  for (int k = 0; k < 3; k++) a.L[k] = d.L[k];
  Sites st;
  st.init(x, y, z, a.s, a.L);
  ((out[Is] = natural_slot<L, (int)Is>(a, st)), ...);
}

// Kernel stream mode the launcher picks at step t.
int mode_at(bool aa, bool tiled, long long t) {
  if (!aa) return STREAM_SHIFT;
  if (tiled) return (t & 1) ? STREAM_AAT_ODD : STREAM_AAT_EVEN;
  return (t & 1) ? STREAM_AA_ODD : STREAM_AA_EVEN;
}

template <class L>
void maps_at(const Domain &d, long long t, int mode, int bx, int lane, int y, int z, std::vector<long long> &rd,
             std::vector<long long> &wr) {
  auto seq = std::make_index_sequence<L::Q>{};
  switch (mode) {
    case STREAM_SHIFT: node_maps<L, STREAM_SHIFT>(d, t, bx, lane, y, z, rd, wr, seq); break;
    case STREAM_AA_EVEN: node_maps<L, STREAM_AA_EVEN>(d, t, bx, lane, y, z, rd, wr, seq); break;
    case STREAM_AA_ODD: node_maps<L, STREAM_AA_ODD>(d, t, bx, lane, y, z, rd, wr, seq); break;
    case STREAM_AAT_EVEN: node_maps<L, STREAM_AAT_EVEN>(d, t, bx, lane, y, z, rd, wr, seq); break;
    default: node_maps<L, STREAM_AAT_ODD>(d, t, bx, lane, y, z, rd, wr, seq); break;
  }
}

template <class L>
void check(int lx, int ly, int lz, bool aa) {
  Domain d;
  d.L[0] = lx;
  d.L[1] = ly;
  d.L[2] = lz;
  d.n = (long long)lx * ly * lz;
  d.pitch = (d.n + 63) / 64 * 64;  // the engine's 256-byte padding for 4-byte storage
  const bool tiled = aa && lx % TILE == 0;
  const char *names[] = {"shift", "aa-even", "aa-odd", "aat-even", "aat-odd"};
  const int Q = L::Q;
  const int bxs = (lx + DIRECT_BLOCK - 1) / DIRECT_BLOCK;
  std::vector<long long> rd(Q), wr(Q), rd1(Q), wr1(Q), cold(Q);
  for (long long t = 0; t < 4; t++) {
    const int mode = mode_at(aa, tiled, t), next = mode_at(aa, tiled, t + 1);
    const char *name = names[mode];
    std::vector<int> seen((size_t)(Q * d.pitch), 0);
    for (int z = 0; z < lz; z++)
      for (int y = 0; y < ly; y++)
        for (int bx = 0; bx < bxs; bx++)
          for (int lane = 0; lane < DIRECT_BLOCK; lane++) {
            const int x = bx * DIRECT_BLOCK + lane;
            if (x >= lx) continue;  // threads past the row end are inactive
            const long long n = x + (long long)lx * (y + (long long)ly * z);
            maps_at<L>(d, t, mode, bx, lane, y, z, rd, wr);
            cold_slots<L>(d, t, aa, tiled, x, y, z, cold, std::make_index_sequence<L::Q>{});
            for (int i = 0; i < Q; i++) {
              const long long limit = tiled ? Q * d.n : Q * d.pitch;
              if (rd[i] < 0 || rd[i] >= limit) fail("read out of range", name, d.L, t, n, i, rd[i], limit);
              if (wr[i] < 0 || wr[i] >= limit) fail("write out of range", name, d.L, t, n, i, wr[i], limit);
              if (rd[i] >= 0 && rd[i] < Q * d.pitch) seen[(size_t)rd[i]]++;
              const long long same = mode == STREAM_SHIFT ? rd[i] : rd[L::opp(i)];
              if (wr[i] != same) fail("write not in place", name, d.L, t, n, i, wr[i], same);
              if (cold[i] != rd[i]) fail("natural_slot differs", name, d.L, t, n, i, cold[i], rd[i]);
              // The neighbour n + e_i (periodic) at step t + 1.
              const int xn = (x + L::e(0, i) + lx) % lx, yn = (y + L::e(1, i) + ly) % ly,
                        zn = (z + L::e(2, i) + lz) % lz;
              maps_at<L>(d, t + 1, next, xn / DIRECT_BLOCK, xn % DIRECT_BLOCK, yn, zn, rd1, wr1);
              if (wr[i] != rd1[i]) fail("not streamed to neighbour", name, d.L, t, n, i, wr[i], rd1[i]);
            }
          }
    long long touched = 0;
    for (size_t k = 0; k < seen.size(); k++) {
      if (seen[k] > 1) fail("element read twice", name, d.L, t, (long long)k, -1, seen[k], 1);
      touched += seen[k] == 1;
    }
    if (touched != Q * d.n) fail("reads do not cover the domain", name, d.L, t, -1, -1, touched, Q * d.n);
  }
}

// The tiled odd step adds 32-bit unsigned row and x offsets, which the
// engine allows only while Q N < 2^32.  At the largest such D3Q15 domain,
// 1024 x 1024 x 273 (Q N = 4,293,918,720), the offsets of nodes on every
// face and corner (where the wraps and the largest offsets are) must equal
// the 64-bit tiled index of the neighbour slot.  No memory is touched.
template <class L>
void check_largest_tiled(int lx, int ly, int lz) {
  const int Q = L::Q;
  const long long n = (long long)lx * ly * lz;
  if (Q * n >= (1ll << 32)) {
    fail("test domain is not tileable", "aat-odd", nullptr, 1, 0, 0, Q * n, 1ll << 32);
    return;
  }
  int L3[3] = {lx, ly, lz}, s[3];
  for (int k = 0; k < 3; k++) s[k] = 1 % L3[k];  // the odd step's shift
  const int xs_[] = {0, 1, 63, 64, lx - 65, lx - 64, lx - 1}, ys_[] = {0, 1, ly - 2, ly - 1},
            zs_[] = {0, 1, lz - 2, lz - 1};
  for (int z : zs_)
    for (int y : ys_)
      for (int x : xs_) {
        TiledSites ts;
        ts.init_odd(x / TILE, x % TILE, y, z, s, L3, Q);
        Sites st;
        st.init(x, y, z, s, L3);
        const long long node = x + (long long)lx * (y + (long long)ly * z);
        unroll_host<Q>([&](auto ic) {
          constexpr int i = decltype(ic)::value;
          const unsigned got = ts.row[sel(L::e(1, i))][sel(L::e(2, i))] + ts.x[sel(L::e(0, i))] +
                               (unsigned)(L::opp(i) * TILE);
          const long long want = tiled_index(Q, st.template slot<L>(i), L::opp(i));
          if ((long long)got != want) fail("32-bit offset wraps", "aat-odd", L3, 1, node, i, got, want);
        });
      }
}

}  // namespace

int main() {
  const int d3[][3] = {{64, 3, 4}, {128, 2, 3}, {192, 1, 2}, {64, 1, 1}, {70, 3, 2}, {33, 4, 3}, {96, 2, 2}};
  const int d2[][3] = {{64, 5, 1}, {128, 3, 1}, {192, 2, 1}, {40, 3, 1}, {100, 2, 1}};
  int cases = 0;
  for (bool aa : {false, true}) {
    for (auto &s : d3) check<D3Q15>(s[0], s[1], s[2], aa), cases++;
    for (auto &s : d2) check<D2Q9>(s[0], s[1], s[2], aa), cases++;
  }
  check_largest_tiled<D3Q15>(1024, 1024, 273);
  cases++;
  if (failures) {
    std::printf("%d failures\n", failures);
    return 1;
  }
  std::printf("OK %d cases\n", cases);
  return 0;
}
