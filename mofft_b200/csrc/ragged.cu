// Ragged batches: many FP32 transforms of different lengths, batch sizes and
// directions in one CUDA graph.
//
// Persistent queue.  Items of the lengths one CTA tile runs in one pass
// (2^6 .. 2^13, 3*2^5 .. 3*2^11) run in ONE persistent kernel launch driven
// by a work-descriptor queue (tiles); in a single-launch plan every item
// does.
//
// Groups.  The other items are grouped by (length, direction), and each
// group runs that length's tuned schedule (compiled wisdom, else the model)
// once over all the group's transforms: pointer tables, one pair per pass,
// give every transform its own input, output and (for two-pass schedules in
// place) workspace, so a group takes one launch per pass.  The graph runs the
// groups on four parallel branches next to the persistent launch.  A group
// whose tuned schedule cannot run from tables joins the persistent queue as
// two-pass tiles.
//
// Tiles.  Every item (length n, batch, direction, buffers) is cut into
// tiles of work for one 512-thread CTA: a single-pass tile computes
// 512 / TPL whole transforms of length n (the rows_body of the one-pass
// kernels); a two-pass item (n = L0 * L1 beyond one CTA) has first-pass tiles
// (32 columns of the L0-point DFTs) and second-pass tiles (32 columns of the
// L1-point DFTs), the cols_body of the four-step kernels.  The queue holds
// every first-pass tile of every item (largest items first), then every
// second-pass tile.  CTAs pull tiles with an atomic counter.
//
// Dependencies.  A second-pass tile of item i may start only when all
// first-pass tiles of item i are done: the CTA that finishes a first-pass
// tile fences and increments done[i]; a second-pass tile's CTA waits until
// done[i] reaches the count.  Because tiles are pulled in queue order, every
// first-pass tile has been pulled -- by a running CTA that waits on nothing --
// before any second-pass tile is pulled, so the wait always ends.  It is
// still bounded (about 1 s); on timeout the CTA sets the error flag, skips the
// tile, and the host reports MOFFT_INTERNAL_ERROR.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "fft_device.cuh"
#include "mofft_cuda.h"
#include "mofft_host.h"

using namespace mofft;

namespace {

constexpr int kThreads = 512;
constexpr int kColsLines = 32;
constexpr unsigned kMaxSpins = 1u << 22;   // x 256 ns sleep: about 1 s

struct RItem {
  const float2 *in;
  float2 *mid;        // first-pass destination of a two-pass item
  float2 *out;
  const float2 *tw0;  // internal stage table of the (first) pass
  const float2 *tw1;  // internal stage table of the second pass
  const float2 *hi1;  // second-pass super twiddle, two-level
  const float2 *lo1;
  long long n, batch, dist;
  int passes, cfg0, cfg1, L0, split1, pass1_tiles;
  float sign;
  int pad;
};

struct RTile {
  int item;
  int pass;
  long long b;
  long long j0;
};

// Single-pass configurations: (id, L, TPL, staged, radices...) with
// TB = 512 / TPL transforms per tile; radix-16 stages derive their twiddles
// from four table entries and the tiles keep their lines as {re, im} pairs,
// as the tuned standalone kernels do (the column tiles too).
#define MOFFT_RAGGED_ROWS(X)                 \
  X(0, 64, 4, true, 16, 4)                  \
  X(1, 128, 8, true, 16, 8)                 \
  X(2, 256, 16, true, 16, 16)               \
  X(3, 512, 32, false, 16, 16, 2)           \
  X(4, 1024, 64, false, 16, 16, 4)          \
  X(5, 2048, 128, false, 16, 16, 8)         \
  X(6, 4096, 256, false, 16, 16, 16)        \
  X(7, 8192, 512, false, 16, 16, 16, 2)     \
  X(9, 96, 8, true, 6, 16)                  \
  X(10, 192, 16, true, 12, 16)              \
  X(11, 384, 32, false, 6, 4, 16)           \
  X(12, 768, 64, false, 3, 16, 16)          \
  X(13, 1536, 128, false, 6, 16, 16)        \
  X(14, 3072, 256, false, 12, 16, 16)       \
  X(15, 6144, 512, false, 6, 4, 16, 16)

// Column-pass configurations (id, L, TPL, radices...), C = 32 lines.
// Lengths 12288 and 16384 also run as two passes (96 x 128, 128 x 128):
// single-pass tiles of 32 points per thread would set the register budget
// of every tile path of the persistent kernel.
#define MOFFT_RAGGED_COLS(X) \
  X(17, 128, 16, 16, 8)      \
  X(18, 192, 16, 12, 16)     \
  X(19, 256, 16, 16, 16)     \
  X(20, 96, 16, 6, 16)

struct ConfigInfo {
  int id, length, tpl, cols;
  int radix_count;
  int radices[6];
  size_t smem;
};

template <int... R>
constexpr int kArgCount = (int)sizeof...(R);

#define MOFFT_ROWS_INFO(ID, L, TPL, ST, ...)                         \
  {ID, L, TPL, 0, kArgCount<__VA_ARGS__>, {__VA_ARGS__},             \
   2ull * (kThreads / TPL) * pair_pitch<float>(L, TPL, kThreads / TPL) * sizeof(float)},
#define MOFFT_COLS_INFO(ID, L, TPL, ...)                             \
  {ID, L, TPL, 1, kArgCount<__VA_ARGS__>, {__VA_ARGS__},             \
   ColsGeom<float, L, TPL, kColsLines>::SMEM},

const ConfigInfo kConfigs[] = {MOFFT_RAGGED_ROWS(MOFFT_ROWS_INFO) MOFFT_RAGGED_COLS(MOFFT_COLS_INFO)};

__device__ __forceinline__ RowsArgs<float> rows_args_of(const RItem &it) {  // NOLINT
  RowsArgs<float> a;
  a.in = it.in;
  a.out = it.out;
  a.tw = it.tw0;
  a.batch = it.batch;
  a.in_dist = it.dist;
  a.out_dist = it.dist;
  a.sign = it.sign;
  a.in_table = nullptr;
  a.out_table = nullptr;
  a.status = nullptr;
  a.lose_copy = 0;
  return a;
}

__device__ __forceinline__ ColsArgs<float> cols_args_of(const RItem &it, int pass) {
  ColsArgs<float> a;
  a.batch = it.batch;
  a.in_dist = it.dist;
  a.out_dist = it.dist;
  a.total = it.n;
  a.in_table = nullptr;
  a.out_table = nullptr;
  if (pass == 0) {
    a.in = it.in;
    a.out = it.mid;
    a.tw = it.tw0;
    a.tw_hi = it.tw0;
    a.tw_lo = it.tw0;
    a.ns_outer = 1;
    a.split_shift = 0;
    a.sign_in = it.sign;
    a.sign_out = 1.0f;
  } else {
    a.in = it.mid;
    a.out = it.out;
    a.tw = it.tw1;
    a.tw_hi = it.hi1;
    a.tw_lo = it.lo1;
    a.ns_outer = it.L0;
    a.split_shift = it.split1;
    a.sign_in = 1.0f;
    a.sign_out = it.sign;
  }
  return a;
}

// One non-inlined function per configuration, so that each allocates its
// registers on its own and the largest configuration does not make all others
// spill.
#define MOFFT_ROWS_FN(ID, L, TPL, ST, ...)                                          \
  __device__ __noinline__ void tile_##ID(const RItem *__restrict__ itp, int pass,    \
                                         long long b, long long j0,                   \
                                         unsigned char *smem) {                       \
    rows_body<float, L, TPL, kThreads / TPL, ((ST) ? kStaged : 0) | kDerivedTw | kPairX, \
              __VA_ARGS__>(rows_args_of(*itp), b, smem);                               \
  }
#define MOFFT_COLS_FN(ID, L, TPL, ...)                                              \
  __device__ __noinline__ void tile_##ID(const RItem *__restrict__ itp, int pass,    \
                                         long long b, long long j0,                   \
                                         unsigned char *smem) {                       \
    cols_body_pair<float, L, TPL, kColsLines, __VA_ARGS__>(cols_args_of(*itp, pass), b, j0, \
                                                      smem);                          \
  }
MOFFT_RAGGED_ROWS(MOFFT_ROWS_FN)
MOFFT_RAGGED_COLS(MOFFT_COLS_FN)
#undef MOFFT_ROWS_FN
#undef MOFFT_COLS_FN

__device__ __forceinline__ void run_tile(int cfg, const RItem *__restrict__ itp, int pass,
                                         long long b, long long j0, unsigned char *smem) {
  switch (cfg) {
#define MOFFT_CASE(ID, ...) \
  case ID:                  \
    tile_##ID(itp, pass, b, j0, smem); \
    break;
    MOFFT_RAGGED_ROWS(MOFFT_CASE)
    MOFFT_RAGGED_COLS(MOFFT_CASE)
#undef MOFFT_CASE
    default:
      break;
  }
}

// Two CTAs per SM: while one waits on memory the other computes.  The next
// tile index is fetched while the current tile runs.  A prefetched first-pass
// tile is always held behind a current first-pass tile (queue order), which
// never waits, so prefetching cannot starve a dependency.
__global__ void __launch_bounds__(kThreads, 2)
ragged_kernel(const RItem *__restrict__ items, const RTile *__restrict__ tiles,
              int tile_count, int *next, int *done, int *error, int need_bias) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_tile[2];
  __shared__ int s_skip;
  if (threadIdx.x == 0) s_tile[0] = atomicAdd(next, 1);
  __syncthreads();
  for (int iter = 0;; ++iter) {
    const int ti = s_tile[iter & 1];
    if (ti >= tile_count) break;
    const RTile tl = tiles[ti];
    const RItem *itp = items + tl.item;
    if (threadIdx.x == 0) {
      s_tile[(iter + 1) & 1] = atomicAdd(next, 1);
      int skip = 0;
      if (tl.pass == 1) {
        unsigned spins = 0;
        const int need = itp->pass1_tiles + need_bias;
        while (atomicAdd(&done[tl.item], 0) < need) {
          if (++spins > kMaxSpins) {
            atomicExch(error, 1);
            skip = 1;
            break;
          }
          __nanosleep(256);
        }
        __threadfence();
      }
      s_skip = skip;
    }
    __syncthreads();
    const int skip = s_skip;
    if (!skip)
      run_tile(tl.pass == 0 ? itp->cfg0 : itp->cfg1, itp, tl.pass, tl.b, tl.j0, smem);
    // only a first-pass tile of a two-pass item publishes data that another
    // CTA reads in this launch: its writes are fenced before the count rises
    if (tl.pass == 0 && itp->passes == 2) __threadfence();
    __syncthreads();
    if (threadIdx.x == 0 && tl.pass == 0 && itp->passes == 2 && !skip)
      atomicAdd(&done[tl.item], 1);
  }
}

int rows_config_for(long long n) {
  for (const ConfigInfo &c : kConfigs)
    if (!c.cols && c.length == n) return c.id;
  return -1;
}

int cols_config_for(int L) {
  for (const ConfigInfo &c : kConfigs)
    if (c.cols && c.length == L) return c.id;
  return -1;
}

const ConfigInfo &config(int id) {
  for (const ConfigInfo &c : kConfigs)
    if (c.id == id) return c;
  return kConfigs[0];
}

size_t round256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

// Items the persistent queue does not run in one pass, grouped by (length,
// direction): one tuned plan per group, run through pointer tables (one pair
// per pass) so that a group takes one launch per pass whatever its items.
struct RaggedGroup {
  mofft_core *core = nullptr;
  long long transforms = 0;
  int passes = 0;
  size_t table_off = 0;         // first pointer of this group's tables
};

struct mofft_ragged_plan {
  int device = 0;
  int item_count = 0;
  int tile_count = 0;
  int grid = 0;
  size_t smem = 0;
  std::vector<RaggedGroup> groups;
  void **d_ptr_tables = nullptr;  // every group's pointer tables
  int graph_launches = 0;         // kernels one execution launches
  // the graph's parallel branches: groups spread over them (largest first,
  // each to the branch with the fewest points so far) so that independent
  // launches overlap on the device
  static constexpr int kBranches = 4;
  cudaStream_t branch[kBranches] = {};
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kBranches] = {};
  RItem *d_items = nullptr;
  RTile *d_tiles = nullptr;
  int *d_counters = nullptr;     // next, error, done[items]
  void *d_tw = nullptr;
  std::vector<void *> work;      // per-item workspace (in-place two-pass)
  std::vector<mofft_ragged_item> items;
  std::vector<mofft_plan_f32 *> item_plans;   // per-item plans (baseline)
  cudaStream_t capture_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

static mofft_status ragged_fail(mofft_ragged_plan *p, mofft_status st) {
  mofft_ragged_plan_destroy(p);
  return st;
}

// A tuned plan for one group, if its schedule runs through pointer tables
// (at most two passes of specialised kernels).
static mofft_core *group_core(long long n, mofft_direction direction, long long transforms) {
  mofft_core *c = nullptr;
  if (mofft_core_create_pretuned(&c, 32, (size_t)n, (size_t)transforms, (size_t)n, direction,
                                 MOFFT_OUT_OF_PLACE) != MOFFT_SUCCESS)
    return nullptr;
  bool ok = c->sched.pass_count >= 1 && c->sched.pass_count <= 2;
  for (int q = 0; ok && q < c->sched.pass_count; ++q)
    ok = c->sched.pass[q].kind == MOFFT_KERNEL_ROWS || c->sched.pass[q].kind == MOFFT_KERNEL_COLS;
  if (!ok) {
    mofft_core_destroy(c);
    return nullptr;
  }
  return c;
}

static mofft_status ragged_create(mofft_ragged_plan **out, const mofft_ragged_item *items,
                                  size_t count, bool group_large) {
  if (!out) return MOFFT_INVALID_ARGUMENT;
  *out = nullptr;
  if (!items || count == 0 || count > (1u << 20)) return MOFFT_INVALID_ARGUMENT;
  if (!mofft_hardware_supports(32)) return MOFFT_UNSUPPORTED_HARDWARE;
  mofft_ragged_plan *p = new (std::nothrow) mofft_ragged_plan();
  if (!p) return MOFFT_ALLOCATION_FAILURE;
  cudaGetDevice(&p->device);
  p->items.assign(items, items + count);
  p->item_count = (int)count;
  p->work.assign(count, nullptr);
  // --- tuned groups for the items without a one-pass tile configuration
  std::vector<int> group_of(count, -1);
  if (group_large) {
    std::vector<std::pair<long long, int>> keys;   // (length, direction) per group
    std::vector<long long> transforms;
    for (size_t i = 0; i < count; ++i) {
      const mofft_ragged_item &u = items[i];
      if (!u.input || !u.output || u.batch == 0 || u.length < 2 ||
          (u.direction != MOFFT_FORWARD && u.direction != MOFFT_BACKWARD) ||
          rows_config_for((long long)u.length) >= 0)
        continue;
      const std::pair<long long, int> key((long long)u.length, (int)u.direction);
      size_t g = 0;
      while (g < keys.size() && keys[g] != key) ++g;
      if (g == keys.size()) {
        keys.push_back(key);
        transforms.push_back(0);
      }
      transforms[g] += (long long)u.batch;
      group_of[i] = (int)g;
    }
    std::vector<int> usable(keys.size(), -1);
    for (size_t g = 0; g < keys.size(); ++g) {
      mofft_core *c = group_core(keys[g].first, (mofft_direction)keys[g].second, transforms[g]);
      if (!c) continue;   // these items stay in the persistent queue
      RaggedGroup rg;
      rg.core = c;
      rg.transforms = transforms[g];
      rg.passes = c->sched.pass_count;
      usable[g] = (int)p->groups.size();
      p->groups.push_back(rg);
    }
    for (size_t i = 0; i < count; ++i)
      if (group_of[i] >= 0) group_of[i] = usable[group_of[i]];
  }
  // --- shape every item and lay out its twiddle tables
  std::vector<RItem> host_items(count);
  std::vector<size_t> tw0_off(count), tw1_off(count), hi_off(count), lo_off(count);
  size_t tw_bytes = 0;
  for (size_t i = 0; i < count; ++i) {
    const mofft_ragged_item &u = items[i];
    RItem &it = host_items[i];
    memset(&it, 0, sizeof(it));
    if (!u.input || !u.output || u.batch == 0 ||
        (u.direction != MOFFT_FORWARD && u.direction != MOFFT_BACKWARD))
      return ragged_fail(p, MOFFT_INVALID_ARGUMENT);
    it.n = (long long)u.length;
    it.batch = (long long)u.batch;
    it.dist = (long long)u.length;
    it.sign = u.direction == MOFFT_BACKWARD ? -1.0f : 1.0f;
    if (group_of[i] >= 0) continue;   // a tuned group runs it
    const int r = rows_config_for(it.n);
    if (r >= 0) {
      it.passes = 1;
      it.cfg0 = r;
      tw0_off[i] = tw_bytes;
      tw_bytes = round256(tw_bytes + (mofft_stage_table_entries(config(r).radices,
                                                                 config(r).radix_count) + 1) * 8);
      continue;
    }
    // two passes n = L0 * L1 with column configurations, most balanced first
    int best0 = -1, best1 = -1;
    for (const ConfigInfo &a : kConfigs) {
      if (!a.cols || it.n % a.length) continue;
      const int c1 = cols_config_for((int)(it.n / a.length));
      if (c1 < 0) continue;
      if (best0 < 0 || std::abs(a.length - config(c1).length) <
                           std::abs(config(best0).length - config(best1).length)) {
        best0 = a.id;
        best1 = c1;
      }
    }
    if (best0 < 0) return ragged_fail(p, MOFFT_UNSUPPORTED_SIZE);
    it.passes = 2;
    it.cfg0 = best0;
    it.cfg1 = best1;
    it.L0 = config(best0).length;
    const unsigned long long m = (unsigned long long)it.n;
    it.split1 = (mofft_ceil_log2_u64(m) + 1) / 2;
    tw0_off[i] = tw_bytes;
    tw_bytes = round256(tw_bytes + (mofft_stage_table_entries(config(best0).radices,
                                                               config(best0).radix_count) + 1) * 8);
    tw1_off[i] = tw_bytes;
    tw_bytes = round256(tw_bytes + (mofft_stage_table_entries(config(best1).radices,
                                                               config(best1).radix_count) + 1) * 8);
    const size_t lo_n = size_t(1) << it.split1;
    const size_t hi_n = (m + lo_n - 1) >> it.split1;
    hi_off[i] = tw_bytes;
    tw_bytes = round256(tw_bytes + hi_n * 8);
    lo_off[i] = tw_bytes;
    tw_bytes = round256(tw_bytes + lo_n * 8);
  }
  std::vector<unsigned char> host_tw(tw_bytes + 256);
  for (size_t i = 0; i < count; ++i) {
    if (group_of[i] >= 0) continue;
    const RItem &it = host_items[i];
    const ConfigInfo &c0 = config(it.cfg0);
    mofft_fill_stage_table(host_tw.data() + tw0_off[i], 32, c0.radices, c0.radix_count);
    if (it.passes == 2) {
      const ConfigInfo &c1 = config(it.cfg1);
      mofft_fill_stage_table(host_tw.data() + tw1_off[i], 32, c1.radices, c1.radix_count);
      const size_t lo_n = size_t(1) << it.split1;
      const size_t hi_n = ((size_t)it.n + lo_n - 1) >> it.split1;
      mofft_write_twiddles(host_tw.data() + hi_off[i], 32, (uint64_t)it.n, 0, lo_n, hi_n);
      mofft_write_twiddles(host_tw.data() + lo_off[i], 32, (uint64_t)it.n, 0, 1, lo_n);
    }
  }
  bool branches_ok = cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming) == cudaSuccess;
  for (int b = 0; b < mofft_ragged_plan::kBranches && branches_ok; ++b)
    branches_ok = cudaStreamCreateWithFlags(&p->branch[b], cudaStreamNonBlocking) == cudaSuccess &&
                  cudaEventCreateWithFlags(&p->join[b], cudaEventDisableTiming) == cudaSuccess;
  if (!branches_ok || cudaStreamCreateWithFlags(&p->capture_stream, cudaStreamNonBlocking) !=
                          cudaSuccess) {
    cudaGetLastError();
    return ragged_fail(p, MOFFT_INTERNAL_ERROR);
  }
  // uploads go through the plan's stream and are waited for: a cudaMemcpy
  // from pageable memory may return before its DMA has landed
  if (cudaMalloc(&p->d_tw, host_tw.size()) != cudaSuccess ||
      cudaMemcpyAsync(p->d_tw, host_tw.data(), host_tw.size(), cudaMemcpyHostToDevice,
                      p->capture_stream) != cudaSuccess ||
      cudaStreamSynchronize(p->capture_stream) != cudaSuccess) {
    cudaGetLastError();
    return ragged_fail(p, MOFFT_ALLOCATION_FAILURE);
  }
  const unsigned char *tw = static_cast<const unsigned char *>(p->d_tw);
  // --- buffers, then the tile queue
  std::vector<RTile> first, second;
  for (size_t i = 0; i < count; ++i) {
    if (group_of[i] >= 0) continue;
    RItem &it = host_items[i];
    it.in = static_cast<const float2 *>(items[i].input);
    it.out = static_cast<float2 *>(items[i].output);
    it.tw0 = reinterpret_cast<const float2 *>(tw + tw0_off[i]);
    if (it.passes == 1) {
      const int tb = kThreads / config(it.cfg0).tpl;
      for (long long b = 0; b < it.batch; b += tb) first.push_back({(int)i, 0, b, 0});
      continue;
    }
    it.tw1 = reinterpret_cast<const float2 *>(tw + tw1_off[i]);
    it.hi1 = reinterpret_cast<const float2 *>(tw + hi_off[i]);
    it.lo1 = reinterpret_cast<const float2 *>(tw + lo_off[i]);
    if (items[i].input == items[i].output) {
      if (cudaMalloc(&p->work[i], (size_t)(it.batch * it.n) * sizeof(float2)) != cudaSuccess) {
        cudaGetLastError();
        return ragged_fail(p, MOFFT_ALLOCATION_FAILURE);
      }
      it.mid = static_cast<float2 *>(p->work[i]);
    } else {
      it.mid = it.out;   // the second pass runs in place on the output
    }
    const long long groups0 = (it.n / it.L0) / kColsLines;
    const long long groups1 = (it.L0) / kColsLines;   // (n / L1) / C with n / L1 = L0
    it.pass1_tiles = (int)(groups0 * it.batch);
    for (long long b = 0; b < it.batch; ++b)
      for (long long g = 0; g < groups0; ++g) first.push_back({(int)i, 0, b, g * kColsLines});
    for (long long b = 0; b < it.batch; ++b)
      for (long long g = 0; g < groups1; ++g) second.push_back({(int)i, 1, b, g * kColsLines});
  }
  // largest items first within each phase (better tail balance)
  auto weight = [&](const RTile &t) { return host_items[t.item].n; };
  std::stable_sort(first.begin(), first.end(),
                   [&](const RTile &a, const RTile &b) { return weight(a) > weight(b); });
  std::vector<RTile> tiles(first);
  tiles.insert(tiles.end(), second.begin(), second.end());
  p->tile_count = (int)tiles.size();
  for (const ConfigInfo &c : kConfigs) p->smem = std::max(p->smem, c.smem);
  if (cudaMalloc(&p->d_items, count * sizeof(RItem)) != cudaSuccess ||
      cudaMalloc(&p->d_tiles, std::max<size_t>(1, tiles.size()) * sizeof(RTile)) !=
          cudaSuccess ||
      cudaMalloc(&p->d_counters, (count + 2) * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return ragged_fail(p, MOFFT_ALLOCATION_FAILURE);
  }
  if (cudaMemsetAsync(p->d_counters, 0, (count + 2) * sizeof(int), p->capture_stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(p->d_items, host_items.data(), count * sizeof(RItem),
                      cudaMemcpyHostToDevice, p->capture_stream) != cudaSuccess ||
      cudaMemcpyAsync(p->d_tiles, tiles.data(), tiles.size() * sizeof(RTile),
                      cudaMemcpyHostToDevice, p->capture_stream) != cudaSuccess ||
      cudaStreamSynchronize(p->capture_stream) != cudaSuccess ||
      cudaFuncSetAttribute(ragged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)p->smem) != cudaSuccess) {
    cudaGetLastError();
    return ragged_fail(p, MOFFT_INTERNAL_ERROR);
  }
  int per_sm = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ragged_kernel, kThreads, p->smem);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
  p->grid = std::max(1, std::min(per_sm * sms, p->tile_count));
  // --- pointer tables of the tuned groups: per pass the inputs, then the
  // outputs of its transforms; a two-pass transform goes through its output
  // (out of place) or a workspace of its item (in place) between the passes
  if (!p->groups.empty()) {
    size_t total = 0;
    for (RaggedGroup &g : p->groups) {
      g.table_off = total;
      total += (size_t)(2 * g.passes) * (size_t)g.transforms;
    }
    std::vector<void *> host(total, nullptr);
    std::vector<long long> next(p->groups.size(), 0);
    for (size_t i = 0; i < count; ++i) {
      if (group_of[i] < 0) continue;
      const RaggedGroup &g = p->groups[group_of[i]];
      const mofft_ragged_item &u = items[i];
      const long long n = (long long)u.length;
      float2 *in = static_cast<float2 *>(const_cast<void *>(u.input));
      float2 *outp = static_cast<float2 *>(u.output);
      float2 *mid = outp;
      if (g.passes == 2 && u.input == u.output) {
        if (cudaMalloc(&p->work[i], (size_t)u.batch * (size_t)n * sizeof(float2)) !=
            cudaSuccess) {
          cudaGetLastError();
          return ragged_fail(p, MOFFT_ALLOCATION_FAILURE);
        }
        mid = static_cast<float2 *>(p->work[i]);
      }
      const long long T = g.transforms;
      void **tab = host.data() + g.table_off;
      for (long long b = 0; b < (long long)u.batch; ++b) {
        const long long t = next[group_of[i]]++;
        tab[t] = in + b * n;
        if (g.passes == 1) {
          tab[T + t] = outp + b * n;
        } else {
          tab[T + t] = mid + b * n;
          tab[2 * T + t] = mid + b * n;
          tab[3 * T + t] = outp + b * n;
        }
      }
    }
    if (cudaMalloc(&p->d_ptr_tables, total * sizeof(void *)) != cudaSuccess ||
        cudaMemcpyAsync(p->d_ptr_tables, host.data(), total * sizeof(void *),
                        cudaMemcpyHostToDevice, p->capture_stream) != cudaSuccess ||
        cudaStreamSynchronize(p->capture_stream) != cudaSuccess) {
      cudaGetLastError();
      return ragged_fail(p, MOFFT_ALLOCATION_FAILURE);
    }
  }
  p->graph_launches = p->tile_count > 0 ? 1 : 0;
  for (const RaggedGroup &g : p->groups) p->graph_launches += g.passes;
  *out = p;
  return MOFFT_SUCCESS;
}

extern "C" mofft_status mofft_ragged_plan_create_f32(mofft_ragged_plan **out,
                                                     const mofft_ragged_item *items,
                                                     size_t count) {
  return ragged_create(out, items, count, true);
}

extern "C" mofft_status mofft_ragged_plan_create_single_launch_f32(
    mofft_ragged_plan **out, const mofft_ragged_item *items, size_t count) {
  return ragged_create(out, items, count, false);
}

static cudaError_t ragged_enqueue(mofft_ragged_plan *p, cudaStream_t s, int need_bias = 0) {
  cudaError_t e = cudaMemsetAsync(p->d_counters, 0, (p->item_count + 2) * sizeof(int), s);
  if (e != cudaSuccess) return e;
  int *next = p->d_counters;
  int *error = p->d_counters + 1;
  int *done = p->d_counters + 2;
  ragged_kernel<<<p->grid, kThreads, p->smem, s>>>(p->d_items, p->d_tiles, p->tile_count,
                                                     next, done, error, need_bias);
  return cudaGetLastError();
}

extern "C" mofft_status mofft_ragged_execute(mofft_ragged_plan *p, void *stream) {
  if (!p) return MOFFT_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!p->exec) {
    // capture the steady-state step (counter reset + persistent kernel) once
    if (cudaStreamBeginCapture(p->capture_stream, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess) {
      cudaGetLastError();
      return MOFFT_INTERNAL_ERROR;
    }
    // the persistent queue on the capture stream, the tuned groups on the
    // branches forked from it, all joined before the graph ends
    mofft_status gs = MOFFT_SUCCESS;
    cudaError_t e = cudaEventRecord(p->fork, p->capture_stream);
    for (int b = 0; b < mofft_ragged_plan::kBranches && e == cudaSuccess; ++b)
      e = cudaStreamWaitEvent(p->branch[b], p->fork, 0);
    if (e == cudaSuccess && p->tile_count > 0) e = ragged_enqueue(p, p->capture_stream);
    std::vector<size_t> order(p->groups.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    auto points = [&](size_t i) {
      return (double)p->groups[i].transforms * (double)p->groups[i].core->length;
    };
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t a, size_t b) { return points(a) > points(b); });
    double load[mofft_ragged_plan::kBranches] = {0.0};
    for (size_t i : order) {
      if (e != cudaSuccess || gs != MOFFT_SUCCESS) break;
      int b = 0;
      for (int q = 1; q < mofft_ragged_plan::kBranches; ++q)
        if (load[q] < load[b]) b = q;
      load[b] += points(i);
      const RaggedGroup &rg = p->groups[i];
      void **tab = p->d_ptr_tables + rg.table_off;
      const long long T = rg.transforms;
      const void *const *ins[2] = {(const void *const *)tab, (const void *const *)(tab + 2 * T)};
      void *const *outs[2] = {tab + T, tab + 3 * T};
      gs = mofft_core_enqueue_tables(rg.core, ins, outs, T, p->branch[b]);
    }
    for (int b = 0; b < mofft_ragged_plan::kBranches; ++b) {
      const cudaError_t r = cudaEventRecord(p->join[b], p->branch[b]);
      const cudaError_t w = cudaStreamWaitEvent(p->capture_stream, p->join[b], 0);
      if (e == cudaSuccess) e = r != cudaSuccess ? r : w;
    }
    if (gs != MOFFT_SUCCESS && e == cudaSuccess) e = cudaErrorUnknown;
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(p->capture_stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess || !g) {
      cudaGetLastError();
      if (g) cudaGraphDestroy(g);
      return MOFFT_INTERNAL_ERROR;
    }
    if (cudaGraphInstantiate(&p->exec, g, 0) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphDestroy(g);
      p->exec = nullptr;
      return MOFFT_INTERNAL_ERROR;
    }
    p->graph = g;
  }
  if (cudaGraphLaunch(p->exec, s) != cudaSuccess) {
    cudaGetLastError();
    return MOFFT_INTERNAL_ERROR;
  }
  mofft_count_launches((uint64_t)p->graph_launches);
  return MOFFT_SUCCESS;
}

// One run of the queue in which no second-pass dependency can be met: every
// second-pass tile gives up after its bounded wait, sets the error word and
// skips its work.  Checks that a lost dependency ends in an error status on a
// usable context, without any GPU fault.
extern "C" mofft_status mofft_ragged_check_lost_dependency(mofft_ragged_plan *p,
                                                           void *stream) {
  if (!p) return MOFFT_INVALID_ARGUMENT;
  if (p->tile_count == 0) return MOFFT_SUCCESS;
  if (ragged_enqueue(p, static_cast<cudaStream_t>(stream), 1 << 30) != cudaSuccess) {
    cudaGetLastError();
    return MOFFT_INTERNAL_ERROR;
  }
  mofft_count_launches(1);
  return MOFFT_SUCCESS;
}

extern "C" mofft_status mofft_ragged_status(mofft_ragged_plan *p) {
  if (!p) return MOFFT_INVALID_ARGUMENT;
  int error = 0;
  if (cudaMemcpy(&error, p->d_counters + 1, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return MOFFT_INTERNAL_ERROR;
  }
  for (const RaggedGroup &g : p->groups)
    if (mofft_core_check_status(g.core) != MOFFT_SUCCESS) return MOFFT_INTERNAL_ERROR;
  return error ? MOFFT_INTERNAL_ERROR : MOFFT_SUCCESS;
}

extern "C" mofft_status mofft_ragged_execute_per_item(mofft_ragged_plan *p, void *stream) {
  if (!p) return MOFFT_INVALID_ARGUMENT;
  if (p->item_plans.empty()) {
    p->item_plans.assign(p->items.size(), nullptr);
    for (size_t i = 0; i < p->items.size(); ++i) {
      const mofft_ragged_item &u = p->items[i];
      const mofft_status st = mofft_plan_create_batched_f32(
          &p->item_plans[i], u.length, u.batch, 0, (mofft_direction)u.direction,
          u.input == u.output ? MOFFT_IN_PLACE : MOFFT_OUT_OF_PLACE, nullptr, nullptr);
      if (st != MOFFT_SUCCESS) return st;
    }
  }
  for (size_t i = 0; i < p->items.size(); ++i) {
    mofft_plan_set_stream_f32(p->item_plans[i], stream);
    const mofft_ragged_item &u = p->items[i];
    const mofft_status st =
        mofft_execute_f32(p->item_plans[i], static_cast<const mofft_complex_f32 *>(u.input),
                          static_cast<mofft_complex_f32 *>(u.output));
    if (st != MOFFT_SUCCESS) return st;
  }
  return MOFFT_SUCCESS;
}

extern "C" void mofft_ragged_plan_destroy(mofft_ragged_plan *p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->capture_stream) cudaStreamDestroy(p->capture_stream);
  for (int b = 0; b < mofft_ragged_plan::kBranches; ++b) {
    if (p->branch[b]) cudaStreamDestroy(p->branch[b]);
    if (p->join[b]) cudaEventDestroy(p->join[b]);
  }
  if (p->fork) cudaEventDestroy(p->fork);
  for (mofft_plan_f32 *plan : p->item_plans) mofft_plan_destroy_f32(plan);
  for (RaggedGroup &g : p->groups)
    if (g.core) mofft_core_destroy(g.core);
  if (p->d_ptr_tables) cudaFree(p->d_ptr_tables);
  for (void *w : p->work)
    if (w) cudaFree(w);
  if (p->d_items) cudaFree(p->d_items);
  if (p->d_tiles) cudaFree(p->d_tiles);
  if (p->d_counters) cudaFree(p->d_counters);
  if (p->d_tw) cudaFree(p->d_tw);
  delete p;
}

extern "C" mofft_status mofft_ragged_plan_info(const mofft_ragged_plan *p, size_t *tiles,
                                               int *grid) {
  if (!p || !tiles || !grid) return MOFFT_INVALID_ARGUMENT;
  *tiles = (size_t)p->tile_count;
  *grid = p->grid;
  return MOFFT_SUCCESS;
}
