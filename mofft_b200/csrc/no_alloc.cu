// Allocation-free execution of two-pass FP32 transforms.
//
// The plan API allocates device memory when a plan is created (twiddle
// tables, and for in-place multi-pass transforms a workspace).  Some callers
// cannot do that: code that runs inside a host framework which reserves the
// whole GPU memory budget up front and forbids further cudaMalloc calls, and
// latency-critical loops in which a cudaMalloc / cudaFree (which may
// synchronize the device) is not acceptable.  mofft_execute_fixed_scratch_f32
// serves them: it allocates nothing.  The intermediate array of the four-step
// transform and its twiddle tables live in one file-scope __device__ array
// whose size is fixed at build time; every GPU that loads libmofft.so holds
// that array until the process exits.
//
// Host code must not use the array's name as a device address (on the host
// it only names a stand-in).  The first call on each device, with that
// device current, resolves the array's device address with
// cudaGetSymbolAddress and caches it; that first call should therefore come
// before any stream capture on that device.  All calls share the array and
// it keeps the last call's contents: nothing in it needs to start at zero
// (each call rewrites the twiddle region and fully overwrites the data region
// before reading it), and calls whose executions overlap on the GPU race on
// it -- callers must order them, e.g. on one stream.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "mofft_cuda.h"
#include "mofft_host.h"

namespace {

constexpr size_t kScratchPoints = MOFFT_FIXED_SCRATCH_POINTS;
constexpr size_t kTwiddleEntries = size_t(1) << 16;
constexpr int kMaxRegions = 128;
constexpr int kMaxDevices = 64;

// Data region (kScratchPoints complex64) followed by the twiddle region.
static __device__ __align__(256) float2 g_fixed_scratch[kScratchPoints + kTwiddleEntries];

std::mutex g_setup_mutex;
void *g_scratch_address[kMaxDevices];

// One twiddle run: count entries W_den^(k*step), k = 0..count-1, at offset
// (den == 0: count zero entries).
struct FillRegions {
  int count;
  unsigned long long den[kMaxRegions];
  unsigned long long step[kMaxRegions];
  unsigned int entries[kMaxRegions];
  unsigned int offset[kMaxRegions];
};

__global__ void fill_twiddle_regions(float2 *base, const FillRegions d,
                                     unsigned int total) {
  for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += gridDim.x * blockDim.x) {
    int r = 0;
    unsigned int start = 0;
    while (r < d.count && i >= start + d.entries[r]) {
      start += d.entries[r];
      ++r;
    }
    if (r >= d.count) continue;
    if (d.den[r] == 0) {  // the spare entry behind a stage table
      base[d.offset[r] + (i - start)] = make_float2(0.0f, 0.0f);
      continue;
    }
    const unsigned long long k = i - start;
    const unsigned long long e = (k * d.step[r]) % d.den[r];
    double s, c;
    sincospi(2.0 * (double)e / (double)d.den[r], &s, &c);
    base[d.offset[r] + k] = make_float2((float)c, (float)-s);
  }
}

int ceil_log2(unsigned long long x) {
  int s = 0;
  while ((1ull << s) < x) ++s;
  return s;
}

size_t round32(size_t x) { return (x + 31) & ~size_t(31); }

// Resolve (once per device, with that device current) the device address of
// g_fixed_scratch and opt the kernels into their shared memory sizes.
mofft_status scratch_address(int device, float2 **out) {
  if (device < 0 || device >= kMaxDevices) return MOFFT_UNSUPPORTED_HARDWARE;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_address[device]) {
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_fixed_scratch) != cudaSuccess || !ptr) {
      cudaGetLastError();
      return MOFFT_INTERNAL_ERROR;
    }
    if (mofft_cuda_prepare_device() != 0) {
      cudaGetLastError();
      return MOFFT_INTERNAL_ERROR;
    }
    g_scratch_address[device] = ptr;
  }
  *out = static_cast<float2 *>(g_scratch_address[device]);
  return MOFFT_SUCCESS;
}

bool is_device_memory(const void *p) {
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" mofft_status mofft_execute_fixed_scratch_f32(
    const mofft_complex_f32 *input, mofft_complex_f32 *output, size_t length,
    size_t batch, mofft_direction direction, void *stream) {
  if (!input || !output || batch == 0 ||
      (direction != MOFFT_FORWARD && direction != MOFFT_BACKWARD))
    return MOFFT_INVALID_ARGUMENT;
  if (length < 2 || !mofft_is_smooth13(length)) return MOFFT_UNSUPPORTED_SIZE;
  if (batch > kScratchPoints / length) return MOFFT_UNSUPPORTED_SIZE;
  if (!mofft_hardware_supports(32)) return MOFFT_UNSUPPORTED_HARDWARE;
  if (!is_device_memory(input) || !is_device_memory(output))
    return MOFFT_INVALID_ARGUMENT;

  // Only two-pass schedules need the intermediate array this entry point
  // provides.  The tuned schedule of the compiled wisdom runs when it has two
  // passes (the same kernels an out-of-place PRETUNED plan runs); otherwise
  // the model's schedule runs when it has two (a tuned three-pass schedule
  // would need a second intermediate array).
  int chain[MOFFT_MAX_STAGES];
  int preferred[MOFFT_MAX_PASSES];
  mofft_schedule sched;
  sched.pass_count = 0;
  const int tuned = mofft_wisdom_lookup(length, 32, chain, MOFFT_MAX_STAGES, preferred);
  if (tuned > 0 && preferred[0] >= 0 && preferred[1] >= 0 &&
      (MOFFT_MAX_PASSES < 3 || preferred[2] < 0)) {
    if (!mofft_group_chain_preferred(32, 0, chain, tuned, (long long)length, preferred,
                                     &sched))
      sched.pass_count = 0;
  }
  if (sched.pass_count != 2) {
    int count = mofft_model_chain(32, 0, length, chain, MOFFT_MAX_STAGES);
    if (count <= 0 || !mofft_group_chain(32, 0, chain, count, (long long)length, &sched))
      return MOFFT_UNSUPPORTED_SIZE;
    // A length that a thread-block cluster computes in one pass still has its
    // two-pass schedule here: this entry point is the two-pass path.
    const mofft_kernel_desc *d = mofft_cuda_kernel_get(sched.pass[0].kernel);
    if (sched.pass_count == 1 && d && d->cluster > 0) {
      count = mofft_model_chain_multipass(32, 0, length, chain, MOFFT_MAX_STAGES);
      if (count <= 0 || !mofft_group_chain(32, 0, chain, count, (long long)length, &sched))
        return MOFFT_UNSUPPORTED_SIZE;
    }
  }
  if (sched.pass_count != 2) return MOFFT_UNSUPPORTED_SIZE;

  // Twiddle layout: per pass the internal stage table, then (second pass)
  // the two-level super-stage table, as the plan builder lays them out.
  FillRegions regions;
  regions.count = 0;
  size_t cursor = 0;
  size_t tw_off[2], hi_off[2], lo_off[2];
  int split_shift[2] = {0, 0};
  for (int p = 0; p < 2; ++p) {
    const mofft_pass &ps = sched.pass[p];
    tw_off[p] = cursor;
    unsigned long long ns = 1;
    for (int s = 0; s < ps.radix_count; ++s) {
      const unsigned long long R = (unsigned long long)ps.radices[s];
      if (ns > 1) {
        for (unsigned long long r = 1; r < R; ++r) {
          if (regions.count >= kMaxRegions) return MOFFT_UNSUPPORTED_SIZE;
          regions.den[regions.count] = ns * R;
          regions.step[regions.count] = r;
          regions.entries[regions.count] = (unsigned int)ns;
          regions.offset[regions.count] = (unsigned int)cursor;
          ++regions.count;
          cursor += ns;
        }
      }
      ns *= R;
    }
    // one spare entry behind the stage table, zero as in a plan's table
    if (regions.count >= kMaxRegions) return MOFFT_UNSUPPORTED_SIZE;
    regions.den[regions.count] = 0;
    regions.step[regions.count] = 0;
    regions.entries[regions.count] = 1;
    regions.offset[regions.count] = (unsigned int)cursor;
    ++regions.count;
    cursor = round32(cursor + 1);
    hi_off[p] = lo_off[p] = cursor;
    if (ps.ns_outer > 1) {
      const unsigned long long m = (unsigned long long)ps.ns_outer * ps.length;
      const int shift = (ceil_log2(m) + 1) / 2;
      const unsigned long long lo_n = 1ull << shift;
      const unsigned long long hi_n = (m + lo_n - 1) >> shift;
      if (regions.count + 2 > kMaxRegions) return MOFFT_UNSUPPORTED_SIZE;
      split_shift[p] = shift;
      hi_off[p] = cursor;
      regions.den[regions.count] = m;
      regions.step[regions.count] = lo_n;
      regions.entries[regions.count] = (unsigned int)hi_n;
      regions.offset[regions.count] = (unsigned int)cursor;
      ++regions.count;
      cursor = round32(cursor + hi_n);
      lo_off[p] = cursor;
      regions.den[regions.count] = m;
      regions.step[regions.count] = 1;
      regions.entries[regions.count] = (unsigned int)lo_n;
      regions.offset[regions.count] = (unsigned int)cursor;
      ++regions.count;
      cursor = round32(cursor + lo_n);
    }
  }
  if (cursor > kTwiddleEntries) return MOFFT_UNSUPPORTED_SIZE;

  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return MOFFT_INTERNAL_ERROR;
  }
  float2 *scratch = nullptr;
  mofft_status st = scratch_address(device, &scratch);
  if (st != MOFFT_SUCCESS) return st;
  float2 *data = scratch;
  float2 *tw = scratch + kScratchPoints;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  unsigned int total = 0;
  for (int r = 0; r < regions.count; ++r) total += regions.entries[r];
  if (total > 0) {
    const unsigned int blocks = (total + 255) / 256 < 1024 ? (total + 255) / 256 : 1024;
    fill_twiddle_regions<<<blocks, 256, 0, s>>>(tw, regions, total);
    if (cudaGetLastError() != cudaSuccess) return MOFFT_INTERNAL_ERROR;
  }

  // pass 1: input -> scratch, pass 2: scratch -> output (input == output is
  // fine: the second pass never reads the input).
  const bool backward = direction == MOFFT_BACKWARD;
  for (int p = 0; p < 2; ++p) {
    const mofft_pass &ps = sched.pass[p];
    mofft_pass_args a;
    memset(&a, 0, sizeof(a));
    a.in = p == 0 ? static_cast<const void *>(input) : static_cast<const void *>(data);
    a.out = p == 0 ? static_cast<void *>(data) : static_cast<void *>(output);
    a.tw = tw + tw_off[p];
    a.tw_hi = tw + hi_off[p];
    a.tw_lo = tw + lo_off[p];
    a.batch = (long long)batch;
    a.in_dist = (long long)length;
    a.out_dist = (long long)length;
    a.total = (long long)length;
    a.ns_outer = ps.ns_outer;
    a.split_shift = split_shift[p];
    a.conj_in = backward && p == 0;
    a.conj_out = backward && p == 1;
    a.generic_cols = 1;
    a.length = ps.length;
    a.lines = ps.lines;
    a.radix_count = ps.radix_count;
    memcpy(a.radices, ps.radices, sizeof(a.radices));
    if (mofft_cuda_launch_pass(ps.kernel, &a, stream) != 0) {
      cudaGetLastError();
      return MOFFT_INTERNAL_ERROR;
    }
  }
  return MOFFT_SUCCESS;
}
