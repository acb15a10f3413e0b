/* Analytical cost model behind the mofft_estimated_* API.
 *
 * The byte accounting restates the reference's estimate_stage_cost and
 * mofft_estimated_plan_cost_breakdown_with_layout (src/mofft.c:133-325)
 * exactly: every stage reads and writes all N points, later stages also read
 * a compact twiddle table of stage_length entries, materialised transposes
 * add a full read+write pass, direct strided input and the section layout pay
 * cache-line overfetch.  The line size is 128 bytes, which is also B200's L2
 * line.  What is re-parameterised for B200 are the time constants:
 *   arithmetic: generated codelet add/mul counts (+6 flops per twiddle) over
 *               the FP32 (72 TFLOP/s) or FP64 (36 TFLOP/s) CUDA-core rate,
 *               per warp-wide batch of 32 butterflies;
 *   memory:     bytes over L2 bandwidth (20 TB/s) when the working set fits
 *               in 100 MB of L2, else over HBM3e (6.5 TB/s).
 * Costs are reported in nanoseconds. */
#include <float.h>
#include <math.h>
#include <string.h>

#include "generated/codelet_costs.h"
#include "mofft_host.h"

#define LINE_BYTES 128u
#define LANES 32u
#define FP32_FLOPS 72.0e12
#define FP64_FLOPS 36.0e12
#define HBM_BPS 6.5e12
#define L2_BPS 20.0e12
#define L2_RESIDENT_BYTES (100u * 1024u * 1024u)

static size_t sat_mul(size_t a, size_t b) {
  return a != 0 && b > SIZE_MAX / a ? SIZE_MAX : a * b;
}
static size_t sat_add(size_t a, size_t b) { return b > SIZE_MAX - a ? SIZE_MAX : a + b; }

static int codelet_flops(int radix) {
  for (int i = 0; i < MOFFT_CODELET_COST_COUNT; ++i)
    if (k_mofft_codelet_costs[i].radix == radix)
      return k_mofft_codelet_costs[i].adds + k_mofft_codelet_costs[i].muls;
  return -1;
}

double mofft_estimated_radix_cost(int radix, int precision_bits, int first_stage) {
  if ((precision_bits != 32 && precision_bits != 64) || !mofft_is_supported_radix(radix))
    return DBL_MAX;
  const int flops = codelet_flops(radix);
  if (flops < 0) return DBL_MAX;
  const double total = (double)flops + (first_stage ? 0.0 : 6.0 * (radix - 1));
  const double rate = precision_bits == 32 ? FP32_FLOPS : FP64_FLOPS;
  return total * LANES / rate * 1e9;
}

static double memory_cost(size_t working_set, size_t reads, size_t writes) {
  const double bw = working_set <= L2_RESIDENT_BYTES ? L2_BPS : HBM_BPS;
  return ((double)reads + (double)writes) / bw * 1e9;
}

static double transpose_cost(size_t working_set, size_t data_bytes,
                             size_t parent_batch, size_t complex_bytes,
                             int blocked) {
  const size_t useful = sat_mul(parent_batch, complex_bytes);
  double reads = (double)data_bytes;
  if (!blocked && useful < LINE_BYTES)
    reads = (double)data_bytes * (double)LINE_BYTES / (double)(useful ? useful : 1);
  const double bw = working_set <= L2_RESIDENT_BYTES ? L2_BPS : HBM_BPS;
  return (reads + (double)data_bytes) / bw * 1e9;
}

typedef struct {
  double kernel_cost, memory_cost, total_cost;
  size_t logical_read_bytes, logical_write_bytes, working_set_bytes;
} stage_cost;

static int estimate_stage(int radix, int precision_bits, int first_stage,
                          size_t transform_length, size_t stage_length,
                          size_t extra_read_bytes, stage_cost *r) {
  if (radix < 2 || (precision_bits != 32 && precision_bits != 64) ||
      transform_length == 0 || stage_length == 0 ||
      stage_length > transform_length || transform_length % (size_t)radix != 0 || !r)
    return 0;
  const double unit = mofft_estimated_radix_cost(radix, precision_bits, first_stage);
  if (unit == DBL_MAX) return 0;
  const size_t independent = transform_length / (size_t)radix;
  r->kernel_cost = unit * (double)((independent + LANES - 1) / LANES);
  const size_t cb = mofft_complex_bytes(precision_bits);
  const size_t data = sat_mul(transform_length, cb);
  const size_t tw = first_stage ? 0 : sat_mul(stage_length, cb);
  r->logical_read_bytes = sat_add(data, tw);
  r->logical_write_bytes = data;
  r->working_set_bytes = sat_add(sat_mul(data, 2), tw);
  r->memory_cost = memory_cost(r->working_set_bytes,
                               sat_add(r->logical_read_bytes, extra_read_bytes),
                               r->logical_write_bytes);
  r->total_cost = r->kernel_cost > r->memory_cost ? r->kernel_cost : r->memory_cost;
  return 1;
}

double mofft_estimated_stage_cost(int radix, int precision_bits, int first_stage,
                                  size_t transform_length, size_t stage_length) {
  stage_cost c;
  return estimate_stage(radix, precision_bits, first_stage, transform_length,
                        stage_length, 0, &c)
             ? c.total_cost
             : DBL_MAX;
}

static size_t divide_by_utilisation(size_t bytes, size_t useful, size_t line) {
  if (useful >= line) return bytes;
  if (useful == 0 || bytes > SIZE_MAX / line) return SIZE_MAX;
  const size_t product = bytes * line;
  if (product > SIZE_MAX - (useful - 1)) return SIZE_MAX;
  return (product + useful - 1) / useful;
}

mofft_status mofft_estimated_plan_cost_breakdown_with_layout(
    size_t length, int precision_bits, const int *radices, size_t radix_count,
    uint64_t blocked_transpose_mask, int direct_input, mofft_stage_layout layout,
    mofft_plan_cost_breakdown *b) {
  if (!radices || radix_count == 0 || radix_count > MOFFT_MAX_PLAN_DEPTH ||
      length < 2 || (precision_bits != 32 && precision_bits != 64) ||
      (direct_input != 0 && direct_input != 1) ||
      (layout != MOFFT_STAGE_LAYOUT_TRANSPOSE && layout != MOFFT_STAGE_LAYOUT_SECTION) ||
      (radix_count - 1 < 64 && (blocked_transpose_mask >> (radix_count - 1))) || !b)
    return MOFFT_INVALID_ARGUMENT;
  memset(b, 0, sizeof(*b));
  /* the reference's direct-input threshold: half of its vector lanes */
  const size_t lanes = precision_bits == 32 ? 16 : 8;
  const size_t cb = mofft_complex_bytes(precision_bits);
  const size_t data = sat_mul(length, cb);
  size_t n = length;
  for (size_t level = 0; level < radix_count; ++level) {
    const int radix = radices[level];
    if (!mofft_is_supported_radix(radix) || n % (size_t)radix != 0)
      return MOFFT_INVALID_ARGUMENT;
    const size_t remainder = n / (size_t)radix;
    size_t extra = 0;
    const int fused = radix_count == 2 && level == 0;
    if (remainder != 1 && layout == MOFFT_STAGE_LAYOUT_SECTION) {
      const size_t transferred = divide_by_utilisation(data, sat_mul(remainder, cb), LINE_BYTES);
      extra = transferred > data ? transferred - data : 0;
    } else if (remainder != 1 && !fused) {
      const size_t parent_batch = length / n;
      const size_t useful = sat_mul(parent_batch, cb);
      if (direct_input && parent_batch >= lanes / 2) {
        const size_t transferred = divide_by_utilisation(data, useful, LINE_BYTES);
        extra = transferred > data ? transferred - data : 0;
      } else {
        const int blocked = (int)((blocked_transpose_mask >> level) & UINT64_C(1));
        const size_t ws = sat_mul(data, 2);
        b->layout_cost += transpose_cost(ws, data, parent_batch, cb, blocked);
        b->logical_read_bytes = sat_add(b->logical_read_bytes, data);
        b->logical_write_bytes = sat_add(b->logical_write_bytes, data);
        const size_t layout_reads = blocked ? data : divide_by_utilisation(data, useful, LINE_BYTES);
        b->transferred_read_bytes = sat_add(b->transferred_read_bytes, layout_reads);
        b->transferred_write_bytes = sat_add(b->transferred_write_bytes, data);
        if (ws > b->peak_working_set_bytes) b->peak_working_set_bytes = ws;
      }
    }
    stage_cost s;
    if (!estimate_stage(radix, precision_bits, remainder == 1, length, n, extra, &s))
      return MOFFT_INVALID_ARGUMENT;
    b->kernel_cost += s.kernel_cost;
    b->memory_cost += s.memory_cost;
    b->total_cost += s.total_cost;
    b->logical_read_bytes = sat_add(b->logical_read_bytes, s.logical_read_bytes);
    b->logical_write_bytes = sat_add(b->logical_write_bytes, s.logical_write_bytes);
    b->transferred_read_bytes =
        sat_add(b->transferred_read_bytes, sat_add(s.logical_read_bytes, extra));
    b->transferred_write_bytes = sat_add(b->transferred_write_bytes, s.logical_write_bytes);
    if (s.working_set_bytes > b->peak_working_set_bytes)
      b->peak_working_set_bytes = s.working_set_bytes;
    n = remainder;
  }
  if (n != 1) return MOFFT_INVALID_ARGUMENT;
  b->total_cost += b->layout_cost;
  return MOFFT_SUCCESS;
}

double mofft_estimated_plan_cost_with_layout(size_t length, int precision_bits,
                                             const int *radices, size_t radix_count,
                                             uint64_t blocked_transpose_mask,
                                             int direct_input, mofft_stage_layout layout) {
  mofft_plan_cost_breakdown b;
  return mofft_estimated_plan_cost_breakdown_with_layout(
             length, precision_bits, radices, radix_count, blocked_transpose_mask,
             direct_input, layout, &b) == MOFFT_SUCCESS
             ? b.total_cost
             : DBL_MAX;
}

double mofft_estimated_plan_cost(size_t length, int precision_bits,
                                 const int *radices, size_t radix_count,
                                 uint64_t blocked_transpose_mask, int direct_input) {
  return mofft_estimated_plan_cost_with_layout(length, precision_bits, radices,
                                               radix_count, blocked_transpose_mask,
                                               direct_input, MOFFT_STAGE_LAYOUT_TRANSPOSE);
}
