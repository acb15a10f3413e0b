/* Device-time model of a GPU schedule: the planner's prior.
 *
 * The reference ranks factorizations with its cost model
 * (choose_factorization, src/mofft.c:327-351) and shortlists MEASURE
 * candidates by model cost before timing them (src/mofft.c:874-922).  Its
 * model prices SME codelets, cache lines and transposes; this one prices what
 * decides a schedule's time on B200 and is used the same two ways (the
 * PRETUNED split choice in mofft_model_chain, the MEASURE shortlist order).
 * Per pass:
 *
 *   memory   every pass reads and writes every point once, 2 N B c bytes
 *            (c = 8 or 16) at the HBM copy bandwidth, derated by
 *              - the run length of the strided side of a column pass: a tile
 *                of C adjacent lines moves runs of C c bytes, and runs
 *                shorter than a 128-byte line waste part of each DRAM burst
 *                (the first pass of a multi-pass transform writes whole
 *                lines; later passes read and write runs);
 *              - latency hiding: the bytes one SM holds in flight (resident
 *                CTAs x tile bytes) against the ~64 KB a B200 SM needs to
 *                cover DRAM latency at its share of the bandwidth;
 *   issue    instructions per point: each stage's codelet arithmetic
 *            (adds + muls of the generated radix-R codelet per point, FMA-
 *            fused), a twiddle multiply on every stage but a pass's first
 *            (and on the first of a later pass: the super-stage twiddle), a
 *            shared-memory exchange between stages, global load and store;
 *            FP64 arithmetic at a lower rate; over the SMs' issue rate;
 *            the runtime-stage kernels pay their stage loop;
 *   time     max(memory, issue) + a quarter of the smaller (imperfect
 *            overlap) + a launch.
 *
 * Constants: 148 SMs, 228 KB shared memory and 2048 threads per SM, four
 * schedulers at 1.9 GHz, copy bandwidth 6.5 TB/s. */
#include <float.h>
#include <math.h>
#include <string.h>

#include "generated/codelet_costs.h"
#include "mofft_host.h"

#define GM_SMS 148.0
#define GM_HBM_BPS 6.5e12
#define GM_THREAD_INSTR_PER_S (GM_SMS * 4.0 * 32.0 * 1.9e9)
#define GM_SMEM_PER_SM (228.0 * 1024.0)
#define GM_THREADS_PER_SM 2048.0
#define GM_INFLIGHT_BYTES (64.0 * 1024.0)
#define GM_LAUNCH_S 3.0e-6
#define GM_ISSUE_EFF 0.7

static double codelet_instr_per_point(int radix) {
  /* the generator's count: one instruction per add, a product feeding a sum
   * fused into one FMA */
  for (int i = 0; i < MOFFT_CODELET_COST_COUNT; ++i)
    if (k_mofft_codelet_costs[i].radix == radix)
      return (double)k_mofft_codelet_costs[i].instr / radix;
  return 8.0;
}

/* Fraction of each DRAM burst a run of `bytes` contiguous bytes uses. */
static double run_efficiency(double bytes) {
  if (bytes >= 128.0) return 1.0;
  return 0.3 + 0.7 * bytes / 128.0;
}

static double pass_seconds(int precision_bits, size_t length, size_t batch,
                           const mofft_pass *ps, int first_pass) {
  const mofft_kernel_desc *d = mofft_cuda_kernel_get(ps->kernel);
  if (!d) return DBL_MAX;
  const double cb = precision_bits == 32 ? 8.0 : 16.0;
  const double points = (double)length * (double)batch;
  const int cols = ps->kind == MOFFT_KERNEL_COLS || ps->kind == MOFFT_KERNEL_TENSOR_COLS ||
                   (ps->kind == MOFFT_KERNEL_GENERIC && (size_t)ps->length != length);
  const int lines = ps->kind == MOFFT_KERNEL_GENERIC ? ps->lines : d->lines;
  /* memory */
  double e_read = 0.95, e_write = 0.95;
  if (cols) {
    const double run = (double)(lines > 0 ? lines : 1) * cb;
    e_read = run_efficiency(run);
    e_write = ps->ns_outer > 1 ? run_efficiency(run) : 0.95;
  }
  const double e_mem = 2.0 / (1.0 / e_read + 1.0 / e_write);
  const double smem =
      (double)(ps->kind == MOFFT_KERNEL_GENERIC ? ps->smem_bytes : d->smem_bytes);
  const double threads = (double)(d->threads > 0 ? d->threads : 256);
  double ctas = floor(GM_THREADS_PER_SM / threads);
  if (smem > 0.0 && GM_SMEM_PER_SM / smem < ctas) ctas = floor(GM_SMEM_PER_SM / smem);
  if (ctas > 32.0) ctas = 32.0;
  if (ctas < 1.0) ctas = 1.0;
  const double tile = (double)ps->length * (double)(lines > 0 ? lines : 1) * cb;
  double e_lat = ctas * tile / GM_INFLIGHT_BYTES;
  if (d->prefetch || ps->kind == MOFFT_KERNEL_TENSOR) e_lat = 1.0;
  if (e_lat > 1.0) e_lat = 1.0;
  const double t_mem = 2.0 * points * cb / (GM_HBM_BPS * e_mem * e_lat);
  /* issue */
  double instr = 4.0; /* global load / store, addressing */
  for (int s = 0; s < ps->radix_count; ++s) {
    instr += codelet_instr_per_point(ps->radices[s]);
    if (s > 0 || !first_pass) instr += 5.0; /* twiddle load + complex multiply */
    if (s > 0) instr += 4.0;                /* exchange: store and load re, im */
  }
  if (ps->kind == MOFFT_KERNEL_GENERIC) instr *= 2.0;
  if (precision_bits == 64) instr *= 1.6;
  if (ps->kind == MOFFT_KERNEL_TENSOR || ps->kind == MOFFT_KERNEL_TENSOR_COLS) instr *= 0.6;
  const double t_issue = points * instr / (GM_THREAD_INSTR_PER_S * GM_ISSUE_EFF);
  const double hi = t_mem > t_issue ? t_mem : t_issue;
  const double lo = t_mem > t_issue ? t_issue : t_mem;
  return hi + 0.25 * lo + GM_LAUNCH_S;
}

double mofft_gpu_schedule_seconds(int precision_bits, size_t length, size_t batch,
                                  const mofft_schedule *s) {
  if (!s || s->pass_count <= 0) return DBL_MAX;
  double total = 0.0;
  for (int p = 0; p < s->pass_count; ++p) {
    const double t = pass_seconds(precision_bits, length, batch, &s->pass[p], p == 0);
    if (t == DBL_MAX) return DBL_MAX;
    total += t;
  }
  return total;
}

double mofft_schedule_model_seconds(int precision_bits, size_t length, size_t batch,
                                    const int *kernels, size_t pass_count) {
  if ((precision_bits != 32 && precision_bits != 64) || length < 2 || batch == 0 ||
      !kernels || pass_count == 0 || pass_count > MOFFT_MAX_PASSES)
    return DBL_MAX;
  int chain[MOFFT_MAX_STAGES];
  int preferred[MOFFT_MAX_PASSES];
  int depth = 0;
  size_t product = 1;
  for (int i = 0; i < MOFFT_MAX_PASSES; ++i) preferred[i] = -1;
  for (size_t p = 0; p < pass_count; ++p) {
    const mofft_kernel_desc *d = mofft_cuda_kernel_get(kernels[p]);
    if (!d || d->precision_bits != precision_bits || d->radix_count <= 0 ||
        depth + d->radix_count > MOFFT_MAX_STAGES)
      return DBL_MAX;
    memcpy(chain + depth, d->radices, (size_t)d->radix_count * sizeof(int));
    depth += d->radix_count;
    product *= (size_t)d->length;
    preferred[p] = kernels[p];
  }
  if (product != length) return DBL_MAX;
  mofft_schedule s;
  if (!mofft_group_chain_preferred(precision_bits, 0, chain, depth, (long long)length,
                                   preferred, &s) ||
      s.pass_count != (int)pass_count)
    return DBL_MAX;
  for (size_t p = 0; p < pass_count; ++p)
    if (s.pass[p].kernel != kernels[p]) return DBL_MAX;
  return mofft_gpu_schedule_seconds(precision_bits, length, batch, &s);
}
