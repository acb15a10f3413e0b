/* MEASURE planner: the GPU autotuner behind MOFFT_PLANNER_MEASURE.
 *
 * Semantics follow the reference's search_best_plan (src/mofft.c:798-1052):
 *  - a bounded candidate list (options->candidate_limit), in model order,
 *    covering every kernel bank before spending the rest of the budget;
 *  - a deterministic xorshift shuffle of the measurement order
 *    (src/mofft.c:932-942);
 *  - a deterministic xorshift input (src/mofft.c:959-972);
 *  - per candidate: one warm execution, a finite-output check, then
 *    `timing_samples` samples, each the median of `iterations` executions,
 *    and the candidate's score is the median of its samples;
 *  - in-place candidates get their input reset outside the timed region;
 *  - the winner is rebuilt and returned, with diagnostics.
 * What changes on the GPU: candidates are complete device schedules (radix
 * chain x pass split x kernel family), executions are timed with CUDA events
 * on the plan's stream, and only one candidate's device state is alive at a
 * time besides the shared input/output buffers. */
#include <cuda_runtime_api.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "mofft_host.h"

typedef struct {
  int chain[MOFFT_MAX_STAGES];
  int count;
  unsigned bank;
  int preferred[MOFFT_MAX_PASSES];   /* kernel instances to use, -1 = default */
  double model;
  size_t model_rank;
  double samples[32];
  double median;
} candidate;

static double median_of(double *v, size_t n) {
  if (n == 0) return INFINITY;
  for (size_t i = 1; i < n; ++i) {
    const double x = v[i];
    size_t j = i;
    while (j > 0 && x < v[j - 1]) {
      v[j] = v[j - 1];
      --j;
    }
    v[j] = x;
  }
  return n & 1 ? v[n / 2] : 0.5 * (v[n / 2 - 1] + v[n / 2]);
}

static int same_candidate(const candidate *a, const candidate *b) {
  if (a->count != b->count || a->bank != b->bank) return 0;
  for (int i = 0; i < a->count; ++i)
    if (a->chain[i] != b->chain[i]) return 0;
  for (int i = 0; i < MOFFT_MAX_PASSES; ++i)
    if (a->preferred[i] != b->preferred[i]) return 0;
  return 1;
}

static void no_preference(candidate *c) {
  for (int i = 0; i < MOFFT_MAX_PASSES; ++i) c->preferred[i] = -1;
}

/* Model score of a schedule: its predicted device seconds over `batch`
 * transforms (mofft_gpu_model.c), the prior that orders the shortlist. */
static double model_score(int precision_bits, const candidate *c, size_t length,
                          size_t batch) {
  mofft_schedule s;
  if (!mofft_group_chain_preferred(precision_bits, c->bank, c->chain, c->count,
                                   (long long)length, c->preferred, &s))
    return INFINITY;
  const double t = mofft_gpu_schedule_seconds(precision_bits, length, batch, &s);
  return t < DBL_MAX ? t : INFINITY;
}

static void add_candidate(candidate *pool, int *count, int capacity,
                          const candidate *c) {
  for (int i = 0; i < *count; ++i)
    if (same_candidate(&pool[i], c)) return;
  if (*count < capacity) pool[(*count)++] = *c;
}

static int model_compare(const void *l, const void *r) {
  const candidate *a = (const candidate *)l, *b = (const candidate *)r;
  if (a->model < b->model) return -1;
  if (a->model > b->model) return 1;
  if (a->bank != b->bank) return a->bank < b->bank ? -1 : 1;
  if (a->count != b->count) return a->count < b->count ? -1 : 1;
  for (int i = 0; i < a->count; ++i)
    if (a->chain[i] != b->chain[i]) return a->chain[i] < b->chain[i] ? -1 : 1;
  for (int i = 0; i < MOFFT_MAX_PASSES; ++i)
    if (a->preferred[i] != b->preferred[i]) return a->preferred[i] < b->preferred[i] ? -1 : 1;
  return 0;
}

static int time_compare(const void *l, const void *r) {
  const candidate *a = (const candidate *)l, *b = (const candidate *)r;
  if (a->median < b->median) return -1;
  if (a->median > b->median) return 1;
  return model_compare(l, r);
}

/* Every complete schedule the planner can express for this length. */
static int enumerate(int precision_bits, size_t length, size_t batch, candidate *pool,
                     int capacity) {
  int count = 0;
  candidate c;
  for (unsigned bank = 0; bank < MOFFT_KERNEL_BANK_COUNT; ++bank) {
    memset(&c, 0, sizeof(c));
    no_preference(&c);
    c.bank = bank;
    c.count = mofft_model_chain(precision_bits, bank, length, c.chain,
                                MOFFT_MAX_STAGES);
    if (c.count > 0) add_candidate(pool, &count, capacity, &c);
  }
  /* every specialised single-pass kernel of this length */
  const int n = mofft_cuda_kernel_count();
  for (int i = 0; i < n; ++i) {
    const mofft_kernel_desc *d = mofft_cuda_kernel_get(i);
    if (d->kind != MOFFT_KERNEL_ROWS || d->precision_bits != precision_bits ||
        (size_t)d->length != length)
      continue;
    memset(&c, 0, sizeof(c));
    no_preference(&c);
    c.preferred[0] = i;
    c.bank = 0;
    c.count = d->radix_count;
    memcpy(c.chain, d->radices, (size_t)d->radix_count * sizeof(int));
    add_candidate(pool, &count, capacity, &c);
  }
  /* two-pass splits with specialised column kernels on both sides */
  for (int i = 0; i < n; ++i) {
    const mofft_kernel_desc *a = mofft_cuda_kernel_get(i);
    if (a->kind != MOFFT_KERNEL_COLS || a->precision_bits != precision_bits ||
        length % (size_t)a->length != 0)
      continue;
    const size_t rest = length / (size_t)a->length;
    for (int j = 0; j < n; ++j) {
      const mofft_kernel_desc *b = mofft_cuda_kernel_get(j);
      if (b->kind != MOFFT_KERNEL_COLS || b->precision_bits != precision_bits ||
          (size_t)b->length != rest)
        continue;
      memset(&c, 0, sizeof(c));
      no_preference(&c);
      c.preferred[0] = i;
      c.preferred[1] = j;
      c.bank = 0;
      memcpy(c.chain, a->radices, (size_t)a->radix_count * sizeof(int));
      memcpy(c.chain + a->radix_count, b->radices,
             (size_t)b->radix_count * sizeof(int));
      c.count = a->radix_count + b->radix_count;
      mofft_schedule s;
      if (mofft_group_chain_preferred(precision_bits, 0, c.chain, c.count,
                                      (long long)length, c.preferred, &s) &&
          s.pass_count == 2 && s.pass[0].kernel == i && s.pass[1].kernel == j)
        add_candidate(pool, &count, capacity, &c);
    }
  }
  /* three-pass splits of narrow column kernels (lines of 64..512 points,
   * whose tiles span 16 or more adjacent columns): more passes, but longer
   * contiguous runs in the strided passes */
  for (int i = 0; i < n; ++i) {
    const mofft_kernel_desc *a = mofft_cuda_kernel_get(i);
    if (a->kind != MOFFT_KERNEL_COLS || a->precision_bits != precision_bits ||
        a->length < 64 || a->length > 512 || length % (size_t)a->length != 0)
      continue;
    for (int j = 0; j < n; ++j) {
      const mofft_kernel_desc *b = mofft_cuda_kernel_get(j);
      if (b->kind != MOFFT_KERNEL_COLS || b->precision_bits != precision_bits ||
          b->length < 64 || b->length > 512 ||
          (length / (size_t)a->length) % (size_t)b->length != 0)
        continue;
      const size_t rest = length / (size_t)a->length / (size_t)b->length;
      for (int k = 0; k < n; ++k) {
        const mofft_kernel_desc *d = mofft_cuda_kernel_get(k);
        if (d->kind != MOFFT_KERNEL_COLS || d->precision_bits != precision_bits ||
            d->length < 64 || d->length > 512 || (size_t)d->length != rest)
          continue;
        memset(&c, 0, sizeof(c));
        no_preference(&c);
        c.preferred[0] = i;
        c.preferred[1] = j;
        c.preferred[2] = k;
        c.bank = 0;
        memcpy(c.chain, a->radices, (size_t)a->radix_count * sizeof(int));
        memcpy(c.chain + a->radix_count, b->radices, (size_t)b->radix_count * sizeof(int));
        memcpy(c.chain + a->radix_count + b->radix_count, d->radices,
               (size_t)d->radix_count * sizeof(int));
        c.count = a->radix_count + b->radix_count + d->radix_count;
        mofft_schedule s;
        if (mofft_group_chain_preferred(precision_bits, 0, c.chain, c.count,
                                        (long long)length, c.preferred, &s) &&
            s.pass_count == 3 && s.pass[0].kernel == i && s.pass[1].kernel == j &&
            s.pass[2].kernel == k)
          add_candidate(pool, &count, capacity, &c);
      }
    }
  }
  /* the generic family with its default chain */
  memset(&c, 0, sizeof(c));
  no_preference(&c);
  c.bank = 1;
  c.count = mofft_auto_radices((long long)length, c.chain, MOFFT_MAX_STAGES);
  if (c.count > 0) add_candidate(pool, &count, capacity, &c);
  for (int i = 0; i < count; ++i)
    pool[i].model = model_score(precision_bits, &pool[i], length, batch);
  int kept = 0;
  for (int i = 0; i < count; ++i)
    if (isfinite(pool[i].model)) pool[kept++] = pool[i];
  return kept;
}

static int output_is_finite(const void *d_out, size_t bytes, int precision_bits) {
  void *host = malloc(bytes);
  if (!host) return 0;
  int ok = cudaMemcpy(host, d_out, bytes, cudaMemcpyDeviceToHost) == cudaSuccess;
  if (ok) {
    if (precision_bits == 32) {
      const float *v = (const float *)host;
      for (size_t i = 0; i < bytes / sizeof(float); ++i)
        if (!isfinite(v[i])) { ok = 0; break; }
    } else {
      const double *v = (const double *)host;
      for (size_t i = 0; i < bytes / sizeof(double); ++i)
        if (!isfinite(v[i])) { ok = 0; break; }
    }
  }
  free(host);
  return ok;
}

mofft_status mofft_search_best(mofft_core **out, int precision_bits,
                               size_t length, size_t batch, size_t distance,
                               mofft_direction direction,
                               mofft_placement placement,
                               const mofft_plan_options *options,
                               mofft_plan_diagnostics *diagnostics) {
  *out = NULL;
  if (length < 2 || !mofft_is_smooth13(length)) return MOFFT_UNSUPPORTED_SIZE;
  if (distance == 0) distance = length;
  /* Candidates are timed on at most 2^25 points (256 MiB FP32, 512 MiB
   * FP64 per buffer: larger than L2, so still HBM-bound like the real batch):
   * the planner's device memory and host input stay bounded however large
   * the plan's batch is. */
  size_t mbatch = batch;
  if (mbatch > 1 && mbatch * distance > ((size_t)1 << 25)) {
    mbatch = ((size_t)1 << 25) / distance;
    if (mbatch < 1) mbatch = 1;
  }
  enum { kPool = 256 };
  candidate *pool = (candidate *)calloc(kPool, sizeof(candidate));
  if (!pool) return MOFFT_ALLOCATION_FAILURE;
  const int pool_count = enumerate(precision_bits, length, mbatch, pool, kPool);
  if (pool_count == 0) {
    free(pool);
    return MOFFT_UNSUPPORTED_SIZE;
  }
  qsort(pool, (size_t)pool_count, sizeof(candidate), model_compare);
  /* one candidate of every bank first, then the rest in model order */
  const size_t limit = options->candidate_limit;
  candidate *sel = (candidate *)calloc(limit, sizeof(candidate));
  if (!sel) {
    free(pool);
    return MOFFT_ALLOCATION_FAILURE;
  }
  size_t nsel = 0;
  for (unsigned bank = 0; bank < MOFFT_KERNEL_BANK_COUNT && nsel < limit; ++bank)
    for (int i = 0; i < pool_count; ++i)
      if (pool[i].bank == bank) {
        sel[nsel++] = pool[i];
        break;
      }
  for (int i = 0; i < pool_count && nsel < limit; ++i) {
    int seen = 0;
    for (size_t j = 0; j < nsel; ++j)
      if (same_candidate(&sel[j], &pool[i])) { seen = 1; break; }
    if (!seen) sel[nsel++] = pool[i];
  }
  free(pool);
  /* rank of each shortlisted candidate by model seconds (1 = the model's
   * first choice), recorded before the measurement order is shuffled */
  for (size_t i = 0; i < nsel; ++i) {
    size_t rank = 1;
    for (size_t j = 0; j < nsel; ++j)
      if (sel[j].model < sel[i].model || (sel[j].model == sel[i].model && j < i)) ++rank;
    sel[i].model_rank = rank;
  }
  uint32_t shuffle = (uint32_t)length ^ ((uint32_t)precision_bits << 16) ^
                     UINT32_C(0x9e3779b9);
  for (size_t i = nsel; i > 1; --i) {
    shuffle ^= shuffle << 13;
    shuffle ^= shuffle >> 17;
    shuffle ^= shuffle << 5;
    const size_t j = (size_t)shuffle % i;
    candidate t = sel[i - 1];
    sel[i - 1] = sel[j];
    sel[j] = t;
  }

  const size_t cb = mofft_complex_bytes(precision_bits);
  const size_t bytes = mbatch * distance * cb;
  void *h_in = malloc(bytes);
  void *d_in = NULL, *d_out = NULL, *d_work = NULL;
  cudaEvent_t ev0 = NULL, ev1 = NULL;
  mofft_status status = MOFFT_SUCCESS;
  if (!h_in || cudaMalloc(&d_in, bytes) != cudaSuccess ||
      cudaMalloc(&d_out, bytes) != cudaSuccess ||
      (placement == MOFFT_IN_PLACE && cudaMalloc(&d_work, bytes) != cudaSuccess) ||
      cudaEventCreate(&ev0) != cudaSuccess || cudaEventCreate(&ev1) != cudaSuccess) {
    cudaGetLastError();
    status = MOFFT_ALLOCATION_FAILURE;
    goto done;
  }
  {
    uint32_t state = UINT32_C(0x7f4a7c15);
    for (size_t i = 0; i < bytes / cb; ++i) {
      state ^= state << 13; state ^= state >> 17; state ^= state << 5;
      const double re = ((double)(state & UINT32_C(0xffff)) / 32768.0) - 1.0;
      state ^= state << 13; state ^= state >> 17; state ^= state << 5;
      const double im = ((double)(state & UINT32_C(0xffff)) / 32768.0) - 1.0;
      if (precision_bits == 32) {
        ((float *)h_in)[2 * i] = (float)re;
        ((float *)h_in)[2 * i + 1] = (float)im;
      } else {
        ((double *)h_in)[2 * i] = re;
        ((double *)h_in)[2 * i + 1] = im;
      }
    }
    /* complete the upload before candidates launch on their own streams */
    if (cudaMemcpy(d_in, h_in, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaDeviceSynchronize() != cudaSuccess) {
      cudaGetLastError();
      status = MOFFT_INTERNAL_ERROR;
      goto done;
    }
  }
  const uint32_t samples = options->timing_samples;
  const size_t iterations = length * mbatch < 65536 ? 8 : (length * mbatch < (1u << 22) ? 4 : 2);
  for (size_t i = 0; i < nsel; ++i) {
    candidate *cand = &sel[i];
    mofft_core *c = NULL;
    status = mofft_core_create_tuned(&c, precision_bits, length, mbatch, distance,
                                     direction, placement, cand->chain, cand->count,
                                     cand->preferred);
    if (status == MOFFT_SUCCESS && cand->bank != 0) {
      c->kernel_bank = cand->bank;
      status = mofft_core_build(c);
    }
    if (status != MOFFT_SUCCESS) {
      mofft_core_destroy(c);
      goto done;
    }
    cudaStream_t s = (cudaStream_t)c->stream;
    const void *src = placement == MOFFT_IN_PLACE ? d_work : d_in;
    void *dst = placement == MOFFT_IN_PLACE ? d_work : d_out;
    if (placement == MOFFT_IN_PLACE)
      cudaMemcpyAsync(d_work, d_in, bytes, cudaMemcpyDeviceToDevice, s);
    status = mofft_core_enqueue(c, src, dst, s);
    if (status == MOFFT_SUCCESS && cudaStreamSynchronize(s) != cudaSuccess)
      status = MOFFT_INTERNAL_ERROR;
    if (status == MOFFT_SUCCESS && !output_is_finite(dst, bytes, precision_bits))
      status = MOFFT_INTERNAL_ERROR;
    for (uint32_t sample = 0; sample < samples && status == MOFFT_SUCCESS; ++sample) {
      double times[8];
      for (size_t it = 0; it < iterations && status == MOFFT_SUCCESS; ++it) {
        if (placement == MOFFT_IN_PLACE)
          cudaMemcpyAsync(d_work, d_in, bytes, cudaMemcpyDeviceToDevice, s);
        cudaEventRecord(ev0, s);
        status = mofft_core_enqueue(c, src, dst, s);
        cudaEventRecord(ev1, s);
        float ms = 0.0f;
        if (status == MOFFT_SUCCESS &&
            (cudaEventSynchronize(ev1) != cudaSuccess ||
             cudaEventElapsedTime(&ms, ev0, ev1) != cudaSuccess))
          status = MOFFT_INTERNAL_ERROR;
        times[it] = (double)ms * 1e-3;
      }
      if (status == MOFFT_SUCCESS) cand->samples[sample] = median_of(times, iterations);
    }
    if (status == MOFFT_SUCCESS && !output_is_finite(dst, bytes, precision_bits))
      status = MOFFT_INTERNAL_ERROR;
    cand->median = median_of(cand->samples, samples);
    if (status == MOFFT_SUCCESS && !isfinite(cand->median)) status = MOFFT_INTERNAL_ERROR;
    mofft_core_destroy(c);
    if (status != MOFFT_SUCCESS) {
      cudaGetLastError();
      goto done;
    }
  }
  qsort(sel, nsel, sizeof(candidate), time_compare);
  status = mofft_core_create_tuned(out, precision_bits, length, batch, distance,
                                   direction, placement, sel[0].chain, sel[0].count,
                                   sel[0].preferred);
  if (status == MOFFT_SUCCESS && sel[0].bank != 0) {
    (*out)->kernel_bank = sel[0].bank;
    status = mofft_core_build(*out);
    if (status != MOFFT_SUCCESS) {
      mofft_core_destroy(*out);
      *out = NULL;
    }
  }
  if (status == MOFFT_SUCCESS) {
    mofft_core *c = *out;
    c->measured = 1;
    c->measure_candidates = nsel;
    c->measure_winner_model_rank = sel[0].model_rank;
    c->measure_winner_seconds = sel[0].median;
    c->measure_winner_model_seconds = sel[0].model;
    c->measure_model_first_rank = 0;
    for (size_t i = 0; i < nsel; ++i)
      if (sel[i].model_rank == 1) c->measure_model_first_rank = i + 1;
  }
  if (status == MOFFT_SUCCESS && diagnostics) {
    diagnostics->measured = 1;
    diagnostics->candidates_measured = nsel;
    diagnostics->selected_median_seconds = sel[0].median;
    diagnostics->length = length;
    diagnostics->precision_bits = precision_bits;
    diagnostics->direction = direction;
    diagnostics->placement = placement;
    diagnostics->radix_count = (size_t)(*out)->depth;
    memcpy(diagnostics->radices, (*out)->factors, (size_t)(*out)->depth * sizeof(int));
    diagnostics->blocked_transpose_mask = (*out)->blocked_transpose_mask;
    diagnostics->direct_input = (*out)->direct_input;
    diagnostics->stage_layout = (*out)->stage_layout;
    diagnostics->kernel_bank = (*out)->kernel_bank;
    diagnostics->kernel_bank_count = MOFFT_KERNEL_BANK_COUNT;
  }
done:
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (d_in) cudaFree(d_in);
  if (d_out) cudaFree(d_out);
  if (d_work) cudaFree(d_work);
  free(h_in);
  free(sel);
  return status;
}
