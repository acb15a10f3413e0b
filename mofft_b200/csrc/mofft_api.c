/* MoFFT on B200: plan objects, the PRETUNED planner, device twiddle tables
 * and the execute driver.  This is the B200 counterpart of the reference's
 * runtime (src/mofft.c): the same public semantics (status codes, argument
 * validation, ownership, diagnostics), with the SME streaming-mode driver
 * replaced by a short list of CUDA kernel launches ("passes").
 *
 * Mapping of the reference's plan onto the GPU schedule:
 *  - The reference's radix chain (factors[0] outermost ... factors[d-1]
 *    innermost, src/mofft.c:353-417) is kept as the plan's public identity.
 *    Its innermost radix is applied first (src/mofft.c:1936-1943), which is
 *    exactly the first stage of a Stockham autosort transform, so the GPU
 *    stage list is the chain reversed.
 *  - Consecutive stages are grouped into passes: one pass when the length fits
 *    one CTA's shared memory, otherwise a four-step / six-step split in which
 *    each pass is one kernel.  The grouping is canonical (fewest passes, then
 *    specialised kernels, then balance), so a recipe's radix chain reproduces
 *    the same schedule on import.
 *  - Twiddles are computed in extended precision from an exact reduction of
 *    the angle fraction and rounded once to the plan precision
 *    (src/mofft.c:1082-1140 computes them in double); they live on the device
 *    for the plan's lifetime.
 */
#define _GNU_SOURCE
#include <cuda_runtime_api.h>
#include <errno.h>
#include <float.h>
#include <math.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mofft_internal.h"
#include "mofft_host.h"

/* ------------------------------------------------------------------------ */
/* small helpers                                                             */
/* ------------------------------------------------------------------------ */

static const int k_ref_radices[] = {64, 32, 16, 15, 14, 13, 12, 11, 10,
                                    9,  8,  7,  6,  5,  4,  3,  2};

static atomic_ullong g_launches = 0;

int mofft_is_supported_radix(int radix) {
  for (size_t i = 0; i < sizeof(k_ref_radices) / sizeof(k_ref_radices[0]); ++i)
    if (k_ref_radices[i] == radix) return 1;
  return 0;
}

int mofft_is_smooth13(size_t n) {
  if (n < 2) return 0;
  static const int primes[] = {2, 3, 5, 7, 11, 13};
  for (size_t i = 0; i < 6; ++i)
    while (n % (size_t)primes[i] == 0) n /= (size_t)primes[i];
  return n == 1;
}

double mofft_monotonic_seconds(void) {
  struct timespec now;
  if (clock_gettime(CLOCK_MONOTONIC, &now) != 0) return -1.0;
  return (double)now.tv_sec + (double)now.tv_nsec * 1e-9;
}

size_t mofft_complex_bytes(int precision_bits) {
  return precision_bits == 32 ? 8u : 16u;
}

/* ------------------------------------------------------------------------ */
/* hardware probe (the analogue of mofft_hardware_supports, src/mofft.c:96) */
/* ------------------------------------------------------------------------ */

static atomic_int g_hw_support = -1;

int mofft_hardware_supports(int precision_bits) {
  (void)precision_bits; /* B200 runs FP32 and FP64 natively */
  int cached = atomic_load(&g_hw_support);
  if (cached >= 0) return cached;
  int count = 0;
  int supported = 0;
  if (cudaGetDeviceCount(&count) == cudaSuccess && count > 0) {
    int device = 0;
    struct cudaDeviceProp prop;
    if (cudaGetDevice(&device) == cudaSuccess &&
        cudaGetDeviceProperties(&prop, device) == cudaSuccess)
      supported = prop.major == 10 && prop.minor == 0; /* sm_100 */
  } else {
    cudaGetLastError();
  }
  int expected = -1;
  atomic_compare_exchange_strong(&g_hw_support, &expected, supported);
  return atomic_load(&g_hw_support);
}

/* GPU family word of recipes: compute capability and SM count. */
int mofft_device_family(uint32_t *family) {
  int device = 0;
  struct cudaDeviceProp prop;
  if (cudaGetDevice(&device) != cudaSuccess ||
      cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  *family = ((uint32_t)prop.major << 24) | ((uint32_t)prop.minor << 16) |
            ((uint32_t)prop.multiProcessorCount & 0xffffu);
  return 1;
}

/* Per-device one-time kernel attribute setup. */
static atomic_int g_prepared[64];

static int prepare_current_device(void) {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return 0;
  if (device < 0 || device >= 64) return 0;
  if (atomic_load(&g_prepared[device]) == 1) return 1;
  if (mofft_cuda_prepare_device() != 0) return 0;
  atomic_store(&g_prepared[device], 1);
  return 1;
}

/* ------------------------------------------------------------------------ */
/* twiddles: exp(-2*pi*i*num/den) with exact octant reduction               */
/* ------------------------------------------------------------------------ */

void mofft_cis_turns(uint64_t num, uint64_t den, long double *c,
                     long double *s) {
  /* angle = 2*pi*num/den, returned as cos(angle), sin(angle) */
  num %= den;
  const unsigned __int128 eight = (unsigned __int128)num * 8u;
  uint64_t octant = (uint64_t)(eight / den);
  uint64_t rest = (uint64_t)(eight - (unsigned __int128)octant * den);
  int mirror = (int)(octant & 1u);
  if (mirror) rest = den - rest;
  const long double quarter_pi = 0.785398163397448309615660845819875721L;
  const long double x = quarter_pi * ((long double)rest / (long double)den);
  long double sx = sinl(x), cx = cosl(x);
  if (mirror) {
    long double t = sx;
    sx = cx;
    cx = t;
  }
  switch ((octant / 2u) & 3u) {
    case 0: *c = cx; *s = sx; break;
    case 1: *c = -sx; *s = cx; break;
    case 2: *c = -cx; *s = -sx; break;
    default: *c = sx; *s = -cx; break;
  }
}

/* Writes count forward twiddles W_den^(e) = exp(-2 pi i e/den) for
 * e = first + k*step into dst (precision_bits wide complex). */
void mofft_write_twiddles(void *dst, int precision_bits, uint64_t den,
                          uint64_t first, uint64_t step, size_t count) {
  for (size_t k = 0; k < count; ++k) {
    long double c, s;
    mofft_cis_turns((first + (uint64_t)k * step) % den, den, &c, &s);
    if (precision_bits == 32) {
      ((float *)dst)[2 * k] = (float)c;
      ((float *)dst)[2 * k + 1] = (float)-s;
    } else {
      ((double *)dst)[2 * k] = (double)c;
      ((double *)dst)[2 * k + 1] = (double)-s;
    }
  }
}

/* Internal stage table of an in-CTA chain: stage (R, Ns>1) stores
 * W_{Ns*R}^{jm*r} at (r-1)*Ns + jm. */
size_t mofft_stage_table_entries(const int *radices, int count) {
  size_t total = 0, ns = 1;
  for (int i = 0; i < count; ++i) {
    if (ns > 1) total += (size_t)(radices[i] - 1) * ns;
    ns *= (size_t)radices[i];
  }
  return total;
}

void mofft_fill_stage_table(void *dst, int precision_bits, const int *radices,
                            int count) {
  const size_t cb = mofft_complex_bytes(precision_bits);
  unsigned char *p = (unsigned char *)dst;
  size_t ns = 1;
  for (int i = 0; i < count; ++i) {
    const size_t R = (size_t)radices[i];
    if (ns > 1) {
      for (size_t r = 1; r < R; ++r) {
        mofft_write_twiddles(p, precision_bits, ns * R, 0, r, ns);
        p += ns * cb;
      }
    }
    ns *= R;
  }
}

int mofft_ceil_log2_u64(uint64_t x) {
  int s = 0;
  while (((uint64_t)1 << s) < x) ++s;
  return s;
}

/* ------------------------------------------------------------------------ */
/* kernel selection and canonical pass grouping                              */
/* ------------------------------------------------------------------------ */

#define SMEM_LIMIT (227u * 1024u)

/* Generic (runtime stage list) kernel that can run every radix of `chain`:
 * the narrow variant (radix <= 16) when possible, else the wide one. */
/* Runtime-stage kernel of kernel bank `bank` (its codelet family) whose
 * largest radix covers the chain: the narrow variant when it suffices. */
static int generic_kernel_index(int precision_bits, unsigned bank, const int *chain,
                                int count) {
  int max_radix = 0;
  for (int i = 0; i < count; ++i)
    if (chain[i] > max_radix) max_radix = chain[i];
  int best = -1, best_cap = 1 << 30;
  const int n = mofft_cuda_kernel_count();
  for (int i = 0; i < n; ++i) {
    const mofft_kernel_desc *d = mofft_cuda_kernel_get(i);
    if (d->kind != MOFFT_KERNEL_GENERIC || d->precision_bits != precision_bits ||
        d->bank != (int)bank)
      continue;
    const int cap = d->radices[0];
    if (cap >= max_radix && cap < best_cap) {
      best = i;
      best_cap = cap;
    }
  }
  return best;
}

static int chain_equal(const int *a, int na, const int *b, int nb) {
  if (na != nb) return 0;
  for (int i = 0; i < na; ++i)
    if (a[i] != b[i]) return 0;
  return 1;
}

/* Specialised kernel whose in-CTA chain equals `chain`.  The thread-block
 * cluster kernels are never found here: they run when a tuned or explicit
 * kernel list names them (MEASURE times them against the others). */
static int find_special(int precision_bits, int kind, const int *chain,
                        int count, long long total, long long ns_outer) {
  long long length = 1;
  for (int i = 0; i < count; ++i) length *= chain[i];
  const int n = mofft_cuda_kernel_count();
  for (int i = 0; i < n; ++i) {
    const mofft_kernel_desc *d = mofft_cuda_kernel_get(i);
    if (d->kind != kind || d->precision_bits != precision_bits ||
        d->length != length || d->cluster > 0 ||
        !chain_equal(d->radices, d->radix_count, chain, count))
      continue;
    if (kind == MOFFT_KERNEL_COLS) {
      const long long lines_total = total / length;
      if (lines_total % d->lines != 0) continue;
      if (ns_outer != 1 && ns_outer % d->lines != 0) continue;
    }
    return i;
  }
  return -1;
}

static long long gcd_ll(long long a, long long b) {
  while (b) {
    long long t = a % b;
    a = b;
    b = t;
  }
  return a;
}

static int generic_rows_lines(int precision_bits, int length) {
  int lines = length >= 1024 ? 1 : 1024 / length;
  while (lines > 1 &&
         mofft_cuda_generic_smem(precision_bits, length, lines, 0) > SMEM_LIMIT)
    lines /= 2;
  return mofft_cuda_generic_smem(precision_bits, length, lines, 0) <= SMEM_LIMIT
             ? lines : 0;
}

static int generic_cols_lines(int precision_bits, int length, long long total,
                              long long ns_outer) {
  long long g = total / length;
  if (ns_outer > 1) g = gcd_ll(g, ns_outer);
  for (int lines = 16; lines >= 1; --lines) {
    if (g % lines != 0) continue;
    if (mofft_cuda_generic_smem(precision_bits, length, lines, 1) <= SMEM_LIMIT)
      return lines;
  }
  return 0;
}

typedef struct {
  int passes;
  int generic;
  double imbalance;
} group_score;

static int score_less(const group_score *a, const group_score *b) {
  if (a->passes != b->passes) return a->passes < b->passes;
  if (a->generic != b->generic) return a->generic < b->generic;
  return a->imbalance < b->imbalance - 1e-9;
}

/* Fill one pass for stages [begin, end) of `chain`.  Returns 1 if some kernel
 * can run it (specialised when allowed, else generic). */
static int kernel_fits(int k, int precision_bits, int kind, const int *chain,
                       int count, long long total, long long ns_outer) {
  const mofft_kernel_desc *d = mofft_cuda_kernel_get(k);
  if (!d || d->kind != kind || d->precision_bits != precision_bits ||
      !chain_equal(d->radices, d->radix_count, chain, count))
    return 0;
  if (kind == MOFFT_KERNEL_COLS) {
    if ((total / d->length) % d->lines != 0) return 0;
    if (ns_outer != 1 && ns_outer % d->lines != 0) return 0;
  }
  return 1;
}

static int make_pass(int precision_bits, unsigned bank, const int *chain,
                     int begin, int end, long long total, long long ns_outer,
                     int single, const int *preferred, mofft_pass *out) {
  const int count = end - begin;
  if (count < 1 || count > MOFFT_CUDA_MAX_STAGES) return 0;
  long long length = 1;
  for (int i = begin; i < end; ++i) length *= chain[i];
  if (length > (1 << 24)) return 0;
  memset(out, 0, sizeof(*out));
  out->length = (int)length;
  out->radix_count = count;
  memcpy(out->radices, chain + begin, (size_t)count * sizeof(int));
  out->ns_outer = ns_outer;
  const int kind = single ? MOFFT_KERNEL_ROWS : MOFFT_KERNEL_COLS;
  if (bank == 0 && count <= 8) {
    int k = -1;
    for (int i = 0; preferred && i < MOFFT_MAX_PASSES && k < 0; ++i)
      if (preferred[i] >= 0 &&
          kernel_fits(preferred[i], precision_bits, kind, chain + begin, count, total,
                      ns_outer))
        k = preferred[i];
    if (k < 0)
      k = find_special(precision_bits, kind, chain + begin, count, total, ns_outer);
    if (k >= 0) {
      const mofft_kernel_desc *d = mofft_cuda_kernel_get(k);
      out->kernel = k;
      out->kind = kind;
      out->lines = d->lines;
      out->smem_bytes = d->smem_bytes;
      return 1;
    }
  }
  const int g = generic_kernel_index(precision_bits, bank, chain + begin, count);
  if (g < 0) return 0;
  int lines = single ? generic_rows_lines(precision_bits, (int)length)
                     : generic_cols_lines(precision_bits, (int)length, total,
                                          ns_outer);
  if (lines <= 0) return 0;
  out->kernel = g;
  out->kind = MOFFT_KERNEL_GENERIC;
  out->lines = lines;
  out->smem_bytes = mofft_cuda_generic_smem(precision_bits, (int)length, lines,
                                            single ? 0 : 1);
  return 1;
}

/* Evaluate the split of `chain` at the given boundaries. */
static int try_split(int precision_bits, unsigned bank, const int *chain,
                     int count, const int *cuts, int passes, long long total,
                     const int *preferred, mofft_schedule *sched,
                     group_score *score) {
  long long ns = 1;
  double lo = 1e300, hi = 0;
  int generic = 0;
  for (int p = 0; p < passes; ++p) {
    const int begin = p == 0 ? 0 : cuts[p - 1];
    const int end = p == passes - 1 ? count : cuts[p];
    if (!make_pass(precision_bits, bank, chain, begin, end, total, ns,
                   passes == 1, preferred, &sched->pass[p]))
      return 0;
    if (sched->pass[p].kind == MOFFT_KERNEL_GENERIC) ++generic;
    const double l = log2((double)sched->pass[p].length);
    if (l < lo) lo = l;
    if (l > hi) hi = l;
    ns *= sched->pass[p].length;
  }
  sched->pass_count = passes;
  score->passes = passes;
  score->generic = generic;
  score->imbalance = hi - lo;
  return 1;
}

/* Canonical grouping of a Stockham stage chain into passes. */
int mofft_group_chain_preferred(int precision_bits, unsigned bank,
                                const int *chain, int count, long long total,
                                const int *preferred, mofft_schedule *best) {
  group_score best_score = {1 << 30, 1 << 30, 1e300};
  int found = 0;
  mofft_schedule cand;
  group_score score;
  /* A tuned list of two or more kernels fixes the pass count and each pass's
   * kernel (the autotuner measured that schedule, e.g. three narrow passes
   * where two wide ones exist); without a matching split, group canonically. */
  int npref = 0;
  while (preferred && npref < MOFFT_MAX_PASSES && preferred[npref] >= 0) ++npref;
  if (npref >= 2 && npref <= count) {
    int cuts[MOFFT_MAX_PASSES];
    for (int i = 0; i < npref - 1; ++i) cuts[i] = i + 1;
    for (;;) {
      if (try_split(precision_bits, bank, chain, count, cuts, npref, total,
                    preferred, &cand, &score)) {
        int match = 1;
        for (int p = 0; p < npref; ++p)
          if (cand.pass[p].kernel != preferred[p]) match = 0;
        if (match) {
          *best = cand;
          return 1;
        }
      }
      int i = npref - 2;
      while (i >= 0 && cuts[i] == count - (npref - 1 - i)) --i;
      if (i < 0) break;
      ++cuts[i];
      for (int k = i + 1; k < npref - 1; ++k) cuts[k] = cuts[k - 1] + 1;
    }
  }
  for (int passes = 1; passes <= MOFFT_MAX_PASSES && passes <= count; ++passes) {
    int cuts[MOFFT_MAX_PASSES];
    /* enumerate increasing cut positions in [1, count-1] */
    for (int i = 0; i < passes - 1; ++i) cuts[i] = i + 1;
    for (;;) {
      if (try_split(precision_bits, bank, chain, count, cuts, passes, total,
                    preferred, &cand, &score) &&
          (!found || score_less(&score, &best_score))) {
        *best = cand;
        best_score = score;
        found = 1;
      }
      /* next combination */
      int i = passes - 2;
      while (i >= 0 && cuts[i] == count - (passes - 1 - i)) --i;
      if (i < 0) break;
      ++cuts[i];
      for (int k = i + 1; k < passes - 1; ++k) cuts[k] = cuts[k - 1] + 1;
    }
    if (found) break;
  }
  return found;
}

int mofft_group_chain(int precision_bits, unsigned bank, const int *chain,
                      int count, long long total, mofft_schedule *best) {
  return mofft_group_chain_preferred(precision_bits, bank, chain, count, total,
                                     NULL, best);
}

/* Default in-CTA radix chain for a runtime-stage (generic) line of length L. */
int mofft_auto_radices(long long length, int *out, int capacity) {
  int count = 0;
  long long n = length;
  static const int pref[] = {16, 8, 4, 2};
  static const int odd[] = {13, 11, 9, 7, 5, 3};
  for (size_t i = 0; i < sizeof(odd) / sizeof(odd[0]); ++i)
    while (n % odd[i] == 0) {
      if (count >= capacity) return -1;
      out[count++] = odd[i];
      n /= odd[i];
    }
  for (size_t i = 0; i < sizeof(pref) / sizeof(pref[0]); ++i)
    while (n % pref[i] == 0) {
      if (count >= capacity) return -1;
      out[count++] = pref[i];
      n /= pref[i];
    }
  return n == 1 ? count : -1;
}

/* Preferred chain of a pass of length L: the first registered specialised
 * kernel of that kind and length, else the generic default chain. */
static int preferred_chain(int precision_bits, unsigned bank, int kind,
                           long long length, long long total,
                           long long ns_outer, int *out, int capacity) {
  if (bank == 0) {
    const int n = mofft_cuda_kernel_count();
    for (int i = 0; i < n; ++i) {
      const mofft_kernel_desc *d = mofft_cuda_kernel_get(i);
      if (d->kind != kind || d->precision_bits != precision_bits ||
          d->length != length || d->radix_count > capacity || d->cluster > 0)
        continue;
      if (kind == MOFFT_KERNEL_COLS) {
        if ((total / length) % d->lines != 0) continue;
        if (ns_outer != 1 && ns_outer % d->lines != 0) continue;
      }
      memcpy(out, d->radices, (size_t)d->radix_count * sizeof(int));
      return d->radix_count;
    }
  }
  return mofft_auto_radices(length, out, capacity);
}

static void collect_divisors(long long n, long long lo, long long hi,
                             long long *out, int *count, int capacity) {
  *count = 0;
  for (long long d = 1; d * d <= n; ++d) {
    if (n % d) continue;
    long long pair[2] = {d, n / d};
    for (int k = 0; k < (d * d == n ? 1 : 2); ++k)
      if (pair[k] >= lo && pair[k] <= hi && *count < capacity)
        out[(*count)++] = pair[k];
  }
}

static int model_chain(int precision_bits, unsigned bank, size_t length, int *chain,
                       int capacity, int one_pass);

/* Analytical PRETUNED chain for a whole transform of `length`. */
int mofft_model_chain(int precision_bits, unsigned bank, size_t length,
                      int *chain, int capacity) {
  return model_chain(precision_bits, bank, length, chain, capacity, 1);
}

/* The best chain of two or more passes (callers that need the intermediate
 * array of a multi-pass schedule even where one pass exists). */
int mofft_model_chain_multipass(int precision_bits, unsigned bank, size_t length,
                                int *chain, int capacity) {
  return model_chain(precision_bits, bank, length, chain, capacity, 0);
}

static int model_chain(int precision_bits, unsigned bank, size_t length, int *chain,
                       int capacity, int one_pass) {
  mofft_schedule sched;
  /* one pass */
  int count = one_pass ? preferred_chain(precision_bits, bank, MOFFT_KERNEL_ROWS,
                                         (long long)length, (long long)length, 1, chain,
                                         capacity)
                       : 0;
  if (count > 0 && mofft_group_chain(precision_bits, bank, chain, count,
                                     (long long)length, &sched) &&
      sched.pass_count == 1)
    return count;
  /* multi-pass: best balanced split whose passes have kernels */
  enum { kMaxDiv = 4096 };
  static __thread long long divs[kMaxDiv];
  int ndiv = 0;
  const long long n = (long long)length;
  collect_divisors(n, 2, 1 << 16, divs, &ndiv, kMaxDiv);
  int best_count = -1;
  group_score best = {1 << 30, 1 << 30, 1e300};
  double best_seconds = 1e300;
  /* Splits of the fewest passes are ranked by the device-time model
   * (mofft_gpu_model.c) over a batch of about 2^25 points, the choice the
   * reference's choose_factorization makes with its cost model
   * (src/mofft.c:327-351); a split the model cannot price ranks by the
   * canonical grouping score. */
  const size_t model_batch = n >= (1LL << 25) ? 1 : (size_t)((1LL << 25) / n);
  int tmp[MOFFT_MAX_STAGES];
  for (int passes = 2; passes <= 3 && best_count < 0; ++passes) {
    for (int a = 0; a < ndiv; ++a) {
      for (int b = 0; b < (passes == 3 ? ndiv : 1); ++b) {
        long long L[3];
        L[0] = divs[a];
        if (passes == 2) {
          L[1] = n / L[0];
        } else {
          L[1] = divs[b];
          if ((n / L[0]) % L[1] != 0) continue;
          L[2] = n / L[0] / L[1];
        }
        int total_count = 0;
        long long ns = 1;
        int ok = 1;
        int cuts[MOFFT_MAX_PASSES];
        for (int p = 0; p < passes && ok; ++p) {
          if (L[p] < 2 || L[p] > (1 << 16)) { ok = 0; break; }
          const int c = preferred_chain(precision_bits, bank, MOFFT_KERNEL_COLS,
                                        L[p], n, ns, tmp + total_count,
                                        MOFFT_MAX_STAGES - total_count);
          if (c <= 0) { ok = 0; break; }
          total_count += c;
          if (p < passes - 1) cuts[p] = total_count;
          ns *= L[p];
        }
        if (!ok) continue;
        group_score score;
        if (!try_split(precision_bits, bank, tmp, total_count, cuts, passes, n,
                       NULL, &sched, &score))
          continue;
        const double seconds =
            mofft_gpu_schedule_seconds(precision_bits, (size_t)n, model_batch, &sched);
        int better;
        if (best_count < 0 || score.passes != best.passes)
          better = best_count < 0 || score.passes < best.passes;
        else if (seconds < 1e300 && best_seconds < 1e300 &&
                 fabs(seconds - best_seconds) > 1e-3 * best_seconds)
          better = seconds < best_seconds;
        else
          better = score_less(&score, &best);
        if (better) {
          best = score;
          best_seconds = seconds;
          best_count = total_count;
          memcpy(chain, tmp, (size_t)total_count * sizeof(int));
        }
      }
    }
  }
  return best_count;
}

/* ------------------------------------------------------------------------ */
/* plan lifecycle                                                            */
/* ------------------------------------------------------------------------ */

static void release_device(mofft_core *c) {
  if (c->d_twiddles) cudaFree(c->d_twiddles);
  if (c->d_work) cudaFree(c->d_work);
  if (c->d_stage[0]) cudaFree(c->d_stage[0]);
  if (c->d_stage[1]) cudaFree(c->d_stage[1]);
  c->d_twiddles = c->d_work = c->d_stage[0] = c->d_stage[1] = NULL;
  c->twiddle_bytes = c->work_bytes = c->stage_bytes = 0;
}

void mofft_core_destroy(mofft_core *c) {
  if (!c) return;
  int saved = -1;
  cudaGetDevice(&saved);
  if (saved != c->device) cudaSetDevice(c->device);
  release_device(c);
  if (c->stream) cudaStreamDestroy((cudaStream_t)c->stream);
  if (c->stream2) cudaStreamDestroy((cudaStream_t)c->stream2);
  if (c->stream3) cudaStreamDestroy((cudaStream_t)c->stream3);
  for (int i = 0; i < 64; ++i) {
    if (c->ev_up[i]) cudaEventDestroy((cudaEvent_t)c->ev_up[i]);
    if (c->ev_done[i]) cudaEventDestroy((cudaEvent_t)c->ev_done[i]);
  }
  if (saved >= 0 && saved != c->device) cudaSetDevice(saved);
  pthread_mutex_destroy(&c->lock);
  free(c);
}

static size_t align256(size_t x) { return (x + 255u) & ~(size_t)255u; }

static int is_tensor_kind(int kind) {
  return kind == MOFFT_KERNEL_TENSOR || kind == MOFFT_KERNEL_TENSOR_COLS;
}

/* Passes that read a constant table next to their twiddles: the tensor-core
 * kernels (operand tiles) and every kernel that carries a table of its own
 * (the radix-64 tensor-core kernel, the cluster kernels). */
static int pass_has_aux(const mofft_pass *ps) {
  return is_tensor_kind(ps->kind) || mofft_cuda_kernel_aux_bytes(ps->kernel) > 0;
}

/* Passes whose kernel reports bounded-wait timeouts in an error word: the
 * tensor-core kernels, the prefetching ROWS kernels and the cluster kernels
 * (their wait for the exchanged tiles). */
static int pass_has_status(const mofft_pass *ps) {
  if (is_tensor_kind(ps->kind)) return 1;
  const mofft_kernel_desc *d = mofft_cuda_kernel_get(ps->kernel);
  return ps->kind == MOFFT_KERNEL_ROWS && d && (d->prefetch || d->cluster > 0);
}

static int schedule_has_status(const mofft_core *c) {
  for (int p = 0; p < c->sched.pass_count; ++p)
    if (pass_has_status(&c->sched.pass[p])) return 1;
  return 0;
}

/* Build device state (twiddles, workspace) for c->sched. */
static mofft_status materialise_schedule(mofft_core *c) {
  const size_t cb = mofft_complex_bytes(c->precision_bits);
  size_t bytes = 0;
  for (int p = 0; p < c->sched.pass_count; ++p) {
    mofft_pass *ps = &c->sched.pass[p];
    ps->tw_offset = bytes;
    bytes = align256(bytes + mofft_stage_table_entries(ps->radices, ps->radix_count) * cb + cb);
    ps->split_shift = 0;
    ps->tw_hi_offset = ps->tw_lo_offset = bytes;
    if (ps->ns_outer > 1) {
      const uint64_t m = (uint64_t)ps->ns_outer * (uint64_t)ps->length;
      const int shift = (mofft_ceil_log2_u64(m) + 1) / 2;
      ps->split_shift = shift;
      const size_t lo_n = (size_t)1 << shift;
      const size_t hi_n = (size_t)((m + lo_n - 1) >> shift);
      ps->tw_hi_offset = bytes;
      bytes = align256(bytes + hi_n * cb);
      ps->tw_lo_offset = bytes;
      bytes = align256(bytes + lo_n * cb);
    }
    ps->aux_offset = ps->status_offset = 0;
    if (pass_has_aux(ps)) {
      ps->aux_offset = bytes;
      const size_t own = mofft_cuda_kernel_aux_bytes(ps->kernel);
      bytes = align256(bytes + (own ? own
                                    : mofft_cuda_tensor_aux_bytes(
                                          mofft_cuda_kernel_get(ps->kernel)->form)));
    }
    if (pass_has_status(ps)) {
      ps->status_offset = bytes;
      bytes = align256(bytes + sizeof(int));
    }
  }
  if (bytes == 0) bytes = 256;
  unsigned char *host = (unsigned char *)calloc(1, bytes);
  if (!host) return MOFFT_ALLOCATION_FAILURE;
  for (int p = 0; p < c->sched.pass_count; ++p) {
    const mofft_pass *ps = &c->sched.pass[p];
    mofft_fill_stage_table(host + ps->tw_offset, c->precision_bits, ps->radices,
                     ps->radix_count);
    if (ps->ns_outer > 1) {
      const uint64_t m = (uint64_t)ps->ns_outer * (uint64_t)ps->length;
      const size_t lo_n = (size_t)1 << ps->split_shift;
      const size_t hi_n = (size_t)((m + lo_n - 1) >> ps->split_shift);
      mofft_write_twiddles(host + ps->tw_hi_offset, c->precision_bits, m, 0, lo_n, hi_n);
      mofft_write_twiddles(host + ps->tw_lo_offset, c->precision_bits, m, 0, 1, lo_n);
    }
    if (mofft_cuda_kernel_aux_bytes(ps->kernel)) {
      if (mofft_cuda_kernel_fill_aux(ps->kernel, host + ps->aux_offset) != 0) {
        free(host);
        return MOFFT_INTERNAL_ERROR;
      }
    } else if (is_tensor_kind(ps->kind)) {
      double fr[256], fi[256];
      for (int k = 0; k < 16; ++k)
        for (int r = 0; r < 16; ++r) {
          long double cr, si;
          mofft_cis_turns((uint64_t)((k * r) % 16), 16, &cr, &si);
          fr[k * 16 + r] = (double)cr;
          fi[k * 16 + r] = -(double)si; /* forward sign */
        }
      if (mofft_cuda_tensor_fill_aux(mofft_cuda_kernel_get(ps->kernel)->form,
                                     host + ps->aux_offset, fr, fi) != 0) {
        free(host);
        return MOFFT_INTERNAL_ERROR;
      }
    }
  }
  release_device(c);
  if (cudaMalloc(&c->d_twiddles, bytes) != cudaSuccess) {
    cudaGetLastError();
    free(host);
    return MOFFT_ALLOCATION_FAILURE;
  }
  c->twiddle_bytes = bytes;
  /* A cudaMemcpy from pageable memory may return before its DMA has landed,
   * and plans run on non-blocking streams: copy on the plan's stream and
   * wait for it, so the tables are complete before any later launch. */
  if (cudaMemcpyAsync(c->d_twiddles, host, bytes, cudaMemcpyHostToDevice,
                      (cudaStream_t)c->stream) != cudaSuccess ||
      cudaStreamSynchronize((cudaStream_t)c->stream) != cudaSuccess) {
    cudaGetLastError();
    free(host);
    return MOFFT_INTERNAL_ERROR;
  }
  free(host);
  const int P = c->sched.pass_count;
  const int need_work = P >= 3 || (P == 2 && c->placement == MOFFT_IN_PLACE);
  if (need_work) {
    const size_t work = c->batch * c->length * cb;
    if (cudaMalloc(&c->d_work, work) != cudaSuccess) {
      cudaGetLastError();
      return MOFFT_ALLOCATION_FAILURE;
    }
    c->work_bytes = work;
  }
  return MOFFT_SUCCESS;
}

/* Set c->factors/depth (reference order) from a Stockham chain. */
static void set_factors_from_chain(mofft_core *c, const int *chain, int count) {
  c->depth = count;
  for (int i = 0; i < count; ++i) c->factors[i] = chain[count - 1 - i];
}

static int chain_from_factors(const mofft_core *c, int *chain) {
  for (int i = 0; i < c->depth; ++i) chain[i] = c->factors[c->depth - 1 - i];
  return c->depth;
}

static int tensor_kernel_index(int kind, int form) {
  const int n = mofft_cuda_kernel_count();
  for (int i = 0; i < n; ++i) {
    const mofft_kernel_desc *d = mofft_cuda_kernel_get(i);
    if (d->kind == kind && d->form == form) return i;
  }
  return -1;
}

/* Schedule of the tensor-core kernels of c->form: one pass of the whole-
 * transform kernel when it has c->length, else two passes of the column
 * kernel when c->length is the square of its line length. */
static mofft_status build_tensor_schedule(mofft_core *c) {
  mofft_schedule sched;
  memset(&sched, 0, sizeof(sched));
  int k = tensor_kernel_index(MOFFT_KERNEL_TENSOR, c->form);
  const mofft_kernel_desc *d = k >= 0 ? mofft_cuda_kernel_get(k) : NULL;
  int passes = 0, kind = MOFFT_KERNEL_TENSOR;
  if (d && c->precision_bits == d->precision_bits && c->length == (size_t)d->length) {
    passes = 1;
  } else {
    k = tensor_kernel_index(MOFFT_KERNEL_TENSOR_COLS, c->form);
    d = k >= 0 ? mofft_cuda_kernel_get(k) : NULL;
    if (d && c->precision_bits == d->precision_bits &&
        c->length == (size_t)d->length * (size_t)d->length) {
      passes = 2;
      kind = MOFFT_KERNEL_TENSOR_COLS;
    }
  }
  if (passes == 0) return MOFFT_UNSUPPORTED_SIZE;
  sched.pass_count = passes;
  long long ns = 1;
  for (int p = 0; p < passes; ++p) {
    mofft_pass *ps = &sched.pass[p];
    ps->kernel = k;
    ps->kind = kind;
    ps->length = d->length;
    ps->lines = d->lines;
    ps->radix_count = d->radix_count;
    memcpy(ps->radices, d->radices, (size_t)d->radix_count * sizeof(int));
    ps->ns_outer = ns;
    ps->smem_bytes = d->smem_bytes;
    ns *= d->length;
  }
  c->sched = sched;
  return materialise_schedule(c);
}

/* Failure check of a one-pass plan whose kernel bulk-copies its input (the
 * tensor-core kernel, a prefetching ROWS kernel): one forward launch whose
 * first input copy per CTA is never issued, so every CTA's bounded wait runs
 * out.  Returns the status the plan then reports (MOFFT_INTERNAL_ERROR when
 * the timeout path works) and clears the error word, so the plan stays
 * usable.  The ROWS kernel loads the line itself after the timeout, so its
 * output is still the forward transform. */
mofft_status mofft_core_check_lost_copy(mofft_core *c, const void *in, void *out) {
  if (c->sched.pass_count != 1 || c->sched.pass[0].kind == MOFFT_KERNEL_TENSOR_COLS ||
      !pass_has_status(&c->sched.pass[0]))
    return MOFFT_INVALID_ARGUMENT;
  const mofft_pass *ps = &c->sched.pass[0];
  mofft_pass_args a;
  memset(&a, 0, sizeof(a));
  a.in = in;
  a.out = out;
  a.tw = (const unsigned char *)c->d_twiddles + ps->tw_offset;
  if (pass_has_aux(ps)) a.aux = (const unsigned char *)c->d_twiddles + ps->aux_offset;
  a.status = (int *)((unsigned char *)c->d_twiddles + ps->status_offset);
  a.batch = (long long)c->batch;
  a.in_dist = (long long)c->distance;
  a.out_dist = (long long)c->distance;
  a.total = (long long)c->length;
  a.ns_outer = 1;
  a.length = ps->length;
  a.lose_copy = 1;
  cudaStream_t s = (cudaStream_t)c->stream;
  if (mofft_cuda_launch_pass(ps->kernel, &a, s) != 0 || cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return MOFFT_INTERNAL_ERROR;
  }
  atomic_fetch_add(&g_launches, 1);
  const mofft_status observed = mofft_core_check_status(c);
  if (cudaMemsetAsync(a.status, 0, sizeof(int), s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return MOFFT_INTERNAL_ERROR;
  }
  return observed;
}

mofft_status mofft_core_check_status(const mofft_core *c) {
  for (int p = 0; p < c->sched.pass_count; ++p) {
    const mofft_pass *ps = &c->sched.pass[p];
    if (!pass_has_status(ps)) continue;
    int word = 0;
    if (cudaMemcpy(&word, (const unsigned char *)c->d_twiddles + ps->status_offset,
                   sizeof(word), cudaMemcpyDeviceToHost) != cudaSuccess) {
      cudaGetLastError();
      return MOFFT_INTERNAL_ERROR;
    }
    if (word != 0) return MOFFT_INTERNAL_ERROR;
  }
  return MOFFT_SUCCESS;
}

/* (Re)build the GPU schedule from c->factors, c->kernel_bank and c->form. */
mofft_status mofft_core_build(mofft_core *c) {
  if (c->form != 0) return build_tensor_schedule(c);
  int chain[MOFFT_MAX_STAGES];
  const int count = chain_from_factors(c, chain);
  mofft_schedule sched;
  if (!mofft_group_chain_preferred(c->precision_bits, c->kernel_bank, chain, count,
                                   (long long)c->length, c->preferred, &sched))
    return MOFFT_UNSUPPORTED_SIZE;
  c->sched = sched;
  return materialise_schedule(c);
}

/* Allocate a core with validated shape; chain==NULL selects the model. */
mofft_status mofft_core_create(mofft_core **out, int precision_bits,
                               size_t length, size_t batch, size_t distance,
                               mofft_direction direction,
                               mofft_placement placement, const int *chain,
                               int chain_count) {
  return mofft_core_create_tuned(out, precision_bits, length, batch, distance,
                                 direction, placement, chain, chain_count, NULL);
}

mofft_status mofft_core_create_pretuned(mofft_core **out, int precision_bits, size_t length,
                                        size_t batch, size_t distance,
                                        mofft_direction direction, mofft_placement placement) {
  int chain[MOFFT_MAX_STAGES];
  int preferred[MOFFT_MAX_PASSES];
  const int tuned = mofft_wisdom_lookup(length, precision_bits, chain, MOFFT_MAX_STAGES,
                                        preferred);
  return mofft_core_create_tuned(out, precision_bits, length, batch, distance, direction,
                                 placement, tuned > 0 ? chain : NULL, tuned,
                                 tuned > 0 ? preferred : NULL);
}

mofft_status mofft_core_create_tuned(mofft_core **out, int precision_bits,
                                     size_t length, size_t batch,
                                     size_t distance, mofft_direction direction,
                                     mofft_placement placement, const int *chain,
                                     int chain_count, const int *preferred) {
  *out = NULL;
  if (!mofft_hardware_supports(precision_bits)) return MOFFT_UNSUPPORTED_HARDWARE;
  if (length < 2 || length > ((size_t)1 << 34)) return MOFFT_UNSUPPORTED_SIZE;
  if (!mofft_is_smooth13(length)) return MOFFT_UNSUPPORTED_SIZE;
  if (batch == 0) return MOFFT_INVALID_ARGUMENT;
  if (distance == 0) distance = length;
  if (distance < length) return MOFFT_INVALID_ARGUMENT;
  if (batch > SIZE_MAX / distance / 16) return MOFFT_ALLOCATION_FAILURE;
  if (!prepare_current_device()) return MOFFT_UNSUPPORTED_HARDWARE;
  mofft_core *c = (mofft_core *)calloc(1, sizeof(*c));
  if (!c) return MOFFT_ALLOCATION_FAILURE;
  pthread_mutex_init(&c->lock, NULL);
  c->length = length;
  c->direction = direction;
  c->placement = placement;
  c->precision_bits = precision_bits;
  c->batch = batch;
  c->distance = distance;
  c->direct_input = 1;
  c->stage_layout = MOFFT_STAGE_LAYOUT_TRANSPOSE;
  for (int i = 0; i < MOFFT_MAX_PASSES; ++i)
    c->preferred[i] = preferred ? preferred[i] : -1;
  cudaGetDevice(&c->device);
  int tmp[MOFFT_MAX_STAGES];
  int count = chain_count;
  if (!chain) {
    count = mofft_model_chain(precision_bits, 0, length, tmp, MOFFT_MAX_STAGES);
    if (count <= 0) {
      mofft_core_destroy(c);
      return MOFFT_UNSUPPORTED_SIZE;
    }
    chain = tmp;
  }
  set_factors_from_chain(c, chain, count);
  cudaStream_t stream = NULL;
  if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    mofft_core_destroy(c);
    return MOFFT_INTERNAL_ERROR;
  }
  c->stream = stream;
  mofft_status st = mofft_core_build(c);
  if (st != MOFFT_SUCCESS) {
    mofft_core_destroy(c);
    return st;
  }
  *out = c;
  return MOFFT_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* execute                                                                   */
/* ------------------------------------------------------------------------ */

static int is_device_pointer(const void *p) {
  struct cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

static mofft_status enqueue_with_work(const mofft_core *c, const void *in, void *out,
                                      size_t batch, size_t distance, void *work,
                                      void *stream);

/* Enqueue the plan's passes: in -> out on `stream` (device pointers). */
mofft_status mofft_core_enqueue(const mofft_core *c, const void *in, void *out,
                                void *stream) {
  return mofft_core_enqueue_batch(c, in, out, c->batch, c->distance, stream);
}

/* The same for `batch` transforms `distance` elements apart (a plan made for
 * one transform serving a request of many).  A schedule that routes through
 * the plan's workspace needs batch <= the plan's batch. */
mofft_status mofft_core_enqueue_batch(const mofft_core *c, const void *in, void *out,
                                      size_t batch, size_t distance, void *stream) {
  if (c->d_work && batch > c->batch) return MOFFT_INTERNAL_ERROR;
  return enqueue_with_work(c, in, out, batch, distance, c->d_work, stream);
}

/* Passes of c over `batch` transforms; `work` (dense, batch x length
 * elements, or NULL) is the intermediate buffer of schedules that need one. */
static mofft_status enqueue_with_work(const mofft_core *c, const void *in, void *out,
                                      size_t batch, size_t distance, void *work,
                                      void *stream) {
  const size_t cb = mofft_complex_bytes(c->precision_bits);
  const int P = c->sched.pass_count;
  const int backward = c->direction == MOFFT_BACKWARD;
  const void *src = in;
  if (distance < c->length) return MOFFT_INVALID_ARGUMENT;
  long long src_dist = (long long)distance;
  for (int p = 0; p < P; ++p) {
    const mofft_pass *ps = &c->sched.pass[p];
    void *dst;
    long long dst_dist;
    if (p == P - 1) {
      dst = out;
      dst_dist = (long long)distance;
    } else if (src != out) {
      dst = out;
      dst_dist = (long long)distance;
    } else {
      if (!work) return MOFFT_INTERNAL_ERROR;
      dst = work;
      dst_dist = (long long)c->length;
    }
    mofft_pass_args a;
    memset(&a, 0, sizeof(a));
    a.in = src;
    a.out = dst;
    a.tw = (const unsigned char *)c->d_twiddles + ps->tw_offset;
    a.tw_hi = (const unsigned char *)c->d_twiddles + ps->tw_hi_offset;
    a.tw_lo = (const unsigned char *)c->d_twiddles + ps->tw_lo_offset;
    a.batch = (long long)batch;
    a.in_dist = src_dist;
    a.out_dist = dst_dist;
    a.total = (long long)c->length;
    a.ns_outer = ps->ns_outer;
    a.split_shift = ps->split_shift;
    a.conj_in = backward && p == 0;
    a.conj_out = backward && p == P - 1;
    if (pass_has_aux(ps))
      a.aux = (const unsigned char *)c->d_twiddles + ps->aux_offset;
    if (pass_has_status(ps))
      a.status = (int *)((unsigned char *)c->d_twiddles + ps->status_offset);
    a.generic_cols = P > 1;
    a.length = ps->length;
    a.lines = ps->lines;
    a.radix_count = ps->radix_count;
    memcpy(a.radices, ps->radices, sizeof(a.radices));
    const int err = mofft_cuda_launch_pass(ps->kernel, &a, stream);
    atomic_fetch_add(&g_launches, 1);
    if (err != 0) {
      cudaGetLastError();
      return MOFFT_INTERNAL_ERROR;
    }
    (void)cb;
    src = dst;
    src_dist = dst_dist;
  }
  return MOFFT_SUCCESS;
}

static mofft_status ensure_staging(mofft_core *c) {
  const size_t bytes = c->batch * c->distance * mofft_complex_bytes(c->precision_bits);
  if (!c->stream2 || !c->stream3) {
    cudaStream_t s2 = (cudaStream_t)c->stream2, s3 = (cudaStream_t)c->stream3;
    if ((!s2 && cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking) != cudaSuccess) ||
        (!s3 && cudaStreamCreateWithFlags(&s3, cudaStreamNonBlocking) != cudaSuccess)) {
      cudaGetLastError();
      return MOFFT_INTERNAL_ERROR;
    }
    c->stream2 = s2;
    c->stream3 = s3;
  }
  for (int i = 0; i < 64; ++i) {
    if (!c->ev_up[i]) {
      cudaEvent_t e;
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return MOFFT_INTERNAL_ERROR;
      }
      c->ev_up[i] = e;
    }
    if (!c->ev_done[i]) {
      cudaEvent_t e;
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return MOFFT_INTERNAL_ERROR;
      }
      c->ev_done[i] = e;
    }
  }
  if (c->stage_bytes >= bytes && c->d_stage[0] && c->d_stage[1])
    return MOFFT_SUCCESS;
  if (c->d_stage[0]) cudaFree(c->d_stage[0]);
  if (c->d_stage[1]) cudaFree(c->d_stage[1]);
  c->d_stage[0] = c->d_stage[1] = NULL;
  c->stage_bytes = 0;
  if (cudaMalloc(&c->d_stage[0], bytes) != cudaSuccess ||
      cudaMalloc(&c->d_stage[1], bytes) != cudaSuccess) {
    cudaGetLastError();
    if (c->d_stage[0]) cudaFree(c->d_stage[0]);
    c->d_stage[0] = NULL;
    return MOFFT_ALLOCATION_FAILURE;
  }
  c->stage_bytes = bytes;
  return MOFFT_SUCCESS;
}

mofft_status mofft_core_execute(const mofft_core *cc, const void *in, void *out) {
  mofft_core *c = (mofft_core *)cc; /* staging buffers are lazily owned state */
  if (!c || !in || !out) return MOFFT_INVALID_ARGUMENT;
  if ((c->placement == MOFFT_IN_PLACE) != (in == out)) return MOFFT_INVALID_ARGUMENT;
  if (!mofft_hardware_supports(c->precision_bits)) return MOFFT_UNSUPPORTED_HARDWARE;
  int saved = -1;
  cudaGetDevice(&saved);
  if (saved != c->device && cudaSetDevice(c->device) != cudaSuccess) {
    cudaGetLastError();
    return MOFFT_INTERNAL_ERROR;
  }
  mofft_status st = MOFFT_SUCCESS;
  const int dev_in = is_device_pointer(in);
  const int dev_out = in == out ? dev_in : is_device_pointer(out);
  void *stream = c->user_stream ? c->user_stream : c->stream;
  if (dev_in && dev_out) {
    st = mofft_core_enqueue(c, in, out, stream);
    if (st == MOFFT_SUCCESS && !c->user_stream &&
        cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) {
      cudaGetLastError();
      st = MOFFT_INTERNAL_ERROR;
    }
    if (st == MOFFT_SUCCESS && !c->user_stream && schedule_has_status(c))
      st = mofft_core_check_status(c);
  } else if (dev_in != dev_out) {
    st = MOFFT_INVALID_ARGUMENT; /* mixed host/device buffers */
  } else {
    /* host buffers: stage through plan-owned device memory, blocking */
    pthread_mutex_lock(&c->lock);
    st = ensure_staging(c);
    if (st == MOFFT_SUCCESS) {
      /* Chunks of about 24 MiB flow through three streams: uploads in order
       * on one, each chunk's passes on another once its upload has landed,
       * downloads on a third once its passes are done.  Each copy engine
       * (host to device, device to host) and the SMs then work back to back,
       * and only real data dependencies (events) order them. */
      const size_t cb = mofft_complex_bytes(c->precision_bits);
      const size_t span = ((c->batch - 1) * c->distance + c->length) * cb;
      const size_t chunk_bytes = (size_t)24 << 20;
      size_t chunks = (span + chunk_bytes - 1) / chunk_bytes;
      if (chunks > c->batch) chunks = c->batch;
      if (chunks > 64) chunks = 64;
      if (chunks < 1) chunks = 1;
      cudaStream_t up = (cudaStream_t)c->stream2, run = (cudaStream_t)c->stream,
                   down = (cudaStream_t)c->stream3;
      for (size_t k = 0; k < chunks && st == MOFFT_SUCCESS; ++k) {
        const size_t b0 = k * c->batch / chunks, b1 = (k + 1) * c->batch / chunks;
        if (b1 == b0) continue;
        const size_t off = b0 * c->distance * cb;
        const size_t bytes = ((b1 - b0 - 1) * c->distance + c->length) * cb;
        unsigned char *din = (unsigned char *)c->d_stage[0] + off;
        unsigned char *dout = (unsigned char *)c->d_stage[1] + off;
        void *work = c->d_work ? (unsigned char *)c->d_work + b0 * c->length * cb : NULL;
        cudaEvent_t uploaded = (cudaEvent_t)c->ev_up[k], done = (cudaEvent_t)c->ev_done[k];
        if (cudaMemcpyAsync(din, (const unsigned char *)in + off, bytes,
                            cudaMemcpyHostToDevice, up) != cudaSuccess ||
            cudaEventRecord(uploaded, up) != cudaSuccess ||
            cudaStreamWaitEvent(run, uploaded, 0) != cudaSuccess)
          st = MOFFT_INTERNAL_ERROR;
        if (st == MOFFT_SUCCESS)
          st = enqueue_with_work(c, din, dout, b1 - b0, c->distance, work, run);
        if (st == MOFFT_SUCCESS &&
            (cudaEventRecord(done, run) != cudaSuccess ||
             cudaStreamWaitEvent(down, done, 0) != cudaSuccess ||
             cudaMemcpyAsync((unsigned char *)out + off, dout, bytes, cudaMemcpyDeviceToHost,
                             down) != cudaSuccess))
          st = MOFFT_INTERNAL_ERROR;
      }
      cudaStream_t streams[3] = {up, run, down};
      for (int i = 0; i < 3; ++i)
        if (cudaStreamSynchronize(streams[i]) != cudaSuccess && st == MOFFT_SUCCESS)
          st = MOFFT_INTERNAL_ERROR;
      if (st != MOFFT_SUCCESS) cudaGetLastError();
      if (st == MOFFT_SUCCESS && schedule_has_status(c)) st = mofft_core_check_status(c);
    }
    pthread_mutex_unlock(&c->lock);
  }
  if (saved >= 0 && saved != c->device) cudaSetDevice(saved);
  return st;
}

uint64_t mofft_launch_count(void) { return (uint64_t)atomic_load(&g_launches); }

void mofft_count_launches(uint64_t n) { atomic_fetch_add(&g_launches, n); }

/* Schedule the planner would build, without touching a GPU. */
mofft_status mofft_schedule_preview(int precision_bits, size_t length,
                                    const int *radices, size_t radix_count,
                                    unsigned int bank,
                                    mofft_plan_schedule *out, int *chain_out,
                                    size_t *chain_count) {
  if (!out || (precision_bits != 32 && precision_bits != 64) ||
      bank >= MOFFT_KERNEL_BANK_COUNT)
    return MOFFT_INVALID_ARGUMENT;
  if (length < 2 || !mofft_is_smooth13(length)) return MOFFT_UNSUPPORTED_SIZE;
  int chain[MOFFT_MAX_STAGES];
  int count;
  if (radices) {
    if (radix_count == 0 || radix_count > MOFFT_MAX_STAGES) return MOFFT_INVALID_ARGUMENT;
    size_t rem = length;
    for (size_t i = 0; i < radix_count; ++i) {
      if (!mofft_is_supported_radix(radices[i]) || rem % (size_t)radices[i])
        return MOFFT_INVALID_ARGUMENT;
      rem /= (size_t)radices[i];
    }
    if (rem != 1) return MOFFT_INVALID_ARGUMENT;
    count = (int)radix_count;
    for (int i = 0; i < count; ++i) chain[i] = radices[count - 1 - i];
  } else {
    count = mofft_model_chain(precision_bits, bank, length, chain, MOFFT_MAX_STAGES);
    if (count <= 0) return MOFFT_UNSUPPORTED_SIZE;
  }
  mofft_schedule s;
  if (!mofft_group_chain(precision_bits, bank, chain, count, (long long)length, &s))
    return MOFFT_UNSUPPORTED_SIZE;
  memset(out, 0, sizeof(*out));
  out->pass_count = s.pass_count;
  for (int p = 0; p < s.pass_count && p < 4; ++p) {
    out->lengths[p] = s.pass[p].length;
    out->kernels[p] = s.pass[p].kernel;
    out->smem_bytes[p] = s.pass[p].smem_bytes;
  }
  if (chain_out && chain_count) {
    /* reference order: outermost radix first */
    for (int i = 0; i < count; ++i) chain_out[i] = chain[count - 1 - i];
    *chain_count = (size_t)count;
  }
  return MOFFT_SUCCESS;
}

/* Pointer-table batch with one table pair per pass: pass p of transform b
 * reads in_tables[p][b] and writes out_tables[p][b] (device arrays of device
 * pointers), so a caller routes each transform through storage of its own
 * between the passes.  Schedules of at most two passes of specialised kernels
 * (MOFFT_UNSUPPORTED_SIZE otherwise).  Launches are counted by the caller. */
mofft_status mofft_core_enqueue_tables(const mofft_core *c, const void *const *const *in_tables,
                                       void *const *const *out_tables, long long batch,
                                       void *stream) {
  const int P = c->sched.pass_count;
  if (P > 2 || batch <= 0) return MOFFT_UNSUPPORTED_SIZE;
  for (int p = 0; p < P; ++p)
    if (c->sched.pass[p].kind == MOFFT_KERNEL_GENERIC ||
        is_tensor_kind(c->sched.pass[p].kind))
      return MOFFT_UNSUPPORTED_SIZE;
  const int backward = c->direction == MOFFT_BACKWARD;
  for (int p = 0; p < P; ++p) {
    const mofft_pass *ps = &c->sched.pass[p];
    mofft_pass_args a;
    memset(&a, 0, sizeof(a));
    a.in_table = in_tables[p];
    a.out_table = out_tables[p];
    a.tw = (const unsigned char *)c->d_twiddles + ps->tw_offset;
    a.tw_hi = (const unsigned char *)c->d_twiddles + ps->tw_hi_offset;
    a.tw_lo = (const unsigned char *)c->d_twiddles + ps->tw_lo_offset;
    a.batch = batch;
    a.total = (long long)c->length;
    a.ns_outer = ps->ns_outer;
    a.split_shift = ps->split_shift;
    a.conj_in = backward && p == 0;
    a.conj_out = backward && p == P - 1;
    a.length = ps->length;
    a.lines = ps->lines;
    a.radix_count = ps->radix_count;
    memcpy(a.radices, ps->radices, sizeof(a.radices));
    if (pass_has_aux(ps))
      a.aux = (const unsigned char *)c->d_twiddles + ps->aux_offset;
    if (pass_has_status(ps))
      a.status = (int *)((unsigned char *)c->d_twiddles + ps->status_offset);
    const int err = mofft_cuda_launch_pass(ps->kernel, &a, stream);
    if (err != 0) {
      cudaGetLastError();
      return MOFFT_INTERNAL_ERROR;
    }
  }
  return MOFFT_SUCCESS;
}

/* Indirect batch: `batch` transforms, transform b read from in_table[b] and
 * written to out_table[b] (device arrays of device pointers).  Out-of-place
 * routing only (the second pass of a two-pass schedule runs in place on the
 * output); schedules with a generic pass or more than two passes are not
 * supported (MOFFT_UNSUPPORTED_SIZE). */
mofft_status mofft_core_enqueue_indirect(const mofft_core *c, const void *const *in_table,
                                         void *const *out_table, long long batch,
                                         void *stream) {
  const void *const *ins[2] = {in_table, (const void *const *)out_table};
  void *const *outs[2] = {out_table, out_table};
  const mofft_status st = mofft_core_enqueue_tables(c, ins, outs, batch, stream);
  if (st == MOFFT_SUCCESS) atomic_fetch_add(&g_launches, (uint64_t)c->sched.pass_count);
  return st;
}
