/* ORACLE -- test infrastructure only.
 *
 * This file is the CPU restatement of the reference's transform, used as the
 * checker of the GPU library in tests/, as the checker in
 * __graft_entry__.smoke(), and as the timed CPU baseline ("port") in bench.py.
 * Nothing in the product (libmofft.so, mofft_b200/) links or calls it.
 *
 * What it restates (ruge-zhang/MoFFT 0.4.0):
 *  - the execute driver, TRANSPOSE layout with direct strided input
 *    (src/mofft.c:1932-2045): the innermost radix r = factors[d-1] runs first
 *    as  cur[k*B + b] = sum_j x[j*B + b] W_r^{jk}  (B = N/r; the codelet
 *    contract of compiler/mofft_compiler/validate.py:115-127), then for each
 *    level = d-2 .. 0 with n = level length, R = factors[level], m = n/R,
 *    P = N/n:
 *       out[k*(N/R) + g*P + o] = sum_j cur[(g*R + j)*P + o] * t(j,g) * W_R^{jk}
 *    with t(j,g) = exp(dir*2*pi*i*j*g/n) (the compact twiddle table of
 *    src/mofft.c:1082-1110, index k1*m + b);
 *  - the codelets as dense DFT-matrix products (the SME outer-product method,
 *    compiler/mofft_compiler/emitter.py:56-65 coefficients);
 *  - the length rule: prime factors <= 13, radices {64,32,16,15,...,2}
 *    (src/mofft.c:27-28) chosen by a memoised minimum-cost search over that
 *    list as choose_factorization does (src/mofft.c:327-351); the cost per
 *    stage here is radix + 8 (DFT-matrix work plus one memory pass), because
 *    the reference's generated SME cost tables do not exist off Apple
 *    hardware.  Any factorization computes the same DFT.
 *
 * Three arithmetic widths:
 *  - long double with exactly reduced twiddle angles: the parity oracle;
 *  - float and double with twiddles computed in double and rounded, as the
 *    reference does: the CPU baseline (OpenMP over the batch).
 * Plus a direct O(n^2) DFT in long double (tests/test_fft.c:20-26 style) and
 * the splitmix64 input generator shared with the GPU tests.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static const int k_radices[] = {64, 32, 16, 15, 14, 13, 12, 11, 10,
                                9,  8,  7,  6,  5,  4,  3,  2};
#define NRAD (int)(sizeof(k_radices) / sizeof(k_radices[0]))

/* ---------------------------------------------------------------- factors */

/* Memoised minimum-cost chain over the reference's radix list (the shape of
 * choose_factorization, src/mofft.c:327-351), keyed by the remaining length. */
typedef struct {
  size_t key;
  double cost;
  int radix;
} memo_slot;

#define MEMO_SIZE 16384

static double chain_cost(size_t n, memo_slot *memo) {
  if (n == 1) return 0.0;
  size_t h = (n * UINT64_C(0x9E3779B97F4A7C15)) >> 50;
  for (;;) {
    memo_slot *slot = &memo[h & (MEMO_SIZE - 1)];
    if (slot->key == n) return slot->cost;
    if (slot->key == 0) break;
    ++h;
  }
  double best = 1e300;
  int best_radix = 0;
  for (int i = 0; i < NRAD; ++i) {
    const int r = k_radices[i];
    if (n % (size_t)r) continue;
    const double c = chain_cost(n / (size_t)r, memo) + (double)r + 8.0;
    if (c < best) {
      best = c;
      best_radix = r;
    }
  }
  h = (n * UINT64_C(0x9E3779B97F4A7C15)) >> 50;
  for (;;) {
    memo_slot *slot = &memo[h & (MEMO_SIZE - 1)];
    if (slot->key == 0) {
      slot->key = n;
      slot->cost = best;
      slot->radix = best_radix;
      break;
    }
    ++h;
  }
  return best;
}

static int memo_radix(size_t n, const memo_slot *memo) {
  size_t h = (n * UINT64_C(0x9E3779B97F4A7C15)) >> 50;
  for (;;) {
    const memo_slot *slot = &memo[h & (MEMO_SIZE - 1)];
    if (slot->key == n) return slot->radix;
    if (slot->key == 0) return 0;
    ++h;
  }
}

int oracle_plan_factors(size_t n, int *factors) {
  if (n < 2) return -1;
  size_t m = n;
  static const int primes[] = {2, 3, 5, 7, 11, 13};
  for (int i = 0; i < 6; ++i)
    while (m % (size_t)primes[i] == 0) m /= (size_t)primes[i];
  if (m != 1) return -1;
  memo_slot *memo = (memo_slot *)calloc(MEMO_SIZE, sizeof(memo_slot));
  if (!memo) return -1;
  chain_cost(n, memo);
  int depth = 0;
  while (n > 1 && depth < ORACLE_MAX_DEPTH) {
    const int r = memo_radix(n, memo);
    if (r == 0) break;
    factors[depth++] = r;
    n /= (size_t)r;
  }
  free(memo);
  return n == 1 ? depth : -1;
}

/* ------------------------------------------------------- exact twiddles */

static void cis_turns_ld(unsigned long long num, unsigned long long den,
                         long double *c, long double *s) {
  num %= den;
  const unsigned __int128 eight = (unsigned __int128)num * 8u;
  unsigned long long octant = (unsigned long long)(eight / den);
  unsigned long long rest = (unsigned long long)(eight - (unsigned __int128)octant * den);
  const int mirror = (int)(octant & 1u);
  if (mirror) rest = den - rest;
  const long double x = 0.785398163397448309615660845819875721L *
                        ((long double)rest / (long double)den);
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

/* --------------------------------------------------- generic transform */

#define DEFINE_FFT(NAME, T, TW)                                                 \
  static void NAME(const T *x, T *y, T *scratch, size_t N, int dir,             \
                   const int *f, int d, const T *coef_re, const T *coef_im,     \
                   const size_t *coef_off, const T *tw, const size_t *tw_off) { \
    /* x, y interleaved; scratch holds 2N complex */                            \
    T *cur = scratch, *nxt = scratch + 2 * N;                                   \
    {                                                                           \
      const int r = f[d - 1];                                                   \
      const size_t B = N / (size_t)r;                                           \
      const T *cr = coef_re + coef_off[d - 1], *ci = coef_im + coef_off[d - 1]; \
      T *dst = d == 1 ? y : cur;                                                \
      for (int k = 0; k < r; ++k) {                                             \
        T *o = dst + 2 * (size_t)k * B;                                         \
        for (size_t b = 0; b < B; ++b) { o[2 * b] = 0; o[2 * b + 1] = 0; }      \
        for (int j = 0; j < r; ++j) {                                           \
          const T wr = cr[j * r + k], wi = ci[j * r + k];                       \
          const T *in = x + 2 * (size_t)j * B;                                  \
          for (size_t b = 0; b < B; ++b) {                                      \
            const T ar = in[2 * b], ai = in[2 * b + 1];                         \
            o[2 * b] += ar * wr - ai * wi;                                      \
            o[2 * b + 1] += ar * wi + ai * wr;                                  \
          }                                                                     \
        }                                                                       \
      }                                                                         \
      if (d == 1) return;                                                       \
    }                                                                           \
    size_t n = N;                                                               \
    size_t lengths[ORACLE_MAX_DEPTH];                                           \
    for (int l = 0; l < d; ++l) { lengths[l] = n; n /= (size_t)f[l]; }          \
    for (int level = d - 2; level >= 0; --level) {                              \
      const size_t nl = lengths[level];                                         \
      const int R = f[level];                                                   \
      const size_t m = nl / (size_t)R, P = N / nl, S = N / (size_t)R;           \
      const T *cr = coef_re + coef_off[level], *ci = coef_im + coef_off[level]; \
      const T *t = tw + 2 * tw_off[level];                                      \
      T *dst = level == 0 ? y : nxt;                                            \
      T row_re[64], row_im[64];                               \
      for (size_t g = 0; g < m; ++g) {                                          \
        for (size_t o = 0; o < P; ++o) {                                        \
          for (int j = 0; j < R; ++j) {                                         \
            const T *src = cur + 2 * (((g * (size_t)R + (size_t)j) * P) + o);   \
            const T twr = t[2 * ((size_t)j * m + g)];                           \
            const T twi = t[2 * ((size_t)j * m + g) + 1];                       \
            row_re[j] = src[0] * twr - src[1] * twi;                            \
            row_im[j] = src[0] * twi + src[1] * twr;                            \
          }                                                                     \
          for (int k = 0; k < R; ++k) {                                         \
            TW acc_r = 0, acc_i = 0;                                            \
            for (int j = 0; j < R; ++j) {                                       \
              const T wr = cr[j * R + k], wi = ci[j * R + k];                   \
              acc_r += row_re[j] * wr - row_im[j] * wi;                         \
              acc_i += row_re[j] * wi + row_im[j] * wr;                         \
            }                                                                   \
            T *out = dst + 2 * ((size_t)k * S + g * P + o);                     \
            out[0] = (T)acc_r;                                                  \
            out[1] = (T)acc_i;                                                  \
          }                                                                     \
        }                                                                       \
      }                                                                         \
      T *tmp = cur;                                                             \
      cur = nxt;                                                                \
      nxt = tmp;                                                                \
    }                                                                           \
  }

DEFINE_FFT(fft_f32, float, float)
DEFINE_FFT(fft_f64, double, double)
DEFINE_FFT(fft_ld, long double, long double)

/* Coefficient and twiddle tables for a factor chain, in type T.
 * mode 0: float, 1: double, 2: long double (exactly reduced). */
typedef struct {
  void *coef_re, *coef_im, *tw;
  size_t coef_off[ORACLE_MAX_DEPTH], tw_off[ORACLE_MAX_DEPTH];
} tables;

static int build_tables(tables *tb, size_t N, int dir, const int *f, int d,
                        int mode) {
  const size_t es = mode == 0 ? sizeof(float) : mode == 1 ? sizeof(double)
                                                          : sizeof(long double);
  size_t coef = 0, tw = 0, n = N;
  for (int l = 0; l < d; ++l) {
    tb->coef_off[l] = coef;
    coef += (size_t)f[l] * (size_t)f[l];
    tb->tw_off[l] = tw;
    if (l < d - 1) tw += n; /* compact table: R x m = n entries */
    n /= (size_t)f[l];
  }
  tb->coef_re = malloc(coef * es);
  tb->coef_im = malloc(coef * es);
  tb->tw = malloc((tw + 1) * 2 * es);
  if (!tb->coef_re || !tb->coef_im || !tb->tw) return 0;
  for (int l = 0; l < d; ++l) {
    const int R = f[l];
    for (int j = 0; j < R; ++j)
      for (int k = 0; k < R; ++k) {
        const size_t idx = tb->coef_off[l] + (size_t)(j * R + k);
        const unsigned long long e = (unsigned long long)((j * k) % R);
        if (mode == 2) {
          long double c, s;
          cis_turns_ld(e, (unsigned long long)R, &c, &s);
          ((long double *)tb->coef_re)[idx] = c;
          ((long double *)tb->coef_im)[idx] = dir * s;
        } else {
          const double a = (double)dir * 2.0 * 3.141592653589793238462643383279502884 *
                           (double)e / (double)R;
          if (mode == 0) {
            ((float *)tb->coef_re)[idx] = (float)cos(a);
            ((float *)tb->coef_im)[idx] = (float)sin(a);
          } else {
            ((double *)tb->coef_re)[idx] = cos(a);
            ((double *)tb->coef_im)[idx] = sin(a);
          }
        }
      }
  }
  n = N;
  for (int l = 0; l < d - 1; ++l) {
    const int R = f[l];
    const size_t m = n / (size_t)R;
    for (int k1 = 0; k1 < R; ++k1)
      for (size_t b = 0; b < m; ++b) {
        const size_t idx = 2 * (tb->tw_off[l] + (size_t)k1 * m + b);
        if (mode == 2) {
          long double c, s;
          cis_turns_ld((unsigned long long)k1 * b, (unsigned long long)n, &c, &s);
          ((long double *)tb->tw)[idx] = c;
          ((long double *)tb->tw)[idx + 1] = dir * s;
        } else {
          const double a = (double)dir * 2.0 * 3.141592653589793238462643383279502884 *
                           (double)k1 * (double)b / (double)n;
          if (mode == 0) {
            ((float *)tb->tw)[idx] = (float)cos(a);
            ((float *)tb->tw)[idx + 1] = (float)sin(a);
          } else {
            ((double *)tb->tw)[idx] = cos(a);
            ((double *)tb->tw)[idx + 1] = sin(a);
          }
        }
      }
    n /= (size_t)R;
  }
  return 1;
}

static void free_tables(tables *tb) {
  free(tb->coef_re);
  free(tb->coef_im);
  free(tb->tw);
}

static int resolve_factors(size_t n, const int *factors, int depth, int *out) {
  if (factors && depth > 0) {
    size_t p = 1;
    for (int i = 0; i < depth; ++i) {
      out[i] = factors[i];
      p *= (size_t)factors[i];
    }
    return p == n ? depth : -1;
  }
  return oracle_plan_factors(n, out);
}

#define DEFINE_BATCH(NAME, FFT, T, MODE, IO)                                     \
  int NAME(const IO *in, IO *out, size_t n, size_t batch, size_t dist,          \
           int dir, const int *factors, int depth, int threads) {               \
    int f[ORACLE_MAX_DEPTH];                                                    \
    const int d = resolve_factors(n, factors, depth, f);                        \
    if (d <= 0 || (dir != -1 && dir != 1)) return -1;                           \
    tables tb;                                                                  \
    memset(&tb, 0, sizeof(tb));                                                 \
    if (!build_tables(&tb, n, dir, f, d, MODE)) { free_tables(&tb); return -2; } \
    int failed = 0;                                                             \
    if (threads <= 0) threads = 1;                                              \
    _Pragma("omp parallel num_threads(threads) reduction(|:failed)")            \
    {                                                                           \
      T *scratch = (T *)malloc(4 * n * sizeof(T));                              \
      T *xin = (T *)malloc(2 * n * sizeof(T));                                  \
      T *yout = (T *)malloc(2 * n * sizeof(T));                                 \
      if (!scratch || !xin || !yout) failed = 1;                                \
      _Pragma("omp for schedule(static)")                                       \
      for (long long b = 0; b < (long long)batch; ++b) {                        \
        if (!scratch || !xin || !yout) continue;                                \
        const IO *src = in + 2 * (size_t)b * dist;                              \
        IO *dst = out + 2 * (size_t)b * dist;                                   \
        for (size_t i = 0; i < 2 * n; ++i) xin[i] = (T)src[i];                  \
        FFT(xin, yout, scratch, n, dir, f, d, (const T *)tb.coef_re,            \
            (const T *)tb.coef_im, tb.coef_off, (const T *)tb.tw, tb.tw_off);   \
        for (size_t i = 0; i < 2 * n; ++i) dst[i] = (IO)yout[i];                \
      }                                                                         \
      free(scratch);                                                            \
      free(xin);                                                                \
      free(yout);                                                               \
    }                                                                           \
    free_tables(&tb);                                                           \
    return failed ? -2 : d;                                                     \
  }

DEFINE_BATCH(oracle_fft_f32_batch, fft_f32, float, 0, float)
DEFINE_BATCH(oracle_fft_f64_batch, fft_f64, double, 1, double)
DEFINE_BATCH(oracle_fft_ld_batch, fft_ld, long double, 2, double)

int oracle_fft_ld(const double *in, double *out, size_t n, int dir,
                  const int *factors, int depth) {
  return oracle_fft_ld_batch(in, out, n, 1, n, dir, factors, depth, 1);
}

int oracle_dft_ld(const double *in, double *out, size_t n, int dir) {
  if (n == 0 || (dir != -1 && dir != 1)) return -1;
  long double *c = (long double *)malloc(n * sizeof(long double));
  long double *s = (long double *)malloc(n * sizeof(long double));
  if (!c || !s) {
    free(c);
    free(s);
    return -2;
  }
  for (size_t e = 0; e < n; ++e) cis_turns_ld(e, n, &c[e], &s[e]);
  for (size_t k = 0; k < n; ++k) {
    long double re = 0, im = 0;
    for (size_t j = 0; j < n; ++j) {
      const size_t e = (size_t)(((unsigned __int128)j * k) % n);
      const long double wr = c[e], wi = dir * s[e];
      re += in[2 * j] * wr - in[2 * j + 1] * wi;
      im += in[2 * j] * wi + in[2 * j + 1] * wr;
    }
    out[2 * k] = (double)re;
    out[2 * k + 1] = (double)im;
  }
  free(c);
  free(s);
  return 0;
}

/* ------------------------------------------------------------- inputs */

static uint64_t splitmix64(uint64_t *state) {
  uint64_t z = (*state += UINT64_C(0x9E3779B97F4A7C15));
  z = (z ^ (z >> 30)) * UINT64_C(0xBF58476D1CE4E5B9);
  z = (z ^ (z >> 27)) * UINT64_C(0x94D049BB133111EB);
  return z ^ (z >> 31);
}

static double uniform_pm1(uint64_t *state) {
  const double u = (double)(splitmix64(state) >> 11) * (1.0 / 9007199254740992.0);
  return 2.0 * u - 1.0;
}

void oracle_fill_uniform_f64(double *out, size_t count, uint64_t seed) {
  uint64_t state = seed;
  for (size_t i = 0; i < count; ++i) {
    out[2 * i] = uniform_pm1(&state);
    out[2 * i + 1] = uniform_pm1(&state);
  }
}

void oracle_fill_uniform_f32(float *out, size_t count, uint64_t seed) {
  uint64_t state = seed;
  for (size_t i = 0; i < count; ++i) {
    out[2 * i] = (float)uniform_pm1(&state);
    out[2 * i + 1] = (float)uniform_pm1(&state);
  }
}
