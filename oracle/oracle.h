/* ORACLE -- test infrastructure only (see oracle.c).  Interleaved complex
 * buffers; direction -1 = forward, +1 = backward; factors outermost first. */
#ifndef MOFFT_ORACLE_H
#define MOFFT_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#define ORACLE_MAX_DEPTH 64

/* Reference-style radix chain for n (prime factors <= 13); returns depth or
 * -1 for unsupported n. */
int oracle_plan_factors(size_t n, int *factors);

/* long double restatement of the reference transform (parity oracle). */
int oracle_fft_ld(const double *in, double *out, size_t n, int dir,
                  const int *factors, int depth);
int oracle_fft_ld_batch(const double *in, double *out, size_t n, size_t batch,
                        size_t dist, int dir, const int *factors, int depth,
                        int threads);
/* Reference-precision ports (CPU baseline). */
int oracle_fft_f32_batch(const float *in, float *out, size_t n, size_t batch,
                         size_t dist, int dir, const int *factors, int depth,
                         int threads);
int oracle_fft_f64_batch(const double *in, double *out, size_t n, size_t batch,
                         size_t dist, int dir, const int *factors, int depth,
                         int threads);
/* Direct O(n^2) DFT, long double accumulation, exactly reduced angles. */
int oracle_dft_ld(const double *in, double *out, size_t n, int dir);

/* splitmix64 uniform[-1,1) inputs: per point two draws, real then imaginary. */
void oracle_fill_uniform_f64(double *out, size_t count, uint64_t seed);
void oracle_fill_uniform_f32(float *out, size_t count, uint64_t seed);

#endif
