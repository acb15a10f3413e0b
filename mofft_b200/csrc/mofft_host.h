/* Functions shared between the host translation units of libmofft. */
#ifndef MOFFT_HOST_H
#define MOFFT_HOST_H

#include "mofft_internal.h"

#ifdef __cplusplus
extern "C" {
#endif

int mofft_is_supported_radix(int radix);
int mofft_is_smooth13(size_t n);
double mofft_monotonic_seconds(void);
size_t mofft_complex_bytes(int precision_bits);
int mofft_hardware_supports(int precision_bits);
int mofft_device_family(uint32_t *family);
void mofft_cis_turns(uint64_t num, uint64_t den, long double *c,
                     long double *s);

int mofft_group_chain(int precision_bits, unsigned bank, const int *chain,
                      int count, long long total, mofft_schedule *best);
/* As mofft_group_chain, preferring the listed kernel instances (registry
 * indices, MOFFT_MAX_PASSES entries, -1 = none) where they fit a pass. */
int mofft_group_chain_preferred(int precision_bits, unsigned bank,
                                const int *chain, int count, long long total,
                                const int *preferred, mofft_schedule *best);
int mofft_auto_radices(long long length, int *out, int capacity);
int mofft_model_chain(int precision_bits, unsigned bank, size_t length,
                      int *chain, int capacity);
/* The best chain of two or more passes for `length` (-1 if none). */
int mofft_model_chain_multipass(int precision_bits, unsigned bank, size_t length,
                                int *chain, int capacity);

mofft_status mofft_core_create(mofft_core **out, int precision_bits,
                               size_t length, size_t batch, size_t distance,
                               mofft_direction direction,
                               mofft_placement placement, const int *chain,
                               int chain_count);
mofft_status mofft_core_create_tuned(mofft_core **out, int precision_bits,
                                     size_t length, size_t batch,
                                     size_t distance, mofft_direction direction,
                                     mofft_placement placement, const int *chain,
                                     int chain_count, const int *preferred);
mofft_status mofft_core_build(mofft_core *c);
/* Blocking: MOFFT_INTERNAL_ERROR if a tensor-core kernel of c recorded a
 * timed-out wait, else MOFFT_SUCCESS. */
mofft_status mofft_core_check_status(const mofft_core *c);
mofft_status mofft_core_check_lost_copy(mofft_core *c, const void *in, void *out);
void mofft_core_destroy(mofft_core *c);
mofft_status mofft_core_enqueue(const mofft_core *c, const void *in, void *out,
                                void *stream);
mofft_status mofft_core_enqueue_batch(const mofft_core *c, const void *in, void *out,
                                      size_t batch, size_t distance, void *stream);
mofft_status mofft_core_execute(const mofft_core *c, const void *in, void *out);
mofft_status mofft_core_enqueue_tables(const mofft_core *c, const void *const *const *in_tables,
                                       void *const *const *out_tables, long long batch,
                                       void *stream);
/* A PRETUNED core: the compiled wisdom's schedule for (length, precision)
 * where one exists, else the model's. */
mofft_status mofft_core_create_pretuned(mofft_core **out, int precision_bits, size_t length,
                                        size_t batch, size_t distance,
                                        mofft_direction direction, mofft_placement placement);
mofft_status mofft_core_enqueue_indirect(const mofft_core *c, const void *const *in_table,
                                         void *const *out_table, long long batch,
                                         void *stream);

/* Twiddle tables (mofft_api.c): W_den^(first + k*step), k < count; the
 * internal stage table of an in-CTA chain; ceil(log2 x). */
void mofft_write_twiddles(void *dst, int precision_bits, uint64_t den,
                          uint64_t first, uint64_t step, size_t count);
size_t mofft_stage_table_entries(const int *radices, int count);
void mofft_fill_stage_table(void *dst, int precision_bits, const int *radices,
                            int count);
int mofft_ceil_log2_u64(uint64_t x);
/* Adds n to the process-wide libmofft launch counter. */
void mofft_count_launches(uint64_t n);

/* Device-time model of a schedule over `batch` transforms (mofft_gpu_model.c),
 * seconds; DBL_MAX for a schedule it cannot price. */
double mofft_gpu_schedule_seconds(int precision_bits, size_t length, size_t batch,
                                  const mofft_schedule *s);

/* MEASURE planner (mofft_measure.c). */
mofft_status mofft_search_best(mofft_core **out, int precision_bits,
                               size_t length, size_t batch, size_t distance,
                               mofft_direction direction,
                               mofft_placement placement,
                               const mofft_plan_options *options,
                               mofft_plan_diagnostics *diagnostics);

/* Compiled wisdom (device plan cache) lookup: returns chain length or 0;
 * `preferred` (MOFFT_MAX_PASSES entries, may be NULL) receives the tuned
 * kernel instances as registry indices (-1 = none). */
int mofft_wisdom_lookup(size_t length, int precision_bits, int *chain,
                        int capacity, int *preferred);

/* Kernel banks (the reference's compiled code families, portfolio.py:31-35):
 * 0 the specialised kernels with the default codelets (runtime-stage kernels
 * where none is specialised), 1-3 the runtime-stage kernels with the
 * like-terms, even-odd and vector-reuse rewrite codelets. */
#define MOFFT_KERNEL_BANK_COUNT 4u

#ifdef __cplusplus
}
#endif
#endif
