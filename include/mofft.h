/* MoFFT public C API, served by NVIDIA B200 (sm_100a) kernels.
 *
 * Every declaration below keeps the name, parameter list, type and enum value
 * of the reference library's public header (include/mofft.h:11-231 of
 * ruge-zhang/MoFFT 0.4.0) so that existing callers relink without source
 * changes.  Behavioural notes specific to this implementation:
 *
 *  - Buffers may live in host memory (pageable or pinned) or in device
 *    memory.  Device buffers run in place on the GPU; host buffers are
 *    staged through plan-owned device memory.  Either way mofft_execute_*
 *    returns after the result is in `output`, unless a stream was attached
 *    with mofft_plan_set_stream_* (mofft_b200.h), in which case execution is
 *    enqueued on that stream and the call returns immediately.
 *  - Transforms are unnormalised in both directions; forward uses
 *    exp(-2*pi*i*j*k/n) (MOFFT_FORWARD = -1), backward exp(+2*pi*i*j*k/n).
 *  - Supported lengths are 2 <= n whose prime factors are all <= 13, as in the
 *    reference.  Other lengths return MOFFT_UNSUPPORTED_SIZE.
 *  - A plan is bound to the CUDA device that was current when it was created.
 */
#ifndef MOFFT_H
#define MOFFT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Interleaved complex values: real part first. */
typedef struct { float real, imag; } mofft_complex_f32;
typedef struct { double real, imag; } mofft_complex_f64;

typedef enum {
  MOFFT_SUCCESS = 0,
  MOFFT_INVALID_ARGUMENT = 1,
  MOFFT_UNSUPPORTED_SIZE = 2,
  MOFFT_ALLOCATION_FAILURE = 3,
  MOFFT_UNSUPPORTED_HARDWARE = 4,
  MOFFT_INTERNAL_ERROR = 5,
  MOFFT_WISDOM_NOT_FOUND = 6,
  MOFFT_INCOMPATIBLE_RECIPE = 7,
  MOFFT_BUFFER_TOO_SMALL = 8
} mofft_status;

typedef enum { MOFFT_FORWARD = -1, MOFFT_BACKWARD = 1 } mofft_direction;
typedef enum { MOFFT_OUT_OF_PLACE = 0, MOFFT_IN_PLACE = 1 } mofft_placement;
typedef enum {
  MOFFT_TRANSPOSE_LINEAR = 0,
  MOFFT_TRANSPOSE_BLOCKED = 1
} mofft_transpose_strategy;
typedef enum {
  MOFFT_STAGE_LAYOUT_TRANSPOSE = 0,
  MOFFT_STAGE_LAYOUT_SECTION = 1
} mofft_stage_layout;

/* PRETUNED: use the compiled device plan cache (wisdom) for this length when
 * it has an entry, else the analytical B200 planner.  MEASURE: time a bounded
 * set of complete candidate schedules on the GPU with CUDA events and keep the
 * fastest.  Neither mode compiles code at run time. */
typedef enum {
  MOFFT_PLANNER_PRETUNED = 0,
  MOFFT_PLANNER_MEASURE = 1
} mofft_planner_mode;

enum {
  /* PRETUNED only: fail with MOFFT_WISDOM_NOT_FOUND when the length has no
   * compiled wisdom entry instead of using the analytical planner. */
  MOFFT_PLAN_STRICT_WISDOM = 1u << 0
};

/* Zero candidate_limit / timing_samples select the defaults (16 / 5); the
 * maxima are 64 candidates and 31 samples. */
typedef struct {
  mofft_planner_mode mode;
  uint32_t flags;
  size_t candidate_limit;
  uint32_t timing_samples;
} mofft_plan_options;

#define MOFFT_MAX_PLAN_DEPTH 64
typedef struct {
  int measured;
  int used_wisdom;
  int used_model_fallback;
  size_t candidates_measured;
  size_t radix_count;
  int radices[MOFFT_MAX_PLAN_DEPTH];
  unsigned int kernel_bank;
  unsigned int kernel_bank_count;
  uint64_t blocked_transpose_mask;
  int direct_input;
  mofft_stage_layout stage_layout;
  double planning_seconds;
  double selected_median_seconds;
  /* Shape of the plan, so an imported recipe is enough to size buffers. */
  size_t length;
  int precision_bits;
  mofft_direction direction;
  mofft_placement placement;
} mofft_plan_diagnostics;

/* Flags of the bound-array constructors. */
enum {
  MOFFT_FLAG_PRETUNED = 0,
  MOFFT_FLAG_MEASURE = 1u << 0,
  MOFFT_FLAG_WISDOM_ONLY = 1u << 1
};

typedef struct {
  double kernel_cost;
  double memory_cost;
  double layout_cost;
  double total_cost;
  size_t logical_read_bytes;
  size_t logical_write_bytes;
  size_t transferred_read_bytes;
  size_t transferred_write_bytes;
  size_t peak_working_set_bytes;
} mofft_plan_cost_breakdown;

typedef struct mofft_plan_f32 mofft_plan_f32;
typedef struct mofft_plan_f64 mofft_plan_f64;

/* Replaces include/mofft.h:107-113 (implementation src/mofft.c:1232-1280). */
mofft_status mofft_plan_create_f32(mofft_plan_f32 **plan, size_t length,
                                   mofft_direction direction,
                                   mofft_placement placement);
mofft_status mofft_plan_create_f64(mofft_plan_f64 **plan, size_t length,
                                   mofft_direction direction,
                                   mofft_placement placement);

/* Fills PRETUNED defaults; a NULL options pointer means the same.
 * Replaces include/mofft.h:116-127 (src/mofft.c:739-762, 1282-1382). */
void mofft_plan_options_init(mofft_plan_options *options);
mofft_status mofft_plan_create_with_options_f32(
    mofft_plan_f32 **plan, size_t length, mofft_direction direction,
    mofft_placement placement, const mofft_plan_options *options,
    mofft_plan_diagnostics *diagnostics);
mofft_status mofft_plan_create_with_options_f64(
    mofft_plan_f64 **plan, size_t length, mofft_direction direction,
    mofft_placement placement, const mofft_plan_options *options,
    mofft_plan_diagnostics *diagnostics);

/* Replaces include/mofft.h:129-136 (src/mofft.c:1384-1442).
 * Bound-array lifecycle: NULL on failure; flags are 0, MOFFT_FLAG_MEASURE or
 * MOFFT_FLAG_WISDOM_ONLY.  Placement follows input == output and the plan
 * keeps both addresses for mofft_execute_plan_*. */
mofft_plan_f32 *mofft_plan_dft_1d_f32(
    size_t length, const mofft_complex_f32 *input,
    mofft_complex_f32 *output, mofft_direction direction, uint32_t flags);
mofft_plan_f64 *mofft_plan_dft_1d_f64(
    size_t length, const mofft_complex_f64 *input,
    mofft_complex_f64 *output, mofft_direction direction, uint32_t flags);
mofft_status mofft_execute_plan_f32(const mofft_plan_f32 *plan);
mofft_status mofft_execute_plan_f64(const mofft_plan_f64 *plan);

/* Replaces include/mofft.h:140-145 (src/mofft.c:1054-1080, 1444-1470).
 * Explicit radix chain, outermost level first (the last radix is the first
 * stage applied).  Every radix must be one of 2..16, 32, 64 and the product
 * must equal length. */
mofft_status mofft_plan_create_with_radices_f32(
    mofft_plan_f32 **plan, size_t length, mofft_direction direction,
    mofft_placement placement, const int *radices, size_t radix_count);
mofft_status mofft_plan_create_with_radices_f64(
    mofft_plan_f64 **plan, size_t length, mofft_direction direction,
    mofft_placement placement, const int *radices, size_t radix_count);
/* Replaces include/mofft.h:147-171 (src/mofft.c:1498-1598).
 * Layout knobs of the reference's CPU driver.  They are validated, kept, and
 * exported in recipes; on the GPU every level exchange happens inside shared
 * memory, so they do not change the result. */
mofft_status mofft_plan_set_transpose_strategy_f32(
    mofft_plan_f32 *plan, mofft_transpose_strategy strategy);
mofft_status mofft_plan_set_transpose_strategy_f64(
    mofft_plan_f64 *plan, mofft_transpose_strategy strategy);
mofft_status mofft_plan_set_blocked_transpose_mask_f32(
    mofft_plan_f32 *plan, uint64_t blocked_levels);
mofft_status mofft_plan_set_blocked_transpose_mask_f64(
    mofft_plan_f64 *plan, uint64_t blocked_levels);
mofft_status mofft_plan_set_direct_input_f32(mofft_plan_f32 *plan,
                                              int enabled);
mofft_status mofft_plan_set_direct_input_f64(mofft_plan_f64 *plan,
                                              int enabled);
mofft_status mofft_plan_set_stage_layout_f32(mofft_plan_f32 *plan,
                                              mofft_stage_layout layout);
mofft_status mofft_plan_set_stage_layout_f64(mofft_plan_f64 *plan,
                                              mofft_stage_layout layout);
/* Kernel banks select the GPU kernel family: bank 0 is the specialised
 * register-resident Stockham family, bank 1 the runtime-stage-list family. */
mofft_status mofft_plan_set_kernel_bank_f32(mofft_plan_f32 *plan,
                                             unsigned int bank);
mofft_status mofft_plan_set_kernel_bank_f64(mofft_plan_f64 *plan,
                                             unsigned int bank);
mofft_status mofft_plan_get_kernel_bank_f32(const mofft_plan_f32 *plan,
                                             unsigned int *bank);
mofft_status mofft_plan_get_kernel_bank_f64(const mofft_plan_f64 *plan,
                                             unsigned int *bank);

/* Replaces include/mofft.h:176-194 (src/mofft.c:1600-1842).
 * 64 lowercase hex digits identifying this build (kernels, planner, wisdom).
 * Recipes are text records scoped to the build and the GPU family (compute
 * capability and SM count); they hold no pointers or timings. */
const char *mofft_build_id(void);
/* Size query: buffer NULL and capacity 0; *required counts the final NUL.  A
 * short buffer is left untouched and MOFFT_BUFFER_TOO_SMALL is returned. */
mofft_status mofft_plan_export_f32(const mofft_plan_f32 *plan, char *buffer,
                                   size_t capacity, size_t *required);
mofft_status mofft_plan_export_f64(const mofft_plan_f64 *plan, char *buffer,
                                   size_t capacity, size_t *required);
/* recipe_size counts the final NUL.  Import builds a fresh plan without
 * measuring; a build / GPU family / precision mismatch gives
 * MOFFT_INCOMPATIBLE_RECIPE and *plan = NULL.  Buffer addresses are never
 * restored. */
mofft_status mofft_plan_import_f32(mofft_plan_f32 **plan, const char *recipe,
                                   size_t recipe_size,
                                   mofft_plan_diagnostics *diagnostics);
mofft_status mofft_plan_import_f64(mofft_plan_f64 **plan, const char *recipe,
                                   size_t recipe_size,
                                   mofft_plan_diagnostics *diagnostics);

/* Replaces include/mofft.h:196-203 (src/mofft.c:2169-2211). */
mofft_status mofft_execute_f32(const mofft_plan_f32 *plan,
                               const mofft_complex_f32 *input,
                               mofft_complex_f32 *output);
mofft_status mofft_execute_f64(const mofft_plan_f64 *plan,
                               const mofft_complex_f64 *input,
                               mofft_complex_f64 *output);

void mofft_plan_destroy_f32(mofft_plan_f32 *plan);
void mofft_plan_destroy_f64(mofft_plan_f64 *plan);
/* Replaces include/mofft.h:205-227 (src/mofft.c:133-325, 2213-2218).
 * Analytical cost model (B200 parameters: HBM / L2 bandwidth, FP32 / FP64
 * throughput, 128-byte lines), in microseconds. */
double mofft_estimated_radix_cost(int radix, int precision_bits,
                                  int first_stage);
double mofft_estimated_stage_cost(int radix, int precision_bits,
                                  int first_stage, size_t transform_length,
                                  size_t stage_length);
double mofft_estimated_plan_cost(size_t length, int precision_bits,
                                 const int *radices, size_t radix_count,
                                 uint64_t blocked_transpose_mask,
                                 int direct_input);
double mofft_estimated_plan_cost_with_layout(
    size_t length, int precision_bits, const int *radices, size_t radix_count,
    uint64_t blocked_transpose_mask, int direct_input,
    mofft_stage_layout layout);
mofft_status mofft_estimated_plan_cost_breakdown_with_layout(
    size_t length, int precision_bits, const int *radices, size_t radix_count,
    uint64_t blocked_transpose_mask, int direct_input,
    mofft_stage_layout layout, mofft_plan_cost_breakdown *breakdown);
/* Replaces include/mofft.h:228-231 (src/mofft.c:2219-2242). */
int mofft_wisdom_is_formal(void);
const char *mofft_wisdom_source(void);
const char *mofft_status_string(mofft_status status);
const char *mofft_version(void);

#ifdef __cplusplus
}
#endif
#endif
