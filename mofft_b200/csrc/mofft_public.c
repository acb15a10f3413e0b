/* Public entry points of include/mofft.h and include/mofft_b200.h.
 *
 * Argument validation, status codes, ownership and diagnostics follow the
 * reference implementation entry for entry (src/mofft.c:1232-1598 for plan
 * creation, options and setters; :1384-1442 for the bound-array API;
 * :1600-1842 for recipes; :2169-2211 for execute/destroy), so that callers
 * observe the same contract.  The work itself is delegated to the GPU core
 * (mofft_api.c). */
#include <cuda_runtime_api.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mofft_host.h"
#include "mofft_recipe.h"

#ifndef MOFFT_BINARY_ID
#define MOFFT_BINARY_ID "0000000000000000000000000000000000000000000000000000000000000000"
#endif

#define DEFAULT_SEARCH_CANDIDATES 16
#define DEFAULT_TIMING_SAMPLES 5
#define MAX_SEARCH_CANDIDATES 64
#define MAX_TIMING_SAMPLES 31

/* ------------------------------------------------------------------------ */
/* options and diagnostics                                                   */
/* ------------------------------------------------------------------------ */

void mofft_plan_options_init(mofft_plan_options *options) {
  if (!options) return;
  options->mode = MOFFT_PLANNER_PRETUNED;
  options->flags = 0;
  options->candidate_limit = 0;
  options->timing_samples = 0;
}

#define FORM_BITS ((uint32_t)MOFFT_PLAN_FORM_TF32X3 | (uint32_t)MOFFT_PLAN_FORM_BF16X3)

/* Same acceptance rules as the reference's validate_options
 * (src/mofft.c:739-762); the precision-form bits are this library's. */
static mofft_status validate_options(const mofft_plan_options *given,
                                     mofft_plan_options *resolved) {
  if (given) *resolved = *given;
  else mofft_plan_options_init(resolved);
  if ((resolved->mode != MOFFT_PLANNER_PRETUNED &&
       resolved->mode != MOFFT_PLANNER_MEASURE) ||
      (resolved->flags & ~((uint32_t)MOFFT_PLAN_STRICT_WISDOM | FORM_BITS)) != 0 ||
      (resolved->flags & FORM_BITS) == FORM_BITS ||
      (resolved->mode == MOFFT_PLANNER_MEASURE && resolved->flags != 0))
    return MOFFT_INVALID_ARGUMENT;
  if (resolved->candidate_limit == 0)
    resolved->candidate_limit = DEFAULT_SEARCH_CANDIDATES;
  if (resolved->timing_samples == 0)
    resolved->timing_samples = DEFAULT_TIMING_SAMPLES;
  if (resolved->candidate_limit > MAX_SEARCH_CANDIDATES ||
      resolved->timing_samples > MAX_TIMING_SAMPLES)
    return MOFFT_INVALID_ARGUMENT;
  return MOFFT_SUCCESS;
}

static void copy_plan_diagnostics(mofft_plan_diagnostics *d,
                                  const mofft_core *c) {
  if (!d) return;
  d->radix_count = (size_t)c->depth;
  memcpy(d->radices, c->factors, (size_t)c->depth * sizeof(int));
  d->blocked_transpose_mask = c->blocked_transpose_mask;
  d->direct_input = c->direct_input;
  d->stage_layout = c->stage_layout;
  d->kernel_bank = c->kernel_bank;
  d->kernel_bank_count = MOFFT_KERNEL_BANK_COUNT;
  d->length = c->length;
  d->precision_bits = c->precision_bits;
  d->direction = (mofft_direction)c->direction;
  d->placement = c->placement;
}

static int valid_shape(mofft_direction direction, mofft_placement placement) {
  return (direction == MOFFT_FORWARD || direction == MOFFT_BACKWARD) &&
         (placement == MOFFT_IN_PLACE || placement == MOFFT_OUT_OF_PLACE);
}

/* Plan creation shared by every constructor that takes options. */
static mofft_status create_with_options(mofft_core **out, int precision_bits,
                                        size_t length, size_t batch,
                                        size_t distance,
                                        mofft_direction direction,
                                        mofft_placement placement,
                                        const mofft_plan_options *given,
                                        mofft_plan_diagnostics *diagnostics) {
  if (diagnostics) memset(diagnostics, 0, sizeof(*diagnostics));
  if (!valid_shape(direction, placement)) return MOFFT_INVALID_ARGUMENT;
  mofft_plan_options options;
  mofft_status status = validate_options(given, &options);
  if (status != MOFFT_SUCCESS) return status;
  const int form = (options.flags & MOFFT_PLAN_FORM_TF32X3)   ? MOFFT_FORM_TF32X3
                   : (options.flags & MOFFT_PLAN_FORM_BF16X3) ? MOFFT_FORM_BF16X3
                                                              : MOFFT_FORM_FP32;
  if (form != MOFFT_FORM_FP32 && precision_bits != 32) return MOFFT_INVALID_ARGUMENT;
  if (!mofft_hardware_supports(precision_bits)) return MOFFT_UNSUPPORTED_HARDWARE;
  const double start = mofft_monotonic_seconds();
  if (start < 0.0) return MOFFT_INTERNAL_ERROR;
  if (options.mode == MOFFT_PLANNER_MEASURE) {
    status = mofft_search_best(out, precision_bits, length, batch, distance,
                               direction, placement, &options, diagnostics);
    if (status != MOFFT_SUCCESS) return status;
    if (diagnostics) {
      diagnostics->planning_seconds = mofft_monotonic_seconds() - start;
      diagnostics->kernel_bank_count = MOFFT_KERNEL_BANK_COUNT;
    }
    return MOFFT_SUCCESS;
  }
  int chain[MOFFT_MAX_STAGES];
  int preferred[MOFFT_MAX_PASSES];
  int wisdom = mofft_wisdom_lookup(length, precision_bits, chain,
                                   MOFFT_MAX_STAGES, preferred);
  if (!wisdom && (options.flags & MOFFT_PLAN_STRICT_WISDOM))
    return MOFFT_WISDOM_NOT_FOUND;
  /* A tuned schedule never costs memory the untuned one does not: a
   * schedule of three or more passes, or of two passes in place, needs a
   * batch-sized workspace; when the tuned schedule needs one and the model
   * schedule does not, the plan keeps the model schedule (unless the caller
   * insists on wisdom). */
  if (wisdom && !(options.flags & MOFFT_PLAN_STRICT_WISDOM)) {
    int tuned_passes = 0;
    while (tuned_passes < MOFFT_MAX_PASSES && preferred[tuned_passes] >= 0) ++tuned_passes;
    const int in_place = placement == MOFFT_IN_PLACE;
    mofft_plan_schedule model;
    if ((tuned_passes >= 3 || (tuned_passes == 2 && in_place)) &&
        mofft_schedule_preview(precision_bits, length, NULL, 0, 0, &model, NULL, NULL) ==
            MOFFT_SUCCESS &&
        !(model.pass_count >= 3 || (model.pass_count == 2 && in_place)))
      wisdom = 0;
  }
  status = mofft_core_create_tuned(out, precision_bits, length, batch, distance,
                                   direction, placement, wisdom ? chain : NULL,
                                   wisdom, preferred);
  if (status == MOFFT_SUCCESS && form != MOFFT_FORM_FP32) {
    (*out)->form = form;
    status = mofft_core_build(*out);
    if (status != MOFFT_SUCCESS) {
      mofft_core_destroy(*out);
      *out = NULL;
      return status;
    }
  }
  if (status == MOFFT_SUCCESS && diagnostics) {
    diagnostics->used_wisdom = wisdom != 0;
    diagnostics->used_model_fallback = wisdom == 0;
    copy_plan_diagnostics(diagnostics, *out);
    diagnostics->planning_seconds = mofft_monotonic_seconds() - start;
  }
  return status;
}

/* Reference chain validation (set_specific_factors, src/mofft.c:1060-1080). */
static mofft_status chain_from_radices(size_t length, const int *radices,
                                       size_t count, int *chain) {
  if (!radices || count == 0 || count > MOFFT_MAX_STAGES || length < 2)
    return MOFFT_INVALID_ARGUMENT;
  size_t remaining = length;
  for (size_t level = 0; level < count; ++level) {
    const int radix = radices[level];
    if (!mofft_is_supported_radix(radix) || remaining % (size_t)radix != 0)
      return MOFFT_INVALID_ARGUMENT;
    remaining /= (size_t)radix;
  }
  if (remaining != 1) return MOFFT_INVALID_ARGUMENT;
  for (size_t i = 0; i < count; ++i) chain[i] = radices[count - 1 - i];
  return MOFFT_SUCCESS;
}

static mofft_status create_with_radices(mofft_core **out, int precision_bits,
                                        size_t length, size_t batch,
                                        size_t distance,
                                        mofft_direction direction,
                                        mofft_placement placement,
                                        const int *radices, size_t count) {
  if (!valid_shape(direction, placement)) return MOFFT_INVALID_ARGUMENT;
  int chain[MOFFT_MAX_STAGES];
  mofft_status status = chain_from_radices(length, radices, count, chain);
  if (status != MOFFT_SUCCESS) return status;
  return mofft_core_create(out, precision_bits, length, batch, distance,
                           direction, placement, chain, (int)count);
}

/* ------------------------------------------------------------------------ */
/* setters (src/mofft.c:1492-1598)                                           */
/* ------------------------------------------------------------------------ */

static mofft_status set_transpose_strategy(mofft_core *c,
                                           mofft_transpose_strategy s) {
  if (!c || (s != MOFFT_TRANSPOSE_LINEAR && s != MOFFT_TRANSPOSE_BLOCKED))
    return MOFFT_INVALID_ARGUMENT;
  c->blocked_transpose_mask =
      s == MOFFT_TRANSPOSE_BLOCKED
          ? (c->depth <= 1 ? 0 : (UINT64_C(1) << (c->depth - 1)) - 1)
          : 0;
  return MOFFT_SUCCESS;
}

static mofft_status set_blocked_mask(mofft_core *c, uint64_t levels) {
  if (!c) return MOFFT_INVALID_ARGUMENT;
  const int transpose_count = c->depth > 1 ? c->depth - 1 : 0;
  if (transpose_count < 64 && (levels >> transpose_count)) return MOFFT_INVALID_ARGUMENT;
  c->blocked_transpose_mask = levels;
  return MOFFT_SUCCESS;
}

static mofft_status set_direct_input(mofft_core *c, int enabled) {
  if (!c || (enabled != 0 && enabled != 1)) return MOFFT_INVALID_ARGUMENT;
  c->direct_input = enabled;
  return MOFFT_SUCCESS;
}

static mofft_status set_stage_layout(mofft_core *c, mofft_stage_layout layout) {
  if (!c || (layout != MOFFT_STAGE_LAYOUT_TRANSPOSE &&
             layout != MOFFT_STAGE_LAYOUT_SECTION))
    return MOFFT_INVALID_ARGUMENT;
  c->stage_layout = layout;
  return MOFFT_SUCCESS;
}

static mofft_status set_kernel_bank(mofft_core *c, unsigned bank) {
  if (!c || bank >= MOFFT_KERNEL_BANK_COUNT) return MOFFT_INVALID_ARGUMENT;
  if (bank == c->kernel_bank) return MOFFT_SUCCESS;
  const unsigned old = c->kernel_bank;
  c->kernel_bank = bank;
  int saved = -1;
  cudaGetDevice(&saved);
  if (saved != c->device) cudaSetDevice(c->device);
  mofft_status st = mofft_core_build(c);
  if (st != MOFFT_SUCCESS) {
    c->kernel_bank = old;
    if (mofft_core_build(c) != MOFFT_SUCCESS) st = MOFFT_INTERNAL_ERROR;
  }
  if (saved >= 0 && saved != c->device) cudaSetDevice(saved);
  return st;
}

/* Precision forms (FP32 plans only): tensor-core forms swap the schedule for
 * one tensor-core kernel; on failure the previous form is rebuilt. */
mofft_status mofft_plan_set_precision_form_f32(mofft_plan_f32 *plan,
                                               mofft_precision_form form) {
  if (!plan || (form != MOFFT_FORM_FP32 && form != MOFFT_FORM_TF32X3 &&
                form != MOFFT_FORM_BF16X3))
    return MOFFT_INVALID_ARGUMENT;
  mofft_core *c = &plan->core;
  if ((int)form == c->form) return MOFFT_SUCCESS;
  const int old = c->form;
  c->form = (int)form;
  int saved = -1;
  cudaGetDevice(&saved);
  if (saved != c->device) cudaSetDevice(c->device);
  mofft_status st = mofft_core_build(c);
  if (st != MOFFT_SUCCESS) {
    c->form = old;
    if (mofft_core_build(c) != MOFFT_SUCCESS) st = MOFFT_INTERNAL_ERROR;
  }
  if (saved >= 0 && saved != c->device) cudaSetDevice(saved);
  return st;
}

mofft_status mofft_plan_get_precision_form_f32(const mofft_plan_f32 *plan,
                                               mofft_precision_form *form) {
  if (!plan || !form) return MOFFT_INVALID_ARGUMENT;
  *form = (mofft_precision_form)plan->core.form;
  return MOFFT_SUCCESS;
}

mofft_status mofft_plan_check_lost_copy_f32(mofft_plan_f32 *plan,
                                            const mofft_complex_f32 *input,
                                            mofft_complex_f32 *output) {
  if (!plan || !input || !output) return MOFFT_INVALID_ARGUMENT;
  mofft_core *c = &plan->core;
  int saved = -1;
  cudaGetDevice(&saved);
  if (saved != c->device) cudaSetDevice(c->device);
  const mofft_status st = mofft_core_check_lost_copy(c, input, output);
  if (saved >= 0 && saved != c->device) cudaSetDevice(saved);
  return st;
}

mofft_status mofft_plan_check_f32(mofft_plan_f32 *plan) {
  if (!plan) return MOFFT_INVALID_ARGUMENT;
  mofft_core *c = &plan->core;
  int saved = -1;
  cudaGetDevice(&saved);
  if (saved != c->device) cudaSetDevice(c->device);
  void *stream = c->user_stream ? c->user_stream : c->stream;
  mofft_status st = MOFFT_SUCCESS;
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) {
    cudaGetLastError();
    st = MOFFT_INTERNAL_ERROR;
  }
  if (st == MOFFT_SUCCESS) st = mofft_core_check_status(c);
  if (saved >= 0 && saved != c->device) cudaSetDevice(saved);
  return st;
}

/* ------------------------------------------------------------------------ */
/* recipes (format of src/mofft.c:1760-1842, GPU family in the CPU slot)     */
/* ------------------------------------------------------------------------ */

const char *mofft_build_id(void) { return MOFFT_BINARY_ID; }

static mofft_status import_core(mofft_core **out, int precision_bits,
                                const char *recipe, size_t size,
                                mofft_plan_diagnostics *diagnostics) {
  if (diagnostics) memset(diagnostics, 0, sizeof(*diagnostics));
  mofft_recipe f;
  mofft_status st = mofft_recipe_read(recipe, size, precision_bits, &f);
  if (st != MOFFT_SUCCESS) return st;
  st = create_with_radices(out, precision_bits, f.length, 1, 0, f.direction,
                           f.placement, f.radices, f.depth);
  if (st != MOFFT_SUCCESS) return st;
  st = set_blocked_mask(*out, f.mask);
  if (st == MOFFT_SUCCESS) st = set_direct_input(*out, f.direct_input);
  if (st == MOFFT_SUCCESS) st = set_stage_layout(*out, f.layout);
  if (st == MOFFT_SUCCESS) st = set_kernel_bank(*out, f.bank);
  if (st != MOFFT_SUCCESS) {
    mofft_core_destroy(*out);
    *out = NULL;
    return st;
  }
  if (diagnostics) {
    diagnostics->used_wisdom = 1;
    copy_plan_diagnostics(diagnostics, *out);
  }
  return MOFFT_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* typed entry points                                                        */
/* ------------------------------------------------------------------------ */

static int options_from_bound_flags(uint32_t flags, mofft_plan_options *o) {
  if ((flags & ~((uint32_t)MOFFT_FLAG_MEASURE | (uint32_t)MOFFT_FLAG_WISDOM_ONLY)) != 0 ||
      ((flags & MOFFT_FLAG_MEASURE) && (flags & MOFFT_FLAG_WISDOM_ONLY)))
    return 0;
  mofft_plan_options_init(o);
  o->mode = (flags & MOFFT_FLAG_MEASURE) ? MOFFT_PLANNER_MEASURE : MOFFT_PLANNER_PRETUNED;
  if (flags & MOFFT_FLAG_WISDOM_ONLY) o->flags |= MOFFT_PLAN_STRICT_WISDOM;
  return 1;
}

#define CORE(p) (&(p)->core)

/* Plan whose schedule runs exactly `kernels` (registry indices, one per pass,
 * first pass first); the kernels' in-CTA radix lists, concatenated, are the
 * plan's chain. */
static mofft_status create_with_kernels(mofft_core **out, int precision_bits,
                                        size_t length, size_t batch, size_t distance,
                                        mofft_direction direction,
                                        mofft_placement placement, const int *kernels,
                                        size_t count) {
  if (!kernels || count == 0 || count > MOFFT_MAX_PASSES || !valid_shape(direction, placement))
    return MOFFT_INVALID_ARGUMENT;
  int chain[MOFFT_MAX_STAGES];
  int preferred[MOFFT_MAX_PASSES];
  int depth = 0;
  size_t product = 1;
  for (int i = 0; i < MOFFT_MAX_PASSES; ++i) preferred[i] = -1;
  for (size_t p = 0; p < count; ++p) {
    const mofft_kernel_desc *d = mofft_cuda_kernel_get(kernels[p]);
    if (!d || d->precision_bits != precision_bits ||
        d->kind != (count == 1 ? MOFFT_KERNEL_ROWS : MOFFT_KERNEL_COLS) ||
        d->radix_count <= 0 || depth + d->radix_count > MOFFT_MAX_STAGES)
      return MOFFT_INVALID_ARGUMENT;
    memcpy(chain + depth, d->radices, (size_t)d->radix_count * sizeof(int));
    depth += d->radix_count;
    product *= (size_t)d->length;
    preferred[p] = kernels[p];
  }
  if (product != length) return MOFFT_INVALID_ARGUMENT;
  if (!mofft_hardware_supports(precision_bits)) return MOFFT_UNSUPPORTED_HARDWARE;
  mofft_status st = mofft_core_create_tuned(out, precision_bits, length, batch, distance,
                                            direction, placement, chain, depth, preferred);
  if (st != MOFFT_SUCCESS) return st;
  const mofft_core *c = *out;
  int ok = c->sched.pass_count == (int)count;
  for (size_t p = 0; ok && p < count; ++p) ok = c->sched.pass[p].kernel == kernels[p];
  if (!ok) {
    mofft_core_destroy(*out);
    *out = NULL;
    return MOFFT_UNSUPPORTED_SIZE;
  }
  return MOFFT_SUCCESS;
}

#define DEFINE_TYPED_API(SUF, BITS, PLAN, CPLX)                                  \
  mofft_status mofft_plan_create_##SUF(PLAN **out, size_t length,                \
                                       mofft_direction direction,                \
                                       mofft_placement placement) {              \
    if (!out || !valid_shape(direction, placement)) return MOFFT_INVALID_ARGUMENT; \
    *out = NULL;                                                                 \
    int chain[MOFFT_MAX_STAGES];                                                 \
    int preferred[MOFFT_MAX_PASSES];                                             \
    const int wisdom = mofft_wisdom_lookup(length, BITS, chain, MOFFT_MAX_STAGES, \
                                           preferred);                           \
    return mofft_core_create_tuned((mofft_core **)out, BITS, length, 1, 0,       \
                                   direction, placement, wisdom ? chain : NULL,  \
                                   wisdom, preferred);                           \
  }                                                                              \
  mofft_status mofft_plan_create_with_options_##SUF(                             \
      PLAN **out, size_t length, mofft_direction direction,                      \
      mofft_placement placement, const mofft_plan_options *options,              \
      mofft_plan_diagnostics *diagnostics) {                                     \
    if (!out) return MOFFT_INVALID_ARGUMENT;                                     \
    *out = NULL;                                                                 \
    return create_with_options((mofft_core **)out, BITS, length, 1, 0,          \
                               direction, placement, options, diagnostics);     \
  }                                                                              \
  mofft_status mofft_plan_create_batched_##SUF(                                  \
      PLAN **out, size_t length, size_t batch, size_t distance,                  \
      mofft_direction direction, mofft_placement placement,                      \
      const mofft_plan_options *options, mofft_plan_diagnostics *diagnostics) {  \
    if (!out) return MOFFT_INVALID_ARGUMENT;                                     \
    *out = NULL;                                                                 \
    if (diagnostics) memset(diagnostics, 0, sizeof(*diagnostics));              \
    if (batch == 0 || (distance != 0 && distance < length))                      \
      return MOFFT_INVALID_ARGUMENT;                                             \
    return create_with_options((mofft_core **)out, BITS, length, batch,         \
                               distance, direction, placement, options,          \
                               diagnostics);                                     \
  }                                                                              \
  mofft_status mofft_plan_create_with_radices_##SUF(                             \
      PLAN **out, size_t length, mofft_direction direction,                      \
      mofft_placement placement, const int *radices, size_t radix_count) {      \
    if (!out) return MOFFT_INVALID_ARGUMENT;                                     \
    *out = NULL;                                                                 \
    return create_with_radices((mofft_core **)out, BITS, length, 1, 0,          \
                               direction, placement, radices, radix_count);     \
  }                                                                              \
  mofft_status mofft_plan_create_batched_with_radices_##SUF(                     \
      PLAN **out, size_t length, size_t batch, size_t distance,                  \
      mofft_direction direction, mofft_placement placement,                      \
      const int *radices, size_t radix_count) {                                  \
    if (!out) return MOFFT_INVALID_ARGUMENT;                                     \
    *out = NULL;                                                                 \
    if (batch == 0 || (distance != 0 && distance < length))                      \
      return MOFFT_INVALID_ARGUMENT;                                             \
    return create_with_radices((mofft_core **)out, BITS, length, batch,         \
                               distance, direction, placement, radices,          \
                               radix_count);                                     \
  }                                                                              \
  mofft_status mofft_plan_create_batched_with_kernels_##SUF(                     \
      PLAN **out, size_t length, size_t batch, size_t distance,                  \
      mofft_direction direction, mofft_placement placement,                      \
      const int *kernels, size_t count) {                                        \
    if (!out) return MOFFT_INVALID_ARGUMENT;                                     \
    *out = NULL;                                                                 \
    if (batch == 0 || (distance != 0 && distance < length))                      \
      return MOFFT_INVALID_ARGUMENT;                                             \
    return create_with_kernels((mofft_core **)out, BITS, length, batch,         \
                               distance, direction, placement, kernels, count);  \
  }                                                                              \
  PLAN *mofft_plan_dft_1d_##SUF(size_t length, const CPLX *input, CPLX *output,  \
                                mofft_direction direction, uint32_t flags) {     \
    if (!input || !output) return NULL;                                          \
    mofft_plan_options options;                                                  \
    if (!options_from_bound_flags(flags, &options)) return NULL;                 \
    PLAN *plan = NULL;                                                           \
    const mofft_placement placement =                                            \
        input == output ? MOFFT_IN_PLACE : MOFFT_OUT_OF_PLACE;                   \
    if (mofft_plan_create_with_options_##SUF(&plan, length, direction,           \
                                             placement, &options, NULL) !=       \
        MOFFT_SUCCESS)                                                           \
      return NULL;                                                               \
    plan->core.bound_input = input;                                              \
    plan->core.bound_output = output;                                            \
    plan->core.has_bound_arrays = 1;                                             \
    return plan;                                                                 \
  }                                                                              \
  mofft_status mofft_execute_plan_##SUF(const PLAN *plan) {                      \
    if (!plan || !plan->core.has_bound_arrays) return MOFFT_INVALID_ARGUMENT;    \
    return mofft_core_execute(CORE(plan), plan->core.bound_input,                \
                              plan->core.bound_output);                          \
  }                                                                              \
  mofft_status mofft_execute_##SUF(const PLAN *plan, const CPLX *input,          \
                                   CPLX *output) {                               \
    if (!plan || !input || !output) return MOFFT_INVALID_ARGUMENT;               \
    return mofft_core_execute(CORE(plan), input, output);                        \
  }                                                                              \
  void mofft_plan_destroy_##SUF(PLAN *plan) {                                    \
    if (plan) mofft_core_destroy(CORE(plan));                                    \
  }                                                                              \
  mofft_status mofft_plan_set_transpose_strategy_##SUF(                          \
      PLAN *plan, mofft_transpose_strategy strategy) {                           \
    return set_transpose_strategy(plan ? CORE(plan) : NULL, strategy);           \
  }                                                                              \
  mofft_status mofft_plan_set_blocked_transpose_mask_##SUF(PLAN *plan,           \
                                                           uint64_t levels) {    \
    return set_blocked_mask(plan ? CORE(plan) : NULL, levels);                   \
  }                                                                              \
  mofft_status mofft_plan_set_direct_input_##SUF(PLAN *plan, int enabled) {      \
    return set_direct_input(plan ? CORE(plan) : NULL, enabled);                  \
  }                                                                              \
  mofft_status mofft_plan_set_stage_layout_##SUF(PLAN *plan,                     \
                                                 mofft_stage_layout layout) {    \
    return set_stage_layout(plan ? CORE(plan) : NULL, layout);                   \
  }                                                                              \
  mofft_status mofft_plan_set_kernel_bank_##SUF(PLAN *plan, unsigned int bank) { \
    return set_kernel_bank(plan ? CORE(plan) : NULL, bank);                      \
  }                                                                              \
  mofft_status mofft_plan_get_kernel_bank_##SUF(const PLAN *plan,                \
                                                unsigned int *bank) {            \
    if (!plan || !bank) return MOFFT_INVALID_ARGUMENT;                           \
    *bank = plan->core.kernel_bank;                                              \
    return MOFFT_SUCCESS;                                                        \
  }                                                                              \
  mofft_status mofft_plan_export_##SUF(const PLAN *plan, char *buffer,           \
                                       size_t capacity, size_t *required) {      \
    return mofft_recipe_write(plan ? CORE(plan) : NULL, buffer, capacity,       \
                              required);                                         \
  }                                                                              \
  mofft_status mofft_plan_import_##SUF(PLAN **out, const char *recipe,           \
                                       size_t recipe_size,                       \
                                       mofft_plan_diagnostics *diagnostics) {    \
    if (!out) return MOFFT_INVALID_ARGUMENT;                                     \
    *out = NULL;                                                                 \
    return import_core((mofft_core **)out, BITS, recipe, recipe_size,           \
                       diagnostics);                                             \
  }                                                                              \
  mofft_status mofft_plan_set_stream_##SUF(PLAN *plan, void *stream) {           \
    if (!plan) return MOFFT_INVALID_ARGUMENT;                                    \
    plan->core.user_stream = stream;                                             \
    return MOFFT_SUCCESS;                                                        \
  }                                                                              \
  mofft_status mofft_plan_get_batch_##SUF(const PLAN *plan, size_t *batch,       \
                                          size_t *distance) {                    \
    if (!plan || !batch || !distance) return MOFFT_INVALID_ARGUMENT;             \
    *batch = plan->core.batch;                                                   \
    *distance = plan->core.distance;                                             \
    return MOFFT_SUCCESS;                                                        \
  }                                                                              \
  mofft_status mofft_plan_get_schedule_##SUF(const PLAN *plan,                   \
                                             mofft_plan_schedule *s) {           \
    if (!plan || !s) return MOFFT_INVALID_ARGUMENT;                              \
    memset(s, 0, sizeof(*s));                                                    \
    const mofft_core *c = CORE(plan);                                            \
    s->pass_count = c->sched.pass_count;                                         \
    for (int p = 0; p < c->sched.pass_count && p < 4; ++p) {                     \
      s->lengths[p] = c->sched.pass[p].length;                                   \
      s->kernels[p] = c->sched.pass[p].kernel;                                   \
      s->smem_bytes[p] = c->sched.pass[p].smem_bytes;                            \
    }                                                                            \
    s->workspace_bytes = c->work_bytes;                                          \
    s->twiddle_bytes = c->twiddle_bytes;                                         \
    return MOFFT_SUCCESS;                                                        \
  }                                                                              \
  mofft_status mofft_plan_get_measure_report_##SUF(const PLAN *plan,             \
                                                   mofft_measure_report *r) {    \
    if (!plan || !r || !plan->core.measured) return MOFFT_INVALID_ARGUMENT;      \
    const mofft_core *c = CORE(plan);                                            \
    r->candidates = c->measure_candidates;                                       \
    r->winner_model_rank = c->measure_winner_model_rank;                         \
    r->model_first_measured_rank = c->measure_model_first_rank;                  \
    r->winner_seconds = c->measure_winner_seconds;                               \
    r->winner_model_seconds = c->measure_winner_model_seconds;                   \
    return MOFFT_SUCCESS;                                                        \
  }

DEFINE_TYPED_API(f32, 32, mofft_plan_f32, mofft_complex_f32)
DEFINE_TYPED_API(f64, 64, mofft_plan_f64, mofft_complex_f64)
#undef DEFINE_TYPED_API

/* ------------------------------------------------------------------------ */
/* misc                                                                      */
/* ------------------------------------------------------------------------ */

const char *mofft_status_string(mofft_status status) {
  switch (status) {
    case MOFFT_SUCCESS: return "success";
    case MOFFT_INVALID_ARGUMENT: return "invalid argument";
    case MOFFT_UNSUPPORTED_SIZE: return "unsupported size";
    case MOFFT_ALLOCATION_FAILURE: return "allocation failure";
    case MOFFT_UNSUPPORTED_HARDWARE: return "unsupported hardware";
    case MOFFT_INTERNAL_ERROR: return "internal error";
    case MOFFT_WISDOM_NOT_FOUND: return "compiled wisdom not found";
    case MOFFT_INCOMPATIBLE_RECIPE: return "incompatible plan recipe";
    case MOFFT_BUFFER_TOO_SMALL: return "output buffer too small";
    default: return "unknown status";
  }
}

const char *mofft_version(void) { return "0.4.0"; }

int mofft_kernel_count(void) { return mofft_cuda_kernel_count(); }

int mofft_kernel_info(int index, char *name, size_t capacity,
                      int *precision_bits, int *kind, int *length, int *lines,
                      int *threads, int *radix_count, int *radices) {
  const mofft_kernel_desc *d = mofft_cuda_kernel_get(index);
  if (!d) return -1;
  if (name && capacity) {
    strncpy(name, d->name, capacity - 1);
    name[capacity - 1] = '\0';
  }
  if (precision_bits) *precision_bits = d->precision_bits;
  if (kind) *kind = d->kind;
  if (length) *length = d->length;
  if (lines) *lines = d->lines;
  if (threads) *threads = d->threads;
  if (radix_count) *radix_count = d->radix_count;
  if (radices)
    for (int i = 0; i < 8; ++i) radices[i] = d->radices[i];
  return 0;
}
