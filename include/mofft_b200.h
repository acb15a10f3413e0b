/* B200 extensions to the MoFFT C API (no counterpart in the reference, which
 * computes one transform per call on one CPU core).
 *
 *  - Batched plans: `batch` transforms of `length` points, transform b starting
 *    at element b*distance of the buffer (distance >= length; 0 = length).
 *    mofft_execute_f32/f64 then processes the whole batch.
 *  - Streams: attaching a cudaStream_t makes mofft_execute_* asynchronous on
 *    that stream (device buffers only); NULL restores blocking behaviour.
 *  - Kernel introspection for tests, the autotuner and the benchmark.
 */
#ifndef MOFFT_B200_H
#define MOFFT_B200_H

#include "mofft.h"

#ifdef __cplusplus
extern "C" {
#endif

mofft_status mofft_plan_create_batched_f32(
    mofft_plan_f32 **plan, size_t length, size_t batch, size_t distance,
    mofft_direction direction, mofft_placement placement,
    const mofft_plan_options *options, mofft_plan_diagnostics *diagnostics);
mofft_status mofft_plan_create_batched_f64(
    mofft_plan_f64 **plan, size_t length, size_t batch, size_t distance,
    mofft_direction direction, mofft_placement placement,
    const mofft_plan_options *options, mofft_plan_diagnostics *diagnostics);

/* Batched plan with an explicit radix chain (outermost first). */
mofft_status mofft_plan_create_batched_with_radices_f32(
    mofft_plan_f32 **plan, size_t length, size_t batch, size_t distance,
    mofft_direction direction, mofft_placement placement, const int *radices,
    size_t radix_count);
mofft_status mofft_plan_create_batched_with_radices_f64(
    mofft_plan_f64 **plan, size_t length, size_t batch, size_t distance,
    mofft_direction direction, mofft_placement placement, const int *radices,
    size_t radix_count);

/* Batched plan with an explicit kernel per pass: `kernels` holds `count`
 * registry indices (mofft_kernel_info), first pass first -- one one-pass
 * (kind 0) kernel, or two to four column-pass (kind 1) kernels whose line
 * lengths multiply to `length`.  The plan runs exactly those kernels (the
 * tuned variants the autotuner chooses between, e.g. for tests or for
 * replaying a measurement); the kernels' radix lists form the plan's chain.
 * MOFFT_INVALID_ARGUMENT for kernels that do not form such a schedule,
 * MOFFT_UNSUPPORTED_SIZE if the schedule cannot be built. */
mofft_status mofft_plan_create_batched_with_kernels_f32(
    mofft_plan_f32 **plan, size_t length, size_t batch, size_t distance,
    mofft_direction direction, mofft_placement placement, const int *kernels,
    size_t count);
mofft_status mofft_plan_create_batched_with_kernels_f64(
    mofft_plan_f64 **plan, size_t length, size_t batch, size_t distance,
    mofft_direction direction, mofft_placement placement, const int *kernels,
    size_t count);

/* `stream` is a cudaStream_t (NULL = blocking calls on a plan-owned stream). */
mofft_status mofft_plan_set_stream_f32(mofft_plan_f32 *plan, void *stream);
mofft_status mofft_plan_set_stream_f64(mofft_plan_f64 *plan, void *stream);

/* Number of transforms and element distance of a plan. */
mofft_status mofft_plan_get_batch_f32(const mofft_plan_f32 *plan,
                                      size_t *batch, size_t *distance);
mofft_status mofft_plan_get_batch_f64(const mofft_plan_f64 *plan,
                                      size_t *batch, size_t *distance);

/* GPU schedule of a plan: number of passes (kernel launches per execute) and,
 * per pass, the line length, registry kernel index and shared memory bytes. */
typedef struct {
  int pass_count;
  int lengths[4];
  int kernels[4];
  size_t smem_bytes[4];
  size_t workspace_bytes;     /* device workspace owned by the plan */
  size_t twiddle_bytes;       /* device twiddle tables owned by the plan */
} mofft_plan_schedule;
mofft_status mofft_plan_get_schedule_f32(const mofft_plan_f32 *plan,
                                         mofft_plan_schedule *schedule);
mofft_status mofft_plan_get_schedule_f64(const mofft_plan_f64 *plan,
                                         mofft_plan_schedule *schedule);

/* The schedule the planner builds for (precision, length, radix chain or
 * NULL for the PRETUNED model, kernel bank), computed on the host without a
 * GPU.  chain_out (64 entries, may be NULL) receives the radix chain,
 * outermost first. */
mofft_status mofft_schedule_preview(int precision_bits, size_t length,
                                    const int *radices, size_t radix_count,
                                    unsigned int bank,
                                    mofft_plan_schedule *schedule,
                                    int *chain_out, size_t *chain_count);

/* How the MEASURE planner's model order compared with its timings (no
 * counterpart in the reference, whose diagnostics report only the winner):
 * the number of schedules timed, the model rank of the fastest one (1 = the
 * model's first choice was fastest), the measured rank of the model's first
 * choice, the winner's median time and the model's prediction for it.
 * MOFFT_INVALID_ARGUMENT for a plan that was not measured. */
typedef struct {
  size_t candidates;
  size_t winner_model_rank;
  size_t model_first_measured_rank;
  double winner_seconds;
  double winner_model_seconds;
} mofft_measure_report;
mofft_status mofft_plan_get_measure_report_f32(const mofft_plan_f32 *plan,
                                               mofft_measure_report *report);
mofft_status mofft_plan_get_measure_report_f64(const mofft_plan_f64 *plan,
                                               mofft_measure_report *report);

/* Device-time model of the schedule that runs `kernels` (registry indices,
 * one per pass, first pass first) over `batch` transforms of `length`, in
 * seconds, computed on the host without a GPU; DBL_MAX when the kernels do
 * not form a schedule of that length.  The planner's prior, as the
 * reference's cost model is (src/mofft.c:327-351 ranks factorizations,
 * :874-922 shortlists MEASURE candidates): PRETUNED plans pick among the
 * splits of their pass count by it, MEASURE times candidates in its order. */
double mofft_schedule_model_seconds(int precision_bits, size_t length, size_t batch,
                                    const int *kernels, size_t pass_count);

/* Ragged batches (no counterpart in the reference): many FP32 transforms of
 * different lengths, batch sizes and directions in one CUDA graph.  Items
 * hold device buffers (input == output runs in place).  Items of the lengths
 * one persistent kernel runs in one pass (2^6 .. 2^13, 3*2^5 .. 3*2^11) are
 * tiles of its work-descriptor queue (one launch for all of them); the other
 * items are grouped by (length, direction), and each group runs its tuned
 * schedule (compiled wisdom, else the model) once over all its transforms
 * through pointer tables, one launch per pass, on parallel graph branches
 * next to the persistent launch.  A group whose schedule does not run through
 * tables (more than two passes, a runtime-stage kernel) joins the persistent
 * queue as two-pass tiles, which take products of two column lengths in
 * {96, 128, 192, 256}; other lengths give MOFFT_UNSUPPORTED_SIZE.
 * mofft_ragged_plan_create_single_launch_f32 puts every item into the
 * persistent queue (one launch in all).
 * mofft_ragged_execute enqueues the whole batch on `stream` (a
 * cudaStream_t); mofft_ragged_status (blocking) reports whether the last
 * execution completed every tile and every bounded wait of the groups'
 * kernels.  mofft_ragged_execute_per_item runs the same items as one
 * ordinary batched plan each (the comparison point). */
typedef struct mofft_ragged_plan mofft_ragged_plan;
typedef struct {
  size_t length;
  size_t batch;
  mofft_direction direction;
  const void *input;   /* device, batch * length complex64, dense */
  void *output;
} mofft_ragged_item;
mofft_status mofft_ragged_plan_create_f32(mofft_ragged_plan **plan,
                                          const mofft_ragged_item *items,
                                          size_t count);
mofft_status mofft_ragged_plan_create_single_launch_f32(mofft_ragged_plan **plan,
                                                        const mofft_ragged_item *items,
                                                        size_t count);
mofft_status mofft_ragged_execute(mofft_ragged_plan *plan, void *stream);
mofft_status mofft_ragged_execute_per_item(mofft_ragged_plan *plan,
                                           void *stream);
mofft_status mofft_ragged_status(mofft_ragged_plan *plan);
/* Failure check: runs the plan's persistent queue once on `stream` with
 * every second-pass dependency made unsatisfiable, so each second-pass tile
 * gives up after its bounded wait (about a second per tile and CTA) and skips
 * its work; mofft_ragged_status then reports MOFFT_INTERNAL_ERROR and the
 * next mofft_ragged_execute runs normally.  Plans without two-pass tiles
 * (every plan whose long items all run as tuned groups) have no waits and
 * report success.  For tests of the timeout path. */
mofft_status mofft_ragged_check_lost_dependency(mofft_ragged_plan *plan,
                                                void *stream);
mofft_status mofft_ragged_plan_info(const mofft_ragged_plan *plan,
                                    size_t *tiles, int *grid);
void mofft_ragged_plan_destroy(mofft_ragged_plan *plan);

/* Allocation-free execution (no counterpart in the reference).
 *
 * For callers that cannot allocate device memory: code embedded in a host
 * framework that reserves the whole GPU memory budget up front and forbids
 * further cudaMalloc calls, and latency-critical loops where a cudaMalloc /
 * cudaFree (which may synchronize the device) is not acceptable.  Plans
 * allocate at creation; this call allocates nothing.  It runs a batched FP32
 * transform whose schedule has two passes (four-step: lengths beyond one
 * CTA's shared memory, e.g. 2^15..2^22) from the device buffer `input` to
 * the device buffer `output` (they may be equal), enqueued on `stream` (a
 * cudaStream_t, NULL for the default stream); the call returns without
 * waiting.  The intermediate array and its twiddle tables live in a static
 * device array of MOFFT_FIXED_SCRATCH_POINTS complex values (32 MiB plus 512
 * KiB of twiddles) that every GPU loading the library holds until exit.
 *
 * It runs the compiled wisdom's tuned schedule of the length when that has
 * two passes (the kernels an out-of-place PRETUNED plan runs), else the
 * model's schedule when that has two.
 *
 * Limits: batch * length <= MOFFT_FIXED_SCRATCH_POINTS, else
 * MOFFT_UNSUPPORTED_SIZE; lengths that run in one pass (they need no scratch)
 * and lengths with neither a tuned nor a model two-pass schedule, also
 * MOFFT_UNSUPPORTED_SIZE; host buffers give MOFFT_INVALID_ARGUMENT.  The first call on each device sets up the array's
 * device address (with that device current), so make that first call before
 * any stream capture on that device.  All calls share the array and it keeps
 * the last call's contents; calls whose executions overlap on the GPU race on
 * it, so order them (for example on one stream). */
#define MOFFT_FIXED_SCRATCH_POINTS (1u << 22)
mofft_status mofft_execute_fixed_scratch_f32(const mofft_complex_f32 *input,
                                             mofft_complex_f32 *output,
                                             size_t length, size_t batch,
                                             mofft_direction direction,
                                             void *stream);

/* Precision forms of FP32 plans (no counterpart in the reference, whose
 * transforms run in the plan's own precision on the CPU cores).
 *
 *   MOFFT_FORM_FP32    FP32 butterflies on the CUDA cores (the default).
 *   MOFFT_FORM_TF32X3  the radix-16 stages (three for n = 4096, four in two
 *                      column passes for n = 65536) as DFT-matrix
 *                      GEMMs on the tensor cores; every operand x is split
 *                      into TF32 terms hi + lo and each product is
 *                      lo*hi + hi*lo + hi*hi, accumulated in FP32 (about 21
 *                      significant bits per product).
 *   MOFFT_FORM_BF16X3  the same with BF16 terms (about 16 bits).
 *
 * Tensor-core forms exist for FP32 plans of length 4096 and 65536 (others:
 * MOFFT_UNSUPPORTED_SIZE, the plan keeps its form); they run direct batches
 * (not the serving engine's pointer tables).  Twiddle multiplications and
 * the shuffles between stages stay FP32 on the CUDA cores.  The kernel bounds
 * every wait on the tensor core: a wait that timed out makes the blocking
 * execute return MOFFT_INTERNAL_ERROR; with an attached stream,
 * mofft_plan_check_f32 (blocking) reports it.  Recipes record the FP32
 * schedule; the form is not part of a recipe. */
typedef enum {
  MOFFT_FORM_FP32 = 0,
  MOFFT_FORM_TF32X3 = 1,
  MOFFT_FORM_BF16X3 = 2
} mofft_precision_form;
/* The form can also be chosen at creation: these bits of
 * mofft_plan_options.flags (PRETUNED mode, FP32 plans; at most one of them)
 * create the plan with that form.  With an FP64 plan, with MEASURE or with
 * both bits the options are MOFFT_INVALID_ARGUMENT; a length without a
 * tensor-core kernel gives MOFFT_UNSUPPORTED_SIZE. */
enum {
  MOFFT_PLAN_FORM_TF32X3 = 1u << 8,
  MOFFT_PLAN_FORM_BF16X3 = 1u << 9
};
mofft_status mofft_plan_set_precision_form_f32(mofft_plan_f32 *plan,
                                               mofft_precision_form form);
mofft_status mofft_plan_get_precision_form_f32(const mofft_plan_f32 *plan,
                                               mofft_precision_form *form);
/* Synchronizes the plan's stream and reports MOFFT_INTERNAL_ERROR when a
 * kernel of the plan that bounds its waits (the tensor-core kernels, the
 * prefetching one-pass kernel rows_float_16384_t512_b1_sfalse_dxp, the
 * thread-block-cluster kernels cluster_*) recorded a wait that ran out.
 * Blocking executes without an attached stream check this themselves. */
mofft_status mofft_plan_check_f32(mofft_plan_f32 *plan);
/* Failure check of a one-pass plan whose kernel bulk-copies its input: one
 * forward launch on device buffers `input` / `output` in which the first
 * input copy of every CTA is never issued, so each CTA's bounded wait runs
 * out (about a second).  The tensor-core n = 4096 kernel then frees its
 * tensor memory and returns, leaving `output` unspecified; the prefetching
 * one-pass kernel loads those lines itself, so `output` is still the forward
 * transform; in a cluster kernel CTA 0 of every cluster never sends its
 * tiles, so every CTA's wait for its tiles runs out and `output` is
 * unspecified.  Returns the status an execute would then report --
 * MOFFT_INTERNAL_ERROR when the timeout path works -- and clears the plan's
 * error word, so the plan stays usable.  MOFFT_INVALID_ARGUMENT for plans
 * that run neither kernel.  For tests of the timeout path. */
mofft_status mofft_plan_check_lost_copy_f32(mofft_plan_f32 *plan,
                                            const mofft_complex_f32 *input,
                                            mofft_complex_f32 *output);

/* Kernel registry introspection.  kind: 0 one-pass rows kernel, 1 column pass
 * of a multi-pass transform, 2 generic (runtime radix list), 3 tensor-core
 * precision form. */
int mofft_kernel_count(void);
/* Fills name (NUL-terminated, truncated to capacity) and shape of entry i;
 * returns 0 on success, -1 when i is out of range. */
int mofft_kernel_info(int index, char *name, size_t capacity,
                      int *precision_bits, int *kind, int *length, int *lines,
                      int *threads, int *radix_count, int *radices);
/* Kernel launches issued by this process so far (all plans). */
uint64_t mofft_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif
