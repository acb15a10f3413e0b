/* Internal declarations shared by the C host library's translation units. */
#ifndef MOFFT_INTERNAL_H
#define MOFFT_INTERNAL_H

#include <pthread.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/mofft.h"
#include "../../include/mofft_b200.h"
#include "mofft_cuda.h"

#define MOFFT_MAX_PASSES 4
#define MOFFT_MAX_STAGES 64

/* One kernel launch of a plan's schedule. */
typedef struct {
  int kernel;               /* registry index */
  int kind;                 /* mofft_kernel_kind of that entry */
  int length;               /* line length L of this pass */
  int lines;                /* lines per CTA (generic kernel) */
  int radix_count;          /* in-CTA stages of this pass */
  int radices[MOFFT_CUDA_MAX_STAGES];
  long long ns_outer;       /* product of earlier passes' lengths */
  int split_shift;          /* two-level super twiddle split */
  size_t tw_offset;         /* byte offsets into the plan's twiddle buffer */
  size_t tw_hi_offset;
  size_t tw_lo_offset;
  size_t smem_bytes;
  size_t aux_offset;        /* tensor-core passes: B operand tiles */
  size_t status_offset;     /* tensor-core passes: error word */
} mofft_pass;

typedef struct {
  int pass_count;
  mofft_pass pass[MOFFT_MAX_PASSES];
} mofft_schedule;

typedef struct mofft_core {
  /* reference-visible plan state (src/mofft.c:43-61) */
  size_t length;
  int direction;
  mofft_placement placement;
  int precision_bits;
  int depth;                            /* radix chain length */
  int factors[MOFFT_MAX_STAGES];        /* outermost first */
  uint64_t blocked_transpose_mask;
  int direct_input;
  mofft_stage_layout stage_layout;
  unsigned int kernel_bank;
  /* Tuned kernel instances (registry indices, -1 = none) that the pass
   * grouping prefers over the first matching instance: the autotuner's and
   * the compiled wisdom's choice among variants of the same radix chain. */
  int preferred[MOFFT_MAX_PASSES];
  const void *bound_input;
  void *bound_output;
  int has_bound_arrays;
  /* precision form (mofft_precision_form); tensor-core forms replace the
   * schedule with one tensor-core kernel and keep factors[] as they were */
  int form;
  /* batched extension */
  size_t batch;
  size_t distance;
  /* device state */
  int device;
  mofft_schedule sched;
  void *d_twiddles;
  size_t twiddle_bytes;
  void *d_work;
  size_t work_bytes;
  void *stream;            /* plan-owned cudaStream_t */
  void *user_stream;       /* attached cudaStream_t, or NULL */
  void *d_stage[2];        /* host-pointer staging buffers (lazy) */
  void *stream3;           /* download stream of the host-buffer pipeline */
  void *ev_up[64];         /* per-chunk events: upload done, passes done */
  void *ev_done[64];
  void *stream2;           /* second plan-owned stream of the host-buffer
                              pipeline (lazy) */
  size_t stage_bytes;
  pthread_mutex_t lock;
  /* MEASURE plans: how the model's order compared with the timings */
  int measured;
  size_t measure_candidates;
  size_t measure_winner_model_rank;     /* 1-based, in model order */
  size_t measure_model_first_rank;      /* measured rank of the model's pick */
  double measure_winner_seconds;
  double measure_winner_model_seconds;
} mofft_core;

struct mofft_plan_f32 { mofft_core core; };
struct mofft_plan_f64 { mofft_core core; };

#endif
