/* Internal C-ABI between the C host library (mofft_api.c) and the CUDA
 * kernels (fft_kernels.cu).  Plain C types only: the host side never sees a
 * CUDA template.  A "pass" is one kernel launch over a batch; a plan is a
 * short list of passes (one for lengths that fit one CTA, two or three for
 * four-step / six-step). */
#ifndef MOFFT_CUDA_H
#define MOFFT_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MOFFT_CUDA_MAX_STAGES 24

typedef enum {
  MOFFT_KERNEL_ROWS = 0,    /* single pass, whole transforms per CTA */
  MOFFT_KERNEL_COLS = 1,    /* one pass of a multi-pass transform */
  MOFFT_KERNEL_GENERIC = 2, /* runtime stage list, ROWS or COLS addressing */
  MOFFT_KERNEL_TENSOR = 3,  /* whole transforms per CTA, DFT-matrix stages on
                               the tensor cores (a precision form) */
  MOFFT_KERNEL_TENSOR_COLS = 4  /* one column pass of a multi-pass transform,
                                   DFT-matrix stages on the tensor cores */
} mofft_kernel_kind;

typedef struct {
  const char *name;
  int precision_bits;   /* 32 or 64 */
  int kind;             /* mofft_kernel_kind */
  int length;           /* line length L; 0 for the generic kernel */
  int lines;            /* transforms (ROWS) or columns (COLS) per CTA */
  int threads;          /* threads per CTA */
  int staged;           /* ROWS: input/output staged through shared memory */
  int radix_count;      /* in-CTA Stockham stages, first to last */
  int radices[8];
  size_t smem_bytes;    /* dynamic shared memory per CTA */
  int form;             /* mofft_precision_form; 0 for the CUDA-core kernels */
  int prefetch;         /* ROWS: persistent CTAs that bulk-copy the next line
                           (the pass takes an error word, `status`) */
  int bank;             /* kernel bank whose codelets it runs: 0 default,
                           1 like-terms, 2 even-odd, 3 vector-reuse families
                           (runtime-stage kernels) */
  int cluster;          /* ROWS: CTAs of the thread-block cluster that computes
                           one transform (0: one CTA per transform) */
} mofft_kernel_desc;

typedef struct {
  const void *in;
  void *out;
  const void *tw;        /* internal stage twiddle table of the line DFT */
  const void *tw_hi;     /* super-stage twiddle (COLS, ns_outer > 1) */
  const void *tw_lo;
  long long batch;
  long long in_dist;     /* complex elements between batch entries */
  long long out_dist;
  long long total;       /* COLS: transform length M */
  long long ns_outer;    /* COLS: product of the earlier passes' lengths */
  int split_shift;       /* COLS: log2 of the two-level twiddle split */
  int conj_in;           /* 1: negate imaginary part on load */
  int conj_out;          /* 1: negate imaginary part on store */
  /* Indirect batch (device arrays of `batch` pointers, or NULL): transform b
   * of this pass reads in_table[b] and writes out_table[b] (specialised
   * kernels only). */
  const void *const *in_table;
  void *const *out_table;
  /* tensor-core kernels: constant B operand tiles and the error word the
   * kernel sets when a wait on the tensor core timed out; prefetching ROWS
   * kernels: the error word their line-copy waits set (may be NULL) */
  const void *aux;
  int *status;
  int lose_copy;         /* failure check: the kernel's first copy is never
                            issued, so its wait runs out (0 in normal use) */
  /* generic kernel only */
  int generic_cols;      /* 0 ROWS addressing, 1 COLS addressing */
  int length;            /* line length L */
  int lines;             /* lines per CTA */
  int radix_count;
  int radices[MOFFT_CUDA_MAX_STAGES];
} mofft_pass_args;

int mofft_cuda_kernel_count(void);
const mofft_kernel_desc *mofft_cuda_kernel_get(int index);
/* Dynamic shared memory the generic kernel needs for (L, lines, cols). */
size_t mofft_cuda_generic_smem(int precision_bits, int length, int lines,
                               int cols);
/* Opt every kernel into its shared-memory size on the current device.
 * Returns a cudaError_t value (0 = success). */
int mofft_cuda_prepare_device(void);
/* Bytes of the B operand tiles of a tensor-core precision form (0 if the
 * form has no tensor-core kernel), and their host-side construction from the
 * 16-point forward DFT matrix fr + i fi (row-major F[k][r]). */
size_t mofft_cuda_tensor_aux_bytes(int form);
int mofft_cuda_tensor_fill_aux(int form, void *dst, const double *fr,
                               const double *fi);
/* Kernels that carry a constant table of their own (the radix-64 tensor-core
 * kernel: DFT-matrix operand tiles and twiddles): its size in bytes (0 for
 * every other kernel) and its host-side construction into dst. */
size_t mofft_cuda_kernel_aux_bytes(int kernel);
int mofft_cuda_kernel_fill_aux(int kernel, void *dst);
/* Launch one pass on `stream` (a cudaStream_t).  Returns a cudaError_t. */
int mofft_cuda_launch_pass(int kernel, const mofft_pass_args *args,
                           void *stream);

#ifdef __cplusplus
}
#endif
#endif
