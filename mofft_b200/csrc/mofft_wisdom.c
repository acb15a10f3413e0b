/* Device plan cache: compiled wisdom lookup (the B200 analogue of the
 * reference's generated mofft_generated_wisdom_lookup,
 * tools/compile_wisdom.py:98-157).  Entries map (length, precision) to the
 * tuned Stockham stage chain; the canonical pass grouping turns the chain
 * into the same device schedule every time. */
#include <string.h>

#include "generated/wisdom_table.h"
#include "mofft_host.h"

static int kernel_index_by_name(const char *name) {
  const int n = mofft_cuda_kernel_count();
  for (int i = 0; i < n; ++i)
    if (strcmp(mofft_cuda_kernel_get(i)->name, name) == 0) return i;
  return -1;
}

int mofft_wisdom_lookup(size_t length, int precision_bits, int *chain,
                        int capacity, int *preferred) {
  if (preferred)
    for (int p = 0; p < MOFFT_MAX_PASSES; ++p) preferred[p] = -1;
  for (int i = 0; i < MOFFT_WISDOM_COUNT; ++i) {
    const mofft_wisdom_entry *e = &k_mofft_wisdom[i];
    if (e->length == length && e->precision_bits == precision_bits &&
        e->count <= capacity) {
      memcpy(chain, e->chain, (size_t)e->count * sizeof(int));
      for (int p = 0; preferred && p < MOFFT_MAX_PASSES && p < 4 && e->kernels[p]; ++p)
        preferred[p] = kernel_index_by_name(e->kernels[p]);
      return e->count;
    }
  }
  return 0;
}

int mofft_wisdom_is_formal(void) { return MOFFT_WISDOM_FORMAL; }

const char *mofft_wisdom_source(void) { return MOFFT_WISDOM_SOURCE; }
