/* MOFFT_PLAN_V1 recipe reader and writer (mofft_recipe.c). */
#ifndef MOFFT_RECIPE_H
#define MOFFT_RECIPE_H

#include "mofft_internal.h"

#ifdef __cplusplus
extern "C" {
#endif

#define MOFFT_RECIPE_MAX_BYTES 1024

/* The fields of a recipe that passed every check. */
typedef struct {
  uint32_t family;
  size_t length;
  mofft_direction direction;
  mofft_placement placement;
  unsigned bank;
  uint64_t mask;
  int direct_input;
  mofft_stage_layout layout;
  int depth;
  int radices[MOFFT_MAX_STAGES]; /* outermost first */
} mofft_recipe;

/* Parses `size` bytes (the NUL included) for a plan of `precision_bits`;
 * MOFFT_SUCCESS fills *out, any other status leaves it unspecified. */
mofft_status mofft_recipe_read(const char *recipe, size_t size, int precision_bits,
                               mofft_recipe *out);
/* Writes c's recipe into buffer (capacity bytes); *required receives the
 * size with the NUL.  buffer NULL with capacity 0 only queries the size. */
mofft_status mofft_recipe_write(const mofft_core *c, char *buffer, size_t capacity,
                                size_t *required);

#ifdef __cplusplus
}
#endif
#endif
