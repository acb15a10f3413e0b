/* Generated by mofft_b200/codegen/compile_wisdom.py -- do not edit. */
#pragma once
#include <stddef.h>
typedef struct { size_t length; int precision_bits; int count; int chain[24]; } mofft_wisdom_entry;
static const mofft_wisdom_entry k_mofft_wisdom[] = {
  {0u, 0, 0, {0}},
};
#define MOFFT_WISDOM_COUNT 0
#define MOFFT_WISDOM_FORMAL 0
#define MOFFT_WISDOM_SOURCE "none"
