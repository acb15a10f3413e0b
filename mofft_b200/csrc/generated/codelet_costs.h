// Generated by mofft_b200/codegen/gen_codelets.py -- do not edit.
// Real additions / multiplications of one forward radix-R codelet.
#pragma once
typedef struct { int radix; int adds; int muls; } mofft_codelet_cost;
static const mofft_codelet_cost k_mofft_codelet_costs[] = {
  {2, 4, 0},
  {3, 12, 4},
  {4, 16, 0},
  {5, 32, 16},
  {6, 40, 16},
  {7, 60, 36},
  {8, 52, 4},
  {9, 80, 40},
  {10, 92, 48},
  {11, 140, 100},
  {12, 104, 32},
  {13, 192, 144},
  {14, 160, 96},
  {15, 172, 100},
  {16, 144, 24},
  {32, 376, 88},
  {64, 928, 248},
};
#define MOFFT_CODELET_COST_COUNT 17
