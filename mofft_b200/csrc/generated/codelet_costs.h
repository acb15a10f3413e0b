// Generated by mofft_b200/codegen/gen_codelets.py -- do not edit.
// Real additions / multiplications of one forward radix-R codelet (the
// default form), its instructions with products fused into sums (FMA)
// and its peak live temporaries.
#pragma once
typedef struct { int radix; int adds; int muls; int instr; int live; } mofft_codelet_cost;
static const mofft_codelet_cost k_mofft_codelet_costs[] = {
  {2, 4, 0, 4, 7},
  {3, 12, 4, 14, 9},
  {4, 16, 0, 16, 11},
  {5, 32, 16, 36, 19},
  {6, 40, 16, 40, 23},
  {7, 60, 36, 66, 27},
  {8, 52, 4, 56, 19},
  {9, 80, 40, 100, 21},
  {10, 92, 48, 108, 29},
  {11, 140, 100, 150, 43},
  {12, 104, 32, 120, 27},
  {13, 192, 144, 204, 51},
  {14, 160, 96, 184, 41},
  {15, 172, 100, 210, 39},
  {16, 144, 24, 160, 35},
  {32, 376, 88, 432, 67},
  {64, 920, 264, 1072, 131},
};
#define MOFFT_CODELET_COST_COUNT 17
