// Column-pass kernels for the 3*2^a and 5*2^a factors of multi-pass lengths.
#include "fft_instances.cuh"

namespace mofft {
const Entry *entries_cols_mixed(int *count) {
  static const Entry e[] = {
      COLS(float, 48, 3, 32, 3, 16),
      COLS(float, 96, 6, 32, 6, 16),
      COLS(float, 192, 12, 16, 12, 16),
      COLS(float, 384, 24, 16, 6, 4, 16),
      COLS(float, 768, 48, 16, 3, 16, 16),
      COLS(float, 1536, 96, 8, 6, 16, 16),
      COLS(float, 80, 5, 32, 5, 16),
      COLS(float, 160, 10, 16, 10, 16),
      COLS(float, 320, 20, 16, 5, 4, 16),
      COLS(float, 640, 40, 16, 5, 8, 16),
      COLS(float, 1280, 80, 8, 5, 16, 16),
      COLS(double, 48, 3, 16, 3, 16),
      COLS(double, 96, 6, 16, 6, 16),
      COLS(double, 192, 12, 16, 12, 16),
      COLS(double, 384, 24, 8, 6, 4, 16),
      COLS(double, 768, 48, 8, 3, 16, 16),
      COLS(double, 1536, 96, 4, 6, 16, 16),
      COLS(double, 80, 5, 16, 5, 16),
      COLS(double, 160, 10, 16, 10, 16),
      COLS(double, 320, 20, 8, 5, 4, 16),
      COLS(double, 640, 40, 8, 5, 8, 16),
      COLS(double, 1280, 80, 4, 5, 16, 16),
      COLSP(float, 80, 5, 32, 5, 16),
      COLSP(float, 160, 10, 16, 10, 16),
      COLSP(float, 192, 12, 16, 12, 16),
      COLSP(float, 1536, 96, 8, 6, 16, 16),
      COLSP(double, 80, 5, 16, 5, 16),
      COLSP(double, 96, 6, 16, 6, 16),
      COLSP(double, 160, 10, 16, 10, 16),
      COLSP(double, 192, 12, 16, 12, 16),
      COLSP(double, 384, 24, 8, 6, 4, 16),
      COLSP(double, 1536, 96, 4, 6, 16, 16),
  };
  *count = (int)(sizeof(e) / sizeof(e[0]));
  return e;
}
}  // namespace mofft
