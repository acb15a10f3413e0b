// FP64 multi-pass (four-step / six-step) column kernels.
#include "fft_instances.cuh"

namespace mofft {
const Entry *entries_cols_f64(int *count) {
  static const Entry e[] = {
      COLS(double, 16, 2, 16, 8, 2),
      COLS(double, 32, 4, 16, 8, 4),
      COLS(double, 64, 8, 16, 8, 8),
      COLS(double, 128, 8, 16, 16, 8),
      COLS(double, 256, 16, 8, 16, 16),
      COLS(double, 512, 32, 8, 16, 16, 2),
      COLS(double, 1024, 64, 4, 16, 16, 4),
      COLS(double, 2048, 128, 4, 16, 16, 8),
      COLS(double, 256, 16, 16, 16, 16),
      COLS(double, 128, 8, 32, 16, 8),
      COLSP(double, 64, 8, 16, 8, 8),
      COLSP(double, 128, 8, 16, 16, 8),
      COLSP(double, 256, 16, 16, 16, 16),
      COLSP(double, 256, 16, 8, 16, 16),
      COLSP(double, 512, 32, 8, 16, 16, 2),
      COLSP(double, 1024, 64, 4, 16, 16, 4),
      COLSP(double, 2048, 128, 4, 16, 16, 8),
  };
  *count = (int)(sizeof(e) / sizeof(e[0]));
  return e;
}
}  // namespace mofft
