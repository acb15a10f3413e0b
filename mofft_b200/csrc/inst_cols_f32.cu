// FP32 multi-pass (four-step / six-step) column kernels.
#include "fft_instances.cuh"

namespace mofft {
const Entry *entries_cols_f32(int *count) {
  static const Entry e[] = {
      COLS(float, 16, 1, 32, 16),
      COLS(float, 32, 4, 32, 8, 4),
      COLS(float, 64, 4, 32, 16, 4),
      COLS(float, 128, 8, 16, 16, 8),
      COLS(float, 256, 16, 16, 16, 16),
      COLS(float, 512, 32, 16, 16, 16, 2),
      COLS(float, 1024, 64, 8, 16, 16, 4),
      COLS(float, 2048, 64, 8, 16, 16, 8),
      COLS(float, 4096, 128, 4, 16, 16, 16),
      COLS(float, 1024, 32, 16, 16, 16, 4),
      COLS(float, 2048, 128, 8, 16, 16, 8),
      COLS(float, 4096, 256, 4, 16, 16, 16),
      COLS(float, 64, 4, 64, 16, 4),
      COLS(float, 128, 8, 32, 16, 8),
      COLS(float, 512, 32, 8, 16, 16, 2),
      COLS(float, 1024, 64, 4, 16, 16, 4),
      COLSP(float, 64, 4, 32, 16, 4),
      COLSP(float, 128, 8, 16, 16, 8),
      COLSP(float, 128, 8, 32, 16, 8),
      COLSP(float, 256, 16, 16, 16, 16),
      COLSP(float, 512, 32, 8, 16, 16, 2),
      COLSP(float, 1024, 64, 8, 16, 16, 4),
      COLSP(float, 2048, 128, 8, 16, 16, 8),
      COLSP(float, 4096, 256, 4, 16, 16, 16),
  };
  *count = (int)(sizeof(e) / sizeof(e[0]));
  return e;
}
}  // namespace mofft
