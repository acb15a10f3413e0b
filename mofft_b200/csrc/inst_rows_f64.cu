// FP64 single-pass kernels: whole transforms per CTA.
#include "fft_instances.cuh"

namespace mofft {
const Entry *entries_rows_f64(int *count) {
  static const Entry e[] = {
      ROWS(double, 2, 1, 128, true, 2),
      ROWS(double, 4, 1, 128, true, 4),
      ROWS(double, 8, 1, 128, true, 8),
      ROWS(double, 16, 1, 128, true, 16),
      ROWS(double, 32, 4, 32, true, 8, 4),
      ROWS(double, 64, 8, 16, true, 8, 8),
      ROWS(double, 128, 16, 8, true, 8, 16),
      ROWS(double, 256, 16, 8, false, 16, 16),
      ROWS(double, 256, 32, 4, false, 8, 32),
      ROWS(double, 512, 64, 2, false, 8, 8, 8),
      ROWS(double, 1024, 128, 2, false, 8, 8, 16),
      ROWS(double, 1024, 64, 2, false, 16, 16, 4),
      ROWS(double, 2048, 256, 1, false, 8, 16, 16),
      ROWS(double, 4096, 256, 1, false, 16, 16, 16),
      ROWS(double, 4096, 512, 1, false, 8, 8, 8, 8),
      ROWS(double, 8192, 512, 1, false, 16, 16, 16, 2),
      ROWS(double, 64, 4, 32, true, 16, 4),
      ROWS(double, 128, 8, 16, true, 16, 8),
      ROWS(double, 32, 2, 64, true, 16, 2),
      ROWSD(double, 1024, 64, 2, false, 16, 16, 4),
      ROWSD(double, 4096, 256, 1, false, 16, 16, 16),
      ROWSD(double, 8192, 512, 1, false, 16, 16, 16, 2),
      ROWSX(double, 2048, 128, 2, 16, 16, 8),
      ROWSX(double, 4096, 256, 1, 16, 16, 16),
      ROWSX(double, 8192, 512, 1, 16, 16, 16, 2),
      // exchanges move {re, im} pairs: one 16-byte shared access per value
      ROWSDP(double, 256, 16, 8, 16, 16),
      ROWSDP(double, 512, 32, 4, 16, 16, 2),
      ROWSDP(double, 1024, 64, 2, 16, 16, 4),
      ROWSDP(double, 2048, 128, 2, 16, 16, 8),
      ROWSDP(double, 4096, 256, 1, 16, 16, 16),
      ROWSDP(double, 8192, 512, 1, 16, 16, 16, 2),
      // staged tiles kept as {re, im} pairs
      ROWSSP(double, 16, 1, 128, 16),
      ROWSSP(double, 32, 4, 32, 8, 4),
      ROWSSP(double, 64, 8, 16, 8, 8),
      ROWSSP(double, 64, 4, 32, 16, 4),
      ROWSSP(double, 128, 8, 16, 16, 8),
  };
  *count = (int)(sizeof(e) / sizeof(e[0]));
  return e;
}
}  // namespace mofft
