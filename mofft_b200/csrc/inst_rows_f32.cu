// FP32 single-pass kernels: whole transforms per CTA.
#include "fft_instances.cuh"

namespace mofft {
const Entry *entries_rows_f32(int *count) {
  static const Entry e[] = {
      ROWS(float, 2, 1, 256, true, 2),
      ROWS(float, 4, 1, 256, true, 4),
      ROWS(float, 8, 1, 256, true, 8),
      ROWS(float, 16, 1, 256, true, 16),
      ROWS(float, 32, 4, 64, true, 8, 4),
      ROWS(float, 64, 4, 64, true, 16, 4),
      ROWS(float, 128, 8, 32, true, 16, 8),
      ROWS(float, 256, 16, 16, true, 16, 16),
      ROWS(float, 256, 16, 16, false, 16, 16),
      ROWS(float, 512, 32, 8, false, 16, 16, 2),
      ROWS(float, 512, 64, 4, false, 8, 8, 8),
      ROWS(float, 1024, 64, 4, false, 16, 16, 4),
      ROWS(float, 1024, 64, 2, false, 16, 16, 4),
      ROWS(float, 1024, 32, 8, false, 32, 32),
      ROWS(float, 2048, 128, 2, false, 16, 16, 8),
      ROWS(float, 2048, 128, 1, false, 16, 16, 8),
      ROWS(float, 4096, 256, 1, false, 16, 16, 16),
      ROWS(float, 4096, 512, 1, false, 16, 16, 16),
      ROWS(float, 8192, 512, 1, false, 16, 16, 16, 2),
      ROWS(float, 16384, 512, 1, false, 16, 16, 16, 4),
      // derived radix-16 twiddles (fewer table loads through L1)
      ROWSD(float, 256, 16, 16, true, 16, 16),
      ROWSD(float, 512, 32, 8, false, 16, 16, 2),
      ROWSD(float, 1024, 64, 4, false, 16, 16, 4),
      ROWSD(float, 2048, 128, 2, false, 16, 16, 8),
      ROWSD(float, 4096, 256, 1, false, 16, 16, 16),
      ROWSD(float, 4096, 512, 1, false, 16, 16, 16),
      ROWSD(float, 8192, 512, 1, false, 16, 16, 16, 2),
      ROWSD(float, 16384, 512, 1, false, 16, 16, 16, 4),
      // more or fewer points per thread for the small staged lengths
      ROWS(float, 32, 2, 128, true, 16, 2),
      ROWS(float, 64, 2, 128, true, 16, 4),
      ROWS(float, 64, 8, 32, true, 8, 8),
      ROWS(float, 128, 4, 64, true, 16, 8),
      ROWS(float, 128, 16, 16, true, 8, 16),
      // radix-32 stages: one exchange fewer for the long lines
      ROWSD2(float, 8192, 256, 1, 32, 16, 16),
      ROWSD2(float, 8192, 256, 1, 16, 16, 32),
      ROWSD(float, 16384, 512, 1, false, 32, 32, 16),
      ROWSD(float, 16384, 512, 1, false, 16, 32, 32),
      // split exchanges (one component at a time: half the shared memory)
      ROWSX(float, 2048, 128, 2, 16, 16, 8),
      ROWSX(float, 4096, 256, 1, 16, 16, 16),
      ROWSX(float, 8192, 512, 1, 16, 16, 16, 2),
      ROWSX(float, 16384, 512, 1, 16, 16, 16, 4),
      ROWSX(float, 16384, 1024, 1, 16, 16, 16, 4),
      // exchanges move {re, im} pairs: one 8-byte shared access per value
      ROWSDP(float, 512, 32, 8, 16, 16, 2),
      ROWSDP(float, 1024, 64, 4, 16, 16, 4),
      ROWSDP(float, 1024, 64, 2, 16, 16, 4),
      ROWSDP(float, 2048, 128, 1, 16, 16, 8),
      ROWSDP(float, 2048, 128, 2, 16, 16, 8),
      ROWSDP(float, 4096, 256, 1, 16, 16, 16),
      ROWSDP(float, 8192, 512, 1, 16, 16, 16, 2),
      ROWSDP(float, 16384, 1024, 1, 16, 16, 16, 4),
      // persistent CTAs, next line bulk-copied while this one is transformed
      // (measured on 2^26 points against the kernels above: ahead only for
      // 16384, 0.55 against 0.51 of the HBM roofline; at 4096-12288 and for
      // FP64 2048-8192 the same scheme measured 0-30 % slower, the lines
      // being bound by registers and exchanges rather than by load latency)
      ROWSP(float, 16384, 512, 32, 32, 16),
      // staged tiles kept as {re, im} pairs (no de-interleaving copies)
      ROWSSP(float, 16, 1, 256, 16),
      ROWSSP(float, 32, 4, 64, 8, 4),
      ROWSSP(float, 32, 2, 128, 16, 2),
      ROWSSP(float, 64, 4, 64, 16, 4),
      ROWSSP(float, 64, 8, 32, 8, 8),
      ROWSSP(float, 128, 8, 32, 16, 8),
      ROWSSP(float, 256, 16, 16, 16, 16),
  };
  *count = (int)(sizeof(e) / sizeof(e[0]));
  return e;
}
}  // namespace mofft
