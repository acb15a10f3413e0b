// Single-pass kernels for lengths 3*2^k and 5*2^k (FP32 and FP64).  The odd
// radix runs first (Ns = 1), where its scatter stride is odd and therefore
// free of shared-memory bank conflicts.
#include "fft_instances.cuh"

namespace mofft {
const Entry *entries_rows_mixed(int *count) {
  static const Entry e[] = {
      ROWS(float, 48, 3, 64, true, 3, 16),
      ROWS(float, 80, 5, 48, true, 5, 16),
      ROWS(float, 96, 6, 32, true, 6, 16),
      ROWS(float, 160, 10, 24, true, 10, 16),
      ROWS(float, 192, 12, 16, true, 12, 16),
      ROWS(float, 320, 20, 8, true, 5, 4, 16),
      ROWS(float, 384, 24, 8, true, 6, 4, 16),
      ROWS(float, 640, 40, 4, false, 5, 8, 16),
      ROWS(float, 768, 48, 4, false, 3, 16, 16),
      ROWS(float, 1280, 80, 2, false, 5, 16, 16),
      ROWS(float, 1536, 96, 2, false, 6, 16, 16),
      ROWS(float, 2560, 160, 1, false, 10, 16, 16),
      ROWS(float, 3072, 192, 1, false, 12, 16, 16),
      ROWS(float, 5120, 320, 1, false, 5, 4, 16, 16),
      ROWS(float, 6144, 384, 1, false, 6, 4, 16, 16),
      ROWS(float, 10240, 640, 1, false, 5, 8, 16, 16),
      ROWS(float, 12288, 768, 1, false, 3, 16, 16, 16),
      ROWS(double, 48, 3, 32, true, 3, 16),
      ROWS(double, 80, 5, 24, true, 5, 16),
      ROWS(double, 96, 6, 16, true, 6, 16),
      ROWS(double, 160, 10, 12, true, 10, 16),
      ROWS(double, 192, 12, 8, true, 12, 16),
      ROWS(double, 320, 20, 4, true, 5, 4, 16),
      ROWS(double, 384, 24, 4, true, 6, 4, 16),
      ROWS(double, 640, 40, 4, false, 5, 8, 16),
      ROWS(double, 768, 48, 4, false, 3, 16, 16),
      ROWS(double, 1280, 80, 2, false, 5, 16, 16),
      ROWS(double, 1536, 96, 2, false, 6, 16, 16),
      ROWS(double, 2560, 160, 1, false, 10, 16, 16),
      ROWS(double, 3072, 192, 1, false, 12, 16, 16),
      ROWS(double, 5120, 320, 1, false, 5, 4, 16, 16),
      ROWS(double, 6144, 384, 1, false, 6, 4, 16, 16),
      // derived radix-16 twiddles; registered before the table-twiddle
      // instances below because the planner takes the first instance of a
      // chain when no tuned kernel applies (in-place plans, where the tuned
      // two-pass schedules of these lengths would need a workspace)
      ROWSD(double, 10240, 640, 1, false, 5, 8, 16, 16),
      ROWSD(double, 12288, 768, 1, false, 3, 16, 16, 16),
      // split exchanges (one component per exchange: half the shared memory)
      ROWSX(double, 2560, 160, 1, 10, 16, 16),
      ROWSX(double, 3072, 192, 1, 12, 16, 16),
      ROWSX(double, 5120, 320, 1, 5, 4, 16, 16),
      ROWSX(double, 6144, 384, 1, 6, 4, 16, 16),
      ROWSX2(double, 2560, 160, 1, 10, 16, 16),
      ROWSX2(double, 3072, 192, 1, 12, 16, 16),
      ROWSX2(double, 5120, 320, 1, 5, 4, 16, 16),
      ROWSX2(double, 6144, 384, 1, 6, 4, 16, 16),
      ROWSX(float, 5120, 320, 1, 5, 4, 16, 16),
      ROWSX(float, 6144, 384, 1, 6, 4, 16, 16),
      ROWSX(float, 10240, 640, 1, 5, 8, 16, 16),
      ROWSX(float, 12288, 768, 1, 3, 16, 16, 16),
      // exchanges move {re, im} pairs
      ROWSDP(float, 1536, 96, 2, 6, 16, 16),
      ROWSDP(float, 3072, 192, 1, 12, 16, 16),
      ROWSDP(float, 5120, 320, 1, 5, 4, 16, 16),
      ROWSDP(float, 6144, 384, 1, 6, 4, 16, 16),
      ROWSDP(float, 10240, 640, 1, 5, 8, 16, 16),
      ROWSDP(float, 12288, 768, 1, 3, 16, 16, 16),
      ROWSDP(double, 3072, 192, 1, 12, 16, 16),
      ROWSDP(double, 6144, 384, 1, 6, 4, 16, 16),
      // derived radix-16 twiddles (5 table loads per butterfly instead of 15)
      ROWSD(float, 80, 5, 48, true, 5, 16),
      ROWSD(float, 96, 6, 32, true, 6, 16),
      ROWSD(float, 160, 10, 24, true, 10, 16),
      ROWSD(float, 192, 12, 16, true, 12, 16),
      ROWSD(float, 320, 20, 8, true, 5, 4, 16),
      ROWSD(float, 384, 24, 8, true, 6, 4, 16),
      ROWSD(float, 640, 40, 4, false, 5, 8, 16),
      ROWSD(float, 768, 48, 4, false, 3, 16, 16),
      ROWSD(double, 80, 5, 24, true, 5, 16),
      ROWSD(double, 96, 6, 16, true, 6, 16),
      ROWSD(double, 160, 10, 12, true, 10, 16),
      ROWSD(double, 192, 12, 8, true, 12, 16),
      ROWSD(double, 320, 20, 4, true, 5, 4, 16),
      ROWSD(double, 384, 24, 4, true, 6, 4, 16),
      ROWSD(double, 640, 40, 4, false, 5, 8, 16),
      ROWSD(double, 768, 48, 4, false, 3, 16, 16),
      ROWSD(float, 1280, 80, 2, false, 5, 16, 16),
      ROWSD(float, 1536, 96, 2, false, 6, 16, 16),
      ROWSD(float, 2560, 160, 1, false, 10, 16, 16),
      ROWSD(float, 3072, 192, 1, false, 12, 16, 16),
      ROWSD(float, 5120, 320, 1, false, 5, 4, 16, 16),
      ROWSD(float, 6144, 384, 1, false, 6, 4, 16, 16),
      ROWSD(float, 10240, 640, 1, false, 5, 8, 16, 16),
      ROWSD(float, 12288, 768, 1, false, 3, 16, 16, 16),
      ROWSD(double, 1280, 80, 2, false, 5, 16, 16),
      ROWSD(double, 1536, 96, 2, false, 6, 16, 16),
      ROWS(double, 10240, 640, 1, false, 5, 8, 16, 16),
      ROWS(double, 12288, 768, 1, false, 3, 16, 16, 16),
  };
  *count = (int)(sizeof(e) / sizeof(e[0]));
  return e;
}
}  // namespace mofft
