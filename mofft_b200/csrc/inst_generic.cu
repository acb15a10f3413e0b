// Runtime-stage-list kernels (any radix chain of the reference's set).
#include "fft_instances.cuh"

namespace mofft {
const Entry *entries_generic(int *count) {
  static const Entry e[] = {
      GenericInst<float>::entry("generic_float"),
      GenericInst<double>::entry("generic_double"),
  };
  *count = (int)(sizeof(e) / sizeof(e[0]));
  return e;
}
}  // namespace mofft
