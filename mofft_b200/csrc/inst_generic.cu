// Runtime-stage-list kernels (any radix chain of the reference's set).
#include "fft_instances.cuh"

namespace mofft {
const Entry *entries_generic(int *count) {
  static const Entry e[] = {
      GenericInst<float, false>::entry("generic_float"),
      GenericInst<double, false>::entry("generic_double"),
      GenericInst<float, true>::entry("generic_float_wide"),
      GenericInst<double, true>::entry("generic_double_wide"),
  };
  *count = (int)(sizeof(e) / sizeof(e[0]));
  return e;
}
}  // namespace mofft
