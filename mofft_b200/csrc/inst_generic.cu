// Runtime-stage-list kernels (any radix chain of the reference's set).
#include "fft_instances.cuh"

namespace mofft {
const Entry *entries_generic(int *count) {
  static const Entry e[] = {
      GenericInst<float, false>::entry("generic_float"),
      GenericInst<double, false>::entry("generic_double"),
      GenericInst<float, true>::entry("generic_float_wide"),
      GenericInst<double, true>::entry("generic_double_wide"),
      // rewrite-family banks 1-3 (like-terms, even-odd, vector-reuse codelets)
      GenericInst<float, false, 1>::entry("generic_float_lt"),
      GenericInst<double, false, 1>::entry("generic_double_lt"),
      GenericInst<float, true, 1>::entry("generic_float_wide_lt"),
      GenericInst<double, true, 1>::entry("generic_double_wide_lt"),
      GenericInst<float, false, 2>::entry("generic_float_eo"),
      GenericInst<double, false, 2>::entry("generic_double_eo"),
      GenericInst<float, true, 2>::entry("generic_float_wide_eo"),
      GenericInst<double, true, 2>::entry("generic_double_wide_eo"),
      GenericInst<float, false, 3>::entry("generic_float_vr"),
      GenericInst<double, false, 3>::entry("generic_double_vr"),
      GenericInst<float, true, 3>::entry("generic_float_wide_vr"),
      GenericInst<double, true, 3>::entry("generic_double_wide_vr"),
  };
  *count = (int)(sizeof(e) / sizeof(e[0]));
  return e;
}
}  // namespace mofft
