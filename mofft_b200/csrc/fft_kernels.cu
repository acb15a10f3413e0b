// Kernel registry and the launch shim behind the internal C-ABI of
// mofft_cuda.h.  Each registry entry is one compiled variant (precision, line
// length, threads per line, lines per CTA, in-CTA radix chain).  The host
// planner picks entries; the MEASURE planner times them.
#include <vector>

#include "fft_instances.cuh"

using namespace mofft;

namespace {

const std::vector<Entry> &registry() {
  static const std::vector<Entry> all = [] {
    std::vector<Entry> v;
    const Entry *(*lists[])(int *) = {entries_generic, entries_rows_f32,
                                      entries_rows_f64, entries_cols_f32,
                                      entries_cols_f64, entries_rows_mixed,
                                      entries_cols_mixed, entries_tensor64,
                                      entries_tensor, entries_cluster};
    for (auto list : lists) {
      int n = 0;
      const Entry *e = list(&n);
      v.insert(v.end(), e, e + n);
    }
    return v;
  }();
  return all;
}

}  // namespace

extern "C" int mofft_cuda_kernel_count(void) { return (int)registry().size(); }

extern "C" const mofft_kernel_desc *mofft_cuda_kernel_get(int index) {
  const auto &r = registry();
  if (index < 0 || index >= (int)r.size()) return nullptr;
  return &r[index].desc;
}

extern "C" size_t mofft_cuda_generic_smem(int precision_bits, int length,
                                          int lines, int cols) {
  return precision_bits == 32 ? generic_smem<float>(length, lines, cols)
                              : generic_smem<double>(length, lines, cols);
}

extern "C" int mofft_cuda_prepare_device(void) {
  for (const Entry &e : registry()) {
    size_t smem = e.desc.smem_bytes;
    if (smem > 227 * 1024) smem = 227 * 1024;
    cudaError_t err = cudaFuncSetAttribute(
        e.func(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return (int)err;
  }
  return 0;
}

extern "C" size_t mofft_cuda_kernel_aux_bytes(int kernel) {
  const auto &r = registry();
  if (kernel < 0 || kernel >= (int)r.size()) return 0;
  return r[kernel].fill_aux ? r[kernel].aux_bytes : 0;
}

extern "C" int mofft_cuda_kernel_fill_aux(int kernel, void *dst) {
  const auto &r = registry();
  if (kernel < 0 || kernel >= (int)r.size() || !r[kernel].fill_aux || !dst)
    return (int)cudaErrorInvalidValue;
  return r[kernel].fill_aux(dst);
}

extern "C" int mofft_cuda_launch_pass(int kernel, const mofft_pass_args *args,
                                      void *stream) {
  const auto &r = registry();
  if (kernel < 0 || kernel >= (int)r.size() || !args) return (int)cudaErrorInvalidValue;
  return (int)r[kernel].launch(args, static_cast<cudaStream_t>(stream));
}
