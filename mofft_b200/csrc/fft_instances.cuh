// Registry entry templates shared by the kernel instance files.
#pragma once
#include <cuda_runtime.h>

#include "fft_device.cuh"
#include "mofft_cuda.h"

namespace mofft {

typedef cudaError_t (*launch_fn)(const mofft_pass_args *, cudaStream_t);
typedef const void *(*func_fn)();

struct Entry {
  mofft_kernel_desc desc;
  launch_fn launch;
  func_fn func;
  // kernels with a constant table of their own (e.g. DFT-matrix operands):
  // its size and its host-side construction; 0 / null for the others
  size_t aux_bytes;
  int (*fill_aux)(void *dst);
};

template <typename T>
RowsArgs<T> rows_args(const mofft_pass_args *p) {
  RowsArgs<T> a;
  a.in = static_cast<const cplx_t<T> *>(p->in);
  a.out = static_cast<cplx_t<T> *>(p->out);
  a.tw = static_cast<const cplx_t<T> *>(p->tw);
  a.batch = p->batch;
  a.in_dist = p->in_dist;
  a.out_dist = p->out_dist;
  a.sign = p->conj_in ? T(-1) : T(1);
  a.in_table = reinterpret_cast<const cplx_t<T> *const *>(p->in_table);
  a.out_table = reinterpret_cast<cplx_t<T> *const *>(p->out_table);
  a.status = p->status;
  a.lose_copy = p->lose_copy;
  return a;
}

template <typename T>
ColsArgs<T> cols_args(const mofft_pass_args *p) {
  ColsArgs<T> a;
  a.in = static_cast<const cplx_t<T> *>(p->in);
  a.out = static_cast<cplx_t<T> *>(p->out);
  a.tw = static_cast<const cplx_t<T> *>(p->tw);
  a.tw_hi = static_cast<const cplx_t<T> *>(p->tw_hi);
  a.tw_lo = static_cast<const cplx_t<T> *>(p->tw_lo);
  a.batch = p->batch;
  a.in_dist = p->in_dist;
  a.out_dist = p->out_dist;
  a.total = p->total;
  a.ns_outer = p->ns_outer;
  a.split_shift = p->split_shift;
  a.sign_in = p->conj_in ? T(-1) : T(1);
  a.sign_out = p->conj_out ? T(-1) : T(1);
  a.in_table = reinterpret_cast<const cplx_t<T> *const *>(p->in_table);
  a.out_table = reinterpret_cast<cplx_t<T> *const *>(p->out_table);
  return a;
}

template <typename T, int L, int TPL, int TB, int FLAGS, int... Rs>
struct RowsInst {
  static constexpr bool kPf = (FLAGS & kPrefetch) != 0;
  static_assert(!kPf || (TB == 1 && (FLAGS & kSplitX) != 0 && (FLAGS & kStaged) == 0),
                "prefetching kernels run one split-exchange line per CTA step");
  static constexpr size_t smem() {
    if constexpr (kPf) return prefetch_smem<T, L, TPL>();
    if constexpr ((FLAGS & kPairX) != 0)
      return 2ull * TB * pair_pitch<T>(L, TPL, TB, pair_shift(FLAGS)) * sizeof(T);
    return ((FLAGS & kSplitX) ? 1ull : 2ull) * TB * rows_line<T>(L, TPL, TB) * sizeof(T);
  }
  static const void *func() {
    if constexpr (kPf)
      return reinterpret_cast<const void *>(&rows_prefetch_kernel<T, L, TPL, FLAGS, Rs...>);
    else if constexpr ((FLAGS & kTwoCtas) != 0)
      return reinterpret_cast<const void *>(&rows_kernel_2cta<T, L, TPL, TB, FLAGS, Rs...>);
    else
      return reinterpret_cast<const void *>(&rows_kernel<T, L, TPL, TB, FLAGS, Rs...>);
  }
  // Prefetching kernels: resident CTAs per SM times the SM count, cached per
  // device (0 when the device cannot be queried).
  static int persistent_grid() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (cached[dev] > 0) return cached[dev];
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, rows_prefetch_kernel<T, L, TPL, FLAGS, Rs...>, TPL, smem()) !=
            cudaSuccess)
      return 0;
    if (per_sm < 1) return sms;  // shared-memory attribute not set yet: do not cache
    cached[dev] = per_sm * sms;
    return cached[dev];
  }
  static cudaError_t launch(const mofft_pass_args *p, cudaStream_t s) {
    if (p->conj_in != p->conj_out) return cudaErrorInvalidValue;
    if constexpr (kPf) {
      if (p->batch <= 0) return cudaSuccess;
      const int resident = persistent_grid();
      if (resident <= 0) return cudaErrorInvalidConfiguration;
      const long long grid = p->batch < resident ? p->batch : resident;
      rows_prefetch_kernel<T, L, TPL, FLAGS, Rs...>
          <<<(unsigned)grid, TPL, smem(), s>>>(rows_args<T>(p));
      return cudaGetLastError();
    }
    const long long grid = (p->batch + TB - 1) / TB;
    if (grid <= 0) return cudaSuccess;
    if (grid > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    if constexpr ((FLAGS & kTwoCtas) != 0)
      rows_kernel_2cta<T, L, TPL, TB, FLAGS, Rs...>
          <<<(unsigned)grid, TPL * TB, smem(), s>>>(rows_args<T>(p));
    else
      rows_kernel<T, L, TPL, TB, FLAGS, Rs...>
          <<<(unsigned)grid, TPL * TB, smem(), s>>>(rows_args<T>(p));
    return cudaGetLastError();
  }
  static Entry entry(const char *name) {
    Entry e{};
    e.desc.name = name;
    e.desc.precision_bits = sizeof(T) == 4 ? 32 : 64;
    e.desc.kind = MOFFT_KERNEL_ROWS;
    e.desc.length = L;
    e.desc.lines = TB;
    e.desc.threads = TPL * TB;
    e.desc.staged = (FLAGS & kStaged) ? 1 : 0;
    e.desc.prefetch = kPf ? 1 : 0;
    const int rs[] = {Rs...};
    e.desc.radix_count = (int)sizeof...(Rs);
    for (int i = 0; i < 8; ++i) e.desc.radices[i] = i < (int)sizeof...(Rs) ? rs[i] : 0;
    e.desc.smem_bytes = smem();
    e.launch = &launch;
    e.func = &func;
    return e;
  }
};

template <typename T, int L, int TPL, int C, int... Rs>
struct ColsInst {
  using G = ColsGeom<T, L, TPL, C>;
  static const void *func() {
    return reinterpret_cast<const void *>(&cols_kernel<T, L, TPL, C, Rs...>);
  }
  static cudaError_t launch(const mofft_pass_args *p, cudaStream_t s) {
    if (p->total % L != 0 || (p->total / L) % C != 0) return cudaErrorInvalidValue;
    if (p->ns_outer != 1 && p->ns_outer % C != 0) return cudaErrorInvalidValue;
    const long long groups = (p->total / L) / C;
    const long long grid = groups * p->batch;
    if (grid <= 0) return cudaSuccess;
    if (grid > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    cols_kernel<T, L, TPL, C, Rs...>
        <<<(unsigned)grid, G::THREADS, G::SMEM, s>>>(cols_args<T>(p));
    return cudaGetLastError();
  }
  static Entry entry(const char *name) {
    Entry e{};
    e.desc.name = name;
    e.desc.precision_bits = sizeof(T) == 4 ? 32 : 64;
    e.desc.kind = MOFFT_KERNEL_COLS;
    e.desc.length = L;
    e.desc.lines = C;
    e.desc.threads = G::THREADS;
    e.desc.staged = 0;
    const int rs[] = {Rs...};
    e.desc.radix_count = (int)sizeof...(Rs);
    for (int i = 0; i < 8; ++i) e.desc.radices[i] = i < (int)sizeof...(Rs) ? rs[i] : 0;
    e.desc.smem_bytes = G::SMEM;
    e.launch = &launch;
    e.func = &func;
    return e;
  }
};

// Column pass whose exchanges move {re, im} pairs (cols_kernel_pair).
template <typename T, int L, int TPL, int C, int... Rs>
struct ColsPairInst {
  using G = ColsGeom<T, L, TPL, C>;
  static const void *func() {
    return reinterpret_cast<const void *>(&cols_kernel_pair<T, L, TPL, C, Rs...>);
  }
  static cudaError_t launch(const mofft_pass_args *p, cudaStream_t s) {
    if (p->total % L != 0 || (p->total / L) % C != 0) return cudaErrorInvalidValue;
    if (p->ns_outer != 1 && p->ns_outer % C != 0) return cudaErrorInvalidValue;
    const long long groups = (p->total / L) / C;
    const long long grid = groups * p->batch;
    if (grid <= 0) return cudaSuccess;
    if (grid > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    cols_kernel_pair<T, L, TPL, C, Rs...>
        <<<(unsigned)grid, G::THREADS, G::SMEM, s>>>(cols_args<T>(p));
    return cudaGetLastError();
  }
  static Entry entry(const char *name) {
    Entry e{};
    e.desc.name = name;
    e.desc.precision_bits = sizeof(T) == 4 ? 32 : 64;
    e.desc.kind = MOFFT_KERNEL_COLS;
    e.desc.length = L;
    e.desc.lines = C;
    e.desc.threads = G::THREADS;
    e.desc.staged = 0;
    const int rs[] = {Rs...};
    e.desc.radix_count = (int)sizeof...(Rs);
    for (int i = 0; i < 8; ++i) e.desc.radices[i] = i < (int)sizeof...(Rs) ? rs[i] : 0;
    e.desc.smem_bytes = G::SMEM;
    e.launch = &launch;
    e.func = &func;
    return e;
  }
};

template <typename T>
size_t generic_smem(int L, int lines, int cols) {
  const size_t words = cols ? (size_t)L * (lines + 1) : (size_t)lines * spad_len<T>(L);
  return 4 * words * sizeof(T);
}

template <typename T, bool WIDE, int BANK = 0>
struct GenericInst {
  static const void *func() {
    return reinterpret_cast<const void *>(&generic_kernel<T, WIDE, BANK>);
  }
  static cudaError_t launch(const mofft_pass_args *p, cudaStream_t s) {
    GenericArgs<T> a;
    a.in = static_cast<const cplx_t<T> *>(p->in);
    a.out = static_cast<cplx_t<T> *>(p->out);
    a.tw = static_cast<const cplx_t<T> *>(p->tw);
    a.tw_hi = static_cast<const cplx_t<T> *>(p->tw_hi);
    a.tw_lo = static_cast<const cplx_t<T> *>(p->tw_lo);
    a.batch = p->batch;
    a.in_dist = p->in_dist;
    a.out_dist = p->out_dist;
    a.total = p->generic_cols ? p->total : p->length;
    a.ns_outer = p->generic_cols ? p->ns_outer : 1;
    a.split_shift = p->split_shift;
    a.cols = p->generic_cols;
    a.length = p->length;
    a.lines = p->lines;
    a.stage_count = p->radix_count;
    if (p->radix_count < 1 || p->radix_count > kMaxGenericStages || p->lines < 1)
      return cudaErrorInvalidValue;
    if (p->in_table || p->out_table) return cudaErrorNotSupported;
    long long prod = 1;
    for (int i = 0; i < kMaxGenericStages; ++i) {
      a.radices[i] = i < p->radix_count ? p->radices[i] : 0;
      if (i < p->radix_count) prod *= p->radices[i];
    }
    if (prod != p->length) return cudaErrorInvalidValue;
    for (int i = 0; i < p->radix_count; ++i)
      if (!WIDE && p->radices[i] > 16) return cudaErrorInvalidValue;
    a.sign_in = p->conj_in ? T(-1) : T(1);
    a.sign_out = p->conj_out ? T(-1) : T(1);
    long long grid;
    if (a.cols) {
      if (p->total % p->length != 0 || (p->total / p->length) % p->lines != 0)
        return cudaErrorInvalidValue;
      if (p->ns_outer != 1 && p->ns_outer % p->lines != 0) return cudaErrorInvalidValue;
      grid = (p->total / p->length) / p->lines * p->batch;
    } else {
      grid = (p->batch + p->lines - 1) / p->lines;
    }
    if (grid <= 0) return cudaSuccess;
    if (grid > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    const size_t smem = generic_smem<T>(p->length, p->lines, p->generic_cols);
    generic_kernel<T, WIDE, BANK><<<(unsigned)grid, 256, smem, s>>>(a);
    return cudaGetLastError();
  }
  static Entry entry(const char *name) {
    Entry e{};
    e.desc.name = name;
    e.desc.bank = BANK;
    e.desc.precision_bits = sizeof(T) == 4 ? 32 : 64;
    e.desc.kind = MOFFT_KERNEL_GENERIC;
    e.desc.length = 0;
    e.desc.lines = 0;
    e.desc.threads = 256;
    e.desc.staged = 0;
    // radices[0] records the largest radix this variant runs
    e.desc.radix_count = 0;
    for (int i = 0; i < 8; ++i) e.desc.radices[i] = 0;
    e.desc.radices[0] = WIDE ? 64 : 16;
    e.desc.smem_bytes = 227 * 1024;
    e.launch = &launch;
    e.func = &func;
    return e;
  }
};


// ST: true/false (staged I/O); ROWSD: staged flag plus derived radix-16
// twiddles (name suffix _d).
#define ROWS(T, L, TPL, TB, ST, ...) \
  RowsInst<T, L, TPL, TB, (ST) ? kStaged : 0, __VA_ARGS__>::entry( \
      "rows_" #T "_" #L "_t" #TPL "_b" #TB "_s" #ST)
#define ROWSD(T, L, TPL, TB, ST, ...) \
  RowsInst<T, L, TPL, TB, ((ST) ? kStaged : 0) | kDerivedTw, __VA_ARGS__>::entry( \
      "rows_" #T "_" #L "_t" #TPL "_b" #TB "_s" #ST "_d")
#define ROWSDP(T, L, TPL, TB, ...) \
  RowsInst<T, L, TPL, TB, kDerivedTw | kPairX, __VA_ARGS__>::entry( \
      "rows_" #T "_" #L "_t" #TPL "_b" #TB "_sfalse_dp")
#define ROWSDP0(T, L, TPL, TB, ...) \
  RowsInst<T, L, TPL, TB, kDerivedTw | kPairX | kPairPad0, __VA_ARGS__>::entry( \
      "rows_" #T "_" #L "_t" #TPL "_b" #TB "_sfalse_dp0")
#define ROWSDP5(T, L, TPL, TB, ...) \
  RowsInst<T, L, TPL, TB, kDerivedTw | kPairX | kPairPad32, __VA_ARGS__>::entry( \
      "rows_" #T "_" #L "_t" #TPL "_b" #TB "_sfalse_dp5")
#define ROWSSP(T, L, TPL, TB, ...) \
  RowsInst<T, L, TPL, TB, kStaged | kDerivedTw | kPairX, __VA_ARGS__>::entry( \
      "rows_" #T "_" #L "_t" #TPL "_b" #TB "_strue_dp")
#define ROWSX(T, L, TPL, TB, ...) \
  RowsInst<T, L, TPL, TB, kDerivedTw | kSplitX, __VA_ARGS__>::entry( \
      "rows_" #T "_" #L "_t" #TPL "_b" #TB "_sfalse_dx")
#define ROWSX2(T, L, TPL, TB, ...) \
  RowsInst<T, L, TPL, TB, kDerivedTw | kSplitX | kTwoCtas, __VA_ARGS__>::entry( \
      "rows_" #T "_" #L "_t" #TPL "_b" #TB "_sfalse_dx2")
#define ROWSD2(T, L, TPL, TB, ...) \
  RowsInst<T, L, TPL, TB, kDerivedTw | kTwoCtas, __VA_ARGS__>::entry( \
      "rows_" #T "_" #L "_t" #TPL "_b" #TB "_sfalse_d2")
#define ROWSP(T, L, TPL, ...) \
  RowsInst<T, L, TPL, 1, kDerivedTw | kSplitX | kPrefetch, __VA_ARGS__>::entry( \
      "rows_" #T "_" #L "_t" #TPL "_b1_sfalse_dxp")
#define ROWSP2(T, L, TPL, ...) \
  RowsInst<T, L, TPL, 1, kDerivedTw | kSplitX | kPrefetch | kTwoCtas, __VA_ARGS__>::entry( \
      "rows_" #T "_" #L "_t" #TPL "_b1_sfalse_dxp2")
#define COLS(T, L, TPL, C, ...) \
  ColsInst<T, L, TPL, C, __VA_ARGS__>::entry("cols_" #T "_" #L "_t" #TPL "_c" #C)
#define COLSP(T, L, TPL, C, ...) \
  ColsPairInst<T, L, TPL, C, __VA_ARGS__>::entry("cols_" #T "_" #L "_t" #TPL "_c" #C "_p")

// Each instance file defines one of these.
const Entry *entries_generic(int *count);
const Entry *entries_rows_f32(int *count);
const Entry *entries_rows_f64(int *count);
const Entry *entries_cols_f32(int *count);
const Entry *entries_cols_f64(int *count);
const Entry *entries_rows_mixed(int *count);
const Entry *entries_cols_mixed(int *count);
const Entry *entries_tensor(int *count);
const Entry *entries_tensor64(int *count);
const Entry *entries_cluster(int *count);

}  // namespace mofft
