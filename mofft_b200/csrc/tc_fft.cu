// Tensor-core precision forms of the FP32 transform (tcgen05, sm_100a).
//
// n = 4096 = 16^3 as three radix-16 Stockham stages, each a DFT-matrix GEMM
// on the 5th-generation tensor cores.  A stage over the 256 butterflies of a
// transform is the real GEMM
//
//     D[j][n] = sum_kk A[j][kk] * B[kk][n],   j < 256, n < 32, kk < 32,
//
// where row j of A holds butterfly j's twiddled inputs (16 real parts, then
// 16 imaginary parts) and B is the real form of the 16-point DFT matrix F:
// columns n < 16 give Re(F v)_n = sum Fr v_re - Fi v_im, columns 16 + k give
// Im(F v)_k = sum Fi v_re + Fr v_im.  M = 256 runs as two M = 128 MMAs whose
// accumulators live in TMEM (32 columns each); K = 32 is split in K-steps of
// one instruction.
//
// Split precision (FP32 accumulate):
//   3xTF32:  x = hi + lo with hi = tf32(x), lo = tf32(x - hi) (about 21
//            significant bits); A*B ~ A_lo*B_hi + A_hi*B_lo + A_hi*B_hi.
//   BF16x3:  the same with bfloat16 pieces (about 16 significant bits).
// The small terms are accumulated first.
//
// Per stage: every thread (one per butterfly, 256 threads) gathers and
// twiddles its inputs (CUDA cores), splits them and stores its A row in the
// canonical K-major no-swizzle layout; after a proxy fence and a CTA barrier
// one elected thread issues the MMAs and commits them to an mbarrier; every
// thread then reads its own TMEM row (32x32b.x32) and scatters the 16 complex
// outputs with the Stockham index map.  Every mbarrier wait is bounded: on
// timeout the CTA records an error, waits once more (bounded), frees its TMEM
// and returns; the host reports MOFFT_INTERNAL_ERROR.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "fft_device.cuh"
#include "fft_instances.cuh"
#include "mofft_cuda.h"

namespace mofft {

constexpr int kFormTf32x3 = 1;  // MOFFT_FORM_TF32X3
constexpr int kFormBf16x3 = 2;  // MOFFT_FORM_BF16X3

namespace tc {

constexpr int kN = 4096;
constexpr int kR = 16;
constexpr int kBF = kN / kR;              // 256 butterflies per stage
constexpr int kThreads = 256;
constexpr int kTmemCols = 64;             // two 128 x 32 FP32 accumulators
constexpr unsigned kMaxWaitIters = 1u << 24;
constexpr uint64_t kWaitNs = 1000000000ull;  // one second

template <int FORM> struct FormTraits;
template <> struct FormTraits<kFormTf32x3> {
  static constexpr int kElemBytes = 4;
  static constexpr int kKPerInstr = 8;    // 32 bytes of K per row per MMA
  static constexpr uint32_t kFormat = 2;  // TF32
};
template <> struct FormTraits<kFormBf16x3> {
  static constexpr int kElemBytes = 2;
  static constexpr int kKPerInstr = 16;
  static constexpr uint32_t kFormat = 1;  // BF16
};

// Shared memory plan (bytes).  Tiles are 1024-byte aligned.
template <int FORM>
struct Smem {
  static constexpr int kSteps = 32 / FormTraits<FORM>::kKPerInstr;
  static constexpr int kATile = 128 * 32;                 // one M=128 tile, one K-step
  static constexpr int kAHalf = 2 * kSteps * kATile;      // both M tiles, all K-steps
  static constexpr int kBTile = 32 * 32;                  // N=32 rows, one K-step
  static constexpr int kBHalf = kSteps * kBTile;
  static constexpr int kData = 2 * spad_len<float>(kN) * 4;
  static constexpr int kOffAHi = 0;
  static constexpr int kOffALo = kOffAHi + kAHalf;
  static constexpr int kOffBHi = kOffALo + kAHalf;
  static constexpr int kOffBLo = kOffBHi + kBHalf;
  static constexpr int kOffData = kOffBLo + kBHalf;
  static constexpr int kOffBar = (kOffData + kData + 15) & ~15;
  static constexpr int kOffTmem = kOffBar + 8;
  static constexpr int kBytes = kOffTmem + 16 + 1024;     // + alignment slack
};

// Byte offset of element (row, kk) of a K-major, no-swizzle operand tile of
// one K-step: 8-row core matrices of 16-byte rows; the two 16-byte K chunks
// of a core-matrix group are 128 bytes apart (LBO) and 8-row groups 256 bytes
// apart (SBO).
__device__ __forceinline__ int canon_offset(int row, int kbyte) {
  return (row >> 3) * 256 + (kbyte >> 4) * 128 + (row & 7) * 16 + (kbyte & 15);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);          // start address
  d |= (uint64_t)(128 >> 4) << 16;                // leading byte offset (K chunk)
  d |= (uint64_t)(256 >> 4) << 32;                // stride byte offset (8 rows)
  d |= (uint64_t)1 << 46;                         // descriptor version (sm100)
  return d;                                       // base offset 0, no swizzle
}

template <int FORM>
__device__ __forceinline__ uint32_t instr_desc() {
  constexpr uint32_t fmt = FormTraits<FORM>::kFormat;
  return (1u << 4)            // D format F32
         | (fmt << 7)         // A format
         | (fmt << 10)        // B format
         | ((32u >> 3) << 17) // N = 32
         | ((128u >> 4) << 24);  // M = 128
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

template <int FORM>
__device__ __forceinline__ void split_store(unsigned char *hi_tile, unsigned char *lo_tile,
                                            int row, const float (&v)[32]);

template <>
__device__ __forceinline__ void split_store<kFormTf32x3>(unsigned char *hi_base,
                                                         unsigned char *lo_base, int row,
                                                         const float (&v)[32]) {
  // 4 K-steps of 8 values, each two 16-byte chunks
#pragma unroll
  for (int s = 0; s < 4; ++s) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      uint32_t h[4], l[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float x = v[s * 8 + c * 4 + e];
        h[e] = to_tf32(x);
        l[e] = to_tf32(x - __uint_as_float(h[e]));
      }
      const int off = s * Smem<kFormTf32x3>::kATile * 2 + canon_offset(row, c * 16);
      *reinterpret_cast<uint4 *>(hi_base + off) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4 *>(lo_base + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
  }
}

template <>
__device__ __forceinline__ void split_store<kFormBf16x3>(unsigned char *hi_base,
                                                         unsigned char *lo_base, int row,
                                                         const float (&v)[32]) {
  // 2 K-steps of 16 values, each two 16-byte chunks of 8 bf16
#pragma unroll
  for (int s = 0; s < 2; ++s) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      uint32_t h[4], l[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float x0 = v[s * 16 + c * 8 + 2 * e];
        const float x1 = v[s * 16 + c * 8 + 2 * e + 1];
        const __nv_bfloat16 h0 = __float2bfloat16_rn(x0);
        const __nv_bfloat16 h1 = __float2bfloat16_rn(x1);
        const __nv_bfloat16 l0 = __float2bfloat16_rn(x0 - __bfloat162float(h0));
        const __nv_bfloat16 l1 = __float2bfloat16_rn(x1 - __bfloat162float(h1));
        h[e] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
        l[e] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
      }
      const int off = s * Smem<kFormBf16x3>::kATile * 2 + canon_offset(row, c * 16);
      *reinterpret_cast<uint4 *>(hi_base + off) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4 *>(lo_base + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
  }
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the completion of the mbarrier phase of `parity`: gives up
// after kWaitNs of wall time (or kMaxWaitIters polls) and returns false.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const uint64_t t0 = global_ns();
  for (unsigned it = 0; it < kMaxWaitIters; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if ((it & 63u) == 63u && global_ns() - t0 > kWaitNs) return false;
  }
  return false;
}

template <int FORM>
__device__ __forceinline__ void issue_mmas(uint32_t tmem_d, uint32_t a_hi, uint32_t a_lo,
                                           uint32_t b_hi, uint32_t b_lo) {
  constexpr int kSteps = Smem<FORM>::kSteps;
  const uint32_t idesc = instr_desc<FORM>();
#pragma unroll
  for (int tile = 0; tile < 2; ++tile) {
    const uint32_t d = tmem_d + tile * 32;   // column offset of this M tile
    int first = 1;
#pragma unroll
    for (int term = 0; term < 3; ++term) {
      // term 0: A_lo*B_hi, 1: A_hi*B_lo, 2: A_hi*B_hi (small terms first)
      const uint32_t abase = term == 0 ? a_lo : a_hi;
      const uint32_t bbase = term == 1 ? b_lo : b_hi;
#pragma unroll
      for (int s = 0; s < kSteps; ++s) {
        const uint64_t da = smem_desc(abase + (uint32_t)((s * 2 + tile) * Smem<FORM>::kATile));
        const uint64_t db = smem_desc(bbase + (uint32_t)(s * Smem<FORM>::kBTile));
        const uint32_t accumulate = first ? 0u : 1u;
        first = 0;
        if constexpr (FORM == kFormTf32x3) {
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
              :
              : "r"(d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
              : "memory");
        } else {
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
              :
              : "r"(d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
              : "memory");
        }
      }
    }
  }
}

struct TcArgs {
  const float2 *in;
  float2 *out;
  const float2 *tw;          // stage twiddles of the chain [16, 16, 16]
  const unsigned char *bmat; // B tiles (hi then lo), laid out as in shared memory
  int *status;               // set to 1 when a wait timed out
  long long in_dist;
  long long out_dist;
  float sign;                // -1: conjugate on load and store (backward)
};

template <int FORM>
__global__ void __launch_bounds__(kThreads, 2) tc_fft4096_kernel(const TcArgs a) {
  using S = Smem<FORM>;
  extern __shared__ unsigned char smem_raw[];
  // 1024-byte align the tile area
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char *a_hi = base + S::kOffAHi;
  unsigned char *a_lo = base + S::kOffALo;
  unsigned char *b_hi = base + S::kOffBHi;
  float *sre = reinterpret_cast<float *>(base + S::kOffData);
  float *sim = sre + spad_len<float>(kN);
  uint64_t *bar = reinterpret_cast<uint64_t *>(base + S::kOffBar);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(base + S::kOffTmem);
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const long long b = blockIdx.x;

  // B tiles: the constant DFT matrix, copied from global memory
  for (int i = tid; i < 2 * S::kBHalf / 16; i += kThreads)
    reinterpret_cast<uint4 *>(b_hi)[i] = __ldg(reinterpret_cast<const uint4 *>(a.bmat) + i);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(1)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t bar_addr = smem_u32(bar);
  const float2 *gin = a.in + b * a.in_dist;
  float2 *gout = a.out + b * a.out_dist;

  const int j = tid;        // this thread's butterfly = its row of A and D
  const int tile = j >> 7;  // M tile; the row inside it is 32 * (warp & 3) + lane
  const uint32_t tmem_row = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(tile * 32);
  int twoff = 0;
  bool failed = false;
  int issued_parity = -1;   // parity of the last committed, not yet observed MMA group
#pragma unroll 1
  for (int stage = 0; stage < 3; ++stage) {
    const int lg = 4 * stage;  // log2 of Ns
    const int ns = 1 << lg;
    float v[32];
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const int idx = j + r * kBF;
      if (stage == 0) {
        const float2 x = __ldcg(gin + idx);
        v[r] = x.x;
        v[16 + r] = x.y * a.sign;
      } else {
        v[r] = sre[spad<float>(idx)];
        v[16 + r] = sim[spad<float>(idx)];
      }
    }
    const int jm = j & (ns - 1);
    if (ns > 1) {
#pragma unroll
      for (int r = 1; r < kR; ++r) {
        const float2 w = __ldg(a.tw + twoff + (r - 1) * ns + jm);
        cmul<float>(v[r], v[16 + r], w.x, w.y);
      }
      twoff += (kR - 1) * ns;
    }
    split_store<FORM>(a_hi + (size_t)tile * S::kATile, a_lo + (size_t)tile * S::kATile,
                      j & 127, v);
    // make the generic-proxy stores visible to the tensor core, then hand
    // the operands to the issuing thread
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      issue_mmas<FORM>(tmem, smem_u32(a_hi), smem_u32(a_lo), smem_u32(b_hi),
                       smem_u32(b_hi) + S::kBHalf);
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              bar_addr)
          : "memory");
    }
    issued_parity = stage & 1;
    const bool ok = mbar_wait(bar_addr, (uint32_t)(stage & 1));
    if (__syncthreads_or(!ok)) {  // uniform across the CTA
      failed = true;
      break;
    }
    issued_parity = -1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    uint32_t d[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]),
          "=r"(d[6]), "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]),
          "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]), "=r"(d[16]), "=r"(d[17]),
          "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]),
          "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]),
          "=r"(d[30]), "=r"(d[31])
        : "r"(tmem_row)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    // Stockham scatter: y[(j / Ns) Ns R + j mod Ns + k Ns] = D[j][k]
    const int basei = ((j >> lg) << (lg + 4)) + jm;
    if (stage < 2) {
#pragma unroll
      for (int k = 0; k < kR; ++k) {
        const int idx = basei + k * ns;
        sre[spad<float>(idx)] = __uint_as_float(d[k]);
        sim[spad<float>(idx)] = __uint_as_float(d[16 + k]);
      }
      __syncthreads();
    } else {
#pragma unroll
      for (int k = 0; k < kR; ++k) {
        float2 o;
        o.x = __uint_as_float(d[k]);
        o.y = __uint_as_float(d[16 + k]) * a.sign;
        gout[basei + k * ns] = o;
      }
    }
  }
  if (failed) {
    if (tid == 0) atomicExch(a.status, 1);
    // one more bounded wait for the MMAs still in flight before the TMEM
    // they write is released
    if (issued_parity >= 0) (void)mbar_wait(bar_addr, (uint32_t)issued_parity);
  }
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

template <int FORM>
struct TcInst {
  static constexpr size_t smem() { return (size_t)Smem<FORM>::kBytes; }
  static const void *func() {
    return reinterpret_cast<const void *>(&tc_fft4096_kernel<FORM>);
  }
  static cudaError_t launch(const mofft_pass_args *p, cudaStream_t s) {
    if (p->conj_in != p->conj_out) return cudaErrorInvalidValue;
    if (p->in_table || p->out_table) return cudaErrorNotSupported;
    if (!p->aux || !p->status) return cudaErrorInvalidValue;
    if (p->batch <= 0) return cudaSuccess;
    if (p->batch > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    TcArgs a;
    a.in = static_cast<const float2 *>(p->in);
    a.out = static_cast<float2 *>(p->out);
    a.tw = static_cast<const float2 *>(p->tw);
    a.bmat = static_cast<const unsigned char *>(p->aux);
    a.status = p->status;
    a.in_dist = p->in_dist;
    a.out_dist = p->out_dist;
    a.sign = p->conj_in ? -1.0f : 1.0f;
    tc_fft4096_kernel<FORM><<<(unsigned)p->batch, kThreads, smem(), s>>>(a);
    return cudaGetLastError();
  }
  static Entry entry(const char *name) {
    Entry e;
    e.desc.name = name;
    e.desc.precision_bits = 32;
    e.desc.kind = MOFFT_KERNEL_TENSOR;
    e.desc.length = kN;
    e.desc.lines = 1;
    e.desc.threads = kThreads;
    e.desc.staged = 0;
    e.desc.radix_count = 3;
    for (int i = 0; i < 8; ++i) e.desc.radices[i] = i < 3 ? kR : 0;
    e.desc.smem_bytes = smem();
    e.desc.form = FORM;
    e.launch = &launch;
    e.func = &func;
    return e;
  }
};

// ---- host side: the B operand tables ------------------------------------

static uint32_t host_f32_bits(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  return u;
}

static float host_bits_f32(uint32_t u) {
  float x;
  memcpy(&x, &u, 4);
  return x;
}

// round to nearest, ties away from zero, keeping 10 explicit mantissa bits
static float host_tf32(double x) {
  uint32_t u = host_f32_bits((float)x);
  u = (u + 0x1000u) & 0xFFFFE000u;
  return host_bits_f32(u);
}

// round to nearest even bfloat16; returns the 16-bit pattern
static uint16_t host_bf16(double x, double *value) {
  const uint32_t u = host_f32_bits((float)x);
  const uint32_t r = (u + 0x7FFFu + ((u >> 16) & 1u)) >> 16;
  *value = (double)host_bits_f32(r << 16);
  return (uint16_t)r;
}

static int host_canon_offset(int row, int kbyte) {
  return (row >> 3) * 256 + (kbyte >> 4) * 128 + (row & 7) * 16 + (kbyte & 15);
}

}  // namespace tc

const Entry *entries_tensor(int *n) {
  static const Entry e[] = {
      tc::TcInst<kFormTf32x3>::entry("tensor_float_4096_tf32x3_r16x3"),
      tc::TcInst<kFormBf16x3>::entry("tensor_float_4096_bf16x3_r16x3"),
  };
  *n = (int)(sizeof(e) / sizeof(e[0]));
  return e;
}

}  // namespace mofft

using namespace mofft;

extern "C" size_t mofft_cuda_tensor_aux_bytes(int form) {
  if (form == kFormTf32x3) return 2 * (size_t)tc::Smem<kFormTf32x3>::kBHalf;
  if (form == kFormBf16x3) return 2 * (size_t)tc::Smem<kFormBf16x3>::kBHalf;
  return 0;
}

// B[n][kk] of the real 32 x 32 form of the forward 16-point DFT F (fr + i fi,
// row-major F[k][r]): n < 16 gives Re(F v)_n, n = 16 + k gives Im(F v)_k for
// v = (v_re[0..15], v_im[0..15]).  Written as hi tiles then lo tiles, one
// K-major no-swizzle tile of 32 rows per K-step.
extern "C" int mofft_cuda_tensor_fill_aux(int form, void *dst, const double *fr,
                                          const double *fi) {
  if (form != kFormTf32x3 && form != kFormBf16x3) return (int)cudaErrorInvalidValue;
  unsigned char *out = static_cast<unsigned char *>(dst);
  const int kper = form == kFormTf32x3 ? 8 : 16;
  const int elem = form == kFormTf32x3 ? 4 : 2;
  const size_t half = mofft_cuda_tensor_aux_bytes(form) / 2;
  memset(out, 0, 2 * half);
  for (int n = 0; n < 32; ++n) {
    for (int kk = 0; kk < 32; ++kk) {
      const int k = n & 15, r = kk & 15;
      double x;
      if (n < 16) x = kk < 16 ? fr[k * 16 + r] : -fi[k * 16 + r];
      else x = kk < 16 ? fi[k * 16 + r] : fr[k * 16 + r];
      const int step = kk / kper;
      const int kbyte = (kk % kper) * elem;
      const size_t off = (size_t)step * 1024 + (size_t)tc::host_canon_offset(n, kbyte);
      if (form == kFormTf32x3) {
        const float hi = tc::host_tf32(x);
        const float lo = tc::host_tf32(x - (double)hi);
        memcpy(out + off, &hi, 4);
        memcpy(out + half + off, &lo, 4);
      } else {
        double hv, lv;
        const uint16_t hb = tc::host_bf16(x, &hv);
        const uint16_t lb = tc::host_bf16(x - hv, &lv);
        memcpy(out + off, &hb, 2);
        memcpy(out + half + off, &lb, 2);
      }
    }
  }
  return 0;
}
