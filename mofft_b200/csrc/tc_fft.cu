// Tensor-core precision forms of the FP32 transform (tcgen05, sm_100a).
//
// n = 4096 = 16^3 as three radix-16 Stockham stages, each a DFT-matrix GEMM
// on the 5th-generation tensor cores.  A stage over the 256 butterflies of a
// transform is the real GEMM
//
//     D[j][n] = sum_kk A[j][kk] * B[n][kk],   j < 256, n < 32, kk < 32,
//
// where row j of A holds butterfly j's twiddled inputs (16 real parts, then
// 16 imaginary parts) and B is the real form of the 16-point DFT matrix F:
// rows n < 16 give Re(F v)_n = sum Fr v_re - Fi v_im, rows 16 + k give
// Im(F v)_k = sum Fi v_re + Fr v_im.  M = 256 runs as two M = 128 MMAs; A
// and the accumulators D live in tensor memory (TMEM), B (constant, K-major,
// no swizzle) in shared memory.
//
// Split precision (FP32 accumulate):
//   3xTF32:  x = hi + lo with hi = tf32(x), lo = tf32(x - hi) (about 21
//            significant bits); A*B ~ A_lo*B_hi + A_hi*B_lo + A_hi*B_hi.
//   BF16x3:  the same with bfloat16 pieces (about 16 significant bits).
// The small terms are accumulated first.
//
// Persistent CTAs of 256 threads (one per butterfly) loop over transforms.
// A transform's 32 KB arrive in shared memory by one bulk asynchronous copy
// issued while the previous transform is still in its stages 1-2.  Per stage
// each thread gathers its 16 inputs from shared memory, twiddles and splits
// them and writes its A rows to its own TMEM lane (tcgen05.st); one thread
// issues the MMAs and commits them to an mbarrier; each thread reads its D
// row back (tcgen05.ld) and scatters the 16 outputs with the Stockham index
// map (to shared memory, or to global memory after the last stage).  Shared
// memory traffic per stage is one gather and one scatter, as in the CUDA-core
// kernel; the butterfly arithmetic moves to the tensor cores.
//
// Every wait (copy arrival, MMA completion) is bounded by one second of wall
// time.  On a timeout the CTA stops, records the error word, waits (again
// bounded) for its own copy and MMAs in flight, frees its TMEM and returns;
// the host reports MOFFT_INTERNAL_ERROR.
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

template <int FORM> struct FormTraits;
template <> struct FormTraits<kFormTf32x3> {
  static constexpr int kKPerInstr = 8;    // 32 bytes of K per row per MMA
  static constexpr uint32_t kFormat = 2;  // TF32
  static constexpr int kACols = 32;       // TMEM columns of one A tile (K = 32)
  static constexpr int kTmemCols = 256;   // D 64 + A_hi 64 + A_lo 64, rounded
  static constexpr int kMinBlocks = 2;
};
template <> struct FormTraits<kFormBf16x3> {
  static constexpr int kKPerInstr = 16;
  static constexpr uint32_t kFormat = 1;  // BF16
  static constexpr int kACols = 16;       // two bf16 per 32-bit column
  static constexpr int kTmemCols = 128;   // D 64 + A_hi 32 + A_lo 32
  static constexpr int kMinBlocks = 2;
};

// Shared memory plan (bytes, from a 1024-byte aligned base) and TMEM columns.
template <int FORM>
struct Plan {
  using F = FormTraits<FORM>;
  static constexpr int kSteps = 32 / F::kKPerInstr;       // MMAs per term per tile
  static constexpr int kBTile = 32 * 32;                  // N = 32 rows, one K-step
  static constexpr int kBHalf = kSteps * kBTile;          // hi (or lo) B tiles
  static constexpr int kIn = kN * 8;                      // one transform, interleaved
  static constexpr int kData = 2 * spad_len<float>(kN) * 4;
  static constexpr int kOffIn = 0;
  static constexpr int kOffB = kOffIn + kIn;
  static constexpr int kOffData = kOffB + 2 * kBHalf;
  static constexpr int kOffBar = (kOffData + kData + 15) & ~15;  // [0] MMA, [1] copy
  static constexpr int kOffTmem = kOffBar + 16;
  static constexpr int kBytes = kOffTmem + 16 + 1024;     // + alignment slack
  static constexpr uint32_t kColD = 0;                    // D tile t at 32 t
  static constexpr uint32_t kColAHi = 64;                 // A_hi tile t at 64 + kACols t
  static constexpr uint32_t kColALo = 64 + 2 * F::kACols;
};

// Shared-memory descriptor of a K-major, no-swizzle operand tile of one
// K-step: 8-row core matrices of 16-byte rows; the two 16-byte K chunks are
// 128 bytes apart (leading byte offset), 8-row groups 256 bytes apart
// (stride byte offset).
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
  return (1u << 4)               // D format F32
         | (fmt << 7)            // A format
         | (fmt << 10)           // B format
         | ((32u >> 3) << 17)    // N = 32
         | ((128u >> 4) << 24);  // M = 128; A and B K-major
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b, float *ra, float *rb) {
  const __nv_bfloat16 ha = __float2bfloat16_rn(a);
  const __nv_bfloat16 hb = __float2bfloat16_rn(b);
  *ra = a - __bfloat162float(ha);
  *rb = b - __bfloat162float(hb);
  return (uint32_t)__bfloat16_as_ushort(ha) | ((uint32_t)__bfloat16_as_ushort(hb) << 16);
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
      "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]),
      "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]),
      "r"(r[14]), "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]),
      "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]),
      "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
      : "memory");
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
      "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]),
      "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]),
      "r"(r[14]), "r"(r[15])
      : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&d)[32]) {
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
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Split this thread's 32 operand values and write them to its TMEM lane:
// A_hi of its tile at a_hi, A_lo at a_lo (column addresses of this lane).
template <int FORM>
__device__ __forceinline__ void store_split(uint32_t a_hi, uint32_t a_lo, const float (&v)[32]);

template <>
__device__ __forceinline__ void store_split<kFormTf32x3>(uint32_t a_hi, uint32_t a_lo,
                                                         const float (&v)[32]) {
  uint32_t h[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) h[i] = to_tf32(v[i]);
  tmem_st32(a_hi, h);
#pragma unroll
  for (int i = 0; i < 32; ++i) h[i] = to_tf32(v[i] - __uint_as_float(h[i]));
  tmem_st32(a_lo, h);
}

template <>
__device__ __forceinline__ void store_split<kFormBf16x3>(uint32_t a_hi, uint32_t a_lo,
                                                         const float (&v)[32]) {
  uint32_t h[16], l[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    float ra, rb, da, db;
    h[i] = pack_bf16(v[2 * i], v[2 * i + 1], &ra, &rb);
    l[i] = pack_bf16(ra, rb, &da, &db);
  }
  tmem_st16(a_hi, h);
  tmem_st16(a_lo, l);
}

// Waits and copies: line_wait (bounded mbarrier wait, one second of
// %globaltimer) and line_copy (one bulk asynchronous copy of a transform's
// 32 KB, no multicast) of fft_device.cuh.

template <int FORM>
__device__ __forceinline__ void issue_mmas(uint32_t tmem, uint32_t b_hi, uint32_t b_lo) {
  using P = Plan<FORM>;
  constexpr int kSteps = P::kSteps;
  constexpr uint32_t kColsPerStep = FormTraits<FORM>::kACols / kSteps;
  const uint32_t idesc = instr_desc<FORM>();
#pragma unroll
  for (int tile = 0; tile < 2; ++tile) {
    const uint32_t d = tmem + P::kColD + 32u * tile;
    const uint32_t ahi = tmem + P::kColAHi + (uint32_t)(FormTraits<FORM>::kACols * tile);
    const uint32_t alo = tmem + P::kColALo + (uint32_t)(FormTraits<FORM>::kACols * tile);
    int first = 1;
#pragma unroll
    for (int term = 0; term < 3; ++term) {
      // term 0: A_lo*B_hi, 1: A_hi*B_lo, 2: A_hi*B_hi (small terms first)
      const uint32_t abase = term == 0 ? alo : ahi;
      const uint32_t bbase = term == 1 ? b_lo : b_hi;
#pragma unroll
      for (int s = 0; s < kSteps; ++s) {
        const uint32_t ta = abase + kColsPerStep * s;
        const uint64_t db = smem_desc(bbase + (uint32_t)(s * P::kBTile));
        const uint32_t accumulate = first ? 0u : 1u;
        first = 0;
        if constexpr (FORM == kFormTf32x3) {
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}"
              :
              : "r"(d), "r"(ta), "l"(db), "r"(idesc), "r"(accumulate)
              : "memory");
        } else {
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}"
              :
              : "r"(d), "r"(ta), "l"(db), "r"(idesc), "r"(accumulate)
              : "memory");
        }
      }
    }
  }
}

// v[r] *= w^r (r = 1..15; v holds 16 real parts then 16 imaginary parts)
// from the table entries of w, w^2, w^4 and w^8 (row r - 1 of the stage table
// starts at tw + (r - 1) * ns); the other powers are products of at most
// three of them.
__device__ __forceinline__ void twiddle16(float (&v)[32], const float2 *__restrict__ tw,
                                          int ns) {
  float wr[16], wi[16];
  const float2 a1 = __ldg(tw);
  const float2 a2 = __ldg(tw + ns);
  const float2 a4 = __ldg(tw + 3 * ns);
  const float2 a8 = __ldg(tw + 7 * ns);
  wr[1] = a1.x; wi[1] = a1.y;
  wr[2] = a2.x; wi[2] = a2.y;
  wr[4] = a4.x; wi[4] = a4.y;
  wr[8] = a8.x; wi[8] = a8.y;
  constexpr int kPairs[11][3] = {{3, 2, 1},  {5, 4, 1},  {6, 4, 2},  {7, 4, 3},
                                 {9, 8, 1},  {10, 8, 2}, {11, 8, 3}, {12, 8, 4},
                                 {13, 8, 5}, {14, 8, 6}, {15, 8, 7}};
#pragma unroll
  for (int i = 0; i < 11; ++i) {
    const int d = kPairs[i][0], x = kPairs[i][1], y = kPairs[i][2];
    wr[d] = wr[x] * wr[y] - wi[x] * wi[y];
    wi[d] = wr[x] * wi[y] + wi[x] * wr[y];
  }
#pragma unroll
  for (int r = 1; r < 16; ++r) cmul<float>(v[r], v[16 + r], wr[r], wi[r]);
}

struct TcArgs {
  const float2 *in;
  float2 *out;
  const float2 *tw;          // stage twiddles of the chain [16, 16, 16]
  const unsigned char *bmat; // B tiles (hi then lo), laid out as in shared memory
  int *status;               // set to 1 when a wait timed out
  long long batch;
  long long in_dist;
  long long out_dist;
  float sign;                // -1: conjugate on load and store (backward)
  int bulk;                  // 1: inputs 16-byte aligned, bulk copies allowed
  int lose_copy;             // failure check: the first copy is never issued
};

template <int FORM>
__global__ void __launch_bounds__(kThreads, FormTraits<FORM>::kMinBlocks)
    tc_fft4096_kernel(const TcArgs a) {
  using P = Plan<FORM>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const float2 *s_in = reinterpret_cast<const float2 *>(base + P::kOffIn);
  unsigned char *b_tiles = base + P::kOffB;
  float *sre = reinterpret_cast<float *>(base + P::kOffData);
  float *sim = sre + spad_len<float>(kN);
  uint64_t *bars = reinterpret_cast<uint64_t *>(base + P::kOffBar);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(base + P::kOffTmem);
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const uint32_t mma_bar = smem_u32(&bars[0]);
  const uint32_t load_bar = smem_u32(&bars[1]);
  const uint32_t in_addr = smem_u32(base + P::kOffIn);

  for (int i = tid; i < 2 * P::kBHalf / 16; i += kThreads)
    reinterpret_cast<uint4 *>(b_tiles)[i] = __ldg(reinterpret_cast<const uint4 *>(a.bmat) + i);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mma_bar), "r"(1) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(load_bar), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(FormTraits<FORM>::kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // B tiles are read by the tensor core: order the generic stores first
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  if (a.bulk && !a.lose_copy && tid == 0 && (long long)blockIdx.x < a.batch)
    line_copy(in_addr, a.in + (long long)blockIdx.x * a.in_dist, kN * 8, load_bar);

  const int j = tid;        // this thread's butterfly = its row of A and D
  const int tile = j >> 7;  // M tile; the TMEM lane is j & 127 = 32 (warp & 3) + lane
  const uint32_t lane_off = (uint32_t)(32 * (warp & 3)) << 16;
  const uint32_t t_d = tmem + lane_off + P::kColD + 32u * tile;
  const uint32_t t_hi = tmem + lane_off + P::kColAHi + (uint32_t)(FormTraits<FORM>::kACols * tile);
  const uint32_t t_lo = tmem + lane_off + P::kColALo + (uint32_t)(FormTraits<FORM>::kACols * tile);
  const uint32_t b_hi = smem_u32(b_tiles);
  const uint32_t b_lo = b_hi + P::kBHalf;

  bool failed = false;
  int load_pending = a.bulk && (long long)blockIdx.x < a.batch;  // thread 0's view
  uint32_t mma_phase = 0;
  int mma_pending = 0;
  uint32_t load_phase = 0;
#pragma unroll 1
  for (long long b = blockIdx.x; b < a.batch; b += gridDim.x) {
    const float2 *gin = a.in + b * a.in_dist;
    float2 *gout = a.out + b * a.out_dist;
    if (a.bulk) {
      const bool ok = line_wait(load_bar, load_phase);
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      load_phase ^= 1u;
      load_pending = 0;
    }
    int twoff = 0;
#pragma unroll 1
    for (int stage = 0; stage < 3; ++stage) {
      const int lg = 4 * stage;  // log2 of Ns
      const int ns = 1 << lg;
      const int jm = j & (ns - 1);
      float v[32];
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        const int idx = j + r * kBF;
        if (stage == 0) {
          const float2 x = a.bulk ? s_in[idx] : __ldcg(gin + idx);
          v[r] = x.x;
          v[16 + r] = x.y * a.sign;
        } else {
          v[r] = sre[spad<float>(idx)];
          v[16 + r] = sim[spad<float>(idx)];
        }
      }
      if (ns > 1) {
        twiddle16(v, a.tw + twoff + jm, ns);
        twoff += (kR - 1) * ns;
      }
      store_split<FORM>(t_hi, t_lo, v);
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        issue_mmas<FORM>(tmem, b_hi, b_lo);
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                mma_bar)
            : "memory");
        if (stage == 0 && a.bulk && b + gridDim.x < a.batch) {
          // every thread has read this transform's input: prefetch the next
          line_copy(in_addr, a.in + (b + gridDim.x) * a.in_dist, kN * 8, load_bar);
          load_pending = 1;
        }
      }
      mma_pending = 1;
      const bool ok = line_wait(mma_bar, mma_phase);
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      mma_phase ^= 1u;
      mma_pending = 0;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint32_t d[32];
      tmem_ld32(t_d, d);
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
      } else {
#pragma unroll
        for (int k = 0; k < kR; ++k) {
          float2 o;
          o.x = __uint_as_float(d[k]);
          o.y = __uint_as_float(d[16 + k]) * a.sign;
          __stcs(gout + basei + k * ns, o);
        }
      }
      __syncthreads();
    }
    if (failed) break;
  }
  if (failed) {
    if (tid == 0) {
      atomicExch(a.status, 1);
      // bounded waits for this CTA's own work in flight before its shared
      // memory and TMEM are released
      if (mma_pending) (void)line_wait(mma_bar, mma_phase);
      if (load_pending) (void)line_wait(load_bar, load_phase);
    }
  }
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(FormTraits<FORM>::kTmemCols)
                 : "memory");
  }
}

template <int FORM>
struct TcInst {
  static constexpr size_t smem() { return (size_t)Plan<FORM>::kBytes; }
  static const void *func() {
    return reinterpret_cast<const void *>(&tc_fft4096_kernel<FORM>);
  }
  // Resident CTAs per SM (registers, shared memory, threads and the TMEM
  // columns each CTA allocates) times the SM count; cached per device.
  static int persistent_grid() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (cached[dev] > 0) return cached[dev];
    cudaFuncAttributes fa;
    int sms = 0, regs_sm = 0, smem_sm = 0, reserved = 0, threads_sm = 0;
    if (cudaFuncGetAttributes(&fa, tc_fft4096_kernel<FORM>) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) !=
            cudaSuccess)
      return 0;
    const int warp_regs = ((fa.numRegs * 32 + 255) / 256) * 256;  // per-warp granule
    int per_sm = regs_sm / (warp_regs * (kThreads / 32));
    const int by_smem = smem_sm / ((int)smem() + reserved);
    const int by_threads = threads_sm / kThreads;
    const int by_tmem = 512 / FormTraits<FORM>::kTmemCols;
    if (by_smem < per_sm) per_sm = by_smem;
    if (by_threads < per_sm) per_sm = by_threads;
    if (by_tmem < per_sm) per_sm = by_tmem;
    if (per_sm < 1) per_sm = 1;
    cached[dev] = per_sm * sms;
    return cached[dev];
  }
  static cudaError_t launch(const mofft_pass_args *p, cudaStream_t s) {
    if (p->conj_in != p->conj_out) return cudaErrorInvalidValue;
    if (p->in_table || p->out_table) return cudaErrorNotSupported;
    if (!p->aux || !p->status) return cudaErrorInvalidValue;
    if (p->batch <= 0) return cudaSuccess;
    const int resident = persistent_grid();
    if (resident <= 0) return cudaErrorInvalidConfiguration;
    TcArgs a;
    a.in = static_cast<const float2 *>(p->in);
    a.out = static_cast<float2 *>(p->out);
    a.tw = static_cast<const float2 *>(p->tw);
    a.bmat = static_cast<const unsigned char *>(p->aux);
    a.status = p->status;
    a.batch = p->batch;
    a.in_dist = p->in_dist;
    a.out_dist = p->out_dist;
    a.sign = p->conj_in ? -1.0f : 1.0f;
    // bulk copies need 16-byte aligned sources: an aligned base and an even
    // distance (complex64 elements are 8 bytes)
    a.bulk = ((reinterpret_cast<uintptr_t>(p->in) & 15u) == 0 && (p->in_dist % 2) == 0) ? 1 : 0;
    a.lose_copy = p->lose_copy;
    const long long grid = p->batch < resident ? p->batch : resident;
    tc_fft4096_kernel<FORM><<<(unsigned)grid, kThreads, smem(), s>>>(a);
    return cudaGetLastError();
  }
  static Entry entry(const char *name) {
    Entry e{};
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

// ---------------------------------------------------------------------------
// Column passes on the tensor cores: one pass of a four-step transform whose
// lines have 256 = 16 x 16 points (n = 65536 runs two of them).  A tile is 16
// adjacent lines of one batch entry; its 256 butterflies per stage (16 per
// line) are the 256 rows of the same GEMMs as above.  Thread j owns line
// c = j mod 16 and butterfly bb = j / 16, so that consecutive threads read
// consecutive lines: every global access is a 16-element (128-byte) run.
// Pass with Ns = 1: outputs are staged in shared memory and the tile (16
// whole lines, contiguous) is written with coalesced stores; pass with
// Ns > 1: the super-stage twiddle W_{Ns 256}^{(line mod Ns) i} is applied on
// load from the two-level table and outputs go to y[line + k Ns].
// ---------------------------------------------------------------------------
constexpr int kColsL = 256;
constexpr int kColsC = 16;
constexpr int kColsPitch = kColsL + kColsL / 32 + 1;   // padded words per line

template <int FORM>
struct ColsPlan {
  using F = FormTraits<FORM>;
  static constexpr int kBHalf = Plan<FORM>::kBHalf;
  static constexpr int kData = 2 * kColsC * kColsPitch * 4;
  static constexpr int kOffB = 0;
  static constexpr int kOffData = kOffB + 2 * kBHalf;
  static constexpr int kOffBar = (kOffData + kData + 15) & ~15;
  static constexpr int kOffTmem = kOffBar + 16;
  static constexpr int kBytes = kOffTmem + 16 + 1024;
};

struct TcColsArgs {
  const float2 *in;
  float2 *out;
  const float2 *tw;          // stage table of the 256-point line [16, 16]
  const float2 *tw_hi;       // super-stage twiddle, two-level table
  const float2 *tw_lo;
  const unsigned char *bmat;
  int *status;
  long long batch;
  long long in_dist;
  long long out_dist;
  long long total;           // transform length M
  long long ns;              // Ns of this pass (1 or a multiple of 16)
  int split_shift;
  float sign_in;
  float sign_out;
};

__device__ __forceinline__ int cpad(int i) { return i + (i >> 5); }

template <int FORM>
__global__ void __launch_bounds__(kThreads, FormTraits<FORM>::kMinBlocks)
    tc_cols256_kernel(const TcColsArgs a) {
  using P = ColsPlan<FORM>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char *b_tiles = base + P::kOffB;
  float *sre = reinterpret_cast<float *>(base + P::kOffData);
  float *sim = sre + kColsC * kColsPitch;
  uint64_t *bars = reinterpret_cast<uint64_t *>(base + P::kOffBar);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(base + P::kOffTmem);
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const uint32_t mma_bar = smem_u32(&bars[0]);

  for (int i = tid; i < 2 * P::kBHalf / 16; i += kThreads)
    reinterpret_cast<uint4 *>(b_tiles)[i] = __ldg(reinterpret_cast<const uint4 *>(a.bmat) + i);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mma_bar), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(FormTraits<FORM>::kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const int j = tid;
  const int c = j & (kColsC - 1);   // line within the tile
  const int bb = j >> 4;            // butterfly within the line
  const int tile_row = j >> 7;
  const uint32_t lane_off = (uint32_t)(32 * (warp & 3)) << 16;
  const uint32_t t_d = tmem + lane_off + Plan<FORM>::kColD + 32u * tile_row;
  const uint32_t t_hi =
      tmem + lane_off + Plan<FORM>::kColAHi + (uint32_t)(FormTraits<FORM>::kACols * tile_row);
  const uint32_t t_lo =
      tmem + lane_off + Plan<FORM>::kColALo + (uint32_t)(FormTraits<FORM>::kACols * tile_row);
  const uint32_t b_hi = smem_u32(b_tiles);
  const uint32_t b_lo = b_hi + P::kBHalf;
  const long long lines_total = a.total / kColsL;
  const long long groups = lines_total / kColsC;
  const long long tiles = a.batch * groups;
  const long long mask = (1LL << a.split_shift) - 1;

  bool failed = false;
  int mma_pending = 0;
  uint32_t mma_phase = 0;
#pragma unroll 1
  for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const long long b = tile / groups;
    const long long line0 = (tile - b * groups) * kColsC;
    const long long line = line0 + c;
    const long long jq = line / a.ns;
    const long long jm = line - jq * a.ns;
    const float2 *gin = a.in + b * a.in_dist + line;
    float2 *out_b = a.out + b * a.out_dist;
#pragma unroll 1
    for (int stage = 0; stage < 2; ++stage) {
      float v[32];
      if (stage == 0) {
#pragma unroll
        for (int r = 0; r < kR; ++r) {
          const int i = bb + 16 * r;
          const float2 x = __ldcg(gin + (long long)i * lines_total);
          float re = x.x, im = x.y * a.sign_in;
          if (jm != 0 && i != 0) {
            const long long e = jm * (long long)i;
            const float2 hi = __ldg(a.tw_hi + (e >> a.split_shift));
            const float2 lo = __ldg(a.tw_lo + (e & mask));
            float wr = hi.x, wi = hi.y;
            cmul<float>(wr, wi, lo.x, lo.y);
            cmul<float>(re, im, wr, wi);
          }
          v[r] = re;
          v[16 + r] = im;
        }
      } else {
#pragma unroll
        for (int r = 0; r < kR; ++r) {
          v[r] = sre[c * kColsPitch + cpad(bb + 16 * r)];
          v[16 + r] = sim[c * kColsPitch + cpad(bb + 16 * r)];
        }
        twiddle16(v, a.tw + bb, 16);   // W_256^{bb r}
      }
      store_split<FORM>(t_hi, t_lo, v);
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        issue_mmas<FORM>(tmem, b_hi, b_lo);
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                mma_bar)
            : "memory");
      }
      mma_pending = 1;
      const bool ok = line_wait(mma_bar, mma_phase);
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      mma_phase ^= 1u;
      mma_pending = 0;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint32_t d[32];
      tmem_ld32(t_d, d);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      if (stage == 0 || a.ns == 1) {
        // line outputs at 16 bb + k (stage 0) or bb + 16 k (stage 1)
#pragma unroll
        for (int k = 0; k < kR; ++k) {
          const int idx = stage == 0 ? 16 * bb + k : bb + 16 * k;
          sre[c * kColsPitch + cpad(idx)] = __uint_as_float(d[k]);
          sim[c * kColsPitch + cpad(idx)] = __uint_as_float(d[16 + k]);
        }
        __syncthreads();
        if (stage == 1) {
          // 16 whole lines, contiguous in the output: coalesced stores
          float2 *dst = out_b + line0 * kColsL;
#pragma unroll
          for (int q = 0; q < kColsC * kColsL / kThreads; ++q) {
            const int e = tid + q * kThreads;
            const int cc = e / kColsL;
            const int k = e - cc * kColsL;
            float2 o;
            o.x = sre[cc * kColsPitch + cpad(k)];
            o.y = sim[cc * kColsPitch + cpad(k)] * a.sign_out;
            __stcs(dst + e, o);
          }
          __syncthreads();
        }
      } else {
        // y[(line / Ns) Ns 256 + line mod Ns + k' Ns], k' = bb + 16 k
        float2 *dst = out_b + jq * a.ns * kColsL + jm;
#pragma unroll
        for (int k = 0; k < kR; ++k) {
          float2 o;
          o.x = __uint_as_float(d[k]);
          o.y = __uint_as_float(d[16 + k]) * a.sign_out;
          __stcs(dst + (long long)(bb + 16 * k) * a.ns, o);
        }
        __syncthreads();
      }
    }
    if (failed) break;
  }
  if (failed && tid == 0) {
    atomicExch(a.status, 1);
    if (mma_pending) (void)line_wait(mma_bar, mma_phase);
  }
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(FormTraits<FORM>::kTmemCols)
                 : "memory");
  }
}

template <int FORM>
struct TcColsInst {
  static constexpr size_t smem() { return (size_t)ColsPlan<FORM>::kBytes; }
  static const void *func() {
    return reinterpret_cast<const void *>(&tc_cols256_kernel<FORM>);
  }
  static int persistent_grid() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (cached[dev] > 0) return cached[dev];
    cudaFuncAttributes fa;
    int sms = 0, regs_sm = 0, smem_sm = 0, reserved = 0, threads_sm = 0;
    if (cudaFuncGetAttributes(&fa, tc_cols256_kernel<FORM>) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) !=
            cudaSuccess)
      return 0;
    const int warp_regs = ((fa.numRegs * 32 + 255) / 256) * 256;
    int per_sm = regs_sm / (warp_regs * (kThreads / 32));
    const int by_smem = smem_sm / ((int)smem() + reserved);
    const int by_threads = threads_sm / kThreads;
    const int by_tmem = 512 / FormTraits<FORM>::kTmemCols;
    if (by_smem < per_sm) per_sm = by_smem;
    if (by_threads < per_sm) per_sm = by_threads;
    if (by_tmem < per_sm) per_sm = by_tmem;
    if (per_sm < 1) per_sm = 1;
    cached[dev] = per_sm * sms;
    return cached[dev];
  }
  static cudaError_t launch(const mofft_pass_args *p, cudaStream_t s) {
    if (p->in_table || p->out_table) return cudaErrorNotSupported;
    if (!p->aux || !p->status) return cudaErrorInvalidValue;
    if (p->total % kColsL != 0 || (p->total / kColsL) % kColsC != 0) return cudaErrorInvalidValue;
    if (p->ns_outer != 1 && p->ns_outer % kColsC != 0) return cudaErrorInvalidValue;
    if (p->ns_outer > 1 && (p->split_shift < 0 || p->split_shift > 40))
      return cudaErrorInvalidValue;
    const long long tiles = p->batch * ((p->total / kColsL) / kColsC);
    if (tiles <= 0) return cudaSuccess;
    const int resident = persistent_grid();
    if (resident <= 0) return cudaErrorInvalidConfiguration;
    TcColsArgs a;
    a.in = static_cast<const float2 *>(p->in);
    a.out = static_cast<float2 *>(p->out);
    a.tw = static_cast<const float2 *>(p->tw);
    a.tw_hi = static_cast<const float2 *>(p->tw_hi);
    a.tw_lo = static_cast<const float2 *>(p->tw_lo);
    a.bmat = static_cast<const unsigned char *>(p->aux);
    a.status = p->status;
    a.batch = p->batch;
    a.in_dist = p->in_dist;
    a.out_dist = p->out_dist;
    a.total = p->total;
    a.ns = p->ns_outer;
    a.split_shift = p->ns_outer > 1 ? p->split_shift : 0;
    a.sign_in = p->conj_in ? -1.0f : 1.0f;
    a.sign_out = p->conj_out ? -1.0f : 1.0f;
    const long long grid = tiles < resident ? tiles : resident;
    tc_cols256_kernel<FORM><<<(unsigned)grid, kThreads, smem(), s>>>(a);
    return cudaGetLastError();
  }
  static Entry entry(const char *name) {
    Entry e{};
    e.desc.name = name;
    e.desc.precision_bits = 32;
    e.desc.kind = MOFFT_KERNEL_TENSOR_COLS;
    e.desc.length = kColsL;
    e.desc.lines = kColsC;
    e.desc.threads = kThreads;
    e.desc.staged = 0;
    e.desc.radix_count = 2;
    for (int i = 0; i < 8; ++i) e.desc.radices[i] = i < 2 ? kR : 0;
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
      tc::TcColsInst<kFormTf32x3>::entry("tensor_cols_float_256_tf32x3_c16"),
      tc::TcColsInst<kFormBf16x3>::entry("tensor_cols_float_256_bf16x3_c16"),
  };
  *n = (int)(sizeof(e) / sizeof(e[0]));
  return e;
}

}  // namespace mofft

using namespace mofft;

extern "C" size_t mofft_cuda_tensor_aux_bytes(int form) {
  if (form == kFormTf32x3) return 2 * (size_t)tc::Plan<kFormTf32x3>::kBHalf;
  if (form == kFormBf16x3) return 2 * (size_t)tc::Plan<kFormBf16x3>::kBHalf;
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
