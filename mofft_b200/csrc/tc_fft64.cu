// Split-BF16 tensor-core form of the FP32 4096-point transform as two
// radix-64 DFT-matrix GEMMs (tcgen05, sm_100a).
//
// Four-step over n = 64 n1 + n2, k = k1 + 64 k2:
//
//   Y[k1][n2] = sum_n1 x[64 n1 + n2] F[n1][k1]          (stage 1, 64-point DFTs)
//   Z[k1][n2] = Y[k1][n2] W_4096^(n2 k1)                 (twiddle)
//   X[k1 + 64 k2] = sum_n2 Z[k1][n2] F[n2][k2]           (stage 2)
//
// with F[a][b] = W_64^(ab) = Fr + i Fi (symmetric).  Both stages are the
// same real GEMM shape on the tensor cores: M = 128 rows (64 rows of each of
// two transforms), N = 64 (+64), K = 64 (+64), B = the DFT matrix:
//
//   D_re = A_re Fr + A_im (-Fi),   D_im = A_re Fi + A_im Fr
//
// (the minus sign is the instruction's B-negate bit, so only Fr and Fi are
// stored).  Stage 1: rows m = n2 of transform t (lane 64 t + n2), K = n1;
// stage 2: rows m = k1, K = n2.  The stage-2 operand is the transpose of
// stage 1's accumulator, so the thread that reads accumulator row n2 writes
// operand column n2: stage 1's operand is K-major, stage 2's MN-major, both
// in the 128-byte swizzled layout, in which every warp store of the
// conversions is conflict-free.  Stage 2's accumulator row k1 holds
// X[k1 + 64 k2] for all k2, so the output leaves TMEM in natural order with
// coalesced stores (consecutive lanes, consecutive k1).
//
// Split precision: every operand x = hi + lo (bfloat16 pieces, about 16
// significant bits), products lo*hi + hi*lo + hi*hi accumulated in FP32 in
// TMEM, small terms first; B's pieces are prepared on the host from the
// DFT matrix in long double.
//
// Work division: one persistent CTA per SM.  Warp 0 allocates TMEM and one of
// its threads issues every MMA; one thread of warp 1 streams the input: each
// pair of transforms (64 KB) arrives in a shared staging buffer by bulk
// copies (no multicast) as soon as the previous pair has been read out of
// it, so HBM reads run while the groups and the tensor core work.  Two
// groups of eight warps (warps 2-9, 10-17; each warp reads the TMEM lane
// quarter of its index mod 4, two warps per quarter, each taking half of the
// quarter's columns) take turns over the CTA's pairs: while one
// group converts or drains a pair, the tensor core runs the other group's
// GEMMs.  A group: splits its staged pair into its stage-1 operand, waits
// for stage 1, twiddles and splits the accumulator into its stage-2 operand
// (same shared buffer), waits for stage 2 and stores the output.
// Accumulators of both stages share the group's 128 TMEM columns.  Inputs
// that are not 16-byte aligned (odd distances) skip the staging: the groups
// load them from global memory, prefetched into L2 one pair ahead.
//
// Every wait (operand ready, MMAs complete) is bounded by one second of
// wall time.  On a timeout the waiting thread records the error word and
// raises the CTA's abort flag; every thread leaves its loop at its next check,
// the issuing thread waits (bounded) for its MMAs in flight, and TMEM is
// released.  The host reports MOFFT_INTERNAL_ERROR.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "fft_device.cuh"
#include "fft_instances.cuh"
#include "mofft_cuda.h"
#include "mofft_host.h"

namespace mofft {
namespace tc64 {

constexpr int kN = 4096;
#ifndef MOFFT_TC64_GROUPS
#define MOFFT_TC64_GROUPS 2
#endif
constexpr int kGroups = MOFFT_TC64_GROUPS;
// two groups of eight warps with an input staging buffer, or three groups of
// four warps (their operands take the staging buffer's shared memory)
constexpr bool kStaging = kGroups == 2;
constexpr int kGroupWarps = kGroups == 2 ? 8 : 4;
constexpr int kGroupThreads = 32 * kGroupWarps;
constexpr int kFirstGroupWarp = 2;          // warp 0: MMA issue, warp 1: input stream
constexpr int kThreads = 32 * kFirstGroupWarp + kGroups * kGroupThreads;
constexpr int kFormBf16x3 = 2;                            // MOFFT_FORM_BF16X3

// Shared memory (bytes from a 1024-byte aligned base).
constexpr int kTile = 64 * 64 * 2;          // one 64 x 64 bf16 B tile, K-major SW128
constexpr int kOffB = 0;                    // Fr_hi, Fi_hi, Fr_lo, Fi_lo
constexpr int kAPart = 128 * 64 * 2;        // M = 128 rows x K = 64 (one part), bf16
constexpr int kAArray = 2 * kAPart;         // both parts (re, im)
constexpr int kOffA = 4 * kTile;            // group g: hi at + 2 g kAArray, lo at + kAArray
constexpr int kStage = 2 * kN * 8;         // one pair of transforms, interleaved
constexpr int kOffS = kOffA + kGroups * 2 * kAArray;   // staging of the next pair
constexpr int kOffBar = kOffS + (kStaging ? kStage : 0);
constexpr int kOffFlags = kOffBar + 128;    // abort flag, TMEM base
constexpr int kBytes = kOffFlags + 16 + 1024;
static_assert(kBytes <= 227 * 1024, "shared memory of the radix-64 kernel");
constexpr uint32_t kTmemCols = kGroups == 2 ? 256 : 512;  // group g: D_re at 128 g, D_im + 64

// Aux buffer of a plan (global memory): the B tiles as laid out in shared
// memory, then the twiddle table W_4096^(k1 n2) at [k1][n2].
constexpr size_t kAuxTiles = 4 * kTile;
constexpr size_t kAuxBytes = kAuxTiles + (size_t)kN * sizeof(float2);

// Byte offset of element (row, k) of a K-major, 128-byte swizzled tile of
// bf16 with 64 K elements per row: 8-row groups of 1024 bytes, 16-byte chunk
// c of row r at chunk c ^ (r mod 8).
__host__ __device__ constexpr int kmajor_off(int row, int k) {
  return (row >> 3) * 1024 + (row & 7) * 128 + ((((k >> 3) ^ row) & 7) << 4) + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: start, leading / stride byte offsets,
// descriptor version 1 (bit 46), 128-byte swizzle (layout type 2, bits 61-63).
__device__ __forceinline__ uint64_t desc_sw128(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// Instruction descriptor: D F32, A and B BF16, M = 128, N = 64, A K-major or
// MN-major, B K-major, B optionally negated.
__device__ __forceinline__ uint32_t idesc(bool a_mn, bool b_neg) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((b_neg ? 1u : 0u) << 14) |
         ((a_mn ? 1u : 0u) << 15) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id,
                                    bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(d), "l"(a), "l"(b), "r"(id), "r"(accumulate ? 1u : 0u)
      : "memory");
}

__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
      : "memory");
}

__device__ __forceinline__ void arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&d)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]),
        "=r"(d[6]), "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]),
        "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// bf16 pair {lo half: a, hi half: b}, rounded to nearest.
__device__ __forceinline__ uint32_t bf16x2(float a, float b) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
  return r;
}

// Eight values -> one 16-byte chunk of hi pieces and one of lo pieces.
__device__ __forceinline__ void split8(const float *v, uint4 &hi, uint4 &lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    h[j] = bf16x2(v[2 * j], v[2 * j + 1]);
    const float h0 = __uint_as_float(h[j] << 16);
    const float h1 = __uint_as_float(h[j] & 0xFFFF0000u);
    l[j] = bf16x2(v[2 * j] - h0, v[2 * j + 1] - h1);
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// Bounded wait (one second of %globaltimer, as line_wait) whose polls
// suspend the waiting thread for up to 20 us each (the try_wait suspend-time
// hint), so that waiting warps leave the issue slots to the working ones.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
  const unsigned long long t0 = line_clock_ns();
  for (unsigned it = 0; it < (1u << 24); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(20000u)
        : "memory");
    if (ok) return true;
    if (line_clock_ns() - t0 > kLineWaitNs) return false;
  }
  return false;
}

struct Args {
  const float2 *in;
  float2 *out;
  const unsigned char *aux;   // B tiles, then the twiddle table
  int *status;                // set to 1 when a wait timed out
  long long batch;
  long long in_dist;
  long long out_dist;
  float sign;                 // -1: conjugate on load and store (backward)
  int bulk;                   // 1: transforms are 16-byte aligned (bulk copies)
  int lose_mma;               // failure check: the first GEMM is never issued
};

// Stage GEMMs of one group: 3 terms x 4 K-steps x 4 products (48 MMAs).
// a_hi / a_lo: the group's operand arrays; a_mn: MN-major (stage 2).
__device__ __forceinline__ void issue_stage(uint32_t d_re, uint32_t a_hi, uint32_t a_lo,
                                            uint32_t b_base, bool a_mn) {
  const uint32_t id_pos = idesc(a_mn, false);
  const uint32_t id_neg = idesc(a_mn, true);
  const uint32_t d_im = d_re + 64;
  bool first = true;
#pragma unroll
  for (int term = 0; term < 3; ++term) {
    // term 0: A_lo * B_hi, 1: A_hi * B_lo, 2: A_hi * B_hi (small terms first)
    const uint32_t a = term == 0 ? a_lo : a_hi;
    const uint32_t fr = b_base + (term == 1 ? 2 * kTile : 0);
    const uint32_t fi = fr + kTile;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      uint64_t a_re, a_im;
      if (a_mn) {
        // K groups of 8 rows, 2048 bytes apart; the two M atoms 1024 apart
        a_re = desc_sw128(a + (uint32_t)(2 * s) * 2048u, 1024, 2048);
        a_im = desc_sw128(a + (uint32_t)(8 + 2 * s) * 2048u, 1024, 2048);
      } else {
        // 8-row groups 1024 bytes apart; K advances 32 bytes per step
        a_re = desc_sw128(a + (uint32_t)s * 32u, 16, 1024);
        a_im = desc_sw128(a + kAPart + (uint32_t)s * 32u, 16, 1024);
      }
      const uint64_t b_r = desc_sw128(fr + (uint32_t)s * 32u, 16, 1024);
      const uint64_t b_i = desc_sw128(fi + (uint32_t)s * 32u, 16, 1024);
      mma(d_re, a_re, b_r, id_pos, !first);
      mma(d_re, a_im, b_i, id_neg, true);
      mma(d_im, a_re, b_i, id_pos, !first);
      mma(d_im, a_im, b_r, id_pos, true);
      first = false;
    }
  }
}

__global__ void __launch_bounds__(kThreads, 1) tc64_fft4096_kernel(const Args a) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t *bars = reinterpret_cast<uint64_t *>(base + kOffBar);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(base + kOffFlags);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(base + kOffFlags + 4);
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  // a_full[g] at bars[g] (a group's arrivals), d_full[g] at
  // bars[kGroups + g] (MMA commit), fin at bars[2 kGroups], s_full[g] at
  // bars[2 kGroups + 1 + g] (staged bytes of group g's pairs, so that each
  // barrier's phases are one group's pairs in order), s_empty after them
  // (arrivals of the group that read the staging buffer)
  const uint32_t bar0 = smem_u32(bars);
  const uint32_t d_full0 = bar0 + 8 * kGroups, fin = bar0 + 16 * kGroups;
  const uint32_t s_full0 = fin + 8, s_empty = fin + 24;

  for (int i = tid; i < (int)(kAuxTiles / 16); i += kThreads)
    reinterpret_cast<uint4 *>(base + kOffB)[i] = __ldg(reinterpret_cast<const uint4 *>(a.aux) + i);
  if (tid == 0) {
    for (int g = 0; g < kGroups; ++g) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar0 + 8 * g),
                   "r"(kGroupThreads) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(d_full0 + 8 * g),
                   "r"(1) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(fin), "r"(1) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_full0), "r"(1) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_full0 + 8), "r"(1)
                 : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_empty),
                 "r"(kGroupThreads) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *abort_flag = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // B tiles -> tensor core
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const long long pairs = (a.batch + 1) / 2;
  const long long stride = gridDim.x;

  if (tid == 0) {
    // ------------------------------------------------------------ MMA issue
    // Serve whichever group's operand is ready (each group's jobs come in
    // order: stage 1, stage 2 of its pair i, then of pair i + kGroups), so
    // that one group's slow phase does not hold the tensor core from another.
    uint32_t aphase[kGroups];
    int stg[kGroups];
    long long nxt[kGroups];                  // CTA-local pair index per group
#pragma unroll
    for (int g = 0; g < kGroups; ++g) {
      aphase[g] = 0u;
      stg[g] = 0;
      nxt[g] = g;
    }
    const uint32_t b_base = smem_u32(base + kOffB);
    bool lose = a.lose_mma != 0;
    bool failed = false;
    unsigned long long last = line_clock_ns();
    for (unsigned spin = 0;; ++spin) {
      bool any = false, served = false;
#pragma unroll
      for (int g = 0; g < kGroups; ++g) {
        if (blockIdx.x + nxt[g] * stride >= pairs) continue;
        any = true;
        uint32_t ready;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(ready)
            : "r"(bar0 + 8 * g), "r"(aphase[g])
            : "memory");
        if (!ready) continue;
        served = true;
        const int stage = stg[g];
        aphase[g] ^= 1u;
        if (++stg[g] == 2) {
          stg[g] = 0;
          nxt[g] += kGroups;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (lose) {  // failure check: this GEMM never runs, its group times out
          lose = false;
          continue;
        }
        const uint32_t a_hi = smem_u32(base + kOffA + g * 2 * kAArray);
        issue_stage(tmem + 128u * g, a_hi, a_hi + kAArray, b_base, stage == 1);
        commit(d_full0 + 8 * g);
      }
      if (!any) break;
      if (served) {
        last = line_clock_ns();
      } else if ((spin & 63u) == 63u &&
                 (*abort_flag || line_clock_ns() - last > kLineWaitNs)) {
        failed = true;   // no group became ready for a second, or one gave up
        break;
      }
    }
    if (failed) {
      *abort_flag = 1;
      atomicExch(a.status, 1);
    }
    // every MMA issued above has completed before TMEM is released
    commit(fin);
    (void)bar_wait(fin, 0);
  } else if (kStaging && tid == 32 && a.bulk) {
    // ------------------------------------------------------------- producer
    const uint32_t stage_addr = smem_u32(base + kOffS);
    bool failed = false;
    long long issued = -1;   // last pair index whose copies were issued
    for (long long i = 0;; ++i) {
      const long long pair = blockIdx.x + i * stride;
      if (pair >= pairs) break;
      // the group that converted the previous pair has read the buffer
      if (i > 0 && (*abort_flag || !bar_wait(s_empty, (uint32_t)((i - 1) & 1)))) {
        failed = true;
        break;
      }
      const bool two = 2 * pair + 1 < a.batch;
      const uint32_t s_full = s_full0 + 8 * (uint32_t)(i & 1);   // group i mod 2
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s_full),
                   "r"((two ? 2 : 1) * kN * 8) : "memory");
      for (int t = 0; t < (two ? 2 : 1); ++t)
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
            "[%3];" ::"r"(stage_addr + (uint32_t)(t * kN * 8)),
            "l"(a.in + (2 * pair + t) * a.in_dist), "r"(kN * 8), "r"(s_full)
            : "memory");
      issued = i;
    }
    if (failed) {
      *abort_flag = 1;
      atomicExch(a.status, 1);
    }
    // the last copy has landed before the shared memory is released
    if (issued >= 0)
      (void)bar_wait(s_full0 + 8 * (uint32_t)(issued & 1), (uint32_t)((issued >> 1) & 1));
  } else if (warp >= kFirstGroupWarp) {
    // --------------------------------------------------------------- groups
    // Eight warps per group; the two warps of a TMEM lane quarter share its
    // rows, half h taking half of each row's K chunks (conversion) or
    // columns (epilogues).
    const int gw = warp - kFirstGroupWarp;
    const int g = gw / kGroupWarps;
    const int h = kGroupWarps == 8 ? (gw % kGroupWarps) >> 2 : 0;
    const int q = warp & 3;                  // TMEM lane quarter
    const int m = q * 32 + (tid & 31);       // row of both stages' GEMMs
    const int t = m >> 6;                    // transform of the pair
    const int r64 = m & 63;                  // n2 (stage 1 row), k1 (stage 2 row)
    unsigned char *a_hi = base + kOffA + g * 2 * kAArray;
    unsigned char *a_lo = a_hi + kAArray;
    const uint32_t a_bar = bar0 + 8 * g;
    const uint32_t d_bar = d_full0 + 8 * g;
    const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + 128u * g;
    // This thread's twiddles W_4096^(n2 k1) depend only on its fixed n2 and
    // k1 half: the table entries of W^n2, W^2n2, W^4n2, W^8n2 and of the two
    // chunk bases W^(16 c2 n2) are read once, and each chunk's sixteen powers
    // are derived from them (at most three chained products) instead of
    // loaded per pair (the table does not stay in L1 beside this shared
    // memory footprint).
    const float2 *tw = reinterpret_cast<const float2 *>(a.aux + kAuxTiles);
    const float2 p1 = __ldg(tw + 1 * 64 + r64), p2 = __ldg(tw + 2 * 64 + r64);
    const float2 p4 = __ldg(tw + 4 * 64 + r64), p8 = __ldg(tw + 8 * 64 + r64);
    constexpr int kChunks = 4 * 4 / kGroupWarps;   // 16-column chunks per thread
    const int c2_first = kChunks * h;
    float2 base_c2[kChunks];                       // W^(16 c2 n2) of each chunk
#pragma unroll
    for (int j = 0; j < kChunks; ++j) base_c2[j] = __ldg(tw + (16 * (c2_first + j)) * 64 + r64);
    uint32_t dphase = 0;
    bool failed = false;
    for (long long i = g; !failed; i += kGroups) {
      const long long pair = blockIdx.x + i * stride;
      if (pair >= pairs) break;
      const long long b = 2 * pair + t;
      const bool valid = b < a.batch;
      // unaligned inputs: bulk prefetch of this group's next pair into L2
      if (!a.bulk && gw % kGroupWarps == 0 && (tid & 31) == 0) {
        const long long nb = 2 * (pair + kGroups * stride);
        for (int k = 0; k < 2; ++k)
          if (nb + k < a.batch)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(
                             a.in + (nb + k) * a.in_dist),
                         "r"(kN * 8)
                         : "memory");
      }
      // stage-1 operand: row m = n2 of transform t, K = n1 (re part, then im)
      if (a.bulk && (*abort_flag || !bar_wait(s_full0 + 8 * (uint32_t)g,
                                                (uint32_t)((i >> 1) & 1)))) {
        failed = true;
        break;
      }
      {
        const float2 *src = a.bulk ? reinterpret_cast<const float2 *>(base + kOffS) +
                                         t * kN + r64
                                   : a.in + (valid ? b : 0) * a.in_dist + r64;
        // row base (8-row group, row); the swizzled chunk is added per c
        unsigned char *row_hi = a_hi + (m >> 3) * 1024 + (m & 7) * 128;
        unsigned char *row_lo = a_lo + (m >> 3) * 1024 + (m & 7) * 128;
#pragma unroll
        for (int c = 2 * kChunks * h; c < 2 * kChunks * (h + 1); ++c) {
          float re[8], im[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const float2 v = !valid ? make_float2(0.f, 0.f)
                             : a.bulk ? src[64 * (8 * c + k)] : __ldcg(src + 64 * (8 * c + k));
            re[k] = v.x;
            im[k] = v.y * a.sign;
          }
          uint4 h, l;
          const int off = (((c ^ m) & 7) << 4);
          split8(re, h, l);
          *reinterpret_cast<uint4 *>(row_hi + off) = h;
          *reinterpret_cast<uint4 *>(row_lo + off) = l;
          split8(im, h, l);
          *reinterpret_cast<uint4 *>(row_hi + kAPart + off) = h;
          *reinterpret_cast<uint4 *>(row_lo + kAPart + off) = l;
        }
      }
      if (a.bulk) arrive(s_empty);   // the staged pair has been read
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      arrive(a_bar);
      if (*abort_flag || !bar_wait(d_bar, dphase)) {
        failed = true;
        break;
      }
      dphase ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // twiddle the stage-1 accumulator (row n2) into the stage-2 operand:
      // rows k1 (M, 8 per chunk), K = n2 (re part) and 64 + n2 (im part)
      {
        const int kr = r64 & 7;
        const int kg = r64 >> 3;
        unsigned char *col_hi = a_hi + kg * 2048 + t * 1024 + kr * 128;
        unsigned char *col_lo = a_lo + kg * 2048 + t * 1024 + kr * 128;
#pragma unroll 1
        for (int c2 = c2_first; c2 < c2_first + kChunks; ++c2) {
          uint32_t yr[16], yi[16];
          tmem_ld16(trow + 16 * c2, yr);
          tmem_ld16(trow + 64 + 16 * c2, yi);
          tmem_wait_ld();
          float zr[16], zi[16];
          {
            // powers W^(n2 k), k < 16, times the chunk base W^(16 c2 n2)
            float wr[16], wi[16];
            wr[0] = 1.f; wi[0] = 0.f;
            wr[1] = p1.x; wi[1] = p1.y;
            wr[2] = p2.x; wi[2] = p2.y;
            wr[4] = p4.x; wi[4] = p4.y;
            wr[8] = p8.x; wi[8] = p8.y;
#pragma unroll
            for (int k = 3; k < 16; ++k) {
              if ((k & (k - 1)) == 0) continue;
              const int hb = k >= 8 ? 8 : (k >= 4 ? 4 : 2);
              const int lb = k - hb;
              wr[k] = wr[hb] * wr[lb] - wi[hb] * wi[lb];
              wi[k] = wr[hb] * wi[lb] + wi[hb] * wr[lb];
            }
            float2 bs = base_c2[0];
#pragma unroll
            for (int j = 1; j < kChunks; ++j)
              if (c2 == c2_first + j) bs = base_c2[j];
#pragma unroll
            for (int k = 0; k < 16; ++k) {
              const float vr = wr[k] * bs.x - wi[k] * bs.y;
              const float vi = wr[k] * bs.y + wi[k] * bs.x;
              const float xr = __uint_as_float(yr[k]), xi = __uint_as_float(yi[k]);
              zr[k] = xr * vr - xi * vi;
              zi[k] = xr * vi + xi * vr;
            }
          }
#pragma unroll
          for (int h2 = 0; h2 < 2; ++h2) {
            const int c = 2 * c2 + h2;
            const int off = ((c ^ kr) & 7) << 4;
            uint4 h, l;
            split8(zr + 8 * h2, h, l);
            *reinterpret_cast<uint4 *>(col_hi + off) = h;
            *reinterpret_cast<uint4 *>(col_lo + off) = l;
            split8(zi + 8 * h2, h, l);
            *reinterpret_cast<uint4 *>(col_hi + 8 * 2048 + off) = h;
            *reinterpret_cast<uint4 *>(col_lo + 8 * 2048 + off) = l;
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      arrive(a_bar);
      if (*abort_flag || !bar_wait(d_bar, dphase)) {
        failed = true;
        break;
      }
      dphase ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // stage-2 accumulator row k1: X[k1 + 64 k2], k2 = 0..63
      {
        float2 *dst = a.out + (valid ? b : 0) * a.out_dist + r64;
#pragma unroll 1
        for (int c2 = c2_first; c2 < c2_first + kChunks; ++c2) {
          uint32_t xr[16], xi[16];
          tmem_ld16(trow + 16 * c2, xr);
          tmem_ld16(trow + 64 + 16 * c2, xi);
          tmem_wait_ld();
          if (valid) {
#pragma unroll
            for (int k = 0; k < 16; ++k)
              __stcs(dst + 64 * (16 * c2 + k),
                     make_float2(__uint_as_float(xr[k]), __uint_as_float(xi[k]) * a.sign));
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    if (failed) {
      *abort_flag = 1;
      atomicExch(a.status, 1);
    }
  }
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

struct Inst {
  static constexpr size_t smem() { return (size_t)kBytes; }
  static const void *func() { return reinterpret_cast<const void *>(&tc64_fft4096_kernel); }
  static cudaError_t launch(const mofft_pass_args *p, cudaStream_t s) {
    if (p->conj_in != p->conj_out) return cudaErrorInvalidValue;
    if (p->in_table || p->out_table) return cudaErrorNotSupported;
    if (!p->aux || !p->status) return cudaErrorInvalidValue;
    if (p->batch <= 0) return cudaSuccess;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        sms <= 0)
      return cudaErrorInvalidConfiguration;
    Args a;
    a.in = static_cast<const float2 *>(p->in);
    a.out = static_cast<float2 *>(p->out);
    a.aux = static_cast<const unsigned char *>(p->aux);
    a.status = p->status;
    a.batch = p->batch;
    a.in_dist = p->in_dist;
    a.out_dist = p->out_dist;
    a.sign = p->conj_in ? -1.0f : 1.0f;
    a.bulk = (kStaging && (reinterpret_cast<uintptr_t>(p->in) & 15u) == 0 &&
              (p->in_dist % 2) == 0) ? 1 : 0;
    a.lose_mma = p->lose_copy;
    const long long pairs = (p->batch + 1) / 2;
    const long long grid = pairs < sms ? pairs : sms;   // one CTA per SM
    tc64_fft4096_kernel<<<(unsigned)grid, kThreads, smem(), s>>>(a);
    return cudaGetLastError();
  }
  static int fill_aux(void *dst);
  static Entry entry(const char *name) {
    Entry e{};
    e.desc.name = name;
    e.desc.precision_bits = 32;
    e.desc.kind = MOFFT_KERNEL_TENSOR;
    e.desc.length = kN;
    e.desc.lines = 2;
    e.desc.threads = kThreads;
    e.desc.staged = 0;
    e.desc.radix_count = 2;
    for (int i = 0; i < 8; ++i) e.desc.radices[i] = i < 2 ? 64 : 0;
    e.desc.smem_bytes = smem();
    e.desc.form = kFormBf16x3;
    e.launch = &launch;
    e.func = &func;
    e.aux_bytes = kAuxBytes;
    e.fill_aux = &fill_aux;
    return e;
  }
};

// bf16 rounding of a double (nearest, ties to even) and its value.
uint16_t host_bf16(double x, double *value) {
  const float f = (float)x;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  const uint32_t rounded = u + 0x7FFFu + ((u >> 16) & 1u);
  const uint16_t h = (uint16_t)(rounded >> 16);
  const uint32_t back = (uint32_t)h << 16;
  float bf;
  std::memcpy(&bf, &back, 4);
  *value = (double)bf;
  return h;
}

// B tiles of the 64-point forward DFT F[a][b] = W_64^(ab) = Fr + i Fi (hi
// pieces of Fr and Fi, then lo pieces; row = output index, K = input index,
// K-major 128-byte swizzled as the kernel's shared memory holds them), then
// the FP32 twiddle table W_4096^(k1 n2) at [k1][n2].  Angles are reduced
// exactly and evaluated in long double.
int Inst::fill_aux(void *dst) {
  unsigned char *out = static_cast<unsigned char *>(dst);
  std::memset(out, 0, kAuxBytes);
  for (int row = 0; row < 64; ++row) {
    for (int k = 0; k < 64; ++k) {
      long double c, s;
      mofft_cis_turns((uint64_t)((row * k) % 64), 64, &c, &s);
      const double fr = (double)c, fi = -(double)s;
      const int off = kmajor_off(row, k);
      double hv, lv;
      uint16_t h = host_bf16(fr, &hv);
      uint16_t l = host_bf16(fr - hv, &lv);
      std::memcpy(out + 0 * kTile + off, &h, 2);
      std::memcpy(out + 2 * kTile + off, &l, 2);
      h = host_bf16(fi, &hv);
      l = host_bf16(fi - hv, &lv);
      std::memcpy(out + 1 * kTile + off, &h, 2);
      std::memcpy(out + 3 * kTile + off, &l, 2);
    }
  }
  float2 *tw = reinterpret_cast<float2 *>(out + kAuxTiles);
  for (int k1 = 0; k1 < 64; ++k1)
    for (int n2 = 0; n2 < 64; ++n2) {
      long double c, s;
      mofft_cis_turns((uint64_t)(k1 * n2), (uint64_t)kN, &c, &s);
      tw[k1 * 64 + n2] = make_float2((float)c, (float)-s);
    }
  return 0;
}

}  // namespace tc64

const Entry *entries_tensor64(int *n) {
  static const Entry e[] = {tc64::Inst::entry("tensor_float_4096_bf16x3_r64x2")};
  *n = (int)(sizeof(e) / sizeof(e[0]));
  return e;
}

}  // namespace mofft
