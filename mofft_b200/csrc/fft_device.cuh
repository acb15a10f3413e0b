// Device code for the MoFFT B200 transform: Stockham autosort stages held in
// registers and exchanged through shared memory.
//
// Notation.  A line is one length-L DFT that a CTA computes completely.  The
// in-CTA algorithm is the Stockham autosort form: with Ns the product of the
// radices already applied, stage (R, Ns) maps butterfly j in [0, L/R) as
//
//   v[r]  = x[j + r*(L/R)] * W_{Ns*R}^{(j mod Ns)*r}           (r < R)
//   v     = DFT_R(v)
//   y[(j div Ns)*Ns*R + (j mod Ns) + k*Ns] = v[k]               (k < R)
//
// which leaves the result in natural order after the last stage.  This is the
// same transform as the reference's mixed-radix Cooley-Tukey driver
// (src/mofft.c:1932-2045: first codelet, then per level a twiddled "other"
// codelet after a transpose), reorganised so that no transpose pass exists:
// the transpose becomes the scatter index of the shared-memory exchange.
//
// Every kernel computes the forward transform (FFTW sign, exp(-2 pi i jk/n)).
// Backward transforms use bwd(x) = conj(fwd(conj(x))): the imaginary part is
// negated on load and on store (sign = -1), which is exact.
//
// Transforms longer than one CTA use the same Stockham step with a "super
// radix" L per pass (four-step / six-step): pass p computes L_p-point DFTs over
// lines strided by M/L_p, applies the super-stage twiddle W_{Ns*L}^{(j mod
// Ns)*i} on load, and scatters with the same index map.  Those are the COLS
// kernels below.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "generated/codelets.cuh"

namespace mofft {

template <typename T> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };
template <typename T> using cplx_t = typename Cplx<T>::type;

// Shared memory holds real and imaginary parts in separate arrays (4- or
// 8-byte words).  One pad word per 32 words (fp32) / 16 words (fp64) keeps
// both the gather (j + r*L/R) and the scatter side of every exchange at one or
// two wavefronts per warp access.
template <typename T> struct Pad;
template <> struct Pad<float> { static constexpr int shift = 5; };
template <> struct Pad<double> { static constexpr int shift = 4; };
template <typename T>
__host__ __device__ constexpr int spad(int a) { return a + (a >> Pad<T>::shift); }
template <typename T>
__host__ __device__ constexpr int spad_len(int n) { return n + (n >> Pad<T>::shift) + 1; }

// Shared-memory words between the lines of a multi-line ROWS tile: at least
// spad_len(L), rounded up so that the line pitch is congruent to the threads
// per line modulo one 128-byte bank row.  The threads of a warp then spread
// the lines they work on over disjoint banks (a bank simulation of the
// staged kernels' copies and exchanges: 1.5-1.7 -> 1.2-1.5 wavefronts per
// access for most instances).  One-line tiles keep spad_len(L).
template <typename T>
__host__ __device__ constexpr int rows_line(int L, int TPL, int TB) {
  const int row = sizeof(T) == 4 ? 32 : 16;
  int b = spad_len<T>(L);
  if (TB > 1)
    while (b % row != TPL % row) ++b;
  return b;
}

template <typename T>
__device__ __forceinline__ void cmul(T& xr, T& xi, T wr, T wi) {
  const T r = xr * wr - xi * wi;
  const T i = xr * wi + xi * wr;
  xr = r;
  xi = i;
}

// Data is read once: load through L2 only (ld.global.cg), which also keeps
// reads coherent with writes of other CTAs of the same launch (the ragged
// persistent kernel reads its second pass after a device-scope fence).
template <typename T>
__device__ __forceinline__ cplx_t<T> ld_global(const cplx_t<T>* p) { return __ldcg(p); }

template <typename T>
__device__ __forceinline__ void st_global(cplx_t<T>* p, T re, T im) {
  cplx_t<T> v;
  v.x = re;
  v.y = im;
  *p = v;
}

// ---------------------------------------------------------------------------
// Compile-time stage list.
// ---------------------------------------------------------------------------
template <int... Rs> struct RadixList {};

template <int L, int... Rs> struct StageProduct;
template <int L> struct StageProduct<L> { static constexpr int value = 1; };
template <int L, int R, int... Rest> struct StageProduct<L, R, Rest...> {
  static constexpr int value = R * StageProduct<L, Rest...>::value;
};

// Size (in complex entries) of the internal twiddle table of a stage list:
// stage s with Ns > 1 stores (R_s - 1) * Ns entries, r-major.
__host__ __device__ constexpr int stage_table_size(int R, int Ns) {
  return Ns > 1 ? (R - 1) * Ns : 0;
}

// ---------------------------------------------------------------------------
// Register stage: each thread owns PER = ceil((L/R)/TPL) butterflies of one
// line.  Source and destination are global memory (first / last stage) or the
// line's shared-memory slice (padded SoA).  Addressing of a line element i is
// abstracted by the Layout policy:
//   RowsLayout: a line is contiguous in global memory and in shared memory.
//   ColsLayout: C lines are interleaved element-major in shared memory and in
//               global memory the lines are adjacent (line stride 1, element
//               stride S), so consecutive threads touch consecutive lines.
// ---------------------------------------------------------------------------
enum Where { kGlobal = 0, kShared = 1 };

template <typename T>
struct RowsLayout {
  T* sre;          // this line's shared real part
  T* sim;
  const cplx_t<T>* gin;   // this line's first input element
  cplx_t<T>* gout;        // this line's first output element
  T sign;                 // -1 for backward (conjugation), +1 forward
  bool active;            // this line is inside the batch
  __device__ __forceinline__ int saddr(int i) const { return spad<T>(i); }
  __device__ __forceinline__ void gload(int i, T& re, T& im) const {
    if (active) {
      const cplx_t<T> v = ld_global<T>(gin + i);
      re = v.x;
      im = v.y * sign;
    } else {
      re = T(0);
      im = T(0);
    }
  }
  __device__ __forceinline__ void gstore(int i, T re, T im) const {
    if (active) st_global<T>(gout + i, re, im * sign);
  }
  template <int R>
  __device__ __forceinline__ void super_twiddle(int, int, T (&)[R], T (&)[R]) const {}
};

// A line whose shared-memory exchanges move {re, im} pairs: one 8-byte
// (FP32) / 16-byte (FP64) access per value instead of two.  One pad pair per
// 16 pairs puts the stride-16 scatter of a radix-16 stage (Ns = 1) on
// distinct bank pairs; the other gathers and scatters run 16 consecutive
// pairs per half-warp.
// SH: one pad pair per 2^SH pairs (0: no padding, for lines whose
// first-stage stride is odd, e.g. the radix-5 stage of 5*2^k lengths).
template <typename T, int SH = 4>
struct RowsPairLayout : RowsLayout<T> {
  static constexpr bool kPairTag = true;
  cplx_t<T>* sp;    // this line's shared pairs
  __device__ __forceinline__ int paddr(int i) const { return SH ? i + (i >> SH) : i; }
  __device__ __forceinline__ void sget(int i, T& re, T& im) const {
    const cplx_t<T> v = sp[paddr(i)];
    re = v.x;
    im = v.y;
  }
  __device__ __forceinline__ void sput(int i, T re, T im) const {
    cplx_t<T> v;
    v.x = re;
    v.y = im;
    sp[paddr(i)] = v;
  }
};

// Pairs per line of a RowsPairLayout tile.
__host__ __device__ constexpr int pair_line(int L, int SH = 4) {
  return SH ? L + (L >> SH) + 1 : L + 1;
}

template <class Lay, class = void>
struct IsPairLayout {
  static constexpr bool value = false;
};
template <class Lay>
struct IsPairLayout<Lay, decltype((void)Lay::kPairTag, void())> {
  static constexpr bool value = true;
};

template <typename T, int C, int PITCH, bool TW>
struct ColsLayout {
  T* sre;          // shared base of the tile (all C lines)
  T* sim;
  int c;           // this thread's line within the tile
  const cplx_t<T>* gin;   // element 0 of this line
  cplx_t<T>* gout;        // element 0 of this line's output
  long long in_stride;    // element stride in global memory (S = M / L)
  long long out_stride;   // element stride of the output (Ns_outer)
  T sign_in, sign_out;
  bool active;
  // super-stage twiddle on load: W^{e}, e = jmod * i, two-level table
  const cplx_t<T>* tw_hi;
  const cplx_t<T>* tw_lo;
  long long jmod;         // (j mod Ns_outer) of this line
  int split_shift;        // K = 1 << split_shift
  __device__ __forceinline__ int saddr(int i) const { return i * PITCH + c; }
  __device__ __forceinline__ void gload(int i, T& re, T& im) const {
    if (active) {
      const cplx_t<T> v = ld_global<T>(gin + (long long)i * in_stride);
      re = v.x;
      im = v.y * sign_in;
    } else {
      re = T(0);
      im = T(0);
    }
  }
  // W^e from the two-level table (entry 0 of both tables is exactly 1).
  __device__ __forceinline__ void super_w(long long e, T& wr, T& wi) const {
    const cplx_t<T> hi = __ldg(tw_hi + (e >> split_shift));
    const cplx_t<T> lo = __ldg(tw_lo + (e & ((1LL << split_shift) - 1)));
    wr = hi.x;
    wi = hi.y;
    cmul<T>(wr, wi, lo.x, lo.y);
  }
  // Super-stage twiddle of butterfly j's loaded inputs (TW: passes with
  // Ns_outer > 1): v[r] *= W^{jmod (j + r BF)}, no branch, so that every
  // load issues together.  For R <= 16 it is W^{jmod j} u^r with
  // u = W^{jmod BF}: u, u^2, u^4, u^8 come from the table and every other
  // power is a product of two earlier ones (at most three products in a
  // chain), so a butterfly needs at most five lookups instead of R.
  template <int R>
  __device__ __forceinline__ void super_twiddle(int j, int BF, T (&vr)[R], T (&vi)[R]) const {
    if constexpr (TW) {
      if constexpr (R <= 16) {
        T ur[R], ui[R];
        T br, bi;
        super_w(jmod * (long long)j, br, bi);
        const long long u = jmod * (long long)BF;
#pragma unroll
        for (int k = 1; k < R; k <<= 1) super_w(u * k, ur[k], ui[k]);
#pragma unroll
        for (int r = 3; r < R; ++r) {
          if ((r & (r - 1)) == 0) continue;          // a power of two: loaded
          int h = 1;
          while (h * 2 <= r) h *= 2;                 // highest power of two in r
          const int l = r - h;
          ur[r] = ur[h] * ur[l] - ui[h] * ui[l];
          ui[r] = ur[h] * ui[l] + ui[h] * ur[l];
        }
        cmul<T>(vr[0], vi[0], br, bi);
#pragma unroll
        for (int r = 1; r < R; ++r) {
          T xr = ur[r], xi = ui[r];
          cmul<T>(xr, xi, br, bi);
          cmul<T>(vr[r], vi[r], xr, xi);
        }
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          T xr, xi;
          super_w(jmod * (long long)(j + r * BF), xr, xi);
          cmul<T>(vr[r], vi[r], xr, xi);
        }
      }
    }
  }
  __device__ __forceinline__ void gstore(int i, T re, T im) const {
    if (active) st_global<T>(gout + (long long)i * out_stride, re, im * sign_out);
  }
};

// Kernel flags (template parameter FLAGS of the ROWS kernels).
constexpr int kStaged = 1;       // I/O staged through shared memory
constexpr int kDerivedTw = 2;    // radix-16/32 twiddles from w, w^2, w^4, w^8 (, w^16)
constexpr int kSplitX = 4;       // exchanges move one component at a time
constexpr int kTwoCtas = 8;      // registers capped for two resident CTAs per SM
constexpr int kPrefetch = 16;    // persistent CTAs; the next line arrives by bulk copy
constexpr int kPairX = 32;       // exchanges move {re, im} pairs (RowsPairLayout)
constexpr int kPairPad32 = 64;   // with kPairX: one pad pair per 32 pairs
constexpr int kPairPad0 = 128;   // with kPairX: no padding

// Pad shift of a pair-exchange ROWS kernel's layout.
__host__ __device__ constexpr int pair_shift(int flags) {
  return (flags & kPairPad0) ? 0 : ((flags & kPairPad32) ? 5 : 4);
}

// Twiddles of one radix-16 butterfly: v[r] *= w^r.  Loads the table entries
// of w^1, w^2, w^4 and w^8 and forms the other powers with at most three
// chained complex products (three roundings), instead of 15 table loads.
template <typename T, int NS, int TWOFF>
__device__ __forceinline__ void twiddle16_derived(T (&vr)[16], T (&vi)[16], int jm,
                                                  const cplx_t<T>* __restrict__ tw) {
  T wr[16], wi[16];
  const cplx_t<T> a1 = __ldg(tw + TWOFF + 0 * NS + jm);
  const cplx_t<T> a2 = __ldg(tw + TWOFF + 1 * NS + jm);
  const cplx_t<T> a4 = __ldg(tw + TWOFF + 3 * NS + jm);
  const cplx_t<T> a8 = __ldg(tw + TWOFF + 7 * NS + jm);
  wr[1] = a1.x; wi[1] = a1.y;
  wr[2] = a2.x; wi[2] = a2.y;
  wr[4] = a4.x; wi[4] = a4.y;
  wr[8] = a8.x; wi[8] = a8.y;
#define MOFFT_WMUL(D, A, B)                          \
  wr[D] = wr[A] * wr[B] - wi[A] * wi[B];             \
  wi[D] = wr[A] * wi[B] + wi[A] * wr[B];
  MOFFT_WMUL(3, 2, 1) MOFFT_WMUL(5, 4, 1) MOFFT_WMUL(6, 4, 2) MOFFT_WMUL(7, 4, 3)
  MOFFT_WMUL(9, 8, 1) MOFFT_WMUL(10, 8, 2) MOFFT_WMUL(11, 8, 3) MOFFT_WMUL(12, 8, 4)
  MOFFT_WMUL(13, 8, 5) MOFFT_WMUL(14, 8, 6) MOFFT_WMUL(15, 8, 7)
#undef MOFFT_WMUL
#pragma unroll
  for (int r = 1; r < 16; ++r) cmul<T>(vr[r], vi[r], wr[r], wi[r]);
}

// Twiddles of one radix-32 butterfly: w^1 .. w^15 as in the radix-16 case
// plus the table entry of w^16, and w^(16+k) = w^16 w^k (at most four chained
// products), so 5 table loads instead of 31.
template <typename T, int NS, int TWOFF>
__device__ __forceinline__ void twiddle32_derived(T (&vr)[32], T (&vi)[32], int jm,
                                                  const cplx_t<T>* __restrict__ tw) {
  T wr[16], wi[16];
  const cplx_t<T> a1 = __ldg(tw + TWOFF + 0 * NS + jm);
  const cplx_t<T> a2 = __ldg(tw + TWOFF + 1 * NS + jm);
  const cplx_t<T> a4 = __ldg(tw + TWOFF + 3 * NS + jm);
  const cplx_t<T> a8 = __ldg(tw + TWOFF + 7 * NS + jm);
  const cplx_t<T> a16 = __ldg(tw + TWOFF + 15 * NS + jm);
  wr[1] = a1.x; wi[1] = a1.y;
  wr[2] = a2.x; wi[2] = a2.y;
  wr[4] = a4.x; wi[4] = a4.y;
  wr[8] = a8.x; wi[8] = a8.y;
#define MOFFT_WMUL(D, A, B)                          \
  wr[D] = wr[A] * wr[B] - wi[A] * wi[B];             \
  wi[D] = wr[A] * wi[B] + wi[A] * wr[B];
  MOFFT_WMUL(3, 2, 1) MOFFT_WMUL(5, 4, 1) MOFFT_WMUL(6, 4, 2) MOFFT_WMUL(7, 4, 3)
  MOFFT_WMUL(9, 8, 1) MOFFT_WMUL(10, 8, 2) MOFFT_WMUL(11, 8, 3) MOFFT_WMUL(12, 8, 4)
  MOFFT_WMUL(13, 8, 5) MOFFT_WMUL(14, 8, 6) MOFFT_WMUL(15, 8, 7)
#undef MOFFT_WMUL
#pragma unroll
  for (int r = 1; r < 16; ++r) cmul<T>(vr[r], vi[r], wr[r], wi[r]);
  cmul<T>(vr[16], vi[16], a16.x, a16.y);
#pragma unroll
  for (int k = 1; k < 16; ++k) {
    const T pr = a16.x * wr[k] - a16.y * wi[k];
    const T pi = a16.x * wi[k] + a16.y * wr[k];
    cmul<T>(vr[16 + k], vi[16 + k], pr, pi);
  }
}

template <typename T, int L, int TPL, int R, int NS, Where SRC, Where DST,
          int TWOFF, bool DTW, class Layout>
__device__ __forceinline__ void reg_stage(const Layout& lay, int t,
                                          const cplx_t<T>* __restrict__ tw) {
  constexpr int BF = L / R;
  constexpr int PER = (BF + TPL - 1) / TPL;
  constexpr bool EVEN = (BF % TPL) == 0;
  T vr[PER][R];
  T vi[PER][R];
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    const int j = t + m * TPL;
    if (EVEN || j < BF) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int idx = j + r * BF;
        if (SRC == kGlobal) {
          lay.gload(idx, vr[m][r], vi[m][r]);
        } else if constexpr (IsPairLayout<Layout>::value) {
          lay.sget(idx, vr[m][r], vi[m][r]);
        } else {
          vr[m][r] = lay.sre[lay.saddr(idx)];
          vi[m][r] = lay.sim[lay.saddr(idx)];
        }
      }
      if constexpr (SRC == kGlobal) lay.template super_twiddle<R>(j, BF, vr[m], vi[m]);
      if (NS > 1) {
        const int jm = j % NS;
        if constexpr (DTW && R == 16) {
          twiddle16_derived<T, NS, TWOFF>(vr[m], vi[m], jm, tw);
        } else if constexpr (DTW && R == 32) {
          twiddle32_derived<T, NS, TWOFF>(vr[m], vi[m], jm, tw);
        } else {
#pragma unroll
          for (int r = 1; r < R; ++r) {
            const cplx_t<T> w = __ldg(tw + TWOFF + (r - 1) * NS + jm);
            cmul<T>(vr[m][r], vi[m][r], w.x, w.y);
          }
        }
      }
      Dft<R>::fwd(vr[m], vi[m]);
    }
  }
  if (SRC == kShared && DST == kShared) __syncthreads();
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    const int j = t + m * TPL;
    if (EVEN || j < BF) {
      const int base = (j / NS) * NS * R + (j % NS);
#pragma unroll
      for (int k = 0; k < R; ++k) {
        const int idx = base + k * NS;
        if (DST == kGlobal) {
          lay.gstore(idx, vr[m][k], vi[m][k]);
        } else if constexpr (IsPairLayout<Layout>::value) {
          lay.sput(idx, vr[m][k], vi[m][k]);
        } else {
          lay.sre[lay.saddr(idx)] = vr[m][k];
          lay.sim[lay.saddr(idx)] = vi[m][k];
        }
      }
    }
  }
  if (DST == kShared) __syncthreads();
}

// Recursive stage driver over a compile-time radix list.
template <typename T, int L, int TPL, int NS, int TWOFF, bool FIRST_SHARED,
          bool LAST_SHARED, bool IS_FIRST, bool DTW, int... Rs>
struct StageRunner;

template <typename T, int L, int TPL, int NS, int TWOFF, bool FS, bool LS,
          bool IS_FIRST, bool DTW, int R>
struct StageRunner<T, L, TPL, NS, TWOFF, FS, LS, IS_FIRST, DTW, R> {
  template <class Layout>
  __device__ __forceinline__ static void run(const Layout& lay, int t,
                                             const cplx_t<T>* tw) {
    constexpr Where src = (IS_FIRST && !FS) ? kGlobal : kShared;
    constexpr Where dst = LS ? kShared : kGlobal;
    reg_stage<T, L, TPL, R, NS, src, dst, TWOFF, DTW>(lay, t, tw);
  }
};

template <typename T, int L, int TPL, int NS, int TWOFF, bool FS, bool LS,
          bool IS_FIRST, bool DTW, int R, int R2, int... Rest>
struct StageRunner<T, L, TPL, NS, TWOFF, FS, LS, IS_FIRST, DTW, R, R2, Rest...> {
  template <class Layout>
  __device__ __forceinline__ static void run(const Layout& lay, int t,
                                             const cplx_t<T>* tw) {
    constexpr Where src = (IS_FIRST && !FS) ? kGlobal : kShared;
    reg_stage<T, L, TPL, R, NS, src, kShared, TWOFF, DTW>(lay, t, tw);
    StageRunner<T, L, TPL, NS * R, TWOFF + stage_table_size(R, NS), FS, LS,
                false, DTW, R2, Rest...>::run(lay, t, tw);
  }
};

// ---------------------------------------------------------------------------
// Split-exchange stage chain (FLAGS & kSplitX, one-pass kernels with direct
// global I/O).  Values stay in registers between stages and each exchange
// moves the real parts through a single shared buffer, then the imaginary
// parts through the same buffer, so a line needs L words of shared memory
// instead of 2L: twice the resident CTAs for the long one-pass lengths.
// ---------------------------------------------------------------------------
// Word offset of element i in a split-exchange buffer.  FP64 pads one
// element per 32 (a bank simulation of the split exchanges of the FP64
// lines, 2560-6144 points, gives 1.2-1.3 wavefronts per access against
// 1.3-1.8 with the one-per-16 padding of the two-array exchanges; powers of
// two stay conflict-free); FP32 keeps spad.
template <typename T>
__device__ __forceinline__ int split_pad(int i) {
  if constexpr (sizeof(T) == 8) return i + (i >> 5);
  else return spad<T>(i);
}

// A thread runs butterflies j = t + m TPL (m < PER) of a stage with BF = L/R
// butterflies; when TPL does not divide BF the last m is partial (j < BF).
template <typename T, int R, int NS, int TWOFF, bool DTW, int PER, int TPL, int BF>
__device__ __forceinline__ void split_compute(T (&vr)[PER][R], T (&vi)[PER][R], int t,
                                              const cplx_t<T>* __restrict__ tw) {
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    const int j = t + m * TPL;
    if (BF % TPL != 0 && j >= BF) continue;
    if (NS > 1) {
      const int jm = j % NS;
      if constexpr (DTW && R == 16) {
        twiddle16_derived<T, NS, TWOFF>(vr[m], vi[m], jm, tw);
      } else if constexpr (DTW && R == 32) {
        twiddle32_derived<T, NS, TWOFF>(vr[m], vi[m], jm, tw);
      } else {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const cplx_t<T> w = __ldg(tw + TWOFF + (r - 1) * NS + jm);
          cmul<T>(vr[m][r], vi[m][r], w.x, w.y);
        }
      }
    }
    Dft<R>::fwd(vr[m], vi[m]);
  }
}

// Stockham output positions of stage (R, NS): y[(j/NS) NS R + j%NS + k NS].
template <typename T, int R, int NS, int PER, int TPL, int BF>
__device__ __forceinline__ void split_put(T* buf, const T (&v)[PER][R], int t) {
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    const int j = t + m * TPL;
    if (BF % TPL != 0 && j >= BF) continue;
    const int base = (j / NS) * NS * R + (j % NS);
#pragma unroll
    for (int k = 0; k < R; ++k) buf[split_pad<T>(base + k * NS)] = v[m][k];
  }
}

// Input positions of stage (R, *) of an L-point line: x[j + r L/R].
template <typename T, int L, int R, int PER, int TPL>
__device__ __forceinline__ void split_get(const T* buf, T (&v)[PER][R], int t) {
  constexpr int BF = L / R;
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    const int j = t + m * TPL;
    if (BF % TPL != 0 && j >= BF) continue;
#pragma unroll
    for (int r = 0; r < R; ++r) v[m][r] = buf[split_pad<T>(j + r * BF)];
  }
}

template <typename T, int L, int TPL, int NS, int TWOFF, bool DTW, int R, int... Rest>
struct SplitRunner {
  static constexpr int BF = L / R;
  static constexpr int PER = (BF + TPL - 1) / TPL;
  __device__ __forceinline__ static void run(T* buf, const RowsLayout<T>& lay, int t,
                                             const cplx_t<T>* tw, T (&vr)[PER][R],
                                             T (&vi)[PER][R]) {
    split_compute<T, R, NS, TWOFF, DTW, PER, TPL, BF>(vr, vi, t, tw);
    if constexpr (sizeof...(Rest) == 0) {
#pragma unroll
      for (int m = 0; m < PER; ++m) {
        const int j = t + m * TPL;
        if (BF % TPL != 0 && j >= BF) continue;
        const int base = (j / NS) * NS * R + (j % NS);
#pragma unroll
        for (int k = 0; k < R; ++k) lay.gstore(base + k * NS, vr[m][k], vi[m][k]);
      }
    } else {
      using Next = SplitRunner<T, L, TPL, NS * R, TWOFF + stage_table_size(R, NS), DTW, Rest...>;
      constexpr int R2 = Next::kRadix;
      T nr[Next::PER][R2];
      T ni[Next::PER][R2];
      split_put<T, R, NS, PER, TPL, BF>(buf, vr, t);
      __syncthreads();
      split_get<T, L, R2, Next::PER, TPL>(buf, nr, t);
      __syncthreads();
      split_put<T, R, NS, PER, TPL, BF>(buf, vi, t);
      __syncthreads();
      split_get<T, L, R2, Next::PER, TPL>(buf, ni, t);
      __syncthreads();
      Next::run(buf, lay, t, tw, nr, ni);
    }
  }
  static constexpr int kRadix = R;
};

// One-pass tile with split exchanges: first stage loads global memory,
// last stage stores it, shared memory holds one component per line.
template <typename T, int L, int TPL, int TB, bool DTW, int R0, int... Rs>
__device__ __forceinline__ void rows_body_split(const RowsLayout<T>& lay, T* buf, int t,
                                                const cplx_t<T>* tw) {
  using First = SplitRunner<T, L, TPL, 1, 0, DTW, R0, Rs...>;
  constexpr int BF = L / R0;
  T vr[First::PER][R0];
  T vi[First::PER][R0];
#pragma unroll
  for (int m = 0; m < First::PER; ++m) {
    const int j = t + m * TPL;
    if (BF % TPL != 0 && j >= BF) continue;
#pragma unroll
    for (int r = 0; r < R0; ++r) lay.gload(j + r * BF, vr[m][r], vi[m][r]);
  }
  First::run(buf, lay, t, tw, vr, vi);
}

// ---------------------------------------------------------------------------
// ROWS kernel: single pass.  A CTA computes TB complete transforms of length
// L (each by TPL threads).  With STAGED, the CTA's TB*L contiguous input
// elements are first copied to shared memory with coalesced vector loads and
// the output leaves the same way (used when TPL is too small to coalesce).
// ---------------------------------------------------------------------------
template <typename T>
struct RowsArgs {
  const cplx_t<T>* in;
  cplx_t<T>* out;
  const cplx_t<T>* tw;      // internal stage tables
  long long batch;
  long long in_dist;
  long long out_dist;
  T sign;
  // Indirect batch (may be null): transform b reads in_table[b] and writes
  // out_table[b] instead of in + b*in_dist / out + b*out_dist.  This lets one
  // launch serve transforms that live in unrelated buffers.
  const cplx_t<T>* const* in_table;
  cplx_t<T>* const* out_table;
  // Prefetching kernels only: error word (may be null) that records a line
  // copy whose bounded wait ran out, and the failure check that never issues
  // a CTA's first copy.
  int* status;
  int lose_copy;
};

template <typename T>
__device__ __forceinline__ const cplx_t<T>* batch_in(const cplx_t<T>* base, long long dist,
                                                     const cplx_t<T>* const* table,
                                                     long long b) {
  return table ? table[b] : base + b * dist;
}
template <typename T>
__device__ __forceinline__ cplx_t<T>* batch_out(cplx_t<T>* base, long long dist,
                                                cplx_t<T>* const* table, long long b) {
  return table ? table[b] : base + b * dist;
}

// Pair-layout line pitch of a TB-line tile, in pairs: at least pair_line(L)
// and, for TB > 1, congruent to the threads per line modulo one 128-byte row
// of pairs, so that the lines a warp works on fall on distinct bank pairs.
template <typename T>
__host__ __device__ constexpr int pair_pitch(int L, int TPL, int TB, int SH = 4) {
  const int row = sizeof(T) == 4 ? 16 : 8;
  int p = pair_line(L, SH);
  if (TB > 1)
    while (p % row != TPL % row) ++p;
  return p;
}

// ROWS tile whose line lives in shared memory as {re, im} pairs
// (RowsPairLayout).  Staged tiles copy their lines between global and shared
// memory as they are (interleaved complex), 16 bytes per access where the
// tile is one dense aligned block, so the copies do no de-interleaving.
template <typename T, int L, int TPL, int TB, bool STAGED, bool DTW, int SH, int... Rs>
__device__ __forceinline__ void rows_body_pair(const RowsArgs<T>& a, long long b0,
                                               unsigned char* smem_raw,
                                               const RowsLayout<T>& lay, int line, int t) {
  constexpr int PP = pair_pitch<T>(L, TPL, TB, SH);
  cplx_t<T>* sp = reinterpret_cast<cplx_t<T>*>(smem_raw);
  RowsPairLayout<T, SH> lp;
  static_cast<RowsLayout<T>&>(lp) = lay;
  lp.sp = sp + line * PP;
  if constexpr (!STAGED) {
    StageRunner<T, L, TPL, 1, 0, false, false, true, DTW, Rs...>::run(lp, t, a.tw);
  } else {
    constexpr int kThreadsTile = TPL * TB;
    constexpr int kVecs = (int)(TB * L * sizeof(cplx_t<T>) / 16);
    constexpr int kPer = kVecs / kThreadsTile;
    constexpr int kPerVec = (int)(16 / sizeof(cplx_t<T>));
    constexpr bool kVecOk = kVecs % kThreadsTile == 0 && kPer >= 1 && kPer <= 16 &&
                            (TB * L * sizeof(cplx_t<T>)) % 16 == 0;
    bool dense = false;
    if constexpr (kVecOk) {
      dense = a.in_table == nullptr && a.out_table == nullptr && a.in_dist == L &&
              a.out_dist == L && b0 + TB <= a.batch &&
              ((reinterpret_cast<uintptr_t>(a.in) | reinterpret_cast<uintptr_t>(a.out)) & 15) ==
                  0;
    }
    const long long lines = (a.batch - b0) < TB ? (a.batch - b0) : TB;
    if constexpr (kVecOk) {
      if (dense) {
        const uint4* src = reinterpret_cast<const uint4*>(a.in + b0 * L);
        uint4 v[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) v[k] = __ldcg(src + threadIdx.x + k * kThreadsTile);
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
          const cplx_t<T>* c = reinterpret_cast<const cplx_t<T>*>(&v[k]);
#pragma unroll
          for (int e = 0; e < kPerVec; ++e) {
            const int q = (threadIdx.x + k * kThreadsTile) * kPerVec + e;
            const int ln = q / L;
            const int i = q - ln * L;
            cplx_t<T> w = c[e];
            w.y *= a.sign;
            sp[ln * PP + lp.paddr(i)] = w;
          }
        }
      }
    }
    if (!dense) {
      for (int q = threadIdx.x; q < TB * L; q += kThreadsTile) {
        const int ln = q / L;
        const int i = q - ln * L;
        if (ln < lines) {
          cplx_t<T> w = ld_global<T>(batch_in<T>(a.in, a.in_dist, a.in_table, b0 + ln) + i);
          w.y *= a.sign;
          sp[ln * PP + lp.paddr(i)] = w;
        }
      }
    }
    __syncthreads();
    StageRunner<T, L, TPL, 1, 0, true, true, true, DTW, Rs...>::run(lp, t, a.tw);
    if constexpr (kVecOk) {
      if (dense) {
        uint4* dst = reinterpret_cast<uint4*>(a.out + b0 * L);
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
          uint4 v;
          cplx_t<T>* c = reinterpret_cast<cplx_t<T>*>(&v);
#pragma unroll
          for (int e = 0; e < kPerVec; ++e) {
            const int q = (threadIdx.x + k * kThreadsTile) * kPerVec + e;
            const int ln = q / L;
            const int i = q - ln * L;
            c[e] = sp[ln * PP + lp.paddr(i)];
            c[e].y *= a.sign;
          }
          dst[threadIdx.x + k * kThreadsTile] = v;
        }
      }
    }
    if (!dense) {
      for (int q = threadIdx.x; q < TB * L; q += kThreadsTile) {
        const int ln = q / L;
        const int i = q - ln * L;
        if (ln < lines) {
          const cplx_t<T> w = sp[ln * PP + lp.paddr(i)];
          st_global<T>(batch_out<T>(a.out, a.out_dist, a.out_table, b0 + ln) + i, w.x,
                       w.y * a.sign);
        }
      }
    }
  }
}

// Body of one ROWS tile: transforms b0 .. b0+TB-1, run by threads
// 0 .. TPL*TB-1 of the CTA (every thread of the CTA must call it).
template <typename T, int L, int TPL, int TB, int FLAGS, int... Rs>
__device__ __forceinline__ void rows_body(const RowsArgs<T>& a, long long b0,
                                          unsigned char* smem_raw) {
  static_assert(StageProduct<L, Rs...>::value == L, "radices must multiply to L");
  constexpr bool STAGED = (FLAGS & kStaged) != 0;
  constexpr bool DTW = (FLAGS & kDerivedTw) != 0;
  constexpr int LINE = rows_line<T>(L, TPL, TB);
  T* sre = reinterpret_cast<T*>(smem_raw);
  T* sim = sre + TB * LINE;
  const int line = threadIdx.x / TPL;
  const int t = threadIdx.x % TPL;
  const long long b = b0 + line;
  RowsLayout<T> lay;
  lay.sre = sre + line * LINE;
  lay.sim = sim + line * LINE;
  lay.active = b < a.batch;
  lay.gin = lay.active ? batch_in<T>(a.in, a.in_dist, a.in_table, b) : a.in;
  lay.gout = lay.active ? batch_out<T>(a.out, a.out_dist, a.out_table, b) : a.out;
  lay.sign = a.sign;
  if constexpr ((FLAGS & kPairX) != 0) {
    static_assert((FLAGS & kSplitX) == 0, "pair and split exchanges exclude each other");
    rows_body_pair<T, L, TPL, TB, STAGED, DTW, pair_shift(FLAGS), Rs...>(a, b0, smem_raw, lay,
                                                                         line, t);
    return;
  }
  // Dense full tile: the TB lines are one contiguous, 16-byte aligned block
  // of TB*L elements, copied with unrolled 16-byte vector accesses so that a
  // thread has all of its loads in flight at once.
  constexpr int kThreadsTile = TPL * TB;
  constexpr int kVecs = (int)(TB * L * sizeof(cplx_t<T>) / 16);
  constexpr int kPer = kVecs / kThreadsTile;
  constexpr int kPerVec = (int)(16 / sizeof(cplx_t<T>));      // elements per vector
  constexpr bool kVecOk = STAGED && kVecs % kThreadsTile == 0 && kPer <= 16 &&
                          (TB * L * sizeof(cplx_t<T>)) % 16 == 0;
  bool dense = false;
  if constexpr (kVecOk) {
    dense = a.in_table == nullptr && a.out_table == nullptr && a.in_dist == L &&
            a.out_dist == L && b0 + TB <= a.batch &&
            ((reinterpret_cast<uintptr_t>(a.in) | reinterpret_cast<uintptr_t>(a.out)) & 15) == 0;
  }
  if constexpr (kVecOk) {
    if (dense) {
      const uint4* src = reinterpret_cast<const uint4*>(a.in + b0 * L);
      uint4 v[kPer > 0 ? kPer : 1];
#pragma unroll
      for (int k = 0; k < kPer; ++k) v[k] = __ldcg(src + threadIdx.x + k * kThreadsTile);
#pragma unroll
      for (int k = 0; k < kPer; ++k) {
        const cplx_t<T>* c = reinterpret_cast<const cplx_t<T>*>(&v[k]);
#pragma unroll
        for (int e = 0; e < kPerVec; ++e) {
          const int q = (threadIdx.x + k * kThreadsTile) * kPerVec + e;
          const int ln = q / L;
          const int i = q - ln * L;
          sre[ln * LINE + spad<T>(i)] = c[e].x;
          sim[ln * LINE + spad<T>(i)] = c[e].y * a.sign;
        }
      }
      __syncthreads();
    }
  }
  if (STAGED && !dense) {
    // Cooperative load of lines b0 .. b0+TB-1 (each L contiguous elements).
    const long long lines = (a.batch - b0) < TB ? (a.batch - b0) : TB;
    for (int q = threadIdx.x; q < TB * L; q += TPL * TB) {
      const int ln = q / L;
      const int i = q - ln * L;
      if (ln < lines) {
        const cplx_t<T> v =
            ld_global<T>(batch_in<T>(a.in, a.in_dist, a.in_table, b0 + ln) + i);
        sre[ln * LINE + spad<T>(i)] = v.x;
        sim[ln * LINE + spad<T>(i)] = v.y * a.sign;
      }
    }
    __syncthreads();
  }
  if constexpr ((FLAGS & kSplitX) != 0) {
    static_assert(!STAGED, "split exchanges run with direct global I/O");
    rows_body_split<T, L, TPL, TB, DTW, Rs...>(lay, sre + line * LINE, t, a.tw);
  } else {
    StageRunner<T, L, TPL, 1, 0, STAGED, STAGED, true, DTW, Rs...>::run(lay, t, a.tw);
  }
  if constexpr (kVecOk) {
    if (dense) {
      uint4* dst = reinterpret_cast<uint4*>(a.out + b0 * L);
#pragma unroll
      for (int k = 0; k < kPer; ++k) {
        uint4 v;
        cplx_t<T>* c = reinterpret_cast<cplx_t<T>*>(&v);
#pragma unroll
        for (int e = 0; e < kPerVec; ++e) {
          const int q = (threadIdx.x + k * kThreadsTile) * kPerVec + e;
          const int ln = q / L;
          const int i = q - ln * L;
          c[e].x = sre[ln * LINE + spad<T>(i)];
          c[e].y = sim[ln * LINE + spad<T>(i)] * a.sign;
        }
        dst[threadIdx.x + k * kThreadsTile] = v;
      }
    }
  }
  if (STAGED && !dense) {
    const long long lines = (a.batch - b0) < TB ? (a.batch - b0) : TB;
    for (int q = threadIdx.x; q < TB * L; q += TPL * TB) {
      const int ln = q / L;
      const int i = q - ln * L;
      if (ln < lines)
        st_global<T>(batch_out<T>(a.out, a.out_dist, a.out_table, b0 + ln) + i,
                     sre[ln * LINE + spad<T>(i)],
                     sim[ln * LINE + spad<T>(i)] * a.sign);
    }
  }
}

template <typename T, int L, int TPL, int TB, int FLAGS, int... Rs>
__global__ void __launch_bounds__(TPL * TB)
rows_kernel(const RowsArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  rows_body<T, L, TPL, TB, FLAGS, Rs...>(a, (long long)blockIdx.x * TB, smem_raw);
}

// The same with registers capped for two resident CTAs per SM (kTwoCtas).
template <typename T, int L, int TPL, int TB, int FLAGS, int... Rs>
__global__ void __launch_bounds__(TPL * TB, 2)
rows_kernel_2cta(const RowsArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  rows_body<T, L, TPL, TB, FLAGS, Rs...>(a, (long long)blockIdx.x * TB, smem_raw);
}

// ---------------------------------------------------------------------------
// Prefetching ROWS kernel (kPrefetch with kSplitX, one line per CTA step).
// A long one-pass line leaves room for one or two CTAs per SM, and a CTA that
// loads, transforms and stores its line in turn keeps HBM busy only while it
// loads.  Here the CTAs are persistent: while a CTA transforms line b, the
// input of its next line b + gridDim.x is already on its way into shared
// memory by one bulk asynchronous copy (cp.async.bulk, no multicast) that
// completes a transaction count on an mbarrier.  Shared memory holds that
// staging line (L complex, interleaved as in global memory) and the
// split-exchange buffer (L words).
//
// Every wait is bounded (kLineWaitNs of %globaltimer, or kLineWaitIters
// polls).  When it runs out the CTA records bit kLineCopyTimedOut in the
// status word, loads that line from global memory itself, stops prefetching
// and, before it exits, waits once more (bounded) for the copy it issued, so
// the output stays correct and no copy lands after the CTA has gone.
// ---------------------------------------------------------------------------
constexpr unsigned kLineWaitIters = 1u << 26;
constexpr unsigned long long kLineWaitNs = 1000000000ull;  // one second
constexpr int kLineCopyTimedOut = 4;

__device__ __forceinline__ unsigned long long line_clock_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the completion of the phase of `parity` of the mbarrier at
// shared address `bar`; false when it gave up.
__device__ __forceinline__ bool line_wait(uint32_t bar, uint32_t parity) {
  const unsigned long long t0 = line_clock_ns();
  for (unsigned it = 0; it < kLineWaitIters; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if ((it & 63u) == 63u && line_clock_ns() - t0 > kLineWaitNs) return false;
  }
  return false;
}

// One line into shared memory: the arrival that expects `bytes`, then the
// bulk copy that completes them (source and destination 16-byte aligned,
// bytes a multiple of 16).
__device__ __forceinline__ void line_copy(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// Shared memory of a prefetching CTA: mbarrier (16 bytes), staging line,
// split-exchange buffer.
template <typename T, int L, int TPL>
__host__ __device__ constexpr size_t prefetch_smem() {
  return 16 + (size_t)L * 2 * sizeof(T) + (size_t)rows_line<T>(L, TPL, 1) * sizeof(T);
}

template <typename T, int L, int TPL, int FLAGS, int R0, int... Rs>
__device__ __forceinline__ void rows_prefetch_body(const RowsArgs<T>& a, unsigned char* smem) {
  static_assert(StageProduct<L, R0, Rs...>::value == L, "radices must multiply to L");
  constexpr bool DTW = (FLAGS & kDerivedTw) != 0;
  using First = SplitRunner<T, L, TPL, 1, 0, DTW, R0, Rs...>;
  constexpr int BF = L / R0;
  constexpr uint32_t kLineBytes = (uint32_t)(L * sizeof(cplx_t<T>));
  static_assert(kLineBytes % 16 == 0, "bulk copies move multiples of 16 bytes");
  const cplx_t<T>* stage = reinterpret_cast<const cplx_t<T>*>(smem + 16);
  T* buf = reinterpret_cast<T*>(smem + 16 + kLineBytes);
  const uint32_t bar = (uint32_t)__cvta_generic_to_shared(smem);
  const uint32_t stage_addr = (uint32_t)__cvta_generic_to_shared(smem + 16);
  const int t = threadIdx.x;
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // Block-uniform prefetch state.
  bool prefetching = true;   // cleared once a wait has run out
  bool expect = false;       // line b's input is meant to be in `stage`
  bool issued = false;       // ... and its copy was issued
  bool stale = false;        // a copy whose wait ran out may still land
  uint32_t parity = 0, stale_parity = 0;
  auto start = [&](long long line, bool skip) {
    expect = issued = false;
    if (!prefetching || line >= a.batch) return;
    const cplx_t<T>* src = batch_in<T>(a.in, a.in_dist, a.in_table, line);
    if ((reinterpret_cast<uintptr_t>(src) & 15u) != 0) return;
    expect = true;
    if (skip) return;
    issued = true;
    if (t == 0) line_copy(stage_addr, src, kLineBytes, bar);
  };
  start(blockIdx.x, a.lose_copy != 0);

  for (long long b = blockIdx.x; b < a.batch; b += gridDim.x) {
    RowsLayout<T> lay;
    lay.sre = buf;
    lay.sim = buf;
    lay.active = true;
    lay.gin = batch_in<T>(a.in, a.in_dist, a.in_table, b);
    lay.gout = batch_out<T>(a.out, a.out_dist, a.out_table, b);
    lay.sign = a.sign;
    T vr[First::PER][R0];
    T vi[First::PER][R0];
    bool landed = expect ? line_wait(bar, parity) : true;
    landed = __syncthreads_and(landed) != 0;
    if (expect && landed) {
      parity ^= 1u;
#pragma unroll
      for (int m = 0; m < First::PER; ++m) {
        const int j = t + m * TPL;
        if (BF % TPL != 0 && j >= BF) continue;
#pragma unroll
        for (int r = 0; r < R0; ++r) {
          const cplx_t<T> v = stage[j + r * BF];
          vr[m][r] = v.x;
          vi[m][r] = v.y * a.sign;
        }
      }
    } else {
      if (expect) {
        if (t == 0 && a.status) atomicOr(a.status, kLineCopyTimedOut);
        prefetching = false;
        stale = issued;
        stale_parity = parity;
      }
#pragma unroll
      for (int m = 0; m < First::PER; ++m) {
        const int j = t + m * TPL;
        if (BF % TPL != 0 && j >= BF) continue;
#pragma unroll
        for (int r = 0; r < R0; ++r) lay.gload(j + r * BF, vr[m][r], vi[m][r]);
      }
    }
    __syncthreads();  // every thread is done with `stage` (and with `buf`)
    start(b + gridDim.x, false);
    First::run(buf, lay, t, a.tw, vr, vi);
  }
  if (stale && t == 0) (void)line_wait(bar, stale_parity);
}

template <typename T, int L, int TPL, int FLAGS, int... Rs>
__global__ void __launch_bounds__(TPL, (FLAGS & kTwoCtas) ? 2 : 1)
rows_prefetch_kernel(const RowsArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  rows_prefetch_body<T, L, TPL, FLAGS, Rs...>(a, smem_raw);
}

// ---------------------------------------------------------------------------
// COLS kernel: one pass of a multi-pass transform of total length M.
// Lines are the super-butterflies j in [0, M/L); a CTA owns C consecutive
// lines of one batch entry.  Line j reads x[j + i*S] (S = M/L), multiplies by
// W_{Ns*L}^{(j mod Ns)*i} and writes y[(j div Ns)*Ns*L + (j mod Ns) + k*Ns].
// When Ns == 1 the C output lines form one contiguous block that is stored
// from shared memory with coalesced writes (STAGED_OUT).
// ---------------------------------------------------------------------------
template <typename T>
struct ColsArgs {
  const cplx_t<T>* in;
  cplx_t<T>* out;
  const cplx_t<T>* tw;      // internal stage tables of the L-point DFT
  const cplx_t<T>* tw_hi;   // super-stage twiddle, two-level table
  const cplx_t<T>* tw_lo;
  long long batch;
  long long in_dist;        // distance between batch entries
  long long out_dist;
  long long total;          // M
  long long ns_outer;       // Ns of this pass (product of earlier super radices)
  int split_shift;
  T sign_in;
  T sign_out;
  const cplx_t<T>* const* in_table;   // indirect batch, may be null
  cplx_t<T>* const* out_table;
};

template <typename T, int L, int TPL, int C>
struct ColsGeom {
  static constexpr int PITCH = C + 1;           // words per element row
  static constexpr int WORDS = L * PITCH;       // per real/imag array
  static constexpr size_t SMEM = 2ull * WORDS * sizeof(T);
  static constexpr int THREADS = TPL * C;
};

// Addressing of this thread's line of a COLS tile (lines j0 .. j0+C-1 of
// batch entry b).
template <typename T, int L, int TPL, int C, bool TW, class Layout>
__device__ __forceinline__ void cols_layout(Layout& lay, const ColsArgs<T>& a, long long b,
                                            long long j0, T* sre, T* sim) {
  using G = ColsGeom<T, L, TPL, C>;
  const long long lines_total = a.total / L;            // M / L
  const int c = threadIdx.x % C;
  const long long j = j0 + c;
  const long long ns = a.ns_outer;
  const long long jq = j / ns;
  const long long jm = j - jq * ns;
  lay.sre = sre;
  lay.sim = sim;
  lay.c = c;
  const cplx_t<T>* in_b = batch_in<T>(a.in, a.in_dist, a.in_table, b);
  cplx_t<T>* out_b = batch_out<T>(a.out, a.out_dist, a.out_table, b);
  lay.gin = in_b + j;
  lay.in_stride = lines_total;
  lay.gout = out_b + jq * ns * L + jm;
  lay.out_stride = ns;
  lay.sign_in = a.sign_in;
  lay.sign_out = a.sign_out;
  lay.active = b < a.batch;
  lay.tw_hi = a.tw_hi;
  lay.tw_lo = a.tw_lo;
  lay.jmod = jm;
  lay.split_shift = a.split_shift;
  (void)G::THREADS;
}

// Body of one COLS tile: lines j0 .. j0+C-1 of batch entry b, run by threads
// 0 .. TPL*C-1 of the CTA (every thread of the CTA must call it).
template <typename T, int L, int TPL, int C, int... Rs>
__device__ __forceinline__ void cols_body(const ColsArgs<T>& a, long long b,
                                          long long j0, unsigned char* smem_raw) {
  static_assert(StageProduct<L, Rs...>::value == L, "radices must multiply to L");
  using G = ColsGeom<T, L, TPL, C>;
  T* sre = reinterpret_cast<T*>(smem_raw);
  T* sim = sre + G::WORDS;
  const int t = threadIdx.x / C;
  if (a.ns_outer == 1) {
    ColsLayout<T, C, G::PITCH, false> lay;
    cols_layout<T, L, TPL, C, false>(lay, a, b, j0, sre, sim);
    StageRunner<T, L, TPL, 1, 0, false, true, true, true, Rs...>::run(lay, t, a.tw);
    // lines j0..j0+C-1 are contiguous: out[b*dist + j0*L + c*L + k]
    cplx_t<T>* dst = batch_out<T>(a.out, a.out_dist, a.out_table, b) + j0 * L;
    if (lay.active) {
      for (int q = threadIdx.x; q < C * L; q += G::THREADS) {
        const int cc = q / L;
        const int k = q - cc * L;
        st_global<T>(dst + q, sre[k * G::PITCH + cc],
                     sim[k * G::PITCH + cc] * a.sign_out);
      }
    }
  } else {
    ColsLayout<T, C, G::PITCH, true> lay;
    cols_layout<T, L, TPL, C, true>(lay, a, b, j0, sre, sim);
    StageRunner<T, L, TPL, 1, 0, false, false, true, true, Rs...>::run(lay, t, a.tw);
  }
}

// Pair-exchange column tile: the C lines live in shared memory as {re, im}
// pairs (element-major, ColsGeom's PITCH = C + 1 pairs per element row), so
// each value crosses it as one 8- / 16-byte access; the odd pitch keeps the
// first pass's contiguous output copy (stride PITCH) on distinct banks.
template <typename T, int C, int PITCH, bool TW>
struct ColsPairLayout : ColsLayout<T, C, PITCH, TW> {
  static constexpr bool kPairTag = true;
  cplx_t<T>* sp;
  __device__ __forceinline__ int paddr(int i) const { return i * PITCH + this->c; }
  __device__ __forceinline__ void sget(int i, T& re, T& im) const {
    const cplx_t<T> v = sp[paddr(i)];
    re = v.x;
    im = v.y;
  }
  __device__ __forceinline__ void sput(int i, T re, T im) const {
    cplx_t<T> v;
    v.x = re;
    v.y = im;
    sp[paddr(i)] = v;
  }
};

template <typename T, int L, int TPL, int C, int... Rs>
__device__ __forceinline__ void cols_body_pair(const ColsArgs<T>& a, long long b,
                                               long long j0, unsigned char* smem_raw) {
  static_assert(StageProduct<L, Rs...>::value == L, "radices must multiply to L");
  using G = ColsGeom<T, L, TPL, C>;
  cplx_t<T>* sp = reinterpret_cast<cplx_t<T>*>(smem_raw);
  const int t = threadIdx.x / C;
  if (a.ns_outer == 1) {
    ColsPairLayout<T, C, G::PITCH, false> lay;
    cols_layout<T, L, TPL, C, false>(lay, a, b, j0, nullptr, nullptr);
    lay.sp = sp;
    StageRunner<T, L, TPL, 1, 0, false, true, true, true, Rs...>::run(lay, t, a.tw);
    cplx_t<T>* dst = batch_out<T>(a.out, a.out_dist, a.out_table, b) + j0 * L;
    if (lay.active) {
      for (int q = threadIdx.x; q < C * L; q += G::THREADS) {
        const int cc = q / L;
        const int k = q - cc * L;
        const cplx_t<T> v = sp[k * G::PITCH + cc];
        st_global<T>(dst + q, v.x, v.y * a.sign_out);
      }
    }
  } else {
    ColsPairLayout<T, C, G::PITCH, true> lay;
    cols_layout<T, L, TPL, C, true>(lay, a, b, j0, nullptr, nullptr);
    lay.sp = sp;
    StageRunner<T, L, TPL, 1, 0, false, false, true, true, Rs...>::run(lay, t, a.tw);
  }
}

template <typename T, int L, int TPL, int C, int... Rs>
__global__ void __launch_bounds__(TPL * C)
cols_kernel_pair(const ColsArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long long groups = (a.total / L) / C;
  const long long b = blockIdx.x / groups;
  const long long j0 = (blockIdx.x - b * groups) * C;
  cols_body_pair<T, L, TPL, C, Rs...>(a, b, j0, smem_raw);
}

template <typename T, int L, int TPL, int C, int... Rs>
__global__ void __launch_bounds__(TPL * C)
cols_kernel(const ColsArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long long groups = (a.total / L) / C;           // C divides M/L
  const long long b = blockIdx.x / groups;
  const long long j0 = (blockIdx.x - b * groups) * C;
  cols_body<T, L, TPL, C, Rs...>(a, b, j0, smem_raw);
}

// ---------------------------------------------------------------------------
// Generic kernel: runtime stage list, any radix of the reference set, used for
// lengths without a specialised instance.  Shared memory ping-pongs between two
// buffers; a CTA owns `lines` lines (ROWS: transforms; COLS: super-butterflies
// of a multi-pass transform, exactly as in cols_kernel).
// ---------------------------------------------------------------------------
constexpr int kMaxGenericStages = 24;

template <typename T>
struct GenericArgs {
  const cplx_t<T>* in;
  cplx_t<T>* out;
  const cplx_t<T>* tw;      // internal stage tables (runtime stage list)
  const cplx_t<T>* tw_hi;
  const cplx_t<T>* tw_lo;
  long long batch;
  long long in_dist;
  long long out_dist;
  long long total;          // COLS: M; ROWS: L
  long long ns_outer;       // COLS only
  int split_shift;
  int cols;                 // 0 = ROWS, 1 = COLS
  int length;               // L
  int lines;                // lines per CTA
  int stage_count;
  int radices[kMaxGenericStages];
  T sign_in;
  T sign_out;
};

template <typename T, int R, int BANK>
__device__ __forceinline__ void generic_butterfly(
    const GenericArgs<T>& a, const T* __restrict__ sre_src,
    const T* __restrict__ sim_src, T* __restrict__ sre_dst,
    T* __restrict__ sim_dst, int line, int j, int L, int NS, int twoff,
    bool first, bool last, int line_words, long long b, long long jline) {
  T vr[R];
  T vi[R];
  const int BF = L / R;
  const bool cols = a.cols != 0;
  // element address helpers: ROWS keeps each line contiguous, COLS interleaves
  // the lines (element-major) like cols_kernel.
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int idx = j + r * BF;
    if (first) {
      cplx_t<T> v;
      if (cols) {
        const long long S = a.total / L;
        v = ld_global<T>(a.in + b * a.in_dist + jline + (long long)idx * S);
      } else {
        v = ld_global<T>(a.in + b * a.in_dist + idx);
      }
      vr[r] = v.x;
      vi[r] = v.y * a.sign_in;
      if (cols && idx != 0) {
        const long long jm = jline % a.ns_outer;
        if (jm != 0) {
          const long long e = jm * (long long)idx;
          const cplx_t<T> hi = __ldg(a.tw_hi + (e >> a.split_shift));
          const cplx_t<T> lo = __ldg(a.tw_lo + (e & ((1LL << a.split_shift) - 1)));
          T wr = hi.x, wi = hi.y;
          cmul<T>(wr, wi, lo.x, lo.y);
          cmul<T>(vr[r], vi[r], wr, wi);
        }
      }
    } else {
      const int s = cols ? idx * (a.lines + 1) + line : line * line_words + spad<T>(idx);
      vr[r] = sre_src[s];
      vi[r] = sim_src[s];
    }
  }
  if (NS > 1) {
    const int jm = j % NS;
#pragma unroll
    for (int r = 1; r < R; ++r) {
      const cplx_t<T> w = __ldg(a.tw + twoff + (r - 1) * NS + jm);
      cmul<T>(vr[r], vi[r], w.x, w.y);
    }
  }
  BankDft<R, BANK>::fwd(vr, vi);
  const int base = (j / NS) * NS * R + (j % NS);
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const int idx = base + k * NS;
    if (last && !(cols && a.ns_outer == 1)) {
      if (cols) {
        const long long ns = a.ns_outer;
        const long long jq = jline / ns, jm = jline - jq * ns;
        st_global<T>(a.out + b * a.out_dist + jq * ns * L + jm + (long long)idx * ns,
                     vr[k], vi[k] * a.sign_out);
      } else {
        st_global<T>(a.out + b * a.out_dist + idx, vr[k], vi[k] * a.sign_out);
      }
    } else {
      const int s = cols ? idx * (a.lines + 1) + line : line * line_words + spad<T>(idx);
      sre_dst[s] = vr[k];
      sim_dst[s] = vi[k];
    }
  }
}

// WIDE selects the variant that also handles radix 32 and 64; chains without
// them use the narrow variant, whose register footprint allows several CTAs
// per SM.
template <typename T, bool WIDE, int BANK>
__device__ __forceinline__ void generic_dispatch(
    int R, const GenericArgs<T>& a, const T* sre_src, const T* sim_src,
    T* sre_dst, T* sim_dst, int line, int j, int L, int NS, int twoff,
    bool first, bool last, int line_words, long long b, long long jline) {
#define MOFFT_GENERIC_CASE(RR)                                                  \
  case RR:                                                                      \
    generic_butterfly<T, RR, BANK>(a, sre_src, sim_src, sre_dst, sim_dst, line, j, L, \
                             NS, twoff, first, last, line_words, b, jline);     \
    break;
  switch (R) {
    MOFFT_GENERIC_CASE(2) MOFFT_GENERIC_CASE(3) MOFFT_GENERIC_CASE(4)
    MOFFT_GENERIC_CASE(5) MOFFT_GENERIC_CASE(6) MOFFT_GENERIC_CASE(7)
    MOFFT_GENERIC_CASE(8) MOFFT_GENERIC_CASE(9) MOFFT_GENERIC_CASE(10)
    MOFFT_GENERIC_CASE(11) MOFFT_GENERIC_CASE(12) MOFFT_GENERIC_CASE(13)
    MOFFT_GENERIC_CASE(14) MOFFT_GENERIC_CASE(15) MOFFT_GENERIC_CASE(16)
    default:
      if (WIDE) {
        if (R == 32)
          generic_butterfly<T, 32, BANK>(a, sre_src, sim_src, sre_dst, sim_dst, line, j, L,
                                   NS, twoff, first, last, line_words, b, jline);
        else if (R == 64)
          generic_butterfly<T, 64, BANK>(a, sre_src, sim_src, sre_dst, sim_dst, line, j, L,
                                   NS, twoff, first, last, line_words, b, jline);
      }
      break;
  }
#undef MOFFT_GENERIC_CASE
}

// BANK: the kernel bank whose codelets the stages run (0 default, 1-3 the
// rewrite families of BankDft).
template <typename T, bool WIDE, int BANK>
__global__ void __launch_bounds__(256, WIDE ? 1 : 2) generic_kernel(const GenericArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int L = a.length;
  const bool cols = a.cols != 0;
  const int line_words = cols ? 0 : spad_len<T>(L);
  const int buf_words = cols ? L * (a.lines + 1) : a.lines * line_words;
  T* bufs[2][2];
  T* base = reinterpret_cast<T*>(smem_raw);
  bufs[0][0] = base;
  bufs[0][1] = base + buf_words;
  bufs[1][0] = base + 2 * buf_words;
  bufs[1][1] = base + 3 * buf_words;
  long long b, jfirst;
  if (cols) {
    const long long groups = (a.total / L) / a.lines;
    b = blockIdx.x / groups;
    jfirst = (blockIdx.x - b * groups) * a.lines;
  } else {
    b = (long long)blockIdx.x * a.lines;
    jfirst = 0;
  }
  int NS = 1;
  int twoff = 0;
  int cur = 0;
  for (int s = 0; s < a.stage_count; ++s) {
    const int R = a.radices[s];
    const int BF = L / R;
    const bool first = s == 0;
    const bool last = s == a.stage_count - 1;
    const int work = BF * a.lines;
    for (int w = threadIdx.x; w < work; w += blockDim.x) {
      int line, j;
      if (cols) {
        line = w % a.lines;
        j = w / a.lines;
      } else {
        line = w / BF;
        j = w - line * BF;
      }
      const long long bb = cols ? b : b + line;
      if (bb >= a.batch) continue;
      const long long jline = cols ? jfirst + line : 0;
      generic_dispatch<T, WIDE, BANK>(R, a, bufs[cur][0], bufs[cur][1], bufs[cur ^ 1][0],
                          bufs[cur ^ 1][1], line, j, L, NS, twoff, first, last,
                          line_words, cols ? b : bb, jline);
    }
    __syncthreads();
    cur ^= 1;
    twoff += stage_table_size(R, NS);
    NS *= R;
  }
  if (cols && a.ns_outer == 1 && b < a.batch) {
    // lines jfirst .. jfirst+lines-1 are contiguous in the output
    cplx_t<T>* dst = a.out + b * a.out_dist + jfirst * L;
    const int pitch = a.lines + 1;
    for (int q = threadIdx.x; q < a.lines * L; q += blockDim.x) {
      const int cc = q / L;
      const int k = q - cc * L;
      st_global<T>(dst + q, bufs[cur][0][k * pitch + cc],
                   bufs[cur][1][k * pitch + cc] * a.sign_out);
    }
  }
}

}  // namespace mofft
