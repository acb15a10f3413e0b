// One-pass transforms longer than one CTA's shared memory: a thread-block
// cluster of K CTAs computes one transform of N = N1 * N2 points, and the
// cluster's distributed shared memory carries the transpose of the four-step
// algorithm.  The line then crosses HBM once (read once, written once) where
// a multi-pass schedule of column kernels moves it once per pass.
//
//   x[N2 n1 + n2]  ->  X[k1 + N1 k2]
//
//   phase A   CTA c owns the columns n2 in [c CA, (c+1) CA), CA = N2 / K.  It
//             loads them (for each n1, CA adjacent elements) and computes
//             their N1-point DFTs Y[k1][n2]: Stockham stages with
//             shared-memory exchanges, the column kernels' tile (ColsLayout).
//   exchange  Z[k1][n2] = Y[k1][n2] W_N^{n2 k1} belongs to the CTA that owns
//             row k1 (d = k1 / CB, CB = N1 / K).  Every CTA writes its Z into
//             its own shared memory as K tiles, tile d holding rows
//             d CB .. d CB + CB - 1 of its CA columns, then sends tile d to
//             CTA d with one bulk asynchronous copy (shared::cta to
//             shared::cluster, no multicast) that completes a transaction
//             count on CTA d's mbarrier.  The copy engine moves the tiles;
//             the threads issue K copies instead of one remote store per
//             element.
//   phase B   CTA d waits (bounded) until its mbarrier has seen all K tiles,
//             computes the N2-point DFTs of its CB rows and stores
//             X[k1 + N1 k2]: CB adjacent outputs per k2.
//
// The tiles arrive in a receive buffer of their own, so no CTA waits for
// another one to finish reading: a cluster barrier at the start (every
// mbarrier is initialised before any copy targets it; its arrival is made
// early and waited for just before the copies) and one at the end (a CTA
// arrives once all its tiles have landed and waits before it exits, so no
// CTA leaves while a copy still reads its shared memory) are the only
// cluster-wide synchronisation.  Both are hardware barriers that every
// thread reaches on the same path.  The tile wait is bounded by one second
// of %globaltimer; when it runs out the CTA sets bit kClusterTileTimedOut of
// the pass's error word and finishes on what arrived (the host then reports
// MOFFT_INTERNAL_ERROR).  The tiles that were sent had long landed by then,
// so the end barrier still means that no copy is in flight.
//
// Twiddles: the kernel's own table (aux): the internal stage tables of the
// N1- and N2-point chains, then W_N^{n2 j} (j < N1 / RL, RL the last phase-A
// radix) and W_N^{n2 (N1/RL) k} (k < RL), both [row][n2] so that the lanes of
// a warp read adjacent entries; the exchange twiddle of k1 = j + k N1/RL is
// their product.
//
// This is the transform the reference computes with its four-step driver for
// lengths beyond one codelet tile (src/mofft.c:1932-2045, first codelet,
// twiddle, transpose, second codelet), with the transpose carried by the
// cluster's shared memory instead of a materialised array.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "fft_device.cuh"
#include "fft_instances.cuh"
#include "mofft_cuda.h"
#include "mofft_host.h"

namespace mofft {
namespace {

namespace cg = cooperative_groups;

constexpr int kClusterTileTimedOut = 8;

// Address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_map(uint32_t addr, uint32_t rank) {
  uint32_t out;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(addr), "r"(rank));
  return out;
}

// One tile to another CTA's shared memory (dst and bar are shared::cluster
// addresses of that CTA, src a shared::cta address of this one; both
// 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void tile_send(uint32_t dst, uint32_t src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(dst),
      "r"(src), "r"(bytes), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void cluster_arrive_relaxed() {
  asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Phase B: the receive buffer holds K tiles, tile s from CTA s: its CB rows
// of CA columns (columns s CA .. s CA + CA - 1), real parts (row pitch CA + 1
// words) then imaginary parts, BW words each.  Element i of this thread's row
// c lives in tile i / CA, column i % CA.
template <typename T, int CA, int BW>
struct ClusterTileLayout {
  T* sre;                 // receive buffer (real parts of tile 0)
  T* sim;                 // sre + BW
  int c;                  // this thread's row
  cplx_t<T>* gout;        // X[k1] of this row
  long long out_stride;   // N1
  T sign;
  bool active;
  __device__ __forceinline__ int saddr(int i) const {
    return (i / CA) * (2 * BW) + c * (CA + 1) + (i % CA);
  }
  __device__ __forceinline__ void gload(int, T& re, T& im) const {
    re = T(0);
    im = T(0);
  }
  __device__ __forceinline__ void gstore(int i, T re, T im) const {
    if (active) st_global<T>(gout + (long long)i * out_stride, re, im * sign);
  }
  template <int R>
  __device__ __forceinline__ void super_twiddle(int, int, T (&)[R], T (&)[R]) const {}
};

constexpr int chain_table(const int* r, int n) {
  int t = 0, ns = 1;
  for (int i = 0; i < n; ++i) {
    if (ns > 1) t += (r[i] - 1) * ns;
    ns *= r[i];
  }
  return t;
}
constexpr int round32(int x) { return (x + 31) & ~31; }
constexpr int round_up(int x, int m) { return (x + m - 1) / m * m; }

// Geometry of one instance.  HeadA: the phase-A radices before the last one
// (RL); RsB: the phase-B radices.
template <typename TT, int N1_, int N2_, int K_, int TPLA_, int TPLB_, int RL_, class HeadA,
          class RsB>
struct ClusterFft;

template <typename TT, int N1_, int N2_, int K_, int TPLA_, int TPLB_, int RL_, int... HA,
          int... RB>
struct ClusterFft<TT, N1_, N2_, K_, TPLA_, TPLB_, RL_, RadixList<HA...>, RadixList<RB...>> {
  using T = TT;
  using Head = RadixList<HA...>;
  using Tail = RadixList<RB...>;
  static constexpr int N1 = N1_, N2 = N2_, K = K_, TPLA = TPLA_, TPLB = TPLB_, RL = RL_;
  static constexpr int N = N1 * N2;
  static constexpr int CA = N2 / K;            // phase-A columns per CTA
  static constexpr int CB = N1 / K;            // phase-B rows per CTA
  static constexpr int THREADS = TPLA * CA;
  static constexpr int NSL = N1 / RL;          // product of the head radices
  static constexpr int PA = CA + 1;            // phase-A words per element row
  static constexpr int WA = N1 * PA;           // phase-A words per component
  static constexpr int BW = CB * (CA + 1);     // words of one component of a tile
  static constexpr uint32_t TILE_BYTES = 2u * BW * sizeof(T);
  // words of the phase-A / send buffer and its byte offset of the receive
  // buffer (16-byte aligned); the mbarrier takes the first 16 bytes
  static constexpr int PW = round_up(2 * WA > 2 * K * BW ? 2 * WA : 2 * K * BW,
                                     16 / (int)sizeof(T));
  static constexpr size_t OFF_P = 16;
  static constexpr size_t OFF_R = OFF_P + (size_t)PW * sizeof(T);
  static constexpr size_t SMEM = OFF_R + (size_t)K * TILE_BYTES;
  static constexpr int kA[] = {HA..., RL};
  static constexpr int kB[] = {RB...};
  static constexpr int NA = (int)sizeof...(HA) + 1;
  static constexpr int NB = (int)sizeof...(RB);
  static constexpr int HEAD_TABLE = chain_table(kA, NA - 1);
  // aux layout, complex entries: stage tables of A and B (each with one
  // spare entry), then W_N^{n2 j} [j][n2] and W_N^{n2 NSL k} [k][n2]
  static constexpr int OFF_B = round32(chain_table(kA, NA) + 1);
  static constexpr int OFF_BASE = OFF_B + round32(chain_table(kB, NB) + 1);
  static constexpr int OFF_U = OFF_BASE + NSL * N2;
  static constexpr int AUX = OFF_U + RL * N2;
  // resident CTAs per SM the registers allow at 64 (FP32) / 128 (FP64)
  // registers a thread
  static constexpr int MIN_CTAS_RAW = 65536 / (THREADS * (sizeof(T) == 4 ? 64 : 128));
  static constexpr int MIN_CTAS = MIN_CTAS_RAW < 1 ? 1 : (MIN_CTAS_RAW > 4 ? 4 : MIN_CTAS_RAW);
  static_assert(N1 % K == 0 && N2 % K == 0, "K divides both factors");
  static_assert(THREADS == TPLB * CB, "both phases use every thread");
  static_assert(StageProduct<N1, HA..., RL>::value == N1, "phase-A radices");
  static_assert(StageProduct<N2, RB...>::value == N2, "phase-B radices");
  static_assert(CA * 2 * sizeof(T) >= 128 && CB * 2 * sizeof(T) >= 128,
                "coalesced rows of at least 128 bytes");
  static_assert(K >= 2 && K <= 16, "cluster sizes up to 16 (above 8: non-portable)");
  static_assert(THREADS <= 1024 && THREADS >= K, "one CTA, one copy thread per tile");
  static_assert(TILE_BYTES % 16 == 0, "bulk copies move multiples of 16 bytes");
  static_assert(OFF_R % 16 == 0, "16-byte aligned receive buffer");
  static_assert(SMEM <= 227 * 1024, "shared memory of one CTA");
};

template <class F, class HeadA, class RsB>
struct ClusterBody;

template <class F, int... HA, int... RB>
struct ClusterBody<F, RadixList<HA...>, RadixList<RB...>> {
  using T = typename F::T;
  static constexpr int RL = F::RL;
  static constexpr int NSL = F::NSL;
  static constexpr int CA = F::CA;
  static constexpr int CB = F::CB;
  static constexpr int BW = F::BW;
  __device__ __forceinline__ static void run(const RowsArgs<T>& a,
                                             const cplx_t<T>* __restrict__ aux) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* p = reinterpret_cast<T*>(smem_raw + F::OFF_P);
    T* rbuf = reinterpret_cast<T*>(smem_raw + F::OFF_R);
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(smem_raw);
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      // this CTA's K incoming tiles complete the phase
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                   "r"((uint32_t)(F::K * F::TILE_BYTES))
                   : "memory");
    }
    // start barrier: arrive now, wait just before the first copy
    cluster_arrive_relaxed();

    const long long b = blockIdx.x / F::K;
    const cplx_t<T>* in_b = batch_in<T>(a.in, a.in_dist, a.in_table, b);
    cplx_t<T>* out_b = batch_out<T>(a.out, a.out_dist, a.out_table, b);

    // ---- phase A: N1-point DFTs of columns rank*CA .. rank*CA+CA-1
    const int col = threadIdx.x % CA;
    const int ta = threadIdx.x / CA;
    ColsLayout<T, CA, F::PA, false> la;
    la.sre = p;
    la.sim = p + F::WA;
    la.c = col;
    la.gin = in_b + rank * CA + col;
    la.gout = nullptr;
    la.in_stride = F::N2;
    la.out_stride = 0;
    la.sign_in = a.sign;
    la.sign_out = T(1);
    la.active = true;
    la.tw_hi = nullptr;
    la.tw_lo = nullptr;
    la.jmod = 0;
    la.split_shift = 0;
    if constexpr (sizeof...(HA) > 0)
      StageRunner<T, F::N1, F::TPLA, 1, 0, false, true, true, true, HA...>::run(la, ta, aux);

    // last phase-A stage (radix RL, Ns = NSL): butterfly j < NSL yields
    // k1 = j + k NSL
    constexpr int BF = NSL;
    constexpr int PER = (BF + F::TPLA - 1) / F::TPLA;
    constexpr bool EVEN = (BF % F::TPLA) == 0;
    T vr[PER][RL];
    T vi[PER][RL];
#pragma unroll
    for (int m = 0; m < PER; ++m) {
      const int j = ta + m * F::TPLA;
      if (EVEN || j < BF) {
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int idx = j + r * BF;
          if constexpr (sizeof...(HA) == 0) {
            la.gload(idx, vr[m][r], vi[m][r]);
          } else {
            vr[m][r] = la.sre[la.saddr(idx)];
            vi[m][r] = la.sim[la.saddr(idx)];
          }
        }
        if constexpr (NSL > 1) {
          if constexpr (RL == 16) {
            twiddle16_derived<T, NSL, F::HEAD_TABLE>(vr[m], vi[m], j, aux);
          } else if constexpr (RL == 32) {
            twiddle32_derived<T, NSL, F::HEAD_TABLE>(vr[m], vi[m], j, aux);
          } else {
#pragma unroll
            for (int r = 1; r < RL; ++r) {
              const cplx_t<T> w = __ldg(aux + F::HEAD_TABLE + (r - 1) * NSL + j);
              cmul<T>(vr[m][r], vi[m][r], w.x, w.y);
            }
          }
        }
        Dft<RL>::fwd(vr[m], vi[m]);
      }
    }
    if constexpr (sizeof...(HA) > 0) __syncthreads();   // the buffer is read

    // ---- exchange: Z[k1][n2] into tile d = k1 / CB, row k1 - d CB
    const int n2 = rank * CA + col;
#pragma unroll
    for (int m = 0; m < PER; ++m) {
      const int j = ta + m * F::TPLA;
      if (EVEN || j < BF) {
        const cplx_t<T> w0 = __ldg(aux + F::OFF_BASE + j * F::N2 + n2);
#pragma unroll
        for (int k = 0; k < RL; ++k) {
          T wr = w0.x, wi = w0.y;
          if (k > 0) {
            const cplx_t<T> u = __ldg(aux + F::OFF_U + k * F::N2 + n2);
            cmul<T>(wr, wi, u.x, u.y);
          }
          T xr = vr[m][k], xi = vi[m][k];
          cmul<T>(xr, xi, wr, wi);
          const int k1 = j + k * NSL;
          const int d = k1 / CB;
          const int q = d * (2 * BW) + (k1 - d * CB) * (CA + 1) + col;
          p[q] = xr;
          p[q + BW] = xi;
        }
      }
    }
    // the tiles are read by the copy engine (async proxy)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    // every mbarrier of the cluster is initialised and armed
    cluster_wait();
    if (threadIdx.x < F::K && !(a.lose_copy && rank == 0)) {
      const uint32_t d = threadIdx.x;
      const uint32_t src = (uint32_t)__cvta_generic_to_shared(p + d * (2 * BW));
      const uint32_t dst = cluster_map(
          (uint32_t)__cvta_generic_to_shared(rbuf + rank * (2 * BW)), d);
      tile_send(dst, src, F::TILE_BYTES, cluster_map(bar, d));
    }
    // every tile of this CTA's rows has landed (bounded wait)
    if (!line_wait(bar, 0)) {
      if (threadIdx.x == 0 && a.status) atomicOr(a.status, kClusterTileTimedOut);
    }
    // end barrier: arrive once the tiles are in, wait before exit
    cluster_arrive_relaxed();

    // ---- phase B: N2-point DFTs of rows rank*CB .. rank*CB+CB-1
    ClusterTileLayout<T, CA, BW> lb;
    lb.sre = rbuf;
    lb.sim = rbuf + BW;
    lb.c = threadIdx.x % CB;
    lb.gout = out_b + rank * CB + lb.c;
    lb.out_stride = F::N1;
    lb.sign = a.sign;
    lb.active = true;
    StageRunner<T, F::N2, F::TPLB, 1, 0, true, false, true, true, RB...>::run(
        lb, (int)(threadIdx.x / CB), aux + F::OFF_B);
    // no CTA exits while a tile it sent may still be read
    cluster_wait();
  }
};

template <class F>
__global__ void __launch_bounds__(F::THREADS, F::MIN_CTAS)
cluster_kernel(const RowsArgs<typename F::T> a, const cplx_t<typename F::T>* aux) {
  ClusterBody<F, typename F::Head, typename F::Tail>::run(a, aux);
}

template <class F>
struct ClusterInst {
  using T = typename F::T;
  static const void* func() { return reinterpret_cast<const void*>(&cluster_kernel<F>); }
  static cudaError_t launch(const mofft_pass_args* p, cudaStream_t s) {
    if (p->conj_in != p->conj_out || !p->aux) return cudaErrorInvalidValue;
    if (p->batch <= 0) return cudaSuccess;
    const long long grid = p->batch * F::K;
    if (grid > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    if (F::K > 8) {
      // clusters of more than 8 CTAs are opted into once per device
      static int allowed[64] = {0};
      int dev = 0;
      if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return cudaErrorInvalidDevice;
      if (!allowed[dev]) {
        const cudaError_t e = cudaFuncSetAttribute(
            cluster_kernel<F>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
        allowed[dev] = 1;
      }
    }
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(F::THREADS, 1, 1);
    cfg.dynamicSmemBytes = F::SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = F::K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const RowsArgs<T> a = rows_args<T>(p);
    const cplx_t<T>* aux = static_cast<const cplx_t<T>*>(p->aux);
    return cudaLaunchKernelEx(&cfg, cluster_kernel<F>, a, aux);
  }
  // The kernel's twiddle table (see the layout in ClusterFft).
  static int fill_aux(void* dst) {
    const int bits = sizeof(T) == 4 ? 32 : 64;
    const size_t cb = 2 * sizeof(T);
    unsigned char* p = static_cast<unsigned char*>(dst);
    memset(p, 0, (size_t)F::AUX * cb);
    mofft_fill_stage_table(p, bits, F::kA, F::NA);
    mofft_fill_stage_table(p + (size_t)F::OFF_B * cb, bits, F::kB, F::NB);
    for (int j = 0; j < F::NSL; ++j)
      mofft_write_twiddles(p + (size_t)(F::OFF_BASE + j * F::N2) * cb, bits, (uint64_t)F::N, 0,
                           (uint64_t)j, (size_t)F::N2);
    for (int k = 0; k < F::RL; ++k)
      mofft_write_twiddles(p + (size_t)(F::OFF_U + k * F::N2) * cb, bits, (uint64_t)F::N, 0,
                           (uint64_t)F::NSL * (uint64_t)k, (size_t)F::N2);
    return 0;
  }
  static Entry entry(const char* name) {
    Entry e{};
    e.desc.name = name;
    e.desc.precision_bits = sizeof(T) == 4 ? 32 : 64;
    e.desc.kind = MOFFT_KERNEL_ROWS;
    e.desc.length = F::N;
    e.desc.lines = 1;
    e.desc.threads = F::THREADS;
    e.desc.cluster = F::K;
    e.desc.radix_count = F::NA + F::NB;
    for (int i = 0; i < 8; ++i)
      e.desc.radices[i] = i < F::NA ? F::kA[i] : (i < F::NA + F::NB ? F::kB[i - F::NA] : 0);
    e.desc.smem_bytes = F::SMEM;
    e.launch = &launch;
    e.func = &func;
    e.aux_bytes = (size_t)F::AUX * 2 * sizeof(T);
    e.fill_aux = &fill_aux;
    return e;
  }
};

#define MOFFT_UNPAREN(...) __VA_ARGS__
#define MOFFT_CLUSTER(T, N1, N2, K, TPLA, TPLB, RL, HEAD, TAIL)                          \
  ClusterInst<ClusterFft<T, N1, N2, K, TPLA, TPLB, RL, RadixList<MOFFT_UNPAREN HEAD>,    \
                         RadixList<MOFFT_UNPAREN TAIL>>>::entry(                         \
      "cluster_" #T "_" #N1 "x" #N2 "_k" #K)

}  // namespace

const Entry* entries_cluster(int* count) {
  static const Entry e[] = {
      // 4096 FP32 / 2048 FP64 points per CTA, three to four resident CTAs
      // per SM
      MOFFT_CLUSTER(float, 128, 128, 4, 8, 8, 8, (16), (16, 8)),
      MOFFT_CLUSTER(float, 128, 256, 8, 8, 16, 8, (16), (16, 16)),
      MOFFT_CLUSTER(float, 256, 256, 16, 16, 16, 16, (16), (16, 16)),
      MOFFT_CLUSTER(double, 128, 128, 8, 8, 8, 8, (16), (16, 8)),
      MOFFT_CLUSTER(double, 128, 256, 16, 8, 16, 8, (16), (16, 16)),
  };
  *count = (int)(sizeof(e) / sizeof(e[0]));
  return e;
}

}  // namespace mofft
