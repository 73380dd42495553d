// dev_tc.cu — split-BF16 GEMM on the sm_100a tensor cores (tcgen05 + TMA).
//
// C = alpha * op(A) op(B) + beta * C with FP64 operands.  Each operand is split
// into NSL BF16 slices x = x0 + x1 (+ x2) (x0 = bf16(x), x1 = bf16(x - x0),
// x2 = bf16(x - x0 - x1)) stored K-major and zero padded (rows to 128, K to 64).
// NSL = 3 accumulates the six products x0y0 x0y1 x1y0 x1y1 x0y2 x2y0 in FP32
// (relative error ~2^-24 of sum |a||b|, FP32-like); NSL = 2 accumulates
// x0y0 x0y1 x1y0 (~2^-16, for sums whose element errors average out, such as
// the (T) energy).
//
// Kernel: persistent, one CTA per SM over 128 x TN output tiles (TN = 128,
// 160 or 256).  TMA loads (3-D tensor maps: k, row, slice; 64-wide boxes of
// 128 or TN rows, 128-byte swizzle) feed a ring of at most 216 KiB (2 or 3
// stages); tcgen05.mma kind::f16 (BF16 x BF16 -> F32, M=128 N=TN K=16) accumulates in
// one of two tensor-memory accumulators while eight epilogue warps drain the
// other with tcgen05.ld and write C (FP64 or FP32, through an index map whose
// rows run along the lanes).  Every mbarrier wait is bounded (1 s); on
// time-out the kernel records an error code, lets its own loads and MMAs in
// flight finish (bounded), frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ecg_dev.h"
#include "ecg_tune.h"
#include "tma_util.cuh"

namespace ecg {
namespace dev {

namespace {

// Tiles: 128 rows (M) x TN columns (N), K = 64; TN = 128, TN_WIDE = 160 or
// TN_XWIDE = 256, chosen per GEMM by tile_n: 160 covers N = 300 or 318 in 320
// columns where 128 needs 384; 256 (two-slice operands only: two stages of
// 96 KiB) halves the A-operand traffic per MMA where it pads N by at most 2%
// more than 128 does.
constexpr int TM = 128, TK = 64, TN_WIDE = 160, TN_XWIDE = 256;
constexpr int TILE_BYTES_A = TM * TK * 2;  // 16 KiB per slice
constexpr int RING_BYTES = 216 * 1024;
// longest K (in 64-wide k-blocks) one FP32 tensor-memory accumulator sums
// before its partial product is handed to an FP64 reduction
constexpr int KB_ACC = (int)(TC_ACC_K / TK);
// Bound on every mbarrier wait: 1 s.  The main-loop waits (producer, MMA
// issuer, epilogue) take the stream's bound instead when one is set (kernel
// argument wait_ns); the final waits for the kernel's own TMA loads and MMAs
// in flight always keep the full second, so nothing is in flight when the CTA
// frees its tensor memory and exits.
using tma::WAIT_NS;
using tma::gtime;
using tma::mbar_expect_tx;
using tma::mbar_init;
using tma::mbar_wait;
using tma::smem_u32;
using tma::tma_load_3d;

template <int NSL, int TN>
struct TcCfg {
  static constexpr int TILE_BYTES_B = TN * TK * 2;
  static constexpr int STAGE_BYTES = NSL * (TILE_BYTES_A + TILE_BYTES_B);
  static constexpr int STAGES = RING_BYTES / STAGE_BYTES;
  static constexpr int NPAIR = NSL == 3 ? 6 : 3;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*barriers*/ + 1024 /*align*/;
  // two TN-column accumulators; allocations are powers of two
  static constexpr uint32_t TMEM_COLS = 2 * TN <= 256 ? 256 : 512;
  // instruction descriptor: kind::f16, A/B BF16, D F32, both K-major, M=128, N=TN
  static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) |
                                    ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
  static_assert(TN % 16 == 0 && TN <= 256 && STAGES >= 2, "tile shape");
  static_assert(SMEM_BYTES <= 227 * 1024, "shared memory");
  static_assert(TILE_BYTES_B % 1024 == 0, "128-byte-swizzle tiles start on 1024 bytes");
};
// slice pairs (a, b): hi*hi, hi*mid, mid*hi, mid*mid, hi*lo, lo*hi (the first
// three for NSL = 2)
__host__ __device__ constexpr int pair_a(int p) { return p == 2 || p == 3 ? 1 : p == 5 ? 2 : 0; }
__host__ __device__ constexpr int pair_b(int p) { return p == 1 || p == 3 ? 1 : p == 4 ? 2 : 0; }

__device__ int g_tc_error = 0;

// UMMA shared-memory descriptor, K-major operand in the 128-byte-swizzled
// canonical layout: 128-byte rows, 8-row (1024-byte) groups.
__device__ __forceinline__ uint64_t umma_desc(const void* p) {
  const uint32_t a = smem_u32(p);
  uint64_t d = (uint64_t)((a & 0x3FFFF) >> 4);  // start address
  d |= (uint64_t)1 << 16;                        // leading byte offset (unused for SW128 K-major)
  d |= (uint64_t)(1024 >> 4) << 32;              // stride byte offset: 8-row group
  d |= (uint64_t)1 << 46;                        // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                        // layout: SWIZZLE_128B
  return d;
}

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                     uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          smem_u32(bar)));
}

// Persistent, warp-specialised kernel: gridDim.x CTAs (one per SM) loop over
// work items (m-tile, n-tile, k-slice).  Warp 0 lane 0: TMA producer over a
// STAGES-deep shared-memory ring (full/empty mbarriers).  Warp 1: owns the
// tensor-memory allocation, lane 0 issues the MMAs into one of two TN-column
// accumulators and commits.  Warps 2..9: epilogue, each reading
// the 32 accumulator lanes its warp index (mod 4) may access and one half of
// the columns, writing C and releasing the accumulator, so the epilogue of
// one tile overlaps the MMAs of the next.
constexpr int EPI_WARPS = 8;  // two per TMEM lane quarter, TN/2 columns each
constexpr int THREADS_TC = 32 * (2 + EPI_WARPS);

// TMA descriptors of up to TC_MAX_SEG K segments, each read from its own k = 0.
struct TcMaps {
  CUtensorMap a[TC_MAX_SEG], b[TC_MAX_SEG];
};

// K layout of the segments: segment s covers the k-blocks [kb_end[s-1],
// kb_end[s]) (kb_end nondecreasing, unused trailing segments repeat the total);
// its last k-block issues kk_last[s] of the TK/16 MMA steps, the rest of that
// block being zero padding.
struct TcSegs {
  int kb_end[TC_MAX_SEG];
  int kk_last[TC_MAX_SEG];
};

// Segment of global k-block kg: index, first k-block, end, MMA steps of its
// last k-block (selects only, no indexed parameter reads).
struct SegPos {
  int s, start, end, kk_last;
};
__device__ __forceinline__ SegPos seg_of(const TcSegs& sg, int kg) {
  SegPos p{0, 0, sg.kb_end[0], sg.kk_last[0]};
#pragma unroll
  for (int t = 1; t < TC_MAX_SEG; ++t)
    if (kg >= sg.kb_end[t - 1]) p = SegPos{t, sg.kb_end[t - 1], sg.kb_end[t], sg.kk_last[t]};
  return p;
}

// Output element (m, n) lives at C[rowoff(m) + coloff(n)] (FP64, or FP32 when
// f32) with rowoff(m) = (m % dm)*scm + (m / dm)*scm2 (dm = 0: m*scm) and
// coloff(n) = (n % dn)*scn + (n / dn)*scn2 (dn = 0: n*scn).  Lanes of an
// epilogue warp hold consecutive rows, so scm == 1 gives coalesced stores.
struct TcOut {
  void* C;
  int64_t scm, scn, dn, scn2, dm, scm2;
  int f32;
};

// Epilogue of one 16-column chunk: this lane's row (offset rowoff), columns
// col0 .. col0+15.  Read-modify-write loads are all issued before the stores.
// FP32 output with beta 0 or 1 and an alpha that FP32 holds exactly is
// updated in FP32 (one rounding, as the FP64 expression rounded to FP32
// gives): the FP64 route costs three conversions per element, which bounded
// the epilogue of the (T) GEMMs.  Column arithmetic is 32-bit (N < 2^31).
template <typename CT>
__device__ __forceinline__ void epi_chunk(CT* __restrict__ C, int64_t rowoff, const uint32_t* r,
                                          int64_t col0, int64_t N, const TcOut& out,
                                          double alpha, double beta, bool f32math) {
  int64_t off[16];
  if (out.dn == 0) {
    const int64_t b = rowoff + col0 * out.scn;
#pragma unroll
    for (int j = 0; j < 16; ++j) off[j] = b + j * out.scn;
  } else {
    const uint32_t dn = (uint32_t)out.dn, nq = (uint32_t)col0 / dn;
    int64_t nr = (uint32_t)col0 - nq * dn;
    int64_t coff = nr * out.scn + (int64_t)nq * out.scn2;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      off[j] = rowoff + coff;
      ++nr;
      coff += out.scn;
      if (nr == out.dn) {
        nr = 0;
        coff += out.scn2 - out.dn * out.scn;
      }
    }
  }
  if (sizeof(CT) == 4 && f32math) {
    const float a = (float)alpha;
    if (beta != 0.0) {  // beta == 1
      CT old[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) old[j] = (col0 + j < N) ? C[off[j]] : (CT)0;
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (col0 + j < N) C[off[j]] = (CT)fmaf(a, __uint_as_float(r[j]), (float)old[j]);
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (col0 + j < N) C[off[j]] = (CT)(a * __uint_as_float(r[j]));
    }
  } else if (beta != 0.0) {
    CT old[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) old[j] = (col0 + j < N) ? C[off[j]] : (CT)0;
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (col0 + j < N)
        C[off[j]] = (CT)(alpha * (double)__uint_as_float(r[j]) + beta * (double)old[j]);
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (col0 + j < N) C[off[j]] = (CT)(alpha * (double)__uint_as_float(r[j]));
  }
}

template <int NSL, int TN>
__global__ void __launch_bounds__(THREADS_TC, 1)
    mgemm_bf16_kernel(const __grid_constant__ TcMaps maps, TcOut out, int64_t M, int64_t N,
                      double alpha, double beta, const TcSegs segs, int kb_per_split,
                      int kblocks_total,
                      int64_t split_stride, int mtiles, int ntiles, int nsplit,
                      const TcMaps* __restrict__ mtab, unsigned long long wait_ns) {
  using Cfg = TcCfg<NSL, TN>;
  constexpr int STAGES = Cfg::STAGES, STAGE_BYTES = Cfg::STAGE_BYTES;
  constexpr int TILE_BYTES_B = Cfg::TILE_BYTES_B;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* tiles = smem;
  uint64_t* full = (uint64_t*)(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* tfull = empty + STAGES;  // [2] accumulator ready
  uint64_t* tempty = tfull + 2;      // [2] accumulator drained
  uint32_t* tmem_slot = (uint32_t*)(tempty + 2);
  int* abort_flag = (int*)(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t items = (int64_t)mtiles * ntiles * nsplit;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], EPI_WARPS);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    asm volatile("fence.proxy.async.shared::cta;\n" ::);
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(Cfg::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;

  // the dimension with fewer tiles runs fastest, so that CTAs working at the
  // same time share the tiles of the larger operand through L2
  const bool mfast = mtiles <= ntiles;
  auto item_coords = [&](int64_t it, int& mt, int& nt, int& z) {
    if (mfast) {
      mt = (int)(it % mtiles);
      nt = (int)((it / mtiles) % ntiles);
    } else {
      nt = (int)(it % ntiles);
      mt = (int)((it / ntiles) % mtiles);
    }
    z = (int)(it / ((int64_t)mtiles * ntiles));
  };
  // z is a K slice (mtab == nullptr) or a batch item with its own operand maps
  // (mtab[z]), each covering all k-blocks
  auto item_kblocks = [&](int z) {
    return mtab ? kblocks_total : min(kb_per_split, kblocks_total - z * kb_per_split);
  };

  if (warp == 0) {
    if (lane == 0) {
      int64_t g = 0;  // global k-block counter of this CTA
      for (int64_t it = blockIdx.x; it < items && !*(volatile int*)abort_flag; it += gridDim.x) {
        int mt, nt, z;
        item_coords(it, mt, nt, z);
        const int nk = item_kblocks(z), kb0 = mtab ? 0 : z * kb_per_split;
        const TcMaps* mp = mtab ? mtab + z : &maps;
        for (int kb = 0; kb < nk; ++kb, ++g) {
          const int s = (int)(g % STAGES);
          const int64_t u = g / STAGES;
          if (u > 0 && !mbar_wait(&empty[s], (uint32_t)((u - 1) & 1), wait_ns)) {
            atomicExch(&g_tc_error, 1);
            atomicExch(abort_flag, 1);
            break;
          }
          uint8_t* st = tiles + s * STAGE_BYTES;
          const int kg = kb0 + kb;
          const SegPos sp = seg_of(segs, kg);
          const CUtensorMap* ma = &mp->a[sp.s];
          const CUtensorMap* mb = &mp->b[sp.s];
          const int kx = (kg - sp.start) * TK;
          mbar_expect_tx(&full[s], STAGE_BYTES);
          for (int t = 0; t < NSL; ++t) {
            tma_load_3d(st + t * TILE_BYTES_A, ma, &full[s], kx, mt * TM, t);
            tma_load_3d(st + NSL * TILE_BYTES_A + t * TILE_BYTES_B, mb, &full[s], kx, nt * TN, t);
          }
        }
      }
      // drain: every issued load must land before the CTA can exit
      for (int s = 0; s < STAGES && g > 0; ++s) {
        const int64_t last = g - 1 - ((g - 1 - s) % STAGES + STAGES) % STAGES;
        if (last >= 0) mbar_wait(&full[last % STAGES], (uint32_t)((last / STAGES) & 1));
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int64_t g = 0, lt = 0, last = -1;
      for (int64_t it = blockIdx.x; it < items && !*(volatile int*)abort_flag;
           it += gridDim.x, ++lt) {
        int mt, nt, z;
        item_coords(it, mt, nt, z);
        const int nk = item_kblocks(z), kb0 = mtab ? 0 : z * kb_per_split;
        const int acc = (int)(lt & 1);
        const int64_t ua = lt >> 1;
        if (ua > 0 && !mbar_wait(&tempty[acc], (uint32_t)((ua - 1) & 1), wait_ns)) {
          atomicExch(&g_tc_error, 4);
          atomicExch(abort_flag, 1);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        const uint32_t dcol = tmem + (uint32_t)(acc * TN);
        bool ok = true;
        for (int kb = 0; kb < nk; ++kb, ++g) {
          const int s = (int)(g % STAGES);
          if (!mbar_wait(&full[s], (uint32_t)((g / STAGES) & 1), wait_ns)) {
            atomicExch(&g_tc_error, 2);
            atomicExch(abort_flag, 1);
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
          const uint8_t* st = tiles + s * STAGE_BYTES;
          const uint8_t* As = st;
          const uint8_t* Bs = st + NSL * TILE_BYTES_A;
          const SegPos sp = seg_of(segs, kb0 + kb);
          const int nkk = (kb0 + kb == sp.end - 1) ? sp.kk_last : TK / 16;
#pragma unroll
          for (int p = 0; p < Cfg::NPAIR; ++p) {
            const uint64_t da = umma_desc(As + pair_a(p) * TILE_BYTES_A);
            const uint64_t db = umma_desc(Bs + pair_b(p) * TILE_BYTES_B);
#pragma unroll
            for (int kk = 0; kk < TK / 16; ++kk)
              if (kk < nkk)
                umma(dcol, da + (uint64_t)(kk * 2), db + (uint64_t)(kk * 2), Cfg::IDESC,
                     (kb > 0 || p > 0 || kk > 0) ? 1u : 0u);
          }
          umma_commit(&empty[s]);
        }
        umma_commit(&tfull[acc]);
        last = lt;
        if (!ok) break;
      }
      // the MMAs in flight must finish before the accumulators are freed
      if (last >= 0) mbar_wait(&tfull[last & 1], (uint32_t)((last >> 1) & 1));
    }
  } else {
    // epilogue warps 2..9: TMEM lane quarter q = warp % 4, column half hw
    const int q = warp & 3, hw = (warp - 2) >> 2;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    const bool f32math = (beta == 0.0 || beta == 1.0) && (double)(float)alpha == alpha;
    int64_t lt = 0;
    for (int64_t it = blockIdx.x; it < items; it += gridDim.x, ++lt) {
      int mt, nt, z;
      item_coords(it, mt, nt, z);
      const int acc = (int)(lt & 1);
      const int64_t row = (int64_t)mt * TM + q * 32 + lane;
      int64_t rowoff = (int64_t)z * split_stride;
      if (out.dm > 0) {
        const int64_t mq = row / out.dm;
        rowoff += (row - mq * out.dm) * out.scm + mq * out.scm2;
      } else {
        rowoff += row * out.scm;
      }
      // every lane waits; the warp goes on only if all lanes saw the
      // accumulator ready and no time-out was recorded, so the warp-wide
      // tcgen05.ld below always runs converged
      const bool ready = mbar_wait(&tfull[acc], (uint32_t)((lt >> 1) & 1), wait_ns);
      if (!__all_sync(0xffffffffu, ready)) {
        if (lane == 0) {
          atomicExch(&g_tc_error, 3);
          atomicExch(abort_flag, 1);
        }
        break;
      }
      if (__any_sync(0xffffffffu, *(volatile int*)abort_flag != 0)) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
#pragma unroll 1
      for (int c = hw * (TN / 2); c < (hw + 1) * (TN / 2); c += 16) {
        uint32_t r[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
            "%13,%14,%15}, [%16];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
              "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
              "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(tmem + lane_base + (uint32_t)(acc * TN + c)));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::);
        if (row < M) {
          const int64_t col0 = (int64_t)nt * TN + c;
          if (out.f32)
            epi_chunk((float*)out.C, rowoff, r, col0, N, out, alpha, beta, f32math);
          else
            epi_chunk((double*)out.C, rowoff, r, col0, N, out, alpha, beta, false);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(
                          smem_u32(&tempty[acc])));
    }
  }
  __syncwarp();
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(Cfg::TMEM_COLS));
  }
}

// X(r,k) = src[r*sr + k*sk] (FP64, R x K) -> dst[s][r][k] BF16 (s < nsl), zero
// padded to Rp x Kp.  32x32 tiles through shared memory so that reads are
// coalesced whichever of sr / sk is the unit stride.
__global__ void split_kernel(const double* __restrict__ src, int64_t R, int64_t K, int64_t sr,
                             int64_t sk, int64_t Rp, int64_t Kp, int nsl,
                             __nv_bfloat16* __restrict__ dst) {
  __shared__ double tile[32][33];
  // tile indices in 32 bits (an operand whose BF16 slices fit in device
  // memory has fewer than 2^25 tiles): one 64-bit division per tile would
  // cost more instructions than its 1024 elements
  const uint32_t tk = (uint32_t)((Kp + 31) / 32), ntile = tk * (uint32_t)((Rp + 31) / 32);
  const bool rfast = (sr == 1);
  for (uint32_t t = blockIdx.x; t < ntile; t += gridDim.x) {
    const int64_t r0 = (int64_t)(t / tk) * 32, k0 = (int64_t)(t % tk) * 32;
    // the four loads of a thread are issued before any of them is used
    double xs[4];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int j = threadIdx.y + 8 * jj;
      int64_t r, k;
      if (rfast) { r = r0 + threadIdx.x; k = k0 + j; } else { r = r0 + j; k = k0 + threadIdx.x; }
      xs[jj] = (r < R && k < K) ? src[r * sr + k * sk] : 0.0;
    }
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int j = threadIdx.y + 8 * jj;
      if (rfast) tile[j][threadIdx.x] = xs[jj];   // tile[k][r]
      else tile[threadIdx.x][j] = xs[jj];         // tile[k][r]
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
      const int64_t r = r0 + j, k = k0 + threadIdx.x;
      if (r < Rp && k < Kp) {
        const double x = tile[threadIdx.x][j];
        const __nv_bfloat16 h0 = __double2bfloat16(x);
        const double e1 = x - (double)__bfloat162float(h0);
        const __nv_bfloat16 h1 = __double2bfloat16(e1);
        const double e2 = e1 - (double)__bfloat162float(h1);
        const int64_t o = r * Kp + k, sl = Rp * Kp;
        dst[o] = h0;
        dst[o + sl] = h1;
        if (nsl == 3) dst[o + 2 * sl] = __double2bfloat16(e2);
      }
    }
    __syncthreads();
  }
}

}  // namespace

EncodeFn g_encode = nullptr;
std::mutex g_encode_mu;

int encode_fn(EncodeFn* out) {
  std::lock_guard<std::mutex> lk(g_encode_mu);
  if (!g_encode) {
    cudaDriverEntryPointQueryResult q;
    void* f = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !f)
      return e ? (int)e : (int)cudaErrorSymbolNotFound;
    g_encode = (EncodeFn)f;
  }
  *out = g_encode;
  return 0;
}

namespace {


// rows: extent of the map (rows past it read as zero); slice_stride in BF16
// elements (default: rows * k_p, a dense [slice][row][k] block)
int make_map(EncodeFn enc, CUtensorMap* m, const void* base, int64_t rows, int64_t k_p, int nsl,
             int64_t slice_stride = 0, int box_rows = TM) {
  if (slice_stride == 0) slice_stride = rows * k_p;
  cuuint64_t dims[3] = {(cuuint64_t)k_p, (cuuint64_t)rows, (cuuint64_t)nsl};
  cuuint64_t strides[2] = {(cuuint64_t)(k_p * 2), (cuuint64_t)(slice_stride * 2)};
  cuuint32_t box[3] = {(cuuint32_t)TK, (cuuint32_t)box_rows, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides,
                   box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : (int)cudaErrorInvalidValue;
}

int64_t pad_rows(int64_t r) { return (r + TM - 1) / TM * TM; }
int64_t pad_k(int64_t k) { return (k + TK - 1) / TK * TK; }

// Tile width for N columns of operands with nsl slices: the widest of 256
// (two slices only) and 160 that pads N by at most 2% more than 128 does (and
// N >= the width), else 128.  Wider tiles read fewer operand bytes per MMA.
// A B operand has N rows at least, so the map of the chosen box exists; a
// last tile reaching past the operand's rows reads zeros (TMA out-of-bounds
// fill).
int tile_n(int64_t n, int nsl) {
  const int64_t p128 = (n + 127) / 128 * 128, p160 = (n + TN_WIDE - 1) / TN_WIDE * TN_WIDE;
  const int64_t p256 = (n + TN_XWIDE - 1) / TN_XWIDE * TN_XWIDE;
  if (nsl == 2 && n >= TN_XWIDE && p256 * 50 <= p128 * 51) return TN_XWIDE;
  return (n >= TN_WIDE && p160 * 50 <= p128 * 51) ? TN_WIDE : 128;
}

// The B-operand descriptor for tile width tn, or nullptr if not encoded.
const unsigned char* b_map(const TcOperand* b, int tn) {
  if (tn == TN_XWIDE) return b->xwide ? b->map_x : nullptr;
  if (tn == TN_WIDE) return b->wide ? b->map_w : nullptr;
  return b->map;
}

// All descriptors of an operand whose fields are set; the maps' row extent
// is `extent` (rows past it read as zero).
int encode_operand(EncodeFn enc, TcOperand* op, int64_t extent) {
  op->wide = op->xwide = false;
  std::memset(op->map_w, 0, sizeof(op->map_w));
  std::memset(op->map_x, 0, sizeof(op->map_x));
  int e = make_map(enc, reinterpret_cast<CUtensorMap*>(op->map), op->base, extent, op->k_p,
                   op->slices, op->slice_stride);
  if (e || extent < TN_WIDE) return e;
  e = make_map(enc, reinterpret_cast<CUtensorMap*>(op->map_w), op->base, extent, op->k_p,
               op->slices, op->slice_stride, TN_WIDE);
  op->wide = (e == 0);
  if (e || extent < TN_XWIDE) return e;
  e = make_map(enc, reinterpret_cast<CUtensorMap*>(op->map_x), op->base, extent, op->k_p,
               op->slices, op->slice_stride, TN_XWIDE);
  op->xwide = (e == 0);
  return e;
}

// Segment k-block layout of nseg segments of K depths k[s] (padded to TK).
TcSegs make_segs(int nseg, const int64_t* k) {
  TcSegs sg;
  int end = 0;
  for (int t = 0; t < TC_MAX_SEG; ++t) {
    if (t < nseg) {
      const int64_t kp = pad_k(k[t]);
      end += (int)(kp / TK);
      sg.kk_last[t] = (int)((k[t] - (kp - TK) + 15) / 16);
    } else {
      sg.kk_last[t] = TK / 16;
    }
    sg.kb_end[t] = end;
  }
  return sg;
}

// Total K depth of the segments (without the zero padding of each segment's
// last k-block).
double seg_depth(const TcSegs& sg) {
  double k = 0.0;
  int prev = 0;
  for (int t = 0; t < TC_MAX_SEG; ++t) {
    const int nkb = sg.kb_end[t] - prev;
    if (nkb > 0) k += (double)(nkb - 1) * TK + 16.0 * sg.kk_last[t];
    prev = sg.kb_end[t];
  }
  return k;
}

// Checks the segments of g (A[s]/B[s] until the first null A[s]) and returns
// their number, or 0 if they do not form a valid GEMM of g's shape.
int gemm_segments(const TcGemm& g, int64_t* k) {
  int ns = 0;
  const TcOperand* A0 = g.A[0];
  const TcOperand* B0 = g.B[0];
  if (!A0 || !B0) return 0;
  for (; ns < TC_MAX_SEG && g.A[ns]; ++ns) {
    const TcOperand* A = g.A[ns];
    const TcOperand* B = g.B[ns];
    if (!B || A->k != B->k || A->k <= 0 || A->rows < g.m || B->rows < g.n ||
        A->slices != A0->slices || B->slices != A0->slices)
      return 0;
    k[ns] = A->k;
  }
  for (int t = ns; t < TC_MAX_SEG; ++t)
    if (g.B[t]) return 0;
  return ns;
}

void launch_split(cudaStream_t st, const double* src, int64_t R, int64_t K, int64_t sr,
                  int64_t sk, int64_t Rp, int64_t Kp, int nsl, __nv_bfloat16* dst) {
  const int64_t tiles = ((Rp + 31) / 32) * ((Kp + 31) / 32);
  const unsigned g = (unsigned)(tiles < 148 * 16 ? tiles : 148 * 16);
  split_kernel<<<g, dim3(32, 8), 0, st>>>(src, R, K, sr, sk, Rp, Kp, nsl, dst);
  note_launches(1);
}

// K slices of a GEMM with `tiles` output tiles and kbt k-blocks: enough to
// fill the SMs when the output has fewer tiles than SMs (at least 4 k-blocks
// per slice), and so that no FP32 accumulator sums more than KB_ACC k-blocks
// (the slices' partial products are added in FP64).
int split_count(int64_t tiles, int kbt) {
  int S = 1;
  if (tiles < 148 && kbt >= 8) S = (int)std::min<int64_t>((148 + tiles - 1) / tiles, kbt / 4);
  return std::max(S, (kbt + KB_ACC - 1) / KB_ACC);
}

// Launch over pre-split operands; S > 1 splits the combined k-blocks into S
// slices that write FP64 partial products P[z][n][m] (column-major m x n).
// cudaFuncSetAttribute acts on the current device only: one flag per device.
template <int NSL, int TN>
void set_smem_attr() {
  static std::atomic<bool> done[128] = {};
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) {
    cudaGetLastError();
    d = -1;
  }
  if (d >= 0 && d < 128 && done[d].load(std::memory_order_acquire)) return;
  if (cudaFuncSetAttribute(mgemm_bf16_kernel<NSL, TN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           TcCfg<NSL, TN>::SMEM_BYTES) == cudaSuccess) {
    if (d >= 0 && d < 128) done[d].store(true, std::memory_order_release);
  } else {
    cudaGetLastError();
  }
}

// The stream's main-loop wait bound (0: the default second).
unsigned long long wait_bound(cudaStream_t st) {
  const uint64_t w = tc_wait((stream_t)st);
  return w ? (unsigned long long)w : WAIT_NS;
}

template <int NSL, int TN>
int launch_tc(cudaStream_t st, const TcMaps& maps, const TcSegs& segs, int kbt, int64_t m,
              int64_t n, int64_t mp, int64_t np, double alpha, double beta, const TcOut& out,
              int S) {
  using Cfg = TcCfg<NSL, TN>;
  set_smem_attr<NSL, TN>();
  const int mt = (int)(mp / TM), nt = (int)(np / TN);
  const int kps = (kbt + S - 1) / S;
  S = (kbt + kps - 1) / kps;
  const int64_t items = (int64_t)mt * nt * S;
  const unsigned grid = (unsigned)(items < 148 ? items : 148);
  const unsigned long long wns = wait_bound(st);
  // useful BF16 products: 2 m n K per slice pair (zero padding not counted)
  const double work = 2.0 * (double)m * (double)n * (double)seg_depth(segs) * Cfg::NPAIR;
  const int slot = ktime_begin((stream_t)st, KT_TCGEMM);
  if (S == 1) {
    mgemm_bf16_kernel<NSL, TN><<<grid, THREADS_TC, Cfg::SMEM_BYTES, st>>>(
        maps, out, m, n, alpha, beta, segs, kps, kbt, 0, mt, nt, 1, nullptr, wns);
    note_launches(1);
    ktime_end((stream_t)st, KT_TCGEMM, slot, work);
    return (int)cudaGetLastError();
  }
  if (out.f32 || out.dn > 0 || out.dm > 0) return (int)cudaErrorInvalidValue;
  // partial products in FP32, exactly as tensor memory accumulated them (one
  // accumulation each), summed in FP64 by the reduction
  float* P = reinterpret_cast<float*>(splitk_buffer((stream_t)st, ((size_t)S * m * n + 1) / 2));
  if (!P) return (int)cudaErrorMemoryAllocation;
  TcOut po{P, 1, m, 0, 0, 0, 0, 1};
  mgemm_bf16_kernel<NSL, TN><<<grid, THREADS_TC, Cfg::SMEM_BYTES, st>>>(
      maps, po, m, n, 1.0, 0.0, segs, kps, kbt, m * n, mt, nt, S, nullptr, wns);
  note_launches(1);
  int e = (int)cudaGetLastError();
  if (e) return e;
  e = splitk_reduce_f32((stream_t)st, m, n, S, P, alpha, beta, (double*)out.C, out.scm, out.scn);
  ktime_end((stream_t)st, KT_TCGEMM, slot, work);
  return e;
}

}  // namespace

size_t tc_operand_elems(int64_t rows, int64_t k, int slices) {
  return (size_t)slices * (size_t)pad_rows(rows) * (size_t)pad_k(k);
}

int tc_split(stream_t s, const double* src, int64_t rows, int64_t k, int64_t sr, int64_t sk,
             int slices, void* dst, TcOperand* op) {
  if (rows <= 0 || k <= 0 || !dst || !op || (slices != 2 && slices != 3))
    return (int)cudaErrorInvalidValue;
  if (((uintptr_t)dst & 15) != 0) return (int)cudaErrorMisalignedAddress;
  EncodeFn enc = nullptr;
  int e = encode_fn(&enc);
  if (e) return e;
  static_assert(sizeof(CUtensorMap) == sizeof(op->map), "tensor map storage");
  op->rows = rows;
  op->k = k;
  op->rows_p = pad_rows(rows);
  op->k_p = pad_k(k);
  op->slices = slices;
  op->base = dst;
  op->slice_stride = op->rows_p * op->k_p;
  launch_split((cudaStream_t)s, src, rows, k, sr, sk, op->rows_p, op->k_p, slices,
               (__nv_bfloat16*)dst);
  e = (int)cudaGetLastError();
  if (e) return e;
  return encode_operand(enc, op, op->rows_p);
}

int64_t tc_pad_rows(int64_t rows) { return pad_rows(rows); }
int64_t tc_pad_k(int64_t k) { return pad_k(k); }

int tc_bind(void* dst, int64_t rows, int64_t k, int slices, TcOperand* op) {
  if (rows <= 0 || k <= 0 || !dst || !op || (slices != 2 && slices != 3))
    return (int)cudaErrorInvalidValue;
  if (((uintptr_t)dst & 15) != 0) return (int)cudaErrorMisalignedAddress;
  EncodeFn enc = nullptr;
  int e = encode_fn(&enc);
  if (e) return e;
  op->rows = rows;
  op->k = k;
  op->rows_p = pad_rows(rows);
  op->k_p = pad_k(k);
  op->slices = slices;
  op->base = dst;
  op->slice_stride = op->rows_p * op->k_p;
  return encode_operand(enc, op, op->rows_p);
}

namespace {

// dst[k + t*sl] = slice t of x (t = 0, 1, 2), the split of split_kernel
__device__ __forceinline__ void put_slices3(__nv_bfloat16* dst, int64_t sl, int64_t k, double x) {
  const __nv_bfloat16 h0 = __double2bfloat16(x);
  const double e1 = x - (double)__bfloat162float(h0);
  const __nv_bfloat16 h1 = __double2bfloat16(e1);
  const double e2 = e1 - (double)__bfloat162float(h1);
  dst[k] = h0;
  dst[k + sl] = h1;
  dst[k + 2 * sl] = __double2bfloat16(e2);
}

// One thread per (pair row pr, packed index k < kp_p) of the symmetric
// operand, in the element order of ladder_pack_v: X[c,d] = V[c + v a' + lda
// (d + v b')] with (c, d) = cdp[k], c <= d; X[d,c] is reread from L2 by the
// neighbouring rows' threads.  Row pr gets X[c,d] + X[d,c] (X[c,c] on the
// diagonal) at k, and for a < b and c < d row pr - a' - 1 of the
// antisymmetric operand gets X[c,d] - X[d,c] at k - d = d(d-1)/2 + c; the K
// padding of both is written as zeros.
// One thread per element; the tiled kernel below replaces it wherever its
// tile count fits 32 bits (always, for blocks that fit in device memory).
// IT: index type of the element loop.
template <typename VT, typename IT>
__global__ void ladder_pack_split_kernel(int nv, int a0, int na, int npairs,
                                         const int2* __restrict__ pairs,
                                         const int2* __restrict__ cdp, const VT* __restrict__ V,
                                         int64_t kp_p, int64_t sl_p, int64_t kp_m, int64_t sl_m,
                                         __nv_bfloat16* __restrict__ Vp,
                                         __nv_bfloat16* __restrict__ Vm) {
  const int64_t v = nv, lda = v * na, ncdp = v * (v + 1) / 2, ncdm = v * (v - 1) / 2;
  const int64_t mpad = kp_m - ncdm;
  const IT total = (IT)kp_p * (IT)npairs, kpi = (IT)kp_p;
  for (IT idx = blockIdx.x * (IT)blockDim.x + threadIdx.x; idx < total;
       idx += (IT)gridDim.x * blockDim.x) {
    const int64_t k = idx % kpi, pr = idx / kpi;
    const int2 ab = pairs[pr];
    const int64_t ap = ab.x - a0, bp = ab.y - a0;
    const bool minus = ab.x < ab.y;
    __nv_bfloat16* om = minus ? Vm + (pr - ap - 1) * kp_m : Vm;
    if (k < ncdp) {
      const int2 cd = cdp[k];
      const double x = (double)V[cd.x + v * ap + lda * (cd.y + v * bp)];
      const double y = (double)V[cd.y + v * ap + lda * (cd.x + v * bp)];
      put_slices3(Vp + pr * kp_p, sl_p, k, cd.x == cd.y ? x : x + y);
      if (minus && cd.x < cd.y) put_slices3(om, sl_m, k - cd.y, x - y);
    } else {
      put_slices3(Vp + pr * kp_p, sl_p, k, 0.0);
    }
    if (minus && k < mpad) put_slices3(om, sl_m, ncdm + k, 0.0);
  }
}

// Upper-triangle tile id -> (tile row tc, tile column td), tc <= td, in the
// order id = td (td + 1) / 2 + tc.
__device__ __forceinline__ void tri_tile(uint32_t id, uint32_t& tc, uint32_t& td) {
  uint32_t t = (uint32_t)((sqrtf(8.0f * (float)id + 1.0f) - 1.0f) * 0.5f);
  while (t * (t + 1) / 2 > id) --t;
  while ((t + 1) * (t + 2) / 2 <= id) ++t;
  td = t;
  tc = id - t * (t + 1) / 2;
}

// ladder_pack_split_kernel by 32 x 32 tiles of (c, d), c0 <= d0, one pair
// (a, b) per tile: X[c,d] read along c, the mirrored X[d,c] along d into
// shared memory, so every load and store is coalesced.  The block of a pair's
// first tile also writes the zero padding of its rows (k >= ncdp of V+,
// k >= ncdm of V-).  Block 32 x 8.
template <typename VT>
__global__ void ladder_pack_split_tiled_kernel(int nv, int a0, int na, int npairs,
                                               const int2* __restrict__ pairs,
                                               const VT* __restrict__ V, int64_t kp_p,
                                               int64_t sl_p, int64_t kp_m, int64_t sl_m,
                                               __nv_bfloat16* __restrict__ Vp,
                                               __nv_bfloat16* __restrict__ Vm) {
  __shared__ double ys[32][33];
  const int v = nv;
  const int64_t lda = (int64_t)v * na, ncdp = (int64_t)v * (v + 1) / 2;
  const int64_t ncdm = (int64_t)v * (v - 1) / 2;
  const uint32_t T = (uint32_t)(v + 31) / 32, NT = T * (T + 1) / 2;
  const uint32_t total = NT * (uint32_t)npairs;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t pr = t / NT, id = t - pr * NT;
    uint32_t tc, td;
    tri_tile(id, tc, td);
    const int c0 = (int)tc * 32, d0 = (int)td * 32;
    const int2 ab = pairs[pr];
    const int64_t ap = ab.x - a0, bp = ab.y - a0;
    const bool minus = ab.x < ab.y;
    __nv_bfloat16* op = Vp + (int64_t)pr * kp_p;
    __nv_bfloat16* om = minus ? Vm + ((int64_t)pr - ap - 1) * kp_m : Vm;
    const VT* X = V + v * ap + lda * v * bp;  // X[c,d] = X[c + lda d]
    double xr[4], yr[4];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int d = d0 + ty + 8 * jj, c = c0 + tx;
      xr[jj] = (d < v && c <= d) ? (double)X[c + lda * d] : 0.0;
      const int cm = c0 + ty + 8 * jj, dm = d0 + tx;  // X[dm, cm] for (c, d) = (cm, dm)
      yr[jj] = (cm < v && dm < v) ? (double)X[dm + lda * cm] : 0.0;
    }
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) ys[ty + 8 * jj][tx] = yr[jj];  // ys[c - c0][d - d0]
    __syncthreads();
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int d = d0 + ty + 8 * jj, c = c0 + tx;
      if (d < v && c <= d) {
        const double x = xr[jj], y = ys[tx][ty + 8 * jj];
        const int64_t k = (int64_t)d * (d + 1) / 2 + c;
        put_slices3(op, sl_p, k, c == d ? x : x + y);
        if (minus && c < d) put_slices3(om, sl_m, k - d, x - y);
      }
    }
    if (id == 0) {
      const int f = ty * 32 + tx;
      for (int64_t k = ncdp + f; k < kp_p; k += 256) put_slices3(op, sl_p, k, 0.0);
      if (minus)
        for (int64_t k = ncdm + f; k < kp_m; k += 256) put_slices3(om, sl_m, k, 0.0);
    }
    __syncthreads();
  }
}

}  // namespace

int ladder_pack_v_split(stream_t s, int nv, int a0, int na, int npairs, const int* pairs,
                        const int* cdp, const void* V, bool v_f32, void* Vp, void* Vm) {
  if (nv <= 0 || npairs <= 0 || !V || !Vp || !cdp) return (int)cudaErrorInvalidValue;
  const int64_t v = nv;
  const int npm = npairs - na;  // the block's a < b pairs
  if (npm > 0 && !Vm) return (int)cudaErrorInvalidValue;
  const int64_t kp_p = pad_k(v * (v + 1) / 2), sl_p = pad_rows(npairs) * kp_p;
  const int64_t kp_m = v > 1 ? pad_k(v * (v - 1) / 2) : 0;
  const int64_t sl_m = npm > 0 ? pad_rows(npm) * kp_m : 0;
  if (kp_m - v * (v - 1) / 2 > kp_p) return (int)cudaErrorInvalidValue;
  cudaStream_t st = (cudaStream_t)s;
  const int64_t T = (v + 31) / 32, tiles = T * (T + 1) / 2 * npairs;
  if (tiles < ((int64_t)1 << 32) - 148 * 16) {
    const unsigned g = (unsigned)std::min<int64_t>(tiles, 148 * 16);
#define ECG_PACK_TILED(VT)                                                                     \
  ladder_pack_split_tiled_kernel<VT><<<g, dim3(32, 8), 0, st>>>(                               \
      nv, a0, na, npairs, (const int2*)pairs, (const VT*)V, kp_p, sl_p, kp_m, sl_m,            \
      (__nv_bfloat16*)Vp, (__nv_bfloat16*)Vm)
    if (v_f32) ECG_PACK_TILED(float);
    else ECG_PACK_TILED(double);
#undef ECG_PACK_TILED
  } else {
    const int64_t total = kp_p * npairs;
    const unsigned g = (unsigned)std::min<int64_t>((total + 255) / 256, 148 * 16);
#define ECG_PACK_SPLIT(VT)                                                                    \
  ladder_pack_split_kernel<VT, uint64_t><<<g, 256, 0, st>>>(                                  \
      nv, a0, na, npairs, (const int2*)pairs, (const int2*)cdp, (const VT*)V, kp_p, sl_p, kp_m, \
      sl_m, (__nv_bfloat16*)Vp, (__nv_bfloat16*)Vm)
    if (v_f32) ECG_PACK_SPLIT(float);
    else ECG_PACK_SPLIT(double);
#undef ECG_PACK_SPLIT
  }
  note_launches(1);
  return (int)cudaGetLastError();
}

int tc_view(const TcOperand& parent, int64_t row0, int64_t rows, TcOperand* out) {
  if (!out || !parent.base || row0 < 0 || rows <= 0 || row0 + rows > parent.rows_p)
    return (int)cudaErrorInvalidValue;
  EncodeFn enc = nullptr;
  int e = encode_fn(&enc);
  if (e) return e;
  *out = parent;
  out->rows = rows;
  out->rows_p = pad_rows(rows);
  out->base = (__nv_bfloat16*)parent.base + row0 * parent.k_p;
  return encode_operand(enc, out, rows);
}

// Launch over pre-split operands with tile width tn and split count S.
static int tc_gemm_run(cudaStream_t st, const TcGemm& g, int ns, const TcSegs& segs, int kbt,
                       int tn, int S) {
  const int nsl = g.A[0]->slices;
  TcMaps maps;
  for (int t = 0; t < TC_MAX_SEG; ++t) {
    std::memcpy(&maps.a[t], g.A[t < ns ? t : 0]->map, sizeof(CUtensorMap));
    std::memcpy(&maps.b[t], b_map(g.B[t < ns ? t : 0], tn), sizeof(CUtensorMap));
  }
  TcOut out{g.C, g.scm, g.scn, g.dn, g.scn2, g.dm, g.scm2, g.f32 ? 1 : 0};
  const int64_t mp = pad_rows(g.m), np = (g.n + tn - 1) / tn * tn;
  if (nsl == 3)
    return tn == TN_WIDE
               ? launch_tc<3, TN_WIDE>(st, maps, segs, kbt, g.m, g.n, mp, np, g.alpha, g.beta,
                                       out, S)
               : launch_tc<3, 128>(st, maps, segs, kbt, g.m, g.n, mp, np, g.alpha, g.beta, out,
                                   S);
  if (tn == TN_XWIDE)
    return launch_tc<2, TN_XWIDE>(st, maps, segs, kbt, g.m, g.n, mp, np, g.alpha, g.beta, out,
                                  S);
  return tn == TN_WIDE
             ? launch_tc<2, TN_WIDE>(st, maps, segs, kbt, g.m, g.n, mp, np, g.alpha, g.beta, out,
                                     S)
             : launch_tc<2, 128>(st, maps, segs, kbt, g.m, g.n, mp, np, g.alpha, g.beta, out, S);
}

// Split counts a plain FP64 output allows: at least enough K slices that no
// FP32 accumulation sums more than KB_ACC k-blocks.
static int tc_min_split(int kbt) { return (kbt + KB_ACC - 1) / KB_ACC; }

int tc_gemm(stream_t s, const TcGemm& g) {
  if (g.m <= 0 || g.n <= 0) return 0;
  int64_t k[TC_MAX_SEG];
  const int ns = gemm_segments(g, k);
  if (ns == 0) return (int)cudaErrorInvalidValue;
  const int nsl = g.A[0]->slices;
  const TcSegs segs = make_segs(ns, k);
  const int kbt = segs.kb_end[TC_MAX_SEG - 1];
  const bool plain = !g.f32 && g.dn == 0 && g.dm == 0;
  // tile widths every B operand has a descriptor for
  auto usable = [&](int tn) {
    for (int t = 0; t < ns; ++t)
      if (!b_map(g.B[t], tn)) return false;
    return true;
  };
  auto split_for = [&](int tn) {
    if (!plain) return 1;
    const int64_t np = (g.n + tn - 1) / tn * tn;
    return split_count(pad_rows(g.m) / TM * (np / tn), kbt);
  };
  // the fixed rule
  int tn = tile_n(g.n, nsl);
  if (!usable(tn)) tn = 128;
  int S = split_for(tn);
  cudaStream_t st = (cudaStream_t)s;
  const std::string key = "tc " + std::to_string(g.m) + " " + std::to_string(g.n) + " " +
                          std::to_string(kbt) + " " + std::to_string(nsl) + " " +
                          std::to_string(plain ? 1 : g.f32 ? 2 : 0);
  int enc = 0;
  if (tune_get(key, &enc)) {
    const int t = enc % 4, tw = t == 1 ? TN_WIDE : t == 2 ? TN_XWIDE : 128;
    if (usable(tw)) {
      tn = tw;
      S = plain ? std::max(enc / 4, tc_min_split(kbt)) : 1;
    }
  } else if (tuning() && g.dn == 0 && g.dm == 0 && g.scm == 1 && !stream_capturing(s)) {
    struct Cand {
      int tn, S;
    };
    std::vector<Cand> cand;
    for (int tw : {128, TN_WIDE, TN_XWIDE}) {
      if ((tw == TN_XWIDE && nsl != 2) || !usable(tw) || (tw > 128 && g.n < tw)) continue;
      const int d = split_for(tw);
      for (int Sx : {d, d * 2, std::max(d / 2, 1), tc_min_split(kbt)}) {
        if (!plain && Sx != 1) continue;
        if (plain && (Sx < tc_min_split(kbt) || Sx > kbt)) continue;
        bool dup = false;
        for (auto& c : cand) dup |= (c.tn == tw && c.S == Sx);
        if (!dup) cand.push_back({tw, Sx});
      }
    }
    const int64_t esz = g.f32 ? 4 : 8;
    const TuneOut out{g.C, g.m * esz, g.n, g.scn * esz};
    const int best = tune_pick(
        s, (int)cand.size(),
        [&](int i) { return tc_gemm_run(st, g, ns, segs, kbt, cand[i].tn, cand[i].S); }, out);
    if (best >= 0) {
      tn = cand[best].tn;
      S = cand[best].S;
      tune_put(key, (tn == TN_WIDE ? 1 : tn == TN_XWIDE ? 2 : 0) + 4 * S);
    }
  }
  return tc_gemm_run(st, g, ns, segs, kbt, tn, S);
}

size_t tc_maps_bytes() { return sizeof(TcMaps); }

int tc_maps_fill(int nseg, const TcOperand* const* A, const TcOperand* const* B, int64_t n,
                 void* dst) {
  if (nseg < 1 || nseg > TC_MAX_SEG || !A || !B || !dst || n <= 0)
    return (int)cudaErrorInvalidValue;
  for (int t = 0; t < nseg; ++t)
    if (!A[t] || !B[t]) return (int)cudaErrorInvalidValue;
  const int tn = tile_n(n, A[0]->slices);
  for (int t = 0; t < nseg; ++t)
    if (!b_map(B[t], tn)) return (int)cudaErrorInvalidValue;
  TcMaps* m = reinterpret_cast<TcMaps*>(dst);
  for (int t = 0; t < TC_MAX_SEG; ++t) {
    std::memcpy(&m->a[t], A[t < nseg ? t : 0]->map, sizeof(CUtensorMap));
    std::memcpy(&m->b[t], b_map(B[t < nseg ? t : 0], tn), sizeof(CUtensorMap));
  }
  return 0;
}

namespace {
template <int NSL, int TN>
void launch_batched(cudaStream_t st, const TcOut& out, const TcGemm& g, const TcSegs& segs,
                    int kbt, int64_t c_stride, int mt, int nt, int batch, const void* mtab) {
  using Cfg = TcCfg<NSL, TN>;
  set_smem_attr<NSL, TN>();
  const int64_t items = (int64_t)mt * nt * batch;
  const unsigned grid = (unsigned)(items < 148 ? items : 148);
  TcMaps dummy;
  std::memset(&dummy, 0, sizeof(dummy));
  const int slot = ktime_begin((stream_t)st, KT_TCGEMM);
  mgemm_bf16_kernel<NSL, TN><<<grid, THREADS_TC, Cfg::SMEM_BYTES, st>>>(
      dummy, out, g.m, g.n, g.alpha, g.beta, segs, kbt, kbt, c_stride, mt, nt, batch,
      (const TcMaps*)mtab, wait_bound(st));
  ktime_end((stream_t)st, KT_TCGEMM, slot,
            2.0 * (double)g.m * (double)g.n * (double)seg_depth(segs) * Cfg::NPAIR * batch);
}
}  // namespace

int tc_gemm_batched(stream_t s, const TcGemm& g, int batch, const void* mtab, int64_t c_stride) {
  if (g.m <= 0 || g.n <= 0 || batch <= 0) return 0;
  int64_t k[TC_MAX_SEG];
  const int ns = gemm_segments(g, k);
  if (ns == 0 || !mtab || ((uintptr_t)mtab & 63) != 0) return (int)cudaErrorInvalidValue;
  // the tables were filled by tc_maps_fill with the same tile-width rule
  const int nsl = g.A[0]->slices;
  const int tn = tile_n(g.n, nsl);
  for (int t = 0; t < ns; ++t)
    if (!b_map(g.B[t], tn)) return (int)cudaErrorInvalidValue;
  const TcSegs segs = make_segs(ns, k);
  const int kbt = segs.kb_end[TC_MAX_SEG - 1];
  const int64_t mp = pad_rows(g.m), np = (g.n + tn - 1) / tn * tn;
  const int mt = (int)(mp / TM), nt = (int)(np / tn);
  TcOut out{g.C, g.scm, g.scn, g.dn, g.scn2, g.dm, g.scm2, g.f32 ? 1 : 0};
  cudaStream_t st = (cudaStream_t)s;
  if (nsl == 3) {
    if (tn == TN_WIDE)
      launch_batched<3, TN_WIDE>(st, out, g, segs, kbt, c_stride, mt, nt, batch, mtab);
    else
      launch_batched<3, 128>(st, out, g, segs, kbt, c_stride, mt, nt, batch, mtab);
  } else if (tn == TN_XWIDE) {
    launch_batched<2, TN_XWIDE>(st, out, g, segs, kbt, c_stride, mt, nt, batch, mtab);
  } else if (tn == TN_WIDE) {
    launch_batched<2, TN_WIDE>(st, out, g, segs, kbt, c_stride, mt, nt, batch, mtab);
  } else {
    launch_batched<2, 128>(st, out, g, segs, kbt, c_stride, mt, nt, batch, mtab);
  }
  note_launches(1);
  return (int)cudaGetLastError();
}

// C(m,n) = alpha sum_k A(m,k) B(k,n) + beta C(m,n) with the strided operands of
// gemm_strided (batch 1): split both operands into three slices, run the
// tensor-core kernel.
int gemm_strided_mixed(stream_t s, const Gemm& q) {
  if (q.batch != 1 || q.dn != 0 || q.kseg != 0) return (int)cudaErrorInvalidValue;
  if (q.m <= 0 || q.n <= 0) return 0;
  if (q.k <= 0 || q.alpha == 0.0) return gemm_strided(s, q);
  EncodeFn enc = nullptr;
  int e = encode_fn(&enc);
  if (e) return e;
  constexpr int NSL = 3;
  const int64_t m = q.m, n = q.n, k = q.k;
  const int64_t mp = pad_rows(m), np = pad_rows(n), kp = pad_k(k);
  __nv_bfloat16* buf = (__nv_bfloat16*)split_scratch(
      s, (size_t)NSL * (mp + np) * kp * sizeof(__nv_bfloat16));
  if (!buf) return (int)cudaErrorMemoryAllocation;
  __nv_bfloat16* As = buf;
  __nv_bfloat16* Bs = buf + (size_t)NSL * mp * kp;
  cudaStream_t st = (cudaStream_t)s;
  launch_split(st, q.A, m, k, q.sam, q.sak, mp, kp, NSL, As);  // A(m,k) = A[m sam + k sak]
  launch_split(st, q.B, n, k, q.sbn, q.sbk, np, kp, NSL, Bs);  // B(k,n) = B[k sbk + n sbn]
  // B rows are padded to 128; a wider tile reads 160-row boxes from them
  // (n >= 160 then; rows past np read as zero)
  const TcSegs segs = make_segs(1, &k);
  const int kbt = (int)(kp / TK);
  TcOut out{q.C, q.scm, q.scn, 0, 0, 0, 0, 0};
  auto run = [&](int tn, int S) {
    const int64_t npt = (n + tn - 1) / tn * tn;
    TcMaps maps;
    int r = make_map(enc, &maps.a[0], As, mp, kp, NSL);
    if (!r) r = make_map(enc, &maps.b[0], Bs, np, kp, NSL, 0, tn);
    if (r) return r;
    for (int t = 1; t < TC_MAX_SEG; ++t) {
      maps.a[t] = maps.a[0];
      maps.b[t] = maps.b[0];
    }
    if (tn == TN_WIDE)
      return launch_tc<NSL, TN_WIDE>(st, maps, segs, kbt, m, n, mp, npt, q.alpha, q.beta, out,
                                     S);
    return launch_tc<NSL, 128>(st, maps, segs, kbt, m, n, mp, npt, q.alpha, q.beta, out, S);
  };
  auto split_for = [&](int tn) {
    const int64_t npt = (n + tn - 1) / tn * tn;
    return split_count((mp / TM) * (npt / tn), kbt);
  };
  int tn = tile_n(n, NSL);
  int S = split_for(tn);
  const std::string key = "tcmix " + std::to_string(m) + " " + std::to_string(n) + " " +
                          std::to_string(kbt);
  int code = 0;
  if (tune_get(key, &code)) {
    const int tw = (code % 4) == 1 && n >= TN_WIDE ? TN_WIDE : 128;
    tn = tw;
    S = std::max(code / 4, tc_min_split(kbt));
  } else if (tuning() && q.scm == 1 && !stream_capturing(s)) {
    struct Cand {
      int tn, S;
    };
    std::vector<Cand> cand;
    for (int tw : {128, TN_WIDE}) {
      if (tw > 128 && n < tw) continue;
      const int d = split_for(tw);
      for (int Sx : {d, d * 2, std::max(d / 2, 1), tc_min_split(kbt)}) {
        if (Sx < tc_min_split(kbt) || Sx > kbt) continue;
        bool dup = false;
        for (auto& c : cand) dup |= (c.tn == tw && c.S == Sx);
        if (!dup) cand.push_back({tw, Sx});
      }
    }
    const TuneOut to{q.C, m * 8, n, q.scn * 8};
    const int best = tune_pick(
        s, (int)cand.size(), [&](int i) { return run(cand[i].tn, cand[i].S); }, to);
    if (best >= 0) {
      tn = cand[best].tn;
      S = cand[best].S;
      tune_put(key, (tn == TN_WIDE ? 1 : 0) + 4 * S);
    }
  }
  return run(tn, S);
}

int gemm_mixed(stream_t s, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
               const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
               int64_t ldc) {
  Gemm q;
  q.m = m; q.n = n; q.k = k; q.alpha = alpha; q.beta = beta;
  q.A = A; q.B = B; q.C = C;
  const bool at = (ta == 'T' || ta == 't'), bt = (tb == 'T' || tb == 't');
  q.sam = at ? lda : 1; q.sak = at ? 1 : lda;
  q.sbk = bt ? ldb : 1; q.sbn = bt ? 1 : ldb;
  q.scm = 1; q.scn = ldc;
  return gemm_strided_mixed(s, q);
}

int tc_error(int* code) {
  int h = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&h, g_tc_error, sizeof(int));
  if (e != cudaSuccess) return (int)e;
  if (h) {
    int zero = 0;
    cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int));
  }
  int d = 0, en = 0;
  if (int r = dtma_error(&d)) return r;
  if (int r = energy_error(&en)) return r;
  *code = h ? h : d ? 16 + d : (en ? 32 + en : 0);
  return 0;
}

}  // namespace dev
}  // namespace ecg
