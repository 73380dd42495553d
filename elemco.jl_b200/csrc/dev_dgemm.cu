// dev_dgemm.cu — FP64 GEMM with TMA-staged operands (sm_100a).
//
// C(m,n) = alpha * A(m,k) B(k,n) + beta * C with C addressed through a row
// stride and a column map (plain column stride, or a split column index as the
// (T) K builds use), batched (3-D tensor maps, one batch item per grid z) or split over
// K (grid z = K slice, partial products into the stream's split-K buffer,
// summed in a fixed order by splitk_reduce).  tcgen05 has no FP64 kind, so the
// products run on the FP64 MMA pipe (mma.sync m8n8k4 f64).  What the Tensor
// Memory Accelerator takes over is the operand staging: one thread issues the
// TMA copies of a 16-deep k-slab of the A and B tiles into a ring of STAGES
// shared-memory stages (128-byte swizzle, mbarrier completion), so the MMA
// warps spend no instructions on address arithmetic or copies, and each warp
// releases a stage through an `empty` mbarrier instead of a block barrier.
//
// Shared layouts (doubles; rows of 128 bytes whose 16-byte chunks are XOR-
// swizzled with the row index mod 8, as TMA's 128-byte swizzle writes them):
//  * operand contiguous along k ("k-fast"): [row][k 0..15], one box per stage
//  * operand contiguous along its row index ("i-fast"): [row/16][k 0..15]
//    [row%16], one 16 x 16 box per 16 rows
// An MMA may take its 8 rows (columns) and its 4 k in any order, provided the
// epilogue writes each accumulator to the row and column it stands for.  The
// orders below make every half-warp's fragment reads hit 16 distinct 8-byte
// bank pairs under the swizzle (lane group g = lane/4, t = lane%4, k = kb + t):
//  * k-fast: row 2(g%4) + g/4 of an 8-row block
//  * i-fast: MMA s in {0,1} of a 16-row block reads row
//            (g&1) + 8((g>>1)&1) + 2(g>>2) + 4s
//
// Every mbarrier wait is bounded (the stream's tensor-core bound, default
// 1 s): on time-out the kernel records an error code (read by dtma_error),
// waits (bounded) for its own copies in flight and returns without writing C.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>

#include "ecg_dev.h"
#include "tma_util.cuh"

namespace ecg {
namespace dev {

namespace {

using namespace tma;

constexpr int DK = 16;  // k depth of a stage: 16 doubles, one 128-byte swizzle row

__device__ int g_dtma_error = 0;

template <int BM, int BN, int WM, int WN, int STAGES>
struct DCfg {
  static constexpr int WARPS_M = BM / WM;
  static constexpr int WARPS = (BM / WM) * (BN / WN);
  static constexpr int THREADS = WARPS * 32;
  static constexpr int A_BYTES = BM * DK * 8;
  static constexpr int B_BYTES = BN * DK * 8;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int SMEM = STAGES * STAGE_BYTES + 1024 /*align*/ + 2 * STAGES * 8;
  static_assert(BM % WM == 0 && BN % WN == 0 && WM % 16 == 0 && WN % 16 == 0, "tile shape");
  static_assert(A_BYTES % 1024 == 0 && B_BYTES % 1024 == 0, "swizzled tiles start on 1024 bytes");
  static_assert(SMEM <= 227 * 1024, "shared memory");
};

struct DOut {
  // element (i, j) of grid-z item z at C + z*scb + i*scm + colmap(j), colmap(j)
  // = (j % dn)*scn + (j / dn)*scn2 (dn = 0: j*scn)
  double* C;
  int64_t m, n, scn, scb;
  double alpha, beta;
  int64_t scm = 1, dn = 0, scn2 = 0;
};

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

// Row (within a 16-row block) that lane group g reads in MMA s of an i-fast
// operand.
__device__ __forceinline__ int jmap(int g, int s) {
  return (g & 1) + 8 * ((g >> 1) & 1) + 2 * (g >> 2) + 4 * s;
}
// Row (within an 8-row block) that lane group g reads of a k-fast operand.
__device__ __forceinline__ int pmap(int g) { return 2 * (g & 3) + (g >> 2); }

// Per-lane fragment offsets (doubles, within one stage's tile) of an operand
// whose warp sub-tile starts at row w0 and has NB 8-row blocks.  k-fast:
// o[q] for k-step kb = 4q, block rb at o[q] + 128 rb.  i-fast: o[2 rb + (q & 1)]
// + 64 q.
template <bool KF, int NB>
struct FragOff {
  static constexpr int N = KF ? 4 : 2 * NB;
  uint32_t o[N];
  __device__ __forceinline__ FragOff(int w0, int g, int t) {
    if constexpr (KF) {
      const int p = pmap(g);
      const uint32_t rowbase = (uint32_t)((w0 + p) * 16 + (t & 1));
      const int y = (t >> 1) ^ p;
#pragma unroll
      for (int q = 0; q < 4; ++q) o[q] = rowbase + (uint32_t)((4 * q) ^ (y << 1));
    } else {
#pragma unroll
      for (int rb = 0; rb < NB; ++rb) {
        const int j = jmap(g, rb & 1);
        const uint32_t base = (uint32_t)(((w0 >> 4) + (rb >> 1)) * 256 + t * 16 + (j & 1) +
                                         (((j >> 1) ^ t) << 1));
        o[2 * rb] = base;
        o[2 * rb + 1] = base ^ 8u;
      }
    }
  }
  __device__ __forceinline__ uint32_t at(int rb, int q) const {
    if constexpr (KF)
      return o[q] + 128u * rb;
    else
      return o[2 * rb + (q & 1)] + 64u * q;
  }
};

// Row (or column) of the tile that accumulator row g of block rb stands for.
template <bool KF>
__device__ __forceinline__ int frag_row(int w0, int rb, int g) {
  if constexpr (KF)
    return w0 + 8 * rb + pmap(g);
  else
    return w0 + 16 * (rb >> 1) + jmap(g, rb & 1);
}

// RMW2: read-modify-write epilogue that loads a group of C values before
// storing any (the (T) K builds, whose beta = 1 GEMMs spend most of their
// epilogue waiting on those loads); the CCSD GEMMs run faster with the
// one-by-one epilogue, so it is a separate instantiation.
template <int BM, int BN, int WM, int WN, int STAGES, int MINB, bool AKF, bool BKF, bool RMW2>
__global__ void __launch_bounds__(DCfg<BM, BN, WM, WN, STAGES>::THREADS, MINB)
    dgemm_tma_kernel(const __grid_constant__ CUtensorMap ma, const __grid_constant__ CUtensorMap mb,
                     DOut out, int64_t k, int64_t kslice, int split,
                     unsigned long long wait_ns) {
  using Cfg = DCfg<BM, BN, WM, WN, STAGES>;
  constexpr int MT = WM / 8, NTL = WN / 8;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = (uint64_t*)(smem + STAGES * Cfg::STAGE_BYTES);
  uint64_t* empty = full + STAGES;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int z = blockIdx.z;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int64_t kbeg = split ? (int64_t)z * kslice : 0;
  const int64_t kend = split ? (kbeg + kslice < k ? kbeg + kslice : k) : k;
  const int KT = kend > kbeg ? (int)((kend - kbeg + DK - 1) / DK) : 0;
  const int bz = split ? 0 : z;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], Cfg::WARPS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    asm volatile("fence.proxy.async.shared::cta;\n" ::);
  }
  __syncthreads();

  auto issue = [&](int t) {
    const int s = t % STAGES;
    uint8_t* a = smem + s * Cfg::STAGE_BYTES;
    uint8_t* b = a + Cfg::A_BYTES;
    const int kk = (int)(kbeg + (int64_t)t * DK);
    mbar_expect_tx(&full[s], Cfg::STAGE_BYTES);
    if constexpr (AKF) {
      tma_load_3d(a, &ma, &full[s], kk, m0, bz);
    } else {
#pragma unroll
      for (int q = 0; q < BM / 16; ++q) tma_load_3d(a + q * 2048, &ma, &full[s], m0 + 16 * q, kk, bz);
    }
    if constexpr (BKF) {
      tma_load_3d(b, &mb, &full[s], kk, n0, bz);
    } else {
#pragma unroll
      for (int q = 0; q < BN / 16; ++q) tma_load_3d(b + q * 2048, &mb, &full[s], n0 + 16 * q, kk, bz);
    }
  };

  int issued = 0;
  if (tid == 0) {
    asm volatile("prefetch.tensormap [%0];\n" ::"l"((uint64_t)&ma) : "memory");
    asm volatile("prefetch.tensormap [%0];\n" ::"l"((uint64_t)&mb) : "memory");
    for (; issued < KT && issued < STAGES; ++issued) issue(issued);
  }

  const int g = lane >> 2, t4 = lane & 3;
  const int wm0 = (warp % Cfg::WARPS_M) * WM, wn0 = (warp / Cfg::WARPS_M) * WN;
  const FragOff<AKF, MT> fa(wm0, g, t4);
  const FragOff<BKF, NTL> fb(wn0, g, t4);

  double acc[MT][NTL][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NTL; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  bool ok = true;
  int consumed = 0;
  for (int t = 0; t < KT; ++t) {
    const int s = t % STAGES;
    const bool ready = mbar_wait(&full[s], (uint32_t)((t / STAGES) & 1), wait_ns);
    if (!__all_sync(~0u, ready)) {
      ok = false;
      break;
    }
    consumed = t + 1;
    const double* As = (const double*)(smem + s * Cfg::STAGE_BYTES);
    const double* Bs = (const double*)(smem + s * Cfg::STAGE_BYTES + Cfg::A_BYTES);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double af[MT], bf[NTL];
#pragma unroll
      for (int i = 0; i < MT; ++i) af[i] = As[fa.at(i, q)];
#pragma unroll
      for (int j = 0; j < NTL; ++j) bf[j] = Bs[fb.at(j, q)];
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NTL; ++j) dmma884(acc[i][j], af[i], bf[j]);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    // thread 0 refills the stage that tile t-1 used once every warp has
    // released it (one tile of slack, so the wait rarely blocks)
    bool refill_ok = true;
    if (tid == 0 && t >= 1 && issued < KT) {
      const int tp = t - 1;
      if (mbar_wait(&empty[tp % STAGES], (uint32_t)((tp / STAGES) & 1), wait_ns))
        issue(issued++);
      else
        refill_ok = false;
    }
    if (!__all_sync(~0u, refill_ok)) {
      ok = false;
      break;
    }
  }
  if (!ok) {
    if (lane == 0) atomicExch(&g_dtma_error, 1);
    // nothing of this CTA's may be in flight when it exits: thread 0 waits
    // (bounded) for the tiles it issued that no wait has seen complete
    if (tid == 0)
      for (int t = consumed; t < issued; ++t)
        mbar_wait(&full[t % STAGES], (uint32_t)((t / STAGES) & 1), WAIT_NS);
    return;
  }

  double* C = out.C + (int64_t)z * out.scb;
  int64_t coff[NTL][2];
#pragma unroll
  for (int j = 0; j < NTL; ++j)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t col = n0 + frag_row<BKF>(wn0, j, 2 * t4 + h);
      coff[j][h] = col >= out.n ? -1
                   : out.dn > 0 ? (col % out.dn) * out.scn + (col / out.dn) * out.scn2
                                : col * out.scn;
    }
  if (!RMW2 || out.beta == 0.0) {
#pragma unroll
    for (int i = 0; i < MT; ++i) {
      const int64_t row = m0 + frag_row<AKF>(wm0, i, g);
      if (row >= out.m) continue;
      double* Cr = C + row * out.scm;
#pragma unroll
      for (int j = 0; j < NTL; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          if (coff[j][h] >= 0) {
            double* cp = Cr + coff[j][h];
            double v = out.alpha * acc[i][j][h];
            if (out.beta != 0.0) v += out.beta * *cp;
            *cp = v;
          }
        }
    }
    return;
  }
  // read-modify-write: ER rows of fragments at a time (16 C values a lane)
  // are all loaded before any store, so the loads overlap instead of waiting
  // one by one behind stores the compiler cannot prove disjoint
  constexpr int ER = NTL > 4 ? 1 : 2;
#pragma unroll
  for (int i0 = 0; i0 < MT; i0 += ER) {
    double cv[ER][NTL][2];
#pragma unroll
    for (int ii = 0; ii < ER; ++ii) {
      const int64_t row = m0 + frag_row<AKF>(wm0, i0 + ii, g);
      const double* Cr = C + row * out.scm;
#pragma unroll
      for (int j = 0; j < NTL; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h)
          cv[ii][j][h] = (row < out.m && coff[j][h] >= 0) ? Cr[coff[j][h]] : 0.0;
    }
#pragma unroll
    for (int ii = 0; ii < ER; ++ii) {
      const int64_t row = m0 + frag_row<AKF>(wm0, i0 + ii, g);
      if (row >= out.m) continue;
      double* Cr = C + row * out.scm;
#pragma unroll
      for (int j = 0; j < NTL; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h)
          if (coff[j][h] >= 0)
            Cr[coff[j][h]] = out.alpha * acc[i0 + ii][j][h] + out.beta * cv[ii][j][h];
    }
  }
}

// 3-D map over a double operand: inner extent d0 (unit stride), d1 rows
// s1 doubles apart, d2 batch items s2 doubles apart; box (16, b1, 1),
// 128-byte swizzle, out-of-range elements read as zero.
int dmap(CUtensorMap* m, const double* base, int64_t d0, int64_t d1, int64_t s1, int64_t d2,
         int64_t s2, int b1) {
  EncodeFn enc = nullptr;
  if (int e = encode_fn(&enc)) return e;
  cuuint64_t dims[3] = {(cuuint64_t)d0, (cuuint64_t)d1, (cuuint64_t)d2};
  cuuint64_t strides[2] = {(cuuint64_t)(s1 * 8), (cuuint64_t)(s2 * 8)};
  cuuint32_t box[3] = {(cuuint32_t)DK, (cuuint32_t)b1, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(base), dims,
                   strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : (int)cudaErrorInvalidValue;
}

// a stride (doubles) TMA accepts: a positive multiple of 16 bytes below 2^40 bytes
bool stride_ok(int64_t s) { return s > 0 && s % 2 == 0 && s < ((int64_t)1 << 37); }

// The map of operand X(i, k) = X[i*si + k*sk + z*sz] (i < ni, k < nk, z <
// nz): k-fast when sk == 1 (box 16 k x rows), else i-fast (si == 1; box
// 16 i x 16 k).  Returns false when TMA cannot address it.
bool operand_map(CUtensorMap* m, bool* kfast, const double* X, int64_t ni, int64_t nk,
                 int64_t si, int64_t sk, int64_t nz, int64_t sz, int rows) {
  if (((uintptr_t)X & 15) != 0) return false;
  if (nz > 1 && !stride_ok(sz)) return false;
  // a single item's map still needs a valid third stride: the item's extent
  auto zs = [&](int64_t s1, int64_t d1) { return nz > 1 ? sz : (s1 * d1 + 1) / 2 * 2; };
  if (sk == 1 && (nk > 1 || si != 1)) {
    const int64_t s1 = ni > 1 ? si : (nk + 1) / 2 * 2;
    if (!stride_ok(s1)) return false;
    *kfast = true;
    return dmap(m, X, nk, ni, s1, nz, zs(s1, ni), rows) == 0;
  }
  if (si == 1) {
    const int64_t s1 = nk > 1 ? sk : (ni + 1) / 2 * 2;
    if (!stride_ok(s1)) return false;
    *kfast = false;
    return dmap(m, X, ni, nk, s1, nz, zs(s1, nk), 16) == 0;
  }
  return false;
}

template <int BM, int BN, int WM, int WN, int STAGES, int MINB, bool AKF, bool BKF,
          bool RMW2 = false>
int launch_dtma(cudaStream_t st, const CUtensorMap& ma, const CUtensorMap& mb, const DOut& out,
                int64_t k, int64_t kslice, int nz, int split) {
  using Cfg = DCfg<BM, BN, WM, WN, STAGES>;
  auto kern = dgemm_tma_kernel<BM, BN, WM, WN, STAGES, MINB, AKF, BKF, RMW2>;
  // cudaFuncSetAttribute acts on the current device only: one flag per device
  static std::atomic<bool> done[128] = {};
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) {
    cudaGetLastError();
    d = -1;
  }
  if (d < 0 || d >= 128 || !done[d].load(std::memory_order_acquire)) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM) ==
        cudaSuccess) {
      if (d >= 0 && d < 128) done[d].store(true, std::memory_order_release);
    } else {
      cudaGetLastError();
    }
  }
  const int64_t gx = (out.m + BM - 1) / BM, gy = (out.n + BN - 1) / BN;
  if (gy > 65535 || nz > 65535) return (int)cudaErrorInvalidConfiguration;
  dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)nz);
  unsigned long long w = tc_wait((stream_t)st);
  kern<<<grid, Cfg::THREADS, Cfg::SMEM, st>>>(ma, mb, out, k, kslice, split,
                                              w ? w : WAIT_NS);
  note_launches(1);
  return (int)cudaGetLastError();
}

typedef int (*DtmaLaunch)(cudaStream_t, const CUtensorMap&, const CUtensorMap&, const DOut&,
                          int64_t, int64_t, int, int);

// Tile configurations: 0: 64x64 (4 warps of 32x32, 4 stages, 3 CTAs/SM);
// 1: 128x64 (4 warps of 64x32, 4 stages, 2 CTAs/SM); 2: 64x128 (4 warps of
// 32x64, 4 stages, 2 CTAs/SM); 3: 128x128 (8 warps of 64x32, 4 stages).
template <bool AKF, bool BKF>
DtmaLaunch pick(int cfg) {
  switch (cfg) {
    case 1: return launch_dtma<128, 64, 64, 32, 4, 2, AKF, BKF>;
    case 2: return launch_dtma<64, 128, 32, 64, 4, 2, AKF, BKF>;
    case 3: return launch_dtma<128, 128, 64, 32, 4, 1, AKF, BKF>;
    default: return launch_dtma<64, 64, 32, 32, 4, 3, AKF, BKF>;
  }
}
// The (T) K builds' configuration: 64x64 with the grouped read-modify-write.
template <bool AKF, bool BKF>
DtmaLaunch pick_rmw() {
  return launch_dtma<64, 64, 32, 32, 4, 3, AKF, BKF, true>;
}
constexpr int CFG_BM[DTMA_CONFIGS] = {64, 128, 64, 128};
constexpr int CFG_BN[DTMA_CONFIGS] = {64, 64, 128, 128};

}  // namespace

bool dgemm_tma_usable(const Gemm& q) {
  return q.scm == 1 && q.dn == 0 && dgemm_tma_usable_mapped(q);
}

bool dgemm_tma_usable_mapped(const Gemm& q) {
  if (q.kseg || q.ptab || q.m <= 0 || q.n <= 0 || q.k <= 0 || q.dn < 0) return false;
  if (q.m >= ((int64_t)1 << 31) || q.n >= ((int64_t)1 << 31) || q.k >= ((int64_t)1 << 31))
    return false;
  CUtensorMap m;
  bool kf;
  return operand_map(&m, &kf, q.A, q.m, q.k, q.sam, q.sak, q.batch, q.sab, 64) &&
         operand_map(&m, &kf, q.B, q.n, q.k, q.sbn, q.sbk, q.batch, q.sbb, 64);
}

int dgemm_tma(stream_t s, const Gemm& q, int cfg, int nsplit) {
  if (cfg < 0 || cfg >= DTMA_CONFIGS) return (int)cudaErrorInvalidValue;
  cudaStream_t st = (cudaStream_t)s;
  // the split-K reduction writes C through plain strides only
  if (nsplit > 1 && (q.batch != 1 || q.dn > 0)) return (int)cudaErrorInvalidValue;
  CUtensorMap ma, mb;
  bool akf = false, bkf = false;
  if (!operand_map(&ma, &akf, q.A, q.m, q.k, q.sam, q.sak, q.batch, q.sab, CFG_BM[cfg]) ||
      !operand_map(&mb, &bkf, q.B, q.n, q.k, q.sbn, q.sbk, q.batch, q.sbb, CFG_BN[cfg]))
    return -1;
  DtmaLaunch f = akf ? (bkf ? pick<true, true>(cfg) : pick<true, false>(cfg))
                     : (bkf ? pick<false, true>(cfg) : pick<false, false>(cfg));
  if (q.mapped_tma && cfg == 0)
    f = akf ? (bkf ? pick_rmw<true, true>() : pick_rmw<true, false>())
            : (bkf ? pick_rmw<false, true>() : pick_rmw<false, false>());
  if (nsplit <= 1) {
    DOut o{q.C, q.m, q.n, q.scn, q.scb, q.alpha, q.beta, q.scm, q.dn, q.scn2};
    return f(st, ma, mb, o, q.k, q.k, (int)q.batch, 0);
  }
  int64_t kc = (q.k + nsplit - 1) / nsplit;
  kc = (kc + DK - 1) / DK * DK;
  const int64_t S = (q.k + kc - 1) / kc;
  double* P = splitk_buffer(s, (size_t)S * q.m * q.n);
  if (!P) return (int)cudaErrorMemoryAllocation;
  DOut o{P, q.m, q.n, q.m, q.m * q.n, 1.0, 0.0};
  if (int e = f(st, ma, mb, o, q.k, kc, (int)S, 1)) return e;
  return splitk_reduce(s, q.m, q.n, (int)S, P, q.alpha, q.beta, q.C, q.scm, q.scn);
}

int dtma_error(int* code) {
  int h = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&h, g_dtma_error, sizeof(int));
  if (e != cudaSuccess) return (int)e;
  *code = h;
  if (h) {
    int zero = 0;
    cudaMemcpyToSymbol(g_dtma_error, &zero, sizeof(int));
  }
  return 0;
}

}  // namespace dev
}  // namespace ecg
