// dev_tc.cu — split-BF16 GEMM on the sm_100a tensor cores (tcgen05 + TMA).
//
// C = alpha * op(A) op(B) + beta * C with FP64 operands and result.  Each
// operand is split into three BF16 slices x = x0 + x1 + x2 (x0 = bf16(x),
// x1 = bf16(x - x0), x2 = bf16(x - x0 - x1)) stored K-major and zero padded
// (M, N to 128, K to 64).  The six products x0y0, x0y1, x1y0, x1y1, x0y2, x2y0
// are accumulated in FP32 in tensor memory, which reproduces an FP32-accurate
// product (relative error ~2^-24 of sum |a||b|).
//
// Kernel: persistent, one CTA per SM over 128x128 output tiles.  TMA loads
// (3-D tensor maps: k, row, slice; 64x128 boxes, 128-byte swizzle) feed a
// two-stage shared-memory ring; tcgen05.mma kind::f16 (BF16 x BF16 -> F32,
// M=128 N=128 K=16) accumulates in one of two tensor-memory accumulators
// while four epilogue warps drain the other with tcgen05.ld and write FP64 C.
// Every mbarrier wait is bounded (1 s); on time-out the kernel records an
// error code, lets its own loads land (bounded), frees its tensor memory and
// returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "ecg_dev.h"

namespace ecg {
namespace dev {

namespace {

constexpr int TM = 128, TN = 128, TK = 64, STAGES = 2, SLICES = 3;
constexpr int TILE_BYTES_A = TM * TK * 2;  // 16 KiB per slice
constexpr int TILE_BYTES_B = TN * TK * 2;
constexpr int STAGE_BYTES = SLICES * (TILE_BYTES_A + TILE_BYTES_B);  // 96 KiB
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*barriers*/ + 1024 /*align*/;
constexpr unsigned long long WAIT_NS = 1000000000ull;  // 1 s bound on every mbarrier wait

__device__ int g_tc_error = 0;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes));
}

__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

// Parity wait bounded by WAIT_NS of wall time; returns false on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  const unsigned long long t0 = gtime();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity));
    if (done) return true;
    if (gtime() - t0 > WAIT_NS) return false;
  }
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

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

// Instruction descriptor: kind::f16, A/B BF16, D F32, both K-major, M=128, N=128.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                           ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(IDESC), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          smem_u32(bar)));
}

// Persistent, warp-specialised kernel: gridDim.x CTAs (one per SM) loop over
// work items (m-tile, n-tile, k-slice).  Warp 0 lane 0: TMA producer over a
// STAGES-deep shared-memory ring (full/empty mbarriers).  Warp 1: owns the
// 256-column tensor-memory allocation, lane 0 issues the MMAs into one of two
// 128-column accumulators and commits.  Warps 2..5: epilogue, each reading
// the 32 accumulator lanes its warp index (mod 4) may access, writing FP64 C
// and releasing the accumulator, so the epilogue of one tile overlaps the
// MMAs of the next.
constexpr int EPI_WARPS = 4;
constexpr int THREADS_TC = 32 * (2 + EPI_WARPS);
constexpr uint32_t TMEM_COLS_P = 2 * TN;

__global__ void __launch_bounds__(THREADS_TC, 1)
    mgemm_bf16x3_kernel(const __grid_constant__ CUtensorMap tmA,
                        const __grid_constant__ CUtensorMap tmB, double* __restrict__ C,
                        int64_t M, int64_t N, int64_t scm, int64_t scn, double alpha, double beta,
                        int kb_per_split, int kblocks_total, int64_t split_stride, int mtiles,
                        int ntiles, int nsplit) {
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
                 "r"(TMEM_COLS_P));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;

  auto item_coords = [&](int64_t it, int& mt, int& nt, int& z) {
    mt = (int)(it % mtiles);
    nt = (int)((it / mtiles) % ntiles);
    z = (int)(it / ((int64_t)mtiles * ntiles));
  };
  auto item_kblocks = [&](int z) { return min(kb_per_split, kblocks_total - z * kb_per_split); };

  if (warp == 0) {
    if (lane == 0) {
      int64_t g = 0;  // global k-block counter of this CTA
      for (int64_t it = blockIdx.x; it < items && !*(volatile int*)abort_flag; it += gridDim.x) {
        int mt, nt, z;
        item_coords(it, mt, nt, z);
        const int nk = item_kblocks(z), kb0 = z * kb_per_split;
        for (int kb = 0; kb < nk; ++kb, ++g) {
          const int s = (int)(g % STAGES);
          const int64_t u = g / STAGES;
          if (u > 0 && !mbar_wait(&empty[s], (uint32_t)((u - 1) & 1))) {
            atomicExch(&g_tc_error, 1);
            atomicExch(abort_flag, 1);
            break;
          }
          uint8_t* st = tiles + s * STAGE_BYTES;
          mbar_expect_tx(&full[s], STAGE_BYTES);
          for (int t = 0; t < SLICES; ++t) {
            tma_load_3d(st + t * TILE_BYTES_A, &tmA, &full[s], (kb0 + kb) * TK, mt * TM, t);
            tma_load_3d(st + SLICES * TILE_BYTES_A + t * TILE_BYTES_B, &tmB, &full[s],
                        (kb0 + kb) * TK, nt * TN, t);
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
        const int nk = item_kblocks(z);
        const int acc = (int)(lt & 1);
        const int64_t ua = lt >> 1;
        if (ua > 0 && !mbar_wait(&tempty[acc], (uint32_t)((ua - 1) & 1))) {
          atomicExch(&g_tc_error, 4);
          atomicExch(abort_flag, 1);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        const uint32_t dcol = tmem + (uint32_t)(acc * TN);
        bool ok = true;
        for (int kb = 0; kb < nk; ++kb, ++g) {
          const int s = (int)(g % STAGES);
          if (!mbar_wait(&full[s], (uint32_t)((g / STAGES) & 1))) {
            atomicExch(&g_tc_error, 2);
            atomicExch(abort_flag, 1);
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
          const uint8_t* st = tiles + s * STAGE_BYTES;
          const uint8_t* As = st;
          const uint8_t* Bs = st + SLICES * TILE_BYTES_A;
          // slice pairs (a, b): hi*hi, hi*mid, mid*hi, mid*mid, hi*lo, lo*hi
          const int pa[6] = {0, 0, 1, 1, 0, 2}, pb[6] = {0, 1, 0, 1, 2, 0};
#pragma unroll
          for (int p = 0; p < 6; ++p) {
            const uint64_t da = umma_desc(As + pa[p] * TILE_BYTES_A);
            const uint64_t db = umma_desc(Bs + pb[p] * TILE_BYTES_B);
#pragma unroll
            for (int kk = 0; kk < TK / 16; ++kk)
              umma(dcol, da + (uint64_t)(kk * 2), db + (uint64_t)(kk * 2),
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
    // epilogue warps 2..5: TMEM lane quarter q = warp % 4
    const int q = warp & 3;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    int64_t lt = 0;
    for (int64_t it = blockIdx.x; it < items; it += gridDim.x, ++lt) {
      int mt, nt, z;
      item_coords(it, mt, nt, z);
      const int acc = (int)(lt & 1);
      if (!mbar_wait(&tfull[acc], (uint32_t)((lt >> 1) & 1))) {
        atomicExch(&g_tc_error, 3);
        atomicExch(abort_flag, 1);
        break;
      }
      if (*(volatile int*)abort_flag) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      double* Cz = C + (int64_t)z * split_stride;
      const int64_t row = (int64_t)mt * TM + q * 32 + lane;
#pragma unroll 1
      for (int c = 0; c < TN; c += 32) {
        uint32_t r[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
            "%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
              "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
              "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
              "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
              "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
              "=r"(r[31])
            : "r"(tmem + lane_base + (uint32_t)(acc * TN + c)));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::);
        if (row < M) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int64_t col = (int64_t)nt * TN + c + j;
            if (col < N) {
              double* cp = Cz + row * scm + col * scn;
              double v = alpha * (double)__uint_as_float(r[j]);
              if (beta != 0.0) v += beta * *cp;
              *cp = v;
            }
          }
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
                 "r"(TMEM_COLS_P));
  }
}

// X(r,k) = src[r*sr + k*sk] (FP64, R x K) -> dst[s][r][k] BF16, zero padded to
// Rp x Kp.  32x32 tiles through shared memory so that reads are coalesced
// whichever of sr / sk is the unit stride.
__global__ void split3_kernel(const double* __restrict__ src, int64_t R, int64_t K, int64_t sr,
                              int64_t sk, int64_t Rp, int64_t Kp, __nv_bfloat16* __restrict__ dst) {
  __shared__ double tile[32][33];
  const int64_t tk = (Kp + 31) / 32, tr = (Rp + 31) / 32, ntile = tk * tr;
  const bool rfast = (sr == 1);
  for (int64_t t = blockIdx.x; t < ntile; t += gridDim.x) {
    const int64_t r0 = (t / tk) * 32, k0 = (t % tk) * 32;
    for (int j = threadIdx.y; j < 32; j += 8) {
      int64_t r, k;
      if (rfast) { r = r0 + threadIdx.x; k = k0 + j; } else { r = r0 + j; k = k0 + threadIdx.x; }
      double x = (r < R && k < K) ? src[r * sr + k * sk] : 0.0;
      if (rfast) tile[j][threadIdx.x] = x;   // tile[k][r]
      else tile[threadIdx.x][j] = x;         // tile[k][r]
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
        const __nv_bfloat16 h2 = __double2bfloat16(e2);
        const int64_t o = r * Kp + k, sl = Rp * Kp;
        dst[o] = h0;
        dst[o + sl] = h1;
        dst[o + 2 * sl] = h2;
      }
    }
    __syncthreads();
  }
}

// Driver entry point for tensor-map encoding (no libcuda link needed).
typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                             const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                             const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                             CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeFn g_encode = nullptr;
std::mutex g_tc_mu;
__nv_bfloat16* g_split = nullptr;
size_t g_split_len = 0;

int encode_fn(EncodeFn* out) {
  std::lock_guard<std::mutex> lk(g_tc_mu);
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

__nv_bfloat16* split_buffer(size_t n) {
  std::lock_guard<std::mutex> lk(g_tc_mu);
  if (n > g_split_len) {
    if (g_split) cudaFree(g_split);
    g_split = nullptr;
    g_split_len = 0;
    size_t want = n + n / 4;
    if (cudaMalloc(&g_split, want * sizeof(__nv_bfloat16)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    g_split_len = want;
  }
  return g_split;
}

int make_map(EncodeFn enc, CUtensorMap* m, __nv_bfloat16* base, int64_t rows_p, int64_t k_p) {
  cuuint64_t dims[3] = {(cuuint64_t)k_p, (cuuint64_t)rows_p, (cuuint64_t)SLICES};
  cuuint64_t strides[2] = {(cuuint64_t)(k_p * 2), (cuuint64_t)(rows_p * k_p * 2)};
  cuuint32_t box[3] = {(cuuint32_t)TK, (cuuint32_t)TM, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, (void*)base, dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : (int)cudaErrorInvalidValue;
}

}  // namespace

// C(m,n) = alpha sum_k A(m,k) B(k,n) + beta C(m,n) with the strided operands of
// gemm_strided (batch 1): split both operands, run the tensor-core kernel.
int gemm_strided_mixed(stream_t s, const Gemm& q) {
  if (q.batch != 1) return (int)cudaErrorInvalidValue;
  if (q.m <= 0 || q.n <= 0) return 0;
  if (q.k <= 0 || q.alpha == 0.0) return gemm_strided(s, q);
  EncodeFn enc = nullptr;
  int e = encode_fn(&enc);
  if (e) return e;
  static_assert(TM == TN, "one padding rule for A and B");
  const int64_t m = q.m, n = q.n, k = q.k;
  const int64_t mp = (m + TM - 1) / TM * TM, np = (n + TN - 1) / TN * TN;
  const int64_t kp = (k + TK - 1) / TK * TK;
  __nv_bfloat16* buf = split_buffer((size_t)SLICES * (mp + np) * kp);
  if (!buf) return (int)cudaErrorMemoryAllocation;
  __nv_bfloat16* As = buf;
  __nv_bfloat16* Bs = buf + (size_t)SLICES * mp * kp;
  cudaStream_t st = (cudaStream_t)s;
  auto launch_split = [&](const double* src, int64_t R, int64_t sr, int64_t sk, int64_t Rp,
                          __nv_bfloat16* dst) {
    int64_t tiles = ((Rp + 31) / 32) * ((kp + 31) / 32);
    unsigned g = (unsigned)(tiles < 148 * 16 ? tiles : 148 * 16);
    split3_kernel<<<g, dim3(32, 8), 0, st>>>(src, R, k, sr, sk, Rp, kp, dst);
  };
  launch_split(q.A, m, q.sam, q.sak, mp, As);  // A(m,k) = A[m sam + k sak]
  launch_split(q.B, n, q.sbn, q.sbk, np, Bs);  // B(k,n) = B[k sbk + n sbn]
  CUtensorMap mA, mB;
  if ((e = make_map(enc, &mA, As, mp, kp))) return e;
  if ((e = make_map(enc, &mB, Bs, np, kp))) return e;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(mgemm_bf16x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         SMEM_BYTES);
    attr = true;
  }
  const int kbt = (int)(kp / TK);
  const int64_t tiles = (mp / TM) * (np / TN);
  // split K when the output has fewer tiles than SMs (at least 4 k-blocks per slice)
  int S = 1;
  if (tiles < 148 && kbt >= 8) S = (int)std::min<int64_t>((148 + tiles - 1) / tiles, kbt / 4);
  const int kps = (kbt + S - 1) / S;
  S = (kbt + kps - 1) / kps;
  const int mt = (int)(mp / TM), nt = (int)(np / TN);
  const int64_t items = (int64_t)mt * nt * S;
  const unsigned grid = (unsigned)(items < 148 ? items : 148);
  if (S == 1) {
    mgemm_bf16x3_kernel<<<grid, THREADS_TC, SMEM_BYTES, st>>>(mA, mB, q.C, m, n, q.scm, q.scn,
                                                              q.alpha, q.beta, kps, kbt, 0, mt,
                                                              nt, 1);
    return (int)cudaGetLastError();
  }
  double* P = splitk_buffer((size_t)S * m * n);
  if (!P) return (int)cudaErrorMemoryAllocation;
  mgemm_bf16x3_kernel<<<grid, THREADS_TC, SMEM_BYTES, st>>>(mA, mB, P, m, n, 1, m, 1.0, 0.0, kps,
                                                            kbt, m * n, mt, nt, S);
  e = (int)cudaGetLastError();
  if (e) return e;
  return splitk_reduce(s, m, n, S, P, q.alpha, q.beta, q.C, q.scm, q.scn);
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
  *code = h;
  if (h) {
    int zero = 0;
    cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int));
  }
  return 0;
}

}  // namespace dev
}  // namespace ecg
