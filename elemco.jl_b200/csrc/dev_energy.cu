// dev_energy.cu — the fused X / (T) energy kernel for FP32 K (mixed precision).
//
// For a batch of occupied triplets, each with its K[a,b,c] (v^3, FP32, a
// fastest), forms X_abc = (4 K_abc + K_bca + K_cab - 2 K_acb - 2 K_cba
// - 2 K_bac) / D_abc and the two sums of cc_triples.jl:113-156:
//   sum_abc K'_abc X_abc   (K' = K, or the K built from covariant U2 for Lambda)
//   sum_abc X_abc Y_abc,   Y_abc = g_i[a] M_jk[b,c] + g_j[b] M_ik[a,c]
//                                + g_k[c] M_ij[a,b] + (f, N likewise)
// The six orderings of an element share their K values, so the work is cut
// into orbits: cube triples A <= B <= C of 8^3 cubes, whose six permuted cubes
// hold every ordering of every element of cube (A, B, C) once; ties (A = B or
// B = C) visit elements 2 or 6 times and are weighted 1/2, 1/6.
//
// One warp owns an orbit, with no block barrier (the warps of a block run
// independent orbits).  One lane stages the orbit with the Tensor Memory
// Accelerator: the six K cubes (and K') as 8^3 boxes of a 4-D tensor map over
// the batch's K slots, and the 8x8 blocks of (M, N) of the six ordered
// position pairs as boxes of interleaved FP32 copies (a transposed copy
// serves the pairs whose block is read transposed); all complete on the
// warp's mbarrier, and out-of-range elements read as zero.  The (g, f)
// vectors and orbital energies come with cp.async and plain loads.  Staging
// with TMA keeps the orbit's 21 KB off the SM's load pipeline: per-lane
// cp.async copies had left the kernel waiting on its own loads.
//
// Evaluation: 16 elements per lane.  Lane bits hold l0 and l1 (two bits
// each) and l2 (one bit); the loops run over the upper bits, so the (M, N)
// values of the (l0, l1) position pairs, the l0 and l1 vectors and the
// denominator parts stay in registers.  Cubes are dense [z][y][x] (TMA boxes
// have no padding); for this lane assignment, the one with the fewest bank
// conflicts on dense cubes in a search over all, the six orderings' reads
// take 3.3 wavefronts on average.  Per-element arithmetic is FP32 (K is FP32
// here); each lane's orbit sums are added in FP64, and the blocks' partial
// sums are reduced in a fixed order.
//
// Every mbarrier wait is bounded (the stream's tensor-core bound, default
// 1 s); on time-out the warp records an error code (read by energy_error),
// waits (bounded) for its own copies and stops.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "ecg_dev.h"
#include "tma_util.cuh"
#include "triples_perm.h"

namespace ecg {
namespace dev {

namespace {

using namespace tma;

constexpr int EC_CUBE = 512;  // floats per staged cube, [z][y][x]

__device__ int g_energy_error = 0;

template <bool HAS_U>
struct EnergyWarpSmem {
  static constexpr int CUBES_BYTES = 6 * EC_CUBE * 4;
  static constexpr int U_OFF = CUBES_BYTES;
  static constexpr int MN_OFF = U_OFF + (HAS_U ? CUBES_BYTES : 0);
  static constexpr int VEC_OFF = MN_OFF + 3 * 6 * 64 * 8;  // (M,N): [w][pair][pos] float2
  static constexpr int E_OFF = VEC_OFF + 3 * 3 * 8 * 8;     // (g,f): [pos][occ][l] float2
  static constexpr int BAR_OFF = E_OFF + 32 * 4;            // orbital energies [pos][l]
  static constexpr int BYTES = (BAR_OFF + 8 + 127) / 128 * 128;
  static constexpr int WARPS = HAS_U ? 6 : 8;
  static constexpr int THREADS = 32 * WARPS;
  static constexpr int SMEM = WARPS * BYTES + 128;  // + alignment of the base
  // bytes one orbit's TMA boxes deliver (out-of-range elements included)
  static constexpr uint32_t TX = (HAS_U ? 2 : 1) * CUBES_BYTES + 3 * 6 * 64 * 8;
  static_assert(MN_OFF % 128 == 0 && U_OFF % 128 == 0, "TMA destinations on 128 bytes");
  static_assert(SMEM <= 227 * 1024 - 256, "shared memory");
};

// Coefficient of index l_c in the staged address of ordering q's cube: the
// cube holds K at (l[perm3(q,0)], l[perm3(q,1)], l[perm3(q,2)]), pitches 1, 8, 64.
__host__ __device__ constexpr int cube_coef(int q, int c) {
  return perm3(q, 0) == c ? 1 : perm3(q, 1) == c ? 8 : 64;
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}

__device__ __forceinline__ int pick3(int i, int s0, int s1, int s2) {
  return i == 0 ? s0 : (i == 1 ? s1 : s2);
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(~0u, x, o);
  return x;
}

// Batch item y = blockIdx.y; warp w of block b takes orbits b*WARPS + w,
// stepping by gridDim.x*WARPS, and the block leaves its two sums at
// part[(2y + c) * gridDim.x + b].  mk / mu: K / K' slots (x, y, z, slot);
// mm / mt: (M, N) pairs (a, b, pair) and their transposes (b, a, pair).
template <bool HAS_U>
__global__ void __launch_bounds__(EnergyWarpSmem<HAS_U>::THREADS, 1)
    triples_energy_f32_kernel(const __grid_constant__ CUtensorMap mk,
                              const __grid_constant__ CUtensorMap mu,
                              const __grid_constant__ CUtensorMap mm,
                              const __grid_constant__ CUtensorMap mt, int nv,
                              const double* __restrict__ eijk_tab, const double* __restrict__ ev,
                              const TriplesTermsF* __restrict__ tt_tab,
                              const int* __restrict__ tri, int ntri, double* part,
                              unsigned long long wait_ns) {
  using L = EnergyWarpSmem<HAS_U>;
  extern __shared__ unsigned char esm_raw[];
  __shared__ double red[2][L::WARPS];
  unsigned char* esm = (unsigned char*)(((uintptr_t)esm_raw + 127) & ~(uintptr_t)127);
  const int y = blockIdx.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const TriplesTermsF tt = tt_tab[y];
  const float2* gfv[3] = {reinterpret_cast<const float2*>(tt.gf[0]),
                          reinterpret_cast<const float2*>(tt.gf[1]),
                          reinterpret_cast<const float2*>(tt.gf[2])};
  const double eijk = eijk_tab[y];
  unsigned char* wb = esm + warp * L::BYTES;
  float* cK = reinterpret_cast<float*>(wb);
  float* cU = reinterpret_cast<float*>(wb + L::U_OFF);
  float2* mn = reinterpret_cast<float2*>(wb + L::MN_OFF);
  float2* vg = reinterpret_cast<float2*>(wb + L::VEC_OFF);
  float* pe = reinterpret_cast<float*>(wb + L::E_OFF);
  uint64_t* bar = reinterpret_cast<uint64_t*>(wb + L::BAR_OFF);
  const int v = nv;
  if (lane == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    if (warp == 0) {
      asm volatile("prefetch.tensormap [%0];\n" ::"l"((uint64_t)&mk) : "memory");
      asm volatile("prefetch.tensormap [%0];\n" ::"l"((uint64_t)&mm) : "memory");
      asm volatile("prefetch.tensormap [%0];\n" ::"l"((uint64_t)&mt) : "memory");
      if (HAS_U) asm volatile("prefetch.tensormap [%0];\n" ::"l"((uint64_t)&mu) : "memory");
    }
  }
  __syncwarp();
  // evaluation roles: element (l0lo + 4a, l1lo + 4b, l2lo + 2c)
  const int l0lo = lane & 3, l1lo = (lane >> 2) & 3, l2lo = lane >> 4;

  double eK = 0.0, eY = 0.0;
  uint32_t phase = 0;
  for (int t = blockIdx.x * L::WARPS + warp; t < ntri; t += gridDim.x * L::WARPS) {
    const int S[3] = {tri[3 * t] * 8, tri[3 * t + 1] * 8, tri[3 * t + 2] * 8};
    // ---- stage the orbit ----
    if (lane == 0) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      mbar_expect_tx(bar, L::TX);
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const int x = S[perm3(q, 0)], yy = S[perm3(q, 1)], z = S[perm3(q, 2)];
        tma_load_4d(cK + q * EC_CUBE, &mk, bar, x, yy, z, y);
        if (HAS_U) tma_load_4d(cU + q * EC_CUBE, &mu, bar, x, yy, z, y);
      }
#pragma unroll
      for (int pr = 0; pr < 6; ++pr) {
        const int px = pr >> 1, py0 = pr & 1, py = py0 < px ? py0 : py0 + 1;
#pragma unroll
        for (int w = 0; w < 3; ++w) {
          float2* dst = mn + (w * 6 + pr) * 64;
          if (px < py)  // block [S_px + i, S_py + j] at i + 8j
            tma_load_3d(dst, &mm, bar, S[px], S[py], tt.mnpair[w]);
          else          // at j + 8i: from the transposed copy
            tma_load_3d(dst, &mt, bar, S[py], S[px], tt.mnpair[w]);
        }
      }
    }
    for (int u = lane; u < 72; u += 32) {  // (g, f) of occupied r at position p: u = (p*3 + r)*8 + l
      const int p = u / 24, r = (u >> 3) % 3, l = u & 7;
      const int x = pick3(p, S[0], S[1], S[2]) + l;
      const float2* src = r == 0 ? gfv[0] : r == 1 ? gfv[1] : gfv[2];
      cp_async8(vg + u, src + (x < v ? x : 0), x < v);
    }
    if (lane < 24) {  // virtual orbital energies; far above any denominator outside [0, v)
      const int x = pick3(lane >> 3, S[0], S[1], S[2]) + (lane & 7);
      pe[lane] = x < v ? (float)ev[x] : 1e30f;
    }
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
    const bool landed = mbar_wait(bar, phase, wait_ns);
    if (!__all_sync(~0u, landed)) {
      if (lane == 0) atomicExch(&g_energy_error, 1);
      mbar_wait(bar, phase, WAIT_NS);  // nothing of this warp's may stay in flight
      break;
    }
    phase ^= 1u;
    __syncwarp();

    // ---- evaluate: 16 elements per lane ----
    const bool ab = (S[0] == S[1]), bc = (S[1] == S[2]);
    const float wgt = (ab && bc) ? (1.0f / 6.0f) : (ab || bc) ? 0.5f : 1.0f;
    int kb[6];
#pragma unroll
    for (int q = 0; q < 6; ++q)
      kb[q] = q * EC_CUBE + cube_coef(q, 0) * l0lo + cube_coef(q, 1) * l1lo +
              cube_coef(q, 2) * l2lo;
    float ek = 0.0f, ey = 0.0f;
#pragma unroll
    for (int ia = 0; ia < 2; ++ia) {
      const int l0 = l0lo + 4 * ia;
      const float e0 = (float)(eijk - (double)pe[l0]);
      float2 v0[3];
#pragma unroll
      for (int r = 0; r < 3; ++r) v0[r] = vg[(0 * 3 + r) * 8 + l0];
#pragma unroll
      for (int ib = 0; ib < 2; ++ib) {
        const int l1 = l1lo + 4 * ib;
        const float e01 = e0 - pe[8 + l1];
        float2 v1[3], m01[3], m10[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) v1[r] = vg[(1 * 3 + r) * 8 + l1];
#pragma unroll
        for (int w = 0; w < 3; ++w) {
          m01[w] = mn[(w * 6 + 0) * 64 + l0 + 8 * l1];
          m10[w] = mn[(w * 6 + 2) * 64 + l0 + 8 * l1];
        }
#pragma unroll
        for (int ic = 0; ic < 4; ++ic) {
          const int l2 = l2lo + 2 * ic;
          const float dinv = __fdividef(1.0f, e01 - pe[16 + l2]);
          float2 v2[3], m02[3], m20[3], m12[3], m21[3];
#pragma unroll
          for (int r = 0; r < 3; ++r) v2[r] = vg[(2 * 3 + r) * 8 + l2];
#pragma unroll
          for (int w = 0; w < 3; ++w) {
            m02[w] = mn[(w * 6 + 1) * 64 + l0 + 8 * l2];
            m20[w] = mn[(w * 6 + 4) * 64 + l0 + 8 * l2];
            m12[w] = mn[(w * 6 + 3) * 64 + l1 + 8 * l2];
            m21[w] = mn[(w * 6 + 5) * 64 + l1 + 8 * l2];
          }
          float k[6];
#pragma unroll
          for (int q = 0; q < 6; ++q)
            k[q] = cK[kb[q] + 4 * ia * cube_coef(q, 0) + 4 * ib * cube_coef(q, 1) +
                      2 * ic * cube_coef(q, 2)];
          float se = 0.0f, so = 0.0f;
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            if (perm3_parity(q)) so += k[q];
            else se += k[q];
          }
          const float ce = se - 2.0f * so, co = so - 2.0f * se;
          float X[6];
#pragma unroll
          for (int q = 0; q < 6; ++q) X[q] = (3.0f * k[q] + (perm3_parity(q) ? co : ce)) * dinv;
          // Y of ordering (p0,p1,p2): the pair (x, y) with third position z
          // adds to the orderings (z,x,y), (x,z,y), (x,y,z) through w = 0, 1, 2
          float yq[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
          auto add_pair = [&](int x, int yy, const float2(&m)[3], const float2(&vz)[3]) {
            const int z = 3 - x - yy;
            float& y0 = yq[perm3_index(z, x)];
            float& y1 = yq[perm3_index(x, z)];
            float& y2 = yq[perm3_index(x, yy)];
            y0 = fmaf(vz[0].y, m[0].y, fmaf(vz[0].x, m[0].x, y0));
            y1 = fmaf(vz[1].y, m[1].y, fmaf(vz[1].x, m[1].x, y1));
            y2 = fmaf(vz[2].y, m[2].y, fmaf(vz[2].x, m[2].x, y2));
          };
          add_pair(0, 1, m01, v2);
          add_pair(1, 0, m10, v2);
          add_pair(0, 2, m02, v1);
          add_pair(2, 0, m20, v1);
          add_pair(1, 2, m12, v0);
          add_pair(2, 1, m21, v0);
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            const float kp = HAS_U ? cU[kb[q] + 4 * ia * cube_coef(q, 0) +
                                        4 * ib * cube_coef(q, 1) + 2 * ic * cube_coef(q, 2)]
                                   : k[q];
            ek = fmaf(kp, X[q], ek);
            ey = fmaf(X[q], yq[q], ey);
          }
        }
      }
    }
    eK += (double)(wgt * ek);
    eY += (double)(wgt * ey);
    __syncwarp();  // every lane is done with the buffers before they are refilled
  }
  asm volatile("cp.async.wait_group 0;\n" ::);
  eK = warp_sum(eK);
  eY = warp_sum(eY);
  if (lane == 0) {
    red[0][warp] = eK;
    red[1][warp] = eY;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0;
    for (int w = 0; w < L::WARPS; ++w) {
      s0 += red[0][w];
      s1 += red[1][w];
    }
    part[(2 * y) * gridDim.x + blockIdx.x] = s0;
    part[(2 * y + 1) * gridDim.x + blockIdx.x] = s1;
  }
}

// out[2y + c] = sum_i part[(2y + c) * nparts + i], one warp per (y, c), fixed order
__global__ void energy_final_kernel(int nparts, const double* __restrict__ part,
                                    double* __restrict__ out) {
  const int q = blockIdx.x, lane = threadIdx.x;
  double acc = 0.0;
  for (int i = lane; i < nparts; i += 32) acc += part[(int64_t)q * nparts + i];
  acc = warp_sum(acc);
  if (lane == 0) out[q] = acc;
}

// (M, N)[a + vpe b] and its transpose [b + vpe a] per occupied pair, FP32 pairs.
__global__ void mn_pack_kernel(int v, int vpe, int64_t npairs, const double* __restrict__ M,
                               const double* __restrict__ N, float2* __restrict__ mn,
                               float2* __restrict__ mt) {
  const int64_t vv = (int64_t)v * v, total = vv * npairs, pitch = (int64_t)vpe * v;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / vv, r = i - p * vv, b = r / v, a = r - b * v;
    const float2 x = make_float2((float)M[i], (float)N[i]);
    mn[p * pitch + a + (int64_t)vpe * b] = x;
    mt[p * pitch + b + (int64_t)vpe * a] = x;
  }
}

int encode(CUtensorMap* m, CUtensorMapDataType type, int rank, const void* base,
           const cuuint64_t* dims, const cuuint64_t* strides, const cuuint32_t* box) {
  EncodeFn enc = nullptr;
  if (int e = encode_fn(&enc)) return e;
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(m, type, (cuuint32_t)rank, const_cast<void*>(base), dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : (int)cudaErrorInvalidValue;
}

template <bool HAS_U>
int launch_energy(cudaStream_t st, dim3 grid, const CUtensorMap* maps, int nv,
                  const double* eijk_tab, const double* ev, const TriplesTermsF* tt_tab,
                  const int* tri, int ntri, double* scratch) {
  using L = EnergyWarpSmem<HAS_U>;
  auto kern = triples_energy_f32_kernel<HAS_U>;
  // cudaFuncSetAttribute acts on the current device only: one flag per device
  static std::atomic<bool> done[128] = {};
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) {
    cudaGetLastError();
    return (int)cudaErrorInvalidDevice;
  }
  if (d < 0 || d >= 128 || !done[d].load(std::memory_order_acquire)) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM);
    if (e != cudaSuccess) return (int)e;
    if (d >= 0 && d < 128) done[d].store(true, std::memory_order_release);
  }
  const unsigned long long w = tc_wait((stream_t)st);
  kern<<<grid, L::THREADS, L::SMEM, st>>>(maps[0], maps[1], maps[2], maps[3], nv, eijk_tab, ev,
                                          tt_tab, tri, ntri, scratch, w ? w : WAIT_NS);
  note_launches(1);
  return (int)cudaGetLastError();
}

}  // namespace

int64_t triples_mn_elems(int nv, int64_t npairs) {
  return (int64_t)((nv + 1) / 2 * 2) * nv * npairs;
}

int triples_mn_pack(stream_t s, int nv, int64_t npairs, const double* M, const double* N,
                    void* mn, void* mt) {
  if (nv <= 0 || npairs <= 0 || ((uintptr_t)mn & 15) || ((uintptr_t)mt & 15))
    return (int)cudaErrorInvalidValue;
  const int vpe = (nv + 1) / 2 * 2;
  const int64_t total = (int64_t)nv * nv * npairs;
  const int64_t blocks = std::min<int64_t>((total + 255) / 256, 148 * 16);
  mn_pack_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)s>>>(
      nv, vpe, npairs, M, N, reinterpret_cast<float2*>(mn), reinterpret_cast<float2*>(mt));
  note_launches(1);
  return (int)cudaGetLastError();
}

int triples_energy_f32_batched(stream_t s, int nv, int vp, int nitems, int nslots, const float* K,
                               const float* KU, int64_t kstride, const void* mn, const void* mt,
                               int64_t npairs, const double* eijk_tab, const double* ev,
                               const TriplesTermsF* tt_tab, const int* tri, double* scratch,
                               double* out) {
  const int64_t ntri = triples_cube_count(nv);
  if (nv <= 0 || nv > 1290 || vp < nv || vp % 4 != 0 || kstride < (int64_t)vp * nv * nv ||
      kstride % 4 != 0 || nitems <= 0 || nitems > nslots || nitems > 65535 || !eijk_tab ||
      !tt_tab || !K || !mn || !mt || npairs <= 0 || npairs >= ((int64_t)1 << 31) ||
      ((uintptr_t)K & 15) || ((uintptr_t)KU & 15) || ((uintptr_t)mn & 15) ||
      ((uintptr_t)mt & 15))
    return (int)cudaErrorInvalidValue;
  CUtensorMap maps[4];
  {
    const cuuint64_t dk[4] = {(cuuint64_t)nv, (cuuint64_t)nv, (cuuint64_t)nv, (cuuint64_t)nslots};
    const cuuint64_t sk[3] = {(cuuint64_t)vp * 4, (cuuint64_t)vp * nv * 4, (cuuint64_t)kstride * 4};
    const cuuint32_t bk[4] = {8, 8, 8, 1};
    if (int e = encode(&maps[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, K, dk, sk, bk)) return e;
    if (KU) {
      if (int e = encode(&maps[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, KU, dk, sk, bk)) return e;
    } else {
      maps[1] = maps[0];
    }
    const int64_t vpe = (nv + 1) / 2 * 2;
    const cuuint64_t dm[3] = {(cuuint64_t)nv, (cuuint64_t)nv, (cuuint64_t)npairs};
    const cuuint64_t sm[2] = {(cuuint64_t)vpe * 8, (cuuint64_t)vpe * nv * 8};
    const cuuint32_t bm[3] = {8, 8, 1};
    // (M, N) FP32 pairs move as 8-byte elements
    if (int e = encode(&maps[2], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, mn, dm, sm, bm)) return e;
    if (int e = encode(&maps[3], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, mt, dm, sm, bm)) return e;
  }
  const int g = (int)triples_energy_grid(nv);
  cudaStream_t st = (cudaStream_t)s;
  const dim3 grid((unsigned)g, (unsigned)nitems);
  const int slot = ktime_begin(s, KT_TRIPLES);
  const double kbytes = (double)nitems * (double)nv * nv * nv * 4.0 * (KU ? 2.0 : 1.0);
  const int e = KU ? launch_energy<true>(st, grid, maps, nv, eijk_tab, ev, tt_tab, tri, (int)ntri,
                                         scratch)
                   : launch_energy<false>(st, grid, maps, nv, eijk_tab, ev, tt_tab, tri,
                                          (int)ntri, scratch);
  ktime_end(s, KT_TRIPLES, slot, kbytes);
  if (e) return e;
  energy_final_kernel<<<2 * nitems, 32, 0, st>>>(g, scratch, out);
  note_launches(1);
  return (int)cudaGetLastError();
}

int energy_error(int* code) {
  int h = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&h, g_energy_error, sizeof(int));
  if (e != cudaSuccess) return (int)e;
  *code = h;
  if (h) {
    int zero = 0;
    cudaMemcpyToSymbol(g_energy_error, &zero, sizeof(int));
  }
  return 0;
}

}  // namespace dev
}  // namespace ecg
