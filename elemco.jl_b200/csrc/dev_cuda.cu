// dev_cuda.cu — CUDA implementation of the device layer (ecg_dev.h) for
// sm_100a: FP64 GEMM on the double-precision MMA pipe, tensor permutation,
// amplitude updates and deterministic reductions.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "ecg_dev.h"
#include "ecg_tune.h"
#include "triples_perm.h"

namespace ecg {
namespace dev {

static std::atomic<int64_t> g_launches{0};
int64_t launches() { return g_launches.load(); }
void note_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
static inline int launched() {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return (int)cudaGetLastError();
}

int set_device(int device) { return (int)cudaSetDevice(device); }

// ---- per-stream state ------------------------------------------------------
//
// Scratch that the GEMM launchers need beyond their operands — the split-K
// partial products and the BF16 slices of gemm_mixed — belongs to the stream
// (and device) the GEMM runs on.  A context owns one stream, so contexts on
// different devices, or on different host threads, never share it.  A buffer
// grows only after its stream has drained, so no kernel of that stream still
// reads the old one, and never during stream capture.  The tensor-core wait
// bound is kept here too.  Entries of streams the library did not create
// (a caller's stream) live until process exit.
namespace {
struct StreamState {
  double* splitk = nullptr;
  size_t splitk_len = 0;  // doubles
  void* split = nullptr;
  size_t split_bytes = 0;
  unsigned long long tc_wait_ns = 0;  // 0: the default bound
};
std::mutex g_ss_mu;
std::map<std::pair<cudaStream_t, int>, StreamState> g_ss;

int current_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return d;
}

// The state of stream s on the current device (created empty on first use);
// the caller holds g_ss_mu.  std::map nodes stay put while others are added.
StreamState& stream_state_locked(cudaStream_t s) { return g_ss[{s, current_device()}]; }

bool capturing(cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return cs != cudaStreamCaptureStatusNone;
}

// Grow *p (holding *have bytes) to at least `want` bytes (plus `extra`
// headroom) for stream s; nullptr if that needs an allocation during capture
// or the allocation fails.
void* grow(cudaStream_t s, void** p, size_t* have, size_t want, size_t extra) {
  if (want <= *have) return *p;
  if (capturing(s)) return nullptr;
  if (*p) {
    cudaStreamSynchronize(s);
    cudaFree(*p);
  }
  *p = nullptr;
  *have = 0;
  if (cudaMalloc(p, want + extra) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return nullptr;
  }
  *have = want + extra;
  return *p;
}
}  // namespace

int stream_create(stream_t* s) {
  cudaStream_t st;
  int e = (int)cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  *s = (stream_t)st;
  return e;
}

void stream_destroy(stream_t s) {
  cudaStream_t st = (cudaStream_t)s;
  cudaStreamSynchronize(st);
  {
    std::lock_guard<std::mutex> lk(g_ss_mu);
    auto it = g_ss.find({st, current_device()});
    if (it != g_ss.end()) {
      if (it->second.splitk) cudaFree(it->second.splitk);
      if (it->second.split) cudaFree(it->second.split);
      g_ss.erase(it);
    }
  }
  cudaStreamDestroy(st);
}

double* splitk_buffer(stream_t s, size_t n) {
  std::lock_guard<std::mutex> lk(g_ss_mu);
  StreamState& ss = stream_state_locked((cudaStream_t)s);
  size_t have = ss.splitk_len * sizeof(double);
  const size_t want = std::max(n, (size_t)1 << 22) * sizeof(double);
  void* p = ss.splitk;
  void* r = grow((cudaStream_t)s, &p, &have, want, 0);
  ss.splitk = (double*)p;
  ss.splitk_len = have / sizeof(double);
  return (double*)r;
}

void* split_scratch(stream_t s, size_t bytes) {
  std::lock_guard<std::mutex> lk(g_ss_mu);
  StreamState& ss = stream_state_locked((cudaStream_t)s);
  return grow((cudaStream_t)s, &ss.split, &ss.split_bytes, bytes, bytes / 4);
}

int set_tc_wait(stream_t s, uint64_t ns) {
  std::lock_guard<std::mutex> lk(g_ss_mu);
  stream_state_locked((cudaStream_t)s).tc_wait_ns = ns;
  return 0;
}

uint64_t tc_wait(stream_t s) {
  std::lock_guard<std::mutex> lk(g_ss_mu);
  return stream_state_locked((cudaStream_t)s).tc_wait_ns;
}
int sync(stream_t s) { return (int)cudaStreamSynchronize((cudaStream_t)s); }
const char* error_string(int code) { return cudaGetErrorString((cudaError_t)code); }
int check_launch() { return (int)cudaGetLastError(); }

void* dmalloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMalloc(&p, bytes < 256 ? 256 : bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}
void dfree(void* p) {
  if (p) cudaFree(p);
}
void* hmalloc_pinned(size_t bytes) {
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}
void hfree_pinned(void* p) {
  if (p) cudaFreeHost(p);
}
int h2d(void* dst, const void* src, size_t bytes, stream_t s) {
  if (!bytes) return 0;
  return (int)cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, (cudaStream_t)s);
}
int d2h(void* dst, const void* src, size_t bytes, stream_t s) {
  if (!bytes) return 0;
  return (int)cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)s);
}
int d2d(void* dst, const void* src, size_t bytes, stream_t s) {
  if (!bytes) return 0;
  return (int)cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)s);
}
int graph_capture_begin(stream_t s) {
  return (int)cudaStreamBeginCapture((cudaStream_t)s, cudaStreamCaptureModeThreadLocal);
}

int graph_capture_run(stream_t s, int64_t* nodes) {
  cudaStream_t st = (cudaStream_t)s;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(st, &g);
  if (e != cudaSuccess) return (int)e;
  size_t n = 0;
  cudaGraphGetNodes(g, nullptr, &n);
  if (nodes) *nodes = (int64_t)n;
  cudaGraphExec_t x = nullptr;
  e = cudaGraphInstantiate(&x, g, 0);
  if (e == cudaSuccess) {
    e = cudaGraphLaunch(x, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaGraphExecDestroy(x);
  }
  cudaGraphDestroy(g);
  return (int)e;
}

void graph_capture_abort(stream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing((cudaStream_t)s, &cs) == cudaSuccess &&
      cs != cudaStreamCaptureStatusNone) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture((cudaStream_t)s, &g);
    if (g) cudaGraphDestroy(g);
  }
  cudaGetLastError();
}

int memset0(void* dst, size_t bytes, stream_t s) {
  if (!bytes) return 0;
  return (int)cudaMemsetAsync(dst, 0, bytes, (cudaStream_t)s);
}

// One flag per device (cudaFuncSetAttribute acts on the current device only):
// test() reports whether the current device's flag is set, set(e) sets it when
// the attribute call e succeeded.  Two threads may both set it; that is
// harmless (the attribute call is idempotent).
struct DeviceFlags {
  std::atomic<bool> f[128] = {};
  bool test() {
    const int d = current_device();
    return d >= 0 && d < 128 && f[d].load(std::memory_order_acquire);
  }
  void set(cudaError_t e) {
    const int d = current_device();
    if (e == cudaSuccess && d >= 0 && d < 128) f[d].store(true, std::memory_order_release);
    if (e != cudaSuccess) cudaGetLastError();
  }
};

// ---------------------------------------------------------------- GEMM
//
// Column-major C(m,n) = alpha*opA(A)(m,k)*opB(B)(k,n) + beta*C.  Tiles of
// BM x BN per CTA, BK deep, staged through shared memory with a
// STAGES-deep cp.async ring; each warp owns a WM x WN sub-tile computed
// with mma.sync m8n8k4 f64 (the FP64 MMA pipe).  Shared tiles are stored
// k-major ([k][m] and [k][n]) with a row pitch of BM+4 / BN+4 doubles so that
// the 8x4 fragment reads of a half-warp hit 32 distinct banks.

struct GemmArgs {
  const double* A;
  const double* B;
  double* C;
  int64_t m, n, k;
  int64_t sam, sak, sab, sbk, sbn, sbb, scm, scn, scb;
  double alpha, beta;
  int a_kfast, b_nfast;  // loader thread order follows the unit-stride index
  int64_t klast;         // split-K: depth of the last z-slice (0 = all slices use k)
  int64_t dn = 0, scn2 = 0;  // dn > 0: column n at (n % dn)*scn + (n / dn)*scn2
  int64_t kseg = 0;          // kseg > 0: k >= kseg reads A1/B1 with strides sak1/sbk1
  const double* A1 = nullptr;
  int64_t sak1 = 0;
  const double* B1 = nullptr;
  int64_t sbk1 = 0;
  const int64_t* ptab = nullptr;  // GF_PTAB: offsets of A, B, C, A1, B1 per batch item
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

// m16n8kK FP64 MMA (K = 4, 8, 16; sm_90+ shapes).  Fragments, with g = lane/4
// and t = lane%4: A (16 x K) a[2j] = A(g, t+4j), a[2j+1] = A(g+8, t+4j);
// B (K x 8) b[j] = B(t+4j, g); C (16 x 8) c0,c1 = C(g, 2t..2t+1),
// c2,c3 = C(g+8, 2t..2t+1).
template <int K>
__device__ __forceinline__ void dmma16(double (&d)[4], const double* a, const double* b) {
  if constexpr (K == 4) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
        "{%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(b[0]));
  } else if constexpr (K == 8) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
  } else {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
        "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]),
          "d"(a[7]), "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
  }
}

template <int BM, int BN, int BK, int WM, int WN, int STAGES, int MINB = 1>
struct GemmCfg {
  static constexpr int WARPS_M = BM / WM;
  static constexpr int WARPS_N = BN / WN;
  static constexpr int THREADS = WARPS_M * WARPS_N * 32;
  static constexpr int LDA_S = BM + 4;
  static constexpr int LDB_S = BN + 4;
  static constexpr int A_STAGE = BK * LDA_S;
  static constexpr int B_STAGE = BK * LDB_S;
  static constexpr size_t SMEM = (size_t)STAGES * (A_STAGE + B_STAGE) * sizeof(double);
};

// KMMA = 0: mma.m8n8k4 (8-row fragments); KMMA = 4, 8, 16: mma.m16n8kKMMA.
// FLAGS: bit 0 = two K segments (kseg/A1/B1), bit 1 = split column index (dn),
// bit 2 = batch items placed by an offset table (ptab) instead of strides;
// plain GEMMs instantiate none, so their loader and epilogue stay minimal.
constexpr int GF_SEG = 1, GF_DN = 2, GF_PTAB = 4;
template <int BM, int BN, int BK, int WM, int WN, int STAGES, int MINB, int KMMA, int FLAGS>
__global__ void __launch_bounds__(GemmCfg<BM, BN, BK, WM, WN, STAGES>::THREADS, MINB)
    dgemm_kernel(GemmArgs g) {
  using Cfg = GemmCfg<BM, BN, BK, WM, WN, STAGES>;
  constexpr int NT = Cfg::THREADS;
  constexpr int RH = (KMMA == 0) ? 8 : 16;  // rows of one MMA fragment
  constexpr int NACC = (KMMA == 0) ? 2 : 4;  // accumulators per fragment and thread
  constexpr int MT = WM / RH, NTL = WN / 8;
  static_assert(KMMA == 0 || BK % KMMA == 0, "BK must be a multiple of the MMA depth");
  extern __shared__ double smem[];
  double* As = smem;
  double* Bs = smem + STAGES * Cfg::A_STAGE;

  const int64_t bz = blockIdx.z;
  const double* A;
  const double* B;
  double* C;
  const double* A1 = g.A1;
  const double* B1 = g.B1;
  if constexpr ((FLAGS & GF_PTAB) != 0) {
    const int64_t* pt = g.ptab + 5 * bz;
    A = g.A + pt[0];
    B = g.B + pt[1];
    C = g.C + pt[2];
    if constexpr ((FLAGS & GF_SEG) != 0) {
      A1 = g.A1 + pt[3];
      B1 = g.B1 + pt[4];
    }
  } else {
    A = g.A + bz * g.sab;
    B = g.B + bz * g.sbb;
    C = g.C + bz * g.scb;
  }
  const int64_t m0 = (int64_t)blockIdx.x * BM;
  const int64_t n0 = (int64_t)blockIdx.y * BN;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int wm0 = (warp % Cfg::WARPS_M) * WM;
  const int wn0 = (warp / Cfg::WARPS_M) * WN;
  const int gq = lane >> 2, tq = lane & 3;
  const int64_t kdep = (g.klast > 0 && bz == (int64_t)gridDim.z - 1) ? g.klast : g.k;
  const int64_t KT = (kdep + BK - 1) / BK;

  auto load_tile = [&](int stage, int64_t kt) {
    const int64_t k0 = kt * BK;
    double* as = As + stage * Cfg::A_STAGE;
    double* bs = Bs + stage * Cfg::B_STAGE;
#pragma unroll
    for (int r = 0; r < (BM * BK + NT - 1) / NT; ++r) {
      int e = tid + r * NT;
      if (e < BM * BK) {
        int mm, kk;
        if (!g.a_kfast) { mm = e % BM; kk = e / BM; } else { kk = e % BK; mm = e / BK; }
        int64_t gm = m0 + mm, gk = k0 + kk;
        bool ok = gm < g.m && gk < kdep;
        const double* src = A;
        if constexpr ((FLAGS & GF_SEG) != 0) {
          if (ok)
            src = (gk >= g.kseg) ? A1 + gm * g.sam + (gk - g.kseg) * g.sak1
                                 : A + gm * g.sam + gk * g.sak;
        } else {
          if (ok) src = A + gm * g.sam + gk * g.sak;
        }
        cp_async8(as + kk * Cfg::LDA_S + mm, src, ok);
      }
    }
#pragma unroll
    for (int r = 0; r < (BN * BK + NT - 1) / NT; ++r) {
      int e = tid + r * NT;
      if (e < BN * BK) {
        int nn, kk;
        if (!g.b_nfast) { kk = e % BK; nn = e / BK; } else { nn = e % BN; kk = e / BN; }
        int64_t gn = n0 + nn, gk = k0 + kk;
        bool ok = gn < g.n && gk < kdep;
        const double* src = B;
        if constexpr ((FLAGS & GF_SEG) != 0) {
          if (ok)
            src = (gk >= g.kseg) ? B1 + (gk - g.kseg) * g.sbk1 + gn * g.sbn
                                 : B + gk * g.sbk + gn * g.sbn;
        } else {
          if (ok) src = B + gk * g.sbk + gn * g.sbn;
        }
        cp_async8(bs + kk * Cfg::LDB_S + nn, src, ok);
      }
    }
  };

  double acc[MT][NTL][NACC];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NTL; ++j)
#pragma unroll
      for (int c = 0; c < NACC; ++c) acc[i][j][c] = 0.0;

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < KT) load_tile(s, s);
    cp_async_commit();
  }
  for (int64_t kt = 0; kt < KT; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    int64_t nxt = kt + STAGES - 1;
    if (nxt < KT) load_tile((int)(nxt % STAGES), nxt);
    cp_async_commit();
    const double* as = As + (kt % STAGES) * Cfg::A_STAGE;
    const double* bs = Bs + (kt % STAGES) * Cfg::B_STAGE;
    if constexpr (KMMA == 0) {
#pragma unroll
      for (int kk = 0; kk < BK; kk += 4) {
        double af[MT], bf[NTL];
#pragma unroll
        for (int i = 0; i < MT; ++i) af[i] = as[(kk + tq) * Cfg::LDA_S + wm0 + i * 8 + gq];
#pragma unroll
        for (int j = 0; j < NTL; ++j) bf[j] = bs[(kk + tq) * Cfg::LDB_S + wn0 + j * 8 + gq];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NTL; ++j) {
            double d2[2] = {acc[i][j][0], acc[i][j][1]};
            dmma884(d2, af[i], bf[j]);
            acc[i][j][0] = d2[0];
            acc[i][j][1] = d2[1];
          }
      }
    } else {
      constexpr int KQ = KMMA / 4;
#pragma unroll
      for (int kk = 0; kk < BK; kk += KMMA) {
        double af[MT][2 * KQ], bf[NTL][KQ];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int q = 0; q < KQ; ++q) {
            const double* ap = as + (kk + tq + 4 * q) * Cfg::LDA_S + wm0 + i * 16 + gq;
            af[i][2 * q] = ap[0];
            af[i][2 * q + 1] = ap[8];
          }
#pragma unroll
        for (int j = 0; j < NTL; ++j)
#pragma unroll
          for (int q = 0; q < KQ; ++q)
            bf[j][q] = bs[(kk + tq + 4 * q) * Cfg::LDB_S + wn0 + j * 8 + gq];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NTL; ++j) {
            double d4[4] = {acc[i][j][0], acc[i][j][1], acc[i][j][2], acc[i][j][3]};
            dmma16<KMMA>(d4, af[i], bf[j]);
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[i][j][c] = d4[c];
          }
      }
    }
  }
  cp_async_wait<0>();

  int64_t coff[NTL][2];
#pragma unroll
  for (int j = 0; j < NTL; ++j)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t col = n0 + wn0 + j * 8 + 2 * tq + h;
      if constexpr ((FLAGS & GF_DN) != 0)
        coff[j][h] = (col % g.dn) * g.scn + (col / g.dn) * g.scn2;
      else
        coff[j][h] = col * g.scn;
    }
  if (g.beta == 0.0) {
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int rr = 0; rr < NACC / 2; ++rr) {
        const int64_t row = m0 + wm0 + i * RH + 8 * rr + gq;
        if (row >= g.m) continue;
#pragma unroll
        for (int j = 0; j < NTL; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int64_t col = n0 + wn0 + j * 8 + 2 * tq + h;
            if (col < g.n) C[row * g.scm + coff[j][h]] = g.alpha * acc[i][j][2 * rr + h];
          }
      }
    return;
  }
  // read-modify-write: per fragment row, all C values are loaded before any
  // store (the compiler cannot prove the stores disjoint from later loads)
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int rr = 0; rr < NACC / 2; ++rr) {
      const int64_t row = m0 + wm0 + i * RH + 8 * rr + gq;
      if (row >= g.m) continue;
      double cv[NTL][2];
#pragma unroll
      for (int j = 0; j < NTL; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int64_t col = n0 + wn0 + j * 8 + 2 * tq + h;
          cv[j][h] = col < g.n ? g.beta * C[row * g.scm + coff[j][h]] : 0.0;
        }
#pragma unroll
      for (int j = 0; j < NTL; ++j) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int64_t col = n0 + wn0 + j * 8 + 2 * tq + h;
          if (col < g.n) C[row * g.scm + coff[j][h]] = g.alpha * acc[i][j][2 * rr + h] + cv[j][h];
        }
      }
    }
}

template <int BM, int BN, int BK, int WM, int WN, int STAGES, int MINB = 1, int KMMA = 0,
          int FLAGS = 0>
static int launch_gemm(const GemmArgs& g, int64_t batch, cudaStream_t st) {
  using Cfg = GemmCfg<BM, BN, BK, WM, WN, STAGES>;
  static DeviceFlags attr;
  if (!attr.test())
    attr.set(cudaFuncSetAttribute(dgemm_kernel<BM, BN, BK, WM, WN, STAGES, MINB, KMMA, FLAGS>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM));
  int64_t gx = (g.m + BM - 1) / BM, gy = (g.n + BN - 1) / BN;
  if (gy > 65535 || batch > 65535) return (int)cudaErrorInvalidConfiguration;
  dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)batch);
  dgemm_kernel<BM, BN, BK, WM, WN, STAGES, MINB, KMMA, FLAGS>
      <<<grid, Cfg::THREADS, Cfg::SMEM, st>>>(g);
  return launched();
}

static unsigned grid_for(int64_t n, int threads = 256, int64_t cap = 148 * 16);


// C = alpha sum_z P[z] + beta C, the partials (FP64, or FP32 for the
// tensor-core GEMM, whose partials are FP32 accumulations) summed in FP64 in
// slice order.
// IT: index type of the element loop (32-bit unsigned whenever m * n allows).
template <typename PT, typename IT>
__global__ void splitk_reduce_kernel(int64_t m, int64_t n, int S, const PT* __restrict__ P,
                                     double alpha, double beta, double* C, int64_t scm,
                                     int64_t scn) {
  const int64_t total = m * n;
  const IT tot = (IT)total, mi = (IT)m;
  for (IT idx = blockIdx.x * (IT)blockDim.x + threadIdx.x; idx < tot;
       idx += (IT)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int z = 0; z < S; ++z) acc += (double)P[z * total + (int64_t)idx];
    double* c = C + (int64_t)(idx % mi) * scm + (int64_t)(idx / mi) * scn;
    double v = alpha * acc;
    if (beta != 0.0) v += beta * *c;
    *c = v;
  }
}

template <typename PT>
void launch_reduce(cudaStream_t st, int64_t m, int64_t n, int S, const PT* P, double alpha,
                   double beta, double* C, int64_t scm, int64_t scn) {
  const unsigned g = grid_for(m * n);
  if (m * n < ((int64_t)1 << 32) - 256 * 148 * 16)
    splitk_reduce_kernel<PT, uint32_t><<<g, 256, 0, st>>>(m, n, S, P, alpha, beta, C, scm, scn);
  else
    splitk_reduce_kernel<PT, uint64_t><<<g, 256, 0, st>>>(m, n, S, P, alpha, beta, C, scm, scn);
}

// ---- split-K GEMM without any allocation --------------------------------
//
// For callers that cannot allocate device memory (code running under a
// framework's memory manager, inside stream capture, or in a process whose
// device memory is fully handed out): the partial products live in this
// fixed file-scope array, 2^22 doubles (32 MiB), which every GPU that loads
// the library keeps until process exit.  Host code cannot use the symbol as
// a device address; its address is looked up once per device with
// cudaGetSymbolAddress (on the first call on that device, with that device
// current) and cached.
static constexpr size_t kNoAllocScratchDoubles = (size_t)1 << 22;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];
static double* g_noalloc_ptr[128] = {nullptr};
static std::mutex g_noalloc_mu;

size_t noalloc_scratch_doubles() { return kNoAllocScratchDoubles; }

static int noalloc_scratch_ptr(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= 128) return (int)cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return (int)e;
    g_noalloc_ptr[dev] = (double*)p;
  }
  *out = g_noalloc_ptr[dev];
  return 0;
}

int gemm_splitk_noalloc(stream_t s, char ta, char tb, int64_t m, int64_t n, int64_t k,
                        double alpha, const double* A, int64_t lda, const double* B, int64_t ldb,
                        double beta, double* C, int64_t ldc, int* nsplit) {
  if (m <= 0 || n <= 0 || k <= 0) return (int)cudaErrorInvalidValue;
  if ((uint64_t)n > kNoAllocScratchDoubles / (uint64_t)m) return (int)cudaErrorInvalidValue;
  double* P = nullptr;
  int e = noalloc_scratch_ptr(&P);
  if (e) return e;
  bool at = (ta == 'T' || ta == 't'), bt = (tb == 'T' || tb == 't');
  int64_t ldcm = 1, ldcn = ldc;  // C(i,j) at C[i*ldcm + j*ldcn]
  if ((n + 63) / 64 > 65535) {
    // more column tiles than the grid's y extent: compute C^T = op(B)^T op(A)^T
    // (the m <-> n swap puts the long dimension on the grid's x axis)
    std::swap(m, n);
    std::swap(A, B);
    std::swap(lda, ldb);
    const bool t = at;
    at = !bt;
    bt = !t;
    std::swap(ldcm, ldcn);
  }
  const int64_t tiles64 = ((m + 63) / 64) * ((n + 63) / 64);
  int64_t S = std::min<int64_t>((2 * 148 + tiles64 - 1) / tiles64, (k + 255) / 256);
  S = std::max<int64_t>(1, std::min<int64_t>(S, 64));
  while (S > 1 && (size_t)S * m * n > kNoAllocScratchDoubles) --S;
  int64_t kc = (k + S - 1) / S;
  kc = (kc + 15) / 16 * 16;
  S = (k + kc - 1) / kc;
  GemmArgs h{A, B, P, m, n, kc, at ? lda : 1, at ? 1 : lda, 0, bt ? ldb : 1, bt ? 1 : ldb, 0,
             1, m, m * n, 1.0, 0.0, (at && lda != 1) ? 1 : 0, (bt && ldb != 1) ? 1 : 0,
             k - (S - 1) * kc};
  h.sab = kc * h.sak;
  h.sbb = kc * h.sbk;
  cudaStream_t st = (cudaStream_t)s;
  e = launch_gemm<64, 64, 16, 32, 32, 3, 3>(h, S, st);
  if (e) return e;
  launch_reduce(st, m, n, (int)S, P, alpha, beta, C, ldcm, ldcn);
  if (nsplit) *nsplit = (int)S;
  return launched();
}

int splitk_reduce(stream_t s, int64_t m, int64_t n, int S, const double* P, double alpha,
                  double beta, double* C, int64_t scm, int64_t scn) {
  launch_reduce((cudaStream_t)s, m, n, S, P, alpha, beta, C, scm, scn);
  return launched();
}

int splitk_reduce_f32(stream_t s, int64_t m, int64_t n, int S, const float* P, double alpha,
                      double beta, double* C, int64_t scm, int64_t scn) {
  launch_reduce((cudaStream_t)s, m, n, S, P, alpha, beta, C, scm, scn);
  return launched();
}

// Event timing of kernel families (a diagnostic; enable, run, read): each
// timed launch is bracketed by an event pair on its stream, and its
// algorithmic work (flops or bytes) is added to the family's total.
// Launches made during stream capture are not timed.
namespace {
struct Family {
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  size_t used = 0;
  double work = 0.0;
};
bool g_timing = false;
Family g_fam[KT_FAMILIES];
std::mutex g_fam_mu;
}  // namespace

void gemm_timing(bool enable) {
  std::lock_guard<std::mutex> lk(g_fam_mu);
  g_timing = enable;
  for (auto& f : g_fam) {
    f.used = 0;
    f.work = 0.0;
  }
}

int ktime_begin(stream_t s, int family) {
  if (!g_timing || family < 0 || family >= KT_FAMILIES || capturing((cudaStream_t)s)) return -1;
  std::lock_guard<std::mutex> lk(g_fam_mu);
  Family& f = g_fam[family];
  if (f.used == f.ev.size()) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    f.ev.push_back({a, b});
  }
  cudaEventRecord(f.ev[f.used].first, (cudaStream_t)s);
  return (int)f.used++;
}

void ktime_end(stream_t s, int family, int slot, double work) {
  if (slot < 0) return;
  std::lock_guard<std::mutex> lk(g_fam_mu);
  Family& f = g_fam[family];
  cudaEventRecord(f.ev[slot].second, (cudaStream_t)s);
  f.work += work;
}

void kernel_time(int family, double* ms, int64_t* n, double* work) {
  std::lock_guard<std::mutex> lk(g_fam_mu);
  double tot = 0.0;
  Family& f = g_fam[family < 0 || family >= KT_FAMILIES ? 0 : family];
  for (size_t i = 0; i < f.used; ++i) {
    cudaEventSynchronize(f.ev[i].second);
    float t = 0.f;
    cudaEventElapsedTime(&t, f.ev[i].first, f.ev[i].second);
    tot += t;
  }
  if (ms) *ms = tot;
  if (n) *n = (int64_t)f.used;
  if (work) *work = f.work;
  f.used = 0;
  f.work = 0.0;
}

void gemm_time(double* ms, int64_t* n, double* flops) { kernel_time(KT_DGEMM, ms, n, flops); }

// ---- autotuner table (ecg_tune.h) ----------------------------------------
namespace {
std::mutex g_tune_mu;
std::map<std::string, int> g_tune;
std::atomic<bool> g_tuning{false};
}  // namespace

void set_tuning(bool on) { g_tuning.store(on); }
bool tuning() { return g_tuning.load(); }
bool stream_capturing(stream_t s) { return capturing((cudaStream_t)s); }

bool tune_get(const std::string& key, int* value) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(key);
  if (it == g_tune.end()) return false;
  *value = it->second;
  return true;
}

void tune_put(const std::string& key, int value) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = value;
}

size_t tune_size() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  return g_tune.size();
}

std::string tune_dump() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  std::string out;
  for (auto& kv : g_tune) out += kv.first + " " + std::to_string(kv.second) + "\n";
  return out;
}

int tune_parse(const std::string& text) {
  std::map<std::string, int> add;
  size_t pos = 0;
  while (pos < text.size()) {
    size_t end = text.find('\n', pos);
    if (end == std::string::npos) end = text.size();
    const std::string line = text.substr(pos, end - pos);
    pos = end + 1;
    if (line.empty() || line[0] == '#') continue;
    const size_t sp = line.rfind(' ');
    if (sp == std::string::npos || sp == 0) return -1;
    char* e = nullptr;
    const long v = std::strtol(line.c_str() + sp + 1, &e, 10);
    if (!e || *e != '\0') return -1;
    add[line.substr(0, sp)] = (int)v;
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (auto& kv : add) g_tune[kv.first] = kv.second;
  return (int)add.size();
}

int tune_pick(stream_t s, int ncand, const std::function<int(int)>& run, const TuneOut& out) {
  cudaStream_t st = (cudaStream_t)s;
  void* save = nullptr;
  const size_t bytes = (size_t)out.rows_bytes * (size_t)out.ncols;
  if (cudaMalloc(&save, bytes ? bytes : 16) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  auto copy = [&](bool restore) {
    if (restore)
      return cudaMemcpy2DAsync(out.C, out.ldc_bytes, save, out.rows_bytes, out.rows_bytes,
                               out.ncols, cudaMemcpyDeviceToDevice, st);
    return cudaMemcpy2DAsync(save, out.rows_bytes, out.C, out.ldc_bytes, out.rows_bytes,
                             out.ncols, cudaMemcpyDeviceToDevice, st);
  };
  int best = -1;
  float best_ms = 0.f;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  if (copy(false) == cudaSuccess) {
    for (int i = 0; i < ncand; ++i) {
      float ms = 0.f;
      bool ok = run(i) == 0;  // warm-up run (first use of the configuration)
      ok = ok && copy(true) == cudaSuccess;
      ok = ok && cudaEventRecord(a, st) == cudaSuccess;
      ok = ok && run(i) == 0;
      ok = ok && cudaEventRecord(b, st) == cudaSuccess;
      ok = ok && cudaEventSynchronize(b) == cudaSuccess;
      ok = ok && cudaEventElapsedTime(&ms, a, b) == cudaSuccess;
      copy(true);
      if (!ok) {
        cudaGetLastError();
        continue;
      }
      if (best < 0 || ms < best_ms) {
        best = i;
        best_ms = ms;
      }
    }
  }
  cudaStreamSynchronize(st);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(save);
  return best;
}

static int gemm_launch(stream_t s, const Gemm& q);
struct PlainChoice;
static int plain_gemm(stream_t s, const GemmArgs& g, const Gemm& q);

int gemm_strided(stream_t s, const Gemm& q) {
  if (!g_timing || q.m <= 0 || q.n <= 0 || q.batch <= 0 || q.k <= 0) return gemm_launch(s, q);
  const int slot = ktime_begin(s, KT_DGEMM);
  int r = gemm_launch(s, q);
  ktime_end(s, KT_DGEMM, slot, 2.0 * (double)q.m * (double)q.n * (double)q.k * (double)q.batch);
  return r;
}

static int gemm_launch(stream_t s, const Gemm& q) {
  if (q.m <= 0 || q.n <= 0 || q.batch <= 0) return 0;
  if ((q.n + 63) / 64 > 65535 && (q.m + 63) / 64 <= 65535 && q.kseg == 0 && q.dn == 0 &&
      !q.ptab) {
    // more column tiles than the grid's y extent: C^T = B^T A^T puts the long
    // dimension on the grid's x axis
    Gemm t = q;
    t.m = q.n;
    t.n = q.m;
    t.A = q.B;
    t.sam = q.sbn;
    t.sak = q.sbk;
    t.sab = q.sbb;
    t.B = q.A;
    t.sbk = q.sak;
    t.sbn = q.sam;
    t.sbb = q.sab;
    t.scm = q.scn;
    t.scn = q.scm;
    return gemm_launch(s, t);
  }
  cudaStream_t st = (cudaStream_t)s;
  if (q.k <= 0 || q.alpha == 0.0) {
    // empty contraction: C = beta C
    if (q.beta == 1.0) return 0;
    for (int64_t b = 0; b < q.batch; ++b) {
      double* Cb = q.C + b * q.scb;
      int e = 0;
      if (q.scm == 1)
        e = geam(s, q.m, q.n, 0.0, Cb, q.scn, q.beta, Cb, q.scn);
      else if (q.scn == 1)
        e = geam(s, q.n, q.m, 0.0, Cb, q.scm, q.beta, Cb, q.scm);
      else
        for (int64_t j = 0; j < q.n && !e; ++j)
          for (int64_t i = 0; i < q.m && !e; ++i) {
            double* p = Cb + j * q.scn + i * q.scm;
            e = axpby(s, 1, 0.0, p, q.beta, p);
          }
      if (e) return e;
    }
    return 0;
  }
  GemmArgs g{q.A, q.B, q.C, q.m, q.n, q.k, q.sam, q.sak, q.sab, q.sbk, q.sbn, q.sbb,
             q.scm, q.scn, q.scb, q.alpha, q.beta, (q.sam != 1 && q.sak == 1) ? 1 : 0,
             (q.sbk != 1 && q.sbn == 1) ? 1 : 0, 0};
  const int flags = (q.kseg > 0 ? GF_SEG : 0) | (q.dn > 0 ? GF_DN : 0) | (q.ptab ? GF_PTAB : 0);
  if (q.mapped_tma && (flags & ~GF_DN) == 0 && dgemm_tma_usable_mapped(q)) {
    const int e = dgemm_tma(s, q, 0, 1);
    if (e != -1) return e;
  }
  if (flags) {
    if ((!q.ptab && q.batch != 1) || (q.kseg > 0 && (q.kseg >= q.k || !q.A1 || !q.B1)))
      return (int)cudaErrorInvalidValue;
    g.dn = q.dn;
    g.scn2 = q.scn2;
    g.kseg = q.kseg;
    g.A1 = q.A1;
    g.sak1 = q.sak1;
    g.B1 = q.B1;
    g.sbk1 = q.sbk1;
    g.ptab = q.ptab;
    const int64_t nb = q.batch;
    switch (flags) {
      case GF_SEG: return launch_gemm<64, 64, 16, 32, 32, 3, 3, 0, GF_SEG>(g, nb, st);
      case GF_DN: return launch_gemm<64, 64, 16, 32, 32, 3, 3, 0, GF_DN>(g, nb, st);
      case GF_SEG | GF_DN:
        return launch_gemm<64, 64, 16, 32, 32, 3, 3, 0, GF_SEG | GF_DN>(g, nb, st);
      case GF_PTAB: return launch_gemm<64, 64, 16, 32, 32, 3, 3, 0, GF_PTAB>(g, nb, st);
      case GF_PTAB | GF_SEG:
        return launch_gemm<64, 64, 16, 32, 32, 3, 3, 0, GF_PTAB | GF_SEG>(g, nb, st);
      case GF_PTAB | GF_DN:
        return launch_gemm<64, 64, 16, 32, 32, 3, 3, 0, GF_PTAB | GF_DN>(g, nb, st);
      default:
        return launch_gemm<64, 64, 16, 32, 32, 3, 3, 0, GF_PTAB | GF_SEG | GF_DN>(g, nb, st);
    }
  }
  return plain_gemm(s, g, q);
}

// Plain GEMM configurations: cp.async-staged tiles (cfg 0: 64x64, warps
// 32x32, 3 CTAs per SM; 1: 128x64, warps 64x32, 2 CTAs; 2: 64x128, warps
// 32x64, 2 CTAs) or TMA-staged tiles (cfg CFG_TMA + c: dgemm_tma configuration
// c), and the split-K count S (> 1: K slices whose partial products a
// fixed-order reduction sums; cp.async split-K runs cfg 0's tile).
constexpr int CFG_TMA = 4;
struct PlainChoice {
  int cfg, S;
};

// The fixed rule: 64x64 tiles, TMA-staged where TMA can address both operands
// (15-20% faster than cp.async staging on every CCSD shape measured on B200,
// bitwise the same results); K split when the output covers too few tiles to
// fill the SMs and K is long enough.
static PlainChoice default_plain(const Gemm& q, bool tma = true) {
  const int cfg = (tma && dgemm_tma_usable(q)) ? CFG_TMA : 0;
  const int64_t tiles64 = ((q.m + 63) / 64) * ((q.n + 63) / 64);
  if (q.batch == 1 && tiles64 < 148 && q.k >= 512) {
    int64_t S = std::min<int64_t>((2 * 148 + tiles64 - 1) / tiles64, q.k / 256);
    return PlainChoice{cfg, (int)std::max<int64_t>(2, std::min<int64_t>(S, 64))};
  }
  return PlainChoice{cfg, 1};
}

static int launch_plain(stream_t s, const GemmArgs& g, const Gemm& q, PlainChoice c) {
  cudaStream_t st = (cudaStream_t)s;
  if (c.cfg >= CFG_TMA) {
    const int e = dgemm_tma(s, q, c.cfg - CFG_TMA, c.S);
    if (e != -1) return e;
    c = default_plain(q, false);  // TMA cannot address an operand
  }
  if (c.S > 1 && q.batch == 1) {
    int64_t kc = (q.k + c.S - 1) / c.S;
    kc = (kc + 15) / 16 * 16;
    const int64_t S = (q.k + kc - 1) / kc;
    double* P = splitk_buffer(s, (size_t)S * q.m * q.n);
    if (!P) return (int)cudaErrorMemoryAllocation;
    GemmArgs h = g;
    h.k = kc;
    h.klast = q.k - (S - 1) * kc;
    h.sab = kc * q.sak;
    h.sbb = kc * q.sbk;
    h.C = P;
    h.scm = 1;
    h.scn = q.m;
    h.scb = q.m * q.n;
    h.alpha = 1.0;
    h.beta = 0.0;
    int e = launch_gemm<64, 64, 16, 32, 32, 3, 3>(h, S, st);
    if (e) return e;
    launch_reduce(st, q.m, q.n, (int)S, P, q.alpha, q.beta, q.C, q.scm, q.scn);
    return launched();
  }
  switch (c.cfg) {
    case 1: return launch_gemm<128, 64, 16, 64, 32, 3, 2>(g, q.batch, st);
    case 2: return launch_gemm<64, 128, 16, 32, 64, 3, 2>(g, q.batch, st);
    default: return launch_gemm<64, 64, 16, 32, 32, 3, 3>(g, q.batch, st);
  }
}

static int plain_gemm(stream_t s, const GemmArgs& g, const Gemm& q) {
  PlainChoice c = default_plain(q);
  const std::string key = "dgemmt " + std::to_string(q.m) + " " + std::to_string(q.n) + " " +
                          std::to_string(q.k) + " " + std::to_string(q.batch) + " " +
                          std::to_string(g.a_kfast) + std::to_string(g.b_nfast);
  int enc = 0;
  if (tune_get(key, &enc)) {
    c = PlainChoice{enc % 8, enc / 8};
  } else if (tuning() && q.scm == 1 && !capturing((cudaStream_t)s)) {
    std::vector<PlainChoice> cand = {{0, 1}, {1, 1}, {2, 1}};
    const bool tma = dgemm_tma_usable(q);
    if (tma)
      for (int t = 0; t < DTMA_CONFIGS; ++t) cand.push_back({CFG_TMA + t, 1});
    const PlainChoice d = default_plain(q, false);
    if (q.batch == 1 && q.k >= 512) {
      // split counts around the rule's and the small ones that round the
      // CTA count up to whole waves; long contractions also try the
      // 128x128 TMA tile split
      for (int S : {d.S, 2 * d.S, d.S / 2, 2, 3, 4, 6, 8, 12, 16})
        if (S >= 2 && S <= 64 && q.k / S >= 64) {
          auto add = [&](int cfg) {
            for (auto& x : cand)
              if (x.S == S && x.cfg == cfg) return;
            cand.push_back({cfg, S});
          };
          add(0);
          if (tma) add(CFG_TMA);
          if (tma && q.k >= 4096) add(CFG_TMA + 3);
        }
    }
    // tune_pick restores the output region it is given: the m x n columns of
    // C, for batch > 1 the n*batch columns of items stored back to back
    // (other batched layouts are not tuned)
    if (q.batch == 1 || q.scb == q.scn * q.n) {
      const TuneOut out{q.C, q.m * 8, q.n * q.batch, q.scn * 8};
      const int best = tune_pick(
          s, (int)cand.size(), [&](int i) { return launch_plain(s, g, q, cand[i]); }, out);
      if (best >= 0) {
        c = cand[best];
        tune_put(key, c.S * 8 + c.cfg);
      }
    }
  }
  return launch_plain(s, g, q, c);
}

int gemm(stream_t s, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
         const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
         int64_t ldc, int64_t batch, int64_t sa, int64_t sb, int64_t sc) {
  Gemm q;
  q.m = m; q.n = n; q.k = k; q.batch = batch; q.alpha = alpha; q.beta = beta;
  q.A = A; q.B = B; q.C = C;
  bool at = (ta == 'T' || ta == 't'), bt = (tb == 'T' || tb == 't');
  q.sam = at ? lda : 1; q.sak = at ? 1 : lda; q.sab = sa;
  q.sbk = bt ? ldb : 1; q.sbn = bt ? 1 : ldb; q.sbb = sb;
  q.scm = 1; q.scn = ldc; q.scb = sc;
  return gemm_strided(s, q);
}

// ---------------------------------------------------------------- permute

struct PermArgs {
  int nd;
  int64_t odim[8];   // out dims
  int64_t istr[8];   // in stride of out dim d
  int64_t ostr[8];   // out stride of out dim d
  int q;             // out dim that is the in-fastest dim (perm[q] == 0)
  int64_t total;
  double alpha, beta;
  const double* in;
  double* out;
};

// Index arithmetic of the permutation kernels runs in IT (32-bit unsigned
// whenever the element count allows it: a 64-bit division by a run-time value
// costs several times the instructions of a 32-bit one, and at a few divisions
// per element it, not memory, bounded these kernels); offsets stay 64-bit.

// Plain elementwise permutation (out-fastest index also drives the input
// fastest or the tensor is small): one thread per output element.
template <typename IT>
__global__ void permute_plain_kernel(PermArgs p) {
  const IT total = (IT)p.total;
  for (IT idx = blockIdx.x * (IT)blockDim.x + threadIdx.x; idx < total;
       idx += (IT)gridDim.x * blockDim.x) {
    IT r = idx;
    int64_t off = 0;
#pragma unroll 8
    for (int d = 0; d < p.nd; ++d) {
      const IT od = (IT)p.odim[d];
      const IT x = r % od;
      r /= od;
      off += (int64_t)x * p.istr[d];
    }
    double v = p.alpha * p.in[off];
    if (p.beta != 0.0) v += p.beta * p.out[idx];
    p.out[idx] = v;
  }
}

// Permutation that keeps the fastest index (out dim 0 = in dim 0, stride 1 on
// both sides): one warp per row of out dim 0, the row's offsets computed once
// and its elements copied with coalesced loads and stores.
template <typename IT>
__global__ void permute_rows_kernel(PermArgs p) {
  const IT rows = (IT)(p.total / p.odim[0]);
  const int64_t n0 = p.odim[0];
  const int lane = threadIdx.x & 31;
  const IT nwarp = (IT)gridDim.x * (blockDim.x >> 5);
  for (IT row = blockIdx.x * (IT)(blockDim.x >> 5) + (threadIdx.x >> 5); row < rows;
       row += nwarp) {
    IT r = row;
    int64_t ioff = 0;
    for (int d = 1; d < p.nd; ++d) {
      const IT od = (IT)p.odim[d];
      const IT x = r % od;
      r /= od;
      ioff += (int64_t)x * p.istr[d];
    }
    const double* in = p.in + ioff;
    double* out = p.out + (int64_t)row * n0;
    for (int64_t x = lane; x < n0; x += 32) {
      double v = p.alpha * in[x];
      if (p.beta != 0.0) v += p.beta * out[x];
      out[x] = v;
    }
  }
}

// Tiled permutation: 32x32 tiles spanning out dim 0 (written contiguously)
// and out dim q (read contiguously); all other dims enumerate tiles.
template <typename IT>
__global__ void permute_tiled_kernel(PermArgs p, IT tiles0, IT tilesq, IT rest) {
  __shared__ double tile[32][33];
  const IT ntile = tiles0 * tilesq * rest;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (IT t = blockIdx.x; t < ntile; t += gridDim.x) {
    const IT t0 = t % tiles0;
    const IT tq = (t / tiles0) % tilesq;
    IT r = t / (tiles0 * tilesq);
    int64_t ibase = 0, obase = 0;
    for (int d = 1; d < p.nd; ++d) {
      if (d == p.q) continue;
      const IT od = (IT)p.odim[d];
      const IT x = r % od;
      r /= od;
      ibase += (int64_t)x * p.istr[d];
      obase += (int64_t)x * p.ostr[d];
    }
    const int64_t x0b = (int64_t)t0 * 32, xqb = (int64_t)tq * 32;
    // read: contiguous along q (input fastest); the four loads of a thread
    // are issued before any of them is used
    double ld[4];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int64_t x0 = x0b + ty + 8 * jj, xq = xqb + tx;
      ld[jj] = (x0 < p.odim[0] && xq < p.odim[p.q])
                   ? p.in[ibase + x0 * p.istr[0] + xq * p.istr[p.q]] : 0.0;
    }
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) tile[ty + 8 * jj][tx] = ld[jj];
    __syncthreads();
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int j = ty + 8 * jj;
      const int64_t x0 = x0b + tx, xq = xqb + j;
      if (x0 < p.odim[0] && xq < p.odim[p.q]) {
        int64_t o = obase + x0 + xq * p.ostr[p.q];
        double v = p.alpha * tile[tx][j];
        if (p.beta != 0.0) v += p.beta * p.out[o];
        p.out[o] = v;
      }
    }
    __syncthreads();
  }
}

int permute(stream_t s, int nd, const int64_t* in_dims, const int* perm, double alpha,
            const double* in, double beta, double* out) {
  if (nd < 1 || nd > 8) return (int)cudaErrorInvalidValue;
  PermArgs p{};
  p.nd = nd;
  int64_t istride[8];
  istride[0] = 1;
  for (int d = 1; d < nd; ++d) istride[d] = istride[d - 1] * in_dims[d - 1];
  p.total = 1;
  for (int d = 0; d < nd; ++d) {
    p.odim[d] = in_dims[perm[d]];
    p.istr[d] = istride[perm[d]];
    p.ostr[d] = p.total;
    p.total *= p.odim[d];
    if (perm[d] == 0) p.q = d;
  }
  if (p.total == 0) return 0;
  p.alpha = alpha;
  p.beta = beta;
  p.in = in;
  p.out = out;
  cudaStream_t st = (cudaStream_t)s;
  // 32-bit index arithmetic while every index (element, row, tile) fits
  const bool small = p.total < ((int64_t)1 << 32) - 256 * 148 * 16;
  if (p.q == 0 && p.odim[0] >= 32) {
    const int64_t rows = p.total / p.odim[0];
    int64_t blocks = (rows + 7) / 8;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (small)
      permute_rows_kernel<uint32_t><<<(unsigned)blocks, 256, 0, st>>>(p);
    else
      permute_rows_kernel<uint64_t><<<(unsigned)blocks, 256, 0, st>>>(p);
  } else if (p.q == 0 || p.odim[0] < 8 || p.odim[p.q] < 8) {
    int64_t blocks = (p.total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (small)
      permute_plain_kernel<uint32_t><<<(unsigned)blocks, 256, 0, st>>>(p);
    else
      permute_plain_kernel<uint64_t><<<(unsigned)blocks, 256, 0, st>>>(p);
  } else {
    int64_t t0 = (p.odim[0] + 31) / 32, tq = (p.odim[p.q] + 31) / 32;
    int64_t rest = p.total / (p.odim[0] * p.odim[p.q]);
    int64_t blocks = t0 * tq * rest;
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (small)
      permute_tiled_kernel<uint32_t><<<(unsigned)blocks, dim3(32, 8), 0, st>>>(
          p, (uint32_t)t0, (uint32_t)tq, (uint32_t)rest);
    else
      permute_tiled_kernel<uint64_t><<<(unsigned)blocks, dim3(32, 8), 0, st>>>(
          p, (uint64_t)t0, (uint64_t)tq, (uint64_t)rest);
  }
  return launched();
}

// ---------------------------------------------------------------- elementwise

__global__ void axpby_kernel(int64_t n, double alpha, const double* x, double beta, double* y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double v = alpha * x[i];
    if (beta != 0.0) v += beta * y[i];
    y[i] = v;
  }
}

static unsigned grid_for(int64_t n, int threads, int64_t cap) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (unsigned)b;
}

__global__ void to_f32_kernel(int64_t n, const double* __restrict__ x, float* __restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = (float)x[i];
}

int to_f32(stream_t s, int64_t n, const double* x, float* y) {
  if (n <= 0) return 0;
  to_f32_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, (cudaStream_t)s>>>(n, x, y);
  return launched();
}

__global__ void to_f32_pairs_kernel(int64_t n, const double* __restrict__ a,
                                    const double* __restrict__ b, float2* __restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = make_float2((float)a[i], (float)b[i]);
}

int to_f32_pairs(stream_t s, int64_t n, const double* a, const double* b, void* out) {
  if (n <= 0) return 0;
  to_f32_pairs_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, (cudaStream_t)s>>>(
      n, a, b, reinterpret_cast<float2*>(out));
  return launched();
}

// exponent field all ones: infinity or NaN
__global__ void nonfinite_kernel(int64_t n, const double* __restrict__ x, double* flag) {
  bool bad = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    bad |= ((__double_as_longlong(x[i]) >> 52) & 0x7ff) == 0x7ff;
  if (__syncthreads_or(bad) && threadIdx.x == 0) *flag = 1.0;
}

int nonfinite(stream_t s, int64_t n, const double* x, double* flag) {
  cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(double), (cudaStream_t)s);
  if (e != cudaSuccess) return (int)e;
  if (n <= 0) return 0;
  nonfinite_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, (cudaStream_t)s>>>(n, x, flag);
  return launched();
}

int axpby(stream_t s, int64_t n, double alpha, const double* x, double beta, double* y) {
  if (n <= 0) return 0;
  axpby_kernel<<<grid_for(n), 256, 0, (cudaStream_t)s>>>(n, alpha, x, beta, y);
  return launched();
}

__global__ void strided_sum_kernel(int64_t nb, int64_t sb, int64_t nk, int64_t sk, double alpha,
                                   const double* in, double beta, double* out) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nb;
       b += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int64_t k = 0; k < nk; ++k) acc += in[b * sb + k * sk];
    double v = alpha * acc;
    if (beta != 0.0) v += beta * out[b];
    out[b] = v;
  }
}

int strided_sum(stream_t s, int64_t nb, int64_t sb, int64_t nk, int64_t sk, double alpha,
                const double* in, double beta, double* out) {
  if (nb <= 0) return 0;
  strided_sum_kernel<<<grid_for(nb), 256, 0, (cudaStream_t)s>>>(nb, sb, nk, sk, alpha, in, beta,
                                                                 out);
  return launched();
}

__global__ void update_doubles_kernel(int nv, int no, const double* eo, const double* ev,
                                      double shift, const double* R, double* T) {
  const int64_t n = (int64_t)nv * nv * no * no;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int a = (int)(idx % nv);
    int b = (int)((idx / nv) % nv);
    int i = (int)((idx / ((int64_t)nv * nv)) % no);
    int j = (int)(idx / ((int64_t)nv * nv * no));
    T[idx] -= R[idx] / (ev[a] + ev[b] - eo[i] - eo[j] + shift);
  }
}

__global__ void update_singles_kernel(int nv, int no, const double* eo, const double* ev,
                                      double shift, const double* R, double* T) {
  const int64_t n = (int64_t)nv * no;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int a = (int)(idx % nv);
    int i = (int)(idx / nv);
    T[idx] -= R[idx] / (ev[a] - eo[i] + shift);
  }
}

int update_doubles(stream_t s, int nv, int no, const double* eo, const double* ev, double shift,
                   const double* R, double* T) {
  int64_t n = (int64_t)nv * nv * no * no;
  if (n <= 0) return 0;
  update_doubles_kernel<<<grid_for(n), 256, 0, (cudaStream_t)s>>>(nv, no, eo, ev, shift, R, T);
  return launched();
}
int update_singles(stream_t s, int nv, int no, const double* eo, const double* ev, double shift,
                   const double* R, double* T) {
  int64_t n = (int64_t)nv * no;
  if (n <= 0) return 0;
  update_singles_kernel<<<grid_for(n), 256, 0, (cudaStream_t)s>>>(nv, no, eo, ev, shift, R, T);
  return launched();
}

// ---------------------------------------------------------------- reductions
//
// Fixed grid (RED_BLOCKS x 256) + a single-block final pass in a fixed order:
// results are bitwise reproducible run to run.

static constexpr int RED_BLOCKS = 592;
int64_t reduce_scratch_len() { return 2 * RED_BLOCKS; }

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = (l < (int)(blockDim.x >> 5)) ? sh[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;
}

__global__ void dot_partial_kernel(int64_t n, const double* x, const double* y, double* part) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    acc += x[i] * y[i];
  double r = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

// Partial sums of <X|Y> and <X^T|Y> (X^T[a,b,i,j] = X[b,a,i,j]) over 32 x 32
// tiles of each (a,b) slice: the block reads the tile of X and Y and the
// mirrored tile of X, all coalesced, and takes the transposed elements from
// shared memory.  Tiles go to blocks in a fixed order, so the sums are
// deterministic.
__global__ void cs_dot_partial_kernel(int nv, int no, const double* X, const double* Y,
                                      double* part) {
  __shared__ double sh[32];
  __shared__ double xt[32][33];
  const int64_t vv = (int64_t)nv * nv;
  const uint32_t T = (uint32_t)(nv + 31) / 32, ntile = T * T * (uint32_t)no * (uint32_t)no;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  double d = 0.0, ex = 0.0;
  for (uint32_t t = blockIdx.x; t < ntile; t += gridDim.x) {
    const uint32_t ta = t % T, tb = (t / T) % T, ij = t / (T * T);
    const double* Xs = X + ij * vv;
    const double* Ys = Y + ij * vv;
    const int a0 = ta * 32, b0 = tb * 32;
    // all twelve loads of a thread are issued before any of them is used:
    // xt[j][tx] = X[b0 + tx, a0 + j], and X, Y at (a0 + tx, b0 + j)
    double rt[4], rx[4], ry[4];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int j = ty + 8 * jj, a = a0 + tx, b = b0 + j;
      rt[jj] = (b0 + tx < nv && a0 + j < nv) ? Xs[(b0 + tx) + (int64_t)nv * (a0 + j)] : 0.0;
      const bool in = a < nv && b < nv;
      const int64_t i = a + (int64_t)nv * b;
      rx[jj] = in ? Xs[i] : 0.0;
      ry[jj] = in ? Ys[i] : 0.0;
    }
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) xt[ty + 8 * jj][tx] = rt[jj];
    __syncthreads();
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      d += rx[jj] * ry[jj];
      ex += xt[tx][ty + 8 * jj] * ry[jj];  // X[b, a]
    }
    __syncthreads();
  }
  double r0 = block_sum(d, sh);
  double r1 = block_sum(ex, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = r0;
    part[RED_BLOCKS + blockIdx.x] = r1;
  }
}

__global__ void final_sum_kernel(int nparts, int nout, const double* part, double* out) {
  __shared__ double sh[32];
  for (int o = 0; o < nout; ++o) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += part[o * RED_BLOCKS + i];
    double r = block_sum(acc, sh);
    if (threadIdx.x == 0) out[o] = r;
  }
}

int dot(stream_t s, int64_t n, const double* x, const double* y, double* scratch, double* out) {
  cudaStream_t st = (cudaStream_t)s;
  dot_partial_kernel<<<RED_BLOCKS, 256, 0, st>>>(n, x, y, scratch);
  int e = launched();
  if (e) return e;
  final_sum_kernel<<<1, 256, 0, st>>>(RED_BLOCKS, 1, scratch, out);
  return launched();
}

int cs_dot(stream_t s, int nv, int no, const double* X, const double* Y, double* scratch,
           double* out) {
  cudaStream_t st = (cudaStream_t)s;
  const uint64_t T = ((uint64_t)nv + 31) / 32;
  if (T * T * (uint64_t)no * (uint64_t)no >= ((uint64_t)1 << 32) - RED_BLOCKS)
    return (int)cudaErrorInvalidValue;  // tile index beyond 32 bits
  cs_dot_partial_kernel<<<RED_BLOCKS, 256, 0, st>>>(nv, no, X, Y, scratch);
  int e = launched();
  if (e) return e;
  final_sum_kernel<<<1, 256, 0, st>>>(RED_BLOCKS, 2, scratch, out);
  return launched();
}

__global__ void geam_kernel(int64_t m, int64_t n, double alpha, const double* A, int64_t lda,
                            double beta, double* C, int64_t ldc) {
  const int64_t total = m * n;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int64_t i = idx % m, j = idx / m;
    double v = alpha * A[i + j * lda];
    if (beta != 0.0) v += beta * C[i + j * ldc];
    C[i + j * ldc] = v;
  }
}

int geam(stream_t s, int64_t m, int64_t n, double alpha, const double* A, int64_t lda,
         double beta, double* C, int64_t ldc) {
  if (m <= 0 || n <= 0) return 0;
  geam_kernel<<<grid_for(m * n), 256, 0, (cudaStream_t)s>>>(m, n, alpha, A, lda, beta, C, ldc);
  return launched();
}

__global__ void outer_kernel(int64_t na, int64_t ni, int64_t nb, int64_t nj, double alpha,
                             const double* X, const double* Y, double beta, double* out) {
  const int64_t total = na * nb * ni * nj;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int64_t a = idx % na, b = (idx / na) % nb, i = (idx / (na * nb)) % ni, j = idx / (na * nb * ni);
    double v = alpha * X[a + i * na] * Y[b + j * nb];
    if (beta != 0.0) v += beta * out[idx];
    out[idx] = v;
  }
}

int outer(stream_t s, int64_t na, int64_t ni, int64_t nb, int64_t nj, double alpha,
          const double* X, const double* Y, double beta, double* out) {
  int64_t total = na * nb * ni * nj;
  if (total <= 0) return 0;
  outer_kernel<<<grid_for(total), 256, 0, (cudaStream_t)s>>>(na, ni, nb, nj, alpha, X, Y, beta,
                                                              out);
  return launched();
}

struct CombineArgs {
  const double* X[8];
};

__global__ void combine_kernel(int64_t n, int m, CombineArgs a, const double* coef, double* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double v = coef[0] * a.X[0][i];
    for (int k = 1; k < m; ++k) v += coef[k] * a.X[k][i];
    out[i] = v;
  }
}

int combine(stream_t s, int64_t n, int m, const double* const* X, const double* coef,
            double* out) {
  if (m < 1 || m > 8) return (int)cudaErrorInvalidValue;
  if (n <= 0) return 0;
  CombineArgs a{};
  for (int k = 0; k < m; ++k) a.X[k] = X[k];
  combine_kernel<<<grid_for(n), 256, 0, (cudaStream_t)s>>>(n, m, a, coef, out);
  return launched();
}

// ---------------------------------------------------------------- ladder

__global__ void ladder_pack_t_kernel(int nv, int no, const double* __restrict__ T,
                                     const int2* __restrict__ cdp, const int2* __restrict__ ijp,
                                     double* __restrict__ Ts, double* __restrict__ Ta,
                                     int64_t ldp, int64_t ldm) {
  const int64_t v = nv, o = no, ncdp = v * (v + 1) / 2;
  const int64_t nijp = o * (o + 1) / 2, total = ncdp * nijp;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = idx % ncdp, q = idx / ncdp;
    const int2 cd = cdp[k], ij = ijp[q];
    const int64_t ij0 = v * v * (ij.x + o * ij.y);
    const double x = T[cd.x + v * cd.y + ij0], y = T[cd.y + v * cd.x + ij0];
    Ts[k + ldp * q] = 0.5 * (x + y);
    if (cd.x < cd.y && ij.x < ij.y) Ta[(k - cd.y) + ldm * (q - ij.y)] = 0.5 * (x - y);
  }
}

int ladder_pack_t(stream_t s, int nv, int no, const double* T2, const int* cdp, const int* ijp,
                  double* Ts, double* Ta, int64_t ldp, int64_t ldm) {
  int64_t total = (int64_t)nv * (nv + 1) / 2 * ((int64_t)no * (no + 1) / 2);
  ladder_pack_t_kernel<<<grid_for(total), 256, 0, (cudaStream_t)s>>>(
      nv, no, T2, (const int2*)cdp, (const int2*)ijp, Ts, Ta, ldp, ldm);
  return launched();
}

// One thread per element; the tiled kernel below replaces it wherever its
// tile count fits 32 bits (always, for blocks that fit in device memory).
// IT: index type of the element loop.
template <typename IT>
__global__ void ladder_pack_v_kernel(int nv, int a0, int na, int npairs,
                                     const int2* __restrict__ pairs, const int2* __restrict__ cdp,
                                     const double* __restrict__ V, double* __restrict__ Vp,
                                     double* __restrict__ Vm, int64_t ldp, int64_t ldm) {
  const int64_t v = nv;
  const IT ncdp = (IT)(v * (v + 1) / 2), total = ncdp * (IT)npairs;
  const int64_t lda = v * na;  // Vblk[c + v a' + v na (d + v b'')]
  for (IT idx = blockIdx.x * (IT)blockDim.x + threadIdx.x; idx < total;
       idx += (IT)gridDim.x * blockDim.x) {
    const int64_t k = idx % ncdp, pr = idx / ncdp;
    const int2 cd = cdp[k], ab = pairs[pr];
    const int64_t ap = ab.x - a0, bp = ab.y - a0;
    const double x = V[cd.x + v * ap + lda * (cd.y + v * bp)];
    const double y = V[cd.y + v * ap + lda * (cd.x + v * bp)];
    Vp[k + ldp * pr] = (cd.x == cd.y) ? x : x + y;
    if (cd.x < cd.y && ab.x < ab.y) Vm[(k - cd.y) + ldm * (pr - ap - 1)] = x - y;
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

// The same packing by 32 x 32 tiles of (c, d), c0 <= d0, one pair (a, b) per
// tile: X[c,d] = V[c + v a' + lda (d + v b')] is read along c, the mirrored
// X[d,c] along d into shared memory, so every load and store is coalesced
// (the element kernel gathers X[d,c] with stride lda).  Block 32 x 8.
__global__ void ladder_pack_v_tiled_kernel(int nv, int a0, int na, int npairs,
                                           const int2* __restrict__ pairs,
                                           const double* __restrict__ V,
                                           double* __restrict__ Vp, double* __restrict__ Vm,
                                           int64_t ldp, int64_t ldm) {
  __shared__ double ys[32][33];
  const int v = nv;
  const int64_t lda = (int64_t)v * na;
  const uint32_t T = (uint32_t)(v + 31) / 32, NT = T * (T + 1) / 2;
  const uint32_t total = NT * (uint32_t)npairs;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t pr = t / NT;
    uint32_t tc, td;
    tri_tile(t - pr * NT, tc, td);
    const int c0 = (int)tc * 32, d0 = (int)td * 32;
    const int2 ab = pairs[pr];
    const int64_t ap = ab.x - a0, bp = ab.y - a0;
    const double* X = V + v * ap + lda * v * bp;  // X[c,d] = X[c + lda d]
    double xr[4], yr[4];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int d = d0 + ty + 8 * jj, c = c0 + tx;
      xr[jj] = (d < v && c <= d) ? X[c + lda * d] : 0.0;
      const int cm = c0 + ty + 8 * jj, dm = d0 + tx;  // X[dm, cm] for (c, d) = (cm, dm)
      yr[jj] = (cm < v && dm < v) ? X[dm + lda * cm] : 0.0;
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
        Vp[k + ldp * pr] = (c == d) ? x : x + y;
        if (c < d && ab.x < ab.y) Vm[(k - d) + ldm * ((int64_t)pr - ap - 1)] = x - y;
      }
    }
    __syncthreads();
  }
}

int ladder_pack_v(stream_t s, int nv, int a0, int na, int npairs, const int* pairs,
                  const int* cdp, const double* Vblk, double* Vp, double* Vm, int64_t ldp,
                  int64_t ldm) {
  const int64_t T = (nv + 31) / 32, tiles = T * (T + 1) / 2 * npairs;
  if (tiles < ((int64_t)1 << 32) - 148 * 16) {
    const unsigned g = (unsigned)std::min<int64_t>(tiles, 148 * 16);
    ladder_pack_v_tiled_kernel<<<g, dim3(32, 8), 0, (cudaStream_t)s>>>(
        nv, a0, na, npairs, (const int2*)pairs, Vblk, Vp, Vm, ldp, ldm);
  } else {
    const int64_t total = (int64_t)nv * (nv + 1) / 2 * npairs;
    ladder_pack_v_kernel<uint64_t><<<grid_for(total), 256, 0, (cudaStream_t)s>>>(
        nv, a0, na, npairs, (const int2*)pairs, (const int2*)cdp, Vblk, Vp, Vm, ldp, ldm);
  }
  return launched();
}

__global__ void ladder_unpack_kernel(int nv, int no, int a0, int npairs,
                                     const int2* __restrict__ pairs, const int2* __restrict__ ijp,
                                     const double* __restrict__ Lp, const double* __restrict__ Lm,
                                     double* __restrict__ R2) {
  const int64_t v = nv, o = no, nijp = o * (o + 1) / 2, total = (int64_t)npairs * nijp;
  int64_t npm = 0;  // minus pairs of this block = npairs - na' where na' = #a in block
  {
    // count of a values in the block = number of pairs with a == b
    // (pairs with b == a are the first of each a); derived from the last pair
    const int2 last = pairs[npairs - 1];
    npm = npairs - (last.x - a0 + 1);
  }
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pr = idx % npairs, q = idx / npairs;
    const int2 ab = pairs[pr], ij = ijp[q];
    const double p = Lp[idx];
    double m = 0.0;
    if (ab.x < ab.y && ij.x < ij.y) m = Lm[(pr - (ab.x - a0) - 1) + npm * (q - ij.y)];
    const int64_t a = ab.x, b = ab.y, i = ij.x, j = ij.y;
    R2[a + v * b + v * v * (i + o * j)] += p + m;
    if (a != b) R2[b + v * a + v * v * (i + o * j)] += p - m;
    if (i != j) R2[a + v * b + v * v * (j + o * i)] += p - m;
    if (a != b && i != j) R2[b + v * a + v * v * (j + o * i)] += p + m;
  }
}

int ladder_unpack(stream_t s, int nv, int no, int a0, int npairs, const int* pairs,
                  const int* ijp, const double* Lp, const double* Lm, double* R2) {
  int64_t total = (int64_t)npairs * ((int64_t)no * (no + 1) / 2);
  ladder_unpack_kernel<<<grid_for(total), 256, 0, (cudaStream_t)s>>>(
      nv, no, a0, npairs, (const int2*)pairs, (const int2*)ijp, Lp, Lm, R2);
  return launched();
}

// ---------------------------------------------------------------- (T)
//
constexpr int TCUBE = 8;
constexpr int TPITCH = 9;                             // padded row pitch of a staged cube
constexpr int TCUBE_ELEMS = TCUBE * TPITCH * TPITCH;  // 648
// Staged M/N blocks, in K's precision: for each ordered position pair (x, y)
// (pair_index) and matrix w (M0 M1 M2 N0 N1 N2) the 8x8 block
// [S_x + l_x, S_y + l_y] at (l_lo, l_hi) = (l[min(x,y)], l[max(x,y)]), l_lo
// fastest: within a warp l0 varies fastest, then l1, so the reads are free of
// bank conflicts.
constexpr int TS_MAT = 6 * 6 * 64;
// Staged vectors g0 g1 g2 f0 f1 f2, in K's precision: [w][position][l].
constexpr int TS_VEC = 6 * 3 * 8;

int64_t triples_cube_count(int nv) {
  const int64_t nt = (nv + TCUBE - 1) / TCUBE;
  return nt * (nt + 1) * (nt + 2) / 6;
}

void triples_cube_table(int nv, int* tri) {
  const int nt = (nv + TCUBE - 1) / TCUBE;
  int64_t t = 0;
  for (int C = 0; C < nt; ++C)
    for (int B = 0; B <= C; ++B)
      for (int A = 0; A <= B; ++A) {
        tri[3 * t] = A;
        tri[3 * t + 1] = B;
        tri[3 * t + 2] = C;
        ++t;
      }
}

__device__ __forceinline__ int pick3(int i, int s0, int s1, int s2) {
  return i == 0 ? s0 : (i == 1 ? s1 : s2);
}

template <int BYTES>
__device__ __forceinline__ void cp_async_n(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? BYTES : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gmem), "n"(BYTES),
               "r"(sz));
}

// One block per orbit of cube triples A <= B <= C at a time.  The six cubes
// K[S_s0 + x, S_s1 + y, S_s2 + z] (s a permutation, S = 8*(A,B,C)) are staged
// in shared memory with the M/N blocks and vectors they need (all in K's
// precision; orbital energies in FP64); the loads of the next NBUF-1 orbits
// (cp.async, NBUF buffers) are in flight while the current one is evaluated,
// and the cube triple of the orbit after those is read one iteration ahead.
// Thread (x,y,z) owns the element e0 = S + (x,y,z) and its six orderings: it
// reads K at each ordering (one value per cube), forms their six X values
// with one reciprocal of the common denominator, and adds sum_e K_e X_e and
// sum_e X_e Y_e over the orderings.  Every ordered element of the orbit is
// reached |stabiliser| times (1, 2 or 6 when two or three of A, B, C
// coincide), which the weight undoes.
template <typename T, bool HAS_U>
struct EnergySmem {
  static constexpr int CUBES = 6 * TCUBE_ELEMS;
  static constexpr int r16(int b) { return (b + 15) / 16 * 16; }
  static constexpr int MAT_OFF = r16((HAS_U ? 2 : 1) * CUBES * (int)sizeof(T));
  static constexpr int VEC_OFF = MAT_OFF + r16(TS_MAT * (int)sizeof(T));
  static constexpr int EV_OFF = VEC_OFF + r16(TS_VEC * (int)sizeof(T));  // 24 doubles
  static constexpr int S_OFF = EV_OFF + 24 * 8;                          // cube origins
  static constexpr int BUF = S_OFF + 16;
  static constexpr int NBUF = (220 * 1024) / BUF < 4 ? (220 * 1024) / BUF : 4;
  static constexpr int BYTES = NBUF * BUF;
  static_assert(NBUF >= 2, "two staging buffers at least");
};

// Batch item y = blockIdx.y reads K + y*kstride (and KU), its denominator
// shift and terms from eijk_tab[y] / tt_tab[y], and
// leaves its partial sums at part[(2y + c) * gridDim.x + blockIdx.x].
template <typename T, bool HAS_U>
__global__ void __launch_bounds__(512, 1) triples_energy_kernel(
    int nv, const T* __restrict__ K, const T* __restrict__ KU, int64_t kstride,
    const double* __restrict__ eijk_tab, const double* __restrict__ ev,
    const TriplesTerms* __restrict__ tt_tab, const int* __restrict__ tri, int ntri,
    double* part) {
  using L = EnergySmem<T, HAS_U>;
  constexpr int NB = L::NBUF;
  const int y = blockIdx.y;
  K += (int64_t)y * kstride;
  if (HAS_U) KU += (int64_t)y * kstride;
  const TriplesTerms tt = tt_tab[y];
  const double eijk = eijk_tab[y];
  extern __shared__ __align__(16) unsigned char tsm_raw[];
  __shared__ double sh[32];
  const int v = nv, tid = threadIdx.x;
  const int l[3] = {tid & 7, (tid >> 3) & 7, tid >> 6};
  const int lme = l[0] + TPITCH * (l[1] + TPITCH * l[2]);
  // this thread's element in each cube of the orbit: ordering q of e0
  int koff[6];
#pragma unroll
  for (int q = 0; q < 6; ++q)
    koff[q] = q * TCUBE_ELEMS + l[perm3(q, 0)] + TPITCH * (l[perm3(q, 1)] + TPITCH * l[perm3(q, 2)]);

  // Staging roles, fixed per thread.  Threads 0..383 stage element (i, j) =
  // (l0, l1) of position pair pr = l2 of all six matrices (source row
  // S_px + i, column S_py + j); threads 384..511 stage the vectors, the
  // orbital energies and the cube origins.
  const int pr = l[2], spx = pr >> 1, spy0 = pr & 1, spy = spy0 < spx ? spy0 : spy0 + 1;
  const int mdst = pr * 6 * 64 + (spx < spy ? l[0] + 8 * l[1] : l[1] + 8 * l[0]);
  const T* msrc[6] = {(const T*)tt.M[0], (const T*)tt.M[1], (const T*)tt.M[2],
                      (const T*)tt.N[0], (const T*)tt.N[1], (const T*)tt.N[2]};
  auto vsrc = [&](int w) {
    return (const T*)(w == 0 ? tt.g[0] : w == 1 ? tt.g[1] : w == 2 ? tt.g[2] : w == 3 ? tt.f[0]
                      : w == 4 ? tt.f[1] : tt.f[2]);
  };
  const int f0 = tid - 384;

  // cp.async of orbit t (cube origins S) into buffer b (one commit group)
  auto issue = [&](int b, const int (&S)[3]) {
    unsigned char* base = tsm_raw + b * L::BUF;
    T* cK = reinterpret_cast<T*>(base);
    T* cU = cK + L::CUBES;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const int x = S[perm3(q, 0)] + l[0];
      const int y = S[perm3(q, 1)] + l[1];
      const int z = S[perm3(q, 2)] + l[2];
      const bool ok = x < v && y < v && z < v;
      const int idx = ok ? x + v * (y + v * z) : 0;
      cp_async_n<(int)sizeof(T)>(cK + q * TCUBE_ELEMS + lme, K + idx, ok);
      if (HAS_U) cp_async_n<(int)sizeof(T)>(cU + q * TCUBE_ELEMS + lme, KU + idx, ok);
    }
    if (pr < 6) {
      T* pm = reinterpret_cast<T*>(base + L::MAT_OFF);
      const int r0 = pick3(spx, S[0], S[1], S[2]) + l[0];
      const int c0 = pick3(spy, S[0], S[1], S[2]) + l[1];
      const bool ok = r0 < v && c0 < v;
      const int64_t off = ok ? r0 + (int64_t)v * c0 : 0;
#pragma unroll
      for (int w = 0; w < 6; ++w) cp_async_n<(int)sizeof(T)>(pm + mdst + w * 64, msrc[w] + off, ok);
    } else {
      T* pv = reinterpret_cast<T*>(base + L::VEC_OFF);
      // vector entries f = w*24 + pos*8 + i, f < 144
      for (int f = f0; f < TS_VEC; f += 128) {
        const int w = f / 24, pos = (f >> 3) % 3, i = f & 7;
        const int x = pick3(pos, S[0], S[1], S[2]) + i;
        const bool ok = x < v;
        cp_async_n<(int)sizeof(T)>(pv + f, vsrc(w) + (ok ? x : 0), ok);
      }
      if (f0 >= 16 && f0 < 40) {  // orbital energies: entry e = pos*8 + i
        double* pe = reinterpret_cast<double*>(base + L::EV_OFF);
        const int e = f0 - 16, pos = e >> 3, i = e & 7;
        const int x = pick3(pos, S[0], S[1], S[2]) + i;
        const bool ok = x < v;
        cp_async_n<8>(pe + e, ev + (ok ? x : 0), ok);
      } else if (f0 >= 40 && f0 < 43) {
        reinterpret_cast<int*>(base + L::S_OFF)[f0 - 40] = pick3(f0 - 40, S[0], S[1], S[2]);
      }
    }
    cp_async_commit();
  };
  // cube origins of orbit t (read ahead of their use)
  auto origins = [&](int t, int (&S)[3]) {
    if (t < ntri) {
      S[0] = tri[3 * t] * TCUBE;
      S[1] = tri[3 * t + 1] * TCUBE;
      S[2] = tri[3 * t + 2] * TCUBE;
    }
  };

  double eK = 0.0, eY = 0.0;
  // prologue: orbits u = 0 .. NB-2 of this block into buffers u (an empty
  // group for a missing orbit keeps the group count in step)
  int ti = blockIdx.x;  // next orbit to issue
  int nS[3] = {0, 0, 0};
  origins(ti, nS);
#pragma unroll 1
  for (int u = 0; u < NB - 1; ++u, ti += gridDim.x) {
    const int S[3] = {nS[0], nS[1], nS[2]};
    origins(ti + gridDim.x, nS);
    if (ti < ntri) issue(u, S);
    else cp_async_commit();
  }
  int b = 0;
  for (int t = blockIdx.x; t < ntri; t += gridDim.x, ti += gridDim.x,
           b = (b + 1 == NB) ? 0 : b + 1) {
    // NB-2 later orbits may still be in flight; this one has landed for this
    // thread, and after the barrier for every thread, which has also finished
    // evaluating the previous orbit, so its buffer can be refilled
    cp_async_wait<NB - 2>();
    __syncthreads();
    {
      const int S[3] = {nS[0], nS[1], nS[2]};
      origins(ti + gridDim.x, nS);
      if (ti < ntri) issue(b == 0 ? NB - 1 : b - 1, S);
      else cp_async_commit();
    }
    const unsigned char* base = tsm_raw + b * L::BUF;
    const T* cK = reinterpret_cast<const T*>(base);
    const T* cU = cK + L::CUBES;
    const T* pm = reinterpret_cast<const T*>(base + L::MAT_OFF);
    const T* pv = reinterpret_cast<const T*>(base + L::VEC_OFF);
    const double* pe = reinterpret_cast<const double*>(base + L::EV_OFF);
    const int* sS = reinterpret_cast<const int*>(base + L::S_OFF);
    const int S0 = sS[0], S1 = sS[1], S2 = sS[2];
    if (S0 + l[0] < v && S1 + l[1] < v && S2 + l[2] < v) {
      double k[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) k[q] = (double)cK[koff[q]];
      const double dinv = __drcp_rn(eijk - pe[l[0]] - pe[8 + l[1]] - pe[16 + l[2]]);
      double se = 0.0, so = 0.0;
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        if (perm3_parity(q)) so += k[q];
        else se += k[q];
      }
      const double ce = se - 2.0 * so, co = so - 2.0 * se;
      double X[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) X[q] = (3.0 * k[q] + (perm3_parity(q) ? co : ce)) * dinv;
      // Y of ordering q = (p0,p1,p2): g0[p0] M0[p1,p2] + g1[p1] M1[p0,p2]
      // + g2[p2] M2[p0,p1] + (f, N likewise).  Each ordered pair (x, y) with
      // third position z serves three orderings: (z,x,y) through M0/N0,
      // (x,z,y) through M1/N1 and (x,y,z) through M2/N2.
      double vg[3][6];  // vectors at the three positions: vg[pos][w]
#pragma unroll
      for (int pos = 0; pos < 3; ++pos)
#pragma unroll
        for (int w = 0; w < 6; ++w) vg[pos][w] = (double)pv[(w * 3 + pos) * 8 + l[pos]];
      double yq[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int x = 0; x < 3; ++x)
#pragma unroll
        for (int yy = 0; yy < 3; ++yy) {
          if (x == yy) continue;
          const int z = 3 - x - yy;
          const int lo = x < yy ? l[x] : l[yy], hi = x < yy ? l[yy] : l[x];
          const T* mb = pm + pair_index(x, yy) * 6 * 64 + lo + 8 * hi;
          yq[perm3_index(z, x)] += vg[z][0] * (double)mb[0] + vg[z][3] * (double)mb[3 * 64];
          yq[perm3_index(x, z)] += vg[z][1] * (double)mb[64] + vg[z][4] * (double)mb[4 * 64];
          yq[perm3_index(x, yy)] += vg[z][2] * (double)mb[2 * 64] + vg[z][5] * (double)mb[5 * 64];
        }
      double ek = 0.0, ey = 0.0;
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        ek += (HAS_U ? (double)cU[koff[q]] : k[q]) * X[q];
        ey += X[q] * yq[q];
      }
      const bool ab = (S0 == S1), bc = (S1 == S2);
      const double wgt = (ab && bc) ? (1.0 / 6.0) : (ab || bc) ? 0.5 : 1.0;
      eK += wgt * ek;
      eY += wgt * ey;
    }
  }
  cp_async_wait<0>();
  const double r0 = block_sum(eK, sh);
  const double r1 = block_sum(eY, sh);
  if (threadIdx.x == 0) {
    part[(2 * y) * gridDim.x + blockIdx.x] = r0;
    part[(2 * y + 1) * gridDim.x + blockIdx.x] = r1;
  }
}

// out[2y + c] = sum_i part[(2y + c) * nparts + i], one block per (y, c), fixed order
__global__ void final_sum_pairs_kernel(int nparts, const double* part, double* out) {
  __shared__ double sh[32];
  const int q = blockIdx.x;
  double acc = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += part[(int64_t)q * nparts + i];
  const double r = block_sum(acc, sh);
  if (threadIdx.x == 0) out[q] = r;
}

int64_t triples_energy_grid(int nv) {
  // one resident block per SM: 128 registers a thread keep the evaluation free
  // of spills; the double-buffered loads overlap it with the next orbit
  const int64_t ntri = triples_cube_count(nv);
  return ntri < 148 ? ntri : 148;
}

int64_t triples_energy_scratch_len(int nv, int nitems) { return 2 * triples_energy_grid(nv) * nitems; }

int triples_energy_batched(stream_t s, int nv, int nitems, const void* K, const void* KU,
                           int64_t kstride, bool k_f32, const double* eijk_tab, const double* ev,
                           const TriplesTerms* tt_tab, const int* tri, double* scratch,
                           double* out) {
  const int64_t ntri = triples_cube_count(nv);
  // FP32 K goes to triples_energy_f32_batched (dev_energy.cu)
  if (k_f32 || nv > 1290 || nitems <= 0 || nitems > 65535 || !eijk_tab || !tt_tab)
    return (int)cudaErrorInvalidValue;
  const int g = (int)triples_energy_grid(nv);
  static DeviceFlags attr;
  if (!attr.test()) {
    cudaError_t e = cudaFuncSetAttribute(triples_energy_kernel<double, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         EnergySmem<double, false>::BYTES);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(triples_energy_kernel<double, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               EnergySmem<double, true>::BYTES);
    attr.set(e);
  }
  cudaStream_t st = (cudaStream_t)s;
  const dim3 grid((unsigned)g, (unsigned)nitems);
  // algorithmic bytes: each element of K (and of KU) read once
  const int slot = ktime_begin(s, KT_TRIPLES);
  const double kbytes = (double)nitems * (double)nv * nv * nv * 8.0 * (KU ? 2.0 : 1.0);
  if (KU)
    triples_energy_kernel<double, true><<<grid, 512, EnergySmem<double, true>::BYTES, st>>>(
        nv, (const double*)K, (const double*)KU, kstride, eijk_tab, ev, tt_tab, tri,
        (int)ntri, scratch);
  else
    triples_energy_kernel<double, false><<<grid, 512, EnergySmem<double, false>::BYTES, st>>>(
        nv, (const double*)K, nullptr, kstride, eijk_tab, ev, tt_tab, tri, (int)ntri,
        scratch);
  ktime_end(s, KT_TRIPLES, slot, kbytes);
  int e = launched();
  if (e) return e;
  final_sum_pairs_kernel<<<2 * nitems, 256, 0, st>>>(g, scratch, out);
  return launched();
}

}  // namespace dev
}  // namespace ecg
