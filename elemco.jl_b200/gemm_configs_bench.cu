// gemm_configs_bench.cu — times the FP64 dgemm_kernel tile configurations of
// csrc/dev_cuda.cu on the shapes of the CCSD/(T) contractions (CUDA events,
// median of 5, random operands) after checking each configuration against a host reference on
// a small ragged problem.  Stand-alone developer benchmark, not part of
// libecgpu:
//   nvcc -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a \
//        -Ielemco.jl_b200/csrc -Iinclude -o gemm_configs_bench elemco.jl_b200/gemm_configs_bench.cu
#include "csrc/dev_cuda.cu"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>
using namespace ecg::dev;
typedef int (*LF)(const GemmArgs&, int64_t, cudaStream_t);
struct C { const char* name; LF f; int bm, bn; };
// KMMA: 0 = mma.m8n8k4, 4/8/16 = mma.m16n8k{4,8,16}
static C cfgs[] = {
  {"64x64x16 w32x32 s3 m3 k0 *", launch_gemm<64,64,16,32,32,3,3,0>, 64,64},
  {"64x64x16 w32x32 s3 m3 k4",   launch_gemm<64,64,16,32,32,3,3,4>, 64,64},
  {"64x64x16 w32x32 s3 m3 k8",   launch_gemm<64,64,16,32,32,3,3,8>, 64,64},
  {"64x64x16 w32x32 s3 m3 k16",  launch_gemm<64,64,16,32,32,3,3,16>, 64,64},
  {"64x64x32 w32x32 s3 m2 k16",  launch_gemm<64,64,32,32,32,3,2,16>, 64,64},
  {"64x64x32 w32x32 s3 m2 k8",   launch_gemm<64,64,32,32,32,3,2,8>, 64,64},
  {"128x64x16 w32x32 s3 m2 k8",  launch_gemm<128,64,16,32,32,3,2,8>, 128,64},
  {"128x64x16 w64x32 s3 m2 k8",  launch_gemm<128,64,16,64,32,3,2,8>, 128,64},
  {"64x128x16 w32x64 s3 m2 k8",  launch_gemm<64,128,16,32,64,3,2,8>, 64,128},
  {"128x128x16 w64x32 s3 m1 k8", launch_gemm<128,128,16,64,32,3,1,8>, 128,128},
  {"128x128x16 w32x64 s3 m1 k16", launch_gemm<128,128,16,32,64,3,1,16>, 128,128},
  {"128x128x32 w64x32 s2 m1 k16", launch_gemm<128,128,32,64,32,2,1,16>, 128,128},
};

// Operands are filled with pseudo-random values in [-1, 1) (a hash of the
// index): zero-filled operands draw less power and run at unrepresentative
// clocks.
__global__ void fill_random(double* p, size_t n, uint64_t seed) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    uint64_t x = (i + 1) * 0x9E3779B97F4A7C15ull ^ seed;
    x ^= x >> 31;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 29;
    p[i] = (double)(x >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  }
}

static GemmArgs args(const double* A, const double* B, double* Cm, int64_t m, int64_t n,
                     int64_t k, int ta, int bn) {
  // A(m,k): column-major (ta = 0) or transposed storage; B(k,n): column-major
  // (bn = 0) or n-fastest storage (B[k*n + n'])
  GemmArgs g{A, B, Cm, m, n, k, ta ? k : 1, ta ? 1 : m, 0, bn ? n : 1, bn ? 1 : k, 0,
             1, m, 0, 1.0, 0.0, ta ? 1 : 0, bn ? 1 : 0, 0};
  return g;
}

int main() {
  cudaStream_t st;
  cudaStreamCreate(&st);
  // correctness on a ragged problem, both B storage orders
  {
    const int64_t m = 197, n = 133, k = 61;
    std::mt19937_64 rng(3);
    std::normal_distribution<double> nd;
    std::vector<double> hA(m * k), hB(k * n), ref(m * n, 0.0), out(m * n);
    for (auto& x : hA) x = nd(rng);
    for (auto& x : hB) x = nd(rng);
    double *A, *B, *Cm;
    cudaMalloc(&A, hA.size() * 8);
    cudaMalloc(&B, hB.size() * 8);
    cudaMalloc(&Cm, out.size() * 8);
    cudaMemcpy(A, hA.data(), hA.size() * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(B, hB.data(), hB.size() * 8, cudaMemcpyHostToDevice);
    for (int bn = 0; bn < 2; ++bn) {
      for (int64_t j = 0; j < n; ++j)
        for (int64_t i = 0; i < m; ++i) {
          double s = 0;
          for (int64_t l = 0; l < k; ++l) s += hA[i + m * l] * hB[bn ? l * n + j : l + k * j];
          ref[i + m * j] = s;
        }
      for (auto& c : cfgs) {
        cudaMemset(Cm, 0, out.size() * 8);
        int err = c.f(args(A, B, Cm, m, n, k, 0, bn), 1, st);
        cudaStreamSynchronize(st);
        cudaMemcpy(out.data(), Cm, out.size() * 8, cudaMemcpyDeviceToHost);
        double e = 0;
        for (size_t q = 0; q < out.size(); ++q) e = std::max(e, std::fabs(out[q] - ref[q]));
        printf("check %-30s B %s  launch %d  max err %.3e %s\n", c.name, bn ? "n-fast" : "k-fast",
               err, e, e < 1e-11 ? "ok" : "WRONG");
      }
    }
    cudaFree(A);
    cudaFree(B);
    cudaFree(Cm);
  }
  struct S { int64_t m, n, k; int ta, bn; const char* what; };
  std::vector<S> shapes = {
    {1216, 1216, 1216, 0, 0, "ring o3v3 (H2O)4"}, {1216, 1216, 336, 0, 0, "DF build K=nQ"},
    {5776, 5776, 336, 0, 0, "ladder V (H2O)4"},   {5776, 256, 5776, 0, 0, "ladder contract (H2O)4"},
    {7632, 7632, 7632, 0, 0, "ring (H2O)6/VTZ"},  {101124, 2544, 846, 0, 0, "ladder V (H2O)6"},
    {2544, 576, 101124, 0, 0, "ladder contract (H2O)6"},
    {318, 101124, 318, 0, 1, "(T) W vvvo v=318"}, {8192, 8192, 8192, 0, 0, "square 8192"},
  };
  size_t maxe = 0;
  for (auto& s : shapes) maxe = std::max(maxe, (size_t)std::max({s.m * s.k, s.k * s.n, s.m * s.n}));
  double *A, *B, *Cm;
  cudaMalloc(&A, maxe * 8);
  cudaMalloc(&B, maxe * 8);
  cudaMalloc(&Cm, maxe * 8);
  fill_random<<<148 * 8, 256>>>(A, maxe, 1);
  fill_random<<<148 * 8, 256>>>(B, maxe, 2);
  cudaMemset(Cm, 0, maxe * 8);
  cudaDeviceSynchronize();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (auto& s : shapes) {
    printf("%-26s m=%ld n=%ld k=%ld\n", s.what, s.m, s.n, s.k);
    for (auto& c : cfgs) {
      GemmArgs g = args(A, B, Cm, s.m, s.n, s.k, s.ta, s.bn);
      int reps = (s.m * s.n * s.k > 2e11) ? 2 : 5;
      std::vector<float> t;
      for (int r = 0; r < reps + 1; ++r) {
        cudaEventRecord(e0, st);
        int err = c.f(g, 1, st);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        if (err) { printf("   %-30s launch err %d\n", c.name, err); break; }
        float ms;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r) t.push_back(ms);
      }
      if (t.empty()) continue;
      std::sort(t.begin(), t.end());
      double ms = t[t.size() / 2];
      int64_t tiles = ((s.m + c.bm - 1) / c.bm) * ((s.n + c.bn - 1) / c.bn);
      printf("   %-30s %9.3f ms %7.2f TF/s tiles %ld\n", c.name, ms, 2.0 * s.m * s.n * s.k / ms / 1e9,
             tiles);
    }
  }
  cudaError_t e = cudaGetLastError();
  printf("last error %d\n", (int)e);
  return 0;
}
