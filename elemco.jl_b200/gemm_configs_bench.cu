// gemm_configs_bench.cu — times the FP64 dgemm_kernel tile configurations of
// csrc/dev_cuda.cu on the shapes of the CCSD/(T) contractions (CUDA events,
// median of 5).  Stand-alone developer benchmark, not part of libecgpu:
//   nvcc -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a \
//        -Ielemco.jl_b200/csrc -Iinclude -o gemm_configs_bench elemco.jl_b200/gemm_configs_bench.cu
#include "csrc/dev_cuda.cu"
#include <cstdio>
#include <vector>
#include <algorithm>
using namespace ecg::dev;
typedef int (*LF)(const GemmArgs&, int64_t, cudaStream_t);
struct C { const char* name; LF f; int bm, bn; };
static C cfgs[] = {
  {"64x64x16 w32x32 s3 m3 *",  launch_gemm<64,64,16,32,32,3,3>, 64,64},
  {"64x64x16 w32x32 s4 m3",   launch_gemm<64,64,16,32,32,4,3>, 64,64},
  {"64x64x16 w32x32 s2 m4",   launch_gemm<64,64,16,32,32,2,4>, 64,64},
  {"64x64x16 w32x32 s3 m2",   launch_gemm<64,64,16,32,32,3,2>, 64,64},
  {"128x64x16 w32x32 s3 m1",  launch_gemm<128,64,16,32,32,3,1>, 128,64},
  {"128x64x16 w32x32 s3 m2",  launch_gemm<128,64,16,32,32,3,2>, 128,64},
  {"64x128x16 w32x32 s3 m2",  launch_gemm<64,128,16,32,32,3,2>, 64,128},
  {"32x64x16 w32x32 s3 m4",   launch_gemm<32,64,16,32,32,3,4>, 32,64},
  {"128x128x16 w64x32 s3 m1", launch_gemm<128,128,16,64,32,3,1>, 128,128},
  {"128x64x16 w64x32 s3 m2",  launch_gemm<128,64,16,64,32,3,2>, 128,64},
  {"64x128x16 w32x64 s3 m2",  launch_gemm<64,128,16,32,64,3,2>, 64,128},
  {"64x64x16 w32x32 s3 m1",   launch_gemm<64,64,16,32,32,3,1>, 64,64},
  {"64x64x16 w32x32 s3 m3",   launch_gemm<64,64,16,32,32,3,3>, 64,64},
  {"64x64x16 w32x32 s4 m4",   launch_gemm<64,64,16,32,32,4,4>, 64,64},
  {"64x64x32 w32x32 s3 m2",   launch_gemm<64,64,32,32,32,3,2>, 64,64},
  {"128x128x32 w64x32 s2 m1", launch_gemm<128,128,32,64,32,2,1>, 128,128},
  {"128x64x32 w64x32 s3 m1",  launch_gemm<128,64,32,64,32,3,1>, 128,64},
  {"64x128x32 w32x64 s3 m1",  launch_gemm<64,128,32,32,64,3,1>, 64,128},
};
int main() {
  struct S { int64_t m,n,k; int ta; const char* what; };
  std::vector<S> shapes = {
    {1216,1216,1216,0,"ring o3v3 (H2O)4"}, {1216,1216,336,0,"DF build K=nQ"},
    {5776,5776,336,0,"ladder V (H2O)4"}, {5776,256,5776,0,"ladder contract (H2O)4"},
    {5776,256,256,0,"T2*I"}, {1216,336,1216,0,"W3"}, {76,25536,16,0,"dBvv"},
    {7632,7632,7632,0,"ring (H2O)6/VTZ"}, {101124,2544,846,0,"ladder V (H2O)6"},
    {2544,576,101124,0,"ladder contract (H2O)6"}, {8192,8192,8192,0,"square 8192"},
    {1216,1216,1216,1,"ring, A transposed"},
  };
  size_t maxe = 0;
  for (auto& s: shapes) maxe = std::max(maxe, (size_t)std::max({s.m*s.k, s.k*s.n, s.m*s.n}));
  double *A,*B,*Cm; cudaMalloc(&A, maxe*8); cudaMalloc(&B, maxe*8); cudaMalloc(&Cm, maxe*8);
  cudaMemset(A,0,maxe*8); cudaMemset(B,0,maxe*8); cudaMemset(Cm,0,maxe*8);
  cudaStream_t st; cudaStreamCreate(&st);
  cudaEvent_t e0,e1; cudaEventCreate(&e0); cudaEventCreate(&e1);
  for (auto& s: shapes) {
    printf("%-26s m=%ld n=%ld k=%ld\n", s.what, s.m, s.n, s.k);
    for (auto& c: cfgs) {
      GemmArgs g{A,B,Cm,s.m,s.n,s.k, s.ta? s.k:1, s.ta?1:s.m, 0, 1, s.k, 0, 1, s.m, 0, 1.0, 0.0, s.ta?1:0, 0, 0};
      int reps = (s.m*s.n*s.k > 2e11) ? 2 : 5;
      std::vector<float> t;
      for (int r = 0; r < reps + 1; ++r) {
        cudaEventRecord(e0, st); int err = c.f(g, 1, st); cudaEventRecord(e1, st); cudaEventSynchronize(e1);
        if (err) { printf("   %-28s launch err %d\n", c.name, err); break; }
        float ms; cudaEventElapsedTime(&ms, e0, e1); if (r) t.push_back(ms);
      }
      if (t.empty()) continue;
      std::sort(t.begin(), t.end());
      double ms = t[t.size()/2];
      int64_t tiles = ((s.m+c.bm-1)/c.bm)*((s.n+c.bn-1)/c.bn);
      printf("   %-28s %9.3f ms %7.2f TF/s tiles %ld\n", c.name, ms, 2.0*s.m*s.n*s.k/ms/1e9, tiles);
    }
  }
  cudaError_t e = cudaGetLastError(); printf("last error %d\n", (int)e);
  return 0;
}
