// ecg_dev.h — the device layer of libecgpu: memory, copies and kernel
// launchers.  The host orchestration (residuals, DIIS, drivers) talks to the
// GPU only through these functions; dev_cuda.cu implements them with CUDA
// kernels for sm_100a.  Every launcher is asynchronous on the given stream
// and returns 0 or a nonzero CUDA error code.
#pragma once
#include <cstddef>
#include <cstdint>

namespace ecg {
namespace dev {

using stream_t = void*;

int set_device(int device);
int stream_create(stream_t* s);
void stream_destroy(stream_t s);
int sync(stream_t s);
const char* error_string(int code);
int check_launch();  // cudaGetLastError as int

void* dmalloc(size_t bytes);   // nullptr on failure
void dfree(void* p);
void* hmalloc_pinned(size_t bytes);
void hfree_pinned(void* p);
int h2d(void* dst, const void* src, size_t bytes, stream_t s);
int d2h(void* dst, const void* src, size_t bytes, stream_t s);
int d2d(void* dst, const void* src, size_t bytes, stream_t s);
int memset0(void* dst, size_t bytes, stream_t s);

// C(m,n) = alpha * sum_k opA(A)(m,k) opB(B)(k,n) + beta * C(m,n), column-major;
// ta/tb = 'N' or 'T'.  batch > 1 uses strides sa/sb/sc between instances.
int gemm(stream_t s, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
         const double* A, int64_t lda, const double* B, int64_t ldb, double beta,
         double* C, int64_t ldc, int64_t batch = 1, int64_t sa = 0, int64_t sb = 0,
         int64_t sc = 0);

// Fully strided batched GEMM: C(m,n) = alpha sum_k A(m,k) B(k,n) + beta C(m,n)
// with A(m,k) = A[b*sab + m*sam + k*sak], B(k,n) = B[b*sbb + k*sbk + n*sbn],
// C(m,n) = C[b*scb + m*scm + n*scn] for batch b.  Batches must not write
// overlapping C elements.
struct Gemm {
  int64_t m = 0, n = 0, k = 0, batch = 1;
  double alpha = 1.0, beta = 0.0;
  const double* A = nullptr;
  int64_t sam = 1, sak = 0, sab = 0;
  const double* B = nullptr;
  int64_t sbk = 1, sbn = 0, sbb = 0;
  double* C = nullptr;
  int64_t scm = 1, scn = 0, scb = 0;
};
int gemm_strided(stream_t s, const Gemm& g);
// Split-BF16 tensor-core version of gemm_strided (batch must be 1).
int gemm_strided_mixed(stream_t s, const Gemm& g);

// out = alpha * permute(in) + beta * out.  in has rank nd with dims
// in_dims (column-major, first fastest); out dimension d is in dimension
// perm[d].  beta == 0 never reads out.
int permute(stream_t s, int nd, const int64_t* in_dims, const int* perm, double alpha,
            const double* in, double beta, double* out);

// y = alpha * x + beta * y   (beta == 0: y = alpha * x)
int axpby(stream_t s, int64_t n, double alpha, const double* x, double beta, double* y);

// out[b] = beta*out[b] + alpha * sum_{k<nk} in[b*sb + k*sk]
int strided_sum(stream_t s, int64_t nb, int64_t sb, int64_t nk, int64_t sk, double alpha,
                const double* in, double beta, double* out);

// Doubles (or singles) update with level shift, in place:
// T[a,b,i,j] += -R[a,b,i,j] / (ev[a]+ev[b]-eo[i]-eo[j]+shift)
int update_doubles(stream_t s, int nv, int no, const double* eo, const double* ev,
                   double shift, const double* R, double* T);
int update_singles(stream_t s, int nv, int no, const double* eo, const double* ev,
                   double shift, const double* R, double* T);

// Deterministic reductions into out[slot...] (device scalars):
//   dot:      out[0] = sum x*y over n
//   cs_dot:   for nv x nv x no x no:  out[0] = sum X[a,b,i,j] Y[a,b,i,j],
//             out[1] = sum X[b,a,i,j] Y[a,b,i,j]
// `scratch` must hold at least reduce_scratch_len() doubles.
int64_t reduce_scratch_len();
int dot(stream_t s, int64_t n, const double* x, const double* y, double* scratch, double* out);
int cs_dot(stream_t s, int nv, int no, const double* X, const double* Y, double* scratch,
           double* out);

// C(i,j) = alpha * A(i,j) + beta * C(i,j) for an m x n column-major block
// (leading dimensions lda, ldc); beta == 0 never reads C.
int geam(stream_t s, int64_t m, int64_t n, double alpha, const double* A, int64_t lda,
         double beta, double* C, int64_t ldc);

// out[a,b,i,j] = alpha * X[a,i] * Y[b,j] + beta * out[a,b,i,j]
// (X: na x ni, Y: nb x nj, out: na x nb x ni x nj).
int outer(stream_t s, int64_t na, int64_t ni, int64_t nb, int64_t nj, double alpha,
          const double* X, const double* Y, double beta, double* out);

// out = sum_{k<m} coef[k] * X[k]   (coef on the device)
int combine(stream_t s, int64_t n, int m, const double* const* X, const double* coef,
            double* out);

// (T) pieces for one occupied triplet (src/cc/cc_triples.jl:113-136):
//   X[a,b,c] = (4K[abc]-2K[acb]-2K[cba]-2K[bac]+K[cab]+K[bca]) / (eijk-ev[a]-ev[b]-ev[c])
//   *eout    = sum K*X  (skipped when eout == nullptr)
int triples_x(stream_t s, int nv, const double* K, double eijk, const double* ev, double* X,
              double* scratch, double* eout);
// K[a,b,c] = W0[a,b,c] + W1[b,a,c] + W2[a,c,b] + W3[c,b,a] + W4[b,c,a] + W5[c,a,b]
// (the six index permutations of W^{ijk}, W^{jik}, W^{ikj}, W^{kji}, W^{jki},
// W^{kij}); 8^3 cubes staged through shared memory.
int triples_sumw(stream_t s, int nv, const double* const* W, double* K);
// Cube-tiled variant of triples_x (same result).
int triples_x_cube(stream_t s, int nv, const double* K, double eijk, const double* ev, double* X,
                   double* scratch, double* eout);
// IntX[:,i] += fac X.M_jk, IntX[:,j] += fac X.M_ik, IntX[:,k] += fac X.M_ij and the same for
// IntY with N_*; M/N are nv x nv slices.  One block per virtual index, fixed order.
int triples_int(stream_t s, int nv, const double* X, const double* Mjk, const double* Mik,
                const double* Mij, const double* Njk, const double* Nik, const double* Nij,
                double fac, double* IntX, double* IntY, int i, int j, int k);

// Split-K GEMM (column-major, device pointers) whose partial products use a
// fixed file-scope device array instead of allocated memory; m*n must not
// exceed noalloc_scratch_doubles().  *nsplit receives the K split used.
size_t noalloc_scratch_doubles();
int gemm_splitk_noalloc(stream_t s, char ta, char tb, int64_t m, int64_t n, int64_t k,
                        double alpha, const double* A, int64_t lda, const double* B, int64_t ldb,
                        double beta, double* C, int64_t ldc, int* nsplit);

// Split-BF16 tensor-core GEMM (tcgen05, FP32 accumulate, ~FP32 accuracy),
// same interface as gemm().  tc_error() returns and clears the time-out code
// of the tensor-core kernels (0 = none).
int gemm_mixed(stream_t s, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
               const double* A, int64_t lda, const double* B, int64_t ldb, double beta,
               double* C, int64_t ldc);
int tc_error(int* code);
// Shared split-K scratch (grown on demand) and its fixed-order reduction
// C(i,j) = alpha sum_z P[z][i + j m] + beta C(i,j), C at C[i*scm + j*scn].
double* splitk_buffer(size_t n);
int splitk_reduce(stream_t s, int64_t m, int64_t n, int S, const double* P, double alpha,
                  double beta, double* C, int64_t scm, int64_t scn);

// GEMM event timing (process-wide): enable, then read and reset the totals.
void gemm_timing(bool enable);
void gemm_time(double* ms, int64_t* launches, double* flops);

// Symmetric/antisymmetric particle-particle ladder helpers.  Pair tables hold
// (x,y) as int pairs: cdp enumerates c<=d (d outer), ijp i<=j, pairs the
// (a,b), a<=b of one a-block.  Packed "minus" indices follow arithmetically:
// idx-(c,d) = idx+(c,d) - d (c<d); pair-(a,b) = pair+(a,b) - (a-a0) - 1 (a<b).
//   ladder_pack_t: Ts[cd+,ij+] = (T[c,d,i,j]+T[d,c,i,j])/2, Ta[cd-,ij-] = (T[c,d,i,j]-T[d,c,i,j])/2
//   ladder_pack_v: Vblk[c,a',d,b''] (a' = a-a0, b'' = b-a0) ->
//                  Vp[cd+,pair+] = V[acbd]+V[adbc] (c<d), V[acbc] (c=d);  Vm[cd-,pair-] = V[acbd]-V[adbc]
//   ladder_unpack: R2[a,b,i,j] += Lp+Lm, R2[b,a,i,j] += Lp-Lm, R2[a,b,j,i] += Lp-Lm, R2[b,a,j,i] += Lp+Lm
int ladder_pack_t(stream_t s, int nv, int no, const double* T2, const int* cdp, const int* ijp,
                  double* Ts, double* Ta);
int ladder_pack_v(stream_t s, int nv, int a0, int na, int npairs, const int* pairs,
                  const int* cdp, const double* Vblk, double* Vp, double* Vm);
int ladder_unpack(stream_t s, int nv, int no, int a0, int npairs, const int* pairs,
                  const int* ijp, const double* Lp, const double* Lm, double* R2);

// Count of kernels launched through this layer in this process.
int64_t launches();

}  // namespace dev
}  // namespace ecg
