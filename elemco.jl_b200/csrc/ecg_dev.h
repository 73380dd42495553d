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
// Waits for s, frees the scratch the layer holds for it (splitk_buffer,
// split_scratch) and destroys it.
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
// Record the launches issued on s after graph_capture_begin into a CUDA graph;
// graph_capture_run ends the capture, runs the graph once, waits for it and
// frees it (*nodes: the number of graph nodes).
int graph_capture_begin(stream_t s);
int graph_capture_run(stream_t s, int64_t* nodes);
void graph_capture_abort(stream_t s);  // end a capture in progress, discarding it

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
// Optional (batch 1 only):
//   dn > 0    C(m,n) = C[m*scm + (n % dn)*scn + (n / dn)*scn2]  (n splits into
//             two tensor indices, e.g. (b,c) of a v^3 cube written permuted)
//   kseg > 0  two K segments: k < kseg reads A, B as above; k >= kseg reads
//             A1[m*sam + (k-kseg)*sak1] and B1[(k-kseg)*sbk1 + n*sbn].
//   ptab      device table of 5 offsets (elements) per batch item b, for A, B,
//             C, A1, B1, used in place of b*sab, b*sbb, b*scb (batch >= 1).
struct Gemm {
  int64_t m = 0, n = 0, k = 0, batch = 1;
  double alpha = 1.0, beta = 0.0;
  const double* A = nullptr;
  int64_t sam = 1, sak = 0, sab = 0;
  const double* B = nullptr;
  int64_t sbk = 1, sbn = 0, sbb = 0;
  double* C = nullptr;
  int64_t scm = 1, scn = 0, scb = 0;
  int64_t dn = 0, scn2 = 0;
  int64_t kseg = 0;
  const double* A1 = nullptr;
  int64_t sak1 = 0;
  const double* B1 = nullptr;
  int64_t sbk1 = 0;
  const int64_t* ptab = nullptr;
  // run on the TMA-staged kernel whenever it can address the operands, also
  // with a row stride or column map (the (T) K builds; other callers keep
  // the dispatcher's choice)
  bool mapped_tma = false;
};
int gemm_strided(stream_t s, const Gemm& g);
// FP64 GEMM with TMA-staged operands (dev_dgemm.cu): no kseg/ptab (C through
// scm and scn or the dn/scn2 column map; no K split with dn), each operand
// contiguous along its row index or along k with its other strides even
// (16-byte multiples) and a 16-byte-aligned base.  cfg selects the tile (0: 64x64, 1: 128x64, 2: 64x128,
// 3: 128x128); nsplit > 1 (batch 1) cuts K into slices summed in a fixed
// order.  Returns -1, launching nothing, when TMA cannot address an operand.
// dgemm_tma_usable: the cases the plain-GEMM dispatcher sends to it (C with
// unit row stride, no column map); dgemm_tma_usable_mapped: all it accepts.
constexpr int DTMA_CONFIGS = 4;
bool dgemm_tma_usable(const Gemm& q);
bool dgemm_tma_usable_mapped(const Gemm& q);
int dgemm_tma(stream_t s, const Gemm& q, int cfg, int nsplit);
// Time-out code of the TMA FP64 GEMM's bounded waits since the last call
// (0 = none); reading clears it.
int dtma_error(int* code);
// Split-BF16 tensor-core version of gemm_strided (batch 1, no dn/kseg).
int gemm_strided_mixed(stream_t s, const Gemm& g);

// Pre-split operand of the tensor-core GEMM: X(r,k) as `slices` (2 or 3)
// BF16 slices [slices][rows_p][k_p] (k fastest; rows padded to 128, k to 64,
// zero filled) and the TMA descriptor over them.  tc_operand_elems() is the
// BF16 element count of the storage; tc_split() fills it (dst 16-byte
// aligned) from the FP64 source X(r,k) = src[r*sr + k*sk] and encodes the
// descriptor.  Three slices reproduce FP32-level products, two slices
// ~2^-16 relative.
struct TcOperand {
  alignas(64) unsigned char map[128];
  // the same operand with 160- and 256-row boxes, for 160- and 256-column
  // tiles when it is the B operand (each encoded, and its flag set, when the
  // row extent is at least the box)
  alignas(64) unsigned char map_w[128];
  alignas(64) unsigned char map_x[128];
  bool wide = false, xwide = false;
  int64_t rows = 0, rows_p = 0, k = 0, k_p = 0;
  int slices = 0;
  void* base = nullptr;        // first BF16 element of row 0, slice 0
  int64_t slice_stride = 0;    // BF16 elements between slices
};
size_t tc_operand_elems(int64_t rows, int64_t k, int slices);
int tc_split(stream_t s, const double* src, int64_t rows, int64_t k, int64_t sr, int64_t sk,
             int slices, void* dst, TcOperand* op);
// Rows [row0, row0 + rows) of a split operand as an operand of their own (no
// copy: a descriptor over the same storage; rows past the view read as zero).
int tc_view(const TcOperand& parent, int64_t row0, int64_t rows, TcOperand* out);
// Descriptor over slices already written to dst in tc_split's layout
// ([slice][tc_pad_rows(rows)][tc_pad_k(k)], K fastest, zero K padding).
int tc_bind(void* dst, int64_t rows, int64_t k, int slices, TcOperand* op);
int64_t tc_pad_rows(int64_t rows);
int64_t tc_pad_k(int64_t k);
// ladder_pack_v fused with the three-slice split of its outputs: the a-block's
// V (FP32 when v_f32, else FP64; layout of ladder_pack_v) is packed into the
// symmetric (rows: the block's npairs pairs, K = v(v+1)/2) and antisymmetric
// (rows: its a < b pairs, K = v(v-1)/2) operands, written as BF16 slices in
// tc_split's layout at Vp / Vm (bind them with tc_bind).
int ladder_pack_v_split(stream_t s, int nv, int a0, int na, int npairs, const int* pairs,
                        const int* cdp, const void* V, bool v_f32, void* Vp, void* Vm);
// C(m,n) = alpha sum_k A(m,k) B(k,n) + beta C(m,n) over pre-split operands
// (all with the same slice count): the K sum runs over up to TC_MAX_SEG
// segments A[s]/B[s], s = 0, 1, ... (the first null A[s] ends the list), each
// with its own K depth and operands.  A plain FP64 C (no index maps) may be
// computed in K slices summed in FP64 (to fill the GPU and to bound the FP32
// accumulation length).  C is FP64, or FP32 when f32, at
// C[rowoff(m) + coloff(n)] with rowoff(m) = (m % dm)*scm + (m / dm)*scm2
// (dm = 0: m*scm) and coloff(n) = (n % dn)*scn + (n / dn)*scn2 (dn = 0:
// n*scn).  Stores are coalesced when scm == 1.
constexpr int TC_MAX_SEG = 4;
// Longest K one FP32 tensor-memory accumulator sums: FP64 outputs with a
// longer K are computed in K slices whose partial products are added in FP64;
// FP32 outputs are one accumulation, so callers keep their K within this.
constexpr int64_t TC_ACC_K = 1024;
struct TcGemm {
  int64_t m = 0, n = 0;
  double alpha = 1.0, beta = 0.0;
  const TcOperand* A[TC_MAX_SEG] = {nullptr, nullptr, nullptr, nullptr};
  const TcOperand* B[TC_MAX_SEG] = {nullptr, nullptr, nullptr, nullptr};
  void* C = nullptr;
  bool f32 = false;
  int64_t scm = 1, scn = 0, dn = 0, scn2 = 0, dm = 0, scm2 = 0;
};
int tc_gemm(stream_t s, const TcGemm& g);
// Batched form: `batch` GEMMs of the shape of g (g.A/g.B give the segments
// and operand shapes), item b reading the operand descriptors mtab[b] (device
// memory, 64-byte aligned, tc_maps_bytes() each, written by tc_maps_fill on
// the host from nseg segments A[s]/B[s]) and writing C + b*c_stride through
// g's index map.  One launch.
size_t tc_maps_bytes();
// n: the GEMM's column count (it selects the tile width, as in tc_gemm_batched).
int tc_maps_fill(int nseg, const TcOperand* const* A, const TcOperand* const* B, int64_t n,
                 void* host_dst);
int tc_gemm_batched(stream_t s, const TcGemm& g, int batch, const void* mtab, int64_t c_stride);

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

// y[i] = (float)x[i]
int to_f32(stream_t s, int64_t n, const double* x, float* y);
// out[i] = (float(a[i]), float(b[i])) as float2 pairs (out 8-byte aligned)
int to_f32_pairs(stream_t s, int64_t n, const double* a, const double* b, void* out);
// *flag = 1 if any of x[0..n) is an infinity or NaN, else 0 (device double)
int nonfinite(stream_t s, int64_t n, const double* x, double* flag);

// (T) energies of occupied triplets (src/cc/cc_triples.jl:113-156) from
// K[a,b,c] (FP64, or FP32 when k_f32), without storing X:
//   X[a,b,c] = (4K[abc]-2K[acb]-2K[cba]-2K[bac]+K[cab]+K[bca]) / (eijk-ev[a]-ev[b]-ev[c])
//   out[0]   = sum KE*X      (KE = KU when given, else K)
//   out[1]   = sum X*Y,  Y[a,b,c] = g0[a] M0[b,c] + g1[b] M1[a,c] + g2[c] M2[a,b]
//                              + f0[a] N0[b,c] + f1[b] N1[a,c] + f2[c] N2[a,b]
// The 8^3 cubes of K are visited in orbits of the index permutations, so each
// element of K is read once.  `tri` holds the cube triples A <= B <= C (3
// ints each) for nt = ceil(nv/8) cubes per axis: triples_cube_count(nv) of
// them, written by triples_cube_table().  g, f (length nv) and M, N (nv x nv)
// hold elements of K's precision; ev (FP64) the virtual orbital energies.
// nv <= 1290 (32-bit element offsets).
struct TriplesTerms {
  const void* g[3];
  const void* f[3];
  const void* M[3];
  const void* N[3];
};
int64_t triples_cube_count(int nv);
void triples_cube_table(int nv, int* tri);
// FP64 K: item b reads K + b*kstride (KU likewise), eijk_tab[b] and tt_tab[b]
// (device tables) and writes out[2b], out[2b+1]; partial sums land in
// `scratch` (at least triples_energy_scratch_len(nv, nitems) doubles) and are
// summed in a fixed order.  One launch (plus one fixed-order reduction
// launch).  k_f32 must be false (FP32 K: triples_energy_f32_batched).
int64_t triples_energy_scratch_len(int nv, int nitems);
int64_t triples_energy_grid(int nv);  // blocks per batch item of the energy kernels
int triples_energy_batched(stream_t s, int nv, int nitems, const void* K, const void* KU,
                           int64_t kstride, bool k_f32, const double* eijk_tab, const double* ev,
                           const TriplesTerms* tt_tab, const int* tri, double* scratch,
                           double* out);
// The same for FP32 K (and K') (dev_energy.cu).  K[a,b,c] of slot i sits at
// K + i*kstride + a + vp*(b + v*c), vp >= v a multiple of 4 (TMA strides of
// 16 bytes); nslots >= nitems slots at K (and KU), 16-byte aligned.  The
// (M, N) terms are FP32 pairs per occupied pair p = x + o*y, packed by
// triples_mn_pack: mn[p][a + vpe*b] and their transposes mt[p][b + vpe*a]
// (vpe = v rounded up to even; triples_mn_elems float2 each).  Per item,
// gf[r] points at the (g, f)[a] FP32 pairs of occupied index r of the triplet
// (i, j, k) and mnpair[w] is the pair index of (j,k), (i,k), (i,j).
struct TriplesTermsF {
  const void* gf[3];
  int32_t mnpair[3];
};
int64_t triples_mn_elems(int nv, int64_t npairs);
int triples_mn_pack(stream_t s, int nv, int64_t npairs, const double* M, const double* N,
                    void* mn, void* mt);
int triples_energy_f32_batched(stream_t s, int nv, int vp, int nitems, int nslots, const float* K,
                               const float* KU, int64_t kstride, const void* mn, const void* mt,
                               int64_t npairs, const double* eijk_tab, const double* ev,
                               const TriplesTermsF* tt_tab, const int* tri, double* scratch,
                               double* out);
// Time-out code of the FP32 energy kernel's bounded waits (0 = none); reading
// clears it.
int energy_error(int* code);

// Split-K GEMM (column-major, device pointers) whose partial products use a
// fixed file-scope device array instead of allocated memory; m*n must not
// exceed noalloc_scratch_doubles().  *nsplit receives the K split used.
size_t noalloc_scratch_doubles();
int gemm_splitk_noalloc(stream_t s, char ta, char tb, int64_t m, int64_t n, int64_t k,
                        double alpha, const double* A, int64_t lda, const double* B, int64_t ldb,
                        double beta, double* C, int64_t ldc, int* nsplit);

// Split-BF16 tensor-core GEMM (tcgen05, FP32 accumulate, ~FP32 accuracy),
// same interface as gemm().  tc_error() returns and clears the time-out code
// of the kernels with bounded mbarrier waits (0 = none; 1-4 tensor-core GEMM,
// 17 TMA-staged FP64 GEMM, 33 FP32 (T) energy kernel).
int gemm_mixed(stream_t s, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
               const double* A, int64_t lda, const double* B, int64_t ldb, double beta,
               double* C, int64_t ldc);
int tc_error(int* code);
// Split-K scratch of stream s on the current device (at least n doubles;
// grown on demand, after s has drained, never during stream capture: nullptr
// then, or when the allocation fails) and its fixed-order reduction
// C(i,j) = alpha sum_z P[z][i + j m] + beta C(i,j), C at C[i*scm + j*scn].
double* splitk_buffer(stream_t s, size_t n);
// Scratch of stream s for gemm_mixed's BF16 operand slices (same rules).
void* split_scratch(stream_t s, size_t bytes);
// Bound (ns) of the tensor-core kernels' main-loop waits on stream s
// (0 = the default second); the kernels' final waits keep the second.
int set_tc_wait(stream_t s, uint64_t ns);
uint64_t tc_wait(stream_t s);
int splitk_reduce(stream_t s, int64_t m, int64_t n, int S, const double* P, double alpha,
                  double beta, double* C, int64_t scm, int64_t scn);
// The same for FP32 partials (summed in FP64).
int splitk_reduce_f32(stream_t s, int64_t m, int64_t n, int S, const float* P, double alpha,
                      double beta, double* C, int64_t scm, int64_t scn);

// Event timing of kernel families (process-wide diagnostic): enable, then
// read and reset a family's summed device ms, launch count and algorithmic
// work (flops for the GEMMs, bytes for the (T) energy kernel).  Launches
// during stream capture are not timed.  ktime_begin returns a slot (-1: not
// timed) for ktime_end, which records the end event and adds the work.
enum { KT_DGEMM = 0, KT_TCGEMM = 1, KT_TRIPLES = 2, KT_FAMILIES = 3 };
void gemm_timing(bool enable);
void gemm_time(double* ms, int64_t* launches, double* flops);  // KT_DGEMM
void kernel_time(int family, double* ms, int64_t* launches, double* work);
int ktime_begin(stream_t s, int family);
void ktime_end(stream_t s, int family, int slot, double work);

// Symmetric/antisymmetric particle-particle ladder helpers.  Pair tables hold
// (x,y) as int pairs: cdp enumerates c<=d (d outer), ijp i<=j, pairs the
// (a,b), a<=b of one a-block.  Packed "minus" indices follow arithmetically:
// idx-(c,d) = idx+(c,d) - d (c<d); pair-(a,b) = pair+(a,b) - (a-a0) - 1 (a<b).
//   ladder_pack_t: Ts[cd+,ij+] = (T[c,d,i,j]+T[d,c,i,j])/2, Ta[cd-,ij-] = (T[c,d,i,j]-T[d,c,i,j])/2
//   ladder_pack_v: Vblk[c,a',d,b''] (a' = a-a0, b'' = b-a0) ->
//                  Vp[cd+,pair+] = V[acbd]+V[adbc] (c<d), V[acbc] (c=d);  Vm[cd-,pair-] = V[acbd]-V[adbc]
//   ladder_unpack: R2[a,b,i,j] += Lp+Lm, R2[b,a,i,j] += Lp-Lm, R2[a,b,j,i] += Lp-Lm, R2[b,a,j,i] += Lp+Lm
// The packed cd index runs fastest, with leading dimensions ldp (>= v(v+1)/2)
// for Ts / Vp and ldm (>= v(v-1)/2) for Ta / Vm (even values let TMA stage them).
int ladder_pack_t(stream_t s, int nv, int no, const double* T2, const int* cdp, const int* ijp,
                  double* Ts, double* Ta, int64_t ldp, int64_t ldm);
int ladder_pack_v(stream_t s, int nv, int a0, int na, int npairs, const int* pairs,
                  const int* cdp, const double* Vblk, double* Vp, double* Vm, int64_t ldp,
                  int64_t ldm);
int ladder_unpack(stream_t s, int nv, int no, int a0, int npairs, const int* pairs,
                  const int* ijp, const double* Lp, const double* Lm, double* R2);

// Gaussian integrals over contracted Cartesian shells (dev_ints.cu).  A shell
// has centre (x, y, z), angular momentum l <= INT_LMAX, nprim primitives whose
// exponents/coefficients start at poff in the exponent/coefficient arrays,
// and its first Cartesian function at boff of the output dimension.
// Components of degree l are ordered i = l..0, j = l-i..0 (x^i y^j z^k).
// Outputs are accumulated (zero them first).
constexpr int INT_LMAX = 4;   // largest shell angular momentum (g)
constexpr int INT_LTOT = 12;  // largest l_a + l_b + l_c (+ l_d) of a Coulomb integral
struct IntShell {
  double x, y, z;
  int l, nprim, poff, boff;
};
// kind 0 overlap, 1 kinetic, 2 nuclear attraction (natom charges Z at xyz),
// 3 dipole about origin (three nn x nn matrices); out[m + nn*n].
int int1e_cart(stream_t s, int kind, const IntShell* sh, int nsh, const double* ex,
               const double* co, int natom, const double* Z, const double* xyz,
               const double* origin, int64_t nn, double* out);
// (P|Q), out[P + np*Q]
int int2c2e_cart(stream_t s, const IntShell* aux, int nsh, const double* ex, const double* co,
                 int64_t np, double* out);
// (mn|P), out[m + nm*(n + nm*P)]; ex/co hold both bases' primitives
int int3c2e_cart(stream_t s, const IntShell* ao, int nao_sh, const IntShell* aux, int naux_sh,
                 const double* ex, const double* co, int64_t nm, double* out);

// Count of kernels launched through this layer in this process.
int64_t launches();
void note_launches(int n);  // add n launches made outside dev_cuda.cu

}  // namespace dev
}  // namespace ecg
