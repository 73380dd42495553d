/*
 * ecgpu.h — C ABI of libecgpu.so, the B200 (sm_100a) closed-shell
 * coupled-cluster library that stands in for ElemCo.jl's CCSD/DCSD, (T),
 * Lambda and DIIS path.
 *
 * All arrays are column-major (Julia order, first index fastest), float64,
 * host memory owned by the caller.  Orbitals are ordered occupied first
 * (no of them), then virtual (nv); n = no + nv.  Every call returns an int
 * status (ECG_OK = 0); on failure ecg_last_error() holds a message.  Calls on
 * one context must not overlap (one host thread per context); each context
 * owns one CUDA stream and its device memory.
 *
 * Reference interfaces each entry point replaces are cited as
 * file:line inside the ElemCo.jl project.
 */
#ifndef ECGPU_H
#define ECGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ECG_OK 0
#define ECG_ERR_ARG 1        /* bad argument / shape mismatch                */
#define ECG_ERR_CUDA 2       /* CUDA runtime error                           */
#define ECG_ERR_OOM 3        /* device memory (or the context's cap) exhausted */
#define ECG_ERR_NONFINITE 4  /* NaN/Inf detected in inputs or results        */
#define ECG_ERR_TIMEOUT 5    /* a bounded device-side wait gave up           */
#define ECG_ERR_STATE 6      /* call order violated (e.g. no system set)     */

#define ECG_PREC_FP64 0      /* all-FP64 path                                 */
#define ECG_PREC_MIXED 1     /* reduced-precision tensor-core products + FP64 refinement */

/* Dot product of the CC DIIS (ecg_cc_opts.diis_dot). */
#define ECG_DIIS_CS 0        /* closed-shell custom dots of perform! (src/cc/cc.jl:2498-2499,2598) */
#define ECG_DIIS_PLAIN 1     /* plain dot (diis.jl:155-167), closed-shell CC before ElemCo.jl 0.13 */

typedef struct ecg_ctx ecg_ctx;

/* Options of the iterative solvers; mirrors CcOptions/DiisOptions
 * (src/infos/options.jl:128-282). */
typedef struct ecg_cc_opts {
  double thr;      /* squared residual norm threshold, default 1e-10 (options.jl:130) */
  double conven;   /* energy threshold factor, default 0.1 (options.jl:132)           */
  int32_t maxit;   /* default 50 (options.jl:134)                                     */
  double shifts;   /* singles level shift, default 0.15 (options.jl:136)              */
  double shiftp;   /* doubles level shift, default 0.2 (options.jl:138)               */
  int32_t maxdiis; /* default 6 (options.jl:274)                                      */
  double resthr;   /* default 10.0 (options.jl:276)                                   */
  int32_t diis_dot; /* ECG_DIIS_CS (default) or ECG_DIIS_PLAIN; CC iterations only    */
} ecg_cc_opts;

/* Fill *o with the reference defaults. */
void ecg_default_opts(ecg_cc_opts* o);

/* Context lifetime.  Replaces nothing in the reference (which has no device
 * state); the Julia glue wraps it in a finalizer. */
int ecg_create(int device, ecg_ctx** out);
int ecg_destroy(ecg_ctx* ctx);
const char* ecg_last_error(const ecg_ctx* ctx);
/* Cap the context's device memory (bytes, 0 = no cap); exceeding it returns
 * ECG_ERR_OOM.  Used to test the out-of-memory path without exhausting HBM. */
int ecg_set_mem_cap(ecg_ctx* ctx, uint64_t bytes);
int ecg_set_precision(ecg_ctx* ctx, int prec);

/* Context options (no counterpart in the reference), value 0 = automatic:
 *  ECG_OPT_TRIPLES_BATCH  at most this many occupied triplets per (T) batch
 *                         (one K slot each; the sweep's batches after the first
 *                         replay from one CUDA graph)
 *  ECG_OPT_TC_WAIT_NS     bound in ns on the tensor-core GEMM's main-loop
 *                         waits on this context's stream (default 1 s); a wait
 *                         that runs out makes the call return ECG_ERR_TIMEOUT
 *                         and the context stays usable (the kernel's final
 *                         waits on its own copies keep the 1 s bound)
 *  ECG_OPT_AUTOTUNE       1: GEMM shapes without an entry in the tuning table
 *                         are tuned on first use (see ecg_tune_save); 0: the
 *                         table's entries, else the fixed rules, are used.
 *                         The table is process-wide (all contexts and GPUs). */
#define ECG_OPT_TRIPLES_BATCH 1
#define ECG_OPT_TC_WAIT_NS 2
#define ECG_OPT_AUTOTUNE 3
int ecg_set_option(ecg_ctx* ctx, int32_t key, int64_t value);

/* GEMM autotuner table (no counterpart in the reference; the reference's
 * contractions run through TensorOperations/BLAS).  For each GEMM shape the
 * FP64 GEMM (TMA-staged tiles 64x64 / 128x64 / 64x128 / 128x128 or cp.async-
 * staged tiles 64x64 / 128x64 / 64x128, split-K count) and the tensor-core
 * GEMM (tile width 128 / 160 / 256 columns, split-K count within the FP32
 * accumulation bound) can choose from several configurations; with
 * ECG_OPT_AUTOTUNE on, the first call of a shape times each candidate on its
 * own operands (the result is unchanged) and records the fastest.
 * ecg_tune_save writes the table to a text file ("key value" lines),
 * ecg_tune_load merges such a file into it; *entries (may be NULL) receives
 * the table size afterwards. */
int ecg_tune_save(ecg_ctx* ctx, const char* path, int64_t* entries);
int ecg_tune_load(ecg_ctx* ctx, const char* path, int64_t* entries);

/* Upload the system.  B[p,q,Q] (n x n x nq) are the density-fitting factors
 * with (pq|rs) = sum_Q B[p,q,Q] B[r,s,Q] — the `mmL` file of
 * src/integrals/dftools.jl:92-134 / decomptools.jl:22-52; h1 (n x n) the
 * one-electron integrals and e0 the core energy (FDump int1/int0,
 * src/integrals/dump.jl:107-128).  Replaces the int2 build of
 * src/integrals/dfdump.jl:29-119 (the 4-index int2 is never formed). */
int ecg_set_system(ecg_ctx* ctx, int32_t no, int32_t nv, int32_t nq,
                   const double* B, const double* h1, double e0);

/* Fock matrix (n x n), orbital energies (n) and HF energy:
 * calc_fock_matrix / calc_HF_energy (src/cc/cctools.jl:35-78),
 * gen_fock (src/scf/fockfactory.jl:27-30). */
int ecg_fock(ecg_ctx* ctx, double* fock, double* eps, double* e_hf);

/* MP2 start amplitudes T1 (nv x no), T2 (nv x nv x no x no) and energy:
 * calc_MP2 (src/cc/cc.jl:1011-1024). */
int ecg_mp2(ecg_ctx* ctx, double* T1, double* T2, double* e_mp2);

/* One closed-shell CCSD (dc=0) or DCSD (dc=1) residual:
 * calc_cc_resid (src/cc/cc.jl:1343-1489). */
int ecg_cc_residual(ecg_ctx* ctx, int dc, const double* T1, const double* T2,
                    double* R1, double* R2);

/* Whole CC iteration loop on the device: cc_iterations! closed shell
 * (src/cc/cc.jl:2518-2656) with update_singles!/update_doubles!
 * (cctools.jl:265-300), DIIS perform! (src/solvers/diis.jl:246-305) and the
 * energies (cc.jl:97-249).  T1/T2 hold the start guess on entry and the
 * converged amplitudes on exit.  out[0] = Hylleraas correlation energy
 * ("E"), out[1] = same-spin, out[2] = opposite-spin part, out[3] = last
 * squared residual norm, out[4] = last energy change.  *iterations receives
 * the iteration count; *converged 1/0. */
int ecg_cc_solve(ecg_ctx* ctx, int dc, const ecg_cc_opts* opts, double* T1,
                 double* T2, double* out, int32_t* iterations, int32_t* converged);

/* Iteration-level interface used for benchmarking and for callers that keep
 * the loop on the host: load amplitudes into the context's device state,
 * run `nsteps` iterations of the cc_iterations! body (residual, Hylleraas
 * energy, update, DIIS, energy), read the amplitudes back.  Host pointers may
 * be NULL to skip the copy (device-resident amplitudes; ECG_ERR_STATE if the
 * context holds none for this system). */
int ecg_cc_load(ecg_ctx* ctx, const double* T1, const double* T2, const ecg_cc_opts* opts);
int ecg_cc_step(ecg_ctx* ctx, int dc, int32_t nsteps, double* out);
int ecg_cc_store(ecg_ctx* ctx, double* T1, double* T2);

/* Closed-shell (T) and [T]: calc_pertT_closed_shell
 * (src/cc/cc_triples.jl:39-157).  T1 and T2 may both be NULL to use the
 * amplitudes the context holds (those of the last ecg_mp2, ecg_cc_solve,
 * amplitude load or iteration on this system; ECG_ERR_STATE if there are
 * none), which skips their upload.  The same holds for ecg_lambda_pert_t. */
int ecg_pert_t(ecg_ctx* ctx, const double* T1, const double* T2, double* e_t,
               double* e_t_bracket);

/* Lambda equations.  ecg_lambda_residual: calc_ccsd_vector_times_Jacobian
 * closed shell (src/cc/cc_lagrange.jl:9-220) for multipliers U1/U2
 * (contravariant, as in the reference) at amplitudes T1/T2.
 * ecg_lambda_solve: lm_cc_iterations! (cc_lagrange.jl:1155-1223); U1/U2 are
 * outputs.  ecg_lambda_pert_t: calc_ΛpertT_closed_shell
 * (cc_triples.jl:159-295). */
int ecg_lambda_residual(ecg_ctx* ctx, int dc, const double* T1, const double* T2,
                        const double* U1, const double* U2, double* R1, double* R2);
int ecg_lambda_solve(ecg_ctx* ctx, int dc, const ecg_cc_opts* opts, const double* T1,
                     const double* T2, double* U1, double* U2, double* out,
                     int32_t* iterations, int32_t* converged);
int ecg_lambda_pert_t(ecg_ctx* ctx, const double* T1, const double* T2,
                      const double* U1, const double* U2, double* e_t,
                      double* e_t_bracket);

/* One-particle density matrices D1 and T1-dressed dD1 (n x n):
 * calc_1RDM closed shell (src/cc/cc_lagrange.jl:793-848). */
int ecg_one_rdm(ecg_ctx* ctx, const double* T1, const double* T2,
                const double* U1, const double* U2, double* D1, double* dD1);

/* Analytic gradient of the converged CCSD/DCSD energy with respect to the MO
 * one-electron matrix h (n x n, orbitals held fixed): G = dD1 + the HF
 * density (2 on the occupied diagonal), dD1 the T1-dressed 1RDM of
 * calc_1RDM (src/cc/cc_lagrange.jl:786-791) at converged amplitudes T1/T2 and
 * multipliers U1/U2 (ecg_lambda_solve).  For a one-electron perturbation
 * h + lambda P, dE/dlambda = sum_pq G[p,q] P[p,q].  The reference stops at
 * the densities; this contraction is the pullback behind the Julia/Python
 * rrule of the CC energy. */
int ecg_energy_gradient(ecg_ctx* ctx, const double* T1, const double* T2,
                        const double* U1, const double* U2, double* G);

/* Stand-alone DIIS on device vectors of length len (src/solvers/diis.jl:34-305,
 * plain dot).  Vectors are host arrays; the history stays on the device. */
typedef struct ecg_diis ecg_diis;
int ecg_diis_create(ecg_ctx* ctx, int32_t maxdiis, double resthr, int64_t len,
                    ecg_diis** out);
int ecg_diis_perform(ecg_diis* d, double* vec, const double* res);
int ecg_diis_destroy(ecg_diis* d);

/* One cc_iterations! body with host amplitudes: T1/T2 are uploaded (if
 * non-NULL), one iteration runs with the DIIS history kept in the context
 * (ecg_cc_load must have been called once), and the new amplitudes are
 * written back.  out as in ecg_cc_step. */
int ecg_cc_step_host(ecg_ctx* ctx, int dc, double* T1, double* T2, double* out);

/* ------------------------------------------------------------------------
 * Diagnostics and instrumentation (no counterpart in the reference).
 * ---------------------------------------------------------------------- */

/* The context's CUDA stream (a cudaStream_t), for callers that record their
 * own events around library calls. */
int ecg_get_stream(ecg_ctx* ctx, void** stream);

/* Number of kernels launched through the library in this process so far. */
int64_t ecg_kernel_launches(const ecg_ctx* ctx);

/* Kernel timing: when enabled, every launch of the FP64 GEMM, the tensor-core
 * GEMM and the (T) energy kernel in this process (outside CUDA graph
 * capture) is bracketed by CUDA events on its stream.  ecg_kernel_time
 * returns, for one family, the summed device milliseconds, the launch count
 * and the summed algorithmic work since the last read, and resets them:
 *   ECG_KT_DGEMM    FP64 GEMM (with its split-K reduction), flops 2*m*n*k*batch
 *   ECG_KT_TCGEMM   split-BF16 tcgen05 GEMM (kernel and split-K reduction),
 *                   BF16 product flops 2*m*n*k*(slice products)
 *   ECG_KT_TRIPLES  (T) energy kernel, bytes of K (and K of Lambda) read
 * ecg_gemm_time is ecg_kernel_time for ECG_KT_DGEMM. */
#define ECG_KT_DGEMM 0
#define ECG_KT_TCGEMM 1
#define ECG_KT_TRIPLES 2
int ecg_set_gemm_timing(ecg_ctx* ctx, int enable);
int ecg_gemm_time(ecg_ctx* ctx, double* ms, int64_t* launches, double* flops);
int ecg_kernel_time(ecg_ctx* ctx, int32_t family, double* ms, int64_t* launches,
                    double* work);

/* The library's GEMM / permutation on host buffers (column-major), for
 * self-tests of the device kernels:
 * C = alpha op(A) op(B) + beta C  with op 'N' or 'T'.  With the context's
 * precision set to ECG_PREC_MIXED the split-BF16 tensor-core GEMM is used. */
int ecg_diag_gemm(ecg_ctx* ctx, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
                  const double* A, int64_t lda, const double* B, int64_t ldb, double beta,
                  double* C, int64_t ldc);
/* out = alpha permute(in) + beta out, in of rank nd with dims in_dims; out
 * dimension d is input dimension perm[d]. */
int ecg_diag_permute(ecg_ctx* ctx, int nd, const int64_t* in_dims, const int* perm, double alpha,
                     const double* in, double beta, double* out);

/* ------------------------------------------------------------------------
 * Gaussian integrals (the molecular-integral producer of the DF-HF and
 * integral-transformation steps before the CC path).  A basis is a list of
 * contracted shells in plain arrays, as ElemCo.jl's BasisSet hands them to
 * libcint (src/system/libcint5.jl:25-81, src/system/basisset.jl):
 *   l[s]       angular momentum of shell s (0..4)
 *   nprim[s]   its primitives
 *   centre     3 doubles per shell (bohr)
 *   exps/coefs exponents and contraction coefficients, shell after shell, the
 *              coefficients multiplying normalised primitives as in the
 *              basis-set files
 * Functions are real solid harmonics (2l+1 per shell, m = -l..l) normalised
 * to unit self-overlap; outputs are column-major over them.  The engine is
 * McMurchie-Davidson on the GPU.
 * ---------------------------------------------------------------------- */
typedef struct ecg_shells {
  int32_t nshell;
  const int32_t* l;
  const int32_t* nprim;
  const double* centre;
  const double* exps;
  const double* coefs;
} ecg_shells;

/* Number of (spherical) basis functions. */
int ecg_shells_nbf(const ecg_shells* basis, int32_t* nbf);

/* One-electron integrals (n x n; ECG_INT_DIPOLE: three matrices x, y, z of
 * <m|(r - origin)|n>, origin NULL = 0): overlap, kinetic, nuclear attraction
 * over natom point charges, dipole.  The reference's overlap/kinetic/nuclear
 * (src/system/integrals_2idx.jl:11-100, libcint int1e_ovlp/kin/nuc). */
#define ECG_INT_OVERLAP 0
#define ECG_INT_KINETIC 1
#define ECG_INT_NUCLEAR 2
#define ECG_INT_DIPOLE 3
int ecg_int1e(ecg_ctx* ctx, int32_t kind, const ecg_shells* basis, int32_t natom,
              const double* charge, const double* atom_xyz, const double* origin, double* out);
/* Two-centre Coulomb metric (P|Q) of a fitting basis (naux x naux):
 * eri_2e2idx (src/system/integrals_2idx.jl, libcint int2c2e). */
int ecg_int2c2e(ecg_ctx* ctx, const ecg_shells* fit, double* out);
/* Three-centre Coulomb integrals (mn|P), out[m + nao*(n + nao*P)]:
 * eri_2e3idx (src/system/integrals_2e3idx.jl:108-158, libcint int3c2e). */
int ecg_int3c2e(ecg_ctx* ctx, const ecg_shells* ao, const ecg_shells* fit, double* out);

/* Density-fitted three-index factors kept on the device between calls:
 * AAL[m,n,L] = sum_P (mn|P) M[P,L], M (naux x nL, column-major) with
 * M M^T = (P|Q)^{-1} on the span kept (the caller's pivoted Cholesky of
 * ecg_int2c2e).  The reference's generate_AO_DF_integrals
 * (src/integrals/dftools.jl:28-84), which the reference writes to a file
 * `AAL`; here the factors stay in HBM (n^2 nL doubles, counted against the
 * context's memory cap) for the Fock builds of DF-HF and the MO transform.
 * The handle belongs to its context: destroy it before the context. */
typedef struct ecg_df ecg_df;
int ecg_df_create(ecg_ctx* ctx, const ecg_shells* ao, const ecg_shells* fit, const double* M,
                  int64_t nL, ecg_df** out);
/* Closed-shell DF Fock matrix in the AO basis, F = h + 2 J - K
 * (n x n, column-major) from the occupied orbitals Cocc (n x nocc):
 * LoA[L,j,n] = sum_m AAL[m,n,L] C[m,j], J = AAL . (sum LoA[L,j,n] C[n,j]),
 * K[m,n] = sum_{L,j} LoA[L,j,m] LoA[L,j,n] — the reference's gen_dffock
 * (src/scf/fockfactory.jl:202-245), which recomputes (mn|P) in batches for
 * every build.  nocc = 0 returns h. */
int ecg_df_fock(ecg_df* df, const double* h, const double* Cocc, int64_t nocc, double* F);
/* MO three-index factors B[p,q,L] = sum_{m,n} C[m,p] AAL[m,n,L] C[n,q]
 * (nmo x nmo x nL, column-major) of the orbitals C (n x nmo): the reference's
 * generate_3idx_integrals (src/integrals/dftools.jl:92-136, file `mmL`). */
int ecg_df_mo(ecg_df* df, const double* C, int64_t nmo, double* B);
int ecg_df_destroy(ecg_df* df);

/* ------------------------------------------------------------------------
 * Allocation-free entry point (no counterpart in the reference).
 *
 * For callers that must not allocate device memory in their call path — code
 * that runs under another framework's memory manager, inside CUDA stream
 * capture, or in a process whose device memory is already handed out.  It
 * computes C = alpha op(A) op(B) + beta C (column-major, op 'N' or 'T') on
 * DEVICE pointers with the library's FP64 split-K GEMM; the split-K partial
 * products go to a fixed 32 MiB device array inside the library (2^22
 * doubles; every GPU that loads the library holds it until process exit), so
 * m*n may be at most 4194304 (larger sizes return ECG_ERR_ARG).  The call
 * makes no cudaMalloc/cudaFree.  The first call on a device looks up that
 * array's device address (with the device current) and must come before any
 * stream capture on that device.  All calls share the one array, so calls
 * whose kernels overlap on the GPU (different streams, other threads) race
 * and give wrong results; every call overwrites the partial products it
 * reads, nothing needs to start at zero.  `stream` is a cudaStream_t (NULL =
 * legacy default stream); the call is asynchronous on it.  *nsplit (may be
 * NULL) receives the number of K slices used.
 * ---------------------------------------------------------------------- */
int ecg_gemm_noalloc(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
                     const double* A, int64_t lda, const double* B, int64_t ldb, double beta,
                     double* C, int64_t ldc, void* stream, int32_t* nsplit);

#ifdef __cplusplus
}
#endif
#endif /* ECGPU_H */
