// ecg_api.cpp — extern "C" entry points of libecgpu (declared in
// include/ecgpu.h).  Each call catches the library's exceptions and turns
// them into a status code plus a per-context message.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <new>

#include <cstdio>

#include "ecg_core.h"
#include "ecg_lambda.h"
#include "ecg_triples.h"
#include "ecg_tune.h"

using namespace ecg;

static thread_local std::string g_noctx_err;
void ecg::noctx_error_store(const char* msg) { g_noctx_err = msg; }

struct ecg_diis {
  ecg_ctx* ctx;
  uint64_t generation;  // the context's system generation its buffers belong to
  DiisState st;
  double* v;
  double* r;
};

static void need_system(Ctx& c) {
  if (!c.have_system) throw Error(ECG_ERR_STATE, "no system set (call ecg_set_system first)");
}

static void need_ptr(const void* p, const char* what) {
  if (!p) throw Error(ECG_ERR_ARG, std::string("NULL pointer: ") + what);
}

static void check_finite(const double* x, int64_t n, const char* what) {
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(x[i])) throw Error(ECG_ERR_NONFINITE, std::string("non-finite value in ") + what);
}

static void opts_or_default(const ecg_cc_opts* in, ecg_cc_opts& o) {
  if (in) o = *in;
  else ecg_default_opts(&o);
  if (o.maxdiis < 1 || o.maxdiis > 8) throw Error(ECG_ERR_ARG, "maxdiis must be in 1..8");
  if (o.maxit < 0) throw Error(ECG_ERR_ARG, "maxit must be >= 0");
  if (o.diis_dot != ECG_DIIS_CS && o.diis_dot != ECG_DIIS_PLAIN)
    throw Error(ECG_ERR_ARG, "diis_dot must be ECG_DIIS_CS or ECG_DIIS_PLAIN");
}

// Device scalar slot of the non-finite input flag.
constexpr int kFlagSlot = 255;

// Copies n host doubles to device memory d and checks them there (one pass
// over HBM instead of a host scan); a non-finite value raises
// ECG_ERR_NONFINITE after the copy.
static void h2d_finite(Ctx& c, double* d, const double* h, int64_t n, const char* what) {
  check(dev::h2d(d, h, n * 8, c.st), what);
  check(dev::nonfinite(c.st, n, d, c.dscal + kFlagSlot), what);
  check(dev::d2h(c.hscal + kFlagSlot, c.dscal + kFlagSlot, sizeof(double), c.st), "d2h flag");
  check(dev::sync(c.st), "sync");
  if (c.hscal[kFlagSlot] != 0.0)
    throw Error(ECG_ERR_NONFINITE, std::string("non-finite value in ") + what);
}

static void load_T(Ctx& c, const double* T1, const double* T2) {
  need_ptr(T1, "T1");
  need_ptr(T2, "T2");
  check_finite(T1, c.n1(), "T1");
  c.t_resident = false;
  check(dev::h2d(c.T1(), T1, c.n1() * 8, c.st), "h2d T1");
  h2d_finite(c, c.T2(), T2, c.n2(), "T2");
  c.t_resident = true;
}

// Host amplitudes, or (both NULL) the amplitudes the context holds.
static void load_T_or_resident(Ctx& c, const double* T1, const double* T2) {
  if (T1 || T2) return load_T(c, T1, T2);
  if (!c.t_resident)
    throw Error(ECG_ERR_STATE, "no amplitudes on the device: pass T1 and T2");
}

extern "C" {

void ecg_default_opts(ecg_cc_opts* o) {
  if (!o) return;
  o->thr = 1.0e-10;
  o->conven = 0.1;
  o->maxit = 50;
  o->shifts = 0.15;
  o->shiftp = 0.2;
  o->maxdiis = 6;
  o->resthr = 10.0;
  o->diis_dot = ECG_DIIS_CS;
}

int ecg_create(int device, ecg_ctx** out) {
  if (!out) return ECG_ERR_ARG;
  *out = nullptr;
  ecg_ctx* c = new (std::nothrow) ecg_ctx();
  if (!c) return ECG_ERR_OOM;
  int st = guarded(c, [&] {
    c->device = device;
    check(dev::set_device(device), "cudaSetDevice");
    check(dev::stream_create(&c->st), "cudaStreamCreate");
    ecg_default_opts(&c->opts);
  });
  if (st != ECG_OK) {
    g_noctx_err = c->err;
    delete c;
    return st;
  }
  *out = c;
  return ECG_OK;
}

int ecg_destroy(ecg_ctx* c) {
  if (!c) return ECG_OK;
  dev::set_device(c->device);
  c->free_all();
  if (c->st) dev::stream_destroy(c->st);
  delete c;
  return ECG_OK;
}

const char* ecg_last_error(const ecg_ctx* c) {
  if (!c) return g_noctx_err.c_str();
  return c->err.c_str();
}

int ecg_set_mem_cap(ecg_ctx* c, uint64_t bytes) {
  if (!c) return ECG_ERR_ARG;
  c->memcap = bytes;
  return ECG_OK;
}

int ecg_set_precision(ecg_ctx* c, int prec) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    if (prec != ECG_PREC_FP64 && prec != ECG_PREC_MIXED)
      throw Error(ECG_ERR_ARG, "precision must be ECG_PREC_FP64 or ECG_PREC_MIXED");
    c->prec = prec;
  });
}

int ecg_set_option(ecg_ctx* c, int32_t key, int64_t value) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    if (value < 0) throw Error(ECG_ERR_ARG, "option values must be >= 0");
    switch (key) {
      case ECG_OPT_TRIPLES_BATCH:
        c->triples_batch = value;
        break;
      case ECG_OPT_TC_WAIT_NS:
        check(dev::set_device(c->device), "cudaSetDevice");
        check(dev::set_tc_wait(c->st, (uint64_t)value), "set_tc_wait");
        break;
      case ECG_OPT_AUTOTUNE:
        dev::set_tuning(value != 0);
        break;
      default:
        throw Error(ECG_ERR_ARG, "unknown option key " + std::to_string(key));
    }
  });
}

int ecg_tune_save(ecg_ctx* c, const char* path, int64_t* entries) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_ptr(path, "path");
    FILE* f = std::fopen(path, "w");
    if (!f) throw Error(ECG_ERR_ARG, std::string("cannot write ") + path);
    const std::string text = dev::tune_dump();
    const size_t w = std::fwrite(text.data(), 1, text.size(), f);
    std::fclose(f);
    if (w != text.size()) throw Error(ECG_ERR_ARG, std::string("short write to ") + path);
    if (entries) *entries = (int64_t)dev::tune_size();
  });
}

int ecg_tune_load(ecg_ctx* c, const char* path, int64_t* entries) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_ptr(path, "path");
    FILE* f = std::fopen(path, "r");
    if (!f) throw Error(ECG_ERR_ARG, std::string("cannot read ") + path);
    std::string text;
    char buf[4096];
    size_t r;
    while ((r = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, r);
    std::fclose(f);
    if (dev::tune_parse(text) < 0) throw Error(ECG_ERR_ARG, std::string("bad tuning file ") + path);
    if (entries) *entries = (int64_t)dev::tune_size();
  });
}

int ecg_set_system(ecg_ctx* c, int32_t no, int32_t nv, int32_t nq, const double* B,
                   const double* h1, double e0) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_ptr(B, "B");
    need_ptr(h1, "h1");
    if (!std::isfinite(e0)) throw Error(ECG_ERR_NONFINITE, "non-finite e0");
    check(dev::set_device(c->device), "cudaSetDevice");
    setup_system(*c, no, nv, nq, B, h1, e0);
  });
}

int ecg_fock(ecg_ctx* c, double* fock, double* eps, double* e_hf) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    const int64_t n = c->n;
    if (fock) std::memcpy(fock, c->fock_host.data(), n * n * 8);
    if (eps)
      for (int64_t p = 0; p < n; ++p) eps[p] = c->fock_host[p + p * n];
    if (e_hf) {
      // calc_HF_energy closed shell (cctools.jl:65-72)
      double e = c->e0;
      for (int64_t i = 0; i < c->no; ++i) e += c->fock_host[i + i * n] + c->h_host[i + i * n];
      *e_hf = e;
    }
  });
}

int ecg_mp2(ecg_ctx* c, double* T1, double* T2, double* e_mp2) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    dev::stream_t s = c->st;
    const double* eo = c->eps;
    const double* ev = c->eps + c->no;
    // T2 = -<ab|ij>/D, T1 = -f[v,o]/D without level shift (cc.jl:1012-1017)
    check(dev::memset0(c->T, (c->n1() + c->n2()) * 8, s), "memset");
    check(dev::update_doubles(s, c->nv, c->no, eo, ev, 0.0, c->Kvvoo, c->T2()), "mp2 T2");
    check(dev::geam(s, c->nv, c->no, 1.0, c->fock + c->no, c->n, 0.0, c->R1(), c->nv), "fvo");
    check(dev::update_singles(s, c->nv, c->no, eo, ev, 0.0, c->R1(), c->T1()), "mp2 T1");
    check(dev::cs_dot(s, c->nv, c->no, c->T2(), c->Kvvoo, c->red, c->dscal), "mp2 e");
    check(dev::dot(s, c->n1(), c->fvo_t, c->T1(), c->red, c->dscal + 2), "mp2 e1");
    if (T1) check(dev::d2h(T1, c->T1(), c->n1() * 8, s), "d2h");
    if (T2) check(dev::d2h(T2, c->T2(), c->n2() * 8, s), "d2h");
    sync_scalars(*c, 3);
    c->t_resident = true;
    if (e_mp2) *e_mp2 = 2.0 * c->hscal[0] - c->hscal[1] + 2.0 * c->hscal[2];
  });
}

int ecg_cc_residual(ecg_ctx* c, int dc, const double* T1, const double* T2, double* R1,
                    double* R2) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    load_T(*c, T1, T2);
    cc_residual(*c, dc != 0);
    if (R1) check(dev::d2h(R1, c->R1(), c->n1() * 8, c->st), "d2h R1");
    if (R2) check(dev::d2h(R2, c->R2(), c->n2() * 8, c->st), "d2h R2");
    check(dev::sync(c->st), "sync");
  });
}

int ecg_cc_load(ecg_ctx* c, const double* T1, const double* T2, const ecg_cc_opts* opts) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    ecg_cc_opts o;
    opts_or_default(opts, o);
    load_T_or_resident(*c, T1, T2);
    cc_init_iterations(*c, o);
    check(dev::sync(c->st), "sync");
  });
}

int ecg_cc_step(ecg_ctx* c, int dc, int32_t nsteps, double* out) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    if (c->diis.len == 0) throw Error(ECG_ERR_STATE, "call ecg_cc_load first");
    IterResult r{};
    c->mixed_active = (c->prec == ECG_PREC_MIXED);
    struct Restore {
      Ctx& c;
      ~Restore() { c.mixed_active = false; }
    } restore{*c};
    for (int32_t k = 0; k < nsteps; ++k) r = cc_iteration(*c, dc != 0);
    if (out) {
      out[0] = r.E;
      out[1] = r.ESS;
      out[2] = r.EOS;
      out[3] = r.normR;
      out[4] = r.dE;
    }
  });
}

int ecg_cc_store(ecg_ctx* c, double* T1, double* T2) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    if (T1) check(dev::d2h(T1, c->T1(), c->n1() * 8, c->st), "d2h T1");
    if (T2) check(dev::d2h(T2, c->T2(), c->n2() * 8, c->st), "d2h T2");
    check(dev::sync(c->st), "sync");
  });
}

int ecg_cc_solve(ecg_ctx* c, int dc, const ecg_cc_opts* opts, double* T1, double* T2,
                 double* out, int32_t* iterations, int32_t* converged) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    ecg_cc_opts o;
    opts_or_default(opts, o);
    load_T(*c, T1, T2);
    cc_init_iterations(*c, o);
    const double thren = std::sqrt(o.thr) * o.conven;
    IterResult r{};
    int it = 0;
    bool conv = false;
    // ECG_PREC_MIXED: iterate with split-BF16 tensor-core products until the
    // squared residual is below 100 thr, then refine with FP64 iterations;
    // convergence is only declared on an FP64 residual.  (Running the mixed
    // phase down to thr itself was measured slower: more iterations in total.)
    bool mixed_phase = (c->prec == ECG_PREC_MIXED);
    struct Restore {
      Ctx& c;
      ~Restore() { c.mixed_active = false; }
    } restore{*c};
    for (it = 1; it <= o.maxit; ++it) {
      c->mixed_active = mixed_phase;
      r = cc_iteration(*c, dc != 0);
      if (mixed_phase) {
        if (r.normR < 100.0 * o.thr) mixed_phase = false;
        continue;
      }
      if (r.normR < o.thr && std::fabs(r.dE) < thren) {
        conv = true;
        break;
      }
    }
    if (it > o.maxit) it = o.maxit;
    check(dev::d2h(T1, c->T1(), c->n1() * 8, c->st), "d2h T1");
    check(dev::d2h(T2, c->T2(), c->n2() * 8, c->st), "d2h T2");
    check(dev::sync(c->st), "sync");
    if (out) {
      out[0] = r.E;
      out[1] = r.ESS;
      out[2] = r.EOS;
      out[3] = r.normR;
      out[4] = r.dE;
    }
    if (iterations) *iterations = it;
    if (converged) *converged = conv ? 1 : 0;
  });
}

int ecg_pert_t(ecg_ctx* c, const double* T1, const double* T2, double* e_t, double* e_tb) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    load_T_or_resident(*c, T1, T2);
    double et = 0, etb = 0;
    c->mixed_active = (c->prec == ECG_PREC_MIXED);
    struct Restore {
      Ctx& c;
      ~Restore() { c.mixed_active = false; }
    } restore{*c};
    pert_triples(*c, nullptr, nullptr, &et, &etb);
    if (e_t) *e_t = et;
    if (e_tb) *e_tb = etb;
  });
}

int ecg_lambda_pert_t(ecg_ctx* c, const double* T1, const double* T2, const double* U1,
                      const double* U2, double* e_t, double* e_tb) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    load_T_or_resident(*c, T1, T2);
    need_ptr(U1, "U1");
    need_ptr(U2, "U2");
    check_finite(U1, c->n1(), "U1");
    check_finite(U2, c->n2(), "U2");
    double et = 0, etb = 0;
    c->mixed_active = (c->prec == ECG_PREC_MIXED);
    struct Restore {
      Ctx& c;
      ~Restore() { c.mixed_active = false; }
    } restore{*c};
    pert_triples(*c, U1, U2, &et, &etb);
    if (e_t) *e_t = et;
    if (e_tb) *e_tb = etb;
  });
}

int ecg_lambda_residual(ecg_ctx* c, int dc, const double* T1, const double* T2, const double* U1,
                        const double* U2, double* R1, double* R2) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    load_T(*c, T1, T2);
    need_ptr(U1, "U1");
    need_ptr(U2, "U2");
    check_finite(U1, c->n1(), "U1");
    check_finite(U2, c->n2(), "U2");
    lambda_prepare(*c, dc != 0);
    lambda_load_U(*c, U1, U2);
    lambda_residual(*c, dc != 0);
    lambda_store_R(*c, R1, R2);
  });
}

int ecg_lambda_solve(ecg_ctx* c, int dc, const ecg_cc_opts* opts, const double* T1,
                     const double* T2, double* U1, double* U2, double* out, int32_t* iterations,
                     int32_t* converged) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    ecg_cc_opts o;
    opts_or_default(opts, o);
    load_T(*c, T1, T2);
    need_ptr(U1, "U1");
    need_ptr(U2, "U2");
    LambdaResult r = lambda_solve(*c, dc != 0, o);
    lambda_store_U(*c, U1, U2);
    if (out) {
      out[0] = r.norm;
      out[1] = r.normR;
      out[2] = r.dnorm;
    }
    if (iterations) *iterations = r.iterations;
    if (converged) *converged = r.converged ? 1 : 0;
  });
}

int ecg_one_rdm(ecg_ctx* c, const double* T1, const double* T2, const double* U1,
                const double* U2, double* D1, double* dD1) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    load_T(*c, T1, T2);
    need_ptr(U1, "U1");
    need_ptr(U2, "U2");
    lambda_load_U(*c, U1, U2);
    one_rdm(*c, D1, dD1);
  });
}

int ecg_energy_gradient(ecg_ctx* c, const double* T1, const double* T2, const double* U1,
                        const double* U2, double* G) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    need_ptr(G, "G");
    load_T(*c, T1, T2);
    need_ptr(U1, "U1");
    need_ptr(U2, "U2");
    lambda_load_U(*c, U1, U2);
    // correlation part: the 1RDM with all T1 terms; reference part: the
    // closed-shell HF density, 2 on the occupied diagonal
    one_rdm(*c, nullptr, G);
    const int64_t n = c->n;
    for (int64_t i = 0; i < c->no; ++i) G[i + n * i] += 2.0;
  });
}

int ecg_diis_create(ecg_ctx* c, int32_t maxdiis, double resthr, int64_t len, ecg_diis** out) {
  if (!c || !out) return ECG_ERR_ARG;
  *out = nullptr;
  ecg_diis* d = new (std::nothrow) ecg_diis();
  if (!d) return ECG_ERR_OOM;
  d->ctx = c;
  int st = guarded(c, [&] {
    need_system(*c);
    if (len <= 0) throw Error(ECG_ERR_ARG, "len must be positive");
    diis_reset(*c, d->st, maxdiis, resthr, len, false);
    d->generation = c->generation;
    d->v = c->alloc(len, "diis vec");
    d->r = c->alloc(len, "diis res");
  });
  if (st != ECG_OK) {
    delete d;
    return st;
  }
  *out = d;
  return ECG_OK;
}

int ecg_diis_perform(ecg_diis* d, double* vec, const double* res) {
  if (!d) return ECG_ERR_ARG;
  Ctx* c = d->ctx;
  return guarded(c, [&] {
    need_ptr(vec, "vec");
    need_ptr(res, "res");
    check_finite(vec, d->st.len, "vec");
    check_finite(res, d->st.len, "res");
    if (d->generation != c->generation)
      throw Error(ECG_ERR_STATE, "DIIS object belongs to an earlier system: set_system freed "
                                 "its buffers; create a new one");
    check(dev::h2d(d->v, vec, d->st.len * 8, c->st), "h2d");
    check(dev::h2d(d->r, res, d->st.len * 8, c->st), "h2d");
    diis_perform(*c, d->st, d->v, d->r);
    check(dev::d2h(vec, d->v, d->st.len * 8, c->st), "d2h");
    check(dev::sync(c->st), "sync");
  });
}

int ecg_diis_destroy(ecg_diis* d) {
  delete d;  // device slots belong to the context and are freed with it
  return ECG_OK;
}

int64_t ecg_kernel_launches(const ecg_ctx*) { return dev::launches(); }

// Allocation-free FP64 GEMM on device pointers (see include/ecgpu.h): argument
// checks on the host, then dev::gemm_splitk_noalloc, which uses only the
// library's static scratch array.
int ecg_gemm_noalloc(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
                     const double* A, int64_t lda, const double* B, int64_t ldb, double beta,
                     double* C, int64_t ldc, void* stream, int32_t* nsplit) {
  return guarded(nullptr, [&] {
    const bool at = (ta == 'T' || ta == 't'), bt = (tb == 'T' || tb == 't');
    if (!(at || ta == 'N' || ta == 'n') || !(bt || tb == 'N' || tb == 'n'))
      throw Error(ECG_ERR_ARG, "ta/tb must be 'N' or 'T'");
    if (m <= 0 || n <= 0 || k <= 0) throw Error(ECG_ERR_ARG, "m, n, k must be positive");
    need_ptr(A, "A");
    need_ptr(B, "B");
    need_ptr(C, "C");
    if (lda < (at ? k : m) || ldb < (bt ? n : k) || ldc < m)
      throw Error(ECG_ERR_ARG, "leading dimension too small");
    const uint64_t cap = dev::noalloc_scratch_doubles();
    if ((uint64_t)n > cap / (uint64_t)m)  // m*n > cap, without forming the product
      throw Error(ECG_ERR_ARG, "m*n = " + std::to_string(m) + "*" + std::to_string(n) +
                                   " exceeds the allocation-free scratch (" +
                                   std::to_string(cap) + " output elements)");
    int S = 0;
    int e = dev::gemm_splitk_noalloc(stream, at ? 'T' : 'N', bt ? 'T' : 'N', m, n, k, alpha, A,
                                     lda, B, ldb, beta, C, ldc, &S);
    check(e, "ecg_gemm_noalloc");
    if (nsplit) *nsplit = S;
  });
}

int ecg_cc_step_host(ecg_ctx* c, int dc, double* T1, double* T2, double* out) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_system(*c);
    if (c->diis.len == 0) throw Error(ECG_ERR_STATE, "call ecg_cc_load first");
    if (T1 && T2) load_T(*c, T1, T2);
    IterResult r = cc_iteration(*c, dc != 0);
    if (T1) check(dev::d2h(T1, c->T1(), c->n1() * 8, c->st), "d2h T1");
    if (T2) check(dev::d2h(T2, c->T2(), c->n2() * 8, c->st), "d2h T2");
    check(dev::sync(c->st), "sync");
    if (out) {
      out[0] = r.E;
      out[1] = r.ESS;
      out[2] = r.EOS;
      out[3] = r.normR;
      out[4] = r.dE;
    }
  });
}

int ecg_get_stream(ecg_ctx* c, void** stream) {
  if (!c || !stream) return ECG_ERR_ARG;
  *stream = c->st;
  return ECG_OK;
}

int ecg_set_gemm_timing(ecg_ctx* c, int enable) {
  if (!c) return ECG_ERR_ARG;
  dev::gemm_timing(enable != 0);
  return ECG_OK;
}

int ecg_kernel_time(ecg_ctx* c, int32_t family, double* ms, int64_t* launches, double* work) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    if (family < 0 || family >= dev::KT_FAMILIES) throw Error(ECG_ERR_ARG, "unknown family");
    check(dev::sync(c->st), "sync");
    dev::kernel_time(family, ms, launches, work);
  });
}

int ecg_gemm_time(ecg_ctx* c, double* ms, int64_t* launches, double* flops) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    check(dev::sync(c->st), "sync");
    dev::gemm_time(ms, launches, flops);
  });
}

int ecg_diag_gemm(ecg_ctx* c, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
                  const double* A, int64_t lda, const double* B, int64_t ldb, double beta,
                  double* C, int64_t ldc) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    need_ptr(A, "A");
    need_ptr(B, "B");
    need_ptr(C, "C");
    if (m < 0 || n < 0 || k < 0) throw Error(ECG_ERR_ARG, "negative dimension");
    const bool at = (ta == 'T' || ta == 't'), bt = (tb == 'T' || tb == 't');
    const int64_t ar = at ? k : m, ac = at ? m : k, br = bt ? n : k, bc = bt ? k : n;
    if (lda < std::max<int64_t>(1, ar) || ldb < std::max<int64_t>(1, br) ||
        ldc < std::max<int64_t>(1, m))
      throw Error(ECG_ERR_ARG, "leading dimension too small");
    const size_t sA = lda * ac, sB = ldb * bc, sC = ldc * n;
    size_t n0 = c->allocs.size();
    struct Scope {
      Ctx& c;
      size_t n0;
      ~Scope() { c.release_to(n0); }
    } scope{*c, n0};
    double* dA = c->alloc(sA, "diag A");
    double* dB = c->alloc(sB, "diag B");
    double* dC = c->alloc(sC, "diag C");
    check(dev::h2d(dA, A, sA * 8, c->st), "h2d");
    check(dev::h2d(dB, B, sB * 8, c->st), "h2d");
    check(dev::h2d(dC, C, sC * 8, c->st), "h2d");
    if (c->prec == ECG_PREC_MIXED)
      check(dev::gemm_mixed(c->st, ta, tb, m, n, k, alpha, dA, lda, dB, ldb, beta, dC, ldc),
            "gemm_mixed");
    else
      check(dev::gemm(c->st, ta, tb, m, n, k, alpha, dA, lda, dB, ldb, beta, dC, ldc), "gemm");
    check(dev::d2h(C, dC, sC * 8, c->st), "d2h");
    check(dev::sync(c->st), "sync");
    int tc = 0;
    check(dev::tc_error(&tc), "tc_error");
    if (tc) throw Error(ECG_ERR_TIMEOUT, "GEMM wait timed out (code " +
                                             std::to_string(tc) + ")");
  });
}

int ecg_diag_permute(ecg_ctx* c, int nd, const int64_t* in_dims, const int* perm, double alpha,
                     const double* in, double beta, double* out) {
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    if (nd < 1 || nd > 8) throw Error(ECG_ERR_ARG, "rank must be 1..8");
    need_ptr(in_dims, "in_dims");
    need_ptr(perm, "perm");
    int64_t total = 1;
    bool seen[8] = {false};
    for (int d = 0; d < nd; ++d) {
      if (in_dims[d] < 0 || perm[d] < 0 || perm[d] >= nd || seen[perm[d]])
        throw Error(ECG_ERR_ARG, "bad dims or permutation");
      seen[perm[d]] = true;
      total *= in_dims[d];
    }
    size_t n0 = c->allocs.size();
    struct Scope {
      Ctx& c;
      size_t n0;
      ~Scope() { c.release_to(n0); }
    } scope{*c, n0};
    double* di = c->alloc(total, "diag in");
    double* dout = c->alloc(total, "diag out");
    check(dev::h2d(di, in, total * 8, c->st), "h2d");
    check(dev::h2d(dout, out, total * 8, c->st), "h2d");
    check(dev::permute(c->st, nd, in_dims, perm, alpha, di, beta, dout), "permute");
    check(dev::d2h(out, dout, total * 8, c->st), "d2h");
    check(dev::sync(c->st), "sync");
  });
}

}  // extern "C"
