// ecg_core.h — the context behind the C ABI: device-resident system,
// amplitudes, DIIS history and workspace for one closed-shell CC problem.
#pragma once
#include <cstdint>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include "../../include/ecgpu.h"
#include "ecg_dev.h"
#include "ecg_tensor.h"

namespace ecg {

// Device DIIS history (src/solvers/diis.jl:34-72), vectors in HBM.
struct DiisState {
  int maxdiis = 6;
  double resthr = 10.0;
  int next = 0, ndim = 0;
  int64_t len = 0;           // vector length
  std::vector<double*> amp;  // device slots
  std::vector<double*> res;
  std::vector<double> bmat;  // (maxdiis+1)^2, row-major on host
  bool cs = true;            // closed-shell custom dots vs plain dot
};

struct Ctx {
  int device = 0;
  dev::stream_t st = nullptr;
  std::string err;
  uint64_t memcap = 0, memused = 0;
  uint64_t handle_bytes = 0;  // device memory of handles (DF factors), part of memused
  std::vector<std::pair<void*, size_t>> allocs;
  uint64_t generation = 0;  // bumped whenever free_all() releases the system's buffers
  int prec = ECG_PREC_FP64;
  int64_t triples_batch = 0;  // ECG_OPT_TRIPLES_BATCH (0 = automatic)
  bool mixed_active = false;  // route large GEMMs to the split-BF16 tensor-core GEMM

  // system
  bool have_system = false;
  int no = 0, nv = 0, nq = 0, n = 0;
  double e0 = 0.0;
  Extents ext;
  // undressed DF factors, column-major blocks [p,q,Q]
  double *Bvv = nullptr, *Bov = nullptr, *Bvo = nullptr, *Boo = nullptr;
  double* h = nullptr;     // n x n
  double* fock = nullptr;  // n x n
  double* eps = nullptr;   // n
  double* klcd = nullptr;  // [k,l,c,d] = <kl|cd>
  double* Kvvoo = nullptr; // [a,b,i,j] = <ij|ab>
  double* fvo_t = nullptr; // [a,i] = f[i,a]
  std::vector<double> h_host, fock_host;

  // dressed quantities
  double *dBvv = nullptr, *dBvo = nullptr, *dBoo = nullptr, *dBvvT = nullptr;
  double *dh = nullptr, *dfock = nullptr, *J = nullptr;

  // amplitudes: T = [T1 (nv*no) | T2 (nv^2 no^2)], same for R
  double *T = nullptr, *R = nullptr;
  // T holds amplitudes of this system (from mp2, a load or the CC iterations)
  bool t_resident = false;
  double* TT = nullptr;  // outer-product scratch nv^2 no^2

  // device scalars + reduction scratch, pinned host mirror
  double* dscal = nullptr;
  double* red = nullptr;
  double* hscal = nullptr;
  double* dcoef = nullptr;

  Arena ws;
  double* ws_base = nullptr;
  // storage for BF16-split operands kept across GEMMs (mixed precision)
  void* tc_base = nullptr;
  size_t tc_bytes = 0;

  // ladder pair tables (device int pairs) and a-blocks
  int *cdp = nullptr, *ijp = nullptr, *pairs = nullptr;
  struct LadderBlock {
    int a0, na, npp, npm;
    int64_t poff;  // offset (in pairs) into `pairs`
  };
  std::vector<LadderBlock> lblocks;

  DiisState diis;
  ecg_cc_opts opts;

  // Lambda equations: U = [U1 | U2], RU its residual, vT = v_{mb}^{cd} T^{ij}_{cd}
  double *U = nullptr, *RU = nullptr, *vT = nullptr;
  double *D1 = nullptr, *dD1 = nullptr;  // n x n
  bool lambda_ready = false;
  DiisState ldiis;
  int64_t n1() const { return (int64_t)nv * no; }
  int64_t n2() const { return (int64_t)nv * nv * no * no; }
  double* T1() { return T; }
  double* T2() { return T + n1(); }
  double* R1() { return R; }
  double* R2() { return R + n1(); }

  double* alloc(int64_t ndoubles, const char* what);
  void release_to(size_t nallocs);  // free allocations made after the first nallocs
  void ensure_ws(int64_t ndoubles);  // grow the workspace arena (outside any capture)
  void* ensure_tc(size_t bytes);     // grow the split-operand storage (contents are lost)
  void free_all();
  Contractor con() { return Contractor(st, &ws, &ext, mixed_active); }
};

// ecg_cc.cpp
void setup_system(Ctx& c, int no, int nv, int nq, const double* B, const double* h1, double e0);
void dress(Ctx& c, const double* T1);                // dressed B, h, Fock (cc.jl:453-815)
void cc_residual(Ctx& c, bool dc);                   // R = residual(T)   (cc.jl:1343-1489)
// R2 += sum_cd (sum_Q Bf[a,c,Q] Bf[b,d,Q]) T2[c,d,i,j];  BfT[d,b,Q] = Bf[b,d,Q]
void ladder(Ctx& c, const double* Bf, const double* BfT, const double* T2, double* R2);
struct IterResult {
  double E, ESS, EOS, normR, dE, En;
};
void cc_init_iterations(Ctx& c, const ecg_cc_opts& o);
IterResult cc_iteration(Ctx& c, bool dc);
void diis_reset(Ctx& c, DiisState& d, int maxdiis, double resthr, int64_t len, bool cs);
// DIIS perform on device vectors (src/solvers/diis.jl:246-305)
void diis_perform(Ctx& c, DiisState& d, double* amps, const double* res);
double scal(Ctx& c, int i);
void sync_scalars(Ctx& c, int count);

// Runs f, turning the library's exceptions into a status code and a message
// (per context, or per thread for calls without one).
void noctx_error_store(const char* msg);  // the message ecg_last_error(NULL) returns
template <class F>
int guarded(Ctx* c, F&& f) {
  try {
    f();
    if (c) c->err.clear();
    return ECG_OK;
  } catch (const Error& e) {
    if (c) c->err = e.what();
    else noctx_error_store(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    if (c) c->err = "host out of memory";
    return ECG_ERR_OOM;
  } catch (const std::exception& e) {
    if (c) c->err = e.what();
    return ECG_ERR_ARG;
  }
}

}  // namespace ecg

struct ecg_ctx : ecg::Ctx {};
