// ecg_ints.cpp — C ABI of the integral engine (declared in include/ecgpu.h):
// shells from the caller's plain arrays, Cartesian integrals on the GPU
// (dev_ints.cu), transformation to real solid harmonics and normalisation;
// and the density-fitted factors kept on the device (ecg_df_*) for the DF-HF
// Fock builds and the MO transform of the CC integrals.
//
// Contraction coefficients are those of the basis-set files, which multiply
// normalised primitives: the engine uses c_k a_k^{(2l+3)/4} (the l-dependent
// constant of the primitive norm is common to a shell and drops out with the
// final normalisation), as ElemCo.jl does (src/system/basiscentre.jl:300-311).
// Spherical functions are the real solid harmonics S_lm (m = -l..l) of
// Helgaker, Jorgensen and Olsen, "Molecular Electronic-Structure Theory",
// eq. (6.4.47)-(6.4.50), each scaled to unit self-overlap.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ecg_core.h"

using namespace ecg;

namespace {

int ncart(int l) { return (l + 1) * (l + 2) / 2; }

double binom(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double r = 1.0;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

double fact(int n) {
  double r = 1.0;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}

int cart_index(int l, int i, int j) {
  // components ordered i = l..0, then j = l-i..0
  int n = 0;
  for (int a = l; a > i; --a) n += l - a + 1;
  return n + (l - i - j);
}

// Rows m = -l..l of the (2l+1) x ncart(l) matrix of S_lm in Cartesian
// monomials x^i y^j z^k (column cart_index(l, i, j)).
std::vector<double> solid_harmonics(int l) {
  const int nc = ncart(l);
  std::vector<double> M((2 * l + 1) * nc, 0.0);
  for (int m = -l; m <= l; ++m) {
    const int am = std::abs(m);
    const int dm = m < 0 ? 1 : 0;  // 2 v_m
    const double N = 1.0 / (std::pow(2.0, am) * fact(l)) *
                     std::sqrt(2.0 * fact(l + am) * fact(l - am) / (m == 0 ? 2.0 : 1.0));
    for (int t = 0; t <= (l - am) / 2; ++t)
      for (int u = 0; u <= t; ++u)
        for (int k = dm; k <= am; k += 2) {  // k = 2v
          const int sgn = ((t + (k - dm) / 2) & 1) ? -1 : 1;
          const double C = sgn * std::pow(0.25, t) * binom(l, t) * binom(l - t, am + t) *
                           binom(t, u) * binom(am, k);
          const int px = 2 * t + am - 2 * u - k, py = 2 * u + k, pz = l - 2 * t - am;
          if (px < 0 || pz < 0) continue;
          M[(m + l) * nc + cart_index(l, px, py)] += N * C;
        }
  }
  return M;
}

struct Basis {
  std::vector<dev::IntShell> sh;
  std::vector<double> ex, co;
  int ncart = 0, nsph = 0;
  std::vector<int> sph_off;
};

Basis make_basis(const ecg_shells* b, int prim_base, int cart_base) {
  if (!b || b->nshell < 0) throw Error(ECG_ERR_ARG, "NULL or empty shell list");
  if (b->nshell > 0 && (!b->l || !b->nprim || !b->centre || !b->exps || !b->coefs))
    throw Error(ECG_ERR_ARG, "NULL shell array");
  Basis B;
  int poff = prim_base;
  for (int s = 0; s < b->nshell; ++s) {
    const int l = b->l[s], np = b->nprim[s];
    if (l < 0 || l > dev::INT_LMAX)
      throw Error(ECG_ERR_ARG, "shell angular momentum must be 0.." +
                                   std::to_string(dev::INT_LMAX));
    if (np <= 0) throw Error(ECG_ERR_ARG, "shell without primitives");
    dev::IntShell q{b->centre[3 * s], b->centre[3 * s + 1], b->centre[3 * s + 2], l, np, poff,
                    cart_base + B.ncart};
    if (!std::isfinite(q.x) || !std::isfinite(q.y) || !std::isfinite(q.z))
      throw Error(ECG_ERR_NONFINITE, "non-finite shell centre");
    for (int k = 0; k < np; ++k) {
      const double a = b->exps[poff - prim_base + k], c = b->coefs[poff - prim_base + k];
      if (!(a > 0.0) || !std::isfinite(a) || !std::isfinite(c))
        throw Error(ECG_ERR_ARG, "exponents must be positive and finite");
      B.ex.push_back(a);
      B.co.push_back(c * std::pow(a, (2 * l + 3) / 4.0));
    }
    B.sh.push_back(q);
    B.sph_off.push_back(B.nsph);
    B.ncart += ncart(l);
    B.nsph += 2 * l + 1;
    poff += np;
  }
  return B;
}

// T (nsph x ncart, column-major): block-diagonal solid-harmonic transform.
std::vector<double> sph_transform(const Basis& B) {
  std::vector<double> T((size_t)B.nsph * B.ncart, 0.0);
  int c0 = 0;
  for (size_t s = 0; s < B.sh.size(); ++s) {
    const int l = B.sh[s].l, nc = ncart(l);
    const std::vector<double> M = solid_harmonics(l);
    for (int r = 0; r < 2 * l + 1; ++r)
      for (int c = 0; c < nc; ++c) T[(B.sph_off[s] + r) + (size_t)B.nsph * (c0 + c)] = M[r * nc + c];
    c0 += nc;
  }
  return T;
}

// out (ns x ns) = T X T^T for X (nc x nc) on the host, T = sph_transform(B):
// T is block diagonal (shell by shell), so each product runs over one shell's
// Cartesian components only (O(nc * sum_s ns_s nc_s) instead of O(ns nc^2)).
void transform2(const Basis& B, const std::vector<double>& T, const double* X, double* out) {
  const int64_t ns = B.nsph, nc = B.ncart;
  std::vector<double> Y((size_t)ns * nc);  // Y = T X
  int64_t c0 = 0;
  for (size_t s = 0; s < B.sh.size(); ++s) {
    const int64_t l = B.sh[s].l, ncs = ncart((int)l), r0 = B.sph_off[s];
    for (int64_t j = 0; j < nc; ++j)
      for (int64_t i = 0; i < 2 * l + 1; ++i) {
        double acc = 0.0;
        for (int64_t k = 0; k < ncs; ++k) acc += T[(r0 + i) + ns * (c0 + k)] * X[(c0 + k) + nc * j];
        Y[(r0 + i) + ns * j] = acc;
      }
    c0 += ncs;
  }
  c0 = 0;
  for (size_t s = 0; s < B.sh.size(); ++s) {
    const int64_t l = B.sh[s].l, ncs = ncart((int)l), r0 = B.sph_off[s];
    for (int64_t j = 0; j < 2 * l + 1; ++j)
      for (int64_t i = 0; i < ns; ++i) {
        double acc = 0.0;
        for (int64_t k = 0; k < ncs; ++k) acc += Y[i + ns * (c0 + k)] * T[(r0 + j) + ns * (c0 + k)];
        out[i + ns * (r0 + j)] = acc;
      }
    c0 += ncs;
  }
}

// Device copies of shells and primitives (released by the caller's scope).
struct DevBasis {
  dev::IntShell* sh = nullptr;
  double* ex = nullptr;
  double* co = nullptr;
};

DevBasis upload(Ctx& c, const std::vector<dev::IntShell>& sh, const std::vector<double>& ex,
                const std::vector<double>& co) {
  DevBasis d;
  d.sh = (dev::IntShell*)c.alloc(((int64_t)(sh.size() * sizeof(dev::IntShell)) + 7) / 8 + 1,
                                 "shells");
  d.ex = c.alloc((int64_t)ex.size() + 1, "exponents");
  d.co = c.alloc((int64_t)co.size() + 1, "coefficients");
  check(dev::h2d(d.sh, sh.data(), sh.size() * sizeof(dev::IntShell), c.st), "h2d shells");
  check(dev::h2d(d.ex, ex.data(), ex.size() * 8, c.st), "h2d exponents");
  check(dev::h2d(d.co, co.data(), co.size() * 8, c.st), "h2d coefficients");
  return d;
}

struct Scope {
  Ctx& c;
  size_t n0;
  ~Scope() { c.release_to(n0); }
};

// Spherical one-electron matrix of kind (0 S, 1 T, 2 V, 3 dipole: ncomp 3)
// before normalisation; returns it in out (ncomp x nsph^2).
void one_electron(Ctx& c, const Basis& B, int kind, int natom, const double* Z,
                  const double* xyz, const double* origin, std::vector<double>& out) {
  const int ncomp = kind == 3 ? 3 : 1;
  const int64_t nc = B.ncart, ns = B.nsph;
  Scope scope{c, c.allocs.size()};
  DevBasis d = upload(c, B.sh, B.ex, B.co);
  double* dZ = nullptr;
  double* dX = nullptr;
  if (kind == 2) {
    dZ = c.alloc(natom + 1, "charges");
    dX = c.alloc(3 * natom + 1, "atom xyz");
    check(dev::h2d(dZ, Z, natom * 8, c.st), "h2d");
    check(dev::h2d(dX, xyz, 3 * natom * 8, c.st), "h2d");
  }
  double* dout = c.alloc(ncomp * nc * nc, "int1e");
  check(dev::memset0(dout, ncomp * nc * nc * 8, c.st), "memset");
  check(dev::int1e_cart(c.st, kind, d.sh, (int)B.sh.size(), d.ex, d.co, natom, dZ, dX, origin,
                        nc, dout),
        "int1e");
  std::vector<double> cart(ncomp * nc * nc);
  check(dev::d2h(cart.data(), dout, cart.size() * 8, c.st), "d2h");
  check(dev::sync(c.st), "sync");
  const std::vector<double> T = sph_transform(B);
  out.assign(ncomp * ns * ns, 0.0);
  for (int q = 0; q < ncomp; ++q)
    transform2(B, T, cart.data() + q * nc * nc, out.data() + q * ns * ns);
}

// 1 / sqrt of the spherical self-overlaps
std::vector<double> norms(Ctx& c, const Basis& B) {
  std::vector<double> S;
  one_electron(c, B, 0, 0, nullptr, nullptr, nullptr, S);
  std::vector<double> d(B.nsph);
  for (int i = 0; i < B.nsph; ++i) {
    const double s = S[i + (size_t)B.nsph * i];
    if (!(s > 0.0)) throw Error(ECG_ERR_ARG, "basis function of zero norm");
    d[i] = 1.0 / std::sqrt(s);
  }
  return d;
}

void check_ltot(const Basis& a, const Basis* b, const Basis& c) {
  int la = 0, lb = 0, lc = 0;
  for (auto& s : a.sh) la = std::max(la, s.l);
  if (b)
    for (auto& s : b->sh) lb = std::max(lb, s.l);
  for (auto& s : c.sh) lc = std::max(lc, s.l);
  if (la + lb + lc > dev::INT_LTOT)
    throw Error(ECG_ERR_ARG, "angular momenta too high for the integral engine (sum of shell "
                             "l above " + std::to_string(dev::INT_LTOT) + ")");
}

// (mn|P) of ao x ao x fit on the device, spherical and normalised, as
// Z[m + nao*(n + nao*P)] in an allocation of c's stack (with the
// intermediates below it: the caller's scope releases them all).
double* int3c2e_device(Ctx& c, const ecg_shells* ao, const ecg_shells* fit, int64_t* nao,
                       int64_t* naux) {
  const Basis A = make_basis(ao, 0, 0);
  // P0: the fitting basis on its own (normalisation, transform); P: the same
  // shells with primitive offsets past A's, for the kernel's joint arrays
  const Basis P0 = make_basis(fit, 0, 0);
  const Basis P = make_basis(fit, (int)A.ex.size(), 0);
  check_ltot(A, &A, P);
  const std::vector<double> dA = norms(c, A), dP = norms(c, P0);
  std::vector<double> TA = sph_transform(A), TP = sph_transform(P0);
  for (int64_t k = 0; k < A.ncart; ++k)
    for (int64_t i = 0; i < A.nsph; ++i) TA[i + A.nsph * k] *= dA[i];
  for (int64_t k = 0; k < P.ncart; ++k)
    for (int64_t i = 0; i < P.nsph; ++i) TP[i + P.nsph * k] *= dP[i];
  const int64_t na = A.ncart, np = P.ncart, sa = A.nsph, sp = P.nsph;
  std::vector<double> ex(A.ex), co(A.co);
  ex.insert(ex.end(), P.ex.begin(), P.ex.end());
  co.insert(co.end(), P.co.begin(), P.co.end());
  DevBasis dao = upload(c, A.sh, ex, co);
  DevBasis daux = upload(c, P.sh, {}, {});
  double* X = c.alloc(na * na * np, "int3c cart");
  check(dev::memset0(X, na * na * np * 8, c.st), "memset");
  check(dev::int3c2e_cart(c.st, dao.sh, (int)A.sh.size(), daux.sh, (int)P.sh.size(), dao.ex,
                          dao.co, na, X),
        "int3c2e");
  double* dTA = c.alloc(sa * na, "TA");
  double* dTP = c.alloc(sp * np, "TP");
  check(dev::h2d(dTA, TA.data(), TA.size() * 8, c.st), "h2d");
  check(dev::h2d(dTP, TP.data(), TP.size() * 8, c.st), "h2d");
  // Y1[m,n,P] = sum_Pc X[m,n,Pc] TP[P,Pc]
  double* Y1 = c.alloc(na * na * sp, "int3c 1");
  check(dev::gemm(c.st, 'N', 'T', na * na, sp, np, 1.0, X, na * na, dTP, sp, 0.0, Y1, na * na),
        "gemm P");
  // Y2[m,n',P] = sum_n Y1[m,n,P] TA[n',n]  (batched over P)
  double* Y2 = c.alloc(na * sa * sp, "int3c 2");
  check(dev::gemm(c.st, 'N', 'T', na, sa, na, 1.0, Y1, na, dTA, sa, 0.0, Y2, na, sp, na * na, 0,
                  na * sa),
        "gemm n");
  // Z[m',n',P] = sum_m TA[m',m] Y2[m,n',P]
  double* Z = c.alloc(sa * sa * sp, "int3c 3");
  check(dev::gemm(c.st, 'N', 'N', sa, sa * sp, na, 1.0, dTA, sa, Y2, na, 0.0, Z, sa), "gemm m");
  *nao = sa;
  *naux = sp;
  return Z;
}

}  // namespace

// Density-fitted three-index factors held on the device between calls.
struct ecg_df {
  ecg_ctx* ctx = nullptr;
  double* aal = nullptr;  // AAL[m + n*(m' + n*L)], n = nao
  size_t bytes = 0;
  int64_t n = 0, nL = 0;
};

extern "C" {

int ecg_shells_nbf(const ecg_shells* b, int32_t* nbf) {
  if (!b || !nbf || b->nshell < 0) return ECG_ERR_ARG;
  if (b->nshell > 0 && !b->l) return ECG_ERR_ARG;
  int32_t n = 0;
  for (int s = 0; s < b->nshell; ++s) {
    if (b->l[s] < 0 || b->l[s] > dev::INT_LMAX) return ECG_ERR_ARG;
    n += 2 * b->l[s] + 1;
  }
  *nbf = n;
  return ECG_OK;
}

int ecg_int1e(ecg_ctx* ctx, int32_t kind, const ecg_shells* b, int32_t natom,
              const double* charge, const double* atom_xyz, const double* origin, double* out) {
  Ctx* c = ctx;
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    if (kind < ECG_INT_OVERLAP || kind > ECG_INT_DIPOLE) throw Error(ECG_ERR_ARG, "unknown kind");
    if (!out) throw Error(ECG_ERR_ARG, "NULL output");
    if (kind == ECG_INT_NUCLEAR && (natom <= 0 || !charge || !atom_xyz))
      throw Error(ECG_ERR_ARG, "nuclear attraction needs natom > 0, charges and positions");
    check(dev::set_device(c->device), "cudaSetDevice");
    const Basis B = make_basis(b, 0, 0);
    const int kd = kind == ECG_INT_OVERLAP ? 0 : kind == ECG_INT_KINETIC ? 1
                   : kind == ECG_INT_NUCLEAR ? 2 : 3;
    const double zero[3] = {0.0, 0.0, 0.0};
    std::vector<double> M;
    one_electron(*c, B, kd, natom, charge, atom_xyz, origin ? origin : zero, M);
    const std::vector<double> d = norms(*c, B);
    const int64_t n = B.nsph;
    const int ncomp = kd == 3 ? 3 : 1;
    for (int q = 0; q < ncomp; ++q)
      for (int64_t j = 0; j < n; ++j)
        for (int64_t i = 0; i < n; ++i)
          out[q * n * n + i + n * j] = M[q * n * n + i + n * j] * d[i] * d[j];
  });
}

int ecg_int2c2e(ecg_ctx* ctx, const ecg_shells* fit, double* out) {
  Ctx* c = ctx;
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    if (!out) throw Error(ECG_ERR_ARG, "NULL output");
    check(dev::set_device(c->device), "cudaSetDevice");
    const Basis P = make_basis(fit, 0, 0);
    check_ltot(P, nullptr, P);
    const int64_t nc = P.ncart, ns = P.nsph;
    std::vector<double> cart(nc * nc);
    {
      Scope scope{*c, c->allocs.size()};
      DevBasis d = upload(*c, P.sh, P.ex, P.co);
      double* dout = c->alloc(nc * nc, "int2c");
      check(dev::memset0(dout, nc * nc * 8, c->st), "memset");
      check(dev::int2c2e_cart(c->st, d.sh, (int)P.sh.size(), d.ex, d.co, nc, dout), "int2c2e");
      check(dev::d2h(cart.data(), dout, cart.size() * 8, c->st), "d2h");
      check(dev::sync(c->st), "sync");
    }
    const std::vector<double> T = sph_transform(P);
    const std::vector<double> d = norms(*c, P);
    transform2(P, T, cart.data(), out);
    for (int64_t j = 0; j < ns; ++j)
      for (int64_t i = 0; i < ns; ++i) out[i + ns * j] *= d[i] * d[j];
  });
}

int ecg_int3c2e(ecg_ctx* ctx, const ecg_shells* ao, const ecg_shells* fit, double* out) {
  Ctx* c = ctx;
  if (!c) return ECG_ERR_ARG;
  return guarded(c, [&] {
    if (!out) throw Error(ECG_ERR_ARG, "NULL output");
    check(dev::set_device(c->device), "cudaSetDevice");
    Scope scope{*c, c->allocs.size()};
    int64_t n = 0, naux = 0;
    const double* Z = int3c2e_device(*c, ao, fit, &n, &naux);
    check(dev::d2h(out, Z, n * n * naux * 8, c->st), "d2h");
    check(dev::sync(c->st), "sync");
  });
}

int ecg_df_create(ecg_ctx* ctx, const ecg_shells* ao, const ecg_shells* fit, const double* M,
                  int64_t nL, ecg_df** out) {
  Ctx* c = ctx;
  if (!c || !out) return ECG_ERR_ARG;
  *out = nullptr;
  ecg_df* d = new (std::nothrow) ecg_df();
  if (!d) return ECG_ERR_OOM;
  d->ctx = ctx;
  const int st = guarded(c, [&] {
    if (!M) throw Error(ECG_ERR_ARG, "NULL fitting matrix");
    if (nL <= 0) throw Error(ECG_ERR_ARG, "nL must be positive");
    int32_t nao = 0, naux = 0;
    if (ecg_shells_nbf(ao, &nao) != ECG_OK || ecg_shells_nbf(fit, &naux) != ECG_OK)
      throw Error(ECG_ERR_ARG, "invalid basis");
    if (nL > naux) throw Error(ECG_ERR_ARG, "nL exceeds the fitting basis");
    check(dev::set_device(c->device), "cudaSetDevice");
    d->n = nao;
    d->nL = nL;
    d->bytes = (size_t)std::max<int64_t>((int64_t)nao * nao * nL, 1) * 8;
    if (c->memcap && c->memused + d->bytes > c->memcap)
      throw Error(ECG_ERR_OOM, "device memory cap exceeded allocating the DF factors");
    d->aal = (double*)dev::dmalloc(d->bytes);
    if (!d->aal) throw Error(ECG_ERR_OOM, "cudaMalloc failed for the DF factors");
    c->memused += d->bytes;
    c->handle_bytes += d->bytes;
    Scope scope{*c, c->allocs.size()};
    int64_t n = 0, np = 0;
    const double* Z = int3c2e_device(*c, ao, fit, &n, &np);
    double* dM = c->alloc(np * nL, "fitting matrix");
    check(dev::h2d(dM, M, np * nL * 8, c->st), "h2d");
    // AAL[mn, L] = sum_P (mn|P) M[P, L]
    check(dev::gemm(c->st, 'N', 'N', n * n, nL, np, 1.0, Z, n * n, dM, np, 0.0, d->aal, n * n),
          "gemm AAL");
    check(dev::sync(c->st), "sync");
  });
  if (st != ECG_OK) {
    ecg_df_destroy(d);
    return st;
  }
  *out = d;
  return ECG_OK;
}

int ecg_df_fock(ecg_df* d, const double* h, const double* Cocc, int64_t nocc, double* F) {
  if (!d) return ECG_ERR_ARG;
  Ctx* c = d->ctx;
  return guarded(c, [&] {
    if (!h || !F || (nocc > 0 && !Cocc)) throw Error(ECG_ERR_ARG, "NULL argument");
    if (nocc < 0 || nocc > d->n) throw Error(ECG_ERR_ARG, "nocc out of range");
    check(dev::set_device(c->device), "cudaSetDevice");
    const int64_t n = d->n, nL = d->nL;
    Scope scope{*c, c->allocs.size()};
    double* dF = c->alloc(n * n, "Fock");
    check(dev::h2d(dF, h, n * n * 8, c->st), "h2d");
    if (nocc > 0) {
      double* dC = c->alloc(n * nocc, "occupied orbitals");
      double* Ct = c->alloc(n * nocc, "occupied orbitals^T");
      double* Y = c->alloc(nocc * n * nL, "LoA");
      double* Yp = c->alloc(nocc * n * nL, "LoA permuted");
      double* cL = c->alloc(nL, "cL");
      check(dev::h2d(dC, Cocc, n * nocc * 8, c->st), "h2d");
      // Y[j, nu, L] = sum_mu C[mu, j] AAL[mu, nu, L]
      check(dev::gemm(c->st, 'T', 'N', nocc, n * nL, n, 1.0, dC, n, d->aal, n, 0.0, Y, nocc),
            "gemm LoA");
      // cL[L] = sum_{j, nu} Y[j, nu, L] C[nu, j]
      const int64_t d2[2] = {n, nocc};
      const int p2[2] = {1, 0};
      check(dev::permute(c->st, 2, d2, p2, 1.0, dC, 0.0, Ct), "permute C");
      check(dev::gemm(c->st, 'T', 'N', nL, 1, nocc * n, 1.0, Y, nocc * n, Ct, nocc * n, 0.0, cL,
                      nL),
            "gemm cL");
      // F += 2 sum_L AAL[mu, nu, L] cL[L]
      check(dev::gemm(c->st, 'N', 'N', n * n, 1, nL, 2.0, d->aal, n * n, cL, nL, 1.0, dF, n * n),
            "gemm J");
      // F -= sum_{L, j} Y[j, mu, L] Y[j, nu, L], over Yp[j, L, nu]
      const int64_t d3[3] = {nocc, n, nL};
      const int p3[3] = {0, 2, 1};
      check(dev::permute(c->st, 3, d3, p3, 1.0, Y, 0.0, Yp), "permute LoA");
      check(dev::gemm(c->st, 'T', 'N', n, n, nocc * nL, -1.0, Yp, nocc * nL, Yp, nocc * nL, 1.0,
                      dF, n),
            "gemm K");
    }
    check(dev::d2h(F, dF, n * n * 8, c->st), "d2h");
    check(dev::sync(c->st), "sync");
  });
}

int ecg_df_mo(ecg_df* d, const double* C, int64_t nmo, double* B) {
  if (!d) return ECG_ERR_ARG;
  Ctx* c = d->ctx;
  return guarded(c, [&] {
    if (!C || !B) throw Error(ECG_ERR_ARG, "NULL argument");
    if (nmo <= 0) throw Error(ECG_ERR_ARG, "nmo must be positive");
    check(dev::set_device(c->device), "cudaSetDevice");
    const int64_t n = d->n, nL = d->nL;
    Scope scope{*c, c->allocs.size()};
    double* dC = c->alloc(n * nmo, "orbitals");
    double* T1 = c->alloc(nmo * n * nL, "mAL");
    double* dB = c->alloc(nmo * nmo * nL, "mmL");
    check(dev::h2d(dC, C, n * nmo * 8, c->st), "h2d");
    // T1[p, nu, L] = sum_mu C[mu, p] AAL[mu, nu, L]
    check(dev::gemm(c->st, 'T', 'N', nmo, n * nL, n, 1.0, dC, n, d->aal, n, 0.0, T1, nmo),
          "gemm mAL");
    // B[p, q, L] = sum_nu T1[p, nu, L] C[nu, q], batched over L
    check(dev::gemm(c->st, 'N', 'N', nmo, nmo, n, 1.0, T1, nmo, dC, n, 0.0, dB, nmo, nL, nmo * n,
                    0, nmo * nmo),
          "gemm mmL");
    check(dev::d2h(B, dB, nmo * nmo * nL * 8, c->st), "d2h");
    check(dev::sync(c->st), "sync");
  });
}

int ecg_df_destroy(ecg_df* d) {
  if (!d) return ECG_OK;
  if (d->aal) {
    Ctx* c = d->ctx;
    if (c->st) dev::sync(c->st);
    dev::dfree(d->aal);
    c->memused -= d->bytes;
    c->handle_bytes -= d->bytes;
  }
  delete d;
  return ECG_OK;
}

}  // extern "C"
