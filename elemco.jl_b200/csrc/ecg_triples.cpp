// ecg_triples.cpp — closed-shell (T) and Lambda-(T).
//
// For each occupied triplet i <= j <= k (i = j = k skipped, weights 2/1 as in
// cc_triples.jl:62-72) K[a,b,c] is accumulated from the 12 contractions of
// cc_triples.jl:89-104, each one strided batched FP64 GEMM reading the
// integrals in place:
//   V[b,d,c,k] = (bd|ck) = <bc|dk>  (the reference's vvvo[b,c,d,k])
//   O[l,j,c,k] = (lj|ck) = <lc|jk>  (the reference's ovoo[l,c,j,k])
// both built once from the DF factors.  A fused kernel forms X and sum K*X,
// a second one accumulates IntX/IntY.  Per-triplet energies are summed on the
// host in triplet order, so the result is deterministic.
#include "ecg_triples.h"

#include <cmath>
#include <vector>

namespace ecg {

namespace {

struct TriplesCtx {
  int64_t o, v;
  const double* T2;  // amplitudes entering K
  const double* Vn;
  const double* On;
};

// K[a,b,c] (+)= the 12 terms of cc_triples.jl:89-104 for amplitudes tc.T2.
void build_K(Ctx& c, const TriplesCtx& t, double* K, int i, int j, int k) {
  const int64_t o = t.o, v = t.v, v2 = v * v, v3 = v2 * v, o2 = o * o;
  dev::stream_t s = c.st;
  check(dev::memset0(K, v3 * 8, s), "memset K");
  auto Tij = [&](int x, int y) { return t.T2 + v2 * (x + o * y); };   // T2[:,:,x,y]
  auto Tx = [&](int x) { return t.T2 + v2 * o * x; };                 // T2[:,:,:,x]
  auto Vx = [&](int x) { return t.Vn + v3 * x; };                     // vvvo[:,:,:,x]
  auto Oxy = [&](int x, int y) { return t.On + o * x + o2 * v * y; };  // ovoo[:,:,x,y]
  auto run = [&](dev::Gemm g, const char* what) {
    g.beta = 1.0;
    g.C = K;
    check(dev::gemm_strided(s, g), what);
  };
  dev::Gemm g;
  // 1. T2ij[a,d] vvvk[b,c,d]      M=a N=b K=d batch c
  g = dev::Gemm{};
  g.m = v; g.n = v; g.k = v; g.batch = v; g.alpha = 1.0;
  g.A = Tij(i, j); g.sam = 1; g.sak = v; g.sab = 0;
  g.B = Vx(k); g.sbk = v; g.sbn = 1; g.sbb = v2;
  g.scm = 1; g.scn = v; g.scb = v2;
  run(g, "K1");
  // 2. T2ij[d,b] vvvk[a,c,d]      M=a N=b K=d batch c
  g = dev::Gemm{};
  g.m = v; g.n = v; g.k = v; g.batch = v; g.alpha = 1.0;
  g.A = Vx(k); g.sam = 1; g.sak = v; g.sab = v2;
  g.B = Tij(i, j); g.sbk = 1; g.sbn = v; g.sbb = 0;
  g.scm = 1; g.scn = v; g.scb = v2;
  run(g, "K2");
  // 3. T2ik[a,d] vvvj[c,b,d]      M=a N=c K=d batch b
  g = dev::Gemm{};
  g.m = v; g.n = v; g.k = v; g.batch = v; g.alpha = 1.0;
  g.A = Tij(i, k); g.sam = 1; g.sak = v; g.sab = 0;
  g.B = Vx(j); g.sbk = v; g.sbn = 1; g.sbb = v2;
  g.scm = 1; g.scn = v2; g.scb = v;
  run(g, "K3");
  // 4. T2ik[d,c] vvvj[a,b,d]      M=a N=c K=d batch b
  g = dev::Gemm{};
  g.m = v; g.n = v; g.k = v; g.batch = v; g.alpha = 1.0;
  g.A = Vx(j); g.sam = 1; g.sak = v; g.sab = v2;
  g.B = Tij(i, k); g.sbk = 1; g.sbn = v; g.sbb = 0;
  g.scm = 1; g.scn = v2; g.scb = v;
  run(g, "K4");
  // 5. T2jk[b,d] vvvi[c,a,d]      M=b N=c K=d batch a
  g = dev::Gemm{};
  g.m = v; g.n = v; g.k = v; g.batch = v; g.alpha = 1.0;
  g.A = Tij(j, k); g.sam = 1; g.sak = v; g.sab = 0;
  g.B = Vx(i); g.sbk = v; g.sbn = 1; g.sbb = v2;
  g.scm = v; g.scn = v2; g.scb = 1;
  run(g, "K5");
  // 6. T2jk[d,c] vvvi[b,a,d]      M=b N=c K=d batch a
  g = dev::Gemm{};
  g.m = v; g.n = v; g.k = v; g.batch = v; g.alpha = 1.0;
  g.A = Vx(i); g.sam = 1; g.sak = v; g.sab = v2;
  g.B = Tij(j, k); g.sbk = 1; g.sbn = v; g.sbb = 0;
  g.scm = v; g.scn = v2; g.scb = 1;
  run(g, "K6");
  // 7. -T2i[b,a,l] ovjk[l,c]      M=b N=c K=l batch a
  g = dev::Gemm{};
  g.m = v; g.n = v; g.k = o; g.batch = v; g.alpha = -1.0;
  g.A = Tx(i); g.sam = 1; g.sak = v2; g.sab = v;
  g.B = Oxy(j, k); g.sbk = 1; g.sbn = o2; g.sbb = 0;
  g.scm = v; g.scn = v2; g.scb = 1;
  run(g, "K7");
  // 8. -T2j[a,b,l] ovik[l,c]      M=(a,b) N=c K=l
  g = dev::Gemm{};
  g.m = v2; g.n = v; g.k = o; g.batch = 1; g.alpha = -1.0;
  g.A = Tx(j); g.sam = 1; g.sak = v2;
  g.B = Oxy(i, k); g.sbk = 1; g.sbn = o2;
  g.scm = 1; g.scn = v2;
  run(g, "K8");
  // 9. -T2i[c,a,l] ovkj[l,b]      M=c N=b K=l batch a
  g = dev::Gemm{};
  g.m = v; g.n = v; g.k = o; g.batch = v; g.alpha = -1.0;
  g.A = Tx(i); g.sam = 1; g.sak = v2; g.sab = v;
  g.B = Oxy(k, j); g.sbk = 1; g.sbn = o2; g.sbb = 0;
  g.scm = v2; g.scn = v; g.scb = 1;
  run(g, "K9");
  // 10. -T2k[a,c,l] ovij[l,b]     M=a N=b K=l batch c
  g = dev::Gemm{};
  g.m = v; g.n = v; g.k = o; g.batch = v; g.alpha = -1.0;
  g.A = Tx(k); g.sam = 1; g.sak = v2; g.sab = v;
  g.B = Oxy(i, j); g.sbk = 1; g.sbn = o2; g.sbb = 0;
  g.scm = 1; g.scn = v; g.scb = v2;
  run(g, "K10");
  // 11. -T2j[c,b,l] ovki[l,a]     M=c N=a K=l batch b
  g = dev::Gemm{};
  g.m = v; g.n = v; g.k = o; g.batch = v; g.alpha = -1.0;
  g.A = Tx(j); g.sam = 1; g.sak = v2; g.sab = v;
  g.B = Oxy(k, i); g.sbk = 1; g.sbn = o2; g.sbb = 0;
  g.scm = v2; g.scn = 1; g.scb = v;
  run(g, "K11");
  // 12. -T2k[b,c,l] ovji[l,a]     M=(b,c) N=a K=l
  g = dev::Gemm{};
  g.m = v2; g.n = v; g.k = o; g.batch = 1; g.alpha = -1.0;
  g.A = Tx(k); g.sam = 1; g.sak = v2;
  g.B = Oxy(j, i); g.sbk = 1; g.sbn = o2;
  g.scm = v; g.scn = 1;
  run(g, "K12");
}

}  // namespace

void pert_triples(Ctx& c, const double* U1h, const double* U2h, double* et, double* etb) {
  const int64_t o = c.no, v = c.nv, Q = c.nq, v3 = v * v * v;
  const bool lam = (U1h != nullptr);
  dev::stream_t s = c.st;
  // integrals, allocated per call (v^3 o + o^3 v doubles) and freed on exit
  struct Scope {
    Ctx& c;
    size_t n0;
    ~Scope() { c.release_to(n0); }
  } scope{c, c.allocs.size()};
  double* Vn = c.alloc(v3 * o, "(T) vvvo");
  double* On = c.alloc(o * o * o * v, "(T) ovoo");
  double* K = c.alloc(v3, "(T) K");
  double* X = c.alloc(v3, "(T) X");
  double* KU = lam ? c.alloc(v3, "(T) K(Lambda)") : nullptr;
  double* U2 = lam ? c.alloc(c.n2(), "(T) U2") : nullptr;
  double* U2c = lam ? c.alloc(c.n2(), "(T) U2 covariant") : nullptr;
  double* IntXY = c.alloc(2 * v * o, "(T) IntX/IntY");
  int64_t ntrip = 0;
  for (int64_t kk = 0; kk < o; ++kk)
    for (int64_t jj = 0; jj <= kk; ++jj)
      for (int64_t ii = 0; ii <= jj; ++ii)
        if (!(ii == jj && jj == kk)) ++ntrip;
  double* Et = c.alloc(std::max<int64_t>(ntrip, 1), "(T) energies");
  Contractor con = c.con();
  con(1.0, c.Bvv, "bdQ", c.Bvo, "ckQ", 0.0, Vn, "bdck");
  con(1.0, c.Boo, "ljQ", c.Bvo, "ckQ", 0.0, On, "ljck");
  check(dev::memset0(IntXY, 2 * v * o * 8, s), "memset");
  double* IntX = IntXY;
  double* IntY = IntXY + v * o;
  if (lam) {
    check(dev::h2d(U2, U2h, c.n2() * 8, s), "h2d U2");
    // contra2covariant (cctools.jl:935-938): (2 U2[a,b,i,j] + U2[b,a,i,j]) / 3
    check(dev::axpby(s, c.n2(), 2.0 / 3.0, U2, 0.0, U2c), "U2c");
    con.permute(1.0 / 3.0, U2, "baij", 1.0, U2c, "abij");
  }
  std::vector<double> fac;
  fac.reserve(ntrip);
  const double* eps = c.fock_host.data();
  const int64_t n = c.n;
  const double* ev = c.eps + o;
  TriplesCtx tT{o, v, c.T2(), Vn, On};
  TriplesCtx tU{o, v, U2c, Vn, On};
  const double* Nsrc = lam ? U2c : c.T2();
  int64_t t = 0;
  for (int k = 0; k < o; ++k)
    for (int j = 0; j <= k; ++j) {
      const double prefac = (j == k) ? 1.0 : 2.0;
      for (int i = 0; i <= j; ++i) {
        double f = prefac;
        if (i == j) {
          if (j == k) continue;
          f = 1.0;
        }
        const double eijk = eps[i + i * n] + eps[j + j * n] + eps[k + k * n];
        build_K(c, tT, K, i, j, k);
        if (!lam) {
          check(dev::triples_x(s, (int)v, K, eijk, ev, X, c.red, Et + t), "triples X");
        } else {
          check(dev::triples_x(s, (int)v, K, eijk, ev, X, c.red, nullptr), "triples X");
          build_K(c, tU, KU, i, j, k);
          check(dev::dot(s, v3, KU, X, c.red, Et + t), "triples E");
        }
        const int64_t v2 = v * v;
        auto M = [&](int x, int y) { return c.Kvvoo + v2 * (x + o * y); };
        auto N = [&](int x, int y) { return Nsrc + v2 * (x + o * y); };
        check(dev::triples_int(s, (int)v, X, M(j, k), M(i, k), M(i, j), N(j, k), N(i, k), N(i, j),
                               f, IntX, IntY, i, j, k),
              "triples Int");
        fac.push_back(f);
        ++t;
      }
    }
  std::vector<double> Eh(ntrip), IX(2 * v * o);
  if (ntrip) check(dev::d2h(Eh.data(), Et, ntrip * 8, s), "d2h");
  check(dev::d2h(IX.data(), IntXY, 2 * v * o * 8, s), "d2h");
  std::vector<double> T1h(v * o);
  check(dev::d2h(T1h.data(), c.T1(), v * o * 8, s), "d2h");
  check(dev::sync(s), "sync");
  double Enb3 = 0.0;
  for (int64_t q = 0; q < ntrip; ++q) Enb3 += fac[q] * Eh[q];
  // singles and Fock contributions (cc_triples.jl:143-156 / :286-294)
  double En3 = 0.0;
  for (int64_t i = 0; i < o; ++i)
    for (int64_t a = 0; a < v; ++a) {
      double x = IX[a + v * i], y = IX[v * o + a + v * i];
      if (!lam) En3 += T1h[a + v * i] * x;
      else En3 += 0.5 * U1h[a + v * i] * x;
      En3 += c.fock_host[i + (o + a) * n] * y;
    }
  En3 += Enb3;
  if (!std::isfinite(En3)) throw Error(ECG_ERR_NONFINITE, "non-finite (T) energy");
  *et = En3;
  *etb = Enb3;
  (void)Q;
}

}  // namespace ecg
