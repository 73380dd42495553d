// ecg_triples.cpp — closed-shell (T) and Lambda-(T).
//
// For each occupied triplet i <= j <= k (i = j = k skipped, weights 2/1 as in
// cc_triples.jl:62-72) the 12 contractions of cc_triples.jl:89-104 are
// regrouped as K = P[W]:
//   W^{xyz}[a,b,c] = sum_d T^{xy}_{ad} (bd|cz) - sum_l T^{xl}_{ab} (ly|cz)
//   K[a,b,c] = W^{ijk}[a,b,c] + W^{jik}[b,a,c] + W^{ikj}[a,c,b]
//            + W^{kji}[c,b,a] + W^{jki}[b,c,a] + W^{kij}[c,a,b]
// so each W is two plain GEMMs (M=v N=v^2 K=v and M=v^2 N=v K=o) that read
// vvvo[b,c,d,k] = <bc|dk> and ovoo in place, and a cube-tiled kernel sums the
// six permuted W's.  A fused kernel forms X and sum K*X, another accumulates
// IntX/IntY.  Per-triplet energies are summed on the host in triplet order,
// so the result is deterministic.
#include "ecg_triples.h"

#include <cmath>
#include <vector>

namespace ecg {

namespace {

// W^{xyz} for amplitudes T (T2 or covariant U2) into Wout.
void build_W(Ctx& c, const double* T, const double* V3, const double* On, double* Wout, int x,
             int y, int z) {
  const int64_t o = c.no, v = c.nv, v2 = v * v, v3 = v2 * v, o2 = o * o;
  dev::stream_t s = c.st;
  dev::Gemm g;
  // W[a,(b,c)] = sum_d T[a,d,x,y] vvvo[(b,c),d,z]
  g.m = v; g.n = v2; g.k = v; g.alpha = 1.0; g.beta = 0.0;
  g.A = T + v2 * (x + o * y); g.sam = 1; g.sak = v;
  g.B = V3 + v3 * z; g.sbk = v2; g.sbn = 1;
  g.C = Wout; g.scm = 1; g.scn = v;
  check(c.mixed_active ? dev::gemm_strided_mixed(s, g) : dev::gemm_strided(s, g), "W vvvo");
  // W[(a,b),c] -= sum_l T[a,b,x,l] ovoo[l,c,y,z]
  g = dev::Gemm{};
  g.m = v2; g.n = v; g.k = o; g.alpha = -1.0; g.beta = 1.0;
  g.A = T + v2 * x; g.sam = 1; g.sak = v2 * o;
  g.B = On + o * y + o2 * v * z; g.sbk = 1; g.sbn = o2;
  g.C = Wout; g.scm = 1; g.scn = v2;
  check(c.mixed_active ? dev::gemm_strided_mixed(s, g) : dev::gemm_strided(s, g), "W ovoo");
}

// K^{ijk} = P[W] for amplitudes T.
void build_K(Ctx& c, const double* T, const double* V3, const double* On, double* const* W,
             double* K, int i, int j, int k) {
  const int perm[6][3] = {{i, j, k}, {j, i, k}, {i, k, j}, {k, j, i}, {j, k, i}, {k, i, j}};
  for (int q = 0; q < 6; ++q) build_W(c, T, V3, On, W[q], perm[q][0], perm[q][1], perm[q][2]);
  check(dev::triples_sumw(c.st, (int)c.nv, W, K), "sum W");
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
  double* V3 = c.alloc(v3 * o, "(T) vvvo");
  double* On = c.alloc(o * o * o * v, "(T) ovoo");
  double* Wb[6];
  for (int q = 0; q < 6; ++q) Wb[q] = c.alloc(v3, "(T) W");
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
  // vvvo[b,c,d,k] = (bd|ck): per k, a GEMM batched over d
  for (int64_t kk = 0; kk < o; ++kk) {
    dev::Gemm g;
    g.m = v; g.n = v; g.k = Q; g.batch = v; g.alpha = 1.0; g.beta = 0.0;
    g.A = c.Bvv; g.sam = 1; g.sak = v * v; g.sab = v;
    g.B = c.Bvo + v * kk; g.sbk = v * o; g.sbn = 1; g.sbb = 0;
    g.C = V3 + v3 * kk; g.scm = 1; g.scn = v; g.scb = v * v;
    check(dev::gemm_strided(s, g), "vvvo");
  }
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
        build_K(c, c.T2(), V3, On, Wb, K, i, j, k);
        if (!lam) {
          check(dev::triples_x_cube(s, (int)v, K, eijk, ev, X, c.red, Et + t), "triples X");
        } else {
          check(dev::triples_x_cube(s, (int)v, K, eijk, ev, X, c.red, nullptr), "triples X");
          build_K(c, U2c, V3, On, Wb, KU, i, j, k);
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
  if (c.mixed_active) {
    int tc = 0;
    check(dev::tc_error(&tc), "tc_error");
    if (tc) throw Error(ECG_ERR_TIMEOUT, "tensor-core GEMM wait timed out in (T)");
  }
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
