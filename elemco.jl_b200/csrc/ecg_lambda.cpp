// ecg_lambda.cpp — closed-shell Lambda equations from dressed DF factors.
//
// Every dressed integral of calc_ccsd_vector_times_Jacobian
// (src/cc/cc_lagrange.jl:9-220) is a product of two dressed DF factors, so
// each term with a three-virtual integral (d_vovv) becomes two cheap
// three-index contractions, and the kext Lambda term (Kxoo = int2 * dU2,
// cc_lagrange.jl:39-75) becomes the transposed dressed ladder
//   R2[e,f,m,n] += sum_ab (ae|bf)^ U2[a,b,m,n]
// plus  R1[e,m] += 2 sum_{Qa} dB[a,e,Q] sum_{bj} dB[b,j,Q] U2[a,b,m,j].
// Only vT = v_{mb}^{cd} T^{ij}_{cd} (cc_lagrange.jl:948-952) goes through the
// explicit d_vovv block, once per Lambda solve.
#include "ecg_lambda.h"

#include <cmath>
#include <cstring>

namespace ecg {

static void ensure_lambda_buffers(Ctx& c) {
  if (c.U) return;
  c.U = c.alloc(c.n1() + c.n2(), "U");
  c.RU = c.alloc(c.n1() + c.n2(), "RU");
  c.vT = c.alloc((int64_t)c.no * c.no * c.no * c.nv, "vT");
  c.D1 = c.alloc((int64_t)c.n * c.n, "D1");
  c.dD1 = c.alloc((int64_t)c.n * c.n, "dD1");
}

void lambda_prepare(Ctx& c, bool dc) {
  (void)dc;
  ensure_lambda_buffers(c);
  const int64_t o = c.no, v = c.nv;
  // one o v^3 block for d_vovv plus a same-sized permute temporary
  c.ensure_ws(2 * o * v * v * v + 16 * c.n2() + (1 << 20));
  dress(c, c.T1());
  Contractor con = c.con();
  const int64_t mark = c.ws.mark();
  // d_vovv[b,m,d,c] = (bd|mc)^  stored as [b,d,c,m]
  double* dvovv = c.ws.get(o * v * v * v);
  con(1.0, c.dBvv, "bdQ", c.Bov, "mcQ", 0.0, dvovv, "bdcm");
  // vT[m,b,i,j] = sum_dc d_vovv[b,m,d,c] T2[d,c,j,i]
  con(1.0, dvovv, "bdcm", c.T2(), "dcji", 0.0, c.vT, "mbij");
  c.ws.release(mark);
  check(dev::sync(c.st), "sync");
  c.lambda_ready = true;
}

void lambda_load_U(Ctx& c, const double* U1h, const double* U2h) {
  ensure_lambda_buffers(c);
  check(dev::h2d(c.U, U1h, c.n1() * 8, c.st), "h2d U1");
  check(dev::h2d(c.U + c.n1(), U2h, c.n2() * 8, c.st), "h2d U2");
}

void lambda_store_U(Ctx& c, double* U1h, double* U2h) {
  check(dev::d2h(U1h, c.U, c.n1() * 8, c.st), "d2h U1");
  check(dev::d2h(U2h, c.U + c.n1(), c.n2() * 8, c.st), "d2h U2");
  check(dev::sync(c.st), "sync");
}

void lambda_store_R(Ctx& c, double* R1h, double* R2h) {
  if (R1h) check(dev::d2h(R1h, c.RU, c.n1() * 8, c.st), "d2h R1");
  if (R2h) check(dev::d2h(R2h, c.RU + c.n1(), c.n2() * 8, c.st), "d2h R2");
  check(dev::sync(c.st), "sync");
}

// D1 and dD1 (n x n, device) from U in c.U and T in c.T (cc_lagrange.jl:793-848).
static void one_rdm_device(Ctx& c) {
  const int64_t n = c.n, o = c.no, v = c.nv, n2 = c.n2();
  dev::stream_t s = c.st;
  Contractor con = c.con();
  const double* U1 = c.U;
  const double* U2 = c.U + c.n1();
  const double* T1 = c.T1();
  const double* T2 = c.T2();
  const int64_t mark = c.ws.mark();
  double* Doo = c.ws.get(o * o);
  double* Dvv = c.ws.get(v * v);
  double* Dov = c.ws.get(o * v);
  double* Dvo = c.ws.get(v * o);
  double* dDoo = c.ws.get(o * o);
  double* dDvv = c.ws.get(v * v);
  double* dDvo = c.ws.get(v * o);
  double* tT2 = c.ws.get(n2);
  con(-2.0, U2, "cdik", T2, "cdjk", 0.0, Doo, "ij");
  con(2.0, U2, "bckl", T2, "ackl", 0.0, Dvv, "ab");
  con.permute(1.0, U1, "ai", 0.0, Dov, "ia");
  // Dvo[a,i] = sum_ck U1[c,k] (2 T2[a,c,i,k] - T2[a,c,k,i])
  check(dev::axpby(s, n2, 2.0, T2, 0.0, tT2), "tT2");
  con.permute(-1.0, T2, "abji", 1.0, tT2, "abij");
  con(1.0, tT2, "acik", U1, "ck", 0.0, Dvo, "ai");
  // T1-dressed pieces
  check(dev::axpby(s, o * o, 1.0, Doo, 0.0, dDoo), "dDoo");
  con(-1.0, Dov, "ic", T1, "cj", 1.0, dDoo, "ij");
  check(dev::axpby(s, v * v, 1.0, Dvv, 0.0, dDvv), "dDvv");
  con(1.0, T1, "ak", Dov, "kb", 1.0, dDvv, "ab");
  check(dev::axpby(s, v * o, 1.0, Dvo, 0.0, dDvo), "dDvo");
  check(dev::axpby(s, v * o, 2.0, T1, 1.0, dDvo), "dDvo");
  con(-1.0, Dvv, "ac", T1, "ci", 1.0, dDvo, "ai");
  con(1.0, T1, "ak", dDoo, "ki", 1.0, dDvo, "ai");
  // assemble n x n matrices
  check(dev::geam(s, o, o, 1.0, Doo, o, 0.0, c.D1, n), "D1");
  check(dev::geam(s, v, v, 1.0, Dvv, v, 0.0, c.D1 + o + o * n, n), "D1");
  check(dev::geam(s, o, v, 1.0, Dov, o, 0.0, c.D1 + o * n, n), "D1");
  check(dev::geam(s, v, o, 1.0, Dvo, v, 0.0, c.D1 + o, n), "D1");
  check(dev::geam(s, o, o, 1.0, dDoo, o, 0.0, c.dD1, n), "dD1");
  check(dev::geam(s, v, v, 1.0, dDvv, v, 0.0, c.dD1 + o + o * n, n), "dD1");
  check(dev::geam(s, o, v, 1.0, Dov, o, 0.0, c.dD1 + o * n, n), "dD1");
  check(dev::geam(s, v, o, 1.0, dDvo, v, 0.0, c.dD1 + o, n), "dD1");
  c.ws.release(mark);
}

void one_rdm(Ctx& c, double* D1h, double* dD1h) {
  one_rdm_device(c);
  const int64_t n = c.n;
  if (D1h) check(dev::d2h(D1h, c.D1, n * n * 8, c.st), "d2h D1");
  if (dD1h) check(dev::d2h(dD1h, c.dD1, n * n * 8, c.st), "d2h dD1");
  check(dev::sync(c.st), "sync");
}

// copy an r x q block at offset `off` of an n x n column-major matrix
static double* block(Ctx& c, const double* M, int64_t rows, int64_t cols, int64_t off) {
  double* b = c.ws.get(rows * cols);
  check(dev::geam(c.st, rows, cols, 1.0, M + off, c.n, 0.0, b, rows), "block");
  return b;
}

void lambda_residual(Ctx& c, bool dc) {
  if (!c.lambda_ready) throw Error(ECG_ERR_STATE, "Lambda intermediates not prepared");
  const int64_t n = c.n, o = c.no, v = c.nv, Q = c.nq, n1 = c.n1(), n2 = c.n2();
  dev::stream_t s = c.st;
  Contractor con = c.con();
  const double* T1 = c.T1();
  const double* T2 = c.T2();
  const double* U1 = c.U;
  const double* U2 = c.U + n1;
  double* R1 = c.RU;
  double* R2 = c.RU + n1;
  one_rdm_device(c);
  const int64_t mark = c.ws.mark();
  const int64_t oo = 0, vo = o, ov = o * n, vv = o + o * n;
  double* D1oo = block(c, c.D1, o, o, oo);
  double* D1vv = block(c, c.D1, v, v, vv);
  double* dDoo = block(c, c.dD1, o, o, oo);
  double* dDvv = block(c, c.dD1, v, v, vv);
  double* dDov = block(c, c.dD1, o, v, ov);
  double* dDvo = block(c, c.dD1, v, o, vo);
  double* dfov = block(c, c.dfock, o, v, ov);
  double* dfoo = block(c, c.dfock, o, o, oo);
  double* dfvv = block(c, c.dfock, v, v, vv);

  // R1 = 2 f_ov^T ; R2 = 2 v_mn^ef - v_nm^ef   (cc_lagrange.jl:25-33)
  check(dev::axpby(s, n1, 2.0, c.fvo_t, 0.0, R1), "R1");
  check(dev::axpby(s, n2, 2.0, c.Kvvoo, 0.0, R2), "R2");
  con.permute(-1.0, c.Kvvoo, "efnm", 1.0, R2, "efmn");
  // R2 += U2[e,f,i,j] (d_oooo + v T2)[m,n,i,j]   (:34-40)
  double* I = c.ws.get(o * o * o * o);
  con(1.0, c.dBoo, "miQ", c.dBoo, "njQ", 0.0, I, "mnij");
  if (!dc) con(1.0, c.klcd, "mncd", T2, "cdij", 1.0, I, "mnij");
  con(1.0, I, "mnij", U2, "efij", 1.0, R2, "efmn");
  // kext Lambda (:42-75): transposed dressed ladder and its singles part
  ladder(c, c.dBvvT, c.dBvv, U2, R2);
  double* Z = c.ws.get(v * o * Q);
  con(1.0, U2, "abmj", c.dBvo, "bjQ", 0.0, Z, "amQ");
  con(2.0, c.dBvv, "aeQ", Z, "amQ", 1.0, R1, "em");

  // tR2 (:77-121)
  const double fac = dc ? 0.25 : 0.5;
  double* tR2 = c.ws.get(n2);
  con(fac, D1oo, "mk", c.Kvvoo, "efkn", 0.0, tR2, "efmn");
  con(-fac, D1vv, "ce", c.Kvvoo, "cfmn", 1.0, tR2, "efmn");
  double* tT2 = c.ws.get(n2);
  check(dev::axpby(s, n2, 2.0, T2, 0.0, tT2), "tT2");
  con.permute(-1.0, T2, "efnm", 1.0, tT2, "efmn");
  double* xoo = c.ws.get(o * o);
  double* xvv = c.ws.get(v * v);
  con(1.0, tT2, "cdil", c.klcd, "mlcd", 0.0, xoo, "mi");
  con(1.0, tT2, "ackl", c.klcd, "klec", 0.0, xvv, "ae");
  double* W = c.ws.get(n2);
  con(1.0, c.dBvo, "aiQ", c.Bov, "meQ", 0.0, W, "amie");
  con(1.0, c.klcd, "kmce", tT2, "acik", 1.0, W, "amie");
  con(1.0, U2, "afin", W, "amie", 1.0, tR2, "efmn");
  // U1 terms of tR2 (:106-121)
  double* dfovT = c.ws.get(v * o);
  con.permute(1.0, dfov, "nf", 0.0, dfovT, "fn");
  check(dev::outer(s, v, o, v, o, 0.5, U1, dfovT, 1.0, tR2), "outer");
  double* P = c.ws.get(v * o * Q);
  con(1.0, c.dBvv, "afQ", U1, "an", 0.0, P, "fnQ");
  con(0.5, P, "fnQ", c.Bov, "meQ", 1.0, tR2, "efmn");
  con(1.0, c.dBoo, "niQ", U1, "fi", 0.0, P, "nfQ");
  con(-0.5, c.Bov, "meQ", P, "nfQ", 1.0, tR2, "efmn");
  // pR2 = 2 tR2 - tR2[e,f,n,m]
  double* pR2 = c.ws.get(n2);
  check(dev::axpby(s, n2, 2.0, tR2, 0.0, pR2), "pR2");
  con.permute(-1.0, tR2, "efnm", 1.0, pR2, "efmn");

  // D2 = U2 tT2 (:127-147)
  double* D2 = tR2;  // reuse
  con(1.0, U2, "acik", tT2, "cbkj", 0.0, D2, "abij");
  double* Zd = Z;
  con(1.0, D2, "adml", c.Bov, "ldQ", 0.0, Zd, "amQ");
  con(2.0, c.dBvv, "aeQ", Zd, "amQ", 1.0, R1, "em");
  con(-2.0, Zd, "eiQ", c.dBoo, "miQ", 1.0, R1, "em");
  if (!dc) con(-1.0, D2, "fcnl", c.klcd, "mlce", 1.0, pR2, "efmn");
  // Dbar = U2 T2 + U2^T T2 (:148-170)
  con(1.0, U2, "acik", T2, "cbkj", 0.0, D2, "abij");
  con(1.0, U2, "caik", T2, "bckj", 1.0, D2, "abij");
  if (!dc) con(1.0, D2, "ednk", c.klcd, "kmfd", 1.0, pR2, "efmn");
  double* Zo = c.ws.get(o * o * Q);
  con(1.0, D2, "acmk", c.dBvv, "acQ", 0.0, Zo, "mkQ");
  con(-2.0, c.Bov, "keQ", Zo, "mkQ", 1.0, R1, "em");
  double* Zv = c.ws.get(v * v * Q);
  con(1.0, D2, "ecik", c.dBoo, "kiQ", 0.0, Zv, "ecQ");
  con(2.0, Zv, "ecQ", c.Bov, "mcQ", 1.0, R1, "em");
  // D_ij^kl = U2 T2 (:173-189)
  double* D4 = I;
  con(1.0, U2, "cdij", T2, "cdkl", 0.0, D4, "ijkl");
  con(1.0, D4, "mjkl", c.dBoo, "ljQ", 0.0, Zo, "mkQ");
  con(2.0, c.Bov, "keQ", Zo, "mkQ", 1.0, R1, "em");
  if (!dc) con(1.0, D4, "mnkl", c.klcd, "klef", 1.0, R2, "efmn");
  // R1 -= 2 U2 vT (:190-197)
  con(-2.0, U2, "ebij", c.vT, "mbij", 1.0, R1, "em");
  // Fock-like terms (:198-204)
  const double fac2 = dc ? 0.5 : 1.0;
  double* Xvv = c.ws.get(v * v);
  double* Xoo = c.ws.get(o * o);
  check(dev::axpby(s, v * v, 1.0, dfvv, 0.0, Xvv), "Xvv");
  check(dev::axpby(s, v * v, -fac2, xvv, 1.0, Xvv), "Xvv");
  check(dev::axpby(s, o * o, 1.0, dfoo, 0.0, Xoo), "Xoo");
  check(dev::axpby(s, o * o, fac2, xoo, 1.0, Xoo), "Xoo");
  con(1.0, Xvv, "ae", U2, "afmn", 1.0, pR2, "efmn");
  con(-1.0, U2, "efin", Xoo, "mi", 1.0, pR2, "efmn");
  // d_vovo terms (:205-212)
  con(1.0, c.dBvv, "aeQ", c.dBoo, "miQ", 0.0, W, "amei");
  con(-1.0, U2, "afin", W, "amei", 1.0, pR2, "efmn");
  con(-1.0, U2, "ebin", W, "bmfi", 1.0, pR2, "efmn");
  // R2 += pR2 + pR2[f,e,n,m]
  check(dev::axpby(s, n2, 1.0, pR2, 1.0, R2), "R2 += pR2");
  con.permute(1.0, pR2, "fenm", 1.0, R2, "efmn");

  // singles (:207-218)
  // R1 += sum_pq dD1[p,q] (2 <qm|pe> - <qm|ep>)  with undressed integrals
  double* g = c.ws.get(Q);
  con(1.0, dDoo, "ij", c.Boo, "jiQ", 0.0, g, "Q");
  con(1.0, dDov, "ia", c.Bvo, "aiQ", 1.0, g, "Q");
  con(1.0, dDvo, "ai", c.Bov, "iaQ", 1.0, g, "Q");
  con(1.0, dDvv, "ab", c.Bvv, "baQ", 1.0, g, "Q");
  con(2.0, c.Bov, "meQ", g, "Q", 1.0, R1, "em");
  double* Ho = Zo;  // [m,j,Q]
  con(1.0, c.Boo, "miQ", dDoo, "ij", 0.0, Ho, "mjQ");
  con(1.0, c.Bov, "maQ", dDvo, "aj", 1.0, Ho, "mjQ");
  con(-1.0, Ho, "mjQ", c.Bov, "jeQ", 1.0, R1, "em");
  double* Hv = P;  // [m,b,Q]
  con(1.0, c.Boo, "miQ", dDov, "ib", 0.0, Hv, "mbQ");
  con(1.0, c.Bov, "maQ", dDvv, "ab", 1.0, Hv, "mbQ");
  con(-1.0, Hv, "mbQ", c.Bvv, "beQ", 1.0, R1, "em");
  // R1 -= 2 U2[e,b,i,j] d_vooo[b,m,j,i]
  con(1.0, U2, "ebij", c.dBvo, "bjQ", 0.0, Z, "eiQ");
  con(-2.0, Z, "eiQ", c.dBoo, "miQ", 1.0, R1, "em");
  // R1 += D_m^k f_k^e - D_d^e f_m^d + U1 (f - x)_vv - U1 (f + x)_oo
  con(1.0, D1oo, "mk", dfov, "ke", 1.0, R1, "em");
  con(-1.0, D1vv, "de", dfov, "md", 1.0, R1, "em");
  check(dev::axpby(s, v * v, 1.0, dfvv, 0.0, Xvv), "Xvv");
  check(dev::axpby(s, v * v, -1.0, xvv, 1.0, Xvv), "Xvv");
  check(dev::axpby(s, o * o, 1.0, dfoo, 0.0, Xoo), "Xoo");
  check(dev::axpby(s, o * o, 1.0, xoo, 1.0, Xoo), "Xoo");
  con(1.0, U1, "am", Xvv, "ae", 1.0, R1, "em");
  con(-1.0, U1, "ei", Xoo, "mi", 1.0, R1, "em");
  c.ws.release(mark);
}

LambdaResult lambda_solve(Ctx& c, bool dc, const ecg_cc_opts& o) {
  const int64_t n1 = c.n1(), n2 = c.n2();
  dev::stream_t s = c.st;
  lambda_prepare(c, dc);
  double* U1 = c.U;
  double* U2 = c.U + n1;
  // guess: U2 = 2 tau - tau[a,b,j,i], tau = T2 + T1 T1; U1 = 2 T1 (cctools.jl:919-930)
  check(dev::outer(s, c.nv, c.no, c.nv, c.no, 1.0, c.T1(), c.T1(), 0.0, c.TT), "outer");
  check(dev::axpby(s, n2, 1.0, c.T2(), 1.0, c.TT), "tau");
  check(dev::axpby(s, n2, 2.0, c.TT, 0.0, U2), "U2");
  c.con().permute(-1.0, c.TT, "abji", 1.0, U2, "abij");
  check(dev::axpby(s, n1, 2.0, c.T1(), 0.0, U1), "U1");
  // TT = T1 T1 for the correlation norm
  check(dev::outer(s, c.nv, c.no, c.nv, c.no, 1.0, c.T1(), c.T1(), 0.0, c.TT), "outer");
  diis_reset(c, c.ldiis, o.maxdiis, o.resthr, n1 + n2, false);
  const double thren = std::sqrt(o.thr) * o.conven;
  const double* eo = c.eps;
  const double* ev = c.eps + c.no;
  LambdaResult r;
  double prev = 0.0;
  // ECG_PREC_MIXED: the Lambda residual's large GEMMs use split-BF16 tensor-core
  // products until the squared residual is below 100 thr, then FP64
  // iterations refine; convergence is only declared on an FP64 residual.
  bool mixed_phase = (c.prec == ECG_PREC_MIXED);
  struct Restore {
    Ctx& c;
    ~Restore() { c.mixed_active = false; }
  } restore{c};
  for (int it = 1; it <= o.maxit; ++it) {
    c.mixed_active = mixed_phase;
    lambda_residual(c, dc);
    double* R1 = c.RU;
    double* R2 = c.RU + n1;
    check(dev::update_doubles(s, c.nv, c.no, eo, ev, o.shiftp, R2, U2), "upd U2");
    check(dev::cs_dot(s, c.nv, c.no, R2, R2, c.red, c.dscal + 0), "norm");
    check(dev::dot(s, n1, R1, R1, c.red, c.dscal + 2), "norm");
    check(dev::update_singles(s, c.nv, c.no, eo, ev, o.shifts, R1, U1), "upd U1");
    sync_scalars(c, 3);
    const double NormR2 = (2.0 * c.hscal[0] + c.hscal[1]) / 3.0;
    const double NormR1 = 0.5 * c.hscal[2];
    diis_perform(c, c.ldiis, c.U, c.RU);
    // calc_correlation_norm (cc_lagrange.jl:1065-1078)
    check(dev::dot(s, n2, U2, c.T2(), c.red, c.dscal + 10), "cnorm");
    check(dev::dot(s, n2, U2, c.TT, c.red, c.dscal + 11), "cnorm");
    check(dev::dot(s, n1, U1, c.T1(), c.red, c.dscal + 12), "cnorm");
    sync_scalars(c, 13);
    const double norm = c.hscal[10] + c.hscal[11] + c.hscal[12];
    r.normR = NormR1 + NormR2;
    r.dnorm = norm - prev;
    r.norm = norm;
    r.iterations = it;
    prev = norm;
    if (!std::isfinite(norm) || !std::isfinite(r.normR))
      throw Error(ECG_ERR_NONFINITE, "non-finite value in Lambda iteration");
    if (mixed_phase) {
      if (r.normR < 100.0 * o.thr) mixed_phase = false;
      continue;
    }
    if (r.normR < o.thr && std::fabs(r.dnorm) < thren) {
      r.converged = true;
      break;
    }
  }
  return r;
}

}  // namespace ecg
