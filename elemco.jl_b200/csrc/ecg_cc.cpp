// ecg_cc.cpp — closed-shell CCSD/DCSD on the device from density-fitting
// factors: T1 dressing, the residual, energies, amplitude update and DIIS.
//
// The reference (ElemCo.jl) forms T1-dressed 4-index integral blocks from the
// full int2 array and contracts the kext ladder against all n orbitals.  Here
// every integral is a product of dressed DF factors
//   B^Q = (1 - t) B^Q (1 + t),   t[v,o] = T1,
// which is the same similarity transform the reference applies block by block
// in calc_dressed_ints (src/cc/cc.jl:453-774).  The kext term (cc.jl:1400-1425)
// then becomes the particle-particle ladder over dressed B_vv plus the
// (ai|bj) term, and its singles pieces fold into the dressed Fock matrix and a
// three-index intermediate (see cc_residual below).  No 4-index integral with
// more than two virtual indices is ever stored.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "ecg_core.h"

namespace ecg {

double* Ctx::alloc(int64_t nd, const char* what) {
  size_t bytes = (size_t)std::max<int64_t>(nd, 1) * sizeof(double);
  if (memcap && memused + bytes > memcap)
    throw Error(ECG_ERR_OOM, std::string("device memory cap exceeded allocating ") + what);
  void* p = dev::dmalloc(bytes);
  if (!p) throw Error(ECG_ERR_OOM, std::string("cudaMalloc failed for ") + what);
  allocs.push_back({p, bytes});
  memused += bytes;
  return (double*)p;
}

void Ctx::release_to(size_t nallocs) {
  if (allocs.size() <= nallocs) return;
  if (st) dev::sync(st);
  while (allocs.size() > nallocs) {
    auto a = allocs.back();
    allocs.pop_back();
    dev::dfree(a.first);
    memused -= a.second;
  }
}

void Ctx::ensure_ws(int64_t nd) {
  if (ws.capacity() >= nd) return;
  if (st) dev::sync(st);
  for (size_t q = 0; q < allocs.size(); ++q)
    if (allocs[q].first == (void*)ws_base) {
      dev::dfree(allocs[q].first);
      memused -= allocs[q].second;
      allocs.erase(allocs.begin() + q);
      break;
    }
  ws_base = alloc(nd, "workspace");
  ws.init(ws_base, nd);
}

void* Ctx::ensure_tc(size_t bytes) {
  if (tc_bytes >= bytes) return tc_base;
  if (st) dev::sync(st);
  for (size_t q = 0; q < allocs.size(); ++q)
    if (allocs[q].first == tc_base) {
      dev::dfree(allocs[q].first);
      memused -= allocs[q].second;
      allocs.erase(allocs.begin() + q);
      break;
    }
  tc_base = nullptr;
  tc_bytes = 0;
  tc_base = alloc((int64_t)((bytes + 7) / 8), "split-operand storage");
  tc_bytes = bytes;
  return tc_base;
}

void Ctx::free_all() {
  if (st) dev::sync(st);
  for (auto& a : allocs) dev::dfree(a.first);
  allocs.clear();
  memused = handle_bytes;  // handles keep their memory across systems
  if (hscal) dev::hfree_pinned(hscal);
  hscal = nullptr;
  have_system = false;
  t_resident = false;
  // buffers allocated on first use must be allocated again for the next system
  U = RU = vT = D1 = dD1 = nullptr;
  lambda_ready = false;
  tc_base = nullptr;
  tc_bytes = 0;
  ws_base = nullptr;
  ws.init(nullptr, 0);
  ++generation;
}

double scal(Ctx& c, int i) { return c.hscal[i]; }

void sync_scalars(Ctx& c, int count) {
  check(dev::d2h(c.hscal, c.dscal, sizeof(double) * count, c.st), "d2h scalars");
  check(dev::sync(c.st), "stream sync");
  int tc = 0;
  check(dev::tc_error(&tc), "tc_error");
  if (tc)
    throw Error(ECG_ERR_TIMEOUT, "GEMM wait timed out (code " + std::to_string(tc) + ")");
}

// --------------------------------------------------------------- setup

// a-block size of the symmetric ladder: Vblk holds v^2 na (v - a0) doubles.
static int64_t ladder_na(int64_t nv) {
  const int64_t budget = (int64_t)1 << 28;  // doubles (2 GiB) for one V block
  int64_t na = (nv + 7) / 8;
  na = std::min<int64_t>(na, std::max<int64_t>(1, budget / std::max<int64_t>(nv * nv * nv, 1)));
  return std::max<int64_t>(1, std::min(na, nv));
}

// Pair tables for the symmetric ladder (host build, one upload).
static void ladder_setup(Ctx& c) {
  const int v = c.nv, o = c.no;
  std::vector<int> cd, ij, pr;
  for (int d = 0; d < v; ++d)
    for (int x = 0; x <= d; ++x) {
      cd.push_back(x);
      cd.push_back(d);
    }
  for (int j = 0; j < o; ++j)
    for (int i = 0; i <= j; ++i) {
      ij.push_back(i);
      ij.push_back(j);
    }
  const int na = (int)ladder_na(v);
  c.lblocks.clear();
  for (int a0 = 0; a0 < v; a0 += na) {
    Ctx::LadderBlock b{a0, std::min(na, v - a0), 0, 0, (int64_t)pr.size() / 2};
    for (int a = a0; a < a0 + b.na; ++a)
      for (int bb = a; bb < v; ++bb) {
        pr.push_back(a);
        pr.push_back(bb);
      }
    b.npp = (int)((int64_t)pr.size() / 2 - b.poff);
    b.npm = b.npp - b.na;
    c.lblocks.push_back(b);
  }
  auto up = [&](std::vector<int>& x, const char* what) {
    int* d = (int*)c.alloc(((int64_t)x.size() + 1) / 2, what);
    check(dev::h2d(d, x.data(), x.size() * sizeof(int), c.st), "h2d tables");
    return d;
  };
  c.cdp = up(cd, "ladder cd pairs");
  c.ijp = up(ij, "ladder ij pairs");
  c.pairs = up(pr, "ladder ab pairs");
  check(dev::sync(c.st), "sync tables");
}

void setup_system(Ctx& c, int no, int nv, int nq, const double* B, const double* h1, double e0) {
  if (no <= 0 || nv <= 0 || nq <= 0) throw Error(ECG_ERR_ARG, "no, nv, nq must be positive");
  c.free_all();
  c.lambda_ready = false;
  c.diis = DiisState();
  c.ldiis = DiisState();
  c.no = no;
  c.nv = nv;
  c.nq = nq;
  c.n = no + nv;
  c.e0 = e0;
  c.ext.no = no;
  c.ext.nv = nv;
  c.ext.nq = nq;
  c.ext.n = c.n;
  const int64_t n = c.n, o = no, v = nv, Q = nq;
  for (int64_t i = 0; i < n * n * Q; ++i)
    if (!std::isfinite(B[i])) throw Error(ECG_ERR_NONFINITE, "non-finite value in B");
  for (int64_t i = 0; i < n * n; ++i)
    if (!std::isfinite(h1[i])) throw Error(ECG_ERR_NONFINITE, "non-finite value in h1");

  c.Bvv = c.alloc(v * v * Q, "Bvv");
  c.Bov = c.alloc(o * v * Q, "Bov");
  c.Bvo = c.alloc(v * o * Q, "Bvo");
  c.Boo = c.alloc(o * o * Q, "Boo");
  c.h = c.alloc(n * n, "h");
  c.fock = c.alloc(n * n, "fock");
  c.eps = c.alloc(n, "eps");
  c.klcd = c.alloc(o * o * v * v, "klcd");
  c.Kvvoo = c.alloc(o * o * v * v, "Kvvoo");
  c.fvo_t = c.alloc(v * o, "fvo_t");
  c.dBvv = c.alloc(v * v * Q, "dBvv");
  c.dBvvT = c.alloc(v * v * Q, "dBvvT");
  c.dBvo = c.alloc(v * o * Q, "dBvo");
  c.dBoo = c.alloc(o * o * Q, "dBoo");
  c.dh = c.alloc(n * n, "dh");
  c.dfock = c.alloc(n * n, "dfock");
  c.J = c.alloc(Q, "J");
  c.T = c.alloc(c.n1() + c.n2(), "T");
  c.R = c.alloc(c.n1() + c.n2(), "R");
  c.TT = c.alloc(c.n2(), "TT");
  c.dscal = c.alloc(256, "scalars");
  c.red = c.alloc(dev::reduce_scratch_len(), "reduce scratch");
  c.dcoef = c.alloc(64, "coefficients");
  c.hscal = (double*)dev::hmalloc_pinned(256 * sizeof(double));
  if (!c.hscal) throw Error(ECG_ERR_OOM, "pinned host scalars");

  const int64_t n2 = c.n2(), na = ladder_na(v);
  int64_t wsn = 16 * n2 + 6 * v * o * Q + 3 * v * v * Q + 2 * n * n * Q + 4 * o * o * o * o +
                3 * na * v * v * v + 8 * n * n + (1 << 16);
  c.ws_base = c.alloc(wsn, "workspace");
  c.ws.init(c.ws_base, wsn);

  // split B[p,q,Q] into the four blocks on the host (input staging only)
  std::vector<double> bvv(v * v * Q), bov(o * v * Q), bvo(v * o * Q), boo(o * o * Q);
  for (int64_t q = 0; q < Q; ++q) {
    const double* Bq = B + q * n * n;
    for (int64_t j = 0; j < n; ++j)
      for (int64_t i = 0; i < n; ++i) {
        double x = Bq[i + j * n];
        if (i < o && j < o) boo[i + j * o + q * o * o] = x;
        else if (i < o) bov[i + (j - o) * o + q * o * v] = x;
        else if (j < o) bvo[(i - o) + j * v + q * v * o] = x;
        else bvv[(i - o) + (j - o) * v + q * v * v] = x;
      }
  }
  check(dev::h2d(c.Bvv, bvv.data(), bvv.size() * 8, c.st), "h2d");
  check(dev::h2d(c.Bov, bov.data(), bov.size() * 8, c.st), "h2d");
  check(dev::h2d(c.Bvo, bvo.data(), bvo.size() * 8, c.st), "h2d");
  check(dev::h2d(c.Boo, boo.data(), boo.size() * 8, c.st), "h2d");
  check(dev::h2d(c.h, h1, n * n * 8, c.st), "h2d");
  c.h_host.assign(h1, h1 + n * n);
  ladder_setup(c);

  // undressed Fock = dressing with T1 = 0 (gen_fock, src/scf/fockfactory.jl:27-30)
  dress(c, nullptr);
  check(dev::d2d(c.fock, c.dfock, n * n * 8, c.st), "d2d");
  check(dev::strided_sum(c.st, n, n + 1, 1, 0, 1.0, c.fock, 0.0, c.eps), "eps");
  // fvo_t[a,i] = f[i,a]
  {
    std::vector<double> tmp(n * n);
    check(dev::d2h(tmp.data(), c.fock, n * n * 8, c.st), "d2h");
    check(dev::sync(c.st), "sync");
    c.fock_host = tmp;
    std::vector<double> fvo(v * o);
    for (int64_t i = 0; i < o; ++i)
      for (int64_t a = 0; a < v; ++a) fvo[a + i * v] = tmp[i + (o + a) * n];
    check(dev::h2d(c.fvo_t, fvo.data(), fvo.size() * 8, c.st), "h2d");
  }
  // <kl|cd> = (kc|ld) = sum_Q B[k,c,Q] B[l,d,Q]   (ints2 "oovv", undressed)
  Contractor con = c.con();
  con(1.0, c.Bov, "kcQ", c.Bov, "ldQ", 0.0, c.klcd, "klcd");
  con.permute(1.0, c.klcd, "ijab", 0.0, c.Kvvoo, "abij");
  check(dev::sync(c.st), "setup sync");
  c.have_system = true;
}

// --------------------------------------------------------------- dressing

// Dressed DF factors, one-electron matrix and Fock matrix.
//   calc_dressed_ints (cc.jl:453-774): every d_* block equals
//     (p^ q^ | r^ s^) = sum_Q dB[p,q,Q] dB[r,s,Q],  dB = (1-t) B (1+t);
//   dress_fock_closedshell (cc.jl:777-815): dh = (1-t) h (1+t),
//     df = dh + 2 sum_k (pq|kk)^ - sum_k (pk|kq)^.
// T1 == nullptr means t = 0 (undressed; used for the plain Fock matrix).
void dress(Ctx& c, const double* T1) {
  const int64_t n = c.n, o = c.no, v = c.nv, Q = c.nq;
  dev::stream_t s = c.st;
  Contractor con = c.con();
  check(dev::d2d(c.dBvv, c.Bvv, v * v * Q * 8, s), "d2d");
  check(dev::d2d(c.dBoo, c.Boo, o * o * Q * 8, s), "d2d");
  check(dev::d2d(c.dBvo, c.Bvo, v * o * Q * 8, s), "d2d");
  check(dev::d2d(c.dh, c.h, n * n * 8, s), "d2d");
  if (T1) {
    // dB_vv = B_vv - T1 B_ov
    con(-1.0, T1, "ai", c.Bov, "ibQ", 1.0, c.dBvv, "abQ");
    // dB_oo = B_oo + B_ov T1   (per Q)
    check(dev::gemm(s, 'N', 'N', o, o, v, 1.0, c.Bov, o, T1, v, 1.0, c.dBoo, o, Q, o * v, 0,
                    o * o),
          "gemm dBoo");
    // dB_vo = B_vo - T1 B_oo + dB_vv T1
    con(-1.0, T1, "ai", c.Boo, "ijQ", 1.0, c.dBvo, "ajQ");
    check(dev::gemm(s, 'N', 'N', v, o, v, 1.0, c.dBvv, v, T1, v, 1.0, c.dBvo, v, Q, v * v, 0,
                    v * o),
          "gemm dBvo");
    // dh = (1 - t) h (1 + t)   (cc.jl:783-787)
    check(dev::gemm(s, 'N', 'N', n, o, v, 1.0, c.h + o * n, n, T1, v, 1.0, c.dh, n), "gemm dh");
    check(dev::gemm(s, 'N', 'N', v, n, o, -1.0, T1, v, c.dh, n, 1.0, c.dh + o, n), "gemm dh");
  }
  // J[Q] = sum_k dB[k,k,Q]
  check(dev::strided_sum(s, Q, o * o, o, o + 1, 1.0, c.dBoo, 0.0, c.J), "J");
  check(dev::d2d(c.dfock, c.dh, n * n * 8, s), "d2d");
  const int64_t mark = c.ws.mark();
  double* G = c.ws.get(v * v);
  struct Blk {
    const double* Bpq;
    int64_t rows, cols, off;
    const double* L;
    const char* il;
    const double* Rm;
    const char* ir;
    const char* ig;
  };
  Blk blks[4] = {
      {c.dBoo, o, o, 0, c.dBoo, "ikQ", c.dBoo, "kjQ", "ij"},
      {c.dBvo, v, o, o, c.dBvo, "akQ", c.dBoo, "kjQ", "aj"},
      {c.Bov, o, v, o * n, c.dBoo, "ikQ", c.Bov, "kbQ", "ib"},
      {c.dBvv, v, v, o + o * n, c.dBvo, "akQ", c.Bov, "kbQ", "ab"},
  };
  for (auto& b : blks) {
    // Coulomb 2 sum_Q dB[p,q,Q] J[Q], exchange - sum_{kQ} dB[p,k,Q] dB[k,q,Q]
    check(dev::gemm(s, 'N', 'N', b.rows * b.cols, 1, Q, 2.0, b.Bpq, b.rows * b.cols, c.J, Q, 0.0,
                    G, b.rows * b.cols),
          "gemm coulomb");
    con(-1.0, b.L, b.il, b.Rm, b.ir, 1.0, G, b.ig);
    check(dev::geam(s, b.rows, b.cols, 1.0, G, b.rows, 1.0, c.dfock + b.off, n), "geam fock");
  }
  c.ws.release(mark);
  // transposed copy used by the ladder: dBvvT[d,b,Q] = dB_vv[b,d,Q]
  con.permute(1.0, c.dBvv, "bdQ", 0.0, c.dBvvT, "dbQ");
}

// --------------------------------------------------------------- residual

// Particle-particle ladder  R2[a,b,i,j] += sum_cd (ac|bd)^ T2[c,d,i,j] with
// (ac|bd)^ = sum_Q Bf[a,c,Q] Bf[b,d,Q] (replaces the kext GEMM,
// cc.jl:1400-1410).  T2 is split into its parts symmetric / antisymmetric
// under c<->d (and then also i<->j); with V+-[ab,cd] = V[acbd] +- V[adbc]
//   L+[ab,ij] = sum_{c<=d} V+ T+,   L-[ab,ij] = sum_{c<d} V- T-
// are symmetric / antisymmetric in (a,b) and (i,j), so only a<=b, i<=j, c<=d
// are formed: a quarter of the contraction flops and, by building V for
// a<=b only (blocks of a against all b >= a0), about half of the DF rebuild.
// V is never stored beyond one a-block.  BfT[c,a,Q] = Bf[a,c,Q].
void ladder(Ctx& c, const double* Bf, const double* BfT, const double* T2, double* R2) {
  (void)Bf;
  const int64_t o = c.no, v = c.nv, Q = c.nq;
  const int64_t ncdp = v * (v + 1) / 2, ncdm = v * (v - 1) / 2;
  const int64_t nijp = o * (o + 1) / 2, nijm = o * (o - 1) / 2;
  // leading dimensions of the packed cd index, rounded up to even so that the
  // TMA-staged FP64 GEMM can address the packed operands
  const int64_t ldp = (ncdp + 1) / 2 * 2, ldm = std::max<int64_t>((ncdm + 1) / 2 * 2, 2);
  dev::stream_t s = c.st;
  const int64_t mark = c.ws.mark();
  double* Ts = c.ws.get(ldp * nijp);
  double* Ta = c.ws.get(std::max<int64_t>(ldm * nijm, 1));
  check(dev::ladder_pack_t(s, (int)v, (int)o, T2, c.cdp, c.ijp, Ts, Ta, ldp, ldm),
        "ladder pack T");
  int64_t maxpp = 0, maxv = 0;
  for (auto& b : c.lblocks) {
    maxpp = std::max<int64_t>(maxpp, b.npp);
    maxv = std::max<int64_t>(maxv, v * b.na * v * (v - b.a0));
  }
  double* V = c.ws.get(maxv);
  double* Vp = c.ws.get(ldp * maxpp);
  double* Vm = c.ws.get(std::max<int64_t>(ldm * maxpp, 1));
  double* Lp = c.ws.get(maxpp * nijp);
  double* Lm = c.ws.get(std::max<int64_t>(maxpp * nijm, 1));
  // Mixed precision: the operands shared by every a-block (BfT for the V
  // build, the packed T2 for the contractions) are split into BF16 slices once
  // per call, each block reads row ranges of them; the per-block V+/- are
  // packed straight into BF16 slices (one pass over V, written in FP32 by the
  // tensor cores, which accumulate it in FP32).  Which GEMMs go to the tensor
  // cores follows gemm_prec's size rule but not its length rule: the V build
  // contracts over the auxiliary index and still runs mixed (measured on
  // (H2O)6/cc-pVTZ, the whole mixed ladder moves the mixed-product fixed
  // point by -4 uEh, the other short contractions by +10).
  const double big = 67108864.0;
  const bool mv = c.mixed_active && (double)(v * c.lblocks[0].na) * (double)(v * v) * Q >= big;
  const bool mp = c.mixed_active && (double)maxpp * nijp * ncdp >= big;
  const bool mm = c.mixed_active && nijm > 0 && (double)maxpp * nijm * ncdm >= big;
  constexpr int NSL = 3;
  dev::TcOperand oB, oTs, oTa, oVp, oVm;
  uint16_t *pB = nullptr, *pTs = nullptr, *pTa = nullptr, *pVp = nullptr, *pVm = nullptr;
  if (mv || mp || mm) {
    const size_t eB = mv ? dev::tc_operand_elems(v * v, Q, NSL) : 0;
    const size_t eTs = mp ? dev::tc_operand_elems(nijp, ncdp, NSL) : 0;
    const size_t eVp = mp ? dev::tc_operand_elems(maxpp, ncdp, NSL) : 0;
    const size_t eTa = mm ? dev::tc_operand_elems(nijm, ncdm, NSL) : 0;
    const size_t eVm = mm ? dev::tc_operand_elems(maxpp, ncdm, NSL) : 0;
    uint16_t* base = (uint16_t*)c.ensure_tc(2 * (eB + eTs + eVp + eTa + eVm));
    pB = base;
    pTs = pB + eB;
    pVp = pTs + eTs;
    pTa = pVp + eVp;
    pVm = pTa + eTa;
    if (mv) check(dev::tc_split(s, BfT, v * v, Q, 1, v * v, NSL, pB, &oB), "split BfT");
    if (mp) check(dev::tc_split(s, Ts, nijp, ncdp, ldp, 1, NSL, pTs, &oTs), "split T+");
    if (mm) check(dev::tc_split(s, Ta, nijm, ncdm, ldm, 1, NSL, pTa, &oTa), "split T-");
  }
  const bool fused = mp && mm;  // V+/- packed into BF16 slices directly
  const bool vf32 = fused && mv && Q <= dev::TC_ACC_K;
  for (auto& b : c.lblocks) {
    const int64_t nb = v - b.a0;
    // V[c,a',d,b''] = sum_Q BfT[c,a0+a',Q] BfT[d,a0+b'',Q]
    if (mv) {
      dev::TcOperand a, bb;
      check(dev::tc_view(oB, v * b.a0, v * b.na, &a), "view BfT");
      check(dev::tc_view(oB, v * b.a0, v * nb, &bb), "view BfT");
      dev::TcGemm g;
      g.m = v * b.na; g.n = v * nb; g.A[0] = &a; g.B[0] = &bb;
      g.C = V; g.scm = 1; g.scn = v * b.na; g.f32 = vf32;
      check(dev::tc_gemm(s, g), "gemm ladder V");
    } else {
      check(dev::gemm(s, 'N', 'T', v * b.na, v * nb, Q, 1.0, BfT + v * b.a0, v * v,
                      BfT + v * b.a0, v * v, 0.0, V, v * b.na),
            "gemm ladder V");
    }
    const int* pairs = c.pairs + 2 * b.poff;
    if (fused) {
      check(dev::ladder_pack_v_split(s, (int)v, b.a0, b.na, b.npp, pairs, c.cdp, V, vf32, pVp,
                                     pVm),
            "pack V");
      check(dev::tc_bind(pVp, b.npp, ncdp, NSL, &oVp), "bind V+");
      if (b.npm > 0) check(dev::tc_bind(pVm, b.npm, ncdm, NSL, &oVm), "bind V-");
    } else {
      check(dev::ladder_pack_v(s, (int)v, b.a0, b.na, b.npp, pairs, c.cdp, V, Vp, Vm, ldp, ldm),
            "pack V");
    }
    if (mp) {
      if (!fused) check(dev::tc_split(s, Vp, b.npp, ncdp, ldp, 1, NSL, pVp, &oVp), "split V+");
      dev::TcGemm g;
      g.m = b.npp; g.n = nijp; g.A[0] = &oVp; g.B[0] = &oTs;
      g.C = Lp; g.scm = 1; g.scn = b.npp;
      check(dev::tc_gemm(s, g), "gemm ladder +");
    } else {
      check(dev::gemm(s, 'T', 'N', b.npp, nijp, ncdp, 1.0, Vp, ldp, Ts, ldp, 0.0, Lp, b.npp),
            "gemm ladder +");
    }
    if (b.npm > 0 && nijm > 0) {
      if (mm) {
        if (!fused) check(dev::tc_split(s, Vm, b.npm, ncdm, ldm, 1, NSL, pVm, &oVm), "split V-");
        dev::TcGemm g;
        g.m = b.npm; g.n = nijm; g.A[0] = &oVm; g.B[0] = &oTa;
        g.C = Lm; g.scm = 1; g.scn = b.npm;
        check(dev::tc_gemm(s, g), "gemm ladder -");
      } else {
        check(dev::gemm(s, 'T', 'N', b.npm, nijm, ncdm, 1.0, Vm, ldm, Ta, ldm, 0.0, Lm,
                        b.npm),
              "gemm ladder -");
      }
    }
    check(dev::ladder_unpack(s, (int)v, (int)o, b.a0, b.npp, pairs, c.ijp, Lp, Lm, R2),
          "ladder unpack");
  }
  c.ws.release(mark);
}

// calc_cc_resid closed shell (src/cc/cc.jl:1343-1489), DF form.
void cc_residual(Ctx& c, bool dc) {
  const int64_t n = c.n, o = c.no, v = c.nv, Q = c.nq, n2 = c.n2();
  dev::stream_t s = c.st;
  Contractor con = c.con();
  const double* T1 = c.T1();
  const double* T2 = c.T2();
  double* R1 = c.R1();
  double* R2 = c.R2();
  dress(c, T1);
  const int64_t mark = c.ws.mark();
  double* Tt = c.ws.get(n2);
  // T2t[a,b,i,j] = 2 T2[a,b,i,j] - T2[b,a,i,j]   (cc.jl:1354)
  check(dev::axpby(s, n2, 2.0, T2, 0.0, Tt), "Tt");
  con.permute(-1.0, T2, "baij", 1.0, Tt, "abij");

  // ---- singles (cc.jl:1357-1375 and the R1 part of kext, :1418-1420) ----
  // R1 = df[v,o] + sum_{Qc} dB[a,c,Q] W[c,i,Q] - sum_{jQ} W[a,j,Q] dB[j,i,Q]
  //      + sum_{jb} T2t[a,b,i,j] df[j,b],
  // W[c,i,Q] = sum_{ld} T2t[c,d,i,l] B[l,d,Q].  (The (ai|kk)-type pieces of
  // the kext singles equal df - dh and are carried by df[v,o].)
  check(dev::geam(s, v, o, 1.0, c.dfock + o, n, 0.0, R1, v), "R1 = df_vo");
  double* W3 = c.ws.get(v * o * Q);
  con(1.0, Tt, "cdil", c.Bov, "ldQ", 0.0, W3, "ciQ");
  con(1.0, c.dBvv, "acQ", W3, "ciQ", 1.0, R1, "ai");
  con(-1.0, W3, "ajQ", c.dBoo, "jiQ", 1.0, R1, "ai");
  double* fov = c.ws.get(o * v);
  check(dev::geam(s, o, v, 1.0, c.dfock + o * n, n, 0.0, fov, o), "fov");
  con(1.0, Tt, "abij", fov, "jb", 1.0, R1, "ai");

  // ---- I_klij T^kl_ab (cc.jl:1387-1398) ----
  double* I = c.ws.get(o * o * o * o);
  con(1.0, c.dBoo, "kiQ", c.dBoo, "ljQ", 0.0, I, "klij");
  if (!dc) con(1.0, c.klcd, "klcd", T2, "cdij", 1.0, I, "klij");
  con(1.0, T2, "abkl", I, "klij", 0.0, R2, "abij");

  // ---- kext doubles: dressed ladder + (ai|bj)^ (cc.jl:1400-1417) ----
  con(1.0, c.dBvo, "aiQ", c.dBvo, "bjQ", 1.0, R2, "abij");
  ladder(c, c.dBvv, c.dBvvT, T2, R2);

  // ---- quadratic term, CCSD only (cc.jl:1433-1437) ----
  double* Y = c.ws.get(n2);
  if (!dc) {
    con(1.0, c.klcd, "klcd", T2, "adkj", 0.0, Y, "lcaj");
    con(1.0, Y, "lcaj", T2, "cbil", 1.0, R2, "abij");
  }

  // ---- x_ad, x_ki (cc.jl:1440-1450) ----
  const double fac = dc ? 0.5 : 1.0;
  double* xad = c.ws.get(v * v);
  double* xki = c.ws.get(o * o);
  check(dev::geam(s, v, v, 1.0, c.dfock + o + o * n, n, 0.0, xad, v), "xad");
  check(dev::geam(s, o, o, 1.0, c.dfock, n, 0.0, xki, o), "xki");
  con(-fac, c.klcd, "klcd", Tt, "cakl", 1.0, xad, "ad");
  con(fac, c.klcd, "klcd", Tt, "cdil", 1.0, xki, "ki");

  // ---- P(ia;jb) terms (cc.jl:1452-1484) ----
  double* R2r = c.ws.get(n2);
  con(1.0, xad, "ad", T2, "dbij", 0.0, R2r, "abij");
  con(-1.0, T2, "abkj", xki, "ki", 1.0, R2r, "abij");
  double* W = c.ws.get(n2);
  // d_voov[a,k,i,c] = (ai|kc)^ + 0.5 <kl|cd> T2t[a,d,i,l]
  con(1.0, c.dBvo, "aiQ", c.Bov, "kcQ", 0.0, W, "akic");
  con(0.5, c.klcd, "klcd", Tt, "adil", 1.0, W, "akic");
  con(1.0, W, "akic", Tt, "cbkj", 1.0, R2r, "abij");
  if (!dc) {
    // T2t - T2 = T2[a,b,i,j] - T2[b,a,i,j]
    check(dev::axpby(s, n2, -1.0, T2, 1.0, Tt), "Tt-T2");
    con(1.0, c.klcd, "klcd", T2, "daki", 0.0, Y, "lcai");
    con(-1.0, Y, "lcai", Tt, "cblj", 1.0, R2r, "abij");
  }
  // d_vovo[a,k,c,i] = (ac|ki)^
  con(1.0, c.dBvv, "acQ", c.dBoo, "kiQ", 0.0, W, "akci");
  con(-1.0, W, "akci", T2, "cbkj", 1.0, R2r, "abij");
  con(-1.0, W, "bkci", T2, "ackj", 1.0, R2r, "abij");
  // R2 += R2r + R2r[b,a,j,i]
  check(dev::axpby(s, n2, 1.0, R2r, 1.0, R2), "R2 += R2r");
  con.permute(1.0, R2r, "baji", 1.0, R2, "abij");
  c.ws.release(mark);
  (void)Q;
}

// --------------------------------------------------------------- DIIS

// Solve the DIIS equations like `svd(bmat)\rhs` (src/solvers/diis.jl:261):
// pseudo-inverse dropping singular values below eps*smax.  B is symmetric, so
// its singular values are |eigenvalues|; a cyclic Jacobi eigensolver is used.
static void sym_pinv_solve(int m, const std::vector<double>& B, const std::vector<double>& rhs,
                           std::vector<double>& x) {
  std::vector<double> A(B), V(m * m, 0.0);
  for (int i = 0; i < m; ++i) V[i * m + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < m; ++p)
      for (int q = p + 1; q < m; ++q) off += A[p * m + q] * A[p * m + q];
    if (off < 1e-300) break;
    for (int p = 0; p < m; ++p)
      for (int q = p + 1; q < m; ++q) {
        double apq = A[p * m + q];
        if (apq == 0.0) continue;
        double app = A[p * m + p], aqq = A[q * m + q];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < m; ++k) {
          double akp = A[k * m + p], akq = A[k * m + q];
          A[k * m + p] = cs * akp - sn * akq;
          A[k * m + q] = sn * akp + cs * akq;
        }
        for (int k = 0; k < m; ++k) {
          double apk = A[p * m + k], aqk = A[q * m + k];
          A[p * m + k] = cs * apk - sn * aqk;
          A[q * m + k] = sn * apk + cs * aqk;
        }
        for (int k = 0; k < m; ++k) {
          double vkp = V[k * m + p], vkq = V[k * m + q];
          V[k * m + p] = cs * vkp - sn * vkq;
          V[k * m + q] = sn * vkp + cs * vkq;
        }
      }
  }
  double smax = 0.0;
  for (int i = 0; i < m; ++i) smax = std::max(smax, std::fabs(A[i * m + i]));
  const double cut = 2.220446049250313e-16 * smax;
  x.assign(m, 0.0);
  for (int i = 0; i < m; ++i) {
    double lam = A[i * m + i];
    if (std::fabs(lam) < cut || lam == 0.0) continue;
    double proj = 0.0;
    for (int k = 0; k < m; ++k) proj += V[k * m + i] * rhs[k];
    for (int k = 0; k < m; ++k) x[k] += V[k * m + i] * proj / lam;
  }
}

void diis_reset(Ctx& c, DiisState& d, int maxdiis, double resthr, int64_t len, bool cs) {
  if (maxdiis < 1 || maxdiis > 8) throw Error(ECG_ERR_ARG, "maxdiis must be in 1..8");
  if (d.len != len || (int)d.amp.size() != maxdiis) {
    d.amp.assign(maxdiis, nullptr);
    d.res.assign(maxdiis, nullptr);
    for (int i = 0; i < maxdiis; ++i) {
      d.amp[i] = c.alloc(len, "diis amp");
      d.res[i] = c.alloc(len, "diis res");
    }
  }
  d.maxdiis = maxdiis;
  d.resthr = resthr;
  d.len = len;
  d.next = 0;
  d.ndim = 0;
  d.cs = cs;
  d.bmat.assign((maxdiis + 1) * (maxdiis + 1), 0.0);
}

// Launch the dot of `res` with DIIS slot i into scalars [2+3i, 4+3i].
static void diis_dot(Ctx& c, DiisState& d, const double* res, const double* other, int slot) {
  double* out = c.dscal + 128 + 3 * slot;
  if (d.cs) {
    check(dev::dot(c.st, c.n1(), res, other, c.red, out), "diis dot1");
    check(dev::cs_dot(c.st, c.nv, c.no, res + c.n1(), other + c.n1(), c.red, out + 1), "diis dot2");
  } else {
    check(dev::dot(c.st, d.len, res, other, c.red, out), "diis dot");
  }
}

static double diis_dot_value(Ctx& c, const DiisState& d, int slot) {
  const double* h = c.hscal + 128 + 3 * slot;
  if (d.cs) return 2.0 * h[0] + 2.0 * h[1] - h[2];
  return h[0];
}

// perform! (diis.jl:246-305) on device vectors; the B matrix and the small
// linear solve live on the host in FP64.  `amps` is replaced by the
// extrapolated vector.
void diis_perform(Ctx& c, DiisState& d, double* amps, const double* res) {
  if (d.ndim < d.maxdiis) d.ndim += 1;
  const int ithis = d.next, nd = d.ndim, M = d.maxdiis + 1;
  check(dev::d2d(d.amp[ithis], amps, d.len * 8, c.st), "diis save amps");
  check(dev::d2d(d.res[ithis], res, d.len * 8, c.st), "diis save res");
  for (int i = 0; i < nd; ++i) diis_dot(c, d, res, i == ithis ? res : d.res[i], i);
  sync_scalars(c, 128 + 3 * nd);
  for (int i = 0; i < nd; ++i) {
    double dv = diis_dot_value(c, d, i);
    d.bmat[i * M + ithis] = dv;
    d.bmat[ithis * M + i] = dv;
    d.bmat[i * M + nd] = -1.0;
    d.bmat[nd * M + i] = -1.0;
  }
  d.bmat[nd * M + nd] = 0.0;
  const double thisdot = diis_dot_value(c, d, ithis);
  std::vector<double> B((nd + 1) * (nd + 1)), rhs(nd + 1, 0.0), x;
  for (int i = 0; i <= nd; ++i)
    for (int j = 0; j <= nd; ++j) B[i * (nd + 1) + j] = d.bmat[i * M + j];
  rhs[nd] = -1.0;
  sym_pinv_solve(nd + 1, B, rhs, x);
  if (nd == 1 && d.next == 0 && thisdot > d.resthr) {
    d.ndim = 0;
    return;
  } else if (nd < d.maxdiis) {
    d.next = nd;
  } else {
    double cmin = 1.0e10;
    for (int i = 0; i < nd; ++i)
      if (std::fabs(x[i]) < cmin && (i != ithis || nd == 1)) {
        cmin = std::fabs(x[i]);
        d.next = i;
      }
  }
  for (int i = 0; i < nd; ++i) c.hscal[200 + i] = x[i];
  check(dev::h2d(c.dcoef, c.hscal + 200, nd * 8, c.st), "h2d coef");
  std::vector<const double*> X(d.amp.begin(), d.amp.begin() + nd);
  check(dev::combine(c.st, d.len, nd, X.data(), c.dcoef, amps), "diis combine");
  // the coefficient upload reads pinned memory asynchronously
  check(dev::sync(c.st), "diis sync");
}

// --------------------------------------------------------------- iteration

void cc_init_iterations(Ctx& c, const ecg_cc_opts& o) {
  c.opts = o;
  diis_reset(c, c.diis, o.maxdiis, o.resthr, c.n1() + c.n2(), o.diis_dot == ECG_DIIS_CS);
}

// Energy-type reductions of T (and R) into scalars starting at `base`:
//   [base+0,1] cs_dot(T2, <ij|ab>), [base+2,3] cs_dot(T1 T1, <ij|ab>),
//   [base+4] dot(f_ov^T, T1)
static void energy_dots(Ctx& c, int base) {
  dev::stream_t s = c.st;
  check(dev::cs_dot(s, c.nv, c.no, c.T2(), c.Kvvoo, c.red, c.dscal + base), "e dot");
  check(dev::outer(s, c.nv, c.no, c.nv, c.no, 1.0, c.T1(), c.T1(), 0.0, c.TT), "outer");
  check(dev::cs_dot(s, c.nv, c.no, c.TT, c.Kvvoo, c.red, c.dscal + base + 2), "e dot");
  check(dev::dot(s, c.n1(), c.fvo_t, c.T1(), c.red, c.dscal + base + 4), "e dot");
}

// One pass of the cc_iterations! body (src/cc/cc.jl:2546-2628).
IterResult cc_iteration(Ctx& c, bool dc) {
  dev::stream_t s = c.st;
  cc_residual(c, dc);
  // norms and Hylleraas pieces (cc.jl:2568-2577; calc_hylleraas cc.jl:195-249)
  check(dev::cs_dot(s, c.nv, c.no, c.R2(), c.R2(), c.red, c.dscal + 0), "norm R2");
  check(dev::dot(s, c.n1(), c.R1(), c.R1(), c.red, c.dscal + 2), "norm R1");
  energy_dots(c, 3);  // 3..7
  check(dev::cs_dot(s, c.nv, c.no, c.T2(), c.R2(), c.red, c.dscal + 8), "rdot");
  check(dev::dot(s, c.n1(), c.R1(), c.T1(), c.red, c.dscal + 10), "rdot1");
  sync_scalars(c, 11);
  double sc[11];
  std::memcpy(sc, c.hscal, sizeof sc);
  // update (cctools.jl:284-300)
  const double* eo = c.eps;
  const double* ev = c.eps + c.no;
  check(dev::update_doubles(s, c.nv, c.no, eo, ev, c.opts.shiftp, c.R2(), c.T2()), "upd2");
  check(dev::update_singles(s, c.nv, c.no, eo, ev, c.opts.shifts, c.R1(), c.T1()), "upd1");
  diis_perform(c, c.diis, c.T, c.R);
  energy_dots(c, 20);
  sync_scalars(c, 25);
  const double* e = c.hscal + 20;

  IterResult r{};
  const double NormR2 = 2.0 * sc[0] - sc[1], NormR1 = 2.0 * sc[2];
  const double pd = sc[3], pex = sc[4], d1 = sc[5], ex1 = sc[6], fT = sc[7];
  const double rd = sc[8], rex = sc[9], RT = sc[10];
  const double ET1SS = d1 - ex1, ET1OS = d1;
  const double ET2d = pd + rd, ET2ex = pex + rex;
  const double ET2SS = ET2d - ET2ex, ET2OS = ET2d;
  const double ET1 = ET1SS + ET1OS + 2.0 * fT + 2.0 * RT;
  r.E = ET2SS + ET2OS + ET1;
  r.ESS = ET2SS + ET1SS;
  r.EOS = ET2OS + ET1OS;
  r.En = (2.0 * e[0] - e[1]) + (2.0 * e[2] - e[3]) + 2.0 * e[4];
  r.dE = r.En - r.E;
  r.normR = NormR1 + NormR2;
  if (!std::isfinite(r.E) || !std::isfinite(r.normR))
    throw Error(ECG_ERR_NONFINITE, "non-finite energy or residual norm in CC iteration");
  return r;
}

}  // namespace ecg
