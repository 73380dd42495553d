// ecg_triples.cpp — closed-shell (T) and Lambda-(T).
//
// For each occupied triplet i <= j <= k (i = j = k skipped, weights 2/1 as in
// cc_triples.jl:62-72) the 12 contractions of cc_triples.jl:89-104 are
// regrouped as K = P[W]:
//   W^{xyz}[a,b,c] = sum_d T^{xy}_{ad} (bd|cz) - sum_l T^{xl}_{ab} (ly|cz)
//   K[a,b,c] = W^{ijk}[a,b,c] + W^{jik}[b,a,c] + W^{ikj}[a,c,b]
//            + W^{kji}[c,b,a] + W^{jki}[b,c,a] + W^{kij}[c,a,b]
// The six vvvo GEMMs (M=v, N=v^2, K=v) accumulate straight into K: each
// epilogue writes W^{xyz}[a',(b',c')] to its permuted position in K.  vvvo is
// held in two layouts, [b,c,d,k] and [c,b,d,k], chosen per permutation so
// that the (b',c') pair maps to K through at most one index split; with that
// choice the permutations pair up into three GEMMs of K depth 2v whose two
// halves write the same K positions.  On the
// tensor cores, whose epilogue lanes run along the GEMM rows, a GEMM whose
// a' index is not the unit stride of K is run transposed (rows (b',c')).
// With T^{xy}_{ab} = T^{yx}_{ba} the six ovoo GEMMs pair up into three GEMMs
// with a two-segment K of 2o, also accumulated into K.  A fused kernel forms
// X and both energy sums (sum K X and the singles/Fock term sum X Y,
// cc_triples.jl:113-156); per-triplet energies are summed on the host in
// triplet order, so the result is deterministic.
//
// Mixed precision: every operand is split into two BF16 slices once per call
// (vvvo in both layouts, T^{xy} per pair, T2[:,:,x,:] and T2[:,:,:,x] per
// occupied index, -ovoo per pair), the GEMMs run on the tensor cores and K is
// kept in FP32.  Each ovoo pair writes K through the same index map, and with
// the same rows and columns, as one vvvo pair, so every K orientation is one
// tensor-core GEMM of four K segments (v, v, o, o): three launches per batch,
// each with a single pass over K.
#include "ecg_triples.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace ecg {

namespace {

// BF16 slices of the (T) operands in mixed precision: two slices (products
// hi*hi + hi*lo + lo*hi, ~2^-16 relative per product) keep the (T) energy
// within ~1e-8 relative of FP64, since the element errors average out.
constexpr int kTriplesSlices = 2;

// One W GEMM of K = P[W]: amplitudes T^{xy}, integrals of occupied z in the
// [b,c,d] (l2 = false) or [c,b,d] (l2 = true) layout, and where W[a',n] lands
// in K: K[a'*scm + (n % dn)*scn + (n / dn)*scn2] (dn = 0: n*scn).
struct PermW {
  int x, y, z;
  bool l2;
  int64_t scm, scn, dn, scn2;
};

// n = b' + v c' in the [b,c,d] layout, n = c' + v b' in the [c,b,d] layout.
// K[a,b,c] sits at a + vp b + vp v c (vp >= v: the padded pitch of the a
// index; vp = v for FP64 K, a multiple of 4 for FP32 K so that the energy
// kernel's TMA copies start on 16 bytes).
void perm_table(int i, int j, int k, int64_t v, int64_t vp, PermW* P) {
  const int64_t pv = vp * v;
  P[1] = {j, i, k, false, vp, 1, v, pv};   // W^{jik} -> K[b',a',c'] = vp a' + b' + vp v c'
  P[4] = {j, k, i, true, vp, 1, v, pv};    // W^{jki} -> K[c',a',b'] = vp a' + c' + vp v b'
  if (vp == v) {  // unpadded: the column index n maps with one stride
    P[0] = {i, j, k, false, 1, v, 0, 0};   // W^{ijk} -> K[a',b',c'] = a' + v n
    P[2] = {i, k, j, true, 1, v, 0, 0};    // W^{ikj} -> K[a',c',b'] = a' + v n
    P[3] = {k, j, i, true, pv, 1, 0, 0};   // W^{kji} -> K[c',b',a'] = v^2 a' + n
    P[5] = {k, i, j, false, pv, 1, 0, 0};  // W^{kij} -> K[b',c',a'] = v^2 a' + n
  } else {
    P[0] = {i, j, k, false, 1, vp, v, pv};  // K[a',b',c'] = a' + vp b' + vp v c'
    P[2] = {i, k, j, true, 1, vp, v, pv};   // K[a',c',b'] = a' + vp c' + vp v b'
    P[3] = {k, j, i, true, pv, 1, v, vp};   // K[c',b',a'] = c' + vp b' + vp v a'
    P[5] = {k, i, j, false, pv, 1, v, vp};  // K[b',c',a'] = b' + vp c' + vp v a'
  }
}

// BF16 operands of one amplitude tensor (T2 or covariant U2).
struct SplitAmps {
  std::vector<dev::TcOperand> pair;  // T^{xy}[a,d]: rows a, k d        (x + o*y)
  std::vector<dev::TcOperand> G;     // T2[:,:,x,l]: rows (a,b), k l    (x)
  std::vector<dev::TcOperand> C;     // T2[:,:,l,x]: rows (a,b), k l    (x)
};

uint16_t* alloc_bf16(Ctx& c, size_t elems, const char* what) {
  return reinterpret_cast<uint16_t*>(c.alloc((int64_t)((elems + 3) / 4), what));
}

void split_amps(Ctx& c, const double* T, SplitAmps& S) {
  const int64_t o = c.no, v = c.nv, v2 = v * v;
  dev::stream_t s = c.st;
  S.pair.resize(o * o);
  S.G.resize(o);
  S.C.resize(o);
  const size_t ep = dev::tc_operand_elems(v, v, kTriplesSlices);
  const size_t eg = dev::tc_operand_elems(v2, o, kTriplesSlices);
  uint16_t* bp = alloc_bf16(c, ep * o * o, "(T) T^{xy} BF16");
  uint16_t* bg = alloc_bf16(c, 2 * eg * o, "(T) T2 slices BF16");
  for (int64_t y = 0; y < o; ++y)
    for (int64_t x = 0; x < o; ++x)
      check(dev::tc_split(s, T + v2 * (x + o * y), v, v, 1, v, kTriplesSlices,
                          bp + ep * (x + o * y), &S.pair[x + o * y]),
            "split T^{xy}");
  for (int64_t x = 0; x < o; ++x) {
    check(dev::tc_split(s, T + v2 * x, v2, o, 1, v2 * o, kTriplesSlices, bg + eg * x, &S.G[x]),
          "split T2 G");
    check(dev::tc_split(s, T + v2 * o * x, v2, o, 1, v2, kTriplesSlices, bg + eg * (o + x),
                        &S.C[x]),
          "split T2 C");
  }
}

// Everything the K builds read: FP64 integrals and amplitudes, or their
// BF16 splits.
struct TriplesOps {
  bool mixed = false;
  const double* V1 = nullptr;  // [b,c,d,k]
  const double* V2 = nullptr;  // [c,b,d,k]
  const double* On = nullptr;  // [l,j,c,k]
  std::vector<dev::TcOperand> V1s, V2s, Ons;
};

// One occupied triplet of the sweep: indices, weight (cc_triples.jl:62-72) and
// the denominator shift e_i + e_j + e_k.
struct Trip {
  int i, j, k;
  double f, eijk;
};

// Host-built tables of one amplitude tensor's K builds for the whole sweep,
// uploaded once: FP64 offset tables [9 GEMMs][triplet][A, B, C, A1, B1] or
// tensor-core descriptor tables [3 GEMMs][triplet][maps of 4 segments].  The C offset is the
// triplet's slot in its batch.
struct KTables {
  std::vector<int64_t> ptab;
  std::vector<unsigned char> mtab;
  int64_t* ptab_d = nullptr;
  unsigned char* mtab_d = nullptr;
};

constexpr int kGemmsFP64 = 9, kGemmsMixed = 3;

void fill_tables(Ctx& c, const TriplesOps& ops, const SplitAmps* Sp, const std::vector<Trip>& tr,
                 int NB, int64_t kstride, int64_t vp, KTables& kt) {
  const int64_t o = c.no, v = c.nv, v2 = v * v, v3 = v2 * v, o2 = o * o;
  const int64_t nt = (int64_t)tr.size();
  auto on = [&](int y, int z) { return o * y + o2 * v * z; };
  if (!ops.mixed) {
    kt.ptab.assign(kGemmsFP64 * nt * 5, 0);
    for (int64_t t = 0; t < nt; ++t) {
      const int i = tr[t].i, j = tr[t].j, k = tr[t].k;
      const int64_t offC = (t % NB) * kstride;
      PermW P[6];
      perm_table(i, j, k, v, vp, P);
      auto put = [&](int q, int64_t a, int64_t b, int64_t a1, int64_t b1) {
        int64_t* e = kt.ptab.data() + (q * nt + t) * 5;
        e[0] = a; e[1] = b; e[2] = offC; e[3] = a1; e[4] = b1;
      };
      for (int q = 0; q < 6; ++q) put(q, v2 * (P[q].x + o * P[q].y), v3 * P[q].z, 0, 0);
      put(6, v2 * i, on(j, k), v2 * o * j, on(i, k));
      put(7, on(k, j), v2 * i, on(i, j), v2 * o * k);
      put(8, v2 * o * k, on(j, i), v2 * j, on(k, i));
    }
    return;
  }
  const size_t mb = dev::tc_maps_bytes();
  kt.mtab.assign(kGemmsMixed * nt * mb, 0);
  auto op = [&](int y, int z) { return &ops.Ons[y + o * z]; };
  for (int64_t t = 0; t < nt; ++t) {
    const int i = tr[t].i, j = tr[t].j, k = tr[t].k;
    PermW P[6];
    perm_table(i, j, k, v, vp, P);
    // ovoo pairs (A of both segments, B of both segments) in the order of
    // the vvvo pairs they share K's index map with
    const dev::TcOperand* ovoo[3][4] = {
        {op(j, i), op(k, i), &Sp->C[k], &Sp->G[j]},   // rows a, columns (b,c)
        {&Sp->G[i], &Sp->C[k], op(k, j), op(i, j)},   // rows (a,c), columns b
        {&Sp->G[i], &Sp->C[j], op(j, k), op(i, k)}};  // rows (a,b), columns c
    const int pairs[3][2] = {{0, 2}, {1, 4}, {3, 5}};
    for (int q = 0; q < 3; ++q) {
      const PermW& p0 = P[pairs[q][0]];
      const PermW& p1 = P[pairs[q][1]];
      const dev::TcOperand* T0 = &Sp->pair[p0.x + o * p0.y];
      const dev::TcOperand* T1 = &Sp->pair[p1.x + o * p1.y];
      const dev::TcOperand* V0 = p0.l2 ? &ops.V2s[p0.z] : &ops.V1s[p0.z];
      const dev::TcOperand* V1 = p1.l2 ? &ops.V2s[p1.z] : &ops.V1s[p1.z];
      const bool rows_a = p0.scm == 1;
      const dev::TcOperand* A[4] = {rows_a ? T0 : V0, rows_a ? T1 : V1, ovoo[q][0], ovoo[q][1]};
      const dev::TcOperand* B[4] = {rows_a ? V0 : T0, rows_a ? V1 : T1, ovoo[q][2], ovoo[q][3]};
      check(dev::tc_maps_fill(4, A, B, rows_a ? v2 : v, kt.mtab.data() + (q * nt + t) * mb),
            "maps");
    }
  }
}

void upload_tables(Ctx& c, KTables& kt) {
  dev::stream_t s = c.st;
  if (!kt.ptab.empty()) {
    kt.ptab_d = reinterpret_cast<int64_t*>(c.alloc((int64_t)kt.ptab.size(), "(T) offset table"));
    check(dev::h2d(kt.ptab_d, kt.ptab.data(), kt.ptab.size() * 8, s), "h2d");
  }
  if (!kt.mtab.empty()) {
    kt.mtab_d = reinterpret_cast<unsigned char*>(
        c.alloc((int64_t)((kt.mtab.size() + 7) / 8), "(T) descriptor table"));
    check(dev::h2d(kt.mtab_d, kt.mtab.data(), kt.mtab.size(), s), "h2d");
  }
}

// K^{ijk} = P[W] for triplets t0 .. t0+nb-1 into K slots 0 .. nb-1 (FP64 or
// FP32), one launch per GEMM kind.
void build_K_batch(Ctx& c, const TriplesOps& ops, const double* T, const SplitAmps* Sp,
                   const KTables& kt, int64_t nt, int64_t t0, int nb, void* K, int64_t kstride,
                   int64_t vp) {
  const int64_t o = c.no, v = c.nv, v2 = v * v, o2 = o * o;
  dev::stream_t s = c.st;
  PermW P[6];
  perm_table(0, 0, 0, v, vp, P);  // output maps and layouts do not depend on i, j, k
  if (!ops.mixed) {
    auto tab = [&](int q) { return kt.ptab_d + (q * nt + t0) * 5; };
    // The vvvo GEMMs (M = v, N = v^2, K = v): one GEMM per triplet, its
    // operands placed from the host copy of the offset table; each fills the
    // GPU by itself (v/64 x v^2/64 tiles) and runs on the TMA-staged kernel
    // through K's index map.  Per K element the six contributions still add in
    // the order q = 0..5.
    for (int q = 0; q < 6; ++q)
      for (int it = 0; it < nb; ++it) {
        const int64_t* e = kt.ptab.data() + (q * nt + t0 + it) * 5;
        dev::Gemm g;
        g.m = v; g.n = v2; g.k = v; g.batch = 1; g.alpha = 1.0; g.beta = q ? 1.0 : 0.0;
        g.A = T + e[0]; g.sam = 1; g.sak = v;
        g.B = (P[q].l2 ? ops.V2 : ops.V1) + e[1]; g.sbk = v2; g.sbn = 1;
        g.C = (double*)K + e[2];
        g.scm = P[q].scm; g.scn = P[q].scn; g.dn = P[q].dn; g.scn2 = P[q].scn2;
        g.mapped_tma = true;
        check(dev::gemm_strided(s, g), "W vvvo");
      }
    dev::Gemm g;
    g.k = 2 * o; g.kseg = o; g.alpha = -1.0; g.beta = 1.0; g.C = (double*)K; g.batch = nb;
    // (1) rows (a,b), columns c
    g.m = v2; g.n = v; g.A = T; g.sam = 1; g.sak = v2 * o; g.A1 = T; g.sak1 = v2;
    g.B = ops.On; g.sbk = 1; g.sbn = o2; g.B1 = ops.On; g.sbk1 = 1;
    g.scm = 1; g.scn = v2; g.dn = 0; g.scn2 = 0; g.ptab = tab(6);
    check(dev::gemm_strided(s, g), "W ovoo 1");
    // (2) rows b, columns (a,c)
    g.m = v; g.n = v2; g.A = ops.On; g.sam = o2; g.sak = 1; g.A1 = ops.On; g.sak1 = 1;
    g.B = T; g.sbk = v2 * o; g.sbn = 1; g.B1 = T; g.sbk1 = v2;
    g.scm = v; g.scn = 1; g.dn = v; g.scn2 = v2; g.ptab = tab(7);
    check(dev::gemm_strided(s, g), "W ovoo 2");
    // (3) rows (b,c), columns a
    g.m = v2; g.n = v; g.A = T; g.sam = 1; g.sak = v2; g.A1 = T; g.sak1 = v2 * o;
    g.B = ops.On; g.sbk = 1; g.sbn = o2; g.B1 = ops.On; g.sbk1 = 1;
    g.scm = v; g.scn = 1; g.dn = 0; g.scn2 = 0; g.ptab = tab(8);
    check(dev::gemm_strided(s, g), "W ovoo 3");
    return;
  }
  const size_t mb = dev::tc_maps_bytes();
  auto tab = [&](int q) { return kt.mtab_d + (q * nt + t0) * mb; };
  // shape representatives (every triplet's operands have the same shapes)
  const dev::TcOperand* Tp = &Sp->pair[0];
  const dev::TcOperand* Vp = &ops.V1s[0];
  const dev::TcOperand* Op = &ops.Ons[0];
  const dev::TcOperand* Gp = &Sp->G[0];
  const int pairs[3][2] = {{0, 2}, {1, 4}, {3, 5}};
  for (int q = 0; q < 3; ++q) {
    const PermW& p0 = P[pairs[q][0]];
    dev::TcGemm g;
    g.alpha = 1.0; g.beta = q ? 1.0 : 0.0; g.C = K; g.f32 = true;
    if (p0.scm == 1) {  // rows a', columns (b',c'); ovoo rows a
      g.m = v; g.n = v2;
      g.A[0] = g.A[1] = Tp; g.B[0] = g.B[1] = Vp; g.A[2] = g.A[3] = Op; g.B[2] = g.B[3] = Gp;
      g.scm = 1; g.scn = p0.scn; g.dn = p0.dn; g.scn2 = p0.scn2;
    } else {            // rows (b',c'), columns a'; ovoo rows (a,b) or (a,c)
      g.m = v2; g.n = v;
      g.A[0] = g.A[1] = Vp; g.B[0] = g.B[1] = Tp; g.A[2] = g.A[3] = Gp; g.B[2] = g.B[3] = Op;
      g.scm = p0.scn; g.dm = p0.dn; g.scm2 = p0.scn2; g.scn = p0.scm;
    }
    check(dev::tc_gemm_batched(s, g, nb, tab(q), kstride), "W");
  }
}

}  // namespace

void pert_triples(Ctx& c, const double* U1h, const double* U2h, double* et, double* etb) {
  const int64_t o = c.no, v = c.nv, v2 = v * v, v3 = v2 * v, n = c.n;
  const bool lam = (U1h != nullptr);
  const bool mixed = c.mixed_active;
  dev::stream_t s = c.st;
  // everything allocated here is freed on exit
  struct Scope {
    Ctx& c;
    size_t n0;
    ~Scope() { c.release_to(n0); }
  } scope{c, c.allocs.size()};

  TriplesOps ops;
  ops.mixed = mixed;
  double* On = c.alloc(o * o * o * v, "(T) ovoo");
  ops.On = On;
  Contractor con = c.con();
  con(1.0, c.Boo, "ljQ", c.Bvo, "ckQ", 0.0, On, "ljck");
  // vvvo[b,c,d,k] = (bd|ck): per k, a GEMM batched over d; [c,b,d,k] by permutation
  const int64_t d3[3] = {v, v, v};
  const int swap01[3] = {1, 0, 2};
  auto build_v = [&](int64_t kk, double* out) {
    dev::Gemm g;
    g.m = v; g.n = v; g.k = c.nq; g.batch = v; g.alpha = 1.0; g.beta = 0.0;
    g.A = c.Bvv; g.sam = 1; g.sak = v * v; g.sab = v;
    g.B = c.Bvo + v * kk; g.sbk = v * o; g.sbn = 1; g.sbb = 0;
    g.C = out; g.scm = 1; g.scn = v; g.scb = v * v;
    check(dev::gemm_strided(s, g), "vvvo");
  };
  if (!mixed) {
    double* V1 = c.alloc(v3 * o, "(T) vvvo [b,c,d,k]");
    double* V2 = c.alloc(v3 * o, "(T) vvvo [c,b,d,k]");
    for (int64_t kk = 0; kk < o; ++kk) {
      build_v(kk, V1 + v3 * kk);
      check(dev::permute(s, 3, d3, swap01, 1.0, V1 + v3 * kk, 0.0, V2 + v3 * kk), "vvvo perm");
    }
    ops.V1 = V1;
    ops.V2 = V2;
  } else {
    const size_t evs = dev::tc_operand_elems(v2, v, kTriplesSlices);
    const size_t eos = dev::tc_operand_elems(v, o, kTriplesSlices);
    uint16_t* bv = alloc_bf16(c, 2 * evs * o, "(T) vvvo BF16");
    uint16_t* bo = alloc_bf16(c, eos * o * o, "(T) ovoo BF16");
    const size_t mark = c.allocs.size();
    double* Vt = c.alloc(v3, "(T) vvvo slab");
    double* Vt2 = c.alloc(v3, "(T) vvvo slab");
    ops.V1s.resize(o);
    ops.V2s.resize(o);
    ops.Ons.resize(o * o);
    for (int64_t kk = 0; kk < o; ++kk) {
      build_v(kk, Vt);
      check(dev::tc_split(s, Vt, v2, v, 1, v2, kTriplesSlices, bv + evs * kk, &ops.V1s[kk]),
            "split vvvo");
      check(dev::permute(s, 3, d3, swap01, 1.0, Vt, 0.0, Vt2), "vvvo perm");
      check(dev::tc_split(s, Vt2, v2, v, 1, v2, kTriplesSlices, bv + evs * (o + kk),
                          &ops.V2s[kk]),
            "split vvvo");
    }
    // -ovoo: the ovoo segments share the vvvo GEMMs' alpha = 1 (the BF16
    // split of -x is the negated split of x)
    check(dev::axpby(s, o * o * o * v, -1.0, On, 0.0, On), "-ovoo");
    for (int64_t z = 0; z < o; ++z)
      for (int64_t y = 0; y < o; ++y)
        check(dev::tc_split(s, On + o * y + o * o * v * z, v, o, o * o, 1, kTriplesSlices,
                            bo + eos * (y + o * z), &ops.Ons[y + o * z]),
              "split ovoo");
    check(dev::sync(s), "sync");
    c.release_to(mark);
  }

  double* U2c = nullptr;
  if (lam) {
    double* U2 = c.alloc(c.n2(), "(T) U2");
    U2c = c.alloc(c.n2(), "(T) U2 covariant");
    check(dev::h2d(U2, U2h, c.n2() * 8, s), "h2d U2");
    // contra2covariant (cctools.jl:935-938): (2 U2[a,b,i,j] + U2[b,a,i,j]) / 3
    check(dev::axpby(s, c.n2(), 2.0 / 3.0, U2, 0.0, U2c), "U2c");
    con.permute(1.0 / 3.0, U2, "baij", 1.0, U2c, "abij");
  }
  SplitAmps ST, SU;
  if (mixed) {
    split_amps(c, c.T2(), ST);
    if (lam) split_amps(c, U2c, SU);
  }

  // the sweep: triplet order and weights of cc_triples.jl:62-72
  const double* eps = c.fock_host.data();
  std::vector<Trip> tr;
  for (int k = 0; k < o; ++k)
    for (int j = 0; j <= k; ++j)
      for (int i = 0; i <= j; ++i) {
        if (i == j && j == k) continue;
        const double f = (i == j) ? 1.0 : (j == k ? 1.0 : 2.0);
        tr.push_back({i, j, k, f, eps[i + i * n] + eps[j + j * n] + eps[k + k * n]});
      }
  const int64_t nt = (int64_t)tr.size();
  if (nt == 0) {
    *et = *etb = 0.0;
    return;
  }
  // batches of NB triplets, one K slot each, within a 4 GiB budget
  const int64_t esz = mixed ? 4 : 8;
  const int64_t vp = mixed ? (v + 3) / 4 * 4 : v;  // K's a pitch (see perm_table)
  const int64_t kstride = (vp * v2 + 31) / 32 * 32;
  const int64_t per = kstride * esz * (lam ? 2 : 1);
  int64_t nbmax = std::min<int64_t>({256, nt, ((int64_t)4 << 30) / per});
  if (c.triples_batch > 0) nbmax = std::min(nbmax, c.triples_batch);
  const int NB = (int)std::max<int64_t>(1, nbmax);
  void* K = c.alloc((NB * kstride * esz + 7) / 8, "(T) K slots");
  void* KU = lam ? (void*)c.alloc((NB * kstride * esz + 7) / 8, "(T) K(Lambda) slots") : nullptr;
  KTables KT, KUt;
  fill_tables(c, ops, &ST, tr, NB, kstride, vp, KT);
  upload_tables(c, KT);
  if (lam) {
    fill_tables(c, ops, &SU, tr, NB, kstride, vp, KUt);
    upload_tables(c, KUt);
  }

  // energy terms per triplet: g = T1 (or U1/2), f[a,i] = fock[i, o+a], <ij|ab>, T2 (or U2c)
  std::vector<double> gh(v * o), fh(v * o);
  {
    std::vector<double> T1h(v * o);
    if (!lam) {
      check(dev::d2h(T1h.data(), c.T1(), v * o * 8, s), "d2h");
      check(dev::sync(s), "sync");
    }
    for (int64_t i = 0; i < o; ++i)
      for (int64_t a = 0; a < v; ++a) {
        gh[a + v * i] = lam ? 0.5 * U1h[a + v * i] : T1h[a + v * i];
        fh[a + v * i] = c.fock_host[i + (o + a) * n];
      }
  }
  double* gf = c.alloc(2 * v * o, "(T) singles/Fock vectors");
  check(dev::h2d(gf, gh.data(), v * o * 8, s), "h2d");
  check(dev::h2d(gf + v * o, fh.data(), v * o * 8, s), "h2d");
  const double* Nsrc = lam ? U2c : c.T2();
  std::vector<double> eijk(nt);
  for (int64_t t = 0; t < nt; ++t) eijk[t] = tr[t].eijk;
  double* eijk_d = c.alloc(nt, "(T) denominators");
  check(dev::h2d(eijk_d, eijk.data(), nt * 8, s), "h2d");
  // energy terms per triplet.  FP64: g, f, M = <ij|ab>, N = T2 (or U2c) as
  // separate arrays.  Mixed precision: FP32 copies interleaved in pairs,
  // (g, f)[a] per occupied index and (M, N)[a + v b] per occupied pair, which
  // the FP32 energy kernel stages with one 8-byte copy per position (they
  // enter only the singles/Fock term sum X Y).
  dev::TriplesTerms* terms_d = nullptr;
  dev::TriplesTermsF* termsf_d = nullptr;
  float* MNp = nullptr;
  float* MNt = nullptr;
  if (mixed) {
    float* GF = reinterpret_cast<float*>(c.alloc(v * o, "(T) FP32 (g, f)"));  // float2 [occ][a]
    const int64_t mne = dev::triples_mn_elems((int)v, o * o);
    MNp = reinterpret_cast<float*>(c.alloc(mne, "(T) FP32 (M, N)"));
    MNt = reinterpret_cast<float*>(c.alloc(mne, "(T) FP32 (M, N) transposed"));
    check(dev::to_f32_pairs(s, v * o, gf, gf + v * o, GF), "FP32 (g, f)");
    check(dev::triples_mn_pack(s, (int)v, o * o, c.Kvvoo, Nsrc, MNp, MNt),
          "FP32 (<ij|ab>, amplitudes)");
    auto gfp = [&](int x) { return static_cast<const void*>(GF + 2 * v * x); };
    std::vector<dev::TriplesTermsF> terms(nt);
    for (int64_t t = 0; t < nt; ++t) {
      const int i = tr[t].i, j = tr[t].j, k = tr[t].k;
      dev::TriplesTermsF& tt = terms[t];
      tt.gf[0] = gfp(i); tt.gf[1] = gfp(j); tt.gf[2] = gfp(k);
      tt.mnpair[0] = (int32_t)(j + o * k);
      tt.mnpair[1] = (int32_t)(i + o * k);
      tt.mnpair[2] = (int32_t)(i + o * j);
    }
    termsf_d = reinterpret_cast<dev::TriplesTermsF*>(
        c.alloc((int64_t)((nt * sizeof(dev::TriplesTermsF) + 7) / 8), "(T) energy terms"));
    check(dev::h2d(termsf_d, terms.data(), nt * sizeof(dev::TriplesTermsF), s), "h2d");
  } else {
    auto at = [&](const double* p, int64_t off) { return static_cast<const void*>(p + off); };
    auto M = [&](int x, int y) { return at(c.Kvvoo, v2 * (x + o * y)); };
    auto N = [&](int x, int y) { return at(Nsrc, v2 * (x + o * y)); };
    std::vector<dev::TriplesTerms> terms(nt);
    for (int64_t t = 0; t < nt; ++t) {
      const int i = tr[t].i, j = tr[t].j, k = tr[t].k;
      dev::TriplesTerms& tt = terms[t];
      tt.g[0] = at(gf, v * i); tt.g[1] = at(gf, v * j); tt.g[2] = at(gf, v * k);
      tt.f[0] = at(gf, v * (o + i)); tt.f[1] = at(gf, v * (o + j)); tt.f[2] = at(gf, v * (o + k));
      tt.M[0] = M(j, k); tt.M[1] = M(i, k); tt.M[2] = M(i, j);
      tt.N[0] = N(j, k); tt.N[1] = N(i, k); tt.N[2] = N(i, j);
    }
    terms_d = reinterpret_cast<dev::TriplesTerms*>(
        c.alloc((int64_t)((nt * sizeof(dev::TriplesTerms) + 7) / 8), "(T) energy terms"));
    check(dev::h2d(terms_d, terms.data(), nt * sizeof(dev::TriplesTerms), s), "h2d");
  }
  const int64_t ncube = dev::triples_cube_count((int)v);
  std::vector<int> trih(3 * ncube);
  dev::triples_cube_table((int)v, trih.data());
  int* tri = reinterpret_cast<int*>(c.alloc((3 * ncube + 1) / 2, "(T) cube table"));
  check(dev::h2d(tri, trih.data(), 3 * ncube * sizeof(int), s), "h2d");
  double* part = c.alloc(dev::triples_energy_scratch_len((int)v, NB), "(T) partial sums");
  double* Et = c.alloc(2 * nt, "(T) energies");

  // batch loop: the first batch runs directly (first-use set-up of the
  // kernels), the others are recorded as one CUDA graph and run once
  const int64_t nbatch = (nt + NB - 1) / NB;
  try {
    for (int64_t bi = 0; bi < nbatch; ++bi) {
      if (bi == 1) check(dev::graph_capture_begin(s), "graph capture");
      const int64_t t0 = bi * NB;
      const int nb = (int)std::min<int64_t>(NB, nt - t0);
      build_K_batch(c, ops, c.T2(), &ST, KT, nt, t0, nb, K, kstride, vp);
      if (lam) build_K_batch(c, ops, U2c, &SU, KUt, nt, t0, nb, KU, kstride, vp);
      if (mixed)
        check(dev::triples_energy_f32_batched(s, (int)v, (int)vp, nb, NB,
                                              static_cast<const float*>(K),
                                              static_cast<const float*>(KU), kstride, MNp, MNt,
                                              o * o, eijk_d + t0, c.eps + o, termsf_d + t0, tri,
                                              part, Et + 2 * t0),
              "triples energy");
      else
        check(dev::triples_energy_batched(s, (int)v, nb, K, KU, kstride, false, eijk_d + t0,
                                          c.eps + o, terms_d + t0, tri, part, Et + 2 * t0),
              "triples energy");
    }
    if (nbatch > 1) {
      int64_t nodes = 0;
      check(dev::graph_capture_run(s, &nodes), "(T) graph");
    }
  } catch (...) {
    dev::graph_capture_abort(s);
    throw;
  }
  std::vector<double> Eh(2 * nt);
  check(dev::d2h(Eh.data(), Et, 2 * nt * 8, s), "d2h");
  check(dev::sync(s), "sync");
  int tc = 0;
  check(dev::tc_error(&tc), "tc_error");
  if (tc) throw Error(ECG_ERR_TIMEOUT, "GEMM wait timed out in (T) (code " + std::to_string(tc) + ")");
  // sum K X, and the singles / Fock term sum X Y (cc_triples.jl:143-156 / :286-294)
  double Enb3 = 0.0, Esf = 0.0;
  for (int64_t q = 0; q < nt; ++q) {
    Enb3 += tr[q].f * Eh[2 * q];
    Esf += tr[q].f * Eh[2 * q + 1];
  }
  const double En3 = Enb3 + Esf;
  if (!std::isfinite(En3)) throw Error(ECG_ERR_NONFINITE, "non-finite (T) energy");
  *et = En3;
  *etb = Enb3;
}

}  // namespace ecg
