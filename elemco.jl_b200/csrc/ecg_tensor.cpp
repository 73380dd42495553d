// ecg_tensor.cpp — workspace arena and TTGT tensor contraction (see header).
#include "ecg_tensor.h"

#include <cstring>

#include "../../include/ecgpu.h"

namespace ecg {

void check(int code, const char* what) {
  if (code != 0) throw Error(ECG_ERR_CUDA, std::string(what) + ": " + dev::error_string(code));
}

// Mixed precision sends a contraction to the split-BF16 tensor cores when it
// is large (2^26 multiply-adds or more) and long: K > 1024.  The short ones,
// the density-fitting contractions over the auxiliary index (K = nQ <= 1024)
// and the like, stay FP64.  Measured on (H2O)6/cc-pVTZ CCSD, where the
// mixed-product iteration converges to a point off the FP64 one: with every
// large contraction mixed that point is 10.9 uEh off and its FP64 residual
// 4.4e-10 (three FP64 refinement iterations); keeping the short contractions
// FP64 leaves 0.5 uEh and 3.4e-11 (their products alone moved it by about
// +10 uEh, the long ones by +4, the ladder by -4), the solve takes one FP64
// iteration less (3.6 -> 3.0 s) for 7% more time per mixed iteration.
int gemm_prec(bool mixed, dev::stream_t s, char ta, char tb, int64_t m, int64_t n, int64_t k,
              double alpha, const double* A, int64_t lda, const double* B, int64_t ldb,
              double beta, double* C, int64_t ldc) {
  if (mixed && k > 1024 && (double)m * (double)n * (double)k >= 67108864.0)
    return dev::gemm_mixed(s, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  return dev::gemm(s, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

double* Arena::get(int64_t n) {
  int64_t need = (n + 31) & ~int64_t(31);  // 256-byte granularity
  if (top_ + need > cap_)
    throw Error(ECG_ERR_OOM, "workspace arena exhausted (" + std::to_string((top_ + need) * 8) +
                                 " of " + std::to_string(cap_ * 8) + " bytes)");
  double* p = base_ + top_;
  top_ += need;
  if (top_ > peak_) peak_ = top_;
  return p;
}

int64_t Extents::operator()(char c) const {
  if (c >= 'a' && c <= 'h') return nv;
  if (c >= 'i' && c <= 'o') return no;
  if (c >= 'p' && c <= 'u') return n;
  if (c == 'Q' || c == 'P' || c == 'L') return nq;
  throw Error(ECG_ERR_ARG, std::string("unknown index character '") + c + "'");
}

int64_t Contractor::size(const char* idx) const {
  int64_t s = 1;
  for (const char* c = idx; *c; ++c) s *= (*ext_)(*c);
  return s;
}

// Permutation mapping tensor with index string `from` to index string `to`.
static void perm_of(const std::string& from, const std::string& to, int* perm) {
  for (size_t d = 0; d < to.size(); ++d) {
    size_t p = from.find(to[d]);
    if (p == std::string::npos) throw Error(ECG_ERR_ARG, "index mismatch " + from + " -> " + to);
    perm[d] = (int)p;
  }
}

void Contractor::permute(double alpha, const double* in, const char* ii, double beta,
                         double* out, const char* io) {
  std::string si(ii), so(io);
  if (si.size() != so.size()) throw Error(ECG_ERR_ARG, "permute rank mismatch " + si + "/" + so);
  int64_t dims[8];
  int perm[8];
  for (size_t d = 0; d < si.size(); ++d) dims[d] = (*ext_)(si[d]);
  perm_of(si, so, perm);
  if (si == so) {
    check(dev::axpby(s_, size(ii), alpha, in, beta, out), "axpby");
    return;
  }
  check(dev::permute(s_, (int)si.size(), dims, perm, alpha, in, beta, out), "permute");
}

static std::string subseq(const std::string& s, const std::string& keep) {
  std::string r;
  for (char c : s)
    if (keep.find(c) != std::string::npos) r += c;
  return r;
}

void Contractor::operator()(double alpha, const double* A, const char* ia_, const double* B,
                            const char* ib_, double beta, double* C, const char* ic_) {
  const std::string ia(ia_), ib(ib_), ic(ic_);
  std::string M, N, K;
  for (char c : ia) {
    bool inB = ib.find(c) != std::string::npos, inC = ic.find(c) != std::string::npos;
    if (inB && inC) throw Error(ECG_ERR_ARG, "batch index in contraction " + ia + "," + ib);
    if (inB) K += c;
    else if (inC) M += c;
    else throw Error(ECG_ERR_ARG, "index summed in one operand only: " + ia);
  }
  for (char c : ib) {
    bool inA = ia.find(c) != std::string::npos, inC = ic.find(c) != std::string::npos;
    if (!inA && inC) N += c;
    else if (!inA && !inC) throw Error(ECG_ERR_ARG, "index summed in one operand only: " + ib);
  }
  if (M.size() + N.size() != ic.size())
    throw Error(ECG_ERR_ARG, "output indices mismatch " + ic);

  const int64_t sA = size(ia_), sB = size(ib_), sC = size(ic_);
  std::string Mo[2] = {subseq(ic, M), subseq(ia, M)};
  std::string No[2] = {subseq(ic, N), subseq(ib, N)};
  std::string Ko[2] = {subseq(ia, K), subseq(ib, K)};
  int64_t best = -1;
  std::string bM, bN, bK;
  bool bCT = false;
  for (auto& mo : Mo)
    for (auto& no : No)
      for (auto& ko : Ko)
        for (int ct = 0; ct < 2; ++ct) {
          bool aok = (ia == mo + ko) || (ia == ko + mo);
          bool bok = (ib == ko + no) || (ib == no + ko);
          bool cok = ct ? (ic == no + mo) : (ic == mo + no);
          int64_t cost = (aok ? 0 : sA) + (bok ? 0 : sB) + (cok ? 0 : 3 * sC);
          if (best < 0 || cost < best) {
            best = cost;
            bM = mo;
            bN = no;
            bK = ko;
            bCT = ct;
          }
        }
  const int64_t mM = size(bM.c_str()), mN = size(bN.c_str()), mK = size(bK.c_str());
  const int64_t mark = ws_->mark();
  // A as (M,K): 'N' if stored M+K, 'T' if stored K+M
  const double* Ap = A;
  char ta;
  if (ia == bM + bK) ta = 'N';
  else if (ia == bK + bM) ta = 'T';
  else {
    double* t = ws_->get(sA);
    permute(1.0, A, ia_, 0.0, t, (bM + bK).c_str());
    Ap = t;
    ta = 'N';
  }
  const double* Bp = B;
  char tb;
  if (ib == bK + bN) tb = 'N';
  else if (ib == bN + bK) tb = 'T';
  else {
    double* t = ws_->get(sB);
    permute(1.0, B, ib_, 0.0, t, (bK + bN).c_str());
    Bp = t;
    tb = 'N';
  }
  const int64_t lda = (ta == 'N') ? mM : mK;
  const int64_t ldb = (tb == 'N') ? mK : mN;
  const std::string cform = bCT ? bN + bM : bM + bN;
  double* Cp = C;
  double cbeta = beta;
  bool cperm = (ic != cform);
  if (cperm) {
    Cp = ws_->get(sC);
    cbeta = 0.0;
  }
  if (!bCT) {
    check(gemm_prec(mixed_, s_, ta, tb, mM, mN, mK, alpha, Ap, lda, Bp, ldb, cbeta, Cp, mM),
          "gemm");
  } else {
    // C^T(N,M) = opB^T (N,K) * opA^T (K,M)
    char tb2 = (tb == 'N') ? 'T' : 'N';
    char ta2 = (ta == 'N') ? 'T' : 'N';
    check(gemm_prec(mixed_, s_, tb2, ta2, mN, mM, mK, alpha, Bp, ldb, Ap, lda, cbeta, Cp, mN),
          "gemm");
  }
  if (cperm) permute(1.0, Cp, cform.c_str(), beta, C, ic_);
  ws_->release(mark);
}

}  // namespace ecg
