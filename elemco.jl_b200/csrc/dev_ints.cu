// dev_ints.cu — Gaussian integrals over contracted Cartesian shells on the GPU
// (McMurchie-Davidson): overlap, kinetic energy, nuclear attraction, dipole
// (one-electron), and two-/three-centre Coulomb integrals (P|Q), (mn|P) for
// density fitting.  Replaces ElemCo.jl's libcint calls (src/system/libcint5.jl,
// integrals_2idx.jl, integrals_2e3idx.jl).
//
// A Cartesian function of shell s is (x-X)^i (y-Y)^j (z-Z)^k exp(-a r_s^2)
// with i+j+k = l, components ordered i = l..0, then j = l-i..0 (xx, xy, xz,
// yy, yz, zz for d).  A shell's contracted function is sum_k c_k g(a_k); the
// caller folds any normalisation into c_k and transforms to spherical
// functions afterwards.
//
// Hermite expansion (1D, exponents a on A, b on B, p = a + b, P the product
// centre): E^{i+1,j}_t = E^{ij}_{t-1}/(2p) + X_PA E^{ij}_t + (t+1) E^{ij}_{t+1},
// likewise for j with X_PB; E^{00}_0 = 1 (the Gaussian-product prefactor
// exp(-ab/p |AB|^2) is applied once per primitive pair).  Coulomb integrals
// over Hermite functions R_{tuv}(alpha, R_PQ) follow from the Boys function by
// R^n_{000} = (-2 alpha)^n F_n(alpha R^2) and the recursions
// R^n_{t+1,u,v} = t R^{n+1}_{t-1,u,v} + X R^{n+1}_{t,u,v} (u, v alike).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "ecg_dev.h"

namespace ecg {
namespace dev {

namespace {

constexpr int LMAX = INT_LMAX;             // largest shell angular momentum
constexpr int LPAIR = 2 * LMAX;            // largest l_a + l_b
constexpr int LTOT = INT_LTOT;             // largest total of a Coulomb integral
constexpr int ETSZ = (LMAX + 1) * (LMAX + 1) * (LPAIR + 1);  // one 1D E table
constexpr int LKIN = LMAX + 2;             // kinetic energy needs j up to l_b + 2
constexpr int ETSZ_K = (LMAX + 1) * (LKIN + 1) * (LMAX + LKIN + 1);

__host__ __device__ constexpr int tet(int s) { return (s + 1) * (s + 2) * (s + 3) / 6; }
__device__ __forceinline__ int hidx(int t, int u, int v) {
  const int s = t + u + v, w = u + v;
  return s * (s + 1) * (s + 2) / 6 + w * (w + 1) / 2 + v;
}
__device__ __forceinline__ int ncart(int l) { return (l + 1) * (l + 2) / 2; }
// exponents (i, j, k) of Cartesian component c of degree l
__device__ __forceinline__ void cart_ijk(int l, int c, int& i, int& j, int& k) {
  int n = 0;
  for (i = l; i >= 0; --i)
    for (j = l - i; j >= 0; --j, ++n)
      if (n == c) {
        k = l - i - j;
        return;
      }
  i = j = k = 0;
}

// Boys function F_n(T), n = 0..m: for T < 40 the series
// F_m(T) = e^{-T} sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)) and downward
// recursion F_{n-1} = (2T F_n + e^{-T}) / (2n - 1); for larger T
// F_0 = sqrt(pi/T) erf(sqrt T) / 2 and upward recursion
// F_{n+1} = ((2n+1) F_n - e^{-T}) / (2T) (stable there).
__device__ void boys(int m, double T, double* F) {
  const double et = exp(-T);
  if (T < 40.0) {
    double term = 1.0 / (2 * m + 1), sum = term;
    for (int k = 1; k < 400; ++k) {
      term *= 2.0 * T / (2 * m + 2 * k + 1);
      sum += term;
      if (term < 1e-17 * sum) break;
    }
    F[m] = et * sum;
    for (int n = m; n > 0; --n) F[n - 1] = (2.0 * T * F[n] + et) / (2 * n - 1);
  } else {
    const double st = sqrt(T);
    F[0] = 0.5 * sqrt(M_PI / T) * erf(st);
    for (int n = 0; n < m; ++n) F[n + 1] = ((2 * n + 1) * F[n] - et) / (2.0 * T);
  }
}

// 1D Hermite coefficients E[(i*(lb+1)+j)*(la+lb+1)+t], i <= la, j <= lb.
__device__ void etab(int la, int lb, double p, double xpa, double xpb, double* E) {
  const int nt = la + lb + 1;
  const double h = 0.5 / p;
  for (int x = 0; x < (la + 1) * (lb + 1) * nt; ++x) E[x] = 0.0;
  auto at = [&](int i, int j, int t) -> double& { return E[(i * (lb + 1) + j) * nt + t]; };
  at(0, 0, 0) = 1.0;
  for (int i = 0; i <= la; ++i) {
    if (i > 0)
      for (int t = 0; t <= i; ++t) {
        double v = xpa * at(i - 1, 0, t);
        if (t > 0) v += h * at(i - 1, 0, t - 1);
        if (t + 1 <= i - 1) v += (t + 1) * at(i - 1, 0, t + 1);
        at(i, 0, t) = v;
      }
    for (int j = 1; j <= lb; ++j)
      for (int t = 0; t <= i + j; ++t) {
        double v = xpb * at(i, j - 1, t);
        if (t > 0) v += h * at(i, j - 1, t - 1);
        if (t + 1 <= i + j - 1) v += (t + 1) * at(i, j - 1, t + 1);
        at(i, j, t) = v;
      }
  }
}

// Hermite Coulomb integrals R[hidx(t,u,v)], t+u+v <= L, scaled so that
// R^0_{tuv} is returned; work holds 2 tet(L) doubles.
__device__ void hermite_r(int L, double alpha, double X, double Y, double Z, double* R,
                          double* work) {
  double F[LTOT + 1];
  boys(L, alpha * (X * X + Y * Y + Z * Z), F);
  double* cur = work;               // level n
  double* nxt = work + tet(LTOT);   // level n + 1
  double m2a = 1.0;
  for (int n = 0; n < L; ++n) m2a *= -2.0 * alpha;
  for (int n = L; n >= 0; --n) {
    // cur = level n from nxt = level n + 1 (totals <= L - n)
    for (int s = 0; s <= L - n; ++s)
      for (int w = 0; w <= s; ++w)
        for (int v = 0; v <= w; ++v) {
          const int u = w - v, t = s - w;
          double r;
          if (s == 0) {
            r = m2a * F[n];
          } else if (t > 0) {
            r = X * nxt[hidx(t - 1, u, v)];
            if (t > 1) r += (t - 1) * nxt[hidx(t - 2, u, v)];
          } else if (u > 0) {
            r = Y * nxt[hidx(t, u - 1, v)];
            if (u > 1) r += (u - 1) * nxt[hidx(t, u - 2, v)];
          } else {
            r = Z * nxt[hidx(t, u, v - 1)];
            if (v > 1) r += (v - 1) * nxt[hidx(t, u, v - 2)];
          }
          cur[hidx(t, u, v)] = r;
        }
    double* tmp = cur;
    cur = nxt;
    nxt = tmp;
    if (alpha != 0.0) m2a /= -2.0 * alpha;
  }
  // the last level written (n = 0) is in nxt after the swap
  for (int x = 0; x < tet(L); ++x) R[x] = nxt[x];
}

struct Sh {
  double x, y, z;
  int l, np, poff, boff;
};
__device__ __forceinline__ Sh load_shell(const IntShell* s, int i) {
  const IntShell& q = s[i];
  return Sh{q.x, q.y, q.z, q.l, q.nprim, q.poff, q.boff};
}

// Coulomb block between the charge distributions of shell pair (a, b) and
// shell pair (c, d), where b and/or d may be absent (nullptr: an s function
// of exponent 0 on the partner's centre).  Accumulates
// out[(ia + na*ib) * sab + (ic + nc*id) * scd] += (ab|cd) over the contracted
// primitives, with component indices local to the shells.
__device__ void coulomb_block(const Sh& a, const Sh* b, const Sh& c, const Sh* d,
                              const double* ex, const double* co, double* out, int64_t oa,
                              int64_t ob, int64_t oc, int64_t od) {
  const int la = a.l, lb = b ? b->l : 0, lc = c.l, ld = d ? d->l : 0;
  const int nab = la + lb, ncd = lc + ld, L = nab + ncd;
  double Eab[3][ETSZ], Ecd[3][ETSZ];
  double R[tet(LTOT)], work[2 * tet(LTOT)], W[tet(LPAIR)];
  const int npb = b ? b->np : 1, npd = d ? d->np : 1;
  const int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
  const double two_pi52 = 2.0 * pow(M_PI, 2.5);
  for (int pa = 0; pa < a.np; ++pa)
    for (int pb = 0; pb < npb; ++pb) {
      const double ea = ex[a.poff + pa], eb = b ? ex[b->poff + pb] : 0.0;
      const double cab = co[a.poff + pa] * (b ? co[b->poff + pb] : 1.0);
      const double p = ea + eb;
      const double Bx = b ? b->x : a.x, By = b ? b->y : a.y, Bz = b ? b->z : a.z;
      const double Px = (ea * a.x + eb * Bx) / p, Py = (ea * a.y + eb * By) / p,
                   Pz = (ea * a.z + eb * Bz) / p;
      const double ab2 = (a.x - Bx) * (a.x - Bx) + (a.y - By) * (a.y - By) +
                         (a.z - Bz) * (a.z - Bz);
      const double Kab = exp(-ea * eb / p * ab2) * cab;
      if (Kab == 0.0) continue;
      etab(la, lb, p, Px - a.x, Px - Bx, Eab[0]);
      etab(la, lb, p, Py - a.y, Py - By, Eab[1]);
      etab(la, lb, p, Pz - a.z, Pz - Bz, Eab[2]);
      for (int pc = 0; pc < c.np; ++pc)
        for (int pd = 0; pd < npd; ++pd) {
          const double ec = ex[c.poff + pc], ed = d ? ex[d->poff + pd] : 0.0;
          const double ccd = co[c.poff + pc] * (d ? co[d->poff + pd] : 1.0);
          const double q = ec + ed;
          const double Dx = d ? d->x : c.x, Dy = d ? d->y : c.y, Dz = d ? d->z : c.z;
          const double Qx = (ec * c.x + ed * Dx) / q, Qy = (ec * c.y + ed * Dy) / q,
                       Qz = (ec * c.z + ed * Dz) / q;
          const double cd2 = (c.x - Dx) * (c.x - Dx) + (c.y - Dy) * (c.y - Dy) +
                             (c.z - Dz) * (c.z - Dz);
          const double Kcd = exp(-ec * ed / q * cd2) * ccd;
          if (Kcd == 0.0) continue;
          etab(lc, ld, q, Qx - c.x, Qx - Dx, Ecd[0]);
          etab(lc, ld, q, Qy - c.y, Qy - Dy, Ecd[1]);
          etab(lc, ld, q, Qz - c.z, Qz - Dz, Ecd[2]);
          const double alpha = p * q / (p + q);
          hermite_r(L, alpha, Px - Qx, Py - Qy, Pz - Qz, R, work);
          const double pref = two_pi52 / (p * q * sqrt(p + q)) * Kab * Kcd;
          const int ntc = ncd + 1, nta = nab + 1;
          for (int ic = 0; ic < nc; ++ic)
            for (int id = 0; id < nd; ++id) {
              int ci, cj, ck, di, dj, dk;
              cart_ijk(lc, ic, ci, cj, ck);
              cart_ijk(ld, id, di, dj, dk);
              const double* ecx = Ecd[0] + (ci * (ld + 1) + di) * ntc;
              const double* ecy = Ecd[1] + (cj * (ld + 1) + dj) * ntc;
              const double* ecz = Ecd[2] + (ck * (ld + 1) + dk) * ntc;
              // W[tuv] = sum_{tau nu phi} (-1)^{tau+nu+phi} E^{cd} R_{t+tau,u+nu,v+phi}
              for (int s = 0; s <= nab; ++s)
                for (int w = 0; w <= s; ++w)
                  for (int v = 0; v <= w; ++v) {
                    const int u = w - v, t = s - w;
                    double acc = 0.0;
                    for (int tau = 0; tau <= ci + di; ++tau)
                      for (int nu = 0; nu <= cj + dj; ++nu)
                        for (int phi = 0; phi <= ck + dk; ++phi) {
                          const double e = ecx[tau] * ecy[nu] * ecz[phi];
                          if (e == 0.0) continue;
                          const double r = R[hidx(t + tau, u + nu, v + phi)];
                          acc += ((tau + nu + phi) & 1) ? -e * r : e * r;
                        }
                    W[hidx(t, u, v)] = acc;
                  }
              for (int ia = 0; ia < na; ++ia)
                for (int ib = 0; ib < nb; ++ib) {
                  int ai, aj, ak, bi, bj, bk;
                  cart_ijk(la, ia, ai, aj, ak);
                  cart_ijk(lb, ib, bi, bj, bk);
                  const double* eax = Eab[0] + (ai * (lb + 1) + bi) * nta;
                  const double* eay = Eab[1] + (aj * (lb + 1) + bj) * nta;
                  const double* eaz = Eab[2] + (ak * (lb + 1) + bk) * nta;
                  double acc = 0.0;
                  for (int t = 0; t <= ai + bi; ++t)
                    for (int u = 0; u <= aj + bj; ++u)
                      for (int v = 0; v <= ak + bk; ++v)
                        acc += eax[t] * eay[u] * eaz[v] * W[hidx(t, u, v)];
                  out[ia * oa + ib * ob + ic * oc + id * od] += pref * acc;
                }
            }
        }
    }
}

// (mn|P): item -> (shell a, shell b <= a, aux shell P); Cartesian output
// out[m + nm*(n + nm*P)] (both orders of m, n written).
__global__ void int3c_kernel(const IntShell* __restrict__ ao, int nao_sh,
                             const IntShell* __restrict__ aux, int naux_sh,
                             const double* __restrict__ ex, const double* __restrict__ co,
                             int64_t nm, double* out) {
  const int64_t npair = (int64_t)nao_sh * (nao_sh + 1) / 2;
  const int64_t items = npair * naux_sh;
  for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < items;
       it += (int64_t)gridDim.x * blockDim.x) {
    const int P = (int)(it % naux_sh);
    int64_t pr = it / naux_sh;
    int ia = (int)((sqrt(8.0 * (double)pr + 1.0) - 1.0) / 2.0);
    while ((int64_t)ia * (ia + 1) / 2 > pr) --ia;
    while ((int64_t)(ia + 1) * (ia + 2) / 2 <= pr) ++ia;
    const int ib = (int)(pr - (int64_t)ia * (ia + 1) / 2);
    const Sh a = load_shell(ao, ia), b = load_shell(ao, ib), c = load_shell(aux, P);
    double* o = out + a.boff + nm * (b.boff + nm * (int64_t)c.boff);
    coulomb_block(a, &b, c, nullptr, ex, co, o, 1, nm, nm * nm, 0);
    if (ia != ib) {
      // mirror: out[n, m, P] = out[m, n, P]
      const int na = ncart(a.l), nb = ncart(b.l), nc = ncart(c.l);
      double* o2 = out + b.boff + nm * (a.boff + nm * (int64_t)c.boff);
      for (int k = 0; k < nc; ++k)
        for (int j = 0; j < nb; ++j)
          for (int i = 0; i < na; ++i)
            o2[j + nm * (i + nm * (int64_t)k)] = o[i + nm * (j + nm * (int64_t)k)];
    }
  }
}

// (P|Q): item -> (P, Q <= P); out[P + np*Q] (both orders written).
__global__ void int2c_kernel(const IntShell* __restrict__ aux, int naux_sh,
                             const double* __restrict__ ex, const double* __restrict__ co,
                             int64_t np_, double* out) {
  const int64_t items = (int64_t)naux_sh * (naux_sh + 1) / 2;
  for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < items;
       it += (int64_t)gridDim.x * blockDim.x) {
    int ip = (int)((sqrt(8.0 * (double)it + 1.0) - 1.0) / 2.0);
    while ((int64_t)ip * (ip + 1) / 2 > it) --ip;
    while ((int64_t)(ip + 1) * (ip + 2) / 2 <= it) ++ip;
    const int iq = (int)(it - (int64_t)ip * (ip + 1) / 2);
    const Sh a = load_shell(aux, ip), c = load_shell(aux, iq);
    double* o = out + a.boff + np_ * (int64_t)c.boff;
    coulomb_block(a, nullptr, c, nullptr, ex, co, o, 1, 0, np_, 0);
    if (ip != iq) {
      const int na = ncart(a.l), nc = ncart(c.l);
      double* o2 = out + c.boff + np_ * (int64_t)a.boff;
      for (int j = 0; j < nc; ++j)
        for (int i = 0; i < na; ++i) o2[j + np_ * i] = o[i + np_ * j];
    }
  }
}

// One-electron integrals of shell pair (a, b <= a): kind 0 overlap, 1 kinetic,
// 2 nuclear attraction (-sum_C Z_C / |r - C|), 3 dipole (x, y, z components
// about `origin` at out, out + n^2, out + 2 n^2).  out[m + n*nn], both orders.
__global__ void int1e_kernel(int kind, const IntShell* __restrict__ sh, int nsh,
                             const double* __restrict__ ex, const double* __restrict__ co,
                             int natom, const double* __restrict__ Z,
                             const double* __restrict__ xyz, double ox, double oy, double oz,
                             int64_t nn, double* out) {
  const int64_t items = (int64_t)nsh * (nsh + 1) / 2;
  for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < items;
       it += (int64_t)gridDim.x * blockDim.x) {
    int ia = (int)((sqrt(8.0 * (double)it + 1.0) - 1.0) / 2.0);
    while ((int64_t)ia * (ia + 1) / 2 > it) --ia;
    while ((int64_t)(ia + 1) * (ia + 2) / 2 <= it) ++ia;
    const int ib = (int)(it - (int64_t)ia * (ia + 1) / 2);
    const Sh a = load_shell(sh, ia), b = load_shell(sh, ib);
    const int la = a.l, lb = b.l, na = ncart(la), nb = ncart(lb);
    const int ncomp = kind == 3 ? 3 : 1;
    for (int pa = 0; pa < a.np; ++pa)
      for (int pb = 0; pb < b.np; ++pb) {
        const double ea = ex[a.poff + pa], eb = ex[b.poff + pb];
        const double p = ea + eb;
        const double Px = (ea * a.x + eb * b.x) / p, Py = (ea * a.y + eb * b.y) / p,
                     Pz = (ea * a.z + eb * b.z) / p;
        const double ab2 = (a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y) +
                           (a.z - b.z) * (a.z - b.z);
        const double K = exp(-ea * eb / p * ab2) * co[a.poff + pa] * co[b.poff + pb];
        if (K == 0.0) continue;
        const int lbk = kind == 1 ? lb + 2 : lb;
        double E[3][ETSZ_K];
        etab(la, lbk, p, Px - a.x, Px - b.x, E[0]);
        etab(la, lbk, p, Py - a.y, Py - b.y, E[1]);
        etab(la, lbk, p, Pz - a.z, Pz - b.z, E[2]);
        const int nt = la + lbk + 1;
        auto Ex = [&](int d, int i, int j, int t) { return E[d][(i * (lbk + 1) + j) * nt + t]; };
        const double sp = sqrt(M_PI / p);
        double R[tet(LPAIR)], work[2 * tet(LTOT)];
        const double P3[3] = {Px, Py, Pz}, O3[3] = {ox, oy, oz};
        for (int ia_ = 0; ia_ < na; ++ia_)
          for (int ib_ = 0; ib_ < nb; ++ib_) {
            int ai[3], bi[3];
            cart_ijk(la, ia_, ai[0], ai[1], ai[2]);
            cart_ijk(lb, ib_, bi[0], bi[1], bi[2]);
            double val[3] = {0.0, 0.0, 0.0};
            if (kind == 0 || kind == 1 || kind == 3) {
              double S[3], T[3], D[3];
              for (int d = 0; d < 3; ++d) {
                const int i = ai[d], j = bi[d];
                S[d] = Ex(d, i, j, 0) * sp;
                if (kind == 1) {
                  double t = -2.0 * eb * eb * Ex(d, i, j + 2, 0) + eb * (2 * j + 1) * Ex(d, i, j, 0);
                  if (j >= 2) t -= 0.5 * j * (j - 1) * Ex(d, i, j - 2, 0);
                  T[d] = t * sp;
                }
                if (kind == 3) {
                  double m1 = Ex(d, i, j, 0) * (P3[d] - O3[d]);
                  if (i + j >= 1) m1 += Ex(d, i, j, 1);
                  D[d] = m1 * sp;
                }
              }
              if (kind == 0) val[0] = S[0] * S[1] * S[2];
              if (kind == 1)
                val[0] = T[0] * S[1] * S[2] + S[0] * T[1] * S[2] + S[0] * S[1] * T[2];
              if (kind == 3) {
                val[0] = D[0] * S[1] * S[2];
                val[1] = S[0] * D[1] * S[2];
                val[2] = S[0] * S[1] * D[2];
              }
            } else {
              const int L = la + lb;
              for (int C = 0; C < natom; ++C) {
                hermite_r(L, p, Px - xyz[3 * C], Py - xyz[3 * C + 1], Pz - xyz[3 * C + 2], R,
                          work);
                double acc = 0.0;
                for (int t = 0; t <= ai[0] + bi[0]; ++t)
                  for (int u = 0; u <= ai[1] + bi[1]; ++u)
                    for (int v = 0; v <= ai[2] + bi[2]; ++v)
                      acc += Ex(0, ai[0], bi[0], t) * Ex(1, ai[1], bi[1], u) *
                             Ex(2, ai[2], bi[2], v) * R[hidx(t, u, v)];
                val[0] -= Z[C] * 2.0 * M_PI / p * acc;
              }
            }
            for (int q = 0; q < ncomp; ++q) {
              double* o = out + q * nn * nn;
              o[(a.boff + ia_) + nn * (b.boff + ib_)] += K * val[q];
              if (ia != ib) o[(b.boff + ib_) + nn * (a.boff + ia_)] += K * val[q];
            }
          }
      }
  }
}

unsigned grid_of(int64_t items, int threads) {
  int64_t g = (items + threads - 1) / threads;
  if (g > 148 * 64) g = 148 * 64;
  return (unsigned)(g < 1 ? 1 : g);
}

}  // namespace

int int1e_cart(stream_t s, int kind, const IntShell* sh, int nsh, const double* ex,
               const double* co, int natom, const double* Z, const double* xyz,
               const double* origin, int64_t nn, double* out) {
  if (kind < 0 || kind > 3) return (int)cudaErrorInvalidValue;
  const int64_t items = (int64_t)nsh * (nsh + 1) / 2;
  const double ox = origin ? origin[0] : 0.0, oy = origin ? origin[1] : 0.0,
               oz = origin ? origin[2] : 0.0;
  int1e_kernel<<<grid_of(items, 64), 64, 0, (cudaStream_t)s>>>(kind, sh, nsh, ex, co, natom, Z,
                                                               xyz, ox, oy, oz, nn, out);
  note_launches(1);
  return (int)cudaGetLastError();
}

int int2c2e_cart(stream_t s, const IntShell* aux, int nsh, const double* ex, const double* co,
                 int64_t np_, double* out) {
  const int64_t items = (int64_t)nsh * (nsh + 1) / 2;
  int2c_kernel<<<grid_of(items, 64), 64, 0, (cudaStream_t)s>>>(aux, nsh, ex, co, np_, out);
  note_launches(1);
  return (int)cudaGetLastError();
}

int int3c2e_cart(stream_t s, const IntShell* ao, int nao_sh, const IntShell* aux, int naux_sh,
                 const double* ex, const double* co, int64_t nm, double* out) {
  const int64_t items = (int64_t)nao_sh * (nao_sh + 1) / 2 * naux_sh;
  int3c_kernel<<<grid_of(items, 64), 64, 0, (cudaStream_t)s>>>(ao, nao_sh, aux, naux_sh, ex, co,
                                                               nm, out);
  note_launches(1);
  return (int)cudaGetLastError();
}

}  // namespace dev
}  // namespace ecg
