// hf_host.cpp -- host-side inputs of the flow: Coulomb TBMEs of the 2-D
// harmonic-oscillator quantum dot and the Hartree-Fock normal-ordered
// Hamiltonian in the (M_L,M_S)-blocked layout.  The reference keeps these on
// the host too; they are not the hot path, only its input.
//
//   v_int      Anisimovas & Matulis closed form, src/ME_general.f90:2205-2276,
//              with the reference's mixed real(16)/real(8) arithmetic
//              (__float128 for the real(16) factorial products; every real(8)
//              assignment rounds).  The innermost sum depends only on the four
//              integers gs(1..4) and is memoised per thread (exact).
//              The two alternating sums accumulate terms of up to ~1e21 in
//              real(8); from radial quantum numbers n ~ 7 on (emax >= 15) the
//              cancellation leaves no correct digit (e.g. <(9,1)(9,-1)|V|
//              (9,-1)(9,1)> = 0.2843 exactly, 1.3e5 in that arithmetic).  The
//              QD_TBME_QUAD option keeps every sum and factor in __float128
//              (relative error ~1e-13 up to emax = 20; a test checks it
//              against exact rational arithmetic).
//   ME.bin     the stream file read at src/HFQDmod.f90:97-127: records of
//              int32 n1,m1,n2,m2,n3,m3,n4,m4 and float64 Vdir (hbar-omega = 1).
//   HF         src/HFQDmod.f90:186-254: density of the lowest N states, mean
//              field, block diagonalisation in (m_l, m_s), |delta e| < 1e-6
//              over the first N eigenvalues; then the Fock matrix, the HF-basis
//              two-body blocks (new_VMAT/HF_Vmatrix, ME_general.f90:1362-1492,
//              :2179-2202) and E0 = HF_E2 (HFQDmod.f90:292-323).
//   Streamlined: the HO->HF two-body transform uses D = CC - CB, since
//   CC V CC^T + CB V CB^T - CC V CB^T - CB V CC^T = D V D^T, and D is sparse
//   (coefficients only couple equal (m_l, m_s)); dsyev is replaced by a
//   Jacobi eigensolver on the small single-particle blocks.
#include <quadmath.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "qd_internal.hpp"

namespace qd {
namespace {

typedef __float128 q128;

// ---- real(16) special functions (ME_general.f90:2314-2384) -----------------
q128 fac_over_fac(int a1, int a2) {
  q128 s1 = 1;
  if (a1 > a2) {
    for (int i = a2 + 1; i <= a1; ++i) s1 = s1 * i;
    return s1;
  }
  for (int i = a1 + 1; i <= a2; ++i) s1 = s1 * i;
  return 1 / s1;
}
q128 qfac(int n) {
  q128 s1 = 1;
  for (int i = 1; i <= n; ++i) s1 = s1 * i;
  return s1;
}
q128 bin_coef(int n, int k) { return fac_over_fac(n, k) / qfac(n - k); }

// gamma (ME_general.f90:2314-2336), for whole and half-integer x; real(8) result
double gamma_hi(double x) {
  const double sqpi = 1.77245385090551602;
  int x_c = (int)std::floor(x);
  if (std::fabs((double)(float)x_c - x) < 1e-3) return (double)qfac(x_c - 1);
  x_c = (int)std::floor(x - 0.5);
  double p4 = std::pow(4.0, x_c);
  return (double)(fac_over_fac(2 * x_c, x_c) / p4 * sqpi);
}

struct VintCache {
  std::vector<double> memo;  // sm_int by (gs1,gs2,gs3,gs4), NaN = not yet computed
  std::vector<q128> memoq;   // the same in __float128 (QD_TBME_QUAD), NaN = not yet computed
  std::vector<q128> gamq;    // gamma(k/2) in __float128
  std::vector<q128> halfq;   // 0.5**((G+1)/2) in __float128
  int gsd = 0;               // gs values < gsd
  std::vector<q128> binc;    // bin_coef(n,k) at n*(bmax+1)+k
  std::vector<q128> fact;    // fac(n) = ((1*1)*2)*...*n, as fac() computes it
  std::vector<double> gam;   // gamma(k/2), k >= 1
  std::vector<double> half;  // 0.5d0**((G+1)*0.5), by G
  int bmax = 0;
  void build(int nb, int ng) {
    bmax = nb;
    binc.assign((size_t)(nb + 1) * (nb + 1), 0);
    for (int n = 0; n <= nb; ++n)
      for (int k = 0; k <= n; ++k) binc[(size_t)n * (nb + 1) + k] = bin_coef(n, k);
    fact.assign(nb + 1, 0);
    for (int n = 0; n <= nb; ++n) fact[n] = qfac(n);
    gam.assign(ng + 1, 0.0);
    for (int k = 1; k <= ng; ++k) gam[k] = gamma_hi(0.5 * k);
    half.assign(ng + 1, 0.0);
    for (int G = 0; G <= ng; ++G) half[G] = std::pow(0.5, ((double)G + 1.0) * 0.5);
    gsd = nb / 2;
    memo.assign((size_t)gsd * gsd * gsd * gsd, std::nan(""));
  }
  void build_quad(int nb, int ng) {
    build(nb, ng);
    memo.clear();
    memoq.assign((size_t)gsd * gsd * gsd * gsd, nanq(""));
    gamq.assign(ng + 1, 0);
    for (int k = 1; k <= ng; ++k) {
      if (k % 2 == 0) {
        gamq[k] = qfac(k / 2 - 1);  // gamma(j) = (j-1)!
      } else {
        const int j = (k - 1) / 2;  // gamma(j + 1/2) = (2j)! / (4^j j!) sqrt(pi)
        gamq[k] = fac_over_fac(2 * j, j) / powq(4, j) * sqrtq(acosq((q128)-1));
      }
    }
    halfq.assign(ng + 1, 0);
    for (int G = 0; G <= ng; ++G) halfq[G] = powq((q128)0.5, ((q128)G + 1) / 2);
  }
  q128 bc(int n, int k) const { return binc[(size_t)n * (bmax + 1) + k]; }
  double g2(double x) const { return gam[(int)std::lround(2 * x)]; }  // gamma(x), x half-integer
};

// v_int(qi,qj,qk,ql,hw) with q = (n, ml, ms)
double v_int(const int* qi, const int* qj, const int* qk, const int* ql, double hw, VintCache& C) {
  double vout = 0.0, sm = 0.0;
  if (!(qi[2] == ql[2] && qk[2] == qj[2])) return 0.0;
  for (int j1 = 0; j1 <= qi[0]; ++j1)
    for (int j2 = 0; j2 <= qj[0]; ++j2)
      for (int j3 = 0; j3 <= qk[0]; ++j3)
        for (int j4 = 0; j4 <= ql[0]; ++j4) {
          int gs[4];
          gs[0] = j1 + j4 + (std::abs(qi[1]) + qi[1]) / 2 + (std::abs(ql[1]) - ql[1]) / 2;
          gs[3] = j1 + j4 + (std::abs(qi[1]) - qi[1]) / 2 + (std::abs(ql[1]) + ql[1]) / 2;
          gs[1] = j2 + j3 + (std::abs(qj[1]) + qj[1]) / 2 + (std::abs(qk[1]) - qk[1]) / 2;
          gs[2] = j2 + j3 + (std::abs(qj[1]) - qj[1]) / 2 + (std::abs(qk[1]) + qk[1]) / 2;
          const double G = (double)(gs[0] + gs[1] + gs[2] + gs[3]);
          double& slot = C.memo[(((size_t)gs[0] * C.gsd + gs[1]) * C.gsd + gs[2]) * C.gsd + gs[3]];
          double sm_int;
          if (!std::isnan(slot)) {
            sm_int = slot;
          } else {
            sm_int = 0.0;
            for (int l1 = 0; l1 <= gs[0]; ++l1)
              for (int l2 = 0; l2 <= gs[1]; ++l2)
                for (int l3 = 0; l3 <= gs[2]; ++l3) {
                  const int l4 = l1 + l2 - l3;  // kron_del(l1+l2, l3+l4): other l4 add exact zeros
                  if (l4 < 0 || l4 > gs[3]) continue;
                  const double LAM = (double)(l1 + l2 + l3 + l4);
                  const int sgn = ((gs[1] + gs[2] - l2 - l3) & 1) ? -1 : 1;
                  q128 t = (q128)sgn * C.bc(gs[0], l1);
                  t = t * C.bc(gs[1], l2);
                  t = t * C.bc(gs[2], l3);
                  t = t * C.bc(gs[3], l4);
                  t = t * (q128)C.g2(1.0 + LAM * 0.5);
                  t = t * (q128)C.g2((G - LAM + 1.0) * 0.5);
                  sm_int = (double)((q128)sm_int + t);
                }
            slot = sm_int;
          }
          const int s4 = ((j1 + j2 + j3 + j4) & 1) ? -1 : 1;
          q128 den = C.fact[j1];
          den = den * C.fact[j2];
          den = den * C.fact[j3];
          den = den * C.fact[j4];
          q128 t = (q128)s4 / den;
          t = t * C.bc(qi[0] + std::abs(qi[1]), qi[0] - j1);
          t = t * C.bc(qj[0] + std::abs(qj[1]), qj[0] - j2);
          t = t * C.bc(qk[0] + std::abs(qk[1]), qk[0] - j3);
          t = t * C.bc(ql[0] + std::abs(ql[1]), ql[0] - j4);
          t = t * (q128)C.half[(int)G];
          t = t * (q128)sm_int;
          sm = (double)((q128)sm + t);
        }
  q128 f = fac_over_fac(qi[0], qi[0] + std::abs(qi[1]));
  f = f * fac_over_fac(qj[0], qj[0] + std::abs(qj[1]));
  f = f * fac_over_fac(qk[0], qk[0] + std::abs(qk[1]));
  f = f * fac_over_fac(ql[0], ql[0] + std::abs(ql[1]));
  const double a = std::sqrt(hw) * sm;
  vout = (double)((q128)a * sqrtq(f));
  return vout;
}

// v_int with every sum and factor in __float128 (QD_TBME_QUAD); the loop
// structure is that of v_int above.
double v_int_quad(const int* qi, const int* qj, const int* qk, const int* ql, double hw, VintCache& C) {
  if (!(qi[2] == ql[2] && qk[2] == qj[2])) return 0.0;
  q128 sm = 0;
  for (int j1 = 0; j1 <= qi[0]; ++j1)
    for (int j2 = 0; j2 <= qj[0]; ++j2)
      for (int j3 = 0; j3 <= qk[0]; ++j3)
        for (int j4 = 0; j4 <= ql[0]; ++j4) {
          int gs[4];
          gs[0] = j1 + j4 + (std::abs(qi[1]) + qi[1]) / 2 + (std::abs(ql[1]) - ql[1]) / 2;
          gs[3] = j1 + j4 + (std::abs(qi[1]) - qi[1]) / 2 + (std::abs(ql[1]) + ql[1]) / 2;
          gs[1] = j2 + j3 + (std::abs(qj[1]) + qj[1]) / 2 + (std::abs(qk[1]) - qk[1]) / 2;
          gs[2] = j2 + j3 + (std::abs(qj[1]) - qj[1]) / 2 + (std::abs(qk[1]) + qk[1]) / 2;
          const int G = gs[0] + gs[1] + gs[2] + gs[3];
          q128& slot = C.memoq[(((size_t)gs[0] * C.gsd + gs[1]) * C.gsd + gs[2]) * C.gsd + gs[3]];
          if (isnanq(slot)) {
            q128 acc = 0;
            for (int l1 = 0; l1 <= gs[0]; ++l1)
              for (int l2 = 0; l2 <= gs[1]; ++l2)
                for (int l3 = 0; l3 <= gs[2]; ++l3) {
                  const int l4 = l1 + l2 - l3;
                  if (l4 < 0 || l4 > gs[3]) continue;
                  const int LAM = l1 + l2 + l3 + l4;
                  const int sgn = ((gs[1] + gs[2] - l2 - l3) & 1) ? -1 : 1;
                  q128 t = (q128)sgn * C.bc(gs[0], l1) * C.bc(gs[1], l2) * C.bc(gs[2], l3) * C.bc(gs[3], l4);
                  acc += t * C.gamq[2 + LAM] * C.gamq[G - LAM + 1];  // gamma(1+LAM/2) gamma((G-LAM+1)/2)
                }
            slot = acc;
          }
          const int s4 = ((j1 + j2 + j3 + j4) & 1) ? -1 : 1;
          q128 t = (q128)s4 / (C.fact[j1] * C.fact[j2] * C.fact[j3] * C.fact[j4]);
          t = t * C.bc(qi[0] + std::abs(qi[1]), qi[0] - j1) * C.bc(qj[0] + std::abs(qj[1]), qj[0] - j2);
          t = t * C.bc(qk[0] + std::abs(qk[1]), qk[0] - j3) * C.bc(ql[0] + std::abs(ql[1]), ql[0] - j4);
          sm += t * C.halfq[G] * slot;
        }
  q128 f = fac_over_fac(qi[0], qi[0] + std::abs(qi[1]));
  f = f * fac_over_fac(qj[0], qj[0] + std::abs(qj[1]));
  f = f * fac_over_fac(qk[0], qk[0] + std::abs(qk[1]));
  f = f * fac_over_fac(ql[0], ql[0] + std::abs(ql[1]));
  return (double)(sqrtq((q128)hw) * sm * sqrtq(f));
}

// spatial orbitals in nm_index order (ME_general.f90:2140-2149)
struct Spatial {
  int emax, N;
  std::vector<int> n, ml;  // per orbital
  explicit Spatial(int e) : emax(e) {
    for (int R = 0; R < e; ++R)
      for (int m = -R; m <= R; m += 2) {
        n.push_back((R - std::abs(m)) / 2);
        ml.push_back(m);
      }
    N = (int)n.size();
  }
  int index(int nn, int m) const {
    int R = std::abs(m) + 2 * nn;
    return R * (R + 1) / 2 + (R + m) / 2;
  }
};

}  // namespace

// Direct spatial TBMEs D(a,b,c,d) = <ab|V|cd> at hbar-omega = 1 for all
// m-conserving quadruples, grouped by M = ml_a + ml_b; pairs (a,b) of a block
// in loop order a (outer), b (inner).
struct TBME {
  int emax = 0, N = 0;
  std::vector<int> pair_block, pair_idx;  // by a*N + b
  std::vector<std::vector<std::pair<int, int>>> pairs;  // per block
  std::vector<std::vector<double>> D;                    // per block, row-major n_M x n_M
};

static int build_tbme(int emax, TBME& T, int nthreads, unsigned options) {
  const bool quad = (options & QD_TBME_QUAD) != 0;
  Spatial S(emax);
  const int N = S.N;
  T.emax = emax;
  T.N = N;
  const int MMAX = 2 * (emax - 1);
  T.pairs.assign(2 * MMAX + 1, {});
  T.pair_block.assign((size_t)N * N, -1);
  T.pair_idx.assign((size_t)N * N, -1);
  for (int a = 0; a < N; ++a)
    for (int b = 0; b < N; ++b) {
      int M = S.ml[a] + S.ml[b] + MMAX;
      T.pair_block[(size_t)a * N + b] = M;
      T.pair_idx[(size_t)a * N + b] = (int)T.pairs[M].size();
      T.pairs[M].push_back({a, b});
    }
  T.D.assign(T.pairs.size(), {});
  for (size_t M = 0; M < T.pairs.size(); ++M) T.D[M].assign(T.pairs[M].size() * T.pairs[M].size(), 0.0);
  // list of canonical quadruples; symmetric partners are filled from them:
  //   <ab|cd> = <ba|dc> = <cd|ab> = <dc|ba>
  struct Q {
    int M, p, r;
  };
  std::vector<Q> work;
  for (size_t M = 0; M < T.pairs.size(); ++M) {
    const auto& P = T.pairs[M];
    for (int p = 0; p < (int)P.size(); ++p)
      for (int r = 0; r < (int)P.size(); ++r) {
        const int a = P[p].first, b = P[p].second, c = P[r].first, d = P[r].second;
        // one representative per orbit of 8: {(p,r), (r,p), (ba,dc), (dc,ba)}
        // and the same with every m_l negated (time reversal), the smallest
        // (block, p, r) triple; every entry is then written exactly once
        const int pba = T.pair_idx[(size_t)b * N + a], pdc = T.pair_idx[(size_t)d * N + c];
        const int ta = S.index(S.n[a], -S.ml[a]), tb = S.index(S.n[b], -S.ml[b]);
        const int tc = S.index(S.n[c], -S.ml[c]), td = S.index(S.n[d], -S.ml[d]);
        const int Mt = T.pair_block[(size_t)ta * N + tb];
        const int tab = T.pair_idx[(size_t)ta * N + tb], tcd = T.pair_idx[(size_t)tc * N + td];
        const int tba = T.pair_idx[(size_t)tb * N + ta], tdc = T.pair_idx[(size_t)td * N + tc];
        typedef std::tuple<int, int, int> K;
        const K me((int)M, p, r);
        const K orbit[7] = {K((int)M, r, p), K((int)M, pba, pdc), K((int)M, pdc, pba), K(Mt, tab, tcd),
                            K(Mt, tcd, tab), K(Mt, tba, tdc), K(Mt, tdc, tba)};
        bool canon = true;
        for (const K& k : orbit) canon = canon && !(k < me);
        if (!canon) continue;
        work.push_back({(int)M, p, r});
      }
  }
  int maxn = 0;
  for (int i = 0; i < N; ++i) maxn = std::max(maxn, S.n[i] + std::abs(S.ml[i]));
  // bin_coef arguments stay below ~3*emax, gs values below ~2*emax
  const int nb = 4 * emax + 16, ng = 8 * emax + 32;
#pragma omp parallel num_threads(nthreads)
  {
    VintCache C;
    if (quad)
      C.build_quad(nb, ng);
    else
      C.build(nb, ng);
#pragma omp for schedule(dynamic, 64)
    for (long long w = 0; w < (long long)work.size(); ++w) {
      const Q& q = work[w];
      const auto& P = T.pairs[q.M];
      const int a = P[q.p].first, b = P[q.p].second, c = P[q.r].first, d = P[q.r].second;
      int qa[3] = {S.n[a], S.ml[a], -1}, qb[3] = {S.n[b], S.ml[b], -1};
      int qc[3] = {S.n[c], S.ml[c], -1}, qd_[3] = {S.n[d], S.ml[d], -1};
      // <ab|V|cd>_direct = v_int(a,b,d,c) (get_ints, ME_general.f90:776-779)
      const double v = quad ? v_int_quad(qa, qb, qd_, qc, 1.0, C) : v_int(qa, qb, qd_, qc, 1.0, C);
      const int pba = T.pair_idx[(size_t)b * N + a], pdc = T.pair_idx[(size_t)d * N + c];
      const size_t n = P.size();
      double* D = T.D[q.M].data();
      D[(size_t)q.p * n + q.r] = v;
      D[(size_t)q.r * n + q.p] = v;
      D[(size_t)pba * n + pdc] = v;
      D[(size_t)pdc * n + pba] = v;
      // time-reversed partners (all m_l negated), block -M
      const int ta = S.index(S.n[a], -S.ml[a]), tb = S.index(S.n[b], -S.ml[b]);
      const int tc = S.index(S.n[c], -S.ml[c]), td = S.index(S.n[d], -S.ml[d]);
      const int Mt = T.pair_block[(size_t)ta * N + tb];
      const size_t nt = T.pairs[Mt].size();
      double* Dt = T.D[Mt].data();
      const int tab = T.pair_idx[(size_t)ta * N + tb], tcd = T.pair_idx[(size_t)tc * N + td];
      const int tba = T.pair_idx[(size_t)tb * N + ta], tdc = T.pair_idx[(size_t)td * N + tc];
      Dt[(size_t)tab * nt + tcd] = v;
      Dt[(size_t)tcd * nt + tab] = v;
      Dt[(size_t)tba * nt + tdc] = v;
      Dt[(size_t)tdc * nt + tba] = v;
    }
  }
  (void)maxn;
  return QD_OK;
}

// ---- ME.bin ------------------------------------------------------------------
static int write_mebin(const TBME& T, const char* path) {
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    set_error("qd_tbme_write: cannot open %s", path);
    return QD_ERR_ARG;
  }
  Spatial S(T.emax);
  for (size_t M = 0; M < T.pairs.size(); ++M) {
    const auto& P = T.pairs[M];
    const size_t n = P.size();
    for (size_t p = 0; p < n; ++p)
      for (size_t r = 0; r < n; ++r) {
        int32_t rec[8] = {S.n[P[p].first], S.ml[P[p].first], S.n[P[p].second], S.ml[P[p].second],
                          S.n[P[r].first], S.ml[P[r].first], S.n[P[r].second], S.ml[P[r].second]};
        double v = T.D[M][p * n + r];
        std::fwrite(rec, sizeof(rec), 1, f);
        std::fwrite(&v, sizeof(v), 1, f);
      }
  }
  std::fclose(f);
  return QD_OK;
}

// Read ME.bin for emax (records beyond emax are skipped, as HFQDmod.f90:113-116)
static int read_mebin(const char* path, int emax, TBME& T) {
  Spatial S(emax);
  const int N = S.N, MMAX = 2 * (emax - 1);
  T.emax = emax;
  T.N = N;
  T.pairs.assign(2 * MMAX + 1, {});
  T.pair_block.assign((size_t)N * N, -1);
  T.pair_idx.assign((size_t)N * N, -1);
  for (int a = 0; a < N; ++a)
    for (int b = 0; b < N; ++b) {
      int M = S.ml[a] + S.ml[b] + MMAX;
      T.pair_block[(size_t)a * N + b] = M;
      T.pair_idx[(size_t)a * N + b] = (int)T.pairs[M].size();
      T.pairs[M].push_back({a, b});
    }
  T.D.assign(T.pairs.size(), {});
  for (size_t M = 0; M < T.pairs.size(); ++M) T.D[M].assign(T.pairs[M].size() * T.pairs[M].size(), 0.0);
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("ME.bin: cannot open %s", path);
    return QD_ERR_ARG;
  }
  int32_t rec[8];
  double v;
  while (std::fread(rec, sizeof(rec), 1, f) == 1) {
    if (std::fread(&v, sizeof(v), 1, f) != 1) {
      std::fclose(f);
      set_error("ME.bin: truncated record (failfile)");
      return QD_ERR_ARG;
    }
    bool skip = false;
    for (int k = 0; k < 4; ++k)
      if (2 * rec[2 * k] + std::abs(rec[2 * k + 1]) > emax - 1) skip = true;
    if (skip) continue;
    const int a = S.index(rec[0], rec[1]), b = S.index(rec[2], rec[3]);
    const int c = S.index(rec[4], rec[5]), d = S.index(rec[6], rec[7]);
    const int M = T.pair_block[(size_t)a * N + b];
    if (M != T.pair_block[(size_t)c * N + d]) continue;  // not m-conserving: zero
    const size_t n = T.pairs[M].size();
    T.D[M][(size_t)T.pair_idx[(size_t)a * N + b] * n + T.pair_idx[(size_t)c * N + d]] = v;
    T.D[M][(size_t)T.pair_idx[(size_t)c * N + d] * n + T.pair_idx[(size_t)a * N + b]] = v;
  }
  std::fclose(f);
  return QD_OK;
}

// ---- Hartree-Fock -----------------------------------------------------------------
// Jacobi eigen-decomposition of a symmetric k x k matrix (row-major a), in
// place; eigenvalues ascending in w, eigenvectors in the columns of V, each
// with its largest-magnitude component positive.
static void jacobi(int k, std::vector<double>& a, std::vector<double>& w, std::vector<double>& V) {
  V.assign((size_t)k * k, 0.0);
  for (int i = 0; i < k; ++i) V[(size_t)i * k + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < k; ++p)
      for (int q = p + 1; q < k; ++q) off += a[(size_t)p * k + q] * a[(size_t)p * k + q];
    if (off < 1e-30) break;
    for (int p = 0; p < k; ++p)
      for (int q = p + 1; q < k; ++q) {
        double apq = a[(size_t)p * k + q];
        if (std::fabs(apq) < 1e-300) continue;
        double app = a[(size_t)p * k + p], aqq = a[(size_t)q * k + q];
        double th = (aqq - app) / (2 * apq);
        double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1));
        double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int r = 0; r < k; ++r) {
          double arp = a[(size_t)r * k + p], arq = a[(size_t)r * k + q];
          a[(size_t)r * k + p] = c * arp - s * arq;
          a[(size_t)r * k + q] = s * arp + c * arq;
        }
        for (int r = 0; r < k; ++r) {
          double apr = a[(size_t)p * k + r], aqr = a[(size_t)q * k + r];
          a[(size_t)p * k + r] = c * apr - s * aqr;
          a[(size_t)q * k + r] = s * apr + c * aqr;
        }
        for (int r = 0; r < k; ++r) {
          double vrp = V[(size_t)r * k + p], vrq = V[(size_t)r * k + q];
          V[(size_t)r * k + p] = c * vrp - s * vrq;
          V[(size_t)r * k + q] = s * vrp + c * vrq;
        }
      }
  }
  std::vector<int> ord(k);
  for (int i = 0; i < k; ++i) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](int x, int y) { return a[(size_t)x * k + x] < a[(size_t)y * k + y]; });
  std::vector<double> V2((size_t)k * k);
  w.assign(k, 0.0);
  for (int j = 0; j < k; ++j) {
    int c = ord[j];
    w[j] = a[(size_t)c * k + c];
    int big = 0;
    for (int r = 0; r < k; ++r)
      if (std::fabs(V[(size_t)r * k + c]) > std::fabs(V[(size_t)big * k + c]) + 1e-14) big = r;
    double sg = V[(size_t)big * k + c] < 0 ? -1.0 : 1.0;
    for (int r = 0; r < k; ++r) V2[(size_t)r * k + j] = sg * V[(size_t)r * k + c];
  }
  V = V2;
}

struct HFResult {
  std::vector<double> coefs;  // m x m, column j = HF state j in the HO basis (states order)
  std::vector<double> eig;    // m, states order
  std::vector<double> F;      // m x m Fock matrix in the HF basis
  int iterations = 0;
};

// HF iteration (HFQDmod.f90:186-237) on spin-orbitals in states order.
// mix: fraction of the new density taken each iteration (1 = the reference's
// plain Roothaan iteration; below 1 damps the oscillation that large dots at
// small hbar-omega show).
static int run_hf(int nbody, int emax, double hw, const TBME& T, HFResult& R, int nthreads, double mix) {
  const int m = emax * (emax + 1);
  Spatial S(emax);
  std::vector<int> sn(m), sml(m), sms(m);
  {
    int j = 0;
    for (int Rr = 0; Rr < emax; ++Rr)
      for (int ml = -Rr; ml <= Rr; ml += 2)
        for (int ms = -1; ms <= 1; ms += 2) {
          sn[j] = (Rr - std::abs(ml)) / 2;
          sml[j] = ml;
          sms[j] = ms;
          ++j;
        }
  }
  std::vector<int> sp(m);  // spatial orbital of each state
  for (int s = 0; s < m; ++s) sp[s] = S.index(sn[s], sml[s]);
  const double sqhw = std::sqrt(hw);
  auto Dv = [&](int a, int b, int c, int d) -> double {  // direct spatial <ab|V|cd> * sqrt(hw)
    int M = T.pair_block[(size_t)a * T.N + b];
    if (M != T.pair_block[(size_t)c * T.N + d]) return 0.0;
    size_t n = T.pairs[M].size();
    return T.D[M][(size_t)T.pair_idx[(size_t)a * T.N + b] * n + T.pair_idx[(size_t)c * T.N + d]] * sqhw;
  };
  // (ml,ms) blocks of the single-particle basis
  std::vector<std::vector<int>> blocks;
  {
    std::vector<std::pair<int, int>> keys;
    for (int s = 0; s < m; ++s) {
      std::pair<int, int> k(sml[s], sms[s]);
      auto it = std::find(keys.begin(), keys.end(), k);
      if (it == keys.end()) {
        keys.push_back(k);
        blocks.push_back({s});
      } else {
        blocks[it - keys.begin()].push_back(s);
      }
    }
  }
  std::vector<double> C((size_t)m * m, 0.0), eig(m, 0.0), eold(m, 0.0), den((size_t)m * m), Fm((size_t)m * m);
  std::vector<double> den_old;
  for (int i = 0; i < m; ++i) C[(size_t)i * m + i] = 1.0;  // column-major: C[row + col*m]
  double crit = 1.0;
  int it = 0;
  while (crit > 1e-6) {
    if (++it > 2000) {
      set_error("Hartree-Fock did not converge");
      return QD_ERR_NOCONV;
    }
    // den = C[:,1:n] C[:,1:n]^T
    std::fill(den.begin(), den.end(), 0.0);
    for (int k = 0; k < nbody; ++k)
      for (int j = 0; j < m; ++j)
        for (int i = 0; i < m; ++i) den[(size_t)i + (size_t)j * m] += C[(size_t)i + (size_t)k * m] * C[(size_t)j + (size_t)k * m];
    if (mix < 1.0 && !den_old.empty())
      for (size_t e = 0; e < den.size(); ++e) den[e] = mix * den[e] + (1.0 - mix) * den_old[e];
    den_old = den;
    // V(i,k) = sum_{j,l} den(l,j) <j i|V|l k>_AS  (construct_V, HFQDmod.f90:260-290)
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
    for (int k = 0; k < m; ++k)
      for (int i = 0; i < m; ++i) {
        double v = 0.0;
        if (sml[i] == sml[k] && sms[i] == sms[k]) {
          for (const auto& blk : blocks)
            for (int j : blk)
              for (int l : blk) {
                const double dlj = den[(size_t)l + (size_t)j * m];
                if (dlj == 0.0) continue;
                double dir = (sms[j] == sms[l] && sms[i] == sms[k]) ? Dv(sp[j], sp[i], sp[l], sp[k]) : 0.0;
                double exc = (sms[j] == sms[k] && sms[i] == sms[l]) ? Dv(sp[j], sp[i], sp[k], sp[l]) : 0.0;
                v += dlj * (dir - exc);
              }
        }
        Fm[(size_t)i + (size_t)k * m] = v + (i == k ? (2 * sn[i] + std::abs(sml[i]) + 1) * hw : 0.0);
      }
    eold = eig;
    // block diagonalisation; eigvecs_to_normal (ME_general.f90:540-574)
    std::fill(C.begin(), C.end(), 0.0);
    for (const auto& blk : blocks) {
      const int k = (int)blk.size();
      std::vector<double> a((size_t)k * k), w, V;
      for (int r = 0; r < k; ++r)
        for (int c = 0; c < k; ++c) a[(size_t)r * k + c] = Fm[(size_t)blk[r] + (size_t)blk[c] * m];
      jacobi(k, a, w, V);
      for (int r = 0; r < k; ++r) {
        for (int c = 0; c < k; ++c) C[(size_t)blk[r] + (size_t)blk[c] * m] = V[(size_t)r * k + c];
        eig[blk[r]] = w[r];
      }
    }
    crit = 0.0;
    for (int i = 0; i < nbody; ++i) crit += std::fabs(eold[i] - eig[i]);
  }
  // F_HF = C^T F C
  std::vector<double> tmp((size_t)m * m, 0.0);
  R.F.assign((size_t)m * m, 0.0);
#pragma omp parallel for num_threads(nthreads)
  for (int j = 0; j < m; ++j)
    for (int k = 0; k < m; ++k) {
      const double c = C[(size_t)k + (size_t)j * m];
      if (c == 0.0) continue;
      for (int i = 0; i < m; ++i) tmp[(size_t)i + (size_t)j * m] += Fm[(size_t)i + (size_t)k * m] * c;
    }
#pragma omp parallel for num_threads(nthreads)
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) {
      double s = 0.0;
      for (int k = 0; k < m; ++k) s += C[(size_t)k + (size_t)i * m] * tmp[(size_t)k + (size_t)j * m];
      R.F[(size_t)i + (size_t)j * m] = s;
    }
  R.coefs = C;
  R.eig = eig;
  R.iterations = it;
  return QD_OK;
}

// The HF-basis Hamiltonian in vectorize order: E0 (HF_E2), f (convertF),
// two-body blocks D V D^T (new_VMAT / HF_Vmatrix).
static int build_hamiltonian(int nbody, int emax, double hw, const TBME& T, const HFResult& R, qd_layout* L,
                             std::vector<double>& vec, int nthreads) {
  const int m = L->m, n = L->n, mp = L->mp;
  Spatial S(emax);
  std::vector<int> sp(m), sms(m);
  for (int s = 0; s < m; ++s) {
    sp[s] = S.index(L->qn[3 * s], L->qn[3 * s + 1]);
    sms[s] = L->qn[3 * s + 2];
  }
  const double sqhw = std::sqrt(hw);
  auto Dv = [&](int a, int b, int c, int d) -> double {
    int M = T.pair_block[(size_t)a * T.N + b];
    if (M != T.pair_block[(size_t)c * T.N + d]) return 0.0;
    size_t nn = T.pairs[M].size();
    return T.D[M][(size_t)T.pair_idx[(size_t)a * T.N + b] * nn + T.pair_idx[(size_t)c * T.N + d]] * sqhw;
  };
  // antisymmetrised HO-basis element <p1 p2|V|p3 p4> (p1<p2, p3<p4 states)
  auto vas = [&](int p1, int p2, int p3, int p4) -> double {
    double dir = (sms[p1] == sms[p3] && sms[p2] == sms[p4]) ? Dv(sp[p1], sp[p2], sp[p3], sp[p4]) : 0.0;
    double exc = (sms[p1] == sms[p4] && sms[p2] == sms[p3]) ? Dv(sp[p1], sp[p2], sp[p4], sp[p3]) : 0.0;
    return dir - exc;
  };
  vec.assign(L->neq, 0.0);
  const std::vector<double>& C = R.coefs;  // C[row + col*m]
  // one-body (convertF, ME_general.f90:1495-1555)
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) vec[L->o_fhh + i + (i64)j * n] = R.F[(size_t)i + (size_t)j * m];
  for (int j = 0; j < mp; ++j)
    for (int i = 0; i < mp; ++i) vec[L->o_fpp + i + (i64)j * mp] = R.F[(size_t)(n + i) + (size_t)(n + j) * m];
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < mp; ++i) vec[L->o_fph + i + (i64)j * mp] = R.F[(size_t)(n + i) + (size_t)j * m];
  // two-body, block by block: HFV = D V D^T with D(i,j) = C(b_j,a_i) C(d_j,c_i) - C(d_j,a_i) C(b_j,c_i)
  // for HF pair i = (a_i, c_i) and HO pair j = (b_j, d_j) of the same block.
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int q = 0; q < L->nblock; ++q) {
    const int nt = L->blk[q].w;
    if (nt == 0) continue;
    const int2* pr = &L->pairs[L->pbase[q]];
    // sparse D: per HF pair, the HO pairs with a non-zero coefficient
    std::vector<std::vector<std::pair<int, double>>> Drow(nt);
    std::vector<int> pos((size_t)m * m, -1);
    for (int j = 0; j < nt; ++j) pos[(size_t)pr[j].x * m + pr[j].y] = j;
    for (int i = 0; i < nt; ++i) {
      const int a = pr[i].x, c = pr[i].y;
      // C(x,y) != 0 only for x in the (ml,ms) group of y: b and d range over
      // the union of the groups of a and c
      std::vector<int> cand;
      for (int g : {L->gid[a], L->gid[c]})
        for (int u = L->gstart[g]; u < L->gstart[g + 1]; ++u) cand.push_back(L->gmem[u]);
      std::sort(cand.begin(), cand.end());
      cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
      for (int b : cand)
        for (int d : cand) {
          if (b >= d) continue;  // pair (b,d) as stored: D(i,(b,d)) = C(b,a)C(d,c) - C(d,a)C(b,c)
          const double val = C[(size_t)b + (size_t)a * m] * C[(size_t)d + (size_t)c * m] -
                             C[(size_t)d + (size_t)a * m] * C[(size_t)b + (size_t)c * m];
          if (val == 0.0) continue;
          const int j = pos[(size_t)b * m + d];
          if (j < 0) continue;
          Drow[i].push_back({j, val});
        }
    }
    // W = D V (nt x nt), then HFV = W D^T
    std::vector<double> W((size_t)nt * nt, 0.0), V((size_t)nt * nt);
    for (int j = 0; j < nt; ++j)
      for (int k = 0; k < nt; ++k) V[(size_t)j * nt + k] = vas(pr[j].x, pr[j].y, pr[k].x, pr[k].y);
    for (int i = 0; i < nt; ++i)
      for (const auto& e : Drow[i]) {
        const double* vr = &V[(size_t)e.first * nt];
        double* wr = &W[(size_t)i * nt];
        for (int k = 0; k < nt; ++k) wr[k] += e.second * vr[k];
      }
    const int nh = L->blk[q].x, nb = L->blk[q].y, np = L->blk[q].z;
    const i64* o = &L->boff[6 * q];
    auto put = [&](int slot, int rows, int roff, int coff, int i, int k, double v) {
      vec[o[slot] + (i - roff) + (i64)(k - coff) * rows] = v;
    };
    for (int i = 0; i < nt; ++i)
      for (int k = 0; k < nt; ++k) {
        double s = 0.0;
        for (const auto& e : Drow[k]) s += W[(size_t)i * nt + e.first] * e.second;
        const int ci = i < nh ? 0 : (i < nh + nb ? 1 : 2), ck = k < nh ? 0 : (k < nh + nb ? 1 : 2);
        if (ci < ck) continue;
        const int offs[3] = {0, nh, nh + nb};
        const int rows = ci == 0 ? nh : (ci == 1 ? nb : np);
        int slot = 0;
        if (ci == 0) slot = 0;
        else if (ci == 1) slot = ck == 0 ? 5 : 3;
        else slot = ck == 0 ? 2 : (ck == 1 ? 4 : 1);
        put(slot, rows, offs[ci], offs[ck], i, k, s);
      }
  }
  // HF_E2: E0 = sum_{i<=N} eig(i) - sum_blocks sum_j Vhhhh(j,j)
  double sm = 0.0, sm2 = 0.0;
  for (int q = 0; q < L->nblock; ++q)
    for (int j = 0; j < L->blk[q].x; ++j) sm = sm + vec[L->boff[6 * q] + j + (i64)j * L->blk[q].x];
  for (int i = 0; i < n; ++i) sm2 = sm2 + R.eig[i];
  vec[0] = sm2 - sm;
  return QD_OK;
}

}  // namespace qd

// ---- C ABI ----------------------------------------------------------------------
using namespace qd;

extern "C" int qd_tbme_write(int emax, const char* path, int nthreads, unsigned options) {
  if (emax < 1 || !path || (options & ~QD_TBME_QUAD)) {
    set_error("qd_tbme_write: bad arguments");
    return QD_ERR_ARG;
  }
  TBME T;
  int rc = build_tbme(emax, T, nthreads > 0 ? nthreads : 1, options);
  if (rc) return rc;
  return write_mebin(T, path);
}

namespace qd {
namespace {
// The TBMEs depend only on (emax, options) and are computed at hbar-omega = 1
// (HF scales them by sqrt(hw)): keep the last two sets, so that a grid of
// (N, hbar-omega) instances computes each set once.
struct TbmeCache {
  std::mutex mu;
  std::vector<std::pair<std::pair<int, unsigned>, std::shared_ptr<const TBME>>> sets;
};
TbmeCache& tbme_cache() {
  static TbmeCache c;
  return c;
}
int cached_tbme(int emax, unsigned options, int nthreads, std::shared_ptr<const TBME>* out) {
  TbmeCache& c = tbme_cache();
  {
    std::lock_guard<std::mutex> lock(c.mu);
    for (auto& e : c.sets)
      if (e.first == std::make_pair(emax, options)) {
        *out = e.second;
        return QD_OK;
      }
  }
  auto T = std::make_shared<TBME>();
  int rc = build_tbme(emax, *T, nthreads, options);
  if (rc) return rc;
  std::lock_guard<std::mutex> lock(c.mu);
  c.sets.push_back({{emax, options}, T});
  if (c.sets.size() > 2) c.sets.erase(c.sets.begin());
  *out = T;
  return QD_OK;
}
}  // namespace
}  // namespace qd

extern "C" int qd_hf_hamiltonian(int nbody, int emax, double hw, const char* mebin, int nthreads, double mix,
                                 unsigned options, double* eig_out, double* vec_out, int64_t neq, int* iterations) {
  if (nbody < 0 || emax < 1 || !eig_out || !vec_out || !(mix > 0.0 && mix <= 1.0) || (options & ~QD_TBME_QUAD)) {
    set_error("qd_hf_hamiltonian: bad arguments");
    return QD_ERR_ARG;
  }
  const int nt = nthreads > 0 ? nthreads : 1;
  std::shared_ptr<const TBME> Tp;
  int rc;
  if (mebin) {
    auto t = std::make_shared<TBME>();
    if ((rc = read_mebin(mebin, emax, *t))) return rc;
    Tp = t;
  } else if ((rc = cached_tbme(emax, options, nt, &Tp))) {
    return rc;
  }
  const TBME& T = *Tp;
  HFResult R;
  if ((rc = run_hf(nbody, emax, hw, T, R, nt, mix))) return rc;
  qd_layout L;
  if ((rc = layout_build(&L, nbody, emax, R.eig.data()))) return rc;
  if (neq != L.neq) {
    set_error("qd_hf_hamiltonian: vec has %lld entries, layout needs %lld", (long long)neq, (long long)L.neq);
    return QD_ERR_ARG;
  }
  std::vector<double> vec;
  if ((rc = build_hamiltonian(nbody, emax, hw, T, R, &L, vec, nt))) return rc;
  std::memcpy(vec_out, vec.data(), sizeof(double) * L.neq);
  std::memcpy(eig_out, R.eig.data(), sizeof(double) * L.m);
  if (iterations) *iterations = R.iterations;
  return QD_OK;
}

extern "C" double qd_v_int(const int* qi, const int* qj, const int* qk, const int* ql, double hw) {
  VintCache C;
  int big = 0;
  for (const int* q : {qi, qj, qk, ql}) big = std::max(big, q[0] + std::abs(q[1]));
  C.build(4 * big + 16, 8 * big + 32);
  return v_int(qi, qj, qk, ql, hw, C);
}

extern "C" double qd_v_int_quad(const int* qi, const int* qj, const int* qk, const int* ql, double hw) {
  VintCache C;
  int big = 0;
  for (const int* q : {qi, qj, qk, ql}) big = std::max(big, q[0] + std::abs(q[1]));
  C.build_quad(4 * big + 16, 8 * big + 32);
  return v_int_quad(qi, qj, qk, ql, hw, C);
}
