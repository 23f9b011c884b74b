// oracle.cpp -- CPU restatement of the qd_IMSRG IM-SRG(2) commutator engine.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker that the parity tests,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg compare the CUDA
// engine against.  Nothing in the product (qd_imsrg_b200/) links or calls it.
//
// Parity status: UNPINNED by the reference itself.  The reference (Fortran 90)
// ships no tests, golden vectors or fixtures, and no Fortran compiler exists
// in this image, so the restatement cannot be compared with a reference
// build.  It is cross-checked instead against an independent dense
// (m^4-tensor) formulation of the IM-SRG(2) commutator at tiny bases and
// against algebraic identities (tests/test_oracle_*.py).
//
// The restatement is literal: same loops, same element reads (including the
// herm-factor reads of transposed classes), same constants, same quirks.
// All indices below are 1-based like the Fortran; column-major storage.
// The only liberties taken are ones that are bit-identical to the literal
// loop: loop iterations in which every v_elem() call returns exactly zero
// (its two pairs lie in different (M_L,M_S) blocks) are skipped, and
// independent output elements are distributed over OpenMP threads.
//
// Reference files followed (paths inside the reference project):
//   src/ME_general.f90   types :13-62, build_cross_coupled :363-448,
//                        add_arrays :592-618, copy_arrays :620-660,
//                        set_to_zero :662-686, arrange_states :688-716,
//                        calc_h0 :800-821, construct_cc_ints :923-952,
//                        reindex :956-1116, fermionic index :1348-1357,
//                        v_elem :1557-1680, get_num_elements :1755-1778,
//                        f_elem :1780-1813, vectorize :1871-1989,
//                        mat_2_norm :2112-2138
//   src/commutators.f90  commutator_110 :12-33, _220 :36-70, _121 :73-134,
//                        _111 :137-195, _221 :198-352, _122 :355-676,
//                        _222 :679-985, matrix_mult222 :987-1132,
//                        calc_cc :1135-1159
//   src/IMSRG_tools.f90  build_white :377-434, copy_cc :437-461,
//                        allocate_everything :465-537
//   src/magnus_IMSRG.f90 s_evolve :194-248, BCH_EXPAND :253-318,
//                        MAGNUS_EXPAND :321-369, euler_step :372-384
//   src/HFQDmod.f90      HF_E2 :292-323, MBPT2 :325-362

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <dlfcn.h>

namespace {

typedef long long i64;

// Optional BLAS: when orc_use_blas() has loaded a Fortran-ABI dgemm (e.g.
// scipy's bundled OpenBLAS), dgemm() below calls it, as the reference links
// BLAS dgemm (src/makefile:14).  Inside OpenMP regions it is told to run
// single-threaded (the reference also calls dgemm from its OpenMP loop over
// blocks, commutators.f90:698-706).
typedef void (*fdgemm_t)(const char*, const char*, const int*, const int*, const int*, const double*,
                         const double*, const int*, const double*, const int*, const double*, double*,
                         const int*, size_t, size_t);
typedef int (*fsetthreads_t)(int);
fdgemm_t g_blas_dgemm = nullptr;
fsetthreads_t g_blas_threads_local = nullptr;

// ---------------------------------------------------------------------------
// dgemm: C = alpha*op(A)*op(B) + beta*C, column-major (BLAS semantics).
// Summation over k in increasing order for every C element.
// ---------------------------------------------------------------------------
void dgemm(char ta, char tb, int M, int N, int K, double alpha, const double* A, int lda,
           const double* B, int ldb, double beta, double* C, int ldc) {
  if (M <= 0 || N <= 0) return;
  if (g_blas_dgemm) {
#ifdef _OPENMP
    if (g_blas_threads_local) g_blas_threads_local(omp_in_parallel() ? 1 : omp_get_max_threads());
#endif
    g_blas_dgemm(&ta, &tb, &M, &N, &K, &alpha, A, &lda, B, &ldb, &beta, C, &ldc, 1, 1);
    return;
  }
  bool at = (ta == 'T' || ta == 't');
  bool bt = (tb == 'T' || tb == 't');
#pragma omp parallel for schedule(dynamic, 4) if ((i64)M * N * K > 200000)
  for (int j = 0; j < N; ++j) {
    std::vector<double> acc(M, 0.0);
    for (int k = 0; k < K; ++k) {
      double b = bt ? B[j + (i64)k * ldb] : B[k + (i64)j * ldb];
      if (!at) {
        const double* a = A + (i64)k * lda;
        for (int i = 0; i < M; ++i) acc[i] += a[i] * b;
      } else {
        for (int i = 0; i < M; ++i) acc[i] += A[k + (i64)i * lda] * b;
      }
    }
    for (int i = 0; i < M; ++i) {
      double c = alpha * acc[i];
      if (beta != 0.0) c += beta * C[i + (i64)j * ldc];
      C[i + (i64)j * ldc] = c;
    }
  }
}

// ---------------------------------------------------------------------------
// Layout: arrange_states + reindex + build_cross_coupled
// ---------------------------------------------------------------------------
struct Blk {
  int nhh = 0, nph = 0, npp = 0, ntot = 0, lam[2] = {0, 0};
  std::vector<int> qnhh, qnph, qnpp;  // (k,1:2) at [2*(k-1)+0/1], 1-based states
  i64 o_hhhh = 0, o_pppp = 0, o_pphh = 0, o_phph = 0, o_ppph = 0, o_phhh = 0;
};

struct CCBlk {
  int r = 0, nb = 0;
  std::vector<int> qnab, qnhp;  // (r,1:2), (nb,1:2)
  i64 off = 0;                  // offset of X(r,nb) in a flat X store
  i64 off2 = 0;                 // offset of an r x r matrix in a flat store
};

struct Layout {
  int n = 0, m = 0, emax = 0, nblock = 0, g = 0;
  std::vector<int> qn;       // (m,3): n_princ, ml, ms
  std::vector<double> eig;   // (m)
  std::vector<int> i_array;  // (g,3)
  std::vector<Blk> blk;
  i64 neq = 0;
  i64 o_fhh = 1, o_fpp = 0, o_fph = 0;
  int ccn = 0;
  std::vector<int> ccmap;  // (m*m,2)
  std::vector<CCBlk> cc;
  i64 xsize = 0, x2size = 0;
  // (ml,ms) single-particle groups, for the zero-term skips
  std::vector<int> gid;                   // per state (1-based index)
  std::vector<std::vector<int>> members;  // per group: states in increasing order
  int ia(int II, int c) const { return i_array[(i64)(II - 1) * 3 + (c - 1)]; }
  int QN(int s, int c) const { return qn[(s - 1) * 3 + (c - 1)]; }
};

// arrange_states, ME_general.f90:688-716 (the unused "order" output is omitted)
void arrange_states(int maxE, std::vector<int>& qn) {
  int m = maxE * (maxE + 1);
  qn.assign(m * 3, 0);
  int j = 1;
  for (int R = 0; R <= maxE - 1; ++R)
    for (int ML = -R; ML <= R; ML += 2)
      for (int MS = -1; MS <= 1; MS += 2) {
        int n_princ = (R - std::abs(ML)) / 2;
        qn[(j - 1) * 3 + 0] = n_princ;
        qn[(j - 1) * 3 + 1] = ML;
        qn[(j - 1) * 3 + 2] = MS;
        ++j;
      }
}

// reindex, ME_general.f90:956-1116.  Returns false if the holes it finds are
// not states 1..n (convertF, ME_general.f90:1517-1525, assumes they are).
bool reindex(Layout& L) {
  int M = L.m, n = L.n, emax = L.emax;
  L.nblock = 12 * emax - 9;
  L.g = M * (M - 1) / 2;
  L.i_array.assign((i64)L.g * 3, 0);
  L.blk.assign(L.nblock, Blk());
  double eF;
  if (n > 0) {
    std::vector<double> ecop = L.eig, ec2 = L.eig;
    int i = 1, j = 0;
    eF = 0.0;
    for (;;) {
      double mn = *std::min_element(ecop.begin(), ecop.end());
      if (ec2[i - 1] == mn) {
        ecop[i - 1] = 1000.0;
        ec2[i - 1] = 1000.0;
        ++j;
        if (j == n) {
          eF = L.eig[i - 1];
          break;
        }
        i = 1;
      } else {
        ++i;
      }
    }
    eF = eF + 1.e-6;
  } else {
    eF = 0.0;
  }
  for (int s = 1; s <= M; ++s) {
    bool hole = L.eig[s - 1] <= eF;
    if (hole != (s <= n)) return false;
  }
  int qq = 1;
  for (int MS = -2; MS <= 2; MS += 2) {
    for (int ML = 2 - 2 * emax; ML <= 2 * emax - 2; ++ML) {
      Blk& b = L.blk[qq - 1];
      for (int i = 1; i <= M - 1; ++i)
        for (int j = i + 1; j <= M; ++j) {
          int II = (i - 1) * M - i * (i - 1) / 2 + j - i;
          if (L.QN(i, 3) + L.QN(j, 3) != MS) continue;
          if (L.QN(i, 2) + L.QN(j, 2) != ML) continue;
          int* ia = &L.i_array[(i64)(II - 1) * 3];
          if (L.eig[i - 1] <= eF) {
            if (L.eig[j - 1] <= eF) {
              b.qnhh.push_back(i); b.qnhh.push_back(j);
              ia[0] = 1; ia[1] = qq; ia[2] = (int)b.qnhh.size() / 2;
            } else {
              b.qnph.push_back(i); b.qnph.push_back(j);
              ia[0] = 2; ia[1] = qq; ia[2] = (int)b.qnph.size() / 2;
            }
          } else {
            if (L.eig[j - 1] <= eF) {
              b.qnph.push_back(i); b.qnph.push_back(j);
              ia[0] = 2; ia[1] = qq; ia[2] = (int)b.qnph.size() / 2;
            } else {
              b.qnpp.push_back(i); b.qnpp.push_back(j);
              ia[0] = 3; ia[1] = qq; ia[2] = (int)b.qnpp.size() / 2;
            }
          }
        }
      b.lam[0] = ML;
      b.lam[1] = MS;
      b.nhh = (int)b.qnhh.size() / 2;
      b.nph = (int)b.qnph.size() / 2;
      b.npp = (int)b.qnpp.size() / 2;
      b.ntot = b.nhh + b.nph + b.npp;
      ++qq;
    }
  }
  return true;
}

// vectorize order, ME_general.f90:1871-1975: E0, fhh, fpp, fph, then per block
// Vhhhh, Vpppp, Vpphh, Vphph, Vppph, Vphhh (each column-major).
void offsets(Layout& L) {
  int n = L.n, mp = L.m - L.n;
  i64 k = 1;
  L.o_fhh = k; k += (i64)n * n;
  L.o_fpp = k; k += (i64)mp * mp;
  L.o_fph = k; k += (i64)mp * n;
  for (auto& b : L.blk) {
    b.o_hhhh = k; k += (i64)b.nhh * b.nhh;
    b.o_pppp = k; k += (i64)b.npp * b.npp;
    b.o_pphh = k; k += (i64)b.npp * b.nhh;
    b.o_phph = k; k += (i64)b.nph * b.nph;
    b.o_ppph = k; k += (i64)b.npp * b.nph;
    b.o_phhh = k; k += (i64)b.nph * b.nhh;
  }
  L.neq = k;
}

// build_cross_coupled, ME_general.f90:363-448 (maps only; X is per operator)
void build_cross_coupled(Layout& L) {
  int M = L.m;
  int mlmax_sp = -1000000;
  for (int s = 1; s <= M; ++s) mlmax_sp = std::max(mlmax_sp, L.QN(s, 2));
  int MLmax = 2 * mlmax_sp, MSmax = 2;
  L.ccn = 10 * MLmax + 5;
  L.ccmap.assign((i64)M * M * 2, 0);
  L.cc.assign(L.ccn, CCBlk());
  int q = 1;
  for (int ML = -MLmax; ML <= MLmax; ++ML)
    for (int MS = -MSmax; MS <= MSmax; ++MS) {
      CCBlk& c = L.cc[q - 1];
      int r = 0;
      for (int i = 1; i <= M; ++i)
        for (int j = 1; j <= M; ++j) {
          if (L.QN(i, 2) - L.QN(j, 2) != ML) continue;
          if (L.QN(i, 3) - L.QN(j, 3) != MS) continue;
          ++r;
          L.ccmap[((i64)M * (i - 1) + j - 1) * 2 + 0] = q;
          L.ccmap[((i64)M * (i - 1) + j - 1) * 2 + 1] = r;
          c.qnab.push_back(i); c.qnab.push_back(j);
          if (i <= L.n && j > L.n) { c.qnhp.push_back(i); c.qnhp.push_back(j); }
        }
      c.r = r;
      c.nb = (int)c.qnhp.size() / 2;
      ++q;
    }
  i64 o = 0, o2 = 0;
  for (auto& c : L.cc) {
    c.off = o; o += (i64)c.r * c.nb;
    c.off2 = o2; o2 += (i64)c.r * c.r;
  }
  L.xsize = o;
  L.x2size = o2;
}

void build_groups(Layout& L) {
  int M = L.m;
  L.gid.assign(M + 1, -1);
  L.members.clear();
  std::vector<std::pair<int, int>> keys;
  for (int s = 1; s <= M; ++s) {
    std::pair<int, int> k(L.QN(s, 2), L.QN(s, 3));
    int id = -1;
    for (size_t t = 0; t < keys.size(); ++t)
      if (keys[t] == k) { id = (int)t; break; }
    if (id < 0) {
      id = (int)keys.size();
      keys.push_back(k);
      L.members.push_back({});
    }
    L.gid[s] = id;
    L.members[id].push_back(s);
  }
}

// ---------------------------------------------------------------------------
// Operators (type full_ham): one flat array in vectorize order + herm.
// ---------------------------------------------------------------------------
struct Op {
  const Layout* L;
  int herm;
  std::vector<double> v;
  Op(const Layout* l, int h) : L(l), herm(h), v(l->neq, 0.0) {}
  double& E0() { return v[0]; }
  // one-body arrays: fhh(n,n), fpp(m-n,m-n), fph(m-n,n)
  double& fhh(int i, int j) { return v[L->o_fhh + (i - 1) + (i64)(j - 1) * L->n]; }
  double& fpp(int i, int j) { return v[L->o_fpp + (i - 1) + (i64)(j - 1) * (L->m - L->n)]; }
  double& fph(int i, int j) { return v[L->o_fph + (i - 1) + (i64)(j - 1) * (L->m - L->n)]; }
  double* Vhhhh(int q) { return &v[L->blk[q - 1].o_hhhh]; }
  double* Vpppp(int q) { return &v[L->blk[q - 1].o_pppp]; }
  double* Vpphh(int q) { return &v[L->blk[q - 1].o_pphh]; }
  double* Vphph(int q) { return &v[L->blk[q - 1].o_phph]; }
  double* Vppph(int q) { return &v[L->blk[q - 1].o_ppph]; }
  double* Vphhh(int q) { return &v[L->blk[q - 1].o_phhh]; }
};

struct CC {
  const Layout* L;
  double herm = 1.0;
  bool zero = true;  // X known to be identically zero (never filled)
  std::vector<double> X;
  explicit CC(const Layout* l) : L(l), X(l->xsize, 0.0) {}
};

inline double el(const double* a, int ld, int i, int j) { return a[(i - 1) + (i64)(j - 1) * ld]; }
inline double& elr(double* a, int ld, int i, int j) { return a[(i - 1) + (i64)(j - 1) * ld]; }

// v_elem, ME_general.f90:1557-1680.  Energy order == states order here
// (convertF sets eh(i)=i, ep(i)=n+i).
double v_elem(int a1, int a2, int a3, int a4, Op& rec) {
  if (a1 == a2 || a3 == a4) return 0.0;
  const Layout& L = *rec.L;
  int M = L.m;
  int k[4] = {a1, a2, a3, a4};
  int pre = 1;
  if (k[0] > k[1]) { std::swap(k[0], k[1]); pre = -1; }
  if (k[2] > k[3]) { std::swap(k[2], k[3]); pre = -1 * pre; }
  int II = (k[0] - 1) * M - k[0] * (k[0] - 1) / 2 + k[1] - k[0];
  int JJ = (k[2] - 1) * M - k[2] * (k[2] - 1) / 2 + k[3] - k[2];
  int w2 = L.ia(JJ, 3), p2 = L.ia(JJ, 2);
  int w1 = L.ia(II, 3), p1 = L.ia(II, 2);
  if (p1 != p2) return 0.0;
  const Blk& b = L.blk[p1 - 1];
  int c1 = L.ia(II, 1), c2 = L.ia(JJ, 1);
  int h = rec.herm;
  switch (c1) {
    case 1:
      switch (c2) {
        case 1: return el(rec.Vhhhh(p1), b.nhh, w1, w2) * pre;
        case 2: return el(rec.Vphhh(p1), b.nph, w2, w1) * pre * h;
        case 3: return el(rec.Vpphh(p1), b.npp, w2, w1) * pre * h;
      }
      break;
    case 2:
      switch (c2) {
        case 1: return el(rec.Vphhh(p1), b.nph, w1, w2) * pre;
        case 2: return el(rec.Vphph(p1), b.nph, w1, w2) * pre;
        case 3: return el(rec.Vppph(p1), b.npp, w2, w1) * pre * h;
      }
      break;
    case 3:
      switch (c2) {
        case 1: return el(rec.Vpphh(p1), b.npp, w1, w2) * pre;
        case 2: return el(rec.Vppph(p1), b.npp, w1, w2) * pre;
        case 3: return el(rec.Vpppp(p1), b.npp, w1, w2) * pre;
      }
      break;
  }
  return 0.0;
}

// ---------------------------------------------------------------------------
// Algebra: add_arrays, copy_arrays, set_to_zero, mat_2_norm
// ---------------------------------------------------------------------------
void add_arrays(Op& r1, double s1, Op& r2, double s2, Op& r3) {
  i64 N = r1.L->neq;
  for (i64 i = 0; i < N; ++i) r3.v[i] = s1 * r1.v[i] + s2 * r2.v[i];
}
void copy_arrays(Op& r1, Op& r2) { r2.v = r1.v; }
void set_to_zero(Op& r1) { std::fill(r1.v.begin(), r1.v.end(), 0.0); }

// mat_2_norm, ME_general.f90:2112-2138: the square root of the sum of
// squares of every stored one- and two-body entry (E0 excluded), in the
// reference's order: od = od + sum(fph**2) + sum(fpp**2) + sum(fhh**2)
// (:2125), then per block q (:2127-2133)
// od = od + sum(Vhhhh**2) + sum(Vpppp**2) + sum(Vpphh**2) + sum(Vphph**2)
//         + sum(Vphhh**2) + sum(Vppph**2), each line summed left to right.
namespace {
double sumsq(const double* x, i64 n) {
  double s = 0.0;
  for (i64 i = 0; i < n; ++i) s += x[i] * x[i];
  return s;
}
}  // namespace
double mat_2_norm(Op& r) {
  const Layout& L = *r.L;
  const i64 n = L.n, mp = L.m - L.n;
  double od = 0.0;
  od = od + sumsq(&r.v[L.o_fph], mp * n) + sumsq(&r.v[L.o_fpp], mp * mp) + sumsq(&r.v[L.o_fhh], n * n);
  for (int q = 1; q <= L.nblock; ++q) {
    const Blk& b = L.blk[q - 1];
    const i64 nh = b.nhh, nb = b.nph, np = b.npp;
    od = od + sumsq(r.Vhhhh(q), nh * nh) + sumsq(r.Vpppp(q), np * np) + sumsq(r.Vpphh(q), np * nh) +
         sumsq(r.Vphph(q), nb * nb) + sumsq(r.Vphhh(q), nb * nh) + sumsq(r.Vppph(q), np * nb);
  }
  return std::sqrt(od);
}

// ---------------------------------------------------------------------------
// Commutators
// ---------------------------------------------------------------------------
// commutator_110, commutators.f90:12-33
double commutator_110(int m, int n, Op& r1, Op& r2) {
  std::vector<double> Q((size_t)m * m);
  dgemm('N', 'T', m, m, n, 1.0, &r1.v[r1.L->o_fph], m, &r2.v[r2.L->o_fph], m, 0.0, Q.data(), m);
  double c = 0.0;
  for (int i = 1; i <= m; ++i) c = c + el(Q.data(), m, i, i);
  c = (r1.herm - r2.herm) * c;
  return c;
}

// commutator_220, commutators.f90:36-70
double commutator_220(Op& r1, Op& r2) {
  double c = 0.0;
  const Layout& L = *r1.L;
  for (int j = 1; j <= L.nblock; ++j) {
    const Blk& b = L.blk[j - 1];
    if (b.npp * b.nhh == 0) continue;
    int m = b.npp, n = b.nhh;
    std::vector<double> Q((size_t)m * m);
    dgemm('N', 'T', m, m, n, 1.0, r1.Vpphh(j), m, r2.Vpphh(j), m, 0.0, Q.data(), m);
    for (int i = 1; i <= m; ++i) c = c + el(Q.data(), m, i, i) * (r1.herm - r2.herm);
  }
  return c;
}

// commutator_121, commutators.f90:73-134.  A (i,a) iteration is skipped only
// when all four v_elem calls of that iteration vanish by block structure.
void commutator_121(Op& r1, Op& r2, Op& r3) {
  const Layout& L = *r2.L;
  int n = L.n, m = L.m - L.n;
  int h1x = r1.herm, h2x = r2.herm;
  auto live = [&](int x, int y, int i, int a) {
    // v(a,x,i,y) needs ml_a+ml_x==ml_i+ml_y; v(i,x,a,y) needs ml_i+ml_x==ml_a+ml_y
    int dl = L.QN(a, 2) - L.QN(i, 2), ds = L.QN(a, 3) - L.QN(i, 3);
    int tl = L.QN(y, 2) - L.QN(x, 2), ts = L.QN(y, 3) - L.QN(x, 3);
    return (dl == tl && ds == ts) || (dl == -tl && ds == -ts);
  };
  // r3 = r3 + f1(a,i)*(h1*v2(a,x,i,y) - v2(i,x,a,y)) - f2(a,i)*(h2*v1(a,x,i,y) - v1(i,x,a,y)),
  // evaluated left to right as in the Fortran.
  auto acc = [&](double r3v, int x, int y, int i, int a) {
    return r3v + r1.fph(a, i) * (h1x * v_elem(a + n, x, i, y, r2) - v_elem(i, x, a + n, y, r2)) -
           r2.fph(a, i) * (h2x * v_elem(a + n, x, i, y, r1) - v_elem(i, x, a + n, y, r1));
  };
#pragma omp parallel for schedule(dynamic, 1)
  for (int h2 = 1; h2 <= n; ++h2) {
    for (int h1 = 1; h1 <= n; ++h1)
      for (int i = 1; i <= n; ++i)
        for (int a = 1; a <= m; ++a) {
          if (!live(h1, h2, i, a + n)) continue;
          r3.fhh(h1, h2) = acc(r3.fhh(h1, h2), h1, h2, i, a);
        }
    for (int p1 = 1; p1 <= m; ++p1)
      for (int i = 1; i <= n; ++i)
        for (int a = 1; a <= m; ++a) {
          if (!live(p1 + n, h2, i, a + n)) continue;
          r3.fph(p1, h2) = acc(r3.fph(p1, h2), p1 + n, h2, i, a);
        }
  }
#pragma omp parallel for schedule(dynamic, 1)
  for (int p2 = 1; p2 <= m; ++p2)
    for (int p1 = 1; p1 <= m; ++p1)
      for (int i = 1; i <= n; ++i)
        for (int a = 1; a <= m; ++a) {
          if (!live(p1 + n, p2 + n, i, a + n)) continue;
          r3.fpp(p1, p2) = acc(r3.fpp(p1, p2), p1 + n, p2 + n, i, a);
        }
}

// commutator_111, commutators.f90:137-195 (overwrites r3's one-body part)
void commutator_111(Op& r1, Op& r2, Op& r3) {
  const Layout& L = *r2.L;
  int n = L.n, m = L.m - L.n;
  double h1 = r1.herm, h2 = r2.herm;
  {
    std::vector<double> Q1((size_t)n * n), Q2((size_t)n * n);
    dgemm('N', 'N', n, n, n, 1.0, &r1.v[L.o_fhh], n, &r2.v[L.o_fhh], n, 0.0, Q1.data(), n);
    dgemm('T', 'N', n, n, m, 1.0, &r2.v[L.o_fph], m, &r1.v[L.o_fph], m, 0.0, Q2.data(), n);
    for (int j = 1; j <= n; ++j)
      for (int i = 1; i <= n; ++i)
        r3.fhh(i, j) = el(Q1.data(), n, i, j) - h2 * el(Q2.data(), n, i, j) +
                       h1 * (el(Q2.data(), n, j, i) - h2 * el(Q1.data(), n, j, i));
  }
  {
    std::vector<double> Q1((size_t)m * m), Q2((size_t)m * m);
    dgemm('N', 'N', m, m, m, 1.0, &r2.v[L.o_fpp], m, &r1.v[L.o_fpp], m, 0.0, Q1.data(), m);
    dgemm('N', 'T', m, m, n, 1.0, &r1.v[L.o_fph], m, &r2.v[L.o_fph], m, 0.0, Q2.data(), m);
    for (int j = 1; j <= m; ++j)
      for (int i = 1; i <= m; ++i)
        r3.fpp(i, j) = h2 * el(Q2.data(), m, i, j) +
                       h1 * (h2 * el(Q1.data(), m, j, i) - el(Q2.data(), m, j, i)) -
                       el(Q1.data(), m, i, j);
  }
  {
    std::vector<double> Q1((size_t)m * n), Q2((size_t)m * n), Q3((size_t)m * n), Q4((size_t)m * n);
    dgemm('N', 'N', m, n, n, 1.0, &r1.v[L.o_fph], m, &r2.v[L.o_fhh], n, 0.0, Q1.data(), m);
    dgemm('N', 'N', m, n, n, 1.0, &r2.v[L.o_fph], m, &r1.v[L.o_fhh], n, 0.0, Q2.data(), m);
    dgemm('N', 'N', m, n, m, 1.0, &r1.v[L.o_fpp], m, &r2.v[L.o_fph], m, 0.0, Q3.data(), m);
    dgemm('N', 'N', m, n, m, 1.0, &r2.v[L.o_fpp], m, &r1.v[L.o_fph], m, 0.0, Q4.data(), m);
    for (i64 k = 0; k < (i64)m * n; ++k) r3.v[L.o_fph + k] = Q1[k] - Q2[k] + Q3[k] - Q4[k];
  }
}

// commutator_221, commutators.f90:198-352
void commutator_221(Op& r1, Op& r2, Op& r3, Op& w1, Op& w2) {
  const Layout& L = *r2.L;
  int m = L.m, n = L.n;
  double h1 = r1.herm, h2 = r2.herm;
  for (int w = 1; w <= L.nblock; ++w) {
    const Blk& b = L.blk[w - 1];
    int nh = b.nhh, np = b.npp, nb = b.nph;
    std::fill_n(w1.Vhhhh(w), (size_t)nh * nh, 0.0);
    std::fill_n(w2.Vhhhh(w), (size_t)nh * nh, 0.0);
    std::fill_n(w1.Vpppp(w), (size_t)np * np, 0.0);
    std::fill_n(w2.Vpppp(w), (size_t)np * np, 0.0);
    std::fill_n(w1.Vpphh(w), (size_t)np * nh, 0.0);
    std::fill_n(w2.Vpphh(w), (size_t)np * nh, 0.0);
    std::fill_n(w1.Vppph(w), (size_t)np * nb, 0.0);
    std::fill_n(w2.Vppph(w), (size_t)np * nb, 0.0);
    std::fill_n(w1.Vphhh(w), (size_t)nb * nh, 0.0);
    std::fill_n(w2.Vphhh(w), (size_t)nb * nh, 0.0);
    std::fill_n(w1.Vphph(w), (size_t)nb * nb, 0.0);
    std::fill_n(w1.Vphph(w), (size_t)nb * nb, 0.0);  // w2%Vphph is not zeroed (quirk)
    if (np * nh != 0)
      dgemm('N', 'T', np, np, nh, 1.0, r1.Vpphh(w), np, r2.Vpphh(w), np, 0.0, w1.Vpppp(w), np);
    if (np * nb != 0)
      dgemm('T', 'N', nb, nb, np, 1.0, r2.Vppph(w), np, r1.Vppph(w), np, 0.0, w1.Vphph(w), nb);
    if (nh * np != 0)
      dgemm('T', 'N', nh, nh, np, 1.0, r2.Vpphh(w), np, r1.Vpphh(w), np, 0.0, w1.Vhhhh(w), nh);
    if (nh * nb != 0)
      dgemm('N', 'T', nb, nb, nh, 1.0, r1.Vphhh(w), nb, r2.Vphhh(w), nb, 0.0, w2.Vphph(w), nb);
    if (nh * nb * np != 0) {
      dgemm('T', 'N', nb, nh, np, 1.0, r2.Vppph(w), np, r1.Vpphh(w), np, 0.0, w1.Vphhh(w), nb);
      dgemm('T', 'N', nb, nh, np, 1.0, r1.Vppph(w), np, r2.Vpphh(w), np, 0.0, w2.Vphhh(w), nb);
      dgemm('N', 'T', np, nb, nh, 1.0, r1.Vpphh(w), np, r2.Vphhh(w), nb, 0.0, w1.Vppph(w), np);
      dgemm('N', 'T', np, nb, nh, 1.0, r2.Vpphh(w), np, r1.Vphhh(w), nb, 0.0, w2.Vppph(w), np);
    }
  }
  // Targets whose two indices lie in different (ml,ms) groups receive only
  // exact zeros from v_elem; they are skipped.
  auto same = [&](int x, int y) { return L.gid[x] == L.gid[y]; };
#pragma omp parallel for schedule(dynamic, 4)
  for (int p = 1; p <= m - n; ++p)
    for (int p2 = 1; p2 <= m - n; ++p2) {
      if (!same(p + n, p2 + n)) continue;
      for (int i = 1; i <= n; ++i)
        r3.fpp(p, p2) = r3.fpp(p, p2) + h1 * v_elem(i, p2 + n, i, p + n, w1) - h2 * v_elem(i, p + n, i, p2 + n, w1);
      for (int a = n + 1; a <= m; ++a)
        r3.fpp(p, p2) = r3.fpp(p, p2) - h1 * v_elem(a, p2 + n, a, p + n, w1) + h2 * v_elem(a, p + n, a, p2 + n, w1);
    }
  for (int h = 1; h <= n; ++h)
    for (int hh2 = 1; hh2 <= n; ++hh2) {
      if (!same(h, hh2)) continue;
      for (int i = 1; i <= n; ++i)
        r3.fhh(h, hh2) = r3.fhh(h, hh2) + h1 * v_elem(i, hh2, i, h, w1) - h2 * v_elem(i, h, i, hh2, w1);
      for (int a = n + 1; a <= m; ++a)
        r3.fhh(h, hh2) = r3.fhh(h, hh2) - h1 * v_elem(a, hh2, a, h, w2) + h2 * v_elem(a, h, a, hh2, w2);
    }
#pragma omp parallel for schedule(dynamic, 4)
  for (int p = 1; p <= m - n; ++p)
    for (int h = 1; h <= n; ++h) {
      if (!same(p + n, h)) continue;
      for (int i = 1; i <= n; ++i)
        r3.fph(p, h) = r3.fph(p, h) + h1 * v_elem(i, p + n, i, h, w2) - h2 * v_elem(i, p + n, i, h, w1);
      for (int a = n + 1; a <= m; ++a)
        r3.fph(p, h) = r3.fph(p, h) - h1 * v_elem(a, p + n, a, h, w2) + h2 * v_elem(a, p + n, a, h, w1);
    }
}

// One-body element reads used by commutator_122 (fhh(x,i) / fph(x-n,i) in the
// hole loop, fph(a,x) / fpp(a,x-n) in the particle loop).
inline double fh(Op& r, int x, int i) { int n = r.L->n; return x <= n ? r.fhh(x, i) : r.fph(x - n, i); }
inline double fp(Op& r, int a, int x) { int n = r.L->n; return x <= n ? r.fph(a, x) : r.fpp(a, x - n); }

// commutator_122, commutators.f90:355-676 (overwrites every two-body
// sub-block).  All six sub-block loops of the reference share one algebraic
// form in the leg indices (b1,b2 | k1,k2) with a sign pre:
//   hole loop i:      + f1(b1,i)V2(i,b2,k1,k2) + f1(b2,i)V2(b1,i,k1,k2)
//                     - h1[f1(k1,i)V2(b1,b2,i,k2) + f1(k2,i)V2(b1,b2,k1,i)] - (1<->2)
//   particle loop a:  + h1[f1'(a,b1)V2(a,b2,k1,k2) + f1'(a,b2)V2(b1,a,k1,k2)]
//                     - [f1'(a,k1)V2(b1,b2,a,k2) + f1'(a,k2)V2(b1,b2,k1,a)] - (1<->2)
// with f(x,i) = fhh(x,i) for a hole x, fph(x-n,i) for a particle x, and
// f'(a,x) = fph(a,x) for a hole x, fpp(a,x-n) for a particle x, exactly the
// reads of the reference.  Loop variables whose eight v_elem calls all vanish
// (the variable is in none of the four legs' (ml,ms) groups) are skipped.
// The hhhh, pppp and pphh loops of the reference have no "pre" factor and
// chain the accumulator first ("r3 + t1 + t2 - t3 - t4", left to right); the
// phhh, ppph and phph loops wrap the whole update as "r3 + pre*( ... )".
void c122_elem(Op& r1, Op& r2, int b1, int b2, int k1, int k2, int pre, bool has_pre, double& out,
               const std::vector<int>& holes_u, const std::vector<int>& parts_u) {
  int n = r1.L->n;
  double h1 = r1.herm, h2 = r2.herm;
  for (int i : holes_u) {
    double t1 = fh(r1, b1, i) * v_elem(i, b2, k1, k2, r2);
    double t2 = fh(r1, b2, i) * v_elem(b1, i, k1, k2, r2);
    double t3 = h1 * (fh(r1, k1, i) * v_elem(b1, b2, i, k2, r2) + fh(r1, k2, i) * v_elem(b1, b2, k1, i, r2));
    double t4 = (fh(r2, b1, i) * v_elem(i, b2, k1, k2, r1) + fh(r2, b2, i) * v_elem(b1, i, k1, k2, r1) -
                 h2 * (fh(r2, k1, i) * v_elem(b1, b2, i, k2, r1) + fh(r2, k2, i) * v_elem(b1, b2, k1, i, r1)));
    if (has_pre)
      out = out + pre * (t1 + t2 - t3 - t4);
    else
      out = out + t1 + t2 - t3 - t4;
  }
  for (int ax : parts_u) {
    int a = ax - n;
    double t1 = h1 * (fp(r1, a, b1) * v_elem(a + n, b2, k1, k2, r2) + fp(r1, a, b2) * v_elem(b1, a + n, k1, k2, r2));
    double t2 = (fp(r1, a, k1) * v_elem(b1, b2, a + n, k2, r2) + fp(r1, a, k2) * v_elem(b1, b2, k1, a + n, r2));
    double t3 = (h2 * (fp(r2, a, b1) * v_elem(a + n, b2, k1, k2, r1) + fp(r2, a, b2) * v_elem(b1, a + n, k1, k2, r1)) -
                 (fp(r2, a, k1) * v_elem(b1, b2, a + n, k2, r1) + fp(r2, a, k2) * v_elem(b1, b2, k1, a + n, r1)));
    if (has_pre)
      out = out + pre * (t1 - t2 - t3);
    else
      out = out + t1 - t2 - t3;
  }
}

void union_groups(const Layout& L, int b1, int b2, int k1, int k2, std::vector<int>& hu, std::vector<int>& pu) {
  int gs[4] = {L.gid[b1], L.gid[b2], L.gid[k1], L.gid[k2]};
  std::vector<int> all;
  for (int t = 0; t < 4; ++t) {
    bool dup = false;
    for (int u = 0; u < t; ++u) dup |= gs[u] == gs[t];
    if (dup) continue;
    const auto& mm = L.members[gs[t]];
    all.insert(all.end(), mm.begin(), mm.end());
  }
  std::sort(all.begin(), all.end());
  hu.clear();
  pu.clear();
  for (int s : all) (s <= L.n ? hu : pu).push_back(s);
}

void commutator_122(Op& r1, Op& r2, Op& r3, bool literal) {
  const Layout& L = *r2.L;
  int n = L.n, m = L.m;
  std::vector<int> allh, allp;
  for (int s = 1; s <= n; ++s) allh.push_back(s);
  for (int s = n + 1; s <= m; ++s) allp.push_back(s);
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 1; q <= L.nblock; ++q) {
    const Blk& b = L.blk[q - 1];
    int nh = b.nhh, np = b.npp, nb = b.nph;
    std::vector<int> hu, pu;
    // pre == 0 marks the loops without a "pre" factor (hhhh, pppp, pphh)
    auto run = [&](int b1, int b2, int k1, int k2, int pre, double& out) {
      bool has_pre = pre != 0;
      int p = has_pre ? pre : 1;
      if (literal) {
        c122_elem(r1, r2, b1, b2, k1, k2, p, has_pre, out, allh, allp);
      } else {
        union_groups(L, b1, b2, k1, k2, hu, pu);
        c122_elem(r1, r2, b1, b2, k1, k2, p, has_pre, out, hu, pu);
      }
    };
    if (nh > 0) {
      double* C = r3.Vhhhh(q);
      std::fill_n(C, (size_t)nh * nh, 0.0);
      for (int JJ = 1; JJ <= nh; ++JJ)
        for (int II = 1; II <= nh; ++II)
          run(b.qnhh[2 * (II - 1)], b.qnhh[2 * (II - 1) + 1], b.qnhh[2 * (JJ - 1)], b.qnhh[2 * (JJ - 1) + 1], 0,
              elr(C, nh, II, JJ));
    }
    if (np > 0) {
      double* C = r3.Vpppp(q);
      std::fill_n(C, (size_t)np * np, 0.0);
      for (int JJ = 1; JJ <= np; ++JJ)
        for (int II = 1; II <= np; ++II)
          run(b.qnpp[2 * (II - 1)], b.qnpp[2 * (II - 1) + 1], b.qnpp[2 * (JJ - 1)], b.qnpp[2 * (JJ - 1) + 1], 0,
              elr(C, np, II, JJ));
    }
    if (np * nh > 0) {
      double* C = r3.Vpphh(q);
      std::fill_n(C, (size_t)np * nh, 0.0);
      for (int JJ = 1; JJ <= nh; ++JJ)
        for (int II = 1; II <= np; ++II)
          run(b.qnpp[2 * (II - 1)], b.qnpp[2 * (II - 1) + 1], b.qnhh[2 * (JJ - 1)], b.qnhh[2 * (JJ - 1) + 1], 0,
              elr(C, np, II, JJ));
    }
    if (nh * nb > 0) {
      double* C = r3.Vphhh(q);
      std::fill_n(C, (size_t)nb * nh, 0.0);
      for (int JJ = 1; JJ <= nh; ++JJ)
        for (int II = 1; II <= nb; ++II)
          run(b.qnph[2 * (II - 1) + 1], b.qnph[2 * (II - 1)], b.qnhh[2 * (JJ - 1)], b.qnhh[2 * (JJ - 1) + 1], -1,
              elr(C, nb, II, JJ));
    }
    if (np * nb > 0) {
      double* C = r3.Vppph(q);
      std::fill_n(C, (size_t)np * nb, 0.0);
      for (int JJ = 1; JJ <= nb; ++JJ)
        for (int II = 1; II <= np; ++II)
          run(b.qnpp[2 * (II - 1)], b.qnpp[2 * (II - 1) + 1], b.qnph[2 * (JJ - 1) + 1], b.qnph[2 * (JJ - 1)], -1,
              elr(C, np, II, JJ));
    }
    if (nb > 0) {
      double* C = r3.Vphph(q);
      std::fill_n(C, (size_t)nb * nb, 0.0);
      for (int JJ = 1; JJ <= nb; ++JJ)
        for (int II = 1; II <= nb; ++II)
          run(b.qnph[2 * (II - 1) + 1], b.qnph[2 * (II - 1)], b.qnph[2 * (JJ - 1) + 1], b.qnph[2 * (JJ - 1)], 1,
              elr(C, nb, II, JJ));
    }
  }
}

// calc_cc, commutators.f90:1135-1159: X(r,nb) = v_elem(j,k,i,l,H)
void calc_cc(Op& H, CC& HCC) {
  const Layout& L = *H.L;
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 1; q <= L.ccn; ++q) {
    const CCBlk& c = L.cc[q - 1];
    for (int r = 1; r <= c.r; ++r) {
      int i = c.qnab[2 * (r - 1)], j = c.qnab[2 * (r - 1) + 1];
      for (int nb = 1; nb <= c.nb; ++nb) {
        int k = c.qnhp[2 * (nb - 1)], l = c.qnhp[2 * (nb - 1) + 1];
        HCC.X[c.off + (r - 1) + (i64)(nb - 1) * c.r] = v_elem(j, k, i, l, H);
      }
    }
  }
  HCC.zero = false;
}

// matrix_mult222, commutators.f90:987-1132 (w1 blocks used as scratch)
void matrix_mult222(Op& r1, Op& r2, Op& r3, Op& w1, int q, int nh, int np, int nb) {
  double h1 = r1.herm, h2 = r2.herm;
  auto addT = [](double* C, const double* W, int n, double a, double b) {
    // C = C + (a*W^T + b*W)
    for (int j = 1; j <= n; ++j)
      for (int i = 1; i <= n; ++i) elr(C, n, i, j) = elr(C, n, i, j) + (a * el(W, n, j, i) + b * el(W, n, i, j));
  };
  auto add = [](double* C, const double* W, i64 cnt, double s) {
    for (i64 k = 0; k < cnt; ++k) C[k] = C[k] + s * W[k];
  };
  if (nh * np > 0) {
    dgemm('T', 'N', nh, nh, np, 1.0, r2.Vpphh(q), np, r1.Vpphh(q), np, 0.0, w1.Vhhhh(q), nh);
    addT(r3.Vhhhh(q), w1.Vhhhh(q), nh, h1, -h2);
    dgemm('N', 'T', np, np, nh, 1.0, r1.Vpphh(q), np, r2.Vpphh(q), np, 0.0, w1.Vpppp(q), np);
    addT(r3.Vpppp(q), w1.Vpppp(q), np, h1, -h2);
    dgemm('N', 'N', np, nh, np, 1.0, r1.Vpppp(q), np, r2.Vpphh(q), np, 0.0, w1.Vpphh(q), np);
    add(r3.Vpphh(q), w1.Vpphh(q), (i64)np * nh, 1.0);
    dgemm('N', 'N', np, nh, np, 1.0, r2.Vpppp(q), np, r1.Vpphh(q), np, 0.0, w1.Vpphh(q), np);
    add(r3.Vpphh(q), w1.Vpphh(q), (i64)np * nh, -1.0);
    dgemm('N', 'N', np, nh, nh, 1.0, r1.Vpphh(q), np, r2.Vhhhh(q), nh, 0.0, w1.Vpphh(q), np);
    add(r3.Vpphh(q), w1.Vpphh(q), (i64)np * nh, -1.0);
    dgemm('N', 'N', np, nh, nh, 1.0, r2.Vpphh(q), np, r1.Vhhhh(q), nh, 0.0, w1.Vpphh(q), np);
    add(r3.Vpphh(q), w1.Vpphh(q), (i64)np * nh, 1.0);
  }
  if (nh > 0) {
    dgemm('N', 'N', nh, nh, nh, 1.0, r1.Vhhhh(q), nh, r2.Vhhhh(q), nh, 0.0, w1.Vhhhh(q), nh);
    addT(r3.Vhhhh(q), w1.Vhhhh(q), nh, h1 * h2, -1.0);
  }
  if (np > 0) {
    dgemm('N', 'N', np, np, np, 1.0, r2.Vpppp(q), np, r1.Vpppp(q), np, 0.0, w1.Vpppp(q), np);
    addT(r3.Vpppp(q), w1.Vpppp(q), np, h1 * h2, -1.0);
  }
  if (nb * np * nh > 0) {
    dgemm('T', 'N', nb, nh, np, 1.0, r1.Vppph(q), np, r2.Vpphh(q), np, 0.0, w1.Vphhh(q), nb);
    add(r3.Vphhh(q), w1.Vphhh(q), (i64)nb * nh, h1);
    dgemm('T', 'N', nb, nh, np, 1.0, r2.Vppph(q), np, r1.Vpphh(q), np, 0.0, w1.Vphhh(q), nb);
    add(r3.Vphhh(q), w1.Vphhh(q), (i64)nb * nh, -h2);
    dgemm('N', 'T', np, nb, nh, 1.0, r1.Vpphh(q), np, r2.Vphhh(q), nb, 0.0, w1.Vppph(q), np);
    add(r3.Vppph(q), w1.Vppph(q), (i64)np * nb, -h2);
    dgemm('N', 'T', np, nb, nh, 1.0, r2.Vpphh(q), np, r1.Vphhh(q), nb, 0.0, w1.Vppph(q), np);
    add(r3.Vppph(q), w1.Vppph(q), (i64)np * nb, h1);
  }
  if (nb * nh > 0) {
    dgemm('N', 'N', nb, nh, nh, 1.0, r1.Vphhh(q), nb, r2.Vhhhh(q), nh, 0.0, w1.Vphhh(q), nb);
    add(r3.Vphhh(q), w1.Vphhh(q), (i64)nb * nh, -1.0);
    dgemm('N', 'N', nb, nh, nh, 1.0, r2.Vphhh(q), nb, r1.Vhhhh(q), nh, 0.0, w1.Vphhh(q), nb);
    add(r3.Vphhh(q), w1.Vphhh(q), (i64)nb * nh, 1.0);
    dgemm('N', 'T', nb, nb, nh, 1.0, r1.Vphhh(q), nb, r2.Vphhh(q), nb, 0.0, w1.Vphph(q), nb);
    addT(r3.Vphph(q), w1.Vphph(q), nb, h1, -h2);
  }
  if (nb * np > 0) {
    dgemm('N', 'N', np, nb, np, 1.0, r1.Vpppp(q), np, r2.Vppph(q), np, 0.0, w1.Vppph(q), np);
    add(r3.Vppph(q), w1.Vppph(q), (i64)np * nb, 1.0);
    dgemm('N', 'N', np, nb, np, 1.0, r2.Vpppp(q), np, r1.Vppph(q), np, 0.0, w1.Vppph(q), np);
    add(r3.Vppph(q), w1.Vppph(q), (i64)np * nb, -1.0);
    dgemm('T', 'N', nb, nb, np, 1.0, r2.Vppph(q), np, r1.Vppph(q), np, 0.0, w1.Vphph(q), nb);
    addT(r3.Vphph(q), w1.Vphph(q), nb, h1, -h2);
  }
}

// commutator_222, commutators.f90:679-985 with construct_cc_ints,
// ME_general.f90:923-952.  XCC = HCC%herm*X_eta*X_H^T, YCC = ETACC%herm*X_H*X_eta^T.
void commutator_222(Op& r1, Op& r2, Op& r3, Op& w1, CC& HCC, CC& ETACC) {
  const Layout& L = *r2.L;
  int M = L.m;
  std::vector<double> XCC, YCC;
  bool have_cc = !(HCC.zero && ETACC.zero);
  if (have_cc) {
    XCC.assign(L.x2size, 0.0);
    YCC.assign(L.x2size, 0.0);
    for (int q = 1; q <= L.ccn; ++q) {
      const CCBlk& c = L.cc[q - 1];
      int r = c.r, nb = c.nb;
      if (r == 0 || nb == 0) continue;
      dgemm('N', 'T', r, r, nb, HCC.herm, &ETACC.X[c.off], r, &HCC.X[c.off], r, 0.0, &XCC[c.off2], r);
      dgemm('N', 'T', r, r, nb, ETACC.herm, &HCC.X[c.off], r, &ETACC.X[c.off], r, 0.0, &YCC[c.off2], r);
    }
  }
  auto mp = [&](int x, int y, int& q, int& r) {
    i64 k = (i64)M * (x - 1) + y - 1;
    q = L.ccmap[2 * k];
    r = L.ccmap[2 * k + 1];
  };
  auto XC = [&](const std::vector<double>& Z, int q, int ra, int rb) {
    const CCBlk& c = L.cc[q - 1];
    return Z[c.off2 + (ra - 1) + (i64)(rb - 1) * c.r];
  };
  auto ph = [&](int b1, int b2, int k1, int k2) {
    // legs named (1,2 | 3,4) = (b1,b2 | k1,k2), as in commutators.f90:725-751
    int q31, r31, q24, r24, q32, r32, q14, r14, q41, r41, q23, r23, q42, r42, q13, r13;
    mp(k1, b1, q31, r31); mp(b2, k2, q24, r24);
    mp(k1, b2, q32, r32); mp(b1, k2, q14, r14);
    mp(k2, b1, q41, r41); mp(b2, k1, q23, r23);
    mp(k2, b2, q42, r42); mp(b1, k1, q13, r13);
    double X = XC(XCC, q31, r31, r24) - XC(XCC, q32, r32, r14) + XC(XCC, q42, r42, r13) - XC(XCC, q41, r41, r23);
    X = X - XC(YCC, q42, r42, r13) + XC(YCC, q41, r41, r23) - XC(YCC, q31, r31, r24) + XC(YCC, q32, r32, r14);
    return X;
  };
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 1; q <= L.nblock; ++q) {
    const Blk& b = L.blk[q - 1];
    int nh = b.nhh, np = b.npp, nb = b.nph;
    matrix_mult222(r1, r2, r3, w1, q, nh, np, nb);
    if (!have_cc) continue;  // X == 0: every term below is an exact zero
    for (int JJ = 1; JJ <= nh; ++JJ)
      for (int II = 1; II <= nh; ++II) {
        double X = ph(b.qnhh[2 * (II - 1)], b.qnhh[2 * (II - 1) + 1], b.qnhh[2 * (JJ - 1)], b.qnhh[2 * (JJ - 1) + 1]);
        elr(r3.Vhhhh(q), nh, II, JJ) = elr(r3.Vhhhh(q), nh, II, JJ) + X;
      }
    for (int JJ = 1; JJ <= np; ++JJ)
      for (int II = 1; II <= np; ++II) {
        double X = ph(b.qnpp[2 * (II - 1)], b.qnpp[2 * (II - 1) + 1], b.qnpp[2 * (JJ - 1)], b.qnpp[2 * (JJ - 1) + 1]);
        elr(r3.Vpppp(q), np, II, JJ) = elr(r3.Vpppp(q), np, II, JJ) + X;
      }
    for (int JJ = 1; JJ <= nh; ++JJ)
      for (int II = 1; II <= np; ++II) {
        double X = ph(b.qnpp[2 * (II - 1)], b.qnpp[2 * (II - 1) + 1], b.qnhh[2 * (JJ - 1)], b.qnhh[2 * (JJ - 1) + 1]);
        elr(r3.Vpphh(q), np, II, JJ) = elr(r3.Vpphh(q), np, II, JJ) + X;
      }
    for (int JJ = 1; JJ <= nb; ++JJ)
      for (int II = 1; II <= np; ++II) {
        double X = ph(b.qnpp[2 * (II - 1)], b.qnpp[2 * (II - 1) + 1], b.qnph[2 * (JJ - 1) + 1], b.qnph[2 * (JJ - 1)]);
        elr(r3.Vppph(q), np, II, JJ) = elr(r3.Vppph(q), np, II, JJ) + X * -1;
      }
    for (int JJ = 1; JJ <= nh; ++JJ)
      for (int II = 1; II <= nb; ++II) {
        double X = ph(b.qnph[2 * (II - 1) + 1], b.qnph[2 * (II - 1)], b.qnhh[2 * (JJ - 1)], b.qnhh[2 * (JJ - 1) + 1]);
        elr(r3.Vphhh(q), nb, II, JJ) = elr(r3.Vphhh(q), nb, II, JJ) + X * -1;
      }
    for (int JJ = 1; JJ <= nb; ++JJ)
      for (int II = 1; II <= nb; ++II) {
        double X = ph(b.qnph[2 * (II - 1) + 1], b.qnph[2 * (II - 1)], b.qnph[2 * (JJ - 1) + 1], b.qnph[2 * (JJ - 1)]);
        elr(r3.Vphph(q), nb, II, JJ) = elr(r3.Vphph(q), nb, II, JJ) + X;
      }
  }
}

// build_white, IMSRG_tools.f90:377-434
void build_white(Op& gen, Op& rec) {
  const Layout& L = *rec.L;
  int n = L.n, m = L.m;
  for (int a = n + 1; a <= m; ++a)
    for (int i = 1; i <= n; ++i)
      gen.fph(a - n, i) = rec.fph(a - n, i) / (rec.fpp(a - n, a - n) - rec.fhh(i, i) - v_elem(a, i, a, i, rec));
  for (int q = 1; q <= L.nblock; ++q) {
    const Blk& b = L.blk[q - 1];
    if (b.npp * b.nhh == 0) continue;
    for (int i = 1; i <= b.npp; ++i)
      for (int j = 1; j <= b.nhh; ++j) {
        int p1 = b.qnpp[2 * (i - 1)], p2 = b.qnpp[2 * (i - 1) + 1];
        int hh1 = b.qnhh[2 * (j - 1)], hh2 = b.qnhh[2 * (j - 1) + 1];
        double efs = rec.fpp(p1 - n, p1 - n);
        efs = efs + rec.fpp(p2 - n, p2 - n);
        efs = efs - rec.fhh(hh1, hh1);
        efs = efs - rec.fhh(hh2, hh2);
        double Aph = v_elem(p1, p2, p1, p2, rec) + v_elem(hh1, hh2, hh1, hh2, rec) - v_elem(p1, hh1, p1, hh1, rec) -
                     v_elem(p1, hh2, p1, hh2, rec) - v_elem(p2, hh1, p2, hh1, rec) - v_elem(p2, hh2, p2, hh2, rec);
        elr(gen.Vpphh(q), b.npp, i, j) = el(rec.Vpphh(q), b.npp, i, j) / (efs + Aph);
      }
  }
}

// MBPT2, HFQDmod.f90:325-362
double MBPT2(Op& rec) {
  const Layout& L = *rec.L;
  int N = L.n;
  double sm = 0.0;
  for (int i = 1; i <= L.nblock; ++i) {
    const Blk& b = L.blk[i - 1];
    for (int II = 1; II <= b.npp; ++II) {
      int p1 = b.qnpp[2 * (II - 1)], p2 = b.qnpp[2 * (II - 1) + 1];
      double f12 = rec.fpp(p1 - N, p1 - N) + rec.fpp(p2 - N, p2 - N);
      for (int JJ = 1; JJ <= b.nhh; ++JJ) {
        int hh1 = b.qnhh[2 * (JJ - 1)], hh2 = b.qnhh[2 * (JJ - 1) + 1];
        double denom = rec.fhh(hh1, hh1) + rec.fhh(hh2, hh2) - f12;
        double x = el(rec.Vpphh(i), b.npp, II, JJ);
        sm = sm + x * x / denom;
      }
    }
  }
  return sm;
}

// HF_E2, HFQDmod.f90:292-323 (sets E0 as a side effect)
double HF_E2(Op& rec) {
  const Layout& L = *rec.L;
  double sm = 0.0, sm2 = 0.0;
  for (int i = 1; i <= L.nblock; ++i) {
    const Blk& b = L.blk[i - 1];
    for (int j = 1; j <= b.nhh; ++j) sm = sm + el(rec.Vhhhh(i), b.nhh, j, j);
  }
  for (int i = 1; i <= L.n; ++i) sm2 = sm2 + L.eig[i - 1];
  rec.E0() = sm2 - sm;
  return sm2 - sm;
}

// The sequence of one commutator [r1,r2] -> r3 as in BCH_EXPAND
// (magnus_IMSRG.f90:297-311) and dGam (gs_IMSRG.f90:256-268).
void full_commutator(Op& A, Op& B, Op& C, Op& w1, Op& w2, CC& ACC, CC& BCC) {
  const Layout& L = *A.L;
  set_to_zero(C);
  double ex = commutator_110(L.m - L.n, L.n, A, B);
  double ex2 = commutator_220(A, B);
  C.E0() = ex + ex2;
  commutator_111(A, B, C);
  commutator_121(A, B, C);
  commutator_221(A, B, C, w1, w2);
  set_to_zero(w1);
  commutator_122(A, B, C, false);
  commutator_222(A, B, C, w1, BCC, ACC);
}

// A bounded sample of one commutator for timing the CPU baseline: phase 0
// computes E0 and the one-body parts (110, 220, 111, 121, 221); every phase
// computes the two-body parts (122, ladders, particle-hole gather) of the
// blocks q with (q-1) % stride == phase and the cross-coupled products of the
// cross-coupled blocks with the same rule.  Phases 0..stride-1 together do
// the work of one whole commutator once.
void sampled_commutator(Op& A, Op& B, Op& C, Op& w1, Op& w2, CC& ACC, CC& BCC, int stride, int phase) {
  const Layout& L = *A.L;
  if (phase == 0) {
    double ex = commutator_110(L.m - L.n, L.n, A, B);
    double ex2 = commutator_220(A, B);
    C.E0() = ex + ex2;
    commutator_111(A, B, C);
    commutator_121(A, B, C);
    commutator_221(A, B, C, w1, w2);
  }
  // 122 on the selected blocks
  std::vector<int> hu, pu;
#pragma omp parallel for schedule(dynamic, 1) private(hu, pu)
  for (int q = 1 + phase; q <= L.nblock; q += stride) {
    const Blk& b = L.blk[q - 1];
    auto run = [&](int b1, int b2, int k1, int k2, int pre, double& out) {
      bool has_pre = pre != 0;
      union_groups(L, b1, b2, k1, k2, hu, pu);
      c122_elem(A, B, b1, b2, k1, k2, has_pre ? pre : 1, has_pre, out, hu, pu);
    };
    auto P = [&](const std::vector<int>& v, int k, int c) { return v[2 * (k - 1) + c]; };
    int nh = b.nhh, np = b.npp, nb = b.nph;
    for (int JJ = 1; JJ <= nh; ++JJ)
      for (int II = 1; II <= nh; ++II) run(P(b.qnhh, II, 0), P(b.qnhh, II, 1), P(b.qnhh, JJ, 0), P(b.qnhh, JJ, 1), 0, elr(C.Vhhhh(q), nh, II, JJ));
    for (int JJ = 1; JJ <= np; ++JJ)
      for (int II = 1; II <= np; ++II) run(P(b.qnpp, II, 0), P(b.qnpp, II, 1), P(b.qnpp, JJ, 0), P(b.qnpp, JJ, 1), 0, elr(C.Vpppp(q), np, II, JJ));
    for (int JJ = 1; JJ <= nh; ++JJ)
      for (int II = 1; II <= np; ++II) run(P(b.qnpp, II, 0), P(b.qnpp, II, 1), P(b.qnhh, JJ, 0), P(b.qnhh, JJ, 1), 0, elr(C.Vpphh(q), np, II, JJ));
    for (int JJ = 1; JJ <= nh; ++JJ)
      for (int II = 1; II <= nb; ++II) run(P(b.qnph, II, 1), P(b.qnph, II, 0), P(b.qnhh, JJ, 0), P(b.qnhh, JJ, 1), -1, elr(C.Vphhh(q), nb, II, JJ));
    for (int JJ = 1; JJ <= nb; ++JJ)
      for (int II = 1; II <= np; ++II) run(P(b.qnpp, II, 0), P(b.qnpp, II, 1), P(b.qnph, JJ, 1), P(b.qnph, JJ, 0), -1, elr(C.Vppph(q), np, II, JJ));
    for (int JJ = 1; JJ <= nb; ++JJ)
      for (int II = 1; II <= nb; ++II) run(P(b.qnph, II, 1), P(b.qnph, II, 0), P(b.qnph, JJ, 1), P(b.qnph, JJ, 0), 1, elr(C.Vphph(q), nb, II, JJ));
  }
  // cross-coupled products of the selected cc blocks (none when the X are
  // known to be zero, as commutator_222 skips them: the ph terms add zeros)
  const bool have_cc = !(ACC.zero && BCC.zero);
  std::vector<double> XCC(have_cc ? L.x2size : 0, 0.0), YCC(have_cc ? L.x2size : 0, 0.0);
  for (int q = 1 + phase; have_cc && q <= L.ccn; q += stride) {
    const CCBlk& c = L.cc[q - 1];
    if (c.r == 0 || c.nb == 0) continue;
    dgemm('N', 'T', c.r, c.r, c.nb, BCC.herm, &ACC.X[c.off], c.r, &BCC.X[c.off], c.r, 0.0, &XCC[c.off2], c.r);
    dgemm('N', 'T', c.r, c.r, c.nb, ACC.herm, &BCC.X[c.off], c.r, &ACC.X[c.off], c.r, 0.0, &YCC[c.off2], c.r);
  }
  // ladders + particle-hole gather of the selected blocks
  const int M = L.m;
  auto mp = [&](int x, int y, int& q, int& r) {
    i64 k = (i64)M * (x - 1) + y - 1;
    q = L.ccmap[2 * k];
    r = L.ccmap[2 * k + 1];
  };
  auto XC = [&](const std::vector<double>& Z, int q, int ra, int rb) {
    const CCBlk& c = L.cc[q - 1];
    return Z[c.off2 + (ra - 1) + (i64)(rb - 1) * c.r];
  };
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 1 + phase; q <= L.nblock; q += stride) {
    const Blk& b = L.blk[q - 1];
    matrix_mult222(A, B, C, w1, q, b.nhh, b.npp, b.nph);
    if (!have_cc) continue;
    auto ph = [&](int b1, int b2, int k1, int k2) {
      int q31, r31, q24, r24, q32, r32, q14, r14, q41, r41, q23, r23, q42, r42, q13, r13;
      mp(k1, b1, q31, r31); mp(b2, k2, q24, r24);
      mp(k1, b2, q32, r32); mp(b1, k2, q14, r14);
      mp(k2, b1, q41, r41); mp(b2, k1, q23, r23);
      mp(k2, b2, q42, r42); mp(b1, k1, q13, r13);
      double X = XC(XCC, q31, r31, r24) - XC(XCC, q32, r32, r14) + XC(XCC, q42, r42, r13) - XC(XCC, q41, r41, r23);
      X = X - XC(YCC, q42, r42, r13) + XC(YCC, q41, r41, r23) - XC(YCC, q31, r31, r24) + XC(YCC, q32, r32, r14);
      return X;
    };
    auto P = [&](const std::vector<int>& v, int k, int c) { return v[2 * (k - 1) + c]; };
    int nh = b.nhh, np = b.npp, nb = b.nph;
    for (int JJ = 1; JJ <= nh; ++JJ)
      for (int II = 1; II <= nh; ++II) elr(C.Vhhhh(q), nh, II, JJ) += ph(P(b.qnhh, II, 0), P(b.qnhh, II, 1), P(b.qnhh, JJ, 0), P(b.qnhh, JJ, 1));
    for (int JJ = 1; JJ <= np; ++JJ)
      for (int II = 1; II <= np; ++II) elr(C.Vpppp(q), np, II, JJ) += ph(P(b.qnpp, II, 0), P(b.qnpp, II, 1), P(b.qnpp, JJ, 0), P(b.qnpp, JJ, 1));
    for (int JJ = 1; JJ <= nh; ++JJ)
      for (int II = 1; II <= np; ++II) elr(C.Vpphh(q), np, II, JJ) += ph(P(b.qnpp, II, 0), P(b.qnpp, II, 1), P(b.qnhh, JJ, 0), P(b.qnhh, JJ, 1));
    for (int JJ = 1; JJ <= nb; ++JJ)
      for (int II = 1; II <= np; ++II) elr(C.Vppph(q), np, II, JJ) += -ph(P(b.qnpp, II, 0), P(b.qnpp, II, 1), P(b.qnph, JJ, 1), P(b.qnph, JJ, 0));
    for (int JJ = 1; JJ <= nh; ++JJ)
      for (int II = 1; II <= nb; ++II) elr(C.Vphhh(q), nb, II, JJ) += -ph(P(b.qnph, II, 1), P(b.qnph, II, 0), P(b.qnhh, JJ, 0), P(b.qnhh, JJ, 1));
    for (int JJ = 1; JJ <= nb; ++JJ)
      for (int II = 1; II <= nb; ++II) elr(C.Vphph(q), nb, II, JJ) += ph(P(b.qnph, II, 1), P(b.qnph, II, 0), P(b.qnph, JJ, 1), P(b.qnph, JJ, 0));
  }
}

struct Sampler {
  Op w1, w2;
  CC a, b;
  explicit Sampler(const Layout* l) : w1(l, 1), w2(l, 1), a(l), b(l) {}
};

// BCH_EXPAND, magnus_IMSRG.f90:253-318.  Returns the number of commutators.
// flags bit 0: calc_cc on G and AD before every commutator_222 (run_magnus
//              never fills the cross-coupled X, so without it the ph channel
//              is absent, as in the reference);
int BCH_EXPAND(Op& HS, Op& G, Op& H, Op& INT1, Op& INT2, Op& AD, Op& w1, Op& w2, CC& HCC, CC& OCC, int flags) {
  const int pandya = flags & 1;
  const double conv = 1e-5;
  const double cof[11] = {1.0, 0.5, 0.166666666666666666, 0.04166666666666666, 0.0083333333333333333,
                          .001388888888888, 1.984126984e-4, 2.48015873e-5, 2.755731922e-6, 2.755731922e-7,
                          2.505210839e-8};
  // Fortran single-precision literal: "conv = 1e-5" is real(4) converted to real(8)
  const double convd = (double)(float)conv;
  const Layout& L = *H.L;
  int m = L.m, n = L.n;
  INT2.herm = 1;
  INT1.herm = 1;
  AD.herm = 1;
  copy_arrays(H, HS);
  copy_arrays(HS, INT2);
  int count = 0;
  for (int i = 2; i <= 12; ++i) {
    copy_arrays(HS, INT1);
    copy_arrays(INT2, AD);
    set_to_zero(INT2);
    double ex = commutator_110(m - n, n, G, AD);
    double ex2 = commutator_220(G, AD);
    INT2.E0() = ex + ex2;
    commutator_111(G, AD, INT2);
    commutator_121(G, AD, INT2);
    commutator_221(G, AD, INT2, w1, w2);
    set_to_zero(w1);
    commutator_122(G, AD, INT2, false);
    if (pandya) {
      calc_cc(G, OCC);
      OCC.herm = G.herm;
      calc_cc(AD, HCC);
      HCC.herm = AD.herm;
    }
    commutator_222(G, AD, INT2, w1, HCC, OCC);
    ++count;
    add_arrays(INT1, 1.0, INT2, cof[i - 2], HS);
    if (mat_2_norm(INT2) * cof[i - 2] / mat_2_norm(INT1) < convd) break;
  }
  return count;
}

}  // namespace

// ===========================================================================
// C ABI for the Python test harness
// ===========================================================================
extern "C" {

void orc_set_threads(int t) {
#ifdef _OPENMP
  if (t > 0) omp_set_num_threads(t);
#else
  (void)t;
#endif
}

int orc_get_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// eig == NULL: oscillator energies 2n+|ml|+1 (calc_h0, ME_general.f90:800-821)
void* orc_layout_new(int n, int emax, const double* eig, int* err) {
  Layout* L = new Layout();
  L->n = n;
  L->emax = emax;
  L->m = emax * (emax + 1);
  arrange_states(emax, L->qn);
  L->eig.resize(L->m);
  for (int s = 1; s <= L->m; ++s)
    L->eig[s - 1] = eig ? eig[s - 1] : (double)(2 * L->QN(s, 1) + std::abs(L->QN(s, 2)) + 1);
  if (!reindex(*L)) {
    if (err) *err = 1;
    delete L;
    return nullptr;
  }
  offsets(*L);
  build_cross_coupled(*L);
  build_groups(*L);
  if (err) *err = 0;
  return L;
}
void orc_layout_free(void* h) { delete (Layout*)h; }
i64 orc_layout_neq(void* h) { return ((Layout*)h)->neq; }
int orc_layout_nblock(void* h) { return ((Layout*)h)->nblock; }
int orc_layout_msp(void* h) { return ((Layout*)h)->m; }
int orc_layout_ccn(void* h) { return ((Layout*)h)->ccn; }
void orc_layout_qn(void* h, int* out) { std::memcpy(out, ((Layout*)h)->qn.data(), sizeof(int) * ((Layout*)h)->qn.size()); }
void orc_layout_blocks(void* h, int* dims /* nblock x 6: nhh,nph,npp,ML,MS,ntot */, i64* offs /* nblock x 6 */) {
  Layout* L = (Layout*)h;
  for (int q = 0; q < L->nblock; ++q) {
    const Blk& b = L->blk[q];
    int* d = dims + 6 * q;
    d[0] = b.nhh; d[1] = b.nph; d[2] = b.npp; d[3] = b.lam[0]; d[4] = b.lam[1]; d[5] = b.ntot;
    if (offs) {
      i64* o = offs + 6 * q;
      o[0] = b.o_hhhh; o[1] = b.o_pppp; o[2] = b.o_pphh; o[3] = b.o_phph; o[4] = b.o_ppph; o[5] = b.o_phhh;
    }
  }
}
// pair lists of block q (1-based): kind 0=hh,1=ph,2=pp
int orc_layout_pairs(void* h, int q, int kind, int* out) {
  Layout* L = (Layout*)h;
  const Blk& b = L->blk[q - 1];
  const std::vector<int>& v = kind == 0 ? b.qnhh : (kind == 1 ? b.qnph : b.qnpp);
  std::memcpy(out, v.data(), sizeof(int) * v.size());
  return (int)v.size() / 2;
}
void orc_layout_i_array(void* h, int* out) {
  Layout* L = (Layout*)h;
  std::memcpy(out, L->i_array.data(), sizeof(int) * L->i_array.size());
}
void orc_layout_cc(void* h, int* r, int* nb) {
  Layout* L = (Layout*)h;
  for (int q = 0; q < L->ccn; ++q) { r[q] = L->cc[q].r; nb[q] = L->cc[q].nb; }
}
void orc_layout_ccmap(void* h, int* out) {
  Layout* L = (Layout*)h;
  std::memcpy(out, L->ccmap.data(), sizeof(int) * L->ccmap.size());
}

void* orc_op_new(void* L, int herm) { return new Op((Layout*)L, herm); }
void orc_op_free(void* o) { delete (Op*)o; }
void orc_op_set(void* o, const double* v) { Op* p = (Op*)o; std::memcpy(p->v.data(), v, sizeof(double) * p->v.size()); }
void orc_op_get(void* o, double* v) { Op* p = (Op*)o; std::memcpy(v, p->v.data(), sizeof(double) * p->v.size()); }
void orc_op_set_herm(void* o, int h) { ((Op*)o)->herm = h; }
int orc_op_get_herm(void* o) { return ((Op*)o)->herm; }

void* orc_cc_new(void* L) { return new CC((Layout*)L); }
void orc_cc_free(void* c) { delete (CC*)c; }
void orc_cc_set_herm(void* c, double h) { ((CC*)c)->herm = h; }
void orc_calc_cc(void* op, void* cc) { calc_cc(*(Op*)op, *(CC*)cc); }
void orc_cc_get_X(void* c, double* out) { CC* p = (CC*)c; std::memcpy(out, p->X.data(), sizeof(double) * p->X.size()); }
i64 orc_cc_xsize(void* c) { return (i64)((CC*)c)->X.size(); }

double orc_v_elem(int a, int b, int c, int d, void* op) { return v_elem(a, b, c, d, *(Op*)op); }

double orc_commutator_110(void* r1, void* r2) {
  Op* a = (Op*)r1;
  return commutator_110(a->L->m - a->L->n, a->L->n, *a, *(Op*)r2);
}
double orc_commutator_220(void* r1, void* r2) { return commutator_220(*(Op*)r1, *(Op*)r2); }
void orc_commutator_111(void* r1, void* r2, void* r3) { commutator_111(*(Op*)r1, *(Op*)r2, *(Op*)r3); }
void orc_commutator_121(void* r1, void* r2, void* r3) { commutator_121(*(Op*)r1, *(Op*)r2, *(Op*)r3); }
void orc_commutator_221(void* r1, void* r2, void* r3, void* w1, void* w2) {
  commutator_221(*(Op*)r1, *(Op*)r2, *(Op*)r3, *(Op*)w1, *(Op*)w2);
}
void orc_commutator_122(void* r1, void* r2, void* r3, int literal) {
  commutator_122(*(Op*)r1, *(Op*)r2, *(Op*)r3, literal != 0);
}
void orc_commutator_222(void* r1, void* r2, void* r3, void* w1, void* hcc, void* etacc) {
  commutator_222(*(Op*)r1, *(Op*)r2, *(Op*)r3, *(Op*)w1, *(CC*)hcc, *(CC*)etacc);
}

// Whole commutator C = [A,B]; pandya != 0 fills the cross-coupled matrices
// of both operators first (as dGam does, gs_IMSRG.f90:243-250).
void orc_commutator(void* A, void* B, void* C, int pandya) {
  Op& a = *(Op*)A;
  const Layout* L = a.L;
  Op w1(L, 1), w2(L, 1);
  CC acc(L), bcc(L);
  if (pandya) {
    calc_cc(a, acc);
    acc.herm = a.herm;
    calc_cc(*(Op*)B, bcc);
    bcc.herm = ((Op*)B)->herm;
  }
  full_commutator(a, *(Op*)B, *(Op*)C, w1, w2, acc, bcc);
}

// Use a Fortran-ABI dgemm from a shared library (e.g. scipy's OpenBLAS).
// Returns 1 on success, 0 if the library or symbol is unavailable.
int orc_use_blas(const char* path, const char* dgemm_sym, const char* threads_sym) {
  if (!path) {
    g_blas_dgemm = nullptr;
    g_blas_threads_local = nullptr;
    return 1;
  }
  void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return 0;
  void* f = dlsym(h, dgemm_sym);
  if (!f) return 0;
  g_blas_dgemm = (fdgemm_t)f;
  g_blas_threads_local = threads_sym ? (fsetthreads_t)dlsym(h, threads_sym) : nullptr;
  return 1;
}

// Bounded sample of [A,B] (see sampled_commutator); cross-coupled matrices of
// both operators are filled on phase 0 and reused by later phases.
void* orc_sampler_new(void* A) { return new Sampler(((Op*)A)->L); }
void orc_commutator_sample(void* sampler, void* A, void* B, void* C, int stride, int phase, int pandya) {
  Sampler* s = (Sampler*)sampler;
  Op& a = *(Op*)A;
  Op& b = *(Op*)B;
  if (phase == 0 && pandya) {
    calc_cc(a, s->a);
    s->a.herm = a.herm;
    calc_cc(b, s->b);
    s->b.herm = b.herm;
  }
  sampled_commutator(a, b, *(Op*)C, s->w1, s->w2, s->a, s->b, stride, phase);
}
void orc_sampler_free(void* sampler) { delete (Sampler*)sampler; }

void orc_build_white(void* gen, void* rec) { build_white(*(Op*)gen, *(Op*)rec); }
void orc_add_arrays(void* r1, double s1, void* r2, double s2, void* r3) {
  add_arrays(*(Op*)r1, s1, *(Op*)r2, s2, *(Op*)r3);
}
void orc_copy_arrays(void* r1, void* r2) { copy_arrays(*(Op*)r1, *(Op*)r2); }
void orc_set_to_zero(void* r1) { set_to_zero(*(Op*)r1); }
double orc_mat_2_norm(void* r) { return mat_2_norm(*(Op*)r); }
double orc_mbpt2(void* r) { return MBPT2(*(Op*)r); }
double orc_hf_e2(void* r) { return HF_E2(*(Op*)r); }

int orc_bch_expand(void* HS, void* G, void* H, int flags) {
  Op& h = *(Op*)H;
  const Layout* L = h.L;
  Op INT1(L, 1), INT2(L, 1), AD(L, 1), w1(L, 1), w2(L, 1);
  CC hcc(L), occ(L);
  hcc.herm = 1.0;
  occ.herm = -1.0;
  return BCH_EXPAND(*(Op*)HS, *(Op*)G, h, INT1, INT2, AD, w1, w2, hcc, occ, flags);
}

// s_evolve with build_white, magnus_IMSRG.f90:194-248 (TDA/spectrum
// diagnostics omitted; they do not feed back into the flow).  HAM is the
// normal-ordered HF Hamiltonian (herm=+1), HS receives the evolved one.
// flags as BCH_EXPAND.
// trace: per accepted-or-rejected iteration, 7 doubles:
//   iteration, s, E0, nrm1, nrm2, crit, bch_terms (negative when rejected)
// Returns the number of trace rows written, or -1 if max_iter was reached.
int orc_magnus_flow(void* HAMp, void* HSp, int flags, int max_iter, double* trace, double* s_out) {
  const double conv_criteria = (double)1e-9f;  // Fortran real(4) literal 1e-9
  Op& HAM = *(Op*)HAMp;
  Op& HS = *(Op*)HSp;
  const Layout* L = HAM.L;
  Op ETA(L, -1), G(L, -1), DG(L, -1), ETA0(L, -1), G0(L, -1), HS0(L, 1);
  Op INT1(L, 1), INT2(L, 1), AD(L, 1), w1(L, 1), w2(L, 1);
  CC HCC(L), OCC(L);
  HCC.herm = 1.0;
  OCC.herm = -1.0;
  double s = 0.0, stp = (double)0.7f;  // "stp=.7" is a real(4) literal
  copy_arrays(HAM, HS);
  HS.herm = 1;
  build_white(ETA, HS);
  double nrm1 = mat_2_norm(ETA);
  double crit = std::fabs(MBPT2(HAM));
  int iteration = 0, rows = 0, loops = 0;
  while (crit > conv_criteria) {
    if (loops++ >= max_iter) return -1;
    copy_arrays(G, G0);
    copy_arrays(ETA, DG);  // MAGNUS_EXPAND returns after DG = ETA (magnus_IMSRG.f90:342-345)
    add_arrays(G, 1.0, DG, stp, G);
    s = s + stp;
    copy_arrays(HS, HS0);
    int terms = BCH_EXPAND(HS, G, HAM, INT1, INT2, AD, w1, w2, HCC, OCC, flags);
    copy_arrays(ETA, ETA0);
    build_white(ETA, HS);
    double nrm2 = mat_2_norm(ETA);
    double* t = trace + 7 * rows;
    t[0] = iteration; t[1] = s; t[2] = HS.E0(); t[3] = nrm1; t[4] = nrm2; t[5] = crit; t[6] = terms;
    ++rows;
    if (nrm1 * 1.5 < nrm2) {
      t[6] = -terms;
      s = s - stp;
      copy_arrays(G0, G);
      copy_arrays(HS0, HS);
      copy_arrays(ETA0, ETA);
      stp = stp / 2.0 + (double)1e-3f;
      continue;
    }
    crit = std::fabs(MBPT2(HS));
    iteration = iteration + 1;
  }
  if (s_out) *s_out = s;
  return rows;
}

}  // extern "C"
