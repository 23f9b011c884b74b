// eom.cu -- EOM-IMSRG matrix-vector product for any (M_L, M_S) target.
//
// matvec_prod (src/EOM_IMSRG.f90:551-649) maps the Lanczos vector v to
// w = the 1p1h and 2p2h entries of [H, Q(v)] that carry the target's
// (M_L, M_S), through HQ_comm_1b / HQ_comm_2b (src/commutators.f90:1162-1272).
// A target other than (0, 0) connects different (M_L, M_S) blocks, so the
// excitation operator does not fit the scalar block layout; it gets its own
// device form here:
//   * 1p1h amplitudes: a dense m_p x n array Qf (Qf_elem,
//     src/ME_general.f90:1835-1870: only particle-hole entries);
//   * 2p2h amplitudes: per bra block q (particle pairs of (M_L, M_S)_q) the
//     column-major matrix Qb[q] of npp(q) x nhh(q'), q' the block of
//     (M_L, M_S)_q minus the target (Q_elem, src/ME_general.f90:1170-1224,
//     reads the same antisymmetric entries with the same ordering signs).
//     The Qb hold exactly the vector's 2p2h entries: a permutation of the
//     reference's unwrap order (src/EOM_IMSRG.f90:815-884).
// One call:
//   k_eom_unwrap  v -> Qf, Qb (a scatter; Qf's other entries stay zero)
//   grouped GEMM  Wb[q] = Vpppp[q] Qb[q] + Qb[q] Vhhhh[q'] on the DMMA pipe:
//                 the c<d and k<l sums of HQ_comm_2b
//   k_eom_2b      w(2p2h) = Wb + the one-body, three-leg and particle-hole
//                 sums of HQ_comm_2b, one thread per entry
//   k_eom_1b      w(1p1h) = HQ_comm_1b, one CTA per entry
// Every sum runs only over the states where its factors can be non-zero:
// Q carries the target, V conserves (M_L, M_S), so each one-body index and
// each particle-hole partner lies in one (m_l, m_s) group, and the ladder
// partners of a pair are the pairs of one block.  Dropped terms are exact
// zeros (Q_elem / Qf_elem / V_elem return 0 there), so the result is the
// reference's up to the order of the additions.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "dev_common.cuh"

#define EOM_TRY(x)       \
  do {                   \
    int rc_ = (x);       \
    if (rc_) return rc_; \
  } while (0)

namespace qd {

struct EomDev {
  int tml, tms;             // target (M_L, M_S): Ml = m_l(a) - m_l(i), Ms = s(a) - s(i) with s = +-1
  int mlmax;                // largest |m_l| of a state
  const int* gof;           // (m_l, s) -> group, index (m_l + mlmax) * 2 + (s + 1) / 2; -1 none
  const int* ml;            // per state
  const int* ms;
  const int* partner;       // per block: the ket block of (M_L, M_S)_q - target, or -1
  const i64* qoff;          // per block: offset of Qb[q]
  const double* qf;         // m_p x n
  const double* qb;
};

namespace {

__device__ __forceinline__ int eom_grp(const EomDev& E, int ml, int ms) {
  if (ml < -E.mlmax || ml > E.mlmax || (ms != 1 && ms != -1)) return -1;
  return __ldg(&E.gof[(ml + E.mlmax) * 2 + ((ms + 1) >> 1)]);
}

// Q_elem(x, y, z, w) (0-based states): non-zero only for particles x != y
// and holes z != w whose pairs differ by the target.
__device__ __forceinline__ double eom_q(const DevLayout& L, const EomDev& E, int x, int y, int z, int w) {
  if (x < L.n || y < L.n || z >= L.n || w >= L.n || x == y || z == w) return 0.0;
  const int e1 = __ldg(&L.ptab[x * L.m + y]), e2 = __ldg(&L.ptab[z * L.m + w]);
  const int q1 = pt_blk(e1);
  if (__ldg(&E.partner[q1]) != pt_blk(e2)) return 0.0;
  const double v = E.qb[__ldg(&E.qoff[q1]) + pt_idx(e1) + (i64)pt_idx(e2) * __ldg(&L.blk[q1]).z];
  return (pt_swap(e1) ^ pt_swap(e2)) ? -v : v;
}

// Qf_elem(x, y): particle x, hole y
__device__ __forceinline__ double eom_qf(const DevLayout& L, const EomDev& E, int x, int y) {
  return (x >= L.n && y < L.n) ? E.qf[(x - L.n) + (i64)y * L.mp] : 0.0;
}

// f_elem(x, y) of H (src/ME_general.f90:1780-1813)
__device__ __forceinline__ double eom_f(const DevLayout& L, const double* __restrict__ H, double hh, int x, int y) {
  if (x < L.n) {
    if (y < L.n) return H[L.o_fhh + x + (i64)y * L.n];
    return H[L.o_fph + (y - L.n) + (i64)x * L.mp] * hh;
  }
  if (y < L.n) return H[L.o_fph + (x - L.n) + (i64)y * L.mp];
  return H[L.o_fpp + (x - L.n) + (i64)(y - L.n) * L.mp];
}

// members of group g: [*b, *e) into L.gmem; holes first (they are the
// lowest states of every group)
__device__ __forceinline__ void grp_range(const DevLayout& L, int g, int* b, int* e) {
  if (g < 0) {
    *b = *e = 0;
    return;
  }
  *b = __ldg(&L.gstart[g]);
  *e = __ldg(&L.gstart[g + 1]);
}

__global__ void k_eom_unwrap(const double* __restrict__ v, i64 n1, i64 n2, const int2* __restrict__ out1,
                             const int* __restrict__ pos2, int nb, int mp, double* __restrict__ qf,
                             double* __restrict__ qb) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n1) {
    const int2 o = out1[e];
    qf[(o.x - nb) + (i64)o.y * mp] = v[e];
  } else if (e < n1 + n2) {
    qb[pos2[e - n1]] = v[e];
  }
}

// HQ_comm_2b(a, b, i, j) (src/commutators.f90:1214-1272) minus its two ladder
// sums, plus those sums from Wb.  a < b particles, i < j holes (0-based).
__global__ void __launch_bounds__(128, 4) k_eom_2b(DevLayout L, EomDev E, const double* __restrict__ H, double hh,
                                                const int4* __restrict__ out2, const int* __restrict__ pos2, i64 n2,
                                                const double* __restrict__ wb, double* __restrict__ w) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n2) return;
  const int4 o = out2[e];
  const int a = o.x, b = o.y, i = o.z, j = o.w;
  const int la = __ldg(&E.ml[a]), lb = __ldg(&E.ml[b]), li = __ldg(&E.ml[i]), lj = __ldg(&E.ml[j]);
  const int sa = __ldg(&E.ms[a]), sb = __ldg(&E.ms[b]), si = __ldg(&E.ms[i]), sj = __ldg(&E.ms[j]);
  const int n = L.n;
  double sm = 0.0;
  int gb, ge;
  // 12 -> 2: f(a,c) Q(c,b,i,j) - f(b,c) Q(c,a,i,j), c particle
  grp_range(L, eom_grp(E, E.tml + li + lj - lb, E.tms + si + sj - sb), &gb, &ge);
  for (int t = gb; t < ge; ++t) {
    const int c = __ldg(&L.gmem[t]);
    if (c >= n) sm += eom_f(L, H, hh, a, c) * eom_q(L, E, c, b, i, j);
  }
  grp_range(L, eom_grp(E, E.tml + li + lj - la, E.tms + si + sj - sa), &gb, &ge);
  for (int t = gb; t < ge; ++t) {
    const int c = __ldg(&L.gmem[t]);
    if (c >= n) sm -= eom_f(L, H, hh, b, c) * eom_q(L, E, c, a, i, j);
  }
  //        Qf(c,i) V(a,b,c,j) - Qf(c,j) V(a,b,c,i)
  grp_range(L, eom_grp(E, li + E.tml, si + E.tms), &gb, &ge);
  for (int t = gb; t < ge; ++t) {
    const int c = __ldg(&L.gmem[t]);
    if (c >= n) sm += eom_qf(L, E, c, i) * dv_elem(L, H, hh, a, b, c, j);
  }
  grp_range(L, eom_grp(E, lj + E.tml, sj + E.tms), &gb, &ge);
  for (int t = gb; t < ge; ++t) {
    const int c = __ldg(&L.gmem[t]);
    if (c >= n) sm -= eom_qf(L, E, c, j) * dv_elem(L, H, hh, a, b, c, i);
  }
  //        -Q(a,b,k,j) f(k,i) + Q(a,b,k,i) f(k,j), k hole
  grp_range(L, eom_grp(E, la + lb - E.tml - lj, sa + sb - E.tms - sj), &gb, &ge);
  for (int t = gb; t < ge; ++t) {
    const int k = __ldg(&L.gmem[t]);
    if (k < n) sm -= eom_q(L, E, a, b, k, j) * eom_f(L, H, hh, k, i);
  }
  grp_range(L, eom_grp(E, la + lb - E.tml - li, sa + sb - E.tms - si), &gb, &ge);
  for (int t = gb; t < ge; ++t) {
    const int k = __ldg(&L.gmem[t]);
    if (k < n) sm += eom_q(L, E, a, b, k, i) * eom_f(L, H, hh, k, j);
  }
  //        -V(b,k,j,i) Qf(a,k) + V(a,k,j,i) Qf(b,k)
  grp_range(L, eom_grp(E, la - E.tml, sa - E.tms), &gb, &ge);
  for (int t = gb; t < ge; ++t) {
    const int k = __ldg(&L.gmem[t]);
    if (k < n) sm -= dv_elem(L, H, hh, b, k, j, i) * eom_qf(L, E, a, k);
  }
  grp_range(L, eom_grp(E, lb - E.tml, sb - E.tms), &gb, &ge);
  for (int t = gb; t < ge; ++t) {
    const int k = __ldg(&L.gmem[t]);
    if (k < n) sm += dv_elem(L, H, hh, a, k, j, i) * eom_qf(L, E, b, k);
  }
  // 22 -> 2, particle-hole: for each hole k the particle c of each term lies
  // in the group fixed by V's conservation
  for (int k = 0; k < n; ++k) {
    const int lk = __ldg(&E.ml[k]), sk = __ldg(&E.ms[k]);
    grp_range(L, eom_grp(E, lb + lk - li, sb + sk - si), &gb, &ge);
    for (int t = gb; t < ge; ++t) {
      const int c = __ldg(&L.gmem[t]);
      if (c >= n) sm -= dv_elem(L, H, hh, b, k, c, i) * eom_q(L, E, a, c, k, j);
    }
    grp_range(L, eom_grp(E, la + lk - li, sa + sk - si), &gb, &ge);
    for (int t = gb; t < ge; ++t) {
      const int c = __ldg(&L.gmem[t]);
      if (c >= n) sm += dv_elem(L, H, hh, a, k, c, i) * eom_q(L, E, b, c, k, j);
    }
    grp_range(L, eom_grp(E, lb + lk - lj, sb + sk - sj), &gb, &ge);
    for (int t = gb; t < ge; ++t) {
      const int c = __ldg(&L.gmem[t]);
      if (c >= n) sm += dv_elem(L, H, hh, b, k, c, j) * eom_q(L, E, a, c, k, i);
    }
    grp_range(L, eom_grp(E, la + lk - lj, sa + sk - sj), &gb, &ge);
    for (int t = gb; t < ge; ++t) {
      const int c = __ldg(&L.gmem[t]);
      if (c >= n) sm -= dv_elem(L, H, hh, a, k, c, j) * eom_q(L, E, b, c, k, i);
    }
  }
  w[e] = wb[pos2[e]] + sm;
}

constexpr int EOM1_THREADS = 128;

// HQ_comm_1b(a, i) (src/commutators.f90:1162-1211), one CTA per entry.
__global__ void __launch_bounds__(EOM1_THREADS, 4) k_eom_1b(DevLayout L, EomDev E, const double* __restrict__ H,
                                                         double hh, const int2* __restrict__ out1,
                                                         double* __restrict__ w) {
  __shared__ double red[EOM1_THREADS / 32];
  const int2 o = out1[blockIdx.x];
  const int a = o.x, i = o.y, n = L.n;
  const int la = __ldg(&E.ml[a]), li = __ldg(&E.ml[i]);
  const int sa = __ldg(&E.ms[a]), si = __ldg(&E.ms[i]);
  const int tid = threadIdx.x;
  double sm = 0.0;
  int gb, ge;
  // 11 -> 1: f(a,b) Qf(b,i) - Qf(a,j) f(j,i)
  grp_range(L, eom_grp(E, li + E.tml, si + E.tms), &gb, &ge);
  for (int t = gb + tid; t < ge; t += EOM1_THREADS) {
    const int b = __ldg(&L.gmem[t]);
    if (b >= n) sm += eom_f(L, H, hh, a, b) * eom_qf(L, E, b, i);
  }
  grp_range(L, eom_grp(E, la - E.tml, sa - E.tms), &gb, &ge);
  for (int t = gb + tid; t < ge; t += EOM1_THREADS) {
    const int j = __ldg(&L.gmem[t]);
    if (j < n) sm -= eom_qf(L, E, a, j) * eom_f(L, H, hh, j, i);
  }
  // 12 -> 1 and 21 -> 1, per hole j: f(j,b) Q(a,b,i,j) and Qf(b,j) V(a,j,i,b)
  for (int j = tid; j < n; j += EOM1_THREADS) {
    const int lj = __ldg(&E.ml[j]), sj = __ldg(&E.ms[j]);
    grp_range(L, eom_grp(E, E.tml + li + lj - la, E.tms + si + sj - sa), &gb, &ge);
    for (int t = gb; t < ge; ++t) {
      const int b = __ldg(&L.gmem[t]);
      if (b >= n) sm += eom_f(L, H, hh, j, b) * eom_q(L, E, a, b, i, j);
    }
    grp_range(L, eom_grp(E, lj + E.tml, sj + E.tms), &gb, &ge);
    for (int t = gb; t < ge; ++t) {
      const int b = __ldg(&L.gmem[t]);
      if (b >= n) sm += eom_qf(L, E, b, j) * dv_elem(L, H, hh, a, j, i, b);
    }
  }
  // 22 -> 1: sum over b < c particles and holes j of Q(c,b,i,j) V(a,j,c,b);
  // V is non-zero only for the particle pairs of the block of (a, j)
  for (int j = 0; j < n; ++j) {
    const int ep = __ldg(&L.ptab[a * L.m + j]);
    const int q = pt_blk(ep);
    const int npp = __ldg(&L.blk[q]).z;
    for (int k = tid; k < npp; k += EOM1_THREADS) {
      const int2 bc = block_pair(L, q, 2, k);  // b < c
      sm += eom_q(L, E, bc.y, bc.x, i, j) * dv_elem(L, H, hh, a, j, bc.y, bc.x);
    }
  }
  //          minus the sum over particles b and holes k < j of Q(a,b,k,j) V(k,j,i,b)
  for (int k = tid; k < n; k += EOM1_THREADS) {
    const int lk = __ldg(&E.ml[k]), sk = __ldg(&E.ms[k]);
    for (int j = k + 1; j < n; ++j) {
      const int lj = __ldg(&E.ml[j]), sj = __ldg(&E.ms[j]);
      grp_range(L, eom_grp(E, lk + lj - li, sk + sj - si), &gb, &ge);
      for (int t = gb; t < ge; ++t) {
        const int b = __ldg(&L.gmem[t]);
        if (b >= n) sm -= eom_q(L, E, a, b, k, j) * dv_elem(L, H, hh, k, j, i, b);
      }
    }
  }
  sm = block_sum<EOM1_THREADS>(sm, red);
  if (tid == 0) w[blockIdx.x] = sm;
}

}  // namespace

// Host tables of a target: the unwrap order of the 1p1h entries (particle
// outer, hole inner) and of the 2p2h entries (a < b outer, i < j inner), the
// position of each 2p2h entry in Qb, and the ket partner and offset of each
// bra block.
struct EomTables {
  std::vector<int2> out1;
  std::vector<int4> out2;
  std::vector<int> pos2;
  std::vector<int> partner;
  std::vector<i64> qoff;
  i64 nqb = 0;
};

static void eom_tables(const qd_layout* L, int tml, int tms, EomTables& T, bool counts_only, i64* n1, i64* n2) {
  const int n = L->n, m = L->m;
  auto ml = [&](int s) { return L->qn[3 * s + 1]; };
  auto ms = [&](int s) { return L->qn[3 * s + 2]; };
  // (M_L, M_S) of every non-empty block, from its first pair
  std::vector<std::pair<int, int>> bm(L->nblock, {0, 0});
  std::vector<bool> has(L->nblock, false);
  std::map<std::pair<int, int>, int> byM;
  for (int q = 0; q < L->nblock; ++q) {
    const int4 d = L->blk[q];
    if (d.x + d.y + d.z == 0) continue;
    const int2 p = L->pairs[L->pbase[q]];
    bm[q] = {ml(p.x) + ml(p.y), ms(p.x) + ms(p.y)};
    has[q] = true;
    byM[bm[q]] = q;
  }
  T.partner.assign(L->nblock, -1);
  T.qoff.assign(L->nblock, 0);
  i64 off = 0;
  for (int q = 0; q < L->nblock; ++q) {
    T.qoff[q] = off;
    if (!has[q] || L->blk[q].z == 0) continue;
    auto it = byM.find({bm[q].first - tml, bm[q].second - tms});
    if (it == byM.end() || L->blk[it->second].x == 0) continue;
    T.partner[q] = it->second;
    off += (i64)L->blk[q].z * L->blk[it->second].x;
  }
  T.nqb = off;
  i64 c1 = 0;
  for (int a = n; a < m; ++a)
    for (int i = 0; i < n; ++i)
      if (ml(a) - ml(i) == tml && ms(a) - ms(i) == tms) {
        if (!counts_only) T.out1.push_back(make_int2(a, i));
        ++c1;
      }
  i64 c2 = 0;
  for (int a = n; a < m; ++a)
    for (int b = a + 1; b < m; ++b)
      for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
          if (ml(a) + ml(b) - ml(i) - ml(j) != tml || ms(a) + ms(b) - ms(i) - ms(j) != tms) continue;
          if (!counts_only) {
            const int e1 = L->ptab[a * m + b], e2 = L->ptab[i * m + j];
            const int q1 = pt_blk(e1);
            T.out2.push_back(make_int4(a, b, i, j));
            T.pos2.push_back((int)(T.qoff[q1] + pt_idx(e1) + (i64)pt_idx(e2) * L->blk[q1].z));
          }
          ++c2;
        }
  *n1 = c1;
  *n2 = c2;
}

namespace {
struct EomPlan {
  i64 n1 = 0, n2 = 0;
  int2* d_out1 = nullptr;
  int4* d_out2 = nullptr;
  int* d_pos2 = nullptr;
  int* d_partner = nullptr;
  i64* d_qoff = nullptr;
  int* d_gof = nullptr;
  int* d_ml = nullptr;
  int* d_ms = nullptr;
  double* d_qf = nullptr;
  double* d_qb = nullptr;
  double* d_wb = nullptr;
  int mlmax = 0;
  GemmProgram prog;
  std::vector<void*> allocs;
  void free_all() {
    for (void* p : allocs) cudaFree(p);
    allocs.clear();
    prog.clear_device();
  }
};
std::map<std::tuple<const qd_layout*, int, int>, EomPlan>& eom_plans() {
  static std::map<std::tuple<const qd_layout*, int, int>, EomPlan> m;
  return m;
}
std::mutex g_eom_mutex;

template <typename T>
int eom_upload(EomPlan& p, T** dst, const T* src, size_t count) {
  *dst = nullptr;
  if (count == 0) return QD_OK;
  QD_CUDA(cudaMalloc((void**)dst, count * sizeof(T)));
  p.allocs.push_back(*dst);
  if (src) QD_CUDA(cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice));
  return QD_OK;
}

int eom_plan(qd_layout* L, int tml, int tms, EomPlan** out) {
  std::lock_guard<std::mutex> lock(g_eom_mutex);
  auto key = std::make_tuple((const qd_layout*)L, tml, tms);
  auto it = eom_plans().find(key);
  if (it != eom_plans().end()) {
    *out = &it->second;
    return QD_OK;
  }
  EomPlan p;
  EomTables T;
  eom_tables(L, tml, tms, T, false, &p.n1, &p.n2);
  if (p.n2 >= ((i64)1 << 31)) {
    set_error("qd_eom_matvec_target: %lld 2p2h entries exceed the 32-bit index range", (long long)p.n2);
    return QD_ERR_ARG;
  }
  const int m = L->m;
  std::vector<int> vml(m), vms(m);
  for (int s = 0; s < m; ++s) {
    vml[s] = L->qn[3 * s + 1];
    vms[s] = L->qn[3 * s + 2];
    p.mlmax = std::max(p.mlmax, std::abs(vml[s]));
  }
  std::vector<int> gof((2 * p.mlmax + 1) * 2, -1);
  for (int s = 0; s < m; ++s) gof[(vml[s] + p.mlmax) * 2 + ((vms[s] + 1) >> 1)] = L->gid[s];
  int rc = QD_OK;
  if (!rc) rc = eom_upload(p, &p.d_out1, T.out1.data(), T.out1.size());
  if (!rc) rc = eom_upload(p, &p.d_out2, T.out2.data(), T.out2.size());
  if (!rc) rc = eom_upload(p, &p.d_pos2, T.pos2.data(), T.pos2.size());
  if (!rc) rc = eom_upload(p, &p.d_partner, T.partner.data(), T.partner.size());
  if (!rc) rc = eom_upload(p, &p.d_qoff, T.qoff.data(), T.qoff.size());
  if (!rc) rc = eom_upload(p, &p.d_gof, gof.data(), gof.size());
  if (!rc) rc = eom_upload(p, &p.d_ml, vml.data(), vml.size());
  if (!rc) rc = eom_upload(p, &p.d_ms, vms.data(), vms.size());
  if (!rc) rc = eom_upload<double>(p, &p.d_qf, nullptr, (size_t)L->mp * L->n);
  if (!rc) rc = eom_upload<double>(p, &p.d_qb, nullptr, (size_t)T.nqb);
  if (!rc) rc = eom_upload<double>(p, &p.d_wb, nullptr, (size_t)T.nqb);
  if (!rc) rc = build_eom_ladders(L, T.partner, T.qoff, p.prog);
  if (rc) {
    p.free_all();
    return rc;
  }
  auto ins = eom_plans().emplace(key, std::move(p));
  *out = &ins.first->second;
  return QD_OK;
}
}  // namespace

void drop_eom_plans(const qd_layout* L) {
  std::lock_guard<std::mutex> lock(g_eom_mutex);
  for (auto it = eom_plans().begin(); it != eom_plans().end();) {
    if (std::get<0>(it->first) == L) {
      it->second.free_all();
      it = eom_plans().erase(it);
    } else {
      ++it;
    }
  }
}

}  // namespace qd

using namespace qd;

extern "C" int qd_eom_dim(const qd_layout* L, int ml, int ms, int64_t* n1, int64_t* n2) {
  if (!L || !n1 || !n2) {
    set_error("qd_eom_dim: null argument");
    return QD_ERR_ARG;
  }
  EomTables T;
  i64 a = 0, b = 0;
  eom_tables(L, ml, ms, T, true, &a, &b);
  *n1 = a;
  *n2 = b;
  return QD_OK;
}

extern "C" int qd_eom_matvec_target(const qd_op* H, int ml, int ms, const double* d_v, double* d_w, int64_t n) {
  if (!H || !d_v || !d_w) {
    set_error("qd_eom_matvec_target: null argument");
    return QD_ERR_ARG;
  }
  qd_layout* L = H->L;
  if (L->device == QD_HOST_ONLY) {
    set_error("layout was created host-only (QD_HOST_ONLY)");
    return QD_ERR_STATE;
  }
  QD_CUDA(cudaSetDevice(L->device));
  EomPlan* p;
  EOM_TRY(eom_plan(L, ml, ms, &p));
  if (n != p->n1 + p->n2) {
    set_error("qd_eom_matvec_target: vector length %lld, the target (%d, %d) has %lld + %lld entries", (long long)n,
              ml, ms, (long long)p->n1, (long long)p->n2);
    return QD_ERR_ARG;
  }
  if (n == 0) return QD_OK;
  const int n_ = L->n, mp = L->mp;
  cudaStream_t s = L->stream;
  if (p->n1 > 0) QD_CUDA(cudaMemsetAsync(p->d_qf, 0, sizeof(double) * mp * n_, s));
  const int T = 256;
  k_eom_unwrap<<<(unsigned)((n + T - 1) / T), T, 0, s>>>(d_v, p->n1, p->n2, p->d_out1, p->d_pos2, n_, mp, p->d_qf,
                                                          p->d_qb);
  ++L->nlaunch;
  EomDev E;
  E.tml = ml;
  E.tms = ms;
  E.mlmax = p->mlmax;
  E.gof = p->d_gof;
  E.ml = p->d_ml;
  E.ms = p->d_ms;
  E.partner = p->d_partner;
  E.qoff = p->d_qoff;
  E.qf = p->d_qf;
  E.qb = p->d_qb;
  const double hh = (double)H->herm;
  if (p->n2 > 0) {
    const double* bufs[NBUF] = {H->d, p->d_qb, nullptr, nullptr, p->d_wb, nullptr, nullptr};
    EOM_TRY(run_program_f64(L, p->prog, bufs, 1.0, 1.0, H->zero_mask, 0u));
    k_eom_2b<<<(unsigned)((p->n2 + 127) / 128), 128, 0, s>>>(L->dev, E, H->d, hh, p->d_out2, p->d_pos2, p->n2,
                                                             p->d_wb, d_w + p->n1);
    ++L->nlaunch;
  }
  if (p->n1 > 0) {
    k_eom_1b<<<(unsigned)p->n1, EOM1_THREADS, 0, s>>>(L->dev, E, H->d, hh, p->d_out1, d_w);
    ++L->nlaunch;
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}
