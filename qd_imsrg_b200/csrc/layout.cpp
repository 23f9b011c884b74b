// layout.cpp -- host construction of the (M_L,M_S)-blocked two-body layout.
//
// Follows the reference's index builders so that the flat operator array is
// byte-compatible with vectorize() of a Fortran full_ham:
//   arrange_states  src/ME_general.f90:688-716   (single-particle order)
//   reindex         src/ME_general.f90:956-1116  (blocks, pair classes, i_array)
//   build_cross_coupled src/ME_general.f90:363-448 (Pandya blocks and map)
//   get_num_elements    src/ME_general.f90:1755-1778
// States are 0-based here; pair lists handed out through the C ABI are 1-based.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "qd_internal.hpp"

namespace qd {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int cuda_fail(cudaError_t e, const char* what) {
  set_error("CUDA error %d (%s) in %s", (int)e, cudaGetErrorString(e), what);
  return e == cudaErrorMemoryAllocation ? QD_ERR_OOM : QD_ERR_CUDA;
}

const char* last_error() { return g_err; }

int layout_build(qd_layout* L, int nbody, int emax, const double* eig) {
  if (emax < 1 || nbody < 0) {
    set_error("qd_layout_create: bad sizes nbody=%d emax=%d", nbody, emax);
    return QD_ERR_ARG;
  }
  const int m = emax * (emax + 1);
  if (nbody > m) {
    set_error("qd_layout_create: nbody=%d exceeds %d states", nbody, m);
    return QD_ERR_ARG;
  }
  L->n = nbody;
  L->m = m;
  L->mp = m - nbody;
  L->emax = emax;
  // arrange_states: shells R, then ML = -R..R step 2, then MS = -1, +1
  L->qn.clear();
  for (int R = 0; R < emax; ++R)
    for (int ml = -R; ml <= R; ml += 2)
      for (int ms = -1; ms <= 1; ms += 2) {
        L->qn.push_back((R - std::abs(ml)) / 2);
        L->qn.push_back(ml);
        L->qn.push_back(ms);
      }
  L->eig.resize(m);
  for (int s = 0; s < m; ++s)
    L->eig[s] = eig ? eig[s] : (double)(2 * L->qn[3 * s] + std::abs(L->qn[3 * s + 1]) + 1);

  // Fermi level as in reindex: the N-th smallest energy (ties broken by the
  // lowest state index first) plus 1e-6.
  double eF = 0.0;
  if (nbody > 0) {
    std::vector<int> order(m);
    for (int s = 0; s < m; ++s) order[s] = s;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return L->eig[a] < L->eig[b]; });
    eF = L->eig[order[nbody - 1]] + 1.e-6;
  }
  std::vector<char> hole(m);
  for (int s = 0; s < m; ++s) {
    hole[s] = nbody > 0 && L->eig[s] <= eF;
    if ((bool)hole[s] != (s < nbody)) {
      set_error("qd_layout_create: the hole states (eig <= eF) are not states 1..%d", nbody);
      return QD_ERR_LAYOUT;
    }
  }

  // reindex: blocks MS in {-2,0,2} outer, ML in [2-2emax, 2emax-2] inner;
  // pairs a<b in loop order, classed hh/ph/pp, each class in loop order.
  L->nblock = 12 * emax - 9;
  L->blk.assign(L->nblock, int4{0, 0, 0, 0});
  L->pairs.clear();
  L->pbase.assign(L->nblock + 1, 0);
  L->ptab.assign((size_t)m * m, -1);
  int q = 0;
  for (int MS = -2; MS <= 2; MS += 2)
    for (int ML = 2 - 2 * emax; ML <= 2 * emax - 2; ++ML, ++q) {
      std::vector<int2> hh, ph, pp;
      for (int a = 0; a < m - 1; ++a)
        for (int b = a + 1; b < m; ++b) {
          if (L->qn[3 * a + 2] + L->qn[3 * b + 2] != MS) continue;
          if (L->qn[3 * a + 1] + L->qn[3 * b + 1] != ML) continue;
          int cls;
          if (hole[a] && hole[b]) {
            cls = 0;
            hh.push_back(int2{a, b});
          } else if (hole[a] || hole[b]) {
            cls = 1;
            ph.push_back(int2{a, b});
          } else {
            cls = 2;
            pp.push_back(int2{a, b});
          }
          int idx = cls == 0 ? (int)hh.size() - 1 : (cls == 1 ? (int)ph.size() - 1 : (int)pp.size() - 1);
          if (idx > 0x1FFF || q > 0x3FF) {
            set_error("qd_layout_create: basis too large for the pair table");
            return QD_ERR_ARG;
          }
          L->ptab[(size_t)a * m + b] = pt_pack(idx, q, cls, 0);
          L->ptab[(size_t)b * m + a] = pt_pack(idx, q, cls, 1);
        }
      L->blk[q] = int4{(int)hh.size(), (int)ph.size(), (int)pp.size(), (int)(hh.size() + ph.size() + pp.size())};
      L->pbase[q] = (int)L->pairs.size();
      L->pairs.insert(L->pairs.end(), hh.begin(), hh.end());
      L->pairs.insert(L->pairs.end(), ph.begin(), ph.end());
      L->pairs.insert(L->pairs.end(), pp.begin(), pp.end());
    }
  L->pbase[L->nblock] = (int)L->pairs.size();

  // vectorize offsets
  const int n = nbody, mp = m - nbody;
  i64 k = 1;
  L->o_fhh = k; k += (i64)n * n;
  L->o_fpp = k; k += (i64)mp * mp;
  L->o_fph = k; k += (i64)mp * n;
  L->boff.assign((size_t)6 * L->nblock, 0);
  for (int b = 0; b < L->nblock; ++b) {
    i64 nh = L->blk[b].x, nb = L->blk[b].y, np = L->blk[b].z;
    i64* o = &L->boff[6 * b];
    o[0] = k; k += nh * nh;  // Vhhhh
    o[1] = k; k += np * np;  // Vpppp
    o[2] = k; k += np * nh;  // Vpphh
    o[3] = k; k += nb * nb;  // Vphph
    o[4] = k; k += np * nb;  // Vppph
    o[5] = k; k += nb * nh;  // Vphhh
  }
  L->neq = k;

  // single-particle (ml,ms) groups
  L->gid.assign(m, -1);
  std::vector<std::pair<int, int>> keys;
  std::vector<std::vector<int>> mem;
  for (int s = 0; s < m; ++s) {
    std::pair<int, int> key(L->qn[3 * s + 1], L->qn[3 * s + 2]);
    int g = -1;
    for (size_t t = 0; t < keys.size(); ++t)
      if (keys[t] == key) g = (int)t;
    if (g < 0) {
      g = (int)keys.size();
      keys.push_back(key);
      mem.push_back({});
    }
    L->gid[s] = g;
    mem[g].push_back(s);
  }
  L->gstart.assign(keys.size() + 1, 0);
  L->gmem.clear();
  for (size_t g = 0; g < keys.size(); ++g) {
    L->gstart[g] = (int)L->gmem.size();
    L->gmem.insert(L->gmem.end(), mem[g].begin(), mem[g].end());
  }
  L->gstart[keys.size()] = (int)L->gmem.size();

  // build_cross_coupled: ML in [-MLmax, MLmax], MS in [-2, 2]; rows are all
  // ordered pairs (i,j) with ml_i-ml_j = ML, ms_i-ms_j = MS; columns are the
  // (hole i, particle j) pairs among them, in loop order.  The reference
  // orders the rows by (i, j); here they go by the (ml,ms) group of i first,
  // so that the rows (i in G1, j in G2) are one run and a product block
  // Z[(G1,G2),(G3,G4)] is a dense sub-matrix.  ccref keeps the reference
  // row of each row (for downloads).
  int mlmax_sp = 0;
  for (int s = 0; s < m; ++s) mlmax_sp = std::max(mlmax_sp, L->qn[3 * s + 1]);
  L->mlmax = 2 * mlmax_sp;
  L->ncc = 10 * L->mlmax + 5;
  L->ccmap.assign((size_t)m * m, int2{-1, -1});
  L->ccdim.assign(L->ncc, int2{0, 0});
  L->ccab.clear();
  L->ccref.clear();
  L->cchp.clear();
  L->ccab_base.assign(L->ncc + 1, 0);
  L->cchp_base.assign(L->ncc + 1, 0);
  L->ccxoff.assign(L->ncc, 0);
  L->cczoff.assign(L->ncc, 0);
  int cq = 0;
  i64 xo = 0, zo = 0;
  for (int ML = -L->mlmax; ML <= L->mlmax; ++ML)
    for (int MS = -2; MS <= 2; ++MS, ++cq) {
      L->ccab_base[cq] = (int)L->ccab.size();
      L->cchp_base[cq] = (int)L->cchp.size();
      int r = 0, nb = 0;
      // reference row of (i, j): position in the (i, j) loop order
      std::vector<int> refrow;
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
          if (L->qn[3 * i + 1] - L->qn[3 * j + 1] != ML) continue;
          if (L->qn[3 * i + 2] - L->qn[3 * j + 2] != MS) continue;
          refrow.push_back(i * m + j);
          if (i < n && j >= n) {
            L->cchp.push_back(int2{i, j});
            ++nb;
          }
        }
      std::vector<int> refpos((size_t)m * m, -1);
      for (size_t t = 0; t < refrow.size(); ++t) refpos[refrow[t]] = (int)t;
      for (size_t g = 0; g < keys.size(); ++g)
        for (int i : mem[g])
          for (int j = 0; j < m; ++j) {
            if (L->qn[3 * i + 1] - L->qn[3 * j + 1] != ML) continue;
            if (L->qn[3 * i + 2] - L->qn[3 * j + 2] != MS) continue;
            L->ccmap[(size_t)i * m + j] = int2{cq, r};
            L->ccab.push_back(int2{i, j});
            L->ccref.push_back(refpos[(size_t)i * m + j]);
            ++r;
          }
      L->ccdim[cq] = int2{r, nb};
      L->ccxoff[cq] = xo;
      L->cczoff[cq] = zo;
      xo += (i64)r * nb;
      zo += (i64)r * r;
    }
  L->ccab_base[L->ncc] = (int)L->ccab.size();
  L->cchp_base[L->ncc] = (int)L->cchp.size();
  L->xsize = xo;
  L->zsize = zo;

  // flat two-body sub-block index (vectorize order) and per-part numbering
  L->s2off.clear();
  L->s2id.clear();
  L->pcum.assign((size_t)6 * L->nblock, 0);
  i64 cnt[6] = {0, 0, 0, 0, 0, 0};
  // vectorize order within a block: hhhh, pppp, pphh, phph, ppph, phhh
  const int vec_part[6] = {P_HHHH, P_PPPP, P_PPHH, P_PHPH, P_PPPH, P_PHHH};
  for (int b = 0; b < L->nblock; ++b) {
    i64 nh = L->blk[b].x, nb = L->blk[b].y, np = L->blk[b].z;
    i64 sz[6] = {nh * nh, np * np, np * nh, nb * nb, np * nb, nb * nh};
    for (int t = 0; t < 6; ++t) {
      int p = vec_part[t] - P_HHHH;
      L->pcum[(size_t)p * L->nblock + b] = cnt[p];
      cnt[p] += sz[t];
      if (sz[t] > 0) {
        L->s2off.push_back(L->boff[6 * b + t]);
        L->s2id.push_back((b << 3) | p);
      }
    }
  }
  for (int p = 0; p < 6; ++p) L->dev.pcnt[p] = cnt[p];
  return QD_OK;
}

template <class T>
static int up(qd_layout* L, const std::vector<T>& v, const T** out) {
  size_t bytes = std::max<size_t>(1, v.size()) * sizeof(T);
  void* p = nullptr;
  QD_CUDA(cudaMalloc(&p, bytes));
  L->dev_allocs.push_back(p);
  if (!v.empty()) QD_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  *out = (const T*)p;
  return QD_OK;
}

int layout_upload(qd_layout* L) {
  DevLayout& D = L->dev;
  D.n = L->n;
  D.m = L->m;
  D.mp = L->mp;
  D.nblock = L->nblock;
  D.ncc = L->ncc;
  D.mlmax = L->mlmax;
  D.o_fhh = L->o_fhh;
  D.o_fpp = L->o_fpp;
  D.o_fph = L->o_fph;
  D.neq = L->neq;
  int rc;
  if ((rc = up(L, L->blk, &D.blk))) return rc;
  if ((rc = up(L, L->boff, &D.boff))) return rc;
  if ((rc = up(L, L->pairs, &D.pairs))) return rc;
  if ((rc = up(L, L->pbase, &D.pbase))) return rc;
  if ((rc = up(L, L->ptab, &D.ptab))) return rc;
  if ((rc = up(L, L->gid, &D.gid))) return rc;
  if ((rc = up(L, L->gstart, &D.gstart))) return rc;
  if ((rc = up(L, L->gmem, &D.gmem))) return rc;
  if ((rc = up(L, L->ccmap, &D.ccmap))) return rc;
  if ((rc = up(L, L->ccdim, &D.ccdim))) return rc;
  if ((rc = up(L, L->ccxoff, &D.ccxoff))) return rc;
  if ((rc = up(L, L->cczoff, &D.cczoff))) return rc;
  if ((rc = up(L, L->ccab, &D.ccab))) return rc;
  if ((rc = up(L, L->ccab_base, &D.ccab_base))) return rc;
  if ((rc = up(L, L->cchp, &D.cchp))) return rc;
  if ((rc = up(L, L->cchp_base, &D.cchp_base))) return rc;
  if ((rc = up(L, L->s2off, &D.s2off))) return rc;
  if ((rc = up(L, L->s2id, &D.s2id))) return rc;
  if ((rc = up(L, L->pcum, &D.pcum))) return rc;
  D.ns2 = (int)L->s2off.size();
  D.o2 = L->o_fph + (i64)L->mp * L->n;
  return QD_OK;
}

void GemmProgram::clear_device() {
  if (d_probs) cudaFree(d_probs);
  if (d_segs) cudaFree(d_segs);
  for (auto* m : {&tasks, &tasks_short})
    for (auto& kv : *m)
      if (kv.second.first) cudaFree(kv.second.first);
  d_probs = nullptr;
  d_segs = nullptr;
  tasks.clear();
  tasks_short.clear();
}

void layout_free_device(qd_layout* L) {
  for (void* p : L->dev_allocs) cudaFree(p);
  L->dev_allocs.clear();
  L->prog_ladder.clear_device();
  L->prog_221.clear_device();
  L->prog_111.clear_device();
  L->prog_pandya.clear_device();
  split_free(L);
  graphs_free(L);
  if (L->d_z) cudaFree(L->d_z);
  if (L->d_red) cudaFree(L->d_red);
  if (L->d_axn) cudaFree(L->d_axn);
  L->d_axn = nullptr;
  if (L->h_red) cudaFreeHost(L->h_red);
  L->d_z = nullptr;
  L->d_red = nullptr;
  L->h_red = nullptr;
  L->d_ccflag = nullptr;  // in dev_allocs
  L->d_tgt221 = nullptr;
  L->ntgt221 = -1;
  if (L->own_stream && L->stream) cudaStreamDestroy(L->stream);
  L->stream = nullptr;
}

i64 part_count(const qd_layout* L, int part) {
  i64 s = 0;
  for (int b = 0; b < L->nblock; ++b) {
    i64 nh = L->blk[b].x, nb = L->blk[b].y, np = L->blk[b].z;
    switch (part) {
      case P_HHHH: s += nh * nh; break;
      case P_PPPP: s += np * np; break;
      case P_PPHH: s += np * nh; break;
      case P_PHPH: s += nb * nb; break;
      case P_PPPH: s += np * nb; break;
      case P_PHHH: s += nb * nh; break;
      default: break;
    }
  }
  return s;
}

// ---------------------------------------------------------------------------
// Seeded random operator (synthetic inputs): Philox-4x32-10 (Salmon, Moraes,
// Dror, Shaw, SC'11) keyed by the seed, counter = element index, two 32-bit
// words -> 53-bit uniforms, Box-Muller cosine branch.
// ---------------------------------------------------------------------------
static inline void philox4x32_10(uint32_t ctr[4], uint32_t key[2]) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)M0 * ctr[0];
    uint64_t p1 = (uint64_t)M1 * ctr[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ ctr[1] ^ k0;
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ ctr[3] ^ k1;
    uint32_t n3 = lo0;
    ctr[0] = n0; ctr[1] = n1; ctr[2] = n2; ctr[3] = n3;
    k0 += W0;
    k1 += W1;
  }
}

static inline double normal_at(uint64_t seed, uint64_t i) {
  uint32_t c[4] = {(uint32_t)i, (uint32_t)(i >> 32), 0x51ED0u, 0u};
  uint32_t k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  philox4x32_10(c, k);
  uint64_t a = ((uint64_t)c[0] << 21) ^ (uint64_t)(c[1] >> 11);  // 53 bits
  uint64_t b = ((uint64_t)c[2] << 21) ^ (uint64_t)(c[3] >> 11);
  a &= (1ull << 53) - 1;
  b &= (1ull << 53) - 1;
  double u1 = ((double)a + 1.0) / 9007199254740992.0;  // (0,1]
  double u2 = (double)b / 9007199254740992.0;          // [0,1)
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

void fill_random(const qd_layout* L, int herm, uint64_t seed, double sigma, int conserve, double* v) {
  const int n = L->n, mp = L->mp;
  for (i64 i = 0; i < L->neq; ++i) v[i] = sigma * normal_at(seed, (uint64_t)i);
  v[0] = 0.0;
  auto sym = [&](double* a, int k) {
    for (int j = 0; j < k; ++j)
      for (int i = 0; i <= j; ++i) {
        double x = a[i + (i64)j * k], y = a[j + (i64)i * k];
        double s = (x + herm * y) / 2;
        a[i + (i64)j * k] = s;
        a[j + (i64)i * k] = (y + herm * x) / 2;
      }
  };
  sym(v + L->o_fhh, n);
  sym(v + L->o_fpp, mp);
  if (conserve) {
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i)
        if (L->gid[i] != L->gid[j]) v[L->o_fhh + i + (i64)j * n] = 0.0;
    for (int j = 0; j < mp; ++j)
      for (int i = 0; i < mp; ++i)
        if (L->gid[n + i] != L->gid[n + j]) v[L->o_fpp + i + (i64)j * mp] = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < mp; ++i)
        if (L->gid[n + i] != L->gid[j]) v[L->o_fph + i + (i64)j * mp] = 0.0;
  }
  for (int b = 0; b < L->nblock; ++b) {
    const i64* o = &L->boff[6 * b];
    sym(v + o[0], L->blk[b].x);
    sym(v + o[1], L->blk[b].z);
    sym(v + o[3], L->blk[b].y);
  }
}

}  // namespace qd
