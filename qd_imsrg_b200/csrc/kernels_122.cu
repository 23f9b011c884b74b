// kernels_122.cu -- commutator_122 (src/commutators.f90:355-676) as two
// shared-memory-staged sparse passes per (M_L,M_S) block.
//
// In block q the pairs are ordered [hh | ph | pp] (block-local index P); the
// full block matrix V(P1,P2) holds the stored classes (class(P1) >=
// class(P2)) and herm * their transposes above.  For the stored output
// element <b1 b2|k1 k2> = C(P1,P2):
//   bra legs: C += sum_{t in G(b1)} [FA(b1,t) VB(t b2|P2) - FB(b1,t) VA(t b2|P2)]
//                + sum_{t in G(b2)} [FA(b2,t) VB(b1 t|P2) - FB(b2,t) VA(b1 t|P2)]
//   ket legs: C -= sum_{t in G(k1)} [FA'(k1,t) VB(P1|t k2) - FB'(k1,t) VA(P1|t k2)]
//                + sum_{t in G(k2)} [FA'(k2,t) VB(P1|k1 t) - FB'(k2,t) VA(P1|k1 t)]
// G(x) = states with the (m_l, m_s) of x: the only t whose pair (t,b2) lies in
// block q.  F/F' are the reference's one-body reads (see dev_common.cuh).
//
// Pass 1 (bra, SET): a CTA stages TJ columns of V_A and V_B (all ntot rows,
// upper classes through herm) in shared memory and writes those columns of
// every stored class.  Pass 2 (ket, ACC): a CTA stages TJ rows and adds the
// ket legs of those rows.  Each pass reads both operators about once; the
// gathers over t hit shared memory.  A warp covers 32/TJ rows x TJ columns, so
// the per-term lookups (static leg table: partner pair and sign; per-call
// F table: group-diagonal one-body reads) are shared by TJ lanes and the
// shared-memory reads of one row group are contiguous.
#include <algorithm>
#include <mutex>

#include "dev_common.cuh"

namespace qd {

constexpr int T122 = 512;  // threads per CTA
constexpr size_t SMEM_MAX_ATTR_122 = 227 * 1024;  // opt-in shared memory per CTA on sm_100
// TJ: columns (bra pass) / rows (ket pass) staged per CTA; a warp handles
// 32/TJ rows (bra) or columns (ket) at a time, TJ lanes each.

struct Task122 {
  int q;
  short cls;   // column class (bra pass) or row class (ket pass)
  short pad;
  int first;   // first column / row within the class
};

// vectorize slot of the stored part (row class c1 >= column class c2):
// (0,0) hhhh 0, (2,2) pppp 1, (2,0) pphh 2, (1,1) phph 3, (2,1) ppph 4, (1,0) phhh 5
__device__ __forceinline__ int slot_of(int c1, int c2) {
  if (c1 == 0) return 0;
  if (c1 == 1) return c2 == 0 ? 5 : 3;
  return c2 == 0 ? 2 : (c2 == 1 ? 4 : 1);
}
__device__ __forceinline__ int off_of(int c, int4 bd) { return c == 0 ? 0 : (c == 1 ? bd.x : bd.x + bd.y); }
__device__ __forceinline__ int cnt_of(int c, int4 bd) { return c == 0 ? bd.x : (c == 1 ? bd.y : bd.z); }
__device__ __forceinline__ int cls_of(int P, int nh, int nb) { return P < nh ? 0 : (P < nh + nb ? 1 : 2); }

// V(P1, P2) of one operator for block q, any classes (upper via herm); parts
// set in zmask are known to be zero and not read
__device__ __forceinline__ double vfull(const double* __restrict__ op, const i64* o, int4 bd, double herm,
                                        unsigned zmask, int P1, int P2) {
  int c1 = cls_of(P1, bd.x, bd.y), c2 = cls_of(P2, bd.x, bd.y);
  int r1 = P1 - off_of(c1, bd), r2 = P2 - off_of(c2, bd);
  if (c1 >= c2) {
    const int sl = slot_of(c1, c2);
    if ((zmask >> (P_HHHH + sl)) & 1u) return 0.0;
    return op[__ldg(o + sl) + r1 + (i64)r2 * cnt_of(c1, bd)];
  }
  const int sl = slot_of(c2, c1);
  if ((zmask >> (P_HHHH + sl)) & 1u) return 0.0;
  return herm * op[__ldg(o + sl) + r2 + (i64)r1 * cnt_of(c2, bd)];
}

// Leg-table entry (static per layout), for pair P = (x1<x2) of a block:
//   leg 0: t = G(x1)[k], t != x2, partner pair (t,x2); leg 1: t = G(x2)[k],
//   t != x1, partner pair (x1,t).  Packed: block-local index of the partner
//   (13 bits) | k (5 bits) << 13 | leg << 18 | (ordering sign < 0) << 19.
__device__ __forceinline__ int leg_idx(int e) { return e & 0x1FFF; }
__device__ __forceinline__ int leg_k(int e) { return (e >> 13) & 31; }
__device__ __forceinline__ int leg_leg(int e) { return (e >> 18) & 1; }
__device__ __forceinline__ double leg_sign(int e) { return ((e >> 19) & 1) ? -1.0 : 1.0; }

// F tables (per call): [2][m][gmax] double2: (FA, FB) for the bra legs, then
// (FA', FB') for the ket legs, of (state s, k-th member t of G(s)).
__global__ void k_ftab(DevLayout L, const double* __restrict__ A, double hA, const double* __restrict__ B, double hB,
                       double2* __restrict__ F, int gmax) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= L.m * gmax) return;
  int s = e / gmax, k = e % gmax;
  int g = __ldg(&L.gid[s]);
  int b = __ldg(&L.gstart[g]), sz = __ldg(&L.gstart[g + 1]) - b;
  double fab = 0.0, fbb = 0.0, fak = 0.0, fbk = 0.0;
  if (k < sz) {
    int t = __ldg(&L.gmem[b + k]);
    if (t < L.n) {
      double xa = f_hole(L, A, s, t), xb = f_hole(L, B, s, t);
      fab = xa; fbb = xb; fak = hA * xa; fbk = hB * xb;
    } else {
      double xa = f_part(L, A, t, s), xb = f_part(L, B, t, s);
      fab = hA * xa; fbb = hB * xb; fak = xa; fbk = xb;
    }
  }
  F[e] = make_double2(fab, fbb);
  F[L.m * gmax + e] = make_double2(fak, fbk);
}

// sum over the leg entries [l0, l1) of sg * (FA * VB - FB * VA), unrolled by 4
// so that the four entries' loads are independent
template <int TJ>
__device__ __forceinline__ double leg_sum(const int* __restrict__ legs, int l0, int l1, int s0, int s1,
                                          const double2* __restrict__ Ft, int gmax, const double2* sV, int lane_off) {
  double acc = 0.0;
  int u = l0;
  for (; u + 4 <= l1; u += 4) {
    int e[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) e[r] = __ldg(&legs[u + r]);
    double2 f[4], v[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      f[r] = __ldg(&Ft[(leg_leg(e[r]) ? s1 : s0) * gmax + leg_k(e[r])]);
      v[r] = sV[leg_idx(e[r]) * TJ + lane_off];
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) acc += leg_sign(e[r]) * (f[r].x * v[r].y - f[r].y * v[r].x);
  }
  for (; u < l1; ++u) {
    const int e = __ldg(&legs[u]);
    const double2 f = __ldg(&Ft[(leg_leg(e) ? s1 : s0) * gmax + leg_k(e)]);
    const double2 v = sV[leg_idx(e) * TJ + lane_off];
    acc += leg_sign(e) * (f.x * v.y - f.y * v.x);
  }
  return acc;
}

template <int TJ>
__global__ void __launch_bounds__(T122) k_122_bra(DevLayout L, const Task122* __restrict__ tasks,
                                                  const int* __restrict__ legstart, const int* __restrict__ legs,
                                                  const double2* __restrict__ Ftab, int gmax,
                                                  const double* __restrict__ A, double hA, unsigned zA,
                                                  const double* __restrict__ B, double hB, unsigned zB,
                                                  double* __restrict__ C) {
  extern __shared__ double2 smv[];  // (VA, VB) of each (row, column)
  const Task122 tk = tasks[blockIdx.x];
  const int q = tk.q, c2 = tk.cls;
  const int4 bd = __ldg(&L.blk[q]);
  const int nh = bd.x, nb = bd.y, ntot = bd.w;
  const int ncol = min(TJ, cnt_of(c2, bd) - tk.first);
  const int offc2 = off_of(c2, bd);
  const i64* o = L.boff + 6 * q;
  for (int e = threadIdx.x; e < ntot * TJ; e += blockDim.x) {
    int P1 = e % ntot, j = e / ntot;
    double va = 0.0, vb = 0.0;
    if (j < ncol) {
      int P2 = offc2 + tk.first + j;
      va = vfull(A, o, bd, hA, zA, P1, P2);
      vb = vfull(B, o, bd, hB, zB, P1, P2);
    }
    smv[P1 * TJ + j] = make_double2(va, vb);
  }
  __syncthreads();
  const int pb = __ldg(&L.pbase[q]);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  constexpr int RPW = 32 / TJ;
  const int j = lane % TJ, sub = lane / TJ;
  for (int base = offc2 + warp * RPW; base < ntot; base += nwarp * RPW) {
    const int P1 = base + sub;
    if (P1 >= ntot) continue;
    const int2 br = __ldg(&L.pairs[pb + P1]);
    const double acc = leg_sum<TJ>(legs, __ldg(&legstart[pb + P1]), __ldg(&legstart[pb + P1 + 1]), br.x, br.y, Ftab,
                               gmax, smv, j);
    if (j < ncol) {
      const int c1 = cls_of(P1, nh, nb);
      const int rows = cnt_of(c1, bd);
      C[__ldg(o + slot_of(c1, c2)) + (P1 - off_of(c1, bd)) + (i64)(tk.first + j) * rows] = acc;
    }
  }
}

template <int TJ>
__global__ void __launch_bounds__(T122) k_122_ket(DevLayout L, const Task122* __restrict__ tasks,
                                                  const int* __restrict__ legstart, const int* __restrict__ legs,
                                                  const double2* __restrict__ Ftab, int gmax,
                                                  const double* __restrict__ A, double hA, unsigned zA,
                                                  const double* __restrict__ B, double hB, unsigned zB,
                                                  double* __restrict__ C) {
  extern __shared__ double2 smv[];
  const Task122 tk = tasks[blockIdx.x];
  const int q = tk.q, c1 = tk.cls;
  const int4 bd = __ldg(&L.blk[q]);
  const int nh = bd.x, nb = bd.y, ntot = bd.w;
  const int rows = cnt_of(c1, bd);
  const int nrow = min(TJ, rows - tk.first);
  const int offc1 = off_of(c1, bd);
  const i64* o = L.boff + 6 * q;
  for (int e = threadIdx.x; e < ntot * TJ; e += blockDim.x) {
    int i = e % TJ, P2 = e / TJ;
    double va = 0.0, vb = 0.0;
    if (i < nrow) {
      int P1 = offc1 + tk.first + i;
      va = vfull(A, o, bd, hA, zA, P1, P2);
      vb = vfull(B, o, bd, hB, zB, P1, P2);
    }
    smv[P2 * TJ + i] = make_double2(va, vb);
  }
  __syncthreads();
  const int pb = __ldg(&L.pbase[q]);
  const double2* Fket = Ftab + (i64)L.m * gmax;
  const int ncols = offc1 + rows;  // output columns: classes <= c1
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  constexpr int RPW = 32 / TJ;
  const int i = lane % TJ, sub = lane / TJ;
  for (int base = warp * RPW; base < ncols; base += nwarp * RPW) {
    const int P2 = base + sub;
    if (P2 >= ncols) continue;
    const int2 kt = __ldg(&L.pairs[pb + P2]);
    const double acc = leg_sum<TJ>(legs, __ldg(&legstart[pb + P2]), __ldg(&legstart[pb + P2 + 1]), kt.x, kt.y, Fket,
                               gmax, smv, i);
    if (i < nrow) {
      const int c2 = cls_of(P2, nh, nb);
      C[__ldg(o + slot_of(c1, c2)) + (i64)(P2 - off_of(c2, bd)) * rows + tk.first + i] -= acc;
    }
  }
}

// ---- host side --------------------------------------------------------------
namespace {
// Tasks are grouped in buckets of similar block size; each bucket is one
// launch whose dynamic shared memory fits its largest block.
struct Bucket122 {
  int tj;       // 8 or 4
  int first;    // range in the task arrays
  int count;
  size_t smem;
};
struct Plan122 {
  Task122* d_bra = nullptr;
  Task122* d_ket = nullptr;
  int* d_legstart = nullptr;
  int* d_legs = nullptr;
  double2* d_ftab = nullptr;
  int nbra = 0, nket = 0, gmax = 0;
  std::vector<Bucket122> buckets;
};
std::map<const qd_layout*, Plan122>& plans() {
  static std::map<const qd_layout*, Plan122> m;
  return m;
}
// plans of different layouts are built and dropped from concurrent host
// threads (batched flows); map nodes stay put, so a found plan needs no lock
std::mutex g_plan_mutex;
}  // namespace

static int plan_122(qd_layout* L, Plan122** out) {
  std::lock_guard<std::mutex> lock(g_plan_mutex);
  auto it = plans().find(L);
  if (it != plans().end()) {
    *out = &it->second;
    return QD_OK;
  }
  Plan122 p;
  // group sizes
  int ngroup = (int)L->gstart.size() - 1;
  for (int g = 0; g < ngroup; ++g) p.gmax = std::max(p.gmax, L->gstart[g + 1] - L->gstart[g]);
  if (p.gmax > 31) {
    set_error("commutator_122: (ml,ms) group of %d states exceeds the leg-table range", p.gmax);
    return QD_ERR_ARG;
  }
  // leg table over all pairs of all blocks (global pair index = pbase[q] + P)
  std::vector<int> legstart(L->pairs.size() + 1, 0), legs;
  const int m = L->m;
  for (int q = 0; q < L->nblock; ++q) {
    const int nh = L->blk[q].x, nb = L->blk[q].y;
    for (int P = 0; P < L->blk[q].w; ++P) {
      const int gp = L->pbase[q] + P;
      legstart[gp] = (int)legs.size();
      const int x1 = L->pairs[gp].x, x2 = L->pairs[gp].y;
      for (int leg = 0; leg < 2; ++leg) {
        const int xs = leg ? x2 : x1, other = leg ? x1 : x2;
        const int g = L->gid[xs];
        for (int k = 0; k < L->gstart[g + 1] - L->gstart[g]; ++k) {
          const int t = L->gmem[L->gstart[g] + k];
          if (t == other) continue;
          const int a = leg ? x1 : t, b = leg ? t : x2;
          const int e = L->ptab[(size_t)a * m + b];
          if (pt_blk(e) != q) {
            set_error("commutator_122: leg partner outside its block (layout inconsistency)");
            return QD_ERR_LAYOUT;
          }
          const int c = pt_cls(e);
          const int idx = pt_idx(e) + (c == 0 ? 0 : (c == 1 ? nh : nh + nb));
          if (idx > 0x1FFF) {
            set_error("commutator_122: block too large for the leg table");
            return QD_ERR_ARG;
          }
          legs.push_back(idx | (k << 13) | (leg << 18) | (pt_swap(e) << 19));
        }
      }
    }
  }
  legstart[L->pairs.size()] = (int)legs.size();
  // buckets: (max block size, TJ)
  const int lim[4] = {200, 400, 800, 1 << 30};
  const int tjs[4] = {8, 8, 8, 4};
  std::vector<Task122> hb;
  int maxtot = 0;
  for (int bkt = 0; bkt < 4; ++bkt) {
    const int lo = bkt ? lim[bkt - 1] : 0;
    std::vector<std::pair<int, Task122>> v;
    int bmax = 0;
    for (int q = 0; q < L->nblock; ++q) {
      const int ntot = L->blk[q].w;
      if (ntot <= lo || ntot > lim[bkt]) continue;
      const int cnt[3] = {L->blk[q].x, L->blk[q].y, L->blk[q].z};
      bmax = std::max(bmax, ntot);
      for (int c = 0; c < 3; ++c)
        for (int f = 0; f < cnt[c]; f += tjs[bkt]) v.push_back({ntot, Task122{q, (short)c, 0, f}});
    }
    if (v.empty()) continue;
    std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    Bucket122 bk;
    bk.tj = tjs[bkt];
    bk.first = (int)hb.size();
    bk.count = (int)v.size();
    bk.smem = sizeof(double2) * (size_t)bmax * bk.tj;
    if (bk.smem > SMEM_MAX_ATTR_122) {
      set_error("commutator_122: block of %d pairs exceeds shared memory", bmax);
      return QD_ERR_ARG;
    }
    for (auto& x : v) hb.push_back(x.second);
    p.buckets.push_back(bk);
    maxtot = std::max(maxtot, bmax);
  }
  std::vector<Task122>& hk = hb;  // the ket pass uses the same (block, class, first) tasks
  p.nbra = (int)hb.size();
  p.nket = (int)hk.size();
  if (p.nbra) {
    QD_CUDA(cudaMalloc(&p.d_bra, hb.size() * sizeof(Task122)));
    QD_CUDA(cudaMemcpy(p.d_bra, hb.data(), hb.size() * sizeof(Task122), cudaMemcpyHostToDevice));
    QD_CUDA(cudaMalloc(&p.d_ket, hk.size() * sizeof(Task122)));
    QD_CUDA(cudaMemcpy(p.d_ket, hk.data(), hk.size() * sizeof(Task122), cudaMemcpyHostToDevice));
  }
  QD_CUDA(cudaMalloc(&p.d_legstart, legstart.size() * sizeof(int)));
  QD_CUDA(cudaMemcpy(p.d_legstart, legstart.data(), legstart.size() * sizeof(int), cudaMemcpyHostToDevice));
  QD_CUDA(cudaMalloc(&p.d_legs, std::max<size_t>(1, legs.size()) * sizeof(int)));
  if (!legs.empty()) QD_CUDA(cudaMemcpy(p.d_legs, legs.data(), legs.size() * sizeof(int), cudaMemcpyHostToDevice));
  QD_CUDA(cudaMalloc(&p.d_ftab, sizeof(double2) * 2 * (size_t)L->m * p.gmax));
  L->ws_bytes += (i64)(legstart.size() + legs.size()) * 4 + (i64)sizeof(double) * 4 * L->m * p.gmax;
  // the attribute is process-wide: set it to the device limit, so that plans
  // built concurrently for other layouts can never lower it below a need
  if (!p.buckets.empty()) {
    const int lim = (int)SMEM_MAX_ATTR_122;
    QD_CUDA(cudaFuncSetAttribute(k_122_bra<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    QD_CUDA(cudaFuncSetAttribute(k_122_ket<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    QD_CUDA(cudaFuncSetAttribute(k_122_bra<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    QD_CUDA(cudaFuncSetAttribute(k_122_ket<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  }
  plans()[L] = p;
  *out = &plans()[L];
  return QD_OK;
}

void drop_122_plan(const qd_layout* L) {
  std::lock_guard<std::mutex> lock(g_plan_mutex);
  auto it = plans().find(L);
  if (it == plans().end()) return;
  for (void* ptr : {(void*)it->second.d_bra, (void*)it->second.d_ket, (void*)it->second.d_legstart,
                    (void*)it->second.d_legs, (void*)it->second.d_ftab})
    if (ptr) cudaFree(ptr);
  plans().erase(it);
}

int launch_122(qd_layout* L, const qd_op* A, const qd_op* B, double* C) {
  Plan122* p;
  int rc = plan_122(L, &p);
  if (rc) return rc;
  if (p->nbra == 0) return QD_OK;
  const int nf = L->m * p->gmax;
  k_ftab<<<(nf + 127) / 128, 128, 0, L->stream>>>(L->dev, A->d, (double)A->herm, B->d, (double)B->herm, p->d_ftab,
                                                  p->gmax);
  for (const Bucket122& b : p->buckets) {
    const Task122* tb = p->d_bra + b.first;
    if (b.tj == 8)
      k_122_bra<8><<<b.count, T122, b.smem, L->stream>>>(L->dev, tb, p->d_legstart, p->d_legs, p->d_ftab, p->gmax,
                                                          A->d, (double)A->herm, A->zero_mask, B->d, (double)B->herm,
                                                          B->zero_mask, C);
    else
      k_122_bra<4><<<b.count, T122, b.smem, L->stream>>>(L->dev, tb, p->d_legstart, p->d_legs, p->d_ftab, p->gmax,
                                                          A->d, (double)A->herm, A->zero_mask, B->d, (double)B->herm,
                                                          B->zero_mask, C);
    ++L->nlaunch;
  }
  for (const Bucket122& b : p->buckets) {
    const Task122* tk = p->d_ket + b.first;
    if (b.tj == 8)
      k_122_ket<8><<<b.count, T122, b.smem, L->stream>>>(L->dev, tk, p->d_legstart, p->d_legs, p->d_ftab, p->gmax,
                                                          A->d, (double)A->herm, A->zero_mask, B->d, (double)B->herm,
                                                          B->zero_mask, C);
    else
      k_122_ket<4><<<b.count, T122, b.smem, L->stream>>>(L->dev, tk, p->d_legstart, p->d_legs, p->d_ftab, p->gmax,
                                                          A->d, (double)A->herm, A->zero_mask, B->d, (double)B->herm,
                                                          B->zero_mask, C);
    ++L->nlaunch;
  }
  L->nlaunch += 1;
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

}  // namespace qd
