// kernels_122.cu -- commutator_122 (src/commutators.f90:355-676) as two
// shared-memory-staged passes per (M_L,M_S) block, evaluated group pair by
// group pair as small dense products.
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
// Group pairs.  The pairs of block q split into the sets S(g,h) of pairs with
// one state in (m_l,m_s) group g and one in group h (g <= h).  Indexing S(g,h)
// as cells (k1,k2) <-> (t1,t2) = (G_g[k1], G_h[k2]) and writing the block's
// antisymmetric matrix in that orientation, M(k1,k2) = V(t1 t2|.) (= -V of the
// stored pair when t1 > t2; 0 on the diagonal when g = h), the bra legs of
// every pair of S(g,h) are
//   Y = F_g M + M F_h^T,   F_g(k1',k1) = F(G_g[k1'], k1-th member of G_g),
// and C(pair) = (orientation sign) * Y(cell).  The ket legs are the same with
// F' and V transposed.  Each product runs along "fibers": a fixed k2 (F_g,
// length |G_g|) or a fixed k1 (F_h, length |G_h|).  A warp takes one group
// pair and direction at a time and forms the product on the FP64 tensor pipe
// (mma.sync m8n8k4): F as A fragments held in registers, the staged cells as
// B fragments, FA * VB and -FB * VA into one accumulator.
//
// Pass 1 (bra, SET): a CTA stages TJ columns of V_A and V_B (all ntot rows,
// upper classes through herm) in shared memory in cell order, runs the k1
// fibers, then the k2 fibers, and writes those columns of every stored class.
// Pass 2 (ket, ACC): a CTA stages TJ rows and subtracts the ket legs of those
// rows.  Each pass reads both operators about once; the products read shared
// memory and registers only.
#include <algorithm>
#include <map>
#include <mutex>
#include <type_traits>

#include "dev_common.cuh"

namespace qd {

constexpr int T122 = 256;                          // threads per CTA
constexpr int GMAX122 = 16;                        // largest (m_l,m_s) group (fiber length)
constexpr size_t SMEM_MAX_ATTR_122 = 227 * 1024;   // opt-in shared memory per CTA on sm_100
constexpr size_t SMEM_TARGET_122 = 74 * 1024;      // per-CTA staging goal: three CTAs per SM
constexpr size_t SMEM_STATIC_122 = 1024;           // bound on the pass kernels' static shared memory
// Per-pass TJ rule (measured on the N=20 R=20 flow, 122 ms per flow): both
// passes at TJ >= 2 within 74 KB, 592; the ket pass at TJ >= 4 within 112 or
// 150 KB (whole 32-byte sectors, fewer CTAs), 812-820; TJ = 1 on the largest
// blocks of either pass, 637-808; 8 staging loads in flight per thread
// instead of 4 (U122), 611.  Parallelism beats sector efficiency here.
constexpr size_t KET_SMEM_TARGET_122 = 74 * 1024;   // ket pass: three CTAs per SM
constexpr int KET_MIN_TJ_122 = 2;
constexpr int BRA_MIN_TJ_122 = 2;

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

// Static tables of a layout (built once, see plan_122):
//   meta[q]   = {cells of block q, first group pair, end of its group pairs, 0}
//   sub[u]    = {first cell, |G_g| | |G_h| << 8 | (g = h) << 16, offset of F_g,
//               offset of F_h} (group pairs of a block in decreasing size)
//   cell[gp]  = for the pair gp = pbase[q] + P: {primary cell << 1 | (orientation sign < 0),
//               mirror cell (the same pair seen as (t2,t1) when g = h) or -1}
//   sbase[s]  = offset of state s's row in the group-major F table
// Per call: F table [2][nfent] double2 (FA, FB) bra, then (FA', FB') ket,
// group-major: F[goff_g + k1' * |G_g| + k].
__global__ void k_ftab(DevLayout L, const int* __restrict__ sbase, const double* __restrict__ A, double hA,
                       const double* __restrict__ B, double hB, double2* __restrict__ F, int gmax, int nfent) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= L.m * gmax) return;
  int s = e / gmax, k = e % gmax;
  int g = __ldg(&L.gid[s]);
  int b = __ldg(&L.gstart[g]), sz = __ldg(&L.gstart[g + 1]) - b;
  if (k >= sz) return;
  const int t = __ldg(&L.gmem[b + k]);
  double fab, fbb, fak, fbk;
  if (t < L.n) {
    const double xa = f_hole(L, A, s, t), xb = f_hole(L, B, s, t);
    fab = xa; fbb = xb; fak = hA * xa; fbk = hB * xb;
  } else {
    const double xa = f_part(L, A, t, s), xb = f_part(L, B, t, s);
    fab = hA * xa; fbb = hB * xb; fak = xa; fbk = xb;
  }
  const int pos = __ldg(&sbase[s]) + k;
  F[pos] = make_double2(fab, fbb);
  F[nfent + pos] = make_double2(fak, fbk);
}

__device__ __forceinline__ void dmma122(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// One direction of one group pair, by one warp, on the FP64 tensor pipe:
// Y(r, col) = sum_k F(r,k) (FA * VB - FB * VA)(k, col) as m8n8k4 products.
// DIR 0: F = F_g (N = |G_g|), columns col = (k2, j), cell (k, col) =
// base + k n2 + k2 (assigns: it reaches every cell once); DIR 1: F = F_h
// (N = |G_h|), columns col = (k1, j), cell = base + k1 n2 + k (adds).
// Fragments (m8n8k4): A row lane/4, k lane%4; B k lane%4, column lane/4;
// D row lane/4, columns 2 (lane%4) + {0,1}.  Out-of-range rows, k and
// columns are selected to zero (never multiplied with shared-memory data).
template <int N, int TJ, int DIR>
__device__ __forceinline__ void pair_dir(int base, int n1, int n2, int fofs, int lane, const double2* __restrict__ Vc,
                                         double* __restrict__ Yc, const double2* __restrict__ F) {
  constexpr int MT = (N + 7) / 8, KS = (N + 3) / 4;
  double fa[MT][KS], fb[MT][KS];
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int ks = 0; ks < KS; ++ks) {
      const int r = 8 * mt + (lane >> 2), k = 4 * ks + (lane & 3);
      double2 f = make_double2(0.0, 0.0);
      if (r < N && k < N) f = __ldg(&F[fofs + r * N + k]);
      fa[mt][ks] = f.x;
      fb[mt][ks] = -f.y;
    }
  const int ncol = (DIR ? n1 : n2) * TJ;
  auto cell = [&](int k, int col) -> int {  // staged element of (k, col)
    return DIR ? (base + (col / TJ) * n2 + k) * TJ + (col % TJ) : (base + k * n2) * TJ + col;
  };
  for (int c0 = 0; c0 < ncol; c0 += 8) {
    double d[MT][2];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) d[mt][0] = d[mt][1] = 0.0;
    const int bcol = c0 + (lane >> 2);
#pragma unroll
    for (int ks = 0; ks < KS; ++ks) {
      const int k = 4 * ks + (lane & 3);
      double2 v = make_double2(0.0, 0.0);
      if (k < N && bcol < ncol) v = Vc[cell(k, bcol)];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        dmma122(d[mt][0], d[mt][1], fa[mt][ks], v.y);
        dmma122(d[mt][0], d[mt][1], fb[mt][ks], v.x);
      }
    }
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = 8 * mt + (lane >> 2), c = c0 + 2 * (lane & 3) + e;
        if (r < N && c < ncol) {
          double* y = Yc + cell(r, c);
          if (DIR)
            *y += d[mt][e];
          else
            *y = d[mt][e];
        }
      }
  }
}

// all group pairs of the block, one direction; warps take group pairs in turn
// (no two group pairs share a cell, no two fibers of a direction share a cell)
template <int TJ, int DIR, int GM>
__device__ __forceinline__ void run_dir(const int4* __restrict__ sub, int ns, const double2* Vc, double* Yc,
                                        const double2* __restrict__ F) {
  const int lane = threadIdx.x & 31;
  for (int u = threadIdx.x >> 5; u < ns; u += T122 / 32) {
    const int4 d = __ldg(&sub[u]);
    const int n1 = d.y & 0xFF, n2 = (d.y >> 8) & 0xFF;
    const int fofs = DIR ? d.w : d.z;
    switch (DIR ? n2 : n1) {
#define QD_DIR_CASE(N)                                                         \
  case N:                                                                      \
    if constexpr (N <= GM) pair_dir<N, TJ, DIR>(d.x, n1, n2, fofs, lane, Vc, Yc, F); \
    break;
      QD_DIR_CASE(1) QD_DIR_CASE(2) QD_DIR_CASE(3) QD_DIR_CASE(4)
      QD_DIR_CASE(5) QD_DIR_CASE(6) QD_DIR_CASE(7) QD_DIR_CASE(8)
      QD_DIR_CASE(9) QD_DIR_CASE(10) QD_DIR_CASE(11) QD_DIR_CASE(12)
      QD_DIR_CASE(13) QD_DIR_CASE(14) QD_DIR_CASE(15) QD_DIR_CASE(16)
#undef QD_DIR_CASE
      default: break;
    }
  }
}

// stage (VA, VB) of a pair into its cell(s), staged column/row j
template <int TJ>
__device__ __forceinline__ void stage_cell(double2* Vc, int2 cl, int j, double va, double vb) {
  const double s = (cl.x & 1) ? -1.0 : 1.0;
  Vc[(cl.x >> 1) * TJ + j] = make_double2(s * va, s * vb);
  if (cl.y >= 0) Vc[cl.y * TJ + j] = make_double2(-s * va, -s * vb);
}

constexpr int U122 = 4;  // staging loads in flight per thread

// Pass kernels.  KET = 0: bra pass over TJ columns of class ct = tk.cls
// (SET); KET = 1: ket pass over TJ rows of class ct (subtract).  The staged
// operand values V(P1,P2) are read class segment by class segment of the
// other index: segment c (cnt_c pairs) of stored part (max(c,ct), min(c,ct))
// is contiguous along the pair index when its rows are the varying index,
// else strided; the upper segments carry herm.
template <int TJ, int KET, int GM>
__global__ void __launch_bounds__(T122, GM <= 10 ? 3 : 2) k_122_pass(DevLayout L, const Task122* __restrict__ tasks,
                                                   const int4* __restrict__ meta, const int4* __restrict__ sub,
                                                   const int2* __restrict__ cell, const double2* __restrict__ Ftab,
                                                   const double* __restrict__ A, double hA, unsigned zA,
                                                   const double* __restrict__ B, double hB, unsigned zB,
                                                   double* __restrict__ C) {
  extern __shared__ double2 smv[];
  const Task122 tk = tasks[blockIdx.x];
  const int q = tk.q, ct = tk.cls;
  const int4 bd = __ldg(&L.blk[q]);
  const int4 mt = __ldg(&meta[q]);
  double2* Vc = smv;                                        // [cells][TJ] (VA, VB)
  double* Yc = reinterpret_cast<double*>(smv + mt.x * TJ);  // [cells][TJ]
  int* pc = reinterpret_cast<int*>(Yc + mt.x * TJ);          // [ntot] primary cell << 1 | sign
  const int nct = cnt_of(ct, bd);
  const int nj = min(TJ, nct - tk.first);  // staged columns (bra) / rows (ket)
  const int pb = __ldg(&L.pbase[q]);
  const i64* o = L.boff + 6 * q;
  const int ns = mt.z - mt.y;
  sub += mt.y;
  // cells of no pair: the diagonal (t,t) of same-group pairs
  for (int u = threadIdx.x; u < ns; u += T122) {
    const int4 d = __ldg(&sub[u]);
    if (d.y >> 16) {
      const int n = d.y & 0xFF;
      for (int k = 0; k < n; ++k)
#pragma unroll
        for (int j = 0; j < TJ; ++j) Vc[(d.x + k * (n + 1)) * TJ + j] = make_double2(0.0, 0.0);
    }
  }
  for (int c = 0; c < 3; ++c) {
    const int nc = cnt_of(c, bd);
    if (nc == 0) continue;
    // element (r, j): the pair r of segment c against staged index j
    const bool lower = KET ? (ct >= c) : (c >= ct);  // stored without transposition
    const int sl = KET ? (lower ? slot_of(ct, c) : slot_of(c, ct)) : (lower ? slot_of(c, ct) : slot_of(ct, c));
    const bool za = (zA >> (P_HHHH + sl)) & 1u, zb = (zB >> (P_HHHH + sl)) & 1u;
    const double fa = lower ? 1.0 : hA, fb = lower ? 1.0 : hB;
    // bra: V(row r of c, column first+j); ket: V(row first+j, column r of c).
    // The stored part's rows are segment c (bra lower, ket upper): address
    // r + (first+j) * nc; else its rows are class ct: (first+j) + r * nct.
    const bool crow = KET ? !lower : lower;
    const i64 rs = crow ? 1 : nct, js = crow ? nc : 1;
    const i64 b0 = __ldg(o + sl) + (crow ? (i64)tk.first * nc : (i64)tk.first);
    const int offc = off_of(c, bd);
    const int total = nc * TJ;
    for (int e0 = threadIdx.x; e0 < total; e0 += U122 * T122) {
      double va[U122], vb[U122];
      int2 cl[U122];
#pragma unroll
      for (int u = 0; u < U122; ++u) {
        const int e = e0 + u * T122;
        const int r = e / TJ, j = e % TJ;
        va[u] = vb[u] = 0.0;
        cl[u] = make_int2(-1, -1);
        if (e < total && j < nj) {
          const i64 a = b0 + r * rs + j * js;
          cl[u] = __ldg(&cell[pb + offc + r]);
          if (!za) va[u] = fa * __ldg(A + a);
          if (!zb) vb[u] = fb * __ldg(B + a);
        }
      }
#pragma unroll
      for (int u = 0; u < U122; ++u)
        if (cl[u].x >= 0) {
          const int e = e0 + u * T122;
          stage_cell<TJ>(Vc, cl[u], e % TJ, va[u], vb[u]);
          if (e % TJ == 0) pc[offc + e / TJ] = cl[u].x;
        }
    }
  }
  __syncthreads();
  run_dir<TJ, 0, GM>(sub, ns, Vc, Yc, Ftab);
  __syncthreads();
  run_dir<TJ, 1, GM>(sub, ns, Vc, Yc, Ftab);
  __syncthreads();
  // output: bra -> rows of classes c >= ct of the staged columns (SET);
  // ket -> columns of classes c <= ct of the staged rows (subtract)
  for (int c = KET ? 0 : ct; c <= (KET ? ct : 2); ++c) {
    const int nc = cnt_of(c, bd);
    if (nc == 0) continue;
    const int sl = KET ? slot_of(ct, c) : slot_of(c, ct);
    const i64 rs = KET ? nct : 1, js = KET ? 1 : nc;
    const i64 b0 = __ldg(o + sl) + (KET ? (i64)tk.first : (i64)tk.first * nc);
    const int offc = off_of(c, bd);
    for (int e0 = threadIdx.x; e0 < nc * TJ; e0 += U122 * T122) {
#pragma unroll
      for (int u = 0; u < U122; ++u) {
        const int e = e0 + u * T122;
        const int r = e / TJ, j = e % TJ;
        if (e >= nc * TJ || j >= nj) continue;
        const int cx = pc[offc + r];
        const double y = Yc[(cx >> 1) * TJ + j];
        double* out = C + b0 + r * rs + j * js;
        if (KET)
          *out -= (cx & 1) ? -y : y;
        else
          *out = (cx & 1) ? -y : y;
      }
    }
  }
}

// ---- host side --------------------------------------------------------------
namespace {
// Tasks are grouped in buckets by TJ; each bucket is one launch per pass
// whose dynamic shared memory fits its largest block.
struct Bucket122 {
  int tj;       // 1, 2, 4, 8 or 16
  int first;    // range in the task array
  int count;
  size_t smem;
};
struct Plan122 {
  Task122* d_task = nullptr;
  int4* d_meta = nullptr;
  int4* d_sub = nullptr;
  int2* d_cell = nullptr;
  int* d_sbase = nullptr;
  double2* d_ftab = nullptr;
  int ntask = 0, gmax = 0, nfent = 0;
  std::vector<Bucket122> buckets[2];  // bra pass, ket pass
};
std::map<const qd_layout*, Plan122>& plans() {
  static std::map<const qd_layout*, Plan122> m;
  return m;
}
// plans of different layouts are built and dropped from concurrent host
// threads (batched flows); map nodes stay put, so a found plan needs no lock
std::mutex g_plan_mutex;

size_t smem_122(int cells, int npair, int tj) {
  return (sizeof(double2) + sizeof(double)) * (size_t)cells * tj + sizeof(int) * (size_t)((npair + 3) & ~3);
}
}  // namespace

// the attribute is process-wide: set it to the device limit, so that plans
// built concurrently for other layouts can never lower it below a need
template <int GM>
static int set_attr_122() {
  const void* fns[10] = {(const void*)k_122_pass<16, 0, GM>, (const void*)k_122_pass<16, 1, GM>,
                         (const void*)k_122_pass<8, 0, GM>,  (const void*)k_122_pass<8, 1, GM>,
                         (const void*)k_122_pass<4, 0, GM>,  (const void*)k_122_pass<4, 1, GM>,
                         (const void*)k_122_pass<2, 0, GM>,  (const void*)k_122_pass<2, 1, GM>,
                         (const void*)k_122_pass<1, 0, GM>,  (const void*)k_122_pass<1, 1, GM>};
  for (const void* fn : fns) {
    cudaFuncAttributes fa;
    QD_CUDA(cudaFuncGetAttributes(&fa, fn));  // static + dynamic shared memory <= the limit
    QD_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SMEM_MAX_ATTR_122 - (int)fa.sharedSizeBytes));
  }
  return QD_OK;
}

template <int GM, int KET>
static void pass_122(const Plan122* p, qd_layout* L, const qd_op* A, const qd_op* B, double* C) {
  const double2* ft = p->d_ftab + (KET ? p->nfent : 0);
  for (const Bucket122& b : p->buckets[KET]) {
#define QD_122_LAUNCH(TJ)                                                                                          \
  k_122_pass<TJ, KET, GM><<<b.count, T122, b.smem, L->stream>>>(L->dev, p->d_task + b.first, p->d_meta, p->d_sub, \
                                                                p->d_cell, ft, A->d, (double)A->herm,             \
                                                                A->zero_mask, B->d, (double)B->herm,              \
                                                                B->zero_mask, C)
    switch (b.tj) {
      case 16: QD_122_LAUNCH(16); break;
      case 8: QD_122_LAUNCH(8); break;
      case 4: QD_122_LAUNCH(4); break;
      case 2: QD_122_LAUNCH(2); break;
      default: QD_122_LAUNCH(1); break;
    }
#undef QD_122_LAUNCH
    ++L->nlaunch;
  }
}

static int plan_122(qd_layout* L, Plan122** out) {
  std::lock_guard<std::mutex> lock(g_plan_mutex);
  auto it = plans().find(L);
  if (it != plans().end()) {
    *out = &it->second;
    return QD_OK;
  }
  Plan122 p;
  const int m = L->m;
  const int ngroup = (int)L->gstart.size() - 1;
  std::vector<int> gsz(ngroup), goff(ngroup + 1, 0), kpos(m, 0), sbase(m, 0);
  for (int g = 0; g < ngroup; ++g) {
    gsz[g] = L->gstart[g + 1] - L->gstart[g];
    p.gmax = std::max(p.gmax, gsz[g]);
    goff[g + 1] = goff[g] + gsz[g] * gsz[g];
    for (int k = 0; k < gsz[g]; ++k) kpos[L->gmem[L->gstart[g] + k]] = k;
  }
  if (p.gmax > GMAX122) {
    set_error("commutator_122: (ml,ms) group of %d states exceeds %d", p.gmax, GMAX122);
    return QD_ERR_ARG;
  }
  p.nfent = goff[ngroup];
  for (int s = 0; s < m; ++s) sbase[s] = goff[L->gid[s]] + kpos[s] * gsz[L->gid[s]];

  // group pairs and cells of every block
  std::vector<int4> meta(L->nblock), sub;
  std::vector<int2> cell(L->pairs.size(), int2{-1, -1});
  for (int q = 0; q < L->nblock; ++q) {
    const int nh = L->blk[q].x, nb = L->blk[q].y, ntot = L->blk[q].w, pb = L->pbase[q];
    std::map<std::pair<int, int>, int> subs;  // (g <= h) -> first cell
    std::vector<std::pair<int, int>> order;
    int ncell = 0;
    for (int P = 0; P < ntot; ++P) {
      const int2 pr = L->pairs[pb + P];
      const int g = std::min(L->gid[pr.x], L->gid[pr.y]), h = std::max(L->gid[pr.x], L->gid[pr.y]);
      if (subs.emplace(std::make_pair(g, h), ncell).second) {
        order.push_back({g, h});
        ncell += gsz[g] * gsz[h];
      }
    }
    std::vector<int4> sv;
    for (const auto& gh : order) {
      const int g = gh.first, h = gh.second, base = subs[gh], n1 = gsz[g], n2 = gsz[h];
      for (int k1 = 0; k1 < n1; ++k1)
        for (int k2 = 0; k2 < n2; ++k2) {
          if (g == h && k1 == k2) continue;  // (t,t): no pair, M = 0
          const int t1 = L->gmem[L->gstart[g] + k1], t2 = L->gmem[L->gstart[h] + k2];
          const int e = L->ptab[(size_t)t1 * m + t2];
          if (e < 0 || pt_blk(e) != q) {
            set_error("commutator_122: group pair outside its block (layout inconsistency)");
            return QD_ERR_LAYOUT;
          }
          const int c = pt_cls(e);
          const int P = pt_idx(e) + (c == 0 ? 0 : (c == 1 ? nh : nh + nb));
          const int cidx = base + k1 * n2 + k2;
          if (g != h || k1 < k2)
            cell[pb + P].x = cidx << 1 | pt_swap(e);
          else
            cell[pb + P].y = cidx;
        }
      sv.push_back(int4{base, n1 | n2 << 8 | (g == h) << 16, goff[g], goff[h]});
    }
    for (int P = 0; P < ntot; ++P)
      if (cell[pb + P].x < 0) {
        set_error("commutator_122: pair without a group-pair cell (layout inconsistency)");
        return QD_ERR_LAYOUT;
      }
    // largest group pairs first: the warps take them in turn
    std::stable_sort(sv.begin(), sv.end(), [](const int4& a, const int4& b) {
      return (a.y & 0xFF) * ((a.y >> 8) & 0xFF) > (b.y & 0xFF) * ((b.y >> 8) & 0xFF);
    });
    meta[q] = int4{ncell, (int)sub.size(), (int)(sub.size() + sv.size()), 0};
    sub.insert(sub.end(), sv.begin(), sv.end());
  }

  // tasks per pass: TJ = the largest power of two (min_tj..16) whose staging
  // fits the pass's per-CTA goal; larger blocks first within a bucket.  The
  // ket pass stages rows of column-major parts in TJ-long runs, so its TJ
  // starts at KET_MIN_TJ_122 (whole 32-byte sectors).
  std::vector<Task122> ht;
  for (int pass = 0; pass < 2; ++pass) {
    const size_t target = pass ? KET_SMEM_TARGET_122 : SMEM_TARGET_122;
    const int min_tj = pass ? KET_MIN_TJ_122 : BRA_MIN_TJ_122;
    const int tjs[5] = {16, 8, 4, 2, 1};
    for (int bkt = 0; bkt < 5; ++bkt) {
      const int tj = tjs[bkt];
      if (tj < min_tj) continue;
      std::vector<std::pair<int, Task122>> v;
      int cmax = 0;
      for (int q = 0; q < L->nblock; ++q) {
        const int nc = meta[q].x;
        if (L->blk[q].w == 0) continue;
        int want = min_tj;
        for (int t : tjs)
          if (t >= min_tj && smem_122(nc, L->blk[q].w, t) <= target) {
            want = t;
            break;
          }
        if (want != tj) continue;
        if (smem_122(nc, L->blk[q].w, tj) > SMEM_MAX_ATTR_122 - SMEM_STATIC_122) {
          set_error("commutator_122: block of %d cells exceeds shared memory", nc);
          return QD_ERR_ARG;
        }
        cmax = std::max(cmax, (int)smem_122(nc, L->blk[q].w, tj));
        const int cnt[3] = {L->blk[q].x, L->blk[q].y, L->blk[q].z};
        for (int c = 0; c < 3; ++c)
          for (int f = 0; f < cnt[c]; f += tj) v.push_back({nc, Task122{q, (short)c, 0, f}});
      }
      if (v.empty()) continue;
      std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
      Bucket122 bk;
      bk.tj = tj;
      bk.first = (int)ht.size();
      bk.count = (int)v.size();
      bk.smem = (size_t)cmax;
      for (auto& x : v) ht.push_back(x.second);
      p.buckets[pass].push_back(bk);
    }
  }
  p.ntask = (int)ht.size();
  auto up = [&](auto& vec, auto** dptr) -> int {
    using T = typename std::decay<decltype(vec[0])>::type;
    QD_CUDA(cudaMalloc(dptr, std::max<size_t>(1, vec.size()) * sizeof(T)));
    if (!vec.empty()) QD_CUDA(cudaMemcpy(*dptr, vec.data(), vec.size() * sizeof(T), cudaMemcpyHostToDevice));
    L->ws_bytes += (i64)(vec.size() * sizeof(T));
    return QD_OK;
  };
  int rc;
  if ((rc = up(ht, &p.d_task)) || (rc = up(meta, &p.d_meta)) || (rc = up(sub, &p.d_sub)) ||
      (rc = up(cell, &p.d_cell)) || (rc = up(sbase, &p.d_sbase)))
    return rc;
  QD_CUDA(cudaMalloc(&p.d_ftab, sizeof(double2) * 2 * (size_t)std::max(1, p.nfent)));
  L->ws_bytes += (i64)sizeof(double2) * 2 * p.nfent;
  if (!p.buckets[0].empty() || !p.buckets[1].empty()) {
    int rc2 = p.gmax <= 10 ? set_attr_122<10>() : set_attr_122<16>();
    if (rc2) return rc2;
  }
  plans()[L] = p;
  *out = &plans()[L];
  return QD_OK;
}

void drop_122_plan(const qd_layout* L) {
  std::lock_guard<std::mutex> lock(g_plan_mutex);
  auto it = plans().find(L);
  if (it == plans().end()) return;
  const Plan122& p = it->second;
  for (void* ptr : {(void*)p.d_task, (void*)p.d_meta, (void*)p.d_sub, (void*)p.d_cell, (void*)p.d_sbase,
                    (void*)p.d_ftab})
    if (ptr) cudaFree(ptr);
  plans().erase(it);
}

int launch_122(qd_layout* L, const qd_op* A, const qd_op* B, double* C) {
  Plan122* p;
  int rc = plan_122(L, &p);
  if (rc) return rc;
  if (p->ntask == 0) return QD_OK;
  const int nf = L->m * p->gmax;
  k_ftab<<<(nf + 127) / 128, 128, 0, L->stream>>>(L->dev, p->d_sbase, A->d, (double)A->herm, B->d,
                                                  (double)B->herm, p->d_ftab, p->gmax, p->nfent);
  ++L->nlaunch;
  if (p->gmax <= 10) {
    pass_122<10, 0>(p, L, A, B, C);
    pass_122<10, 1>(p, L, A, B, C);
  } else {
    pass_122<16, 0>(p, L, A, B, C);
    pass_122<16, 1>(p, L, A, B, C);
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

}  // namespace qd
