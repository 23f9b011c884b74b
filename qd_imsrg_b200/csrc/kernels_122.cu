// kernels_122.cu -- commutator_122 (src/commutators.f90:355-676) as one pass
// over independent group-pair tiles.
//
// In block q the pairs are ordered [hh | ph | pp]; the full block matrix
// V(P1,P2) holds the stored classes (class(P1) >= class(P2)) and herm * their
// transposes above.  For the stored output element <b1 b2|k1 k2> = C(P1,P2):
//   bra legs: C += sum_{t in G(b1)} [FA(b1,t) VB(t b2|P2) - FB(b1,t) VA(t b2|P2)]
//                + sum_{t in G(b2)} [FA(b2,t) VB(b1 t|P2) - FB(b2,t) VA(b1 t|P2)]
//   ket legs: C -= sum_{t in G(k1)} [FA'(k1,t) VB(P1|t k2) - FB'(k1,t) VA(P1|t k2)]
//                + sum_{t in G(k2)} [FA'(k2,t) VB(P1|k1 t) - FB'(k2,t) VA(P1|k1 t)]
// G(x) = states with the (m_l, m_s) of x: the only t whose pair (t,b2) lies in
// block q.  F/F' are the reference's one-body reads (see dev_common.cuh).
//
// Group pairs.  The pairs of block q split into the sets S(g,h) of pairs with
// one state in (m_l,m_s) group g and one in group h (g <= h).  A bra leg of
// a pair in S(g,h) replaces a state by another of the same group, so it stays
// in S(g,h); a ket leg likewise stays in the column pair's set.  Hence the
// block matrix splits into tiles S_a x S_b, and C on tile (a,b) depends only
// on A and B on the same tile and on four small one-body matrices:
//   C[S_a, S_b] = (F_g (x) 1 + 1 (x) F_h) T  -  T (F'_g' (x) 1 + 1 (x) F'_h')^T
// with T the tile in "cell" coordinates: S(g,h) indexed by cells (k1,k2) <->
// (G_g[k1], G_h[k2]), T = +-V of the stored pair (the sign orients the pair;
// when g = h both orientations (k1,k2), (k2,k1) are cells and (k,k) is 0).
//
// Kernel: one CTA per tile.  The tile of each operand needed is gathered with
// cp.async into shared memory (rows of one class of S_a are runs of
// consecutive stored rows, so the gathers coalesce in runs), the orientation
// and herm signs are applied in place, then every stored output cell sums its
// four legs from shared memory and is written once.  C is written exactly
// once (122 overwrites the two-body part), A and B are read once, apart from
// the off-diagonal class blocks, which tiles (a,b) and (b,a) both read.
// When an operand's one-body part has no hh and no pp entries (the Magnus
// generator Omega), F couples holes to particles only: a leg of a hole sums
// over the particles of its group and a leg of a particle over its holes
// (holes are the lowest members of every group).  Tiles whose parts of A are
// known to be zero skip the A term (and then stage B alone).
#include <algorithm>
#include <map>
#include <cstdio>
#include <mutex>
#include <string>
#include <type_traits>

#include "dev_common.cuh"

namespace qd {

#ifndef TRY
#define TRY(x)           \
  do {                   \
    int rc_ = (x);       \
    if (rc_) return rc_; \
  } while (0)
#endif

constexpr size_t SMEM_MAX_122 = 227 * 1024;       // opt-in shared memory per CTA on sm_100

// vectorize slot of the stored part (row class c1 >= column class c2):
// (0,0) hhhh 0, (2,2) pppp 1, (2,0) pphh 2, (1,1) phph 3, (2,1) ppph 4, (1,0) phhh 5
__host__ __device__ __forceinline__ int slot_of(int c1, int c2) {
  if (c1 == 0) return 0;
  if (c1 == 1) return c2 == 0 ? 5 : 3;
  return c2 == 0 ? 2 : (c2 == 1 ? 4 : 1);
}
__device__ __forceinline__ int cnt_of(int c, int4 bd) { return c == 0 ? bd.x : (c == 1 ? bd.y : bd.z); }

// Group-pair descriptor (two int4 per group pair u):
//   d0 = {q, n1 | n2 << 8 | (g == h) << 16, holes(g) | holes(h) << 8, F offset of g}
//   d1 = {F offset of h, first pair entry, 0, cnt_hh | cnt_ph << 10 | cnt_pp << 20}
// Pair entries (int2, sorted by class then index within the class):
//   {index w within its class, primary cell | (mirror cell + 1) << 8 | (sign < 0) << 16 |
//    k1 << 17 | k2 << 21}, the primary cell being (k1, k2) = k1 * n2 + k2
struct GpDesc {
  int q, n1, n2, hg, hh, fg, fh, pstart, cntw;
  // pairs of class c (0 hh, 1 ph, 2 pp), decoded from the packed word (no local array)
  __device__ __forceinline__ int cnt(int c) const { return (cntw >> (10 * c)) & 0x3FF; }
  // pairs of the classes before c
  __device__ __forceinline__ int off(int c) const { return c == 0 ? 0 : (c == 1 ? cnt(0) : cnt(0) + cnt(1)); }
};
__device__ __forceinline__ GpDesc load_gp(const int4* __restrict__ gpd, int u) {
  const int4 a = __ldg(&gpd[2 * u]), b = __ldg(&gpd[2 * u + 1]);
  GpDesc d;
  d.q = a.x;
  d.n1 = a.y & 0xFF;
  d.n2 = (a.y >> 8) & 0xFF;
  d.hg = a.z & 0xFF;
  d.hh = (a.z >> 8) & 0xFF;
  d.fg = a.w;
  d.fh = b.x;
  d.pstart = b.y;
  d.cntw = b.w;
  return d;
}

// Static tables of a layout (built once, see plan_122):
//   sbase[s] = offset of state s's row in the group-major F table
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

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N committed groups of this thread are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// q = a / b and r = a % b for 0 <= a < 2^22 - 1 and b >= 1, through one
// single-precision reciprocal instead of an integer division: the exact value
// of (a + 1/2) / b is q + (r + 1/2) / b, at least 1/(2b) away from an integer,
// and the two correctly rounded float operations err by at most
// (a + 1/2) / b * 2^-23 < 1/(2b); so truncation gives q.
__device__ __forceinline__ int2 divmod_small(int a, int b) {
  const int q = __float2int_rz(((float)a + 0.5f) * __frcp_rn((float)b));
  return make_int2(q, a - q * b);
}

template <int TW>
__device__ __forceinline__ constexpr int xb_of() { return TW == 2 ? 1 : 0; }

// class of a pair from the kinds of its two states: 0 hh, 1 ph, 2 pp
__host__ __device__ __forceinline__ int pair_class(bool hole1, bool hole2) { return (hole1 ? 0 : 1) + (hole2 ? 0 : 1); }

// Whether a leg's sum over the holes (t_hole) or the particles of its group
// can add anything: the one-body factor F(k, t) of a sparse operand (no hh
// and pp entries) couples a hole k only to particles t and a particle only to
// holes; the staged operand must be able to be non-zero on the cells reached,
// whose class pair is (class of (t, other), fixed class) -- nz holds one bit
// per class pair (c1 * 3 + c2, symmetric) of the operand's non-zero parts.
__host__ __device__ __forceinline__ bool leg_ok(int sparse, bool k_hole, bool t_hole, bool other_hole, int cfix,
                                                unsigned nz) {
  if (sparse && k_hole == t_hole) return false;
  return (nz >> (pair_class(t_hole, other_hole) * 3 + cfix)) & 1u;
}

// Bit 31 of a term's leg mask: its one-body factor couples holes to
// particles only, so every leg changes the class of the pair it acts on.
constexpr unsigned LEG_SPARSE = 1u << 31;

// Stored output regions (c1 >= c2) in the order of the output loop:
// (0,0) (1,0) (1,1) (2,0) (2,1) (2,2) -> 0..5; bit r of an output mask.
__host__ __device__ __forceinline__ int out_region(int c1, int c2) { return (c1 * (c1 + 1)) / 2 + c2; }
constexpr unsigned OUT_ALL = 0x3Fu;
// none: k_122_pppp and k_122_gen write every part for a generator-like A
constexpr unsigned OUT_NONE = 0u;

// Regions (c1 * 3 + c2) of the staged operand that the legs of a tile read
// when every leg changes the class of its pair by one: the four neighbours of
// each stored output region (c1 >= c2) of the tile that the launch writes.
// All regions otherwise.
__device__ __forceinline__ unsigned regions_read(unsigned leg, const int ca[3], const int cb[3], unsigned outmask) {
  if (!(leg & LEG_SPARSE)) return 0x1FFu;
  unsigned need = 0;
  for (int c1 = 0; c1 < 3; ++c1)
    for (int c2 = 0; c2 <= c1; ++c2) {
      if (ca[c1] == 0 || cb[c2] == 0 || !((outmask >> out_region(c1, c2)) & 1u)) continue;
      if (c1 > 0) need |= 1u << ((c1 - 1) * 3 + c2);
      if (c1 < 2) need |= 1u << ((c1 + 1) * 3 + c2);
      if (c2 > 0) need |= 1u << (c1 * 3 + c2 - 1);
      if (c2 < 2) need |= 1u << (c1 * 3 + c2 + 1);
    }
  return need;
}

// Sum over t of F(k, t) T[base + t * stride] for one leg: F(k, .) is the
// leg's one-body row (component fy: 0 FA, 1 FB), t runs over the holes
// [0, h) of the leg's group when bit 1 of ok is set and over its particles
// [h, n) when bit 0 is set.
__device__ __forceinline__ double leg_sum(const double2* __restrict__ Frow, int fy, const double* __restrict__ T,
                                          int base, int stride, int n, int h, unsigned ok) {
  const int lo = (ok & 2u) ? 0 : h, hi = (ok & 1u) ? n : h;
  const double* Fd = reinterpret_cast<const double*>(Frow) + fy;
  double y = 0.0;
  for (int t = lo; t < hi; ++t) y += Fd[2 * t] * T[base + t * stride];
  return y;
}

// One instance of a launch that covers several layouts (batched flows): its
// layout view, plan tables, F table and operands.
struct Inst122 {
  DevLayout L;
  const int2* tiles;
  const int4* gpd;
  const int2* gpp;
  const double2* F;
  int nfent;
  const double* A;
  double hA;
  unsigned zA;
  unsigned legA;
  const double* B;
  double hB;
  unsigned zB;
  unsigned legB;
  double* C;
  unsigned outmask;
};

// Task: {tile, op}; op bit 0: the B term (FA x TB), bit 1: the A term
// (-FB x TA), bit 2: accumulate into C instead of setting it.  op & 3 == 0
// writes zeros.  TW = doubles per staged cell: 1 (one operand), 2 (A and B);
// T122 = threads per CTA (picked per launch bucket by the autotuner below).
// MULTI: the tasks come from several layouts and each names its instance in
// tinst (a separate instantiation: the single-layout kernel keeps its
// arguments in the parameter bank instead of registers).
template <int TW, int T122, bool MULTI>
__global__ void __launch_bounds__(T122, 1024 / T122) k_122_tile(DevLayout L, const int2* __restrict__ tasks,
                                                   const int2* __restrict__ tiles, const int4* __restrict__ gpd,
                                                   const int2* __restrict__ gpp,
                                                   const double2* __restrict__ F, int nfent,
                                                   const double* __restrict__ A, double hA, unsigned zA, unsigned legA,
                                                   const double* __restrict__ B, double hB, unsigned zB, unsigned legB,
                                                   double* __restrict__ C, unsigned outmask,
                                                   const int* __restrict__ tinst, const Inst122* __restrict__ insts) {
  extern __shared__ __align__(16) double sm122[];
  if constexpr (MULTI) {  // a task of several layouts' task lists: this instance's tables and operands
    const Inst122& I = insts[tinst[blockIdx.x]];
    L = I.L;
    tiles = I.tiles;
    gpd = I.gpd;
    gpp = I.gpp;
    F = I.F;
    nfent = I.nfent;
    A = I.A;
    hA = I.hA;
    zA = I.zA;
    legA = I.legA;
    B = I.B;
    hB = I.hB;
    zB = I.zB;
    legB = I.legB;
    C = I.C;
    outmask = I.outmask;
  }
  const int2 task = tasks[blockIdx.x];
  const int2 tl = __ldg(&tiles[task.x]);
  const int op = task.y;
  const bool useB = op & 1, useA = (op >> 1) & 1, acc = (op >> 2) & 1;
  const GpDesc da = load_gp(gpd, tl.x), db = load_gp(gpd, tl.y);
  const int q = da.q;
  const int n1 = da.n1, n2 = da.n2, n3 = db.n1, n4 = db.n2;
  const int nr = n1 * n2, nc = n3 * n4, ld = nc | 1;
  const int pa = da.cnt(0) + da.cnt(1) + da.cnt(2), pb = db.cnt(0) + db.cnt(1) + db.cnt(2);
  const int4 bd = __ldg(&L.blk[q]);
  const i64* boff = L.boff + 6 * q;
  // shared memory: T [nr][ld][TW] | F1 F2 F3 F4 (double2) | row, column pairs (int2)
  double* T = sm122;
  const int tsz = (nr * ld * TW + 1) & ~1;
  double2* F1 = reinterpret_cast<double2*>(sm122 + tsz);
  double2* F2 = F1 + n1 * n1;
  double2* F3 = F2 + n2 * n2;
  double2* F4 = F3 + n3 * n3;
  const int tid = threadIdx.x;
  const bool work = useA || useB;
  // a task that writes zeros stages nothing: its shared memory holds the pair lists alone
  int2* pr = work ? reinterpret_cast<int2*>(F4 + n4 * n4) : reinterpret_cast<int2*>(sm122);
  int2* pc = pr + pa;

  if (work) {
    for (int i = tid; i < n1 * n1; i += T122) F1[i] = __ldg(&F[da.fg + i]);
    for (int i = tid; i < n2 * n2; i += T122) F2[i] = __ldg(&F[da.fh + i]);
    for (int i = tid; i < n3 * n3; i += T122) F3[i] = __ldg(&F[nfent + db.fg + i]);
    for (int i = tid; i < n4 * n4; i += T122) F4[i] = __ldg(&F[nfent + db.fh + i]);
  }
  for (int i = tid; i < pa; i += T122) pr[i] = __ldg(&gpp[da.pstart + i]);
  for (int i = tid; i < pb; i += T122) pc[i] = __ldg(&gpp[db.pstart + i]);
  __syncthreads();

  if (work) {
    // Cells that no stored element reaches -- the (t,t) cells of g = h and
    // the parts known to be zero -- stay 0: zero the tile first.
    for (int i = 2 * tid; i < tsz; i += 2 * T122) *reinterpret_cast<double2*>(T + i) = make_double2(0.0, 0.0);
    __syncthreads();
    // gather: region (c1 rows of S_a, c2 columns of S_b); the stored element
    // is (P1,P2) of part (c1,c2) when c1 >= c2, else (P2,P1) of part (c2,c1),
    // taken with herm.  It lands on its cell with the orientation sign of the
    // two pairs, and on the mirror cells (g = h) with the opposite ones.
    // The loops stay rolled: the kernel's code must fit the instruction cache.
    int ca[3], cb[3];
    for (int c = 0; c < 3; ++c) {
      ca[c] = da.cnt(c);
      cb[c] = db.cnt(c);
    }
#pragma unroll 1
    for (int x = 0; x < 2; ++x) {
      if (x == 0 ? !useA : !useB) continue;
      const double* src = x == 0 ? A : B;
      const unsigned zm = x == 0 ? zA : zB;
      // the A term's legs carry FB (legA), the B term's FA (legB)
      const unsigned need = regions_read(x == 0 ? legA : legB, ca, cb, outmask);
      const double hx = x == 0 ? hA : hB;
      const int xo = TW == 2 ? x : 0;
#pragma unroll 1
      for (int rg = 0; rg < 9; ++rg) {
        const int c1 = rg / 3, c2 = rg - 3 * c1;
        const int r1 = da.cnt(c1), r2 = db.cnt(c2);
        const bool lower = c1 >= c2;
        const int part = lower ? slot_of(c1, c2) : slot_of(c2, c1);
        if (r1 == 0 || r2 == 0 || ((zm >> (P_HHHH + part)) & 1u) || !((need >> rg) & 1u)) continue;
        const int o1 = da.off(c1), o2 = db.off(c2);
        const double* srcp = src + __ldg(boff + part);
        const i64 ldv = lower ? cnt_of(c1, bd) : cnt_of(c2, bd);
        const double hf = lower ? 1.0 : hx;
        const int total = r1 * r2;
        // e = fast + nf * slow, walked without dividing: the memory-contiguous
        // index (rows for stored parts, columns for transposed ones) is fast
        const int nf = lower ? r1 : r2;
        const int2 i0 = divmod_small(tid, nf), di = divmod_small(T122, nf);
        int fa = i0.y, sl = i0.x;
        const int dfa = di.y, dsl = di.x;
#pragma unroll 4
        for (int e = tid; e < total; e += T122) {
          const int p = lower ? fa : sl, u = lower ? sl : fa;
          fa += dfa;
          sl += dsl;
          if (fa >= nf) {
            fa -= nf;
            ++sl;
          }
          const int2 P = pr[o1 + p], Q = pc[o2 + u];
          const i64 addr = lower ? P.x + (i64)Q.x * ldv : Q.x + (i64)P.x * ldv;
          const double v = hf * __ldg(srcp + addr);
          const double sv = ((P.y ^ Q.y) & (1 << 16)) ? -v : v;
          const int r = P.y & 0xFF, rm = ((P.y >> 8) & 0xFF) - 1;
          const int s = Q.y & 0xFF, sm = ((Q.y >> 8) & 0xFF) - 1;
          T[(r * ld + s) * TW + xo] = sv;
          if (rm >= 0) T[(rm * ld + s) * TW + xo] = -sv;
          if (sm >= 0) {
            T[(r * ld + sm) * TW + xo] = -sv;
            if (rm >= 0) T[(rm * ld + sm) * TW + xo] = sv;
          }
        }
      }
    }
    __syncthreads();
  }

  // stored output cells: regions with c1 >= c2, rows of S_a fastest
#pragma unroll 1
  for (int rg = 0; rg < 6; ++rg) {
    const int c1 = rg < 1 ? 0 : (rg < 3 ? 1 : 2), c2 = rg - (c1 * (c1 + 1)) / 2;  // (0,0) (1,0) (1,1) (2,0) (2,1) (2,2)
    const int r1 = da.cnt(c1), r2 = db.cnt(c2);
    if (r1 == 0 || r2 == 0 || !((outmask >> rg) & 1u)) continue;
    const int o1 = da.off(c1), o2 = db.off(c2);
    const i64 base = __ldg(boff + slot_of(c1, c2));
    const i64 ldc = cnt_of(c1, bd);
    // leg masks of this region (see leg_masks): bra legs fix class c2, ket legs c1
    const unsigned okB = ((legB >> (8 * c2)) & 0xFFu) | (((legB >> (8 * c1)) & 0xFFu) << 8);
    const unsigned okA = ((legA >> (8 * c2)) & 0xFFu) | (((legA >> (8 * c1)) & 0xFFu) << 8);
    const int2 i0 = divmod_small(tid, r1), di = divmod_small(T122, r1);
    int p = i0.y, u = i0.x;
    const int dp = di.y, du = di.x;
    for (int e = tid; e < r1 * r2; e += T122) {
      const int2 P = pr[o1 + p], Q = pc[o2 + u];
      p += dp;
      u += du;
      if (p >= r1) {
        p -= r1;
        ++u;
      }
      double y = 0.0;
      if (work) {
        const int r = P.y & 0xFF, s = Q.y & 0xFF;
        const int k1 = (P.y >> 17) & 15, k2 = (P.y >> 21) & 15;
        const int l1 = (Q.y >> 17) & 15, l2 = (Q.y >> 21) & 15;
        const int h1 = k1 < da.hg, h2 = k2 < da.hh, h3 = l1 < db.hg, h4 = l2 < db.hh;
        const int b1 = h1 * 4 + h2 * 2, b2 = h2 * 4 + h1 * 2, b3 = 8 + h3 * 4 + h4 * 2, b4 = 8 + h4 * 4 + h3 * 2;
        const int bL1 = (k2 * ld + s) * TW, sL1 = n2 * ld * TW;  // T((t,k2), s)
        const int bL2 = (k1 * n2 * ld + s) * TW, sL2 = ld * TW;  // T((k1,t), s)
        const int bL3 = (r * ld + l2) * TW, sL3 = n4 * TW;       // T(r, (t,l2))
        const int bL4 = (r * ld + l1 * n4) * TW, sL4 = TW;       // T(r, (l1,t))
        if (useB) {  // FA x TB
          const double* Tb = T + xb_of<TW>();
          y += leg_sum(F1 + k1 * n1, 0, Tb, bL1, sL1, n1, da.hg, okB >> b1);
          y += leg_sum(F2 + k2 * n2, 0, Tb, bL2, sL2, n2, da.hh, okB >> b2);
          y -= leg_sum(F3 + l1 * n3, 0, Tb, bL3, sL3, n3, db.hg, okB >> b3);
          y -= leg_sum(F4 + l2 * n4, 0, Tb, bL4, sL4, n4, db.hh, okB >> b4);
        }
        if (useA) {  // -FB x TA
          y -= leg_sum(F1 + k1 * n1, 1, T, bL1, sL1, n1, da.hg, okA >> b1);
          y -= leg_sum(F2 + k2 * n2, 1, T, bL2, sL2, n2, da.hh, okA >> b2);
          y += leg_sum(F3 + l1 * n3, 1, T, bL3, sL3, n3, db.hg, okA >> b3);
          y += leg_sum(F4 + l2 * n4, 1, T, bL4, sL4, n4, db.hh, okA >> b4);
        }
        if ((P.y ^ Q.y) & (1 << 16)) y = -y;
      }
      double* out = C + base + P.x + (i64)Q.x * ldc;
      if (acc)
        *out += y;
      else
        *out = y;
    }
  }
}

// ---- commutator_122 for a generator-like A --------------------------------
// When A's one-body part holds only fph (no hh or pp entries) and its
// two-body part only Vpphh -- the Magnus generator Omega, the White
// generator eta -- the leg sums above collapse, on the two largest output
// parts of a block, to a few columns (or rows) of B each: every term dropped
// is an exact zero (FA couples holes to particles only; A's other parts are
// zero).  With fA(p, h) = A's fph, fB(p, h) = B's fph, pairs indexed within
// the block, s the ordering sign of a pair (v_elem's), hA, hB the herm
// factors and only holes t in G(x) or particles as stated:
//   C_pppp = hB W^T - hA W,
//     W(:, (a,b)) = sum_{t in G(a)} fA(a,t) B_ppph(:, (t,b)) - sum_{t in G(b)} fA(b,t) B_ppph(:, (t,a));
//   C_ppph(:, (h,p)) = - sum_{particles t in G(h)} s fA(t,h) B_pppp(:, (t,p))
//                      - sum_{t in G(p)} s [hA fA(p,t) B_pphh(:, (h,t)) - hB fB(p,t) A_pphh(:, (h,t))]
//   C_ppph((a,b), :) += sum_{t in G(a)} fA(a,t) B_phph((t,b), :) - sum_{t in G(b)} fA(b,t) B_phph((t,a), :).
// (Both checked against the oracle's commutator_122 in numpy before this
// kernel was written.)  B_ppph and B_phph are small (L2 resident); the
// kernels stream C_pppp and C_ppph out once.  Term tables (per layout):
//   pp pair: {ph index of (t, b) or (t, a), t | (a or b - n) << 8 | neg << 20}
//   ph pair: {column, hole | (particle - n) << 8 | neg << 20, kind}: kind 0 a
//            B_pppp column with coefficient -s fA(t, h); kind 1 an hh column
//            (h, t) of B_pphh and A_pphh.
__host__ __device__ __forceinline__ bool gen_like(unsigned zmask) {
  return (zmask | (1u << P_FPH) | (1u << P_PPHH)) == ALL_PARTS;
}

constexpr int SP_T = 256, SP_B = 64, SP_LD = SP_B + 1;
// k_122_pppp tiles: 32 x 32 (two W tiles of 8.4 KB per CTA: seven CTAs per SM)
constexpr int PP_B = 32, PP_LD = PP_B + 1;

__device__ __forceinline__ double sp_coef(const DevLayout& L, const double* __restrict__ f, int code) {
  const double v = __ldg(&f[L.o_fph + ((code >> 8) & 0xFFF) + (i64)(code & 0xFF) * L.mp]);
  return (code >> 20) & 1 ? -v : v;
}

// A term staged in shared memory: its coefficient, and the source element
// off + fixed * (m & MULT_MASK) of operand B (bit 30 of m set) or A.
struct StagedTerm {
  double c;
  int off, m;
};
constexpr int MULT_MASK = 0x3FFFFFFF;

// One task = the tile pair (I, J), (J, I) of a block's C_pppp (32 x 32 each).
// The W terms of the tile's columns (J, then I) are staged in shared memory
// first, with their coefficients resolved; each W element then reads only
// its B_ppph entries.
__global__ void __launch_bounds__(SP_T) k_122_pppp(DevLayout L, const int4* __restrict__ tasks,
                                                  const int* __restrict__ ppbase, const int* __restrict__ ppstart,
                                                  const int2* __restrict__ ppterm, const double* __restrict__ A,
                                                  double hA, const double* __restrict__ B, double hB, unsigned zB,
                                                  double* __restrict__ C) {
  extern __shared__ __align__(16) double spw[];  // W1[c][r] = W(I0 + r, J0 + c), W2[c][r] = W(J0 + r, I0 + c), terms
  __shared__ int sst[2][PP_B + 1];               // per pass: each column's first staged term
  const int4 t = tasks[blockIdx.x];
  const int q = t.x, I0 = t.y * PP_B, J0 = t.z * PP_B;
  const int4 bd = __ldg(&L.blk[q]);
  const int np = bd.z;
  const i64* boff = L.boff + 6 * q;
  const bool live = !((zB >> P_PPPH) & 1u);
  const double* X = B + __ldg(boff + 4);  // B_ppph, np x nph
  const int pb = __ldg(&ppbase[q]);
  const int tid = threadIdx.x, r = tid & (PP_B - 1), cg = tid >> 5;
  const bool diag = t.y == t.z;
  const int npass = diag ? 1 : 2;
  StagedTerm* T = reinterpret_cast<StagedTerm*>(spw + 2 * PP_B * PP_LD);
  int base = 0;
  for (int pass = 0; pass < npass; ++pass) {
    const int C0 = pass == 0 ? J0 : I0, nc = live ? min(PP_B, np - C0) : 0;
    const int e0 = __ldg(&ppstart[pb + C0]);
    for (int i = tid; i <= PP_B; i += SP_T) sst[pass][i] = base + (i <= nc ? __ldg(&ppstart[pb + C0 + i]) : __ldg(&ppstart[pb + C0 + nc])) - e0;
    const int ne = nc > 0 ? __ldg(&ppstart[pb + C0 + nc]) - e0 : 0;
    for (int i = tid; i < ne; i += SP_T) {
      const int2 tm = __ldg(&ppterm[e0 + i]);
      T[base + i] = StagedTerm{sp_coef(L, A, tm.y), tm.x * np, 0};
    }
    base += ne;
  }
  __syncthreads();
  for (int pass = 0; pass < npass; ++pass) {
    const int R0 = pass == 0 ? I0 : J0;
    double* W = spw + pass * PP_B * PP_LD;
    const int row = R0 + r;
    for (int cc = cg; cc < PP_B; cc += SP_T / PP_B) {
      double w = 0.0;
      if (row < np)
        for (int e = sst[pass][cc]; e < sst[pass][cc + 1]; ++e) w += T[e].c * X[row + (i64)T[e].off];
      W[cc * PP_LD + r] = w;
    }
  }
  __syncthreads();
  const double* W1 = spw;
  const double* W2 = diag ? spw : spw + PP_B * PP_LD;
  double* out = C + __ldg(boff + 1);
  for (int idx = tid; idx < PP_B * PP_B; idx += SP_T) {
    const int rr = idx & (PP_B - 1), c = idx >> 5;
    if (I0 + rr < np && J0 + c < np)  // C(I0 + rr, J0 + c) = hB W(J0 + c, I0 + rr) - hA W(I0 + rr, J0 + c)
      out[(I0 + rr) + (i64)(J0 + c) * np] = hB * W2[rr * PP_LD + c] - hA * W1[c * PP_LD + rr];
  }
  if (diag) return;
  for (int idx = tid; idx < PP_B * PP_B; idx += SP_T) {
    const int rr = idx & (PP_B - 1), c = idx >> 5;
    if (J0 + rr < np && I0 + c < np)  // C(J0 + rr, I0 + c) = hB W(I0 + c, J0 + rr) - hA W(J0 + rr, I0 + c)
      out[(J0 + rr) + (i64)(I0 + c) * np] = hB * W1[rr * PP_LD + c] - hA * W2[c * PP_LD + rr];
  }
}

// The other five parts of a block for a generator-like A, one 64 x 64 tile
// of one part per task {q, part, ti, tj}: every output element (R, c) is
//   sum over the terms of its row pair of coef * M[idx + c ld] (M[c + idx ld] transposed)
// + sum over the terms of its column pair of coef * M[R + idx ld] (M[idx + R ld] transposed),
// M a stored part of A or B in block q with ld rows.  Term {idx, coefficient
// offset, flags, source}: flags bit 0 negate, 1 times hA, 2 times hB, 3 the
// coefficient is B's entry (else A's); source (operand << 4) | (T << 3) | slot.
// The closed forms (derived from the leg sums, each checked against the
// oracle's commutator_122 in numpy first), with s an ordering sign:
//   ppph rows (a,b): +-fA(a|b,t) B_phph((t,b|a), .);  columns (h,p):
//        -s fA(t,h) B_pppp(., (t,p)) [particles t in G(h)],
//        -s hA fA(p,t) B_pphh(., (h,t)) + s hB fB(p,t) A_pphh(., (h,t)) [holes t in G(p)]
//   pphh rows (a,b): +-fA(a|b,t) B_phhh((t,b|a), .) - s hB fppB(t,a|b) A_pphh((t,b)|(a,t), .);
//        columns (k,l): +-fA(t,k|l) B_ppph(., (l|k,t)) + s hB fhhB(k|l,t) A_pphh(., (t,l)|(k,t))
//   phhh rows (h,p): s hA fA(t,h) B_pphh((t,p), .) - s hB fB(t,h) A_pphh((t,p), .) + s fA(p,t) B_hhhh((h,t), .);
//        columns (k,l): +-fA(t,k|l) B_phph(., (l|k,t))
//   phph rows (h,p): s hA fA(t,h) B_ppph((t,p), .) + s hB fA(p,t) B_phhh(., (h,t))^T;
//        columns (k,l): -s hB fA(t,k) B_ppph((t,l), .)^T - s hA fA(l,t) B_phhh(., (k,t))
//   hhhh rows (a,b): -+hA fA(t,a|b) B_phhh((b|a,t), .);  columns (k,l): +-hB fA(t,k|l) B_phhh((l|k,t), .)^T
struct GenTables {
  const int* gbase;   // 3 * nblock: first hh, ph, pp pair of each block
  const int* rstart;  // per part: per row pair its first term (one more entry at the end)
  const int* cstart;
  const int4* rterm;
  const int4* cterm;
  int rso[6], cso[6];  // offset of each part's start array (slot order)
};

// Resolve a term for one tile: its coefficient and its source element as
// off + fixed * m (row term: fixed = output column; column term: output row).
__device__ __forceinline__ StagedTerm stage_term(const DevLayout& L, const int4& tm, int q, int4 bd, bool row_term,
                                                 const double* __restrict__ A, double hA,
                                                 const double* __restrict__ B, double hB) {
  const int opd = tm.w >> 4, slot = tm.w & 7;
  const bool tr = (tm.w >> 3) & 1;
  const int ld = part_rows(P_HHHH + slot, bd);
  const int bo = (int)__ldg(L.boff + 6 * q + slot);
  StagedTerm st;
  if (row_term != tr) {
    st.off = bo + tm.x;
    st.m = ld;
  } else {
    st.off = bo + tm.x * ld;
    st.m = 1;
  }
  st.m |= opd << 30;
  double c = __ldg(&((tm.z >> 3) & 1 ? B : A)[tm.y]);
  if (tm.z & 2) c *= hA;
  if (tm.z & 4) c *= hB;
  if (tm.z & 1) c = -c;
  st.c = c;
  return st;
}

// The tile's column terms, then its row terms, are staged once per CTA in
// shared memory (dynamic size: the most terms of any tile of the launch).
__global__ void __launch_bounds__(SP_T) k_122_gen(DevLayout L, const int4* __restrict__ tasks, GenTables G,
                                                 const double* __restrict__ A, double hA,
                                                 const double* __restrict__ B, double hB,
                                                 double* __restrict__ C) {
  extern __shared__ __align__(16) double sgt[];
  StagedTerm* T = reinterpret_cast<StagedTerm*>(sgt);
  __shared__ int scs[SP_B + 1], srs[SP_B + 1];
  const int4 t = tasks[blockIdx.x];
  const int q = t.x, slot = t.y, I0 = t.z * SP_B, J0 = t.w * SP_B;
  const int4 bd = __ldg(&L.blk[q]);
  int cr, cc;
  part_classes(P_HHHH + slot, cr, cc);
  const int nrow = part_rows(P_HHHH + slot, bd), ncol = cc == 0 ? bd.x : (cc == 1 ? bd.y : bd.z);
  const int nrt = min(SP_B, nrow - I0), nct = min(SP_B, ncol - J0);
  const int* rs = G.rstart + G.rso[slot] + __ldg(&G.gbase[cr * L.nblock + q]) + I0;
  const int* cs = G.cstart + G.cso[slot] + __ldg(&G.gbase[cc * L.nblock + q]) + J0;
  const int c0 = __ldg(&cs[0]), nce = __ldg(&cs[nct]) - c0;
  const int r0 = __ldg(&rs[0]), nre = __ldg(&rs[nrt]) - r0;
  const int tid = threadIdx.x;
  for (int i = tid; i <= SP_B; i += SP_T) {
    scs[i] = __ldg(&cs[min(i, nct)]) - c0;
    srs[i] = nce + __ldg(&rs[min(i, nrt)]) - r0;
  }
  for (int i = tid; i < nce; i += SP_T) T[i] = stage_term(L, __ldg(&G.cterm[c0 + i]), q, bd, false, A, hA, B, hB);
  for (int i = tid; i < nre; i += SP_T) T[nce + i] = stage_term(L, __ldg(&G.rterm[r0 + i]), q, bd, true, A, hA, B, hB);
  __syncthreads();
  const int r = tid & (SP_B - 1), cg = tid >> 6;
  if (r >= nrt) return;  // after the only barrier
  const int row = I0 + r;
  const int er0 = srs[r], er1 = srs[r + 1];
  double* out = C + __ldg(L.boff + 6 * q + slot);
  for (int k = cg; k < nct; k += SP_T / SP_B) {
    const int col = J0 + k;
    double y = 0.0;
    for (int e = scs[k]; e < scs[k + 1]; ++e) {
      const StagedTerm s = T[e];
      y += s.c * ((s.m >> 30) ? B : A)[s.off + (i64)row * (s.m & MULT_MASK)];
    }
    for (int e = er0; e < er1; ++e) {
      const StagedTerm s = T[e];
      y += s.c * ((s.m >> 30) ? B : A)[s.off + (i64)col * (s.m & MULT_MASK)];
    }
    out[row + (i64)col * nrow] = y;
  }
}

// ---- particle-hole channel of commutator_222 over the same tiles ----------
// (src/commutators.f90:716-980, ME_general.f90:923-952.)  With Z = XCC - YCC
// in cross-coupled coordinates and the stored output element oriented as the
// cells (k1,k2) of S(g,h), (l1,l2) of S(g',h') -- states x = G_g[k1],
// y = G_h[k2], u = G_g'[l1], v = G_h'[l2] --
//   C += Z[(u,x),(y,v)] - Z[(u,y),(x,v)] + Z[(v,y),(x,u)] - Z[(v,x),(y,u)].
// The cc rows are group-major (all rows (i in G1, j in G2) form one run), so
// each term reads one dense sub-matrix of one cc block: rows G1 x G2 (one run
// of |G1||G2| doubles per column), columns G3 x G4.  Term t (sign (-1)^t):
//   t  rows (G1,G2)  columns (G3,G4)  element (rows; columns)
//   0  (g', g)       (h, h')          (l1,k1; k2,l2)
//   1  (g', h)       (g, h')          (l1,k2; k1,l2)
//   2  (h', h)       (g, g')          (l2,k2; k1,l1)
//   3  (h', g)       (h, g')          (l2,k1; k2,l1)
// Modes (per launch bucket, by the tile's size):
//   PD_ALL4   the four sub-matrices staged at once (one wait), one pass over
//             the stored cells adds the four elements into C;
//   PD_PAIRS  two buffers: terms 0,1 in flight, then term t+2 is copied
//             while term t is added into a shared accumulator per cell;
//   PD_SINGLE one buffer and the accumulator, the terms one after another;
//   PD_DIRECT no staging: each cell reads its four elements from global
//             memory (tiles too large for the others).
// Every cell adds the four terms in the order 0, 1, 2, 3 in all modes.
constexpr int TPD = 256;
enum { PD_DIRECT = 0, PD_ALL4 = 1, PD_PAIRS = 2, PD_SINGLE = 3 };

struct PdTerm {  // geometry of one term's sub-matrix
  const double* zb;  // element (0, 0)
  i64 ldz;           // leading dimension of the cc block
  int nrow, ncol, m2, m4;
};

__device__ __forceinline__ PdTerm pd_term(int t, const DevLayout& L, const int2* __restrict__ zrow, int ng,
                                          const double* __restrict__ Z, int2 gb, int2 gk, int n1, int n2, int n3,
                                          int n4) {
  int G1, G2, G3, G4, m1, m3;
  PdTerm d;
  if (t == 0) {
    G1 = gk.x; G2 = gb.x; G3 = gb.y; G4 = gk.y; m1 = n3; d.m2 = n1; m3 = n2; d.m4 = n4;
  } else if (t == 1) {
    G1 = gk.x; G2 = gb.y; G3 = gb.x; G4 = gk.y; m1 = n3; d.m2 = n2; m3 = n1; d.m4 = n4;
  } else if (t == 2) {
    G1 = gk.y; G2 = gb.y; G3 = gb.x; G4 = gk.x; m1 = n4; d.m2 = n2; m3 = n1; d.m4 = n3;
  } else {
    G1 = gk.y; G2 = gb.x; G3 = gb.y; G4 = gk.x; m1 = n4; d.m2 = n1; m3 = n2; d.m4 = n3;
  }
  const int2 zr = __ldg(&zrow[G1 * ng + G2]);
  const int cs = __ldg(&zrow[G3 * ng + G4]).y;
  d.ldz = __ldg(&L.ccdim[zr.x]).x;
  d.zb = Z + __ldg(&L.cczoff[zr.x]) + zr.y + (i64)cs * d.ldz;
  d.nrow = m1 * d.m2;
  d.ncol = m3 * d.m4;
  return d;
}

// (row, column) of the cell's element in term t's sub-matrix
__device__ __forceinline__ int2 pd_rc(int t, const PdTerm& d, int k1, int k2, int l1, int l2) {
  if (t == 0) return make_int2(l1 * d.m2 + k1, k2 * d.m4 + l2);
  if (t == 1) return make_int2(l1 * d.m2 + k2, k1 * d.m4 + l2);
  if (t == 2) return make_int2(l2 * d.m2 + k2, k1 * d.m4 + l1);
  return make_int2(l2 * d.m2 + k1, k2 * d.m4 + l1);
}
// its position in the staged copy (column-major, nrow rows)
__device__ __forceinline__ int pd_index(int t, const PdTerm& d, int k1, int k2, int l1, int l2) {
  const int2 ij = pd_rc(t, d, k1, k2, l1, l2);
  return ij.x + ij.y * d.nrow;
}

// copy term d's sub-matrix into dst (runs of nrow doubles, coalesced)
__device__ __forceinline__ void pd_stage(const PdTerm& d, double* dst, int tid) {
  const int total = d.nrow * d.ncol;
  const int2 i0 = divmod_small(tid, d.nrow), di = divmod_small(TPD, d.nrow);
  int fr = i0.y, fc = i0.x;
  for (int e = tid; e < total; e += TPD) {
    cp_async8(&dst[e], d.zb + fr + (i64)fc * d.ldz);
    fr += di.y;
    fc += di.x;
    if (fr >= d.nrow) {
      fr -= d.nrow;
      ++fc;
    }
  }
}

template <int MODE>
__global__ void __launch_bounds__(TPD) k_pandya_tile(DevLayout L, const int* __restrict__ tasks,
                                                     const int2* __restrict__ tiles, const int4* __restrict__ gpd,
                                                     const int2* __restrict__ gpp, const int2* __restrict__ gpg,
                                                     const int2* __restrict__ zrow, int ng,
                                                     const double* __restrict__ Z, double* __restrict__ C) {
  extern __shared__ __align__(16) double smp[];
  const int2 tl = __ldg(&tiles[__ldg(&tasks[blockIdx.x])]);
  const GpDesc da = load_gp(gpd, tl.x), db = load_gp(gpd, tl.y);
  const int2 gb = __ldg(&gpg[tl.x]), gk = __ldg(&gpg[tl.y]);  // (g, h), (g', h')
  const int n1 = da.n1, n2 = da.n2, n3 = db.n1, n4 = db.n2;
  const int cells = n1 * n2 * n3 * n4;
  const int pa = da.cnt(0) + da.cnt(1) + da.cnt(2), pb = db.cnt(0) + db.cnt(1) + db.cnt(2);
  const int q = da.q;
  const int4 bd = __ldg(&L.blk[q]);
  const i64* boff = L.boff + 6 * q;
  int nst = 0;  // stored cells: regions c1 >= c2
#pragma unroll 1
  for (int c1 = 0; c1 < 3; ++c1)
    for (int c2 = 0; c2 <= c1; ++c2) nst += da.cnt(c1) * db.cnt(c2);
  // shared memory: sub-matrix buffers | accumulator | row, column pairs
  constexpr int NBUF = MODE == PD_ALL4 ? 4 : (MODE == PD_PAIRS ? 2 : (MODE == PD_SINGLE ? 1 : 0));
  constexpr bool ACCUM = MODE == PD_PAIRS || MODE == PD_SINGLE;
  double* Zs = smp;
  double* Y = smp + NBUF * cells;
  int2* pr = reinterpret_cast<int2*>(Y + (ACCUM ? nst : 0));
  int2* pc = pr + pa;
  const int tid = threadIdx.x;
  for (int i = tid; i < pa; i += TPD) pr[i] = __ldg(&gpp[da.pstart + i]);
  for (int i = tid; i < pb; i += TPD) pc[i] = __ldg(&gpp[db.pstart + i]);
  PdTerm d[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) d[t] = pd_term(t, L, zrow, ng, Z, gb, gk, n1, n2, n3, n4);
  if (MODE == PD_ALL4) {
#pragma unroll
    for (int t = 0; t < 4; ++t) pd_stage(d[t], Zs + t * cells, tid);
    cp_async_wait_all();
  } else if (MODE == PD_PAIRS) {
    pd_stage(d[0], Zs, tid);
    cp_async_commit();
    pd_stage(d[1], Zs + cells, tid);
    cp_async_commit();
    cp_async_wait_group<1>();
  } else if (MODE == PD_SINGLE) {
    pd_stage(d[0], Zs, tid);
    cp_async_wait_all();
  }
  __syncthreads();

  // passes over the stored cells: ALL4 and DIRECT one (all terms), PAIRS and
  // SINGLE one per term
  constexpr int NPASS = ACCUM ? 4 : 1;
#pragma unroll 1
  for (int pass = 0; pass < NPASS; ++pass) {
    const double* buf = Zs + (MODE == PD_PAIRS ? (pass & 1) * cells : 0);
    // this pass's term geometry (recomputed: an array indexed by the pass
    // would live in local memory)
    const PdTerm dp = ACCUM ? pd_term(pass, L, zrow, ng, Z, gb, gk, n1, n2, n3, n4) : d[0];
    int j0 = 0;  // first accumulator slot of the region
#pragma unroll 1
    for (int rg = 0; rg < 6; ++rg) {
      const int c1 = rg < 1 ? 0 : (rg < 3 ? 1 : 2), c2 = rg - (c1 * (c1 + 1)) / 2;
      const int r1 = da.cnt(c1), r2 = db.cnt(c2);
      if (r1 == 0 || r2 == 0) continue;
      const int o1 = da.off(c1), o2 = db.off(c2);
      const i64 base = __ldg(boff + slot_of(c1, c2));
      const i64 ldc = cnt_of(c1, bd);
      const int2 i0 = divmod_small(tid, r1), di = divmod_small(TPD, r1);
      int p = i0.y, u = i0.x;
      for (int e = tid; e < r1 * r2; e += TPD) {
        const int2 P = pr[o1 + p], Q = pc[o2 + u];
        p += di.y;
        u += di.x;
        if (p >= r1) {
          p -= r1;
          ++u;
        }
        const int k1 = (P.y >> 17) & 15, k2 = (P.y >> 21) & 15;
        const int l1 = (Q.y >> 17) & 15, l2 = (Q.y >> 21) & 15;
        double y;
        bool last = true;
        if (MODE == PD_ALL4) {
          y = Zs[pd_index(0, d[0], k1, k2, l1, l2)];
          y -= Zs[cells + pd_index(1, d[1], k1, k2, l1, l2)];
          y += Zs[2 * cells + pd_index(2, d[2], k1, k2, l1, l2)];
          y -= Zs[3 * cells + pd_index(3, d[3], k1, k2, l1, l2)];
        } else if (MODE == PD_DIRECT) {
          double z[4];
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const int2 ij = pd_rc(t, d[t], k1, k2, l1, l2);
            z[t] = __ldg(d[t].zb + ij.x + (i64)ij.y * d[t].ldz);
          }
          y = z[0] - z[1] + z[2] - z[3];
        } else {
          const double z = buf[pd_index(pass, dp, k1, k2, l1, l2)];
          y = (pass == 0 ? 0.0 : Y[j0 + e]) + ((pass & 1) ? -z : z);
          last = pass == 3;
          if (!last) Y[j0 + e] = y;
        }
        if (last) {
          if ((P.y ^ Q.y) & (1 << 16)) y = -y;
          C[base + P.x + (i64)Q.x * ldc] += y;
        }
      }
      j0 += r1 * r2;
    }
    if (MODE == PD_PAIRS && pass < 3) {
      __syncthreads();  // buffer (pass & 1) is free again
      if (pass < 2) {   // term pass + 2 into it, while term pass + 1 lands
        pd_stage(pd_term(pass + 2, L, zrow, ng, Z, gb, gk, n1, n2, n3, n4), Zs + (pass & 1) * cells, tid);
        cp_async_commit();
        cp_async_wait_group<1>();
      } else {
        cp_async_wait_group<0>();
      }
      __syncthreads();
    } else if (MODE == PD_SINGLE && pass < 3) {
      __syncthreads();
      pd_stage(pd_term(pass + 1, L, zrow, ng, Z, gb, gk, n1, n2, n3, n4), Zs, tid);
      cp_async_wait_all();
      __syncthreads();
    }
  }
}

// ---- host side --------------------------------------------------------------
namespace {
struct TileInfo {
  int a, b;          // group pairs
  int cells;         // nr * nc
  int nf, npair;     // F entries (double2) and pair entries of the two group pairs
  int nr, nc;
  unsigned parts;    // two-body parts the tile touches (bit = vectorize slot)
  int nst;           // stored output cells
  bool holefree;     // none of the four (m_l, m_s) groups holds a hole
  unsigned outs;     // stored output regions of the tile (bit out_region(c1, c2))
};
struct PdBucket {  // one launch of the particle-hole tile kernel
  int first, count;
  size_t smem;
  int mode;  // PD_ALL4, PD_PAIRS, PD_SINGLE or PD_DIRECT
};
struct Bucket122 {
  int tw;       // doubles per staged cell
  int first;    // range in the task array
  int count;
  size_t smem;
  int list = 0;          // 0 one operand (sets C), 1 both operands, 2 one operand (accumulates)
  int threads = 256;    // CTA size (autotuned)
  float ms[3] = {0, 0, 0};  // measured time of the 64-, 128- and 256-thread variants
};
struct TaskSet {
  int2* d_task = nullptr;
  std::vector<int2> h_task;  // host copy (merged launches of several layouts)
  std::vector<Bucket122> buckets;
  bool tuned = false;
  unsigned outmask = OUT_ALL;  // output regions the tiles write (OUT_NONE: A generator-like)
  int bounds_id = 0;           // which bucketing (see kBounds) the tuner kept
  float ms_total = 0.f;        // tuned time of this bucketing
  std::vector<TaskSet> alts;   // the other bucketings, until tuned
};
struct Plan122 {
  int4* d_gpd = nullptr;
  int2* d_gpp = nullptr;
  int2* d_tiles = nullptr;
  int* d_sbase = nullptr;
  double2* d_ftab = nullptr;
  int gmax = 0, nfent = 0;
  std::vector<TileInfo> tiles;
  std::map<std::pair<unsigned, unsigned>, TaskSet> sets;  // per (zero mask A, zero mask B)
  // particle-hole channel: groups (g, h) of each group pair, the first cc row
  // of each group pair (G1, G2) as {cc block, row}, the tasks (tile indices)
  int2* d_gpg = nullptr;
  int2* d_zrow = nullptr;
  int ng = 0;
  int* d_ptask = nullptr;
  std::vector<PdBucket> pbuckets;
  // generator-like A: term tables of k_122_pppp / k_122_gen and their tasks
  int* d_ppbase = nullptr;   // per block: first pp pair
  int* d_ppstart = nullptr;  // per pp pair: first term (one more entry at the end)
  int2* d_ppterm = nullptr;
  int* d_gbase = nullptr;    // 3 * nblock: first hh, ph, pp pair of each block
  int* d_rstart = nullptr;   // k_122_gen row and column term starts, per slot at gen_rso / gen_cso
  int* d_cstart = nullptr;
  int4* d_rterm = nullptr;
  int4* d_cterm = nullptr;
  int gen_rso[6] = {0}, gen_cso[6] = {0};
  int4* d_sptask = nullptr;  // C_pppp tile pairs, then the k_122_gen tiles
  int nsp_pppp = 0, nsp_gen = 0;
  int pppp_terms = 0, gen_terms = 0;  // the most terms one task of each kernel stages
};
std::map<const qd_layout*, Plan122>& plans() {
  static std::map<const qd_layout*, Plan122> m;
  return m;
}
// plans of different layouts are built and dropped from concurrent host
// threads (batched flows)
std::mutex g_plan_mutex;

size_t tile_smem(const TileInfo& t, int tw) {
  const size_t ld = (size_t)(t.nc | 1);
  const size_t tsz = ((size_t)t.nr * ld * tw + 1) & ~(size_t)1;
  return 8 * tsz + 16 * (size_t)t.nf + 8 * (size_t)t.npair;
}
// a task that only writes zeros keeps just the two pair lists
size_t zero_smem(const TileInfo& t) { return 8 * (size_t)t.npair; }

template <class T>
int upload_vec(qd_layout* L, const std::vector<T>& vec, T** dptr) {
  QD_CUDA(cudaMalloc(dptr, std::max<size_t>(1, vec.size()) * sizeof(T)));
  if (!vec.empty()) QD_CUDA(cudaMemcpy(*dptr, vec.data(), vec.size() * sizeof(T), cudaMemcpyHostToDevice));
  L->ws_bytes += (i64)(vec.size() * sizeof(T));
  return QD_OK;
}
}  // namespace

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
  std::vector<int> gsz(ngroup), goff(ngroup + 1, 0), kpos(m, 0), sbase(m, 0), holes(ngroup, 0);
  for (int g = 0; g < ngroup; ++g) {
    gsz[g] = L->gstart[g + 1] - L->gstart[g];
    p.gmax = std::max(p.gmax, gsz[g]);
    goff[g + 1] = goff[g] + gsz[g] * gsz[g];
    for (int k = 0; k < gsz[g]; ++k) {
      const int s = L->gmem[L->gstart[g] + k];
      kpos[s] = k;
      if (s < L->n) {
        if (k != holes[g]) {  // holes must be the lowest members of every group
          set_error("commutator_122: holes are not the lowest states of their (ml,ms) group");
          return QD_ERR_LAYOUT;
        }
        ++holes[g];
      }
    }
  }
  if (p.gmax > 16) {  // cells of a group pair fit the 8-bit cell fields
    set_error("commutator_122: (ml,ms) group of %d states exceeds 16", p.gmax);
    return QD_ERR_ARG;
  }
  p.nfent = goff[ngroup];
  for (int s = 0; s < m; ++s) sbase[s] = goff[L->gid[s]] + kpos[s] * gsz[L->gid[s]];

  std::vector<int4> gpd;
  std::vector<int2> gpp, gpg;
  struct GpHost {
    int n1, n2, cnt[3], nf, npair;
  };
  for (int q = 0; q < L->nblock; ++q) {
    const int nh = L->blk[q].x, nb = L->blk[q].y, ntot = L->blk[q].w, pb = L->pbase[q];
    // group pairs in order of first appearance; per group pair its pairs in
    // class order (pairs are enumerated [hh | ph | pp], each class by index)
    std::map<std::pair<int, int>, int> idx;
    std::vector<std::pair<int, int>> order;
    std::vector<std::vector<int2>> plist;  // {w, packed cells}
    std::vector<GpHost> gh;
    for (int P = 0; P < ntot; ++P) {
      const int2 pr = L->pairs[pb + P];  // 0-based states, pr.x < pr.y
      const int c = P < nh ? 0 : (P < nh + nb ? 1 : 2);
      const int w = P - (c == 0 ? 0 : (c == 1 ? nh : nh + nb));
      const int gi = L->gid[pr.x], gj = L->gid[pr.y];
      const int g = std::min(gi, gj), h = std::max(gi, gj);
      auto ins = idx.emplace(std::make_pair(g, h), (int)order.size());
      if (ins.second) {
        order.push_back({g, h});
        plist.emplace_back();
        gh.push_back(GpHost{gsz[g], gsz[h], {0, 0, 0}, 0, 0});
      }
      const int u = ins.first->second;
      int t1, t2;
      if (g != h) {
        t1 = gi == g ? pr.x : pr.y;
        t2 = gi == g ? pr.y : pr.x;
      } else {
        t1 = pr.x;
        t2 = pr.y;
      }
      const int n2c = gsz[h];
      const int r = kpos[t1] * n2c + kpos[t2];
      const int neg = t1 > t2 ? 1 : 0;
      const int rm = g == h ? kpos[t2] * n2c + kpos[t1] : -1;
      if (gsz[g] * gsz[h] > 256 || r >= 255 || rm >= 255) {
        set_error("commutator_122: group pair of %d cells exceeds the cell fields", gsz[g] * gsz[h]);
        return QD_ERR_ARG;
      }
      plist[u].push_back(int2{w, r | ((rm + 1) << 8) | (neg << 16) | (kpos[t1] << 17) | (kpos[t2] << 21)});
      gh[u].cnt[c] += 1;
    }
    const int u0 = (int)gpd.size() / 2;
    for (size_t u = 0; u < order.size(); ++u) {
      const int g = order[u].first, h = order[u].second;
      GpHost& d = gh[u];
      if (d.cnt[0] > 1023 || d.cnt[1] > 1023 || d.cnt[2] > 1023) {
        set_error("commutator_122: group pair class count exceeds 1023");
        return QD_ERR_ARG;
      }
      d.nf = d.n1 * d.n1 + d.n2 * d.n2;
      d.npair = d.cnt[0] + d.cnt[1] + d.cnt[2];
      gpd.push_back(int4{q, d.n1 | (d.n2 << 8) | ((g == h ? 1 : 0) << 16), holes[g] | (holes[h] << 8), goff[g]});
      gpd.push_back(int4{goff[h], (int)gpp.size(), 0, d.cnt[0] | (d.cnt[1] << 10) | (d.cnt[2] << 20)});
      gpg.push_back(int2{g, h});
      gpp.insert(gpp.end(), plist[u].begin(), plist[u].end());
    }
    // tiles: every ordered pair of group pairs with at least one stored
    // output cell (a row class >= a column class)
    for (size_t a = 0; a < order.size(); ++a)
      for (size_t b = 0; b < order.size(); ++b) {
        const GpHost &A = gh[a], &B = gh[b];
        bool out = false;
        unsigned parts = 0;
        for (int c1 = 0; c1 < 3; ++c1)
          for (int c2 = 0; c2 < 3; ++c2)
            if (A.cnt[c1] > 0 && B.cnt[c2] > 0) {
              parts |= 1u << (c1 >= c2 ? slot_of(c1, c2) : slot_of(c2, c1));
              if (c1 >= c2) out = true;
            }
        if (!out) continue;
        TileInfo t;
        t.outs = 0;
        for (int c1 = 0; c1 < 3; ++c1)
          for (int c2 = 0; c2 <= c1; ++c2)
            if (A.cnt[c1] > 0 && B.cnt[c2] > 0) t.outs |= 1u << out_region(c1, c2);
        t.a = u0 + (int)a;
        t.b = u0 + (int)b;
        t.nr = A.n1 * A.n2;
        t.nc = B.n1 * B.n2;
        t.cells = t.nr * t.nc;
        t.nf = A.nf + B.nf;
        t.npair = A.npair + B.npair;
        t.parts = parts;
        t.holefree = holes[order[a].first] == 0 && holes[order[a].second] == 0 && holes[order[b].first] == 0 &&
                     holes[order[b].second] == 0;
        t.nst = 0;
        for (int c1 = 0; c1 < 3; ++c1)
          for (int c2 = 0; c2 <= c1; ++c2) t.nst += A.cnt[c1] * B.cnt[c2];
        p.tiles.push_back(t);
      }
  }
  for (const TileInfo& t : p.tiles)
    if (tile_smem(t, 1) > SMEM_MAX_122) {
      set_error("commutator_122: tile of %d cells exceeds shared memory", t.cells);
      return QD_ERR_ARG;
    }
  std::vector<int2> th(p.tiles.size());
  for (size_t i = 0; i < p.tiles.size(); ++i) th[i] = int2{p.tiles[i].a, p.tiles[i].b};
  int rc;
  if ((rc = upload_vec(L, gpd, &p.d_gpd)) || (rc = upload_vec(L, gpp, &p.d_gpp)) ||
      (rc = upload_vec(L, th, &p.d_tiles)) ||
      (rc = upload_vec(L, sbase, &p.d_sbase)))
    return rc;
  // generator-like A: the pp pairs' W terms (k_122_pppp) and the row and
  // column terms of the other five parts (k_122_gen), per block
  {
    const int n = L->n, mp = L->mp;
    const int ofph = (int)L->o_fph, ofpp = (int)L->o_fpp, ofhh = (int)L->o_fhh;
    std::vector<int> gbase(3 * L->nblock), ppstart(1, 0);
    std::vector<int2> ppterm;
    // per slot: its terms and, per pair of its classes (block order), their starts
    std::vector<int> rst[6], cst[6];
    std::vector<int4> rterm_s[6], cterm_s[6];
    std::vector<int4> ptask, gtask;
    int cnt[3] = {0, 0, 0};
    enum { NEG = 1, MA = 2, MB = 4, CB = 8 };
    auto fA = [&](int pt, int h) { return ofph + (pt - n) + h * mp; };  // A's or B's fph(p, h)
    auto fpp = [&](int t, int b) { return ofpp + (t - n) + (b - n) * mp; };
    auto fhh = [&](int k, int t) { return ofhh + k + t * n; };
    auto src = [](int opd, int slot, int tr) { return (opd << 4) | (tr << 3) | slot; };
    for (int q = 0; q < L->nblock; ++q) {
      const int nh = L->blk[q].x, nb = L->blk[q].y, np = L->blk[q].z, pb = L->pbase[q];
      for (int c = 0; c < 3; ++c) gbase[c * L->nblock + q] = cnt[c];
      cnt[0] += nh;
      cnt[1] += nb;
      cnt[2] += np;
      std::map<std::pair<int, int>, int> ihh, iph, ipp;
      for (int k = 0; k < nh; ++k) ihh[{L->pairs[pb + k].x, L->pairs[pb + k].y}] = k;
      for (int k = 0; k < nb; ++k) iph[{L->pairs[pb + nh + k].x, L->pairs[pb + nh + k].y}] = k;
      for (int k = 0; k < np; ++k) ipp[{L->pairs[pb + nh + nb + k].x, L->pairs[pb + nh + nb + k].y}] = k;
      auto grp = [&](int x) { return std::make_pair(L->gstart[L->gid[x]], L->gstart[L->gid[x] + 1]); };
      // members t of G(x) that are holes (want_hole) or particles, excluding `skip`
      auto each = [&](int x, bool want_hole, int skip, auto fn) {
        const auto mr = grp(x);
        for (int u = mr.first; u < mr.second; ++u) {
          const int tt = L->gmem[u];
          if ((tt < n) == want_hole && tt != skip) fn(tt);
        }
      };
      // index and ordering sign of the pair {u, v} in a class map
      auto srt = [](const std::map<std::pair<int, int>, int>& m, int u, int v, int* idx, int* sg) {
        auto f = m.find({std::min(u, v), std::max(u, v)});
        if (f == m.end()) return false;
        *idx = f->second;
        *sg = u < v ? 1 : -1;
        return true;
      };
      const auto hhp = [&](int k) { return L->pairs[pb + k]; };
      const auto php = [&](int k) { return L->pairs[pb + nh + k]; };
      const auto ppp = [&](int k) { return L->pairs[pb + nh + nb + k]; };
      int idx, sg;
      // pp pairs (a, b): W terms +fA(a,t) B_ppph(., (t,b)), -fA(b,t) B_ppph(., (t,a)), holes t
      for (int k = 0; k < np; ++k) {
        const int x0 = ppp(k).x, y0 = ppp(k).y;
        for (int side = 0; side < 2; ++side) {
          const int x = side ? y0 : x0, y = side ? x0 : y0;
          each(x, true, -1, [&](int t) {
            auto f = iph.find({t, y});
            if (f != iph.end()) ppterm.push_back(int2{f->second, (t) | ((x - n) << 8) | ((side ? 1 : 0) << 20)});
          });
        }
        ppstart.push_back((int)ppterm.size());
      }
      // row terms, per slot over the pairs of its row class
      auto rows_of = [&](int slot, int k) {
        std::vector<int4>& T = rterm_s[slot];
        if (slot == 4 || slot == 2) {  // rows pp (x, y)
          const int x0 = ppp(k).x, y0 = ppp(k).y;
          for (int side = 0; side < 2; ++side) {
            const int x = side ? y0 : x0, y = side ? x0 : y0;
            each(x, true, -1, [&](int t) {
              auto f = iph.find({t, y});
              if (f != iph.end()) T.push_back(int4{f->second, fA(x, t), side ? NEG : 0, src(1, slot == 4 ? 3 : 5, 0)});
            });
            if (slot == 2)  // -s hB fppB(t, x) A_pphh((t,y)) over particles t in G(x)
              each(x, false, y, [&](int t) {
                if (srt(ipp, side ? y : t, side ? t : y, &idx, &sg))
                  T.push_back(int4{idx, fpp(t, x), MB | CB | (sg > 0 ? NEG : 0), src(0, 2, 0)});
              });
          }
        } else if (slot == 5 || slot == 3) {  // rows ph (h, p)
          const int h = php(k).x, pt = php(k).y;
          each(h, false, pt, [&](int t) {
            if (!srt(ipp, t, pt, &idx, &sg)) return;
            if (slot == 5) {
              T.push_back(int4{idx, fA(t, h), MA | (sg < 0 ? NEG : 0), src(1, 2, 0)});
              T.push_back(int4{idx, fA(t, h), MB | CB | (sg > 0 ? NEG : 0), src(0, 2, 0)});
            } else {
              T.push_back(int4{idx, fA(t, h), MA | (sg < 0 ? NEG : 0), src(1, 4, 0)});
            }
          });
          each(pt, true, h, [&](int t) {
            if (!srt(ihh, h, t, &idx, &sg)) return;
            if (slot == 5)
              T.push_back(int4{idx, fA(pt, t), sg < 0 ? NEG : 0, src(1, 0, 0)});
            else
              T.push_back(int4{idx, fA(pt, t), MB | (sg < 0 ? NEG : 0), src(1, 5, 1)});
          });
        } else {  // slot 0, rows hh (b1, b2)
          const int b1 = hhp(k).x, b2 = hhp(k).y;
          each(b1, false, -1, [&](int t) {
            auto f = iph.find({b2, t});
            if (f != iph.end()) T.push_back(int4{f->second, fA(t, b1), MA | NEG, src(1, 5, 0)});
          });
          each(b2, false, -1, [&](int t) {
            auto f = iph.find({b1, t});
            if (f != iph.end()) T.push_back(int4{f->second, fA(t, b2), MA, src(1, 5, 0)});
          });
        }
      };
      auto cols_of = [&](int slot, int k) {
        std::vector<int4>& T = cterm_s[slot];
        if (slot == 4) {  // columns ph (h, p)
          const int h = php(k).x, pt = php(k).y;
          each(h, false, pt, [&](int t) {
            if (srt(ipp, t, pt, &idx, &sg)) T.push_back(int4{idx, fA(t, h), sg > 0 ? NEG : 0, src(1, 1, 0)});
          });
          each(pt, true, h, [&](int t) {
            if (!srt(ihh, h, t, &idx, &sg)) return;
            T.push_back(int4{idx, fA(pt, t), MA | (sg > 0 ? NEG : 0), src(1, 2, 0)});
            T.push_back(int4{idx, fA(pt, t), MB | CB | (sg < 0 ? NEG : 0), src(0, 2, 0)});
          });
        } else if (slot == 3) {  // columns ph (k1, k2)
          const int k1 = php(k).x, k2 = php(k).y;
          each(k1, false, k2, [&](int t) {
            if (srt(ipp, t, k2, &idx, &sg)) T.push_back(int4{idx, fA(t, k1), MB | (sg > 0 ? NEG : 0), src(1, 4, 1)});
          });
          each(k2, true, k1, [&](int t) {
            if (srt(ihh, k1, t, &idx, &sg)) T.push_back(int4{idx, fA(k2, t), MA | (sg > 0 ? NEG : 0), src(1, 5, 0)});
          });
        } else {  // columns hh (k1, k2): slots 2, 5, 0
          const int k1 = hhp(k).x, k2 = hhp(k).y;
          for (int side = 0; side < 2; ++side) {
            const int kk = side ? k2 : k1, ko = side ? k1 : k2;
            each(kk, false, -1, [&](int t) {
              auto f = iph.find({ko, t});
              if (f == iph.end()) return;
              const int ng = side ? NEG : 0;
              if (slot == 2) T.push_back(int4{f->second, fA(t, kk), ng, src(1, 4, 0)});
              else if (slot == 5) T.push_back(int4{f->second, fA(t, kk), ng, src(1, 3, 0)});
              else T.push_back(int4{f->second, fA(t, kk), MB | ng, src(1, 5, 1)});
            });
            if (slot == 2)  // +s hB fhhB(kk, t) A_pphh(., (t,ko)) over holes t in G(kk)
              each(kk, true, ko, [&](int t) {
                if (srt(ihh, side ? ko : t, side ? t : ko, &idx, &sg))
                  T.push_back(int4{idx, fhh(kk, t), MB | CB | (sg < 0 ? NEG : 0), src(0, 2, 0)});
              });
          }
        }
      };
      const int rows_n[6] = {nh, 0, np, nb, np, nb}, cols_n[6] = {nh, 0, nh, nb, nb, nh};
      for (int slot : {0, 2, 3, 4, 5}) {
        int cr, cc;
        part_classes(P_HHHH + slot, cr, cc);
        const int nr = cr == 0 ? nh : (cr == 1 ? nb : np), nc = cc == 0 ? nh : (cc == 1 ? nb : np);
        for (int k = 0; k < nr; ++k) {
          rows_of(slot, k);
          rst[slot].push_back((int)rterm_s[slot].size());  // end of pair k's terms
        }
        for (int k = 0; k < nc; ++k) {
          cols_of(slot, k);
          cst[slot].push_back((int)cterm_s[slot].size());
        }
        if (rows_n[slot] > 0 && cols_n[slot] > 0)
          for (int i = 0; i < (rows_n[slot] + SP_B - 1) / SP_B; ++i)
            for (int j = 0; j < (cols_n[slot] + SP_B - 1) / SP_B; ++j) gtask.push_back(int4{q, slot, i, j});
      }
      const int tr = (np + PP_B - 1) / PP_B;
      for (int i = 0; i < tr; ++i)
        for (int j = i; j < tr; ++j) ptask.push_back(int4{q, i, j, 0});
    }
    // per slot start arrays: one entry per pair of its class (in block order) plus one
    // concatenated: per slot a start 0 then the pairs' ends, shifted by the
    // slot's first term in the joint term arrays
    std::vector<int> rall, call;
    std::vector<int4> rterm, cterm;
    for (int slot = 0; slot < 6; ++slot) {
      p.gen_rso[slot] = (int)rall.size();
      p.gen_cso[slot] = (int)call.size();
      const int r0 = (int)rterm.size(), c0 = (int)cterm.size();
      rall.push_back(r0);
      for (int e : rst[slot]) rall.push_back(r0 + e);
      call.push_back(c0);
      for (int e : cst[slot]) call.push_back(c0 + e);
      rterm.insert(rterm.end(), rterm_s[slot].begin(), rterm_s[slot].end());
      cterm.insert(cterm.end(), cterm_s[slot].begin(), cterm_s[slot].end());
    }
    p.nsp_pppp = (int)ptask.size();
    p.nsp_gen = (int)gtask.size();
    // the most terms one task stages (its shared memory)
    p.pppp_terms = 0;
    for (const int4& tk : ptask) {
      const int q = tk.x, np = L->blk[q].z, pbq = gbase[2 * L->nblock + q];
      int ne = 0;
      for (int pass = 0; pass < (tk.y == tk.z ? 1 : 2); ++pass) {
        const int c0 = (pass == 0 ? tk.z : tk.y) * PP_B, nc = std::min(PP_B, np - c0);
        ne += ppstart[pbq + c0 + nc] - ppstart[pbq + c0];
      }
      p.pppp_terms = std::max(p.pppp_terms, ne);
    }
    p.gen_terms = 0;
    for (const int4& tk : gtask) {
      const int q = tk.x, slot = tk.y;
      int cr, cc;
      part_classes(P_HHHH + slot, cr, cc);
      const int4 bd = L->blk[q];
      const int nr = cr == 0 ? bd.x : (cr == 1 ? bd.y : bd.z), nc = cc == 0 ? bd.x : (cc == 1 ? bd.y : bd.z);
      const int i0 = tk.z * SP_B, j0 = tk.w * SP_B, nrt = std::min(SP_B, nr - i0), nct = std::min(SP_B, nc - j0);
      const int* rr = rall.data() + p.gen_rso[slot] + gbase[cr * L->nblock + q] + i0;
      const int* cs = call.data() + p.gen_cso[slot] + gbase[cc * L->nblock + q] + j0;
      p.gen_terms = std::max(p.gen_terms, (rr[nrt] - rr[0]) + (cs[nct] - cs[0]));
    }
    if (2 * PP_B * PP_LD * sizeof(double) + (size_t)p.pppp_terms * sizeof(StagedTerm) > SMEM_MAX_122 - 1024 ||
        (size_t)p.gen_terms * sizeof(StagedTerm) > SMEM_MAX_122 - 1024) {
      set_error("commutator_122: %d / %d terms of one tile exceed shared memory", p.pppp_terms, p.gen_terms);
      return QD_ERR_ARG;
    }
    std::vector<int4> all = ptask;
    all.insert(all.end(), gtask.begin(), gtask.end());
    std::vector<int> ppbase(L->nblock);
    for (int q = 0; q < L->nblock; ++q) ppbase[q] = gbase[2 * L->nblock + q];
    if ((rc = upload_vec(L, ppbase, &p.d_ppbase)) || (rc = upload_vec(L, ppstart, &p.d_ppstart)) ||
        (rc = upload_vec(L, ppterm, &p.d_ppterm)) || (rc = upload_vec(L, gbase, &p.d_gbase)) ||
        (rc = upload_vec(L, rall, &p.d_rstart)) || (rc = upload_vec(L, call, &p.d_cstart)) ||
        (rc = upload_vec(L, rterm, &p.d_rterm)) || (rc = upload_vec(L, cterm, &p.d_cterm)) ||
        (rc = upload_vec(L, all, &p.d_sptask)))
      return rc;
  }
  // particle-hole channel: first cc row of each (G1, G2) and the launches
  p.ng = ngroup;
  std::vector<int2> zrow((size_t)ngroup * ngroup);
  for (int g1 = 0; g1 < ngroup; ++g1)
    for (int g2 = 0; g2 < ngroup; ++g2)
      zrow[(size_t)g1 * ngroup + g2] = L->ccmap[(size_t)L->gmem[L->gstart[g1]] * m + L->gmem[L->gstart[g2]]];
  {
    // per tile the first mode that fits: all four terms staged, two buffers
    // (each while at least three CTAs fit an SM), one buffer, none; buckets
    // by mode, then by size interval, largest first
    struct PdT {
      int mode;
      size_t sm;
      int tile;
    };
    std::vector<PdT> lst;
    for (size_t i = 0; i < p.tiles.size(); ++i) {
      const TileInfo& t = p.tiles[i];
      const size_t c = (size_t)t.cells, ns = (size_t)t.nst, np = (size_t)t.npair;
      const size_t s4 = 8 * (4 * c + np), s2 = 8 * (2 * c + ns + np), s1 = 8 * (c + ns + np);
      const size_t third = SMEM_MAX_122 / 3;
      if (s4 <= third)
        lst.push_back({PD_ALL4, s4, (int)i});
      else if (s2 <= third)
        lst.push_back({PD_PAIRS, s2, (int)i});
      else if (s1 <= SMEM_MAX_122)
        lst.push_back({PD_SINGLE, s1, (int)i});
      else
        lst.push_back({PD_DIRECT, 8 * np, (int)i});
    }
    const size_t bounds[4] = {24 * 1024, 56 * 1024, 112 * 1024, SMEM_MAX_122};
    auto interval = [&](size_t sm) {
      int l = 0;
      while (l < 3 && sm > bounds[l]) ++l;
      return l;
    };
    std::stable_sort(lst.begin(), lst.end(), [&](const PdT& x, const PdT& y) {
      return x.mode != y.mode ? x.mode < y.mode : x.sm > y.sm;
    });
    std::vector<int> tasks;
    size_t i = 0;
    while (i < lst.size()) {
      const int mode = lst[i].mode, l = interval(lst[i].sm);
      PdBucket b{(int)tasks.size(), 0, lst[i].sm, mode};
      while (i < lst.size() && lst[i].mode == mode && interval(lst[i].sm) == l) tasks.push_back(lst[i++].tile);
      b.count = (int)tasks.size() - b.first;
      p.pbuckets.push_back(b);
    }
    int rc2;
    if ((rc2 = upload_vec(L, gpg, &p.d_gpg)) || (rc2 = upload_vec(L, zrow, &p.d_zrow)) ||
        (rc2 = upload_vec(L, tasks, &p.d_ptask)))
      return rc2;
  }
  QD_CUDA(cudaMalloc(&p.d_ftab, sizeof(double2) * 2 * (size_t)std::max(1, p.nfent)));
  L->ws_bytes += (i64)sizeof(double2) * 2 * p.nfent;
  for (const void* fn : {(const void*)k_122_tile<1, 64, false>, (const void*)k_122_tile<2, 64, false>,
                         (const void*)k_122_tile<1, 128, false>, (const void*)k_122_tile<2, 128, false>,
                         (const void*)k_122_tile<1, 256, false>, (const void*)k_122_tile<2, 256, false>,
                         (const void*)k_122_tile<1, 256, true>, (const void*)k_122_tile<2, 256, true>,
                         (const void*)k_pandya_tile<PD_ALL4>, (const void*)k_pandya_tile<PD_PAIRS>,
                         (const void*)k_pandya_tile<PD_SINGLE>, (const void*)k_pandya_tile<PD_DIRECT>,
                         (const void*)k_122_pppp, (const void*)k_122_gen}) {
    cudaFuncAttributes fa;
    QD_CUDA(cudaFuncGetAttributes(&fa, fn));
    QD_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SMEM_MAX_122 - (int)fa.sharedSizeBytes));
  }
  plans()[L] = p;
  *out = &plans()[L];
  return QD_OK;
}

// Tasks for one pair of zero-part masks: per tile the terms it needs, in
// buckets of similar shared memory (largest first).  A tile that needs both
// terms but does not fit with both operands staged runs as a B task that
// sets C and an A task (in a later launch) that accumulates.
// Bucketings the autotuner chooses from: the size bounds (bytes of shared
// memory) that split each list into launches.  More buckets give small tiles
// more CTAs per SM; fewer keep the tiles of one column strip in one launch.
constexpr int kNumBounds = 4, kBoundsLen = 6;
const size_t kBounds[kNumBounds][kBoundsLen] = {
    {24 * 1024, 56 * 1024, 112 * 1024, SMEM_MAX_122, SMEM_MAX_122, SMEM_MAX_122},
    {56 * 1024, SMEM_MAX_122, SMEM_MAX_122, SMEM_MAX_122, SMEM_MAX_122, SMEM_MAX_122},
    {SMEM_MAX_122, SMEM_MAX_122, SMEM_MAX_122, SMEM_MAX_122, SMEM_MAX_122, SMEM_MAX_122},
    {8 * 1024, 16 * 1024, 24 * 1024, 56 * 1024, 112 * 1024, SMEM_MAX_122}};

// One bucketing of the task lists: buckets by size bound (largest first),
// and within a bucket the tiles sharing a column strip (block q, column
// group pair b) together: their gathers read the same columns, whose memory
// atoms also hold neighbouring group pairs' rows, so concurrent CTAs hit in
// L2.
static int build_variant(qd_layout* L, const Plan122* p, std::vector<std::pair<size_t, int2>> lst_in[3], int bid,
                         TaskSet& ts) {
  std::vector<int2> all;
  const size_t* bounds = kBounds[bid];
  ts.bounds_id = bid;
  for (int l = 0; l < 3; ++l) {
    std::vector<std::pair<size_t, int2>> v = lst_in[l];
    std::stable_sort(v.begin(), v.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    size_t i = 0;
    while (i < v.size()) {
      // bucket: tasks down to the next size bound below the first one
      const size_t top = v[i].first;
      size_t lower = 0;
      for (int k = 0; k < kBoundsLen; ++k)
        if (bounds[k] < top) lower = std::max(lower, bounds[k]);
      Bucket122 b;
      b.tw = l == 1 ? 2 : 1;
      b.list = l;
      b.first = (int)all.size();
      b.smem = top;
      while (i < v.size() && v[i].first > lower) all.push_back(v[i++].second);
      b.count = (int)all.size() - b.first;
      ts.buckets.push_back(b);
    }
  }
  for (const Bucket122& bk : ts.buckets)
    std::stable_sort(all.begin() + bk.first, all.begin() + bk.first + bk.count, [&](const int2& x, const int2& y) {
      const TileInfo &tx = p->tiles[x.x], &ty = p->tiles[y.x];
      return tx.b != ty.b ? tx.b < ty.b : tx.a < ty.a;
    });
  int rc = upload_vec(L, all, &ts.d_task);
  if (rc) return rc;
  ts.h_task = all;
  return QD_OK;
}

static int task_set(qd_layout* L, Plan122* p, unsigned zA, unsigned zB, TaskSet** out) {
  std::lock_guard<std::mutex> lock(g_plan_mutex);
  auto key = std::make_pair(zA, zB);
  auto it = p->sets.find(key);
  if (it != p->sets.end()) {
    *out = &it->second;
    return QD_OK;
  }
  const unsigned one = (1u << P_FHH) | (1u << P_FPP) | (1u << P_FPH);
  const bool fa0 = (zA & one) == one, fb0 = (zB & one) == one;  // a one-body part entirely zero
  // a one-body part without hh and pp entries (the Magnus generator's) couples
  // holes to particles only: on a tile whose four groups hold no hole every
  // leg of its term sums over nothing
  const unsigned hp = (1u << P_FHH) | (1u << P_FPP);
  const bool spa = (zA & hp) == hp, spb = (zB & hp) == hp;
  const unsigned za2 = (zA >> P_HHHH) & 63u, zb2 = (zB >> P_HHHH) & 63u;
  // lists: 0 one operand (set), 1 both operands (set), 2 one operand (accumulate)
  std::vector<std::pair<size_t, int2>> lst[3];
  const unsigned outmask = gen_like(zA) ? OUT_NONE : OUT_ALL;
  for (size_t i = 0; i < p->tiles.size(); ++i) {
    const TileInfo& t = p->tiles[i];
    if (!(t.outs & outmask)) continue;  // every output of the tile comes from k_122_pppp / k_122_gen
    const bool nb = !fa0 && (t.parts & ~zb2) && !(spa && t.holefree);
    const bool na = !fb0 && (t.parts & ~za2) && !(spb && t.holefree);
    const int op = (nb ? 1 : 0) | (na ? 2 : 0);
    if (op == 3) {
      if (tile_smem(t, 2) <= SMEM_MAX_122) {
        lst[1].push_back({tile_smem(t, 2), int2{(int)i, 3}});
      } else {
        lst[0].push_back({tile_smem(t, 1), int2{(int)i, 1}});
        lst[2].push_back({tile_smem(t, 1), int2{(int)i, 2 | 4}});
      }
    } else {
      lst[0].push_back({op ? tile_smem(t, 1) : zero_smem(t), int2{(int)i, op}});  // op 0: writes zeros
    }
  }
  TaskSet ts;
  for (int bid = 0; bid < kNumBounds; ++bid) {
    TaskSet& v = bid == 0 ? ts : (ts.alts.emplace_back(), ts.alts.back());
    v.outmask = outmask;
    int rc = build_variant(L, p, lst, bid, v);
    if (rc) return rc;
  }
  p->sets[key] = ts;
  *out = &p->sets[key];
  return QD_OK;
}

void drop_122_plan(const qd_layout* L) {
  std::lock_guard<std::mutex> lock(g_plan_mutex);
  auto it = plans().find(L);
  if (it == plans().end()) return;
  Plan122& p = it->second;
  for (void* ptr : {(void*)p.d_gpd, (void*)p.d_gpp, (void*)p.d_tiles, (void*)p.d_sbase,
                    (void*)p.d_ftab, (void*)p.d_gpg, (void*)p.d_zrow, (void*)p.d_ptask, (void*)p.d_ppbase,
                    (void*)p.d_ppstart, (void*)p.d_ppterm, (void*)p.d_gbase, (void*)p.d_rstart,
                    (void*)p.d_cstart, (void*)p.d_rterm, (void*)p.d_cterm, (void*)p.d_sptask})
    if (ptr) cudaFree(ptr);
  for (auto& kv : p.sets) {
    if (kv.second.d_task) cudaFree(kv.second.d_task);
    for (TaskSet& t : kv.second.alts)
      if (t.d_task) cudaFree(t.d_task);
  }
  plans().erase(it);
}

// class pairs (c1 * 3 + c2, both orders) on which an operand can be non-zero
static unsigned nz_mask(unsigned zmask) {
  unsigned nz = 0;
  for (int c1 = 0; c1 < 3; ++c1)
    for (int c2 = 0; c2 < 3; ++c2) {
      const int part = c1 >= c2 ? slot_of(c1, c2) : slot_of(c2, c1);
      if (!((zmask >> (P_HHHH + part)) & 1u)) nz |= 1u << (c1 * 3 + c2);
    }
  return nz;
}

// Leg masks of one term, per launch: byte cfix (0..2) holds bit
// kh * 4 + oh * 2 + th, set when a leg with fixed class cfix can add anything
// whose fixed state has kind kh, whose other state on the same side has kind
// oh and whose summed states have kind th (1 = hole); `sparse` is the one-body
// factor's sparsity, zstaged the zero-part mask of the staged operand.
static unsigned leg_masks(int sparse, unsigned zstaged) {
  const unsigned nz = nz_mask(zstaged);
  unsigned m = sparse ? LEG_SPARSE : 0u;
  for (int cfix = 0; cfix < 3; ++cfix)
    for (int bits = 0; bits < 8; ++bits)
      if (leg_ok(sparse, (bits >> 2) & 1, bits & 1, (bits >> 1) & 1, cfix, nz)) m |= 1u << (8 * cfix + bits);
  return m;
}

static int launch_bucket(qd_layout* L, const Plan122* p, const TaskSet* ts, const Bucket122& b, int threads,
                         const qd_op* A, const qd_op* B, int spA, int spB, double* C) {
  // the B term (FA x TB) and the A term (-FB x TA)
  const unsigned legB = leg_masks(spA, B->zero_mask), legA = leg_masks(spB, A->zero_mask);
#define QD_122_LAUNCH(TW, NT)                                                                                   \
  k_122_tile<TW, NT, false><<<b.count, NT, b.smem, L->stream>>>(L->dev, ts->d_task + b.first, p->d_tiles, p->d_gpd,   \
                                                         p->d_gpp, p->d_ftab, p->nfent, A->d,                   \
                                                         (double)A->herm, A->zero_mask, legA, B->d,             \
                                                         (double)B->herm, B->zero_mask, legB, C, ts->outmask,   \
                                                         nullptr, nullptr)
  if (b.tw == 2) {
    if (threads == 64) QD_122_LAUNCH(2, 64); else if (threads == 128) QD_122_LAUNCH(2, 128); else QD_122_LAUNCH(2, 256);
  } else {
    if (threads == 64) QD_122_LAUNCH(1, 64); else if (threads == 128) QD_122_LAUNCH(1, 128); else QD_122_LAUNCH(1, 256);
  }
#undef QD_122_LAUNCH
  ++L->nlaunch;
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// Autotuner: the first launch of a task set times every bucket with 64-, 128-
// and 256-thread CTAs (CUDA events, best of two runs each) on the real operands,
// writing into a scratch operator of the layout, and keeps the fastest size
// per bucket.  Every output cell is summed by one thread in a fixed order
// whatever the CTA size, so the choice never changes a result.
static int tune_variant(qd_layout* L, Plan122* p, TaskSet* ts, const qd_op* A, const qd_op* B, int spA, int spB,
                        double* scratch, cudaEvent_t e0, cudaEvent_t e1) {
  ts->ms_total = 0.f;
  for (Bucket122& b : ts->buckets) {
    for (int v = 0; v < 3; ++v) {
      const int threads = 64 << v;
      float best = 1e30f;
      for (int rep = 0; rep < 2; ++rep) {
        QD_CUDA(cudaEventRecord(e0, L->stream));
        TRY(launch_bucket(L, p, ts, b, threads, A, B, spA, spB, scratch));
        QD_CUDA(cudaEventRecord(e1, L->stream));
        QD_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        QD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, ms);
      }
      b.ms[v] = best;
    }
    int v = 0;
    for (int k = 1; k < 3; ++k)
      if (b.ms[k] < b.ms[v]) v = k;
    b.threads = 64 << v;
    ts->ms_total += b.ms[v];
  }
  return QD_OK;
}

// Autotuner: the first launch of a task set times, for every bucketing
// (kBounds), every bucket with 64-, 128- and 256-thread CTAs (CUDA events, best of
// two runs each) on the real operands, writing into a scratch operator of
// the layout; it keeps the CTA size per bucket and the bucketing with the
// least total time.  Every output cell is summed by one thread in a fixed
// order whatever the bucketing or CTA size, so the choice never changes a
// result.
static int tune_122(qd_layout* L, Plan122* p, TaskSet* ts, const qd_op* A, const qd_op* B, int spA, int spB) {
  double* scratch = scratch_operator(L);
  if (!scratch) return QD_OK;  // no scratch: keep the defaults
  cudaEvent_t e0, e1;
  QD_CUDA(cudaEventCreate(&e0));
  QD_CUDA(cudaEventCreate(&e1));
  const long long n0 = L->nlaunch;
  TRY(tune_variant(L, p, ts, A, B, spA, spB, scratch, e0, e1));
  for (TaskSet& alt : ts->alts) TRY(tune_variant(L, p, &alt, A, B, spA, spB, scratch, e0, e1));
  int best = -1;
  float tbest = ts->ms_total;
  for (size_t k = 0; k < ts->alts.size(); ++k)
    if (ts->alts[k].ms_total < tbest) {
      tbest = ts->alts[k].ms_total;
      best = (int)k;
    }
  // keep the winner in *ts; the others stay in alts for the report (their task arrays are freed)
  std::vector<TaskSet> others;
  TaskSet win;
  if (best >= 0) {
    win = ts->alts[best];
    ts->alts[best] = TaskSet();
    TaskSet cur = *ts;
    cur.alts.clear();
    others.push_back(cur);
  }
  for (TaskSet& t : ts->alts)
    if (t.d_task || !t.buckets.empty()) others.push_back(t);
  if (best >= 0) {
    *ts = win;
  }
  ts->alts.clear();
  for (TaskSet& t : others) {
    if (t.d_task) cudaFree(t.d_task);
    t.d_task = nullptr;
    t.h_task.clear();
    ts->alts.push_back(t);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  L->nlaunch = n0;  // tuning launches are not the caller's work
  ts->tuned = true;
  return QD_OK;
}

// Text summary of the autotuned buckets of every task set of the layout.
std::string tuning_report_122(const qd_layout* L) {
  std::lock_guard<std::mutex> lock(g_plan_mutex);
  auto it = plans().find(L);
  if (it == plans().end()) return "";
  std::string out;
  char line[256];
  for (const auto& kv : it->second.sets) {
    const TaskSet& ts = kv.second;
    snprintf(line, sizeof(line), "commutator_122 masks A=0x%03x B=0x%03x: bucketing %d kept (%.4f ms)",
             kv.first.first, kv.first.second, ts.bounds_id, ts.ms_total);
    out += line;
    for (const TaskSet& t : ts.alts) {
      snprintf(line, sizeof(line), ", bucketing %d %.4f ms", t.bounds_id, t.ms_total);
      out += line;
    }
    out += "\n";
    for (const Bucket122& b : kv.second.buckets) {
      snprintf(line, sizeof(line),
               "  tiles %6d staged %d smem %6zu B: 64 thr %.4f ms, 128 thr %.4f ms, 256 thr %.4f ms -> %d\n",
               b.count, b.tw, b.smem, b.ms[0], b.ms[1], b.ms[2], b.threads);
      out += line;
    }
  }
  return out;
}

static bool capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

static int spars(const qd_op* X) {
  const unsigned hp = (1u << P_FHH) | (1u << P_FPP);
  return (X->zero_mask & hp) == hp;
}

// Build (and autotune on A, B) the plan and the task set of a pair of
// zero-part masks ahead of a stream capture, which must neither allocate
// nor synchronise.  A and B may be views with the masks zA, zB.
int prepare_122(qd_layout* L, const qd_op* A, const qd_op* B) {
  Plan122* p;
  int rc = plan_122(L, &p);
  if (rc) return rc;
  TaskSet* ts;
  if ((rc = task_set(L, p, A->zero_mask, B->zero_mask, &ts))) return rc;
  if (!ts->tuned && !ts->buckets.empty() && !L->prof.on && !capturing(L->stream)) {
    // the F tables of these operands first: the timed launches read them
    const int nf = L->m * p->gmax;
    k_ftab<<<(nf + 127) / 128, 128, 0, L->stream>>>(L->dev, p->d_sbase, A->d, (double)A->herm, B->d,
                                                    (double)B->herm, p->d_ftab, p->gmax, p->nfent);
    QD_CUDA(cudaGetLastError());
    TRY(tune_122(L, p, ts, A, B, spars(A), spars(B)));
  }
  return QD_OK;
}

// Every two-body part of C for a generator-like A (k_122_pppp, k_122_gen)
// on stream st.
static int launch_122_gen(qd_layout* L, const Plan122* p, const qd_op* A, const qd_op* B, double* C,
                          cudaStream_t st) {
  if (p->nsp_pppp > 0) {
    k_122_pppp<<<p->nsp_pppp, SP_T, 2 * PP_B * PP_LD * sizeof(double) + p->pppp_terms * sizeof(StagedTerm), st>>>(
        L->dev, p->d_sptask, p->d_ppbase, p->d_ppstart, p->d_ppterm, A->d, (double)A->herm, B->d, (double)B->herm,
        B->zero_mask, C);
    ++L->nlaunch;
  }
  if (p->nsp_gen > 0) {
    GenTables G;
    G.gbase = p->d_gbase;
    G.rstart = p->d_rstart;
    G.cstart = p->d_cstart;
    G.rterm = p->d_rterm;
    G.cterm = p->d_cterm;
    for (int k = 0; k < 6; ++k) {
      G.rso[k] = p->gen_rso[k];
      G.cso[k] = p->gen_cso[k];
    }
    k_122_gen<<<p->nsp_gen, SP_T, p->gen_terms * sizeof(StagedTerm), st>>>(
        L->dev, p->d_sptask + p->nsp_pppp, G, A->d, (double)A->herm, B->d, (double)B->herm, C);
    ++L->nlaunch;
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

int launch_122(qd_layout* L, const qd_op* A, const qd_op* B, double* C) {
  Plan122* p;
  int rc = plan_122(L, &p);
  if (rc) return rc;
  if (p->tiles.empty()) return QD_OK;
  TaskSet* ts;
  if ((rc = task_set(L, p, A->zero_mask, B->zero_mask, &ts))) return rc;
  const int spA = spars(A), spB = spars(B);
  if (ts->outmask != OUT_ALL) TRY(launch_122_gen(L, p, A, B, C, L->stream));
  if (ts->buckets.empty()) return QD_OK;  // no group-pair tiles: their F tables are not needed
  const int nf = L->m * p->gmax;
  k_ftab<<<(nf + 127) / 128, 128, 0, L->stream>>>(L->dev, p->d_sbase, A->d, (double)A->herm, B->d,
                                                  (double)B->herm, p->d_ftab, p->gmax, p->nfent);
  ++L->nlaunch;
  if (!ts->tuned && !L->prof.on && !capturing(L->stream)) TRY(tune_122(L, p, ts, A, B, spA, spB));
  for (const Bucket122& b : ts->buckets) TRY(launch_bucket(L, p, ts, b, b.threads, A, B, spA, spB, C));
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

int prepare_pandya(qd_layout* L) {
  Plan122* p;
  return plan_122(L, &p);
}

int launch_pandya_tiles(qd_layout* L, const double* Z, double* C) {
  Plan122* p;
  int rc = plan_122(L, &p);
  if (rc) return rc;
  for (const PdBucket& b : p->pbuckets) {
    if (b.count == 0) continue;
#define QD_PD_LAUNCH(M)                                                                                       \
  k_pandya_tile<M><<<b.count, TPD, b.smem, L->stream>>>(L->dev, p->d_ptask + b.first, p->d_tiles, p->d_gpd, \
                                                        p->d_gpp, p->d_gpg, p->d_zrow, p->ng, Z, C)
    switch (b.mode) {
      case PD_ALL4: QD_PD_LAUNCH(PD_ALL4); break;
      case PD_PAIRS: QD_PD_LAUNCH(PD_PAIRS); break;
      case PD_SINGLE: QD_PD_LAUNCH(PD_SINGLE); break;
      default: QD_PD_LAUNCH(PD_DIRECT); break;
    }
#undef QD_PD_LAUNCH
    ++L->nlaunch;
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// ---- one launch over several layouts' tiles (batched flows) ---------------
namespace {
struct Merged122 {
  int2* d_task = nullptr;
  int* d_tinst = nullptr;
  std::vector<Bucket122> buckets;
  Inst122* d_inst = nullptr;
  Inst122* h_inst = nullptr;  // pinned staging of the per-call instance table
  std::vector<const qd_layout*> layouts;
};
std::map<std::vector<uintptr_t>, Merged122>& merged122() {
  static std::map<std::vector<uintptr_t>, Merged122> m;
  return m;
}
std::mutex g_m122_mutex;
}  // namespace

// commutator_122 of every item in one set of launches: the items' tiles are
// merged per list (set with one operand, set with both, accumulate) and per
// shared-memory bucket, largest first, each task carrying its instance; the
// items' layouts share `st`.  Merged lists are cached per (layout, masks)
// tuple; the instance table is uploaded per call from pinned memory, which
// the caller rewrites only after synchronising the stream.
int launch_122_batched(cudaStream_t st, const std::vector<Item122>& items) {
  if (items.empty()) return QD_OK;
  const size_t n = items.size();
  std::vector<Plan122*> pl(n);
  std::vector<TaskSet*> tsv(n);
  std::vector<uintptr_t> key;
  for (size_t i = 0; i < n; ++i) {
    qd_layout* L = items[i].L;
    TRY(plan_122(L, &pl[i]));
    TRY(task_set(L, pl[i], items[i].A->zero_mask, items[i].B->zero_mask, &tsv[i]));
    key.push_back((uintptr_t)L);
    key.push_back(((uintptr_t)items[i].A->zero_mask << 16) | items[i].B->zero_mask);
  }
  Merged122* m;
  {
    std::lock_guard<std::mutex> lock(g_m122_mutex);
    auto f = merged122().find(key);
    if (f == merged122().end()) {
      Merged122 mg;
      std::vector<std::pair<size_t, std::pair<int2, int>>> lists[3];
      for (size_t i = 0; i < n; ++i) {
        mg.layouts.push_back(items[i].L);
        for (const Bucket122& b : tsv[i]->buckets)
          for (int k = b.first; k < b.first + b.count; ++k) {
            const int2 t = tsv[i]->h_task[k];
            const TileInfo& ti = pl[i]->tiles[t.x];
            lists[b.list].push_back({t.y == 0 ? zero_smem(ti) : tile_smem(ti, b.tw), {t, (int)i}});
          }
      }
      std::vector<int2> ht;
      std::vector<int> hi;
      const size_t bounds[4] = {24 * 1024, 56 * 1024, 112 * 1024, SMEM_MAX_122};
      for (int l = 0; l < 3; ++l) {
        auto& v = lists[l];
        std::stable_sort(v.begin(), v.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
        size_t k = 0;
        while (k < v.size()) {
          const size_t top = v[k].first;
          size_t lower = 0;
          for (size_t bnd : bounds)
            if (bnd < top) lower = bnd;
          Bucket122 b;
          b.tw = l == 1 ? 2 : 1;
          b.list = l;
          b.first = (int)ht.size();
          b.smem = top;
          while (k < v.size() && v[k].first > lower) {
            ht.push_back(v[k].second.first);
            hi.push_back(v[k].second.second);
            ++k;
          }
          b.count = (int)ht.size() - b.first;
          mg.buckets.push_back(b);
          {  // column strips together within the bucket (see task_set)
            std::vector<size_t> ord(b.count);
            for (int x = 0; x < b.count; ++x) ord[x] = b.first + x;
            std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) {
              const TileInfo &tx = pl[hi[x]]->tiles[ht[x].x], &ty = pl[hi[y]]->tiles[ht[y].x];
              if (hi[x] != hi[y]) return hi[x] < hi[y];
              return tx.b != ty.b ? tx.b < ty.b : tx.a < ty.a;
            });
            std::vector<int2> t2(b.count);
            std::vector<int> i2(b.count);
            for (int x = 0; x < b.count; ++x) {
              t2[x] = ht[ord[x]];
              i2[x] = hi[ord[x]];
            }
            std::copy(t2.begin(), t2.end(), ht.begin() + b.first);
            std::copy(i2.begin(), i2.end(), hi.begin() + b.first);
          }
        }
      }
      QD_CUDA(cudaMalloc(&mg.d_task, std::max<size_t>(1, ht.size()) * sizeof(int2)));
      QD_CUDA(cudaMalloc(&mg.d_tinst, std::max<size_t>(1, hi.size()) * sizeof(int)));
      if (!ht.empty()) {
        QD_CUDA(cudaMemcpy(mg.d_task, ht.data(), ht.size() * sizeof(int2), cudaMemcpyHostToDevice));
        QD_CUDA(cudaMemcpy(mg.d_tinst, hi.data(), hi.size() * sizeof(int), cudaMemcpyHostToDevice));
      }
      QD_CUDA(cudaMalloc(&mg.d_inst, n * sizeof(Inst122)));
      QD_CUDA(cudaMallocHost(&mg.h_inst, n * sizeof(Inst122)));
      f = merged122().emplace(key, mg).first;
    }
    m = &f->second;
  }
  for (size_t i = 0; i < n; ++i) {
    const Item122& it = items[i];
    const Plan122* p = pl[i];
    if (!tsv[i]->buckets.empty()) {  // F tables for the group-pair tiles
      const int nf = it.L->m * p->gmax;
      k_ftab<<<(nf + 127) / 128, 128, 0, st>>>(it.L->dev, p->d_sbase, it.A->d, (double)it.A->herm, it.B->d,
                                               (double)it.B->herm, p->d_ftab, p->gmax, p->nfent);
      ++it.L->nlaunch;
    }
    Inst122& I = m->h_inst[i];
    I.L = it.L->dev;
    I.tiles = p->d_tiles;
    I.gpd = p->d_gpd;
    I.gpp = p->d_gpp;
    I.F = p->d_ftab;
    I.nfent = p->nfent;
    I.A = it.A->d;
    I.hA = (double)it.A->herm;
    I.zA = it.A->zero_mask;
    I.legA = leg_masks(spars(it.B), it.A->zero_mask);
    I.B = it.B->d;
    I.hB = (double)it.B->herm;
    I.zB = it.B->zero_mask;
    I.legB = leg_masks(spars(it.A), it.B->zero_mask);
    I.C = it.C;
    I.outmask = tsv[i]->outmask;
    if (I.outmask != OUT_ALL) TRY(launch_122_gen(it.L, p, it.A, it.B, it.C, st));
  }
  QD_CUDA(cudaMemcpyAsync(m->d_inst, m->h_inst, n * sizeof(Inst122), cudaMemcpyHostToDevice, st));
  const DevLayout& L0 = items[0].L->dev;
  for (const Bucket122& b : m->buckets) {
    if (b.tw == 2)
      k_122_tile<2, 256, true><<<b.count, 256, b.smem, st>>>(L0, m->d_task + b.first, nullptr, nullptr, nullptr, nullptr, 0,
                                                       nullptr, 0.0, 0u, 0u, nullptr, 0.0, 0u, 0u, nullptr, 0u,
                                                       m->d_tinst + b.first, m->d_inst);
    else
      k_122_tile<1, 256, true><<<b.count, 256, b.smem, st>>>(L0, m->d_task + b.first, nullptr, nullptr, nullptr, nullptr, 0,
                                                       nullptr, 0.0, 0u, 0u, nullptr, 0.0, 0u, 0u, nullptr, 0u,
                                                       m->d_tinst + b.first, m->d_inst);
    ++items[0].L->nlaunch;
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// Drop every merged list that involves layout L (called when L goes).
void drop_merged_122(const qd_layout* L) {
  std::lock_guard<std::mutex> lock(g_m122_mutex);
  auto& mm = merged122();
  for (auto it = mm.begin(); it != mm.end();) {
    auto& ls = it->second.layouts;
    if (std::find(ls.begin(), ls.end(), L) != ls.end()) {
      if (it->second.d_task) cudaFree(it->second.d_task);
      if (it->second.d_tinst) cudaFree(it->second.d_tinst);
      if (it->second.d_inst) cudaFree(it->second.d_inst);
      if (it->second.h_inst) cudaFreeHost(it->second.h_inst);
      it = mm.erase(it);
    } else {
      ++it;
    }
  }
}

}  // namespace qd
