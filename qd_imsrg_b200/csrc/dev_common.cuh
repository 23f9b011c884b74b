// dev_common.cuh -- device helpers shared by the engine's kernels.
#pragma once

#include "qd_internal.hpp"

namespace qd {

constexpr int RED_BLOCKS = 296;  // 2 x 148 SMs: partial sums of the deterministic reductions
constexpr int RED_THREADS = 256;

// v_elem (src/ME_general.f90:1557-1680) on a device operator, 0-based states.
// Energy order equals states order (convertF sets eh(i)=i, ep(a)=n+a).
__device__ __forceinline__ double dv_elem(const DevLayout& L, const double* __restrict__ op, double herm, int a,
                                          int b, int c, int d) {
  if (a == b || c == d) return 0.0;
  const int e1 = __ldg(&L.ptab[a * L.m + b]);
  const int e2 = __ldg(&L.ptab[c * L.m + d]);
  const int q = pt_blk(e1);
  if (q != pt_blk(e2)) return 0.0;
  const double sgn = (pt_swap(e1) ^ pt_swap(e2)) ? -1.0 : 1.0;
  const int w1 = pt_idx(e1), w2 = pt_idx(e2);
  const int4 bd = __ldg(&L.blk[q]);  // nh, nb, np
  const i64* o = L.boff + 6 * q;
  double v;
  switch (pt_cls(e1) * 3 + pt_cls(e2)) {
    case 0: v = op[__ldg(o + 0) + w1 + (i64)w2 * bd.x]; break;         // Vhhhh(w1,w2)
    case 1: v = herm * op[__ldg(o + 5) + w2 + (i64)w1 * bd.y]; break;  // herm*Vphhh(w2,w1)
    case 2: v = herm * op[__ldg(o + 2) + w2 + (i64)w1 * bd.z]; break;  // herm*Vpphh(w2,w1)
    case 3: v = op[__ldg(o + 5) + w1 + (i64)w2 * bd.y]; break;         // Vphhh(w1,w2)
    case 4: v = op[__ldg(o + 3) + w1 + (i64)w2 * bd.y]; break;         // Vphph(w1,w2)
    case 5: v = herm * op[__ldg(o + 4) + w2 + (i64)w1 * bd.z]; break;  // herm*Vppph(w2,w1)
    case 6: v = op[__ldg(o + 2) + w1 + (i64)w2 * bd.z]; break;         // Vpphh(w1,w2)
    case 7: v = op[__ldg(o + 4) + w1 + (i64)w2 * bd.z]; break;         // Vppph(w1,w2)
    default: v = op[__ldg(o + 1) + w1 + (i64)w2 * bd.z]; break;        // Vpppp(w1,w2)
  }
  return sgn * v;
}

// One-body reads exactly as commutator_122 makes them:
//   hole-loop read f(x,i):      fhh(x,i) (x hole) or fph(x-n,i) (x particle)
//   particle-loop read f'(a,x): fph(a-n,x) (x hole) or fpp(a-n,x-n) (x particle)
__device__ __forceinline__ double f_hole(const DevLayout& L, const double* __restrict__ op, int x, int i) {
  return x < L.n ? op[L.o_fhh + x + (i64)i * L.n] : op[L.o_fph + (x - L.n) + (i64)i * L.mp];
}
__device__ __forceinline__ double f_part(const DevLayout& L, const double* __restrict__ op, int a, int x) {
  return x < L.n ? op[L.o_fph + (a - L.n) + (i64)x * L.mp] : op[L.o_fpp + (a - L.n) + (i64)(x - L.n) * L.mp];
}

// Bra/ket pair lists of the six stored sub-blocks (part ids P_HHHH..P_PHHH):
// bra class and ket class (0 hh, 1 ph, 2 pp).
__host__ __device__ inline void part_classes(int part, int& cb, int& ck) {
  switch (part) {
    case P_HHHH: cb = 0; ck = 0; break;
    case P_PPPP: cb = 2; ck = 2; break;
    case P_PPHH: cb = 2; ck = 0; break;
    case P_PHPH: cb = 1; ck = 1; break;
    case P_PPPH: cb = 2; ck = 1; break;
    default: cb = 1; ck = 0; break;  // P_PHHH
  }
}

// k-th pair of class cls in block q (0-based states, a<b)
__device__ __forceinline__ int2 block_pair(const DevLayout& L, int q, int cls, int k) {
  const int4 bd = __ldg(&L.blk[q]);
  int base = __ldg(&L.pbase[q]) + (cls == 0 ? 0 : (cls == 1 ? bd.x : bd.x + bd.y));
  return __ldg(&L.pairs[base + k]);
}

// Two-body flat decode: the stored two-body entries occupy [o2, neq) of the
// vectorize array as a sequence of non-empty sub-blocks; s2off (sorted) holds
// their start offsets and s2id their (block << 3 | part - P_HHHH).
struct Flat2B {
  const i64* off;
  const int* id;
  int n;
};

__device__ __forceinline__ int find_seg(const i64* __restrict__ off, int n, i64 e) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= e) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// rows of a part's sub-block in block bd
__host__ __device__ inline int part_rows(int part, int4 bd) {
  switch (part) {
    case P_HHHH: return bd.x;
    case P_PPPP: return bd.z;
    case P_PPHH: return bd.z;
    case P_PHPH: return bd.y;
    case P_PPPH: return bd.z;
    default: return bd.y;
  }
}

// element e of two-body part p -> (block, offset of the element in vectorize order)
__device__ __forceinline__ void part_elem(const DevLayout& L, int p, i64 e, int& q, i64& pos, int& row, int& col) {
  const i64* cum = L.pcum + (i64)p * L.nblock;
  q = find_seg(cum, L.nblock, e);
  i64 loc = e - __ldg(cum + q);
  const int4 bd = __ldg(&L.blk[q]);
  int part = P_HHHH + p;
  int rows = part_rows(part, bd);
  row = (int)(loc % rows);
  col = (int)(loc / rows);
  // the six block offsets are stored in part order (hhhh, pppp, pphh, phph, ppph, phhh)
  pos = __ldg(L.boff + 6 * q + p) + loc;
}

// block-level sum of a double across a CTA (fixed order => deterministic)
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < NT / 32; ++i) s += sh[i];
  __syncthreads();
  return s;
}

}  // namespace qd
