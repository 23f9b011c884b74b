// kernels_body.cu -- the v_elem-driven one-body contractions of the
// commutator: commutator_121 and the trace part of commutator_221.
#include <vector>

#include "dev_common.cuh"

namespace qd {

// one-body target t in vectorize order of the one-body part:
//   fhh(x,y) n*n, then fpp n_p*n_p, then fph n_p*n  -> (x,y) as 0-based states
__host__ __device__ inline void decode1b(int n, int mp, i64 t, int& x, int& y) {
  i64 nhh = (i64)n * n, npp = (i64)mp * mp;
  if (t < nhh) {
    x = (int)(t % n);
    y = (int)(t / n);
  } else if (t < nhh + npp) {
    t -= nhh;
    x = n + (int)(t % mp);
    y = n + (int)(t / mp);
  } else {
    t -= nhh + npp;
    x = n + (int)(t % mp);
    y = (int)(t / mp);
  }
}

// ---------------------------------------------------------------------------
// commutator_121 (src/commutators.f90:73-134), accumulating into the
// one-body part of C.  For a target (x,y):
//   C(x,y) += sum_{i,a} fA(a,i) [hA VB(a,x,i,y) - VB(i,x,a,y)]
//                     - fB(a,i) [hB VA(a,x,i,y) - VA(i,x,a,y)]
// VB(a,x,i,y) is non-zero only for (i hole, a particle) with
// ml_i - ml_a = ml_x - ml_y (and ms alike): the (hole, particle) column list
// of cross-coupled block ccmap(x,y); VB(i,x,a,y) needs the block ccmap(y,x).
// Every term carries a factor fph(a,i) of A or B; a cross-coupled block in
// which both are zero (for operators that conserve (m_l, m_s): every block
// but Delta m_l = Delta m_s = 0) adds exact zeros and is skipped (ccflag).
// ---------------------------------------------------------------------------
__global__ void k_ccflag(DevLayout L, const double* __restrict__ A, const double* __restrict__ B,
                         int* __restrict__ flag) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;  // (hole i, particle a) = (e % n, n + e / n)
  if (e >= L.n * L.mp) return;
  const int i = e % L.n, a = L.n + e / L.n;
  const i64 f = L.o_fph + (a - L.n) + (i64)i * L.mp;
  if (A[f] != 0.0 || B[f] != 0.0) flag[__ldg(&L.ccmap[i * L.m + a]).x] = 1;
}

// stored part holding pairs of classes c1, c2 (0 hh, 1 ph, 2 pp), as a P_* bit
__device__ __forceinline__ unsigned part_bit_of(int c1, int c2) {
  const int hi = c1 > c2 ? c1 : c2, lo = c1 > c2 ? c2 : c1;
  const int part = hi == 0 ? P_HHHH : (hi == 1 ? (lo == 0 ? P_PHHH : P_PHPH) : (lo == 0 ? P_PPHH : (lo == 1 ? P_PPPH : P_PPPP)));
  return 1u << part;
}

// One warp per target: the lanes split the (hole, particle) column sums of
// the target's cross-coupled blocks and a fixed shuffle tree adds them (only
// the targets of flagged blocks do work, about 2,900 of 176,400 at N=20,
// R=20 for (m_l, m_s)-conserving operators, so one thread per target would
// leave most SMs idle).
constexpr int T121 = 256;
__global__ void __launch_bounds__(T121) k_121(DevLayout L, const double* __restrict__ A, double hA,
                                              const double* __restrict__ B, double hB, unsigned zA, unsigned zB,
                                              const int* __restrict__ flag, double* __restrict__ C) {
  const i64 n1 = (i64)L.n * L.n + (i64)L.mp * L.mp + (i64)L.mp * L.n;
  const i64 t = ((i64)blockIdx.x * T121 + threadIdx.x) >> 5;  // warp-uniform
  const int lane = threadIdx.x & 31;
  if (t >= n1) return;
  int x, y;
  decode1b(L.n, L.mp, t, x, y);
  const int n = L.n, mp = L.mp;
  const int q1 = __ldg(&L.ccmap[x * L.m + y]).x, q2 = __ldg(&L.ccmap[y * L.m + x]).x;
  const bool on1 = __ldg(flag + q1) != 0, on2 = __ldg(flag + q2) != 0;
  if (!on1 && !on2) return;
  // the two-body elements of each sum lie in one part fixed by the target's
  // hole/particle types: a part known to be zero makes its terms exact zeros
  const bool px = x >= n, py = y >= n;
  const unsigned part1 = part_bit_of(px ? 2 : 1, py ? 1 : 0);  // <a x|i y>, a particle, i hole
  const unsigned part2 = part_bit_of(px ? 1 : 0, py ? 2 : 1);  // <i x|a y>
  const bool b1 = !(zB & part1), a1 = !(zA & part1), b2 = !(zB & part2), a2 = !(zA & part2);
  double s = 0.0;
  if (on1 && (a1 || b1)) {
    const int base = __ldg(&L.cchp_base[q1]), nb = __ldg(&L.ccdim[q1]).y;
    for (int k = lane; k < nb; k += 32) {
      const int2 ia = __ldg(&L.cchp[base + k]);
      const int i = ia.x, a = ia.y;
      const double fa = A[L.o_fph + (a - n) + (i64)i * mp], fb = B[L.o_fph + (a - n) + (i64)i * mp];
      const double tb = b1 ? fa * hA * dv_elem(L, B, hB, a, x, i, y) : 0.0;
      const double ta = a1 ? fb * hB * dv_elem(L, A, hA, a, x, i, y) : 0.0;
      s += tb - ta;
    }
  }
  if (on2 && (a2 || b2)) {
    const int base = __ldg(&L.cchp_base[q2]), nb = __ldg(&L.ccdim[q2]).y;
    for (int k = lane; k < nb; k += 32) {
      const int2 ia = __ldg(&L.cchp[base + k]);
      const int i = ia.x, a = ia.y;
      const double fa = A[L.o_fph + (a - n) + (i64)i * mp], fb = B[L.o_fph + (a - n) + (i64)i * mp];
      const double tb = b2 ? -fa * dv_elem(L, B, hB, i, x, a, y) : 0.0;
      const double ta = a2 ? fb * dv_elem(L, A, hA, i, x, a, y) : 0.0;
      s += tb + ta;
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) C[L.o_fhh + t] += s;
}

int launch_121(qd_layout* L, const qd_op* A, const qd_op* B, double* C) {
  const i64 n1 = (i64)L->n * L->n + (i64)L->mp * L->mp + (i64)L->mp * L->n;
  if (n1 == 0 || L->ncc == 0) return QD_OK;
  if (!L->d_ccflag) {
    void* p = nullptr;
    QD_CUDA(cudaMalloc(&p, sizeof(int) * L->ncc));
    L->dev_allocs.push_back(p);
    L->d_ccflag = (int*)p;
  }
  QD_CUDA(cudaMemsetAsync(L->d_ccflag, 0, sizeof(int) * L->ncc, L->stream));
  const int nhp = L->n * L->mp;
  if (nhp > 0) {
    k_ccflag<<<(nhp + 255) / 256, 256, 0, L->stream>>>(L->dev, A->d, B->d, L->d_ccflag);
    ++L->nlaunch;
  }
  k_121<<<(unsigned)((n1 * 32 + T121 - 1) / T121), T121, 0, L->stream>>>(L->dev, A->d, (double)A->herm, B->d,
                                                                         (double)B->herm, A->zero_mask, B->zero_mask,
                                                                         L->d_ccflag, C);
  ++L->nlaunch;
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// ---------------------------------------------------------------------------
// Trace part of commutator_221 (src/commutators.f90:280-348) on the
// intermediates w1, w2 (read through v_elem with their own herm).  Only
// targets whose two states share (ml,ms) receive non-zero terms.
// ---------------------------------------------------------------------------
__global__ void k_221_trace(DevLayout L, double hA, double hB, const double* __restrict__ w1, double h1w,
                            const double* __restrict__ w2, double h2w, double* __restrict__ C) {
  const int n = L.n, mp = L.mp, m = L.m;
  const i64 nhh = (i64)n * n, npp = (i64)mp * mp;
  const i64 n1 = nhh + npp + (i64)mp * n;
  i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n1) return;
  int x, y;
  decode1b(n, mp, t, x, y);
  if (__ldg(&L.gid[x]) != __ldg(&L.gid[y])) return;
  double s = 0.0;
  if (t < nhh) {  // fhh(h,h2): x = h, y = h2
    for (int i = 0; i < n; ++i) s += hA * dv_elem(L, w1, h1w, i, y, i, x) - hB * dv_elem(L, w1, h1w, i, x, i, y);
    for (int a = n; a < m; ++a) s += -hA * dv_elem(L, w2, h2w, a, y, a, x) + hB * dv_elem(L, w2, h2w, a, x, a, y);
  } else if (t < nhh + npp) {  // fpp(p,p2): x = p, y = p2
    for (int i = 0; i < n; ++i) s += hA * dv_elem(L, w1, h1w, i, y, i, x) - hB * dv_elem(L, w1, h1w, i, x, i, y);
    for (int a = n; a < m; ++a) s += -hA * dv_elem(L, w1, h1w, a, y, a, x) + hB * dv_elem(L, w1, h1w, a, x, a, y);
  } else {  // fph(p,h): x = p, y = h
    for (int i = 0; i < n; ++i) s += hA * dv_elem(L, w2, h2w, i, x, i, y) - hB * dv_elem(L, w1, h1w, i, x, i, y);
    for (int a = n; a < m; ++a) s += -hA * dv_elem(L, w2, h2w, a, x, a, y) + hB * dv_elem(L, w1, h1w, a, x, a, y);
  }
  C[L.o_fhh + t] += s;
}

int launch_221_trace(qd_layout* L, const qd_op* A, const qd_op* B, const qd_op* w1, const qd_op* w2, double* C) {
  i64 n1 = (i64)L->n * L->n + (i64)L->mp * L->mp + (i64)L->mp * L->n;
  if (n1 > 0) {
    k_221_trace<<<(unsigned)((n1 + 127) / 128), 128, 0, L->stream>>>(L->dev, (double)A->herm, (double)B->herm, w1->d,
                                                                     (double)w1->herm, w2->d, (double)w2->herm, C);
    ++L->nlaunch;
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// ---------------------------------------------------------------------------
// commutator_221 without its intermediates.  The trace above reads w1 and
// w2 (herm +1, as allocate_everything leaves them) only at
//   fhh: w1 hhhh (i legs), w2 phph (a legs);  fpp: w1 phph, w1 pppp;
//   fph: w2/w1 phhh (i legs), w2/w1 ppph (a legs),
// and each stored element of those parts is one column dot product of the
// products commutator_221 forms (src/commutators.f90:211-278):
//   w1 hhhh = Bpphh^T Apphh   w1 pppp = Apphh Bpphh^T   w1 phph = Bppph^T Appph
//   w2 phph = Aphhh Bphhh^T   w1 phhh = Bppph^T Apphh   w2 phhh = Appph^T Bpphh
//   w1 ppph = Apphh Bphhh^T   w2 ppph = Bpphh Aphhh^T
// k_221_fused evaluates exactly those elements on the fly (one CTA per
// target whose states share (m_l, m_s); threads over the hole/particle leg,
// fixed-order block sum), so the w1/w2 products and their memsets (2 x 8 neq
// bytes written per commutator) disappear.  Used by the full commutator;
// qd_commutator_221 keeps the reference's visible w1/w2.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double w221_stored(const DevLayout& L, int which, int q, int sl, int r, int c,
                                              const double* __restrict__ A, const double* __restrict__ B,
                                              unsigned zA, unsigned zB) {
  // an operand part known to be zero makes the element an exact zero
  auto zero = [&](unsigned za, unsigned zb) { return ((zA & za) | (zB & zb)) != 0u; };
  const unsigned pphh = 1u << P_PPHH, ppph = 1u << P_PPPH, phhh = 1u << P_PHHH;
  const int4 bd = __ldg(&L.blk[q]);
  const int nh = bd.x, nb = bd.y, np = bd.z;
  const i64* o = L.boff + 6 * q;
  double s = 0.0;
  // slots: 0 hhhh, 1 pppp, 2 pphh, 3 phph, 4 ppph, 5 phhh
  if (which == 1) {
    switch (sl) {
      case 0: {  // Bpphh^T Apphh
        if (zero(pphh, pphh)) break;
        const double* u = B + __ldg(o + 2) + (i64)r * np;
        const double* v = A + __ldg(o + 2) + (i64)c * np;
        for (int k = 0; k < np; ++k) s += u[k] * v[k];
        break;
      }
      case 1: {  // Apphh Bpphh^T
        if (zero(pphh, pphh)) break;
        const double* u = A + __ldg(o + 2) + r;
        const double* v = B + __ldg(o + 2) + c;
        for (int k = 0; k < nh; ++k) s += u[(i64)k * np] * v[(i64)k * np];
        break;
      }
      case 3: {  // Bppph^T Appph
        if (zero(ppph, ppph)) break;
        const double* u = B + __ldg(o + 4) + (i64)r * np;
        const double* v = A + __ldg(o + 4) + (i64)c * np;
        for (int k = 0; k < np; ++k) s += u[k] * v[k];
        break;
      }
      case 5: {  // Bppph^T Apphh
        if (zero(pphh, ppph)) break;
        const double* u = B + __ldg(o + 4) + (i64)r * np;
        const double* v = A + __ldg(o + 2) + (i64)c * np;
        for (int k = 0; k < np; ++k) s += u[k] * v[k];
        break;
      }
      case 4: {  // Apphh Bphhh^T
        if (zero(pphh, phhh)) break;
        const double* u = A + __ldg(o + 2) + r;
        const double* v = B + __ldg(o + 5) + c;
        for (int k = 0; k < nh; ++k) s += u[(i64)k * np] * v[(i64)k * nb];
        break;
      }
      default: break;
    }
  } else {
    switch (sl) {
      case 3: {  // Aphhh Bphhh^T
        if (zero(phhh, phhh)) break;
        const double* u = A + __ldg(o + 5) + r;
        const double* v = B + __ldg(o + 5) + c;
        for (int k = 0; k < nh; ++k) s += u[(i64)k * nb] * v[(i64)k * nb];
        break;
      }
      case 5: {  // Appph^T Bpphh
        if (zero(ppph, pphh)) break;
        const double* u = A + __ldg(o + 4) + (i64)r * np;
        const double* v = B + __ldg(o + 2) + (i64)c * np;
        for (int k = 0; k < np; ++k) s += u[k] * v[k];
        break;
      }
      case 4: {  // Bpphh Aphhh^T
        if (zero(phhh, pphh)) break;
        const double* u = B + __ldg(o + 2) + r;
        const double* v = A + __ldg(o + 5) + c;
        for (int k = 0; k < nh; ++k) s += u[(i64)k * np] * v[(i64)k * nb];
        break;
      }
      default: break;
    }
  }
  return s;
}

// v_elem(w, a, b, c, d) of intermediate w (herm +1) through w221_stored
__device__ __forceinline__ double w221(const DevLayout& L, int which, const double* __restrict__ A,
                                       const double* __restrict__ B, unsigned zA, unsigned zB, int a, int b, int c,
                                       int d) {
  if (a == b || c == d) return 0.0;
  const int e1 = __ldg(&L.ptab[a * L.m + b]);
  const int e2 = __ldg(&L.ptab[c * L.m + d]);
  const int q = pt_blk(e1);
  if (q != pt_blk(e2)) return 0.0;
  const double sgn = (pt_swap(e1) ^ pt_swap(e2)) ? -1.0 : 1.0;
  int c1 = pt_cls(e1), c2 = pt_cls(e2), i1 = pt_idx(e1), i2 = pt_idx(e2);
  if (c1 < c2) {  // upper class: herm (+1) times the transposed stored element
    int t = c1; c1 = c2; c2 = t;
    t = i1; i1 = i2; i2 = t;
  }
  int sl;
  if (c1 == 0) sl = 0;
  else if (c1 == 1) sl = c2 == 0 ? 5 : 3;
  else sl = c2 == 0 ? 2 : (c2 == 1 ? 4 : 1);
  return sgn * w221_stored(L, which, q, sl, i1, i2, A, B, zA, zB);
}

// Term descriptor of one w221 read: the stored element (which, q, slot, r, c)
// of intermediate `which`, or none; the dot product that forms it is
// resolved by w221_dot.
struct W221Term {
  int q, sl, r, c;  // sl < 0: the read is an exact zero
  int which;
};

__device__ __forceinline__ W221Term w221_term(const DevLayout& L, int which, unsigned zA, unsigned zB, int a, int b,
                                              int c, int d, double& sgn) {
  W221Term t{0, -1, 0, 0, which};
  sgn = 0.0;
  if (a == b || c == d) return t;
  const int e1 = __ldg(&L.ptab[a * L.m + b]);
  const int e2 = __ldg(&L.ptab[c * L.m + d]);
  const int q = pt_blk(e1);
  if (q != pt_blk(e2)) return t;
  sgn = (pt_swap(e1) ^ pt_swap(e2)) ? -1.0 : 1.0;
  int c1 = pt_cls(e1), c2 = pt_cls(e2), i1 = pt_idx(e1), i2 = pt_idx(e2);
  if (c1 < c2) {  // upper class: herm (+1) times the transposed stored element
    int x = c1; c1 = c2; c2 = x;
    x = i1; i1 = i2; i2 = x;
  }
  int sl;
  if (c1 == 0) sl = 0;
  else if (c1 == 1) sl = c2 == 0 ? 5 : 3;
  else sl = c2 == 0 ? 2 : (c2 == 1 ? 4 : 1);
  // parts of the operands the product reads (as in w221_stored)
  const unsigned pphh = 1u << P_PPHH, ppph = 1u << P_PPPH, phhh = 1u << P_PHHH;
  unsigned za = 0, zb = 0;
  bool live = true;
  if (which == 1) {
    switch (sl) {
      case 0: case 1: za = pphh; zb = pphh; break;
      case 3: za = ppph; zb = ppph; break;
      case 5: za = pphh; zb = ppph; break;
      case 4: za = pphh; zb = phhh; break;
      default: live = false; break;
    }
  } else {
    switch (sl) {
      case 3: za = phhh; zb = phhh; break;
      case 5: za = ppph; zb = pphh; break;
      case 4: za = phhh; zb = pphh; break;
      default: live = false; break;
    }
  }
  if (!live || ((zA & za) | (zB & zb))) return t;
  t.q = q;
  t.sl = sl;
  t.r = i1;
  t.c = i2;
  return t;
}

// The dot product of w221_stored for term t: u[k * su] v[k * sv], k < K.
__device__ __forceinline__ void w221_dot(const DevLayout& L, const W221Term& t, const double* __restrict__ A,
                                         const double* __restrict__ B, const double*& u, const double*& v, int& K,
                                         int& su, int& sv) {
  const int4 bd = __ldg(&L.blk[t.q]);
  const int nh = bd.x, nb = bd.y, np = bd.z;
  const i64* o = L.boff + 6 * t.q;
  const int r = t.r, c = t.c;
  if (t.which == 1) {
    switch (t.sl) {
      case 0: u = B + __ldg(o + 2) + (i64)r * np; v = A + __ldg(o + 2) + (i64)c * np; K = np; su = sv = 1; break;
      case 1: u = A + __ldg(o + 2) + r; v = B + __ldg(o + 2) + c; K = nh; su = sv = np; break;
      case 3: u = B + __ldg(o + 4) + (i64)r * np; v = A + __ldg(o + 4) + (i64)c * np; K = np; su = sv = 1; break;
      case 5: u = B + __ldg(o + 4) + (i64)r * np; v = A + __ldg(o + 2) + (i64)c * np; K = np; su = sv = 1; break;
      default: u = A + __ldg(o + 2) + r; v = B + __ldg(o + 5) + c; K = nh; su = np; sv = nb; break;  // 4
    }
  } else {
    switch (t.sl) {
      case 3: u = A + __ldg(o + 5) + r; v = B + __ldg(o + 5) + c; K = nh; su = sv = nb; break;
      case 5: u = A + __ldg(o + 4) + (i64)r * np; v = B + __ldg(o + 2) + (i64)c * np; K = np; su = sv = 1; break;
      default: u = B + __ldg(o + 2) + r; v = A + __ldg(o + 5) + c; K = nh; su = np; sv = nb; break;  // 4
    }
  }
}

// One CTA per target whose two states share (m_l, m_s).  Phase 1: thread u
// resolves the two w221 reads of leg state u; a read whose dot product is
// short (n_h = K <= 16 entries) is summed by the thread itself, a long one
// (n_p entries, up to 1,264) is left as a term descriptor in shared memory.
// Phase 2: the CTA walks the long terms in order, thread k taking the
// entries k, k + T221, ... of each.  One block sum at the end.  Fixed
// assignment and order: deterministic.
constexpr int T221 = 128;
constexpr int K221_SHORT = 32;

__global__ void __launch_bounds__(T221) k_221_fused(DevLayout L, const int* __restrict__ targets, double hA,
                                                    double hB, const double* __restrict__ A,
                                                    const double* __restrict__ B, unsigned zA, unsigned zB,
                                                    double* __restrict__ C) {
  extern __shared__ double sh221[];
  double* coef = sh221;                                      // [2m]
  int4* term = reinterpret_cast<int4*>(sh221 + 2 * L.m);     // [2m]: {q | which << 16, sl, r, c}; sl < 0: none
  __shared__ double red[T221 / 32];
  const int n = L.n, mp = L.mp, m = L.m;
  const i64 nhh = (i64)n * n, npp = (i64)mp * mp;
  const i64 t = __ldg(targets + blockIdx.x);
  int x, y;
  decode1b(n, mp, t, x, y);
  double s = 0.0;
  for (int u = threadIdx.x; u < m; u += T221) {
    // the two reads of leg state u and their coefficients (commutators.f90:280-348)
    int w0, w1;
    int a0, b0, c0, d0;
    double f0, f1;
    if (t < nhh) {  // fhh(h,h2): x = h, y = h2
      w0 = w1 = u < n ? 1 : 2;
      a0 = u; b0 = y; c0 = u; d0 = x;
    } else if (t < nhh + npp) {  // fpp(p,p2)
      w0 = w1 = 1;
      a0 = u; b0 = y; c0 = u; d0 = x;
    } else {  // fph(p,h)
      w0 = 2;
      w1 = 1;
      a0 = u; b0 = x; c0 = u; d0 = y;
    }
    f0 = u < n ? hA : -hA;
    f1 = u < n ? -hB : hB;
    // second read: (u, x | u, y) in every case
    for (int k = 0; k < 2; ++k) {
      double sg;
      const W221Term tt = k == 0 ? w221_term(L, w0, zA, zB, a0, b0, c0, d0, sg)
                                 : w221_term(L, w1, zA, zB, u, x, u, y, sg);
      const double cf = (k == 0 ? f0 : f1) * sg;
      int4 d = make_int4(0, -1, 0, 0);
      if (tt.sl >= 0) {
        const double* pu;
        const double* pv;
        int K, su, sv;
        w221_dot(L, tt, A, B, pu, pv, K, su, sv);
        if (K <= K221_SHORT) {
          double p = 0.0;
          for (int j = 0; j < K; ++j) p += pu[(i64)j * su] * pv[(i64)j * sv];
          s += cf * p;
        } else {
          d = make_int4(tt.q | (tt.which << 16), tt.sl, tt.r, tt.c);
        }
      }
      term[2 * u + k] = d;
      coef[2 * u + k] = cf;
    }
  }
  __syncthreads();
  for (int k = 0; k < 2 * m; ++k) {
    const int4 d = term[k];
    if (d.y < 0) continue;  // uniform: every thread reads the same descriptor
    W221Term tt{d.x & 0xFFFF, d.y, d.z, d.w, d.x >> 16};
    const double* u;
    const double* v;
    int K, su, sv;
    w221_dot(L, tt, A, B, u, v, K, su, sv);
    double p = 0.0;
    for (int j = threadIdx.x; j < K; j += T221) p += u[(i64)j * su] * v[(i64)j * sv];
    s += coef[k] * p;
  }
  s = block_sum<T221>(s, red);
  if (threadIdx.x == 0) C[L.o_fhh + t] += s;
}

int launch_221_fused(qd_layout* L, const qd_op* A, const qd_op* B, double* C) {
  if (L->ntgt221 < 0) {  // targets whose two states share (m_l, m_s)
    std::vector<int> tg;
    const i64 n1 = (i64)L->n * L->n + (i64)L->mp * L->mp + (i64)L->mp * L->n;
    for (i64 t = 0; t < n1; ++t) {
      int x, y;
      decode1b(L->n, L->mp, t, x, y);
      if (L->gid[x] == L->gid[y]) tg.push_back((int)t);
    }
    void* p = nullptr;
    QD_CUDA(cudaMalloc(&p, sizeof(int) * std::max<size_t>(1, tg.size())));
    L->dev_allocs.push_back(p);
    if (!tg.empty()) QD_CUDA(cudaMemcpy(p, tg.data(), sizeof(int) * tg.size(), cudaMemcpyHostToDevice));
    L->d_tgt221 = (const int*)p;
    L->ntgt221 = (int)tg.size();
  }
  if (L->ntgt221 > 0) {
    const size_t smem = (sizeof(double) + sizeof(int4)) * 2 * (size_t)L->m;
    if (smem > 48 * 1024) QD_CUDA(cudaFuncSetAttribute(k_221_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_221_fused<<<L->ntgt221, T221, smem, L->stream>>>(L->dev, L->d_tgt221, (double)A->herm, (double)B->herm,
                                                      A->d, B->d, A->zero_mask, B->zero_mask, C);
    ++L->nlaunch;
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

}  // namespace qd
