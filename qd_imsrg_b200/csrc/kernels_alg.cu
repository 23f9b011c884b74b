// kernels_alg.cu -- bandwidth-bound kernels of the commutator engine:
// axpy (add_arrays), deterministic FP64 reductions (commutator_110/220 traces,
// mat_2_norm, MBPT2, HF_E2), the White generator, the Pandya re-coupling
// (calc_cc) and the particle-hole gather of commutator_222.
#include "dev_common.cuh"

namespace qd {

// BCH_EXPAND's truncated coefficients cof(1..11) (magnus_IMSRG.f90:265-267),
// for terms whose coefficient is picked on the device (whole BCH step in one
// graph): term k (0-based) adds cof[k] * INT2.
__constant__ double c_bch_cof[11] = {1.0, 0.5, 0.166666666666666666, 0.04166666666666666,
                                     0.0083333333333333333, .001388888888888, 1.984126984e-4, 2.48015873e-5,
                                     2.755731922e-6, 2.755731922e-7, 2.505210839e-8};

// ---------------------------------------------------------------------------
// add_arrays (src/ME_general.f90:592-618): c = sa*a + sb*b over the whole
// vectorize array (E0 included).  double2-vectorised when all three pointers
// share 16-byte alignment.  Products and sum are rounded separately (no FMA
// contraction), as in the reference's build, so the result is bit-identical.
// ---------------------------------------------------------------------------
__global__ void k_axpy(const double* __restrict__ a, double sa, const double* __restrict__ b, double sb,
                       double* __restrict__ c, i64 n) {
  i64 stride = (i64)gridDim.x * blockDim.x;
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    c[i] = __dadd_rn(__dmul_rn(sa, a[i]), __dmul_rn(sb, b[i]));
}
__global__ void k_axpy2(const double2* __restrict__ a, double sa, const double2* __restrict__ b, double sb,
                        double2* __restrict__ c, i64 n2) {
  i64 stride = (i64)gridDim.x * blockDim.x;
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += stride) {
    double2 x = a[i], y = b[i];
    c[i] = make_double2(__dadd_rn(__dmul_rn(sa, x.x), __dmul_rn(sb, y.x)),
                       __dadd_rn(__dmul_rn(sa, x.y), __dmul_rn(sb, y.y)));
  }
}

// zero every entry of op outside the parts in `keep` (bit P_* per part, bit
// P_COUNT for E0)
__global__ void k_keep_parts(DevLayout L, double* __restrict__ op, unsigned keep) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= L.neq) return;
  int part;
  if (e < L.o_fhh)
    part = P_COUNT;
  else if (e < L.o_fpp)
    part = P_FHH;
  else if (e < L.o_fph)
    part = P_FPP;
  else if (e < L.o2)
    part = P_FPH;
  else
    part = P_HHHH + (__ldg(L.s2id + find_seg(L.s2off, L.ns2, e)) & 7);
  if (!((keep >> part) & 1u)) op[e] = 0.0;
}

int launch_keep_parts(qd_layout* L, double* op, unsigned keep) {
  if (L->neq > 0) k_keep_parts<<<(unsigned)((L->neq + 255) / 256), 256, 0, L->stream>>>(L->dev, op, keep);
  ++L->nlaunch;
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

int launch_axpy(qd_layout* L, const double* a, double sa, const double* b, double sb, double* c, i64 n) {
  const int threads = 256, blocks = 148 * 8;
  if ((((uintptr_t)a | (uintptr_t)b | (uintptr_t)c) & 15) == 0) {
    k_axpy2<<<blocks, threads, 0, L->stream>>>((const double2*)a, sa, (const double2*)b, sb, (double2*)c, n / 2);
    ++L->nlaunch;
    if (n & 1) {
      k_axpy<<<1, 32, 0, L->stream>>>(a + n - 1, sa, b + n - 1, sb, c + n - 1, 1);
      ++L->nlaunch;
    }
  } else {
    k_axpy<<<blocks, threads, 0, L->stream>>>(a, sa, b, sb, c, n);
    ++L->nlaunch;
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// ---------------------------------------------------------------------------
// Deterministic two-stage reductions.  Stage 1: RED_BLOCKS CTAs, fixed
// element->thread assignment, fixed tree -> partial[b].  Stage 2: one CTA sums
// the partials in a fixed order and writes scale*sum (+ add*out) to *out.
// ---------------------------------------------------------------------------
struct RedDotRange {  // sum a[i]*b[i] (or a[i]^2) over [o, o+n)
  const double* a;
  const double* b;
  i64 o;
  __device__ double operator()(i64 i) const {
    double x = a[o + i];
    return x * (b ? b[o + i] : x);
  }
};

struct RedDotPart {  // sum over all entries of one two-body part: a*b (or a^2)
  DevLayout L;
  const double* a;
  const double* b;
  int p;
  __device__ double operator()(i64 e) const {
    int q, row, col;
    i64 pos;
    part_elem(L, p, e, q, pos, row, col);
    double x = a[pos];
    return x * (b ? b[pos] : x);
  }
};

// MBPT2 (src/HFQDmod.f90:325-362): Vpphh^2 / (fhh(h1,h1)+fhh(h2,h2)-(fpp(p1,p1)+fpp(p2,p2)))
struct RedMBPT2 {
  DevLayout L;
  const double* h;
  __device__ double operator()(i64 e) const {
    int q, row, col;
    i64 pos;
    part_elem(L, P_PPHH - P_HHHH, e, q, pos, row, col);
    int2 pp = block_pair(L, q, 2, row), hh = block_pair(L, q, 0, col);
    const int n = L.n, mp = L.mp;
    double f12 = h[L.o_fpp + (pp.x - n) + (i64)(pp.x - n) * mp] + h[L.o_fpp + (pp.y - n) + (i64)(pp.y - n) * mp];
    double denom = h[L.o_fhh + hh.x + (i64)hh.x * n] + h[L.o_fhh + hh.y + (i64)hh.y * n] - f12;
    double x = h[pos];
    return x * x / denom;
  }
};

// HF_E2 trace: sum over blocks of Vhhhh(j,j)
struct RedHHTrace {
  DevLayout L;
  const double* h;
  __device__ double operator()(i64 e) const {
    int q, row, col;
    i64 pos;
    part_elem(L, P_HHHH - P_HHHH, e, q, pos, row, col);
    return row == col ? h[pos] : 0.0;
  }
};

template <class F>
__global__ void __launch_bounds__(RED_THREADS) k_reduce(F f, i64 n, double* __restrict__ partial) {
  __shared__ double sh[RED_THREADS / 32];
  double s = 0.0;
  i64 stride = (i64)gridDim.x * blockDim.x;
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) s += f(i);
  s = block_sum<RED_THREADS>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// out = scale * sum(partial) + add * (*out)
__global__ void k_reduce_final(const double* __restrict__ partial, int np, double scale, double add,
                               double* __restrict__ out) {
  __shared__ double sh[RED_THREADS / 32];
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) s += partial[i];
  s = block_sum<RED_THREADS>(s, sh);
  if (threadIdx.x == 0) *out = scale * s + (add != 0.0 ? add * (*out) : 0.0);
}

__global__ void k_sqrt(double* x) { *x = sqrt(*x); }

int ensure_reduction(qd_layout* L) {
  if (!L->d_red) {
    QD_CUDA(cudaMalloc(&L->d_red, sizeof(double) * (RED_BLOCKS + 64)));
    L->ws_bytes += sizeof(double) * (RED_BLOCKS + 64);
  }
  if (!L->h_red) QD_CUDA(cudaMallocHost(&L->h_red, sizeof(double) * 64));
  return QD_OK;
}

template <class F>
static int reduce_to(qd_layout* L, const F& f, i64 n, double scale, double add, double* dout) {
  int rc = ensure_reduction(L);
  if (rc) return rc;
  if (n > 0) {
    k_reduce<F><<<RED_BLOCKS, RED_THREADS, 0, L->stream>>>(f, n, L->d_red);
    k_reduce_final<<<1, RED_THREADS, 0, L->stream>>>(L->d_red, RED_BLOCKS, scale, add, dout);
    L->nlaunch += 2;
  } else {
    k_reduce_final<<<1, RED_THREADS, 0, L->stream>>>(L->d_red, 0, scale, add, dout);
    ++L->nlaunch;
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// Device scalar slots in d_red beyond the partials
double* red_slot(qd_layout* L, int k) { return L->d_red + RED_BLOCKS + k; }

int reduce_dot_range(qd_layout* L, const double* a, const double* b, i64 o, i64 n, double scale, double add,
                     double* dout) {
  return reduce_to(L, RedDotRange{a, b, o}, n, scale, add, dout);
}
int reduce_dot_part(qd_layout* L, const double* a, const double* b, int part, double scale, double add, double* dout) {
  int p = part - P_HHHH;
  return reduce_to(L, RedDotPart{L->dev, a, b, p}, L->dev.pcnt[p], scale, add, dout);
}
int reduce_mbpt2(qd_layout* L, const double* h, double* dout) {
  return reduce_to(L, RedMBPT2{L->dev, h}, L->dev.pcnt[P_PPHH - P_HHHH], 1.0, 0.0, dout);
}
int reduce_hhtrace(qd_layout* L, const double* h, double* dout) {
  return reduce_to(L, RedHHTrace{L->dev, h}, L->dev.pcnt[0], 1.0, 0.0, dout);
}
// BCH_EXPAND's exit test on the device (magnus_IMSRG.f90:316): after the
// term whose coefficient index is *kidx, continue while
// |INT2| cof / |INT1| >= conv and fewer than 11 terms ran; the answer sets the
// graph's loop condition (and, for the first term of a two-term loop body,
// the condition of the second).  *kidx advances by one.
__global__ void k_bch_decide(const double* __restrict__ norms, int* __restrict__ kidx, double conv,
                             cudaGraphConditionalHandle hloop, cudaGraphConditionalHandle hnext, int set_next) {
  const int k = *kidx;
  const double cof = c_bch_cof[k];
  const bool stop = norms[1] * cof / norms[0] < conv;  // NaN continues, as the host test does
  const unsigned go = (!stop && k + 1 < 11) ? 1u : 0u;
  *kidx = k + 1;
  cudaGraphSetConditional(hloop, go);
  if (set_next) cudaGraphSetConditional(hnext, go);
}

int launch_bch_decide(qd_layout* L, const double* norms, int* kidx, double conv, cudaGraphConditionalHandle hloop,
                      cudaGraphConditionalHandle hnext, int set_next) {
  k_bch_decide<<<1, 1, 0, L->stream>>>(norms, kidx, conv, hloop, hnext, set_next);
  ++L->nlaunch;
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// mat_2_norm (src/ME_general.f90:2112-2138): sqrt of the sum of squares of
// every stored one- and two-body entry (E0 excluded), sqrt on the device.
// The entries are summed in vectorize order by the fixed two-stage tree; the
// reference's order (fph, fpp, fhh, then per block hhhh, pppp, pphh, phph,
// phhh, ppph) differs only in rounding.
int reduce_norm(qd_layout* L, const double* a, double* dout) {
  int rc = reduce_to(L, RedDotRange{a, nullptr, L->o_fhh}, L->neq - L->o_fhh, 1.0, 0.0, dout);
  if (rc) return rc;
  k_sqrt<<<1, 1, 0, L->stream>>>(dout);
  ++L->nlaunch;
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// ---------------------------------------------------------------------------
// One BCH_EXPAND term update in one pass (magnus_IMSRG.f90:298-316):
//   c = sa*a + sb*b  (add_arrays, bit-identical: no FMA contraction)
// together with mat_2_norm of both inputs, |a| = |INT1| (HS before the
// update) and |b| = |INT2|, over every stored entry but E0.  Fixed grid and
// fixed element -> thread assignment: deterministic.  Partial sums: 2 per
// CTA (a, b).
// ---------------------------------------------------------------------------
constexpr int AXN_BLOCKS = 4 * 148, AXN_THREADS = 256;


// 16-byte accesses: the arrays are 16-byte aligned (cudaMalloc) and walked
// as pairs of entries; entry 0 (E0) is left out of the norms, an odd last
// entry is handled by thread 0.
__global__ void __launch_bounds__(AXN_THREADS) k_axpy_norms(const double* __restrict__ a, double sa,
                                                            const double* __restrict__ b, double sb,
                                                            double* __restrict__ c, i64 n, i64 o1,
                                                            double* __restrict__ partial,
                                                            const int* __restrict__ kidx) {
  __shared__ double sh[AXN_THREADS / 32];
  if (kidx) sb = c_bch_cof[*kidx];  // coefficient of the term the device counter names
  double an = 0.0, bn = 0.0;
  const i64 stride = (i64)gridDim.x * blockDim.x;
  const i64 n2 = n >> 1;
  const double2* a2 = reinterpret_cast<const double2*>(a);
  const double2* b2 = reinterpret_cast<const double2*>(b);
  double2* c2 = reinterpret_cast<double2*>(c);
  for (i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x; j < n2; j += stride) {
    const double2 x = a2[j], y = b2[j];
    c2[j] = make_double2(__dadd_rn(__dmul_rn(sa, x.x), __dmul_rn(sb, y.x)),
                         __dadd_rn(__dmul_rn(sa, x.y), __dmul_rn(sb, y.y)));
    if (2 * j >= o1) {
      an += x.x * x.x;
      bn += y.x * y.x;
    }
    if (2 * j + 1 >= o1) {
      an += x.y * x.y;
      bn += y.y * y.y;
    }
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const double x = a[n - 1], y = b[n - 1];
    c[n - 1] = __dadd_rn(__dmul_rn(sa, x), __dmul_rn(sb, y));
    if (n - 1 >= o1) {
      an += x * x;
      bn += y * y;
    }
  }
  an = block_sum<AXN_THREADS>(an, sh);
  bn = block_sum<AXN_THREADS>(bn, sh);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = an;
    partial[gridDim.x + blockIdx.x] = bn;
  }
}

// out[0] = |a|, out[1] = |b|
__global__ void k_axpy_norms_final(const double* __restrict__ partial, int np, double* __restrict__ out) {
  __shared__ double sh[RED_THREADS / 32];
  double v[2];
  for (int k = 0; k < 2; ++k) {
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partial[k * np + i];
    v[k] = block_sum<RED_THREADS>(s, sh);
  }
  if (threadIdx.x == 0) {
    out[0] = sqrt(v[0]);
    out[1] = sqrt(v[1]);
  }
}

int launch_axpy_norms(qd_layout* L, const double* a, double sa, const double* b, double sb, double* c,
                      double* dout2, const int* kidx) {
  if (!L->d_axn) {
    QD_CUDA(cudaMalloc(&L->d_axn, sizeof(double) * 2 * AXN_BLOCKS));
    L->ws_bytes += sizeof(double) * 2 * AXN_BLOCKS;
  }
  if ((((uintptr_t)a | (uintptr_t)b | (uintptr_t)c) & 15) != 0) {
    set_error("launch_axpy_norms: operator arrays must be 16-byte aligned");
    return QD_ERR_ARG;
  }
  k_axpy_norms<<<AXN_BLOCKS, AXN_THREADS, 0, L->stream>>>(a, sa, b, sb, c, L->neq, L->o_fhh, L->d_axn, kidx);
  k_axpy_norms_final<<<1, RED_THREADS, 0, L->stream>>>(L->d_axn, AXN_BLOCKS, dout2);
  L->nlaunch += 2;
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// ---------------------------------------------------------------------------
// build_white (src/IMSRG_tools.f90:377-434)
// ---------------------------------------------------------------------------
__global__ void k_white_1b(DevLayout L, double* __restrict__ gen, const double* __restrict__ h, double herm) {
  i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = L.n, mp = L.mp;
  if (e >= (i64)mp * n) return;
  int a = (int)(e % mp), i = (int)(e / mp);  // fph(a,i), a particle-local
  int as = n + a;
  double d = h[L.o_fpp + a + (i64)a * mp] - h[L.o_fhh + i + (i64)i * n] - dv_elem(L, h, herm, as, i, as, i);
  gen[L.o_fph + e] = h[L.o_fph + e] / d;
}

__global__ void k_white_2b(DevLayout L, double* __restrict__ gen, const double* __restrict__ h, double herm) {
  i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= L.pcnt[P_PPHH - P_HHHH]) return;
  int q, row, col;
  i64 pos;
  part_elem(L, P_PPHH - P_HHHH, e, q, pos, row, col);
  int2 p = block_pair(L, q, 2, row), hh = block_pair(L, q, 0, col);
  const int n = L.n, mp = L.mp;
  double efs = h[L.o_fpp + (p.x - n) + (i64)(p.x - n) * mp];
  efs = efs + h[L.o_fpp + (p.y - n) + (i64)(p.y - n) * mp];
  efs = efs - h[L.o_fhh + hh.x + (i64)hh.x * n];
  efs = efs - h[L.o_fhh + hh.y + (i64)hh.y * n];
  double Aph = dv_elem(L, h, herm, p.x, p.y, p.x, p.y) + dv_elem(L, h, herm, hh.x, hh.y, hh.x, hh.y) -
               dv_elem(L, h, herm, p.x, hh.x, p.x, hh.x) - dv_elem(L, h, herm, p.x, hh.y, p.x, hh.y) -
               dv_elem(L, h, herm, p.y, hh.x, p.y, hh.x) - dv_elem(L, h, herm, p.y, hh.y, p.y, hh.y);
  gen[pos] = h[pos] / (efs + Aph);
}

int launch_white(qd_layout* L, double* gen, const double* h, int herm) {
  i64 n1 = (i64)L->mp * L->n;
  if (n1 > 0) {
    k_white_1b<<<(unsigned)((n1 + 255) / 256), 256, 0, L->stream>>>(L->dev, gen, h, (double)herm);
    ++L->nlaunch;
  }
  i64 n2 = L->dev.pcnt[P_PPHH - P_HHHH];
  if (n2 > 0) {
    k_white_2b<<<(unsigned)((n2 + 255) / 256), 256, 0, L->stream>>>(L->dev, gen, h, (double)herm);
    ++L->nlaunch;
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// ---------------------------------------------------------------------------
// calc_cc (src/commutators.f90:1135-1159): X_q(r,nb) = v_elem(j,k,i,l,H)
// with (i,j) the r-th row pair and (k,l) the nb-th (hole,particle) column pair.
// ---------------------------------------------------------------------------
__global__ void k_calc_cc(DevLayout L, const double* __restrict__ h, double herm, double* __restrict__ X,
                          i64 xsize) {
  i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= xsize) return;
  int q = find_seg(L.ccxoff, L.ncc, e);
  i64 loc = e - __ldg(L.ccxoff + q);
  int2 d = __ldg(&L.ccdim[q]);
  int r = (int)(loc % d.x), c = (int)(loc / d.x);
  int2 ab = __ldg(&L.ccab[__ldg(&L.ccab_base[q]) + r]);
  int2 kl = __ldg(&L.cchp[__ldg(&L.cchp_base[q]) + c]);
  X[e] = dv_elem(L, h, herm, ab.y, kl.x, ab.x, kl.y);
}

int launch_calc_cc(qd_layout* L, const qd_op* H, double* X) {
  if (L->xsize > 0) {
    k_calc_cc<<<(unsigned)((L->xsize + 255) / 256), 256, 0, L->stream>>>(L->dev, H->d, (double)H->herm, X, L->xsize);
    ++L->nlaunch;
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// Device memory of the particle-hole channel: Z and the tile plan that
// re-couples it (built here, ahead of any stream capture).
int ensure_z(qd_layout* L) {
  if (!L->d_z && L->zsize > 0) {
    QD_CUDA(cudaMalloc(&L->d_z, sizeof(double) * L->zsize));
    L->ws_bytes += sizeof(double) * L->zsize;
  }
  return prepare_pandya(L);
}

}  // namespace qd
