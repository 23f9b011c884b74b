// kernels_body.cu -- the v_elem-driven contractions of the commutator:
// commutator_121, the trace part of commutator_221 and commutator_122.
#include "dev_common.cuh"

namespace qd {

// one-body target t in vectorize order of the one-body part:
//   fhh(x,y) n*n, then fpp n_p*n_p, then fph n_p*n  -> (x,y) as 0-based states
__device__ __forceinline__ void decode1b(const DevLayout& L, i64 t, int& x, int& y) {
  const int n = L.n, mp = L.mp;
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
// ---------------------------------------------------------------------------
__global__ void k_121(DevLayout L, const double* __restrict__ A, double hA, const double* __restrict__ B, double hB,
                      double* __restrict__ C) {
  const i64 n1 = (i64)L.n * L.n + (i64)L.mp * L.mp + (i64)L.mp * L.n;
  i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n1) return;
  int x, y;
  decode1b(L, t, x, y);
  const int n = L.n, mp = L.mp;
  double s = 0.0;
  {
    int q = __ldg(&L.ccmap[x * L.m + y]).x;
    int base = __ldg(&L.cchp_base[q]), nb = __ldg(&L.ccdim[q]).y;
    for (int k = 0; k < nb; ++k) {
      int2 ia = __ldg(&L.cchp[base + k]);
      const int i = ia.x, a = ia.y;
      double fa = A[L.o_fph + (a - n) + (i64)i * mp], fb = B[L.o_fph + (a - n) + (i64)i * mp];
      s += fa * hA * dv_elem(L, B, hB, a, x, i, y) - fb * hB * dv_elem(L, A, hA, a, x, i, y);
    }
  }
  {
    int q = __ldg(&L.ccmap[y * L.m + x]).x;
    int base = __ldg(&L.cchp_base[q]), nb = __ldg(&L.ccdim[q]).y;
    for (int k = 0; k < nb; ++k) {
      int2 ia = __ldg(&L.cchp[base + k]);
      const int i = ia.x, a = ia.y;
      double fa = A[L.o_fph + (a - n) + (i64)i * mp], fb = B[L.o_fph + (a - n) + (i64)i * mp];
      s += -fa * dv_elem(L, B, hB, i, x, a, y) + fb * dv_elem(L, A, hA, i, x, a, y);
    }
  }
  C[L.o_fhh + t] += s;
}

int launch_121(qd_layout* L, const qd_op* A, const qd_op* B, double* C) {
  i64 n1 = (i64)L->n * L->n + (i64)L->mp * L->mp + (i64)L->mp * L->n;
  if (n1 > 0) {
    k_121<<<(unsigned)((n1 + 127) / 128), 128, 0, L->stream>>>(L->dev, A->d, (double)A->herm, B->d, (double)B->herm,
                                                               C);
    ++L->nlaunch;
  }
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
  decode1b(L, t, x, y);
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

}  // namespace qd
