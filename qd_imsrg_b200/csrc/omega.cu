// omega.cu -- per-element access to the Magnus operator Omega for the learned
// warm start: Omega of the White-generator flow has non-zero entries only in
// fph and Vpphh (build_white writes no other part; euler_step adds those
// parts), so its "entries" are fph (m-n) x n followed by every block's Vpphh,
// in vectorize order.
//
//   qd_omega_count     number of entries
//   qd_omega_gather    the entries of an operator (double, device)
//   qd_omega_scatter   an operator that is zero except its Omega entries
//                      (value * scale, times a per-entry factor if given)
//   qd_omega_features  16 float features per entry (the network's input)
#include "dev_common.cuh"

namespace qd {

__device__ __forceinline__ i64 omega_pos(const DevLayout& L, i64 e, int& q, int& row, int& col) {
  const i64 nph = (i64)L.mp * L.n;
  if (e < nph) {
    q = -1;
    row = (int)(e % L.mp);
    col = (int)(e / L.mp);
    return L.o_fph + e;
  }
  i64 pos;
  part_elem(L, P_PPHH - P_HHHH, e - nph, q, pos, row, col);
  return pos;
}

__global__ void k_omega_gather(DevLayout L, const double* __restrict__ G, double* __restrict__ out, i64 n) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  int q, r, c;
  out[e] = G[omega_pos(L, e, q, r, c)];
}

__global__ void k_omega_scatter(DevLayout L, const float* __restrict__ in, float scale,
                                const double* __restrict__ escale, double* __restrict__ G, i64 n) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  int q, r, c;
  G[omega_pos(L, e, q, r, c)] = (double)scale * (double)in[e] * (escale ? escale[e] : 1.0);
}

// Features of entry e (all scaled to O(1)):
//   0-3  single-particle energies of (a, b, i, j) / (10 hbar-omega), from the
//        diagonal of H's one-body part (fph entry (a,i): a, -, i, -)
//   4-7  reference occupations of (a, b, i, j) (holes 1, particles 0)
//   8    the H element at the entry / sqrt(hbar-omega) * 10
//   9    hbar-omega        10  N / 20
//   11   M_L / 10          12  M_S / 2   (the block's channel; 0 for fph)
//   13   s / 10            14  R / 20    15  1 for fph, 0 for Vpphh
__global__ void k_omega_features(DevLayout L, const double* __restrict__ H, double hw, double nbody, double emax,
                                 double s, float* __restrict__ X, i64 n) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  int q, row, col;
  const i64 pos = omega_pos(L, e, q, row, col);
  const int nh = L.n, mp = L.mp;
  auto eh = [&](int i) { return H[L.o_fhh + i + (i64)i * nh]; };
  auto ep = [&](int a) { return H[L.o_fpp + (a - nh) + (i64)(a - nh) * mp]; };
  float f[16];
  const double inv = 1.0 / (10.0 * hw);
  double ML = 0.0, MS = 0.0;
  if (q < 0) {  // fph(a, i): a = n + row, i = col
    f[0] = (float)(ep(nh + row) * inv);
    f[1] = 0.f;
    f[2] = (float)(eh(col) * inv);
    f[3] = 0.f;
    f[4] = 0.f; f[5] = 0.f; f[6] = 1.f; f[7] = 0.f;
    f[15] = 1.f;
  } else {
    const int2 pp = block_pair(L, q, 2, row), hh = block_pair(L, q, 0, col);
    f[0] = (float)(ep(pp.x) * inv);
    f[1] = (float)(ep(pp.y) * inv);
    f[2] = (float)(eh(hh.x) * inv);
    f[3] = (float)(eh(hh.y) * inv);
    f[4] = 0.f; f[5] = 0.f; f[6] = 1.f; f[7] = 1.f;
    f[15] = 0.f;
    // blocks: M_S in {-2, 0, 2} outer, M_L in [2 - 2 emax, 2 emax - 2] inner
    const int nml = L.nblock / 3;
    ML = (double)(q % nml - (nml - 1) / 2);
    MS = (double)(2 * (q / nml) - 2);
  }
  f[8] = (float)(H[pos] / sqrt(hw) * 10.0);
  f[9] = (float)hw;
  f[10] = (float)(nbody / 20.0);
  f[11] = (float)(ML / 10.0);
  f[12] = (float)(MS / 2.0);
  f[13] = (float)(s / 10.0);
  f[14] = (float)(emax / 20.0);
  float4* o = reinterpret_cast<float4*>(X + e * 16);
  o[0] = make_float4(f[0], f[1], f[2], f[3]);
  o[1] = make_float4(f[4], f[5], f[6], f[7]);
  o[2] = make_float4(f[8], f[9], f[10], f[11]);
  o[3] = make_float4(f[12], f[13], f[14], f[15]);
}

i64 omega_count(const qd_layout* L) { return (i64)L->mp * L->n + L->dev.pcnt[P_PPHH - P_HHHH]; }

}  // namespace qd

using namespace qd;

extern "C" {

int qd_omega_count(const qd_layout* L, int64_t* n) {
  if (!L || !n) {
    set_error("qd_omega_count: null argument");
    return QD_ERR_ARG;
  }
  *n = omega_count(L);
  return QD_OK;
}

int qd_omega_gather(const qd_op* G, double* d_out, int64_t n) {
  if (!G || !d_out) {
    set_error("qd_omega_gather: null argument");
    return QD_ERR_ARG;
  }
  qd_layout* L = G->L;
  if (n != omega_count(L)) {
    set_error("qd_omega_gather: %lld entries given, Omega has %lld", (long long)n, (long long)omega_count(L));
    return QD_ERR_ARG;
  }
  QD_CUDA(cudaSetDevice(L->device));
  if (n > 0) k_omega_gather<<<(unsigned)((n + 255) / 256), 256, 0, L->stream>>>(L->dev, G->d, d_out, n);
  ++L->nlaunch;
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

int qd_omega_scatter(qd_op* G, const float* d_in, float scale, const double* d_escale, int64_t n) {
  if (!G || !d_in) {
    set_error("qd_omega_scatter: null argument");
    return QD_ERR_ARG;
  }
  qd_layout* L = G->L;
  if (n != omega_count(L)) {
    set_error("qd_omega_scatter: %lld entries given, Omega has %lld", (long long)n, (long long)omega_count(L));
    return QD_ERR_ARG;
  }
  QD_CUDA(cudaSetDevice(L->device));
  QD_CUDA(cudaMemsetAsync(G->d, 0, sizeof(double) * L->neq, L->stream));
  if (n > 0)
    k_omega_scatter<<<(unsigned)((n + 255) / 256), 256, 0, L->stream>>>(L->dev, d_in, scale, d_escale, G->d, n);
  ++L->nlaunch;
  G->herm = -1;
  G->zero_mask = ALL_PARTS & ~((1u << P_FPH) | (1u << P_PPHH));
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

int qd_omega_features(const qd_op* H, double hw, double s, float* d_X, int64_t n) {
  if (!H || !d_X || !(hw > 0.0)) {
    set_error("qd_omega_features: bad argument");
    return QD_ERR_ARG;
  }
  qd_layout* L = H->L;
  if (n != omega_count(L)) {
    set_error("qd_omega_features: %lld rows given, Omega has %lld entries", (long long)n,
              (long long)omega_count(L));
    return QD_ERR_ARG;
  }
  if (((uintptr_t)d_X & 15) != 0) {
    set_error("qd_omega_features: the feature array must be 16-byte aligned");
    return QD_ERR_ARG;
  }
  QD_CUDA(cudaSetDevice(L->device));
  if (n > 0)
    k_omega_features<<<(unsigned)((n + 255) / 256), 256, 0, L->stream>>>(L->dev, H->d, hw, (double)L->n,
                                                                         (double)L->emax, s, d_X, n);
  ++L->nlaunch;
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

}  // extern "C"
