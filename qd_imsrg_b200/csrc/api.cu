// api.cu -- extern "C" entry points (include/qd_imsrg.h).
//
// Host orchestration of the reference's call sequences on device-resident
// operators; every numeric step is a kernel on the layout's stream.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <utility>

#include "dev_common.cuh"

namespace qd {
const char* last_error();
void drop_122_plan(const qd_layout* L);
}  // namespace qd

using namespace qd;

// Layout-owned workspaces used by qd_commutator (allocated on first use).
namespace {
struct Workspace {
  qd_op* w1 = nullptr;
  qd_op* w2 = nullptr;
  qd_cc* ca = nullptr;
  qd_cc* cb = nullptr;
};
std::map<const qd_layout*, Workspace>& workspaces() {
  static std::map<const qd_layout*, Workspace> m;
  return m;
}

#define CHECK(cond, code, ...)    \
  do {                            \
    if (!(cond)) {                \
      qd::set_error(__VA_ARGS__); \
      return code;                \
    }                             \
  } while (0)
#define TRY(x)               \
  do {                       \
    int rc_ = (x);           \
    if (rc_) return rc_;     \
  } while (0)

int use_device(const qd_layout* L) {
  if (L->device == QD_HOST_ONLY) {
    qd::set_error("layout was created host-only (QD_HOST_ONLY)");
    return QD_ERR_STATE;
  }
  QD_CUDA(cudaSetDevice(L->device));
  return QD_OK;
}

int op_new(qd_layout* L, int herm, qd_op** out) {
  qd_op* op = new qd_op();
  op->L = L;
  op->herm = herm;
  cudaError_t e = cudaMalloc(&op->d, sizeof(double) * L->neq);
  if (e != cudaSuccess) {
    delete op;
    return cuda_fail(e, "cudaMalloc(operator)");
  }
  QD_CUDA(cudaMemsetAsync(op->d, 0, sizeof(double) * L->neq, L->stream));
  op->zero_mask = ALL_PARTS;
  *out = op;
  return QD_OK;
}

void op_free(qd_op* op) {
  if (!op) return;
  if (op->d) cudaFree(op->d);
  delete op;
}

int cc_new(qd_layout* L, double herm, qd_cc** out) {
  qd_cc* c = new qd_cc();
  c->L = L;
  c->herm = herm;
  if (L->xsize > 0) {
    cudaError_t e = cudaMalloc(&c->d, sizeof(double) * L->xsize);
    if (e != cudaSuccess) {
      delete c;
      return cuda_fail(e, "cudaMalloc(cc)");
    }
    QD_CUDA(cudaMemsetAsync(c->d, 0, sizeof(double) * L->xsize, L->stream));
  }
  *out = c;
  return QD_OK;
}

int scalar_out(qd_layout* L, const double* dslot, double* out) {
  QD_CUDA(cudaMemcpyAsync(L->h_red, dslot, sizeof(double), cudaMemcpyDeviceToHost, L->stream));
  QD_CUDA(cudaStreamSynchronize(L->stream));
  *out = L->h_red[0];
  return QD_OK;
}

int same_layout(const qd_op* a, const qd_op* b) {
  CHECK(a && b, QD_ERR_ARG, "null operator handle");
  CHECK(a->L == b->L, QD_ERR_ARG, "operators belong to different layouts");
  return QD_OK;
}

// zero mask of a host vector: parts that are identically zero
unsigned host_zero_mask(const qd_layout* L, const double* v) {
  auto zero = [&](i64 o, i64 n) {
    for (i64 i = 0; i < n; ++i)
      if (v[o + i] != 0.0) return false;
    return true;
  };
  unsigned m = 0;
  if (zero(L->o_fhh, (i64)L->n * L->n)) m |= 1u << P_FHH;
  if (zero(L->o_fpp, (i64)L->mp * L->mp)) m |= 1u << P_FPP;
  if (zero(L->o_fph, (i64)L->mp * L->n)) m |= 1u << P_FPH;
  for (int p = 0; p < 6; ++p) {
    bool z = true;
    for (int q = 0; q < L->nblock && z; ++q) {
      i64 nh = L->blk[q].x, nb = L->blk[q].y, np = L->blk[q].z;
      i64 sz[6] = {nh * nh, np * np, np * nh, nb * nb, np * nb, nb * nh};
      z = zero(L->boff[6 * q + p], sz[p]);
    }
    if (z) m |= 1u << (P_HHHH + p);
  }
  return m;
}

// RAII stage timer: records an event pair around a stage when profiling is on
struct StageTimer {
  qd_layout* L;
  int id;
  cudaEvent_t a = nullptr, b = nullptr;
  StageTimer(qd_layout* l, int i) : L(l), id(i) {
    if (L->prof.on && cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess)
      cudaEventRecord(a, L->stream);
  }
  ~StageTimer() {
    if (L->prof.on && a && b) {
      cudaEventRecord(b, L->stream);
      L->prof.pending[id].push_back({a, b});
    }
  }
};

void prof_collect(qd_layout* L) {
  for (int s = 0; s < S_COUNT; ++s) {
    for (auto& pr : L->prof.pending[s]) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) {
        L->prof.ms[s] += ms;
        L->prof.count[s] += 1;
      }
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
    L->prof.pending[s].clear();
  }
}

// ---- the stages of one commutator [A,B] -> C ------------------------------
int stage_e0(qd_layout* L, const qd_op* A, const qd_op* B, double* dout, double add) {
  StageTimer tm(L, S_E0);
  const double dh = (double)(A->herm - B->herm);
  TRY(reduce_dot_range(L, A->d, B->d, L->o_fph, (i64)L->mp * L->n, dh, add, dout));
  TRY(reduce_dot_part(L, A->d, B->d, P_PPHH, dh, 1.0, dout));
  return QD_OK;
}

int stage_111(qd_layout* L, const qd_op* A, const qd_op* B, qd_op* C) {
  StageTimer tm(L, S_111);
  const double* bufs[7] = {A->d, B->d, nullptr, nullptr, C->d, nullptr, nullptr};
  TRY(run_program(L, L->prog_111, bufs, (double)A->herm, (double)B->herm, A->zero_mask, B->zero_mask));
  C->zero_mask &= ~((1u << P_FHH) | (1u << P_FPP) | (1u << P_FPH));
  return QD_OK;
}

int stage_221(qd_layout* L, const qd_op* A, const qd_op* B, qd_op* C, qd_op* w1, qd_op* w2) {
  StageTimer tm(L, S_221);
  QD_CUDA(cudaMemsetAsync(w1->d, 0, sizeof(double) * L->neq, L->stream));
  QD_CUDA(cudaMemsetAsync(w2->d, 0, sizeof(double) * L->neq, L->stream));
  const double* bufs[7] = {A->d, B->d, nullptr, nullptr, w1->d, w2->d, nullptr};
  TRY(run_program(L, L->prog_221, bufs, (double)A->herm, (double)B->herm, A->zero_mask, B->zero_mask));
  w1->zero_mask = 0;
  w2->zero_mask = 0;
  TRY(launch_221_trace(L, A, B, w1, w2, C->d));
  return QD_OK;
}

int stage_222(qd_layout* L, const qd_op* A, const qd_op* B, qd_op* C, const qd_cc* HCC, const qd_cc* ETACC) {
  const double* bufs[7] = {A->d, B->d, nullptr, nullptr, C->d, nullptr, nullptr};
  {
    StageTimer tm(L, S_LADDER);
    TRY(run_program(L, L->prog_ladder, bufs, (double)A->herm, (double)B->herm, A->zero_mask, B->zero_mask));
  }
  if (HCC && ETACC && HCC->filled && ETACC->filled && L->zsize > 0) {
    CHECK(std::fabs(HCC->herm) == 1.0 && std::fabs(ETACC->herm) == 1.0, QD_ERR_ARG,
          "cross-coupled herm must be +1 or -1");
    TRY(ensure_z(L));
    const double* zb[7] = {nullptr, nullptr, ETACC->d, HCC->d, nullptr, nullptr, L->d_z};
    {
      StageTimer tm(L, S_PANDYA_GEMM);
      TRY(run_program(L, L->prog_pandya, zb, ETACC->herm, HCC->herm, 0u, 0u));
    }
    StageTimer tm(L, S_PANDYA_GATHER);
    TRY(launch_pandya_gather(L, L->d_z, C->d));
  }
  C->zero_mask = 0;
  return QD_OK;
}

int commutator_seq(qd_layout* L, const qd_op* A, const qd_op* B, qd_op* C, qd_op* w1, qd_op* w2, qd_cc* ACC,
                   qd_cc* BCC, bool pandya) {
  TRY(build_programs(L));
  TRY(stage_e0(L, A, B, C->d, 0.0));
  TRY(stage_111(L, A, B, C));
  {
    StageTimer tm(L, S_121);
    TRY(launch_121(L, A, B, C->d));
  }
  TRY(stage_221(L, A, B, C, w1, w2));
  {
    StageTimer tm(L, S_122);
    TRY(launch_122(L, A, B, C->d));
  }
  if (pandya) {
    StageTimer tm(L, S_CALC_CC);
    TRY(launch_calc_cc(L, A, ACC->d));
    ACC->filled = true;
    ACC->herm = A->herm;
    TRY(launch_calc_cc(L, B, BCC->d));
    BCC->filled = true;
    BCC->herm = B->herm;
  }
  TRY(stage_222(L, A, B, C, pandya ? BCC : nullptr, pandya ? ACC : nullptr));
  C->zero_mask = 0;
  return QD_OK;
}

int get_ws(qd_layout* L, Workspace** out) {
  Workspace& w = workspaces()[L];
  if (!w.w1) TRY(op_new(L, 1, &w.w1));
  if (!w.w2) TRY(op_new(L, 1, &w.w2));
  if (!w.ca) TRY(cc_new(L, -1.0, &w.ca));
  if (!w.cb) TRY(cc_new(L, 1.0, &w.cb));
  *out = &w;
  return QD_OK;
}

void drop_ws(const qd_layout* L) {
  auto& m = workspaces();
  auto it = m.find(L);
  if (it == m.end()) return;
  op_free(it->second.w1);
  op_free(it->second.w2);
  for (qd_cc* c : {it->second.ca, it->second.cb})
    if (c) {
      if (c->d) cudaFree(c->d);
      delete c;
    }
  m.erase(it);
}

const double kCof[11] = {1.0, 0.5, 0.166666666666666666, 0.04166666666666666, 0.0083333333333333333,
                         .001388888888888, 1.984126984e-4, 2.48015873e-5, 2.755731922e-6, 2.755731922e-7,
                         2.505210839e-8};

}  // namespace

extern "C" {

const char* qd_last_error(void) { return qd::last_error(); }
const char* qd_version(void) { return "qd_imsrg_b200 0.1 (sm_100a, FP64 DMMA)"; }

int qd_layout_create(int nbody, int emax, const double* eig, int device, qd_layout** out) {
  CHECK(out, QD_ERR_ARG, "qd_layout_create: null output");
  *out = nullptr;
  if (device == QD_HOST_ONLY) {
    qd_layout* L = new qd_layout();
    L->device = QD_HOST_ONLY;
    int rc = layout_build(L, nbody, emax, eig);
    if (rc) {
      delete L;
      return rc;
    }
    *out = L;
    return QD_OK;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    qd::set_error("qd_layout_create: no CUDA device");
    return QD_ERR_NODEVICE;
  }
  qd_layout* L = new qd_layout();
  if (device < 0) {
    cudaGetDevice(&L->device);
  } else {
    L->device = device;
  }
  int rc = layout_build(L, nbody, emax, eig);
  if (rc) {
    delete L;
    return rc;
  }
  if ((rc = use_device(L)) || (rc = layout_upload(L))) {
    layout_free_device(L);
    delete L;
    return rc;
  }
  cudaError_t e = cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    layout_free_device(L);
    delete L;
    return cuda_fail(e, "cudaStreamCreate");
  }
  L->own_stream = true;
  if ((rc = ensure_reduction(L))) {
    layout_free_device(L);
    delete L;
    return rc;
  }
  *out = L;
  return QD_OK;
}

int qd_layout_destroy(qd_layout* L) {
  if (!L) return QD_OK;
  if (L->device == QD_HOST_ONLY) {
    delete L;
    return QD_OK;
  }
  cudaSetDevice(L->device);
  cudaStreamSynchronize(L->stream);
  drop_ws(L);
  drop_122_plan(L);
  layout_free_device(L);
  delete L;
  return QD_OK;
}

int qd_layout_info(const qd_layout* L, int* nbody, int* msp, int* nblock, int64_t* neq, int* ncc) {
  CHECK(L, QD_ERR_ARG, "null layout");
  if (nbody) *nbody = L->n;
  if (msp) *msp = L->m;
  if (nblock) *nblock = L->nblock;
  if (neq) *neq = L->neq;
  if (ncc) *ncc = L->ncc;
  return QD_OK;
}

int qd_layout_blocks(const qd_layout* L, int* d) {
  CHECK(L && d, QD_ERR_ARG, "null argument");
  for (int q = 0; q < L->nblock; ++q) {
    d[5 * q + 0] = L->blk[q].x;
    d[5 * q + 1] = L->blk[q].y;
    d[5 * q + 2] = L->blk[q].z;
    int MS = -2 + 2 * (q / (4 * L->emax - 3));
    int ML = 2 - 2 * L->emax + q % (4 * L->emax - 3);
    d[5 * q + 3] = ML;
    d[5 * q + 4] = MS;
  }
  return QD_OK;
}

int qd_layout_offsets(const qd_layout* L, int64_t* off6) {
  CHECK(L && off6, QD_ERR_ARG, "null argument");
  for (size_t i = 0; i < L->boff.size(); ++i) off6[i] = L->boff[i];
  return QD_OK;
}

int qd_layout_pairs(const qd_layout* L, int q, int kind, int* out, int* count) {
  CHECK(L && q >= 0 && q < L->nblock && kind >= 0 && kind <= 2, QD_ERR_ARG, "qd_layout_pairs: bad arguments");
  int nh = L->blk[q].x, nb = L->blk[q].y, np = L->blk[q].z;
  int base = L->pbase[q] + (kind == 0 ? 0 : (kind == 1 ? nh : nh + nb));
  int cnt = kind == 0 ? nh : (kind == 1 ? nb : np);
  if (count) *count = cnt;
  if (out)
    for (int k = 0; k < cnt; ++k) {
      out[2 * k] = L->pairs[base + k].x + 1;
      out[2 * k + 1] = L->pairs[base + k].y + 1;
    }
  return QD_OK;
}

int qd_layout_set_stream(qd_layout* L, void* stream) {
  CHECK(L, QD_ERR_ARG, "null layout");
  TRY(use_device(L));
  QD_CUDA(cudaStreamSynchronize(L->stream));
  if (L->own_stream && L->stream) cudaStreamDestroy(L->stream);
  if (stream) {
    L->stream = (cudaStream_t)stream;
    L->own_stream = false;
  } else {
    QD_CUDA(cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking));
    L->own_stream = true;
  }
  return QD_OK;
}

int qd_layout_synchronize(qd_layout* L) {
  CHECK(L, QD_ERR_ARG, "null layout");
  TRY(use_device(L));
  QD_CUDA(cudaStreamSynchronize(L->stream));
  return QD_OK;
}

int qd_layout_profile(qd_layout* L, int enable) {
  CHECK(L, QD_ERR_ARG, "null layout");
  TRY(use_device(L));
  QD_CUDA(cudaStreamSynchronize(L->stream));
  prof_collect(L);
  for (int s = 0; s < S_COUNT; ++s) {
    L->prof.ms[s] = 0.0;
    L->prof.count[s] = 0;
  }
  L->prof.on = enable != 0;
  return QD_OK;
}

int qd_layout_profile_read(qd_layout* L, double* ms, int64_t* counts, int nstage) {
  CHECK(L, QD_ERR_ARG, "null layout");
  TRY(use_device(L));
  QD_CUDA(cudaStreamSynchronize(L->stream));
  prof_collect(L);
  for (int s = 0; s < nstage && s < S_COUNT; ++s) {
    if (ms) ms[s] = L->prof.ms[s];
    if (counts) counts[s] = L->prof.count[s];
  }
  return QD_OK;
}

int qd_layout_launches(const qd_layout* L, int64_t* n) {
  CHECK(L && n, QD_ERR_ARG, "null argument");
  *n = L->nlaunch;
  return QD_OK;
}

int qd_layout_workspace_bytes(const qd_layout* L, int64_t* bytes) {
  CHECK(L && bytes, QD_ERR_ARG, "null argument");
  *bytes = L->ws_bytes;
  return QD_OK;
}

int qd_op_create(qd_layout* L, int herm, qd_op** out) {
  CHECK(L && out, QD_ERR_ARG, "null argument");
  TRY(use_device(L));
  return op_new(L, herm, out);
}

int qd_op_destroy(qd_op* op) {
  if (!op) return QD_OK;
  cudaSetDevice(op->L->device);
  cudaStreamSynchronize(op->L->stream);
  op_free(op);
  return QD_OK;
}

int qd_op_upload(qd_op* op, const double* v, int64_t neq) {
  CHECK(op && v, QD_ERR_ARG, "null argument");
  CHECK(neq == op->L->neq, QD_ERR_ARG, "qd_op_upload: %lld entries given, layout has %lld", (long long)neq,
        (long long)op->L->neq);
  TRY(use_device(op->L));
  QD_CUDA(cudaMemcpyAsync(op->d, v, sizeof(double) * neq, cudaMemcpyHostToDevice, op->L->stream));
  op->zero_mask = host_zero_mask(op->L, v);
  QD_CUDA(cudaStreamSynchronize(op->L->stream));
  return QD_OK;
}

int qd_op_upload_device(qd_op* op, const double* v, int64_t neq) {
  CHECK(op && v, QD_ERR_ARG, "null argument");
  CHECK(neq == op->L->neq, QD_ERR_ARG, "qd_op_upload_device: size mismatch");
  TRY(use_device(op->L));
  QD_CUDA(cudaMemcpyAsync(op->d, v, sizeof(double) * neq, cudaMemcpyDeviceToDevice, op->L->stream));
  op->zero_mask = 0;
  return QD_OK;
}

int qd_op_download(const qd_op* op, double* v, int64_t neq) {
  CHECK(op && v, QD_ERR_ARG, "null argument");
  CHECK(neq == op->L->neq, QD_ERR_ARG, "qd_op_download: size mismatch");
  TRY(use_device(op->L));
  QD_CUDA(cudaMemcpyAsync(v, op->d, sizeof(double) * neq, cudaMemcpyDeviceToHost, op->L->stream));
  QD_CUDA(cudaStreamSynchronize(op->L->stream));
  return QD_OK;
}

int qd_op_set_herm(qd_op* op, int herm) {
  CHECK(op && (herm == 1 || herm == -1), QD_ERR_ARG, "herm must be +1 or -1");
  op->herm = herm;
  return QD_OK;
}
int qd_op_get_herm(const qd_op* op, int* herm) {
  CHECK(op && herm, QD_ERR_ARG, "null argument");
  *herm = op->herm;
  return QD_OK;
}
int qd_op_device_ptr(qd_op* op, double** dptr) {
  CHECK(op && dptr, QD_ERR_ARG, "null argument");
  *dptr = op->d;
  op->zero_mask = 0;  // the caller may write through the pointer
  return QD_OK;
}

int qd_random_operator(const qd_layout* L, int herm, uint64_t seed, double sigma, int conserve, double* v,
                       int64_t neq) {
  CHECK(L && v && neq == L->neq, QD_ERR_ARG, "qd_random_operator: bad arguments");
  CHECK(herm == 1 || herm == -1, QD_ERR_ARG, "herm must be +1 or -1");
  fill_random(L, herm, seed, sigma, conserve, v);
  return QD_OK;
}

int qd_add_arrays(const qd_op* r1, double s1, const qd_op* r2, double s2, qd_op* r3) {
  TRY(same_layout(r1, r2));
  TRY(same_layout(r1, r3));
  qd_layout* L = r1->L;
  TRY(use_device(L));
  TRY(launch_axpy(L, r1->d, s1, r2->d, s2, r3->d, L->neq));
  unsigned m1 = s1 == 0.0 ? ALL_PARTS : r1->zero_mask, m2 = s2 == 0.0 ? ALL_PARTS : r2->zero_mask;
  r3->zero_mask = m1 & m2;
  return QD_OK;
}

int qd_copy_arrays(const qd_op* r1, qd_op* r2) {
  TRY(same_layout(r1, r2));
  if (r1 == r2) return QD_OK;
  TRY(use_device(r1->L));
  QD_CUDA(cudaMemcpyAsync(r2->d, r1->d, sizeof(double) * r1->L->neq, cudaMemcpyDeviceToDevice, r1->L->stream));
  r2->zero_mask = r1->zero_mask;
  return QD_OK;
}

int qd_set_to_zero(qd_op* r1) {
  CHECK(r1, QD_ERR_ARG, "null operator");
  TRY(use_device(r1->L));
  QD_CUDA(cudaMemsetAsync(r1->d, 0, sizeof(double) * r1->L->neq, r1->L->stream));
  r1->zero_mask = ALL_PARTS;
  return QD_OK;
}

int qd_mat_2_norm(const qd_op* r, double* out) {
  CHECK(r && out, QD_ERR_ARG, "null argument");
  qd_layout* L = r->L;
  TRY(use_device(L));
  TRY(reduce_norm1b(L, r->d, red_slot(L, 0)));
  return scalar_out(L, red_slot(L, 0), out);
}

int qd_commutator_110(const qd_op* r1, const qd_op* r2, double* c) {
  TRY(same_layout(r1, r2));
  CHECK(c, QD_ERR_ARG, "null output");
  qd_layout* L = r1->L;
  TRY(use_device(L));
  TRY(reduce_dot_range(L, r1->d, r2->d, L->o_fph, (i64)L->mp * L->n, (double)(r1->herm - r2->herm), 0.0,
                       red_slot(L, 0)));
  return scalar_out(L, red_slot(L, 0), c);
}

int qd_commutator_220(const qd_op* r1, const qd_op* r2, double* c) {
  TRY(same_layout(r1, r2));
  CHECK(c, QD_ERR_ARG, "null output");
  qd_layout* L = r1->L;
  TRY(use_device(L));
  TRY(reduce_dot_part(L, r1->d, r2->d, P_PPHH, (double)(r1->herm - r2->herm), 0.0, red_slot(L, 0)));
  return scalar_out(L, red_slot(L, 0), c);
}

int qd_commutator_111(const qd_op* r1, const qd_op* r2, qd_op* r3) {
  TRY(same_layout(r1, r2));
  TRY(same_layout(r1, r3));
  TRY(use_device(r1->L));
  TRY(build_programs(r1->L));
  return stage_111(r1->L, r1, r2, r3);
}

int qd_commutator_121(const qd_op* r1, const qd_op* r2, qd_op* r3) {
  TRY(same_layout(r1, r2));
  TRY(same_layout(r1, r3));
  TRY(use_device(r1->L));
  TRY(launch_121(r1->L, r1, r2, r3->d));
  r3->zero_mask &= ~((1u << P_FHH) | (1u << P_FPP) | (1u << P_FPH));
  return QD_OK;
}

int qd_commutator_221(const qd_op* r1, const qd_op* r2, qd_op* r3, qd_op* w1, qd_op* w2) {
  TRY(same_layout(r1, r2));
  TRY(same_layout(r1, r3));
  TRY(same_layout(r1, w1));
  TRY(same_layout(r1, w2));
  TRY(use_device(r1->L));
  TRY(build_programs(r1->L));
  TRY(stage_221(r1->L, r1, r2, r3, w1, w2));
  r3->zero_mask &= ~((1u << P_FHH) | (1u << P_FPP) | (1u << P_FPH));
  return QD_OK;
}

int qd_commutator_122(const qd_op* r1, const qd_op* r2, qd_op* r3) {
  TRY(same_layout(r1, r2));
  TRY(same_layout(r1, r3));
  TRY(use_device(r1->L));
  TRY(launch_122(r1->L, r1, r2, r3->d));
  r3->zero_mask &= (1u << P_FHH) | (1u << P_FPP) | (1u << P_FPH);
  return QD_OK;
}

int qd_commutator_222(const qd_op* r1, const qd_op* r2, qd_op* r3, qd_op* w1, const qd_cc* HCC, const qd_cc* ETACC) {
  (void)w1;
  TRY(same_layout(r1, r2));
  TRY(same_layout(r1, r3));
  TRY(use_device(r1->L));
  TRY(build_programs(r1->L));
  unsigned keep = r3->zero_mask & ((1u << P_FHH) | (1u << P_FPP) | (1u << P_FPH));
  TRY(stage_222(r1->L, r1, r2, r3, HCC, ETACC));
  r3->zero_mask = keep;
  return QD_OK;
}

int qd_commutator(const qd_op* A, const qd_op* B, qd_op* C, unsigned flags) {
  TRY(same_layout(A, B));
  TRY(same_layout(A, C));
  CHECK(C != A && C != B, QD_ERR_ARG, "qd_commutator: output aliases an input");
  qd_layout* L = A->L;
  TRY(use_device(L));
  Workspace* w;
  TRY(get_ws(L, &w));
  return commutator_seq(L, A, B, C, w->w1, w->w2, w->ca, w->cb, (flags & QD_PANDYA) != 0);
}

int qd_cc_create(qd_layout* L, double herm, qd_cc** out) {
  CHECK(L && out, QD_ERR_ARG, "null argument");
  TRY(use_device(L));
  return cc_new(L, herm, out);
}
int qd_cc_destroy(qd_cc* cc) {
  if (!cc) return QD_OK;
  cudaSetDevice(cc->L->device);
  cudaStreamSynchronize(cc->L->stream);
  if (cc->d) cudaFree(cc->d);
  delete cc;
  return QD_OK;
}
int qd_cc_set_herm(qd_cc* cc, double herm) {
  CHECK(cc, QD_ERR_ARG, "null cc");
  cc->herm = herm;
  return QD_OK;
}
int qd_calc_cc(const qd_op* H, qd_cc* HCC) {
  CHECK(H && HCC && H->L == HCC->L, QD_ERR_ARG, "qd_calc_cc: bad arguments");
  TRY(use_device(H->L));
  TRY(launch_calc_cc(H->L, H, HCC->d));
  HCC->filled = true;
  return QD_OK;
}
int qd_cc_download(const qd_cc* cc, double* host, int64_t n, int64_t* needed) {
  CHECK(cc, QD_ERR_ARG, "null cc");
  if (needed) *needed = cc->L->xsize;
  if (!host) return QD_OK;
  CHECK(n >= cc->L->xsize, QD_ERR_ARG, "qd_cc_download: buffer too small");
  TRY(use_device(cc->L));
  if (cc->L->xsize > 0)
    QD_CUDA(cudaMemcpyAsync(host, cc->d, sizeof(double) * cc->L->xsize, cudaMemcpyDeviceToHost, cc->L->stream));
  QD_CUDA(cudaStreamSynchronize(cc->L->stream));
  return QD_OK;
}

int qd_build_white(qd_op* gen, const qd_op* H) {
  TRY(same_layout(gen, H));
  TRY(use_device(H->L));
  TRY(launch_white(H->L, gen->d, H->d, H->herm));
  gen->zero_mask &= ~((1u << P_FPH) | (1u << P_PPHH));
  return QD_OK;
}

int qd_mbpt2(const qd_op* H, double* out) {
  CHECK(H && out, QD_ERR_ARG, "null argument");
  TRY(use_device(H->L));
  TRY(reduce_mbpt2(H->L, H->d, red_slot(H->L, 0)));
  return scalar_out(H->L, red_slot(H->L, 0), out);
}

int qd_hf_e2(qd_op* H, double* out) {
  CHECK(H, QD_ERR_ARG, "null operator");
  qd_layout* L = H->L;
  TRY(use_device(L));
  double tr;
  TRY(reduce_hhtrace(L, H->d, red_slot(L, 0)));
  TRY(scalar_out(L, red_slot(L, 0), &tr));
  double sm2 = 0.0;
  for (int i = 0; i < L->n; ++i) sm2 = sm2 + L->eig[i];
  double e = sm2 - tr;
  QD_CUDA(cudaMemcpyAsync(H->d, &e, sizeof(double), cudaMemcpyHostToDevice, L->stream));
  QD_CUDA(cudaStreamSynchronize(L->stream));
  if (out) *out = e;
  return QD_OK;
}

int qd_bch_expand(qd_op* HS, const qd_op* G, const qd_op* H, qd_op* INT1, qd_op* INT2, qd_op* AD, qd_op* w1,
                  qd_op* w2, qd_cc* HCC, qd_cc* OCC, unsigned flags, int* nterms) {
  TRY(same_layout(HS, G));
  TRY(same_layout(HS, H));
  TRY(same_layout(HS, INT2));
  TRY(same_layout(HS, AD));
  TRY(same_layout(HS, w1));
  TRY(same_layout(HS, w2));
  (void)INT1;  // the norm of INT1 (= HS before the update) is taken from HS itself
  qd_layout* L = HS->L;
  TRY(use_device(L));
  TRY(build_programs(L));
  const bool pandya = (flags & QD_PANDYA) != 0;
  auto norm = (flags & QD_FULL_NORM) ? reduce_norm_full : reduce_norm1b;
  CHECK(!pandya || (HCC && OCC), QD_ERR_ARG, "qd_bch_expand: QD_PANDYA needs HCC and OCC");
  const double conv = (double)1e-5f;  // "conv = 1e-5" is a real(4) literal in the reference
  INT2->herm = 1;
  AD->herm = 1;
  TRY(qd_copy_arrays(H, HS));
  TRY(qd_copy_arrays(HS, INT2));
  int count = 0;
  for (int i = 2; i <= 12; ++i) {
    std::swap(INT2->d, AD->d);  // AD = previous term; INT2 becomes the output buffer
    std::swap(INT2->zero_mask, AD->zero_mask);
    TRY(norm(L, HS->d, red_slot(L, 1)));  // |INT1| = |HS| before the update
    if (pandya) {
      TRY(commutator_seq(L, G, AD, INT2, w1, w2, OCC, HCC, true));
    } else {
      TRY(commutator_seq(L, G, AD, INT2, w1, w2, nullptr, nullptr, false));
    }
    ++count;
    TRY(norm(L, INT2->d, red_slot(L, 2)));
    const double cof = kCof[i - 2];
    TRY(launch_axpy(L, HS->d, 1.0, INT2->d, cof, HS->d, L->neq));
    HS->zero_mask &= INT2->zero_mask;
    QD_CUDA(cudaMemcpyAsync(L->h_red + 1, red_slot(L, 1), 2 * sizeof(double), cudaMemcpyDeviceToHost, L->stream));
    QD_CUDA(cudaStreamSynchronize(L->stream));
    const double n1 = L->h_red[1], n2 = L->h_red[2];
    if (n2 * cof / n1 < conv) break;
  }
  if (nterms) *nterms = count;
  return QD_OK;
}

int qd_magnus_expand(qd_op* DG, const qd_op* G, const qd_op* ETA) {
  (void)G;
  return qd_copy_arrays(ETA, DG);
}

int qd_euler_step(qd_op* G, const qd_op* DG, double* s, double stp) {
  TRY(qd_add_arrays(G, 1.0, DG, stp, G));
  if (s) *s = *s + stp;
  return QD_OK;
}

int qd_magnus_flow(const qd_op* HAM, qd_op* HS, unsigned flags, int max_iter, double* trace,
                   qd_flow_result* result) {
  TRY(same_layout(HAM, HS));
  qd_layout* L = HAM->L;
  TRY(use_device(L));
  const double conv_criteria = (double)1e-9f;  // real(4) literal in the reference
  qd_op *ETA = nullptr, *G = nullptr, *DG = nullptr, *ETA0 = nullptr, *G0 = nullptr, *HS0 = nullptr;
  qd_op *INT1 = nullptr, *INT2 = nullptr, *AD = nullptr, *w1 = nullptr, *w2 = nullptr;
  qd_cc *HCC = nullptr, *OCC = nullptr;
  int rc = QD_OK;
  auto cleanup = [&]() {
    cudaStreamSynchronize(L->stream);
    for (qd_op* o : {ETA, G, DG, ETA0, G0, HS0, INT1, INT2, AD, w1, w2}) op_free(o);
    for (qd_cc* c : {HCC, OCC})
      if (c) {
        if (c->d) cudaFree(c->d);
        delete c;
      }
  };
#define FLOW(x)          \
  do {                   \
    rc = (x);            \
    if (rc) {            \
      cleanup();         \
      return rc;         \
    }                    \
  } while (0)
  FLOW(op_new(L, -1, &ETA));
  FLOW(op_new(L, -1, &G));
  FLOW(op_new(L, -1, &DG));
  FLOW(op_new(L, -1, &ETA0));
  FLOW(op_new(L, -1, &G0));
  FLOW(op_new(L, 1, &HS0));
  FLOW(op_new(L, 1, &INT1));
  FLOW(op_new(L, 1, &INT2));
  FLOW(op_new(L, 1, &AD));
  FLOW(op_new(L, 1, &w1));
  FLOW(op_new(L, 1, &w2));
  FLOW(cc_new(L, 1.0, &HCC));
  FLOW(cc_new(L, -1.0, &OCC));
  double s = 0.0, stp = (double)0.7f;  // "stp=.7" is a real(4) literal
  FLOW(qd_copy_arrays(HAM, HS));
  HS->herm = 1;
  auto eta_norm = [&](const qd_op* op, double* out) -> int {
    if (!(flags & QD_FULL_NORM)) return qd_mat_2_norm(op, out);
    TRY(reduce_norm_full(L, op->d, red_slot(L, 0)));
    return scalar_out(L, red_slot(L, 0), out);
  };
  FLOW(qd_build_white(ETA, HS));
  double nrm1, crit;
  FLOW(eta_norm(ETA, &nrm1));
  FLOW(qd_mbpt2(HAM, &crit));
  crit = std::fabs(crit);
  int iteration = 0, rows = 0, loops = 0, rejected = 0, comms = 0;
  while (crit > conv_criteria) {
    if (loops++ >= max_iter) {
      cleanup();
      if (result) {
        result->rows = rows;
        result->iterations = iteration;
        result->rejected = rejected;
        result->commutators = comms;
        result->s = s;
      }
      qd::set_error("qd_magnus_flow: not converged after %d steps (crit %.3e)", max_iter, crit);
      return QD_ERR_NOCONV;
    }
    FLOW(qd_copy_arrays(G, G0));
    FLOW(qd_magnus_expand(DG, G, ETA));
    FLOW(qd_euler_step(G, DG, &s, stp));
    FLOW(qd_copy_arrays(HS, HS0));
    int terms = 0;
    FLOW(qd_bch_expand(HS, G, HAM, INT1, INT2, AD, w1, w2, HCC, OCC, flags, &terms));
    comms += terms;
    FLOW(qd_copy_arrays(ETA, ETA0));
    FLOW(qd_build_white(ETA, HS));
    double nrm2;
    FLOW(eta_norm(ETA, &nrm2));
    double E0;
    QD_CUDA(cudaMemcpyAsync(L->h_red + 8, HS->d, sizeof(double), cudaMemcpyDeviceToHost, L->stream));
    QD_CUDA(cudaStreamSynchronize(L->stream));
    E0 = L->h_red[8];
    if (!std::isfinite(E0) || !std::isfinite(nrm2)) {
      cleanup();
      qd::set_error("qd_magnus_flow: non-finite energy or generator norm at step %d", loops);
      return QD_ERR_NAN;
    }
    if (trace && rows < max_iter) {
      double* t = trace + 7 * rows;
      t[0] = iteration; t[1] = s; t[2] = E0; t[3] = nrm1; t[4] = nrm2; t[5] = crit; t[6] = terms;
    }
    ++rows;
    if (nrm1 * 1.5 < nrm2) {
      if (trace && rows - 1 < max_iter) trace[7 * (rows - 1) + 6] = -terms;
      ++rejected;
      s = s - stp;
      FLOW(qd_copy_arrays(G0, G));
      FLOW(qd_copy_arrays(HS0, HS));
      FLOW(qd_copy_arrays(ETA0, ETA));
      stp = stp / 2.0 + (double)1e-3f;
      continue;
    }
    double mb;
    FLOW(qd_mbpt2(HS, &mb));
    crit = std::fabs(mb);
    iteration = iteration + 1;
  }
  double E0;
  QD_CUDA(cudaMemcpyAsync(L->h_red + 8, HS->d, sizeof(double), cudaMemcpyDeviceToHost, L->stream));
  QD_CUDA(cudaStreamSynchronize(L->stream));
  E0 = L->h_red[8];
  cleanup();
#undef FLOW
  if (result) {
    result->E0 = E0;
    result->s = s;
    result->iterations = iteration;
    result->rejected = rejected;
    result->commutators = comms;
    result->rows = rows;
  }
  return QD_OK;
}

}  // extern "C"
