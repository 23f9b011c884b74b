// api.cu -- extern "C" entry points (include/qd_imsrg.h).
//
// Host orchestration of the reference's call sequences on device-resident
// operators; every numeric step is a kernel on the layout's stream.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

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
  // Magnus flow: ETA, G, DG, ETA0, G0, HS0, INT1, INT2, AD, w1, w2 and HCC,
  // OCC, allocated by the first flow on the layout and kept
  qd_op* flow[11] = {nullptr};
  qd_cc* flow_cc[2] = {nullptr};
  qd_op* eta = nullptr;  // dGam's generator
  qd_op* eomq = nullptr;  // EOM matvec: excitation operator, second commutator
  qd_op* eomt = nullptr;
};
std::map<const qd_layout*, Workspace>& workspaces() {
  static std::map<const qd_layout*, Workspace> m;
  return m;
}
std::mutex g_ws_mutex;  // workspaces of different layouts from concurrent host threads

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
  ++L->children;
  QD_CUDA(cudaMemsetAsync(op->d, 0, sizeof(double) * L->neq, L->stream));
  op->zero_mask = ALL_PARTS;
  *out = op;
  return QD_OK;
}

// Tear down a layout's device state and the layout itself.
void layout_finish(qd_layout* L) {
  drop_merged_gemm(L);
  drop_merged_122(L);
  drop_122_plan(L);
  drop_eom_plans(L);
  layout_free_device(L);
  delete L;
}

// A layout destroyed while operators or cross-coupled matrices still refer
// to it (e.g. a garbage collector finalising the layout first) stays alive
// until the last of them is freed.
void release_child(qd_layout* L) {
  if (--L->children == 0 && L->closing) layout_finish(L);
}

void op_free(qd_op* op) {
  if (!op) return;
  qd_layout* L = op->L;
  if (op->d) cudaFree(op->d);
  delete op;
  release_child(L);
}

void cc_free(qd_cc* c) {
  if (!c) return;
  qd_layout* L = c->L;
  if (c->d) cudaFree(c->d);
  delete c;
  release_child(L);
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
  }
  ++L->children;
  if (c->d) QD_CUDA(cudaMemsetAsync(c->d, 0, sizeof(double) * L->xsize, L->stream));
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

// commutator_221 with the reference's visible intermediates w1, w2
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
    TRY(launch_pandya_tiles(L, L->d_z, C->d));
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
  {  // w1, w2 are workspaces of the whole commutator: the fused 221 leaves them untouched
    (void)w1;
    (void)w2;
    StageTimer tm(L, S_221);
    TRY(launch_221_fused(L, A, B, C->d));
  }
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
  std::lock_guard<std::mutex> lock(g_ws_mutex);
  Workspace& w = workspaces()[L];
  if (!w.w1) TRY(op_new(L, 1, &w.w1));
  if (!w.w2) TRY(op_new(L, 1, &w.w2));
  if (!w.ca) TRY(cc_new(L, -1.0, &w.ca));
  if (!w.cb) TRY(cc_new(L, 1.0, &w.cb));
  *out = &w;
  return QD_OK;
}

void drop_ws(const qd_layout* L) {
  Workspace w;
  {
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    auto& m = workspaces();
    auto it = m.find(L);
    if (it == m.end()) return;
    w = it->second;
    m.erase(it);
  }
  op_free(w.w1);
  op_free(w.w2);
  cc_free(w.ca);
  cc_free(w.cb);
  for (qd_op* o : w.flow) op_free(o);
  for (qd_cc* c : w.flow_cc) cc_free(c);
  op_free(w.eta);
  op_free(w.eomq);
  op_free(w.eomt);
}

}  // namespace

// A workspace operator of the layout that the full commutator never reads
// or writes (the reference's w1/w2, which the fused 221 replaces), for the
// autotuner's timed launches; NULL if none is allocated yet.
double* qd::scratch_operator(qd_layout* L) {
  std::lock_guard<std::mutex> lock(g_ws_mutex);
  auto it = workspaces().find(L);
  if (it == workspaces().end()) return nullptr;
  const Workspace& w = it->second;
  for (qd_op* o : {w.w1, w.w2, w.flow[9], w.flow[10]})
    if (o) return o->d;
  return nullptr;
}

namespace {

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
  if (L->children > 0)
    L->closing = true;  // the last operator or cc freed finishes the teardown
  else
    layout_finish(L);
  (void)cudaGetLastError();
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

int qd_layout_set_split(qd_layout* L, int slices) {
  CHECK(L, QD_ERR_ARG, "null layout");
  CHECK(slices >= 0 && slices <= 8, QD_ERR_ARG, "qd_layout_set_split: slices must be 0..8");
  L->split_slices = slices;
  return QD_OK;
}

int qd_layout_set_graphs(qd_layout* L, int enable) {
  CHECK(L, QD_ERR_ARG, "null layout");
  if (!enable && L->graphs) {
    TRY(use_device(L));
    QD_CUDA(cudaStreamSynchronize(L->stream));
    graphs_free(L);
  }
  L->use_graphs = enable != 0;
  return QD_OK;
}

int qd_layout_graph_stats(const qd_layout* L, int64_t* captured, int64_t* replays) {
  CHECK(L, QD_ERR_ARG, "null layout");
  if (captured) *captured = L->graphs_captured;
  if (replays) *replays = L->graph_replays;
  return QD_OK;
}

int qd_layout_get_split(const qd_layout* L, int* slices) {
  CHECK(L && slices, QD_ERR_ARG, "null argument");
  *slices = L->split_slices;
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

int qd_layout_tuning(const qd_layout* L, char* buf, int64_t len, int64_t* needed) {
  CHECK(L, QD_ERR_ARG, "null layout");
  const std::string r = tuning_report_122(L);
  if (needed) *needed = (int64_t)r.size() + 1;
  if (buf && len > 0) {
    const size_t n = std::min<size_t>((size_t)len - 1, r.size());
    std::memcpy(buf, r.data(), n);
    buf[n] = 0;
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
  (void)cudaGetLastError();  // teardown errors are not reported; do not leave them pending
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
  TRY(reduce_norm(L, r->d, red_slot(L, 0)));
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

// dGam (src/gs_IMSRG.f90:223-273): ETA = build_white(H) on a zeroed
// operator, HCC = calc_cc(H) (herm +1), ETACC = calc_cc(ETA) (herm -1),
// DER = [ETA, H] with every term: 110+220 into E0, 111, 121, 221, 122, 222
// with the particle-hole channel (the reference's order).
int qd_dgam(const qd_op* H, qd_op* DER, qd_cc* HCC, qd_cc* ETACC) {
  TRY(same_layout(H, DER));
  CHECK(H != DER, QD_ERR_ARG, "qd_dgam: DER aliases H");
  qd_layout* L = H->L;
  CHECK((!HCC || HCC->L == L) && (!ETACC || ETACC->L == L), QD_ERR_ARG, "qd_dgam: cross-coupled matrix of another layout");
  TRY(use_device(L));
  Workspace* w;
  TRY(get_ws(L, &w));
  if (!w->eta) TRY(op_new(L, -1, &w->eta));
  qd_op* eta = w->eta;
  eta->herm = -1;
  QD_CUDA(cudaMemsetAsync(eta->d, 0, sizeof(double) * L->neq, L->stream));
  eta->zero_mask = ALL_PARTS;
  TRY(qd_build_white(eta, H));
  TRY(commutator_seq(L, eta, H, DER, w->w1, w->w2, ETACC ? ETACC : w->ca, HCC ? HCC : w->cb, true));
  return QD_OK;
}

// EOM matrix-vector product (matvec_prod, src/EOM_IMSRG.f90:551-649, with
// HQ_comm_1b/2b, src/commutators.f90:1162-1272) for the scalar target
// (M_L, M_S) = (0, 0): the particle-hole and pphh parts of [H, Q] for the
// excitation operator Q (its fph and Vpphh).  The layout stores each
// operator with herm = +-1, so Q = (Q+ + Q-)/2, Q+- the same amplitudes as
// herm +-1 operators, and [H, Q] is the average of two full commutators with
// the particle-hole channel; every other part of HQ is zero.
int qd_eom_matvec(const qd_op* H, const qd_op* Q, qd_op* HQ) {
  TRY(same_layout(H, Q));
  TRY(same_layout(H, HQ));
  CHECK(HQ != H && HQ != Q, QD_ERR_ARG, "qd_eom_matvec: HQ aliases an input");
  qd_layout* L = H->L;
  TRY(use_device(L));
  Workspace* w;
  TRY(get_ws(L, &w));
  if (!w->eomq) TRY(op_new(L, 1, &w->eomq));
  if (!w->eomt) TRY(op_new(L, 1, &w->eomt));
  const unsigned exc = (1u << P_FPH) | (1u << P_PPHH);
  qd_op* X = w->eomq;
  QD_CUDA(cudaMemcpyAsync(X->d, Q->d, sizeof(double) * L->neq, cudaMemcpyDeviceToDevice, L->stream));
  TRY(launch_keep_parts(L, X->d, exc));
  X->zero_mask = (ALL_PARTS & ~exc) | (Q->zero_mask & exc);
  X->herm = 1;
  TRY(commutator_seq(L, H, X, HQ, w->w1, w->w2, w->cb, w->ca, true));
  X->herm = -1;
  TRY(commutator_seq(L, H, X, w->eomt, w->w1, w->w2, w->cb, w->ca, true));
  TRY(launch_axpy(L, HQ->d, 0.5, w->eomt->d, 0.5, HQ->d, L->neq));
  TRY(launch_keep_parts(L, HQ->d, exc));
  HQ->herm = 1;
  HQ->zero_mask = ALL_PARTS & ~exc;
  return QD_OK;
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
  cc_free(cc);
  (void)cudaGetLastError();
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
  const qd_layout* L = cc->L;
  TRY(use_device(L));
  if (L->xsize == 0) return QD_OK;
  // device rows are group-major; the host gets the reference's (i, j) row order
  std::vector<double> tmp((size_t)L->xsize);
  QD_CUDA(cudaMemcpyAsync(tmp.data(), cc->d, sizeof(double) * L->xsize, cudaMemcpyDeviceToHost, L->stream));
  QD_CUDA(cudaStreamSynchronize(L->stream));
  for (int q = 0; q < L->ncc; ++q) {
    const int r = L->ccdim[q].x, nb = L->ccdim[q].y, rb = L->ccab_base[q];
    const i64 xo = L->ccxoff[q];
    for (int c = 0; c < nb; ++c)
      for (int t = 0; t < r; ++t) host[xo + L->ccref[rb + t] + (i64)c * r] = tmp[xo + t + (i64)c * r];
  }
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

// ---- one BCH term, replayed as a CUDA graph --------------------------------
// A term is INT2 = [G, AD], HS += cof INT2 with |HS| and |INT2| into
// red_slot(1) and their copy to h_red[1..2].  Its launches depend only on the
// buffers, the zero-part masks, herm, the flags, the slice count and cof, so
// a term seen before on the same key is captured once (thread-local capture
// mode, after an eager run has built every plan and workspace) and replayed
// with one cudaGraphLaunch.  A capture that fails leaves the key eager.
namespace {
struct TermKey {
  const void* p[8];  // G, AD, INT2, HS, w1, w2, OCC, HCC data
  unsigned mg, mad, mhs;
  int gh, term, flags, split;
  bool operator<(const TermKey& o) const { return std::memcmp(this, &o, sizeof(TermKey)) < 0; }
};
struct TermGraph {
  int seen = 0;
  bool failed = false;
  cudaGraphExec_t exec = nullptr;
  long long launches = 0;
};
using TermGraphs = std::map<TermKey, TermGraph>;

int bch_term(qd_layout* L, const qd_op* G, qd_op* AD, qd_op* INT2, qd_op* HS, qd_op* w1, qd_op* w2, qd_cc* HCC,
             qd_cc* OCC, bool pandya, double cof, const int* kidx = nullptr) {
  if (pandya) {
    TRY(commutator_seq(L, G, AD, INT2, w1, w2, OCC, HCC, true));
  } else {
    TRY(commutator_seq(L, G, AD, INT2, w1, w2, nullptr, nullptr, false));
  }
  {
    StageTimer tm(L, S_GLUE);
    TRY(launch_axpy_norms(L, HS->d, 1.0, INT2->d, cof, HS->d, red_slot(L, 1), kidx));
  }
  if (!kidx)  // host decides: copy both norms back
    QD_CUDA(cudaMemcpyAsync(L->h_red + 1, red_slot(L, 1), 2 * sizeof(double), cudaMemcpyDeviceToHost, L->stream));
  return QD_OK;
}
}  // namespace

static int bch_term_graph(qd_layout* L, const qd_op* G, qd_op* AD, qd_op* INT2, qd_op* HS, qd_op* w1, qd_op* w2,
                          qd_cc* HCC, qd_cc* OCC, bool pandya, int term, double cof) {
  if (!L->use_graphs || L->prof.on) return bch_term(L, G, AD, INT2, HS, w1, w2, HCC, OCC, pandya, cof);
  if (!L->graphs) L->graphs = new TermGraphs();
  TermKey k;
  std::memset(&k, 0, sizeof(k));
  k.p[0] = G->d;
  k.p[1] = AD->d;
  k.p[2] = INT2->d;
  k.p[3] = HS->d;
  k.p[4] = w1->d;
  k.p[5] = w2->d;
  k.p[6] = OCC ? OCC->d : nullptr;
  k.p[7] = HCC ? HCC->d : nullptr;
  k.mg = G->zero_mask;
  k.mad = AD->zero_mask;
  k.mhs = HS->zero_mask;
  k.gh = G->herm;
  k.term = term;
  k.flags = pandya ? 1 : 0;
  k.split = L->split_slices;
  TermGraph& tg = (*reinterpret_cast<TermGraphs*>(L->graphs))[k];
  if (tg.exec) {
    QD_CUDA(cudaGraphLaunch(tg.exec, L->stream));
    L->nlaunch += tg.launches;
    ++L->graph_replays;
    INT2->zero_mask = 0;  // what the captured commutator_seq leaves on the host side
    if (pandya) {
      OCC->filled = true;
      OCC->herm = G->herm;
      HCC->filled = true;
      HCC->herm = AD->herm;
    }
    return QD_OK;
  }
  if (tg.failed || tg.seen == 0) {
    ++tg.seen;
    return bch_term(L, G, AD, INT2, HS, w1, w2, HCC, OCC, pandya, cof);
  }
  // second sight: capture, instantiate, launch
  const long long n0 = L->nlaunch;
  cudaGraph_t graph = nullptr;
  int rc = QD_OK;
  cudaError_t e = cudaStreamBeginCapture(L->stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    rc = bch_term(L, G, AD, INT2, HS, w1, w2, HCC, OCC, pandya, cof);
    e = cudaStreamEndCapture(L->stream, &graph);
  }
  if (e == cudaSuccess && rc == QD_OK && graph) e = cudaGraphInstantiate(&tg.exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess || rc != QD_OK || !tg.exec) {
    (void)cudaGetLastError();
    if (tg.exec) cudaGraphExecDestroy(tg.exec);
    tg.exec = nullptr;
    tg.failed = true;
    L->nlaunch = n0;
    return bch_term(L, G, AD, INT2, HS, w1, w2, HCC, OCC, pandya, cof);
  }
  tg.launches = L->nlaunch - n0;
  ++L->graphs_captured;
  QD_CUDA(cudaGraphLaunch(tg.exec, L->stream));
  return QD_OK;
}

}  // extern "C"

namespace {
// ---- a whole BCH_EXPAND as one CUDA graph --------------------------------
// The exit test runs on the device (k_bch_decide), so the term loop is a
// graph "while" node and a BCH step needs one host synchronisation (for the
// term count) instead of one per term.  Layout of the graph:
//   prologue: HS = H; AD = H; INT2 = [G, AD]; HS += cof(1) INT2; decide
//   while (go): INT2' = [G, INT2]; HS += cof INT2'; decide (sets go, more)
//               if (more): INT2 = [G, INT2']; HS += cof INT2; decide (sets go)
// The two buffers of INT2 and AD alternate between the two halves of the
// loop body, so no operator is copied.  The term coefficient comes from a
// device counter (the number of terms so far), which the host reads back.
// Built like the per-term graphs: a key seen once runs eagerly (which builds
// every plan and workspace), the second time it is captured; a capture that
// fails leaves the key eager.
struct StepKey {
  const void* p[9];  // G, HS, H, INT2, AD, w1, w2, OCC, HCC data
  unsigned mg, mh;
  int gh, hh, flags, split;
  bool operator<(const StepKey& o) const { return std::memcmp(this, &o, sizeof(StepKey)) < 0; }
};
struct StepGraph {
  int seen = 0;
  bool failed = false;
  cudaGraphExec_t exec = nullptr;
  long long first = 0, per_term = 0;  // launches of the prologue and of one later term
};
using StepGraphs = std::map<StepKey, StepGraph>;

int* bch_counter(qd_layout* L) { return reinterpret_cast<int*>(red_slot(L, 16)); }

// A conditional node of `type` on handle h after the current dependencies of
// a stream capturing into graph g; *body receives its body graph.
int add_conditional(cudaStream_t st, cudaGraph_t g, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                    cudaGraph_t* body) {
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  QD_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &nd));
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};  // aggregate: the rest zero
  cp.conditional.handle = h;
  cp.conditional.type = type;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  QD_CUDA(cudaGraphAddNode(&node, g, deps, nd, &cp));
  QD_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
  *body = cp.conditional.phGraph_out[0];
  return QD_OK;
}

// Capture the step graph: P (INT2's buffer) and Q (AD's buffer) alternate.
int capture_step(qd_layout* L, qd_op* HS, const qd_op* G, const qd_op* H, double* P, double* Q, qd_op* w1,
                 qd_op* w2, qd_cc* HCC, qd_cc* OCC, bool pandya, cudaGraphExec_t* exec, long long* first,
                 long long* per_term) {
  const double conv = (double)1e-5f;
  int* k = bch_counter(L);
  cudaStream_t st = L->stream;
  qd_op ad = *H, out = *H;  // host views of the two buffers (herm +1, as BCH_EXPAND sets)
  ad.herm = out.herm = 1;
  cudaGraph_t g = nullptr;
  QD_CUDA(cudaGraphCreate(&g, 0));
  int rc = QD_OK;
  cudaGraph_t body = nullptr, body2 = nullptr, cap = nullptr;
  cudaGraphConditionalHandle hloop, hmore;
  const long long n0 = L->nlaunch;
  do {
    if (cudaGraphConditionalHandleCreate(&hloop, g, 0, 0) != cudaSuccess) { rc = QD_ERR_CUDA; break; }
    if (cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      rc = QD_ERR_CUDA;
      break;
    }
    // prologue: HS = H, AD = H (Q), term 1 into P
    int r2 = QD_OK;
    if (cudaMemsetAsync(k, 0, sizeof(int), st) != cudaSuccess ||
        cudaMemcpyAsync(HS->d, H->d, sizeof(double) * L->neq, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(Q, H->d, sizeof(double) * L->neq, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      r2 = QD_ERR_CUDA;
    ad.d = Q;
    ad.zero_mask = H->zero_mask;
    out.d = P;
    HS->zero_mask = H->zero_mask;
    if (!r2) r2 = bch_term(L, G, &ad, &out, HS, w1, w2, HCC, OCC, pandya, 0.0, k);
    if (!r2) r2 = launch_bch_decide(L, red_slot(L, 1), k, conv, hloop, hloop, 0);
    *first = L->nlaunch - n0;
    if (!r2) r2 = add_conditional(st, g, hloop, cudaGraphCondTypeWhile, &body);
    if (cudaStreamEndCapture(st, &cap) != cudaSuccess || r2) {
      rc = r2 ? r2 : QD_ERR_CUDA;
      break;
    }
    // loop body, first half: AD = P, INT2 = Q; then "more" guards the second half
    if (cudaGraphConditionalHandleCreate(&hmore, body, 0, 0) != cudaSuccess ||
        cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      rc = QD_ERR_CUDA;
      break;
    }
    const long long n1 = L->nlaunch;
    ad.d = P;
    ad.zero_mask = 0;
    out.d = Q;
    r2 = bch_term(L, G, &ad, &out, HS, w1, w2, HCC, OCC, pandya, 0.0, k);
    if (!r2) r2 = launch_bch_decide(L, red_slot(L, 1), k, conv, hloop, hmore, 1);
    *per_term = L->nlaunch - n1;
    if (!r2) r2 = add_conditional(st, body, hmore, cudaGraphCondTypeIf, &body2);
    if (cudaStreamEndCapture(st, &cap) != cudaSuccess || r2) {
      rc = r2 ? r2 : QD_ERR_CUDA;
      break;
    }
    // second half: AD = Q, INT2 = P
    if (cudaStreamBeginCaptureToGraph(st, body2, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess) {
      rc = QD_ERR_CUDA;
      break;
    }
    ad.d = Q;
    out.d = P;
    r2 = bch_term(L, G, &ad, &out, HS, w1, w2, HCC, OCC, pandya, 0.0, k);
    if (!r2) r2 = launch_bch_decide(L, red_slot(L, 1), k, conv, hloop, hloop, 0);
    if (cudaStreamEndCapture(st, &cap) != cudaSuccess || r2) {
      rc = r2 ? r2 : QD_ERR_CUDA;
      break;
    }
    if (cudaGraphInstantiate(exec, g, 0) != cudaSuccess) rc = QD_ERR_CUDA;
  } while (false);
  if (rc) {  // leave no capture open and no error pending
    cudaStreamCaptureStatus cs;
    if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(st, &junk);
      if (junk) cudaGraphDestroy(junk);
    }
    (void)cudaGetLastError();
    *exec = nullptr;
  }
  cudaGraphDestroy(g);
  L->nlaunch = n0;
  return rc;
}

// The eager BCH_EXPAND loop (per-term graphs where enabled).
int bch_eager(qd_layout* L, qd_op* HS, const qd_op* G, const qd_op* H, qd_op* INT2, qd_op* AD, qd_op* w1, qd_op* w2,
              qd_cc* HCC, qd_cc* OCC, bool pandya, int* nterms);

// Whole step as a graph when possible; *done = false leaves it to the caller.
int bch_step_graph(qd_layout* L, qd_op* HS, const qd_op* G, const qd_op* H, qd_op* INT2, qd_op* AD, qd_op* w1,
                   qd_op* w2, qd_cc* HCC, qd_cc* OCC, bool pandya, int* nterms, bool* done) {
  *done = false;
  if (!L->use_graphs || L->prof.on || L->split_slices > 0) return QD_OK;
  if (!L->step_graphs) L->step_graphs = new StepGraphs();
  StepKey key;
  std::memset(&key, 0, sizeof(key));
  const void* ptrs[9] = {G->d, HS->d, H->d, INT2->d, AD->d, w1->d, w2->d, OCC ? OCC->d : nullptr,
                         HCC ? HCC->d : nullptr};
  for (int i = 0; i < 9; ++i) key.p[i] = ptrs[i];
  key.mg = G->zero_mask;
  key.mh = H->zero_mask;
  key.gh = G->herm;
  key.hh = H->herm;
  key.flags = pandya ? 1 : 0;
  key.split = L->split_slices;
  StepGraph& sg = (*reinterpret_cast<StepGraphs*>(L->step_graphs))[key];
  double* P = INT2->d;
  double* Q = AD->d;
  if (!sg.exec) {
    if (sg.failed || sg.seen++ == 0) return QD_OK;  // eager (first sight builds plans for H's masks)
    // plans and task lists of the later terms ([G, X] with X a full operator)
    qd_op full = *H;  // H as a full operator: the masks of AD in the later terms
    full.zero_mask = 0;
    TRY(prepare_program(L, L->prog_ladder, G->zero_mask, 0u));
    TRY(prepare_program(L, L->prog_111, G->zero_mask, 0u));
    TRY(prepare_program(L, L->prog_pandya, 0u, 0u));
    TRY(prepare_122(L, G, &full));
    TRY(prepare_program(L, L->prog_ladder, G->zero_mask, H->zero_mask));
    TRY(prepare_program(L, L->prog_111, G->zero_mask, H->zero_mask));
    TRY(prepare_122(L, G, H));
    if (pandya) TRY(ensure_z(L));
    QD_CUDA(cudaStreamSynchronize(L->stream));
    if (capture_step(L, HS, G, H, P, Q, w1, w2, HCC, OCC, pandya, &sg.exec, &sg.first, &sg.per_term)) {
      sg.failed = true;
      return QD_OK;
    }
    ++L->graphs_captured;
  }
  QD_CUDA(cudaGraphLaunch(sg.exec, L->stream));
  int* hk = reinterpret_cast<int*>(L->h_red + 16);
  QD_CUDA(cudaMemcpyAsync(hk, bch_counter(L), sizeof(int), cudaMemcpyDeviceToHost, L->stream));
  QD_CUDA(cudaStreamSynchronize(L->stream));
  const int terms = *hk;
  L->nlaunch += sg.first + sg.per_term * (terms - 1);
  ++L->graph_replays;
  // host-side state the eager loop leaves: HS and the workspaces hold full
  // operators; the two workspace buffers keep their handles
  HS->zero_mask = 0;
  INT2->zero_mask = 0;
  AD->zero_mask = 0;
  if (pandya) {
    OCC->filled = true;
    OCC->herm = G->herm;
    HCC->filled = true;
    HCC->herm = 1;
  }
  *nterms = terms;
  *done = true;
  return QD_OK;
}

}  // namespace

extern "C" {

int qd_bch_expand(qd_op* HS, const qd_op* G, const qd_op* H, qd_op* INT1, qd_op* INT2, qd_op* AD, qd_op* w1,
                  qd_op* w2, qd_cc* HCC, qd_cc* OCC, unsigned flags, int* nterms) {
  TRY(same_layout(HS, G));
  TRY(same_layout(HS, H));
  TRY(same_layout(HS, INT2));
  TRY(same_layout(HS, AD));
  TRY(same_layout(HS, w1));
  TRY(same_layout(HS, w2));
  (void)INT1;  // not written: the norm of INT1 (= HS before the update) is taken from HS itself
  qd_layout* L = HS->L;
  TRY(use_device(L));
  TRY(build_programs(L));
  const bool pandya = (flags & QD_PANDYA) != 0;
  CHECK(!pandya || (HCC && OCC), QD_ERR_ARG, "qd_bch_expand: QD_PANDYA needs HCC and OCC");
  INT2->herm = 1;
  AD->herm = 1;
  bool done = false;
  int count = 0;
  TRY(bch_step_graph(L, HS, G, H, INT2, AD, w1, w2, HCC, OCC, pandya, &count, &done));
  if (!done) TRY(bch_eager(L, HS, G, H, INT2, AD, w1, w2, HCC, OCC, pandya, &count));
  if (nterms) *nterms = count;
  return QD_OK;
}

}  // extern "C"

namespace {
int bch_eager(qd_layout* L, qd_op* HS, const qd_op* G, const qd_op* H, qd_op* INT2, qd_op* AD, qd_op* w1, qd_op* w2,
              qd_cc* HCC, qd_cc* OCC, bool pandya, int* nterms) {
  const double conv = (double)1e-5f;  // "conv = 1e-5" is a real(4) literal in the reference
  double* const p0 = INT2->d;
  TRY(qd_copy_arrays(H, HS));
  TRY(qd_copy_arrays(HS, INT2));
  int count = 0;
  for (int i = 2; i <= 12; ++i) {
    std::swap(INT2->d, AD->d);  // AD = previous term; INT2 becomes the output buffer
    std::swap(INT2->zero_mask, AD->zero_mask);
    const double cof = kCof[i - 2];
    TRY(bch_term_graph(L, G, AD, INT2, HS, w1, w2, HCC, OCC, pandya, i, cof));
    ++count;
    HS->zero_mask &= INT2->zero_mask;
    QD_CUDA(cudaStreamSynchronize(L->stream));
    const double n1 = L->h_red[1], n2 = L->h_red[2];
    if (n2 * cof / n1 < conv) break;
  }
  if (INT2->d != p0) {  // the workspaces keep their buffers (contents unspecified)
    std::swap(INT2->d, AD->d);
    std::swap(INT2->zero_mask, AD->zero_mask);
  }
  if (nterms) *nterms = count;
  return QD_OK;
}
}  // namespace

extern "C" {

int qd_magnus_expand(qd_op* DG, const qd_op* G, const qd_op* ETA) {
  (void)G;
  return qd_copy_arrays(ETA, DG);
}

int qd_euler_step(qd_op* G, const qd_op* DG, double* s, double stp) {
  TRY(qd_add_arrays(G, 1.0, DG, stp, G));
  if (s) *s = *s + stp;
  return QD_OK;
}

}  // extern "C"

// ---- the Magnus flow as a stepping object (s_evolve, magnus_IMSRG.f90:194-248)
struct qd_flow {
  qd_layout* L = nullptr;
  const qd_op* HAM = nullptr;
  qd_op* HS = nullptr;
  double* hs_home = nullptr;  // the caller's HS buffer (HS and HS0 trade buffers during the flow)
  unsigned flags = 0;
  qd_op *ETA = nullptr, *G = nullptr, *DG = nullptr, *ETA0 = nullptr, *G0 = nullptr, *HS0 = nullptr;
  qd_op *INT1 = nullptr, *INT2 = nullptr, *AD = nullptr, *w1 = nullptr, *w2 = nullptr;
  qd_cc *HCC = nullptr, *OCC = nullptr;
  double s = 0.0, stp = (double)0.7f;  // "stp=.7" is a real(4) literal
  double nrm1 = 0.0, crit = 0.0, E0 = 0.0;
  int iteration = 0, rejected = 0, comms = 0, rows = 0;
};

namespace {
const double kConvCriteria = (double)1e-9f;  // real(4) literal in the reference

int flow_eta_norm(qd_flow* f, const qd_op* op, double* out) { return qd_mat_2_norm(op, out); }

// Operators of one role pair (G/G0, HS/HS0, ETA/ETA0) trade buffers instead
// of copying: "G0 = G" becomes a swap after which G's buffer is rewritten.
void swap_ops(qd_op* a, qd_op* b) {
  std::swap(a->d, b->d);
  std::swap(a->zero_mask, b->zero_mask);
}

// Give the caller's HS its own buffer back (copying the current contents).
int flow_home_hs(qd_flow* f) {
  if (f->HS->d == f->hs_home) return QD_OK;
  QD_CUDA(cudaMemcpyAsync(f->hs_home, f->HS->d, sizeof(double) * f->L->neq, cudaMemcpyDeviceToDevice, f->L->stream));
  swap_ops(f->HS, f->HS0);  // HS0 held hs_home: after the swap HS->d == hs_home again
  f->HS0->zero_mask = f->HS->zero_mask;
  return QD_OK;
}

int flow_e0(qd_flow* f, double* e0) {
  qd_layout* L = f->L;
  QD_CUDA(cudaMemcpyAsync(L->h_red + 8, f->HS->d, sizeof(double), cudaMemcpyDeviceToHost, L->stream));
  QD_CUDA(cudaStreamSynchronize(L->stream));
  *e0 = L->h_red[8];
  return QD_OK;
}
}  // namespace

extern "C" {

int qd_flow_create(const qd_op* HAM, qd_op* HS, unsigned flags, qd_flow** out) {
  CHECK(out, QD_ERR_ARG, "qd_flow_create: null output");
  *out = nullptr;
  TRY(same_layout(HAM, HS));
  CHECK(HAM != HS, QD_ERR_ARG, "qd_flow_create: HS must not alias HAM");
  qd_layout* L = HAM->L;
  TRY(use_device(L));
  // workspaces: allocated by the first flow on this layout and kept (they
  // hold 11 operators; freeing them per flow would cost a device sync each)
  Workspace* ws;
  {
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    ws = &workspaces()[L];
  }
  const int fherm[11] = {-1, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1};
  for (int k = 0; k < 11; ++k)
    if (!ws->flow[k]) TRY(op_new(L, fherm[k], &ws->flow[k]));
  if (!ws->flow_cc[0]) TRY(cc_new(L, 1.0, &ws->flow_cc[0]));
  if (!ws->flow_cc[1]) TRY(cc_new(L, -1.0, &ws->flow_cc[1]));
  qd_flow* f = new qd_flow();
  f->L = L;
  f->HAM = HAM;
  f->HS = HS;
  f->flags = flags;
  qd_op** o = ws->flow;
  f->ETA = o[0]; f->G = o[1]; f->DG = o[2]; f->ETA0 = o[3]; f->G0 = o[4]; f->HS0 = o[5];
  f->INT1 = o[6]; f->INT2 = o[7]; f->AD = o[8]; f->w1 = o[9]; f->w2 = o[10];
  f->HCC = ws->flow_cc[0];
  f->OCC = ws->flow_cc[1];
  for (int k = 0; k < 11; ++k) o[k]->herm = fherm[k];
  f->HCC->herm = 1.0;
  f->OCC->herm = -1.0;
  f->HCC->filled = f->OCC->filled = false;  // run_magnus never fills them (the Pandya option does, per commutator)
  f->hs_home = HS->d;
  int rc = QD_OK;
  // the generator and the Magnus operator start from zero (allocate_everything);
  // ETA0 too, as ETA and ETA0 trade buffers and build_white writes only fph
  // and Vpphh
  for (qd_op* z : {f->ETA, f->ETA0, f->G}) {
    if (cudaMemsetAsync(z->d, 0, sizeof(double) * L->neq, L->stream) != cudaSuccess) rc = QD_ERR_CUDA;
    z->zero_mask = ALL_PARTS;
  }
  if (!rc) rc = qd_copy_arrays(HAM, HS);
  HS->herm = 1;
  if (!rc) rc = qd_build_white(f->ETA, HS);
  if (!rc) rc = flow_eta_norm(f, f->ETA, &f->nrm1);
  if (!rc) rc = qd_mbpt2(HAM, &f->crit);
  if (!rc) rc = flow_e0(f, &f->E0);
  if (rc) {
    delete f;
    return rc;
  }
  f->crit = std::fabs(f->crit);
  *out = f;
  return QD_OK;
}

int qd_flow_warm_start(qd_flow* f, const qd_op* G, double s) {
  CHECK(f && G, QD_ERR_ARG, "qd_flow_warm_start: null argument");
  CHECK(G->L == f->L, QD_ERR_ARG, "qd_flow_warm_start: Omega on another layout");
  CHECK(G != f->G, QD_ERR_ARG, "qd_flow_warm_start: pass a copy of the flow's own Omega");
  TRY(use_device(f->L));
  TRY(qd_copy_arrays(G, f->G));
  f->G->herm = -1;
  f->s = s;
  int terms = 0;
  TRY(qd_bch_expand(f->HS, f->G, f->HAM, f->INT1, f->INT2, f->AD, f->w1, f->w2, f->HCC, f->OCC, f->flags, &terms));
  f->comms += terms;
  TRY(qd_build_white(f->ETA, f->HS));
  double mb;
  TRY(qd_mbpt2(f->HS, &mb));
  f->crit = std::fabs(mb);
  TRY(flow_e0(f, &f->E0));
  CHECK(std::isfinite(f->E0) && std::isfinite(f->crit), QD_ERR_NAN, "qd_flow_warm_start: non-finite state");
  return QD_OK;
}

}  // extern "C"

namespace {
// s_evolve's loop body in two halves around BCH_EXPAND (the batched flows run
// the BCH of several instances between them).  flow_begin returns
// *converged = true (and fills info) when there is nothing to do.
int flow_begin(qd_flow* f, qd_flow_step_info* inf, bool* converged) {
  std::memset(inf, 0, sizeof(*inf));
  *converged = f->crit <= kConvCriteria;
  if (*converged) {
    inf->s = f->s;
    inf->E0 = f->E0;
    inf->nrm1 = f->nrm1;
    inf->crit = f->crit;
    inf->converged = 1;
    return QD_OK;
  }
  // G0 = G; MAGNUS_EXPAND: DG = ETA; euler_step: G = G + stp DG.  G and G0
  // trade buffers and G = 1 G0 + stp ETA is written in one pass (the same
  // arithmetic as add_arrays(G, 1, DG, stp, G) with DG = ETA).
  swap_ops(f->G, f->G0);
  TRY(qd_add_arrays(f->G0, 1.0, f->ETA, f->stp, f->G));
  f->s = f->s + f->stp;
  swap_ops(f->HS, f->HS0);  // HS0 = HS: BCH_EXPAND rewrites every entry of HS
  return QD_OK;
}

int flow_end(qd_flow* f, int terms, qd_flow_step_info* inf) {
  f->comms += terms;
  swap_ops(f->ETA, f->ETA0);  // ETA0 = ETA: build_white rewrites fph and Vpphh, the rest stays 0
  TRY(qd_build_white(f->ETA, f->HS));
  double nrm2, E0;
  TRY(flow_eta_norm(f, f->ETA, &nrm2));
  TRY(flow_e0(f, &E0));
  CHECK(std::isfinite(E0) && std::isfinite(nrm2), QD_ERR_NAN,
        "qd_flow_step: non-finite energy or generator norm at s = %g", f->s);
  inf->s = f->s;
  inf->E0 = E0;
  inf->nrm1 = f->nrm1;
  inf->nrm2 = nrm2;
  inf->crit = f->crit;  // the criterion before this step, as the reference's trace
  inf->terms = terms;
  ++f->rows;
  if (f->nrm1 * 1.5 < nrm2) {  // reject: back to the previous state, smaller step
    ++f->rejected;
    f->s = f->s - f->stp;
    swap_ops(f->G, f->G0);
    swap_ops(f->HS, f->HS0);
    swap_ops(f->ETA, f->ETA0);
    f->stp = f->stp / 2.0 + (double)1e-3f;
    inf->accepted = 0;
  } else {
    double mb;
    TRY(qd_mbpt2(f->HS, &mb));
    f->crit = std::fabs(mb);
    f->E0 = E0;
    f->iteration += 1;
    inf->accepted = 1;
  }
  inf->converged = f->crit <= kConvCriteria ? 1 : 0;
  return QD_OK;
}
}  // namespace

extern "C" {

int qd_flow_step(qd_flow* f, qd_flow_step_info* info) {
  CHECK(f, QD_ERR_ARG, "qd_flow_step: null flow");
  TRY(use_device(f->L));
  qd_flow_step_info inf;
  bool conv = false;
  TRY(flow_begin(f, &inf, &conv));
  if (!conv) {
    int terms = 0;
    TRY(qd_bch_expand(f->HS, f->G, f->HAM, f->INT1, f->INT2, f->AD, f->w1, f->w2, f->HCC, f->OCC, f->flags,
                      &terms));
    TRY(flow_end(f, terms, &inf));
  }
  if (info) *info = inf;
  return QD_OK;
}

int qd_flow_omega(const qd_flow* f, qd_op** G) {
  CHECK(f && G, QD_ERR_ARG, "qd_flow_omega: null argument");
  *G = f->G;
  return QD_OK;
}

int qd_flow_state(const qd_flow* f, qd_flow_result* r) {
  CHECK(f && r, QD_ERR_ARG, "qd_flow_state: null argument");
  r->E0 = f->E0;
  r->s = f->s;
  r->iterations = f->iteration;
  r->rejected = f->rejected;
  r->commutators = f->comms;
  r->rows = f->rows;
  return QD_OK;
}

int qd_flow_destroy(qd_flow* f) {
  if (!f) return QD_OK;
  cudaSetDevice(f->L->device);
  flow_home_hs(f);
  cudaStreamSynchronize(f->L->stream);
  (void)cudaGetLastError();
  delete f;  // the workspaces stay with the layout
  return QD_OK;
}

int qd_magnus_flow(const qd_op* HAM, qd_op* HS, unsigned flags, int max_iter, double* trace,
                   qd_flow_result* result) {
  qd_flow* f = nullptr;
  TRY(qd_flow_create(HAM, HS, flags, &f));
  int rc = QD_OK, loops = 0;
  while (f->crit > kConvCriteria) {
    if (loops++ >= max_iter) {
      qd::set_error("qd_magnus_flow: not converged after %d steps (crit %.3e)", max_iter, f->crit);
      rc = QD_ERR_NOCONV;
      break;
    }
    qd_flow_step_info inf;
    if ((rc = qd_flow_step(f, &inf))) break;
    const int row = f->rows - 1;
    if (trace && row < max_iter) {
      double* t = trace + 7 * row;
      t[0] = f->iteration - inf.accepted; t[1] = inf.s; t[2] = inf.E0; t[3] = inf.nrm1; t[4] = inf.nrm2;
      t[5] = inf.crit; t[6] = inf.accepted ? inf.terms : -inf.terms;
    }
  }
  if (result) qd_flow_state(f, result);
  std::string msg = rc ? qd::last_error() : std::string();
  qd_flow_destroy(f);
  if (rc) qd::set_error("%s", msg.c_str());
  return rc;
}

}  // extern "C"

namespace {
// ---- batched flows: several instances in lockstep, one launch per stage ---
// One commutator C = [A, B] per item, every item's layout on the same stream:
// the small stages (E0, 111, 121, 221, Pandya re-coupling) per item, the
// 122 tiles and the ladder GEMM tasks of all items in one launch each.
struct CommItem {
  qd_layout* L;
  const qd_op *A, *B;
  qd_op* C;
  qd_cc *ACC, *BCC;
};

// Streams of a lockstep batch: each instance's small stages run on its own
// layout's stream; the merged launches run on `st` after a join (events) and
// the instances' streams wait for them before going on.
struct BatchCtx {
  cudaStream_t st = nullptr;
  cudaEvent_t ev_st = nullptr;
  std::map<const qd_layout*, cudaEvent_t> ev;
};

int join_to(cudaStream_t st, const std::vector<qd_layout*>& Ls, BatchCtx& bc) {
  for (qd_layout* L : Ls) {
    cudaEvent_t e = bc.ev[L];
    QD_CUDA(cudaEventRecord(e, L->stream));
    QD_CUDA(cudaStreamWaitEvent(st, e, 0));
  }
  return QD_OK;
}

int fork_from(cudaStream_t st, const std::vector<qd_layout*>& Ls, BatchCtx& bc) {
  QD_CUDA(cudaEventRecord(bc.ev_st, st));
  for (qd_layout* L : Ls) QD_CUDA(cudaStreamWaitEvent(L->stream, bc.ev_st, 0));
  return QD_OK;
}

int commutator_batch(BatchCtx& bc, std::vector<CommItem>& items, bool pandya) {
  std::vector<Item122> i122;
  std::vector<GemmItem> gl;
  std::vector<qd_layout*> Ls;
  for (CommItem& it : items) {
    qd_layout* L = it.L;
    Ls.push_back(L);
    TRY(build_programs(L));
    TRY(stage_e0(L, it.A, it.B, it.C->d, 0.0));
    TRY(stage_111(L, it.A, it.B, it.C));
    TRY(launch_121(L, it.A, it.B, it.C->d));
    TRY(launch_221_fused(L, it.A, it.B, it.C->d));
    if (pandya) {
      TRY(launch_calc_cc(L, it.A, it.ACC->d));
      it.ACC->filled = true;
      it.ACC->herm = it.A->herm;
      TRY(launch_calc_cc(L, it.B, it.BCC->d));
      it.BCC->filled = true;
      it.BCC->herm = it.B->herm;
    }
    i122.push_back(Item122{L, it.A, it.B, it.C->d});
    GemmItem g;
    g.L = L;
    g.P = &L->prog_ladder;
    const double* bufs[NBUF] = {it.A->d, it.B->d, nullptr, nullptr, it.C->d, nullptr, nullptr};
    for (int k = 0; k < NBUF; ++k) g.bufs[k] = bufs[k];
    g.hv0 = (double)it.A->herm;
    g.hv1 = (double)it.B->herm;
    g.maskA = it.A->zero_mask;
    g.maskB = it.B->zero_mask;
    gl.push_back(g);
  }
  TRY(join_to(bc.st, Ls, bc));
  TRY(launch_122_batched(bc.st, i122));
  TRY(run_programs_batched(bc.st, gl));
  TRY(fork_from(bc.st, Ls, bc));
  for (CommItem& it : items) {
    qd_layout* L = it.L;
    if (pandya && L->zsize > 0) {  // the particle-hole channel, as stage_222 after its ladders
      TRY(ensure_z(L));
      const double* zb[7] = {nullptr, nullptr, it.ACC->d, it.BCC->d, nullptr, nullptr, L->d_z};
      TRY(run_program(L, L->prog_pandya, zb, it.ACC->herm, it.BCC->herm, 0u, 0u));
      TRY(launch_pandya_tiles(L, L->d_z, it.C->d));
    }
    it.C->zero_mask = 0;
  }
  return QD_OK;
}

// BCH_EXPAND of several flows in lockstep: every term is one batched
// commutator over the instances whose series is still running; the host
// reads all norms once per term and applies each instance's exit test.
int bch_batch(BatchCtx& bc, const std::vector<qd_flow*>& fl, std::vector<int>& terms) {
  const double conv = (double)1e-5f;
  const bool pandya = fl.empty() ? false : (fl[0]->flags & QD_PANDYA) != 0;
  std::vector<double*> p0(fl.size());
  std::vector<int> live;
  for (size_t j = 0; j < fl.size(); ++j) {
    qd_flow* f = fl[j];
    f->INT2->herm = 1;
    f->AD->herm = 1;
    TRY(qd_copy_arrays(f->HAM, f->HS));
    TRY(qd_copy_arrays(f->HS, f->INT2));
    p0[j] = f->INT2->d;
    terms[j] = 0;
    live.push_back((int)j);
  }
  for (int i = 2; i <= 12 && !live.empty(); ++i) {
    const double cof = kCof[i - 2];
    std::vector<CommItem> items;
    for (int j : live) {
      qd_flow* f = fl[j];
      std::swap(f->INT2->d, f->AD->d);
      std::swap(f->INT2->zero_mask, f->AD->zero_mask);
      items.push_back(CommItem{f->L, f->G, f->AD, f->INT2, f->OCC, f->HCC});
    }
    TRY(commutator_batch(bc, items, pandya));
    for (int j : live) {
      qd_flow* f = fl[j];
      qd_layout* L = f->L;
      TRY(launch_axpy_norms(L, f->HS->d, 1.0, f->INT2->d, cof, f->HS->d, red_slot(L, 1)));
      QD_CUDA(cudaMemcpyAsync(L->h_red + 1, red_slot(L, 1), 2 * sizeof(double), cudaMemcpyDeviceToHost,
                              L->stream));
      f->HS->zero_mask &= f->INT2->zero_mask;
      ++terms[j];
    }
    for (int j : live) QD_CUDA(cudaStreamSynchronize(fl[j]->L->stream));
    std::vector<int> next;
    for (int j : live) {
      const double n1 = fl[j]->L->h_red[1], n2 = fl[j]->L->h_red[2];
      if (!(n2 * cof / n1 < conv)) next.push_back(j);
    }
    live.swap(next);
  }
  for (size_t j = 0; j < fl.size(); ++j)  // the workspaces keep their buffers
    if (fl[j]->INT2->d != p0[j]) {
      std::swap(fl[j]->INT2->d, fl[j]->AD->d);
      std::swap(fl[j]->INT2->zero_mask, fl[j]->AD->zero_mask);
    }
  return QD_OK;
}

// The lockstep batch: every layout on one stream (restored afterwards); per
// flow step the instances not yet converged run their step halves and one
// batched BCH_EXPAND.  An instance that fails or exceeds max_iter leaves the
// batch with its own status.
int flow_batch_lockstep(int count, const qd_op* const* HAM, qd_op* const* HS, unsigned flags, int max_iter,
                        qd_flow_result* results, int* status, std::vector<std::string>& msg) {
  std::vector<qd_layout*> Ls(count);
  for (int i = 0; i < count; ++i) {
    Ls[i] = HAM[i]->L;
    TRY(use_device(Ls[i]));
  }
  BatchCtx bc;
  QD_CUDA(cudaStreamCreateWithFlags(&bc.st, cudaStreamNonBlocking));
  QD_CUDA(cudaEventCreateWithFlags(&bc.ev_st, cudaEventDisableTiming));
  for (qd_layout* L : Ls) {
    cudaEvent_t e;
    QD_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    bc.ev[L] = e;
  }
  std::vector<qd_flow*> fl(count, nullptr);
  std::vector<int> loops(count, 0);
  int rc = QD_OK;
  for (int i = 0; i < count; ++i) {
    std::memset(&results[i], 0, sizeof(qd_flow_result));
    status[i] = qd_flow_create(HAM[i], HS[i], flags, &fl[i]);
    if (status[i] != QD_OK) msg[i] = qd::last_error();
  }
  while (rc == QD_OK) {
    std::vector<qd_flow*> act;
    std::vector<int> idx;
    std::vector<qd_flow_step_info> inf(count);
    for (int i = 0; i < count; ++i) {
      if (status[i] != QD_OK || !fl[i] || fl[i]->crit <= kConvCriteria) continue;
      if (loops[i]++ >= max_iter) {
        status[i] = QD_ERR_NOCONV;
        char b[128];
        snprintf(b, sizeof(b), "not converged after %d steps (crit %.3e)", max_iter, fl[i]->crit);
        msg[i] = b;
        continue;
      }
      bool conv = false;
      status[i] = flow_begin(fl[i], &inf[i], &conv);
      if (status[i] != QD_OK) {
        msg[i] = qd::last_error();
        continue;
      }
      act.push_back(fl[i]);
      idx.push_back(i);
    }
    if (act.empty()) break;
    std::vector<int> terms(act.size(), 0);
    rc = bch_batch(bc, act, terms);
    if (rc) break;
    for (size_t k = 0; k < act.size(); ++k) {
      const int i = idx[k];
      status[i] = flow_end(act[k], terms[k], &inf[i]);
      if (status[i] != QD_OK) msg[i] = qd::last_error();
    }
  }
  const std::string batch_err = rc ? qd::last_error() : std::string();
  for (int i = 0; i < count; ++i) {
    if (fl[i]) {
      qd_flow_state(fl[i], &results[i]);
      qd_flow_destroy(fl[i]);
    }
    if (rc) {
      status[i] = rc;
      msg[i] = batch_err;
    }
  }
  cudaStreamSynchronize(bc.st);
  for (auto& kv : bc.ev) cudaEventDestroy(kv.second);
  cudaEventDestroy(bc.ev_st);
  cudaStreamDestroy(bc.st);
  return QD_OK;
}
}  // namespace

extern "C" {

int qd_magnus_flow_batch(int count, const qd_op* const* HAM, qd_op* const* HS, unsigned flags, int max_iter,
                         qd_flow_result* results, int* status) {
  CHECK(count >= 0, QD_ERR_ARG, "qd_magnus_flow_batch: negative count");
  if (count == 0) return QD_OK;
  CHECK(HAM && HS && results && status, QD_ERR_ARG, "qd_magnus_flow_batch: null argument");
  for (int i = 0; i < count; ++i) {
    CHECK(HAM[i] && HS[i], QD_ERR_ARG, "qd_magnus_flow_batch: null operator %d", i);
    for (int j = 0; j < i; ++j)
      CHECK(HAM[i]->L != HAM[j]->L, QD_ERR_ARG,
            "qd_magnus_flow_batch: instances %d and %d share a layout (one stream per instance)", j, i);
  }
  std::vector<std::string> msg(count);
  bool lockstep = !(flags & QD_BATCH_STREAMS);
  for (int i = 0; i < count && lockstep; ++i)
    lockstep = HAM[i]->L->device == HAM[0]->L->device && HAM[i]->L->split_slices == 0 && !HAM[i]->L->prof.on;
  if (lockstep) {
    TRY(flow_batch_lockstep(count, HAM, HS, flags & ~QD_BATCH_STREAMS, max_iter, results, status, msg));
    for (int i = 0; i < count; ++i)
      if (status[i] != QD_OK) {
        qd::set_error("qd_magnus_flow_batch: instance %d: %s", i, msg[i].c_str());
        return status[i];
      }
    return QD_OK;
  }
  // one host thread per instance; each flow runs on its own layout's stream,
  // so the instances' kernels run concurrently on the device
  flags &= ~QD_BATCH_STREAMS;
  std::vector<std::thread> th;
  th.reserve(count);
  for (int i = 0; i < count; ++i)
    th.emplace_back([&, i]() {
      std::memset(&results[i], 0, sizeof(qd_flow_result));
      status[i] = qd_magnus_flow(HAM[i], HS[i], flags, max_iter, nullptr, &results[i]);
      if (status[i] != QD_OK) msg[i] = qd::last_error();
    });
  for (auto& t : th) t.join();
  for (int i = 0; i < count; ++i)
    if (status[i] != QD_OK) {
      qd::set_error("qd_magnus_flow_batch: instance %d: %s", i, msg[i].c_str());
      return status[i];
    }
  return QD_OK;
}

}  // extern "C"

namespace qd {
void graphs_free(qd_layout* L) {
  if (auto* m = reinterpret_cast<TermGraphs*>(L->graphs)) {
    for (auto& kv : *m)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    delete m;
    L->graphs = nullptr;
  }
  if (auto* m = reinterpret_cast<StepGraphs*>(L->step_graphs)) {
    for (auto& kv : *m)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    delete m;
    L->step_graphs = nullptr;
  }
}
}  // namespace qd
