// qd_internal.hpp -- host/device structures of the IM-SRG(2) commutator engine.
//
// Layout mirrors the reference's type(full_ham) / type(block) / type(cc_mat)
// (src/ME_general.f90:13-62) with everything needed on the device flattened
// into index tables:
//   * one FP64 array per operator in vectorize order (ME_general.f90:1871-1989)
//   * per (M_L,M_S) block: nhh, nph, npp and the six sub-block offsets
//   * a dense m*m pair table: ordered pair (a,b) -> (class, block, index, swap),
//     which is reindex's i_array (ME_general.f90:1028-1080) plus the ordering
//     sign of v_elem (ME_general.f90:1586-1599)
//   * cross-coupled (Pandya) blocks of build_cross_coupled (ME_general.f90:363-448)
//   * single-particle (m_l, m_s) groups: the only one-body couplings that reach
//     a block-diagonal two-body element (used to restrict the 122 sums).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/qd_imsrg.h"

namespace qd {

typedef long long i64;

// class ids of the nine stored parts of an operator (bit positions of
// qd_op::zero_mask)
enum Part { P_FHH = 0, P_FPP, P_FPH, P_HHHH, P_PPPP, P_PPHH, P_PHPH, P_PPPH, P_PHHH, P_COUNT };
constexpr unsigned ALL_PARTS = (1u << P_COUNT) - 1;

// pair-table packing: idx (13 bits) | block (10 bits) | class-1 (2 bits) | swap (1 bit)
__host__ __device__ inline int pt_idx(int e) { return e & 0x1FFF; }
__host__ __device__ inline int pt_blk(int e) { return (e >> 13) & 0x3FF; }
__host__ __device__ inline int pt_cls(int e) { return (e >> 23) & 0x3; }  // 0 hh, 1 ph, 2 pp
__host__ __device__ inline int pt_swap(int e) { return (e >> 25) & 0x1; }
inline int pt_pack(int idx, int blk, int cls, int swap) {
  return idx | (blk << 13) | (cls << 23) | (swap << 25);
}

// Device view of a layout (passed by value to kernels).
struct DevLayout {
  int n, m, mp, nblock, ncc, mlmax;
  i64 o_fhh, o_fpp, o_fph, neq;
  const int4* blk;        // nhh, nph, npp, ntot
  const i64* boff;        // 6 per block: hhhh, pppp, pphh, phph, ppph, phhh
  const int2* pairs;      // per block: hh pairs, ph pairs, pp pairs (0-based, a<b)
  const int* pbase;       // start of block q's pairs
  const int* ptab;        // m*m ordered pair -> packed, -1 on the diagonal
  const int* gid;         // (ml,ms) group of each state
  const int* gstart;      // CSR of group members (increasing states)
  const int* gmem;
  const int2* ccmap;      // m*m: (cc block, row), 0-based
  const int2* ccdim;      // r, nb per cc block
  const i64* ccxoff;      // offset of X(r,nb) per cc block
  const i64* cczoff;      // offset of the r x r product per cc block
  const int2* ccab;       // concatenated (i,j) row pairs of the cc blocks
  const int* ccab_base;
  const int2* cchp;       // concatenated (hole, particle) column pairs
  const int* cchp_base;
  // all non-empty two-body sub-blocks in vectorize order: start offset and
  // (block << 3) | (part - P_HHHH)
  const i64* s2off;
  const int* s2id;
  int ns2;
  i64 o2;                 // first two-body entry of the vectorize array
  // per two-body part p (0..5 = P_HHHH..P_PHHH): start of block q's entries
  // in the part's own flat numbering (pcum[p*nblock + q]) and the total
  const i64* pcum;
  i64 pcnt[6];
  // X (cross-coupled) flat numbering: cc block of each X entry via ccxoff
};

// ---- grouped FP64 GEMM program --------------------------------------------
enum GemmMode { GM_ACC = 0, GM_ACC_PAIR = 1, GM_SET = 2, GM_SET_PAIR = 3 };

struct GSeg {       // acc += alpha * op(A) * op(B), alpha = c * hv[0]^pa * hv[1]^pb
  i64 offA, offB;
  int lda, ldb, K;
  signed char srcA, srcB, tA, tB;
  signed char pa, pb, depA, depB;  // dep: part id of the source operator (-1 none)
  double c;
};
struct GProb {
  int M, N, ldc, seg0, nseg, mode, outbuf, pad;
  i64 offC;
  double sc;                       // pair transpose coefficient sc * hv[0]^spa * hv[1]^spb
  signed char spa, spb, pad2[6];
};
struct GTask {
  int prob;
  short ti, tj;
};

constexpr int NBUF = 7;
struct Bufs {
  const double* p[NBUF];
};
// One instance of a launch that covers several layouts' programs (batched
// flows): its program tables, operand buffers, herm factors and masks.
struct GInst {
  const GProb* probs;
  const GSeg* segs;
  Bufs bufs;
  double hv0, hv1;
  unsigned maskA, maskB;
};

struct GemmProgram {
  std::vector<GProb> probs;
  std::vector<GSeg> segs;
  GProb* d_probs = nullptr;
  GSeg* d_segs = nullptr;
  // task lists cached per (maskA, maskB): problems with a long K, and
  // K-short problems (every active segment together K <= 16)
  std::map<std::pair<unsigned, unsigned>, std::pair<GTask*, int>> tasks, tasks_short;
  void clear_device();
};

}  // namespace qd

namespace qd {
// stages timed by the optional per-stage CUDA-event profiler
enum Stage { S_E0 = 0, S_111, S_121, S_221, S_122, S_CALC_CC, S_LADDER, S_PANDYA_GEMM, S_PANDYA_GATHER, S_GLUE,
             S_COUNT };
struct StageProf {
  bool on = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending[S_COUNT];
  double ms[S_COUNT] = {0};
  long long count[S_COUNT] = {0};
};
}  // namespace qd

struct qd_layout {
  int device = 0;
  int children = 0;      // live operators and cross-coupled matrices on this layout
  bool closing = false;  // qd_layout_destroy was called while children were alive
  qd::StageProf prof;
  long long nlaunch = 0;  // kernels this library launched for the layout
  int n = 0, m = 0, mp = 0, emax = 0, nblock = 0, ncc = 0, mlmax = 0;
  qd::i64 neq = 0, o_fhh = 1, o_fpp = 0, o_fph = 0;
  std::vector<int> qn;      // m x 3 (n, ml, ms)
  std::vector<double> eig;  // m
  std::vector<int4> blk;
  std::vector<qd::i64> boff;
  std::vector<int2> pairs;
  std::vector<int> pbase;
  std::vector<int> ptab, gid, gstart, gmem;
  std::vector<int2> ccmap, ccdim, ccab, cchp;
  std::vector<int> ccab_base, cchp_base;
  // Rows of a cc block are ordered by the (ml,ms) group of their first state,
  // then (i, j): the rows (i in G1, j in G2) form one run.  ccref maps each
  // row (indexed like ccab) to its row in the reference's (i, j) loop order.
  std::vector<int> ccref;
  std::vector<qd::i64> ccxoff, cczoff;
  qd::i64 xsize = 0, zsize = 0;
  std::vector<qd::i64> s2off, pcum;
  std::vector<int> s2id;
  // device copies
  qd::DevLayout dev{};
  std::vector<void*> dev_allocs;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // work arena (grown on demand, freed with the layout)
  double* d_z = nullptr;          // Pandya products, zsize doubles
  double* d_red = nullptr;        // reduction partials
  double* h_red = nullptr;        // pinned scalar results
  double* d_axn = nullptr;        // partial sums of the fused BCH update (axpy + norms)
  int* d_ccflag = nullptr;        // per cross-coupled block: fph of A or B non-zero (121)
  const int* d_tgt221 = nullptr;  // one-body targets whose states share (m_l, m_s) (fused 221)
  int ntgt221 = -1;
  qd::i64 ws_bytes = 0;
  // GEMM programs
  qd::GemmProgram prog_ladder, prog_221, prog_111, prog_pandya;
  bool programs_built = false;
  // split form of the GEMM programs: slices per operand (0 = plain FP64)
  int split_slices = 0;
  void* split = nullptr;  // plans and workspaces (split_gemm.cu)
  // BCH terms replayed as CUDA graphs (api.cu)
  bool use_graphs = true;
  void* graphs = nullptr;       // per-term graphs
  void* step_graphs = nullptr;  // whole BCH steps with the truncation decided on the device
  long long graphs_captured = 0, graph_replays = 0;
};

struct qd_op {
  qd_layout* L = nullptr;
  int herm = 1;
  double* d = nullptr;
  unsigned zero_mask = 0;  // parts known to be identically zero
};

struct qd_cc {
  qd_layout* L = nullptr;
  double herm = 1.0;
  double* d = nullptr;  // X, xsize doubles
  bool filled = false;  // calc_cc has written X (otherwise X == 0)
};

namespace qd {

// error plumbing
void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
#define QD_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return qd::cuda_fail(e_, #call); \
  } while (0)

int layout_build(qd_layout* L, int nbody, int emax, const double* eig);
int layout_upload(qd_layout* L);
void layout_free_device(qd_layout* L);
int ensure_reduction(qd_layout* L);
int ensure_z(qd_layout* L);
int build_programs(qd_layout* L);

// part helpers
i64 part_count(const qd_layout* L, int part);  // total elements of a part over all blocks

// kernels (kernels_*.cu)
int launch_axpy(qd_layout* L, const double* a, double sa, const double* b, double sb, double* c, i64 n);
int launch_axpy_norms(qd_layout* L, const double* a, double sa, const double* b, double sb, double* c,
                      double* dout2, const int* kidx = nullptr);
int launch_bch_decide(qd_layout* L, const double* norms, int* kidx, double conv, cudaGraphConditionalHandle hloop,
                      cudaGraphConditionalHandle hnext, int set_next);
int prepare_program(qd_layout* L, GemmProgram& P, unsigned maskA, unsigned maskB);
// one program of one instance in a batched launch
struct GemmItem {
  qd_layout* L;
  GemmProgram* P;
  const double* bufs[NBUF];
  double hv0, hv1;
  unsigned maskA, maskB;
};
int run_programs_batched(cudaStream_t st, const std::vector<GemmItem>& items);
void drop_merged_gemm(const qd_layout* L);
// commutator_122 of one instance in a batched launch
struct Item122 {
  qd_layout* L;
  const qd_op* A;
  const qd_op* B;
  double* C;
};
int launch_122_batched(cudaStream_t st, const std::vector<Item122>& items);
void drop_merged_122(const qd_layout* L);
int prepare_122(qd_layout* L, const qd_op* A, const qd_op* B);
std::string tuning_report_122(const qd_layout* L);
double* scratch_operator(qd_layout* L);
int reduce_dot_range(qd_layout* L, const double* a, const double* b, i64 o, i64 n, double scale, double add,
                     double* dout);
int reduce_dot_part(qd_layout* L, const double* a, const double* b, int part, double scale, double add, double* dout);
int reduce_mbpt2(qd_layout* L, const double* h, double* dout);
int reduce_hhtrace(qd_layout* L, const double* h, double* dout);
int reduce_norm(qd_layout* L, const double* a, double* dout);
double* red_slot(qd_layout* L, int k);
int launch_white(qd_layout* L, double* gen, const double* h, int herm);
int launch_keep_parts(qd_layout* L, double* op, unsigned keep);
int launch_121(qd_layout* L, const qd_op* A, const qd_op* B, double* C);
int launch_221_trace(qd_layout* L, const qd_op* A, const qd_op* B, const qd_op* w1, const qd_op* w2, double* C);
int launch_221_fused(qd_layout* L, const qd_op* A, const qd_op* B, double* C);
int launch_122(qd_layout* L, const qd_op* A, const qd_op* B, double* C);
int launch_calc_cc(qd_layout* L, const qd_op* H, double* X);
// Particle-hole channel (commutators.f90:716-980): C += the four re-coupled
// Z terms, over the commutator_122 tiles (kernels_122.cu).
int launch_pandya_tiles(qd_layout* L, const double* Z, double* C);
int prepare_pandya(qd_layout* L);
int run_program(qd_layout* L, GemmProgram& P, const double* const* bufs, double hv0, double hv1, unsigned maskA,
                unsigned maskB);
int run_program_f64(qd_layout* L, GemmProgram& P, const double* const* bufs, double hv0, double hv1, unsigned maskA,
                    unsigned maskB);
int build_eom_ladders(qd_layout* L, const std::vector<int>& partner, const std::vector<i64>& qoff, GemmProgram& P);
void drop_eom_plans(const qd_layout* L);
void fill_random(const qd_layout* L, int herm, uint64_t seed, double sigma, int conserve, double* out);
int run_program_split(qd_layout* L, GemmProgram& P, const double* const* bufs, double hv0, double hv1, unsigned maskA,
                      unsigned maskB);
void split_free(qd_layout* L);
void graphs_free(qd_layout* L);

}  // namespace qd
