// gemm_f64.cu -- grouped FP64 block GEMM on the DMMA tensor pipe.
//
// All dense contractions of one commutator stage (the ladders of
// matrix_mult222, the intermediates of commutator_221, the one-body products
// of commutator_111 and the Pandya products of construct_cc_ints) run as ONE
// launch over a task list that covers every (M_L,M_S) block of uneven size.
//
// Problem = one output sub-block C (M x N, column-major, ldc) and a list of
// K-segments  acc += alpha_s * op(A_s) op(B_s); the segments are concatenated
// along K so every output tile is accumulated in registers and written once.
// Epilogue modes:
//   ACC       C += V
//   SET       C  = V
//   ACC_PAIR  C += V + sigma V^T      (M == N; the CTA computes the tile pair
//   SET_PAIR  C  = V + sigma V^T       (I,J),(J,I) so V^T is at hand)
// The pair modes carry the "hA*W^T - hB*W" transpose-adds of the reference
// (src/commutators.f90:1002-1127, :154-169) without a second GEMM.
//
// Tile 64x64x16, 4 warps (2x2), each warp 32x32 = 4x4 DMMA m8n8k4 fragments;
// 3-stage cp.async (8-byte, zero-fill) pipeline; FP64 accumulate.
// tcgen05 has no f64 kind, so mma.sync DMMA is the FP64 tensor path here.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#define TRY_GEMM(x)      \
  do {                   \
    int rc_ = (x);       \
    if (rc_) return rc_; \
  } while (0)

#include "dev_common.cuh"

namespace qd {

constexpr int BM = 64, BN = 64, BK = 16, LDS = 68, NSTAGE = 3, TLD = 65;
constexpr int GEMM_THREADS = 128;
constexpr int SMEM_PIPE = 2 * NSTAGE * BK * LDS;  // doubles
constexpr int SMEM_TILE = BN * TLD;               // doubles
constexpr size_t GEMM_SMEM = sizeof(double) * (SMEM_PIPE + SMEM_TILE);

__device__ __forceinline__ void cp_async8(double* s, const double* g, bool pred) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(g), "r"(sz));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ bool seg_active(const GSeg& s, unsigned mA, unsigned mB) {
  auto dead = [&](int src, int dep) {
    if (dep < 0) return false;
    unsigned m = src == 0 ? mA : (src == 1 ? mB : 0u);
    return ((m >> dep) & 1u) != 0;
  };
  return !dead(s.srcA, s.depA) && !dead(s.srcB, s.depB);
}

// Load the (row0, col0) tile's k-slab [k0, k0+BK) of segment s (operands at
// A, B) into stage buffers sA[k][m], sB[k][n].  Each thread walks a fixed
// column (or row) with a pointer stride; out-of-range elements are zero-filled.
__device__ __forceinline__ void load_stage(const GSeg& s, const double* A, const double* B, int M, int N, int row0,
                                           int col0, int k0, double* sA, double* sB) {
  const int tid = threadIdx.x;
  constexpr int IT = (BM * BK) / GEMM_THREADS;  // 8
  if (!s.tA) {  // A(m,k) at A[m + k*lda]: threads along m
    const int mm = tid & (BM - 1), kk0 = tid >> 6;
    const bool rok = row0 + mm < M;
    const double* g = A + (row0 + mm) + (i64)(k0 + kk0) * s.lda;
    const i64 step = (i64)2 * s.lda;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int kk = kk0 + 2 * it;
      const bool ok = rok && (k0 + kk < s.K);
      cp_async8(sA + kk * LDS + mm, ok ? g : A, ok);
      g += step;
    }
  } else {  // op(A)(m,k) = A[k + m*lda]: threads along k
    const int kk = tid & (BK - 1), mm0 = tid >> 4;
    const bool kok = k0 + kk < s.K;
    const double* g = A + (k0 + kk) + (i64)(row0 + mm0) * s.lda;
    const i64 step = (i64)8 * s.lda;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int mm = mm0 + 8 * it;
      const bool ok = kok && (row0 + mm < M);
      cp_async8(sA + kk * LDS + mm, ok ? g : A, ok);
      g += step;
    }
  }
  if (!s.tB) {  // B(k,n) at B[k + n*ldb]: threads along k
    const int kk = tid & (BK - 1), nn0 = tid >> 4;
    const bool kok = k0 + kk < s.K;
    const double* g = B + (k0 + kk) + (i64)(col0 + nn0) * s.ldb;
    const i64 step = (i64)8 * s.ldb;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int nn = nn0 + 8 * it;
      const bool ok = kok && (col0 + nn < N);
      cp_async8(sB + kk * LDS + nn, ok ? g : B, ok);
      g += step;
    }
  } else {  // op(B)(k,n) = B[n + k*ldb]: threads along n
    const int nn = tid & (BN - 1), kk0 = tid >> 6;
    const bool nok = col0 + nn < N;
    const double* g = B + (col0 + nn) + (i64)(k0 + kk0) * s.ldb;
    const i64 step = (i64)2 * s.ldb;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int kk = kk0 + 2 * it;
      const bool ok = nok && (k0 + kk < s.K);
      cp_async8(sB + kk * LDS + nn, ok ? g : B, ok);
      g += step;
    }
  }
}

// Active segments of the CTA's problem, kept in shared memory.
struct SegList {
  GSeg seg[8];
  const double* A[8];  // operand bases (buffer + offset)
  const double* B[8];
  double alpha[8];
  int nact;
  int total;  // k-tiles over all active segments
};

// Advance a (segment, k0) cursor by one k-tile.
__device__ __forceinline__ void cursor_next(const SegList& sl, int& si, int& k0) {
  k0 += BK;
  if (k0 >= sl.seg[si].K) {
    ++si;
    k0 = 0;
  }
}

// Accumulate the tile (row0, col0) of problem P into acc[4][4][2].
__device__ void tile_mainloop(const GProb& P, const SegList& sl, int row0, int col0, double* smem,
                              double acc[4][4][2]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp & 1, wn = warp >> 1;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int total = sl.total;
  if (total == 0) return;
  double* sA = smem;
  double* sB = smem + NSTAGE * BK * LDS;
  int ls = 0, lk = 0;  // load cursor
  int cs = 0, ck = 0;  // compute cursor
#pragma unroll
  for (int st = 0; st < NSTAGE - 1; ++st) {
    if (st < total) {
      load_stage(sl.seg[ls], sl.A[ls], sl.B[ls], P.M, P.N, row0, col0, lk, sA + st * BK * LDS,
                 sB + st * BK * LDS);
      cursor_next(sl, ls, lk);
    }
    cp_commit();
  }
  for (int g = 0; g < total; ++g) {
    const int gl = g + NSTAGE - 1;
    if (gl < total) {
      const int b = gl % NSTAGE;
      load_stage(sl.seg[ls], sl.A[ls], sl.B[ls], P.M, P.N, row0, col0, lk, sA + b * BK * LDS,
                 sB + b * BK * LDS);
      cursor_next(sl, ls, lk);
    }
    cp_commit();
    cp_wait<NSTAGE - 1>();
    __syncthreads();
    const double alpha = sl.alpha[cs];
    const double* a_s = sA + (g % NSTAGE) * BK * LDS;
    const double* b_s = sB + (g % NSTAGE) * BK * LDS;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double af[4], bf[4];
      const int kr = kk + (lane & 3);
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = a_s[kr * LDS + wm * 32 + i * 8 + (lane >> 2)];
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = b_s[kr * LDS + wn * 32 + j * 8 + (lane >> 2)];
      if (alpha != 1.0) {
#pragma unroll
        for (int i = 0; i < 4; ++i) af[i] *= alpha;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
    cursor_next(sl, cs, ck);
    __syncthreads();
  }
  cp_wait<0>();
  __syncthreads();
}

// accumulator fragments -> smem tile T[col*TLD + row]
__device__ __forceinline__ void stash(double* T, const double acc[4][4][2]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp & 1, wn = warp >> 1;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int r = wm * 32 + i * 8 + (lane >> 2);
      int c = wn * 32 + j * 8 + 2 * (lane & 3);
      T[c * TLD + r] = acc[i][j][0];
      T[(c + 1) * TLD + r] = acc[i][j][1];
    }
}

__global__ void __launch_bounds__(GEMM_THREADS) k_grouped_gemm(const GTask* __restrict__ tasks,
                                                               const GProb* __restrict__ probs,
                                                               const GSeg* __restrict__ segs, Bufs bufs, double hv0,
                                                               double hv1, unsigned maskA, unsigned maskB,
                                                               const int* __restrict__ tinst,
                                                               const GInst* __restrict__ insts) {
  extern __shared__ double smem[];
  if (tinst) {  // a task of several instances' programs: this instance's operands
    const GInst& I = insts[tinst[blockIdx.x]];
    probs = I.probs;
    segs = I.segs;
    bufs = I.bufs;
    hv0 = I.hv0;
    hv1 = I.hv1;
    maskA = I.maskA;
    maskB = I.maskB;
  }
  const GTask t = tasks[blockIdx.x];
  const GProb P = probs[t.prob];
  double* out = const_cast<double*>(bufs.p[P.outbuf]) + P.offC;

  __shared__ SegList sl;
  if (threadIdx.x == 0) {
    int na = 0, tot = 0;
    for (int k = 0; k < P.nseg && na < 8; ++k) {
      const GSeg sg = segs[P.seg0 + k];
      if (!seg_active(sg, maskA, maskB) || sg.K <= 0) continue;
      sl.seg[na] = sg;
      sl.A[na] = bufs.p[sg.srcA] + sg.offA;
      sl.B[na] = bufs.p[sg.srcB] + sg.offB;
      sl.alpha[na] = sg.c * (sg.pa ? hv0 : 1.0) * (sg.pb ? hv1 : 1.0);
      tot += (sg.K + BK - 1) / BK;
      ++na;
    }
    sl.nact = na;
    sl.total = tot;
  }
  __syncthreads();
  const bool pair = P.mode == GM_ACC_PAIR || P.mode == GM_SET_PAIR;
  const bool acc_mode = P.mode == GM_ACC || P.mode == GM_ACC_PAIR;
  double* T1 = smem + SMEM_PIPE;  // first tile stash (pair mode)
  double* T2 = smem;              // aliases the pipeline buffers after the main loop
  double acc[4][4][2];

  const int r0 = t.ti * BM, c0 = t.tj * BN;
  tile_mainloop(P, sl, r0, c0, smem, acc);

  if (!pair) {
    stash(T2, acc);
    __syncthreads();
    const int mr = min(BM, P.M - r0), nc = min(BN, P.N - c0);
    for (int idx = threadIdx.x; idx < BM * BN; idx += GEMM_THREADS) {
      int r = idx & (BM - 1), c = idx >> 6;
      if (r < mr && c < nc) {
        double* p = out + (r0 + r) + (i64)(c0 + c) * P.ldc;
        double v = T2[c * TLD + r];
        *p = acc_mode ? *p + v : v;
      }
    }
    return;
  }
  const double sigma = P.sc * (P.spa ? hv0 : 1.0) * (P.spb ? hv1 : 1.0);
  if (t.ti == t.tj) {
    stash(T1, acc);
    __syncthreads();
    const int mr = min(BM, P.M - r0);
    for (int idx = threadIdx.x; idx < BM * BN; idx += GEMM_THREADS) {
      int r = idx & (BM - 1), c = idx >> 6;
      if (r < mr && c < mr) {
        double* p = out + (r0 + r) + (i64)(r0 + c) * P.ldc;
        double v = T1[c * TLD + r] + sigma * T1[r * TLD + c];
        *p = acc_mode ? *p + v : v;
      }
    }
    return;
  }
  // off-diagonal tile pair: V(I,J) -> T1, then V(J,I) -> T2
  stash(T1, acc);
  __syncthreads();
  tile_mainloop(P, sl, c0, r0, smem, acc);
  stash(T2, acc);
  __syncthreads();
  const int mI = min(BM, P.M - r0), mJ = min(BM, P.M - c0);
  // C(I,J) (rows r0.., cols c0..) = T1 + sigma * T2^T
  for (int idx = threadIdx.x; idx < BM * BN; idx += GEMM_THREADS) {
    int r = idx & (BM - 1), c = idx >> 6;
    if (r < mI && c < mJ) {
      double* p = out + (r0 + r) + (i64)(c0 + c) * P.ldc;
      double v = T1[c * TLD + r] + sigma * T2[r * TLD + c];
      *p = acc_mode ? *p + v : v;
    }
  }
  // C(J,I) (rows c0.., cols r0..) = T2 + sigma * T1^T
  for (int idx = threadIdx.x; idx < BM * BN; idx += GEMM_THREADS) {
    int r = idx & (BM - 1), c = idx >> 6;
    if (r < mJ && c < mI) {
      double* p = out + (c0 + r) + (i64)(r0 + c) * P.ldc;
      double v = T2[c * TLD + r] + sigma * T1[r * TLD + c];
      *p = acc_mode ? *p + v : v;
    }
  }
}

// ---------------------------------------------------------------------------
// K-short problems: every active segment together spans K <= KS_K (in the
// Magnus flow the generator holds only fph and Vpphh, so the pppp and ppph
// ladders become rank-n_h updates, n_h <= 16).  Such a tile is one read-
// modify-write of C: no pipeline, the panels of all segments are staged once
// (alpha folded in), the two products of a pair tile are formed from four
// panels, and the shared memory is reused for the two transpose stashes
// (66.5 KB per CTA: three CTAs of eight warps on an SM).
// ---------------------------------------------------------------------------
constexpr int KS_K = 16, KS_THREADS = 256, KS_LDS = 68;
constexpr int KS_PANEL = KS_K * KS_LDS;                            // doubles per panel
// shared memory: stash 1 [BN*TLD] | panels A1 B1 A2 B2 (stash 2 overlaps the panels once the products are done)
constexpr int KS_PANEL0 = BN * TLD;
constexpr size_t KS_SMEM = sizeof(double) * (KS_PANEL0 + 4 * KS_PANEL > 2 * BN * TLD ? KS_PANEL0 + 4 * KS_PANEL
                                                                                      : 2 * BN * TLD);

// panel of op(A) rows [row0, row0+64) (sA[k][m]) and op(B) columns
// [col0, col0+64) (sB[k][n]) over the concatenated active segments; zeros
// outside M, N and beyond the total K
__device__ __forceinline__ void ks_panels(const SegList& sl, int M, int N, int row0, int col0, double* sA,
                                          double* sB) {
  for (int i = threadIdx.x; i < KS_PANEL; i += KS_THREADS) {
    sA[i] = 0.0;
    sB[i] = 0.0;
  }
  __syncthreads();
  int kb = 0;
  for (int si = 0; si < sl.nact; ++si) {
    const GSeg& s = sl.seg[si];
    const double* A = sl.A[si];
    const double* B = sl.B[si];
    const double al = sl.alpha[si];
    for (int e = threadIdx.x; e < s.K * BM; e += KS_THREADS) {
      // element (m or n fastest when that index is contiguous in memory)
      int m, k;
      if (!s.tA) { m = e % BM; k = e / BM; } else { k = e % s.K; m = e / s.K; }
      if (row0 + m < M) sA[(kb + k) * KS_LDS + m] = al * (s.tA ? A[k + (i64)(row0 + m) * s.lda] : A[(row0 + m) + (i64)k * s.lda]);
      int n, k2;
      if (s.tB) { n = e % BN; k2 = e / BN; } else { k2 = e % s.K; n = e / s.K; }
      if (col0 + n < N) sB[(kb + k2) * KS_LDS + n] = s.tB ? B[(col0 + n) + (i64)k2 * s.ldb] : B[k2 + (i64)(col0 + n) * s.ldb];
    }
    kb += s.K;
  }
  __syncthreads();
}

// acc[4][2][2] (warp tile 32 x 16) = sA^T sB over KS_K
__device__ __forceinline__ void ks_mma(const double* sA, const double* sB, double acc[4][2][2]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp & 1, wn = warp >> 1;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll
  for (int kk = 0; kk < KS_K; kk += 4) {
    const int kr = kk + (lane & 3);
    double af[4], bf[2];
#pragma unroll
    for (int i = 0; i < 4; ++i) af[i] = sA[kr * KS_LDS + wm * 32 + i * 8 + (lane >> 2)];
#pragma unroll
    for (int j = 0; j < 2; ++j) bf[j] = sB[kr * KS_LDS + wn * 16 + j * 8 + (lane >> 2)];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
  }
}

__device__ __forceinline__ void ks_stash(double* T, const double acc[4][2][2]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp & 1, wn = warp >> 1;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int r = wm * 32 + i * 8 + (lane >> 2);
      const int c = wn * 16 + j * 8 + 2 * (lane & 3);
      T[c * TLD + r] = acc[i][j][0];
      T[(c + 1) * TLD + r] = acc[i][j][1];
    }
}

__global__ void __launch_bounds__(KS_THREADS, 3) k_gemm_kshort(const GTask* __restrict__ tasks,
                                                            const GProb* __restrict__ probs,
                                                            const GSeg* __restrict__ segs, Bufs bufs, double hv0,
                                                            double hv1, unsigned maskA, unsigned maskB,
                                                            const int* __restrict__ tinst,
                                                            const GInst* __restrict__ insts) {
  extern __shared__ double smem[];
  __shared__ SegList sl;
  if (tinst) {  // a task of several instances' programs: this instance's operands
    const GInst& I = insts[tinst[blockIdx.x]];
    probs = I.probs;
    segs = I.segs;
    bufs = I.bufs;
    hv0 = I.hv0;
    hv1 = I.hv1;
    maskA = I.maskA;
    maskB = I.maskB;
  }
  const GTask t = tasks[blockIdx.x];
  const GProb P = probs[t.prob];
  double* out = const_cast<double*>(bufs.p[P.outbuf]) + P.offC;
  if (threadIdx.x == 0) {
    int na = 0, tot = 0;
    for (int k = 0; k < P.nseg && na < 8; ++k) {
      const GSeg sg = segs[P.seg0 + k];
      if (!seg_active(sg, maskA, maskB) || sg.K <= 0) continue;
      sl.seg[na] = sg;
      sl.A[na] = bufs.p[sg.srcA] + sg.offA;
      sl.B[na] = bufs.p[sg.srcB] + sg.offB;
      sl.alpha[na] = sg.c * (sg.pa ? hv0 : 1.0) * (sg.pb ? hv1 : 1.0);
      tot += sg.K;
      ++na;
    }
    sl.nact = na;
    sl.total = tot;  // <= KS_K (the host routes only such problems here)
  }
  __syncthreads();
  const bool pair = P.mode == GM_ACC_PAIR || P.mode == GM_SET_PAIR;
  const bool acc_mode = P.mode == GM_ACC || P.mode == GM_ACC_PAIR;
  const int r0 = t.ti * BM, c0 = t.tj * BN;
  double* pA1 = smem + KS_PANEL0;
  double* pB1 = pA1 + KS_PANEL;
  double* T = smem;  // stash 1: below the panels
  double v1[4][2][2];
  if (!pair || t.ti == t.tj) {
    ks_panels(sl, P.M, P.N, r0, c0, pA1, pB1);
    ks_mma(pA1, pB1, v1);
    __syncthreads();
    ks_stash(T, v1);
    __syncthreads();
    const double sigma = pair ? P.sc * (P.spa ? hv0 : 1.0) * (P.spb ? hv1 : 1.0) : 0.0;
    const int mr = min(BM, P.M - r0), nc = min(BN, P.N - c0);
    // read-modify-write of C: a thread's loads of a chunk first, then the stores
    constexpr int PER = BM * BN / KS_THREADS, CH = 8;
#pragma unroll
    for (int k0 = 0; k0 < PER; k0 += CH) {
      double cv[CH];
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        const int idx = threadIdx.x + (k0 + k) * KS_THREADS, r = idx & (BM - 1), c = idx >> 6;
        cv[k] = (acc_mode && r < mr && c < nc) ? out[(r0 + r) + (i64)(c0 + c) * P.ldc] : 0.0;
      }
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        const int idx = threadIdx.x + (k0 + k) * KS_THREADS, r = idx & (BM - 1), c = idx >> 6;
        if (r < mr && c < nc) {
          const double v = pair ? T[c * TLD + r] + sigma * T[r * TLD + c] : T[c * TLD + r];
          out[(r0 + r) + (i64)(c0 + c) * P.ldc] = acc_mode ? cv[k] + v : v;
        }
      }
    }
    return;
  }
  // off-diagonal tile pair: V(I,J) = A_I B_J^T and V(J,I) = A_J B_I^T, each
  // stashed right after its product (one accumulator live at a time), then
  // C(I,J) = V(I,J) + sigma V(J,I)^T and C(J,I) = V(J,I) + sigma V(I,J)^T
  // written column by column
  double* pA2 = pB1 + KS_PANEL;
  double* pB2 = pA2 + KS_PANEL;
  double* T1 = smem;
  double* T2 = smem + BN * TLD;  // overlaps the panels: written after every product is done
  ks_panels(sl, P.M, P.N, r0, c0, pA1, pB1);
  ks_panels(sl, P.M, P.N, c0, r0, pA2, pB2);
  ks_mma(pA1, pB1, v1);
  ks_stash(T1, v1);
  ks_mma(pA2, pB2, v1);
  __syncthreads();
  ks_stash(T2, v1);
  __syncthreads();
  const double sigma = P.sc * (P.spa ? hv0 : 1.0) * (P.spb ? hv1 : 1.0);
  const int mI = min(BM, P.M - r0), mJ = min(BM, P.M - c0);
  constexpr int PER = BM * BN / KS_THREADS;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const double* Ta = side == 0 ? T1 : T2;
    const double* Tb = side == 0 ? T2 : T1;
    const int rb = side == 0 ? r0 : c0, cb = side == 0 ? c0 : r0;
    const int mr = side == 0 ? mI : mJ, nc = side == 0 ? mJ : mI;
    constexpr int CH = 8;
#pragma unroll
    for (int k0 = 0; k0 < PER; k0 += CH) {
      double cv[CH];  // read-modify-write of C: a chunk's loads first, then its stores
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        const int idx = threadIdx.x + (k0 + k) * KS_THREADS, r = idx & (BM - 1), c = idx >> 6;
        cv[k] = (acc_mode && r < mr && c < nc) ? out[(rb + r) + (i64)(cb + c) * P.ldc] : 0.0;
      }
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        const int idx = threadIdx.x + (k0 + k) * KS_THREADS, r = idx & (BM - 1), c = idx >> 6;
        if (r < mr && c < nc) {
          const double x = Ta[c * TLD + r] + sigma * Tb[r * TLD + c];
          out[(rb + r) + (i64)(cb + c) * P.ldc] = acc_mode ? cv[k] + x : x;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Host side: program construction and launch
// ---------------------------------------------------------------------------
namespace {

struct Builder {
  GemmProgram& P;
  int cur = -1;
  explicit Builder(GemmProgram& p) : P(p) {}
  void prob(int M, int N, i64 offC, int ldc, int mode, int outbuf, double sc = 0.0, int spa = 0, int spb = 0) {
    GProb g;
    std::memset(&g, 0, sizeof(g));
    g.M = M;
    g.N = N;
    g.ldc = ldc;
    g.offC = offC;
    g.mode = mode;
    g.outbuf = outbuf;
    g.seg0 = (int)P.segs.size();
    g.nseg = 0;
    g.sc = sc;
    g.spa = (signed char)spa;
    g.spb = (signed char)spb;
    P.probs.push_back(g);
    cur = (int)P.probs.size() - 1;
  }
  // acc += c * hv0^pa * hv1^pb * op(A) op(B)
  void seg(int srcA, i64 offA, int lda, bool tA, int depA, int srcB, i64 offB, int ldb, bool tB, int depB, int K,
           double c, int pa = 0, int pb = 0) {
    if (K <= 0) return;
    GSeg s;
    std::memset(&s, 0, sizeof(s));
    s.offA = offA;
    s.offB = offB;
    s.lda = std::max(1, lda);
    s.ldb = std::max(1, ldb);
    s.K = K;
    s.srcA = (signed char)srcA;
    s.srcB = (signed char)srcB;
    s.tA = tA;
    s.tB = tB;
    s.depA = (signed char)depA;
    s.depB = (signed char)depB;
    s.pa = (signed char)pa;
    s.pb = (signed char)pb;
    s.c = c;
    P.segs.push_back(s);
    P.probs[cur].nseg++;
  }
  void drop_if_empty() {
    if (cur >= 0 && P.probs[cur].nseg == 0) {
      P.probs.pop_back();
      cur = -1;
    }
  }
};

// operand buffer ids
enum { BA = 0, BB = 1, BXA = 2, BXB = 3, BO0 = 4, BO1 = 5, BZ = 6 };
const bool N_ = false, T_ = true;

}  // namespace

int build_programs(qd_layout* L) {
  if (L->programs_built) return QD_OK;
  const int n = L->n, mp = L->mp;
  // ---- matrix_mult222 ladders (ACC into C) ----
  {
    GemmProgram& P = L->prog_ladder;
    Builder b(P);
    for (int q = 0; q < L->nblock; ++q) {
      const int nh = L->blk[q].x, nb = L->blk[q].y, np = L->blk[q].z;
      const i64* o = &L->boff[6 * q];
      const i64 hhhh = o[0], pppp = o[1], pphh = o[2], phph = o[3], ppph = o[4], phhh = o[5];
      if (nh > 0) {  // V = -hB Bpphh^T Apphh - Ahhhh Bhhhh ; C += V + s V^T
        b.prob(nh, nh, hhhh, nh, GM_ACC_PAIR, BO0, -1.0, 1, 1);
        if (np > 0) b.seg(BB, pphh, np, T_, P_PPHH, BA, pphh, np, N_, P_PPHH, np, -1.0, 0, 1);
        b.seg(BA, hhhh, nh, N_, P_HHHH, BB, hhhh, nh, N_, P_HHHH, nh, -1.0);
        b.drop_if_empty();
      }
      if (np > 0) {  // V = -hB Apphh Bpphh^T - Bpppp Apppp
        b.prob(np, np, pppp, np, GM_ACC_PAIR, BO0, -1.0, 1, 1);
        if (nh > 0) b.seg(BA, pphh, np, N_, P_PPHH, BB, pphh, np, T_, P_PPHH, nh, -1.0, 0, 1);
        b.seg(BB, pppp, np, N_, P_PPPP, BA, pppp, np, N_, P_PPPP, np, -1.0);
        b.drop_if_empty();
      }
      if (nb > 0) {  // V = -hB (Aphhh Bphhh^T + Bppph^T Appph)
        b.prob(nb, nb, phph, nb, GM_ACC_PAIR, BO0, -1.0, 1, 1);
        if (nh > 0) b.seg(BA, phhh, nb, N_, P_PHHH, BB, phhh, nb, T_, P_PHHH, nh, -1.0, 0, 1);
        if (np > 0) b.seg(BB, ppph, np, T_, P_PPPH, BA, ppph, np, N_, P_PPPH, np, -1.0, 0, 1);
        b.drop_if_empty();
      }
      if (np > 0 && nh > 0) {  // Apppp Bpphh - Bpppp Apphh - Apphh Bhhhh + Bpphh Ahhhh
        b.prob(np, nh, pphh, np, GM_ACC, BO0);
        b.seg(BA, pppp, np, N_, P_PPPP, BB, pphh, np, N_, P_PPHH, np, 1.0);
        b.seg(BB, pppp, np, N_, P_PPPP, BA, pphh, np, N_, P_PPHH, np, -1.0);
        b.seg(BA, pphh, np, N_, P_PPHH, BB, hhhh, nh, N_, P_HHHH, nh, -1.0);
        b.seg(BB, pphh, np, N_, P_PPHH, BA, hhhh, nh, N_, P_HHHH, nh, 1.0);
        b.drop_if_empty();
      }
      if (nb > 0 && nh > 0) {  // hA Appph^T Bpphh - hB Bppph^T Apphh - Aphhh Bhhhh + Bphhh Ahhhh
        b.prob(nb, nh, phhh, nb, GM_ACC, BO0);
        if (np > 0) {
          b.seg(BA, ppph, np, T_, P_PPPH, BB, pphh, np, N_, P_PPHH, np, 1.0, 1, 0);
          b.seg(BB, ppph, np, T_, P_PPPH, BA, pphh, np, N_, P_PPHH, np, -1.0, 0, 1);
        }
        b.seg(BA, phhh, nb, N_, P_PHHH, BB, hhhh, nh, N_, P_HHHH, nh, -1.0);
        b.seg(BB, phhh, nb, N_, P_PHHH, BA, hhhh, nh, N_, P_HHHH, nh, 1.0);
        b.drop_if_empty();
      }
      if (np > 0 && nb > 0) {  // -hB Apphh Bphhh^T + hA Bpphh Aphhh^T + Apppp Bppph - Bpppp Appph
        b.prob(np, nb, ppph, np, GM_ACC, BO0);
        if (nh > 0) {
          b.seg(BA, pphh, np, N_, P_PPHH, BB, phhh, nb, T_, P_PHHH, nh, -1.0, 0, 1);
          b.seg(BB, pphh, np, N_, P_PPHH, BA, phhh, nb, T_, P_PHHH, nh, 1.0, 1, 0);
        }
        b.seg(BA, pppp, np, N_, P_PPPP, BB, ppph, np, N_, P_PPPH, np, 1.0);
        b.seg(BB, pppp, np, N_, P_PPPP, BA, ppph, np, N_, P_PPPH, np, -1.0);
        b.drop_if_empty();
      }
    }
  }
  // ---- commutator_221 intermediates (SET into w1 = BO0, w2 = BO1) ----
  {
    GemmProgram& P = L->prog_221;
    Builder b(P);
    for (int q = 0; q < L->nblock; ++q) {
      const int nh = L->blk[q].x, nb = L->blk[q].y, np = L->blk[q].z;
      const i64* o = &L->boff[6 * q];
      const i64 hhhh = o[0], pppp = o[1], pphh = o[2], phph = o[3], ppph = o[4], phhh = o[5];
      if (np * nh != 0) {
        b.prob(np, np, pppp, np, GM_SET, BO0);  // w1%Vpppp = Apphh Bpphh^T
        b.seg(BA, pphh, np, N_, P_PPHH, BB, pphh, np, T_, P_PPHH, nh, 1.0);
      }
      if (np * nb != 0) {
        b.prob(nb, nb, phph, nb, GM_SET, BO0);  // w1%Vphph = Bppph^T Appph
        b.seg(BB, ppph, np, T_, P_PPPH, BA, ppph, np, N_, P_PPPH, np, 1.0);
      }
      if (nh * np != 0) {
        b.prob(nh, nh, hhhh, nh, GM_SET, BO0);  // w1%Vhhhh = Bpphh^T Apphh
        b.seg(BB, pphh, np, T_, P_PPHH, BA, pphh, np, N_, P_PPHH, np, 1.0);
      }
      if (nh * nb != 0) {
        b.prob(nb, nb, phph, nb, GM_SET, BO1);  // w2%Vphph = Aphhh Bphhh^T
        b.seg(BA, phhh, nb, N_, P_PHHH, BB, phhh, nb, T_, P_PHHH, nh, 1.0);
      }
      if (nh * nb * np != 0) {
        b.prob(nb, nh, phhh, nb, GM_SET, BO0);  // w1%Vphhh = Bppph^T Apphh
        b.seg(BB, ppph, np, T_, P_PPPH, BA, pphh, np, N_, P_PPHH, np, 1.0);
        b.prob(nb, nh, phhh, nb, GM_SET, BO1);  // w2%Vphhh = Appph^T Bpphh
        b.seg(BA, ppph, np, T_, P_PPPH, BB, pphh, np, N_, P_PPHH, np, 1.0);
        b.prob(np, nb, ppph, np, GM_SET, BO0);  // w1%Vppph = Apphh Bphhh^T
        b.seg(BA, pphh, np, N_, P_PPHH, BB, phhh, nb, T_, P_PHHH, nh, 1.0);
        b.prob(np, nb, ppph, np, GM_SET, BO1);  // w2%Vppph = Bpphh Aphhh^T
        b.seg(BB, pphh, np, N_, P_PPHH, BA, phhh, nb, T_, P_PHHH, nh, 1.0);
      }
    }
  }
  // ---- commutator_111 (SET into C's one-body part) ----
  {
    GemmProgram& P = L->prog_111;
    Builder b(P);
    if (n > 0) {  // V = Afhh Bfhh - hB Bfph^T Afph ; fhh = V + s V^T
      b.prob(n, n, L->o_fhh, n, GM_SET_PAIR, BO0, -1.0, 1, 1);
      b.seg(BA, L->o_fhh, n, N_, P_FHH, BB, L->o_fhh, n, N_, P_FHH, n, 1.0);
      if (mp > 0) b.seg(BB, L->o_fph, mp, T_, P_FPH, BA, L->o_fph, mp, N_, P_FPH, mp, -1.0, 0, 1);
    }
    if (mp > 0) {  // V = hB Afph Bfph^T - Bfpp Afpp ; fpp = V + s V^T
      b.prob(mp, mp, L->o_fpp, mp, GM_SET_PAIR, BO0, -1.0, 1, 1);
      if (n > 0) b.seg(BA, L->o_fph, mp, N_, P_FPH, BB, L->o_fph, mp, T_, P_FPH, n, 1.0, 0, 1);
      b.seg(BB, L->o_fpp, mp, N_, P_FPP, BA, L->o_fpp, mp, N_, P_FPP, mp, -1.0);
    }
    if (mp > 0 && n > 0) {  // fph = Afph Bfhh - Bfph Afhh + Afpp Bfph - Bfpp Afph
      b.prob(mp, n, L->o_fph, mp, GM_SET, BO0);
      b.seg(BA, L->o_fph, mp, N_, P_FPH, BB, L->o_fhh, n, N_, P_FHH, n, 1.0);
      b.seg(BB, L->o_fph, mp, N_, P_FPH, BA, L->o_fhh, n, N_, P_FHH, n, -1.0);
      b.seg(BA, L->o_fpp, mp, N_, P_FPP, BB, L->o_fph, mp, N_, P_FPH, mp, 1.0);
      b.seg(BB, L->o_fpp, mp, N_, P_FPP, BA, L->o_fph, mp, N_, P_FPH, mp, -1.0);
    }
  }
  // ---- construct_cc_ints as Z = XCC - YCC = hB P - hA P^T, P = X_A X_B^T ----
  {
    GemmProgram& P = L->prog_pandya;
    Builder b(P);
    for (int q = 0; q < L->ncc; ++q) {
      const int r = L->ccdim[q].x, nb = L->ccdim[q].y;
      if (r == 0) continue;
      b.prob(r, r, L->cczoff[q], r, GM_SET_PAIR, BZ, -1.0, 1, 1);  // nb == 0 writes zeros
      if (nb > 0) b.seg(BXA, L->ccxoff[q], r, N_, -1, BXB, L->ccxoff[q], r, T_, -1, nb, 1.0, 0, 1);
    }
  }
  // upload
  for (GemmProgram* P : {&L->prog_ladder, &L->prog_221, &L->prog_111, &L->prog_pandya}) {
    size_t pb = std::max<size_t>(1, P->probs.size()) * sizeof(GProb);
    size_t sb = std::max<size_t>(1, P->segs.size()) * sizeof(GSeg);
    QD_CUDA(cudaMalloc(&P->d_probs, pb));
    QD_CUDA(cudaMalloc(&P->d_segs, sb));
    if (!P->probs.empty())
      QD_CUDA(cudaMemcpy(P->d_probs, P->probs.data(), P->probs.size() * sizeof(GProb), cudaMemcpyHostToDevice));
    if (!P->segs.empty())
      QD_CUDA(cudaMemcpy(P->d_segs, P->segs.data(), P->segs.size() * sizeof(GSeg), cudaMemcpyHostToDevice));
  }
  QD_CUDA(cudaFuncSetAttribute(k_grouped_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM));
  QD_CUDA(cudaFuncSetAttribute(k_gemm_kshort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KS_SMEM));
  L->programs_built = true;
  return QD_OK;
}

// Ladder sums of the EOM product for a non-scalar target (eom.cu): per bra
// block q with ket block partner[q] (pairs of M_q minus the target), the
// npp(q) x nhh(partner[q]) output Wb[q] = Vpppp[q] Qb[q] + Qb[q] Vhhhh[partner[q]]
// (the c<d and k<l sums of HQ_comm_2b, src/commutators.f90:1246-1258).
// Buffers: H = BA, the amplitude matrices Qb = BB, the output Wb = BO0.
int build_eom_ladders(qd_layout* L, const std::vector<int>& partner, const std::vector<i64>& qoff, GemmProgram& P) {
  Builder b(P);
  for (int q = 0; q < L->nblock; ++q) {
    const int q2 = partner[q];
    if (q2 < 0) continue;
    const int np = L->blk[q].z, nh2 = L->blk[q2].x;
    if (np == 0 || nh2 == 0) continue;
    b.prob(np, nh2, qoff[q], np, GM_SET, BO0);
    b.seg(BA, L->boff[6 * q + 1], np, N_, P_PPPP, BB, qoff[q], np, N_, -1, np, 1.0);
    b.seg(BB, qoff[q], np, N_, -1, BA, L->boff[6 * q2 + 0], nh2, N_, P_HHHH, nh2, 1.0);
  }
  size_t pb = std::max<size_t>(1, P.probs.size()) * sizeof(GProb);
  size_t sb = std::max<size_t>(1, P.segs.size()) * sizeof(GSeg);
  QD_CUDA(cudaMalloc(&P.d_probs, pb));
  QD_CUDA(cudaMalloc(&P.d_segs, sb));
  if (!P.probs.empty())
    QD_CUDA(cudaMemcpy(P.d_probs, P.probs.data(), P.probs.size() * sizeof(GProb), cudaMemcpyHostToDevice));
  if (!P.segs.empty())
    QD_CUDA(cudaMemcpy(P.d_segs, P.segs.data(), P.segs.size() * sizeof(GSeg), cudaMemcpyHostToDevice));
  return QD_OK;
}

static bool seg_active_host(const GSeg& s, unsigned mA, unsigned mB) {
  auto dead = [&](int src, int dep) {
    if (dep < 0) return false;
    unsigned m = src == 0 ? mA : (src == 1 ? mB : 0u);
    return ((m >> dep) & 1u) != 0;
  };
  return !dead(s.srcA, s.depA) && !dead(s.srcB, s.depB);
}

// Host task lists of P for (mA, mB): [0] long-K problems, [1] K-short ones,
// each as (cost, task), longest first.  Every tile (tile pair in the pair
// modes) of every problem that has an active segment (SET problems always:
// they must write); problems whose active segments span K <= KS_K (at most
// 8 of them) go to the K-short kernel.
static void task_vectors(const GemmProgram& P, unsigned mA, unsigned mB, std::vector<std::pair<double, GTask>> v[2]) {
  for (size_t pi = 0; pi < P.probs.size(); ++pi) {
    const GProb& g = P.probs[pi];
    double kt = 0.0;
    int ksum = 0, nact = 0;
    for (int k = 0; k < g.nseg; ++k) {
      const GSeg& s = P.segs[g.seg0 + k];
      if (seg_active_host(s, mA, mB) && s.K > 0) {
        kt += (s.K + BK - 1) / BK;
        ksum += s.K;
        ++nact;
      }
    }
    bool set = g.mode == GM_SET || g.mode == GM_SET_PAIR;
    if (kt == 0.0 && !set) continue;
    const int which = (ksum <= KS_K && nact <= 8) ? 1 : 0;
    int tm = (g.M + BM - 1) / BM, tn = (g.N + BN - 1) / BN;
    bool pair = g.mode == GM_ACC_PAIR || g.mode == GM_SET_PAIR;
    for (int i = 0; i < tm; ++i)
      for (int j = pair ? i : 0; j < tn; ++j) {
        GTask t;
        t.prob = (int)pi;
        t.ti = (short)i;
        t.tj = (short)j;
        double cost = (kt + 1.0) * ((pair && i != j) ? 2.0 : 1.0);
        v[which].push_back({cost, t});
      }
  }
  for (int w = 0; w < 2; ++w)
    std::stable_sort(v[w].begin(), v[w].end(), [](const auto& a, const auto& b) { return a.first > b.first; });
}

static int get_tasks(qd_layout* L, GemmProgram& P, unsigned mA, unsigned mB, GTask** d_tasks, int* ntasks,
                     GTask** d_short, int* nshort) {
  (void)L;
  auto key = std::make_pair(mA, mB);
  auto it = P.tasks.find(key);
  if (it != P.tasks.end()) {
    *d_tasks = it->second.first;
    *ntasks = it->second.second;
    *d_short = P.tasks_short[key].first;
    *nshort = P.tasks_short[key].second;
    return QD_OK;
  }
  std::vector<std::pair<double, GTask>> v[2];
  task_vectors(P, mA, mB, v);
  GTask* d[2] = {nullptr, nullptr};
  for (int w = 0; w < 2; ++w) {
    std::vector<GTask> h(v[w].size());
    for (size_t i = 0; i < v[w].size(); ++i) h[i] = v[w][i].second;
    if (!h.empty()) {
      QD_CUDA(cudaMalloc(&d[w], h.size() * sizeof(GTask)));
      QD_CUDA(cudaMemcpy(d[w], h.data(), h.size() * sizeof(GTask), cudaMemcpyHostToDevice));
    }
  }
  P.tasks[key] = std::make_pair(d[0], (int)v[0].size());
  P.tasks_short[key] = std::make_pair(d[1], (int)v[1].size());
  *d_tasks = d[0];
  *ntasks = (int)v[0].size();
  *d_short = d[1];
  *nshort = (int)v[1].size();
  return QD_OK;
}

// Build (allocate and upload) the task lists of P for a pair of zero-part
// masks ahead of a stream capture, which must not allocate.
int prepare_program(qd_layout* L, GemmProgram& P, unsigned maskA, unsigned maskB) {
  int rc = build_programs(L);
  if (rc) return rc;
  GTask *d1, *d2;
  int n1, n2;
  return get_tasks(L, P, maskA, maskB, &d1, &n1, &d2, &n2);
}

int run_program(qd_layout* L, GemmProgram& P, const double* const* bufs, double hv0, double hv1, unsigned maskA,
                unsigned maskB) {
  int rc = build_programs(L);
  if (rc) return rc;
  if (L->split_slices > 0) return run_program_split(L, P, bufs, hv0, hv1, maskA, maskB);
  return run_program_f64(L, P, bufs, hv0, hv1, maskA, maskB);
}

// P in FP64 on the DMMA pipe whatever the layout's form (P's tables must be
// on the device: build_programs or build_eom_ladders).
int run_program_f64(qd_layout* L, GemmProgram& P, const double* const* bufs, double hv0, double hv1, unsigned maskA,
                    unsigned maskB) {
  int rc = build_programs(L);  // sets the kernels' shared-memory limits
  if (rc) return rc;
  GTask *d_tasks = nullptr, *d_short = nullptr;
  int nt = 0, ns = 0;
  if ((rc = get_tasks(L, P, maskA, maskB, &d_tasks, &nt, &d_short, &ns))) return rc;
  Bufs b;
  for (int i = 0; i < NBUF; ++i) b.p[i] = bufs[i];
  if (nt > 0) {
    k_grouped_gemm<<<nt, GEMM_THREADS, GEMM_SMEM, L->stream>>>(d_tasks, P.d_probs, P.d_segs, b, hv0, hv1, maskA,
                                                                maskB, nullptr, nullptr);
    ++L->nlaunch;
  }
  if (ns > 0) {
    k_gemm_kshort<<<ns, KS_THREADS, KS_SMEM, L->stream>>>(d_short, P.d_probs, P.d_segs, b, hv0, hv1, maskA, maskB,
                                                          nullptr, nullptr);
    ++L->nlaunch;
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// ---- one launch over several instances' programs (batched flows) ---------
namespace {
struct MergedGemm {
  GTask* d_task[2] = {nullptr, nullptr};  // long-K, K-short
  int* d_tinst[2] = {nullptr, nullptr};
  int n[2] = {0, 0};
  GInst* d_inst = nullptr;
  GInst* h_inst = nullptr;  // pinned staging of the per-call instance table
  std::vector<const qd_layout*> layouts;
};
std::map<std::vector<uintptr_t>, MergedGemm>& merged_gemm() {
  static std::map<std::vector<uintptr_t>, MergedGemm> m;
  return m;
}
std::mutex g_merged_gemm_mutex;

void free_merged(MergedGemm& m) {
  for (int w = 0; w < 2; ++w) {
    if (m.d_task[w]) cudaFree(m.d_task[w]);
    if (m.d_tinst[w]) cudaFree(m.d_tinst[w]);
  }
  if (m.d_inst) cudaFree(m.d_inst);
  if (m.h_inst) cudaFreeHost(m.h_inst);
}
}  // namespace

// Every item's program P on its operands, as one launch per kernel (long-K
// and K-short tasks of all items interleaved, longest first); the items'
// layouts share `st`.  The task lists are cached per (layout, program,
// masks) tuple; the instance table is uploaded per call from pinned memory,
// which the caller rewrites only after synchronising the stream.
int run_programs_batched(cudaStream_t st, const std::vector<GemmItem>& items) {
  if (items.empty()) return QD_OK;
  std::vector<uintptr_t> key;
  for (const GemmItem& it : items) {
    TRY_GEMM(build_programs(it.L));
    key.push_back((uintptr_t)it.L);
    key.push_back((uintptr_t)it.P);
    key.push_back(((uintptr_t)it.maskA << 16) | it.maskB);
  }
  MergedGemm* m;
  {
    std::lock_guard<std::mutex> lock(g_merged_gemm_mutex);
    auto f = merged_gemm().find(key);
    if (f == merged_gemm().end()) {
      MergedGemm mg;
      std::vector<std::pair<double, std::pair<GTask, int>>> all[2];
      for (size_t i = 0; i < items.size(); ++i) {
        std::vector<std::pair<double, GTask>> v[2];
        task_vectors(*items[i].P, items[i].maskA, items[i].maskB, v);
        for (int w = 0; w < 2; ++w)
          for (auto& x : v[w]) all[w].push_back({x.first, {x.second, (int)i}});
        mg.layouts.push_back(items[i].L);
      }
      for (int w = 0; w < 2; ++w) {
        std::stable_sort(all[w].begin(), all[w].end(), [](const auto& a, const auto& b) { return a.first > b.first; });
        std::vector<GTask> ht(all[w].size());
        std::vector<int> hi(all[w].size());
        for (size_t k = 0; k < all[w].size(); ++k) {
          ht[k] = all[w][k].second.first;
          hi[k] = all[w][k].second.second;
        }
        mg.n[w] = (int)ht.size();
        if (!ht.empty()) {
          QD_CUDA(cudaMalloc(&mg.d_task[w], ht.size() * sizeof(GTask)));
          QD_CUDA(cudaMemcpy(mg.d_task[w], ht.data(), ht.size() * sizeof(GTask), cudaMemcpyHostToDevice));
          QD_CUDA(cudaMalloc(&mg.d_tinst[w], hi.size() * sizeof(int)));
          QD_CUDA(cudaMemcpy(mg.d_tinst[w], hi.data(), hi.size() * sizeof(int), cudaMemcpyHostToDevice));
        }
      }
      QD_CUDA(cudaMalloc(&mg.d_inst, items.size() * sizeof(GInst)));
      QD_CUDA(cudaMallocHost(&mg.h_inst, items.size() * sizeof(GInst)));
      f = merged_gemm().emplace(key, mg).first;
    }
    m = &f->second;
  }
  for (size_t i = 0; i < items.size(); ++i) {
    const GemmItem& it = items[i];
    GInst& g = m->h_inst[i];
    g.probs = it.P->d_probs;
    g.segs = it.P->d_segs;
    for (int b = 0; b < NBUF; ++b) g.bufs.p[b] = it.bufs[b];
    g.hv0 = it.hv0;
    g.hv1 = it.hv1;
    g.maskA = it.maskA;
    g.maskB = it.maskB;
  }
  QD_CUDA(cudaMemcpyAsync(m->d_inst, m->h_inst, items.size() * sizeof(GInst), cudaMemcpyHostToDevice, st));
  Bufs none;
  for (int b = 0; b < NBUF; ++b) none.p[b] = nullptr;
  if (m->n[0] > 0) {
    k_grouped_gemm<<<m->n[0], GEMM_THREADS, GEMM_SMEM, st>>>(m->d_task[0], nullptr, nullptr, none, 0.0, 0.0, 0u, 0u,
                                                             m->d_tinst[0], m->d_inst);
    ++items[0].L->nlaunch;
  }
  if (m->n[1] > 0) {
    k_gemm_kshort<<<m->n[1], KS_THREADS, KS_SMEM, st>>>(m->d_task[1], nullptr, nullptr, none, 0.0, 0.0, 0u, 0u,
                                                        m->d_tinst[1], m->d_inst);
    ++items[0].L->nlaunch;
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// Drop every merged task list that involves layout L (called when L goes).
void drop_merged_gemm(const qd_layout* L) {
  std::lock_guard<std::mutex> lock(g_merged_gemm_mutex);
  auto& mm = merged_gemm();
  for (auto it = mm.begin(); it != mm.end();) {
    if (std::find(it->second.layouts.begin(), it->second.layouts.end(), L) != it->second.layouts.end()) {
      free_merged(it->second);
      it = mm.erase(it);
    } else {
      ++it;
    }
  }
}

}  // namespace qd
