// split_gemm.cu -- split-precision FP64 products on the tcgen05 tensor cores.
//
// The FP64 block contractions (src/commutators.f90 matrix_mult222 and
// construct_cc_ints, which call dgemm) can run in split form: each operand is
// written as a short sum of BF16 "slices" whose products are exact in the
// tensor cores' FP32 accumulators (an Ozaki-style error-free splitting:
// Ozaki, Ogita, Oishi, Rump, Numer. Algorithms 59 (2012) 95), and the slice
// products are summed in FP64.
//
// Splitting.  A row i of op(A) (a column of op(B)) gets the exponent e_i with
// max_k |x(i,k)| < 2^e_i; r = x / 2^e_i in (-1, 1) (exact), and
//   d_1 = rint(128 r), r <- 128 r - d_1;  d_s = rint(128 r), ...   (exact)
// so x = 2^e_i sum_{s=1..S} d_s 2^-7s + O(2^(e_i - 7S - 1)), |d_1| <= 128,
// |d_s| <= 64 for s >= 2: every digit is an integer that BF16 holds exactly.
//
// Products.  C(m,n) = 2^(e_m + f_n) sum_{s+t <= S+1} 2^-7(s+t) sum_k a_s b_t.
// The slice pairs of one diagonal d = s + t share a TMEM accumulator (FP32);
// its partial sums are integers whose magnitude over a K chunk of KC terms
// is at most KC * bound(d) (bound = 2^14 for d <= 3, 2^12 (d+1) above), so
// with KC * bound < 2^24 every FP32 sum is exact.  After each chunk the
// diagonals are read from TMEM (tcgen05.ld) and added in FP64 with their
// scale 2^(e_m + f_n - 7d).  The only rounding is the truncation of the
// slice series and the FP64 summation.
//
// Kernel.  One CTA (128 threads) per 128 x 64 output tile; per 64-wide K
// step the S slices of the A tile (128 x 64) and of the B tile (64 x 64) are
// staged in shared memory in the K-major 128-byte-swizzled layout (cp.async),
// one thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32, M=128,
// N=64, K=16) for every slice pair of the triangle and commits to an
// mbarrier; accumulators live in TMEM (S diagonals x 64 columns).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "dev_common.cuh"

namespace qd {

constexpr int SG_BM = 128, SG_BN = 64, SG_BK = 64, SG_THREADS = 128;
constexpr int SG_MAXS = 8;
constexpr size_t SG_ATILE = (size_t)SG_BM * SG_BK * 2;  // bytes per A slice tile
constexpr size_t SG_BTILE = (size_t)SG_BN * SG_BK * 2;  // bytes per B slice tile
constexpr long long SG_SPIN = 1LL << 22;                // mbarrier polls before giving up

// Operand role: the slices of one op(A) (rows i = m) or op(B) (rows i = n),
// K-major: slice s of row i at sl[((s * rpad) + i) * kpad + k]; ex[i] = e_i.
struct SRole {
  const __nv_bfloat16* sl;
  const int* ex;
  int rpad, kpad;
};
struct SSeg {
  int ra, rb;    // roles of op(A) and op(B)
  int K;
  double alpha;
};
struct SProb {
  int M, N, ldc, seg0, nseg, mode;  // mode: 0 SET, 1 ACC, 2 C = V + beta C
  i64 offC;
  double* C;
  double beta;
};
struct STask {
  int prob;
  short ti, tj;
};

// K chunk over which every diagonal's FP32 sums stay exact
__host__ __device__ inline int split_kchunk(int S) {
  long long worst = 1LL << 14;
  for (int d = 4; d <= S + 1; ++d) worst = std::max(worst, (long long)4096 * (d + 1));
  long long kc = ((1LL << 24) - 1) / worst;
  kc = (kc / SG_BK) * SG_BK;
  return (int)std::max<long long>(SG_BK, std::min<long long>(kc, 1024));
}

__host__ __device__ inline int split_tmem_cols(int S) {
  int need = S * SG_BN, c = 32;
  while (c < need) c <<= 1;
  return c;
}

// ---------------------------------------------------------------------------
// slicing: role (x(i,k) = X[i*si + k*sk]) -> exponents and S slices
// ---------------------------------------------------------------------------
// one warp per row i: max |x(i,k)| over k, then the slices of the row
__global__ void k_split_slice(const double* __restrict__ X, i64 si, i64 sk, int R, int K, int S, int rpad, int kpad,
                              __nv_bfloat16* __restrict__ sl, int* __restrict__ ex) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= rpad) return;
  const int i = warp;
  double mx = 0.0;
  if (i < R)
    for (int k = lane; k < K; k += 32) mx = fmax(mx, fabs(X[i * si + k * sk]));
  for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  const int e = mx > 0.0 ? ilogb(mx) + 1 : 0;
  if (lane == 0 && i < R) ex[i] = e;
  for (int k = lane; k < kpad; k += 32) {
    double r = (i < R && k < K) ? scalbn(X[i * si + k * sk], -e) : 0.0;
    for (int s = 0; s < S; ++s) {
      const double t = r * 128.0;
      const double d = rint(t);
      r = t - d;
      sl[((i64)s * rpad + i) * kpad + k] = __float2bfloat16_rn((float)d);
    }
  }
}

// ---------------------------------------------------------------------------
// tcgen05 helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// K-major, 128-byte swizzle, 8-row atoms 1024 bytes apart (SBO), LBO 16 bytes
__device__ __forceinline__ uint64_t umma_desc(unsigned saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)64 << 32) | ((uint64_t)1 << 46) |
         ((uint64_t)2 << 61);
}
// kind::f16: D f32 (bits 4-5 = 1), A bf16 (7-9 = 1), B bf16 (10-12 = 1),
// both K-major, N >> 3 at 17, M >> 4 at 24
constexpr uint32_t SG_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(SG_BN >> 3) << 17) |
                              ((uint32_t)(SG_BM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(unsigned dtmem, uint64_t ad, uint64_t bd, unsigned accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "l"(ad), "l"(bd), "r"(SG_IDESC), "r"(accum));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// wait for the phase with parity `ph`; false if it did not complete in time
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned ph) {
  for (long long it = 0; it < SG_SPIN; ++it) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(ph)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(unsigned taddr, float* v) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void cp16(unsigned saddr, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}

// stage rows [row0, row0+rows) x K [k0, k0+64) of slice s of role r into a
// swizzled tile: 16-byte chunk c of row i lands at i*128 + ((c ^ (i & 7)) * 16)
__device__ __forceinline__ void stage_tile(unsigned sbase, const SRole& ro, int s, int row0, int rows, int k0) {
  const __nv_bfloat16* g = ro.sl + ((i64)s * ro.rpad + row0) * ro.kpad + k0;
  for (int e = threadIdx.x; e < rows * 8; e += SG_THREADS) {
    const int i = e >> 3, c = e & 7;
    cp16(sbase + i * 128 + ((c ^ (i & 7)) << 4), g + (i64)i * ro.kpad + c * 8);
  }
}

// ---------------------------------------------------------------------------
// the grouped split GEMM
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(SG_THREADS, 1)
    k_split_gemm(const STask* __restrict__ tasks, const SProb* __restrict__ probs, const SSeg* __restrict__ segs,
                 const SRole* __restrict__ roles, int S, int* __restrict__ err) {
  extern __shared__ uint8_t smraw[];
  __shared__ uint64_t bar;
  __shared__ unsigned tslot;
  __shared__ int fx[SG_BN];
  __shared__ int fail;
  // 1024-byte aligned tiles: A slices then B slices
  const unsigned sraw = smem_u32(smraw);
  const unsigned sA = (sraw + 1023u) & ~1023u;
  const unsigned sB = sA + (unsigned)(S * SG_ATILE);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ncols = split_tmem_cols(S);

  const STask t = tasks[blockIdx.x];
  const SProb P = probs[t.prob];
  const int row0 = t.ti * SG_BM, col0 = t.tj * SG_BN;
  const int m = row0 + threadIdx.x;  // this thread's output row (TMEM lane)

  if (threadIdx.x == 0) {
    mbar_init(&bar);
    fail = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tbase = tslot;
  const int kc = split_kchunk(S);

  double acc[SG_BN];
#pragma unroll
  for (int j = 0; j < SG_BN; ++j) acc[j] = 0.0;
  unsigned phase = 0;

  for (int sg = 0; sg < P.nseg && !fail; ++sg) {
    const SSeg G = segs[P.seg0 + sg];
    const SRole RA = roles[G.ra], RB = roles[G.rb];
    if (threadIdx.x < SG_BN) fx[threadIdx.x] = (col0 + threadIdx.x < P.N) ? RB.ex[col0 + threadIdx.x] : 0;
    const int em = m < P.M ? RA.ex[m] : 0;
    const int ksteps = (G.K + SG_BK - 1) / SG_BK;
    for (int c0 = 0; c0 < ksteps && !fail; c0 += kc / SG_BK) {
      const int c1 = min(ksteps, c0 + kc / SG_BK);
      unsigned init = 0;  // diagonals written in this chunk
      for (int ks = c0; ks < c1; ++ks) {
        for (int s = 0; s < S; ++s) {
          stage_tile(sA + s * (unsigned)SG_ATILE, RA, s, row0, SG_BM, ks * SG_BK);
          stage_tile(sB + s * (unsigned)SG_BTILE, RB, s, col0, SG_BN, ks * SG_BK);
        }
        asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
          tc_fence_after();
#pragma unroll 1
          for (int k16 = 0; k16 < SG_BK / 16; ++k16)
            for (int s = 0; s < S; ++s)
              for (int u = 0; u + s < S; ++u) {  // slice pair (s+1, u+1), diagonal s+u+2
                const int d = s + u;
                const uint64_t ad = umma_desc(sA + s * (unsigned)SG_ATILE + k16 * 32);
                const uint64_t bd = umma_desc(sB + u * (unsigned)SG_BTILE + k16 * 32);
                umma_bf16(tbase + d * SG_BN, ad, bd, (init >> d) & 1u);
                init |= 1u << d;
              }
          umma_commit(&bar);
        }
        // the tiles are reused by the next step: wait for the MMAs
        if (!mbar_wait(&bar, phase)) {
          if (lane == 0) atomicExch(&fail, 1);
        }
        phase ^= 1u;
        __syncthreads();
        if (fail) break;
      }
      if (fail) break;
      tc_fence_after();
      // read the diagonals of this chunk and add them in FP64
      for (int d = 0; d < S; ++d) {
        const double rs = ldexp(G.alpha, em - 7 * (d + 2));
#pragma unroll
        for (int q = 0; q < SG_BN / 16; ++q) {
          float v[16];
          tmem_ld16(tbase + ((unsigned)(warp * 32) << 16) + d * SG_BN + q * 16, v);
#pragma unroll
          for (int j = 0; j < 16; ++j) acc[q * 16 + j] = fma((double)v[j], ldexp(rs, fx[q * 16 + j]), acc[q * 16 + j]);
        }
      }
      tc_fence_before();
      __syncthreads();
    }
    __syncthreads();  // fx is rewritten by the next segment
  }
  if (fail && threadIdx.x == 0) atomicExch(err, 1);
  // epilogue: thread = row m, columns col0.. (consecutive rows per column)
  if (!fail && m < P.M) {
    double* out = P.C + P.offC + m;
    const int nn = min(SG_BN, P.N - col0);
#pragma unroll
    for (int j = 0; j < SG_BN; ++j) {
      if (j >= nn) break;
      double* p = out + (i64)(col0 + j) * P.ldc;
      if (P.mode == 0)
        *p = acc[j];
      else if (P.mode == 1)
        *p += acc[j];
      else
        *p = acc[j] + (P.beta == 0.0 ? 0.0 : P.beta * *p);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(ncols) : "memory");
  }
}

size_t split_gemm_smem(int S) { return (size_t)S * (SG_ATILE + SG_BTILE) + 1024; }

}  // namespace qd

using namespace qd;

// ---------------------------------------------------------------------------
// C ABI: one split-precision product with dgemm's argument meaning
// ---------------------------------------------------------------------------
extern "C" int qd_gemm_split(int device, void* stream, char transa, char transb, int M, int N, int K, double alpha,
                             const double* A, int lda, const double* B, int ldb, double beta, double* C, int ldc,
                             int slices) {
  const bool ta = transa == 'T' || transa == 't', tb = transb == 'T' || transb == 't';
  if (!(ta || transa == 'N' || transa == 'n') || !(tb || transb == 'N' || transb == 'n') || M < 0 || N < 0 ||
      K < 0 || slices < 1 || slices > SG_MAXS || (M > 0 && N > 0 && (!C || ldc < M)) ||
      (M > 0 && K > 0 && (!A || lda < (ta ? K : M))) || (N > 0 && K > 0 && (!B || ldb < (tb ? N : K)))) {
    set_error("qd_gemm_split: bad argument");
    return QD_ERR_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("qd_gemm_split: no CUDA device");
    return QD_ERR_NODEVICE;
  }
  QD_CUDA(cudaSetDevice(device));
  cudaStream_t st = (cudaStream_t)stream;
  if (M == 0 || N == 0) return QD_OK;
  const int S = slices;
  const int mpad = (M + SG_BM - 1) / SG_BM * SG_BM, npad = (N + SG_BN - 1) / SG_BN * SG_BN;
  const int kpad = std::max(SG_BK, (K + SG_BK - 1) / SG_BK * SG_BK);
  const size_t bytesA = (size_t)S * mpad * kpad * 2, bytesB = (size_t)S * npad * kpad * 2;
  uint8_t* ws = nullptr;
  const size_t off_ex = bytesA + bytesB, off_err = off_ex + sizeof(int) * (mpad + npad);
  const size_t off_meta = (off_err + sizeof(int) + 255) & ~(size_t)255;
  const int ntask = (mpad / SG_BM) * (npad / SG_BN);
  const size_t bytes = off_meta + sizeof(SRole) * 2 + sizeof(SSeg) + sizeof(SProb) + sizeof(STask) * ntask + 64;
  QD_CUDA(cudaMallocAsync((void**)&ws, bytes, st));
  __nv_bfloat16* slA = (__nv_bfloat16*)ws;
  __nv_bfloat16* slB = (__nv_bfloat16*)(ws + bytesA);
  int* exA = (int*)(ws + off_ex);
  int* exB = exA + mpad;
  int* d_err = (int*)(ws + off_err);
  QD_CUDA(cudaMemsetAsync(exA, 0, sizeof(int) * (mpad + npad) + sizeof(int), st));
  // op(A)(m,k) = ta ? A[k + m lda] : A[m + k lda]; op(B)(k,n) = tb ? B[n + k ldb] : B[k + n ldb]
  const double* Ab = K > 0 ? A : C;
  const double* Bb = K > 0 ? B : C;
  k_split_slice<<<(mpad * 32 + 255) / 256, 256, 0, st>>>(Ab, ta ? lda : 1, ta ? 1 : lda, M, K, S, mpad, kpad, slA,
                                                        exA);
  k_split_slice<<<(npad * 32 + 255) / 256, 256, 0, st>>>(Bb, tb ? 1 : ldb, tb ? ldb : 1, N, K, S, npad, kpad, slB,
                                                        exB);
  // one problem, one segment, every tile
  uint8_t* hmeta = (uint8_t*)malloc(bytes - off_meta);
  SRole* hr = (SRole*)hmeta;
  hr[0] = SRole{slA, exA, mpad, kpad};
  hr[1] = SRole{slB, exB, npad, kpad};
  SSeg* hs = (SSeg*)(hr + 2);
  *hs = SSeg{0, 1, K, alpha};
  SProb* hp = (SProb*)(hs + 1);
  *hp = SProb{M, N, ldc, 0, K > 0 ? 1 : 0, 2, 0, C, beta};
  STask* ht = (STask*)(hp + 1);
  for (int i = 0, k = 0; i < mpad / SG_BM; ++i)
    for (int j = 0; j < npad / SG_BN; ++j, ++k) ht[k] = STask{0, (short)i, (short)j};
  uint8_t* dmeta = ws + off_meta;
  QD_CUDA(cudaMemcpyAsync(dmeta, hmeta, bytes - off_meta, cudaMemcpyHostToDevice, st));
  QD_CUDA(cudaStreamSynchronize(st));
  free(hmeta);
  const size_t smem = split_gemm_smem(S);
  QD_CUDA(cudaFuncSetAttribute(k_split_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const SRole* dr = (const SRole*)dmeta;
  const SSeg* ds = (const SSeg*)(dr + 2);
  const SProb* dp = (const SProb*)(ds + 1);
  const STask* dt = (const STask*)(dp + 1);
  k_split_gemm<<<ntask, SG_THREADS, smem, st>>>(dt, dp, ds, dr, S, d_err);
  QD_CUDA(cudaGetLastError());
  int herr = 0;
  QD_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  QD_CUDA(cudaStreamSynchronize(st));
  QD_CUDA(cudaFreeAsync(ws, st));
  if (herr) {
    set_error("qd_gemm_split: tensor-core wait timed out");
    return QD_ERR_CUDA;
  }
  return QD_OK;
}
